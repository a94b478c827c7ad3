// Instantiations of the two-kernel point path: double inputs, PREC_FP64.
#include "launch.hpp"

namespace psb {
cudaError_t launch_split_d0(const Args<double>& a, int st, int kc, bool bodies, cudaStream_t s) {
    return dispatch_split_p<double, PREC_FP64>(a, st, kc, bodies, s);
}
}  // namespace psb
