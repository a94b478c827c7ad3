// Instantiations of the two-kernel point path: float inputs, PREC_FP64.
#include "launch.hpp"

namespace psb {
cudaError_t launch_split_f0(const Args<float>& a, int st, int kc, bool bodies, cudaStream_t s) {
    return dispatch_split_p<float, PREC_FP64>(a, st, kc, bodies, s);
}
}  // namespace psb
