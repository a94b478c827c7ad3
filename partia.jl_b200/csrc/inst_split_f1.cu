// Instantiations of the two-kernel point path: float inputs, PREC_FP32C.
#include "launch.hpp"

namespace psb {
cudaError_t launch_split_f1(const Args<float>& a, int st, int kc, bool bodies, cudaStream_t s) {
    return dispatch_split_p<float, PREC_FP32C>(a, st, kc, bodies, s);
}
}  // namespace psb
