// Instantiations of the point kernels for float inputs, precision mode 0.
#include "launch.hpp"
namespace psb {
cudaError_t launch_points_f0(const Args<float>& a, int st, int kc, int what, cudaStream_t s) {
    return dispatch_points_p<float, 0>(a, st, kc, what, s);
}
}  // namespace psb
