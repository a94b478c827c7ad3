// Instantiations of the point kernels for float inputs, precision mode 1.
#include "launch.hpp"
namespace psb {
cudaError_t launch_points_f1(const Args<float>& a, int st, int kc, int what, cudaStream_t s) {
    return dispatch_points_p<float, 1>(a, st, kc, what, s);
}
}  // namespace psb
