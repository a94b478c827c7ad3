// Instantiations of the point kernels for double inputs, precision mode 0.
#include "launch.hpp"
namespace psb {
cudaError_t launch_points_d0(const Args<double>& a, int st, int kc, int what, cudaStream_t s) {
    return dispatch_points_p<double, 0>(a, st, kc, what, s);
}
}  // namespace psb
