// Instantiations of the point kernels for double inputs, precision mode 1.
#include "launch.hpp"
namespace psb {
cudaError_t launch_points_d1(const Args<double>& a, int st, int kc, int what, cudaStream_t s) {
    return dispatch_points_p<double, 1>(a, st, kc, what, s);
}
}  // namespace psb
