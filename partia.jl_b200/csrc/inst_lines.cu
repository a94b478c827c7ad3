// Instantiations of the line kernels and the launch front ends.
#include "launch.hpp"
namespace psb {
cudaError_t launch_points_d0(const Args<double>&, int, int, int, cudaStream_t);
cudaError_t launch_points_d1(const Args<double>&, int, int, int, cudaStream_t);
cudaError_t launch_points_f0(const Args<float>&, int, int, int, cudaStream_t);
cudaError_t launch_points_f1(const Args<float>&, int, int, int, cudaStream_t);

template <> cudaError_t launch_points<double>(const Args<double>& a, int prec, int st, int kc, int what, cudaStream_t s) {
    return prec == PREC_FP64 ? launch_points_d0(a, st, kc, what, s) : launch_points_d1(a, st, kc, what, s);
}
template <> cudaError_t launch_points<float>(const Args<float>& a, int prec, int st, int kc, int what, cudaStream_t s) {
    return prec == PREC_FP64 ? launch_points_f0(a, st, kc, what, s) : launch_points_f1(a, st, kc, what, s);
}
template <> cudaError_t launch_lines<double>(const Args<double>& a, int prec, int st, int kc, int what, cudaStream_t s) {
    return prec == PREC_FP64 ? dispatch_lines_p<double, PREC_FP64>(a, st, kc, what, s)
                             : dispatch_lines_p<double, PREC_FP32C>(a, st, kc, what, s);
}
template <> cudaError_t launch_lines<float>(const Args<float>& a, int prec, int st, int kc, int what, cudaStream_t s) {
    return prec == PREC_FP64 ? dispatch_lines_p<float, PREC_FP64>(a, st, kc, what, s)
                             : dispatch_lines_p<float, PREC_FP32C>(a, st, kc, what, s);
}
}  // namespace psb
