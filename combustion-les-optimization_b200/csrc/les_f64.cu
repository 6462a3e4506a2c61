// les_f64.cu -- plain FP64 form of the solver step: the stage, boundary and diagnostic
// kernels in double precision.
//
// Built with -fmad=false: every multiply and add is rounded separately, as in the
// reference (built for baseline x86-64, which has no FMA), so that apart from the libm
// transcendentals and the order of the <rho_f> sum the kernels perform the reference's
// floating-point operations one for one.
#include "les_launch.cuh"

namespace les {

cudaError_t step_f64(DevCtx& c, double dt, int t_loop, bool device_mode) {
    return step_impl<double>(c, dt, t_loop, device_mode);
}
cudaError_t rhs_only_f64(DevCtx& c, int t_loop) { return rhs_only_impl<double>(c, t_loop); }
cudaError_t batch_head_f64(DevCtx& c) { return batch_head<double>(c); }
cudaError_t batch_tail_f64(DevCtx& c) { return batch_tail<double>(c); }
cudaError_t batch_stages_f64(DevCtx& c0, const MemberTab* mt, int nmem, cudaStream_t st) {
    return batch_stages<double>(c0, mt, nmem, st);
}
cudaError_t umax_f64(DevCtx& c) { return umax_impl<double>(c); }
cudaError_t monitor_f64(DevCtx& c) { return monitor_impl<double>(c); }
cudaError_t probe_f64(DevCtx& c, int n, int kline) { return probe_impl<double>(c, n, kline); }
cudaError_t check_f64(DevCtx& c, int field) { return check_impl<double>(c, field); }

cudaError_t prepare_tma_f64() { return prepare_scalar_tma<double, double>(); }

}  // namespace les
