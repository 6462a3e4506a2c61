// les_f32.cu -- precision form of the solver step: fields stored and advanced in FP32
// (advection, SGS, sources, properties); the stage <rho_f>, the dt maxima, the monitor
// sums and the SEM inflow plane are accumulated in FP64.  Built with FMA contraction.
#include "les_launch.cuh"

namespace les {

cudaError_t step_f32(DevCtx& c, double dt, int t_loop, bool device_mode) {
    return step_impl<float>(c, dt, t_loop, device_mode);
}
cudaError_t rhs_only_f32(DevCtx& c, int t_loop) { return rhs_only_impl<float>(c, t_loop); }
cudaError_t batch_head_f32(DevCtx& c) { return batch_head<float>(c); }
cudaError_t batch_tail_f32(DevCtx& c) { return batch_tail<float>(c); }
cudaError_t batch_stages_f32(DevCtx& c0, const MemberTab* mt, int nmem, cudaStream_t st) {
    return batch_stages<float>(c0, mt, nmem, st);
}
cudaError_t umax_f32(DevCtx& c) { return umax_impl<float>(c); }
cudaError_t monitor_f32(DevCtx& c) { return monitor_impl<float>(c); }
cudaError_t probe_f32(DevCtx& c, int n, int kline) { return probe_impl<float>(c, n, kline); }
cudaError_t check_f32(DevCtx& c, int field) { return check_impl<float>(c, field); }

cudaError_t prepare_tma_f32() { return prepare_scalar_tma<float, double>(); }

}  // namespace les
