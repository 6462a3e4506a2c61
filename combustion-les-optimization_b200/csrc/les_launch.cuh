// les_launch.cuh -- stream-ordered launch sequence of one solver step, templated on the
// field type.  Included once per precision translation unit.
#pragma once

#include "les_ctx.h"
#include "les_kernels.cuh"
#include "les_tma.cuh"

namespace les {

// The state Phi_n is FP64 in both forms; R is the form's type of every other field.
using RS = double;

template <typename R>
static F11<R> f11(void* const* p) {
    F11<R> f;
    for (int q = 0; q < NSTATE; q++) f.p[q] = (R*)p[q];
    return f;
}

template <typename R>
static PropBuf<R> props(const DevCtx& c) {
    PropBuf<R> P;
    P.mu_mix = (R*)c.mu_mix;
    P.nu = (R*)c.nu;
    for (int s = 0; s < NSP; s++) P.D[s] = (R*)c.D[s];
    P.aT = (R*)c.aT;
    P.nu_t = (R*)c.nu_t;
    P.S_mag = (R*)c.S_mag;
    P.ST = (R*)c.ST;
    P.mu_eff = (R*)c.mu_eff;
    P.dbg_cp = c.debug ? (R*)c.dbg_cp : nullptr;
    P.dbg_lam = c.debug ? (R*)c.dbg_lam : nullptr;
    P.dbg_alpha = c.debug ? (R*)c.dbg_alpha : nullptr;
    P.grad_g = (R*)c.grad_g;
    return P;
}

static inline dim3 cell_block(const DevCtx& c, int cls) {
    const Shape t = kShapes[c.shape[cls]];
    return dim3((unsigned)t.bx, (unsigned)t.by, (unsigned)t.bz);
}
static inline dim3 cell_grid(const DevCtx& c, int cls) {
    const Shape t = kShapes[c.shape[cls]];
    return dim3((unsigned)((c.nz + t.bx - 1) / t.bx), (unsigned)((c.ny + t.by - 1) / t.by),
                (unsigned)((c.nx + t.bz - 1) / t.bz));
}

// The strain, flow and scalar passes with the kernel instance of their tile's block size.
template <typename R, bool BATCH>
static inline void launch_strain(dim3 g, dim3 b, cudaStream_t st, const Consts& hC, const uint8_t* attr,
                                 const F11<R>& F, const PropBuf<R>& P, const Batch& B) {
    if (b.x * b.y * b.z == 512) k_strain<R, BATCH, 512><<<g, b, 0, st>>>(hC, attr, F, P, B);
    else k_strain<R, BATCH><<<g, b, 0, st>>>(hC, attr, F, P, B);
}
template <typename R, bool BATCH>
static inline void launch_flow(dim3 g, dim3 b, cudaStream_t st, const Consts& hC, const uint8_t* attr,
                               const F11<R>& F, const PropBuf<R>& P, const KFlow<R>& kf, const KDbg<R>& kd,
                               Scalars* dS, const Batch& B) {
    if (b.x * b.y * b.z == 512) k_rhs_flow<R, BATCH, 512><<<g, b, 0, st>>>(hC, attr, F, P, kf, kd, dS, B);
    else k_rhs_flow<R, BATCH><<<g, b, 0, st>>>(hC, attr, F, P, kf, kd, dS, B);
}
template <typename R, bool BATCH>
static inline void launch_scalar(dim3 g, dim3 b, cudaStream_t st, const Consts& hC, const uint8_t* attr,
                                 const F11<R>& F, const PropBuf<R>& P, const F11<RS>& S, const F11<R>& St,
                                 const AccBuf<R>& acc, const KFlow<R>& kf, const KDbg<R>& kd, Scalars* dS,
                                 int stage, const Batch& B) {
    if (b.x * b.y * b.z == 512)
        k_rhs_scalar<R, RS, BATCH, 512><<<g, b, 0, st>>>(hC, attr, F, P, S, St, acc, kf, kd, dS, stage, B);
    else
        k_rhs_scalar<R, RS, BATCH><<<g, b, 0, st>>>(hC, attr, F, P, S, St, acc, kf, kd, dS, stage, B);
}

// Every launch that writes per-block partials checks the buffer first: `per_block` values
// per block for `blocks` blocks must fit in c.part.
static inline bool part_fits(const DevCtx& c, size_t blocks, size_t per_block) {
    return blocks * per_block <= c.part_len;
}
static inline size_t cell_blocks(const DevCtx& c, int cls) {
    dim3 g = cell_grid(c, cls);
    return (size_t)g.x * g.y * g.z;
}

// The end of a step after the four RK stages: boundary conditions, EOS, time averages and,
// in the device loop, the step's history and counters.
template <typename R>
void step_tail(DevCtx& c, cudaStream_t st, bool device_mode) {
    F11<RS> S = f11<RS>(c.S);
    PropBuf<R> P = props<R>(c);
    const dim3 gE = cell_grid(c, SH_EOS), bE = cell_block(c, SH_EOS);
    {
        const int tpb = 128;
        k_bc_iface<RS, R><<<dim3((c.nz + tpb - 1) / tpb, c.ny), tpb, 0, st>>>(c.hC, c.attr, S, c.plane, c.noise,
                                                                                c.inlet_pos);
        if (c.nx > 2) {
            k_bc_jface<RS, R><<<dim3((c.nz + tpb - 1) / tpb, c.nx - 2), tpb, 0, st>>>(c.hC, c.attr, S);
            k_bc_kface<RS, R><<<dim3((c.ny + tpb - 1) / tpb, c.nx - 2), tpb, 0, st>>>(c.hC, c.attr, S);
        }
        k_bc_eos<RS, R><<<gE, bE, 0, st>>>(c.hC, c.attr, S, c.part, c.dS);
    }
    if (c.avg) {
        AvgBuf A;
        for (int q = 0; q < NAVG; q++) A.p[q] = c.avg + (size_t)q * c.n;
        k_time_avg<RS, R><<<MON_BLOCKS, NT, 0, st>>>(S, A, c.dS, c.n, c.avg_start);
    }
    if (device_mode) {
        const int tpb = 64;
        k_loop_post<RS, R><<<dim3((c.ny + tpb - 1) / tpb, c.loop_nst > 0 ? c.loop_nst : 1), tpb, 0, st>>>(
            c.hC, S, P, c.dS, c.loop_st, c.loop_nst, c.loop_kline, c.loop_cap, c.hist_probe, c.hist_dt, c.hist_umax);
        k_loop_monitor<RS, R><<<MON_BLOCKS, NT, 0, st>>>(c.hC, S, c.part, c.dS, c.n, c.loop_cap, c.hist_mon);
        k_loop_tick<<<1, 1, 0, st>>>(c.dS);
    }
}

// One time step.  Host-driven (device_mode false): dt and t_loop come from the caller and
// the inflow from lesgpu_set_inflow.  Device loop (true): dt, the vortex update and the
// inflow noise are computed on the GPU first, and the step's history is recorded at the
// end; every launch then reads only device memory, so the sequence can be graph-captured.
template <typename R>
cudaError_t step_impl(DevCtx& c, double dt, int t_loop, bool device_mode) {
    cudaStream_t st = c.stream;
    if (!part_fits(c, cell_blocks(c, SH_FILTER), 3) || !part_fits(c, cell_blocks(c, SH_EOS), 1) ||
        !part_fits(c, MON_BLOCKS, 6))
        return cudaErrorInvalidValue;
    const dim3 gA = cell_grid(c, SH_FILTER), bA = cell_block(c, SH_FILTER);
    const dim3 gB = cell_grid(c, SH_STRAIN), bB = cell_block(c, SH_STRAIN);
    const dim3 gC = cell_grid(c, SH_FLOW), bC = cell_block(c, SH_FLOW);
    const dim3 gD = cell_grid(c, SH_SCALAR), bD = cell_block(c, SH_SCALAR);
    F11<RS> S = f11<RS>(c.S);
    F11<R> St = f11<R>(c.St), F = f11<R>(c.F);
    PropBuf<R> P = props<R>(c);
    AccBuf<R> acc;
    for (int q = 0; q < NACC; q++) acc.p[q] = (R*)c.acc[q];
    KDbg<R> kd;
    for (int q = 0; q < NACC; q++) kd.p[q] = c.debug ? (R*)c.kd[q] : nullptr;
    KDbg<R> knone;
    for (int q = 0; q < NACC; q++) knone.p[q] = nullptr;
    KFlow<R> kf;
    for (int q = 0; q < 4; q++) kf.p[q] = (R*)c.kflow[q];

    int tm = tmark_begin(c, 0);
    if (device_mode) loop_pre(c);
    else k_set_step<<<1, 1, 0, st>>>(c.dS, dt, t_loop);
    // SEM inflow plane (:943-1075).  Only the boundary conditions read it, so it runs on a
    // side stream beside the four RK stages (joined before the BC); with kernel timing on
    // it runs in line so that its events bracket it alone.
    const bool overlap = !c.timing && c.side && c.n_inlet > 0;
    if (overlap) {
        cudaEventRecord(c.ev_fork, st);
        cudaStreamWaitEvent(c.side, c.ev_fork, 0);
        sem_inflow(c, c.side);
        cudaEventRecord(c.ev_join, c.side);
    } else {
        sem_inflow(c, st);
    }
    tmark_end(c, tm);
    // four RK4 stages (:4428-4544)
    for (int s = 0; s < 4; s++) {
        tm = tmark_begin(c, 1);
        if (s == 0) k_filter_props<R, RS><<<gA, bA, 0, st>>>(c.hC, c.attr, S, F, P, c.part, c.dS, 0, Batch{});
        else k_filter_props<R, R><<<gA, bA, 0, st>>>(c.hC, c.attr, St, F, P, c.part, c.dS, s == 3 ? 1 : 0, Batch{});
        tmark_end(c, tm);
        tm = tmark_begin(c, 2);
        launch_strain<R, false>(gB, bB, st, c.hC, c.attr, F, P, Batch{});
        tmark_end(c, tm);
        // the k-arrays of the first stage are kept for inspection when requested
        const KDbg<R>& kds = (s == 0) ? kd : knone;
        tm = tmark_begin(c, 3);
        launch_flow<R, false>(gC, bC, st, c.hC, c.attr, F, P, kf, kds, c.dS, Batch{});
        tmark_end(c, tm);
        tm = tmark_begin(c, 5);
        if (c.scalar_tma && c.tma_ok) launch_scalar_tma<R, RS>(c, st, F, P, S, St, acc, kf, kds, s);
        else launch_scalar<R, false>(gD, bD, st, c.hC, c.attr, F, P, S, St, acc, kf, kds, c.dS, s, Batch{});
        tmark_end(c, tm);
    }
    // apply_boundary_conditions (:2967-3161)
    if (overlap) cudaStreamWaitEvent(st, c.ev_join, 0);
    tm = tmark_begin(c, 4);
    step_tail<R>(c, st, device_mode);
    tmark_end(c, tm);
    tmark_flush(c);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ batched members
// Several members of one grid shape and precision, stepped together: each member's step head
// (dt, vortex and noise draws, SEM plane) and tail (boundary conditions, history) on its own
// stream as above, and the four RK stages of all of them in one launch per pass, whose grid is
// the first member's grid repeated along z once per member.  Every block reads its member's
// arena offset, attribute map, reductions and model constants from the member table (les_common.cuh,
// MemberTab); the tiles are the first member's.

template <typename R>
cudaError_t batch_head(DevCtx& c) {
    loop_pre(c);
    sem_inflow(c, c.stream);
    return cudaGetLastError();
}

template <typename R>
cudaError_t batch_tail(DevCtx& c) {
    step_tail<R>(c, c.stream, true);
    return cudaGetLastError();
}

template <typename R>
cudaError_t batch_stages(DevCtx& c0, const MemberTab* mt, int nmem, cudaStream_t st) {
    if (nmem < 1 || !part_fits(c0, cell_blocks(c0, SH_FILTER), 3)) return cudaErrorInvalidValue;
    auto grid = [&](int cls, Batch& b) {
        dim3 g = cell_grid(c0, cls);
        b.mt = mt;
        b.gz = (int)g.z;
        g.z *= (unsigned)nmem;
        return g;
    };
    Batch BA, BB, BC, BD;
    const dim3 gA = grid(SH_FILTER, BA), bA = cell_block(c0, SH_FILTER);
    const dim3 gB = grid(SH_STRAIN, BB), bB = cell_block(c0, SH_STRAIN);
    const dim3 gC = grid(SH_FLOW, BC), bC = cell_block(c0, SH_FLOW);
    const dim3 gD = grid(SH_SCALAR, BD), bD = cell_block(c0, SH_SCALAR);
    if (gA.z > 65535u || gB.z > 65535u || gC.z > 65535u || gD.z > 65535u) return cudaErrorInvalidConfiguration;
    F11<RS> S = f11<RS>(c0.S);
    F11<R> St = f11<R>(c0.St), F = f11<R>(c0.F);
    PropBuf<R> P = props<R>(c0);
    AccBuf<R> acc;
    for (int q = 0; q < NACC; q++) acc.p[q] = (R*)c0.acc[q];
    KDbg<R> knone;
    for (int q = 0; q < NACC; q++) knone.p[q] = nullptr;
    KFlow<R> kf;
    for (int q = 0; q < 4; q++) kf.p[q] = (R*)c0.kflow[q];
    for (int s = 0; s < 4; s++) {
        if (s == 0) k_filter_props<R, RS, true><<<gA, bA, 0, st>>>(c0.hC, c0.attr, S, F, P, c0.part, c0.dS, 0, BA);
        else k_filter_props<R, R, true><<<gA, bA, 0, st>>>(c0.hC, c0.attr, St, F, P, c0.part, c0.dS, s == 3 ? 1 : 0, BA);
        launch_strain<R, true>(gB, bB, st, c0.hC, c0.attr, F, P, BB);
        launch_flow<R, true>(gC, bC, st, c0.hC, c0.attr, F, P, kf, knone, c0.dS, BC);
        launch_scalar<R, true>(gD, bD, st, c0.hC, c0.attr, F, P, S, St, acc, kf, knone, c0.dS, s, BD);
    }
    return cudaGetLastError();
}

// Stage-1 right-hand side at the current state with the inspection buffers filled (when
// debug buffers exist); the state itself is not advanced (dt = 0 leaves the stage state
// equal to Phi_n).  The four kernels are bracketed by the kernel-timing marks, which the
// tile autotuner reads.
template <typename R>
cudaError_t rhs_only_impl(DevCtx& c, int t_loop) {
    cudaStream_t st = c.stream;
    if (!part_fits(c, cell_blocks(c, SH_FILTER), 3)) return cudaErrorInvalidValue;
    F11<RS> S = f11<RS>(c.S);
    F11<R> St = f11<R>(c.St), F = f11<R>(c.F);
    PropBuf<R> P = props<R>(c);
    AccBuf<R> acc;
    for (int q = 0; q < NACC; q++) acc.p[q] = (R*)c.acc[q];
    KDbg<R> kd;
    for (int q = 0; q < NACC; q++) kd.p[q] = (R*)c.kd[q];
    KFlow<R> kf;
    for (int q = 0; q < 4; q++) kf.p[q] = (R*)c.kflow[q];
    k_set_step<<<1, 1, 0, st>>>(c.dS, 0.0, t_loop);
    int tm = tmark_begin(c, 1);
    k_filter_props<R, RS><<<cell_grid(c, SH_FILTER), cell_block(c, SH_FILTER), 0, st>>>(c.hC, c.attr, S, F, P,
                                                                                       c.part, c.dS, 1, Batch{});
    tmark_end(c, tm);
    tm = tmark_begin(c, 2);
    launch_strain<R, false>(cell_grid(c, SH_STRAIN), cell_block(c, SH_STRAIN), st, c.hC, c.attr, F, P, Batch{});
    tmark_end(c, tm);
    tm = tmark_begin(c, 3);
    launch_flow<R, false>(cell_grid(c, SH_FLOW), cell_block(c, SH_FLOW), st, c.hC, c.attr, F, P, kf, kd, c.dS,
                          Batch{});
    tmark_end(c, tm);
    tm = tmark_begin(c, 5);
    if (c.scalar_tma && c.tma_ok)
        launch_scalar_tma<R, RS>(c, st, F, P, S, St, acc, kf, kd, 0);
    else
        launch_scalar<R, false>(cell_grid(c, SH_SCALAR), cell_block(c, SH_SCALAR), st, c.hC, c.attr, F, P, S, St,
                                acc, kf, kd, c.dS, 0, Batch{});
    tmark_end(c, tm);
    tmark_flush(c);
    return cudaGetLastError();
}

template <typename R>
cudaError_t umax_impl(DevCtx& c) {
    if (!part_fits(c, cell_blocks(c, SH_EOS), 1)) return cudaErrorInvalidValue;
    k_umax<RS, R><<<cell_grid(c, SH_EOS), cell_block(c, SH_EOS), 0, c.stream>>>(c.hC, c.attr, f11<RS>(c.S), c.part,
                                                                               c.dS);
    return cudaGetLastError();
}

template <typename R>
cudaError_t monitor_impl(DevCtx& c) {
    const int nb = MON_BLOCKS;
    if (!part_fits(c, nb, 6)) return cudaErrorInvalidValue;
    k_monitor<RS, R><<<nb, NT, 0, c.stream>>>(c.hC, f11<RS>(c.S), c.part, c.dS, c.n);
    return cudaGetLastError();
}

template <typename R>
cudaError_t probe_impl(DevCtx& c, int n, int kline) {
    const int tpb = 64;
    k_probe<RS, R><<<dim3((c.ny + tpb - 1) / tpb, n), tpb, 0, c.stream>>>(c.hC, f11<RS>(c.S), props<R>(c), c.probe_st,
                                                                          n, kline, c.probe_out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t check_impl(DevCtx& c, int field) {
    cudaMemsetAsync(c.flag, 0, sizeof(int), c.stream);
    if (field < NSTATE) k_check_finite<RS, R><<<592, 256, 0, c.stream>>>((const RS*)c.S[field], c.n, c.flag);
    else k_check_finite<R, R><<<592, 256, 0, c.stream>>>((const R*)c.nu_t, c.n, c.flag);
    return cudaGetLastError();
}

}  // namespace les
