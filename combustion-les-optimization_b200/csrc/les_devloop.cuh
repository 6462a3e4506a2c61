// les_devloop.cuh -- the host side of one time step, moved onto the GPU so that steps can
// be queued (and graph-replayed) without a host round trip:
//
//   * dt from the device maxima (les_combustion_solver.c:4399-4411);
//   * update_vortices (:900-939): advection and recycling, 6 rand() draws per recycled
//     vortex in vortex order;
//   * the inflow white noise of apply_boundary_conditions (:2990-2992): 3 draws per inlet
//     cell in (j, k) order, after the vortex draws.
//
// glibc's rand() is x[n] = x[n-31] + x[n-3] (mod 2^32), returned as x[n] >> 1.  The
// recurrence is linear, so x[n+m] = sum_j J[m][j] * w[j] (mod 2^32) for the current window
// w[j] = x[n-31+j]; the coefficient rows J[m] are integer tables computed once on the host.
// Every draw of a step is then an independent 31-term dot product, and the window after
// D draws is rows D-31..D-1.  The draws are bit-identical to calling rand() serially.
//
// Compiled only into the FP64 unit (no FMA contraction): vortex and noise arithmetic must
// match the host C code operation for operation.
#pragma once

#include "les_common.cuh"

namespace les {

__device__ __forceinline__ unsigned int jump_draw(const unsigned int* __restrict__ J, const unsigned int* w, int m) {
    const unsigned int* row = J + (size_t)m * 31;
    unsigned int acc = 0u;
#pragma unroll
    for (int j = 0; j < 31; j++) acc += row[j] * w[j];
    return acc;
}

__device__ __forceinline__ double draw01(unsigned int x) { return (double)(int)(x >> 1) / (double)2147483647; }

// One block of LOOP_THREADS threads.
constexpr int LOOP_THREADS = 1024;

__global__ void __launch_bounds__(LOOP_THREADS) k_loop_pre(const Consts* __restrict__ C, Scalars* __restrict__ Sc,
                                                           LoopState* __restrict__ L, const unsigned int* __restrict__ J,
                                                           int jrows, double* __restrict__ vort, int nv,
                                                           double* __restrict__ noise, int n_inlet, double lx_vort,
                                                           double ly, double lz, double u_in, double ti, double ell,
                                                           double courant, double courant_d, double dx) {
    __shared__ unsigned int w[31];
    __shared__ int wsum[LOOP_THREADS / 32];
    __shared__ int s_total;
    __shared__ double s_dt;
    const int tid = threadIdx.x;
    if (tid < 31) w[tid] = L->win[tid];
    if (tid == 0) {
        // dt (:4399-4411): |u|max falls back to the inlet velocity below 1e-10 (:1484)
        double um = Sc->umax > 1e-10 ? Sc->umax : u_in;
        double dt_conv = courant * dx / (um + 1e-10);
        double dt_nu = courant_d * (dx * dx) / (Sc->numax + 1e-10);
        double dt_al = courant_d * (dx * dx) / (Sc->alphamax + 1e-10);
        double dt = fmin(dt_conv, fmin(dt_nu, dt_al));
        s_dt = dt;
        Sc->dt = dt;
        Sc->umax_used = um;
    }
    __syncthreads();
    const double dt = s_dt;
    const double half_box = lx_vort / 2.0;
    const double u_rms = u_in * ti;
    const double min_r = ell * 0.5, max_r = ell * 1.5;
    // pass 1: advect, flag recycled vortices, exclusive scan of the flags in vortex order
    int base = 0;
    for (int c0 = 0; c0 < nv; c0 += LOOP_THREADS) {
        const int v = c0 + tid;
        double xn = 0.0;
        int rec = 0;
        if (v < nv) {
            xn = vort[7 * (size_t)v] + u_in * dt;
            rec = xn > half_box ? 1 : 0;
        }
        // block-wide exclusive scan of rec
        const int lane = tid & 31, wid = tid >> 5;
        unsigned int bal = __ballot_sync(0xffffffffu, rec);
        int pre = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        if (tid < 32) {
            int x = (tid < LOOP_THREADS / 32) ? wsum[tid] : 0;
            int inc = x;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (tid < LOOP_THREADS / 32) wsum[tid] = inc - x;   // exclusive warp offsets
            if (tid == 31) s_total = inc;
        }
        __syncthreads();
        const int rank = base + wsum[wid] + pre;
        if (v < nv) {
            double* V = vort + 7 * (size_t)v;
            if (rec) {
                V[0] = xn - lx_vort;
                const int m = 6 * rank;
                double ry = draw01(jump_draw(J, w, m + 0));
                double rz = draw01(jump_draw(J, w, m + 1));
                V[1] = ry * ly;
                V[2] = rz * lz;
                double ru = draw01(jump_draw(J, w, m + 2));
                double rv = draw01(jump_draw(J, w, m + 3));
                double rw = draw01(jump_draw(J, w, m + 4));
                V[4] = (ru * 2.0 - 1.0) * u_rms;
                V[5] = (rv * 2.0 - 1.0) * u_rms;
                V[6] = (rw * 2.0 - 1.0) * u_rms;
                double rr = draw01(jump_draw(J, w, m + 5));
                V[3] = min_r + (max_r - min_r) * rr;
            } else {
                V[0] = xn;
            }
        }
        base += s_total;
        __syncthreads();
    }
    const int n_rec = base;
    // inflow white noise: r = (rand()/RAND_MAX)*2 - 1, three per inlet cell
    const int m0 = 6 * n_rec;
    for (int q = tid; q < 3 * n_inlet; q += LOOP_THREADS) {
        unsigned int x = jump_draw(J, w, m0 + q);
        noise[q] = ((double)(int)(x >> 1) / 2147483647) * 2.0 - 1.0;
    }
    // advance the window by D draws: w'[j] = x[n + D - 31 + j]
    const int D = m0 + 3 * n_inlet;
    __shared__ unsigned int wn[31];
    if (tid < 31) {
        const int t = D - 31 + tid;
        wn[tid] = (t < 0) ? w[31 + t] : jump_draw(J, w, t);
    }
    __syncthreads();
    if (tid < 31) L->win[tid] = wn[tid];
    if (tid == 0) {
        L->n_rec = n_rec;
        L->draws = D;
        L->total_draws += (unsigned long long)D;
        if (D > jrows) Sc->nonfinite |= 2;   // table too short: flagged, checked by the host
    }
}

}  // namespace les
