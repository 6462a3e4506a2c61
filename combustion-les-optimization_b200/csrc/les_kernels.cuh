// les_kernels.cuh -- solver-step kernels, templated on the field type R (double for the
// plain form, float for the precision form).  Global sums and maxima are always
// accumulated in double.
//
// One RK4 stage is four passes over the grid:
//   A  k_filter_props : 7-point box filter of the 11 stage fields (apply_box_filter,
//                       les_combustion_solver.c:1307-1470) and the cell-local mixture
//                       properties (update_nu_mix :1489, update_Dk :1684, update_Cp_mix
//                       :1762, update_lambda_mix_alpha :1798); partial sums for <rho_f>.
//   B  k_strain       : resolved strain, G-dependent Smagorinsky nu_t (calculate_nu_t
//                       :1569), SSR-SGS flame speed (:1913) and mu_eff = mu + rho_f nu_t.
//   C1 k_rhs_flow     : momentum and G right-hand sides (calculate_RHS :2552-2825).
//   C2 k_rhs_scalar   : species and temperature right-hand sides (:2837-2962) fused with
//                       the RK4 stage update (:4432-4455) or the final combine (:4517-4544).
// After the fourth stage the boundary kernels replay apply_boundary_conditions
// (:2967-3161) in the reference's face order.
//
// Every kernel takes the constant table by value (__grid_constant__): divisors, their
// reciprocals and the species data are read from the constant bank.  Divisions by
// constants use cdv() (correctly rounded, see les_common.cuh); divisions by per-cell
// values are IEEE divisions.
#pragma once

#include <type_traits>

#include "les_common.cuh"

namespace les {

template <typename R>
struct F11 {                 // u v w T G rho Y0..Y4
    R* p[NSTATE];
};
template <typename R>
struct PropBuf {
    R* mu_mix;
    R* nu;
    R* D[NSP];
    R* aT;                   // lambda / (rho_f Cp), or 0 when the reference skips the term
    R* nu_t;
    R* S_mag;
    R* ST;
    R* mu_eff;
    R* dbg_cp;               // optional (nullptr): Cp, lambda, alpha for inspection
    R* dbg_lam;
    R* dbg_alpha;
    R* grad_g;               // optional (nullptr): |grad G| of the last RHS evaluation
};
template <typename R>
struct AccBuf {              // RK4 running sum of k: rhou rhov rhow T G Y0..Y4
    R* p[NACC];
};
template <typename R>
struct KDbg {                // optional (nullptr): the stage's k-arrays for inspection
    R* p[NACC];
};
template <typename R>
struct KFlow {               // momentum and G right-hand sides handed from C1 to C2
    R* p[4];                 // k_rhou k_rhov k_rhow k_G
};

#define LES_KERNEL_CONSTS const __grid_constant__ Consts C

// A member's fields in a batched launch: every per-cell field lives in the member's arena at
// the same offset as in the first member's, so its pointers are the first member's shifted by
// the arenas' distance.  Optional buffers outside the arena (inspection, |grad G|) are off in
// batched launches.
template <typename T>
__device__ __forceinline__ void shift_all(T& s, long long d) {
#pragma unroll
    for (int q = 0; q < (int)(sizeof(s.p) / sizeof(s.p[0])); q++) s.p[q] = shifted(s.p[q], d);
}
template <typename R>
__device__ __forceinline__ void shift_props(PropBuf<R>& P, long long d) {
    P.mu_mix = shifted(P.mu_mix, d);
    P.nu = shifted(P.nu, d);
#pragma unroll
    for (int s = 0; s < NSP; s++) P.D[s] = shifted(P.D[s], d);
    P.aT = shifted(P.aT, d);
    P.nu_t = shifted(P.nu_t, d);
    P.S_mag = shifted(P.S_mag, d);
    P.ST = shifted(P.ST, d);
    P.mu_eff = shifted(P.mu_eff, d);
    P.dbg_cp = P.dbg_lam = P.dbg_alpha = nullptr;
    P.grad_g = nullptr;
}

// Minimum resident blocks per SM requested from the register allocator (filter / flow /
// scalar).  These kernels are latency-bound; swept on B200 at 256x128x128: FP64 5/4/4 (the
// scalar pass at 3 blocks 3.41 ms, at 4 3.17 ms; the filter at 4 3.14 ms, at 5 3.02 ms; the
// flow pass at 5 slower), FP32 8/8/6/6 for filter/strain/flow/scalar (the scalar pass at 4
// blocks 2.01 ms, at 5 1.84 ms, at 6 1.76 ms; the flow pass at 8 0.616 ms, at 7 0.616, at 6
// 0.597).
#ifndef LES_MINB_FILTER
#define LES_MINB_FILTER 5
#endif
#ifndef LES_MINB_STRAIN
#define LES_MINB_STRAIN 3
#endif
#ifndef LES_MINB_FLOW
#define LES_MINB_FLOW 4
#endif
#ifndef LES_MINB_SCALAR
#define LES_MINB_SCALAR 4
#endif
#ifndef LES_MINB_FILTER_F32
#define LES_MINB_FILTER_F32 8
#endif
#ifndef LES_MINB_STRAIN_F32
#define LES_MINB_STRAIN_F32 8
#endif
#ifndef LES_MINB_FLOW_F32
#define LES_MINB_FLOW_F32 6
#endif
#ifndef LES_MINB_SCALAR_F32
#define LES_MINB_SCALAR_F32 6
#endif
template <typename R>
struct MinBlocks {
    static constexpr int filter = LES_MINB_FILTER, strain = LES_MINB_STRAIN, flow = LES_MINB_FLOW,
                         scalar = LES_MINB_SCALAR;
};
template <>
struct MinBlocks<float> {
    static constexpr int filter = LES_MINB_FILTER_F32, strain = LES_MINB_STRAIN_F32, flow = LES_MINB_FLOW_F32,
                         scalar = LES_MINB_SCALAR_F32;
};
// The same register budget for a block of `ntb` threads: the resident threads per SM of the
// 256-thread budget in whole blocks (at least one).
constexpr int lb_blocks(int minb, int ntb) { return (minb * NT) / ntb > 0 ? (minb * NT) / ntb : 1; }

// ---------------------------------------------------------------------------- helpers

// The scalar pass reads Phi_n, the RK running sum, the flow pass's right-hand sides and the
// diffusivities once per stage and writes the running sum back for the next stage only:
// these go through ld.global.cs / st.global.cs (evict first), so they do not push the
// stencil fields' halo planes out of L2.  Measured at 256x128x128 on B200: DRAM traffic of
// the FP64 scalar pass 414-494 B/cell per launch (plain loads 479-531; with an L2 prefetch
// of these operands 530-622 at 3 % less time); FP32 scalar pass 1.73 -> 1.66 ms per step.
#ifndef LES_SCALAR_STREAM
#define LES_SCALAR_STREAM 1
#endif
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
    if constexpr (LES_SCALAR_STREAM != 0) return __ldcs(p);
    else return *p;
}
template <typename T>
__device__ __forceinline__ void st_stream(T* p, T v) {
    if constexpr (LES_SCALAR_STREAM != 0) __stcs(p, v);
    else *p = v;
}

template <typename R>
__device__ __forceinline__ R fit_prop(const R co[4], int zero, R L, R L2, R L3) {
    // calculate_property_from_fit (:385-391): exp(a0 + a1 L + a2 L^2 + a3 L^3); the T <= 0
    // guard is handled by the callers.
    if (zero) return R(0);
    R lp = (R)co[0] + (R)co[1] * L + (R)co[2] * L2 + (R)co[3] * L3;
    return qexp(lp);
}

template <typename R>
__device__ __forceinline__ R eos_rho(const Consts& C, R T, const R Y[NSP], R fallback) {
    const auto& K = kc<R>(C);
    // update_rho_from_EOS (:1894-1905)
    R syw = R(0);
#pragma unroll
    for (int s = 0; s < NSP; s++) syw += cdv(Y[s], K.d_mwk[s]);
    if (syw > R(1e-9) && T > R(1.0)) {
        R W = qdiv(R(1.0), syw);
        R Rm = qdiv((R)R_UNIV, W);
        return qdiv((R)P_CONST, Rm * T);
    }
    return fallback;
}
// The same on the FP64 state, with the state division of the precision form Form.
template <typename Form>
__device__ __forceinline__ double eos_rho_state(const Consts& C, double T, const double Y[NSP], double fallback) {
    double syw = 0.0;
#pragma unroll
    for (int s = 0; s < NSP; s++) syw += cdv(Y[s], C.d_mwk[s]);
    if (syw > 1e-9 && T > 1.0) {
        double W = sdiv<Form>(1.0, syw);
        double Rm = sdiv<Form>(R_UNIV, W);
        return sdiv<Form>(P_CONST, Rm * T);
    }
    return fallback;
}

// Cell-local mixture properties of one fluid cell (attr == 3).
// The diffusivities D_k are handed to store_d as soon as they are known (before the mixing
// rules, so that they and the fit polynomial's powers of ln T are not held across them).
template <typename R, typename StoreD>
__device__ __forceinline__ void cell_props(const Consts& C, R Tl, const R Yf[NSP], R rhof, R& mu_mix, R& nu,
                                           const StoreD& store_d, R& aT, R& cp_out, R& lam_out, R& alpha) {
    const auto& K = kc<R>(C);
    R X[NSP];
    R syw = R(0);
    bool tpos = Tl > R(0);
    R ym[NSP];
#pragma unroll
    for (int s = 0; s < NSP; s++) ym[s] = cdv(Yf[s], K.d_mwk[s]);
    if (tpos) {
#pragma unroll
        for (int s = 0; s < NSP; s++) syw += ym[s];
    }
    bool ok = tpos && !(syw < R(1e-9));
    // Cp (:1772-1786) -- independent of the mole fractions
    R Cp;
    if (!tpos) {
        Cp = R(1000.0);
    } else {
        R T2 = Tl * Tl, T3 = pow3_rn(Tl), T4 = pow4_rn(Tl);
        R cp = R(0);
#pragma unroll
        for (int s = 0; s < NSP; s++) {
            const auto* a = (Tl > (R)K.t_mid[s]) ? K.nasa_high[s] : K.nasa_low[s];
            R cpr = (R)a[0] + (R)a[1] * Tl + (R)a[2] * T2 + (R)a[3] * T3 + (R)a[4] * T4;
            R cpm = cpr * (R)R_UNIV;
            R cpk = (K.mwk[s] < R(1e-9)) ? R(1000.0) : cdv(cpm, K.d_mwk[s]);
            cp += Yf[s] * cpk;
        }
        Cp = fmax(R(100.0), cp);
    }
    cp_out = Cp;
    if (!ok) {
        nu = R(1.5e-5);
        mu_mix = R(1.8e-5);
        R D[NSP];
#pragma unroll
        for (int s = 0; s < NSP; s++) D[s] = R(1e-5);
        store_d(D);
        R lam = R(0.025);
        lam_out = lam;
        alpha = R(1.8e-5);
        aT = (rhof > R(1e-6) && Cp > R(1e-6)) ? qdiv(lam, rhof * Cp) : R(0);
        return;
    }
    // The FP32 form takes reciprocals once where the FP64 form (the reference's arithmetic)
    // divides per term.
    constexpr bool kF32 = std::is_same<R, float>::value;
    if constexpr (kF32) {
        const R isyw = qdiv(R(1.0), syw);
#pragma unroll
        for (int s = 0; s < NSP; s++) X[s] = ym[s] * isyw;
    } else {
        const R ysyw = qdiv(R(1.0), syw);
#pragma unroll
        for (int s = 0; s < NSP; s++) X[s] = mdiv(ym[s], syw, ysyw);
    }
    const R L = qlog(Tl);
    const R L2 = L * L;
    const R L3 = pow3_rn(L);
    {
        // Hirschfelder-Curtiss (:1716-1749): sx_a = sum over b != a (ascending b) of X_b / D_ab.
        // With a symmetric fit table each D_ab is evaluated once per unordered pair and both
        // sums take their term from it; the rows are visited in ascending order, so each sx_a
        // still receives its terms in ascending b.  1 / D_ab is taken directly as
        // exp(-P_ab(ln T)) * 1e4 (D_ab = exp(P_ab) * 1e-4), one exponential and no division: the
        // terms X_b / D_ab differ from the reference's quotients by at most ~2 ulp (the FP64
        // property pass 2.82 -> 2.53 ms per 256x128x128 step); the skip rule D_ab > 1e-12 reads
        // 1 / D_ab < 1e12.
        R sxa[NSP], D[NSP];
#pragma unroll
        for (int a = 0; a < NSP; a++) sxa[a] = R(0);
        if (C.dco_sym) {
#pragma unroll
            for (int a = 0; a < NSP; a++)
#pragma unroll
                for (int b = a + 1; b < NSP; b++) {
                    if (!(X[a] > R(1e-12) || X[b] > R(1e-12))) continue;
                    if (C.dco_zero[a][b]) continue;          // D_ab = 0 fails D_ab > 1e-12
                    const auto& co = K.dco[a][b];
                    const R lp = (R)co[0] + (R)co[1] * L + (R)co[2] * L2 + (R)co[3] * L3;
                    const R y = qexp(-lp) * R(1e4);
                    if (!(y < R(1e12))) continue;
                    if (X[b] > R(1e-12)) sxa[a] += X[b] * y;
                    if (X[a] > R(1e-12)) sxa[b] += X[a] * y;
                }
        } else {
#pragma unroll
            for (int a = 0; a < NSP; a++)
#pragma unroll
                for (int b = 0; b < NSP; b++) {
                    if (a == b || !(X[b] > R(1e-12))) continue;
                    const R v = fit_prop<R>(K.dco[a][b], C.dco_zero[a][b], L, L2, L3) * R(1e-4);
                    if (v > R(1e-12)) sxa[a] += qdiv(X[b], v);
                }
        }
#pragma unroll
        for (int a = 0; a < NSP; a++) {
            const R sx = sxa[a];
            R Dv;
            if (fabs(R(1.0) - X[a]) < R(1e-9)) {
                int o = (a != N2) ? N2 : O2;
                Dv = fit_prop<R>(K.dco[a][o], C.dco_zero[a][o], L, L2, L3) * R(1e-4);
            } else if (sx > R(1e-12)) {
                Dv = qdiv(R(1.0) - X[a], sx);
            } else {
                Dv = R(1e-5);
            }
            // pressure correction PATM / (p0 + P_f) (:1743-1746): P is identically zero in the
            // reference (it is never assigned a non-zero value), so the factor is exactly 1.
            D[a] = fmax(R(1e-9), fmin(R(1e-2), Dv));
        }
        store_d(D);
    }
    // pure-species viscosity and conductivity (:394-398, :431-437)
    // species with X < 1e-12 take no part in either mixing rule: their pure-species values
    // are not evaluated
    R muk[NSP];
#pragma unroll
    for (int s = 0; s < NSP; s++) {
        muk[s] = R(1.0);
        if (!(X[s] < R(1e-12))) muk[s] = fit_prop<R>(K.eta[s], C.eta_zero[s], L, L2, L3) * R(0.1);
    }
    // Wilke (:1530-1546) and Wassiljew (:1842-1863) share the same phi_ij, the same skip
    // rule and the same summation order, so one denominator per species serves both.
    // sqrt(mu_a / mu_b) is taken as sqrt(mu_a) * (1 / sqrt(mu_b)): 5 square roots and 5
    // reciprocals instead of 20 quotients and 20 square roots.  In FP64 this differs from the
    // reference's sqrt of the rounded quotient by at most 2 ulp (the FP64 property pass went
    // from 3.02 to 2.77 ms per 256x128x128 step); mu_a / mu_a stays exactly 1 for a positive
    // finite mu_a.
    R mu = R(0), lam = R(0);
    R rsmu[NSP];
#pragma unroll
    for (int s = 0; s < NSP; s++) {
        rsmu[s] = R(1.0);
        if (X[s] < R(1e-12)) continue;
        if constexpr (kF32) rsmu[s] = rsqrtf(muk[s]);
        else rsmu[s] = qdiv(R(1.0), qsqrt(muk[s]));
    }
#pragma unroll
    for (int a = 0; a < NSP; a++) {
        if (X[a] < R(1e-12)) continue;
        const R smu_a = qsqrt(muk[a]);
        R den = R(0);
#pragma unroll
        for (int b = 0; b < NSP; b++) {
            if (X[b] < R(1e-12)) continue;
            // as in the reference, a zero or infinite mu_a gives NaN on the diagonal too
            const R sr = (a == b && muk[a] > R(0) && muk[a] <= R(1e300)) ? R(1.0) : smu_a * rsmu[b];
            R t = R(1.0) + sr * (R)K.wpow[a][b];
            R ph = cdv(t * t, K.d_wden[a][b]);
            den += X[b] * ph;
        }
        if (den > R(1e-9)) {
            // the pure-species conductivity only where it is used
            const R lamk = fit_prop<R>(K.lam[a], C.lam_zero[a], L, L2, L3) * R(1e-5);
            if constexpr (kF32) {
                const R iden = qdiv(R(1.0), den);
                mu += (X[a] * muk[a]) * iden;
                lam += (X[a] * lamk) * iden;
            } else {
                const R yden = qdiv(R(1.0), den);
                mu += mdiv(X[a] * muk[a], den, yden);
                lam += mdiv(X[a] * lamk, den, yden);
            }
        }
    }
    mu_mix = fmax(R(1e-7), mu);
    R nuv = (rhof > R(1e-3)) ? qdiv(mu_mix, rhof) : R(1.5e-5);
    nu = fmax(R(1e-7), nuv);
    R lmix = fmax(R(1e-3), lam);
    lam_out = lmix;
    R q = R(0);
    bool qok = (rhof > R(1e-6) && Cp > R(1e-6));
    if (qok) q = qdiv(lmix, rhof * Cp);
    alpha = fmax(R(1e-7), qok ? q : R(1.8e-5));
    aT = q;
}

// ------------------------------------------------------------------ pass A: filter + props

template <typename R, typename RI = R, bool BATCH = false>
__global__ void __launch_bounds__(NT, MinBlocks<R>::filter)
    k_filter_props(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<RI> in, F11<R> F, PropBuf<R> P,
                   double* __restrict__ part, Scalars* __restrict__ S, int want_max, Batch B) {
    const auto& K = kc<R>(C);
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    int bz = blockIdx.z;
    if constexpr (BATCH) {
        const int m = blockIdx.z / B.gz;
        bz = blockIdx.z - m * B.gz;
        const MemberTab& e = B.mt[m];
        shift_all(in, e.delta);
        shift_all(F, e.delta);
        shift_props(P, e.delta);
        attr = e.attr;
        part = e.part;
        S = e.S;
    }
    const int nx = C.nx, ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = bz * blockDim.z + threadIdx.z;
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const ptrdiff_t sI = (ptrdiff_t)ny * nz, sJ = (ptrdiff_t)nz;
    double mass = 0.0, mnu = 0.0, mal = 0.0;
    if (k < nz && j < ny && i < C.nx) {
        const size_t id = cid(i, j, k, ny, nz);
        const int a = attr[id];
        const bool filt = (a == 3) && i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1;
        R f[NSTATE];
#pragma unroll
        for (int q = 0; q < NSTATE; q++) {
            const RI* __restrict__ x = in.p[q] + id;
            if (filt) {
                f[q] = cdv(R(x[-sI]) + R(x[-sJ]) + R(x[-1]) + R(FILTER_W) * R(x[0]) + R(x[1]) + R(x[sJ]) + R(x[sI]),
                           K.d_filter);
            } else {
                f[q] = R(x[0]);
            }
            F.p[q][id] = f[q];
        }
        if (a == 1 || a == 2 || a == 3 || a == 5) mass = (((double)f[5] * C.dx) * C.dy) * C.dz;
        if (a == 3) {
            R mu_mix, nu, aT, cp, lam, alpha;
            auto store_d = [&](const R* D) {
#pragma unroll
                for (int s = 0; s < NSP; s++) P.D[s][id] = D[s];
            };
            cell_props<R>(C, f[3], &f[6], f[5], mu_mix, nu, store_d, aT, cp, lam, alpha);
            P.mu_mix[id] = mu_mix;
            P.nu[id] = nu;
            P.aT[id] = aT;
            if (P.dbg_cp) { P.dbg_cp[id] = cp; P.dbg_lam[id] = lam; P.dbg_alpha[id] = alpha; }
            mnu = (double)nu;
            mal = (double)alpha;
        } else if (P.dbg_cp) {
            // property values of non-fluid cells are never read by the step; they are filled
            // only for inspection, with the reference's defaults
            P.mu_mix[id] = R(1.8e-5);
            P.nu[id] = R(1.5e-5);
#pragma unroll
            for (int s = 0; s < NSP; s++) P.D[s][id] = R(0);
            P.aT[id] = R(0);
            P.dbg_cp[id] = R(1000.0); P.dbg_lam[id] = R(0); P.dbg_alpha[id] = R(0);
        }
    }
    // partial sums for the stage's <rho_f> (:2536-2550) and, on the last stage, the
    // nu/alpha maxima that feed the next dt (:4401-4408); in a batched launch, over the
    // member's own blocks
    const unsigned nblk = gridDim.x * gridDim.y * (BATCH ? (unsigned)B.gz : gridDim.z);
    const unsigned bid = ((unsigned)bz * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    double bm = block_sum<NT>(mass, sh, tid);
    double bn = 0.0, ba = 0.0;
    if (want_max) {
        bn = block_max<NT>(mnu, sh, tid);
        ba = block_max<NT>(mal, sh, tid);
    }
    if (tid == 0) {
        part[bid] = bm;
        if (want_max) { part[nblk + bid] = bn; part[2 * nblk + bid] = ba; }
        __threadfence();
        unsigned t = atomicAdd(&S->counter[0], 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double s = 0.0, mn = 0.0, ma = 0.0;
        // unrolled so that the partials' loads are in flight together; each thread still adds
        // its entries in ascending order, so the sum is unchanged
#pragma unroll 8
        for (unsigned q = tid; q < nblk; q += NT) {
            s += __ldcg(&part[q]);
            if (want_max) { mn = fmax(mn, __ldcg(&part[nblk + q])); ma = fmax(ma, __ldcg(&part[2 * nblk + q])); }
        }
        s = block_sum<NT>(s, sh, tid);
        if (want_max) { mn = block_max<NT>(mn, sh, tid); ma = block_max<NT>(ma, sh, tid); }
        if (tid == 0) {
            S->rho_avg = (C.total_volume > 0) ? (s / C.total_volume) : 1.2;
            if (want_max) { S->numax = mn; S->alphamax = ma; }
            S->counter[0] = 0u;
        }
    }
}

// ------------------------------------------------------------------ pass B: strain + nu_t + S_T

template <typename R, bool BATCH = false, int NTB = NT>
__global__ void __launch_bounds__(NTB, lb_blocks(MinBlocks<R>::strain, NTB))
    k_strain(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> F, PropBuf<R> P, Batch B) {
    const auto& K = kc<R>(C);
    int bz = blockIdx.z;
    ModelK<R> M;
    if constexpr (BATCH) {
        const int m = blockIdx.z / B.gz;
        bz = blockIdx.z - m * B.gz;
        const MemberTab& e = B.mt[m];
        shift_all(F, e.delta);
        shift_props(P, e.delta);
        attr = e.attr;
        M = member_model<R>(e);
    } else {
        M = model_of<R>(C);
    }
    const int nx = C.nx, ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = bz * blockDim.z + threadIdx.z;
    if (k >= nz || j >= ny || i >= C.nx) return;
    const ptrdiff_t sI = (ptrdiff_t)ny * nz, sJ = (ptrdiff_t)nz;
    const size_t id = cid(i, j, k, ny, nz);
    const bool interior = i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1;
    const int a = attr[id];
    if (interior && a == 3) {
        const R* __restrict__ uf = F.p[0] + id;
        const R* __restrict__ vf = F.p[1] + id;
        const R* __restrict__ wf = F.p[2] + id;
        R du_dx = cdv(uf[sI] - uf[-sI], K.d_2dx);
        R dv_dy = cdv(vf[sJ] - vf[-sJ], K.d_2dy);
        R dw_dz = cdv(wf[1] - wf[-1], K.d_2dz);
        R du_dy = cdv(uf[sJ] - uf[-sJ], K.d_2dy);
        R du_dz = cdv(uf[1] - uf[-1], K.d_2dz);
        R dv_dx = cdv(vf[sI] - vf[-sI], K.d_2dx);
        R dv_dz = cdv(vf[1] - vf[-1], K.d_2dz);
        R dw_dx = cdv(wf[sI] - wf[-sI], K.d_2dx);
        R dw_dy = cdv(wf[sJ] - wf[-sJ], K.d_2dy);
        R S11 = du_dx, S22 = dv_dy, S33 = dw_dz;
        R S12 = R(0.5) * (du_dy + dv_dx), S13 = R(0.5) * (du_dz + dw_dx), S23 = R(0.5) * (dv_dz + dw_dy);
        R Sij = R(2.0) * (S12 * S12 + S13 * S13 + S23 * S23) + S11 * S11 + S22 * S22 + S33 * S33;
        R Smag = qsqrt(R(2.0) * Sij);
        R div = du_dx + dv_dy + dw_dz;
        R g = F.p[4][id];
        if (g < R(0.0)) g = R(0.0);
        if (g > R(1.0)) g = R(1.0);
        R cs = M.cs_u + (M.cs_b - M.cs_u) * g;
        cs += M.cs_boost * R(4.0) * g * (R(1.0) - g);
        const R dx = (R)K.dx;
        R nut = (cs * dx) * (cs * dx) * Smag;
        P.nu_t[id] = nut;
        P.S_mag[id] = Smag;
        P.mu_eff[id] = P.mu_mix[id] + F.p[5][id] * nut;
        // SSR-SGS turbulent flame speed (:1926-1957)
        R nul = P.nu[id];
        R num = Sij - (div * div) * R(1.0 / 3.0);
        R X = qdiv((R)K.dx4, nul * nul) * num;
        R d_eta;
        if (X < R(SMALL)) {
            d_eta = R(1.0);
        } else {
            R pX = qpow(X, R(0.75));
            R arg = R(SSR_B) * pX;
            d_eta = R(SSR_A) * pX * (arg > R(1.0) ? qlog(arg) : R(0.0));
        }
        R eta = qdiv(dx, d_eta + R(SMALL));
        R Dce = R(8.0) * eta;
        R asf = R(8.0) * qexp(qdiv((R)K.ssr_cdF, Dce + R(SMALL)));
        R base = cdv(asf * eta, K.d_dx);
        R wr = qpow(base, (R)K.ssr_exp);
        R te = R(0.0);
        if (K.tau_sl > R(SMALL)) te = cdv(dx * fmax(R(0.0), div), K.d_tau_sl);
        R ratio = wr + te;
        R st = (R)K.s_l * fmax(R(0.0), ratio);
        P.ST[id] = fmax((R)K.s_l, st);
    } else {
        P.nu_t[id] = R(0);
        P.S_mag[id] = R(0);
        P.ST[id] = interior ? (R)K.s_l : R(0);
        P.mu_eff[id] = R(0);
    }
}

// ------------------------------------------------------------------ pass C: right-hand sides

// teno5_reconstruct (:2190-2236)
template <typename R>
__device__ __forceinline__ R teno5_rec(const Consts& C, R v0, R v1, R v2, R v3, R v4) {
    const auto& K = kc<R>(C);
    R a0 = v0 - R(2.0) * v1 + v2, b0 = v0 - R(4.0) * v1 + R(3.0) * v2;
    R a1 = v1 - R(2.0) * v2 + v3, b1 = v1 - v3;
    R a2 = v2 - R(2.0) * v3 + v4, b2 = R(3.0) * v2 - R(4.0) * v3 + v4;
    R is0 = R(13.0 / 12.0) * (a0 * a0) + R(1.0 / 4.0) * (b0 * b0);
    R is1 = R(13.0 / 12.0) * (a1 * a1) + R(1.0 / 4.0) * (b1 * b1);
    R is2 = R(13.0 / 12.0) * (a2 * a2) + R(1.0 / 4.0) * (b2 * b2);
    int d0 = (is0 < R(TENO_CUT)) ? 1 : 0, d1 = (is1 < R(TENO_CUT)) ? 1 : 0, d2 = (is2 < R(TENO_CUT)) ? 1 : 0;
    R p0 = cdv(R(2.0) * v0 - R(7.0) * v1 + R(11.0) * v2, K.d_six);
    R p1 = cdv(-v1 + R(5.0) * v2 + R(2.0) * v3, K.d_six);
    R p2 = cdv(R(2.0) * v2 + R(5.0) * v3 - v4, K.d_six);
    if (d0 + d1 + d2 == 0) {
        if (is0 <= is1 && is0 <= is2) return p0;
        else if (is1 <= is0 && is1 <= is2) return p1;
        else return p2;
    }
    R w0 = (R)d0 * R(0.1), w1 = (R)d1 * R(0.6), w2 = (R)d2 * R(0.3);
    R ws = w0 + w1 + w2;
    if (ws < R(1e-40)) return p1;
    // ws takes one of seven values: divide by the tabulated divisor (same bits as x / ws)
    return cdv(w0 * p0 + w1 * p1 + w2 * p2, K.d_tenows[d0 + 2 * d1 + 4 * d2]);
}

// One axis of the TENO5 G-advection (:2258-2295).
template <typename R>
__device__ __forceinline__ R teno_axis(const Consts& C, R vel, const R* __restrict__ q, ptrdiff_t s, const DCT<R>& d) {
    R q0 = q[-3 * s], q1 = q[-2 * s], q2 = q[-s], q3 = q[0], q4 = q[s], q5 = q[2 * s], q6 = q[3 * s];
    if (vel >= R(0.0)) {
        R ph = teno5_rec<R>(C, q1, q2, q3, q4, q5);
        R mh = teno5_rec<R>(C, q0, q1, q2, q3, q4);
        return cdv(vel * (ph - mh), d);
    } else {
        R mh = teno5_rec<R>(C, q5, q4, q3, q2, q1);
        R ph = teno5_rec<R>(C, q6, q5, q4, q3, q2);
        return cdv(vel * (ph - mh), d);
    }
}

// calculate_weno5_smoothness + calculate_weno5_gradient_1d (:735-827)
template <typename R>
__device__ __forceinline__ void weno_is(R v1, R v2, R v3, R v4, R v5, R& is0, R& is1, R& is2) {
    R a0 = v1 - R(2.0) * v2 + v3, b0 = v1 - R(4.0) * v2 + R(3.0) * v3;
    R a1 = v2 - R(2.0) * v3 + v4, b1 = v2 - v4;
    R a2 = v3 - R(2.0) * v4 + v5, b2 = R(3.0) * v3 - R(4.0) * v4 + v5;
    is0 = R(13.0 / 12.0) * (a0 * a0) + R(1.0 / 4.0) * (b0 * b0);
    is1 = R(13.0 / 12.0) * (a1 * a1) + R(1.0 / 4.0) * (b1 * b1);
    is2 = R(13.0 / 12.0) * (a2 * a2) + R(1.0 / 4.0) * (b2 * b2);
}
template <typename R>
__device__ __forceinline__ R weno5_grad(const Consts& C, const R* __restrict__ q, ptrdiff_t s, const DCT<R>& dx) {
    const auto& K = kc<R>(C);
    R p0 = q[-2 * s], p1 = q[-s], p2 = q[0], p3 = q[s], p4 = q[2 * s], p5 = q[3 * s];
    const R eps = R(1.0e-6);
    R i0, i1, i2;
    weno_is<R>(p1, p2, p3, p4, p5, i0, i1, i2);
    R e0 = eps + i0, e1 = eps + i1, e2 = eps + i2;
    R a0 = qdiv(R(3.0 / 10.0), e0 * e0), a1 = qdiv(R(6.0 / 10.0), e1 * e1), a2 = qdiv(R(1.0 / 10.0), e2 * e2);
    R sa = a0 + a1 + a2;
    R ysa = qdiv(R(1.0), sa);
    R w0 = mdiv(a0, sa, ysa), w1 = mdiv(a1, sa, ysa), w2 = mdiv(a2, sa, ysa);
    R s0 = cdv(R(2.0) * p1 - R(7.0) * p2 + R(11.0) * p3, K.d_six);
    R s1 = cdv(-p2 + R(5.0) * p3 + R(2.0) * p4, K.d_six);
    R s2 = cdv(R(2.0) * p3 + R(5.0) * p4 - p5, K.d_six);
    R ph = w0 * s0 + w1 * s1 + w2 * s2;
    weno_is<R>(p0, p1, p2, p3, p4, i0, i1, i2);
    e0 = eps + i0; e1 = eps + i1; e2 = eps + i2;
    a0 = qdiv(R(1.0 / 10.0), e0 * e0); a1 = qdiv(R(6.0 / 10.0), e1 * e1); a2 = qdiv(R(3.0 / 10.0), e2 * e2);
    sa = a0 + a1 + a2;
    ysa = qdiv(R(1.0), sa);
    w0 = mdiv(a0, sa, ysa); w1 = mdiv(a1, sa, ysa); w2 = mdiv(a2, sa, ysa);
    R m0 = cdv(-p0 + R(5.0) * p1 + R(2.0) * p2, K.d_six);
    R m1 = cdv(R(2.0) * p1 + R(5.0) * p2 - p3, K.d_six);
    R m2 = cdv(R(11.0) * p2 - R(7.0) * p3 + R(2.0) * p4, K.d_six);
    R mh = w0 * m0 + w1 * m1 + w2 * m2;
    return cdv(ph - mh, dx);
}

// superbee_limiter (:2017-2028)
template <typename R>
__device__ __forceinline__ R superbee(R r) {
    if (r <= R(0.0)) return R(0.0);
    R t1 = fmin(R(2.0) * r, R(1.0));
    R t2 = fmin(r, R(2.0));
    return fmax(t1, t2);
}

// superbee(dup / ddn) as the reference evaluates it (r = 1e9 when |ddn| < SMALL, :2064),
// dividing only where the limiter depends on the quotient's value.  For quotients <= 0, in
// (0.5, 1] or >= 2 the limiter is exactly 0, 1 or 2 whatever the rounding (division is
// monotonic and 0.5, 1, 2 are representable), and exact comparisons of |dup| with |ddn|
// decide those cases; NaN operands take the division.
template <typename R>
__device__ __forceinline__ R superbee_of(R dup, R ddn) {
    const R addn = fabs(ddn);
    if (addn < R(SMALL)) return R(2.0);                   // superbee(1e9)
    const R adup = fabs(dup);
    if (adup == adup && addn == addn) {
        if (dup == R(0) || ((dup > R(0)) != (ddn > R(0)))) return R(0.0);
        if (adup >= R(2.0) * addn) return R(2.0);
        if (adup <= addn && adup > R(0.5) * addn) return R(1.0);
    }
    return superbee<R>(qdiv(dup, ddn));
}

// MUSCL-superbee along one axis (:2058-2094); values at offsets -2..+2.  Both faces have
// the same ddn for either sign of the velocity; the sign only selects the upwind value and
// dup, so the two branches of the reference become selects (base + x or base - x, the same
// roundings as the reference's two expressions).
template <typename R>
__device__ __forceinline__ R muscl_axis(R vel, R pm2, R pm1, R p0, R pp1, R pp2, const DCT<R>& d) {
    const bool pos = vel >= R(0.0);
    const R ddn_m = p0 - pm1;
    const R dup_m = pos ? (pm1 - pm2) : (pp1 - p0);
    const R x_m = R(0.5) * superbee_of<R>(dup_m, ddn_m) * ddn_m;
    const R phi_imh = pos ? pm1 + x_m : p0 - x_m;
    const R ddn_p = pp1 - p0;
    const R dup_p = pos ? (p0 - pm1) : (pp2 - pp1);
    const R x_p = R(0.5) * superbee_of<R>(dup_p, ddn_p) * ddn_p;
    const R phi_iph = pos ? p0 + x_p : pp1 - x_p;
    return cdv(vel * (phi_iph - phi_imh), d);
}

// Stencil access to one field around the current cell, q(di, dj, dk): global memory (the
// cell's address and the i/j strides) or the shared-memory planes of a staged tile.  The
// helpers below take either, so both read paths run the same arithmetic.
template <typename R>
struct GAcc {
    const R* __restrict__ p;
    ptrdiff_t sI, sJ;
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const { return p[di * sI + dj * sJ + dk]; }
};
template <typename R>
__device__ __forceinline__ GAcc<R> gacc(const R* p, ptrdiff_t sI, ptrdiff_t sJ) {
    GAcc<R> a;
    a.p = p; a.sI = sI; a.sJ = sJ;
    return a;
}
// NP planes centred on the cell (di in [-NP/2, NP/2]); pl[d] points at the cell's (j, k) in
// plane i + d - NP/2, rows bw apart.  Every call site passes constant offsets, so pl[] stays
// in registers.
template <typename R, int NP>
struct SAcc {
    const R* pl[NP];
    int bw;
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const { return pl[di + NP / 2][dj * bw + dk]; }
};

// First-order upwind fallback used by the non-conservative schemes near faces
// (:642-651, :2043-2052).
template <typename R, typename A>
__device__ __forceinline__ R upwind3(const Consts& C, const A& q, R u, R v, R w) {
    const auto& K = kc<R>(C);
    R f;
    if (u >= R(0.0)) f = cdv(u * (q(0, 0, 0) - q(-1, 0, 0)), K.d_dx);
    else f = cdv(u * (q(1, 0, 0) - q(0, 0, 0)), K.d_dx);
    if (v >= R(0.0)) f += cdv(v * (q(0, 0, 0) - q(0, -1, 0)), K.d_dy);
    else f += cdv(v * (q(0, 1, 0) - q(0, 0, 0)), K.d_dy);
    if (w >= R(0.0)) f += cdv(w * (q(0, 0, 0) - q(0, 0, -1)), K.d_dz);
    else f += cdv(w * (q(0, 0, 1) - q(0, 0, 0)), K.d_dz);
    return f;
}

// calculate_convection_muscl (:2037-2159)
template <typename R, typename A>
__device__ __forceinline__ R conv_muscl(const Consts& C, const A& q, bool band2, R u, R v, R w) {
    const auto& K = kc<R>(C);
    if (band2) return upwind3<R>(C, q, u, v, w);
    R cx = muscl_axis<R>(u, q(-2, 0, 0), q(-1, 0, 0), q(0, 0, 0), q(1, 0, 0), q(2, 0, 0), K.d_dx);
    R cy = muscl_axis<R>(v, q(0, -2, 0), q(0, -1, 0), q(0, 0, 0), q(0, 1, 0), q(0, 2, 0), K.d_dy);
    R cz = muscl_axis<R>(w, q(0, 0, -2), q(0, 0, -1), q(0, 0, 0), q(0, 0, 1), q(0, 0, 2), K.d_dz);
    return cx + cy + cz;
}

// Face-averaged SGS diffusion div((nu_t/Sc) grad phi) (:2751-2760, :2853-2860, :2932-2939).
// The six face coefficients depend only on nu_t, so they are computed once per cell.
template <typename R>
struct SgsFaces {
    R iph, imh, jph, jmh, kph, kmh;
};
template <typename R, typename A>
__device__ __forceinline__ SgsFaces<R> sgs_faces(const A& nut, const DCT<R>& c2) {
    R n0 = nut(0, 0, 0);
    SgsFaces<R> g;
    g.iph = cdv(nut(1, 0, 0) + n0, c2); g.imh = cdv(n0 + nut(-1, 0, 0), c2);
    g.jph = cdv(nut(0, 1, 0) + n0, c2); g.jmh = cdv(n0 + nut(0, -1, 0), c2);
    g.kph = cdv(nut(0, 0, 1) + n0, c2); g.kmh = cdv(n0 + nut(0, 0, -1), c2);
    return g;
}
template <typename R, typename A>
__device__ __forceinline__ R sgs_div(const Consts& C, const A& q, const SgsFaces<R>& g) {
    const auto& K = kc<R>(C);
    R p0 = q(0, 0, 0);
    R sx = cdv(cdv(g.iph * (q(1, 0, 0) - p0), K.d_dx) - cdv(g.imh * (p0 - q(-1, 0, 0)), K.d_dx), K.d_dx);
    R sy = cdv(cdv(g.jph * (q(0, 1, 0) - p0), K.d_dy) - cdv(g.jmh * (p0 - q(0, -1, 0)), K.d_dy), K.d_dy);
    R sz = cdv(cdv(g.kph * (q(0, 0, 1) - p0), K.d_dz) - cdv(g.kmh * (p0 - q(0, 0, -1)), K.d_dz), K.d_dz);
    return sx + sy + sz;
}

template <typename R, typename A>
__device__ __forceinline__ R lap3(const Consts& C, const A& q) {
    const auto& K = kc<R>(C);
    R p0 = q(0, 0, 0);
    R a = cdv(q(1, 0, 0) - R(2.0) * p0 + q(-1, 0, 0), K.d_dxx);
    R b = cdv(q(0, 1, 0) - R(2.0) * p0 + q(0, -1, 0), K.d_dyy);
    R c = cdv(q(0, 0, 1) - R(2.0) * p0 + q(0, 0, -1), K.d_dzz);
    return a + b + c;
}

// C1: momentum (:2552-2697) with calculate_convection_conservative (:683-727) and the G
// equation (:2706-2825).  Writes k_rhou, k_rhov, k_rhow, k_G of fluid cells.
template <typename R, bool BATCH = false, int NTB = NT>
__global__ void __launch_bounds__(NTB, lb_blocks(MinBlocks<R>::flow, NTB))
    k_rhs_flow(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> F, PropBuf<R> P, KFlow<R> kf,
               KDbg<R> kd, const Scalars* __restrict__ Sc, Batch B) {
    const auto& K = kc<R>(C);
    int bz = blockIdx.z;
    ModelK<R> M;
    if constexpr (BATCH) {
        const int m = blockIdx.z / B.gz;
        bz = blockIdx.z - m * B.gz;
        const MemberTab& e = B.mt[m];
        shift_all(F, e.delta);
        shift_props(P, e.delta);
        shift_all(kf, e.delta);
#pragma unroll
        for (int q = 0; q < NACC; q++) kd.p[q] = nullptr;
        attr = e.attr;
        Sc = e.S;
        M = member_model<R>(e);
    } else {
        M = model_of<R>(C);
    }
    const int nx = C.nx, ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = bz * blockDim.z + threadIdx.z;
    if (k >= nz || j >= ny || i >= C.nx) return;
    const ptrdiff_t sI = (ptrdiff_t)ny * nz, sJ = (ptrdiff_t)nz;
    const size_t id = cid(i, j, k, ny, nz);
    if (attr[id] != 3) return;
    const R* __restrict__ uf = F.p[0] + id;
    const R* __restrict__ vf = F.p[1] + id;
    const R* __restrict__ wf = F.p[2] + id;
    const R* __restrict__ Gf = F.p[4] + id;
    const R* __restrict__ rf = F.p[5] + id;
    const R u0 = uf[0], v0 = vf[0], w0 = wf[0];
    const bool band2 = (i < 2 || i >= nx - 2 || j < 2 || j >= ny - 2 || k < 2 || k >= nz - 2);
    const bool band3 = (i < 3 || i >= nx - 3 || j < 3 || j >= ny - 3 || k < 3 || k >= nz - 3);
    R kmom[3];
    {
        const R r0 = rf[0];
        // face mass fluxes; in the near-face band the reference writes 0.5*(a+b)*0.5*(c+d),
        // in the interior (0.5*(a+b))*(0.5*(c+d)) -- equal values, since scaling by 0.5 is exact
        R mf_iph = (R(0.5) * (rf[sI] + r0)) * (R(0.5) * (uf[sI] + u0));
        R mf_imh = (R(0.5) * (r0 + rf[-sI])) * (R(0.5) * (u0 + uf[-sI]));
        R mf_jph = (R(0.5) * (rf[sJ] + r0)) * (R(0.5) * (vf[sJ] + v0));
        R mf_jmh = (R(0.5) * (r0 + rf[-sJ])) * (R(0.5) * (v0 + vf[-sJ]));
        R mf_kph = (R(0.5) * (rf[1] + r0)) * (R(0.5) * (wf[1] + w0));
        R mf_kmh = (R(0.5) * (r0 + rf[-1])) * (R(0.5) * (w0 + wf[-1]));
        const R mu_eff = P.mu_eff[id];
        const R* comps[3] = {uf, vf, wf};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const R* __restrict__ ph = comps[q];
            R pc = ph[0];
            R p_iph, p_imh, p_jph, p_jmh, p_kph, p_kmh;
            if (band2) {
                p_iph = (mf_iph > R(0)) ? pc : ph[sI];
                p_imh = (mf_imh > R(0)) ? ph[-sI] : pc;
                p_jph = (mf_jph > R(0)) ? pc : ph[sJ];
                p_jmh = (mf_jmh > R(0)) ? ph[-sJ] : pc;
                p_kph = (mf_kph > R(0)) ? pc : ph[1];
                p_kmh = (mf_kmh > R(0)) ? ph[-1] : pc;
            } else {
                // With the reference's face coefficients UW2 = 0, UW1 = DW1 = 0.5 (:164-166)
                // both upwind branches give 0.5*phi_L + 0.5*phi_R, so no branch is taken.
                p_iph = R(0.5) * pc + R(0.5) * ph[sI];
                p_imh = R(0.5) * ph[-sI] + R(0.5) * pc;
                p_jph = R(0.5) * pc + R(0.5) * ph[sJ];
                p_jmh = R(0.5) * ph[-sJ] + R(0.5) * pc;
                p_kph = R(0.5) * pc + R(0.5) * ph[1];
                p_kmh = R(0.5) * ph[-1] + R(0.5) * pc;
            }
            R conv = cdv(mf_iph * p_iph - mf_imh * p_imh, K.d_dx) + cdv(mf_jph * p_jph - mf_jmh * p_jmh, K.d_dy) +
                     cdv(mf_kph * p_kph - mf_kmh * p_kmh, K.d_dz);
            kmom[q] = -conv + mu_eff * lap3<R>(C, gacc(ph, sI, sJ));
        }
        R grav = (r0 - (R)Sc->rho_avg) * R(G_GRAVITY);
        R fx = R(0), fy = R(0), fz = R(0);
        if (C.flame_accel) {
            R Gl = Gf[0];
            if (Gl > R(0.01) && Gl < R(0.99)) {
                R dGx = cdv(Gf[sI] - Gf[-sI], K.d_2dx);
                R dGy = cdv(Gf[sJ] - Gf[-sJ], K.d_2dy);
                R dGz = cdv(Gf[1] - Gf[-1], K.d_2dz);
                if (dGx < R(0.0)) dGx = R(0.0);
                if (dGy < R(0.0)) dGy = R(0.0);
                R zrel = ((R)k * (R)K.dz) - (R)K.inlet_center_z;
                if (zrel > R(0.0)) {
                    if (dGz < R(0.0)) dGz = R(0.0);
                } else {
                    if (dGz > R(0.0)) dGz = R(0.0);
                }
                R df = Gl - M.accel_center;
                R window = qexp(cdv(-(df * df), M.d_w2));
                // tip_mask is the literal 1.0 in the momentum source (:2638)
                R cf = M.accel_strength * r0 * window * R(1.0);
                fx = cf * dGx * R(0.05);
                fy = cf * dGy * R(1.0);
                fz = cf * dGz * R(1.0);
                R zp = (R)k * (R)K.dz, ramp = R(1.0);
                if (zp < R(RAMP_DIST)) ramp = cdv(zp, K.d_ramp);
                fx *= ramp; fy *= ramp; fz *= ramp;
            }
        }
        const R lim = R(FORCE_LIMIT);
        if (fx > lim) fx = lim;
        if (fx < -lim) fx = -lim;
        if (fy > lim) fy = lim;
        if (fy < -lim) fy = -lim;
        if (fz > lim) fz = lim;
        if (fz < -lim) fz = -lim;
        kmom[0] = kmom[0] + grav + fx;
        kmom[1] = kmom[1] + fy;
        kmom[2] = kmom[2] + fz;
    }
    R kG;
    {
        R conv;
        if (band3) {
            if (band2) {
                conv = upwind3<R>(C, gacc(Gf, sI, sJ), u0, v0, w0);
            } else {
                // calculate_convection_non_conservative interior branch (:652-677); the
                // zero UW2 coefficient again makes both upwind branches identical.
                R pc = Gf[0];
                R p_iph = R(0.5) * pc + R(0.5) * Gf[sI], p_imh = R(0.5) * Gf[-sI] + R(0.5) * pc;
                R p_jph = R(0.5) * pc + R(0.5) * Gf[sJ], p_jmh = R(0.5) * Gf[-sJ] + R(0.5) * pc;
                R p_kph = R(0.5) * pc + R(0.5) * Gf[1], p_kmh = R(0.5) * Gf[-1] + R(0.5) * pc;
                R cx = cdv(u0 * (p_iph - p_imh), K.d_dx);
                R cy = cdv(v0 * (p_jph - p_jmh), K.d_dy);
                R cz = cdv(w0 * (p_kph - p_kmh), K.d_dz);
                conv = cx + cy + cz;
            }
        } else {
            R fxa = teno_axis<R>(C, u0, Gf, sI, K.d_dx);
            R fya = teno_axis<R>(C, v0, Gf, sJ, K.d_dy);
            R fza = teno_axis<R>(C, w0, Gf, 1, K.d_dz);
            conv = fxa + fya + fza;
        }
        SgsFaces<R> gf = sgs_faces<R>(gacc<R>(P.nu_t + id, sI, sJ), K.d_sct2);
        R sgs = sgs_div<R>(C, gacc(Gf, sI, sJ), gf);
        R gx, gy, gz;
        if (Sc->t_loop >= C.weno_step && !band3) {
            gx = weno5_grad<R>(C, Gf, sI, K.d_dx);
            gy = weno5_grad<R>(C, Gf, sJ, K.d_dy);
            gz = weno5_grad<R>(C, Gf, 1, K.d_dz);
        } else {
            gx = cdv(Gf[sI] - Gf[-sI], K.d_2dx);
            gy = cdv(Gf[sJ] - Gf[-sJ], K.d_2dy);
            gz = cdv(Gf[1] - Gf[-1], K.d_2dz);
        }
        R gmag = qsqrt(gx * gx + gy * gy + gz * gz);
        if (P.grad_g) P.grad_g[id] = gmag;   // grad_G_magnitude_for_debug (:2783)
        R prop = P.ST[id] * gmag;
        R art = R(0);
        if (C.flame_accel) {
            R Gl = Gf[0];
            if (Gl > R(0.1) && Gl < R(0.99)) {
                R df = Gl - M.accel_center;
                R window = qexp(cdv(-(df * df), M.d_w2));
                // tip_mask = 1 - exp(-r^2 / 0^2) is exactly 1 for every fluid cell (j >= 1)
                // because TIP_PROTECTION_RADIUS is 0.0 (:234, :2806-2807).
                R adc = R(5.0) * (P.nu_t[id] + R(1.0e-5)) * window * R(1.0);
                art = adc * lap3<R>(C, gacc(Gf, sI, sJ));
            }
        }
        kG = -conv + prop + sgs + art;
    }
    kf.p[0][id] = kmom[0];
    kf.p[1][id] = kmom[1];
    kf.p[2][id] = kmom[2];
    kf.p[3][id] = kG;
    if (kd.p[0]) {
        kd.p[0][id] = kmom[0];
        kd.p[1][id] = kmom[1];
        kd.p[2][id] = kmom[2];
        kd.p[4][id] = kG;
    }
}

// C2: species (:2837-2904) and temperature (:2912-2962), then the RK4 bookkeeping.
// stage: 0,1,2 -> intermediate stage with coefficient 0.5/0.5/1.0, 3 -> final combine.
// Where the scalar pass reads its stencil fields (filtered T and Y_k, nu_t): global memory,
// or the shared-memory tile of the staged kernel (les_tma.cuh).
template <typename R>
struct GSrc {
    const R* T;
    const R* Y[NSP];
    const R* nut;
    ptrdiff_t sI, sJ;
    __device__ __forceinline__ GAcc<R> y(int s) const { return gacc(Y[s], sI, sJ); }
    __device__ __forceinline__ GAcc<R> t() const { return gacc(T, sI, sJ); }
    __device__ __forceinline__ GAcc<R> nu() const { return gacc(nut, sI, sJ); }
};

// One cell of the scalar pass (the body shared by both read paths).
template <typename R, typename RS, typename Src>
__device__ __forceinline__ void rhs_scalar_cell(const Consts& C, const uint8_t* __restrict__ attr, const F11<R>& F,
                                                const PropBuf<R>& P, const F11<RS>& S0, const F11<R>& St,
                                                const AccBuf<R>& acc, const KFlow<R>& kf, const KDbg<R>& kd,
                                                const Scalars* __restrict__ Sc, int stage, int i, int j, int k,
                                                const Src& src, const R relax) {
    const auto& K = kc<R>(C);
    const int nx = C.nx, ny = C.ny, nz = C.nz;
    const size_t id = cid(i, j, k, ny, nz);
    const int a = attr[id];

    if (a != 3) {
        // non-fluid cells: the temp state is Phi_n with the current velocity (:4444, :4454);
        // rho_temp is only ever written on outlet/fluid cells (:1893), so it stays 0 on
        // inlet/wall/symmetry cells.  These values are the same for all stages of a step.
        if (stage == 0) {
            RS Y0[NSP];
#pragma unroll
            for (int q = 0; q < NSTATE; q++)
                if (q != 5) St.p[q][id] = R(S0.p[q][id]);
#pragma unroll
            for (int s = 0; s < NSP; s++) Y0[s] = S0.p[6 + s][id];
            if (a == 2) St.p[5][id] = R(eos_rho_state<R>(C, S0.p[3][id], Y0, S0.p[5][id]));
        } else if (stage == 3 && a == 2) {
            RS Y0[NSP];
#pragma unroll
            for (int s = 0; s < NSP; s++) Y0[s] = S0.p[6 + s][id];
            S0.p[5][id] = eos_rho_state<R>(C, S0.p[3][id], Y0, S0.p[5][id]);
        }
        if (kd.p[0]) {
#pragma unroll
            for (int q = 0; q < NACC; q++) kd.p[q][id] = R(0);
        }
        return;
    }

    const R u0 = F.p[0][id], v0 = F.p[1][id], w0 = F.p[2][id];
    const bool band2 = (i < 2 || i >= nx - 2 || j < 2 || j >= ny - 2 || k < 2 || k >= nz - 2);
    R kv[NACC];
    R g = F.p[4][id];
    if (g < R(0.0)) g = R(0.0);
    if (g > R(1.0)) g = R(1.0);
    // Temperature; in the FP64 form ahead of the species, which leaves the register allocator
    // fewer values live across the species loop (spills 100/260 -> 44/148 bytes per thread),
    // in the FP32 form after them (fewer spills that way round).  Either order gives the same
    // bits: the two are independent.
    auto temperature = [&]() {
        const auto qT = src.t();
        R conv = conv_muscl<R>(C, qT, band2, u0, v0, w0);
        R mol = ld_stream(P.aT + id) * lap3<R>(C, qT);
        const SgsFaces<R> gt = sgs_faces<R>(src.nu(), K.d_prt2);
        R sgs = sgs_div<R>(C, qT, gt);
        R Tt = (R)K.t_in + g * (R)K.t_burnt_span;
        R nud = relax * (Tt - qT(0, 0, 0));
        kv[3] = -conv + mol + sgs + nud;
    };
    constexpr bool kF32s = std::is_same<R, float>::value;
    if constexpr (!kF32s) temperature();
    const SgsFaces<R> gs = sgs_faces<R>(src.nu(), K.d_sct2);
#pragma unroll
    for (int s = 0; s < NSP; s++) {
        R tgt;
        if (s == C3H8) tgt = (R)K.inletYk[C3H8] * (R(1.0) - g);
        else if (s == O2) tgt = fmax(R(0.0), (R)K.inletYk[O2] - (R)K.cons_o2 * g);
        else if (s == CO2) tgt = (R)K.inletYk[CO2] + (R)K.prod_co2 * g;
        else if (s == H2O) tgt = (R)K.inletYk[H2O] + (R)K.prod_h2o * g;
        else tgt = (R)K.inletYk[N2];
        const auto qY = src.y(s);
        R conv = conv_muscl<R>(C, qY, band2, u0, v0, w0);
        R mol = ld_stream(P.D[s] + id) * lap3<R>(C, qY);
        R sgs = sgs_div<R>(C, qY, gs);
        R nud = relax * (tgt - qY(0, 0, 0));
        kv[5 + s] = -conv + mol + sgs + nud;
    }
    if constexpr (kF32s) temperature();
    kv[0] = ld_stream(kf.p[0] + id);
    kv[1] = ld_stream(kf.p[1] + id);
    kv[2] = ld_stream(kf.p[2] + id);
    kv[4] = ld_stream(kf.p[3] + id);
    if (kd.p[0]) {
        kd.p[3][id] = kv[3];
#pragma unroll
        for (int s = 0; s < NSP; s++) kd.p[5 + s][id] = kv[5 + s];
    }

    // ---- RK4 bookkeeping.  acc holds k1, k1 + 2k2, (k1 + 2k2) + 2k3: exactly the
    // left-to-right partial sums of k1 + 2.0*k2 + 2.0*k3 + k4 (:4520).
    const bool fin = (stage == 3);
    const double dt = Sc->dt;
    R incr[NACC];
    if (stage == 0) {
#pragma unroll
        for (int q = 0; q < NACC; q++) { incr[q] = kv[q]; st_stream(acc.p[q] + id, kv[q]); }
    } else if (stage < 3) {
#pragma unroll
        for (int q = 0; q < NACC; q++) { incr[q] = kv[q]; st_stream(acc.p[q] + id, ld_stream(acc.p[q] + id) + R(2.0) * kv[q]); }
    } else {
#pragma unroll
        for (int q = 0; q < NACC; q++) incr[q] = ld_stream(acc.p[q] + id) + kv[q];
    }
    // The update itself runs in the state's type: in the FP32 form the right-hand sides are
    // FP32 and Phi_n, the stage update and the final combine FP64, so increments far below
    // the state's FP32 ulp are not rounded away step after step.
    const RS cdt = fin ? (RS)(dt / 6.0) : (RS)((stage == 2 ? 1.0 : 0.5) * dt);
    const RS rho_n = ld_stream(S0.p[5] + id);
    RS Tn = ld_stream(S0.p[3] + id) + cdt * (RS)incr[3];
    RS Gn = ld_stream(S0.p[4] + id) + cdt * (RS)incr[4];
    RS Y[NSP];
#pragma unroll
    for (int s = 0; s < NSP; s++) Y[s] = ld_stream(S0.p[6 + s] + id) + cdt * (RS)incr[5 + s];
    Tn = fmax(RS(200.0), fmin(RS(3000.0), Tn));
    Gn = fmax(RS(0.0), fmin(RS(1.0), Gn));
    RS sy = RS(0);
#pragma unroll
    for (int s = 0; s < NSP; s++) {
        Y[s] = fmax(RS(0.0), fmin(RS(1.0), Y[s]));
        sy += Y[s];
    }
    if (sy > RS(SMALL)) {
#pragma unroll
        for (int s = 0; s < NSP; s++) Y[s] = sdiv<R>(Y[s], sy);
    }
    RS rn = eos_rho_state<R>(C, Tn, Y, rho_n);
    RS vel[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        RS m = rho_n * ld_stream(S0.p[q] + id) + cdt * (RS)incr[q];   // rhou = rho*u after the BC (:3146)
        vel[q] = (rn > RS(SMALL)) ? sdiv<R>(m, rn) : RS(0);
    }
    if (fin) {
        RS* const* out = S0.p;
        out[0][id] = vel[0]; out[1][id] = vel[1]; out[2][id] = vel[2];
        out[3][id] = Tn; out[4][id] = Gn; out[5][id] = rn;
#pragma unroll
        for (int s = 0; s < NSP; s++) out[6 + s][id] = Y[s];
    } else {
        R* const* out = St.p;
        out[0][id] = R(vel[0]); out[1][id] = R(vel[1]); out[2][id] = R(vel[2]);
        out[3][id] = R(Tn); out[4][id] = R(Gn); out[5][id] = R(rn);
#pragma unroll
        for (int s = 0; s < NSP; s++) out[6 + s][id] = R(Y[s]);
    }
}

template <typename R, typename RS = R, bool BATCH = false, int NTB = NT>
__global__ void __launch_bounds__(NTB, lb_blocks(MinBlocks<R>::scalar, NTB))
    k_rhs_scalar(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> F, PropBuf<R> P, F11<RS> S0, F11<R> St,
                 AccBuf<R> acc, KFlow<R> kf, KDbg<R> kd, const Scalars* __restrict__ Sc, int stage, Batch B) {
    int bz = blockIdx.z;
    R relax;
    if constexpr (BATCH) {
        const int m = blockIdx.z / B.gz;
        bz = blockIdx.z - m * B.gz;
        const MemberTab& e = B.mt[m];
        shift_all(F, e.delta);
        shift_props(P, e.delta);
        shift_all(S0, e.delta);
        shift_all(St, e.delta);
        shift_all(acc, e.delta);
        shift_all(kf, e.delta);
#pragma unroll
        for (int q = 0; q < NACC; q++) kd.p[q] = nullptr;
        attr = e.attr;
        Sc = e.S;
        relax = member_model<R>(e).relax;
    } else {
        relax = (R)kc<R>(C).relax;
    }
    const int ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = bz * blockDim.z + threadIdx.z;
    if (k >= nz || j >= ny || i >= C.nx) return;
    const size_t id = cid(i, j, k, ny, nz);
    GSrc<R> src;
    src.sI = (ptrdiff_t)ny * nz;
    src.sJ = (ptrdiff_t)nz;
    src.T = F.p[3] + id;
#pragma unroll
    for (int s = 0; s < NSP; s++) src.Y[s] = F.p[6 + s] + id;
    src.nut = P.nu_t + id;
    rhs_scalar_cell<R, RS>(C, attr, F, P, S0, St, acc, kf, kd, Sc, stage, i, j, k, src, relax);
}

// ------------------------------------------------------------------ boundary conditions
// apply_boundary_conditions (:2967-3161) in its face order: i-faces (with the SEM +
// white-noise inflow), then for every interior i the j-faces, then the k-faces, then the
// equation of state and mass-fraction renormalisation everywhere.

template <typename R>
__device__ __forceinline__ void copy_cell(F11<R>& S, size_t dst, size_t src) {
#pragma unroll
    for (int q = 0; q < NSTATE; q++)
        if (q != 5) S.p[q][dst] = S.p[q][src];
}
template <typename R>
__device__ __forceinline__ void ambient_cell(const Consts& C, F11<R>& S, size_t dst) {
    const auto& K = kc<R>(C);
    S.p[0][dst] = R(0); S.p[1][dst] = R(0); S.p[2][dst] = R(0);
    S.p[3][dst] = (R)K.t_amb; S.p[4][dst] = R(0);
#pragma unroll
    for (int s = 0; s < NSP; s++) S.p[6 + s][dst] = (R)K.ambientYk[s];
}

template <typename R, typename Form = R>
__global__ void k_bc_iface(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> S,
                           const double* __restrict__ plane, const double* __restrict__ noise,
                           const int* __restrict__ inlet_pos) {
    const auto& K = kc<R>(C);
    const int nx = C.nx, ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= nz) return;
    const size_t i0 = cid(0, j, k, ny, nz), i1 = cid(1, j, k, ny, nz);
    const int a0 = attr[i0];
    if (a0 == 1) {
        const size_t p = (size_t)j * nz + k;
        const size_t npl = (size_t)ny * nz;
        const int q = inlet_pos[p];
        const R amp = (R)K.noise_amp;
        R r1 = (R)noise[3 * q + 0], r2 = (R)noise[3 * q + 1], r3 = (R)noise[3 * q + 2];
        S.p[0][i0] = fmax(R(0.0), (R)K.u_in + (R)plane[p] + amp * r1);
        S.p[1][i0] = (R)plane[npl + p] + amp * r2;
        S.p[2][i0] = (R)plane[2 * npl + p] + amp * r3;
        S.p[3][i0] = (R)K.t_in;
        S.p[4][i0] = R(0);
#pragma unroll
        for (int s = 0; s < NSP; s++) S.p[6 + s][i0] = (R)K.inletYk[s];
    } else if (a0 == 4) {
        if (S.p[0][i1] < R(0)) ambient_cell<R>(C, S, i0);
        else copy_cell<R>(S, i0, i1);
    } else if (a0 == 6) {
        S.p[0][i0] = R(0); S.p[1][i0] = R(0); S.p[2][i0] = R(0);
        S.p[3][i0] = S.p[3][i1];
        S.p[4][i0] = S.p[4][i1];
#pragma unroll
        for (int s = 0; s < NSP; s++) S.p[6 + s][i0] = S.p[6 + s][i1];
    }
    const size_t in = cid(nx - 1, j, k, ny, nz), im = cid(nx - 2, j, k, ny, nz);
    if (attr[in] == 2) copy_cell<R>(S, in, im);
}

template <typename R, typename Form = R>
__global__ void k_bc_jface(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> S) {
    const int ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y + 1;
    if (k >= nz) return;
    const size_t b = cid(i, 0, k, ny, nz), n1 = cid(i, 1, k, ny, nz);
    if (attr[b] == 5) {
        S.p[3][b] = S.p[3][n1];
        S.p[4][b] = S.p[4][n1];
#pragma unroll
        for (int s = 0; s < NSP; s++) S.p[6 + s][b] = S.p[6 + s][n1];
        S.p[0][b] = S.p[0][n1];
        S.p[1][b] = R(0.0);
        S.p[2][b] = S.p[2][n1];
    }
    const size_t t = cid(i, ny - 1, k, ny, nz), tm = cid(i, ny - 2, k, ny, nz);
    if (attr[t] == 4) {
        if (S.p[1][tm] < R(0)) ambient_cell<R>(C, S, t);
        else copy_cell<R>(S, t, tm);
    }
}

template <typename R, typename Form = R>
__global__ void k_bc_kface(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> S) {
    const int ny = C.ny, nz = C.nz;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y + 1;
    if (j >= ny) return;
    const size_t b = cid(i, j, 0, ny, nz), n1 = cid(i, j, 1, ny, nz);
    if (attr[b] == 4) {
        if (S.p[2][n1] > R(0)) ambient_cell<R>(C, S, b);
        else copy_cell<R>(S, b, n1);
    }
    const size_t t = cid(i, j, nz - 1, ny, nz), tm = cid(i, j, nz - 2, ny, nz);
    if (attr[t] == 4) {
        if (S.p[2][tm] < R(0)) ambient_cell<R>(C, S, t);
        else copy_cell<R>(S, t, tm);
    }
}

// EOS + renormalisation everywhere (:3130-3160) fused with the max-velocity reduction
// over inlet/fluid cells for the next dt (:1472-1485).
template <typename R, typename Form = R>
__global__ void __launch_bounds__(NT) k_bc_eos(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> S,
                                               double* __restrict__ part, Scalars* __restrict__ Sc) {
    const auto& K = kc<R>(C);
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    const int ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z * blockDim.z + threadIdx.z;
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    double vmax = 0.0;
    if (k < nz && j < ny && i < C.nx) {
        const size_t id = cid(i, j, k, ny, nz);
        const int a = attr[id];
        R Y[NSP];
#pragma unroll
        for (int s = 0; s < NSP; s++) Y[s] = S.p[6 + s][id];
        R T = S.p[3][id];
        R syw = R(0);
#pragma unroll
        for (int s = 0; s < NSP; s++) syw += cdv(Y[s], K.d_mwk[s]);
        R rho = (syw > R(1e-9) && T > R(1.0)) ? sdiv<Form>(P_CONST, sdiv<Form>(R_UNIV, sdiv<Form>(1.0, syw)) * T)
                                              : R(1.2);
        S.p[5][id] = rho;
        if (a == 3 || a == 2 || a == 5) {
            R sy = R(0);
#pragma unroll
            for (int s = 0; s < NSP; s++) sy += Y[s];
            if (sy > R(1e-6)) {
#pragma unroll
                for (int s = 0; s < NSP; s++) S.p[6 + s][id] = sdiv<Form>(Y[s], sy);
            }
        }
        if (a == 1 || a == 3) {
            R u = S.p[0][id], v = S.p[1][id], w = S.p[2][id];
            vmax = (double)sqrt(u * u + v * v + w * w);
        }
    }
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    double bm = block_max<NT>(vmax, sh, tid);
    if (tid == 0) {
        part[bid] = bm;
        __threadfence();
        unsigned t = atomicAdd(&Sc->counter[1], 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double m = 0.0;
#pragma unroll 8
        for (unsigned q = tid; q < nblk; q += NT) m = fmax(m, __ldcg(&part[q]));
        m = block_max<NT>(m, sh, tid);
        if (tid == 0) {
            Sc->umax = m;
            Sc->counter[1] = 0u;
        }
    }
}

// Max velocity over inlet/fluid cells without touching the state (after an upload).
template <typename R, typename Form = R>
__global__ void __launch_bounds__(NT) k_umax(LES_KERNEL_CONSTS, const uint8_t* __restrict__ attr, F11<R> S,
                                             double* __restrict__ part, Scalars* __restrict__ Sc) {
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    const int ny = C.ny, nz = C.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z * blockDim.z + threadIdx.z;
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    double vmax = 0.0;
    if (k < nz && j < ny && i < C.nx) {
        const size_t id = cid(i, j, k, ny, nz);
        const int a = attr[id];
        if (a == 1 || a == 3) {
            R u = S.p[0][id], v = S.p[1][id], w = S.p[2][id];
            vmax = (double)sqrt(u * u + v * v + w * w);
        }
    }
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    double bm = block_max<NT>(vmax, sh, tid);
    if (tid == 0) {
        part[bid] = bm;
        __threadfence();
        unsigned t = atomicAdd(&Sc->counter[2], 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double m = 0.0;
#pragma unroll 8
        for (unsigned q = tid; q < nblk; q += NT) m = fmax(m, __ldcg(&part[q]));
        m = block_max<NT>(m, sh, tid);
        if (tid == 0) {
            Sc->umax = m;
            Sc->counter[2] = 0u;
        }
    }
}

// ------------------------------------------------------------------ diagnostics

template <typename R, typename Form = R>
__global__ void __launch_bounds__(NT) k_monitor(LES_KERNEL_CONSTS, F11<R> S, double* __restrict__ part,
                                                Scalars* __restrict__ Sc, size_t n) {
    // write_monitor_log (:3884-3897)
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    const int tid = threadIdx.x;
    double mass = 0.0, tmin = 1.0e9, tmax = -1.0e9, gmin = 1.0e9, gmax = -1.0e9, ymin = 1.0e9;
    for (size_t id = (size_t)blockIdx.x * NT + tid; id < n; id += (size_t)gridDim.x * NT) {
        double r = (double)S.p[5][id], T = (double)S.p[3][id], G = (double)S.p[4][id], Y = (double)S.p[6][id];
        mass += ((r * C.dx) * C.dy) * C.dz;
        tmin = fmin(tmin, T); tmax = fmax(tmax, T);
        gmin = fmin(gmin, G); gmax = fmax(gmax, G);
        ymin = fmin(ymin, Y);
    }
    const unsigned nblk = gridDim.x;
    double v[6];
    v[0] = block_sum<NT>(mass, sh, tid);
    v[1] = block_min<NT>(tmin, sh, tid);
    v[2] = block_max<NT>(tmax, sh, tid);
    v[3] = block_min<NT>(gmin, sh, tid);
    v[4] = block_max<NT>(gmax, sh, tid);
    v[5] = block_min<NT>(ymin, sh, tid);
    if (tid == 0) {
        for (int q = 0; q < 6; q++) part[q * nblk + blockIdx.x] = v[q];
        __threadfence();
        unsigned t = atomicAdd(&Sc->counter[3], 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double acc[6] = {0.0, 1.0e9, -1.0e9, 1.0e9, -1.0e9, 1.0e9};
#pragma unroll 4
        for (unsigned q = tid; q < nblk; q += NT) {
            acc[0] += __ldcg(&part[q]);
            acc[1] = fmin(acc[1], __ldcg(&part[nblk + q]));
            acc[2] = fmax(acc[2], __ldcg(&part[2 * nblk + q]));
            acc[3] = fmin(acc[3], __ldcg(&part[3 * nblk + q]));
            acc[4] = fmax(acc[4], __ldcg(&part[4 * nblk + q]));
            acc[5] = fmin(acc[5], __ldcg(&part[5 * nblk + q]));
        }
        acc[0] = block_sum<NT>(acc[0], sh, tid);
        acc[1] = block_min<NT>(acc[1], sh, tid);
        acc[2] = block_max<NT>(acc[2], sh, tid);
        acc[3] = block_min<NT>(acc[3], sh, tid);
        acc[4] = block_max<NT>(acc[4], sh, tid);
        acc[5] = block_min<NT>(acc[5], sh, tid);
        if (tid == 0) {
            for (int q = 0; q < 6; q++) Sc->mon[q] = acc[q];
            Sc->counter[3] = 0u;
        }
    }
}

template <typename RS, typename R = RS>
__global__ void k_probe(LES_KERNEL_CONSTS, F11<RS> S, PropBuf<R> P, const int* __restrict__ st, int n, int kline,
                        double* __restrict__ out) {
    const int ny = C.ny, nz = C.nz;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (j >= ny || q >= n) return;
    const size_t id = cid(st[q], j, kline, ny, nz);
    double* o = out + ((size_t)q * ny + j) * 6;
    o[0] = (double)S.p[0][id];
    o[1] = (double)S.p[1][id];
    o[2] = (double)S.p[2][id];
    o[3] = (double)S.p[4][id];
    o[4] = (double)P.nu_t[id];
    o[5] = (double)P.S_mag[id];
}

// Host-driven steps: dt and t_loop come from the caller.
static __global__ void k_set_step(Scalars* __restrict__ Sc, double dt, int t_loop) {
    Sc->dt = dt;
    Sc->t_loop = t_loop;
}

// Device loop, after the boundary conditions: the probe lines of record_flame_region_data
// (:3403-3471) and dt/|u|max of this step go to history slot run_step.
template <typename RS, typename R = RS>
__global__ void k_loop_post(LES_KERNEL_CONSTS, F11<RS> S, PropBuf<R> P, const Scalars* __restrict__ Sc,
                            const int* __restrict__ st, int n, int kline, int cap, double* __restrict__ hprobe,
                            double* __restrict__ hdt, double* __restrict__ humax) {
    const int ny = C.ny, nz = C.nz;
    const int slot = Sc->run_step;
    if (slot < 0 || slot >= cap) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        hdt[slot] = Sc->dt;
        humax[slot] = Sc->umax_used;
    }
    if (j >= ny || q >= n) return;
    const size_t id = cid(st[q], j, kline, ny, nz);
    double* o = hprobe + (((size_t)slot * n + q) * ny + j) * 6;
    o[0] = (double)S.p[0][id];
    o[1] = (double)S.p[1][id];
    o[2] = (double)S.p[2][id];
    o[3] = (double)S.p[4][id];
    o[4] = (double)P.nu_t[id];
    o[5] = (double)P.S_mag[id];
}

// Device loop: the monitor reductions (:3874-3918) on steps with t_loop % 10 == 0, written
// to history slot run_step (other slots are left untouched).
template <typename R, typename Form = R>
__global__ void __launch_bounds__(NT) k_loop_monitor(LES_KERNEL_CONSTS, F11<R> S, double* __restrict__ part,
                                                     Scalars* __restrict__ Sc, size_t n, int cap,
                                                     double* __restrict__ hmon) {
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    if (Sc->t_loop % 10 != 0) return;          // uniform across the grid
    const int slot = Sc->run_step;
    if (slot < 0 || slot >= cap) return;
    const int tid = threadIdx.x;
    double mass = 0.0, tmin = 1.0e9, tmax = -1.0e9, gmin = 1.0e9, gmax = -1.0e9, ymin = 1.0e9;
    for (size_t id = (size_t)blockIdx.x * NT + tid; id < n; id += (size_t)gridDim.x * NT) {
        double r = (double)S.p[5][id], T = (double)S.p[3][id], G = (double)S.p[4][id], Y = (double)S.p[6][id];
        mass += ((r * C.dx) * C.dy) * C.dz;
        tmin = fmin(tmin, T); tmax = fmax(tmax, T);
        gmin = fmin(gmin, G); gmax = fmax(gmax, G);
        ymin = fmin(ymin, Y);
    }
    const unsigned nblk = gridDim.x;
    double v[6];
    v[0] = block_sum<NT>(mass, sh, tid);
    v[1] = block_min<NT>(tmin, sh, tid);
    v[2] = block_max<NT>(tmax, sh, tid);
    v[3] = block_min<NT>(gmin, sh, tid);
    v[4] = block_max<NT>(gmax, sh, tid);
    v[5] = block_min<NT>(ymin, sh, tid);
    if (tid == 0) {
        for (int q = 0; q < 6; q++) part[q * nblk + blockIdx.x] = v[q];
        __threadfence();
        unsigned t = atomicAdd(&Sc->counter[3], 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double acc[6] = {0.0, 1.0e9, -1.0e9, 1.0e9, -1.0e9, 1.0e9};
#pragma unroll 4
        for (unsigned q = tid; q < nblk; q += NT) {
            acc[0] += __ldcg(&part[q]);
            acc[1] = fmin(acc[1], __ldcg(&part[nblk + q]));
            acc[2] = fmax(acc[2], __ldcg(&part[2 * nblk + q]));
            acc[3] = fmin(acc[3], __ldcg(&part[3 * nblk + q]));
            acc[4] = fmax(acc[4], __ldcg(&part[4 * nblk + q]));
            acc[5] = fmin(acc[5], __ldcg(&part[5 * nblk + q]));
        }
        acc[0] = block_sum<NT>(acc[0], sh, tid);
        acc[1] = block_min<NT>(acc[1], sh, tid);
        acc[2] = block_max<NT>(acc[2], sh, tid);
        acc[3] = block_min<NT>(acc[3], sh, tid);
        acc[4] = block_max<NT>(acc[4], sh, tid);
        acc[5] = block_min<NT>(acc[5], sh, tid);
        if (tid == 0) {
            for (int q = 0; q < 6; q++) hmon[(size_t)slot * 6 + q] = acc[q];
            Sc->counter[3] = 0u;
        }
    }
}

// update_time_averages (:3166-3191) after the boundary conditions of steps with
// t_loop >= start (:4577-4579): first and second moments summed per cell in FP64.
template <typename RS, typename Form = RS>
__global__ void __launch_bounds__(NT) k_time_avg(F11<RS> S, AvgBuf A, Scalars* __restrict__ Sc, size_t n, int start) {
    if (Sc->t_loop < start) return;            // uniform across the grid
    for (size_t id = (size_t)blockIdx.x * NT + threadIdx.x; id < n; id += (size_t)gridDim.x * NT) {
        const double u = (double)S.p[0][id], v = (double)S.p[1][id], w = (double)S.p[2][id];
        const double G = (double)S.p[4][id];
        A.p[0][id] += u;
        A.p[1][id] += v;
        A.p[2][id] += w;
        A.p[9][id] += G;
        A.p[3][id] += u * u;
        A.p[4][id] += v * v;
        A.p[5][id] += w * w;
        A.p[6][id] += u * v;
        A.p[7][id] += u * w;
        A.p[8][id] += v * w;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) Sc->avg_steps += 1;
}

// Device loop, last launch of a step: advance the step counters.
static __global__ void k_loop_tick(Scalars* __restrict__ Sc) {
    Sc->t_loop += 1;
    Sc->run_step += 1;
}

template <typename R, typename Form = R>
__global__ void k_check_finite(const R* __restrict__ x, size_t n, int* __restrict__ flag) {
    for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < n; id += (size_t)gridDim.x * blockDim.x)
        if (!isfinite((double)x[id])) atomicExch(flag, 1);
}

}  // namespace les
