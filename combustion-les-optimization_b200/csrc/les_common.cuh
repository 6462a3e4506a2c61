// les_common.cuh -- shared device-side definitions for the solver-step kernels.
//
// Field layout: structure of arrays, one contiguous array of NX*NY*NZ values per field in
// the reference's [i][j][k] order (k fastest; les_combustion_solver.c:286), so host
// uploads/downloads are plain copies and a warp reads 32 consecutive k-cells.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace les {

constexpr int NSP = 5;
constexpr int C3H8 = 0, O2 = 1, N2 = 2, CO2 = 3, H2O = 4;   // :129-133
constexpr int NSTATE = 11;                                  // u v w T G rho Y0..Y4
constexpr int NACC = 10;                                    // rhou rhov rhow T G Y0..Y4
// thread-block shape of the per-cell passes: 32 consecutive k-cells x 8 j-rows
constexpr int BX = 32, BY = 8, NT = BX * BY;
// grid of the grid-stride monitor reductions (4 blocks per SM on 148 SMs)
constexpr int MON_BLOCKS = 592;

// Fixed constants of the reference (les_combustion_solver.c:136-188, 2164-2166, 234-245).
constexpr double R_UNIV = 8.314462;
constexpr double PATM = 101325.0;
constexpr double P_CONST = 101325.0;
constexpr double G_GRAVITY = -9.81;
constexpr double SMALL = 1e-10;
constexpr double FILTER_W = 50.0;
constexpr double TENO_CUT = 1.0e-6;
constexpr double FORCE_LIMIT = 500.0;
constexpr double RAMP_DIST = 0.03;
constexpr double SSR_A = 0.2340, SSR_B = 0.2187;

// A divisor with its reciprocal rounded to nearest.  x / c is evaluated as q = x*r followed
// by one fma correction q + (x - q*c)*r (Markstein's iteration), which returns the
// correctly rounded quotient for normal operands -- the same bits as IEEE division -- in
// 3 FP64 operations instead of a division sequence.
template <typename T>
struct DCT {
    T c, r;
};
using DC = DCT<double>;

// Model constants that vary between the members of an ensemble (the constants a Bayesian
// optimiser proposes: les_combustion_solver.c:257-262, :2834).
template <typename R>
struct ModelK {
    R cs_u, cs_b, cs_boost, accel_strength, accel_center, relax;
    DCT<R> d_w2;
};

// Constants that enter the per-cell arithmetic.  The FP32 form reads float copies of them
// (ConstsF, filled on the host), so no double-to-float conversion runs per cell; the FP64
// form reads the double originals.  X(name, dims) for values, XD(name, dims) for divisors.
#define LES_FCONSTS(X, XD)                                                                      \
    X(dx, ) X(dy, ) X(dz, ) X(dx4, ) X(inlet_center_z, )                                          \
    X(mwk, [NSP]) X(t_mid, [NSP]) X(nasa_high, [NSP][7]) X(nasa_low, [NSP][7])                  \
    X(eta, [NSP][4]) X(lam, [NSP][4]) X(dco, [NSP][NSP][4]) X(wpow, [NSP][NSP])                  \
    X(cs_u, ) X(cs_b, ) X(cs_boost, ) X(accel_strength, ) X(accel_center, ) X(relax, )           \
    X(s_l, ) X(ssr_cdF, ) X(ssr_exp, ) X(tau_sl, ) X(t_in, ) X(t_amb, ) X(t_burnt_span, )        \
    X(inletYk, [NSP]) X(ambientYk, [NSP]) X(cons_o2, ) X(prod_co2, ) X(prod_h2o, )               \
    X(u_in, ) X(noise_amp, )                                                                     \
    XD(d_dx, ) XD(d_dy, ) XD(d_dz, ) XD(d_2dx, ) XD(d_2dy, ) XD(d_2dz, ) XD(d_dxx, ) XD(d_dyy, ) \
    XD(d_dzz, ) XD(d_six, ) XD(d_filter, ) XD(d_sct2, ) XD(d_prt2, ) XD(d_ramp, ) XD(d_w2, )      \
    XD(d_tau_sl, ) XD(d_mwk, [NSP]) XD(d_wden, [NSP][NSP]) XD(d_tenows, [8])

struct ConstsF {
#define LES_DECL_F(name, dims) float name dims;
#define LES_DECL_FD(name, dims) DCT<float> name dims;
    LES_FCONSTS(LES_DECL_F, LES_DECL_FD)
#undef LES_DECL_F
#undef LES_DECL_FD
};

// Per-context constants, passed to every kernel by value (__grid_constant__), so reads go
// through the constant bank.  All derived values are computed on the host with the same
// operations the reference applies to its macros, so they are bit-identical.
struct Consts {
    int nx, ny, nz, flame_accel;
    int weno_step, dco_sym, n_inlet, pad0;
    double dx, dy, dz;
    double two_dx, two_dy, two_dz;      // 2.0*DX ...
    double dxx, dyy, dzz;               // DX*DX ...
    double dx4;                         // pow(DX, 4.0)
    double inlet_center_z;              // LZ/2.0
    double total_volume;                // serial sum of DX*DY*DZ over attr {1,2,3,5} (:2545)
    // species (:292-305)
    double mw[NSP], mwk[NSP];           // g/mol and mw/1000.0
    double t_mid[NSP];
    double nasa_high[NSP][7], nasa_low[NSP][7];
    double eta[NSP][4], lam[NSP][4], dco[NSP][NSP][4];
    int eta_zero[NSP], lam_zero[NSP], dco_zero[NSP][NSP];
    double wpow[NSP][NSP];              // pow(M_j/M_i, 0.25)           [i][j]
    double wden[NSP][NSP];              // sqrt(8.0)*sqrt(1.0 + M_i/M_j) [i][j]
    // divisors of the reference's divisions by constants, with reciprocals
    DC d_dx, d_dy, d_dz, d_2dx, d_2dy, d_2dz, d_dxx, d_dyy, d_dzz;
    DC d_six, d_filter, d_sct2, d_prt2, d_ramp, d_w2, d_tau_sl;
    DC d_mwk[NSP];
    DC d_wden[NSP][NSP];
    DC d_tenows[8];                     // TENO weight sums by cut-off pattern d0 + 2 d1 + 4 d2
    // model (:257-262, :2834, :2700-2704)
    double cs_u, cs_b, cs_boost;
    double accel_strength, accel_center, two_w2;   // two_w2 = 2.0*W*W
    double relax;
    double s_l, nu_u, d3;
    double ssr_cdF;                     // 10.0 * (nu_u / (S_L + 1e-10))
    double tau_sl;                      // tau * S_L
    double sc_t2, pr_t2;                // 2.0*Sc_t, 2.0*Pr_t
    double t_in, t_amb, t_burnt_span;   // T_u, T_amb, T_b - T_u
    double inletYk[NSP], ambientYk[NSP];
    double cons_o2, prod_co2, prod_h2o; // inletYk[C3H8] * stoich
    double u_in, noise_amp;             // INLET_VELOCITY, 0.10*INLET_VELOCITY
    double ti_rms;                      // INLET_VELOCITY * INLET_TURBULENCE_INTENSITY
    double ssr_exp;                     // 2.0 - D3, the SSR-SGS wrinkling exponent
    ConstsF f;                          // float copies for the FP32 form
};

// The constant set a kernel of field type R computes with: Consts itself for double, its
// float copies for float.
template <typename R>
struct KSel;
template <>
struct KSel<double> {
    using type = Consts;
    __host__ __device__ static const Consts& get(const Consts& C) { return C; }
};
template <>
struct KSel<float> {
    using type = ConstsF;
    __host__ __device__ static const ConstsF& get(const Consts& C) { return C.f; }
};
template <typename R>
__host__ __device__ __forceinline__ const typename KSel<R>::type& kc(const Consts& C) {
    return KSel<R>::get(C);
}

// The model constants of the cell's member: the launch's own constants, or the member table's.
template <typename R>
__host__ __device__ __forceinline__ ModelK<R> model_of(const Consts& C) {
    const auto& K = kc<R>(C);
    ModelK<R> m;
    m.cs_u = K.cs_u; m.cs_b = K.cs_b; m.cs_boost = K.cs_boost; m.accel_strength = K.accel_strength;
    m.accel_center = K.accel_center; m.relax = K.relax; m.d_w2 = K.d_w2;
    return m;
}


// Host: fill C.f from the double values.
inline void to_float(float& d, double s) { d = (float)s; }
inline void to_float(DCT<float>& d, const DC& s) { d.c = (float)s.c; d.r = (float)s.r; }
template <typename D, typename S, size_t N>
inline void to_float(D (&d)[N], const S (&s)[N]) {
    for (size_t q = 0; q < N; q++) to_float(d[q], s[q]);
}
inline void fill_float_consts(Consts& C) {
#define LES_CONV(name, dims) to_float(C.f.name, C.name);
    LES_FCONSTS(LES_CONV, LES_CONV)
#undef LES_CONV
}

// A batched launch (les_launch.cuh, batch_stages) steps several members of one grid shape in
// one launch; each block finds its member's buffers and model constants here.
struct Scalars;
struct MemberTab {
    long long delta;            // byte offset of this member's field arena from the first member's
    const uint8_t* attr;        // attribute map
    Scalars* S;                 // reduction results, dt, step counters
    double* part;               // per-block partials
    ModelK<double> md;          // model constants, FP64 form
    ModelK<float> mf;           // and FP32 form
};
// Kernel argument of the batched stage kernels: the member table and the z-extent of one
// member's grid of blocks (blockIdx.z = member * gz + block z within the member).
struct Batch {
    const MemberTab* mt;
    int gz;
};

template <typename R>
__device__ __forceinline__ const ModelK<R>& member_model(const MemberTab& e);
template <>
__device__ __forceinline__ const ModelK<double>& member_model<double>(const MemberTab& e) { return e.md; }
template <>
__device__ __forceinline__ const ModelK<float>& member_model<float>(const MemberTab& e) { return e.mf; }

template <typename T>
__device__ __forceinline__ T* shifted(T* p, long long d) {
    return (T*)((char*)p + d);
}

// Reduction results written by the kernels' last-block epilogues.
struct Scalars {
    double rho_avg;                     // <rho_f> of the current stage (:2550)
    double umax, numax, alphamax;       // dt inputs (:1472-1485, :4401-4408)
    double mon[6];                      // monitor reductions
    double sem[6];                      // SEM sums (debug)
    unsigned int counter[4];            // last-block counters (0: filter, 1: bc, 2: aux, 3: monitor)
    int nonfinite;                      // bit 1: rand() jump table too short (device loop)
    double dt;                          // dt of the step being computed
    double umax_used;                   // |u|max that produced dt (after the inlet fallback)
    int t_loop;                         // reference time-step index of the step being computed
    int run_step;                       // index of the step within the current device-loop run
    int avg_steps;                      // steps summed into the time averages (time_avg_steps)
    int pad1;
};

// Running sums of update_time_averages (les_combustion_solver.c:3166-3191), in the order of
// stats_backup.bin (:3740-3754): u v w uu vv ww uv uw vw G.
constexpr int NAVG = 10;
struct AvgBuf {
    double* p[NAVG];
};

// rand() stream state of the device-resident loop (les_devloop.cuh).
struct LoopState {
    unsigned int win[31];     // x[n-31 .. n-1] of the rand() stream, oldest first
    int n_rec;                // vortices recycled in the last step (diagnostic)
    int draws;                // rand() draws of the last step
    unsigned long long total_draws;
};

__device__ __forceinline__ size_t cid(int i, int j, int k, int ny, int nz) {
    return ((size_t)i * (size_t)ny + (size_t)j) * (size_t)nz + (size_t)k;
}

__device__ __forceinline__ double cdv(double x, const DC& d) {
    double q = x * d.r;
    double e = fma(-q, d.c, x);
    return fma(e, d.r, q);
}
__device__ __forceinline__ float cdv(float x, const DCT<float>& d) { return x * d.r; }

// Arithmetic of the per-cell formulas.  The FP64 form uses IEEE double operations, as the
// reference does; the FP32 form uses the hardware approximations (MUFU ex2/lg2/rcp/sqrt,
// ~2 ulp), which its stated error budget covers.
__device__ __forceinline__ double qdiv(double a, double b) { return a / b; }
#ifdef LES_FP32_IEEE_MATH
// build option: the FP32 form with IEEE float operations (for error attribution)
__device__ __forceinline__ float qdiv(float a, float b) { return a / b; }
__device__ __forceinline__ float qexp(float x) { return expf(x); }
__device__ __forceinline__ float qlog(float x) { return logf(x); }
__device__ __forceinline__ float qpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ float qsqrt(float x) { return sqrtf(x); }
#else
__device__ __forceinline__ float qdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float qexp(float x) { return __expf(x); }
__device__ __forceinline__ float qlog(float x) { return __logf(x); }
__device__ __forceinline__ float qpow(float a, float b) { return __powf(a, b); }
__device__ __forceinline__ float qsqrt(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#endif
__device__ __forceinline__ double qexp(double x) { return exp(x); }
__device__ __forceinline__ double qlog(double x) { return log(x); }
__device__ __forceinline__ double qpow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ double qsqrt(double x) { return sqrt(x); }

// a / b for several numerators sharing one denominator b, given y = 1/b from one IEEE
// division: q = a*y corrected once with an fma (Markstein), which is the correctly rounded
// quotient for normal operands -- checked against IEEE division on the GPU over 2^31 random
// pairs (lesgpu_selfcheck_division).  A denominator that is zero, subnormal or not finite
// takes the IEEE division.
__device__ __forceinline__ double mdiv(double a, double b, double y) {
    const double ab = fabs(b);
    if (!(ab >= 2.2250738585072014e-308 && ab <= 1.7976931348623157e308)) return a / b;
    const double q = a * y;
    return fma(fma(-q, b, a), y, q);
}
__device__ __forceinline__ float mdiv(float a, float b, float y) { return a * y; }

// Division of FP64 state quantities (RK update, EOS, renormalisation).  The FP64 form divides
// in IEEE double, as the reference does.  The FP32 form keeps its state in FP64 only so that
// small increments survive; there a float reciprocal refined by one Newton step and one
// quotient correction in double (relative error ~1e-15) replaces the division sequence.
template <typename Form>
__device__ __forceinline__ double sdiv(double a, double b);
template <>
__device__ __forceinline__ double sdiv<double>(double a, double b) { return a / b; }
template <>
__device__ __forceinline__ double sdiv<float>(double a, double b) {
    double y = (double)__frcp_rn((float)b);
    y = fma(y, fma(-b, y, 1.0), y);
    const double q = a * y;
    return fma(fma(-q, b, a), y, q);
}

// x^3 and x^4 rounded once: glibc pow() returns the correctly rounded power for these
// arguments, while a plain product rounds twice.  The exact square is split with fma,
// the rest is carried as a double-double and rounded once at the end.
__device__ __forceinline__ double pow3_rn(double x) {
    double p = x * x;
    double e = fma(x, x, -p);
    double h = p * x;
    double l = fma(p, x, -h);
    l = fma(e, x, l);
    return h + l;
}
__device__ __forceinline__ double pow4_rn(double x) {
    double p = x * x;
    double e = fma(x, x, -p);
    double h = p * p;
    double l = fma(p, p, -h);
    l = fma(2.0 * p, e, l);
    return h + l;
}
__device__ __forceinline__ float pow3_rn(float x) { return x * x * x; }
__device__ __forceinline__ float pow4_rn(float x) { float p = x * x; return p * p; }

// Deterministic block reductions (fixed shuffle tree, fixed warp order).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh, int tid) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < NT / 32) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;   // valid in thread 0
}
template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh, int tid) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = -1.0e300;
    if (wid == 0) {
        r = (lane < NT / 32) ? sh[lane] : -1.0e300;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}
template <int NT>
__device__ __forceinline__ double block_min(double v, double* sh, int tid) {
    return -block_max<NT>(-v, sh, tid);
}

}  // namespace les
