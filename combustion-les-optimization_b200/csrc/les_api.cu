// les_api.cu -- implementation of the C ABI in include/les_gpu.h.
//
// Owns the device arena of one solver context, the host-side derivation of the constant
// table (with the same operations the reference applies to its macros and loaded species
// data), uploads/downloads in the reference's [i][j][k] order, and the stream-ordered step.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <cstring>
#include <vector>

#include "les_ctx.h"
#include "les_gpu.h"

using les::DevCtx;

struct lesgpu_ctx {
    DevCtx d;
    lesgpu_config cfg;
    lesgpu_species sp;
};

namespace {

int fail(lesgpu_ctx* c, int code, const std::string& msg) {
    if (c) c->d.err = msg;
    return code;
}

int cuda_fail(lesgpu_ctx* c, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    if (c) c->d.err = m;
    return LESGPU_ECUDA;
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);   \
    } while (0)

#define CKC(c, call)                                               \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail((c), e_, #call);   \
    } while (0)

bool all_zero4(const double* c) { return c[0] == 0.0 && c[1] == 0.0 && c[2] == 0.0 && c[3] == 0.0; }

// Constant table: grid spacings and the species/model constants in the form the kernels use.
void build_consts(const lesgpu_config& g, const lesgpu_species& sp, les::Consts& C) {
    memset(&C, 0, sizeof(C));
    C.nx = g.nx; C.ny = g.ny; C.nz = g.nz;
    C.flame_accel = g.flame_accel;
    C.weno_step = g.weno_transition_step;
    C.dx = g.lx / (double)g.nx;          // DX (:104-106)
    C.dy = g.ly / (double)g.ny;
    C.dz = g.lz / (double)g.nz;
    C.two_dx = 2.0 * C.dx; C.two_dy = 2.0 * C.dy; C.two_dz = 2.0 * C.dz;
    C.dxx = C.dx * C.dx; C.dyy = C.dy * C.dy; C.dzz = C.dz * C.dz;
    C.dx4 = pow(C.dx, 4.0);
    C.inlet_center_z = g.lz / 2.0;       // INLET_CENTER_Z (:110)
    for (int s = 0; s < les::NSP; s++) {
        C.mw[s] = sp.mw[s];
        C.mwk[s] = sp.mw[s] / 1000.0;
        C.t_mid[s] = sp.t_mid[s];
        for (int q = 0; q < 7; q++) { C.nasa_high[s][q] = sp.nasa_high[s][q]; C.nasa_low[s][q] = sp.nasa_low[s][q]; }
        for (int q = 0; q < 4; q++) { C.eta[s][q] = sp.eta[s][q]; C.lam[s][q] = sp.lambda[s][q]; }
        C.eta_zero[s] = all_zero4(sp.eta[s]);
        C.lam_zero[s] = all_zero4(sp.lambda[s]);
    }
    int sym = 1;
    for (int a = 0; a < les::NSP; a++)
        for (int b = 0; b < les::NSP; b++) {
            for (int q = 0; q < 4; q++) C.dco[a][b][q] = sp.dcoef[a][b][q];
            C.dco_zero[a][b] = all_zero4(sp.dcoef[a][b]);
            if (a != b && memcmp(sp.dcoef[a][b], sp.dcoef[b][a], 4 * sizeof(double)) != 0) sym = 0;
            // Wilke / Wassiljew pair constants (:1540, :1855), evaluated with the host libm
            // exactly as the reference evaluates them per cell.
            C.wpow[a][b] = pow(sp.mw[b] / sp.mw[a], 0.25);
            C.wden[a][b] = sqrt(8.0) * sqrt(1.0 + sp.mw[a] / sp.mw[b]);
        }
    C.dco_sym = sym;
    C.cs_u = g.cs_unburned; C.cs_b = g.cs_burnt; C.cs_boost = g.cs_flame_boost;
    C.accel_strength = g.accel_strength;
    C.accel_center = g.accel_center;
    C.two_w2 = 2.0 * g.accel_width * g.accel_width;
    C.relax = g.relax;
    C.s_l = g.s_l; C.nu_u = g.nu_unburnt; C.d3 = g.d3;
    double dF = g.nu_unburnt / (g.s_l + 1e-10);                         // :1941
    C.ssr_cdF = 10.0 * dF;                                              // :1943
    double tau = (g.rho_unburnt_approx / g.rho_burnt_approx) - 1.0;     // :2703
    C.tau_sl = tau * g.s_l;
    C.sc_t2 = 2.0 * g.sc_t; C.pr_t2 = 2.0 * g.pr_t;
    C.t_in = g.inlet_temperature; C.t_amb = g.ambient_temperature;
    C.t_burnt_span = g.burnt_gas_temperature - g.inlet_temperature;
    // inlet composition and stoichiometry (:4101-4120)
    const double phi = g.equivalence_ratio;
    double m_f = 1.0, m_o2 = 5.0 / phi, m_n2 = m_o2 * 3.76;
    double mass_total = m_f * sp.mw[0] + m_o2 * sp.mw[1] + m_n2 * sp.mw[2];
    C.inletYk[0] = (m_f * sp.mw[0]) / mass_total;
    C.inletYk[1] = (m_o2 * sp.mw[1]) / mass_total;
    C.inletYk[2] = (m_n2 * sp.mw[2]) / mass_total;
    C.inletYk[3] = 0.0; C.inletYk[4] = 0.0;
    C.ambientYk[0] = 0.0; C.ambientYk[1] = 0.232; C.ambientYk[2] = 0.768; C.ambientYk[3] = 0.0; C.ambientYk[4] = 0.0;
    double st_o2 = (5.0 * sp.mw[1]) / sp.mw[0];
    double st_co2 = (3.0 * sp.mw[3]) / sp.mw[0];
    double st_h2o = (4.0 * sp.mw[4]) / sp.mw[0];
    C.cons_o2 = C.inletYk[0] * st_o2;
    C.prod_co2 = C.inletYk[0] * st_co2;
    C.prod_h2o = C.inletYk[0] * st_h2o;
    C.u_in = g.inlet_velocity;
    C.noise_amp = 0.10 * g.inlet_velocity;                              // :2987
    C.ti_rms = g.inlet_velocity * g.turbulence_intensity;              // :1050
    auto dc = [](double c) { les::DC d; d.c = c; d.r = 1.0 / c; return d; };
    C.d_dx = dc(C.dx); C.d_dy = dc(C.dy); C.d_dz = dc(C.dz);
    C.d_2dx = dc(C.two_dx); C.d_2dy = dc(C.two_dy); C.d_2dz = dc(C.two_dz);
    C.d_dxx = dc(C.dxx); C.d_dyy = dc(C.dyy); C.d_dzz = dc(C.dzz);
    C.d_six = dc(6.0);
    C.d_filter = dc(6.0 + 50.0);
    C.d_sct2 = dc(C.sc_t2); C.d_prt2 = dc(C.pr_t2);
    C.d_ramp = dc(0.03);
    C.d_w2 = dc(C.two_w2);
    C.d_tau_sl = dc(C.tau_sl > 0 ? C.tau_sl : 1.0);
    for (int a = 0; a < les::NSP; a++) {
        C.d_mwk[a] = dc(C.mwk[a]);
        for (int b = 0; b < les::NSP; b++) C.d_wden[a][b] = dc(C.wden[a][b]);
    }
    // TENO weight sums w0 + w1 + w2 (w = d * {0.1, 0.6, 0.3}) for each cut-off pattern, with
    // the kernel's operation order (teno5_reconstruct, :2224-2231)
    for (int q = 0; q < 8; q++) {
        const int d0 = q & 1, d1 = (q >> 1) & 1, d2 = (q >> 2) & 1;
        const double w0 = (double)d0 * 0.1, w1 = (double)d1 * 0.6, w2 = (double)d2 * 0.3;
        const double ws = w0 + w1 + w2;
        C.d_tenows[q] = dc(q == 0 ? 1.0 : ws);
    }
    C.ssr_exp = 2.0 - C.d3;                                             // :1946
    les::fill_float_consts(C);
}

unsigned char* read_record(FILE* fp, int* len) {
    int n;
    if (fread(&n, sizeof(int), 1, fp) != 1 || n < 0 || n > (1 << 26)) return nullptr;
    unsigned char* b = (unsigned char*)malloc((size_t)n + 1);
    if (!b) return nullptr;
    if (fread(b, 1, (size_t)n, fp) != (size_t)n) { free(b); return nullptr; }
    int e;
    if (fread(&e, sizeof(int), 1, fp) != 1 || e != n) { free(b); return nullptr; }
    if (len) *len = n;
    return b;
}

// 11 state fields (Phi_n, always 8-byte) and 48 fields of the form's element size.
constexpr size_t kStateFields = 11;
size_t fields_for_precision() { return 59; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    // looked up once; the initialisation of a function-local static is thread-safe, so
    // contexts may be created from several host threads
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (EncodeTiledFn)p;
        return nullptr;
    }();
    return fn;
}

// Tensor maps of the scalar pass's staged fields (filtered Y_0..Y_4, T, then nu_t): 3-D
// (k, j, i) views of the arena fields; boxes of (BW x BH x 1) with BH = 12 for the fields and
// 10 for nu_t; zero fill outside the grid.  Built only when a row (NZ values) is a multiple
// of 16 bytes, as tensor copies require.
bool make_tma_maps(DevCtx& d) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc || (d.nz * d.esz) % 16 != 0) return false;
    const bool f64 = d.esz == 8;
    const cuuint64_t dims[3] = {(cuuint64_t)d.nz, (cuuint64_t)d.ny, (cuuint64_t)d.nx};
    const cuuint64_t strides[2] = {(cuuint64_t)d.nz * d.esz, (cuuint64_t)d.ny * d.nz * d.esz};
    const cuuint32_t bw = f64 ? 36 : 40;
    const cuuint32_t boxf[3] = {bw, 12, 1}, boxn[3] = {bw, 10, 1}, es[3] = {1, 1, 1};
    const CUtensorMapDataType dt = f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUtensorMap* m = reinterpret_cast<CUtensorMap*>(d.tma_maps);
    void* src[7] = {d.F[6], d.F[7], d.F[8], d.F[9], d.F[10], d.F[3], d.nu_t};
    for (int q = 0; q < 7; q++) {
        CUresult r = enc(&m[q], dt, 3, src[q], dims, strides, q < 6 ? boxf : boxn, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    return true;
}

void free_loop(DevCtx& d);

}  // namespace

namespace les {

int tmark_begin(DevCtx& c, int cls) {
    if (!c.timing) return -1;
    const int slot = c.ev_used;
    if (2 * (slot + 1) > (int)c.ev_pool.size()) {
        for (int q = 0; q < 2; q++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            c.ev_pool.push_back(e);
        }
    }
    if ((int)c.ev_cls.size() <= slot) c.ev_cls.resize(slot + 1);
    c.ev_cls[slot] = cls;
    cudaEventRecord(c.ev_pool[2 * slot], c.stream);
    c.ev_used++;
    return slot;
}

void tmark_end(DevCtx& c, int slot) {
    if (slot < 0) return;
    cudaEventRecord(c.ev_pool[2 * slot + 1], c.stream);
}

void tmark_flush(DevCtx& c) {
    if (!c.timing || c.ev_used == 0) return;
    cudaStreamSynchronize(c.stream);
    for (int q = 0; q < c.ev_used; q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c.ev_pool[2 * q], c.ev_pool[2 * q + 1]) == cudaSuccess) {
            c.kms[c.ev_cls[q]] += ms;
            c.kcount[c.ev_cls[q]] += 1;
        }
    }
    c.ev_used = 0;
}

}  // namespace les

// ---------------------------------------------------------------- device-resident loop helpers

namespace {

// Rows J[m] (m = 0..rows-1) of the rand() jump-ahead: x[n+m] = sum_j J[m][j] * x[n-31+j]
// (mod 2^32), from x[t] = x[t-31] + x[t-3] applied to coefficient vectors.
std::vector<unsigned int> jump_table(int rows) {
    std::vector<unsigned int> J((size_t)rows * 31, 0u);
    auto row = [&](int t) -> const unsigned int* { return &J[(size_t)t * 31]; };
    unsigned int unit[31][31];
    for (int a = 0; a < 31; a++)
        for (int b = 0; b < 31; b++) unit[a][b] = (a == b) ? 1u : 0u;
    for (int t = 0; t < rows; t++) {
        const unsigned int* a = (t - 31 < 0) ? unit[t] : row(t - 31);         // x[t-31]
        const unsigned int* b = (t - 3 < 0) ? unit[t + 28] : row(t - 3);     // x[t-3]
        unsigned int* o = &J[(size_t)t * 31];
        for (int j = 0; j < 31; j++) o[j] = a[j] + b[j];
    }
    return J;
}

// Device buffers of a context come from the device's stream-ordered pool, allocated and freed
// on the context's stream.  cudaFree waits for the whole device, so a serving loop that creates
// and retires solves while others step would stall every stream at each retirement.  A buffer
// is used on another stream (or by a synchronous copy) only after the context's stream has
// been synchronised once since its allocation.
template <typename T>
cudaError_t dalloc(DevCtx& d, T** p, size_t bytes) {
    return cudaMallocAsync((void**)p, bytes, d.stream);
}
inline void dfree(DevCtx& d, void* p) {
    if (p) cudaFreeAsync(p, d.stream);
}

void free_loop(DevCtx& d) {
    if (d.graph) { cudaGraphExecDestroy(d.graph); d.graph = nullptr; }
    d.graph_ok = false;
    void* bufs[] = {d.J, d.dL, d.loop_st, d.hist_probe, d.hist_dt, d.hist_umax, d.hist_mon};
    for (void* b : bufs) dfree(d, b);
    d.J = nullptr; d.dL = nullptr; d.loop_st = nullptr;
    d.hist_probe = d.hist_dt = d.hist_umax = d.hist_mon = nullptr;
    d.loop_ready = false;
}

int alloc_history(lesgpu_ctx* ctx, const int* st, int n, int kline, int cap) {
    DevCtx& d = ctx->d;
    if (d.graph) { cudaGraphExecDestroy(d.graph); d.graph = nullptr; }
    d.graph_ok = false;
    void* bufs[] = {d.loop_st, d.hist_probe, d.hist_dt, d.hist_umax, d.hist_mon};
    for (void* b : bufs) dfree(d, b);
    d.loop_st = nullptr; d.hist_probe = d.hist_dt = d.hist_umax = d.hist_mon = nullptr;
    d.loop_nst = n; d.loop_kline = kline; d.loop_cap = cap;
    CK(dalloc(d, &d.loop_st, (n > 0 ? n : 1) * sizeof(int)));
    CK(dalloc(d, &d.hist_probe, (size_t)cap * (n > 0 ? n : 1) * d.ny * 6 * sizeof(double)));
    CK(dalloc(d, &d.hist_dt, (size_t)cap * sizeof(double)));
    CK(dalloc(d, &d.hist_umax, (size_t)cap * sizeof(double)));
    CK(dalloc(d, &d.hist_mon, (size_t)cap * 6 * sizeof(double)));
    CK(cudaStreamSynchronize(d.stream));
    if (n > 0) CK(cudaMemcpy(d.loop_st, st, n * sizeof(int), cudaMemcpyHostToDevice));
    return LESGPU_OK;
}

}  // namespace

extern "C" {

int lesgpu_load_species(const char* chem_path, const char* tran_path, lesgpu_species* out) {
    if (!chem_path || !tran_path || !out) return LESGPU_EINVAL;
    memset(out, 0, sizeof(*out));
    FILE* fp = fopen(chem_path, "rb");
    if (!fp) return LESGPU_EIO;
    int len = 0, mm = 0, kk = 0;
    unsigned char* b = read_record(fp, &len);
    if (!b) { fclose(fp); return LESGPU_EIO; }
    free(b);
    b = read_record(fp, &len);
    if (!b || len < 20) { free(b); fclose(fp); return LESGPU_EIO; }
    memcpy(&mm, b + 12, 4); memcpy(&kk, b + 16, 4);
    free(b);
    if (kk != LESGPU_NSP || mm < 0 || mm > 64) { fclose(fp); return LESGPU_EIO; }
    b = read_record(fp, &len);
    if (!b) { fclose(fp); return LESGPU_EIO; }
    free(b);
    b = read_record(fp, &len);
    size_t per = 16 + 4 * (size_t)mm + 8 + 8 + 4 + 24 + 2 * 56;
    if (!b || (size_t)len < 8 + per * LESGPU_NSP) { free(b); fclose(fp); return LESGPU_EIO; }
    for (int i = 0; i < LESGPU_NSP; i++) {
        size_t base = 8 + (size_t)i * per;
        size_t mwo = base + 16 + 4 * (size_t)mm + 8;
        size_t tmo = mwo + 8 + 4 + 16;
        memcpy(&out->mw[i], b + mwo, 8);
        memcpy(&out->t_mid[i], b + tmo, 8);
        memcpy(out->nasa_high[i], b + tmo + 8, 56);
        memcpy(out->nasa_low[i], b + tmo + 8 + 56, 56);
    }
    free(b);
    fclose(fp);
    fp = fopen(tran_path, "rb");
    if (!fp) return LESGPU_EIO;
    for (int r = 0; r < 4; r++) {
        b = read_record(fp, &len);
        if (!b) { fclose(fp); return LESGPU_EIO; }
        free(b);
    }
    b = read_record(fp, &len);
    if (!b || len < 32 * LESGPU_NSP) { free(b); fclose(fp); return LESGPU_EIO; }
    for (int i = 0; i < LESGPU_NSP; i++) memcpy(out->lambda[i], b + 32 * i, 32);
    free(b);
    b = read_record(fp, &len);
    if (!b || len < 32 * LESGPU_NSP) { free(b); fclose(fp); return LESGPU_EIO; }
    for (int i = 0; i < LESGPU_NSP; i++) memcpy(out->eta[i], b + 32 * i, 32);
    free(b);
    b = read_record(fp, &len);
    if (!b || len < 32 * LESGPU_NSP * LESGPU_NSP) { free(b); fclose(fp); return LESGPU_EIO; }
    for (int i = 0; i < LESGPU_NSP; i++)
        for (int j = 0; j < LESGPU_NSP; j++) memcpy(out->dcoef[i][j], b + 32 * (i * LESGPU_NSP + j), 32);
    free(b);
    fclose(fp);
    for (int i = 0; i < LESGPU_NSP; i++)
        if (!(out->mw[i] > 0.0)) return LESGPU_EIO;
    return LESGPU_OK;
}

size_t lesgpu_bytes_for_grid(int nx, int ny, int nz, int precision) {
    size_t n = (size_t)nx * ny * nz;
    size_t esz = (precision == LESGPU_FP32) ? 4 : 8;
    size_t nb = les::max_cell_blocks(nx, ny, nz);
    if (nb < (size_t)les::MON_BLOCKS) nb = les::MON_BLOCKS;
    size_t planes = (size_t)ny * nz;
    return kStateFields * n * 8 + (fields_for_precision() - kStateFields) * n * esz + n +   // fields + attribute
           (6 * nb + 64) * sizeof(double) +                       // reduction partials
           planes * (3 * sizeof(double) + 2 * sizeof(int)) +      // SEM planes + inlet maps
           3 * planes * sizeof(double) + sizeof(les::Consts) + sizeof(les::Scalars) + (1 << 16);
}

int lesgpu_create(const lesgpu_config* cfg, const lesgpu_species* sp, lesgpu_ctx** out) {
    if (!cfg || !sp || !out) return LESGPU_EINVAL;
    *out = nullptr;
    if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 4 || cfg->num_vortices < 0) return LESGPU_EINVAL;
    if (cfg->precision != LESGPU_FP64 && cfg->precision != LESGPU_FP32) return LESGPU_EINVAL;
    if ((size_t)cfg->ny * cfg->nz > (size_t)1 << 30 || (size_t)cfg->nx > 65535) return LESGPU_EINVAL;
    lesgpu_ctx* ctx = new (std::nothrow) lesgpu_ctx();
    if (!ctx) return LESGPU_ENOMEM;
    ctx->cfg = *cfg;
    ctx->sp = *sp;
    DevCtx& d = ctx->d;
    d.nx = cfg->nx; d.ny = cfg->ny; d.nz = cfg->nz;
    d.n = (size_t)cfg->nx * cfg->ny * cfg->nz;
    d.precision = cfg->precision;
    d.esz = (cfg->precision == LESGPU_FP32) ? 4 : 8;
    build_consts(*cfg, *sp, d.hC);
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) { int r = cuda_fail(ctx, e, "cudaSetDevice"); delete ctx; return r; }
    e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { int r = cuda_fail(ctx, e, "cudaStreamCreate"); delete ctx; return r; }
    e = cudaStreamCreateWithFlags(&d.side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) { int r = cuda_fail(ctx, e, "side stream"); lesgpu_destroy(ctx); return r; }
    // one arena for all per-cell fields; each field starts on a 256-byte boundary.  The
    // state Phi_n is FP64 in both forms (the RK update runs in FP64); the rest is FP32 in
    // the precision form.
    const size_t fb = ((d.n * d.esz + 255) / 256) * 256;
    const size_t fb8 = ((d.n * 8 + 255) / 256) * 256;
    const size_t nf = fields_for_precision();
    d.arena_bytes = kStateFields * fb8 + (nf - kStateFields) * fb;
    e = dalloc(d, &d.arena_raw, d.arena_bytes + 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        d.arena_raw = nullptr;
        ctx->d.err = "device arena allocation failed";
        lesgpu_destroy(ctx);
        return LESGPU_ENOMEM;
    }
    d.arena = (void*)(((uintptr_t)d.arena_raw + 255) & ~(uintptr_t)255);
    cudaMemsetAsync(d.arena, 0, d.arena_bytes, d.stream);
    char* p = (char*)d.arena;
    auto take = [&]() { void* r = p; p += fb; return r; };
    for (int q = 0; q < les::NSTATE; q++) { d.S[q] = p; p += fb8; }
    for (int q = 0; q < les::NSTATE; q++) d.St[q] = take();
    for (int q = 0; q < les::NSTATE; q++) d.F[q] = take();
    d.mu_mix = take(); d.nu = take();
    for (int s = 0; s < les::NSP; s++) d.D[s] = take();
    d.aT = take(); d.nu_t = take(); d.S_mag = take(); d.ST = take(); d.mu_eff = take();
    for (int q = 0; q < les::NACC; q++) d.acc[q] = take();
    for (int q = 0; q < 4; q++) d.kflow[q] = take();
    // per-block partials: 3 per block of the per-cell grid (filter pass, any tile shape) and
    // 6 per block of the monitor grid
    size_t nb = les::max_cell_blocks(d.nx, d.ny, d.nz);
    d.part_len = 6 * (nb > (size_t)les::MON_BLOCKS ? nb : (size_t)les::MON_BLOCKS) + 64;
    size_t planes = (size_t)d.ny * d.nz;
    bool ok = dalloc(d, &d.attr, d.n) == cudaSuccess &&
              dalloc(d, &d.dC, sizeof(les::Consts)) == cudaSuccess &&
              dalloc(d, &d.dS, sizeof(les::Scalars)) == cudaSuccess &&
              dalloc(d, &d.part, d.part_len * sizeof(double)) == cudaSuccess &&
              dalloc(d, &d.plane, 3 * planes * sizeof(double)) == cudaSuccess &&
              dalloc(d, &d.noise, 3 * planes * sizeof(double)) == cudaSuccess &&
              dalloc(d, &d.inlet_list, planes * sizeof(int)) == cudaSuccess &&
              dalloc(d, &d.inlet_pos, planes * sizeof(int)) == cudaSuccess &&
              dalloc(d, &d.flag, sizeof(int)) == cudaSuccess;
    if (!ok) { cudaGetLastError(); ctx->d.err = "device allocation failed"; lesgpu_destroy(ctx); return LESGPU_ENOMEM; }
    d.nv_cap = cfg->num_vortices > 0 ? cfg->num_vortices : 1;
    if (dalloc(d, &d.vort, (size_t)d.nv_cap * 7 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        d.vort = nullptr;
        ctx->d.err = "vortex buffer allocation failed";
        lesgpu_destroy(ctx);
        return LESGPU_ENOMEM;
    }
    // the pinned staging buffer of the host-driven inflow is allocated on first use
    static_assert(sizeof(les::TmaMapsStorage) == sizeof(d.tma_maps), "tensor map storage");
    if (make_tma_maps(d)) {
        cudaError_t pe = (d.precision == LESGPU_FP64) ? les::prepare_tma_f64() : les::prepare_tma_f32();
        d.tma_ok = (pe == cudaSuccess);
        if (pe != cudaSuccess) cudaGetLastError();
    }
    cudaMemsetAsync(d.dS, 0, sizeof(les::Scalars), d.stream);
    cudaMemsetAsync(d.attr, 0, d.n, d.stream);
    cudaMemsetAsync(d.plane, 0, 3 * planes * sizeof(double), d.stream);
    cudaMemsetAsync(d.noise, 0, 3 * planes * sizeof(double), d.stream);
    cudaMemcpyAsync(d.dC, &d.hC, sizeof(les::Consts), cudaMemcpyHostToDevice, d.stream);
    e = cudaStreamSynchronize(d.stream);
    if (e != cudaSuccess) { int r = cuda_fail(ctx, e, "create"); lesgpu_destroy(ctx); return r; }
    d.total_bytes = d.arena_bytes + d.n + d.part_len * sizeof(double) + 3 * planes * sizeof(double) * 2 +
                    2 * planes * sizeof(int) + (size_t)d.nv_cap * 7 * sizeof(double) + sizeof(les::Consts) +
                    sizeof(les::Scalars);
    *out = ctx;
    return LESGPU_OK;
}

void lesgpu_destroy(lesgpu_ctx* ctx) {
    if (!ctx) return;
    DevCtx& d = ctx->d;
    if (d.stream) cudaStreamSynchronize(d.stream);
    if (d.side) cudaStreamSynchronize(d.side);
    // every buffer was allocated on d.stream, which exists whenever one of them does
    void* bufs[] = {d.arena_raw, d.attr, d.dC, d.dS, d.part, d.plane, d.noise, d.vort, d.inlet_list, d.inlet_pos,
                    d.probe_st, d.probe_out, d.flag, d.dbg_cp, d.dbg_lam, d.dbg_alpha, d.avg, d.grad_g,
                    d.ps_edges, d.ps_sums, d.ps_yflame, d.ps_rowbin};
    for (void* b : bufs) dfree(d, b);
    for (int q = 0; q < les::NACC; q++) dfree(d, d.kd[q]);
    if (d.h_pinned) cudaFreeHost(d.h_pinned);
    for (cudaEvent_t e : d.ev_pool) cudaEventDestroy(e);
    for (int q = 0; q < 16; q++)
        if (d.marks[q]) cudaEventDestroy(d.marks[q]);
    free_loop(d);
    if (d.side) { cudaStreamSynchronize(d.side); cudaStreamDestroy(d.side); }
    if (d.ev_fork) cudaEventDestroy(d.ev_fork);
    if (d.ev_join) cudaEventDestroy(d.ev_join);
    if (d.stream) cudaStreamDestroy(d.stream);
    delete ctx;
}

const char* lesgpu_last_error(const lesgpu_ctx* ctx) { return ctx ? ctx->d.err.c_str() : "null context"; }

size_t lesgpu_device_bytes(const lesgpu_ctx* ctx) { return ctx ? ctx->d.total_bytes : 0; }

static void drop_graph(DevCtx& d);

int lesgpu_upload_attribute(lesgpu_ctx* ctx, const int* attr) {
    if (!ctx || !attr) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    std::vector<uint8_t> a8(d.n);
    for (size_t q = 0; q < d.n; q++) {
        if (attr[q] < 0 || attr[q] > 6) return fail(ctx, LESGPU_EINVAL, "attribute codes must be in 0..6");
        a8[q] = (uint8_t)attr[q];
    }
    // inlet cells of the i = 0 face in (j, k) order (:4366-4367)
    const size_t planes = (size_t)d.ny * d.nz;
    std::vector<int> list, pos(planes, -1);
    for (int j = 0; j < d.ny; j++)
        for (int k = 0; k < d.nz; k++) {
            size_t p = (size_t)j * d.nz + k;
            if (attr[p] == 1) { pos[p] = (int)list.size(); list.push_back((int)p); }
        }
    // total fluid volume of the <rho_f> average, summed serially as the reference does (:2545)
    const double dv = d.hC.dx * d.hC.dy * d.hC.dz;
    double tv = 0.0;
    for (size_t q = 0; q < d.n; q++) {
        int v = attr[q];
        if (v == 1 || v == 2 || v == 3 || v == 5) tv += dv;
    }
    d.hC.total_volume = tv;
    d.hC.n_inlet = (int)list.size();
    d.n_inlet = (int)list.size();
    d.h_inlet = list;
    CK(cudaMemcpyAsync(d.attr, a8.data(), d.n, cudaMemcpyHostToDevice, d.stream));
    if (!list.empty())
        CK(cudaMemcpyAsync(d.inlet_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, d.stream));
    CK(cudaMemcpyAsync(d.inlet_pos, pos.data(), planes * sizeof(int), cudaMemcpyHostToDevice, d.stream));
    CK(cudaMemcpyAsync(d.dC, &d.hC, sizeof(les::Consts), cudaMemcpyHostToDevice, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    d.have_attr = true;
    // a captured step holds the constants (total volume, inlet count) by value
    drop_graph(d);
    return LESGPU_OK;
}

static int copy_field_in(lesgpu_ctx* ctx, void* dst, const double* src, size_t esz) {
    DevCtx& d = ctx->d;
    if (esz == 8) {
        CK(cudaMemcpyAsync(dst, src, d.n * 8, cudaMemcpyHostToDevice, d.stream));
        CK(cudaStreamSynchronize(d.stream));
        return LESGPU_OK;
    }
    std::vector<float> tmp(d.n);
    for (size_t q = 0; q < d.n; q++) tmp[q] = (float)src[q];
    CK(cudaMemcpyAsync(dst, tmp.data(), d.n * 4, cudaMemcpyHostToDevice, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    return LESGPU_OK;
}

static int copy_field_out(lesgpu_ctx* ctx, double* dst, const void* src, size_t esz) {
    DevCtx& d = ctx->d;
    if (esz == 8) {
        CK(cudaMemcpyAsync(dst, src, d.n * 8, cudaMemcpyDeviceToHost, d.stream));
        CK(cudaStreamSynchronize(d.stream));
        return LESGPU_OK;
    }
    std::vector<float> tmp(d.n);
    CK(cudaMemcpyAsync(tmp.data(), src, d.n * 4, cudaMemcpyDeviceToHost, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    for (size_t q = 0; q < d.n; q++) dst[q] = (double)tmp[q];
    return LESGPU_OK;
}

int lesgpu_upload_state(lesgpu_ctx* ctx, const double* const* fields, int nfields) {
    if (!ctx || !fields || nfields < 1 || nfields > LESGPU_NSTATE) return LESGPU_EINVAL;
    if (!ctx->d.have_attr) return fail(ctx, LESGPU_ESTATE, "upload the attribute map before the state");
    for (int q = 0; q < nfields; q++) {
        if (!fields[q]) return LESGPU_EINVAL;
        int r = copy_field_in(ctx, ctx->d.S[q], fields[q], 8);
        if (r) return r;
    }
    DevCtx& d = ctx->d;
    // dt inputs as after start-up or a restart: nu and alpha are not part of the state
    // (never restored by the reference), so their maxima start at zero (:4401-4408).  The
    // step counters of a running device loop are kept.
    CK(cudaMemsetAsync((char*)d.dS + offsetof(les::Scalars, numax), 0, sizeof(double), d.stream));
    CK(cudaMemsetAsync((char*)d.dS + offsetof(les::Scalars, alphamax), 0, sizeof(double), d.stream));
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::umax_f64(d) : les::umax_f32(d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "umax");
    CK(cudaStreamSynchronize(d.stream));
    d.have_state = (nfields == LESGPU_NSTATE) || d.have_state;
    return LESGPU_OK;
}

int lesgpu_download_state(lesgpu_ctx* ctx, double* const* fields, int nfields) {
    if (!ctx || !fields || nfields < 1 || nfields > LESGPU_NSTATE) return LESGPU_EINVAL;
    for (int q = 0; q < nfields; q++) {
        if (!fields[q]) return LESGPU_EINVAL;
        int r = copy_field_out(ctx, fields[q], ctx->d.S[q], 8);
        if (r) return r;
    }
    return LESGPU_OK;
}

static int ensure_debug(lesgpu_ctx* ctx) {
    DevCtx& d = ctx->d;
    if (d.dbg_cp) return LESGPU_OK;
    size_t bytes = d.n * d.esz;
    CK(dalloc(d, &d.dbg_cp, bytes));
    CK(dalloc(d, &d.dbg_lam, bytes));
    CK(dalloc(d, &d.dbg_alpha, bytes));
    for (int q = 0; q < les::NACC; q++) CK(dalloc(d, &d.kd[q], bytes));
    CK(cudaMemsetAsync(d.dbg_cp, 0, bytes, d.stream));
    CK(cudaMemsetAsync(d.dbg_lam, 0, bytes, d.stream));
    CK(cudaMemsetAsync(d.dbg_alpha, 0, bytes, d.stream));
    for (int q = 0; q < les::NACC; q++) CK(cudaMemsetAsync(d.kd[q], 0, bytes, d.stream));
    d.total_bytes += 13 * bytes;
    return LESGPU_OK;
}

int lesgpu_set_debug(lesgpu_ctx* ctx, int enable) {
    if (!ctx) return LESGPU_EINVAL;
    if (enable) {
        int r = ensure_debug(ctx);
        if (r) return r;
    }
    ctx->d.debug = enable != 0;
    return LESGPU_OK;
}

int lesgpu_get_field(lesgpu_ctx* ctx, int id, double* out) {
    if (!ctx || !out) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    const void* src = nullptr;
    if (id >= LESGPU_F_U && id <= LESGPU_F_Y4) src = d.S[id];
    else if (id == LESGPU_F_NU_T) src = d.nu_t;
    else if (id == LESGPU_F_S_MAG) src = d.S_mag;
    else if (id == LESGPU_F_GRAD_G) {
        if (!d.grad_g) return fail(ctx, LESGPU_ESTATE, "enable lesgpu_keep_grad_g before the step to read this field");
        src = d.grad_g;
    }
    else if (id >= LESGPU_F_U_F && id <= LESGPU_F_Y4_F) src = d.F[id - LESGPU_F_U_F];
    else if (id == LESGPU_F_NU) src = d.nu;
    else if (id == LESGPU_F_MU_MIX) src = d.mu_mix;
    else if (id == LESGPU_F_ST) src = d.ST;
    else if (id >= LESGPU_F_D0 && id <= LESGPU_F_D4) src = d.D[id - LESGPU_F_D0];
    else if (id == LESGPU_F_CP || id == LESGPU_F_LAMBDA || id == LESGPU_F_ALPHA ||
             (id >= LESGPU_F_K_RHOU && id <= LESGPU_F_K_Y4)) {
        if (!d.debug) return fail(ctx, LESGPU_ESTATE, "enable lesgpu_set_debug before the step to read this field");
        if (id == LESGPU_F_CP) src = d.dbg_cp;
        else if (id == LESGPU_F_LAMBDA) src = d.dbg_lam;
        else if (id == LESGPU_F_ALPHA) src = d.dbg_alpha;
        else src = d.kd[id - LESGPU_F_K_RHOU];
    } else {
        return fail(ctx, LESGPU_EINVAL, "unknown field id");
    }
    return copy_field_out(ctx, out, src, (id >= LESGPU_F_U && id <= LESGPU_F_Y4) ? 8 : d.esz);
}

int lesgpu_dt_inputs(lesgpu_ctx* ctx, double* umax, double* numax, double* alphamax) {
    if (!ctx || !umax || !numax || !alphamax) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state) return fail(ctx, LESGPU_ESTATE, "no state uploaded");
    les::Scalars h;
    CK(cudaMemcpyAsync(&h, d.dS, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    if (h.nonfinite & 4) return fail(ctx, LESGPU_ECUDA, "a tensor copy of the staged scalar pass timed out");
    *umax = h.umax > 1e-10 ? h.umax : ctx->cfg.inlet_velocity;   // :1484
    *numax = h.numax;
    *alphamax = h.alphamax;
    return LESGPU_OK;
}

int lesgpu_set_dt_inputs(lesgpu_ctx* ctx, double numax, double alphamax) {
    if (!ctx || !(numax >= 0.0) || !(alphamax >= 0.0)) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state) return fail(ctx, LESGPU_ESTATE, "no state uploaded");
    CK(cudaMemcpyAsync((char*)d.dS + offsetof(les::Scalars, numax), &numax, sizeof(double), cudaMemcpyHostToDevice,
                       d.stream));
    CK(cudaMemcpyAsync((char*)d.dS + offsetof(les::Scalars, alphamax), &alphamax, sizeof(double),
                       cudaMemcpyHostToDevice, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    return LESGPU_OK;
}

int lesgpu_set_inflow(lesgpu_ctx* ctx, const double* vortices, int nv, const double* noise) {
    if (!ctx || nv < 0 || (nv > 0 && !vortices)) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_attr) return fail(ctx, LESGPU_ESTATE, "upload the attribute map first");
    if (nv > d.nv_cap) {
        double* nb = nullptr;
        CK(cudaStreamSynchronize(d.stream));
        CK(dalloc(d, &nb, (size_t)nv * 7 * sizeof(double)));
        dfree(d, d.vort);
        d.vort = nb;
        d.nv_cap = nv;
    }
    d.nv = nv;
    if (nv > 0) CK(cudaMemcpyAsync(d.vort, vortices, (size_t)nv * 7 * sizeof(double), cudaMemcpyHostToDevice, d.stream));
    if (d.n_inlet > 0) {
        if (!noise) return LESGPU_EINVAL;
        if (d.h_pinned == nullptr) {
            d.h_pinned_len = 3 * (size_t)d.ny * d.nz * sizeof(double);
            if (cudaMallocHost(&d.h_pinned, d.h_pinned_len) != cudaSuccess) {
                cudaGetLastError();
                d.h_pinned = nullptr;
                d.h_pinned_len = 0;
                return fail(ctx, LESGPU_ENOMEM, "pinned staging buffer unavailable");
            }
        }
        // pack r1, r2, r3 of the inlet cells (the only cells the inflow condition reads);
        // the pinned buffer is reused, so wait for the previous upload to finish first
        CK(cudaStreamSynchronize(d.stream));
        const size_t planes = (size_t)d.ny * d.nz;
        for (int q = 0; q < d.n_inlet; q++) {
            size_t p = (size_t)d.h_inlet[q];
            d.h_pinned[3 * q + 0] = noise[p];
            d.h_pinned[3 * q + 1] = noise[planes + p];
            d.h_pinned[3 * q + 2] = noise[2 * planes + p];
        }
        CK(cudaMemcpyAsync(d.noise, d.h_pinned, 3 * (size_t)d.n_inlet * sizeof(double), cudaMemcpyHostToDevice,
                           d.stream));
    }
    d.have_inflow = true;
    return LESGPU_OK;
}

int lesgpu_step(lesgpu_ctx* ctx, double dt, int t_loop) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state || !d.have_attr) return fail(ctx, LESGPU_ESTATE, "state and attribute map must be uploaded");
    if (d.n_inlet > 0 && !d.have_inflow) return fail(ctx, LESGPU_ESTATE, "lesgpu_set_inflow must precede each step");
    if (!(dt > 0.0) || !isfinite(dt)) return fail(ctx, LESGPU_EINVAL, "dt must be positive and finite");
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::step_f64(d, dt, t_loop, false)
                                                 : les::step_f32(d, dt, t_loop, false);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "step");
    d.have_inflow = false;
    return LESGPU_OK;
}


int lesgpu_loop_begin(lesgpu_ctx* ctx, const unsigned int rng_window[31], const double* vortices, int nv, int t_loop) {
    if (!ctx || !rng_window || nv < 0 || (nv > 0 && !vortices)) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state || !d.have_attr) return fail(ctx, LESGPU_ESTATE, "state and attribute map must be uploaded");
    CK(cudaStreamSynchronize(d.stream));
    free_loop(d);
    if (nv > d.nv_cap) {
        dfree(d, d.vort);
        d.vort = nullptr;
        CK(dalloc(d, &d.vort, (size_t)nv * 7 * sizeof(double)));
        d.nv_cap = nv;
    }
    d.nv = nv;
    // at most 6 draws per vortex and 3 per inlet cell in one step
    d.jrows = 6 * nv + 3 * d.n_inlet;
    if (d.jrows < 31) d.jrows = 31;
    std::vector<unsigned int> J = jump_table(d.jrows);
    CK(dalloc(d, &d.J, J.size() * sizeof(unsigned int)));
    CK(dalloc(d, &d.dL, sizeof(les::LoopState)));
    CK(cudaStreamSynchronize(d.stream));
    if (nv > 0) CK(cudaMemcpy(d.vort, vortices, (size_t)nv * 7 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.J, J.data(), J.size() * sizeof(unsigned int), cudaMemcpyHostToDevice));
    les::LoopState ls{};
    for (int j = 0; j < 31; j++) ls.win[j] = rng_window[j];
    CK(cudaMemcpy(d.dL, &ls, sizeof(ls), cudaMemcpyHostToDevice));
    const lesgpu_config& g = ctx->cfg;
    d.lp_lbox = g.length_scale; d.lp_ly = g.ly; d.lp_lz = g.lz; d.lp_uin = g.inlet_velocity;
    d.lp_ti = g.turbulence_intensity; d.lp_ell = g.length_scale; d.lp_cfl = g.courant;
    d.lp_cfld = g.courant_diffusion; d.lp_dx = g.lx / (double)g.nx;
    // default history: the reference's 7 probe stations on the line k = NZ/2 (:274, :3406)
    const double xs[7] = {0.010, 0.015, 0.020, 0.025, 0.030, 0.035, 0.040};
    std::vector<int> st;
    for (double x : xs) {
        int ip = (int)(x / d.lp_dx);
        if (ip > 0 && ip < d.nx - 1) st.push_back(ip);
    }
    int r = alloc_history(ctx, st.data(), (int)st.size(), d.nz / 2, 64);
    if (r) return r;
    // step counters in the scalar block
    les::Scalars h;
    CK(cudaMemcpy(&h, d.dS, sizeof(h), cudaMemcpyDeviceToHost));
    h.t_loop = t_loop;
    h.run_step = 0;
    h.nonfinite = 0;
    CK(cudaMemcpy(d.dS, &h, sizeof(h), cudaMemcpyHostToDevice));
    d.loop_ready = true;
    d.total_bytes += J.size() * sizeof(unsigned int);
    return LESGPU_OK;
}

int lesgpu_loop_config(lesgpu_ctx* ctx, const int* i_stations, int n, int k_line, int capacity_steps) {
    if (!ctx || n < 0 || (n > 0 && !i_stations) || capacity_steps < 1) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.loop_ready) return fail(ctx, LESGPU_ESTATE, "lesgpu_loop_begin first");
    if (k_line < 0 || k_line >= d.nz) return fail(ctx, LESGPU_EINVAL, "k_line out of range");
    for (int q = 0; q < n; q++)
        if (i_stations[q] < 0 || i_stations[q] >= d.nx) return fail(ctx, LESGPU_EINVAL, "station out of range");
    CK(cudaStreamSynchronize(d.stream));
    return alloc_history(ctx, i_stations, n, k_line, capacity_steps);
}

int lesgpu_run(lesgpu_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.loop_ready) return fail(ctx, LESGPU_ESTATE, "lesgpu_loop_begin first");
    if (nsteps > d.loop_cap) return fail(ctx, LESGPU_EINVAL, "nsteps exceeds the history capacity (lesgpu_loop_config)");
    if (nsteps == 0) return LESGPU_OK;
    // run_step restarts at 0 for every run (history slots)
    CK(cudaMemsetAsync((char*)d.dS + offsetof(les::Scalars, run_step), 0, sizeof(int), d.stream));
    const bool fp64 = d.precision == LESGPU_FP64;
    if (d.timing) {
        for (int q = 0; q < nsteps; q++) {
            cudaError_t e = fp64 ? les::step_f64(d, 0.0, 0, true) : les::step_f32(d, 0.0, 0, true);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "run");
        }
        return LESGPU_OK;
    }
    if (!d.graph_ok) {
        // capture one device-loop step; every launch reads its varying inputs (dt, t_loop,
        // history slot) from device memory, so the graph is replayed unchanged
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(d.stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = fp64 ? les::step_f64(d, 0.0, 0, true) : les::step_f32(d, 0.0, 0, true);
        cudaError_t e2 = cudaStreamEndCapture(d.stream, &gr);
        if (e != cudaSuccess) { if (gr) cudaGraphDestroy(gr); return cuda_fail(ctx, e, "capture"); }
        if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&d.graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
        d.graph_ok = true;
    }
    for (int q = 0; q < nsteps; q++) CK(cudaGraphLaunch(d.graph, d.stream));
    return LESGPU_OK;
}

int lesgpu_loop_history(lesgpu_ctx* ctx, int nsteps, double* dt, double* umax, double* probes, double* monitor) {
    if (!ctx || nsteps < 0) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.loop_ready) return fail(ctx, LESGPU_ESTATE, "lesgpu_loop_begin first");
    if (nsteps > d.loop_cap) return fail(ctx, LESGPU_EINVAL, "nsteps exceeds the history capacity");
    CK(cudaStreamSynchronize(d.stream));
    les::Scalars h;
    CK(cudaMemcpy(&h, d.dS, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.nonfinite & 2) return fail(ctx, LESGPU_ESTATE, "rand() jump table too short");
    if (h.nonfinite & 4) return fail(ctx, LESGPU_ECUDA, "a tensor copy of the staged scalar pass timed out");
    if (nsteps == 0) return LESGPU_OK;
    if (dt) CK(cudaMemcpy(dt, d.hist_dt, nsteps * sizeof(double), cudaMemcpyDeviceToHost));
    if (umax) CK(cudaMemcpy(umax, d.hist_umax, nsteps * sizeof(double), cudaMemcpyDeviceToHost));
    if (probes && d.loop_nst > 0)
        CK(cudaMemcpy(probes, d.hist_probe, (size_t)nsteps * d.loop_nst * d.ny * 6 * sizeof(double),
                      cudaMemcpyDeviceToHost));
    if (monitor) CK(cudaMemcpy(monitor, d.hist_mon, (size_t)nsteps * 6 * sizeof(double), cudaMemcpyDeviceToHost));
    return LESGPU_OK;
}

int lesgpu_loop_end(lesgpu_ctx* ctx, unsigned int rng_window[31], double* vortices, int* t_loop) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.loop_ready) return fail(ctx, LESGPU_ESTATE, "lesgpu_loop_begin first");
    CK(cudaStreamSynchronize(d.stream));
    les::LoopState ls;
    CK(cudaMemcpy(&ls, d.dL, sizeof(ls), cudaMemcpyDeviceToHost));
    les::Scalars h;
    CK(cudaMemcpy(&h, d.dS, sizeof(h), cudaMemcpyDeviceToHost));
    if (rng_window)
        for (int j = 0; j < 31; j++) rng_window[j] = ls.win[j];
    if (vortices && d.nv > 0) CK(cudaMemcpy(vortices, d.vort, (size_t)d.nv * 7 * sizeof(double), cudaMemcpyDeviceToHost));
    if (t_loop) *t_loop = h.t_loop;
    d.total_bytes -= (size_t)d.jrows * 31 * sizeof(unsigned int);
    free_loop(d);
    if (h.nonfinite & 2) return fail(ctx, LESGPU_ESTATE, "rand() jump table too short");
    if (h.nonfinite & 4) return fail(ctx, LESGPU_ECUDA, "a tensor copy of the staged scalar pass timed out");
    return LESGPU_OK;
}

int lesgpu_eval_rhs(lesgpu_ctx* ctx, int t_loop) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state || !d.have_attr) return fail(ctx, LESGPU_ESTATE, "state and attribute map must be uploaded");
    int r = lesgpu_set_debug(ctx, 1);
    if (r) return r;
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::rhs_only_f64(d, t_loop) : les::rhs_only_f32(d, t_loop);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "eval_rhs");
    CK(cudaStreamSynchronize(d.stream));
    return LESGPU_OK;
}

int lesgpu_probe_lines(lesgpu_ctx* ctx, const int* i_stations, int n, int k_line, double* out) {
    if (!ctx || n < 0 || (n > 0 && (!i_stations || !out))) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (n == 0) return LESGPU_OK;
    if (k_line < 0 || k_line >= d.nz) return fail(ctx, LESGPU_EINVAL, "k_line out of range");
    for (int q = 0; q < n; q++)
        if (i_stations[q] < 0 || i_stations[q] >= d.nx) return fail(ctx, LESGPU_EINVAL, "station out of range");
    if (n > d.probe_cap) {
        CK(cudaStreamSynchronize(d.stream));
        dfree(d, d.probe_st);
        dfree(d, d.probe_out);
        d.probe_st = nullptr;
        d.probe_out = nullptr;
        CK(dalloc(d, &d.probe_st, n * sizeof(int)));
        CK(dalloc(d, &d.probe_out, (size_t)n * d.ny * 6 * sizeof(double)));
        d.probe_cap = n;
    }
    CK(cudaMemcpyAsync(d.probe_st, i_stations, n * sizeof(int), cudaMemcpyHostToDevice, d.stream));
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::probe_f64(d, n, k_line) : les::probe_f32(d, n, k_line);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "probe");
    CK(cudaMemcpyAsync(out, d.probe_out, (size_t)n * d.ny * 6 * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    return LESGPU_OK;
}

int lesgpu_monitor(lesgpu_ctx* ctx, double out[6]) {
    if (!ctx || !out) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::monitor_f64(d) : les::monitor_f32(d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "monitor");
    les::Scalars h;
    CK(cudaMemcpyAsync(&h, d.dS, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    for (int q = 0; q < 6; q++) out[q] = h.mon[q];
    return LESGPU_OK;
}

int lesgpu_check_finite(lesgpu_ctx* ctx, int field_id) {
    if (!ctx || field_id < 0 || field_id > LESGPU_F_NU_T) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    cudaError_t e = (d.precision == LESGPU_FP64) ? les::check_f64(d, field_id) : les::check_f32(d, field_id);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "check_finite");
    int h = 0;
    CK(cudaMemcpyAsync(&h, d.flag, sizeof(int), cudaMemcpyDeviceToHost, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    if (h) return fail(ctx, LESGPU_ENONFINITE, "non-finite value found");
    return LESGPU_OK;
}

int lesgpu_kernel_timing(lesgpu_ctx* ctx, int enable) {
    if (!ctx) return LESGPU_EINVAL;
    ctx->d.timing = enable != 0;
    for (int q = 0; q < 8; q++) { ctx->d.kms[q] = 0.0; ctx->d.kcount[q] = 0; }
    return LESGPU_OK;
}

int lesgpu_mark(lesgpu_ctx* ctx, int slot) {
    if (!ctx || slot < 0 || slot >= 16) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.marks[slot]) CK(cudaEventCreate(&d.marks[slot]));
    CK(cudaEventRecord(d.marks[slot], d.stream));
    return LESGPU_OK;
}

int lesgpu_elapsed_ms(lesgpu_ctx* ctx, int a, int b, double* ms) {
    if (!ctx || !ms || a < 0 || b < 0 || a >= 16 || b >= 16) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.marks[a] || !d.marks[b]) return fail(ctx, LESGPU_ESTATE, "marker not recorded");
    CK(cudaEventSynchronize(d.marks[b]));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, d.marks[a], d.marks[b]));
    *ms = f;
    return LESGPU_OK;
}

int lesgpu_kernel_times(lesgpu_ctx* ctx, double* ms, long long* launches, int n) {
    if (!ctx || !ms || !launches || n < 0) return LESGPU_EINVAL;
    les::tmark_flush(ctx->d);
    for (int q = 0; q < n && q < LESGPU_NK; q++) {
        ms[q] = ctx->d.kms[q];
        launches[q] = ctx->d.kcount[q];
        ctx->d.kms[q] = 0.0;
        ctx->d.kcount[q] = 0;
    }
    return LESGPU_OK;
}

int lesgpu_selfcheck_division(const double* divisors, int nd, size_t n, unsigned long long seed,
                              unsigned long long* mismatches) {
    if (!divisors || nd <= 0 || !mismatches) return LESGPU_EINVAL;
    return les::selfcheck_division(divisors, nd, n, seed, mismatches);
}

int lesgpu_sync(lesgpu_ctx* ctx) {
    if (!ctx) return LESGPU_EINVAL;
    CK(cudaStreamSynchronize(ctx->d.stream));
    return LESGPU_OK;
}

int lesgpu_bind_device(int device) {
    if (device < 0) return LESGPU_EINVAL;
    return cudaSetDevice(device) == cudaSuccess ? LESGPU_OK : LESGPU_ECUDA;
}

// ---------------------------------------------------------------- tiles and autotuning

static void drop_graph(DevCtx& d) {
    if (d.graph) cudaGraphExecDestroy(d.graph);
    d.graph = nullptr;
    d.graph_ok = false;
}

int lesgpu_set_tiles(lesgpu_ctx* ctx, const int tiles[5]) {
    if (!ctx || !tiles) return LESGPU_EINVAL;
    for (int q = 0; q < les::NSH_CLASSES; q++)
        if (!les::shape_allowed(q, tiles[q])) return fail(ctx, LESGPU_EINVAL, "tile index out of range for its class");
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    for (int q = 0; q < les::NSH_CLASSES; q++) d.shape[q] = tiles[q];
    drop_graph(d);
    return LESGPU_OK;
}

int lesgpu_set_scalar_staging(lesgpu_ctx* ctx, int enable) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (enable && !d.tma_ok) return fail(ctx, LESGPU_EINVAL, "staged scalar pass unavailable for this grid");
    CK(cudaStreamSynchronize(d.stream));
    d.scalar_tma = enable != 0;
    drop_graph(d);
    return LESGPU_OK;
}

int lesgpu_get_scalar_staging(const lesgpu_ctx* ctx) { return (ctx && ctx->d.scalar_tma) ? 1 : 0; }

int lesgpu_get_tiles(const lesgpu_ctx* ctx, int tiles[5]) {
    if (!ctx || !tiles) return LESGPU_EINVAL;
    for (int q = 0; q < les::NSH_CLASSES; q++) tiles[q] = ctx->d.shape[q];
    return LESGPU_OK;
}

int lesgpu_autotune(lesgpu_ctx* ctx, int reps, int tiles_out[5], double* ms_out) {
    if (!ctx || reps < 1) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.have_state || !d.have_attr) return fail(ctx, LESGPU_ESTATE, "state and attribute map must be uploaded");
    CK(cudaStreamSynchronize(d.stream));
    // the stage kernels overwrite the dt inputs, <rho_f> and the step counters: keep a copy
    les::Scalars saved;
    CK(cudaMemcpy(&saved, d.dS, sizeof(saved), cudaMemcpyDeviceToHost));
    const bool was_timing = d.timing;
    int old[les::NSH_CLASSES];
    for (int q = 0; q < les::NSH_CLASSES; q++) old[q] = d.shape[q];
    const int cls_of[4] = {LESGPU_K_FILTER, LESGPU_K_STRAIN, LESGPU_K_RHS_FLOW, LESGPU_K_RHS_SCALAR};
    static_assert(les::NSHAPES == LESGPU_NTILES, "tile table and ABI disagree");
    double ms[4][les::NSHAPES];
    cudaError_t e = cudaSuccess;
    for (int t = 0; t < les::NSHAPES && e == cudaSuccess; t++) {
        // a 512-thread tile is timed for the strain, flow and scalar classes; the filter and
        // EOS kernels keep the first tile meanwhile
        for (int q = 0; q < les::NSH_CLASSES; q++) d.shape[q] = les::shape_allowed(q, t) ? t : 0;
        d.timing = false;
        e = (d.precision == LESGPU_FP64) ? les::rhs_only_f64(d, 0) : les::rhs_only_f32(d, 0);   // warm-up
        d.timing = true;
        for (int q = 0; q < 8; q++) { d.kms[q] = 0.0; d.kcount[q] = 0; }
        for (int r = 0; r < reps && e == cudaSuccess; r++)
            e = (d.precision == LESGPU_FP64) ? les::rhs_only_f64(d, 0) : les::rhs_only_f32(d, 0);
        for (int c = 0; c < 4; c++)
            ms[c][t] = (les::shape_allowed(c, t) && d.kcount[cls_of[c]] > 0)
                           ? d.kms[cls_of[c]] / (double)d.kcount[cls_of[c]] : 1e30;
    }
    d.timing = was_timing;
    for (int q = 0; q < 8; q++) { d.kms[q] = 0.0; d.kcount[q] = 0; }
    cudaError_t e2 = cudaStreamSynchronize(d.stream);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaMemcpy(d.dS, &saved, sizeof(saved), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        for (int q = 0; q < les::NSH_CLASSES; q++) d.shape[q] = old[q];
        return cuda_fail(ctx, e, "autotune");
    }
    int best[les::NSH_CLASSES];
    for (int c = 0; c < 4; c++) {
        best[c] = 0;
        for (int t = 1; t < les::NSHAPES; t++)
            if (ms[c][t] < ms[c][best[c]]) best[c] = t;
    }
    best[les::SH_EOS] = best[les::SH_FILTER];
    for (int q = 0; q < les::NSH_CLASSES; q++) d.shape[q] = best[q];
    // The TMA-staged scalar pass (les_tma.cuh) is not timed here: on B200 it is slower than the
    // plain pass at every grid measured (256x128x128 FP64: 4.03 against 3.07 ms per step), so
    // tuning it would only cost time on every new grid shape.  It stays selectable with
    // lesgpu_set_scalar_staging, which the autotuner leaves as it is.
    drop_graph(d);
    if (tiles_out)
        for (int q = 0; q < les::NSH_CLASSES; q++) tiles_out[q] = best[q];
    if (ms_out)
        for (int c = 0; c < 4; c++)
            for (int t = 0; t < les::NSHAPES; t++) ms_out[c * les::NSHAPES + t] = ms[c][t];
    return LESGPU_OK;
}

int lesgpu_keep_grad_g(lesgpu_ctx* ctx, int enable) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    if (enable && !d.grad_g) {
        const size_t bytes = d.n * d.esz;
        CK(dalloc(d, &d.grad_g, bytes));
        CK(cudaMemsetAsync(d.grad_g, 0, bytes, d.stream));   // non-fluid cells stay 0, as in the reference (:2820)
        CK(cudaStreamSynchronize(d.stream));
        d.total_bytes += bytes;
    } else if (!enable && d.grad_g) {
        dfree(d, d.grad_g);
        d.grad_g = nullptr;
        d.total_bytes -= d.n * d.esz;
    }
    drop_graph(d);
    return LESGPU_OK;
}

// ---------------------------------------------------------------- profile statistics

static void pstat_free(DevCtx& d) {
    void* bufs[] = {d.ps_edges, d.ps_sums, d.ps_yflame, d.ps_rowbin};
    for (void* b : bufs) dfree(d, b);
    d.ps_edges = d.ps_sums = d.ps_yflame = nullptr;
    d.ps_rowbin = nullptr;
    d.ps_rows_cap = 0;
    d.ps_nsums = 0;
    d.ps_on = false;
}

static bool increasing(const double* e, int n) {
    for (int q = 0; q < n; q++)
        if (!(e[q] < e[q + 1])) return false;
    return true;
}

int lesgpu_pstat_begin(lesgpu_ctx* ctx, const double* y_edges_mm, int n_y, const double* g_rc_edges, int n_grc,
                       const double* g_ho_edges, int n_gho, const double* u_edges, const double* v_edges, int n_pdf) {
    if (!ctx || !y_edges_mm || !g_rc_edges || !g_ho_edges || !u_edges || !v_edges) return LESGPU_EINVAL;
    if (n_y < 1 || n_grc < 1 || n_gho < 1 || n_pdf < 1 || n_y > 4096 || n_grc > 4096 || n_gho > 4096 || n_pdf > 4096)
        return fail(ctx, LESGPU_EINVAL, "bin counts must be in 1..4096");
    if (!increasing(y_edges_mm, n_y) || !increasing(g_rc_edges, n_grc) || !increasing(g_ho_edges, n_gho) ||
        !increasing(u_edges, n_pdf) || !increasing(v_edges, n_pdf))
        return fail(ctx, LESGPU_EINVAL, "bin edges must increase");
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    pstat_free(d);
    std::vector<double> e;
    e.insert(e.end(), y_edges_mm, y_edges_mm + n_y + 1);
    e.insert(e.end(), g_rc_edges, g_rc_edges + n_grc + 1);
    e.insert(e.end(), g_ho_edges, g_ho_edges + n_gho + 1);
    e.insert(e.end(), u_edges, u_edges + n_pdf + 1);
    e.insert(e.end(), v_edges, v_edges + n_pdf + 1);
    d.ps_ny = n_y; d.ps_ngrc = n_grc; d.ps_ngho = n_gho; d.ps_npdf = n_pdf;
    d.ps_nsums = 4 + 9 * (size_t)n_y + 7 * (size_t)n_grc + 4 * (size_t)n_gho + 4 * (size_t)n_pdf;
    CK(dalloc(d, &d.ps_edges, e.size() * sizeof(double)));
    CK(dalloc(d, &d.ps_sums, d.ps_nsums * sizeof(double)));
    CK(cudaMemcpyAsync(d.ps_edges, e.data(), e.size() * sizeof(double), cudaMemcpyHostToDevice, d.stream));
    CK(cudaMemsetAsync(d.ps_sums, 0, d.ps_nsums * sizeof(double), d.stream));
    CK(cudaStreamSynchronize(d.stream));
    d.ps_on = true;
    return LESGPU_OK;
}

int lesgpu_pstat_accumulate(lesgpu_ctx* ctx, int nsteps, int n_lines) {
    if (!ctx || nsteps < 0 || n_lines < 0) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.ps_on) return fail(ctx, LESGPU_ESTATE, "lesgpu_pstat_begin first");
    if (!d.loop_ready || !d.hist_probe) return fail(ctx, LESGPU_ESTATE, "no device-loop history");
    if (nsteps > d.loop_cap || n_lines > d.loop_nst)
        return fail(ctx, LESGPU_EINVAL, "more steps or lines than the history holds");
    if (nsteps == 0 || n_lines == 0) return LESGPU_OK;
    const size_t rows = (size_t)d.loop_cap * d.loop_nst * d.ny;
    if (rows > d.ps_rows_cap) {          // scratch sized for the whole history once
        dfree(d, d.ps_yflame);
        dfree(d, d.ps_rowbin);
        d.ps_yflame = nullptr;
        d.ps_rowbin = nullptr;
        CK(dalloc(d, &d.ps_yflame, (size_t)d.loop_cap * d.loop_nst * sizeof(double)));
        CK(dalloc(d, &d.ps_rowbin, rows * 5 * sizeof(int)));
        d.ps_rows_cap = rows;
    }
    cudaError_t e = les::pstat_accumulate(d, nsteps, n_lines);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pstat_accumulate");
    return LESGPU_OK;
}

size_t lesgpu_pstat_size(const lesgpu_ctx* ctx) { return (ctx && ctx->d.ps_on) ? ctx->d.ps_nsums : 0; }

int lesgpu_pstat_layout(const lesgpu_ctx* ctx, int* n_y, int* n_grc, int* n_gho, int* n_pdf, double* edges,
                        size_t* n_edges) {
    if (!ctx) return LESGPU_EINVAL;
    const DevCtx& d = ctx->d;
    if (!d.ps_on) return LESGPU_ESTATE;
    if (n_y) *n_y = d.ps_ny;
    if (n_grc) *n_grc = d.ps_ngrc;
    if (n_gho) *n_gho = d.ps_ngho;
    if (n_pdf) *n_pdf = d.ps_npdf;
    const size_t ne = (size_t)d.ps_ny + d.ps_ngrc + d.ps_ngho + 2 * (size_t)d.ps_npdf + 5;
    if (n_edges) *n_edges = ne;
    if (edges) {
        cudaError_t e = cudaMemcpy(edges, d.ps_edges, ne * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return LESGPU_ECUDA;
    }
    return LESGPU_OK;
}

int lesgpu_pstat_read(lesgpu_ctx* ctx, double* out) {
    if (!ctx || !out) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.ps_on) return fail(ctx, LESGPU_ESTATE, "lesgpu_pstat_begin first");
    CK(cudaStreamSynchronize(d.stream));
    CK(cudaMemcpy(out, d.ps_sums, d.ps_nsums * sizeof(double), cudaMemcpyDeviceToHost));
    return LESGPU_OK;
}

int lesgpu_pstat_end(lesgpu_ctx* ctx) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    pstat_free(d);
    return LESGPU_OK;
}

// ---------------------------------------------------------------- time averages

int lesgpu_avg_begin(lesgpu_ctx* ctx, int start_step) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    const size_t bytes = (size_t)les::NAVG * d.n * sizeof(double);
    if (!d.avg) {
        CK(dalloc(d, &d.avg, bytes));
        d.total_bytes += bytes;
    }
    CK(cudaMemsetAsync(d.avg, 0, bytes, d.stream));
    CK(cudaMemsetAsync((char*)d.dS + offsetof(les::Scalars, avg_steps), 0, sizeof(int), d.stream));
    CK(cudaStreamSynchronize(d.stream));
    d.avg_start = start_step;
    drop_graph(d);
    return LESGPU_OK;
}

int lesgpu_avg_end(lesgpu_ctx* ctx) {
    if (!ctx) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    CK(cudaStreamSynchronize(d.stream));
    if (d.avg) {
        dfree(d, d.avg);
        d.avg = nullptr;
        d.total_bytes -= (size_t)les::NAVG * d.n * sizeof(double);
    }
    drop_graph(d);
    return LESGPU_OK;
}

int lesgpu_avg_download(lesgpu_ctx* ctx, double* const* sums, int* count) {
    if (!ctx || !sums || !count) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.avg) return fail(ctx, LESGPU_ESTATE, "time averages are not enabled (lesgpu_avg_begin)");
    CK(cudaStreamSynchronize(d.stream));
    for (int q = 0; q < les::NAVG; q++) {
        if (!sums[q]) return LESGPU_EINVAL;
        CK(cudaMemcpy(sums[q], d.avg + (size_t)q * d.n, d.n * sizeof(double), cudaMemcpyDeviceToHost));
    }
    CK(cudaMemcpy(count, (char*)d.dS + offsetof(les::Scalars, avg_steps), sizeof(int), cudaMemcpyDeviceToHost));
    return LESGPU_OK;
}

int lesgpu_avg_upload(lesgpu_ctx* ctx, const double* const* sums, int count) {
    if (!ctx || !sums || count < 0) return LESGPU_EINVAL;
    DevCtx& d = ctx->d;
    if (!d.avg) return fail(ctx, LESGPU_ESTATE, "time averages are not enabled (lesgpu_avg_begin)");
    CK(cudaStreamSynchronize(d.stream));
    for (int q = 0; q < les::NAVG; q++) {
        if (!sums[q]) return LESGPU_EINVAL;
        CK(cudaMemcpy(d.avg + (size_t)q * d.n, sums[q], d.n * sizeof(double), cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy((char*)d.dS + offsetof(les::Scalars, avg_steps), &count, sizeof(int), cudaMemcpyHostToDevice));
    return LESGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- groups

struct lesgpu_group {
    std::vector<lesgpu_ctx*> m;
    int device = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> joins, ready;
    cudaGraphExec_t exec = nullptr;
    // batched form: members in batches of one shape, each batch's RK stages on its own stream
    std::vector<std::vector<int>> batches;
    std::vector<cudaStream_t> bstreams;
    std::vector<cudaEvent_t> heads, stages;
    std::vector<les::MemberTab*> tabs;     // device member tables, one per batch
};

namespace {

// Members batch together when their constants agree except the model constants an ensemble
// varies (read per member from the member table), and their tiles and arena layout agree.
les::Consts masked_consts(const les::Consts& c) {
    les::Consts m;
    std::memcpy(&m, &c, sizeof(m));
    m.cs_u = m.cs_b = m.cs_boost = m.accel_strength = m.accel_center = m.two_w2 = m.relax = 0.0;
    m.d_w2 = les::DC{0.0, 0.0};
    m.f.cs_u = m.f.cs_b = m.f.cs_boost = m.f.accel_strength = m.f.accel_center = m.f.relax = 0.0f;
    m.f.d_w2 = les::DCT<float>{0.0f, 0.0f};
    return m;
}

bool batchable(const DevCtx& a, const DevCtx& b) {
    if (a.nx != b.nx || a.ny != b.ny || a.nz != b.nz || a.precision != b.precision) return false;
    for (int q = 0; q < les::NSH_CLASSES; q++)
        if (a.shape[q] != b.shape[q]) return false;
    // per-cell fields at the same offsets within the two arenas
    auto off = [](const DevCtx& d, const void* p) { return (const char*)p - (const char*)d.arena; };
    for (int q = 0; q < les::NSTATE; q++)
        if (off(a, a.S[q]) != off(b, b.S[q]) || off(a, a.St[q]) != off(b, b.St[q]) || off(a, a.F[q]) != off(b, b.F[q]))
            return false;
    for (int q = 0; q < les::NACC; q++)
        if (off(a, a.acc[q]) != off(b, b.acc[q])) return false;
    for (int q = 0; q < 4; q++)
        if (off(a, a.kflow[q]) != off(b, b.kflow[q])) return false;
    if (off(a, a.mu_mix) != off(b, b.mu_mix) || off(a, a.nu_t) != off(b, b.nu_t) || off(a, a.mu_eff) != off(b, b.mu_eff))
        return false;
    const les::Consts ca = masked_consts(a.hC), cb = masked_consts(b.hC);
    return std::memcmp(&ca, &cb, sizeof(ca)) == 0;
}

les::MemberTab member_entry(const DevCtx& d0, const DevCtx& d) {
    les::MemberTab e{};
    e.delta = (long long)((const char*)d.arena - (const char*)d0.arena);
    e.attr = d.attr;
    e.S = d.dS;
    e.part = d.part;
    e.md = les::model_of<double>(d.hC);
    e.mf = les::model_of<float>(d.hC);
    return e;
}

}  // namespace

extern "C" {

void lesgpu_group_destroy(lesgpu_group* g) {
    if (!g) return;
    if (g->root) cudaStreamSynchronize(g->root);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    for (les::MemberTab* t : g->tabs) if (t && g->root) cudaFreeAsync(t, g->root);
    if (g->root) cudaStreamSynchronize(g->root);
    for (cudaEvent_t e : g->heads) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : g->stages) if (e) cudaEventDestroy(e);
    for (cudaStream_t st : g->bstreams) if (st) cudaStreamDestroy(st);
    for (cudaEvent_t e : g->joins) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : g->ready) if (e) cudaEventDestroy(e);
    if (g->fork) cudaEventDestroy(g->fork);
    if (g->done) cudaEventDestroy(g->done);
    if (g->root) cudaStreamDestroy(g->root);
    delete g;
}

int lesgpu_group_create(lesgpu_ctx* const* ctxs, int n, lesgpu_group** out) {
    if (!ctxs || n < 1 || !out) return LESGPU_EINVAL;
    *out = nullptr;
    for (int q = 0; q < n; q++) {
        if (!ctxs[q]) return LESGPU_EINVAL;
        const DevCtx& d = ctxs[q]->d;
        if (!d.loop_ready) return fail(ctxs[q], LESGPU_ESTATE, "group members need lesgpu_loop_begin first");
        if (d.timing) return fail(ctxs[q], LESGPU_ESTATE, "group members must have kernel timing off");
        if (ctxs[q]->cfg.device != ctxs[0]->cfg.device)
            return fail(ctxs[q], LESGPU_EINVAL, "group members must share one device");
        for (int r = 0; r < q; r++)
            if (ctxs[r] == ctxs[q]) return fail(ctxs[q], LESGPU_EINVAL, "context listed twice in a group");
    }
    lesgpu_group* g = new (std::nothrow) lesgpu_group();
    if (!g) return LESGPU_ENOMEM;
    g->m.assign(ctxs, ctxs + n);
    g->device = ctxs[0]->cfg.device;
    lesgpu_ctx* c0 = ctxs[0];
    cudaError_t e = cudaSetDevice(g->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->root, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
    g->joins.assign(n, nullptr);
    g->ready.assign(n, nullptr);
    for (int q = 0; q < n && e == cudaSuccess; q++) {
        e = cudaEventCreateWithFlags(&g->joins[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ready[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctxs[q]->d.stream);
    }
    if (e != cudaSuccess) { int r = cuda_fail(c0, e, "group_create"); lesgpu_group_destroy(g); return r; }
    // capture: fork from the root stream into every member stream, one device-loop step per
    // member, join back into the root
    cudaGraph_t gr = nullptr;
    e = cudaStreamBeginCapture(g->root, cudaStreamCaptureModeThreadLocal);
    cudaError_t el = cudaSuccess;
    if (e == cudaSuccess) {
        el = cudaEventRecord(g->fork, g->root);
        for (int q = 0; q < n && el == cudaSuccess; q++) {
            DevCtx& d = ctxs[q]->d;
            el = cudaStreamWaitEvent(d.stream, g->fork, 0);
            if (el == cudaSuccess)
                el = (d.precision == LESGPU_FP64) ? les::step_f64(d, 0.0, 0, true) : les::step_f32(d, 0.0, 0, true);
            if (el == cudaSuccess) el = cudaEventRecord(g->joins[q], d.stream);
            if (el == cudaSuccess) el = cudaStreamWaitEvent(g->root, g->joins[q], 0);
        }
        cudaError_t ee = cudaStreamEndCapture(g->root, &gr);
        if (el == cudaSuccess) el = ee;
    } else {
        el = e;
    }
    if (el == cudaSuccess) el = cudaGraphInstantiate(&g->exec, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (el != cudaSuccess) {
        cudaGetLastError();
        int r = cuda_fail(c0, el, "group capture");
        lesgpu_group_destroy(g);
        return r;
    }
    *out = g;
    return LESGPU_OK;
}

int lesgpu_group_create_batched(lesgpu_ctx* const* ctxs, int n, int max_per_batch, lesgpu_group** out) {
    if (!ctxs || n < 1 || !out || max_per_batch < 0) return LESGPU_EINVAL;
    *out = nullptr;
    for (int q = 0; q < n; q++) {
        if (!ctxs[q]) return LESGPU_EINVAL;
        const DevCtx& d = ctxs[q]->d;
        if (!d.loop_ready) return fail(ctxs[q], LESGPU_ESTATE, "group members need lesgpu_loop_begin first");
        if (d.timing) return fail(ctxs[q], LESGPU_ESTATE, "group members must have kernel timing off");
        if (d.debug || d.grad_g || d.scalar_tma)
            return fail(ctxs[q], LESGPU_ESTATE, "batched members need inspection, |grad G| and the staged pass off");
        if (ctxs[q]->cfg.device != ctxs[0]->cfg.device)
            return fail(ctxs[q], LESGPU_EINVAL, "group members must share one device");
        for (int r = 0; r < q; r++)
            if (ctxs[r] == ctxs[q]) return fail(ctxs[q], LESGPU_EINVAL, "context listed twice in a group");
    }
    lesgpu_group* g = new (std::nothrow) lesgpu_group();
    if (!g) return LESGPU_ENOMEM;
    g->m.assign(ctxs, ctxs + n);
    g->device = ctxs[0]->cfg.device;
    lesgpu_ctx* c0 = ctxs[0];
    // batches: each member joins the first batch whose first member it matches and that has
    // room (at most max_per_batch members; 0: no limit)
    for (int q = 0; q < n; q++) {
        size_t b = 0;
        while (b < g->batches.size() &&
               (!batchable(ctxs[g->batches[b][0]]->d, ctxs[q]->d) ||
                (max_per_batch > 0 && (int)g->batches[b].size() >= max_per_batch)))
            b++;
        if (b == g->batches.size()) g->batches.emplace_back();
        g->batches[b].push_back(q);
    }
    const size_t nb = g->batches.size();
    cudaError_t e = cudaSetDevice(g->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->root, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
    g->joins.assign(n, nullptr);
    g->ready.assign(n, nullptr);
    g->heads.assign(n, nullptr);
    g->bstreams.assign(nb, nullptr);
    g->stages.assign(nb, nullptr);
    g->tabs.assign(nb, nullptr);
    for (int q = 0; q < n && e == cudaSuccess; q++) {
        e = cudaEventCreateWithFlags(&g->joins[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ready[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->heads[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctxs[q]->d.stream);
    }
    for (size_t b = 0; b < nb && e == cudaSuccess; b++) {
        e = cudaStreamCreateWithFlags(&g->bstreams[b], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->stages[b], cudaEventDisableTiming);
        std::vector<les::MemberTab> tab;
        const DevCtx& d0 = ctxs[g->batches[b][0]]->d;
        for (int q : g->batches[b]) tab.push_back(member_entry(d0, ctxs[q]->d));
        // from the stream-ordered pool, like every other device buffer (no device-wide
        // synchronisation when the group is destroyed)
        if (e == cudaSuccess)
            e = cudaMallocAsync((void**)&g->tabs[b], tab.size() * sizeof(les::MemberTab), g->root);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g->tabs[b], tab.data(), tab.size() * sizeof(les::MemberTab), cudaMemcpyHostToDevice,
                                g->root);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->root);
    }
    if (e != cudaSuccess) { int r = cuda_fail(c0, e, "group_create_batched"); lesgpu_group_destroy(g); return r; }
    // capture one step: every member's dt and draws (then its SEM plane) on its stream; each
    // batch's RK stages on the batch stream once its members' dt is set; every member's
    // boundary conditions and history on its stream once its batch is done
    cudaGraph_t gr = nullptr;
    e = cudaStreamBeginCapture(g->root, cudaStreamCaptureModeThreadLocal);
    cudaError_t el = cudaSuccess;
    if (e == cudaSuccess) {
        el = cudaEventRecord(g->fork, g->root);
        for (int q = 0; q < n && el == cudaSuccess; q++) {
            DevCtx& d = ctxs[q]->d;
            el = cudaStreamWaitEvent(d.stream, g->fork, 0);
            if (el == cudaSuccess) el = les::loop_pre(d);
            if (el == cudaSuccess) el = cudaEventRecord(g->heads[q], d.stream);
            if (el == cudaSuccess) el = les::sem_inflow(d, d.stream);
        }
        for (size_t b = 0; b < nb && el == cudaSuccess; b++) {
            for (int q : g->batches[b])
                if (el == cudaSuccess) el = cudaStreamWaitEvent(g->bstreams[b], g->heads[q], 0);
            DevCtx& d0 = ctxs[g->batches[b][0]]->d;
            const int nm = (int)g->batches[b].size();
            if (el == cudaSuccess)
                el = (d0.precision == LESGPU_FP64) ? les::batch_stages_f64(d0, g->tabs[b], nm, g->bstreams[b])
                                                   : les::batch_stages_f32(d0, g->tabs[b], nm, g->bstreams[b]);
            if (el == cudaSuccess) el = cudaEventRecord(g->stages[b], g->bstreams[b]);
            for (int q : g->batches[b]) {
                DevCtx& d = ctxs[q]->d;
                if (el == cudaSuccess) el = cudaStreamWaitEvent(d.stream, g->stages[b], 0);
                if (el == cudaSuccess)
                    el = (d.precision == LESGPU_FP64) ? les::batch_tail_f64(d) : les::batch_tail_f32(d);
                if (el == cudaSuccess) el = cudaEventRecord(g->joins[q], d.stream);
                if (el == cudaSuccess) el = cudaStreamWaitEvent(g->root, g->joins[q], 0);
            }
        }
        cudaError_t ee = cudaStreamEndCapture(g->root, &gr);
        if (el == cudaSuccess) el = ee;
    } else {
        el = e;
    }
    if (el == cudaSuccess) el = cudaGraphInstantiate(&g->exec, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (el != cudaSuccess) {
        cudaGetLastError();
        int r = cuda_fail(c0, el, "batched group capture");
        lesgpu_group_destroy(g);
        return r;
    }
    *out = g;
    return LESGPU_OK;
}

int lesgpu_group_batches(const lesgpu_group* g) { return g ? (int)(g->batches.empty() ? g->m.size() : g->batches.size()) : 0; }

int lesgpu_group_run(lesgpu_group* g, int nsteps) {
    if (!g || nsteps < 0) return LESGPU_EINVAL;
    if (nsteps == 0) return LESGPU_OK;
    for (lesgpu_ctx* c : g->m) {
        if (!c->d.loop_ready) return fail(c, LESGPU_ESTATE, "member's device-loop session has ended");
        if (nsteps > c->d.loop_cap) return fail(c, LESGPU_EINVAL, "nsteps exceeds a member's history capacity");
    }
    lesgpu_ctx* c0 = g->m[0];
    const int n = (int)g->m.size();
    // order after each member's earlier work, then restart every member's history slot
    for (int q = 0; q < n; q++) {
        DevCtx& d = g->m[q]->d;
        CKC(c0, cudaEventRecord(g->ready[q], d.stream));
        CKC(c0, cudaStreamWaitEvent(g->root, g->ready[q], 0));
        CKC(c0, cudaMemsetAsync((char*)d.dS + offsetof(les::Scalars, run_step), 0, sizeof(int), g->root));
    }
    for (int s = 0; s < nsteps; s++) CKC(c0, cudaGraphLaunch(g->exec, g->root));
    // later work on a member's stream (history read-back, sync) waits for the replays
    CKC(c0, cudaEventRecord(g->done, g->root));
    for (int q = 0; q < n; q++) CKC(c0, cudaStreamWaitEvent(g->m[q]->d.stream, g->done, 0));
    return LESGPU_OK;
}

}  // extern "C"
