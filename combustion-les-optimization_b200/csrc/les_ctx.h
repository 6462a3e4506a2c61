// les_ctx.h -- device context shared by the C-ABI layer and the per-precision launchers.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "les_common.cuh"

namespace les {

// Thread-block tiles of the per-cell kernels, (k extent, j extent, i extent).  Every kernel
// indexes through blockDim, so the tile is a launch parameter chosen per kernel class
// (lesgpu_set_tiles / lesgpu_autotune); the results do not depend on it except through the
// order of the block partial sums of <rho_f>.  Tiles spanning several i-planes keep the
// i-neighbours a block reads in its own SM's L1.  The first NSHAPES_256 tiles have 256
// threads and serve every class; the 512-thread tiles after them serve the classes without
// block reductions (strain, flow, scalar), whose kernels are instantiated for both sizes: a
// larger tile reads fewer halo cells per cell it computes, so the resident blocks' stencil
// tiles take less of L1 (the scalar pass at 256x128x128 on B200: 0.71 ms per launch with
// 16x4x8 against 0.75 with the best 256-thread tile; 1024-thread tiles were no faster in
// FP64 and slower in FP32).
struct Shape {
    int bx, by, bz;
};
constexpr int NSHAPES_256 = 8;
constexpr int NSHAPES = 13;
constexpr Shape kShapes[NSHAPES] = {{32, 8, 1}, {64, 4, 1}, {16, 16, 1}, {128, 2, 1}, {32, 4, 2},
                                    {16, 8, 2}, {32, 2, 4}, {16, 4, 4}, {32, 8, 2}, {32, 4, 4},
                                    {16, 8, 4}, {16, 4, 8}, {64, 4, 2}};
enum { SH_FILTER = 0, SH_STRAIN = 1, SH_FLOW = 2, SH_SCALAR = 3, SH_EOS = 4, NSH_CLASSES = 5 };
constexpr int shape_threads(int s) { return kShapes[s].bx * kShapes[s].by * kShapes[s].bz; }
// whether tile s may serve kernel class cls (the filter and EOS kernels reduce over 256-thread blocks)
constexpr bool shape_allowed(int cls, int s) {
    return s >= 0 && s < NSHAPES && (s < NSHAPES_256 || (cls != SH_FILTER && cls != SH_EOS));
}

inline size_t blocks_for_shape(int nx, int ny, int nz, int s) {
    const Shape t = kShapes[s];
    return (size_t)((nz + t.bx - 1) / t.bx) * (size_t)((ny + t.by - 1) / t.by) * (size_t)((nx + t.bz - 1) / t.bz);
}
inline size_t max_cell_blocks(int nx, int ny, int nz) {
    size_t m = 0;
    for (int s = 0; s < NSHAPES; s++) {
        size_t b = blocks_for_shape(nx, ny, nz, s);
        if (b > m) m = b;
    }
    return m;
}

struct DevCtx {
    int nx = 0, ny = 0, nz = 0, precision = 0;
    size_t n = 0;                       // cells
    size_t esz = 8;                     // bytes per field value
    Consts hC{};                        // host copy of the constants
    Consts* dC = nullptr;
    Scalars* dS = nullptr;
    uint8_t* attr = nullptr;
    void* S[NSTATE] = {};               // state Phi_n (updated in place by the final combine)
    void* St[NSTATE] = {};              // stage state (u_temp, ..., rho_temp)
    void* F[NSTATE] = {};               // filtered stage fields
    void* mu_mix = nullptr;
    void* nu = nullptr;
    void* D[NSP] = {};
    void* aT = nullptr;
    void* nu_t = nullptr;
    void* S_mag = nullptr;
    void* ST = nullptr;
    void* mu_eff = nullptr;
    void* acc[NACC] = {};
    void* kflow[4] = {};                // momentum and G right-hand sides of the stage
    void* dbg_cp = nullptr;             // optional inspection buffers (lesgpu_get_field)
    void* dbg_lam = nullptr;
    void* dbg_alpha = nullptr;
    void* kd[NACC] = {};
    void* grad_g = nullptr;             // optional |grad G| field (lesgpu_keep_grad_g)
    bool debug = false;
    double* part = nullptr;             // per-block partials of the reductions
    size_t part_len = 0;
    double* plane = nullptr;            // SEM fluctuation planes, 3 x NY x NZ
    double* noise = nullptr;            // packed white noise, 3 per inlet cell
    double* vort = nullptr;             // vortices, 7 doubles each
    int nv_cap = 0;
    int nv = 0;
    int* inlet_list = nullptr;          // plane index j*NZ+k of inlet cells, (j,k) order
    int* inlet_pos = nullptr;           // plane index -> position in inlet_list (or -1)
    int n_inlet = 0;
    std::vector<int> h_inlet;           // host copy of inlet_list
    int* probe_st = nullptr;
    double* probe_out = nullptr;
    int probe_cap = 0;
    int* flag = nullptr;
    void* arena = nullptr;              // one allocation backing all fields (256-byte aligned)
    void* arena_raw = nullptr;          // the pool allocation it starts in
    size_t arena_bytes = 0;
    size_t total_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;        // SEM plane, overlapped with the RK stages
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double* h_pinned = nullptr;         // pinned staging for small transfers
    size_t h_pinned_len = 0;
    bool have_attr = false, have_state = false, have_inflow = false;
    // device-resident time loop (les_devloop.cuh)
    bool loop_ready = false;
    unsigned int* J = nullptr;          // rand() jump-ahead rows, jrows x 31
    int jrows = 0;
    void* dL = nullptr;                 // LoopState
    int* loop_st = nullptr;             // probe stations
    int loop_nst = 0, loop_kline = 0, loop_cap = 0;
    double* hist_probe = nullptr;       // cap x nst x NY x 6
    double* hist_dt = nullptr;          // cap
    double* hist_umax = nullptr;        // cap
    double* hist_mon = nullptr;         // cap x 6
    double lp_lbox = 0, lp_ly = 0, lp_lz = 0, lp_uin = 0, lp_ti = 0, lp_ell = 0, lp_cfl = 0, lp_cfld = 0, lp_dx = 0;
    cudaGraphExec_t graph = nullptr;    // one captured device-loop step
    bool graph_ok = false;
    int shape[NSH_CLASSES] = {0, 0, 0, 0, 0};   // tile (index into kShapes) per kernel class
    // scalar pass with TMA-staged stencil fields (les_tma.cuh): tensor maps of the six
    // filtered scalars and nu_t (7 CUtensorMap, 128 bytes each), built at create time
    alignas(64) unsigned char tma_maps[7 * 128] = {};
    bool tma_ok = false;                // maps built (row stride a multiple of 16 bytes)
    bool scalar_tma = false;            // the scalar pass uses them
    // time averages (lesgpu_avg_*): NAVG running sums, FP64, in one allocation
    double* avg = nullptr;
    int avg_start = 0;
    // profile statistics of the probe rows (lesgpu_pstat_*, les_pstat.cu): bin edges, the
    // running moment sums, and per-row scratch for one history chunk
    bool ps_on = false;
    int ps_ny = 0, ps_ngrc = 0, ps_ngho = 0, ps_npdf = 0;   // bins of each kind
    double* ps_edges = nullptr;         // y (mm), G right-closed, G half-open, u, v edges
    double* ps_sums = nullptr;          // moment sums (lesgpu_pstat_read layout)
    size_t ps_nsums = 0;
    double* ps_yflame = nullptr;        // y_flame per history line (cap x lines)
    int* ps_rowbin = nullptr;           // 5 bin indices per row (cap x lines x NY)
    size_t ps_rows_cap = 0;
    // kernel timing: event pairs recorded around each kernel class during a step
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_cls;            // class of each recorded pair
    int ev_used = 0;
    cudaEvent_t marks[16] = {};
    double kms[8] = {0};
    long long kcount[8] = {0};
    std::string err;
};

// Storage size of the tensor maps (7 CUtensorMap of 128 bytes).
struct TmaMapsStorage {
    unsigned char b[7 * 128];
};

// Profile statistics (les_pstat.cu): accumulate the rows of the last nsteps history slots
// (the first m lines, the probe stations) into ps_sums, on the context's stream.
cudaError_t pstat_accumulate(DevCtx& c, int nsteps, int m);

// Kernel-timing helpers (les_api.cu): tmark_begin returns a pair slot or -1.
int tmark_begin(DevCtx& c, int cls);
void tmark_end(DevCtx& c, int slot);
void tmark_flush(DevCtx& c);

// Per-precision entry points (les_f64.cu / les_f32.cu).
cudaError_t sem_inflow(DevCtx& c, cudaStream_t st);
int selfcheck_division(const double* divisors, int nd, size_t n, unsigned long long seed, unsigned long long* bad);
cudaError_t loop_pre(DevCtx& c);
cudaError_t step_f64(DevCtx& c, double dt, int t_loop, bool device_mode);
cudaError_t umax_f64(DevCtx& c);
cudaError_t monitor_f64(DevCtx& c);
cudaError_t probe_f64(DevCtx& c, int n, int kline);
cudaError_t check_f64(DevCtx& c, int field);
cudaError_t rhs_only_f64(DevCtx& c, int t_loop);
cudaError_t step_f32(DevCtx& c, double dt, int t_loop, bool device_mode);
// Batched members (les_launch.cuh): step head and tail of one member, the RK stages of nmem
// members of one shape in one launch per pass.
cudaError_t batch_head_f64(DevCtx& c);
cudaError_t batch_tail_f64(DevCtx& c);
cudaError_t batch_stages_f64(DevCtx& c0, const MemberTab* mt, int nmem, cudaStream_t st);
cudaError_t batch_head_f32(DevCtx& c);
cudaError_t batch_tail_f32(DevCtx& c);
cudaError_t batch_stages_f32(DevCtx& c0, const MemberTab* mt, int nmem, cudaStream_t st);
cudaError_t rhs_only_f32(DevCtx& c, int t_loop);
cudaError_t umax_f32(DevCtx& c);
cudaError_t monitor_f32(DevCtx& c);
cudaError_t probe_f32(DevCtx& c, int n, int kline);
cudaError_t check_f32(DevCtx& c, int field);
cudaError_t prepare_tma_f64();
cudaError_t prepare_tma_f32();

}  // namespace les
