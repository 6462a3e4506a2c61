// les_pstat.cu -- profile statistics of the probe rows, accumulated on the device from the
// device loop's history, so that an ensemble member or a served request needs no probe file.
//
// The rows are those record_flame_region_data writes (les_combustion_solver.c:3403-3471): on
// each probe station's line k = NZ/2, the lower crossing of G = 0.5 gives y_flame (linear
// interpolation, :3419-3434); if y_flame > 0 every row j with |j*DY - y_flame| <= 1.0 m is a
// sample (u, v, w, G).  The statistics are the ones the reference's post-processing draws
// from those rows, kept as moment sums over the whole run:
//
//   global          N, sum u, sum v, sum w                       (the means of analysis.py:118)
//   y bins          per flame-distance bin (e_b, e_b+1] in mm: n, sum u, v, w, G, uu, vv, ww, uv
//                   (analysis.py:112-130, fluctuations about the global means)
//   G bins (right)  per (e_b, e_b+1]: n, sum u, v, w, uu, vv, uv  (analysis.py:218-236)
//   G bins (half)   per [e_b, e_b+1): n, sum u, v, uv              (bayesian_optimizer.py:98-117)
//   PDFs            counts of u and v per [e_b, e_b+1) (last bin closed), unburnt G < 0.5 and
//                   burnt G >= 0.5                                 (analysis.py:82-110)
//
// Sums are in FP64 and deterministic: one warp per output bin scans the chunk's rows in a
// fixed order and reduces with a fixed shuffle tree.  Built without FMA contraction, so
// y_flame has the host writer's bits.
#include "les_ctx.h"

namespace les {

namespace {

constexpr int PS_Y = 9, PS_RC = 7, PS_HO = 4;   // moments per bin of each kind
constexpr int ROWBIN = 5;                        // y, G right-closed, G half-open, u, v

struct PsView {
    const double* ey;   // ny + 1
    const double* erc;  // ngrc + 1
    const double* eho;  // ngho + 1
    const double* eu;   // npdf + 1
    const double* ev;   // npdf + 1
    int ny, ngrc, ngho, npdf;
};

__device__ __forceinline__ PsView ps_view(const double* e, int ny, int ngrc, int ngho, int npdf) {
    PsView v;
    v.ey = e;
    v.erc = v.ey + ny + 1;
    v.eho = v.erc + ngrc + 1;
    v.eu = v.eho + ngho + 1;
    v.ev = v.eu + npdf + 1;
    v.ny = ny; v.ngrc = ngrc; v.ngho = ngho; v.npdf = npdf;
    return v;
}

// First index i with e[i] >= x (numpy searchsorted, side='left').
__device__ __forceinline__ int lower_bound(const double* e, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// First index i with e[i] > x (side='right').
__device__ __forceinline__ int upper_bound(const double* e, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// (e_b, e_b+1]: pandas.cut's default, -1 outside.
__device__ __forceinline__ int bin_right_closed(const double* e, int nb, double x) {
    if (!(x > e[0]) || x > e[nb]) return -1;
    return lower_bound(e, nb + 1, x) - 1;
}
// [e_b, e_b+1): the optimiser's bins, -1 outside (so x == e_nb is in no bin).
__device__ __forceinline__ int bin_half_open(const double* e, int nb, double x) {
    if (!(x >= e[0]) || !(x < e[nb])) return -1;
    return upper_bound(e, nb + 1, x) - 1;
}
// numpy.histogram: [e_b, e_b+1) with the last bin closed, -1 outside.
__device__ __forceinline__ int bin_histogram(const double* e, int nb, double x) {
    if (!(x >= e[0]) || !(x <= e[nb])) return -1;
    const int b = upper_bound(e, nb + 1, x) - 1;
    return b < nb ? b : nb - 1;
}

// y_flame of every (step, probe line): the lower G = 0.5 crossing (:3419-3434), -1 if none.
__global__ void k_ps_lines(const double* __restrict__ hist, int nsteps, int L, int m, int ny, double dy,
                           double* __restrict__ yfl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsteps * m) return;
    const int q = t / m, l = t % m;
    const double* row = hist + ((size_t)q * L + l) * ny * 6;
    double y_flame = -1.0;
    for (int j = 0; j < ny - 1; j++) {
        const double G1 = row[6 * j + 3], G2 = row[6 * (j + 1) + 3];
        if ((G1 - 0.5) * (G2 - 0.5) <= 0.0) {
            const double y1 = j * dy, y2 = (j + 1) * dy;
            if (fabs(G2 - G1) < 1e-9) y_flame = y1;
            else y_flame = y1 + (0.5 - G1) / (G2 - G1) * (y2 - y1);
            break;
        }
    }
    yfl[t] = y_flame;
}

// Bin indices of every row; rows that record_flame_region_data would not write get y bin -2.
__global__ void k_ps_rows(const double* __restrict__ hist, int nsteps, int L, int m, int ny, double dy,
                          const double* __restrict__ yfl, const double* __restrict__ edges, int nyb, int ngrc, int ngho,
                          int npdf, int* __restrict__ rowbin) {
    const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t R = (size_t)nsteps * m * ny;
    if (r >= R) return;
    const int j = (int)(r % ny);
    const size_t line = r / ny;
    const int q = (int)(line / m), l = (int)(line % m);
    const PsView e = ps_view(edges, nyb, ngrc, ngho, npdf);
    int* out = rowbin + r * ROWBIN;
    const double y_flame = yfl[line];
    const double y_rel = j * dy - y_flame;
    if (!(y_flame > 0.0) || !(fabs(y_rel) <= 1.0)) {    // SAMPLING_RANGE (:280, :3451)
        out[0] = -2; out[1] = -1; out[2] = -1; out[3] = -1; out[4] = -1;
        return;
    }
    const double* c = hist + (((size_t)q * L + l) * ny + j) * 6;
    const double u = c[0], v = c[1], G = c[3];
    out[0] = bin_right_closed(e.ey, nyb, y_rel * 1000.0);
    out[1] = bin_right_closed(e.erc, ngrc, G);
    out[2] = bin_half_open(e.eho, ngho, G);
    const int burnt = (G >= 0.5) ? npdf : 0;            // analysis.py:90-91: G < 0.5 unburnt
    const int bu = bin_histogram(e.eu, npdf, u), bv = bin_histogram(e.ev, npdf, v);
    out[3] = bu >= 0 ? bu + burnt : -1;
    out[4] = bv >= 0 ? bv + burnt : -1;
}

__device__ __forceinline__ double warp_sum(double x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    return x;
}

// One warp per output group: the global sums, then every bin of every kind.
__global__ void k_ps_reduce(const double* __restrict__ hist, int nsteps, int L, int m, int ny,
                            const int* __restrict__ rowbin, int nyb, int ngrc, int ngho, int npdf,
                            double* __restrict__ sums) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int ngroups = 1 + nyb + ngrc + ngho + 4 * npdf;
    if (warp >= ngroups) return;
    int kind, b;
    if (warp == 0) { kind = 0; b = 0; }
    else if (warp < 1 + nyb) { kind = 1; b = warp - 1; }
    else if (warp < 1 + nyb + ngrc) { kind = 2; b = warp - 1 - nyb; }
    else if (warp < 1 + nyb + ngrc + ngho) { kind = 3; b = warp - 1 - nyb - ngrc; }
    else { kind = 4; b = warp - 1 - nyb - ngrc - ngho; }    // 0 .. 4 npdf - 1
    // PDF groups: [u unburnt | v unburnt | u burnt | v burnt], npdf each
    const int pdf_var = (kind == 4) ? ((b / npdf) & 1) : 0;            // 0: u, 1: v
    const int pdf_code = (kind == 4) ? ((b % npdf) + ((b / (2 * npdf)) ? npdf : 0)) : 0;
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const size_t R = (size_t)nsteps * m * ny;
    for (size_t r = lane; r < R; r += 32) {
        const int* rb = rowbin + r * ROWBIN;
        bool take;
        switch (kind) {
            case 0: take = rb[0] != -2; break;
            case 1: take = rb[0] == b; break;
            case 2: take = rb[1] == b; break;
            case 3: take = rb[2] == b; break;
            default: take = rb[3 + pdf_var] == pdf_code; break;
        }
        if (!take) continue;
        const int j = (int)(r % ny);
        const size_t line = r / ny;
        const double* c = hist + (((size_t)(line / m) * L + (int)(line % m)) * ny + j) * 6;
        const double u = c[0], v = c[1], w = c[2], G = c[3];
        a[0] += 1.0;
        if (kind == 0) { a[1] += u; a[2] += v; a[3] += w; }
        else if (kind == 1) {
            a[1] += u; a[2] += v; a[3] += w; a[4] += G;
            a[5] += u * u; a[6] += v * v; a[7] += w * w; a[8] += u * v;
        } else if (kind == 2) {
            a[1] += u; a[2] += v; a[3] += w; a[4] += u * u; a[5] += v * v; a[6] += u * v;
        } else if (kind == 3) {
            a[1] += u; a[2] += v; a[3] += u * v;
        }
    }
    const int nmom = kind == 0 ? 4 : kind == 1 ? PS_Y : kind == 2 ? PS_RC : kind == 3 ? PS_HO : 1;
    size_t off;
    switch (kind) {
        case 0: off = 0; break;
        case 1: off = 4 + (size_t)b * PS_Y; break;
        case 2: off = 4 + (size_t)nyb * PS_Y + (size_t)b * PS_RC; break;
        case 3: off = 4 + (size_t)nyb * PS_Y + (size_t)ngrc * PS_RC + (size_t)b * PS_HO; break;
        default: off = 4 + (size_t)nyb * PS_Y + (size_t)ngrc * PS_RC + (size_t)ngho * PS_HO + b; break;
    }
    for (int k = 0; k < nmom; k++) {
        const double s = warp_sum(a[k]);
        if (lane == 0) sums[off + k] += s;
    }
}

}  // namespace

cudaError_t pstat_accumulate(DevCtx& c, int nsteps, int m) {
    if (!c.ps_on || nsteps <= 0 || m <= 0) return cudaSuccess;
    if (m > c.loop_nst || nsteps > c.loop_cap) return cudaErrorInvalidValue;
    const size_t lines = (size_t)nsteps * m, rows = lines * c.ny;
    if (rows > c.ps_rows_cap) return cudaErrorInvalidValue;
    const int tpb = 256;
    k_ps_lines<<<(unsigned)((lines + tpb - 1) / tpb), tpb, 0, c.stream>>>(c.hist_probe, nsteps, c.loop_nst, m, c.ny,
                                                                          c.hC.dy, c.ps_yflame);
    k_ps_rows<<<(unsigned)((rows + tpb - 1) / tpb), tpb, 0, c.stream>>>(c.hist_probe, nsteps, c.loop_nst, m, c.ny,
                                                                        c.hC.dy, c.ps_yflame, c.ps_edges, c.ps_ny,
                                                                        c.ps_ngrc, c.ps_ngho, c.ps_npdf, c.ps_rowbin);
    const int ngroups = 1 + c.ps_ny + c.ps_ngrc + c.ps_ngho + 4 * c.ps_npdf;
    k_ps_reduce<<<(unsigned)((ngroups * 32 + tpb - 1) / tpb), tpb, 0, c.stream>>>(
        c.hist_probe, nsteps, c.loop_nst, m, c.ny, c.ps_rowbin, c.ps_ny, c.ps_ngrc, c.ps_ngho, c.ps_npdf, c.ps_sums);
    return cudaGetLastError();
}

}  // namespace les
