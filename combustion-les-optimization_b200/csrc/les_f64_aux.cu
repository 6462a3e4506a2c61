// les_f64_aux.cu -- the parts of a step that both precision forms share and that must give
// the host's bits: the SEM inflow plane (bit-identical to the reference's plane for the same
// vortices), the device-loop dt and rand() draws (bit-identical to the host-driven loop), and
// the division self-check.  Always built with -fmad=false, whatever the stage kernels use.
#include <vector>

#include "les_ctx.h"
#include "les_sem.cuh"
#include "les_devloop.cuh"

namespace les {

cudaError_t sem_inflow(DevCtx& c, cudaStream_t st) {
    if (c.n_inlet <= 0) return cudaSuccess;
    const int tpb = 128;
    k_sem_plane<<<(c.n_inlet + tpb - 1) / tpb, tpb, 7 * 512 * sizeof(double), st>>>(c.dC, c.inlet_list, c.n_inlet,
                                                                                   c.vort, c.nv, c.plane);
    k_sem_normalize<<<1, 256, 0, st>>>(c.dC, c.inlet_list, c.n_inlet, c.plane, c.dS);
    return cudaGetLastError();
}

// Checks cdv() against IEEE division: n pseudo-random dividends spanning 2^-60..2^60 for
// each divisor; counts quotients whose bit patterns differ.
__global__ void k_selfcheck_div(const DC* __restrict__ ds, int nd, size_t n, unsigned long long seed,
                                unsigned long long* __restrict__ bad) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    for (int d = 0; d < nd; d++) {
        const DC dc = ds[d];
        for (size_t q = tid; q < n; q += stride) {
            unsigned long long z = seed + q * 0x9E3779B97F4A7C15ull + (unsigned long long)d * 0xD1B54A32D192ED03ull;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            unsigned long long e = (unsigned long long)(1023 - 60 + (int)((z >> 52) % 121));
            unsigned long long bits = (z & 0x000FFFFFFFFFFFFFull) | (e << 52) | ((z >> 63) << 63);
            double x = __longlong_as_double((long long)bits);
            if (__double_as_longlong(x / dc.c) != __double_as_longlong(cdv(x, dc))) local++;
        }
    }
    if (local) atomicAdd(bad, local);
}

int selfcheck_division(const double* divisors, int nd, size_t n, unsigned long long seed, unsigned long long* bad) {
    DC* dd = nullptr;
    unsigned long long* db = nullptr;
    std::vector<DC> h(nd);
    for (int q = 0; q < nd; q++) { h[q].c = divisors[q]; h[q].r = 1.0 / divisors[q]; }
    if (cudaMalloc(&dd, nd * sizeof(DC)) != cudaSuccess) return -3;
    if (cudaMalloc(&db, sizeof(unsigned long long)) != cudaSuccess) { cudaFree(dd); return -3; }
    cudaMemcpy(dd, h.data(), nd * sizeof(DC), cudaMemcpyHostToDevice);
    cudaMemset(db, 0, sizeof(unsigned long long));
    k_selfcheck_div<<<1184, 256>>>(dd, nd, n, seed, db);
    cudaError_t e = cudaMemcpy(bad, db, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(dd);
    cudaFree(db);
    return e == cudaSuccess ? 0 : -2;
}

cudaError_t loop_pre(DevCtx& c) {
    k_loop_pre<<<1, LOOP_THREADS, 0, c.stream>>>(c.dC, c.dS, (LoopState*)c.dL, c.J, c.jrows, c.vort, c.nv, c.noise,
                                                 c.n_inlet, c.lp_lbox, c.lp_ly, c.lp_lz, c.lp_uin, c.lp_ti, c.lp_ell,
                                                 c.lp_cfl, c.lp_cfld, c.lp_dx);
    return cudaGetLastError();
}

}  // namespace les
