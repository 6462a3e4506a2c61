// les_tma.cuh -- the scalar pass with its stencil fields staged in shared memory by the
// Tensor Memory Accelerator.
//
// The scalar pass reads six fields with a +-2 stencil in all three directions (filtered T and
// Y_k: MUSCL, Laplacian, SGS flux) and nu_t with +-1.  From global memory each cell issues
// ~13 loads per field, mostly L1/L2 hits whose latency the kernel cannot hide at its
// occupancy.  Here a block owns a 32 x 8 (k, j) tile and marches through a segment of
// i-planes: the (k, j) tile plus a 2-cell halo of each field, one i-plane at a time, is
// copied by cp.async.bulk.tensor into a ring of five shared-memory planes (three for nu_t),
// and the plane four ahead is in flight while the current one is computed.  Every value is
// fetched from global memory once per block; all stencil reads hit shared memory.
//
// Copies: one elected thread arms an mbarrier with the step's byte count and issues the
// seven tensor copies of the step (6 fields at plane p, nu_t at plane p - 1); all threads
// wait on the barrier's phase.  Halo coordinates outside the grid are filled with zeros by
// the copy engine (those values are never used by cells that compute).  Tile x-coordinates
// are multiples of 32 minus 2 (FP64) or 4 (FP32): 16-byte aligned, as tensor copies require.
// Every wait is bounded: a wait that runs out sets bit 4 of Scalars::nonfinite (read by the
// host), waits (bounded) for the copies already issued, and the block returns.
#pragma once

#include <cuda.h>

#include "les_kernels.cuh"

namespace les {

constexpr int TMA_TK = 32, TMA_TJ = 8;     // tile (k, j)
constexpr int TMA_RING = 5, TMA_NRING = 3; // planes kept for the +-2 and +-1 stencils
constexpr int TMA_NF = NSP + 1;            // staged +-2 fields: Y_0..Y_4, T

// Box geometry per field type: the x-extent covers k0 - 2 .. k0 + 33 and starts on a
// 16-byte boundary.
template <typename R>
struct TmaGeom {
    static constexpr int KOFF = (sizeof(R) == 8) ? 2 : 4;           // box starts at k0 - KOFF
    static constexpr int BW = (sizeof(R) == 8) ? 36 : 40;            // box width (k)
    static constexpr int BH = TMA_TJ + 4, BHN = TMA_TJ + 2;          // box heights (j)
    static constexpr int FBYTES = BW * BH * (int)sizeof(R);          // one field plane
    static constexpr int NBYTES = BW * BHN * (int)sizeof(R);         // one nu_t plane
    static constexpr int NSTRIDE = (NBYTES + 127) / 128 * 128;       // 128-byte aligned slots
    static constexpr int SMEM = TMA_NF * TMA_RING * FBYTES + TMA_NRING * NSTRIDE + 64 + 16;   // + barriers, flag
    static constexpr int STEP_BYTES = TMA_NF * FBYTES + NBYTES;
};

struct TmaMaps {
    CUtensorMap f[TMA_NF];     // Y_0..Y_4, T (filtered)
    CUtensorMap nut;
};

template <typename R, int NP>
struct SSrcPlanes {
    SAcc<R, 5> Yv[NSP], Tv;
    SAcc<R, 3> Nv;
    __device__ __forceinline__ const SAcc<R, 5>& y(int s) const { return Yv[s]; }
    __device__ __forceinline__ const SAcc<R, 5>& t() const { return Tv; }
    __device__ __forceinline__ const SAcc<R, 3>& nu() const { return Nv; }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One step of the ring: the six field planes at i-plane z and, when with_nu, the nu_t plane
// z - 1.  step_bytes counts all seven; without nu_t the barrier expects nu_bytes fewer.
__device__ __forceinline__ void tma_issue_step(const TmaMaps& M, uint32_t bar, uint32_t fdst0, uint32_t ndst,
                                               int fbytes_slot, int step_bytes, int nu_bytes, bool with_nu, int x,
                                               int y, int z) {
    const int bytes = with_nu ? step_bytes : step_bytes - nu_bytes;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
#pragma unroll
    for (int f = 0; f < TMA_NF; f++) {
        const uint64_t map = reinterpret_cast<uint64_t>(&M.f[f]);
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];" ::"r"(fdst0 + (uint32_t)(f * fbytes_slot)),
            "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
            : "memory");
    }
    if (!with_nu) return;
    const uint64_t nmap = reinterpret_cast<uint64_t>(&M.nut);
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(ndst),
        "l"(nmap), "r"(x), "r"(y + 1), "r"(z - 1), "r"(bar)
        : "memory");
}

// Bounded wait for `phase` of the barrier; false when the limit ran out.
__device__ __forceinline__ bool tma_wait(uint32_t bar, uint32_t phase) {
    for (int it = 0; it < (1 << 24); it++) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The scalar pass over a (32 x 8) tile and i-planes [blockIdx.z * iseg, + iseg).
template <typename R, typename RS>
__global__ void __launch_bounds__(TMA_TK* TMA_TJ, (sizeof(R) == 8) ? 2 : 3)
    k_rhs_scalar_tma(LES_KERNEL_CONSTS, const __grid_constant__ TmaMaps M, const uint8_t* __restrict__ attr, F11<R> F,
                     PropBuf<R> P, F11<RS> S0, F11<R> St, AccBuf<R> acc, KFlow<R> kf, KDbg<R> kd,
                     Scalars* __restrict__ Sc, int stage, int iseg) {
    using G = TmaGeom<R>;
    extern __shared__ __align__(128) unsigned char tma_smem[];
    R* fring = reinterpret_cast<R*>(tma_smem);                                          // [NF][RING][BH][BW]
    unsigned char* nbase = tma_smem + TMA_NF * TMA_RING * G::FBYTES;                   // [NRING] slots
    uint64_t* bars = reinterpret_cast<uint64_t*>(nbase + TMA_NRING * G::NSTRIDE);      // [RING]
    int& abort_flag = *reinterpret_cast<int*>(bars + 8);

    const int tid = threadIdx.y * TMA_TK + threadIdx.x;
    const int k0 = blockIdx.x * TMA_TK, j0 = blockIdx.y * TMA_TJ;
    const int i0 = blockIdx.z * iseg;
    const int i1 = min(i0 + iseg, C.nx);
    const int x = k0 - G::KOFF, y = j0 - 2;
    const int nsteps = (i1 - i0) + 4;      // field planes i0-2 .. i1+1

    if (tid == 0) {
        abort_flag = 0;
        for (int b = 0; b < TMA_RING; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t fdst = smem_u32(fring);
    const uint32_t ndst = smem_u32(nbase);
    // ring slot of field plane at step r: r % RING (RING planes apart per field f: f * RING + slot).
    // Step r also brings nu_t plane i0 - 3 + r into slot r % NRING.  The prologue issues RING
    // steps at once, so steps 0 and 1 would share nu_t slots with steps 3 and 4 while both
    // copies are in flight (their completion order is not defined); their planes i0 - 3 and
    // i0 - 2 are never read, so those two steps bring no nu_t.
    int issued = 0;   // steps issued (thread 0)
    auto issue = [&](int r) {
        issued = r + 1;
        const int slot = r % TMA_RING, nslot = r % TMA_NRING;
        tma_issue_step(M, smem_u32(&bars[slot]), fdst + (uint32_t)(slot * G::FBYTES),
                       ndst + (uint32_t)(nslot * G::NSTRIDE), TMA_RING * G::FBYTES, G::STEP_BYTES, G::NBYTES,
                       r >= 2, x, y, i0 - 2 + r);
    };
    if (tid == 0) {
        const int pro = nsteps < TMA_RING ? nsteps : TMA_RING;
        for (int r = 0; r < pro; r++) issue(r);
    }
    int waited = 0;   // steps waited so far (each step is waited exactly once)
    const int kl = threadIdx.x, jl = threadIdx.y;
    const int k = k0 + kl, j = j0 + jl;
    for (int i = i0; i < i1; i++) {
        const int rc = i - i0 + 2;                  // step of the centre plane
        // wait for every step up to rc + 2
        bool ok = true;
        while (waited <= rc + 2 && waited < nsteps) {
            if (!tma_wait(smem_u32(&bars[waited % TMA_RING]), (uint32_t)((waited / TMA_RING) & 1))) {
                ok = false;
                break;
            }
            waited++;
        }
        if (!ok) atomicOr(&abort_flag, 1);
        __syncthreads();
        if (abort_flag) break;
        // the operands of the next plane that stay in global memory, requested into L2 while
        // this plane is computed (staged pass 4.49 -> 4.03 ms per 256x128x128 step in FP64,
        // 2.52 -> 2.07 in FP32)
        if (k < C.nz && j < C.ny && i + 1 < i1) {
            const size_t idn = cid(i + 1, j, k, C.ny, C.nz);
#pragma unroll
            for (int q = 0; q < NSTATE; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(S0.p[q] + idn));
            if (stage > 0) {
#pragma unroll
                for (int q = 0; q < NACC; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(acc.p[q] + idn));
            }
#pragma unroll
            for (int q = 0; q < 4; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(kf.p[q] + idn));
#pragma unroll
            for (int q = 0; q < NSP; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(P.D[q] + idn));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(P.aT + idn));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(attr + idn));
#pragma unroll
            for (int q = 0; q < 5; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(F.p[q] + idn));
        }
        if (k < C.nz && j < C.ny) {
            SSrcPlanes<R, 5> src;
#pragma unroll
            for (int d = 0; d < 5; d++) {
                const int slot = (rc - 2 + d) % TMA_RING;
                const int off = (jl + 2) * G::BW + (kl + G::KOFF);
#pragma unroll
                for (int s = 0; s < NSP; s++) src.Yv[s].pl[d] = fring + (size_t)(s * TMA_RING + slot) * (G::FBYTES / sizeof(R)) + off;
                src.Tv.pl[d] = fring + (size_t)(NSP * TMA_RING + slot) * (G::FBYTES / sizeof(R)) + off;
            }
#pragma unroll
            for (int s = 0; s < NSP; s++) src.Yv[s].bw = G::BW;
            src.Tv.bw = G::BW;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int nslot = (rc - 1 + d + 1) % TMA_NRING;   // nu plane i-1+d arrived with step rc-1+d+1
                src.Nv.pl[d] = reinterpret_cast<const R*>(nbase + nslot * G::NSTRIDE) + (jl + 1) * G::BW +
                               (kl + G::KOFF);
            }
            src.Nv.bw = G::BW;
            rhs_scalar_cell<R, RS>(C, attr, F, P, S0, St, acc, kf, kd, Sc, stage, i, j, k, src, (R)kc<R>(C).relax);
        }
        __syncthreads();                            // the plane of step rc - 2 is free
        if (tid == 0 && rc + 3 < nsteps) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(rc + 3);
        }
    }
    if (abort_flag) {
        // drain the copies already issued (bounded) before the block's shared memory goes away
        if (tid == 0) {
            for (int r = waited; r < issued; r++) tma_wait(smem_u32(&bars[r % TMA_RING]), (uint32_t)((r / TMA_RING) & 1));
            atomicOr(&Sc->nonfinite, 4);
        }
    }
}

// Launch of the staged scalar pass: i-segments sized so that the grid is about two waves of
// resident blocks (at least 4 planes per segment).
template <typename R, typename RS>
cudaError_t launch_scalar_tma(const DevCtx& c, cudaStream_t st, const F11<R>& F, const PropBuf<R>& P,
                              const F11<RS>& S, const F11<R>& St, const AccBuf<R>& acc, const KFlow<R>& kf,
                              const KDbg<R>& kd, int stage) {
    using G = TmaGeom<R>;
    const int gx = (c.nz + TMA_TK - 1) / TMA_TK, gy = (c.ny + TMA_TJ - 1) / TMA_TJ;
    const long long target = 148LL * ((sizeof(R) == 8) ? 2 : 3) * 2;
    long long iseg = ((long long)c.nx * gx * gy + target - 1) / target;
    if (iseg < 4) iseg = 4;
    if (iseg > c.nx) iseg = c.nx;
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)((c.nx + iseg - 1) / iseg));
    k_rhs_scalar_tma<R, RS><<<grid, dim3(TMA_TK, TMA_TJ), G::SMEM, st>>>(
        c.hC, *reinterpret_cast<const TmaMaps*>(c.tma_maps), c.attr, F, P, S, St, acc, kf, kd, c.dS, stage, (int)iseg);
    return cudaGetLastError();
}

// Once per process and instantiation: allow the staged kernel its dynamic shared memory.
template <typename R, typename RS>
cudaError_t prepare_scalar_tma() {
    return cudaFuncSetAttribute(k_rhs_scalar_tma<R, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TmaGeom<R>::SMEM);
}

}  // namespace les
