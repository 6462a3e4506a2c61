// les_sem.cuh -- synthetic-eddy inflow plane kernels.  Compiled only into the FP64 unit
// (no FMA contraction) and shared by both precision forms: the plane is always FP64.
#pragma once

#include "les_common.cuh"

namespace les {

// ------------------------------------------------------------------ SEM inflow plane

// generate_inlet_turbulence_SEM plane sum (:965-1003): one thread per inlet cell, vortices
// summed in index order so every cell's value is the reference's serial sum.
__global__ void k_sem_plane(const Consts* __restrict__ C, const int* __restrict__ inlet_list, int n_inlet,
                            const double* __restrict__ vort, int nv, double* __restrict__ plane) {
    extern __shared__ double sv[];   // staged vortices, 7 doubles each
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int ny = C->ny, nz = C->nz;
    const size_t npl = (size_t)ny * nz;
    int p = (q < n_inlet) ? inlet_list[q] : 0;
    const int j = p / nz, k = p % nz;
    const double y = j * C->dy, z = k * C->dz;
    double su = 0.0, svv = 0.0, sw = 0.0;
    const int chunk = 512;
    for (int base = 0; base < nv; base += chunk) {
        const int m = min(chunk, nv - base);
        __syncthreads();
        for (int t = threadIdx.x; t < 7 * m; t += blockDim.x) sv[t] = vort[7 * (size_t)base + t];
        __syncthreads();
        if (q < n_inlet) {
            for (int v = 0; v < m; v++) {
                const double* V = &sv[7 * v];
                double ddx = 0.0 - V[0];
                double ddy = y - V[1];
                double ddz = z - V[2];
                double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                double rad = V[3];
                if (dist < rad) {
                    double infl = 1.0 - (dist / rad);
                    su += V[4] * infl;
                    svv += V[5] * infl;
                    sw += V[6] * infl;
                }
            }
        }
    }
    if (q < n_inlet) {
        plane[p] = su;
        plane[npl + p] = svv;
        plane[2 * npl + p] = sw;
    }
}

// Mean removal and rms rescale (:1005-1074).  The three running sums are serial, in the
// reference's (j, k) order, so the plane is bit-identical to the reference's.
__global__ void k_sem_normalize(const Consts* __restrict__ C, const int* __restrict__ inlet_list, int n_inlet,
                                double* __restrict__ plane, Scalars* __restrict__ Sc) {
    __shared__ double tot[3];
    const size_t npl = (size_t)C->ny * C->nz;
    const int t = threadIdx.x;
    if (n_inlet <= 0) return;
    if (t < 3) {
        double s = 0.0;
        const double* pl = plane + t * npl;
        for (int q = 0; q < n_inlet; q++) s += pl[inlet_list[q]];
        tot[t] = s / n_inlet;
        Sc->sem[t] = s;
    }
    __syncthreads();
    for (int q = t; q < n_inlet; q += blockDim.x) {
        const int p = inlet_list[q];
        plane[p] -= tot[0];
        plane[npl + p] -= tot[1];
        plane[2 * npl + p] -= tot[2];
    }
    __syncthreads();
    if (t < 3) {
        double s = 0.0;
        const double* pl = plane + t * npl;
        for (int q = 0; q < n_inlet; q++) {
            double x = pl[inlet_list[q]];
            s += x * x;
        }
        double rms = sqrt(s / n_inlet);
        tot[t] = (rms > SMALL) ? C->ti_rms / rms : 0.0;
        Sc->sem[3 + t] = rms;
    }
    __syncthreads();
    for (int q = t; q < n_inlet; q += blockDim.x) {
        const int p = inlet_list[q];
        plane[p] *= tot[0];
        plane[npl + p] *= tot[1];
        plane[2 * npl + p] *= tot[2];
    }
}

}  // namespace les
