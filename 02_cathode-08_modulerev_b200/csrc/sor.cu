// sor.cu — red-black point SOR replacing solver_SOR
// (include/solverFuncs.hpp:169-217), plus the device residual of the
// box-union system.
//
// solver_SOR sweeps lexicographically; a GPU sweep updates the two colours
// (i+j even, then odd) of the block cells.  Update formula, neighbour source
// (the in/out solution array, grid or not), the 1e-100 guard on aP, the
// relaxation factor, the per-sweep error max|(new-old)/(new+old+1e-6)|*2 and
// the loop exit (after the sweep that takes the count past maxITR, or when
// the error is no longer > error_cnv) are those of solverFuncs.hpp:185-210.
// Both orderings converge to the same fixed point.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "grid.h"

namespace cth {

struct SorState {
    int done;
    int count;
    double error;
};

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// NaN-propagating max (a NaN error must stop the loop as in the reference,
// where `error > error_cnv` is false for NaN)
__device__ __forceinline__ double nmax(double a, double b) {
    if (a != a) return a;
    if (b != b) return b;
    return a > b ? a : b;
}

__global__ void k_sor_color(const double* __restrict__ aP, const double* __restrict__ aE,
                            const double* __restrict__ aW, const double* __restrict__ aN,
                            const double* __restrict__ aS, const double* __restrict__ b,
                            const unsigned char* __restrict__ mask, double* __restrict__ x, int ni,
                            int nj, int ld, double alpha, int color, double* __restrict__ part,
                            const SorState* __restrict__ stt) {
    __shared__ double red[32];
    if (stt->done) return;  // uniform: the loop already ended
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    double err = 0.0;
    if (i <= ni && ((i + j) & 1) == color) {
        const size_t p = (size_t)j * ld + i;
        if (mask[p]) {
            const double xo = x[p];
            const double tmp = (aE[p] * x[p + 1] + aW[p] * x[p - 1] + aN[p] * x[p + ld] +
                                aS[p] * x[p - ld] + b[p]) / (aP[p] + 1e-100);
            const double xn = (1.0 - alpha) * xo + alpha * tmp;
            err = fabs((xn - xo) / (xn + xo + 1e-6)) * 2.0;
            x[p] = xn;
        }
    }
    // block max (NaN-propagating)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double v = err;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = (lane < nw) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s = nmax(s, __shfl_down_sync(0xffffffffu, s, o));
        if (lane == 0) part[(size_t)color * gridDim.x * gridDim.y + blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void k_sor_finish(const double* __restrict__ part, int n, SorState* stt, int maxITR,
                             double tol) {
    __shared__ double red[32];
    if (stt->done) return;
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) v = nmax(v, part[k]);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < ((int)blockDim.x + 31) / 32; k++) s = nmax(s, red[k]);
        stt->count += 1;
        stt->error = s;
        if (stt->count > maxITR || !(s > tol)) stt->done = 1;
    }
}

int sor_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, double alpha,
                  int maxITR, double error_cnv, double* solution, cudaStream_t s,
                  cth_status* st) {
    // solver_SOR reads i±1, j±1 of every grid cell: grid cells must be interior
    if (g->i0 < 1 || g->i1 > g->ni || g->j0 < 1 || g->j1 > g->nj) {
        set_error("SOR: grid cells on the ghost frame would read outside the array");
        return CTH_ERR_ARG;
    }
    Workspace& w = g->ws;
    dim3 blk(256), grd((g->ni + 255) / 256, g->nj);
    const int nb = grd.x * grd.y;
    if (2 * nb > w.npart) {
        set_error("partial buffer too small");
        return CTH_ERR_ALLOC;
    }
    SorState* stt = reinterpret_cast<SorState*>(w.stat + 8);
    CTH_CUDA(cudaMemsetAsync(stt, 0, sizeof(SorState), s));
    const int batch = 8;
    SorState h{};
    for (int launched = 0;;) {
        for (int k = 0; k < batch; k++) {
            k_sor_color<<<grd, blk, 0, s>>>(aP, aE, aW, aN, aS, b, g->mask_full, solution, g->ni,
                                            g->nj, g->ld, alpha, 0, w.part, stt);
            k_sor_color<<<grd, blk, 0, s>>>(aP, aE, aW, aN, aS, b, g->mask_full, solution, g->ni,
                                            g->nj, g->ld, alpha, 1, w.part, stt);
            k_sor_finish<<<1, 1024, 0, s>>>(w.part, 2 * nb, stt, maxITR, error_cnv);
            g->launches += 3;
        }
        launched += batch;
        CTH_CUDA(cudaGetLastError());
        CTH_CUDA(cudaMemcpyAsync(w.h_stat, stt, sizeof(SorState), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        std::memcpy(&h, w.h_stat, sizeof(SorState));
        if (h.done) break;
        if (launched > maxITR + batch + 1) break;  // cannot happen: done is set past maxITR
    }
    cth_status loc{};
    loc.iterations = h.count;
    loc.residual = h.error;
    loc.converged = !(h.error > error_cnv) && std::isfinite(h.error);
    loc.nonfinite = !std::isfinite(h.error);
    if (st) *st = loc;
    if (loc.nonfinite) return CTH_NONFINITE;
    return loc.converged ? CTH_OK : CTH_NOT_CONVERGED;
}

// ---------------------------------------------------------------------------
__global__ void k_residual(const double* __restrict__ aP, const double* __restrict__ aE,
                           const double* __restrict__ aW, const double* __restrict__ aN,
                           const double* __restrict__ aS, const double* __restrict__ b,
                           const unsigned char* __restrict__ mask, const double* __restrict__ x,
                           double* __restrict__ r, int ni, int nj, int ld,
                           double* __restrict__ part) {
    __shared__ double red[2][32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    double rr = 0.0, bb = 0.0;
    if (i <= ni + 1) {
        const size_t p = (size_t)j * ld + i;
        double res = 0.0;
        if (mask[p]) {
            res = b[p] - aP[p] * x[p];
            if (i + 1 <= ni + 1 && mask[p + 1]) res += aE[p] * x[p + 1];
            if (i >= 1 && mask[p - 1]) res += aW[p] * x[p - 1];
            if (j + 1 <= nj + 1 && mask[p + ld]) res += aN[p] * x[p + ld];
            if (j >= 1 && mask[p - ld]) res += aS[p] * x[p - ld];
            rr = res * res;
            bb = b[p] * b[p];
        }
        if (r) r[p] = res;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_down_sync(0xffffffffu, rr, o);
        bb += __shfl_down_sync(0xffffffffu, bb, o);
    }
    if (lane == 0) { red[0][wid] = rr; red[1][wid] = bb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < ((int)blockDim.x + 31) / 32; k++) { s0 += red[0][k]; s1 += red[1][k]; }
        const size_t nb = (size_t)gridDim.x * gridDim.y;
        part[blockIdx.y * gridDim.x + blockIdx.x] = s0;
        part[nb + blockIdx.y * gridDim.x + blockIdx.x] = s1;
    }
}

__global__ void k_sum2(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double red[2][32];
    double a = 0.0, c = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) { a += part[k]; c += part[n + k]; }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if (lane == 0) { red[0][wid] = a; red[1][wid] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < ((int)blockDim.x + 31) / 32; k++) { s0 += red[0][k]; s1 += red[1][k]; }
        out[0] = s0;
        out[1] = s1;
    }
}

int residual_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                 const double* aN, const double* aS, const double* b, const double* x,
                 double* r, double* rnorm, double* bnorm, cudaStream_t s) {
    Workspace& w = g->ws;
    dim3 blk(256), grd((g->ni + 2 + 255) / 256, g->nj + 2);
    const int nb = grd.x * grd.y;
    if (2 * nb > w.npart) {
        set_error("partial buffer too small");
        return CTH_ERR_ALLOC;
    }
    k_residual<<<grd, blk, 0, s>>>(aP, aE, aW, aN, aS, b, g->mask_full, x, r, g->ni, g->nj, g->ld,
                                   w.part);
    k_sum2<<<1, 1024, 0, s>>>(w.part, nb, w.stat + 16);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(w.h_stat, w.stat + 16, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (rnorm) *rnorm = std::sqrt(w.h_stat[0]);
    if (bnorm) *bnorm = std::sqrt(w.h_stat[1]);
    return CTH_OK;
}

}  // namespace cth
