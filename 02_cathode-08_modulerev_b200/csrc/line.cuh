// line.cuh — device building blocks shared by the solvers: deterministic
// block / grid reductions, 16-byte vector access of 4 consecutive cells, and
// the exact z-line tridiagonal solve.
#pragma once

#include <cuda_runtime.h>

namespace cth {

// ---------------------------------------------------------------------------
// block reductions (fixed order -> deterministic)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// sum over the block; result valid in thread 0
static __device__ inline double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = (lane < nw) ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

// ---------------------------------------------------------------------------
// Deterministic grid-wide sum: every block stores its partial, the last block
// to arrive (atomic ticket) sums all partials in a fixed order.  Returns true
// in the last block (the sum is valid in its thread 0).
// ---------------------------------------------------------------------------
static __device__ inline bool last_block_sum(double v, double* part, unsigned int* counter, double* red,
                               double* total) {
    __shared__ bool am_last;
    const int nb = gridDim.x * gridDim.y;
    const double s = block_sum(v, red);
    if (threadIdx.x == 0) {
        part[blockIdx.y * gridDim.x + blockIdx.x] = s;
        __threadfence();
        const unsigned int ticket = atomicAdd(counter, 1u);
        am_last = (ticket == (unsigned int)(nb - 1));
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += __ldcg(part + k);
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) {
        *total = acc;
        *counter = 0u;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Exact solve of one tridiagonal z-line by one CTA (substructuring):
//   lo_i x_{i-1} + dg_i x_i + up_i x_{i+1} = d_i,   i = 0..n-1.
// Thread t owns the 4 cells [4t, 4t+4) in registers (one 16-byte vector load
// per array); the chunk's last cell is its separator u_t.  Each thread
// eliminates its chunk interior (Thomas) and writes it as
// x = y + v u_{t-1} + w u_t; the separators satisfy a tridiagonal system of
// blockDim.x unknowns, solved by parallel cyclic reduction in shared memory;
// the interiors follow.  O(n) work, log2(blockDim.x) barrier steps.
// ---------------------------------------------------------------------------
constexpr int CH = 4;  // cells per thread

// shared-memory bytes of the separator system with NR right-hand sides
template <typename T>
__host__ __device__ inline size_t line_smem(int nt, int nr) {
    return (size_t)(6 + 3 * nr) * nt * sizeof(T);
}

// correctly rounded reciprocal (one reciprocal per cell and reduction step)
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }

// 4 consecutive elements, 16-byte aligned
__device__ __forceinline__ void ld4(const float* p, float v[4]) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
    const double2 q0 = reinterpret_cast<const double2*>(p)[0];
    const double2 q1 = reinterpret_cast<const double2*>(p)[1];
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}
__device__ __forceinline__ void st4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double v[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// lo/dg/up/d: the thread's 4 cells.  Cells past the end of the line must be
// decoupled identity rows (lo = up = 0, dg = 1, d = 0) and the line's last
// cell must have up = 0, so every chunk is handled alike: cells 0..2 are the
// interior, cell 3 the separator.  x: the solution of the 4 cells.
// red: (6+3NR)*blockDim.x shared elements.
template <typename T, int NR>
__device__ __forceinline__ void line_solve(const T lo[CH], const T dg[CH], const T up[CH], const T d[NR][CH],
                                           T* red, T x[NR][CH]) {
    const int nt = blockDim.x, t = threadIdx.x;
    T* ra = red;
    T* rb = ra + nt;
    T* rc = rb + nt;
    T* rd = rc + nt;          // NR * nt
    T* fy = rd + NR * nt;     // NR * nt
    T* fv = fy + NR * nt;
    T* fw = fv + nt;
    T* uu = fw + nt;          // NR * nt
    T* ri = uu + NR * nt;     // 1 / rb

    // forward elimination of the interior cells 0..2
    const T i0 = rcp(dg[0]);
    const T c0 = up[0] * i0;
    const T v0p = -lo[0] * i0;
    const T i1 = rcp(dg[1] - lo[1] * c0);
    const T c1 = up[1] * i1;
    const T v1p = -lo[1] * v0p * i1;
    const T i2 = rcp(dg[2] - lo[2] * c1);
    const T v2p = -lo[2] * v1p * i2;
    const T w2p = -up[2] * i2;
    T y0p[NR], y1p[NR], y2p[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        y0p[r] = d[r][0] * i0;
        y1p[r] = (d[r][1] - lo[1] * y0p[r]) * i1;
        y2p[r] = (d[r][2] - lo[2] * y1p[r]) * i2;
    }
    // first-interior relation x_0 = yF + vF u_{t-1} + wF u_t
    const T v1 = v1p - c1 * v2p, w1 = -c1 * w2p;
    const T vF = v0p - c0 * v1, wF = -c0 * w1;
    T yF[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) yF[r] = y0p[r] - c0 * (y1p[r] - c1 * y2p[r]);
#pragma unroll
    for (int r = 0; r < NR; r++) fy[r * nt + t] = yF[r];
    fv[t] = vF;
    fw[t] = wF;
    __syncthreads();
    // separator row: lo3 x_2 + dg3 u_t + up3 x_{next,0} = d3, with
    // x_2 = y2p + v2p u_{t-1} + w2p u_t (last-interior relation)
    {
        const bool nxt = (t + 1 < nt);
        const T vN = nxt ? fv[t + 1] : T(0), wN = nxt ? fw[t + 1] : T(0);
        ra[t] = lo[3] * v2p;
        const T bsep = dg[3] + lo[3] * w2p + up[3] * vN;
        rb[t] = bsep;
        ri[t] = rcp(bsep);
        rc[t] = up[3] * wN;
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const T yN = nxt ? fy[r * nt + t + 1] : T(0);
            rd[r * nt + t] = d[r][3] - lo[3] * y2p[r] - up[3] * yN;
        }
    }
    __syncthreads();
    for (int s = 1; s < nt; s <<= 1) {
        T a_ = ra[t], b_ = rb[t], c_ = rc[t];
        T d_[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) d_[r] = rd[r * nt + t];
        T an = T(0), cn = T(0);
        if (t >= s) {
            const T k1 = -a_ * ri[t - s];
            an = k1 * ra[t - s];
            b_ += k1 * rc[t - s];
#pragma unroll
            for (int r = 0; r < NR; r++) d_[r] += k1 * rd[r * nt + t - s];
        }
        if (t + s < nt) {
            const T k2 = -c_ * ri[t + s];
            cn = k2 * rc[t + s];
            b_ += k2 * ra[t + s];
#pragma unroll
            for (int r = 0; r < NR; r++) d_[r] += k2 * rd[r * nt + t + s];
        }
        __syncthreads();
        ra[t] = an; rb[t] = b_; rc[t] = cn;
        ri[t] = rcp(b_);
#pragma unroll
        for (int r = 0; r < NR; r++) rd[r * nt + t] = d_[r];
        __syncthreads();
    }
    {
        const T ib = ri[t];
#pragma unroll
        for (int r = 0; r < NR; r++) uu[r * nt + t] = rd[r * nt + t] * ib;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const T uR = uu[r * nt + t];
        const T uL = (t > 0) ? uu[r * nt + t - 1] : T(0);
        const T x2 = y2p[r] + v2p * uL + w2p * uR;
        const T x1 = y1p[r] + v1p * uL - c1 * x2;
        const T x0 = y0p[r] + v0p * uL - c0 * x1;
        x[r][0] = x0; x[r][1] = x1; x[r][2] = x2; x[r][3] = uR;
    }
}

// ---------------------------------------------------------------------------
// complex double for the frequency-domain solves; interleaved (re, im) in memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ cd rcp(cd a) {
    const double s = rcp(a.x * a.x + a.y * a.y);
    return cd(a.x * s, -a.y * s);
}
__device__ __forceinline__ void ld4(const cd* p, cd v[4]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) { const double2 t = q[k]; v[k] = cd(t.x, t.y); }
}
__device__ __forceinline__ void st4(cd* p, const cd v[4]) {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) q[k] = make_double2(v[k].x, v[k].y);
}

// Deterministic grid-wide sums of K values (same last-block scheme as
// last_block_sum); part holds K*nblocks doubles.
template <int K>
static __device__ inline bool last_block_sumk(const double (&v)[K], double* part, unsigned int* counter,
                                              double* red, double (&total)[K]) {
    __shared__ bool am_last;
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    double s[K];
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = block_sum(v[k], red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) part[k * nb + bid] = s[k];
        __threadfence();
        const unsigned int ticket = atomicAdd(counter, 1u);
        am_last = (ticket == (unsigned int)(nb - 1));
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; k++) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += __ldcg(part + k * nb + b);
        acc = block_sum(acc, red);
        if (threadIdx.x == 0) total[k] = acc;
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

}  // namespace cth
