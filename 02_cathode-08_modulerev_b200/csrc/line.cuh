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
#pragma unroll 4
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
// Factorised z-line solve.  The tridiagonal operator of a line is fixed for a
// whole multigrid solve, so its elimination is done once (line_factor) and a
// relaxation only applies it to a right-hand side (line_solve_fac): no
// reciprocals, five warp-shuffle reduction steps and two block barriers.
//
// Structure (exact, the same substructuring as line_solve, two levels deep):
//   * thread t: chunk of 4 cells, interior cells 0..2 eliminated, cell 3 is
//     the separator u_t; x_k = y_k + v_k u_{t-1} + w_k u_t;
//   * warp w: separators of lanes 0..30 solved inside the warp by parallel
//     cyclic reduction over shuffles, in terms of the warp separators
//     S_{w-1} = u_{32w-1} and S_w = u_{32w+31}: u = Y + V S_{w-1} + W S_w;
//   * the nw = blockDim/32 warp separators form a tridiagonal system solved
//     by warp 0 (cyclic reduction over shuffles).
// Per-thread factors (LF_* slots, stored as 7 groups of 4), per-warp factors
// of the warp-separator system (LG_* slots, 4 groups of 4).
// ---------------------------------------------------------------------------
enum LineFacSlot {
    LF_I0 = 0, LF_I1, LF_I2, LF_M1, LF_M2, LF_C0, LF_C1, LF_V0, LF_V1, LF_V2, LF_W2, LF_LO3, LF_UP3,
    LF_K1 = 13, LF_K2 = 18, LF_IB = 23, LF_V = 24, LF_W = 25, LF_RA = 26, LF_N = 28
};
enum LineFac2Slot { LG_UP3 = 0, LG_RC = 1, LG_K1 = 2, LG_K2 = 7, LG_IB = 12, LG_N = 16 };
constexpr int LF_Q = LF_N / 4, LG_Q = LG_N / 4;

__device__ __forceinline__ float shup(float v, int s) { return __shfl_up_sync(0xffffffffu, v, s); }
__device__ __forceinline__ double shup(double v, int s) { return __shfl_up_sync(0xffffffffu, v, s); }
__device__ __forceinline__ float shdn(float v, int s) { return __shfl_down_sync(0xffffffffu, v, s); }
__device__ __forceinline__ double shdn(double v, int s) { return __shfl_down_sync(0xffffffffu, v, s); }
__device__ __forceinline__ float shix(float v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ double shix(double v, int l) { return __shfl_sync(0xffffffffu, v, l); }

// factor storage of one line: nt threads x LF_N values, nw warps x LG_N values
template <typename T>
__host__ __device__ inline size_t line_fac_size(int nt) { return (size_t)nt * LF_N + (size_t)(nt / 32) * LG_N; }

// shared memory of line_factor (9 * 32 values) / line_solve_fac (8 * 32 values
// of exchange + the warp-separator factors, LG_N * 32)
template <typename T>
__host__ __device__ inline size_t line_fac_smem() { return (8 + LG_N) * 32 * sizeof(T); }

// Matrix part.  lo/dg/up as for line_solve.  fac: this line's factor block.
template <typename T>
__device__ __forceinline__ void line_factor(const T lo[CH], const T dg[CH], const T up[CH], T* sh, T* fac) {
    const int nt = blockDim.x, t = threadIdx.x, lane = t & 31, w = t >> 5, nw = nt >> 5;
    T* s_vF = sh;
    T* s_wF = sh + 32;
    T* s_V0 = sh + 64;
    T* s_W0 = sh + 96;
    T* s_A = sh + 128;
    T* s_B = sh + 160;
    T* s_C = sh + 192;
    T* s_up = sh + 224;
    T* s_rc = sh + 256;
    T f[LF_N];
#pragma unroll
    for (int k = 0; k < LF_N; k++) f[k] = T(0);
    const T i0 = rcp(dg[0]);
    const T c0 = up[0] * i0;
    const T v0p = -lo[0] * i0;
    const T i1 = rcp(dg[1] - lo[1] * c0);
    const T c1 = up[1] * i1;
    const T v1p = -lo[1] * v0p * i1;
    const T i2 = rcp(dg[2] - lo[2] * c1);
    const T v2p = -lo[2] * v1p * i2;
    const T w2p = -up[2] * i2;
    const T v1 = v1p - c1 * v2p, w1 = -c1 * w2p;
    const T vF = v0p - c0 * v1, wF = -c0 * w1;
    f[LF_I0] = i0; f[LF_I1] = i1; f[LF_I2] = i2;
    f[LF_M1] = -lo[1] * i1; f[LF_M2] = -lo[2] * i2;
    f[LF_C0] = c0; f[LF_C1] = c1;
    f[LF_V0] = v0p; f[LF_V1] = v1p; f[LF_V2] = v2p; f[LF_W2] = w2p;
    f[LF_LO3] = lo[3]; f[LF_UP3] = up[3];
    if (lane == 0) { s_vF[w] = vF; s_wF[w] = wF; }
    __syncthreads();
    T vN = shdn(vF, 1), wN = shdn(wF, 1);
    if (lane == 31) {
        vN = (w + 1 < nw) ? s_vF[w + 1] : T(0);
        wN = (w + 1 < nw) ? s_wF[w + 1] : T(0);
    }
    const T ra = lo[3] * v2p;
    const T rb = dg[3] + lo[3] * w2p + up[3] * vN;
    const T rc = up[3] * wN;
    // separators of lanes 0..30 inside the warp; lane 31 is an identity row
    T a = (lane == 0 || lane == 31) ? T(0) : ra;
    T b = (lane == 31) ? T(1) : rb;
    T c = (lane >= 30) ? T(0) : rc;
    T dv = (lane == 0) ? -ra : T(0);
    T dw = (lane == 30) ? -rc : T(0);
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int s = 1 << q;
        const T aL = shup(a, s), bL = shup(b, s), cL = shup(c, s), dvL = shup(dv, s), dwL = shup(dw, s);
        const T aR = shdn(a, s), bR = shdn(b, s), cR = shdn(c, s), dvR = shdn(dv, s), dwR = shdn(dw, s);
        const T k1 = (lane >= s && lane <= 30) ? -a * rcp(bL) : T(0);
        const T k2 = (lane + s <= 30) ? -c * rcp(bR) : T(0);
        const T na = k1 * aL, nc = k2 * cR;
        b = b + k1 * cL + k2 * aR;
        dv = dv + k1 * dvL + k2 * dvR;
        dw = dw + k1 * dwL + k2 * dwR;
        a = na;
        c = nc;
        f[LF_K1 + q] = k1;
        f[LF_K2 + q] = k2;
    }
    const T ib = rcp(b);
    const T V = dv * ib, W = dw * ib;
    f[LF_IB] = ib; f[LF_V] = V; f[LF_W] = W; f[LF_RA] = ra;
    const T V30 = shix(V, 30), W30 = shix(W, 30);
    if (lane == 0) { s_V0[w] = V; s_W0[w] = W; }
    __syncthreads();
    if (lane == 31) {
        const T V0n = (w + 1 < nw) ? s_V0[w + 1] : T(0);
        const T W0n = (w + 1 < nw) ? s_W0[w + 1] : T(0);
        s_A[w] = ra * V30;
        s_B[w] = rb + ra * W30 + rc * V0n;
        s_C[w] = rc * W0n;
        s_up[w] = up[3];
        s_rc[w] = rc;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < LF_Q; q++) st4(fac + ((size_t)q * nt + t) * 4, f + 4 * q);
    if (w == 0) {
        T g[LG_N];
#pragma unroll
        for (int k = 0; k < LG_N; k++) g[k] = T(0);
        const bool on = lane < nw;
        a = on ? s_A[lane] : T(0);
        b = on ? s_B[lane] : T(1);
        c = on ? s_C[lane] : T(0);
        g[LG_UP3] = on ? s_up[lane] : T(0);
        g[LG_RC] = on ? s_rc[lane] : T(0);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const int s = 1 << q;
            if (s >= nw) break;
            const T aL = shup(a, s), bL = shup(b, s), cL = shup(c, s);
            const T aR = shdn(a, s), bR = shdn(b, s), cR = shdn(c, s);
            const T k1 = (on && lane >= s) ? -a * rcp(bL) : T(0);
            const T k2 = (lane + s < nw) ? -c * rcp(bR) : T(0);
            const T na = k1 * aL, nc = k2 * cR;
            b = b + k1 * cL + k2 * aR;
            a = na;
            c = nc;
            g[LG_K1 + q] = k1;
            g[LG_K2 + q] = k2;
        }
        g[LG_IB] = rcp(b);
        T* f2 = fac + (size_t)nt * LF_N;
        if (on) {
#pragma unroll
            for (int q = 0; q < LG_Q; q++) st4(f2 + ((size_t)q * nw + lane) * 4, g + 4 * q);
        }
    }
}

// factor registers of one thread (loaded before the right-hand side exists);
// the warp-separator factors go to shared memory (sh + 256, slot-major), read
// by warp 0 after line_solve_fac's first barrier
template <typename T>
struct LineFacRegs {
    T f[LF_N];
};

template <typename T>
__device__ __forceinline__ void line_fac_load(const T* fac, LineFacRegs<T>& R, T* sh) {
    const int nt = blockDim.x, t = threadIdx.x, nw = nt >> 5;
#pragma unroll
    for (int q = 0; q < LF_Q; q++) ld4(fac + ((size_t)q * nt + t) * 4, R.f + 4 * q);
    if (t < nw) {
        const T* f2 = fac + (size_t)nt * LF_N;
        T* sg = sh + 256;
#pragma unroll
        for (int q = 0; q < LG_Q; q++) {
            T g[4];
            ld4(f2 + ((size_t)q * nw + t) * 4, g);
#pragma unroll
            for (int r = 0; r < 4; r++) sg[(4 * q + r) * 32 + t] = g[r];
        }
    }
}

// Right-hand-side part: x = A^{-1} d for NR right-hand sides (sh: line_fac_smem
// bytes; NR <= 2).
template <typename T, int NR>
__device__ __forceinline__ void line_solve_fac(const LineFacRegs<T>& R, const T d[NR][CH], T* sh, T x[NR][CH]) {
    const int nt = blockDim.x, t = threadIdx.x, lane = t & 31, w = t >> 5, nw = nt >> 5;
    T* s_yF = sh;             // NR * 32
    T* s_Y0 = sh + 64;        // NR * 32
    T* s_P = sh + 128;        // NR * 32
    T* s_S = sh + 192;        // NR * 32
    const T* sg = sh + 256;   // LG_N * 32
    const T* f = R.f;
    T y0[NR], y1[NR], y2[NR], Y[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        y0[r] = d[r][0] * f[LF_I0];
        y1[r] = d[r][1] * f[LF_I1] + f[LF_M1] * y0[r];
        y2[r] = d[r][2] * f[LF_I2] + f[LF_M2] * y1[r];
        const T yF = y0[r] - f[LF_C0] * (y1[r] - f[LF_C1] * y2[r]);
        const T yN = shdn(yF, 1);
        T dd = d[r][3] - f[LF_LO3] * y2[r] - f[LF_UP3] * yN;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const int s = 1 << q;
            const T dL = shup(dd, s), dR = shdn(dd, s);
            dd = dd + f[LF_K1 + q] * dL + f[LF_K2 + q] * dR;
        }
        Y[r] = dd * f[LF_IB];
        const T Y30 = shix(Y[r], 30);
        if (lane == 0) { s_yF[r * 32 + w] = yF; s_Y0[r * 32 + w] = Y[r]; }
        if (lane == 31) s_P[r * 32 + w] = d[r][3] - f[LF_LO3] * y2[r] - f[LF_RA] * Y30;
    }
    __syncthreads();
    if (w == 0) {
        const bool on = lane < nw;
#pragma unroll
        for (int r = 0; r < NR; r++) {
            T D = T(0);
            if (on) {
                D = s_P[r * 32 + lane];
                if (lane + 1 < nw)
                    D = D - sg[LG_UP3 * 32 + lane] * s_yF[r * 32 + lane + 1] - sg[LG_RC * 32 + lane] * s_Y0[r * 32 + lane + 1];
            }
#pragma unroll
            for (int q = 0; q < 5; q++) {
                const int s = 1 << q;
                if (s >= nw) break;
                const T dL = shup(D, s), dR = shdn(D, s);
                if (on) D = D + sg[(LG_K1 + q) * 32 + lane] * dL + sg[(LG_K2 + q) * 32 + lane] * dR;
            }
            if (on) s_S[r * 32 + lane] = D * sg[LG_IB * 32 + lane];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const T Sm = (w > 0) ? s_S[r * 32 + w - 1] : T(0);
        const T Sw = s_S[r * 32 + w];
        const T u = (lane == 31) ? Sw : Y[r] + f[LF_V] * Sm + f[LF_W] * Sw;
        T uL = shup(u, 1);
        if (lane == 0) uL = Sm;
        const T x2 = y2[r] + f[LF_V2] * uL + f[LF_W2] * u;
        const T x1 = y1[r] + f[LF_V1] * uL - f[LF_C1] * x2;
        const T x0 = y0[r] + f[LF_V0] * uL - f[LF_C0] * x1;
        x[r][0] = x0; x[r][1] = x1; x[r][2] = x2; x[r][3] = u;
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

// complex float (the FP32 preconditioner hierarchy): 4 values = two 16-byte accesses
__device__ __forceinline__ cf rcp(cf a) {
    const float s = rcp(a.x * a.x + a.y * a.y);
    return cf(a.x * s, -a.y * s);
}
__device__ __forceinline__ void ld4(const cf* p, cf v[4]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = q[0], b = q[1];
    v[0] = cf(a.x, a.y); v[1] = cf(a.z, a.w); v[2] = cf(b.x, b.y); v[3] = cf(b.z, b.w);
}
__device__ __forceinline__ void st4(cf* p, const cf v[4]) {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    q[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
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
    // the K partial sums of one position are loaded together (their L2 loads in
    // flight at once); each sum keeps its order over the positions
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
#pragma unroll 2
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        double u[K];
#pragma unroll
        for (int k = 0; k < K; k++) u[k] = __ldcg(part + k * nb + b);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += u[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double t = block_sum(acc[k], red);
        if (threadIdx.x == 0) total[k] = t;
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

}  // namespace cth
