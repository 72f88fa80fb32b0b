// smg.cu — semicoarsening multigrid for the reference's 5-point solves.
//
// Replaces HYPRE Struct SMG as called by solver_SMG
// (include/solverFuncs.hpp:26-163).  Algorithm (Schaffer's semicoarsening MG,
// the published method behind HYPRE SMG, restated for sm_100a):
//   * coarsen in r only: row J of level l+1 is row 2J of level l;
//   * smoother: zebra z-line Gauss-Seidel, each z-line (fixed r row) solved
//     exactly by parallel cyclic reduction in shared memory, one CTA per line;
//   * interpolation of the odd (F) rows: the F line's own tridiagonal operator
//     applied inversely to its lumped coupling toward the C row below / above;
//   * Galerkin coarse operators R A P with R = P^T (9-point on coarse levels);
//   * outer loop = defect correction: FP64 residual b - A x on the caller's
//     FP64 coefficients, V-cycle on the residual in the working precision
//     (FP32 for CTH_PREC_MIXED, FP64 for CTH_PREC_FP64), x += e.  The cycle
//     sees the operator times a power of two sA that brings one diagonal
//     coefficient to [1, 2) and each residual times a power of two that brings
//     sA times the previous residual's norm there: the reference's systems
//     carry coefficients near 1e-18 and right-hand sides down to 1e-38, which
//     FP32 holds only as subnormals (powers of two are exact, so the FP64
//     cycles give the same bits as unscaled).
// Stopping rule of HYPRE SMG: ||b - A x||_2 / ||b||_2 < tol, at most maxITR
// cycles, zero initial guess (solverFuncs.hpp:106-126).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <cstdio>
#include <type_traits>

#include "grid.h"
#include "line.cuh"

namespace cth {


template <typename T>
struct LevelArgs {
    const T* a;       // npt planes
    size_t plane;     // nrow*ld
    T* x;
    const T* b;
    int nrow, ncol, ld;
    const T* fac;     // factorised line operators (real precisions)
};

// the real precisions relax with factorised line operators; the complex
// hierarchy eliminates each line in every relaxation
template <typename T> constexpr bool kFac = !std::is_same<T, cd>::value && !std::is_same<T, cf>::value;

// ---------------------------------------------------------------------------
// level-0 preparation: masked copy of the caller's FP64 planes into the level
// layout in precision T (couplings to non-grid cells dropped, non-grid cells
// identity), b0 = b (grid cells); the last block records ||b||^2 and whether
// the cycle loop runs at all (sets the graph's loop condition when use_cond).
// L2 policy for streams that should leave the cache to other data first
__device__ __forceinline__ unsigned long long l2_evict_first() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ double ld_hint(const double* p, unsigned long long pol) {
    double v;
    asm("ld.global.L2::cache_hint.f64 %0, [%1], %2;\n" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_hint(double* p, double v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;\n" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

// ---------------------------------------------------------------------------
// FP64 residual r = b - A x0 of one grid cell (couplings to non-grid cells dropped)
__device__ __forceinline__ double guess_resid(const SolveArgs* __restrict__ args, const double* __restrict__ x0,
                                              const unsigned char* __restrict__ mask, size_t p, size_t q,
                                              int c, int r, int ncol, int nrow, int ldl, int ld_u,
                                              unsigned long long pol) {
    double v = ld_hint(args->b + q, pol) - ld_hint(args->aP + q, pol) * ld_hint(x0 + q, pol);
    if (c > 0 && mask[p - 1]) v += ld_hint(args->aW + q, pol) * ld_hint(x0 + q - 1, pol);
    if (c + 1 < ncol && mask[p + 1]) v += ld_hint(args->aE + q, pol) * ld_hint(x0 + q + 1, pol);
    if (r > 0 && mask[p - ldl]) v += ld_hint(args->aS + q, pol) * ld_hint(x0 + q - ld_u, pol);
    if (r + 1 < nrow && mask[p + ldl]) v += ld_hint(args->aN + q, pol) * ld_hint(x0 + q + ld_u, pol);
    return v;
}

// Initial-guess test: ||b - A x||^2 of the candidates and ||b||^2 over the grid
// cells; the last block records in ST_GUESS which candidate k_prep0 starts
// from (the smaller relative residual, if at most guess_tol) or zero.  No
// guess: one thread writes 0.
__global__ void k_guess(const SolveArgs* __restrict__ args, const unsigned char* __restrict__ mask, int ld_u,
                        int i0, int j0, int ncol, int nrow, int ldl, double* __restrict__ part,
                        unsigned int* counter, double* __restrict__ stat) {
    __shared__ double red[32];
    if (args->x0 == nullptr) {
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) stat[ST_GUESS] = 0.0;
        return;
    }
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    const double* xb = args->x0b;
    const unsigned long long pol = l2_evict_first();   // the FP64 streams leave L2 first
    double v[3] = {0.0, 0.0, 0.0};  // ||r(x0)||^2, ||r(x0b)||^2, ||b||^2
    if (c < ncol) {
        const size_t p = (size_t)r * ldl + c;
        const size_t q = (size_t)(r + j0) * ld_u + (c + i0);
        if (mask[p]) {
            const double ra = guess_resid(args, args->x0, mask, p, q, c, r, ncol, nrow, ldl, ld_u, pol);
            v[0] = ra * ra;
            if (xb) {
                const double rb = guess_resid(args, xb, mask, p, q, c, r, ncol, nrow, ldl, ld_u, pol);
                v[1] = rb * rb;
            }
            const double bv = ld_hint(args->b + q, pol);
            v[2] = bv * bv;
        }
    }
    double tot[3];
    if (last_block_sumk<3>(v, part, counter, red, tot) && threadIdx.x == 0) {
        const double bb = tot[2];
        const double ra = (bb > 0.0) ? sqrt(tot[0] / bb) : 0.0;
        const double rb = (xb && bb > 0.0) ? sqrt(tot[1] / bb) : INFINITY;
        const bool second = isfinite(rb) && !(ra <= rb);
        const double r0 = second ? rb : ra;
        const bool use = isfinite(r0) && bb > 0.0 && r0 <= args->guess_tol;
        stat[ST_GUESS] = use ? (second ? 100.0 : 1.0) + r0 : -(1.0 + (isfinite(r0) ? fmin(r0, 1e30) : 1e30));
    }
}

// programmatic dependent launch: wait for the preceding kernel of the stream / graph
// (a no-op when the kernel was launched without the attribute), and let the next
// kernel start its own prologue
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// power of two 2^-e with |v| 2^-e in [1, 2); 1 for zero or non-finite v
__device__ __forceinline__ double pow2_scale(double v) {
    return (isfinite(v) && v != 0.0) ? ldexp(1.0, -ilogb(v)) : 1.0;
}

// cells per thread of k_prep0
constexpr int PREP_CELLS = 4;

// largest of the non-negative values v over the block, then over the grid into
// *gmax (a double's bits as a 64-bit integer: for v >= 0 the integer order is the
// numeric order, so the result does not depend on the order of the blocks)
__device__ __forceinline__ void grid_max_nonneg(double v, double* red, unsigned long long* gmax) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) m = fmax(m, red[k]);
        atomicMax(gmax, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

// Preparation of a solve: the initial residual (from the chosen guess or zero),
// the scaled first right-hand side b0, the statistics and the loop condition.
// REUSE = false: also writes the scaled working-precision operator a0 of the
// hierarchy, which the set-up that follows factorises.  REUSE = true (hierarchy
// slots): a0 holds the operator the slot's hierarchy was built from; the kernel
// measures the largest row-relative change max_m |a_m - a0_m| / |a_P| of the new
// scaled operator against it and decides on the device whether the set-up runs
// (stat[ST_SETUP], the conditional node cond_setup): when the slot is new, when
// the slot's last solve did not converge, or when the change exceeds
// args->reuse_tol.  The cycle then uses the
// hierarchy of the kept operator as the preconditioner of the FP64 defect
// correction, whose residuals and stopping rule use the caller's operator.
template <typename T, bool REUSE>
__global__ void k_prep0(const SolveArgs* __restrict__ args, const unsigned char* __restrict__ mask,
                        int ld_u, int i0, int j0, int ncol, int nrow, int ldl, size_t qref, T* __restrict__ a0,
                        T* __restrict__ b0, double* __restrict__ x64, double* __restrict__ part,
                        unsigned int* counter, double* __restrict__ stat, cudaGraphConditionalHandle cond,
                        int use_cond, double* __restrict__ sst, unsigned long long* gmax,
                        cudaGraphConditionalHandle cond_setup) {
    __shared__ double red[32];
    // a warp covers 32 * PREP_CELLS consecutive cells of row r, lane l the cells
    // base + 32 k + l (each load instruction of the warp reads one contiguous run)
    const int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 * PREP_CELLS) + (threadIdx.x & 31);
    const int r = blockIdx.y;
    const double sA = pow2_scale(args->aP[qref]);
    const double gw = stat[ST_GUESS];
    const bool guess = gw >= 1.0;
    const double* xg = (gw >= 100.0) ? args->x0b : args->x0;
    double v2[2] = {0.0, 0.0};  // ||r0||^2, ||b||^2
    double dmax = 0.0;          // REUSE: largest row-relative change of this thread's cells
    const unsigned long long pol = l2_evict_first();   // the FP64 streams leave L2 first
#pragma unroll
    for (int k = 0; k < PREP_CELLS; k++) {
        const int c = base + 32 * k;
        if (c >= ncol) break;
        const double* __restrict__ aP = args->aP;
        const size_t plane = (size_t)nrow * ldl;
        const size_t p = (size_t)r * ldl + c;
        const size_t q = (size_t)(r + j0) * ld_u + (c + i0);
        T vP = T(1), vW = T(0), vE = T(0), vS = T(0), vN = T(0), vb = T(0);
        if (mask[p]) {
            vP = (T)(ld_hint(aP + q, pol) * sA);
            if (c > 0 && mask[p - 1]) vW = (T)(ld_hint(args->aW + q, pol) * sA);
            if (c + 1 < ncol && mask[p + 1]) vE = (T)(ld_hint(args->aE + q, pol) * sA);
            if (r > 0 && mask[p - ldl]) vS = (T)(ld_hint(args->aS + q, pol) * sA);
            if (r + 1 < nrow && mask[p + ldl]) vN = (T)(ld_hint(args->aN + q, pol) * sA);
            const double bv = ld_hint(args->b + q, pol);
            v2[1] += bv * bv;
            if (guess) {
                const double rv = guess_resid(args, xg, mask, p, q, c, r, ncol, nrow, ldl, ld_u, pol);
                vb = (T)(rv * sA);
                v2[0] += rv * rv;
                st_hint(x64 + p, ld_hint(xg + q, pol), pol);
            } else {
                vb = (T)(bv * sA);
                v2[0] += bv * bv;
            }
        }
        if constexpr (REUSE) {
            if (mask[p]) {
                const double oP = a0[P * plane + p], oW = a0[W * plane + p], oE = a0[E * plane + p];
                const double oS = a0[S * plane + p], oN = a0[N * plane + p];
                double d = fabs((double)vP - oP);
                d = fmax(d, fabs((double)vW - oW));
                d = fmax(d, fabs((double)vE - oE));
                d = fmax(d, fabs((double)vS - oS));
                d = fmax(d, fabs((double)vN - oN));
                const double rel = d / fabs((double)vP);
                dmax = fmax(dmax, (rel >= 0.0) ? rel : INFINITY);   // NaN counts as a change
            }
        } else {
            a0[P * plane + p] = vP;
            a0[W * plane + p] = vW;
            a0[E * plane + p] = vE;
            a0[S * plane + p] = vS;
            a0[N * plane + p] = vN;
        }
        b0[p] = vb;
    }
    if constexpr (REUSE) grid_max_nonneg(dmax, red, gmax);
    double t2[2];
    if (last_block_sumk<2>(v2, part, counter, red, t2) && threadIdx.x == 0) {
        const double rr = t2[0], bb = t2[1];
        const bool fin = isfinite(rr) && isfinite(bb);
        // from zero: run at least one cycle (reference SMG); from a guess: stop
        // at once when it already meets the tolerance
        const bool met = guess && rr <= args->tol * args->tol * bb;
        const bool keep = fin && rr > 0.0 && args->maxit > 0 && !met;
        stat[ST_RR] = rr;
        stat[ST_BB] = bb;
        stat[ST_RELRES] = (bb > 0.0) ? sqrt(rr / bb) : 0.0;
        stat[ST_NONFINITE] = fin ? 0.0 : 1.0;
        stat[ST_ITER] = 0.0;
        stat[ST_CONV] = (fin && (rr == 0.0 || met)) ? 1.0 : 0.0;
        stat[ST_KEEP] = keep ? 1.0 : 0.0;
        stat[ST_ASCALE] = sA;
        stat[ST_XSCALE] = 1.0;
        stat[ST_SETUP] = 1.0;
        stat[ST_RETRY] = 0.0;
        if (use_cond) cudaGraphSetConditional(cond, keep ? 1u : 0u);
        if constexpr (REUSE) {
            const double change = __longlong_as_double((long long)atomicExch(gmax, 0ull));
            // the change compares the scaled operators, so a new power-of-two scale alone
            // (both operators scaled to the same reference coefficient) keeps the hierarchy
            const bool setup = sst[SW_VALID] == 0.0 || sst[SW_LASTCONV] == 0.0 || !(change <= args->reuse_tol);
            stat[ST_SETUP] = setup ? 1.0 : 0.0;
            if (setup) {
                sst[SW_VALID] = 1.0;
                sst[SW_ASCALE] = sA;
                sst[SW_SETUPS] += 1.0;
            } else {
                sst[SW_REUSES] += 1.0;
            }
            sst[SW_CHANGE] = change;
            if (use_cond) cudaGraphSetConditional(cond_setup, setup ? 1u : 0u);
        }
    }
}

// the scaled working-precision operator a0 of a slot's hierarchy, written when its
// set-up runs (the same values k_prep0<T, false> writes)
template <typename T>
__global__ void k_prep_op(const SolveArgs* __restrict__ args, const unsigned char* __restrict__ mask, int ld_u,
                          int i0, int j0, int ncol, int nrow, int ldl, T* __restrict__ a0,
                          const double* __restrict__ stat) {
    const int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 * PREP_CELLS) + (threadIdx.x & 31);
    const int r = blockIdx.y;
    const double sA = stat[ST_ASCALE];
#pragma unroll
    for (int k = 0; k < PREP_CELLS; k++) {
        const int c = base + 32 * k;
        if (c >= ncol) break;
        const size_t plane = (size_t)nrow * ldl;
        const size_t p = (size_t)r * ldl + c;
        const size_t q = (size_t)(r + j0) * ld_u + (c + i0);
        T vP = T(1), vW = T(0), vE = T(0), vS = T(0), vN = T(0);
        if (mask[p]) {
            vP = (T)(args->aP[q] * sA);
            if (c > 0 && mask[p - 1]) vW = (T)(args->aW[q] * sA);
            if (c + 1 < ncol && mask[p + 1]) vE = (T)(args->aE[q] * sA);
            if (r > 0 && mask[p - ldl]) vS = (T)(args->aS[q] * sA);
            if (r + 1 < nrow && mask[p + ldl]) vN = (T)(args->aN[q] * sA);
        }
        a0[P * plane + p] = vP;
        a0[W * plane + p] = vW;
        a0[E * plane + p] = vE;
        a0[S * plane + p] = vS;
        a0[N * plane + p] = vN;
    }
}

// ---------------------------------------------------------------------------
// interpolation weights of the F rows (odd rows) of one level: two line solves
// per F row, right-hand sides = lumped couplings toward the C rows.
// ---------------------------------------------------------------------------
// The line kernels run one CTA of bd threads per z-line (4 cells per thread).
// BND is their __launch_bounds__: 256 for lines of up to 1024 cells (registers
// unconstrained), 512 and 1024 for the longer lines, where the register budget
// of a CTA of bd threads caps the registers per thread (the FP64 and complex
// relaxations then spill; without the cap they could not launch at all).
template <typename T, int NPT, int BND = 256>
__global__ void __launch_bounds__(BND) k_weights(LevelArgs<T> L, const unsigned char* __restrict__ mask, T* __restrict__ wS,
                          T* __restrict__ wN) {
    const int j = 2 * blockIdx.x + 1;
    if (j >= L.nrow) return;
    extern __shared__ unsigned char smem_raw[];
    T* red = reinterpret_cast<T*>(smem_raw);
    const int n = L.ncol, s0 = CH * threadIdx.x;
    const int cnt = max(0, min(CH, n - s0));
    const size_t pl = L.plane;
    const size_t p = (size_t)j * L.ld + s0;
    T lo[CH], dg[CH], up[CH], d[2][CH];
#pragma unroll
    for (int k = 0; k < CH; k++) { lo[k] = T(0); dg[k] = T(1); up[k] = T(0); d[0][k] = T(0); d[1][k] = T(0); }
    if (cnt > 0) {
        const T* a = L.a;
        T aw[CH], ae[CH], as_[CH], an[CH];
        ld4(a + P * pl + p, dg);
        ld4(a + W * pl + p, aw);
        ld4(a + E * pl + p, ae);
        ld4(a + S * pl + p, as_);
        ld4(a + N * pl + p, an);
        T sw[CH] = {0, 0, 0, 0}, se[CH] = {0, 0, 0, 0}, nw[CH] = {0, 0, 0, 0}, ne[CH] = {0, 0, 0, 0};
        if (NPT == 9) {
            ld4(a + SW * pl + p, sw);
            ld4(a + SE * pl + p, se);
            ld4(a + NW * pl + p, nw);
            ld4(a + NE * pl + p, ne);
        }
#pragma unroll
        for (int k = 0; k < CH; k++) {
            const int i = s0 + k;
            if (k < cnt) {
                lo[k] = (i > 0) ? -aw[k] : T(0);
                up[k] = (i + 1 < n) ? -ae[k] : T(0);
                const size_t pk = p + k;
                if (mask[pk]) {
                    if (mask[pk - L.ld]) d[0][k] = as_[k] + ((NPT == 9) ? sw[k] + se[k] : T(0));
                    if (j + 1 < L.nrow && mask[pk + L.ld]) d[1][k] = an[k] + ((NPT == 9) ? nw[k] + ne[k] : T(0));
                }
            } else {
                dg[k] = T(1);
            }
        }
    }
    T x[2][CH];
    line_solve<T, 2>(lo, dg, up, d, red, x);
    if (cnt > 0) {
        st4(wS + p, x[0]);
        st4(wN + p, x[1]);
    }
}

// ---------------------------------------------------------------------------
// line factorisation of every row of one level (real precisions), once per
// solve; for the odd (F) rows of a non-coarsest level also the interpolation
// weights (two right-hand sides through the fresh factors).
// ---------------------------------------------------------------------------
template <typename T, int NPT>
__device__ __forceinline__ void factor_row(const LevelArgs<T>& L, const unsigned char* __restrict__ mask,
                                           T* __restrict__ fac, T* __restrict__ wS, T* __restrict__ wN,
                                           int weights, int j, T* sh) {
    const int n = L.ncol, s0 = CH * threadIdx.x;
    const int cnt = max(0, min(CH, n - s0));
    const size_t pl = L.plane;
    const size_t p = (size_t)j * L.ld + s0;
    const bool wts = weights && (j & 1);
    T lo[CH], dg[CH], up[CH], d[2][CH];
#pragma unroll
    for (int k = 0; k < CH; k++) { lo[k] = T(0); dg[k] = T(1); up[k] = T(0); d[0][k] = T(0); d[1][k] = T(0); }
    if (cnt > 0) {
        const T* a = L.a;
        T aw[CH], ae[CH];
        ld4(a + P * pl + p, dg);
        ld4(a + W * pl + p, aw);
        ld4(a + E * pl + p, ae);
        T as_[CH] = {0, 0, 0, 0}, an[CH] = {0, 0, 0, 0};
        T sw[CH] = {0, 0, 0, 0}, se[CH] = {0, 0, 0, 0}, nw[CH] = {0, 0, 0, 0}, ne[CH] = {0, 0, 0, 0};
        if (wts) {
            ld4(a + S * pl + p, as_);
            ld4(a + N * pl + p, an);
            if (NPT == 9) {
                ld4(a + SW * pl + p, sw);
                ld4(a + SE * pl + p, se);
                ld4(a + NW * pl + p, nw);
                ld4(a + NE * pl + p, ne);
            }
        }
#pragma unroll
        for (int k = 0; k < CH; k++) {
            const int i = s0 + k;
            if (k < cnt) {
                lo[k] = (i > 0) ? -aw[k] : T(0);
                up[k] = (i + 1 < n) ? -ae[k] : T(0);
                const size_t pk = p + k;
                if (wts && mask[pk]) {
                    if (mask[pk - L.ld]) d[0][k] = as_[k] + ((NPT == 9) ? sw[k] + se[k] : T(0));
                    if (j + 1 < L.nrow && mask[pk + L.ld]) d[1][k] = an[k] + ((NPT == 9) ? nw[k] + ne[k] : T(0));
                }
            } else {
                dg[k] = T(1);
            }
        }
    }
    T* frow = fac + (size_t)j * line_fac_size<T>(blockDim.x);
    line_factor<T>(lo, dg, up, sh, frow);
    if (!wts) return;
    __syncthreads();
    LineFacRegs<T> R;
    line_fac_load<T>(frow, R, sh);
    T x[2][CH];
    line_solve_fac<T, 2>(R, d, sh, x);
    if (cnt > 0) {
        st4(wS + p, x[0]);
        st4(wN + p, x[1]);
    }
}

template <typename T, int NPT, int BND = 256>
__global__ void __launch_bounds__(BND) k_factor(LevelArgs<T> L, const unsigned char* __restrict__ mask, T* __restrict__ fac,
                         T* __restrict__ wS, T* __restrict__ wN, int weights) {
    __shared__ T sh[(8 + LG_N) * 32];
    // the level's operator comes from the preceding kernel (programmatic dependent launch)
    griddep_wait();
    griddep_launch();
    factor_row<T, NPT>(L, mask, fac, wS, wN, weights, blockIdx.x, sh);
}

// P(g, i -> J): weight of coarse row J in fine row g at column i
template <typename T>
__device__ __forceinline__ T pw(const unsigned char* __restrict__ mask, const T* __restrict__ wS,
                                const T* __restrict__ wN, int g, int i, int J, int ld) {
    const size_t p = (size_t)g * ld + i;
    if ((g & 1) == 0) return (g / 2 == J && mask[p]) ? T(1) : T(0);
    if ((g - 1) / 2 == J) return wS[p];
    if ((g + 1) / 2 == J) return wN[p];
    return T(0);
}

// ---------------------------------------------------------------------------
// Galerkin coarse operator R A P (R = P^T): one thread per coarse cell.
// Launched with programmatic dependent launch after the factorisation of the
// fine level, which writes the interpolation weights: the fine operator (made
// by the kernel before that one) and the masks are loaded before the wait, the
// weights after it.  The sums run in a fixed order (fine rows 2J-1, 2J, 2J+1,
// stencil points, coarse rows), the same for every launch configuration.
// ---------------------------------------------------------------------------
template <typename T, int NPT>
__global__ void k_galerkin(LevelArgs<T> F, const unsigned char* __restrict__ maskf,
                           const T* __restrict__ wS, const T* __restrict__ wN, T* __restrict__ ac,
                           int nrowc, const unsigned char* __restrict__ maskc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.ncol) return;
    const int J = blockIdx.y;
    const int ld = F.ld, ncol = F.ncol;
    const size_t plc = (size_t)nrowc * ld;
    const size_t q = (size_t)J * ld + i;
    const int oi[9] = {0, -1, 1, 0, 0, -1, 1, -1, 1};
    const int oj[9] = {0, 0, 0, -1, 1, -1, -1, 1, 1};
    const bool active = maskc[q] != 0;
    // A[gf - 1][k]: stencil point k of fine row f = 2J - 2 + gf (zero where the
    // row or the neighbour lies outside the level)
    T A[3][NPT];
    // W[gg][ci][jj]: weight of fine point (2J - 2 + gg, i - 1 + ci) toward coarse
    // row J - 1 + jj (P couples rows only: semicoarsening)
    T W[5][3][3];
#pragma unroll
    for (int gg = 0; gg < 5; gg++)
#pragma unroll
        for (int ci = 0; ci < 3; ci++)
#pragma unroll
            for (int jj = 0; jj < 3; jj++) W[gg][ci][jj] = T(0);
#pragma unroll
    for (int gf = 1; gf <= 3; gf++) {
        const int f = 2 * J - 2 + gf;
        const size_t pf = (size_t)f * ld + i;
#pragma unroll
        for (int k = 0; k < NPT; k++) {
            const int ii = i + oi[k], g = f + oj[k];
            const bool in = active && f >= 0 && f < F.nrow && ii >= 0 && ii < ncol && g >= 0 && g < F.nrow;
            A[gf - 1][k] = in ? F.a[k * F.plane + pf] : T(0);
        }
    }
#pragma unroll
    for (int gg = 0; gg < 5; gg += 2) {
        const int g = 2 * J - 2 + gg;
#pragma unroll
        for (int ci = 0; ci < 3; ci++) {
            const int ii = i - 1 + ci;
            if (active && g >= 0 && g < F.nrow && ii >= 0 && ii < ncol)
                W[gg][ci][gg / 2] = maskf[(size_t)g * ld + ii] ? T(1) : T(0);
        }
    }
    griddep_wait();
    griddep_launch();
#pragma unroll
    for (int gg = 1; gg < 5; gg += 2) {
        const int g = 2 * J - 2 + gg;
#pragma unroll
        for (int ci = 0; ci < 3; ci++) {
            const int ii = i - 1 + ci;
            if (active && g >= 0 && g < F.nrow && ii >= 0 && ii < ncol) {
                const size_t pp = (size_t)g * ld + ii;
                W[gg][ci][(gg - 1) / 2] = wS[pp];
                W[gg][ci][(gg + 1) / 2] = wN[pp];
            }
        }
    }
    T acc[3][3];
#pragma unroll
    for (int u = 0; u < 3; u++)
#pragma unroll
        for (int v = 0; v < 3; v++) acc[u][v] = T(0);
    if (active) {
#pragma unroll
        for (int gf = 1; gf <= 3; gf++) {
            const T rw = W[gf][1][1];
            if (rw == T(0)) continue;
#pragma unroll
            for (int k = 0; k < NPT; k++) {
                const T av = A[gf - 1][k];
                if (av == T(0)) continue;
                const T mv = (k == P) ? av : -av;
#pragma unroll
                for (int dJ = -1; dJ <= 1; dJ++) {
                    const int Jp = J + dJ;
                    if (Jp < 0 || Jp >= nrowc) continue;
                    const T pv = W[gf + oj[k]][1 + oi[k]][dJ + 1];
                    if (pv != T(0)) acc[dJ + 1][oi[k] + 1] += rw * mv * pv;
                }
            }
        }
    }
    if (!active || acc[1][1] == T(0)) {
        ac[P * plc + q] = T(1);
#pragma unroll
        for (int k = 1; k < 9; k++) ac[k * plc + q] = T(0);
        return;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const T v = acc[oj[k] + 1][oi[k] + 1];
        ac[k * plc + q] = (k == P) ? v : -v;
    }
}


// ---------------------------------------------------------------------------
// zebra z-line relaxation: one CTA per row of the given parity.
//   zero_guess: the level's x is zero except rows relaxed earlier in this
//               kernel sequence (first C-row relaxation of a cycle).
//   prolong:    add the coarse-grid correction to the F-row neighbours on the
//               fly (first C-row relaxation after the coarse solve).
// ---------------------------------------------------------------------------
template <typename T>
struct ProlongArgs {
    const T* ec;   // coarse x
    const T* wS;
    const T* wN;
    int nrowc;
};

// Loads of x and b.  CG = true reads through L2: in the fused coarse tail the
// data were written by other CTAs of the same cluster earlier in the kernel,
// and an SM's L1 may hold an older copy of the line.
template <bool CG> __device__ __forceinline__ float ldg(const float* p) {
    if constexpr (CG) return __ldcg(p); else return *p;
}
template <bool CG> __device__ __forceinline__ double ldg(const double* p) {
    if constexpr (CG) return __ldcg(p); else return *p;
}
template <bool CG> __device__ __forceinline__ cd ldg(const cd* p) {
    if constexpr (CG) {
        const double2 q = __ldcg(reinterpret_cast<const double2*>(p));
        return cd(q.x, q.y);
    } else {
        return *p;
    }
}
__device__ __forceinline__ void ld4cg(const float* p, float v[4]) {
    const float4 q = __ldcg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4cg(const double* p, double v[4]) {
    const double2 q0 = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 q1 = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}
template <bool CG> __device__ __forceinline__ cf ldg(const cf* p) {
    if constexpr (CG) {
        const float2 q = __ldcg(reinterpret_cast<const float2*>(p));
        return cf(q.x, q.y);
    } else {
        return *p;
    }
}
__device__ __forceinline__ void ld4cg(const cf* p, cf v[4]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldcg(q), b = __ldcg(q + 1);
    v[0] = cf(a.x, a.y); v[1] = cf(a.z, a.w); v[2] = cf(b.x, b.y); v[3] = cf(b.z, b.w);
}
__device__ __forceinline__ void ld4cg(const cd* p, cd v[4]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) { const double2 t = __ldcg(q + k); v[k] = cd(t.x, t.y); }
}
template <bool CG, typename T> __device__ __forceinline__ void ld4g(const T* p, T v[4]) {
    if constexpr (CG) ld4cg(p, v); else ld4(p, v);
}

template <typename T, int NPT, bool CG>
__device__ __forceinline__ T xnb(const LevelArgs<T>& L, const ProlongArgs<T>& pa, bool prolong,
                                 int ii, int jj) {
    const size_t p = (size_t)jj * L.ld + ii;
    T v = ldg<CG>(L.x + p);
    if (prolong) {
        // jj is an F row (odd)
        v += pa.wS[p] * ldg<CG>(pa.ec + (size_t)((jj - 1) >> 1) * L.ld + ii);
        const int Jn = (jj + 1) >> 1;
        if (Jn < pa.nrowc) v += pa.wN[p] * ldg<CG>(pa.ec + (size_t)Jn * L.ld + ii);
    }
    return v;
}

// 4 cells [s0, s0+4) of row jj of x (with the coarse correction when prolong)
template <typename T, bool CG>
__device__ __forceinline__ void xrow4(const LevelArgs<T>& L, const ProlongArgs<T>& pa, bool prolong,
                                      int s0, int jj, T v[CH]) {
    const size_t p = (size_t)jj * L.ld + s0;
    ld4g<CG>(L.x + p, v);
    if (prolong) {
        T ws[CH], wn[CH], e0[CH];
        ld4(pa.wS + p, ws);
        ld4g<CG>(pa.ec + (size_t)((jj - 1) >> 1) * L.ld + s0, e0);
#pragma unroll
        for (int k = 0; k < CH; k++) v[k] += ws[k] * e0[k];
        const int Jn = (jj + 1) >> 1;
        if (Jn < pa.nrowc) {
            T e1[CH];
            ld4(pa.wN + p, wn);
            ld4g<CG>(pa.ec + (size_t)Jn * L.ld + s0, e1);
#pragma unroll
            for (int k = 0; k < CH; k++) v[k] += wn[k] * e1[k];
        }
    }
}

// residual r = b - A x of the 4 cells [s0, s0+4) of row f of level F
// (NPTF-point stencil); used to restrict into the next coarser level on the fly
template <typename T, int NPTF, bool CG>
__device__ __forceinline__ void resid4(const LevelArgs<T>& F, int f, int s0, T r[CH]) {
    const int n = F.ncol;
    const size_t pl = F.plane;
    const size_t p = (size_t)f * F.ld + s0;
    const T* a = F.a;
    T ap[CH], aw[CH], ae[CH], xc[CH];
    ld4g<CG>(F.b + p, r);
    ld4(a + P * pl + p, ap);
    ld4(a + W * pl + p, aw);
    ld4(a + E * pl + p, ae);
    ld4g<CG>(F.x + p, xc);
    const T xl = (s0 > 0) ? ldg<CG>(F.x + p - 1) : T(0);
    const T xr = (s0 + CH < n) ? ldg<CG>(F.x + p + CH) : T(0);
#pragma unroll
    for (int k = 0; k < CH; k++) r[k] -= ap[k] * xc[k];
    r[0] += aw[0] * xl;
#pragma unroll
    for (int k = 1; k < CH; k++) r[k] += aw[k] * xc[k - 1];
#pragma unroll
    for (int k = 0; k < CH - 1; k++) r[k] += ae[k] * xc[k + 1];
    r[CH - 1] += ae[CH - 1] * xr;
#pragma unroll
    for (int side = 0; side < 2; side++) {
        const int g = side == 0 ? f - 1 : f + 1;
        if (g < 0 || g >= F.nrow) continue;
        const size_t q = (size_t)g * F.ld + s0;
        T as_[CH], xg[CH];
        ld4(a + (side == 0 ? S : N) * pl + p, as_);
        ld4g<CG>(F.x + q, xg);
#pragma unroll
        for (int k = 0; k < CH; k++) r[k] += as_[k] * xg[k];
        if (NPTF == 9) {
            T dl[CH], dr[CH];
            ld4(a + (side == 0 ? SW : NW) * pl + p, dl);
            ld4(a + (side == 0 ? SE : NE) * pl + p, dr);
            const T gl = (s0 > 0) ? ldg<CG>(F.x + q - 1) : T(0);
            const T gr = (s0 + CH < n) ? ldg<CG>(F.x + q + CH) : T(0);
            r[0] += dl[0] * gl;
#pragma unroll
            for (int k = 1; k < CH; k++) r[k] += dl[k] * xg[k - 1];
#pragma unroll
            for (int k = 0; k < CH - 1; k++) r[k] += dr[k] * xg[k + 1];
            r[CH - 1] += dr[CH - 1] * gr;
        }
    }
}

// zebra z-line relaxation, one CTA per row of the given parity.
//   zero_guess: x of this level is zero (first C-row relaxation of a cycle);
//   prolong:    add the coarse correction to the F-row neighbours on the fly;
//   NPTF > 0:   (with zero_guess, C rows) the right-hand side is the residual
//               of the finer level F restricted on the fly (its C rows 2j and
//               2j+2), stored into this level's b for rows j and j+1.

// The coefficients of a level are never written inside a cycle, so they are read
// before the wait; b, the restricted residual and x come from earlier kernels of
// the cycle and are read after it.
// relax_line: relaxation of row j by the whole CTA (red: the line solver's
// shared memory).  DEP: launched with programmatic dependent launch; CG: x and
// b may have been written by other CTAs of the running kernel.
template <typename T, int NPT, int NPTF, bool DEP, bool CG>
__device__ __forceinline__ void relax_line(const LevelArgs<T>& L, int j, int zero_guess, int prolong,
                                           const ProlongArgs<T>& pa, const LevelArgs<T>& F, T* red) {
    const int n = L.ncol, s0 = CH * threadIdx.x;
    const int cnt = max(0, min(CH, n - s0));
    const size_t pl = L.plane;
    const size_t p = (size_t)j * L.ld + s0;
    const bool pr = prolong != 0;
    const bool has_s = !zero_guess && j > 0, has_n = !zero_guess && j + 1 < L.nrow;
    T lo[CH], dg[CH], up[CH], d[1][CH];
    T aw[CH], ae[CH], as_[CH], an[CH], sw[CH], se[CH], nw[CH], ne[CH];
#pragma unroll
    for (int k = 0; k < CH; k++) {
        lo[k] = T(0); dg[k] = T(1); up[k] = T(0); d[0][k] = T(0);
        as_[k] = an[k] = sw[k] = se[k] = nw[k] = ne[k] = T(0);
    }
    const T* a = L.a;
    LineFacRegs<T> R;
    if constexpr (kFac<T>) line_fac_load<T>(L.fac + (size_t)j * line_fac_size<T>(blockDim.x), R, red);
    if (cnt > 0) {
        if constexpr (!kFac<T>) {
            ld4(a + P * pl + p, dg);
            ld4(a + W * pl + p, aw);
            ld4(a + E * pl + p, ae);
        }
        if (has_s) {
            ld4(a + S * pl + p, as_);
            if (NPT == 9) {
                ld4(a + SW * pl + p, sw);
                ld4(a + SE * pl + p, se);
            }
        }
        if (has_n) {
            ld4(a + N * pl + p, an);
            if (NPT == 9) {
                ld4(a + NW * pl + p, nw);
                ld4(a + NE * pl + p, ne);
            }
        }
    }
    if constexpr (DEP) {
        griddep_wait();
        griddep_launch();
    }
    if (cnt > 0) {
        if (NPTF > 0) {
            resid4<T, NPTF, CG>(F, 2 * j, s0, d[0]);
            st4(const_cast<T*>(L.b) + p, d[0]);
            if (j + 1 < L.nrow) {
                T r1[CH];
                resid4<T, NPTF, CG>(F, 2 * j + 2, s0, r1);
                st4(const_cast<T*>(L.b) + p + L.ld, r1);
            }
        } else {
            ld4g<CG>(L.b + p, d[0]);
        }
        if (has_s) {
            T xs[CH];
            xrow4<T, CG>(L, pa, pr, s0, j - 1, xs);
#pragma unroll
            for (int k = 0; k < CH; k++) d[0][k] += as_[k] * xs[k];
            if (NPT == 9) {
                const T xl = (s0 > 0) ? xnb<T, NPT, CG>(L, pa, pr, s0 - 1, j - 1) : T(0);
                const T xr = (s0 + CH < n) ? xnb<T, NPT, CG>(L, pa, pr, s0 + CH, j - 1) : T(0);
                d[0][0] += sw[0] * xl;
#pragma unroll
                for (int k = 1; k < CH; k++) d[0][k] += sw[k] * xs[k - 1];
#pragma unroll
                for (int k = 0; k < CH - 1; k++) d[0][k] += se[k] * xs[k + 1];
                d[0][CH - 1] += se[CH - 1] * xr;
            }
        }
        if (has_n) {
            T xn[CH];
            xrow4<T, CG>(L, pa, pr, s0, j + 1, xn);
#pragma unroll
            for (int k = 0; k < CH; k++) d[0][k] += an[k] * xn[k];
            if (NPT == 9) {
                const T xl = (s0 > 0) ? xnb<T, NPT, CG>(L, pa, pr, s0 - 1, j + 1) : T(0);
                const T xr = (s0 + CH < n) ? xnb<T, NPT, CG>(L, pa, pr, s0 + CH, j + 1) : T(0);
                d[0][0] += nw[0] * xl;
#pragma unroll
                for (int k = 1; k < CH; k++) d[0][k] += nw[k] * xn[k - 1];
#pragma unroll
                for (int k = 0; k < CH - 1; k++) d[0][k] += ne[k] * xn[k + 1];
                d[0][CH - 1] += ne[CH - 1] * xr;
            }
        }
#pragma unroll
        for (int k = 0; k < CH; k++) {
            const int i = s0 + k;
            if (k < cnt) {
                lo[k] = (i > 0) ? -aw[k] : T(0);
                up[k] = (i + 1 < n) ? -ae[k] : T(0);
            } else {
                dg[k] = T(1);
                d[0][k] = T(0);
            }
        }
    }
    T x[1][CH];
    if constexpr (kFac<T>) line_solve_fac<T, 1>(R, d, red, x);
    else line_solve<T, 1>(lo, dg, up, d, red, x);
    if (cnt > 0) st4(L.x + p, x[0]);
}

template <typename T, int NPT, int NPTF, int BND = 256>
__global__ void __launch_bounds__(BND) k_relax(LevelArgs<T> L, int parity, int zero_guess, int prolong, ProlongArgs<T> pa,
                        LevelArgs<T> F) {
    const int j = 2 * blockIdx.x + parity;
    if (j >= L.nrow) return;
    extern __shared__ unsigned char smem_raw[];
    relax_line<T, NPT, NPTF, true, false>(L, j, zero_guess, prolong, pa, F, reinterpret_cast<T*>(smem_raw));
}

// ---------------------------------------------------------------------------
// Fused coarse tail of the V-cycle.  The levels l0..nlev-1 (at most TAIL_ROWS
// rows each, hence at most TAIL_CTAS lines of one colour) run in one launch of
// a single thread-block cluster: CTA c relaxes row 2c + parity in every phase,
// a phase ends with a cluster barrier (release / acquire at cluster scope),
// and x and b are read through L2.  The phases are those of vcycle() from l0
// down, in the same order, so the tail replaces ~4 launches per coarse level.
// ---------------------------------------------------------------------------
constexpr int TAIL_CTAS = 8;
constexpr int TAIL_ROWS = 2 * TAIL_CTAS;
constexpr int TAIL_MAXLEV = 8;

template <typename T>
struct TailArgs {
    LevelArgs<T> lev[TAIL_MAXLEV + 1];  // lev[0]: level l0-1 (restriction source); lev[1+k]: level l0+k
    const T* wS[TAIL_MAXLEV];           // interpolation weights of level l0+k toward level l0+k+1
    const T* wN[TAIL_MAXLEV];
    int nl;     // number of tail levels
    int nu1, nu2;
    int fine5;  // the restriction source is level 0 (5-point operator)
};

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <typename T>
__device__ __forceinline__ void tail_phase(const TailArgs<T>& A, int k, int parity, int zero, int prolong,
                                           int restr, T* red) {
    const LevelArgs<T>& L = A.lev[1 + k];
    const int j = 2 * (int)blockIdx.x + parity;
    if (j < L.nrow) {
        ProlongArgs<T> pa{nullptr, nullptr, nullptr, 0};
        if (prolong) {
            pa.ec = A.lev[2 + k].x;
            pa.wS = A.wS[k];
            pa.wN = A.wN[k];
            pa.nrowc = A.lev[2 + k].nrow;
        }
        if (restr) {
            if (A.fine5 && k == 0) relax_line<T, 9, 5, false, true>(L, j, 1, 0, pa, A.lev[k], red);
            else relax_line<T, 9, 9, false, true>(L, j, 1, 0, pa, A.lev[k], red);
        } else {
            relax_line<T, 9, 0, false, true>(L, j, zero, prolong, pa, L, red);
        }
    }
    cluster_sync_all();
}

template <typename T>
__global__ void k_tail(TailArgs<T> A) {
    extern __shared__ unsigned char smem_raw[];
    T* red = reinterpret_cast<T*>(smem_raw);
    griddep_wait();
    griddep_launch();
    const int last = A.nl - 1;
    for (int k = 0; k < last; k++) {
        for (int it = 0; it < A.nu1; it++) {
            tail_phase<T>(A, k, 0, it == 0, 0, it == 0, red);
            tail_phase<T>(A, k, 1, 0, 0, 0, red);
        }
    }
    tail_phase<T>(A, last, 0, 1, 0, 1, red);
    if (A.lev[1 + last].nrow > 1) tail_phase<T>(A, last, 1, 0, 0, 0, red);
    for (int k = last - 1; k >= 0; k--) {
        for (int it = 0; it < A.nu2; it++) {
            tail_phase<T>(A, k, 0, 0, it == 0, 0, red);
            tail_phase<T>(A, k, 1, 0, 0, 0, red);
        }
    }
}

// cells per thread and threads per block of k_update
constexpr int UPD_CELLS = 4;
constexpr int UPD_THREADS = 256;
constexpr size_t kUpdSmem = 6 * UPD_CELLS * UPD_THREADS * sizeof(double);

// 8-byte asynchronous global -> shared copy (completion per thread: cp_async_wait_all)
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// the same with an L2 eviction-priority policy (createpolicy)
__device__ __forceinline__ void cp_async8_hint(void* smem, const void* gmem, unsigned long long pol) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// defect correction, iteration it = stat[ST_ITER] + 1: x_it = x_{it-1} + e with
// x_k in x64[k & 1]; r = b - A x_it with the caller's FP64 coefficients; next
// cycle's right-hand side b0 = r (precision T).  The last block finishes the
// FP64 norm, the iteration count, the stopping rule and the loop condition.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(UPD_THREADS, 4) k_update(const SolveArgs* __restrict__ args,
                                                          const unsigned char* __restrict__ mask,
                         int ld_u, int i0, int j0, int ncol, int nrow, int ldl,
                         double* __restrict__ x64a, double* __restrict__ x64b,
                         const T* __restrict__ e, T* __restrict__ b0, double* __restrict__ part,
                         unsigned int* counter, double* __restrict__ stat,
                         cudaGraphConditionalHandle cond, int use_cond, double* __restrict__ sst,
                         cudaGraphConditionalHandle cond_rs, cudaGraphConditionalHandle cond2) {
    __shared__ double red[32];
    // dynamic shared memory (kUpdSmem): the caller's aP, aE, aW, aN, aS and b of this
    // thread's cells, [6][UPD_CELLS][UPD_THREADS]
    extern __shared__ double upd_smem[];
    double(*sco)[UPD_CELLS][UPD_THREADS] = reinterpret_cast<double(*)[UPD_CELLS][UPD_THREADS]>(upd_smem);
    // a warp covers 32 * UPD_CELLS consecutive cells of row r; lane l owns the cells
    // base + 32 k + l, so every load and store instruction of the warp reads one
    // contiguous run, and the west / east neighbours come from the adjacent lanes
    const int lane = threadIdx.x & 31;
    const int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 * UPD_CELLS);
    const int r = blockIdx.y;
    const bool run = base < ncol;   // uniform over the warp
    const size_t prow = (size_t)r * ldl;
    const size_t qrow = (size_t)(r + j0) * ld_u + i0;
    // before the wait on the cycle's last relaxation (programmatic dependent launch):
    // the caller's operator and right-hand side, constant during the solve, start
    // their asynchronous copies into shared memory, and the static mask is read
    // the FP64 streams (the caller's operator and b, the FP64 iterate) are read and
    // written evict-first in L2, so that they do not push the cycle's hierarchy out
    const unsigned long long pol = l2_evict_first();
    unsigned char mk[UPD_CELLS];
    if (run) {
        const double* __restrict__ src[6] = {args->aP, args->aE, args->aW, args->aN, args->aS, args->b};
#pragma unroll
        for (int k = 0; k < UPD_CELLS; k++) {
            const int c = min(base + 32 * k + lane, ncol - 1);
#pragma unroll
            for (int m = 0; m < 6; m++) cp_async8_hint(&sco[m][k][threadIdx.x], src[m] + qrow + c, pol);
            mk[k] = mask[prow + c];
        }
    }
    cp_async_commit();
    griddep_wait();
    griddep_launch();
    const int it = (int)stat[ST_ITER] + 1;
    const double* __restrict__ xin = (it & 1) ? x64a : x64b;
    double* __restrict__ xout = (it & 1) ? x64b : x64a;
    // e solves the cycle's system for xs x (the previous right-hand side's scale);
    // this right-hand side is scaled so that sA times the previous residual norm is O(1)
    const double sA = stat[ST_ASCALE];
    const double ie = 1.0 / stat[ST_XSCALE];
    const double xs = pow2_scale(sqrt(stat[ST_RR]) * sA);
    const double sb = sA * xs;
    double rr = 0.0;
    if (run) {
        // addresses clamped into the level (the row's end, the missing neighbour rows);
        // the values that do not exist are left out below
        const int rn = (r + 1 < nrow) ? r + 1 : r, rs = (r > 0) ? r - 1 : r;
        double xr[UPD_CELLS], xn[UPD_CELLS], xsr[UPD_CELLS];
        T er[UPD_CELLS], en[UPD_CELLS], esr[UPD_CELLS];
#pragma unroll
        for (int k = 0; k < UPD_CELLS; k++) {
            const int c = min(base + 32 * k + lane, ncol - 1);
            xr[k] = ld_hint(xin + prow + c, pol);
            er[k] = e[prow + c];
            xn[k] = ld_hint(xin + (size_t)rn * ldl + c, pol);
            en[k] = e[(size_t)rn * ldl + c];
            xsr[k] = ld_hint(xin + (size_t)rs * ldl + c, pol);
            esr[k] = e[(size_t)rs * ldl + c];
        }
        // the cells just outside the warp's run: base - 1 (lane 0) and base + 32 UPD_CELLS (lane 31)
        const int cl = base - 1, cr = base + 32 * UPD_CELLS;
        double xl = 0.0, xrr = 0.0;
        if (lane == 0 && cl >= 0) xl = xin[prow + cl] + (double)e[prow + cl] * ie;
        if (lane == 31 && cr < ncol) xrr = xin[prow + cr] + (double)e[prow + cr] * ie;
        // x + e of the own cells (zero beyond the row's end)
        double xc[UPD_CELLS];
#pragma unroll
        for (int k = 0; k < UPD_CELLS; k++)
            xc[k] = (base + 32 * k + lane < ncol) ? xr[k] + (double)er[k] * ie : 0.0;
        cp_async_wait_all();   // this thread's own copies: no barrier needed
#pragma unroll
        for (int k = 0; k < UPD_CELLS; k++) {
            const int c = base + 32 * k + lane;
            // west / east neighbours from the adjacent lanes (the run's ends from the next k)
            const double up = __shfl_up_sync(0xffffffffu, xc[k], 1);
            const double dn = __shfl_down_sync(0xffffffffu, xc[k], 1);
            const double prevlast = __shfl_sync(0xffffffffu, xc[k > 0 ? k - 1 : 0], 31);
            const double nextfirst = __shfl_sync(0xffffffffu, xc[k + 1 < UPD_CELLS ? k + 1 : k], 0);
            const double xw = (lane > 0) ? up : (k > 0 ? prevlast : xl);
            const double xe = (lane < 31) ? dn : (k + 1 < UPD_CELLS ? nextfirst : xrr);
            if (c >= ncol) continue;
            const size_t p = prow + c;
            const double vP = sco[0][k][threadIdx.x], vE = sco[1][k][threadIdx.x], vW = sco[2][k][threadIdx.x];
            const double vN = sco[3][k][threadIdx.x], vS = sco[4][k][threadIdx.x], vb = sco[5][k][threadIdx.x];
            double res = 0.0;
            if (mk[k]) {
                res = vb - vP * xc[k];
                if (c + 1 < ncol) res += vE * xe;
                if (c > 0) res += vW * xw;
                if (r + 1 < nrow) res += vN * (xn[k] + (double)en[k] * ie);
                if (r > 0) res += vS * (xsr[k] + (double)esr[k] * ie);
            }
            st_hint(xout + p, xc[k], pol);
            b0[p] = (T)(res * sb);
            rr += res * res;
        }
    } else {
        cp_async_wait_all();
    }
    double tot;
    if (last_block_sum(rr, part, counter, red, &tot) && threadIdx.x == 0) {
        const double bb = stat[ST_BB];
        const double rel = (bb > 0.0) ? sqrt(tot) / sqrt(bb) : 0.0;
        const bool fin = isfinite(tot);
        const bool conv = fin && rel < args->tol;
        const bool keep = fin && !conv && it < args->maxit;
        // a hierarchy slot's first loop (sst): a cycle on the kept hierarchy that
        // reduced the residual by less than kRetryRate ends the loop; the solve
        // rebuilds the hierarchy from its operator and continues in a second loop
        const bool retry = sst && keep && stat[ST_SETUP] == 0.0 && !(tot <= kRetryRate * kRetryRate * stat[ST_RR]);
        stat[ST_RR] = tot;
        stat[ST_RELRES] = rel;
        stat[ST_NONFINITE] = fin ? 0.0 : 1.0;
        stat[ST_ITER] = (double)it;
        stat[ST_CONV] = conv ? 1.0 : 0.0;
        stat[ST_KEEP] = keep ? 1.0 : 0.0;
        stat[ST_XSCALE] = xs;
        if (retry) {
            stat[ST_SETUP] = 1.0;
            stat[ST_RETRY] = 1.0;
            sst[SW_SETUPS] += 1.0;
            sst[SW_RETRIES] += 1.0;
        }
        if (use_cond) {
            cudaGraphSetConditional(cond, (keep && !retry) ? 1u : 0u);
            if (retry) {
                cudaGraphSetConditional(cond_rs, 1u);
                cudaGraphSetConditional(cond2, 1u);
            }
        }
    }
}

// write the accumulated solution x64[it & 1] into the caller's solution array
__global__ void k_store(const SolveArgs* __restrict__ args, const double* __restrict__ x64a,
                        const double* __restrict__ x64b, const double* __restrict__ stat,
                        const unsigned char* __restrict__ mask, int ncol, int nrow, int ldl,
                        int ld_u, int i0, int j0, double* __restrict__ sst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (sst && c == 0 && r == 0) {   // the slot's record of its last solve
        sst[SW_LASTCONV] = stat[ST_CONV];
        sst[SW_LASTITER] = stat[ST_ITER];
    }
    if (c >= ncol) return;
    const int it = (int)stat[ST_ITER];
    const double* __restrict__ x = (it & 1) ? x64b : x64a;
    const size_t p = (size_t)r * ldl + c;
    if (mask[p]) args->solution[(size_t)(r + j0) * ld_u + (c + i0)] = x[p];
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
template <typename T>
static Hierarchy<T>& hier(cth_grid* g);
template <>
Hierarchy<float>& hier<float>(cth_grid* g) { return g->h32[g->cur]; }
template <>
Hierarchy<double>& hier<double>(cth_grid* g) { return g->h64[g->cur]; }
template <>
Hierarchy<cd>& hier<cd>(cth_grid* g) { return g->hc; }
template <>
Hierarchy<cf>& hier<cf>(cth_grid* g) { return g->hcf; }

template <typename T>
static int alloc_hierarchy(cth_grid* g) {
    Hierarchy<T>& h = hier<T>(g);
    if (h.allocated) return CTH_OK;
    CTH_CUDA(cudaSetDevice(g->device));
    h.a.assign(g->nlev, nullptr);
    h.x.assign(g->nlev, nullptr);
    h.b.assign(g->nlev, nullptr);
    h.wS.assign(g->nlev, nullptr);
    h.wN.assign(g->nlev, nullptr);
    h.fac.assign(g->nlev, nullptr);
    for (int l = 0; l < g->nlev; l++) {
        const size_t n = (size_t)g->nrow[l] * g->ldl;
        const int npt = (l == 0) ? 5 : 9;
        CTH_CUDA(cudaMalloc(&h.a[l], n * npt * sizeof(T)));
        CTH_CUDA(cudaMalloc(&h.x[l], n * sizeof(T)));
        CTH_CUDA(cudaMalloc(&h.b[l], n * sizeof(T)));
        CTH_CUDA(cudaMalloc(&h.wS[l], n * sizeof(T)));
        CTH_CUDA(cudaMalloc(&h.wN[l], n * sizeof(T)));
        CTH_CUDA(cth::zero_fill(h.a[l], n * npt * sizeof(T)));
        CTH_CUDA(cth::zero_fill(h.x[l], n * sizeof(T)));
        CTH_CUDA(cth::zero_fill(h.b[l], n * sizeof(T)));
        CTH_CUDA(cth::zero_fill(h.wS[l], n * sizeof(T)));
        CTH_CUDA(cth::zero_fill(h.wN[l], n * sizeof(T)));
        if constexpr (kFac<T>) {
            const size_t nf = (size_t)g->nrow[l] * line_fac_size<T>(g->bd);
            CTH_CUDA(cudaMalloc(&h.fac[l], nf * sizeof(T)));
            CTH_CUDA(cth::zero_fill(h.fac[l], nf * sizeof(T)));
        }
    }
    h.allocated = true;
    return CTH_OK;
}

int ensure_hierarchy_f32(cth_grid* g) { return alloc_hierarchy<float>(g); }
int ensure_hierarchy_f64(cth_grid* g) { return alloc_hierarchy<double>(g); }

template <typename T>
static LevelArgs<T> level_args(cth_grid* g, int l) {
    Hierarchy<T>& h = hier<T>(g);
    LevelArgs<T> L;
    L.a = h.a[l];
    L.plane = (size_t)g->nrow[l] * g->ldl;
    L.x = h.x[l];
    L.b = h.b[l];
    L.nrow = g->nrow[l];
    L.ncol = g->ncol;
    L.ld = g->ldl;
    L.fac = h.fac.empty() ? nullptr : h.fac[l];
    return L;
}

// dynamic shared memory of a relaxation CTA
template <typename T>
static size_t relax_smem(int bd) {
    if constexpr (kFac<T>) return line_fac_smem<T>();
    else return line_smem<T>(bd, 1);
}

template <typename T, int NPT, int NPTF>
static void launch_relax(cth_grid* g, int l, int parity, int zero_guess, int prolong,
                         cudaStream_t s) {
    const int nr = g->nrow[l];
    const int rows = parity == 0 ? (nr + 1) / 2 : nr / 2;
    if (rows <= 0) return;
    Hierarchy<T>& h = hier<T>(g);
    ProlongArgs<T> pa{nullptr, nullptr, nullptr, 0};
    if (prolong) {
        pa.ec = h.x[l + 1];
        pa.wS = h.wS[l];
        pa.wN = h.wN[l];
        pa.nrowc = g->nrow[l + 1];
    }
    const size_t smem = relax_smem<T>(g->bd);
    LevelArgs<T> L = level_args<T>(g, l);
    // algorithmic bytes: 5 coefficients + b + x written + neighbour-row x, per cell
    LevelArgs<T> F = L;
    if (NPTF > 0) F = level_args<T>(g, l - 1);
    int slot = -1;
    if (l == 0) slot = prof_mark(g, PROF_RELAX0, (double)rows * g->ncol * 8.0 * sizeof(T), s);
    else if (l == 1 && NPTF > 0)
        slot = prof_mark(g, PROF_RESTRICT0, (double)g->nrow[1] * g->ncol * (9.0 + 8.0) * sizeof(T), s);
    else  // coarse levels: NPT coefficients + b + x in + x out per cell of the colour
        slot = prof_mark(g, PROF_RELAXC, (double)rows * g->ncol * (NPT + 3.0) * sizeof(T), s);
    auto kern = g->bnd == 1024 ? k_relax<T, NPT, NPTF, 1024>
              : g->bnd == 512  ? k_relax<T, NPT, NPTF, 512>
                               : k_relax<T, NPT, NPTF, 256>;
    if (g->pdl) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(rows);
        cfg.blockDim = dim3(g->bd);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, L, parity, zero_guess, prolong, pa, F);
    } else {
        kern<<<rows, g->bd, smem, s>>>(L, parity, zero_guess, prolong, pa, F);
    }
    g->launches++;
    if (slot >= 0) prof_done(g, slot, s);
}

template <typename T>
static void relax(cth_grid* g, int l, int parity, int zero_guess, int prolong, cudaStream_t s,
                  bool restrict_from_finer = false) {
    if (l == 0) launch_relax<T, 5, 0>(g, l, parity, zero_guess, prolong, s);
    else if (!restrict_from_finer) launch_relax<T, 9, 0>(g, l, parity, zero_guess, prolong, s);
    else if (l == 1) launch_relax<T, 9, 5>(g, l, parity, 1, 0, s);
    else launch_relax<T, 9, 9>(g, l, parity, 1, 0, s);
}

// the levels l0..nlev-1 as one cluster launch (k_tail)
template <typename T>
static void launch_tail(cth_grid* g, int l0, cudaStream_t s) {
    Hierarchy<T>& h = hier<T>(g);
    TailArgs<T> A{};
    A.nl = g->nlev - l0;
    A.nu1 = g->nu1;
    A.nu2 = g->nu2;
    A.fine5 = l0 == 1;
    A.lev[0] = level_args<T>(g, l0 - 1);
    for (int k = 0; k < A.nl; k++) {
        A.lev[1 + k] = level_args<T>(g, l0 + k);
        if (l0 + k + 1 < g->nlev) {
            A.wS[k] = h.wS[l0 + k];
            A.wN[k] = h.wN[l0 + k];
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(TAIL_CTAS);
    cfg.blockDim = dim3(g->bd);
    cfg.dynamicSmemBytes = relax_smem<T>(g->bd);
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = TAIL_CTAS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g->pdl ? 2 : 1;
    cudaLaunchKernelEx(&cfg, k_tail<T>, A);
    g->launches++;
}

// the levels from l down are handled by the fused tail
template <typename T> constexpr int tail_bit() { return 1; }
template <> constexpr int tail_bit<double>() { return 2; }
template <> constexpr int tail_bit<cd>() { return 4; }
template <> constexpr int tail_bit<cf>() { return 8; }   // no fused tail for the FP32 complex hierarchy

template <typename T>
static bool tail_from(const cth_grid* g, int l) {
    return g->tail && (g->tail_types & tail_bit<T>()) && l > 0 && g->nrow[l] <= TAIL_ROWS &&
           g->nlev - l <= TAIL_MAXLEV;
}

// V(nu1, nu2) cycle on level l.  The first C-row relaxation of every coarse
// level computes its right-hand side by restricting the finer residual.
template <typename T>
static void vcycle(cth_grid* g, int l, cudaStream_t s) {
    if (tail_from<T>(g, l)) {
        launch_tail<T>(g, l, s);
        return;
    }
    const bool fused = l > 0;
    if (l == g->nlev - 1) {
        relax<T>(g, l, 0, 1, 0, s, fused);
        if (g->nrow[l] > 1) relax<T>(g, l, 1, 0, 0, s);
        return;
    }
    for (int k = 0; k < g->nu1; k++) {
        relax<T>(g, l, 0, k == 0, 0, s, fused && k == 0);
        relax<T>(g, l, 1, 0, 0, s);
    }
    vcycle<T>(g, l + 1, s);
    for (int k = 0; k < g->nu2; k++) {
        relax<T>(g, l, 0, 0, k == 0, s);
        relax<T>(g, l, 1, 0, 0, s);
    }
}

// launch of a kernel that calls griddep_wait() before it reads what the kernels
// before it wrote: with programmatic dependent launch when the grid uses it
template <typename... KArgs, typename... Args>
static void launch_dep(cth_grid* g, void (*kern)(KArgs...), dim3 grd, dim3 blk, size_t smem, cudaStream_t s,
                       Args... args) {
    if (g->pdl) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grd;
        cfg.blockDim = blk;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, args...);
    } else {
        kern<<<grd, blk, smem, s>>>(args...);
    }
    g->launches++;
}

// Galerkin operator of level l + 1 from level l
template <typename T>
static void galerkin(cth_grid* g, int l, const LevelArgs<T>& L, cudaStream_t s) {
    Hierarchy<T>& h = hier<T>(g);
    const dim3 blk(128), grd((g->ncol + 127) / 128, g->nrow[l + 1]);
    if (l == 0)
        launch_dep(g, k_galerkin<T, 5>, grd, blk, 0, s, L, (const unsigned char*)g->mask[l], (const T*)h.wS[l],
                   (const T*)h.wN[l], h.a[l + 1], g->nrow[l + 1], (const unsigned char*)g->mask[l + 1]);
    else
        launch_dep(g, k_galerkin<T, 9>, grd, blk, 0, s, L, (const unsigned char*)g->mask[l], (const T*)h.wS[l],
                   (const T*)h.wN[l], h.a[l + 1], g->nrow[l + 1], (const unsigned char*)g->mask[l + 1]);
}

template <typename T>
static void setup_levels(cth_grid* g, cudaStream_t s) {
    Hierarchy<T>& h = hier<T>(g);
    const int slot = prof_mark(g, PROF_SETUP, 0.0, s);
    if constexpr (kFac<T>) {
        // per level: factorise every line (and the F-row weights), then the
        // Galerkin operator of the next level
        for (int l = 0; l < g->nlev; l++) {
            LevelArgs<T> L = level_args<T>(g, l);
            const int wts = l + 1 < g->nlev;
            auto kf = l == 0 ? (g->bnd == 1024 ? k_factor<T, 5, 1024> : g->bnd == 512 ? k_factor<T, 5, 512>
                                                                                      : k_factor<T, 5, 256>)
                             : (g->bnd == 1024 ? k_factor<T, 9, 1024> : g->bnd == 512 ? k_factor<T, 9, 512>
                                                                                      : k_factor<T, 9, 256>);
            launch_dep(g, kf, dim3(g->nrow[l]), dim3(g->bd), 0, s, L, g->mask[l], h.fac[l], h.wS[l], h.wN[l], wts);
            if (!wts) break;
            galerkin<T>(g, l, L, s);
        }
    } else {
        for (int l = 0; l + 1 < g->nlev; l++) {
            LevelArgs<T> L = level_args<T>(g, l);
            const int frows = g->nrow[l] / 2;
            const size_t smem = line_smem<T>(g->bd, 2);
            if (frows > 0) {
                auto kw = l == 0 ? (g->bnd == 1024 ? k_weights<T, 5, 1024> : g->bnd == 512 ? k_weights<T, 5, 512>
                                                                                          : k_weights<T, 5, 256>)
                                 : (g->bnd == 1024 ? k_weights<T, 9, 1024> : g->bnd == 512 ? k_weights<T, 9, 512>
                                                                                          : k_weights<T, 9, 256>);
                kw<<<frows, g->bd, smem, s>>>(L, g->mask[l], h.wS[l], h.wN[l]);
                g->launches++;
            }
            galerkin<T>(g, l, L, s);
        }
    }
    prof_done(g, slot, s);
}

// kernel sequence of one solve, split into the part before the cycle loop,
// one loop iteration, and the part after it; each returns its kernel count
// sst: the slot words of a hierarchy slot (null: the set-up runs in this part)
template <typename T>
static int enqueue_pre(cth_grid* g, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond,
                       double* sst = nullptr, cudaGraphConditionalHandle cond_setup = 0) {
    Hierarchy<T>& h = hier<T>(g);
    Workspace& w = g->ws;
    const int ncol = g->ncol, nrow0 = g->nrow[0], ldl = g->ldl;
    dim3 blk(256), grd((ncol + 255) / 256, nrow0);
    dim3 grdp((ncol + 256 * PREP_CELLS - 1) / (256 * PREP_CELLS), nrow0);
    unsigned long long* gmax = reinterpret_cast<unsigned long long*>(w.slotstat + 2 * kSlots * kSlotWords);
    cudaMemsetAsync(w.x64[0], 0, sizeof(double) * (size_t)nrow0 * ldl, s);
    k_guess<<<grd, blk, 0, s>>>(w.d_args, g->mask[0], g->ld, g->i0, g->j0, ncol, nrow0, ldl, w.part, w.counter,
                                w.stat);
    if (sst) {
        k_prep0<T, true><<<grdp, blk, 0, s>>>(w.d_args, g->mask[0], g->ld, g->i0, g->j0, ncol, nrow0, ldl, g->qref,
                                              h.a[0], h.b[0], w.x64[0], w.part, w.counter, w.stat, cond, use_cond,
                                              sst, gmax, cond_setup);
        return 2;
    }
    k_prep0<T, false><<<grdp, blk, 0, s>>>(w.d_args, g->mask[0], g->ld, g->i0, g->j0, ncol, nrow0, ldl, g->qref,
                                           h.a[0], h.b[0], w.x64[0], w.part, w.counter, w.stat, cond, use_cond,
                                           nullptr, gmax, 0);
    const long long l0 = g->launches;
    setup_levels<T>(g, s);
    const int n = 2 + (int)(g->launches - l0);
    g->launches = l0;
    return n;
}

// the set-up of a slot's hierarchy (run when k_prep0<T, true> decided so)
template <typename T>
static int enqueue_setup(cth_grid* g, cudaStream_t s) {
    Hierarchy<T>& h = hier<T>(g);
    Workspace& w = g->ws;
    const int ncol = g->ncol, nrow0 = g->nrow[0], ldl = g->ldl;
    dim3 blk(256), grdp((ncol + 256 * PREP_CELLS - 1) / (256 * PREP_CELLS), nrow0);
    k_prep_op<T><<<grdp, blk, 0, s>>>(w.d_args, g->mask[0], g->ld, g->i0, g->j0, ncol, nrow0, ldl, h.a[0], w.stat);
    const long long l0 = g->launches;
    setup_levels<T>(g, s);
    const int n = 1 + (int)(g->launches - l0);
    g->launches = l0;
    return n;
}

// sst (a slot's first loop): the cycle may end the loop for a rebuild (k_update,
// handles cond_rs / cond2 of the rebuild and the second loop)
template <typename T>
static int enqueue_body(cth_grid* g, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond,
                        double* sst = nullptr, cudaGraphConditionalHandle cond_rs = 0,
                        cudaGraphConditionalHandle cond2 = 0) {
    Hierarchy<T>& h = hier<T>(g);
    Workspace& w = g->ws;
    const int ncol = g->ncol, nrow0 = g->nrow[0], ldl = g->ldl;
    dim3 blk(UPD_THREADS), grd((ncol + UPD_THREADS * UPD_CELLS - 1) / (UPD_THREADS * UPD_CELLS), nrow0);
    const long long l0 = g->launches;
    vcycle<T>(g, 0, s);
    const int slot = prof_mark(g, PROF_UPDATE, (double)nrow0 * ncol * (8.0 * 8.0 + 2.0 * sizeof(T) + 1.0), s);
    // programmatic dependent launch: the caller's operator is copied in before the wait
    launch_dep(g, k_update<T>, grd, blk, kUpdSmem, s, (const SolveArgs*)w.d_args, (const unsigned char*)g->mask[0], g->ld,
               g->i0, g->j0, ncol, nrow0, ldl, w.x64[0], w.x64[1], (const T*)h.x[0], h.b[0], w.part, w.counter,
               w.stat, cond, use_cond, sst, cond_rs, cond2);
    prof_done(g, slot, s);
    const int n = (int)(g->launches - l0);
    g->launches = l0;
    return n;
}

static int enqueue_post(cth_grid* g, cudaStream_t s, double* sst = nullptr) {
    Workspace& w = g->ws;
    dim3 blk(256), grd((g->ncol + 255) / 256, g->nrow[0]);
    k_store<<<grd, blk, 0, s>>>(w.d_args, w.x64[0], w.x64[1], w.stat, g->mask[0], g->ncol, g->nrow[0],
                                g->ldl, g->ld, g->i0, g->j0, sst);
    return 1;
}

// a conditional node (IF or WHILE on handle c) after the current capture
// dependencies of cs, its body captured from cs2 by fill(cs2); cs then continues
// after the node
template <typename F>
static cudaError_t capture_conditional(cudaStream_t cs, cudaStream_t cs2, cudaGraphConditionalHandle c,
                                       cudaGraphConditionalNodeType type, F fill) {
    cudaStreamCaptureStatus cst;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
    cudaGraphNode_t cnode = nullptr;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = c;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(cs2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            fill(cs2);
            cudaGraph_t bout = nullptr;
            e = cudaStreamEndCapture(cs2, &bout);
        }
    }
    return e;
}

// capture the whole solve as one graph: pre -> while(keep){ body } -> post; with
// a hierarchy slot (sst): pre -> if(setup){ set-up } -> while(keep){ body } -> post
template <typename T>
static int build_graph(cth_grid* g, SolveGraph& G, double* sst) {
    if (G.valid && G.nu1 == g->nu1 && G.nu2 == g->nu2) return CTH_OK;
    if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
    if (G.graph) { cudaGraphDestroy(G.graph); G.graph = nullptr; }
    G.valid = false;
    cudaStream_t cs = g->cap[0], cs2 = g->cap[1];
    CTH_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    cudaStreamCaptureStatus cst;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, nullptr, nullptr);
    cudaGraphConditionalHandle cond = 0, cond_setup = 0;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess && sst)
        e = cudaGraphConditionalHandleCreate(&cond_setup, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraph_t junk;
        cudaStreamEndCapture(cs, &junk);
        if (junk) cudaGraphDestroy(junk);
        return cuda_fail(e, "graph conditional handle");
    }
    cudaGraphConditionalHandle cond_rs = 0, cond2 = 0;
    if (e == cudaSuccess && sst) e = cudaGraphConditionalHandleCreate(&cond_rs, graph, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess && sst) e = cudaGraphConditionalHandleCreate(&cond2, graph, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) G.n_pre = enqueue_pre<T>(g, cs, cond, 1, sst, cond_setup);
    G.n_setup = 0;
    if (e == cudaSuccess && sst)
        e = capture_conditional(cs, cs2, cond_setup, cudaGraphCondTypeIf,
                                [&](cudaStream_t st) { G.n_setup = enqueue_setup<T>(g, st); });
    if (e == cudaSuccess)
        e = capture_conditional(cs, cs2, cond, cudaGraphCondTypeWhile, [&](cudaStream_t st) {
            G.n_body = enqueue_body<T>(g, st, cond, 1, sst, cond_rs, cond2);
        });
    // a slot's rebuild after a slow cycle on the kept hierarchy, and the second loop
    if (e == cudaSuccess && sst)
        e = capture_conditional(cs, cs2, cond_rs, cudaGraphCondTypeIf,
                                [&](cudaStream_t st) { enqueue_setup<T>(g, st); });
    if (e == cudaSuccess && sst)
        e = capture_conditional(cs, cs2, cond2, cudaGraphCondTypeWhile,
                                [&](cudaStream_t st) { enqueue_body<T>(g, st, cond2, 1); });
    if (e == cudaSuccess) G.n_post = enqueue_post(g, cs, sst);
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cs, &out);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&G.exec, out, 0);
    if (e != cudaSuccess) {
        if (out) cudaGraphDestroy(out);
        cudaGetLastError();
        return cuda_fail(e, "solve graph capture");
    }
    G.graph = out;
    G.nu1 = g->nu1;
    G.nu2 = g->nu2;
    G.valid = true;
    return CTH_OK;
}

// Enqueues a solve on stream s.  With graphs on, the call returns after the graph
// launch and the asynchronous status copy (*pending = 1): solve_finish reads the
// status after synchronising s, so several grids can solve concurrently on
// different streams.  Without graphs the solve completes here (*pending = 0).
// the solve's arguments reach the device as kernel parameters (copied at launch), so
// the host may enqueue the next solve on the same grid before this one has run
__global__ void k_set_args(SolveArgs a, SolveArgs* dst) { *dst = a; }

// words of the device status copied to the host after a solve
constexpr int kStatCopy = ST_RETRY + 1;

template <typename T>
static int solve_launch_h(cth_grid* g, const double* aP, const double* aE, const double* aW,
                          const double* aN, const double* aS, const double* b, int maxITR,
                          double tol, double* solution, cudaStream_t s, int prec, int* pending,
                          double* h_dst, const double* x0, double guess_tol, const double* x0b, int slot) {
    *pending = 0;
    const bool reuse = slot >= 0;
    int rc = alloc_hierarchy<T>(g);
    if (rc != CTH_OK) return rc;
    Workspace& w = g->ws;
    {
        dim3 grd((g->ncol + 255) / 256, g->nrow[0]);
        if (3 * (int)(grd.x * grd.y) > w.npart) {
            set_error("partial-sum buffer too small");
            return CTH_ERR_ALLOC;
        }
    }
    double* sst = reuse ? w.slotstat + ((size_t)prec * kSlots + slot) * kSlotWords : nullptr;
    SolveArgs* ha = w.h_args;
    ha->aP = aP; ha->aE = aE; ha->aW = aW; ha->aN = aN; ha->aS = aS; ha->b = b;
    ha->solution = solution;
    ha->tol = tol;
    ha->maxit = maxITR;
    ha->x0 = x0;
    ha->x0b = x0 ? x0b : nullptr;
    ha->guess_tol = guess_tol;
    ha->reuse_tol = g->reuse_tol;
    k_set_args<<<1, 1, 0, s>>>(*ha, w.d_args);
    const bool graph = g->use_graphs && !g->prof.on;
    if (graph) {
        SolveGraph& G = g->graphs[prec][g->cur];
        rc = build_graph<T>(g, G, sst);
        if (rc != CTH_OK) return rc;
        CTH_CUDA(cudaGraphLaunch(G.exec, s));
        CTH_CUDA(cudaMemcpyAsync(h_dst ? h_dst : w.h_stat, w.stat, kStatCopy * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
        g->pending_stream = s;
        *pending = 1 + prec + 2 * g->cur;
        return CTH_OK;
    }
    g->launches += enqueue_pre<T>(g, s, 0, 0, sst);
    CTH_CUDA(cudaMemcpyAsync(w.h_stat, w.stat, kStatCopy * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (sst && w.h_stat[ST_SETUP] != 0.0) g->launches += enqueue_setup<T>(g, s);
    bool retried = false;
    while (w.h_stat[ST_KEEP] != 0.0) {
        if (sst && !retried && w.h_stat[ST_RETRY] != 0.0) {
            g->launches += enqueue_setup<T>(g, s);
            retried = true;
        }
        g->launches += enqueue_body<T>(g, s, 0, 0, retried ? nullptr : sst);
        CTH_CUDA(cudaMemcpyAsync(w.h_stat, w.stat, kStatCopy * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
    }
    g->launches += enqueue_post(g, s, sst);
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaStreamSynchronize(s));
    prof_collect(g);
    if (h_dst) std::memcpy(h_dst, w.h_stat, kStatCopy * sizeof(double));
    return CTH_OK;
}

// the solve on hierarchy 0 (set up every solve) or on the hierarchy of a slot
template <typename T>
static int solve_launch(cth_grid* g, const double* aP, const double* aE, const double* aW,
                        const double* aN, const double* aS, const double* b, int maxITR,
                        double tol, double* solution, cudaStream_t s, int prec, int* pending,
                        double* h_dst, const double* x0, double guess_tol, const double* x0b, int slot) {
    const int sl = (g->reuse_tol > 0.0 && slot >= 0 && slot < kSlots) ? slot : -1;
    g->cur = sl >= 0 ? 1 + sl : 0;
    const int rc = solve_launch_h<T>(g, aP, aE, aW, aN, aS, b, maxITR, tol, solution, s, prec, pending, h_dst, x0,
                                     guess_tol, x0b, sl);
    g->cur = 0;
    return rc;
}

int solve_parse(cth_grid* g, int pending, const double* h, cth_status* st) {
    if (pending) {
        const SolveGraph& G = g->graphs[(pending - 1) & 1][(pending - 1) >> 1];
        // a slot's set-up runs once when ST_SETUP is set: before the cycles, or after
        // the first loop when a cycle on the kept hierarchy was slow (ST_RETRY)
        g->launches += G.n_pre + (h[ST_SETUP] != 0.0 ? G.n_setup : 0) + (long long)G.n_body * (long long)h[ST_ITER] +
                       G.n_post;
    }
    CTH_CUDA(cudaGetLastError());
    cth_status loc{};
    loc.initial_residual = std::sqrt(h[ST_BB]);
    loc.iterations = (int)h[ST_ITER];
    loc.residual = h[ST_RELRES];
    loc.nonfinite = h[ST_NONFINITE] != 0.0;
    loc.converged = h[ST_CONV] != 0.0;
    const double gw = h[ST_GUESS];
    loc.guess = gw >= 100.0 ? 2 : (gw >= 1.0 ? 1 : (gw <= -1.0 ? -1 : 0));
    loc.guess_residual = gw >= 100.0 ? gw - 100.0 : (gw >= 1.0 ? gw - 1.0 : (gw <= -1.0 ? -gw - 1.0 : -1.0));
    if (st) *st = loc;
    if (loc.nonfinite) return CTH_NONFINITE;
    return loc.converged ? CTH_OK : CTH_NOT_CONVERGED;
}

int solve_finish(cth_grid* g, int pending, cth_status* st) {
    if (pending) CTH_CUDA(cudaStreamSynchronize(g->pending_stream));
    return solve_parse(g, pending, g->ws.h_stat, st);
}

int smg_solve_launch(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                     const double* aS, const double* b, int maxITR, double error_cnv, int precision,
                     double* solution, cudaStream_t s, int* pending, double* h_dst, const double* x0,
                     double guess_tol, const double* x0b, int slot) {
    if (slot < 0) slot = g->api_slot;
    if (x0 && !(guess_tol >= 0.0 && guess_tol <= 10.0)) {
        set_error("initial-guess threshold must be in [0, 10]");
        return CTH_ERR_ARG;
    }
    if (precision == CTH_PREC_MIXED)
        return solve_launch<float>(g, aP, aE, aW, aN, aS, b, maxITR, error_cnv, solution, s, precision, pending,
                                   h_dst, x0, guess_tol, x0b, slot);
    if (precision == CTH_PREC_FP64)
        return solve_launch<double>(g, aP, aE, aW, aN, aS, b, maxITR, error_cnv, solution, s, precision, pending,
                                    h_dst, x0, guess_tol, x0b, slot);
    set_error("unknown precision mode");
    return CTH_ERR_ARG;
}

int smg_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, int maxITR,
                  double error_cnv, int precision, double* solution, cudaStream_t s,
                  cth_status* st) {
    int pending = 0;
    const int rc = smg_solve_launch(g, aP, aE, aW, aN, aS, b, maxITR, error_cnv, precision, solution, s, &pending,
                                    nullptr);
    if (rc != CTH_OK) return rc;
    return solve_finish(g, pending, st);
}

// complex multigrid used as the preconditioner of the complex Krylov solves
int cmg_alloc(cth_grid* g) { return alloc_hierarchy<cd>(g); }
int cmg_setup(cth_grid* g, cudaStream_t s) {
    const long long l0 = g->launches;
    setup_levels<cd>(g, s);
    const int n = (int)(g->launches - l0);
    g->launches = l0;
    return n;
}
int cmg_vcycle(cth_grid* g, cudaStream_t s) {
    const long long l0 = g->launches;
    vcycle<cd>(g, 0, s);
    const int n = (int)(g->launches - l0);
    g->launches = l0;
    return n;
}

// the same preconditioner with an FP32 complex hierarchy (mixed precision): the
// operators of every level and the interpolation weights are set up in FP64 (the
// Galerkin sums of an indefinite operator cancel, which FP32 accumulation does not
// survive on the coarse levels) and then rounded; the cycle runs in FP32 on the
// rounded right-hand side and its result is widened back
__global__ void k_cd_to_cf(const cd* __restrict__ src, cf* __restrict__ dst, size_t n) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = cf(src[k]);
}
constexpr int kMaxSeg = 48;
struct CvtSegs {
    const cd* src[kMaxSeg];
    cf* dst[kMaxSeg];
    size_t n[kMaxSeg];
    int count;
};
// grid-stride rounding of up to kMaxSeg arrays in one launch (blockIdx.y = segment)
__global__ void k_cd_to_cf_segs(CvtSegs S) {
    const int sgi = blockIdx.y;
    if (sgi >= S.count) return;
    const cd* __restrict__ src = S.src[sgi];
    cf* __restrict__ dst = S.dst[sgi];
    const size_t n = S.n[sgi];
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = cf(src[k]);
}
__global__ void k_cf_to_cd(const cf* __restrict__ src, cd* __restrict__ dst, size_t n) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = cd(src[k].x, src[k].y);
}
int cmg32_alloc(cth_grid* g) { return alloc_hierarchy<cf>(g); }
int cmg32_setup(cth_grid* g, cudaStream_t s) {
    const long long l0 = g->launches;
    setup_levels<cd>(g, s);
    int k = (int)(g->launches - l0);
    g->launches = l0;
    CvtSegs S{};
    for (int l = 0; l < g->nlev; l++) {
        const size_t n = (size_t)g->nrow[l] * g->ldl;
        const int npt = (l == 0) ? 5 : 9;
        const cd* src[3] = {g->hc.a[l], g->hc.wS[l], g->hc.wN[l]};
        cf* dst[3] = {g->hcf.a[l], g->hcf.wS[l], g->hcf.wN[l]};
        const size_t cnt[3] = {n * npt, n, n};
        for (int t = 0; t < 3; t++) {
            if (S.count == kMaxSeg) {
                k_cd_to_cf_segs<<<dim3(64, S.count), 256, 0, s>>>(S);
                k++;
                S.count = 0;
            }
            S.src[S.count] = src[t];
            S.dst[S.count] = dst[t];
            S.n[S.count] = cnt[t];
            S.count++;
        }
    }
    if (S.count > 0) {
        k_cd_to_cf_segs<<<dim3(64, S.count), 256, 0, s>>>(S);
        k++;
    }
    return k;
}
int cmg32_vcycle(cth_grid* g, cudaStream_t s) {
    const size_t n = (size_t)g->nrow[0] * g->ldl;
    const unsigned nb = (unsigned)((n + 255) / 256);
    k_cd_to_cf<<<nb, 256, 0, s>>>(g->hc.b[0], g->hcf.b[0], n);
    const long long l0 = g->launches;
    vcycle<cf>(g, 0, s);
    const int k = 2 + (int)(g->launches - l0);
    g->launches = l0;
    k_cf_to_cd<<<nb, 256, 0, s>>>(g->hcf.x[0], g->hc.x[0], n);
    return k;
}

// Device time of the z-line relaxation of one level in its operating mode: reps
// pairs of (even rows, odd rows) captured in one graph with programmatic
// dependent launch, as the smoother runs inside a cycle, timed with CUDA events
// on the grid's stream.  Uses the level's operator and factors of the last
// solve of that precision; the level's x is overwritten (scratch of the cycle).
template <typename T>
static int time_relax_impl(cth_grid* g, int l, int reps, double* us, double* bytes) {
    Hierarchy<T>& h = hier<T>(g);
    if (!h.allocated) {
        set_error("cth_grid_time_relax: no solve of this precision has run on the grid");
        return CTH_ERR_ARG;
    }
    cudaStream_t cs = g->cap[0];
    const bool prof = g->prof.on;
    g->prof.on = false;
    const long long l0 = g->launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CTH_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < reps; r++) {
        relax<T>(g, l, 0, 0, 0, cs);
        relax<T>(g, l, 1, 0, 0, cs);
    }
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    g->launches = l0;
    g->prof.on = prof;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, g->stream);  // warm
    if (e == cudaSuccess) e = cudaEventRecord(e0, g->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, g->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, g->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cth_grid_time_relax");
    const int nr = g->nrow[l];
    *us = 1e3 * (double)ms / (2.0 * reps);
    // algorithmic bytes per launch (one colour): rows x cells x 8 words
    *bytes = 0.5 * (double)nr * g->ncol * 8.0 * sizeof(T);
    return CTH_OK;
}

// reps cycles (V-cycle + FP64 update, or the V-cycle alone) captured one after
// another in one graph without the conditional loop, on the hierarchy of the last
// solve; the solve's state is left undefined (the next solve prepares its own)
template <typename T>
static int time_cycle_impl(cth_grid* g, int reps, int with_update, double* us) {
    Hierarchy<T>& h = hier<T>(g);
    if (!h.allocated) {
        set_error("cth_grid_time_cycle: no solve of this precision has run on the grid");
        return CTH_ERR_ARG;
    }
    cudaStream_t cs = g->cap[0];
    const bool prof = g->prof.on;
    g->prof.on = false;
    const long long l0 = g->launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CTH_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < reps; r++) {
        if (with_update) enqueue_body<T>(g, cs, 0, 0);
        else vcycle<T>(g, 0, cs);
    }
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    g->launches = l0;
    g->prof.on = prof;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, g->stream);  // warm
    if (e == cudaSuccess) e = cudaEventRecord(e0, g->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, g->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, g->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cth_grid_time_cycle");
    *us = 1e3 * (double)ms / reps;
    return CTH_OK;
}

int time_cycle(cth_grid* g, int precision, int reps, int with_update, double* us) {
    if (reps < 1 || reps > 1000) {
        set_error("cth_grid_time_cycle: repetitions out of range");
        return CTH_ERR_ARG;
    }
    auto first = [&](auto* hs) {
        for (int k = 0; k < kHier; k++)
            if (hs[k].allocated) return k;
        return 0;
    };
    int rc;
    if (precision == CTH_PREC_MIXED) {
        g->cur = first(g->h32);
        rc = time_cycle_impl<float>(g, reps, with_update, us);
    } else if (precision == CTH_PREC_FP64) {
        g->cur = first(g->h64);
        rc = time_cycle_impl<double>(g, reps, with_update, us);
    } else {
        set_error("unknown precision mode");
        rc = CTH_ERR_ARG;
    }
    g->cur = 0;
    return rc;
}

int time_relax(cth_grid* g, int precision, int level, int reps, double* us, double* bytes) {
    if (level < 0 || level >= g->nlev || reps < 1 || reps > 1000) {
        set_error("cth_grid_time_relax: level or repetitions out of range");
        return CTH_ERR_ARG;
    }
    // the first hierarchy of the precision that a solve has built (slot hierarchies included)
    auto first = [&](auto* hs) {
        for (int k = 0; k < kHier; k++)
            if (hs[k].allocated) return k;
        return 0;
    };
    int rc;
    if (precision == CTH_PREC_MIXED) {
        g->cur = first(g->h32);
        rc = time_relax_impl<float>(g, level, reps, us, bytes);
        g->cur = 0;
        return rc;
    }
    if (precision == CTH_PREC_FP64) {
        g->cur = first(g->h64);
        rc = time_relax_impl<double>(g, level, reps, us, bytes);
        g->cur = 0;
        return rc;
    }
    set_error("unknown precision mode");
    return CTH_ERR_ARG;
}

template <typename T, int B>
static cudaError_t line_smem_attr_b(int bytes) {
    const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(k_relax<T, 5, 0, B>, A, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_relax<T, 9, 0, B>, A, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_relax<T, 9, 5, B>, A, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_relax<T, 9, 9, B>, A, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_weights<T, 5, B>, A, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_weights<T, 9, B>, A, bytes);
    return e;
}

// the dynamic shared memory limit of the line kernels of type T at launch bound bnd
template <typename T>
static cudaError_t line_smem_attr(int bnd, int bytes) {
    return bnd == 1024 ? line_smem_attr_b<T, 1024>(bytes)
         : bnd == 512  ? line_smem_attr_b<T, 512>(bytes)
                       : line_smem_attr_b<T, 256>(bytes);
}

// dynamic shared memory limits for the line kernels (called once per grid)
int configure_kernels(cth_grid* g) {
    const int smem64 = (int)line_smem<double>(g->bd, 2);
    const int smem32 = (int)line_smem<float>(g->bd, 2);
    if (smem64 > 227 * 1024) {
        set_error("z-line too long for the shared-memory line solver");
        return CTH_ERR_UNSUPPORTED;
    }
#define CTH_ATTR(K, BYTES) CTH_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, BYTES))
    // launch bounds of the line kernels for this line's thread count
    g->bnd = g->bd <= 256 ? 256 : (g->bd <= 512 ? 512 : 1024);
    if (smem64 > 48 * 1024) CTH_CUDA(line_smem_attr<double>(g->bnd, smem64));
    const int smemc = (int)line_smem<cd>(g->bd, 2);
    if (smemc > 227 * 1024) {
        set_error("z-line too long for the shared-memory complex line solver");
        return CTH_ERR_UNSUPPORTED;
    }
    if (smemc > 48 * 1024) CTH_CUDA(line_smem_attr<cd>(g->bnd, smemc));
    const int smemcf = (int)line_smem<cf>(g->bd, 2);
    if (smemcf > 48 * 1024) CTH_CUDA(line_smem_attr<cf>(g->bnd, smemcf));
    if (smem32 > 48 * 1024) CTH_CUDA(line_smem_attr<float>(g->bnd, smem32));
    // the fused tail runs only where a CTA of the line's width fits the registers
    g->tail_types = 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_tail<float>) == cudaSuccess && fa.maxThreadsPerBlock >= g->bd) g->tail_types |= 1;
    if (cudaFuncGetAttributes(&fa, k_tail<double>) == cudaSuccess && fa.maxThreadsPerBlock >= g->bd) g->tail_types |= 2;
    if (cudaFuncGetAttributes(&fa, k_tail<cd>) == cudaSuccess && fa.maxThreadsPerBlock >= g->bd) g->tail_types |= 4;
    cudaGetLastError();
    // the fused tail needs one right-hand side of line-solver memory
    if (line_smem<cd>(g->bd, 1) > 48 * 1024) CTH_ATTR((k_tail<cd>), (int)line_smem<cd>(g->bd, 1));
    if (line_smem<double>(g->bd, 1) > 48 * 1024) CTH_ATTR((k_tail<double>), (int)line_smem<double>(g->bd, 1));
    if (line_smem<float>(g->bd, 1) > 48 * 1024) CTH_ATTR((k_tail<float>), (int)line_smem<float>(g->bd, 1));
    // the defect correction's shared copy of the caller's operator (plus its static reduction words)
    CTH_ATTR((k_update<float>), (int)kUpdSmem);
    CTH_ATTR((k_update<double>), (int)kUpdSmem);
#undef CTH_ATTR
    return CTH_OK;
}

}  // namespace cth
