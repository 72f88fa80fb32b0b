// helm.cu — complex 5-point solves of the frequency-domain microwave path.
//
// Replaces the direct sparse factorisation (Eigen SparseLU) that
// EmfieldModule::solve_Microwave / solve_Microwave_impedanceTest use for their
// complex field systems (include/emfieldModule.hpp:2995-2998, :5780-5783): the
// system aP x_P - aE x_E - aW x_W - aN x_N - aS x_S = b on the block union of the
// field's unknowns (couplings to non-unknowns dropped, as the Eigen assembly
// inserts only unknown-to-unknown entries, :5749-5766) is solved by BiCGStab in
// complex FP64, right-preconditioned with one V-cycle of the semicoarsening
// multigrid of smg.cu in complex arithmetic (r is coarsened, z-lines are solved
// exactly, so the propagation direction along z is never coarsened), from a
// zero initial guess until ||r||_2 / ||b||_2 < tol.  Each solve is one CUDA graph whose iteration loop
// is a device-side conditional node; the scalars of the recurrence live in
// device memory and are updated by the last block of each reduction.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "grid.h"
#include "line.cuh"

namespace cth {

// scalar words (double) of the recurrence
enum C5Word {
    C5_RHO = 0,      // complex <rh, r>
    C5_RHO_OLD = 2,  // complex
    C5_ALPHA = 4,    // complex
    C5_OMEGA = 6,    // complex
    C5_BETA = 8,     // complex
    C5_BB = 10,
    C5_RR = 11,
    C5_RELRES = 12,
    C5_ITER = 13,
    C5_CONV = 14,
    C5_BAD = 15,     // breakdown or non-finite
    C5_KEEP = 16,
    C5_NWORDS = 24
};

struct C5Dev {
    cd *aP, *aW, *aE, *aS, *aN;   // level-0 planes of the complex hierarchy
    cd *b0, *x0;                  // preconditioner right-hand side / result
    cd *x, *r, *rh, *p, *ph, *v, *s, *sh, *t;
    double* sc;
    int ncol, nrow, ld;
};

int cmg_alloc(cth_grid* g);
int cmg_setup(cth_grid* g, cudaStream_t s);
int cmg_vcycle(cth_grid* g, cudaStream_t s);

__device__ __forceinline__ cd sc_c(const double* sc, int w) { return cd(sc[w], sc[w + 1]); }
__device__ __forceinline__ void sc_set(double* sc, int w, cd v) { sc[w] = v.x; sc[w + 1] = v.y; }

// y = A x at cell (c, rr) of the level-0 layout
__device__ __forceinline__ cd apply5(const C5Dev& W, const cd* __restrict__ x, int c, int rr) {
    const size_t p = (size_t)rr * W.ld + c;
    cd y = W.aP[p] * x[p];
    if (c > 0) y -= W.aW[p] * x[p - 1];
    if (c + 1 < W.ncol) y -= W.aE[p] * x[p + 1];
    if (rr > 0) y -= W.aS[p] * x[p - W.ld];
    if (rr + 1 < W.nrow) y -= W.aN[p] * x[p + W.ld];
    return y;
}

// masked copy of the caller's planes, r = rh = b, x = p = v = 0; last block
// initialises the recurrence
__global__ void k_c5_prep(const SolveArgs* __restrict__ args, const unsigned char* __restrict__ mask,
                          int ld_u, int i0, int j0, C5Dev W, double* __restrict__ part,
                          unsigned int* counter, cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double red[32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    double bb = 0.0;
    if (c < W.ncol) {
        const size_t p = (size_t)rr * W.ld + c;
        const size_t q = (size_t)(rr + j0) * ld_u + (c + i0);
        const cd* A0 = reinterpret_cast<const cd*>(args->aP);
        cd vP(1.0), vW, vE, vS, vN, vb;
        if (mask[p]) {
            vP = A0[q];
            if (c > 0 && mask[p - 1]) vW = reinterpret_cast<const cd*>(args->aW)[q];
            if (c + 1 < W.ncol && mask[p + 1]) vE = reinterpret_cast<const cd*>(args->aE)[q];
            if (rr > 0 && mask[p - W.ld]) vS = reinterpret_cast<const cd*>(args->aS)[q];
            if (rr + 1 < W.nrow && mask[p + W.ld]) vN = reinterpret_cast<const cd*>(args->aN)[q];
            vb = reinterpret_cast<const cd*>(args->b)[q];
            bb = abs2(vb);
        }
        W.aP[p] = vP; W.aW[p] = vW; W.aE[p] = vE; W.aS[p] = vS; W.aN[p] = vN;
        W.r[p] = vb; W.rh[p] = vb;
        W.x[p] = cd(); W.p[p] = cd(); W.v[p] = cd();
    }
    double tot;
    if (last_block_sum(bb, part, counter, red, &tot) && threadIdx.x == 0) {
        double* sc = W.sc;
        const bool fin = isfinite(tot);
        const bool keep = fin && tot > 0.0 && args->maxit > 0;
        sc_set(sc, C5_RHO, cd(tot));
        sc_set(sc, C5_RHO_OLD, cd(1.0));
        sc_set(sc, C5_ALPHA, cd(1.0));
        sc_set(sc, C5_OMEGA, cd(1.0));
        sc_set(sc, C5_BETA, cd(0.0));
        sc[C5_BB] = tot;
        sc[C5_RR] = tot;
        sc[C5_RELRES] = tot > 0.0 ? 1.0 : 0.0;
        sc[C5_ITER] = 0.0;
        sc[C5_CONV] = (fin && tot == 0.0) ? 1.0 : 0.0;
        sc[C5_BAD] = fin ? 0.0 : 1.0;
        sc[C5_KEEP] = keep ? 1.0 : 0.0;
        if (use_cond) cudaGraphSetConditional(cond, keep ? 1u : 0u);
    }
}

// MODE 0: p = r + beta (p - omega v);  MODE 1: s = r - alpha v.  The vector
// is also the right-hand side of the following preconditioner V-cycle.
template <int MODE>
__global__ void k_c5_vec(C5Dev W) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    if (c >= W.ncol) return;
    const size_t p = (size_t)rr * W.ld + c;
    cd y;
    if (MODE == 0) {
        const cd beta = sc_c(W.sc, C5_BETA), omega = sc_c(W.sc, C5_OMEGA);
        y = W.r[p] + beta * (W.p[p] - omega * W.v[p]);
        W.p[p] = y;
    } else {
        const cd alpha = sc_c(W.sc, C5_ALPHA);
        y = W.r[p] - alpha * W.v[p];
        W.s[p] = y;
    }
    W.b0[p] = y;
}

// the preconditioner result x0 is kept (MODE 0: ph, MODE 1: sh), then
// MODE 0: v = A ph, alpha = rho / <rh, v>;  MODE 1: t = A sh, omega = <t, s> / <t, t>
template <int MODE>
__global__ void k_c5_mv(C5Dev W, double* __restrict__ part, unsigned int* counter) {
    __shared__ double red[32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    double acc[3] = {0.0, 0.0, 0.0};
    if (c < W.ncol) {
        const size_t p = (size_t)rr * W.ld + c;
        if (MODE == 0) {
            W.ph[p] = W.x0[p];
            const cd y = apply5(W, W.x0, c, rr);
            W.v[p] = y;
            const cd h = conj(W.rh[p]) * y;
            acc[0] = h.x; acc[1] = h.y;
        } else {
            W.sh[p] = W.x0[p];
            const cd y = apply5(W, W.x0, c, rr);
            W.t[p] = y;
            const cd h = conj(y) * W.s[p];
            acc[0] = h.x; acc[1] = h.y; acc[2] = abs2(y);
        }
    }
    double tot[3];
    if (last_block_sumk<3>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        double* sc = W.sc;
        if (MODE == 0) {
            const cd den(tot[0], tot[1]);
            if (abs2(den) == 0.0 || !isfinite(tot[0]) || !isfinite(tot[1])) {
                sc[C5_BAD] = 1.0;
                sc_set(sc, C5_ALPHA, cd(0.0));
            } else {
                sc_set(sc, C5_ALPHA, cdiv(sc_c(sc, C5_RHO), den));
            }
        } else {
            if (tot[2] == 0.0 || !isfinite(tot[2])) {
                sc_set(sc, C5_OMEGA, cd(0.0));
                if (!(tot[2] == 0.0)) sc[C5_BAD] = 1.0;
            } else {
                sc_set(sc, C5_OMEGA, cd(tot[0] / tot[2], tot[1] / tot[2]));
            }
        }
    }
}

// x += alpha ph + omega sh; r = s - omega t; stopping rule and next beta
__global__ void k_c5_upd(C5Dev W, const SolveArgs* __restrict__ args, double* __restrict__ part,
                         unsigned int* counter, cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double red[32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    double acc[3] = {0.0, 0.0, 0.0};
    if (c < W.ncol) {
        const size_t p = (size_t)rr * W.ld + c;
        const cd alpha = sc_c(W.sc, C5_ALPHA), omega = sc_c(W.sc, C5_OMEGA);
        W.x[p] = W.x[p] + alpha * W.ph[p] + omega * W.sh[p];
        const cd rn = W.s[p] - omega * W.t[p];
        W.r[p] = rn;
        const cd h = conj(W.rh[p]) * rn;
        acc[0] = abs2(rn); acc[1] = h.x; acc[2] = h.y;
    }
    double tot[3];
    if (last_block_sumk<3>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        double* sc = W.sc;
        const int it = (int)sc[C5_ITER] + 1;
        const double bb = sc[C5_BB];
        const double rel = bb > 0.0 ? sqrt(tot[0] / bb) : 0.0;
        const bool fin = isfinite(tot[0]) && isfinite(tot[1]) && isfinite(tot[2]);
        const cd rho_old = sc_c(sc, C5_RHO), rho(tot[1], tot[2]);
        const cd alpha = sc_c(sc, C5_ALPHA), omega = sc_c(sc, C5_OMEGA);
        bool bad = sc[C5_BAD] != 0.0 || !fin;
        const bool conv = fin && rel < args->tol;
        if (!conv && (abs2(rho_old) == 0.0 || abs2(omega) == 0.0)) bad = true;
        const cd beta = bad ? cd(0.0) : cdiv(rho, rho_old) * cdiv(alpha, omega);
        sc_set(sc, C5_RHO_OLD, rho_old);
        sc_set(sc, C5_RHO, rho);
        sc_set(sc, C5_BETA, beta);
        sc[C5_RR] = tot[0];
        sc[C5_RELRES] = rel;
        sc[C5_ITER] = (double)it;
        sc[C5_CONV] = conv ? 1.0 : 0.0;
        sc[C5_BAD] = bad ? 1.0 : 0.0;
        const bool keep = !conv && !bad && it < args->maxit;
        sc[C5_KEEP] = keep ? 1.0 : 0.0;
        if (use_cond) cudaGraphSetConditional(cond, keep ? 1u : 0u);
    }
}

__global__ void k_c5_store(const SolveArgs* __restrict__ args, C5Dev W, const unsigned char* __restrict__ mask,
                           int ld_u, int i0, int j0) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    if (c >= W.ncol) return;
    const size_t p = (size_t)rr * W.ld + c;
    if (mask[p]) reinterpret_cast<cd*>(args->solution)[(size_t)(rr + j0) * ld_u + (c + i0)] = W.x[p];
}

// ---------------------------------------------------------------------------
static C5Dev c5dev(cth_grid* g) {
    C5Work& w = g->c5;
    C5Dev W;
    const size_t n0 = (size_t)g->nrow[0] * g->ldl;
    cd* a0 = g->hc.a[0];
    W.aP = a0 + P * n0;
    W.aW = a0 + cth::W * n0;
    W.aE = a0 + E * n0;
    W.aS = a0 + S * n0;
    W.aN = a0 + N * n0;
    W.b0 = g->hc.b[0];
    W.x0 = g->hc.x[0];
    cd** f[9] = {&W.x, &W.r, &W.rh, &W.p, &W.ph, &W.v, &W.s, &W.sh, &W.t};
    for (int k = 0; k < 9; k++) *f[k] = reinterpret_cast<cd*>(w.buf) + k * n0;
    W.sc = w.sc;
    W.ncol = g->ncol;
    W.nrow = g->nrow[0];
    W.ld = g->ldl;
    return W;
}

static int c5_alloc(cth_grid* g) {
    C5Work& w = g->c5;
    if (w.buf) return CTH_OK;
    int rc = cmg_alloc(g);
    if (rc != CTH_OK) return rc;
    const size_t n0 = (size_t)g->nrow[0] * g->ldl;
    CTH_CUDA(cudaMalloc(&w.buf, 9 * n0 * sizeof(cd)));
    CTH_CUDA(cth::zero_fill(w.buf, 9 * n0 * sizeof(cd)));
    CTH_CUDA(cudaMalloc(&w.sc, C5_NWORDS * sizeof(double)));
    CTH_CUDA(cth::zero_fill(w.sc, C5_NWORDS * sizeof(double)));
    const int nb = ((g->ncol + 255) / 256) * g->nrow[0];
    w.npart = 3 * nb + 8;
    CTH_CUDA(cudaMalloc(&w.part, w.npart * sizeof(double)));
    return CTH_OK;
}

static int c5_pre(cth_grid* g, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond) {
    C5Dev W = c5dev(g);
    dim3 blk(256), grd((g->ncol + 255) / 256, g->nrow[0]);
    k_c5_prep<<<grd, blk, 0, s>>>(g->ws.d_args, g->mask[0], g->ld, g->i0, g->j0, W, g->c5.part, g->ws.counter,
                                  cond, use_cond);
    return 1 + cmg_setup(g, s);
}

static int c5_body(cth_grid* g, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond) {
    C5Dev W = c5dev(g);
    dim3 blk(256), grd((g->ncol + 255) / 256, g->nrow[0]);
    int n = 0;
    k_c5_vec<0><<<grd, blk, 0, s>>>(W);
    n += 1 + cmg_vcycle(g, s);
    k_c5_mv<0><<<grd, blk, 0, s>>>(W, g->c5.part, g->ws.counter);
    k_c5_vec<1><<<grd, blk, 0, s>>>(W);
    n += 2 + cmg_vcycle(g, s);
    k_c5_mv<1><<<grd, blk, 0, s>>>(W, g->c5.part, g->ws.counter);
    k_c5_upd<<<grd, blk, 0, s>>>(W, g->ws.d_args, g->c5.part, g->ws.counter, cond, use_cond);
    return n + 2;
}

static int c5_post(cth_grid* g, cudaStream_t s) {
    C5Dev W = c5dev(g);
    dim3 blk(256), grd((g->ncol + 255) / 256, g->nrow[0]);
    k_c5_store<<<grd, blk, 0, s>>>(g->ws.d_args, W, g->mask[0], g->ld, g->i0, g->j0);
    return 1;
}

static int c5_build_graph(cth_grid* g, SolveGraph& G) {
    if (G.valid) return CTH_OK;
    cudaStream_t cs = g->cap[0], cs2 = g->cap[1];
    CTH_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
    cudaGraphConditionalHandle cond = 0;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        G.n_pre = c5_pre(g, cs, cond, 1);
        e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
    }
    cudaGraphNode_t cnode = nullptr;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(cs2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            G.n_body = c5_body(g, cs2, cond, 1);
            cudaGraph_t bout = nullptr;
            e = cudaStreamEndCapture(cs2, &bout);
        }
    }
    if (e == cudaSuccess) G.n_post = c5_post(g, cs);
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cs, &out);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&G.exec, out, 0);
    if (e != cudaSuccess) {
        if (out) cudaGraphDestroy(out);
        cudaGetLastError();
        return cuda_fail(e, "complex solve graph capture");
    }
    G.graph = out;
    G.valid = true;
    return CTH_OK;
}

int c5_configure(cth_grid*) { return CTH_OK; }

int c5_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                 const double* aS, const double* b, int maxit, double tol, double* solution, cudaStream_t s,
                 cth_status* st) {
    int rc = c5_alloc(g);
    if (rc != CTH_OK) return rc;
    Workspace& w = g->ws;
    SolveArgs* ha = w.h_args;
    ha->aP = aP; ha->aE = aE; ha->aW = aW; ha->aN = aN; ha->aS = aS; ha->b = b;
    ha->solution = solution;
    ha->tol = tol;
    ha->maxit = maxit;
    CTH_CUDA(cudaMemcpyAsync(w.d_args, ha, sizeof(SolveArgs), cudaMemcpyHostToDevice, s));
    double h[C5_NWORDS];
    if (g->use_graphs) {
        rc = c5_build_graph(g, g->c5graph);
        if (rc != CTH_OK) return rc;
        CTH_CUDA(cudaGraphLaunch(g->c5graph.exec, s));
        CTH_CUDA(cudaMemcpyAsync(w.h_stat, g->c5.sc, C5_NWORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        std::memcpy(h, w.h_stat, sizeof(h));
        g->launches += g->c5graph.n_pre + (long long)g->c5graph.n_body * (long long)h[C5_ITER] + g->c5graph.n_post;
    } else {
        g->launches += c5_pre(g, s, 0, 0);
        for (;;) {
            CTH_CUDA(cudaMemcpyAsync(w.h_stat, g->c5.sc, C5_NWORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
            CTH_CUDA(cudaStreamSynchronize(s));
            if (w.h_stat[C5_KEEP] == 0.0) break;
            g->launches += c5_body(g, s, 0, 0);
        }
        g->launches += c5_post(g, s);
        CTH_CUDA(cudaStreamSynchronize(s));
        std::memcpy(h, w.h_stat, sizeof(h));
    }
    CTH_CUDA(cudaGetLastError());
    cth_status loc{};
    loc.iterations = (int)h[C5_ITER];
    loc.residual = h[C5_RELRES];
    loc.initial_residual = std::sqrt(h[C5_BB]);
    loc.converged = h[C5_CONV] != 0.0;
    loc.nonfinite = h[C5_BAD] != 0.0 && !loc.converged;
    if (st) *st = loc;
    if (loc.nonfinite) return CTH_NONFINITE;
    return loc.converged ? CTH_OK : CTH_NOT_CONVERGED;
}

}  // namespace cth
