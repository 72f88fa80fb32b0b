// capi.cu — extern "C" entry points of libcathode_b200.so (include/cathode_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "grid.h"

namespace cth {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }

int cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
            ") at " + what;
    return CTH_ERR_CUDA;
}

int configure_kernels(cth_grid* g);

// [i][j] (i outer, row length nj+2) -> device layout (j outer, ld): 32x32 tiles
__global__ void k_ij_to_dev(const double* __restrict__ src, double* __restrict__ dst, int ni2,
                            int nj2, int ld) {
    __shared__ double tile[32][33];
    const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, j = j0 + threadIdx.x;
        if (i < ni2 && j < nj2) tile[k][threadIdx.x] = src[(size_t)i * nj2 + j];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int j = j0 + k, i = i0 + threadIdx.x;
        if (i < ni2 && j < nj2) dst[(size_t)j * ld + i] = tile[threadIdx.x][k];
    }
}

__global__ void k_dev_to_ij(const double* __restrict__ src, double* __restrict__ dst, int ni2,
                            int nj2, int ld) {
    __shared__ double tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int j = j0 + k, i = i0 + threadIdx.x;
        if (i < ni2 && j < nj2) tile[k][threadIdx.x] = src[(size_t)j * ld + i];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, j = j0 + threadIdx.x;
        if (i < ni2 && j < nj2) dst[(size_t)i * nj2 + j] = tile[threadIdx.x][k];
    }
}

// complex (16-byte) element versions
__global__ void k_ij_to_dev_c(const double2* __restrict__ src, double2* __restrict__ dst, int ni2, int nj2,
                              int ld) {
    __shared__ double2 tile[32][33];
    const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, j = j0 + threadIdx.x;
        if (i < ni2 && j < nj2) tile[k][threadIdx.x] = src[(size_t)i * nj2 + j];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int j = j0 + k, i = i0 + threadIdx.x;
        if (i < ni2 && j < nj2) dst[(size_t)j * ld + i] = tile[threadIdx.x][k];
    }
}

__global__ void k_dev_to_ij_c(const double2* __restrict__ src, double2* __restrict__ dst, int ni2, int nj2,
                              int ld) {
    __shared__ double2 tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int j = j0 + k, i = i0 + threadIdx.x;
        if (i < ni2 && j < nj2) tile[k][threadIdx.x] = src[(size_t)j * ld + i];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, j = j0 + threadIdx.x;
        if (i < ni2 && j < nj2) dst[(size_t)i * nj2 + j] = tile[threadIdx.x][k];
    }
}

int to_device_layout(cth_grid* g, const double* src, double* dst, cudaStream_t s) {
    dim3 blk(32, 8), grd((g->nj + 2 + 31) / 32, (g->ni + 2 + 31) / 32);
    k_ij_to_dev<<<grd, blk, 0, s>>>(src, dst, g->ni + 2, g->nj + 2, g->ld);
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

int from_device_layout(cth_grid* g, const double* src, double* dst, cudaStream_t s) {
    dim3 blk(32, 8), grd((g->ni + 2 + 31) / 32, (g->nj + 2 + 31) / 32);
    k_dev_to_ij<<<grd, blk, 0, s>>>(src, dst, g->ni + 2, g->nj + 2, g->ld);
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

int prof_mark(cth_grid* g, int c, double bytes, cudaStream_t s) {
    Profiler& p = g->prof;
    if (!p.on) return -1;
    if (p.used * 2 + 2 > p.ev.size()) {
        for (int k = 0; k < 64; k++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            p.ev.push_back(e);
        }
        p.cls.resize(p.ev.size() / 2);
        p.bytes.resize(p.ev.size() / 2);
    }
    const size_t k = p.used++;
    p.cls[k] = c;
    p.bytes[k] = bytes;
    cudaEventRecord(p.ev[2 * k], s);
    return (int)k;
}

void prof_done(cth_grid* g, int slot, cudaStream_t s) {
    if (slot < 0) return;
    cudaEventRecord(g->prof.ev[2 * slot + 1], s);
}

void prof_collect(cth_grid* g) {
    Profiler& p = g->prof;
    for (size_t k = 0; k < p.used; k++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.ev[2 * k], p.ev[2 * k + 1]) == cudaSuccess) {
            p.ms[p.cls[k]] += ms;
            p.n[p.cls[k]] += 1;
            p.nbytes[p.cls[k]] += p.bytes[k];
        }
    }
    p.used = 0;
}

int ensure_staging(cth_grid* g) {
    Workspace& w = g->ws;
    if (w.stage) return CTH_OK;
    CTH_CUDA(cudaSetDevice(g->device));
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    CTH_CUDA(cudaMalloc(&w.stage, 7 * g->plane * sizeof(double)));
    CTH_CUDA(cth::zero_fill(w.stage, 7 * g->plane * sizeof(double)));
    CTH_CUDA(cudaMalloc(&w.stage_ij, nij * sizeof(double)));
    return CTH_OK;
}

static void free_grid(cth_grid* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    auto fr = [](void* p) { if (p) cudaFree(p); };
    fr(g->mask_full);
    for (auto p : g->mask) fr(p);
    for (int k = 0; k < cth::kHier; k++) {
        for (auto* v : {&g->h32[k].a, &g->h32[k].x, &g->h32[k].b, &g->h32[k].wS, &g->h32[k].wN, &g->h32[k].fac})
            for (auto p : *v) fr(p);
        for (auto* v : {&g->h64[k].a, &g->h64[k].x, &g->h64[k].b, &g->h64[k].wS, &g->h64[k].wN, &g->h64[k].fac})
            for (auto p : *v) fr(p);
    }
    for (auto* v : {&g->hc.a, &g->hc.x, &g->hc.b, &g->hc.wS, &g->hc.wN, &g->hc.fac})
        for (auto p : *v) fr(p);
    for (auto* v : {&g->hcf.a, &g->hcf.x, &g->hcf.b, &g->hcf.wS, &g->hcf.wN, &g->hcf.fac})
        for (auto p : *v) fr(p);
    fr(g->ws.x64[0]);
    fr(g->ws.x64[1]);
    fr(g->ws.part);
    fr(g->ws.stat);
    fr(g->ws.stage);
    fr(g->ws.stage_ij);
    if (g->ws.h_stat) cudaFreeHost(g->ws.h_stat);
    if (g->ws.h_args) cudaFreeHost(g->ws.h_args);
    fr(g->ws.d_args);
    fr(g->ws.counter);
    fr(g->ws.slotstat);
    fr(g->c5.buf);
    fr(g->c5.sc);
    fr(g->c5.part);
    fr(g->c5.cstage);
    fr(g->c5.cstage_ij);
    if (g->c5graph.exec) cudaGraphExecDestroy(g->c5graph.exec);
    if (g->c5graph.graph) cudaGraphDestroy(g->c5graph.graph);
    for (auto& row : g->graphs)
        for (auto& G : row) {
            if (G.exec) cudaGraphExecDestroy(G.exec);
            if (G.graph) cudaGraphDestroy(G.graph);
        }
    for (auto c : g->cap) if (c) cudaStreamDestroy(c);
    if (g->stream) cudaStreamDestroy(g->stream);
    for (auto e : g->prof.ev) cudaEventDestroy(e);
    delete g;
}

}  // namespace cth

using namespace cth;

static const char kVersion[] = "cathode_b200 0.1 (sm_100a)";

// host mask of the reference's [i][j] layout (solverFuncs.hpp:43-47)
static std::vector<unsigned char> host_mask(int ni, int nj, const std::vector<int>& ibl,
                                            const std::vector<int>& jbl) {
    std::vector<unsigned char> m((size_t)(ni + 2) * (nj + 2), 0);
    const int nb = (int)ibl.size() / 2;
    for (int b = 0; b < nb; b++)
        for (int i = std::max(0, ibl[2 * b]); i <= std::min(ni + 1, ibl[2 * b + 1]); i++)
            for (int j = std::max(0, jbl[2 * b]); j <= std::min(nj + 1, jbl[2 * b + 1]); j++)
                m[(size_t)i * (nj + 2) + j] = 1;
    return m;
}

extern "C" {

const char* cth_version(void) { return kVersion; }
const char* cth_last_error(void) { return g_err.c_str(); }

int cth_grid_create(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl, int device,
                    cth_grid** out) {
    if (!out || ni < 1 || nj < 1 || n_bl < 1 || !i_bl || !j_bl) {
        set_error("cth_grid_create: invalid arguments");
        return CTH_ERR_ARG;
    }
    *out = nullptr;
    cth_grid* g = new cth_grid();
    g->ni = ni;
    g->nj = nj;
    g->n_bl = n_bl;
    g->ibl.assign(i_bl, i_bl + 2 * n_bl);
    g->jbl.assign(j_bl, j_bl + 2 * n_bl);
    g->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { free_grid(g); return cuda_fail(e, "cudaSetDevice"); }
    g->ld = ((ni + 2 + 31) / 32) * 32;
    g->plane = (size_t)(nj + 2) * g->ld;
    std::vector<unsigned char> hm = host_mask(ni, nj, g->ibl, g->jbl);
    // bounding box
    g->i0 = ni + 2; g->i1 = -1; g->j0 = nj + 2; g->j1 = -1;
    for (int i = 0; i <= ni + 1; i++)
        for (int j = 0; j <= nj + 1; j++)
            if (hm[(size_t)i * (nj + 2) + j]) {
                g->i0 = std::min(g->i0, i); g->i1 = std::max(g->i1, i);
                g->j0 = std::min(g->j0, j); g->j1 = std::max(g->j1, j);
            }
    if (g->i1 < 0) {
        set_error("cth_grid_create: the block union is empty");
        free_grid(g);
        return CTH_ERR_ARG;
    }
    g->ncol = g->i1 - g->i0 + 1;
    g->ldl = ((g->ncol + 31) / 32) * 32;
    g->qref = (size_t)g->jbl[0] * g->ld + g->ibl[0];
    if (g->ncol > 4096) {
        set_error("cth_grid_create: z-lines longer than 4096 cells are not supported");
        free_grid(g);
        return CTH_ERR_UNSUPPORTED;
    }
    // line solver: 4 cells per thread, 32..1024 threads per z-line
    g->bd = std::max(32, (((g->ncol + 3) / 4 + 31) / 32) * 32);
    g->ept = 4;
    // levels
    for (int r = g->j1 - g->j0 + 1;; r = (r + 1) / 2) {
        g->nrow.push_back(r);
        if (r == 1) break;
    }
    g->nlev = (int)g->nrow.size();
    // masks: device layout + per-level layout
    std::vector<unsigned char> mfull(g->plane, 0);
    for (int i = 0; i <= ni + 1; i++)
        for (int j = 0; j <= nj + 1; j++) mfull[(size_t)j * g->ld + i] = hm[(size_t)i * (nj + 2) + j];
    std::vector<std::vector<unsigned char>> ml(g->nlev);
    ml[0].assign((size_t)g->nrow[0] * g->ldl, 0);
    for (int r = 0; r < g->nrow[0]; r++)
        for (int c = 0; c < g->ncol; c++)
            ml[0][(size_t)r * g->ldl + c] = hm[(size_t)(c + g->i0) * (nj + 2) + (r + g->j0)];
    for (int l = 1; l < g->nlev; l++) {
        ml[l].assign((size_t)g->nrow[l] * g->ldl, 0);
        for (int r = 0; r < g->nrow[l]; r++)
            for (int c = 0; c < g->ncol; c++)
                ml[l][(size_t)r * g->ldl + c] = ml[l - 1][(size_t)(2 * r) * g->ldl + c];
    }
    int rc = CTH_OK;
    auto chk = [&](cudaError_t ce, const char* w) {
        if (ce != cudaSuccess && rc == CTH_OK) rc = cuda_fail(ce, w);
    };
    chk(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    chk(cudaMalloc(&g->mask_full, g->plane), "cudaMalloc mask");
    if (rc == CTH_OK) chk(cudaMemcpy(g->mask_full, mfull.data(), g->plane, cudaMemcpyHostToDevice), "memcpy mask");
    g->mask.assign(g->nlev, nullptr);
    for (int l = 0; l < g->nlev && rc == CTH_OK; l++) {
        chk(cudaMalloc(&g->mask[l], ml[l].size()), "cudaMalloc level mask");
        if (rc == CTH_OK) chk(cudaMemcpy(g->mask[l], ml[l].data(), ml[l].size(), cudaMemcpyHostToDevice), "memcpy level mask");
    }
    const size_t n0 = (size_t)g->nrow[0] * g->ldl;
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.x64[0], n0 * sizeof(double)), "cudaMalloc x64");
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.x64[1], n0 * sizeof(double)), "cudaMalloc x64");
    // partial-sum blocks: enough for 256-wide blocks over the full padded index space, twice
    g->ws.npart = 3 * (((ni + 2 + 255) / 256) * (nj + 2) + 64);
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.part, (size_t)g->ws.npart * sizeof(double)), "cudaMalloc part");
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.stat, 32 * sizeof(double)), "cudaMalloc stat");
    if (rc == CTH_OK) chk(cth::zero_fill(g->ws.stat, 32 * sizeof(double)), "memset stat");
    if (rc == CTH_OK) chk(cudaMallocHost(&g->ws.h_stat, 32 * sizeof(double)), "cudaMallocHost");
    if (rc == CTH_OK) chk(cudaMallocHost(&g->ws.h_args, sizeof(cth::SolveArgs)), "cudaMallocHost args");
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.d_args, sizeof(cth::SolveArgs)), "cudaMalloc args");
    if (rc == CTH_OK) chk(cudaMalloc(&g->ws.counter, 64), "cudaMalloc counter");
    if (rc == CTH_OK) chk(cth::zero_fill(g->ws.counter, 64), "memset counter");
    {
        const size_t nss = (2 * cth::kSlots * cth::kSlotWords + 1) * sizeof(double);
        if (rc == CTH_OK) chk(cudaMalloc(&g->ws.slotstat, nss), "cudaMalloc slot words");
        if (rc == CTH_OK) chk(cth::zero_fill(g->ws.slotstat, nss), "memset slot words");
    }
    if (rc == CTH_OK) chk(cudaStreamCreateWithFlags(&g->cap[0], cudaStreamNonBlocking), "capture stream");
    if (rc == CTH_OK) chk(cudaStreamCreateWithFlags(&g->cap[1], cudaStreamNonBlocking), "capture stream");
    if (rc == CTH_OK) rc = configure_kernels(g);
    if (rc == CTH_OK) rc = c5_configure(g);
    if (rc != CTH_OK) {
        free_grid(g);
        return rc;
    }
    *out = g;
    return CTH_OK;
}

void cth_grid_destroy(cth_grid* g) { free_grid(g); }

int cth_grid_ld(const cth_grid* g) { return g ? g->ld : 0; }
int cth_grid_levels(const cth_grid* g) { return g ? g->nlev : 0; }

long long cth_launch_count(const cth_grid* g) { return g ? g->launches : -1; }

int cth_profile(cth_grid* g, int enable) {
    if (!g) { set_error("cth_profile: null grid"); return CTH_ERR_ARG; }
    Profiler& p = g->prof;
    p.on = enable != 0;
    p.used = 0;
    for (int c = 0; c < PROF_NCLASS; c++) { p.ms[c] = 0; p.n[c] = 0; p.nbytes[c] = 0; }
    return CTH_OK;
}

int cth_grid_time_relax(cth_grid* g, int precision, int level, int reps, double* us_per_launch,
                        double* bytes_per_launch) {
    if (!g || !us_per_launch || !bytes_per_launch) {
        set_error("cth_grid_time_relax: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    return time_relax(g, precision, level, reps, us_per_launch, bytes_per_launch);
}

int cth_grid_time_cycle(cth_grid* g, int precision, int reps, int with_update, double* us_per_cycle) {
    if (!g || !us_per_cycle) {
        set_error("cth_grid_time_cycle: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    return time_cycle(g, precision, reps, with_update, us_per_cycle);
}

int cth_profile_read(const cth_grid* g, int cls, double* ms, long long* launches, double* bytes) {
    if (!g || cls < 0 || cls >= PROF_NCLASS) { set_error("cth_profile_read: invalid arguments"); return CTH_ERR_ARG; }
    if (ms) *ms = g->prof.ms[cls];
    if (launches) *launches = g->prof.n[cls];
    if (bytes) *bytes = g->prof.nbytes[cls];
    return CTH_OK;
}

int cth_grid_set_graphs(cth_grid* g, int enable) {
    if (!g) { set_error("cth_grid_set_graphs: null grid"); return CTH_ERR_ARG; }
    g->use_graphs = enable != 0;
    return CTH_OK;
}

static void drop_graph(cth::SolveGraph& G) {
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.graph) cudaGraphDestroy(G.graph);
    G.exec = nullptr;
    G.graph = nullptr;
    G.valid = false;
}

int cth_grid_set_tail(cth_grid* g, int enable) {
    if (!g) { set_error("cth_grid_set_tail: null grid"); return CTH_ERR_ARG; }
    if ((enable != 0) != g->tail) {
        CTH_CUDA(cudaSetDevice(g->device));
        CTH_CUDA(cudaDeviceSynchronize());
        g->tail = enable != 0;
        for (auto& row : g->graphs)
            for (auto& G : row) drop_graph(G);
        drop_graph(g->c5graph);
    }
    return CTH_OK;
}

int cth_grid_set_reuse(cth_grid* g, double tol, int slot) {
    if (!g || !(tol >= 0.0) || slot < -1 || slot >= cth::kSlots) {
        set_error("cth_grid_set_reuse: tolerance must be >= 0 and the slot in -1..14");
        return CTH_ERR_ARG;
    }
    g->reuse_tol = tol;
    g->api_slot = slot;
    return CTH_OK;
}

int cth_grid_reuse_stats(cth_grid* g, int precision, int slot, double* out) {
    if (!g || !out || slot < 0 || slot >= cth::kSlots || (precision != CTH_PREC_FP64 && precision != CTH_PREC_MIXED)) {
        set_error("cth_grid_reuse_stats: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    CTH_CUDA(cudaDeviceSynchronize());
    double w[cth::kSlotWords];
    CTH_CUDA(cudaMemcpy(w, g->ws.slotstat + ((size_t)precision * cth::kSlots + slot) * cth::kSlotWords, sizeof(w),
                        cudaMemcpyDeviceToHost));
    out[0] = w[cth::SW_SETUPS];
    out[1] = w[cth::SW_REUSES];
    out[2] = w[cth::SW_CHANGE];
    out[3] = w[cth::SW_LASTITER];
    out[4] = w[cth::SW_RETRIES];
    return CTH_OK;
}

int cth_grid_set_cycle(cth_grid* g, int nu_pre, int nu_post) {
    if (!g || nu_pre < 1 || nu_post < 1 || nu_pre > 8 || nu_post > 8) {
        set_error("cth_grid_set_cycle: sweeps must be in 1..8");
        return CTH_ERR_ARG;
    }
    g->nu1 = nu_pre;
    g->nu2 = nu_post;
    return CTH_OK;
}

static int upload_inputs(cth_grid* g, const double* const* src, int n, double* base) {
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    for (int k = 0; k < n; k++) {
        CTH_CUDA(cudaMemcpyAsync(g->ws.stage_ij, src[k], nij * sizeof(double), cudaMemcpyHostToDevice,
                                 g->stream));
        int rc = to_device_layout(g, g->ws.stage_ij, base + k * g->plane, g->stream);
        if (rc != CTH_OK) return rc;
    }
    return CTH_OK;
}

// copy the grid cells of a device-layout plane into the caller's [i][j] array
static int download_grid_cells(cth_grid* g, const double* dev_plane, double* host_ij) {
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    int rc = from_device_layout(g, dev_plane, g->ws.stage_ij, g->stream);
    if (rc != CTH_OK) return rc;
    std::vector<double> tmp(nij);
    CTH_CUDA(cudaMemcpyAsync(tmp.data(), g->ws.stage_ij, nij * sizeof(double), cudaMemcpyDeviceToHost,
                             g->stream));
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    // write back block cells only (solverFuncs.hpp:143-152)
    const int nb = g->n_bl, nj2 = g->nj + 2;
    for (int b = 0; b < nb; b++)
        for (int i = std::max(0, g->ibl[2 * b]); i <= std::min(g->ni + 1, g->ibl[2 * b + 1]); i++)
            for (int j = std::max(0, g->jbl[2 * b]); j <= std::min(g->nj + 1, g->jbl[2 * b + 1]); j++)
                host_ij[(size_t)i * nj2 + j] = tmp[(size_t)i * nj2 + j];
    return CTH_OK;
}

int cth_smg_solve(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, int maxITR,
                  double error_cnv, int precision, double* solution, cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution || maxITR < 0) {
        set_error("cth_smg_solve: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    int rc = ensure_staging(g);
    if (rc != CTH_OK) return rc;
    const double* src[6] = {aP, aE, aW, aN, aS, b};
    double* base = g->ws.stage;
    rc = upload_inputs(g, src, 6, base);
    if (rc != CTH_OK) return rc;
    double* xdev = base + 6 * g->plane;
    const double* P_ = base;
    int res = smg_solve_dev(g, P_, P_ + g->plane, P_ + 2 * g->plane, P_ + 3 * g->plane,
                            P_ + 4 * g->plane, P_ + 5 * g->plane, maxITR, error_cnv, precision, xdev,
                            g->stream, st);
    if (res < 0) return res;
    rc = download_grid_cells(g, xdev, solution);
    if (rc != CTH_OK) return rc;
    return res;
}

int cth_smg_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                      const double* aN, const double* aS, const double* b, int maxITR,
                      double error_cnv, int precision, double* solution, void* stream,
                      cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution || maxITR < 0) {
        set_error("cth_smg_solve_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    return smg_solve_dev(g, aP, aE, aW, aN, aS, b, maxITR, error_cnv, precision, solution,
                         (cudaStream_t)stream, st);
}

int cth_smg_solve_guess_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                            const double* aN, const double* aS, const double* b, const double* x0,
                            double max_guess_relres, int maxITR, double error_cnv, int precision,
                            double* solution, void* stream, cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !x0 || !solution || maxITR < 0 ||
        !(max_guess_relres >= 0.0 && max_guess_relres <= 10.0)) {
        set_error("cth_smg_solve_guess_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    int pending = 0;
    const int rc = smg_solve_launch(g, aP, aE, aW, aN, aS, b, maxITR, error_cnv, precision, solution,
                                    (cudaStream_t)stream, &pending, nullptr, x0, max_guess_relres);
    if (rc < 0) return rc;
    return solve_finish(g, pending, st);
}

int cth_sor_solve(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, double alpha_SOR,
                  int maxITR, double error_cnv, double* solution, cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution) {
        set_error("cth_sor_solve: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    int rc = ensure_staging(g);
    if (rc != CTH_OK) return rc;
    const double* src[7] = {aP, aE, aW, aN, aS, b, solution};
    double* base = g->ws.stage;
    rc = upload_inputs(g, src, 7, base);
    if (rc != CTH_OK) return rc;
    double* xdev = base + 6 * g->plane;
    const double* P_ = base;
    int res = sor_solve_dev(g, P_, P_ + g->plane, P_ + 2 * g->plane, P_ + 3 * g->plane,
                            P_ + 4 * g->plane, P_ + 5 * g->plane, alpha_SOR, maxITR, error_cnv, xdev,
                            g->stream, st);
    if (res < 0) return res;
    rc = download_grid_cells(g, xdev, solution);
    if (rc != CTH_OK) return rc;
    return res;
}

int cth_sor_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                      const double* aN, const double* aS, const double* b, double alpha_SOR,
                      int maxITR, double error_cnv, double* solution, void* stream,
                      cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution) {
        set_error("cth_sor_solve_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    return sor_solve_dev(g, aP, aE, aW, aN, aS, b, alpha_SOR, maxITR, error_cnv, solution,
                         (cudaStream_t)stream, st);
}

int cth_c5_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                     const double* aN, const double* aS, const double* b, int maxITR, double tol,
                     double* solution, void* stream, cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution || maxITR < 0) {
        set_error("cth_c5_solve_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    return c5_solve_dev(g, aP, aE, aW, aN, aS, b, maxITR, tol, solution, (cudaStream_t)stream, st);
}

int cth_c5_solve(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                 const double* aS, const double* b, int maxITR, double tol, double* solution,
                 cth_status* st) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !solution || maxITR < 0) {
        set_error("cth_c5_solve: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    C5Work& c = g->c5;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    if (!c.cstage) {
        CTH_CUDA(cudaMalloc(&c.cstage, 7 * g->plane * 2 * sizeof(double)));
        CTH_CUDA(cth::zero_fill(c.cstage, 7 * g->plane * 2 * sizeof(double)));
        CTH_CUDA(cudaMalloc(&c.cstage_ij, nij * 2 * sizeof(double)));
    }
    const double* src[6] = {aP, aE, aW, aN, aS, b};
    dim3 blk(32, 8), g1((g->nj + 2 + 31) / 32, (g->ni + 2 + 31) / 32), g2((g->ni + 2 + 31) / 32, (g->nj + 2 + 31) / 32);
    for (int k = 0; k < 6; k++) {
        CTH_CUDA(cudaMemcpyAsync(c.cstage_ij, src[k], nij * 2 * sizeof(double), cudaMemcpyHostToDevice, g->stream));
        k_ij_to_dev_c<<<g1, blk, 0, g->stream>>>(reinterpret_cast<const double2*>(c.cstage_ij),
                                                 reinterpret_cast<double2*>(c.cstage + k * g->plane * 2),
                                                 g->ni + 2, g->nj + 2, g->ld);
    }
    double* base = c.cstage;
    const size_t pl = g->plane * 2;
    int res = c5_solve_dev(g, base, base + pl, base + 2 * pl, base + 3 * pl, base + 4 * pl, base + 5 * pl,
                           maxITR, tol, base + 6 * pl, g->stream, st);
    if (res < 0) return res;
    k_dev_to_ij_c<<<g2, blk, 0, g->stream>>>(reinterpret_cast<const double2*>(base + 6 * pl),
                                             reinterpret_cast<double2*>(c.cstage_ij), g->ni + 2, g->nj + 2, g->ld);
    std::vector<double> tmp(nij * 2);
    CTH_CUDA(cudaMemcpyAsync(tmp.data(), c.cstage_ij, nij * 2 * sizeof(double), cudaMemcpyDeviceToHost, g->stream));
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    const int nj2 = g->nj + 2;
    for (int bl = 0; bl < g->n_bl; bl++)
        for (int i = std::max(0, g->ibl[2 * bl]); i <= std::min(g->ni + 1, g->ibl[2 * bl + 1]); i++)
            for (int j = std::max(0, g->jbl[2 * bl]); j <= std::min(g->nj + 1, g->jbl[2 * bl + 1]); j++) {
                solution[2 * ((size_t)i * nj2 + j)] = tmp[2 * ((size_t)i * nj2 + j)];
                solution[2 * ((size_t)i * nj2 + j) + 1] = tmp[2 * ((size_t)i * nj2 + j) + 1];
            }
    return res;
}

int cth_mw_er_assemble_dev(cth_grid* g, const double* ne, const double* nu, const double* epsr,
                           const cth_mw_params* prm, double* aP, double* aE, double* aW, double* aN,
                           double* aS, double* b, void* stream) {
    if (!g || !ne || !nu || !epsr || !prm || !aP || !aE || !aW || !aN || !aS || !b || prm->dx <= 0.0 ||
        prm->dr <= 0.0 || !(prm->r2 > prm->r1) || prm->r1 <= 0.0) {
        set_error("cth_mw_er_assemble_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    return mw_er_assemble_dev(g, ne, nu, epsr, prm, aP, aE, aW, aN, aS, b, (cudaStream_t)stream);
}

int cth_residual_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                     const double* aN, const double* aS, const double* b, const double* x,
                     double* r, double* rnorm, double* bnorm, void* stream) {
    if (!g || !aP || !aE || !aW || !aN || !aS || !b || !x) {
        set_error("cth_residual_dev: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    return residual_dev(g, aP, aE, aW, aN, aS, b, x, r, rnorm, bnorm, (cudaStream_t)stream);
}

int cth_to_device_layout(cth_grid* g, const double* src_ij, double* dst_dev, void* stream) {
    if (!g || !src_ij || !dst_dev) { set_error("cth_to_device_layout: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(g->device));
    return to_device_layout(g, src_ij, dst_dev, (cudaStream_t)stream);
}

int cth_from_device_layout(cth_grid* g, const double* src_dev, double* dst_ij, void* stream) {
    if (!g || !src_dev || !dst_ij) { set_error("cth_from_device_layout: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(g->device));
    return from_device_layout(g, src_dev, dst_ij, (cudaStream_t)stream);
}

}  // extern "C"
