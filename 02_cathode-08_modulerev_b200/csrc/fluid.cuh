// fluid.cuh — shared pieces of the FluidModule kernels: the field store, the
// side-flag bits of the fluid blocks, physical constants and the uniform-step
// table lookups of miniFuncs.hpp:35-91.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>

#include "grid.h"

#define CTH_FS_NSCAL 96
#define CTH_FS_NPART_PER_BLOCK 16
#define CTH_KEEP_WALL_MAX 4

namespace cth { struct RestartWriter; }

struct cth_fields {
    cth_grid* g = nullptr;
    cth::RestartWriter* restart = nullptr;  // restart-file writer (restart.cu): pinned staging, writer thread
    int* ghost_rules = nullptr;      // device, 7 ints per rule (i0, i1, j0, j1, di, dj, rhoe_mode)
    int n_ghost_rules = 0;
    int keep_wall[4 * CTH_KEEP_WALL_MAX] = {};  // r-face boxes where the energy sweep keeps Gr_wall
    int n_keep_wall = 0;
    cth_ion_op* ion_ops[CTH_ION_NPROG] = {};  // wall programs of the ion step
    int ion_nops[CTH_ION_NPROG] = {};
    int* ion_boxes[4] = {};                    // residual boxes (rhoi, Uix, Uir, Uip)
    int ion_nbox[4] = {};
    int ion_box_total[4] = {};
    bool aux_ready = false;
    cudaStream_t net_stream = nullptr;   // learned warm-start inference, concurrent with the ion step
    cudaStream_t ion_stream = nullptr;   // the ion step beside an inference, at the highest priority
    cudaEvent_t ion_event[2] = {nullptr, nullptr};
    cudaEvent_t net_event[2] = {nullptr, nullptr};
    double* stage_many = nullptr;        // staging of the batched transfers, stage_planes [i][j] planes
    // planned downloads (cth_fields_set_download_plan): each field is copied to its
    // host array on copy_stream as soon as the step's sweep that finalises it is done
    std::vector<std::string> plan_names;
    std::vector<double*> plan_host;
    std::vector<char> plan_queued;
    double* plan_stage = nullptr;        // one [i][j] staging plane per planned field
    int plan_cap = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
    bool copies_pending = false;
    // planned uploads (cth_fields_set_upload_plan), consumed by the next step: the
    // fields that the step reads first in its energy (rhoeps) or neutral (rhon,
    // rhom) sweep arrive while the sweeps before them run
    std::vector<std::string> up_names;
    std::vector<const double*> up_host;
    double* up_stage = nullptr;
    int up_cap = 0;
    cudaEvent_t up_ready[3] = {nullptr, nullptr, nullptr};  // fields read from the start / energy / neutrals
    bool up_wait[3] = {false, false, false};
    int stage_planes = 0;
    int warm_fields = 0;                 // field-valued solves start from the field's current values
    double warm_tol = 1.0;               // their guess threshold (relative residual)
    int net_misses = 0;                  // consecutive predictions that the device-side guess selection did not take
    long long net_runs = 0, net_wins = 0;  // predictions run / taken by the guess selection
    // streams / events of the concurrent ion solves
    cudaStream_t aux_stream[2] = {};
    cudaEvent_t aux_event[3] = {};
    std::map<std::string, double*> planes;
    unsigned char* flags = nullptr;  // device layout
    std::map<std::string, std::pair<double*, int>> tables;
    double* scal = nullptr;          // device scalars (reductions), CTH_FS_NSCAL doubles
    double* h_scal = nullptr;        // pinned host copy
    double* h_solve = nullptr;       // pinned status slots of enqueued MG solves, 8 doubles each
    double* part = nullptr;          // per-block partials, CTH_FS_NPART_PER_BLOCK per block
    int npart = 0;
};

// planned downloads: queue (on the copy stream, after the work queued on s) the
// planned fields that the step's stage `stage` finalises (1 ions, 2 potential,
// 3 electron density, 4 electron energy, 5 neutrals; 0: every field not yet
// queued); copies_wait makes s wait for copies still in flight
int plan_flush(cth_fields* fs, int stage, cudaStream_t s);
int copies_wait(cth_fields* fs, cudaStream_t s);
// planned uploads: issue them on the copy stream (the compute stream waits for the
// fields read from the start); upload_wait(fs, k, s) makes s wait for group k
// (1: read first by the energy sweep, 2: by the neutral sweep)
int plan_upload(cth_fields* fs, cudaStream_t s);
int upload_wait(cth_fields* fs, int group, cudaStream_t s);

namespace cth {

// side flags of a cell (1 = ordinary interior face on that side)
enum { F_BLX = 1, F_BRX = 2, F_BLR_WALL = 4, F_BLR_CEN = 8, F_BRR_WALL = 16, F_BRR_OPEN = 32, F_BRX_BIAS = 64,
       F_BRR_INLET = 128 };

// flag of cell (i, j); 0 outside the (ni+2) x (nj+2) index space
__device__ __forceinline__ unsigned flag_at(const unsigned char* __restrict__ f, int i, int j, int ni, int nj,
                                            int ld) {
    // the flag plane is never written by a kernel: read-only loads, free to move
    return (i >= 0 && i <= ni + 1 && j >= 0 && j <= nj + 1) ? __ldg(f + (size_t)j * ld + i) : 0u;
}

constexpr double kBoltz = 1.380649e-23;    // constants.hpp:5
constexpr double kE0f = 1.60217662e-19;    // constants.hpp:6
constexpr double kEps0f = 8.8541878128e-12;// constants.hpp:7

// uniform-step table lookups of miniFuncs.hpp:35-91.  In range the arithmetic is
// the reference's.  Outside it the reference indexes its vector with whatever
// (int)(x / dx) gives: below zero that reads before the table, and past INT_MAX
// iL + 1 wraps negative -- values a diverging run produces.  Here the index is
// formed only after the range test: a negative argument extrapolates from the
// first interval, a large one takes the reference's end-of-table branch, NaN
// stays NaN.
__device__ __forceinline__ int lookup_left(double t) { return t > 0.0 ? (int)t : 0; }

__device__ __forceinline__ double d_func_Te(const double* __restrict__ v, int n, double Te, double dTe) {
    const double t = Te / dTe;
    if (isnan(t)) return t;
    if (!(t < (double)(n - 2))) return v[n - 1];
    const int iL = lookup_left(t);
    const int iR = iL + 1;
    const double Te_L = iL * dTe;
    return (v[iR] - v[iL]) / (dTe + 1e-100) * (Te - Te_L) + v[iL];
}

__device__ __forceinline__ double d_func_dTe(const double* __restrict__ v, int n, double Te, double dTe) {
    const double t = Te / dTe;
    if (isnan(t)) return t;
    const int iL = (t < (double)(n - 2)) ? lookup_left(t) : n - 2;
    const int iR = iL + 1;
    return (v[iR] - v[iL]) / (iR * dTe - iL * dTe + 1e-100);
}

__device__ __forceinline__ double d_func_Ei(const double* __restrict__ v, int n, double Ei, double dEi,
                                            double massi) {
    const double t = Ei / dEi;
    if (isnan(t)) return t;
    if (t < (double)(n - 2)) {
        const int iL = lookup_left(t);
        const int iR = iL + 1;
        const double Ei_L = iL * dEi;
        return (v[iR] - v[iL]) / (dEi + 1e-100) * (Ei - Ei_L) + v[iL];
    }
    const double imax = n - 1;
    const double v_max = sqrt(imax * dEi / massi);
    const double v_tmp = sqrt(Ei / massi);
    return v[n - 1] / v_max * v_tmp;
}

struct Tab {
    const double* v;
    int n;
};

// Deterministic reduction of K per-thread values over a 2-D grid: every block
// writes its partial, the last block to finish combines the partials in block
// order and writes out[0..K).  Entry k is max-reduced when bit k of maxmask is
// set, summed otherwise.  Every thread of every block must call it.
template <int K>
__device__ void grid_reduce(const double (&s)[K], unsigned maxmask, double* __restrict__ part,
                            unsigned int* counter, double* __restrict__ out) {
    __shared__ double red[K][32];
    __shared__ bool am_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const bool mx = (maxmask >> k) & 1u;
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            v = mx ? fmax(v, u) : v + u;
        }
        if (lane == 0) red[k][wid] = v;
    }
    __syncthreads();
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const bool mx = (maxmask >> k) & 1u;
        double v = red[k][0];
        for (int w = 1; w < nw; w++) v = mx ? fmax(v, red[k][w]) : v + red[k][w];
        part[(size_t)k * nb + bid] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        am_last = (t == (unsigned int)(nb - 1));
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // the last block combines the partials with all its threads: thread t takes the
    // partials t, t + blockDim, ... in order (the K entries side by side, so their
    // L2 loads are in flight together), then a fixed warp / cross-warp tree
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
#pragma unroll 2
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
        double u[K];
#pragma unroll
        for (int k = 0; k < K; k++) u[k] = __ldcg(part + (size_t)k * nb + q);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = ((maxmask >> k) & 1u) ? fmax(acc[k], u[k]) : acc[k] + u[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        const bool mx = (maxmask >> k) & 1u;
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            v = mx ? fmax(v, u) : v + u;
        }
        if (lane == 0) red[k][wid] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const bool mx = (maxmask >> k) & 1u;
        double t = red[k][0];
        for (int w = 1; w < nw; w++) t = mx ? fmax(t, red[k][w]) : t + red[k][w];
        out[k] = t;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// calcRes statistics of one comparison (miniFuncs.hpp:292-376), as the pair (a, b):
// mode 0 (max|d|, 0), 1 (sum d^2/(o^2+eps), count), 2 (max|d|, max|o|), 3 (sum d^2, sum o^2)
__device__ __forceinline__ void res_stat(int mode, double nw, double od, double& a, double& b) {
    const double d = nw - od;
    if (mode == 0) { a = fabs(d); b = 0.0; }
    else if (mode == 1) { a = (d * d) / (od * od + 1e-100); b = 1.0; }
    else if (mode == 2) { a = fabs(d); b = fabs(od); }
    else { a = d * d; b = od * od; }
}

// first cell of this thread when a warp covers 32 * cells consecutive cells of a
// row and lane l owns the cells first + 32 k: every load and store instruction of
// the warp then touches one contiguous run
__device__ __forceinline__ int warp_strided_first(int cells) {
    return (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 * cells) + (threadIdx.x & 31);
}

// the same statistics accumulated over several cells of one thread (the modes'
// max or sum, as the grid reduction combines them afterwards)
__device__ __forceinline__ void res_acc(int mode, double nw, double od, double& a, double& b) {
    const double d = nw - od;
    if (mode == 0) { a = fmax(a, fabs(d)); }
    else if (mode == 1) { a += (d * d) / (od * od + 1e-100); b += 1.0; }
    else if (mode == 2) { a = fmax(a, fabs(d)); b = fmax(b, fabs(od)); }
    else { a += d * d; b += od * od; }
}

inline double finish_res(int mode, double a, double b) {
    if (mode == 0) return a;
    if (mode == 1) return sqrt(a / b);
    if (mode == 2) return a / b;
    return sqrt(a / b);
}

// maximum of v over the fluid cells (flags != 0), written to *out (fields.cu)
__global__ void k_max_flagged(const double* __restrict__ v, const unsigned char* __restrict__ flags, int ni,
                              int nj, int ld, double* __restrict__ part, unsigned int* counter,
                              double* __restrict__ out);

// ghost rules of the fluid store applied in order to a plane (fields.cu);
// which = 0: rhoe (rule mode 0 zeroes, 1 copies), 1: copy always
void restart_release(cth_fields* fs);
void apply_ghost_rules(cth_fields* fs, double* plane, int which, cudaStream_t s);

// named device planes of the store (created zeroed on first use), and tables
double* field_ptr(cth_fields* fs, const std::string& name);
Tab table(cth_fields* fs, const char* name, bool* ok);

}  // namespace cth
