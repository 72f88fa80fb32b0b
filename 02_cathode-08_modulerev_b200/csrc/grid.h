// grid.h — internal state of a cth_grid (not part of the C ABI).
//
// HBM layout
//   * "device layout": ghost-padded (ni+2) x (nj+2) planes, r-major:
//     element (i,j) at j*ld + i, ld = round_up(ni+2, 32).  z-lines (fixed j)
//     are contiguous, which is what the z-line smoothers read.
//   * "level layout": the multigrid levels cover the bounding box of the grid
//     cells, [i0..i1] x [j0..j1].  Level l has nrow[l] rows (semicoarsened in
//     r: row J of level l+1 is row 2J of level l) and ncol = i1-i0+1 columns,
//     element (c, r) at r*ldl + c, ldl = round_up(ncol, 32).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/cathode_b200.h"

#include <cuda_runtime.h>

namespace cth {

// Zero freshly allocated device memory before any stream can use it.  cudaMemset
// on device memory returns before the fill is done and runs on the legacy
// default stream, which does not order work on non-blocking streams (the batched
// instances' streams): wait for it here, once per allocation.
inline cudaError_t zero_fill(void* p, size_t bytes) {
    cudaError_t e = cudaMemset(p, 0, bytes);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}

// complex double of the frequency-domain solves; interleaved (re, im) in memory
struct cd {
    double x, y;
    __host__ __device__ cd() : x(0.0), y(0.0) {}
    __host__ __device__ cd(double r) : x(r), y(0.0) {}
    __host__ __device__ cd(double r, double i) : x(r), y(i) {}
};
__host__ __device__ inline cd operator+(cd a, cd b) { return cd(a.x + b.x, a.y + b.y); }
__host__ __device__ inline cd operator-(cd a, cd b) { return cd(a.x - b.x, a.y - b.y); }
__host__ __device__ inline cd operator-(cd a) { return cd(-a.x, -a.y); }
__host__ __device__ inline cd operator*(cd a, cd b) { return cd(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ inline cd& operator-=(cd& a, cd b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ inline bool operator==(cd a, cd b) { return a.x == b.x && a.y == b.y; }
__host__ __device__ inline bool operator!=(cd a, cd b) { return !(a == b); }
__host__ __device__ inline cd conj(cd a) { return cd(a.x, -a.y); }
__host__ __device__ inline double abs2(cd a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ inline cd cdiv(cd a, cd b) {
    const double s = 1.0 / (b.x * b.x + b.y * b.y);
    return cd((a.x * b.x + a.y * b.y) * s, (a.y * b.x - a.x * b.y) * s);
}

// complex float: the FP32 preconditioner hierarchy of the complex solves (mixed precision);
// interleaved (re, im) in memory
struct cf {
    float x, y;
    __host__ __device__ cf() : x(0.f), y(0.f) {}
    __host__ __device__ cf(float r) : x(r), y(0.f) {}
    __host__ __device__ cf(float r, float i) : x(r), y(i) {}
    __host__ __device__ explicit cf(cd a) : x((float)a.x), y((float)a.y) {}
};
__host__ __device__ inline cf operator+(cf a, cf b) { return cf(a.x + b.x, a.y + b.y); }
__host__ __device__ inline cf operator-(cf a, cf b) { return cf(a.x - b.x, a.y - b.y); }
__host__ __device__ inline cf operator-(cf a) { return cf(-a.x, -a.y); }
__host__ __device__ inline cf operator*(cf a, cf b) { return cf(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline cf& operator+=(cf& a, cf b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ inline cf& operator-=(cf& a, cf b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ inline bool operator==(cf a, cf b) { return a.x == b.x && a.y == b.y; }
__host__ __device__ inline bool operator!=(cf a, cf b) { return !(a == b); }
__host__ __device__ inline cf conj(cf a) { return cf(a.x, -a.y); }
__host__ __device__ inline float abs2(cf a) { return a.x * a.x + a.y * a.y; }

// stencil slots: level 0 stores the first 5, coarse levels all 9.
// Convention of the reference: (A x)_P = a[P] x_P - sum_k a[k] x_k.
enum Slot { P = 0, W = 1, E = 2, S = 3, N = 4, SW = 5, SE = 6, NW = 7, NE = 8 };

template <typename T>
struct Hierarchy {
    bool allocated = false;
    std::vector<T*> a;   // per level: npt planes of nrow*ldl
    std::vector<T*> x;   // per level
    std::vector<T*> b;   // per level
    std::vector<T*> wS;  // per level (F rows used): weight toward the C row below
    std::vector<T*> wN;  // per level: weight toward the C row above
    std::vector<T*> fac; // per level: factorised z-line operators (real precisions)
};

// per-kernel-class timing with CUDA events on the launching stream
enum ProfClass { PROF_RELAX0 = 0, PROF_UPDATE = 1, PROF_RESTRICT0 = 2, PROF_SETUP = 3, PROF_RELAXC = 4, PROF_NCLASS = 5 };

struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> ev;      // pairs (start, stop)
    std::vector<int> cls;             // class of each pair
    std::vector<double> bytes;        // algorithmic bytes of each pair
    size_t used = 0;
    double ms[PROF_NCLASS] = {};
    long long n[PROF_NCLASS] = {};
    double nbytes[PROF_NCLASS] = {};
};

// caller arguments of one solve, read by the kernels from device memory so
// that a captured graph stays valid for any caller arrays
struct SolveArgs {
    const double* aP;
    const double* aE;
    const double* aW;
    const double* aN;
    const double* aS;
    const double* b;
    double* solution;
    double tol;
    int maxit;
    int pad;
    const double* x0;   // initial guess (null: zero, the reference's start)
    const double* x0b;  // second candidate (null: none); the better of the two is used
    double guess_tol;   // a guess is used when ||b - A x0|| <= guess_tol ||b|| (guess_tol <= 10)
    double reuse_tol;   // hierarchy slots: largest row-relative operator change that keeps the hierarchy
};

// device status words of a solve (double array).  ST_GUESS: 0 no guess;
// 1 + r0 first candidate used; 100 + r0 second candidate used; -(1 + r0)
// guesses rejected (r0 = relative residual of the used / the better guess)
// ST_ASCALE, ST_XSCALE (device only): the powers of two that the working-precision
// cycle's operator and right-hand side are scaled by (see k_prep0 / k_update).
// ST_SETUP: 1 when this solve builds its hierarchy (before its cycles or after a
// retry), 0 while it runs on a kept one.  ST_RETRY: 1 when a cycle on a kept
// hierarchy reduced the residual by less than kRetryRate and the solve rebuilt
// the hierarchy from its operator and went on from the current iterate.
enum StatWord { ST_RR = 0, ST_RELRES = 1, ST_BB = 2, ST_NONFINITE = 3, ST_ITER = 4, ST_CONV = 5, ST_KEEP = 6,
                ST_GUESS = 7, ST_ASCALE = 8, ST_XSCALE = 9, ST_SETUP = 10, ST_RETRY = 11 };
constexpr double kRetryRate = 0.5;

// Hierarchy slots.  Hierarchy 0 serves the solves that build their hierarchy
// every time (the reference's SMG set-up per solve); hierarchies 1..kSlots
// belong to the slots 0..kSlots-1 of the solves that keep theirs while the
// operator stays within a tolerance of the one it was built from.  Per slot and
// precision the device keeps kSlotWords words (SlotWord).
constexpr int kSlots = 15;
constexpr int kHier = kSlots + 1;
constexpr int kSlotWords = 8;
// hierarchy slots of the time step's equations: one per operator that recurs
// step after step (the predictor and the corrector of a predictor-corrector
// iteration solve with the same operator and share a slot)
enum EqSlot { SLOT_ION_MOMENTUM = 0, SLOT_ION_CONTINUITY = 1, SLOT_PHI = 2, SLOT_RHOE = 3, SLOT_EPS = 4,
              SLOT_RHON = 5, SLOT_RHOM = 6 };
// doubles between the pinned host status copies of concurrent solves (the copy
// holds the words ST_RR..ST_RETRY)
constexpr int kStatStride = 16;
enum SlotWord { SW_VALID = 0, SW_ASCALE = 1, SW_SETUPS = 2, SW_REUSES = 3, SW_CHANGE = 4, SW_LASTCONV = 5,
                SW_LASTITER = 6, SW_RETRIES = 7 };

struct SolveGraph {
    bool valid = false;
    int nu1 = 0, nu2 = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int n_pre = 0, n_body = 0, n_post = 0;  // kernels per section
    int n_setup = 0;                        // kernels of the conditional set-up (hierarchy slots)
};

// complex 5-point solver workspace (level-0 layout, 14 complex planes)
struct C5Work {
    void* buf = nullptr;      // 9 planes of complex doubles (Krylov vectors)
    double* sc = nullptr;     // recurrence scalars
    double* part = nullptr;   // reduction partials
    int npart = 0;
    double* cstage = nullptr;     // host-API staging: 7 complex planes in device layout
    double* cstage_ij = nullptr;  // one complex [i][j] array
};

struct Workspace {
    double* x64[2] = {nullptr, nullptr};  // level-0 layout accumulated solution
    double* part = nullptr;               // per-block partial sums
    int npart = 0;
    double* stat = nullptr;               // device status words
    double* h_stat = nullptr;             // pinned mirror
    // host-API staging: 6 input planes + solution in device layout, one [i][j] buffer
    double* stage = nullptr;
    double* stage_ij = nullptr;
    double* h_pinned = nullptr;           // pinned [i][j] buffer for transfers
    SolveArgs* d_args = nullptr;
    SolveArgs* h_args = nullptr;          // pinned
    unsigned int* counter = nullptr;      // last-block reduction counter
    // 2 precisions x kSlots x kSlotWords slot words, then one word (as a 64-bit
    // integer) for the largest operator change of the running solve
    double* slotstat = nullptr;
};

}  // namespace cth

struct cth_grid {
    int ni = 0, nj = 0, n_bl = 0;
    std::vector<int> ibl, jbl;
    int device = 0;
    int ld = 0;          // device layout leading dimension
    size_t plane = 0;    // (nj+2)*ld
    int i0 = 0, i1 = -1, j0 = 0, j1 = -1;
    size_t qref = 0;  // a grid cell (the first block's first cell) in the caller's layout: operator scale
    int ncol = 0, ldl = 0;
    int nlev = 0;
    std::vector<int> nrow;
    int nu1 = 1, nu2 = 1;
    int bd = 32, ept = 1;      // line solve: threads per z-line / cells per thread (chunk)
    unsigned char* mask_full = nullptr;          // device layout
    std::vector<unsigned char*> mask;            // per level, level layout
    cth::Hierarchy<float> h32[cth::kHier];   // [0]: rebuilt every solve; [1 + s]: slot s
    cth::Hierarchy<double> h64[cth::kHier];
    int cur = 0;               // hierarchy the host driver is working on
    double reuse_tol = 0.0;    // > 0: solves given a slot keep their hierarchy (see kSlots)
    int api_slot = -1;         // slot of the solves entered through the C ABI (-1: none)
    cth::Workspace ws;
    cudaStream_t stream = nullptr;
    long long launches = 0;    // kernels launched by this grid since creation
    cth::Profiler prof;
    cth::SolveGraph graphs[2][cth::kHier]; // per precision (CTH_PREC_FP64, CTH_PREC_MIXED) and hierarchy
    cth::C5Work c5;
    cth::Hierarchy<cth::cd> hc;    // complex hierarchy (preconditioner of the complex solves)
    cth::Hierarchy<cth::cf> hcf;   // its FP32 twin (mixed-precision preconditioner)
    cth::SolveGraph c5graph;
    cudaStream_t cap[2] = {nullptr, nullptr};  // capture streams
    bool use_graphs = true;
    bool pdl = true;  // relaxations launched with programmatic dependent launch
    bool tail = false; // coarse levels of at most 16 rows run as one cluster launch (off: measured slower)
    int bnd = 256;       // launch bounds of the line kernels: 256, 512 or 1024 (>= bd)
    int tail_types = 0;  // bit per precision (float, double, complex) whose tail kernel fits
    cudaStream_t pending_stream = nullptr;  // stream of the last enqueued graph solve
};

namespace cth {
void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
int ensure_hierarchy_f32(cth_grid* g);
int ensure_hierarchy_f64(cth_grid* g);
int ensure_staging(cth_grid* g);
int smg_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, int maxITR,
                  double error_cnv, int precision, double* solution, cudaStream_t s,
                  cth_status* st);
// split form of smg_solve_dev: enqueue on s with the status copied to h_dst (pinned
// host, 8 doubles; null = the grid's own), then either solve_finish (synchronise and
// read the grid's copy) or, after the caller's own synchronisation, solve_parse(h_dst)
// slot: hierarchy slot of the equation (0..kSlots-1; used when g->reuse_tol > 0),
// -1: the C ABI's slot (g->api_slot), i.e. none unless the caller chose one.
int smg_solve_launch(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                     const double* aS, const double* b, int maxITR, double error_cnv, int precision,
                     double* solution, cudaStream_t s, int* pending, double* h_dst,
                     const double* x0 = nullptr, double guess_tol = 0.0, const double* x0b = nullptr,
                     int slot = -1);
int solve_finish(cth_grid* g, int pending, cth_status* st);
int time_relax(cth_grid* g, int precision, int level, int reps, double* us, double* bytes);
int time_cycle(cth_grid* g, int precision, int reps, int with_update, double* us);
int solve_parse(cth_grid* g, int pending, const double* h, cth_status* st);
int sor_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, double alpha,
                  int maxITR, double error_cnv, double* solution, cudaStream_t s,
                  cth_status* st);
int residual_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                 const double* aN, const double* aS, const double* b, const double* x,
                 double* r, double* rnorm, double* bnorm, cudaStream_t s);
int to_device_layout(cth_grid* g, const double* src_ij_dev, double* dst, cudaStream_t s);
// profiling: mark() before a launch of class c, done() after it; collect() after a sync
int prof_mark(cth_grid* g, int c, double bytes, cudaStream_t s);
void prof_done(cth_grid* g, int slot, cudaStream_t s);
void prof_collect(cth_grid* g);
int from_device_layout(cth_grid* g, const double* src, double* dst_ij_dev, cudaStream_t s);
int c5_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                 const double* aS, const double* b, int maxit, double tol, double* solution, cudaStream_t s,
                 cth_status* st);
int c5_configure(cth_grid* g);
int mw_er_assemble_dev(cth_grid* g, const double* ne, const double* nu, const double* epsr,
                       const cth_mw_params* prm, double* aP, double* aE, double* aW, double* aN, double* aS,
                       double* b, cudaStream_t s);
}  // namespace cth

#define CTH_CUDA(call)                                        \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return cth::cuda_fail(_e, #call); \
    } while (0)
