// noalloc.cu — residual of the box-union system for callers that cannot
// allocate device memory.
//
// Who needs this: code that may not call cudaMalloc at the moment it wants a
// residual norm.  Examples are a host program that hands all device memory to
// its own pool allocator up front and forbids libraries from allocating
// afterwards, and a real-time loop that cannot afford the implicit
// synchronisation an allocation may cause.  Such callers cannot create a
// cth_grid (its constructor allocates the mask, the multigrid hierarchy and
// the reduction buffers), so this entry point takes the block table directly
// and keeps all of its scratch in one file-scope device array instead.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, once per device, with that device current); make that
// first call before any stream capture.  Every call then waits for its stream:
// it copies the two sums to the host and synchronises, and returns with the
// norms on the host.
//
// Scratch: g_noalloc_scratch, CTH_NOALLOC_SCRATCH_BYTES = 8 MiB per GPU that
// loads the library, held until the process exits.  The first 256 KiB hold
// the per-block partial sums (at most 16384 blocks per half) and the two
// final sums; the rest holds the grid-cell mask of the ghost-padded plane,
// so (nj+2) * ld may not exceed CTH_NOALLOC_MAX_PLANE cells.
//
// Every call on a device shares that array and the array keeps the contents
// of the last call.  Each call rebuilds the whole mask region it uses and
// every partial-sum slot it reads, so no stale value reaches a result; but two
// calls whose work overlaps on the GPU (different streams, or different host
// threads without ordering) race on the array and may return wrong norms.
#include <cuda_runtime.h>

#include <mutex>

#include "grid.h"

namespace cth {

// kernels shared with the grid-based residual (sor.cu)
__global__ void k_residual(const double* __restrict__ aP, const double* __restrict__ aE,
                           const double* __restrict__ aW, const double* __restrict__ aN,
                           const double* __restrict__ aS, const double* __restrict__ b,
                           const unsigned char* __restrict__ mask, const double* __restrict__ x,
                           double* __restrict__ r, int ni, int nj, int ld,
                           double* __restrict__ part);
__global__ void k_sum2(const double* __restrict__ part, int n, double* __restrict__ out);

}  // namespace cth

static constexpr size_t kPartBytes = 256 * 1024;
static constexpr int kMaxBlocks = 64;  // block-table entries passed by value

static __device__ __align__(256) unsigned char g_noalloc_scratch[CTH_NOALLOC_SCRATCH_BYTES];

struct BlockTable {
    int n;
    int i0[kMaxBlocks], i1[kMaxBlocks], j0[kMaxBlocks], j1[kMaxBlocks];
};

// mask of the ghost-padded plane (j*ld + i), every byte of the plane written
__global__ void k_noalloc_mask(unsigned char* __restrict__ mask, int ni, int nj, int ld,
                               BlockTable bt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= ld || j > nj + 1) return;
    unsigned char m = 0;
    if (i <= ni + 1)
        for (int k = 0; k < bt.n; k++)
            if (i >= bt.i0[k] && i <= bt.i1[k] && j >= bt.j0[k] && j <= bt.j1[k]) m = 1;
    mask[(size_t)j * ld + i] = m;
}

// device address of g_noalloc_scratch, looked up once per device
static std::mutex g_mu;
static void* g_ptr[64] = {nullptr};

static int scratch_for_current_device(unsigned char** out) {
    int dev = -1;
    CTH_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        cth::set_error("cth_residual_noalloc: device ordinal out of range");
        return CTH_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ptr[dev]) {
        void* p = nullptr;
        // host code must not use the symbol itself as an address: ask the runtime
        CTH_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_ptr[dev]);
    return CTH_OK;
}

extern "C" int cth_residual_noalloc(int ni, int nj, int ld, const int* i_bl, const int* j_bl, int n_bl,
                                    const double* aP, const double* aE, const double* aW,
                                    const double* aN, const double* aS, const double* b,
                                    const double* x, double* r, double* rnorm, double* bnorm,
                                    void* stream) {
    if (ni < 1 || nj < 1 || ld < ni + 2 || !i_bl || !j_bl || n_bl < 1 || !aP || !aE || !aW || !aN ||
        !aS || !b || !x) {
        cth::set_error("cth_residual_noalloc: invalid arguments");
        return CTH_ERR_ARG;
    }
    if (n_bl > kMaxBlocks) {
        cth::set_error("cth_residual_noalloc: more than 64 blocks");
        return CTH_ERR_ARG;
    }
    const size_t plane = (size_t)(nj + 2) * (size_t)ld;
    if (plane > (size_t)CTH_NOALLOC_MAX_PLANE) {
        cth::set_error("cth_residual_noalloc: (nj+2)*ld exceeds CTH_NOALLOC_MAX_PLANE cells of the "
                       "static scratch array");
        return CTH_ERR_ARG;
    }
    dim3 blk(256), grd((ni + 2 + 255) / 256, nj + 2);
    const size_t nb = (size_t)grd.x * grd.y;
    if ((2 * nb + 2) * sizeof(double) > kPartBytes) {
        cth::set_error("cth_residual_noalloc: grid too large for the partial-sum region of the static "
                       "scratch array");
        return CTH_ERR_ARG;
    }
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc != CTH_OK) return rc;
    double* part = reinterpret_cast<double*>(base);
    double* sums = part + 2 * nb;
    unsigned char* mask = base + kPartBytes;
    BlockTable bt{};
    bt.n = n_bl;
    for (int k = 0; k < n_bl; k++) {
        bt.i0[k] = i_bl[2 * k];
        bt.i1[k] = i_bl[2 * k + 1];
        bt.j0[k] = j_bl[2 * k];
        bt.j1[k] = j_bl[2 * k + 1];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 mgrd((ld + 255) / 256, nj + 2);
    k_noalloc_mask<<<mgrd, blk, 0, s>>>(mask, ni, nj, ld, bt);
    cth::k_residual<<<grd, blk, 0, s>>>(aP, aE, aW, aN, aS, b, mask, x, r, ni, nj, ld, part);
    cth::k_sum2<<<1, 1024, 0, s>>>(part, (int)nb, sums);
    CTH_CUDA(cudaGetLastError());
    double h[2] = {0.0, 0.0};
    CTH_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (rnorm) *rnorm = sqrt(h[0]);
    if (bnorm) *bnorm = sqrt(h[1]);
    return CTH_OK;
}
