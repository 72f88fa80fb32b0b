// diag.cu — the microwave diagnostics of OutputModule::output_phase
// (outputModule.hpp:38-184) on the device: the representative field
// Emag_rep = sqrt(mean over the cells i = 1..ni, j = 1..nj of |Ex|^2 + |Er|^2 +
// |Ephi|^2 at the cell centre) (:43-60), and per cell of the grid's blocks
// (jdgBnd_Ep) the normalised divergences of E and J and of the total current
// (:97-105):
//   divE  = (div E) dx / Emag_rep
//   divJ  = (div J) dx / (Emag_rep w eps0)
//   divEJ = (divJ + i w eps0 divE) dx / (Emag_rep w eps0)  -- of the two normalised
//           values, as the reference writes it
// with div F = (r_{j+1/2} F_r[j+1] - r_{j-1/2} F_r[j]) / (dr r_j) + (F_x[i+1] - F_x[i]) / dx;
// zero on cells outside the blocks.  The phase factor of the output does not
// enter these three columns.
#include <cuda_runtime.h>

#include <cmath>

#include "grid.h"

namespace cth {

constexpr double kEps0D = 8.8541878128e-12;  // constants.hpp:7

struct DivArgs {
    const cd *Ex, *Er, *Ep, *Jx, *Jr, *Jp;
    cd *divE, *divJ, *divEJ;
    const unsigned char* mask;
    double dx, dr, rmin, w;
    int ni, nj, ld;
};

__device__ __forceinline__ double rad(const DivArgs& A, int j) { return A.rmin + (j - 0.5) * A.dr; }

// one block per row j = 1..nj: the row's sum of |E|^2 at the cell centres, i ascending
__global__ void k_div_rows(DivArgs A, double* __restrict__ part) {
    const int j = blockIdx.x + 1;
    __shared__ double s[256];
    double acc = 0.0;
    const double rj = rad(A, j), rL = (rad(A, j - 1) + rj) / 2.0, rR = (rad(A, j + 1) + rj) / 2.0;
    for (int i = 1 + threadIdx.x; i <= A.ni; i += blockDim.x) {
        const size_t q = (size_t)j * A.ld + i;
        const cd ex = (A.Ex[q] + A.Ex[q + 1]) * 0.5;
        const cd er = (A.Er[q + A.ld] * rR + A.Er[q] * rL) * (1.0 / (2.0 * rj));
        acc += abs2(ex) + abs2(er) + abs2(A.Ep[q]);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[j] = s[0];
}

__global__ void k_div_rep(DivArgs A, double* __restrict__ part) {
    if (threadIdx.x != 0) return;
    double t = 0.0;
    for (int j = 1; j <= A.nj; j++) t += part[j];
    part[0] = sqrt(t / ((double)A.ni * A.nj));
}

__global__ void k_div_cells(DivArgs A, const double* __restrict__ part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t q = (size_t)j * A.ld + i;
    if (i < 1 || i > A.ni || j < 1 || j > A.nj || !A.mask[q]) {
        A.divE[q] = cd();
        A.divJ[q] = cd();
        A.divEJ[q] = cd();
        return;
    }
    const double rep = part[0];
    const double rj = rad(A, j), rL = (rad(A, j - 1) + rj) / 2.0, rR = (rad(A, j + 1) + rj) / 2.0;
    const cd dE = (A.Er[q + A.ld] * rR - A.Er[q] * rL) * (1.0 / (A.dr * rj)) + (A.Ex[q + 1] - A.Ex[q]) * (1.0 / A.dx);
    const cd dJ = (A.Jr[q + A.ld] * rR - A.Jr[q] * rL) * (1.0 / (A.dr * rj)) + (A.Jx[q + 1] - A.Jx[q]) * (1.0 / A.dx);
    const cd divE = dE * (A.dx / rep);
    const cd divJ = dJ * (A.dx / (rep * A.w * kEps0D));
    const cd divEJ = (divJ + cd(0.0, A.w * kEps0D) * divE) * (A.dx / (rep * A.w * kEps0D));
    A.divE[q] = divE;
    A.divJ[q] = divJ;
    A.divEJ[q] = divEJ;
}

}  // namespace cth

using namespace cth;

extern "C" int cth_mw_divergence(cth_grid* g, const double* E1x, const double* E1r, const double* E1p,
                                 const double* J1x, const double* J1r, const double* J1p, double dx, double dr,
                                 double rmin, double omegam, double* divE, double* divJ, double* divEJ,
                                 double* Emag_rep, void* stream) {
    if (!g || !E1x || !E1r || !E1p || !J1x || !J1r || !J1p || !divE || !divJ || !divEJ || dx <= 0.0 || dr <= 0.0 ||
        omegam <= 0.0) {
        set_error("cth_mw_divergence: invalid arguments");
        return CTH_ERR_ARG;
    }
    if (g->ws.npart < g->nj + 2) {
        set_error("cth_mw_divergence: reduction scratch too small");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DivArgs A{};
    A.Ex = reinterpret_cast<const cd*>(E1x);
    A.Er = reinterpret_cast<const cd*>(E1r);
    A.Ep = reinterpret_cast<const cd*>(E1p);
    A.Jx = reinterpret_cast<const cd*>(J1x);
    A.Jr = reinterpret_cast<const cd*>(J1r);
    A.Jp = reinterpret_cast<const cd*>(J1p);
    A.divE = reinterpret_cast<cd*>(divE);
    A.divJ = reinterpret_cast<cd*>(divJ);
    A.divEJ = reinterpret_cast<cd*>(divEJ);
    A.mask = g->mask_full;
    A.dx = dx;
    A.dr = dr;
    A.rmin = rmin;
    A.w = omegam;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    double* part = g->ws.part;
    k_div_rows<<<g->nj, 256, 0, s>>>(A, part);
    k_div_rep<<<1, 32, 0, s>>>(A, part);
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    k_div_cells<<<grd, blk, 0, s>>>(A, part);
    g->launches += 3;
    CTH_CUDA(cudaGetLastError());
    double rep = 0.0;
    CTH_CUDA(cudaMemcpyAsync(&rep, part, sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (Emag_rep) *Emag_rep = rep;
    return std::isfinite(rep) && rep > 0.0 ? CTH_OK : CTH_NONFINITE;
}
