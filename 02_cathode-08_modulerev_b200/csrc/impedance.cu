// impedance.cu — the reference's impedance test on the device (flag_impTest == 1,
// src/main.cpp:126-132): the coax of InitialModule::makeBoundary_impedanceTest
// (initialModule.hpp:1061-1330; r in [rmin, rmax] = [r1, r2], epsr = epsr_diele
// in the cells) and EmfieldModule::solve_Microwave_impedanceTest
// (emfieldModule.hpp:5528-6099) without plasma (rho = 0, :5531-5536): the Er
// equation on the r-faces i = 1..ni, j = 2..nj with the test's boundary codes --
// port excitation (code 7, :5616-5633) at the left end, first-order open
// (code 1, :5642-5657) at the right end, Gauss (code 2, :5675-5682 and
// :5706-5712) on the inner and outer conductors -- solved by the complex
// BiCGStab of helm.cu; then the ghosts of the code-7 and Gauss walls
// (:5788-5815), the port current and voltage at the reference plane x_ref = 0
// (:5835-5861), the wave amplitudes for Z0 and the rescale of the field and the
// excitation current to Pmw of forward power (:5880-5960, :6001-6036).
#include <cuda_runtime.h>

#include <cmath>

#include "grid.h"

namespace cth {

constexpr double kMu0I = 1.2566370614e-6;    // constants.hpp:8
constexpr double kEps0I = 8.8541878128e-12;  // constants.hpp:7

struct ImpArgs {
    cd *aP, *aE, *aW, *aN, *aS, *b;
    cd* E;
    const double* epsr;
    cth_impedance_params p;
    int ni, nj, ld;
};

__device__ __forceinline__ double r_at(const cth_impedance_params& p, int j) { return p.rmin + (j - 0.5) * p.dr; }

// one thread per Er face (i, j), i = 1..ni, j = 2..nj: interior coefficients, then the walls'
// surgery in the reference's loop order (left, right, lower, upper)
__global__ void k_imp_assemble(ImpArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 2;
    if (i > A.ni || j > A.nj) return;
    const cth_impedance_params& p = A.p;
    const double dx = p.dx, dr = p.dr, w = p.omegam;
    const size_t q = (size_t)j * A.ld + i;
    const double rj = r_at(p, j), rjm = r_at(p, j - 1), rjp = r_at(p, j + 1), rjmm = r_at(p, j - 2);
    const double rC = (rjm + rj) / 2.0, rR = (rj + rjp) / 2.0, rL = (rjmm + rjm) / 2.0;
    const double eps_t = (A.epsr[q] + A.epsr[q - A.ld]) / 2.0;
    cd aP(rC * (1.0 / rj + 1.0 / rjm) * dx * dx + 2.0 * dr * dr - kEps0I * eps_t * kMu0I * w * w * dx * dx * dr * dr,
          0.0);
    cd aE(dr * dr, 0.0), aW(dr * dr, 0.0), aN(rR / rj * dx * dx, 0.0), aS(rL / rjm * dx * dx, 0.0), b(0.0, 0.0);
    if (i == 1) {   // code 7: the incident wave of the port
        const double c0 = sqrt(1.0 / (kEps0I * eps_t * kMu0I));
        const cd deno(2.0 * c0 + 1e-100, w * dx);
        const cd R(2.0 * c0, -w * dx);
        const double r_t = (rj + rjm) / 2.0;
        const double Er_Fw = p.J1r_exc / r_t / log(p.r2 / p.r1) * 1e3;
        const cd S(0.0, 4.0 * w * dx * Er_Fw);
        aP = aP - aW * cdiv(R, deno);
        b = b + aW * cdiv(S, deno);
        aW = cd(0.0, 0.0);
    }
    if (i == A.ni) {   // code 1: first-order open end
        const double c0 = sqrt(1.0 / (kEps0I * eps_t * kMu0I));
        const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx) + 1e-100;
        const cd R((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx), -4.0 * c0 * w * dx);
        aP = aP - aE * cd(R.x / deno, R.y / deno);
        aE = cd(0.0, 0.0);
    }
    if (j == 2) {   // code 2 on the inner conductor
        const double rRg = (rj + rjm) / 2.0, rLg = (rjm + rjmm) / 2.0;
        aP = aP - aS * (rRg / rLg);
        aS = cd(0.0, 0.0);
    }
    if (j == A.nj) {   // code 2 on the outer conductor
        const double rRg = (rjp + rj) / 2.0, rLg = (rj + rjm) / 2.0;
        aP = aP - aN * (rLg / rRg);
        aN = cd(0.0, 0.0);
    }
    A.aP[q] = aP;
    A.aE[q] = aE;
    A.aW[q] = aW;
    A.aN[q] = aN;
    A.aS[q] = aS;
    A.b[q] = b;
}

// ghosts (:5788-5815) and the port (:5835-5861, :5880-5960); one block; the sums over the
// reference plane in the reference's order (j ascending) by one thread
__global__ void k_imp_port(ImpArgs A, double* __restrict__ out) {
    const cth_impedance_params& p = A.p;
    const int ld = A.ld, ni = A.ni, nj = A.nj;
    const double dx = p.dx, w = p.omegam;
    for (int j = 2 + threadIdx.x; j <= nj; j += blockDim.x) {   // left ghost (code 7)
        const size_t q = (size_t)j * ld + 1;
        const double eps_t = (A.epsr[q] + A.epsr[q - ld]) / 2.0;
        const double c0 = sqrt(1.0 / (kEps0I * eps_t * kMu0I));
        const cd deno(2.0 * c0 + 1e-100, w * dx);
        const cd R(2.0 * c0, -w * dx);
        const double r_t = (r_at(p, j) + r_at(p, j - 1)) / 2.0;
        const double Er_Fw = p.J1r_exc / r_t / log(p.r2 / p.r1) * 1e3;
        const cd S(0.0, 4.0 * w * dx * Er_Fw);
        A.E[q - 1] = cdiv(R, deno) * A.E[q] + cdiv(S, deno);
    }
    for (int i = 1 + threadIdx.x; i <= ni; i += blockDim.x) {   // Gauss ghosts with E1x = 0
        int j = 2;
        double rR = (r_at(p, j) + r_at(p, j - 1)) / 2.0, rL = (r_at(p, j - 1) + r_at(p, j - 2)) / 2.0;
        A.E[(size_t)(j - 1) * ld + i] = A.E[(size_t)j * ld + i] * (rR / rL);
        j = nj;
        rR = (r_at(p, j + 1) + r_at(p, j)) / 2.0;
        rL = (r_at(p, j) + r_at(p, j - 1)) / 2.0;
        A.E[(size_t)(j + 1) * ld + i] = A.E[(size_t)j * ld + i] * (rL / rR);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int i = int(0.0 / dx + 1.5);   // x_ref = 0
    cd I_ref(0.0, 0.0), coef(0.0, 0.0);
    int n = 0;
    for (int j = 2; j <= nj; j++) {
        const double r_t = (r_at(p, j) + r_at(p, j - 1)) / 2.0;
        const cd d = A.E[(size_t)j * ld + i] - A.E[(size_t)j * ld + i - 1];
        const cd H = cd(-d.y, d.x) * (1.0 / dx / (w * kMu0I));   // (dE / dx) / (w mu0) * i
        I_ref = I_ref + H * (2.0 * M_PI * r_t);
        coef = coef + (A.E[(size_t)j * ld + i] + A.E[(size_t)j * ld + i - 1]) * (0.5 * r_t);
        n++;
    }
    I_ref = I_ref * (1.0 / n);
    coef = coef * (1.0 / n);
    const cd V = coef * log(p.r2 / p.r1);
    const double s2 = 2.0 * sqrt(2.0 * p.Z0);
    const cd a2 = (V - I_ref * p.Z0) * (1.0 / s2);
    const cd b2 = (V + I_ref * p.Z0) * (1.0 / s2);
    const double P_fwd = b2.x * b2.x + b2.y * b2.y;
    const double ratio = p.Pmw / P_fwd;
    out[0] = V.x; out[1] = V.y; out[2] = I_ref.x; out[3] = I_ref.y;
    out[4] = P_fwd; out[5] = a2.x * a2.x + a2.y * a2.y; out[6] = ratio; out[7] = sqrt(ratio);
}

__global__ void k_imp_scale(cd* __restrict__ E, const double* __restrict__ out, size_t n) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) E[k] = E[k] * out[7];
}

}  // namespace cth

using namespace cth;

extern "C" int cth_mw_impedance_test(cth_grid* g, const double* epsr, const cth_impedance_params* prm, int maxITR,
                                     double tol, double* E1r, void* stream, cth_impedance_result* res) {
    if (!g || !epsr || !prm || !E1r || maxITR < 0 || prm->dx <= 0.0 || prm->dr <= 0.0 || prm->r1 <= 0.0 ||
        prm->r2 <= prm->r1 || prm->Z0 <= 0.0 || g->nj < 2) {
        set_error("cth_mw_impedance_test: invalid arguments");
        return CTH_ERR_ARG;
    }
    if (g->n_bl != 1 || g->ibl[0] != 1 || g->ibl[1] != g->ni || g->jbl[0] != 2 || g->jbl[1] != g->nj) {
        set_error("cth_mw_impedance_test: the grid's single block must be the Er faces [1, ni] x [2, nj]");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    C5Work& c = g->c5;
    if (!c.cstage) {
        CTH_CUDA(cudaMalloc(&c.cstage, 7 * g->plane * 2 * sizeof(double)));
        CTH_CUDA(zero_fill(c.cstage, 7 * g->plane * 2 * sizeof(double)));
        CTH_CUDA(cudaMalloc(&c.cstage_ij, (size_t)(g->ni + 2) * (g->nj + 2) * 2 * sizeof(double)));
    }
    const size_t pl = g->plane * 2;
    double* base = c.cstage;
    ImpArgs A{};
    A.aP = reinterpret_cast<cd*>(base);
    A.aE = reinterpret_cast<cd*>(base + pl);
    A.aW = reinterpret_cast<cd*>(base + 2 * pl);
    A.aN = reinterpret_cast<cd*>(base + 3 * pl);
    A.aS = reinterpret_cast<cd*>(base + 4 * pl);
    A.b = reinterpret_cast<cd*>(base + 5 * pl);
    A.E = reinterpret_cast<cd*>(E1r);
    A.epsr = epsr;
    A.p = *prm;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 127) / 128, g->nj - 1);
    k_imp_assemble<<<grd, blk, 0, s>>>(A);
    g->launches++;
    CTH_CUDA(cudaGetLastError());
    cth_status st{};
    const int rc = c5_solve_dev(g, base, base + pl, base + 2 * pl, base + 3 * pl, base + 4 * pl, base + 5 * pl,
                                maxITR, tol, E1r, s, &st);
    if (rc < 0) return rc;
    double* out = base + 6 * pl;   // the seventh staging plane holds the port results
    k_imp_port<<<1, 256, 0, s>>>(A, out);
    const size_t n = (size_t)(g->nj + 2) * g->ld;
    k_imp_scale<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A.E, out, n);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    double h[8];
    CTH_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (res) {
        res->V[0] = h[0]; res->V[1] = h[1]; res->I[0] = h[2]; res->I[1] = h[3];
        res->P_fwd = h[4]; res->P_ref = h[5]; res->ratio = h[6]; res->J1r_exc_factor = h[7];
        res->solve = st;
    }
    if (!std::isfinite(h[6])) {
        set_error("cth_mw_impedance_test: the forward power is zero or not finite");
        return CTH_NONFINITE;
    }
    return rc;
}
