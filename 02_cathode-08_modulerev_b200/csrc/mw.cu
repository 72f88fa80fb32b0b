// mw.cu — assembly of the microwave Er system on the device.
//
// Er equation of EmfieldModule::solve_Microwave (include/emfieldModule.hpp:2350-2395)
// with B = 0: the conductivity tensor reduces to sigma_rr = n e^2 / (m (nu + i w))
// and every Hall coupling to Ex and Ephi vanishes (those terms carry the Hall
// factors), so Er is an independent complex 5-point system.  Per r-face
// (i, j-1/2), i = 1..ni, j = 2..nj, with face averages of n, nu and epsr:
//   aP = r_f (1/r_j + 1/r_{j-1}) dx^2 + 2 dr^2 - eps0 epsr mu0 w^2 dx^2 dr^2
//        + i w mu0 sigma_rr dx^2 dr^2,
//   aE = aW = dr^2, aN = r_{j+1/2}/r_j dx^2, aS = r_{j-3/2}/r_{j-1} dx^2.
// Boundary codes of the impedance test applied to the r-z rectangle:
//   z = 0 faces: port excitation (code 7, :5616-5633) where r1 <= r_f <= r2,
//                first-order open (code 1, :5602-5612) elsewhere;
//   z = L faces: open (code 1, :5642-5657);
//   r = R:       Gauss (code 2, :5706-5712), its coupling to Ex dropped;
//   axis face:   Er = 0 (not an unknown; the j = 2 south coupling is dropped).
#include <cuda_runtime.h>

#include <cmath>

#include "grid.h"

namespace cth {

constexpr double kE0 = 1.60217662e-19;     // constants.hpp:6
constexpr double kEPS0 = 8.8541878128e-12; // constants.hpp:7
constexpr double kMU0 = 1.2566370614e-6;   // constants.hpp:8

__global__ void k_mw_er_assemble(const double* __restrict__ ne, const double* __restrict__ nu,
                                 const double* __restrict__ epsr, cth_mw_params prm, int ni, int nj, int ld,
                                 cd* __restrict__ aP, cd* __restrict__ aE, cd* __restrict__ aW,
                                 cd* __restrict__ aN, cd* __restrict__ aS, cd* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > ni + 1) return;
    const size_t p = (size_t)j * ld + i;
    cd vP, vE, vW, vN, vS, vb;
    if (i >= 1 && i <= ni && j >= 2 && j <= nj) {
        const double dx = prm.dx, dr = prm.dr, w = prm.omegam;
        const double rj = prm.rmin + (j - 0.5) * dr, rjm = prm.rmin + (j - 1.5) * dr;
        const double rjp = prm.rmin + (j + 0.5) * dr, rjmm = prm.rmin + (j - 2.5) * dr;
        const double r_f = 0.5 * (rjm + rj);
        const double rR = 0.5 * (rj + rjp);
        const double rL = 0.5 * (rjmm + rjm);
        const double nu_t = 0.5 * (nu[p] + nu[p - ld]);
        const double rho_t = 0.5 * (ne[p] + ne[p - ld]);
        const double eps_t = 0.5 * (epsr[p] + epsr[p - ld]);
        // coef = rho e^2 / (m nu_c + EPS) / (1 + EPS), nu_c = nu + i w, EPS = 1e-100 (1 + i)
        const cd den(prm.masse * nu_t + 1e-100, prm.masse * w + 1e-100);
        const cd coef = cdiv(cd(rho_t * kE0 * kE0), den * cd(1.0 + 1e-100, 1e-100));
        const double g2 = dx * dx * dr * dr;
        const cd iwm(0.0, w * kMU0);
        vP = cd(r_f * (1.0 / rj + 1.0 / rjm) * dx * dx + 2.0 * dr * dr - kEPS0 * eps_t * kMU0 * w * w * g2) +
             iwm * coef * cd(g2);
        vE = cd(dr * dr);
        vW = cd(dr * dr);
        vN = cd(rR / rj * dx * dx);
        vS = cd(rL / rjm * dx * dx);
        const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
        if (i == 1) {
            if (r_f >= prm.r1 && r_f <= prm.r2) {
                const cd deno(2.0 * c0 + 1e-100, w * dx);
                const cd R(2.0 * c0, -w * dx);
                const double Er_Fw = prm.J1r_exc / r_f / log(prm.r2 / prm.r1) * 1e3;
                const cd S = cd(0.0, 4.0 * w * dx) * cd(Er_Fw);
                vP = vP - vW * cdiv(R, deno);
                vb = vb + vW * cdiv(S, deno);
            } else {
                const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx) + 1e-100;
                const cd R((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx), -4.0 * c0 * w * dx);
                vP = vP - vW * cd(R.x / deno, R.y / deno);
            }
            vW = cd();
        }
        if (i == ni) {
            const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx) + 1e-100;
            const cd R((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx), -4.0 * c0 * w * dx);
            vP = vP - vE * cd(R.x / deno, R.y / deno);
            vE = cd();
        }
        if (j == nj) {
            const double rRn = 0.5 * (rjp + rj), rLn = 0.5 * (rj + rjm);
            vP = vP - vN * cd(rLn / rRn);
            vN = cd();
        }
        if (j == 2) vS = cd();
    }
    aP[p] = vP; aE[p] = vE; aW[p] = vW; aN[p] = vN; aS[p] = vS; b[p] = vb;
}

int mw_er_assemble_dev(cth_grid* g, const double* ne, const double* nu, const double* epsr,
                       const cth_mw_params* prm, double* aP, double* aE, double* aW, double* aN, double* aS,
                       double* b, cudaStream_t s) {
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    k_mw_er_assemble<<<grd, blk, 0, s>>>(ne, nu, epsr, *prm, g->ni, g->nj, g->ld, reinterpret_cast<cd*>(aP),
                                         reinterpret_cast<cd*>(aE), reinterpret_cast<cd*>(aW),
                                         reinterpret_cast<cd*>(aN), reinterpret_cast<cd*>(aS),
                                         reinterpret_cast<cd*>(b));
    g->launches++;
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

}  // namespace cth
