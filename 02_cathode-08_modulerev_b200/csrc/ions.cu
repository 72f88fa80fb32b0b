// ions.cu — the ion sub-step of the time loop on the device (src/main.cpp:191-197):
// FluidModule::solve_Uix_tmp, solve_Uir_tmp, solve_Uip_tmp (fluidModule.hpp:123-1404),
// solve_rhoi_constTe (:1405-1755) and correct_Ui_constTe (:1763-2072).
//
// The three momentum equations are implicit upwind systems on their own index
// sets: Uix on the x faces, Uir on the r faces, Uip on the cells; each is solved
// on a grid whose blocks are that set's blocks.  Their interiors are assembled
// one thread per face (the face set is "both neighbouring cells in the fluid");
// the wall conditions of the reference are written per named wall segment, with
// ranges that differ between the loops (convex corners, the rows they write),
// so they run as a wall program: an ordered list of segment operations that one
// CTA executes in order, as the reference's loops do.  The continuity equation
// and the velocity correction follow the per-cell side flags.
#include <cuda_runtime.h>

#include <cmath>

#include "fluid.cuh"

namespace cth {

struct IonArgs {
    double *Uix, *Uir, *Uip, *rhoi, *rhoUix, *rhoUir, *rhoUix_wall, *rhoUir_wall;
    double *Uix_old, *Uir_old, *Uip_old, *rhoi_old;
    const double *phi, *Ex, *Er, *Bx, *Br, *rate_ionize, *nui_m;
    double *aP, *aE, *aW, *aN, *aS, *b;
    const unsigned char* flags;
    cth_ion_params prm;
    int ni, nj, ld;
};

#define FL(ii, jj) flag_at(A.flags, (ii), (jj), A.ni, A.nj, A.ld)

__device__ __forceinline__ double rcell(const cth_ion_params& P, int j) { return P.rmin + (j - 0.5) * P.dr; }

__global__ void k_ion_begin(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    A.Uix_old[p] = A.Uix[p];
    A.Uir_old[p] = A.Uir[p];
    A.Uip_old[p] = A.Uip[p];
    A.rhoi_old[p] = A.rhoi[p];
}

// ---- momentum interiors (coefficient planes zeroed outside the set) --------

// Uix on x faces (fluidModule.hpp:152-214)
__global__ void k_uix_assemble(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (FL(i, j) && FL(i - 1, j)) {
        const cth_ion_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_i = P.dt * double(P.ndt_i);
        const double rj = rcell(P, j), rL = (rj + rcell(P, j - 1)) / 2.0, rR = (rj + rcell(P, j + 1)) / 2.0;
        const double qL = rL / rj, qR = rR / rj;
        const double* Uo = A.Uix_old;
        const double* Ro = A.Uir_old;
        const double ULx = (Uo[p] + Uo[p - 1]) / 2.0, URx = (Uo[p] + Uo[p + 1]) / 2.0;
        const double ULr = (Ro[p] + Ro[p - 1]) / 2.0, URr = (Ro[p + ld] + Ro[p - 1 + ld]) / 2.0;
        const double rho_t = (A.rhoi[p] + A.rhoi[p - 1]) / 2.0;
        const double riz = (A.rate_ionize[p] + A.rate_ionize[p - 1]) / 2.0;
        const double nui = (A.nui_m[p] + A.nui_m[p - 1]) / 2.0;
        const double dndx = (A.rhoi[p] - A.rhoi[p - 1]) / dx;
        const double Uip_t = (A.Uip_old[p] + A.Uip_old[p - 1]) / 2.0;
        const double Br_t = (A.Br[p] + A.Br[p - 1]) / 2.0;
        const double lor = -kE0f * Uip_t * Br_t;
        vE = -(URx - fabs(URx)) / (2.0 * dx);
        vW = (ULx + fabs(ULx)) / (2.0 * dx);
        vN = -qR * (URr - fabs(URr)) / (2.0 * dr);
        vS = qL * (ULr + fabs(ULr)) / (2.0 * dr);
        vP = 1.0 / dt_i + riz / (rho_t + 1e-100) + nui + vE + vW + vN + vS;
        vb = Uo[p] / dt_i + (kE0f * A.Ex[p] + lor) / P.massi - kBoltz * P.Ti / (P.massi * rho_t + 1e-100) * dndx;
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// Uir on r faces (fluidModule.hpp:614-671)
__global__ void k_uir_assemble(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (FL(i, j) && FL(i, j - 1)) {
        const cth_ion_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_i = P.dt * double(P.ndt_i);
        const double rj = rcell(P, j), rjm = rcell(P, j - 1), rjmm = rcell(P, j - 2), rjp = rcell(P, j + 1);
        const double r_t = (rj + rjm) / 2.0, rL = (rjm + rjmm) / 2.0, rR = (rjp + rj) / 2.0;
        const double* Uo = A.Uix_old;
        const double* Ro = A.Uir_old;
        const double ULx = (rj * Uo[p] + rjm * Uo[p - ld]) / (2.0 * r_t);
        const double URx = (rj * Uo[p + 1] + rjm * Uo[p + 1 - ld]) / (2.0 * r_t);
        const double ULr = (r_t * Ro[p] + rL * Ro[p - ld]) / (2.0 * rjm);
        const double URr = (r_t * Ro[p] + rR * Ro[p + ld]) / (2.0 * rj);
        const double rho_t = (A.rhoi[p] + A.rhoi[p - ld]) / 2.0;
        const double riz = (A.rate_ionize[p] + A.rate_ionize[p - ld]) / 2.0;
        const double nui = (A.nui_m[p] + A.nui_m[p - ld]) / 2.0;
        const double dndr = (A.rhoi[p] - A.rhoi[p - ld]) / dr;
        const double Bx_t = (rj * A.Bx[p] + rjm * A.Bx[p - ld]) / (2.0 * r_t);
        const double Uip_t = (rj * A.Uip_old[p] + rjm * A.Uip_old[p - ld]) / (2.0 * r_t);
        const double lor = kE0f * Uip_t * Bx_t;
        const double cen = -Uip_t * Uip_t / r_t;
        vE = -(URx - fabs(URx)) / (2.0 * dx);
        vW = (ULx + fabs(ULx)) / (2.0 * dx);
        vN = -rj / r_t * (URr - fabs(URr)) / (2.0 * dr);
        vS = rjm / r_t * (ULr + fabs(ULr)) / (2.0 * dr);
        vP = 1.0 / dt_i + riz / (rho_t + 1e-100) + nui + vE + vW + vN + vS;
        vb = Ro[p] / dt_i + (kE0f * A.Er[p] + lor) / P.massi - kBoltz * P.Ti / (P.massi * rho_t + 1e-100) * dndr +
             cen;
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// Uip on cells (fluidModule.hpp:1067-1112)
__global__ void k_uip_assemble(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (FL(i, j)) {
        const cth_ion_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_i = P.dt * double(P.ndt_i);
        const double rj = rcell(P, j), rL = (rj + rcell(P, j - 1)) / 2.0, rR = (rj + rcell(P, j + 1)) / 2.0;
        const double qL = rL / rj, qR = rR / rj;
        const double* Uo = A.Uix_old;
        const double* Ro = A.Uir_old;
        const double ULx = Uo[p], URx = Uo[p + 1], ULr = Ro[p], URr = Ro[p + ld];
        const double Ux_t = (Uo[p + 1] + Uo[p]) / 2.0;
        const double Ur_t = (rL * Ro[p] + rR * Ro[p + ld]) / (2.0 * rj);
        const double lor = kE0f * (Ux_t * A.Br[p] - Ur_t * A.Bx[p]);
        const double cen = A.Uip[p] * Ur_t / rj;
        vE = -(URx - fabs(URx)) / (2.0 * dx);
        vW = (ULx + fabs(ULx)) / (2.0 * dx);
        vN = -qR * (URr - fabs(URr)) / (2.0 * dr);
        vS = qL * (ULr + fabs(ULr)) / (2.0 * dr);
        vP = 1.0 / dt_i + A.rate_ionize[p] / (A.rhoi[p] + 1e-100) + A.nui_m[p] + vE + vW + vN + vS;
        vb = A.Uip_old[p] / dt_i + lor / P.massi + cen;
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// ---- wall programs -----------------------------------------------------------

// wall velocity of energy conservation (fluidModule.hpp:224-228):
// sign sqrt(U_old^2 + max(2 e (phi_face - bias) / m_i, 0)), phi_face the mean of
// the two cells of the face (x face: i-1, i; r face: j-1, j)
__device__ __forceinline__ double ui_wall(const IonArgs& A, const double* Uold, int i, int j, const cth_ion_op& o) {
    const size_t p = (size_t)j * A.ld + i;
    const size_t q = o.pair == 0 ? p - 1 : p - A.ld;
    const double dphi = (A.phi[p] + A.phi[q]) / 2.0 - (o.bias ? A.prm.V_bias : 0.0);
    return o.sign * sqrt(Uold[p] * Uold[p] + fmax(2.0 * kE0f * dphi / A.prm.massi, 0.0));
}

__device__ __forceinline__ double* coef(const IonArgs& A, int dir) {
    return dir == 0 ? A.aW : dir == 1 ? A.aE : dir == 2 ? A.aS : A.aN;
}

__device__ __forceinline__ double rscale(const cth_ion_params& P, int kind, int j) {
    if (kind == 1) return rcell(P, j) / rcell(P, j - 1);
    if (kind == 2) return rcell(P, j) / rcell(P, j + 1);
    return 1.0;
}

// one CTA executes the operations in order; U is the unknown of the program
// (Uix, Uir or Uip) and Uold its value at the start of the ion step
__global__ void k_wall_program(IonArgs A, const cth_ion_op* __restrict__ ops, int nops, double* U,
                               const double* Uold) {
    for (int q = 0; q < nops; q++) {
        const cth_ion_op o = ops[q];
        const int wi = o.i1 - o.i0 + 1, wj = o.j1 - o.j0 + 1;
        for (int k = threadIdx.x; k < wi * wj; k += blockDim.x) {
            const int i = o.i0 + k / wj, j = o.j0 + k % wj;
            const size_t p = (size_t)j * A.ld + i;
            const size_t t = (size_t)(j + o.dj) * A.ld + (i + o.di);
            switch (o.kind) {
                case CTH_ION_WALL_FOLD: {
                    double* a = coef(A, o.dir);
                    A.b[p] = A.b[p] + a[p] * ui_wall(A, Uold, i, j, o);
                    a[p] = 0.0;
                } break;
                case CTH_ION_ZERO_COEF:
                    coef(A, o.dir)[p] = 0.0;
                    break;
                case CTH_ION_FOLD_SUB: {
                    double* a = coef(A, o.dir);
                    A.aP[p] = A.aP[p] - (o.scale ? a[p] * rscale(A.prm, o.scale, j) : a[p]);
                    a[p] = 0.0;
                } break;
                case CTH_ION_OPEN_FOLD: {
                    const double r_t = (rcell(A.prm, j) + rcell(A.prm, j - 1)) / 2.0;
                    const double rR = (rcell(A.prm, j + 1) + rcell(A.prm, j)) / 2.0;
                    A.b[p] = A.b[p] + A.aN[p] * r_t / rR * fmax(Uold[p], 0.0);
                    A.aN[p] = 0.0;
                } break;
                case CTH_ION_SET_WALL:
                    U[t] = ui_wall(A, Uold, i, j, o);
                    break;
                case CTH_ION_SET_ZERO:
                    U[t] = 0.0;
                    break;
                case CTH_ION_COPY:
                    U[t] = o.scale ? rscale(A.prm, o.scale, j) * U[p] : U[p];
                    break;
                case CTH_ION_SET_OPEN: {
                    const double r_t = (rcell(A.prm, j) + rcell(A.prm, j - 1)) / 2.0;
                    const double rR = (rcell(A.prm, j + 1) + rcell(A.prm, j)) / 2.0;
                    U[t] = r_t / rR * fmax(Uold[p], 0.0);
                } break;
                default:
                    break;
            }
        }
        __syncthreads();
    }
}

// ---- continuity ---------------------------------------------------------------

__device__ __forceinline__ double kin_flux(double u, double vth, double um, double sign) {
    const double ut = u / (um + 1e-100);
    return sign * 0.25 * vth * (exp(-ut * ut) + ut * sqrt(M_PI) * (erf(ut) + sign * 1.0));
}

// ion continuity with numerical diffusion and implicit kinetic wall fluxes
// (fluidModule.hpp:1415-1539)
__global__ void k_rhoi_assemble(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (fc) {
        const cth_ion_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_i = P.dt * double(P.ndt_i);
        const double rj = rcell(P, j), rL = (rj + rcell(P, j - 1)) / 2.0, rR = (rj + rcell(P, j + 1)) / 2.0;
        const double qL = rL / rj, qR = rR / rj;
        const double ULx = A.Uix[p], URx = A.Uix[p + 1], ULr = A.Uir[p], URr = A.Uir[p + ld];
        const double* nu = A.nui_m;
        const double Te_rep = P.Te_rep_eV * kE0f / kBoltz;
        const double nu_star = 1.0 / P.rmax * sqrt(kBoltz * Te_rep / P.massi);
        const double c = kBoltz * (P.Ti + Te_rep);
        const double DLx = c / (P.massi * ((nu[p] + nu[p - 1]) / 2.0 + nu_star) + 1e-100);
        const double DRx = c / (P.massi * ((nu[p] + nu[p + 1]) / 2.0 + nu_star) + 1e-100);
        const double DLr = c / (P.massi * ((nu[p] + nu[p - ld]) / 2.0 + nu_star) + 1e-100);
        const double DRr = c / (P.massi * ((nu[p] + nu[p + ld]) / 2.0 + nu_star) + 1e-100);
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bRx = (fc & F_BRX) ? 1.0 : 0.0;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = (fc & F_BRR_WALL) ? 1.0 : 0.0;
        const double vth = sqrt(8.0 * kBoltz * P.Ti / (M_PI * P.massi));
        const double um = sqrt(2.0 * kBoltz * P.Ti / P.massi);
        const double GLx = (fc & F_BLX) ? 0.0 : kin_flux(ULx, vth, um, -1.0);
        const double GRx = (fc & F_BRX) ? 0.0 : kin_flux(URx, vth, um, 1.0);
        const double GLr = (fc & F_BLR_WALL) ? 0.0 : kin_flux(ULr, vth, um, -1.0);
        const double GRr = (fc & F_BRR_WALL) ? 0.0 : kin_flux(URr, vth, um, 1.0);
        vP = (URx + fabs(URx)) / (2.0 * dx) * bRx - (ULx - fabs(ULx)) / (2.0 * dx) * bLx +
             qR * (URr + fabs(URr)) / (2.0 * dr) * bRr - qL * (ULr - fabs(ULr)) / (2.0 * dr) * bLr +
             ((DRx * bRx + DLx * bLx) / (dx * dx) + (qR * DRr * bRr + qL * DLr * bLr) / (dr * dr)) - GLx / dx +
             GRx / dx - qL * GLr / dr + qR * GRr / dr + 1.0 / dt_i;
        vE = (-(URx - fabs(URx)) / (2.0 * dx) + DRx / (dx * dx)) * bRx;
        vW = ((ULx + fabs(ULx)) / (2.0 * dx) + DLx / (dx * dx)) * bLx;
        vN = (-qR * (URr - fabs(URr)) / (2.0 * dr) + qR * DRr / (dr * dr)) * bRr;
        vS = (qL * (ULr + fabs(ULr)) / (2.0 * dr) + qL * DLr / (dr * dr)) * bLr;
        const double* ro = A.rhoi_old;
        const double div =
            (DRx * ro[p + 1] * bRx - (DRx * bRx + DLx * bLx) * ro[p] + DLx * ro[p - 1] * bLx) / (dx * dx) +
            (qR * DRr * ro[p + ld] * bRr - (qR * DRr * bRr + qL * DLr * bLr) * ro[p] + qL * DLr * ro[p - ld] * bLr) /
                (dr * dr);
        vb = ro[p] / dt_i + A.rate_ionize[p] - div;
        if (!(fc & F_BRR_OPEN)) {
            vP = vP - vN;
            vN = 0.0;
        }
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// wall fluxes of the solved density, positivity and the open ghost (fluidModule.hpp:1578-1752)
__global__ void k_rhoi_post(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    if (!fc) return;
    const cth_ion_params& P = A.prm;
    const double vth = sqrt(8.0 * kBoltz * P.Ti / (M_PI * P.massi));
    const double um = sqrt(2.0 * kBoltz * P.Ti / P.massi);
    double n = A.rhoi[p];
    if (!(fc & F_BLX)) A.rhoUix_wall[p] = n * kin_flux(A.Uix[p], vth, um, -1.0);
    if (!(fc & F_BRX)) A.rhoUix_wall[p + 1] = n * kin_flux(A.Uix[p + 1], vth, um, 1.0);
    if (!(fc & F_BLR_WALL)) A.rhoUir_wall[p] = n * kin_flux(A.Uir[p], vth, um, -1.0);
    if (!(fc & F_BRR_WALL)) A.rhoUir_wall[p + ld] = n * kin_flux(A.Uir[p + ld], vth, um, 1.0);
    if (!(fc & F_BRR_OPEN)) {
        A.rhoUir[p + ld] = n * A.Uir[p + ld];
        A.rhoUir_wall[p + ld] = 0.0;
    }
    if (n < 0.0) {
        n = fmax(A.rhoi_old[p], 0.0);
        A.rhoi[p] = n;
    }
    if (!(fc & F_BRR_OPEN)) A.rhoi[p + ld] = n;
}

// velocity correction by the change of the density gradient (fluidModule.hpp:1774-1835)
__global__ void k_ion_correct(IonArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const cth_ion_params& P = A.prm;
    const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
    const double Te_rep = P.Te_rep_eV * kE0f / kBoltz;
    const double nu_star = 1.0 / P.rmax * sqrt(kBoltz * Te_rep / P.massi);
    const double* n = A.rhoi;
    const double* no = A.rhoi_old;
    if (fc && fw) {
        const double D = kBoltz * (P.Ti + Te_rep) / (P.massi * ((A.nui_m[p] + A.nui_m[p - 1]) / 2.0 + nu_star) + 1e-100);
        const double rho_t = (n[p] + n[p - 1]) / 2.0;
        const double g_old = (no[p] - no[p - 1]) / P.dx;
        const double g_new = (n[p] - n[p - 1]) / P.dx;
        const double U = A.Uix[p];
        const double fl = n[p - 1] * (U + fabs(U)) / 2.0 + n[p] * (U - fabs(U)) / 2.0;
        A.rhoUix[p] = fl - D * (g_new - g_old);
        A.Uix[p] = U - D / (rho_t + 1e-100) * (g_new - g_old);
    }
    if ((fc && fs) || (fs && !(fs & F_BRR_OPEN))) {
        const double D =
            kBoltz * (P.Ti + Te_rep) / (P.massi * ((A.nui_m[p] + A.nui_m[p - ld]) / 2.0 + nu_star) + 1e-100);
        const double rho_t = (n[p] + n[p - ld]) / 2.0;
        const double g_old = (no[p] - no[p - ld]) / P.dr;
        const double g_new = (n[p] - n[p - ld]) / P.dr;
        const double U = A.Uir[p];
        const double fl = n[p - ld] * (U + fabs(U)) / 2.0 + n[p] * (U - fabs(U)) / 2.0;
        A.rhoUir[p] = fl - D * (g_new - g_old);
        A.Uir[p] = U - D / (rho_t + 1e-100) * (g_new - g_old);
    }
}

#undef FL

// ion residuals (fluidModule.hpp:1960-2070) over host-given index boxes, one
// thread per (box, i, j); boxes may overlap (the reference counts such faces twice)
__global__ void k_ion_res(const double* __restrict__ nw, const double* __restrict__ od,
                          const int* __restrict__ boxes, int nbox, int total, int ld, int mode, double eps_l2,
                          double CFL, double* __restrict__ part, unsigned int* counter, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (t < total) {
        int k = t, q = 0;
        for (; q < nbox; q++) {
            const int* B = boxes + 4 * q;
            const int n = (B[1] - B[0] + 1) * (B[3] - B[2] + 1);
            if (k < n) break;
            k -= n;
        }
        const int* B = boxes + 4 * q;
        const int wj = B[3] - B[2] + 1;
        const int i = B[0] + k / wj, j = B[2] + k % wj;
        const size_t p = (size_t)j * ld + i;
        const double a = nw[p], o = od[p];
        if (mode == 0)
            s[0] = fabs((a - o) / (a + o + 1e-100) * 2.0 / CFL);
        else
            s[0] = (a - o) * (a - o) / (o * o + eps_l2) / CFL;
    }
    grid_reduce<2>(s, mode == 0 ? 0x1u : 0x0u, part, counter, out);
}

static int ion_res(cth_fields* fs, const double* nw, const double* od, int which, double eps_l2, int mode,
                   double CFL, cudaStream_t s, double* out_dev) {
    const int total = fs->ion_box_total[which];
    if (total <= 0) return CTH_OK;
    const int nb = (total + 255) / 256;
    k_ion_res<<<nb, 256, 0, s>>>(nw, od, fs->ion_boxes[which], fs->ion_nbox[which], total, fs->g->ld, mode, eps_l2,
                                 CFL, fs->part, fs->g->ws.counter, out_dev);
    fs->g->launches++;
    return CTH_OK;
}

static int ion_step(cth_fields* fs, cth_grid* gx, cth_grid* gr, const cth_ion_params* prm, cudaStream_t s,
                    cth_ion_result* res) {
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_ion_step: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    if (gx->ld != g->ld || gr->ld != g->ld || gx->ni != g->ni || gr->nj != g->nj || gx->device != g->device ||
        gr->device != g->device) {
        set_error("cth_ion_step: the face grids must have the cell grid's shape and device");
        return CTH_ERR_ARG;
    }
    IonArgs A{};
    struct { const char* name; double** dst; } rw[] = {
        {"Uix", &A.Uix}, {"Uir", &A.Uir}, {"Uip", &A.Uip}, {"rhoi", &A.rhoi}, {"rhoUix", &A.rhoUix},
        {"rhoUir", &A.rhoUir}, {"rhoUix_wall", &A.rhoUix_wall}, {"rhoUir_wall", &A.rhoUir_wall},
        {"Uix_old", &A.Uix_old}, {"Uir_old", &A.Uir_old}, {"Uip_old", &A.Uip_old}, {"rhoi_old", &A.rhoi_old},
        {"pc_aP", &A.aP}, {"pc_aE", &A.aE}, {"pc_aW", &A.aW}, {"pc_aN", &A.aN}, {"pc_aS", &A.aS}, {"pc_b", &A.b}};
    for (auto& e : rw) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    struct { const char* name; const double** dst; } ro[] = {
        {"phi", &A.phi}, {"Ex", &A.Ex}, {"Er", &A.Er}, {"Bx", &A.Bx}, {"Br", &A.Br},
        {"rate_ionize", &A.rate_ionize}, {"nui_m", &A.nui_m}};
    for (auto& e : ro) {
        double* q = field_ptr(fs, e.name);
        if (!q) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
        *e.dst = q;
    }
    A.flags = fs->flags;
    A.prm = *prm;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    int solver_rc = 0;
    cth_status st[4] = {};
    auto solve = [&](cth_grid* gg, double* x, int k) -> int {
        int rc;
        if (prm->flag_iter == 0)
            rc = sor_solve_dev(gg, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, 1.9, prm->maxITR_SOR, prm->error_cnv_SOR, x, s,
                               &st[k]);
        else
            rc = smg_solve_dev(gg, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                               prm->precision, x, s, &st[k]);
        if (rc > solver_rc) solver_rc = rc;
        return rc;
    };
    auto program = [&](const IonArgs& AA, int which, double* U, const double* Uold, cudaStream_t ss) {
        if (fs->ion_nops[which] > 0) {
            k_wall_program<<<1, 256, 0, ss>>>(AA, fs->ion_ops[which], fs->ion_nops[which], U, Uold);
            g->launches++;
        }
    };
    // the three momentum components use only the values at the start of the ion
    // step, so each gets its own coefficient planes and their solves (on three
    // grids) run concurrently on three streams; results equal the sequential order
    IonArgs AX = A, AR = A, AC = A;
    {
        const char* pre[3] = {"ionx_", "ionr_", "ionp_"};
        IonArgs* dst[3] = {&AX, &AR, &AC};
        const char* nm[6] = {"aP", "aE", "aW", "aN", "aS", "b"};
        for (int c = 0; c < 3; c++) {
            double** q[6] = {&dst[c]->aP, &dst[c]->aE, &dst[c]->aW, &dst[c]->aN, &dst[c]->aS, &dst[c]->b};
            for (int k = 0; k < 6; k++) {
                *q[k] = field_ptr(fs, std::string(pre[c]) + nm[k]);
                if (!*q[k]) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
            }
        }
    }
    k_ion_begin<<<grd, blk, 0, s>>>(A);
    k_uix_assemble<<<grd, blk, 0, s>>>(AX);
    k_uir_assemble<<<grd, blk, 0, s>>>(AR);
    k_uip_assemble<<<grd, blk, 0, s>>>(AC);
    g->launches += 4;
    program(AX, CTH_ION_PROG_UIX_ASM, A.Uix, A.Uix_old, s);
    program(AR, CTH_ION_PROG_UIR_ASM, A.Uir, A.Uir_old, s);
    program(AC, CTH_ION_PROG_UIP_ASM, A.Uip, A.Uip_old, s);
    CTH_CUDA(cudaGetLastError());
    int pend_m[4] = {0, 0, 0, 0};  // MG solves whose status is read after the last synchronisation
    if (prm->flag_iter == 0) {
        // SOR: sequential, each component on its own coefficient planes
        const IonArgs* As[3] = {&AX, &AR, &AC};
        cth_grid* gs[3] = {gx, gr, g};
        double* Us[3] = {A.Uix, A.Uir, A.Uip};
        const double* Uo[3] = {A.Uix_old, A.Uir_old, A.Uip_old};
        const int post[3] = {CTH_ION_PROG_UIX_POST, CTH_ION_PROG_UIR_POST, CTH_ION_PROG_UIP_POST};
        for (int c = 0; c < 3; c++) {
            const IonArgs& C = *As[c];
            const int rc = sor_solve_dev(gs[c], C.aP, C.aE, C.aW, C.aN, C.aS, C.b, 1.9, prm->maxITR_SOR,
                                         prm->error_cnv_SOR, Us[c], s, &st[c]);
            if (rc < 0) return rc;
            if (rc > solver_rc) solver_rc = rc;
            program(C, post[c], Us[c], Uo[c], s);
        }
    } else {
        if (!fs->aux_ready) {
            // highest priority: when a prediction runs beside the ion step, the
            // latency-bound solve chain is scheduled first
            int lo = 0, hi = 0;
            CTH_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            for (int k = 0; k < 2; k++)
                CTH_CUDA(cudaStreamCreateWithPriority(&fs->aux_stream[k], cudaStreamNonBlocking, hi));
            for (int k = 0; k < 3; k++) CTH_CUDA(cudaEventCreateWithFlags(&fs->aux_event[k], cudaEventDisableTiming));
            fs->aux_ready = true;
        }
        cudaStream_t s1 = fs->aux_stream[0], s2 = fs->aux_stream[1];
        CTH_CUDA(cudaEventRecord(fs->aux_event[0], s));
        CTH_CUDA(cudaStreamWaitEvent(s1, fs->aux_event[0], 0));
        CTH_CUDA(cudaStreamWaitEvent(s2, fs->aux_event[0], 0));
        int pend[3] = {0, 0, 0};
        int rc = smg_solve_launch(gx, AX.aP, AX.aE, AX.aW, AX.aN, AX.aS, AX.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                                  prm->precision, A.Uix, s1, &pend[0], fs->h_solve + 0 * kStatStride,
                                  fs->warm_fields ? A.Uix : nullptr, fs->warm_tol, nullptr, SLOT_ION_MOMENTUM);
        if (rc < 0) return rc;
        program(AX, CTH_ION_PROG_UIX_POST, A.Uix, A.Uix_old, s1);
        rc = smg_solve_launch(gr, AR.aP, AR.aE, AR.aW, AR.aN, AR.aS, AR.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                              prm->precision, A.Uir, s2, &pend[1], fs->h_solve + 1 * kStatStride,
                              fs->warm_fields ? A.Uir : nullptr, fs->warm_tol, nullptr, SLOT_ION_MOMENTUM);
        if (rc < 0) return rc;
        program(AR, CTH_ION_PROG_UIR_POST, A.Uir, A.Uir_old, s2);
        rc = smg_solve_launch(g, AC.aP, AC.aE, AC.aW, AC.aN, AC.aS, AC.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                              prm->precision, A.Uip, s, &pend[2], fs->h_solve + 2 * kStatStride,
                              fs->warm_fields ? A.Uip : nullptr, fs->warm_tol, nullptr, SLOT_ION_MOMENTUM);
        if (rc < 0) return rc;
        program(AC, CTH_ION_PROG_UIP_POST, A.Uip, A.Uip_old, s);
        CTH_CUDA(cudaEventRecord(fs->aux_event[1], s1));
        CTH_CUDA(cudaEventRecord(fs->aux_event[2], s2));
        CTH_CUDA(cudaStreamWaitEvent(s, fs->aux_event[1], 0));
        CTH_CUDA(cudaStreamWaitEvent(s, fs->aux_event[2], 0));
        for (int c = 0; c < 3; c++) pend_m[c] = pend[c];
    }
    CTH_CUDA(cudaGetLastError());
    // continuity and correction
    k_rhoi_assemble<<<grd, blk, 0, s>>>(A);
    g->launches++;
    CTH_CUDA(cudaGetLastError());
    if (prm->flag_iter == 0) {
        if (solve(g, A.rhoi, 3) < 0) return CTH_ERR_CUDA;
    } else {
        const int rc = smg_solve_launch(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                                        prm->precision, A.rhoi, s, &pend_m[3], fs->h_solve + 3 * kStatStride,
                                        fs->warm_fields ? A.rhoi : nullptr, fs->warm_tol, nullptr,
                                        SLOT_ION_CONTINUITY);
        if (rc < 0) return rc;
    }
    k_rhoi_post<<<grd, blk, 0, s>>>(A);
    k_ion_correct<<<grd, blk, 0, s>>>(A);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    // residuals
    double* out = fs->scal + 48;
    const double* nw[4] = {A.rhoi, A.Uix, A.Uir, A.Uip};
    const double* od[4] = {A.rhoi_old, A.Uix_old, A.Uir_old, A.Uip_old};
    const double eps[4] = {1e10, 1e-6, 1e-6, 1e-6};
    const int mode = prm->flag_error == 0 ? 0 : 1;
    for (int k = 0; k < 4; k++) {
        CTH_CUDA(cudaMemsetAsync(out + 2 * k, 0, 2 * sizeof(double), s));
        ion_res(fs, nw[k], od[k], k, eps[k], mode, prm->CFL, s, out + 2 * k);
    }
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(fs->h_scal, out, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (prm->flag_iter != 0) {
        cth_grid* gs[4] = {gx, gr, g, g};
        for (int c = 0; c < 4; c++) {
            const int rc = solve_parse(gs[c], pend_m[c], fs->h_solve + kStatStride * c, &st[c]);
            if (rc < 0) return rc;
            if (rc > solver_rc) solver_rc = rc;
        }
    }
    if (res) {
        double e[4];
        for (int k = 0; k < 4; k++) {
            const double a = fs->h_scal[2 * k];
            e[k] = mode == 0 ? a : sqrt(a / double(fs->ion_box_total[k] > 0 ? fs->ion_box_total[k] : 1));
        }
        res->error_rhoi = e[0];
        res->error_Uix = e[1];
        res->error_Uir = e[2];
        res->error_Uip = e[3];
        res->solver_rc = solver_rc;
        for (int k = 0; k < 4; k++) res->solver[k] = st[k];
    }
    return CTH_OK;
}

}  // namespace cth

using namespace cth;

extern "C" int cth_ion_program_upload(cth_fields* fs, int which, const cth_ion_op* ops, int n) {
    if (!fs || which < 0 || which >= CTH_ION_NPROG || n < 0 || (n > 0 && !ops)) {
        set_error("cth_ion_program_upload: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    for (int q = 0; q < n; q++) {
        const cth_ion_op& o = ops[q];
        const bool box = o.i0 <= o.i1 && o.j0 <= o.j1 && o.i0 >= 0 && o.i1 <= g->ni + 1 && o.j0 >= 0 &&
                         o.j1 <= g->nj + 1;
        const bool tgt = o.i0 + o.di >= 0 && o.i1 + o.di <= g->ni + 1 && o.j0 + o.dj >= 0 &&
                         o.j1 + o.dj <= g->nj + 1;
        const bool ok_kind = o.kind >= CTH_ION_WALL_FOLD && o.kind <= CTH_ION_SET_OPEN;
        const bool reads_pair = o.kind == CTH_ION_WALL_FOLD || o.kind == CTH_ION_SET_WALL;
        const bool pair_ok = !reads_pair || (o.pair == 0 ? o.i0 >= 1 : o.j0 >= 1);
        if (!box || !tgt || !ok_kind || !pair_ok || o.dir < 0 || o.dir > 3 || o.pair < 0 || o.pair > 1 ||
            o.scale < 0 || o.scale > 2) {
            set_error("cth_ion_program_upload: operation " + std::to_string(q) + " out of range");
            return CTH_ERR_ARG;
        }
    }
    CTH_CUDA(cudaSetDevice(g->device));
    if (fs->ion_ops[which]) { cudaFree(fs->ion_ops[which]); fs->ion_ops[which] = nullptr; }
    fs->ion_nops[which] = 0;
    if (n == 0) return CTH_OK;
    CTH_CUDA(cudaMalloc(&fs->ion_ops[which], n * sizeof(cth_ion_op)));
    CTH_CUDA(cudaMemcpy(fs->ion_ops[which], ops, n * sizeof(cth_ion_op), cudaMemcpyHostToDevice));
    fs->ion_nops[which] = n;
    return CTH_OK;
}

extern "C" int cth_ion_boxes_upload(cth_fields* fs, int which, const int* boxes, int n) {
    if (!fs || which < 0 || which > 3 || n < 0 || (n > 0 && !boxes)) {
        set_error("cth_ion_boxes_upload: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    long long total = 0;
    for (int q = 0; q < n; q++) {
        const int* B = boxes + 4 * q;
        if (B[0] > B[1] || B[2] > B[3] || B[0] < 0 || B[1] > g->ni + 1 || B[2] < 0 || B[3] > g->nj + 1) {
            set_error("cth_ion_boxes_upload: box out of range");
            return CTH_ERR_ARG;
        }
        total += (long long)(B[1] - B[0] + 1) * (B[3] - B[2] + 1);
    }
    if (total > (long long)fs->npart * 64) {
        set_error("cth_ion_boxes_upload: boxes too large");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    if (fs->ion_boxes[which]) { cudaFree(fs->ion_boxes[which]); fs->ion_boxes[which] = nullptr; }
    fs->ion_nbox[which] = 0;
    fs->ion_box_total[which] = 0;
    if (n == 0) return CTH_OK;
    CTH_CUDA(cudaMalloc(&fs->ion_boxes[which], 4 * n * sizeof(int)));
    CTH_CUDA(cudaMemcpy(fs->ion_boxes[which], boxes, 4 * n * sizeof(int), cudaMemcpyHostToDevice));
    fs->ion_nbox[which] = n;
    fs->ion_box_total[which] = (int)total;
    return CTH_OK;
}

extern "C" int cth_ion_step(cth_fields* fs, cth_grid* gx, cth_grid* gr, const cth_ion_params* prm, void* stream,
                            cth_ion_result* res) {
    if (!fs || !gx || !gr || !prm || prm->dx <= 0.0 || prm->dr <= 0.0 || prm->dt <= 0.0 || prm->ndt_i < 1 ||
        prm->rmax <= 0.0 || prm->CFL <= 0.0) {
        set_error("cth_ion_step: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return ion_step(fs, gx, gr, prm, (cudaStream_t)stream, res);
}
