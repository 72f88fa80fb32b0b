// mw3.cu — the magnetised 3-component microwave system on the device.
//
// EmfieldModule::solve_Microwave (include/emfieldModule.hpp:2249-2998) couples
// three complex fields through the magnetised cold-plasma conductivity:
//   Ex on x-faces (i-1/2, j), Er on r-faces (i, j-1/2), Ephi on cells (i, j),
// each row an 11-point stencil (its own 5-point operator plus the face or cell
// averages of the other two components, :2300-2453), assembled into one sparse
// matrix of unknown-to-unknown couplings (:2785-2990) and factorised with Eigen
// SparseLU (:2995-2998).
//
// Geometry: each field's unknowns are the union of its block table (the x-face,
// r-face and cell blocks gx.i_flx_bl / gr.i_flr_bl / gc.i_flc_bl, six blocks on
// the cathode with the coax feed), held as the masks of three grids.  Assembly
// is the interior stencil on every unknown, then the boundary surgery of the
// reference's 12 lists (MicrowaveBC, include/arrays.hpp:649: for Ex, Er, Ephi in
// turn the W, E, S, N lists, each entry (i, j, code) with codes 0-7,
// :2456-2784), one launch per list in the reference's order; entries of one
// list are distinct rows, so a list's threads never touch the same
// coefficient.  The r-z rectangle (r in [0, R], z in [0, L]) is the special
// case of one block per field and the lists of its walls:
//   Ex   Gauss (code 2) at z = 0 and z = L, conductor (code 0) at r = R;
//   Er   port excitation (code 7) on the z = 0 faces with r1 <= r <= r2, open
//        (code 1) on the other z = 0 faces and at z = L, Gauss (code 2) at r = R;
//   Ephi open (code 1) at z = 0, conductor (code 0) at z = L and r = R;
// Ex i = 2..ni, j = 1..nj; Er i = 1..ni, j = 2..nj; Ephi i = 1..ni, j = 1..nj.
//
// Solver: BiCGStab in complex FP64 on the coupled operator, right-
// preconditioned block-diagonally by one complex semicoarsening V-cycle per
// field (the smg.cu hierarchy of the field's grid, built on the field's own
// 5-point block; rows of the bounding box off the unknowns are identity rows).
// Vectors live in the library layout (row j, column i, leading dimension ld),
// one plane per field,
// and stay exactly zero off their unknowns, so the coupled apply needs no
// neighbour tests: a coupling to a non-unknown multiplies a zero, which is the
// reference's dropped matrix entry.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "grid.h"
#include "line.cuh"

namespace cth {

int cmg_alloc(cth_grid* g);
int cmg_setup(cth_grid* g, cudaStream_t s);
int cmg_vcycle(cth_grid* g, cudaStream_t s);
int cmg32_alloc(cth_grid* g);
int cmg32_setup(cth_grid* g, cudaStream_t s);
int cmg32_vcycle(cth_grid* g, cudaStream_t s);

namespace m3 {

constexpr double kE0 = 1.60217662e-19;      // constants.hpp:6
constexpr double kEPS0 = 8.8541878128e-12;  // constants.hpp:7
constexpr double kMU0 = 1.2566370614e-6;    // constants.hpp:8

// coefficient slots of one field's rows; C0..C5 are the couplings:
//   Ex   C0..C3 = Er at NE (i, j+1), SE (i, j), NW (i-1, j+1), SW (i-1, j);  C4, C5 = Ephi at (i, j), (i-1, j)
//   Er   C0..C3 = Ex at NE (i+1, j), SE (i+1, j-1), NW (i, j), SW (i, j-1);  C4, C5 = Ephi at (i, j), (i, j-1)
//   Ephi C0, C1 = Ex at (i+1, j), (i, j);  C2, C3 = Er at (i, j+1), (i, j)
enum Slot3 { QP = 0, QE, QW, QN, QS, C0, C1, C2, C3, C4, C5, NQ };

// scalar words of the recurrence
enum Word3 {
    RHO = 0, RHO_OLD = 2, ALPHA = 4, OMEGA = 6, BETA = 8,
    BB = 10, RR = 11, RELRES = 12, ITER = 13, CONV = 14, BAD = 15, KEEP = 16,
    GUESS = 17,   // 0 no guess; 1 + r0: started from the guess; -(1 + r0): guess rejected (r0 its relative residual)
    NWORDS = 24
};

struct Lev0 {
    cd* b[3];   // preconditioner right-hand side, level 0 of each field's hierarchy
    cd* x[3];   // preconditioner result
    int i0[3], j0[3], ldl[3];
};

// per-call arguments, in device memory so that one captured graph serves every call
struct Args3 {
    int maxit;
    double tol;
    cd* out;  // three field planes
    const cd* x0;      // initial guess (three field planes, read on the unknowns) or null: zero start
    double guess_tol;  // the guess is used when ||b - A x0|| <= guess_tol ||b||
};

struct Dev3 {
    cd* a;  // [3][NQ] planes
    cd* b;  // [3] planes
    cd *x, *r, *rh, *p, *ph, *v, *s, *sh, *t;  // [3] planes each
    double* sc;
    const unsigned char* mk[3];  // unknowns of each field (library layout)
    int ni, nj, ld;
    size_t pl;
};

__device__ __forceinline__ cd sc_c(const double* sc, int w) { return cd(sc[w], sc[w + 1]); }
__device__ __forceinline__ void sc_set(double* sc, int w, cd v) { sc[w] = v.x; sc[w + 1] = v.y; }

// (A X)_row of field c at (i, j); X = three planes, zero off their unknowns
__device__ __forceinline__ cd apply3(const Dev3& D, const cd* __restrict__ X, int c, int i, int j) {
    const size_t pl = D.pl, q = (size_t)j * D.ld + i;
    const int ld = D.ld;
    const cd* A = D.a + (size_t)c * NQ * pl;
    const cd* F = X + (size_t)c * pl;
    const cd* Ex = X;
    const cd* Er = X + pl;
    const cd* Ep = X + 2 * pl;
    cd y = A[QP * pl + q] * F[q];
    y -= A[QE * pl + q] * F[q + 1];
    y -= A[QW * pl + q] * F[q - 1];
    y -= A[QN * pl + q] * F[q + ld];
    y -= A[QS * pl + q] * F[q - ld];
    if (c == 0) {
        y -= A[C0 * pl + q] * Er[q + ld];
        y -= A[C1 * pl + q] * Er[q];
        y -= A[C2 * pl + q] * Er[q - 1 + ld];
        y -= A[C3 * pl + q] * Er[q - 1];
        y -= A[C4 * pl + q] * Ep[q];
        y -= A[C5 * pl + q] * Ep[q - 1];
    } else if (c == 1) {
        y -= A[C0 * pl + q] * Ex[q + 1];
        y -= A[C1 * pl + q] * Ex[q + 1 - ld];
        y -= A[C2 * pl + q] * Ex[q];
        y -= A[C3 * pl + q] * Ex[q - ld];
        y -= A[C4 * pl + q] * Ep[q];
        y -= A[C5 * pl + q] * Ep[q - ld];
    } else {
        y -= A[C0 * pl + q] * Ex[q + 1];
        y -= A[C1 * pl + q] * Ex[q];
        y -= A[C2 * pl + q] * Er[q + ld];
        y -= A[C3 * pl + q] * Er[q];
    }
    return y;
}

// ---------------------------------------------------------------------------
// assembly
// ---------------------------------------------------------------------------
struct Sig {
    cd coef, hx, hr;
};

// coef and Hall factors of the conductivity (emfieldModule.hpp:2312-2318), with
// the reference's EPS = 1e-100 (1 + i) guards
__device__ __forceinline__ Sig sigma(double rho, double nu, double bx, double br, double w, double me) {
    const cd den(me * nu + 1e-100, me * w + 1e-100);
    Sig s;
    s.hx = cdiv(cd(kE0 * bx), den);
    s.hr = cdiv(cd(kE0 * br), den);
    const cd mag2 = s.hx * s.hx + s.hr * s.hr;
    s.coef = cdiv(cdiv(cd(rho * kE0 * kE0), den), cd(1.0 + 1e-100, 1e-100) + mag2);
    return s;
}

__device__ __forceinline__ cd mulr(cd a, double v) { return cd(a.x * v, a.y * v); }
__device__ __forceinline__ cd divr(cd a, double v) { return cd(a.x / v, a.y / v); }

// first-order open boundary factor along z of codes 1 (:2579-2588, :2720-2729)
__device__ __forceinline__ cd open_z(double eps_t, double w, double dx) {
    const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
    const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx) + 1e-100;
    return cd(((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx)) / deno, (-4.0 * c0 * w * dx) / deno);
}

// the same along r, on the r-weighted stencil of the north faces (:2553-2566,
// :2771-2782); r(j) and r(j+1) are the cell radii either side of the face
__device__ __forceinline__ cd open_rad(double eps_t, double w, double dr, double rj, double rjp) {
    const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
    const double rt = (rjp + rj) / 2.0;
    const double qL = rj / (rt + 1e-100), qR = rjp / (rt + 1e-100);
    const double t1 = 2.0 * c0 * sqrt(qR), t2 = w * dr * qR;
    const double deno = t1 * t1 + t2 * t2 + 1e-100;
    const cd R((2.0 * c0) * (2.0 * c0) * sqrt(qL * qR) - (w * dr) * (w * dr) * qL * qR,
               -2.0 * c0 * w * dr * (qL * sqrt(qR) + qR * sqrt(qL)));
    return divr(R, deno);
}

// interior stencils of the three fields on their unknowns (the boundary
// surgery follows, list by list)
// J3 != nullptr: the explicit variant solve_Microwave_explicit (:3328-4400): no plasma
// conductivity in the operator (ne, nu, Bx, Br are not read) and b = -i w mu0 dx^2 dr^2 J on
// the unknowns, J = sigma E of the previous field (J3[0..2]: J1x, J1r, J1p planes)
__global__ void k_m3_assemble(const double* __restrict__ ne, const double* __restrict__ nu,
                              const double* __restrict__ Bx, const double* __restrict__ Br,
                              const double* __restrict__ epsr, cth_mw_params prm, Dev3 D, const cd* J1x,
                              const cd* J1r, const cd* J1p) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    const int ld = D.ld;
    const size_t pl = D.pl, q = (size_t)j * ld + i;
    const double dx = prm.dx, dr = prm.dr, w = prm.omegam, me = prm.masse;
    const double g2 = dx * dx * dr * dr;
    const cd iwm(0.0, w * kMU0);
    auto r_of = [&](int jj) { return prm.rmin + (jj - 0.5) * dr; };
    const double rj = r_of(j), rjm = r_of(j - 1), rjp = r_of(j + 1);
    // ---- Ex (x-face between cells i-1 and i), :2300-2348 ----
    if (D.mk[0][q]) {
        cd* A = D.a;
        const double qL = (rjm + rj) / 2.0 / (rj + 1e-100);
        const double qR = (rjp + rj) / 2.0 / (rj + 1e-100);
        const Sig s = J1x ? Sig{} : sigma((ne[q] + ne[q - 1]) / 2.0, (nu[q] + nu[q - 1]) / 2.0,
                                          (Bx[q] + Bx[q - 1]) / 2.0, (Br[q] + Br[q - 1]) / 2.0, w, me);
        const double eps_t = (epsr[q] + epsr[q - 1]) / 2.0;
        const cd s_xr = s.coef * (s.hx * s.hr), s_xp = s.coef * s.hr, s_xx = s.coef * (cd(1.0) + s.hx * s.hx);
        const cd aP = cd(2.0 * dx * dx + 2.0 * dr * dr - kEPS0 * eps_t * kMU0 * w * w * g2) + iwm * s_xx * cd(g2);
        const cd aE(dr * dr), aW(dr * dr), aN(qR * dx * dx), aS(qL * dx * dx);
        const cd kp = iwm * s_xp * cd(-0.5 * g2), kr = iwm * s_xr * cd(-0.25 * g2);
        const cd cNE = kr * cd(qR), cSE = kr * cd(qL), cNW = kr * cd(qR), cSW = kr * cd(qL);
        A[QP * pl + q] = aP; A[QE * pl + q] = aE; A[QW * pl + q] = aW; A[QN * pl + q] = aN; A[QS * pl + q] = aS;
        A[C0 * pl + q] = cNE; A[C1 * pl + q] = cSE; A[C2 * pl + q] = cNW; A[C3 * pl + q] = cSW;
        A[C4 * pl + q] = kp; A[C5 * pl + q] = kp;
        D.b[q] = J1x ? cd(0.0, -w * kMU0 * g2) * J1x[q] : cd();
    }
    // ---- Er (r-face between cells j-1 and j), :2352-2411 ----
    if (D.mk[1][q]) {
        cd* A = D.a + (size_t)NQ * pl;
        const double rjmm = r_of(j - 2);
        const double r_t = (rjm + rj) / 2.0, rR = (rj + rjp) / 2.0, rL = (rjmm + rjm) / 2.0;
        const Sig s = J1r ? Sig{} : sigma((ne[q] + ne[q - ld]) / 2.0, (nu[q] + nu[q - ld]) / 2.0,
                                          (rj * Bx[q] + rjm * Bx[q - ld]) / (2.0 * r_t),
                                          (rj * Br[q] + rjm * Br[q - ld]) / (2.0 * r_t), w, me);
        const double eps_t = (epsr[q] + epsr[q - ld]) / 2.0;
        const cd s_rr = s.coef * (cd(1.0) + s.hr * s.hr), s_rp = s.coef * (-s.hx), s_rx = s.coef * (s.hx * s.hr);
        const cd aP = cd(r_t * (1.0 / rj + 1.0 / rjm) * dx * dx + 2.0 * dr * dr - kEPS0 * eps_t * kMU0 * w * w * g2) +
                iwm * s_rr * cd(g2);
        const cd aE(dr * dr), aW(dr * dr), aN(rR / rj * dx * dx), aS(rL / rjm * dx * dx);
        const cd kp = iwm * s_rp * cd(-0.5 * g2), kx = iwm * s_rx * cd(-0.25 * g2);
        const cd cNN = kp * cd(rj / r_t), cSS = kp * cd(rjm / r_t);
        const cd cNE = kx * cd(rj / r_t), cNW = kx * cd(rj / r_t), cSE = kx * cd(rjm / r_t), cSW = kx * cd(rjm / r_t);
        A[QP * pl + q] = aP; A[QE * pl + q] = aE; A[QW * pl + q] = aW; A[QN * pl + q] = aN; A[QS * pl + q] = aS;
        A[C0 * pl + q] = cNE; A[C1 * pl + q] = cSE; A[C2 * pl + q] = cNW; A[C3 * pl + q] = cSW;
        A[C4 * pl + q] = cNN; A[C5 * pl + q] = cSS;
        D.b[pl + q] = J1r ? cd(0.0, -w * kMU0 * g2) * J1r[q] : cd();
    }
    // ---- Ephi (cell), :2414-2453 ----
    if (D.mk[2][q]) {
        cd* A = D.a + (size_t)2 * NQ * pl;
        const double qL = (rjm + rj) / 2.0 / (rj + 1e-100);
        const double qR = (rjp + rj) / 2.0 / (rj + 1e-100);
        const Sig s = J1p ? Sig{} : sigma(ne[q], nu[q], Bx[q], Br[q], w, me);
        const cd s_pr = s.coef * s.hx, s_pp = s.coef, s_px = s.coef * (-s.hr);
        const cd aP = cd(2.0 * dx * dx + 2.0 * dr * dr + g2 / (rj * rj) - kEPS0 * epsr[q] * kMU0 * w * w * g2) +
                iwm * s_pp * cd(g2);
        const cd aE(dr * dr), aW(dr * dr), aN(qR * dx * dx), aS(qL * dx * dx);
        const cd kx = iwm * s_px * cd(-0.5 * g2), kr = iwm * s_pr * cd(-0.5 * g2);
        A[QP * pl + q] = aP; A[QE * pl + q] = aE; A[QW * pl + q] = aW; A[QN * pl + q] = aN; A[QS * pl + q] = aS;
        A[C0 * pl + q] = kx; A[C1 * pl + q] = kx; A[C2 * pl + q] = kr * cd(qR); A[C3 * pl + q] = kr * cd(qL);
        A[C4 * pl + q] = cd(); A[C5 * pl + q] = cd();
        D.b[2 * pl + q] = J1p ? cd(0.0, -w * kMU0 * g2) * J1p[q] : cd();
    }
}

// boundary surgery of one list (list = 4 field + side; fields Ex, Er, Ephi;
// sides W, E, S, N), one entry (i, j, code) per thread, after
// emfieldModule.hpp:2456-2784.  Codes the reference does not define for a list
// leave the row as it is, as there.  jflc is gc.j_flc_bl[0][0], which the Er
// south code 3 compares with the cell radius (:2672).
__global__ void k_m3_bc(Dev3 D, const int* __restrict__ ent, int n, int list, const double* __restrict__ epsr,
                        cth_mw_params prm, double jflc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = ent[3 * k], j = ent[3 * k + 1], code = ent[3 * k + 2];
    const int ld = D.ld;
    const size_t pl = D.pl, q = (size_t)j * ld + i;
    const int c = list >> 2, side = list & 3;
    cd* A = D.a + (size_t)c * NQ * pl + q;
    const double dx = prm.dx, dr = prm.dr, w = prm.omegam;
    auto r = [&](int jj) { return prm.rmin + (jj - 0.5) * dr; };
#define AT(slot) A[(size_t)(slot) * pl]
    if (c == 0) {
        const double qL = (r(j - 1) + r(j)) / 2.0 / (r(j) + 1e-100), qR = (r(j + 1) + r(j)) / 2.0 / (r(j) + 1e-100);
        if (side == 0) {  // :2458-2489
            const cd a = AT(QW);
            if (code == 0) {
                AT(QW) = cd();
            } else if (code == 2) {
                AT(QP) -= a; AT(C2) += mulr(divr(mulr(a, dx), dr), qR); AT(C3) -= mulr(divr(mulr(a, dx), dr), qL);
                AT(QW) = cd();
            } else if (code == 3) {
                const double deno = 1.0 + dx / dr * qL;
                AT(QP) -= divr(a, deno); AT(C2) += divr(mulr(a, dx / dr * qR), deno); AT(QW) = cd();
            } else if (code == 4) {
                const double deno = 1.0 + dx / dr * qR;
                AT(QP) -= divr(a, deno); AT(C3) -= divr(mulr(a, dx / dr * qL), deno); AT(QW) = cd();
            }
        } else if (side == 1) {  // :2491-2514
            const cd a = AT(QE);
            if (code == 0) {
                AT(QE) = cd();
            } else if (code == 2) {
                AT(QP) -= a; AT(C0) -= mulr(divr(mulr(a, dx), dr), qR); AT(C1) += mulr(divr(mulr(a, dx), dr), qL);
                AT(QE) = cd();
            } else if (code == 4) {
                const double deno = 1.0 + dx / dr * qR;
                AT(QP) -= divr(a, deno); AT(C1) += divr(mulr(a, dx / dr * qL), deno); AT(QE) = cd();
            }
        } else if (side == 2) {  // :2516-2531
            const cd a = AT(QS);
            if (code == 0) {
                AT(QP) += mulr(a, r(j) / r(j - 1)); AT(QS) = cd();
            } else if (code == 6) {
                const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
                AT(QP) -= mulr(a, dr / dx * r(j) / rL); AT(QW) += mulr(a, -dr / dx * r(j) / rL);
                AT(C2) += mulr(a, rR / rL); AT(QS) = cd();
            }
        } else {  // :2533-2571
            const cd a = AT(QN);
            const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
            if (code == 0) {
                AT(QP) += mulr(a, r(j) / r(j + 1)); AT(QN) = cd();
            } else if (code == 1) {
                AT(QP) -= a * open_rad((epsr[q] + epsr[q - 1]) / 2.0, w, dr, r(j), r(j + 1)); AT(QN) = cd();
            } else if (code == 5) {
                AT(QP) -= mulr(a, dr / dx * r(j) / rR); AT(QE) += mulr(a, -dr / dx * r(j) / rR);
                AT(C1) += mulr(a, rL / rR); AT(QN) = cd();
            } else if (code == 6) {
                AT(QP) -= mulr(a, dr / dx * r(j) / rR); AT(QW) += mulr(a, -dr / dx * r(j) / rR);
                AT(C3) += mulr(a, -rL / rR); AT(QN) = cd();
            }
        }
    } else if (c == 1) {
        const double eps_t = (epsr[q] + epsr[q - ld]) / 2.0;
        if (side == 0) {  // :2574-2622
            const cd a = AT(QW);
            if (code == 0) {
                AT(QP) += a; AT(QW) = cd();
            } else if (code == 1) {
                AT(QP) -= a * open_z(eps_t, w, dx); AT(QW) = cd();
            } else if (code == 5) {
                const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
                AT(QP) -= mulr(a, dx / dr * rL / r(j)); AT(QN) += mulr(a, -dx / dr * rR / r(j));
                AT(C0) += mulr(a, -1.0); AT(QW) = cd();
            } else if (code == 6) {
                const double rR = (r(j) + r(j - 1)) / 2.0, rL = (r(j - 1) + r(j - 2)) / 2.0;
                AT(QP) -= mulr(a, dx / dr * rR / r(j - 1)); AT(QS) += mulr(a, -dx / dr * rL / r(j - 1));
                AT(C1) += mulr(a, 1.0); AT(QW) = cd();
            } else if (code == 7) {  // port excitation (:2606-2621)
                const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
                const cd deno(2.0 * c0 + 1e-100, w * dx);
                const cd Rq(2.0 * c0, -w * dx);
                const double rt = (r(j) + r(j - 1)) / 2.0;
                const cd S = cd(0.0, 4.0 * w * dx) * cd(prm.J1r_exc / rt / log(prm.r2 / prm.r1) * 1e3);
                AT(QP) -= cdiv(a * Rq, deno);
                D.b[pl + q] += cdiv(a * S, deno);
                AT(QW) = cd();
            }
        } else if (side == 1) {  // :2624-2656
            const cd a = AT(QE);
            if (code == 0) {
                AT(QP) += a; AT(QE) = cd();
            } else if (code == 1) {
                const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
                const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx);
                const cd R((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx), -4.0 * c0 * w * dx);
                AT(QP) -= divr(a * R, deno + 1e-100); AT(QE) = cd();
            } else if (code == 5) {
                const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
                AT(QP) -= mulr(a, dx / dr * rL / r(j)); AT(QN) += mulr(a, -dx / dr * rR / r(j));
                AT(C2) += mulr(a, 1.0); AT(QE) = cd();
            }
        } else if (side == 2) {  // :2658-2681
            const cd a = AT(QS);
            const double rR = (r(j) + r(j - 1)) / 2.0, rL = (r(j - 1) + r(j - 2)) / 2.0;
            const cd g = divr(mulr(divr(mulr(a, dr), dx), r(j - 1)), rL);
            if (code == 2) {
                AT(QP) -= divr(mulr(a, rR), rL); AT(C1) += g; AT(C3) -= g; AT(QS) = cd();
            } else if (code == 3) {
                double deno = dr / dx * r(j - 1) / rL;
                if (r(j) < jflc) deno = 1.0;
                AT(QP) -= divr(divr(mulr(a, rR), rL), deno); AT(C0) += divr(g, deno); AT(QS) = cd();
            }
        } else {  // :2683-2711
            const cd a = AT(QN);
            const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
            const cd g = divr(mulr(divr(mulr(a, dr), dx), r(j)), rR);
            if (code == 2) {
                AT(QP) -= divr(mulr(a, rL), rR); AT(C0) -= g; AT(C2) += g; AT(QN) = cd();
            } else if (code == 3 || code == 4) {
                const double deno = dr / dx * r(j) / rR;
                AT(QP) -= divr(divr(mulr(a, rL), rR), deno);
                if (code == 3) AT(C1) -= divr(g, deno);
                else AT(C3) += divr(g, deno);
                AT(QN) = cd();
            }
        }
    } else {
        if (side == 0) {  // :2713-2730
            const cd a = AT(QW);
            if (code == 0) {
                AT(QP) += a; AT(QW) = cd();
            } else if (code == 1) {
                AT(QP) -= a * open_z(epsr[q], w, dx); AT(QW) = cd();
            }
        } else if (side == 1) {  // :2731-2739
            if (code == 0) { AT(QP) += AT(QE); AT(QE) = cd(); }
        } else if (side == 2) {  // :2741-2749
            if (code == 0) { AT(QP) += mulr(AT(QS), r(j) / r(j - 1)); AT(QS) = cd(); }
        } else {  // :2751-2784
            const cd a = AT(QN);
            if (code == 0) {
                AT(QP) += mulr(a, r(j) / r(j + 1)); AT(QN) = cd();
            } else if (code == 1) {
                AT(QP) -= a * open_rad(epsr[q], w, dr, r(j), r(j + 1)); AT(QN) = cd();
            }
        }
    }
#undef AT
}

// ghost values of one list after the solve (emfieldModule.hpp:3026-3264), one
// entry per thread, lists in the reference's order.  The ghosts a list writes
// are no unknowns of their field (checked when the lists are set), so no thread
// reads a value that another thread of the same list writes; values off the
// unknowns that a list reads are the ghosts of earlier lists or calls, as in
// the reference's persistent fields.  er_dc is gr.Er, which the Er east code 1
// reads, dividing by its deno twice (:3162).
__global__ void k_m3_ghost(const int* __restrict__ ent, int n, int list, cd* __restrict__ E,
                           const double* __restrict__ er_dc, const double* __restrict__ epsr, cth_mw_params prm,
                           double jflc, int ld, size_t pl) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = ent[3 * k], j = ent[3 * k + 1], code = ent[3 * k + 2];
    const size_t q = (size_t)j * ld + i;
    const int c = list >> 2, side = list & 3;
    cd* Ex = E;
    cd* Er = E + pl;
    cd* Ep = E + 2 * pl;
    const double dx = prm.dx, dr = prm.dr, w = prm.omegam;
    auto r = [&](int jj) { return prm.rmin + (jj - 0.5) * dr; };
    if (c == 0) {
        const double qL = (r(j - 1) + r(j)) / 2.0 / (r(j) + 1e-100), qR = (r(j + 1) + r(j)) / 2.0 / (r(j) + 1e-100);
        if (side == 0) {  // :3028-3053
            if (code == 0) {
                Ex[q - 1] = cd();
            } else if (code == 2) {
                Ex[q - 1] = Ex[q] + mulr(mulr(Er[q - 1 + ld], qR) - mulr(Er[q - 1], qL), dx / dr);
            } else if (code == 3) {
                const double deno = 1.0 + dx / dr * qL;
                Ex[q - 1] = divr(Ex[q], deno) + divr(mulr(mulr(Er[q - 1 + ld], qR), dx / dr), deno);
            } else if (code == 4) {
                const double deno = 1.0 + dx / dr * qR;
                Ex[q - 1] = divr(Ex[q], deno) - divr(mulr(mulr(Er[q - 1], qL), dx / dr), deno);
            }
        } else if (side == 1) {  // :3054-3073
            if (code == 0) {
                Ex[q + 1] = cd();
            } else if (code == 2) {
                Ex[q + 1] = Ex[q] - mulr(mulr(Er[q + ld], qR) - mulr(Er[q], qL), dx / dr);
            } else if (code == 4) {
                const double deno = 1.0 + dx / dr * qR;
                Ex[q + 1] = divr(Ex[q], deno) + divr(mulr(Er[q], dx / dr * qL), deno);
            }
        } else if (side == 2) {  // :3074-3083
            if (code == 0) Ex[q - ld] = mulr(Ex[q], -r(j) / r(j - 1));
        } else {  // :3084-3107
            if (code == 0) Ex[q + ld] = mulr(Ex[q], -r(j) / r(j + 1));
            else if (code == 1) Ex[q + ld] = open_rad((epsr[q] + epsr[q - 1]) / 2.0, w, dr, r(j), r(j + 1)) * Ex[q];
        }
    } else if (c == 1) {
        const double eps_t = (epsr[q] + epsr[q - ld]) / 2.0;
        if (side == 0) {  // :3109-3143
            if (code == 0) {
                Er[q - 1] = -Er[q];
            } else if (code == 1) {
                Er[q - 1] = open_z(eps_t, w, dx) * Er[q];
            } else if (code == 7) {
                const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
                const cd deno(2.0 * c0 + 1e-100, w * dx);
                const cd Rq(2.0 * c0, -w * dx);
                const double rt = (r(j) + r(j - 1)) / 2.0;
                const cd S = cd(0.0, 4.0 * w * dx) * cd(prm.J1r_exc / rt / log(prm.r2 / prm.r1) * 1e3);
                Er[q - 1] = cdiv(Rq, deno) * Er[q] + cdiv(S, deno);
            }
        } else if (side == 1) {  // :3144-3166
            if (code == 0) {
                Er[q + 1] = -Er[q];
            } else if (code == 1) {
                const double c0 = sqrt(1.0 / (kEPS0 * eps_t * kMU0));
                const double deno = (2.0 * c0) * (2.0 * c0) + (w * dx) * (w * dx);
                const cd R = divr(cd((2.0 * c0) * (2.0 * c0) - (w * dx) * (w * dx), -4.0 * c0 * w * dx), deno + 1e-100);
                Er[q + 1] = mulr(divr(R, deno + 1e-100), er_dc[q]);
            }
        } else if (side == 2) {  // :3167-3187
            const double rR = (r(j) + r(j - 1)) / 2.0, rL = (r(j - 1) + r(j - 2)) / 2.0;
            if (code == 2) {
                Er[q - ld] = mulr(Er[q], rR / rL) + mulr(Ex[q + 1 - ld] - Ex[q - ld], dr / dx * r(j - 1) / rL);
            } else if (code == 3) {
                double deno = dr / dx * r(j - 1) / rL;
                if (r(j) < jflc) deno = 1.0;
                Er[q - ld] = divr(mulr(Er[q], rR / rL), deno) + divr(mulr(Ex[q + 1 - ld], dr / dx * r(j - 1) / rL), deno);
            }
        } else {  // :3188-3212
            const double rR = (r(j + 1) + r(j)) / 2.0, rL = (r(j) + r(j - 1)) / 2.0;
            const double deno = dr / dx * r(j) / rR;
            if (code == 2)
                Er[q + ld] = mulr(Er[q], rL / rR) - mulr(Ex[q + 1] - Ex[q], dr / dx * r(j) / rR);
            else if (code == 3)
                Er[q + ld] = divr(mulr(Er[q], rL / rR), deno) - divr(mulr(Ex[q + 1], dr / dx * r(j) / rR), deno);
            else if (code == 4)
                Er[q + ld] = divr(mulr(Er[q], rL / rR), deno) + divr(mulr(Ex[q], dr / dx * r(j) / rR), deno);
        }
    } else {
        if (side == 0) {  // :3213-3229
            if (code == 0) Ep[q - 1] = -Ep[q];
            else if (code == 1) Ep[q - 1] = open_z(epsr[q], w, dx) * Ep[q];
        } else if (side == 1) {  // :3230-3236, every code
            Ep[q + 1] = -Ep[q];
        } else if (side == 2) {  // :3237-3243, every code
            Ep[q - ld] = mulr(Ep[q], -r(j) / r(j - 1));
        } else {  // :3244-3264
            if (code == 0) Ep[q + ld] = mulr(Ep[q], -r(j) / r(j + 1));
            else if (code == 1) Ep[q + ld] = open_rad(epsr[q], w, dr, r(j), r(j + 1)) * Ep[q];
        }
    }
}

// level-0 operator of field c's preconditioner hierarchy: its own 5-point block,
// couplings to non-unknowns dropped, identity rows off the unknowns
__global__ void k_m3_block(Dev3 D, int c, cd* __restrict__ a0, int i0, int j0, int ncol, int nrow, int ldl) {
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y;
    if (cc >= ncol) return;
    const size_t n0 = (size_t)nrow * ldl, p = (size_t)rr * ldl + cc;
    const int i = cc + i0, j = rr + j0;
    const size_t pl = D.pl, q = (size_t)j * D.ld + i;
    const cd* A = D.a + (size_t)c * NQ * pl;
    const unsigned char* mk = D.mk[c];
    cd vP(1.0), vW, vE, vS, vN;
    if (mk[q]) {
        vP = A[QP * pl + q];
        if (cc > 0 && mk[q - 1]) vW = A[QW * pl + q];
        if (cc + 1 < ncol && mk[q + 1]) vE = A[QE * pl + q];
        if (rr > 0 && mk[q - D.ld]) vS = A[QS * pl + q];
        if (rr + 1 < nrow && mk[q + D.ld]) vN = A[QN * pl + q];
    }
    a0[P * n0 + p] = vP;
    a0[W * n0 + p] = vW;
    a0[E * n0 + p] = vE;
    a0[S * n0 + p] = vS;
    a0[N * n0 + p] = vN;
}

// x = the caller's guess on the unknowns (zero without one; zero off the unknowns,
// so that the coupled apply needs no neighbour tests)
__global__ void k_m3_x0(Dev3 D, const Args3* __restrict__ args) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    const cd* __restrict__ x0 = args->x0;
    for (int c = 0; c < 3; c++) {
        const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
        if (!D.mk[c][q - (size_t)c * D.pl]) continue;
        D.x[q] = x0 ? x0[q] : cd();
    }
}

// r = b - A x of the guess, its norm and ||b||; the last block decides (sc[GUESS])
__global__ void k_m3_guess(Dev3 D, const Args3* __restrict__ args, double* __restrict__ part,
                           unsigned int* counter) {
    __shared__ double red[32];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    double acc[2] = {0.0, 0.0};
    if (i <= D.ni && args->x0) {
        for (int c = 0; c < 3; c++) {
            const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
            if (!D.mk[c][q - (size_t)c * D.pl]) continue;
            const cd r = D.b[q] - apply3(D, D.x, c, i, j);
            D.r[q] = r;
            acc[0] += abs2(r);
            acc[1] += abs2(D.b[q]);
        }
    }
    double tot[2];
    if (last_block_sumk<2>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        if (!args->x0) {
            D.sc[GUESS] = 0.0;
        } else {
            const double r0 = tot[1] > 0.0 ? sqrt(tot[0] / tot[1]) : INFINITY;
            const bool use = isfinite(r0) && r0 <= args->guess_tol;
            D.sc[GUESS] = use ? 1.0 + r0 : -(1.0 + (isfinite(r0) ? fmin(r0, 1e30) : 1e30));
        }
    }
}

// from the guess (sc[GUESS] >= 1): r = rh = b - A x0, x = x0; otherwise r = rh = b,
// x = 0.  p = v = 0 on the unknowns; ||b||^2, ||r||^2 and the recurrence's start
__global__ void k_m3_prep(Dev3 D, const Args3* __restrict__ args, double* __restrict__ part, unsigned int* counter,
                          cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double red[32];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const bool guess = D.sc[GUESS] >= 1.0;
    double acc[2] = {0.0, 0.0};  // ||b||^2, ||r||^2
    if (i <= D.ni) {
        for (int c = 0; c < 3; c++) {
            const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
            if (!D.mk[c][q - (size_t)c * D.pl]) continue;
            const cd b = D.b[q];
            const cd r = guess ? D.r[q] : b;
            D.r[q] = r; D.rh[q] = r;
            if (!guess) D.x[q] = cd();
            D.p[q] = cd(); D.v[q] = cd();
            acc[0] += abs2(b);
            acc[1] += abs2(r);
        }
    }
    double tot[2];
    if (last_block_sumk<2>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        double* sc = D.sc;
        const double bb = tot[0], rr = tot[1];
        const bool fin = isfinite(bb) && isfinite(rr);
        const double rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        sc_set(sc, RHO, cd(rr));
        sc_set(sc, RHO_OLD, cd(1.0));
        sc_set(sc, ALPHA, cd(1.0));
        sc_set(sc, OMEGA, cd(1.0));
        sc_set(sc, BETA, cd(0.0));
        sc[BB] = bb;
        sc[RR] = rr;
        sc[RELRES] = bb > 0.0 ? rel : 0.0;
        sc[ITER] = 0.0;
        // from zero: at least one iteration unless b = 0; from a guess: stop at once when it meets the tolerance
        const bool met = rr == 0.0 || (guess && rel < args->tol);
        sc[CONV] = (fin && met) ? 1.0 : 0.0;
        sc[BAD] = fin ? 0.0 : 1.0;
        const bool keep = fin && !met && args->maxit > 0;
        sc[KEEP] = keep ? 1.0 : 0.0;
        if (use_cond) cudaGraphSetConditional(cond, keep ? 1u : 0u);
    }
}

// MODE 0: p = r + beta (p - omega v);  MODE 1: s = r - alpha v.  The vector is
// also scattered into the fields' preconditioner right-hand sides.
template <int MODE>
__global__ void k_m3_vec(Dev3 D, Lev0 L) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    const cd beta = sc_c(D.sc, BETA), omega = sc_c(D.sc, OMEGA), alpha = sc_c(D.sc, ALPHA);
    for (int c = 0; c < 3; c++) {
        const size_t q0 = (size_t)j * D.ld + i;
        if (!D.mk[c][q0]) continue;
        const size_t q = (size_t)c * D.pl + q0;
        cd y;
        if (MODE == 0) {
            y = D.r[q] + beta * (D.p[q] - omega * D.v[q]);
            D.p[q] = y;
        } else {
            y = D.r[q] - alpha * D.v[q];
            D.s[q] = y;
        }
        L.b[c][(size_t)(j - L.j0[c]) * L.ldl[c] + (i - L.i0[c])] = y;
    }
}

// the preconditioner results into dst (ph or sh)
__global__ void k_m3_gather(Dev3 D, Lev0 L, cd* __restrict__ dst) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    for (int c = 0; c < 3; c++) {
        const size_t q0 = (size_t)j * D.ld + i;
        if (!D.mk[c][q0]) continue;
        dst[(size_t)c * D.pl + q0] = L.x[c][(size_t)(j - L.j0[c]) * L.ldl[c] + (i - L.i0[c])];
    }
}

// one field's preconditioner result into dst
template <int F>
__global__ void k_m3_gather1(Dev3 D, Lev0 L, cd* __restrict__ dst) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    const size_t q0 = (size_t)j * D.ld + i;
    if (!D.mk[F][q0]) return;
    dst[(size_t)F * D.pl + q0] = L.x[F][(size_t)(j - L.j0[F]) * L.ldl[F] + (i - L.i0[F])];
}

// block Gauss-Seidel across the fields (Ex, then Er, then Ephi): field F's
// preconditioner right-hand side is its part of y (p for MODE 0, s for MODE 1)
// minus the couplings of its rows to the fields already preconditioned, whose
// results z are in dst's planes (Er rows: Ex; Ephi rows: Ex and Er)
template <int MODE, int F>
__global__ void k_m3_gs(Dev3 D, Lev0 L, const cd* __restrict__ z) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > D.ni) return;
    const int ld = D.ld;
    const size_t pl = D.pl, q = (size_t)j * ld + i;
    if (!D.mk[F][q]) return;
    const cd* Y = (MODE == 0 ? D.p : D.s) + (size_t)F * pl;
    const cd* A = D.a + (size_t)F * NQ * pl;
    const cd* zx = z;
    const cd* zr = z + pl;
    cd b = Y[q];
    if (F == 1) {
        b += A[C0 * pl + q] * zx[q + 1] + A[C1 * pl + q] * zx[q + 1 - ld] + A[C2 * pl + q] * zx[q] +
             A[C3 * pl + q] * zx[q - ld];
    } else {
        b += A[C0 * pl + q] * zx[q + 1] + A[C1 * pl + q] * zx[q] + A[C2 * pl + q] * zr[q + ld] +
             A[C3 * pl + q] * zr[q];
    }
    L.b[F][(size_t)(j - L.j0[F]) * L.ldl[F] + (i - L.i0[F])] = b;
}

// MODE 0: v = A ph, alpha = rho / <rh, v>;  MODE 1: t = A sh, omega = <t, s> / <t, t>
template <int MODE>
__global__ void k_m3_mv(Dev3 D, double* __restrict__ part, unsigned int* counter) {
    __shared__ double red[32];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    double acc[3] = {0.0, 0.0, 0.0};
    if (i <= D.ni) {
        for (int c = 0; c < 3; c++) {
            const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
            if (!D.mk[c][q - (size_t)c * D.pl]) continue;
            if (MODE == 0) {
                const cd y = apply3(D, D.ph, c, i, j);
                D.v[q] = y;
                const cd h = conj(D.rh[q]) * y;
                acc[0] += h.x; acc[1] += h.y;
            } else {
                const cd y = apply3(D, D.sh, c, i, j);
                D.t[q] = y;
                const cd h = conj(y) * D.s[q];
                acc[0] += h.x; acc[1] += h.y; acc[2] += abs2(y);
            }
        }
    }
    double tot[3];
    if (last_block_sumk<3>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        double* sc = D.sc;
        if (MODE == 0) {
            const cd den(tot[0], tot[1]);
            if (abs2(den) == 0.0 || !isfinite(tot[0]) || !isfinite(tot[1])) {
                sc[BAD] = 1.0;
                sc_set(sc, ALPHA, cd(0.0));
            } else {
                sc_set(sc, ALPHA, cdiv(sc_c(sc, RHO), den));
            }
        } else {
            if (tot[2] == 0.0 || !isfinite(tot[2])) {
                sc_set(sc, OMEGA, cd(0.0));
                if (!(tot[2] == 0.0)) sc[BAD] = 1.0;
            } else {
                sc_set(sc, OMEGA, cd(tot[0] / tot[2], tot[1] / tot[2]));
            }
        }
    }
}

// x += alpha ph + omega sh; r = s - omega t; stopping rule and next beta
__global__ void k_m3_upd(Dev3 D, const Args3* __restrict__ args, double* __restrict__ part, unsigned int* counter,
                         cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double red[32];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    double acc[3] = {0.0, 0.0, 0.0};
    if (i <= D.ni) {
        const cd alpha = sc_c(D.sc, ALPHA), omega = sc_c(D.sc, OMEGA);
        for (int c = 0; c < 3; c++) {
            const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
            if (!D.mk[c][q - (size_t)c * D.pl]) continue;
            D.x[q] = D.x[q] + alpha * D.ph[q] + omega * D.sh[q];
            const cd rn = D.s[q] - omega * D.t[q];
            D.r[q] = rn;
            const cd h = conj(D.rh[q]) * rn;
            acc[0] += abs2(rn); acc[1] += h.x; acc[2] += h.y;
        }
    }
    double tot[3];
    if (last_block_sumk<3>(acc, part, counter, red, tot) && threadIdx.x == 0) {
        double* sc = D.sc;
        const int it = (int)sc[ITER] + 1;
        const double bb = sc[BB];
        const double rel = bb > 0.0 ? sqrt(tot[0] / bb) : 0.0;
        const bool fin = isfinite(tot[0]) && isfinite(tot[1]) && isfinite(tot[2]);
        const cd rho_old = sc_c(sc, RHO), rho(tot[1], tot[2]);
        const cd alpha = sc_c(sc, ALPHA), omega = sc_c(sc, OMEGA);
        bool bad = sc[BAD] != 0.0 || !fin;
        const bool conv = fin && rel < args->tol;
        if (!conv && (abs2(rho_old) == 0.0 || abs2(omega) == 0.0)) bad = true;
        const cd beta = bad ? cd(0.0) : cdiv(rho, rho_old) * cdiv(alpha, omega);
        sc_set(sc, RHO_OLD, rho_old);
        sc_set(sc, RHO, rho);
        sc_set(sc, BETA, beta);
        sc[RR] = tot[0];
        sc[RELRES] = rel;
        sc[ITER] = (double)it;
        sc[CONV] = conv ? 1.0 : 0.0;
        sc[BAD] = bad ? 1.0 : 0.0;
        const bool keep = !conv && !bad && it < args->maxit;
        sc[KEEP] = keep ? 1.0 : 0.0;
        if (use_cond) cudaGraphSetConditional(cond, keep ? 1u : 0u);
    }
}

// the solution into the caller's planes on the unknowns; entries off the
// unknowns (ghosts) keep their values, as the reference's fields do
__global__ void k_m3_store(Dev3 D, const Args3* __restrict__ args) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= D.ld) return;
    for (int c = 0; c < 3; c++) {
        const size_t q0 = (size_t)j * D.ld + i;
        if (!D.mk[c][q0]) continue;
        const size_t q = (size_t)c * D.pl + q0;
        args->out[q] = D.x[q];
    }
}

// dst = src on the unknowns, zero elsewhere (3 planes)
__global__ void k_m3_mask(Dev3 D, const cd* __restrict__ src, cd* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= D.ld) return;
    for (int c = 0; c < 3; c++) {
        const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
        dst[q] = D.mk[c][q - (size_t)c * D.pl] ? src[q] : cd();
    }
}

// y = A x on the unknowns (zero elsewhere)
__global__ void k_m3_apply(Dev3 D, const cd* __restrict__ x, cd* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= D.ld) return;
    for (int c = 0; c < 3; c++) {
        const size_t q = (size_t)c * D.pl + (size_t)j * D.ld + i;
        y[q] = D.mk[c][q - (size_t)c * D.pl] ? apply3(D, x, c, i, j) : cd();
    }
}

}  // namespace m3
}  // namespace cth

using namespace cth;
using namespace cth::m3;

struct cth_mw3 {
    int device = 0, ni = 0, nj = 0, ld = 0;
    size_t pl = 0;
    cth_grid* g[3] = {nullptr, nullptr, nullptr};
    cd* a = nullptr;    // [3][NQ] planes
    cd* b = nullptr;    // [3] planes
    cd* vec = nullptr;  // 9 vectors x [3] planes
    cd* tmp = nullptr;  // [3] planes (masked copy of an apply input)
    double* sc = nullptr;
    double* h_sc = nullptr;  // pinned
    double* part = nullptr;
    unsigned int* counter = nullptr;
    bool assembled = false;
    long long launches = 0;
    // the Er and Ephi kernels run beside the Ex ones: set 0 for the set-up, set 1
    // for the iteration (a stream that joined a capture stays in it until the
    // capture ends, so the loop body's own capture needs its own side streams)
    cudaStream_t side[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaEvent_t fork[2] = {nullptr, nullptr}, join[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaStream_t cap[2] = {nullptr, nullptr};   // capture streams of the solve graph
    Args3* d_args = nullptr;
    Args3* h_args = nullptr;                    // pinned
    bool use_graphs = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int n_pre = 0, n_body = 0, n_post = 0;      // kernels per section of the graph
    // unknowns (host copies of the grids' masks, [i * (nj + 2) + j]) and the
    // boundary lists: (i, j, code) entries of the 12 lists back to back
    std::vector<unsigned char> hmask[3];
    int* lst = nullptr;
    size_t lst_cap = 0;
    int cnt[12] = {}, off[12] = {};
    double jflc = 0.0;
    bool has_bc = false;
    bool ghosts_ok = false;   // no list writes a ghost onto an unknown
    bool needs_er_dc = false; // the Er east list has code-1 entries (they read gr.Er)
    // rectangle: its lists follow the port radii and cell size of each assembly
    bool rect = false;
    double rect_key[4] = {0.0, 0.0, 0.0, 0.0};
    bool gauss_seidel = false;  // preconditioner: block Jacobi (default) or block Gauss-Seidel across the fields
    int precision = CTH_PREC_FP64;  // the preconditioner's V-cycles: complex FP64, or FP32 (CTH_PREC_MIXED)
};

namespace {

Dev3 dev3(cth_mw3* m) {
    Dev3 D;
    D.a = m->a;
    D.b = m->b;
    cd** f[9] = {&D.x, &D.r, &D.rh, &D.p, &D.ph, &D.v, &D.s, &D.sh, &D.t};
    for (int k = 0; k < 9; k++) *f[k] = m->vec + (size_t)k * 3 * m->pl;
    D.sc = m->sc;
    for (int c = 0; c < 3; c++) D.mk[c] = m->g[c]->mask_full;
    D.ni = m->ni;
    D.nj = m->nj;
    D.ld = m->ld;
    D.pl = m->pl;
    return D;
}

Lev0 lev0(cth_mw3* m) {
    Lev0 L;
    for (int c = 0; c < 3; c++) {
        cth_grid* g = m->g[c];
        L.b[c] = g->hc.b[0];
        L.x[c] = g->hc.x[0];
        L.i0[c] = g->i0;
        L.j0[c] = g->j0;
        L.ldl[c] = g->ldl;
    }
    return L;
}

void destroy(cth_mw3* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    for (int c = 0; c < 3; c++)
        if (m->g[c]) cth_grid_destroy(m->g[c]);
    for (void* p : {(void*)m->a, (void*)m->b, (void*)m->vec, (void*)m->tmp, (void*)m->sc, (void*)m->part,
                    (void*)m->counter})
        if (p) cudaFree(p);
    if (m->h_sc) cudaFreeHost(m->h_sc);
    for (int u = 0; u < 2; u++) {
        for (int k = 0; k < 2; k++) {
            if (m->side[u][k]) cudaStreamDestroy(m->side[u][k]);
            if (m->join[u][k]) cudaEventDestroy(m->join[u][k]);
        }
        if (m->fork[u]) cudaEventDestroy(m->fork[u]);
    }
    for (int k = 0; k < 2; k++)
        if (m->cap[k]) cudaStreamDestroy(m->cap[k]);
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    if (m->d_args) cudaFree(m->d_args);
    if (m->h_args) cudaFreeHost(m->h_args);
    if (m->lst) cudaFree(m->lst);
    delete m;
}

// the three fields' kernels side by side: field 0 on s, fields 1 and 2 on the side
// streams (inside a capture the side streams join it through the fork event)
cudaError_t fork3(cth_mw3* m, int u, cudaStream_t s) {
    cudaError_t e = cudaEventRecord(m->fork[u], s);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = cudaStreamWaitEvent(m->side[u][k], m->fork[u], 0);
    return e;
}

cudaError_t join3(cth_mw3* m, int u, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
        e = cudaEventRecord(m->join[u][k], m->side[u][k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, m->join[u][k], 0);
    }
    return e;
}

// preconditioner hierarchies from the fields' own 5-point blocks, then the
// recurrence's start
cudaError_t solve_pre(cth_mw3* m, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond, int* n) {
    Dev3 D = dev3(m);
    cudaError_t e = fork3(m, 0, s);
    if (e != cudaSuccess) return e;
    for (int c = 0; c < 3; c++) {
        cth_grid* g = m->g[c];
        cudaStream_t sc = c == 0 ? s : m->side[0][c - 1];
        dim3 gb(256), gg((g->ncol + 255) / 256, g->nrow[0]);
        k_m3_block<<<gg, gb, 0, sc>>>(D, c, g->hc.a[0], g->i0, g->j0, g->ncol, g->nrow[0], g->ldl);
        *n += 1 + (m->precision == CTH_PREC_MIXED ? cmg32_setup(g, sc) : cmg_setup(g, sc));
    }
    e = join3(m, 0, s);
    if (e != cudaSuccess) return e;
    dim3 blk(128), grd((m->ni + 127) / 128, m->nj);
    k_m3_x0<<<grd, blk, 0, s>>>(D, m->d_args);
    k_m3_guess<<<grd, blk, 0, s>>>(D, m->d_args, m->part, m->counter);
    k_m3_prep<<<grd, blk, 0, s>>>(D, m->d_args, m->part, m->counter, cond, use_cond);
    *n += 3;
    return cudaGetLastError();
}

// one BiCGStab iteration; the three fields' V-cycles of each preconditioner
// application run side by side
cudaError_t solve_body(cth_mw3* m, cudaStream_t s, cudaGraphConditionalHandle cond, int use_cond, int* n) {
    Dev3 D = dev3(m);
    Lev0 L = lev0(m);
    dim3 blk(128), grd((m->ni + 127) / 128, m->nj);
    // the preconditioner applied to p (mode 0) or s (mode 1), result into dst
    // one field's V-cycle: complex FP64, or FP32 with the right-hand side rounded and the result widened
    auto vcyc = [&](cth_grid* g, cudaStream_t st) -> int {
        return m->precision == CTH_PREC_MIXED ? cmg32_vcycle(g, st) : cmg_vcycle(g, st);
    };
    auto precond = [&](int mode, cd* dst) -> cudaError_t {
        if (!m->gauss_seidel) {  // block Jacobi: the three V-cycles side by side
            cudaError_t e = fork3(m, 1, s);
            if (e != cudaSuccess) return e;
            *n += vcyc(m->g[0], s);
            for (int k = 0; k < 2; k++) *n += vcyc(m->g[1 + k], m->side[1][k]);
            e = join3(m, 1, s);
            if (e != cudaSuccess) return e;
            k_m3_gather<<<grd, blk, 0, s>>>(D, L, dst);
            *n += 1;
            return cudaGetLastError();
        }
        // block Gauss-Seidel: Ex, then Er and Ephi with the known fields' couplings taken out
        *n += vcyc(m->g[0], s);
        k_m3_gather1<0><<<grd, blk, 0, s>>>(D, L, dst);
        if (mode == 0) k_m3_gs<0, 1><<<grd, blk, 0, s>>>(D, L, dst);
        else k_m3_gs<1, 1><<<grd, blk, 0, s>>>(D, L, dst);
        *n += vcyc(m->g[1], s);
        k_m3_gather1<1><<<grd, blk, 0, s>>>(D, L, dst);
        if (mode == 0) k_m3_gs<0, 2><<<grd, blk, 0, s>>>(D, L, dst);
        else k_m3_gs<1, 2><<<grd, blk, 0, s>>>(D, L, dst);
        *n += vcyc(m->g[2], s);
        k_m3_gather1<2><<<grd, blk, 0, s>>>(D, L, dst);
        *n += 5;
        return cudaGetLastError();
    };
    k_m3_vec<0><<<grd, blk, 0, s>>>(D, L);
    cudaError_t e = precond(0, D.ph);
    if (e != cudaSuccess) return e;
    k_m3_mv<0><<<grd, blk, 0, s>>>(D, m->part, m->counter);
    k_m3_vec<1><<<grd, blk, 0, s>>>(D, L);
    e = precond(1, D.sh);
    if (e != cudaSuccess) return e;
    k_m3_mv<1><<<grd, blk, 0, s>>>(D, m->part, m->counter);
    k_m3_upd<<<grd, blk, 0, s>>>(D, m->d_args, m->part, m->counter, cond, use_cond);
    *n += 5;
    return cudaGetLastError();
}

int solve_post(cth_mw3* m, cudaStream_t s) {
    dim3 blk(128), grd((m->ld + 127) / 128, m->nj + 2);
    k_m3_store<<<grd, blk, 0, s>>>(dev3(m), m->d_args);
    return 1;
}

// the whole solve as one graph: set-up, a conditional WHILE node around the
// iteration (its condition set by the reduction kernels), the store
int build_graph(cth_mw3* m) {
    if (m->exec) return CTH_OK;
    cudaStream_t cs = m->cap[0], cs2 = m->cap[1];
    CTH_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
    cudaGraphConditionalHandle cond = 0;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
    int n_pre = 0, n_body = 0;
    if (e == cudaSuccess) e = solve_pre(m, cs, cond, 1, &n_pre);
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
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
            e = solve_body(m, cs2, cond, 1, &n_body);
            cudaGraph_t bout = nullptr;
            const cudaError_t e2 = cudaStreamEndCapture(cs2, &bout);
            if (e == cudaSuccess) e = e2;
        }
    }
    int n_post = 0;
    if (e == cudaSuccess) n_post = solve_post(m, cs);
    cudaGraph_t out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cs, &out);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&m->exec, out, 0);
    if (e != cudaSuccess) {
        if (out) cudaGraphDestroy(out);
        m->exec = nullptr;
        cudaGetLastError();
        return cuda_fail(e, "magnetised microwave solve graph capture");
    }
    m->graph = out;
    m->n_pre = n_pre;
    m->n_body = n_body;
    m->n_post = n_post;
    return CTH_OK;
}

// the lists into device memory (set-up time: waits for the device first, since
// earlier assemblies may still read the old lists)
int upload_lists(cth_mw3* m, const std::vector<int>& ent, const int cnt[12]) {
    // which ghost each (list, code) writes (emfieldModule.hpp:3026-3264)
    static const int off_i[4] = {-1, 1, 0, 0}, off_j[4] = {0, 0, -1, 1};
    static const unsigned char writes[12] = {  // bit per code
        0x1D, 0x15, 0x01, 0x03, 0x83, 0x03, 0x0C, 0x1C, 0x03, 0xFF, 0xFF, 0x03};
    bool ok = true, er_dc = false;
    size_t e = 0;
    for (int L = 0; L < 12; L++) {
        const std::vector<unsigned char>& hm = m->hmask[L >> 2];
        for (int k = 0; k < cnt[L]; k++, e += 3) {
            const int i = ent[e], j = ent[e + 1], code = ent[e + 2];
            if (L == 5 && code == 1) er_dc = true;
            if (!(writes[L] >> code & 1)) continue;
            if (hm[(size_t)(i + off_i[L & 3]) * (m->nj + 2) + (j + off_j[L & 3])]) ok = false;
        }
    }
    m->ghosts_ok = ok;
    m->needs_er_dc = er_dc;
    CTH_CUDA(cudaDeviceSynchronize());
    const size_t n = ent.size() / 3;
    if (n > m->lst_cap) {
        if (m->lst) cudaFree(m->lst);
        m->lst = nullptr;
        m->lst_cap = 0;
        CTH_CUDA(cudaMalloc(&m->lst, n * 3 * sizeof(int)));
        m->lst_cap = n;
    }
    if (n) CTH_CUDA(cudaMemcpy(m->lst, ent.data(), n * 3 * sizeof(int), cudaMemcpyHostToDevice));
    int o = 0;
    for (int L = 0; L < 12; L++) {
        m->cnt[L] = cnt[L];
        m->off[L] = o;
        o += cnt[L];
    }
    m->has_bc = true;
    m->assembled = false;
    return CTH_OK;
}

// the rectangle's walls as the 12 lists (port code 7 on the z = 0 Er faces with
// r1 <= r <= r2, else 1), rebuilt when the cell size or port radii change
int rect_lists(cth_mw3* m, const cth_mw_params* prm, cudaStream_t s) {
    const double key[4] = {prm->dr, prm->rmin, prm->r1, prm->r2};
    if (m->has_bc && std::memcmp(key, m->rect_key, sizeof(key)) == 0) return CTH_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CTH_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
        set_error("cth_mw3_assemble_dev: the rectangle's boundary lists change (new cell size or port radii) "
                  "inside a stream capture");
        return CTH_ERR_ARG;
    }
    const int ni = m->ni, nj = m->nj;
    std::vector<int> L[12];
    auto put = [&](int l, int i, int j, int code) { L[l].insert(L[l].end(), {i, j, code}); };
    auto r = [&](int jj) { return prm->rmin + (jj - 0.5) * prm->dr; };
    for (int j = 1; j <= nj; j++) {
        put(0, 2, j, 2);   // Ex W: Gauss
        put(1, ni, j, 2);  // Ex E: Gauss
        put(8, 1, j, 1);   // Ephi W: open
        put(9, ni, j, 0);  // Ephi E: conductor
    }
    for (int j = 2; j <= nj; j++) {
        const double rt = (r(j) + r(j - 1)) / 2.0;
        put(4, 1, j, (rt >= prm->r1 && rt <= prm->r2) ? 7 : 1);  // Er W: port or open
        put(5, ni, j, 1);                                         // Er E: open
    }
    for (int i = 1; i <= ni; i++) {
        put(7, i, nj, 2);                // Er N: Gauss
        if (i >= 2) put(3, i, nj, 0);    // Ex N: conductor
        put(11, i, nj, 0);               // Ephi N: conductor
    }
    std::vector<int> ent;
    int cnt[12];
    for (int l = 0; l < 12; l++) {
        ent.insert(ent.end(), L[l].begin(), L[l].end());
        cnt[l] = (int)L[l].size() / 3;
    }
    const int rc = upload_lists(m, ent, cnt);
    if (rc == CTH_OK) std::memcpy(m->rect_key, key, sizeof(key));
    return rc;
}

}  // namespace

extern "C" {

int cth_mw3_create_blocks(int ni, int nj, const int* xi_bl, const int* xj_bl, int nx_bl, const int* ri_bl,
                          const int* rj_bl, int nr_bl, const int* ci_bl, const int* cj_bl, int nc_bl, int device,
                          cth_mw3** out) {
    const int* ib[3] = {xi_bl, ri_bl, ci_bl};
    const int* jb[3] = {xj_bl, rj_bl, cj_bl};
    const int nb[3] = {nx_bl, nr_bl, nc_bl};
    bool ok = out && ni >= 4 && nj >= 4;
    // every unknown inside [1, ni] x [1, nj] (the stencils read one ghost layer);
    // Er faces above the axis face (j >= 2)
    for (int c = 0; c < 3 && ok; c++) {
        ok = ib[c] && jb[c] && nb[c] >= 1;
        for (int b = 0; b < nb[c] && ok; b++) {
            const int a0 = ib[c][2 * b], a1 = ib[c][2 * b + 1], b0 = jb[c][2 * b], b1 = jb[c][2 * b + 1];
            if (a0 > a1 || b0 > b1) continue;  // empty block
            ok = a0 >= 1 && a1 <= ni && b0 >= (c == 1 ? 2 : 1) && b1 <= nj;
        }
    }
    if (!ok) {
        set_error("cth_mw3_create_blocks: invalid arguments (ni, nj >= 4; blocks inside [1, ni] x [1, nj], "
                  "Er blocks from j = 2)");
        return CTH_ERR_ARG;
    }
    *out = nullptr;
    cth_mw3* m = new cth_mw3();
    m->device = device;
    m->ni = ni;
    m->nj = nj;
    for (int c = 0; c < 3; c++) {
        m->hmask[c].assign((size_t)(ni + 2) * (nj + 2), 0);
        for (int b = 0; b < nb[c]; b++)
            for (int i = ib[c][2 * b]; i <= ib[c][2 * b + 1]; i++)
                for (int j = jb[c][2 * b]; j <= jb[c][2 * b + 1]; j++) m->hmask[c][(size_t)i * (nj + 2) + j] = 1;
        const int rc = cth_grid_create(ni, nj, ib[c], jb[c], nb[c], device, &m->g[c]);
        if (rc != CTH_OK) {
            destroy(m);
            return rc;
        }
        const int rc2 = cmg_alloc(m->g[c]);
        if (rc2 != CTH_OK) {
            destroy(m);
            return rc2;
        }
    }
    m->ld = m->g[2]->ld;
    m->pl = m->g[2]->plane;
    const size_t pl = m->pl;
    const int nparts = ((ni + 127) / 128) * nj;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&m->a, (size_t)3 * NQ * pl * sizeof(cd));
    if (e == cudaSuccess) e = cudaMalloc(&m->b, (size_t)3 * pl * sizeof(cd));
    if (e == cudaSuccess) e = cudaMalloc(&m->vec, (size_t)27 * pl * sizeof(cd));
    if (e == cudaSuccess) e = cudaMalloc(&m->tmp, (size_t)3 * pl * sizeof(cd));
    if (e == cudaSuccess) e = cudaMalloc(&m->sc, NWORDS * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&m->part, (size_t)(3 * nparts + 8) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&m->counter, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&m->h_sc, NWORDS * sizeof(double));
    if (e == cudaSuccess) e = cth::zero_fill(m->a, (size_t)3 * NQ * pl * sizeof(cd));
    if (e == cudaSuccess) e = cth::zero_fill(m->b, (size_t)3 * pl * sizeof(cd));
    if (e == cudaSuccess) e = cth::zero_fill(m->vec, (size_t)27 * pl * sizeof(cd));
    if (e == cudaSuccess) e = cth::zero_fill(m->sc, NWORDS * sizeof(double));
    if (e == cudaSuccess) e = cth::zero_fill(m->counter, sizeof(unsigned int));
    for (int u = 0; u < 2; u++) {
        for (int k = 0; k < 2 && e == cudaSuccess; k++) {
            e = cudaStreamCreateWithFlags(&m->side[u][k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->join[u][k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->fork[u], cudaEventDisableTiming);
    }
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = cudaStreamCreateWithFlags(&m->cap[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_args, sizeof(Args3));
    if (e == cudaSuccess) e = cudaMallocHost(&m->h_args, sizeof(Args3));
    if (e != cudaSuccess) {
        destroy(m);
        return cuda_fail(e, "cth_mw3_create");
    }
    *out = m;
    return CTH_OK;
}

int cth_mw3_create(int ni, int nj, int device, cth_mw3** out) {
    if (!out || ni < 4 || nj < 4) {
        set_error("cth_mw3_create: invalid arguments (ni, nj >= 4)");
        return CTH_ERR_ARG;
    }
    const int xi[2] = {2, ni}, xj[2] = {1, nj}, ri[2] = {1, ni}, rj[2] = {2, nj}, ci[2] = {1, ni}, cj[2] = {1, nj};
    const int rc = cth_mw3_create_blocks(ni, nj, xi, xj, 1, ri, rj, 1, ci, cj, 1, device, out);
    if (rc == CTH_OK) (*out)->rect = true;
    return rc;
}

int cth_mw3_set_boundary(cth_mw3* m, const cth_bc_list* lists, int j_flc_00) {
    if (!m || !lists) {
        set_error("cth_mw3_set_boundary: invalid arguments");
        return CTH_ERR_ARG;
    }
    const int nj2 = m->nj + 2;
    std::vector<int> ent;
    int cnt[12];
    std::vector<int> seen((size_t)(m->ni + 2) * nj2, -1);
    for (int L = 0; L < 12; L++) {
        const cth_bc_list& l = lists[L];
        if (l.n < 0 || (l.n > 0 && (!l.i || !l.j || !l.code))) {
            set_error("cth_mw3_set_boundary: list with a negative length or a null array");
            return CTH_ERR_ARG;
        }
        const std::vector<unsigned char>& hm = m->hmask[L >> 2];
        for (int k = 0; k < l.n; k++) {
            const int i = l.i[k], j = l.j[k], code = l.code[k];
            const bool ok = i >= 1 && i <= m->ni && j >= 1 && j <= m->nj && code >= 0 && code <= 7 &&
                            hm[(size_t)i * nj2 + j] && seen[(size_t)i * nj2 + j] != L;
            if (!ok) {
                set_error("cth_mw3_set_boundary: an entry is not an unknown of its field, repeats within its list, "
                          "or has a code outside 0-7");
                return CTH_ERR_ARG;
            }
            seen[(size_t)i * nj2 + j] = L;
            ent.push_back(i);
            ent.push_back(j);
            ent.push_back(code);
        }
        cnt[L] = l.n;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    const int rc = upload_lists(m, ent, cnt);
    if (rc != CTH_OK) return rc;
    m->jflc = (double)j_flc_00;
    m->rect = false;
    return CTH_OK;
}

void cth_mw3_destroy(cth_mw3* m) { destroy(m); }

int cth_mw3_ld(const cth_mw3* m) { return m ? m->ld : -1; }

long long cth_mw3_launch_count(const cth_mw3* m) {
    if (!m) return -1;
    long long n = m->launches;
    for (int c = 0; c < 3; c++) n += cth_launch_count(m->g[c]);
    return n;
}

int cth_mw3_copy_planes(const cth_mw3* m, double* a_dst, double* b_dst, void* stream) {
    if (!m || !a_dst || !b_dst) {
        set_error("cth_mw3_copy_planes: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = (cudaStream_t)stream;
    CTH_CUDA(cudaMemcpyAsync(a_dst, m->a, (size_t)3 * NQ * m->pl * sizeof(cd), cudaMemcpyDeviceToDevice, s));
    CTH_CUDA(cudaMemcpyAsync(b_dst, m->b, (size_t)3 * m->pl * sizeof(cd), cudaMemcpyDeviceToDevice, s));
    return CTH_OK;
}

static int mw3_assemble(cth_mw3* m, const double* ne, const double* nu, const double* Bx, const double* Br,
                        const double* epsr, const cth_mw_params* prm, void* stream, const void* J1x, const void* J1r,
                        const void* J1p) {
    CTH_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (m->rect) {
        const int rc = rect_lists(m, prm, s);
        if (rc != CTH_OK) return rc;
    } else if (!m->has_bc) {
        set_error("cth_mw3_assemble_dev: boundary lists not set (cth_mw3_set_boundary)");
        return CTH_ERR_ARG;
    }
    Dev3 D = dev3(m);
    dim3 blk(128), grd((m->ni + 127) / 128, m->nj);
    k_m3_assemble<<<grd, blk, 0, s>>>(ne, nu, Bx, Br, epsr, *prm, D, static_cast<const cd*>(J1x),
                                      static_cast<const cd*>(J1r), static_cast<const cd*>(J1p));
    m->launches++;
    // the lists in the reference's order; entries of one list are distinct rows
    for (int L = 0; L < 12; L++) {
        if (m->cnt[L] == 0) continue;
        k_m3_bc<<<(m->cnt[L] + 127) / 128, 128, 0, s>>>(D, m->lst + 3 * (size_t)m->off[L], m->cnt[L], L, epsr, *prm,
                                                         m->jflc);
        m->launches++;
    }
    CTH_CUDA(cudaGetLastError());
    m->assembled = true;
    return CTH_OK;
}

static bool mw3_params_ok(const cth_mw_params* prm) {
    return prm->dx > 0.0 && prm->dr > 0.0 && prm->rmin == 0.0 && prm->r2 > prm->r1 && prm->r1 > 0.0 &&
           prm->omegam > 0.0 && prm->masse > 0.0;
}

int cth_mw3_assemble_dev(cth_mw3* m, const double* ne, const double* nu, const double* Bx, const double* Br,
                         const double* epsr, const cth_mw_params* prm, void* stream) {
    if (!m || !ne || !nu || !Bx || !Br || !epsr || !prm || !mw3_params_ok(prm)) {
        set_error("cth_mw3_assemble_dev: invalid arguments (the domain starts on the axis: rmin = 0)");
        return CTH_ERR_ARG;
    }
    return mw3_assemble(m, ne, nu, Bx, Br, epsr, prm, stream, nullptr, nullptr, nullptr);
}

int cth_mw3_assemble_explicit_dev(cth_mw3* m, const double* epsr, const void* J1x, const void* J1r,
                                  const void* J1p, const cth_mw_params* prm, void* stream) {
    if (!m || !epsr || !J1x || !J1r || !J1p || !prm || !mw3_params_ok(prm)) {
        set_error("cth_mw3_assemble_explicit_dev: invalid arguments (the domain starts on the axis: rmin = 0)");
        return CTH_ERR_ARG;
    }
    return mw3_assemble(m, nullptr, nullptr, nullptr, nullptr, epsr, prm, stream, J1x, J1r, J1p);
}

int cth_mw3_apply_dev(cth_mw3* m, const double* x3, double* y3, void* stream) {
    if (!m || !x3 || !y3 || !m->assembled) {
        set_error("cth_mw3_apply_dev: invalid arguments or system not assembled");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = (cudaStream_t)stream;
    Dev3 D = dev3(m);
    dim3 blk(128), grd((m->ld + 127) / 128, m->nj + 2);
    k_m3_mask<<<grd, blk, 0, s>>>(D, reinterpret_cast<const cd*>(x3), m->tmp);
    k_m3_apply<<<grd, blk, 0, s>>>(D, m->tmp, reinterpret_cast<cd*>(y3));
    m->launches += 2;
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

int cth_mw3_set_cycle(cth_mw3* m, int nu_pre, int nu_post) {
    if (!m || nu_pre < 1 || nu_post < 1 || nu_pre > 8 || nu_post > 8) {
        set_error("cth_mw3_set_cycle: sweeps must be in 1..8");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    CTH_CUDA(cudaDeviceSynchronize());
    for (int c = 0; c < 3; c++) {
        m->g[c]->nu1 = nu_pre;
        m->g[c]->nu2 = nu_post;
    }
    // the captured solve holds the old cycle: capture again on the next solve
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
    return CTH_OK;
}

int cth_mw3_set_preconditioner(cth_mw3* m, int mode) {
    if (!m || mode < 0 || mode > 1) {
        set_error("cth_mw3_set_preconditioner: mode 0 (block Jacobi) or 1 (block Gauss-Seidel)");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    CTH_CUDA(cudaDeviceSynchronize());
    m->gauss_seidel = mode == 1;
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
    return CTH_OK;
}

int cth_mw3_set_precision(cth_mw3* m, int precision) {
    if (!m || (precision != CTH_PREC_FP64 && precision != CTH_PREC_MIXED)) {
        set_error("cth_mw3_set_precision: CTH_PREC_FP64 or CTH_PREC_MIXED");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    CTH_CUDA(cudaDeviceSynchronize());
    if (precision == CTH_PREC_MIXED)
        for (int c = 0; c < 3; c++) {
            const int rc = cmg32_alloc(m->g[c]);
            if (rc != CTH_OK) return rc;
        }
    m->precision = precision;
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
    return CTH_OK;
}

int cth_mw3_set_graphs(cth_mw3* m, int enable) {
    if (!m) {
        set_error("cth_mw3_set_graphs: null handle");
        return CTH_ERR_ARG;
    }
    m->use_graphs = enable != 0;
    return CTH_OK;
}

int cth_mw3_fill_ghosts(cth_mw3* m, double* E3, const double* epsr, const double* Er_dc, const cth_mw_params* prm,
                        void* stream) {
    if (!m || !E3 || !epsr || !prm || prm->dx <= 0.0 || prm->dr <= 0.0 || prm->rmin != 0.0 || prm->omegam <= 0.0) {
        set_error("cth_mw3_fill_ghosts: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (m->rect) {
        const int rc = rect_lists(m, prm, s);
        if (rc != CTH_OK) return rc;
    } else if (!m->has_bc) {
        set_error("cth_mw3_fill_ghosts: boundary lists not set (cth_mw3_set_boundary)");
        return CTH_ERR_ARG;
    }
    if (!m->ghosts_ok) {
        set_error("cth_mw3_fill_ghosts: a boundary list writes a ghost onto an unknown of its field");
        return CTH_ERR_UNSUPPORTED;
    }
    if (m->needs_er_dc && !Er_dc) {
        set_error("cth_mw3_fill_ghosts: the Er east list has code-1 entries, which read gr.Er (Er_dc)");
        return CTH_ERR_ARG;
    }
    for (int L = 0; L < 12; L++) {
        if (m->cnt[L] == 0) continue;
        k_m3_ghost<<<(m->cnt[L] + 127) / 128, 128, 0, s>>>(m->lst + 3 * (size_t)m->off[L], m->cnt[L], L,
                                                           reinterpret_cast<cd*>(E3), Er_dc, epsr, *prm, m->jflc,
                                                           m->ld, m->pl);
        m->launches++;
    }
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

int cth_mw3_solve_guess_dev(cth_mw3* m, int maxit, double tol, double* E3, const double* x0, double guess_tol,
                            void* stream, cth_status* st) {
    if (!m || !E3 || maxit < 0 || !(tol > 0.0) || !m->assembled || (x0 && !(guess_tol >= 0.0))) {
        set_error("cth_mw3_solve_dev: invalid arguments or system not assembled");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(m->device));
    cudaStream_t s = (cudaStream_t)stream;
    m->h_args->maxit = maxit;
    m->h_args->tol = tol;
    m->h_args->out = reinterpret_cast<cd*>(E3);
    m->h_args->x0 = reinterpret_cast<const cd*>(x0);
    m->h_args->guess_tol = guess_tol;
    CTH_CUDA(cudaMemcpyAsync(m->d_args, m->h_args, sizeof(Args3), cudaMemcpyHostToDevice, s));
    if (m->use_graphs) {
        int rc = build_graph(m);
        if (rc != CTH_OK) return rc;
        CTH_CUDA(cudaGraphLaunch(m->exec, s));
        CTH_CUDA(cudaMemcpyAsync(m->h_sc, m->sc, NWORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        m->launches += m->n_pre + (long long)m->n_body * (long long)m->h_sc[ITER] + m->n_post;
    } else {
        int n = 0;
        CTH_CUDA(solve_pre(m, s, 0, 0, &n));
        m->launches += n;
        for (;;) {
            CTH_CUDA(cudaMemcpyAsync(m->h_sc, m->sc, NWORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
            CTH_CUDA(cudaStreamSynchronize(s));
            if (m->h_sc[KEEP] == 0.0) break;
            n = 0;
            CTH_CUDA(solve_body(m, s, 0, 0, &n));
            m->launches += n;
        }
        m->launches += solve_post(m, s);
        CTH_CUDA(cudaStreamSynchronize(s));
    }
    CTH_CUDA(cudaGetLastError());
    const double* h = m->h_sc;
    cth_status loc{};
    loc.iterations = (int)h[ITER];
    loc.residual = h[RELRES];
    loc.initial_residual = std::sqrt(h[BB]);
    loc.converged = h[CONV] != 0.0;
    loc.nonfinite = h[BAD] != 0.0 && !loc.converged;
    loc.guess = h[GUESS] >= 1.0 ? 1 : (h[GUESS] <= -1.0 ? -1 : 0);
    loc.guess_residual = loc.guess == 0 ? -1.0 : std::fabs(h[GUESS]) - 1.0;
    if (st) *st = loc;
    if (loc.nonfinite) return CTH_NONFINITE;
    return loc.converged ? CTH_OK : CTH_NOT_CONVERGED;
}

int cth_mw3_solve_dev(cth_mw3* m, int maxit, double tol, double* E3, void* stream, cth_status* st) {
    return cth_mw3_solve_guess_dev(m, maxit, tol, E3, nullptr, 0.0, stream, st);
}

}  // extern "C"
