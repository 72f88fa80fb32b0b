// sg_pc.cu — the Scharfetter-Gummel predictor-correctors of FluidModule on the
// device: electron density (solve_rhoe_wdTe_wSEE_PC, fluidModule.hpp:3082-3970)
// and electron energy (solve_Te_wdTe_wSEE_PC, fluidModule.hpp:4006-4957).
//
// Both advance a conserved density n (rhoe or rhoeps = 3/2 n k Te) with face
// fluxes F = A(z) n_L - B(z) n_R (+ the inverse-mobility relaxation of the old
// flux), A = vd/(1 - e^-z), B = vd/(e^z - 1), z = vd h / D (exponent clipped at
// 100), the energy flux carrying a factor 5/3.  Wall faces get the thermal + SEE
// flux, the open top the ion flux (density) or the convected enthalpy (energy).
// The implicit increment system (no wall folding: the walls enter through the
// cleared side flags and the wall fluxes on the right-hand side) is solved by
// the MG (or SOR) replacement; the fluxes are corrected with the same weights
// and n takes the increment where the result stays positive.
//
// Per PC iteration: save, predict (faces), assemble (cells), solve, correct
// (faces and cells + calcRes reductions, the anode current of the density
// sweep).  After the loop: ghost rules of rhoe, or the Te recovery
// (fluidModule.hpp:4843-4876) and the ghost rules of Te.
#include <cuda_runtime.h>

#include <cmath>

#include "fluid.cuh"

namespace cth {

struct SgArgs {
    double *n, *Fx, *Fr, *Fx_w, *Fr_w;
    double *n_old, *Fx_old, *Fr_old, *n_t, *Fx_t, *Fr_t, *d;
    double *Te, *Te_old;            // density sweep: Te_old == Te (not written)
    const double* rhoe_old_see;     // rhoe at the start of the density sweep
    const double *mu_para, *mu_perp, *mu_rr, *mu_xr, *mu_xx, *Ex, *Er, *rhoi, *Uix, *Uir, *rhoUmx, *rhoUmr;
    const double *rate_ionize, *rhoUix_wall;                     // density
    const double *rhoe, *rhoUex, *rhoUer, *Pabs, *rate_eloss;    // energy
    double *aP, *aE, *aW, *aN, *aS, *b;
    const unsigned char* flags;
    Tab eb, rd, ts;
    cth_sg_params prm;
    int ni, nj, ld;
    int nkw;                               // energy sweep: r-face boxes whose Gr_wall is kept
    int kw[4 * CTH_KEEP_WALL_MAX];
};

#define FL(ii, jj) flag_at(A.flags, (ii), (jj), A.ni, A.nj, A.ld)

constexpr double kLimExp = 1.0e2;  // fluidModule.hpp:3099
constexpr double kEpsVd = 1.0e-3;  // fluidModule.hpp:3100

template <bool EN>
__global__ void k_sg_begin(SgArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    const double v = A.n[p];
    A.n_old[p] = v;
    A.Fx_old[p] = A.Fx[p];
    A.Fr_old[p] = A.Fr[p];
    if (EN) A.Te_old[p] = A.Te[p];
    A.d[p] = v - v;
}

__global__ void k_sg_save(SgArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    A.n_t[p] = A.n[p];
    A.Fx_t[p] = A.Fx[p];
    A.Fr_t[p] = A.Fr[p];
}

// SG weights of the face between cells c0 (low side) and c1 (high side)
struct SgFace {
    double mst, vd, da, db;  // A = vd / da, B = vd / db
    __device__ double A() const { return vd / da; }
    __device__ double B() const { return vd / db; }
};

__device__ __forceinline__ SgFace sg_face(const SgArgs& A, size_t c0, size_t c1, double E, double h) {
    const double* T = A.Te_old;
    SgFace f;
    // mobility and old temperature are inputs of every kernel that calls this:
    // read-only loads, which the compiler may issue ahead of the kernel's stores
    const double m1 = __ldg(A.mu_perp + c1), m0 = __ldg(A.mu_perp + c0);
    const double T1 = __ldg(T + c1), T0 = __ldg(T + c0);
    f.mst = (m1 + m0) / 2.0 * 1.0;
    const double Tt = (T1 + T0) / 2.0;
    const double dT = (T1 - T0) / h;
    f.vd = f.mst * (-E - kBoltz / kE0f * dT) + kEpsVd;
    const double D = kBoltz * Tt / kE0f * f.mst;
    const double z = f.vd * h / D;
    f.da = 1.0 - exp(fmin(-z, kLimExp));
    f.db = exp(fmin(z, kLimExp)) - 1.0;
    return f;
}

// wall flux of cell c through face f; sign -1 on the low side, +1 on the high side
// density: fluidModule.hpp:3247-3370, :3453-3527; energy: :4170-4309, :4398-4490
template <bool EN>
__device__ __forceinline__ double sg_wall(const SgArgs& A, size_t c, double E, double Ui, double rhoUm, double h,
                                          double sign) {
    const cth_sg_params& P = A.prm;
    const double Tv = A.Te_old[c];
    const double Te = A.Te[c];
    const double vth = sqrt(8.0 * kBoltz * Tv / (M_PI * P.masse));
    const double delta_phi = fmax(sign * E * h / 2.0, 0.0);
    const double ex = exp(fmin(-kE0f * delta_phi / (kBoltz * Tv + 1e-100), kLimExp));
    const double ceb = d_func_Te(A.eb.v, A.eb.n, Te, P.dTe_SEE);
    const double crd = d_func_Te(A.rd.v, A.rd.n, Te, P.dTe_SEE);
    const double cts = d_func_Te(A.ts.v, A.ts.n, Te, P.dTe_SEE);
    const double gpn = sign * 0.25 * 1.0 * vth * ex;
    if (!EN) {
        const double see =
            -P.coefIISEE_ts * A.rhoi[c] * Ui - (ceb + crd + cts) * A.n_old[c] * gpn - P.coefMISEE_ts * rhoUm;
        return A.n[c] * gpn + see;
    }
    const double gpn_eps = sign * vth * ex / 3.0 * 1.0;
    const double eps_emit = 2.0 * kE0f * P.Te_emitSEE_eV;
    const double see = -eps_emit * P.coefIISEE_ts * A.rhoi[c] * Ui -
                       (ceb + P.ratioEngy_EISEE_rd * crd) * A.n_old[c] * gpn_eps -
                       eps_emit * cts * A.rhoe_old_see[c] * gpn - eps_emit * P.coefMISEE_ts * rhoUm;
    return A.n[c] * gpn_eps + see;
}

template <bool EN>
__device__ __forceinline__ void sg_predict_cell(const SgArgs& A, int i, int j) {
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const cth_sg_params& P = A.prm;
    const double dx = P.dx, dr = P.dr;
    const double rj = P.rmin + (j - 0.5) * dr;
    const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
    const double fac = EN ? 5.0 : 1.0;
    // the fluxes of the last corrector, mobilities, fields, density and ion / neutral
    // fluxes are read only here (the kernel writes Fx, Fr and the wall fluxes):
    // read-only loads, free to move ahead of the stores

    // x face i-1/2
    double vx = __ldg(A.Fx_t + p);
    if (fc && fw) {
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double mpa = (__ldg(A.mu_para + p) + __ldg(A.mu_para + p - 1)) / 2.0;
        const double mpe = (__ldg(A.mu_perp + p) + __ldg(A.mu_perp + p - 1)) / 2.0;
        const double mrr = (__ldg(A.mu_rr + p) + __ldg(A.mu_rr + p - 1)) / 2.0;
        const double mxr = (__ldg(A.mu_xr + p) + __ldg(A.mu_xr + p - 1)) / 2.0;
        const double ixx = mrr / (mpa * mpe);
        const double ixr = -mxr / (mpa * mpe);
        const SgFace f = sg_face(A, p - 1, p, __ldg(A.Ex + p), dx);
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bLrD = ((fw & F_BLR_WALL) && (fw & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = (fc & F_BRR_WALL) ? 1.0 : 0.0;
        const double bRrD = (fw & F_BRR_WALL) ? 1.0 : 0.0;
        const double Fr_i = (rR * __ldg(A.Fr_t + p + ld) * bRr + rL * __ldg(A.Fr_t + p) * bLr + rR * __ldg(A.Fr_t + p - 1 + ld) * bRrD +
                             rL * __ldg(A.Fr_t + p - 1) * bLrD) /
                            (4.0 * rj);
        const double sg = EN ? (f.A() * __ldg(A.n + p - 1) - f.B() * __ldg(A.n + p)) * fac / 3.0 : f.A() * __ldg(A.n + p - 1) - f.B() * __ldg(A.n + p);
        vx = sg + __ldg(A.Fx_t + p) - f.mst * (ixx * __ldg(A.Fx_t + p) + ixr * Fr_i);
    }
    if (fc && !(fc & F_BLX)) {
        vx = sg_wall<EN>(A, p, __ldg(A.Ex + p), __ldg(A.Uix + p), __ldg(A.rhoUmx + p), dx, -1.0);
        A.Fx_w[p] = vx;
    }
    if (fw && !(fw & F_BRX)) {
        vx = sg_wall<EN>(A, p - 1, __ldg(A.Ex + p), __ldg(A.Uix + p), __ldg(A.rhoUmx + p), dx, 1.0);
        A.Fx_w[p] = vx;
    }
    A.Fx[p] = vx;

    // r face j-1/2
    double vr = __ldg(A.Fr_t + p);
    if (fc && fs) {
        const double rjm = P.rmin + (j - 1.5) * dr;
        const double r_t = (rj + rjm) / 2.0;
        const double mpa = (__ldg(A.mu_para + p) + __ldg(A.mu_para + p - ld)) / 2.0;
        const double mpe = (__ldg(A.mu_perp + p) + __ldg(A.mu_perp + p - ld)) / 2.0;
        const double mxx = (__ldg(A.mu_xx + p) + __ldg(A.mu_xx + p - ld)) / 2.0;
        const double mxr = (__ldg(A.mu_xr + p) + __ldg(A.mu_xr + p - ld)) / 2.0;
        const double irr = mxx / (mpa * mpe);
        const double ixr = -mxr / (mpa * mpe);
        const SgFace f = sg_face(A, p - ld, p, __ldg(A.Er + p), dr);
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bLxD = (fs & F_BLX) ? 1.0 : 0.0;
        const double bRx = (fc & F_BRX) ? 1.0 : 0.0, bRxD = (fs & F_BRX) ? 1.0 : 0.0;
        const double Fx_i = (rj * __ldg(A.Fx_t + p + 1) * bRx + rj * __ldg(A.Fx_t + p) * bLx + rjm * __ldg(A.Fx_t + p + 1 - ld) * bRxD +
                             rjm * __ldg(A.Fx_t + p - ld) * bLxD) /
                            (4.0 * r_t);
        const double sg = EN ? (f.A() * __ldg(A.n + p - ld) - f.B() * __ldg(A.n + p)) * fac / 3.0 : f.A() * __ldg(A.n + p - ld) - f.B() * __ldg(A.n + p);
        vr = sg + __ldg(A.Fr_t + p) - f.mst * (ixr * Fx_i + irr * __ldg(A.Fr_t + p));
    }
    bool rec = true;  // energy sweep: the lower wall x2 sets Gr but not Gr_wall (fluidModule.hpp:4428-4449)
    if (EN)
        for (int q = 0; q < A.nkw; q++)
            if (i >= A.kw[4 * q] && i <= A.kw[4 * q + 1] && j >= A.kw[4 * q + 2] && j <= A.kw[4 * q + 3]) rec = false;
    if (fc && !(fc & F_BLR_WALL)) {
        vr = sg_wall<EN>(A, p, __ldg(A.Er + p), __ldg(A.Uir + p), __ldg(A.rhoUmr + p), dr, -1.0);
        if (rec) A.Fr_w[p] = vr;
    }
    if (fs && !(fs & F_BRR_WALL)) {
        vr = sg_wall<EN>(A, p - ld, __ldg(A.Er + p), __ldg(A.Uir + p), __ldg(A.rhoUmr + p), dr, 1.0);
        if (rec) A.Fr_w[p] = vr;
    }
    if (fs && !(fs & F_BRR_OPEN)) {
        vr = EN ? 5.0 / 2.0 * kBoltz * A.Te_old[p - ld] * fmax(A.rhoUer[p], 0.0) : A.rhoi[p - ld] * __ldg(A.Uir + p);
        A.Fr_w[p] = 0.0;
    }
    A.Fr[p] = vr;
}

// kSweepCells cells of a row per thread: consecutive in the prediction (measured
// faster there), warp-strided (warp_strided_first) in the assembly
constexpr int kSweepCells = 4;

template <bool EN>
__global__ void k_sg_predict(SgArgs A) {
    const int i0 = kSweepCells * (blockIdx.x * blockDim.x + threadIdx.x);
#pragma unroll
    for (int k = 0; k < kSweepCells; k++) sg_predict_cell<EN>(A, i0 + k, blockIdx.y);
}

template <bool EN>
__device__ __forceinline__ void sg_assemble_cell(const SgArgs& A, int i, int j) {
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    // inputs through read-only loads (the kernel writes only the coefficient planes), so
    // the compiler may issue the next cell's loads ahead of this cell's stores
    double vP = 0.0, vE = 0.0, vW = 0.0, vN = 0.0, vS = 0.0, vb = 0.0;
    if (fc) {
        const cth_sg_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt = P.dt;
        const double rj = P.rmin + (j - 0.5) * dr;
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double rR = (rj + rjp) / 2.0, rL = (rj + rjm) / 2.0;
        const double qR = (rj + rjp) / 2.0 / rj;
        const double qL = (rj + rjm) / 2.0 / rj;
        const SgFace Lx = sg_face(A, p - 1, p, __ldg(A.Ex + p), dx);
        const SgFace Rx = sg_face(A, p, p + 1, __ldg(A.Ex + p + 1), dx);
        const SgFace Lr = sg_face(A, p - ld, p, __ldg(A.Er + p), dr);
        const SgFace Rr = sg_face(A, p, p + ld, __ldg(A.Er + p + ld), dr);
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bRx = (fc & F_BRX) ? 1.0 : 0.0;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = ((fc & F_BRR_WALL) && (fc & F_BRR_OPEN)) ? 1.0 : 0.0;
        const double tterm = EN ? 3.0 / 5.0 * dx * dr / dt : dx * dr / dt;
        vP = Rx.vd / Rx.da * bRx * dr + Lx.vd / Lx.db * bLx * dr + qR * Rr.vd / Rr.da * bRr * dx +
             qL * Lr.vd / Lr.db * bLr * dx + tterm;
        vE = Rx.vd / Rx.db * bRx * dr;
        vW = Lx.vd / Lx.da * bLx * dr;
        vN = qR * Rr.vd / Rr.db * bRr * dx;
        vS = qL * Lr.vd / Lr.da * bLr * dx;
        const double div = (__ldg(A.Fx + p + 1) - __ldg(A.Fx + p)) / dx + (qR * __ldg(A.Fr + p + ld) - qL * __ldg(A.Fr + p)) / dr;
        if (EN) {
            const double bRxw = bRx, bLxw = bLx;
            const double bLrw = (fc & F_BLR_WALL) ? 1.0 : 0.0, bRrw = (fc & F_BRR_WALL) ? 1.0 : 0.0;
            const double jx = -kE0f * (__ldg(A.rhoUex + p + 1) * __ldg(A.Ex + p + 1) * bRxw + __ldg(A.rhoUex + p) * __ldg(A.Ex + p) * bLxw) / 2.0;
            const double jr = -kE0f * (rR * __ldg(A.rhoUer + p + ld) * __ldg(A.Er + p + ld) * bRrw + rL * __ldg(A.rhoUer + p) * __ldg(A.Er + p) * bLrw) /
                              (2.0 * rj);
            const double R1 = (-__ldg(A.n + p) + __ldg(A.n_old + p)) / dt;
            const double R3 = __ldg(A.Pabs + p) - __ldg(A.rhoe + p) * __ldg(A.rate_eloss + p);
            vb = 3.0 / 5.0 * (R1 + (jx + jr) + R3 + (-div)) * dx * dr;
        } else {
            vb = (-div + __ldg(A.rate_ionize + p) - (__ldg(A.n + p) - __ldg(A.n_old + p)) / dt) * dx * dr;
        }
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

template <bool EN>
__global__ void k_sg_assemble(SgArgs A) {
    const int i0 = warp_strided_first(kSweepCells);
#pragma unroll
    for (int k = 0; k < kSweepCells; k++) sg_assemble_cell<EN>(A, i0 + 32 * k, blockIdx.y);
}

constexpr int kSgStat = 14;  // calcRes pairs (n, Fx, Fr) x (iteration, call) + anode Ii, Ie

// kCorrCells consecutive cells of a row per thread (measured faster here than the
// warp-strided order): a block covers kCorrCells x blockDim cells, so the
// deterministic reduction's per-block tree and its last-block combine (one partial
// per block and statistic) stay short
constexpr int kCorrCells = 4;

template <bool EN>
__global__ void __launch_bounds__(256, 3) k_sg_correct(SgArgs A, double* __restrict__ part, unsigned int* counter,
                                                       double* __restrict__ out) {
    const int i0 = kCorrCells * (blockIdx.x * blockDim.x + threadIdx.x);
    const int j = blockIdx.y;
    const int mode = A.prm.flag_error;
    double s[kSgStat];
#pragma unroll
    for (int k = 0; k < kSgStat; k++) s[k] = 0.0;
#pragma unroll
    for (int kc = 0; kc < kCorrCells; kc++) {
        const int i = i0 + kc;
        if (i > A.ni + 1) break;
        const int ld = A.ld;
        const size_t p = (size_t)j * ld + i;
        const double dx = A.prm.dx, dr = A.prm.dr;
        const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
        // d, E and the reference copies are not written here: read-only loads
        const double dc = __ldg(A.d + p);
        if (fc && fw) {
            const SgFace f = sg_face(A, p - 1, p, __ldg(A.Ex + p), dx);
            const double dw = __ldg(A.d + p - 1);
            const double dF = EN ? (f.A() * dw - f.B() * dc) * 5.0 / 3.0 : f.A() * dw - f.B() * dc;
            const double v = A.Fx[p] + dF;
            A.Fx[p] = v;
            res_acc(mode, v, __ldg(A.Fx_t + p), s[2], s[3]);
            res_acc(mode, v, __ldg(A.Fx_old + p), s[8], s[9]);
        }
        if (fc && fs) {
            const SgFace f = sg_face(A, p - ld, p, __ldg(A.Er + p), dr);
            const double ds = __ldg(A.d + p - ld);
            const double dF = EN ? (f.A() * ds - f.B() * dc) * 5.0 / 3.0 : f.A() * ds - f.B() * dc;
            const double v = A.Fr[p] + dF;
            A.Fr[p] = v;
            res_acc(mode, v, __ldg(A.Fr_t + p), s[4], s[5]);
            res_acc(mode, v, __ldg(A.Fr_old + p), s[10], s[11]);
        }
        if (fc) {
            double v = A.n[p];
            const double nn = v + dc;
            if (nn > 0.0) {
                v = nn;
                A.n[p] = v;
            }
            res_acc(mode, v, __ldg(A.n_t + p), s[0], s[1]);
            res_acc(mode, v, __ldg(A.n_old + p), s[6], s[7]);
            if (!EN && (fc & F_BRX_BIAS)) {
                const double rj = A.prm.rmin + (j - 0.5) * dr;
                s[12] += A.rhoUix_wall[p + 1] * 2.0 * M_PI * rj * dr * (kE0f);
                s[13] += A.Fx_w[p + 1] * 2.0 * M_PI * rj * dr * (-kE0f);
            }
        }
    }
    grid_reduce<kSgStat>(s, (mode == 0 || mode == 2) ? 0xfffu : 0u, part, counter, out);
}

// energy sweep epilogue (fluidModule.hpp:4843-4876): positivity of rhoeps,
// Te = rhoeps / (3/2 (rhoe + 1e-3 max rhoe) k) capped at 1000 eV, and the
// calcRes of rhoeps against its entry value
__global__ void k_te_recover(SgArgs A, const double* __restrict__ rhoe_max, double* __restrict__ part,
                             unsigned int* counter, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int mode = A.prm.flag_error;
    double s[2] = {0.0, 0.0};
    if (i <= A.ni + 1) {
        const size_t p = (size_t)j * A.ld + i;
        if (FL(i, j)) {
            double v = A.n[p];
            if (v < 0.0) {
                v = fmax(A.n_old[p], 0.0);
                A.n[p] = v;
            }
            const double Te_max = 1000.0 * kE0f / kBoltz;
            A.Te[p] = fmin(v / (3.0 / 2.0 * (A.rhoe[p] + *rhoe_max * 0.001) * kBoltz + 1e-100), Te_max);
            res_stat(mode, v, A.n_old[p], s[0], s[1]);
        }
    }
    grid_reduce<2>(s, (mode == 0 || mode == 2) ? 0x3u : 0u, part, counter, out);
}

#undef FL

template <bool EN>
static int solve_sg_pc(cth_fields* fs, const cth_sg_params* prm, cudaStream_t s, cth_pc_result* res) {
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_solve_sg_pc: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    SgArgs A{};
    const char* nk = EN ? "rhoeps" : "rhoe";
    const char* fxk = EN ? "Gx" : "rhoUex";
    const char* frk = EN ? "Gr" : "rhoUer";
    const std::string sn(nk), sx(fxk), sr(frk);
    struct { std::string name; double** dst; } rw[] = {
        {sn, &A.n}, {sx, &A.Fx}, {sr, &A.Fr}, {sx + "_wall", &A.Fx_w}, {sr + "_wall", &A.Fr_w},
        {sn + "_old", &A.n_old}, {sx + "_old", &A.Fx_old}, {sr + "_old", &A.Fr_old}, {"pc_n_t", &A.n_t},
        {"pc_Fx_t", &A.Fx_t}, {"pc_Fr_t", &A.Fr_t}, {"pc_d", &A.d}, {"Te", &A.Te},
        {EN ? "Te_old" : "Te", &A.Te_old}, {"pc_aP", &A.aP}, {"pc_aE", &A.aE}, {"pc_aW", &A.aW}, {"pc_aN", &A.aN},
        {"pc_aS", &A.aS}, {"pc_b", &A.b}};
    for (auto& e : rw) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    struct { const char* name; const double** dst; } ro[] = {
        {"mu_para", &A.mu_para}, {"mu_perp", &A.mu_perp}, {"mu_rr", &A.mu_rr}, {"mu_xr", &A.mu_xr},
        {"mu_xx", &A.mu_xx}, {"Ex", &A.Ex}, {"Er", &A.Er}, {"rhoi", &A.rhoi}, {"Uix", &A.Uix}, {"Uir", &A.Uir},
        {"rhoUmx", &A.rhoUmx}, {"rhoUmr", &A.rhoUmr}, {"rate_ionize", &A.rate_ionize},
        {"rhoUix_wall", &A.rhoUix_wall}, {"rhoe", &A.rhoe}, {"rhoUex", &A.rhoUex}, {"rhoUer", &A.rhoUer},
        {"Pabs", &A.Pabs}, {"rate_eloss", &A.rate_eloss}, {"rhoe_old", &A.rhoe_old_see}};
    for (auto& e : ro) {
        double* q = field_ptr(fs, e.name);
        if (!q) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
        *e.dst = q;
    }
    bool ok = true;
    A.eb = table(fs, "coefEISEE_eb_table", &ok);
    A.rd = table(fs, "coefEISEE_rd_table", &ok);
    A.ts = table(fs, "coefEISEE_ts_table", &ok);
    if (!ok) {
        set_error("cth_solve_sg_pc: SEE tables missing (coefEISEE_eb_table, coefEISEE_rd_table, coefEISEE_ts_table)");
        return CTH_ERR_ARG;
    }
    A.flags = fs->flags;
    A.prm = *prm;
    A.nkw = fs->n_keep_wall;
    for (int q = 0; q < 4 * CTH_KEEP_WALL_MAX; q++) A.kw[q] = fs->keep_wall[q];
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    const int nb = grd.x * grd.y;
    if ((size_t)nb * kSgStat > (size_t)fs->npart) {
        set_error("cth_solve_sg_pc: reduction scratch too small");
        return CTH_ERR_ARG;
    }
    double* out = fs->scal + 16;
    k_sg_begin<EN><<<grd, blk, 0, s>>>(A);
    g->launches++;
    int ncount = 0, solver_rc = 0;
    double e_it[3] = {0, 0, 0}, e_call[3] = {0, 0, 0}, cur[2] = {0, 0};
    cth_status st_last{};
    const int m = prm->flag_error;
    for (;;) {
        ncount++;
        k_sg_save<<<grd, blk, 0, s>>>(A);
        const dim3 grd4((g->ni + 2 + 128 * kSweepCells - 1) / (128 * kSweepCells), g->nj + 2);
        k_sg_predict<EN><<<grd4, blk, 0, s>>>(A);
        k_sg_assemble<EN><<<grd4, blk, 0, s>>>(A);
        g->launches += 3;
        CTH_CUDA(cudaGetLastError());
        int rc, pend = 0;
        if (prm->flag_iter == 0)
            rc = sor_solve_dev(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, 1.9, prm->maxITR_SOR, prm->error_cnv_SOR, A.d, s,
                               &st_last);
        else
            rc = smg_solve_launch(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                                  prm->precision, A.d, s, &pend, fs->h_solve, nullptr, 0.0, nullptr,
                                  EN == 0 ? SLOT_RHOE : SLOT_EPS);
        if (rc < 0) return rc;
        k_sg_correct<EN><<<dim3((g->ni + 2 + 256 * kCorrCells - 1) / (256 * kCorrCells), g->nj + 2), 256, 0, s>>>(
            A, fs->part, g->ws.counter, out);
        g->launches++;
        CTH_CUDA(cudaGetLastError());
        CTH_CUDA(cudaMemcpyAsync(fs->h_scal, out, kSgStat * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        if (pend) rc = solve_parse(g, pend, fs->h_solve, &st_last);
        if (rc < 0) return rc;
        if (rc > solver_rc) solver_rc = rc;
        const double* h = fs->h_scal;
        for (int k = 0; k < 3; k++) {
            e_it[k] = finish_res(m, h[2 * k], h[2 * k + 1]);
            e_call[k] = finish_res(m, h[6 + 2 * k], h[6 + 2 * k + 1]);
        }
        cur[0] = h[12];
        cur[1] = h[13];
        const double eg = fmax(fmax(e_it[0], e_it[1]), e_it[2]);
        if (eg < prm->error_cnv_HES || ncount >= prm->maxITR_HES) break;
    }
    if (EN) {
        k_max_flagged<<<grd, blk, 0, s>>>(A.rhoe, fs->flags, g->ni, g->nj, g->ld, fs->part, g->ws.counter,
                                          fs->scal + 32);
        k_te_recover<<<grd, blk, 0, s>>>(A, fs->scal + 32, fs->part, g->ws.counter, fs->scal + 34);
        g->launches += 2;
        apply_ghost_rules(fs, A.Te, 1, s);
        CTH_CUDA(cudaGetLastError());
        CTH_CUDA(cudaMemcpyAsync(fs->h_scal, fs->scal + 34, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        e_call[0] = finish_res(m, fs->h_scal[0], fs->h_scal[1]);
    } else {
        apply_ghost_rules(fs, A.n, 0, s);
        CTH_CUDA(cudaGetLastError());
    }
    if (res) {
        res->ncount = ncount;
        res->solver_rc = solver_rc;
        res->error_phi = e_call[0];
        res->error_nUex = e_call[1];
        res->error_nUer = e_call[2];
        for (int k = 0; k < 3; k++) res->error_iter[k] = e_it[k];
        res->solver = st_last;
        res->Ii_Anode = EN ? 0.0 : cur[0];
        res->Ie_Anode = EN ? 0.0 : cur[1];
        res->I_Anode = EN ? 0.0 : cur[0] + cur[1];
    }
    return CTH_OK;
}

}  // namespace cth

static bool sg_params_ok(const cth_sg_params* p) {
    return p && p->dx > 0.0 && p->dr > 0.0 && p->dt > 0.0 && p->maxITR_HES >= 1 && p->flag_error >= 0 &&
           p->flag_error <= 3;
}

extern "C" int cth_solve_rhoe_pc(cth_fields* fs, const cth_sg_params* prm, void* stream, cth_pc_result* res) {
    if (!fs || !sg_params_ok(prm)) {
        cth::set_error("cth_solve_rhoe_pc: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return cth::solve_sg_pc<false>(fs, prm, (cudaStream_t)stream, res);
}

extern "C" int cth_solve_Te_pc(cth_fields* fs, const cth_sg_params* prm, void* stream, cth_pc_result* res) {
    if (!fs || !sg_params_ok(prm)) {
        cth::set_error("cth_solve_Te_pc: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return cth::solve_sg_pc<true>(fs, prm, (cudaStream_t)stream, res);
}
