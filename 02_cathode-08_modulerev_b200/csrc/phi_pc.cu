// phi_pc.cu — FluidModule::solve_phi_couple_wdTe_wSEE_PC on the device
// (fluidModule.hpp:2080-3075).
//
// The potential is advanced by a predictor-corrector loop: the electron flux is
// predicted with the inverse mobility tensor, wall faces get the thermal + SEE
// flux, a Poisson equation with dielectric relaxation (face coefficient
// eps0 + e dt n mu_perp) is assembled for the potential increment, solved by
// the semicoarsening MG (or SOR), and the potential, the fields and the fluxes
// are corrected.  The reference visits the fluid blocks and then each named
// wall segment in a fixed order; here every kernel is one thread per (i, j) of
// the index space and the walls come from the per-cell side flags: a wall face
// is the face of a fluid cell whose flag bit is cleared, a ghost cell takes the
// value of the last wall segment the reference would have written (left, right,
// lower, upper, open in that order).
//
// Per PC iteration: save (3 planes), predict (faces), assemble (6 coefficient
// planes), solve, correct A (ghosts, potential, wall fields), correct B
// (interior fields and fluxes + the calcRes reductions).
#include <cuda_runtime.h>

#include <cmath>

#include "fluid.cuh"

namespace cth {

struct PhiArgs {
    double *phi, *Ex, *Er, *nUex, *nUer;
    double *phi_old, *Ex_old, *Er_old, *nUex_old, *nUer_old;
    double *phi_t, *nUex_t, *nUer_t, *dphi;
    const double *rhoe, *rhoe_old, *rhoi, *Te, *mu_para, *mu_perp, *mu_rr, *mu_xr, *mu_xx, *rate_ionize, *Uix,
        *Uir, *rhoUmx, *rhoUmr;
    double *aP, *aE, *aW, *aN, *aS, *b;
    const unsigned char* flags;
    Tab eb, rd, ts;
    cth_phi_params prm;
    int ni, nj, ld;
};

#define FL(ii, jj) flag_at(A.flags, (ii), (jj), A.ni, A.nj, A.ld)

// entry: keep the old values, zero the increment and set the wall ghosts of phi
// (fluidModule.hpp:2126-2240)
__global__ void k_phi_begin(PhiArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const double ph = A.phi[p];
    A.phi_old[p] = ph;
    A.Ex_old[p] = A.Ex[p];
    A.Er_old[p] = A.Er[p];
    A.nUex_old[p] = A.nUex[p];
    A.nUer_old[p] = A.nUer[p];
    A.dphi[p] = ph - ph;
    if (FL(i, j)) return;
    double v = ph;
    unsigned f = FL(i + 1, j);
    if (f && !(f & F_BLX)) v = -A.phi[p + 1];
    f = FL(i - 1, j);
    if (f && !(f & F_BRX)) v = (f & F_BRX_BIAS) ? 2.0 * A.prm.V_bias - A.phi[p - 1] : -A.phi[p - 1];
    f = FL(i, j + 1);
    if (f && !(f & F_BLR_WALL)) v = -A.phi[p + ld];
    f = FL(i, j - 1);
    if (f && !(f & F_BRR_WALL)) v = -A.phi[p - ld];
    if (f && !(f & F_BRR_OPEN)) v = A.phi[p - ld];
    A.phi[p] = v;
}

__global__ void k_phi_save(PhiArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    A.phi_t[p] = A.phi[p];
    A.nUex_t[p] = A.nUex[p];
    A.nUer_t[p] = A.nUer[p];
}

// thermal + secondary-emission electron flux through a wall face of a cell
// (fluidModule.hpp:2346-2457, :2543-2624); sign -1 on the low side, +1 on the high
__device__ __forceinline__ double wall_flux(const PhiArgs& A, size_t c, double E_old, double Ui, double rhoUm,
                                            double h, double sign) {
    const cth_phi_params& P = A.prm;
    const double Te = A.Te[c];
    const double vth = sqrt(8.0 * kBoltz * Te / (M_PI * P.masse));
    const double delta_phi = fmax(sign * E_old * h / 2.0, 0.0);
    const double gpn = sign * 0.25 * vth * exp(fmin(-kE0f * delta_phi / (kBoltz * Te + 1e-100), 100.0));
    const double ceb = d_func_Te(A.eb.v, A.eb.n, Te, P.dTe_SEE);
    const double crd = d_func_Te(A.rd.v, A.rd.n, Te, P.dTe_SEE);
    const double cts = d_func_Te(A.ts.v, A.ts.n, Te, P.dTe_SEE);
    const double see = -P.coefIISEE_ts * A.rhoi[c] * Ui - (ceb + crd + cts) * A.rhoe_old[c] * gpn -
                       P.coefMISEE_ts * rhoUm;
    return A.rhoe[c] * gpn + see;
}

// flux prediction on every face (fluidModule.hpp:2266-2633)
__global__ void k_phi_predict(PhiArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const cth_phi_params& P = A.prm;
    const double dx = P.dx, dr = P.dr;
    const double rj = P.rmin + (j - 0.5) * dr;
    const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);

    // x face i-1/2
    double vx = A.nUex_t[p];
    if (fc && fw) {
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double mpa = (A.mu_para[p] + A.mu_para[p - 1]) / 2.0;
        const double mpe = (A.mu_perp[p] + A.mu_perp[p - 1]) / 2.0;
        const double mst = mpe * 1.0;
        const double mrr = (A.mu_rr[p] + A.mu_rr[p - 1]) / 2.0;
        const double mxr = (A.mu_xr[p] + A.mu_xr[p - 1]) / 2.0;
        const double ixx = mrr / (mpa * mpe);
        const double ixr = -mxr / (mpa * mpe);
        const double rho_t = (A.rhoe[p] + A.rhoe[p - 1]) / 2.0;
        const double dphidx = (A.phi[p] - A.phi[p - 1]) / dx;
        const double dpedx = kBoltz * (A.rhoe[p] * A.Te[p] - A.rhoe[p - 1] * A.Te[p - 1]) / dx;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bLrD = ((fw & F_BLR_WALL) && (fw & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = (fc & F_BRR_WALL) ? 1.0 : 0.0;
        const double bRrD = (fw & F_BRR_WALL) ? 1.0 : 0.0;
        const double nUer_i = (rR * A.nUer_t[p + ld] * bRr + rL * A.nUer_t[p] * bLr +
                               rR * A.nUer_t[p - 1 + ld] * bRrD + rL * A.nUer_t[p - 1] * bLrD) /
                              (4.0 * rj);
        vx = A.nUex_t[p] - (ixx * A.nUex_t[p] + ixr * nUer_i) * mst + mst * (rho_t * dphidx - dpedx / kE0f);
    }
    if (fc && !(fc & F_BLX)) vx = wall_flux(A, p, A.Ex_old[p], A.Uix[p], A.rhoUmx[p], dx, -1.0);
    if (fw && !(fw & F_BRX)) vx = wall_flux(A, p - 1, A.Ex_old[p], A.Uix[p], A.rhoUmx[p], dx, 1.0);
    A.nUex[p] = vx;

    // r face j-1/2
    double vr = A.nUer_t[p];
    if (fc && fs) {
        const double rjm = P.rmin + (j - 1.5) * dr;
        const double r_t = (rj + rjm) / 2.0;
        const double mpa = (A.mu_para[p] + A.mu_para[p - ld]) / 2.0;
        const double mpe = (A.mu_perp[p] + A.mu_perp[p - ld]) / 2.0;
        const double mst = mpe * 1.0;
        const double mxx = (A.mu_xx[p] + A.mu_xx[p - ld]) / 2.0;
        const double mxr = (A.mu_xr[p] + A.mu_xr[p - ld]) / 2.0;
        const double irr = mxx / (mpa * mpe);
        const double ixr = -mxr / (mpa * mpe);
        const double rho_t = (A.rhoe[p] + A.rhoe[p - ld]) / 2.0;
        const double dphidr = (A.phi[p] - A.phi[p - ld]) / dr;
        const double dpedr = kBoltz * (A.rhoe[p] * A.Te[p] - A.rhoe[p - ld] * A.Te[p - ld]) / dr;
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bLxD = (fs & F_BLX) ? 1.0 : 0.0;
        const double bRx = (fc & F_BRX) ? 1.0 : 0.0, bRxD = (fs & F_BRX) ? 1.0 : 0.0;
        const double nUex_i = (rj * A.nUex_t[p + 1] * bRx + rj * A.nUex_t[p] * bLx +
                               rjm * A.nUex_t[p + 1 - ld] * bRxD + rjm * A.nUex_t[p - ld] * bLxD) /
                              (4.0 * r_t);
        vr = A.nUer_t[p] - (ixr * nUex_i + irr * A.nUer_t[p]) * mst + mst * (rho_t * dphidr - dpedr / kE0f);
    }
    if (fc && !(fc & F_BLR_WALL)) vr = wall_flux(A, p, A.Er_old[p], A.Uir[p], A.rhoUmr[p], dr, -1.0);
    if (fs && !(fs & F_BRR_WALL)) vr = wall_flux(A, p - ld, A.Er_old[p], A.Uir[p], A.rhoUmr[p], dr, 1.0);
    if (fs && !(fs & F_BRR_OPEN)) vr = A.rhoi[p - ld] * A.Uir[p];
    A.nUer[p] = vr;
}

// Poisson coefficients with dielectric relaxation and the wall conditions
// (fluidModule.hpp:2636-2816)
__global__ void k_phi_assemble(PhiArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    double vP = 0.0, vE = 0.0, vW = 0.0, vN = 0.0, vS = 0.0, vb = 0.0;
    if (fc) {
        const cth_phi_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt = P.dt;
        const double rj = P.rmin + (j - 0.5) * dr;
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double qR = (rj + rjp) / 2.0 / rj;
        const double qL = (rj + rjm) / 2.0 / rj;
        const double* mu = A.mu_perp;
        const double* n = A.rhoe;
        const double mLx = (mu[p] + mu[p - 1]) / 2.0 * 1.0, mRx = (mu[p] + mu[p + 1]) / 2.0 * 1.0;
        const double mLr = (mu[p] + mu[p - ld]) / 2.0 * 1.0, mRr = (mu[p] + mu[p + ld]) / 2.0 * 1.0;
        const double nLx = (n[p] + n[p - 1]) / 2.0, nRx = (n[p] + n[p + 1]) / 2.0;
        const double nLr = (n[p] + n[p - ld]) / 2.0, nRr = (n[p] + n[p + ld]) / 2.0;
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bRx = (fc & F_BRX) ? 1.0 : 0.0;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = ((fc & F_BRR_WALL) && (fc & F_BRR_OPEN)) ? 1.0 : 0.0;
        const double cRx = kEps0f + kE0f * dt * nRx * mRx * bRx, cLx = kEps0f + kE0f * dt * nLx * mLx * bLx;
        const double cRr = kEps0f + kE0f * dt * nRr * mRr * bRr, cLr = kEps0f + kE0f * dt * nLr * mLr * bLr;
        vP = (cRx + cLx) * dr * dr + (qR * cRr + qL * cLr) * dx * dx;
        vE = cRx * dr * dr;
        vW = cLx * dr * dr;
        vN = qR * cRr * dx * dx;
        vS = qL * cLr * dx * dx;
        const double div = (A.nUex[p + 1] - A.nUex[p]) / dx + (qR * A.nUer[p + ld] - qL * A.nUer[p]) / dr;
        const double lap = -(A.Ex[p + 1] - A.Ex[p]) / dx - (qR * A.Er[p + ld] - qL * A.Er[p]) / dr;
        vb = (kE0f * A.rhoi[p] - kE0f * n[p] - kE0f * dt * A.rate_ionize[p] + kEps0f * lap + kE0f * dt * div) *
             dx * dx * dr * dr;
        if (!(fc & F_BLX)) { vP = vP + vW; vW = 0.0; }
        if (!(fc & F_BRX)) { vP = vP + vE; vE = 0.0; }
        if (!(fc & F_BLR_WALL)) { vP = vP + vS; vS = 0.0; }
        if (!(fc & F_BRR_WALL)) { vP = vP + vN; vN = 0.0; }
        if (!(fc & F_BRR_OPEN)) { vP = vP - vN; vN = 0.0; }
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// ghost increments, potential update and wall fields (fluidModule.hpp:2836-2937)
__global__ void k_phi_correct_a(PhiArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    double d = A.dphi[p];
    if (!fc) {
        unsigned f = FL(i + 1, j);
        if (f && !(f & F_BLX)) d = -A.dphi[p + 1];
        f = FL(i - 1, j);
        if (f && !(f & F_BRX)) d = -A.dphi[p - 1];
        f = FL(i, j + 1);
        if (f && !(f & F_BLR_WALL)) d = -A.dphi[p + ld];
        f = FL(i, j - 1);
        if (f && !(f & F_BRR_WALL)) d = -A.dphi[p - ld];
        if (f && !(f & F_BRR_OPEN)) d = A.dphi[p - ld];
        A.dphi[p] = d;
    } else {
        const double dx = A.prm.dx, dr = A.prm.dr;
        if (!(fc & F_BLX)) A.Ex[p] = A.Ex[p] - (d - (-d)) / dx;
        if (!(fc & F_BRX)) A.Ex[p + 1] = A.Ex[p + 1] - ((-d) - d) / dx;
        if (!(fc & F_BLR_WALL)) A.Er[p] = A.Er[p] - (d - (-d)) / dr;
        if (!(fc & F_BRR_WALL)) A.Er[p + ld] = A.Er[p + ld] - ((-d) - d) / dr;
        if (!(fc & F_BRR_OPEN)) A.Er[p + ld] = 0.0;
    }
    A.phi[p] = A.phi[p] + d;
}

constexpr int kNStat = 12;  // (phi, nUex, nUer) x (vs iteration start, vs call start) x 2

// interior fields and flux corrections, then the residual reductions
// (fluidModule.hpp:2932-3046); the last block writes the 12 totals to out
// kCorrCells cells of a row per thread (warp-strided, warp_strided_first): a block
// covers kCorrCells x blockDim cells, so the deterministic reduction's per-block
// tree and its last-block combine (one partial per block and statistic) stay short
constexpr int kCorrCells = 4;

__global__ void k_phi_correct_b(PhiArgs A, double* __restrict__ part, unsigned int* counter,
                                double* __restrict__ out) {
    const int i0 = warp_strided_first(kCorrCells);
    const int j = blockIdx.y;
    const int mode = A.prm.flag_error;
    double s[kNStat];
#pragma unroll
    for (int k = 0; k < kNStat; k++) s[k] = 0.0;
#pragma unroll
    for (int kc = 0; kc < kCorrCells; kc++) {
        const int i = i0 + 32 * kc;
        if (i > A.ni + 1) break;
        const int ld = A.ld;
        const size_t p = (size_t)j * ld + i;
        const double dx = A.prm.dx, dr = A.prm.dr;
        const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
        // everything but Ex, Er, nUex, nUer is read only here: read-only loads, which the
        // compiler may issue ahead of this kernel's stores
        if (fc && fw) {
            A.Ex[p] = -(__ldg(A.phi + p) - __ldg(A.phi + p - 1)) / dx;
            const double mst = (__ldg(A.mu_perp + p) + __ldg(A.mu_perp + p - 1)) / 2.0 * 1.0;
            const double rho_t = (__ldg(A.rhoe + p) + __ldg(A.rhoe + p - 1)) / 2.0;
            const double v = A.nUex[p] + mst * rho_t * ((__ldg(A.dphi + p) - __ldg(A.dphi + p - 1)) / dx);
            A.nUex[p] = v;
            res_acc(mode, v, __ldg(A.nUex_t + p), s[2], s[3]);
            res_acc(mode, v, __ldg(A.nUex_old + p), s[8], s[9]);
        }
        if (fc && fs) {
            A.Er[p] = -(__ldg(A.phi + p) - __ldg(A.phi + p - ld)) / dr;
            const double mst = (__ldg(A.mu_perp + p) + __ldg(A.mu_perp + p - ld)) / 2.0 * 1.0;
            const double rho_t = (__ldg(A.rhoe + p) + __ldg(A.rhoe + p - ld)) / 2.0;
            const double v = A.nUer[p] + mst * rho_t * ((__ldg(A.dphi + p) - __ldg(A.dphi + p - ld)) / dr);
            A.nUer[p] = v;
            res_acc(mode, v, __ldg(A.nUer_t + p), s[4], s[5]);
            res_acc(mode, v, __ldg(A.nUer_old + p), s[10], s[11]);
        }
        if (fc) {
            const double v = __ldg(A.phi + p);
            res_acc(mode, v, __ldg(A.phi_t + p), s[0], s[1]);
            res_acc(mode, v, __ldg(A.phi_old + p), s[6], s[7]);
        }
    }
    grid_reduce<kNStat>(s, (mode == 0 || mode == 2) ? 0xfffu : 0u, part, counter, out);
}

#undef FL

int solve_phi_pc(cth_fields* fs, const cth_phi_params* prm, cudaStream_t s, cth_pc_result* res) {
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_solve_phi_pc: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    PhiArgs A;
    struct { const char* name; double** dst; } rw[] = {
        {"phi", &A.phi}, {"Ex", &A.Ex}, {"Er", &A.Er}, {"nUex", &A.nUex}, {"nUer", &A.nUer},
        {"phi_old", &A.phi_old}, {"nUex_old", &A.nUex_old}, {"nUer_old", &A.nUer_old},
        {"pc_Ex_old", &A.Ex_old}, {"pc_Er_old", &A.Er_old}, {"pc_phi_t", &A.phi_t}, {"pc_nUex_t", &A.nUex_t},
        {"pc_nUer_t", &A.nUer_t}, {"pc_dphi", &A.dphi}, {"pc_aP", &A.aP}, {"pc_aE", &A.aE}, {"pc_aW", &A.aW},
        {"pc_aN", &A.aN}, {"pc_aS", &A.aS}, {"pc_b", &A.b}};
    for (auto& e : rw) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    struct { const char* name; const double** dst; } ro[] = {
        {"rhoe", &A.rhoe}, {"rhoe_old", &A.rhoe_old}, {"rhoi", &A.rhoi}, {"Te", &A.Te}, {"mu_para", &A.mu_para},
        {"mu_perp", &A.mu_perp}, {"mu_rr", &A.mu_rr}, {"mu_xr", &A.mu_xr}, {"mu_xx", &A.mu_xx},
        {"rate_ionize", &A.rate_ionize}, {"Uix", &A.Uix}, {"Uir", &A.Uir}, {"rhoUmx", &A.rhoUmx},
        {"rhoUmr", &A.rhoUmr}};
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
        set_error("cth_solve_phi_pc: SEE tables missing (coefEISEE_eb_table, coefEISEE_rd_table, coefEISEE_ts_table)");
        return CTH_ERR_ARG;
    }
    A.flags = fs->flags;
    A.prm = *prm;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    const int nb = grd.x * grd.y;
    if ((size_t)nb * kNStat > (size_t)fs->npart) {
        set_error("cth_solve_phi_pc: reduction scratch too small");
        return CTH_ERR_ARG;
    }
    double* out = fs->scal + 16;
    const double* guess = nullptr;
    double* dphi_prev = nullptr;
    double* dphi_prev2 = nullptr;
    if (prm->warm_start != 0 && prm->flag_iter_phi != 0) {
        dphi_prev = field_ptr(fs, "dphi_prev");
        dphi_prev2 = field_ptr(fs, "dphi_prev2");
        guess = (prm->warm_start == 1 || prm->warm_start == 3) ? field_ptr(fs, "dphi_guess") : dphi_prev;
        if (!dphi_prev || !dphi_prev2 || !guess) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    cth_status st_first{};
    k_phi_begin<<<grd, blk, 0, s>>>(A);
    g->launches++;
    int ncount = 0, solver_rc = 0;
    double e_it[3] = {0, 0, 0}, e_call[3] = {0, 0, 0};
    cth_status st_last{};
    for (;;) {
        ncount++;
        k_phi_save<<<grd, blk, 0, s>>>(A);
        k_phi_predict<<<grd, blk, 0, s>>>(A);
        k_phi_assemble<<<grd, blk, 0, s>>>(A);
        g->launches += 3;
        CTH_CUDA(cudaGetLastError());
        // the MG solve is enqueued without a host round trip; its status is read after
        // the one synchronisation of the iteration
        int rc, pend = 0;
        if (prm->flag_iter_phi == 0)
            rc = sor_solve_dev(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, 1.9, prm->maxITR_SOR_phi,
                               prm->error_cnv_SOR_phi, A.dphi, s, &st_last);
        else
            rc = smg_solve_launch(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, prm->maxITR_SOR_phi,
                                  prm->error_cnv_SOR_phi, prm->precision, A.dphi, s, &pend, fs->h_solve,
                                  ncount == 1 ? guess : nullptr, prm->guess_max_relres,
                                  prm->warm_start == 1 ? dphi_prev : nullptr, SLOT_PHI);
        if (rc < 0) return rc;
        if (ncount == 1 && dphi_prev) {
            CTH_CUDA(cudaMemcpyAsync(dphi_prev2, dphi_prev, g->plane * sizeof(double), cudaMemcpyDeviceToDevice, s));
            CTH_CUDA(cudaMemcpyAsync(dphi_prev, A.dphi, g->plane * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
        k_phi_correct_a<<<grd, blk, 0, s>>>(A);
        k_phi_correct_b<<<dim3((g->ni + 2 + 256 * kCorrCells - 1) / (256 * kCorrCells), g->nj + 2), 256, 0, s>>>(
            A, fs->part, g->ws.counter, out);
        g->launches += 2;
        CTH_CUDA(cudaGetLastError());
        CTH_CUDA(cudaMemcpyAsync(fs->h_scal, out, kNStat * sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
        if (pend) rc = solve_parse(g, pend, fs->h_solve, &st_last);
        if (rc < 0) return rc;
        if (rc > solver_rc) solver_rc = rc;
        if (ncount == 1) st_first = st_last;
        const double* h = fs->h_scal;
        const int m = prm->flag_error;
        for (int k = 0; k < 3; k++) {
            e_it[k] = finish_res(m, h[2 * k], h[2 * k + 1]);
            e_call[k] = finish_res(m, h[6 + 2 * k], h[6 + 2 * k + 1]);
        }
        const double eg = fmax(fmax(e_it[0], e_it[1]), e_it[2]);
        if (eg < prm->error_cnv_HES_phi || ncount >= prm->maxITR_HES_phi) break;
    }
    if (res) {
        res->ncount = ncount;
        res->solver_rc = solver_rc;
        res->error_phi = e_call[0];
        res->error_nUex = e_call[1];
        res->error_nUer = e_call[2];
        res->error_iter[0] = e_it[0];
        res->error_iter[1] = e_it[1];
        res->error_iter[2] = e_it[2];
        res->solver = st_last;
        res->first = st_first;
        res->Ii_Anode = res->Ie_Anode = res->I_Anode = 0.0;
    }
    return CTH_OK;
}

}  // namespace cth

extern "C" int cth_solve_phi_pc(cth_fields* fs, const cth_phi_params* prm, void* stream, cth_pc_result* res) {
    if (!fs || !prm || prm->dx <= 0.0 || prm->dr <= 0.0 || prm->maxITR_HES_phi < 1 || prm->flag_error < 0 ||
        prm->flag_error > 3 || prm->warm_start < 0 || prm->warm_start > 3 ||
        (prm->warm_start != 0 && !(prm->guess_max_relres >= 0.0 && prm->guess_max_relres <= 10.0))) {
        cth::set_error("cth_solve_phi_pc: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return cth::solve_phi_pc(fs, prm, (cudaStream_t)stream, res);
}
