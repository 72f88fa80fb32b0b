// energy.cu — the absorbed-power part of EmfieldModule::update_energy_profile
// (include/emfieldModule.hpp:7630-7790): the microwave current density
// J = sigma E of each field component with the magnetised cold-plasma
// conductivity tensor, the absorbed power densities Pabs = Re(J . E*)/2 on the
// x-faces, r-faces and cells, their volume integrals, and the cell profile
// gc.Pabs that the electron energy equation reads.  One thread per (i, j) of
// the index space; the face / cell roles follow the block unions of the
// x-face, r-face and cell grids (a cell in several blocks counts once).
//
// The port part (flag_mwRef, :7792-8105) follows as two more kernels: one block
// sums the Poynting flux out of the outlet row (mWLoss_at_boundary_rR,
// :8631-8664) and the port current and voltage on the reference plane, then
// does the two-port scalar arithmetic (wave amplitudes, de-embedding with the
// feed's S-parameters, the power ratio) on the device; the second rescales
// Pabs and the field / current planes by it.
#include <cuda_runtime.h>

#include <cmath>

#include "fluid.cuh"

namespace cth {

namespace {

constexpr double kE0 = 1.60217662e-19;  // constants.hpp:6

__device__ __forceinline__ cd cs(cd a, double s) { return cd(a.x * s, a.y * s); }
__device__ __forceinline__ cd ld_cd(const double2* p, size_t q) {
    const double2 v = p[q];
    return cd(v.x, v.y);
}

struct Sigma {
    cd coef, Hx, Hr;
};

// emfieldModule.hpp:7655-7662 (and the r-face / cell copies)
__device__ __forceinline__ Sigma sigma(double nu, double rho, double Bx, double Br, double w, double me) {
    const cd EPS(1e-100, 1e-100);
    const cd den = cd(me * nu, me * w) + EPS;  // masse * (nu + i w) + EPS
    Sigma s;
    s.Hx = cdiv(cd(kE0 * Bx), den);
    s.Hr = cdiv(cd(kE0 * Br), den);
    const cd H2 = s.Hx * s.Hx + s.Hr * s.Hr;
    s.coef = cdiv(cdiv(cd(rho * kE0 * kE0), den), cd(1.0) + H2 + EPS);
    return s;
}

struct EnergyArgs {
    const unsigned char *mx, *mr, *mc;  // x-face, r-face and cell block masks
    const double *rhoe, *nu_m1, *Bx, *Br;
    const double2 *E1x, *E1r, *E1p;
    double2 *J1x, *J1r, *J1p;
    double *Pabsx, *Pabsr, *Pabsp, *Pabs;
    cth_energy_params prm;
    int ni, nj, ld;
};

__device__ __forceinline__ double rad(const cth_energy_params& P, int j) { return P.rmin + (j - 0.5) * P.dr; }

__global__ void k_energy(EnergyArgs A, double* __restrict__ part, unsigned int* counter, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    double s[3] = {0.0, 0.0, 0.0};
    if (i <= A.ni + 1) {
        const int ld = A.ld;
        const size_t p = (size_t)j * ld + i;
        const cth_energy_params& P = A.prm;
        const double w = P.omegam, me = P.masse, dV = P.dx * P.dr * 2.0 * M_PI;
        const double rj = rad(P, j);
        // the stencils reach i-1 / j+1 (x-faces), j-1 / i+1 (r-faces), i+1 / j+1
        // (cells); the reference's blocks stay inside those bounds
        if (A.mx[p] && i >= 1 && j <= A.nj) {  // x-face i-1/2 (emfieldModule.hpp:7641-7678)
            const double rL = (rj + rad(P, j - 1)) / 2.0, rR = (rj + rad(P, j + 1)) / 2.0;
            const Sigma S = sigma((A.nu_m1[p] + A.nu_m1[p - 1]) / 2.0, (A.rhoe[p] + A.rhoe[p - 1]) / 2.0,
                                  (A.Bx[p] + A.Bx[p - 1]) / 2.0, (A.Br[p] + A.Br[p - 1]) / 2.0, w, me);
            const cd sxr = S.coef * (S.Hx * S.Hr), sxp = S.coef * S.Hr, sxx = S.coef * (cd(1.0) + S.Hx * S.Hx);
            const cd Ex = ld_cd(A.E1x, p);
            const cd Er = cs(cs(ld_cd(A.E1r, p) + ld_cd(A.E1r, p - 1), rL) + cs(ld_cd(A.E1r, p + ld) + ld_cd(A.E1r, p + ld - 1), rR),
                             1.0 / (4.0 * rj));
            const cd Ep = cs(ld_cd(A.E1p, p) + ld_cd(A.E1p, p - 1), 0.5);
            const cd J = sxr * Er + sxp * Ep + sxx * Ex;
            A.J1x[p] = make_double2(J.x, J.y);
            const double pa = 0.5 * (J.x * Ex.x + J.y * Ex.y);
            A.Pabsx[p] = pa;
            s[0] = pa * (dV * rj);
        }
        if (A.mr[p] && j >= 1 && i <= A.ni) {  // r-face j-1/2 (:7683-7711)
            const double rjm = rad(P, j - 1), rt = (rjm + rj) / 2.0;
            const Sigma S = sigma((A.nu_m1[p] + A.nu_m1[p - ld]) / 2.0, (A.rhoe[p] + A.rhoe[p - ld]) / 2.0,
                                  (rj * A.Bx[p] + rjm * A.Bx[p - ld]) / (2.0 * rt),
                                  (rj * A.Br[p] + rjm * A.Br[p - ld]) / (2.0 * rt), w, me);
            const cd srr = S.coef * (cd(1.0) + S.Hr * S.Hr), srp = S.coef * (-S.Hx), srx = S.coef * (S.Hx * S.Hr);
            const cd Ex = cs(cs(ld_cd(A.E1x, p) + ld_cd(A.E1x, p + 1), rj) + cs(ld_cd(A.E1x, p - ld) + ld_cd(A.E1x, p - ld + 1), rjm),
                             1.0 / (4.0 * rt));
            const cd Er = ld_cd(A.E1r, p);
            const cd Ep = cs(cs(ld_cd(A.E1p, p), rj) + cs(ld_cd(A.E1p, p - ld), rjm), 1.0 / (2.0 * rt));
            const cd J = srr * Er + srp * Ep + srx * Ex;
            A.J1r[p] = make_double2(J.x, J.y);
            const double pa = 0.5 * (J.x * Er.x + J.y * Er.y);
            A.Pabsr[p] = pa;
            s[1] = pa * (dV * rt);
        }
        if (A.mc[p] && i <= A.ni && j <= A.nj) {  // cell (:7715-7746)
            const double qL = (rad(P, j - 1) + rj) / 2.0 / (rj + 1e-100);
            const double qR = (rad(P, j + 1) + rj) / 2.0 / (rj + 1e-100);
            const Sigma S = sigma(A.nu_m1[p], A.rhoe[p], A.Bx[p], A.Br[p], w, me);
            const cd spr = S.coef * S.Hx, spp = S.coef, spx = S.coef * (-S.Hr);
            const cd Ex = cs(ld_cd(A.E1x, p) + ld_cd(A.E1x, p + 1), 0.5);
            const cd Er = cs(cs(ld_cd(A.E1r, p + ld), qR) + cs(ld_cd(A.E1r, p), qL), 0.5);
            const cd Ep = ld_cd(A.E1p, p);
            const cd J = spr * Er + spp * Ep + spx * Ex;
            A.J1p[p] = make_double2(J.x, J.y);
            const double pa = 0.5 * (J.x * Ep.x + J.y * Ep.y);
            A.Pabsp[p] = pa;
            s[2] = pa * (dV * rj);
        }
    }
    grid_reduce<3>(s, 0x0u, part, counter, out);
}

// gc.Pabs on the cell blocks (emfieldModule.hpp:7749-7790)
__global__ void k_energy_cells(EnergyArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    if (!A.mc[p] || i > A.ni || j > A.nj) return;
    A.Pabs[p] = (A.Pabsx[p] + A.Pabsx[p + 1]) / 2.0 + (A.Pabsr[p] + A.Pabsr[p + A.ld]) / 2.0 + A.Pabsp[p];
}


constexpr double kMU0 = 1.2566370614e-6;  // constants.hpp:8
constexpr double kPI = 3.14159265358979323846;

// words of the port result (device, fs->scal + 64)
enum PortWord {
    PW_POUT = 0, PW_IREF = 1, PW_VREF = 3, PW_PFWD = 5, PW_PREF = 6, PW_PERR = 7, PW_PFWD_ALL = 8,
    PW_PREF_ALL = 9, PW_RATIO = 10, PW_PABS_F = 11, PW_GP = 12, PW_ZP = 14, PW_GALL = 16, PW_ZALL = 18,
    PW_PSUM = 20, PW_FIELD_F = 21, PW_EXC_F = 22, PW_FINITE = 23, PW_N = 24
};

struct PortArgs {
    const double2 *E1x, *E1r, *E1p;
    double* out;
    cth_mw_port_params p;
    double power_sum;
    int ld;
};

__device__ __forceinline__ cd cdivr(cd a, double s) { return cd(a.x / s, a.y / s); }

// one block: the outlet loss, the reference-plane current and voltage, the
// two-port arithmetic of :7838-8045 (flag_mwRef = 1) or the plain rescale of
// :8073-8095 (flag_mwRef = 0).  Sums run in a fixed order (strided per thread,
// then a fixed tree), so the result is reproducible.
__global__ void k_mw_port(PortArgs A) {
    __shared__ double red[5][256];
    const int t = threadIdx.x;
    const cth_mw_port_params& p = A.p;
    const int ld = A.ld;
    auto r = [&](int jj) { return p.rmin + (jj - 0.5) * p.dr; };
    auto X = [&](int i, int j) { return ld_cd(A.E1x, (size_t)j * ld + i); };
    auto R = [&](int i, int j) { return ld_cd(A.E1r, (size_t)j * ld + i); };
    auto P = [&](int i, int j) { return ld_cd(A.E1p, (size_t)j * ld + i); };
    const double dx = p.dx, dr = p.dr, w = p.omegam;
    const cd iwm(0.0, 1.0 / (w * kMU0));
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (p.flag_mwRef) {
        // the Poynting flux through the upper faces of row j_out (mWLoss_at_boundary_rR)
        const int j = p.j_out;
        const double rt = (r(j) + r(j + 1)) / 2.0;
        for (int i = p.i_out0 + t; i <= p.i_out1; i += blockDim.x) {
            const cd dRdx_L = cdivr(R(i, j + 1) - R(i - 1, j + 1), dx);
            const cd dXdr_L = cdivr(X(i, j + 1) - X(i, j), dr);
            const cd dRdx_R = cdivr(R(i + 1, j + 1) - R(i, j + 1), dx);
            const cd dXdr_R = cdivr(X(i + 1, j + 1) - X(i + 1, j), dr);
            const cd H1p = cdivr(iwm * (dRdx_R - dXdr_R) + iwm * (dRdx_L - dXdr_L), 2.0);
            const cd H1x = iwm * cdivr(cs(P(i, j + 1), r(j + 1)) - cs(P(i, j), r(j)), rt * dr);
            const cd E1p = cdivr(cs(P(i, j + 1), r(j + 1)) + cs(P(i, j), r(j)), 2.0 * rt);
            const cd Ex_L = cdivr(cs(X(i, j + 1), r(j + 1)) + cs(X(i, j), r(j)), 2.0 * rt);
            const cd Ex_R = cdivr(cs(X(i + 1, j + 1), r(j + 1)) + cs(X(i + 1, j), r(j)), 2.0 * rt);
            const cd E1x = cdivr(Ex_R + Ex_L, 2.0);
            const cd ExH = E1p * conj(H1x) - E1x * conj(H1p);
            const double S = 0.5 * ExH.x;
            acc[0] += 2.0 * kPI * rt * S * dx;
        }
        // current (from H_phi) and voltage (r Er averaged) over the feed's Er faces at i_ref
        const int i = p.i_ref;
        for (int j = p.jf0 + t; j <= p.jf1; j += blockDim.x) {
            const double rt = (r(j) + r(j - 1)) / 2.0;
            const cd H = cdivr(cdivr(R(i, j) - R(i - 1, j), dx), w * kMU0) * cd(0.0, 1.0);
            const cd I = cs(H, 2.0 * kPI * rt);
            const cd V = cs(cdivr(R(i, j) + R(i - 1, j), 2.0), rt);
            acc[1] += I.x; acc[2] += I.y; acc[3] += V.x; acc[4] += V.y;
        }
    }
    for (int k = 0; k < 5; k++) red[k][t] = acc[k];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (t < h)
            for (int k = 0; k < 5; k++) red[k][t] += red[k][t + h];
        __syncthreads();
    }
    if (t != 0) return;
    double* o = A.out;
    for (int k = 0; k < PW_N; k++) o[k] = 0.0;
    const double psum = A.power_sum;
    if (!p.flag_mwRef) {
        const double ratio = p.Pmw / psum;
        o[PW_RATIO] = ratio;
        o[PW_PABS_F] = ratio;
        o[PW_FIELD_F] = 1.0;
        o[PW_EXC_F] = sqrt(ratio);
        o[PW_PSUM] = psum;
        o[PW_FINITE] = isfinite(ratio) ? 1.0 : 0.0;
        return;
    }
    const int nf = p.jf1 - p.jf0 + 1;
    const double P_out = red[0][0];
    const cd I_ref = cdivr(cd(red[1][0], red[2][0]), (double)nf);
    const cd coef = cdivr(cd(red[3][0], red[4][0]), (double)nf);
    const cd V_ref = cs(coef, log(p.r2 / p.r1));
    const double den = 2.0 * sqrt(2.0 * p.Z0);
    const cd a2 = cdivr(V_ref - cs(I_ref, p.Z0), den);
    const cd b2 = cdivr(V_ref + cs(I_ref, p.Z0), den);
    double P_fwd = abs2(b2), P_ref = abs2(a2);
    double P_err = P_fwd - P_ref - psum - P_out;
    const cd S11(p.S11[0], p.S11[1]), S21(p.S21[0], p.S21[1]), S12(p.S12[0], p.S12[1]), S22(p.S22[0], p.S22[1]);
    const cd a1 = cdiv(b2 - S22 * a2, S21);
    const cd b1 = S11 * a1 + S12 * a2;
    double P_fwd_all = abs2(a1), P_ref_all = abs2(b1);
    const double ratio = p.Pmw / P_fwd_all;
    const double ratio_eff = ratio * (psum + P_err) / psum;
    const cd Gp = cdiv(a2, b2), Ga = cdiv(b1, a1);
    const cd Zp = cs(cdiv(cd(1.0) + Gp, cd(1.0) - Gp), p.Z0);
    const cd Za = cs(cdiv(cd(1.0) + Ga, cd(1.0) - Ga), p.Z0);
    o[PW_POUT] = P_out * ratio;
    o[PW_IREF] = I_ref.x; o[PW_IREF + 1] = I_ref.y;
    o[PW_VREF] = V_ref.x; o[PW_VREF + 1] = V_ref.y;
    o[PW_PFWD] = P_fwd * ratio;
    o[PW_PREF] = P_ref * ratio;
    o[PW_PERR] = P_err * ratio;
    o[PW_PFWD_ALL] = P_fwd_all * ratio;
    o[PW_PREF_ALL] = P_ref_all * ratio;
    o[PW_RATIO] = ratio;
    o[PW_PABS_F] = ratio_eff;
    o[PW_FIELD_F] = sqrt(ratio_eff);
    o[PW_EXC_F] = sqrt(ratio);
    o[PW_GP] = Gp.x; o[PW_GP + 1] = Gp.y;
    o[PW_ZP] = Zp.x; o[PW_ZP + 1] = Zp.y;
    o[PW_GALL] = Ga.x; o[PW_GALL + 1] = Ga.y;
    o[PW_ZALL] = Za.x; o[PW_ZALL + 1] = Za.y;
    o[PW_PSUM] = (psum + P_err) * ratio;
    o[PW_FINITE] = (isfinite(ratio_eff) && isfinite(sqrt(ratio_eff)) && isfinite(ratio)) ? 1.0 : 0.0;
}

// Pabs *= its factor; the field and current planes (complex) *= the field
// factor, over the whole (ni+2) x (nj+2) index space; nothing when the factors
// are not finite (the host reports it)
__global__ void k_mw_scale(const double* __restrict__ o, double* __restrict__ Pabs, double2* E1x, double2* E1r,
                           double2* E1p, double2* J1x, double2* J1r, double2* J1p, double2* X1, double2* X2,
                           double2* X3, int ni, int ld) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= ni + 2 || o[PW_FINITE] == 0.0) return;
    const size_t q = (size_t)j * ld + i;
    Pabs[q] *= o[PW_PABS_F];
    const double f = o[PW_FIELD_F];
    if (f == 1.0) return;
    double2* pl[9] = {E1x, E1r, E1p, J1x, J1r, J1p, X1, X2, X3};
    for (int k = 0; k < 9; k++) {
        if (!pl[k]) continue;
        double2 v = pl[k][q];
        v.x *= f;
        v.y *= f;
        pl[k][q] = v;
    }
}

}  // namespace
}  // namespace cth

using namespace cth;

extern "C" int cth_update_energy_profile(cth_fields* fs, cth_grid* gx, cth_grid* gr, const cth_energy_params* prm,
                                         const void* E1x, const void* E1r, const void* E1p, void* J1x, void* J1r,
                                         void* J1p, void* stream, cth_energy_result* res) {
    if (!fs || !gx || !gr || !prm || !E1x || !E1r || !E1p || !J1x || !J1r || !J1p || !(prm->dx > 0.0) ||
        !(prm->dr > 0.0) || !(prm->masse > 0.0)) {
        set_error("cth_update_energy_profile: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    if (gx->ni != g->ni || gx->nj != g->nj || gr->ni != g->ni || gr->nj != g->nj || gx->ld != g->ld ||
        gr->ld != g->ld) {
        set_error("cth_update_energy_profile: the face grids must share the store's index space");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = (cudaStream_t)stream;
    EnergyArgs A;
    A.mx = gx->mask_full;
    A.mr = gr->mask_full;
    A.mc = g->mask_full;
    struct { const char* name; const double** dst; } ro[] = {
        {"rhoe", &A.rhoe}, {"nu_m1", &A.nu_m1}, {"Bx", &A.Bx}, {"Br", &A.Br}};
    for (auto& e : ro) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    struct { const char* name; double** dst; } rw[] = {
        {"Pabsx", &A.Pabsx}, {"Pabsr", &A.Pabsr}, {"Pabsp", &A.Pabsp}, {"Pabs", &A.Pabs}};
    for (auto& e : rw) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    A.E1x = (const double2*)E1x;
    A.E1r = (const double2*)E1r;
    A.E1p = (const double2*)E1p;
    A.J1x = (double2*)J1x;
    A.J1r = (double2*)J1r;
    A.J1p = (double2*)J1p;
    A.prm = *prm;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    if ((size_t)grd.x * grd.y * 3 > (size_t)fs->npart) {
        set_error("cth_update_energy_profile: reduction scratch too small");
        return CTH_ERR_ARG;
    }
    double* out = fs->scal + 40;
    k_energy<<<grd, blk, 0, s>>>(A, fs->part, g->ws.counter, out);
    k_energy_cells<<<grd, blk, 0, s>>>(A);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(fs->h_scal, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    if (res) {
        res->Px = fs->h_scal[0];
        res->Pr = fs->h_scal[1];
        res->Pp = fs->h_scal[2];
        res->power_sum = res->Px + res->Pr + res->Pp;
    }
    return CTH_OK;
}

extern "C" int cth_mw_port_rescale(cth_fields* fs, const cth_mw_port_params* prm, double power_sum, void* E1x,
                                   void* E1r, void* E1p, void* J1x, void* J1r, void* J1p, void* J1x_exc,
                                   void* J1r_exc, void* J1p_exc, void* stream, cth_mw_port_result* res) {
    if (!fs || !prm || !(prm->dx > 0.0) || !(prm->dr > 0.0) || !(prm->omegam > 0.0) || !(prm->Pmw >= 0.0)) {
        set_error("cth_mw_port_rescale: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    const int ni = g->ni, nj = g->nj;
    if (prm->flag_mwRef) {
        const bool ok = E1x && E1r && E1p && J1x && J1r && J1p && prm->r1 > 0.0 && prm->r2 > prm->r1 &&
                        prm->Z0 > 0.0 && prm->i_out0 >= 1 && prm->i_out1 <= ni && prm->j_out >= 1 &&
                        prm->j_out <= nj && prm->i_ref >= 1 && prm->i_ref <= ni + 1 && prm->jf0 >= 1 &&
                        prm->jf1 <= nj + 1 && prm->jf1 >= prm->jf0;
        if (!ok) {
            set_error("cth_mw_port_rescale: invalid port arguments (planes, radii, Z0 or index ranges)");
            return CTH_ERR_ARG;
        }
    }
    CTH_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = (cudaStream_t)stream;
    double* pabs = field_ptr(fs, "Pabs");
    if (!pabs) {
        set_error("field allocation failed");
        return CTH_ERR_ALLOC;
    }
    PortArgs A;
    A.E1x = (const double2*)E1x;
    A.E1r = (const double2*)E1r;
    A.E1p = (const double2*)E1p;
    A.out = fs->scal + 64;
    A.p = *prm;
    A.power_sum = power_sum;
    A.ld = g->ld;
    k_mw_port<<<1, 256, 0, s>>>(A);
    dim3 blk(128), grd((ni + 2 + 127) / 128, nj + 2);
    const bool fields = prm->flag_mwRef != 0;
    k_mw_scale<<<grd, blk, 0, s>>>(A.out, pabs, fields ? (double2*)E1x : nullptr, fields ? (double2*)E1r : nullptr,
                                   fields ? (double2*)E1p : nullptr, fields ? (double2*)J1x : nullptr,
                                   fields ? (double2*)J1r : nullptr, fields ? (double2*)J1p : nullptr,
                                   fields ? (double2*)J1x_exc : nullptr, fields ? (double2*)J1r_exc : nullptr,
                                   fields ? (double2*)J1p_exc : nullptr, ni, g->ld);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(fs->h_scal + 64, A.out, PW_N * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    const double* o = fs->h_scal + 64;
    if (res) {
        res->P_out = o[PW_POUT];
        res->P_fwd = o[PW_PFWD];
        res->P_ref = o[PW_PREF];
        res->P_fwd_all = o[PW_PFWD_ALL];
        res->P_ref_all = o[PW_PREF_ALL];
        res->P_err = o[PW_PERR];
        res->power_sum = o[PW_PSUM];
        res->ratio = o[PW_RATIO];
        res->pabs_factor = o[PW_PABS_F];
        res->field_factor = o[PW_FIELD_F];
        res->J1r_exc_factor = o[PW_EXC_F];
        for (int k = 0; k < 2; k++) {
            res->I_ref[k] = o[PW_IREF + k];
            res->V_ref[k] = o[PW_VREF + k];
            res->Gamma_p[k] = o[PW_GP + k];
            res->Zp[k] = o[PW_ZP + k];
            res->Gamma_all[k] = o[PW_GALL + k];
            res->Zall[k] = o[PW_ZALL + k];
        }
    }
    if (o[PW_FINITE] == 0.0) {
        set_error("cth_mw_port_rescale: the power ratio is not finite (zero forward or absorbed power); nothing "
                  "rescaled");
        return CTH_NONFINITE;
    }
    return CTH_OK;
}
