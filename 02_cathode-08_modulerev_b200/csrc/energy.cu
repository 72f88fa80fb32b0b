// energy.cu — the absorbed-power part of EmfieldModule::update_energy_profile
// (include/emfieldModule.hpp:7630-7790): the microwave current density
// J = sigma E of each field component with the magnetised cold-plasma
// conductivity tensor, the absorbed power densities Pabs = Re(J . E*)/2 on the
// x-faces, r-faces and cells, their volume integrals, and the cell profile
// gc.Pabs that the electron energy equation reads.  One thread per (i, j) of
// the index space; the face / cell roles follow the block unions of the
// x-face, r-face and cell grids (a cell in several blocks counts once).
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
