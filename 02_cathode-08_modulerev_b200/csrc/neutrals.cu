// neutrals.cu — FluidModule::update_rhon (fluidModule.hpp:4963-5410) and
// update_rhom (:5416-5792) on the device: implicit diffusion of the ground-state
// and metastable neutrals with D = D N / n_n, ionisation / excitation sources,
// wall recombination fluxes (ground state), thermal wall losses (metastables),
// the gas inlet on part of the upper wall and the open top.  One thread per cell
// or face; walls, inlet and open boundary from the per-cell side flags.
#include <cuda_runtime.h>

#include <cmath>

#include "fluid.cuh"

namespace cth {

struct NeutArgs {
    double *rhon, *rhom, *rhoUnx, *rhoUnr, *rhoUnx_wall, *rhoUnr_wall, *rhoUmx, *rhoUmr, *rhoUmx_wall, *rhoUmr_wall;
    double *rhon_old, *rhom_old, *rhoUnx_old, *rhoUnr_old, *rhoUmx_old, *rhoUmr_old;
    const double *rhoUix_wall, *rhoUir_wall, *rhoe, *nu_excStep, *nu_super, *nu_excMeta, *nu_exc, *nu_ionz,
        *nu_ionzStep;
    double *aP, *aE, *aW, *aN, *aS, *b;
    const unsigned char* flags;
    cth_neutral_params prm;
    int ni, nj, ld;
};

#define FL(ii, jj) flag_at(A.flags, (ii), (jj), A.ni, A.nj, A.ld)

__device__ __forceinline__ double rc(const cth_neutral_params& P, int j) { return P.rmin + (j - 0.5) * P.dr; }

__device__ __forceinline__ double dnn(const cth_neutral_params& P) {
    const double sigma = M_PI * (2.0 * P.ri) * (2.0 * P.ri);
    return 2.0 / (3.0 * sigma) * sqrt(kBoltz * P.Tn / (M_PI * P.massi));
}

template <int M>
__global__ void k_neut_begin(NeutArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    if (M == 0) {
        A.rhon_old[p] = A.rhon[p];
        A.rhoUnx_old[p] = A.rhoUnx[p];
        A.rhoUnr_old[p] = A.rhoUnr[p];
    } else {
        A.rhom_old[p] = A.rhom[p];
        A.rhoUmx_old[p] = A.rhoUmx[p];
        A.rhoUmr_old[p] = A.rhoUmr[p];
    }
}

// ground state (fluidModule.hpp:4999-5123)
__global__ void k_rhon_assemble(NeutArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (fc) {
        const cth_neutral_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_n = P.dt * double(P.ndt_n);
        const double rj = rc(P, j), rjm = rc(P, j - 1), rjp = rc(P, j + 1);
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double qL = (rj + rjm) / 2.0 / rj, qR = (rj + rjp) / 2.0 / rj;
        const double DnN = dnn(P);
        const double* no = A.rhon_old;
        const double DLx = DnN / ((no[p] + no[p - 1]) / 2.0 + 1e-100);
        const double DRx = DnN / ((no[p] + no[p + 1]) / 2.0 + 1e-100);
        const double DLr = DnN / ((no[p] + no[p - ld]) / 2.0 + 1e-100);
        const double DRr = DnN / ((no[p] + no[p + ld]) / 2.0 + 1e-100);
        const bool inlet = (fc & F_BRR_INLET) != 0;
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bRx = (fc & F_BRX) ? 1.0 : 0.0;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr_wall = (inlet || (fc & F_BRR_WALL)) ? 1.0 : 0.0;
        const double bRr_in = inlet ? 0.0 : 1.0;
        const double bRr_open = (fc & F_BRR_OPEN) ? 1.0 : 0.0;
        const double bRr = bRr_wall * bRr_in * bRr_open;
        const double GLx = (fc & F_BLX) ? 0.0 : -A.rhoUix_wall[p] - A.rhoUmx_wall[p];
        const double GRx = (fc & F_BRX) ? 0.0 : -A.rhoUix_wall[p + 1] - A.rhoUmx_wall[p + 1];
        const double GLr = (fc & F_BLR_WALL) ? 0.0 : -A.rhoUir_wall[p] - A.rhoUmr_wall[p];
        const double GRr = bRr_wall != 0.0 ? 0.0 : -A.rhoUir_wall[p + ld] - A.rhoUmr_wall[p + ld];
        const double Gin = inlet ? -A.rhoUir_wall[p + ld] - A.rhoUmr_wall[p + ld] - P.fn_In : 0.0;
        const double Gop = (fc & F_BRR_OPEN) ? 0.0 : fmax(rL / rR * A.rhoUnr_old[p], 0.0);
        vP = (DRx * bRx + DLx * bLx) * dr * dr + (qR * DRr * bRr + qL * DLr * bLr) * dx * dx + dx * dx * dr * dr / dt_n;
        vE = DRx * dr * dr * bRx;
        vW = DLx * dr * dr * bLx;
        vN = qR * DRr * dx * dx * bRr;
        vS = qL * DLr * dx * dx * bLr;
        const double n = A.rhoe[p];
        const double G = (A.nu_excStep[p] + A.nu_super[p]) * n;
        const double L = (A.nu_excMeta[p] + 0.5 * A.nu_exc[p] + A.nu_ionz[p]) * n;
        vb = no[p] / dt_n * dx * dx * dr * dr + (G - L) * dx * dx * dr * dr + (GLx) * dr * dx * dr -
             (GRx) * dr * dx * dr + qL * (GLr) * dx * dx * dr - qR * (GRr + Gop + Gin) * dx * dx * dr;
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// ground-state fluxes on every face (fluidModule.hpp:5133-5265)
__global__ void k_rhon_fluxes(NeutArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const cth_neutral_params& P = A.prm;
    const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
    const double DnN = dnn(P);
    const double* no = A.rhon_old;
    const double* n = A.rhon;
    if (fc && fw) A.rhoUnx[p] = -(DnN / ((no[p] + no[p - 1]) / 2.0 + 1e-100)) * (n[p] - n[p - 1]) / P.dx;
    if (fc && fs) A.rhoUnr[p] = -(DnN / ((no[p] + no[p - ld]) / 2.0 + 1e-100)) * (n[p] - n[p - ld]) / P.dr;
    if ((fc && !(fc & F_BLX)) || (fw && !(fw & F_BRX))) {
        const double v = -A.rhoUix_wall[p] - A.rhoUmx_wall[p];
        A.rhoUnx[p] = v;
        A.rhoUnx_wall[p] = v;
    }
    if (fc && !(fc & F_BLR_WALL)) {
        const double v = -A.rhoUir_wall[p] - A.rhoUmr_wall[p];
        A.rhoUnr[p] = v;
        A.rhoUnr_wall[p] = v;
    }
    if (fs && !(fs & F_BRR_WALL)) {
        if (fs & F_BRR_INLET) {
            A.rhoUnr[p] = -A.rhoUir_wall[p] - A.rhoUmr_wall[p] - P.fn_In;
        } else {
            const double v = -A.rhoUir_wall[p] - A.rhoUmr_wall[p];
            A.rhoUnr[p] = v;
            A.rhoUnr_wall[p] = v;
        }
    }
    if (fs && !(fs & F_BRR_OPEN)) {
        const double rjc = rc(P, j - 1);
        const double rL = (rjc + rc(P, j - 2)) / 2.0, rR = (rjc + rc(P, j)) / 2.0;
        A.rhoUnr[p] = fmax(rL / rR * A.rhoUnr_old[p - ld], 0.0);
        A.rhoUnr_wall[p] = 0.0;
    }
}

// positivity of rhon on the fluid cells (fluidModule.hpp:5382-5399) and calcRes
__global__ void k_rhon_fix(NeutArgs A, double* __restrict__ part, unsigned int* counter, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int mode = A.prm.flag_error;
    double s[2] = {0.0, 0.0};
    if (i <= A.ni + 1 && FL(i, j)) {
        const size_t p = (size_t)j * A.ld + i;
        double v = A.rhon[p];
        if (v < 0.0) {
            v = fmax(A.rhon_old[p], 0.0);
            A.rhon[p] = v;
        }
        res_stat(mode, v, A.rhon_old[p], s[0], s[1]);
    }
    grid_reduce<2>(s, (mode == 0 || mode == 2) ? 0x3u : 0u, part, counter, out);
}

// metastables (fluidModule.hpp:5436-5568)
__global__ void k_rhom_assemble(NeutArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const unsigned fc = FL(i, j);
    double vP = 0, vE = 0, vW = 0, vN = 0, vS = 0, vb = 0;
    if (fc) {
        const cth_neutral_params& P = A.prm;
        const double dx = P.dx, dr = P.dr, dt_m = P.dt * double(P.ndt_m);
        const double rj = rc(P, j), rjm = rc(P, j - 1), rjp = rc(P, j + 1);
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double qL = (rj + rjm) / 2.0 / rj, qR = (rj + rjp) / 2.0 / rj;
        const double vth = sqrt(8.0 * kBoltz * P.Tn / (M_PI * P.massi));
        const double* nn = A.rhon;
        const double DLx = P.DmN / ((nn[p] + nn[p - 1]) / 2.0 + 1e-100);
        const double DRx = P.DmN / ((nn[p] + nn[p + 1]) / 2.0 + 1e-100);
        const double DLr = P.DmN / ((nn[p] + nn[p - ld]) / 2.0 + 1e-100);
        const double DRr = P.DmN / ((nn[p] + nn[p + ld]) / 2.0 + 1e-100);
        const double bLx = (fc & F_BLX) ? 1.0 : 0.0, bRx = (fc & F_BRX) ? 1.0 : 0.0;
        const double bLr = ((fc & F_BLR_WALL) && (fc & F_BLR_CEN)) ? 1.0 : 0.0;
        const double bRr = ((fc & F_BRR_WALL) && (fc & F_BRR_OPEN)) ? 1.0 : 0.0;
        const double GLx = (fc & F_BLX) ? 0.0 : -0.25 * vth;
        const double GRx = (fc & F_BRX) ? 0.0 : 0.25 * vth;
        const double GLr = (fc & F_BLR_WALL) ? 0.0 : -0.25 * vth;
        const double GRr = (fc & F_BRR_WALL) ? 0.0 : 0.25 * vth;
        const double Gop = (fc & F_BRR_OPEN) ? 0.0 : rL / rR * A.rhoUmr_old[p];
        vP = (DRx * bRx + DLx * bLx) * dr * dr + (qR * DRr * bRr + qL * DLr * bLr) * dx * dx - GLx * dr * dx * dr +
             GRx * dr * dx * dr - qL * GLr * dx * dx * dr + qR * GRr * dx * dx * dr + dx * dx * dr * dr / dt_m;
        vE = DRx * dr * dr * bRx;
        vW = DLx * dr * dr * bLx;
        vN = qR * DRr * dx * dx * bRr;
        vS = qL * DLr * dx * dx * bLr;
        const double n = A.rhoe[p];
        const double G = n * (A.nu_excMeta[p] + 0.5 * A.nu_exc[p]);
        const double L = n * (A.nu_ionzStep[p] + A.nu_excStep[p] + A.nu_super[p]);
        vb = A.rhom_old[p] / dt_m * dx * dx * dr * dr + (G - L) * dx * dx * dr * dr + (0.0) * dr * dx * dr -
             (0.0) * dr * dx * dr + qL * (0.0) * dx * dx * dr - qR * (Gop) * dx * dx * dr;
    }
    A.aP[p] = vP; A.aE[p] = vE; A.aW[p] = vW; A.aN[p] = vN; A.aS[p] = vS; A.b[p] = vb;
}

// positivity of rhom over the given boxes (fluidModule.hpp:5580-5593)
__global__ void k_rhom_fix(NeutArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    bool in = false;
    for (int q = 0; q < A.prm.n_pos_box; q++) {
        const int* B = A.prm.pos_box[q];
        in = in || (i >= B[0] && i <= B[1] && j >= B[2] && j <= B[3]);
    }
    if (!in) return;
    const size_t p = (size_t)j * A.ld + i;
    if (A.rhom[p] < 0.0) A.rhom[p] = fmax(A.rhom_old[p], 0.0);
}

// metastable fluxes (fluidModule.hpp:5595-5700) and calcRes of rhom
__global__ void k_rhom_fluxes(NeutArgs A, double* __restrict__ part, unsigned int* counter,
                              double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int mode = A.prm.flag_error;
    double s[2] = {0.0, 0.0};
    if (i <= A.ni + 1) {
        const int ld = A.ld;
        const size_t p = (size_t)j * ld + i;
        const cth_neutral_params& P = A.prm;
        const unsigned fc = FL(i, j), fw = FL(i - 1, j), fs = FL(i, j - 1);
        const double vth = sqrt(8.0 * kBoltz * P.Tn / (M_PI * P.massi));
        const double* nn = A.rhon;
        const double* m = A.rhom;
        if (fc && fw) A.rhoUmx[p] = -(P.DmN / ((nn[p] + nn[p - 1]) / 2.0 + 1e-100)) * (m[p] - m[p - 1]) / P.dx;
        if (fc && fs) A.rhoUmr[p] = -(P.DmN / ((nn[p] + nn[p - ld]) / 2.0 + 1e-100)) * (m[p] - m[p - ld]) / P.dr;
        if (fc && !(fc & F_BLX)) {
            A.rhoUmx[p] = -0.25 * m[p] * vth;
            A.rhoUmx_wall[p] = A.rhoUmx[p];
        }
        if (fw && !(fw & F_BRX)) {
            A.rhoUmx[p] = 0.25 * m[p - 1] * vth;
            A.rhoUmx_wall[p] = A.rhoUmx[p];
        }
        if (fc && !(fc & F_BLR_WALL)) {
            A.rhoUmr[p] = -0.25 * m[p] * vth;
            A.rhoUmr_wall[p] = A.rhoUmr[p];
        }
        if (fs && !(fs & F_BRR_WALL)) {
            A.rhoUmr[p] = 0.25 * m[p - ld] * vth;
            A.rhoUmr_wall[p] = A.rhoUmr[p];
        }
        if (fs && !(fs & F_BRR_OPEN)) {
            const double rjc = rc(P, j - 1);
            const double rL = (rjc + rc(P, j - 2)) / 2.0, rR = (rjc + rc(P, j)) / 2.0;
            A.rhoUmr[p] = A.rhoUmr_old[p - ld] * rL / rR;
            A.rhoUmr_wall[p] = 0.0;
        }
        if (fc) res_stat(mode, m[p], A.rhom_old[p], s[0], s[1]);
    }
    grid_reduce<2>(s, (mode == 0 || mode == 2) ? 0x3u : 0u, part, counter, out);
}

#undef FL

static int update_neutrals(cth_fields* fs, const cth_neutral_params* prm, cudaStream_t s, cth_neutral_result* res) {
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_update_neutrals: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    NeutArgs A{};
    struct { const char* name; double** dst; } rw[] = {
        {"rhon", &A.rhon}, {"rhom", &A.rhom}, {"rhoUnx", &A.rhoUnx}, {"rhoUnr", &A.rhoUnr},
        {"rhoUnx_wall", &A.rhoUnx_wall}, {"rhoUnr_wall", &A.rhoUnr_wall}, {"rhoUmx", &A.rhoUmx},
        {"rhoUmr", &A.rhoUmr}, {"rhoUmx_wall", &A.rhoUmx_wall}, {"rhoUmr_wall", &A.rhoUmr_wall},
        {"rhon_old", &A.rhon_old}, {"rhom_old", &A.rhom_old}, {"rhoUnx_old", &A.rhoUnx_old},
        {"rhoUnr_old", &A.rhoUnr_old}, {"rhoUmx_old", &A.rhoUmx_old}, {"rhoUmr_old", &A.rhoUmr_old},
        {"pc_aP", &A.aP}, {"pc_aE", &A.aE}, {"pc_aW", &A.aW}, {"pc_aN", &A.aN}, {"pc_aS", &A.aS}, {"pc_b", &A.b}};
    for (auto& e : rw) {
        *e.dst = field_ptr(fs, e.name);
        if (!*e.dst) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    struct { const char* name; const double** dst; } ro[] = {
        {"rhoUix_wall", &A.rhoUix_wall}, {"rhoUir_wall", &A.rhoUir_wall}, {"rhoe", &A.rhoe},
        {"nu_excStep", &A.nu_excStep}, {"nu_super", &A.nu_super}, {"nu_excMeta", &A.nu_excMeta},
        {"nu_exc", &A.nu_exc}, {"nu_ionz", &A.nu_ionz}, {"nu_ionzStep", &A.nu_ionzStep}};
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
    cth_status st[2] = {};
    int solver_rc = 0;
    int pend[2] = {0, 0};  // MG statuses are read after the final synchronisation
    auto solve = [&](double* x, int k) -> int {
        int rc;
        if (prm->flag_iter == 0) {
            rc = sor_solve_dev(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, 1.9, prm->maxITR_SOR, prm->error_cnv_SOR, x, s,
                               &st[k]);
            if (rc > solver_rc) solver_rc = rc;
        } else {
            rc = smg_solve_launch(g, A.aP, A.aE, A.aW, A.aN, A.aS, A.b, prm->maxITR_SOR, prm->error_cnv_SOR,
                                  prm->precision, x, s, &pend[k], fs->h_solve + kStatStride * k,
                                  fs->warm_fields ? x : nullptr, fs->warm_tol, nullptr, SLOT_RHON + k);
        }
        return rc;
    };
    double* out = fs->scal + 56;
    CTH_CUDA(cudaMemsetAsync(out, 0, 4 * sizeof(double), s));
    if (prm->do_rhon) {
        k_neut_begin<0><<<grd, blk, 0, s>>>(A);
        k_rhon_assemble<<<grd, blk, 0, s>>>(A);
        g->launches += 2;
        CTH_CUDA(cudaGetLastError());
        if (solve(A.rhon, 0) < 0) return CTH_ERR_CUDA;
        k_rhon_fluxes<<<grd, blk, 0, s>>>(A);
        k_rhon_fix<<<grd, blk, 0, s>>>(A, fs->part, g->ws.counter, out);
        g->launches += 2;
    }
    if (prm->do_rhom) {
        k_neut_begin<1><<<grd, blk, 0, s>>>(A);
        k_rhom_assemble<<<grd, blk, 0, s>>>(A);
        g->launches += 2;
        CTH_CUDA(cudaGetLastError());
        if (solve(A.rhom, 1) < 0) return CTH_ERR_CUDA;
        k_rhom_fix<<<grd, blk, 0, s>>>(A);
        k_rhom_fluxes<<<grd, blk, 0, s>>>(A, fs->part, g->ws.counter, out + 2);
        g->launches += 2;
    }
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(fs->h_scal, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 2; k++) {
        if (!pend[k]) continue;
        const int rc = solve_parse(g, pend[k], fs->h_solve + kStatStride * k, &st[k]);
        if (rc < 0) return rc;
        if (rc > solver_rc) solver_rc = rc;
    }
    if (res) {
        const int m = prm->flag_error;
        res->error_rhon = finish_res(m, fs->h_scal[0], fs->h_scal[1]);
        res->error_rhom = finish_res(m, fs->h_scal[2], fs->h_scal[3]);
        res->solver_rc = solver_rc;
        res->solver[0] = st[0];
        res->solver[1] = st[1];
    }
    return CTH_OK;
}

}  // namespace cth

extern "C" int cth_update_neutrals(cth_fields* fs, const cth_neutral_params* prm, void* stream,
                                   cth_neutral_result* res) {
    if (!fs || !prm || prm->dx <= 0.0 || prm->dr <= 0.0 || prm->dt <= 0.0 || prm->ndt_n < 1 || prm->ndt_m < 1 ||
        prm->n_pos_box < 0 || prm->n_pos_box > 8 || prm->flag_error < 0 || prm->flag_error > 3) {
        cth::set_error("cth_update_neutrals: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return cth::update_neutrals(fs, prm, (cudaStream_t)stream, res);
}
