// fields.cu — device field store of the fluid state and the transport-coefficient
// update of FluidModule.
//
// A cth_fields holds named planes of the grid's library layout (cell, x-face and
// r-face arrays share the (ni+2) x (nj+2) index space as in the reference,
// fluidModule.hpp:156-173), the per-cell side-flag plane that encodes the
// reference's block-wall expressions, and the rate tables of BolsigVec
// (arrays.hpp:703-716).  Kernels take raw plane pointers.
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "fluid.cuh"
#include "line.cuh"

namespace cth {

struct TransportArgs {
    // inputs
    const double *rhoe, *rhoi, *rhon, *rhom, *Te, *Bx, *Br, *nu_ano, *Uip, *Uix, *rhoUex, *Uir, *rhoUer;
    // in/out and outputs
    double *nu_ano_IAT, *Mache, *nu_elas, *nu_exc, *nu_excReso, *nu_excMeta, *nu_ionz, *nu_ionzStep,
        *nu_excStep, *nu_super, *nu_m, *nu_m1, *rate_ionize, *nui_m, *rate_eloss, *delossdeps, *mu_para,
        *mu_xx, *mu_rr, *mu_xr, *mu_perp, *mu_min;
    Tab t_elas, t_exc, t_excReso, t_excMeta, t_ionz, t_ionzStep, t_excStep, t_super, t_eloss_n, t_eloss_m,
        t_nui;
    const unsigned char* flags;
    const double* rhoe_max;
    cth_transport_params prm;
    int ni, nj, ld;
};

// maximum of rhoe over the fluid cells (flags != 0); the last block stores it
__global__ void k_max_flagged(const double* __restrict__ v, const unsigned char* __restrict__ flags, int ni,
                              int nj, int ld, double* __restrict__ part, unsigned int* counter,
                              double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    double s[1] = {0.0};
    if (i <= ni + 1) {
        const size_t p = (size_t)j * ld + i;
        if (flags[p]) s[0] = fmax(0.0, v[p]);
    }
    grid_reduce<1>(s, 0x1u, part, counter, out);
}

// FluidModule::update_transport_coef (fluidModule.hpp:5799-5976), one thread
// per cell of the (ni+2) x (nj+2) index space
__global__ void k_transport(TransportArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const cth_transport_params& P = A.prm;
    const double dr = P.dr;
    const double rj = P.rmin + (j - 0.5) * dr;
    double iat = A.nu_ano_IAT[p];
    const unsigned char fl = A.flags[p];
    if (fl) {
        // anomalous (Sagdeev / ion-acoustic) frequency on fluid cells (:5818-5908)
        const double rhoe_max = *A.rhoe_max;
        const double bLx = (fl & F_BLX) ? 1.0 : 0.0, bRx = (fl & F_BRX) ? 1.0 : 0.0;
        const double bLr = (fl & F_BLR_WALL) ? 1.0 : 0.0, bRr = (fl & F_BRR_WALL) ? 1.0 : 0.0;
        const double Te = A.Te[p];
        const double ut = sqrt(2.0 * kBoltz * Te / P.masse);
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double rhoUex_t = (A.rhoUex[p + 1] * bRx + A.rhoUex[p] * bLx) / 2.0;
        const double rhoUer_t = (rR * A.rhoUer[p + ld] * bRr + rL * A.rhoUer[p] * bLr) / (2.0 * rj);
        const double den = A.rhoe[p] + rhoe_max * 0.001;
        const double Uex = rhoUex_t / den, Uer = rhoUer_t / den;
        const double Uix = (A.Uix[p] + A.Uix[p + 1]) / 2.0;
        const double Uir = (rL * A.Uir[p] + rR * A.Uir[p + ld]) / (2.0 * rj);
        A.Mache[p] = sqrt(Uex * Uex + Uer * Uer) / (ut + 100.0);
        const double cs = sqrt(2.0 * kBoltz * (Te + P.Ti) / P.massi);
        const double omega_pi = sqrt(A.rhoi[p] * kE0f * kE0f / (P.massi * kEps0f));
        const double ud = sqrt((Uex - Uix) * (Uex - Uix) + (Uer - Uir) * (Uer - Uir));
        iat = 0.01 * omega_pi * ud / cs * Te / P.Ti;
        A.nu_ano_IAT[p] = iat;
    }
    // collision frequencies, sources and mobility tensor on every cell (:5912-5973)
    const double Te = A.Te[p], rhon = A.rhon[p], rhom = A.rhom[p], dTe = P.dTe;
    const double elas = d_func_Te(A.t_elas.v, A.t_elas.n, Te, dTe);
    A.nu_elas[p] = rhon * elas;
    A.nu_exc[p] = rhon * d_func_Te(A.t_exc.v, A.t_exc.n, Te, dTe);
    A.nu_excReso[p] = rhon * d_func_Te(A.t_excReso.v, A.t_excReso.n, Te, dTe);
    A.nu_excMeta[p] = rhon * d_func_Te(A.t_excMeta.v, A.t_excMeta.n, Te, dTe);
    const double ionz = rhon * d_func_Te(A.t_ionz.v, A.t_ionz.n, Te, dTe);
    const double ionzStep = rhom * d_func_Te(A.t_ionzStep.v, A.t_ionzStep.n, Te, dTe);
    A.nu_ionz[p] = ionz;
    A.nu_ionzStep[p] = ionzStep;
    A.nu_excStep[p] = rhom * d_func_Te(A.t_excStep.v, A.t_excStep.n, Te, dTe);
    A.nu_super[p] = rhom * d_func_Te(A.t_super.v, A.t_super.n, Te, dTe);
    const double nu_m_real = rhon * elas;
    const double nu_m = nu_m_real + (double)P.flag_Bohm * A.nu_ano[p] + (double)P.flag_Sagdeev * iat;
    A.nu_m[p] = nu_m;
    A.nu_m1[p] = nu_m_real + P.nu_eff;
    A.rate_ionize[p] = A.rhoe[p] * (ionz + ionzStep);
    double vv = 0.0;
    if (i != 0 && i != A.ni + 1 && j != 0 && j != A.nj + 1) {
        const double rjm = P.rmin + (j - 1.5) * dr, rjp = P.rmin + (j + 0.5) * dr;
        const double rL = (rj + rjm) / 2.0, rR = (rj + rjp) / 2.0;
        const double Uix = (A.Uix[p] + A.Uix[p + 1]) / 2.0;
        const double Uir = (rL * A.Uir[p] + rR * A.Uir[p + ld]) / (2.0 * rj);
        const double Uip = A.Uip[p];
        vv = Uix * Uix + Uir * Uir + Uip * Uip;
    }
    A.nui_m[p] = rhon * d_func_Ei(A.t_nui.v, A.t_nui.n, P.massi * vv, P.dEi, P.massi);
    A.rate_eloss[p] = rhon * d_func_Te(A.t_eloss_n.v, A.t_eloss_n.n, Te, dTe) +
                      rhom * d_func_Te(A.t_eloss_m.v, A.t_eloss_m.n, Te, dTe);
    A.delossdeps[p] = 2.0 / (3.0 * kBoltz) * rhon * d_func_dTe(A.t_eloss_n.v, A.t_eloss_n.n, Te, dTe) +
                      2.0 / (3.0 * kBoltz) * rhom * d_func_dTe(A.t_eloss_m.v, A.t_eloss_m.n, Te, dTe);
    const double mu_para = kE0f / (P.masse * nu_m + 1e-100);
    A.mu_para[p] = mu_para;
    const double Bx = A.Bx[p], Br = A.Br[p];
    const double Bmag = sqrt(Bx * Bx + Br * Br);
    const double Om = kE0f * Bmag / (P.masse * nu_m + 1e-100);
    const double Omx = kE0f * Bx / (P.masse * nu_m + 1e-100);
    const double Omr = kE0f * Br / (P.masse * nu_m + 1e-100);
    const double deno = 1.0 + Om * Om;
    A.mu_xx[p] = mu_para * (1.0 + Omx * Omx) / deno;
    A.mu_rr[p] = mu_para * (1.0 + Omr * Omr) / deno;
    A.mu_xr[p] = mu_para * (Omx * Omr) / deno;
    A.mu_perp[p] = mu_para / deno;
    A.mu_min[p] = mu_para * 2.0 / deno;
}

// ghost rules, one CTA visiting the rules in order (later rules win)
__global__ void k_ghost_rules(const int* __restrict__ rules, int nrules, double* __restrict__ a, int which,
                              int ld) {
    for (int q = 0; q < nrules; q++) {
        const int* R = rules + 7 * q;
        const int wi = R[1] - R[0] + 1, wj = R[3] - R[2] + 1;
        for (int k = threadIdx.x; k < wi * wj; k += blockDim.x) {
            const int i = R[0] + k % wi, j = R[2] + k / wi;
            const size_t src = (size_t)j * ld + i;
            const size_t dst = (size_t)(j + R[5]) * ld + (i + R[4]);
            a[dst] = (which == 0 && R[6] == 0) ? 0.0 : a[src];
        }
        __syncthreads();
    }
}

void apply_ghost_rules(cth_fields* fs, double* plane, int which, cudaStream_t s) {
    if (fs->n_ghost_rules == 0) return;
    k_ghost_rules<<<1, 256, 0, s>>>(fs->ghost_rules, fs->n_ghost_rules, plane, which, fs->g->ld);
    fs->g->launches++;
}

// FluidModule::check_CFL (fluidModule.hpp:57-115): maxima of rhoe, mu_para, Te
// over the index space and of the electron speed over the grid cells
__global__ void k_cfl(const double* __restrict__ rhoe, const double* __restrict__ mu_para,
                      const double* __restrict__ Te, const double* __restrict__ rhoUex,
                      const double* __restrict__ rhoUer, double rmin, double dr, int ni, int nj, int ld,
                      double* __restrict__ part, unsigned int* counter, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (i <= ni + 1) {
        const size_t p = (size_t)j * ld + i;
        s[0] = fmax(0.0, rhoe[p]);
        s[1] = fmax(0.0, mu_para[p]);
        s[2] = fmax(0.0, Te[p]);
        if (i >= 1 && i <= ni && j >= 1 && j <= nj) {
            const double rj = rmin + (j - 0.5) * dr;
            const double rL = (rj + (rmin + (j - 1.5) * dr)) / 2.0, rR = (rj + (rmin + (j + 0.5) * dr)) / 2.0;
            const double ux = (rhoUex[p + 1] + rhoUex[p]) / 2.0 / (rhoe[p] + 1e-100);
            const double ur = (rR * rhoUer[p + ld] + rL * rhoUer[p]) / (2.0 * rj) / (rhoe[p] + 1e-100);
            s[3] = fmax(0.0, sqrt(ux * ux + ur * ur));
        }
    }
    grid_reduce<4>(s, 0xfu, part, counter, out);
}

double* field_ptr(cth_fields* fs, const std::string& name) {
    auto it = fs->planes.find(name);
    if (it != fs->planes.end()) return it->second;
    double* p = nullptr;
    const size_t bytes = fs->g->plane * sizeof(double);
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    if (cth::zero_fill(p, bytes) != cudaSuccess) { cudaFree(p); return nullptr; }
    fs->planes[name] = p;
    return p;
}

Tab table(cth_fields* fs, const char* name, bool* ok) {
    auto it = fs->tables.find(name);
    if (it == fs->tables.end() || it->second.second < 2) {
        *ok = false;
        return Tab{nullptr, 0};
    }
    return Tab{it->second.first, it->second.second};
}

int update_transport_coef(cth_fields* fs, const cth_transport_params* prm, cudaStream_t s) {
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_update_transport_coef: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    TransportArgs A;
    const char* in_names[13] = {"rhoe", "rhoi", "rhon", "rhom", "Te", "Bx", "Br", "nu_ano", "Uip", "Uix",
                                "rhoUex", "Uir", "rhoUer"};
    const double** in_ptrs[13] = {&A.rhoe, &A.rhoi, &A.rhon, &A.rhom, &A.Te, &A.Bx, &A.Br, &A.nu_ano,
                                  &A.Uip, &A.Uix, &A.rhoUex, &A.Uir, &A.rhoUer};
    for (int k = 0; k < 13; k++) {
        double* q = field_ptr(fs, in_names[k]);
        if (!q) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
        *in_ptrs[k] = q;
    }
    const char* out_names[22] = {"nu_ano_IAT", "Mache", "nu_elas", "nu_exc", "nu_excReso", "nu_excMeta",
                                 "nu_ionz", "nu_ionzStep", "nu_excStep", "nu_super", "nu_m", "nu_m1",
                                 "rate_ionize", "nui_m", "rate_eloss", "delossdeps", "mu_para", "mu_xx",
                                 "mu_rr", "mu_xr", "mu_perp", "mu_min"};
    double** out_ptrs[22] = {&A.nu_ano_IAT, &A.Mache, &A.nu_elas, &A.nu_exc, &A.nu_excReso, &A.nu_excMeta,
                             &A.nu_ionz, &A.nu_ionzStep, &A.nu_excStep, &A.nu_super, &A.nu_m, &A.nu_m1,
                             &A.rate_ionize, &A.nui_m, &A.rate_eloss, &A.delossdeps, &A.mu_para, &A.mu_xx,
                             &A.mu_rr, &A.mu_xr, &A.mu_perp, &A.mu_min};
    for (int k = 0; k < 22; k++) {
        double* q = field_ptr(fs, out_names[k]);
        if (!q) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
        *out_ptrs[k] = q;
    }
    bool ok = true;
    A.t_elas = table(fs, "nu_elas_N", &ok);
    A.t_exc = table(fs, "nu_exc_N", &ok);
    A.t_excReso = table(fs, "nu_excReso_N", &ok);
    A.t_excMeta = table(fs, "nu_excMeta_N", &ok);
    A.t_ionz = table(fs, "nu_ionz_N", &ok);
    A.t_ionzStep = table(fs, "nu_ionzStep_N", &ok);
    A.t_excStep = table(fs, "nu_excStep_N", &ok);
    A.t_super = table(fs, "nu_super_N", &ok);
    A.t_eloss_n = table(fs, "rate_eloss_n_N", &ok);
    A.t_eloss_m = table(fs, "rate_eloss_m_N", &ok);
    A.t_nui = table(fs, "nui_m_N", &ok);
    if (!ok) {
        set_error("cth_update_transport_coef: a rate table is missing (upload all eleven BolsigVec tables)");
        return CTH_ERR_ARG;
    }
    A.flags = fs->flags;
    A.rhoe_max = fs->scal;
    A.prm = *prm;
    A.ni = g->ni;
    A.nj = g->nj;
    A.ld = g->ld;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    k_max_flagged<<<grd, blk, 0, s>>>(A.rhoe, fs->flags, g->ni, g->nj, g->ld, fs->part, g->ws.counter, fs->scal);
    k_transport<<<grd, blk, 0, s>>>(A);
    g->launches += 2;
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

}  // namespace cth

using namespace cth;

extern "C" {

int cth_fields_create(cth_grid* g, cth_fields** out) {
    if (!g || !out) { set_error("cth_fields_create: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(g->device));
    cth_fields* fs = new cth_fields();
    fs->g = g;
    const int nblk = ((g->ni + 2 + 127) / 128) * (g->nj + 2) + 8;
    fs->npart = nblk * CTH_FS_NPART_PER_BLOCK;
    if (cudaMalloc(&fs->part, fs->npart * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&fs->scal, CTH_FS_NSCAL * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&fs->h_scal, CTH_FS_NSCAL * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&fs->h_solve, 8 * cth::kStatStride * sizeof(double)) != cudaSuccess) {
        if (fs->part) cudaFree(fs->part);
        if (fs->scal) cudaFree(fs->scal);
        delete fs;
        set_error("cth_fields_create: allocation failed");
        return CTH_ERR_ALLOC;
    }
    cth::zero_fill(fs->scal, CTH_FS_NSCAL * sizeof(double));
    *out = fs;
    return CTH_OK;
}

void cth_fields_destroy(cth_fields* fs) {
    if (!fs) return;
    cudaSetDevice(fs->g->device);
    restart_release(fs);
    for (auto& kv : fs->planes) cudaFree(kv.second);
    for (auto& kv : fs->tables) cudaFree(kv.second.first);
    if (fs->flags) cudaFree(fs->flags);
    if (fs->ghost_rules) cudaFree(fs->ghost_rules);
    if (fs->net_stream) cudaStreamDestroy(fs->net_stream);
    if (fs->copy_stream) {
        cudaStreamSynchronize(fs->copy_stream);
        cudaStreamDestroy(fs->copy_stream);
    }
    if (fs->copy_ready) cudaEventDestroy(fs->copy_ready);
    if (fs->copy_done) cudaEventDestroy(fs->copy_done);
    if (fs->plan_stage) cudaFree(fs->plan_stage);
    if (fs->up_stage) cudaFree(fs->up_stage);
    for (int k = 0; k < 3; k++)
        if (fs->up_ready[k]) cudaEventDestroy(fs->up_ready[k]);
    if (fs->ion_stream) cudaStreamDestroy(fs->ion_stream);
    for (int k = 0; k < 2; k++)
        if (fs->ion_event[k]) cudaEventDestroy(fs->ion_event[k]);
    for (int k = 0; k < 2; k++)
        if (fs->net_event[k]) cudaEventDestroy(fs->net_event[k]);
    if (fs->aux_ready) {
        for (int k = 0; k < 2; k++) cudaStreamDestroy(fs->aux_stream[k]);
        for (int k = 0; k < 3; k++) cudaEventDestroy(fs->aux_event[k]);
    }
    for (int k = 0; k < CTH_ION_NPROG; k++)
        if (fs->ion_ops[k]) cudaFree(fs->ion_ops[k]);
    for (int k = 0; k < 4; k++)
        if (fs->ion_boxes[k]) cudaFree(fs->ion_boxes[k]);
    if (fs->stage_many) cudaFree(fs->stage_many);
    if (fs->part) cudaFree(fs->part);
    if (fs->scal) cudaFree(fs->scal);
    if (fs->h_scal) cudaFreeHost(fs->h_scal);
    if (fs->h_solve) cudaFreeHost(fs->h_solve);
    delete fs;
}

int cth_fields_set_warm_start(cth_fields* fs, int enable, double max_relres) {
    if (!fs || !(max_relres >= 0.0 && max_relres <= 10.0)) {
        set_error("cth_fields_set_warm_start: invalid arguments (threshold in [0, 10])");
        return CTH_ERR_ARG;
    }
    fs->warm_fields = enable != 0;
    fs->warm_tol = max_relres;
    return CTH_OK;
}

double* cth_field(cth_fields* fs, const char* name) {
    if (!fs || !name) { set_error("cth_field: invalid arguments"); return nullptr; }
    cudaSetDevice(fs->g->device);
    double* p = field_ptr(fs, name);
    if (!p) set_error("cth_field: allocation failed");
    return p;
}

int cth_field_upload(cth_fields* fs, const char* name, const double* host_ij) {
    if (!fs || !name || !host_ij) { set_error("cth_field_upload: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    int rc = ensure_staging(g);
    if (rc != CTH_OK) return rc;
    double* dst = field_ptr(fs, name);
    if (!dst) { set_error("cth_field_upload: allocation failed"); return CTH_ERR_ALLOC; }
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    CTH_CUDA(cudaMemcpyAsync(g->ws.stage_ij, host_ij, nij * sizeof(double), cudaMemcpyHostToDevice, g->stream));
    rc = to_device_layout(g, g->ws.stage_ij, dst, g->stream);
    if (rc != CTH_OK) return rc;
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    return CTH_OK;
}

int cth_field_download(cth_fields* fs, const char* name, double* host_ij) {
    if (!fs || !name || !host_ij) { set_error("cth_field_download: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    int rc = ensure_staging(g);
    if (rc != CTH_OK) return rc;
    auto it = fs->planes.find(name);
    if (it == fs->planes.end()) { set_error(std::string("cth_field_download: no field ") + name); return CTH_ERR_ARG; }
    rc = from_device_layout(g, it->second, g->ws.stage_ij, g->stream);
    if (rc != CTH_OK) return rc;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    CTH_CUDA(cudaMemcpyAsync(host_ij, g->ws.stage_ij, nij * sizeof(double), cudaMemcpyDeviceToHost, g->stream));
    CTH_CUDA(cudaStreamSynchronize(g->stream));
    return CTH_OK;
}

// staging for n [i][j] planes of the batched transfers (allocated on first use)
static int ensure_stage_many(cth_fields* fs, int n) {
    if (fs->stage_planes >= n) return CTH_OK;
    cth_grid* g = fs->g;
    if (fs->stage_many) CTH_CUDA(cudaFree(fs->stage_many));
    fs->stage_many = nullptr;
    fs->stage_planes = 0;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    CTH_CUDA(cudaMalloc(&fs->stage_many, (size_t)n * nij * sizeof(double)));
    fs->stage_planes = n;
    return CTH_OK;
}

}  // extern "C"

// the sweep of the step after which a field keeps its value for the rest of the
// step (main.cpp:170-251 order: ions, potential, electron density, electron
// energy, neutrals, transport); 0: not listed, copied at the end of the step
static int final_stage(const std::string& f) {
    static const char* s1[] = {"Uix", "Uir", "Uip", "rhoi", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall"};
    static const char* s2[] = {"phi", "Ex", "Er"};
    for (const char* n : s1)
        if (f == n) return 1;
    for (const char* n : s2)
        if (f == n) return 2;
    if (f == "rhoe") return 3;
    if (f == "Te" || f == "rhoeps") return 4;
    if (f == "rhon" || f == "rhom") return 5;
    return 0;
}

int plan_flush(cth_fields* fs, int stage, cudaStream_t s) {
    if (fs->plan_names.empty()) return CTH_OK;
    cth_grid* g = fs->g;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    bool any = false;
    for (size_t k = 0; k < fs->plan_names.size(); k++) {
        if (fs->plan_queued[k]) continue;
        if (stage != 0 && final_stage(fs->plan_names[k]) != stage) continue;
        if (!any) {
            CTH_CUDA(cudaEventRecord(fs->copy_ready, s));
            CTH_CUDA(cudaStreamWaitEvent(fs->copy_stream, fs->copy_ready, 0));
            any = true;
        }
        int rc = from_device_layout(g, fs->planes.at(fs->plan_names[k]), fs->plan_stage + k * nij, fs->copy_stream);
        if (rc != CTH_OK) return rc;
        CTH_CUDA(cudaMemcpyAsync(fs->plan_host[k], fs->plan_stage + k * nij, nij * sizeof(double),
                                 cudaMemcpyDeviceToHost, fs->copy_stream));
        fs->plan_queued[k] = 1;
    }
    if (any) {
        CTH_CUDA(cudaEventRecord(fs->copy_done, fs->copy_stream));
        fs->copies_pending = true;
    }
    if (stage == 0)
        for (auto& q : fs->plan_queued) q = 0;  // the next step queues them again
    return CTH_OK;
}

int copies_wait(cth_fields* fs, cudaStream_t s) {
    if (fs->copies_pending) CTH_CUDA(cudaStreamWaitEvent(s, fs->copy_done, 0));
    return CTH_OK;
}

// the first sweep of the step that reads a field: 1 the electron energy sweep
// (rhoeps), 2 the neutral sweep (rhon, rhom; the transport update after it reads
// them too); 0 any earlier point (check_CFL, ions, potential, electron density)
static int first_read(const std::string& f) {
    if (f == "rhoeps") return 1;
    if (f == "rhon" || f == "rhom") return 2;
    return 0;
}

static int ensure_copy_stream(cth_fields* fs) {
    if (fs->copy_stream) return CTH_OK;
    CTH_CUDA(cudaStreamCreateWithFlags(&fs->copy_stream, cudaStreamNonBlocking));
    CTH_CUDA(cudaEventCreateWithFlags(&fs->copy_ready, cudaEventDisableTiming));
    CTH_CUDA(cudaEventCreateWithFlags(&fs->copy_done, cudaEventDisableTiming));
    return CTH_OK;
}

int plan_upload(cth_fields* fs, cudaStream_t s) {
    for (int k = 0; k < 3; k++) fs->up_wait[k] = false;
    if (fs->up_names.empty()) return CTH_OK;
    cth_grid* g = fs->g;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    // nothing queued before this step may still read a plane that is overwritten
    CTH_CUDA(cudaEventRecord(fs->copy_ready, s));
    CTH_CUDA(cudaStreamWaitEvent(fs->copy_stream, fs->copy_ready, 0));
    for (int grp = 0; grp < 3; grp++) {
        bool any = false;
        for (size_t k = 0; k < fs->up_names.size(); k++) {
            if (first_read(fs->up_names[k]) != grp) continue;
            CTH_CUDA(cudaMemcpyAsync(fs->up_stage + k * nij, fs->up_host[k], nij * sizeof(double),
                                     cudaMemcpyHostToDevice, fs->copy_stream));
            double* dst = field_ptr(fs, fs->up_names[k].c_str());
            if (!dst) { set_error("planned upload: allocation failed"); return CTH_ERR_ALLOC; }
            const int rc = to_device_layout(g, fs->up_stage + k * nij, dst, fs->copy_stream);
            if (rc != CTH_OK) return rc;
            any = true;
        }
        if (any) {
            CTH_CUDA(cudaEventRecord(fs->up_ready[grp], fs->copy_stream));
            fs->up_wait[grp] = true;
        }
    }
    CTH_CUDA(cudaEventRecord(fs->copy_done, fs->copy_stream));
    fs->copies_pending = true;
    fs->up_names.clear();  // one step
    fs->up_host.clear();
    return upload_wait(fs, 0, s);
}

int upload_wait(cth_fields* fs, int group, cudaStream_t s) {
    if (fs->up_wait[group]) {
        CTH_CUDA(cudaStreamWaitEvent(s, fs->up_ready[group], 0));
        fs->up_wait[group] = false;
    }
    return CTH_OK;
}

extern "C" {

int cth_fields_set_download_plan(cth_fields* fs, const char* const* names, double* const* host_ij, int n) {
    if (!fs || n < 0 || (n > 0 && (!names || !host_ij))) {
        set_error("cth_fields_set_download_plan: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    if (fs->copies_pending) {
        CTH_CUDA(cudaStreamSynchronize(fs->copy_stream));
        fs->copies_pending = false;
    }
    std::vector<std::string> nm;
    std::vector<double*> hp;
    for (int k = 0; k < n; k++) {
        if (!names[k] || !host_ij[k] || fs->planes.find(names[k]) == fs->planes.end()) {
            set_error(std::string("cth_fields_set_download_plan: no field ") + (names[k] ? names[k] : "(null)"));
            return CTH_ERR_ARG;
        }
        nm.emplace_back(names[k]);
        hp.push_back(host_ij[k]);
    }
    if (n > fs->plan_cap) {
        if (fs->plan_stage) CTH_CUDA(cudaFree(fs->plan_stage));
        fs->plan_stage = nullptr;
        fs->plan_cap = 0;
        const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
        CTH_CUDA(cudaMalloc(&fs->plan_stage, (size_t)n * nij * sizeof(double)));
        fs->plan_cap = n;
    }
    {
        const int rce = ensure_copy_stream(fs);
        if (rce != CTH_OK) return rce;
    }
    fs->plan_names = nm;
    fs->plan_host = hp;
    fs->plan_queued.assign(n, 0);
    return CTH_OK;
}

int cth_fields_set_upload_plan(cth_fields* fs, const char* const* names, const double* const* host_ij, int n) {
    if (!fs || n < 0 || (n > 0 && (!names || !host_ij))) {
        set_error("cth_fields_set_upload_plan: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    std::vector<std::string> nm;
    std::vector<const double*> hp;
    for (int k = 0; k < n; k++) {
        if (!names[k] || !host_ij[k]) {
            set_error("cth_fields_set_upload_plan: null name or array");
            return CTH_ERR_ARG;
        }
        nm.emplace_back(names[k]);
        hp.push_back(host_ij[k]);
    }
    if (n > fs->up_cap) {
        if (fs->copies_pending) CTH_CUDA(cudaStreamSynchronize(fs->copy_stream));
        if (fs->up_stage) CTH_CUDA(cudaFree(fs->up_stage));
        fs->up_stage = nullptr;
        fs->up_cap = 0;
        const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
        CTH_CUDA(cudaMalloc(&fs->up_stage, (size_t)n * nij * sizeof(double)));
        fs->up_cap = n;
    }
    {
        const int rce = ensure_copy_stream(fs);
        if (rce != CTH_OK) return rce;
    }
    for (int k = 0; k < 3; k++)
        if (!fs->up_ready[k]) CTH_CUDA(cudaEventCreateWithFlags(&fs->up_ready[k], cudaEventDisableTiming));
    fs->up_names = nm;
    fs->up_host = hp;
    return CTH_OK;
}

int cth_fields_download_wait(cth_fields* fs) {
    if (!fs) {
        set_error("cth_fields_download_wait: null store");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    if (fs->copies_pending) CTH_CUDA(cudaStreamSynchronize(fs->copy_stream));
    fs->copies_pending = false;
    return CTH_OK;
}

int cth_fields_upload_many(cth_fields* fs, const char* const* names, const double* const* host_ij, int n,
                           void* stream) {
    if (!fs || !names || !host_ij || n < 1) { set_error("cth_fields_upload_many: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    {
        // planned downloads still reading the planes finish first
        const int rcw = copies_wait(fs, stream ? (cudaStream_t)stream : g->stream);
        if (rcw != CTH_OK) return rcw;
    }
    int rc = ensure_stage_many(fs, n);
    if (rc != CTH_OK) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    for (int k = 0; k < n; k++) {
        if (!names[k] || !host_ij[k]) { set_error("cth_fields_upload_many: null name or array"); return CTH_ERR_ARG; }
        CTH_CUDA(cudaMemcpyAsync(fs->stage_many + k * nij, host_ij[k], nij * sizeof(double), cudaMemcpyHostToDevice,
                                 s));
    }
    for (int k = 0; k < n; k++) {
        double* dst = field_ptr(fs, names[k]);
        if (!dst) { set_error("cth_fields_upload_many: allocation failed"); return CTH_ERR_ALLOC; }
        rc = to_device_layout(g, fs->stage_many + k * nij, dst, s);
        if (rc != CTH_OK) return rc;
    }
    CTH_CUDA(cudaStreamSynchronize(s));
    return CTH_OK;
}

int cth_fields_download_many(cth_fields* fs, const char* const* names, double* const* host_ij, int n, void* stream) {
    if (!fs || !names || !host_ij || n < 1) {
        set_error("cth_fields_download_many: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    int rc = ensure_stage_many(fs, n);
    if (rc != CTH_OK) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    const size_t nij = (size_t)(g->ni + 2) * (g->nj + 2);
    for (int k = 0; k < n; k++) {
        if (!names[k] || !host_ij[k]) { set_error("cth_fields_download_many: null name or array"); return CTH_ERR_ARG; }
        auto it = fs->planes.find(names[k]);
        if (it == fs->planes.end()) {
            set_error(std::string("cth_fields_download_many: no field ") + names[k]);
            return CTH_ERR_ARG;
        }
        rc = from_device_layout(g, it->second, fs->stage_many + k * nij, s);
        if (rc != CTH_OK) return rc;
    }
    for (int k = 0; k < n; k++)
        CTH_CUDA(cudaMemcpyAsync(host_ij[k], fs->stage_many + k * nij, nij * sizeof(double), cudaMemcpyDeviceToHost,
                                 s));
    CTH_CUDA(cudaStreamSynchronize(s));
    return CTH_OK;
}

int cth_flags_upload(cth_fields* fs, const unsigned char* host_ij) {
    if (!fs || !host_ij) { set_error("cth_flags_upload: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    std::vector<unsigned char> lay(g->plane, 0);
    // the ghost frame never carries a fluid cell (the kernels read its neighbours)
    for (int i = 1; i <= g->ni; i++)
        for (int j = 1; j <= g->nj; j++) lay[(size_t)j * g->ld + i] = host_ij[(size_t)i * (g->nj + 2) + j];
    if (!fs->flags) CTH_CUDA(cudaMalloc(&fs->flags, g->plane));
    CTH_CUDA(cudaMemcpy(fs->flags, lay.data(), g->plane, cudaMemcpyHostToDevice));
    return CTH_OK;
}

int cth_ghost_rules_upload(cth_fields* fs, const int* rules, int n) {
    if (!fs || n < 0 || (n > 0 && !rules)) { set_error("cth_ghost_rules_upload: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    for (int q = 0; q < n; q++) {
        const int* R = rules + 7 * q;
        const bool x = (R[4] == 1 || R[4] == -1) && R[5] == 0 && R[0] == R[1];
        const bool r = (R[5] == 1 || R[5] == -1) && R[4] == 0 && R[2] == R[3];
        const bool in = R[0] <= R[1] && R[2] <= R[3] && R[0] >= 1 && R[1] <= g->ni && R[2] >= 1 && R[3] <= g->nj;
        if (!(x || r) || !in || (R[6] != 0 && R[6] != 1)) {
            set_error("cth_ghost_rules_upload: a rule must be a one-cell-wide segment of grid cells with a unit "
                      "offset across it and mode 0 or 1");
            return CTH_ERR_ARG;
        }
    }
    CTH_CUDA(cudaSetDevice(g->device));
    if (fs->ghost_rules) { cudaFree(fs->ghost_rules); fs->ghost_rules = nullptr; }
    fs->n_ghost_rules = 0;
    if (n == 0) return CTH_OK;
    CTH_CUDA(cudaMalloc(&fs->ghost_rules, 7 * n * sizeof(int)));
    CTH_CUDA(cudaMemcpy(fs->ghost_rules, rules, 7 * n * sizeof(int), cudaMemcpyHostToDevice));
    fs->n_ghost_rules = n;
    return CTH_OK;
}

int cth_energy_keep_walls_upload(cth_fields* fs, const int* boxes, int n) {
    if (!fs || n < 0 || n > CTH_KEEP_WALL_MAX || (n > 0 && !boxes)) {
        set_error("cth_energy_keep_walls_upload: invalid arguments (at most 4 boxes)");
        return CTH_ERR_ARG;
    }
    const cth_grid* g = fs->g;
    for (int q = 0; q < n; q++) {
        const int* B = boxes + 4 * q;
        if (!(B[0] <= B[1] && B[2] <= B[3] && B[0] >= 0 && B[1] <= g->ni + 1 && B[2] >= 0 && B[3] <= g->nj + 1)) {
            set_error("cth_energy_keep_walls_upload: a box must be a non-empty range of the index space");
            return CTH_ERR_ARG;
        }
    }
    for (int q = 0; q < 4 * n; q++) fs->keep_wall[q] = boxes[q];
    fs->n_keep_wall = n;
    return CTH_OK;
}

int cth_check_cfl(cth_fields* fs, cth_cfl* io, void* stream) {
    if (!fs || !io) { set_error("cth_check_cfl: invalid arguments"); return CTH_ERR_ARG; }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    const char* names[5] = {"rhoe", "mu_para", "Te", "rhoUex", "rhoUer"};
    double* q[5];
    for (int k = 0; k < 5; k++) {
        q[k] = field_ptr(fs, names[k]);
        if (!q[k]) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    cudaStream_t s = (cudaStream_t)stream;
    dim3 blk(128), grd((g->ni + 2 + 127) / 128, g->nj + 2);
    k_cfl<<<grd, blk, 0, s>>>(q[0], q[1], q[2], q[3], q[4], io->rmin, io->dr, g->ni, g->nj, g->ld, fs->part,
                              g->ws.counter, fs->scal + 40);
    g->launches++;
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaMemcpyAsync(fs->h_scal, fs->scal + 40, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CTH_CUDA(cudaStreamSynchronize(s));
    const double* h = fs->h_scal;
    io->rhoe_max = h[0];
    io->mu_max = h[1];
    io->Te_max = h[2];
    io->ue_max = h[3] + sqrt(8.0 * kBoltz * h[2] / (M_PI * io->masse));
    io->dt_min = kEps0f / (kE0f * h[0] * h[1]);
    if (io->flag_adp_dt == 1)
        io->dt = io->dt_min * io->CFL;
    else
        io->CFL = io->dt / io->dt_min;
    return CTH_OK;
}

int cth_table_upload(cth_fields* fs, const char* name, const double* values, int n) {
    if (!fs || !name || !values || n < 2) { set_error("cth_table_upload: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    auto it = fs->tables.find(name);
    if (it != fs->tables.end()) {
        cudaFree(it->second.first);
        fs->tables.erase(it);
    }
    double* d = nullptr;
    CTH_CUDA(cudaMalloc(&d, n * sizeof(double)));
    CTH_CUDA(cudaMemcpy(d, values, n * sizeof(double), cudaMemcpyHostToDevice));
    fs->tables[name] = std::make_pair(d, n);
    return CTH_OK;
}

int cth_update_transport_coef(cth_fields* fs, const cth_transport_params* prm, void* stream) {
    if (!fs || !prm || prm->dTe <= 0.0 || prm->dEi <= 0.0) {
        set_error("cth_update_transport_coef: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(fs->g->device));
    return update_transport_coef(fs, prm, (cudaStream_t)stream);
}

}  // extern "C"
