// mwupdate.cu — the microwave update at the end of the reference's time loop
// (src/main.cpp:254-257: every ndiv_MW steps EmfieldModule::solve_Microwave, then
// update_energy_profile) as one call on a discharge's device state: assembly of
// the magnetised system from the store's n_e, nu_m1, Bx, Br and epsr_mw planes,
// the solve, the ghost pass, the absorbed power (J, Pabs, the integrals) and the
// port / rescale part, which scales the store's Pabs to Pmw and the excitation
// current J1r_exc by the root of the ratio for the next update.  The handle holds
// the excitation current and the field and current planes (the caller's, or its
// own), which persist between updates as the reference's fields do.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>

#include "fluid.cuh"

struct cth_mw_update {
    cth_fields* fs = nullptr;
    cth_mw3* m = nullptr;
    int device = 0, ndiv = 100, maxit = 400, warm = 0, runs = 0;
    bool prepared = false;     // the solve's hierarchy and graph are built
    double tol = 1e-10;
    cth_mw_params mw{};
    cth_energy_params ep{};
    cth_mw_port_params port{};
    double J1r_exc = 0.0;      // the excitation of the next solve
    double J_solved = 0.0;     // the excitation the fields in E3 were solved with
    size_t pl = 0;         // complex entries of one plane
    double* E3 = nullptr;  // 3 complex planes (E1x, E1r, E1p)
    double* J3 = nullptr;  // 3 complex planes (J1x, J1r, J1p)
    bool own_E = false, own_J = false;
    cth_unet* net = nullptr;   // learned guess (9 input, 6 output channels) or none
    double* G3 = nullptr;      // 3 complex planes: the network's guess
};

using cth::set_error;

namespace {
// dst = ratio * src over n complex entries (the previous fields scaled to the new excitation)
__global__ void k_scale_planes(const double* __restrict__ src, double ratio, double* __restrict__ dst, size_t n) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = ratio * src[k];
}
}  // namespace

extern "C" int cth_mw_update_create(cth_fields* fs, cth_mw3* m, const cth_mw_update_params* p, double* E3,
                                    double* J3, cth_mw_update** out) {
    if (!fs || !m || !p || !out || p->ndiv_mw < 1 || p->maxit < 1 || !(p->tol > 0.0)) {
        set_error("cth_mw_update_create: invalid arguments");
        return CTH_ERR_ARG;
    }
    *out = nullptr;
    const int ld = cth_mw3_ld(m);
    if (ld != fs->g->ld || fs->g->ni < 1) {
        set_error("cth_mw_update_create: the microwave system and the field store differ in layout");
        return CTH_ERR_ARG;
    }
    cth_mw_update* u = new (std::nothrow) cth_mw_update();
    if (!u) {
        set_error("cth_mw_update_create: out of host memory");
        return CTH_ERR_ALLOC;
    }
    u->fs = fs;
    u->m = m;
    u->device = fs->g->device;
    u->ndiv = p->ndiv_mw;
    u->maxit = p->maxit;
    u->tol = p->tol;
    u->warm = p->warm_start;
    u->mw = p->mw;
    u->port = p->port;
    u->ep = cth_energy_params{p->mw.dx, p->mw.dr, p->mw.rmin, p->mw.omegam, p->mw.masse};
    u->J1r_exc = p->mw.J1r_exc;
    u->pl = (size_t)(fs->g->nj + 2) * ld;
    const size_t bytes = 3 * u->pl * 2 * sizeof(double);
    cudaError_t e = cudaSetDevice(u->device);
    u->E3 = E3;
    u->J3 = J3;
    if (e == cudaSuccess && !E3) {
        u->own_E = true;
        e = cudaMalloc(&u->E3, bytes);
        if (e == cudaSuccess) e = cth::zero_fill(u->E3, bytes);
    }
    if (e == cudaSuccess && !J3) {
        u->own_J = true;
        e = cudaMalloc(&u->J3, bytes);
        if (e == cudaSuccess) e = cth::zero_fill(u->J3, bytes);
    }
    if (e != cudaSuccess) {
        cth_mw_update_destroy(u);
        return cth::cuda_fail(e, "cth_mw_update_create");
    }
    // every store plane the update reads or writes exists from here on, so that no
    // later run allocates (runs may come from the worker threads of a batch)
    for (const char* name : {"rhoe", "nu_m1", "Bx", "Br", "epsr_mw", "Er", "Pabsx", "Pabsr", "Pabsp", "Pabs"}) {
        if (!cth_field(fs, name)) {
            cth_mw_update_destroy(u);
            return CTH_ERR_ALLOC;
        }
    }
    *out = u;
    return CTH_OK;
}

extern "C" void cth_mw_update_destroy(cth_mw_update* u) {
    if (!u) return;
    cudaSetDevice(u->device);
    if (u->own_E && u->E3) cudaFree(u->E3);
    if (u->own_J && u->J3) cudaFree(u->J3);
    if (u->G3) cudaFree(u->G3);
    delete u;
}

extern "C" int cth_mw_update_set_net(cth_mw_update* u, cth_unet* net) {
    if (!u) {
        set_error("cth_mw_update_set_net: invalid arguments");
        return CTH_ERR_ARG;
    }
    u->net = net;
    return CTH_OK;
}

extern "C" int cth_mw_update_due(const cth_mw_update* u, int itime) {
    return (u && itime > 0 && itime % u->ndiv == 0) ? 1 : 0;
}

extern "C" double* cth_mw_update_plane(cth_mw_update* u, int which) {
    if (!u || which < 0 || which > 5) return nullptr;
    return (which < 3 ? u->E3 : u->J3) + (size_t)(which % 3) * u->pl * 2;
}

extern "C" int cth_mw_update_prepare(cth_mw_update* u, void* stream) {
    if (!u) {
        set_error("cth_mw_update_prepare: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_fields* fs = u->fs;
    const double* ne = cth_field(fs, "rhoe");
    const double* nu = cth_field(fs, "nu_m1");
    const double* Bx = cth_field(fs, "Bx");
    const double* Br = cth_field(fs, "Br");
    const double* epsr = cth_field(fs, "epsr_mw");
    if (!ne || !nu || !Bx || !Br || !epsr) {
        set_error("cth_mw_update_prepare: the store lacks a plane the update reads");
        return CTH_ERR_ARG;
    }
    cth_mw_params prm = u->mw;
    prm.J1r_exc = u->J1r_exc;
    int rc = cth_mw3_assemble_dev(u->m, ne, nu, Bx, Br, epsr, &prm, stream);
    if (rc < 0) return rc;
    cth_status st{};
    rc = cth_mw3_solve_dev(u->m, u->maxit, u->tol, u->E3, stream, &st);
    if (rc < 0) return rc;
    u->prepared = true;
    return CTH_OK;
}

extern "C" int cth_mw_update_prepared(const cth_mw_update* u) { return (u && u->prepared) ? 1 : 0; }

extern "C" int cth_mw_update_run(cth_mw_update* u, cth_grid* gx, cth_grid* gr, void* stream,
                                 cth_mw_update_result* res) {
    if (!u || !gx || !gr) {
        set_error("cth_mw_update_run: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_fields* fs = u->fs;
    const double* ne = cth_field(fs, "rhoe");
    const double* nu = cth_field(fs, "nu_m1");
    const double* Bx = cth_field(fs, "Bx");
    const double* Br = cth_field(fs, "Br");
    const double* epsr = cth_field(fs, "epsr_mw");
    const double* Er = cth_field(fs, "Er");
    if (!ne || !nu || !Bx || !Br || !epsr || !Er) {
        set_error("cth_mw_update_run: the store lacks a plane the update reads (rhoe, nu_m1, Bx, Br, epsr_mw, Er)");
        return CTH_ERR_ARG;
    }
    cth_mw_params prm = u->mw;
    prm.J1r_exc = u->J1r_exc;
    int rc = cth_mw3_assemble_dev(u->m, ne, nu, Bx, Br, epsr, &prm, stream);
    if (rc < 0) return rc;
    cth_status st{};
    // the start: the network's guess (the previous fields plus its predicted change),
    // else the previous fields, else zero; a guess is taken only when its residual
    // is at most ||b|| (decided on the device)
    const double* x0 = nullptr;
    if (u->runs > 0 && (u->net || u->warm) && u->J_solved != 0.0) {
        if (!u->G3) {
            CTH_CUDA(cudaMalloc(&u->G3, 3 * u->pl * 2 * sizeof(double)));
            CTH_CUDA(cth::zero_fill(u->G3, 3 * u->pl * 2 * sizeof(double)));
        }
        if (u->net) {
            rc = cth_unet_mw_guess(u->net, fs, u->E3, u->J_solved, prm.J1r_exc, u->G3, stream);
            if (rc < 0) return rc;
        } else {
            const size_t n = 3 * u->pl;
            k_scale_planes<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0,
                             static_cast<cudaStream_t>(stream)>>>(u->E3, prm.J1r_exc / u->J_solved, u->G3, n);
            CTH_CUDA(cudaGetLastError());
        }
        x0 = u->G3;
    }
    const int rs = cth_mw3_solve_guess_dev(u->m, u->maxit, u->tol, u->E3, x0, 1.0, stream, &st);
    if (rs < 0) return rs;
    u->runs++;
    u->J_solved = prm.J1r_exc;
    rc = cth_mw3_fill_ghosts(u->m, u->E3, epsr, Er, &prm, stream);
    if (rc < 0) return rc;
    cth_energy_result er{};
    rc = cth_update_energy_profile(fs, gx, gr, &u->ep, cth_mw_update_plane(u, 0), cth_mw_update_plane(u, 1),
                                   cth_mw_update_plane(u, 2), cth_mw_update_plane(u, 3), cth_mw_update_plane(u, 4),
                                   cth_mw_update_plane(u, 5), stream, &er);
    if (rc < 0) return rc;
    cth_mw_port_result pr{};
    rc = cth_mw_port_rescale(fs, &u->port, er.power_sum, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                             nullptr, nullptr, nullptr, stream, &pr);
    if (rc < 0) return rc;
    if (rc == CTH_OK) u->J1r_exc *= pr.J1r_exc_factor;
    if (res) {
        res->solve = st;
        res->power_sum = er.power_sum;
        res->ratio = pr.ratio;
        res->J1r_exc = u->J1r_exc;
        res->rescale_rc = rc;
    }
    return rs > 0 ? rs : rc;
}
