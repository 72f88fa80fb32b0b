// cathode_emfield.hpp — header-only C++ drop-in for the reference's microwave update.
//
// Include this header in place of include/emfieldModule.hpp, after the
// reference's params.hpp and arrays.hpp (its Params, GridCenter,
// GridInterfaceX, GridInterfaceR and MicrowaveBC types), and link
// libcathode_b200.so and the CUDA runtime: the calls of src/main.cpp:154-155,
// :255-256
//     emfM.solve_Microwave(pm, gc, gx, gr, mb);
//     emfM.update_energy_profile(pm, gc, gx, gr);
// compile unchanged and run on the GPU.  Signatures are those of
// emfieldModule.hpp:74 and :79; the other members of the reference's
// EmfieldModule (the impedance test, which cth_mw_impedance_test covers, and the
// plotting helpers) are not part of this header; solve_Microwave_explicit
// (:3328-4400) is.
//
// solve_Microwave (emfieldModule.hpp:2249-3321): the magnetised 3-component
// system on the unknowns of the six x-face / r-face / cell blocks
// (gx.i_flx_bl, gr.i_flr_bl, gc.i_flc_bl), the 12 MicrowaveBC lists with codes
// 0-7 in the reference's order, the solve (complex FP64 BiCGStab with one
// complex semicoarsening V-cycle per field as preconditioner, to error_cnv, in
// place of Eigen SparseLU) and the ghost post-processing of E1x, E1r, E1p.
// Writes gx.E1x, gr.E1r, gc.E1p; their ghosts persist between calls as in the
// reference.  Reads gc.rhoe, gc.nu_m1, gc.Bx, gc.Br, gc.epsr, gr.Er (the Er
// east code 1 ghost reads the static field, :3162), pm.dx, dr, rmin, omegam,
// J1r_exc, r1, r2, masse and gc.j_flc_bl[0][0] (:2672).
//
// update_energy_profile (:7630-8105): J = sigma E on the six blocks, the
// absorbed power planes and their integrals, then with pm.flag_mwRef the port
// current and voltage at the reference plane, de-embedding through pm.S11..S22
// for pm.Z0, and the rescale to pm.Pmw of gc.Pabs, the fields, the currents and
// the excitation currents (gx.J1x_exc, gr.J1r_exc, gc.J1p_exc); pm.J1r_exc is
// multiplied by the square root of the power ratio (:8016).  Writes gx.J1x,
// gr.J1r, gc.J1p, gx.Pabsx, gr.Pabsr, gc.Pabsp, gc.Pabs and the rescaled fields.
//
// The reference returns no status; here CUDA or argument failures throw
// std::runtime_error and last_status holds the solve's iterations and
// residual (a solve that does not reach error_cnv in maxITR iterations is
// reported there, not thrown, as the reference's SparseLU info is unchecked).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "cathode_b200.h"

namespace cathode_b200 {

inline void check_rc(int rc, const char* what) {
    if (rc < 0) throw std::runtime_error(std::string(what) + ": " + cth_last_error());
}

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// device state of one EmfieldModule: the solver, the three six-block grids of the
// energy profile, a field store for the real planes and nine complex planes
struct EmfieldDevice {
    int ni = -1, nj = -1, ld = 0, device = 0;
    std::vector<int> blocks;          // the six blocks of the three index sets, to detect a change
    cth_mw3* m = nullptr;
    cth_grid *gc = nullptr, *gx = nullptr, *gr = nullptr;
    cth_fields* fs = nullptr;
    void* cplx = nullptr;             // E1x E1r E1p | J1x J1r J1p | J1x_exc J1r_exc J1p_exc
    size_t cplane = 0;                // bytes of one complex plane
    std::vector<double> stage;        // host staging of one complex plane (library layout)
    std::vector<double> flat;         // host [i][j] staging of one real plane

    void release() {
        if (fs) cth_fields_destroy(fs);
        if (gc) cth_grid_destroy(gc);
        if (gx) cth_grid_destroy(gx);
        if (gr) cth_grid_destroy(gr);
        if (m) cth_mw3_destroy(m);
        if (cplx) cudaFree(cplx);
        fs = nullptr; gc = gx = gr = nullptr; m = nullptr; cplx = nullptr; ni = nj = -1;
    }
    double* plane(int k) const { return reinterpret_cast<double*>(static_cast<char*>(cplx) + k * cplane); }
};

template <class VV>
inline void put_real(EmfieldDevice& d, const char* name, const VV& a) {
    const size_t C = (size_t)d.nj + 2;
    for (int i = 0; i < d.ni + 2; i++) std::memcpy(&d.flat[i * C], a[i].data(), C * sizeof(double));
    check_rc(cth_field_upload(d.fs, name, d.flat.data()), name);
}

template <class VV>
inline void get_real(EmfieldDevice& d, const char* name, VV& a) {
    const size_t C = (size_t)d.nj + 2;
    check_rc(cth_field_download(d.fs, name, d.flat.data()), name);
    for (int i = 0; i < d.ni + 2; i++) std::memcpy(a[i].data(), &d.flat[i * C], C * sizeof(double));
}

// [i][j] complex <-> library layout (j * ld + i, re / im interleaved)
template <class VC>
inline void put_cplx(EmfieldDevice& d, int k, const VC& a) {
    std::fill(d.stage.begin(), d.stage.end(), 0.0);
    for (int i = 0; i < d.ni + 2; i++)
        for (int j = 0; j < d.nj + 2; j++) {
            const size_t p = 2 * ((size_t)j * d.ld + i);
            d.stage[p] = a[i][j].real();
            d.stage[p + 1] = a[i][j].imag();
        }
    check_cuda(cudaMemcpy(d.plane(k), d.stage.data(), d.cplane, cudaMemcpyHostToDevice), "cudaMemcpy");
}

template <class VC>
inline void get_cplx(EmfieldDevice& d, int k, VC& a) {
    check_cuda(cudaMemcpy(d.stage.data(), d.plane(k), d.cplane, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int i = 0; i < d.ni + 2; i++)
        for (int j = 0; j < d.nj + 2; j++) {
            const size_t p = 2 * ((size_t)j * d.ld + i);
            a[i][j] = std::complex<double>(d.stage[p], d.stage[p + 1]);
        }
}

}  // namespace cathode_b200

class EmfieldModule {
   public:
    int maxITR = 2000;         // iteration cap of the solve
    double error_cnv = 1e-12;  // relative residual ||b - A E|| / ||b|| the solve reaches
    int device = 0;            // CUDA device of the solve
    cth_status last_status{};  // the last solve's iterations, residual and convergence

    EmfieldModule() = default;
    ~EmfieldModule() { d_.release(); }
    EmfieldModule(const EmfieldModule&) = delete;
    EmfieldModule& operator=(const EmfieldModule&) = delete;

    // EmfieldModule::solve_Microwave (emfieldModule.hpp:74, :2249-3321)
    void solve_Microwave(Params& pm, GridCenter& gc, GridInterfaceX& gx, GridInterfaceR& gr, MicrowaveBC& mb) {
        using namespace cathode_b200;
        prepare(pm, gc, gx, gr, mb);
        const cth_mw_params prm = mw_params(pm);
        check_rc(cth_mw3_assemble_dev(d_.m, cth_field(d_.fs, "rhoe"), cth_field(d_.fs, "nu_m1"),
                                      cth_field(d_.fs, "Bx"), cth_field(d_.fs, "Br"), cth_field(d_.fs, "epsr"), &prm,
                                      nullptr),
                 "cth_mw3_assemble_dev");
        finish(gc, gx, gr, prm);
    }

    // EmfieldModule::solve_Microwave_explicit (emfieldModule.hpp:3328-4400): the plasma current
    // J = sigma E of the present field on the right-hand side, a vacuum + epsr operator, then the
    // same boundary lists, solve and ghost pass.  Writes gx.J1x, gr.J1r, gc.J1p (the J used) and
    // the new gx.E1x, gr.E1r, gc.E1p.
    void solve_Microwave_explicit(Params& pm, GridCenter& gc, GridInterfaceX& gx, GridInterfaceR& gr,
                                  MicrowaveBC& mb) {
        using namespace cathode_b200;
        prepare(pm, gc, gx, gr, mb);
        put_cplx(d_, 3, gx.J1x);   // entries off the blocks keep the caller's values
        put_cplx(d_, 4, gr.J1r);
        put_cplx(d_, 5, gc.J1p);
        const cth_mw_params prm = mw_params(pm);
        // J = sigma E (:3384-3470): the same formulas as the energy profile's currents
        cth_energy_params ep{pm.dx, pm.dr, pm.rmin, pm.omegam, pm.masse};
        cth_energy_result er{};
        check_rc(cth_update_energy_profile(d_.fs, d_.gx, d_.gr, &ep, d_.plane(0), d_.plane(1), d_.plane(2),
                                           d_.plane(3), d_.plane(4), d_.plane(5), nullptr, &er),
                 "cth_update_energy_profile");
        check_rc(cth_mw3_assemble_explicit_dev(d_.m, cth_field(d_.fs, "epsr"), d_.plane(3), d_.plane(4), d_.plane(5),
                                               &prm, nullptr),
                 "cth_mw3_assemble_explicit_dev");
        finish(gc, gx, gr, prm);
        get_cplx(d_, 3, gx.J1x);
        get_cplx(d_, 4, gr.J1r);
        get_cplx(d_, 5, gc.J1p);
    }

    // EmfieldModule::update_energy_profile (emfieldModule.hpp:79, :7630-8105)
    void update_energy_profile(Params& pm, GridCenter& gc, GridInterfaceX& gx, GridInterfaceR& gr) {
        using namespace cathode_b200;
        setup(pm, gc, gx, gr);
        put_real(d_, "rhoe", gc.rhoe);
        put_real(d_, "nu_m1", gc.nu_m1);
        put_real(d_, "Bx", gc.Bx);
        put_real(d_, "Br", gc.Br);
        // the planes written on the block cells only keep the caller's values elsewhere
        put_real(d_, "Pabs", gc.Pabs);
        put_real(d_, "Pabsx", gx.Pabsx);
        put_real(d_, "Pabsr", gr.Pabsr);
        put_real(d_, "Pabsp", gc.Pabsp);
        put_cplx(d_, 0, gx.E1x);
        put_cplx(d_, 1, gr.E1r);
        put_cplx(d_, 2, gc.E1p);
        put_cplx(d_, 3, gx.J1x);
        put_cplx(d_, 4, gr.J1r);
        put_cplx(d_, 5, gc.J1p);
        put_cplx(d_, 6, gx.J1x_exc);
        put_cplx(d_, 7, gr.J1r_exc);
        put_cplx(d_, 8, gc.J1p_exc);
        cth_energy_params ep{pm.dx, pm.dr, pm.rmin, pm.omegam, pm.masse};
        cth_energy_result er{};
        check_rc(cth_update_energy_profile(d_.fs, d_.gx, d_.gr, &ep, d_.plane(0), d_.plane(1), d_.plane(2),
                                           d_.plane(3), d_.plane(4), d_.plane(5), nullptr, &er),
                 "cth_update_energy_profile");
        cth_mw_port_params pp{};
        pp.dx = pm.dx;
        pp.dr = pm.dr;
        pp.rmin = pm.rmin;
        pp.omegam = pm.omegam;
        pp.r1 = pm.r1;
        pp.r2 = pm.r2;
        pp.Z0 = pm.Z0;
        pp.Pmw = pm.Pmw;
        const std::complex<double> S[4] = {pm.S11, pm.S21, pm.S12, pm.S22};
        double* dst[4] = {pp.S11, pp.S21, pp.S12, pp.S22};
        for (int k = 0; k < 4; k++) {
            dst[k][0] = S[k].real();
            dst[k][1] = S[k].imag();
        }
        pp.flag_mwRef = pm.flag_mwRef;
        pp.i_ref = int(0.0 / pm.dx + 0.5) + 1;              // x_ref = 0 (:7800-7801)
        pp.j_out = gc.j_flc_bl[4][1] - 1;                   // mWLoss_at_boundary_rR at x5 (:7853)
        pp.i_out0 = gc.i_flc_bl[4][0];
        pp.i_out1 = gc.i_flc_bl[4][1];
        pp.jf0 = gr.j_flr_bl[pm.n_bl - 1][0];               // the feed's Er faces
        pp.jf1 = gr.j_flr_bl[pm.n_bl - 1][1];
        cth_mw_port_result pr{};
        check_rc(cth_mw_port_rescale(d_.fs, &pp, er.power_sum, d_.plane(0), d_.plane(1), d_.plane(2), d_.plane(3),
                                     d_.plane(4), d_.plane(5), d_.plane(6), d_.plane(7), d_.plane(8), nullptr, &pr),
                 "cth_mw_port_rescale");
        pm.J1r_exc = pm.J1r_exc * pr.J1r_exc_factor;
        last_port = pr;
        get_cplx(d_, 0, gx.E1x);
        get_cplx(d_, 1, gr.E1r);
        get_cplx(d_, 2, gc.E1p);
        get_cplx(d_, 3, gx.J1x);
        get_cplx(d_, 4, gr.J1r);
        get_cplx(d_, 5, gc.J1p);
        get_cplx(d_, 6, gx.J1x_exc);
        get_cplx(d_, 7, gr.J1r_exc);
        get_cplx(d_, 8, gc.J1p_exc);
        get_real(d_, "Pabs", gc.Pabs);
        get_real(d_, "Pabsx", gx.Pabsx);
        get_real(d_, "Pabsr", gr.Pabsr);
        get_real(d_, "Pabsp", gc.Pabsp);
    }

    cth_mw_port_result last_port{};  // the quantities the reference prints after the rescale

   private:
    cathode_b200::EmfieldDevice d_;

    // device state, the 12 boundary lists, the real planes and the present field (ghosts included)
    void prepare(Params& pm, GridCenter& gc, GridInterfaceX& gx, GridInterfaceR& gr, MicrowaveBC& mb) {
        using namespace cathode_b200;
        setup(pm, gc, gx, gr);
        const std::vector<int>* L[12][3] = {
            {&mb.iBndWx, &mb.jBndWx, &mb.sBndWx}, {&mb.iBndEx, &mb.jBndEx, &mb.sBndEx},
            {&mb.iBndSx, &mb.jBndSx, &mb.sBndSx}, {&mb.iBndNx, &mb.jBndNx, &mb.sBndNx},
            {&mb.iBndWr, &mb.jBndWr, &mb.sBndWr}, {&mb.iBndEr, &mb.jBndEr, &mb.sBndEr},
            {&mb.iBndSr, &mb.jBndSr, &mb.sBndSr}, {&mb.iBndNr, &mb.jBndNr, &mb.sBndNr},
            {&mb.iBndWp, &mb.jBndWp, &mb.sBndWp}, {&mb.iBndEp, &mb.jBndEp, &mb.sBndEp},
            {&mb.iBndSp, &mb.jBndSp, &mb.sBndSp}, {&mb.iBndNp, &mb.jBndNp, &mb.sBndNp}};
        cth_bc_list lists[12];
        for (int k = 0; k < 12; k++) {
            if (L[k][0]->size() != L[k][1]->size() || L[k][0]->size() != L[k][2]->size())
                throw std::runtime_error("solve_Microwave: a MicrowaveBC list has columns of different lengths");
            lists[k] = cth_bc_list{L[k][0]->data(), L[k][1]->data(), L[k][2]->data(), (int)L[k][0]->size()};
        }
        check_rc(cth_mw3_set_boundary(d_.m, lists, gc.j_flc_bl[0][0]), "cth_mw3_set_boundary");
        put_real(d_, "rhoe", gc.rhoe);
        put_real(d_, "nu_m1", gc.nu_m1);
        put_real(d_, "Bx", gc.Bx);
        put_real(d_, "Br", gc.Br);
        put_real(d_, "epsr", gc.epsr);
        put_real(d_, "Er", gr.Er);
        put_cplx(d_, 0, gx.E1x);   // the solve writes the unknowns; the ghosts stay the caller's
        put_cplx(d_, 1, gr.E1r);
        put_cplx(d_, 2, gc.E1p);
    }

    // solve of the assembled system, ghost pass, the field back to the caller
    void finish(GridCenter& gc, GridInterfaceX& gx, GridInterfaceR& gr, const cth_mw_params& prm) {
        using namespace cathode_b200;
        check_rc(cth_mw3_solve_dev(d_.m, maxITR, error_cnv, d_.plane(0), nullptr, &last_status), "cth_mw3_solve_dev");
        check_rc(cth_mw3_fill_ghosts(d_.m, d_.plane(0), cth_field(d_.fs, "epsr"), cth_field(d_.fs, "Er"), &prm,
                                     nullptr),
                 "cth_mw3_fill_ghosts");
        get_cplx(d_, 0, gx.E1x);
        get_cplx(d_, 1, gr.E1r);
        get_cplx(d_, 2, gc.E1p);
    }

    static cth_mw_params mw_params(const Params& pm) {
        return cth_mw_params{pm.dx, pm.dr, pm.rmin, pm.omegam, pm.J1r_exc, pm.r1, pm.r2, pm.masse};
    }

    // (re)build the device state when the grid or its blocks change
    void setup(const Params& pm, const GridCenter& gc, const GridInterfaceX& gx, const GridInterfaceR& gr) {
        using namespace cathode_b200;
        const int nb = pm.n_bl;
        std::vector<int> xi, xj, ri, rj, ci, cj;
        for (int b = 0; b < nb; b++) {
            for (int k = 0; k < 2; k++) {
                xi.push_back(gx.i_flx_bl[b][k]); xj.push_back(gx.j_flx_bl[b][k]);
                ri.push_back(gr.i_flr_bl[b][k]); rj.push_back(gr.j_flr_bl[b][k]);
                ci.push_back(gc.i_flc_bl[b][k]); cj.push_back(gc.j_flc_bl[b][k]);
            }
        }
        std::vector<int> key;
        for (auto* v : {&xi, &xj, &ri, &rj, &ci, &cj}) key.insert(key.end(), v->begin(), v->end());
        if (d_.m && d_.ni == pm.ni && d_.nj == pm.nj && d_.blocks == key && d_.device == device) return;
        d_.release();
        d_.ni = pm.ni;
        d_.nj = pm.nj;
        d_.device = device;
        d_.blocks = key;
        check_rc(cth_mw3_create_blocks(pm.ni, pm.nj, xi.data(), xj.data(), nb, ri.data(), rj.data(), nb, ci.data(),
                                       cj.data(), nb, device, &d_.m),
                 "cth_mw3_create_blocks");
        check_rc(cth_grid_create(pm.ni, pm.nj, ci.data(), cj.data(), nb, device, &d_.gc), "cth_grid_create");
        check_rc(cth_grid_create(pm.ni, pm.nj, xi.data(), xj.data(), nb, device, &d_.gx), "cth_grid_create");
        check_rc(cth_grid_create(pm.ni, pm.nj, ri.data(), rj.data(), nb, device, &d_.gr), "cth_grid_create");
        check_rc(cth_fields_create(d_.gc, &d_.fs), "cth_fields_create");
        d_.ld = cth_grid_ld(d_.gc);
        d_.cplane = (size_t)(pm.nj + 2) * d_.ld * 2 * sizeof(double);
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        check_cuda(cudaMalloc(&d_.cplx, 9 * d_.cplane), "cudaMalloc");
        check_cuda(cudaMemset(d_.cplx, 0, 9 * d_.cplane), "cudaMemset");
        check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        d_.stage.assign(d_.cplane / sizeof(double), 0.0);
        d_.flat.assign((size_t)(pm.ni + 2) * (pm.nj + 2), 0.0);
    }
};
