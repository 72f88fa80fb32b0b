/*
 * ref_driver.cpp — C entry points over the reference's own FluidModule and
 * InitialModule, compiled from the unmodified reference headers into
 * oracle/_ref/libref.so by oracle/Makefile (target _ref).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/ (and the checker legs of smoke() /
 * bench.py) load the library; it pins the CPU restatement (oracle/fluid.py)
 * and the device path to the reference's own arithmetic.
 *
 * What runs here is the reference's code: FluidModule::* of fluidModule.hpp
 * (check_CFL :57, solve_Uix_tmp :123, solve_Uir_tmp :601, solve_Uip_tmp :1054,
 * solve_rhoi_constTe :1405, correct_Ui_constTe :1763,
 * solve_phi_couple_wdTe_wSEE_PC :2080, solve_rhoe_wdTe_wSEE_PC :3082,
 * solve_Te_wdTe_wSEE_PC :4006, update_rhon :4963, update_rhom :5416,
 * update_transport_coef :5799) and InitialModule::makeBoundary
 * (initialModule.hpp:207-1058) on the reference's Params / GridCenter /
 * GridInterfaceX / GridInterfaceR / MicrowaveBC / SeeVec / BolsigVec types.
 * Only the linear solves differ: refshim/solverFuncs.hpp replaces HYPRE by
 * the exact solve that SMG converges to; built with -DREF_DROPIN against
 * refshim_dropin/solverFuncs.hpp, the solves are the product's GPU drop-in
 * (include/cathode_solver.hpp over libcathode_b200.so) instead.
 *
 * Written here (not the reference's): the name registries that copy planes,
 * parameters and tables in and out ([i][j] row-major, (ni+2) x (nj+2)), the
 * domain lines of InitialModule::iniParam (initialModule.hpp:59-87, restated
 * because iniParam also creates ./results), and the loop body of
 * src/main.cpp:172-251 without the microwave update (ref_call "step").
 */
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "fluidModule.hpp"
#include "initialModule.hpp"
#include "outputModule.hpp"
#ifdef REF_DROPIN
#include "cathode_emfield.hpp"   // the product's EmfieldModule drop-in (GPU)
#endif

#ifndef REF_DROPIN
extern "C" {
#include "oracle.h"
}
#endif

/* ---------------------------------------------------------------- shim state */
namespace refshim {
int& mode() { static int m = 0; return m; }
bool& capturing() { static bool c = false; return c; }
std::vector<System>& captured() { static std::vector<System> v; return v; }
int& calls() { static int c = 0; return c; }
int& failures() { static int f = 0; return f; }
}  // namespace refshim

using VV = std::vector<std::vector<double> >;
using VI = std::vector<std::vector<int> >;

namespace {

void flatten(const VV& a, std::vector<double>& out) {
    const size_t R = a.size(), C = R ? a[0].size() : 0;
    out.resize(R * C);
    for (size_t i = 0; i < R; ++i) std::memcpy(&out[i * C], a[i].data(), C * sizeof(double));
}

void blocks(const VI& i_bl, const VI& j_bl, int n_bl, std::vector<int>& ib, std::vector<int>& jb) {
    ib.resize(2 * n_bl);
    jb.resize(2 * n_bl);
    for (int b = 0; b < n_bl; ++b) {
        ib[2 * b] = i_bl[b][0]; ib[2 * b + 1] = i_bl[b][1];
        jb[2 * b] = j_bl[b][0]; jb[2 * b + 1] = j_bl[b][1];
    }
}

void record(const VV* planes[6], const std::vector<int>& ib, const std::vector<int>& jb, int n_bl) {
    if (!refshim::capturing()) return;
    refshim::System s;
    s.rows = (int)planes[0]->size();
    s.cols = s.rows ? (int)(*planes[0])[0].size() : 0;
    for (int k = 0; k < 6; ++k) flatten(*planes[k], s.a[k]);
    s.ib = ib; s.jb = jb; s.n_bl = n_bl;
    refshim::captured().push_back(std::move(s));
}

}  // namespace

#ifndef REF_DROPIN
void solver_SMG(VV aP, VV aE, VV aW, VV aN, VV aS, VV b, VI i_bl, VI j_bl, int n_bl, int maxITR,
                double error_cnv, int /*flag_msg*/, VV& solution) {
    refshim::calls()++;
    std::vector<int> ib, jb;
    blocks(i_bl, j_bl, n_bl, ib, jb);
    const VV* planes[6] = {&aP, &aE, &aW, &aN, &aS, &b};
    record(planes, ib, jb, n_bl);
    const int ni = (int)aP.size() - 2, nj = (int)aP[0].size() - 2;
    std::vector<double> f[6], x;
    for (int k = 0; k < 6; ++k) flatten(*planes[k], f[k]);
    flatten(solution, x);
    int rc;
    if (refshim::mode() == 1) {
        int it = 0;
        double rel = 0.0;
        rc = orc_smg_solve(ni, nj, ib.data(), jb.data(), n_bl, f[0].data(), f[1].data(), f[2].data(),
                           f[3].data(), f[4].data(), f[5].data(), maxITR, error_cnv, 1, 1, x.data(), &it, &rel);
        rc = rc < 0 ? rc : 0;
    } else {
        rc = orc_struct5_direct(ni, nj, ib.data(), jb.data(), n_bl, f[0].data(), f[1].data(), f[2].data(),
                                f[3].data(), f[4].data(), f[5].data(), x.data());
    }
    if (rc != 0) refshim::failures()++;
    /* block cells only, as the reference copies the HYPRE vector back (solverFuncs.hpp:143-152) */
    for (int bl = 0; bl < n_bl; ++bl)
        for (int i = ib[2 * bl]; i <= ib[2 * bl + 1]; ++i)
            for (int j = jb[2 * bl]; j <= jb[2 * bl + 1]; ++j) solution[i][j] = x[(size_t)i * (nj + 2) + j];
}

void solver_SOR(VV aP, VV aE, VV aW, VV aN, VV aS, VV b, VI i_bl, VI j_bl, int n_bl, double alpha_SOR,
                int maxITR, double error_cnv, int /*flag_msg*/, VV& solution) {
    refshim::calls()++;
    std::vector<int> ib, jb;
    blocks(i_bl, j_bl, n_bl, ib, jb);
    const VV* planes[6] = {&aP, &aE, &aW, &aN, &aS, &b};
    record(planes, ib, jb, n_bl);
    const int ni = (int)aP.size() - 2, nj = (int)aP[0].size() - 2;
    std::vector<double> f[6], x;
    for (int k = 0; k < 6; ++k) flatten(*planes[k], f[k]);
    flatten(solution, x);
    int n = 0;
    double err = 0.0;
    orc_sor_solve(ni, nj, ib.data(), jb.data(), n_bl, f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                  f[4].data(), f[5].data(), alpha_SOR, maxITR, error_cnv, x.data(), &n, &err);
    for (int i = 0; i < ni + 2; ++i)
        std::memcpy(solution[i].data(), &x[(size_t)i * (nj + 2)], (nj + 2) * sizeof(double));
}

#endif  // REF_DROPIN

/* ------------------------------------------------------------------ the case */
namespace {

struct RefCase {
    Params pm;
    GridCenter gc;
    GridInterfaceX gx;
    GridInterfaceR gr;
    MicrowaveBC mb;
    SeeVec se;
    BolsigVec bo;
    FluidModule flu;
    InitialModule ini;
    OutputModule out;
#ifdef REF_DROPIN
    EmfieldModule emf;
#endif
    bool quiet = true;
    RefCase(int ni, int nj) : gc(ni, nj), gx(ni, nj), gr(ni, nj) {
        pm.ni = ni;
        pm.nj = nj;
        /* keep the sweeps' periodic balance files (written when itime % ndiv_fout == 0) switched off */
        pm.itime = 1;
        pm.ndiv_fout = 1 << 30;
        pm.ntime = -1;
        pm.flag_chk = 0;
        pm.flag_gnuRes = 0;
    }
};

struct Quiet {
    std::streambuf* old = nullptr;
    std::ostringstream sink;
    explicit Quiet(bool on) { if (on) old = std::cout.rdbuf(sink.rdbuf()); }
    ~Quiet() { if (old) std::cout.rdbuf(old); }
};

VV* plane(RefCase& c, const char* n) {
#define GC(m) if (!std::strcmp(n, #m)) return &c.gc.m;
#define GX(m) if (!std::strcmp(n, #m)) return &c.gx.m;
#define GR(m) if (!std::strcmp(n, #m)) return &c.gr.m;
    GC(rhoe) GC(rhoe_old) GC(rhoi) GC(rhoi_old) GC(rhon) GC(rhon_old) GC(rhom) GC(rhom_old) GC(Uip) GC(Uip_old)
    GC(rhoeps) GC(rhoeps_old) GC(nu_m) GC(nu_m1) GC(nui_m) GC(nu_elas) GC(nu_super) GC(nu_ionz) GC(nu_ionzStep)
    GC(nu_exc) GC(nu_excReso) GC(nu_excMeta) GC(nu_excStep) GC(nu_ano) GC(nu_ano_IAT) GC(rate_ionize)
    GC(rate_eloss) GC(delossdeps) GC(mu_para) GC(mu_perp) GC(mu_min) GC(mu_xx) GC(mu_rr) GC(mu_xr) GC(mu_inv_xx)
    GC(mu_inv_rr) GC(mu_inv_xr) GC(Te) GC(Te_old) GC(phi) GC(phi_old) GC(Ap) GC(Bx) GC(Br) GC(epsr) GC(Mache)
    GC(Pabsp) GC(Pabs) GC(distECR)
    GX(rhoUex) GX(rhoUex_old) GX(rhoUix) GX(rhoUix_old) GX(rhoUnx) GX(rhoUnx_old) GX(rhoUmx) GX(rhoUmx_old)
    GX(nUex) GX(nUex_old) GX(Gx) GX(Gx_old) GX(rhoUex_wall) GX(rhoUix_wall) GX(rhoUnx_wall) GX(rhoUmx_wall)
    GX(nUex_wall) GX(Gx_wall) GX(Uix) GX(Uix_old) GX(Ex) GX(Pabsx) GX(scx) GX(scx_old)
    GR(rhoUer) GR(rhoUer_old) GR(rhoUir) GR(rhoUir_old) GR(rhoUnr) GR(rhoUnr_old) GR(rhoUmr) GR(rhoUmr_old)
    GR(nUer) GR(nUer_old) GR(Gr) GR(Gr_old) GR(rhoUer_wall) GR(rhoUir_wall) GR(rhoUnr_wall) GR(rhoUmr_wall)
    GR(nUer_wall) GR(Gr_wall) GR(Uir) GR(Uir_old) GR(Er) GR(Pabsr) GR(scr) GR(scr_old)
#undef GC
#undef GX
#undef GR
    return nullptr;
}

VI* iplane(RefCase& c, const char* n) {
#define M(s, m) if (!std::strcmp(n, #m)) return &c.s.m;
    M(gc, jdgBnd_Ep) M(gc, jdgBnd_flc) M(gc, i_flc_bl) M(gc, j_flc_bl)
    M(gx, jdgBnd_Ex) M(gx, jdgBnd_flx) M(gx, i_flx_bl) M(gx, j_flx_bl)
    M(gr, jdgBnd_Er) M(gr, jdgBnd_flr) M(gr, i_flr_bl) M(gr, j_flr_bl)
#undef M
    return nullptr;
}

double* dparam(Params& p, const char* n) {
#define D(m) if (!std::strcmp(n, #m)) return &p.m;
    D(xL) D(xR) D(rmin) D(rmax) D(width_neutIn) D(V_bias) D(Q_neutIn_mgs) D(fmw) D(Pmw) D(masse) D(massi) D(ri)
    D(Ti) D(Tn) D(DmN) D(epsr_diele) D(S11_mag) D(S11_arg_deg) D(S21_mag) D(S21_arg_deg) D(S12_mag)
    D(S12_arg_deg) D(S22_mag) D(S22_arg_deg) D(Z0) D(h0_stab) D(dh_stab) D(dl_cable) D(phase_pre_deg)
    D(coefIISEE_ts) D(coefMISEE_ts) D(Te_emitSEE_eV) D(ratioEngy_EISEE_rd) D(scale_inertia) D(alpha_Bohm)
    D(nu_eff) D(rhon_ini) D(rhoe_ini) D(Te_ini) D(J1r_exc) D(Te_rep_eV) D(error_cnv_SOR_Ui) D(error_cnv_SOR_rhoi)
    D(error_cnv_SOR_phi) D(error_cnv_HES_phi) D(error_cnv_SOR_rhoe) D(error_cnv_HES_rhoe) D(beta_rhoe)
    D(beta_rhoUe) D(error_cnv_SOR_rhoeps) D(error_cnv_HES_rhoeps) D(dt_ini) D(CFL) D(deltaECR) D(omegam) D(Lx)
    D(Lr) D(gtime) D(dx) D(dr) D(dt) D(I_Anode) D(Ii_Anode) D(Ie_Anode) D(I_Nozzle) D(Ii_Nozzle) D(Ie_Nozzle)
    D(error_rhoi) D(error_Uix) D(error_Uir) D(error_Uip) D(error_rhoe) D(error_rhoUex) D(error_rhoUer)
    D(error_rhoeps) D(error_Gx) D(error_Gr) D(error_phi) D(error_nUex) D(error_nUer) D(error_rhom) D(error_rhon)
    D(dTe) D(dEi) D(dTe_SEE) D(fn_In) D(x1) D(x2) D(x3) D(x4) D(x5) D(x6) D(r1) D(r2) D(r3) D(r4) D(r5) D(r6)
#undef D
    return nullptr;
}

int* iparam(Params& p, const char* n) {
#define I(m) if (!std::strcmp(n, #m)) return &p.m;
    I(ni) I(nj) I(flag_mwRef) I(flag_inertia) I(flag_Sagdeev) I(flag_Bohm) I(flag_PC) I(maxITR_SOR_Ui)
    I(flag_iter_Ui) I(maxITR_SOR_rhoi) I(flag_iter_rhoi) I(maxITR_SOR_phi) I(flag_iter_phi) I(maxITR_HES_phi)
    I(maxITR_SOR_rhoe) I(flag_iter_rhoe) I(maxITR_HES_rhoe) I(maxITR_SOR_rhoeps) I(flag_iter_rhoeps)
    I(maxITR_HES_rhoeps) I(flag_adp_dt) I(ntime) I(ndt_i) I(ndt_m) I(ndt_n) I(ndiv_MW) I(flag_error)
    I(flag_autoFinish) I(flag_chk) I(flag_gnuRes) I(ndiv_fout) I(flag_impTest) I(n_bl) I(itime) I(itime_PC_phi)
    I(itime_PC_rhoe) I(itime_PC_rhoeps) I(nOut) I(flag_restart)
#undef I
    return nullptr;
}

using VC = std::vector<std::vector<std::complex<double> > >;

VC* cplane(RefCase& c, const char* n) {
#define M(s, m) if (!std::strcmp(n, #m)) return &c.s.m;
    M(gx, E1x) M(gx, J1x) M(gx, J1x_exc) M(gr, E1r) M(gr, J1r) M(gr, J1r_exc) M(gc, E1p) M(gc, J1p) M(gc, J1p_exc)
#undef M
    return nullptr;
}

std::vector<double>* table(RefCase& c, const char* n) {
#define B(m) if (!std::strcmp(n, #m)) return &c.bo.m;
#define S(m) if (!std::strcmp(n, #m)) return &c.se.m;
    B(nu_elas_N) B(nu_super_N) B(nu_ionz_N) B(nu_ionzStep_N) B(nu_exc_N) B(nu_excReso_N) B(nu_excMeta_N)
    B(nu_excStep_N) B(rate_eloss_n_N) B(rate_eloss_m_N) B(nui_m_N)
    S(coefEISEE_eb_table) S(coefEISEE_rd_table) S(coefEISEE_ts_table)
#undef B
#undef S
    if (!std::strcmp(n, "x")) return &c.gc.x;
    if (!std::strcmp(n, "r")) return &c.gc.r;
    return nullptr;
}

std::vector<int>* mwlist(MicrowaveBC& m, const char* n) {
#define L(f) if (!std::strcmp(n, "i" #f)) return &m.i##f; if (!std::strcmp(n, "j" #f)) return &m.j##f; \
             if (!std::strcmp(n, "s" #f)) return &m.s##f;
    L(BndWx) L(BndEx) L(BndSx) L(BndNx) L(BndWr) L(BndEr) L(BndSr) L(BndNr) L(BndWp) L(BndEp) L(BndSp) L(BndNp)
#undef L
    return nullptr;
}

/* The loop body of src/main.cpp:172-251 (flag_PC == 1, flag_inertia == 0), without the microwave update. */
void step(RefCase& c) {
    Params& pm = c.pm;
    c.flu.check_CFL(pm, c.gc, c.gx, c.gr);
    pm.gtime = pm.gtime + pm.dt;
    pm.itime = pm.itime + 1;
    if (pm.itime % pm.ndt_i == 0) {
        c.flu.solve_Uix_tmp(pm, c.gc, c.gx, c.gr);
        c.flu.solve_Uir_tmp(pm, c.gc, c.gx, c.gr);
        c.flu.solve_Uip_tmp(pm, c.gc, c.gx, c.gr);
        c.flu.solve_rhoi_constTe(pm, c.gc, c.gx, c.gr);
        c.flu.correct_Ui_constTe(pm, c.gc, c.gx, c.gr);
    }
    if (pm.flag_PC == 1) {
        c.flu.solve_phi_couple_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
        if (pm.flag_inertia == 0) {
            c.flu.solve_rhoe_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
            c.flu.solve_Te_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
        }
    }
    if (pm.itime % pm.ndt_n == 0) c.flu.update_rhon(pm, c.gc, c.gx, c.gr);
    if (pm.itime % pm.ndt_m == 0) c.flu.update_rhom(pm, c.gc, c.gx, c.gr);
    c.flu.update_transport_coef(pm, c.gc, c.gx, c.gr, c.bo);
}

}  // namespace

extern "C" {

void* ref_create(int ni, int nj) {
    if (ni < 1 || nj < 1) return nullptr;
    return new RefCase(ni, nj);
}

void ref_destroy(void* h) { delete static_cast<RefCase*>(h); }

void ref_set_quiet(void* h, int on) { static_cast<RefCase*>(h)->quiet = on != 0; }

int ref_set_param(void* h, const char* name, double v) {
    Params& p = static_cast<RefCase*>(h)->pm;
    if (double* d = dparam(p, name)) { *d = v; return 0; }
    if (int* i = iparam(p, name)) { *i = (int)v; return 0; }
    return -1;
}

int ref_get_param(void* h, const char* name, double* v) {
    Params& p = static_cast<RefCase*>(h)->pm;
    if (double* d = dparam(p, name)) { *v = *d; return 0; }
    if (int* i = iparam(p, name)) { *v = *i; return 0; }
    return -1;
}

/* Copy a (ni+2) x (nj+2) plane in ([i][j] row-major). */
int ref_set_field(void* h, const char* name, const double* src) {
    RefCase& c = *static_cast<RefCase*>(h);
    VV* a = plane(c, name);
    if (!a) return -1;
    const int C = c.pm.nj + 2;
    for (int i = 0; i < c.pm.ni + 2; ++i) std::memcpy((*a)[i].data(), src + (size_t)i * C, C * sizeof(double));
    return 0;
}

int ref_get_field(void* h, const char* name, double* dst) {
    RefCase& c = *static_cast<RefCase*>(h);
    VV* a = plane(c, name);
    if (!a) return -1;
    const int C = c.pm.nj + 2;
    for (int i = 0; i < c.pm.ni + 2; ++i) std::memcpy(dst + (size_t)i * C, (*a)[i].data(), C * sizeof(double));
    return 0;
}

/* Integer planes (block flags jdgBnd_*, and the block tables *_bl, which the
 * reference stores as (ni+2) x (nj+2) int arrays of which rows 0..5 are used). */
int ref_get_int_field(void* h, const char* name, int* dst) {
    RefCase& c = *static_cast<RefCase*>(h);
    VI* a = iplane(c, name);
    if (!a) return -1;
    const int C = c.pm.nj + 2;
    for (int i = 0; i < c.pm.ni + 2; ++i)
        for (int j = 0; j < C; ++j) dst[(size_t)i * C + j] = (*a)[i][j];
    return 0;
}

int ref_set_table(void* h, const char* name, const double* v, int n) {
    std::vector<double>* t = table(*static_cast<RefCase*>(h), name);
    if (!t || n < 0) return -1;
    t->assign(v, v + n);
    return 0;
}

int ref_table_size(void* h, const char* name) {
    std::vector<double>* t = table(*static_cast<RefCase*>(h), name);
    return t ? (int)t->size() : -1;
}

int ref_get_table(void* h, const char* name, double* v) {
    std::vector<double>* t = table(*static_cast<RefCase*>(h), name);
    if (!t) return -1;
    std::copy(t->begin(), t->end(), v);
    return 0;
}

/* Domain set-up of InitialModule::iniParam (initialModule.hpp:59-87) followed
 * by the reference's own InitialModule::makeBoundary: blocks, flags, neutral
 * inlet flux and the 12 MicrowaveBC lists.  Params are taken as set. */
int ref_make_boundary(void* h) {
    RefCase& c = *static_cast<RefCase*>(h);
    Params& pm = c.pm;
    pm.Lx = pm.xR - pm.xL;
    pm.Lr = pm.rmax - pm.rmin;
    pm.dx = pm.Lx / double(pm.ni);
    pm.dr = pm.Lr / double(pm.nj);
    pm.dt = pm.dt_ini;
    pm.omegam = 2.0 * M_PI * pm.fmw;
    for (int i = 0; i < pm.ni + 2; i++) c.gc.x[i] = pm.xL + (i - 0.5) * pm.dx;
    for (int j = 0; j < pm.nj + 2; j++) c.gc.r[j] = pm.rmin + (j - 0.5) * pm.dr;
    Quiet q(c.quiet);
    c.ini.makeBoundary(pm, c.gc, c.gx, c.gr, c.mb);
    return 0;
}

/* Length of a MicrowaveBC list ("iBndWx", "sBndNp", ...) and its content. */
int ref_mw_list(void* h, const char* name, int* dst, int cap) {
    std::vector<int>* v = mwlist(static_cast<RefCase*>(h)->mb, name);
    if (!v) return -1;
    const int n = (int)v->size();
    if (dst) for (int k = 0; k < n && k < cap; ++k) dst[k] = (*v)[k];
    return n;
}

/* Complex planes (E1x, E1r, E1p and the currents), re / im interleaved, [i][j]. */
int ref_set_cfield(void* h, const char* name, const double* src) {
    RefCase& c = *static_cast<RefCase*>(h);
    VC* a = cplane(c, name);
    if (!a) return -1;
    const size_t C = c.pm.nj + 2;
    for (int i = 0; i < c.pm.ni + 2; ++i)
        for (size_t j = 0; j < C; ++j) (*a)[i][j] = std::complex<double>(src[2 * (i * C + j)], src[2 * (i * C + j) + 1]);
    return 0;
}

int ref_get_cfield(void* h, const char* name, double* dst) {
    RefCase& c = *static_cast<RefCase*>(h);
    VC* a = cplane(c, name);
    if (!a) return -1;
    const size_t C = c.pm.nj + 2;
    for (int i = 0; i < c.pm.ni + 2; ++i)
        for (size_t j = 0; j < C; ++j) {
            dst[2 * (i * C + j)] = (*a)[i][j].real();
            dst[2 * (i * C + j) + 1] = (*a)[i][j].imag();
        }
    return 0;
}

/* The complex members of Params: S11, S21, S12, S22 (k = 0..3). */
int ref_set_sparam(void* h, int k, double re, double im) {
    Params& p = static_cast<RefCase*>(h)->pm;
    std::complex<double>* s[4] = {&p.S11, &p.S21, &p.S12, &p.S22};
    if (k < 0 || k > 3) return -1;
    *s[k] = std::complex<double>(re, im);
    return 0;
}

/* The drop-in microwave update (REF_DROPIN builds): the product's EmfieldModule
 * solve_Microwave / update_energy_profile on this case.  out[0..2] = iterations,
 * relative residual and convergence of the solve. */
int ref_microwave(void* h, const char* which, double tol, int maxit, double* out) {
#ifdef REF_DROPIN
    RefCase& c = *static_cast<RefCase*>(h);
    try {
        c.emf.error_cnv = tol;
        c.emf.maxITR = maxit;
        if (!std::strcmp(which, "solve_Microwave")) c.emf.solve_Microwave(c.pm, c.gc, c.gx, c.gr, c.mb);
        else if (!std::strcmp(which, "solve_Microwave_explicit"))
            c.emf.solve_Microwave_explicit(c.pm, c.gc, c.gx, c.gr, c.mb);
        else if (!std::strcmp(which, "update_energy_profile")) c.emf.update_energy_profile(c.pm, c.gc, c.gx, c.gr);
        else return -1;
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        return -2;
    }
    if (out) {
        out[0] = c.emf.last_status.iterations;
        out[1] = c.emf.last_status.residual;
        out[2] = c.emf.last_status.converged;
    }
    return 0;
#else
    (void)h; (void)which; (void)tol; (void)maxit; (void)out;
    return -1;
#endif
}

/* Run one reference method by name, or "step" (the time-loop body). */
int ref_call(void* h, const char* m) {
    RefCase& c = *static_cast<RefCase*>(h);
    Params& pm = c.pm;
    Quiet q(c.quiet);
    const int f0 = refshim::failures();
    if (!std::strcmp(m, "check_CFL")) c.flu.check_CFL(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "solve_Uix_tmp")) c.flu.solve_Uix_tmp(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "solve_Uir_tmp")) c.flu.solve_Uir_tmp(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "solve_Uip_tmp")) c.flu.solve_Uip_tmp(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "solve_rhoi_constTe")) c.flu.solve_rhoi_constTe(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "correct_Ui_constTe")) c.flu.correct_Ui_constTe(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "solve_phi_couple_wdTe_wSEE_PC"))
        c.flu.solve_phi_couple_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
    else if (!std::strcmp(m, "solve_rhoe_wdTe_wSEE_PC")) c.flu.solve_rhoe_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
    else if (!std::strcmp(m, "solve_Te_wdTe_wSEE_PC")) c.flu.solve_Te_wdTe_wSEE_PC(pm, c.gc, c.gx, c.gr, c.se);
    else if (!std::strcmp(m, "update_rhon")) c.flu.update_rhon(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "update_rhom")) c.flu.update_rhom(pm, c.gc, c.gx, c.gr);
    else if (!std::strcmp(m, "update_transport_coef")) c.flu.update_transport_coef(pm, c.gc, c.gx, c.gr, c.bo);
    else if (!std::strcmp(m, "step")) step(c);
    else return -1;
    return refshim::failures() == f0 ? 0 : 1;
}

/* Precision of the drop-in's solver_SMG (CTH_PREC_MIXED 1 / CTH_PREC_FP64 0); -1 when
 * this build uses the exact solve instead. */
int ref_dropin_precision(int p) {
#ifdef REF_DROPIN
    cathode_b200::precision() = p;
    return 0;
#else
    (void)p;
    return -1;
#endif
}

/* The drop-in's solve counts since the last call (calls, not converged, worst final
 * residual of a non-converged call); -1 when this build uses the exact solve. */
int ref_dropin_stats(long* calls, long* not_converged, double* worst) {
#ifdef REF_DROPIN
    cathode_b200::SolveStats& s = cathode_b200::stats();
    *calls = s.calls;
    *not_converged = s.not_converged;
    *worst = s.worst_residual;
    s = cathode_b200::SolveStats();
    return 0;
#else
    *calls = *not_converged = 0;
    *worst = 0.0;
    return -1;
#endif
}

/* The reference's own writer: OutputModule::output (outputModule.hpp:185-1051) run
 * with `dir` as the working directory, so that its results/result<nOut>.csv,
 * results/restart<nOut>.csv and results/current_sum<nOut>.csv land in dir/results. */
int ref_output(void* h, const char* dir) {
    RefCase& c = *static_cast<RefCase*>(h);
    char old[4096];
    if (!getcwd(old, sizeof old)) return -1;
    if (chdir(dir) != 0) return -1;
    mkdir("results", 0777);
    {
        Quiet q(c.quiet);
        c.out.output(c.pm, c.gc, c.gx, c.gr, c.bo);
    }
    return chdir(old) == 0 ? 0 : -1;
}

/* Linear-solve hooks of the shim. */
void ref_solver_mode(int mode) { refshim::mode() = mode; }
int ref_solve_calls(void) { return refshim::calls(); }
void ref_capture(int on) {
    refshim::capturing() = on != 0;
    refshim::captured().clear();
}
int ref_captured_count(void) { return (int)refshim::captured().size(); }

/* Plane k of recorded system `s`: 0 aP, 1 aE, 2 aW, 3 aN, 4 aS, 5 b. */
int ref_captured_plane(int s, int k, double* dst, int n) {
    if (s < 0 || s >= (int)refshim::captured().size() || k < 0 || k > 5) return -1;
    const std::vector<double>& a = refshim::captured()[s].a[k];
    if ((int)a.size() != n) return -1;
    std::copy(a.begin(), a.end(), dst);
    return 0;
}

/* Block table of recorded system `s` (2 ints per block each); returns n_bl. */
int ref_captured_blocks(int s, int* ib, int* jb, int cap) {
    if (s < 0 || s >= (int)refshim::captured().size()) return -1;
    const refshim::System& y = refshim::captured()[s];
    for (int k = 0; k < 2 * y.n_bl && k < 2 * cap; ++k) { ib[k] = y.ib[k]; jb[k] = y.jb[k]; }
    return y.n_bl;
}

}  // extern "C"
