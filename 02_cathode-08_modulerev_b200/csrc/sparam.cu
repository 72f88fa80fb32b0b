// sparam.cu — two-port network helpers of the microwave feed (host code):
// CmpMat2 (include/cmpMat2.hpp:8-34), InitialModule::sParamToABCD /
// ABCDToSParam (include/initialModule.hpp:1689-1739) and the S-parameter
// set-up with the stub and cable corrections (include/initialModule.hpp:107-192).
// The conversions are the textbook two-port relations for a reference
// impedance Z0; where the reference throws, these return CTH_ERR_ARG.
#include <complex>
#include <cmath>

#include "grid.h"

namespace {

using cplx = std::complex<double>;

inline cplx c_in(const double v[2]) { return cplx(v[0], v[1]); }
inline void c_out(cplx z, double v[2]) { v[0] = z.real(); v[1] = z.imag(); }

struct M2 {
    cplx A, B, C, D;
};

inline M2 m_in(const cth_cmat2& T) { return {c_in(T.A), c_in(T.B), c_in(T.C), c_in(T.D)}; }
inline void m_out(const M2& m, cth_cmat2* T) {
    c_out(m.A, T->A); c_out(m.B, T->B); c_out(m.C, T->C); c_out(m.D, T->D);
}
inline M2 mul(const M2& X, const M2& Y) {
    return {X.A * Y.A + X.B * Y.C, X.A * Y.B + X.B * Y.D, X.C * Y.A + X.D * Y.C, X.C * Y.B + X.D * Y.D};
}
inline M2 inv(const M2& X) {
    const cplx d = X.A * X.D - X.B * X.C;
    return {X.D / d, -X.B / d, -X.C / d, X.A / d};
}

int s_to_abcd(cplx S11, cplx S21, cplx S12, cplx S22, double Z0, M2* T) {
    if (std::abs(S21) < 1.0e-14) {
        cth::set_error("sParamToABCD: S21 is too small");
        return CTH_ERR_ARG;
    }
    const cplx den = 2.0 * S21;
    T->A = ((1.0 + S11) * (1.0 - S22) + S12 * S21) / den;
    T->B = Z0 * ((1.0 + S11) * (1.0 + S22) - S12 * S21) / den;
    T->C = 1.0 / Z0 * ((1.0 - S11) * (1.0 - S22) - S12 * S21) / den;
    T->D = ((1.0 - S11) * (1.0 + S22) + S12 * S21) / den;
    return CTH_OK;
}

int abcd_to_s(const M2& T, double Z0, cplx* S11, cplx* S21, cplx* S12, cplx* S22) {
    const cplx den = T.A + T.B / Z0 + T.C * Z0 + T.D;
    if (std::abs(den) < 1.0e-14) {
        cth::set_error("ABCDToSParam: denominator is too small");
        return CTH_ERR_ARG;
    }
    *S11 = (T.A + T.B / Z0 - T.C * Z0 - T.D) / den;
    *S21 = 2.0 / den;
    *S12 = 2.0 * (T.A * T.D - T.B * T.C) / den;
    *S22 = (-T.A + T.B / Z0 - T.C * Z0 + T.D) / den;
    return CTH_OK;
}

}  // namespace

extern "C" {

int cth_cmat2_mul(const cth_cmat2* X, const cth_cmat2* Y, cth_cmat2* out) {
    if (!X || !Y || !out) { cth::set_error("cth_cmat2_mul: null argument"); return CTH_ERR_ARG; }
    m_out(mul(m_in(*X), m_in(*Y)), out);
    return CTH_OK;
}

int cth_cmat2_inv(const cth_cmat2* X, cth_cmat2* out) {
    if (!X || !out) { cth::set_error("cth_cmat2_inv: null argument"); return CTH_ERR_ARG; }
    m_out(inv(m_in(*X)), out);
    return CTH_OK;
}

int cth_sparam_to_abcd(const double S11[2], const double S21[2], const double S12[2], const double S22[2], double Z0,
                       cth_cmat2* T) {
    if (!S11 || !S21 || !S12 || !S22 || !T) { cth::set_error("cth_sparam_to_abcd: null argument"); return CTH_ERR_ARG; }
    M2 m;
    const int rc = s_to_abcd(c_in(S11), c_in(S21), c_in(S12), c_in(S22), Z0, &m);
    if (rc == CTH_OK) m_out(m, T);
    return rc;
}

int cth_abcd_to_sparam(const cth_cmat2* T, double Z0, double S11[2], double S21[2], double S12[2], double S22[2]) {
    if (!T || !S11 || !S21 || !S12 || !S22) { cth::set_error("cth_abcd_to_sparam: null argument"); return CTH_ERR_ARG; }
    cplx a, b, c, d;
    const int rc = abcd_to_s(m_in(*T), Z0, &a, &b, &c, &d);
    if (rc == CTH_OK) { c_out(a, S11); c_out(b, S21); c_out(c, S12); c_out(d, S22); }
    return rc;
}

// S-parameters of the feed at initialisation (initialModule.hpp:107-192):
// polar input, the stub-length change applied as a shunt admittance at the
// stub junction behind a pre-line of phase phase_pre_deg, then the cable
// length change as a phase factor.
int cth_sparam_setup(const cth_sparam_params* p, double S[4][2], double* cable_phase_deg) {
    if (!p || !S || !(p->Z0 > 0.0)) { cth::set_error("cth_sparam_setup: invalid arguments"); return CTH_ERR_ARG; }
    // polar values as mag * (cos, sin) of the angle in degrees
    cplx S11 = cplx(p->S11_mag * std::cos(p->S11_arg_deg / 180.0 * M_PI), p->S11_mag * std::sin(p->S11_arg_deg / 180.0 * M_PI));
    cplx S21 = cplx(p->S21_mag * std::cos(p->S21_arg_deg / 180.0 * M_PI), p->S21_mag * std::sin(p->S21_arg_deg / 180.0 * M_PI));
    cplx S12 = cplx(p->S12_mag * std::cos(p->S12_arg_deg / 180.0 * M_PI), p->S12_mag * std::sin(p->S12_arg_deg / 180.0 * M_PI));
    cplx S22 = cplx(p->S22_mag * std::cos(p->S22_arg_deg / 180.0 * M_PI), p->S22_mag * std::sin(p->S22_arg_deg / 180.0 * M_PI));
    const double ph = p->phase_pre_deg / 180.0 * M_PI;
    const cplx j(0.0, 1.0);
    const M2 Tpre{cplx(std::cos(ph), 0.0), j * p->Z0 * std::sin(ph), j * std::sin(ph) / p->Z0, cplx(std::cos(ph), 0.0)};
    M2 Tbase;
    int rc = s_to_abcd(S11, S21, S12, S22, p->Z0, &Tbase);
    if (rc != CTH_OK) return rc;
    const double eps0 = 8.8541878128e-12, mu0 = 1.2566370614e-6;  // constants.hpp:7-8
    const double c0 = std::sqrt(1.0 / (eps0 * p->epsr_diele * mu0));
    const double beta = p->omegam / c0;
    const double Y0 = 1.0 / p->Z0;
    const double tan0 = std::tan(beta * p->h0_stab);
    const double tanNew = std::tan(beta * (p->h0_stab + p->dh_stab));
    if (std::abs(tan0) < 1.0e-14 || std::abs(tanNew) < 1.0e-14) {
        cth::set_error("short-stub admittance: tan(beta*l) is too small");
        return CTH_ERR_ARG;
    }
    const cplx dYs = (-j * Y0 / tanNew) - (-j * Y0 / tan0);
    const M2 Tcorr{cplx(1.0, 0.0), cplx(0.0, 0.0), dYs, cplx(1.0, 0.0)};
    const M2 Tstub = mul(mul(mul(Tpre, Tcorr), inv(Tpre)), Tbase);
    rc = abcd_to_s(Tstub, p->Z0, &S11, &S21, &S12, &S22);
    if (rc != CTH_OK) return rc;
    const cplx ph_c = std::exp(cplx(0.0, -beta) * p->dl_cable);
    S21 *= ph_c;
    S12 *= ph_c;
    S22 *= ph_c * ph_c;
    c_out(S11, S[0]); c_out(S21, S[1]); c_out(S12, S[2]); c_out(S22, S[3]);
    if (cable_phase_deg) *cable_phase_deg = beta * p->dl_cable / M_PI * 180.0;
    return CTH_OK;
}

}  // extern "C"
