/*
 * mathfn.c — element-wise exp and erf of the C library for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference evaluates exp() and erf() through
 * the C library (fluidModule.hpp: the Scharfetter-Gummel weights at :3240-3241,
 * the wall fluxes, the kinetic ion wall flux at :1498-1526); numpy's own
 * vectorised exp differs from it by one ulp on a few per cent of arguments, and
 * the Scharfetter-Gummel weights amplify such differences where the Peclet
 * number is small.  The oracle therefore takes both functions from here.
 */
#include <math.h>
#include <stddef.h>

void orc_exp(size_t n, const double* x, double* y) {
    for (size_t i = 0; i < n; i++) y[i] = exp(x[i]);
}

void orc_erf(size_t n, const double* x, double* y) {
    for (size_t i = 0; i < n; i++) y[i] = erf(x[i]);
}
