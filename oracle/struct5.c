/*
 * struct5.c — CPU restatement of the reference's 5-point solve boundary.
 *
 * TEST INFRASTRUCTURE ONLY: the product never links this file.  It is the
 * checker for the CUDA path and the timed CPU baseline in bench.py.
 *
 * Reference functions restated here:
 *   solver_SMG   include/solverFuncs.hpp:26-163  (HYPRE 2.31.0 Struct SMG,
 *                not vendored in the reference; restated from the published
 *                semicoarsening-multigrid algorithm: coarsen in one direction,
 *                exact line relaxation in the other, Galerkin coarse grids)
 *   solver_SOR   include/solverFuncs.hpp:169-217
 *   calcRes      include/miniFuncs.hpp:292-376
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j) ((size_t)(i) * (size_t)(nj + 2) + (size_t)(j))

void orc_active_mask(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                     unsigned char* mask) {
    memset(mask, 0, (size_t)(ni + 2) * (size_t)(nj + 2));
    for (int b = 0; b < n_bl; b++)
        for (int i = i_bl[2 * b]; i <= i_bl[2 * b + 1]; i++)
            for (int j = j_bl[2 * b]; j <= j_bl[2 * b + 1]; j++)
                if (i >= 0 && i <= ni + 1 && j >= 0 && j <= nj + 1) mask[IDX(i, j)] = 1;
}

static int bounding_box(int ni, int nj, const unsigned char* mask, int* i0, int* i1, int* j0,
                        int* j1) {
    *i0 = ni + 2; *i1 = -1; *j0 = nj + 2; *j1 = -1;
    for (int i = 0; i <= ni + 1; i++)
        for (int j = 0; j <= nj + 1; j++)
            if (mask[IDX(i, j)]) {
                if (i < *i0) *i0 = i;
                if (i > *i1) *i1 = i;
                if (j < *j0) *j0 = j;
                if (j > *j1) *j1 = j;
            }
    return *i1 >= 0;
}

void orc_struct5_residual(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                          const double* aP, const double* aE, const double* aW,
                          const double* aN, const double* aS, const double* b,
                          const double* x, double* r, double* rr, double* bb) {
    size_t n = (size_t)(ni + 2) * (size_t)(nj + 2);
    unsigned char* m = (unsigned char*)malloc(n);
    orc_active_mask(ni, nj, i_bl, j_bl, n_bl, m);
    double s_rr = 0.0, s_bb = 0.0;
    for (int i = 0; i <= ni + 1; i++)
        for (int j = 0; j <= nj + 1; j++) {
            size_t p = IDX(i, j);
            if (!m[p]) { r[p] = 0.0; continue; }
            double ax = aP[p] * x[p];
            if (i + 1 <= ni + 1 && m[IDX(i + 1, j)]) ax -= aE[p] * x[IDX(i + 1, j)];
            if (i - 1 >= 0 && m[IDX(i - 1, j)]) ax -= aW[p] * x[IDX(i - 1, j)];
            if (j + 1 <= nj + 1 && m[IDX(i, j + 1)]) ax -= aN[p] * x[IDX(i, j + 1)];
            if (j - 1 >= 0 && m[IDX(i, j - 1)]) ax -= aS[p] * x[IDX(i, j - 1)];
            r[p] = b[p] - ax;
            s_rr += r[p] * r[p];
            s_bb += b[p] * b[p];
        }
    *rr = s_rr;
    *bb = s_bb;
    free(m);
}

/* ------------------------------------------------------------------------ */
/* exact banded solve                                                        */
/* ------------------------------------------------------------------------ */
int orc_struct5_direct(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                       const double* aP, const double* aE, const double* aW,
                       const double* aN, const double* aS, const double* b,
                       double* solution) {
    size_t n = (size_t)(ni + 2) * (size_t)(nj + 2);
    unsigned char* m = (unsigned char*)malloc(n);
    orc_active_mask(ni, nj, i_bl, j_bl, n_bl, m);
    int i0, i1, j0, j1;
    if (!bounding_box(ni, nj, m, &i0, &i1, &j0, &j1)) { free(m); return 0; }
    int nI = i1 - i0 + 1, nJ = j1 - j0 + 1;
    /* order unknowns so that the band is the smaller extent */
    int j_fast = (nJ <= nI);
    int bw = j_fast ? nJ : nI;
    long N = (long)nI * nJ;
    int W = 2 * bw + 1;
    double* A = (double*)calloc((size_t)N * W, sizeof(double));
    double* rhs = (double*)malloc(sizeof(double) * N);
    if (!A || !rhs) { free(A); free(rhs); free(m); return -1; }
#define UNK(ii, jj) (j_fast ? (long)(ii) * nJ + (jj) : (long)(jj) * nI + (ii))
#define BAND(r, c) A[(size_t)(r) * W + ((c) - (r) + bw)]
    for (int ii = 0; ii < nI; ii++)
        for (int jj = 0; jj < nJ; jj++) {
            int i = ii + i0, j = jj + j0;
            size_t p = IDX(i, j);
            long row = UNK(ii, jj);
            if (!m[p]) { BAND(row, row) = 1.0; rhs[row] = 0.0; continue; }
            BAND(row, row) = aP[p];
            rhs[row] = b[p];
            if (ii + 1 < nI && m[IDX(i + 1, j)]) BAND(row, UNK(ii + 1, jj)) = -aE[p];
            if (ii - 1 >= 0 && m[IDX(i - 1, j)]) BAND(row, UNK(ii - 1, jj)) = -aW[p];
            if (jj + 1 < nJ && m[IDX(i, j + 1)]) BAND(row, UNK(ii, jj + 1)) = -aN[p];
            if (jj - 1 >= 0 && m[IDX(i, j - 1)]) BAND(row, UNK(ii, jj - 1)) = -aS[p];
        }
    int rc = 0;
    for (long k = 0; k < N && rc == 0; k++) {
        double piv = BAND(k, k);
        if (piv == 0.0) { rc = -1; break; }
        long rmax = k + bw < N - 1 ? k + bw : N - 1;
        for (long r = k + 1; r <= rmax; r++) {
            double l = BAND(r, k);
            if (l == 0.0) continue;
            l /= piv;
            BAND(r, k) = 0.0;
            for (long c = k + 1; c <= rmax; c++) BAND(r, c) -= l * BAND(k, c);
            rhs[r] -= l * rhs[k];
        }
    }
    if (rc == 0) {
        for (long k = N - 1; k >= 0; k--) {
            double s = rhs[k];
            long cmax = k + bw < N - 1 ? k + bw : N - 1;
            for (long c = k + 1; c <= cmax; c++) s -= BAND(k, c) * rhs[c];
            rhs[k] = s / BAND(k, k);
        }
        for (int ii = 0; ii < nI; ii++)
            for (int jj = 0; jj < nJ; jj++) {
                size_t p = IDX(ii + i0, jj + j0);
                if (m[p]) solution[p] = rhs[UNK(ii, jj)];
            }
    }
#undef UNK
#undef BAND
    free(A); free(rhs); free(m);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* semicoarsening multigrid (restatement of SMG as used by solver_SMG)       */
/* ------------------------------------------------------------------------ */
/* Stencil slots, "positive neighbour" convention as in the reference:
 * (A x)_P = a[P] x_P - sum_k a[k] x_k.  Offsets are (di, dj). */
enum { SP = 0, SW_ = 1, SE_ = 2, SS = 3, SN = 4, SSW = 5, SSE = 6, SNW = 7, SNE = 8, NSLOT = 9 };
static const int OFF_I[NSLOT] = {0, -1, 1, 0, 0, -1, 1, -1, 1};
static const int OFF_J[NSLOT] = {0, 0, 0, -1, 1, -1, -1, 1, 1};

typedef struct {
    int nrow, ncol;
    double* a[NSLOT];
    unsigned char* mask;
    double *wS, *wN; /* interpolation weights of F rows toward the C rows below / above */
    double *x, *b, *r;
} mg_level;

#define LC(L, i, j) ((size_t)(j) * (size_t)(L)->ncol + (size_t)(i))

static void level_alloc(mg_level* L, int nrow, int ncol) {
    size_t n = (size_t)nrow * ncol;
    L->nrow = nrow; L->ncol = ncol;
    for (int k = 0; k < NSLOT; k++) L->a[k] = (double*)calloc(n, sizeof(double));
    L->mask = (unsigned char*)calloc(n, 1);
    L->wS = (double*)calloc(n, sizeof(double));
    L->wN = (double*)calloc(n, sizeof(double));
    L->x = (double*)calloc(n, sizeof(double));
    L->b = (double*)calloc(n, sizeof(double));
    L->r = (double*)calloc(n, sizeof(double));
}

static void level_free(mg_level* L) {
    for (int k = 0; k < NSLOT; k++) free(L->a[k]);
    free(L->mask); free(L->wS); free(L->wN); free(L->x); free(L->b); free(L->r);
}

/* interpolation weights for F rows (odd rows): the F line's own tridiagonal
 * operator (diagonal plus in-line couplings) applied inversely to the lumped
 * coupling toward the C row below / above, i.e. the F line is solved exactly
 * for a C-row value that is constant along the line. */
static void line_weights(mg_level* L, int j, int dir, double* out, double* cp, double* dp) {
    int nrow = L->nrow, ncol = L->ncol;
    for (int i = 0; i < ncol; i++) {
        size_t p = LC(L, i, j);
        double s = 0.0;
        int jc = j + dir;
        if (L->mask[p] && jc >= 0 && jc < nrow && L->mask[LC(L, i, jc)]) {
            s = dir < 0 ? L->a[SS][p] + L->a[SSW][p] + L->a[SSE][p]
                        : L->a[SN][p] + L->a[SNW][p] + L->a[SNE][p];
        }
        double lo = (i > 0) ? -L->a[SW_][p] : 0.0;
        double up = (i + 1 < ncol) ? -L->a[SE_][p] : 0.0;
        double diag = L->a[SP][p];
        if (i == 0) { cp[i] = up / diag; dp[i] = s / diag; }
        else {
            double den = diag - lo * cp[i - 1];
            cp[i] = up / den;
            dp[i] = (s - lo * dp[i - 1]) / den;
        }
    }
    for (int i = ncol - 1; i >= 0; i--) {
        double v = dp[i] - ((i + 1 < ncol) ? cp[i] * out[LC(L, i + 1, j)] : 0.0);
        out[LC(L, i, j)] = v;
    }
}

static void build_weights(mg_level* L, double* cp_unused, double* dp_unused) {
    (void)cp_unused; (void)dp_unused;
    int ncol = L->ncol;
#pragma omp parallel
    {
        double* cp = (double*)malloc(sizeof(double) * (size_t)ncol);
        double* dp = (double*)malloc(sizeof(double) * (size_t)ncol);
#pragma omp for schedule(static)
        for (int j = 1; j < L->nrow; j += 2) {
            line_weights(L, j, -1, L->wS, cp, dp);
            line_weights(L, j, +1, L->wN, cp, dp);
        }
        free(cp);
        free(dp);
    }
}

/* P(g, i -> J) for fine row g, column i */
static inline double pw(const mg_level* F, int g, int i, int J) {
    if ((g & 1) == 0) return (g / 2 == J && F->mask[LC(F, i, g)]) ? 1.0 : 0.0;
    if ((g - 1) / 2 == J) return F->wS[LC(F, i, g)];
    if ((g + 1) / 2 == J) return F->wN[LC(F, i, g)];
    return 0.0;
}

static void galerkin(const mg_level* F, mg_level* C) {
    int nrowc = C->nrow, ncol = C->ncol;
#pragma omp parallel for schedule(static)
    for (int J = 0; J < nrowc; J++)
        for (int i = 0; i < ncol; i++) {
            size_t q = LC(C, i, J);
            C->mask[q] = F->mask[LC(F, i, 2 * J)];
            double acc[3][3] = {{0}}; /* [dJ+1][di+1], matrix-sign entries */
            int c = 2 * J;
            for (int f = c - 1; f <= c + 1; f++) {
                if (f < 0 || f >= F->nrow) continue;
                double rw = pw(F, f, i, J);
                if (rw == 0.0) continue;
                for (int k = 0; k < NSLOT; k++) {
                    int ii = i + OFF_I[k], g = f + OFF_J[k];
                    if (ii < 0 || ii >= ncol || g < 0 || g >= F->nrow) continue;
                    double a = F->a[k][LC(F, i, f)];
                    if (a == 0.0) continue;
                    double mval = (k == SP) ? a : -a;
                    for (int dJ = -1; dJ <= 1; dJ++) {
                        int Jp = J + dJ;
                        if (Jp < 0 || Jp >= nrowc) continue;
                        double p = pw(F, g, ii, Jp);
                        if (p != 0.0) acc[dJ + 1][OFF_I[k] + 1] += rw * mval * p;
                    }
                }
            }
            if (!C->mask[q] || acc[1][1] == 0.0) {
                for (int k = 0; k < NSLOT; k++) C->a[k][q] = 0.0;
                C->a[SP][q] = 1.0;
                C->mask[q] = 0;
                continue;
            }
            for (int k = 0; k < NSLOT; k++) {
                double v = acc[OFF_J[k] + 1][OFF_I[k] + 1];
                C->a[k][q] = (k == SP) ? v : -v;
            }
        }
}

/* exact line solve (Thomas) of one row j, neighbours in the rows j-1 / j+1
 * taken from the current x */
static void relax_row(mg_level* L, int j, double* cp, double* dp) {
    int nrow = L->nrow, ncol = L->ncol;
    for (int i = 0; i < ncol; i++) {
        size_t p = LC(L, i, j);
        double d = L->b[p];
        for (int k = SS; k < NSLOT; k++) {
            int ii = i + OFF_I[k], jj = j + OFF_J[k];
            if (ii < 0 || ii >= ncol || jj < 0 || jj >= nrow) continue;
            d += L->a[k][p] * L->x[LC(L, ii, jj)];
        }
        double lo = (i > 0) ? -L->a[SW_][p] : 0.0;
        double up = (i + 1 < ncol) ? -L->a[SE_][p] : 0.0;
        double diag = L->a[SP][p];
        if (i == 0) {
            cp[i] = up / diag;
            dp[i] = d / diag;
        } else {
            double den = diag - lo * cp[i - 1];
            cp[i] = up / den;
            dp[i] = (d - lo * dp[i - 1]) / den;
        }
    }
    for (int i = ncol - 1; i >= 0; i--) {
        double v = dp[i] - ((i + 1 < ncol) ? cp[i] * L->x[LC(L, i + 1, j)] : 0.0);
        L->x[LC(L, i, j)] = v;
    }
}

/* zebra colour: every row of one parity (rows of a colour are independent) */
static void relax_rows(mg_level* L, int parity, double* cp_unused, double* dp_unused) {
    (void)cp_unused; (void)dp_unused;
    int nrow = L->nrow, ncol = L->ncol;
#pragma omp parallel
    {
        double* cp = (double*)malloc(sizeof(double) * (size_t)ncol);
        double* dp = (double*)malloc(sizeof(double) * (size_t)ncol);
#pragma omp for schedule(static)
        for (int j = parity; j < nrow; j += 2) relax_row(L, j, cp, dp);
        free(cp);
        free(dp);
    }
}

static void residual(mg_level* L) {
    int nrow = L->nrow, ncol = L->ncol;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nrow; j++)
        for (int i = 0; i < ncol; i++) {
            size_t p = LC(L, i, j);
            double s = L->b[p] - L->a[SP][p] * L->x[p];
            for (int k = 1; k < NSLOT; k++) {
                int ii = i + OFF_I[k], jj = j + OFF_J[k];
                if (ii < 0 || ii >= ncol || jj < 0 || jj >= nrow) continue;
                s += L->a[k][p] * L->x[LC(L, ii, jj)];
            }
            L->r[p] = L->mask[p] ? s : 0.0;
        }
}

static void vcycle(mg_level* Ls, int nlev, int l, int nu1, int nu2, double* cp, double* dp) {
    mg_level* L = &Ls[l];
    if (l == nlev - 1) {
        relax_rows(L, 0, cp, dp);
        if (L->nrow > 1) {
            for (int s = 0; s < 4; s++) { relax_rows(L, 1, cp, dp); relax_rows(L, 0, cp, dp); }
        }
        return;
    }
    for (int s = 0; s < nu1; s++) { relax_rows(L, 0, cp, dp); relax_rows(L, 1, cp, dp); }
    residual(L);
    mg_level* C = &Ls[l + 1];
#pragma omp parallel for schedule(static)
    for (int J = 0; J < C->nrow; J++)
        for (int i = 0; i < C->ncol; i++) {
            size_t q = LC(C, i, J);
            double s = 0.0;
            for (int f = 2 * J - 1; f <= 2 * J + 1; f++)
                if (f >= 0 && f < L->nrow) s += pw(L, f, i, J) * L->r[LC(L, i, f)];
            C->b[q] = C->mask[q] ? s : 0.0;
            C->x[q] = 0.0;
        }
    vcycle(Ls, nlev, l + 1, nu1, nu2, cp, dp);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < L->nrow; j++)
        for (int i = 0; i < L->ncol; i++) {
            size_t p = LC(L, i, j);
            double e;
            if ((j & 1) == 0) e = pw(L, j, i, j / 2) * C->x[LC(C, i, j / 2)];
            else {
                e = L->wS[p] * C->x[LC(C, i, (j - 1) / 2)];
                if ((j + 1) / 2 < C->nrow) e += L->wN[p] * C->x[LC(C, i, (j + 1) / 2)];
            }
            L->x[p] += e;
        }
    for (int s = 0; s < nu2; s++) { relax_rows(L, 0, cp, dp); relax_rows(L, 1, cp, dp); }
}

int orc_smg_solve(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                  const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b,
                  int maxITR, double error_cnv, int nu1, int nu2,
                  double* solution, int* iters, double* relres) {
    size_t n = (size_t)(ni + 2) * (size_t)(nj + 2);
    unsigned char* m = (unsigned char*)malloc(n);
    orc_active_mask(ni, nj, i_bl, j_bl, n_bl, m);
    int i0, i1, j0, j1;
    *iters = 0; *relres = 0.0;
    if (!bounding_box(ni, nj, m, &i0, &i1, &j0, &j1)) { free(m); return 0; }
    int ncol = i1 - i0 + 1, nrow = j1 - j0 + 1;
    int nlev = 1;
    for (int r = nrow; r > 1; r = (r + 1) / 2) nlev++;
    mg_level* Ls = (mg_level*)calloc((size_t)nlev, sizeof(mg_level));
    int r = nrow;
    for (int l = 0; l < nlev; l++) { level_alloc(&Ls[l], r, ncol); r = (r + 1) / 2; }
    mg_level* L0 = &Ls[0];
    /* level 0: masked copy, couplings to non-grid cells dropped */
    double bb = 0.0;
    for (int jj = 0; jj < nrow; jj++)
        for (int ii = 0; ii < ncol; ii++) {
            int i = ii + i0, j = jj + j0;
            size_t p = IDX(i, j), q = LC(L0, ii, jj);
            L0->mask[q] = m[p];
            if (!m[p]) { L0->a[SP][q] = 1.0; continue; }
            L0->a[SP][q] = aP[p];
            if (ii + 1 < ncol && m[IDX(i + 1, j)]) L0->a[SE_][q] = aE[p];
            if (ii - 1 >= 0 && m[IDX(i - 1, j)]) L0->a[SW_][q] = aW[p];
            if (jj + 1 < nrow && m[IDX(i, j + 1)]) L0->a[SN][q] = aN[p];
            if (jj - 1 >= 0 && m[IDX(i, j - 1)]) L0->a[SS][q] = aS[p];
            bb += b[p] * b[p];
        }
    double* cp = (double*)malloc(sizeof(double) * ncol);
    double* dp = (double*)malloc(sizeof(double) * ncol);
    for (int l = 0; l + 1 < nlev; l++) { build_weights(&Ls[l], cp, dp); galerkin(&Ls[l], &Ls[l + 1]); }

    double* xs = (double*)calloc((size_t)nrow * ncol, sizeof(double));
    double* rs = (double*)malloc(sizeof(double) * (size_t)nrow * ncol);
    int rc = 1;
    if (bb == 0.0) {
        rc = 0;
    } else {
        double nb = sqrt(bb);
        for (int jj = 0; jj < nrow; jj++)
            for (int ii = 0; ii < ncol; ii++) {
                size_t q = LC(L0, ii, jj);
                rs[q] = L0->mask[q] ? b[IDX(ii + i0, jj + j0)] : 0.0;
            }
        for (int it = 1; it <= maxITR; it++) {
            memcpy(L0->b, rs, sizeof(double) * (size_t)nrow * ncol);
            memset(L0->x, 0, sizeof(double) * (size_t)nrow * ncol);
            vcycle(Ls, nlev, 0, nu1, nu2, cp, dp);
            for (size_t q = 0; q < (size_t)nrow * ncol; q++) xs[q] += L0->x[q];
            /* fp64 residual of the accumulated solution */
            double rr = 0.0;
            memcpy(L0->x, xs, sizeof(double) * (size_t)nrow * ncol);
            memcpy(L0->b, rs, sizeof(double) * (size_t)nrow * ncol);
            for (int jj = 0; jj < nrow; jj++)
                for (int ii = 0; ii < ncol; ii++) {
                    size_t q = LC(L0, ii, jj);
                    L0->b[q] = L0->mask[q] ? b[IDX(ii + i0, jj + j0)] : 0.0;
                }
            residual(L0);
            for (size_t q = 0; q < (size_t)nrow * ncol; q++) { rs[q] = L0->r[q]; rr += rs[q] * rs[q]; }
            *iters = it;
            *relres = sqrt(rr) / nb;
            if (*relres < error_cnv) { rc = 0; break; }
        }
    }
    for (int jj = 0; jj < nrow; jj++)
        for (int ii = 0; ii < ncol; ii++) {
            size_t p = IDX(ii + i0, jj + j0);
            if (m[p]) solution[p] = xs[LC(L0, ii, jj)];
        }
    for (int l = 0; l < nlev; l++) level_free(&Ls[l]);
    free(Ls); free(xs); free(rs); free(cp); free(dp); free(m);
    return rc;
}

/* ------------------------------------------------------------------------ */
void orc_sor_solve(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                   const double* aP, const double* aE, const double* aW,
                   const double* aN, const double* aS, const double* b,
                   double alpha_SOR, int maxITR, double error_cnv,
                   double* solution, int* ncount_out, double* error_out) {
    int ncount = 0;
    double error = 0.0;
    do {
        ncount = ncount + 1;
        error = 0.0;
        for (int blk = 0; blk < n_bl; blk++)
            for (int i = i_bl[2 * blk]; i <= i_bl[2 * blk + 1]; i++)
                for (int j = j_bl[2 * blk]; j <= j_bl[2 * blk + 1]; j++) {
                    size_t p = IDX(i, j);
                    double tmp = (aE[p] * solution[IDX(i + 1, j)] + aW[p] * solution[IDX(i - 1, j)] +
                                  aN[p] * solution[IDX(i, j + 1)] + aS[p] * solution[IDX(i, j - 1)] +
                                  b[p]) / (aP[p] + 1e-100);
                    double nw = (1.0 - alpha_SOR) * solution[p] + alpha_SOR * tmp;
                    double e = fabs((nw - solution[p]) / (nw + solution[p] + 1e-6)) * 2.0;
                    if (e > error) error = e;
                    solution[p] = nw;
                }
        if (ncount > maxITR) break;
    } while (error > error_cnv);
    *ncount_out = ncount;
    *error_out = error;
}

/* ------------------------------------------------------------------------ */
double orc_calc_res(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                    const double* vn, const double* vo, double EPS, int flag_error) {
    (void)ni;
    double error = 0.0;
    if (flag_error == 0) {
        for (int blk = 0; blk < n_bl; blk++)
            for (int i = i_bl[2 * blk]; i <= i_bl[2 * blk + 1]; i++)
                for (int j = j_bl[2 * blk]; j <= j_bl[2 * blk + 1]; j++) {
                    double e = fabs(vn[IDX(i, j)] - vo[IDX(i, j)]);
                    if (e > error) error = e;
                }
    } else if (flag_error == 1) {
        long cnt = 0;
        for (int blk = 0; blk < n_bl; blk++)
            for (int i = i_bl[2 * blk]; i <= i_bl[2 * blk + 1]; i++)
                for (int j = j_bl[2 * blk]; j <= j_bl[2 * blk + 1]; j++) {
                    double d = vn[IDX(i, j)] - vo[IDX(i, j)];
                    error += d * d / (vo[IDX(i, j)] * vo[IDX(i, j)] + EPS);
                    cnt++;
                }
        error = sqrt(error / (double)cnt);
    } else if (flag_error == 2) {
        double norm = 0.0;
        for (int blk = 0; blk < n_bl; blk++)
            for (int i = i_bl[2 * blk]; i <= i_bl[2 * blk + 1]; i++)
                for (int j = j_bl[2 * blk]; j <= j_bl[2 * blk + 1]; j++) {
                    double e = fabs(vn[IDX(i, j)] - vo[IDX(i, j)]);
                    if (e > error) error = e;
                    double nm = fabs(vo[IDX(i, j)]);
                    if (nm > norm) norm = nm;
                }
        error = error / norm;
    } else if (flag_error == 3) {
        double norm = 0.0;
        for (int blk = 0; blk < n_bl; blk++)
            for (int i = i_bl[2 * blk]; i <= i_bl[2 * blk + 1]; i++)
                for (int j = j_bl[2 * blk]; j <= j_bl[2 * blk + 1]; j++) {
                    double d = vn[IDX(i, j)] - vo[IDX(i, j)];
                    error += d * d;
                    norm += vo[IDX(i, j)] * vo[IDX(i, j)];
                }
        error = sqrt(error / norm);
    }
    return error;
}
