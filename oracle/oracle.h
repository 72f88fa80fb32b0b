/*
 * oracle.h — CPU restatement of the reference's implicit 5-point solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and the reference arm of bench.py) use it, and only as the
 * checker or as the timed CPU baseline.
 *
 * Array convention (identical to the reference): every field is a
 * (ni+2) x (nj+2) array indexed [i][j], i = axial (x/z) index, j = radial (r)
 * index, flattened row-major as a[i*(nj+2) + j] (the reference stores
 * vector<vector<double>> with the same [i][j] meaning).  Block tables are
 * flattened as i_bl[2*b+0..1], j_bl[2*b+0..1] (inclusive ranges), as in
 * solverFuncs.hpp:32-34 and :43-47.
 *
 * Stencil convention (solverFuncs.hpp:77-81): row P reads
 *     aP*x_P - aE*x_{i+1} - aW*x_{i-1} - aN*x_{j+1} - aS*x_{j-1} = b_P.
 */
#ifndef CATHODE_ORACLE_H
#define CATHODE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Cell (i,j) is a grid cell iff it lies in one of the n_bl boxes
 * (solverFuncs.hpp:43-47).  mask is (ni+2)*(nj+2) bytes, [i][j]. */
void orc_active_mask(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                     unsigned char* mask);

/* r = b - A x on grid cells, with couplings to non-grid cells dropped (the
 * semantics of a HYPRE StructMatrix over a box union).  Non-grid cells of r
 * are set to 0.  Returns sum(r^2) in *rr and sum(b^2) in *bb (grid cells). */
void orc_struct5_residual(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                          const double* aP, const double* aE, const double* aW,
                          const double* aN, const double* aS, const double* b,
                          const double* x, double* r, double* rr, double* bb);

/* Exact solve of the box-union system (banded Gaussian elimination over the
 * bounding box of the grid cells, non-grid cells as identity rows).  Writes
 * grid cells of solution only (solverFuncs.hpp:143-152).  Returns 0, or -1 on
 * a zero pivot / allocation failure. */
int orc_struct5_direct(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                       const double* aP, const double* aE, const double* aW,
                       const double* aN, const double* aS, const double* b,
                       double* solution);

/* Restatement of HYPRE Struct SMG as called by solver_SMG
 * (solverFuncs.hpp:26-163): semicoarsening multigrid (coarsening in j, exact
 * line relaxation along i, Galerkin coarse operators), zero initial guess,
 * stop when ||b-Ax||_2/||b||_2 < error_cnv or after maxITR cycles.  Writes
 * grid cells of solution only.  *iters / *relres report the cycle count and
 * the final relative residual.  Returns 0 converged, 1 not converged,
 * -1 error.  nu1/nu2: pre/post smoothing sweeps (each = both line colours). */
int orc_smg_solve(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                  const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b,
                  int maxITR, double error_cnv, int nu1, int nu2,
                  double* solution, int* iters, double* relres);

/* Faithful restatement of solver_SOR (solverFuncs.hpp:169-217): lexicographic
 * point SOR over blocks in order, i outer, j inner, neighbours read from the
 * in/out solution array (no coupling is dropped), divide by (aP+1e-100), stop
 * when the max relative update fabs((new-old)/(new+old+1e-6))*2 <= error_cnv
 * or after the sweep that takes the count past maxITR.  *ncount / *error
 * report the sweep count and the last max relative update. */
void orc_sor_solve(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                   const double* aP, const double* aE, const double* aW,
                   const double* aN, const double* aS, const double* b,
                   double alpha_SOR, int maxITR, double error_cnv,
                   double* solution, int* ncount, double* error);

/* calcRes (miniFuncs.hpp:292-376): block-restricted change norms between
 * val_new and val_old, flag_error 0..3.  Returns the error. */
double orc_calc_res(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl,
                    const double* val_new, const double* val_old, double EPS,
                    int flag_error);

#ifdef __cplusplus
}
#endif
#endif
