/*
 * cathode_b200.h — C ABI of the B200 implicit-solve library (libcathode_b200.so).
 *
 * Plain C types only: pointers, sizes, doubles.  Every entry point returns an
 * int status (CTH_OK = 0; > 0 = the solve ran but did not meet its stopping
 * rule or produced a non-finite residual; < 0 = argument / CUDA / allocation
 * error, nothing was written).  A human-readable message for the last error
 * on the calling thread is returned by cth_last_error().
 *
 * Array conventions
 * -----------------
 * Host arrays use the reference's convention: a field of the (ni+2) x (nj+2)
 * ghost-padded grid, indexed [i][j] (i = axial z index, j = radial r index),
 * flattened row-major: a[i*(nj+2) + j].  This is exactly the data of the
 * reference's vector<vector<double>> arguments (include/solverFuncs.hpp:26-37).
 *
 * Device arrays ("_dev" entry points) use the library's HBM layout: r-major
 * planes, element (i,j) at a[j*ld + i] with ld = cth_grid_ld(g) >= ni+2, so
 * that z-lines (fixed j) are contiguous.  ld is a multiple of 32 elements.
 *
 * Block tables: i_bl[2*b+0], i_bl[2*b+1] (and j_bl likewise) are the
 * inclusive index ranges of box b, as in solverFuncs.hpp:43-47.  Cells in the
 * union of the boxes are grid cells; couplings from a grid cell to a non-grid
 * cell are dropped (HYPRE StructMatrix semantics) by the SMG-replacement
 * solves, while the SOR replacement reads non-grid neighbours from the
 * solution array exactly as solver_SOR does (solverFuncs.hpp:193-194).
 *
 * Stencil convention (solverFuncs.hpp:77-81):
 *     aP*x_P - aE*x_{i+1} - aW*x_{i-1} - aN*x_{j+1} - aS*x_{j-1} = b_P.
 */
#ifndef CATHODE_B200_H
#define CATHODE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTH_OK 0
#define CTH_NOT_CONVERGED 1
#define CTH_NONFINITE 2
#define CTH_ERR_ARG -1
#define CTH_ERR_CUDA -2
#define CTH_ERR_ALLOC -3
#define CTH_ERR_UNSUPPORTED -4

/* arithmetic of the multigrid cycle */
#define CTH_PREC_FP64 0  /* plain FP64 multigrid                                  */
#define CTH_PREC_MIXED 1 /* FP32 multigrid + FP64 defect correction (FP64 residual) */

typedef struct cth_status {
    int iterations;          /* V-cycles (SMG replacement) or sweeps (SOR replacement) */
    int converged;           /* 1 when the stopping rule was met                        */
    int nonfinite;           /* 1 when a NaN/Inf residual or update was seen             */
    int guess;               /* SMG: 0 started from zero; 1 from the caller's guess
                                (2: from the second candidate, see warm_start 1);
                                -1 guess rejected by its threshold (started from zero)  */
    double residual;         /* SMG: final ||b-Ax||_2/||b||_2; SOR: last max relative update */
    double initial_residual; /* SMG: ||b||_2 of the grid cells; SOR: 0                  */
    double guess_residual;   /* SMG: ||b-A x0||_2/||b||_2 of the guess (-1: no guess)   */
} cth_status;

typedef struct cth_grid cth_grid; /* opaque: grid shape, block union, device workspace */

/* Library / device information ------------------------------------------- */
const char* cth_version(void);
const char* cth_last_error(void);

/* Grid ------------------------------------------------------------------- */
/* Creates the grid of an (ni+2) x (nj+2) index space with n_bl boxes on CUDA
 * device `device`.  Replaces the HYPRE_StructGrid set-up that solver_SMG
 * repeats on every call (include/solverFuncs.hpp:38-49): the block union,
 * its device mask and the multigrid hierarchy are built once per grid. */
int cth_grid_create(int ni, int nj, const int* i_bl, const int* j_bl, int n_bl, int device,
                    cth_grid** out);
void cth_grid_destroy(cth_grid* g);
/* leading dimension (elements) of the device layout */
int cth_grid_ld(const cth_grid* g);
/* number of multigrid levels of the hierarchy */
int cth_grid_levels(const cth_grid* g);
/* set smoothing sweeps per level (pre, post; default 1, 1) */
int cth_grid_set_cycle(cth_grid* g, int nu_pre, int nu_post);
/* enable (default) or disable running each SMG-replacement solve as one
 * captured CUDA graph whose cycle loop is a device-side conditional node; when
 * disabled, or while profiling is on, kernels are launched one by one and the
 * host tests convergence after every cycle.  Results are identical. */
int cth_grid_set_graphs(cth_grid* g, int enable);
/* enable or disable (default) the fused coarse tail: the multigrid levels of
 * at most 16 rows run as one thread-block-cluster launch per cycle instead of
 * one launch per relaxation.  Same sweeps in the same order; results agree to
 * rounding.  Off by default: the separate launches with programmatic
 * dependent launch measured faster on the 512 x 1024 step. */
int cth_grid_set_tail(cth_grid* g, int enable);
/* Hierarchy reuse (no counterpart in the reference, whose SMG builds its
 * hierarchy -- line factorisations, interpolation weights, Galerkin operators
 * -- in every solve).  With tol > 0, a solve given a slot (0..14) keeps the
 * hierarchy of that slot while its operator stays close to the one the
 * hierarchy was built from: before the cycles, a device kernel measures the
 * largest row-relative change max_k |a_k - a_k'| / |a_P| of the scaled
 * operator against the kept one and rebuilds the hierarchy when it exceeds
 * tol (both operators are compared after scaling to the same reference
 * coefficient), when the slot is new or when the slot's previous solve did
 * not converge.  A small coefficient change can still matter (a change of the
 * row sums of a nearly singular operator), so the cycles check themselves: a
 * cycle on the kept hierarchy that reduces the residual by less than a factor
 * 2 ends the first loop, the hierarchy is rebuilt from the solve's operator and
 * a second loop continues from the current iterate.  The kept hierarchy is
 * only the preconditioner of the FP64 defect correction: residuals and the
 * stopping rule use the caller's operator, so every solve meets the same
 * tolerance.  The time step's sweeps give each recurring equation its own
 * slot (cth_fields_* solves on this grid); `slot` (-1: none) is the slot of
 * the solves entered through this header's cth_smg_solve* calls.  tol = 0
 * (default): the hierarchy is built in every solve.  Each slot holds its own
 * hierarchy once used (about 150 bytes per grid cell in FP32, twice that in
 * FP64). */
int cth_grid_set_reuse(cth_grid* g, double tol, int slot);
/* out[0..4]: set-ups, reuses, the last measured change, the last solve's cycle
 * count and the retries of a slot's hierarchy of the given precision
 * (synchronises the device).  A retry: a cycle on the kept hierarchy reduced
 * the residual by less than a factor 2, so the solve rebuilt the hierarchy
 * from its operator and continued from its current iterate (counted among the
 * set-ups too). */
int cth_grid_reuse_stats(cth_grid* g, int precision, int slot, double* out);

/* Instrumentation ------------------------------------------------------------
 * cth_launch_count: kernels this grid has launched since creation.
 * cth_profile(g, 1) resets and enables per-kernel-class timing (CUDA events
 * recorded on the launching stream around each launch of the class);
 * cth_profile_read returns the summed device time (ms), the number of timed
 * launches and the summed algorithmic bytes of a class:
 *   CTH_PROF_RELAX0    finest-level z-line relaxation (one colour per launch)
 *   CTH_PROF_UPDATE    FP64 defect-correction residual
 *   CTH_PROF_RESTRICT0 finest-level restriction
 *   CTH_PROF_SETUP     per-solve set-up (weights + Galerkin products)
 *   CTH_PROF_RELAXC    z-line relaxations of the coarse levels (9-point stencils;
 *                      bytes: 12 words per cell of the colour) */
#define CTH_PROF_RELAX0 0
#define CTH_PROF_UPDATE 1
#define CTH_PROF_RESTRICT0 2
#define CTH_PROF_SETUP 3
#define CTH_PROF_RELAXC 4
long long cth_launch_count(const cth_grid* g);
int cth_profile(cth_grid* g, int enable);
int cth_profile_read(const cth_grid* g, int cls, double* ms, long long* launches, double* bytes);
/* cth_grid_time_relax: device time per launch of the z-line relaxation of one
 * multigrid level in its operating mode -- `reps` pairs of (even rows, odd
 * rows) captured in one CUDA graph with programmatic dependent launch, as the
 * smoother runs inside a cycle -- and the algorithmic bytes of one launch
 * (rows of one colour x cells x 8 words).  Needs a previous solve of that
 * precision on the grid (its operator and factors); overwrites that level's
 * cycle scratch.  Synchronises the grid's stream. */
int cth_grid_time_relax(cth_grid* g, int precision, int level, int reps, double* us_per_launch,
                        double* bytes_per_launch);
/* cth_grid_time_cycle: device time per cycle of `reps` multigrid cycles captured
 * one after another in one CUDA graph, without the solve's device-side loop
 * node: V-cycle + FP64 defect correction (with_update = 1) or the V-cycle
 * alone.  Against the per-cycle time of a solve it separates the loop node's
 * cost.  Needs a previous solve of that precision on the grid; leaves the
 * grid's solve state undefined (the next solve prepares its own).
 * Synchronises the grid's stream. */
int cth_grid_time_cycle(cth_grid* g, int precision, int reps, int with_update, double* us_per_cycle);

/* SMG replacement (host arrays) ----------------------------------------------
 * Drop-in for solver_SMG (include/solverFuncs.hpp:26-163): solves the 5-point
 * system on the block union from a zero initial guess and stops when
 * ||b-Ax||_2/||b||_2 < error_cnv or after maxITR cycles.  Only grid cells of
 * `solution` are written (solverFuncs.hpp:143-152).  `precision` is
 * CTH_PREC_FP64 or CTH_PREC_MIXED.  `st` may be NULL. */
int cth_smg_solve(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, int maxITR,
                  double error_cnv, int precision, double* solution, cth_status* st);

/* SMG replacement (device arrays, library layout, caller's stream) -----------
 * Same contract on device-resident planes.  All pointers are device pointers
 * in the layout above; `solution` grid cells are written, other cells are left
 * untouched.  `stream` is a cudaStream_t (NULL = legacy default stream).  The
 * call returns after the solve completes on `stream`.  Calls on one grid must
 * not overlap (the grid's workspace is shared). */
int cth_smg_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                      const double* aN, const double* aS, const double* b, int maxITR,
                      double error_cnv, int precision, double* solution, void* stream,
                      cth_status* st);
/* Same solve from the device plane x0 as initial guess (no counterpart in the
 * reference, whose SMG always starts from zero): the cycles start from x0 when
 * ||b - A x0||_2 <= max_guess_relres ||b||_2 (at most 10), otherwise from zero (the plain
 * solve is the fallback); st->guess / guess_residual report which.  The
 * stopping rule is unchanged, so the converged residual is the same; x0 may
 * alias solution. */
int cth_smg_solve_guess_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                            const double* aN, const double* aS, const double* b, const double* x0,
                            double max_guess_relres, int maxITR, double error_cnv, int precision,
                            double* solution, void* stream, cth_status* st);

/* SOR replacement (host arrays) ----------------------------------------------
 * Drop-in for solver_SOR (include/solverFuncs.hpp:169-217) with red-black
 * ordering on the GPU: same update formula (neighbours read from `solution`,
 * division by aP+1e-100, relaxation alpha_SOR), same stopping rule (max over
 * grid cells of fabs((new-old)/(new+old+1e-6))*2 <= error_cnv, or the sweep
 * that takes the count past maxITR).  `solution` is the in/out initial guess
 * including its non-grid (ghost) values, which are read but not written. */
int cth_sor_solve(cth_grid* g, const double* aP, const double* aE, const double* aW,
                  const double* aN, const double* aS, const double* b, double alpha_SOR,
                  int maxITR, double error_cnv, double* solution, cth_status* st);

/* SOR replacement (device arrays, library layout) */
int cth_sor_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                      const double* aN, const double* aS, const double* b, double alpha_SOR,
                      int maxITR, double error_cnv, double* solution, void* stream,
                      cth_status* st);

/* Complex 5-point solve (frequency-domain microwave systems) -----------------
 * Replaces the direct sparse factorisation of the reference's complex field
 * systems (Eigen SparseLU, include/emfieldModule.hpp:2995-2998 in
 * solve_Microwave, :5780-5783 in solve_Microwave_impedanceTest): solves
 *     aP x_P - aE x_E - aW x_W - aN x_N - aS x_S = b
 * on the block union (the field's unknowns; couplings to other cells dropped,
 * as the Eigen assembly inserts only unknown-to-unknown entries) by BiCGStab
 * in complex FP64, preconditioned with exact complex z-line solves, from a zero
 * guess until ||r||_2/||b||_2 < tol or maxITR iterations.  Complex arrays are
 * interleaved (re, im) doubles: host arrays [i][j] of (ni+2)*(nj+2) complex
 * values, device arrays planes of (nj+2)*ld complex values, element (i,j) at
 * 2*(j*ld+i).  Only grid cells of `solution` are written.  `st->iterations`
 * counts BiCGStab iterations (two preconditioned products each). */
int cth_c5_solve(cth_grid* g, const double* aP, const double* aE, const double* aW, const double* aN,
                 const double* aS, const double* b, int maxITR, double tol, double* solution,
                 cth_status* st);
int cth_c5_solve_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                     const double* aN, const double* aS, const double* b, int maxITR, double tol,
                     double* solution, void* stream, cth_status* st);

/* Microwave Er system (device arrays) ------------------------------------------
 * Assembles the Er equation of EmfieldModule::solve_Microwave
 * (include/emfieldModule.hpp:2350-2395) with B = 0 — sigma_rr = n e^2/(m(nu+iw)),
 * no Hall coupling to Ex or Ephi — on the r-z rectangle with the impedance test's
 * boundary codes: port excitation (code 7) on the z = 0 faces with
 * r1 <= r <= r2, open (code 1) on the other z = 0 faces and at z = L, Gauss
 * (code 2) at r = R, Er = 0 on the axis face.  ne, nu, epsr: real device planes
 * of cell values (library layout); outputs: complex planes (aP..aS, b) for the
 * Er faces i = 1..ni, j = 2..nj (zero elsewhere).  Solve them with
 * cth_c5_solve_dev on a grid whose single block is i in [1,ni], j in [2,nj]. */
typedef struct cth_mw_params {
    double dx, dr;     /* cell sizes in z and r                       */
    double rmin;       /* r of the lower domain edge (0 on the axis)  */
    double omegam;     /* microwave angular frequency                 */
    double J1r_exc;    /* port excitation current                     */
    double r1, r2;     /* port radii                                  */
    double masse;      /* electron mass                               */
} cth_mw_params;
int cth_mw_er_assemble_dev(cth_grid* g, const double* ne, const double* nu, const double* epsr,
                           const cth_mw_params* prm, double* aP, double* aE, double* aW, double* aN,
                           double* aS, double* b, void* stream);

/* Impedance test (device arrays) ----------------------------------------------
 * The reference's calibration mode (flag_impTest == 1, src/main.cpp:126-132):
 * the coax of InitialModule::makeBoundary_impedanceTest (initialModule.hpp:
 * 1061-1330: r in [rmin, rmax] = [r1, r2], epsr = epsr_diele in the cells) and
 * EmfieldModule::solve_Microwave_impedanceTest (emfieldModule.hpp:5528-6099)
 * without plasma: the Er equation on the faces i = 1..ni, j = 2..nj with the
 * port excitation (code 7) at the left end, the open end (code 1) at the right,
 * Gauss (code 2) on both conductors; the complex BiCGStab solve of
 * cth_c5_solve_dev to tol; then the ghosts of the code-7 and Gauss walls, the
 * port current and voltage at x_ref = 0, the wave amplitudes for Z0, and E1r
 * (every entry) scaled by sqrt(Pmw / P_fwd).  g: a grid whose single block is
 * [1, ni] x [2, nj]; epsr: real device plane of cell values; E1r: complex device
 * plane (library layout, (re, im) interleaved).  The caller multiplies its
 * J1r_exc by res->J1r_exc_factor as the reference does (:6036).  Waits for the
 * stream. */
typedef struct cth_impedance_params {
    double dx, dr, rmin;      /* r_j = rmin + (j - 1/2) dr                  */
    double omegam, J1r_exc;   /* angular frequency, port excitation current */
    double r1, r2;            /* conductor radii                            */
    double Z0, Pmw;           /* line impedance, forward power              */
} cth_impedance_params;
typedef struct cth_impedance_result {
    double V[2], I[2];        /* port voltage and current (re, im)          */
    double P_fwd, P_ref;      /* |b2|^2, |a2|^2 before the rescale (W)      */
    double ratio, J1r_exc_factor;
    cth_status solve;
} cth_impedance_result;
int cth_mw_impedance_test(cth_grid* g, const double* epsr, const cth_impedance_params* prm, int maxITR,
                          double tol, double* E1r, void* stream, cth_impedance_result* res);

/* Microwave diagnostics of OutputModule::output_phase (outputModule.hpp:38-184):
 * Emag_rep = sqrt(mean over cells i = 1..ni, j = 1..nj of |E|^2 at the cell
 * centre), and on the cells of g's blocks (gc.jdgBnd_Ep: the six cell blocks)
 * the normalised divergences divE = div(E) dx / Emag_rep, divJ = div(J) dx /
 * (Emag_rep w eps0) and divEJ = (divJ + i w eps0 divE) dx / (Emag_rep w eps0)
 * (normalising the already normalised values, as the reference does); zero
 * elsewhere.  Complex planes of the library layout; r_j = rmin + (j-1/2) dr.
 * Waits for the stream. */
int cth_mw_divergence(cth_grid* g, const double* E1x, const double* E1r, const double* E1p, const double* J1x,
                      const double* J1r, const double* J1p, double dx, double dr, double rmin, double omegam,
                      double* divE, double* divJ, double* divEJ, double* Emag_rep, void* stream);

/* Magnetised 3-component microwave system of solve_Microwave
 * (include/emfieldModule.hpp:2249-2998): Ex on x-faces, Er on r-faces, Ephi on
 * cells, coupled through the magnetised cold-plasma conductivity (11-point
 * rows, :2300-2453), with the reference's boundary codes 0-7 (:2456-2784).
 * Replaces the assembly of :2785-2990 and the Eigen SparseLU factorisation
 * (:2995-2998) by complex FP64 BiCGStab, right-preconditioned block-diagonally
 * by one complex semicoarsening V-cycle per field.  The domain starts on the
 * axis (prm->rmin must be 0).
 * Field planes (x3, y3, E3): three consecutive complex planes Ex, Er, Ephi of
 * (nj+2) x ld complex values each (library layout, ld = cth_mw3_ld). */
typedef struct cth_mw3 cth_mw3;
/* The r-z rectangle r in [0, R], z in [0, L]: unknowns Ex i = 2..ni,
 * j = 1..nj; Er i = 1..ni, j = 2..nj; Ephi i = 1..ni, j = 1..nj; boundary lists
 * of its walls (rebuilt from prm at each assembly): Ex Gauss (2) at z = 0, L and
 * conductor (0) at r = R; Er port (7) on [r1, r2] at z = 0, open (1) on the
 * other z = 0 faces and at z = L, Gauss (2) at r = R; Ephi open (1) at z = 0,
 * conductor (0) at z = L and r = R. */
int cth_mw3_create(int ni, int nj, int device, cth_mw3** out);
/* A general geometry: the unknowns of each field are the union of its blocks,
 * i_bl / j_bl = n_bl pairs [lo, hi] each (inclusive; the x-face, r-face and
 * cell blocks gx.i_flx_bl, gr.i_flr_bl, gc.i_flc_bl of the reference,
 * initialModule.hpp:219-345, six blocks on the cathode).  Every block inside
 * [1, ni] x [1, nj]; Er blocks from j = 2.  Boundary lists follow with
 * cth_mw3_set_boundary. */
int cth_mw3_create_blocks(int ni, int nj, const int* xi_bl, const int* xj_bl, int nx_bl, const int* ri_bl,
                          const int* rj_bl, int nr_bl, const int* ci_bl, const int* cj_bl, int nc_bl, int device,
                          cth_mw3** out);
/* One boundary list of MicrowaveBC (include/arrays.hpp:649): the entries
 * (i[k], j[k], code[k]), k < n, of iBnd / jBnd / sBnd for one side and field. */
typedef struct cth_bc_list {
    const int* i;
    const int* j;
    const int* code;
    int n;
} cth_bc_list;
/* lists[12]: Ex W, E, S, N (iBndWx .. iBndNx), Er W, E, S, N (iBndWr ..), Ephi
 * W, E, S, N (iBndWp ..), as InitialModule::makeBoundary builds them
 * (initialModule.hpp:420-1055), applied at each assembly in that order.  Every
 * entry must be an unknown of its field, appear once in its list and carry a
 * code in 0..7 (CTH_ERR_ARG otherwise).  j_flc_00 = gc.j_flc_bl[0][0], which the
 * reference's Er south code 3 compares with the cell radius (:2672).  Host
 * arrays; copied (waits for the device). */
int cth_mw3_set_boundary(cth_mw3* m, const cth_bc_list* lists, int j_flc_00);
void cth_mw3_destroy(cth_mw3* m);
int cth_mw3_ld(const cth_mw3* m);
long long cth_mw3_launch_count(const cth_mw3* m);
/* ne, nu, Bx, Br, epsr: real device planes of cell values (library layout) */
int cth_mw3_assemble_dev(cth_mw3* m, const double* ne, const double* nu, const double* Bx, const double* Br,
                         const double* epsr, const cth_mw_params* prm, void* stream);
/* The explicit variant, EmfieldModule::solve_Microwave_explicit
 * (emfieldModule.hpp:3328-4400): the plasma conductivity is left out of the
 * operator (vacuum + epsr interior rows, no Hall couplings) and enters the
 * right-hand side as b = -i w mu0 dx^2 dr^2 J on each field's unknowns, J =
 * sigma E of the field before the solve (complex planes J1x, J1r, J1p of the
 * library layout; cth_update_energy_profile computes exactly this J,
 * :7636-7730 being the same formulas as :3384-3470); the boundary lists are
 * applied as in cth_mw3_assemble_dev.  Solve and ghost pass as for the implicit
 * system. */
int cth_mw3_assemble_explicit_dev(cth_mw3* m, const double* epsr, const void* J1x, const void* J1r,
                                  const void* J1p, const cth_mw_params* prm, void* stream);
/* copies the assembled coefficients into a_dst: 3 fields x 11 complex planes
 * (P, E, W, N, S, then the couplings C0..C5 of the field: Ex rows Er at
 * (i,j+1), (i,j), (i-1,j+1), (i-1,j) and Ephi at (i,j), (i-1,j); Er rows Ex at
 * (i+1,j), (i+1,j-1), (i,j), (i,j-1) and Ephi at (i,j), (i,j-1); Ephi rows Ex
 * at (i+1,j), (i,j) and Er at (i,j+1), (i,j)), and the 3 right-hand sides
 * into b_dst (device buffers; asynchronous on stream) */
int cth_mw3_copy_planes(const cth_mw3* m, double* a_dst, double* b_dst, void* stream);
/* y3 = A x3 on the unknowns (x3 is read on the unknowns only; y3 is zero elsewhere) */
int cth_mw3_apply_dev(cth_mw3* m, const double* x3, double* y3, void* stream);
/* solve from a zero start until ||b - A E||_2 / ||b||_2 < tol; E3 receives the
 * three fields on the unknowns (:3007-3024); its entries off the unknowns keep
 * their values (the ghosts of earlier calls, as in the reference's persistent
 * fields).  CTH_NOT_CONVERGED after maxit. */
int cth_mw3_solve_dev(cth_mw3* m, int maxit, double tol, double* E3, void* stream, cth_status* st);
/* the same from an initial guess (no counterpart in the reference, whose
 * SparseLU has no start): x0 holds three field planes in E3's layout, read on
 * the unknowns (x0 may be E3 itself: the previous solution).  The guess is used
 * when ||b - A x0||_2 <= guess_tol ||b||_2, decided on the device; otherwise the
 * solve starts from zero, as cth_mw3_solve_dev.  Same stopping rule; a guess that
 * already meets it ends the solve with 0 iterations.  st->guess: 1 used, -1
 * rejected; st->guess_residual its relative residual. */
int cth_mw3_solve_guess_dev(cth_mw3* m, int maxit, double tol, double* E3, const double* x0, double guess_tol,
                            void* stream, cth_status* st);
/* the boundary post-processing of solve_Microwave (:3026-3264): ghost values of
 * E1x, E1r, E1p written from E3's unknowns list by list in the reference's
 * order (reading the ghosts of earlier lists and calls where the reference
 * does).  Er_dc = gr.Er (real plane, library layout), which the Er east code 1
 * reads (:3162); it may be NULL when no such entry exists.  CTH_ERR_UNSUPPORTED
 * when a list would write a ghost onto an unknown of its field. */
int cth_mw3_fill_ghosts(cth_mw3* m, double* E3, const double* epsr, const double* Er_dc, const cth_mw_params* prm,
                        void* stream);
/* run the solve as one captured CUDA graph with a device-side conditional loop
 * (default, 1) or kernel by kernel with a host convergence test per iteration
 * (0); same kernels, same results */
int cth_mw3_set_graphs(cth_mw3* m, int enable);
/* smoothing sweeps per level of the three fields' V-cycles (pre, post in 1..8;
 * default 1, 1); waits for the device and drops the captured solve */
int cth_mw3_set_cycle(cth_mw3* m, int nu_pre, int nu_post);
/* preconditioner: 0 = block Jacobi, the three fields' V-cycles side by side
 * (default); 1 = block Gauss-Seidel, Ex then Er then Ephi, each V-cycle's
 * right-hand side with the couplings to the fields before it taken out (the
 * V-cycles run one after another).  Waits for the device, drops the captured
 * solve. */
int cth_mw3_set_preconditioner(cth_mw3* m, int mode);
/* precision of the preconditioner's V-cycles: CTH_PREC_FP64 (complex double,
 * default) or CTH_PREC_MIXED (complex float hierarchy: each field's level-0
 * operator and right-hand side rounded to FP32, the result widened back; the
 * BiCGStab recurrence, its matrix products, residuals and stopping test stay
 * FP64, so the solve reaches the same tolerance).  Waits for the device, drops
 * the captured solve. */
int cth_mw3_set_precision(cth_mw3* m, int precision);

/* Fluid state in HBM -----------------------------------------------------------
 * A field store holds named device planes of the grid's library layout (cell
 * arrays and the x-face (i-1/2) / r-face (j-1/2) arrays share the (ni+2)x(nj+2)
 * index space, as in the reference, fluidModule.hpp:156-173), the per-cell side
 * flags of the fluid blocks and the BolsigVec rate tables (arrays.hpp:703-716).
 * Field names are the reference's member names (rhoe, Te, mu_perp, rhoUex, ...).
 * cth_field returns the device plane (created zeroed on first use).
 * Side-flag bits (1 = ordinary face on that side, 0 = the wall / axis / open
 * boundary of the reference's bLx_wall, bRx_wall, bLr_wall, bLr_cen, bRr_wall,
 * bRr_open expressions, e.g. fluidModule.hpp:2660-2686); a zero byte marks a
 * cell outside the fluid blocks. */
#define CTH_F_BLX 1
#define CTH_F_BRX 2
#define CTH_F_BLR_WALL 4
#define CTH_F_BLR_CEN 8
#define CTH_F_BRR_WALL 16
#define CTH_F_BRR_OPEN 32
#define CTH_F_BRX_BIAS 64 /* the right wall is the biased electrode (z5, fluidModule.hpp:2196-2199) */
#define CTH_F_BRR_INLET 128 /* the upper wall is the neutral gas inlet (fluidModule.hpp:5040-5041) */
typedef struct cth_fields cth_fields;
int cth_fields_create(cth_grid* g, cth_fields** out);
void cth_fields_destroy(cth_fields* fs);
double* cth_field(cth_fields* fs, const char* name);
int cth_field_upload(cth_fields* fs, const char* name, const double* host_ij);
int cth_field_download(cth_fields* fs, const char* name, double* host_ij);
/* Batched transfers of n fields ([i][j] host arrays as for cth_field_upload /
 * cth_field_download): all copies and layout transposes are queued on `stream`
 * (NULL: the grid's stream), then one synchronisation.  With pinned host arrays
 * the copies run at full link speed; the staging for n planes is allocated on
 * the first call.  Ordered after earlier work on `stream` (pass the stream of
 * the time step). */
int cth_fields_upload_many(cth_fields* fs, const char* const* names, const double* const* host_ij, int n,
                           void* stream);
int cth_fields_download_many(cth_fields* fs, const char* const* names, double* const* host_ij, int n, void* stream);
int cth_flags_upload(cth_fields* fs, const unsigned char* host_ij);
/* table names: nu_elas_N nu_exc_N nu_excReso_N nu_excMeta_N nu_ionz_N nu_ionzStep_N
 * nu_excStep_N nu_super_N rate_eloss_n_N rate_eloss_m_N nui_m_N */
int cth_table_upload(cth_fields* fs, const char* name, const double* values, int n);

/* FluidModule::update_transport_coef (fluidModule.hpp:5799-5976): anomalous
 * ion-acoustic frequency and Mach number on the fluid cells, collision
 * frequencies from the rate tables (uniform-step lookups of miniFuncs.hpp:35-91),
 * ionisation source rate_ionize, ion momentum frequency, energy-loss rate and
 * its Te derivative, and the magnetised mobility tensor on every cell. */
typedef struct cth_transport_params {
    double masse, massi, Ti, nu_eff;
    double dTe, dEi;      /* table steps (Params::dTe, Params::dEi)        */
    double dr, rmin;      /* radial grid: r_j = rmin + (j - 1/2) dr       */
    int flag_Bohm, flag_Sagdeev;
} cth_transport_params;
int cth_update_transport_coef(cth_fields* fs, const cth_transport_params* prm, void* stream);

/* FluidModule::solve_phi_couple_wdTe_wSEE_PC (fluidModule.hpp:2080-3075):
 * predictor-corrector for the potential with dielectric relaxation.  Reads the
 * store's rhoe, rhoe_old, rhoi, Te, mu_para, mu_perp, mu_rr, mu_xr, mu_xx,
 * rate_ionize, Uix, Uir, rhoUmx, rhoUmr and the SEE tables coefEISEE_eb_table,
 * coefEISEE_rd_table, coefEISEE_ts_table; updates phi, Ex, Er, nUex, nUer and
 * phi_old, nUex_old, nUer_old (the values at entry).  The grid's blocks must be
 * the fluid blocks the side flags describe.  The inner solve is the SMG
 * replacement (flag_iter_phi != 0, precision as cth_smg_solve_dev) or SOR with
 * alpha 1.9 (flag_iter_phi == 0), from zero, with maxITR_SOR_phi and
 * error_cnv_SOR_phi.  The loop ends when the largest calcRes of phi, nUex, nUer
 * over one iteration is below error_cnv_HES_phi or after maxITR_HES_phi
 * iterations.  Synchronises the stream once per iteration. */
typedef struct cth_phi_params {
    double dt, dx, dr, rmin, V_bias, masse;
    double coefIISEE_ts, coefMISEE_ts, dTe_SEE;
    double error_cnv_HES_phi, error_cnv_SOR_phi;
    int maxITR_HES_phi, maxITR_SOR_phi;
    int flag_error;     /* calcRes mode 0..3 (miniFuncs.hpp:292-376) */
    int flag_iter_phi;  /* 0: SOR, otherwise SMG                     */
    int precision;      /* CTH_PREC_MIXED or CTH_PREC_FP64           */
    /* initial guess of the first inner (SMG) solve; no counterpart in the
     * reference, whose solves start from zero.  0: zero (reference);
     * 1: the better (smaller residual) of the store's plane "dphi_guess"
     * (written by the caller, e.g. the learned predictor) and "dphi_prev";
     * 2: "dphi_prev" = the first-iteration correction of the previous call;
     * 3: "dphi_guess" alone (tested only against the zero start).
     * With warm_start != 0 the first iteration's correction is copied into
     * "dphi_prev" (its former content into "dphi_prev2").  A guess whose
     * relative residual exceeds guess_max_relres
     * (at most 10) is dropped (zero start). */
    int warm_start;
    double guess_max_relres;
} cth_phi_params;

typedef struct cth_pc_result {
    int ncount;            /* PC iterations taken                                 */
    int solver_rc;         /* largest positive return of the inner solves (0 ok)  */
    double error_phi, error_nUex, error_nUer;  /* calcRes against the entry values */
    double error_iter[3];  /* calcRes of the last iteration (phi, nUex, nUer)      */
    cth_status solver;     /* status of the last inner solve                      */
    double Ii_Anode, Ie_Anode, I_Anode;  /* anode currents (density sweep only)    */
    cth_status first;      /* status of the first inner solve (initial-guess report) */
} cth_pc_result;
int cth_solve_phi_pc(cth_fields* fs, const cth_phi_params* prm, void* stream, cth_pc_result* res);

/* FluidModule::check_CFL (fluidModule.hpp:57-115): dt_min = eps0 / (e max(rhoe)
 * max(mu_para)) over the index space; flag_adp_dt == 1 sets dt = dt_min CFL,
 * otherwise CFL = dt / dt_min.  ue_max = max electron speed over the grid cells
 * + the thermal speed at max(Te). */
typedef struct cth_cfl {
    double dt, CFL;           /* in/out                      */
    double masse, rmin, dr;   /* in                          */
    int flag_adp_dt;          /* in                          */
    double dt_min, rhoe_max, mu_max, Te_max, ue_max;  /* out */
} cth_cfl;
int cth_check_cfl(cth_fields* fs, cth_cfl* io, void* stream);

/* Ghost rules applied after the electron sweeps (fluidModule.hpp:3884-3921 for
 * rhoe, :4878-4914 for Te): n rules of 7 ints (i0, i1, j0, j1, di, dj, mode),
 * each a one-cell-wide segment of grid cells whose neighbour (i+di, j+dj) is
 * set to 0 (mode 0, rhoe only) or to the cell's value (mode 1; Te is always
 * copied).  Later rules win where targets coincide. */
int cth_ghost_rules_upload(cth_fields* fs, const int* rules, int n);

/* r-face boxes whose recorded wall flux Gr_wall the electron energy sweep leaves
 * unchanged: the reference's lower-wall loop x2 of solve_Te_wdTe_wSEE_PC sets
 * gr.Gr there but not gr.Gr_wall (fluidModule.hpp:4428-4449; the other walls
 * record it, :4423, :4470, :4494, :4504).  n boxes of 4 ints (i0, i1, j0, j1),
 * inclusive r-face indices, n <= 4; n = 0 records every wall (the default). */
int cth_energy_keep_walls_upload(cth_fields* fs, const int* boxes, int n);

/* Warm start of the field-valued solves (no counterpart in the reference, whose
 * solves start from zero): with enable != 0 the ion momentum (Uix, Uir, Uip),
 * ion continuity (rhoi) and neutral (rhon, rhom) solves of the SMG path start
 * from the field's values at the solve (the previous step's), when that
 * guess's relative residual is at most max_relres (<= 10), otherwise from zero.
 * Same stopping rule.  Default off. */
int cth_fields_set_warm_start(cth_fields* fs, int enable, double max_relres);

/* Planned downloads (no counterpart in the reference): the next cth_fluid_step
 * calls copy each listed field into its host array ([i][j] layout, pinned for
 * full speed) on a copy stream of the store as soon as the sweep that finalises
 * it is done -- the ion fields after the ion step, phi / Ex / Er after the
 * potential, rhoe after the electron density, Te / rhoeps after the energy,
 * rhon / rhom after the neutrals, any other field at the end -- so the copies
 * overlap the remaining sweeps.  cth_fields_download_wait returns when the
 * copies of the last step have landed; a following step or upload waits for
 * them on the device by itself.  n = 0 clears the plan. */
int cth_fields_set_download_plan(cth_fields* fs, const char* const* names, double* const* host_ij, int n);
int cth_fields_download_wait(cth_fields* fs);
/* Planned uploads for the next cth_fluid_step only: the listed fields are copied
 * from their host arrays ([i][j], pinned for full speed) on the store's copy
 * stream at the start of the step; the step waits for the fields it reads from
 * the start at once, for rhoeps only before the electron energy sweep and for
 * rhon / rhom only before the neutral sweep, so those copies overlap the sweeps
 * before.  No host synchronisation; the host arrays must stay valid until the
 * next cth_fields_download_wait (or a synchronisation of the step's stream). */
int cth_fields_set_upload_plan(cth_fields* fs, const char* const* names, const double* const* host_ij, int n);

/* Scharfetter-Gummel predictor-correctors of the electron density
 * (cth_solve_rhoe_pc: FluidModule::solve_rhoe_wdTe_wSEE_PC, fluidModule.hpp:3082-3970)
 * and energy (cth_solve_Te_pc: solve_Te_wdTe_wSEE_PC, fluidModule.hpp:4006-4957).
 * Density: reads Te, mu_*, Ex, Er, rhoi, Uix, Uir, rhoUmx, rhoUmr, rate_ionize,
 * rhoUix_wall; updates rhoe, rhoUex, rhoUer, rhoUex_wall, rhoUer_wall and
 * rhoe_old / rhoUex_old / rhoUer_old (entry values); reports the anode currents.
 * Energy: reads rhoe, rhoe_old, rhoUex, rhoUer, Pabs, rate_eloss and the same
 * fields; updates rhoeps, Gx, Gr, Gx_wall, Gr_wall, Te (recovered from rhoeps)
 * and rhoeps_old, Gx_old, Gr_old, Te_old.  In cth_pc_result the three calcRes
 * errors are those of (n, x flux, r flux). */
typedef struct cth_sg_params {
    double dt, dx, dr, rmin, masse;
    double coefIISEE_ts, coefMISEE_ts, dTe_SEE;
    double Te_emitSEE_eV, ratioEngy_EISEE_rd;  /* energy sweep only */
    double error_cnv_HES, error_cnv_SOR;
    int maxITR_HES, maxITR_SOR;
    int flag_error, flag_iter, precision;
} cth_sg_params;
int cth_solve_rhoe_pc(cth_fields* fs, const cth_sg_params* prm, void* stream, cth_pc_result* res);
int cth_solve_Te_pc(cth_fields* fs, const cth_sg_params* prm, void* stream, cth_pc_result* res);

/* Ion sub-step (src/main.cpp:191-197): FluidModule::solve_Uix_tmp, solve_Uir_tmp,
 * solve_Uip_tmp (fluidModule.hpp:123-1404), solve_rhoi_constTe (:1405-1755) and
 * correct_Ui_constTe (:1763-2072).  gx / gr are grids of the same shape whose
 * blocks are the x-face / r-face blocks (the Uix / Uir unknowns); the store's grid
 * holds the cell blocks.  Reads phi, Ex, Er, Bx, Br, rate_ionize, nui_m; updates
 * Uix, Uir, Uip, rhoi, rhoUix, rhoUir, rhoUix_wall, rhoUir_wall and the *_old
 * copies.  The wall conditions of the three momentum equations are wall programs
 * (ordered segment operations, cth_ion_program_upload) built from the named wall
 * segments of the reference's loops; the residuals run over the boxes of
 * cth_ion_boxes_upload (0 rhoi, 1 Uix, 2 Uir, 3 Uip; 4 ints each: i0, i1, j0, j1). */
typedef struct cth_ion_params {
    double dt, dx, dr, rmin, rmax, massi, Ti, V_bias, Te_rep_eV, CFL, error_cnv_SOR;
    int ndt_i, maxITR_SOR, flag_iter, precision, flag_error;
} cth_ion_params;

typedef struct cth_ion_result {
    double error_rhoi, error_Uix, error_Uir, error_Uip;
    int solver_rc;
    int reserved;
    cth_status solver[4];  /* Uix, Uir, Uip, rhoi */
} cth_ion_result;

/* wall-program operation over the points (i, j) of [i0, i1] x [j0, j1] */
enum {
    CTH_ION_WALL_FOLD = 1, /* b += a_dir U_wall, a_dir = 0                                   */
    CTH_ION_ZERO_COEF = 2, /* a_dir = 0                                                       */
    CTH_ION_FOLD_SUB = 3,  /* aP -= a_dir * scale, a_dir = 0                                  */
    CTH_ION_OPEN_FOLD = 4, /* b += aN r_face/r_up max(U_old, 0), aN = 0 (open top)            */
    CTH_ION_SET_WALL = 5,  /* U(i+di, j+dj) = U_wall                                          */
    CTH_ION_SET_ZERO = 6,  /* U(i+di, j+dj) = 0                                               */
    CTH_ION_COPY = 7,      /* U(i+di, j+dj) = scale * U(i, j)                                 */
    CTH_ION_SET_OPEN = 8   /* U(i+di, j+dj) = r_face/r_up max(U_old(i, j), 0)                 */
};
/* programs: assembly / after-solve for Uix, Uir, Uip */
enum { CTH_ION_PROG_UIX_ASM = 0, CTH_ION_PROG_UIX_POST = 1, CTH_ION_PROG_UIR_ASM = 2, CTH_ION_PROG_UIR_POST = 3,
       CTH_ION_PROG_UIP_ASM = 4, CTH_ION_PROG_UIP_POST = 5, CTH_ION_NPROG = 6 };
typedef struct cth_ion_op {
    int kind, i0, i1, j0, j1;
    int di, dj;   /* target offset (SET_*, COPY)                                         */
    int dir;      /* coefficient: 0 aW, 1 aE, 2 aS, 3 aN                                  */
    int sign;     /* U_wall sign (-1 low side, +1 high side)                              */
    int bias;     /* U_wall measured from V_bias (the biased electrode)                   */
    int pair;     /* U_wall potential: 0 mean of cells i-1, i; 1 mean of cells j-1, j       */
    int scale;    /* 0: 1, 1: r_j / r_{j-1}, 2: r_j / r_{j+1}                              */
} cth_ion_op;
int cth_ion_program_upload(cth_fields* fs, int which, const cth_ion_op* ops, int n);
int cth_ion_boxes_upload(cth_fields* fs, int which, const int* boxes, int n);
int cth_ion_step(cth_fields* fs, cth_grid* gx, cth_grid* gr, const cth_ion_params* prm, void* stream,
                 cth_ion_result* res);

/* Neutrals: FluidModule::update_rhon (fluidModule.hpp:4963-5410) then update_rhom
 * (:5416-5792).  Reads rhoUix_wall, rhoUir_wall, rhoe and the collision
 * frequencies nu_excStep, nu_super, nu_excMeta, nu_exc, nu_ionz, nu_ionzStep;
 * updates rhon, rhom, their face fluxes rhoUnx, rhoUnr, rhoUmx, rhoUmr, the wall
 * fluxes *_wall and the *_old copies.  Cells flagged CTH_F_BRR_INLET take the
 * inlet flux fn_In through their upper face.  rhom is kept non-negative on the
 * pos_box boxes (the reference: fluid blocks 0 and 1). */
typedef struct cth_neutral_params {
    double dt, dx, dr, rmin, fn_In, Tn, ri, massi, DmN, error_cnv_SOR;
    int ndt_n, ndt_m, maxITR_SOR, flag_iter, precision, flag_error;
    int n_pos_box;
    int pos_box[8][4];  /* i0, i1, j0, j1 */
    int do_rhon, do_rhom;  /* run update_rhon / update_rhom (the time loop's ndt_n / ndt_m) */
} cth_neutral_params;
typedef struct cth_neutral_result {
    double error_rhon, error_rhom;
    int solver_rc;
    int reserved;
    cth_status solver[2];
} cth_neutral_result;
int cth_update_neutrals(cth_fields* fs, const cth_neutral_params* prm, void* stream, cth_neutral_result* res);

/* One time step of the fluid model in the order of the reference's time loop
 * (src/main.cpp:170-251): check_CFL (dt or CFL), the ion sub-step every ndt_i
 * steps, the potential, electron density and energy predictor-correctors, the
 * neutral sweeps every ndt_n / ndt_m steps and the transport coefficients.  The
 * dt and CFL of the sub-step parameter blocks are overwritten by the step's. */
typedef struct cth_step_params {
    int itime;                 /* in/out: incremented at the start of the step   */
    int ndt_i, ndt_n, ndt_m;
    int flag_adp_dt;
    double dt, CFL, gtime;     /* in/out                                        */
    cth_ion_params ion;
    cth_phi_params phi;
    cth_sg_params rhoe, eps;
    cth_neutral_params neutral;
    cth_transport_params transport;
    /* learned warm start (no counterpart in the reference): with phi.warm_start
     * == 1 and net not null, cth_unet_predict_dphi fills "dphi_guess" before the
     * potential predictor-corrector (concurrently with the ion step).  After 4
     * consecutive predictions that the device-side guess selection did not take, the network
     * runs only on steps with itime % 8 == 0 until it is chosen again; the other
     * steps start from the previous correction (warm_start 2). */
    struct cth_unet* net;
} cth_step_params;
typedef struct cth_step_result {
    cth_ion_result ion;
    cth_pc_result phi, rhoe, eps;
    cth_neutral_result neutral;
    cth_cfl cfl;
    int ran_ion, ran_rhon, ran_rhom;
    int net_ran;          /* the learned predictor ran in this step */
    int solver_rc;             /* largest positive inner-solve return          */
} cth_step_result;
int cth_fluid_step(cth_fields* fs, cth_grid* gx, cth_grid* gr, cth_step_params* p, void* stream,
                   cth_step_result* res);

/* Residual (device arrays): r = b - A x on grid cells (couplings to non-grid
 * cells dropped), r = 0 elsewhere; *rnorm = ||r||_2, *bnorm = ||b||_2 over grid
 * cells (either may be NULL). */
int cth_residual_dev(cth_grid* g, const double* aP, const double* aE, const double* aW,
                     const double* aN, const double* aS, const double* b, const double* x,
                     double* r, double* rnorm, double* bnorm, void* stream);

/* Residual without allocation (device arrays) ---------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory when they need a residual (a program whose own pool owns all device
 * memory, a loop that cannot take the synchronisation an allocation can
 * cause): same result as
 * cth_residual_dev, but it needs no cth_grid and calls no allocator.  Its
 * scratch is one static device array of CTH_NOALLOC_SCRATCH_BYTES per GPU
 * (held until exit); (nj+2)*ld may not exceed CTH_NOALLOC_MAX_PLANE and n_bl
 * may not exceed 64, otherwise CTH_ERR_ARG.  ld >= ni+2 is the caller's leading
 * dimension of the library layout.  The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and may return
 * wrong norms.  The call synchronises `stream` and returns after the norms are
 * on the host. */
#define CTH_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
#define CTH_NOALLOC_MAX_PLANE (CTH_NOALLOC_SCRATCH_BYTES - 256u * 1024u)
int cth_residual_noalloc(int ni, int nj, int ld, const int* i_bl, const int* j_bl, int n_bl,
                         const double* aP, const double* aE, const double* aW, const double* aN,
                         const double* aS, const double* b, const double* x, double* r,
                         double* rnorm, double* bnorm, void* stream);

/* Restart files ---------------------------------------------------------------
 * The reference's restart CSV: OutputModule::output writes restart<nOut>.csv
 * (outputModule.hpp:429-470: i, j, x, r, 49 fields, zero; %.17e reals, |v| <
 * 1e-100 written as 0, Te and Te_old in eV), InputModule::input_restart_data
 * reads it (inputModule.hpp:667-1157).  x[ni+2], r[nj+2] are the cell-centre
 * coordinates gc.x, gc.r (x_i = xL + (i - 1/2) dx, r_j = rmin + (j - 1/2) dr).
 *
 * cth_restart_write queues the device-to-host copies of the 49 fields on
 * `stream` (later work on that stream cannot change what is written) and
 * returns; a host thread formats and writes the file.  cth_restart_wait joins
 * that thread and returns its status; a second write waits for the first.
 *
 * cth_restart_read reads a file into the store: the 39 variables of the
 * reference's registry that the header holds (the wall fluxes are written but
 * not read), Te from eV; the index range, duplicate and missing cells and the
 * coordinates (1e-12 + 1e-10 relative) are checked (CTH_ERR_ARG with the line
 * where the reference aborts).  Then the reference's post-processing on the
 * device: rhoe = 0 outside the fluid cells, Ex / Er from phi on the interior
 * face blocks of gx / gr, the wall ghosts of phi (V_bias on the biased wall),
 * E on the wall faces, Er = 0 on the axis.  Synchronises `stream`. */
typedef struct cth_restart_params {
    double dx, dr, V_bias;
} cth_restart_params;
typedef struct cth_restart_info {
    int rows;              /* cells read: (ni+2)*(nj+2)                          */
    int variables_read;    /* registry variables present in the header (<= 39)   */
    int unknown_columns;   /* header columns neither registry, coordinate, wall flux nor zero */
} cth_restart_info;
int cth_restart_write(cth_fields* fs, const char* path, const double* x, const double* r, void* stream);
int cth_restart_wait(cth_fields* fs);
int cth_restart_read(cth_fields* fs, cth_grid* gx, cth_grid* gr, const char* path, const double* x,
                     const double* r, const cth_restart_params* prm, void* stream, cth_restart_info* info);

typedef struct cth_mw_update cth_mw_update;  /* the microwave update, declared below */
struct cth_unet;                              /* the network, declared below */

/* Batched instances (the I-V sweeps; no counterpart in the reference, which runs
 * one discharge per process) -------------------------------------------------
 * cth_batch_steps advances n independent instances (own grids, store, step
 * parameters) by `steps` time steps each, with min(nthreads, n) host worker
 * threads; instance k belongs to thread k % T, which interleaves its instances
 * step by step on one stream per instance.  Results are those of the same
 * steps run one instance after another.  Returns the worst status (negative if
 * an instance failed; that instance stops, the others continue); per item: rc,
 * steps done, wall seconds and the anode currents of its last step
 * (FluidModule::solve_rhoe_wdTe_wSEE_PC, fluidModule.hpp:3944-3964);
 * *wall_seconds = the whole batch.  An item with mw set also runs that
 * microwave update after every step whose itime it is due on (its Pmw then
 * drives the instance's heating); mw_runs counts them and mw_power_sum /
 * mw_J1r_exc report the last one. */
typedef struct cth_batch_item {
    cth_fields* fs;
    cth_grid* gx;
    cth_grid* gr;
    cth_step_params* params;
    int rc;
    int steps_done;
    double seconds;
    double I_Anode, Ii_Anode, Ie_Anode;  /* anode currents of the last step (the I-V point) */
    cth_mw_update* mw;                   /* optional microwave update (NULL: none)          */
    int mw_runs;
    double mw_power_sum, mw_J1r_exc;
} cth_batch_item;
int cth_batch_steps(cth_batch_item* items, int n, int steps, int nthreads, double* wall_seconds);

/* Absorbed microwave power: the volume part of EmfieldModule::
 * update_energy_profile (emfieldModule.hpp:7630-7790).  E1x, E1r, E1p are
 * complex (re, im interleaved) device planes of the library layout holding the
 * field on the x-faces (gx.E1x, face i-1/2), r-faces (gr.E1r, face j-1/2) and
 * cells (gc.E1p); gx / gr are grids over the x-face / r-face block unions
 * (the store's grid gives the cell blocks).  Writes J1x, J1r, J1p (complex
 * planes: J = sigma E with the magnetised cold-plasma tensor of rhoe, nu_m1,
 * Bx, Br), the store's planes Pabsx, Pabsr, Pabsp (Re(J.E*)/2) and Pabs (their
 * cell profile) on the block cells, and the volume integrals.  The port,
 * reflection and field-rescaling part (flag_mwRef, :7792-8105) is
 * cth_mw_port_rescale, below. */
typedef struct cth_energy_params {
    double dx, dr, rmin, omegam, masse;
} cth_energy_params;
typedef struct cth_energy_result {
    double Px, Pr, Pp, power_sum;  /* W: integrals over the x-faces, r-faces, cells */
} cth_energy_result;
int cth_update_energy_profile(cth_fields* fs, cth_grid* gx, cth_grid* gr, const cth_energy_params* prm,
                              const void* E1x, const void* E1r, const void* E1p, void* J1x, void* J1r,
                              void* J1p, void* stream, cth_energy_result* res);

/* The rest of update_energy_profile (emfieldModule.hpp:7792-8105), after
 * cth_update_energy_profile (power_sum = its result's power_sum).
 * flag_mwRef = 1: the Poynting flux out through the upper faces of the outlet
 * row j_out, columns i_out0..i_out1 (mWLoss_at_boundary_rR, :8631-8664; the
 * reference passes gc.j_flc_bl[4][1]-1 and gc.i_flc_bl[4][0..1]); the port
 * current (from H_phi) and voltage (mean r Er times ln(r2/r1)) on column i_ref
 * (int(x_ref/dx + 0.5) + 1 with x_ref = 0) over the feed's Er faces jf0..jf1
 * (gr.j_flr_bl[n_bl-1]); the wave amplitudes a2, b2 for Z0, de-embedded
 * through the feed's S-parameters (S11, S21, S12, S22 as {re, im}) to a1, b1;
 * ratio = Pmw / |a1|^2 and ratio_eff = ratio (power_sum + P_err) / power_sum;
 * then Pabs *= ratio_eff and E1x, E1r, E1p, J1x, J1r, J1p and the optional
 * excitation planes J1x_exc, J1r_exc, J1p_exc (NULL: absent) *= sqrt(ratio_eff)
 * over the whole index space.  flag_mwRef = 0: ratio = Pmw / power_sum and
 * Pabs *= ratio only (:8073-8095; the planes may be NULL).  The caller
 * multiplies its J1r_exc by res->J1r_exc_factor (sqrt(ratio)), as the reference
 * updates pm.J1r_exc.  res holds the reference's reported quantities after its
 * rescaling.  Complex planes: library layout, (re, im) interleaved.  Waits for
 * the stream (the result is read back).  CTH_NONFINITE, with nothing
 * rescaled, when the ratio is not finite. */
typedef struct cth_mw_port_params {
    double dx, dr, rmin, omegam;
    double r1, r2;                     /* coax radii of the feed           */
    double Z0, Pmw;                    /* line impedance, incident power   */
    double S11[2], S21[2], S12[2], S22[2];
    int flag_mwRef;
    int i_ref;
    int j_out, i_out0, i_out1;
    int jf0, jf1;
} cth_mw_port_params;
typedef struct cth_mw_port_result {
    double P_out, P_fwd, P_ref, P_fwd_all, P_ref_all, P_err, power_sum; /* W, after the rescale */
    double ratio, pabs_factor, field_factor, J1r_exc_factor;
    double I_ref[2], V_ref[2], Gamma_p[2], Zp[2], Gamma_all[2], Zall[2];
} cth_mw_port_result;
int cth_mw_port_rescale(cth_fields* fs, const cth_mw_port_params* prm, double power_sum, void* E1x, void* E1r,
                        void* E1p, void* J1x, void* J1r, void* J1p, void* J1x_exc, void* J1r_exc, void* J1p_exc,
                        void* stream, cth_mw_port_result* res);

/* The microwave update of the time loop (src/main.cpp:254-257) on a discharge's
 * device state -----------------------------------------------------------------
 * Every ndiv_mw steps the reference calls EmfieldModule::solve_Microwave and
 * update_energy_profile.  cth_mw_update_run does both on the store fs with the
 * system m (rectangle or block geometry, boundary lists set): assembly from the
 * store's rhoe, nu_m1, Bx, Br and epsr_mw planes (upload epsr_mw, the cells'
 * relative permittivity, before the first run), the solve to tol within maxit
 * iterations, the ghost pass (Er of the store for open east faces), the
 * absorbed power into the store's Pabs and the J planes, the port part with
 * port.Pmw (the store's Pabs rescaled to Pmw; flag_mwRef as given), and the
 * excitation current J1r_exc for the next run multiplied by the root of the
 * ratio.  E3 / J3: the caller's device buffers of 3 complex planes each in m's
 * layout (E1x, E1r, E1p / J1x, J1r, J1p), or NULL for planes the handle
 * allocates (zero) and frees; cth_mw_update_plane: 0-2 E, 3-5 J.  They persist
 * between runs as the reference's fields do.  Returns the solve's
 * status (CTH_NOT_CONVERGED after maxit) or the rescale's (CTH_NONFINITE: not
 * rescaled); the stream is synchronised (the integrals are read back). */
typedef struct cth_mw_update_params {
    cth_mw_params mw;           /* the system; mw.J1r_exc is the initial excitation */
    cth_mw_port_params port;    /* port / reflection / rescale, with Pmw            */
    int ndiv_mw;                /* run every ndiv_mw steps                          */
    int maxit;
    double tol;
    int warm_start;             /* 1: the solve starts from the previous update's
                                   fields scaled to the new excitation (the system
                                   is linear in J1r_exc) when their residual is
                                   <= ||b|| (device-side choice,
                                   cth_mw3_solve_guess_dev); 0: zero */
} cth_mw_update_params;
typedef struct cth_mw_update_result {
    cth_status solve;
    double power_sum;           /* absorbed power before the rescale (W)            */
    double ratio;               /* Pmw / delivered power                            */
    double J1r_exc;             /* excitation current for the next run              */
    int rescale_rc;
} cth_mw_update_result;
int cth_mw_update_create(cth_fields* fs, cth_mw3* m, const cth_mw_update_params* p, double* E3, double* J3,
                         cth_mw_update** out);
void cth_mw_update_destroy(cth_mw_update* u);
int cth_mw_update_due(const cth_mw_update* u, int itime);
double* cth_mw_update_plane(cth_mw_update* u, int which);
int cth_mw_update_run(cth_mw_update* u, cth_grid* gx, cth_grid* gr, void* stream, cth_mw_update_result* res);
/* a trained microwave network (cth_unet of 9 input, 6 output channels, see
 * cth_unet_mw_guess) whose guess starts every solve after the first (NULL: none);
 * the guess is taken when its residual is at most ||b||, else the solve starts
 * from the previous fields (warm_start) or zero.  res->solve.guess reports it. */
int cth_mw_update_set_net(cth_mw_update* u, struct cth_unet* net);
/* the first solve of a handle builds its hierarchy and solve graph: this runs the
 * assembly and the solve alone (E's unknowns written, nothing else: no ghosts,
 * no absorbed power, no rescale), so that the build happens before a timed run */
int cth_mw_update_prepare(cth_mw_update* u, void* stream);
int cth_mw_update_prepared(const cth_mw_update* u);   /* 1 once prepare (or a batch) built it */

/* Two-port feed helpers (host) -------------------------------------------------
 * CmpMat2 (cmpMat2.hpp:8-34): 2x2 complex matrices, complex values as
 * {re, im}.  sParamToABCD / ABCDToSParam (initialModule.hpp:1689-1739) for the
 * reference impedance Z0: CTH_ERR_ARG where the reference throws (|S21| or the
 * denominator below 1e-14).  cth_sparam_setup: the S-parameter set-up of
 * initialModule.hpp:107-192 (polar input in degrees; pre-line of phase
 * phase_pre_deg; stub length h0_stab -> h0_stab + dh_stab in a dielectric of
 * epsr_diele at omegam, applied as a shunt admittance at the stub junction;
 * cable length change dl_cable as a phase factor); S = {S11, S21, S12, S22}. */
typedef struct cth_cmat2 {
    double A[2], B[2], C[2], D[2];
} cth_cmat2;
typedef struct cth_sparam_params {
    double S11_mag, S11_arg_deg, S21_mag, S21_arg_deg, S12_mag, S12_arg_deg, S22_mag, S22_arg_deg;
    double Z0, phase_pre_deg, omegam, epsr_diele, h0_stab, dh_stab, dl_cable;
} cth_sparam_params;
int cth_cmat2_mul(const cth_cmat2* X, const cth_cmat2* Y, cth_cmat2* out);
int cth_cmat2_inv(const cth_cmat2* X, cth_cmat2* out);
int cth_sparam_to_abcd(const double S11[2], const double S21[2], const double S12[2], const double S22[2], double Z0,
                       cth_cmat2* T);
int cth_abcd_to_sparam(const cth_cmat2* T, double Z0, double S11[2], double S21[2], double S12[2], double S22[2]);
int cth_sparam_setup(const cth_sparam_params* p, double S[4][2], double* cable_phase_deg);

/* Learned warm start ---------------------------------------------------------
 * No counterpart in the reference.  A 4-level convolutional U-Net (3x3
 * convolutions, ReLU, 2x2 average pooling, nearest upsampling, skip
 * concatenations; channels 32/64/128/256; 1x1 linear output layer), bfloat16
 * weights and activations with FP32 accumulation on the tensor cores, FP32
 * master parameters and Adam.  Images are NHWC FP32 device arrays of H x W
 * pixels (H, W multiples of 8; cin, cout <= 32 channels; base must be 32).
 * Parameter order (FP32): per convolution, in forward order e0a e0b e1a e1b
 * e2a e2b ba bb d2a d2b d1a d1b d0a d0b, weights [cout][3][3][cin] then bias
 * [cout]; last the output layer [cout][32] and its bias.  The first
 * convolution takes the input zero-padded to 32 channels. */
typedef struct cth_unet cth_unet;
cth_unet* cth_unet_create(int H, int W, int cin, int cout, int base, int device);
void cth_unet_destroy(cth_unet* n);
long long cth_unet_nparams(const cth_unet* n);
long long cth_unet_launch_count(const cth_unet* n);  /* kernels of forward passes and predictions */
/* convolutions on the tcgen05 tensor cores with TMA-fed operands and the
 * accumulator in tensor memory (1, default) or on the warp-level mma.sync
 * kernel (0) */
int cth_unet_set_tensor_cores(cth_unet* n, int tcgen05);
/* passes (0..64, default 0) of a 5-point smoother, (4 v + neighbours) / 8 with
 * edge-replicating neighbours, applied to the predicted change of the first
 * potential correction before cth_unet_predict_dphi forms the guess */
int cth_unet_set_smoothing(cth_unet* n, int passes);
/* synchronises; CTH_ERR_CUDA if a tensor-core convolution's bounded wait gave
 * up since the last check (the output of that call is then not valid) */
int cth_unet_check(cth_unet* n);
/* test of the bounded waits of the tcgen05 convolutions: with stall != 0 the
 * kernel issues no loads, so every wait runs out after `polls` polls (default
 * 2^20), the kernel sets the flag that cth_unet_check reports (once) and frees
 * its tensor memory; nothing is in flight.  stall = 0 restores normal work. */
int cth_unet_set_wait_test(cth_unet* n, int stall, int polls);
/* at most `ctas` CTAs (one per SM) for the persistent tcgen05 convolutions
 * (0, default: every SM), leaving the other SMs to work that runs beside the
 * network, e.g. the ion step beside the warm-start prediction */
int cth_unet_set_grid_limit(cth_unet* n, int ctas);
int cth_unet_set_params(cth_unet* n, const float* host, long long count);  /* resets Adam */
int cth_unet_get_params(const cth_unet* n, float* host, long long count);
int cth_unet_get_grads(const cth_unet* n, float* host, long long count);
int cth_unet_set_loss_weights(cth_unet* n, const float* w_host);          /* cout values */
int cth_unet_forward(cth_unet* n, const float* in, float* out, void* stream);
/* gradients of sum(dout * output) with respect to the parameters, after
 * cth_unet_forward on the same stream */
int cth_unet_backward(cth_unet* n, const float* dout, void* stream);
/* forward, weighted masked MSE against target (mask: one value per pixel,
 * msum its sum), backward and one Adam step (t >= 1); *loss = loss before it */
int cth_unet_train_step(cth_unet* n, const float* in, const float* target, const float* mask, double msum,
                        float lr, int t, void* stream, double* loss);
/* Warm start of the potential predictor-corrector from a field store (grid of
 * at most H x W cells, cell (i, j) -> pixel (j-1, i-1)).  Input channels
 * (cin = 6): log10 rhoe, log10 nu_m, |B| from Bx and Br, a zero channel
 * reserved for the microwave field, "dphi_prev2" and "dphi_prev" (the first
 * corrections of the two previous steps); each normalised with the
 * stats (mean[6], std[6]); output channel 2, de-normalised (output mean[3],
 * std[3]), is the change of the first-iteration correction from "dphi_prev"
 * (a zero output reproduces the previous-step guess).  cth_unet_features writes the
 * input (H x W x 6 FP32, device); cth_unet_predict_dphi runs the network and
 * writes the plane "dphi_guess" read by cth_solve_phi_pc with warm_start = 1. */
int cth_unet_set_stats(cth_unet* n, const float* stats);
int cth_unet_features(cth_unet* n, cth_fields* fs, float* out, void* stream);
int cth_unet_predict_dphi(cth_unet* n, cth_fields* fs, void* stream);
/* The microwave warm start (9 input, 6 output channels).  The system is linear
 * in the port excitation J1r_exc, which the rescale changes between updates, so
 * the network works on fields per unit excitation: input = log10 n_e, log10
 * nu_m1, |B| and the real and imaginary parts of the previous fields E1x, E1r,
 * E1p times escale (E3: three interleaved complex planes of the store's layout)
 * at grid cell (i, j) -> pixel (j-1, i-1), normalised by the stats; output =
 * the normalised change of the six parts per unit excitation.
 * cth_unet_mw_features writes the input (H x W x 9 FP32, device);
 * cth_unet_mw_guess (escale = 1 / jprev) runs the network and writes Eguess =
 * (jnow / jprev) Eprev + jnow x the de-normalised change on the grid cells
 * ((jnow / jprev) Eprev elsewhere), jprev the excitation Eprev was solved with,
 * jnow the next solve's; Eguess distinct from Eprev. */
int cth_unet_mw_features(cth_unet* n, cth_fields* fs, const double* E3, double escale, float* out, void* stream);
int cth_unet_mw_guess(cth_unet* n, cth_fields* fs, const double* Eprev, double jprev, double jnow, double* Eguess,
                      void* stream);

/* Layout helpers (device arrays): copy between the reference's [i][j] layout
 * and the library layout. */
int cth_to_device_layout(cth_grid* g, const double* src_ij, double* dst_dev, void* stream);
int cth_from_device_layout(cth_grid* g, const double* src_dev, double* dst_ij, void* stream);

#ifdef __cplusplus
}
#endif
#endif
