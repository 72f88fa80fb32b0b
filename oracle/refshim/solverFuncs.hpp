/*
 * solverFuncs.hpp — stand-in for the reference's include/solverFuncs.hpp when
 * the reference's own FluidModule / InitialModule are compiled into the
 * checker library oracle/_ref/libref.so.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; nothing in the product uses it).
 *
 * The reference's header pulls in HYPRE, MPI and Eigen, none of which exist
 * on this machine.  The recipe (oracle/Makefile, target _ref) puts this
 * directory before the reference's include directory with `-I-`, so the
 * reference's `#include "solverFuncs.hpp"` (fluidModule.hpp:13) resolves
 * here and every other reference header is used unmodified.
 *
 * The two entry points keep the reference's signatures
 * (solverFuncs.hpp:26-37 and :169-180) and semantics:
 *   - solver_SMG: the limit that HYPRE Struct SMG converges to, i.e. the exact
 *     solution of the box-union system (couplings to cells outside the blocks
 *     dropped), by the oracle's banded elimination (oracle/struct5.c); only
 *     block cells of `solution` are written; the initial content of
 *     `solution` is ignored (SMG starts from zero).  With refshim_mode(1) the
 *     oracle's SMG restatement runs instead, with the caller's maxITR and
 *     error_cnv (relative-residual stopping rule).
 *   - solver_SOR: the oracle's restatement of the reference's lexicographic
 *     point SOR (oracle/struct5.c: orc_sor_solve), starting from `solution`.
 * Each call can be recorded (the assembled aP..aS, b) so that tests compare
 * the reference's assembly with other implementations directly.
 */
#pragma once
#include <vector>

#include "refshim/refshim_state.hpp"


void solver_SMG(std::vector<std::vector<double> > aP, std::vector<std::vector<double> > aE,
                std::vector<std::vector<double> > aW, std::vector<std::vector<double> > aN,
                std::vector<std::vector<double> > aS, std::vector<std::vector<double> > b,
                std::vector<std::vector<int> > i_bl, std::vector<std::vector<int> > j_bl,
                int n_bl, int maxITR, double error_cnv, int flag_msg,
                std::vector<std::vector<double> >& solution);

void solver_SOR(std::vector<std::vector<double> > aP, std::vector<std::vector<double> > aE,
                std::vector<std::vector<double> > aW, std::vector<std::vector<double> > aN,
                std::vector<std::vector<double> > aS, std::vector<std::vector<double> > b,
                std::vector<std::vector<int> > i_bl, std::vector<std::vector<int> > j_bl,
                int n_bl, double alpha_SOR, int maxITR, double error_cnv, int flag_msg,
                std::vector<std::vector<double> >& solution);
