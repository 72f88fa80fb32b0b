/*
 * solverFuncs.hpp — the second stand-in for the reference's include/solverFuncs.hpp:
 * the product's header-only drop-in include/cathode_solver.hpp, so that the
 * reference's unmodified fluidModule.hpp calls solver_SMG / solver_SOR on the GPU
 * through libcathode_b200.so (oracle/Makefile, target oracle/_ref/libref_dropin.so).
 *
 * TEST INFRASTRUCTURE ONLY: it checks that the drop-in compiles against the
 * reference's own call sites and gives the reference's results.
 */
#pragma once
#include "refshim/refshim_state.hpp"
#include "cathode_solver.hpp"
