// cathode_solver.hpp — header-only C++ drop-in for the reference's solver entry points.
//
// Include this header instead of include/solverFuncs.hpp and link
// libcathode_b200.so: the reference's call sites in fluidModule.hpp
// (solver_SMG at :396, :871, :1271, :1586, :2837, :3677, :4653, :5131, :5576 and
// solver_SOR at :391, :866, :1267, :1581, :2832, :3672, :4649, :5129, :5574)
// compile unchanged.  Arguments keep the reference's meaning
// (include/solverFuncs.hpp:26-37 and :169-180); the coefficient arrays are taken
// by const reference instead of by value, which is call-compatible.
//
// Semantics kept: zero initial guess and relative-residual stopping rule for
// solver_SMG, the reference SOR update/stopping rule for solver_SOR, only block
// cells of `solution` written, non-convergence silent (flag_msg == 1 prints
// the iteration count and final residual).  CUDA or argument failures throw
// std::runtime_error (the reference has no error path).
#pragma once

#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "cathode_b200.h"

namespace cathode_b200 {

// arithmetic of solver_SMG replacements: CTH_PREC_MIXED (FP32 multigrid with
// FP64 defect correction, default) or CTH_PREC_FP64
inline int& precision() {
    static int p = CTH_PREC_MIXED;
    return p;
}

inline int& device() {
    static int d = 0;
    return d;
}

// counts over the solver_SMG / solver_SOR calls of this process (the reference
// reports nothing; a caller reads these to see whether every solve met its
// tolerance within maxITR)
struct SolveStats {
    long calls = 0;
    long not_converged = 0;     // CTH_NOT_CONVERGED: maxITR reached above the tolerance
    int last_iterations = 0;
    double last_residual = 0.0;
    double worst_residual = 0.0;  // largest final relative residual of a non-converged call
};
inline SolveStats& stats() {
    static SolveStats s;
    return s;
}
inline void record(int rc, const cth_status& st) {
    SolveStats& s = stats();
    s.calls++;
    s.last_iterations = st.iterations;
    s.last_residual = st.residual;
    if (rc == CTH_NOT_CONVERGED) {
        s.not_converged++;
        if (st.residual > s.worst_residual) s.worst_residual = st.residual;
    }
}

typedef std::tuple<int, int, std::vector<int>, std::vector<int>> GridKey;

// one cth_grid per (shape, block table): the HYPRE grid/stencil/solver set-up
// that solver_SMG repeats on every call is done once here
inline cth_grid* grid_for(int ni, int nj, const std::vector<std::vector<int> >& i_bl,
                          const std::vector<std::vector<int> >& j_bl, int n_bl) {
    static std::map<GridKey, cth_grid*> grids;
    static std::mutex mu;
    std::vector<int> ib, jb;
    for (int b = 0; b < n_bl; b++) {
        ib.push_back(i_bl[b][0]);
        ib.push_back(i_bl[b][1]);
        jb.push_back(j_bl[b][0]);
        jb.push_back(j_bl[b][1]);
    }
    GridKey key(ni, nj, ib, jb);
    std::lock_guard<std::mutex> lk(mu);
    auto it = grids.find(key);
    if (it != grids.end()) return it->second;
    cth_grid* g = nullptr;
    int rc = cth_grid_create(ni, nj, ib.data(), jb.data(), n_bl, device(), &g);
    if (rc != CTH_OK) throw std::runtime_error(std::string("cth_grid_create: ") + cth_last_error());
    grids[key] = g;
    return g;
}

// vector<vector<double>> [i][j] -> contiguous [i*(nj+2)+j]
inline void flatten(const std::vector<std::vector<double> >& a, std::vector<double>& out) {
    const size_t ni2 = a.size(), nj2 = a.empty() ? 0 : a[0].size();
    out.resize(ni2 * nj2);
    for (size_t i = 0; i < ni2; i++)
        for (size_t j = 0; j < nj2; j++) out[i * nj2 + j] = a[i][j];
}

inline void unflatten_blocks(const std::vector<double>& flat, const std::vector<std::vector<int> >& i_bl,
                             const std::vector<std::vector<int> >& j_bl, int n_bl,
                             std::vector<std::vector<double> >& solution) {
    const size_t nj2 = solution[0].size();
    for (int b = 0; b < n_bl; b++)
        for (int i = i_bl[b][0]; i <= i_bl[b][1]; i++)
            for (int j = j_bl[b][0]; j <= j_bl[b][1]; j++) solution[i][j] = flat[(size_t)i * nj2 + j];
}

}  // namespace cathode_b200

// solver_SMG (include/solverFuncs.hpp:26-163) on the GPU
inline void solver_SMG(const std::vector<std::vector<double> >& aP, const std::vector<std::vector<double> >& aE,
                       const std::vector<std::vector<double> >& aW, const std::vector<std::vector<double> >& aN,
                       const std::vector<std::vector<double> >& aS, const std::vector<std::vector<double> >& b,
                       const std::vector<std::vector<int> >& i_bl, const std::vector<std::vector<int> >& j_bl,
                       int n_bl, int maxITR, double error_cnv, int flag_msg,
                       std::vector<std::vector<double> >& solution) {
    using namespace cathode_b200;
    const int ni = (int)solution.size() - 2, nj = (int)solution[0].size() - 2;
    cth_grid* g = grid_for(ni, nj, i_bl, j_bl, n_bl);
    std::vector<double> f[7];
    flatten(aP, f[0]); flatten(aE, f[1]); flatten(aW, f[2]); flatten(aN, f[3]); flatten(aS, f[4]);
    flatten(b, f[5]); flatten(solution, f[6]);
    cth_status st;
    int rc = cth_smg_solve(g, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data(),
                           maxITR, error_cnv, precision(), f[6].data(), &st);
    if (rc < 0) throw std::runtime_error(std::string("cth_smg_solve: ") + cth_last_error());
    record(rc, st);
    unflatten_blocks(f[6], i_bl, j_bl, n_bl, solution);
    if (flag_msg == 1) {
        std::printf("Number of Iterations: %d\n", st.iterations);
        std::printf("Final Relative Residual Norm: %g\n", st.residual);
    }
}

// solver_SOR (include/solverFuncs.hpp:169-217) on the GPU (red-black order)
inline void solver_SOR(const std::vector<std::vector<double> >& aP, const std::vector<std::vector<double> >& aE,
                       const std::vector<std::vector<double> >& aW, const std::vector<std::vector<double> >& aN,
                       const std::vector<std::vector<double> >& aS, const std::vector<std::vector<double> >& b,
                       const std::vector<std::vector<int> >& i_bl, const std::vector<std::vector<int> >& j_bl,
                       int n_bl, double alpha_SOR, int maxITR, double error_cnv, int flag_msg,
                       std::vector<std::vector<double> >& solution) {
    using namespace cathode_b200;
    const int ni = (int)solution.size() - 2, nj = (int)solution[0].size() - 2;
    cth_grid* g = grid_for(ni, nj, i_bl, j_bl, n_bl);
    std::vector<double> f[7];
    flatten(aP, f[0]); flatten(aE, f[1]); flatten(aW, f[2]); flatten(aN, f[3]); flatten(aS, f[4]);
    flatten(b, f[5]); flatten(solution, f[6]);
    cth_status st;
    int rc = cth_sor_solve(g, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data(),
                           alpha_SOR, maxITR, error_cnv, f[6].data(), &st);
    if (rc < 0) throw std::runtime_error(std::string("cth_sor_solve: ") + cth_last_error());
    record(rc, st);
    unflatten_blocks(f[6], i_bl, j_bl, n_bl, solution);
    if (flag_msg == 1) std::printf("ncount = %d error_max = %g\n", st.iterations, st.residual);
}
