// Drop-in check: a caller written against the reference's solverFuncs.hpp
// interface (vector<vector<double>> arrays, block tables) links
// libcathode_b200.so through include/cathode_solver.hpp.  It assembles a
// variable-coefficient 5-point system on two blocks, calls solver_SMG and
// solver_SOR, and prints the relative residual of each solution (computed
// here on the host, couplings to non-block cells dropped for SMG).
#include <cmath>
#include <cstdio>
#include <vector>

#include "cathode_solver.hpp"

typedef std::vector<std::vector<double> > Arr;

int main() {
    const int ni = 60, nj = 30;
    Arr aP(ni + 2, std::vector<double>(nj + 2, 0.0)), aE = aP, aW = aP, aN = aP, aS = aP, b = aP, x = aP;
    std::vector<std::vector<int> > i_bl = {{1, 40}, {41, 60}}, j_bl = {{1, 30}, {5, 20}};
    const int n_bl = 2;
    auto in_grid = [&](int i, int j) {
        for (int k = 0; k < n_bl; k++)
            if (i >= i_bl[k][0] && i <= i_bl[k][1] && j >= j_bl[k][0] && j <= j_bl[k][1]) return true;
        return false;
    };
    for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++) {
            double c = 1.0 + 0.5 * std::sin(0.3 * i) * std::cos(0.2 * j);
            aE[i][j] = c; aW[i][j] = c; aN[i][j] = 1.5 * c; aS[i][j] = 1.5 * c;
            aP[i][j] = aE[i][j] + aW[i][j] + aN[i][j] + aS[i][j] + 0.01;
            b[i][j] = std::sin(0.1 * i + 0.2 * j);
        }
    solver_SMG(aP, aE, aW, aN, aS, b, i_bl, j_bl, n_bl, 30, 1e-11, 0, x);
    double rr = 0, bb = 0;
    for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++) {
            if (!in_grid(i, j)) continue;
            double ax = aP[i][j] * x[i][j];
            if (in_grid(i + 1, j)) ax -= aE[i][j] * x[i + 1][j];
            if (in_grid(i - 1, j)) ax -= aW[i][j] * x[i - 1][j];
            if (in_grid(i, j + 1)) ax -= aN[i][j] * x[i][j + 1];
            if (in_grid(i, j - 1)) ax -= aS[i][j] * x[i][j - 1];
            rr += (b[i][j] - ax) * (b[i][j] - ax);
            bb += b[i][j] * b[i][j];
        }
    std::printf("smg_relres %.3e\n", std::sqrt(rr / bb));
    Arr y = aP;
    for (auto& row : y) for (auto& v : row) v = 0.0;
    solver_SOR(aP, aE, aW, aN, aS, b, i_bl, j_bl, n_bl, 1.9, 20000, 1e-13, 0, y);
    rr = 0;
    for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++) {
            if (!in_grid(i, j)) continue;
            double ax = aP[i][j] * y[i][j] - aE[i][j] * y[i + 1][j] - aW[i][j] * y[i - 1][j] -
                        aN[i][j] * y[i][j + 1] - aS[i][j] * y[i][j - 1];
            rr += (b[i][j] - ax) * (b[i][j] - ax);
        }
    std::printf("sor_relres %.3e\n", std::sqrt(rr / bb));
    return 0;
}
