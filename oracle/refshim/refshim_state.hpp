/*
 * refshim_state.hpp — state of the checker's solver stand-ins (recorded systems,
 * solver mode, failure count), shared by refshim/solverFuncs.hpp (exact solves)
 * and refshim_dropin/solverFuncs.hpp (the product's GPU drop-in).
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#include <vector>

namespace refshim {
/* One recorded system: the six (ni+2) x (nj+2) planes flattened [i][j]. */
struct System {
    int rows = 0, cols = 0;
    std::vector<double> a[6];   /* aP, aE, aW, aN, aS, b */
    std::vector<int> ib, jb;    /* block table, 2 ints per block */
    int n_bl = 0;
};
int& mode();                    /* 0 = exact (default), 1 = SMG restatement */
bool& capturing();
std::vector<System>& captured();
int& calls();
int& failures();                /* zero pivots / solver errors seen */
}  // namespace refshim
