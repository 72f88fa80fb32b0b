// fluid.cuh — shared pieces of the FluidModule kernels: the field store, the
// side-flag bits of the fluid blocks, physical constants and the uniform-step
// table lookups of miniFuncs.hpp:35-91.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>

#include "grid.h"

#define CTH_FS_NSCAL 64
#define CTH_FS_NPART_PER_BLOCK 16

struct cth_fields {
    cth_grid* g = nullptr;
    std::map<std::string, double*> planes;
    unsigned char* flags = nullptr;  // device layout
    std::map<std::string, std::pair<double*, int>> tables;
    double* scal = nullptr;          // device scalars (reductions), CTH_FS_NSCAL doubles
    double* h_scal = nullptr;        // pinned host copy
    double* part = nullptr;          // per-block partials, CTH_FS_NPART_PER_BLOCK per block
    int npart = 0;
};

namespace cth {

// side flags of a cell (1 = ordinary interior face on that side)
enum { F_BLX = 1, F_BRX = 2, F_BLR_WALL = 4, F_BLR_CEN = 8, F_BRR_WALL = 16, F_BRR_OPEN = 32, F_BRX_BIAS = 64 };

// flag of cell (i, j); 0 outside the (ni+2) x (nj+2) index space
__device__ __forceinline__ unsigned flag_at(const unsigned char* __restrict__ f, int i, int j, int ni, int nj,
                                            int ld) {
    return (i >= 0 && i <= ni + 1 && j >= 0 && j <= nj + 1) ? f[(size_t)j * ld + i] : 0u;
}

constexpr double kBoltz = 1.380649e-23;    // constants.hpp:5
constexpr double kE0f = 1.60217662e-19;    // constants.hpp:6
constexpr double kEps0f = 8.8541878128e-12;// constants.hpp:7

// uniform-step table lookups of miniFuncs.hpp:35-91
__device__ __forceinline__ double d_func_Te(const double* __restrict__ v, int n, double Te, double dTe) {
    const int iL = (int)(Te / dTe);
    const int iR = iL + 1;
    const double Te_L = iL * dTe;
    if (iR < n - 1) return (v[iR] - v[iL]) / (dTe + 1e-100) * (Te - Te_L) + v[iL];
    return v[n - 1];
}

__device__ __forceinline__ double d_func_dTe(const double* __restrict__ v, int n, double Te, double dTe) {
    int iL = (int)(Te / dTe);
    int iR = iL + 1;
    if (iR >= n - 1) {
        iL = n - 2;
        iR = n - 1;
    }
    return (v[iR] - v[iL]) / (iR * dTe - iL * dTe + 1e-100);
}

__device__ __forceinline__ double d_func_Ei(const double* __restrict__ v, int n, double Ei, double dEi,
                                            double massi) {
    const int iL = (int)(Ei / dEi);
    const int iR = iL + 1;
    const double Ei_L = iL * dEi;
    if (iR < n - 1) return (v[iR] - v[iL]) / (dEi + 1e-100) * (Ei - Ei_L) + v[iL];
    const double imax = n - 1;
    const double v_max = sqrt(imax * dEi / massi);
    const double v_tmp = sqrt(Ei / massi);
    return v[n - 1] / v_max * v_tmp;
}

struct Tab {
    const double* v;
    int n;
};

// named device planes of the store (created zeroed on first use), and tables
double* field_ptr(cth_fields* fs, const std::string& name);
Tab table(cth_fields* fs, const char* name, bool* ok);

}  // namespace cth
