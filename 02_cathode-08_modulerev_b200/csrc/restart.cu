// restart.cu — restart files of the reference's format for the device-resident state.
//
// Writer: the restart<nOut>.csv that OutputModule::output writes
// (outputModule.hpp:429-470): one line per index (i, j) of the ghost-padded
// (ni+2) x (nj+2) space, i outer, with i, j, x, r and 49 fields, then a zero
// column; every real printed in scientific notation with max_digits10 (17)
// digits after the point, values below 1e-100 in magnitude as 0 (truncate,
// miniFuncs.hpp:99-107), Te and Te_old in eV.  The call queues one
// device-to-host copy per field on the caller's stream into pinned staging
// (so later work on that stream cannot change what is written) and returns;
// a host thread waits for the copies, formats the lines on several threads and
// writes the file.  cth_restart_wait joins it.
//
// Reader: InputModule::input_restart_data (inputModule.hpp:667-1157): columns
// by header name, the 39 registered variables (the wall fluxes are written but
// not read back), Te converted from eV; the index range, duplicate cells,
// coordinates (1e-12 absolute + 1e-10 relative) and missing cells are checked
// -- where the reference aborts, this returns CTH_ERR_ARG with the line.  Then,
// on the device: rhoe masked to the fluid cells, Ex / Er recomputed from phi on
// the interior x- / r-face blocks, the wall ghosts of phi (left, right, lower,
// upper, open, the reference's order), Ex / Er on the wall faces from them and
// Er = 0 on the axis (inputModule.hpp:1003-1118).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fluid.cuh"

namespace cth {

// the 49 field columns of the restart file, in the writer's order (outputModule.hpp:436)
static const char* const kCols[] = {
    "rhoi", "rhoi_old", "Uix", "Uix_old", "Uir", "Uir_old", "Uip", "Uip_old", "rhoe", "rhoe_old", "rhoUex",
    "rhoUex_old", "rhoUer", "rhoUer_old", "Te", "Te_old", "Gx", "Gx_old", "Gr", "Gr_old", "phi", "phi_old", "rhom",
    "rhom_old", "rhoUmx", "rhoUmr", "rate_ionize", "scx", "scr", "nUex", "nUex_old", "nUer", "nUer_old", "rhon",
    "rhon_old", "rhoUnx", "rhoUnr", "rhoeps", "rhoeps_old", "rhoUix_wall", "rhoUir_wall", "rhoUex_wall",
    "rhoUer_wall", "rhoUmx_wall", "rhoUmr_wall", "rhoUnx_wall", "rhoUnr_wall", "Gx_wall", "Gr_wall"};
static constexpr int kNCols = sizeof(kCols) / sizeof(kCols[0]);
static constexpr int kNRead = 39;  // the first 39 columns are the reader's registry (inputModule.hpp:755-812)

static bool is_temperature(const char* c) { return !std::strcmp(c, "Te") || !std::strcmp(c, "Te_old"); }

struct RestartWriter {
    double* stage = nullptr;  // pinned, kNCols planes of the device layout
    size_t stage_planes = 0;
    cudaEvent_t copied = nullptr;
    std::thread thread;
    int status = CTH_OK;
    std::string error;
};

void restart_release(cth_fields* fs) {
    if (!fs->restart) return;
    RestartWriter* w = fs->restart;
    if (w->thread.joinable()) w->thread.join();
    if (w->stage) cudaFreeHost(w->stage);
    if (w->copied) cudaEventDestroy(w->copied);
    delete w;
    fs->restart = nullptr;
}

static inline double truncate_small(double c) { return std::fabs(c) < 1e-100 ? 0.0 : c; }

// format rows i in [i0, i1) of the file into out
static void format_rows(const double* stage, size_t plane, int ld, int nj, int i0, int i1, const double* x,
                        const double* r, std::string* out) {
    char buf[64];
    out->clear();
    out->reserve((size_t)(i1 - i0) * (nj + 2) * (kNCols + 3) * 25);
    for (int i = i0; i < i1; i++) {
        for (int j = 0; j < nj + 2; j++) {
            int n = std::snprintf(buf, sizeof buf, "%d,%d,%.17e,%.17e", i, j, x[i], r[j]);
            out->append(buf, n);
            const size_t p = (size_t)j * ld + i;
            for (int c = 0; c < kNCols; c++) {
                double v = truncate_small(stage[c * plane + p]);
                if (is_temperature(kCols[c])) v = v * kBoltz / kE0f;   // K -> eV as written (outputModule.hpp:448)
                n = std::snprintf(buf, sizeof buf, ",%.17e", v);
                out->append(buf, n);
            }
            out->append(",0.00000000000000000e+00\n");
        }
    }
}

static void write_file(RestartWriter* w, std::string path, int ni, int nj, int ld, size_t plane, std::vector<double> x,
                       std::vector<double> r) {
    if (cudaEventSynchronize(w->copied) != cudaSuccess) {
        w->status = CTH_ERR_CUDA;
        w->error = "cth_restart_write: device-to-host copies failed";
        return;
    }
    const int T = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
    const int rows = ni + 2;
    std::vector<std::string> parts(T);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++) {
        const int i0 = (int)((long long)rows * t / T), i1 = (int)((long long)rows * (t + 1) / T);
        pool.emplace_back(format_rows, w->stage, plane, ld, nj, i0, i1, x.data(), r.data(), &parts[t]);
    }
    for (auto& th : pool) th.join();
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        w->status = CTH_ERR_ARG;
        w->error = "cth_restart_write: cannot open " + path + ": " + std::strerror(errno);
        return;
    }
    std::string head = "i,j,x,r";
    for (int c = 0; c < kNCols; c++) head += std::string(",") + kCols[c];
    head += ",zero\n";
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    for (auto& s : parts) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        w->status = CTH_ERR_ARG;
        w->error = "cth_restart_write: writing " + path + " failed";
    }
}

// ------------------------------------------------------------------ reader kernels
struct RestartFix {
    double *phi, *Ex, *Er, *rhoe;
    const unsigned char *cells, *xfaces, *rfaces, *flags;
    double dx, dr, V_bias;
    int ni, nj, ld;
};

#define RFL(ii, jj) flag_at(A.flags, (ii), (jj), A.ni, A.nj, A.ld)

// rhoe on the fluid cells only; E from phi on the interior face blocks (inputModule.hpp:1003-1018, :1060-1068)
__global__ void k_restart_interior(RestartFix A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const size_t p = (size_t)j * A.ld + i;
    A.rhoe[p] = A.rhoe[p] * (A.cells[p] ? 1.0 : 0.0);
    if (A.xfaces[p] && i >= 1) A.Ex[p] = -(A.phi[p] - A.phi[p - 1]) / A.dx;
    if (A.rfaces[p] && j >= 1) A.Er[p] = -(A.phi[p] - A.phi[p - A.ld]) / A.dr;
}

// wall ghosts of phi, the last writer of the reference's loop order winning (left z0 z1 z2 z4, right z3 z5,
// lower x0 x2, upper x1 x4, open x5: inputModule.hpp:1020-1118)
__global__ void k_restart_ghosts(RestartFix A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    if (RFL(i, j)) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    double v = A.phi[p];
    unsigned f = RFL(i + 1, j);
    if (f && !(f & F_BLX)) v = -A.phi[p + 1];
    f = RFL(i - 1, j);
    if (f && !(f & F_BRX)) v = (f & F_BRX_BIAS) ? 2.0 * A.V_bias - A.phi[p - 1] : -A.phi[p - 1];
    f = RFL(i, j + 1);
    if (f && !(f & F_BLR_WALL)) v = -A.phi[p + ld];
    f = RFL(i, j - 1);
    if (f && !(f & F_BRR_WALL)) v = -A.phi[p - ld];
    if (f && !(f & F_BRR_OPEN)) v = A.phi[p - ld];
    A.phi[p] = v;
}

// E on the wall faces; Er = 0 on the axis (x6).  Each wall face takes the ghost value of its own
// segment, as the reference computes E right after that segment's ghost: at a concave corner a
// later segment overwrites the shared ghost cell, but not the face E already computed (e.g. the
// z1 face at the x0 corner, inputModule.hpp:1030-1035 then :1070-1075)
__global__ void k_restart_walls(RestartFix A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > A.ni + 1) return;
    const unsigned fc = RFL(i, j);
    if (!fc) return;
    const int ld = A.ld;
    const size_t p = (size_t)j * ld + i;
    const double ph = A.phi[p];
    if (!(fc & F_BLX)) {
        const double g = -ph;
        A.Ex[p] = -(ph - g) / A.dx;
    }
    if (!(fc & F_BRX)) {
        const double g = (fc & F_BRX_BIAS) ? 2.0 * A.V_bias - ph : -ph;
        A.Ex[p + 1] = -(g - ph) / A.dx;
    }
    if (!(fc & F_BLR_WALL)) {
        const double g = -ph;
        A.Er[p] = -(ph - g) / A.dr;
    }
    if (!(fc & F_BLR_CEN)) A.Er[p] = 0.0;
    if (!(fc & F_BRR_WALL)) {
        const double g = -ph;
        A.Er[p + ld] = -(g - ph) / A.dr;
    }
    if (!(fc & F_BRR_OPEN)) {
        const double g = ph;
        A.Er[p + ld] = -(g - ph) / A.dr;
    }
}

#undef RFL

static std::vector<std::string> split_csv(const char* b, const char* e) {
    std::vector<std::string> out;
    const char* s = b;
    for (const char* q = b; q <= e; q++) {
        if (q == e || *q == ',') {
            out.emplace_back(s, q);
            s = q + 1;
        }
    }
    return out;
}

static std::string trim(const std::string& s) {
    const char* ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return "";
    return s.substr(a, s.find_last_not_of(ws) - a + 1);
}

static bool coordinate_mismatch(double a, double b) {
    const double diff = std::fabs(a - b);
    const double scale = std::max({1.0, std::fabs(a), std::fabs(b)});
    return diff > 1.0e-12 + 1.0e-10 * scale;
}

}  // namespace cth

using namespace cth;

extern "C" int cth_restart_write(cth_fields* fs, const char* path, const double* x, const double* r, void* stream) {
    if (!fs || !path || !x || !r) {
        set_error("cth_restart_write: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    CTH_CUDA(cudaSetDevice(g->device));
    if (!fs->restart) fs->restart = new RestartWriter();
    RestartWriter* w = fs->restart;
    if (w->thread.joinable()) w->thread.join();   // the staging of the previous write is reused
    if (!w->stage) {
        CTH_CUDA(cudaMallocHost(&w->stage, kNCols * g->plane * sizeof(double)));
        CTH_CUDA(cudaEventCreateWithFlags(&w->copied, cudaEventDisableTiming));
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int c = 0; c < kNCols; c++) {
        double* d = field_ptr(fs, kCols[c]);
        if (!d) {
            set_error("field allocation failed");
            return CTH_ERR_ALLOC;
        }
        CTH_CUDA(cudaMemcpyAsync(w->stage + c * g->plane, d, g->plane * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CTH_CUDA(cudaEventRecord(w->copied, s));
    w->status = CTH_OK;
    w->error.clear();
    w->thread = std::thread(write_file, w, std::string(path), g->ni, g->nj, g->ld, g->plane,
                            std::vector<double>(x, x + g->ni + 2), std::vector<double>(r, r + g->nj + 2));
    return CTH_OK;
}

extern "C" int cth_restart_wait(cth_fields* fs) {
    if (!fs) {
        set_error("cth_restart_wait: invalid arguments");
        return CTH_ERR_ARG;
    }
    if (!fs->restart) return CTH_OK;
    RestartWriter* w = fs->restart;
    if (w->thread.joinable()) w->thread.join();
    if (w->status != CTH_OK) set_error(w->error);
    const int st = w->status;
    w->status = CTH_OK;
    return st;
}

extern "C" int cth_restart_read(cth_fields* fs, cth_grid* gx, cth_grid* gr, const char* path, const double* x,
                                const double* r, const cth_restart_params* prm, void* stream,
                                cth_restart_info* info) {
    if (!fs || !gx || !gr || !path || !x || !r || !prm) {
        set_error("cth_restart_read: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_grid* g = fs->g;
    if (!fs->flags) {
        set_error("cth_restart_read: boundary flags not uploaded");
        return CTH_ERR_ARG;
    }
    if (gx->ni != g->ni || gx->nj != g->nj || gr->ni != g->ni || gr->nj != g->nj || gx->ld != g->ld ||
        gr->ld != g->ld) {
        set_error("cth_restart_read: face grids of another shape");
        return CTH_ERR_ARG;
    }
    const int ni = g->ni, nj = g->nj, ld = g->ld;
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        set_error(std::string("cth_restart_read: cannot open ") + path);
        return CTH_ERR_ARG;
    }
    std::string text;
    {
        char buf[1 << 16];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
        std::fclose(f);
    }
    // lines
    std::vector<std::pair<size_t, size_t>> lines;
    for (size_t a = 0; a < text.size();) {
        size_t b = text.find('\n', a);
        if (b == std::string::npos) b = text.size();
        lines.emplace_back(a, b);
        a = b + 1;
    }
    if (lines.empty()) {
        set_error("cth_restart_read: empty file");
        return CTH_ERR_ARG;
    }
    std::vector<std::string> header = split_csv(text.data() + lines[0].first, text.data() + lines[0].second);
    std::unordered_map<std::string, int> col;
    for (size_t k = 0; k < header.size(); k++) col[trim(header[k])] = (int)k;
    for (const char* need : {"i", "j", "x", "r"})
        if (!col.count(need)) {
            set_error(std::string("cth_restart_read: required column is missing: ") + need);
            return CTH_ERR_ARG;
        }
    int cvar[kNRead];
    int nread = 0;
    for (int c = 0; c < kNRead; c++) {
        auto it = col.find(kCols[c]);
        cvar[c] = it == col.end() ? -1 : it->second;
        nread += cvar[c] >= 0;
    }
    int unknown = 0;
    for (auto& h : header) {
        const std::string t = trim(h);
        bool known = t == "i" || t == "j" || t == "x" || t == "r" || t == "zero";
        for (int c = 0; c < kNCols && !known; c++) known = t == kCols[c];
        unknown += !known;
    }
    const int ci = col["i"], cj = col["j"], cx = col["x"], cr = col["r"];
    // parse the rows on several threads into [i][j] host planes of the registered variables
    const size_t nij = (size_t)(ni + 2) * (nj + 2);
    std::vector<double> host((size_t)kNRead * nij, 0.0);
    const int T = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
    std::vector<std::string> errs(T);
    std::vector<std::vector<std::pair<size_t, size_t>>> seen(T);   // (cell, line) per thread
    std::vector<std::thread> pool;
    const size_t nl = lines.size() - 1;
    for (int t = 0; t < T; t++) {
        pool.emplace_back([&, t]() {
            const size_t a = 1 + nl * t / T, b = 1 + nl * (t + 1) / T;
            for (size_t L = a; L < b && errs[t].empty(); L++) {
                const char* s = text.data() + lines[L].first;
                const char* e = text.data() + lines[L].second;
                if (e > s && e[-1] == '\r') e--;
                if (e == s) continue;
                std::vector<const char*> fld;
                fld.push_back(s);
                for (const char* q = s; q < e; q++)
                    if (*q == ',') fld.push_back(q + 1);
                const int nf = (int)fld.size();
                auto num = [&](int k, double* v) -> bool {
                    if (k >= nf) return false;
                    char* end = nullptr;
                    *v = std::strtod(fld[k], &end);
                    return end != fld[k];
                };
                const std::string where = " at line " + std::to_string(L + 1);
                double vi, vj, vx, vr;
                if (!num(ci, &vi) || !num(cj, &vj) || !num(cx, &vx) || !num(cr, &vr)) {
                    errs[t] = "malformed row" + where;
                    break;
                }
                const int i = (int)vi, j = (int)vj;
                if (i < 0 || i > ni + 1 || j < 0 || j > nj + 1) {
                    errs[t] = "index out of range" + where;
                    break;
                }
                const size_t q = (size_t)i * (nj + 2) + j;
                seen[t].emplace_back(q, L + 1);
                if (coordinate_mismatch(x[i], vx) || coordinate_mismatch(r[j], vr)) {
                    errs[t] = "grid coordinate is inconsistent" + where;
                    break;
                }
                for (int c = 0; c < kNRead; c++) {
                    if (cvar[c] < 0) continue;
                    double v;
                    if (!num(cvar[c], &v)) {
                        errs[t] = std::string("failed to convert column ") + kCols[c] + where;
                        break;
                    }
                    if (is_temperature(kCols[c])) v = v * kE0f / kBoltz;   // eV -> K (inputModule.hpp:776-777)
                    host[(size_t)c * nij + q] = v;
                }
            }
        });
    }
    for (auto& th : pool) th.join();
    for (auto& e : errs)
        if (!e.empty()) {
            set_error("cth_restart_read: " + e);
            return CTH_ERR_ARG;
        }
    std::vector<unsigned char> found(nij, 0);
    for (auto& v : seen)
        for (auto& ql : v) {
            if (found[ql.first]) {
                set_error("cth_restart_read: duplicated cell at line " + std::to_string(ql.second));
                return CTH_ERR_ARG;
            }
            found[ql.first] = 1;
        }
    for (size_t q = 0; q < nij; q++)
        if (!found[q]) {
            set_error("cth_restart_read: missing cell i = " + std::to_string(q / (nj + 2)) +
                      ", j = " + std::to_string(q % (nj + 2)));
            return CTH_ERR_ARG;
        }
    // upload ([i][j] -> device layout) the variables present, then the reader's post-processing
    CTH_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<double> lay(g->plane, 0.0);
    for (int c = 0; c < kNRead; c++) {
        if (cvar[c] < 0) continue;
        double* d = field_ptr(fs, kCols[c]);
        if (!d) {
            set_error("field allocation failed");
            return CTH_ERR_ALLOC;
        }
        for (int i = 0; i < ni + 2; i++)
            for (int j = 0; j < nj + 2; j++) lay[(size_t)j * ld + i] = host[(size_t)c * nij + (size_t)i * (nj + 2) + j];
        CTH_CUDA(cudaMemcpyAsync(d, lay.data(), g->plane * sizeof(double), cudaMemcpyHostToDevice, s));
        CTH_CUDA(cudaStreamSynchronize(s));
    }
    RestartFix A{};
    A.phi = field_ptr(fs, "phi");
    A.Ex = field_ptr(fs, "Ex");
    A.Er = field_ptr(fs, "Er");
    A.rhoe = field_ptr(fs, "rhoe");
    if (!A.phi || !A.Ex || !A.Er || !A.rhoe) {
        set_error("field allocation failed");
        return CTH_ERR_ALLOC;
    }
    A.cells = g->mask_full;
    A.xfaces = gx->mask_full;
    A.rfaces = gr->mask_full;
    A.flags = fs->flags;
    A.dx = prm->dx;
    A.dr = prm->dr;
    A.V_bias = prm->V_bias;
    A.ni = ni;
    A.nj = nj;
    A.ld = ld;
    dim3 blk(128), grd((ni + 2 + 127) / 128, nj + 2);
    k_restart_interior<<<grd, blk, 0, s>>>(A);
    k_restart_ghosts<<<grd, blk, 0, s>>>(A);
    k_restart_walls<<<grd, blk, 0, s>>>(A);
    g->launches += 3;
    CTH_CUDA(cudaGetLastError());
    CTH_CUDA(cudaStreamSynchronize(s));
    if (info) {
        info->rows = (int)nij;
        info->variables_read = nread;
        info->unknown_columns = unknown;
    }
    return CTH_OK;
}
