// batch.cu — many independent discharges on one GPU (the batched I-V sweeps of
// bias voltage and microwave power).  Each instance is a complete time loop
// (its own grids, field store and stream); host worker threads advance their
// instances one step at a time, interleaved, so the GPU always holds the
// latency-bound kernels of many instances at once.  Instances share nothing:
// every grid owns its workspace and solve graphs (captured in thread-local
// capture mode), every store its scratch and pinned status slots.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include "fluid.cuh"

extern "C" int cth_batch_steps(cth_batch_item* items, int n, int steps, int nthreads, double* wall_seconds) {
    if (!items || n < 1 || steps < 0 || nthreads < 1) {
        cth::set_error("cth_batch_steps: invalid arguments");
        return CTH_ERR_ARG;
    }
    for (int k = 0; k < n; k++) {
        if (!items[k].fs || !items[k].gx || !items[k].gr || !items[k].params) {
            cth::set_error("cth_batch_steps: incomplete item");
            return CTH_ERR_ARG;
        }
        items[k].rc = 0;
        items[k].steps_done = 0;
        items[k].seconds = 0.0;
        items[k].I_Anode = items[k].Ii_Anode = items[k].Ie_Anode = 0.0;
        items[k].mw_runs = 0;
        items[k].mw_power_sum = items[k].mw_J1r_exc = 0.0;
    }
    std::vector<cudaStream_t> streams(n, nullptr);
    for (int k = 0; k < n; k++) {
        CTH_CUDA(cudaSetDevice(items[k].fs->g->device));
        CTH_CUDA(cudaStreamCreateWithFlags(&streams[k], cudaStreamNonBlocking));
    }
    // the first solve of a microwave handle builds its hierarchy and solve graph:
    // done here, one handle after another on this thread, not in the workers
    for (int k = 0; k < n; k++) {
        cth_mw_update* mw = items[k].mw;
        if (!mw || cth_mw_update_prepared(mw)) continue;
        CTH_CUDA(cudaSetDevice(items[k].fs->g->device));
        const int rc = cth_mw_update_prepare(mw, streams[k]);
        if (rc < 0) return rc;
        CTH_CUDA(cudaStreamSynchronize(streams[k]));
    }
    const int T = std::min(nthreads, n);
    auto worker = [&](int t) {
        std::vector<int> mine;
        for (int k = t; k < n; k += T) mine.push_back(k);
        if (mine.empty()) return;
        cudaSetDevice(items[mine[0]].fs->g->device);
        std::vector<std::chrono::steady_clock::time_point> t0(mine.size(), std::chrono::steady_clock::now());
        for (int s = 0; s < steps; s++) {
            for (size_t q = 0; q < mine.size(); q++) {
                cth_batch_item& it = items[mine[q]];
                if (it.rc < 0) continue;
                cudaSetDevice(it.fs->g->device);
                cth_step_result r;
                const int rc = cth_fluid_step(it.fs, it.gx, it.gr, it.params, streams[mine[q]], &r);
                if (rc < 0) { it.rc = rc; continue; }
                if (rc > it.rc) it.rc = rc;
                it.steps_done++;
                it.I_Anode = r.rhoe.I_Anode;
                it.Ii_Anode = r.rhoe.Ii_Anode;
                it.Ie_Anode = r.rhoe.Ie_Anode;
                if (it.mw && cth_mw_update_due(it.mw, it.params->itime)) {
                    cth_mw_update_result mr;
                    const int mrc = cth_mw_update_run(it.mw, it.gx, it.gr, streams[mine[q]], &mr);
                    if (mrc < 0) { it.rc = mrc; continue; }
                    if (mrc > it.rc) it.rc = mrc;
                    it.mw_runs++;
                    it.mw_power_sum = mr.power_sum;
                    it.mw_J1r_exc = mr.J1r_exc;
                }
            }
        }
        for (size_t q = 0; q < mine.size(); q++) {
            cth_batch_item& it = items[mine[q]];
            cudaSetDevice(it.fs->g->device);
            if (cudaStreamSynchronize(streams[mine[q]]) != cudaSuccess && it.rc >= 0) it.rc = CTH_ERR_CUDA;
            it.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0[q]).count();
        }
    };
    const auto w0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++) pool.emplace_back(worker, t);
    for (auto& th : pool) th.join();
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    if (wall_seconds) *wall_seconds = wall;
    int worst = 0;
    for (int k = 0; k < n; k++) {
        cudaSetDevice(items[k].fs->g->device);
        cudaStreamDestroy(streams[k]);
        if (items[k].rc < 0 && (worst >= 0 || items[k].rc < worst)) worst = items[k].rc;
        else if (worst >= 0 && items[k].rc > worst) worst = items[k].rc;
    }
    if (worst < 0) cth::set_error("cth_batch_steps: an instance failed (see its rc)");
    return worst;
}
