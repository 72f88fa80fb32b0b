// step.cu — one time step of the fluid model in the order of the reference's
// time loop (src/main.cpp:170-251), on one stream; every sub-step is the
// device implementation behind its own entry point.
#include <cuda_runtime.h>

#include "fluid.cuh"

extern "C" int cth_fluid_step(cth_fields* fs, cth_grid* gx, cth_grid* gr, cth_step_params* p, void* stream,
                              cth_step_result* res) {
    if (!fs || !gx || !gr || !p || p->ndt_i < 1 || p->ndt_n < 1 || p->ndt_m < 1) {
        cth::set_error("cth_fluid_step: invalid arguments");
        return CTH_ERR_ARG;
    }
    cth_step_result local{};
    cth_step_result* R = res ? res : &local;
    *R = cth_step_result{};
    // planned downloads of the previous step still reading the planes finish first
    int rc0 = copies_wait(fs, (cudaStream_t)stream);
    if (rc0 < 0) return rc0;
    rc0 = plan_upload(fs, (cudaStream_t)stream);
    if (rc0 < 0) return rc0;
    // check_CFL: dt (adaptive) or CFL (fixed dt)
    R->cfl.dt = p->dt;
    R->cfl.CFL = p->CFL;
    R->cfl.masse = p->transport.masse;
    R->cfl.rmin = p->transport.rmin;
    R->cfl.dr = p->transport.dr;
    R->cfl.flag_adp_dt = p->flag_adp_dt;
    int rc = cth_check_cfl(fs, &R->cfl, stream);
    if (rc < 0) return rc;
    p->dt = R->cfl.dt;
    p->CFL = R->cfl.CFL;
    p->gtime += p->dt;
    p->itime += 1;
    p->ion.dt = p->phi.dt = p->rhoe.dt = p->eps.dt = p->neutral.dt = p->dt;
    p->ion.CFL = p->CFL;
    p->ion.ndt_i = p->ndt_i;
    p->neutral.ndt_n = p->ndt_n;
    p->neutral.ndt_m = p->ndt_m;
    int worst = 0;
    // the learned warm start reads rhoe, nu_m, B and the previous corrections,
    // which the ion step does not change: it runs on its own stream, concurrent
    // with the ion step, and joins before the potential sweep
    // a predictor that the guess selection has not taken for kNetPatience predictions runs
    // only every kNetProbe steps (the other steps start from the previous
    // correction), so it costs nothing while it does not help
    constexpr int kNetPatience = 4, kNetProbe = 8;
    const bool wants_net = p->phi.warm_start == 1 || p->phi.warm_start == 3;
    const bool learned = p->net && wants_net && (fs->net_misses < kNetPatience || p->itime % kNetProbe == 0);
    cth_phi_params phi = p->phi;
    if (wants_net && !learned) phi.warm_start = 2;
    cudaStream_t s = (cudaStream_t)stream;
    if (learned) {
        if (!fs->net_stream) {
            // the prediction at the lowest priority, the ion step beside it at the highest
            int lo = 0, hi = 0;
            CTH_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CTH_CUDA(cudaStreamCreateWithPriority(&fs->net_stream, cudaStreamNonBlocking, lo));
            CTH_CUDA(cudaStreamCreateWithPriority(&fs->ion_stream, cudaStreamNonBlocking, hi));
            for (int k = 0; k < 2; k++) {
                CTH_CUDA(cudaEventCreateWithFlags(&fs->net_event[k], cudaEventDisableTiming));
                CTH_CUDA(cudaEventCreateWithFlags(&fs->ion_event[k], cudaEventDisableTiming));
            }
        }
        CTH_CUDA(cudaEventRecord(fs->net_event[0], s));
        CTH_CUDA(cudaStreamWaitEvent(fs->net_stream, fs->net_event[0], 0));
        rc = cth_unet_predict_dphi(p->net, fs, fs->net_stream);
        if (rc < 0) return rc;
        CTH_CUDA(cudaEventRecord(fs->net_event[1], fs->net_stream));
    }
    if (p->itime % p->ndt_i == 0) {
        // beside a prediction the ion step runs on the high-priority stream
        void* ion_s = stream;
        if (learned) {
            CTH_CUDA(cudaEventRecord(fs->ion_event[0], s));
            CTH_CUDA(cudaStreamWaitEvent(fs->ion_stream, fs->ion_event[0], 0));
            ion_s = (void*)fs->ion_stream;
        }
        rc = cth_ion_step(fs, gx, gr, &p->ion, ion_s, &R->ion);
        if (learned) {
            CTH_CUDA(cudaEventRecord(fs->ion_event[1], fs->ion_stream));
            CTH_CUDA(cudaStreamWaitEvent(s, fs->ion_event[1], 0));
        }
        if (rc < 0) return rc;
        R->ran_ion = 1;
        if (R->ion.solver_rc > worst) worst = R->ion.solver_rc;
    }
    rc = plan_flush(fs, 1, s);
    if (rc < 0) return rc;
    if (learned) CTH_CUDA(cudaStreamWaitEvent(s, fs->net_event[1], 0));
    rc = cth_solve_phi_pc(fs, &phi, stream, &R->phi);
    if (learned && rc >= 0) {
        fs->net_runs++;
        if (R->phi.first.guess == 1) { fs->net_wins++; fs->net_misses = 0; }
        else fs->net_misses++;
    }
    R->net_ran = learned ? 1 : 0;
    if (rc < 0) return rc;
    if (R->phi.solver_rc > worst) worst = R->phi.solver_rc;
    rc = plan_flush(fs, 2, s);
    if (rc < 0) return rc;
    rc = cth_solve_rhoe_pc(fs, &p->rhoe, stream, &R->rhoe);
    if (rc < 0) return rc;
    if (R->rhoe.solver_rc > worst) worst = R->rhoe.solver_rc;
    rc = plan_flush(fs, 3, s);
    if (rc < 0) return rc;
    rc = upload_wait(fs, 1, s);
    if (rc < 0) return rc;
    rc = cth_solve_Te_pc(fs, &p->eps, stream, &R->eps);
    if (rc < 0) return rc;
    if (R->eps.solver_rc > worst) worst = R->eps.solver_rc;
    rc = plan_flush(fs, 4, s);
    if (rc < 0) return rc;
    rc = upload_wait(fs, 2, s);
    if (rc < 0) return rc;
    p->neutral.do_rhon = (p->itime % p->ndt_n == 0);
    p->neutral.do_rhom = (p->itime % p->ndt_m == 0);
    if (p->neutral.do_rhon || p->neutral.do_rhom) {
        rc = cth_update_neutrals(fs, &p->neutral, stream, &R->neutral);
        if (rc < 0) return rc;
        if (R->neutral.solver_rc > worst) worst = R->neutral.solver_rc;
    }
    R->ran_rhon = p->neutral.do_rhon;
    R->ran_rhom = p->neutral.do_rhom;
    rc = plan_flush(fs, 5, s);
    if (rc < 0) return rc;
    rc = cth_update_transport_coef(fs, &p->transport, stream);
    if (rc < 0) return rc;
    rc = plan_flush(fs, 0, s);
    if (rc < 0) return rc;
    R->solver_rc = worst;
    return CTH_OK;
}
