// Engine interface shared by the passes path and the fused path.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "../../include/jst_gpu.h"
#include "jst_internal.h"

namespace jst {

extern const double RK_ALPHA[5];

// State common to both engines, owned by the handle.
struct SolverCore {
    jst_opts opts{};
    int n_rings = 0, n_theta = 0, ni = 0, nj = 0, H = 3;
    PhysConst c{};
    int local_dt = 0;
    long iteration = 10000;
    double targetres = 1e-10;
    double chord = 1.0;
    cudaStream_t st = nullptr;
    Geom g{};
    double* geom_arena = nullptr;
    double* d_xy = nullptr;
    double* d_scratch = nullptr;
};

// Device-to-host copy of `bytes` on the solver's stream into pageable host
// memory, through the process's pinned staging buffers for large reads.
cudaError_t d2h_staged(SolverCore& C, void* dst, const void* src, size_t bytes);

void nonphysical_report(const PhysConst& c, long i, long j, const double u[5], jst_nonphysical* bad);
struct RawConfig;
PhysConst make_phys(const RawConfig& r);
void set_call_error(const std::string& msg);

class Engine {
  public:
    virtual ~Engine() {}
    virtual void init() = 0;
    virtual jst_status advance(jst_nonphysical* bad) = 0;
    virtual jst_status residual_terms(double* dt) = 0;
    // R = Fc - Fv - Fd, R[4] -= S of every interior cell of the current state
    // (5 planes of NI*NJ into out, host memory), from the stage kernels
    virtual jst_status stage_residual(double* out) = 0;
    virtual jst_status timestep(double* dt) = 0;
    virtual bool get_field(int id, double* out) = 0;
    virtual jst_status set_conserved(const double* u5, jst_nonphysical* bad) = 0;
    virtual jst_status wall_force(double* fx, double* fy) = 0;
    virtual jst_status residual(double* out) = 0;
    virtual jst_status totaltime(double* out) = 0;
    virtual jst_status set_totaltime(double t) = 0;
    virtual jst_status time_steps(int nsteps, double* ms, double* stage_ms) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, stream());
        jst_status rc = JST_OK;
        for (int k = 0; k < nsteps && rc == JST_OK; ++k) rc = advance(nullptr);
        cudaEventRecord(b, stream());
        cudaEventSynchronize(b);
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        *ms = t;
        if (stage_ms)
            for (int k = 0; k < 5; ++k) stage_ms[k] = -1.0;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return rc;
    }
    virtual cudaStream_t stream() const = 0;
    virtual void kernel_config(int* ti, int* tj, int* nt) const {
        *ti = 0;
        *tj = 0;
        *nt = 0;
    }
    // jst_staging of the stage kernel (0 when it is not a marching strip)
    virtual int kernel_staging() const { return 0; }
    virtual void set_stage_extra_tx(int) {}
    virtual void set_uniform(double, double, double, double, double) {}
    virtual void run_kernel(const char*) {}

    // Solver::run (solver.rs:203-226): advance, residual, callback, stop
    // below the target.
    virtual jst_status run_steps(int64_t limit, double target, jst_step_cb cb, void* user, int64_t* done,
                                 double* res, jst_nonphysical* bad) {
        *done = 0;
        *res = std::numeric_limits<double>::quiet_NaN();
        for (int64_t k = 1; k <= limit; ++k) {
            jst_status rc = advance(bad);
            if (rc != JST_OK) return rc;
            rc = residual(res);
            if (rc != JST_OK) return rc;
            *done = k;
            if (cb) cb(user, (uint64_t)k, *res);
            if (*res < target) break;
        }
        return JST_OK;
    }
};

// fused.cu
Engine* make_fused_engine(SolverCore* core, std::string& err);

}  // namespace jst
