// Host implementation of the C ABI in include/jst_gpu.h.
//
// The handle owns the parsed configuration, the trimmed mesh, the FP64
// geometry in HBM and one engine: the strict FP64 passes path (passes.cu) or
// the fused tiled path (fused.cu).  Mirrors the reference's Solver
// (jst-rs/src/solver.rs:25-256): new -> geometry, free stream, boundary
// conditions; advance = one 5-stage RK step; run = advance until the step
// limit or the target residual.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/jst_gpu.h"
#include "config_mesh.h"
#include "engine.h"
#include "jst_internal.h"

using namespace jst;

static thread_local std::string g_create_error;

namespace jst {

// Error text for entry points without a handle (read with jst_last_error(NULL)).
void set_call_error(const std::string& msg) { g_create_error = msg; }

const double RK_ALPHA[5] = {0.25, 1.0 / 6.0, 0.375, 0.5, 1.0};  // config.rs:217

// Config::finish (config.rs:173-206) + the constant sub-expressions of
// PhysConst + the free-stream state of Cells::initialize (state.rs:174-190).
PhysConst make_phys(const RawConfig& r) {
    PhysConst c{};
    c.gamma = r.gamma;
    c.r_gas = r.r_gas;
    c.t_suth = r.t_suth;
    c.cfl = r.cfl;
    c.t_inf = r.t_inf;
    c.p_inf = r.p_inf;
    c.k2 = r.k2;
    c.k4 = r.k4;
    c.Cb1 = r.Cb1;
    c.Cb2 = r.Cb2;
    c.Ct3 = r.Ct3;
    c.Ct4 = r.Ct4;
    c.Cw2 = r.Cw2;
    c.fv3 = r.fv3;
    c.rmax = r.rmax;
    c.sigma = r.sigma;
    double cv = r.r_gas / (r.gamma - 1.0);
    double c_inf = std::sqrt(r.gamma * r.r_gas * r.t_inf);
    double aoa = r.aoa * (M_PI / 180.0);
    double rho_inf = r.p_inf / (r.r_gas * r.t_inf);
    double rr = r.t_inf / r.t_ref;
    double mu_inf = r.mu0 * (rr * std::sqrt(rr)) * (r.t_ref + r.t_suth) / (r.t_inf + r.t_suth);
    double u_inf = c_inf * r.mach * std::cos(aoa);
    double v_inf = c_inf * r.mach * std::sin(aoa);
    c.cv = cv;
    c.cp = r.gamma * cv;
    c.cw1 = r.Cb1 / (r.kappa * r.kappa) + (1.0 + r.Cb2) * r.sigma;
    c.cv1_cubed = powi3(r.Cv1);
    c.c_inf = c_inf;
    c.u_inf = u_inf;
    c.v_inf = v_inf;
    c.rho_inf = rho_inf;
    c.mu_inf = mu_inf;
    c.nut_inf = r.nut_inf_ratio * mu_inf / rho_inf;
    c.supersonic = std::hypot(u_inf, v_inf) >= c_inf ? 1 : 0;
    c.suth_num = r.mu0 * (r.t_ref + r.t_suth);
    c.inv_t_ref = 1.0 / r.t_ref;
    c.inv_pr = 1.0 / r.Pr;
    c.inv_prt = 1.0 / r.Prt;
    c.inv_kappa2 = 1.0 / (r.kappa * r.kappa);
    c.cw3_6 = powi6(r.Cw3);
    c.one_plus_cw3_6 = 1.0 + powi6(r.Cw3);
    c.fw_lim = std::pow(c.one_plus_cw3_6, 1.0 / 6.0);
    c.gm1 = r.gamma - 1.0;
    c.rg = r.r_gas * r.gamma;
    c.gm1_q = (r.gamma - 1.0) / 4.0;
    c.inv_gm1 = 1.0 / (r.gamma - 1.0);
    c.half_cfl = 0.5 * r.cfl;
    c.cb1_k2 = r.Cb1 * c.inv_kappa2;
    c.cb2_sigma = r.Cb2 * r.sigma;
    c.r_gas_gamma = r.r_gas * r.gamma;
    c.halo = (int)r.halo;
    // PrimState::from_primitives (state.rs:222-237) of the free stream
    double rho = r.p_inf / (r.r_gas * r.t_inf);
    double p = r.p_inf;
    double t = p / (r.r_gas * rho);
    double e = p / (rho * (r.gamma - 1.0)) + 0.5 * (u_inf * u_inf + v_inf * v_inf);
    c.f_rho = rho;
    c.f_p = p;
    c.f_t = t;
    c.f_vx = u_inf;
    c.f_vy = v_inf;
    c.f_e = e;
    c.f_h = e + p / rho;
    c.f_c = std::sqrt(r.gamma * r.r_gas * t);
    c.f_nut = c.nut_inf;
    double rm = r.t_inf * c.inv_t_ref;
    c.f_mu = rm * std::sqrt(rm) * c.suth_num / (r.t_inf + r.t_suth);  // Config::mu (config.rs:210-213)
    return c;
}

// Host unpack of one cell for NonPhysical reports (solver.rs:158-171).
void nonphysical_report(const PhysConst& c, long i, long j, const double u[5], jst_nonphysical* bad) {
    if (!bad) return;
    bad->i = i;
    bad->j = j;
    double rho = u[0];
    bad->rho = rho;
    if (std::isnan(rho) || rho <= 1e-15) {
        bad->p = std::numeric_limits<double>::quiet_NaN();
        return;
    }
    double inv = 1.0 / rho;
    double vx = u[1] * inv, vy = u[2] * inv;
    bad->p = c.gm1 * (u[3] - rho * (vx * vx + vy * vy) * 0.5);
}

// ------------------------------------------------------- passes engine ----
// Touches every page of a large output buffer from several threads before a
// device-to-host copy into it.  A freshly allocated host array is mapped on
// first write, and the kernel zero-fills each new page on the faulting
// thread; done inside the copy that runs on one thread at a few GB/s (on a
// 4.2 M-cell field, 9 ms of a copy that takes 2 ms into mapped memory).
// Each touch writes back the byte it read, so the caller's data is unchanged
// when the call then fails.
static void prefault(void* p, size_t bytes) {
    constexpr size_t kPage = 4096, kMin = size_t(4) << 20;
    if (bytes < kMin) return;
    const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const size_t per = (bytes + nt - 1) / nt;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([=] {
            volatile char* c = static_cast<volatile char*>(p);
            const size_t a = t * per, b = std::min(bytes, a + per);
            for (size_t k = a; k < b; k += kPage) c[k] = c[k];
        });
    for (auto& x : th) x.join();
}

// Copies n bytes from src to dst with up to 8 host threads, each on its own
// page-aligned range (a fresh destination is mapped by the threads in
// parallel).
static void parallel_copy(void* dst, const void* src, size_t n) {
    constexpr size_t kPage = 4096;
    const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const size_t per = ((n + nt - 1) / nt + kPage - 1) / kPage * kPage;
    std::vector<std::thread> th;
    for (size_t a = 0; a < n; a += per) {
        const size_t b = std::min(n, a + per);
        th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a); });
    }
    for (auto& x : th) x.join();
}

// A device-to-host copy into pageable memory runs through the driver's own
// staging at a few GB/s on one thread.  Reads of 4 MiB and more go instead
// through two pinned 8 MiB buffers: the device fills one at full link rate
// while parallel_copy moves the other on.  The buffers belong to the process
// (portable pinned memory, valid for every device; allocated by the first
// large read, about 10 ms, and kept until exit) and are taken under a mutex,
// so concurrent reads of several solvers take turns.  If they cannot be had,
// the plain copy is used.
static std::mutex g_pin_mu;
static char* g_pin = nullptr;

cudaError_t d2h_staged(SolverCore& C, void* dst, const void* src, size_t bytes) {
    constexpr size_t kMin = size_t(4) << 20, kChunk = size_t(8) << 20;
    std::unique_lock<std::mutex> lk(g_pin_mu, std::defer_lock);
    if (bytes >= kMin) {
        lk.lock();
        if (!g_pin) {
            void* p = nullptr;
            if (cudaHostAlloc(&p, 2 * kChunk, cudaHostAllocPortable) == cudaSuccess) g_pin = static_cast<char*>(p);
            else cudaGetLastError();
        }
    }
    if (bytes < kMin || !g_pin) {
        prefault(dst, bytes);
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, C.st);
        return e != cudaSuccess ? e : cudaStreamSynchronize(C.st);
    }
    char* buf[2] = {g_pin, g_pin + kChunk};
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t q) {
        const size_t off = q * kChunk, n = std::min(kChunk, bytes - off);
        cudaError_t e = cudaMemcpyAsync(buf[q & 1], static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost,
                                        C.st);
        return e == cudaSuccess ? cudaEventRecord(ev[q & 1], C.st) : e;
    };
    cudaError_t e = issue(0);
    for (size_t q = 0; q < nch && e == cudaSuccess; ++q) {
        if (q + 1 < nch) e = issue(q + 1);  // its buffer was emptied by chunk q-1's copy
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[q & 1]);
        if (e == cudaSuccess) {
            const size_t off = q * kChunk;
            parallel_copy(static_cast<char*>(dst) + off, buf[q & 1], std::min(kChunk, bytes - off));
        }
    }
    if (e != cudaSuccess) cudaStreamSynchronize(C.st);  // no copy into the buffers stays in flight
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return e;
}

class PassesEngine : public Engine {
  public:
    PassesEngine(SolverCore* core) : core_(core) {}
    ~PassesEngine() override { passes_destroy(P_); }

    bool create(std::string& err) {
        P_ = passes_create(core_->ni, core_->nj, core_->H, &err);
        return P_ != nullptr;
    }
    void init() override { passes_init(P_, core_->g, core_->c, core_->st); }

    jst_status advance(jst_nonphysical* bad) override {
        cudaStream_t st = core_->st;
        passes_snapshot(P_, st);
        passes_timestep(P_, core_->g, core_->c, 1, st);
        for (int k = 0; k < 5; ++k) {
            passes_residual_terms(P_, core_->g, core_->c, st);
            unsigned long long none = ~0ULL;
            cudaMemcpyAsync(passes_bad_ptr(P_), &none, sizeof none, cudaMemcpyHostToDevice, st);
            passes_update_unpack(P_, core_->g, core_->c, RK_ALPHA[k], core_->local_dt, st);
            unsigned long long key = 0;
            cudaMemcpyAsync(&key, passes_bad_ptr(P_), sizeof key, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return JST_ERR_CUDA;
            if (key != ~0ULL) return report(key, bad);
        }
        passes_residual(P_, st);
        return JST_OK;
    }

    jst_status report(unsigned long long key, jst_nonphysical* bad) {
        long i = (long)(key / core_->nj), j = (long)(key % core_->nj);
        double u[5];
        for (int k = 0; k < 5; ++k) {
            const double* base;
            int stride, h;
            passes_field(P_, 9 + k, &base, &stride, &h);
            cudaMemcpy(&u[k], base + (size_t)(i + h) * stride + (j + h), sizeof(double), cudaMemcpyDeviceToHost);
        }
        nonphysical_report(core_->c, i, j, u, bad);
        return JST_ERR_NONPHYSICAL;
    }

    jst_status residual_terms(double* dt) override {
        if (dt) {
            passes_timestep(P_, core_->g, core_->c, 0, core_->st);
            cudaMemcpyAsync(dt, passes_dt_ptr(P_), sizeof(double), cudaMemcpyDeviceToHost, core_->st);
        }
        passes_residual_terms(P_, core_->g, core_->c, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    // The terms of the passes (time step first, then residual_terms) combined
    // on the host in the order of Solver::update (solver.rs:128-133).
    jst_status stage_residual(double* out) override {
        double dt = 0.0;
        jst_status rc = residual_terms(&dt);
        if (rc != JST_OK) return rc;
        size_t n = (size_t)core_->ni * core_->nj;
        std::vector<double> fv(n), fd(n);
        for (int k = 0; k < 5; ++k) {
            double* r = out + k * n;
            if (!get_field(JST_F_FC0 + k, r) || !get_field(JST_F_FV0 + k, fv.data()) ||
                !get_field(JST_F_FD0 + k, fd.data()))
                return JST_ERR_CUDA;
            for (size_t q = 0; q < n; ++q) r[q] = r[q] - fv[q] - fd[q];
        }
        if (!get_field(JST_F_S, fv.data())) return JST_ERR_CUDA;
        for (size_t q = 0; q < n; ++q) out[4 * n + q] -= fv[q];
        return JST_OK;
    }

    jst_status timestep(double* dt) override {
        passes_timestep(P_, core_->g, core_->c, 0, core_->st);
        cudaMemcpyAsync(dt, passes_dt_ptr(P_), sizeof(double), cudaMemcpyDeviceToHost, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    bool get_field(int id, double* out) override {
        const double* base;
        int stride, h;
        if (!passes_field(P_, id, &base, &stride, &h)) return false;
        prefault(out, sizeof(double) * core_->ni * core_->nj);
        cudaMemcpy2DAsync(out, sizeof(double) * core_->nj, base + (size_t)h * stride + h, sizeof(double) * stride,
                          sizeof(double) * core_->nj, core_->ni, cudaMemcpyDeviceToHost, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess;
    }

    jst_status set_conserved(const double* u5, jst_nonphysical* bad) override {
        size_t n = (size_t)core_->ni * core_->nj;
        for (int k = 0; k < 5; ++k) {
            const double* base;
            int stride, h;
            passes_field(P_, 9 + k, &base, &stride, &h);
            cudaMemcpy2DAsync(const_cast<double*>(base) + (size_t)h * stride + h, sizeof(double) * stride,
                              u5 + k * n, sizeof(double) * core_->nj, sizeof(double) * core_->nj, core_->ni,
                              cudaMemcpyHostToDevice, core_->st);
        }
        unsigned long long none = ~0ULL, key = 0;
        cudaMemcpyAsync(passes_bad_ptr(P_), &none, sizeof none, cudaMemcpyHostToDevice, core_->st);
        passes_unpack(P_, core_->c, core_->st);
        cudaMemcpyAsync(&key, passes_bad_ptr(P_), sizeof key, cudaMemcpyDeviceToHost, core_->st);
        if (cudaStreamSynchronize(core_->st) != cudaSuccess) return JST_ERR_CUDA;
        if (key != ~0ULL) return report(key, bad);
        return JST_OK;
    }

    jst_status wall_force(double* fx, double* fy) override {
        cudaStream_t st = core_->st;
        passes_kernel(P_, core_->g, core_->c, "boundary", st);
        passes_kernel(P_, core_->g, core_->c, "gradient", st);
        passes_kernel(P_, core_->g, core_->c, "viscous", st);
        passes_wall_force(P_, core_->g, core_->d_scratch, st);
        double f[2];
        cudaMemcpyAsync(f, core_->d_scratch, sizeof f, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return JST_ERR_CUDA;
        *fx = f[0];
        *fy = f[1];
        return JST_OK;
    }

    jst_status residual(double* out) override {
        cudaMemcpyAsync(out, passes_residual_ptr(P_), sizeof(double), cudaMemcpyDeviceToHost, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    jst_status totaltime(double* out) override {
        cudaMemcpyAsync(out, passes_totaltime_ptr(P_), sizeof(double), cudaMemcpyDeviceToHost, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    jst_status set_totaltime(double t) override {
        cudaMemcpyAsync(passes_totaltime_ptr(P_), &t, sizeof t, cudaMemcpyHostToDevice, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    void set_uniform(double rho, double vx, double vy, double p, double nut) override {
        passes_set_uniform(P_, core_->c, rho, vx, vy, p, nut, core_->st);
    }
    void run_kernel(const char* name) override { passes_kernel(P_, core_->g, core_->c, name, core_->st); }
    cudaStream_t stream() const override { return core_->st; }

  private:
    SolverCore* core_;
    Passes* P_ = nullptr;
};

}  // namespace jst

// -------------------------------------------------------------- handle ----
struct jst_solver {
    SolverCore core;
    std::unique_ptr<Engine> eng;
    std::string err;
    int64_t step = 0;
    double last_residual = std::numeric_limits<double>::quiet_NaN();
    RawConfig raw;
    ~jst_solver() {
        eng.reset();
        if (core.geom_arena) cudaFree(core.geom_arena);
        if (core.d_xy) cudaFree(core.d_xy);
        if (core.d_scratch) cudaFree(core.d_scratch);
        if (core.st) cudaStreamDestroy(core.st);
    }
};

static jst_status cuda_fail(jst_solver* s, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (s) s->err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? JST_ERR_OOM : JST_ERR_CUDA;
}

extern "C" {

void jst_default_opts(jst_opts* o) {
    std::memset(o, 0, sizeof *o);
    o->precision = JST_PREC_FP64;
    o->dt_mode = JST_DT_GLOBAL;
    o->kernel_path = JST_PATH_FUSED;
    o->device = 0;
    o->use_graph = 1;
    o->nut_inf_ratio = 0.0;
}

const char* jst_version(void) { return "purinecfd_b200 0.1 (sm_100a)"; }

const char* jst_last_error(const jst_solver* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

int jst_ni(const jst_solver* s) { return s ? s->core.ni : -1; }
int jst_nj(const jst_solver* s) { return s ? s->core.nj : -1; }

jst_status jst_create(const char* config_json, const double* xy_in, int n_rings, int n_theta, const jst_opts* opts,
                      jst_solver** out) {
    if (!out || !config_json || !xy_in) {
        g_create_error = "null argument";
        return JST_ERR_ARG;
    }
    *out = nullptr;
    jst_opts o;
    if (opts) o = *opts;
    else jst_default_opts(&o);
    RawConfig raw;
    std::string err;
    if (!parse_config(config_json, raw, err)) {
        g_create_error = err;
        return JST_ERR_CONFIG;
    }
    if (o.nut_inf_ratio > 0.0) raw.nut_inf_ratio = o.nut_inf_ratio;
    if (raw.halo < 3) {
        g_create_error = "simulation.IM must be >= 3: the JST pressure sensor needs three ghost layers";
        return JST_ERR_CONFIG;
    }
    // trim_closing_duplicate (mesh.rs:169-189), tested on the caller's node
    // array; the upload below leaves the duplicate column out (a pitched copy),
    // so the nodes are not copied on the host
    const int n_theta_in = n_theta;
    if (n_theta >= 2) {
        bool closed = true;
        for (long r = 0; r < n_rings && closed; ++r) {
            const double* a = xy_in + 2 * (r * n_theta);
            const double* b = a + 2 * (n_theta - 1);
            closed = std::fabs(a[0] - b[0]) <= 1e-10 && std::fabs(a[1] - b[1]) <= 1e-10;
        }
        if (closed) n_theta -= 1;
    }
    if (n_rings < 4 || n_theta < 8) {
        g_create_error = "mesh too small: the JST 4th-order stencil needs at least 4 rings and 8 circumferential points";
        return JST_ERR_MESH_TOO_SMALL;
    }
    if (o.precision != JST_PREC_FP64 && o.precision != JST_PREC_FP32_SPLIT) return JST_ERR_ARG;
    if (o.kernel_path == JST_PATH_PASSES && o.precision != JST_PREC_FP64) {
        g_create_error = "the passes path is FP64 only";
        return JST_ERR_ARG;
    }

    std::unique_ptr<jst_solver> s(new jst_solver());
    SolverCore& C = s->core;
    s->raw = raw;
    C.opts = o;
    C.n_rings = n_rings;
    C.n_theta = n_theta;
    C.ni = n_rings - 1;
    C.nj = n_theta;
    C.H = (int)raw.halo;
    C.c = make_phys(raw);
    C.local_dt = o.dt_mode == JST_DT_LOCAL ? 1 : 0;
    C.iteration = raw.iteration;
    C.targetres = raw.targetres;
    double xmin = 1e300, xmax = -1e300;
    for (int t = 0; t < n_theta; ++t) {
        xmin = std::min(xmin, xy_in[2 * t]);
        xmax = std::max(xmax, xy_in[2 * t]);
    }
    C.chord = raw.chord > 0.0 ? raw.chord : xmax - xmin;

    if (cudaSetDevice(o.device) != cudaSuccess) {
        g_create_error = "cudaSetDevice failed (no CUDA device?)";
        return JST_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&C.st, cudaStreamNonBlocking) != cudaSuccess) {
        g_create_error = "cudaStreamCreate failed";
        return JST_ERR_CUDA;
    }
    size_t ncell = (size_t)C.ni * C.nj, ntau = (size_t)(C.ni + 1) * C.nj;
    size_t geom_elems = 6 * ncell + 4 * ntau + 4 * ncell;
    if (cudaMalloc(&C.geom_arena, geom_elems * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&C.d_xy, 2 * (size_t)n_rings * n_theta * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&C.d_scratch, 64 * sizeof(double)) != cudaSuccess) {
        g_create_error = "cudaMalloc failed for geometry";
        return JST_ERR_OOM;
    }
    double* q = C.geom_arena;
    Geom& g = C.g;
    g.ni = C.ni;
    g.nj = C.nj;
    g.vol = q; q += ncell;
    g.cx = q; q += ncell;
    g.cy = q; q += ncell;
    g.wdist = q; q += ncell;
    g.inv_vol = q; q += ncell;
    g.inv_d2 = q; q += ncell;
    g.tnx = q; q += ntau;
    g.tny = q; q += ntau;
    g.tmx = q; q += ntau;
    g.tmy = q; q += ntau;
    g.nnx = q; q += ncell;
    g.nny = q; q += ncell;
    g.nmx = q; q += ncell;
    g.nmy = q; q += ncell;
    if (cudaMemcpy2DAsync(C.d_xy, 2 * sizeof(double) * n_theta, xy_in, 2 * sizeof(double) * n_theta_in,
                          2 * sizeof(double) * n_theta, n_rings, cudaMemcpyHostToDevice, C.st) != cudaSuccess) {
        g_create_error = "mesh upload failed";
        return JST_ERR_CUDA;
    }
    geometry_build(C.d_xy, n_rings, n_theta, g, C.st);

    if (o.kernel_path == JST_PATH_PASSES) {
        auto* pe = new PassesEngine(&C);
        s->eng.reset(pe);
        if (!pe->create(err)) {
            g_create_error = err;
            return JST_ERR_OOM;
        }
    } else {
        Engine* fe = make_fused_engine(&C, err);
        if (!fe) {
            g_create_error = err;
            return JST_ERR_OOM;
        }
        s->eng.reset(fe);
    }
    s->eng->init();
    if (cudaStreamSynchronize(C.st) != cudaSuccess) {
        g_create_error = std::string("CUDA error during setup: ") + cudaGetErrorString(cudaGetLastError());
        return JST_ERR_CUDA;
    }
    *out = s.release();
    return JST_OK;
}

jst_status jst_create_from_paths(const char* config_path, const char* mesh_path, const jst_opts* opts,
                                 jst_solver** out) {
    std::ifstream fc(config_path ? config_path : "");
    if (!fc) {
        g_create_error = std::string("cannot read config ") + (config_path ? config_path : "(null)");
        return JST_ERR_CONFIG;
    }
    std::stringstream bc;
    bc << fc.rdbuf();
    std::ifstream fm(mesh_path ? mesh_path : "");
    if (!fm) {
        g_create_error = std::string("I/O error: cannot read mesh ") + (mesh_path ? mesh_path : "(null)");
        return JST_ERR_MESH_IO;
    }
    std::stringstream bm;
    bm << fm.rdbuf();
    std::vector<double> xy;
    int nr = 0, nt = 0;
    std::string err;
    int rc = parse_mesh(bm.str(), xy, &nr, &nt, err);
    if (rc != MESH_OK) {
        g_create_error = err;
        return (jst_status)rc;
    }
    return jst_create(bc.str().c_str(), xy.data(), nr, nt, opts, out);
}

void jst_destroy(jst_solver* s) { delete s; }

jst_status jst_advance(jst_solver* s, jst_nonphysical* bad) {
    if (!s) return JST_ERR_ARG;
    jst_status rc = s->eng->advance(bad);
    if (rc == JST_OK) {
        s->step += 1;
        s->eng->residual(&s->last_residual);
    } else if (rc == JST_ERR_NONPHYSICAL && bad) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "non-physical state at cell (%lld, %lld): rho = %e, p = %e", (long long)bad->i,
                      (long long)bad->j, bad->rho, bad->p);
        s->err = buf;
    } else if (rc == JST_ERR_TIMEOUT) {
        s->err = "a stage kernel's bounded wait for its row copies ran out";
    } else if (rc != JST_OK) {
        s->err = "advance failed";
    }
    return rc;
}

jst_status jst_run(jst_solver* s, int64_t max_steps, jst_step_cb cb, void* user, jst_run_report* rep,
                   jst_nonphysical* bad) {
    if (!s) return JST_ERR_ARG;
    int64_t limit = max_steps < 0 ? (int64_t)s->core.iteration : max_steps;
    double res = std::numeric_limits<double>::quiet_NaN();
    int64_t done = 0;
    jst_nonphysical local_bad;
    jst_nonphysical* b = bad ? bad : &local_bad;
    jst_status rc = JST_OK;
    rc = s->eng->run_steps(limit, s->core.targetres, cb, user, &done, &res, b);
    s->step += done;
    s->last_residual = res;
    if (rc == JST_ERR_NONPHYSICAL) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "non-physical state at cell (%lld, %lld): rho = %e, p = %e", (long long)b->i,
                      (long long)b->j, b->rho, b->p);
        s->err = buf;
    } else if (rc == JST_ERR_TIMEOUT) {
        s->err = "a stage kernel's bounded wait for its row copies ran out";
    }
    if (rep) {
        rep->steps = done;
        rep->residual = res;
        s->eng->totaltime(&rep->totaltime);
        rep->converged = res < s->core.targetres;
    }
    return rc;
}

jst_status jst_residual_terms(jst_solver* s, double* dt) { return s ? s->eng->residual_terms(dt) : JST_ERR_ARG; }

jst_status jst_stage_residual(jst_solver* s, double* out, size_t n) {
    if (!s || !out) return JST_ERR_ARG;
    size_t nc = (size_t)s->core.ni * s->core.nj;
    if (n < 5 * nc) {
        s->err = "jst_stage_residual: out must hold 5*NI*NJ doubles";
        return JST_ERR_ARG;
    }
    jst_status rc = s->eng->stage_residual(out);
    if (rc == JST_ERR_CUDA) return cuda_fail(s, "stage_residual");
    if (rc == JST_ERR_OOM) s->err = "jst_stage_residual: cudaMalloc failed for the residual buffer";
    return rc;
}
jst_status jst_timestep(jst_solver* s, double* dt) { return s && dt ? s->eng->timestep(dt) : JST_ERR_ARG; }

jst_status jst_residual(jst_solver* s, double* out) {
    if (!s || !out) return JST_ERR_ARG;
    *out = s->last_residual;
    return JST_OK;
}

jst_status jst_totaltime(const jst_solver* s, double* out) {
    if (!s || !out) return JST_ERR_ARG;
    return s->eng->totaltime(out);
}

jst_status jst_step_count(const jst_solver* s, int64_t* out) {
    if (!s || !out) return JST_ERR_ARG;
    *out = s->step;
    return JST_OK;
}

jst_status jst_get_field(jst_solver* s, int field, double* out, size_t n) {
    if (!s || !out || field < 0 || field >= JST_F_COUNT) return JST_ERR_ARG;
    size_t nc = (size_t)s->core.ni * s->core.nj;
    if (n < nc) return JST_ERR_ARG;
    const Geom& g = s->core.g;
    const double* geo = nullptr;
    switch (field) {
        case JST_F_VOL: geo = g.vol; break;
        case JST_F_CX: geo = g.cx; break;
        case JST_F_CY: geo = g.cy; break;
        case JST_F_WALL_DIST: geo = g.wdist; break;
        default: break;
    }
    if (geo) {
        if (d2h_staged(s->core, out, geo, nc * sizeof(double)) != cudaSuccess) return cuda_fail(s, "get_field");
        return JST_OK;
    }
    if (!s->eng->get_field(field, out)) {
        s->err = "field not available on this kernel path";
        return JST_ERR_ARG;
    }
    return JST_OK;
}

jst_status jst_get_faces(jst_solver* s, int which, double* out, size_t n) {
    if (!s || !out) return JST_ERR_ARG;
    const Geom& g = s->core.g;
    size_t nf = which == 0 ? (size_t)(g.ni + 1) * g.nj : (size_t)g.ni * g.nj;
    if (n < 4 * nf || (which != 0 && which != 1)) return JST_ERR_ARG;
    std::vector<double> a(nf), b(nf), c(nf), d(nf);
    const double* src[4] = {which == 0 ? g.tnx : g.nnx, which == 0 ? g.tny : g.nny, which == 0 ? g.tmx : g.nmx,
                            which == 0 ? g.tmy : g.nmy};
    std::vector<double>* dst[4] = {&a, &b, &c, &d};
    for (int k = 0; k < 4; ++k)
        if (cudaMemcpy(dst[k]->data(), src[k], nf * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return cuda_fail(s, "get_faces");
    for (size_t f = 0; f < nf; ++f) {
        out[4 * f] = a[f];
        out[4 * f + 1] = b[f];
        out[4 * f + 2] = c[f];
        out[4 * f + 3] = d[f];
    }
    return JST_OK;
}

jst_status jst_set_conserved(jst_solver* s, const double* u5, size_t n, jst_nonphysical* bad) {
    if (!s || !u5 || n < 5 * (size_t)s->core.ni * s->core.nj) return JST_ERR_ARG;
    return s->eng->set_conserved(u5, bad);
}

namespace {
const char kCkptMagic[8] = {'J', 'S', 'T', 'C', 'K', 'P', 'T', '1'};
void ckpt_error(jst_solver* s, const std::string& msg) {
    s->err = msg;
    set_call_error(msg);
}
}

jst_status jst_checkpoint_save(jst_solver* s, const char* path) {
    if (!s || !path) return JST_ERR_ARG;
    const size_t n = (size_t)s->core.ni * s->core.nj;
    std::vector<double> u(5 * n);
    for (int k = 0; k < 5; ++k)
        if (!s->eng->get_field(JST_F_U0 + k, u.data() + k * n)) {
            ckpt_error(s, "cannot read the conserved state");
            return JST_ERR_CUDA;
        }
    double tt = 0.0, res = std::numeric_limits<double>::quiet_NaN();
    if (s->eng->totaltime(&tt) != JST_OK) return JST_ERR_CUDA;
    if (s->step > 0) s->eng->residual(&res);
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        ckpt_error(s, std::string("cannot create ") + path);
        return JST_ERR_ARG;
    }
    int32_t dims[2] = {s->core.ni, s->core.nj};
    int64_t step = s->step;
    bool ok = std::fwrite(kCkptMagic, 1, 8, f) == 8 && std::fwrite(dims, sizeof dims, 1, f) == 1 &&
              std::fwrite(&step, sizeof step, 1, f) == 1 && std::fwrite(&tt, sizeof tt, 1, f) == 1 &&
              std::fwrite(&res, sizeof res, 1, f) == 1 && std::fwrite(u.data(), sizeof(double), u.size(), f) == u.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        ckpt_error(s, std::string("cannot write ") + path);
        return JST_ERR_ARG;
    }
    return JST_OK;
}

jst_status jst_checkpoint_load(jst_solver* s, const char* path, jst_nonphysical* bad) {
    if (!s || !path) return JST_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        ckpt_error(s, std::string("cannot open ") + path);
        return JST_ERR_ARG;
    }
    char magic[8];
    int32_t dims[2];
    int64_t step = 0;
    double tt = 0.0, res = 0.0;
    const size_t n = (size_t)s->core.ni * s->core.nj;
    std::vector<double> u(5 * n);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCkptMagic, 8) == 0 &&
              std::fread(dims, sizeof dims, 1, f) == 1 && dims[0] == s->core.ni && dims[1] == s->core.nj &&
              std::fread(&step, sizeof step, 1, f) == 1 && step >= 0 && std::fread(&tt, sizeof tt, 1, f) == 1 &&
              std::fread(&res, sizeof res, 1, f) == 1 && std::fread(u.data(), sizeof(double), u.size(), f) == u.size();
    std::fclose(f);
    if (!ok) {
        ckpt_error(s, std::string(path) + ": not a checkpoint of a " + std::to_string(s->core.ni) + " x " +
                       std::to_string(s->core.nj) + " mesh, or truncated");
        return JST_ERR_ARG;
    }
    jst_nonphysical tmp{};
    jst_status rc = s->eng->set_conserved(u.data(), bad ? bad : &tmp);
    if (rc != JST_OK) return rc;
    rc = s->eng->set_totaltime(tt);
    if (rc != JST_OK) return rc;
    s->step = step;
    return JST_OK;
}

jst_status jst_forces(jst_solver* s, double* cl, double* cd) {
    if (!s || !cl || !cd) return JST_ERR_ARG;
    double fx = 0, fy = 0;
    jst_status rc = s->eng->wall_force(&fx, &fy);
    if (rc != JST_OK) return rc;
    const PhysConst& c = s->core.c;
    double aoa = s->raw.aoa * (M_PI / 180.0);
    double q = 0.5 * c.rho_inf * (c.u_inf * c.u_inf + c.v_inf * c.v_inf) * s->core.chord;
    *cd = (fx * std::cos(aoa) + fy * std::sin(aoa)) / q;
    *cl = (-fx * std::sin(aoa) + fy * std::cos(aoa)) / q;
    return JST_OK;
}

jst_status jst_write_csv(jst_solver* s, const char* path) {
    if (!s || !path) return JST_ERR_ARG;
    size_t nc = (size_t)s->core.ni * s->core.nj;
    std::vector<double> cx(nc), cy(nc), rho(nc), p(nc), t(nc), u(nc), v(nc), nut(nc);
    jst_status rc;
    if ((rc = jst_get_field(s, JST_F_CX, cx.data(), nc)) || (rc = jst_get_field(s, JST_F_CY, cy.data(), nc)) ||
        (rc = jst_get_field(s, JST_F_RHO, rho.data(), nc)) || (rc = jst_get_field(s, JST_F_P, p.data(), nc)) ||
        (rc = jst_get_field(s, JST_F_T, t.data(), nc)) || (rc = jst_get_field(s, JST_F_U, u.data(), nc)) ||
        (rc = jst_get_field(s, JST_F_V, v.data(), nc)) || (rc = jst_get_field(s, JST_F_NUT, nut.data(), nc)))
        return rc;
    FILE* f = std::fopen(path, "w");
    if (!f) {
        s->err = std::string("cannot write ") + path;
        return JST_ERR_ARG;
    }
    std::fputs("i,j,x,y,rho,p,T,u,v,miubl\n", f);
    for (int i = 0; i < s->core.ni; ++i)
        for (int j = 0; j < s->core.nj; ++j) {
            size_t k = (size_t)i * s->core.nj + j;
            std::fprintf(f, "%d,%d,%s,%s,%s,%s,%s,%s,%s,%s\n", i + 1, j + 1, rust_exp(cx[k], 8).c_str(),
                         rust_exp(cy[k], 8).c_str(), rust_exp(rho[k], 8).c_str(), rust_exp(p[k], 8).c_str(),
                         rust_exp(t[k], 8).c_str(), rust_exp(u[k], 8).c_str(), rust_exp(v[k], 8).c_str(),
                         rust_exp(nut[k], 8).c_str());
        }
    std::fclose(f);
    return JST_OK;
}

jst_status jst_kernel_config(const jst_solver* s, int* ti, int* tj, int* nt) {
    if (!s || !ti || !tj || !nt) return JST_ERR_ARG;
    s->eng->kernel_config(ti, tj, nt);
    return JST_OK;
}

jst_status jst_kernel_staging(const jst_solver* s, int* staging) {
    if (!s || !staging) return JST_ERR_ARG;
    *staging = s->eng->kernel_staging();
    return JST_OK;
}

jst_status jst_time_steps(jst_solver* s, int nsteps, double* ms, double* stage_ms) {
    if (!s || !ms || nsteps < 0) return JST_ERR_ARG;
    int64_t before = 0;
    jst_status rc = s->eng->time_steps(nsteps, ms, stage_ms);
    (void)before;
    if (rc == JST_OK) {
        s->step += nsteps + (stage_ms ? 1 : 0);
        s->eng->residual(&s->last_residual);
    }
    return rc;
}

// Test hooks (declared in include/jst_gpu_debug.h): uniform state on every cell and a
// single kernel by name, for the free-stream properties that must bypass the
// boundary conditions (jst-rs/tests/properties.rs:126-156).
jst_status jst_debug_set_uniform(jst_solver* s, double rho, double vx, double vy, double p, double nut) {
    if (!s) return JST_ERR_ARG;
    s->eng->set_uniform(rho, vx, vy, p, nut);
    return cudaStreamSynchronize(s->core.st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
}

jst_status jst_debug_staging_extra_tx(jst_solver* s, int bytes) {
    if (!s || bytes < 0 || bytes > (1 << 16)) return JST_ERR_ARG;
    s->eng->set_stage_extra_tx(bytes);
    return cudaStreamSynchronize(s->core.st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
}

jst_status jst_debug_kernel(jst_solver* s, const char* name) {
    if (!s || !name) return JST_ERR_ARG;
    s->eng->run_kernel(name);
    return cudaStreamSynchronize(s->core.st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
}

}  // extern "C"
