// Host side of the fused tiled path: one stage kernel per RK stage over a
// tile table, the 5 stages of a step captured once as a CUDA graph, and a
// device-side step counter / convergence flag so that many steps can be
// queued without a host round trip per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "fused_kernels.cuh"

namespace jst {

using fused::Inst;
using fused::InstState;
using fused::TileRef;

namespace {

// Initial state: U_n = pack(free stream) on every cell (state.rs:522-539).
__global__ void k_fill_freestream(double* u0, double* u1, double* u2, double* u3, double* u4, long n, PhysConst c) {
    long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    Prim<double> q;
    q.rho = c.f_rho;
    q.vx = c.f_vx;
    q.vy = c.f_vy;
    q.e = c.f_e;
    q.nut = c.f_nut;
    double u[5];
    pack_cell<double>(q, u);
    u0[id] = u[0];
    u1[id] = u[1];
    u2[id] = u[2];
    u3[id] = u[3];
    u4[id] = u[4];
}

// Per far-field column: tau(NI) normal and the centroid-to-face-midpoint
// distances of cells NI-1..NI-3 (boundary.rs:160-169).
__global__ void k_far_geom(Geom g, double* far) {
    long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.nj) return;
    long ni = g.ni, nj = g.nj;
    long f = ni * nj + j;
    far[5 * j + 0] = g.tnx[f];
    far[5 * j + 1] = g.tny[f];
    for (int k = 0; k < 3; ++k) {
        long cid = (ni - 1 - k) * nj + j;
        far[5 * j + 2 + k] = hypot(g.cx[cid] - g.tmx[f], g.cy[cid] - g.tmy[f]);
    }
}

// Wall force from U_n: per wall column j, the pressure and viscous flux
// through tau face (0, j) exactly as the residual terms form them
// (boundary.rs:30-51 mirror ghost, gradient.rs:22-35 and 87-95, viscous.rs:37-71
// and 128-139).  One block, fixed-order reduction.
__global__ void k_wall_force(Geom g, const double* const* un, PhysConst c, int fresh, double* out) {
    __shared__ double rx[256], ry[256];
    int nj = g.nj;
    double ax = 0.0, ay = 0.0;
    for (int j = threadIdx.x; j < nj; j += 256) {
        auto prim = [&](int i, int jj) {
            int w = jj < 0 ? jj + nj : (jj >= nj ? jj - nj : jj);
            long id = (long)i * nj + w;
            Prim<double> q;
            if (fresh) {
                q.rho = c.f_rho; q.p = c.f_p; q.t = c.f_t; q.vx = c.f_vx; q.vy = c.f_vy; q.e = c.f_e; q.nut = c.f_nut;
            } else {
                q = unpack_cell<double>(un[0][id], un[1][id], un[2][id], un[3][id], un[4][id], c.gm1, c.r_gas);
            }
            return q;
        };
        Prim<double> q0 = prim(0, j), q1 = prim(1, j), ql = prim(0, j - 1), qr = prim(0, j + 1);
        Prim<double> qg = q0;  // wall ghost -1 mirrors cell 0
        qg.vx = -qg.vx;
        qg.vy = -qg.vy;
        qg.nut = -qg.nut;
        int jp = j + 1 < nj ? j + 1 : 0;
        long up = (long)nj + j, dn = j, rt = jp;
        double iv = g.inv_vol[j];
        double gr[8];
        double c0[4] = {q0.vx, q0.vy, q0.t, q0.nut}, cu[4] = {q1.vx, q1.vy, q1.t, q1.nut};
        double cd[4] = {qg.vx, qg.vy, qg.t, qg.nut}, cl[4] = {ql.vx, ql.vy, ql.t, ql.nut};
        double cr[4] = {qr.vx, qr.vy, qr.t, qr.nut};
        for (int k = 0; k < 4; ++k)
            green_gauss<double>(c0[k], cu[k], cd[k], cl[k], cr[k], g.tnx[up], g.tny[up], g.tnx[dn], g.tny[dn],
                                g.nnx[dn], g.nny[dn], g.nnx[rt], g.nny[rt], iv, &gr[2 * k], &gr[2 * k + 1]);
        double u4_0 = q0.rho * q0.nut, u4_g = qg.rho * qg.nut;  // packed rho*nut
        if (!fresh) u4_0 = un[4][j];
        Diff<double> d0 = diffusion_tensor<double>(q0.t, u4_0, q0.vx, q0.vy, gr[0], gr[1], gr[2], gr[3], gr[4], gr[5],
                                                   gr[6], gr[7], c.inv_t_ref, c.suth_num, c.t_suth, c.cv1_cubed,
                                                   c.inv_pr, c.inv_prt, c.cp, c.sigma);
        Diff<double> dg = diffusion_tensor<double>(qg.t, u4_g, qg.vx, qg.vy, gr[0], gr[1], gr[2], gr[3], 0.0, 0.0,
                                                   gr[6], gr[7], c.inv_t_ref, c.suth_num, c.t_suth, c.cv1_cubed,
                                                   c.inv_pr, c.inv_prt, c.cp, c.sigma);
        double nx = g.tnx[j], ny = g.tny[j];
        double hx = 0.5 * nx, hy = 0.5 * ny;
        double fx = (dg.dx1 + d0.dx1) * hx + (dg.dy1 + d0.dy1) * hy;
        double fy = (dg.dx2 + d0.dx2) * hx + (dg.dy2 + d0.dy2) * hy;
        double pw = 0.5 * (qg.p + q0.p);
        ax += -pw * nx + fx;
        ay += -pw * ny + fy;
    }
    rx[threadIdx.x] = ax;
    ry[threadIdx.x] = ay;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            rx[threadIdx.x] += rx[threadIdx.x + w];
            ry[threadIdx.x] += ry[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = rx[0];
        out[1] = ry[0];
    }
}

template <class T> size_t stage_smem(int ti, int tj);

// Tile configurations compiled into the library: (TI, TJ, NT).
#define JST_FOR_TILES(X) X(4, 32, 256) X(8, 32, 256) X(16, 32, 256) X(4, 64, 256) X(8, 64, 256)

template <class T> struct Kernels {
    void (*stage[3])(const TileRef*, const Inst<T>*, int, double) = {nullptr, nullptr, nullptr};  // first, mid, last
    void (*step_dt)(const TileRef*, const Inst<T>*, int, int) = nullptr;
    size_t smem = 0;
    int nt = 256;
};

template <class T, int TI, int TJ, int NT> Kernels<T> kernels_for() {
    Kernels<T> k;
    k.stage[0] = fused::k_stage<T, TI, TJ, NT, true, false>;
    k.stage[1] = fused::k_stage<T, TI, TJ, NT, false, false>;
    k.stage[2] = fused::k_stage<T, TI, TJ, NT, false, true>;
    k.step_dt = fused::k_step_dt<T, NT>;
    k.smem = fused::Layout<T, TI, TJ, NT>::bytes;
    k.nt = NT;
    return k;
}

template <class T> bool pick_kernels(int ti, int tj, Kernels<T>* out) {
#define JST_PICK(a, b, n)                    \
    if (ti == a && tj == b) {                \
        *out = kernels_for<T, a, b, n>();    \
        return true;                         \
    }
    JST_FOR_TILES(JST_PICK)
#undef JST_PICK
    return false;
}

// Default tile per precision and mesh width (the autotuner refines this).
void default_tile(int prec, int nj, int* ti, int* tj) {
    if (prec == JST_PREC_FP64) {
        *ti = 8;
        *tj = 32;
    } else {
        *ti = nj >= 64 ? 16 : 8;
        *tj = 32;
    }
}

}  // namespace

template <class T> class FusedEngine : public Engine {
  public:
    explicit FusedEngine(SolverCore* core) : core_(core) {}
    ~FusedEngine() override {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (arena_) cudaFree(arena_);
        if (h_state_) cudaFreeHost(h_state_);
    }

    bool create(std::string& err) {
        SolverCore& C = *core_;
        int ti = C.opts.tile_i, tj = C.opts.tile_j;
        if (ti <= 0 || tj <= 0) default_tile(C.opts.precision, C.nj, &ti, &tj);
        if (!pick_kernels<T>(ti, tj, &K_)) {
            err = "unsupported tile shape " + std::to_string(ti) + "x" + std::to_string(tj);
            return false;
        }
        ti_ = ti;
        tj_ = tj;
        for (int k = 0; k < 3; ++k)
            if (cudaFuncSetAttribute(K_.stage[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K_.smem) !=
                cudaSuccess) {
                err = "stage kernel needs " + std::to_string(K_.smem) + " bytes of shared memory";
                return false;
            }
        int ni = C.ni, nj = C.nj;
        int tiles_i = (ni + ti - 1) / ti, tiles_j = (nj + tj - 1) / tj;
        ntiles_ = tiles_i * tiles_j;
        std::vector<TileRef> tiles;
        tiles.reserve(ntiles_);
        for (int a = 0; a < tiles_i; ++a)
            for (int b = 0; b < tiles_j; ++b) tiles.push_back(TileRef{0, a * ti, b * tj, a * tiles_j + b});
        size_t n = (size_t)ni * nj;
        size_t bytes = 0;
        auto add = [&](size_t b) {
            size_t o = bytes;
            bytes += (b + 255) / 256 * 256;
            return o;
        };
        size_t o_un = add(5 * n * sizeof(double));
        size_t o_ua = add(5 * n * sizeof(T));
        size_t o_ub = add(5 * n * sizeof(T));
        size_t o_ratio = add(2 * n * sizeof(T));
        size_t o_ldt = add(n * sizeof(double));
        size_t o_partial = add(2 * (size_t)ntiles_ * sizeof(double));
        size_t o_far = add(5 * (size_t)nj * sizeof(double));
        size_t o_st = add(sizeof(InstState));
        size_t o_inst = add(sizeof(Inst<T>));
        size_t o_tiles = add(tiles.size() * sizeof(TileRef));
        size_t o_force = add(8 * sizeof(double));
        size_t o_unptr = add(5 * sizeof(double*));
        hist_cap_ = 4096;
        size_t o_hist = add(hist_cap_ * sizeof(double));
        if (cudaMalloc(&arena_, bytes) != cudaSuccess) {
            err = "cudaMalloc failed for the fused-path state (" + std::to_string(bytes >> 20) + " MiB)";
            return false;
        }
        cudaMemsetAsync(arena_, 0, bytes, C.st);
        char* base = static_cast<char*>(arena_);
        Inst<T> I{};
        I.ni = ni;
        I.nj = nj;
        I.ntiles = ntiles_;
        I.local_dt = C.local_dt;
        I.tnx = C.g.tnx;
        I.tny = C.g.tny;
        I.nnx = C.g.nnx;
        I.nny = C.g.nny;
        I.vol = C.g.vol;
        I.inv_vol = C.g.inv_vol;
        I.inv_d2 = C.g.inv_d2;
        I.far = reinterpret_cast<double*>(base + o_far);
        for (int k = 0; k < 5; ++k) {
            I.un[k] = reinterpret_cast<double*>(base + o_un) + k * n;
            I.ua[k] = reinterpret_cast<T*>(base + o_ua) + k * n;
            I.ub[k] = reinterpret_cast<T*>(base + o_ub) + k * n;
        }
        I.ratio[0] = reinterpret_cast<T*>(base + o_ratio);
        I.ratio[1] = I.ratio[0] + n;
        I.ldt = reinterpret_cast<double*>(base + o_ldt);
        I.partial = reinterpret_cast<double*>(base + o_partial);
        I.res_hist = reinterpret_cast<double*>(base + o_hist);
        I.st = reinterpret_cast<InstState*>(base + o_st);
        I.c = C.c;
        inst_ = I;
        d_inst_ = reinterpret_cast<Inst<T>*>(base + o_inst);
        d_tiles_ = reinterpret_cast<TileRef*>(base + o_tiles);
        d_force_ = reinterpret_cast<double*>(base + o_force);
        d_unptr_ = reinterpret_cast<double**>(base + o_unptr);
        cudaMemcpyAsync(d_inst_, &inst_, sizeof inst_, cudaMemcpyHostToDevice, C.st);
        cudaMemcpyAsync(d_tiles_, tiles.data(), tiles.size() * sizeof(TileRef), cudaMemcpyHostToDevice, C.st);
        cudaMemcpyAsync(d_unptr_, inst_.un, 5 * sizeof(double*), cudaMemcpyHostToDevice, C.st);
        if (cudaMallocHost(&h_state_, sizeof(InstState)) != cudaSuccess) {
            err = "cudaMallocHost failed";
            return false;
        }
        JST_LAUNCH(k_far_geom, (nj + 255) / 256, 256, 0, C.st, C.g, const_cast<double*>(inst_.far));
        return cudaGetLastError() == cudaSuccess;
    }

    void reset_state(int fresh) {
        InstState s{};
        s.dt = 0.0;
        s.totaltime = 0.0;
        s.residual = std::numeric_limits<double>::quiet_NaN();
        s.target = core_->targetres;
        s.bad = fused::NO_BAD;
        s.counter = 0;
        s.step = 0;
        s.fresh = fresh;
        s.done = 0;
        s.max_step = INT_MAX;
        cudaMemcpyAsync(inst_.st, &s, sizeof s, cudaMemcpyHostToDevice, core_->st);
    }

    void init() override {
        SolverCore& C = *core_;
        long n = (long)C.ni * C.nj;
        JST_LAUNCH(k_fill_freestream, (unsigned)((n + 255) / 256), 256, 0, C.st, inst_.un[0], inst_.un[1],
                   inst_.un[2], inst_.un[3], inst_.un[4], n, C.c);
        reset_state(1);
        launch_step_dt();
    }

    void launch_step_dt() {
        JST_LAUNCH(K_.step_dt, ntiles_, K_.nt, 0, core_->st, d_tiles_, d_inst_, ti_, tj_);
    }

    void enqueue_step(cudaStream_t st) {
        for (int s = 0; s < 5; ++s) {
            auto kern = s == 0 ? K_.stage[0] : (s == 4 ? K_.stage[2] : K_.stage[1]);
            JST_LAUNCH(kern, ntiles_, K_.nt, K_.smem, st, d_tiles_, d_inst_, s, RK_ALPHA[s]);
        }
    }

    // One RK step; with use_graph the 5 stage launches are replayed from a
    // captured graph.
    void launch_step() {
        cudaStream_t st = core_->st;
        if (!core_->opts.use_graph) {
            enqueue_step(st);
            return;
        }
        ensure_graph();
        cudaGraphLaunch(graph_exec_, st);
    }

    void ensure_graph() {
        if (graph_exec_ || !core_->opts.use_graph) return;
        cudaStream_t st = core_->st;
        cudaGraph_t g;
        cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        enqueue_step(st);
        cudaStreamEndCapture(st, &g);
        cudaGraphInstantiate(&graph_exec_, g, 0);
        cudaGraphDestroy(g);
    }

    jst_status read_state(InstState* out) {
        cudaMemcpyAsync(h_state_, inst_.st, sizeof(InstState), cudaMemcpyDeviceToHost, core_->st);
        if (cudaStreamSynchronize(core_->st) != cudaSuccess) return JST_ERR_CUDA;
        *out = *h_state_;
        return JST_OK;
    }

    jst_status report(unsigned long long key, jst_nonphysical* bad) {
        long id = (long)(key & 0xffffffffULL);
        long i = id / core_->nj, j = id % core_->nj;
        double u[5];
        for (int k = 0; k < 5; ++k) {
            // stage output of the failing stage: U_n for the last stage, else the stage buffer
            int stage = (int)((key >> 32) % 5);
            if (stage == 4) {
                cudaMemcpy(&u[k], inst_.un[k] + id, sizeof(double), cudaMemcpyDeviceToHost);
            } else {
                T v;
                cudaMemcpy(&v, (stage % 2 == 0 ? inst_.ua[k] : inst_.ub[k]) + id, sizeof(T), cudaMemcpyDeviceToHost);
                u[k] = (double)v;
            }
        }
        nonphysical_report(core_->c, i, j, u, bad);
        return JST_ERR_NONPHYSICAL;
    }

    jst_status advance(jst_nonphysical* bad) override {
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        set_max_step(s.step + 1);
        launch_step();
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        if (s.bad != fused::NO_BAD) return report(s.bad, bad);
        return JST_OK;
    }

    void set_max_step(int m) {
        cudaMemcpyAsync(&inst_.st->max_step, &m, sizeof m, cudaMemcpyHostToDevice, core_->st);
        // the pageable copy completes before later stream work
        cudaStreamSynchronize(core_->st);
    }

    jst_status run_steps(int64_t limit, double target, jst_step_cb cb, void* user, int64_t* done, double* res,
                         jst_nonphysical* bad) override {
        *done = 0;
        *res = std::numeric_limits<double>::quiet_NaN();
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        int start = s.step;
        // target is enforced on the device (done flag); the host only limits the count
        int zero = 0;
        cudaMemcpyAsync(&inst_.st->done, &zero, sizeof zero, cudaMemcpyHostToDevice, core_->st);
        cudaMemcpyAsync(&inst_.st->target, &target, sizeof target, cudaMemcpyHostToDevice, core_->st);
        int64_t cap = std::min<int64_t>(limit, INT_MAX - 1 - start);
        if ((size_t)(start + cap) > hist_cap_) grow_hist((size_t)(start + cap));
        set_max_step((int)(start + cap));
        int64_t queued = 0;
        const int64_t chunk = cb ? 1 : 64;
        int reported = start;
        while (queued < cap) {
            int64_t nq = std::min(chunk, cap - queued);
            for (int64_t k = 0; k < nq; ++k) launch_step();
            queued += nq;
            if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
            if (cb && s.step > reported) {
                std::vector<double> h(s.step - reported);
                cudaMemcpy(h.data(), inst_.res_hist + reported, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
                for (size_t k = 0; k < h.size(); ++k) cb(user, (uint64_t)(reported - start + k + 1), h[k]);
                reported = s.step;
            }
            if (s.bad != fused::NO_BAD || s.done || s.step >= start + cap) break;
        }
        *done = s.step - start;
        *res = s.step > start ? s.residual : std::numeric_limits<double>::quiet_NaN();
        if (s.bad != fused::NO_BAD) return report(s.bad, bad);
        return JST_OK;
    }

    void grow_hist(size_t need) {
        size_t cap = hist_cap_;
        while (cap < need) cap *= 2;
        double* h = nullptr;
        if (cudaMalloc(&h, cap * sizeof(double)) != cudaSuccess) return;
        cudaMemcpyAsync(h, inst_.res_hist, hist_cap_ * sizeof(double), cudaMemcpyDeviceToDevice, core_->st);
        if (extra_hist_) cudaFree(extra_hist_);
        extra_hist_ = h;
        inst_.res_hist = h;
        hist_cap_ = cap;
        cudaMemcpyAsync(d_inst_, &inst_, sizeof inst_, cudaMemcpyHostToDevice, core_->st);
        cudaStreamSynchronize(core_->st);
    }

    jst_status residual_terms(double* dt) override {
        // The fused path keeps the residual terms in shared memory only; the
        // time step is available.
        if (dt) return timestep(dt);
        return JST_OK;
    }

    jst_status timestep(double* dt) override {
        launch_step_dt();
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        *dt = s.dt;
        return JST_OK;
    }

    bool get_field(int id, double* out) override {
        SolverCore& C = *core_;
        size_t n = (size_t)C.ni * C.nj;
        if (id == JST_F_LOCALDT && C.local_dt) {
            return cudaMemcpy(out, inst_.ldt, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
        }
        if (id > JST_F_U4) return false;
        if (id >= JST_F_U0) {
            return cudaMemcpy(out, inst_.un[id - JST_F_U0], n * sizeof(double), cudaMemcpyDeviceToHost) ==
                   cudaSuccess;
        }
        InstState s;
        if (read_state(&s) != JST_OK) return false;
        const PhysConst& c = C.c;
        if (s.fresh) {
            double v[9] = {c.f_rho, c.f_p, c.f_t, c.f_vx, c.f_vy, c.f_e, c.f_h, c.f_c, c.f_nut};
            std::fill(out, out + n, v[id]);
            return true;
        }
        std::vector<double> u(5 * n);
        for (int k = 0; k < 5; ++k)
            if (cudaMemcpy(u.data() + k * n, inst_.un[k], n * sizeof(double), cudaMemcpyDeviceToHost) !=
                cudaSuccess)
                return false;
        for (size_t q = 0; q < n; ++q) {
            // solver.rs:158-181
            double rho = u[q], inv = 1.0 / rho;
            double vx = u[n + q] * inv, vy = u[2 * n + q] * inv, e = u[3 * n + q] * inv;
            double p = c.gm1 * (u[3 * n + q] - rho * (vx * vx + vy * vy) * 0.5);
            double t = p / (c.r_gas * rho);
            double v;
            switch (id) {
                case JST_F_RHO: v = rho; break;
                case JST_F_P: v = p; break;
                case JST_F_T: v = t; break;
                case JST_F_U: v = vx; break;
                case JST_F_V: v = vy; break;
                case JST_F_E: v = e; break;
                case JST_F_H: v = e + p * inv; break;
                case JST_F_C: v = std::sqrt(c.rg * t); break;
                default: v = u[4 * n + q] * inv; break;
            }
            out[q] = v;
        }
        return true;
    }

    jst_status set_conserved(const double* u5, jst_nonphysical* bad) override {
        SolverCore& C = *core_;
        size_t n = (size_t)C.ni * C.nj;
        for (int k = 0; k < 5; ++k)
            cudaMemcpyAsync(inst_.un[k], u5 + k * n, n * sizeof(double), cudaMemcpyHostToDevice, C.st);
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        int zero = 0;
        cudaMemcpyAsync(&inst_.st->fresh, &zero, sizeof zero, cudaMemcpyHostToDevice, C.st);
        cudaStreamSynchronize(C.st);
        for (size_t q = 0; q < n; ++q) {
            double u[5] = {u5[q], u5[n + q], u5[2 * n + q], u5[3 * n + q], u5[4 * n + q]};
            double rho = u[0];
            bool b = std::isnan(rho) || rho <= 1e-15;
            if (!b) {
                double inv = 1.0 / rho, vx = u[1] * inv, vy = u[2] * inv;
                double p = C.c.gm1 * (u[3] - rho * (vx * vx + vy * vy) * 0.5);
                b = std::isnan(p) || p <= 1e-15;
            }
            if (b) {
                nonphysical_report(C.c, (long)(q / C.nj), (long)(q % C.nj), u, bad);
                return JST_ERR_NONPHYSICAL;
            }
        }
        launch_step_dt();
        return cudaStreamSynchronize(C.st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    jst_status wall_force(double* fx, double* fy) override {
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        JST_LAUNCH(k_wall_force, 1, 256, 0, core_->st, core_->g, (const double* const*)d_unptr_, core_->c, s.fresh,
                   d_force_);
        double f[2];
        cudaMemcpyAsync(f, d_force_, sizeof f, cudaMemcpyDeviceToHost, core_->st);
        if (cudaStreamSynchronize(core_->st) != cudaSuccess) return JST_ERR_CUDA;
        *fx = f[0];
        *fy = f[1];
        return JST_OK;
    }

    jst_status residual(double* out) override {
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        *out = s.residual;
        return JST_OK;
    }

    jst_status totaltime(double* out) override {
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        *out = s.totaltime;
        return JST_OK;
    }

    cudaStream_t stream() const override { return core_->st; }

    // nsteps graph-replayed steps with the target disabled, timed with CUDA
    // events on the solver stream; optionally one more step stage by stage.
    jst_status time_steps(int nsteps, double* ms, double* stage_ms) override {
        cudaStream_t st = core_->st;
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        double never = -1.0;
        int zero = 0;
        cudaMemcpyAsync(&inst_.st->target, &never, sizeof never, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(&inst_.st->done, &zero, sizeof zero, cudaMemcpyHostToDevice, st);
        int total = nsteps + (stage_ms ? 1 : 0);
        if ((size_t)(s.step + total) > hist_cap_) grow_hist((size_t)(s.step + total));
        set_max_step(s.step + total);
        ensure_graph();
        cudaEvent_t ev[8];  // 0,1: around the steps; 2..7: stage boundaries of the extra step
        for (auto& e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[0], st);
        for (int q = 0; q < nsteps; ++q) launch_step();
        cudaEventRecord(ev[1], st);
        if (stage_ms) {
            cudaEventRecord(ev[2], st);
            for (int q = 0; q < 5; ++q) {
                auto kern = q == 0 ? K_.stage[0] : (q == 4 ? K_.stage[2] : K_.stage[1]);
                JST_LAUNCH(kern, ntiles_, K_.nt, K_.smem, st, d_tiles_, d_inst_, q, RK_ALPHA[q]);
                cudaEventRecord(ev[3 + q], st);
            }
        }
        if (cudaEventSynchronize(stage_ms ? ev[7] : ev[1]) != cudaSuccess) return JST_ERR_CUDA;
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        *ms = t;
        if (stage_ms)
            for (int q = 0; q < 5; ++q) {
                float tq = 0.f;
                cudaEventElapsedTime(&tq, ev[2 + q], ev[3 + q]);
                stage_ms[q] = tq;
            }
        for (auto& e : ev) cudaEventDestroy(e);
        cudaMemcpyAsync(&inst_.st->target, &core_->targetres, sizeof(double), cudaMemcpyHostToDevice, st);
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        if (s.bad != fused::NO_BAD) return JST_ERR_NONPHYSICAL;
        return JST_OK;
    }

  private:
    SolverCore* core_;
    Kernels<T> K_;
    int ti_ = 8, tj_ = 32, ntiles_ = 0;
    void* arena_ = nullptr;
    double* extra_hist_ = nullptr;
    size_t hist_cap_ = 0;
    Inst<T> inst_{};
    Inst<T>* d_inst_ = nullptr;
    TileRef* d_tiles_ = nullptr;
    double* d_force_ = nullptr;
    double** d_unptr_ = nullptr;
    InstState* h_state_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
};

Engine* make_fused_engine(SolverCore* core, std::string& err) {
    if (core->opts.precision == JST_PREC_FP64) {
        auto* e = new FusedEngine<double>(core);
        if (!e->create(err)) {
            delete e;
            return nullptr;
        }
        return e;
    }
    auto* e = new FusedEngine<float>(core);
    if (!e->create(err)) {
        delete e;
        return nullptr;
    }
    return e;
}

}  // namespace jst
