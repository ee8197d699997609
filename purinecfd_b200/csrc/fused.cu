// Host side of the fused tiled path: one stage kernel per RK stage over a
// tile table, the 5 stages of a step captured once as a CUDA graph, and a
// device-side step counter / convergence flag so that many steps can be
// queued without a host round trip per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include <chrono>
#include <deque>
#include <map>
#include <mutex>
#include <tuple>

#include "config_mesh.h"
#include "engine.h"
#include "fused_kernels.cuh"
#include "march_kernels.cuh"
#include "march2_kernels.cuh"

namespace jst {

using fused::Inst;
using fused::InstState;
using fused::TileRef;

namespace {

// Initial state: U_n = pack(free stream) on every cell (state.rs:174-190).
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
struct UnPtrs {
    const double* u[5];
};

__global__ void k_wall_force(Geom g, UnPtrs un_p, PhysConst c, int fresh, double* out) {
    const double* const* un = un_p.u;
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

void launch_wall_force(const Geom& g, const UnPtrs& up, const PhysConst& c, double* out, cudaStream_t st) {
    JST_LAUNCH(k_wall_force, 1, 256, 0, st, g, up, c, 0, out);
}

// Tile configurations compiled into the library: (TI, TJ, NT).
#define JST_FOR_TILES(X) X(4, 32, 256) X(8, 32, 256) X(16, 32, 256) X(4, 64, 256) X(8, 64, 256) X(8, 32, 192) X(8, 32, 128) X(16, 32, 384)
// Marching-strip configurations: threads per block.  A strip is
// fused::MARCH_W = 26 columns wide, so these are selected by tile_j == 26;
// tile_i is the (maximum) strip height, a run-time choice.  The paired-column
// strips of the split precision (k_march2) are fused::MARCH2_W = 56 columns
// wide: tile_j == 56.
#define JST_FOR_MARCH(X) X(64) X(128) X(256)
#define JST_FOR_MARCH2(X) X(64) X(128)

// Strip width of a strip configuration (0 for a tile configuration).
inline int strip_width(int tj) { return tj == fused::MARCH_W || tj == fused::MARCH2_W ? tj : 0; }

template <class T> struct Kernels {
    void (*stage[3])(const TileRef*, int*, const Inst<T>*, int, double) = {nullptr, nullptr, nullptr};
    void (*step_dt)(const TileRef*, const int*, const Inst<T>*, int, int) = nullptr;
    // stage 0 writing the residual of every cell to Inst::rdump (jst_stage_residual)
    void (*dump)(const TileRef*, int*, const Inst<T>*, int, double) = nullptr;
    // single-instance marching strips (per-lane staging): the same stages with
    // the instance descriptor passed by value (k_march_solo)
    void (*solo[3])(const TileRef*, int*, int, double, Inst<T>) = {nullptr, nullptr, nullptr};
    size_t smem = 0;
    int nt = 256;
    bool march = false;  // warp per work item (else block per tile)
    int staging = 0;     // marching strips: 0 per-lane cp.async, 1 bulk (TMA) row copies
};

template <class T, int TI, int TJ, int NT> Kernels<T> kernels_for() {
    Kernels<T> k;
    k.stage[0] = fused::k_stage<T, TI, TJ, NT, true, false>;
    k.stage[1] = fused::k_stage<T, TI, TJ, NT, false, false>;
    k.stage[2] = fused::k_stage<T, TI, TJ, NT, false, true>;
    k.dump = fused::k_stage<T, TI, TJ, NT, true, false, true>;
    k.step_dt = fused::k_step_dt<T, NT>;
    k.smem = fused::Layout<T, TI, TJ, NT>::bytes;
    k.nt = NT;
    return k;
}

template <class T, int NT, int STG = 0> Kernels<T> march_kernels_for() {
    constexpr bool PIPE = true;
    Kernels<T> k;
    k.stage[0] = fused::k_march<T, NT, true, false, PIPE, false, STG>;
    k.stage[1] = fused::k_march<T, NT, false, false, PIPE, false, STG>;
    k.stage[2] = fused::k_march<T, NT, false, true, PIPE, false, STG>;
    k.dump = fused::k_march<T, NT, true, false, PIPE, true, STG>;
    if constexpr (STG == 0) {
        k.solo[0] = fused::k_march_solo<T, NT, true, false>;
        k.solo[1] = fused::k_march_solo<T, NT, false, false>;
        k.solo[2] = fused::k_march_solo<T, NT, false, true>;
    }
    k.step_dt = fused::k_step_dt<T, NT>;
    k.smem = fused::march_smem_bytes<T, NT, PIPE, STG>();
    k.nt = NT;
    k.march = true;
    k.staging = STG;
    return k;
}

template <class T, int NT> Kernels<T> march2_kernels_for() {
    Kernels<T> k;
    if constexpr (std::is_same<T, float>::value) {
        k.stage[0] = fused::k_march2<NT, true, false>;
        k.stage[1] = fused::k_march2<NT, false, false>;
        k.stage[2] = fused::k_march2<NT, false, true>;
        k.dump = fused::k_march2<NT, true, false, true>;
        k.step_dt = fused::k_step_dt<T, NT>;
        k.smem = fused::march2_smem_bytes<NT>();
        k.nt = NT;
        k.march = true;
    }
    return k;
}

// staging (marching strips only): 0 per-lane cp.async, 1 bulk row copies
template <class T> bool pick_kernels(int ti, int tj, Kernels<T>* out, int nt = 256, int staging = 0) {
#define JST_PICK(a, b, n)                               \
    if (ti == a && tj == b && nt == n) {                \
        *out = kernels_for<T, a, b, n>();               \
        return true;                                    \
    }
    JST_FOR_TILES(JST_PICK)
#undef JST_PICK
#define JST_PICK_MARCH(n)                                           \
    if (ti >= 4 && ti <= 1024 && tj == fused::MARCH_W && nt == n) { \
        *out = staging == 1 ? march_kernels_for<T, n, 1>() : march_kernels_for<T, n>(); \
        return true;                                                \
    }
    JST_FOR_MARCH(JST_PICK_MARCH)
#undef JST_PICK_MARCH
    if constexpr (std::is_same<T, float>::value) {
#define JST_PICK_MARCH2(n)                                           \
    if (ti >= 4 && ti <= 1024 && tj == fused::MARCH2_W && nt == n) { \
        *out = march2_kernels_for<T, n>();                           \
        return true;                                                 \
    }
        JST_FOR_MARCH2(JST_PICK_MARCH2)
#undef JST_PICK_MARCH2
    }
    return false;
}

template <class T> void build_march_geom(const Geom& g, int ni, int nj, T* rec, cudaStream_t st) {
    long n = (long)(ni + 1) * nj;
    JST_LAUNCH(fused::k_march_geom<T>, (unsigned)((n + 255) / 256), 256, 0, st, g.tnx, g.tny, g.nnx, g.nny, g.inv_vol,
               g.inv_d2, g.vol, ni, nj, rec);
}

// Bytes of the paired-column geometry records (split precision only).
template <class T> size_t march2_geom_bytes(int ni, int nj) {
    return std::is_same<T, float>::value ? (size_t)(ni + 1) * fused::mg2_pairs(nj) * fused::M2_N * sizeof(float) : 0;
}

void build_march_geom2(const Geom& g, int ni, int nj, float* rec, cudaStream_t st) {
    long n = (long)(ni + 1) * fused::mg2_pairs(nj);
    JST_LAUNCH(fused::k_march_geom2, (unsigned)((n + 255) / 256), 256, 0, st, g.tnx, g.tny, g.nnx, g.nny, g.inv_vol,
               g.inv_d2, g.vol, ni, nj, rec);
}

// Grid of a stage launch over `items` work items: one block per tile for the
// tile kernels; for the marching kernels enough blocks to give every strip a
// warp, at most the resident limit (warps take strips from a work counter).
template <class T> int stage_grid(const Kernels<T>& K, int items, int resident_blocks) {
    if (!K.march) return std::max(1, items);
    int wpb = K.nt / 32;
    int need = (items + wpb - 1) / wpb;
    return std::max(1, std::min(need, std::max(1, resident_blocks)));
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

// Tile configurations the autotuner times, in order (TI, TJ, threads).
// Marching candidates are (maximum strip height, 26, threads); the tile
// configurations kept here are the ones that were ever fastest on some mesh.
const int kTileCands[][3] = {{4, 32, 256}, {8, 32, 256}, {16, 32, 256}, {16, 26, 64},
                             {32, 26, 64}, {48, 26, 64}, {64, 26, 64},  {32, 26, 128}};

// Below this many cells the autotuner times a short list: on small meshes a
// stage is latency-bound and small tiles win (the marching kernel's row walk
// cannot be hidden behind other strips), and the first use of every
// candidate's kernels costs more than a small solve.
constexpr long kTuneMinCells = 262144;
const int kSmallCands[][3] = {{4, 32, 256}, {8, 32, 256}, {16, 32, 256}};

// Stage input buffer = T copy of U_n, so a middle stage can be timed without
// touching the solution.
template <class T> __global__ void k_copy_state(Inst<T> I, long n) {
    long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    for (int k = 0; k < 5; ++k) I.ua[k][id] = (T)I.un[k][id];
}

struct TuneResult {
    int ti, tj, nt;
    float ms;
    int staging = 0;
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, TuneResult> g_tune_cache;

std::vector<TileRef> make_tiles(int inst, int ni, int nj, int ti, int tj) {
    std::vector<TileRef> t;
    int a_n = (ni + ti - 1) / ti, b_n = (nj + tj - 1) / tj;
    t.reserve((size_t)a_n * b_n);
    for (int a = 0; a < a_n; ++a) {
        // marching strips: a_n bands of nearly equal height, at most ti rows
        // (k_step_dt walks TI rows of each work item)
        int i0 = strip_width(tj) ? (int)((long)a * ni / a_n) : a * ti;
        int i1 = strip_width(tj) ? (int)((long)(a + 1) * ni / a_n) : std::min(a * ti + ti, ni);
        for (int b = 0; b < b_n; ++b) t.push_back(TileRef{inst, i0, b * tj, a * b_n + b, i1});
    }
    return t;
}

// Most work items any configuration the autotuner may pick cuts an NI x NJ
// mesh into (the fixed candidates, and strips of the smallest modelled height).
int tuned_tiles_bound(int ni, int nj) {
    int m = ((ni + 7) / 8) * ((nj + fused::MARCH_W - 1) / fused::MARCH_W);
    for (const auto& cd : kTileCands) m = std::max(m, ((ni + cd[0] - 1) / cd[0]) * ((nj + cd[1] - 1) / cd[1]));
    for (const auto& cd : kSmallCands) m = std::max(m, ((ni + cd[0] - 1) / cd[0]) * ((nj + cd[1] - 1) / cd[1]));
    return m;
}

// Strip height for the marching kernels from a wave model: warps take strips
// from a counter, so a launch lasts about ceil(strips / resident warps)
// strip walks of (rows + 6) rows each.  Returns the height in [8, 128] that
// minimises that over the given instances (nearly equal bands per instance).
int march_height(const std::vector<std::pair<int, std::pair<int, int>>>& insts, long resident_warps,
                 int width = fused::MARCH_W) {
    int best_h = 32;
    double best = 1e300;
    for (int h = 8; h <= 128; ++h) {
        long strips = 0;
        double rows = 0.0;
        for (const auto& in : insts) {
            long cols = (in.second.second + width - 1) / width;
            long bands = (in.second.first + h - 1) / h;
            strips += bands * cols;
            rows += (double)in.second.first * cols;
        }
        if (strips == 0) return best_h;
        long waves = (strips + resident_warps - 1) / std::max(1L, resident_warps);
        double cost = (double)waves * (rows / (double)strips + 6.0);
        if (cost < best) {
            best = cost;
            best_h = h;
        }
    }
    return best_h;
}

// The marching configuration of strip width `width` (26: k_march, 56:
// k_march2) the wave model picks for the given instances (64 threads per
// block), without timing anything.
template <class T>
TuneResult model_choice(const std::vector<std::pair<int, std::pair<int, int>>>& insts, int width = fused::MARCH_W) {
    TuneResult r{32, width, 64, 0.f};
    Kernels<T> K;
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (pick_kernels<T>(32, width, &K, 64) &&
        cudaFuncSetAttribute(K.stage[1], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K.stage[1], K.nt, K.smem) == cudaSuccess)
        r.ti = march_height(insts, (long)sms * std::max(1, occ) * (K.nt / 32), width);
    cudaGetLastError();
    return r;
}

long total_cells(const std::vector<std::pair<int, std::pair<int, int>>>& insts) {
    long n = 0;
    for (const auto& in : insts) n += (long)in.second.first * in.second.second;
    return n;
}

// Times one middle-stage launch per candidate over the given instances
// (their U_a must hold a valid state) and returns the fastest configuration.
template <class T>
TuneResult autotune(const std::vector<std::pair<int, std::pair<int, int>>>& insts, Inst<T>* d_insts,
                    InstState* d_states, int nstates, cudaStream_t st, int grid_hint, const Inst<T>* h_solo = nullptr) {
    TuneResult best{8, 32, 256, 1e30f};
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    TileRef* d_t = nullptr;
    int* d_n = nullptr;
    size_t cap = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<std::array<int, 4>> cands;  // (ti, tj, threads, staging)
    const TuneResult m = model_choice<T>(insts);
    if (total_cells(insts) < kTuneMinCells) {
        for (const auto& cd : kSmallCands) cands.push_back({cd[0], cd[1], cd[2], 0});
        cands.push_back({m.ti, m.tj, 64, 0});
    } else {
        for (const auto& cd : kTileCands) cands.push_back({cd[0], cd[1], cd[2], 0});
        cands.push_back({m.ti, m.tj, 64, 0});
        cands.push_back({m.ti, m.tj, 128, 0});
        // the same strips with bulk (TMA) row staging
        cands.push_back({m.ti, m.tj, 64, 1});
        cands.push_back({m.ti, m.tj, 128, 1});
    }
    if (std::is_same<T, float>::value) {  // paired-column strips
        const TuneResult m2 = model_choice<T>(insts, fused::MARCH2_W);
        cands.push_back({m2.ti, m2.tj, 64, 0});
        if (total_cells(insts) >= kTuneMinCells) cands.push_back({m2.ti, m2.tj, 128, 0});
    }
    for (const auto& cand : cands) {
        Kernels<T> K;
        if (!pick_kernels<T>(cand[0], cand[1], &K, cand[2], cand[3])) continue;
        const bool solo = h_solo && K.solo[1];  // time the kernel a single solve runs
        if (cudaFuncSetAttribute(K.stage[1], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem) != cudaSuccess ||
            (solo && cudaFuncSetAttribute(K.solo[1], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem) !=
                         cudaSuccess)) {
            cudaGetLastError();
            continue;
        }
        std::vector<TileRef> tiles;
        for (const auto& in : insts) {
            auto t = make_tiles(in.first, in.second.first, in.second.second, cand[0], cand[1]);
            tiles.insert(tiles.end(), t.begin(), t.end());
        }
        if (tiles.size() > cap) {
            if (d_t) cudaFree(d_t);
            cap = tiles.size();
            cudaMalloc(&d_t, cap * sizeof(TileRef) + 256);
            if (!d_n) {
                cudaMalloc(&d_n, 4 * sizeof(int));  // strip count + the marching kernels' work counters
                cudaMemsetAsync(d_n, 0, 4 * sizeof(int), st);
            }
        }
        int nt_ = (int)tiles.size();
        cudaMemcpyAsync(d_t, tiles.data(), tiles.size() * sizeof(TileRef), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_n, &nt_, sizeof(int), cudaMemcpyHostToDevice, st);
        int occ = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K.stage[1], K.nt, K.smem);
        int grid = K.march ? stage_grid(K, nt_, sms * std::max(1, occ))
                           : (grid_hint > 0 ? std::min(nt_, sms * std::max(1, occ)) : nt_);
        auto launch = [&]() {
            if (solo) JST_LAUNCH(K.solo[1], grid, K.nt, K.smem, st, d_t, d_n, 1, RK_ALPHA[1], *h_solo);
            else JST_LAUNCH(K.stage[1], grid, K.nt, K.smem, st, d_t, d_n, d_insts, 1, RK_ALPHA[1]);
        };
        launch();  // warm-up
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3; ++r) launch();
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best.ms) best = TuneResult{cand[0], cand[1], cand[2], ms, cand[3]};
    }
    // undo any NonPhysical flag the timing launches may have raised
    std::vector<InstState> hs(nstates);
    cudaMemcpy(hs.data(), d_states, nstates * sizeof(InstState), cudaMemcpyDeviceToHost);
    for (auto& x : hs) x.bad = fused::NO_BAD;
    cudaMemcpy(d_states, hs.data(), nstates * sizeof(InstState), cudaMemcpyHostToDevice);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (d_t) cudaFree(d_t);
    if (d_n) cudaFree(d_n);
    return best;
}

}  // namespace

// One primitive field of U_n (Solver::unpack, solver.rs:158-181) on the
// device, so that a field read copies one plane instead of five.  The _rn
// intrinsics keep the reference's separate roundings (no FMA contraction).
__global__ void k_prim_field(UnPtrs un, long n, int id, PhysConst c, double* out) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    double rho = un.u[0][q], inv = 1.0 / rho;
    double vx = __dmul_rn(un.u[1][q], inv), vy = __dmul_rn(un.u[2][q], inv);
    double e = __dmul_rn(un.u[3][q], inv);
    double ke = __dmul_rn(__dmul_rn(rho, __dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy))), 0.5);
    double p = __dmul_rn(c.gm1, __dsub_rn(un.u[3][q], ke));
    double t = p / __dmul_rn(c.r_gas, rho);
    double v;
    switch (id) {
        case JST_F_RHO: v = rho; break;
        case JST_F_P: v = p; break;
        case JST_F_T: v = t; break;
        case JST_F_U: v = vx; break;
        case JST_F_V: v = vy; break;
        case JST_F_E: v = e; break;
        case JST_F_H: v = __dadd_rn(e, __dmul_rn(p, inv)); break;
        case JST_F_C: v = sqrt(__dmul_rn(c.rg, t)); break;
        default: v = __dmul_rn(un.u[4][q], inv); break;
    }
    out[q] = v;
}

template <class T> class FusedEngine : public Engine {
  public:
    explicit FusedEngine(SolverCore* core) : core_(core) {}
    ~FusedEngine() override {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (rdump_) cudaFree(rdump_);
        if (arena_) cudaFree(arena_);
        if (h_state_) cudaFreeHost(h_state_);
    }

    bool select_kernels(int ti, int tj, int nt, std::string& err, int staging = 0) {
        if (!pick_kernels<T>(ti, tj, &K_, nt, staging)) {
            err = "unsupported tile shape " + std::to_string(ti) + "x" + std::to_string(tj) + "x" + std::to_string(nt);
            return false;
        }
        for (int k = 0; k < 4; ++k)
            if (cudaFuncSetAttribute(k < 3 ? K_.stage[k] : K_.dump, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)K_.smem) != cudaSuccess ||
                (k < 3 && K_.solo[k] &&
                 cudaFuncSetAttribute(K_.solo[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K_.smem) !=
                     cudaSuccess)) {
                err = "stage kernel needs " + std::to_string(K_.smem) + " bytes of shared memory";
                return false;
            }
        int dev = 0, sms = 148, occ = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K_.stage[1], K_.nt, K_.smem);
        resident_ = sms * std::max(1, occ);
        ti_ = ti;
        tj_ = tj;
        return true;
    }

    int sgrid() const { return stage_grid(K_, ntiles_, resident_); }

    bool create(std::string& err) {
        SolverCore& C = *core_;
        int ti = C.opts.tile_i, tj = C.opts.tile_j, nt = C.opts.block_threads > 0 ? C.opts.block_threads : 256;
        tune_ = ti <= 0 || tj <= 0;
        if (tune_) {
            default_tile(C.opts.precision, C.nj, &ti, &tj);
            nt = 256;
        }
        if (!select_kernels(ti, tj, nt, err, C.opts.staging == JST_STAGING_BULK ? 1 : 0)) return false;
        int ni = C.ni, nj = C.nj;
        std::vector<TileRef> tiles = make_tiles(0, ni, nj, ti, tj);
        ntiles_ = (int)tiles.size();
        int max_tiles = ntiles_;  // the autotuner may pick a smaller tile
        if (tune_) max_tiles = std::max(max_tiles, tuned_tiles_bound(ni, nj));
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
        size_t o_uc = add(sizeof(T) == sizeof(double) ? 0 : 5 * n * sizeof(T));
        size_t o_ratio = add(2 * n * sizeof(T));
        size_t o_ldt = add(n * sizeof(double));
        size_t o_partial = add(2 * (size_t)max_tiles * sizeof(double));
        size_t o_far = add(5 * (size_t)nj * sizeof(double));
        size_t o_st = add(sizeof(InstState));
        size_t o_inst = add(sizeof(Inst<T>));
        size_t o_tiles = add((size_t)max_tiles * sizeof(TileRef));
        size_t o_force = add(8 * sizeof(double));
        size_t o_ntiles = add(sizeof(int));
        size_t o_unptr = add(5 * sizeof(double*));
        hist_cap_ = 4096;
        size_t o_hist = add(hist_cap_ * sizeof(double));
        size_t o_field = add(n * sizeof(double));
        size_t o_mg = add((size_t)(ni + 1) * nj * fused::MG_N * sizeof(T));
        size_t o_mg2 = add(march2_geom_bytes<T>(ni, nj));
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
            I.uc[k] = sizeof(T) == sizeof(double) ? nullptr : reinterpret_cast<T*>(base + o_uc) + k * n;
        }
        I.ratio[0] = reinterpret_cast<T*>(base + o_ratio);
        I.ratio[1] = I.ratio[0] + n;
        I.ldt = reinterpret_cast<double*>(base + o_ldt);
        I.partial = reinterpret_cast<double*>(base + o_partial);
        I.res_hist = reinterpret_cast<double*>(base + o_hist);
        I.st = reinterpret_cast<InstState*>(base + o_st);
        I.c = C.c;
        I.cp = fused::make_constp(C.c);
        inst_ = I;
        d_inst_ = reinterpret_cast<Inst<T>*>(base + o_inst);
        d_tiles_ = reinterpret_cast<TileRef*>(base + o_tiles);
        d_force_ = reinterpret_cast<double*>(base + o_force);
        d_ntiles_ = reinterpret_cast<int*>(base + o_ntiles);
        d_unptr_ = reinterpret_cast<double**>(base + o_unptr);
        d_field_ = reinterpret_cast<double*>(base + o_field);
        inst_.mg = reinterpret_cast<T*>(base + o_mg);
        inst_.mg2 = march2_geom_bytes<T>(ni, nj) ? reinterpret_cast<float*>(base + o_mg2) : nullptr;
        upload_inst(C.st);
        cudaMemcpyAsync(d_tiles_, tiles.data(), tiles.size() * sizeof(TileRef), cudaMemcpyHostToDevice, C.st);
        cudaMemcpyAsync(d_ntiles_, &ntiles_, sizeof(int), cudaMemcpyHostToDevice, C.st);
        cudaMemcpyAsync(d_unptr_, inst_.un, 5 * sizeof(double*), cudaMemcpyHostToDevice, C.st);
        if (cudaMallocHost(&h_state_, 3 * sizeof(InstState)) != cudaSuccess) {
            err = "cudaMallocHost failed";
            return false;
        }
        JST_LAUNCH(k_far_geom, (nj + 255) / 256, 256, 0, C.st, C.g, const_cast<double*>(inst_.far));
        build_march_geom(C.g, ni, nj, const_cast<T*>(inst_.mg), C.st);
        if (inst_.mg2) build_march_geom2(C.g, ni, nj, const_cast<float*>(inst_.mg2), C.st);
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
        s.drop = 0.0;
        s.res_first = 0.0;
        cudaMemcpyAsync(inst_.st, &s, sizeof s, cudaMemcpyHostToDevice, core_->st);
        cudaStreamSynchronize(core_->st);
    }

    void init() override {
        SolverCore& C = *core_;
        long n = (long)C.ni * C.nj;
        JST_LAUNCH(k_fill_freestream, (unsigned)((n + 255) / 256), 256, 0, C.st, inst_.un[0], inst_.un[1],
                   inst_.un[2], inst_.un[3], inst_.un[4], n, C.c);
        reset_state(1);
        launch_step_dt();
        if (tune_) tune();
    }

    // Autotuner: time every compiled tile configuration on this mesh (one
    // middle-stage launch on a copy of the state each) and keep the fastest;
    // the choice is cached per (precision, NI, NJ, time-step mode).
    void tune() {
        SolverCore& C = *core_;
        auto key = std::make_tuple((int)sizeof(T), C.ni, C.nj, C.local_dt);
        TuneResult r{};
        bool have = false;
        {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tune_cache.find(key);
            if (it != g_tune_cache.end()) {
                r = it->second;
                have = true;
            }
        }
        if (!have) {
            long n = (long)C.ni * C.nj;
            JST_LAUNCH(k_copy_state<T>, (unsigned)((n + 255) / 256), 256, 0, C.st, inst_, n);
            r = autotune<T>({{0, {C.ni, C.nj}}}, d_inst_, inst_.st, 1, C.st, 0, &inst_);
            std::lock_guard<std::mutex> lock(g_tune_mu);
            g_tune_cache[key] = r;
        }
        std::string err;
        // a staging the options ask for overrides the tuner's
        int stg = C.opts.staging == JST_STAGING_BULK ? 1 : (C.opts.staging == JST_STAGING_PER_LANE ? 0 : r.staging);
        if (!select_kernels(r.ti, r.tj, r.nt, err, stg)) return;
        std::vector<TileRef> tiles = make_tiles(0, C.ni, C.nj, r.ti, r.tj);
        ntiles_ = (int)tiles.size();
        inst_.ntiles = ntiles_;
        upload_inst(C.st);
        cudaMemcpyAsync(d_tiles_, tiles.data(), tiles.size() * sizeof(TileRef), cudaMemcpyHostToDevice, C.st);
        cudaMemcpyAsync(d_ntiles_, &ntiles_, sizeof(int), cudaMemcpyHostToDevice, C.st);
        reset_state(1);
        launch_step_dt();
        cudaStreamSynchronize(C.st);
    }

  public:
    void kernel_config(int* ti, int* tj, int* nt) const override {
        *ti = ti_;
        *tj = tj_;
        *nt = K_.nt;
    }
    int kernel_staging() const override { return K_.march ? (K_.staging == 1 ? JST_STAGING_BULK : JST_STAGING_PER_LANE) : 0; }

    // test hook: bytes the bulk row barrier expects beyond those copied
    void set_stage_extra_tx(int bytes) override {
        inst_.stage_extra_tx = bytes;
        upload_inst(core_->st);
        cudaStreamSynchronize(core_->st);
    }

    void launch_step_dt() {
        JST_LAUNCH(K_.step_dt, ntiles_, K_.nt, 0, core_->st, d_tiles_, d_ntiles_, d_inst_, ti_, tj_);
    }

    // RK stage s (0..4); the marching strips take the instance descriptor by
    // value (a captured graph holds the value, so every change of inst_
    // goes through upload_inst, which drops the graph)
    void launch_stage(int s, cudaStream_t st) {
        const int k = s == 0 ? 0 : (s == 4 ? 2 : 1);
        if (K_.solo[k]) JST_LAUNCH(K_.solo[k], sgrid(), K_.nt, K_.smem, st, d_tiles_, d_ntiles_, s, RK_ALPHA[s], inst_);
        else JST_LAUNCH(K_.stage[k], sgrid(), K_.nt, K_.smem, st, d_tiles_, d_ntiles_, d_inst_, s, RK_ALPHA[s]);
    }

    void enqueue_step(cudaStream_t st) {
        for (int s = 0; s < 5; ++s) launch_stage(s, st);
    }

    // Copies inst_ to the device (stream-ordered) and drops the captured step
    // graph, whose solo launches hold the previous value.
    void upload_inst(cudaStream_t st) {
        cudaMemcpyAsync(d_inst_, &inst_, sizeof inst_, cudaMemcpyHostToDevice, st);
        if (graph_exec_) {
            cudaStreamSynchronize(st);
            cudaGraphExecDestroy(graph_exec_);
            graph_exec_ = nullptr;
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
        if (s.err) return JST_ERR_TIMEOUT;
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
        if (cb) return run_with_callback(start, cap, cb, user, done, res, bad);
        int64_t queued = 0;
        const int64_t chunk = 64;
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
            if (s.bad != fused::NO_BAD || s.done || s.err || s.step >= start + cap) break;
        }
        *done = s.step - start;
        *res = s.step > start ? s.residual : std::numeric_limits<double>::quiet_NaN();
        if (s.err) return JST_ERR_TIMEOUT;
        if (s.bad != fused::NO_BAD) return report(s.bad, bad);
        return JST_OK;
    }

    // The run loop with a per-step callback: one RK step stays queued ahead of
    // the host, which reads the previous step's scalars from pinned memory
    // (copied on the stream right after that step) and calls back in order;
    // a step queued past convergence, NonPhysical or the limit is skipped on
    // the device.
    jst_status run_with_callback(int start, int64_t cap, jst_step_cb cb, void* user, int64_t* done, double* res,
                                 jst_nonphysical* bad) {
        cudaStream_t st = core_->st;
        InstState* slot[2] = {h_state_ + 1, h_state_ + 2};
        cudaEvent_t ev[2];
        for (auto& e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        auto enqueue = [&](int64_t q) {
            launch_step();
            cudaMemcpyAsync(slot[q & 1], inst_.st, sizeof(InstState), cudaMemcpyDeviceToHost, st);
            cudaEventRecord(ev[q & 1], st);
        };
        jst_status rc = JST_OK;
        int64_t queued = 0;
        int reported = start;
        InstState s{};
        enqueue(queued++);
        for (int64_t q = 0; q < cap; ++q) {
            if (queued < cap) enqueue(queued++);
            if (cudaEventSynchronize(ev[q & 1]) != cudaSuccess) {
                rc = JST_ERR_CUDA;
                break;
            }
            s = *slot[q & 1];
            if (s.step > reported) {
                reported = s.step;
                cb(user, (uint64_t)(reported - start), s.residual);
            }
            if (s.bad != fused::NO_BAD || s.done || s.err || s.step >= start + cap) break;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        InstState fin;
        if (read_state(&fin) != JST_OK) return JST_ERR_CUDA;  // also waits for a step queued ahead
        if (rc != JST_OK) return rc;
        *done = fin.step - start;
        *res = fin.step > start ? fin.residual : std::numeric_limits<double>::quiet_NaN();
        if (fin.err) return JST_ERR_TIMEOUT;
        if (fin.bad != fused::NO_BAD) return report(fin.bad, bad);
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
        upload_inst(core_->st);
        cudaStreamSynchronize(core_->st);
    }

    jst_status residual_terms(double* dt) override {
        // The fused path keeps the residual terms in shared memory only; the
        // time step is available.
        if (dt) return timestep(dt);
        return JST_OK;
    }

    // R = Fc - Fv - Fd - S of every cell of the current state from the stage
    // kernel the RK stages run with (its DUMP instantiation of stage 0), after
    // the time step of the current state, as the first stage of a step sees it.
    jst_status stage_residual(double* out) override {
        SolverCore& C = *core_;
        size_t n = (size_t)C.ni * C.nj;
        if (!rdump_) {
            if (cudaMalloc(&rdump_, 5 * n * sizeof(double)) != cudaSuccess) return JST_ERR_OOM;
            inst_.rdump = rdump_;
            upload_inst(C.st);
        }
        launch_step_dt();
        JST_LAUNCH(K_.dump, sgrid(), K_.nt, K_.smem, C.st, d_tiles_, d_ntiles_, d_inst_, 0, RK_ALPHA[0]);
        if (cudaMemcpyAsync(out, rdump_, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, C.st) != cudaSuccess ||
            cudaStreamSynchronize(C.st) != cudaSuccess)
            return JST_ERR_CUDA;
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
        if (id == JST_F_LOCALDT && C.local_dt) return d2h_staged(C, out, inst_.ldt, n * sizeof(double)) == cudaSuccess;
        if (id > JST_F_U4) return false;
        if (id >= JST_F_U0) return d2h_staged(C, out, inst_.un[id - JST_F_U0], n * sizeof(double)) == cudaSuccess;
        InstState s;
        if (read_state(&s) != JST_OK) return false;
        const PhysConst& c = C.c;
        if (s.fresh) {
            double v[9] = {c.f_rho, c.f_p, c.f_t, c.f_vx, c.f_vy, c.f_e, c.f_h, c.f_c, c.f_nut};
            std::fill(out, out + n, v[id]);
            return true;
        }
        UnPtrs up;
        for (int k = 0; k < 5; ++k) up.u[k] = inst_.un[k];
        JST_LAUNCH(k_prim_field, (unsigned)((n + 255) / 256), 256, 0, core_->st, up, (long)n, id, c, d_field_);
        return d2h_staged(C, out, d_field_, n * sizeof(double)) == cudaSuccess;
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
        UnPtrs up;
        for (int k = 0; k < 5; ++k) up.u[k] = inst_.un[k];
        JST_LAUNCH(k_wall_force, 1, 256, 0, core_->st, core_->g, up, core_->c, s.fresh, d_force_);
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

    jst_status set_totaltime(double t) override {
        cudaMemcpyAsync(&inst_.st->totaltime, &t, sizeof t, cudaMemcpyHostToDevice, core_->st);
        return cudaStreamSynchronize(core_->st) == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    cudaStream_t stream() const override { return core_->st; }

    // nsteps graph-replayed steps with the target disabled, timed with CUDA
    // events on the solver stream; optionally kStageReps more steps, run back
    // to back from one graph with an event recorded before, between and
    // after each step's stage launches, whose mean stage durations go to
    // stage_ms.
    static constexpr int kStageReps = 10;
    jst_status time_steps(int nsteps, double* ms, double* stage_ms) override {
        cudaStream_t st = core_->st;
        InstState s;
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        double never = -1.0;
        int zero = 0;
        cudaMemcpyAsync(&inst_.st->target, &never, sizeof never, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(&inst_.st->done, &zero, sizeof zero, cudaMemcpyHostToDevice, st);
        int total = nsteps + (stage_ms ? kStageReps : 0);
        if ((size_t)(s.step + total) > hist_cap_) grow_hist((size_t)(s.step + total));
        set_max_step(s.step + total);
        ensure_graph();
        cudaEvent_t ev[2 + 6 * kStageReps];  // 0,1: around the steps; then 6 per timed-stage step
        for (auto& e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[0], st);
        for (int q = 0; q < nsteps; ++q) launch_step();
        cudaEventRecord(ev[1], st);
        jst_status rc = JST_OK;
        if (cudaEventSynchronize(ev[1]) != cudaSuccess) rc = JST_ERR_CUDA;
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        *ms = t;
        if (stage_ms && rc == JST_OK) {
            cudaGraph_t g;
            cudaGraphExec_t tg = nullptr;
            cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            for (int r = 0; r < kStageReps; ++r) {
                cudaEvent_t* e = ev + 2 + 6 * r;
                cudaEventRecordWithFlags(e[0], st, cudaEventRecordExternal);
                for (int q = 0; q < 5; ++q) {
                    launch_stage(q, st);
                    cudaEventRecordWithFlags(e[1 + q], st, cudaEventRecordExternal);
                }
            }
            if (cudaStreamEndCapture(st, &g) != cudaSuccess) {
                rc = JST_ERR_CUDA;
            } else {
                if (cudaGraphInstantiate(&tg, g, 0) != cudaSuccess) rc = JST_ERR_CUDA;
                cudaGraphDestroy(g);
            }
            if (rc == JST_OK) {
                cudaGraphLaunch(tg, st);
                if (cudaEventSynchronize(ev[1 + 6 * kStageReps]) != cudaSuccess) rc = JST_ERR_CUDA;
            }
            if (tg) cudaGraphExecDestroy(tg);
            for (int q = 0; q < 5 && rc == JST_OK; ++q) {
                double acc = 0.0;
                for (int r = 0; r < kStageReps; ++r) {
                    float tq = 0.f;
                    cudaEventElapsedTime(&tq, ev[2 + 6 * r + q], ev[3 + 6 * r + q]);
                    acc += tq;
                }
                stage_ms[q] = acc / kStageReps;
            }
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (rc != JST_OK) return rc;
        cudaMemcpyAsync(&inst_.st->target, &core_->targetres, sizeof(double), cudaMemcpyHostToDevice, st);
        if (read_state(&s) != JST_OK) return JST_ERR_CUDA;
        if (s.err) return JST_ERR_TIMEOUT;
        if (s.bad != fused::NO_BAD) return JST_ERR_NONPHYSICAL;
        return JST_OK;
    }

  private:
    SolverCore* core_;
    Kernels<T> K_;
    int ti_ = 8, tj_ = 32, ntiles_ = 0, resident_ = 148;
    bool tune_ = false;
    void* arena_ = nullptr;
    double* extra_hist_ = nullptr;
    double* rdump_ = nullptr;
    size_t hist_cap_ = 0;
    Inst<T> inst_{};
    Inst<T>* d_inst_ = nullptr;
    TileRef* d_tiles_ = nullptr;
    double* d_force_ = nullptr;
    int* d_ntiles_ = nullptr;
    double** d_unptr_ = nullptr;
    double* d_field_ = nullptr;
    InstState* h_state_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
};

// ------------------------------------------------------------------ batch ----
// Many independent solves in one persistent stage kernel.  Each instance owns
// a block of a pre-allocated HBM arena (geometry, state, per-tile partials),
// a slot in the device instance table and its tiles in the device tile
// table; the stage kernels read the table size from device memory, so the
// captured graph of K RK steps stays valid while instances come and go.

namespace {

// First-fit allocator over one cudaMalloc'd arena (offsets in bytes).
struct Arena {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    std::map<size_t, size_t> free_;  // offset -> size
    static size_t round(size_t n) { return (n + 255) / 256 * 256; }
    bool init(size_t bytes) {
        cap = round(bytes);
        if (cudaMalloc(&base, cap) != cudaSuccess) return false;
        free_[0] = cap;
        return true;
    }
    bool alloc(size_t n, size_t* off) {
        n = round(n);
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                *off = it->first;
                size_t rem = it->second - n, o2 = it->first + n;
                free_.erase(it);
                if (rem) free_[o2] = rem;
                used += n;
                return true;
            }
        return false;
    }
    void release(size_t off, size_t n) {
        n = round(n);
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    ~Arena() {
        if (base) cudaFree(base);
    }
};

using Clock = std::chrono::steady_clock;

}  // namespace

struct BatchResultFull {
    jst_batch_result r{};
    std::vector<double> fields;
};

class BatchBase {
  public:
    virtual ~BatchBase() {}
    virtual jst_status submit(const char* cfg, const double* xy, int nr, int nt, int64_t max_steps, double drop,
                              double cl_tol, int64_t* id) = 0;
    virtual jst_status step(int nsteps) = 0;
    virtual void stats(int* active, int* queued, double* bytes) = 0;
    virtual int poll(int64_t* ids, int cap) = 0;
    virtual bool result(int64_t id, BatchResultFull** out) = 0;
    virtual void kernel_config(int* ti, int* tj, int* nt) const = 0;
    virtual int kernel_staging() const = 0;
};

template <class T> class Batch : public BatchBase {
    struct Pending {
        int64_t id;
        RawConfig raw;
        std::vector<double> xy;
        int n_rings, n_theta;
        int64_t max_steps;
        double drop, cl_tol, t_submit;
    };
    struct Slot {
        bool used = false;
        int64_t id = -1;
        size_t off = 0, bytes = 0;
        int ni = 0, nj = 0, ntiles = 0;
        int64_t max_steps = 0;
        double drop = 0, cl_tol = 0, t_submit = 0, t_admit = 0;
        double chord = 1, aoa = 0;
        Geom g{};
        std::vector<std::pair<int, double>> cl_hist;
    };

  public:
    explicit Batch(const jst_batch_opts& o) : o_(o) { t0_ = Clock::now(); }
    ~Batch() override {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (small_) cudaFree(small_);
        if (h_states_) cudaFreeHost(h_states_);
        if (st_) cudaStreamDestroy(st_);
    }

    bool create(std::string& err) {
        if (cudaSetDevice(o_.device) != cudaSuccess) {
            err = "cudaSetDevice failed";
            return false;
        }
        cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
        int ti = o_.tile_i, tj = o_.tile_j, nt = o_.block_threads > 0 ? o_.block_threads : 256;
        tune_ = ti <= 0 || tj <= 0;
        if (tune_) {
            default_tile(o_.precision, 128, &ti, &tj);
            nt = 256;
        }
        if (!select_kernels(ti, tj, nt, o_.staging == JST_STAGING_BULK ? 1 : 0)) {
            err = "unsupported tile shape";
            return false;
        }
        nslots_ = std::max(1, o_.max_instances);
        max_tiles_ = 1 << 22;
        size_t bytes = nslots_ * (sizeof(Inst<T>) + sizeof(InstState) + sizeof(int) + 2 * sizeof(double)) +
                       (size_t)max_tiles_ * sizeof(TileRef) + 4096;
        if (cudaMalloc(&small_, bytes) != cudaSuccess) {
            err = "cudaMalloc failed for the batch tables";
            return false;
        }
        cudaMemset(small_, 0, bytes);
        char* q = static_cast<char*>(small_);
        d_insts_ = reinterpret_cast<Inst<T>*>(q);
        q += nslots_ * sizeof(Inst<T>);
        d_states_ = reinterpret_cast<InstState*>(q);
        q += nslots_ * sizeof(InstState);
        d_force_ = reinterpret_cast<double*>(q);
        q += nslots_ * 2 * sizeof(double);
        d_counts_ = reinterpret_cast<int*>(q);
        q += nslots_ * sizeof(int);
        q = reinterpret_cast<char*>(((uintptr_t)q + 255) / 256 * 256);
        d_ntiles_ = reinterpret_cast<int*>(q);
        q += 256;
        d_tiles_ = reinterpret_cast<TileRef*>(q);
        if (cudaMallocHost(&h_states_, nslots_ * sizeof(InstState)) != cudaSuccess) {
            err = "cudaMallocHost failed";
            return false;
        }
        h_insts_.assign(nslots_, Inst<T>{});
        slots_.assign(nslots_, Slot{});
        size_t budget = (size_t)(o_.hbm_budget_gb * 1e9);
        if (budget == 0) {
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            budget = (size_t)(0.5 * fr);
        }
        if (!arena_.init(budget)) {
            err = "cudaMalloc failed for the instance arena";
            return false;
        }
        int zero = 0;
        cudaMemcpy(d_ntiles_, &zero, sizeof zero, cudaMemcpyHostToDevice);
        return true;
    }

    bool select_kernels(int ti, int tj, int nt, int staging = 0) {
        Kernels<T> K;
        if (!pick_kernels<T>(ti, tj, &K, nt, staging)) return false;
        for (int k = 0; k < 3; ++k)
            if (cudaFuncSetAttribute(K.stage[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem) !=
                cudaSuccess)
                return false;
        K_ = K;
        ti_ = ti;
        tj_ = tj;
        int sms = 0, occ = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o_.device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K_.stage[1], K_.nt, K_.smem);
        grid_ = std::max(1, sms * std::max(1, occ));
        return true;
    }

    // Autotuner over the instances admitted so far (before the graph is
    // captured): every candidate tile configuration times one middle-stage
    // launch over the whole batch; the fastest is kept and all instances are
    // re-tiled with it.
    void tune() {
        tune_ = false;
        std::vector<std::pair<int, std::pair<int, int>>> list;
        for (int k = 0; k < nslots_; ++k)
            if (slots_[k].used) list.push_back({k, {slots_[k].ni, slots_[k].nj}});
        if (list.empty()) return;
        for (const auto& in : list) {
            long n = (long)in.second.first * in.second.second;
            JST_LAUNCH(k_copy_state<T>, (unsigned)((n + 255) / 256), 256, 0, st_, h_insts_[in.first], n);
        }
        TuneResult r = autotune<T>(list, d_insts_, d_states_, nslots_, st_, 1);
        const int stg = o_.staging == JST_STAGING_BULK ? 1 : (o_.staging == JST_STAGING_PER_LANE ? 0 : r.staging);
        if (!select_kernels(r.ti, r.tj, r.nt, stg)) return;
        h_tiles_.clear();
        for (int k = 0; k < nslots_; ++k)
            if (slots_[k].used) {
                auto t = make_tiles(k, slots_[k].ni, slots_[k].nj, ti_, tj_);
                slots_[k].ntiles = (int)t.size();
                h_insts_[k].ntiles = (int)t.size();
                cudaMemcpyAsync(d_insts_ + k, &h_insts_[k], sizeof(Inst<T>), cudaMemcpyHostToDevice, st_);
                h_tiles_.insert(h_tiles_.end(), t.begin(), t.end());
            }
        upload_tiles();
    }

    int max_tiles_for(int ni, int nj) const {
        int m = ((ni + ti_ - 1) / ti_) * ((nj + tj_ - 1) / tj_);
        if (tune_) m = std::max(m, tuned_tiles_bound(ni, nj));
        return m;
    }

    double now() const { return std::chrono::duration<double>(Clock::now() - t0_).count(); }

    jst_status submit(const char* cfg, const double* xy, int nr, int nt, int64_t max_steps, double drop,
                      double cl_tol, int64_t* id) override {
        Pending p;
        std::string err;
        if (!parse_config(cfg, p.raw, err)) {
            set_call_error(err);
            return JST_ERR_CONFIG;
        }
        if (p.raw.halo < 3) {
            set_call_error("simulation.IM must be >= 3");
            return JST_ERR_CONFIG;
        }
        p.xy.assign(xy, xy + 2 * (size_t)nr * nt);
        // trim_closing_duplicate (mesh.rs:169-189)
        bool closed = nt >= 2;
        for (int r = 0; r < nr && closed; ++r)
            closed = std::fabs(p.xy[2 * ((size_t)r * nt)] - p.xy[2 * ((size_t)r * nt + nt - 1)]) <= 1e-10 &&
                     std::fabs(p.xy[2 * ((size_t)r * nt) + 1] - p.xy[2 * ((size_t)r * nt + nt - 1) + 1]) <= 1e-10;
        if (closed) {
            std::vector<double> t(2 * (size_t)nr * (nt - 1));
            for (int r = 0; r < nr; ++r)
                std::memcpy(&t[2 * (size_t)r * (nt - 1)], &p.xy[2 * (size_t)r * nt], sizeof(double) * 2 * (nt - 1));
            p.xy.swap(t);
            nt -= 1;
        }
        if (nr < 4 || nt < 8) {
            set_call_error("mesh too small");
            return JST_ERR_MESH_TOO_SMALL;
        }
        p.n_rings = nr;
        p.n_theta = nt;
        p.max_steps = max_steps < 0 ? p.raw.iteration : max_steps;
        p.drop = drop;
        p.cl_tol = cl_tol;
        p.t_submit = now();
        p.id = next_id_++;
        *id = p.id;
        queue_.push_back(std::move(p));
        return JST_OK;
    }

    size_t instance_bytes(int nr, int nt, int ntiles) const {
        size_t n = (size_t)(nr - 1) * nt, ntau = (size_t)nr * nt;
        size_t b = 0;
        auto add = [&](size_t x) { b += (x + 255) / 256 * 256; };
        add((10 * n + 4 * ntau) * sizeof(double));  // geometry
        add(2 * (size_t)nr * nt * sizeof(double));  // nodes
        add(5 * n * sizeof(double));                 // U_n
        add((sizeof(T) == sizeof(double) ? 10 : 15) * n * sizeof(T));  // U_a, U_b (+ U_c)
        add(2 * n * sizeof(T));                      // ratio
        add(n * sizeof(double));                     // localdt
        add(2 * (size_t)ntiles * sizeof(double));    // partials
        add(5 * (size_t)nt * sizeof(double));        // far
        add(ntau * fused::MG_N * sizeof(T));         // marching geometry records
        add(march2_geom_bytes<T>(nr - 1, nt));       // paired-column records (split)
        return b;
    }

    // Admit queued instances while a slot and arena memory are free.
    jst_status admit() {
        bool changed = false;
        while (!queue_.empty()) {
            int slot = -1;
            for (int k = 0; k < nslots_; ++k)
                if (!slots_[k].used) {
                    slot = k;
                    break;
                }
            if (slot < 0) break;
            Pending& p = queue_.front();
            int ni = p.n_rings - 1, nj = p.n_theta;
            int tiles_i = (ni + ti_ - 1) / ti_, tiles_j = (nj + tj_ - 1) / tj_, ntl = tiles_i * tiles_j;
            if ((long)h_tiles_.size() + ntl > max_tiles_) break;
            int ptl = max_tiles_for(ni, nj);
            size_t bytes = instance_bytes(p.n_rings, p.n_theta, ptl), off = 0;
            if (!arena_.alloc(bytes, &off)) break;
            Slot& S = slots_[slot];
            S = Slot{};
            S.used = true;
            S.id = p.id;
            S.off = off;
            S.bytes = bytes;
            S.ni = ni;
            S.nj = nj;
            S.ntiles = ntl;
            S.max_steps = p.max_steps;
            S.drop = p.drop;
            S.cl_tol = p.cl_tol;
            S.t_submit = p.t_submit;
            S.t_admit = now();
            S.aoa = p.raw.aoa * (M_PI / 180.0);
            double xmin = 1e300, xmax = -1e300;
            for (int t = 0; t < nj; ++t) {
                xmin = std::min(xmin, p.xy[2 * t]);
                xmax = std::max(xmax, p.xy[2 * t]);
            }
            S.chord = p.raw.chord > 0 ? p.raw.chord : xmax - xmin;
            PhysConst c = make_phys(p.raw);
            size_t n = (size_t)ni * nj, ntau = (size_t)(ni + 1) * nj;
            char* q = arena_.base + off;
            auto take = [&](size_t bytes_) {
                char* r = q;
                q += (bytes_ + 255) / 256 * 256;
                return r;
            };
            double* geo = reinterpret_cast<double*>(take((10 * n + 4 * ntau) * sizeof(double)));
            Geom& g = S.g;
            g.ni = ni;
            g.nj = nj;
            double* gq = geo;
            g.vol = gq; gq += n;
            g.cx = gq; gq += n;
            g.cy = gq; gq += n;
            g.wdist = gq; gq += n;
            g.inv_vol = gq; gq += n;
            g.inv_d2 = gq; gq += n;
            g.tnx = gq; gq += ntau;
            g.tny = gq; gq += ntau;
            g.tmx = gq; gq += ntau;
            g.tmy = gq; gq += ntau;
            g.nnx = gq; gq += n;
            g.nny = gq; gq += n;
            g.nmx = gq; gq += n;
            g.nmy = gq; gq += n;
            double* d_xy = reinterpret_cast<double*>(take(2 * (size_t)p.n_rings * nj * sizeof(double)));
            Inst<T>& I = h_insts_[slot];
            I = Inst<T>{};
            I.ni = ni;
            I.nj = nj;
            I.ntiles = ntl;
            I.local_dt = o_.dt_mode == JST_DT_LOCAL;
            I.tnx = g.tnx;
            I.tny = g.tny;
            I.nnx = g.nnx;
            I.nny = g.nny;
            I.vol = g.vol;
            I.inv_vol = g.inv_vol;
            I.inv_d2 = g.inv_d2;
            double* un = reinterpret_cast<double*>(take(5 * n * sizeof(double)));
            T* ua = reinterpret_cast<T*>(take((sizeof(T) == sizeof(double) ? 10 : 15) * n * sizeof(T)));
            T* ra = reinterpret_cast<T*>(take(2 * n * sizeof(T)));
            for (int k = 0; k < 5; ++k) {
                I.un[k] = un + k * n;
                I.ua[k] = ua + k * n;
                I.ub[k] = ua + (5 + k) * n;
                I.uc[k] = sizeof(T) == sizeof(double) ? nullptr : ua + (10 + k) * n;
            }
            I.ratio[0] = ra;
            I.ratio[1] = ra + n;
            I.ldt = reinterpret_cast<double*>(take(n * sizeof(double)));
            I.partial = reinterpret_cast<double*>(take(2 * (size_t)ptl * sizeof(double)));
            double* far = reinterpret_cast<double*>(take(5 * (size_t)nj * sizeof(double)));
            I.far = far;
            I.mg = reinterpret_cast<T*>(take((size_t)(ni + 1) * nj * fused::MG_N * sizeof(T)));
            I.mg2 = march2_geom_bytes<T>(ni, nj) ? reinterpret_cast<float*>(take(march2_geom_bytes<T>(ni, nj)))
                                                 : nullptr;
            I.res_hist = nullptr;
            I.st = d_states_ + slot;
            I.c = c;
            I.cp = fused::make_constp(c);
            cudaMemcpyAsync(d_xy, p.xy.data(), p.xy.size() * sizeof(double), cudaMemcpyHostToDevice, st_);
            geometry_build(d_xy, p.n_rings, nj, g, st_);
            JST_LAUNCH(k_far_geom, (nj + 255) / 256, 256, 0, st_, g, far);
            build_march_geom(g, ni, nj, const_cast<T*>(I.mg), st_);
            if (I.mg2) build_march_geom2(g, ni, nj, const_cast<float*>(I.mg2), st_);
            JST_LAUNCH(k_fill_freestream, (unsigned)((n + 255) / 256), 256, 0, st_, I.un[0], I.un[1], I.un[2],
                       I.un[3], I.un[4], (long)n, c);
            InstState s0{};
            s0.residual = std::numeric_limits<double>::quiet_NaN();
            s0.target = p.raw.targetres;
            s0.drop = p.drop;
            s0.bad = fused::NO_BAD;
            s0.fresh = 1;
            s0.max_step = (int)std::min<int64_t>(p.max_steps, INT_MAX - 1);
            h_states_[slot] = s0;
            cudaMemcpyAsync(d_states_ + slot, &h_states_[slot], sizeof(InstState), cudaMemcpyHostToDevice, st_);
            cudaMemcpyAsync(d_insts_ + slot, &h_insts_[slot], sizeof(Inst<T>), cudaMemcpyHostToDevice, st_);
            int tile_off = (int)h_tiles_.size();
            for (const TileRef& t : make_tiles(slot, ni, nj, ti_, tj_)) h_tiles_.push_back(t);
            counts_tmp_ = ntl;
            cudaMemcpyAsync(d_counts_ + slot, &counts_tmp_, sizeof(int), cudaMemcpyHostToDevice, st_);
            cudaMemcpyAsync(d_tiles_ + tile_off, h_tiles_.data() + tile_off, ntl * sizeof(TileRef),
                            cudaMemcpyHostToDevice, st_);
            JST_LAUNCH(K_.step_dt, ntl, K_.nt, 0, st_, d_tiles_ + tile_off, d_counts_ + slot, d_insts_, ti_, tj_);
            cudaStreamSynchronize(st_);  // pageable sources above must stay valid until copied
            ++active_;
            queue_.pop_front();
            changed = true;
        }
        if (changed) upload_tiles();
        return cudaGetLastError() == cudaSuccess ? JST_OK : JST_ERR_CUDA;
    }

    void upload_tiles() {
        ntiles_host_ = (int)h_tiles_.size();
        if (ntiles_host_)
            cudaMemcpyAsync(d_tiles_, h_tiles_.data(), h_tiles_.size() * sizeof(TileRef), cudaMemcpyHostToDevice,
                            st_);
        cudaMemcpyAsync(d_ntiles_, &ntiles_host_, sizeof(int), cudaMemcpyHostToDevice, st_);
        cudaStreamSynchronize(st_);
    }

    void ensure_graph() {
        if (graph_exec_) return;
        int K = std::max(1, o_.steps_per_poll);
        cudaGraph_t g;
        cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal);
        for (int q = 0; q < K; ++q)
            for (int s = 0; s < 5; ++s) {
                auto kern = s == 0 ? K_.stage[0] : (s == 4 ? K_.stage[2] : K_.stage[1]);
                JST_LAUNCH(kern, grid_, K_.nt, K_.smem, st_, d_tiles_, d_ntiles_, d_insts_, s, RK_ALPHA[s]);
            }
        cudaStreamEndCapture(st_, &g);
        cudaGraphInstantiate(&graph_exec_, g, 0);
        cudaGraphDestroy(g);
    }

    void wall_force_launch(int slot) {
        Slot& S = slots_[slot];
        UnPtrs up;
        for (int k = 0; k < 5; ++k) up.u[k] = h_insts_[slot].un[k];
        launch_wall_force(S.g, up, h_insts_[slot].c, d_force_ + 2 * slot, st_);
    }

    void clcd_from(int slot, const double* f, double* cl, double* cd) {
        Slot& S = slots_[slot];
        const PhysConst& c = h_insts_[slot].c;
        double q = 0.5 * c.rho_inf * (c.u_inf * c.u_inf + c.v_inf * c.v_inf) * S.chord;
        *cd = (f[0] * std::cos(S.aoa) + f[1] * std::sin(S.aoa)) / q;
        *cl = (-f[0] * std::sin(S.aoa) + f[1] * std::cos(S.aoa)) / q;
    }

    // Read every instance's device scalars, apply the CL window criterion,
    // retire finished instances.
    jst_status poll_retire() {
        cudaMemcpyAsync(h_states_, d_states_, nslots_ * sizeof(InstState), cudaMemcpyDeviceToHost, st_);
        if (cudaStreamSynchronize(st_) != cudaSuccess) return JST_ERR_CUDA;
        for (int k = 0; k < nslots_; ++k)
            if (slots_[k].used && h_states_[k].err) {
                set_call_error("a stage kernel's bounded wait for its row copies ran out");
                return JST_ERR_TIMEOUT;
            }
        std::vector<int> cl_slots;
        for (int k = 0; k < nslots_; ++k)
            if (slots_[k].used && slots_[k].cl_tol > 0.0 && h_states_[k].bad == fused::NO_BAD) {
                const auto& h = slots_[k].cl_hist;
                if (h.empty() || h_states_[k].step - h.back().first >= 50) cl_slots.push_back(k);
            }
        if (!cl_slots.empty()) {
            for (int k : cl_slots) wall_force_launch(k);
            std::vector<double> f(2 * nslots_);
            cudaMemcpyAsync(f.data(), d_force_, f.size() * sizeof(double), cudaMemcpyDeviceToHost, st_);
            cudaStreamSynchronize(st_);
            for (int k : cl_slots) {
                double cl, cd;
                clcd_from(k, &f[2 * k], &cl, &cd);
                slots_[k].cl_hist.emplace_back(h_states_[k].step, cl);
            }
        }
        bool changed = false;
        for (int k = 0; k < nslots_; ++k) {
            Slot& S = slots_[k];
            if (!S.used) continue;
            const InstState& st = h_states_[k];
            bool bad = st.bad != fused::NO_BAD;
            bool cl_conv = false;
            if (S.cl_tol > 0.0 && S.cl_hist.size() >= 2) {
                const auto& h = S.cl_hist;
                int cur = h.back().first;
                for (size_t q = h.size() - 1; q-- > 0;)
                    if (cur - h[q].first >= 100) {
                        cl_conv = std::fabs(h.back().second - h[q].second) < S.cl_tol;
                        break;
                    }
            }
            if (!(bad || st.done || cl_conv || st.step >= S.max_steps)) continue;
            retire(k, st, bad, st.done || cl_conv);
            changed = true;
        }
        if (changed) {
            std::vector<TileRef> keep;
            keep.reserve(h_tiles_.size());
            for (const TileRef& t : h_tiles_)
                if (slots_[t.inst].used) keep.push_back(t);
            h_tiles_.swap(keep);
            upload_tiles();
        }
        return JST_OK;
    }

    void retire(int slot, const InstState& st, bool bad, bool converged) {
        Slot& S = slots_[slot];
        BatchResultFull R;
        R.r.id = S.id;
        R.r.steps = st.step;
        R.r.residual = st.residual;
        R.r.residual_first = st.res_first;
        R.r.totaltime = st.totaltime;
        R.r.t_submit = S.t_submit;
        R.r.t_admit = S.t_admit;
        R.r.ni = S.ni;
        R.r.nj = S.nj;
        R.r.status = bad ? JST_ERR_NONPHYSICAL : (converged ? JST_OK : JST_ERR_TIMEOUT);
        if (bad) {
            long id = (long)(st.bad & 0xffffffffULL);
            int stage = (int)((st.bad >> 32) % 5);
            double u[5];
            for (int k = 0; k < 5; ++k) {
                if (stage == 4) {
                    cudaMemcpy(&u[k], h_insts_[slot].un[k] + id, sizeof(double), cudaMemcpyDeviceToHost);
                } else {
                    T v;
                    cudaMemcpy(&v, (stage % 2 == 0 ? h_insts_[slot].ua[k] : h_insts_[slot].ub[k]) + id, sizeof(T),
                               cudaMemcpyDeviceToHost);
                    u[k] = (double)v;
                }
            }
            nonphysical_report(h_insts_[slot].c, id / S.nj, id % S.nj, u, &R.r.bad);
            R.r.cl = R.r.cd = std::numeric_limits<double>::quiet_NaN();
        } else {
            wall_force_launch(slot);
            double f[2];
            cudaMemcpyAsync(f, d_force_ + 2 * slot, sizeof f, cudaMemcpyDeviceToHost, st_);
            cudaStreamSynchronize(st_);
            clcd_from(slot, f, &R.r.cl, &R.r.cd);
        }
        if (o_.keep_fields) {
            size_t n = (size_t)S.ni * S.nj;
            R.fields.resize(5 * n);
            for (int k = 0; k < 5; ++k)
                cudaMemcpy(R.fields.data() + k * n, h_insts_[slot].un[k], n * sizeof(double), cudaMemcpyDeviceToHost);
        }
        R.r.t_done = now();
        results_[S.id] = std::move(R);
        finished_.push_back(S.id);
        arena_.release(S.off, S.bytes);
        S.used = false;
        --active_;
    }

    jst_status step(int nsteps) override {
        jst_status rc = admit();
        if (rc != JST_OK) return rc;
        if (tune_ && active_ > 0) tune();
        ensure_graph();
        int K = std::max(1, o_.steps_per_poll), done = 0;
        while (done < nsteps && (active_ > 0 || !queue_.empty())) {
            if (active_ == 0) {
                admit();
                if (active_ == 0) break;
            }
            cudaGraphLaunch(graph_exec_, st_);
            done += K;
            rc = poll_retire();
            if (rc != JST_OK) return rc;
            rc = admit();
            if (rc != JST_OK) return rc;
        }
        return JST_OK;
    }

    void kernel_config(int* ti, int* tj, int* nt) const override {
        *ti = ti_;
        *tj = tj_;
        *nt = K_.nt;
    }
    int kernel_staging() const override { return K_.march ? (K_.staging == 1 ? JST_STAGING_BULK : JST_STAGING_PER_LANE) : 0; }

    void stats(int* a, int* q, double* bytes) override {
        if (a) *a = active_;
        if (q) *q = (int)queue_.size();
        if (bytes) *bytes = (double)arena_.used;
    }

    int poll(int64_t* ids, int cap) override {
        int n = 0;
        while (!finished_.empty() && n < cap) {
            ids[n++] = finished_.front();
            finished_.pop_front();
        }
        return n;
    }

    bool result(int64_t id, BatchResultFull** out) override {
        auto it = results_.find(id);
        if (it == results_.end()) return false;
        *out = &it->second;
        return true;
    }

  private:
    jst_batch_opts o_;
    Clock::time_point t0_;
    cudaStream_t st_ = nullptr;
    Kernels<T> K_;
    int ti_ = 8, tj_ = 32, grid_ = 1, nslots_ = 1, max_tiles_ = 0, ntiles_host_ = 0, counts_tmp_ = 0;
    int active_ = 0;
    bool tune_ = false;
    int64_t next_id_ = 0;
    void* small_ = nullptr;
    Inst<T>* d_insts_ = nullptr;
    InstState* d_states_ = nullptr;
    InstState* h_states_ = nullptr;
    double* d_force_ = nullptr;
    int* d_counts_ = nullptr;
    int* d_ntiles_ = nullptr;
    TileRef* d_tiles_ = nullptr;
    std::vector<Inst<T>> h_insts_;
    std::vector<Slot> slots_;
    std::vector<TileRef> h_tiles_;
    std::deque<Pending> queue_;
    std::map<int64_t, BatchResultFull> results_;
    std::deque<int64_t> finished_;
    Arena arena_;
    cudaGraphExec_t graph_exec_ = nullptr;
};

}  // namespace jst

struct jst_batch {
    std::unique_ptr<jst::BatchBase> impl;
};

// Test hook (declared in include/jst_gpu_debug.h): the marching kernels' FP64
// quotient, square root, exponential and inverse sixth root (jst::dv, sq, ex
// with Q = true, and jst::rroot6) beside the library's, for n operand pairs:
// out[8k..8k+7] = quick a/b, a/b, quick sqrt(b), sqrt(b), quick exp(a),
// exp(a), b^(-1/6), 1 / cbrt(sqrt(b)).
__global__ void k_quick_arith(const double* a, const double* b, double* out, long n) {
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double x = a[k], y = b[k];
    double* o = out + 8 * k;
    o[0] = jst::dv<double, true>(x, y);
    o[1] = __ddiv_rn(x, y);
    o[2] = jst::sq<double, true>(y);
    o[3] = __dsqrt_rn(y);
    o[4] = jst::ex<double, true>(x);
    o[5] = exp(x);
    o[6] = jst::rroot6(y);
    o[7] = __ddiv_rn(1.0, cbrt(__dsqrt_rn(y)));
}

extern "C" jst_status jst_debug_quick_arith(const double* a, const double* b, double* out, size_t n) {
    if (!a || !b || !out || n == 0) return JST_ERR_ARG;
    double* d = nullptr;
    if (cudaMalloc(&d, 10 * n * sizeof(double)) != cudaSuccess) return JST_ERR_OOM;
    cudaMemcpy(d, a, n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d + n, b, n * sizeof(double), cudaMemcpyHostToDevice);
    JST_LAUNCH(k_quick_arith, (unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)0, d, d + n, d + 2 * n, (long)n);
    cudaError_t e = cudaMemcpy(out, d + 2 * n, 8 * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? JST_OK : JST_ERR_CUDA;
}

extern "C" {

void jst_batch_default_opts(jst_batch_opts* o) {
    std::memset(o, 0, sizeof *o);
    o->precision = JST_PREC_FP32_SPLIT;
    o->dt_mode = JST_DT_LOCAL;
    o->max_instances = 256;
    o->steps_per_poll = 20;
    o->hbm_budget_gb = 0.0;
}

jst_status jst_batch_create(const jst_batch_opts* o, jst_batch** out) {
    if (!o || !out) return JST_ERR_ARG;
    std::string err;
    std::unique_ptr<jst::BatchBase> impl;
    if (o->precision == JST_PREC_FP64) {
        auto* b = new jst::Batch<double>(*o);
        impl.reset(b);
        if (!b->create(err)) {
            jst::set_call_error(err);
            return JST_ERR_OOM;
        }
    } else {
        auto* b = new jst::Batch<float>(*o);
        impl.reset(b);
        if (!b->create(err)) {
            jst::set_call_error(err);
            return JST_ERR_OOM;
        }
    }
    *out = new jst_batch{std::move(impl)};
    return JST_OK;
}

void jst_batch_destroy(jst_batch* b) { delete b; }

jst_status jst_batch_submit(jst_batch* b, const char* cfg, const double* xy, int n_rings, int n_theta,
                            int64_t max_steps, double residual_drop, double cl_tol, int64_t* id) {
    if (!b || !cfg || !xy || !id) return JST_ERR_ARG;
    return b->impl->submit(cfg, xy, n_rings, n_theta, max_steps, residual_drop, cl_tol, id);
}

jst_status jst_batch_step(jst_batch* b, int nsteps) { return b ? b->impl->step(nsteps) : JST_ERR_ARG; }

jst_status jst_batch_kernel_config(const jst_batch* b, int* ti, int* tj, int* nt) {
    if (!b || !ti || !tj || !nt) return JST_ERR_ARG;
    b->impl->kernel_config(ti, tj, nt);
    return JST_OK;
}

jst_status jst_batch_kernel_staging(const jst_batch* b, int* staging) {
    if (!b || !staging) return JST_ERR_ARG;
    *staging = b->impl->kernel_staging();
    return JST_OK;
}

jst_status jst_batch_stats(jst_batch* b, int* active, int* queued, double* bytes) {
    if (!b) return JST_ERR_ARG;
    b->impl->stats(active, queued, bytes);
    return JST_OK;
}

jst_status jst_batch_poll(jst_batch* b, int64_t* ids, int cap, int* n) {
    if (!b || !n || (cap > 0 && !ids)) return JST_ERR_ARG;
    *n = b->impl->poll(ids, cap);
    return JST_OK;
}

jst_status jst_batch_result_get(jst_batch* b, int64_t id, jst_batch_result* r, double* fields, size_t n) {
    if (!b || !r) return JST_ERR_ARG;
    jst::BatchResultFull* R = nullptr;
    if (!b->impl->result(id, &R)) return JST_ERR_ARG;
    *r = R->r;
    if (fields) {
        if (R->fields.empty() || n < R->fields.size()) return JST_ERR_ARG;
        std::memcpy(fields, R->fields.data(), R->fields.size() * sizeof(double));
    }
    return JST_OK;
}

}  // extern "C"

namespace jst {

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
