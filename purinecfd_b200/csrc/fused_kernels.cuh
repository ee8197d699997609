// Fused RK-stage kernel: one launch per Runge-Kutta stage over a table of
// (instance, tile) work items.  A tile is TI x TJ interior cells; its block
// stages the tile plus a 3-cell halo of the stage state in shared memory,
// builds the halo's ghost cells in place (wall mirror, far-field Riemann state,
// periodic seam — boundary.rs:23-185), and then, all in shared memory:
//   gradients + diffusion tensors on the tile and its first ring
//   (gradient.rs:38-102, viscous.rs:74-125), pressure sensors
//   (dissipation.rs:73-90), one net flux per face — convective + viscous +
//   JST dissipation, computed once and used by both cells
//   (convection.rs:46-80, viscous.rs:128-164, dissipation.rs:93-185) — the SA
//   source (source.rs:45-88), the RK update U = U_n - alpha*dt*R/V
//   (solver.rs:123-145) and the non-physical check of unpack
//   (solver.rs:151-185).  The last stage also forms the residual
//   (solver.rs:190-200) and the next step's local time steps and their
//   minimum (timestep.rs:24-57) with a last-block-done reduction.
//
// T is the stage arithmetic (double, or float for the split mode); the
// step-start state U_n, the geometry, the time step and all reductions are
// FP64.  Work loops stride by the block size so every phase is a loop over
// work items separated by barriers.
#pragma once

#include <cstring>
#include <type_traits>

#ifdef __CUDACC__
#include <cuda_pipeline.h>
#endif

#include "jst_common.cuh"

#ifndef JST_DYN_SMEM
#define JST_DYN_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#endif
#ifndef JST_TID
#define JST_TID() ((int)threadIdx.x)
#define JST_BID() ((int)blockIdx.x)
#define JST_GRID() (gridDim.x)
#define JST_SYNC() __syncthreads()
#define JST_FENCE() __threadfence()
#endif

namespace jst {
namespace fused {

constexpr unsigned long long NO_BAD = ~0ULL;

// Per-instance device scalars.
struct InstState {
    double dt;         // global time step of the current step
    double totaltime;  // accumulated physical time (solver.rs:110-111)
    double residual;   // residual of the last completed step
    double target;     // solver.targetres
    double drop;       // > 0: also stop when residual < drop * first residual
    double res_first;  // residual of the first completed step
    unsigned long long bad;  // (stage_id << 32) | cell, NO_BAD when none
    unsigned int counter;    // last-block-done counter
    int step;          // completed steps
    int fresh;         // 1 until the first step completed: stage 0 uses the free-stream primitives
    int done;          // residual fell below target
    int max_step;      // device-side step limit (steps beyond it are skipped)
    int err;           // nonzero: a bounded wait in a stage kernel ran out (bulk row staging)
};

// The per-instance constants of the split precision's marching kernels,
// rounded once to FP32 and stored as pairs (both halves equal): the
// paired-column kernel reads a pair with one 64-bit load, the one-column
// kernel the first half; both copy them to shared memory per strip.
struct ConstP {
    float2 inv_t_ref, suth_num, t_suth, cv1_cubed, inv_pr, inv_prt, cp, sigma;
    float2 inv_kappa2, m_ct4, ct3, fv3, cb1, rmax, cw1, m_cb1_k2, cb2_sigma, rg, cfl;
    float2 gm1, r_gas, half_cfl, k2, k4, p_ref2;
    float2 f_rho, f_p, f_t, f_vx, f_vy, f_e, f_nut;
    float2 cw2, cw3_6, one_plus_cw3_6, fw_lim;
};

JST_HD ConstP make_constp(const PhysConst& c) {
    auto s = [](double x) {
        float f = (float)x;
        return float2{f, f};
    };
    ConstP k;
    k.inv_t_ref = s(c.inv_t_ref);
    k.suth_num = s(c.suth_num);
    k.t_suth = s(c.t_suth);
    k.cv1_cubed = s(c.cv1_cubed);
    k.inv_pr = s(c.inv_pr);
    k.inv_prt = s(c.inv_prt);
    k.cp = s(c.cp);
    k.sigma = s(c.sigma);
    k.inv_kappa2 = s(c.inv_kappa2);
    k.m_ct4 = s(-c.Ct4);
    k.ct3 = s(c.Ct3);
    k.fv3 = s(c.fv3);
    k.cb1 = s(c.Cb1);
    k.rmax = s(c.rmax);
    k.cw1 = s(c.cw1);
    k.m_cb1_k2 = s(-c.cb1_k2);
    k.cb2_sigma = s(c.cb2_sigma);
    k.rg = s(c.rg);
    k.cfl = s(c.cfl);
    k.gm1 = s(c.gm1);
    k.r_gas = s(c.r_gas);
    k.half_cfl = s(c.half_cfl);
    k.k2 = s(c.k2);
    k.k4 = s(c.k4);
    k.p_ref2 = s(2.0 * c.p_inf);
    k.f_rho = s(c.f_rho);
    k.f_p = s(c.f_p);
    k.f_t = s(c.f_t);
    k.f_vx = s(c.f_vx);
    k.f_vy = s(c.f_vy);
    k.f_e = s(c.f_e);
    k.f_nut = s(c.f_nut);
    k.cw2 = s(c.Cw2);
    k.cw3_6 = s(c.cw3_6);
    k.one_plus_cw3_6 = s(c.one_plus_cw3_6);
    k.fw_lim = s(c.fw_lim);
    return k;
}

// Per-instance descriptor (read-only during a launch except through `st`).
template <class T> struct Inst {
    int ni, nj;
    int ntiles;       // tiles of this instance
    int local_dt;     // JST_DT_LOCAL
    // geometry, FP64 (geometry.rs:45-63)
    const double *tnx, *tny, *nnx, *nny, *vol, *inv_vol, *inv_d2;
    const double* far;  // per column j: tau(NI) normal x,y and centroid distances of cells NI-1..NI-3 (5*nj)
    // state; the five planes of each array are contiguous (plane k at plane 0
    // + k * ni * nj), which the marching kernel relies on
    double* un[5];      // U_n, the FP64 step-start state
    T* ua[5];           // stage ping-pong buffers
    T* ub[5];
    T* uc[5];           // split mode: T copy of U_n written by the last stage, staged by stage 0
    T* ratio[2];        // V / localdt, indexed by step parity (dissipation.rs:51-56)
    double* ldt;        // localdt of the current step (local time stepping)
    double* partial;    // per tile: min localdt, sum (drho)^2
    double* res_hist;   // residual per completed step (may be null)
    InstState* st;
    PhysConst c;
    // marching kernels: per (row k in 0..NI, column j) the record
    // {tau nx, ny of face row k; n nx, ny, 1/V, 1/d^2, V of cell row k-1; 0}
    // in the stage type (zeros for cell row -1), see k_march_geom
    const T* mg;
    // paired-column marching kernel (split precision): the same records with
    // the two columns of each pair interleaved, see k_march_geom2
    const float* mg2;
    ConstP cp;  // make_constp(c)
    // bulk row staging: bytes the row barrier expects beyond those copied
    // (0; a test sets it so that the bounded wait runs out)
    int stage_extra_tx;
    // residual dump (jst_stage_residual): 5 planes of NI*NJ doubles that the
    // DUMP instantiation of stage 0 writes R = Fc - Fv - Fd - S into
    double* rdump;
};

struct TileRef {
    int inst, i0, j0, tile;  // tile = index within its instance
    int i1;                  // end row (exclusive): rows i0 .. i1-1 belong to this item
};

// Shared-memory layout of one tile.  T-typed arrays first, then the FP64
// block (the tile's geometry), then the reduction / far-field
// scratch.  The primitive arrays (P, Q) are dead once gradients and sensors
// exist, and the face fluxes reuse their space.
template <class T, int TI, int TJ, int NT> struct Layout {
    static constexpr int LI = TI + 6, LJ = TJ + 6, NL = LI * LJ;  // staged cells (halo 3)
    static constexpr int RI = TI + 2, RJ = TJ + 2, NR = RI * RJ;  // tile + first ring
    static constexpr int TT = TI * TJ;
    static constexpr int NSI = (TI + 4) * TJ, NSJ = TI * (TJ + 4);
    static constexpr int GTJ = TJ + 2, NGT = (TI + 3) * GTJ;  // tau normals, rows i0-1..i0+TI+1
    static constexpr int GNJ = TJ + 3, NGN = (TI + 2) * GNJ;  // n normals, rows i0-1..i0+TI
    // T-typed offsets
    static constexpr int oU = 0;
    static constexpr int oSi = oU + 5 * NL;
    static constexpr int oSj = oSi + NSI;
    static constexpr int oD = oSj + NSJ;  // Dx1..4, Dy1..4 on tile + ring
    static constexpr int oS = oD + 8 * NR;  // SA source * V, tile cells
    static constexpr int oR = oS + TT;      // ratio V/localdt on tile + ring (rows clamped)
    static constexpr int NFT = (TI + 1) * TJ, NFN = TI * (TJ + 1);
    static constexpr int oX = oR + NR;      // P (NL) + Q (4 NL)  |  face fluxes Ft (5 NFT) + Fn (5 NFN)
    static constexpr int XSZ = 5 * NL > 5 * (NFT + NFN) ? 5 * NL : 5 * (NFT + NFN);
    static constexpr int tsize = oX + XSZ;
    // FP64 geometry block: tau nx, ny; n nx, ny; 1/V on tile + ring; V and 1/d^2 on the tile
    static constexpr size_t goff = ((size_t)tsize * sizeof(T) + 15) / 16 * 16;
    static constexpr int gTx = 0, gTy = NGT, gNx = 2 * NGT, gNy = 2 * NGT + NGN, gIV = 2 * NGT + 2 * NGN,
                         gV = gIV + NR, gD2 = gV + TT, gsize = gD2 + TT;
    static constexpr size_t red_off = goff + (size_t)gsize * sizeof(double);
    static constexpr size_t bytes = red_off + (size_t)(NT + 7 * LJ) * sizeof(double);
};

template <class T> JST_D T ld(const T* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// Periodic column index (boundary.rs:54-72); a tile may be wider than the ring.
JST_D int wrapj(int j, int nj) {
    if (j < 0) j += nj;
    else if (j >= nj) j -= nj;
    if ((unsigned)j >= (unsigned)nj) j = ((j % nj) + nj) % nj;
    return j;
}

// Primitive state of a staged cell from its conserved state (or the free
// stream on the first stage of the first step).
template <class T, class TS>
JST_D Prim<T> prim_from(const TS* const* src, long idx, int fresh, const PhysConst& c, T* u) {
    Prim<T> q;
    for (int k = 0; k < 5; ++k) u[k] = (T)ld(src[k] + idx);
    if (fresh) {
        q.rho = (T)c.f_rho;
        q.p = (T)c.f_p;
        q.t = (T)c.f_t;
        q.vx = (T)c.f_vx;
        q.vy = (T)c.f_vy;
        q.e = (T)c.f_e;
        q.nut = (T)c.f_nut;
    } else {
        q = unpack_cell<T>(u[0], u[1], u[2], u[3], u[4], (T)c.gm1, (T)c.r_gas);
    }
    return q;
}

// Block-wide reduction helpers over NT threads (fixed shape: deterministic).
// Largest power of two not above n: block sizes of 192 or 384 threads first
// fold their upper part onto it, so that the tree below sees every element.
JST_HD constexpr int pow2_floor(int n) { return n < 2 ? 1 : 2 * pow2_floor(n / 2); }

template <int NT> JST_D double block_sum(double v, double* red) {
    constexpr int P = pow2_floor(NT);
    int t = JST_TID();
    red[t] = v;
    JST_SYNC();
    if (P < NT) {
        if (t < NT - P) red[t] += red[t + P];
        JST_SYNC();
    }
    for (int w = P / 2; w > 0; w >>= 1) {
        if (t < w) red[t] += red[t + w];
        JST_SYNC();
    }
    double r = red[0];
    JST_SYNC();
    return r;
}

template <int NT> JST_D double block_min(double v, double* red) {
    constexpr int P = pow2_floor(NT);
    int t = JST_TID();
    red[t] = v;
    JST_SYNC();
    if (P < NT) {
        if (t < NT - P) red[t] = fmin(red[t], red[t + P]);
        JST_SYNC();
    }
    for (int w = P / 2; w > 0; w >>= 1) {
        if (t < w) red[t] = fmin(red[t], red[t + w]);
        JST_SYNC();
    }
    double r = red[0];
    JST_SYNC();
    return r;
}

// timestep.rs:30-42 for cell (i, j) of instance I with primitive state (u, v, t).
template <class T> JST_D double cell_localdt(const Inst<T>& I, int i, int j, double u, double v, double t) {
    long id = (long)i * I.nj + j;
    int jp = j + 1 < I.nj ? j + 1 : 0;
    long t0 = id, t1 = id + I.nj, n0 = id, n1 = (long)i * I.nj + jp;
    double a = 0.5 * (ld(I.tnx + t0) + ld(I.tnx + t1));
    double b = 0.5 * (ld(I.tny + t0) + ld(I.tny + t1));
    double cc = 0.5 * (ld(I.nnx + n0) + ld(I.nnx + n1));
    double dd = 0.5 * (ld(I.nny + n0) + ld(I.nny + n1));
    double cs = sqrt(I.c.rg * t);
    return local_dt<double>(u, v, cs, a, b, cc, dd, I.c.cfl * ld(I.vol + id));
}

// Last-block-done reduction of the per-tile partials of one instance:
// writes dt (minimum local step) and, when `with_residual`, the residual of
// the step just completed.  Called by every thread of the block that finished
// last.
template <class T, int NT>
JST_D void finish_step(const Inst<T>& I, bool with_residual, double* red) {
    int t = JST_TID();
    double m = __longlong_as_double(0x7ff0000000000000LL);
    double s = 0.0;
    for (int k = t; k < I.ntiles; k += NT) {
        volatile const double* pp = I.partial + 2 * k;
        m = fmin(m, pp[0]);
        s += pp[1];
    }
    double mn = block_min<NT>(m, red);
    double sm = block_sum<NT>(s, red);
    if (t == 0) {
        InstState* st = I.st;
        st->dt = mn;
        if (with_residual) {
            double res = sqrt(sm / (double)I.ni / (double)I.nj);
            int step = st->step;
            st->residual = res;
            if (I.res_hist) I.res_hist[step] = res;
            if (step == 0) st->res_first = res;
            st->step = step + 1;
            st->fresh = 0;
            if (res < st->target || (st->drop > 0.0 && res < st->drop * st->res_first)) st->done = 1;
        }
        st->counter = 0;
    }
}

// Local time steps of every cell of one tile from U_n (or the free stream),
// plus the per-instance minimum: the time step of the first step and of any
// step after the state was overwritten (timestep.rs:24-57).
template <class T, int NT>
__global__ void __launch_bounds__(NT) k_step_dt(const TileRef* tiles, const int* ntiles, const Inst<T>* insts,
                                                 int TI, int TJ) {
    __shared__ double red[NT];
    __shared__ int last;
    const int nt_all = *ntiles;
    for (int tix = JST_BID(); tix < nt_all; tix += (int)JST_GRID()) {
    TileRef tr = tiles[tix];
    const Inst<T>& I = insts[tr.inst];
    int fresh = I.st->fresh;
    double mloc = __longlong_as_double(0x7ff0000000000000LL);
    for (int w = JST_TID(); w < TI * TJ; w += NT) {
        int i = tr.i0 + w / TJ, j = tr.j0 + w % TJ;
        if (i >= tr.i1 || j >= I.nj) continue;
        long id = (long)i * I.nj + j;
        double u, v, t;
        if (fresh) {
            u = I.c.f_vx;
            v = I.c.f_vy;
            t = I.c.f_t;
        } else {
            Prim<double> q = unpack_cell<double>(I.un[0][id], I.un[1][id], I.un[2][id], I.un[3][id], I.un[4][id],
                                                 I.c.gm1, I.c.r_gas);
            u = q.vx;
            v = q.vy;
            t = q.t;
        }
        if (sizeof(T) != sizeof(double))
            for (int k = 0; k < 5; ++k) I.uc[k][id] = (T)I.un[k][id];
        double dl = cell_localdt<T>(I, i, j, u, v, t);
        I.ratio[I.st->step & 1][id] = (T)(ld(I.vol + id) / dl);
        if (I.local_dt) I.ldt[id] = dl;
        mloc = fmin(mloc, dl);
    }
    double mn = block_min<NT>(mloc, red);
    if (JST_TID() == 0) {
        I.partial[2 * tr.tile] = mn;
        I.partial[2 * tr.tile + 1] = 0.0;
        JST_FENCE();
        unsigned prev = atomicAdd(&I.st->counter, 1u);
        last = prev == (unsigned)(I.ntiles - 1);
    }
    JST_SYNC();
    if (last) {
        JST_FENCE();
        finish_step<T, NT>(I, false, red);
    }
    JST_SYNC();
    }
}

// Asynchronous global -> shared copies (cp.async), one element each.
template <int BYTES> JST_D void async_copy(void* dst, const void* src) {
#ifdef __CUDA_ARCH__
    __pipeline_memcpy_async(dst, src, BYTES);
#else
    std::memcpy(dst, src, BYTES);
#endif
}

JST_D void async_commit() {
#ifdef __CUDA_ARCH__
    __pipeline_commit();
#endif
}

// Wait until at most the most recently committed group is still in flight.
JST_D void async_wait_prior1() {
#ifdef __CUDA_ARCH__
    __pipeline_wait_prior(1);
#endif
}

JST_D void async_wait_all() {
#ifdef __CUDA_ARCH__
    __pipeline_commit();
    __pipeline_wait_prior(0);
#endif
}

// The stage kernel.  FIRST: stage 0 (reads U_n, adds dt to the total time).
// LAST: stage 4 (writes U_n in place, residual, next step's time step).
// DUMP (with FIRST only): the residual R of every cell of the current state
// goes to Inst::rdump instead of an update; nothing else is written and the
// instance's step counters and stop flags are ignored.
template <class T, int TI, int TJ, int NT, bool FIRST, bool LAST, bool DUMP = false>
__global__ void __launch_bounds__(NT) k_stage(const TileRef* tiles, int* ntiles, const Inst<T>* insts, int stage,
                                              double alpha) {
    using L = Layout<T, TI, TJ, NT>;
    // Stage 0 reads U_n; in the split mode it stages the T copy of U_n that the
    // previous last stage wrote, so every stage stages T values asynchronously.
    using TS = T;
    using TD = typename std::conditional<LAST, double, T>::type;
    constexpr bool ASYNC_U = true;
    constexpr int LJ = L::LJ, NL = L::NL, RJ = L::RJ, NR = L::NR, TT = L::TT;
    JST_DYN_SMEM(smem_raw);
    T* sm = reinterpret_cast<T*>(smem_raw);
    double* gs = reinterpret_cast<double*>(smem_raw + L::goff);
    double* red = reinterpret_cast<double*>(smem_raw + L::red_off);
    double* farbuf = red + NT;  // 7 values per staged column of a far-field tile
    __shared__ int flags[4];
    __shared__ double adt_s;
    const int nt_all = *ntiles;
    // Persistent over the tile table: blocks stride through (instance, tile) items.
    for (int tix = JST_BID(); tix < nt_all; tix += (int)JST_GRID()) {
    const TileRef tr = tiles[tix];
    const Inst<T>& I = insts[tr.inst];
    const int ni = I.ni, nj = I.nj, i0 = tr.i0, j0 = tr.j0;
    const PhysConst& c = I.c;
    const int tid = JST_TID();

    if (tid == 0) {
        InstState* st = I.st;
        int step = st->step;
        unsigned long long stage_id = (unsigned long long)step * 5 + stage;
        unsigned long long bad = st->bad;
        int skip = !DUMP && (st->done || step >= st->max_step || (bad != NO_BAD && (bad >> 32) < stage_id));
        flags[0] = skip;
        flags[1] = FIRST ? st->fresh : 0;
        flags[2] = step;
        adt_s = alpha * st->dt;  // the step's global time step, read once per tile
        if (FIRST && !DUMP && !skip && tr.tile == 0) st->totaltime += st->dt;
    }
    JST_SYNC();
    if (flags[0]) {
        JST_SYNC();  // flags is rewritten by the next item
        continue;
    }
    const int fresh = flags[1];
    const unsigned long long stage_id = (unsigned long long)flags[2] * 5 + stage;
    const T* ratio = I.ratio[flags[2] & 1];
    T* ratio_next = I.ratio[(flags[2] + 1) & 1];
    (void)ratio_next;

    const TS* src[5];
    TD* dst[5];
    for (int k = 0; k < 5; ++k) {
        if (FIRST) src[k] = sizeof(T) == sizeof(double) ? reinterpret_cast<const TS*>(I.un[k]) : I.uc[k];
        else src[k] = reinterpret_cast<const TS*>((stage % 2 == 1) ? I.ua[k] : I.ub[k]);
        if (LAST) dst[k] = reinterpret_cast<TD*>(I.un[k]);
        else dst[k] = reinterpret_cast<TD*>((stage % 2 == 0) ? I.ua[k] : I.ub[k]);
    }

    T* sU = sm + L::oU;
    T* sSi = sm + L::oSi;
    T* sSj = sm + L::oSj;
    T* sD = sm + L::oD;
    T* sS = sm + L::oS;
    T* sRat = sm + L::oR;
    T* sP = sm + L::oX;
    T* sQ = sP + NL;        // u, v, T, nut

    // ---- A1: stage the tile geometry and the interior rows of U ----------
    for (int e = tid; e < L::NGT; e += NT) {  // tau normals, rows i0-1 .. i0+TI+1
        int r = e / L::GTJ, cc = e - r * L::GTJ;
        int gi = i0 - 1 + r, gj = wrapj(j0 - 1 + cc, nj);
        if (gi >= 0 && gi <= ni) {
            long f = (long)gi * nj + gj;
            async_copy<8>(gs + L::gTx + e, I.tnx + f);
            async_copy<8>(gs + L::gTy + e, I.tny + f);
        } else {
            gs[L::gTx + e] = 0.0;
            gs[L::gTy + e] = 0.0;
        }
    }
    for (int e = tid; e < L::NGN; e += NT) {  // n normals, rows i0-1 .. i0+TI
        int r = e / L::GNJ, cc = e - r * L::GNJ;
        int gi = i0 - 1 + r, gj = wrapj(j0 - 1 + cc, nj);
        if (gi >= 0 && gi < ni) {
            long f = (long)gi * nj + gj;
            async_copy<8>(gs + L::gNx + e, I.nnx + f);
            async_copy<8>(gs + L::gNy + e, I.nny + f);
        } else {
            gs[L::gNx + e] = 0.0;
            gs[L::gNy + e] = 0.0;
        }
    }
    for (int e = tid; e < NR; e += NT) {  // 1/V and V/localdt on tile + ring
        int r = e / RJ, cc = e - r * RJ;
        int gi = i0 - 1 + r, gj = wrapj(j0 - 1 + cc, nj);
        if (gi >= 0 && gi < ni) async_copy<8>(gs + L::gIV + e, I.inv_vol + (long)gi * nj + gj);
        else gs[L::gIV + e] = 0.0;
        int gc = gi < 0 ? 0 : (gi > ni - 1 ? ni - 1 : gi);  // dissipation.rs:59 clamps
        async_copy<sizeof(T)>(sRat + e, ratio + (long)gc * nj + gj);
    }
    for (int e = tid; e < TT; e += NT) {  // V and 1/d^2 on the tile
        int r = e / TJ, cc = e - r * TJ;
        int gi = i0 + r, gj = wrapj(j0 + cc, nj);
        if (gi < ni) {
            async_copy<8>(gs + L::gV + e, I.vol + (long)gi * nj + gj);
            async_copy<8>(gs + L::gD2 + e, I.inv_d2 + (long)gi * nj + gj);
        } else {
            gs[L::gV + e] = 0.0;
            gs[L::gD2 + e] = 0.0;
        }
    }
    constexpr int KA = (NL + NT - 1) / NT;
    TS rawr[ASYNC_U ? 1 : KA][5];
#pragma unroll
    for (int q = 0; q < KA; ++q) {
        int w = tid + q * NT;
        if (w < NL) {
            int li = w / LJ, lj = w - li * LJ;
            int gi = i0 - 3 + li;
            if (gi >= 0 && gi < ni) {
                long id = (long)gi * nj + wrapj(j0 - 3 + lj, nj);
                if constexpr (ASYNC_U) {
                    for (int k = 0; k < 5; ++k) async_copy<sizeof(T)>(sU + k * NL + w, src[k] + id);
                } else {
                    for (int k = 0; k < 5; ++k) rawr[q][k] = ld(src[k] + id);
                }
            }
        }
    }
    async_wait_all();
    // primitives of the interior rows; periodic ghost columns are re-packed
    // from their primitives (boundary.rs:54-72, state.rs:143-156)
#pragma unroll
    for (int q = 0; q < KA; ++q) {
        int w = tid + q * NT;
        if (w < NL) {
            int li = w / LJ, lj = w - li * LJ;
            int gi = i0 - 3 + li, gjr = j0 - 3 + lj;
            if (gi >= 0 && gi < ni) {
                T u[5];
                if constexpr (ASYNC_U) {
                    for (int k = 0; k < 5; ++k) u[k] = sU[k * NL + w];
                } else {
                    for (int k = 0; k < 5; ++k) u[k] = (T)rawr[q][k];
                }
                Prim<T> p;
                if (fresh) {
                    p.rho = (T)c.f_rho;
                    p.p = (T)c.f_p;
                    p.t = (T)c.f_t;
                    p.vx = (T)c.f_vx;
                    p.vy = (T)c.f_vy;
                    p.e = (T)c.f_e;
                    p.nut = (T)c.f_nut;
                } else {
                    p = unpack_cell<T, true>(u[0], u[1], u[2], u[3], u[4], (T)c.gm1, (T)c.r_gas);
                }
                bool seam = gjr < 0 || gjr >= nj;
                if (seam) pack_cell<T>(p, u);
                if (seam || !ASYNC_U)
                    for (int k = 0; k < 5; ++k) sU[k * NL + w] = u[k];
                sP[w] = p.p;
                sQ[0 * NL + w] = p.vx;
                sQ[1 * NL + w] = p.vy;
                sQ[2 * NL + w] = p.t;
                sQ[3 * NL + w] = p.nut;
            }
        }
    }
    JST_SYNC();

    // ---- A2: ghost rows from the staged primitives -----------------------
    const bool wall_tile = i0 == 0;
    const bool far_tile = i0 + TI + 3 > ni;
    if (far_tile) {  // far-field state per staged column (boundary.rs:87-155)
        const int lrow = ni - 1 - i0 + 3;  // staged row of cell NI-1
        for (int lj = tid; lj < LJ; lj += NT) {
            int gj = wrapj(j0 - 3 + lj, nj);
            int o = lrow * LJ + lj;
            double nu[3] = {(double)sQ[3 * NL + o], (double)sQ[3 * NL + o - LJ], (double)sQ[3 * NL + o - 2 * LJ]};
            const double* fg = I.far + 5 * (long)gj;
            double dist[3] = {ld(fg + 2), ld(fg + 3), ld(fg + 4)};
            double t = (double)sQ[2 * NL + o];
            double cs = fresh ? c.f_c : sqrt(c.rg * t);
            FarState f = riemann_face(ld(fg + 0), ld(fg + 1), (double)sQ[o], (double)sQ[NL + o], cs, dist, nu, c);
            double* fb = farbuf + 7 * lj;
            fb[0] = f.rho;
            fb[1] = f.p;
            fb[2] = f.t;
            fb[3] = f.vx;
            fb[4] = f.vy;
            fb[5] = f.e;
            fb[6] = f.nut;
        }
        JST_SYNC();
    }
    if (wall_tile || far_tile) {
        for (int w = tid; w < NL; w += NT) {
            int li = w / LJ, lj = w - li * LJ;
            int gi = i0 - 3 + li;
            if (gi >= 0 && gi < ni) continue;
            Prim<T> q;
            if (gi < 0) {  // wall mirror of cell k = -1-gi (boundary.rs:30-51)
                int os = (-1 - gi + 3) * LJ + lj;
                q.rho = sU[os];
                q.p = sP[os];
                q.t = sQ[2 * NL + os];
                q.vx = -sQ[os];
                q.vy = -sQ[NL + os];
                q.nut = -sQ[3 * NL + os];
                q.e = fresh ? (T)c.f_e : sU[3 * NL + os] * dv<T, true>(T(1), q.rho);
            } else {
                const double* fb = farbuf + 7 * lj;
                q.rho = (T)fb[0];
                q.p = (T)fb[1];
                q.t = (T)fb[2];
                q.vx = (T)fb[3];
                q.vy = (T)fb[4];
                q.e = (T)fb[5];
                q.nut = (T)fb[6];
            }
            T u[5];
            pack_cell<T>(q, u);
            for (int k = 0; k < 5; ++k) sU[k * NL + w] = u[k];
            sP[w] = q.p;
            sQ[0 * NL + w] = q.vx;
            sQ[1 * NL + w] = q.vy;
            sQ[2 * NL + w] = q.t;
            sQ[3 * NL + w] = q.nut;
        }
        JST_SYNC();
    }

    // ---- B1: pressure sensors (dissipation.rs:73-90) ---------------------
    for (int w = tid; w < L::NSI; w += NT) {  // i-direction, rows i0-2 .. i0+TI+1
        int r = w / TJ, tj = w - r * TJ;
        int o = (r + 1) * LJ + tj + 3;
        sSi[w] = pressure_sensor<T, true>(sP[o - LJ], sP[o], sP[o + LJ]);
    }
    for (int w = tid; w < L::NSJ; w += NT) {  // j-direction, columns j0-2 .. j0+TJ+1
        int ti = w / (TJ + 4), cc = w - ti * (TJ + 4);
        int o = (ti + 3) * LJ + cc + 1;
        sSj[w] = pressure_sensor<T, true>(sP[o - 1], sP[o], sP[o + 1]);
    }

    // ---- B2: gradients, diffusion tensors (tile + ring), SA source (tile) -
    for (int w = tid; w < NR; w += NT) {
        int ri = w / RJ, rj = w - ri * RJ;
        int gi = i0 - 1 + ri;
        int li = ri + 2, lj = rj + 2;
        T g[8];
        if (gi >= ni) {
            for (int k = 0; k < 8; ++k) g[k] = T(0);  // far ghost ring (gradient.rs:96)
        } else {
            // the wall ghost ring takes cell 0's gradient with grad T = 0 (gradient.rs:93-95)
            int ci = gi < 0 ? 0 : gi;
            int cl = gi < 0 ? li + 1 : li;
            int rt = ci - i0 + 1;  // geometry row of cell ci in the tau / n / ring boxes
            int tdn = rt * L::GTJ + rj, tup = tdn + L::GTJ;
            int nlf = rt * L::GNJ + rj, nrt = nlf + 1;
            T upx = (T)gs[L::gTx + tup], upy = (T)gs[L::gTy + tup];
            T dnx = (T)gs[L::gTx + tdn], dny = (T)gs[L::gTy + tdn];
            T lfx = (T)gs[L::gNx + nlf], lfy = (T)gs[L::gNy + nlf];
            T rtx = (T)gs[L::gNx + nrt], rty = (T)gs[L::gNy + nrt];
            T iv = (T)gs[L::gIV + rt * RJ + rj];
            int o = cl * LJ + lj;
            for (int q = 0; q < 4; ++q) {
                const T* f = sQ + q * NL;
                if (sizeof(T) == sizeof(double))
                    green_gauss<T>(f[o], f[o + LJ], f[o - LJ], f[o - 1], f[o + 1], upx, upy, dnx, dny, lfx, lfy, rtx,
                                   rty, iv, &g[2 * q], &g[2 * q + 1]);
                else
                    green_gauss_delta<T>(f[o], f[o + LJ], f[o - LJ], f[o - 1], f[o + 1], upx, upy, dnx, dny, lfx,
                                         lfy, rtx, rty, iv, &g[2 * q], &g[2 * q + 1]);
            }
            if (gi < 0) {
                g[4] = T(0);
                g[5] = T(0);
            }
        }
        int o = li * LJ + lj;
        Diff<T> d = diffusion_tensor<T, true>(sQ[2 * NL + o], sU[4 * NL + o], sQ[0 * NL + o], sQ[1 * NL + o],
                                              g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], (T)c.inv_t_ref,
                                              (T)c.suth_num, (T)c.t_suth, (T)c.cv1_cubed, (T)c.inv_pr,
                                              (T)c.inv_prt, (T)c.cp, (T)c.sigma);
        sD[0 * NR + w] = d.dx1;
        sD[1 * NR + w] = d.dx2;
        sD[2 * NR + w] = d.dx3;
        sD[3 * NR + w] = d.dx4;
        sD[4 * NR + w] = d.dy1;
        sD[5 * NR + w] = d.dy2;
        sD[6 * NR + w] = d.dy3;
        sD[7 * NR + w] = d.dy4;
        if (ri >= 1 && ri <= TI && rj >= 1 && rj <= TJ) {
            int tcell = (ri - 1) * TJ + (rj - 1);
            T s5 = sa_source<T, true>(sU[o], sU[4 * NL + o], (T)gs[L::gD2 + tcell], d.chi, d.fv1, g[2], g[1], g[6],
                                      g[7], c);
            sS[tcell] = s5 * (T)gs[L::gV + tcell];
        }
    }
    JST_SYNC();

    const T half_cfl = (T)c.half_cfl, k2 = (T)c.k2, k4 = (T)c.k4, gm1 = (T)c.gm1;
    const T p_ref = sizeof(T) == sizeof(double) ? T(0) : (T)c.p_inf;  // see euler_flux

    // ---- C: net face fluxes G = conv - visc - diss, each face once -------
    T* sFt = sm + L::oX;               // tau faces i0 .. i0+TI (aliases the dead P, Q)
    T* sFn = sFt + 5 * L::NFT;         // n faces j0 .. j0+TJ
    for (int w = tid; w < L::NFT + L::NFN; w += NT) {
        T nx, ny, lam, e2, e4;
        int lo, step, da, db;
        bool tau = w < L::NFT;
        if (tau) {
            int r = w / TJ, tj = w - r * TJ;
            int f = i0 + r, gj = j0 + tj;
            if (f > ni || gj >= nj) continue;
            int gt = (r + 1) * L::GTJ + tj + 1;
            nx = (T)gs[L::gTx + gt];
            ny = (T)gs[L::gTy + gt];
            lo = (r + 3) * LJ + (tj + 3);  // cell f; cell f-1 is lo - LJ
            step = LJ;
            da = r * RJ + (tj + 1);        // ring cells f-1, f
            db = da + RJ;
            T m = tmax<T>(tmax<T>(tmax<T>(sSi[r * TJ + tj], sSi[(r + 1) * TJ + tj]), sSi[(r + 2) * TJ + tj]),
                          sSi[(r + 3) * TJ + tj]);
            e2 = k2 * m;
        } else {
            int v = w - L::NFT;
            int ti = v / (TJ + 1), cc = v - ti * (TJ + 1);
            int gi = i0 + ti, jf = j0 + cc;
            if (gi >= ni || jf > nj) continue;
            int gn = (ti + 1) * L::GNJ + cc + 1;
            nx = (T)gs[L::gNx + gn];
            ny = (T)gs[L::gNy + gn];
            lo = (ti + 3) * LJ + (cc + 3);  // cell jf; cell jf-1 is lo - 1
            step = 1;
            db = (ti + 1) * RJ + (cc + 1);
            da = db - 1;
            const T* S = sSj + ti * (TJ + 4) + cc;
            T m = tmax<T>(tmax<T>(tmax<T>(S[0], S[1]), S[2]), S[3]);
            e2 = k2 * m;
        }
        e4 = tmax<T>(k4 - e2, T(0));
        lam = half_cfl * (sRat[db] + sRat[da]);
        T fu[5], cv[5];
        for (int k = 0; k < 5; ++k) fu[k] = T(0.5) * (sU[k * NL + lo - step] + sU[k * NL + lo]);
        euler_flux<T, true>(fu, nx, ny, gm1, cv, p_ref);
        T hx = T(0.5) * nx, hy = T(0.5) * ny;
        T* out = tau ? sFt + w : sFn + (w - L::NFT);
        const int ostride = tau ? L::NFT : L::NFN;
        for (int k = 0; k < 5; ++k) {
            const T* U = sU + k * NL;
            T d1 = U[lo] - U[lo - step];
            T d3 = U[lo + step] - T(3) * U[lo] + T(3) * U[lo - step] - U[lo - 2 * step];
            T vis = T(0);
            if (k > 0)
                vis = (sD[(k - 1) * NR + da] + sD[(k - 1) * NR + db]) * hx +
                      (sD[(k + 3) * NR + da] + sD[(k + 3) * NR + db]) * hy;
            out[k * ostride] = cv[k] - vis - lam * (d1 * e2 - d3 * e4);
        }
    }
    JST_SYNC();

    // ---- D: RK update, unpack check, last-stage epilogue -----------------
    double mloc = __longlong_as_double(0x7ff0000000000000LL);
    double sres = 0.0;
    for (int w = tid; w < TT; w += NT) {
        int ti = w / TJ, tj = w - ti * TJ;
        int gi = i0 + ti, gj = j0 + tj;
        if (gi >= ni || gj >= nj) continue;
        long id = (long)gi * nj + gj;
        double uo[5];
        for (int k = 0; k < 5; ++k) uo[k] = I.un[k][id];
        T R[5];
        const int fd = ti * (TJ + 1) + tj;
        for (int k = 0; k < 5; ++k)
            R[k] = (sFt[k * L::NFT + w + TJ] - sFt[k * L::NFT + w]) + (sFn[k * L::NFN + fd + 1] - sFn[k * L::NFN + fd]);
        R[4] -= sS[w];
        if constexpr (DUMP) {
            for (int k = 0; k < 5; ++k) I.rdump[k * (long)ni * nj + id] = (double)R[k];
            continue;
        }
        int rc = (ti + 1) * RJ + tj + 1;  // ring index of the cell
        double a = I.local_dt ? alpha * ld(I.ldt + id) : adt_s;
        double sc = a * gs[L::gIV + rc];
        double un[5];
        for (int k = 0; k < 5; ++k) {
            if (sizeof(T) == sizeof(double)) un[k] = uo[k] - (double)R[k] * sc;
            else un[k] = uo[k] - (double)(R[k] * (T)sc);  // FP32 increment, FP64 accumulator
            dst[k][id] = (TD)un[k];
            if (LAST && sizeof(T) != sizeof(double)) I.uc[k][id] = (T)un[k];
        }
        // unpack checks (solver.rs:160-171), on the stored precision
        bool bad;
        Prim<double> q{};
        if (sizeof(T) == sizeof(double)) {
            double rho = un[0];
            bad = isnan(rho) || rho <= 1e-15;
            if (!bad) {
                q = unpack_cell<double, true>(un[0], un[1], un[2], un[3], un[4], c.gm1, c.r_gas);
                bad = isnan(q.p) || q.p <= 1e-15;
            }
        } else {
            T rho = (T)un[0];
            bad = isnan(rho) || rho <= T(1e-15);
            if (!bad) {
                Prim<T> qt = unpack_cell<T, true>(rho, (T)un[1], (T)un[2], (T)un[3], (T)un[4], (T)c.gm1, (T)c.r_gas);
                bad = isnan(qt.p) || qt.p <= T(1e-15);
                q.vx = qt.vx;
                q.vy = qt.vy;
                q.t = qt.t;
            }
        }
        if (bad) {
            atomicMin(&I.st->bad, (stage_id << 32) | (unsigned long long)id);
            continue;
        }
        if (LAST) {
            double d = un[0] - uo[0];  // solver.rs:195
            sres += d * d;
            // timestep.rs:30-42 from the staged geometry, in the stage arithmetic
            int tdn = (ti + 1) * L::GTJ + tj + 1, tup = tdn + L::GTJ;
            int nlf = (ti + 1) * L::GNJ + tj + 1, nrt = nlf + 1;
            T aa = T(0.5) * ((T)gs[L::gTx + tdn] + (T)gs[L::gTx + tup]);
            T bb = T(0.5) * ((T)gs[L::gTy + tdn] + (T)gs[L::gTy + tup]);
            T cc = T(0.5) * ((T)gs[L::gNx + nlf] + (T)gs[L::gNx + nrt]);
            T dd = T(0.5) * ((T)gs[L::gNy + nlf] + (T)gs[L::gNy + nrt]);
            T vol = (T)gs[L::gV + w];
            T qvx = (T)q.vx, qvy = (T)q.vy, qt = (T)q.t;
            T dl = local_dt<T, true>(qvx, qvy, sq<T, true>((T)c.rg * qt), aa, bb, cc, dd, (T)c.cfl * vol);
            ratio_next[id] = dv<T, true>(vol, dl);
            if (I.local_dt) I.ldt[id] = (double)dl;
            mloc = fmin(mloc, (double)dl);
        }
    }
    if (LAST) {
        double mn = block_min<NT>(mloc, red);
        double sr = block_sum<NT>(sres, red);
        if (tid == 0) {
            I.partial[2 * tr.tile] = mn;
            I.partial[2 * tr.tile + 1] = sr;
            JST_FENCE();
            unsigned prev = atomicAdd(&I.st->counter, 1u);
            flags[3] = prev == (unsigned)(I.ntiles - 1);
        }
        JST_SYNC();
        if (flags[3]) {
            JST_FENCE();
            finish_step<T, NT>(I, true, red);
        }
    }
    JST_SYNC();  // shared memory is reused by the next item
    }
}

}  // namespace fused
}  // namespace jst
