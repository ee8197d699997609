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

#include <type_traits>

#include "jst_common.cuh"

#ifndef JST_DYN_SMEM
#define JST_DYN_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#endif
#ifndef JST_TID
#define JST_TID() ((int)threadIdx.x)
#define JST_BID() ((int)blockIdx.x)
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
    unsigned long long bad;  // (stage_id << 32) | cell, NO_BAD when none
    unsigned int counter;    // last-block-done counter
    int step;          // completed steps
    int fresh;         // 1 until the first step completed: stage 0 uses the free-stream primitives
    int done;          // residual fell below target
    int max_step;      // device-side step limit (steps beyond it are skipped)
    int pad;
};

// Per-instance descriptor (read-only during a launch except through `st`).
template <class T> struct Inst {
    int ni, nj;
    int ntiles;       // tiles of this instance
    int local_dt;     // JST_DT_LOCAL
    // geometry, FP64 (geometry.rs:45-63)
    const double *tnx, *tny, *nnx, *nny, *vol, *inv_vol, *inv_d2;
    const double* far;  // per column j: tau(NI) normal x,y and centroid distances of cells NI-1..NI-3 (5*nj)
    // state
    double* un[5];      // U_n, the FP64 step-start state
    T* ua[5];           // stage ping-pong buffers
    T* ub[5];
    T* ratio[2];        // V / localdt, indexed by step parity (dissipation.rs:51-56)
    double* ldt;        // localdt of the current step (local time stepping)
    double* partial;    // per tile: min localdt, sum (drho)^2
    double* res_hist;   // residual per completed step (may be null)
    InstState* st;
    PhysConst c;
};

struct TileRef {
    int inst, i0, j0, tile;  // tile = index within its instance
};

template <class T, int TI, int TJ, int NT> struct Layout {
    static constexpr int LI = TI + 6, LJ = TJ + 6, NL = LI * LJ;  // staged cells (halo 3)
    static constexpr int RI = TI + 2, RJ = TJ + 2, NR = RI * RJ;  // tile + first ring
    static constexpr int NSI = (TI + 4) * TJ, NSJ = TI * (TJ + 4);
    static constexpr int NFT = (TI + 1) * TJ, NFN = TI * (TJ + 1);
    // offsets in elements of T
    static constexpr int oU = 0;
    static constexpr int oP = oU + 5 * NL;
    static constexpr int oQ = oP + NL;  // u, v, T, nut
    static constexpr int oSi = oQ + 4 * NL;
    static constexpr int oSj = oSi + NSI;
    static constexpr int oD = oSj + NSJ;  // Dx1..4, Dy1..4
    static constexpr int oG = oD + 8 * NR;  // dvdx, dudy, dnutdx, dnutdy, chi, fv1 (tile cells)
    static constexpr int oFt = oG + 6 * TI * TJ;
    static constexpr int oFn = oFt + 5 * NFT;
    static constexpr int total = oFn + 5 * NFN;
    static constexpr size_t red_off = ((size_t)total * sizeof(T) + 15) / 16 * 16;  // reduction + far buffers
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
template <int NT> JST_D double block_sum(double v, double* red) {
    int t = JST_TID();
    red[t] = v;
    JST_SYNC();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if (t < w) red[t] += red[t + w];
        JST_SYNC();
    }
    double r = red[0];
    JST_SYNC();
    return r;
}

template <int NT> JST_D double block_min(double v, double* red) {
    int t = JST_TID();
    red[t] = v;
    JST_SYNC();
    for (int w = NT / 2; w > 0; w >>= 1) {
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
            st->step = step + 1;
            st->fresh = 0;
            if (res < st->target) st->done = 1;
        }
        st->counter = 0;
    }
}

// Local time steps of every cell of one tile from U_n (or the free stream),
// plus the per-instance minimum: the time step of the first step and of any
// step after the state was overwritten (timestep.rs:24-57).
template <class T, int NT>
__global__ void __launch_bounds__(NT) k_step_dt(const TileRef* tiles, const Inst<T>* insts, int TI, int TJ) {
    __shared__ double red[NT];
    __shared__ int last;
    TileRef tr = tiles[JST_BID()];
    const Inst<T>& I = insts[tr.inst];
    int fresh = I.st->fresh;
    double mloc = __longlong_as_double(0x7ff0000000000000LL);
    for (int w = JST_TID(); w < TI * TJ; w += NT) {
        int i = tr.i0 + w / TJ, j = tr.j0 + w % TJ;
        if (i >= I.ni || j >= I.nj) continue;
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
}

// The stage kernel.  FIRST: stage 0 (reads U_n, adds dt to the total time).
// LAST: stage 4 (writes U_n in place, residual, next step's time step).
template <class T, int TI, int TJ, int NT, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT) k_stage(const TileRef* tiles, const Inst<T>* insts, int stage, double alpha) {
    using L = Layout<T, TI, TJ, NT>;
    using TS = typename std::conditional<FIRST, double, T>::type;
    using TD = typename std::conditional<LAST, double, T>::type;
    JST_DYN_SMEM(smem_raw);
    T* sm = reinterpret_cast<T*>(smem_raw);
    double* red = reinterpret_cast<double*>(smem_raw + L::red_off);
    double* farbuf = red + NT;  // 7 values per staged column when the tile touches the far field
    __shared__ int flags[4];

    const TileRef tr = tiles[JST_BID()];
    const Inst<T>& I = insts[tr.inst];
    const int ni = I.ni, nj = I.nj, i0 = tr.i0, j0 = tr.j0;
    const PhysConst& c = I.c;
    const int tid = JST_TID();

    if (tid == 0) {
        InstState* st = I.st;
        int step = st->step;
        unsigned long long stage_id = (unsigned long long)step * 5 + stage;
        unsigned long long bad = st->bad;
        int skip = st->done || step >= st->max_step || (bad != NO_BAD && (bad >> 32) < stage_id);
        flags[0] = skip;
        flags[1] = FIRST ? st->fresh : 0;
        flags[2] = step;
        if (FIRST && !skip && tr.tile == 0) st->totaltime += st->dt;
    }
    JST_SYNC();
    if (flags[0]) return;
    const int fresh = flags[1];
    const unsigned long long stage_id = (unsigned long long)flags[2] * 5 + stage;

    const TS* src[5];
    TD* dst[5];
    for (int k = 0; k < 5; ++k) {
        if (FIRST) src[k] = reinterpret_cast<const TS*>(I.un[k]);
        else src[k] = reinterpret_cast<const TS*>((stage % 2 == 1) ? I.ua[k] : I.ub[k]);
        if (LAST) dst[k] = reinterpret_cast<TD*>(I.un[k]);
        else dst[k] = reinterpret_cast<TD*>((stage % 2 == 0) ? I.ua[k] : I.ub[k]);
    }

    const T* ratio = I.ratio[flags[2] & 1];
    T* ratio_next = I.ratio[(flags[2] + 1) & 1];
    (void)ratio_next;
    T* sU = sm + L::oU;
    T* sP = sm + L::oP;
    T* sQ = sm + L::oQ;
    T* sSi = sm + L::oSi;
    T* sSj = sm + L::oSj;
    T* sD = sm + L::oD;
    T* sG = sm + L::oG;
    T* sFt = sm + L::oFt;
    T* sFn = sm + L::oFn;
    constexpr int LJ = L::LJ, NL = L::NL, RJ = L::RJ, NR = L::NR;

    // ---- far-field states of the staged columns (boundary.rs:87-155) -----
    const bool touches_far = i0 + TI + 3 > ni;
    if (touches_far) {
        for (int lj = tid; lj < LJ; lj += NT) {
            int gj = wrapj(j0 - 3 + lj, nj);
            long cid = (long)(ni - 1) * nj + gj;
            T u[5];
            Prim<T> q = prim_from<T, TS>(src, cid, fresh, c, u);
            double nu[3], dist[3];
            nu[0] = (double)q.nut;
            for (int k = 1; k < 3; ++k) {
                T u2[5];
                Prim<T> q2 = prim_from<T, TS>(src, (long)(ni - 1 - k) * nj + gj, fresh, c, u2);
                nu[k] = (double)q2.nut;
            }
            const double* fg = I.far + 5 * (long)gj;
            dist[0] = ld(fg + 2);
            dist[1] = ld(fg + 3);
            dist[2] = ld(fg + 4);
            double cs = fresh ? c.f_c : sqrt(c.rg * (double)q.t);
            FarState f = riemann_face(ld(fg + 0), ld(fg + 1), (double)q.vx, (double)q.vy, cs, dist, nu, c);
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

    // ---- phase A: stage the tile + halo, build ghosts, primitives ---------
    for (int w = tid; w < NL; w += NT) {
        int li = w / LJ, lj = w - li * LJ;
        int gi = i0 - 3 + li, gjr = j0 - 3 + lj;
        int gj = wrapj(gjr, nj);
        T u[5];
        Prim<T> q;
        if (gi >= 0 && gi < ni) {
            q = prim_from<T, TS>(src, (long)gi * nj + gj, fresh, c, u);
            if (gjr < 0 || gjr >= nj) pack_cell<T>(q, u);  // periodic ghost (boundary.rs:54-72)
        } else if (gi < 0) {
            int k = -1 - gi;  // wall mirror of cell k (boundary.rs:30-51)
            q = prim_from<T, TS>(src, (long)k * nj + gj, fresh, c, u);
            q.vx = -q.vx;
            q.vy = -q.vy;
            q.nut = -q.nut;
            pack_cell<T>(q, u);
        } else {
            const double* fb = farbuf + 7 * lj;
            q.rho = (T)fb[0];
            q.p = (T)fb[1];
            q.t = (T)fb[2];
            q.vx = (T)fb[3];
            q.vy = (T)fb[4];
            q.e = (T)fb[5];
            q.nut = (T)fb[6];
            pack_cell<T>(q, u);
        }
        for (int k = 0; k < 5; ++k) sU[k * NL + w] = u[k];
        sP[w] = q.p;
        sQ[0 * NL + w] = q.vx;
        sQ[1 * NL + w] = q.vy;
        sQ[2 * NL + w] = q.t;
        sQ[3 * NL + w] = q.nut;
    }
    JST_SYNC();

    // ---- phase B1: pressure sensors (dissipation.rs:73-90) ---------------
    for (int w = tid; w < L::NSI; w += NT) {  // i-direction, rows i0-2 .. i0+TI+1
        int r = w / TJ, tj = w - r * TJ;
        int li = r + 1, lj = tj + 3;
        sSi[w] = pressure_sensor<T>(sP[(li - 1) * LJ + lj], sP[li * LJ + lj], sP[(li + 1) * LJ + lj]);
    }
    for (int w = tid; w < L::NSJ; w += NT) {  // j-direction, columns j0-2 .. j0+TJ+1
        int ti = w / (TJ + 4), cc = w - ti * (TJ + 4);
        int li = ti + 3, lj = cc + 1;
        sSj[w] = pressure_sensor<T>(sP[li * LJ + lj - 1], sP[li * LJ + lj], sP[li * LJ + lj + 1]);
    }

    // ---- phase B2: gradients + diffusion tensors on tile + ring ----------
    for (int w = tid; w < NR; w += NT) {
        int ri = w / RJ, rj = w - ri * RJ;
        int gi = i0 - 1 + ri, gjr = j0 - 1 + rj;
        int li = ri + 2, lj = rj + 2;
        T g[8];
        if (gi >= ni) {
            for (int k = 0; k < 8; ++k) g[k] = T(0);  // far ghost ring (gradient.rs:96)
        } else {
            // wall ghost ring takes the gradient of cell 0 (gradient.rs:93-95)
            int ci = gi < 0 ? 0 : gi;
            int cl = gi < 0 ? li + 1 : li;
            int gj = wrapj(gjr, nj);
            int jp = gj + 1 < nj ? gj + 1 : 0;
            long up = (long)(ci + 1) * nj + gj, dn = (long)ci * nj + gj, lf = dn, rt = (long)ci * nj + jp;
            T upx = (T)ld(I.tnx + up), upy = (T)ld(I.tny + up), dnx = (T)ld(I.tnx + dn), dny = (T)ld(I.tny + dn);
            T lfx = (T)ld(I.nnx + lf), lfy = (T)ld(I.nny + lf), rtx = (T)ld(I.nnx + rt), rty = (T)ld(I.nny + rt);
            T iv = (T)ld(I.inv_vol + dn);
            int o = cl * LJ + lj;
            for (int q = 0; q < 4; ++q) {
                const T* f = sQ + q * NL;
                green_gauss<T>(f[o], f[o + LJ], f[o - LJ], f[o - 1], f[o + 1], upx, upy, dnx, dny, lfx, lfy, rtx,
                               rty, iv, &g[2 * q], &g[2 * q + 1]);
            }
            if (gi < 0) {
                g[4] = T(0);
                g[5] = T(0);
            }
        }
        int o = li * LJ + lj;
        Diff<T> d = diffusion_tensor<T>(sQ[2 * NL + o], sU[4 * NL + o], sQ[0 * NL + o], sQ[1 * NL + o], g[0], g[1],
                                        g[2], g[3], g[4], g[5], g[6], g[7], (T)c.inv_t_ref, (T)c.suth_num,
                                        (T)c.t_suth, (T)c.cv1_cubed, (T)c.inv_pr, (T)c.inv_prt, (T)c.cp,
                                        (T)c.sigma);
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
            sG[0 * TI * TJ + tcell] = g[2];  // dvdx
            sG[1 * TI * TJ + tcell] = g[1];  // dudy
            sG[2 * TI * TJ + tcell] = g[6];  // dnutdx
            sG[3 * TI * TJ + tcell] = g[7];  // dnutdy
            sG[4 * TI * TJ + tcell] = d.chi;
            sG[5 * TI * TJ + tcell] = d.fv1;
        }
    }
    JST_SYNC();

    const T half_cfl = (T)c.half_cfl, k2 = (T)c.k2, k4 = (T)c.k4, gm1 = (T)c.gm1;

    // ---- phase C: net face fluxes G = conv - visc - diss -----------------
    for (int w = tid; w < L::NFT; w += NT) {  // tau faces i0 .. i0+TI
        int r = w / TJ, tj = w - r * TJ;
        int f = i0 + r, gj = j0 + tj;
        if (f > ni || gj >= nj) continue;
        long fid = (long)f * nj + gj;
        T nx = (T)ld(I.tnx + fid), ny = (T)ld(I.tny + fid);
        int lo = (r + 3) * LJ + (tj + 3);  // cell f (cell f-1 is lo - LJ)
        T fu[5], cv[5];
        for (int k = 0; k < 5; ++k) fu[k] = T(0.5) * (sU[k * NL + lo - LJ] + sU[k * NL + lo]);
        euler_flux<T>(fu, nx, ny, gm1, cv);
        int da = r * RJ + (tj + 1), db = da + RJ;  // D of cells f-1, f
        T hx = T(0.5) * nx, hy = T(0.5) * ny;
        int a = f < ni - 1 ? f : ni - 1, b = f - 1 > 0 ? f - 1 : 0;
        if (a < 0) a = 0;
        if (b > ni - 1) b = ni - 1;
        T lam = half_cfl * (ld(ratio + (long)a * nj + gj) + ld(ratio + (long)b * nj + gj));
        T m = tmax<T>(tmax<T>(tmax<T>(sSi[r * TJ + tj], sSi[(r + 1) * TJ + tj]), sSi[(r + 2) * TJ + tj]),
                      sSi[(r + 3) * TJ + tj]);
        T e2 = k2 * m, e4 = tmax<T>(k4 - e2, T(0));
        for (int k = 0; k < 5; ++k) {
            const T* U = sU + k * NL;
            T d1 = U[lo] - U[lo - LJ];
            T d3 = U[lo + LJ] - T(3) * U[lo] + T(3) * U[lo - LJ] - U[lo - 2 * LJ];
            T vis = T(0);
            if (k > 0)
                vis = (sD[(k - 1) * NR + da] + sD[(k - 1) * NR + db]) * hx +
                      (sD[(k + 3) * NR + da] + sD[(k + 3) * NR + db]) * hy;
            sFt[k * L::NFT + w] = cv[k] - vis - lam * (d1 * e2 - d3 * e4);
        }
    }
    for (int w = tid; w < L::NFN; w += NT) {  // n faces j0 .. j0+TJ
        int ti = w / (TJ + 1), cc = w - ti * (TJ + 1);
        int gi = i0 + ti, jf = j0 + cc;
        if (gi >= ni || jf > nj) continue;
        int jw = jf >= nj ? jf - nj : jf;
        int jm = jw > 0 ? jw - 1 : nj - 1;
        long fid = (long)gi * nj + jw;
        T nx = (T)ld(I.nnx + fid), ny = (T)ld(I.nny + fid);
        int lo = (ti + 3) * LJ + (cc + 3);  // cell jf (cell jf-1 is lo - 1)
        T fu[5], cv[5];
        for (int k = 0; k < 5; ++k) fu[k] = T(0.5) * (sU[k * NL + lo - 1] + sU[k * NL + lo]);
        euler_flux<T>(fu, nx, ny, gm1, cv);
        int db = (ti + 1) * RJ + (cc + 1), da = db - 1;
        T hx = T(0.5) * nx, hy = T(0.5) * ny;
        T lam = half_cfl * (ld(ratio + fid) + ld(ratio + (long)gi * nj + jm));
        const T* S = sSj + ti * (TJ + 4) + cc;
        T m = tmax<T>(tmax<T>(tmax<T>(S[0], S[1]), S[2]), S[3]);
        T e2 = k2 * m, e4 = tmax<T>(k4 - e2, T(0));
        for (int k = 0; k < 5; ++k) {
            const T* U = sU + k * NL;
            T d1 = U[lo] - U[lo - 1];
            T d3 = U[lo + 1] - T(3) * U[lo] + T(3) * U[lo - 1] - U[lo - 2];
            T vis = T(0);
            if (k > 0)
                vis = (sD[(k - 1) * NR + da] + sD[(k - 1) * NR + db]) * hx +
                      (sD[(k + 3) * NR + da] + sD[(k + 3) * NR + db]) * hy;
            sFn[k * L::NFN + w] = cv[k] - vis - lam * (d1 * e2 - d3 * e4);
        }
    }
    JST_SYNC();

    // ---- phase D: source, RK update, unpack check, last-stage epilogue ---
    double mloc = __longlong_as_double(0x7ff0000000000000LL);
    double sres = 0.0;
    for (int w = tid; w < TI * TJ; w += NT) {
        int ti = w / TJ, tj = w - ti * TJ;
        int gi = i0 + ti, gj = j0 + tj;
        if (gi >= ni || gj >= nj) continue;
        long id = (long)gi * nj + gj;
        int lo = (ti + 3) * LJ + (tj + 3);
        T src5 = sa_source<T>(sU[lo], sU[4 * NL + lo], (T)ld(I.inv_d2 + id), sG[4 * TI * TJ + w],
                              sG[5 * TI * TJ + w], sG[0 * TI * TJ + w], sG[1 * TI * TJ + w], sG[2 * TI * TJ + w],
                              sG[3 * TI * TJ + w], c) *
                 (T)ld(I.vol + id);
        T R[5];
        for (int k = 0; k < 5; ++k)
            R[k] = (sFt[k * L::NFT + w + TJ] - sFt[k * L::NFT + w]) +
                   (sFn[k * L::NFN + ti * (TJ + 1) + tj + 1] - sFn[k * L::NFN + ti * (TJ + 1) + tj]);
        R[4] -= src5;
        double a = alpha * (I.local_dt ? ld(I.ldt + id) : I.st->dt);
        double sc = a * ld(I.inv_vol + id);
        double uo[5], un[5];
        for (int k = 0; k < 5; ++k) uo[k] = I.un[k][id];
        for (int k = 0; k < 5; ++k) {
            if (sizeof(T) == sizeof(double)) un[k] = uo[k] - (double)R[k] * sc;
            else un[k] = uo[k] - (double)(R[k] * (T)sc);  // FP32 increment, FP64 accumulator
            dst[k][id] = (TD)un[k];
        }
        // unpack checks (solver.rs:160-171)
        double rho = un[0];
        bool bad = isnan(rho) || rho <= 1e-15;
        Prim<double> q{};
        if (!bad) {
            q = unpack_cell<double>(un[0], un[1], un[2], un[3], un[4], c.gm1, c.r_gas);
            bad = isnan(q.p) || q.p <= 1e-15;
        }
        if (bad) {
            atomicMin(&I.st->bad, (stage_id << 32) | (unsigned long long)id);
            continue;
        }
        if (LAST) {
            double d = un[0] - uo[0];  // solver.rs:195
            sres += d * d;
            double dl = cell_localdt<T>(I, gi, gj, q.vx, q.vy, q.t);
            ratio_next[id] = (T)(ld(I.vol + id) / dl);
            if (I.local_dt) I.ldt[id] = dl;
            mloc = fmin(mloc, dl);
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
}

}  // namespace fused
}  // namespace jst
