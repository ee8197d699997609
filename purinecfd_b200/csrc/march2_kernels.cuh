// Paired-column marching stage kernel for the FP32/FP64 split precision.
//
// The same RK stage as k_march (march_kernels.cuh) and the same row walk, but
// each lane owns two adjacent columns, so that the cell arithmetic of both
// runs in the sm_100 paired FP32 instructions (add / mul / fma .f32x2: one
// instruction for two values) and every load and store moves both columns.
//
// Work item = a strip of 56 output columns j0 .. j0+55 and the rows
// i0 .. i1-1 of one instance.  The warp holds the 64 columns jb .. jb+63,
// jb = j0 - 4 (a 4-column halo each side, of which the stencil reads 3):
// lane L holds columns jb+2L (.x) and jb+2L+1 (.y).  Strips start at
// multiples of 56, so jb is a multiple of 4 and, on a ring with an even
// number of columns, every lane's two columns are adjacent in memory and
// 8-byte aligned (odd rings take the element-wise copies).  j-neighbours:
// column j-1 of .x is the left lane's .y and of .y the lane's own .x, so a
// one-column shift is one register shuffle per pair of values.
//
// Per row k of the walk (the phases lag as in k_march):
//   U(k) -> primitives, j-sensor(k); i-sensor(k-1);
//   gradients, diffusion tensor, SA source of row k-1;
//   tau face k-2; n faces and the RK update of row k-3.
// The formulas are the split path's (face fluxes from twice the face state
// with the pressure reference 2 p_inf, Green-Gauss in difference form, f_w
// from an FP64 g), with the products and sums contracted into paired fused
// multiply-adds; results agree with k_march to FP32 rounding.
#pragma once

namespace jst {
namespace fused {

constexpr int MARCH2_W = 56;  // output columns per strip (64 columns - 2 x 4 halo)

// ---------------------------------------------------------------- pairs ----
// Two FP32 values of one lane, .x for column jb+2L and .y for jb+2L+1.
struct P2 {
    float2 v;
};
#ifdef __CUDA_ARCH__
JST_D P2 p2(float a, float b) { return P2{make_float2(a, b)}; }
JST_D P2 sp(float a) { return P2{make_float2(a, a)}; }
JST_D P2 operator+(P2 a, P2 b) { return P2{__fadd2_rn(a.v, b.v)}; }
JST_D P2 operator*(P2 a, P2 b) { return P2{__fmul2_rn(a.v, b.v)}; }
JST_D P2 pfma(P2 a, P2 b, P2 c) { return P2{__ffma2_rn(a.v, b.v, c.v)}; }
JST_D P2 operator-(P2 a, P2 b) { return P2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }
JST_D P2 operator-(P2 a) { return P2{__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))}; }
// per element: the hardware reciprocal and square root approximations
JST_D float rcp_f(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
JST_D float sqrt_f(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
JST_D P2 prcp(P2 a) { return p2(rcp_f(a.v.x), rcp_f(a.v.y)); }
JST_D P2 pdiv(P2 a, P2 b) { return a * prcp(b); }
JST_D P2 psqrt(P2 a) { return p2(sqrt_f(a.v.x), sqrt_f(a.v.y)); }
JST_D P2 pabs(P2 a) { return p2(fabsf(a.v.x), fabsf(a.v.y)); }
JST_D P2 pmax(P2 a, P2 b) { return p2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
JST_D P2 pmin(P2 a, P2 b) { return p2(fminf(a.v.x, b.v.x), fminf(a.v.y, b.v.y)); }
JST_D P2 psel(bool cx, bool cy, P2 a, P2 b) { return p2(cx ? a.v.x : b.v.x, cy ? a.v.y : b.v.y); }
// j-neighbours of both columns: one column to the left / right, two to the left
JST_D P2 L1(P2 a) { return p2(__shfl_up_sync(0xffffffffu, a.v.y, 1), a.v.x); }
JST_D P2 R1(P2 a) { return p2(a.v.y, __shfl_down_sync(0xffffffffu, a.v.x, 1)); }
JST_D P2 L2(P2 a) { return p2(__shfl_up_sync(0xffffffffu, a.v.x, 1), __shfl_up_sync(0xffffffffu, a.v.y, 1)); }
#endif

// Geometry record pairs (Inst::mg2): per row k in 0..NI and column pair
// p = j/2, 16 floats {tau nx (col 2p, 2p+1), tau ny, n nx, n ny, 1/V, 1/d^2,
// V, 0, 0}: the tau normals of face row k and the n normals, 1/V, 1/d^2, V
// of cell row k-1 (zeros for cell row -1), i.e. the values of the Inst::mg
// record of both columns interleaved, so that every pair is one 64-bit
// value.  A ring with an odd number of columns has a last pair with one
// column (the other half zero).
enum { M2_TX = 0, M2_TY, M2_NX, M2_NY, M2_IV, M2_D2, M2_VOL, M2_FIELDS = 7, M2_N = 16 };
JST_HD int mg2_pairs(int nj) { return (nj + 1) / 2; }

#ifdef __CUDACC__
__global__ void k_march_geom2(const double* tnx, const double* tny, const double* nnx, const double* nny,
                              const double* inv_vol, const double* inv_d2, const double* vol, int ni, int nj,
                              float* rec) {
    const int np2 = mg2_pairs(nj);
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;  // (row, pair)
    if (q >= (long)(ni + 1) * np2) return;
    const long k = q / np2;
    const int p = (int)(q - k * np2);
    float* r = rec + M2_N * q;
    for (int e = 0; e < 2; ++e) {
        const int j = 2 * p + e;
        float f[M2_FIELDS] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (j < nj) {
            const long t = k * nj + j;
            f[M2_TX] = (float)tnx[t];
            f[M2_TY] = (float)tny[t];
            if (k >= 1) {
                const long c = t - nj;
                f[M2_NX] = (float)nnx[c];
                f[M2_NY] = (float)nny[c];
                f[M2_IV] = (float)inv_vol[c];
                f[M2_D2] = (float)inv_d2[c];
                f[M2_VOL] = (float)vol[c];
            }
        }
        for (int g = 0; g < M2_FIELDS; ++g) r[2 * g + e] = f[g];
    }
    r[14] = r[15] = 0.f;
}
#endif

// One row's global inputs of a warp, staged one row ahead: [field][lane].
struct MarchRow2 {
    float4 rec[4][32];   // Inst::mg2 record pair of row k: {TX, TY}, {NX, NY}, {IV, D2}, {VOL, 0}
    float2 u[5][32];     // stage input of row k
    float2 uacc[5][32];  // FP32 copy of U_n of row k-3 (stages 1-3)
    double2 un[5][32];   // U_n of row k-3 (last stage)
    double2 ldt[32];     // local time step of row k-3 (local time stepping)
    double2 ivm[32];     // 1/V of row k-3
    float2 rat[32];      // V/dt of row k-2 (clamped)
};

// The 4-row U window lives in a per-warp shared ring of 5 rows (in
// registers it would take 40 of them and push the kernel into spills).
struct MarchURing2 {
    float2 u[5][5][32];  // [row slot][variable][lane]
};

template <int NT> constexpr size_t march2_smem_bytes() {
    return (size_t)(NT / 32) * (2 * sizeof(MarchRow2) + sizeof(MarchURing2) + (sizeof(ConstP) + 15) / 16 * 16);
}

#ifdef __CUDA_ARCH__
// Primitive state of both columns (solver.rs:158-181 without the checks).
struct Prim2 {
    P2 rho, p, t, vx, vy, e, nut;
};
JST_D Prim2 unpack2(const P2* u, P2 gm1, P2 r_gas) {
    Prim2 q;
    const P2 inv = prcp(u[0]);
    q.rho = u[0];
    q.vx = u[1] * inv;
    q.vy = u[2] * inv;
    q.e = u[3] * inv;
    const P2 ke = pfma(q.vx, q.vx, q.vy * q.vy);
    q.p = gm1 * pfma(u[0] * ke, sp(-0.5f), u[3]);
    q.t = pdiv(q.p, r_gas * u[0]);
    q.nut = u[4] * inv;
    return q;
}
JST_D void pack2(const Prim2& q, P2* u) {
    u[0] = q.rho;
    u[1] = q.rho * q.vx;
    u[2] = q.rho * q.vy;
    u[3] = q.rho * q.e;
    u[4] = q.rho * q.nut;
}
// convection::euler_flux (convection.rs:25-40) of the doubled face state
// fu = w1 + w2 with the pressure reference p_ref2 = 2 p_inf subtracted in the
// momentum flux (closed cells: the cell sums are unchanged)
JST_D void euler_flux2(const P2* fu, P2 nx, P2 ny, P2 gm1, P2 p_ref2, P2* out) {
    const P2 inv = prcp(fu[0]);
    const P2 u = fu[1] * inv, v = fu[2] * inv;
    const P2 p = gm1 * pfma(fu[0] * pfma(u, u, v * v), sp(-0.5f), fu[3]);
    const P2 vn = pfma(nx, u, ny * v);
    const P2 pm = p - p_ref2;
    out[0] = fu[0] * vn;
    out[1] = pfma(fu[1], vn, pm * nx);
    out[2] = pfma(fu[2], vn, pm * ny);
    out[3] = (fu[3] + p) * vn;
    out[4] = fu[4] * vn;
}
// Net face flux out = cv/2 - vis - lam (d1 e2 - d3 e4) (see face_combine in
// march_kernels.cuh), d1 = w2 - w1, d3 = (w3 - w0) + 3 (w1 - w2).
JST_D void face_combine2(const P2* w0, const P2* w1, const P2* w2, const P2* w3, const P2* cv, const P2* dA,
                         const P2* dB, P2 hx, P2 hy, P2 lam, P2 e2, P2 e4, P2* out) {
    const P2 mhx = -hx, mhy = -hy, me4 = -e4, mlam = -lam, half = sp(0.5f), three = sp(3.0f);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const P2 d1 = w2[v] - w1[v];
        const P2 d3 = pfma(w1[v] - w2[v], three, w3[v] - w0[v]);
        const P2 dis = pfma(d1, e2, d3 * me4);
        if (v > 0) {
            const P2 nvis = pfma(dA[v - 1] + dB[v - 1], mhx, (dA[v + 3] + dB[v + 3]) * mhy);
            out[v] = pfma(dis, mlam, pfma(cv[v], half, nvis));
        } else {
            out[v] = pfma(dis, mlam, cv[v] * half);
        }
    }
}
// dissipation::pressure_sensor (dissipation.rs:29-31)
JST_D P2 sensor2(P2 pm, P2 p0, P2 pp) {
    const P2 s = pm + pp;
    return pabs(pdiv(pfma(p0, sp(-2.0f), s), pfma(p0, sp(2.0f), s)));
}
// Green-Gauss gradient in difference form (green_gauss_delta); the minus
// signs of the i-1 and j-1 faces are carried by the negated normals ndn, nlf
JST_D void gg2(P2 c, P2 vup, P2 vdn, P2 vlf, P2 vrt, P2 upx, P2 upy, P2 ndnx, P2 ndny, P2 nlfx, P2 nlfy, P2 rtx,
               P2 rty, P2 h, P2* gx, P2* gy) {
    const P2 du = vup - c, dd = vdn - c, dl = vlf - c, dr = vrt - c;
    *gx = (pfma(du, upx, dd * ndnx) + pfma(dr, rtx, dl * nlfx)) * h;
    *gy = (pfma(du, upy, dd * ndny) + pfma(dr, rty, dl * nlfy)) * h;
}
struct Diff2 {
    P2 chi, fv1, d[8];  // d = dx1..dx4, dy1..dy4
};
// viscous::diffusion_tensor (viscous.rs:37-71) with Sutherland's law
// (config.rs:210-213) and fv1 (viscous.rs:27-30)
JST_D Diff2 diffusion2(P2 t, P2 rho_nu, P2 vx, P2 vy, const P2* g, const ConstP& K) {
    Diff2 o;
    const P2 r = t * P2{K.inv_t_ref};
    const P2 mu = pdiv(r * psqrt(r) * P2{K.suth_num}, t + P2{K.t_suth});
    const P2 chi = pdiv(rho_nu, mu);
    const P2 c3 = chi * chi * chi;
    const P2 f1 = pdiv(c3, c3 + P2{K.cv1_cubed});
    const P2 mu_t = rho_nu * f1;
    const P2 mu_eff = mu + mu_t;
    const P2 lam_cp = pfma(mu, P2{K.inv_pr}, mu_t * P2{K.inv_prt}) * P2{K.cp};
    // g = dudx, dudy, dvdx, dvdy, dtdx, dtdy, dnudx, dnudy
    const P2 txx = mu_eff * pfma(g[0], sp((float)(4.0 / 3.0)), g[3] * sp((float)(-2.0 / 3.0)));
    const P2 tyy = mu_eff * pfma(g[3], sp((float)(4.0 / 3.0)), g[0] * sp((float)(-2.0 / 3.0)));
    const P2 txy = mu_eff * (g[1] + g[2]);
    const P2 nu_diff = P2{K.sigma} * (mu + rho_nu);
    o.chi = chi;
    o.fv1 = f1;
    o.d[0] = txx;
    o.d[1] = txy;
    o.d[2] = pfma(vx, txx, pfma(vy, txy, lam_cp * g[4]));
    o.d[3] = nu_diff * g[6];
    o.d[4] = txy;
    o.d[5] = tyy;
    o.d[6] = pfma(vx, txy, pfma(vy, tyy, lam_cp * g[5]));
    o.d[7] = nu_diff * g[7];
    return o;
}
// source::compute for both cells (source.rs:55-85), before the factor V
JST_D P2 sa_source2(P2 rho, P2 rho_nu, P2 inv_d2, P2 chi, P2 f1, P2 dvdx, P2 dudy, P2 dnx, P2 dny,
                    const ConstP& K) {
    const P2 nu_t = pdiv(rho_nu, rho);
    const P2 inv_kd2 = inv_d2 * P2{K.inv_kappa2};
    const P2 a = chi * chi * P2{K.m_ct4};
    const P2 ft2 = P2{K.ct3} * p2(exp_f32(a.v.x), exp_f32(a.v.y));
    const P2 fv2 = sp(1.0f) - pdiv(chi, pfma(chi, f1, sp(1.0f)));
    const P2 sv = P2{K.fv3} * pabs(dvdx - dudy);
    const P2 s_t = pmax(pfma(nu_t * inv_kd2, fv2, sv), sp(1e-10f));
    const P2 prod = P2{K.cb1} * (sp(1.0f) - ft2) * s_t * rho_nu;
    const P2 r = pmin(pdiv(nu_t, s_t) * inv_kd2, P2{K.rmax});
    // fw as fw_f32 (jst_common.cuh), paired
    const P2 rc = pmax(r, sp(-1e4f));
    const P2 r2 = rc * rc;
    const P2 g = pfma(P2{K.cw2}, r2 * r2 * r2 - rc, rc);
    const P2 gf = pmin(g, sp(1e5f));
    const P2 g2 = gf * gf;
    const P2 q = pdiv(P2{K.one_plus_cw3_6}, pfma(g2 * g2, g2, P2{K.cw3_6}));
    const P2 v = gf * p2(root6_f32(q.v.x), root6_f32(q.v.y));
    const P2 fw = psel(g.v.x > 1e5f, g.v.y > 1e5f, P2{K.fw_lim}, v);
    const P2 destr = pfma(P2{K.cw1}, fw, P2{K.m_cb1_k2} * ft2) * rho * (nu_t * nu_t * inv_d2);
    const P2 diff = P2{K.cb2_sigma} * rho * pfma(dnx, dnx, dny * dny);
    return prod - destr + diff;
}
// timestep::compute for both cells (timestep.rs:30-42)
JST_D P2 local_dt2(P2 u, P2 v, P2 cs, P2 a, P2 b, P2 cc, P2 dd, P2 cfl_vol) {
    const P2 conv = pabs(pfma(u, a, v * b)) + pabs(pfma(u, cc, v * dd));
    const P2 acou = cs * (psqrt(pfma(a, a, b * b)) + psqrt(pfma(cc, cc, dd * dd)));
    return pdiv(cfl_vol, conv + acou);
}
#endif

// sched[0] = number of strips, sched[1] = work counter, sched[2] = exit counter
// (both zero at launch; the last warp to leave resets them).
// DUMP (with FIRST only): the residual R of every cell of the current state
// goes to Inst::rdump instead of an update; nothing else is written and the
// instance's step counters and stop flags are ignored.
template <int NT, bool FIRST, bool LAST, bool DUMP = false>
__global__ void __launch_bounds__(NT, 256 / NT) k_march2(const TileRef* tiles, int* sched, const Inst<float>* insts,
                                                         int stage, double alpha) {
#ifdef __CUDA_ARCH__
    using T = float;
    const int lane = JST_LANE();
    constexpr bool ACC32 = !LAST;  // stages 0-3 accumulate from the FP32 copy of U_n (see k_march)
    JST_DYN_SMEM(smem_raw);
    MarchRow2* rowbuf = reinterpret_cast<MarchRow2*>(smem_raw) + 2 * JST_WARP_IN_BLOCK();
    MarchURing2* uring =
        reinterpret_cast<MarchURing2*>(smem_raw + (size_t)(NT / 32) * 2 * sizeof(MarchRow2)) + JST_WARP_IN_BLOCK();
    // the instance's constants, copied per strip
    constexpr size_t KP = (sizeof(ConstP) + 15) / 16 * 16;
    ConstP* kp = reinterpret_cast<ConstP*>(smem_raw + (size_t)(NT / 32) * (2 * sizeof(MarchRow2) + sizeof(MarchURing2)) +
                                          KP * JST_WARP_IN_BLOCK());
    const int nt_all = sched[0];
    unsigned* work = reinterpret_cast<unsigned*>(sched + 1);
    unsigned* exitc = reinterpret_cast<unsigned*>(sched + 2);
    const unsigned nwarps = (unsigned)JST_GRID() * (NT / 32);
    for (;;) {
        unsigned ticket = 0;
        if (lane == 0) ticket = atomicAdd(work, 1u);
        ticket = jst_shfl_idx(ticket, 0);
        if (ticket >= (unsigned)nt_all) {
            if (lane == 0 && atomicAdd(exitc, 1u) == nwarps - 1) {
                *work = 0u;
                *exitc = 0u;
            }
            break;
        }
        const TileRef tr = tiles[ticket];
        const Inst<T>& I = insts[tr.inst];
        const int ni = I.ni, nj = I.nj, i0 = tr.i0, j0 = tr.j0, i1 = tr.i1;
        const PhysConst& c = I.c;
        {  // the instance's FP32 constant pairs into this warp's copy
            __syncwarp();
            const unsigned long long* s8 = reinterpret_cast<const unsigned long long*>(&I.cp);
            unsigned long long* d8 = reinterpret_cast<unsigned long long*>(kp);
            constexpr int NW = sizeof(ConstP) / 8;
            for (int w = lane; w < NW; w += 32) d8[w] = s8[w];
            __syncwarp();
        }
        const ConstP& K = *kp;

        int hdr[3] = {0, 0, 0};  // skip, fresh, step
        if (lane == 0) {
            InstState* st = I.st;
            int step = st->step;
            unsigned long long sid = (unsigned long long)step * 5 + stage;
            unsigned long long bad = st->bad;
            hdr[0] = !DUMP && (st->done || step >= st->max_step || (bad != NO_BAD && (bad >> 32) < sid));
            hdr[1] = FIRST ? st->fresh : 0;
            hdr[2] = step;
            if (FIRST && !DUMP && !hdr[0] && tr.tile == 0) st->totaltime += st->dt;
        }
        const int skip = jst_shfl_idx(hdr[0], 0);
        if (skip) continue;
        const int fresh = jst_shfl_idx(hdr[1], 0);
        const int step = jst_shfl_idx(hdr[2], 0);
        const bool dt_local = I.local_dt != 0;
        const double adt = dt_local ? alpha : alpha * I.st->dt;
        const unsigned long long stage_id = (unsigned long long)step * 5 + stage;
        const T* ratio = I.ratio[step & 1];
        T* ratio_next = I.ratio[(step + 1) & 1];
        const long np = (long)ni * nj;
        const int np2 = mg2_pairs(nj);
        const T* src = FIRST ? I.uc[0] : ((stage % 2 == 1) ? I.ua[0] : I.ub[0]);
        T* dst = (stage % 2 == 0) ? I.ua[0] : I.ub[0];

        // the lane's two columns: unwrapped, wrapped, periodic ghost, output
        const int cu0 = j0 - 4 + 2 * lane, cu1 = cu0 + 1;
        const int gj0 = wrapj(cu0, nj), gj1 = wrapj(cu1, nj);
        const bool seam0 = cu0 < 0 || cu0 >= nj, seam1 = cu1 < 0 || cu1 >= nj;
        const bool seam = seam0 || seam1;
        const bool out0 = lane >= 2 && lane < 30 && cu0 < nj, out1 = lane >= 2 && lane < 30 && cu1 < nj;
        // both columns adjacent and 8-byte aligned in every plane (always on
        // an even ring: jb and gj0 are even); else element-wise copies
        const bool pairwise = (nj & 1) == 0;
        const P2 gm1 = P2{K.gm1}, rgas = P2{K.r_gas};

        // Stage the global inputs that row kk of the walk reads (the
        // conditions are the ones under which the walk reads them).
        auto cp2 = [&](void* d, const T* base, long row) {  // two FP32 columns of one plane row
            if (pairwise) {
                async_copy<8>(d, base + row * nj + gj0);
            } else {
                async_copy<4>(d, base + row * nj + gj0);
                async_copy<4>(static_cast<float*>(d) + 1, base + row * nj + gj1);
            }
        };
        auto cp2d = [&](void* d, const double* base, long row) {  // two FP64 columns
            if (pairwise) {
                async_copy<16>(d, base + row * nj + gj0);
            } else {
                async_copy<8>(d, base + row * nj + gj0);
                async_copy<8>(static_cast<double*>(d) + 1, base + row * nj + gj1);
            }
        };
        auto issue = [&](auto steady, int kk) {
            constexpr bool S = decltype(steady)::value;
            MarchRow2& B = rowbuf[kk & 1];
            if (S || kk < ni) {
                const long row = kk < 0 ? -1 - kk : kk;
                for (int v = 0; v < 5; ++v) cp2(&B.u[v][lane], src + v * np, row);
            }
            if (S || (kk >= 0 && kk <= ni)) {
                const float* g = I.mg2 + M2_N * ((long)kk * np2);
                if (pairwise) {
                    const float* gp = g + M2_N * (gj0 >> 1);
                    for (int ch = 0; ch < 4; ++ch) async_copy<16>(&B.rec[ch][lane], gp + 4 * ch);
                } else {
                    for (int e = 0; e < 2; ++e) {
                        const int gj = e ? gj1 : gj0;
                        const float* gp = g + M2_N * (gj >> 1) + (gj & 1);
                        float* d = reinterpret_cast<float*>(&B.rec[0][lane]);
                        for (int f = 0; f < M2_FIELDS; ++f)
                            async_copy<4>(reinterpret_cast<float*>(&B.rec[f >> 1][lane]) + 2 * (f & 1) + e,
                                          gp + 2 * f);
                        (void)d;
                    }
                }
            }
            const int rr = kk - 2;
            if (S || (rr >= i0 - 1 && rr <= i1)) {
                const int gc = S ? rr : (rr < 0 ? 0 : (rr > ni - 1 ? ni - 1 : rr));
                cp2(&B.rat[lane], ratio, gc);
            }
            const int m = kk - 3;
            if (S || (m >= i0 && m < i1)) {
                if constexpr (ACC32) {
                    if constexpr (!FIRST)
                        for (int v = 0; v < 5; ++v) cp2(&B.uacc[v][lane], I.uc[0] + v * np, m);
                } else {
                    for (int v = 0; v < 5; ++v) cp2d(&B.un[v][lane], I.un[0] + v * np, m);
                }
                if (dt_local) cp2d(&B.ldt[lane], I.ldt, m);
                cp2d(&B.ivm[lane], I.inv_vol, m);
            }
        };
        issue(std::false_type{}, i0 - 3);
        async_commit();

        // sliding windows (index 0 = oldest row); U rows k-4 .. k-1 in the ring
        P2 pw[2];         // p rows k-2, k-1
        P2 qw[2][4];      // (vx, vy, T, nut) rows k-2, k-1
        P2 nu3 = sp(0.f); // nut row k-3 (far-field extrapolation)
        P2 si[3];         // i-sensor rows k-4 .. k-2
        P2 sj[3];         // j-sensor rows k-3 .. k-1
        P2 dw[2][8];      // diffusion tensor rows k-3, k-2
        P2 sw[2];         // SA source * V rows k-3, k-2
        P2 rt0 = sp(0.f); // V/dt row k-3 (rows clamped to the mesh)
        P2 ft[5];         // tau-face flux of face k-3
        P2 tx[3], ty[3];  // tau normals rows k-3 .. k-1
        P2 nx2[2], ny2[2];  // n normals (left face of each column) rows k-3, k-2
        P2 vw[2];         // V of cell rows k-3, k-2 (last stage)
        for (int sl = 0; sl < 5; ++sl)
            for (int v = 0; v < 5; ++v) uring->u[sl][v][lane] = make_float2(0.f, 0.f);
        for (int a = 0; a < 2; ++a) {
            pw[a] = sw[a] = nx2[a] = ny2[a] = vw[a] = sp(0.f);
            for (int v = 0; v < 4; ++v) qw[a][v] = sp(0.f);
            for (int v = 0; v < 8; ++v) dw[a][v] = sp(0.f);
        }
        for (int a = 0; a < 3; ++a) si[a] = sj[a] = tx[a] = ty[a] = sp(0.f);
        for (int v = 0; v < 5; ++v) ft[v] = sp(0.f);
        double mloc = __longlong_as_double(0x7ff0000000000000LL);
        double sres = 0.0;

        auto row = [&](auto steady, int k) {
            constexpr bool S = decltype(steady)::value;
            if (S) issue(steady, k + 1);
            else if (k + 1 <= i1 + 2) issue(std::false_type{}, k + 1);
            async_commit();
            async_wait_prior1();
            const MarchRow2* B = &rowbuf[k & 1];
            // U of row k-4+a (a = 0..3) from the ring; row k goes to slot s0
            const int s0 = ((k % 5) + 5) % 5;
            auto UA = [&](int a, int v) -> P2 {
                const int sl = s0 + 1 + a;
                return P2{uring->u[sl >= 5 ? sl - 5 : sl][v][lane]};
            };
            // ---- row k: conserved state and primitives ---------------------
            P2 uk[5], pk, qk[4];
            if (S || k < ni) {
                const bool wall = !S && k < 0;  // the wall ghost mirrors cell -1-k (boundary.rs:30-51)
                for (int v = 0; v < 5; ++v) uk[v] = P2{B->u[v][lane]};
                Prim2 p;
                if (fresh) {
                    p.rho = P2{K.f_rho};
                    p.p = P2{K.f_p};
                    p.t = P2{K.f_t};
                    p.vx = P2{K.f_vx};
                    p.vy = P2{K.f_vy};
                    p.e = P2{K.f_e};
                    p.nut = P2{K.f_nut};
                } else {
                    p = unpack2(uk, gm1, rgas);
                }
                if (seam) {  // periodic ghost columns (boundary.rs:54-72)
                    P2 w[5];
                    pack2(p, w);
                    for (int v = 0; v < 5; ++v) uk[v] = psel(seam0, seam1, w[v], uk[v]);
                }
                if (wall) {
                    Prim2 q;
                    q.rho = uk[0];
                    q.p = p.p;
                    q.t = p.t;
                    q.vx = -p.vx;
                    q.vy = -p.vy;
                    q.nut = -p.nut;
                    q.e = fresh ? P2{K.f_e} : pdiv(uk[3], q.rho);
                    pack2(q, uk);
                    p = q;
                }
                pk = p.p;
                qk[0] = p.vx;
                qk[1] = p.vy;
                qk[2] = p.t;
                qk[3] = p.nut;
            } else if (k == ni) {  // far-field ghost rows (boundary.rs:87-155), all three alike
                float q[2][7];
                for (int e = 0; e < 2; ++e) {
                    const int gj = e ? gj1 : gj0;
                    const double* fg = I.far + 5 * (long)gj;
                    const float nu1 = e ? qw[1][3].v.y : qw[1][3].v.x, nu2 = e ? qw[0][3].v.y : qw[0][3].v.x;
                    const float nu33 = e ? nu3.v.y : nu3.v.x;
                    double nu[3] = {(double)nu1, (double)nu2, (double)nu33};
                    double dist[3] = {ld(fg + 2), ld(fg + 3), ld(fg + 4)};
                    const double t = (double)(e ? qw[1][2].v.y : qw[1][2].v.x);
                    const double cs = fresh ? c.f_c : sqrt(c.rg * t);
                    const double ui = (double)(e ? qw[1][0].v.y : qw[1][0].v.x);
                    const double vi = (double)(e ? qw[1][1].v.y : qw[1][1].v.x);
                    FarState f = riemann_face(ld(fg + 0), ld(fg + 1), ui, vi, cs, dist, nu, c);
                    q[e][0] = (float)f.rho;
                    q[e][1] = (float)f.p;
                    q[e][2] = (float)f.t;
                    q[e][3] = (float)f.vx;
                    q[e][4] = (float)f.vy;
                    q[e][5] = (float)f.e;
                    q[e][6] = (float)f.nut;
                }
                Prim2 p;
                p.rho = p2(q[0][0], q[1][0]);
                p.p = p2(q[0][1], q[1][1]);
                p.t = p2(q[0][2], q[1][2]);
                p.vx = p2(q[0][3], q[1][3]);
                p.vy = p2(q[0][4], q[1][4]);
                p.e = p2(q[0][5], q[1][5]);
                p.nut = p2(q[0][6], q[1][6]);
                pack2(p, uk);
                pk = p.p;
                qk[0] = p.vx;
                qk[1] = p.vy;
                qk[2] = p.t;
                qk[3] = p.nut;
            } else {  // rows ni+1, ni+2 repeat row ni
                for (int v = 0; v < 5; ++v) uk[v] = UA(3, v);
                pk = pw[1];
                for (int v = 0; v < 4; ++v) qk[v] = qw[1][v];
            }
            // j-sensor of row k, i-sensor of row k-1 (dissipation.rs:73-90)
            const P2 sjk = sensor2(L1(pk), pk, R1(pk));
            const P2 sik = sensor2(pw[0], pw[1], pk);

            // ---- geometry record of row k --------------------------------------
            P2 gk[8];
            for (int e = 0; e < 8; ++e) gk[e] = sp(0.f);
            if (S || (k >= 0 && k <= ni)) {
                for (int ch = 0; ch < 4; ++ch) {
                    const float4 r4 = B->rec[ch][lane];
                    gk[2 * ch] = p2(r4.x, r4.y);
                    gk[2 * ch + 1] = p2(r4.z, r4.w);
                }
            }
            const P2 txk = gk[M2_TX], tyk = gk[M2_TY];

            // ---- gradients, diffusion tensor, SA source of row r = k-1 -----
            const int r = k - 1;
            P2 dn[8];
            for (int v = 0; v < 8; ++v) dn[v] = sp(0.f);
            P2 snew = sp(0.f), nxr = sp(0.f), nyr = sp(0.f);
            if (S || (r >= i0 - 1 && r <= i1)) {
                if (S || (r >= 0 && r < ni)) {
                    nxr = gk[M2_NX];
                    nyr = gk[M2_NY];
                    const P2 rtx = R1(nxr), rty = R1(nyr);
                    const P2 h = sp(0.5f) * gk[M2_IV];
                    const P2 ndnx = -tx[2], ndny = -ty[2], nlfx = -nxr, nlfy = -nyr;
                    P2 g[8];
                    for (int q = 0; q < 4; ++q) {
                        const P2 cq = qw[1][q];
                        gg2(cq, qk[q], qw[0][q], L1(cq), R1(cq), txk, tyk, ndnx, ndny, nlfx, nlfy, rtx, rty, h,
                            &g[2 * q], &g[2 * q + 1]);
                    }
                    Diff2 d = diffusion2(qw[1][2], UA(3, 4), qw[1][0], qw[1][1], g, K);
                    for (int v = 0; v < 8; ++v) dn[v] = d.d[v];
                    if (S || (r >= i0 && r < i1)) {
                        const P2 s5 = sa_source2(UA(3, 0), UA(3, 4), gk[M2_D2], d.chi, d.fv1, g[2], g[1], g[6], g[7], K);
                        snew = s5 * gk[M2_VOL];
                    }
                    if (!S && r == 0) {
                        // the wall ghost ring (row -1) takes cell 0's gradient with
                        // grad T = 0 (gradient.rs:93-95)
                        P2 gw[8] = {g[0], g[1], g[2], g[3], sp(0.f), sp(0.f), g[6], g[7]};
                        Diff2 w = diffusion2(qw[0][2], UA(2, 4), qw[0][0], qw[0][1], gw, K);
                        for (int v = 0; v < 8; ++v) dw[1][v] = w.d[v];
                    }
                } else if (r >= ni) {  // far ghost ring: zero gradient (gradient.rs:96)
                    P2 gz[8];
                    for (int v = 0; v < 8; ++v) gz[v] = sp(0.f);
                    Diff2 d = diffusion2(qw[1][2], UA(3, 4), qw[1][0], qw[1][1], gz, K);
                    for (int v = 0; v < 8; ++v) dn[v] = d.d[v];
                }
                // r == -1 on a wall strip: written when row 0 is reached
            }

            // ---- V/dt of row k-2 (clamped, dissipation.rs:59) --------------
            P2 rtn = sp(0.f);
            {
                const int rr = k - 2;
                if (S || (rr >= i0 - 1 && rr <= i1)) rtn = P2{B->rat[lane]};
            }

            // ---- tau face f = k-2 (between rows k-3 and k-2) ---------------
            P2 ftn[5];
            for (int v = 0; v < 5; ++v) ftn[v] = sp(0.f);
            const int f = k - 2;
            if (S || (f >= i0 && f <= i1)) {
                const P2 m4 = pmax(pmax(pmax(si[0], si[1]), si[2]), sik);
                const P2 e2 = P2{K.k2} * m4;
                const P2 e4 = pmax(P2{K.k4} - e2, sp(0.f));
                const P2 lam = P2{K.half_cfl} * (rtn + rt0);
                P2 fu[5], cv[5], w0[5], w1[5], w2[5], w3[5];
                for (int v = 0; v < 5; ++v) {
                    w0[v] = UA(0, v);
                    w1[v] = UA(1, v);
                    w2[v] = UA(2, v);
                    w3[v] = UA(3, v);
                    fu[v] = w1[v] + w2[v];
                }
                euler_flux2(fu, tx[1], ty[1], gm1, P2{K.p_ref2}, cv);
                face_combine2(w0, w1, w2, w3, cv, dw[0], dw[1], sp(0.5f) * tx[1], sp(0.5f) * ty[1], lam, e2, e4, ftn);
            }

            // ---- n faces and the update of row m = k-3 ---------------------
            const int m = k - 3;
            if (S || (m >= i0 && m < i1)) {
                P2 fn[5];  // face between each column and the one to its left
                {
                    const P2 m4 = pmax(pmax(pmax(L2(sj[0]), L1(sj[0])), sj[0]), R1(sj[0]));
                    const P2 e2 = P2{K.k2} * m4;
                    const P2 e4 = pmax(P2{K.k4} - e2, sp(0.f));
                    const P2 lam = P2{K.half_cfl} * (rt0 + L1(rt0));
                    P2 um[5], ul1[5], ul2[5], ur1[5], fu[5], cv[5];
                    for (int v = 0; v < 5; ++v) {
                        um[v] = UA(1, v);
                        ul1[v] = L1(um[v]);
                        ul2[v] = L2(um[v]);
                        ur1[v] = R1(um[v]);
                        fu[v] = ul1[v] + um[v];
                    }
                    euler_flux2(fu, nx2[0], ny2[0], gm1, P2{K.p_ref2}, cv);
                    P2 dl[8];
                    for (int v = 0; v < 8; ++v) dl[v] = L1(dw[0][v]);
                    face_combine2(ul2, ul1, um, ur1, cv, dl, dw[0], sp(0.5f) * nx2[0], sp(0.5f) * ny2[0], lam, e2, e4,
                                  fn);
                }
                P2 R[5];
                for (int v = 0; v < 5; ++v) R[v] = (ftn[v] - ft[v]) + (R1(fn[v]) - fn[v]);
                R[4] = R[4] - sw[0];
                const long id0 = (long)m * nj + gj0, id1 = (long)m * nj + gj1;
                if constexpr (DUMP) {
                    for (int v = 0; v < 5; ++v) {
                        if (out0) I.rdump[v * np + id0] = (double)R[v].v.x;
                        if (out1) I.rdump[v * np + id1] = (double)R[v].v.y;
                    }
                } else {
                    // every lane computes the update (the row buffer holds all
                    // 64 columns' inputs), only output columns store
                    const double2 ivm = B->ivm[lane];
                    double a0 = adt, a1 = adt;
                    if (dt_local) {
                        const double2 l = B->ldt[lane];
                        a0 = alpha * l.x;
                        a1 = alpha * l.y;
                    }
                    const P2 sc = p2((float)(a0 * ivm.x), (float)(a1 * ivm.y));
                    const P2 msc = -sc;
                    // each component is formed and stored in turn: the stage
                    // buffer (FP32), or U_n (FP64) and its FP32 copy
                    P2 nv[5];
                    double uo0 = 0.0, uo1 = 0.0, un00 = 0.0, un10 = 0.0;
                    const bool both = pairwise && out0 && out1;
                    for (int v = 0; v < 5; ++v) {
                        if constexpr (ACC32) {
                            const P2 a_ = FIRST ? UA(1, v) : P2{B->uacc[v][lane]};
                            nv[v] = pfma(R[v], msc, a_);
                            if (both) {
                                *reinterpret_cast<float2*>(dst + v * np + id0) = nv[v].v;
                            } else {
                                if (out0) dst[v * np + id0] = nv[v].v.x;
                                if (out1) dst[v * np + id1] = nv[v].v.y;
                            }
                        } else {
                            const double2 uo = B->un[v][lane];
                            const P2 inc = R[v] * sc;  // FP32 increment, FP64 accumulator
                            const double a0_ = uo.x - (double)inc.v.x, a1_ = uo.y - (double)inc.v.y;
                            nv[v] = p2((float)a0_, (float)a1_);
                            if (v == 0) {
                                uo0 = uo.x;
                                uo1 = uo.y;
                                un00 = a0_;
                                un10 = a1_;
                            }
                            if (both) {
                                *reinterpret_cast<double2*>(I.un[0] + v * np + id0) = make_double2(a0_, a1_);
                                *reinterpret_cast<float2*>(I.uc[0] + v * np + id0) = nv[v].v;
                            } else {
                                if (out0) {
                                    I.un[0][v * np + id0] = a0_;
                                    I.uc[0][v * np + id0] = nv[v].v.x;
                                }
                                if (out1) {
                                    I.un[0][v * np + id1] = a1_;
                                    I.uc[0][v * np + id1] = nv[v].v.y;
                                }
                            }
                        }
                    }
                    // unpack checks (solver.rs:160-171) on the stored FP32 values
                    const Prim2 q = unpack2(nv, gm1, rgas);
                    const bool bad0 = out0 && (isnan(nv[0].v.x) || nv[0].v.x <= 1e-15f || isnan(q.p.v.x) ||
                                               q.p.v.x <= 1e-15f);
                    const bool bad1 = out1 && (isnan(nv[0].v.y) || nv[0].v.y <= 1e-15f || isnan(q.p.v.y) ||
                                               q.p.v.y <= 1e-15f);
                    if (bad0) atomicMin(&I.st->bad, (stage_id << 32) | (unsigned long long)id0);
                    if (bad1) atomicMin(&I.st->bad, (stage_id << 32) | (unsigned long long)id1);
                    if constexpr (LAST) {
                        const bool ok0 = out0 && !bad0, ok1 = out1 && !bad1;
                        const double d0 = un00 - uo0, d1 = un10 - uo1;  // solver.rs:195
                        sres += (ok0 ? d0 * d0 : 0.0) + (ok1 ? d1 * d1 : 0.0);
                        // timestep.rs:30-42 in the stage arithmetic
                        const P2 aa = sp(0.5f) * (tx[0] + tx[1]);
                        const P2 bb = sp(0.5f) * (ty[0] + ty[1]);
                        const P2 cc = sp(0.5f) * (nx2[0] + R1(nx2[0]));
                        const P2 dd = sp(0.5f) * (ny2[0] + R1(ny2[0]));
                        const P2 vol = vw[0];
                        const P2 dl = local_dt2(q.vx, q.vy, psqrt(P2{K.rg} * q.t), aa, bb, cc, dd, P2{K.cfl} * vol);
                        const P2 rat = pdiv(vol, dl);
                        if (ok0) {
                            ratio_next[id0] = rat.v.x;
                            if (dt_local) I.ldt[id0] = (double)dl.v.x;
                        }
                        if (ok1) {
                            ratio_next[id1] = rat.v.y;
                            if (dt_local) I.ldt[id1] = (double)dl.v.y;
                        }
                        mloc = ok0 ? fmin(mloc, (double)dl.v.x) : mloc;
                        mloc = ok1 ? fmin(mloc, (double)dl.v.y) : mloc;
                    }
                }
            }

            // ---- slide the windows ------------------------------------------
            for (int v = 0; v < 5; ++v) {
                uring->u[s0][v][lane] = uk[v].v;
                ft[v] = ftn[v];
            }
            nu3 = qw[0][3];
            pw[0] = pw[1];
            pw[1] = pk;
            for (int v = 0; v < 4; ++v) {
                qw[0][v] = qw[1][v];
                qw[1][v] = qk[v];
            }
            si[0] = si[1];
            si[1] = si[2];
            si[2] = sik;
            sj[0] = sj[1];
            sj[1] = sj[2];
            sj[2] = sjk;
            for (int v = 0; v < 8; ++v) {
                dw[0][v] = dw[1][v];
                dw[1][v] = dn[v];
            }
            sw[0] = sw[1];
            sw[1] = snew;
            rt0 = rtn;
            tx[0] = tx[1];
            tx[1] = tx[2];
            tx[2] = txk;
            ty[0] = ty[1];
            ty[1] = ty[2];
            ty[2] = tyk;
            nx2[0] = nx2[1];
            nx2[1] = nxr;
            ny2[0] = ny2[1];
            ny2[1] = nyr;
            if constexpr (LAST) {
                vw[0] = vw[1];
                vw[1] = gk[M2_VOL];
            }
        };
        const int ks0 = i0 + 3, ks1 = i1 - 2;  // steady rows
        int k = i0 - 3;
        // one call site of the non-steady body (warm-up rows, then the tail
        // rows), so that it is compiled inline
        for (int ph = 0; ph < 2; ++ph) {
            for (; k <= (ph == 0 ? ks0 - 1 : i1 + 2) && k <= i1 + 2; ++k) row(std::false_type{}, k);
            if (ph == 0)
                for (; k <= ks1; ++k) row(std::true_type{}, k);
        }

        if (LAST) {
            const double mn = warp_min(mloc);
            const double sr = warp_sum0(sres);
            unsigned last = 0;
            if (lane == 0) {
                I.partial[2 * tr.tile] = mn;
                I.partial[2 * tr.tile + 1] = sr;
                JST_FENCE();
                const unsigned prev = atomicAdd(&I.st->counter, 1u);
                last = prev == (unsigned)(I.ntiles - 1);
            }
            last = jst_shfl_idx(last, 0);
            if (last) {
                JST_FENCE();
                finish_step_warp<T>(I, true);
            }
        }
    }
#endif
}

}  // namespace fused
}  // namespace jst
