// Warp-marching stage kernel: the same RK stage as k_stage (fused_kernels.cuh),
// organised for instruction economy instead of shared-memory tiles.
//
// Work item = a strip of 26 output columns (j0 .. j0+25) and the rows
// i0 .. i1-1 of one instance (the host cuts each instance into bands of
// nearly equal height, chosen so that the strips fill whole waves of warps).  One warp owns a strip: lane L holds column
// j0-3+L (a 3-column halo on each side), so every j-neighbour the stencil
// needs is one or two lanes away and comes from a register shuffle; the warp
// walks down the rows i0-3 .. i1+2 keeping sliding windows of the rows it
// still needs in registers (U: 4 rows, in FP64 a per-warp shared ring;
// primitives: 2, sensors: 3, diffusion tensors: 2, the previous tau-face
// flux).  Every value is loaded from HBM
// once per strip and computed once per cell (plus a 6-row warm-up and the
// 6-lane halo), no block barrier is used, and warps take strips from a
// per-launch work counter so uneven instances balance.
//
// Per row k of the walk (rows lag so that each input is ready):
//   load U(k) -> primitives, j-sensor(k);  i-sensor(k-1);
//   gradients + diffusion tensor + SA source of row k-1;
//   tau face k-2;  n faces of row k-3 and the RK update of row k-3.
// The arithmetic of every term is the one k_stage uses (shared helpers in
// jst_common.cuh), in the same operation order, except two quotients: the
// temperature comes from the cell's reciprocal density and 1/R
// (unpack_cell_r), the SA source takes nu-tilde from the primitive window.
// A single solve launches the walk as k_march_solo (the instance descriptor a
// kernel parameter), a batch as k_march.
#pragma once

#ifndef JST_LANE
#define JST_LANE() ((int)(threadIdx.x & 31))
#define JST_WARP_IN_BLOCK() ((int)(threadIdx.x >> 5))
template <class V> __device__ __forceinline__ V jst_shfl_up(V v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <class V> __device__ __forceinline__ V jst_shfl_down(V v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
template <class V> __device__ __forceinline__ V jst_shfl_xor(V v, int d) { return __shfl_xor_sync(0xffffffffu, v, d); }
template <class V> __device__ __forceinline__ V jst_shfl_idx(V v, int l) { return __shfl_sync(0xffffffffu, v, l); }
#endif

namespace jst {
namespace fused {

constexpr int MARCH_W = 26;  // output columns per strip (32 lanes - 2 x 3 halo)

// Paired FP32 arithmetic (sm_100 f32x2 instructions: one instruction for two
// lanes of data) for the five-component face arithmetic, where components
// (1, 2) and (3, 4) go in pairs and component 0 alone.  A pair lives in one
// 64-bit register (hand-written PTX); the emulation build does it per lane.
#ifdef __CUDA_ARCH__
using f2 = unsigned long long;
JST_D f2 f2_make(float a, float b) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
JST_D void f2_split(f2 r, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
JST_D f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
JST_D f2 f2_add(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
JST_D f2 f2_mul(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
#else
struct f2 {
    float x, y;
};
JST_D f2 f2_make(float a, float b) { return f2{a, b}; }
JST_D void f2_split(f2 r, float& a, float& b) {
    a = r.x;
    b = r.y;
}
JST_D f2 f2_fma(f2 a, f2 b, f2 c) { return f2{fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y)}; }
JST_D f2 f2_add(f2 a, f2 b) { return f2{a.x + b.x, a.y + b.y}; }
JST_D f2 f2_mul(f2 a, f2 b) { return f2{a.x * b.x, a.y * b.y}; }
#endif
JST_D f2 f2_splat(float a) { return f2_make(a, a); }

// Net face flux out = cv2 / 2 - vis - lam (d1 e2 - d3 e4) of the five
// components, with d1 = w2 - w1 and d3 = w3 - 3 w2 + 3 w1 - w0 (w0..w3 the
// states at face-2 .. face+1) and vis = (dA + dB) hx + (dA' + dB') hy from the
// two cells' diffusion tensors (components 1-4; component 0 has none).  cv2
// is the convective flux of twice the face state w1 + w2: the Euler flux is
// homogeneous of degree one in U and scaling by 2 is exact, so cv2 / 2 is bit
// for bit the flux of (w1 + w2) / 2 (convection.rs:55, 64), one multiply per
// component fewer.
template <class T>
JST_D void face_combine(const T* w0, const T* w1, const T* w2, const T* w3, const T* cv, const T* dA, const T* dB,
                        T hx, T hy, T lam, T e2, T e4, T* out) {
    if constexpr (sizeof(T) == sizeof(float)) {
        {  // component 0
            T d1 = w2[0] - w1[0];
            T d3 = w3[0] - T(3) * w2[0] + T(3) * w1[0] - w0[0];
            out[0] = T(0.5) * cv[0] - lam * (d1 * e2 - d3 * e4);
        }
        const f2 m1 = f2_splat(-1.0f), m3 = f2_splat(-3.0f), p3 = f2_splat(3.0f), half = f2_splat(0.5f);
        const f2 mhx2 = f2_splat(-hx), mhy2 = f2_splat(-hy), e22 = f2_splat(e2), me42 = f2_splat(-e4);
        const f2 mlam = f2_splat(-lam);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int a = 1 + 2 * q, b = a + 1;  // components a, b; tensor rows a-1, b-1 (x) and a+3, b+3 (y)
            f2 W0 = f2_make(w0[a], w0[b]), W1 = f2_make(w1[a], w1[b]), W2 = f2_make(w2[a], w2[b]);
            f2 W3 = f2_make(w3[a], w3[b]);
            f2 D1 = f2_fma(W1, m1, W2);
            f2 D3 = f2_fma(W0, m1, f2_fma(W1, p3, f2_fma(W2, m3, W3)));
            f2 DX = f2_add(f2_make(dA[a - 1], dA[b - 1]), f2_make(dB[a - 1], dB[b - 1]));
            f2 DY = f2_add(f2_make(dA[a + 3], dA[b + 3]), f2_make(dB[a + 3], dB[b + 3]));
            f2 NVIS = f2_fma(DX, mhx2, f2_mul(DY, mhy2));
            f2 DIS = f2_fma(D3, me42, f2_mul(D1, e22));
            f2 O = f2_fma(DIS, mlam, f2_fma(f2_make(cv[a], cv[b]), half, NVIS));
            f2_split(O, out[a], out[b]);
        }
    } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            T d1 = w2[v] - w1[v];
            T d3 = w3[v] - T(3) * w2[v] + T(3) * w1[v] - w0[v];
            T vis = T(0);
            if (v > 0) vis = (dA[v - 1] + dB[v - 1]) * hx + (dA[v + 3] + dB[v + 3]) * hy;
            out[v] = (T(0.5) * cv[v] - vis) - lam * (d1 * e2 - d3 * e4);
        }
    }
}

template <class V> JST_D V warp_sum0(V v) {  // lane 0 gets a fixed-order sum
    for (int o = 16; o > 0; o >>= 1) v += jst_shfl_xor(v, o);
    return v;
}
template <class V> JST_D V warp_min(V v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, jst_shfl_xor(v, o));
    return v;
}

// Last-warp-done reduction of the per-strip partials (the warp version of
// finish_step): dt and, when `with_residual`, the residual of the step.
template <class T> JST_D void finish_step_warp(const Inst<T>& I, bool with_residual) {
    const int lane = JST_LANE();
    double m = __longlong_as_double(0x7ff0000000000000LL);
    double s = 0.0;
    for (int k = lane; k < I.ntiles; k += 32) {
        volatile const double* pp = I.partial + 2 * k;
        m = fmin(m, pp[0]);
        s += pp[1];
    }
    double mn = warp_min(m);
    double sm = warp_sum0(s);
    if (lane == 0) {
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

// Geometry record of row k (Inst::mg), 8 values of the stage type.
enum { MG_TX = 0, MG_TY, MG_NX, MG_NY, MG_IV, MG_D2, MG_VOL, MG_N = 8 };

// Builds Inst::mg from the FP64 geometry: the values each row of the walk
// reads, rounded once to the stage type (the same values the stage
// arithmetic used to convert at every use), in one 16-byte-aligned record.
#ifdef __CUDACC__
template <class T>
__global__ void k_march_geom(const double* tnx, const double* tny, const double* nnx, const double* nny,
                             const double* inv_vol, const double* inv_d2, const double* vol, int ni, int nj, T* rec) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)(ni + 1) * nj) return;
    T* r = rec + MG_N * q;
    r[MG_TX] = (T)tnx[q];
    r[MG_TY] = (T)tny[q];
    if (q >= nj) {
        long c = q - nj;
        r[MG_NX] = (T)nnx[c];
        r[MG_NY] = (T)nny[c];
        r[MG_IV] = (T)inv_vol[c];
        r[MG_D2] = (T)inv_d2[c];
        r[MG_VOL] = (T)vol[c];
    } else {
        r[MG_NX] = r[MG_NY] = r[MG_IV] = r[MG_D2] = r[MG_VOL] = T(0);
    }
    r[7] = T(0);
}
#endif

// One row's worth of global inputs of a warp, staged asynchronously one row
// ahead (PIPE variant): [field][lane]; the geometry record in 16-byte chunks
// [chunk][lane] so that each chunk read is one conflict-free 128-bit load.
template <class T> struct MarchRow {
    static constexpr int RCH = MG_N * (int)sizeof(T) / 16, EPC = 16 / (int)sizeof(T);
    alignas(16) T rec[RCH][32][EPC];  // Inst::mg record of row k
    double un[5][32], ldt[32], ivm[32];  // U_n, dt_local, 1/V of row k-3
    T uacc[5][32];                    // FP32 copy of U_n of row k-3 (split, stages 1-3)
    T u[5][32];                       // stage input of row k
    T rat[32];                        // V/dt of row k-2 (clamped)
    T volm[32];                       // V of row k-3 (last stage)
};

// Bulk row staging (STG = 1): the same inputs as MarchRow, but each field's
// segment of the strip's row is moved by one cp.async.bulk copy (the TMA
// unit) issued by lane 0, so the buffer mirrors global memory.  A copy must
// start on a 16-byte boundary and move a multiple of 16 bytes, so a plane of
// T is staged from the column (j0 - 3) rounded down to a multiple of AT
// (16 bytes of T) and AT columns wider than the strip; lane L reads column
// oT + L.  FP64 planes likewise with 2 columns per 16 bytes; the geometry
// records (32 or 64 bytes each) start exactly at j0 - 3.  A segment that
// crosses the periodic seam is copied in two pieces.  The copies of a row
// complete one phase of the row buffer's mbarrier.
template <class T> struct MarchRowB {
    static constexpr int AT = 16 / (int)sizeof(T);  // columns of T per 16 bytes
    static constexpr int WT = 32 + AT;              // columns staged per plane of T
    static constexpr int WD = 34;                   // columns staged per FP64 plane
    alignas(16) T rec[32][MG_N];                    // Inst::mg records of row k, one per lane
    alignas(16) T u[5][WT];                         // stage input of row k
    alignas(16) T uacc[5][WT];                      // FP32 copy of U_n of row k-3 (split, stages 1-3)
    alignas(16) double un[5][WD];                   // U_n of row k-3
    alignas(16) double ldt[WD];                     // dt_local of row k-3
    alignas(16) double ivm[WD];                     // 1/V of row k-3
    alignas(16) T rat[WT];                          // V/dt of row k-2 (clamped)
    alignas(16) T volm[32];                         // V of row k-3 (last stage; per-lane copies)
    alignas(16) unsigned long long bar;             // the row's mbarrier
};

#ifdef __CUDA_ARCH__
JST_D unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
JST_D void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
JST_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
JST_D void proxy_async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// arrive on the barrier and add `bytes` to the transaction count of its phase
JST_D void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// one bulk global -> shared copy (16-byte aligned addresses, size a multiple of 16)
JST_D void bulk_copy(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
JST_D bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of the given parity, at most about `cycles` SM clock
// cycles; false when the limit ran out.
JST_D bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long cycles) {
    const long long t0 = clock64();
    while (!mbar_test(bar, parity))
        if (clock64() - t0 > cycles) return false;
    return true;
}
#endif

// Limit of a row-buffer wait: about 0.1 s at the B200's SM clock, far beyond
// any copy's latency.
constexpr long long kStageWaitCycles = 200000000LL;

// FP64 keeps the 4-row U window in a per-warp shared ring of 5 rows (the
// registers it would take push the FP64 kernel past 255 registers).
template <class T> JST_HD constexpr bool march_u_ring() { return sizeof(T) == sizeof(double); }
template <class T> struct MarchURing {
    T u[5][5][32];  // [row slot][variable][lane]
};

// Per warp: the row buffers, the U ring (FP64) and a copy of the strip's
// instance constants (PhysConst, and for the FP32 arithmetic ConstP), read
// by every row of the walk; in shared memory a constant costs a
// short-latency load instead of a global one (and in FP32 no conversion).
JST_HD constexpr size_t march_phys_bytes() { return (sizeof(PhysConst) + 15) / 16 * 16; }
JST_HD constexpr size_t march_const_bytes() { return march_phys_bytes() + (sizeof(ConstP) + 15) / 16 * 16; }
template <class T, int NT, bool PIPE, int STG = 0> JST_HD constexpr size_t march_buf_bytes() {
    return (size_t)(NT / 32) * ((PIPE ? 2 * (STG ? sizeof(MarchRowB<T>) : sizeof(MarchRow<T>)) : 0) +
                                (march_u_ring<T>() ? sizeof(MarchURing<T>) : 0));
}
template <class T, int NT, bool PIPE, int STG = 0> JST_HD constexpr size_t march_smem_bytes() {
    return march_buf_bytes<T, NT, PIPE, STG>() + (size_t)(NT / 32) * march_const_bytes();
}

// Copies an instance's constants into this warp's slot (8-byte words, one
// per lane), between warp barriers so that the previous strip's reads are
// done.
template <class C> JST_D void warp_copy_const(C* dst, const C* src) {
#ifdef __CUDA_ARCH__
    __syncwarp();
    const unsigned long long* s8 = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d8 = reinterpret_cast<unsigned long long*>(dst);
    for (int w = JST_LANE(); w < (int)(sizeof(C) / 8); w += 32) d8[w] = s8[w];
    __syncwarp();
#endif
}

// Solver::unpack (solver.rs:158-181) for one cell of the marching kernels:
// the temperature p / (R rho) is formed as p (1/rho) (1/R) from the
// reciprocal the velocities already use and the strip's 1/R (two multiplies
// instead of a quotient; within a few units in the last place of it).
template <class T> JST_D Prim<T> unpack_cell_r(T u0, T u1, T u2, T u3, T u4, T gm1, T inv_rgas) {
    Prim<T> q;
    T inv = dv<T, true>(T(1), u0);
    q.rho = u0;
    q.vx = u1 * inv;
    q.vy = u2 * inv;
    q.e = u3 * inv;
    q.p = gm1 * (u3 - u0 * (q.vx * q.vx + q.vy * q.vy) * T(0.5));
    q.t = q.p * inv * inv_rgas;
    q.nut = u4 * inv;
    return q;
}

// A constant in the stage arithmetic: the FP32 copy for T = float, the FP64
// value otherwise.
template <class T> JST_D T kc(double d, float2 f) {
    if constexpr (sizeof(T) == sizeof(float)) return f.x;
    else return d;
}

// source::compute for one cell in FP32 (sa_source_nt) from the FP32 constants.
JST_D float sa_source_f32(float rho, float rho_nu, float nu_tilde, float inv_dist2, float chi, float f1, float dvdx,
                          float dudy, float dnx, float dny, const ConstP& K) {
    const float inv_kd2 = inv_dist2 * K.inv_kappa2.x;
    const float ft2 = K.ct3.x * exp_f32(K.m_ct4.x * chi * chi);
    const float fv2 = 1.0f - dv<float, true>(chi, 1.0f + chi * f1);
    const float sv = K.fv3.x * fabsf(dvdx - dudy);
    const float s_tilde = fmaxf(sv + nu_tilde * inv_kd2 * fv2, 1e-10f);
    const float prod = K.cb1.x * (1.0f - ft2) * s_tilde * rho_nu;
    const float r = fminf(dv<float, true>(nu_tilde, s_tilde) * inv_kd2, K.rmax.x);
    const float fw = fw_f32(r, K.cw2.x, K.cw3_6.x, K.one_plus_cw3_6.x, K.fw_lim.x);
    const float destr = (K.cw1.x * fw + K.m_cb1_k2.x * ft2) * rho * (nu_tilde * nu_tilde * inv_dist2);
    const float diff = K.cb2_sigma.x * rho * (dnx * dnx + dny * dny);
    return prod - destr + diff;
}

// Minimum resident blocks per SM asked of the register allocator: 12 warps
// per SM in FP32 (at most 168 registers a thread; the last stage would take
// ~190 and drop to 8 warps), no cap in FP64.  Measured on B200: the cap
// takes the FP32 last stage from 0.48 to 0.35 ms on 4.2 M cells, and a
// 16-warp cap (128 registers) spills and is slower.
template <class T, int NT> constexpr int march_min_blocks() {
    return sizeof(T) == sizeof(float) ? (12 / (NT / 32) > 0 ? 12 / (NT / 32) : 1) : 1;
}

// sched[0] = number of strips, sched[1] = work counter, sched[2] = exit counter
// (both zero at launch; the last warp to leave resets them).
// PIPE: every global input of row k+1 is copied into a per-warp shared
// buffer while row k is computed, so the walk never waits on HBM latency;
// without PIPE the loads are issued in the row that uses them.  STG selects
// how the copies are made: 0, one cp.async per lane and field; 1, one
// cp.async.bulk (TMA) copy per field's row segment issued by lane 0 and
// completed on the row buffer's mbarrier (MarchRowB), where the ring allows
// it (NJ a multiple of 16 bytes of T and at least 36 columns), else per-lane
// copies into the same layout.  A bounded wait that runs out sets
// InstState::err, and the warp does no further work in the launch.
// DUMP (with FIRST only): the residual R of every cell of the current state
// goes to Inst::rdump instead of an update; nothing else is written and the
// instance's step counters and stop flags are ignored.
// SOLO: every strip belongs to the one instance `solo` points to, a kernel
// parameter (k_march_solo); its descriptor and constants are then read from
// the parameter bank, as instruction operands, instead of being copied to
// the warp's shared slot per strip and reloaded from global memory.
template <class T, int NT, bool FIRST, bool LAST, bool PIPE, bool DUMP, int STG, bool SOLO>
JST_D void march_body(const TileRef* tiles, int* sched, const Inst<T>* insts, int stage, double alpha,
                      const Inst<T>* solo) {
    using TD = typename std::conditional<LAST, double, T>::type;
    const int lane = JST_LANE();
    constexpr bool UR = march_u_ring<T>();
    // Split precision, stages 0-3: their output is stored in FP32, so the RK
    // accumulator starts from the FP32 copy of U_n (what they store differs
    // from rounding U_n - increment once by at most one FP32 rounding); the
    // last stage adds its increment to U_n in FP64.
    constexpr bool ACC32 = sizeof(T) == sizeof(float) && !LAST;
    // FP64, stage 0: the stage input is U_n itself, so the accumulator of the
    // updated row is the U ring's copy of it (the value loaded three rows
    // earlier) instead of a second load
    constexpr bool UN_RING = FIRST && sizeof(T) == sizeof(double) && march_u_ring<T>();
    using RowT = typename std::conditional<STG == 1, MarchRowB<T>, MarchRow<T>>::type;
    RowT* rowbuf = nullptr;
    MarchURing<T>* uring = nullptr;
    JST_DYN_SMEM(smem_raw);
    const int wib = JST_WARP_IN_BLOCK();
    if constexpr (PIPE) rowbuf = reinterpret_cast<RowT*>(smem_raw) + 2 * wib;
    if constexpr (UR)
        uring = reinterpret_cast<MarchURing<T>*>(smem_raw + (PIPE ? (size_t)(NT / 32) * 2 * sizeof(RowT) : 0)) + wib;
    PhysConst* cwarp = reinterpret_cast<PhysConst*>(smem_raw + march_buf_bytes<T, NT, PIPE, STG>() +
                                                    (size_t)wib * march_const_bytes());
    ConstP* kwarp = reinterpret_cast<ConstP*>(reinterpret_cast<unsigned char*>(cwarp) + march_phys_bytes());
    const int nt_all = sched[0];
    unsigned* work = reinterpret_cast<unsigned*>(sched + 1);
    unsigned* exitc = reinterpret_cast<unsigned*>(sched + 2);
    const unsigned nwarps = (unsigned)JST_GRID() * (NT / 32);
    unsigned bphase = 0;  // STG 1: parity of the next phase of each row buffer's barrier (bit b)
    bool dead = false;    // STG 1: a bounded wait ran out; take no more work
#ifdef __CUDA_ARCH__
    if constexpr (STG == 1) {
        if (lane == 0) {
            mbar_init(&rowbuf[0].bar);
            mbar_init(&rowbuf[1].bar);
            mbar_init_fence();
        }
        __syncwarp();
    }
#endif
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
        if (dead) continue;
        const TileRef tr = tiles[ticket];
        const Inst<T>* ip = insts + tr.inst;
        if constexpr (SOLO) ip = solo;
        const Inst<T>& I = *ip;
        const int ni = I.ni, nj = I.nj, i0 = tr.i0, j0 = tr.j0;
        const PhysConst* cp = cwarp;
        const ConstP* kp = kwarp;
        if constexpr (SOLO) {
            cp = &I.c;
            kp = &I.cp;
        } else {
            warp_copy_const(cwarp, &I.c);
            if constexpr (sizeof(T) == sizeof(float)) warp_copy_const(kwarp, &I.cp);
        }
        const PhysConst& c = *cp;
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
        // per-instance values the row walk uses, read once per strip (the step's
        // global time step changes only when the last strip of the last stage
        // has finished)
        const bool dt_local = I.local_dt != 0;
        const double adt = dt_local ? alpha : alpha * I.st->dt;
        const unsigned long long stage_id = (unsigned long long)step * 5 + stage;
        const T* ratio = I.ratio[step & 1];
        T* ratio_next = I.ratio[(step + 1) & 1];
        (void)ratio_next;
        // The five planes of every state array are contiguous (plane k at
        // plane 0 + k * NI * NJ, as both engines allocate them), so one base
        // pointer per array and the plane stride address them all.
        const long np = (long)ni * nj;
        const T* src = FIRST ? (sizeof(T) == sizeof(double) ? reinterpret_cast<const T*>(I.un[0]) : I.uc[0])
                             : ((stage % 2 == 1) ? I.ua[0] : I.ub[0]);
        TD* dst = LAST ? reinterpret_cast<TD*>(I.un[0]) : reinterpret_cast<TD*>((stage % 2 == 0) ? I.ua[0] : I.ub[0]);

        const int i1 = tr.i1;                       // output rows i0 .. i1-1
        const int cu = j0 - 3 + lane;               // unwrapped column of this lane
        const int gj = wrapj(cu, nj);
        const bool seam = cu < 0 || cu >= nj;
        const bool out_lane = lane >= 3 && lane < 3 + MARCH_W && cu < nj;
        const T gm1 = kc<T>(c.gm1, K.gm1), rgas = kc<T>(c.r_gas, K.r_gas);
        const T inv_rgas = T(1) / rgas;  // once per strip
        const T half_cfl = kc<T>(c.half_cfl, K.half_cfl), k2 = kc<T>(c.k2, K.k2), k4 = kc<T>(c.k4, K.k4);
        // face fluxes are formed from twice the face state (see face_combine),
        // so the pressure reference of euler_flux is doubled as well
        const T p_ref2 = sizeof(T) == sizeof(double) ? T(0) : kc<T>(0.0, K.p_ref2);

        // STG 1: bulk copies where the ring allows them (16-byte aligned
        // segments; a segment crosses the seam at most once); the columns
        // oT, oD of the staged segments hold the strip's first column
        constexpr int AT = MarchRowB<T>::AT, WT = MarchRowB<T>::WT, WD = MarchRowB<T>::WD;
        const bool bulk = STG == 1 && nj % AT == 0 && nj >= WT;
        const int sT = (j0 - 3) & ~(AT - 1), sD = (j0 - 3) & ~1;
        const int oT = bulk ? j0 - 3 - sT : 0, oD = bulk ? j0 - 3 - sD : 0;
        const unsigned extra_tx = STG == 1 ? (unsigned)I.stage_extra_tx : 0u;
        bool failed = false;
        (void)sD;
        (void)extra_tx;

        // PIPE: stage the global inputs that row kk of the walk reads.  The
        // conditions are the ones under which the walk reads them.
        auto issue_bulk = [&](auto steady, int kk) {
            constexpr bool S = decltype(steady)::value;
            RowT& B = rowbuf[kk & 1];
#ifdef __CUDA_ARCH__
            if constexpr (STG == 1) {
                __syncwarp();  // every lane has read this buffer's previous row
                if (lane == 0) {
                    unsigned tx = 0;
                    // columns c0 .. c0+w-1 of a row (elements of esz bytes), wrapped
                    auto seg = [&](void* d, const void* rowp, int esz, int c0, int w) {
                        const int a = c0 < 0 ? c0 + nj : c0;
                        const int n1 = w < nj - a ? w : nj - a;
                        bulk_copy(d, static_cast<const char*>(rowp) + (long)a * esz, (unsigned)(n1 * esz), &B.bar);
                        if (n1 < w)
                            bulk_copy(static_cast<char*>(d) + (long)n1 * esz, rowp, (unsigned)((w - n1) * esz), &B.bar);
                        tx += (unsigned)(w * esz);
                    };
                    if (S || kk < ni) {
                        const long row = kk < 0 ? -1 - kk : kk;
                        for (int v = 0; v < 5; ++v) seg(B.u[v], src + v * np + row * nj, (int)sizeof(T), sT, WT);
                    }
                    if (S || (kk >= 0 && kk <= ni))
                        seg(B.rec, I.mg + MG_N * ((long)kk * nj), MG_N * (int)sizeof(T), j0 - 3, 32);
                    const int rr = kk - 2;
                    if (S || (rr >= i0 - 1 && rr <= i1)) {
                        const int gc = S ? rr : (rr < 0 ? 0 : (rr > ni - 1 ? ni - 1 : rr));
                        seg(B.rat, ratio + (long)gc * nj, (int)sizeof(T), sT, WT);
                    }
                    const int m = kk - 3;
                    if (S || (m >= i0 && m < i1)) {
                        const long mr = (long)m * nj;
                        if constexpr (ACC32) {
                            if constexpr (!FIRST)
                                for (int v = 0; v < 5; ++v) seg(B.uacc[v], I.uc[0] + v * np + mr, (int)sizeof(T), sT, WT);
                        } else if constexpr (!UN_RING) {
                            for (int v = 0; v < 5; ++v) seg(B.un[v], I.un[0] + v * np + mr, 8, sD, WD);
                        }
                        if (dt_local) seg(B.ldt, I.ldt + mr, 8, sD, WD);
                        seg(B.ivm, I.inv_vol + mr, 8, sD, WD);
                    }
                    mbar_arrive_tx(&B.bar, tx + extra_tx);
                }
                const int m = kk - 3;
                if (LAST && (S || (m >= i0 && m < i1)))
                    async_copy<sizeof(T)>(&B.volm[lane], I.mg + MG_N * ((long)(m + 1) * nj + gj) + MG_VOL);
            }
#endif
            (void)B;
            (void)kk;
        };
        auto issue = [&](auto steady, int kk) {
            constexpr bool S = decltype(steady)::value;  // kk is a steady row
            if (STG == 1 && bulk) {
                issue_bulk(steady, kk);
                return;
            }
            RowT& B = rowbuf[kk & 1];
            auto rec_dst = [&](int ch) -> T* {
                if constexpr (STG == 1) return &B.rec[lane][ch * MarchRow<T>::EPC];
                else return &B.rec[ch][lane][0];
            };
            if (S || kk < ni) {
                const long id = (long)(kk < 0 ? -1 - kk : kk) * nj + gj;
                for (int v = 0; v < 5; ++v) async_copy<sizeof(T)>(&B.u[v][lane], src + v * np + id);
            }
            if (S || (kk >= 0 && kk <= ni)) {
                const T* g = I.mg + MG_N * ((long)kk * nj + gj);
                for (int ch = 0; ch < MarchRow<T>::RCH; ++ch) async_copy<16>(rec_dst(ch), g + ch * MarchRow<T>::EPC);
            }
            const int rr = kk - 2;
            if (S || (rr >= i0 - 1 && rr <= i1)) {
                const int gc = S ? rr : (rr < 0 ? 0 : (rr > ni - 1 ? ni - 1 : rr));
                async_copy<sizeof(T)>(&B.rat[lane], ratio + (long)gc * nj + gj);
            }
            const int m = kk - 3;
            if (S || (m >= i0 && m < i1)) {
                const long id = (long)m * nj + gj;
                if constexpr (ACC32) {
                    if constexpr (!FIRST)  // stage 0 reads the same values as its stage input
                        for (int v = 0; v < 5; ++v) async_copy<sizeof(T)>(&B.uacc[v][lane], I.uc[0] + v * np + id);
                } else if constexpr (!UN_RING) {
                    for (int v = 0; v < 5; ++v) async_copy<8>(&B.un[v][lane], I.un[0] + v * np + id);
                }
                if (dt_local) async_copy<8>(&B.ldt[lane], I.ldt + id);
                async_copy<8>(&B.ivm[lane], I.inv_vol + id);
                if (LAST) async_copy<sizeof(T)>(&B.volm[lane], I.mg + MG_N * (id + nj) + MG_VOL);
            }
        };
        if constexpr (PIPE) {
            issue(std::false_type{}, i0 - 3);
            async_commit();
        }

        // sliding windows (index 0 = oldest row)
        T u[4][5];      // U rows k-4 .. k-1
        T pw[2];        // p rows k-2, k-1
        T qw[2][4];     // (vx, vy, T, nut) rows k-2, k-1
        T nu3 = T(0);   // nut row k-3 (far-field extrapolation)
        T si[3];        // i-sensor rows k-4 .. k-2
        T sj[3];        // j-sensor rows k-3 .. k-1
        T dw[2][8];     // diffusion tensor rows k-3, k-2
        T sw[2];        // SA source * V rows k-3, k-2
        T rt0 = T(0);   // V/dt row k-3 (rows clamped to the mesh)
        T ft[5];        // tau-face flux of face k-3
        T tx[3], ty[3]; // tau normals rows k-3 .. k-1
        T nx2[2], ny2[2];  // n normals (left face of this column) rows k-3, k-2
        for (int a = 0; a < 4; ++a)
            for (int v = 0; v < 5; ++v) u[a][v] = T(0);
        for (int a = 0; a < 2; ++a) {
            pw[a] = T(0);
            sw[a] = T(0);
            nx2[a] = ny2[a] = T(0);
            for (int v = 0; v < 4; ++v) qw[a][v] = T(0);
            for (int v = 0; v < 8; ++v) dw[a][v] = T(0);
        }
        for (int a = 0; a < 3; ++a) {
            si[a] = sj[a] = T(0);
            tx[a] = ty[a] = T(0);
        }
        for (int v = 0; v < 5; ++v) ft[v] = T(0);
        double mloc = __longlong_as_double(0x7ff0000000000000LL);
        double sres = 0.0;

        // One row of the walk.  S (steady): k in [i0+3, i1-2], where every
        // phase is active, no ghost row is involved and the next row is steady
        // too, so the range tests drop out and the body is one straight block.
        auto row = [&](auto steady, int k) {
            constexpr bool S = decltype(steady)::value;
            const RowT* B = nullptr;
            // U of row k-4+a (a = 0..3): the register window, or the ring slot
            const int s0 = UR ? ((k % 5) + 5) % 5 : 0;  // ring slot of row k
            auto UA = [&](int a, int v) -> T {
                if constexpr (UR) {
                    int sl = s0 + 1 + a;
                    return uring->u[sl >= 5 ? sl - 5 : sl][v][lane];
                } else {
                    return u[a][v];
                }
            };
            if constexpr (PIPE) {
                if (S) issue(steady, k + 1);
                else if (k + 1 <= i1 + 2) issue(std::false_type{}, k + 1);
                async_commit();
                async_wait_prior1();
                B = &rowbuf[k & 1];
#ifdef __CUDA_ARCH__
                if constexpr (STG == 1) if (bulk) {
                    const unsigned b = (unsigned)(k & 1);
                    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&rowbuf[b].bar, (bphase >> b) & 1u,
                                                                              kStageWaitCycles));
                    bphase ^= 1u << b;
                    if (!ok) {  // record it, let the copies in flight land, stop
                        if (lane == 0) atomicOr(&I.st->err, 1);
                        __all_sync(0xffffffffu, mbar_wait_bounded(&rowbuf[b ^ 1u].bar, (bphase >> (b ^ 1u)) & 1u,
                                                                  kStageWaitCycles));
                        failed = true;
                        return;
                    }
                }
#endif
            }
            // ---- row k: conserved state and primitives ---------------------
            T uk[5], pk, qk[4];
            if (S || k < ni) {
                const bool wall = !S && k < 0;
                const int kr = wall ? -1 - k : k;  // the wall ghost mirrors cell -1-k (boundary.rs:30-51)
                const long id = (long)kr * nj + gj;
                for (int v = 0; v < 5; ++v) uk[v] = PIPE ? B->u[v][oT + lane] : ld(src + v * np + id);
                Prim<T> p;
                if (fresh) {
                    p.rho = kc<T>(c.f_rho, K.f_rho);
                    p.p = kc<T>(c.f_p, K.f_p);
                    p.t = kc<T>(c.f_t, K.f_t);
                    p.vx = kc<T>(c.f_vx, K.f_vx);
                    p.vy = kc<T>(c.f_vy, K.f_vy);
                    p.e = kc<T>(c.f_e, K.f_e);
                    p.nut = kc<T>(c.f_nut, K.f_nut);
                } else {
                    p = unpack_cell_r<T>(uk[0], uk[1], uk[2], uk[3], uk[4], gm1, inv_rgas);
                }
                if (seam) pack_cell<T>(p, uk);  // periodic ghost column (boundary.rs:54-72)
                if (wall) {
                    Prim<T> q;
                    q.rho = uk[0];
                    q.p = p.p;
                    q.t = p.t;
                    q.vx = -p.vx;
                    q.vy = -p.vy;
                    q.nut = -p.nut;
                    q.e = fresh ? kc<T>(c.f_e, K.f_e) : uk[3] * dv<T, true>(T(1), q.rho);
                    pack_cell<T>(q, uk);
                    p = q;
                }
                pk = p.p;
                qk[0] = p.vx;
                qk[1] = p.vy;
                qk[2] = p.t;
                qk[3] = p.nut;
            } else if (k == ni) {  // far-field ghost rows (boundary.rs:87-155), all three alike
                const double* fg = I.far + 5 * (long)gj;
                double nu[3] = {(double)qw[1][3], (double)qw[0][3], (double)nu3};
                double dist[3] = {ld(fg + 2), ld(fg + 3), ld(fg + 4)};
                double t = (double)qw[1][2];
                double cs = fresh ? c.f_c : sqrt(c.rg * t);
                FarState f = riemann_face(ld(fg + 0), ld(fg + 1), (double)qw[1][0], (double)qw[1][1], cs, dist, nu, c);
                Prim<T> q;
                q.rho = (T)f.rho;
                q.p = (T)f.p;
                q.t = (T)f.t;
                q.vx = (T)f.vx;
                q.vy = (T)f.vy;
                q.e = (T)f.e;
                q.nut = (T)f.nut;
                pack_cell<T>(q, uk);
                pk = q.p;
                qk[0] = q.vx;
                qk[1] = q.vy;
                qk[2] = q.t;
                qk[3] = q.nut;
            } else {  // rows ni+1, ni+2 repeat row ni
                for (int v = 0; v < 5; ++v) uk[v] = UA(3, v);
                pk = pw[1];
                for (int v = 0; v < 4; ++v) qk[v] = qw[1][v];
            }
            // j-sensor of row k (dissipation.rs:73-90)
            const T sjk = pressure_sensor<T, true>(jst_shfl_up(pk, 1), pk, jst_shfl_down(pk, 1));
            // i-sensor of row k-1
            const T sik = pressure_sensor<T, true>(pw[0], pw[1], pk);

            // ---- geometry record of row k (tau normals of face row k; n
            // normals, 1/V, 1/d^2, V of cell row k-1) -------------------------
            T gk[MG_N];
            for (int e = 0; e < MG_N; ++e) gk[e] = T(0);
            if (S || (k >= 0 && k <= ni)) {
                if constexpr (PIPE) {
                    for (int ch = 0; ch < MarchRow<T>::RCH; ++ch)
                        for (int e = 0; e < MarchRow<T>::EPC; ++e) {
                            if constexpr (STG == 1) gk[ch * MarchRow<T>::EPC + e] = B->rec[lane][ch * MarchRow<T>::EPC + e];
                            else gk[ch * MarchRow<T>::EPC + e] = B->rec[ch][lane][e];
                        }
                } else {
                    const T* g = I.mg + MG_N * ((long)k * nj + gj);
                    for (int e = 0; e < MG_N; ++e) gk[e] = ld(g + e);
                }
            }
            const T txk = gk[MG_TX], tyk = gk[MG_TY];

            // ---- gradients, diffusion tensor, SA source of row r = k-1 -----
            const int r = k - 1;
            T dn[8];
            for (int v = 0; v < 8; ++v) dn[v] = T(0);
            T snew = T(0), nxr = T(0), nyr = T(0);
            if (S || (r >= i0 - 1 && r <= i1)) {
                if (S || (r >= 0 && r < ni)) {
                    nxr = gk[MG_NX];
                    nyr = gk[MG_NY];
                    const T rtx = jst_shfl_down(nxr, 1), rty = jst_shfl_down(nyr, 1);
                    const T iv = gk[MG_IV];
                    T g[8];
                    for (int q = 0; q < 4; ++q) {
                        const T cq = qw[1][q];
                        const T lf = jst_shfl_up(cq, 1), rg = jst_shfl_down(cq, 1);
                        if (sizeof(T) == sizeof(double))
                            green_gauss<T>(cq, qk[q], qw[0][q], lf, rg, txk, tyk, tx[2], ty[2], nxr, nyr, rtx, rty, iv,
                                           &g[2 * q], &g[2 * q + 1]);
                        else
                            green_gauss_delta<T>(cq, qk[q], qw[0][q], lf, rg, txk, tyk, tx[2], ty[2], nxr, nyr, rtx,
                                                 rty, iv, &g[2 * q], &g[2 * q + 1]);
                    }
                    Diff<T> d = diffusion_tensor<T, true>(qw[1][2], UA(3, 4), qw[1][0], qw[1][1], g[0], g[1], g[2],
                                                          g[3], g[4], g[5], g[6], g[7], kc<T>(c.inv_t_ref, K.inv_t_ref), kc<T>(c.suth_num, K.suth_num), kc<T>(c.t_suth, K.t_suth), kc<T>(c.cv1_cubed, K.cv1_cubed), kc<T>(c.inv_pr, K.inv_pr), kc<T>(c.inv_prt, K.inv_prt), kc<T>(c.cp, K.cp), kc<T>(c.sigma, K.sigma));
                    dn[0] = d.dx1;
                    dn[1] = d.dx2;
                    dn[2] = d.dx3;
                    dn[3] = d.dx4;
                    dn[4] = d.dy1;
                    dn[5] = d.dy2;
                    dn[6] = d.dy3;
                    dn[7] = d.dy4;
                    if (S || (r >= i0 && r < i1)) {
                        T s5;
                        if constexpr (sizeof(T) == sizeof(float))
                            s5 = sa_source_f32(UA(3, 0), UA(3, 4), qw[1][3], gk[MG_D2], d.chi, d.fv1, g[2], g[1], g[6],
                                               g[7], K);
                        else
                            s5 = sa_source_nt<T, true>(UA(3, 0), UA(3, 4), qw[1][3], gk[MG_D2], d.chi, d.fv1, g[2],
                                                       g[1], g[6], g[7], c);
                        snew = s5 * gk[MG_VOL];
                    }
                    if (!S && r == 0) {
                        // the wall ghost ring (row -1, one row up in the window) takes cell
                        // 0's gradient with grad T = 0 (gradient.rs:93-95)
                        Diff<T> w = diffusion_tensor<T, true>(qw[0][2], UA(2, 4), qw[0][0], qw[0][1], g[0], g[1],
                                                              g[2], g[3], T(0), T(0), g[6], g[7], kc<T>(c.inv_t_ref, K.inv_t_ref), kc<T>(c.suth_num, K.suth_num), kc<T>(c.t_suth, K.t_suth), kc<T>(c.cv1_cubed, K.cv1_cubed), kc<T>(c.inv_pr, K.inv_pr), kc<T>(c.inv_prt, K.inv_prt), kc<T>(c.cp, K.cp), kc<T>(c.sigma, K.sigma));
                        dw[1][0] = w.dx1;
                        dw[1][1] = w.dx2;
                        dw[1][2] = w.dx3;
                        dw[1][3] = w.dx4;
                        dw[1][4] = w.dy1;
                        dw[1][5] = w.dy2;
                        dw[1][6] = w.dy3;
                        dw[1][7] = w.dy4;
                    }
                } else if (r >= ni) {  // far ghost ring: zero gradient (gradient.rs:96)
                    Diff<T> d = diffusion_tensor<T, true>(qw[1][2], UA(3, 4), qw[1][0], qw[1][1], T(0), T(0), T(0),
                                                          T(0), T(0), T(0), T(0), T(0), kc<T>(c.inv_t_ref, K.inv_t_ref), kc<T>(c.suth_num, K.suth_num), kc<T>(c.t_suth, K.t_suth), kc<T>(c.cv1_cubed, K.cv1_cubed), kc<T>(c.inv_pr, K.inv_pr), kc<T>(c.inv_prt, K.inv_prt), kc<T>(c.cp, K.cp), kc<T>(c.sigma, K.sigma));
                    dn[0] = d.dx1;
                    dn[1] = d.dx2;
                    dn[2] = d.dx3;
                    dn[3] = d.dx4;
                    dn[4] = d.dy1;
                    dn[5] = d.dy2;
                    dn[6] = d.dy3;
                    dn[7] = d.dy4;
                }
                // r == -1 on a wall strip: written when row 0 is reached
            }

            // ---- V/dt of row k-2 (clamped, dissipation.rs:59) --------------
            T rtn = T(0);
            {
                int rr = k - 2;
                int gc = S ? rr : (rr < 0 ? 0 : (rr > ni - 1 ? ni - 1 : rr));
                if (S || (rr >= i0 - 1 && rr <= i1)) rtn = PIPE ? B->rat[oT + lane] : ld(ratio + (long)gc * nj + gj);
            }

            // ---- tau face f = k-2 (between rows k-3 and k-2) ---------------
            T ftn[5];
            for (int v = 0; v < 5; ++v) ftn[v] = T(0);
            const int f = k - 2;
            if (S || (f >= i0 && f <= i1)) {
                T m = tmax<T>(tmax<T>(tmax<T>(si[0], si[1]), si[2]), sik);
                T e2 = k2 * m;
                T e4 = tmax<T>(k4 - e2, T(0));
                T lam = half_cfl * (rtn + rt0);
                T fu[5], cv[5];
                T w0[5], w1[5], w2[5], w3[5];
                for (int v = 0; v < 5; ++v) {
                    w0[v] = UA(0, v);
                    w1[v] = UA(1, v);
                    w2[v] = UA(2, v);
                    w3[v] = UA(3, v);
                    fu[v] = w1[v] + w2[v];
                }
                const T fnx = tx[1], fny = ty[1];
                euler_flux<T, true>(fu, fnx, fny, gm1, cv, p_ref2);
                T hx = T(0.5) * fnx, hy = T(0.5) * fny;
                face_combine<T>(w0, w1, w2, w3, cv, dw[0], dw[1], hx, hy, lam, e2, e4, ftn);
            }

            // ---- n faces and the update of row m = k-3 ---------------------
            const int m = k - 3;
            if (S || (m >= i0 && m < i1)) {
                // face between this lane's column and the one to its left
                T fn[5];
                {
                    T m4 = tmax<T>(tmax<T>(tmax<T>(jst_shfl_up(sj[0], 2), jst_shfl_up(sj[0], 1)), sj[0]),
                                   jst_shfl_down(sj[0], 1));
                    T e2 = k2 * m4;
                    T e4 = tmax<T>(k4 - e2, T(0));
                    T lam = half_cfl * (rt0 + jst_shfl_up(rt0, 1));
                    T ul1[5], ul2[5], ur1[5], fu[5], cv[5], um[5];
                    if constexpr (UR) {
                        // the neighbours' U of row m from the ring (one shared
                        // load each instead of two shuffles of the halves);
                        // lanes 0-2 and 31, whose faces are not used, clamp
                        __syncwarp();  // ring rows written by other lanes
                        int sl = s0 + 2;
                        sl = sl >= 5 ? sl - 5 : sl;
                        const int l1 = lane > 0 ? lane - 1 : 0, l2 = lane > 1 ? lane - 2 : 0;
                        const int r1 = lane < 31 ? lane + 1 : 31;
                        for (int v = 0; v < 5; ++v) {
                            const T* ur = uring->u[sl][v];
                            um[v] = ur[lane];
                            ul1[v] = ur[l1];
                            ul2[v] = ur[l2];
                            ur1[v] = ur[r1];
                            fu[v] = ul1[v] + um[v];
                        }
                    } else {
                        for (int v = 0; v < 5; ++v) {
                            um[v] = UA(1, v);
                            ul1[v] = jst_shfl_up(um[v], 1);
                            ul2[v] = jst_shfl_up(um[v], 2);
                            ur1[v] = jst_shfl_down(um[v], 1);
                            fu[v] = ul1[v] + um[v];
                        }
                    }
                    euler_flux<T, true>(fu, nx2[0], ny2[0], gm1, cv, p_ref2);
                    T hx = T(0.5) * nx2[0], hy = T(0.5) * ny2[0];
                    T dl[8];
                    for (int v = 0; v < 8; ++v) dl[v] = jst_shfl_up(dw[0][v], 1);
                    face_combine<T>(ul2, ul1, um, ur1, cv, dl, dw[0], hx, hy, lam, e2, e4, fn);
                }
                T fnr[5];
                for (int v = 0; v < 5; ++v) fnr[v] = jst_shfl_down(fn[v], 1);
                T nxr3 = T(0), nyr3 = T(0);
                if (LAST) {
                    nxr3 = jst_shfl_down(nx2[0], 1);
                    nyr3 = jst_shfl_down(ny2[0], 1);
                }
                // With PIPE every lane computes the update (the row buffer holds
                // the inputs of all 32 lanes, wrapped columns for the halo
                // lanes) and only the output lanes store, so the update is one
                // straight block; without it only the output lanes load.
                if constexpr (DUMP) {
                    if (out_lane) {
                        const long id = (long)m * nj + gj;
                        for (int v = 0; v < 5; ++v) {
                            T Rv = (ftn[v] - ft[v]) + (fnr[v] - fn[v]);
                            if (v == 4) Rv -= sw[0];
                            I.rdump[v * np + id] = (double)Rv;
                        }
                    }
                } else if (PIPE || out_lane) {
                    const long id = (long)m * nj + gj;
                    T R[5];
                    for (int v = 0; v < 5; ++v) R[v] = (ftn[v] - ft[v]) + (fnr[v] - fn[v]);
                    R[4] -= sw[0];
                    double a = dt_local ? alpha * (PIPE ? B->ldt[oD + lane] : ld(I.ldt + id)) : adt;
                    double sc = a * (PIPE ? B->ivm[oD + lane] : ld(I.inv_vol + id));
                    double un[5], uo0 = 0.0;
                    for (int v = 0; v < 5; ++v) {
                        if constexpr (ACC32) {
                            T a0 = FIRST ? UA(1, v) : (PIPE ? B->uacc[v][oT + lane] : ld(I.uc[0] + v * np + id));
                            T nv = a0 - R[v] * (T)sc;
                            un[v] = (double)nv;
                            if (out_lane) dst[v * np + id] = (TD)nv;
                        } else {
                            double uo;
                            if constexpr (UN_RING) uo = (double)UA(1, v);
                            else uo = PIPE ? B->un[v][oD + lane] : I.un[0][v * np + id];
                            if (v == 0) uo0 = uo;
                            if (sizeof(T) == sizeof(double)) un[v] = uo - (double)R[v] * sc;
                            else un[v] = uo - (double)(R[v] * (T)sc);  // FP32 increment, FP64 accumulator
                            if (out_lane) dst[v * np + id] = (TD)un[v];
                            if (LAST && sizeof(T) != sizeof(double) && out_lane) I.uc[0][v * np + id] = (T)un[v];
                        }
                    }
                    // unpack checks (solver.rs:160-171), on the stored precision;
                    // the primitives are formed whether or not rho passed (the
                    // values of a failed cell are not used)
                    bool bad;
                    Prim<double> q{};
                    if (sizeof(T) == sizeof(double)) {
                        double rho = un[0];
                        q = unpack_cell_r<double>(un[0], un[1], un[2], un[3], un[4], c.gm1, (double)inv_rgas);
                        bad = isnan(rho) || rho <= 1e-15 || isnan(q.p) || q.p <= 1e-15;
                    } else {
                        T rho = (T)un[0];
                        Prim<T> qt = unpack_cell_r<T>(rho, (T)un[1], (T)un[2], (T)un[3], (T)un[4], gm1, inv_rgas);
                        bad = isnan(rho) || rho <= T(1e-15) || isnan(qt.p) || qt.p <= T(1e-15);
                        q.vx = qt.vx;
                        q.vy = qt.vy;
                        q.t = qt.t;
                    }
                    bad = bad && out_lane;
                    if (bad) atomicMin(&I.st->bad, (stage_id << 32) | (unsigned long long)id);
                    if (LAST) {
                        const bool ok = out_lane && !bad;
                        double d = un[0] - uo0;  // solver.rs:195
                        sres += ok ? d * d : 0.0;
                        // timestep.rs:30-42 in the stage arithmetic
                        T aa = T(0.5) * (tx[0] + tx[1]);
                        T bb = T(0.5) * (ty[0] + ty[1]);
                        T cc = T(0.5) * (nx2[0] + nxr3);
                        T dd = T(0.5) * (ny2[0] + nyr3);
                        T vol = PIPE ? B->volm[lane] : ld(I.mg + MG_N * (id + nj) + MG_VOL);
                        T qvx = (T)q.vx, qvy = (T)q.vy, qt = (T)q.t;
                        T dl = local_dt<T, true>(qvx, qvy, sq<T, true>(kc<T>(c.rg, K.rg) * qt), aa, bb, cc, dd,
                                                 kc<T>(c.cfl, K.cfl) * vol);
                        if (ok) {
                            ratio_next[id] = dv<T, true>(vol, dl);
                            if (dt_local) I.ldt[id] = (double)dl;
                        }
                        mloc = ok ? fmin(mloc, (double)dl) : mloc;
                    }
                }
            }

            // ---- slide the windows ------------------------------------------
            for (int v = 0; v < 5; ++v) {
                if constexpr (UR) {
                    uring->u[s0][v][lane] = uk[v];
                } else {
                    u[0][v] = u[1][v];
                    u[1][v] = u[2][v];
                    u[2][v] = u[3][v];
                    u[3][v] = uk[v];
                }
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
        };
        const int ks0 = i0 + 3, ks1 = i1 - 2;  // steady rows
        int k = i0 - 3;
        if constexpr (sizeof(T) == sizeof(double)) {
            // The FP64 non-steady body, called from two sites, is compiled
            // out of line (its captured windows then pass through the
            // stack); a single call site keeps it inline.
            for (int ph = 0; ph < 2; ++ph) {
                for (; k <= (ph == 0 ? ks0 - 1 : i1 + 2) && k <= i1 + 2 && !failed; ++k) row(std::false_type{}, k);
                if (ph == 0)
                    for (; k <= ks1 && !failed; ++k) row(std::true_type{}, k);
            }
        } else {
            for (; k < ks0 && k <= i1 + 2 && !failed; ++k) row(std::false_type{}, k);
            for (; k <= ks1 && !failed; ++k) row(std::true_type{}, k);
            for (; k <= i1 + 2 && !failed; ++k) row(std::false_type{}, k);
        }
        if (failed) {  // the strip is abandoned (InstState::err is set)
            dead = true;
            continue;
        }

        if (LAST) {
            double mn = warp_min(mloc);
            double sr = warp_sum0(sres);
            unsigned last = 0;
            if (lane == 0) {
                I.partial[2 * tr.tile] = mn;
                I.partial[2 * tr.tile + 1] = sr;
                JST_FENCE();
                unsigned prev = atomicAdd(&I.st->counter, 1u);
                last = prev == (unsigned)(I.ntiles - 1);
            }
            last = jst_shfl_idx(last, 0);
            if (last) {
                JST_FENCE();
                finish_step_warp<T>(I, true);
            }
        }
    }
}

template <class T, int NT, bool FIRST, bool LAST, bool PIPE = false, bool DUMP = false, int STG = 0>
__global__ void __launch_bounds__(NT, (march_min_blocks<T, NT>()))
    k_march(const TileRef* tiles, int* sched, const Inst<T>* insts, int stage, double alpha) {
    march_body<T, NT, FIRST, LAST, PIPE, DUMP, STG, false>(tiles, sched, insts, stage, alpha, nullptr);
}

// The single-instance launch: the instance descriptor travels by value.
template <class T, int NT, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT, (march_min_blocks<T, NT>()))
    k_march_solo(const TileRef* tiles, int* sched, int stage, double alpha, const __grid_constant__ Inst<T> solo) {
    march_body<T, NT, FIRST, LAST, true, false, 0, true>(tiles, sched, nullptr, stage, alpha, &solo);
}

}  // namespace fused
}  // namespace jst
