// Shared device arithmetic for the JST + Spalart-Allmaras stage kernels.
//
// Every formula keeps the evaluation order of the reference (jst-rs, cited
// file:line), so that a translation unit compiled without FMA contraction
// (the strict FP64 passes path) reproduces the reference's FP64 results, and
// the fused path differs from it only by contraction/precision.  Functions
// are templated on the arithmetic type T (double or float); geometry and
// constants arrive as double and are converted where T = float.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define JST_HD __host__ __device__ __forceinline__
#define JST_D __device__ __forceinline__
#else
#define JST_HD inline
#define JST_D inline
#endif

#ifndef JST_LAUNCH
#define JST_LAUNCH(kern, grid, block, smem, stream, ...) kern<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__)
#endif

namespace jst {

// Per-solve constants: config.rs:11-111 inputs and config.rs:115-145, 173-206 derived
// values, plus a few constant sub-expressions the reference evaluates inline
// (each is a pure function of constants, so precomputing it is exact).
struct PhysConst {
    double gamma, r_gas, t_suth, cfl, t_inf, p_inf, k2, k4;
    double Cb1, Cb2, Ct3, Ct4, Cw2, fv3, rmax, sigma;
    double cv, cp, cw1, cv1_cubed, c_inf, u_inf, v_inf, rho_inf, mu_inf, nut_inf;
    double suth_num, inv_t_ref, inv_pr, inv_prt, inv_kappa2, cw3_6, one_plus_cw3_6;
    double gm1;          // gamma - 1.0
    double rg;           // r_gas * gamma (== gamma * r_gas)
    double gm1_q;        // (gamma - 1.0) / 4.0          boundary.rs:129
    double inv_gm1;      // 1.0 / (gamma - 1.0)          boundary.rs:140
    double half_cfl;     // 0.5 * cfl                    dissipation.rs:61,67
    double cb1_k2;       // Cb1 * inv_kappa2             source.rs:52
    double cb2_sigma;    // Cb2 * sigma                  source.rs:53
    double r_gas_gamma;  // r_gas * gamma                boundary.rs:139 (c^2/(r_gas*gamma))
    double fw_lim;       // (1 + Cw3^6)^(1/6), the limit of fw for large g
    int supersonic;
    int halo;
    // Free-stream primitive state written by Cells::initialize (state.rs:174-190).
    double f_rho, f_p, f_t, f_vx, f_vy, f_e, f_h, f_c, f_nut, f_mu;
};

// x.powi(n) for the constant exponents the reference uses, expanded by binary
// decomposition as LLVM lowers powi with a constant exponent.
template <class T> JST_HD T powi2(T x) { return x * x; }
template <class T> JST_HD T powi3(T x) { return x * (x * x); }
template <class T> JST_HD T powi6(T x) {
    T x2 = x * x;
    T x4 = x2 * x2;
    return x2 * x4;
}

// Quotient and square root for the fused kernels (Q = true); the strict
// passes path keeps the library's correctly rounded / and sqrt (Q = false).
// In double on the device they avoid the library routines' special-case
// branch, which splits the instruction scheduler's basic blocks in the middle
// of every cell's arithmetic:
//  * a / b: the hardware reciprocal approximation of b refined by one
//    third-order Newton-Raphson step r <- r (1 + e + e^2), e = 1 - b r (the
//    relative error is cubed), then one residual correction of the quotient
//    q <- q + r (a - b q) (Markstein, IA-64 and Elementary Functions, 2000);
//  * sqrt(x): the hardware reciprocal square root approximation y refined by
//    one Newton-Raphson step y <- y (3/2 - x y^2 / 2), then the correction
//    s <- s + (y / 2) (x - s^2) of s = x y (same reference).
// Both stay within one unit in the last place of the correctly rounded
// result for normal finite operands (b != 0, x > 0), which is all these
// kernels divide by or take roots of; a NaN operand gives NaN.  In float the
// quotient is the hardware's approximate division (__fdividef: the
// reciprocal approximation times a, within 2 units in the last place for
// |b| < 2^126, beyond every quantity these kernels divide by), and the root
// the translation unit's square root.
template <class T, bool Q = false> JST_HD T dv(T a, T b) { return a / b; }
template <class T, bool Q = false> JST_HD T sq(T x) { return sqrt(x); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ float dv<float, true>(float a, float b) { return __fdividef(a, b); }
template <> __device__ __forceinline__ double dv<double, true>(double a, double b) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    const double e = fma(-b, r, 1.0);
    r = fma(r, fma(e, e, e), r);
    const double q = a * r;
    return fma(r, fma(-b, q, a), q);
}
template <> __device__ __forceinline__ double sq<double, true>(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * y;
    y = fma(h, fma(-x * y, y, 1.0), y);
    const double s = x * y;
    return fma(0.5 * y, fma(-s, s, x), s);
}
#endif

// exp for the fused kernels (Q = true), in double without the library
// routine's range branch: Cody-Waite reduction x = n ln2 + r, |r| <= ln2/2,
// with ln 2 split into a 42-bit head (n ln2_hi is exact for |n| < 2^11) and
// its tail (Cody and Waite, Software Manual for the Elementary Functions,
// 1980); the Taylor polynomial of e^r to degree 13 (truncation error below
// 2^-57) in Horner form; the scaling by 2^n as two exact powers of two, so
// that a result in the subnormal range is rounded once.  Arguments are
// clamped to [-746, 710] (e^-746 rounds to 0, e^710 overflows); NaN gives NaN.
template <class T, bool Q = false> JST_HD T ex(T x) { return exp(x); }
#ifdef __CUDACC__
// 2^n for -1022 <= n <= 1023, from the exponent field.
__device__ __forceinline__ double pow2i(int n) { return __hiloint2double((n + 1023) << 20, 0); }
#endif
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ double ex<double, true>(double x) {
    x = x < -746.0 ? -746.0 : (x > 710.0 ? 710.0 : x);
    const double n = rint(x * 1.4426950408889634);  // log2(e)
    const double r = fma(-n, 0x1.ef35793c7673p-45, fma(-n, 0x1.62e42fefa38p-1, x));
    double p = 1.0 / 6227020800.0;  // 1/13!
    p = fma(p, r, 1.0 / 479001600.0);
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const int k = (int)n, k1 = k / 2;
    return p * pow2i(k1) * pow2i(k - k1);
}
#endif

#ifdef __CUDACC__
// d^(-1/6) for d > 0 in double without library calls or branches: d is
// scaled by the exact power of two 2^(-6m) into [1, 64); an FP32 estimate of
// the scaled root from the hardware base-2 logarithm and exponential is
// refined by two Newton-Raphson steps for t^-6 = d, t <- t + t (1 - d t^6) / 6
// (each squares the relative error), and multiplied by 2^-m.  d = +inf gives
// 0 (the limit), NaN gives NaN.
__device__ __forceinline__ double rroot6(double d) {
    const int e = ((__double2hiint(d) >> 20) & 0x7ff) - 1023;
    const int m = (e + 1200) / 6 - 200;  // floor(e / 6) for e >= -1200
    const double ds = d * pow2i(-3 * m) * pow2i(-3 * m);
    double t = (double)exp2f(__log2f((float)ds) * (-1.0f / 6.0f));
    for (int it = 0; it < 2; ++it) {
        const double t2 = t * t;
        t = fma(t * (1.0 / 6.0), fma(-ds, t2 * t2 * t2, 1.0), t);
    }
    t *= pow2i(-m);
    return isinf(d) ? 0.0 : t;
}
#endif

template <class T> JST_HD T tmax(T a, T b) { return fmax(a, b); }
template <class T> JST_HD T tmin(T a, T b) { return fmin(a, b); }
template <> JST_HD float tmax<float>(float a, float b) { return fmaxf(a, b); }
template <> JST_HD float tmin<float>(float a, float b) { return fminf(a, b); }

// Primitive state of one cell.
template <class T> struct Prim {
    T rho, p, t, vx, vy, e, nut;
};

// Solver::unpack (solver.rs:158-181) for one cell, without the checks.
template <class T, bool Q = false> JST_HD Prim<T> unpack_cell(T u0, T u1, T u2, T u3, T u4, T gm1, T r_gas) {
    Prim<T> q;
    T rho = u0;
    T inv = dv<T, Q>(T(1), rho);
    q.rho = rho;
    q.vx = u1 * inv;
    q.vy = u2 * inv;
    q.e = u3 * inv;
    q.p = gm1 * (u3 - rho * (q.vx * q.vx + q.vy * q.vy) * T(0.5));
    q.t = dv<T, Q>(q.p, r_gas * rho);
    q.nut = u4 * inv;
    return q;
}

// Cells::pack (state.rs:143-156).
template <class T> JST_HD void pack_cell(const Prim<T>& q, T* u) {
    u[0] = q.rho;
    u[1] = q.rho * q.vx;
    u[2] = q.rho * q.vy;
    u[3] = q.rho * q.e;
    u[4] = q.rho * q.nut;
}

// Config::mu, Sutherland (config.rs:210-213).
template <class T, bool Q = false> JST_HD T mu_of(T t, T inv_t_ref, T suth_num, T t_suth) {
    T r = t * inv_t_ref;
    return dv<T, Q>(r * sq<T, Q>(r) * suth_num, t + t_suth);
}

// convection::euler_flux (convection.rs:25-40): F.n of the face state fu.
// p_ref is subtracted from the pressure in the momentum flux only: with
// closed metrics (sum of n over a cell = 0) the cell sums are unchanged, and
// in FP32 the large constant part of p no longer cancels between the two
// faces of a thin wall cell.  The FP64 paths pass p_ref = 0, i.e. the
// reference's formula.
template <class T, bool Q = false>
JST_HD void euler_flux(const T fu[5], T nx, T ny, T gm1, T out[5], T p_ref = T(0)) {
    T rho = fu[0];
    T inv_rho = dv<T, Q>(T(1), rho);
    T u = fu[1] * inv_rho;
    T v = fu[2] * inv_rho;
    T rho_e = fu[3];
    T p = gm1 * (rho_e - rho * (u * u + v * v) * T(0.5));
    T vn = nx * u + ny * v;
    T pm = p - p_ref;
    out[0] = rho * vn;
    out[1] = fu[1] * vn + pm * nx;
    out[2] = fu[2] * vn + pm * ny;
    out[3] = (rho_e + p) * vn;
    out[4] = fu[4] * vn;
}

// Green-Gauss sum of one scalar (gradient.rs:22-35).  c, up, dn, lf, rt are
// the cell value and its i+1, i-1, j-1, j+1 neighbours; the faces are
// tau(i+1), tau(i), n(j), n(j+1).
template <class T>
JST_HD void green_gauss(T c, T vup, T vdn, T vlf, T vrt, T upx, T upy, T dnx, T dny, T lfx, T lfy, T rtx, T rty,
                        T inv_v, T* gx, T* gy) {
    // the face values' factor 1/2 is applied once, to 1/V: scaling by a
    // power of two is exact, so the result is bit for bit the reference's
    T f_up = c + vup;
    T f_dn = c + vdn;
    T f_lf = c + vlf;
    T f_rt = c + vrt;
    T h = T(0.5) * inv_v;
    *gx = (f_up * upx - f_dn * dnx + f_rt * rtx - f_lf * lfx) * h;
    *gy = (f_up * upy - f_dn * dny + f_rt * rty - f_lf * lfy) * h;
}

// The same Green-Gauss sum in difference form, sum_f 0.5 (phi_nb - phi_c) n_f / V:
// identical to green_gauss when the cell's metrics close (sum of n = 0), and
// free of the cancellation of c * sum(n) in FP32.  Used by the FP32 path.
template <class T>
JST_HD void green_gauss_delta(T c, T vup, T vdn, T vlf, T vrt, T upx, T upy, T dnx, T dny, T lfx, T lfy, T rtx,
                              T rty, T inv_v, T* gx, T* gy) {
    T d_up = vup - c;
    T d_dn = vdn - c;
    T d_lf = vlf - c;
    T d_rt = vrt - c;
    T h = T(0.5) * inv_v;  // as in green_gauss
    *gx = (d_up * upx - d_dn * dnx + d_rt * rtx - d_lf * lfx) * h;
    *gy = (d_up * upy - d_dn * dny + d_rt * rty - d_lf * lfy) * h;
}

// Diffusion tensor columns of one cell (viscous.rs:37-71): returns mu, chi,
// fv1 and Dx[1..4], Dy[1..4] (component 0 is identically zero).
template <class T> struct Diff {
    T mu, chi, fv1;
    T dx1, dx2, dx3, dx4, dy1, dy2, dy3, dy4;
};

template <class T, bool Q = false>
JST_HD Diff<T> diffusion_tensor(T t, T rho_nu, T vx, T vy, T dudx, T dudy, T dvdx, T dvdy, T dtdx, T dtdy, T dnx,
                                T dny, T inv_t_ref, T suth_num, T t_suth, T cv1_cubed, T inv_pr, T inv_prt, T cp,
                                T sigma) {
    Diff<T> d;
    T mu = mu_of<T, Q>(t, inv_t_ref, suth_num, t_suth);
    T chi = dv<T, Q>(rho_nu, mu);
    T c3 = chi * chi * chi;  // viscous.rs:27-30
    T f1 = dv<T, Q>(c3, c3 + cv1_cubed);
    T mu_t = rho_nu * f1;
    T mu_eff = mu + mu_t;
    T lam_eff = mu * inv_pr + mu_t * inv_prt;
    T txx = mu_eff * (T(4.0 / 3.0) * dudx - T(2.0 / 3.0) * dvdy);
    T tyy = mu_eff * (T(4.0 / 3.0) * dvdy - T(2.0 / 3.0) * dudx);
    T txy = mu_eff * (dudy + dvdx);
    T qx = lam_eff * cp * dtdx;
    T qy = lam_eff * cp * dtdy;
    T nu_diff = sigma * (mu + rho_nu);
    d.mu = mu;
    d.chi = chi;
    d.fv1 = f1;
    d.dx1 = txx;
    d.dx2 = txy;
    d.dx3 = vx * txx + vy * txy + qx;
    d.dx4 = nu_diff * dnx;
    d.dy1 = txy;
    d.dy2 = tyy;
    d.dy3 = vx * txy + vy * tyy + qy;
    d.dy4 = nu_diff * dny;
    return d;
}

// dissipation::pressure_sensor (dissipation.rs:29-31).
template <class T, bool Q = false> JST_HD T pressure_sensor(T pm, T p0, T pp) {
    return fabs(dv<T, Q>(pm - T(2) * p0 + pp, pm + T(2) * p0 + pp));
}

// source::fw (source.rs:30-33).
// With Q in double on the device, the root of the quotient is taken as
// fw_lim * (g^6 + Cw3^6)^(-1/6), fw_lim = (1 + Cw3^6)^(1/6) (the same value
// within a few units in the last place, one division fewer).
template <class T, bool Q = false> JST_HD T fw_of(T r, T cw2, T cw3_6, T one_plus_cw3_6, T fw_lim) {
    T g = r + cw2 * (powi6<T>(r) - r);
#ifdef __CUDA_ARCH__
    if constexpr (Q && sizeof(T) == sizeof(double)) return g * fw_lim * rroot6(powi6<T>(g) + cw3_6);
#endif
    (void)fw_lim;
    return g * cbrt(sq<T, Q>(dv<T, Q>(one_plus_cw3_6, powi6<T>(g) + cw3_6)));
}

// fw for the FP32 path.  Near the wall a slightly negative nu-tilde over
// d^2 ~ 1e-12 makes |r| reach 1e7 and more; r^6 then overflows FP32 and the
// reference formula would give inf * 0 = NaN, where FP64 still evaluates it
// (to (1 + Cw3^6)^(1/6) within rounding once g^6 dwarfs Cw3^6).  So g is
// formed in FP64 and, beyond g = 1e5, fw takes that limit.
// The sixth root is taken as 2^(log2(x) / 6) with the hardware base-2
// logarithm and exponential (x > 0 here); in FP32 that is accurate to a few
// units in the last place, against the two library roots sqrt and cbrt.
JST_HD float root6_f32(float x) {
#ifdef __CUDA_ARCH__
    return exp2f(__log2f(x) * (1.0f / 6.0f));
#else
    return std::exp2(std::log2(x) * (1.0f / 6.0f));
#endif
}

JST_HD float exp_f32(float x) {
#ifdef __CUDA_ARCH__
    return __expf(x);
#else
    return std::exp(x);
#endif
}

JST_HD float fw_of_f32(float r, double cw2, double cw3_6, double one_plus_cw3_6, double fw_lim) {
    double rd = (double)r;
    double g = rd + cw2 * (powi6<double>(rd) - rd);
    // both sides evaluated and selected (no branch); g is clamped first so
    // that g^6 stays finite in FP32 (NaN passes through)
    float gf = (float)(g > 1e5 ? 1e5 : g);
    float v = gf * root6_f32((float)one_plus_cw3_6 / (powi6<float>(gf) + (float)cw3_6));
    return g > 1e5 ? (float)fw_lim : v;
}

// fw for the FP32 path without FP64: r is clamped at -1e4 before r^6 is
// formed (r^6 <= 1e24 fits FP32); below the clamp g = r + Cw2 (r^6 - r) is
// beyond 1e5 either way, where fw takes its limit, so the clamp changes no
// result.  Otherwise as fw_of_f32.
JST_HD float fw_f32(float r, float cw2, float cw3_6, float one_plus_cw3_6, float fw_lim) {
    const float rc = fmaxf(r, -1e4f);
    const float g = rc + cw2 * (powi6<float>(rc) - rc);
    const float gf = fminf(g, 1e5f);  // NaN passes through
    const float v = gf * root6_f32(dv<float, true>(one_plus_cw3_6, powi6<float>(gf) + cw3_6));
    return g > 1e5f ? fw_lim : v;
}

// source::compute for one cell (source.rs:55-85), before the factor V,
// given nu_tilde = rho_nu / rho (source.rs:62) as the caller has it.
template <class T, bool Q = false>
JST_HD T sa_source_nt(T rho, T rho_nu, T nu_tilde, T inv_dist2, T chi, T f1, T dvdx, T dudy, T dnx, T dny,
                      const PhysConst& c) {
    T inv_kd2 = inv_dist2 * T(c.inv_kappa2);
    T ft2;
    if constexpr (sizeof(T) == sizeof(float)) ft2 = T(c.Ct3) * exp_f32(-T(c.Ct4) * chi * chi);
    else ft2 = T(c.Ct3) * ex<T, Q>(-T(c.Ct4) * chi * chi);
    T fv2 = T(1) - dv<T, Q>(chi, T(1) + chi * f1);
    T sv = T(c.fv3) * fabs(dvdx - dudy);
    T s_tilde = tmax<T>(sv + nu_tilde * inv_kd2 * fv2, T(1e-10));
    T prod = T(c.Cb1) * (T(1) - ft2) * s_tilde * rho_nu;
    T r = tmin<T>(dv<T, Q>(nu_tilde, s_tilde) * inv_kd2, T(c.rmax));
    T fw;
    if constexpr (sizeof(T) == sizeof(float))
        fw = fw_f32(r, (float)c.Cw2, (float)c.cw3_6, (float)c.one_plus_cw3_6, (float)c.fw_lim);
    else fw = fw_of<T, Q>(r, T(c.Cw2), T(c.cw3_6), T(c.one_plus_cw3_6), T(c.fw_lim));
    T destr = (T(c.cw1) * fw - T(c.cb1_k2) * ft2) * rho * (nu_tilde * nu_tilde * inv_dist2);
    T diff = T(c.cb2_sigma) * rho * (dnx * dnx + dny * dny);
    return prod - destr + diff;
}

template <class T, bool Q = false>
JST_HD T sa_source(T rho, T rho_nu, T inv_dist2, T chi, T f1, T dvdx, T dudy, T dnx, T dny, const PhysConst& c) {
    return sa_source_nt<T, Q>(rho, rho_nu, dv<T, Q>(rho_nu, rho), inv_dist2, chi, f1, dvdx, dudy, dnx, dny, c);
}

// boundary::extrapolate_nut (boundary.rs:158-185).  dist[k], nu[k] belong
// to cell NI-1-k.
JST_HD double extrapolate_nut(const double dist[3], const double nu[3]) {
    const double FLOOR = 1e-10;
    double l1 = dist[0], l2 = dist[1], l3 = dist[2];
    double d12 = l1 - l2, d13 = l1 - l3, d23 = l2 - l3;
    if (fabs(d12) < 1e-14 || fabs(d13) < 1e-14 || fabs(d23) < 1e-14) return fmax(nu[0], FLOOR);
    double v = l2 * l3 / (d12 * d13) * nu[0] + l1 * l3 / (-d12 * d23) * nu[1] + l1 * l2 / (d23 * -d13) * nu[2];
    return v > FLOOR ? v : FLOOR;
}

// boundary::riemann_face (boundary.rs:112-155) for far-field column j, given
// the tau face NI normal (fnx, fny) and midpoint (fmx, fmy), the primitive
// state of cell NI-1 (u, v, c) and, for the nu-tilde extrapolation, the
// centroid distances and nu-tilde of cells NI-1..NI-3.  Returns the face
// state; h and c of the ghost follow as in far_field_riemann (boundary.rs:93-94).
struct FarState {
    double rho, p, t, vx, vy, e, nut;
    int inflow;
};

JST_HD FarState riemann_face(double fnx, double fny, double ui, double vi, double ci, const double dist[3],
                             const double nu[3], const PhysConst& c) {
    double len = hypot(fnx, fny);
    double nx = fnx, ny = fny;
    double gamma = c.gamma;
    double vn_inf = (c.u_inf * nx + c.v_inf * ny) / len;
    double vt_inf = (c.u_inf * ny - c.v_inf * nx) / len;
    double vn_in = (ui * nx + vi * ny) / len;
    double vt_in = (ui * ny - vi * nx) / len;
    double c_face, vn_face, vt_face;
    int inflow;
    if (!c.supersonic) {
        double r_in = vn_in + 2.0 * ci / c.gm1;
        double r_inf = vn_inf - 2.0 * c.c_inf / c.gm1;
        double vn = 0.5 * (r_in + r_inf);
        double cf = c.gm1_q * (r_in - r_inf);
        inflow = vn <= 0.0;
        c_face = cf;
        vn_face = vn;
        vt_face = inflow ? vt_inf : vt_in;
    } else if (vn_inf <= 0.0) {
        c_face = c.c_inf;
        vn_face = vn_inf;
        vt_face = vt_inf;
        inflow = 1;
    } else {
        c_face = ci;
        vn_face = vn_in;
        vt_face = vt_in;
        inflow = 0;
    }
    (void)gamma;
    FarState s;
    double t = c_face * c_face / c.r_gas_gamma;
    double rho = c.rho_inf * pow(t / c.t_inf, c.inv_gm1);
    double p = rho * c.r_gas * t;
    double vx = (vt_face * ny + vn_face * nx) / len;
    double vy = (-vt_face * nx + vn_face * ny) / len;
    s.rho = rho;
    s.p = p;
    s.t = t;
    s.vx = vx;
    s.vy = vy;
    s.e = p / (rho * c.gm1) + 0.5 * (vx * vx + vy * vy);
    s.nut = inflow ? c.nut_inf : extrapolate_nut(dist, nu);
    s.inflow = inflow;
    return s;
}

// timestep::compute for one cell (timestep.rs:30-42): a,b / cc,dd are the
// averaged tau / n normals.
template <class T, bool Q = false> JST_HD T local_dt(T u, T v, T cs, T a, T b, T cc, T dd, T cfl_vol) {
    T conv = fabs(u * a + v * b) + fabs(u * cc + v * dd);
    T acou = cs * (sq<T, Q>(a * a + b * b) + sq<T, Q>(cc * cc + dd * dd));
    return dv<T, Q>(cfl_vol, conv + acou);
}

}  // namespace jst
