// Strict FP64 path: geometry build and one kernel per pass of the reference's
// residual loop, on halo-indexed arrays like the reference's Field<T>
// (field.rs:139-192).  Compiled with --fmad=false so that no a*b+c is fused:
// with the reference's evaluation order kept in jst_common.cuh this
// reproduces the reference's FP64 arithmetic (libm-dependent exp/cbrt/pow/
// hypot aside).  It is the parity mode of the solver and the source of the
// per-term fields (Fc, Fv, Fd, S, gradients, chi, fv1) that the fused path
// does not materialise.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "jst_common.cuh"
#include "jst_internal.h"

namespace jst {

namespace {

constexpr int TB = 256;

inline unsigned nblk(long n) { return (unsigned)((n + TB - 1) / TB); }

__device__ __forceinline__ long gtid() { return (long)blockIdx.x * blockDim.x + threadIdx.x; }

// Node access with circumferential wrap (mesh.rs:511-516).
struct Nodes {
    const double* xy;
    int n_rings, n_theta;
    __device__ __forceinline__ double x(long r, long t) const { return xy[2 * (r * n_theta + t % n_theta)]; }
    __device__ __forceinline__ double y(long r, long t) const { return xy[2 * (r * n_theta + t % n_theta) + 1]; }
};

// ---------------------------------------------------------------- geometry --
// geometry.rs:109-145
__global__ void k_geom_cells(Nodes m, Geom g) {
    long id = gtid();
    long n = (long)g.ni * g.nj;
    if (id >= n) return;
    long i = id / g.nj, j = id % g.nj;
    double ax = m.x(i, j), ay = m.y(i, j);
    double bx = m.x(i + 1, j), by = m.y(i + 1, j);
    double cx = m.x(i + 1, j + 1), cy = m.y(i + 1, j + 1);
    double dx = m.x(i, j + 1), dy = m.y(i, j + 1);
    double d1x = cx - ax, d1y = cy - ay;
    double d2x = bx - dx, d2y = by - dy;
    double vol = 0.5 * fabs(d1x * d2y - d1y * d2x);
    double cr0 = ax * by - bx * ay;
    double cr1 = bx * cy - cx * by;
    double cr2 = cx * dy - dx * cy;
    double cr3 = dx * ay - ax * dy;
    double sgn = 0.5 * (cr0 + cr1 + cr2 + cr3);
    double sx = (ax + bx) * cr0 + (bx + cx) * cr1 + (cx + dx) * cr2 + (dx + ax) * cr3;
    double sy = (ay + by) * cr0 + (by + cy) * cr1 + (cy + dy) * cr2 + (dy + ay) * cr3;
    g.vol[id] = vol;
    g.cx[id] = fabs(sgn) > 1e-30 ? sx / (6.0 * sgn) : 0.0;
    g.cy[id] = fabs(sgn) > 1e-30 ? sy / (6.0 * sgn) : 0.0;
    g.inv_vol[id] = 1.0 / vol;  // geometry.rs:97
}

// geometry.rs:148-185
__global__ void k_geom_faces(Nodes m, Geom g) {
    long id = gtid();
    long nt = (long)(g.ni + 1) * g.nj, nn = (long)g.ni * g.nj;
    if (id < nt) {
        long i = id / g.nj, j = id % g.nj;
        double ax = m.x(i, j), ay = m.y(i, j);
        double bx = m.x(i, j + 1), by = m.y(i, j + 1);
        double dx = bx - ax, dy = by - ay;
        g.tnx[id] = dy;
        g.tny[id] = -dx;
        g.tmx[id] = 0.5 * (ax + bx);
        g.tmy[id] = 0.5 * (ay + by);
    } else if (id < nt + nn) {
        long k = id - nt;
        long i = k / g.nj, j = k % g.nj;
        double ax = m.x(i, j), ay = m.y(i, j);
        double bx = m.x(i + 1, j), by = m.y(i + 1, j);
        double dx = bx - ax, dy = by - ay;
        g.nnx[k] = -dy;
        g.nny[k] = dx;
        g.nmx[k] = 0.5 * (ax + bx);
        g.nmy[k] = 0.5 * (ay + by);
    }
}

// geometry.rs:192-216 and 95-101.  One thread per cell; the wall midpoints of
// a block's window are read through L1/L2.
__global__ void k_geom_wall(Geom g, int window) {
    long id = gtid();
    long n = (long)g.ni * g.nj;
    if (id >= n) return;
    long nj = g.nj;
    long j = id % nj;
    double px = g.cx[id], py = g.cy[id];
    double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    for (long dk = -window; dk <= window; ++dk) {
        long k = ((j + dk) % nj + nj) % nj;
        double ex = px - g.tmx[k], ey = py - g.tmy[k];
        double d = sqrt(powi2(ex) + powi2(ey));
        if (d < best) best = d;
    }
    g.wdist[id] = best;
    g.inv_d2[id] = 1.0 / (best * best);
}

// The same wall distance, one block per (row i, 256 consecutive columns): the
// block's window of wall midpoints is staged in shared memory once, and since
// sqrt is monotonic and correctly rounded, sqrt(min d^2) is the reference's
// min sqrt(d^2) bit for bit, with one square root per cell.
constexpr int kWallBlock = 256;
constexpr size_t kWallSmemMax = 200 * 1024;

__global__ void __launch_bounds__(kWallBlock) k_geom_wall_rows(Geom g, int window) {
    extern __shared__ double wm[];  // x then y of faces j0-window .. j0+kWallBlock-1+window
    const int L = 2 * window + kWallBlock;
    double* sx = wm;
    double* sy = wm + L;
    const long nj = g.nj;
    const long j0 = (long)blockIdx.x * kWallBlock;
    for (int e = threadIdx.x; e < L; e += kWallBlock) {
        long k = ((j0 - window + e) % nj + nj) % nj;  // geometry.rs:206 rem_euclid
        sx[e] = g.tmx[k];
        sy[e] = g.tmy[k];
    }
    __syncthreads();
    const long j = j0 + threadIdx.x;
    if (j >= nj) return;
    const long id = (long)blockIdx.y * nj + j;
    const double px = g.cx[id], py = g.cy[id];
    double best2 = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    for (int e = threadIdx.x; e <= threadIdx.x + 2 * window; ++e) {
        double ex = px - sx[e], ey = py - sy[e];
        double d2 = powi2(ex) + powi2(ey);
        if (d2 < best2) best2 = d2;
    }
    const double best = sqrt(best2);
    g.wdist[id] = best;
    g.inv_d2[id] = 1.0 / (best * best);
}

// ------------------------------------------------------------ passes path --
struct DF {
    double* p;
    int h, stride;
    __device__ __forceinline__ double& operator()(long i, long j) const { return p[(i + h) * (long)stride + j + h]; }
};

struct PS {  // device view of the passes-path state
    int ni, nj, H;
    DF U[5], Uf[5];
    DF rho, p, t, vx, vy, e, hh, c, nut;
    DF g[8];
    DF mu, chi, fv1;
    DF Dx[5], Dy[5];
    DF fc[5], fv[5], fd[5];
    DF src, localdt, sensor_i, sensor_j, spec_ratio, rho_prev;
    double *tflux, *nflux, *tdiff, *ndiff, *tdiss, *ndiss;  // [face*5 + k]
    double *tlam, *nlam, *te2, *te4, *ne2, *ne4;
    double *dt, *totaltime, *partial, *residual;
    unsigned long long* bad;
};

__device__ __forceinline__ void pack_at(const PS& s, long i, long j) {
    double r = s.rho(i, j);
    s.U[0](i, j) = r;
    s.U[1](i, j) = r * s.vx(i, j);
    s.U[2](i, j) = r * s.vy(i, j);
    s.U[3](i, j) = r * s.e(i, j);
    s.U[4](i, j) = r * s.nut(i, j);
}

// Cells::initialize (state.rs:174-190) for interior cells.
__global__ void k_init(PS s, PhysConst c) {
    long id = gtid();
    if (id >= (long)s.ni * s.nj) return;
    long i = id / s.nj, j = id % s.nj;
    s.rho(i, j) = c.f_rho;
    s.p(i, j) = c.f_p;
    s.t(i, j) = c.f_t;
    s.vx(i, j) = c.f_vx;
    s.vy(i, j) = c.f_vy;
    s.e(i, j) = c.f_e;
    s.hh(i, j) = c.f_h;
    s.c(i, j) = c.f_c;
    s.nut(i, j) = c.f_nut;
    pack_at(s, i, j);
    s.mu(i, j) = c.f_mu;
    s.chi(i, j) = 0.0;
    s.fv1(i, j) = 0.0;
}

// state.rs:198-203 for every addressable cell.
__global__ void k_set_uniform(PS s, double rho, double p, double t, double vx, double vy, double e, double h,
                              double cc, double nut) {
    long W = s.nj + 2 * s.H;
    long id = gtid();
    if (id >= (long)(s.ni + 2 * s.H) * W) return;
    long i = id / W - s.H, j = id % W - s.H;
    s.rho(i, j) = rho;
    s.p(i, j) = p;
    s.t(i, j) = t;
    s.vx(i, j) = vx;
    s.vy(i, j) = vy;
    s.e(i, j) = e;
    s.hh(i, j) = h;
    s.c(i, j) = cc;
    s.nut(i, j) = nut;
    pack_at(s, i, j);
}

// boundary.rs:30-51 — thread (k, j).
__global__ void k_bc_wall(PS s) {
    long id = gtid();
    if (id >= (long)s.H * s.nj) return;
    long k = id / s.nj, j = id % s.nj;
    long g = -1 - k;
    s.rho(g, j) = s.rho(k, j);
    s.p(g, j) = s.p(k, j);
    s.t(g, j) = s.t(k, j);
    s.e(g, j) = s.e(k, j);
    s.hh(g, j) = s.hh(k, j);
    s.c(g, j) = s.c(k, j);
    s.vx(g, j) = -s.vx(k, j);
    s.vy(g, j) = -s.vy(k, j);
    s.nut(g, j) = -s.nut(k, j);
    pack_at(s, g, j);
}

// boundary.rs:87-109 — thread j.
__global__ void k_bc_far(PS s, Geom g, PhysConst c) {
    long j = gtid();
    if (j >= s.nj) return;
    long ni = s.ni;
    long f = ni * s.nj + j;  // tau face (NI, j)
    double dist[3], nu[3];
    for (int k = 0; k < 3; ++k) {
        long i = ni - 1 - k;
        long cid = i * s.nj + j;
        dist[k] = hypot(g.cx[cid] - g.tmx[f], g.cy[cid] - g.tmy[f]);
        nu[k] = s.nut(i, j);
    }
    FarState q = riemann_face(g.tnx[f], g.tny[f], s.vx(ni - 1, j), s.vy(ni - 1, j), s.c(ni - 1, j), dist, nu, c);
    double cc = sqrt(c.rg * q.t);
    double h = q.e + q.p / q.rho;
    for (long k = 0; k < s.H; ++k) {
        long gi = ni + k;
        s.rho(gi, j) = q.rho;
        s.p(gi, j) = q.p;
        s.t(gi, j) = q.t;
        s.e(gi, j) = q.e;
        s.hh(gi, j) = h;
        s.c(gi, j) = cc;
        s.vx(gi, j) = q.vx;
        s.vy(gi, j) = q.vy;
        s.nut(gi, j) = q.nut;
        pack_at(s, gi, j);
    }
}

// boundary.rs:54-72 — thread (i, k, side).
__global__ void k_bc_periodic(PS s) {
    long id = gtid();
    long per_row = 2L * s.H;
    if (id >= (long)s.ni * per_row) return;
    long i = id / per_row, r = id % per_row;
    long k = r / 2 + 1, side = r % 2;
    long nj = s.nj;
    long g = side == 0 ? -k : nj - 1 + k;
    long src = side == 0 ? nj - k : k - 1;
    s.rho(i, g) = s.rho(i, src);
    s.p(i, g) = s.p(i, src);
    s.t(i, g) = s.t(i, src);
    s.e(i, g) = s.e(i, src);
    s.hh(i, g) = s.hh(i, src);
    s.c(i, g) = s.c(i, src);
    s.vx(i, g) = s.vx(i, src);
    s.vy(i, g) = s.vy(i, src);
    s.nut(i, g) = s.nut(i, src);
    pack_at(s, i, g);
}

// timestep.rs:24-47 — thread per interior cell.
__global__ void k_timestep(PS s, Geom g, double cfl) {
    long id = gtid();
    long nj = s.nj;
    if (id >= (long)s.ni * nj) return;
    long i = id / nj, j = id % nj;
    long jp = j + 1 < nj ? j + 1 : 0;
    long t0 = i * nj + j, t1 = (i + 1) * nj + j, n0 = i * nj + j, n1 = i * nj + jp;
    double a = 0.5 * (g.tnx[t0] + g.tnx[t1]);
    double b = 0.5 * (g.tny[t0] + g.tny[t1]);
    double cc = 0.5 * (g.nnx[n0] + g.nnx[n1]);
    double dd = 0.5 * (g.nny[n0] + g.nny[n1]);
    s.localdt(i, j) = local_dt<double>(s.vx(i, j), s.vy(i, j), s.c(i, j), a, b, cc, dd, cfl * g.vol[id]);
}

// Exact global minimum of an interior field: per-block minima, then one block.
__global__ void k_min_partial(DF f, int ni, int nj, double* partial) {
    __shared__ double sm[TB];
    long id = gtid();
    double m = __longlong_as_double(0x7ff0000000000000LL);
    if (id < (long)ni * nj) m = f(id / nj, id % nj);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = TB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void k_min_final(const double* partial, int n, double* dt, double* totaltime, int accumulate) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double m = __longlong_as_double(0x7ff0000000000000LL);
    for (int k = 0; k < n; ++k) m = fmin(m, partial[k]);
    *dt = m;
    if (accumulate) *totaltime += m;
}

// convection.rs:46-68 — tau faces then n faces, one thread per face.
__global__ void k_conv_faces(PS s, Geom g, double gm1) {
    long id = gtid();
    long nj = s.nj;
    long nt = (long)(s.ni + 1) * nj, nn = (long)s.ni * nj;
    double fu[5], out[5];
    if (id < nt) {
        long i = id / nj, j = id % nj;
        for (int k = 0; k < 5; ++k) fu[k] = 0.5 * (s.U[k](i - 1, j) + s.U[k](i, j));
        euler_flux<double>(fu, g.tnx[id], g.tny[id], gm1, out);
        for (int k = 0; k < 5; ++k) s.tflux[id * 5 + k] = out[k];
    } else if (id < nt + nn) {
        long f = id - nt;
        long i = f / nj, j = f % nj;
        for (int k = 0; k < 5; ++k) fu[k] = 0.5 * (s.U[k](i, j - 1) + s.U[k](i, j));
        euler_flux<double>(fu, g.nnx[f], g.nny[f], gm1, out);
        for (int k = 0; k < 5; ++k) s.nflux[f * 5 + k] = out[k];
    }
}

// convection.rs:71-80, viscous.rs:156-163 (same circulation form):
// out = a(i+1) - a(i) + b(jp1) - b(j).
__global__ void k_circulation(PS s, const double* tf, const double* nf, int which) {
    long id = gtid();
    long nj = s.nj;
    if (id >= (long)s.ni * nj) return;
    long i = id / nj, j = id % nj;
    long jp = j + 1 < nj ? j + 1 : 0;
    for (int k = 0; k < 5; ++k) {
        double v = tf[((i + 1) * nj + j) * 5 + k] - tf[(i * nj + j) * 5 + k] + nf[(i * nj + jp) * 5 + k] -
                   nf[(i * nj + j) * 5 + k];
        if (which == 0) s.fc[k](i, j) = v;
        else s.fv[k](i, j) = v;
    }
}

// gradient.rs:38-80 — thread per interior cell.
__global__ void k_grad(PS s, Geom g) {
    long id = gtid();
    long nj = s.nj;
    if (id >= (long)s.ni * nj) return;
    long i = id / nj, j = id % nj;
    long jp = j + 1 < nj ? j + 1 : 0;
    long up = (i + 1) * nj + j, dn = i * nj + j, lf = i * nj + j, rt = i * nj + jp;
    double iv = g.inv_vol[id];
    const DF* src[4] = {&s.vx, &s.vy, &s.t, &s.nut};
    for (int q = 0; q < 4; ++q) {
        const DF& f = *src[q];
        double gx, gy;
        green_gauss<double>(f(i, j), f(i + 1, j), f(i - 1, j), f(i, j - 1), f(i, j + 1), g.tnx[up], g.tny[up],
                            g.tnx[dn], g.tny[dn], g.nnx[lf], g.nny[lf], g.nnx[rt], g.nny[rt], iv, &gx, &gy);
        s.g[2 * q](i, j) = gx;
        s.g[2 * q + 1](i, j) = gy;
    }
}

// gradient.rs:87-102 — threads 0..NJ-1 fill wall/far rows, NJ.. the seams.
__global__ void k_grad_ghost(PS s) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    if (id < nj) {
        long j = id;
        for (int k = 0; k < 8; ++k) s.g[k](-1, j) = s.g[k](0, j);
        s.g[4](-1, j) = 0.0;
        s.g[5](-1, j) = 0.0;
        for (int k = 0; k < 8; ++k) s.g[k](ni, j) = 0.0;
    } else if (id < nj + ni) {
        long i = id - nj;
        for (int k = 0; k < 8; ++k) {
            s.g[k](i, -1) = s.g[k](i, nj - 1);
            s.g[k](i, nj) = s.g[k](i, 0);
        }
    }
}

// viscous.rs:74-125 — interior cells, then the first ghost ring (no corners).
__global__ void k_visc_cells(PS s, PhysConst c) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    long n_int = ni * nj;
    long i, j;
    if (id < n_int) {
        i = id / nj;
        j = id % nj;
    } else if (id < n_int + 2 * nj) {
        long r = id - n_int;
        j = r / 2;
        i = (r % 2 == 0) ? -1 : ni;
    } else if (id < n_int + 2 * nj + 2 * ni) {
        long r = id - n_int - 2 * nj;
        i = r / 2;
        j = (r % 2 == 0) ? -1 : nj;
    } else {
        return;
    }
    Diff<double> d = diffusion_tensor<double>(
        s.t(i, j), s.U[4](i, j), s.vx(i, j), s.vy(i, j), s.g[0](i, j), s.g[1](i, j), s.g[2](i, j), s.g[3](i, j),
        s.g[4](i, j), s.g[5](i, j), s.g[6](i, j), s.g[7](i, j), c.inv_t_ref, c.suth_num, c.t_suth, c.cv1_cubed,
        c.inv_pr, c.inv_prt, c.cp, c.sigma);
    s.mu(i, j) = d.mu;
    s.chi(i, j) = d.chi;
    s.fv1(i, j) = d.fv1;
    s.Dx[0](i, j) = 0.0;
    s.Dx[1](i, j) = d.dx1;
    s.Dx[2](i, j) = d.dx2;
    s.Dx[3](i, j) = d.dx3;
    s.Dx[4](i, j) = d.dx4;
    s.Dy[0](i, j) = 0.0;
    s.Dy[1](i, j) = d.dy1;
    s.Dy[2](i, j) = d.dy2;
    s.Dy[3](i, j) = d.dy3;
    s.Dy[4](i, j) = d.dy4;
}

// viscous.rs:128-149 — face diffusion flux, tau faces then n faces.
__global__ void k_visc_faces(PS s, Geom g) {
    long id = gtid();
    long nj = s.nj;
    long nt = (long)(s.ni + 1) * nj, nn = (long)s.ni * nj;
    if (id < nt) {
        long i = id / nj, j = id % nj;
        double hx = 0.5 * g.tnx[id], hy = 0.5 * g.tny[id];
        for (int k = 0; k < 5; ++k)
            s.tdiff[id * 5 + k] = (s.Dx[k](i - 1, j) + s.Dx[k](i, j)) * hx + (s.Dy[k](i - 1, j) + s.Dy[k](i, j)) * hy;
    } else if (id < nt + nn) {
        long f = id - nt;
        long i = f / nj, j = f % nj;
        double hx = 0.5 * g.nnx[f], hy = 0.5 * g.nny[f];
        for (int k = 0; k < 5; ++k)
            s.ndiff[f * 5 + k] = (s.Dx[k](i, j - 1) + s.Dx[k](i, j)) * hx + (s.Dy[k](i, j - 1) + s.Dy[k](i, j)) * hy;
    }
}

// dissipation.rs:44-70 — spectral ratio per interior cell.
__global__ void k_diss_ratio(PS s, Geom g) {
    long id = gtid();
    if (id >= (long)s.ni * s.nj) return;
    long i = id / s.nj, j = id % s.nj;
    s.spec_ratio(i, j) = g.vol[id] / s.localdt(i, j);
}

// dissipation.rs:57-69 — face lambdas.
__global__ void k_diss_lambda(PS s, double half_cfl) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    long nt = (ni + 1) * nj, nn = ni * nj;
    if (id < nt) {
        long i = id / nj, j = id % nj;
        long a = i < 0 ? 0 : (i > ni - 1 ? ni - 1 : i);
        long b = i - 1 < 0 ? 0 : (i - 1 > ni - 1 ? ni - 1 : i - 1);
        s.tlam[id] = half_cfl * (s.spec_ratio(a, j) + s.spec_ratio(b, j));
    } else if (id < nt + nn) {
        long f = id - nt;
        long i = f / nj, j = f % nj;
        long jm = j > 0 ? j - 1 : nj - 1;
        s.nlam[f] = half_cfl * (s.spec_ratio(i, j) + s.spec_ratio(i, jm));
    }
}

// dissipation.rs:73-90 — sensor_i on rows -2..NI+1, sensor_j on columns -2..NJ.
__global__ void k_sensors(PS s) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    long n1 = (ni + 4) * nj, n2 = ni * (nj + 3);
    if (id < n1) {
        long i = id / nj - 2, j = id % nj;
        s.sensor_i(i, j) = pressure_sensor<double>(s.p(i - 1, j), s.p(i, j), s.p(i + 1, j));
    } else if (id < n1 + n2) {
        long r = id - n1;
        long i = r / (nj + 3), j = r % (nj + 3) - 2;
        s.sensor_j(i, j) = pressure_sensor<double>(s.p(i, j - 1), s.p(i, j), s.p(i, j + 1));
    }
}

// dissipation.rs:93-126 (adaptive_coefficients 35-38).
__global__ void k_diss_coef(PS s, double k2, double k4) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    long nt = (ni + 1) * nj, nn = ni * nj;
    if (id < nt) {
        long i = id / nj, j = id % nj;
        double m = fmax(fmax(fmax(s.sensor_i(i - 2, j), s.sensor_i(i - 1, j)), s.sensor_i(i, j)), s.sensor_i(i + 1, j));
        double e2 = k2 * m;
        s.te2[id] = e2;
        s.te4[id] = fmax(k4 - e2, 0.0);
    } else if (id < nt + nn) {
        long f = id - nt;
        long i = f / nj, j = f % nj;
        double m = fmax(fmax(fmax(s.sensor_j(i, j - 2), s.sensor_j(i, j - 1)), s.sensor_j(i, j)), s.sensor_j(i, j + 1));
        double e2 = k2 * m;
        s.ne2[f] = e2;
        s.ne4[f] = fmax(k4 - e2, 0.0);
    }
}

// dissipation.rs:129-166.
__global__ void k_diss_faces(PS s) {
    long id = gtid();
    long ni = s.ni, nj = s.nj;
    long nt = (ni + 1) * nj, nn = ni * nj;
    if (id < nt) {
        long i = id / nj, j = id % nj;
        for (int k = 0; k < 5; ++k) {
            const DF& u = s.U[k];
            double d1 = u(i, j) - u(i - 1, j);
            double d3 = u(i + 1, j) - 3.0 * u(i, j) + 3.0 * u(i - 1, j) - u(i - 2, j);
            s.tdiss[id * 5 + k] = s.tlam[id] * (d1 * s.te2[id] - d3 * s.te4[id]);
        }
    } else if (id < nt + nn) {
        long f = id - nt;
        long i = f / nj, j = f % nj;
        for (int k = 0; k < 5; ++k) {
            const DF& u = s.U[k];
            double d1 = u(i, j) - u(i, j - 1);
            double d3 = u(i, j + 1) - 3.0 * u(i, j) + 3.0 * u(i, j - 1) - u(i, j - 2);
            s.ndiss[f * 5 + k] = s.nlam[f] * (d1 * s.ne2[f] - d3 * s.ne4[f]);
        }
    }
}

// dissipation.rs:176-185.
__global__ void k_diss_assemble(PS s) {
    long id = gtid();
    long nj = s.nj;
    if (id >= (long)s.ni * nj) return;
    long i = id / nj, j = id % nj;
    long jp = j + 1 < nj ? j + 1 : 0;
    for (int k = 0; k < 5; ++k)
        s.fd[k](i, j) = s.tdiss[((i + 1) * nj + j) * 5 + k] + s.ndiss[(i * nj + jp) * 5 + k] -
                        s.tdiss[(i * nj + j) * 5 + k] - s.ndiss[(i * nj + j) * 5 + k];
}

// source.rs:45-88.
__global__ void k_source(PS s, Geom g, PhysConst c) {
    long id = gtid();
    if (id >= (long)s.ni * s.nj) return;
    long i = id / s.nj, j = id % s.nj;
    double v = sa_source<double>(s.U[0](i, j), s.U[4](i, j), g.inv_d2[id], s.chi(i, j), s.fv1(i, j), s.g[2](i, j),
                                 s.g[1](i, j), s.g[6](i, j), s.g[7](i, j), c);
    s.src(i, j) = v * g.vol[id];
}

// solver.rs:123-145 (local: each cell uses alpha*localdt).
__global__ void k_update(PS s, Geom g, double alpha, int local) {
    long id = gtid();
    if (id >= (long)s.ni * s.nj) return;
    long i = id / s.nj, j = id % s.nj;
    double a = local ? alpha * s.localdt(i, j) : alpha * *s.dt;
    double r[5];
    for (int k = 0; k < 5; ++k) r[k] = s.fc[k](i, j) - s.fv[k](i, j) - s.fd[k](i, j);
    r[4] -= s.src(i, j);
    double sc = a * g.inv_vol[id];
    for (int k = 0; k < 5; ++k) s.U[k](i, j) = s.Uf[k](i, j) - r[k] * sc;
}

// solver.rs:151-185.  Good cells are unpacked; the smallest row-major index
// of a failing cell is recorded in *s.bad.
__global__ void k_unpack(PS s, double gm1, double r_gas, double rg) {
    long id = gtid();
    if (id >= (long)s.ni * s.nj) return;
    long i = id / s.nj, j = id % s.nj;
    double rho = s.U[0](i, j);
    if (isnan(rho) || rho <= 1e-15) {
        atomicMin(s.bad, (unsigned long long)id);
        return;
    }
    double inv = 1.0 / rho;
    double vx = s.U[1](i, j) * inv, vy = s.U[2](i, j) * inv;
    double e = s.U[3](i, j) * inv;
    double p = gm1 * (s.U[3](i, j) - rho * (vx * vx + vy * vy) * 0.5);
    if (isnan(p) || p <= 1e-15) {
        atomicMin(s.bad, (unsigned long long)id);
        return;
    }
    double t = p / (r_gas * rho);
    s.rho(i, j) = rho;
    s.vx(i, j) = vx;
    s.vy(i, j) = vy;
    s.nut(i, j) = s.U[4](i, j) * inv;
    s.e(i, j) = e;
    s.p(i, j) = p;
    s.hh(i, j) = e + p * inv;
    s.t(i, j) = t;
    s.c(i, j) = sqrt(rg * t);
}

// Residual sum(rho - rho_prev)^2: fixed-shape per-block tree, then one
// thread sums the block partials in order (run-to-run deterministic).
__global__ void k_res_partial(PS s) {
    __shared__ double sm[TB];
    long id = gtid();
    double v = 0.0;
    if (id < (long)s.ni * s.nj) {
        long i = id / s.nj, j = id % s.nj;
        double d = s.rho(i, j) - s.rho_prev(i, j);
        v = d * d;
    }
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int w = TB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) s.partial[blockIdx.x] = sm[0];
}

__global__ void k_res_final(PS s, int nb) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0.0;
    for (int k = 0; k < nb; ++k) acc += s.partial[k];
    *s.residual = sqrt(acc / (double)s.ni / (double)s.nj);
}

__global__ void k_copy_fields(PS s) {  // U -> U_former, rho -> rho_prev (solver.rs:100-107)
    long n = (long)(s.ni + 2 * s.H) * (s.nj + 2 * s.H);
    long id = gtid();
    if (id >= n) return;
    for (int k = 0; k < 5; ++k) s.Uf[k].p[id] = s.U[k].p[id];
    s.rho_prev.p[id] = s.rho.p[id];
}

// EXT: wall force (see jst_forces): sum over j of -p_w n + Dface(1..2) at
// tau faces of ring 0, one thread, fixed order.
__global__ void k_wall_force(PS s, Geom g, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double ax = 0.0, ay = 0.0;
    for (long j = 0; j < s.nj; ++j) {
        double pw = 0.5 * (s.p(-1, j) + s.p(0, j));
        ax += -pw * g.tnx[j] + s.tdiff[j * 5 + 1];
        ay += -pw * g.tny[j] + s.tdiff[j * 5 + 2];
    }
    out[0] = ax;
    out[1] = ay;
}

}  // namespace

// ------------------------------------------------------------ host side ----
void geometry_build(const double* d_xy, int n_rings, int n_theta, Geom& g, cudaStream_t st) {
    Nodes m{d_xy, n_rings, n_theta};
    long n = (long)g.ni * g.nj, nt = (long)(g.ni + 1) * g.nj;
    JST_LAUNCH(k_geom_cells, nblk(n), TB, 0, st, m, g);
    JST_LAUNCH(k_geom_faces, nblk(nt + n), TB, 0, st, m, g);
    long nj = g.nj;
    int window = (int)std::min(std::max(15L, nj / 5), nj / 2);
    size_t smem = 2 * (size_t)(2 * window + kWallBlock) * sizeof(double);
    if (smem <= kWallSmemMax && g.ni <= 65535 &&
        cudaFuncSetAttribute(k_geom_wall_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
        dim3 grid((unsigned)((nj + kWallBlock - 1) / kWallBlock), (unsigned)g.ni);
        k_geom_wall_rows<<<grid, kWallBlock, smem, st>>>(g, window);
    } else {
        cudaGetLastError();
        JST_LAUNCH(k_geom_wall, nblk(n), TB, 0, st, g, window);
    }
}

struct Passes {
    PS s;
    int ni, nj, H;
    double* arena = nullptr;
    size_t field_elems = 0;
    int nblocks_cells = 0;
};

Passes* passes_create(int ni, int nj, int H, std::string* err) {
    Passes* P = new Passes();
    P->ni = ni;
    P->nj = nj;
    P->H = H;
    size_t W = (size_t)nj + 2 * H;
    size_t fe = (size_t)(ni + 2 * H) * W;
    P->field_elems = fe;
    const int n_cell_fields = 5 + 5 + 9 + 8 + 3 + 5 + 5 + 5 + 5 + 5 + 6;
    size_t nt = (size_t)(ni + 1) * nj, nn = (size_t)ni * nj;
    size_t face_elems = 6 * 5 * nt + 6 * nt;  // generous: n arrays sized like tau
    int nb = nblk((long)ni * nj);
    P->nblocks_cells = nb;
    size_t total = n_cell_fields * fe + face_elems + 8 + (size_t)nb + 64;
    if (cudaMalloc(&P->arena, total * sizeof(double)) != cudaSuccess) {
        *err = "cudaMalloc failed for the passes-path state";
        delete P;
        return nullptr;
    }
    cudaMemset(P->arena, 0, total * sizeof(double));
    double* q = P->arena;
    auto df = [&]() {
        DF f{q, H, (int)W};
        q += fe;
        return f;
    };
    PS& s = P->s;
    s.ni = ni;
    s.nj = nj;
    s.H = H;
    for (int k = 0; k < 5; ++k) s.U[k] = df();
    for (int k = 0; k < 5; ++k) s.Uf[k] = df();
    s.rho = df();
    s.p = df();
    s.t = df();
    s.vx = df();
    s.vy = df();
    s.e = df();
    s.hh = df();
    s.c = df();
    s.nut = df();
    for (int k = 0; k < 8; ++k) s.g[k] = df();
    s.mu = df();
    s.chi = df();
    s.fv1 = df();
    for (int k = 0; k < 5; ++k) s.Dx[k] = df();
    for (int k = 0; k < 5; ++k) s.Dy[k] = df();
    for (int k = 0; k < 5; ++k) s.fc[k] = df();
    for (int k = 0; k < 5; ++k) s.fv[k] = df();
    for (int k = 0; k < 5; ++k) s.fd[k] = df();
    s.src = df();
    s.localdt = df();
    s.sensor_i = df();
    s.sensor_j = df();
    s.spec_ratio = df();
    s.rho_prev = df();
    (void)nn;
    s.tflux = q; q += 5 * nt;
    s.nflux = q; q += 5 * nt;
    s.tdiff = q; q += 5 * nt;
    s.ndiff = q; q += 5 * nt;
    s.tdiss = q; q += 5 * nt;
    s.ndiss = q; q += 5 * nt;
    s.tlam = q; q += nt;
    s.nlam = q; q += nt;
    s.te2 = q; q += nt;
    s.te4 = q; q += nt;
    s.ne2 = q; q += nt;
    s.ne4 = q; q += nt;
    s.dt = q++;
    s.totaltime = q++;
    s.residual = q++;
    s.bad = reinterpret_cast<unsigned long long*>(q++);
    q += 4;
    s.partial = q;
    return P;
}

void passes_destroy(Passes* P) {
    if (!P) return;
    cudaFree(P->arena);
    delete P;
}

static void passes_boundary(Passes* P, const Geom& g, const PhysConst& c, cudaStream_t st) {
    const PS& s = P->s;
    JST_LAUNCH(k_bc_wall, nblk((long)s.H * s.nj), TB, 0, st, s);
    JST_LAUNCH(k_bc_far, nblk(s.nj), TB, 0, st, s, g, c);
    JST_LAUNCH(k_bc_periodic, nblk((long)s.ni * 2 * s.H), TB, 0, st, s);
}

void passes_init(Passes* P, const Geom& g, const PhysConst& c, cudaStream_t st) {
    const PS& s = P->s;
    JST_LAUNCH(k_init, nblk((long)s.ni * s.nj), TB, 0, st, s, c);
    passes_boundary(P, g, c, st);
}

void passes_set_uniform(Passes* P, const PhysConst& c, double rho, double vx, double vy, double p, double nut,
                        cudaStream_t st) {
    // PrimState::from_primitives (state.rs:222-237)
    double t = p / (c.r_gas * rho);
    double e = p / (rho * c.gm1) + 0.5 * (vx * vx + vy * vy);
    double h = e + p / rho;
    double cc = std::sqrt(c.rg * t);
    const PS& s = P->s;
    JST_LAUNCH(k_set_uniform, nblk((long)(s.ni + 2 * s.H) * (s.nj + 2 * s.H)), TB, 0, st, s, rho, p, t, vx, vy, e, h,
               cc, nut);
}

// timestep::compute; leaves the minimum in *s.dt and adds it to the total
// time when accumulate is set (solver.rs:110-111).
void passes_timestep(Passes* P, const Geom& g, const PhysConst& c, int accumulate, cudaStream_t st) {
    const PS& s = P->s;
    long n = (long)s.ni * s.nj;
    JST_LAUNCH(k_timestep, nblk(n), TB, 0, st, s, g, c.cfl);
    JST_LAUNCH(k_min_partial, nblk(n), TB, 0, st, s.localdt, s.ni, s.nj, s.partial);
    JST_LAUNCH(k_min_final, 1, 32, 0, st, s.partial, (int)nblk(n), s.dt, s.totaltime, accumulate);
}

void passes_kernel(Passes* P, const Geom& g, const PhysConst& c, const char* which, cudaStream_t st) {
    const PS& s = P->s;
    long n = (long)s.ni * s.nj, nt = (long)(s.ni + 1) * s.nj;
    std::string w(which);
    if (w == "boundary") {
        passes_boundary(P, g, c, st);
    } else if (w == "convection") {
        JST_LAUNCH(k_conv_faces, nblk(nt + n), TB, 0, st, s, g, c.gm1);
        JST_LAUNCH(k_circulation, nblk(n), TB, 0, st, s, s.tflux, s.nflux, 0);
    } else if (w == "gradient") {
        JST_LAUNCH(k_grad, nblk(n), TB, 0, st, s, g);
        JST_LAUNCH(k_grad_ghost, nblk(s.nj + s.ni), TB, 0, st, s);
    } else if (w == "viscous") {
        JST_LAUNCH(k_visc_cells, nblk(n + 2 * s.nj + 2 * s.ni), TB, 0, st, s, c);
        JST_LAUNCH(k_visc_faces, nblk(nt + n), TB, 0, st, s, g);
        JST_LAUNCH(k_circulation, nblk(n), TB, 0, st, s, s.tdiff, s.ndiff, 1);
    } else if (w == "dissipation") {
        JST_LAUNCH(k_diss_ratio, nblk(n), TB, 0, st, s, g);
        JST_LAUNCH(k_diss_lambda, nblk(nt + n), TB, 0, st, s, c.half_cfl);
        JST_LAUNCH(k_sensors, nblk((long)(s.ni + 4) * s.nj + (long)s.ni * (s.nj + 3)), TB, 0, st, s);
        JST_LAUNCH(k_diss_coef, nblk(nt + n), TB, 0, st, s, c.k2, c.k4);
        JST_LAUNCH(k_diss_faces, nblk(nt + n), TB, 0, st, s);
        JST_LAUNCH(k_diss_assemble, nblk(n), TB, 0, st, s);
    } else if (w == "source") {
        JST_LAUNCH(k_source, nblk(n), TB, 0, st, s, g, c);
    }
}

// Solver::residual_terms (solver.rs:86-94).
void passes_residual_terms(Passes* P, const Geom& g, const PhysConst& c, cudaStream_t st) {
    for (const char* k : {"boundary", "convection", "gradient", "viscous", "dissipation", "source"})
        passes_kernel(P, g, c, k, st);
}

// One RK stage after residual_terms: update + unpack.  Returns nothing; the
// caller reads *s.bad.
void passes_update_unpack(Passes* P, const Geom& g, const PhysConst& c, double alpha, int local, cudaStream_t st) {
    const PS& s = P->s;
    long n = (long)s.ni * s.nj;
    JST_LAUNCH(k_update, nblk(n), TB, 0, st, s, g, alpha, local);
    JST_LAUNCH(k_unpack, nblk(n), TB, 0, st, s, c.gm1, c.r_gas, c.rg);
}

void passes_unpack(Passes* P, const PhysConst& c, cudaStream_t st) {
    const PS& s = P->s;
    JST_LAUNCH(k_unpack, nblk((long)s.ni * s.nj), TB, 0, st, s, c.gm1, c.r_gas, c.rg);
}

void passes_snapshot(Passes* P, cudaStream_t st) {
    const PS& s = P->s;
    JST_LAUNCH(k_copy_fields, nblk((long)(s.ni + 2 * s.H) * (s.nj + 2 * s.H)), TB, 0, st, s);
}

void passes_residual(Passes* P, cudaStream_t st) {
    const PS& s = P->s;
    int nb = nblk((long)s.ni * s.nj);
    JST_LAUNCH(k_res_partial, nb, TB, 0, st, s);
    JST_LAUNCH(k_res_final, 1, 32, 0, st, s, nb);
}

void passes_wall_force(Passes* P, const Geom& g, double* d_out, cudaStream_t st) {
    JST_LAUNCH(k_wall_force, 1, 32, 0, st, P->s, g, d_out);
}

unsigned long long* passes_bad_ptr(Passes* P) { return P->s.bad; }
double* passes_dt_ptr(Passes* P) { return P->s.dt; }
double* passes_totaltime_ptr(Passes* P) { return P->s.totaltime; }
double* passes_residual_ptr(Passes* P) { return P->s.residual; }

// Device pointer + stride of a halo-indexed field (interior copy is done by
// the host with cudaMemcpy2D).
bool passes_field(Passes* P, int id, const double** base, int* stride, int* halo) {
    const PS& s = P->s;
    const DF* f = nullptr;
    switch (id) {
        case 0: f = &s.rho; break;
        case 1: f = &s.p; break;
        case 2: f = &s.t; break;
        case 3: f = &s.vx; break;
        case 4: f = &s.vy; break;
        case 5: f = &s.e; break;
        case 6: f = &s.hh; break;
        case 7: f = &s.c; break;
        case 8: f = &s.nut; break;
        case 9: case 10: case 11: case 12: case 13: f = &s.U[id - 9]; break;
        case 14: case 15: case 16: case 17: case 18: f = &s.fc[id - 14]; break;
        case 19: case 20: case 21: case 22: case 23: f = &s.fv[id - 19]; break;
        case 24: case 25: case 26: case 27: case 28: f = &s.fd[id - 24]; break;
        case 29: f = &s.src; break;
        case 30: case 31: case 32: case 33: case 34: case 35: case 36: case 37: f = &s.g[id - 30]; break;
        case 38: f = &s.chi; break;
        case 39: f = &s.fv1; break;
        case 40: f = &s.localdt; break;
        default: return false;
    }
    *base = f->p;
    *stride = f->stride;
    *halo = f->h;
    return true;
}

}  // namespace jst
