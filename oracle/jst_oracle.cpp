// ORACLE — test infrastructure only, never the product.
//
// A CPU, FP64 restatement of PurineCFD's jst-rs solver loop (the Rust crate
// `jst`), written to be the checker for the CUDA path in purinecfd_b200/.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// this library.  It follows the reference expression by expression: the same
// evaluation order (left-associative sums, no reassociation), no FMA
// contraction (build with -ffp-contract=off), the platform libm for exp, cbrt,
// pow and hypot (what Rust's f64 methods call), and `powi` expanded by binary
// squaring exactly as LLVM lowers it (x^3 = x*(x*x), x^6 = x2*(x2*x2)).
//
// Parity pin: this restatement is checked against the reference's own golden
// data (tests/golden/cyl_10x12.json, cyl_17x40.json — exported by the
// reference's jst-py/tools/dump_golden.py) at the tolerances of the reference's
// jst-rs/tests/golden.rs:11-21.
//
// Citations are file:line within the reference's jst-rs/ crate.
//
// Additions that the reference does not have (marked "EXT"): an optional
// free-stream nu-tilde ratio (the reference hard-codes 0.1, config.rs:196),
// an opt-in local time stepping mode, and a wall-force (CL/CD) integrator.
// With their defaults the restatement is the reference's algorithm unchanged.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- config ----
// config.rs:11-111 (inputs) and config.rs:115-145, 173-206 (derived constants).
struct Config {
    double gamma, r_gas, t_ref, t_suth, mu0;
    double aoa, mach, cfl;
    int halo;
    double t_inf, p_inf;
    long iteration;
    double targetres;
    double Cv1, Pr, Prt, sigma, Cb1, Cb2, Ct3, Ct4, Cw2, Cw3, fv3, kappa, rmax;
    double k2, k4;
    double nut_ratio;  // EXT: 0.1 in the reference (config.rs:196)
    int local_dt;      // EXT: 0 = global minimum step (solver.rs:110-116)

    double cv, cp, cw1, cv1_cubed, c_inf, u_inf, v_inf, rho_inf, mu_inf, nut_inf;
    bool supersonic;
    double suth_num, inv_t_ref, inv_pr, inv_prt, inv_kappa2, cw3_6, one_plus_cw3_6;
};

// x.powi(n) for the constant exponents the reference uses, lowered the way
// LLVM expands powi with a constant exponent (binary decomposition).
inline double powi2(double x) { return x * x; }
inline double powi3(double x) { return x * (x * x); }
inline double powi6(double x) {
    double x2 = x * x;
    double x4 = x2 * x2;
    return x2 * x4;
}

// config.rs:153-156
double sutherland(double mu0, double t, double t_ref, double t_suth) {
    double r = t / t_ref;
    return mu0 * (r * std::sqrt(r)) * (t_ref + t_suth) / (t + t_suth);
}

// config.rs:173-206
void finish(Config& c) {
    double cv = c.r_gas / (c.gamma - 1.0);
    double c_inf = std::sqrt(c.gamma * c.r_gas * c.t_inf);
    double aoa = c.aoa * (M_PI / 180.0);  // f64::to_radians
    double rho_inf = c.p_inf / (c.r_gas * c.t_inf);
    double mu_inf = sutherland(c.mu0, c.t_inf, c.t_ref, c.t_suth);
    double u_inf = c_inf * c.mach * std::cos(aoa);
    double v_inf = c_inf * c.mach * std::sin(aoa);
    c.cv = cv;
    c.cp = c.gamma * cv;
    c.cw1 = c.Cb1 / (c.kappa * c.kappa) + (1.0 + c.Cb2) * c.sigma;
    c.cv1_cubed = powi3(c.Cv1);
    c.c_inf = c_inf;
    c.u_inf = u_inf;
    c.v_inf = v_inf;
    c.rho_inf = rho_inf;
    c.mu_inf = mu_inf;
    c.nut_inf = c.nut_ratio * mu_inf / rho_inf;
    c.supersonic = std::hypot(u_inf, v_inf) >= c_inf;
    c.suth_num = c.mu0 * (c.t_ref + c.t_suth);
    c.inv_t_ref = 1.0 / c.t_ref;
    c.inv_pr = 1.0 / c.Pr;
    c.inv_prt = 1.0 / c.Prt;
    c.inv_kappa2 = 1.0 / (c.kappa * c.kappa);
    c.cw3_6 = powi6(c.Cw3);
    c.one_plus_cw3_6 = 1.0 + powi6(c.Cw3);
}

// config.rs:210-213
inline double mu_of(const Config& c, double t) {
    double r = t * c.inv_t_ref;
    return r * std::sqrt(r) * c.suth_num / (t + c.t_suth);
}

const double RK_ALPHA[5] = {0.25, 1.0 / 6.0, 0.375, 0.5, 1.0};  // config.rs:217

// ----------------------------------------------------------------- field ----
// Halo-indexed row-major storage, i slow / j fast (field.rs:139-192).
struct Field {
    std::vector<double> d;
    int ni = 0, nj = 0, h = 0, stride = 0;
    void init(int ni_, int nj_, int h_) {
        ni = ni_;
        nj = nj_;
        h = h_;
        stride = nj + 2 * h;
        d.assign((size_t)(ni + 2 * h) * stride, 0.0);
    }
    inline size_t off(long i, long j) const { return (size_t)(i + h) * stride + (size_t)(j + h); }
    inline double& operator()(long i, long j) { return d[off(i, j)]; }
    inline double operator()(long i, long j) const { return d[off(i, j)]; }
};

struct V5 {
    double v[5];
};

struct Face {
    double nx, ny, mx, my;
};

// ------------------------------------------------------------------ solver --
struct Solver {
    Config cfg;
    int ni, nj, H;
    std::vector<double> nodes;  // n_rings x n_theta, (x,y) interleaved
    int n_rings, n_theta;

    // geometry.rs:45-63
    Field vol, cx, cy, wall_dist, inv_vol, inv_d2;
    std::vector<Face> tau, nrm;  // (NI+1)xNJ and NIxNJ, no halo

    // state.rs:68-110
    Field U[5], Uf[5];
    Field rho, p, t, vx, vy, e, hh, c, nut;
    Field g[8];  // dudx dudy dvdx dvdy dtdx dtdy dnutdx dnutdy
    Field mu, chi, fv1;
    Field Dx[5], Dy[5];
    Field fc[5], fv[5], fd[5], src, localdt;
    // state.rs:266-317 (face work arrays; flux/diff/dissipation per tau/n face)
    std::vector<double> tflux, nflux, tdiff, ndiff, tdiss, ndiss;  // [face*5+k]
    std::vector<double> tlam, nlam, te2, te4, ne2, ne4;
    Field sensor_i, sensor_j, spec_ratio;

    Field rho_prev;
    double totaltime = 0.0;
    long step = 0;

    // Non-physical report of the last failing unpack (state.rs:242-257).
    long bad_i = 0, bad_j = 0;
    double bad_rho = 0.0, bad_p = 0.0;

    inline const Face& T(long i, long j) const { return tau[(size_t)i * nj + j]; }
    inline const Face& N(long i, long j) const { return nrm[(size_t)i * nj + j]; }
    inline double nodex(long r, long th) const { return nodes[2 * ((size_t)r * n_theta + (th % n_theta))]; }
    inline double nodey(long r, long th) const { return nodes[2 * ((size_t)r * n_theta + (th % n_theta)) + 1]; }
    inline long jp1(long j) const { return j + 1 < nj ? j + 1 : 0; }
};

// ------------------------------------------------------------- geometry ----
// geometry.rs:109-145
void build_cells(Solver& s) {
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double ax = s.nodex(i, j), ay = s.nodey(i, j);
            double bx = s.nodex(i + 1, j), by = s.nodey(i + 1, j);
            double cx = s.nodex(i + 1, j + 1), cy = s.nodey(i + 1, j + 1);
            double dx = s.nodex(i, j + 1), dy = s.nodey(i, j + 1);
            double d1x = cx - ax, d1y = cy - ay;
            double d2x = bx - dx, d2y = by - dy;
            double vol = 0.5 * std::fabs(d1x * d2y - d1y * d2x);
            double cr0 = ax * by - bx * ay;
            double cr1 = bx * cy - cx * by;
            double cr2 = cx * dy - dx * cy;
            double cr3 = dx * ay - ax * dy;
            double sgn = 0.5 * (cr0 + cr1 + cr2 + cr3);
            double sx = (ax + bx) * cr0 + (bx + cx) * cr1 + (cx + dx) * cr2 + (dx + ax) * cr3;
            double sy = (ay + by) * cr0 + (by + cy) * cr1 + (cy + dy) * cr2 + (dy + ay) * cr3;
            s.vol(i, j) = vol;
            if (std::fabs(sgn) > 1e-30) {
                s.cx(i, j) = sx / (6.0 * sgn);
                s.cy(i, j) = sy / (6.0 * sgn);
            }
        }
}

// geometry.rs:148-185
void build_faces(Solver& s) {
    s.tau.assign((size_t)(s.ni + 1) * s.nj, Face{0, 0, 0, 0});
    s.nrm.assign((size_t)s.ni * s.nj, Face{0, 0, 0, 0});
    for (long i = 0; i <= s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double ax = s.nodex(i, j), ay = s.nodey(i, j);
            double bx = s.nodex(i, j + 1), by = s.nodey(i, j + 1);
            double dx = bx - ax, dy = by - ay;
            s.tau[(size_t)i * s.nj + j] = Face{dy, -dx, 0.5 * (ax + bx), 0.5 * (ay + by)};
        }
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double ax = s.nodex(i, j), ay = s.nodey(i, j);
            double bx = s.nodex(i + 1, j), by = s.nodey(i + 1, j);
            double dx = bx - ax, dy = by - ay;
            s.nrm[(size_t)i * s.nj + j] = Face{-dy, dx, 0.5 * (ax + bx), 0.5 * (ay + by)};
        }
}

// geometry.rs:192-216
void build_wall_distance(Solver& s) {
    long nj = s.nj;
    long window = std::min(std::max(15L, nj / 5), nj / 2);
    std::vector<double> wx(nj), wy(nj);
    for (long j = 0; j < nj; ++j) {
        wx[j] = s.T(0, j).mx;
        wy[j] = s.T(0, j).my;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < nj; ++j) {
            double px = s.cx(i, j), py = s.cy(i, j);
            double best = std::numeric_limits<double>::infinity();
            for (long dk = -window; dk <= window; ++dk) {
                long k = ((j + dk) % nj + nj) % nj;
                double d = std::sqrt(powi2(px - wx[k]) + powi2(py - wy[k]));
                if (d < best) best = d;
            }
            s.wall_dist(i, j) = best;
        }
}

// geometry.rs:76-103
void build_geometry(Solver& s) {
    int H = s.H;
    for (Field* f : {&s.vol, &s.cx, &s.cy, &s.wall_dist, &s.inv_vol, &s.inv_d2}) f->init(s.ni, s.nj, H);
    build_cells(s);
    build_faces(s);
    build_wall_distance(s);
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            s.inv_vol(i, j) = 1.0 / s.vol(i, j);
            double d = s.wall_dist(i, j);
            s.inv_d2(i, j) = 1.0 / (d * d);
        }
}

// ------------------------------------------------------------------ state ---
struct Prim {
    double rho, p, t, vx, vy, e, h, c, nut;
};

// state.rs:222-237
Prim from_primitives(const Config& c, double rho, double vx, double vy, double p, double nut) {
    double gamma = c.gamma;
    double t = p / (c.r_gas * rho);
    double e = p / (rho * (gamma - 1.0)) + 0.5 * (vx * vx + vy * vy);
    Prim s;
    s.rho = rho;
    s.p = p;
    s.t = t;
    s.vx = vx;
    s.vy = vy;
    s.e = e;
    s.h = e + p / rho;
    s.c = std::sqrt(gamma * c.r_gas * t);
    s.nut = nut;
    return s;
}

// state.rs:143-156
inline void pack(Solver& s, long i, long j) {
    double r = s.rho(i, j);
    s.U[0](i, j) = r;
    s.U[1](i, j) = r * s.vx(i, j);
    s.U[2](i, j) = r * s.vy(i, j);
    s.U[3](i, j) = r * s.e(i, j);
    s.U[4](i, j) = r * s.nut(i, j);
}

// state.rs:160-171
inline void write_state(Solver& s, long i, long j, const Prim& q) {
    s.rho(i, j) = q.rho;
    s.p(i, j) = q.p;
    s.t(i, j) = q.t;
    s.vx(i, j) = q.vx;
    s.vy(i, j) = q.vy;
    s.e(i, j) = q.e;
    s.hh(i, j) = q.h;
    s.c(i, j) = q.c;
    s.nut(i, j) = q.nut;
    pack(s, i, j);
}

// state.rs:174-190
void initialize(Solver& s) {
    const Config& c = s.cfg;
    Prim q = from_primitives(c, c.p_inf / (c.r_gas * c.t_inf), c.u_inf, c.v_inf, c.p_inf, c.nut_inf);
    double mu = mu_of(c, c.t_inf);
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            write_state(s, i, j, q);
            s.mu(i, j) = mu;
            s.chi(i, j) = 0.0;
            s.fv1(i, j) = 0.0;
        }
}

// state.rs:198-203 — every addressable cell, halo and corners included.
void set_uniform(Solver& s, double rho, double vx, double vy, double p, double nut) {
    Prim q = from_primitives(s.cfg, rho, vx, vy, p, nut);
    for (long i = -s.H; i < s.ni + s.H; ++i)
        for (long j = -s.H; j < s.nj + s.H; ++j) write_state(s, i, j, q);
}

// --------------------------------------------------------------- boundary ---
// boundary.rs:30-51
void wall_mirror(Solver& s) {
    for (long k = 0; k < s.H; ++k) {
        long g = -1 - k;
        for (long j = 0; j < s.nj; ++j) {
            s.rho(g, j) = s.rho(k, j);
            s.p(g, j) = s.p(k, j);
            s.t(g, j) = s.t(k, j);
            s.e(g, j) = s.e(k, j);
            s.hh(g, j) = s.hh(k, j);
            s.c(g, j) = s.c(k, j);
            s.vx(g, j) = -s.vx(k, j);
            s.vy(g, j) = -s.vy(k, j);
            s.nut(g, j) = -s.nut(k, j);
            pack(s, g, j);
        }
    }
}

// boundary.rs:54-72
void periodic_seam(Solver& s) {
    long nj = s.nj;
    for (long i = 0; i < s.ni; ++i)
        for (long k = 1; k <= s.H; ++k) {
            long pairs[2][2] = {{-k, nj - k}, {nj - 1 + k, k - 1}};
            for (auto& pr : pairs) {
                long g = pr[0], src = pr[1];
                s.rho(i, g) = s.rho(i, src);
                s.p(i, g) = s.p(i, src);
                s.t(i, g) = s.t(i, src);
                s.e(i, g) = s.e(i, src);
                s.hh(i, g) = s.hh(i, src);
                s.c(i, g) = s.c(i, src);
                s.vx(i, g) = s.vx(i, src);
                s.vy(i, g) = s.vy(i, src);
                s.nut(i, g) = s.nut(i, src);
                pack(s, i, g);
            }
        }
}

// boundary.rs:158-185
double extrapolate_nut(const Solver& s, long j) {
    const double FLOOR = 1e-10;
    long ni = s.ni;
    const Face& f = s.T(ni, j);
    double dist[3], nu[3];
    for (int k = 0; k < 3; ++k) {
        long i = ni - 1 - k;
        dist[k] = std::hypot(s.cx(i, j) - f.mx, s.cy(i, j) - f.my);
        nu[k] = s.nut(i, j);
    }
    double l1 = dist[0], l2 = dist[1], l3 = dist[2];
    double d12 = l1 - l2, d13 = l1 - l3, d23 = l2 - l3;
    if (std::fabs(d12) < 1e-14 || std::fabs(d13) < 1e-14 || std::fabs(d23) < 1e-14)
        return std::fmax(nu[0], FLOOR);
    double v = l2 * l3 / (d12 * d13) * nu[0] + l1 * l3 / (-d12 * d23) * nu[1] + l1 * l2 / (d23 * -d13) * nu[2];
    return v > FLOOR ? v : FLOOR;
}

// boundary.rs:112-155
Prim riemann_face(const Solver& s, long j, bool* inflow_out) {
    const Config& c = s.cfg;
    long ni = s.ni;
    const Face& f = s.T(ni, j);
    double len = std::hypot(f.nx, f.ny);
    double nx = f.nx, ny = f.ny;
    double gamma = c.gamma;
    double vn_inf = (c.u_inf * nx + c.v_inf * ny) / len;
    double vt_inf = (c.u_inf * ny - c.v_inf * nx) / len;
    double ui = s.vx(ni - 1, j), vi = s.vy(ni - 1, j);
    double vn_in = (ui * nx + vi * ny) / len;
    double vt_in = (ui * ny - vi * nx) / len;
    double c_face, vn_face, vt_face;
    bool inflow;
    if (!c.supersonic) {
        double r_in = vn_in + 2.0 * s.c(ni - 1, j) / (gamma - 1.0);
        double r_inf = vn_inf - 2.0 * c.c_inf / (gamma - 1.0);
        double vn = 0.5 * (r_in + r_inf);
        double cf = (gamma - 1.0) / 4.0 * (r_in - r_inf);
        inflow = vn <= 0.0;
        c_face = cf;
        vn_face = vn;
        vt_face = inflow ? vt_inf : vt_in;
    } else if (vn_inf <= 0.0) {
        c_face = c.c_inf;
        vn_face = vn_inf;
        vt_face = vt_inf;
        inflow = true;
    } else {
        c_face = s.c(ni - 1, j);
        vn_face = vn_in;
        vt_face = vt_in;
        inflow = false;
    }
    double t = c_face * c_face / (c.r_gas * gamma);
    double rho = c.rho_inf * std::pow(t / c.t_inf, 1.0 / (gamma - 1.0));
    double p = rho * c.r_gas * t;
    double vx = (vt_face * ny + vn_face * nx) / len;
    double vy = (-vt_face * nx + vn_face * ny) / len;
    double e = p / (rho * (gamma - 1.0)) + 0.5 * (vx * vx + vy * vy);
    Prim q;
    q.rho = rho;
    q.p = p;
    q.t = t;
    q.vx = vx;
    q.vy = vy;
    q.e = e;
    q.nut = inflow ? c.nut_inf : extrapolate_nut(s, j);
    q.h = 0.0;
    q.c = 0.0;
    if (inflow_out) *inflow_out = inflow;
    return q;
}

// boundary.rs:87-109
void far_field_riemann(Solver& s) {
    const Config& c = s.cfg;
    for (long j = 0; j < s.nj; ++j) {
        Prim q = riemann_face(s, j, nullptr);
        double cc = std::sqrt(c.gamma * c.r_gas * q.t);
        double h = q.e + q.p / q.rho;
        for (long k = 0; k < s.H; ++k) {
            long g = s.ni + k;
            s.rho(g, j) = q.rho;
            s.p(g, j) = q.p;
            s.t(g, j) = q.t;
            s.e(g, j) = q.e;
            s.hh(g, j) = h;
            s.c(g, j) = cc;
            s.vx(g, j) = q.vx;
            s.vy(g, j) = q.vy;
            s.nut(g, j) = q.nut;
            pack(s, g, j);
        }
    }
}

// boundary.rs:23-27
void boundary_apply(Solver& s) {
    wall_mirror(s);
    far_field_riemann(s);
    periodic_seam(s);
}

// --------------------------------------------------------------- timestep ---
// timestep.rs:24-57
double timestep_compute(Solver& s) {
    long nj = s.nj;
    double cfl = s.cfg.cfl;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < nj; ++j) {
            long jp = j + 1 < nj ? j + 1 : 0;
            const Face &f0 = s.T(i, j), &f1 = s.T(i + 1, j);
            const Face &g0 = s.N(i, j), &g1 = s.N(i, jp);
            double a = 0.5 * (f0.nx + f1.nx);
            double b = 0.5 * (f0.ny + f1.ny);
            double cc = 0.5 * (g0.nx + g1.nx);
            double dd = 0.5 * (g0.ny + g1.ny);
            double u = s.vx(i, j), v = s.vy(i, j);
            double conv = std::fabs(u * a + v * b) + std::fabs(u * cc + v * dd);
            double acou = s.c(i, j) * (std::sqrt(a * a + b * b) + std::sqrt(cc * cc + dd * dd));
            s.localdt(i, j) = cfl * s.vol(i, j) / (conv + acou);
        }
    double m = std::numeric_limits<double>::infinity();
#pragma omp parallel for schedule(static) reduction(min : m)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < nj; ++j) m = std::fmin(m, s.localdt(i, j));
    return m;
}

// ------------------------------------------------------------- convection ---
// convection.rs:25-40
inline void euler_flux(const double fu[5], const Face& f, double gamma, double out[5]) {
    double rho = fu[0];
    double inv_rho = 1.0 / rho;
    double u = fu[1] * inv_rho;
    double v = fu[2] * inv_rho;
    double rho_e = fu[3];
    double p = (gamma - 1.0) * (rho_e - rho * (u * u + v * v) * 0.5);
    double vn = f.nx * u + f.ny * v;
    out[0] = rho * vn;
    out[1] = fu[1] * vn + p * f.nx;
    out[2] = fu[2] * vn + p * f.ny;
    out[3] = (rho_e + p) * vn;
    out[4] = fu[4] * vn;
}

// convection.rs:46-86
void convection_compute(Solver& s) {
    double gamma = s.cfg.gamma;
    long nj = s.nj;
#pragma omp parallel for schedule(static)
    for (long i = 0; i <= s.ni; ++i)
        for (long j = 0; j < nj; ++j) {
            double fu[5];
            for (int k = 0; k < 5; ++k) fu[k] = 0.5 * (s.U[k](i - 1, j) + s.U[k](i, j));
            euler_flux(fu, s.T(i, j), gamma, &s.tflux[((size_t)i * nj + j) * 5]);
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < nj; ++j) {
            double fu[5];
            for (int k = 0; k < 5; ++k) fu[k] = 0.5 * (s.U[k](i, j - 1) + s.U[k](i, j));
            euler_flux(fu, s.N(i, j), gamma, &s.nflux[((size_t)i * nj + j) * 5]);
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < nj; ++j) {
            long jp = s.jp1(j);
            for (int k = 0; k < 5; ++k)
                s.fc[k](i, j) = s.tflux[((size_t)(i + 1) * nj + j) * 5 + k] - s.tflux[((size_t)i * nj + j) * 5 + k] +
                                s.nflux[((size_t)i * nj + jp) * 5 + k] - s.nflux[((size_t)i * nj + j) * 5 + k];
        }
}

// --------------------------------------------------------------- gradient ---
// gradient.rs:22-35 (one scalar's Green-Gauss sum)
inline void gg(const Field& src, long i, long j, const Face& up, const Face& dn, const Face& lf, const Face& rt,
               double inv_v, double* gx, double* gy) {
    double c = src(i, j);
    double f_up = 0.5 * (c + src(i + 1, j));
    double f_dn = 0.5 * (c + src(i - 1, j));
    double f_lf = 0.5 * (c + src(i, j - 1));
    double f_rt = 0.5 * (c + src(i, j + 1));
    *gx = (f_up * up.nx - f_dn * dn.nx + f_rt * rt.nx - f_lf * lf.nx) * inv_v;
    *gy = (f_up * up.ny - f_dn * dn.ny + f_rt * rt.ny - f_lf * lf.ny) * inv_v;
}

// gradient.rs:38-102
void gradient_compute(Solver& s) {
    long nj = s.nj, ni = s.ni;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            const Face& up = s.T(i + 1, j);
            const Face& dn = s.T(i, j);
            const Face& lf = s.N(i, j);
            const Face& rt = s.N(i, s.jp1(j));
            double iv = s.inv_vol(i, j);
            gg(s.vx, i, j, up, dn, lf, rt, iv, &s.g[0](i, j), &s.g[1](i, j));
            gg(s.vy, i, j, up, dn, lf, rt, iv, &s.g[2](i, j), &s.g[3](i, j));
            gg(s.t, i, j, up, dn, lf, rt, iv, &s.g[4](i, j), &s.g[5](i, j));
            gg(s.nut, i, j, up, dn, lf, rt, iv, &s.g[6](i, j), &s.g[7](i, j));
        }
    // gradient.rs:87-102
    for (long j = 0; j < nj; ++j) {
        for (int k = 0; k < 8; ++k) s.g[k](-1, j) = s.g[k](0, j);
        s.g[4](-1, j) = 0.0;
        s.g[5](-1, j) = 0.0;
        for (int k = 0; k < 8; ++k) s.g[k](ni, j) = 0.0;
    }
    for (long i = 0; i < ni; ++i)
        for (int k = 0; k < 8; ++k) {
            s.g[k](i, -1) = s.g[k](i, nj - 1);
            s.g[k](i, nj) = s.g[k](i, 0);
        }
}

// ---------------------------------------------------------------- viscous ---
// viscous.rs:37-71 evaluated at one cell
void diffusion_tensor(Solver& s, long i, long j) {
    const Config& c = s.cfg;
    double t = s.t(i, j), rho_nu = s.U[4](i, j), vx = s.vx(i, j), vy = s.vy(i, j);
    double dudx = s.g[0](i, j), dudy = s.g[1](i, j), dvdx = s.g[2](i, j), dvdy = s.g[3](i, j);
    double dtdx = s.g[4](i, j), dtdy = s.g[5](i, j), dnx = s.g[6](i, j), dny = s.g[7](i, j);
    double mu = mu_of(c, t);
    double chi = rho_nu / mu;
    double c3 = chi * chi * chi;  // viscous.rs:27-30
    double f1 = c3 / (c3 + c.cv1_cubed);
    double mu_t = rho_nu * f1;
    double mu_eff = mu + mu_t;
    double lam_eff = mu * c.inv_pr + mu_t * c.inv_prt;
    double txx = mu_eff * (4.0 / 3.0 * dudx - 2.0 / 3.0 * dvdy);
    double tyy = mu_eff * (4.0 / 3.0 * dvdy - 2.0 / 3.0 * dudx);
    double txy = mu_eff * (dudy + dvdx);
    double qx = lam_eff * c.cp * dtdx;
    double qy = lam_eff * c.cp * dtdy;
    double nu_diff = c.sigma * (mu + rho_nu);
    s.mu(i, j) = mu;
    s.chi(i, j) = chi;
    s.fv1(i, j) = f1;
    s.Dx[0](i, j) = 0.0;
    s.Dx[1](i, j) = txx;
    s.Dx[2](i, j) = txy;
    s.Dx[3](i, j) = vx * txx + vy * txy + qx;
    s.Dx[4](i, j) = nu_diff * dnx;
    s.Dy[0](i, j) = 0.0;
    s.Dy[1](i, j) = txy;
    s.Dy[2](i, j) = tyy;
    s.Dy[3](i, j) = vx * txy + vy * tyy + qy;
    s.Dy[4](i, j) = nu_diff * dny;
}

// viscous.rs:152-164 (cell_tensors 74-125, face_diffusion 128-149)
void viscous_compute(Solver& s) {
    long ni = s.ni, nj = s.nj;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) diffusion_tensor(s, i, j);
    for (long j = 0; j < nj; ++j) {
        diffusion_tensor(s, -1, j);
        diffusion_tensor(s, ni, j);
    }
    for (long i = 0; i < ni; ++i) {
        diffusion_tensor(s, i, -1);
        diffusion_tensor(s, i, nj);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i <= ni; ++i)
        for (long j = 0; j < nj; ++j) {
            const Face& f = s.T(i, j);
            double hx = 0.5 * f.nx, hy = 0.5 * f.ny;
            for (int k = 0; k < 5; ++k)
                s.tdiff[((size_t)i * nj + j) * 5 + k] =
                    (s.Dx[k](i - 1, j) + s.Dx[k](i, j)) * hx + (s.Dy[k](i - 1, j) + s.Dy[k](i, j)) * hy;
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            const Face& f = s.N(i, j);
            double hx = 0.5 * f.nx, hy = 0.5 * f.ny;
            for (int k = 0; k < 5; ++k)
                s.ndiff[((size_t)i * nj + j) * 5 + k] =
                    (s.Dx[k](i, j - 1) + s.Dx[k](i, j)) * hx + (s.Dy[k](i, j - 1) + s.Dy[k](i, j)) * hy;
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            long jp = s.jp1(j);
            for (int k = 0; k < 5; ++k)
                s.fv[k](i, j) = s.tdiff[((size_t)(i + 1) * nj + j) * 5 + k] - s.tdiff[((size_t)i * nj + j) * 5 + k] +
                                s.ndiff[((size_t)i * nj + jp) * 5 + k] - s.ndiff[((size_t)i * nj + j) * 5 + k];
        }
}

// ------------------------------------------------------------ dissipation ---
// dissipation.rs:29-31
inline double pressure_sensor(double pm, double p0, double pp) {
    return std::fabs((pm - 2.0 * p0 + pp) / (pm + 2.0 * p0 + pp));
}

// dissipation.rs:188-194 (spectral_radii 44-70, sensors 73-90, coefficients
// 93-126, face_dissipation 129-166, assemble 176-185)
void dissipation_compute(Solver& s) {
    long ni = s.ni, nj = s.nj;
    double cfl = s.cfg.cfl, k2 = s.cfg.k2, k4 = s.cfg.k4;
    // spectral_radii 44-70
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) s.spec_ratio(i, j) = s.vol(i, j) / s.localdt(i, j);
#pragma omp parallel for schedule(static)
    for (long i = 0; i <= ni; ++i) {
        long a = std::min(std::max(i, 0L), ni - 1), b = std::min(std::max(i - 1, 0L), ni - 1);
        for (long j = 0; j < nj; ++j) s.tlam[(size_t)i * nj + j] = 0.5 * cfl * (s.spec_ratio(a, j) + s.spec_ratio(b, j));
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            long jm = j > 0 ? j - 1 : nj - 1;
            s.nlam[(size_t)i * nj + j] = 0.5 * cfl * (s.spec_ratio(i, j) + s.spec_ratio(i, jm));
        }
    // sensors 73-90
    for (long i = -2; i <= ni + 1; ++i)
        for (long j = 0; j < nj; ++j) s.sensor_i(i, j) = pressure_sensor(s.p(i - 1, j), s.p(i, j), s.p(i + 1, j));
    for (long i = 0; i < ni; ++i)
        for (long j = -2; j <= nj; ++j) s.sensor_j(i, j) = pressure_sensor(s.p(i, j - 1), s.p(i, j), s.p(i, j + 1));
    // coefficients 93-126 (adaptive_coefficients 35-38)
#pragma omp parallel for schedule(static)
    for (long i = 0; i <= ni; ++i)
        for (long j = 0; j < nj; ++j) {
            double m = std::fmax(std::fmax(std::fmax(s.sensor_i(i - 2, j), s.sensor_i(i - 1, j)), s.sensor_i(i, j)),
                                 s.sensor_i(i + 1, j));
            double e2 = k2 * m;
            s.te2[(size_t)i * nj + j] = e2;
            s.te4[(size_t)i * nj + j] = std::fmax(k4 - e2, 0.0);
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            double m = std::fmax(std::fmax(std::fmax(s.sensor_j(i, j - 2), s.sensor_j(i, j - 1)), s.sensor_j(i, j)),
                                 s.sensor_j(i, j + 1));
            double e2 = k2 * m;
            s.ne2[(size_t)i * nj + j] = e2;
            s.ne4[(size_t)i * nj + j] = std::fmax(k4 - e2, 0.0);
        }
    // face_dissipation 129-166
#pragma omp parallel for schedule(static)
    for (long i = 0; i <= ni; ++i)
        for (long j = 0; j < nj; ++j) {
            size_t f = (size_t)i * nj + j;
            for (int k = 0; k < 5; ++k) {
                const Field& u = s.U[k];
                double d1 = u(i, j) - u(i - 1, j);
                double d3 = u(i + 1, j) - 3.0 * u(i, j) + 3.0 * u(i - 1, j) - u(i - 2, j);
                s.tdiss[f * 5 + k] = s.tlam[f] * (d1 * s.te2[f] - d3 * s.te4[f]);
            }
        }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            size_t f = (size_t)i * nj + j;
            for (int k = 0; k < 5; ++k) {
                const Field& u = s.U[k];
                double d1 = u(i, j) - u(i, j - 1);
                double d3 = u(i, j + 1) - 3.0 * u(i, j) + 3.0 * u(i, j - 1) - u(i, j - 2);
                s.ndiss[f * 5 + k] = s.nlam[f] * (d1 * s.ne2[f] - d3 * s.ne4[f]);
            }
        }
    // assemble 176-185
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ni; ++i)
        for (long j = 0; j < nj; ++j) {
            long jp = s.jp1(j);
            for (int k = 0; k < 5; ++k)
                s.fd[k](i, j) = s.tdiss[((size_t)(i + 1) * nj + j) * 5 + k] + s.ndiss[((size_t)i * nj + jp) * 5 + k] -
                                s.tdiss[((size_t)i * nj + j) * 5 + k] - s.ndiss[((size_t)i * nj + j) * 5 + k];
        }
}

// ----------------------------------------------------------------- source ---
// source.rs:30-33
inline double fw_of(double r, double cw2, double cw3_6, double one_plus_cw3_6) {
    double g = r + cw2 * (powi6(r) - r);
    return g * std::cbrt(std::sqrt(one_plus_cw3_6 / (powi6(g) + cw3_6)));
}

// source.rs:45-88
void source_compute(Solver& s) {
    const Config& c = s.cfg;
    double cb1_over_kappa2 = c.Cb1 * c.inv_kappa2;
    double cb2_sigma = c.Cb2 * c.sigma;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double rho = s.U[0](i, j);
            double rho_nu = s.U[4](i, j);
            double nu_tilde = rho_nu / rho;
            double inv_dist2 = s.inv_d2(i, j);
            double inv_kd2 = inv_dist2 * c.inv_kappa2;
            double chi = s.chi(i, j), f1 = s.fv1(i, j);
            double ft2 = c.Ct3 * std::exp(-c.Ct4 * chi * chi);
            double fv2 = 1.0 - chi / (1.0 + chi * f1);
            double sv = c.fv3 * std::fabs(s.g[2](i, j) - s.g[1](i, j));
            double s_tilde = std::fmax(sv + nu_tilde * inv_kd2 * fv2, 1e-10);
            double prod = c.Cb1 * (1.0 - ft2) * s_tilde * rho_nu;
            double r = std::fmin(nu_tilde / s_tilde * inv_kd2, c.rmax);
            double destr = (c.cw1 * fw_of(r, c.Cw2, c.cw3_6, c.one_plus_cw3_6) - cb1_over_kappa2 * ft2) * rho *
                           (nu_tilde * nu_tilde * inv_dist2);
            double gx = s.g[6](i, j), gy = s.g[7](i, j);
            double diff = cb2_sigma * rho * (gx * gx + gy * gy);
            s.src(i, j) = (prod - destr + diff) * s.vol(i, j);
        }
}

// ----------------------------------------------------------------- solver ---
// solver.rs:86-94
void residual_terms(Solver& s) {
    boundary_apply(s);
    convection_compute(s);
    gradient_compute(s);
    viscous_compute(s);
    dissipation_compute(s);
    source_compute(s);
}

// solver.rs:123-145.  EXT: in local mode every cell advances with its own
// localdt instead of the global minimum.
void update(Solver& s, double alpha, double dt) {
    double a_glob = alpha * dt;
    bool local = s.cfg.local_dt != 0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double a = local ? alpha * s.localdt(i, j) : a_glob;
            double r[5];
            for (int k = 0; k < 5; ++k) r[k] = s.fc[k](i, j) - s.fv[k](i, j) - s.fd[k](i, j);
            r[4] -= s.src(i, j);
            double sc = a * s.inv_vol(i, j);
            for (int k = 0; k < 5; ++k) s.U[k](i, j) = s.Uf[k](i, j) - r[k] * sc;
        }
}

// solver.rs:151-185.  Row-major scan; the first bad cell is reported and the
// scan stops there, exactly like the reference's serial loop.
bool unpack(Solver& s) {
    const double MIN_DENSITY = 1e-15, MIN_PRESSURE = 1e-15;  // solver.rs:21-22
    double gamma = s.cfg.gamma, r_gas = s.cfg.r_gas;
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double rho = s.U[0](i, j);
            if (std::isnan(rho) || rho <= MIN_DENSITY) {
                s.bad_i = i;
                s.bad_j = j;
                s.bad_rho = rho;
                s.bad_p = std::numeric_limits<double>::quiet_NaN();
                return false;
            }
            double inv = 1.0 / rho;
            double vx = s.U[1](i, j) * inv, vy = s.U[2](i, j) * inv;
            double e = s.U[3](i, j) * inv;
            double p = (gamma - 1.0) * (s.U[3](i, j) - rho * (vx * vx + vy * vy) * 0.5);
            if (std::isnan(p) || p <= MIN_PRESSURE) {
                s.bad_i = i;
                s.bad_j = j;
                s.bad_rho = rho;
                s.bad_p = p;
                return false;
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
            s.c(i, j) = std::sqrt(r_gas * gamma * t);
        }
    return true;
}

// solver.rs:97-120
bool advance(Solver& s) {
    for (int k = 0; k < 5; ++k) s.Uf[k].d = s.U[k].d;
    s.rho_prev.d = s.rho.d;
    double dt = timestep_compute(s);
    s.totaltime += dt;
    for (int st = 0; st < 5; ++st) {
        residual_terms(s);
        update(s, RK_ALPHA[st], dt);
        if (!unpack(s)) return false;
    }
    s.step += 1;
    return true;
}

// solver.rs:190-200 — serial sum, i-major / j-minor.
double residual(const Solver& s) {
    double acc = 0.0;
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) {
            double d = s.rho(i, j) - s.rho_prev(i, j);
            acc += d * d;
        }
    return std::sqrt(acc / (double)s.ni / (double)s.nj);
}

// EXT (no counterpart in the reference): force on the wall, integrated over
// the tau faces of ring i = 0.  Pressure is the face average of cell 0 and its
// mirror ghost (equal to p(0, j)); the viscous part is the face diffusion flux
// the reference already forms at those faces (viscous.rs:133-139, momentum
// components 1 and 2).  The tau normal at i = 0 points into the fluid, so the
// force on the body is sum_j (-p n + D_face).  Returns (Fx, Fy) in the mesh
// frame; lift/drag rotation and normalisation are done by the caller.
// Requires residual_terms() to have run on the current state.
void wall_force(const Solver& s, double* fx, double* fy) {
    double ax = 0.0, ay = 0.0;
    for (long j = 0; j < s.nj; ++j) {
        const Face& f = s.T(0, j);
        double pw = 0.5 * (s.p(-1, j) + s.p(0, j));
        double dx = s.tdiff[((size_t)0 * s.nj + j) * 5 + 1];
        double dy = s.tdiff[((size_t)0 * s.nj + j) * 5 + 2];
        ax += -pw * f.nx + dx;
        ay += -pw * f.ny + dy;
    }
    *fx = ax;
    *fy = ay;
}

void alloc_state(Solver& s) {
    int ni = s.ni, nj = s.nj, H = s.H;
    for (int k = 0; k < 5; ++k) {
        s.U[k].init(ni, nj, H);
        s.Uf[k].init(ni, nj, H);
        s.Dx[k].init(ni, nj, H);
        s.Dy[k].init(ni, nj, H);
        s.fc[k].init(ni, nj, H);
        s.fv[k].init(ni, nj, H);
        s.fd[k].init(ni, nj, H);
    }
    for (Field* f : {&s.rho, &s.p, &s.t, &s.vx, &s.vy, &s.e, &s.hh, &s.c, &s.nut, &s.mu, &s.chi, &s.fv1, &s.src,
                     &s.localdt, &s.sensor_i, &s.sensor_j, &s.spec_ratio, &s.rho_prev})
        f->init(ni, nj, H);
    for (int k = 0; k < 8; ++k) s.g[k].init(ni, nj, H);
    size_t nt = (size_t)(ni + 1) * nj, nn = (size_t)ni * nj;
    s.tflux.assign(nt * 5, 0.0);
    s.tdiff.assign(nt * 5, 0.0);
    s.tdiss.assign(nt * 5, 0.0);
    s.nflux.assign(nn * 5, 0.0);
    s.ndiff.assign(nn * 5, 0.0);
    s.ndiss.assign(nn * 5, 0.0);
    s.tlam.assign(nt, 0.0);
    s.te2.assign(nt, 0.0);
    s.te4.assign(nt, 0.0);
    s.nlam.assign(nn, 0.0);
    s.ne2.assign(nn, 0.0);
    s.ne4.assign(nn, 0.0);
}

// Field lookup by name for the C API.  Returns nullptr when unknown.
const Field* cell_field(const Solver& s, const std::string& n) {
    static const char* gnames[8] = {"dudx", "dudy", "dvdx", "dvdy", "dtdx", "dtdy", "dnutdx", "dnutdy"};
    if (n == "rho") return &s.rho;
    if (n == "p") return &s.p;
    if (n == "T") return &s.t;
    if (n == "u") return &s.vx;
    if (n == "v") return &s.vy;
    if (n == "E") return &s.e;
    if (n == "H") return &s.hh;
    if (n == "c") return &s.c;
    if (n == "nut") return &s.nut;
    if (n == "mu") return &s.mu;
    if (n == "chi") return &s.chi;
    if (n == "fv1") return &s.fv1;
    if (n == "S") return &s.src;
    if (n == "localdt") return &s.localdt;
    if (n == "vol") return &s.vol;
    if (n == "cx") return &s.cx;
    if (n == "cy") return &s.cy;
    if (n == "wall_dist") return &s.wall_dist;
    if (n == "inv_vol") return &s.inv_vol;
    if (n == "inv_d2") return &s.inv_d2;
    if (n == "rho_prev") return &s.rho_prev;
    for (int k = 0; k < 8; ++k)
        if (n == gnames[k]) return &s.g[k];
    if (n.size() == 2 && n[0] == 'U' && n[1] >= '0' && n[1] <= '4') return &s.U[n[1] - '0'];
    if (n.size() == 3 && n[2] >= '0' && n[2] <= '4') {
        int k = n[2] - '0';
        if (n[0] == 'F' && n[1] == 'c') return &s.fc[k];
        if (n[0] == 'F' && n[1] == 'v') return &s.fv[k];
        if (n[0] == 'F' && n[1] == 'd') return &s.fd[k];
        if (n[0] == 'D' && n[1] == 'x') return &s.Dx[k];
        if (n[0] == 'D' && n[1] == 'y') return &s.Dy[k];
    }
    return nullptr;
}

}  // namespace

// ================================================================= C API ====
// Parameter vector layout (all doubles), shared with the Python test helper:
//  0 gamma  1 R  2 T0  3 Ts  4 mu0  5 AOA  6 Ma  7 CFL  8 IM  9 T  10 P
// 11 iteration  12 targetres  13 Cv1  14 Pr  15 Prt  16 sigma  17 Cb1  18 Cb2
// 19 Ct3  20 Ct4  21 Cw2  22 Cw3  23 fv3  24 kappa  25 rmax  26 k2  27 k4
// 28 nut_inf_ratio  29 local_dt
extern "C" {

int jo_nparams(void) { return 30; }

void jo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int jo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Restatement of mesh.rs:109-189.  Returns 0 and fills *n_rings, *n_theta and
// xy (caller-allocated, >= 2*header count doubles) on success; on failure a
// MeshError code: 1 BadHeader, 2 Empty, 3 CountMismatch, 4 BadPoint, 5 TooSmall.
int jo_mesh_parse(const char* text, double* xy, long cap, int* n_rings, int* n_theta, long* err_a, long* err_b) {
    const char* p = text;
    // header line
    const char* eol = strchr(p, '\n');
    std::string header = eol ? std::string(p, eol - p) : std::string(p);
    if (header.empty() && !eol) return 2;
    long ni = 0, nj = 0;
    {
        char* end = nullptr;
        const char* h = header.c_str();
        while (*h == ' ' || *h == '\t' || *h == '\r') ++h;
        if (!(*h >= '0' && *h <= '9')) return 1;
        ni = strtol(h, &end, 10);
        if (end == h || (*end != ' ' && *end != '\t')) return 1;
        h = end;
        while (*h == ' ' || *h == '\t') ++h;
        if (!(*h >= '0' && *h <= '9')) return 1;
        nj = strtol(h, &end, 10);
        if (end == h || (*end != '\0' && *end != ' ' && *end != '\t' && *end != '\r')) return 1;
    }
    long count = 0;
    long lineno = 1;
    p = eol ? eol + 1 : p + strlen(p);
    while (*p) {
        ++lineno;
        const char* e2 = strchr(p, '\n');
        std::string line = e2 ? std::string(p, e2 - p) : std::string(p);
        p = e2 ? e2 + 1 : p + strlen(p);
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos) continue;
        const char* s = line.c_str() + a;
        char* end = nullptr;
        double x = strtod(s, &end);
        if (end == s) {
            if (err_a) *err_a = lineno;
            return 4;
        }
        const char* s2 = end;
        double y = strtod(s2, &end);
        if (end == s2) {
            if (err_a) *err_a = lineno;
            return 4;
        }
        if (2 * count + 1 < cap) {
            xy[2 * count] = x;
            xy[2 * count + 1] = y;
        }
        ++count;
    }
    if (count == 0) return 2;
    if (count != ni * nj) {
        if (err_a) *err_a = ni * nj;
        if (err_b) *err_b = count;
        return 3;
    }
    // trim_closing_duplicate (mesh.rs:169-189)
    if (nj >= 2) {
        bool closed = true;
        for (long r = 0; r < ni && closed; ++r) {
            double ax = xy[2 * (r * nj)], ay = xy[2 * (r * nj) + 1];
            double bx = xy[2 * (r * nj + nj - 1)], by = xy[2 * (r * nj + nj - 1) + 1];
            closed = std::fabs(ax - bx) <= 1e-10 && std::fabs(ay - by) <= 1e-10;
        }
        if (closed) {
            long nn = nj - 1;
            for (long r = 0; r < ni; ++r)
                for (long t = 0; t < nn; ++t) {
                    xy[2 * (r * nn + t)] = xy[2 * (r * nj + t)];
                    xy[2 * (r * nn + t) + 1] = xy[2 * (r * nj + t) + 1];
                }
            nj = nn;
        }
    }
    if (ni < 4 || nj < 8) {
        if (err_a) *err_a = ni;
        if (err_b) *err_b = nj;
        return 5;
    }
    *n_rings = (int)ni;
    *n_theta = (int)nj;
    return 0;
}

// Solver::new (solver.rs:47-62) from a parameter vector and trimmed nodes.
void* jo_new(const double* prm, const double* xy, int n_rings, int n_theta) {
    Solver* s = new Solver();
    Config& c = s->cfg;
    c.gamma = prm[0];
    c.r_gas = prm[1];
    c.t_ref = prm[2];
    c.t_suth = prm[3];
    c.mu0 = prm[4];
    c.aoa = prm[5];
    c.mach = prm[6];
    c.cfl = prm[7];
    c.halo = (int)prm[8];
    c.t_inf = prm[9];
    c.p_inf = prm[10];
    c.iteration = (long)prm[11];
    c.targetres = prm[12];
    c.Cv1 = prm[13];
    c.Pr = prm[14];
    c.Prt = prm[15];
    c.sigma = prm[16];
    c.Cb1 = prm[17];
    c.Cb2 = prm[18];
    c.Ct3 = prm[19];
    c.Ct4 = prm[20];
    c.Cw2 = prm[21];
    c.Cw3 = prm[22];
    c.fv3 = prm[23];
    c.kappa = prm[24];
    c.rmax = prm[25];
    c.k2 = prm[26];
    c.k4 = prm[27];
    c.nut_ratio = prm[28];
    c.local_dt = (int)prm[29];
    finish(c);
    s->n_rings = n_rings;
    s->n_theta = n_theta;
    s->nodes.assign(xy, xy + 2 * (size_t)n_rings * n_theta);
    s->ni = n_rings - 1;
    s->nj = n_theta;
    s->H = c.halo;
    build_geometry(*s);
    alloc_state(*s);
    initialize(*s);
    boundary_apply(*s);
    return s;
}

void jo_free(void* h) { delete static_cast<Solver*>(h); }

int jo_ni(void* h) { return static_cast<Solver*>(h)->ni; }
int jo_nj(void* h) { return static_cast<Solver*>(h)->nj; }

// Derived constants in a fixed order (tests compare them with the product's).
void jo_derived(void* h, double* out) {
    const Config& c = static_cast<Solver*>(h)->cfg;
    double v[] = {c.cv,          c.cp,       c.cw1,        c.cv1_cubed,      c.c_inf,      c.u_inf,
                  c.v_inf,       c.rho_inf,  c.mu_inf,     c.nut_inf,        c.supersonic ? 1.0 : 0.0,
                  c.suth_num,    c.inv_t_ref, c.inv_pr,    c.inv_prt,        c.inv_kappa2, c.cw3_6,
                  c.one_plus_cw3_6};
    memcpy(out, v, sizeof(v));
}

// Returns 0, or 1 on a non-physical state (details via jo_nonphysical).
int jo_advance(void* h) { return advance(*static_cast<Solver*>(h)) ? 0 : 1; }

void jo_nonphysical(void* h, long* i, long* j, double* rho, double* p) {
    Solver* s = static_cast<Solver*>(h);
    *i = s->bad_i;
    *j = s->bad_j;
    *rho = s->bad_rho;
    *p = s->bad_p;
}

// Solver::run (solver.rs:203-226).  max_steps < 0 uses the config's
// iteration count.  history (may be null) receives one residual per step.
// Returns 0 ok, 1 non-physical; *steps_done and *res_out are always set.
int jo_run(void* h, long max_steps, double* history, long* steps_done, double* res_out) {
    Solver* s = static_cast<Solver*>(h);
    long limit = max_steps < 0 ? s->cfg.iteration : max_steps;
    double res = std::numeric_limits<double>::quiet_NaN();
    long done = 0;
    for (long k = 1; k <= limit; ++k) {
        if (!advance(*s)) {
            *steps_done = done;
            *res_out = res;
            return 1;
        }
        res = residual(*s);
        done = k;
        if (history) history[k - 1] = res;
        if (res < s->cfg.targetres) break;
    }
    *steps_done = done;
    *res_out = res;
    return 0;
}

double jo_timestep(void* h) { return timestep_compute(*static_cast<Solver*>(h)); }
void jo_residual_terms(void* h) { residual_terms(*static_cast<Solver*>(h)); }
double jo_residual(void* h) { return residual(*static_cast<Solver*>(h)); }
double jo_totaltime(void* h) { return static_cast<Solver*>(h)->totaltime; }
long jo_step(void* h) { return static_cast<Solver*>(h)->step; }
int jo_unpack(void* h) { return unpack(*static_cast<Solver*>(h)) ? 0 : 1; }
void jo_boundary(void* h) { boundary_apply(*static_cast<Solver*>(h)); }
void jo_set_uniform(void* h, double rho, double vx, double vy, double p, double nut) {
    set_uniform(*static_cast<Solver*>(h), rho, vx, vy, p, nut);
}

// Individual kernels (the free functions the reference exports), for the
// free-stream tests that must bypass boundary::apply.
void jo_kernel(void* h, const char* name) {
    Solver& s = *static_cast<Solver*>(h);
    std::string n(name);
    if (n == "convection") convection_compute(s);
    else if (n == "gradient") gradient_compute(s);
    else if (n == "viscous") viscous_compute(s);
    else if (n == "dissipation") dissipation_compute(s);
    else if (n == "source") source_compute(s);
    else if (n == "boundary") boundary_apply(s);
}

// Copy an interior cell field, i-major / j-minor.  Returns 0 or -1 (unknown).
int jo_get(void* h, const char* name, double* out) {
    Solver& s = *static_cast<Solver*>(h);
    const Field* f = cell_field(s, name);
    if (!f) return -1;
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) out[i * s.nj + j] = (*f)(i, j);
    return 0;
}

// Copy a cell field including its halo: (ni+2H) x (nj+2H), row-major.
int jo_get_halo(void* h, const char* name, double* out) {
    Solver& s = *static_cast<Solver*>(h);
    const Field* f = cell_field(s, name);
    if (!f) return -1;
    memcpy(out, f->d.data(), f->d.size() * sizeof(double));
    return 0;
}

// Overwrite one conserved component on the interior (i-major / j-minor).
void jo_set_u(void* h, int k, const double* in) {
    Solver& s = *static_cast<Solver*>(h);
    for (long i = 0; i < s.ni; ++i)
        for (long j = 0; j < s.nj; ++j) s.U[k](i, j) = in[i * s.nj + j];
}

// Face arrays.  which: 0 tau geometry (nx,ny,mx,my per face), 1 n geometry,
// 2 tau conv flux, 3 n conv flux, 4 tau diff, 5 n diff, 6 tau diss, 7 n diss,
// 8 tau lambda, 9 n lambda.  Returns the number of doubles written.
long jo_faces(void* h, int which, double* out) {
    Solver& s = *static_cast<Solver*>(h);
    const std::vector<double>* v = nullptr;
    switch (which) {
        case 0:
            for (size_t k = 0; k < s.tau.size(); ++k) {
                out[4 * k] = s.tau[k].nx;
                out[4 * k + 1] = s.tau[k].ny;
                out[4 * k + 2] = s.tau[k].mx;
                out[4 * k + 3] = s.tau[k].my;
            }
            return (long)s.tau.size() * 4;
        case 1:
            for (size_t k = 0; k < s.nrm.size(); ++k) {
                out[4 * k] = s.nrm[k].nx;
                out[4 * k + 1] = s.nrm[k].ny;
                out[4 * k + 2] = s.nrm[k].mx;
                out[4 * k + 3] = s.nrm[k].my;
            }
            return (long)s.nrm.size() * 4;
        case 2: v = &s.tflux; break;
        case 3: v = &s.nflux; break;
        case 4: v = &s.tdiff; break;
        case 5: v = &s.ndiff; break;
        case 6: v = &s.tdiss; break;
        case 7: v = &s.ndiss; break;
        case 8: v = &s.tlam; break;
        case 9: v = &s.nlam; break;
        default: return -1;
    }
    memcpy(out, v->data(), v->size() * sizeof(double));
    return (long)v->size();
}

// EXT: wall force in the mesh frame (see wall_force above).
void jo_wall_force(void* h, double* fx, double* fy) { wall_force(*static_cast<Solver*>(h), fx, fy); }

}  // extern "C"
