// Host-side readers for the reference's two input formats:
//  * config.json (jst-rs/src/config.rs:11-111, serde field names and defaults),
//  * the O-mesh text file (jst-rs/src/mesh.rs:109-189).
// Both return the reference's error cases as status codes plus a message.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace jst {

// ------------------------------------------------------------------ JSON ----
// A small recursive-descent JSON reader (objects, arrays, numbers, strings,
// literals) — enough for config.json.
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    double num = 0.0;
    bool is_int = false;  // number written without fraction or exponent
    bool b = false;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    const JVal* get(const std::string& k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class JParser {
  public:
    explicit JParser(const std::string& t) : s(t) {}
    bool parse(JVal& out, std::string& err) {
        try {
            ws();
            value(out);
            ws();
            if (p != s.size()) fail("trailing characters");
            return true;
        } catch (const std::string& e) {
            err = e;
            return false;
        }
    }

  private:
    const std::string& s;
    size_t p = 0;
    [[noreturn]] void fail(const char* what) {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < p && k < s.size(); ++k) {
            if (s[k] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
        }
        throw std::string(what) + " at line " + std::to_string(line) + " column " + std::to_string(col);
    }
    void ws() {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) ++p;
    }
    void value(JVal& v) {
        if (p >= s.size()) fail("EOF while parsing a value");
        char c = s[p];
        if (c == '{') {
            v.kind = JVal::OBJ;
            ++p;
            ws();
            if (p < s.size() && s[p] == '}') {
                ++p;
                return;
            }
            while (true) {
                ws();
                if (p >= s.size() || s[p] != '"') fail("key must be a string");
                JVal key;
                string(key);
                ws();
                if (p >= s.size() || s[p] != ':') fail("expected `:`");
                ++p;
                ws();
                JVal val;
                value(val);
                v.obj.emplace_back(key.str, std::move(val));
                ws();
                if (p < s.size() && s[p] == ',') {
                    ++p;
                    continue;
                }
                if (p < s.size() && s[p] == '}') {
                    ++p;
                    return;
                }
                fail("expected `,` or `}`");
            }
        } else if (c == '[') {
            v.kind = JVal::ARR;
            ++p;
            ws();
            if (p < s.size() && s[p] == ']') {
                ++p;
                return;
            }
            while (true) {
                ws();
                JVal e;
                value(e);
                v.arr.push_back(std::move(e));
                ws();
                if (p < s.size() && s[p] == ',') {
                    ++p;
                    continue;
                }
                if (p < s.size() && s[p] == ']') {
                    ++p;
                    return;
                }
                fail("expected `,` or `]`");
            }
        } else if (c == '"') {
            string(v);
        } else if (s.compare(p, 4, "true") == 0) {
            v.kind = JVal::BOOL;
            v.b = true;
            p += 4;
        } else if (s.compare(p, 5, "false") == 0) {
            v.kind = JVal::BOOL;
            p += 5;
        } else if (s.compare(p, 4, "null") == 0) {
            v.kind = JVal::NUL;
            p += 4;
        } else if (c == '-' || (c >= '0' && c <= '9')) {
            size_t st = p;
            if (s[p] == '-') ++p;
            bool intg = true;
            while (p < s.size() && std::isdigit((unsigned char)s[p])) ++p;
            if (p < s.size() && s[p] == '.') {
                intg = false;
                ++p;
                while (p < s.size() && std::isdigit((unsigned char)s[p])) ++p;
            }
            if (p < s.size() && (s[p] == 'e' || s[p] == 'E')) {
                intg = false;
                ++p;
                if (p < s.size() && (s[p] == '+' || s[p] == '-')) ++p;
                while (p < s.size() && std::isdigit((unsigned char)s[p])) ++p;
            }
            std::string tok = s.substr(st, p - st);
            char* end = nullptr;
            v.kind = JVal::NUM;
            v.num = std::strtod(tok.c_str(), &end);
            v.is_int = intg;
            if (end == tok.c_str() || *end) fail("invalid number");
        } else {
            fail("expected value");
        }
    }
    void string(JVal& v) {
        v.kind = JVal::STR;
        ++p;
        while (p < s.size() && s[p] != '"') {
            if (s[p] == '\\') {
                ++p;
                if (p >= s.size()) break;
                char e = s[p];
                if (e == 'n') v.str += '\n';
                else if (e == 't') v.str += '\t';
                else if (e == 'u') {
                    p += 4;
                    v.str += '?';
                } else v.str += e;
                ++p;
            } else {
                v.str += s[p++];
            }
        }
        if (p >= s.size()) fail("EOF while parsing a string");
        ++p;
    }
};

// ---------------------------------------------------------------- config ----
struct RawConfig {
    double gamma, r_gas, t_ref, t_suth, mu0;
    double aoa, mach, cfl;
    long halo;
    double t_inf, p_inf;
    long iteration = 10000;   // config.rs:52-54
    double targetres = 1e-10; // config.rs:55-57
    double Cv1, Pr, Prt, sigma, Cb1, Cb2, Ct3, Ct4, Cw2, Cw3, fv3, kappa, rmax;
    double k2, k4;
    double nut_inf_ratio = 0.1;  // optional `simulation.nut_inf_ratio`; the reference hard-codes 0.1
    double chord = 0.0;          // optional `simulation.chord` for CL/CD; 0 = wall x-extent
};

// Parses config.json text like serde would for jst-rs's Config: unknown keys
// are ignored, `solver` and its keys are optional, `IM` and `iteration` must be
// non-negative integers, every other field a number.
inline bool parse_config(const std::string& text, RawConfig& c, std::string& err) {
    JVal root;
    if (!JParser(text).parse(root, err)) return false;
    if (root.kind != JVal::OBJ) {
        err = "invalid type: expected struct Config";
        return false;
    }
    auto section = [&](const char* name, bool required) -> const JVal* {
        const JVal* v = root.get(name);
        if (!v) {
            if (required) err = std::string("missing field `") + name + "`";
            return nullptr;
        }
        if (v->kind != JVal::OBJ) {
            err = std::string("invalid type for `") + name + "`: expected a map";
            return nullptr;
        }
        return v;
    };
    auto num = [&](const JVal* sec, const char* key, double* out, bool required) -> bool {
        const JVal* v = sec ? sec->get(key) : nullptr;
        if (!v) {
            if (required) {
                err = std::string("missing field `") + key + "`";
                return false;
            }
            return true;
        }
        if (v->kind != JVal::NUM) {
            err = std::string("invalid type for `") + key + "`: expected f64";
            return false;
        }
        *out = v->num;
        return true;
    };
    auto uint = [&](const JVal* sec, const char* key, long* out, bool required) -> bool {
        const JVal* v = sec ? sec->get(key) : nullptr;
        if (!v) {
            if (required) {
                err = std::string("missing field `") + key + "`";
                return false;
            }
            return true;
        }
        if (v->kind != JVal::NUM || !v->is_int || v->num < 0) {
            err = std::string("invalid type for `") + key + "`: expected usize";
            return false;
        }
        *out = (long)v->num;
        return true;
    };
    const JVal* ph = section("physics", true);
    if (!ph) return false;
    const JVal* sim = section("simulation", true);
    if (!sim) return false;
    const JVal* sa = section("spalart_allmaras", true);
    if (!sa) return false;
    const JVal* dis = section("dissipation", true);
    if (!dis) return false;
    const JVal* sol = root.get("solver");
    if (sol && sol->kind != JVal::OBJ) {
        err = "invalid type for `solver`: expected a map";
        return false;
    }
    bool ok = num(ph, "gamma", &c.gamma, true) && num(ph, "R", &c.r_gas, true) && num(ph, "T0", &c.t_ref, true) &&
              num(ph, "Ts", &c.t_suth, true) && num(ph, "mu0", &c.mu0, true) && num(sim, "AOA", &c.aoa, true) &&
              num(sim, "Ma", &c.mach, true) && num(sim, "CFL", &c.cfl, true) && uint(sim, "IM", &c.halo, true) &&
              num(sim, "T", &c.t_inf, true) && num(sim, "P", &c.p_inf, true) &&
              num(sim, "nut_inf_ratio", &c.nut_inf_ratio, false) && num(sim, "chord", &c.chord, false) &&
              uint(sol, "iteration", &c.iteration, false) && num(sol, "targetres", &c.targetres, false) &&
              num(sa, "Cv1", &c.Cv1, true) && num(sa, "Pr", &c.Pr, true) && num(sa, "Prt", &c.Prt, true) &&
              num(sa, "sigma", &c.sigma, true) && num(sa, "Cb1", &c.Cb1, true) && num(sa, "Cb2", &c.Cb2, true) &&
              num(sa, "Ct3", &c.Ct3, true) && num(sa, "Ct4", &c.Ct4, true) && num(sa, "Cw2", &c.Cw2, true) &&
              num(sa, "Cw3", &c.Cw3, true) && num(sa, "fv3", &c.fv3, true) && num(sa, "kappa", &c.kappa, true) &&
              num(sa, "rmax", &c.rmax, true) && num(dis, "k2", &c.k2, true) && num(dis, "k4", &c.k4, true);
    return ok;
}

// ------------------------------------------------------------------ mesh ----
// Error codes follow the MeshError variants (mesh.rs:17-44); values match
// jst_status's JST_ERR_MESH_*.
enum MeshErr { MESH_OK = 0, MESH_IO = 1, MESH_BAD_HEADER = 2, MESH_EMPTY = 3, MESH_COUNT = 4, MESH_BAD_POINT = 5,
               MESH_TOO_SMALL = 6 };

inline bool parse_usize(const std::string& tok, long* out) {
    const char* s = tok.c_str();
    if (*s == '+') ++s;
    if (!*s) return false;
    long v = 0;
    for (; *s; ++s) {
        if (*s < '0' || *s > '9') return false;
        v = v * 10 + (*s - '0');
        if (v > (1L << 40)) return false;
    }
    *out = v;
    return true;
}

inline bool parse_f64(const std::string& tok, double* out) {
    char* end = nullptr;
    *out = std::strtod(tok.c_str(), &end);
    return end != tok.c_str() && *end == '\0';
}

inline void split_ws(const std::string& line, std::vector<std::string>& toks) {
    toks.clear();
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
        size_t st = i;
        while (i < line.size() && !std::isspace((unsigned char)line[i])) ++i;
        if (i > st) toks.push_back(line.substr(st, i - st));
    }
}

// Mesh::parse (mesh.rs:109-166) + trim_closing_duplicate (169-189).
inline int parse_mesh(const std::string& text, std::vector<double>& xy, int* n_rings, int* n_theta,
                      std::string& err) {
    std::vector<std::string> lines;
    {
        size_t st = 0;
        while (st <= text.size()) {
            size_t e = text.find('\n', st);
            if (e == std::string::npos) {
                if (st < text.size()) lines.push_back(text.substr(st));
                break;
            }
            std::string l = text.substr(st, e - st);
            if (!l.empty() && l.back() == '\r') l.pop_back();
            lines.push_back(l);
            st = e + 1;
        }
    }
    if (lines.empty()) {
        err = "mesh file contains no points";
        return MESH_EMPTY;
    }
    std::vector<std::string> toks;
    split_ws(lines[0], toks);
    long ni = 0, nj = 0;
    if (toks.size() < 2 || !parse_usize(toks[0], &ni) || !parse_usize(toks[1], &nj)) {
        std::string h = lines[0];
        size_t a = h.find_first_not_of(" \t\r"), b = h.find_last_not_of(" \t\r");
        h = a == std::string::npos ? "" : h.substr(a, b - a + 1);
        err = "bad header \"" + h + "\": expected `i_total j_total`";
        return MESH_BAD_HEADER;
    }
    xy.clear();
    xy.reserve(2 * (size_t)std::min<long>(ni * nj, 1L << 28));
    for (size_t k = 1; k < lines.size(); ++k) {
        split_ws(lines[k], toks);
        if (toks.empty()) continue;
        double x, y;
        if (toks.size() < 2 || !parse_f64(toks[0], &x) || !parse_f64(toks[1], &y)) {
            err = "line " + std::to_string(k + 1) + ": cannot parse point";
            return MESH_BAD_POINT;
        }
        xy.push_back(x);
        xy.push_back(y);
    }
    long count = (long)xy.size() / 2;
    if (count == 0) {
        err = "mesh file contains no points";
        return MESH_EMPTY;
    }
    if (count != ni * nj) {
        err = "expected " + std::to_string(ni * nj) + " points from header, found " + std::to_string(count);
        return MESH_COUNT;
    }
    // trim_closing_duplicate
    if (nj >= 2) {
        bool closed = true;
        for (long r = 0; r < ni && closed; ++r) {
            double ax = xy[2 * (r * nj)], ay = xy[2 * (r * nj) + 1];
            double bx = xy[2 * (r * nj + nj - 1)], by = xy[2 * (r * nj + nj - 1) + 1];
            closed = std::fabs(ax - bx) <= 1e-10 && std::fabs(ay - by) <= 1e-10;
        }
        if (closed) {
            long nn = nj - 1;
            std::vector<double> t(2 * (size_t)ni * nn);
            for (long r = 0; r < ni; ++r)
                std::memcpy(&t[2 * (size_t)r * nn], &xy[2 * (size_t)r * nj], sizeof(double) * 2 * nn);
            xy.swap(t);
            nj = nn;
        }
    }
    if (ni < 4 || nj < 8) {
        err = "mesh " + std::to_string(ni) + "x" + std::to_string(nj) +
              " too small: the JST 4th-order stencil needs at least 4 rings and 8 circumferential points";
        return MESH_TOO_SMALL;
    }
    *n_rings = (int)ni;
    *n_theta = (int)nj;
    return MESH_OK;
}

// Rust `{:.Pe}` formatting (LowerExp with precision): mantissa with P
// decimals, exponent with no `+` and no zero padding, e.g. 1.01325000e5.
inline std::string rust_exp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", prec, v);
    std::string s(buf);
    size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    int ex = std::atoi(s.c_str() + e + 1);
    return mant + "e" + std::to_string(ex);
}

}  // namespace jst
