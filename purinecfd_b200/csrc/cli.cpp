// `jst` command-line front end over the C ABI: the flags, stdout lines and
// output files of the reference's CLI (jst-rs/src/bin/jst.rs:10-125), so that
// scripts driving it (e.g. a regex on `wall clock:` and `final residual:`)
// work unchanged.  Extra flags select the precision, time-step mode, kernel
// path and device.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "jst_gpu.h"

namespace {

// Rust `{:.Pe}` (mantissa with P decimals, exponent without `+` or padding).
std::string rexp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", prec, v);
    std::string s(buf);
    size_t e = s.find('e');
    return s.substr(0, e) + "e" + std::to_string(std::atoi(s.c_str() + e + 1));
}

struct Cli {
    std::string mesh = "fangdata.txt", config = "config.json", out = "result.csv", reslog = "res.log";
    std::string checkpoint, restart;
    long steps = -1;
    bool quiet = false, no_output = false;
    long threads = 0;
    int precision = JST_PREC_FP64, dt_mode = JST_DT_GLOBAL, path = JST_PATH_FUSED, device = 0;
};

void usage() {
    std::puts(
        "2D JST + Spalart-Allmaras finite-volume solver (B200)\n\n"
        "Usage: jst [OPTIONS]\n\n"
        "Options:\n"
        "      --mesh <MESH>            [default: fangdata.txt]\n"
        "      --config <CONFIG>        [default: config.json]\n"
        "      --steps <STEPS>          override solver.iteration\n"
        "      --out <OUT>              [default: result.csv]\n"
        "      --reslog <RESLOG>        [default: res.log]\n"
        "      --quiet                  only print the summary\n"
        "      --threads <THREADS>      accepted for compatibility [default: 0]\n"
        "      --no-output              write no output files\n"
        "      --precision <fp64|split> stage arithmetic [default: fp64]\n"
        "      --dt <global|local>      time step mode [default: global]\n"
        "      --path <fused|passes>    kernels [default: fused]\n"
        "      --device <N>             CUDA device [default: 0]\n"
        "      --restart <FILE>         continue from a checkpoint written by --checkpoint\n"
        "      --checkpoint <FILE>      write a checkpoint after the run\n"
        "  -h, --help                   Print help");
}

bool parse(int argc, char** argv, Cli& c) {
    for (int k = 1; k < argc; ++k) {
        std::string a = argv[k];
        std::string v;
        size_t eq = a.find('=');
        if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
            v = a.substr(eq + 1);
            a = a.substr(0, eq);
        }
        auto val = [&]() -> std::string {
            if (!v.empty()) return v;
            if (k + 1 >= argc) {
                std::fprintf(stderr, "error: a value is required for '%s'\n", a.c_str());
                std::exit(2);
            }
            return argv[++k];
        };
        if (a == "-h" || a == "--help") {
            usage();
            std::exit(0);
        } else if (a == "--mesh") c.mesh = val();
        else if (a == "--config") c.config = val();
        else if (a == "--steps") c.steps = std::strtol(val().c_str(), nullptr, 10);
        else if (a == "--out") c.out = val();
        else if (a == "--reslog") c.reslog = val();
        else if (a == "--quiet") c.quiet = true;
        else if (a == "--no-output") c.no_output = true;
        else if (a == "--threads") c.threads = std::strtol(val().c_str(), nullptr, 10);
        else if (a == "--precision") c.precision = val() == "split" ? JST_PREC_FP32_SPLIT : JST_PREC_FP64;
        else if (a == "--dt") c.dt_mode = val() == "local" ? JST_DT_LOCAL : JST_DT_GLOBAL;
        else if (a == "--path") c.path = val() == "passes" ? JST_PATH_PASSES : JST_PATH_FUSED;
        else if (a == "--device") c.device = (int)std::strtol(val().c_str(), nullptr, 10);
        else if (a == "--restart") c.restart = val();
        else if (a == "--checkpoint") c.checkpoint = val();
        else {
            std::fprintf(stderr, "error: unexpected argument '%s' found\n", a.c_str());
            return false;
        }
    }
    return true;
}

struct LogCtx {
    FILE* log;
    bool quiet;
    uint64_t offset;  // steps completed before this run (restart)
};

void on_step(void* user, uint64_t step, double res) {
    LogCtx* c = static_cast<LogCtx*>(user);
    step += c->offset;
    if (!c->quiet) std::printf("step:%6llu | residual:%s\n", (unsigned long long)step, rexp(res, 6).c_str());
    if (c->log) std::fprintf(c->log, "%llu,%s\n", (unsigned long long)step, rexp(res, 6).c_str());
}

}  // namespace

int main(int argc, char** argv) {
    Cli cli;
    if (!parse(argc, argv, cli)) return 2;
    jst_opts o;
    jst_default_opts(&o);
    o.precision = cli.precision;
    o.dt_mode = cli.dt_mode;
    o.kernel_path = cli.path;
    o.device = cli.device;
    jst_solver* s = nullptr;
    jst_status rc = jst_create_from_paths(cli.config.c_str(), cli.mesh.c_str(), &o, &s);
    if (rc != JST_OK) {
        std::fprintf(stderr, "Error: %s\n", jst_last_error(nullptr));
        return 1;
    }
    int ni = jst_ni(s), nj = jst_nj(s);
    std::printf("mesh %s: %d rings x %d points -> %lld cells\n", cli.mesh.c_str(), ni + 1, nj, (long long)ni * nj);
    std::printf("threads: %ld\n", cli.threads > 0 ? cli.threads : 1L);
    LogCtx ctx{nullptr, cli.quiet, 0};
    if (!cli.restart.empty()) {
        jst_nonphysical bad0{};
        if (jst_checkpoint_load(s, cli.restart.c_str(), &bad0) != JST_OK) {
            std::fprintf(stderr, "Error: %s\n", jst_last_error(nullptr));
            jst_destroy(s);
            return 1;
        }
        int64_t done0 = 0;
        jst_step_count(s, &done0);
        ctx.offset = (uint64_t)done0;
        std::printf("restarted from %s at step %lld\n", cli.restart.c_str(), (long long)done0);
    }
    if (!cli.no_output) {
        ctx.log = std::fopen(cli.reslog.c_str(), "w");
        if (!ctx.log) {
            std::fprintf(stderr, "Error: cannot create %s\n", cli.reslog.c_str());
            return 1;
        }
        std::fputs("step,residual\n", ctx.log);
    }
    auto t0 = std::chrono::steady_clock::now();
    jst_run_report rep{};
    jst_nonphysical bad{};
    rc = jst_run(s, cli.steps, on_step, &ctx, &rep, &bad);
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (ctx.log) std::fclose(ctx.log);
    if (rc != JST_OK) {
        std::fprintf(stderr, "Error: %s\n", jst_last_error(s));
        jst_destroy(s);
        return 1;
    }
    std::printf("steps: %lld  final residual: %s%s\n", (long long)rep.steps, rexp(rep.residual, 6).c_str(),
                rep.converged ? "  (converged)" : "");
    std::printf("totaltime (physical): %s s\n", rexp(rep.totaltime, 6).c_str());
    double per = rep.steps > 0 ? wall / (double)rep.steps : 0.0;
    std::printf("wall clock: %.6f s  (%.4f ms/step, %.1f ns/cell/step)\n", wall, per * 1e3,
                per / ((double)ni * nj) * 1e9);
    if (!cli.checkpoint.empty()) {
        if (jst_checkpoint_save(s, cli.checkpoint.c_str()) != JST_OK) {
            std::fprintf(stderr, "Error: %s\n", jst_last_error(nullptr));
            jst_destroy(s);
            return 1;
        }
        std::printf("checkpoint written to %s\n", cli.checkpoint.c_str());
    }
    if (!cli.no_output) {
        rc = jst_write_csv(s, cli.out.c_str());
        if (rc != JST_OK) {
            std::fprintf(stderr, "Error: %s\n", jst_last_error(s));
            jst_destroy(s);
            return 1;
        }
        std::printf("all data is written in %s\n", cli.out.c_str());
    }
    jst_destroy(s);
    return 0;
}
