/*
 * jst_gpu_debug.h — test hooks exported by libjst_gpu.so beside the public
 * C ABI of jst_gpu.h.  They exist so that the test suite can reach single
 * kernels and the device arithmetic directly; a solver integration never
 * needs them.  Same conventions as jst_gpu.h (extern "C", jst_status
 * returns, plain pointers and sizes).
 */
#ifndef JST_GPU_DEBUG_H
#define JST_GPU_DEBUG_H

#include "jst_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Cells::set_uniform (state.rs:198-203) on the passes path: every cell,
 * halo and corners included, set to one primitive state, bypassing the
 * boundary conditions — the precondition of the reference's free-stream
 * properties (jst-rs/tests/properties.rs:126-156).  No effect on the fused
 * path. */
jst_status jst_debug_set_uniform(jst_solver* s, double rho, double vx, double vy, double p, double nut);

/* Runs one reference pass of the passes path by name ("boundary",
 * "convection", "gradient", "viscous", "dissipation", "source") on the
 * current state: the kernel free functions boundary::apply and the
 * *::compute of jst-rs/src/lib.rs:59-71.  Unknown names do nothing; no
 * effect on the fused path. */
jst_status jst_debug_kernel(jst_solver* s, const char* name);

/* Makes every bulk row-copy barrier of the fused path's marching strips
 * expect `bytes` more than its copies deliver (0 restores it), so that the
 * kernels' bounded waits run out and the next step returns JST_ERR_TIMEOUT:
 * the failure path of JST_STAGING_BULK, tested without a fault. */
jst_status jst_debug_staging_extra_tx(jst_solver* s, int bytes);

/* The fused kernels' FP64 quotient, square root, exponential and inverse
 * sixth root beside CUDA's own, for n operand pairs (a[k], b[k]):
 * out[8k .. 8k+7] = quick a/b, a/b, quick sqrt(b), sqrt(b), quick exp(a),
 * exp(a), b^(-1/6), 1/cbrt(sqrt(b)).  a, b and out are host arrays; the call
 * allocates and frees its own device buffer. */
jst_status jst_debug_quick_arith(const double* a, const double* b, double* out, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* JST_GPU_DEBUG_H */
