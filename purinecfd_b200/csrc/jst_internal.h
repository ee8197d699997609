// Internal interfaces between the host code (api.cu) and the kernel
// translation units (passes.cu, fused.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "jst_common.cuh"

namespace jst {

// Geometry in HBM, FP64, structure of arrays without halo (geometry.rs:45-63).
// Cell arrays are NI x NJ, tau-face arrays (NI+1) x NJ, n-face arrays NI x NJ,
// all i-major / j-minor.
struct Geom {
    int ni, nj;
    double *vol, *cx, *cy, *wdist, *inv_vol, *inv_d2;
    double *tnx, *tny, *tmx, *tmy;
    double *nnx, *nny, *nmx, *nmy;
};

// passes.cu ------------------------------------------------------------------
void geometry_build(const double* d_xy, int n_rings, int n_theta, Geom& g, cudaStream_t st);

struct Passes;
Passes* passes_create(int ni, int nj, int H, std::string* err);
void passes_destroy(Passes* P);
void passes_init(Passes* P, const Geom& g, const PhysConst& c, cudaStream_t st);
void passes_set_uniform(Passes* P, const PhysConst& c, double rho, double vx, double vy, double p, double nut,
                        cudaStream_t st);
void passes_timestep(Passes* P, const Geom& g, const PhysConst& c, int accumulate, cudaStream_t st);
void passes_kernel(Passes* P, const Geom& g, const PhysConst& c, const char* which, cudaStream_t st);
void passes_residual_terms(Passes* P, const Geom& g, const PhysConst& c, cudaStream_t st);
void passes_update_unpack(Passes* P, const Geom& g, const PhysConst& c, double alpha, int local, cudaStream_t st);
void passes_unpack(Passes* P, const PhysConst& c, cudaStream_t st);
void passes_snapshot(Passes* P, cudaStream_t st);
void passes_residual(Passes* P, cudaStream_t st);
void passes_wall_force(Passes* P, const Geom& g, double* d_out, cudaStream_t st);
unsigned long long* passes_bad_ptr(Passes* P);
double* passes_dt_ptr(Passes* P);
double* passes_totaltime_ptr(Passes* P);
double* passes_residual_ptr(Passes* P);
bool passes_field(Passes* P, int id, const double** base, int* stride, int* halo);

}  // namespace jst
