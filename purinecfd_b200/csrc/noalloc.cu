// jst_residual_noalloc: the density residual sqrt(sum (rho - rho_prev)^2 / NI / NJ)
// for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they need this number:
// a solver embedded in a plugin whose host owns every device allocation
// through its own pool, a real-time monitoring loop that must not allocate
// (cudaMalloc synchronises the device and can stall other streams), or code
// running inside a region where the host forbids new allocations.  They
// already hold the two density fields and a result slot in memory they own,
// so this entry point takes device pointers for all three and keeps its only
// scratch — one partial sum per thread block — in a fixed file-scope
// __device__ array.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/jst_gpu.h"

namespace jst {
void set_call_error(const std::string& msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 8;
constexpr int kCellsPerBlock = kThreads * kCellsPerThread;  // 2048
constexpr int kMaxBlocks = 8192;
constexpr long kMaxCells = (long)kMaxBlocks * kCellsPerBlock;  // 16,777,216 cells

// The scratch: one FP64 partial per block, 64 KiB.  Every GPU that loads this
// library holds it until the process exits.  All calls share it.
static __device__ __align__(256) double g_noalloc_partials[kMaxBlocks];

// Device addresses of g_noalloc_partials, one per device, looked up once.
constexpr int kMaxDevices = 64;
double* g_partials_addr[kMaxDevices] = {};
std::mutex g_partials_mu;

// Fixed-shape per-block sums: thread t adds cells t, t+256, ... of the block's
// chunk in order, then a tree over the 256 threads.  Deterministic.
__global__ void __launch_bounds__(kThreads) k_noalloc_partial(const double* rho, const double* prev, long n,
                                                             double* partials) {
    __shared__ double red[kThreads];
    long base = (long)blockIdx.x * kCellsPerBlock;
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < kCellsPerThread; ++q) {
        long id = base + q * kThreads + threadIdx.x;
        if (id < n) {
            double d = rho[id] - prev[id];
            acc += d * d;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

// One block: sum the nb partials written by this call, then
// sqrt(acc / NI / NJ) (solver.rs:199).
__global__ void __launch_bounds__(kThreads) k_noalloc_final(const double* partials, int nb, int ni, int nj,
                                                           double* out) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += kThreads) acc += partials[k];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(red[0] / (double)ni / (double)nj);
}

// Device address of the scratch on the current device (set-up on first use).
double* partials_on_current_device(std::string* err) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *err = std::string("cudaGetDevice failed: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        *err = "device ordinal out of range for the residual scratch table";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_partials_mu);
    if (!g_partials_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            *err = std::string("cudaGetSymbolAddress failed for the residual scratch: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_partials_addr[dev] = static_cast<double*>(p);
    }
    return g_partials_addr[dev];
}

}  // namespace

extern "C" jst_status jst_residual_noalloc(const double* rho, const double* rho_prev, int ni, int nj, double* out,
                                           void* stream) {
    if (!rho || !rho_prev || !out || ni <= 0 || nj <= 0) {
        jst::set_call_error("jst_residual_noalloc: null pointer or non-positive size");
        return JST_ERR_ARG;
    }
    long n = (long)ni * nj;
    if (n > kMaxCells) {
        jst::set_call_error("jst_residual_noalloc: " + std::to_string(n) + " cells exceed the maximum of " +
                            std::to_string(kMaxCells) + " (fixed scratch of " + std::to_string(kMaxBlocks) +
                            " partial sums)");
        return JST_ERR_ARG;
    }
    std::string err;
    double* partials = partials_on_current_device(&err);
    if (!partials) {
        jst::set_call_error(err);
        return JST_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int nb = (int)((n + kCellsPerBlock - 1) / kCellsPerBlock);
    k_noalloc_partial<<<nb, kThreads, 0, st>>>(rho, rho_prev, n, partials);
    k_noalloc_final<<<1, kThreads, 0, st>>>(partials, nb, ni, nj, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        jst::set_call_error(std::string("jst_residual_noalloc launch failed: ") + cudaGetErrorString(e));
        return JST_ERR_CUDA;
    }
    return JST_OK;
}
