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
#include <cuda.h>
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

// Device addresses of g_noalloc_partials, one per device, looked up once per
// CUDA context: each entry remembers the unique id (cuCtxGetId) of the
// context it was looked up in, so a context created later on the same device
// (after cudaDeviceReset, or a driver context made current by the host) gets
// its own lookup instead of a stale address.
constexpr int kMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id;
    double* ptr;
};
ScratchAddr g_partials_addr[kMaxDevices] = {};
std::mutex g_partials_mu;

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry points
// (the library does not link libcuda itself).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

bool current_context_id(unsigned long long* id, std::string* err) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess || !a || !b) {
            *err = "cuCtxGetCurrent / cuCtxGetId not available from the CUDA driver";
            return false;
        }
        get_current = reinterpret_cast<CtxGetCurrentFn>(a);
        get_id = reinterpret_cast<CtxGetIdFn>(b);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) {
        *err = "no current CUDA context for the residual scratch lookup";
        return false;
    }
    return true;
}

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

// Device address of the scratch on the current device (set-up on the first
// call in each context, with that device current).
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
    // The entry is valid while the context it was looked up in is the
    // current one.  A thread with no current context yet gets one from the
    // lookup itself (cudaGetSymbolAddress makes the device's primary context
    // current), so the id is read again after it.
    unsigned long long ctx = 0;
    std::string no_ctx;
    const bool have_ctx = current_context_id(&ctx, &no_ctx);
    std::lock_guard<std::mutex> lock(g_partials_mu);
    ScratchAddr& slot = g_partials_addr[dev];
    if (have_ctx && slot.ptr && slot.ctx_id == ctx) return slot.ptr;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
        *err = std::string("cudaGetSymbolAddress failed for the residual scratch: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (!current_context_id(&ctx, err)) return nullptr;
    slot.ptr = static_cast<double*>(p);
    slot.ctx_id = ctx;
    return slot.ptr;
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
