// kofm_noalloc.cu - field reduction that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application that
// owns a fixed device-memory budget and hands out every buffer from its own
// pool, or a caller on a latency-critical path where an allocation's implicit
// device synchronisation is not acceptable.  kofm_reduce needs a context
// (which allocates); this entry point reduces a field the caller already has
// on the device into an output the caller provides, and keeps its only
// scratch -- the per-block partial sums -- in a fixed array compiled into the
// library.
//
// Contract (also in include/kofm.h):
//   * the scratch is g_noalloc_partials below: KOFM_NOALLOC_MAX_PARTIALS
//     doubles (32 KiB), held by every device that loads the library until the
//     process exits;
//   * one partial per KOFM_NOALLOC_CHUNK nodes, so at most
//     KOFM_NOALLOC_MAX_NODES nodes per call; larger fields are rejected with
//     KOFM_ERR_TOO_LARGE before any work is queued;
//   * every call overwrites the partials it uses (nothing needs to start at
//     zero), and all calls share the one array: calls that overlap on the GPU
//     (different streams, or several host threads) race on it;
//   * host code cannot use the array's name as a device address: every call
//     made outside stream capture resolves the address with
//     cudaGetSymbolAddress in the calling thread's current CUDA context and
//     remembers it for that context; a call made while `stream` is being
//     captured uses the remembered address of the current context, so the
//     first call in each context must come before any capture
//     (KOFM_ERR_STATE otherwise).  Resolving afresh outside capture keeps the
//     address right after cudaDeviceReset and for callers that drive their
//     own driver-API contexts, where the array lives at a different address
//     in each context.
#include "kofm.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include <utility>
#include <vector>

namespace {

static __device__ __align__(256) double g_noalloc_partials[KOFM_NOALLOC_MAX_PARTIALS];

// The array's device address per CUDA context, guarded by a mutex (several
// host threads may make their first calls at once).
std::mutex g_addr_mutex;
std::vector<std::pair<CUcontext, double*>> g_addr;

// cuCtxGetCurrent through the runtime's driver entry point (no link-time
// dependency on the driver library).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

bool current_context(CUcontext* out) {
    static CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (CtxGetCurrentFn) nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    *out = nullptr;
    return fn && fn(out) == CUDA_SUCCESS && *out;
}

// Device address of g_noalloc_partials in the current context; 0 on success.
int partials_address(cudaStream_t st, double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return KOFM_ERR_NO_DEVICE;
    // outside capture, cudaGetSymbolAddress also makes the device's primary
    // context current if the calling thread has none yet
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return KOFM_ERR_INVALID_ARG;
    CUcontext ctx = nullptr;
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "kofm: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return KOFM_ERR_NO_DEVICE;
        }
        if (!current_context(&ctx)) return KOFM_ERR_NO_DEVICE;
        std::lock_guard<std::mutex> lock(g_addr_mutex);
        for (auto& a : g_addr)
            if (a.first == ctx) { a.second = static_cast<double*>(p); *out = a.second; return KOFM_OK; }
        g_addr.emplace_back(ctx, static_cast<double*>(p));
        *out = static_cast<double*>(p);
        return KOFM_OK;
    }
    if (!current_context(&ctx)) return KOFM_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    for (const auto& a : g_addr)
        if (a.first == ctx) { *out = a.second; return KOFM_OK; }
    return KOFM_ERR_STATE;  // first call in this context made under capture
}

template <int OP>
__device__ __forceinline__ double op2(double a, double b) {
    return OP == KOFM_OP_SUM ? a + b : (OP == KOFM_OP_MIN ? fmin(a, b) : fmax(a, b));
}
template <int OP>
__device__ __forceinline__ double op_init() {
    return OP == KOFM_OP_SUM ? 0.0 : (OP == KOFM_OP_MIN ? 1.0e308 : -1.0e308);
}

// Block b reduces nodes [b*CHUNK, (b+1)*CHUNK) of the pitch*ny array, counting
// only columns < ncols, into partials[b].
template <int OP>
__global__ void __launch_bounds__(256)
k_noalloc_partial(const float* __restrict__ v, long long n, int pitch, int ncols,
                  double* __restrict__ partials) {
    __shared__ double sh[8];
    const long long s = (long long)blockIdx.x * KOFM_NOALLOC_CHUNK;
    const long long e = s + KOFM_NOALLOC_CHUNK < n ? s + KOFM_NOALLOC_CHUNK : n;
    double acc = op_init<OP>();
    for (long long i = s + threadIdx.x; i < e; i += 256)
        if ((int)(i % pitch) < ncols) acc = op2<OP>(acc, (double)v[i]);
    for (int off = 16; off > 0; off >>= 1) acc = op2<OP>(acc, __shfl_down_sync(0xffffffffu, acc, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = sh[0];
        for (int w = 1; w < 8; ++w) t = op2<OP>(t, sh[w]);
        partials[blockIdx.x] = t;
    }
}

// One block combines the partials in a fixed order (deterministic).
template <int OP>
__global__ void __launch_bounds__(256)
k_noalloc_final(const double* __restrict__ partials, int np, double* __restrict__ out) {
    __shared__ double sh[256];
    const int per = (np + 255) / 256;
    double acc = op_init<OP>();
    for (int i = threadIdx.x * per; i < (threadIdx.x + 1) * per && i < np; ++i)
        acc = op2<OP>(acc, partials[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = op2<OP>(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

template <int OP>
cudaError_t launch(const float* v, long long n, int pitch, int ncols, double* partials, int np,
                   double* out, cudaStream_t st) {
    k_noalloc_partial<OP><<<np, 256, 0, st>>>(v, n, pitch, ncols, partials);
    k_noalloc_final<OP><<<1, 256, 0, st>>>(partials, np, out);
    return cudaGetLastError();
}

}  // namespace

extern "C" int kofm_reduce_field_noalloc(const float* field, int32_t ncols, int32_t pitch,
                                         int32_t ny, int32_t op, double* out, void* stream) {
    if (!field || !out || ncols < 1 || pitch < ncols || ny < 1) return KOFM_ERR_INVALID_ARG;
    if (op < KOFM_OP_SUM || op > KOFM_OP_MAX) return KOFM_ERR_INVALID_ARG;
    const long long n = (long long)pitch * ny;
    if (n > (long long)KOFM_NOALLOC_MAX_NODES) return KOFM_ERR_TOO_LARGE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* partials = nullptr;
    const int sa = partials_address(st, &partials);
    if (sa != KOFM_OK) return sa;
    const int np = (int)((n + KOFM_NOALLOC_CHUNK - 1) / KOFM_NOALLOC_CHUNK);
    cudaError_t e;
    switch (op) {
        case KOFM_OP_SUM: e = launch<KOFM_OP_SUM>(field, n, pitch, ncols, partials, np, out, st); break;
        case KOFM_OP_MIN: e = launch<KOFM_OP_MIN>(field, n, pitch, ncols, partials, np, out, st); break;
        default: e = launch<KOFM_OP_MAX>(field, n, pitch, ncols, partials, np, out, st); break;
    }
    if (e != cudaSuccess) {
        fprintf(stderr, "kofm: no-alloc reduction launch failed: %s\n", cudaGetErrorString(e));
        return KOFM_ERR_CALLING_KERNEL;
    }
    return KOFM_OK;
}
