// noalloc.cu -- a dot product for callers that cannot allocate device memory.
//
// hpcgx_dot needs a problem handle, whose creation allocates its reduction
// scratch with cudaMalloc.  Some callers cannot allocate: code that runs
// inside another framework's memory budget (a caching allocator that owns
// the GPU's memory, where a stray cudaMalloc may fail or fragment the pool),
// and latency-critical loops where cudaMalloc/cudaFree would stall or
// synchronise the device.  hpcgx_dot_noalloc serves them: the per-block
// partial sums live in one fixed array in the library's own device memory
// (a file-scope __device__ array, loaded with the module), so a call
// allocates nothing; the caller passes the input vectors and the device
// location of the result.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hpcgx.h"

namespace hpcgx {
int set_error(int code, const char *msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int64_t kPerBlock = (int64_t)kThreads * kPerThread;   // 2048 elements per block
constexpr int kMaxPartials = HPCGX_DOT_NOALLOC_MAX_N / kPerBlock;  // 32768 blocks
constexpr int kMaxDevices = 64;

static_assert(HPCGX_DOT_NOALLOC_MAX_N % kPerBlock == 0, "limit must be a whole number of blocks");

// Partial sums (one per block) followed by the arrival counter in the last
// 256-byte line: 32768 * 8 B + 256 B = 256.25 KiB on every GPU that loads the
// library, held until the process exits.
static __device__ __align__(256) double g_dot_scratch[kMaxPartials + 32];

// The address of g_dot_scratch, cached per device together with the unique
// id of the context it was resolved in: after cudaDeviceReset (or any other
// teardown of the primary context) the module is loaded again and the array
// may move, so a cached address is only reused in the same context.
struct ScratchCache {
  unsigned long long ctx_id;
  void *addr;
};
ScratchCache g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points, so
// that the library needs no link against libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// *id = 0 when the thread has no current context yet (the runtime creates the
// primary context lazily, e.g. in cudaGetSymbolAddress).
int current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) !=
            cudaSuccess ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) !=
            cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      cudaGetLastError();
      return hpcgx::set_error(HPCGX_ECUDA,
                              "hpcgx_dot_noalloc: driver entry points cuCtxGetCurrent/cuCtxGetId "
                              "unavailable");
    }
    get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    get_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext ctx = nullptr;
  *id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS)
    return hpcgx::set_error(HPCGX_ECUDA, "hpcgx_dot_noalloc: cuCtxGetCurrent failed");
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS)
    return hpcgx::set_error(HPCGX_ECUDA, "hpcgx_dot_noalloc: cuCtxGetId failed");
  return HPCGX_OK;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Each block reduces its 2048 elements to one partial; the last block to
// arrive adds the partials in a fixed order that depends only on the grid
// size (strided per-thread sums, then a warp shuffle tree, then the warps in
// order), so the result does not depend on which block finishes last; it
// writes the result and re-arms the counter.
__global__ void __launch_bounds__(kThreads)
k_dot_noalloc(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
              double *partials, unsigned int *counter, double *result) {
  __shared__ double sh[kThreads / 32];
  __shared__ int amlast;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kPerBlock + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < kPerThread; ++j) {
    const int64_t i = base + (int64_t)j * kThreads;
    if (i < n) acc += x[i] * y[i];
  }
  acc = warp_sum(acc);
  if (lane == 0) sh[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    partials[blockIdx.x] = t;
    __threadfence();
    amlast = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!amlast) return;
  __threadfence();
  double t = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads) t += __ldcg(partials + b);
  t = warp_sum(t);
  __syncthreads();
  if (lane == 0) sh[wid] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
    *result = s;
    *counter = 0u;
  }
}

// Device address of g_dot_scratch on the current device, resolved once per
// device and context.  In host code the symbol name is only a host-side
// handle; the kernel must be given this address instead.
int scratch_for_device(int dev, double **out) {
  if (dev < 0 || dev >= kMaxDevices)
    return hpcgx::set_error(HPCGX_EINVAL, "hpcgx_dot_noalloc: device index out of range");
  unsigned long long ctx_id = 0;
  int rc = current_context_id(&ctx_id);
  if (rc != HPCGX_OK) return rc;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  ScratchCache &c = g_scratch[dev];
  if (!c.addr || ctx_id == 0 || c.ctx_id != ctx_id) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_dot_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return hpcgx::set_error(HPCGX_ECUDA, "hpcgx_dot_noalloc: cudaGetSymbolAddress failed");
    }
    if (ctx_id == 0) {   // the lookup above created the context
      rc = current_context_id(&ctx_id);
      if (rc != HPCGX_OK) return rc;
    }
    c.addr = ptr;
    c.ctx_id = ctx_id;
  }
  *out = static_cast<double *>(c.addr);
  return HPCGX_OK;
}

}  // namespace

extern "C" int hpcgx_dot_noalloc(int64_t n, const double *x, const double *y, double *result,
                                 void *stream) {
  if (n < 0 || n > HPCGX_DOT_NOALLOC_MAX_N)
    return hpcgx::set_error(HPCGX_EINVAL,
                            "hpcgx_dot_noalloc: n must be in [0, HPCGX_DOT_NOALLOC_MAX_N = "
                            "67108864]; use hpcgx_dot for longer vectors");
  if (!result || (n > 0 && (!x || !y)))
    return hpcgx::set_error(HPCGX_EINVAL, "hpcgx_dot_noalloc: null vector or result pointer");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return hpcgx::set_error(HPCGX_ECUDA, "hpcgx_dot_noalloc: no current CUDA device");
  double *scratch = nullptr;
  int rc = scratch_for_device(dev, &scratch);
  if (rc != HPCGX_OK) return rc;
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kMaxPartials);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The counter must start at zero; a normal launch leaves it at zero, this
  // clears whatever an interrupted earlier launch may have left.
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return hpcgx::set_error(HPCGX_ECUDA, cudaGetErrorString(e));
  const int blocks = n > 0 ? (int)((n + kPerBlock - 1) / kPerBlock) : 1;
  k_dot_noalloc<<<blocks, kThreads, 0, s>>>(n, x, y, scratch, counter, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) return hpcgx::set_error(HPCGX_ECUDA, cudaGetErrorString(e));
  return HPCGX_OK;
}
