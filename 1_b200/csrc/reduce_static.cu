// Allocation-free reduction (mmx_reduce_static, include/mmx.h).
//
// Same reductions as gpu_reduce (sum, max, max |x|, min, sum |x|), for
// callers that must not touch the device allocator: code that runs while
// another thread captures a CUDA graph in global capture mode (where
// cudaMalloc is an error), host callbacks, and embedders that budget all
// device memory up front.  gpu_reduce allocates its per-block partials with
// cudaMalloc on its first call on a device; this variant keeps them in a
// fixed array compiled into the library.
//
// The scratch array is a file-scope __device__ array: every GPU that loads
// the library holds its 8 KB until the process exits.  In host code the
// name g_reduce_scratch is only a host-side stand-in, not a device address;
// the device address is obtained once per device (per CUDA context) with
// cudaGetSymbolAddress (the first call on a device does it, with that
// device current) and passed to the kernels.
//
// Limits and sharing: one partial per block of 4096 elements, at most
// MMX_REDUCE_STATIC_BLOCKS blocks, so n <= 4,194,304; larger n is rejected
// with MMX_ERR_SIZE.  Every call reuses the same array; each call writes
// every partial it later reads, so nothing needs clearing between calls,
// but calls that overlap on the GPU (for instance on two streams) race on
// the array and must be serialised by the caller.
#include <math.h>
#include <mutex>

#include "mmx_common.cuh"
#include "../../include/mmx.h"

#define RS_THREADS 256
#define RS_PER_THREAD 16
#define RS_CHUNK (RS_THREADS * RS_PER_THREAD)

static_assert(MMX_REDUCE_STATIC_MAX_N == MMX_REDUCE_STATIC_BLOCKS * RS_CHUNK, "scratch size and limit disagree");

static __device__ __align__(256) double g_reduce_scratch[MMX_REDUCE_STATIC_BLOCKS];

__device__ __forceinline__ double rs_op(int op, double a, double b) {
  switch (op) {
    case 1:
    case 5: return a + b;
    case 2:
    case 3: return fmax(a, b);
    default: return fmin(a, b);
  }
}
__device__ __forceinline__ double rs_ident(int op) { return op == 2 ? -INFINITY : op == 4 ? INFINITY : 0.0; }
__device__ __forceinline__ double rs_load(int op, float v) {
  return (op == 3 || op == 5) ? (double)fabsf(v) : (double)v;
}

__device__ double rs_block(int op, double v) {
  __shared__ double sh[RS_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) v = rs_op(op, v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < RS_THREADS / 32 ? sh[threadIdx.x] : rs_ident(op);
    for (int o = 16; o > 0; o >>= 1) v = rs_op(op, v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// block b reduces elements [b * RS_CHUNK, (b + 1) * RS_CHUNK) into part[b]
__global__ void __launch_bounds__(RS_THREADS) k_rs_partial(int op, const float* __restrict__ in, int n,
                                                           double* __restrict__ part) {
  double v = rs_ident(op);
  int base = blockIdx.x * RS_CHUNK;
#pragma unroll
  for (int j = 0; j < RS_PER_THREAD; j++) {
    int i = base + j * RS_THREADS + threadIdx.x;
    if (i < n) v = rs_op(op, v, rs_load(op, in[i]));
  }
  v = rs_block(op, v);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_final(int op, const double* __restrict__ part, int nb,
                                                         float* __restrict__ out) {
  double v = rs_ident(op);
  for (int i = threadIdx.x; i < nb; i += RS_THREADS) v = rs_op(op, v, part[i]);
  v = rs_block(op, v);
  if (threadIdx.x == 0) out[0] = (float)v;
}

// Device address of g_reduce_scratch, looked up once per CUDA context (the
// module, and so the array, is loaded per context: a context created anew,
// e.g. after cudaDeviceReset, holds it at a new address).  The context is
// read with the driver's cuCtxGetCurrent, reached through the runtime's
// entry-point table so the library does not link the driver library; the
// call is legal while another thread captures a graph.
typedef int (*ctx_get_fn)(void**);
static std::mutex g_rs_mu;
struct RsEntry {
  void* ctx;
  int dev;
  double* addr;
};
static RsEntry g_rs_cache[64];
static int g_rs_n = 0;
static ctx_get_fn g_ctx_get = nullptr;

static int rs_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    mmx_set_error(cudaGetErrorString(e));
    return MMX_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_rs_mu);
  if (!g_ctx_get) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f) {
      mmx_set_error("mmx_reduce_static: cuCtxGetCurrent not available");
      return MMX_ERR_CUDA;
    }
    g_ctx_get = (ctx_get_fn)f;
  }
  // A thread that has made no runtime call yet has no context bound (the
  // runtime binds the device's primary context at its first launch): it
  // uses the device's entry, which is the primary context's.
  void* ctx = nullptr;
  if (g_ctx_get(&ctx) != 0) ctx = nullptr;
  for (int i = 0; i < g_rs_n; i++)
    if (g_rs_cache[i].dev == dev && (!ctx || g_rs_cache[i].ctx == ctx)) {
      *out = g_rs_cache[i].addr;
      return MMX_OK;
    }
  // set-up: looks the array up (loading the module into the context if
  // needed), then records the context it belongs to
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_reduce_scratch);
  if (e != cudaSuccess || p == nullptr) {
    mmx_set_error(e != cudaSuccess ? cudaGetErrorString(e) : "mmx_reduce_static: no symbol address");
    return MMX_ERR_CUDA;
  }
  if (g_ctx_get(&ctx) != 0) ctx = nullptr;
  // replace a stale entry of this device (an earlier context), else append
  int slot = -1;
  for (int i = 0; i < g_rs_n; i++)
    if (g_rs_cache[i].dev == dev) slot = i;
  if (slot < 0) {
    if (g_rs_n == 64) {
      mmx_set_error("mmx_reduce_static: too many devices");
      return MMX_ERR_ARG;
    }
    slot = g_rs_n++;
  }
  g_rs_cache[slot] = RsEntry{ctx, dev, (double*)p};
  *out = (double*)p;
  return MMX_OK;
}

extern "C" int mmx_reduce_static(int operation, const float* input, int n, float* result, cudaStream_t stream) {
  if (operation < 1 || operation > 5) {
    mmx_set_error("mmx_reduce_static: unknown operation (1 add, 2 max, 3 maxabs, 4 min, 5 sumabs)");
    return MMX_ERR_ARG;
  }
  if (!input || !result || n <= 0) {
    mmx_set_error("mmx_reduce_static: null pointer or n <= 0");
    return MMX_ERR_ARG;
  }
  if (n > MMX_REDUCE_STATIC_MAX_N) {
    mmx_set_error("mmx_reduce_static: n exceeds MMX_REDUCE_STATIC_MAX_N (4194304 elements)");
    return MMX_ERR_SIZE;
  }
  double* part = nullptr;
  int rc = rs_scratch(&part);
  if (rc != MMX_OK) return rc;
  int nb = (n + RS_CHUNK - 1) / RS_CHUNK;
  k_rs_partial<<<nb, RS_THREADS, 0, stream>>>(operation, input, n, part);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_rs_final<<<1, RS_THREADS, 0, stream>>>(operation, part, nb, result);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    mmx_set_error(cudaGetErrorString(e));
    return MMX_ERR_CUDA;
  }
  return MMX_OK;
}
