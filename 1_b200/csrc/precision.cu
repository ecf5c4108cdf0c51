// Precision form: DFT stages as split-BF16 GEMMs on tcgen05 tensor cores.
//
// mmx_dft_tc: batched complex DFTs of length 32 as one tensor-core GEMM per
// 256 vectors (dft_tc.cuh).  It is the building block of the split-
// precision Y convolution of 2D films (mmx_params.precision), and is
// exported on its own so its error against an FP64 DFT can be measured.
#include <mutex>
#include <vector>
#include <cmath>
#include <cstring>

#include "dft_tc.cuh"
#include "mmx_common.cuh"
#include "../../include/mmx.h"

namespace {

constexpr int DL = 32;           // DFT length of one GEMM
constexpr int DK = 2 * DL;       // interleaved real K (and M) extent
constexpr int DN = 256;          // vectors per CTA (GEMM N)
constexpr int DT = 128;          // threads: 4 warps, one per TMEM sub-partition
constexpr uint32_t TMEM_COLS = 256;
constexpr int WAIT_ITERS = 1 << 22;

// DFT matrix exp(sign 2 pi i j k / L) in the interleaved real form, split
// into bfloat16 hi and lo, laid out as canonical K-major 64 x 64 tiles.
// Built on the host in float64.
void build_dft_tiles(int L, int sign, std::vector<uint16_t>& hi, std::vector<uint16_t>& lo) {
  const int K = 2 * L;
  hi.assign((size_t)2 * L * K, 0);
  lo.assign((size_t)2 * L * K, 0);
  auto bf = [](float x) -> uint16_t {  // round to nearest even
    uint32_t u;
    memcpy(&u, &x, 4);
    uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(r >> 16);
  };
  auto unbf = [](uint16_t h) -> float {
    uint32_t u = (uint32_t)h << 16;
    float x;
    memcpy(&x, &u, 4);
    return x;
  };
  for (int j = 0; j < L; j++)
    for (int i = 0; i < L; i++) {
      double ang = sign * 2.0 * M_PI * (double)((j * i) % L) / (double)L;
      float c = (float)cos(ang), s = (float)sin(ang);
      float blk[2][2] = {{c, -s}, {s, c}};
      for (int rm = 0; rm < 2; rm++)
        for (int rk = 0; rk < 2; rk++) {
          float v = blk[rm][rk];
          uint16_t h = bf(v);
          uint16_t l = bf(v - unbf(h));
          uint32_t off = dtc::kmajor_off(2 * j + rm, 2 * i + rk, K) / 2;
          hi[off] = h;
          lo[off] = l;
        }
    }
}

struct DftTables {
  uint16_t* fwd = nullptr;  // hi tile then lo tile
  uint16_t* inv = nullptr;
};
std::mutex g_dft_mu;
DftTables g_dft[64];  // per device

int dft_tables(const uint16_t** out, int inverse) {
  int dev = 0;
  MMX_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { mmx_set_error("device index out of range"); return MMX_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_dft_mu);
  uint16_t*& p = inverse ? g_dft[dev].inv : g_dft[dev].fwd;
  if (!p) {
    std::vector<uint16_t> hi, lo;
    build_dft_tiles(DL, inverse ? 1 : -1, hi, lo);
    if (cudaMalloc(&p, 2 * hi.size() * sizeof(uint16_t)) != cudaSuccess) {
      p = nullptr;
      mmx_set_error("out of device memory");
      return MMX_ERR_MEM;
    }
    MMX_TRY(cudaMemcpy(p, hi.data(), hi.size() * 2, cudaMemcpyHostToDevice));
    MMX_TRY(cudaMemcpy(p + hi.size(), lo.data(), lo.size() * 2, cudaMemcpyHostToDevice));
  }
  *out = p;
  return MMX_OK;
}

}  // namespace

// Batched length-32 DFTs: out[v] = DFT(in[v]) for v < nvec, one CTA per 256
// vectors.  Shared memory: W hi/lo (2 x 8 KB), X hi/lo (2 x 32 KB).
__global__ void __launch_bounds__(DT) k_dft32_tc(const float2* __restrict__ in, float2* __restrict__ out, int nvec,
                                                 const uint16_t* __restrict__ wtiles, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) uint64_t bar;
  constexpr int WB = DK * DK * 2;  // bytes of one W tile
  constexpr int XB = DN * DK * 2;  // bytes of one X tile
  unsigned char* w_hi = smem;
  unsigned char* w_lo = smem + WB;
  unsigned char* x_hi = smem + 2 * WB;
  unsigned char* x_lo = smem + 2 * WB + XB;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int v0 = blockIdx.x * DN;

  if (warp == 0) dtc::tmem_alloc(&tmem_slot, TMEM_COLS);
  if (threadIdx.x == 0) dtc::mbar_init(&bar, 1);
  // W tiles: a plain copy (already in the canonical layout)
  {
    const uint4* src = reinterpret_cast<const uint4*>(wtiles);
    uint4* dst = reinterpret_cast<uint4*>(w_hi);
    for (int i = threadIdx.x; i < 2 * WB / 16; i += DT) dst[i] = __ldg(&src[i]);
  }
  // X tiles: vector n's element i (complex) -> K index 2i (re), 2i+1 (im)
  for (int e = threadIdx.x; e < DN * DL; e += DT) {
    int n = e / DL, i = e % DL;
    float2 x = (v0 + n < nvec) ? in[(size_t)(v0 + n) * DL + i] : make_float2(0.f, 0.f);
    __nv_bfloat16 h, l;
    dtc::split_bf16(x.x, h, l);
    uint32_t o = dtc::kmajor_off(n, 2 * i, DK);
    *reinterpret_cast<__nv_bfloat16*>(x_hi + o) = h;
    *reinterpret_cast<__nv_bfloat16*>(x_lo + o) = l;
    dtc::split_bf16(x.y, h, l);
    o = dtc::kmajor_off(n, 2 * i + 1, DK);
    *reinterpret_cast<__nv_bfloat16*>(x_hi + o) = h;
    *reinterpret_cast<__nv_bfloat16*>(x_lo + o) = l;
  }
  dtc::fence_async_smem();
  dtc::fence_before_sync();
  __syncthreads();
  dtc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0) {
    dtc::gemm_split<DK, DN>(tmem, w_hi, w_lo, x_hi, x_lo);
    dtc::mma_commit(&bar);
  }
  bool ok = dtc::mbar_wait(&bar, 0, WAIT_ITERS);
  ok = __syncthreads_and(ok);  // uniform: the TMEM loads below are warp-collective
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  dtc::fence_after_sync();
  if (ok) {
    // warp w: accumulator rows 16w..16w+15 in lanes 0..15
    const uint32_t tbase = tmem + ((uint32_t)(32 * warp) << 16);
    const int m = 16 * warp + lane;  // valid for lane < 16
    const int j = m >> 1, ri = m & 1;
    for (int c = 0; c < DN; c += 8) {
      float v[8];
      dtc::tmem_ld8(tbase + c, v);
      dtc::tmem_wait_ld();
      if (lane < 16) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          int n = c + q;
          if (v0 + n < nvec) {
            float* o = reinterpret_cast<float*>(&out[(size_t)(v0 + n) * DL + j]);
            o[ri] = v[q];
          }
        }
      }
    }
  }
  dtc::fence_before_sync();
  __syncthreads();
  if (warp == 0) dtc::tmem_free(tmem, TMEM_COLS);
}

extern "C" int mmx_dft_tc(const float2* in, float2* out, int nvec, int inverse, cudaStream_t st) {
  if (!in || !out || nvec < 0) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  if (nvec == 0) return MMX_OK;
  const uint16_t* w = nullptr;
  MMX_CHECK_RC(dft_tables(&w, inverse));
  static int* d_err = nullptr;
  if (!d_err) {
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) { mmx_set_error("out of device memory"); return MMX_ERR_MEM; }
  }
  MMX_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  const size_t smem = 2 * (DK * DK * 2) + 2 * (DN * DK * 2);
  MMX_TRY(cudaFuncSetAttribute(k_dft32_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_dft32_tc<<<(nvec + DN - 1) / DN, DT, smem, st>>>(in, out, nvec, w, d_err);
  MMX_TRY(cudaGetLastError());
  int h_err = 0;
  MMX_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MMX_TRY(cudaStreamSynchronize(st));
  if (h_err) { mmx_set_error("tensor-core DFT: completion wait timed out"); return MMX_ERR_CUDA; }
  return MMX_OK;
}
