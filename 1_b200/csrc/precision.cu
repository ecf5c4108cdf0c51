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
uint16_t bf16_rne(float x) {  // round to nearest even (finite x)
  uint32_t u;
  memcpy(&u, &x, 4);
  uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}
float bf16_val(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float x;
  memcpy(&x, &u, 4);
  return x;
}
void build_dft_tiles(int L, int sign, std::vector<uint16_t>& hi, std::vector<uint16_t>& lo) {
  const int K = 2 * L;
  hi.assign((size_t)2 * L * K, 0);
  lo.assign((size_t)2 * L * K, 0);
  auto bf = bf16_rne;
  auto unbf = bf16_val;
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

// The same matrix split three ways (hi, mid, lo: each the bfloat16
// rounding of what the previous parts leave), three consecutive tiles.
void build_dft_tiles3(int L, int sign, std::vector<uint16_t>& out) {
  const int K = 2 * L;
  const size_t T = (size_t)2 * L * K;
  out.assign(3 * T, 0);
  for (int j = 0; j < L; j++)
    for (int i = 0; i < L; i++) {
      double ang = sign * 2.0 * M_PI * (double)((j * i) % L) / (double)L;
      float c = (float)cos(ang), s = (float)sin(ang);
      float blk[2][2] = {{c, -s}, {s, c}};
      for (int rm = 0; rm < 2; rm++)
        for (int rk = 0; rk < 2; rk++) {
          float v = blk[rm][rk];
          const uint32_t off = dtc::kmajor_off(2 * j + rm, 2 * i + rk, K) / 2;
          for (int part = 0; part < 3; part++) {
            uint16_t h = bf16_rne(v);
            out[part * T + off] = h;
            v -= bf16_val(h);
          }
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

DftTables g_dft3[64];  // per device, three-way split

int dft_tables3(const uint16_t** out, int inverse) {
  int dev = 0;
  MMX_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { mmx_set_error("device index out of range"); return MMX_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_dft_mu);
  uint16_t*& p = inverse ? g_dft3[dev].inv : g_dft3[dev].fwd;
  if (!p) {
    std::vector<uint16_t> t;
    build_dft_tiles3(DL, inverse ? 1 : -1, t);
    if (cudaMalloc(&p, t.size() * sizeof(uint16_t)) != cudaSuccess) {
      p = nullptr;
      mmx_set_error("out of device memory");
      return MMX_ERR_MEM;
    }
    MMX_TRY(cudaMemcpy(p, t.data(), t.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
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

// ---------------------------------------------------------------------
// Split-precision Y convolution of a 2D film, P1 = 1024 (Ny = 512).
//
// The 1024-point transform along Y is two layers of 32-point DFTs with the
// index maps n = 32 n1 + n2 and k = k1 + 32 k2 (Cooley-Tukey):
//   F1  A[k1][n2] = sum_n1 W32^(n1 k1) y[32 n1 + n2]     (rows n1 >= 16 are padding: 0)
//   tw  A[k1][n2] *= W1024^(n2 k1)
//   F2  X[k1 + 32 k2] = sum_n2 W32^(n2 k2) A[k1][n2]
// then H = K X per bin (the 2D kernel product of gpu_kernelmul4), and the
// inverse in reverse order, keeping only the outputs y < 512.
//
// A CTA takes 4 kz columns, one per TMEM lane quarter.  Each layer is, per
// component c, one tensor-core GEMM D_c[128 x 64] = X_c[128 x 64] . W^T with
// the 128 vectors v = (kz, 32-point index) as M, so vector v's 32 complex
// outputs land in TMEM lane v, columns 64 c .. 64 c + 63 (re, im
// interleaved).  Both operands are split three ways into bfloat16 (x = hi +
// mid + lo, each the rounding of the remainder) and the six products with
// weight >= 2^-16 relative (hh, hm, mh, hl, lh, mm) are accumulated in FP32:
// about 24 significant bits per operand, the FP32 transform's precision.
// Two warps share each lane quarter and split every epilogue's columns in
// halves; thread 0 issues all MMAs.
// ---------------------------------------------------------------------
namespace {
constexpr int YT = 256;                        // threads: 8 warps, two per TMEM sub-partition
constexpr int YKZ = 4;                         // kz columns per CTA, one per TMEM lane quarter
constexpr int YL = 1024;                       // padded Y length
constexpr int YK = 3 * 64;                     // operand K extent: 3 components x 64
constexpr int YLBO = 144;                      // bytes between K-adjacent core matrices (128 + 16)
constexpr int YSBO = (YK / 8) * YLBO;          // bytes between 8-row groups (3456)
constexpr int YXB = 16 * YSBO;                 // bytes of one 128-row operand tile (55296)
constexpr int YWB = 64 * 64 * 2;               // bytes of one W tile
constexpr size_t YSMEM = 3 * (size_t)YXB + 6 * (size_t)YWB + YL * sizeof(float2);
constexpr int YN = 512;                        // data length along Y
constexpr int YSP = YN + 8;                    // staging pitch of one (component, kz) line, float2
constexpr int KTS = 520;                       // kernel line pitch (floats) of the kz-major coefficients
static_assert(3 * YKZ * YSP * sizeof(float2) <= 6 * (size_t)YWB + YL * sizeof(float2),
              "the input staging lies in the W and twiddle area");

struct YconvTc {
  float2* S;
  int64_t CS;
  int HZ, N1;
  const float* kt;     // kernel coefficients Kxx, Kyy, Kzz, Kyz as [4][HZ][KTS] (fy fastest)
  int64_t ktcs;        // component stride of kt
  const uint16_t* wf;  // forward W: hi, mid, lo tiles
  const uint16_t* wi;  // inverse W: hi, mid, lo tiles
  const float2* tw;    // [32][32]: tw[32 a + b] = exp(-2 pi i a b / 1024)
  int* err;
};

// byte offset of (row r, K index k) in an operand tile: canonical K-major
// core matrices, K-adjacent ones YLBO bytes apart so that a warp's 32
// stores at K = 2 n (n = lane) into one row hit 32 distinct banks
__host__ __device__ __forceinline__ uint32_t xoff(int r, int k) {
  return (uint32_t)((r >> 3) * YSBO + (k >> 3) * YLBO + (r & 7) * 16 + (k & 7) * 2);
}

// x = h + m + l, each a bfloat16 rounding of what is left
__device__ __forceinline__ void split3(float x, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);
  m = __float2bfloat16_rn(r1);
  l = __float2bfloat16_rn(r1 - __bfloat162float(m));
}

// (re, im) at K positions k, k+1 (k even): one 4-byte store into each of
// the three tiles
__device__ __forceinline__ void put_pair(unsigned char* x, int r, int k, float2 v) {
  __nv_bfloat162 h, m, l;
  split3(v.x, h.x, m.x, l.x);
  split3(v.y, h.y, m.y, l.y);
  const uint32_t o = xoff(r, k);
  *reinterpret_cast<__nv_bfloat162*>(x + o) = h;
  *reinterpret_cast<__nv_bfloat162*>(x + YXB + o) = m;
  *reinterpret_cast<__nv_bfloat162*>(x + 2 * YXB + o) = l;
}

// four complex values at K positions k0 .. k0+7 (k0 a multiple of 8): one
// 16-byte store into each of the three tiles
__device__ __forceinline__ void put_quad(unsigned char* x, int r, int k0, const float2* v) {
  __align__(16) __nv_bfloat162 h[4], m[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    split3(v[q].x, h[q].x, m[q].x, l[q].x);
    split3(v[q].y, h[q].y, m[q].y, l[q].y);
  }
  const uint32_t o = xoff(r, k0);
  *reinterpret_cast<uint4*>(x + o) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(x + YXB + o) = *reinterpret_cast<const uint4*>(m);
  *reinterpret_cast<uint4*>(x + 2 * YXB + o) = *reinterpret_cast<const uint4*>(l);
}

// One thread: for every component c, D_c (TMEM columns 64 c ..) = the split
// product of the operand rows' K slice [64 c, 64 c + kmax) and W
// (N = 64 outputs x 64 inputs, canonical K-major, LBO 128, SBO 1024).
__device__ __forceinline__ void gemm3(uint32_t tmem, const unsigned char* x, const unsigned char* w, int kmax) {
  constexpr uint32_t idesc = dtc::idesc_bf16(128, 64);
  constexpr int PA[6] = {0, 0, 1, 0, 2, 1};  // operand part of each product
  constexpr int PB[6] = {0, 1, 0, 2, 0, 1};  // W part of each product
  const uint32_t xa = dtc::smem_u32(x), wb = dtc::smem_u32(w);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    for (int kk = 0; kk < kmax; kk += 16) {
#pragma unroll
      for (int p = 0; p < 6; p++) {
        const uint64_t ad = dtc::smem_desc(xa + PA[p] * YXB + (c * 8 + kk / 8) * YLBO, YLBO, YSBO);
        const uint64_t bd = dtc::smem_desc(wb + PB[p] * YWB + (kk / 8) * 128, 128, 1024);
        dtc::mma_bf16(tmem + 64 * c, ad, bd, idesc, (kk > 0 || p > 0) ? 1u : 0u);
      }
    }
  }
}
}  // namespace

__global__ void __launch_bounds__(YT, 1) k_yconv2d_tc(YconvTc a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) uint64_t bar;
  unsigned char* xs = smem;                        // hi, mid, lo operand tiles
  unsigned char* wf = smem + 3 * YXB;              // forward DFT: hi, mid, lo
  unsigned char* wi = wf + 3 * YWB;                // inverse DFT: hi, mid, lo
  float2* tw = reinterpret_cast<float2*>(wi + 3 * YWB);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warps q and q + 4 share TMEM lane quarter q (kz column q of the CTA);
  // half h of every epilogue's columns goes to warp q + 4h
  const int quarter = warp & 3, half = warp >> 2;
  const int HZ = a.HZ;
  const int kz = blockIdx.x * YKZ + quarter;
  const int row0 = 32 * quarter;               // the quarter's 32 operand rows / TMEM lanes

  if (warp == 0) dtc::tmem_alloc(&tmem_slot, 256);
  if (threadIdx.x == 0) dtc::mbar_init(&bar, 1);
  // the CTA's input, y < 512 of its 4 kz columns and 3 components, staged
  // through the W / twiddle area as lines stg[(c * 4 + kzl) * YSP + y]: a
  // warp's load covers 8 y rows x 4 adjacent kz (32 contiguous bytes each).
  // All of the CTA's global reads (input, W tiles, twiddles) are issued
  // before the first store, so their latencies overlap.
  const int kz0 = blockIdx.x * YKZ;
  const int skz = threadIdx.x & 3, sy = threadIdx.x >> 2;  // staging: kz, y offset (0 .. 63)
  constexpr int NS = 3 * YN * YKZ / YT;                   // staged values per thread
  constexpr int NW = 3 * YWB / 16 / YT;                   // 16-byte words of each W per thread
  constexpr int NTW = YL / YT;                            // twiddles per thread
  static_assert(NS * YT == 3 * YN * YKZ && NW * YT * 16 == 3 * YWB && NTW * YT == YL && YT / 4 * 8 == YN,
                "load partition");
  uint4 wreg[2 * NW];
  float2 treg[NTW];
  {
    float2 sreg[NS];
    const bool in = kz0 + skz < HZ;
#pragma unroll
    for (int u = 0; u < NS; u++) {  // component u / 8, y = 64 (u % 8) + sy
      const int c = u >> 3, y = (u & 7) * 64 + sy;
      sreg[u] = in ? a.S[c * a.CS + (int64_t)y * HZ + kz0 + skz] : make_float2(0.f, 0.f);
    }
    const uint4* s0 = reinterpret_cast<const uint4*>(a.wf);
    const uint4* s1 = reinterpret_cast<const uint4*>(a.wi);
#pragma unroll
    for (int u = 0; u < NW; u++) {
      wreg[u] = __ldg(&s0[threadIdx.x + u * YT]);
      wreg[NW + u] = __ldg(&s1[threadIdx.x + u * YT]);
    }
#pragma unroll
    for (int u = 0; u < NTW; u++) treg[u] = __ldg(&a.tw[threadIdx.x + u * YT]);
    float2* stg = reinterpret_cast<float2*>(wf);
#pragma unroll
    for (int u = 0; u < NS; u++) stg[((u >> 3) * YKZ + skz) * YSP + (u & 7) * 64 + sy] = sreg[u];
  }
  __syncthreads();
  // F1 operand, row (kz, n2 = lane): K = 64 c + 2 n1 (+1), value y[32 n1 + n2]
  // for n1 in this half's 8 of the 16 data rows; n1 >= 16 (K 32 .. 63 of the
  // component, the zero padding) is never read: F1 uses K < 32
  {
    const float2* stg = reinterpret_cast<const float2*>(wf);
    const int n2 = lane;
    const int r = row0 + lane;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2* line = stg + (c * YKZ + quarter) * YSP;
#pragma unroll
      for (int qq = 0; qq < 2; qq++) {
        const int q4 = 2 * half + qq;
        float2 v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) v[q] = line[32 * (4 * q4 + q) + n2];
        put_quad(xs, r, 64 * c + 8 * q4, v);
      }
    }
  }
  __syncthreads();  // staging read before the W tiles overwrite it
  {
    uint4* d0 = reinterpret_cast<uint4*>(wf);
    uint4* d1 = reinterpret_cast<uint4*>(wi);
#pragma unroll
    for (int u = 0; u < NW; u++) {
      d0[threadIdx.x + u * YT] = wreg[u];
      d1[threadIdx.x + u * YT] = wreg[NW + u];
    }
#pragma unroll
    for (int u = 0; u < NTW; u++) tw[threadIdx.x + u * YT] = treg[u];
  }
  dtc::fence_async_smem();
  dtc::fence_before_sync();
  __syncthreads();
  dtc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)row0 << 16);  // the quarter's TMEM lanes
  bool ok = true;
  uint32_t phase = 0;
  auto run_gemm = [&](const unsigned char* w, int kmax) {
    if (threadIdx.x == 0) {
      gemm3(tmem, xs, w, kmax);
      dtc::mma_commit(&bar);
    }
    bool done = dtc::mbar_wait(&bar, phase, WAIT_ITERS);
    phase ^= 1u;
    ok = __syncthreads_and(done && ok);
    dtc::fence_after_sync();
  };
  auto operand_ready = [&]() {
    dtc::tmem_wait_ld();
    dtc::fence_async_smem();
    dtc::fence_before_sync();
    __syncthreads();
    dtc::fence_after_sync();
  };
  // this thread's 32 outputs (16 complex) of component c in its half:
  // columns 64c + 32h .. 64c + 32h + 31 of its lane
  auto read_half = [&](int c, float* v) {
    dtc::tmem_ld32(tl + 64 * c + 32 * half, v);
    dtc::tmem_wait_ld();
  };

  // ---- F1: thread (kz, n2) gets A[k1][n2], k1 in its half ----
  run_gemm(wf, 32);
  if (ok) {
    const int n2 = lane;
    for (int c = 0; c < 3; c++) {
      float v[32];
      read_half(c, v);
      // twiddle W1024^(n2 k1) -> F2 operand row (kz, k1), K = 64 c + 2 n2
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int k1 = 16 * half + j;
        const float2 w = tw[32 * k1 + n2];  // lanes: consecutive n2
        const float zr = v[2 * j], zi = v[2 * j + 1];
        const float2 t = make_float2(fmaf(zr, w.x, -zi * w.y), fmaf(zr, w.y, zi * w.x));
        put_pair(xs, row0 + k1, 64 * c + 2 * n2, t);
      }
    }
  }
  operand_ready();
  // ---- F2: thread (kz, k1) gets the bins k = k1 + 32 k2 of all three
  // components, k2 in its half ----
  if (ok) run_gemm(wf, 64);
  if (ok) {
    const int k1 = lane;
    const float* kline = a.kt + (int64_t)(kz < HZ ? kz : HZ - 1) * KTS;
    float vx[32], vy[32], vz[32];
    dtc::tmem_ld32(tl + 0 * 64 + 32 * half, vx);
    dtc::tmem_ld32(tl + 1 * 64 + 32 * half, vy);
    dtc::tmem_ld32(tl + 2 * 64 + 32 * half, vz);
    dtc::tmem_wait_ld();
    // H = K X (gpu_kernelmul4) -> I1 operand row (kz, k1), K = 64 c + 2 k2
#pragma unroll
    for (int k2q = 0; k2q < 4; k2q++) {
      float2 hx[4], hy[4], hz[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int k2l = 4 * k2q + q;   // index within the half
        const int k2 = 16 * half + k2l;
        const int k = k1 + 32 * k2;
        const bool neg = k > YL / 2;
        const int fy = neg ? YL - k : k;
        const float* kp = kline + fy;  // lanes: consecutive fy
        const float Kxx = __ldg(kp), Kyy = __ldg(kp + a.ktcs), Kzz = __ldg(kp + 2 * a.ktcs);
        float Kyz = __ldg(kp + 3 * a.ktcs);
        if (neg) Kyz = -Kyz;
        const float2 mx = make_float2(vx[2 * k2l], vx[2 * k2l + 1]);
        const float2 my = make_float2(vy[2 * k2l], vy[2 * k2l + 1]);
        const float2 mz = make_float2(vz[2 * k2l], vz[2 * k2l + 1]);
        hx[q] = make_float2(mx.x * Kxx, mx.y * Kxx);
        hy[q] = make_float2(fmaf(mz.x, Kyz, my.x * Kyy), fmaf(mz.y, Kyz, my.y * Kyy));
        hz[q] = make_float2(fmaf(mz.x, Kzz, my.x * Kyz), fmaf(mz.y, Kzz, my.y * Kyz));
      }
      const int kb = 32 * half + 8 * k2q;
      put_quad(xs, row0 + k1, 0 * 64 + kb, hx);
      put_quad(xs, row0 + k1, 1 * 64 + kb, hy);
      put_quad(xs, row0 + k1, 2 * 64 + kb, hz);
    }
  }
  operand_ready();
  // ---- I1: thread (kz, k1) gets (n2) outputs, n2 in its half; twiddle
  // W1024^(-n2 k1) ----
  if (ok) run_gemm(wi, 64);
  if (ok) {
    const int k1 = lane;
    for (int c = 0; c < 3; c++) {
      float v[32];
      read_half(c, v);
      // -> I2 operand row (kz, n2), K = 64 c + 2 k1
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int n2 = 16 * half + j;
        const float2 w = tw[32 * n2 + k1];  // lanes: consecutive k1
        const float zr = v[2 * j], zi = v[2 * j + 1];
        const float2 t = make_float2(fmaf(zr, w.x, zi * w.y), fmaf(zi, w.x, -zr * w.y));  // z conj(w)
        put_pair(xs, row0 + n2, 64 * c + 2 * k1, t);
      }
    }
  }
  operand_ready();
  // ---- I2: thread (kz, n2) gets y = 32 n1 + n2; y < 512 (n1 < 16, the
  // first half of the columns) goes to staging lines in the operand area
  // (free once this GEMM has completed), then out in the same 4-kz-wide
  // rows as the input ----
  if (ok) run_gemm(wi, 64);
  if (ok && half == 0) {
    float2* stg = reinterpret_cast<float2*>(xs);
    const int n2 = lane;
    for (int c = 0; c < 3; c++) {
      float v[32];
      read_half(c, v);
      float2* line = stg + (c * YKZ + quarter) * YSP;
#pragma unroll
      for (int n1 = 0; n1 < 16; n1++) line[32 * n1 + n2] = make_float2(v[2 * n1], v[2 * n1 + 1]);
    }
  }
  __syncthreads();
  if (ok) {
    const float2* stg = reinterpret_cast<const float2*>(xs);
    if (kz0 + skz < HZ) {
#pragma unroll 8
      for (int u = 0; u < NS; u++) {
        const int c = u >> 3, y = (u & 7) * 64 + sy;
        a.S[c * a.CS + (int64_t)y * HZ + kz0 + skz] = stg[(c * YKZ + skz) * YSP + y];
      }
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
  dtc::tmem_wait_ld();
  dtc::fence_before_sync();
  __syncthreads();
  if (warp == 0) dtc::tmem_free(tmem, 256);
}

namespace {
std::mutex g_tw_mu;
float2* g_tw1024[64];
}  // namespace

// Builds the per-device tables (DFT tiles, twiddles) and sets the kernel's
// shared-memory limit; called when a precision-form solver is created, so
// that no allocation happens while its steps are captured into a graph.
static int yconv2d_tc_prepare(const uint16_t** wf, const uint16_t** wi, float2** tw) {
  MMX_CHECK_RC(dft_tables3(wf, 0));
  MMX_CHECK_RC(dft_tables3(wi, 1));
  int dev = 0;
  MMX_TRY(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lock(g_tw_mu);
    if (!g_tw1024[dev]) {
      std::vector<float2> t(YL);  // W1024^(a b) for a, b < 32, row-major
      for (int i = 0; i < YL; i++) {
        double ang = -2.0 * M_PI * (double)(((i >> 5) * (i & 31)) % YL) / YL;
        t[i] = make_float2((float)cos(ang), (float)sin(ang));
      }
      if (cudaMalloc(&g_tw1024[dev], sizeof(float2) * YL) != cudaSuccess) {
        g_tw1024[dev] = nullptr;
        mmx_set_error("out of device memory");
        return MMX_ERR_MEM;
      }
      MMX_TRY(cudaMemcpy(g_tw1024[dev], t.data(), sizeof(float2) * YL, cudaMemcpyHostToDevice));
      MMX_TRY(cudaFuncSetAttribute(k_yconv2d_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)YSMEM));
    }
    *tw = g_tw1024[dev];
  }
  return MMX_OK;
}

// kt[a][kz][fy] = kh[a][fy][kz] for a = Kxx, Kyy, Kzz, Kyz (the first four
// components of the kernel octant), fy <= 512, line pitch KTS
__global__ void k_kernel_kz_major(const float* __restrict__ kh, int64_t kcs, int HZ, float* __restrict__ kt) {
  const int64_t n = 4 * (int64_t)HZ * KTS;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int fy = (int)(e % KTS);
    const int64_t rest = e / KTS;
    const int kz = (int)(rest % HZ), c = (int)(rest / HZ);
    kt[e] = fy <= YL / 2 ? kh[c * kcs + (int64_t)fy * HZ + kz] : 0.f;
  }
}

// The kz-major copy of a 2D film's kernel octant (kh[c][fy][kz], fy <= 512,
// component stride kcs) that the split-precision Y convolution reads:
// 4 x HZ x KTS floats, allocated here, freed by the caller.
int mmx_yconv2d_tc_kernel(const float* kh, int64_t kcs, int HZ, float** kt) {
  if (!kh || !kt || HZ < 1) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  const size_t bytes = sizeof(float) * 4 * (size_t)HZ * KTS;
  if (cudaMalloc(kt, bytes) != cudaSuccess) {
    *kt = nullptr;
    mmx_set_error("out of device memory");
    return MMX_ERR_MEM;
  }
  k_kernel_kz_major<<<296, 256>>>(kh, kcs, HZ, *kt);
  MMX_TRY(cudaGetLastError());
  MMX_TRY(cudaDeviceSynchronize());
  return MMX_OK;
}

int mmx_yconv2d_tc_prepare() {
  const uint16_t *wf, *wi;
  float2* tw;
  return yconv2d_tc_prepare(&wf, &wi, &tw);
}

// Launches the split-precision Y convolution over the spectrum of a 2D film
// with P1 = 1024 and Ny = 512 (kernel kt from mmx_yconv2d_tc_kernel).
int mmx_yconv2d_tc_launch(float2* S, int64_t CS, int HZ, int N1, const float* kt, int* err, cudaStream_t st) {
  if (N1 != YN) { mmx_set_error("split-precision Y convolution: Ny = 512 only"); return MMX_ERR_ARG; }
  const uint16_t *wf = nullptr, *wi = nullptr;
  float2* tw = nullptr;
  MMX_CHECK_RC(yconv2d_tc_prepare(&wf, &wi, &tw));
  YconvTc a;
  a.S = S;
  a.CS = CS;
  a.HZ = HZ;
  a.N1 = N1;
  a.kt = kt;
  a.ktcs = (int64_t)HZ * KTS;
  a.wf = wf;
  a.wi = wi;
  a.tw = tw;
  a.err = err;
  k_yconv2d_tc<<<(HZ + YKZ - 1) / YKZ, YT, YSMEM, st>>>(a);
  MMX_TRY(cudaGetLastError());
  return MMX_OK;
}
