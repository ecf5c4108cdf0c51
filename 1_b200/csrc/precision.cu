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

// ---------------------------------------------------------------------
// Split-precision Y convolution of a 2D film, P1 = 1024 (Ny = 512).
//
// The 1024-point transform along Y is two layers of 32-point DFTs with the
// index maps n = 32 n1 + n2 and k = k1 + 32 k2 (Cooley-Tukey):
//   F1  A[k1][n2] = sum_n1 W32^(n1 k1) y[32 n1 + n2]     (rows n1 >= 16 are padding: 0)
//   tw  A[k1][n2] *= W1024^(n2 k1)
//   F2  X[k1 + 32 k2] = sum_n2 W32^(n2 k2) A[k1][n2]
// then H = K X per bin (the 2D kernel product of gpu_kernelmul4), and the
// inverse in reverse order, keeping only the outputs y < 512.  Each layer is
// one tensor-core GEMM D[64 x 192] = W[64 x 64] . X[64 x 192] over the 192
// vectors of a CTA (2 kz columns x 3 components x 32), split-BF16 operands,
// FP32 accumulation in TMEM; between layers each thread reads its
// accumulator row back (tcgen05.ld), pairs real and imaginary parts with a
// lane shuffle, applies the twiddle or the kernel product in FP32, and
// writes the next layer's operand tile.
// ---------------------------------------------------------------------
namespace {
constexpr int YT = 128;              // threads
constexpr int YKZ = 2;               // kz columns per CTA
constexpr int YCOLS = 3 * YKZ;       // (component, kz) columns
constexpr int YNV = 32 * YCOLS;      // GEMM N (vectors)
constexpr int YL = 1024;             // padded Y length
constexpr int YWB = 64 * 64 * 2;     // bytes of one W tile
constexpr int YXB = YNV * 64 * 2;    // bytes of one X tile
constexpr size_t YSMEM = 4 * (size_t)YWB + 2 * (size_t)YXB + YL * sizeof(float2);

struct YconvTc {
  float2* S;
  int64_t CS;
  int HZ, N1;
  const float* kh;
  int64_t kcs;
  const uint16_t* wf;
  const uint16_t* wi;
  const float2* tw;  // exp(-2 pi i t / 1024)
  int* err;
};

// (re, im) at K positions 2i, 2i+1 of a vector: adjacent bfloat16s, one
// 32-bit store into each of the hi and lo tiles
__device__ __forceinline__ void put_split2(unsigned char* hi, unsigned char* lo, uint32_t off, float2 v) {
  __nv_bfloat162 h, l;
  dtc::split_bf16(v.x, h.x, l.x);
  dtc::split_bf16(v.y, h.y, l.y);
  *reinterpret_cast<__nv_bfloat162*>(hi + off) = h;
  *reinterpret_cast<__nv_bfloat162*>(lo + off) = l;
}

// (re, im) of this lane's accumulator element and its partner lane's
__device__ __forceinline__ float2 pair_ri(float mine, int ri) {
  float other = __shfl_xor_sync(0xffffffffu, mine, 1);
  return ri ? make_float2(other, mine) : make_float2(mine, other);
}
}  // namespace

__global__ void __launch_bounds__(YT) k_yconv2d_tc(YconvTc a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(8) uint64_t bar;
  unsigned char* wf_hi = smem;
  unsigned char* wf_lo = smem + YWB;
  unsigned char* wi_hi = smem + 2 * YWB;
  unsigned char* wi_lo = smem + 3 * YWB;
  unsigned char* x_hi = smem + 4 * YWB;
  unsigned char* x_lo = smem + 4 * YWB + YXB;
  float2* tw = reinterpret_cast<float2*>(smem + 4 * YWB + 2 * YXB);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kz0 = blockIdx.x * YKZ;
  const int HZ = a.HZ;

  if (warp == 0) dtc::tmem_alloc(&tmem_slot, 256);
  if (threadIdx.x == 0) dtc::mbar_init(&bar, 1);
  {
    const uint4* s0 = reinterpret_cast<const uint4*>(a.wf);
    const uint4* s1 = reinterpret_cast<const uint4*>(a.wi);
    uint4* d0 = reinterpret_cast<uint4*>(wf_hi);
    uint4* d1 = reinterpret_cast<uint4*>(wi_hi);
    for (int i = threadIdx.x; i < 2 * YWB / 16; i += YT) {
      d0[i] = __ldg(&s0[i]);
      d1[i] = __ldg(&s1[i]);
    }
    for (int i = threadIdx.x; i < YL; i += YT) tw[i] = __ldg(&a.tw[i]);
  }
  // F1 operand: vector (col, n2), K index 2 n1 + ri, value y[32 n1 + n2]
  for (int e = threadIdx.x; e < YCOLS * 32 * 32; e += YT) {
    int kzl = e % YKZ;
    int rest = e / YKZ;
    int n2 = rest % 32;
    int n1 = (rest / 32) % 32;
    int c = rest / (32 * 32);
    int y = 32 * n1 + n2, kz = kz0 + kzl;
    float2 v = make_float2(0.f, 0.f);
    if (y < a.N1 && kz < HZ) v = a.S[c * a.CS + (int64_t)y * HZ + kz];
    int vec = 32 * (3 * kzl + c) + n2;
    put_split2(x_hi, x_lo, dtc::kmajor_off(vec, 2 * n1, 64), v);
  }
  const uint32_t tbase = 0;  // set after the allocation is visible
  (void)tbase;
  dtc::fence_async_smem();
  dtc::fence_before_sync();
  __syncthreads();
  dtc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t tw_addr = tmem + ((uint32_t)(32 * warp) << 16);
  const int m = 16 * warp + (lane & 15);  // accumulator row of this lane (lanes >= 16 duplicate)
  const int hi_idx = m >> 1, ri = m & 1;
  bool ok = true;
  uint32_t phase = 0;

  auto run_gemm = [&](const unsigned char* wh, const unsigned char* wl) {
    if (threadIdx.x == 0) {
      dtc::gemm_split<64, YNV>(tmem, wh, wl, x_hi, x_lo);
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

  // ---- F1 ----
  run_gemm(wf_hi, wf_lo);
  // rows: (k1, ri); columns: (col, n2).  twiddle W1024^(n2 k1) -> F2 operand (col, k1) x (n2, ri)
  if (ok) {
    const int k1 = hi_idx;
    for (int c8 = 0; c8 < YNV; c8 += 32) {
      float v[32];
      dtc::tmem_ld32(tw_addr + c8, v);
      dtc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 32; q++) {
        int col = (c8 + q) >> 5, n2 = (c8 + q) & 31;
        float2 z = pair_ri(v[q], ri);
        float2 w = tw[(n2 * k1) & (YL - 1)];
        float2 t = make_float2(fmaf(z.x, w.x, -z.y * w.y), fmaf(z.x, w.y, z.y * w.x));
        if (lane < 16 && ri == 0) put_split2(x_hi, x_lo, dtc::kmajor_off(32 * col + k1, 2 * n2, 64), t);
      }
    }
  }
  operand_ready();
  // ---- F2 ----
  if (ok) run_gemm(wf_hi, wf_lo);
  // rows: (k2, ri); columns: (col, k1); bin k = k1 + 32 k2.  H = K X -> I1 operand (col, k1) x (k2, ri)
  if (ok) {
    const int k2 = hi_idx;
    for (int kzl = 0; kzl < YKZ; kzl++) {
      const int kz = kz0 + kzl;
      const int kzc = kz < HZ ? kz : HZ - 1;
      for (int k1c = 0; k1c < 32; k1c += 8) {
        float v[3][8];
#pragma unroll
        for (int c = 0; c < 3; c++) dtc::tmem_ld8(tw_addr + 32 * (3 * kzl + c) + k1c, v[c]);
        dtc::tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int k1 = k1c + q, k = k1 + 32 * k2;
          float2 mx = pair_ri(v[0][q], ri), my = pair_ri(v[1][q], ri), mz = pair_ri(v[2][q], ri);
          const bool neg = k > YL / 2;
          const int fy = neg ? YL - k : k;
          const float* kp = a.kh + (int64_t)fy * HZ + kzc;
          float Kxx = __ldg(kp), Kyy = __ldg(kp + a.kcs), Kzz = __ldg(kp + 2 * a.kcs), Kyz = __ldg(kp + 3 * a.kcs);
          if (neg) Kyz = -Kyz;
          float2 hx = make_float2(mx.x * Kxx, mx.y * Kxx);
          float2 hy = make_float2(fmaf(mz.x, Kyz, my.x * Kyy), fmaf(mz.y, Kyz, my.y * Kyy));
          float2 hz = make_float2(fmaf(mz.x, Kzz, my.x * Kyz), fmaf(mz.y, Kzz, my.y * Kyz));
          if (lane < 16 && ri == 0) {
            put_split2(x_hi, x_lo, dtc::kmajor_off(32 * (3 * kzl + 0) + k1, 2 * k2, 64), hx);
            put_split2(x_hi, x_lo, dtc::kmajor_off(32 * (3 * kzl + 1) + k1, 2 * k2, 64), hy);
            put_split2(x_hi, x_lo, dtc::kmajor_off(32 * (3 * kzl + 2) + k1, 2 * k2, 64), hz);
          }
        }
      }
    }
  }
  operand_ready();
  // ---- I1 ----
  if (ok) run_gemm(wi_hi, wi_lo);
  // rows: (n2, ri); columns: (col, k1).  twiddle W1024^(-n2 k1) -> I2 operand (col, n2) x (k1, ri)
  if (ok) {
    const int n2 = hi_idx;
    for (int c8 = 0; c8 < YNV; c8 += 32) {
      float v[32];
      dtc::tmem_ld32(tw_addr + c8, v);
      dtc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 32; q++) {
        int col = (c8 + q) >> 5, k1 = (c8 + q) & 31;
        float2 z = pair_ri(v[q], ri);
        float2 w = tw[(n2 * k1) & (YL - 1)];
        // z * conj(w)
        float2 t = make_float2(fmaf(z.x, w.x, z.y * w.y), fmaf(z.y, w.x, -z.x * w.y));
        if (lane < 16 && ri == 0) put_split2(x_hi, x_lo, dtc::kmajor_off(32 * col + n2, 2 * k1, 64), t);
      }
    }
  }
  operand_ready();
  // ---- I2 ----
  if (ok) run_gemm(wi_hi, wi_lo);
  // rows: (n1, ri); columns: (col, n2); y = 32 n1 + n2 < N1 stored
  if (ok && warp < 2) {
    const int n1 = hi_idx;
    for (int c8 = 0; c8 < YNV; c8 += 32) {
      float v[32];
      dtc::tmem_ld32(tw_addr + c8, v);
      dtc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 32; q++) {
        int col = (c8 + q) >> 5, n2 = (c8 + q) & 31;
        float2 z = pair_ri(v[q], ri);
        int c = col % 3, kzl = col / 3;
        int y = 32 * n1 + n2, kz = kz0 + kzl;
        if (lane < 16 && ri == 0 && y < a.N1 && kz < HZ) a.S[c * a.CS + (int64_t)y * HZ + kz] = z;
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
  MMX_CHECK_RC(dft_tables(wf, 0));
  MMX_CHECK_RC(dft_tables(wi, 1));
  int dev = 0;
  MMX_TRY(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lock(g_tw_mu);
    if (!g_tw1024[dev]) {
      std::vector<float2> t(YL);
      for (int i = 0; i < YL; i++) {
        double ang = -2.0 * M_PI * i / YL;
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

int mmx_yconv2d_tc_prepare() {
  const uint16_t *wf, *wi;
  float2* tw;
  return yconv2d_tc_prepare(&wf, &wi, &tw);
}

// Launches the split-precision Y convolution over the spectrum of a 2D film
// with P1 = 1024 (kernel octant kh[4][513][HZ], component stride kcs).
int mmx_yconv2d_tc_launch(float2* S, int64_t CS, int HZ, int N1, const float* kh, int64_t kcs, int* err,
                          cudaStream_t st) {
  const uint16_t *wf = nullptr, *wi = nullptr;
  float2* tw = nullptr;
  MMX_CHECK_RC(yconv2d_tc_prepare(&wf, &wi, &tw));
  YconvTc a;
  a.S = S;
  a.CS = CS;
  a.HZ = HZ;
  a.N1 = N1;
  a.kh = kh;
  a.kcs = kcs;
  a.wf = wf;
  a.wi = wi;
  a.tw = tw;
  a.err = err;
  k_yconv2d_tc<<<(HZ + YKZ - 1) / YKZ, YT, YSMEM, st>>>(a);
  MMX_TRY(cudaGetLastError());
  return MMX_OK;
}
