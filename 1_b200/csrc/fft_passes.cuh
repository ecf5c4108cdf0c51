// Pass kernels of the zero-aware padded FFT (see fft_engine.cu).
#pragma once
#include "fft_engine.cuh"

// Rows along Z: real (ld_real floats apart, n_real valid values) <->
// half spectrum (HZ = M + 1 complex values, ld_spec apart).  Row r maps to
// component c, x plane, y row:  r = (c * planes_per_comp + x) *
// rows_per_plane + y.
struct ZPass {
  LineFFT f;               // complex FFT of length M = P2 / 2
  const float2* twP;       // exp(-2 pi i t / P2), t < P2
  int nrows;
  int rows_per_plane;
  int planes_per_comp;
  int ld_real;
  int n_real;              // data values per row (N2)
  int ld_spec;             // HZ
  int64_t plane_stride_spec;
  int64_t comp_stride_real;
  int64_t comp_stride_spec;
};

// Strided columns: line (plane p, column c) has element i at
// p * plane_stride + i * stride_i + c (complex units).  Elements i >= n_in
// are zero; only i < n_out are stored.
struct ColPass {
  LineFFT f;
  int nplanes;
  int64_t plane_stride;
  int ncols;
  int64_t stride_i;
  int n_in;
  int n_out;
  int inv;
};

struct BoxPlan {
  int N[3], P[3], HZ;
  LineFFT fz, fy, fx;
  const float2* twz;
};

__device__ __forceinline__ void zrow_offsets(const ZPass& z, int r, int64_t* roff, int64_t* soff) {
  int per_comp = z.planes_per_comp * z.rows_per_plane;
  int c = r / per_comp;
  int q = r - c * per_comp;
  int x = q / z.rows_per_plane;
  int y = q - x * z.rows_per_plane;
  *roff = c * z.comp_stride_real + (int64_t)q * z.ld_real;
  *soff = c * z.comp_stride_spec + x * z.plane_stride_spec + (int64_t)y * z.ld_spec;
}

// Optional stage combination applied while loading a row: the value
// transformed is  m0 + sum_j (dt a_j) k_j  (the Runge-Kutta stage input of
// src/go/sim/rk.go:316-322, same operation order), also stored to 'out'.
#define ZCOMB_MAXK 7
struct ZComb {
  const float* m0;
  const float* k[ZCOMB_MAXK];
  float a[ZCOMB_MAXK];
  int nk;
  const float* dt;   // device scalar
  float* out;
};

__device__ __forceinline__ float zcomb_value(const ZComb& cb, float dt, int64_t gi) {
  float q = cb.m0[gi];
#pragma unroll
  for (int j = 0; j < ZCOMB_MAXK; j++) {
    if (j >= cb.nk) break;
    if (cb.a[j] == 0.f) continue;
    q = __fadd_rn(q, __fmul_rn(__fmul_rn(dt, cb.a[j]), cb.k[j][gi]));
  }
  return q;
}

// The same for the two adjacent elements gi, gi + 1 (gi even, 8-byte
// aligned rows): 8-byte loads, each component rounded as above.
__device__ __forceinline__ float2 zcomb_value2(const ZComb& cb, float dt, int64_t gi) {
  float2 q = __ldg(reinterpret_cast<const float2*>(cb.m0 + gi));
#pragma unroll
  for (int j = 0; j < ZCOMB_MAXK; j++) {
    if (j >= cb.nk) break;
    if (cb.a[j] == 0.f) continue;
    const float f = __fmul_rn(dt, cb.a[j]);
    const float2 kk = __ldg(reinterpret_cast<const float2*>(cb.k[j] + gi));
    q.x = __fadd_rn(q.x, __fmul_rn(f, kk.x));
    q.y = __fadd_rn(q.y, __fmul_rn(f, kk.y));
  }
  return q;
}

// Forward R2C rows.  Tile: 'lines' rows of M complex values, line-major.
template <int THREADS, int EPT, bool POW2, bool COMB>
__global__ void FFT_BOUNDS(THREADS) k_z_r2c(const float* __restrict__ src, float2* __restrict__ dst, ZPass z,
                                               int lines, ZComb cb) {
  extern __shared__ float2 sm[];
  const int M = z.f.L;
  const int nt = THREADS;
  const int r0 = blockIdx.x * lines;
  const int nl = min(lines, z.nrows - r0);
  // load (x_2n, x_2n+1) pairs, zero beyond the data
  for (int e = threadIdx.x; e < nl * M; e += nt) {
    int l = e / M, n = e - l * M;
    int64_t roff, soff;
    zrow_offsets(z, r0 + l, &roff, &soff);
    int i0 = 2 * n, i1 = 2 * n + 1;
    float a = 0.f, b = 0.f;
    if (COMB) {
      float dt = *cb.dt;
      if (i0 < z.n_real) { a = zcomb_value(cb, dt, roff + i0); cb.out[roff + i0] = a; }
      if (i1 < z.n_real) { b = zcomb_value(cb, dt, roff + i1); cb.out[roff + i1] = b; }
    } else {
      const float* row = src + roff;
      a = i0 < z.n_real ? row[i0] : 0.f;
      b = i1 < z.n_real ? row[i1] : 0.f;
    }
    sm[l * M + n] = make_float2(a, b);
  }
  for (int e = nl * M + threadIdx.x; e < lines * M; e += nt) sm[e] = make_float2(0.f, 0.f);
  __syncthreads();
  tile_fft<EPT, POW2>(sm, z.f, lines, 1, M, false, false);
  // split: X_k = E_k + w^k O_k, k = 0..M
  for (int e = threadIdx.x; e < nl * (M + 1); e += nt) {
    int l = e / (M + 1), k = e - l * (M + 1);
    int64_t roff, soff;
    zrow_offsets(z, r0 + l, &roff, &soff);
    float2 Zk = sm[l * M + (k == M ? 0 : k)];
    float2 Zm = sm[l * M + (k == 0 ? 0 : M - k)];
    float2 E = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    float2 O = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
    float2 w = __ldg(&z.twP[k]);
    float2 wo = cmul(w, O);
    dst[soff + k] = make_float2(E.x + wo.x, E.y + wo.y);
  }
}

// Inverse C2R rows (unnormalised), only the first n_real outputs stored.
template <int THREADS, int EPT, bool POW2>
__global__ void FFT_BOUNDS(THREADS) k_z_c2r(const float2* __restrict__ src, float* __restrict__ dst, ZPass z,
                                               int lines) {
  extern __shared__ float2 sm[];
  const int M = z.f.L;
  const int ld = M + 1;
  const int nt = THREADS;
  const int r0 = blockIdx.x * lines;
  const int nl = min(lines, z.nrows - r0);
  for (int e = threadIdx.x; e < nl * ld; e += nt) {
    int l = e / ld, k = e - l * ld;
    int64_t roff, soff;
    zrow_offsets(z, r0 + l, &roff, &soff);
    float2 v = src[soff + k];
    if (k == 0 || k == M) v.y = 0.f;  // C2R ignores these imaginary parts
    sm[l * ld + k] = v;
  }
  for (int e = nl * ld + threadIdx.x; e < lines * ld; e += nt) sm[e] = make_float2(0.f, 0.f);
  __syncthreads();
  // Z'_k = (X_k + conj X_{M-k}) + i (X_k - conj X_{M-k}) w^{-k}, k < M
  {
    constexpr int IT = EPT;
    float2 v[IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
      int e = it * nt + threadIdx.x;
      if (e < lines * M) {
        int l = e / M, k = e - l * M;
        float2 Xk = sm[l * ld + k], Xm = sm[l * ld + (M - k)];
        float2 A = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
        float2 B = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
        float2 w = __ldg(&z.twP[k]);
        w.y = -w.y;
        float2 C = cmul(B, w);
        v[it] = make_float2(A.x - C.y, A.y + C.x);
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; it++) {
      int e = it * nt + threadIdx.x;
      if (e < lines * M) {
        int l = e / M, k = e - l * M;
        sm[l * ld + k] = v[it];
      }
    }
    __syncthreads();
  }
  tile_fft<EPT, POW2>(sm, z.f, lines, 1, ld, false, true);
  for (int e = threadIdx.x; e < nl * M; e += nt) {
    int l = e / M, n = e - l * M;
    int i0 = 2 * n;
    if (i0 >= z.n_real) continue;
    int64_t roff, soff;
    zrow_offsets(z, r0 + l, &roff, &soff);
    float2 v = sm[l * ld + n];
    float* row = dst + roff;
    row[i0] = v.x;
    if (i0 + 1 < z.n_real) row[i0 + 1] = v.y;
  }
}

// Strided column transform.  Tile: tk adjacent columns x L, index-major.
template <int THREADS, int EPT, bool POW2>
__global__ void FFT_BOUNDS(THREADS) k_col(const float2* src, float2* dst, ColPass cp,
                                             int tk) {
  extern __shared__ float2 sm[];
  const int L = cp.f.L;
  const int nt = THREADS;
  const int c0 = blockIdx.x * tk;
  const int64_t pbase = (int64_t)blockIdx.y * cp.plane_stride + c0;
  const int nc = min(tk, cp.ncols - c0);
  for (int e = threadIdx.x; e < L * tk; e += nt) {
    int i = e / tk, l = e - i * tk;
    float2 v = make_float2(0.f, 0.f);
    if (i < cp.n_in && l < nc) v = src[pbase + i * cp.stride_i + l];
    sm[e] = v;
  }
  __syncthreads();
  tile_fft<EPT, POW2>(sm, cp.f, tk, tk, 1, true, cp.inv != 0);
  for (int e = threadIdx.x; e < cp.n_out * tk; e += nt) {
    int i = e / tk, l = e - i * tk;
    if (l < nc) dst[pbase + i * cp.stride_i + l] = sm[e];
  }
}

// Launch-shape dispatch: tile <= 2048 -> 256 x 8, <= 4096 -> 256 x 16,
// <= 8192 -> 512 x 16; POW2 when the line length is a power of two.
#define SHAPE_DISPATCH(tile, pow2, ...)                                                 \
  do {                                                                                  \
    if ((tile) <= 2048) {                                                               \
      constexpr int T = 256, E = 8;                                                     \
      if (pow2) { constexpr bool P2 = true; __VA_ARGS__; }                              \
      else { constexpr bool P2 = false; __VA_ARGS__; }                                  \
    } else if ((tile) <= 4096) {                                                        \
      constexpr int T = 256, E = 16;                                                    \
      if (pow2) { constexpr bool P2 = true; __VA_ARGS__; }                              \
      else { constexpr bool P2 = false; __VA_ARGS__; }                                  \
    } else if ((tile) <= 8192) {                                                        \
      constexpr int T = 512, E = 16;                                                    \
      if (pow2) { constexpr bool P2 = true; __VA_ARGS__; }                              \
      else { constexpr bool P2 = false; __VA_ARGS__; }                                  \
    } else {                                                                            \
      return cudaErrorInvalidValue;                                                     \
    }                                                                                   \
  } while (0)

template <typename K>
static inline void allow_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_z_r2c(const float* src, float2* dst, const ZPass& zp, cudaStream_t st, const ZComb* cb = nullptr);
cudaError_t launch_z_c2r(const float2* src, float* dst, const ZPass& zp, cudaStream_t st);
cudaError_t launch_col(const float2* src, float2* dst, const ColPass& cp, cudaStream_t st);
int box_plan_init(BoxPlan* p, const int N[3], const int P[3]);
ZPass box_zpass(const BoxPlan* p, int ncomp, int n_x_planes, int64_t comp_stride_real, int64_t comp_stride_spec);
cudaError_t box_forward(const BoxPlan* p, const float* in, float2* spec, cudaStream_t st);
cudaError_t box_inverse(const BoxPlan* p, float2* spec, float* out, cudaStream_t st);
