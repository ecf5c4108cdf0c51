// Transforms of any padded size for the drop-in FFT plan (gpuFFT3dPlan_*).
//
// The reference plans its transforms with cufftPlan3d / cufftPlan2d
// (src/gpukern/gpu_fft0.cu:57-68), which accept every size.  The engine's
// zero-aware passes (fft_engine.cu) take padded sizes whose factors are
// 2, 3, 5 and 7; a plan with another prime factor in a padded size, or an
// odd padded Z size, takes this path instead:
//
//   forward  real (N0,N1,N2) -> zero-padded complex box (P0,P1,P2), a
//            complex transform along Z, Y and X, then the half spectrum
//            kz <= P2/2 packed into the reference's (P0,P1,P2+2)-float rows;
//   inverse  the half spectrum unfolded to the full box by Hermitian
//            symmetry, the inverse transforms, the real part of the N box
//            (unnormalised, as the complex-to-real transform).
//
// Each axis pass gathers a chunk of lines into an index-major scratch tile
// T[i][line], transforms the tile's columns with the engine's column pass,
// and scatters the results back.  A line length with a prime factor above
// 7 uses Bluestein's algorithm (L. Bluestein, "A linear filtering approach
// to the computation of discrete Fourier transform", IEEE Trans. Audio
// Electroacoust. 18 (1970) 451-455): with the chirp c_n = exp(-i pi n^2/L),
//   X_k = c_k sum_n (x_n c_n) conj(c_(k-n)),
// a cyclic convolution of length M (a power of two >= 2L - 1) done with two
// power-of-two transforms and the product with the precomputed transform
// of the chirp; the inverse transform is conj(DFT(conj(x))).
#include <math.h>
#include <string.h>

#include <complex>
#include <vector>

#include "fft_passes.cuh"
#include "fft_generic.cuh"

namespace {

constexpr int64_t T_CAP = (int64_t)1 << 23;  // scratch tile, complex elements (64 MB)

// lines of a (P0,P1,P2) complex box along one axis: line l starts at
// (l / inner_n) * outer_stride + (l % inner_n) * inner_stride, elements es apart
struct Lines {
  int64_t n, inner_n, outer_stride, inner_stride, es;
};

Lines lines_of(const int P[3], int axis) {
  Lines r;
  const int64_t P0 = P[0], P1 = P[1], P2 = P[2];
  if (axis == 2) { r.n = P0 * P1; r.inner_n = 1; r.outer_stride = P2; r.inner_stride = 0; r.es = 1; }
  else if (axis == 1) { r.n = P0 * P2; r.inner_n = P2; r.outer_stride = P1 * P2; r.inner_stride = 1; r.es = P2; }
  else { r.n = P1 * P2; r.inner_n = P1 * P2; r.outer_stride = 0; r.inner_stride = 1; r.es = P1 * P2; }
  return r;
}

__device__ __forceinline__ float2 cmul2(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__global__ void k_g_load_real(const float* __restrict__ in, float2* __restrict__ w, int N0, int N1, int N2, int P0,
                              int P1, int P2) {
  const int64_t n = (int64_t)P0 * P1 * P2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int z = (int)(e % P2);
    int64_t r = e / P2;
    int y = (int)(r % P1), x = (int)(r / P1);
    float v = (x < N0 && y < N1 && z < N2) ? in[((int64_t)x * N1 + y) * N2 + z] : 0.f;
    w[e] = make_float2(v, 0.f);
  }
}

__global__ void k_g_gather(const float2* __restrict__ w, float2* __restrict__ T, int L, int len, int64_t nl,
                           int64_t l0, Lines ln, const float2* __restrict__ chirp, int conj) {
  const int64_t n = (int64_t)len * nl;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t l = e % nl;
    int i = (int)(e / nl);
    float2 v = make_float2(0.f, 0.f);
    if (i < L) {
      int64_t g = l0 + l;
      int64_t off = (g / ln.inner_n) * ln.outer_stride + (g % ln.inner_n) * ln.inner_stride;
      v = w[off + (int64_t)i * ln.es];
      if (conj) v.y = -v.y;
      if (chirp) v = cmul2(v, chirp[i]);
    }
    T[e] = v;
  }
}

__global__ void k_g_mul(float2* __restrict__ T, const float2* __restrict__ B, int len, int64_t nl) {
  const int64_t n = (int64_t)len * nl;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    T[e] = cmul2(T[e], B[e / nl]);
}

__global__ void k_g_scatter(float2* __restrict__ w, const float2* __restrict__ T, int L, int64_t nl, int64_t l0,
                            Lines ln, const float2* __restrict__ chirp, int conj, float scale) {
  const int64_t n = (int64_t)L * nl;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t l = e % nl;
    int k = (int)(e / nl);
    float2 v = T[e];
    if (chirp) v = cmul2(v, chirp[k]);
    v.x *= scale;
    v.y *= scale;
    if (conj) v.y = -v.y;
    int64_t g = l0 + l;
    int64_t off = (g / ln.inner_n) * ln.outer_stride + (g % ln.inner_n) * ln.inner_stride;
    w[off + (int64_t)k * ln.es] = v;
  }
}

// half spectrum kz < H into rows of P2 + 2 floats (the reference's buffer)
__global__ void k_g_pack(const float2* __restrict__ w, float* __restrict__ out, int P0, int P1, int P2) {
  const int H = P2 / 2 + 1;
  const int64_t n = (int64_t)P0 * P1 * H;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int kz = (int)(e % H);
    int64_t row = e / H;
    float2 v = w[row * P2 + kz];
    out[row * (P2 + 2) + 2 * kz] = v.x;
    out[row * (P2 + 2) + 2 * kz + 1] = v.y;
  }
}

// full box from the half spectrum: X[x][y][z] = conj X[-x][-y][-z] for z >= H
__global__ void k_g_unpack(const float* __restrict__ in, float2* __restrict__ w, int P0, int P1, int P2) {
  const int H = P2 / 2 + 1;
  const int64_t n = (int64_t)P0 * P1 * P2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int z = (int)(e % P2);
    int64_t r = e / P2;
    int y = (int)(r % P1), x = (int)(r / P1);
    float2 v;
    if (z < H) {
      const float* p = in + r * (P2 + 2) + 2 * z;
      v = make_float2(p[0], p[1]);
    } else {
      int xm = (P0 - x) % P0, ym = (P1 - y) % P1;
      const float* p = in + ((int64_t)xm * P1 + ym) * (P2 + 2) + 2 * (P2 - z);
      v = make_float2(p[0], -p[1]);
    }
    w[e] = v;
  }
}

__global__ void k_g_store_real(const float2* __restrict__ w, float* __restrict__ out, int N0, int N1, int N2, int P1,
                               int P2) {
  const int64_t n = (int64_t)N0 * N1 * N2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int z = (int)(e % N2);
    int64_t r = e / N2;
    int y = (int)(r % N1), x = (int)(r / N1);
    out[e] = w[((int64_t)x * P1 + y) * P2 + z].x;
  }
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)mmx_sm_count() * 8;
  return (int)(b < 1 ? 1 : (b < cap ? b : cap));
}

// radix-2 transform in double (host), sign -1
void host_fft(std::vector<std::complex<double>>& a) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    double ang = -2.0 * M_PI / (double)len;
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; k++) {
        std::complex<double> w(cos(ang * (double)k), sin(ang * (double)k));
        std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

bool smooth(int L) {
  LineFFT f;
  return fft_factor(L, &f);
}

}  // namespace

bool generic_plan_needed(const int N[3], const int P[3]) {
  for (int d = 0; d < 3; d++)
    if (P[d] > 1 && !smooth(P[d])) return true;
  return (P[2] % 2) != 0 || (P[2] / 2 > 1 && !smooth(P[2] / 2));
}

int generic_plan_init(GenericPlan* g, const int N[3], const int P[3]) {
  memset(g, 0, sizeof(*g));
  int64_t box = 1, tneed = 0;
  for (int d = 0; d < 3; d++) {
    g->N[d] = N[d];
    g->P[d] = P[d];
    if (N[d] < 1 || P[d] < N[d]) return MMX_ERR_SIZE;
    box *= P[d];
  }
  for (int d = 0; d < 3; d++) {
    GenericAxis& a = g->ax[d];
    a.L = P[d];
    if (a.L == 1) continue;
    if (fft_factor(a.L, &a.f)) {
      if (a.L > 8192) return MMX_ERR_SIZE;
      a.bluestein = 0;
      a.f.tw = fft_twiddles(a.L);
      a.f.tws = 1;
      if (!a.f.tw) return MMX_ERR_MEM;
      a.len = a.L;
    } else {
      if (a.L > 4096) return MMX_ERR_SIZE;
      a.bluestein = 1;
      int M = 1;
      while (M < 2 * a.L - 1) M <<= 1;
      a.len = M;
      if (!fft_factor(M, &a.f)) return MMX_ERR_SIZE;
      a.f.tw = fft_twiddles(M);
      a.f.tws = 1;
      if (!a.f.tw) return MMX_ERR_MEM;
      // chirp c_n = exp(-i pi n^2 / L), n^2 reduced mod 2L in integers
      std::vector<float2> c(a.L);
      std::vector<std::complex<double>> b(M, 0.0);
      for (int n = 0; n < a.L; n++) {
        long long q = ((long long)n * n) % (2LL * a.L);
        double ang = M_PI * (double)q / (double)a.L;
        c[n] = make_float2((float)cos(ang), (float)-sin(ang));
        std::complex<double> cb(cos(ang), sin(ang));  // conj(c_n)
        b[n] = cb;
        if (n > 0) b[M - n] = cb;
      }
      host_fft(b);
      std::vector<float2> B(M);
      for (int i = 0; i < M; i++) B[i] = make_float2((float)b[i].real(), (float)b[i].imag());
      if (cudaMalloc(&a.chirp, sizeof(float2) * a.L) != cudaSuccess ||
          cudaMalloc(&a.B, sizeof(float2) * M) != cudaSuccess) {
        generic_plan_free(g);
        return MMX_ERR_MEM;
      }
      cudaMemcpy(a.chirp, c.data(), sizeof(float2) * a.L, cudaMemcpyHostToDevice);
      cudaMemcpy(a.B, B.data(), sizeof(float2) * M, cudaMemcpyHostToDevice);
    }
    Lines ln = lines_of(P, d);
    int64_t t = (int64_t)a.len * ln.n;
    if (t > tneed) tneed = t;
  }
  g->tcap = tneed < T_CAP ? tneed : T_CAP;
  if (g->tcap < 8192) g->tcap = 8192;
  if (cudaMalloc(&g->work, sizeof(float2) * (size_t)box) != cudaSuccess ||
      cudaMalloc(&g->T, sizeof(float2) * (size_t)g->tcap) != cudaSuccess) {
    generic_plan_free(g);
    return MMX_ERR_MEM;
  }
  return MMX_OK;
}

void generic_plan_free(GenericPlan* g) {
  for (int d = 0; d < 3; d++) {
    cudaFree(g->ax[d].chirp);
    cudaFree(g->ax[d].B);
    g->ax[d].chirp = g->ax[d].B = nullptr;
  }
  cudaFree(g->work);
  cudaFree(g->T);
  g->work = g->T = nullptr;
}

// one complex transform of every line of the box along 'axis'
static cudaError_t axis_pass(GenericPlan* g, int axis, bool inv, cudaStream_t st) {
  GenericAxis& a = g->ax[axis];
  if (a.L <= 1) return cudaSuccess;
  Lines ln = lines_of(g->P, axis);
  int64_t chunk = g->tcap / a.len;
  if (chunk < 1) chunk = 1;
  for (int64_t l0 = 0; l0 < ln.n; l0 += chunk) {
    int64_t nl = ln.n - l0 < chunk ? ln.n - l0 : chunk;
    ColPass cp;
    memset(&cp, 0, sizeof(cp));
    cp.f = a.f;
    cp.nplanes = 1;
    cp.plane_stride = 0;
    cp.ncols = (int)nl;
    cp.stride_i = nl;
    cp.n_in = a.len;
    cp.n_out = a.len;
    cudaError_t e;
    if (!a.bluestein) {
      k_g_gather<<<grid_for(a.len * nl), 256, 0, st>>>(g->work, g->T, a.L, a.len, nl, l0, ln, nullptr, 0);
      cp.inv = inv ? 1 : 0;
      if ((e = launch_col(g->T, g->T, cp, st)) != cudaSuccess) return e;
      k_g_scatter<<<grid_for(a.L * nl), 256, 0, st>>>(g->work, g->T, a.L, nl, l0, ln, nullptr, 0, 1.f);
    } else {
      k_g_gather<<<grid_for(a.len * nl), 256, 0, st>>>(g->work, g->T, a.L, a.len, nl, l0, ln, a.chirp, inv);
      cp.inv = 0;
      if ((e = launch_col(g->T, g->T, cp, st)) != cudaSuccess) return e;
      k_g_mul<<<grid_for(a.len * nl), 256, 0, st>>>(g->T, a.B, a.len, nl);
      cp.inv = 1;
      if ((e = launch_col(g->T, g->T, cp, st)) != cudaSuccess) return e;
      k_g_scatter<<<grid_for(a.L * nl), 256, 0, st>>>(g->work, g->T, a.L, nl, l0, ln, a.chirp, inv,
                                                      1.f / (float)a.len);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t generic_forward(GenericPlan* g, const float* in, float* out, cudaStream_t st) {
  const int* N = g->N;
  const int* P = g->P;
  int64_t box = (int64_t)P[0] * P[1] * P[2];
  k_g_load_real<<<grid_for(box), 256, 0, st>>>(in, g->work, N[0], N[1], N[2], P[0], P[1], P[2]);
  cudaError_t e = cudaGetLastError();
  for (int d = 2; d >= 0 && e == cudaSuccess; d--) e = axis_pass(g, d, false, st);
  if (e != cudaSuccess) return e;
  k_g_pack<<<grid_for((int64_t)P[0] * P[1] * (P[2] / 2 + 1)), 256, 0, st>>>(g->work, out, P[0], P[1], P[2]);
  return cudaGetLastError();
}

cudaError_t generic_inverse(GenericPlan* g, const float* in, float* out, cudaStream_t st) {
  const int* N = g->N;
  const int* P = g->P;
  int64_t box = (int64_t)P[0] * P[1] * P[2];
  k_g_unpack<<<grid_for(box), 256, 0, st>>>(in, g->work, P[0], P[1], P[2]);
  cudaError_t e = cudaGetLastError();
  for (int d = 0; d < 3 && e == cudaSuccess; d++) e = axis_pass(g, d, true, st);
  if (e != cudaSuccess) return e;
  k_g_store_real<<<grid_for((int64_t)N[0] * N[1] * N[2]), 256, 0, st>>>(g->work, out, N[0], N[1], N[2], P[1], P[2]);
  return cudaGetLastError();
}
