// Fused LLG solver (extended mmx_* ABI).
//
// One effective-field evaluation of an (N0,N1,N2) grid padded to
// (P0,P1,P2) runs as
//   3D: Zf -> Yf -> Xconv -> Yi -> Zi+epilogue        (5 kernels)
//   2D: Zf -> Yconv -> Zi+epilogue                     (3 kernels)
// over one spectrum buffer S[3][N0][P1][HZ] (complex, HZ = P2/2 + 1):
//  * Zf  : R2C of the magnetisation rows, all three components (zero
//          padding in Z implicit, only the N0 x N1 data rows exist);
//  * Yf  : column FFT of the N1 data rows of each (component, x) plane;
//  * Xconv: for each (ky, kz) column, forward X FFT of the N0 data planes,
//          multiplication by the symmetric demag(+exchange) kernel and
//          inverse X FFT, writing only the N0 planes the next pass reads
//          (in 2D the Y transform plays this role);
//  * Yi  : inverse column FFT, only the N1 output rows are stored;
//  * Zi+epilogue: C2R of the three components of a row in shared memory,
//          then the local fields, the LLG torque and the solver stage
//          update per cell (Heun predictor/corrector, RK stage, or just
//          the field).
// The kernel spectrum is real; it is stored as one octant (kx <= P0/2,
// ky <= P1/2, all kz) and unfolded with the parity of each component
// (diagonal components even, XY odd in kx,ky, XZ odd in kx, YZ odd in ky).
#include <math.h>
#include <string.h>
#include <string>
#include <vector>

#include "demag_gpu.cuh"
#include "fft_passes.cuh"
#include "llg_ops.cuh"
#include "epilogue.cuh"
#include "kernmul.cuh"
#include "fft_fixed_kernels.cuh"
#include "solver_state.cuh"
#include "../../include/mmx.h"

static thread_local std::string g_err = "";
void mmx_set_error(const char* msg) { g_err = msg ? msg : ""; }
extern "C" const char* mmx_last_error(void) { return g_err.c_str(); }

int mmx_sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// ---------------------------------------------------------------------
// Kernel octant extraction (the octant layout is in kernmul.cuh)
// ---------------------------------------------------------------------
__global__ void k_extract_octant(const float2* __restrict__ spec, float* __restrict__ kh, int O0, int O1, int P1,
                                 int HZ, float norm) {
  int64_t n = (int64_t)O0 * O1 * HZ;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int kz = (int)(e % HZ);
    int ky = (int)((e / HZ) % O1);
    int kx = (int)(e / ((int64_t)HZ * O1));
    kh[e] = __fmul_rn(spec[((int64_t)kx * P1 + ky) * HZ + kz].x, norm);
  }
}

// ---------------------------------------------------------------------
// Xconv (3D): columns (ky, kz) flattened, tile of tk columns x 3 comps.
// Tile layout: element x of line (c, t) at sm[x * 3tk + c * tk + t].
// ---------------------------------------------------------------------
template <int THREADS, int EPT, bool POW2>
__global__ void FFT_BOUNDS(THREADS) k_xconv(float2* __restrict__ S, LineFFT fx, KernOct K, int N0, int P1, int HZ,
                                               int64_t CS, int tk) {
  extern __shared__ float2 sm[];
  const int P0 = fx.L;
  const int ncol = P1 * HZ;
  const int col0 = blockIdx.x * tk;
  const int nc = min(tk, ncol - col0);
  const int nl = 3 * tk;
  const int64_t plane = (int64_t)P1 * HZ;
  for (int e = threadIdx.x; e < P0 * nl; e += THREADS) {
    int i = e / nl, l = e - i * nl;
    int c = l / tk, t = l - c * tk;
    float2 v = make_float2(0.f, 0.f);
    if (i < N0 && t < nc) v = S[c * CS + i * plane + col0 + t];
    sm[e] = v;
  }
  __syncthreads();
  tile_fft<EPT, POW2>(sm, fx, nl, nl, 1, true, false);
  for (int e = threadIdx.x; e < P0 * tk; e += THREADS) {
    int kx = e / tk, t = e - kx * tk;
    if (t >= nc) continue;
    int col = col0 + t;
    int ky = col / HZ, kz = col - ky * HZ;
    float Kxx, Kyy, Kzz, Kyz, Kxz, Kxy;
    kern_at(K, kx, ky, kz, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
    float2* b = sm + kx * nl + t;
    float2 mx = b[0], my = b[tk], mz = b[2 * tk];
    kmul6(mx, my, mz, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
    b[0] = mx;
    b[tk] = my;
    b[2 * tk] = mz;
  }
  __syncthreads();
  tile_fft<EPT, POW2>(sm, fx, nl, nl, 1, true, true);
  for (int e = threadIdx.x; e < N0 * nl; e += THREADS) {
    int i = e / nl, l = e - i * nl;
    int c = l / tk, t = l - c * tk;
    if (t < nc) S[c * CS + i * plane + col0 + t] = sm[e];
  }
}

// Yconv (2D, N0 = P0 = 1): columns kz, tile of tk columns x 3 comps.
template <int THREADS, int EPT, bool POW2>
__global__ void FFT_BOUNDS(THREADS) k_yconv2d(float2* __restrict__ S, LineFFT fy, KernOct K, int N1, int HZ,
                                                 int64_t CS, int tk) {
  extern __shared__ float2 sm[];
  const int P1 = fy.L;
  const int kz0 = blockIdx.x * tk;
  const int nc = min(tk, HZ - kz0);
  const int nl = 3 * tk;
  for (int e = threadIdx.x; e < P1 * nl; e += THREADS) {
    int i = e / nl, l = e - i * nl;
    int c = l / tk, t = l - c * tk;
    float2 v = make_float2(0.f, 0.f);
    if (i < N1 && t < nc) v = S[c * CS + (int64_t)i * HZ + kz0 + t];
    sm[e] = v;
  }
  __syncthreads();
  tile_fft<EPT, POW2>(sm, fy, nl, nl, 1, true, false);
  for (int e = threadIdx.x; e < P1 * tk; e += THREADS) {
    int ky = e / tk, t = e - ky * tk;
    if (t >= nc) continue;
    float Kxx, Kyy, Kzz, Kyz, Kxz, Kxy;
    kern_at(K, 0, ky, kz0 + t, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
    float2* b = sm + ky * nl + t;
    float2 mx = b[0], my = b[tk], mz = b[2 * tk];
    kmul4(mx, my, mz, Kxx, Kyy, Kzz, Kyz);
    b[0] = mx;
    b[tk] = my;
    b[2 * tk] = mz;
  }
  __syncthreads();
  tile_fft<EPT, POW2>(sm, fy, nl, nl, 1, true, true);
  for (int e = threadIdx.x; e < N1 * nl; e += THREADS) {
    int i = e / nl, l = e - i * nl;
    int c = l / tk, t = l - c * tk;
    if (t < nc) S[c * CS + (int64_t)i * HZ + kz0 + t] = sm[e];
  }
}

// ---------------------------------------------------------------------
// Zi + epilogue: inverse Z (C2R) of the three components of R rows in
// shared memory, then the per-cell solver update.
// ---------------------------------------------------------------------
template <int THREADS, int EPT, bool POW2, int MODE>
__global__ void FFT_BOUNDS(THREADS) k_zinv_epi(const float2* __restrict__ S, LineFFT fz,
                                                  const float2* __restrict__ twP, int N0, int P1, int HZ, int64_t CS,
                                                  int rows, int nrows_total, EpiArgs ea) {
  extern __shared__ float2 sm[];
  const int M = fz.L;
  const int ld = M + 1;
  const int nl = 3 * rows;
  const int nt = THREADS;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, nrows_total - r0);
  const int N1 = ea.N1, N2 = ea.N2;
  for (int e = threadIdx.x; e < nl * ld; e += nt) {
    int l = e / ld, k = e - l * ld;
    int r = l / 3, c = l - 3 * r;
    float2 v = make_float2(0.f, 0.f);
    if (r < nr) {
      int gr = r0 + r;
      int x = gr / N1, y = gr - x * N1;
      v = S[c * CS + ((int64_t)x * P1 + y) * HZ + k];
      if (k == 0 || k == M) v.y = 0.f;
    }
    sm[e] = v;
  }
  __syncthreads();
  {
    float2 v[EPT];
#pragma unroll
    for (int it = 0; it < EPT; it++) {
      int e = it * nt + threadIdx.x;
      if (e < nl * M) {
        int l = e / M, k = e - l * M;
        float2 Xk = sm[l * ld + k], Xm = sm[l * ld + (M - k)];
        float2 A = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
        float2 B = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
        float2 w = __ldg(&twP[k]);
        w.y = -w.y;
        float2 C = cmul(B, w);
        v[it] = make_float2(A.x - C.y, A.y + C.x);
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < EPT; it++) {
      int e = it * nt + threadIdx.x;
      if (e < nl * M) {
        int l = e / M, k = e - l * M;
        sm[l * ld + k] = v[it];
      }
    }
    __syncthreads();
  }
  tile_fft<EPT, POW2>(sm, fz, nl, 1, ld, false, true);

  float lmax = 0.f;
  double eacc = 0.0;
  for (int e = threadIdx.x; e < nr * N2; e += nt) {
    int r = e / N2, z = e - r * N2;
    int64_t g = (int64_t)(r0 + r) * N2 + z;
    const float2* base = sm + (r * 3) * ld + (z >> 1);
    float hx = (z & 1) ? base[0].y : base[0].x;
    float hy = (z & 1) ? base[ld].y : base[ld].x;
    float hz = (z & 1) ? base[2 * ld].y : base[2 * ld].x;
    epi_cell<MODE>(ea, g, hx, hy, hz, lmax, &eacc);
  }
  epi_flush_max<MODE>(ea, lmax, eacc);
}

// ---------------------------------------------------------------------
// Small helper kernels
// ---------------------------------------------------------------------
__global__ void k_normalize3(float* __restrict__ m, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = m[i], y = m[n + i], z = m[2 * n + i];
    llg_normalize(x, y, z);
    m[i] = x;
    m[n + i] = y;
    m[2 * n + i] = z;
  }
}

// maxabs of a 3n vector into *out (out must be zeroed first)
__global__ void k_maxabs(const float* __restrict__ a, int64_t n, float* out) {
  float v = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v = fmaxf(v, fabsf(a[i]));
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, v);
}

// ---------------------------------------------------------------------
// Solver object
// ---------------------------------------------------------------------
static void set_tableau(mmx_solver* s) {
  memset(s->a, 0, sizeof(s->a));
  memset(s->b, 0, sizeof(s->b));
  memset(s->b2, 0, sizeof(s->b2));
  memset(s->c, 0, sizeof(s->c));
  s->fsal = 0;
  s->adaptive = 0;
  switch (s->p.solver) {
    case MMX_SOLVER_RK2:
    case MMX_SOLVER_RK12:
      s->stages = 2;
      s->c[1] = 1.f; s->a[1][0] = 1.f; s->b[0] = .5f; s->b[1] = .5f;
      if (s->p.solver == MMX_SOLVER_RK12) { s->adaptive = 1; s->errorder = 1.; s->b2[0] = 1.f; }
      break;
    case MMX_SOLVER_RK23:
      s->stages = 4; s->fsal = 1;
      s->c[1] = (float)(1. / 2.); s->c[2] = (float)(3. / 4.); s->c[3] = 1.f;
      s->a[1][0] = (float)(1. / 2.);
      s->a[2][1] = (float)(3. / 4.);
      s->a[3][0] = (float)(2. / 9.); s->a[3][1] = (float)(1. / 3.); s->a[3][2] = (float)(4. / 9.);
      s->b[0] = (float)(2. / 9.); s->b[1] = (float)(1. / 3.); s->b[2] = (float)(4. / 9.);
      s->adaptive = 1; s->errorder = 2.;
      s->b2[0] = (float)(7. / 24); s->b2[1] = (float)(1. / 4.); s->b2[2] = (float)(1. / 3.); s->b2[3] = (float)(1. / 8.);
      break;
    case MMX_SOLVER_RK4:
      s->stages = 4;
      s->c[1] = .5f; s->c[2] = .5f; s->c[3] = 1.f;
      s->a[1][0] = .5f; s->a[2][1] = .5f; s->a[3][2] = 1.f;
      s->b[0] = (float)(1. / 6.); s->b[1] = (float)(1. / 3.); s->b[2] = (float)(1. / 3.); s->b[3] = (float)(1. / 6.);
      break;
    case MMX_SOLVER_RKCK: {
      s->stages = 6;
      double c[6] = {0., 1. / 5., 3. / 10., 3. / 5., 1., 7. / 8.};
      double a[6][6] = {{0}, {1. / 5.}, {3. / 40., 9. / 40.}, {3. / 10., -9. / 10., 6. / 5.},
                        {-11. / 54., 5. / 2., -70. / 27., 35. / 27.},
                        {1631. / 55296., 175. / 512., 575. / 13824., 44275. / 110592., 253. / 4096.}};
      double b[6] = {37. / 378., 0, 250. / 621., 125. / 594., 0, 512. / 1771.};
      double b2[6] = {2825. / 27648., 0, 18575. / 48384., 13525. / 55296., 277. / 14336., 1. / 4.};
      for (int i = 0; i < 6; i++) {
        s->c[i] = (float)c[i]; s->b[i] = (float)b[i]; s->b2[i] = (float)b2[i];
        for (int j = 0; j < 6; j++) s->a[i][j] = (float)a[i][j];
      }
      s->adaptive = 1; s->errorder = 4.;
      break;
    }
    case MMX_SOLVER_RKDP: {
      s->stages = 7; s->fsal = 1;
      double c[7] = {0., 1. / 5., 3. / 10., 4. / 5., 8. / 9., 1., 1.};
      double a[7][7] = {{0}, {1. / 5.}, {3. / 40., 9. / 40.}, {44. / 45., -56. / 15., 32. / 9.},
                        {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.},
                        {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.},
                        {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.}};
      double b[7] = {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0};
      double b2[7] = {5179. / 57600., 0., 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100., 1. / 40.};
      for (int i = 0; i < 7; i++) {
        s->c[i] = (float)c[i]; s->b[i] = (float)b[i]; s->b2[i] = (float)b2[i];
        for (int j = 0; j < 7; j++) s->a[i][j] = (float)a[i][j];
      }
      s->adaptive = 1; s->errorder = 4.;
      break;
    }
    default:
      s->stages = 0;
  }
}

// ------------------------------ launches ------------------------------
static PassTimer* timer_for(mmx_solver* s, const char* name) {
  for (auto& t : s->timers)
    if (t.name == name) return &t;
  s->timers.push_back(PassTimer());
  s->timers.back().name = name;
  return &s->timers.back();
}

struct ScopedPass {
  mmx_solver* s;
  cudaStream_t st;
  PassTimer* t = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  const char* nm = nullptr;
  ScopedPass(mmx_solver* s_, const char* name, cudaStream_t st_) : s(s_), st(st_) {
    if (s->capture_events) {
      // inside the capture of the profiling graph: event-record nodes,
      // chained (a pass starts at the previous pass's end event) so a step
      // of n passes carries n + 1 event nodes
      nm = name;
      cudaEventCreate(&b);
      if (s->gevents.empty()) {
        cudaEventCreate(&a);
        cudaEventRecordWithFlags(a, st, cudaEventRecordExternal);
      } else {
        a = s->gevents.back().b;
      }
      return;
    }
    if (!s->profile) return;
    t = timer_for(s, name);
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  ~ScopedPass() {
    if (nm) {
      cudaEventRecordWithFlags(b, st, cudaEventRecordExternal);
      s->gevents.push_back({nm, a, b, s->gevents.empty()});
      return;
    }
    if (!t) return;
    cudaEventRecord(b, st);
    t->pending.push_back({a, b});
    t->launches++;
  }
};

static void flush_timers(mmx_solver* s) {
  for (auto& t : s->timers) {
    for (auto& pr : t.pending) {
      cudaEventSynchronize(pr.second);
      float ms = 0;
      cudaEventElapsedTime(&ms, pr.first, pr.second);
      t.ms += ms;
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    t.pending.clear();
  }
}

static cudaError_t launch_xconv(mmx_solver* s, cudaStream_t st) {
  int P0 = s->P[0];
  if (fx_ok(P0)) {
    ConvArgs a;
    a.S = s->S;
    a.K = s->K;
    a.n_data = s->N[0];
    a.ncols = s->P[1] * s->HZ;
    a.HZ = s->HZ;
    a.stride = (int64_t)s->P[1] * s->HZ;
    a.CS = s->CS;
    a.tw = s->bp.fx.tw;
    a.tws = s->bp.fx.tws;
    ScopedPass sp(s, "xconv", st);
    switch (P0) {
#define C_(L) \
  case L: return fx_launch_conv<L, false>(a, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int tk = 1;
  while (tk < 32 && P0 * 3 * tk * 2 <= (is_pow2(P0) ? 4096 : 2048)) tk *= 2;
  size_t smem = sizeof(float2) * (size_t)P0 * 3 * tk;
  int ncol = s->P[1] * s->HZ;
  ScopedPass sp(s, "xconv", st);
  SHAPE_DISPATCH(P0 * 3 * tk, is_pow2(P0), {
    allow_smem(k_xconv<T, E, P2>, smem);
    k_xconv<T, E, P2><<<div_up(ncol, tk), T, smem, st>>>(s->S, s->bp.fx, s->K, s->N[0], s->P[1], s->HZ, s->CS, tk);
  });
  return cudaGetLastError();
}

int mmx_yconv2d_tc_launch(float2* S, int64_t CS, int HZ, int N1, const float* kt, int* err, cudaStream_t st);
int mmx_yconv2d_tc_prepare();
int mmx_yconv2d_tc_kernel(const float* kh, int64_t kcs, int HZ, float** kt);

static cudaError_t launch_yconv2d(mmx_solver* s, cudaStream_t st) {
  int P1 = s->P[1];
  if (s->p.precision) {
    ScopedPass sp(s, "yconv2d_tc", st);
    int rc = mmx_yconv2d_tc_launch(s->S, s->CS, s->HZ, s->N[1], s->kt_tc, reinterpret_cast<int*>(s->scratch + 15),
                                   st);
    return rc == MMX_OK ? cudaSuccess : cudaErrorLaunchFailure;
  }
  if (fx_ok(P1)) {
    ConvArgs a;
    a.S = s->S;
    a.K = s->K;
    a.n_data = s->N[1];
    a.ncols = s->HZ;
    a.HZ = s->HZ;
    a.stride = s->HZ;
    a.CS = s->CS;
    a.tw = s->bp.fy.tw;
    a.tws = s->bp.fy.tws;
    ScopedPass sp(s, "yconv2d", st);
    switch (P1) {
#define C_(L) \
  case L: return fx_launch_conv<L, true>(a, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int tk = 1;
  while (tk < 32 && P1 * 3 * tk * 2 <= (is_pow2(P1) ? 4096 : 2048) && tk * 2 <= s->HZ) tk *= 2;
  size_t smem = sizeof(float2) * (size_t)P1 * 3 * tk;
  ScopedPass sp(s, "yconv2d", st);
  SHAPE_DISPATCH(P1 * 3 * tk, is_pow2(P1), {
    allow_smem(k_yconv2d<T, E, P2>, smem);
    k_yconv2d<T, E, P2><<<div_up(s->HZ, tk), T, smem, st>>>(s->S, s->bp.fy, s->K, s->N[1], s->HZ, s->CS, tk);
  });
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_zinv(mmx_solver* s, const EpiArgs& ea, cudaStream_t st) {
  int M = s->P[2] / 2;
  int nrows = s->N[0] * s->N[1];
  if (fx_ok(M)) {
    ScopedPass sp(s, "zinv_epi", st);
    switch (M) {
#define C_(L) \
  case L: return fx_launch_zinv<L, MODE>(s->S, s->bp.twz, s->bp.twz, s->P[1], s->HZ, s->CS, nrows, ea, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int rows = 1;
  while (3 * (rows * 2) * (M + 1) <= (is_pow2(M) ? 4096 : 2048) && rows * 2 <= nrows) rows *= 2;
  size_t smem = sizeof(float2) * (size_t)3 * rows * (M + 1);
  ScopedPass sp(s, "zinv_epi", st);
  SHAPE_DISPATCH(3 * rows * (M + 1), is_pow2(M), {
    allow_smem(k_zinv_epi<T, E, P2, MODE>, smem);
    k_zinv_epi<T, E, P2, MODE><<<div_up(nrows, rows), T, smem, st>>>(s->S, s->bp.fz, s->bp.twz, s->N[0], s->P[1],
                                                                        s->HZ, s->CS, rows, nrows, ea);
  });
  return cudaGetLastError();
}

// inverse Z + Heun epilogue + the next evaluation's forward Z in one pass
template <int MODE>
static cudaError_t launch_zinv_fwd(mmx_solver* s, const EpiArgs& ea, cudaStream_t st) {
  int M = s->P[2] / 2;
  int nrows = s->N[0] * s->N[1];
  ScopedPass sp(s, "zinv_epi_zfwd", st);
  switch (M) {
#define C_(L) \
  case L: return fx_launch_zinv_fwd<L, MODE>(s->S, s->bp.twz, s->bp.twz, s->P[1], s->HZ, s->CS, nrows, ea, st);
    FX_SIZES(C_)
#undef C_
  }
  return cudaErrorInvalidValue;
}

// Fixed-step Heun with an open Z boundary and a compiled Z length: each
// inverse-Z epilogue also produces the next evaluation's forward Z, so the
// spectrum buffer holds zfwd(m) between steps (spec_ready).
static bool heun_fused(const mmx_solver* s) {
  int M = s->P[2] / 2;
  return s->p.solver == MMX_SOLVER_HEUN && s->p.max_error == 0.f && s->N[2] == M && s->p.periodic[2] == 0 &&
         fx_ok(M);
}

static cudaError_t conv_rest(mmx_solver* s, cudaStream_t st);

static cudaError_t zfwd_only(mmx_solver* s, const float* m, cudaStream_t st) {
  ZPass z = box_zpass(&s->bp, 3, s->N[0], s->n, s->CS);
  ScopedPass sp(s, "zfwd", st);
  return launch_z_r2c(m, s->S, z, st);
}

// forward part of the field evaluation: m -> S (after the kernel multiply)
static cudaError_t conv_front(mmx_solver* s, const float* m, cudaStream_t st) {
  cudaError_t e = zfwd_only(s, m, st);
  if (e != cudaSuccess) return e;
  return conv_rest(s, st);
}

// the passes after the forward Z: Y / kernel product (X) / inverse Y
static cudaError_t conv_rest(mmx_solver* s, cudaStream_t st) {
  cudaError_t e;
  if (s->is2d) return launch_yconv2d(s, st);
  {
    ColPass y;
    y.f = s->bp.fy;
    y.nplanes = 3 * s->N[0];
    y.plane_stride = (int64_t)s->P[1] * s->HZ;
    y.ncols = s->HZ;
    y.stride_i = s->HZ;
    y.n_in = s->N[1];
    y.n_out = s->P[1];
    y.inv = 0;
    ScopedPass sp(s, "yfwd", st);
    e = launch_col(s->S, s->S, y, st);
    if (e != cudaSuccess) return e;
  }
  e = launch_xconv(s, st);
  if (e != cudaSuccess) return e;
  {
    ColPass y;
    y.f = s->bp.fy;
    y.nplanes = 3 * s->N[0];
    y.plane_stride = (int64_t)s->P[1] * s->HZ;
    y.ncols = s->HZ;
    y.stride_i = s->HZ;
    y.n_in = s->P[1];
    y.n_out = s->N[1];
    y.inv = 1;
    ScopedPass sp(s, "yinv", st);
    e = launch_col(s->S, s->S, y, st);
  }
  return e;
}

EpiArgs solver_base_args(mmx_solver* s) {
  EpiArgs ea;
  memset(&ea, 0, sizeof(ea));
  ea.N1 = s->N[1];
  ea.N2 = s->N[2];
  ea.n = s->n;
  for (int d = 0; d < 3; d++) {
    ea.lf.hext[d] = s->p.hext[d];
    ea.lf.u[d] = s->p.anis_axis[d];
  }
  ea.lf.anis = s->p.anis_type;
  ea.lf.K = s->p.anis_k;
  ea.alpha = s->p.alpha;
  return ea;
}

// ------------------------------ steps ---------------------------------
static cudaError_t heun_step(mmx_solver* s, cudaStream_t st) {
  // dtGilbert = dt / (1 + alpha^2)   (torque.go:49-51)
  float dtg = f32_div(s->dt, f32_add(1.f, f32_mul(s->p.alpha, s->p.alpha)));
  cudaError_t e;
  EpiArgs ea = solver_base_args(s);
  ea.dtg = dtg;
  const bool fused = heun_fused(s);
  // predictor
  if (!fused || !s->spec_ready) {
    e = zfwd_only(s, s->m, st);
    if (e != cudaSuccess) return e;
  }
  e = conv_rest(s, st);
  if (e != cudaSuccess) return e;
  ea.m_in = s->m;
  ea.out0 = s->t0;
  ea.out1 = s->m1;
  e = fused ? launch_zinv_fwd<EPI_HEUN1>(s, ea, st) : launch_zinv<EPI_HEUN1>(s, ea, st);
  if (e != cudaSuccess) return e;
  // corrector
  if (!fused) {
    e = zfwd_only(s, s->m1, st);
    if (e != cudaSuccess) return e;
  }
  e = conv_rest(s, st);
  if (e != cudaSuccess) return e;
  ea.m_in = s->m1;
  ea.aux0 = s->t0;
  ea.aux1 = s->m;
  ea.out0 = s->m;
  ea.out1 = nullptr;
  ea.err = s->p.max_error != 0.f ? s->scratch : nullptr;
  if (ea.err) {
    e = cudaMemsetAsync(s->scratch, 0, sizeof(float), st);
    if (e != cudaSuccess) return e;
  }
  e = fused ? launch_zinv_fwd<EPI_HEUN2>(s, ea, st) : launch_zinv<EPI_HEUN2>(s, ea, st);
  s->spec_ready = fused ? 1 : 0;
  return e;
}

// RK stage i: combine the stage input, transform, torque epilogue.
static cudaError_t rk_stage(mmx_solver* s, int i, cudaStream_t st, float* dt_dev) {
  cudaError_t e;
  const float* src = s->m;
  ZComb cb;
  memset(&cb, 0, sizeof(cb));
  bool comb = false;
  for (int j = 0; j < s->stages; j++)
    if (s->a[i][j] != 0.f) comb = true;
  ZPass z = box_zpass(&s->bp, 3, s->N[0], s->n, s->CS);
  if (comb) {
    cb.m0 = s->m;
    for (int j = 0; j < s->stages; j++) { cb.k[j] = s->kb[j]; cb.a[j] = s->a[i][j]; }
    cb.nk = s->stages;
    cb.dt = dt_dev;
    cb.out = s->m1;
    src = s->m1;
  }
  {
    ScopedPass sp(s, "zfwd", st);
    e = launch_z_r2c(s->m, s->S, z, st, comb ? &cb : nullptr);
    if (e != cudaSuccess) return e;
  }
  // remaining passes of the field evaluation
  if (s->is2d) {
    e = launch_yconv2d(s, st);
  } else {
    ColPass y;
    y.f = s->bp.fy;
    y.nplanes = 3 * s->N[0];
    y.plane_stride = (int64_t)s->P[1] * s->HZ;
    y.ncols = s->HZ;
    y.stride_i = s->HZ;
    y.n_in = s->N[1];
    y.n_out = s->P[1];
    y.inv = 0;
    {
      ScopedPass sp(s, "yfwd", st);
      e = launch_col(s->S, s->S, y, st);
    }
    if (e != cudaSuccess) return e;
    e = launch_xconv(s, st);
    if (e != cudaSuccess) return e;
    y.n_in = s->P[1];
    y.n_out = s->N[1];
    y.inv = 1;
    {
      ScopedPass sp(s, "yinv", st);
      e = launch_col(s->S, s->S, y, st);
    }
  }
  if (e != cudaSuccess) return e;
  EpiArgs ea = solver_base_args(s);
  ea.dtg = f32_div(1.f, f32_add(1.f, f32_mul(s->p.alpha, s->p.alpha)));  // Torque = DeltaM(dt=1)
  ea.m_in = src;
  ea.dt_dev = dt_dev;
  for (int j = 0; j < s->stages; j++) ea.kbuf[j] = s->kb[j];
  ea.stage = i;
  if (s->noise_sigma != 0.f) {
    ea.lf.sigma = s->noise_sigma;
    ea.lf.seed = s->p.thermal_seed;
    ea.lf.step_lo = (unsigned int)s->noise_step;
    ea.lf.step_hi = (unsigned int)((unsigned long long)s->noise_step >> 32);
  }
  // calcHeffEnergy at the last stage (FSAL) or the first (rk.go:321-337)
  if (s->want_energy && s->eacc && (s->fsal ? i == s->stages - 1 : i == 0)) ea.energy = s->eacc;
  if (i == s->stages - 1) {
    // last stage: k_last, then m_high (b) and, if adaptive, m_low (b2)
    ea.out0 = s->kb[i];
    ea.aux0 = s->m;
    ea.out1 = s->mnew;
    ea.rk.nk = s->stages;
    for (int j = 0; j < s->stages; j++) { ea.rk.a[j] = s->b[j]; ea.rk.b2[j] = s->b2[j]; }
    ea.rk.final_stage = 1;
    ea.rk.adaptive = s->adaptive;
    ea.err = s->adaptive ? s->scratch : nullptr;
    // the precision form keeps float64 for the embedded error norm
    if (s->p.precision && s->adaptive) return launch_zinv<EPI_RK64>(s, ea, st);
    return launch_zinv<EPI_RK>(s, ea, st);
  }
  ea.out0 = s->kb[i];
  if (i == 0) ea.err = s->scratch + 1;  // max |k0|: the reference's 'torque'
  return launch_zinv<EPI_TORQUE>(s, ea, st);
}

// renorm_reject: normalise m also when the step was rejected (the host
// controller's end of a step whose every trial failed); the device
// controller leaves m untouched on a rejected trial and retries.
__global__ void k_finalize_accept(float* __restrict__ m, const float* __restrict__ mnew, int64_t n,
                                  const int* __restrict__ accept, int renorm_reject = 1) {
  bool acc = *accept != 0;
  if (!acc && !renorm_reject) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x, y, z;
    if (acc) { x = mnew[i]; y = mnew[n + i]; z = mnew[2 * n + i]; }
    else { x = m[i]; y = m[n + i]; z = m[2 * n + i]; }
    llg_normalize(x, y, z);
    m[i] = x;
    m[n + i] = y;
    m[2 * n + i] = z;
  }
}

// <m> in one launch (simoutput.go:236, simget.go:32): per-component sums in
// float64 (block reduction + one atomic per block); the last block to
// finish (counted on 'done') divides by the cell count, writes the three
// values to 'out' (device memory, or page-locked host memory the kernel can
// reach) and clears acc and done for the next call.
__global__ void k_avg_m(const float* __restrict__ m, int64_t n, double* __restrict__ acc, unsigned int* done,
                        float* __restrict__ out) {
  __shared__ double sh[3][32];
  __shared__ bool last;
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v[0] += m[i];
    v[1] += m[n + i];
    v[2] += m[2 * n + i];
  }
  for (int c = 0; c < 3; c++)
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int c = 0; c < 3; c++) sh[c][w] = v[c];
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    for (int c = 0; c < 3; c++) {
      double t = l < nw ? sh[c][l] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (l == 0) atomicAdd(&acc[c], t);
    }
    if (l == 0) {
      __threadfence();
      last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (last && threadIdx.x < 3) {
    __threadfence();
    const double total = atomicAdd(&acc[threadIdx.x], 0.0);
    out[threadIdx.x] = (float)(total / (double)n);
    acc[threadIdx.x] = 0.0;
    if (threadIdx.x == 0) *done = 0u;
  }
}

int solver_grid_1d(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)mmx_sm_count() * 8;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// RK.step (rk.go:279-445): up to 10 trials.  The stage kernels read dt
// from device memory; the controller runs on the host in float32 exactly
// as the Go code.  Fixed-step tableaux never read back; adaptive ones read
// 8 bytes (error, maximum torque) per trial, the same synchronisation the
// reference's two reductions per step impose.
static int rk_step(mmx_solver* s, cudaStream_t st) {
  float* dt_dev = s->scratch + 2;
  int* acc_dev = reinterpret_cast<int*>(s->scratch + 3);
  const int last = s->stages - 1;
  const float ut = s->p.unit_time;
  const bool bounds = s->p.min_dm != 0.f || s->p.max_dm != 0.f || s->p.min_dt != 0.f || s->p.max_dt != 0.f;
  double time0 = s->time;
  int good = 0, trials = 0;
  const bool want_e = s->want_energy && s->eacc;
  const int e_stage = s->fsal ? s->stages - 1 : 0;
  // the thermal noise, fixed for the step's trials (updateTempNoise at the
  // step start, rk.go:289-292; temperature.go:27-36)
  const bool thermal = s->p.thermal_k != 0.f;
  s->noise_sigma = thermal ? (float)sqrt((double)f32_div(s->p.thermal_k, s->dt)) : 0.f;
  s->noise_step = s->steps;
  // energy must not rise when it is wanted (rk.go:297-301,425)
  float prevE = s->energy;
  if (prevE == 0.f) prevE = 9999999999.f;
  while (!good && trials < 10) {
    trials++;
    for (int i = 0; i < s->stages; i++) {
      if (want_e && i == e_stage && !(s->fsal && i == 0 && s->fsal_init))
        MMX_TRY(cudaMemsetAsync(s->eacc, 0, sizeof(double), st));
      if (s->fsal && i == 0 && s->fsal_init) {
        // FSAL copy k0 <- k_last (rk.go:311-315), done as a buffer swap.
        // The reference repeats it on a retry, so the retry starts from the
        // rejected attempt's last torque; the clean mode keeps k0.
        if (trials == 1 || s->p.faithful) {
          float* t = s->kb[0];
          s->kb[0] = s->kb[last];
          s->kb[last] = t;
        }
        MMX_TRY(cudaMemsetAsync(s->scratch + 1, 0, sizeof(float), st));
        k_maxabs<<<solver_grid_1d(3 * s->n), 256, 0, st>>>(s->kb[0], 3 * s->n, s->scratch + 1);
        MMX_TRY(cudaGetLastError());
      } else {
        if (i == 0) MMX_TRY(cudaMemsetAsync(s->scratch + 1, 0, sizeof(float), st));
        if (i == last && s->adaptive) MMX_TRY(cudaMemsetAsync(s->scratch, 0, sizeof(float), st));
        MMX_TRY(cudaMemcpyAsync(dt_dev, &s->dt, sizeof(float), cudaMemcpyHostToDevice, st));
        cudaError_t e = rk_stage(s, i, st, dt_dev);
        if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
        s->fsal_init = 1;
      }
      if (i == 0 && bounds && !thermal) {
        // dt bounds from the maximum torque (rk.go:348-373; not with a
        // thermal field)
        float mt = 0;
        MMX_TRY(cudaMemcpyAsync(&mt, s->scratch + 1, sizeof(float), cudaMemcpyDeviceToHost, st));
        MMX_TRY(cudaStreamSynchronize(st));
        s->torque = mt;
        float dm = f32_mul(s->dt, mt);
        if (dm < s->p.min_dm) s->dt = f32_div(s->p.min_dm, mt);
        if (f32_mul(s->dt, ut) < s->p.min_dt) s->dt = f32_div(s->p.min_dt, ut);
        if (s->p.max_dm != 0.f && dm > s->p.max_dm) s->dt = f32_div(s->p.max_dm, mt);
        if (s->p.max_dt != 0.f && f32_mul(s->dt, ut) > s->p.max_dt) s->dt = f32_div(s->p.max_dt, ut);
        if (s->dt != s->dt) { mmx_set_error("dt = NaN"); return MMX_ERR_NAN; }
      }
    }
    s->time = time0 + (double)s->dt;
    double esum = 0;
    if (want_e) MMX_TRY(cudaMemcpyAsync(&esum, s->eacc, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (!s->adaptive) {
      good = 1;
      int one = 1;
      MMX_TRY(cudaMemcpyAsync(acc_dev, &one, sizeof(int), cudaMemcpyHostToDevice, st));
      if (want_e) {
        MMX_TRY(cudaStreamSynchronize(st));
        s->energy = (float)(esum * (double)solver_cell_volume(s));
      }
      break;
    }
    float sc[2];
    MMX_TRY(cudaMemcpyAsync(sc, s->scratch, sizeof(float) * 2, cudaMemcpyDeviceToHost, st));
    MMX_TRY(cudaStreamSynchronize(st));
    if (want_e) s->energy = (float)(esum * (double)solver_cell_volume(s));
    float err = sc[0];
    s->torque = sc[1];
    s->step_error = err;
    float factor = (float)pow((double)f32_div(s->p.max_error, err), 1. / s->errorder);
    if (factor > 2.f) factor = 2.f;
    if (factor < 0.01f) factor = 0.01f;
    s->dt = f32_mul(s->dt, factor);
    if (s->dt != s->dt || err != err) { mmx_set_error("dt = NaN"); return MMX_ERR_NAN; }
    if (err > f32_mul(2.f, s->p.max_error) || (want_e && s->energy > prevE)) {
      good = 0;
    } else {
      good = 1;
      if (f32_mul(s->dt, ut) < s->p.min_dt) s->dt = f32_div(s->p.min_dt, ut);
      if (s->p.max_dt != 0.f && f32_mul(s->dt, ut) > s->p.max_dt) s->dt = f32_div(s->p.max_dt, ut);
    }
    int accv = good;
    MMX_TRY(cudaMemcpyAsync(acc_dev, &accv, sizeof(int), cudaMemcpyHostToDevice, st));
  }
  // m <- normalize(m_high) if accepted, else normalize(m)   (rk.go:444)
  k_finalize_accept<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->mnew, s->n, acc_dev);
  MMX_TRY(cudaGetLastError());
  return MMX_OK;
}

static int heun_adaptive_update(mmx_solver* s, cudaStream_t st) {
  float err = 0;
  MMX_TRY(cudaMemcpyAsync(&err, s->scratch, sizeof(float), cudaMemcpyDeviceToHost, st));
  MMX_TRY(cudaStreamSynchronize(st));
  s->step_error = err;
  float factor = f32_div(s->p.max_error, err);
  if (factor > 2.f) factor = 2.f;
  if (factor < 0.01f) factor = 0.01f;
  s->dt = f32_mul(s->dt, factor);
  return MMX_OK;
}

// ------------------------------ API -----------------------------------
extern "C" int mmx_face_kernel6(const int P[3], const int periodic[3], const float cellsize[3], int accuracy,
                                int exch6, float* k6, cudaStream_t stream) {
  if (!P || !periodic || !cellsize || !k6 || accuracy <= 0) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  FaceKernelArgs a;
  for (int d = 0; d < 3; d++) {
    a.P[d] = P[d];
    a.periodic[d] = periodic[d];
    a.cs[d] = cellsize[d];
    if (P[d] < 1) { mmx_set_error("bad size"); return MMX_ERR_SIZE; }
  }
  a.accuracy = accuracy;
  // loop bounds of demag.go:136-154
  for (int d = 0; d < 3; d++) {
    int lo = -(P[d] - 1) / 2, hi = P[d] / 2 - 1;
    if (d == 0 && P[0] == 1 && periodic[0] == 0) hi = 0;
    lo *= periodic[d] + 1;
    hi *= periodic[d] + 1;
    a.lo[d] = lo;
    a.hi[d] = hi;
  }
  int64_t n3 = (int64_t)P[0] * P[1] * P[2];
  int blocks = (int)((n3 + 127) / 128);
  int cap = mmx_sm_count() * 16;
  if (blocks > cap) blocks = cap;
  k_face_kernel6<<<blocks, 128, 0, stream>>>(k6, a);
  MMX_TRY(cudaGetLastError());
  if (exch6) {
    k_add_exch6<<<1, 1, 0, stream>>>(k6, P[0], P[1], P[2], cellsize[0], cellsize[1], cellsize[2]);
    MMX_TRY(cudaGetLastError());
  }
  return MMX_OK;
}

static void free_profile_graph(mmx_solver* s);
static void solver_free(mmx_solver* s) {
  if (!s) return;
  solver_run_free(s);
  free_profile_graph(s);
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  for (int g = 0; g < 2; g++)
    if (s->dgraph[g]) cudaGraphExecDestroy(s->dgraph[g]);
  cudaFree(s->rkdev);
  cudaFree(s->S);
  cudaFree(s->kh);
  cudaFree(s->kt_tc);
  cudaFree(s->m);
  cudaFree(s->t0);
  cudaFree(s->m1);
  cudaFree(s->mnew);
  cudaFree(s->scratch);
  for (int i = 0; i < RK_MAXS; i++) cudaFree(s->kb[i]);
  for (auto& t : s->timers)
    for (auto& pr : t.pending) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
  delete s;
}

extern "C" int mmx_solver_create(const mmx_params* p, mmx_solver** out) {
  if (!p || !out) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  *out = nullptr;
  mmx_solver* s = new mmx_solver();
  s->p = *p;
  if (s->p.accuracy <= 0) s->p.accuracy = 8;
  for (int d = 0; d < 3; d++) {
    s->N[d] = p->size[d];
    if (s->N[d] < 1) { delete s; mmx_set_error("size must be >= 1"); return MMX_ERR_SIZE; }
    s->P[d] = (s->N[d] > 1 && p->periodic[d] == 0) ? 2 * s->N[d] : s->N[d];
  }
  if (p->precision && !(p->size[0] == 1 && s->P[1] == 1024 && s->N[1] == 512 && p->periodic[1] == 0)) {
    delete s;
    mmx_set_error("precision form: 2D films with Ny = 512 (padded 1024) only");
    return MMX_ERR_SIZE;
  }
  if (s->N[2] < 2 || s->N[1] < 2) {
    delete s;
    mmx_set_error("internal Y and Z sizes must be >= 2 (gpu_fft0.cu:39-41)");
    return MMX_ERR_SIZE;
  }
  s->is2d = s->P[0] == 1;
  s->n = (int64_t)s->N[0] * s->N[1] * s->N[2];
  int rc = box_plan_init(&s->bp, s->N, s->P);
  if (rc != MMX_OK) { delete s; mmx_set_error("unsupported padded size (radices 2,3,5,7; <= 16384)"); return rc; }
  s->HZ = s->bp.HZ;
  s->CS = (int64_t)s->N[0] * s->P[1] * s->HZ;
  set_tableau(s);
  if (p->solver != MMX_SOLVER_HEUN && s->stages == 0) { delete s; mmx_set_error("unknown solver"); return MMX_ERR_ARG; }
  if (p->thermal_k != 0.f && (p->solver == MMX_SOLVER_HEUN || p->thermal_k < 0.f || p->precision)) {
    delete s;
    mmx_set_error("thermal field: RK solvers with the FP32 transforms only (the reference runs it with rk12)");
    return MMX_ERR_ARG;
  }
  s->dt = p->dt;
  size_t n3 = 3 * (size_t)s->n;
#define ALLOC(ptr, bytes)                                                   \
  if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) {                         \
    solver_free(s);                                                         \
    mmx_set_error("out of device memory");                                  \
    return MMX_ERR_MEM;                                                     \
  }
  ALLOC(s->S, sizeof(float2) * 3 * (size_t)s->CS);
  ALLOC(s->m, sizeof(float) * n3);
  ALLOC(s->m1, sizeof(float) * n3);
  ALLOC(s->scratch, sizeof(float) * 16);
  cudaMemset(s->m, 0, sizeof(float) * n3);
  cudaMemset(s->scratch, 0, sizeof(float) * 16);
  if (p->solver == MMX_SOLVER_HEUN) {
    ALLOC(s->t0, sizeof(float) * n3);
  } else {
    for (int i = 0; i < s->stages; i++) ALLOC(s->kb[i], sizeof(float) * n3);
    ALLOC(s->mnew, sizeof(float) * n3);
  }
  // kernel: real space on the GPU, transformed component by component
  {
    int64_t p3 = (int64_t)s->P[0] * s->P[1] * s->P[2];
    float* k6 = nullptr;
    float2* spec = nullptr;
    int O0 = s->P[0] / 2 + 1, O1 = s->P[1] / 2 + 1;
    int64_t ocs = (int64_t)O0 * O1 * s->HZ;
    ALLOC(s->kh, sizeof(float) * 6 * ocs);
    if (cudaMalloc(&k6, sizeof(float) * 6 * p3) != cudaSuccess ||
        cudaMalloc(&spec, sizeof(float2) * (size_t)s->P[0] * s->P[1] * s->HZ) != cudaSuccess) {
      cudaFree(k6);
      solver_free(s);
      mmx_set_error("out of device memory (kernel build)");
      return MMX_ERR_MEM;
    }
    float cs[3] = {p->cellsize[0], p->cellsize[1], p->cellsize[2]};
    rc = mmx_face_kernel6(s->P, p->periodic, cs, s->p.accuracy, p->exch_type == 6, k6, 0);
    BoxPlan full;
    if (rc == MMX_OK) rc = box_plan_init(&full, s->P, s->P);
    // loadKernel6 (conv.go:126-160): same transform, real part x 1/N
    float norm = f32_div(1.f, (float)p3);
    for (int c = 0; c < 6 && rc == MMX_OK; c++) {
      if (s->is2d && (c == 4 || c == 5)) {
        cudaMemset(s->kh + c * ocs, 0, sizeof(float) * ocs);
        continue;
      }
      if (box_forward(&full, k6 + c * p3, spec, 0) != cudaSuccess) rc = MMX_ERR_CUDA;
      k_extract_octant<<<solver_grid_1d(ocs), 256>>>(spec, s->kh + c * ocs, O0, O1, s->P[1], s->HZ, norm);
    }
    cudaError_t ce = cudaDeviceSynchronize();
    cudaFree(k6);
    cudaFree(spec);
    if (rc != MMX_OK || ce != cudaSuccess) {
      solver_free(s);
      mmx_set_error(ce != cudaSuccess ? cudaGetErrorString(ce) : "kernel build failed");
      return rc != MMX_OK ? rc : MMX_ERR_CUDA;
    }
    s->K.kh = s->kh;
    s->K.O0 = O0;
    s->K.O1 = O1;
    s->K.HZ = s->HZ;
    s->K.P0 = s->P[0];
    s->K.P1 = s->P[1];
    s->K.cs = ocs;
  }
#undef ALLOC
  if (s->p.precision) {
    rc = mmx_yconv2d_tc_prepare();
    if (rc == MMX_OK) rc = mmx_yconv2d_tc_kernel(s->K.kh, s->K.cs, s->HZ, &s->kt_tc);
    if (rc != MMX_OK) { solver_free(s); return rc; }
  }
  *out = s;
  return MMX_OK;
}

extern "C" int mmx_solver_destroy(mmx_solver* s) {
  solver_free(s);
  return MMX_OK;
}

extern "C" int mmx_solver_set_m(mmx_solver* s, const float* m, int on_host, cudaStream_t st) {
  if (!s || !m) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  MMX_TRY(cudaMemcpyAsync(s->m, m, sizeof(float) * 3 * s->n, on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
  MMX_TRY(cudaStreamSynchronize(st));
  s->fsal_init = 0;
  s->spec_ready = 0;
  return MMX_OK;
}

extern "C" int mmx_solver_get_m(mmx_solver* s, float* m, int on_host, cudaStream_t st) {
  if (!s || !m) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  MMX_TRY(cudaMemcpyAsync(m, s->m, sizeof(float) * 3 * s->n, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
  MMX_TRY(cudaStreamSynchronize(st));
  return MMX_OK;
}

extern "C" int mmx_solver_normalize(mmx_solver* s, cudaStream_t st) {
  if (!s) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  s->spec_ready = 0;
  k_normalize3<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->n);
  MMX_TRY(cudaGetLastError());
  return MMX_OK;
}

extern "C" int mmx_solver_field(mmx_solver* s, const float* m, float* h, cudaStream_t st) {
  if (!s || !m || !h) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  s->spec_ready = 0;
  cudaError_t e = conv_front(s, m, st);
  if (e == cudaSuccess) {
    EpiArgs ea = solver_base_args(s);
    ea.m_in = m;
    ea.out0 = h;
    e = launch_zinv<EPI_FIELD>(s, ea, st);
  }
  if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
  return MMX_OK;
}

int solver_field_conv(mmx_solver* s, const float* m, float* h, cudaStream_t st) {
  s->spec_ready = 0;
  cudaError_t e = conv_front(s, m, st);
  if (e == cudaSuccess) {
    EpiArgs ea = solver_base_args(s);
    memset(&ea.lf, 0, sizeof(ea.lf));  // h + 0: the convolution alone
    ea.m_in = m;
    ea.out0 = h;
    e = launch_zinv<EPI_FIELD>(s, ea, st);
  }
  if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
  return MMX_OK;
}

static int step_once(mmx_solver* s, cudaStream_t st);
int solver_step_once(mmx_solver* s, cudaStream_t st) { return step_once(s, st); }
float solver_cell_volume(const mmx_solver* s) {
  return f32_mul(f32_mul(s->p.cellsize[0], s->p.cellsize[1]), s->p.cellsize[2]);
}

static int step_once(mmx_solver* s, cudaStream_t st) {
  if (s->p.solver == MMX_SOLVER_HEUN) {
    cudaError_t e = heun_step(s, st);
    if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
    s->time += (double)s->dt;
    if (s->p.max_error != 0.f) return heun_adaptive_update(s, st);
    return MMX_OK;
  }
  return rk_step(s, st);
}

// ---------------------------------------------------------------------
// Device-side controller of the adaptive RK solvers (mmx_solver_device_control).
// One trial of RK.step (rk.go:279-445) is a fixed launch sequence captured
// once as a CUDA graph: FSAL copy k0 <- k_last (a copy instead of the host
// path's pointer swap), the stages (their dt read from device memory),
// then a one-thread controller that applies rk.go's float32 rules --
// factor = (maxErr/err)^(1/order) clamped to [0.01, 2], reject when
// err > 2 maxErr, the min/max dt clamps -- accumulates the time in float64
// and flags acceptance for the finalisation.  A rejected trial leaves m
// untouched; the next replay retries with the reduced dt.  No host
// synchronisation per step.
// ---------------------------------------------------------------------
__global__ void k_fsal_copy(float* __restrict__ k0, const float* __restrict__ klast, int64_t n3,
                            const RkDev* __restrict__ dev, int faithful, float* __restrict__ torque) {
  const bool copy = dev->accept || faithful;  // rk.go:311-315 (retry: faithful reuses the rejected k_last)
  float lmax = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
    float v = copy ? klast[i] : k0[i];
    if (copy) k0[i] = v;
    lmax = fmaxf(lmax, fabsf(v));
  }
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(torque, lmax);
}

struct RkCtl {
  float max_error, min_dm, max_dm, min_dt, max_dt, unit_time;
  double inv_order;
  int bounds;
};

// dt bounds from the maximum torque of stage 0 (rk.go:348-373)
__global__ void k_rk_bounds(float* __restrict__ scratch, RkDev* __restrict__ dev, RkCtl c) {
  float mt = scratch[1];
  float dt = scratch[2];
  float dm = __fmul_rn(dt, mt);
  if (dm < c.min_dm) dt = __fdiv_rn(c.min_dm, mt);
  if (__fmul_rn(dt, c.unit_time) < c.min_dt) dt = __fdiv_rn(c.min_dt, c.unit_time);
  if (c.max_dm != 0.f && dm > c.max_dm) dt = __fdiv_rn(c.max_dm, mt);
  if (c.max_dt != 0.f && __fmul_rn(dt, c.unit_time) > c.max_dt) dt = __fdiv_rn(c.max_dt, c.unit_time);
  if (dt != dt) dev->bad = 1;
  scratch[2] = dt;
  dev->dt = dt;
}

// the error rule of rk.go:401-439 in float32; time in float64
__global__ void k_rk_control(float* __restrict__ scratch, RkDev* __restrict__ dev, RkCtl c) {
  const float err = scratch[0];
  const float dt = scratch[2];
  float factor = (float)pow((double)__fdiv_rn(c.max_error, err), c.inv_order);
  if (factor > 2.f) factor = 2.f;
  if (factor < 0.01f) factor = 0.01f;
  float nd = __fmul_rn(dt, factor);
  if (nd != nd || err != err) dev->bad = 1;
  int acc = !(err > __fmul_rn(2.f, c.max_error));
  if (acc) {
    dev->time += (double)dt;
    dev->accepted++;
    if (__fmul_rn(nd, c.unit_time) < c.min_dt) nd = __fdiv_rn(c.min_dt, c.unit_time);
    if (c.max_dt != 0.f && __fmul_rn(nd, c.unit_time) > c.max_dt) nd = __fdiv_rn(c.max_dt, c.unit_time);
  }
  dev->trials++;
  dev->accept = acc;
  dev->err = err;
  dev->torque = scratch[1];
  dev->dt = nd;
  scratch[2] = nd;
  reinterpret_cast<int*>(scratch)[3] = acc;
}

static RkCtl rk_ctl(const mmx_solver* s) {
  RkCtl c;
  c.max_error = s->p.max_error;
  c.min_dm = s->p.min_dm;
  c.max_dm = s->p.max_dm;
  c.min_dt = s->p.min_dt;
  c.max_dt = s->p.max_dt;
  c.unit_time = s->p.unit_time;
  c.inv_order = 1. / s->errorder;
  c.bounds = s->p.min_dm != 0.f || s->p.max_dm != 0.f || s->p.min_dt != 0.f || s->p.max_dt != 0.f;
  return c;
}

// one trial; first: stage 0 evaluated (no FSAL value yet)
static cudaError_t rk_device_trial(mmx_solver* s, cudaStream_t st, bool first) {
  float* dt_dev = s->scratch + 2;
  const int* acc_dev = reinterpret_cast<const int*>(s->scratch + 3);
  RkDev* dev = reinterpret_cast<RkDev*>(s->rkdev);
  const RkCtl c = rk_ctl(s);
  const int last = s->stages - 1;
  cudaError_t e;
  for (int i = 0; i < s->stages; i++) {
    if (i == 0) {
      if ((e = cudaMemsetAsync(s->scratch + 1, 0, sizeof(float), st)) != cudaSuccess) return e;
      if (s->fsal && !first) {
        k_fsal_copy<<<solver_grid_1d(3 * s->n), 256, 0, st>>>(s->kb[0], s->kb[last], 3 * s->n, dev, s->p.faithful,
                                                              s->scratch + 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      } else if ((e = rk_stage(s, 0, st, dt_dev)) != cudaSuccess) {
        return e;
      }
      if (c.bounds) {
        k_rk_bounds<<<1, 1, 0, st>>>(s->scratch, dev, c);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      continue;
    }
    if (i == last && (e = cudaMemsetAsync(s->scratch, 0, sizeof(float), st)) != cudaSuccess) return e;
    if ((e = rk_stage(s, i, st, dt_dev)) != cudaSuccess) return e;
  }
  k_rk_control<<<1, 1, 0, st>>>(s->scratch, dev, c);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_finalize_accept<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->mnew, s->n, acc_dev, 0);
  return cudaGetLastError();
}

static int rk_device_download(mmx_solver* s) {
  RkDev h;
  // trials may be in flight on any stream (the graphs replay on the caller's)
  MMX_TRY(cudaDeviceSynchronize());
  MMX_TRY(cudaMemcpy(&h, s->rkdev, sizeof(h), cudaMemcpyDeviceToHost));
  if (h.bad) { mmx_set_error("dt = NaN"); return MMX_ERR_NAN; }
  s->time = h.time;
  s->dt = h.dt;
  s->steps = s->steps_base + h.accepted;
  s->torque = h.torque;
  s->step_error = h.err;
  s->trials = h.trials;
  return MMX_OK;
}

cudaError_t solver_device_trial(mmx_solver* s, cudaStream_t st, bool first) { return rk_device_trial(s, st, first); }
int solver_device_download(mmx_solver* s) { return rk_device_download(s); }

extern "C" int mmx_solver_device_control(mmx_solver* s, int on) {
  if (!s) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (on && (!s->adaptive || s->p.solver == MMX_SOLVER_HEUN)) {
    mmx_set_error("device control: adaptive RK solvers (rk12, rk23, rkck, rkdp) only");
    return MMX_ERR_ARG;
  }
  if (on && s->p.thermal_k != 0.f) {
    mmx_set_error("device control: not with a thermal field (its noise is drawn per step on the host controller)");
    return MMX_ERR_ARG;
  }
  if (on && !s->devctl) {
    if (!s->rkdev && cudaMalloc(&s->rkdev, sizeof(RkDev)) != cudaSuccess) {
      mmx_set_error("out of device memory");
      return MMX_ERR_MEM;
    }
    RkDev h;
    memset(&h, 0, sizeof(h));
    h.time = s->time;
    h.dt = s->dt;
    h.accept = 1;
    MMX_TRY(cudaMemcpy(s->rkdev, &h, sizeof(h), cudaMemcpyHostToDevice));
    MMX_TRY(cudaMemcpy(s->scratch + 2, &s->dt, sizeof(float), cudaMemcpyHostToDevice));
    s->steps_base = s->steps;
    s->devctl = 1;
  } else if (!on && s->devctl) {
    MMX_CHECK_RC(rk_device_download(s));
    s->devctl = 0;
    s->fsal_init = 0;  // the host path starts its FSAL chain afresh
  }
  return MMX_OK;
}

// n trials, each one graph replay
static int rk_device_steps(mmx_solver* s, int n, cudaStream_t st) {
  for (int k = 0; k < n; k++) {
    const int g = (s->fsal && s->fsal_init) ? 1 : 0;
    if (!s->dgraph[g] || s->dgraph_stream[g] != st) {
      if (s->dgraph[g]) { cudaGraphExecDestroy(s->dgraph[g]); s->dgraph[g] = nullptr; }
      cudaStream_t cap = st;
      bool own = false;
      if (cap == 0) { MMX_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
      cudaGraph_t gr;
      MMX_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = rk_device_trial(s, cap, g == 0);
      cudaError_t e2 = cudaStreamEndCapture(cap, &gr);
      if (own) cudaStreamDestroy(cap);
      if (e != cudaSuccess || e2 != cudaSuccess) { mmx_set_error("graph capture failed"); return MMX_ERR_CUDA; }
      MMX_TRY(cudaGraphInstantiate(&s->dgraph[g], gr, 0));
      cudaGraphDestroy(gr);
      s->dgraph_stream[g] = st;
    }
    MMX_TRY(cudaGraphLaunch(s->dgraph[g], st));
    s->fsal_init = 1;
  }
  return MMX_OK;
}

static bool rk_fixed(const mmx_solver* s) {
  const bool bounds = s->p.min_dm != 0.f || s->p.max_dm != 0.f || s->p.min_dt != 0.f || s->p.max_dt != 0.f;
  return s->p.solver != MMX_SOLVER_HEUN && !s->adaptive && !s->fsal && !bounds;
}

// One fixed-step RK step as pure launches (no host traffic), for graph
// capture: the device dt and accept flag are uploaded beforehand.
static cudaError_t rk_fixed_launches(mmx_solver* s, cudaStream_t st) {
  float* dt_dev = s->scratch + 2;
  const int* acc_dev = reinterpret_cast<const int*>(s->scratch + 3);
  for (int i = 0; i < s->stages; i++) {
    if (i == 0) {
      cudaError_t e = cudaMemsetAsync(s->scratch + 1, 0, sizeof(float), st);
      if (e != cudaSuccess) return e;
    }
    cudaError_t e = rk_stage(s, i, st, dt_dev);
    if (e != cudaSuccess) return e;
  }
  k_finalize_accept<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->mnew, s->n, acc_dev);
  return cudaGetLastError();
}

static cudaError_t step_launches(mmx_solver* s, cudaStream_t st) {
  return s->p.solver == MMX_SOLVER_HEUN ? heun_step(s, st) : rk_fixed_launches(s, st);
}

static void free_profile_graph(mmx_solver* s) {
  if (s->pgexec) cudaGraphExecDestroy(s->pgexec);
  s->pgexec = nullptr;
  for (auto& g : s->gevents) {
    if (g.own_a) cudaEventDestroy(g.a);
    cudaEventDestroy(g.b);
  }
  s->gevents.clear();
}

// Fixed-step solvers with profile mode 2: each step replays a graph whose
// passes are bracketed by event-record nodes; after each replay the pass
// times are added to the timers.
static int profiled_graph_steps(mmx_solver* s, int nsteps, cudaStream_t st) {
  for (int k = 0; k < nsteps; k++) {
    if (heun_fused(s) && !s->spec_ready) {
      cudaError_t e = zfwd_only(s, s->m, st);
      if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
      s->spec_ready = 1;
    }
    if (!s->pgexec || s->pgstream != st) {
      free_profile_graph(s);
      cudaStream_t cap = st;
      bool own = false;
      if (cap == 0) { MMX_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
      cudaGraph_t g;
      MMX_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      s->capture_events = 1;
      cudaError_t e = step_launches(s, cap);
      s->capture_events = 0;
      cudaError_t e2 = cudaStreamEndCapture(cap, &g);
      if (own) cudaStreamDestroy(cap);
      if (e != cudaSuccess || e2 != cudaSuccess) { mmx_set_error("graph capture failed"); return MMX_ERR_CUDA; }
      MMX_TRY(cudaGraphInstantiate(&s->pgexec, g, 0));
      cudaGraphDestroy(g);
      s->pgstream = st;
    }
    MMX_TRY(cudaGraphLaunch(s->pgexec, st));
    MMX_TRY(cudaStreamSynchronize(st));
    for (auto& g : s->gevents) {
      float ms = 0;
      MMX_TRY(cudaEventElapsedTime(&ms, g.a, g.b));
      PassTimer* t = timer_for(s, g.name.c_str());
      t->ms += ms;
      t->launches++;
    }
    s->time += (double)s->dt;
    s->steps++;
  }
  return MMX_OK;
}

extern "C" int mmx_solver_step(mmx_solver* s, int nsteps, cudaStream_t st) {
  if (!s || nsteps < 0) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  if (s->devctl) return rk_device_steps(s, nsteps, st);
  const bool fixed_graphable =
      ((s->p.solver == MMX_SOLVER_HEUN && s->p.max_error == 0.f) || rk_fixed(s)) && s->p.thermal_k == 0.f;
  if (s->profile == 2 && fixed_graphable && !s->want_energy) {
    if (s->p.solver != MMX_SOLVER_HEUN && s->dt_uploaded != s->dt) {
      float v[2] = {s->dt, 0.f};
      int one = 1;
      memcpy(&v[1], &one, sizeof(int));
      MMX_TRY(cudaMemcpyAsync(s->scratch + 2, v, sizeof(v), cudaMemcpyHostToDevice, st));
      MMX_TRY(cudaStreamSynchronize(st));
      s->dt_uploaded = s->dt;
    }
    return profiled_graph_steps(s, nsteps, st);
  }
  bool graphable = s->use_graph && !s->profile && !s->want_energy && fixed_graphable;
  if (graphable && s->p.solver != MMX_SOLVER_HEUN && s->dt_uploaded != s->dt) {
    float v[2] = {s->dt, 0.f};
    int one = 1;
    memcpy(&v[1], &one, sizeof(int));
    MMX_TRY(cudaMemcpyAsync(s->scratch + 2, v, sizeof(v), cudaMemcpyHostToDevice, st));
    MMX_TRY(cudaStreamSynchronize(st));
    s->dt_uploaded = s->dt;
  }
  for (int k = 0; k < nsteps; k++) {
    if (graphable && heun_fused(s) && !s->spec_ready) {
      // the captured step expects the forward Z spectrum of m in S
      cudaError_t e = zfwd_only(s, s->m, st);
      if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
      s->spec_ready = 1;
    }
    if (graphable) {
      if (!s->gexec || s->gstream != st) {
        if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
        cudaStream_t cap = st;
        bool own = false;
        if (cap == 0) { MMX_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
        cudaGraph_t g;
        MMX_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = step_launches(s, cap);
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        if (own) cudaStreamDestroy(cap);
        if (e != cudaSuccess || e2 != cudaSuccess) { mmx_set_error("graph capture failed"); return MMX_ERR_CUDA; }
        MMX_TRY(cudaGraphInstantiate(&s->gexec, g, 0));
        cudaGraphDestroy(g);
        s->gstream = st;
      }
      MMX_TRY(cudaGraphLaunch(s->gexec, st));
      s->time += (double)s->dt;
    } else {
      int rc = step_once(s, st);
      if (rc != MMX_OK) return rc;
    }
    s->steps++;
  }
  if (s->profile) flush_timers(s);
  return MMX_OK;
}

extern "C" int mmx_solver_avg_m(mmx_solver* s, float* out3, int on_host, cudaStream_t st) {
  if (!s || !out3) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  // scratch: float 4..6 the staging of a host result, 8..13 the float64
  // sums, 14 the block counter (all zero between calls)
  double* acc = reinterpret_cast<double*>(s->scratch + 8);
  unsigned int* done = reinterpret_cast<unsigned int*>(s->scratch + 14);
  float* dst = out3;
  bool copy = false;
  if (on_host) {
    // page-locked host memory is written by the kernel itself; other host
    // memory through the staging floats and a copy
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, out3) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer) {
      dst = static_cast<float*>(pa.devicePointer);
    } else {
      cudaGetLastError();  // an unregistered pointer is not an error here
      dst = s->scratch + 4;
      copy = true;
    }
  }
  k_avg_m<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->n, acc, done, dst);
  MMX_TRY(cudaGetLastError());
  if (copy) MMX_TRY(cudaMemcpyAsync(out3, dst, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
  return MMX_OK;
}

extern "C" int mmx_solver_state(mmx_solver* s, double* time, float* dt, float* max_torque, float* step_error,
                                long long* steps) {
  if (!s) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (s->devctl) MMX_CHECK_RC(rk_device_download(s));
  if (s->p.precision) {
    int tc_err = 0;
    MMX_TRY(cudaMemcpy(&tc_err, s->scratch + 15, sizeof(int), cudaMemcpyDeviceToHost));
    if (tc_err) { mmx_set_error("tensor-core convolution: completion wait timed out"); return MMX_ERR_CUDA; }
  }
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  if (max_torque) *max_torque = s->torque;
  if (step_error) *step_error = s->step_error;
  if (steps) *steps = s->steps;
  return MMX_OK;
}

extern "C" int mmx_solver_set_hext(mmx_solver* s, const float hext[3]) {
  if (!s || !hext) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  for (int d = 0; d < 3; d++) s->p.hext[d] = hext[d];
  if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  return MMX_OK;
}

extern "C" float* mmx_solver_m_device(mmx_solver* s) { return s ? s->m : nullptr; }
extern "C" float* mmx_solver_torque_device(mmx_solver* s) { return s ? s->scratch + 1 : nullptr; }

extern "C" int mmx_solver_use_graph(mmx_solver* s, int on) {
  if (!s) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  s->use_graph = on;
  if (!on && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  return MMX_OK;
}

extern "C" int mmx_solver_profile(mmx_solver* s, int on) {
  if (!s) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (s->profile) flush_timers(s);
  s->profile = on;
  if (on) s->timers.clear();
  return MMX_OK;
}

extern "C" int mmx_solver_pass_times(mmx_solver* s, int max, char (*names)[32], double* ms, long long* launches,
                                     int* n) {
  if (!s || !n) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  flush_timers(s);
  int k = 0;
  for (auto& t : s->timers) {
    if (k >= max) break;
    if (names) { strncpy(names[k], t.name.c_str(), 31); names[k][31] = 0; }
    if (ms) ms[k] = t.ms;
    if (launches) launches[k] = t.launches;
    k++;
  }
  *n = k;
  return MMX_OK;
}
