// Zero-aware 3D real-to-complex FFT passes of the LLG engine and the
// drop-in gpuFFT3dPlan entry points (reference: src/gpukern/gpu_fft0.cu).
//
// Layout (internal axis order, Z contiguous):
//   real data  (N0, N1, N2)                  -- one magnetisation component
//   spectrum   (P0, P1, HZ) complex,  HZ = P2/2 + 1
// which is exactly the in-place cuFFT R2C layout the reference uses:
// buffer of (P0, P1, P2+2) floats (gpu_fft0.cu:57-59,96-109).
//
// Passes (one kernel each):
//   Z  : real rows -> half spectrum, via a complex FFT of length P2/2 on
//        (x_2n, x_2n+1) pairs and the standard split; only rows with data
//        (x < N0, y < N1) are transformed, zero padding is implicit.
//   Y  : strided columns, only the N1 data rows are loaded.
//   X  : strided columns, only the N0 data planes are loaded.
// The inverse runs X, Y, Z and produces only the N0 x N1 x N2 outputs.
#include <map>
#include <mutex>
#include <vector>
#include <math.h>
#include <string.h>

#include "fft_engine.cuh"
#include "fft_passes.cuh"
#include "fft_fixed_kernels.cuh"

bool fft_factor(int L, LineFFT* f) {
  f->L = L;
  f->nst = 0;
  f->code = 0;
  int m = L;
  const int order[6] = {8, 4, 2, 3, 5, 7};
  const int codes[6] = {5, 2, 0, 1, 3, 4};
  for (int oi = 0; oi < 6; oi++) {
    int r = order[oi];
    while (m % r == 0) {
      if (f->nst >= FFT_MAX_STAGES) return false;
      f->code |= (unsigned long long)codes[oi] << (3 * f->nst);
      f->nst++;
      m /= r;
    }
  }
  return m == 1;
}

static std::mutex g_tw_mu;
static std::map<std::pair<int, int>, float2*> g_tw;

const float2* fft_twiddles(int Lt) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tw_mu);
  auto key = std::make_pair(dev, Lt);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) return it->second;
  std::vector<float2> h((size_t)Lt);
  for (int t = 0; t < Lt; t++) {
    // exact multiples of pi/2 are set exactly; the rest from double sin/cos
    double a = -2.0 * M_PI * (double)t / (double)Lt;
    double c = cos(a), s = sin(a);
    if ((4LL * t) % Lt == 0) {
      int q = (int)((4LL * t) / Lt) & 3;
      const double cc[4] = {1, 0, -1, 0}, ss[4] = {0, -1, 0, 1};
      c = cc[q];
      s = ss[q];
    }
    h[t] = make_float2((float)c, (float)s);
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, sizeof(float2) * (size_t)Lt) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), sizeof(float2) * (size_t)Lt, cudaMemcpyHostToDevice);
  g_tw[key] = d;
  return d;
}

// ---------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------
cudaError_t launch_z_r2c(const float* src, float2* dst, const ZPass& zp, cudaStream_t st, const ZComb* cb) {
  int M = zp.f.L;
  if (fx_ok(M)) {
    ZComb none;
    memset(&none, 0, sizeof(none));
    switch (M) {
#define C_(L) \
  case L: return cb ? fx_launch_zr2c<L, true>(src, dst, zp, *cb, st) : fx_launch_zr2c<L, false>(src, dst, zp, none, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int lines = 1;
  while (M * lines * 2 <= (is_pow2(M) ? 4096 : 2048) && lines * 2 <= zp.nrows) lines *= 2;
  size_t smem = sizeof(float2) * (size_t)M * lines;
  dim3 grid(div_up(zp.nrows, lines));
  ZComb none;
  memset(&none, 0, sizeof(none));
  SHAPE_DISPATCH(M * lines, is_pow2(M), {
    if (cb) {
      allow_smem(k_z_r2c<T, E, P2, true>, smem);
      k_z_r2c<T, E, P2, true><<<grid, T, smem, st>>>(src, dst, zp, lines, *cb);
    } else {
      allow_smem(k_z_r2c<T, E, P2, false>, smem);
      k_z_r2c<T, E, P2, false><<<grid, T, smem, st>>>(src, dst, zp, lines, none);
    }
  });
  return cudaGetLastError();
}

cudaError_t launch_z_c2r(const float2* src, float* dst, const ZPass& zp, cudaStream_t st) {
  int M = zp.f.L;
  if (fx_ok(M)) {
    switch (M) {
#define C_(L) \
  case L: return fx_launch_zc2r<L>(src, dst, zp, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int lines = 1;
  while ((M + 1) * lines * 2 <= (is_pow2(M) ? 4096 : 2048) && lines * 2 <= zp.nrows) lines *= 2;
  size_t smem = sizeof(float2) * (size_t)(M + 1) * lines;
  dim3 grid(div_up(zp.nrows, lines));
  SHAPE_DISPATCH((M + 1) * lines, is_pow2(M), {
    allow_smem(k_z_c2r<T, E, P2>, smem);
    k_z_c2r<T, E, P2><<<grid, T, smem, st>>>(src, dst, zp, lines);
  });
  return cudaGetLastError();
}

cudaError_t launch_col(const float2* src, float2* dst, const ColPass& cp, cudaStream_t st) {
  int L = cp.f.L;
  if (fx_ok(L)) {
    switch (L) {
#define C_(LL) \
  case LL: return cp.inv ? fx_launch_col<LL, true>(src, dst, cp, st) : fx_launch_col<LL, false>(src, dst, cp, st);
      FX_SIZES(C_)
#undef C_
    }
  }
  int tk = 1;
  while (tk < 32 && L * tk * 2 <= (is_pow2(L) ? 4096 : 2048) && tk * 2 <= cp.ncols) tk *= 2;
  size_t smem = sizeof(float2) * (size_t)L * tk;
  dim3 grid(div_up(cp.ncols, tk), cp.nplanes);
  SHAPE_DISPATCH(L * tk, is_pow2(L), {
    allow_smem(k_col<T, E, P2>, smem);
    k_col<T, E, P2><<<grid, T, smem, st>>>(src, dst, cp, tk);
  });
  return cudaGetLastError();
}

// ---------------------------------------------------------------------
// Transform plans over a padded box: forward and inverse of one component.
// ---------------------------------------------------------------------
int box_plan_init(BoxPlan* p, const int N[3], const int P[3]) {
  memset(p, 0, sizeof(*p));
  for (int d = 0; d < 3; d++) {
    p->N[d] = N[d];
    p->P[d] = P[d];
    if (N[d] < 1 || P[d] < N[d]) return MMX_ERR_SIZE;
  }
  if (P[2] % 2 != 0 || P[2] < 2) return MMX_ERR_SIZE;
  p->HZ = P[2] / 2 + 1;
  if (!fft_factor(P[2] / 2, &p->fz) || !fft_factor(P[1], &p->fy) || !fft_factor(P[0], &p->fx)) return MMX_ERR_SIZE;
  if (P[2] / 2 > 8192 || P[1] > 8192 || P[0] > 8192) return MMX_ERR_SIZE;
  // z uses the P2-length table at stride 2 for its half-length FFT and at
  // stride 1 for the real/complex split
  p->twz = fft_twiddles(P[2]);
  p->fz.tw = p->twz;
  p->fz.tws = 2;
  p->fy.tw = fft_twiddles(P[1]);
  p->fy.tws = 1;
  p->fx.tw = fft_twiddles(P[0]);
  p->fx.tws = 1;
  if (!p->twz || !p->fy.tw || !p->fx.tw) return MMX_ERR_MEM;
  return MMX_OK;
}

ZPass box_zpass(const BoxPlan* p, int ncomp, int n_x_planes, int64_t comp_stride_real, int64_t comp_stride_spec) {
  ZPass z;
  z.f = p->fz;
  z.twP = p->twz;
  z.rows_per_plane = p->N[1];
  z.nrows = ncomp * n_x_planes * p->N[1];
  z.ld_real = p->N[2];
  z.n_real = p->N[2];
  z.ld_spec = p->HZ;
  z.plane_stride_spec = (int64_t)p->P[1] * p->HZ;
  z.planes_per_comp = n_x_planes;
  z.comp_stride_real = comp_stride_real;
  z.comp_stride_spec = comp_stride_spec;
  return z;
}

cudaError_t box_forward(const BoxPlan* p, const float* in, float2* spec, cudaStream_t st) {
  // Z: rows (x < N0, y < N1)
  ZPass z = box_zpass(p, 1, p->N[0], 0, 0);
  cudaError_t e = launch_z_r2c(in, spec, z, st);
  if (e != cudaSuccess) return e;
  // Y: planes x < N0, columns kz < HZ, N1 data rows -> P1 outputs
  ColPass y;
  y.f = p->fy;
  y.nplanes = p->N[0];
  y.plane_stride = (int64_t)p->P[1] * p->HZ;
  y.ncols = p->HZ;
  y.stride_i = p->HZ;
  y.n_in = p->N[1];
  y.n_out = p->P[1];
  y.inv = 0;
  e = launch_col(spec, spec, y, st);
  if (e != cudaSuccess || p->P[0] == 1) return e;
  // X: columns (ky, kz), N0 data planes -> P0 outputs
  ColPass x;
  x.f = p->fx;
  x.nplanes = 1;
  x.plane_stride = 0;
  x.ncols = p->P[1] * p->HZ;
  x.stride_i = (int64_t)p->P[1] * p->HZ;
  x.n_in = p->N[0];
  x.n_out = p->P[0];
  x.inv = 0;
  return launch_col(spec, spec, x, st);
}

cudaError_t box_inverse(const BoxPlan* p, float2* spec, float* out, cudaStream_t st) {
  cudaError_t e;
  if (p->P[0] > 1) {
    ColPass x;
    x.f = p->fx;
    x.nplanes = 1;
    x.plane_stride = 0;
    x.ncols = p->P[1] * p->HZ;
    x.stride_i = (int64_t)p->P[1] * p->HZ;
    x.n_in = p->P[0];
    x.n_out = p->N[0];
    x.inv = 1;
    e = launch_col(spec, spec, x, st);
    if (e != cudaSuccess) return e;
  }
  ColPass y;
  y.f = p->fy;
  y.nplanes = p->N[0];
  y.plane_stride = (int64_t)p->P[1] * p->HZ;
  y.ncols = p->HZ;
  y.stride_i = p->HZ;
  y.n_in = p->P[1];
  y.n_out = p->N[1];
  y.inv = 1;
  e = launch_col(spec, spec, y, st);
  if (e != cudaSuccess) return e;
  ZPass z = box_zpass(p, 1, p->N[0], 0, 0);
  return launch_z_c2r(spec, out, z, st);
}
