// Shared-memory mixed-radix Stockham FFT used by every transform of the
// LLG engine.  A CTA owns a tile of lines in shared memory; each stage
// reads all of its butterfly inputs into registers, synchronises, applies
// twiddles and the radix-R DFT, and writes the outputs in Stockham (self
// sorting) order, so the tile is transformed in place and the result is in
// natural order.
//
// Radices 2, 4, 8 have specialised butterflies; 3, 5, 7 use a constant
// table DFT.  A line length is any product of these.
//
// Twiddles come from a per-length table tw[t] = exp(-2 pi i t / Lt) in
// float, computed in double on the host; a stage of radix R at span ns
// uses tw[(q * (j mod ns) * (L / (ns R))) * tws] with Lt = L * tws.
#pragma once
#include "mmx_common.cuh"

#define FFT_MAX_STAGES 16

// Radix codes, 3 bits per stage (kernel parameters must not be indexed
// with a runtime index, which would copy them to local memory).
#define FFT_RADIX_OF(code) ((code) == 0 ? 2 : (code) == 1 ? 3 : (code) == 2 ? 4 : (code) == 3 ? 5 : (code) == 4 ? 7 : 8)

struct LineFFT {
  int L;                       // complex length of the line
  int nst;                     // number of stages
  unsigned long long code;     // radix code of stage s in bits [3s, 3s+3)
  const float2* tw;            // twiddle table, length L * tws
  int tws;                     // table stride (table built for a multiple of L)
};

// complex product with two fused multiply-adds (the transforms are
// compared with the FP64 oracle within a tolerance, never bit for bit)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 mul_mi(float2 a, bool inv) {
  return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
struct Radix {
  // out = DFT_R(v), sign -1 (forward) or +1 (inverse)
  __device__ __forceinline__ static void dft(float2* v, bool inv);
};

template <>
__device__ __forceinline__ void Radix<2>::dft(float2* v, bool) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void Radix<4>::dft(float2* v, bool inv) {
  float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  float2 t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]), inv);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <>
__device__ __forceinline__ void Radix<8>::dft(float2* v, bool inv) {
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  Radix<4>::dft(e, inv);
  Radix<4>::dft(o, inv);
  const float h = 0.70710678118654752440f;
  // W8^1, W8^2, W8^3 for the given direction
  float2 w1 = inv ? make_float2(h, h) : make_float2(h, -h);
  float2 w3 = inv ? make_float2(-h, h) : make_float2(-h, -h);
  float2 o1 = cmul(o[1], w1);
  float2 o2 = mul_mi(o[2], inv);
  float2 o3 = cmul(o[3], w3);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

// Radix 16 (fixed-size transforms only): two radix-8 DFTs of the even and
// odd samples combined with the twiddles W16^k.
template <>
__device__ __forceinline__ void Radix<16>::dft(float2* v, bool inv) {
  float2 e[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    e[k] = v[2 * k];
    o[k] = v[2 * k + 1];
  }
  Radix<8>::dft(e, inv);
  Radix<8>::dft(o, inv);
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
  // W16^k = exp(-+ 2 pi i k / 16), k = 1..7 (conjugated for the inverse)
  const float wr[8] = {1.f, c1, h, s1, 0.f, -s1, -h, -c1};
  const float wi[8] = {0.f, s1, h, c1, 1.f, c1, h, s1};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    float2 t = k == 0 ? o[0] : k == 4 ? mul_mi(o[4], inv) : cmul(o[k], make_float2(wr[k], inv ? wi[k] : -wi[k]));
    v[k] = cadd(e[k], t);
    v[k + 8] = csub(e[k], t);
  }
}

// Radix-R DFTs whose upper half of inputs is zero (a zero-padded line's
// first stage): the zero terms are never added.
template <int R>
__device__ __forceinline__ void dft_half(float2* v, bool inv) {
  Radix<R>::dft(v, inv);
}
template <>
__device__ __forceinline__ void dft_half<8>(float2* v, bool inv) {
  // DFT4 of [a, b, 0, 0] = (a + b, a + W4 b, a - b, a - W4 b)
  float2 mb = mul_mi(v[2], inv), md = mul_mi(v[3], inv);
  float2 e[4] = {cadd(v[0], v[2]), cadd(v[0], mb), csub(v[0], v[2]), csub(v[0], mb)};
  float2 o[4] = {cadd(v[1], v[3]), cadd(v[1], md), csub(v[1], v[3]), csub(v[1], md)};
  const float h = 0.70710678118654752440f;
  float2 w1 = inv ? make_float2(h, h) : make_float2(h, -h);
  float2 w3 = inv ? make_float2(-h, h) : make_float2(-h, -h);
  float2 o1 = cmul(o[1], w1);
  float2 o2 = mul_mi(o[2], inv);
  float2 o3 = cmul(o[3], w3);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}
template <>
__device__ __forceinline__ void dft_half<16>(float2* v, bool inv) {
  float2 e[8], o[8];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    e[k] = v[2 * k];
    o[k] = v[2 * k + 1];
  }
  dft_half<8>(e, inv);
  dft_half<8>(o, inv);
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
  const float wr[8] = {1.f, c1, h, s1, 0.f, -s1, -h, -c1};
  const float wi[8] = {0.f, s1, h, c1, 1.f, c1, h, s1};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    float2 t = k == 0 ? o[0] : k == 4 ? mul_mi(o[4], inv) : cmul(o[k], make_float2(wr[k], inv ? wi[k] : -wi[k]));
    v[k] = cadd(e[k], t);
    v[k + 8] = csub(e[k], t);
  }
}

// Odd radices: direct DFT with constant twiddles cos/sin(2 pi k / R).
template <int R>
__device__ __forceinline__ void odd_dft(float2* v, bool inv, const float* c, const float* s) {
  float2 out[R];
#pragma unroll
  for (int o = 0; o < R; o++) {
    float2 acc = v[0];
#pragma unroll
    for (int q = 1; q < R; q++) {
      int t = (o * q) % R;
      float2 w = make_float2(c[t], inv ? s[t] : -s[t]);
      float2 p = cmul(v[q], w);
      acc = cadd(acc, p);
    }
    out[o] = acc;
  }
#pragma unroll
  for (int o = 0; o < R; o++) v[o] = out[o];
}

template <>
__device__ __forceinline__ void Radix<3>::dft(float2* v, bool inv) {
  const float c[3] = {1.f, -0.5f, -0.5f};
  const float s[3] = {0.f, 0.86602540378443864676f, -0.86602540378443864676f};
  odd_dft<3>(v, inv, c, s);
}
template <>
__device__ __forceinline__ void Radix<5>::dft(float2* v, bool inv) {
  const float c[5] = {1.f, 0.30901699437494742410f, -0.80901699437494742410f, -0.80901699437494742410f,
                      0.30901699437494742410f};
  const float s[5] = {0.f, 0.95105651629515357212f, 0.58778525229247312917f, -0.58778525229247312917f,
                      -0.95105651629515357212f};
  odd_dft<5>(v, inv, c, s);
}
template <>
__device__ __forceinline__ void Radix<7>::dft(float2* v, bool inv) {
  const float c[7] = {1.f, 0.62348980185873353053f, -0.22252093395631440429f, -0.90096886790241912624f,
                      -0.90096886790241912624f, -0.22252093395631440429f, 0.62348980185873353053f};
  const float s[7] = {0.f, 0.78183148246802980871f, 0.97492791218182360702f, 0.43388373911755812048f,
                      -0.43388373911755812048f, -0.97492791218182360702f, -0.78183148246802980871f};
  odd_dft<7>(v, inv, c, s);
}

// Division by a runtime constant d through a multiply-high
// (round-up method; exact for n < 2^31).
struct FDiv {
  unsigned d, m, s;
};
__host__ __device__ inline FDiv make_fdiv(unsigned d) {
  FDiv f;
  f.d = d;
  unsigned l = 0;
  while ((1ull << l) < d) l++;
  f.s = l;
  f.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  return f;
}
__device__ __forceinline__ unsigned fdiv(const FDiv& f, unsigned n) { return (__umulhi(f.m, n) + n) >> f.s; }

// Tile addressing: element i of line l lives at s[i * si + l * sl].
// 'lfast' selects the thread mapping: consecutive threads walk lines
// (index-major tiles, sl == 1) or indices (line-major tiles, si == 1).
// POW2: the line length and the line count are powers of two and every
// radix is 2, 4 or 8, so index arithmetic reduces to shifts and masks
// (lgL = log2 L, lgl = log2 nlines).
template <int R, int EPT, bool POW2>
__device__ __forceinline__ void fft_stage(float2* s, int L, int lgL, int ns, int lgns, int nlines, const FDiv& fl,
                                          int si, int sl, bool lfast, const float2* __restrict__ tw, int tws,
                                          bool inv) {
  constexpr int IT = (EPT + R - 1) / R;
  constexpr int LGR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 0;
  const int m = POW2 ? (L >> LGR) : L / R;
  const int lgm = lgL - LGR;
  const int total = m * nlines;
  const int nt = blockDim.x;
  const int tid = threadIdx.x;
  float2 v[IT][R];
  const int tstep = POW2 ? (L >> (lgns + LGR)) : L / (ns * R);
#pragma unroll
  for (int it = 0; it < IT; it++) {
    int item = it * nt + tid;
    if (item < total) {
      int l, j;
      if (lfast) { j = (int)fdiv(fl, (unsigned)item); l = item - j * nlines; }
      else if (POW2) { j = item & (m - 1); l = item >> lgm; }
      else { j = item % m; l = item / m; }
      const float2* src = s + l * sl;
      int k = POW2 ? (j & (ns - 1)) : j % ns;
#pragma unroll
      for (int q = 0; q < R; q++) v[it][q] = src[(j + q * m) * si];
      if (ns > 1) {
#pragma unroll
        for (int q = 1; q < R; q++) {
          float2 w = __ldg(&tw[(q * k * tstep) * tws]);
          if (inv) w.y = -w.y;
          v[it][q] = cmul(v[it][q], w);
        }
      }
      Radix<R>::dft(v[it], inv);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; it++) {
    int item = it * nt + tid;
    if (item < total) {
      int l, j;
      if (lfast) { j = (int)fdiv(fl, (unsigned)item); l = item - j * nlines; }
      else if (POW2) { j = item & (m - 1); l = item >> lgm; }
      else { j = item % m; l = item / m; }
      float2* dst = s + l * sl;
      int base;
      if (POW2) base = ((j >> lgns) << (lgns + LGR)) + (j & (ns - 1));
      else base = (j / ns) * ns * R + j % ns;
#pragma unroll
      for (int q = 0; q < R; q++) dst[(base + q * ns) * si] = v[it][q];
    }
  }
  __syncthreads();
}

// Full transform of every line of the tile (unnormalised).
template <int EPT, bool POW2>
__device__ void tile_fft(float2* s, const LineFFT& f, int nlines, int si, int sl, bool lfast, bool inv) {
  int ns = 1, lgns = 0;
  int lgL = POW2 ? 31 - __clz(f.L) : 0;
  const FDiv fl = make_fdiv((unsigned)nlines);
  const unsigned long long code = f.code;
  for (int st = 0; st < f.nst; st++) {
    int c = (int)((code >> (3 * st)) & 7ull);
    int R = FFT_RADIX_OF(c);
    if (POW2) {
      switch (R) {
        case 8: fft_stage<8, EPT, true>(s, f.L, lgL, ns, lgns, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 4: fft_stage<4, EPT, true>(s, f.L, lgL, ns, lgns, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        default: fft_stage<2, EPT, true>(s, f.L, lgL, ns, lgns, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
      }
      lgns += R == 8 ? 3 : R == 4 ? 2 : 1;
    } else {
      switch (R) {
        case 8: fft_stage<8, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 4: fft_stage<4, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 2: fft_stage<2, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 3: fft_stage<3, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 5: fft_stage<5, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        case 7: fft_stage<7, EPT, false>(s, f.L, 0, ns, 0, nlines, fl, si, sl, lfast, f.tw, f.tws, inv); break;
        default: break;
      }
    }
    ns *= R;
  }
}

// Launch shapes: THREADS x EPT elements per tile; (256 x 8), (256 x 16)
// or (512 x 16).  The register budget is 128 per thread in all three.
#define FFT_BOUNDS(THREADS) __launch_bounds__(THREADS, (THREADS) == 256 ? 2 : 1)

static inline bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

// ---------------------------------------------------------------------
// Host-side plan construction helpers (fft_engine.cu).
// ---------------------------------------------------------------------
// Factor L into the supported radices (8 first, then 4, 2, 3, 5, 7).
// Returns false if L has another prime factor or too many stages.
bool fft_factor(int L, LineFFT* f);
// Device twiddle table exp(-2 pi i t / Lt), t < Lt, cached per length for
// the lifetime of the process.
const float2* fft_twiddles(int Lt);
