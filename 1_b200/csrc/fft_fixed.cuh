// Compile-time line FFTs for the hot passes.
//
// Same Stockham (self-sorting, decimation in time) formulation as
// fft_engine.cuh, but with the line length L, the radix of every stage, the
// tile shape and the thread count known at compile time, so every index is
// a shift or a mask and every loop unrolls.  A stage keeps its butterflies
// in registers: the first stage of a transform may load straight from
// global memory (zero padding is a predicate, not a load) and the last may
// store straight to global memory (pruned outputs are not stored), so a
// transform of R^s points makes s-1 round trips through shared memory.
//
// Radix plan: radix-16 or radix-8 stages first, then 4 or 2, then 3, 5, 7
// (a line length is any product of these); the inverse applies the stages in
// reverse order, so that the last forward stage and the first inverse stage
// group the same elements in the same thread (the kernel multiplication
// between them stays in registers).
#pragma once
#include "fft_engine.cuh"

// FMA complex multiply (the transforms need not be bit-reproducible against
// a CPU, only deterministic, which a fixed instruction sequence is)
__device__ __forceinline__ float2 cmul_f(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc_f(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}

__host__ __device__ constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x >> 1); }
// Radix plan of a line length L = 2^a 3^b 5^c 7^d: radix 8 while 8 divides
// the rest, then 4 or 2, then the odd radices.
__host__ __device__ constexpr int first_radix8(int L) {
  return L % 8 == 0 ? 8 : L % 4 == 0 ? 4 : L % 2 == 0 ? 2 : L % 3 == 0 ? 3 : L % 5 == 0 ? 5 : 7;
}
__host__ __device__ constexpr int n_stages8(int L) { return L <= 1 ? 0 : 1 + n_stages8(L / first_radix8(L)); }
// Radix 16 first when it saves a stage (one shared-memory round trip),
// e.g. 256 = 16*16 instead of 8*8*4.
__host__ __device__ constexpr int n_stages(int L);
__host__ __device__ constexpr int first_radix(int L) {
  return (L % 16 == 0 && 1 + n_stages(L / 16) < n_stages8(L)) ? 16 : first_radix8(L);
}
__host__ __device__ constexpr int n_stages(int L) { return L <= 1 ? 0 : 1 + n_stages(L / first_radix(L)); }
// radix of forward stage st
__host__ __device__ constexpr int fwd_radix(int L, int st) {
  return st == 0 ? first_radix(L) : fwd_radix(L / first_radix(L), st - 1);
}
// radix of inverse stage st (reverse order)
__host__ __device__ constexpr int inv_radix(int L, int st) { return fwd_radix(L, n_stages(L) - 1 - st); }
// span (product of the radices applied before stage st)
__host__ __device__ constexpr int fwd_span(int L, int st) { return st == 0 ? 1 : fwd_span(L, st - 1) * fwd_radix(L, st - 1); }
__host__ __device__ constexpr int inv_span(int L, int st) { return st == 0 ? 1 : inv_span(L, st - 1) * inv_radix(L, st - 1); }

// Twiddle table in shared memory: tw[t] = exp(-2 pi i t / L), t < L.
template <int L, int T>
__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ g, int gstride) {
  for (int t = threadIdx.x; t < L; t += T) tw[t] = __ldg(&g[t * gstride]);
}

// Butterfly bookkeeping of a stage of radix R at span NS over a tile of TK
// lines of length L; butterfly b (0 <= b < TK*L/R) of thread tid is
// b = tid + i*T.  LFAST: consecutive butterflies walk the lines (l fastest).
template <int L, int R, int NS, int TK, int T, bool LFAST>
struct St {
  static constexpr int M = L / R;
  static constexpr int NB = (TK * M + T - 1) / T;
  static constexpr int TSTEP = L / (NS * R);
  __device__ __forceinline__ static bool valid(int i) { return (TK * M) % T == 0 || threadIdx.x + i * T < TK * M; }
  __device__ __forceinline__ static void lj(int i, int& l, int& j) {
    int b = threadIdx.x + i * T;  // TK and M are compile-time constants
    if (LFAST) {
      l = b % TK;
      j = b / TK;
    } else {
      j = b % M;
      l = b / M;
    }
  }
  // output index of element q of butterfly j
  __device__ __forceinline__ static int out_idx(int j, int q) { return ((j / NS) * NS * R) + (j % NS) + q * NS; }
  __device__ __forceinline__ static int in_idx(int j, int q) { return j + q * M; }
  __device__ __forceinline__ static void twiddle(float2* v, int j, const float2* tw, bool inv) {
    if (NS == 1) return;
    int k = j % NS;
#pragma unroll
    for (int q = 1; q < R; q++) {
      float2 w = tw[q * k * TSTEP];
      v[q] = inv ? cmulc_f(v[q], w) : cmul_f(v[q], w);
    }
  }
  // the same, from a table in [q][k] order: tw[q * NS + k] = W^(q k TSTEP)
  __device__ __forceinline__ static void twiddle_qk(float2* v, int j, const float2* tw, bool inv) {
    static_assert(NS * R == L, "a [q][k] table holds the last stage's twiddles");
    if (NS == 1) return;
    int k = j % NS;
#pragma unroll
    for (int q = 1; q < R; q++) {
      float2 w = tw[q * NS + k];
      v[q] = inv ? cmulc_f(v[q], w) : cmul_f(v[q], w);
    }
  }
};

template <int R>
__device__ __forceinline__ void dft(float2* v, bool inv) {
  Radix<R>::dft(v, inv);
}

// Generic smem-to-smem stage over a tile: element (l, i) at s[i*SI + l*SL].
template <int L, int R, int NS, int TK, int T, bool LFAST, int SI, int SL>
__device__ __forceinline__ void stage_smem(float2* s, const float2* tw, bool inv) {
  using S = St<L, R, NS, TK, T, LFAST>;
  float2 v[S::NB][R];
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R; q++) v[i][q] = s[S::in_idx(j, q) * SI + l * SL];
    S::twiddle(v[i], j, tw, inv);
    dft<R>(v[i], inv);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R; q++) s[S::out_idx(j, q) * SI + l * SL] = v[i][q];
  }
  __syncthreads();
}

// Middle stages [ST0, ST1) of a forward (INV=false) or inverse transform,
// all in shared memory.
template <int L, int ST, int ST1, int TK, int T, bool LFAST, int SI, int SL, bool INV>
struct MidStages {
  __device__ __forceinline__ static void run(float2* s, const float2* tw) {
    if constexpr (ST < ST1) {
      constexpr int R = INV ? inv_radix(L, ST) : fwd_radix(L, ST);
      constexpr int NS = INV ? inv_span(L, ST) : fwd_span(L, ST);
      stage_smem<L, R, NS, TK, T, LFAST, SI, SL>(s, tw, INV);
      MidStages<L, ST + 1, ST1, TK, T, LFAST, SI, SL, INV>::run(s, tw);
    }
  }
};

// Full transform of the tile in shared memory (all stages smem to smem).
template <int L, int TK, int T, bool LFAST, int SI, int SL, bool INV>
__device__ __forceinline__ void tile_fft_fixed(float2* s, const float2* tw) {
  MidStages<L, 0, n_stages(L), TK, T, LFAST, SI, SL, INV>::run(s, tw);
}

// ---------------------------------------------------------------------
// Row tiles: NLINES lines of L stored row-major with one float2 of padding
// per 16 (element (l, i) at l*PITCH + i + i/16), butterflies mapped with j
// fastest.  The first stage of a Z transform then reads 16 consecutive
// elements of one row per half-warp straight from global memory
// (coalesced), and every shared-memory stage (stride-R first-stage writes
// included) is free of bank conflicts.
// ---------------------------------------------------------------------
__host__ __device__ constexpr int row_pitch(int L) {
  return (L + L / 16) % 16 == 0 ? L + L / 16 + 8 : L + L / 16;
}
__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }

// Row tiles map butterflies j-fastest, so the lanes of a half-warp read the
// twiddles tw[q k] for consecutive k: entries q apart, a gcd(q, 16)-way bank
// conflict for even q.  When the only stage with twiddles is the second of
// two equal-radix stages (256 = 16 * 16, 64 = 8 * 8; the same stage shape in
// the forward and the inverse transform), the table is kept in [q][k] order
// instead (QK) and a half-warp reads consecutive entries.
template <int L>
__host__ __device__ constexpr bool rows_qk() {
  return n_stages(L) == 2 && fwd_radix(L, 0) == fwd_radix(L, 1);
}
template <int L, int T>
__device__ __forceinline__ void load_twiddles_rows(float2* tw, const float2* __restrict__ g, int gstride) {
  if constexpr (rows_qk<L>()) {
    constexpr int R = fwd_radix(L, 0);
    for (int e = threadIdx.x; e < L; e += T) tw[e] = __ldg(&g[(e / R) * (e % R) * gstride]);
  } else {
    load_twiddles<L, T>(tw, g, gstride);
  }
}

template <int L, int R, int NS, int NLINES, int T, int PITCH, bool QK = false>
__device__ __forceinline__ void stage_rows(float2* s, const float2* tw, bool inv) {
  using S = St<L, R, NS, NLINES, T, false>;
  float2 v[S::NB][R];
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R; q++) v[i][q] = s[l * PITCH + padi(S::in_idx(j, q))];
    if constexpr (QK) S::twiddle_qk(v[i], j, tw, inv);
    else S::twiddle(v[i], j, tw, inv);
    dft<R>(v[i], inv);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R; q++) s[l * PITCH + padi(S::out_idx(j, q))] = v[i][q];
  }
  __syncthreads();
}

// A row-tile stage whose outputs past L/2 are never read (the last inverse
// stage of a zero-padded line): only the lower half is computed and stored.
template <int L, int R, int NS, int NLINES, int T, int PITCH, bool QK = false>
__device__ __forceinline__ void stage_rows_lower(float2* s, const float2* tw, bool inv) {
  static_assert(NS * R == L, "the lower-half store is for the last stage");
  using S = St<L, R, NS, NLINES, T, false>;
  float2 v[S::NB][R];
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R; q++) v[i][q] = s[l * PITCH + padi(S::in_idx(j, q))];
    if constexpr (QK) S::twiddle_qk(v[i], j, tw, inv);
    else S::twiddle(v[i], j, tw, inv);
    dft<R>(v[i], inv);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < S::NB; i++) {
    if (!S::valid(i)) continue;
    int l, j;
    S::lj(i, l, j);
#pragma unroll
    for (int q = 0; q < R / 2; q++) s[l * PITCH + padi(S::out_idx(j, q))] = v[i][q];
  }
  __syncthreads();
}

// stages [ST, ST1) of a forward or inverse transform of a row tile
template <int L, int ST, int ST1, int NLINES, int T, int PITCH, bool INV, bool QK = false>
struct MidRows {
  __device__ __forceinline__ static void run(float2* s, const float2* tw) {
    if constexpr (ST < ST1) {
      constexpr int R = INV ? inv_radix(L, ST) : fwd_radix(L, ST);
      constexpr int NS = INV ? inv_span(L, ST) : fwd_span(L, ST);
      stage_rows<L, R, NS, NLINES, T, PITCH, QK>(s, tw, INV);
      MidRows<L, ST + 1, ST1, NLINES, T, PITCH, INV, QK>::run(s, tw);
    }
  }
};

