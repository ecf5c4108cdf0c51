// Fixed-size pass kernels of the zero-aware padded FFT.
// Drop-in replacements for k_col / k_z_r2c / k_z_c2r (fft_passes.cuh) and
// for the fused k_xconv / k_yconv2d / k_zinv_epi (solver.cu) when the line
// length has compiled kernels (FX_SIZES).
#pragma once
#include "epilogue.cuh"
#include "kernmul.cuh"
#include "fft_fixed.cuh"
#include "fft_passes.cuh"

// Row pitch of an index-major tile: odd, so that rows a power of two apart
// fall on different shared-memory banks.
__host__ __device__ constexpr int odd_pitch(int lines) { return (lines % 2) ? lines : lines + 1; }

// ---------------------------------------------------------------------
// Column pass: TK adjacent columns x L, index-major tile (s[i*TKP + l],
// TKP = odd_pitch(TK)).
// Stage 0 loads from global (rows >= n_in are zero), the last stage stores
// to global (only rows < n_out).
// ---------------------------------------------------------------------
// HALF: forward, the input holds data in its lower half only (n_in = L/2);
// inverse, only the lower half of the output is kept (n_out = L/2).
template <int L, int TK, int T, bool INV, bool HALF>
__device__ __forceinline__ void col_body(const float2* src, float2* dst, const ColPass& cp, int tile) {
  __shared__ float2 tw[L];
  extern __shared__ float2 sm[];
  constexpr int NST = n_stages(L);
  constexpr int TKP = odd_pitch(TK);
  load_twiddles<L, T>(tw, cp.f.tw, cp.f.tws);
  // Tiles run over the flattened columns of all planes: column g is column
  // g % ncols of plane g / ncols, so a tile may straddle two planes and no
  // tile at the end of a plane is left mostly empty.
  const int nall = cp.nplanes * cp.ncols;
  auto col_at = [&](int l, int64_t& base) -> bool {
    const int g = tile * TK + l;
    const int pl = g / cp.ncols;
    base = (int64_t)pl * cp.plane_stride + (g - pl * cp.ncols);
    return g < nall;
  };
  // T % TK == 0: every butterfly of a thread is in the same column
  int64_t base0;
  const bool ok0 = col_at((int)threadIdx.x % TK, base0);
  const int64_t sti = cp.stride_i;
  const int n_in = cp.n_in, n_out = cp.n_out;
  constexpr int R0 = INV ? inv_radix(L, 0) : fwd_radix(L, 0);
  using S0 = St<L, R0, 1, TK, T, true>;
  float2 v[S0::NB][R0];
#pragma unroll
  for (int i = 0; i < S0::NB; i++) {
    if (!S0::valid(i)) continue;
    int l, j;
    S0::lj(i, l, j);
    int64_t cbase = base0;
    bool ok = ok0;
    if constexpr (T % TK != 0) ok = col_at(l, cbase);
#pragma unroll
    for (int q = 0; q < R0; q++) {
      int idx = S0::in_idx(j, q);
      v[i][q] = (((HALF && !INV) ? q < R0 / 2 : idx < n_in) && ok) ? src[cbase + idx * sti]
                                                                        : make_float2(0.f, 0.f);
    }
    if (HALF && !INV) dft_half<R0>(v[i], INV);
    else dft<R0>(v[i], INV);
  }
  if constexpr (NST == 1) {
#pragma unroll
    for (int i = 0; i < S0::NB; i++) {
      if (!S0::valid(i)) continue;
      int l, j;
      S0::lj(i, l, j);
      int64_t cbase = base0;
      bool ok = ok0;
      if constexpr (T % TK != 0) ok = col_at(l, cbase);
#pragma unroll
      for (int q = 0; q < R0; q++) {
        int idx = S0::out_idx(j, q);
        if (((HALF && INV) ? q < R0 / 2 : idx < n_out) && ok) dst[cbase + idx * sti] = v[i][q];
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < S0::NB; i++) {
      if (!S0::valid(i)) continue;
      int l, j;
      S0::lj(i, l, j);
#pragma unroll
      for (int q = 0; q < R0; q++) sm[S0::out_idx(j, q) * TKP + l] = v[i][q];
    }
    __syncthreads();
    MidStages<L, 1, NST - 1, TK, T, true, TKP, 1, INV>::run(sm, tw);
    constexpr int RL = INV ? inv_radix(L, NST - 1) : fwd_radix(L, NST - 1);
    constexpr int NSL = INV ? inv_span(L, NST - 1) : fwd_span(L, NST - 1);
    using SL = St<L, RL, NSL, TK, T, true>;
    float2 w[SL::NB][RL];
#pragma unroll
    for (int i = 0; i < SL::NB; i++) {
      if (!SL::valid(i)) continue;
      int l, j;
      SL::lj(i, l, j);
      int64_t cbase = base0;
      bool ok = ok0;
      if constexpr (T % TK != 0) ok = col_at(l, cbase);
#pragma unroll
      for (int q = 0; q < RL; q++) w[i][q] = sm[SL::in_idx(j, q) * TKP + l];
      SL::twiddle(w[i], j, tw, INV);
      dft<RL>(w[i], INV);
#pragma unroll
      for (int q = 0; q < RL; q++) {
        int idx = SL::out_idx(j, q);
        if (((HALF && INV) ? q < RL / 2 : idx < n_out) && ok) dst[cbase + idx * sti] = w[i][q];
      }
    }
  }
}

template <int L, int TK, int T, bool INV, bool HALF>
__global__ void __launch_bounds__(T) k_col_fx(const float2* src, float2* dst, ColPass cp) {
  col_body<L, TK, T, INV, HALF>(src, dst, cp, blockIdx.x);
}

// ---------------------------------------------------------------------
// Fused convolution pass: forward transform of the three components along
// the padded axis, multiplication by the symmetric kernel, inverse
// transform.  3D (D2 = false): X axis, columns = flattened (ky, kz);
// 2D (D2 = true): Y axis, columns = kz.  Tile element (c, t, i) at
// sm[i * 3TK + c * TK + t].  The last forward stage, the kernel product and
// the first inverse stage stay in the registers of one thread, which owns
// the three components of its (column, butterfly).
// ---------------------------------------------------------------------
struct ConvArgs {
  float2* S;
  KernOct K;
  int n_data;       // data rows along the transformed axis (N0 or N1)
  int ncols;        // P1*HZ (3D) or HZ (2D)
  int HZ;
  int64_t stride;   // element stride along the transformed axis
  int64_t CS;       // component stride
  const float2* tw; // twiddles of the transformed length
  int tws;
};

template <int L, int R, int NS, int TK, int T>
using St3 = St<L, R, NS, TK, T, true>;  // (t, j) butterflies, components looped inside

// HALF: the line holds data in its lower half only (n_data = L/2, the
// open-boundary case): the first stage skips the zero half and the last
// inverse stage computes only the stored half.
// STREAM: the spectrum is read and written with evict-first cache hints, so
// that the kernel octant (read once for ky and once for P1 - ky, a pass
// apart) stays in L2 for its second read.  Set for the single-grid 3D pass
// only: there the X convolution gains more (75.3 -> 72.7 us on the 256 x 256
// x 32 grid) than the inverse Y pass loses by reading its input from DRAM
// (38.2 -> 39.2 us).
template <int L, int TK, int T, bool D2, bool HALF, bool STREAM = false>
__device__ __forceinline__ void conv_body(const ConvArgs& a, int bx) {
  auto sload = [](const float2* p) -> float2 { return STREAM ? __ldcs(p) : *p; };
  auto sstore = [](float2* p, float2 v) {
    if (STREAM) __stcs(p, v);
    else *p = v;
  };
  __shared__ float2 tw[L];
  extern __shared__ float2 sm[];
  constexpr int NST = n_stages(L);
  constexpr int NL = 3 * TK;
  constexpr int NLP = odd_pitch(NL);
  load_twiddles<L, T>(tw, a.tw, a.tws);
  const int col0 = bx * TK;
  const int nc = min(TK, a.ncols - col0);
  const int nd = a.n_data;
  // ---- forward stage 0 from global ----
  constexpr int R0 = fwd_radix(L, 0);
  using S0 = St3<L, R0, 1, TK, T>;
  // ---- registers of the last forward / first inverse stage ----
  constexpr int RL = fwd_radix(L, NST - 1);
  constexpr int NSL = fwd_span(L, NST - 1);
  using SL = St3<L, RL, NSL, TK, T>;
  float2 v[SL::NB][3][RL];
  if constexpr (NST == 1) {
#pragma unroll
    for (int i = 0; i < S0::NB; i++) {
      if (!S0::valid(i)) continue;
      int t, j;
      S0::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
#pragma unroll
        for (int q = 0; q < R0; q++) {
          int idx = S0::in_idx(j, q);
          v[i][c][q] = ((HALF ? q < R0 / 2 : idx < nd) && t < nc) ? sload(&a.S[c * a.CS + idx * a.stride + col0 + t])
                                                                  : make_float2(0.f, 0.f);
        }
        if (HALF) dft_half<R0>(v[i][c], false);
        else dft<R0>(v[i][c], false);
      }
    }
  } else {
    float2 u[S0::NB][3][R0];
#pragma unroll
    for (int i = 0; i < S0::NB; i++) {
      if (!S0::valid(i)) continue;
      int t, j;
      S0::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
#pragma unroll
        for (int q = 0; q < R0; q++) {
          int idx = S0::in_idx(j, q);
          u[i][c][q] = ((HALF ? q < R0 / 2 : idx < nd) && t < nc) ? sload(&a.S[c * a.CS + idx * a.stride + col0 + t])
                                                                  : make_float2(0.f, 0.f);
        }
        if (HALF) dft_half<R0>(u[i][c], false);
        else dft<R0>(u[i][c], false);
#pragma unroll
        for (int q = 0; q < R0; q++) sm[S0::out_idx(j, q) * NLP + c * TK + t] = u[i][c][q];
      }
    }
    __syncthreads();
    MidStages<L, 1, NST - 1, NL, T, true, NLP, 1, false>::run(sm, tw);
#pragma unroll
    for (int i = 0; i < SL::NB; i++) {
      if (!SL::valid(i)) continue;
      int t, j;
      SL::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
#pragma unroll
        for (int q = 0; q < RL; q++) v[i][c][q] = sm[SL::in_idx(j, q) * NLP + c * TK + t];
        SL::twiddle(v[i][c], j, tw, false);
        dft<RL>(v[i][c], false);
      }
    }
  }
  // ---- kernel multiplication, H = K M per bin ----
#pragma unroll
  for (int i = 0; i < SL::NB; i++) {
    if (!SL::valid(i)) continue;
    int t, j;
    SL::lj(i, t, j);
    if (t >= nc) continue;
    int col = col0 + t;
    int kyc, kzc;
    if (D2) { kyc = 0; kzc = col; }
    else { kyc = col / a.HZ; kzc = col - kyc * a.HZ; }
#pragma unroll
    for (int q = 0; q < RL; q++) {
      int k = SL::out_idx(j, q);
      float Kxx, Kyy, Kzz, Kyz, Kxz, Kxy;
      if (D2) {
        kern_at(a.K, 0, k, kzc, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
        kmul4_fma(v[i][0][q], v[i][1][q], v[i][2][q], Kxx, Kyy, Kzz, Kyz);
      } else {
        kern_at(a.K, k, kyc, kzc, Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
        kmul6_fma(v[i][0][q], v[i][1][q], v[i][2][q], Kxx, Kyy, Kzz, Kyz, Kxz, Kxy);
      }
    }
  }
  // ---- inverse: first stage in registers (same grouping) ----
  if constexpr (NST == 1) {
#pragma unroll
    for (int i = 0; i < SL::NB; i++) {
      if (!SL::valid(i)) continue;
      int t, j;
      SL::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        dft<RL>(v[i][c], true);
#pragma unroll
        for (int q = 0; q < RL; q++) {
          int idx = SL::out_idx(j, q);
          if ((HALF ? q < RL / 2 : idx < nd) && t < nc) sstore(&a.S[c * a.CS + idx * a.stride + col0 + t], v[i][c][q]);
        }
      }
    }
  } else {
    using I0 = St3<L, inv_radix(L, 0), 1, TK, T>;  // same radix and butterflies as SL
    static_assert(inv_radix(L, 0) == RL && I0::M == NSL, "grouping mismatch");
    __syncthreads();  // the last forward stage read the tile
#pragma unroll
    for (int i = 0; i < SL::NB; i++) {
      if (!SL::valid(i)) continue;
      int t, j;
      SL::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        dft<RL>(v[i][c], true);
#pragma unroll
        for (int q = 0; q < RL; q++) sm[I0::out_idx(j, q) * NLP + c * TK + t] = v[i][c][q];
      }
    }
    __syncthreads();
    MidStages<L, 1, NST - 1, NL, T, true, NLP, 1, true>::run(sm, tw);
    constexpr int RI = inv_radix(L, NST - 1);
    constexpr int NSI = inv_span(L, NST - 1);
    using SI = St3<L, RI, NSI, TK, T>;
#pragma unroll
    for (int i = 0; i < SI::NB; i++) {
      if (!SI::valid(i)) continue;
      int t, j;
      SI::lj(i, t, j);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float2 w[RI];
#pragma unroll
        for (int q = 0; q < RI; q++) w[q] = sm[SI::in_idx(j, q) * NLP + c * TK + t];
        SI::twiddle(w, j, tw, true);
        dft<RI>(w, true);
#pragma unroll
        for (int q = 0; q < RI; q++) {
          int idx = SI::out_idx(j, q);
          if ((HALF ? q < RI / 2 : idx < nd) && t < nc) sstore(&a.S[c * a.CS + idx * a.stride + col0 + t], w[q]);
        }
      }
    }
  }
}

template <int L, int TK, int T, bool D2, bool HALF>
// at least 768 resident threads per SM (6 blocks of 128 for L = 64):
// measured faster than the unconstrained 96-register build (5 blocks) and
// than 7 or 8 blocks (register spills)
__global__ void __launch_bounds__(T, (768 / T) > 0 ? (768 / T) : 1) k_conv_fx(ConvArgs a) {
  conv_body<L, TK, T, D2, HALF, !D2>(a, blockIdx.x);
}

// ---------------------------------------------------------------------
// Z rows.  Tile index-major with an odd row pitch: element n of line l at
// sm[n * SIP + l]; global accesses walk the row (coalesced), stages walk
// the lines (conflict-free).
// ---------------------------------------------------------------------

template <int M, int RT, int T, bool COMB>
__device__ __forceinline__ void zr2c_body(const float* __restrict__ src, float2* __restrict__ dst, const ZPass& z,
                                          const ZComb& cb, int vec2, int bx) {
  __shared__ float2 tw[M];
  __shared__ int64_t roff_s[RT], soff_s[RT];
  extern __shared__ float2 sm[];
  constexpr int PITCH = row_pitch(M);
  constexpr int NST = n_stages(M);
  constexpr bool QK = rows_qk<M>();
  load_twiddles_rows<M, T>(tw, z.f.tw, z.f.tws);
  const int r0 = bx * RT;
  const int nl = min(RT, z.nrows - r0);
  if (threadIdx.x < RT) {
    int64_t ro = 0, so = 0;
    if ((int)threadIdx.x < nl) zrow_offsets(z, r0 + threadIdx.x, &ro, &so);
    roff_s[threadIdx.x] = ro;
    soff_s[threadIdx.x] = so;
  }
  __syncthreads();
  const float dt = COMB ? *cb.dt : 0.f;
  const int nreal = z.n_real;
  // first stage straight from global memory: butterfly j of row l reads the
  // pairs (x_2n, x_2n+1), n = j + q M/R0 (zero past the data)
  constexpr int R0 = fwd_radix(M, 0);
  using S0 = St<M, R0, 1, RT, T, false>;
#pragma unroll
  for (int i = 0; i < S0::NB; i++) {
    if (!S0::valid(i)) continue;
    int l, j;
    S0::lj(i, l, j);
    float2 v[R0];
#pragma unroll
    for (int q = 0; q < R0; q++) {
      const int n = S0::in_idx(j, q);
      float a = 0.f, b = 0.f;
      if (l < nl) {
        const int64_t roff = roff_s[l];
        const int i0 = 2 * n;
        if (COMB && vec2 && i0 + 1 < nreal) {
          const float2 p = zcomb_value2(cb, dt, roff + i0);
          *reinterpret_cast<float2*>(cb.out + roff + i0) = p;
          a = p.x;
          b = p.y;
        } else if (COMB) {
          if (i0 < nreal) { a = zcomb_value(cb, dt, roff + i0); cb.out[roff + i0] = a; }
          if (i0 + 1 < nreal) { b = zcomb_value(cb, dt, roff + i0 + 1); cb.out[roff + i0 + 1] = b; }
        } else if (vec2 && i0 + 1 < nreal) {
          float2 p = __ldg(reinterpret_cast<const float2*>(src + roff + i0));
          a = p.x;
          b = p.y;
        } else {
          if (i0 < nreal) a = src[roff + i0];
          if (i0 + 1 < nreal) b = src[roff + i0 + 1];
        }
      }
      v[q] = make_float2(a, b);
    }
    // open boundary (n_real = M): the upper half of the pairs is padding
    if (nreal == M) dft_half<R0>(v, false);
    else dft<R0>(v, false);
#pragma unroll
    for (int q = 0; q < R0; q++) sm[l * PITCH + padi(S0::out_idx(j, q))] = v[q];
  }
  __syncthreads();
  MidRows<M, 1, NST, RT, T, PITCH, false, QK>::run(sm, tw);
  // R2C split, one thread per pair (k, M - k), k <= M/2:
  // X_k = E_k + w^k O_k and X_{M-k} = conj(E_k - w^k O_k)
  constexpr int HP = M / 2 + 1;
  for (int e = threadIdx.x; e < nl * HP; e += T) {
    int l = e / HP, k = e - l * HP;
    float2 Zk = sm[l * PITCH + padi(k)];
    float2 Zm = sm[l * PITCH + padi(k == 0 ? 0 : M - k)];
    float2 E = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    float2 O = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
    float2 wo = cmul_f(__ldg(&z.twP[k]), O);
    float2* row = dst + soff_s[l];
    row[k] = make_float2(E.x + wo.x, E.y + wo.y);
    if (k < M / 2) row[M - k] = make_float2(E.x - wo.x, wo.y - E.y);
  }
}

template <int M, int RT, int T, bool COMB>
__global__ void __launch_bounds__(T) k_zr2c_fx(const float* __restrict__ src, float2* __restrict__ dst, ZPass z,
                                               ZComb cb, int vec2) {
  zr2c_body<M, RT, T, COMB>(src, dst, z, cb, vec2, blockIdx.x);
}

// Z'_k = (X_k + conj X_{M-k}) + i (X_k - conj X_{M-k}) w^{-k}; X_0, X_M real
__device__ __forceinline__ float2 c2r_pre(float2 Xk, float2 Xm, int k, int M, const float2* __restrict__ twP) {
  if (k == 0) { Xk.y = 0.f; Xm.y = 0.f; }
  float2 A = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
  float2 B = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
  float2 w = __ldg(&twP[k]);
  float2 C = cmulc_f(B, w);
  return make_float2(A.x - C.y, A.y + C.x);
}

template <int M, int RT, int T>
__global__ void __launch_bounds__(T) k_zc2r_fx(const float2* __restrict__ src, float* __restrict__ dst, ZPass z) {
  __shared__ float2 tw[M];
  extern __shared__ float2 sm[];
  constexpr int SIP = odd_pitch(RT);
  load_twiddles<M, T>(tw, z.f.tw, z.f.tws);
  const int r0 = blockIdx.x * RT;
  const int nl = min(RT, z.nrows - r0);
  for (int e = threadIdx.x; e < RT * M; e += T) {
    int l = e / M, k = e - l * M;
    float2 v = make_float2(0.f, 0.f);
    if (l < nl) {
      int64_t roff, soff;
      zrow_offsets(z, r0 + l, &roff, &soff);
      v = c2r_pre(src[soff + k], src[soff + M - k], k, M, z.twP);
    }
    sm[k * SIP + l] = v;
  }
  __syncthreads();
  tile_fft_fixed<M, RT, T, true, SIP, 1, true>(sm, tw);
  for (int e = threadIdx.x; e < nl * M; e += T) {
    int l = e / M, n = e - l * M;
    int i0 = 2 * n;
    if (i0 >= z.n_real) continue;
    int64_t roff, soff;
    zrow_offsets(z, r0 + l, &roff, &soff);
    float2 v = sm[n * SIP + l];
    dst[roff + i0] = v.x;
    if (i0 + 1 < z.n_real) dst[roff + i0 + 1] = v.y;
  }
}

// Inverse Z of the three components of RT spatial rows + the solver epilogue.
struct ZinvArgs {
  float2* S;
  const float2* twz;
  const float2* twP;
  int P1, HZ;
  int64_t CS;
  int nrows;
  EpiArgs ea;
};

// FUSE (Heun modes, open Z boundary): after the epilogue the block's new
// magnetisation rows (the next evaluation's input) are still in its shared
// tile, so the block also runs the next forward Z transform on them and
// writes the same spectrum rows it read -- the next evaluation needs no
// separate forward Z pass and never re-reads m.
template <int M, int RT, int T, int MODE, bool FUSE = false>
__device__ __forceinline__ void zinv_body(const ZinvArgs& za, int bx) {
  __shared__ float2 tw[M];
  __shared__ int64_t rbase_s[RT];
  extern __shared__ float2 sm[];
  constexpr int NL = 3 * RT;
  constexpr int PITCH = row_pitch(M);
  constexpr int NST = n_stages(M);
  const float2* S = za.S;  // not restrict: the fused variant writes these rows back
  const float2* __restrict__ twP = za.twP;
  const int P1 = za.P1, HZ = za.HZ, nrows = za.nrows;
  const int64_t CS = za.CS;
  const EpiArgs& ea = za.ea;
  constexpr bool QK = rows_qk<M>();
  load_twiddles_rows<M, T>(tw, za.twz, 2);
  const int r0 = bx * RT;
  const int nr = min(RT, nrows - r0);
  const int N1 = ea.N1, N2 = ea.N2;
  if (threadIdx.x < RT) {
    int gr = r0 + threadIdx.x;
    int x = gr / N1, y = gr - x * N1;
    rbase_s[threadIdx.x] = ((int64_t)x * P1 + y) * HZ;
  }
  __syncthreads();
  // first inverse stage straight from global memory: line l = 3 r + c,
  // butterfly j combines bins k = j + q M/R0 (each after the C2R split)
  constexpr int R0 = inv_radix(M, 0);
  using S0 = St<M, R0, 1, NL, T, false>;
#pragma unroll
  for (int i = 0; i < S0::NB; i++) {
    if (!S0::valid(i)) continue;
    int l, j;
    S0::lj(i, l, j);
    const int r = l / 3, c = l - 3 * r;
    float2 v[R0];
    const float2* row = S + c * CS + rbase_s[r < nr ? r : 0];
#pragma unroll
    for (int q = 0; q < R0; q++) {
      const int k = S0::in_idx(j, q);
      v[q] = (r < nr) ? c2r_pre(row[k], row[M - k], k, M, twP) : make_float2(0.f, 0.f);
    }
    dft<R0>(v, true);
#pragma unroll
    for (int q = 0; q < R0; q++) sm[l * PITCH + padi(S0::out_idx(j, q))] = v[q];
  }
  __syncthreads();
  if constexpr (NST >= 2) {
    if (N2 == M) {
      // open boundary: the cells use the lower half of each line only
      MidRows<M, 1, NST - 1, NL, T, PITCH, true, QK>::run(sm, tw);
      stage_rows_lower<M, inv_radix(M, NST - 1), inv_span(M, NST - 1), NL, T, PITCH, QK>(sm, tw, true);
    } else {
      MidRows<M, 1, NST, NL, T, PITCH, true, QK>::run(sm, tw);
    }
  } else {
    MidRows<M, 1, NST, NL, T, PITCH, true, QK>::run(sm, tw);
  }
  float lmax = 0.f;
  double eacc = 0.0;
  const int64_t g0 = (int64_t)r0 * N2;
  if (N2 == M) {
    // open boundary along Z: the row has exactly M cells.  Every per-cell
    // input of this thread's cells is loaded before any is used, so the
    // loads are in flight together.
    constexpr int CPT = (RT * M + T - 1) / T;
    EpiIn<MODE> in[CPT];
#pragma unroll
    for (int i = 0; i < CPT; i++) {
      int e = threadIdx.x + i * T;
      if (e < nr * M) epi_load<MODE>(ea, g0 + e, in[i]);
    }
#pragma unroll
    for (int i = 0; i < CPT; i++) {
      int e = threadIdx.x + i * T;
      if (e >= nr * M) continue;
      int r = e / M, zz = e % M;
      float2* base = sm + 3 * r * PITCH + padi(zz >> 1);
      float hx = (zz & 1) ? base[0].y : base[0].x;
      float hy = (zz & 1) ? base[PITCH].y : base[PITCH].x;
      float hz = (zz & 1) ? base[2 * PITCH].y : base[2 * PITCH].x;
      if constexpr (FUSE) {
        // the same 4-byte word that held this cell's field takes its new m
        float nm[3];
        epi_cell_in<MODE>(ea, g0 + e, hx, hy, hz, in[i], lmax, nm);
        float* w = reinterpret_cast<float*>(base) + (zz & 1);
        w[0] = nm[0];
        w[2 * PITCH] = nm[1];
        w[4 * PITCH] = nm[2];
      } else {
        epi_cell_in<MODE>(ea, g0 + e, hx, hy, hz, in[i], lmax, nullptr, &eacc);
      }
    }
    if constexpr (FUSE) {
      epi_flush_max<MODE>(ea, lmax);
      __syncthreads();
      // forward Z of the new rows: pairs n < M/2 hold the data, the rest of
      // each line is padding (zero); then the R2C split into the spectrum
      constexpr int F0 = fwd_radix(M, 0);
      using SF = St<M, F0, 1, NL, T, false>;
      float2 f[SF::NB][F0];
#pragma unroll
      for (int i = 0; i < SF::NB; i++) {
        if (!SF::valid(i)) continue;
        int l, j;
        SF::lj(i, l, j);
#pragma unroll
        for (int q = 0; q < F0; q++)
          f[i][q] = (q < F0 / 2) ? sm[l * PITCH + padi(SF::in_idx(j, q))] : make_float2(0.f, 0.f);
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < SF::NB; i++) {
        if (!SF::valid(i)) continue;
        int l, j;
        SF::lj(i, l, j);
        dft_half<F0>(f[i], false);
#pragma unroll
        for (int q = 0; q < F0; q++) sm[l * PITCH + padi(SF::out_idx(j, q))] = f[i][q];
      }
      __syncthreads();
      MidRows<M, 1, NST, NL, T, PITCH, false, QK>::run(sm, tw);
      // R2C split, one thread per pair (k, M - k), k <= M/2:
      // X_k = E_k + w^k O_k and X_{M-k} = conj(E_k - w^k O_k)
      constexpr int HP = M / 2 + 1;
      for (int e = threadIdx.x; e < 3 * nr * HP; e += T) {
        int l = e / HP, k = e - l * HP;
        int r = l / 3, c = l - 3 * r;
        float2 Zk = sm[l * PITCH + padi(k)];
        float2 Zm = sm[l * PITCH + padi(k == 0 ? 0 : M - k)];
        float2 E = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
        float2 O = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
        float2 wo = cmul_f(__ldg(&twP[k]), O);
        float2* row = za.S + c * CS + rbase_s[r];
        row[k] = make_float2(E.x + wo.x, E.y + wo.y);
        if (k < M / 2) row[M - k] = make_float2(E.x - wo.x, wo.y - E.y);
      }
      return;
    }
  } else {
    for (int e = threadIdx.x; e < nr * N2; e += T) {
      int r = e / N2, zz = e - r * N2;
      const float2* base = sm + 3 * r * PITCH + padi(zz >> 1);
      float hx = (zz & 1) ? base[0].y : base[0].x;
      float hy = (zz & 1) ? base[PITCH].y : base[PITCH].x;
      float hz = (zz & 1) ? base[2 * PITCH].y : base[2 * PITCH].x;
      epi_cell<MODE>(ea, g0 + e, hx, hy, hz, lmax, &eacc);
    }
  }
  epi_flush_max<MODE>(ea, lmax, eacc);
}

template <int M, int RT, int T, int MODE>
__global__ void __launch_bounds__(T) k_zinv_fx(ZinvArgs za) {
  zinv_body<M, RT, T, MODE>(za, blockIdx.x);
}
template <int M, int RT, int T, int MODE>
__global__ void __launch_bounds__(T) k_zinv_fwd_fx(ZinvArgs za) {
  zinv_body<M, RT, T, MODE, true>(za, blockIdx.x);
}

// ---------------------------------------------------------------------
// Launch-shape tables.  Every tile holds about 4096 complex values and
// every thread about 16 (512 threads for the longest lines).
// ---------------------------------------------------------------------
// line lengths with compiled kernels: 2^k (2..4096) and 3*2^k (6..3072)
#define FX_SIZES(X)                                                                                      \
  X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096) X(6) X(12) X(24) X(48) \
      X(96) X(192) X(384) X(768) X(1536) X(3072)
static inline bool fx_ok(int L) {
  if (L < 2) return false;
  int m = L % 3 == 0 ? L / 3 : L;
  return (m & (m - 1)) == 0 && L <= 4096;
}

// Columns per tile: at least 16 up to L = 512 so that a half-warp's 8-byte
// accesses cover one 128-byte row of the tile (no shared-memory bank
// conflicts) and global rows are read in 128-byte pieces.
__host__ __device__ constexpr int fx_col_tk(int L) {
  return L >= 4096 ? 1 : L >= 1024 ? 4096 / L : (4096 / L < 16 ? 16 : (4096 / L > 32 ? 32 : 4096 / L));
}
// columns per convolution tile (a power of two): about 1365/L, at most 16
// (16 columns measured faster than 8 for L = 64)
__host__ __device__ constexpr int conv_tk_raw(int L) {
  return L >= 2048 ? 1 : (1365 / L > 32 ? 32 : (1365 / L < 1 ? 1 : 1365 / L));
}
// butterflies per column in the last forward stage (one thread each)
__host__ __device__ constexpr int conv_bf(int L) { return L / fwd_radix(L, n_stages(L) - 1); }
// Lines whose last stage has fewer than 8 butterflies per column (L = 2, 4,
// 8, 16 in one stage; 6, 12 in two) take 128 / conv_bf columns, so that a
// block still has 128 busy threads: a 16-column tile of L = 8 left 48 of
// its 64 threads idle.
__host__ __device__ constexpr int conv_tkp_narrow(int L) {
  return conv_bf(L) < 8                   ? 128 / conv_bf(L)
         : conv_tk_raw(L) >= 16 ? 16
         : conv_tk_raw(L) >= 8            ? 8
         : conv_tk_raw(L) >= 4            ? 4
         : conv_tk_raw(L) >= 2            ? 2
                                          : 1;
}
// Single-grid passes: lines of 384 points and more also keep at least 4
// adjacent columns (up to 512 threads), so that a warp's accesses cover 8
// rows x 32 contiguous bytes of the spectrum and of the kernel; with one or
// two columns every lane read its own row (the 512 x 512 film's FP32 Y
// convolution: 45.8 -> 20.9 us).  The batch keeps the narrow tiles: its
// instances hold few columns each, and more, smaller blocks measured faster
// there.
__host__ __device__ constexpr int conv_tkp(int L) {
  return conv_tkp_narrow(L) >= 4 ? conv_tkp_narrow(L)
         : 512 / conv_bf(L) >= 4 ? 4
         : 512 / conv_bf(L) >= 2 ? 2
                                 : 1;
}
// shared-memory tile of a convolution block of TK columns (none for
// one-stage lines, whose butterflies stay in registers from load to store)
__host__ __device__ constexpr size_t conv_smem_tk(int L, int TK) {
  return n_stages(L) == 1 ? 0 : sizeof(float2) * (size_t)odd_pitch(3 * TK) * L;
}
__host__ __device__ constexpr size_t conv_smem(int L) { return conv_smem_tk(L, conv_tkp(L)); }
__host__ __device__ constexpr int fx_threads(int elems) {
  return elems / 16 < 64 ? 64 : (elems / 16 > 512 ? 512 : ((elems / 16 + 31) / 32) * 32);
}

template <int L, bool INV>
cudaError_t fx_launch_col(const float2* src, float2* dst, const ColPass& cp, cudaStream_t st) {
  constexpr int TK = fx_col_tk(L);
  constexpr int T = fx_threads(TK * L);
  size_t smem = sizeof(float2) * (size_t)odd_pitch(TK) * L;
  const int grid = div_up(cp.ncols * cp.nplanes, TK);
  const bool half = 2 * (INV ? cp.n_out : cp.n_in) == L;
  if (half) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_col_fx<L, TK, T, INV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_col_fx<L, TK, T, INV, true><<<grid, T, smem, st>>>(src, dst, cp);
  } else {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_col_fx<L, TK, T, INV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_col_fx<L, TK, T, INV, false><<<grid, T, smem, st>>>(src, dst, cp);
  }
  return cudaGetLastError();
}

template <int L, bool D2>
cudaError_t fx_launch_conv(const ConvArgs& a, cudaStream_t st) {
  constexpr int TKP = conv_tkp(L);
  // one thread per (column, radix-8 butterfly): it owns the three components
  constexpr int NBF = TKP * (L / fwd_radix(L, n_stages(L) - 1));
  constexpr int T = NBF < 64 ? 64 : (NBF > 512 ? 512 : ((NBF + 31) / 32) * 32);
  size_t smem = conv_smem(L);
  if (2 * a.n_data == L) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_conv_fx<L, TKP, T, D2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_conv_fx<L, TKP, T, D2, true><<<div_up(a.ncols, TKP), T, smem, st>>>(a);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_conv_fx<L, TKP, T, D2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_conv_fx<L, TKP, T, D2, false><<<div_up(a.ncols, TKP), T, smem, st>>>(a);
  }
  return cudaGetLastError();
}

// rows per Z tile: 2048 elements for the forward pass (smaller blocks, more
// of them resident), 4096 for the three-component inverse pass
__host__ __device__ constexpr int fx_rows(int M, int lines_per_row) {
  return lines_per_row == 1 ? ((2048 / M) < 1 ? 1 : (2048 / M > 32 ? 32 : 2048 / M))
                            : ((4096 / (M * lines_per_row)) < 1 ? 1 : (4096 / (M * lines_per_row) > 32 ? 32 : 4096 / (M * lines_per_row)));
}

template <int M, bool COMB>
cudaError_t fx_launch_zr2c(const float* src, float2* dst, const ZPass& z, const ZComb& cb, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 1);
  constexpr int T = fx_threads(RT * M);
  size_t smem = sizeof(float2) * (size_t)RT * row_pitch(M);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_zr2c_fx<M, RT, T, COMB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // 8-byte loads when every row starts at an even float offset
  int vec2 = (z.ld_real % 2 == 0) && (z.comp_stride_real % 2 == 0) && (((uintptr_t)src & 7) == 0);
  k_zr2c_fx<M, RT, T, COMB><<<div_up(z.nrows, RT), T, smem, st>>>(src, dst, z, cb, vec2);
  return cudaGetLastError();
}

template <int M>
cudaError_t fx_launch_zc2r(const float2* src, float* dst, const ZPass& z, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 1);
  constexpr int T = fx_threads(RT * M);
  size_t smem = sizeof(float2) * (size_t)odd_pitch(RT) * M;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_zc2r_fx<M, RT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_zc2r_fx<M, RT, T><<<div_up(z.nrows, RT), T, smem, st>>>(src, dst, z);
  return cudaGetLastError();
}

template <int M, int MODE>
cudaError_t fx_launch_zinv(const float2* S, const float2* twz, const float2* twP, int P1, int HZ, int64_t CS, int nrows,
                           const EpiArgs& ea, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 3);
  constexpr int T = fx_threads(3 * RT * M);
  size_t smem = sizeof(float2) * (size_t)3 * RT * row_pitch(M);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_zinv_fx<M, RT, T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  ZinvArgs za;
  za.S = const_cast<float2*>(S);
  za.twz = twz;
  za.twP = twP;
  za.P1 = P1;
  za.HZ = HZ;
  za.CS = CS;
  za.nrows = nrows;
  za.ea = ea;
  k_zinv_fx<M, RT, T, MODE><<<div_up(nrows, RT), T, smem, st>>>(za);
  return cudaGetLastError();
}

// inverse Z + Heun epilogue + the next evaluation's forward Z (k_zinv_fwd_fx)
template <int M, int MODE>
cudaError_t fx_launch_zinv_fwd(float2* S, const float2* twz, const float2* twP, int P1, int HZ, int64_t CS, int nrows,
                               const EpiArgs& ea, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 3);
  constexpr int T = fx_threads(3 * RT * M);
  size_t smem = sizeof(float2) * (size_t)3 * RT * row_pitch(M);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_zinv_fwd_fx<M, RT, T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  ZinvArgs za;
  za.S = S;
  za.twz = twz;
  za.twP = twP;
  za.P1 = P1;
  za.HZ = HZ;
  za.CS = CS;
  za.nrows = nrows;
  za.ea = ea;
  k_zinv_fwd_fx<M, RT, T, MODE><<<div_up(nrows, RT), T, smem, st>>>(za);
  return cudaGetLastError();
}
