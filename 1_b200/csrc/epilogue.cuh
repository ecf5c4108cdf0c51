// Per-cell epilogues of the inverse-Z pass: local fields, LLG torque and
// the solver stage update, shared by the generic and the fixed-size
// kernels.  Every operation is an explicitly rounded float32 operation in
// the reference's order (see llg_ops.cuh).
#pragma once
#include "llg_ops.cuh"

// EPI_RK64: EPI_RK with the adaptive solvers' embedded error vector formed
// and normed in float64 (the precision form)
enum { EPI_FIELD = 0, EPI_HEUN1 = 1, EPI_HEUN2 = 2, EPI_TORQUE = 3, EPI_RK = 4, EPI_RK64 = 5 };
__host__ __device__ constexpr bool epi_rk(int mode) { return mode == EPI_RK || mode == EPI_RK64; }

#define RK_MAXS 7
struct RKCoef {
  float a[RK_MAXS];   // row a[i+1][0..i] (next stage input), or b for the final stage
  float b2[RK_MAXS];  // lower-order weights (final stage, adaptive)
  int nk;             // number of k's combined
  int final_stage;    // 1: produce m_high / m_low / error
  int adaptive;
};

struct EpiArgs {
  int N1, N2;
  int64_t n;            // cells per component
  LocalField lf;
  float alpha, dtg;
  const float* m_in;    // magnetisation at which the field was evaluated
  float* out0;
  float* out1;
  const float* aux0;
  const float* aux1;
  float* err;           // device scalar (maxabs target), may be null
  double* energy;       // RK stages: device accumulator of the total energy
                        // density sum (Relax's energy, relax.go:14-23), may be null
  const float* dt_dev;  // RK: device dt
  float* kbuf[RK_MAXS]; // RK: stage torques
  int stage;            // RK: index of this stage's k
  RKCoef rk;
};


// Per-cell inputs an epilogue reads besides the field: m at which the field
// was evaluated, and for Heun's corrector t0 and m (aux0, aux1), for an RK
// stage the step-start m (aux0).  Loaded ahead of the transform so that
// their latency overlaps it.
template <int MODE>
struct EpiIn {
  float m[3];
  float a0[(MODE == EPI_HEUN2 || epi_rk(MODE)) ? 3 : 1];
  float a1[MODE == EPI_HEUN2 ? 3 : 1];
};

template <int MODE>
__device__ __forceinline__ void epi_load(const EpiArgs& ea, int64_t g, EpiIn<MODE>& in) {
  const int64_t n = ea.n;
  in.m[0] = ea.m_in[g];
  in.m[1] = ea.m_in[n + g];
  in.m[2] = ea.m_in[2 * n + g];
  if (MODE == EPI_HEUN2 || epi_rk(MODE)) {
    in.a0[0] = ea.aux0[g];
    in.a0[1] = ea.aux0[n + g];
    in.a0[2] = ea.aux0[2 * n + g];
  }
  if (MODE == EPI_HEUN2) {
    in.a1[0] = ea.aux1[g];
    in.a1[1] = ea.aux1[n + g];
    in.a1[2] = ea.aux1[2 * n + g];
  }
}

// next: if not null, receives the cell's next stage input (Heun: m1est
// after the predictor, m after the corrector)
// eacc: the thread's energy-density sum (RK stages with ea.energy set)
template <int MODE>
__device__ __forceinline__ void epi_cell_in(const EpiArgs& ea, int64_t g, float hx, float hy, float hz,
                                            const EpiIn<MODE>& in, float& lmax, float* next = nullptr,
                                            double* eacc = nullptr);

// cell g (index into one component), field (hx,hy,hz) from the convolution
template <int MODE>
__device__ __forceinline__ void epi_cell(const EpiArgs& ea, int64_t g, float hx, float hy, float hz, float& lmax,
                                         double* eacc = nullptr) {
  EpiIn<MODE> in;
  epi_load<MODE>(ea, g, in);
  epi_cell_in<MODE>(ea, g, hx, hy, hz, in, lmax, nullptr, eacc);
}

template <int MODE>
__device__ __forceinline__ void epi_cell_in(const EpiArgs& ea, int64_t g, float hx, float hy, float hz,
                                            const EpiIn<MODE>& in, float& lmax, float* next, double* eacc) {
    const int64_t n = ea.n;
    float mx = in.m[0], my = in.m[1], mz = in.m[2];
    llg_local(ea.lf, mx, my, mz, hx, hy, hz);
    if constexpr (epi_rk(MODE) || MODE == EPI_TORQUE) {
      // energy density of the stage's m: -1/2 m.h_conv - m.Hext - 1/2 K (m.u)^2
      // = -1/2 m.(h + Hext) with h the full field (the anisotropy terms
      // cancel), summed in float64
      if (ea.energy && eacc) {
        float s = FA(FA(FM(mx, FA(hx, ea.lf.hext[0])), FM(my, FA(hy, ea.lf.hext[1]))), FM(mz, FA(hz, ea.lf.hext[2])));
        *eacc += (double)FM(-0.5f, s);
      }
      // the thermal field, added after the energy density (field.go:64-80)
      if (ea.lf.sigma != 0.f) {
        float nrm[3];
        thermal_normals(ea.lf, g, nrm);
        hx = FA(hx, FM(ea.lf.sigma, nrm[0]));
        hy = FA(hy, FM(ea.lf.sigma, nrm[1]));
        hz = FA(hz, FM(ea.lf.sigma, nrm[2]));
      }
    }
    if (MODE == EPI_FIELD) {
      ea.out0[g] = hx;
      ea.out0[n + g] = hy;
      ea.out0[2 * n + g] = hz;
      return;
    }
    llg_delta_m(mx, my, mz, hx, hy, hz, ea.alpha, ea.dtg);
    if (MODE == EPI_TORQUE) {
      ea.out0[g] = hx;
      ea.out0[n + g] = hy;
      ea.out0[2 * n + g] = hz;
      if (ea.err) lmax = fmaxf(lmax, fmaxf(fabsf(hx), fmaxf(fabsf(hy), fabsf(hz))));
    } else if (MODE == EPI_HEUN1) {
      // t0 = torque*dt; m1est = normalize(m + t0)   (adaptive_heun.go:39-44)
      ea.out0[g] = hx;
      ea.out0[n + g] = hy;
      ea.out0[2 * n + g] = hz;
      float ex = FA(mx, hx), ey = FA(my, hy), ez = FA(mz, hz);
      llg_normalize(ex, ey, ez);
      ea.out1[g] = ex;
      ea.out1[n + g] = ey;
      ea.out1[2 * n + g] = ez;
      if (next) { next[0] = ex; next[1] = ey; next[2] = ez; }
    } else if (MODE == EPI_HEUN2) {
      // t = 0.5 t1 + 0.5 t0; m = normalize(m + t)   (adaptive_heun.go:46-52)
      float tx = FA(FM(0.5f, hx), FM(0.5f, in.a0[0]));
      float ty = FA(FM(0.5f, hy), FM(0.5f, in.a0[1]));
      float tz = FA(FM(0.5f, hz), FM(0.5f, in.a0[2]));
      float nx = FA(in.a1[0], tx), ny = FA(in.a1[1], ty), nz = FA(in.a1[2], tz);
      llg_normalize(nx, ny, nz);
      ea.out0[g] = nx;
      ea.out0[n + g] = ny;
      ea.out0[2 * n + g] = nz;
      if (next) { next[0] = nx; next[1] = ny; next[2] = nz; }
      if (ea.err) {
        // error = maxabs(m1est - m)   (adaptive_heun.go:56-59)
        float d0 = fabsf(FA(mx, FM(-1.f, nx)));
        float d1 = fabsf(FA(my, FM(-1.f, ny)));
        float d2 = fabsf(FA(mz, FM(-1.f, nz)));
        lmax = fmaxf(lmax, fmaxf(d0, fmaxf(d1, d2)));
      }
    } else if (epi_rk(MODE)) {
      float kx = hx, ky = hy, kz = hz;
      float* kd = ea.out0;
      kd[g] = kx;
      kd[n + g] = ky;
      kd[2 * n + g] = kz;
      const float dt = *ea.dt_dev;
      // in.a0: the step-start magnetisation
      float q[3] = {in.a0[0], in.a0[1], in.a0[2]};
      // next stage input (or m_high): m0 + sum_j (dt a_j) k_j, j in order
#pragma unroll
      for (int j = 0; j < RK_MAXS; j++) {
        if (j >= ea.rk.nk) break;
        float a = ea.rk.a[j];
        if (a == 0.f) continue;
        float c = FM(dt, a);
        float k0, k1, k2;
        if (j == ea.stage) { k0 = kx; k1 = ky; k2 = kz; }
        else { k0 = ea.kbuf[j][g]; k1 = ea.kbuf[j][n + g]; k2 = ea.kbuf[j][2 * n + g]; }
        q[0] = FA(q[0], FM(c, k0));
        q[1] = FA(q[1], FM(c, k1));
        q[2] = FA(q[2], FM(c, k2));
      }
      if (MODE == EPI_RK64 && ea.rk.final_stage && ea.rk.adaptive) {
        // the embedded error vector sum_j (b_j - b*_j) dt k_j formed and
        // normed in float64 from the float32 stage torques
        double e0 = 0.0, e1 = 0.0, e2 = 0.0;
#pragma unroll
        for (int j = 0; j < RK_MAXS; j++) {
          if (j >= ea.rk.nk) break;
          const double w = ((double)ea.rk.a[j] - (double)ea.rk.b2[j]) * (double)dt;
          if (w == 0.0) continue;
          float k0, k1, k2;
          if (j == ea.stage) { k0 = kx; k1 = ky; k2 = kz; }
          else { k0 = ea.kbuf[j][g]; k1 = ea.kbuf[j][n + g]; k2 = ea.kbuf[j][2 * n + g]; }
          e0 = fma(w, (double)k0, e0);
          e1 = fma(w, (double)k1, e1);
          e2 = fma(w, (double)k2, e2);
        }
        lmax = fmaxf(lmax, (float)fmax(fabs(e0), fmax(fabs(e1), fabs(e2))));
      } else if (ea.rk.final_stage && ea.rk.adaptive) {
        float lo[3] = {in.a0[0], in.a0[1], in.a0[2]};
#pragma unroll
        for (int j = 0; j < RK_MAXS; j++) {
          if (j >= ea.rk.nk) break;
          float b = ea.rk.b2[j];
          if (b == 0.f) continue;
          float c = FM(b, dt);
          float k0, k1, k2;
          if (j == ea.stage) { k0 = kx; k1 = ky; k2 = kz; }
          else { k0 = ea.kbuf[j][g]; k1 = ea.kbuf[j][n + g]; k2 = ea.kbuf[j][2 * n + g]; }
          lo[0] = FA(lo[0], FM(c, k0));
          lo[1] = FA(lo[1], FM(c, k1));
          lo[2] = FA(lo[2], FM(c, k2));
        }
        float d0 = fabsf(FA(lo[0], FM(-1.f, q[0])));
        float d1 = fabsf(FA(lo[1], FM(-1.f, q[1])));
        float d2 = fabsf(FA(lo[2], FM(-1.f, q[2])));
        lmax = fmaxf(lmax, fmaxf(d0, fmaxf(d1, d2)));
      }
      ea.out1[g] = q[0];
      ea.out1[n + g] = q[1];
      ea.out1[2 * n + g] = q[2];
    }
  
}

// block-wide maximum of lmax into *ea.err (non-negative float atomics) and,
// for RK stages, the warp sums of the energy density into *ea.energy
template <int MODE>
__device__ __forceinline__ void epi_flush_max(const EpiArgs& ea, float lmax, double eacc = 0.0) {
  if ((MODE == EPI_HEUN2 || epi_rk(MODE) || MODE == EPI_TORQUE) && ea.err) {
    for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(ea.err, lmax);
  }
  if constexpr (epi_rk(MODE) || MODE == EPI_TORQUE) {
    if (ea.energy) {
      for (int o = 16; o > 0; o >>= 1) eacc += __shfl_xor_sync(0xffffffffu, eacc, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(ea.energy, eacc);
    }
  }
}
