// Per-cell LLG arithmetic shared by the drop-in primitives and the fused
// epilogues.  Every operation is an explicitly rounded float32 operation
// in the reference's order, so a fused epilogue produces bit-for-bit the
// same values as the corresponding sequence of primitive calls.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FM(a, b) __fmul_rn((a), (b))
#define FA(a, b) __fadd_rn((a), (b))
#define FS(a, b) __fsub_rn((a), (b))

// gpu_deltaM (src/gpukern/gpu_torque.cu:20-53), h overwritten with
// dt_gilb (m x h + alpha m x (m x h)) in the internal frame.
__device__ __forceinline__ void llg_delta_m(float Mx, float My, float Mz, float& Hx, float& Hy, float& Hz,
                                            float alpha, float dtg) {
  float mxHx = FS(FM(My, Hz), FM(Hy, Mz));
  float mxHy = FA(FM(-Mx, Hz), FM(Hx, Mz));
  float mxHz = FS(FM(Mx, Hy), FM(Hx, My));
  float mmx = FA(FM(-My, mxHz), FM(mxHy, Mz));
  float mmy = FS(FM(Mx, mxHz), FM(mxHx, Mz));
  float mmz = FA(FM(-Mx, mxHy), FM(mxHx, My));
  Hx = FM(dtg, FA(mxHx, FM(mmx, alpha)));
  Hy = FM(dtg, FA(mxHy, FM(mmy, alpha)));
  Hz = FM(dtg, FA(mxHz, FM(mmz, alpha)));
}

// gpu_normalize_uniform (gpu_normalize.cu:20-28) with a correctly rounded
// 1/sqrt(|m|^2) instead of the fast-math rsqrtf.
__device__ __forceinline__ void llg_normalize(float& x, float& y, float& z) {
  float s = FA(FA(FM(x, x), FM(y, y)), FM(z, z));
  float inv = __fdiv_rn(1.f, __fsqrt_rn(s));
  x = FM(x, inv);
  y = FM(y, inv);
  z = FM(z, inv);
}

struct LocalField {
  float hext[3];
  int anis;     // 0 none, 1 uniaxial
  float K;
  float u[3];
  // thermal field (RK stages): h += sigma * N(0,1) per cell and component,
  // the same numbers for every stage of a step (rk.go:289-292); 0 = off
  float sigma;
  unsigned int seed, step_lo, step_hi;
};

// Philox-4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11): counter c, key k
__host__ __device__ __forceinline__ unsigned int philox_mulhi(unsigned int a, unsigned int b) {
  return (unsigned int)(((unsigned long long)a * b) >> 32);
}
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    unsigned int hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    unsigned int hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// three standard normals of cell g at step (lo, hi): one Philox block,
// two Box-Muller pairs (u1 in (0, 1], u2 in [0, 1))
__device__ __forceinline__ void thermal_normals(const LocalField& lf, int64_t g, float* nrm) {
  uint4 r = philox4x32_10(make_uint4((unsigned int)g, (unsigned int)((uint64_t)g >> 32), lf.step_lo, lf.step_hi),
                          make_uint2(lf.seed, 0x4D4D5854u));
  float u1 = ((float)(r.x >> 8) + 1.f) * (1.f / 16777216.f);
  float u2 = (float)(r.y >> 8) * (1.f / 16777216.f);
  float u3 = ((float)(r.z >> 8) + 1.f) * (1.f / 16777216.f);
  float u4 = (float)(r.w >> 8) * (1.f / 16777216.f);
  float a = sqrtf(-2.f * logf(u1)), b = sqrtf(-2.f * logf(u3));
  float s1, c1, s2, c2;
  sincospif(2.f * u2, &s1, &c1);
  sincospif(2.f * u4, &s2, &c2);
  nrm[0] = a * c1;
  nrm[1] = a * s1;
  nrm[2] = b * c2;
}

// gpu_add_local_fields, uniform Hext, ANIS_NONE / ANIS_UNIAXIAL
// (gpu_local_contr3.cu:21-36,133-143).
__device__ __forceinline__ void llg_local(const LocalField& lf, float mx, float my, float mz, float& hx, float& hy,
                                          float& hz) {
  if (lf.anis == 1) {
    float mu = FA(FA(FM(mx, lf.u[0]), FM(my, lf.u[1])), FM(mz, lf.u[2]));
    float km = FM(lf.K, mu);
    hx = FA(hx, FA(lf.hext[0], FM(km, lf.u[0])));
    hy = FA(hy, FA(lf.hext[1], FM(km, lf.u[1])));
    hz = FA(hz, FA(lf.hext[2], FM(km, lf.u[2])));
  } else {
    hx = FA(hx, lf.hext[0]);
    hy = FA(hy, lf.hext[1]);
    hz = FA(hz, lf.hext[2]);
  }
}

// non-negative float maximum through the integer ordering of IEEE floats
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}
