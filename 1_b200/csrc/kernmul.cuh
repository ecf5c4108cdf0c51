// Kernel spectrum octant and the per-bin 3x3 kernel products.
#pragma once
#include "llg_ops.cuh"

struct KernOct {
  const float* kh;  // [6][O0][O1][HZ]
  int O0, O1, HZ, P0, P1;
  int64_t cs;       // component stride
};

__device__ __forceinline__ void kern_at(const KernOct& K, int kx, int ky, int kz, float& Kxx, float& Kyy,
                                        float& Kzz, float& Kyz, float& Kxz, float& Kxy) {
  int fx = kx <= K.P0 / 2 ? kx : K.P0 - kx;
  int fy = ky <= K.P1 / 2 ? ky : K.P1 - ky;
  bool nx = kx > K.P0 / 2, ny = ky > K.P1 / 2;
  int64_t o = ((int64_t)fx * K.O1 + fy) * K.HZ + kz;
  Kxx = __ldg(K.kh + o);
  Kyy = __ldg(K.kh + K.cs + o);
  Kzz = __ldg(K.kh + 2 * K.cs + o);
  Kyz = __ldg(K.kh + 3 * K.cs + o);
  Kxz = __ldg(K.kh + 4 * K.cs + o);
  Kxy = __ldg(K.kh + 5 * K.cs + o);
  if (ny) Kyz = -Kyz;
  if (nx) Kxz = -Kxz;
  if (nx != ny) Kxy = -Kxy;
}

// H = K M per bin in the order of gpu_kernelmul6 (gpu_kernmul.cu:51-58)
__device__ __forceinline__ void kmul6(float2& mx, float2& my, float2& mz, float Kxx, float Kyy, float Kzz, float Kyz,
                                      float Kxz, float Kxy) {
  float2 hx, hy, hz;
  hx.x = FA(FA(FM(mx.x, Kxx), FM(my.x, Kxy)), FM(mz.x, Kxz));
  hx.y = FA(FA(FM(mx.y, Kxx), FM(my.y, Kxy)), FM(mz.y, Kxz));
  hy.x = FA(FA(FM(mx.x, Kxy), FM(my.x, Kyy)), FM(mz.x, Kyz));
  hy.y = FA(FA(FM(mx.y, Kxy), FM(my.y, Kyy)), FM(mz.y, Kyz));
  hz.x = FA(FA(FM(mx.x, Kxz), FM(my.x, Kyz)), FM(mz.x, Kzz));
  hz.y = FA(FA(FM(mx.y, Kxz), FM(my.y, Kyz)), FM(mz.y, Kzz));
  mx = hx;
  my = hy;
  mz = hz;
}
// 2D: Kxy = Kxz = 0 (gpu_kernmul.cu:114-119)
__device__ __forceinline__ void kmul4(float2& mx, float2& my, float2& mz, float Kxx, float Kyy, float Kzz,
                                      float Kyz) {
  float2 hx, hy, hz;
  hx.x = FM(mx.x, Kxx);
  hx.y = FM(mx.y, Kxx);
  hy.x = FA(FM(my.x, Kyy), FM(mz.x, Kyz));
  hy.y = FA(FM(my.y, Kyy), FM(mz.y, Kyz));
  hz.x = FA(FM(my.x, Kyz), FM(mz.x, Kzz));
  hz.y = FA(FM(my.y, Kyz), FM(mz.y, Kzz));
  mx = hx;
  my = hy;
  mz = hz;
}

// The same products with fused multiply-adds, for the fused convolution
// passes (their results are compared with the FP64 oracle within a
// tolerance; the drop-in gpu_kernelmul6/4 keep the rounding above).
__device__ __forceinline__ void kmul6_fma(float2& mx, float2& my, float2& mz, float Kxx, float Kyy, float Kzz,
                                          float Kyz, float Kxz, float Kxy) {
  float2 hx, hy, hz;
  hx.x = fmaf(mz.x, Kxz, fmaf(my.x, Kxy, mx.x * Kxx));
  hx.y = fmaf(mz.y, Kxz, fmaf(my.y, Kxy, mx.y * Kxx));
  hy.x = fmaf(mz.x, Kyz, fmaf(my.x, Kyy, mx.x * Kxy));
  hy.y = fmaf(mz.y, Kyz, fmaf(my.y, Kyy, mx.y * Kxy));
  hz.x = fmaf(mz.x, Kzz, fmaf(my.x, Kyz, mx.x * Kxz));
  hz.y = fmaf(mz.y, Kzz, fmaf(my.y, Kyz, mx.y * Kxz));
  mx = hx;
  my = hy;
  mz = hz;
}
__device__ __forceinline__ void kmul4_fma(float2& mx, float2& my, float2& mz, float Kxx, float Kyy, float Kzz,
                                          float Kyz) {
  float2 hx, hy, hz;
  hx.x = mx.x * Kxx;
  hx.y = mx.y * Kxx;
  hy.x = fmaf(mz.x, Kyz, my.x * Kyy);
  hy.y = fmaf(mz.y, Kyz, my.y * Kyy);
  hz.x = fmaf(mz.x, Kzz, my.x * Kyz);
  hz.y = fmaf(mz.y, Kzz, my.y * Kyz);
  mx = hx;
  my = hy;
  mz = hz;
}
