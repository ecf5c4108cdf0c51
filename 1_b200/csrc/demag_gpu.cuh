// Demagnetising kernel generation on the GPU.
//
// Restates FaceKernel6 / faceIntegral (src/go/sim/demag.go:26-84,
// 142-183) and Exch6NgbrKernel (src/go/sim/exchange.go:44-71) with the
// same float32 operations in the same order, so the real-space kernel is
// bit-identical to the one the reference's Go subprocess computes
// (mumaxkern-go, src/go/kernel-main/main.go:43): every product, sum,
// quotient and square root is an explicitly rounded IEEE float32
// operation (no contraction into fused multiply-adds).  The square root
// of the Go code is taken in float64 and rounded, which equals the
// correctly rounded float32 square root.
#pragma once
#include "mmx_common.cuh"

__device__ __forceinline__ float fk_norm(const float v[3]) {
  float s = __fmul_rn(v[0], v[0]);
  s = __fadd_rn(s, __fmul_rn(v[1], v[1]));
  s = __fadd_rn(s, __fmul_rn(v[2], v[2]));
  return __fsqrt_rn(s);
}

__device__ void fk_face_integral(float B[3], const float R[3], const float cs[3], int s, int n) {
  int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
  float charge = __fmul_rn(cs[v], cs[w]);
  float pu1 = __fdiv_rn(cs[u], 2.f);
  float pu2 = -pu1;
  const float four_pi = 12.566370614359172f;
  float tv0 = __fadd_rn(-__fdiv_rn(cs[v], 2.f), __fdiv_rn(cs[v], (float)(2 * n)));
  float tv1 = __fdiv_rn(cs[v], (float)n);
  float tw0 = __fadd_rn(-__fdiv_rn(cs[w], 2.f), __fdiv_rn(cs[w], (float)(2 * n)));
  float tw1 = __fdiv_rn(cs[w], (float)n);
  B[0] = B[1] = B[2] = 0.f;
  for (int i = 0; i < n; i++) {
    float pv = __fadd_rn(tv0, __fmul_rn((float)i, tv1));
    for (int j = 0; j < n; j++) {
      float pw = __fadd_rn(tw0, __fmul_rn((float)j, tw1));
#pragma unroll
      for (int side = 0; side < 2; side++) {
        float pole[3];
        pole[u] = side == 0 ? pu1 : pu2;
        pole[v] = pv;
        pole[w] = pw;
        float R2[3];
#pragma unroll
        for (int d = 0; d < 3; d++) R2[d] = __fsub_rn(R[d], pole[d]);
        float r = fk_norm(R2);
        float inv = __fdiv_rn(1.f, r);
#pragma unroll
        for (int d = 0; d < 3; d++) R2[d] = __fmul_rn(R2[d], inv);
        float den = __fmul_rn(__fmul_rn(four_pi, r), r);
        float sc = __fdiv_rn(side == 0 ? charge : -charge, den);
#pragma unroll
        for (int d = 0; d < 3; d++) B[d] = __fadd_rn(B[d], __fmul_rn(R2[d], sc));
      }
    }
  }
  float fin = __fdiv_rn(1.f, (float)(n * n));
#pragma unroll
  for (int d = 0; d < 3; d++) B[d] = __fmul_rn(B[d], fin);
}

struct FaceKernelArgs {
  int P[3];
  int periodic[3];
  float cs[3];
  int accuracy;
  int lo[3], hi[3];  // loop bounds of demag.go:136-154 (after periodic scaling)
};

// One thread per wrapped output cell; images are accumulated in the Go
// loop order (x, then y, then z, ascending).
__global__ void k_face_kernel6(float* __restrict__ k6, FaceKernelArgs a) {
  const int64_t n3 = (int64_t)a.P[0] * a.P[1] * a.P[2];
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n3;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int zw = (int)(idx % a.P[2]);
    int yw = (int)((idx / a.P[2]) % a.P[1]);
    int xw = (int)(idx / ((int64_t)a.P[2] * a.P[1]));
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    // smallest image >= lo in each dimension
    int x0 = xw;
    while (x0 - a.P[0] >= a.lo[0]) x0 -= a.P[0];
    while (x0 < a.lo[0]) x0 += a.P[0];
    int y0 = yw;
    while (y0 - a.P[1] >= a.lo[1]) y0 -= a.P[1];
    while (y0 < a.lo[1]) y0 += a.P[1];
    int z0 = zw;
    while (z0 - a.P[2] >= a.lo[2]) z0 -= a.P[2];
    while (z0 < a.lo[2]) z0 += a.P[2];
    for (int s = 0; s < 3; s++) {
      for (int x = x0; x <= a.hi[0]; x += a.P[0])
        for (int y = y0; y <= a.hi[1]; y += a.P[1])
          for (int z = z0; z <= a.hi[2]; z += a.P[2]) {
            float R[3] = {__fmul_rn((float)x, a.cs[0]), __fmul_rn((float)y, a.cs[1]), __fmul_rn((float)z, a.cs[2])};
            float B[3];
            fk_face_integral(B, R, a.cs, s, a.accuracy);
            // KernIdx (kernel.go:95-98): order XX,YY,ZZ,YZ,XZ,XY
            if (s == 0) {
              acc[0] = __fadd_rn(acc[0], B[0]);
              acc[5] = __fadd_rn(acc[5], B[1]);
              acc[4] = __fadd_rn(acc[4], B[2]);
            } else if (s == 1) {
              acc[1] = __fadd_rn(acc[1], B[1]);
              acc[3] = __fadd_rn(acc[3], B[2]);
            } else {
              acc[2] = __fadd_rn(acc[2], B[2]);
            }
          }
    }
#pragma unroll
    for (int c = 0; c < 6; c++) k6[c * n3 + idx] = acc[c];
  }
}

// Exch6NgbrKernel folded into the diagonal components (init.go:256-267).
// The seven stencil cells are written in Go's order so that, when two
// wrap onto the same cell (a dimension of size 1 or 2), the last write
// wins, as in exchange.go:58-65; the tensor is then added.
__global__ void k_add_exch6(float* __restrict__ k6, int P0, int P1, int P2, float c0, float c1, float c2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int64_t n3 = (int64_t)P0 * P1 * P2;
  float hx = __fmul_rn(c0, c0), hy = __fmul_rn(c1, c1), hz = __fmul_rn(c2, c2);
  float cc = __fsub_rn(__fsub_rn(__fdiv_rn(-2.f, hx), __fdiv_rn(2.f, hy)), __fdiv_rn(2.f, hz));
  const int cell[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  float val[7] = {cc, __fdiv_rn(1.f, hx), __fdiv_rn(1.f, hx), __fdiv_rn(1.f, hy), __fdiv_rn(1.f, hy),
                  __fdiv_rn(1.f, hz), __fdiv_rn(1.f, hz)};
  const int P[3] = {P0, P1, P2};
  int64_t idx[7];
  float ev[7];
  int ne = 0;
  for (int c = 0; c < 7; c++) {
    int w[3];
    for (int d = 0; d < 3; d++) {
      int t = cell[c][d];
      while (t < 0) t += P[d];
      while (t >= P[d]) t -= P[d];
      w[d] = t;
    }
    int64_t id = ((int64_t)w[0] * P1 + w[1]) * P2 + w[2];
    int f = -1;
    for (int q = 0; q < ne; q++)
      if (idx[q] == id) f = q;
    if (f >= 0) ev[f] = val[c];
    else { idx[ne] = id; ev[ne] = val[c]; ne++; }
  }
  for (int comp = 0; comp < 3; comp++)
    for (int q = 0; q < ne; q++) k6[comp * n3 + idx[q]] = __fadd_rn(k6[comp * n3 + idx[q]], ev[q]);
}
