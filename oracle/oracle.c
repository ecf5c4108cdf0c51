/*
 * CPU ORACLE -- test infrastructure only.
 *
 * This file restates, in plain C, the arithmetic of MuMax 1.1's LLG
 * time-stepping hot path (the Go driver in src/go/sim and the CUDA library
 * src/gpukern of the reference).  It exists so that tests, the smoke check
 * and the CPU baseline of the benchmark can check the CUDA engine against an
 * independent statement of the algorithm.  The product library never links,
 * loads or calls it.
 *
 * It is compiled twice: with REAL=float (the FP32 "faithful" build, which
 * performs every float32 operation of the reference in the reference's
 * order, one rounding per operation, no fused multiply-add) and with
 * REAL=double (the FP64 build of the same code, used for energies, <m> and
 * the error of the reduced-precision forms).
 *
 * Where the reference's result depends on a closed library (cuFFT), the
 * oracle uses its own double-precision mixed-radix FFT and rounds the
 * spectrum to REAL at the points where the reference stores float32
 * buffers.  FFT values are therefore pinned only to rounding level, never
 * bit for bit.
 *
 * Axis convention: every array is internal order [c][X][Y][Z] with Z
 * contiguous (reference: src/go/sim/simgeom.go:19-38).  Internal X is the
 * user's z axis.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL float
#endif
#ifndef PFX
#define PFX o32_
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(PFX, name)

typedef struct { double re, im; } cplx;

/* ------------------------------------------------------------------ */
/* Kernel generation: FaceKernel6 (src/go/sim/demag.go:26-84) and the  */
/* point-charge face integral (demag.go:142-183).                        */
/* ------------------------------------------------------------------ */

/* Go's wrap (src/go/sim/kernel.go:62-72). */
static int wrap_idx(int n, int max) {
  while (n < 0) n += max;
  while (n >= max) n -= max;
  return n;
}

/* Norm of a 3-vector as src/go/mumax/tensor/vector.go:62-64:
 * float32 sum of squares, square root in float64, rounded back. */
static REAL vnorm(const REAL v[3]) {
  REAL s = v[0] * v[0];
  s = s + v[1] * v[1];
  s = s + v[2] * v[2];
  return (REAL)sqrt((double)s);
}

/* faceIntegral: field at R of the two charged faces of a unit cell
 * magnetised along s, n x n point charges per face (demag.go:142-183). */
static void face_integral(REAL B[3], const REAL R[3], const REAL cs[3], int s, int n) {
  int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
  REAL surface = cs[v] * cs[w];
  REAL charge = surface;
  REAL pu1 = cs[u] / (REAL)2.;
  REAL pu2 = -pu1;
  const REAL four_pi = (REAL)(4.0 * 3.14159265358979323846);
  REAL pole[3], R2[3];
  B[0] = B[1] = B[2] = 0;
  for (int i = 0; i < n; i++) {
    REAL pv = -(cs[v] / (REAL)2.);
    pv = pv + cs[v] / (REAL)(2 * n);
    pv = pv + (REAL)i * (cs[v] / (REAL)n);
    for (int j = 0; j < n; j++) {
      REAL pw = -(cs[w] / (REAL)2.);
      pw = pw + cs[w] / (REAL)(2 * n);
      pw = pw + (REAL)j * (cs[w] / (REAL)n);
      for (int side = 0; side < 2; side++) {
        pole[u] = side == 0 ? pu1 : pu2;
        pole[v] = pv;
        pole[w] = pw;
        for (int d = 0; d < 3; d++) R2[d] = R[d] - pole[d];
        REAL r = vnorm(R2);
        REAL inv = (REAL)1. / vnorm(R2);
        for (int d = 0; d < 3; d++) R2[d] *= inv;
        REAL den = four_pi * r;
        den = den * r;
        REAL sc = (side == 0 ? charge : -charge) / den;
        for (int d = 0; d < 3; d++) R2[d] *= sc;
        for (int d = 0; d < 3; d++) B[d] += R2[d];
      }
    }
  }
  REAL fin = (REAL)1. / (REAL)(n * n);
  for (int d = 0; d < 3; d++) B[d] *= fin;
}

/* KernIdx (kernel.go:95-98): 6-component order XX,YY,ZZ,YZ,XZ,XY. */
static const int KIDX[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};

/* FaceKernel6: k[6][PX][PY][PZ], accumulated over periodic images in loop
 * order, indices wrapped (demag.go:26-84). */
void FN(face_kernel6)(const int size[3], const REAL cellsize[3], int accuracy,
                      const int periodic[3], REAL* k) {
  int64_t n3 = (int64_t)size[0] * size[1] * size[2];
  memset(k, 0, sizeof(REAL) * 6 * n3);
  int x1 = -(size[0] - 1) / 2, x2 = size[0] / 2 - 1;
  if (size[0] == 1 && periodic[0] == 0) x2 = 0;
  int y1 = -(size[1] - 1) / 2, y2 = size[1] / 2 - 1;
  int z1 = -(size[2] - 1) / 2, z2 = size[2] / 2 - 1;
  x1 *= periodic[0] + 1; x2 *= periodic[0] + 1;
  y1 *= periodic[1] + 1; y2 *= periodic[1] + 1;
  z1 *= periodic[2] + 1; z2 *= periodic[2] + 1;
  for (int s = 0; s < 3; s++) {
    /* Each wrapped output cell is touched by a fixed, ordered list of
     * images; parallelising over x keeps that order when no image of one x
     * wraps onto another x (always true without periodicity in X). */
#pragma omp parallel for schedule(dynamic) if (periodic[0] == 0)
    for (int x = x1; x <= x2; x++) {
      int xw = wrap_idx(x, size[0]);
      for (int y = y1; y <= y2; y++) {
        int yw = wrap_idx(y, size[1]);
        for (int z = z1; z <= z2; z++) {
          int zw = wrap_idx(z, size[2]);
          REAL R[3] = {(REAL)x * cellsize[0], (REAL)y * cellsize[1], (REAL)z * cellsize[2]};
          REAL B[3];
          face_integral(B, R, cellsize, s, accuracy);
          int64_t idx = ((int64_t)xw * size[1] + yw) * size[2] + zw;
          for (int d = s; d < 3; d++) k[KIDX[s][d] * n3 + idx] += B[d];
        }
      }
    }
  }
}

/* Exch6NgbrKernel added into the diagonal components (exchange.go:44-71,
 * init.go:256-267); in 2D the +-x writes overwrite the centre. */
void FN(add_exch6_kernel)(const int size[3], const REAL cellsize[3], REAL* k) {
  int64_t n3 = (int64_t)size[0] * size[1] * size[2];
  REAL hx = cellsize[0] * cellsize[0];
  REAL hy = cellsize[1] * cellsize[1];
  REAL hz = cellsize[2] * cellsize[2];
  /* Build the exchange kernel separately (it is a fresh tensor in Go),
   * then add element-wise. Only 7 cells are non-zero. */
  int cells[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  REAL c0 = (REAL)-2. / hx;
  c0 = c0 - (REAL)2. / hy;
  c0 = c0 - (REAL)2. / hz;
  REAL vals[7] = {c0, (REAL)1. / hx, (REAL)1. / hx, (REAL)1. / hy, (REAL)1. / hy, (REAL)1. / hz, (REAL)1. / hz};
  for (int s = 0; s < 3; s++) {
    int comp = KIDX[s][s];
    /* exchange tensor E for this component, sparse: last write wins */
    int64_t idxs[7];
    REAL ev[7];
    int ne = 0;
    for (int c = 0; c < 7; c++) {
      int64_t idx = ((int64_t)wrap_idx(cells[c][0], size[0]) * size[1] + wrap_idx(cells[c][1], size[1])) * size[2] +
                    wrap_idx(cells[c][2], size[2]);
      int found = -1;
      for (int q = 0; q < ne; q++) if (idxs[q] == idx) found = q;
      if (found >= 0) ev[found] = vals[c];
      else { idxs[ne] = idx; ev[ne] = vals[c]; ne++; }
    }
    for (int q = 0; q < ne; q++) k[comp * n3 + idxs[q]] += ev[q];
  }
}

/* ------------------------------------------------------------------ */
/* Double-precision mixed-radix FFT (Stockham, radices 2,3,4,5 and a    */
/* generic odd-prime DFT), used along one axis at a time.               */
/* ------------------------------------------------------------------ */

typedef struct {
  int n, nf, f[40];
  cplx* tw; /* exp(-2 pi i t / n) */
} fftplan;

static void plan_init(fftplan* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
  for (int r = 3; m > 1; r += 2) while (m % r == 0) { p->f[p->nf++] = r; m /= r; }
  p->tw = (cplx*)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  for (int t = 0; t < n; t++) {
    double a = -2.0 * M_PI * (double)t / (double)n;
    p->tw[t].re = cos(a);
    p->tw[t].im = sin(a);
  }
}
static void plan_free(fftplan* p) { free(p->tw); }

/* In-place line transform, sign = -1 forward, +1 inverse (unnormalised).
 * work must hold n values. */
static void fft_line(const fftplan* p, cplx* x, cplx* work, int sign) {
  int n = p->n;
  if (n == 1) return;
  cplx* a = x;
  cplx* b = work;
  int ns = 1;
  for (int s = 0; s < p->nf; s++) {
    int r = p->f[s];
    int m = n / r;
    for (int j = 0; j < m; j++) {
      int k = j % ns;
      cplx v[64];
      cplx vv[64];
      for (int q = 0; q < r; q++) {
        cplx in = a[j + q * m];
        int ti = (int)(((int64_t)q * k * (n / (ns * r))) % n);
        cplx w = p->tw[ti];
        if (sign > 0) w.im = -w.im;
        v[q].re = in.re * w.re - in.im * w.im;
        v[q].im = in.re * w.im + in.im * w.re;
      }
      /* radix-r DFT */
      for (int o = 0; o < r; o++) {
        double sr = 0, si = 0;
        for (int q = 0; q < r; q++) {
          int ti = (int)(((int64_t)o * q % r) * (n / r));
          cplx w = p->tw[ti];
          if (sign > 0) w.im = -w.im;
          sr += v[q].re * w.re - v[q].im * w.im;
          si += v[q].re * w.im + v[q].im * w.re;
        }
        vv[o].re = sr;
        vv[o].im = si;
      }
      int base = (j / ns) * ns * r + k;
      for (int o = 0; o < r; o++) b[base + o * ns] = vv[o];
    }
    cplx* t = a; a = b; b = t;
    ns *= r;
  }
  if (a != x) memcpy(x, a, sizeof(cplx) * n);
}

/* ------------------------------------------------------------------ */
/* Padded convolution (src/go/sim/conv.go:57-100, gpu_fft0.cu:96-109,  */
/* gpu_kernmul.cu:25-141) with the spectrum in REAL between stages.     */
/* ------------------------------------------------------------------ */

typedef struct {
  int N[3], P[3], HZ;
  int ktype;       /* 6 (3D) or 4 (2D), conv.go:173-179 */
  int64_t nspec;   /* P0*P1*HZ complex bins */
  REAL* kern;      /* [6][P0][P1][HZ] real kernel spectrum, x 1/(P0 P1 P2) */
  fftplan pl[3];
} conv_t;

/* forward: real (N0,N1,N2) padded into (P0,P1,P2) -> half spectrum
 * (P0,P1,HZ) complex, returned as double. */
static void conv_forward(const conv_t* c, const REAL* in, int nin0, int nin1, int nin2, cplx* out) {
  int P0 = c->P[0], P1 = c->P[1], P2 = c->P[2], HZ = c->HZ;
  memset(out, 0, sizeof(cplx) * (size_t)c->nspec);
#pragma omp parallel
  {
    cplx* line = (cplx*)malloc(sizeof(cplx) * (P0 > P1 ? (P0 > P2 ? P0 : P2) : (P1 > P2 ? P1 : P2)));
    cplx* work = (cplx*)malloc(sizeof(cplx) * (P0 > P1 ? (P0 > P2 ? P0 : P2) : (P1 > P2 ? P1 : P2)));
    /* Z (rows with data only) */
#pragma omp for collapse(2)
    for (int x = 0; x < nin0; x++)
      for (int y = 0; y < nin1; y++) {
        for (int z = 0; z < P2; z++) {
          line[z].re = z < nin2 ? (double)in[((int64_t)x * nin1 + y) * nin2 + z] : 0.0;
          line[z].im = 0;
        }
        fft_line(&c->pl[2], line, work, -1);
        for (int z = 0; z < HZ; z++) out[((int64_t)x * P1 + y) * HZ + z] = line[z];
      }
    /* Y (planes with data only) */
#pragma omp for collapse(2)
    for (int x = 0; x < nin0; x++)
      for (int z = 0; z < HZ; z++) {
        for (int y = 0; y < P1; y++) line[y] = out[((int64_t)x * P1 + y) * HZ + z];
        fft_line(&c->pl[1], line, work, -1);
        for (int y = 0; y < P1; y++) out[((int64_t)x * P1 + y) * HZ + z] = line[y];
      }
    /* X */
    if (P0 > 1) {
#pragma omp for collapse(2)
      for (int y = 0; y < P1; y++)
        for (int z = 0; z < HZ; z++) {
          for (int x = 0; x < P0; x++) line[x] = out[((int64_t)x * P1 + y) * HZ + z];
          fft_line(&c->pl[0], line, work, -1);
          for (int x = 0; x < P0; x++) out[((int64_t)x * P1 + y) * HZ + z] = line[x];
        }
    }
    free(line);
    free(work);
  }
}

/* inverse: half spectrum -> real (N0,N1,N2), unnormalised C2R (the
 * imaginary parts of the kz = 0 and kz = P2/2 bins are ignored, as a C2R
 * transform does). The spectrum is destroyed. */
static void conv_inverse(const conv_t* c, cplx* spec, REAL* out, int n0, int n1, int n2) {
  int P0 = c->P[0], P1 = c->P[1], P2 = c->P[2], HZ = c->HZ;
#pragma omp parallel
  {
    int mx = P0 > P1 ? (P0 > P2 ? P0 : P2) : (P1 > P2 ? P1 : P2);
    cplx* line = (cplx*)malloc(sizeof(cplx) * mx);
    cplx* work = (cplx*)malloc(sizeof(cplx) * mx);
    if (P0 > 1) {
#pragma omp for collapse(2)
      for (int y = 0; y < P1; y++)
        for (int z = 0; z < HZ; z++) {
          for (int x = 0; x < P0; x++) line[x] = spec[((int64_t)x * P1 + y) * HZ + z];
          fft_line(&c->pl[0], line, work, +1);
          for (int x = 0; x < P0; x++) spec[((int64_t)x * P1 + y) * HZ + z] = line[x];
        }
    }
#pragma omp for collapse(2)
    for (int x = 0; x < n0; x++)
      for (int z = 0; z < HZ; z++) {
        for (int y = 0; y < P1; y++) line[y] = spec[((int64_t)x * P1 + y) * HZ + z];
        fft_line(&c->pl[1], line, work, +1);
        for (int y = 0; y < P1; y++) spec[((int64_t)x * P1 + y) * HZ + z] = line[y];
      }
#pragma omp for collapse(2)
    for (int x = 0; x < n0; x++)
      for (int y = 0; y < n1; y++) {
        const cplx* s = &spec[((int64_t)x * P1 + y) * HZ];
        /* rebuild the full Hermitian row, then a complex inverse */
        for (int z = 0; z < HZ; z++) line[z] = s[z];
        line[0].im = 0;
        if (P2 % 2 == 0) line[P2 / 2].im = 0;
        for (int z = HZ; z < P2; z++) {
          line[z].re = s[P2 - z].re;
          line[z].im = -s[P2 - z].im;
        }
        fft_line(&c->pl[2], line, work, +1);
        for (int z = 0; z < n2; z++) out[((int64_t)x * n1 + y) * n2 + z] = (REAL)line[z].re;
      }
    free(line);
    free(work);
  }
}

/* loadKernel6 (conv.go:110-167): transform each needed kernel component
 * with the same FFT, keep the real part, scale by 1/(P0 P1 P2). */
static void conv_init(conv_t* c, const int N[3], const int P[3], const REAL* k6) {
  for (int d = 0; d < 3; d++) { c->N[d] = N[d]; c->P[d] = P[d]; plan_init(&c->pl[d], P[d]); }
  c->HZ = P[2] / 2 + 1;
  c->ktype = P[0] == 1 ? 4 : 6;
  c->nspec = (int64_t)P[0] * P[1] * c->HZ;
  c->kern = (REAL*)calloc((size_t)(6 * c->nspec), sizeof(REAL));
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)c->nspec);
  int64_t n3 = (int64_t)P[0] * P[1] * P[2];
  REAL norm = (REAL)1.0 / (REAL)(float)n3;
  for (int comp = 0; comp < 6; comp++) {
    if (c->ktype == 4 && (comp == 4 || comp == 5)) continue;
    conv_forward(c, k6 + comp * n3, P[0], P[1], P[2], tmp);
    for (int64_t i = 0; i < c->nspec; i++) c->kern[comp * c->nspec + i] = (REAL)tmp[i].re * norm;
  }
  free(tmp);
}

static void conv_free(conv_t* c) {
  free(c->kern);
  for (int d = 0; d < 3; d++) plan_free(&c->pl[d]);
}

/* kernelmul6 / kernelmul4 on REAL spectra (gpu_kernmul.cu:25-62,92-123). */
static void kernelmul(const conv_t* c, REAL* sx, REAL* sy, REAL* sz) {
  const REAL *kxx = c->kern, *kyy = c->kern + c->nspec, *kzz = c->kern + 2 * c->nspec, *kyz = c->kern + 3 * c->nspec,
             *kxz = c->kern + 4 * c->nspec, *kxy = c->kern + 5 * c->nspec;
#pragma omp parallel for
  for (int64_t i = 0; i < c->nspec; i++) {
    int64_t e = 2 * i;
    REAL rx = sx[e], ix = sx[e + 1], ry = sy[e], iy = sy[e + 1], rz = sz[e], iz = sz[e + 1];
    if (c->ktype == 6) {
      REAL Kxx = kxx[i], Kyy = kyy[i], Kzz = kzz[i], Kyz = kyz[i], Kxz = kxz[i], Kxy = kxy[i];
      REAL t;
      t = rx * Kxx; t = t + ry * Kxy; t = t + rz * Kxz; sx[e] = t;
      t = ix * Kxx; t = t + iy * Kxy; t = t + iz * Kxz; sx[e + 1] = t;
      t = rx * Kxy; t = t + ry * Kyy; t = t + rz * Kyz; sy[e] = t;
      t = ix * Kxy; t = t + iy * Kyy; t = t + iz * Kyz; sy[e + 1] = t;
      t = rx * Kxz; t = t + ry * Kyz; t = t + rz * Kzz; sz[e] = t;
      t = ix * Kxz; t = t + iy * Kyz; t = t + iz * Kzz; sz[e + 1] = t;
    } else {
      REAL Kxx = kxx[i], Kyy = kyy[i], Kzz = kzz[i], Kyz = kyz[i];
      REAL t;
      sx[e] = rx * Kxx;
      sx[e + 1] = ix * Kxx;
      t = ry * Kyy; t = t + rz * Kyz; sy[e] = t;
      t = iy * Kyy; t = t + iz * Kyz; sy[e + 1] = t;
      t = ry * Kyz; t = t + rz * Kzz; sz[e] = t;
      t = iy * Kyz; t = t + iz * Kzz; sz[e + 1] = t;
    }
  }
}

/* Conv.Convolve: h = conv(K, m). */
static void convolve(const conv_t* c, const REAL* m, REAL* h) {
  int64_t n = (int64_t)c->N[0] * c->N[1] * c->N[2];
  cplx* spec = (cplx*)malloc(sizeof(cplx) * (size_t)c->nspec);
  REAL* s[3];
  for (int comp = 0; comp < 3; comp++) {
    s[comp] = (REAL*)malloc(sizeof(REAL) * 2 * (size_t)c->nspec);
    conv_forward(c, m + comp * n, c->N[0], c->N[1], c->N[2], spec);
    for (int64_t i = 0; i < c->nspec; i++) {
      s[comp][2 * i] = (REAL)spec[i].re;
      s[comp][2 * i + 1] = (REAL)spec[i].im;
    }
  }
  kernelmul(c, s[0], s[1], s[2]);
  for (int comp = 0; comp < 3; comp++) {
    for (int64_t i = 0; i < c->nspec; i++) {
      spec[i].re = (double)s[comp][2 * i];
      spec[i].im = (double)s[comp][2 * i + 1];
    }
    conv_inverse(c, spec, h + comp * n, c->N[0], c->N[1], c->N[2]);
    free(s[comp]);
  }
  free(spec);
}

/* ------------------------------------------------------------------ */
/* Element-wise primitives, in the reference's operation order.         */
/* ------------------------------------------------------------------ */

/* gpu_add_local_fields, ANIS_NONE and ANIS_UNIAXIAL with uniform Hext
 * (gpu_local_contr3.cu:21-36,133-143,159-229). */
void FN(add_local_fields)(const REAL* m, REAL* h, int64_t N, const REAL hext[3], int anis, REAL K,
                          const REAL u[3]) {
#pragma omp parallel for
  for (int64_t i = 0; i < N; i++) {
    if (anis == 0) {
      for (int c = 0; c < 3; c++) h[c * N + i] = h[c * N + i] + hext[c];
    } else {
      REAL mu = m[i] * u[0];
      mu = mu + m[N + i] * u[1];
      mu = mu + m[2 * N + i] * u[2];
      for (int c = 0; c < 3; c++) {
        REAL t = K * mu;
        t = t * u[c];
        t = hext[c] + t;
        h[c * N + i] = h[c * N + i] + t;
      }
    }
  }
}

/* gpu_scale_dot_product (gpu_linalg.cu:125-140):
 * phi_i = s (a_x b_x + a_y b_y + a_z b_z), left to right. */
void FN(scale_dot_product)(REAL* phi, const REAL* a, const REAL* b, REAL sc, int64_t N) {
#pragma omp parallel for
  for (int64_t i = 0; i < N; i++) {
    REAL d = a[i] * b[i];
    d = d + a[N + i] * b[N + i];
    d = d + a[2 * N + i] * b[2 * N + i];
    phi[i] = sc * d;
  }
}

/* gpu_add_local_fields_H_and_phi, uniform Hext, ANIS_NONE and
 * ANIS_UNIAXIAL (gpu_local_contr3.cu:230-247,362-374,395-466): the fields
 * of add_local_fields, and
 *   phi -= m.Hext + ((0.5 K) mu) (m.u)
 * with each dot product summed left to right. */
void FN(add_local_fields_phi)(const REAL* m, REAL* h, REAL* phi, int64_t N, const REAL hext[3], int anis, REAL K,
                              const REAL u[3]) {
  FN(add_local_fields)(m, h, N, hext, anis, K, u);
#pragma omp parallel for
  for (int64_t i = 0; i < N; i++) {
    REAL mh = m[i] * hext[0];
    mh = mh + m[N + i] * hext[1];
    mh = mh + m[2 * N + i] * hext[2];
    if (anis != 0) {
      REAL mu = m[i] * u[0];
      mu = mu + m[N + i] * u[1];
      mu = mu + m[2 * N + i] * u[2];
      REAL t = (REAL)0.5 * K;
      t = t * mu;
      t = t * mu;
      mh = mh + t;
    }
    phi[i] = phi[i] - mh;
  }
}

/* gpu_deltaM (gpu_torque.cu:20-54): h <- dt_gilb (m x h + alpha m x (m x h))
 * in the internal (left-handed) frame. */
void FN(delta_m)(const REAL* m, REAL* h, int64_t N, REAL alpha, REAL dtg) {
#pragma omp parallel for
  for (int64_t i = 0; i < N; i++) {
    REAL Mx = m[i], My = m[N + i], Mz = m[2 * N + i];
    REAL Hx = h[i], Hy = h[N + i], Hz = h[2 * N + i];
    REAL a = My * Hz, b = Hy * Mz;
    REAL mxHx = a - b;
    a = -Mx * Hz; b = Hx * Mz;
    REAL mxHy = a + b;
    a = Mx * Hy; b = Hx * My;
    REAL mxHz = a - b;
    a = -My * mxHz; b = mxHy * Mz;
    REAL mmx = a + b;
    a = Mx * mxHz; b = mxHx * Mz;
    REAL mmy = a - b;
    a = -Mx * mxHy; b = mxHx * My;
    REAL mmz = a + b;
    REAL t;
    t = mmx * alpha; t = mxHx + t; h[i] = dtg * t;
    t = mmy * alpha; t = mxHy + t; h[N + i] = dtg * t;
    t = mmz * alpha; t = mxHz + t; h[2 * N + i] = dtg * t;
  }
}

/* gpu_normalize_uniform (gpu_normalize.cu:20-28) with a correctly
 * rounded 1/sqrt in place of the fast-math rsqrtf. */
void FN(normalize)(REAL* m, int64_t N) {
#pragma omp parallel for
  for (int64_t i = 0; i < N; i++) {
    REAL s = m[i] * m[i];
    s = s + m[N + i] * m[N + i];
    s = s + m[2 * N + i] * m[2 * N + i];
    REAL inv = (REAL)1. / (REAL)sqrt((double)s);
    if (sizeof(REAL) == 4) inv = (REAL)1.0f / sqrtf((float)s);
    m[i] *= inv;
    m[N + i] *= inv;
    m[2 * N + i] *= inv;
  }
}

/* maximum of |a_i| (gpu_reduction.cu:303-352,609-618; order-free) */
REAL FN(maxabs)(const REAL* a, int64_t n) {
  REAL mx = 0;
  for (int64_t i = 0; i < n; i++) {
    REAL v = a[i] < 0 ? -a[i] : a[i];
    if (v > mx) mx = v;
  }
  return mx;
}

/* Sum in the order of the reference's partial-sum kernel with its launch
 * shape (redux.go:103-121: threads = maxthreads/2 halved while N <= threads,
 * blocks = divUp(N, 2 threads); gpu_reduction.cu:139-190, 576-588). */
REAL FN(ref_sum)(const REAL* a, int64_t n, int maxthreads) {
  int threads = maxthreads / 2;
  if (threads == 0) threads = 1;
  while (n <= threads) threads /= 2;
  int64_t blocks = (n - 1) / (2 * threads) + 1;
  REAL* s = (REAL*)malloc(sizeof(REAL) * threads);
  REAL total = 0;
  int64_t grid = (int64_t)threads * 2 * blocks;
  for (int64_t b = 0; b < blocks; b++) {
    for (int t = 0; t < threads; t++) {
      REAL my = 0;
      for (int64_t i = b * threads * 2 + t; i < n; i += grid) {
        my = my + a[i];
        if (i + threads < n) my = my + a[i + threads];
      }
      s[t] = my;
    }
    for (int w = threads / 2; w >= 1; w /= 2)
      for (int t = 0; t < w; t++) s[t] = s[t] + s[t + w];
    total = total + s[0];
  }
  free(s);
  return total;
}

/* ------------------------------------------------------------------ */
/* Simulation: units, init, field, solvers.                             */
/* ------------------------------------------------------------------ */

enum { SOLVER_HEUN = 0, SOLVER_RK12 = 1, SOLVER_RK23 = 2, SOLVER_RK4 = 3, SOLVER_RKCK = 4, SOLVER_RKDP = 5, SOLVER_RK2 = 6 };

typedef struct {
  int grid[3];       /* user (x,y,z) cell counts */
  double cell[3];    /* user (x,y,z) cell size, m */
  int periodic[3];   /* user (x,y,z) */
  double msat, aexch, alpha;
  double bext[3];    /* applied field, T, user (x,y,z) */
  int anis;          /* 0 none, 1 uniaxial */
  double k1;         /* J/m^3 */
  double axis[3];    /* user (x,y,z) */
  int solver;
  double dt;         /* SI seconds; 0 = default internal 1e-4 */
  double maxerror;   /* 0 = fixed step */
  double mindm, maxdm, mindt, maxdt;
  int exch_type;     /* 6 = 6-neighbour, folded into the kernel */
  int faithful;      /* 1 = keep the FSAL-after-reject quirk */
  int accuracy;      /* face-integral points per side (8) */
  int maxthreads;    /* device maxThreadsPerBlock, sets the sum order */
  double temperature; /* K; 0 = no thermal field */
  int thermal_seed;
} ocfg_t;

typedef struct {
  ocfg_t cfg;
  int N[3], P[3];
  int64_t n;
  REAL L, T, B, ED;   /* units */
  REAL cs[3];         /* internal cell size */
  REAL hext[3], K, u[3], alpha;
  double time;
  REAL dt;
  REAL* m;
  REAL* h;
  conv_t conv;
  /* solver state */
  int stages, fsal, fsal_init, adaptive;
  double errorder;
  REAL a[7][7], b[7], c[7], b2[7];
  REAL* k[7];
  REAL *m0, *mbackup, *m1est, *t0;
  REAL torque, step_error;
  int steps, error;
  int want_energy;  /* Sim.wantEnergy (sim.go:109), set by Relax */
  REAL energy;      /* Sim.energy: the last total energy computed */
  REAL thermal_k;   /* sigma^2 dt of the thermal field (internal units) */
  REAL* noise;      /* the thermal field of the current step (Sim.tempNoise) */
} osim_t;

static void set_tableau(osim_t* s) {
  memset(s->a, 0, sizeof(s->a));
  memset(s->b, 0, sizeof(s->b));
  memset(s->b2, 0, sizeof(s->b2));
  memset(s->c, 0, sizeof(s->c));
  s->fsal = 0;
  s->adaptive = 0;
  switch (s->cfg.solver) {
    case SOLVER_RK2:
    case SOLVER_RK12: /* rk.go:78-99 */
      s->stages = 2;
      s->c[1] = 1; s->a[1][0] = 1; s->b[0] = (REAL).5; s->b[1] = (REAL).5;
      if (s->cfg.solver == SOLVER_RK12) { s->adaptive = 1; s->errorder = 1.; s->b2[0] = 1; }
      break;
    case SOLVER_RK23: /* rk.go:126-139 */
      s->stages = 4; s->fsal = 1;
      s->c[1] = (REAL)(1. / 2.); s->c[2] = (REAL)(3. / 4.); s->c[3] = 1;
      s->a[1][0] = (REAL)(1. / 2.);
      s->a[2][1] = (REAL)(3. / 4.);
      s->a[3][0] = (REAL)(2. / 9.); s->a[3][1] = (REAL)(1. / 3.); s->a[3][2] = (REAL)(4. / 9.);
      s->b[0] = (REAL)(2. / 9.); s->b[1] = (REAL)(1. / 3.); s->b[2] = (REAL)(4. / 9.); s->b[3] = 0;
      s->adaptive = 1; s->errorder = 2.;
      s->b2[0] = (REAL)(7. / 24); s->b2[1] = (REAL)(1. / 4.); s->b2[2] = (REAL)(1. / 3.); s->b2[3] = (REAL)(1. / 8.);
      break;
    case SOLVER_RK4: /* rk.go:149-160 */
      s->stages = 4;
      s->c[1] = (REAL)(1. / 2.); s->c[2] = (REAL)(1. / 2.); s->c[3] = 1;
      s->a[1][0] = (REAL)(1. / 2.); s->a[2][1] = (REAL)(1. / 2.); s->a[3][2] = 1;
      s->b[0] = (REAL)(1. / 6.); s->b[1] = (REAL)(1. / 3.); s->b[2] = (REAL)(1. / 3.); s->b[3] = (REAL)(1. / 6.);
      break;
    case SOLVER_RKCK: { /* rk.go:164-178 */
      s->stages = 6;
      double c[6] = {0., 1. / 5., 3. / 10., 3. / 5., 1., 7. / 8.};
      double a[6][6] = {{0}, {1. / 5.}, {3. / 40., 9. / 40.}, {3. / 10., -9. / 10., 6. / 5.},
                        {-11. / 54., 5. / 2., -70. / 27., 35. / 27.},
                        {1631. / 55296., 175. / 512., 575. / 13824., 44275. / 110592., 253. / 4096.}};
      double b[6] = {37. / 378., 0, 250. / 621., 125. / 594., 0, 512. / 1771.};
      double b2[6] = {2825. / 27648., 0, 18575. / 48384., 13525. / 55296., 277. / 14336., 1. / 4.};
      for (int i = 0; i < 6; i++) {
        s->c[i] = (REAL)c[i]; s->b[i] = (REAL)b[i]; s->b2[i] = (REAL)b2[i];
        for (int j = 0; j < 6; j++) s->a[i][j] = (REAL)a[i][j];
      }
      s->adaptive = 1; s->errorder = 4.;
      break;
    }
    case SOLVER_RKDP: { /* rk.go:196-212 */
      s->stages = 7; s->fsal = 1;
      double c[7] = {0., 1. / 5., 3. / 10., 4. / 5., 8. / 9., 1., 1.};
      double a[7][7] = {{0}, {1. / 5.}, {3. / 40., 9. / 40.}, {44. / 45., -56. / 15., 32. / 9.},
                        {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.},
                        {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.},
                        {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.}};
      double b[7] = {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0};
      double b2[7] = {5179. / 57600., 0., 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100., 1. / 40.};
      for (int i = 0; i < 7; i++) {
        s->c[i] = (REAL)c[i]; s->b[i] = (REAL)b[i]; s->b2[i] = (REAL)b2[i];
        for (int j = 0; j < 7; j++) s->a[i][j] = (REAL)a[i][j];
      }
      s->adaptive = 1; s->errorder = 4.;
      break;
    }
    default:
      s->stages = 0;
  }
}

/* Units (material.go:51-111) with float32 rounding at each operation in
 * the FP32 build. */
static void init_units(osim_t* s) {
  REAL mu0 = (REAL)(4.0e-7 * 3.14159265358979323846);
  REAL gamma0 = (REAL)2.211e5;
  REAL ms = (REAL)s->cfg.msat, A = (REAL)s->cfg.aexch;
  REAL t = mu0 * ms;
  t = t * ms;
  t = A / t;
  s->L = (REAL)sqrt(2. * (double)t);
  REAL g = gamma0 * ms;
  s->T = (REAL)1.0 / g;
  s->B = mu0 * ms;
  REAL ue = A * s->L;
  REAL vol = s->L * s->L;
  vol = vol * s->L;
  s->ED = ue / vol;
}

void* FN(sim_new)(const ocfg_t* cfg, const REAL* m_internal) {
  osim_t* s = (osim_t*)calloc(1, sizeof(osim_t));
  s->cfg = *cfg;
  if (s->cfg.accuracy <= 0) s->cfg.accuracy = 8;
  if (s->cfg.maxthreads <= 0) s->cfg.maxthreads = 1024;
  init_units(s);
  int per[3];
  for (int d = 0; d < 3; d++) {
    s->N[d] = cfg->grid[2 - d];
    per[d] = cfg->periodic[2 - d];
    s->cs[d] = (REAL)cfg->cell[2 - d] / s->L;
    s->P[d] = (s->N[d] > 1 && per[d] == 0) ? 2 * s->N[d] : s->N[d];
    s->hext[d] = (REAL)cfg->bext[2 - d] / s->B;
  }
  s->alpha = (REAL)cfg->alpha;
  s->K = 0;
  if (cfg->anis == 1) {
    s->K = (REAL)cfg->k1 / s->ED;
    /* AnisUniaxial (simanis.go:32-44): internal (x,y,z) = user (z,y,x) */
    REAL ux = (REAL)cfg->axis[2], uy = (REAL)cfg->axis[1], uz = (REAL)cfg->axis[0];
    REAL nn = ux * ux;
    nn = nn + uy * uy;
    nn = nn + uz * uz;
    nn = (REAL)sqrt((double)nn);
    s->u[0] = ux / nn; s->u[1] = uy / nn; s->u[2] = uz / nn;
  }
  s->n = (int64_t)s->N[0] * s->N[1] * s->N[2];
  s->m = (REAL*)malloc(sizeof(REAL) * 3 * s->n);
  s->h = (REAL*)calloc(3 * s->n, sizeof(REAL));
  memcpy(s->m, m_internal, sizeof(REAL) * 3 * s->n);
  /* kernel: FaceKernel6 + exchange folded in (init.go:234-274) */
  int64_t p3 = (int64_t)s->P[0] * s->P[1] * s->P[2];
  REAL* k6 = (REAL*)malloc(sizeof(REAL) * 6 * p3);
  FN(face_kernel6)(s->P, s->cs, s->cfg.accuracy, per, k6);
  if (cfg->exch_type == 6) FN(add_exch6_kernel)(s->P, s->cs, k6);
  conv_init(&s->conv, s->N, s->P, k6);
  free(k6);
  /* solver (init.go:277-287) */
  REAL dtin = (REAL)cfg->dt / s->T;
  s->dt = dtin == 0 ? (REAL)1e-4 : dtin;
  set_tableau(s);
  for (int i = 0; i < 7; i++) s->k[i] = NULL;
  if (cfg->solver == SOLVER_HEUN) {
    s->m1est = (REAL*)calloc(3 * s->n, sizeof(REAL));
    s->t0 = (REAL*)calloc(3 * s->n, sizeof(REAL));
  } else {
    s->k[0] = s->h;
    for (int i = 1; i < s->stages; i++) s->k[i] = (REAL*)calloc(3 * s->n, sizeof(REAL));
    s->m0 = (REAL*)calloc(3 * s->n, sizeof(REAL));
    s->mbackup = (REAL*)calloc(3 * s->n, sizeof(REAL));
  }
  /* thermal field: sigma^2 dt = 2 alpha kB T / (gamma0 mu0 Ms V T_unit) / Ms^2 */
  if (cfg->temperature != 0) {
    double V = cfg->cell[0] * cfg->cell[1] * cfg->cell[2];
    double kB = 1.380650424e-23, g0 = 2.211e5, mu0 = 4.0e-7 * 3.14159265358979323846;
    s->thermal_k = (REAL)(2.0 * cfg->alpha * kB * cfg->temperature / (g0 * mu0 * cfg->msat * V * (double)s->T) /
                          (cfg->msat * cfg->msat));
    s->noise = (REAL*)calloc(3 * s->n, sizeof(REAL));
  }
  /* Sim.Run normalises m before stepping (simrun.go:24) */
  FN(normalize)(s->m, s->n);
  return s;
}

void FN(sim_free)(void* p) {
  osim_t* s = (osim_t*)p;
  conv_free(&s->conv);
  free(s->m); free(s->h);
  for (int i = 1; i < 7; i++) free(s->k[i]);
  free(s->m0); free(s->mbackup); free(s->m1est); free(s->t0);
  free(s->noise);
  free(s);
}

/* calcHeff (field.go:74-80): demag+exchange by convolution, then the
 * local fields. */
void FN(sim_heff)(void* p, const REAL* m, REAL* h) {
  osim_t* s = (osim_t*)p;
  convolve(&s->conv, m, h);
  FN(add_local_fields)(m, h, s->n, s->hext, s->cfg.anis, s->K, s->u);
  /* addThermalField (field.go:74-80, temperature.go:19-22) */
  if (s->noise)
    for (int64_t i = 0; i < 3 * s->n; i++) h[i] = h[i] + s->noise[i];
}

/* Philox-4x32-10 (Salmon et al., SC'11) and two Box-Muller pairs per cell:
 * the engine's thermal-noise stream, restated (counter = cell, step; key =
 * seed and a fixed word). */
static void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1,
             n3 = (uint32_t)p0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}
static void thermal_noise(osim_t* s, REAL sigma, long long step) {
  for (int64_t g = 0; g < s->n; g++) {
    uint32_t c[4] = {(uint32_t)g, (uint32_t)((uint64_t)g >> 32), (uint32_t)step, (uint32_t)((uint64_t)step >> 32)};
    philox10(c, (uint32_t)s->cfg.thermal_seed, 0x4D4D5854u);
    double u1 = ((double)(c[0] >> 8) + 1.0) / 16777216.0, u2 = (double)(c[1] >> 8) / 16777216.0;
    double u3 = ((double)(c[2] >> 8) + 1.0) / 16777216.0, u4 = (double)(c[3] >> 8) / 16777216.0;
    double a = sqrt(-2.0 * log(u1)), b = sqrt(-2.0 * log(u3));
    s->noise[g] = sigma * (REAL)(a * cos(2.0 * M_PI * u2));
    s->noise[s->n + g] = sigma * (REAL)(a * sin(2.0 * M_PI * u2));
    s->noise[2 * s->n + g] = sigma * (REAL)(b * cos(2.0 * M_PI * u4));
  }
}

static void madd(REAL* a, REAL c, const REAL* b, int64_t n) {
#pragma omp parallel for
  for (int64_t i = 0; i < n; i++) a[i] = a[i] + c * b[i];
}

/* AdaptiveHeun.step (adaptive_heun.go:34-76). */
static void heun_step(osim_t* s) {
  int64_t n3 = 3 * s->n;
  REAL dtg = s->dt / ((REAL)1 + s->alpha * s->alpha);
  FN(sim_heff)(s, s->m, s->h);
  FN(delta_m)(s->m, s->h, s->n, s->alpha, dtg);
  memcpy(s->t0, s->h, sizeof(REAL) * n3);
  memcpy(s->m1est, s->m, sizeof(REAL) * n3);
  for (int64_t i = 0; i < n3; i++) s->m1est[i] = s->m1est[i] + s->t0[i];
  FN(normalize)(s->m1est, s->n);
  FN(sim_heff)(s, s->m1est, s->h);
  FN(delta_m)(s->m1est, s->h, s->n, s->alpha, dtg);
  for (int64_t i = 0; i < n3; i++) {
    REAL a = (REAL)0.5 * s->h[i];
    REAL b = (REAL)0.5 * s->t0[i];
    s->h[i] = a + b;
    s->m[i] = s->m[i] + s->h[i];
  }
  FN(normalize)(s->m, s->n);
  s->time += (double)s->dt;
  if (s->cfg.maxerror != 0.) {
    madd(s->m1est, (REAL)-1, s->m, n3);
    REAL err = FN(maxabs)(s->m1est, n3);
    s->step_error = err;
    REAL factor = (REAL)s->cfg.maxerror / err;
    if (factor > 2) factor = 2;
    if (factor < (REAL)0.01) factor = (REAL)0.01;
    s->dt = s->dt * factor;
  }
}

void FN(sim_energy)(void* p, const REAL* m, REAL* out);

/* RK.step (rk.go:279-445). */
static void rk_step(osim_t* s) {
  int order = s->stages;
  int64_t n3 = 3 * s->n;
  double time0 = s->time;
  REAL* m = s->m;
  REAL* m1 = s->m0;
  REAL dtg1 = (REAL)1 / ((REAL)1 + s->alpha * s->alpha);
  memcpy(s->mbackup, m, sizeof(REAL) * n3);
  int good = 0, trials = 0;
  const REAL maxErr = (REAL)s->cfg.maxerror;
  const REAL ut = s->T;
  /* the thermal noise of this step (rk.go:289-292, temperature.go:27-36) */
  const int thermal = s->noise != NULL;
  if (thermal) thermal_noise(s, (REAL)sqrt((double)(s->thermal_k / s->dt)), s->steps);
  /* energy must not rise when it is wanted (rk.go:297-301,425) */
  REAL prevEnergy = s->energy;
  if (prevEnergy == 0) prevEnergy = (REAL)9999999999.;
  while (!good && trials < 10) {
    trials++;
    for (int i = 0; i < order; i++) {
      if (s->fsal && i == 0 && s->fsal_init) {
        memcpy(s->k[0], s->k[order - 1], sizeof(REAL) * n3);
      } else {
        s->time = time0 + (double)(s->c[i] * s->dt);
        memcpy(m1, m, sizeof(REAL) * n3);
        for (int j = 0; j < order; j++)
          if (s->a[i][j] != 0) madd(m1, s->dt * s->a[i][j], s->k[j], n3);
        /* calcHeffEnergy at the last stage (FSAL) or the first (rk.go:321-337) */
        if (s->want_energy && ((s->fsal && i == order - 1) || (!s->fsal && i == 0)))
          FN(sim_energy)(s, m1, &s->energy);
        FN(sim_heff)(s, m1, s->k[i]);
        FN(delta_m)(m1, s->k[i], s->n, s->alpha, dtg1);
        s->fsal_init = 1;
      }
      if (i == 0 && !thermal) {
        REAL maxT = FN(maxabs)(s->k[0], n3);
        s->torque = maxT;
        REAL dm = s->dt * maxT;
        if (dm < (REAL)s->cfg.mindm) s->dt = (REAL)s->cfg.mindm / maxT;
        if (s->dt * ut < (REAL)s->cfg.mindt) s->dt = (REAL)s->cfg.mindt / ut;
        if (s->cfg.maxdm != 0 && dm > (REAL)s->cfg.maxdm) s->dt = (REAL)s->cfg.maxdm / maxT;
        if (s->cfg.maxdt != 0 && s->dt * ut > (REAL)s->cfg.maxdt) s->dt = (REAL)s->cfg.maxdt / ut;
        if (s->dt != s->dt) { s->error = 1; return; }
      }
    }
    s->time = time0 + (double)s->dt;
    if (s->adaptive) {
      memcpy(m1, m, sizeof(REAL) * n3);
      for (int i = 0; i < order; i++)
        if (s->b2[i] != 0) madd(m1, s->b2[i] * s->dt, s->k[i], n3);
    }
    for (int i = 0; i < order; i++)
      if (s->b[i] != 0) madd(m, s->b[i] * s->dt, s->k[i], n3);
    if (s->adaptive) {
      madd(m1, (REAL)-1, m, n3);
      REAL err = FN(maxabs)(m1, n3);
      s->step_error = err;
      REAL factor = (REAL)pow((double)(maxErr / err), 1. / s->errorder);
      if (factor > 2) factor = 2;
      if (factor < (REAL)0.01) factor = (REAL)0.01;
      s->dt = s->dt * factor;
      if (s->dt != s->dt) { s->error = 1; return; }
      if (err > 2 * maxErr || (s->want_energy && s->energy > prevEnergy)) {
        memcpy(m, s->mbackup, sizeof(REAL) * n3);
        good = 0;
        if (!s->cfg.faithful) s->fsal_init = 0;
      } else {
        good = 1;
        if (s->dt * ut < (REAL)s->cfg.mindt) s->dt = (REAL)s->cfg.mindt / ut;
        if (s->cfg.maxdt != 0 && s->dt * ut > (REAL)s->cfg.maxdt) s->dt = (REAL)s->cfg.maxdt / ut;
      }
    } else {
      good = 1;
    }
  }
  FN(normalize)(m, s->n);
}

/* One solver step; returns 0 or an error code (NaN dt). */
int FN(sim_step)(void* p) {
  osim_t* s = (osim_t*)p;
  if (s->cfg.solver == SOLVER_HEUN) heun_step(s);
  else rk_step(s);
  s->steps++;
  if (s->time != s->time) s->error = 1;
  return s->error;
}

int FN(sim_steps)(void* p, int n) {
  for (int i = 0; i < n; i++) {
    int e = FN(sim_step)(p);
    if (e) return e;
  }
  return 0;
}

void FN(sim_get_m)(void* p, REAL* out) {
  osim_t* s = (osim_t*)p;
  memcpy(out, s->m, sizeof(REAL) * 3 * s->n);
}
void FN(sim_set_m)(void* p, const REAL* in) {
  osim_t* s = (osim_t*)p;
  memcpy(s->m, in, sizeof(REAL) * 3 * s->n);
}
double FN(sim_time)(void* p) { return ((osim_t*)p)->time; }
double FN(sim_dt)(void* p) { return (double)((osim_t*)p)->dt; }
double FN(sim_unit)(void* p, int which) {
  osim_t* s = (osim_t*)p;
  switch (which) {
    case 0: return s->L;
    case 1: return s->T;
    case 2: return s->B;
    case 3: return s->ED;
    case 4: return s->K;
    default: return 0;
  }
}
void FN(sim_internal_params)(void* p, REAL* cs3, REAL* hext3, REAL* u3, REAL* alpha_K) {
  osim_t* s = (osim_t*)p;
  for (int d = 0; d < 3; d++) { cs3[d] = s->cs[d]; hext3[d] = s->hext[d]; u3[d] = s->u[d]; }
  alpha_K[0] = s->alpha;
  alpha_K[1] = s->K;
}
/* real-part kernel spectrum (P0,P1,HZ) of component comp, for tests */
void FN(sim_kernel_spectrum)(void* p, int comp, REAL* out) {
  osim_t* s = (osim_t*)p;
  memcpy(out, s->conv.kern + comp * s->conv.nspec, sizeof(REAL) * s->conv.nspec);
}
/* <m> per internal component with the reference's sum order
 * (simoutput.go:236, simget.go:32) */
void FN(sim_avg_m)(void* p, REAL out[3]) {
  osim_t* s = (osim_t*)p;
  for (int c = 0; c < 3; c++) out[c] = FN(ref_sum)(s->m + c * s->n, s->n, s->cfg.maxthreads) / (REAL)s->n;
}
/* Total energy of m, internal units: calcHeffEnergy (field.go:64-71,
 * 83-87): the demag + exchange field h, phi = -1/2 m.h
 * (calcHDemagExchEdens, field.go:17-20), the local fields and their energy
 * density (addLocalFieldsEdens, field.go:44-47), then sumEdens
 * (energy.go:49-52): the Reductor's sum of phi times the cell volume
 * cs_X cs_Y cs_Z (energy.go:38-44).  The FP32 build sums in the
 * reference's partial-sum order; the FP64 build sums in float64. */
void FN(sim_energy)(void* p, const REAL* m, REAL* out) {
  osim_t* s = (osim_t*)p;
  REAL* h = (REAL*)malloc(sizeof(REAL) * 3 * s->n);
  REAL* phi = (REAL*)malloc(sizeof(REAL) * s->n);
  convolve(&s->conv, m, h);
  FN(scale_dot_product)(phi, m, h, (REAL)-0.5, s->n);
  FN(add_local_fields_phi)(m, h, phi, s->n, s->hext, s->cfg.anis, s->K, s->u);
  REAL total;
  if (sizeof(REAL) == 4) {
    total = FN(ref_sum)(phi, s->n, s->cfg.maxthreads);
  } else {
    double acc = 0;
    for (int64_t i = 0; i < s->n; i++) acc += (double)phi[i];
    total = (REAL)acc;
  }
  REAL vol = s->cs[0] * s->cs[1];
  vol = vol * s->cs[2];
  *out = total * vol;
  free(h);
  free(phi);
}

/* Sim.Run with a periodic table output (simrun.go:19-57,
 * simoutput.go:76-90,226-272): before each step, Periodic.NeedSave with
 * the float32 time t = float32(time) * UnitTime (t == 0 or
 * t - sinceoutput >= period) writes one row
 *   {t, <m_x>, <m_y>, <m_z>, torque, min m_z, max m_z}
 * in user order (<m_x> is the internal Z component; <m> is the Reductor's
 * sum / N, simoutput.go:236-239; torque is the last maximum torque,
 * simoutput.go:250-257; min/max of internal component X,
 * simoutput.go:258-261), then sinceoutput = t.  Steps while
 * time < stop (internal units).  Returns the rows written (at most
 * max_rows) or -1 on a NaN; *since carries sinceoutput between calls. */
int FN(sim_run_table)(void* p, double duration, float period, float* rows, int max_rows, float* since) {
  osim_t* s = (osim_t*)p;
  double stop = s->time + duration;
  int nrow = 0;
  FN(normalize)(s->m, s->n);
  while (s->time < stop) {
    float t = (float)s->time;
    volatile float tt = t * (float)s->T;
    t = tt;
    volatile float d = t - *since;
    if ((t == 0.f || d >= period) && nrow < max_rows) {
      float* r = rows + 7 * nrow;
      REAL av[3];
      FN(sim_avg_m)(p, av);
      r[0] = t;
      r[1] = (float)av[2];
      r[2] = (float)av[1];
      r[3] = (float)av[0];
      r[4] = (float)s->torque;
      REAL mn = s->m[0], mx = s->m[0];
      for (int64_t i = 1; i < s->n; i++) {
        if (s->m[i] < mn) mn = s->m[i];
        if (s->m[i] > mx) mx = s->m[i];
      }
      r[5] = (float)mn;
      r[6] = (float)mx;
      *since = t;
      nrow++;
    }
    if (FN(sim_step)(p)) return -1;
  }
  return nrow;
}

/* Sim.Relax (relax.go:14-23): with the energy wanted, one step, then steps
 * while the energy does not rise; the energies compared are the ones the
 * RK steps compute (float32 in the FP32 build).  At most max_steps steps;
 * returns the steps taken, or -1 on a NaN.  wantEnergy stays set, as in
 * the reference. */
long long FN(sim_relax)(void* p, long long max_steps) {
  osim_t* s = (osim_t*)p;
  s->want_energy = 1;
  long long k = 0;
  if (FN(sim_step)(p)) return -1;
  k++;
  REAL prevE = s->energy + 1;
  while (s->energy <= prevE && k < max_steps) {
    prevE = s->energy;
    if (FN(sim_step)(p)) return -1;
    k++;
  }
  return k;
}
double FN(sim_last_energy)(void* p) { return (double)((osim_t*)p)->energy; }

REAL FN(sim_torque)(void* p) { return ((osim_t*)p)->torque; }
REAL FN(sim_step_error)(void* p) { return ((osim_t*)p)->step_error; }

/* Stand-alone padded convolution for tests: h = conv(kernel(size,cell), m)
 * with the kernel built from internal sizes and internal cell size. */
void FN(convolve_standalone)(const int N[3], const int periodic[3], const REAL cs[3], int exch, const REAL* m,
                             REAL* h) {
  int P[3];
  for (int d = 0; d < 3; d++) P[d] = (N[d] > 1 && periodic[d] == 0) ? 2 * N[d] : N[d];
  int64_t p3 = (int64_t)P[0] * P[1] * P[2];
  REAL* k6 = (REAL*)malloc(sizeof(REAL) * 6 * p3);
  FN(face_kernel6)(P, cs, 8, periodic, k6);
  if (exch) FN(add_exch6_kernel)(P, cs, k6);
  conv_t c;
  conv_init(&c, N, P, k6);
  free(k6);
  convolve(&c, m, h);
  conv_free(&c);
}

/* Reference-layout forward transform of a real (N0,N1,N2) array padded to
 * (P0,P1,P2): output (P0,P1,P2+2) floats, interleaved half spectrum, as
 * gpuFFT3dPlan_forward leaves it (gpu_fft0.cu:96-101). */
void FN(fft_forward_padded)(const int N[3], const int P[3], const REAL* in, REAL* out) {
  conv_t c;
  memset(&c, 0, sizeof(c));
  for (int d = 0; d < 3; d++) { c.N[d] = N[d]; c.P[d] = P[d]; plan_init(&c.pl[d], P[d]); }
  c.HZ = P[2] / 2 + 1;
  c.nspec = (int64_t)P[0] * P[1] * c.HZ;
  cplx* spec = (cplx*)malloc(sizeof(cplx) * (size_t)c.nspec);
  conv_forward(&c, in, N[0], N[1], N[2], spec);
  for (int64_t i = 0; i < c.nspec; i++) { out[2 * i] = (REAL)spec[i].re; out[2 * i + 1] = (REAL)spec[i].im; }
  free(spec);
  for (int d = 0; d < 3; d++) plan_free(&c.pl[d]);
}

/* Reference-layout inverse: (P0,P1,P2+2) half spectrum -> real (N0,N1,N2),
 * unnormalised (gpu_fft0.cu:105-109). */
void FN(fft_inverse_padded)(const int N[3], const int P[3], const REAL* in, REAL* out) {
  conv_t c;
  memset(&c, 0, sizeof(c));
  for (int d = 0; d < 3; d++) { c.N[d] = N[d]; c.P[d] = P[d]; plan_init(&c.pl[d], P[d]); }
  c.HZ = P[2] / 2 + 1;
  c.nspec = (int64_t)P[0] * P[1] * c.HZ;
  cplx* spec = (cplx*)malloc(sizeof(cplx) * (size_t)c.nspec);
  for (int64_t i = 0; i < c.nspec; i++) { spec[i].re = in[2 * i]; spec[i].im = in[2 * i + 1]; }
  conv_inverse(&c, spec, out, N[0], N[1], N[2]);
  free(spec);
  for (int d = 0; d < 3; d++) plan_free(&c.pl[d]);
}

int FN(num_threads)(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
