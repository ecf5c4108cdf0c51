// C++ restatement of the reference's Go driver for the LLG hot path,
// driving a libgpukern implementation through its C ABI (see
// include/mmx_driver.h).  Every float32 scalar the Go code computes is
// computed here in float32 with one rounding per operation; float64 where
// the Go code uses float64 (time, sqrt in UnitLength, pow in the RK
// controller).
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "mmx.h"
#include "mmx_driver.h"

static thread_local std::string g_err;
extern "C" const char* mmxd_last_error(void) { return g_err.c_str(); }

// float32 operations with one rounding each
static inline float f_mul(float a, float b) { volatile float r = a * b; return r; }
static inline float f_div(float a, float b) { volatile float r = a / b; return r; }
static inline float f_add(float a, float b) { volatile float r = a + b; return r; }

struct mmxd_lib {
  void* h = nullptr;
  int (*maxthreads)();
  void (*init)(int, int);
  float* (*new_array)(int);
  void (*free_array)(float*);
  void (*memcpy_dir)(float*, float*, int, int);
  void (*zero)(float*, int);
  void (*add)(float*, float*, int);
  void (*madd)(float*, float, float*, int);
  void (*lincomb)(float*, float*, float, float, int);
  float (*reduce)(int, float*, float*, float*, int, int, int);
  void (*normalize)(float*, int);
  void (*deltaM)(float*, float*, float, float*, float, int);
  void (*local)(float*, float*, int, float*, float*, int, float*, float*);
  void (*local_phi)(float*, float*, float*, int, float*, float*, int, float*, float*);
  void (*scale_dot)(float*, float*, float*, float, int);
  void (*kmul6)(float*, float*, float*, float*, float*, float*, float*, float*, float*, int);
  void (*kmul4)(float*, float*, float*, float*, float*, float*, float*, int);
  void* (*plan_new)(int*, int*);
  void (*plan_del)(void*);
  void (*fwd)(void*, float*, float*);
  void (*inv)(void*, float*, float*);
};

template <typename F>
static bool sym(void* h, const char* name, F* out) {
  *out = (F)dlsym(h, name);
  if (!*out) {
    g_err = std::string("missing symbol ") + name;
    return false;
  }
  return true;
}

extern "C" mmxd_lib* mmxd_open(const char* path) {
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    g_err = dlerror();
    return nullptr;
  }
  mmxd_lib* L = new mmxd_lib();
  L->h = h;
  bool ok = sym(h, "gpu_maxthreads", &L->maxthreads) && sym(h, "gpu_init", &L->init) &&
            sym(h, "new_gpu_array", &L->new_array) && sym(h, "free_gpu_array", &L->free_array) &&
            sym(h, "memcpy_gpu_dir", &L->memcpy_dir) && sym(h, "gpu_zero", &L->zero) && sym(h, "gpu_add", &L->add) &&
            sym(h, "gpu_madd", &L->madd) && sym(h, "gpu_linear_combination", &L->lincomb) &&
            sym(h, "gpu_reduce", &L->reduce) && sym(h, "gpu_normalize_uniform", &L->normalize) &&
            sym(h, "gpu_deltaM", &L->deltaM) && sym(h, "gpu_add_local_fields", &L->local) &&
            sym(h, "gpu_add_local_fields_H_and_phi", &L->local_phi) &&
            sym(h, "gpu_scale_dot_product", &L->scale_dot) &&
            sym(h, "gpu_kernelmul6", &L->kmul6) && sym(h, "gpu_kernelmul4", &L->kmul4) &&
            sym(h, "new_gpuFFT3dPlan_padded", &L->plan_new) && sym(h, "delete_gpuFFT3dPlan", &L->plan_del) &&
            sym(h, "gpuFFT3dPlan_forward", &L->fwd) && sym(h, "gpuFFT3dPlan_inverse", &L->inv);
  if (!ok) {
    dlclose(h);
    delete L;
    return nullptr;
  }
  L->init(0, 0);  // Gpu.init (gpu.go:38-49): threads 0 = device maximum
  return L;
}

extern "C" void mmxd_close(mmxd_lib* L) {
  if (!L) return;
  dlclose(L->h);
  delete L;
}

// Reductor (redux.go:103-121)
struct Reductor {
  int op = 0, blocks = 0, threads = 0, N = 0;
  float* dev = nullptr;
  std::vector<float> host;
  void init(mmxd_lib* L, int op_, int n) {
    op = op_;
    N = n;
    threads = L->maxthreads() / 2;
    if (threads == 0) threads = 1;
    while (n <= threads) threads /= 2;
    blocks = (n - 1) / (threads * 2) + 1;
    dev = L->new_array(blocks);
    host.assign(blocks, 0.f);
  }
  float reduce(mmxd_lib* L, float* in) { return L->reduce(op, in, dev, host.data(), blocks, threads, N); }
};

enum { RED_ADD = 1, RED_MAX = 2, RED_MAXABS = 3, RED_MIN = 4 };

struct mmxd_sim {
  mmxd_lib* L;
  mmxd_config cfg;
  int N[3], P[3], per[3];
  int n, n3;
  float unitL, unitT, unitB, unitE;
  float cs[3], hext[3], anisK[3], axes[3], alpha;
  int anis;
  float* m = nullptr;
  float* h = nullptr;
  float* buf[3] = {nullptr, nullptr, nullptr};
  float* kern[6] = {nullptr};
  void* plan = nullptr;
  int ktype = 6;
  int64_t guard = 0;
  // solver
  double time = 0;
  float dt = 0, torque = 0, stepError = 0;
  long long steps = 0;
  int stages = 0, fsal = 0, fsalInit = 0, adaptive = 0;
  double errorder = 1;
  float a[7][7], b[7], b2[7], c[7];
  float* k[7] = {nullptr};
  float *m0 = nullptr, *mbackup = nullptr, *m1est = nullptr, *t0 = nullptr;
  Reductor maxabs, sum, vmin, vmax;
  float avgNorm = 1;
  float* phi = nullptr;     // energy density (initEDens, energy.go:71-78)
  float since = 0;          // Periodic.sinceoutput of the table (simoutput.go:77-80)
  std::vector<float*> owned;
};

// Every 3-component array the reference may unpad into gets
// (P0 - N0) * N1 * N2 guard floats: the reference's gpu_copy_unpad writes
// that many values past its destination (gpu_zeropad.cu:97-107).
static float* alloc3(mmxd_sim* s) {
  float* p = s->L->new_array((int)(s->n3 + s->guard));
  s->owned.push_back(p);
  return p;
}

static void set_tableau(mmxd_sim* s) {
  memset(s->a, 0, sizeof(s->a));
  memset(s->b, 0, sizeof(s->b));
  memset(s->b2, 0, sizeof(s->b2));
  memset(s->c, 0, sizeof(s->c));
  switch (s->cfg.solver) {
    case MMX_SOLVER_RK2:
    case MMX_SOLVER_RK12:  // rk.go:78-99
      s->stages = 2;
      s->c[1] = 1; s->a[1][0] = 1; s->b[0] = .5f; s->b[1] = .5f;
      if (s->cfg.solver == MMX_SOLVER_RK12) { s->adaptive = 1; s->errorder = 1; s->b2[0] = 1; }
      break;
    case MMX_SOLVER_RK23:  // rk.go:126-139
      s->stages = 4; s->fsal = 1;
      s->c[1] = (float)(1. / 2.); s->c[2] = (float)(3. / 4.); s->c[3] = 1;
      s->a[1][0] = (float)(1. / 2.);
      s->a[2][1] = (float)(3. / 4.);
      s->a[3][0] = (float)(2. / 9.); s->a[3][1] = (float)(1. / 3.); s->a[3][2] = (float)(4. / 9.);
      s->b[0] = (float)(2. / 9.); s->b[1] = (float)(1. / 3.); s->b[2] = (float)(4. / 9.);
      s->adaptive = 1; s->errorder = 2;
      s->b2[0] = (float)(7. / 24); s->b2[1] = (float)(1. / 4.); s->b2[2] = (float)(1. / 3.); s->b2[3] = (float)(1. / 8.);
      break;
    case MMX_SOLVER_RK4:  // rk.go:149-160, stepped with the internal dt
      s->stages = 4;
      s->c[1] = .5f; s->c[2] = .5f; s->c[3] = 1;
      s->a[1][0] = .5f; s->a[2][1] = .5f; s->a[3][2] = 1;
      s->b[0] = (float)(1. / 6.); s->b[1] = (float)(1. / 3.); s->b[2] = (float)(1. / 3.); s->b[3] = (float)(1. / 6.);
      break;
    default:
      s->stages = 0;
  }
}

extern "C" void mmxd_sizes(mmxd_sim* s, int N[3], int P[3]) {
  for (int d = 0; d < 3; d++) { N[d] = s->N[d]; P[d] = s->P[d]; }
}
extern "C" void mmxd_internal(mmxd_sim* s, float cs[3], float hext[3], float axis[3], double scal[6]) {
  for (int d = 0; d < 3; d++) { cs[d] = s->cs[d]; hext[d] = s->hext[d]; axis[d] = s->axes[d]; }
  scal[0] = s->alpha; scal[1] = s->anisK[0]; scal[2] = s->dt;
  scal[3] = s->unitT; scal[4] = s->unitB; scal[5] = s->unitL;
}

// Conv.Convolve (conv.go:57-100)
static void convolve(mmxd_sim* s, float* m, float* h) {
  mmxd_lib* L = s->L;
  for (int i = 0; i < 3; i++) L->fwd(s->plan, m + (int64_t)i * s->n, s->buf[i]);
  int nreal = s->P[0] * s->P[1] * (s->P[2] + 2);
  if (s->ktype == 6)
    L->kmul6(s->buf[0], s->buf[1], s->buf[2], s->kern[0], s->kern[1], s->kern[2], s->kern[3], s->kern[4], s->kern[5], nreal);
  else
    L->kmul4(s->buf[0], s->buf[1], s->buf[2], s->kern[0], s->kern[1], s->kern[2], s->kern[3], nreal);
  for (int i = 0; i < 3; i++) L->inv(s->plan, s->buf[i], h + (int64_t)i * s->n);
}

// calcHeff (field.go:74-80): conv + local fields
static void calc_heff(mmxd_sim* s, float* m, float* h) {
  convolve(s, m, h);
  float K[3] = {s->anisK[0], s->anisK[1], s->anisK[2]};
  s->L->local(m, h, s->n, s->hext, nullptr, s->anis, K, s->axes);
}

// DeltaM (torque.go:33-54)
static void delta_m(mmxd_sim* s, float* m, float* h, float dt) {
  float dtg = f_div(dt, f_add(1.f, f_mul(s->alpha, s->alpha)));
  s->L->deltaM(m, h, s->alpha, nullptr, dtg, s->n);
}

extern "C" mmxd_sim* mmxd_new(mmxd_lib* L, const mmxd_config* cfg, const float* m_init, const float* k6) {
  if (!L || !cfg || !m_init || !k6) { g_err = "null argument"; return nullptr; }
  mmxd_sim* s = new mmxd_sim();
  s->L = L;
  s->cfg = *cfg;
  // initMaterial / units (init.go:80-113, material.go:51-111)
  float mu0 = (float)(4.0e-7 * M_PI), gamma0 = 2.211e5f;
  float ms = (float)cfg->msat, A = (float)cfg->aexch;
  float t = f_mul(f_mul(mu0, ms), ms);
  s->unitL = (float)sqrt(2. * (double)f_div(A, t));
  s->unitT = f_div(1.f, f_mul(gamma0, ms));
  s->unitB = f_mul(mu0, ms);
  float vol = f_mul(f_mul(s->unitL, s->unitL), s->unitL);
  s->unitE = f_div(f_mul(A, s->unitL), vol);
  // grid and cell size with the axis swap (simgeom.go:25-55, init.go:116-148)
  for (int d = 0; d < 3; d++) {
    s->N[d] = cfg->grid[2 - d];
    s->per[d] = cfg->periodic[2 - d];
    s->cs[d] = f_div((float)cfg->cell[2 - d], s->unitL);
    s->P[d] = (s->N[d] > 1 && s->per[d] == 0) ? 2 * s->N[d] : s->N[d];  // padSize (kernel.go:80-90)
    s->hext[d] = f_div((float)cfg->bext[2 - d], s->unitB);              // updateHext (field.go:50-61)
  }
  s->alpha = (float)cfg->alpha;
  s->anis = cfg->anis_type;
  s->anisK[0] = s->anisK[1] = s->anisK[2] = 0.f;
  s->axes[0] = s->axes[1] = s->axes[2] = 0.f;
  if (s->anis == 1) {
    s->anisK[0] = f_div((float)cfg->k1, s->unitE);
    float ux = (float)cfg->anis_axis[2], uy = (float)cfg->anis_axis[1], uz = (float)cfg->anis_axis[0];
    float nn = (float)sqrt((double)f_add(f_add(f_mul(ux, ux), f_mul(uy, uy)), f_mul(uz, uz)));
    s->axes[0] = f_div(ux, nn);
    s->axes[1] = f_div(uy, nn);
    s->axes[2] = f_div(uz, nn);
  }
  s->n = s->N[0] * s->N[1] * s->N[2];
  s->n3 = 3 * s->n;
  s->guard = (int64_t)(s->P[0] - s->N[0]) * s->N[1] * s->N[2];
  s->avgNorm = (float)s->n;
  // device memory (initDevMem, init.go:151-168)
  s->m = alloc3(s);
  s->h = alloc3(s);
  L->memcpy_dir((float*)m_init, s->m, s->n3, 1);
  s->maxabs.init(L, RED_MAXABS, s->n3);
  s->sum.init(L, RED_ADD, s->n);
  s->vmin.init(L, RED_MIN, s->n);
  s->vmax.init(L, RED_MAX, s->n);
  // convolution (init.go:234-274, conv.go:35-167)
  s->ktype = s->P[0] == 1 ? 4 : 6;
  int complexN = s->P[0] * s->P[1] * (s->P[2] + 2);
  for (int i = 0; i < 3; i++) {
    s->buf[i] = L->new_array(complexN);
    s->owned.push_back(s->buf[i]);
  }
  s->plan = L->plan_new(s->N, s->P);
  {
    int64_t p3 = (int64_t)s->P[0] * s->P[1] * s->P[2];
    void* kplan = L->plan_new(s->P, s->P);
    float* devIn = L->new_array((int)p3);
    float* devOut = L->new_array(complexN);
    std::vector<float> host((size_t)complexN);
    float norm = f_div(1.f, (float)p3);
    int klen = s->P[0] * s->P[1] * ((s->P[2] + 2) / 2);
    for (int i = 0; i < 6; i++) {
      if (s->ktype == 4 && (i == 4 || i == 5)) continue;  // needKernComp (conv.go:182-193)
      L->memcpy_dir((float*)(k6 + i * p3), devIn, (int)p3, 1);
      L->fwd(kplan, devIn, devOut);
      L->memcpy_dir(devOut, host.data(), complexN, 3);
      for (int j = 0; j < complexN / 2; j++) host[j] = f_mul(host[2 * j], norm);
      s->kern[i] = L->new_array(klen);
      s->owned.push_back(s->kern[i]);
      L->memcpy_dir(host.data(), s->kern[i], klen, 1);
    }
    L->plan_del(kplan);
    L->free_array(devIn);
    L->free_array(devOut);
  }
  // solver (init.go:277-287, solver.go)
  float dtin = f_div((float)cfg->dt, s->unitT);
  s->dt = dtin == 0.f ? 1e-4f : dtin;
  set_tableau(s);
  if (cfg->solver == MMX_SOLVER_HEUN) {
    s->m1est = alloc3(s);
    s->t0 = alloc3(s);
  } else {
    if (s->stages == 0) { g_err = "unsupported solver"; mmxd_free(s); return nullptr; }
    s->k[0] = s->h;
    for (int i = 1; i < s->stages; i++) s->k[i] = alloc3(s);
    s->m0 = alloc3(s);
    s->mbackup = alloc3(s);
  }
  L->normalize(s->m, s->n);  // Sim.Run (simrun.go:24)
  return s;
}

extern "C" void mmxd_free(mmxd_sim* s) {
  if (!s) return;
  for (float* p : s->owned) s->L->free_array(p);
  if (s->maxabs.dev) s->L->free_array(s->maxabs.dev);
  if (s->sum.dev) s->L->free_array(s->sum.dev);
  if (s->vmin.dev) s->L->free_array(s->vmin.dev);
  if (s->vmax.dev) s->L->free_array(s->vmax.dev);
  if (s->phi) s->L->free_array(s->phi);
  if (s->plan) s->L->plan_del(s->plan);
  delete s;
}

// AdaptiveHeun.step (adaptive_heun.go:34-76)
static void heun_step(mmxd_sim* s) {
  mmxd_lib* L = s->L;
  calc_heff(s, s->m, s->h);
  delta_m(s, s->m, s->h, s->dt);
  L->memcpy_dir(s->h, s->t0, s->n3, 2);
  L->memcpy_dir(s->m, s->m1est, s->n3, 2);
  L->add(s->m1est, s->t0, s->n3);
  L->normalize(s->m1est, s->n);
  calc_heff(s, s->m1est, s->h);
  delta_m(s, s->m1est, s->h, s->dt);
  L->lincomb(s->h, s->t0, 0.5f, 0.5f, s->n3);
  L->add(s->m, s->h, s->n3);
  L->normalize(s->m, s->n);
  s->time += (double)s->dt;
  if (s->cfg.maxerror != 0.) {
    L->madd(s->m1est, -1.f, s->m, s->n3);
    float err = s->maxabs.reduce(L, s->m1est);
    s->stepError = err;
    float factor = f_div((float)s->cfg.maxerror, err);
    if (factor > 2.f) factor = 2.f;
    if (factor < 0.01f) factor = 0.01f;
    s->dt = f_mul(s->dt, factor);
  }
}

// RK.step (rk.go:279-445)
static int rk_step(mmxd_sim* s) {
  mmxd_lib* L = s->L;
  int order = s->stages;
  double time0 = s->time;
  float* m = s->m;
  float* m1 = s->m0;
  const float ut = s->unitT;
  const float maxErr = (float)s->cfg.maxerror;
  L->memcpy_dir(m, s->mbackup, s->n3, 2);
  int good = 0, trials = 0;
  while (!good && trials < 10) {
    trials++;
    for (int i = 0; i < order; i++) {
      if (s->fsal && i == 0 && s->fsalInit) {
        if (trials == 1 || s->cfg.faithful) L->memcpy_dir(s->k[order - 1], s->k[0], s->n3, 2);
      } else {
        s->time = time0 + (double)f_mul(s->c[i], s->dt);
        L->memcpy_dir(m, m1, s->n3, 2);
        for (int j = 0; j < order; j++)
          if (s->a[i][j] != 0.f) L->madd(m1, f_mul(s->dt, s->a[i][j]), s->k[j], s->n3);
        calc_heff(s, m1, s->k[i]);
        delta_m(s, m1, s->k[i], 1.0f);  // Torque (torque.go:98-101)
        s->fsalInit = 1;
      }
      if (i == 0) {
        float mt = s->maxabs.reduce(L, s->k[0]);
        s->torque = mt;
        float dm = f_mul(s->dt, mt);
        if (dm < (float)s->cfg.mindm) s->dt = f_div((float)s->cfg.mindm, mt);
        if (f_mul(s->dt, ut) < (float)s->cfg.mindt) s->dt = f_div((float)s->cfg.mindt, ut);
        if (s->cfg.maxdm != 0 && dm > (float)s->cfg.maxdm) s->dt = f_div((float)s->cfg.maxdm, mt);
        if (s->cfg.maxdt != 0 && f_mul(s->dt, ut) > (float)s->cfg.maxdt) s->dt = f_div((float)s->cfg.maxdt, ut);
        if (s->dt != s->dt) { g_err = "dt = NaN"; return MMX_ERR_NAN; }
      }
    }
    s->time = time0 + (double)s->dt;
    if (s->adaptive) {
      L->memcpy_dir(m, m1, s->n3, 2);
      for (int i = 0; i < order; i++)
        if (s->b2[i] != 0.f) L->madd(m1, f_mul(s->b2[i], s->dt), s->k[i], s->n3);
    }
    for (int i = 0; i < order; i++)
      if (s->b[i] != 0.f) L->madd(m, f_mul(s->b[i], s->dt), s->k[i], s->n3);
    if (s->adaptive) {
      L->madd(m1, -1.f, m, s->n3);
      float err = s->maxabs.reduce(L, m1);
      s->stepError = err;
      float factor = (float)pow((double)f_div(maxErr, err), 1. / s->errorder);
      if (factor > 2.f) factor = 2.f;
      if (factor < 0.01f) factor = 0.01f;
      s->dt = f_mul(s->dt, factor);
      if (s->dt != s->dt) { g_err = "dt = NaN"; return MMX_ERR_NAN; }
      if (err > f_mul(2.f, maxErr)) {
        L->memcpy_dir(s->mbackup, m, s->n3, 2);
        good = 0;
      } else {
        good = 1;
        if (f_mul(s->dt, ut) < (float)s->cfg.mindt) s->dt = f_div((float)s->cfg.mindt, ut);
        if (s->cfg.maxdt != 0 && f_mul(s->dt, ut) > (float)s->cfg.maxdt) s->dt = f_div((float)s->cfg.maxdt, ut);
      }
    } else {
      good = 1;
    }
  }
  L->normalize(m, s->n);
  return MMX_OK;
}

static int step(mmxd_sim* s) {
  int rc = MMX_OK;
  if (s->cfg.solver == MMX_SOLVER_HEUN) heun_step(s);
  else rc = rk_step(s);
  s->steps++;
  if (s->time != s->time || isinf(s->time)) { g_err = "time is NaN"; return MMX_ERR_NAN; }
  return rc;
}

extern "C" int mmxd_steps(mmxd_sim* s, int n) {
  for (int i = 0; i < n; i++) {
    int rc = step(s);
    if (rc) return rc;
  }
  return MMX_OK;
}

extern "C" int mmxd_run(mmxd_sim* s, double seconds) {
  double stop = s->time + seconds / (double)s->unitT;
  s->L->normalize(s->m, s->n);
  while (s->time < stop) {
    int rc = step(s);
    if (rc) return rc;
  }
  return MMX_OK;
}

extern "C" int mmxd_get_m(mmxd_sim* s, float* out) {
  s->L->memcpy_dir(s->m, out, s->n3, 3);
  return MMX_OK;
}
extern "C" int mmxd_set_m(mmxd_sim* s, const float* in) {
  s->L->memcpy_dir((float*)in, s->m, s->n3, 1);
  s->fsalInit = 0;
  return MMX_OK;
}
extern "C" int mmxd_heff(mmxd_sim* s, const float* m, float* h) {
  float* dm = alloc3(s);
  float* dh = alloc3(s);
  s->L->memcpy_dir((float*)m, dm, s->n3, 1);
  calc_heff(s, dm, dh);
  s->L->memcpy_dir(dh, h, s->n3, 3);
  s->L->free_array(dm);
  s->L->free_array(dh);
  s->owned.pop_back();
  s->owned.pop_back();
  return MMX_OK;
}
extern "C" int mmxd_avg_m(mmxd_sim* s, float out[3]) {
  for (int c = 0; c < 3; c++) out[c] = f_div(s->sum.reduce(s->L, s->m + (int64_t)c * s->n), s->avgNorm);
  return MMX_OK;
}
// Total energy of m (host array), internal units: calcHeffEnergy
// (field.go:64-71,83-87) -- the demag + exchange field, phi = -1/2 m.h
// (ScaledDotProduct, field.go:17-20), the local fields and their energy
// density (AddLocalFieldsEdens, field.go:44-47), sumEdens (energy.go:49-52):
// the Reductor's sum of phi times the cell volume (energy.go:38-44).
extern "C" int mmxd_energy(mmxd_sim* s, const float* m, float* out) {
  mmxd_lib* L = s->L;
  if (!s->phi) s->phi = L->new_array(s->n);
  float* dm = alloc3(s);
  float* dh = alloc3(s);
  L->memcpy_dir((float*)m, dm, s->n3, 1);
  convolve(s, dm, dh);
  L->scale_dot(s->phi, dm, dh, -0.5f, s->n);
  float K[3] = {s->anisK[0], s->anisK[1], s->anisK[2]};
  L->local_phi(dm, dh, s->phi, s->n, s->hext, nullptr, s->anis, K, s->axes);
  float total = s->sum.reduce(L, s->phi);
  float vol = f_mul(f_mul(s->cs[0], s->cs[1]), s->cs[2]);
  *out = f_mul(total, vol);
  L->free_array(dm);
  L->free_array(dh);
  s->owned.pop_back();
  s->owned.pop_back();
  return MMX_OK;
}

// Sim.Run with a periodic table output (simrun.go:19-57; Periodic.NeedSave
// simoutput.go:83-85; Table.Save simoutput.go:226-272): before each step,
// with t = float32(time) * UnitTime, a row is written when t == 0 or
// t - sinceoutput >= period: {t, <m> in user order (the Reductor's sums /
// N), the last maximum torque, min and max of internal component X (the
// user's m_z)}, then sinceoutput = t.  *nrows = rows written (<= max_rows).
extern "C" int mmxd_run_table(mmxd_sim* s, double seconds, float period, float* rows, int max_rows, int* nrows) {
  mmxd_lib* L = s->L;
  double stop = s->time + seconds / (double)s->unitT;
  L->normalize(s->m, s->n);
  int k = 0;
  while (s->time < stop) {
    float t = f_mul((float)s->time, s->unitT);
    volatile float d = t - s->since;
    if ((t == 0.f || d >= period) && k < max_rows) {
      float* r = rows + 7 * k;
      float av[3];
      mmxd_avg_m(s, av);
      r[0] = t;
      r[1] = av[2];
      r[2] = av[1];
      r[3] = av[0];
      r[4] = s->torque;
      r[5] = s->vmin.reduce(L, s->m);
      r[6] = s->vmax.reduce(L, s->m);
      s->since = t;
      k++;
    }
    int rc = step(s);
    if (rc) { *nrows = k; return rc; }
  }
  *nrows = k;
  return MMX_OK;
}

extern "C" float mmxd_step_error(mmxd_sim* s) { return s->stepError; }
extern "C" double mmxd_time(mmxd_sim* s) { return s->time; }
extern "C" float mmxd_dt(mmxd_sim* s) { return s->dt; }
extern "C" float mmxd_torque(mmxd_sim* s) { return s->torque; }
extern "C" long long mmxd_step_count(mmxd_sim* s) { return s->steps; }
