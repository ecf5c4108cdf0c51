// Batched form: many independent instances of uneven sizes advanced
// together (mmx_batch_*, include/mmx.h).
//
// Every instance is a full fused solver (its own m, stage state, spectrum
// buffer and kernel octant).  A step issues, per pass of the field
// evaluation, ONE launch per distinct line length over all instances that
// share it: the blocks of the launch are the concatenation of every such
// instance's tiles, and each block finds its instance in a device table of
// per-instance arguments by a binary search on the tile offsets.  With the
// batch configuration's sizes (Nx, Ny in {32,48,64,96,128,192,256}, Nz in
// {1,2,4}) a Runge-Kutta stage is at most ~35 launches whatever the number
// of instances, and a whole step is captured in one CUDA graph whose edges
// follow each instance's own chain of launches.
#include <map>
#include <mutex>
#include <string.h>
#include <vector>

#include "fft_fixed_kernels.cuh"
#include "solver_state.cuh"

__device__ __forceinline__ int find_seg(const int* __restrict__ starts, int nseg, int b) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(&starts[mid]) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct BCol {
  const float2* src;
  float2* dst;
  ColPass cp;
};
struct BZr2c {
  const float* src;
  float2* dst;
  ZPass z;
  ZComb cb;
  int vec2;
};
struct BFin {
  float* m;
  const float* mnew;
  int64_t n;
};

template <int L, int TK, int T, bool INV, bool HALF>
__global__ void __launch_bounds__(T) kb_col(const BCol* __restrict__ a, const int* __restrict__ starts, int nseg) {
  int s = find_seg(starts, nseg, blockIdx.x);
  int t = blockIdx.x - starts[s];
  const BCol& c = a[s];
  col_body<L, TK, T, INV, HALF>(c.src, c.dst, c.cp, t);
}
template <int L, int TK, int T, bool D2, bool HALF>
__global__ void __launch_bounds__(T) kb_conv(const ConvArgs* __restrict__ a, const int* __restrict__ starts,
                                             int nseg) {
  int s = find_seg(starts, nseg, blockIdx.x);
  conv_body<L, TK, T, D2, HALF>(a[s], blockIdx.x - starts[s]);
}
template <int M, int RT, int T, bool COMB>
__global__ void __launch_bounds__(T) kb_zr2c(const BZr2c* __restrict__ a, const int* __restrict__ starts, int nseg) {
  int s = find_seg(starts, nseg, blockIdx.x);
  const BZr2c& c = a[s];
  zr2c_body<M, RT, T, COMB>(c.src, c.dst, c.z, c.cb, c.vec2, blockIdx.x - starts[s]);
}
template <int M, int RT, int T, int MODE>
__global__ void __launch_bounds__(T) kb_zinv(const ZinvArgs* __restrict__ a, const int* __restrict__ starts,
                                             int nseg) {
  int s = find_seg(starts, nseg, blockIdx.x);
  zinv_body<M, RT, T, MODE>(a[s], blockIdx.x - starts[s]);
}
// m <- normalize(m_new) for every instance (rk.go:444)
__global__ void kb_finalize(const BFin* __restrict__ a, const int* __restrict__ starts, int nseg) {
  int s = find_seg(starts, nseg, blockIdx.x);
  const BFin& f = a[s];
  int64_t i = (int64_t)(blockIdx.x - starts[s]) * blockDim.x + threadIdx.x;
  if (i >= f.n) return;
  float x = f.mnew[i], y = f.mnew[f.n + i], z = f.mnew[2 * f.n + i];
  llg_normalize(x, y, z);
  f.m[i] = x;
  f.m[f.n + i] = y;
  f.m[2 * f.n + i] = z;
}

// One launch: a kernel family, a line length, and device tables.
struct Launch {
  int kind;       // see enum below
  int L;          // line length selecting the template instance
  int flag;       // INV / D2 / COMB / MODE
  int nseg;
  int blocks;
  void* args;     // device array of per-instance argument structs
  int* starts;    // device array of tile offsets
  int variant = 0;  // tile shape (column passes: 0 = fx_col_tk, 1 = col_tk_alt)
  int half = 0;     // column passes: every instance's data fill half the line
  std::vector<int> inst;  // instances this launch reads or writes (graph dependencies)
  size_t args_off = 0, starts_off = 0;  // offsets into the batch's table block
};
enum { L_ZR2C = 0, L_COL = 1, L_CONV = 2, L_ZINV = 3, L_FIN = 4 };

struct mmx_batch {
  std::vector<mmx_solver*> inst;
  bool owns = true;  // false: a view over solvers owned by the caller
  int solver = 0;
  std::vector<std::vector<Launch>> stage;  // launches of each field evaluation (stage)
  std::vector<Launch> finalize;
  std::vector<void*> owned;
  int use_graph = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  long long cells = 0;
  int launches_per_step = 0;
  float** torque_ptrs = nullptr;  // RK4: per-instance max |k0| slots, cleared each step
  float* gather = nullptr;        // device staging of the gathered torques
  // graph capture: streams and events of the per-instance dependency DAG
  std::vector<cudaStream_t> par;
  std::vector<cudaEvent_t> ev_join;
  // every launch's argument and tile-offset tables live in one device block,
  // staged on the host while the launches are built
  std::vector<char> blob;
  char* dblob = nullptr;
  // per instance: offsets in the block of its Zeeman field in every
  // epilogue table, so a field can change without rebuilding the batch
  std::vector<std::vector<size_t>> hext_off;
};


__global__ void kb_clear(float** p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) *p[i] = 0.f;
}

// ---------------------------------------------------------------------
// launch dispatch over the compiled line lengths
// ---------------------------------------------------------------------
template <typename K>
static void set_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The autotuner's alternative column-tile width: half the default where
// that leaves >= 8 columns (more, smaller blocks), else double (fewer,
// larger blocks).
__host__ __device__ constexpr int col_tk_alt(int L) { return fx_col_tk(L) >= 16 ? fx_col_tk(L) / 2 : 2 * fx_col_tk(L); }
__host__ __device__ constexpr int col_tk_variant(int L, int v) { return v ? col_tk_alt(L) : fx_col_tk(L); }

template <int L, int TK>
static cudaError_t run_col_tk(const Launch& l, cudaStream_t st) {
  constexpr int T = fx_threads(TK * L);
  size_t smem = sizeof(float2) * (size_t)odd_pitch(TK) * L;
#define KB_COL_(INV, HALF)                                                                        \
  set_smem(kb_col<L, TK, T, INV, HALF>, smem);                                                    \
  kb_col<L, TK, T, INV, HALF><<<l.blocks, T, smem, st>>>((const BCol*)l.args, l.starts, l.nseg);
  if (l.flag) {
    if (l.half) { KB_COL_(true, true) } else { KB_COL_(true, false) }
  } else {
    if (l.half) { KB_COL_(false, true) } else { KB_COL_(false, false) }
  }
#undef KB_COL_
  return cudaGetLastError();
}
template <int L>
static cudaError_t run_col(const Launch& l, cudaStream_t st) {
  return l.variant ? run_col_tk<L, col_tk_alt(L)>(l, st) : run_col_tk<L, fx_col_tk(L)>(l, st);
}
template <int L>
static int conv_tk() {
  return conv_tkp_narrow(L);
}
template <int L>
static cudaError_t run_conv(const Launch& l, cudaStream_t st) {
  constexpr int TKP = conv_tkp_narrow(L);
  constexpr int NBF = TKP * (L / fwd_radix(L, n_stages(L) - 1));
  constexpr int T = NBF < 64 ? 64 : (NBF > 512 ? 512 : ((NBF + 31) / 32) * 32);
  size_t smem = conv_smem_tk(L, TKP);
  // variant 1: every instance of the launch has its data in the lower half
#define KB_CONV_(D2, HALF)                                                                              \
  set_smem(kb_conv<L, TKP, T, D2, HALF>, smem);                                                         \
  kb_conv<L, TKP, T, D2, HALF><<<l.blocks, T, smem, st>>>((const ConvArgs*)l.args, l.starts, l.nseg);
  if (l.flag) {
    if (l.variant) { KB_CONV_(true, true) } else { KB_CONV_(true, false) }
  } else {
    if (l.variant) { KB_CONV_(false, true) } else { KB_CONV_(false, false) }
  }
#undef KB_CONV_
  return cudaGetLastError();
}
template <int M>
static cudaError_t run_zr2c(const Launch& l, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 1);
  constexpr int T = fx_threads(RT * M);
  size_t smem = sizeof(float2) * (size_t)RT * row_pitch(M);
  if (l.flag) {
    set_smem(kb_zr2c<M, RT, T, true>, smem);
    kb_zr2c<M, RT, T, true><<<l.blocks, T, smem, st>>>((const BZr2c*)l.args, l.starts, l.nseg);
  } else {
    set_smem(kb_zr2c<M, RT, T, false>, smem);
    kb_zr2c<M, RT, T, false><<<l.blocks, T, smem, st>>>((const BZr2c*)l.args, l.starts, l.nseg);
  }
  return cudaGetLastError();
}
template <int M, int MODE>
static cudaError_t run_zinv_mode(const Launch& l, cudaStream_t st) {
  constexpr int RT = fx_rows(M, 3);
  constexpr int T = fx_threads(3 * RT * M);
  size_t smem = sizeof(float2) * (size_t)3 * RT * row_pitch(M);
  set_smem(kb_zinv<M, RT, T, MODE>, smem);
  kb_zinv<M, RT, T, MODE><<<l.blocks, T, smem, st>>>((const ZinvArgs*)l.args, l.starts, l.nseg);
  return cudaGetLastError();
}
template <int M>
static cudaError_t run_zinv(const Launch& l, cudaStream_t st) {
  switch (l.flag) {
    case EPI_HEUN1: return run_zinv_mode<M, EPI_HEUN1>(l, st);
    case EPI_HEUN2: return run_zinv_mode<M, EPI_HEUN2>(l, st);
    case EPI_TORQUE: return run_zinv_mode<M, EPI_TORQUE>(l, st);
    default: return run_zinv_mode<M, EPI_RK>(l, st);
  }
}

static cudaError_t run_launch(const Launch& l, cudaStream_t st) {
  switch (l.kind) {
    case L_FIN:
      kb_finalize<<<l.blocks, 256, 0, st>>>((const BFin*)l.args, l.starts, l.nseg);
      return cudaGetLastError();
    case L_COL:
      switch (l.L) {
#define C_(LL) \
  case LL: return run_col<LL>(l, st);
        FX_SIZES(C_)
#undef C_
      }
      break;
    case L_CONV:
      switch (l.L) {
#define C_(LL) \
  case LL: return run_conv<LL>(l, st);
        FX_SIZES(C_)
#undef C_
      }
      break;
    case L_ZR2C:
      switch (l.L) {
#define C_(LL) \
  case LL: return run_zr2c<LL>(l, st);
        FX_SIZES(C_)
#undef C_
      }
      break;
    case L_ZINV:
      switch (l.L) {
#define C_(LL) \
  case LL: return run_zinv<LL>(l, st);
        FX_SIZES(C_)
#undef C_
      }
      break;
  }
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------
// building the launch tables
// ---------------------------------------------------------------------
// Appends a launch whose tables are staged in the batch's host block; the
// device pointers are set by batch_upload once every launch is built.
static size_t blob_put(mmx_batch* b, const void* data, size_t bytes) {
  size_t off = (b->blob.size() + 255) & ~(size_t)255;
  b->blob.resize(off + bytes);
  memcpy(b->blob.data() + off, data, bytes);
  return off;
}
template <typename A>
static int add_launch(mmx_batch* b, std::vector<Launch>& out, int kind, int L, int flag, const std::vector<A>& args,
                      const std::vector<int>& tiles) {
  if (args.empty()) return MMX_OK;
  Launch l;
  l.kind = kind;
  l.L = L;
  l.flag = flag;
  l.nseg = (int)args.size();
  std::vector<int> starts(args.size());
  int acc = 0;
  for (size_t i = 0; i < args.size(); i++) {
    starts[i] = acc;
    acc += tiles[i];
  }
  l.blocks = acc;
  l.args = nullptr;
  l.starts = nullptr;
  l.args_off = blob_put(b, args.data(), sizeof(A) * args.size());
  l.starts_off = blob_put(b, starts.data(), sizeof(int) * starts.size());
  out.push_back(l);
  return MMX_OK;
}
static int batch_upload(mmx_batch* b) {
  if (b->blob.empty()) return MMX_OK;
  if (cudaMalloc(&b->dblob, b->blob.size()) != cudaSuccess) {
    mmx_set_error("out of device memory (batch tables)");
    return MMX_ERR_MEM;
  }
  b->owned.push_back(b->dblob);
  MMX_TRY(cudaMemcpy(b->dblob, b->blob.data(), b->blob.size(), cudaMemcpyHostToDevice));
  auto patch = [&](std::vector<Launch>& ls) {
    for (Launch& l : ls) {
      l.args = b->dblob + l.args_off;
      l.starts = reinterpret_cast<int*>(b->dblob + l.starts_off);
    }
  };
  for (auto& st : b->stage) patch(st);
  patch(b->finalize);
  return MMX_OK;
}

// A launch with its own device tables, usable at once (the autotuner's
// timing runs).
template <typename A>
static int add_launch_now(mmx_batch* b, std::vector<Launch>& out, int kind, int L, int flag, const std::vector<A>& args,
                          const std::vector<int>& tiles) {
  if (args.empty()) return MMX_OK;
  Launch l;
  l.kind = kind;
  l.L = L;
  l.flag = flag;
  l.nseg = (int)args.size();
  std::vector<int> starts(args.size());
  int acc = 0;
  for (size_t i = 0; i < args.size(); i++) {
    starts[i] = acc;
    acc += tiles[i];
  }
  l.blocks = acc;
  if (cudaMalloc(&l.args, sizeof(A) * args.size()) != cudaSuccess ||
      cudaMalloc(&l.starts, sizeof(int) * starts.size()) != cudaSuccess) {
    mmx_set_error("out of device memory (batch tables)");
    return MMX_ERR_MEM;
  }
  b->owned.push_back(l.args);
  b->owned.push_back(l.starts);
  cudaMemcpy(l.args, args.data(), sizeof(A) * args.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(l.starts, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice);
  out.push_back(l);
  return MMX_OK;
}

static int col_tiles(int L, int ncols, int nplanes, int variant) {
  int tk = 1;
  switch (L) {
#define C_(LL) \
  case LL: tk = col_tk_variant(LL, variant); break;
    FX_SIZES(C_)
#undef C_
  }
  return div_up(ncols * nplanes, tk);
}
static int conv_tiles(int L, int ncols) {
  int tk = 1;
  switch (L) {
#define C_(LL) \
  case LL: tk = conv_tk<LL>(); break;
    FX_SIZES(C_)
#undef C_
  }
  return div_up(ncols, tk);
}
static int zrows_per_tile(int M, int lines_per_row) {
  switch (M) {
#define C_(LL) \
  case LL: return lines_per_row == 1 ? fx_rows(LL, 1) : fx_rows(LL, 3);
    FX_SIZES(C_)
#undef C_
  }
  return 1;
}

// ---------------------------------------------------------------------
// Autotuner of the column (Y) passes.  For each line length and direction
// the first batch that needs it times both compiled tile widths
// (col_tk_variant) on its own instances -- the Y passes read and write only
// the spectrum buffers, which hold no state between field evaluations, so
// timing them changes nothing -- and keeps the faster.  The choice is kept
// for the process (every later batch, e.g. each regrouping of a serving
// loop, reuses it).  Either width computes every line with the same
// arithmetic, so the choice never changes a result.
// ---------------------------------------------------------------------
struct ColTune {
  int L, inv, tk0, tk1, chosen;
  float ms0, ms1;
};
static std::map<std::pair<int, int>, ColTune> g_col_tune;
static std::mutex g_col_tune_mu;

static void col_args(mmx_batch* b, int L, int inv, const std::vector<int>& ids, int variant, std::vector<BCol>& a,
                     std::vector<int>& t) {
  a.clear();
  t.clear();
  for (int i : ids) {
    mmx_solver* s = b->inst[i];
    BCol c;
    c.src = s->S;
    c.dst = s->S;
    c.cp.f = s->bp.fy;
    c.cp.nplanes = 3 * s->N[0];
    c.cp.plane_stride = (int64_t)s->P[1] * s->HZ;
    c.cp.ncols = s->HZ;
    c.cp.stride_i = s->HZ;
    c.cp.n_in = inv ? s->P[1] : s->N[1];
    c.cp.n_out = inv ? s->N[1] : s->P[1];
    c.cp.inv = inv;
    int tiles = col_tiles(L, c.cp.ncols, c.cp.nplanes, variant);
    a.push_back(c);
    t.push_back(tiles);
  }
}

// every instance of a column launch has its data in (forward) or keeps
// (inverse) the lower half of the line
static int col_half(int L, int inv, const std::vector<BCol>& a) {
  for (const BCol& c : a)
    if (2 * (inv ? c.cp.n_out : c.cp.n_in) != L) return 0;
  return 1;
}

static float time_launch(const Launch& l, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
  if (run_launch(l, st) != cudaSuccess) return -1.f;  // warm-up
  cudaEventRecord(e0, st);
  for (int r = 0; r < 3; r++) run_launch(l, st);
  cudaEventRecord(e1, st);
  if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  return ms / 3.f;
}

static int add_col_launch(mmx_batch* b, std::vector<Launch>& out, int L, int inv, const std::vector<int>& ids) {
  std::vector<BCol> a;
  std::vector<int> t;
  int rc;
  std::lock_guard<std::mutex> lock(g_col_tune_mu);
  auto key = std::make_pair(L, inv);
  auto it = g_col_tune.find(key);
  int variant = 0;
  if (it != g_col_tune.end()) {
    variant = it->second.chosen;
  } else {
    ColTune ct;
    ct.L = L;
    ct.inv = inv;
    ct.tk0 = ct.tk1 = 0;
    switch (L) {
#define C_(LL) \
  case LL: ct.tk0 = col_tk_variant(LL, 0); ct.tk1 = col_tk_variant(LL, 1); break;
      FX_SIZES(C_)
#undef C_
    }
    float ms[2] = {-1.f, -1.f};
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
      for (int v = 0; v < 2; v++) {
        std::vector<Launch> tmp;
        col_args(b, L, inv, ids, v, a, t);
        if ((rc = add_launch_now(b, tmp, L_COL, L, inv, a, t)) != MMX_OK) break;
        tmp.back().variant = v;
        tmp.back().half = col_half(L, inv, a);
        ms[v] = time_launch(tmp.back(), st, e0, e1);
      }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
    ct.ms0 = ms[0];
    ct.ms1 = ms[1];
    ct.chosen = (ms[1] > 0.f && ms[0] > 0.f && ms[1] < ms[0]) ? 1 : 0;
    g_col_tune[key] = ct;
    variant = ct.chosen;
  }
  col_args(b, L, inv, ids, variant, a, t);
  if ((rc = add_launch(b, out, L_COL, L, inv, a, t)) != MMX_OK) return rc;
  out.back().variant = variant;
  out.back().half = col_half(L, inv, a);
  out.back().inst = ids;
  return MMX_OK;
}

extern "C" int mmx_batch_tuning(int max, int* rows, float* ms, int* n) {
  if (!n || (max > 0 && (!rows || !ms))) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_col_tune_mu);
  int k = 0;
  for (auto& kv : g_col_tune) {
    if (k < max) {
      const ColTune& c = kv.second;
      int* r = rows + 5 * k;
      r[0] = c.L; r[1] = c.inv; r[2] = c.tk0; r[3] = c.tk1; r[4] = c.chosen;
      ms[2 * k] = c.ms0;
      ms[2 * k + 1] = c.ms1;
    }
    k++;
  }
  *n = k;
  return MMX_OK;
}

// Builds the launches of one field evaluation: zfwd (optionally with the
// stage combination), yfwd / conv / yinv, zinv with the given epilogue.
// stage_args(i) returns the epilogue arguments, comb_for(i) the combination.
template <typename EpiF, typename CombF, typename SrcF>
static int build_eval(mmx_batch* b, std::vector<Launch>& out, int mode, bool comb, EpiF epi_for, CombF comb_for,
                      SrcF src_for) {
  int rc;
  std::map<int, std::vector<int>> byM, byP1_3d, byP0, byP1_2d;
  for (int i = 0; i < (int)b->inst.size(); i++) {
    mmx_solver* s = b->inst[i];
    byM[s->P[2] / 2].push_back(i);
    if (s->is2d) byP1_2d[s->P[1]].push_back(i);
    else {
      byP1_3d[s->P[1]].push_back(i);
      byP0[s->P[0]].push_back(i);
    }
  }
  // zfwd
  for (auto& g : byM) {
    std::vector<BZr2c> a;
    std::vector<int> t;
    for (int i : g.second) {
      mmx_solver* s = b->inst[i];
      BZr2c z;
      memset(&z, 0, sizeof(z));
      z.z = box_zpass(&s->bp, 3, s->N[0], s->n, s->CS);
      z.dst = s->S;
      z.src = src_for(i);
      if (comb) z.cb = comb_for(i);
      z.vec2 = (z.z.ld_real % 2 == 0) && (s->n % 2 == 0);
      a.push_back(z);
      t.push_back(div_up(z.z.nrows, zrows_per_tile(g.first, 1)));
    }
    if ((rc = add_launch(b, out, L_ZR2C, g.first, comb ? 1 : 0, a, t)) != MMX_OK) return rc;
    out.back().inst = g.second;
  }
  // Y forward (3D)
  for (auto& g : byP1_3d)
    if ((rc = add_col_launch(b, out, g.first, 0, g.second)) != MMX_OK) return rc;
  // X convolution (3D) and Y convolution (2D)
  for (int d2 = 0; d2 < 2; d2++) {
    auto& groups = d2 ? byP1_2d : byP0;
    for (auto& g : groups) {
      std::vector<ConvArgs> a;
      std::vector<int> t;
      for (int i : g.second) {
        mmx_solver* s = b->inst[i];
        ConvArgs c;
        c.S = s->S;
        c.K = s->K;
        c.HZ = s->HZ;
        c.CS = s->CS;
        if (d2) {
          c.n_data = s->N[1];
          c.ncols = s->HZ;
          c.stride = s->HZ;
          c.tw = s->bp.fy.tw;
          c.tws = s->bp.fy.tws;
        } else {
          c.n_data = s->N[0];
          c.ncols = s->P[1] * s->HZ;
          c.stride = (int64_t)s->P[1] * s->HZ;
          c.tw = s->bp.fx.tw;
          c.tws = s->bp.fx.tws;
        }
        a.push_back(c);
        t.push_back(conv_tiles(g.first, c.ncols));
      }
      if ((rc = add_launch(b, out, L_CONV, g.first, d2, a, t)) != MMX_OK) return rc;
      out.back().inst = g.second;
      bool half = true;
      for (const ConvArgs& c : a) half = half && 2 * c.n_data == g.first;
      out.back().variant = half ? 1 : 0;
    }
  }
  // Y inverse (3D)
  for (auto& g : byP1_3d)
    if ((rc = add_col_launch(b, out, g.first, 1, g.second)) != MMX_OK) return rc;
  // Z inverse + epilogue
  for (auto& g : byM) {
    std::vector<ZinvArgs> a;
    std::vector<int> t;
    for (int i : g.second) {
      mmx_solver* s = b->inst[i];
      ZinvArgs z;
      z.S = s->S;
      z.twz = s->bp.twz;
      z.twP = s->bp.twz;
      z.P1 = s->P[1];
      z.HZ = s->HZ;
      z.CS = s->CS;
      z.nrows = s->N[0] * s->N[1];
      z.ea = epi_for(i);
      a.push_back(z);
      t.push_back(div_up(z.nrows, zrows_per_tile(g.first, 3)));
    }
    if ((rc = add_launch(b, out, L_ZINV, g.first, mode, a, t)) != MMX_OK) return rc;
    out.back().inst = g.second;
    for (size_t k = 0; k < g.second.size(); k++)
      b->hext_off[g.second[k]].push_back(out.back().args_off + k * sizeof(ZinvArgs) + offsetof(ZinvArgs, ea) +
                                         offsetof(EpiArgs, lf) + offsetof(LocalField, hext));
  }
  return MMX_OK;
}

static void batch_free(mmx_batch* b) {
  if (!b) return;
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (cudaStream_t q : b->par) cudaStreamDestroy(q);
  for (cudaEvent_t e : b->ev_join) cudaEventDestroy(e);
  for (void* p : b->owned) cudaFree(p);
  if (b->owns)
    for (mmx_solver* s : b->inst) mmx_solver_destroy(s);
  delete b;
}

static int batch_check(mmx_solver* s, int solver) {
  if (s->p.precision) {
    mmx_set_error("batched form: FP32 transforms only (precision = 0)");
    return MMX_ERR_ARG;
  }
  if (s->p.thermal_k != 0.f) {
    mmx_set_error("batched form: no thermal field (its noise is drawn per step on the host controller)");
    return MMX_ERR_ARG;
  }
  if (s->p.solver != solver || s->p.max_error != 0.f) {
    mmx_set_error("all instances of a batch must use the same fixed-step solver (Heun or RK4)");
    return MMX_ERR_ARG;
  }
  for (int d = 0; d < 3; d++) {
    if (!fx_ok(d == 2 ? s->P[2] / 2 : s->P[d]) && !(d == 0 && s->P[0] == 1)) {
      mmx_set_error("batched form: padded sizes must be 2^k or 3*2^k (<= 4096)");
      return MMX_ERR_SIZE;
    }
  }
  return MMX_OK;
}

static int batch_build(mmx_batch* b) {
  int rc = MMX_OK;
  b->hext_off.assign(b->inst.size(), std::vector<size_t>());
  for (mmx_solver* s : b->inst) {
    s->spec_ready = 0;  // the batch's passes reuse the spectrum buffer
    // the stage kernels read dt from the instance's device scalar
    MMX_TRY(cudaMemcpy(s->scratch + 2, &s->dt, sizeof(float), cudaMemcpyHostToDevice));
    b->cells += s->n;
  }
  if (b->solver == MMX_SOLVER_HEUN) {
    b->stage.resize(2);
    auto epi1 = [&](int i) {
      mmx_solver* s = b->inst[i];
      EpiArgs ea = solver_base_args(s);
      ea.dtg = f32_div(s->dt, f32_add(1.f, f32_mul(s->p.alpha, s->p.alpha)));
      ea.m_in = s->m;
      ea.out0 = s->t0;
      ea.out1 = s->m1;
      return ea;
    };
    auto epi2 = [&](int i) {
      mmx_solver* s = b->inst[i];
      EpiArgs ea = solver_base_args(s);
      ea.dtg = f32_div(s->dt, f32_add(1.f, f32_mul(s->p.alpha, s->p.alpha)));
      ea.m_in = s->m1;
      ea.aux0 = s->t0;
      ea.aux1 = s->m;
      ea.out0 = s->m;
      return ea;
    };
    auto nocomb = [&](int) { ZComb c; memset(&c, 0, sizeof(c)); return c; };
    auto src_m = [&](int i) { return (const float*)b->inst[i]->m; };
    auto src_m1 = [&](int i) { return (const float*)b->inst[i]->m1; };  // the normalised Euler estimate
    rc = build_eval(b, b->stage[0], EPI_HEUN1, false, epi1, nocomb, src_m);
    if (rc == MMX_OK) rc = build_eval(b, b->stage[1], EPI_HEUN2, false, epi2, nocomb, src_m1);
  } else {
    b->stage.resize(4);
    for (int st = 0; st < 4 && rc == MMX_OK; st++) {
      auto epi = [&](int i) {
        mmx_solver* s = b->inst[i];
        EpiArgs ea = solver_base_args(s);
        ea.dtg = f32_div(1.f, f32_add(1.f, f32_mul(s->p.alpha, s->p.alpha)));
        ea.m_in = st == 0 ? s->m : s->m1;
        ea.dt_dev = s->scratch + 2;
        for (int j = 0; j < s->stages; j++) ea.kbuf[j] = s->kb[j];
        ea.stage = st;
        ea.out0 = s->kb[st];
        if (st == 0) ea.err = s->scratch + 1;  // max |k0|, the torque the relax loop stops on
        if (st == 3) {
          ea.aux0 = s->m;
          ea.out1 = s->mnew;
          ea.rk.nk = s->stages;
          for (int j = 0; j < s->stages; j++) ea.rk.a[j] = s->b[j];
          ea.rk.final_stage = 1;
          ea.rk.adaptive = 0;
        }
        return ea;
      };
      auto comb = [&](int i) {
        mmx_solver* s = b->inst[i];
        ZComb c;
        memset(&c, 0, sizeof(c));
        c.m0 = s->m;
        for (int j = 0; j < s->stages; j++) { c.k[j] = s->kb[j]; c.a[j] = s->a[st][j]; }
        c.nk = s->stages;
        c.dt = s->scratch + 2;
        c.out = s->m1;
        return c;
      };
      auto src_m = [&](int i) { return (const float*)b->inst[i]->m; };
      rc = build_eval(b, b->stage[st], st == 3 ? EPI_RK : EPI_TORQUE, st > 0, epi, comb, src_m);
    }
    if (rc == MMX_OK) {
      std::vector<BFin> a;
      std::vector<int> t;
      for (mmx_solver* s : b->inst) {
        BFin f;
        f.m = s->m;
        f.mnew = s->mnew;
        f.n = s->n;
        a.push_back(f);
        t.push_back(div_up(s->n, 256));
      }
      rc = add_launch(b, b->finalize, L_FIN, 0, 0, a, t);
      if (rc == MMX_OK) {
        for (int i = 0; i < (int)b->inst.size(); i++) b->finalize.back().inst.push_back(i);
        // clear the per-instance torque maxima before the step
        std::vector<float*> tq;
        for (mmx_solver* s : b->inst) tq.push_back(s->scratch + 1);
        void* d = nullptr;
        if (cudaMalloc(&d, sizeof(float*) * tq.size()) != cudaSuccess) return MMX_ERR_MEM;
        b->owned.push_back(d);
        cudaMemcpy(d, tq.data(), sizeof(float*) * tq.size(), cudaMemcpyHostToDevice);
        b->torque_ptrs = (float**)d;
      }
    }
  }
  if (rc != MMX_OK) return rc;
  if ((rc = batch_upload(b)) != MMX_OK) return rc;
  for (auto& st : b->stage) b->launches_per_step += (int)st.size();
  b->launches_per_step += (int)b->finalize.size() + (b->torque_ptrs ? 1 : 0);
  return MMX_OK;
}

extern "C" int mmx_batch_create(const mmx_params* p, int count, mmx_batch** out) {
  if (!p || count <= 0 || !out) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  *out = nullptr;
  mmx_batch* b = new mmx_batch();
  b->solver = p[0].solver;
  for (int i = 0; i < count; i++) {
    mmx_solver* s = nullptr;
    int rc = mmx_solver_create(&p[i], &s);
    if (rc == MMX_OK) {
      rc = batch_check(s, b->solver);
      if (rc != MMX_OK) mmx_solver_destroy(s);
    }
    if (rc != MMX_OK) { batch_free(b); return rc; }
    b->inst.push_back(s);
  }
  int rc = batch_build(b);
  if (rc != MMX_OK) { batch_free(b); return rc; }
  *out = b;
  return MMX_OK;
}

extern "C" int mmx_batch_create_from(mmx_solver* const* solvers, int count, mmx_batch** out) {
  if (!solvers || count <= 0 || !out) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  *out = nullptr;
  mmx_batch* b = new mmx_batch();
  b->owns = false;
  b->solver = solvers[0]->p.solver;
  for (int i = 0; i < count; i++) {
    int rc = batch_check(solvers[i], b->solver);
    if (rc != MMX_OK) { batch_free(b); return rc; }
    b->inst.push_back(solvers[i]);
  }
  int rc = batch_build(b);
  if (rc != MMX_OK) { batch_free(b); return rc; }
  *out = b;
  return MMX_OK;
}

extern "C" int mmx_batch_destroy(mmx_batch* b) {
  batch_free(b);
  return MMX_OK;
}

extern "C" int mmx_batch_size(mmx_batch* b, int* count, long long* cells, int* launches_per_step) {
  if (!b) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (count) *count = (int)b->inst.size();
  if (cells) *cells = b->cells;
  if (launches_per_step) *launches_per_step = b->launches_per_step;
  return MMX_OK;
}

extern "C" mmx_solver* mmx_batch_instance(mmx_batch* b, int i) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return nullptr;
  return b->inst[i];
}

// While a step is captured into its graph, every launch depends only on the
// latest earlier launch of each instance it touches (each instance's
// buffers are its own), not on a whole pass: small instances run ahead
// through their passes while large ones are still being transformed.
// Launches are spread round-robin over BATCH_DAG_STREAMS streams; events
// carry the per-instance dependencies.
#define BATCH_DAG_STREAMS 16
static cudaError_t batch_step_dag(mmx_batch* b, cudaStream_t st) {
  cudaError_t e;
  const int ninst = (int)b->inst.size();
  size_t nl = 4 + b->finalize.size();
  for (auto& stage : b->stage) nl += stage.size();
  while ((int)b->par.size() < BATCH_DAG_STREAMS) {
    cudaStream_t q;
    if ((e = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking)) != cudaSuccess) return e;
    b->par.push_back(q);
  }
  while (b->ev_join.size() < nl) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    b->ev_join.push_back(ev);
  }
  size_t ne = 0;
  // the origin: the torque maxima cleared on the capturing stream
  if (b->torque_ptrs) {
    kb_clear<<<(ninst + 255) / 256, 256, 0, st>>>(b->torque_ptrs, ninst);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  cudaEvent_t origin = b->ev_join[ne++];
  if ((e = cudaEventRecord(origin, st)) != cudaSuccess) return e;
  std::vector<cudaEvent_t> last(ninst, origin);
  int rr = 0;
  auto run = [&](const Launch& l) -> cudaError_t {
    cudaStream_t q = b->par[rr++ % BATCH_DAG_STREAMS];
    std::vector<cudaEvent_t> waits;
    for (int i : l.inst) {
      bool seen = false;
      for (cudaEvent_t w : waits) seen = seen || w == last[i];
      if (!seen) waits.push_back(last[i]);
    }
    cudaError_t r;
    for (cudaEvent_t w : waits)
      if ((r = cudaStreamWaitEvent(q, w, 0)) != cudaSuccess) return r;
    if ((r = run_launch(l, q)) != cudaSuccess) return r;
    cudaEvent_t done = b->ev_join[ne++];
    if ((r = cudaEventRecord(done, q)) != cudaSuccess) return r;
    for (int i : l.inst) last[i] = done;
    return cudaSuccess;
  };
  for (auto& stage : b->stage)
    for (const Launch& l : stage)
      if ((e = run(l)) != cudaSuccess) return e;
  for (const Launch& l : b->finalize)
    if ((e = run(l)) != cudaSuccess) return e;
  // join: the capturing stream waits for every instance's last launch
  std::vector<cudaEvent_t> tails;
  for (int i = 0; i < ninst; i++) {
    bool seen = false;
    for (cudaEvent_t w : tails) seen = seen || w == last[i];
    if (!seen) tails.push_back(last[i]);
  }
  for (cudaEvent_t w : tails)
    if ((e = cudaStreamWaitEvent(st, w, 0)) != cudaSuccess) return e;
  return cudaSuccess;
}

static cudaError_t batch_step_launches(mmx_batch* b, cudaStream_t st, bool parallel) {
  if (parallel) return batch_step_dag(b, st);
  if (b->torque_ptrs) {
    int n = (int)b->inst.size();
    kb_clear<<<(n + 255) / 256, 256, 0, st>>>(b->torque_ptrs, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  for (auto& stage : b->stage)
    for (const Launch& l : stage) {
      cudaError_t e = run_launch(l, st);
      if (e != cudaSuccess) return e;
    }
  for (const Launch& l : b->finalize) {
    cudaError_t e = run_launch(l, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

extern "C" int mmx_batch_step(mmx_batch* b, int nsteps, cudaStream_t st) {
  if (!b || nsteps < 0) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  for (int k = 0; k < nsteps; k++) {
    if (b->use_graph) {
      if (!b->gexec || b->gstream != st) {
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
        cudaStream_t cap = st;
        bool own = false;
        if (cap == 0) { MMX_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
        cudaGraph_t g;
        MMX_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = batch_step_launches(b, cap, true);
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        if (own) cudaStreamDestroy(cap);
        if (e != cudaSuccess || e2 != cudaSuccess) { mmx_set_error("batch graph capture failed"); return MMX_ERR_CUDA; }
        MMX_TRY(cudaGraphInstantiate(&b->gexec, g, 0));
        cudaGraphDestroy(g);
        b->gstream = st;
      }
      MMX_TRY(cudaGraphLaunch(b->gexec, st));
    } else {
      cudaError_t e = batch_step_launches(b, st, false);
      if (e != cudaSuccess) { mmx_set_error(cudaGetErrorString(e)); return MMX_ERR_CUDA; }
    }
    for (mmx_solver* s : b->inst) {
      s->time += (double)s->dt;
      s->steps++;
    }
  }
  return MMX_OK;
}

__global__ void kb_gather(float* const* __restrict__ p, int n, float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = *p[i];
}

extern "C" int mmx_batch_torques(mmx_batch* b, float* out, int on_host, cudaStream_t st) {
  if (!b || !out) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (!b->torque_ptrs) { mmx_set_error("torques are recorded by RK4 batches only"); return MMX_ERR_STATE; }
  int n = (int)b->inst.size();
  if (!b->gather) {
    if (cudaMalloc(&b->gather, sizeof(float) * n) != cudaSuccess) { mmx_set_error("out of device memory"); return MMX_ERR_MEM; }
    b->owned.push_back(b->gather);
  }
  float* dst = on_host ? b->gather : out;
  kb_gather<<<(n + 255) / 256, 256, 0, st>>>(b->torque_ptrs, n, dst);
  MMX_TRY(cudaGetLastError());
  if (on_host) MMX_TRY(cudaMemcpyAsync(out, b->gather, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  return MMX_OK;
}

extern "C" int mmx_batch_set_hext(mmx_batch* b, int i, const float hext[3]) {
  if (!b || !hext || i < 0 || i >= (int)b->inst.size()) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  MMX_CHECK_RC(mmx_solver_set_hext(b->inst[i], hext));
  for (size_t off : b->hext_off[i]) {
    memcpy(b->blob.data() + off, hext, 3 * sizeof(float));
    MMX_TRY(cudaMemcpy(b->dblob + off, hext, 3 * sizeof(float), cudaMemcpyHostToDevice));
  }
  return MMX_OK;
}

extern "C" int mmx_batch_use_graph(mmx_batch* b, int on) {
  if (!b) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  b->use_graph = on;
  if (!on && b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
  return MMX_OK;
}
