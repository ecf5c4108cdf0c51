// Serving form: a request loop with continuous batching.
//
// Requests are relaxations (Sim.Relax, src/go/sim/relax.go:14-23) and field
// sweeps (Sim.Hysteresis, src/go/sim/simhysteresis.go:16-27: relax at each
// of npoints fields).  The stop rule of a relax is the maximum torque
// max|k0| of a step (the reference's 'torque', rk.go:353-354) falling below
// the request's threshold, checked every check_every steps of that solve.
//
// Each admitted solve is a resident mmx_solver: m, the RK stage buffers and
// its demag+exchange kernel spectrum stay in HBM from admission to
// completion.  Admission is FIFO, limited by the device bytes the resident
// solves hold (their footprint, computed before allocating) and by a slot
// count.  In batched mode every pump advances ALL resident solves by one
// chunk of check_every steps through one mmx_batch (one launch per pass and
// line length, one CUDA graph per step), so requests that arrive while
// others run join at the next chunk boundary and share the launches; when
// a single solve remains resident it steps on its own solver graph, whose
// per-step latency is lower.  In plain mode the same loop runs
// one solve at a time on the single-instance solver: the baseline the
// batching is measured against.
//
// Determinism: a solve is admitted only at a chunk boundary and its stop
// checks fall on multiples of check_every of its OWN step count, and a
// batched instance computes bit-for-bit what it computes alone, so a
// request's result does not depend on what else is resident.
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "mmx_common.cuh"
#include "solver_state.cuh"

namespace {

struct Req {
  long long id = 0;
  mmx_request r;
  std::vector<float> m0;
  std::vector<float> fields;  // npoints x 3
  size_t footprint = 0;
  mmx_solver* s = nullptr;
  int state = MMX_REQ_QUEUED;
  int slot = -1;  // index in the current batch
  int point = 0;
  long long steps = 0, point_steps = 0;
  int converged = 1;
  std::vector<float> avg;        // 3 per finished point
  std::vector<long long> psteps;  // steps per finished point
  std::vector<float> m_final;
  double t_submit = 0, t_admit = -1, t_done = -1;
};

}  // namespace

struct mmx_server {
  mmx_server_config cfg;
  cudaStream_t st = nullptr;
  std::chrono::steady_clock::time_point t0;
  long long next_id = 1;
  std::map<long long, std::unique_ptr<Req>> reqs;
  std::deque<Req*> queue;
  std::vector<Req*> active;
  size_t used = 0;
  mmx_batch* batch = nullptr;
  bool dirty = true;  // membership or a field changed: regroup the batch
  float* torques = nullptr;  // pinned host, one per resident solve
  int torques_cap = 0;
  float* avg_host = nullptr;  // pinned host, 3 per resident solve
  long long chunks = 0, rebuilds = 0;
};

// resident solves at or below which a batched server steps each solve on
// its own graph (measured per step, RK4: one solve 0.129 ms alone vs 0.141
// ms as a batch of one; two solves 0.238 ms one after the other vs 0.159 ms
// batched)
static const int SOLO_MAX = 1;

static double sv_clock(const mmx_server* sv) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - sv->t0).count();
}

// Device bytes mmx_solver_create holds for these parameters, plus the
// transient real-space kernel and spectrum it builds the octant from.
extern "C" int mmx_server_footprint(const mmx_params* p, size_t* bytes) {
  if (!p || !bytes) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  int64_t N[3], P[3];
  for (int d = 0; d < 3; d++) {
    N[d] = p->size[d];
    if (N[d] < 1) { mmx_set_error("size must be >= 1"); return MMX_ERR_SIZE; }
    P[d] = (N[d] > 1 && p->periodic[d] == 0) ? 2 * N[d] : N[d];
  }
  int64_t HZ = P[2] / 2 + 1;
  int64_t n3 = 3 * N[0] * N[1] * N[2];
  int64_t cs = N[0] * P[1] * HZ;
  int64_t ocs = (P[0] / 2 + 1) * (P[1] / 2 + 1) * HZ;
  int vecs = 2;  // m, m1
  if (p->solver == MMX_SOLVER_HEUN) vecs += 1;
  else if (p->solver == MMX_SOLVER_RK4) vecs += 5;
  else if (p->solver == MMX_SOLVER_RK23) vecs += 5;
  else vecs += 8;
  int64_t persistent = 3 * cs * 8 + n3 * 4 * vecs + 64 + 6 * ocs * 4;
  int64_t transient = 6 * P[0] * P[1] * P[2] * 4 + P[0] * P[1] * HZ * 8;
  *bytes = (size_t)(persistent + transient);
  return MMX_OK;
}

extern "C" int mmx_server_create(const mmx_server_config* cfg, cudaStream_t stream, mmx_server** out) {
  if (!cfg || !out) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (cfg->check_every < 1) { mmx_set_error("check_every must be >= 1"); return MMX_ERR_ARG; }
  *out = nullptr;
  mmx_server* sv = new mmx_server();
  sv->cfg = *cfg;
  if (sv->cfg.hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { delete sv; mmx_set_error("cudaMemGetInfo failed"); return MMX_ERR_CUDA; }
    sv->cfg.hbm_budget = fr / 10 * 8;
  }
  if (!sv->cfg.batched) sv->cfg.max_active = 1;
  sv->st = stream;
  sv->t0 = std::chrono::steady_clock::now();
  *out = sv;
  return MMX_OK;
}

static void sv_release_solver(mmx_server* sv, Req* q) {
  if (q->s) {
    mmx_solver_destroy(q->s);
    q->s = nullptr;
    sv->used -= q->footprint;
  }
}

extern "C" int mmx_server_destroy(mmx_server* sv) {
  if (!sv) return MMX_OK;
  if (sv->batch) mmx_batch_destroy(sv->batch);
  for (auto& kv : sv->reqs) sv_release_solver(sv, kv.second.get());
  if (sv->torques) cudaFreeHost(sv->torques);
  if (sv->avg_host) cudaFreeHost(sv->avg_host);
  delete sv;
  return MMX_OK;
}

extern "C" double mmx_server_clock(mmx_server* sv) { return sv ? sv_clock(sv) : 0.0; }

extern "C" int mmx_server_submit(mmx_server* sv, const mmx_request* r, long long* id) {
  if (!sv || !r || !r->m0) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (r->params.solver != MMX_SOLVER_RK4 || r->params.max_error != 0.f) {
    mmx_set_error("served solves use the fixed-step RK4 solver (it records the stop torque)");
    return MMX_ERR_ARG;
  }
  if (r->npoints < 1 || (r->npoints > 1 && !r->hext_points) || !(r->max_torque > 0.f)) {
    mmx_set_error("bad request: npoints >= 1, hext_points for sweeps, max_torque > 0");
    return MMX_ERR_ARG;
  }
  std::unique_ptr<Req> q(new Req());
  q->r = *r;
  size_t n3 = 3 * (size_t)r->params.size[0] * r->params.size[1] * r->params.size[2];
  q->m0.assign(r->m0, r->m0 + n3);
  if (r->hext_points) q->fields.assign(r->hext_points, r->hext_points + 3 * (size_t)r->npoints);
  else q->fields.assign(r->params.hext, r->params.hext + 3);
  q->r.m0 = nullptr;
  q->r.hext_points = nullptr;
  int rc = mmx_server_footprint(&r->params, &q->footprint);
  if (rc != MMX_OK) return rc;
  if (q->footprint > sv->cfg.hbm_budget) {
    mmx_set_error("request footprint exceeds the server's device budget");
    return MMX_ERR_MEM;
  }
  q->id = sv->next_id++;
  q->t_submit = sv_clock(sv);
  if (id) *id = q->id;
  sv->queue.push_back(q.get());
  sv->reqs[q->id] = std::move(q);
  return MMX_OK;
}

static void sv_fail(mmx_server* sv, Req* q) {
  sv_release_solver(sv, q);
  q->state = MMX_REQ_FAILED;
  q->t_done = sv_clock(sv);
}

// Admits queued requests (FIFO) while the slot count and the byte budget allow.
static int sv_admit(mmx_server* sv) {
  while (!sv->queue.empty()) {
    Req* q = sv->queue.front();
    if (sv->cfg.max_active > 0 && (int)sv->active.size() >= sv->cfg.max_active) break;
    if (sv->used + q->footprint > sv->cfg.hbm_budget) break;
    sv->queue.pop_front();
    mmx_params p = q->r.params;
    for (int c = 0; c < 3; c++) p.hext[c] = q->fields[c];
    int rc = mmx_solver_create(&p, &q->s);
    if (rc != MMX_OK) { q->s = nullptr; sv_fail(sv, q); continue; }
    sv->used += q->footprint;
    rc = mmx_solver_set_m(q->s, q->m0.data(), 1, sv->st);
    if (rc == MMX_OK) rc = mmx_solver_normalize(q->s, sv->st);
    if (rc == MMX_OK && !sv->cfg.batched) rc = mmx_solver_use_graph(q->s, 1);
    if (rc != MMX_OK) { sv_fail(sv, q); continue; }
    q->m0.clear();
    q->m0.shrink_to_fit();
    q->state = MMX_REQ_ACTIVE;
    q->t_admit = sv_clock(sv);
    sv->active.push_back(q);
    sv->dirty = true;
  }
  return MMX_OK;
}

static int sv_host_buffers(mmx_server* sv, int n) {
  if (n <= sv->torques_cap) return MMX_OK;
  if (sv->torques) cudaFreeHost(sv->torques);
  if (sv->avg_host) cudaFreeHost(sv->avg_host);
  sv->torques = nullptr;
  sv->avg_host = nullptr;
  int cap = n < 64 ? 64 : 2 * n;
  if (cudaMallocHost(&sv->torques, sizeof(float) * cap) != cudaSuccess ||
      cudaMallocHost(&sv->avg_host, sizeof(float) * 3 * cap) != cudaSuccess) {
    mmx_set_error("out of pinned host memory");
    return MMX_ERR_MEM;
  }
  sv->torques_cap = cap;
  return MMX_OK;
}

extern "C" int mmx_server_pump(mmx_server* sv, int* n_active, int* n_queued) {
  if (!sv) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  int rc = sv_admit(sv);
  if (rc != MMX_OK) return rc;
  const int K = sv->cfg.check_every;
  const int n = (int)sv->active.size();
  if (n > 0) {
    MMX_CHECK_RC(sv_host_buffers(sv, n));
    // with very few resident solves the batch's per-launch overhead
    // outweighs its sharing: step them on their own solvers' graphs (the
    // same kernels and arithmetic, so results do not change)
    const bool solo = !sv->cfg.batched || n <= SOLO_MAX;
    if (!solo) {
      if (sv->dirty || !sv->batch) {
        if (sv->batch) { mmx_batch_destroy(sv->batch); sv->batch = nullptr; }
        std::vector<mmx_solver*> ss;
        for (Req* q : sv->active) {
          q->slot = (int)ss.size();
          ss.push_back(q->s);
        }
        MMX_CHECK_RC(mmx_batch_create_from(ss.data(), n, &sv->batch));
        MMX_CHECK_RC(mmx_batch_use_graph(sv->batch, 1));
        sv->rebuilds++;
        sv->dirty = false;
      }
      MMX_CHECK_RC(mmx_batch_step(sv->batch, K, sv->st));
      MMX_CHECK_RC(mmx_batch_torques(sv->batch, sv->torques, 1, sv->st));
    } else {
      for (int i = 0; i < n; i++) {
        mmx_solver* s = sv->active[i]->s;
        MMX_CHECK_RC(mmx_solver_use_graph(s, 1));
        MMX_CHECK_RC(mmx_solver_step(s, K, sv->st));
        MMX_TRY(cudaMemcpyAsync(sv->torques + i, mmx_solver_torque_device(s), sizeof(float), cudaMemcpyDeviceToHost,
                                sv->st));
      }
    }
    MMX_TRY(cudaStreamSynchronize(sv->st));
    sv->chunks++;
    // stop checks; <m> of every point that finished, in one more round trip
    std::vector<Req*> finished_point;
    for (int i = 0; i < n; i++) {
      Req* q = sv->active[i];
      q->steps += K;
      q->point_steps += K;
      float tq = sv->torques[i];
      if (tq != tq) { sv_fail(sv, q); continue; }
      bool capped = q->r.max_steps > 0 && q->point_steps >= q->r.max_steps;
      if (tq < q->r.max_torque || capped) {
        if (!(tq < q->r.max_torque)) q->converged = 0;
        MMX_CHECK_RC(mmx_solver_avg_m(q->s, sv->avg_host + 3 * finished_point.size(), 1, sv->st));
        finished_point.push_back(q);
      }
    }
    if (!finished_point.empty()) MMX_TRY(cudaStreamSynchronize(sv->st));
    for (size_t j = 0; j < finished_point.size(); j++) {
      Req* q = finished_point[j];
      for (int c = 0; c < 3; c++) q->avg.push_back(sv->avg_host[3 * j + c]);
      q->psteps.push_back(q->point_steps);
      q->point_steps = 0;
      q->point++;
      if (q->point < q->r.npoints) {
        // next field of the sweep, written into the batch's tables in place
        const float* h = &q->fields[3 * (size_t)q->point];
        if (sv->cfg.batched && sv->batch && !sv->dirty) MMX_CHECK_RC(mmx_batch_set_hext(sv->batch, q->slot, h));
        else MMX_CHECK_RC(mmx_solver_set_hext(q->s, h));
      } else {
        if (sv->cfg.keep_m) {
          q->m_final.resize(3 * (size_t)q->s->n);
          MMX_CHECK_RC(mmx_solver_get_m(q->s, q->m_final.data(), 1, sv->st));
        }
        sv_release_solver(sv, q);
        q->state = MMX_REQ_DONE;
        q->t_done = sv_clock(sv);
      }
    }
    // drop finished and failed solves from the resident set
    std::vector<Req*> keep;
    for (Req* q : sv->active) {
      if (q->state == MMX_REQ_ACTIVE) keep.push_back(q);
      else sv->dirty = true;
    }
    sv->active.swap(keep);
    if (sv->active.empty() && sv->batch) { mmx_batch_destroy(sv->batch); sv->batch = nullptr; }
  }
  if (n_active) *n_active = (int)sv->active.size();
  if (n_queued) *n_queued = (int)sv->queue.size();
  return MMX_OK;
}

extern "C" int mmx_server_result(mmx_server* sv, long long id, mmx_result* out, float* avg_m, long long* point_steps) {
  if (!sv || !out) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end()) { mmx_set_error("unknown request id"); return MMX_ERR_ARG; }
  Req* q = it->second.get();
  out->state = q->state;
  out->converged = q->converged;
  out->steps = q->steps;
  out->points_done = (int)q->psteps.size();
  out->t_submit = q->t_submit;
  out->t_admit = q->t_admit;
  out->t_done = q->t_done;
  out->footprint = q->footprint;
  if (avg_m && !q->avg.empty()) memcpy(avg_m, q->avg.data(), sizeof(float) * q->avg.size());
  if (point_steps && !q->psteps.empty()) memcpy(point_steps, q->psteps.data(), sizeof(long long) * q->psteps.size());
  return MMX_OK;
}

extern "C" int mmx_server_result_m(mmx_server* sv, long long id, float* m_host) {
  if (!sv || !m_host) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end()) { mmx_set_error("unknown request id"); return MMX_ERR_ARG; }
  Req* q = it->second.get();
  if (q->state != MMX_REQ_DONE || q->m_final.empty()) { mmx_set_error("no final m kept for this request"); return MMX_ERR_STATE; }
  memcpy(m_host, q->m_final.data(), sizeof(float) * q->m_final.size());
  return MMX_OK;
}

extern "C" int mmx_server_release(mmx_server* sv, long long id) {
  if (!sv) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end()) { mmx_set_error("unknown request id"); return MMX_ERR_ARG; }
  Req* q = it->second.get();
  if (q->state == MMX_REQ_QUEUED || q->state == MMX_REQ_ACTIVE) { mmx_set_error("request still in flight"); return MMX_ERR_STATE; }
  sv->reqs.erase(it);
  return MMX_OK;
}

extern "C" int mmx_server_stats(mmx_server* sv, size_t* used_bytes, long long* chunks, long long* regroups) {
  if (!sv) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (used_bytes) *used_bytes = sv->used;
  if (chunks) *chunks = sv->chunks;
  if (regroups) *regroups = sv->rebuilds;
  return MMX_OK;
}
