// Output step and energy of the fused solver (extended mmx_* ABI):
//
//  * mmx_solver_energy -- the total energy of the resident m, the quantity
//    the reference computes with calcHeffEnergy + sumEdens
//    (src/go/sim/field.go:64-71,83-87, energy.go:38-52): phi = -1/2 m.h_conv
//    (ScaledDotProduct, gpu_linalg.cu:125-140) minus the Zeeman and
//    uniaxial terms (gpu_local_contr3.cu:230-247,362-374), summed over the
//    cells in float64 on the device and multiplied by the cell volume;
//  * mmx_solver_run -- Sim.Run (simrun.go:19-57) with the periodic table
//    output of simoutput.go:76-90,226-272: before each step, when
//    t = float32(time) * UnitTime is 0 or at least 'period' past the last
//    row, one row {t, <m> (user x,y,z), the last maximum torque, min and max
//    of the user's m_z} is reduced on the device.  With the device dt
//    controller (mmx_solver_device_control) the whole run is ONE CUDA graph
//    launch: a WHILE conditional node repeats {row check and reduction,
//    one RK trial, loop condition} until the device time reaches the stop
//    time, so no step, trial or row synchronises with the host.
#include <math.h>
#include <string.h>

#include "epilogue.cuh"
#include "fft_passes.cuh"
#include "solver_state.cuh"
#include "../../include/mmx.h"

struct RunDev {
  double stop;              // internal time to stop at
  long long iters, max_iters;
  float unit_time, period, since, t;
  int save, nrows, max_rows, pad;
  double sum[3];
  unsigned int kmin, kmax;  // ordered keys of min / max of component 0
  float* rows;
};

// float <-> unsigned key with the order of the floats (both signs)
__device__ __forceinline__ unsigned int order_key(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_key_inv(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Periodic.NeedSave at a step boundary (after an accepted trial) of the
// device-controlled solver (simrun.go:27-35, simoutput.go:83-85)
__global__ void k_run_check(RunDev* __restrict__ rd, const RkDev* __restrict__ dev) {
  float t = __fmul_rn(__double2float_rn(dev->time), rd->unit_time);
  rd->t = t;
  rd->save = dev->accept && (t == 0.f || __fsub_rn(t, rd->since) >= rd->period);
}

// the host decided to save at time t (host-driven loop)
__global__ void k_run_force(RunDev* __restrict__ rd, float t) {
  rd->t = t;
  rd->save = 1;
}

// per-component sums (float64) and min / max of component 0
__global__ void k_run_rowsum(RunDev* __restrict__ rd, const float* __restrict__ m, int64_t n) {
  if (!rd->save) return;
  double v[3] = {0.0, 0.0, 0.0};
  float lo = INFINITY, hi = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = m[i];
    v[0] += x;
    v[1] += m[n + i];
    v[2] += m[2 * n + i];
    lo = fminf(lo, x);
    hi = fmaxf(hi, x);
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int c = 0; c < 3; c++) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    for (int c = 0; c < 3; c++) atomicAdd(&rd->sum[c], v[c]);
    atomicMin(&rd->kmin, order_key(lo));
    atomicMax(&rd->kmax, order_key(hi));
  }
}

// writes the row (Table.Save, simoutput.go:226-272) and resets the sums
__global__ void k_run_rowfin(RunDev* __restrict__ rd, const float* __restrict__ torque, int64_t n) {
  if (!rd->save) return;
  if (rd->nrows < rd->max_rows) {
    float* r = rd->rows + 7 * (int64_t)rd->nrows;
    const double dn = (double)n;
    r[0] = rd->t;
    r[1] = (float)(rd->sum[2] / dn);  // user x = internal Z
    r[2] = (float)(rd->sum[1] / dn);
    r[3] = (float)(rd->sum[0] / dn);  // user z = internal X
    r[4] = torque ? *torque : 0.f;
    r[5] = order_key_inv(rd->kmin);
    r[6] = order_key_inv(rd->kmax);
    rd->nrows++;
  }
  rd->since = rd->t;
  rd->sum[0] = rd->sum[1] = rd->sum[2] = 0.0;
  rd->kmin = 0xffffffffu;
  rd->kmax = 0u;
  rd->save = 0;
}

// loop condition of the run graph: time < stop, no NaN, under the cap
__global__ void k_run_cond(RunDev* __restrict__ rd, const RkDev* __restrict__ dev, cudaGraphConditionalHandle h,
                           int count) {
  if (count) rd->iters++;
  const int go = dev->time < rd->stop && !dev->bad && rd->iters < rd->max_iters;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// energy density phi = -1/2 m.h_conv - m.Hext - 1/2 K (m.u)^2 per cell, in
// the order of gpu_scale_dot_product followed by
// gpu_add_local_fields_H_and_phi; summed in float64
__global__ void k_energy(const float* __restrict__ m, const float* __restrict__ h, int64_t n, LocalField lf,
                         double* __restrict__ acc) {
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float mx = m[i], my = m[n + i], mz = m[2 * n + i];
    float phi = FM(-0.5f, FA(FA(FM(mx, h[i]), FM(my, h[n + i])), FM(mz, h[2 * n + i])));
    float mh = FA(FA(FM(mx, lf.hext[0]), FM(my, lf.hext[1])), FM(mz, lf.hext[2]));
    if (lf.anis == 1) {
      float mu = FA(FA(FM(mx, lf.u[0]), FM(my, lf.u[1])), FM(mz, lf.u[2]));
      mh = FA(mh, FM(FM(FM(0.5f, lf.K), mu), mu));
    }
    v += (double)FS(phi, mh);
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(acc, v);
}

void solver_run_free(mmx_solver* s) {
  if (s->rungraph) cudaGraphExecDestroy(s->rungraph);
  s->rungraph = nullptr;
  cudaFree(s->runbuf);
  cudaFree(s->rows_dev);
  cudaFree(s->eacc);
  s->runbuf = nullptr;
  s->rows_dev = nullptr;
  s->eacc = nullptr;
  s->rows_cap = 0;
}


extern "C" int mmx_solver_energy(mmx_solver* s, double* energy, cudaStream_t st) {
  if (!s || !energy) { mmx_set_error("null argument"); return MMX_ERR_ARG; }
  if (!s->eacc && cudaMalloc(&s->eacc, sizeof(double)) != cudaSuccess) {
    mmx_set_error("out of device memory");
    return MMX_ERR_MEM;
  }
  // the convolution into the stage buffer m1 (free between steps)
  MMX_CHECK_RC(solver_field_conv(s, s->m, s->m1, st));
  MMX_TRY(cudaMemsetAsync(s->eacc, 0, sizeof(double), st));
  EpiArgs ea = solver_base_args(s);
  k_energy<<<solver_grid_1d(s->n), 256, 0, st>>>(s->m, s->m1, s->n, ea.lf, s->eacc);
  MMX_TRY(cudaGetLastError());
  double sum = 0;
  MMX_TRY(cudaMemcpyAsync(&sum, s->eacc, sizeof(double), cudaMemcpyDeviceToHost, st));
  MMX_TRY(cudaStreamSynchronize(st));
  *energy = sum * (double)solver_cell_volume(s);
  return MMX_OK;
}

static int run_buffers(mmx_solver* s, int max_rows) {
  if (!s->runbuf && cudaMalloc(&s->runbuf, sizeof(RunDev)) != cudaSuccess) {
    mmx_set_error("out of device memory");
    return MMX_ERR_MEM;
  }
  if (s->rows_cap < max_rows) {
    cudaFree(s->rows_dev);
    s->rows_dev = nullptr;
    s->rows_cap = 0;
    if (cudaMalloc(&s->rows_dev, sizeof(float) * 7 * (size_t)max_rows) != cudaSuccess) {
      mmx_set_error("out of device memory");
      return MMX_ERR_MEM;
    }
    s->rows_cap = max_rows;
    // the run graph holds the old row buffer's address only through
    // RunDev, so it stays valid
  }
  return MMX_OK;
}

// the row reduction launches (after k_run_check or k_run_force)
static cudaError_t row_launches(mmx_solver* s, RunDev* rd, cudaStream_t st) {
  const float* torque = s->p.solver == MMX_SOLVER_HEUN ? nullptr : s->scratch + 1;
  k_run_rowsum<<<solver_grid_1d(s->n), 256, 0, st>>>(rd, s->m, s->n);
  k_run_rowfin<<<1, 1, 0, st>>>(rd, torque, s->n);
  return cudaGetLastError();
}

// outer graph: the loop condition, then a WHILE node whose body is
// {row check, row reduction, one FSAL trial, loop condition}
static int build_run_graph(mmx_solver* s, cudaStream_t st) {
  if (s->rungraph && s->rungraph_stream == st) return MMX_OK;
  if (s->rungraph) { cudaGraphExecDestroy(s->rungraph); s->rungraph = nullptr; }
  RunDev* rd = reinterpret_cast<RunDev*>(s->runbuf);
  RkDev* dev = reinterpret_cast<RkDev*>(s->rkdev);
  cudaGraph_t g = nullptr;
  MMX_TRY(cudaGraphCreate(&g, 0));
  int rc = MMX_OK;
  cudaStream_t cap = nullptr;
  do {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0, 0) != cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    int zero = 0;
    void* args[4] = {&rd, &dev, &h, &zero};
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.func = (void*)k_run_cond;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    cudaGraphNode_t n0, nc;
    if (cudaGraphAddKernelNode(&n0, g, nullptr, 0, &kp) != cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    // the parameter union has no default constructor: zeroed storage
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams* cp = reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp->type = cudaGraphNodeTypeConditional;
    cp->conditional.handle = h;
    cp->conditional.type = cudaGraphCondTypeWhile;
    cp->conditional.size = 1;
    if (cudaGraphAddNode(&nc, g, &n0, 1, cp) != cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    cudaGraph_t body = cp->conditional.phGraph_out[0];
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    if (cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    k_run_check<<<1, 1, 0, cap>>>(rd, dev);
    cudaError_t e = row_launches(s, rd, cap);
    if (e == cudaSuccess) e = solver_device_trial(s, cap, false);
    if (e == cudaSuccess) {
      k_run_cond<<<1, 1, 0, cap>>>(rd, dev, h, 1);
      e = cudaGetLastError();
    }
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &out);
    if (e != cudaSuccess || e2 != cudaSuccess) { rc = MMX_ERR_CUDA; break; }
    if (cudaGraphInstantiate(&s->rungraph, g, 0) != cudaSuccess) { rc = MMX_ERR_CUDA; s->rungraph = nullptr; break; }
    s->rungraph_stream = st;
  } while (0);
  if (cap) cudaStreamDestroy(cap);
  cudaGraphDestroy(g);
  if (rc != MMX_OK) {
    cudaGetLastError();
    mmx_set_error("run graph (WHILE conditional node) could not be built");
  }
  return rc;
}

extern "C" int mmx_solver_run(mmx_solver* s, double seconds, float period, float* rows, int max_rows, int* nrows,
                              long long max_steps, cudaStream_t st) {
  if (!s || !nrows || max_rows < 0 || (max_rows > 0 && !rows) || !(seconds >= 0.0) || !(period >= 0.f)) {
    mmx_set_error("bad argument");
    return MMX_ERR_ARG;
  }
  *nrows = 0;
  MMX_CHECK_RC(run_buffers(s, max_rows > 0 ? max_rows : 1));
  RunDev* rd = reinterpret_cast<RunDev*>(s->runbuf);
  if (s->devctl) MMX_CHECK_RC(solver_device_download(s));
  // Sim.Run: stop = time + seconds / UnitTime, then Normalize(m)
  const double stop = s->time + seconds / (double)s->p.unit_time;
  MMX_CHECK_RC(mmx_solver_normalize(s, st));
  RunDev h;
  memset(&h, 0, sizeof(h));
  h.stop = stop;
  h.max_iters = max_steps > 0 ? 16 * max_steps : (1ll << 40);
  h.unit_time = s->p.unit_time;
  h.period = period;
  h.since = s->since;
  h.max_rows = max_rows;
  h.kmin = 0xffffffffu;
  h.kmax = 0u;
  h.rows = s->rows_dev;
  MMX_TRY(cudaStreamSynchronize(st));
  MMX_TRY(cudaMemcpy(rd, &h, sizeof(h), cudaMemcpyHostToDevice));
  long long steps = 0;
  if (!s->devctl) {
    // host-driven: the host knows the time of every step
    while (s->time < stop && (max_steps <= 0 || steps < max_steps)) {
      float t = f32_mul((float)s->time, s->p.unit_time);
      volatile float d = t - s->since;
      if (t == 0.f || d >= period) {
        k_run_force<<<1, 1, 0, st>>>(rd, t);
        MMX_TRY(row_launches(s, rd, st));
        s->since = t;
      }
      MMX_CHECK_RC(mmx_solver_step(s, 1, st));
      steps++;
    }
  } else if (s->time < stop) {
    if (s->fsal && !s->fsal_init) {
      // the first trial evaluates stage 0 itself: run it outside the loop
      k_run_check<<<1, 1, 0, st>>>(rd, reinterpret_cast<const RkDev*>(s->rkdev));
      MMX_TRY(row_launches(s, rd, st));
      MMX_CHECK_RC(mmx_solver_step(s, 1, st));
    }
    MMX_CHECK_RC(build_run_graph(s, st));
    MMX_TRY(cudaGraphLaunch(s->rungraph, st));
  }
  MMX_TRY(cudaStreamSynchronize(st));
  MMX_TRY(cudaMemcpy(&h, rd, sizeof(h), cudaMemcpyDeviceToHost));
  if (s->devctl) {
    MMX_CHECK_RC(solver_device_download(s));
    s->since = h.since;
  }
  *nrows = h.nrows;
  if (h.nrows > 0) MMX_TRY(cudaMemcpy(rows, s->rows_dev, sizeof(float) * 7 * (size_t)h.nrows, cudaMemcpyDeviceToHost));
  if (s->devctl && h.iters >= h.max_iters && s->time < stop) {
    mmx_set_error("run: trial cap reached before the stop time");
    return MMX_ERR_STATE;
  }
  return MMX_OK;
}

// Sim.Relax (relax.go:14-23): the energy is wanted from now on (and stays
// wanted, as in the reference), one step, then steps while the energy the
// RK steps compute does not rise; the steps themselves reject a trial whose
// energy rose (rk.go:297-301,425).  The energies are compared in float32.
extern "C" int mmx_solver_relax(mmx_solver* s, long long max_steps, long long* steps, float* energy,
                                cudaStream_t st) {
  if (!s || max_steps < 1) { mmx_set_error("bad argument"); return MMX_ERR_ARG; }
  if (s->p.solver == MMX_SOLVER_HEUN) {
    mmx_set_error("relax: the heun step computes no energy; use an RK solver");
    return MMX_ERR_ARG;
  }
  if (s->devctl) {
    mmx_set_error("relax: turn the device dt controller off first");
    return MMX_ERR_STATE;
  }
  if (!s->eacc && cudaMalloc(&s->eacc, sizeof(double)) != cudaSuccess) {
    mmx_set_error("out of device memory");
    return MMX_ERR_MEM;
  }
  s->want_energy = 1;
  long long k = 0;
  MMX_CHECK_RC(solver_step_once(s, st));
  s->steps++;
  k++;
  float prevE = f32_add(s->energy, 1.f);
  while (s->energy <= prevE && k < max_steps) {
    prevE = s->energy;
    MMX_CHECK_RC(solver_step_once(s, st));
    s->steps++;
    k++;
  }
  MMX_TRY(cudaStreamSynchronize(st));
  if (steps) *steps = k;
  if (energy) *energy = s->energy;
  return MMX_OK;
}
