// State of the fused solver (mmx_solver), shared by the single-instance
// solver (solver.cu) and the batched form (batch.cu).
#pragma once
#include <string>
#include <vector>

#include "epilogue.cuh"
#include "fft_passes.cuh"
#include "kernmul.cuh"
#include "../../include/mmx.h"

struct PassTimer {
  std::string name;
  double ms = 0;
  long long launches = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
};

// Device-side state of the adaptive RK controller (mmx_solver_device_control).
struct RkDev {
  double time;
  float dt;
  int accept;
  long long accepted, trials;
  float torque, err;
  int bad;
};

struct mmx_solver {
  mmx_params p;
  int N[3], P[3], HZ;
  int64_t n;
  int is2d;
  BoxPlan bp;
  float2* S = nullptr;
  int64_t CS = 0;
  float* kh = nullptr;
  float* kt_tc = nullptr;  // precision form: the 2D kernel kz-major
  KernOct K;
  float* m = nullptr;
  float* t0 = nullptr;
  float* m1 = nullptr;
  float* scratch = nullptr;  // device scalars: [0] err, [1] torque, [2] dt
  float* kb[RK_MAXS] = {nullptr};
  float* mnew = nullptr;
  // solver scalars (host mirror)
  double time = 0;
  float dt = 0;
  float torque = 0, step_error = 0;
  long long steps = 0;
  int fsal_init = 0;
  int spec_ready = 0;  // S holds the forward Z spectrum of m (fused Heun steps)
  float dt_uploaded = -1.f;  // dt last written to the device scalar by the graph path
  // tableau
  int stages = 0, fsal = 0, adaptive = 0;
  double errorder = 1;
  float a[RK_MAXS][RK_MAXS], b[RK_MAXS], b2[RK_MAXS], c[RK_MAXS];
  // device-side adaptive controller (mmx_solver_device_control)
  int devctl = 0;
  void* rkdev = nullptr;
  long long steps_base = 0, trials = 0;
  cudaGraphExec_t dgraph[2] = {nullptr, nullptr};  // first trial / FSAL trials
  cudaStream_t dgraph_stream[2] = {nullptr, nullptr};
  // graph
  int use_graph = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  // run loop with table output (run.cu)
  void* runbuf = nullptr;                 // RunDev on the device
  float* rows_dev = nullptr;              // device table rows
  int rows_cap = 0;
  float since = 0.f;                      // Periodic.sinceoutput (seconds, float32)
  cudaGraphExec_t rungraph = nullptr;     // devctl: WHILE-conditional run graph
  cudaStream_t rungraph_stream = nullptr;
  double* eacc = nullptr;                 // energy accumulator (one double)
  float noise_sigma = 0.f;                // thermal field of the current step (0: off)
  long long noise_step = 0;               // its step number (the noise counter)
  int want_energy = 0;                    // Sim.wantEnergy: RK steps compute the energy (Relax)
  float energy = 0.f;                     // Sim.energy: the last energy an RK step computed
  // profiling: 1 = events around each launch of directly launched steps;
  // 2 = event-record nodes inside the captured step graph (per-pass times
  // as the graph runs them)
  int profile = 0;
  std::vector<PassTimer> timers;
  int capture_events = 0;  // ScopedPass records graph event nodes
  struct GraphEvent {
    std::string name;
    cudaEvent_t a, b;  // a is the previous pass's b when chained
    bool own_a;
  };
  std::vector<GraphEvent> gevents;
  cudaGraphExec_t pgexec = nullptr;  // the step graph with event nodes
  cudaStream_t pgstream = nullptr;
};

// Host float32 arithmetic (one rounding per operation; x86-64 SSE, no
// contraction) for the scalars the Go driver computes in float32.
static inline float f32_div(float a, float b) { volatile float r = a / b; return r; }
static inline float f32_mul(float a, float b) { volatile float r = a * b; return r; }
static inline float f32_add(float a, float b) { volatile float r = a + b; return r; }

// Fills the per-cell epilogue arguments common to every stage.
EpiArgs solver_base_args(mmx_solver* s);
// Device launch grid for a 1D element-wise kernel over n items.
int solver_grid_1d(int64_t n);
// h = demag + exchange field of the device array m (no local fields).
int solver_field_conv(mmx_solver* s, const float* m, float* h, cudaStream_t st);
// One trial of the device-controlled adaptive RK step (first: no FSAL
// value yet), as plain launches on st (capturable).
cudaError_t solver_device_trial(mmx_solver* s, cudaStream_t st, bool first);
// Reads the device controller's time, dt and step counts back (syncs).
int solver_device_download(mmx_solver* s);
// Frees the run loop's buffers and graph (run.cu).
void solver_run_free(mmx_solver* s);
// One solver step (host controller), as mmx_solver_step takes it.
int solver_step_once(mmx_solver* s, cudaStream_t st);
// Cell volume as the reference's float32 product (energy.go:38-44).
float solver_cell_volume(const mmx_solver* s);
