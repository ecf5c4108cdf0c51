/*
 * Extended C ABI of the B200 LLG engine (libgpukern.so).
 *
 * These entry points have no one-to-one counterpart in the reference: they
 * fuse the primitive sequence the reference's Go driver issues per step
 * (Sim.calcHeff -> Conv.Convolve -> gpuFFT3dPlan_forward x3 ->
 * gpu_kernelmul6/4 -> gpuFFT3dPlan_inverse x3 -> gpu_add_local_fields ->
 * gpu_deltaM -> gpu_madd / gpu_linear_combination -> gpu_normalize_uniform,
 * src/go/sim/field.go:74-80, conv.go:57-100, adaptive_heun.go:34-76,
 * rk.go:279-445) into a handful of kernels that keep the state on the
 * device.  Every function returns an MMX_* status and never aborts; every
 * launch goes to the caller's stream.
 *
 * Units and axes are the reference's internal ones: lengths in exchange
 * lengths sqrt(2A/(mu0 Ms^2)), time in 1/(gamma0 Ms), fields in mu0 Ms
 * (src/go/sim/material.go:51-111); arrays are [3][X][Y][Z] float32 with Z
 * contiguous and internal X = the user's z axis (simgeom.go:19-38).
 */
#ifndef MMX_H
#define MMX_H

#include <cuda_runtime_api.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MMX_OK 0
#define MMX_ERR_ARG 1
#define MMX_ERR_CUDA 2
#define MMX_ERR_SIZE 3
#define MMX_ERR_NAN 4
#define MMX_ERR_MEM 5
#define MMX_ERR_STATE 6

/* solver kinds; tableaux of src/go/sim/rk.go:78-212 and the AdaptiveHeun
 * of adaptive_heun.go:34-76 */
#define MMX_SOLVER_HEUN 0
#define MMX_SOLVER_RK12 1
#define MMX_SOLVER_RK23 2
#define MMX_SOLVER_RK4 3
#define MMX_SOLVER_RKCK 4
#define MMX_SOLVER_RKDP 5
#define MMX_SOLVER_RK2 6

typedef struct mmx_params {
  int size[3];          /* internal (X,Y,Z) cell counts */
  int periodic[3];      /* internal order, 0 = open boundary */
  float cellsize[3];    /* internal units */
  float alpha;          /* Gilbert damping */
  float hext[3];        /* applied field, internal units and order */
  int anis_type;        /* 0 none, 1 uniaxial */
  float anis_k;         /* K1 in internal units (2K/(mu0 Ms^2)) */
  float anis_axis[3];   /* unit axis, internal order */
  int solver;           /* MMX_SOLVER_* */
  float dt;             /* initial / fixed time step, internal units */
  float max_error;      /* 0 = fixed step; else the adaptive tolerance */
  float min_dm, max_dm; /* magnetisation-step bounds (rk.go:348-373); 0 = off */
  float min_dt, max_dt; /* time-step bounds in seconds; 0 = off */
  float unit_time;      /* seconds per internal time unit */
  int exch_type;        /* 6: six-neighbour exchange folded into the kernel; 0: none */
  int faithful;         /* 1: keep the reference's FSAL-after-reject reuse */
  int accuracy;         /* face-integral points per side (reference: 8) */
  int precision;        /* 0: FP32 transforms; 1: split-BF16 tensor-core DFT
                           GEMMs for the Y convolution (2D films, Ny = 512),
                           and the adaptive solvers' error norm in float64 */
  float thermal_k;      /* thermal field (temperature.go:21-36): each RK step adds
                           sigma N(0,1) per cell and component to the field of
                           all its stages, sigma = sqrt(thermal_k / dt) with
                           thermal_k = 2 alpha kB T / (gamma0 mu0 Ms V T_unit Ms^2)
                           (V the cell volume in m^3, T_unit the time unit);
                           0 = off.  RK solvers, host dt controller only */
  unsigned int thermal_seed; /* noise stream: Philox-4x32-10 keyed by the seed,
                           counted by (cell, step) */
} mmx_params;

typedef struct mmx_solver mmx_solver;

/* Last error message of this thread (never NULL). */
const char* mmx_last_error(void);

/* Builds a solver: allocates the state, computes the demag(+exchange)
 * kernel on the GPU (FaceKernel6, demag.go:26-84) and keeps its
 * spectrum resident as one octant per component.  The magnetisation starts
 * at zero; set it with mmx_solver_set_m. */
int mmx_solver_create(const mmx_params* p, mmx_solver** out);
int mmx_solver_destroy(mmx_solver* s);

/* Copies m ([3][X][Y][Z], 3*N floats) in or out; host pointers when
 * on_host != 0, else device pointers.  Synchronous on 'stream'. */
int mmx_solver_set_m(mmx_solver* s, const float* m, int on_host, cudaStream_t stream);
int mmx_solver_get_m(mmx_solver* s, float* m, int on_host, cudaStream_t stream);
/* m <- m / |m| (gpu_normalize_uniform); Sim.Run does this before stepping */
int mmx_solver_normalize(mmx_solver* s, cudaStream_t stream);

/* Advances nsteps solver steps.  Asynchronous on 'stream' for fixed-step
 * solvers; adaptive solvers read their accept flag back once per step. */
int mmx_solver_step(mmx_solver* s, int nsteps, cudaStream_t stream);

/* Effective field h = demag + exchange + Zeeman + anisotropy of the device
 * array m (field.go:74-80); m and h are device arrays of 3*N floats. */
int mmx_solver_field(mmx_solver* s, const float* m, float* h, cudaStream_t stream);

/* <m>: the average magnetisation per internal component (the table output
 * of src/go/sim/simoutput.go:236), summed in float64 on the device.  With
 * on_host != 0, out3 is a host pointer: page-locked memory is written by
 * the reducing kernel itself (one launch, no copy), other host memory by a
 * copy on 'stream'; else a device pointer.  Asynchronous: the values are
 * there once 'stream' has reached this call. */
int mmx_solver_avg_m(mmx_solver* s, float* out3, int on_host, cudaStream_t stream);

/* Total energy of the resident m in internal units (multiply by the
 * energy unit A*L, material.go:51-111, for joules): what the reference
 * computes with calcHeffEnergy + sumEdens (src/go/sim/field.go:64-71,
 * energy.go:38-52) -- phi = -1/2 m.h_demag+exch - m.Hext - 1/2 K (m.u)^2 per
 * cell (gpu_linalg.cu:125-140, gpu_local_contr3.cu:230-247,362-374), summed
 * in float64 on the device, times the cell volume.  Synchronous; uses one
 * field evaluation. */
int mmx_solver_energy(mmx_solver* s, double* energy, cudaStream_t stream);

/* Sim.Run with the periodic table output (src/go/sim/simrun.go:19-57,
 * simoutput.go:76-90,226-272): normalises m, then steps while the time is
 * below time + seconds / UnitTime.  Before each step, when
 * t = float32(time) * UnitTime (seconds) is 0 or at least 'period' past the
 * last row, one row of 7 floats is reduced on the device:
 *   {t, <m_x>, <m_y>, <m_z> (user axes), last maximum torque (0 for heun),
 *    min m_z, max m_z (the user's z = internal X component)}
 * At most max_rows rows are copied to the host array 'rows'; *nrows gets
 * their count; successive calls continue the output schedule.  Fixed-step
 * and host-controlled solvers step from the host (no read-back except the
 * adaptive controller's own); with mmx_solver_device_control the whole run
 * is one CUDA graph launch (a WHILE conditional node over {row check, one
 * RK trial, loop condition}) with no host synchronisation until it ends.
 * max_steps > 0 caps the steps (device controller: 16 x max_steps trials;
 * MMX_ERR_STATE if the cap ends the run early); 0 = no cap.  Synchronous. */
int mmx_solver_run(mmx_solver* s, double seconds, float period, float* rows, int max_rows, int* nrows,
                   long long max_steps, cudaStream_t stream);

/* Sim.Relax (src/go/sim/relax.go:14-23): from this call on the RK steps
 * compute the energy (at the FSAL stage, or the first stage of other
 * tableaux, rk.go:321-337) and reject a trial whose energy rose
 * (rk.go:297-301,425); the solver takes one step, then steps while the
 * energy does not rise, at most max_steps steps.  *steps gets the steps
 * taken and *energy the last energy (internal units, float32 as the
 * reference keeps it).  RK solvers with the host dt controller only (the
 * heun step computes no energy).  The energy stays wanted afterwards, as
 * in the reference.  Synchronous. */
int mmx_solver_relax(mmx_solver* s, long long max_steps, long long* steps, float* energy, cudaStream_t stream);

/* Output formats of the reference's omf package, for a [3][X][Y][Z] host
 * array m of internal size 'size' with internal cell size 'cellsize' in
 * metres: an OVF 1.0 ("rectangular mesh v1.0", Binary 4 big-endian) or
 * OVF 2.0 (Binary 4 little-endian) file, or text with binary = 0, in user
 * axes x, y, z = internal Z, Y, X (src/go/mumax/omf/output.go:41-260).
 * valueunit / valuemultiplier as the reference writes them (e.g. "A/m" and
 * Ms for m); stage_time / total_time go to the OVF 2.0 header. */
int mmx_write_ovf(const char* path, const float* m, const int size[3], const double cellsize[3], int ovf_version,
                  int binary, const char* valueunit, double valuemultiplier, double stage_time, double total_time);
/* ODT 1.0 data table (omf/odt.go:103-131) of rows from mmx_solver_run:
 * columns Time, Mx/Ms, My/Ms, Mz/Ms, max_dm/dt, min_Mz/Ms, max_Mz/Ms
 * (simoutput.go:161-208). */
int mmx_write_odt(const char* path, const float* rows, int nrows, const char* title);

/* Solver scalars: simulated time (internal units), current dt, the last
 * maximum torque and the last error estimate, steps taken. */
int mmx_solver_state(mmx_solver* s, double* time, float* dt, float* max_torque, float* step_error, long long* steps);
/* Sets the applied field (internal units and order) for following steps. */
int mmx_solver_set_hext(mmx_solver* s, const float hext[3]);
/* Device pointer of the resident magnetisation (3*N floats). */
float* mmx_solver_m_device(mmx_solver* s);
/* Device address of the solver's last maximum torque (one float). */
float* mmx_solver_torque_device(mmx_solver* s);

/* Capture one step in a CUDA graph and replay it (fixed-step solvers). */
int mmx_solver_use_graph(mmx_solver* s, int on);
/* Adaptive RK solvers (rk12, rk23, rkck, rkdp): with on != 0 the dt
 * controller runs on the device (rk.go:348-445 in float32, time in
 * float64) and each mmx_solver_step unit is ONE TRIAL, replayed as a CUDA
 * graph with no host synchronisation; a rejected trial leaves m unchanged
 * and the next one retries with the reduced dt.  mmx_solver_state reads the
 * device controller (time, dt, accepted steps).  Turning it off hands the
 * state back to the host controller. */
int mmx_solver_device_control(mmx_solver* s, int on);

/* Per-pass timing with CUDA events on the step's stream; mmx_solver_pass_times
 * returns the accumulated milliseconds and launch counts per pass name.
 * on = 1: each kernel of a directly launched step is bracketed by events;
 * on = 2 (fixed-step solvers): the step is replayed as a graph whose passes
 * are bracketed by event-record nodes, so the times are those of the
 * passes as the graph runs them (one host synchronisation per step). */
int mmx_solver_profile(mmx_solver* s, int on);
int mmx_solver_pass_times(mmx_solver* s, int max, char (*names)[32], double* ms, long long* launches, int* n);

/* Batched form: 'count' independent instances (sizes, materials and fields
 * may all differ) advanced together with a fixed-step Heun or RK4 solver.
 * Each field-evaluation pass is ONE launch per distinct line length over
 * every instance that has it; with use_graph a whole step is one CUDA graph.
 * Instance i is a full solver: set / read its m with mmx_solver_set_m /
 * mmx_solver_get_m on mmx_batch_instance(b, i).  Padded sizes must be 2^k
 * or 3*2^k (<= 4096). */
typedef struct mmx_batch mmx_batch;
int mmx_batch_create(const mmx_params* p, int count, mmx_batch** out);
/* A batch over solvers the caller owns (they outlive the batch); used by a
 * serving loop to regroup resident solves as they join and leave.  After a
 * step of an RK4 batch, each solver's mmx_solver_torque_device slot holds
 * the maximum |k0| (torque) of that step's first stage. */
int mmx_batch_create_from(mmx_solver* const* solvers, int count, mmx_batch** out);
int mmx_batch_destroy(mmx_batch* b);
mmx_solver* mmx_batch_instance(mmx_batch* b, int i);
int mmx_batch_size(mmx_batch* b, int* count, long long* cells, int* launches_per_step);
int mmx_batch_step(mmx_batch* b, int nsteps, cudaStream_t stream);
int mmx_batch_use_graph(mmx_batch* b, int on);
/* Changes the uniform Zeeman field of instance i in place (the batch's
 * argument tables and graph stay valid); synchronous. */
int mmx_batch_set_hext(mmx_batch* b, int i, const float hext[3]);
/* Tile shapes of the batched Y passes are chosen by measurement: the first
 * batch needing a line length times both compiled column-tile widths on its
 * own spectrum buffers and keeps the faster for the process.  This lists
 * the decisions so far: per entry rows[5] = {line length, inverse, width 0,
 * width 1, chosen} and ms[2] = the two measured launch times; *n = entries
 * (at most max are written). */
int mmx_batch_tuning(int max, int* rows, float* ms, int* n);
/* The maximum torque of every instance in the last RK4 step, gathered into
 * out (count floats; host when on_host != 0, asynchronous on 'stream'). */
int mmx_batch_torques(mmx_batch* b, float* out, int on_host, cudaStream_t stream);

/* Serving form: a request loop with continuous batching.  A request is a
 * relaxation (npoints == 1, Sim.Relax, src/go/sim/relax.go:14-23) or a field
 * sweep (npoints > 1 fields, a relaxation at each, Sim.Hysteresis,
 * simhysteresis.go:16-27) of one solve with the fixed-step RK4 solver.  A
 * relaxation stops when the maximum torque max|k0| of a step (the
 * reference's 'torque', rk.go:353-354, internal units) is below max_torque;
 * it is checked every check_every steps of that solve.  Admission is FIFO,
 * bounded by the device bytes of the resident solves (mmx_server_footprint)
 * and by max_active.  Each mmx_server_pump advances every resident solve by
 * check_every steps -- in one mmx_batch when 'batched', else one solve at a
 * time on the single-instance solver (the baseline) -- then retires the
 * solves that finished and admits queued ones into the freed room.  A
 * request's result does not depend on the other resident solves. */
#define MMX_REQ_QUEUED 0
#define MMX_REQ_ACTIVE 1
#define MMX_REQ_DONE 2
#define MMX_REQ_FAILED 3
typedef struct mmx_request {
  mmx_params params;         /* solver must be MMX_SOLVER_RK4 with max_error 0 */
  const float* m0;           /* initial m, host [3][X][Y][Z]; copied by submit */
  int npoints;               /* 1: relax under params.hext; > 1: sweep */
  const float* hext_points;  /* npoints x 3 internal fields, or NULL when npoints == 1 */
  float max_torque;          /* relaxation stop threshold (> 0) */
  long long max_steps;       /* cap per relaxation (0: none); a capped point is not 'converged' */
} mmx_request;
typedef struct mmx_server_config {
  size_t hbm_budget;         /* device bytes the resident solves may hold (0: 80% of free) */
  int max_active;            /* resident solves at most (0: no limit) */
  int check_every;           /* steps per pump: the stop-check interval */
  int batched;               /* 1: continuous batching; 0: one solve at a time */
  int keep_m;                /* keep each finished solve's final m on the host */
} mmx_server_config;
typedef struct mmx_result {
  int state;                 /* MMX_REQ_* */
  int converged;             /* every point met max_torque */
  long long steps;           /* steps taken over all points */
  int points_done;
  double t_submit, t_admit, t_done;  /* seconds on the server clock (-1: not yet) */
  size_t footprint;          /* device bytes the solve held while resident */
} mmx_result;
typedef struct mmx_server mmx_server;
int mmx_server_create(const mmx_server_config* cfg, cudaStream_t stream, mmx_server** out);
int mmx_server_destroy(mmx_server* sv);
int mmx_server_footprint(const mmx_params* p, size_t* bytes);
int mmx_server_submit(mmx_server* sv, const mmx_request* r, long long* id);
int mmx_server_pump(mmx_server* sv, int* n_active, int* n_queued);
/* avg_m: 3 floats per finished point (<m> after its relaxation);
 * point_steps: steps per finished point.  Either may be NULL. */
int mmx_server_result(mmx_server* sv, long long id, mmx_result* out, float* avg_m, long long* point_steps);
int mmx_server_result_m(mmx_server* sv, long long id, float* m_host);
int mmx_server_release(mmx_server* sv, long long id);
double mmx_server_clock(mmx_server* sv);
int mmx_server_stats(mmx_server* sv, size_t* used_bytes, long long* chunks, long long* regroups);

/* Precision form building block: batched complex DFTs of length 32 as one
 * split-BF16 tensor-core GEMM (tcgen05) per 256 vectors: each operand is
 * split into bfloat16 hi + lo and hi.hi + hi.lo + lo.hi is accumulated in
 * FP32.  in/out: device arrays of nvec x 32 complex (float2); inverse != 0
 * uses exp(+2 pi i jk / 32) (unnormalised).  Synchronous. */
int mmx_dft_tc(const float2* in, float2* out, int nvec, int inverse, cudaStream_t stream);

/* Allocation-free reduction.  No counterpart in the reference: a variant of
 * gpu_reduce (same operations, 1 add, 2 max, 3 max |x|, 4 min, 5 sum |x|)
 * for callers that cannot call cudaMalloc -- code running while a CUDA
 * graph is captured in global mode, host callbacks, or embedders that
 * budget all device memory up front.  gpu_reduce allocates its partial
 * sums on its first call; this one keeps them in an 8 KB array compiled
 * into the library (held by every GPU that loads it until exit) and
 * allocates nothing.  'input' (n floats) and 'result' (1 float) are device
 * pointers; the launch is asynchronous on 'stream'.  n is limited to
 * MMX_REDUCE_STATIC_MAX_N; larger n returns MMX_ERR_SIZE.  The first call
 * on a device (per CUDA context: again after a device reset) looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture.  While another thread captures a graph in global mode,
 * pass a non-blocking stream of your own (cudaStreamNonBlocking): a launch
 * on the legacy default stream would join the capture's implicit
 * synchronisation and fail.  Every call shares the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
#define MMX_REDUCE_STATIC_BLOCKS 1024
#define MMX_REDUCE_STATIC_MAX_N (MMX_REDUCE_STATIC_BLOCKS * 4096)
int mmx_reduce_static(int operation, const float* input, int n, float* result, cudaStream_t stream);

/* FaceKernel6 on the GPU: the 6 real-space components (XX,YY,ZZ,YZ,XZ,XY)
 * of the padded grid P, written to k6 (device, 6*P0*P1*P2 floats),
 * bit-identical to src/go/sim/demag.go:26-84 in float32.  If exch6 != 0
 * the six-neighbour exchange stencil is added (exchange.go:44-71). */
int mmx_face_kernel6(const int P[3], const int periodic[3], const float cellsize[3], int accuracy, int exch6,
                     float* k6, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
