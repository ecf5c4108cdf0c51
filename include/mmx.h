/*
 * Extended C ABI of the B200 LLG engine (libgpukern.so).
 *
 * These entry points have no one-to-one counterpart in the reference: they
 * fuse the primitive sequence the reference's Go driver issues per step
 * (Sim.calcHeff -> Conv.Convolve -> gpuFFT3dPlan_forward x3 ->
 * gpu_kernelmul6/4 -> gpuFFT3dPlan_inverse x3 -> gpu_add_local_fields ->
 * gpu_deltaM -> gpu_madd / gpu_linear_combination -> gpu_normalize_uniform,
 * src/go/sim/field.go:427-433, conv.go:57-100, adaptive_heun.go:34-76,
 * rk.go:279-445) into a handful of kernels that keep the state on the
 * device.  Every function returns an MMX_* status and never aborts; every
 * launch goes to the caller's stream.
 *
 * Units and axes are the reference's internal ones: lengths in exchange
 * lengths sqrt(2A/(mu0 Ms^2)), time in 1/(gamma0 Ms), fields in mu0 Ms
 * (src/go/sim/material.go:338-366); arrays are [3][X][Y][Z] float32 with Z
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
} mmx_params;

typedef struct mmx_solver mmx_solver;

/* Last error message of this thread (never NULL). */
const char* mmx_last_error(void);

/* Builds a solver: allocates the state, computes the demag(+exchange)
 * kernel on the GPU (FaceKernel6, demag.go:127-185) and keeps its
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
 * array m (field.go:427-433); m and h are device arrays of 3*N floats. */
int mmx_solver_field(mmx_solver* s, const float* m, float* h, cudaStream_t stream);

/* <m>: the average magnetisation per internal component (the table output
 * of src/go/sim/simoutput.go:236), summed in float64 on the device.  With
 * on_host != 0, out3 is a host pointer filled by an asynchronous copy on
 * 'stream' (pinned memory makes it truly asynchronous); else a device
 * pointer. */
int mmx_solver_avg_m(mmx_solver* s, float* out3, int on_host, cudaStream_t stream);

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

/* Per-pass timing with CUDA events on the step's stream: when on, each
 * kernel of the step is bracketed by events; mmx_solver_pass_times
 * returns the accumulated milliseconds and launch counts per pass name. */
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
 * on a device looks up the array's device address (cudaGetSymbolAddress)
 * and should come before any stream capture.  Every call shares the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
#define MMX_REDUCE_STATIC_BLOCKS 1024
#define MMX_REDUCE_STATIC_MAX_N (MMX_REDUCE_STATIC_BLOCKS * 4096)
int mmx_reduce_static(int operation, const float* input, int n, float* result, cudaStream_t stream);

/* FaceKernel6 on the GPU: the 6 real-space components (XX,YY,ZZ,YZ,XZ,XY)
 * of the padded grid P, written to k6 (device, 6*P0*P1*P2 floats),
 * bit-identical to src/go/sim/demag.go:127-185 in float32.  If exch6 != 0
 * the six-neighbour exchange stencil is added (exchange.go:328-353). */
int mmx_face_kernel6(const int P[3], const int periodic[3], const float cellsize[3], int accuracy, int exch6,
                     float* k6, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
