/*
 * C++ host driver of the LLG hot path: a restatement of the reference's Go
 * simulation driver (src/go/sim: init.go, material.go, conv.go, field.go,
 * torque.go, adaptive_heun.go, rk.go, redux.go, simrun.go) that drives ANY
 * library exporting the libgpukern C ABI (include/gpukern.h) through the
 * same primitive call sequence the Go front end issues.  Loading the B200
 * engine gives the drop-in path; loading the reference's own libgpukern
 * gives the reference path on identical inputs.
 *
 * Inputs follow the reference's user interface: grid, cell size, periodic
 * flags, applied field and anisotropy axis in USER (x,y,z) order and SI
 * units (simgeom.go:25-55, simfield.go:87-98, simanis.go:32-44); the
 * magnetisation is passed in the internal [3][X][Y][Z] layout.
 */
#ifndef MMX_DRIVER_H
#define MMX_DRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mmxd_config {
  int grid[3];         /* user (x,y,z) cell counts */
  double cell[3];      /* user (x,y,z) cell size, m */
  int periodic[3];     /* user (x,y,z), 0 = open */
  double msat;         /* A/m */
  double aexch;        /* J/m */
  double alpha;
  double bext[3];      /* applied field, T, user (x,y,z) */
  int anis_type;       /* 0 none, 1 uniaxial */
  double k1;           /* J/m^3 */
  double anis_axis[3]; /* user (x,y,z), need not be normalised */
  int solver;          /* MMX_SOLVER_* (include/mmx.h) */
  double dt;           /* SI seconds; 0 = the default internal 1e-4 */
  double maxerror;     /* 0 = fixed step */
  double mindm, maxdm, mindt, maxdt;
  int faithful;        /* 1: reproduce the FSAL-after-reject reuse */
} mmxd_config;

typedef struct mmxd_lib mmxd_lib;
typedef struct mmxd_sim mmxd_sim;

/* Last error message of this thread. */
const char* mmxd_last_error(void);

/* dlopen()s a libgpukern implementation (RTLD_LOCAL); NULL on failure. */
mmxd_lib* mmxd_open(const char* path);
void mmxd_close(mmxd_lib* lib);

/* Builds a simulation (Sim.init, init.go:36-77).  k6 is the real-space
 * demag(+exchange) kernel on the padded grid, 6 components XX,YY,ZZ,YZ,XZ,XY
 * of P0*P1*P2 floats (internal order), as FaceKernel6 + Exch6NgbrKernel
 * produce it; m is the initial magnetisation, internal layout.  The
 * magnetisation is normalised as Sim.Run does before stepping. */
mmxd_sim* mmxd_new(mmxd_lib* lib, const mmxd_config* cfg, const float* m, const float* k6);
void mmxd_free(mmxd_sim* s);

/* Internal sizes: N (3), P (3). */
void mmxd_sizes(mmxd_sim* s, int N[3], int P[3]);
/* Internal cell size (3), applied field (3), anisotropy axis (3), and
 * {alpha, K1, dt, unit time, unit field, unit length}. */
void mmxd_internal(mmxd_sim* s, float cs[3], float hext[3], float axis[3], double scal[6]);

int mmxd_steps(mmxd_sim* s, int n);           /* Sim.Steps (simrun.go:88-92) */
int mmxd_run(mmxd_sim* s, double seconds);    /* Sim.Run step loop (simrun.go:19-57) */
int mmxd_get_m(mmxd_sim* s, float* m);        /* 3N floats, internal order */
int mmxd_set_m(mmxd_sim* s, const float* m);
int mmxd_heff(mmxd_sim* s, const float* m, float* h); /* calcHeff (field.go:74-80), host arrays */
int mmxd_avg_m(mmxd_sim* s, float out[3]);    /* <m> per internal component (simoutput.go:236) */
double mmxd_time(mmxd_sim* s);                /* internal units */
float mmxd_dt(mmxd_sim* s);                   /* internal units */
float mmxd_torque(mmxd_sim* s);               /* last maximum torque */
long long mmxd_step_count(mmxd_sim* s);
float mmxd_step_error(mmxd_sim* s);           /* last error estimate of an adaptive step */
/* Total energy of m (host, internal layout) in internal units:
 * calcHeffEnergy + sumEdens (field.go:64-71, energy.go:49-52). */
int mmxd_energy(mmxd_sim* s, const float* m, float* out);
/* Sim.Run for 'seconds' with a table row every 'period' seconds
 * (simrun.go:19-57, simoutput.go:83-85,226-272); 7 floats per row:
 * t (s), <m> (user x,y,z), last maximum torque, min and max of the user's
 * m_z.  *nrows = rows written, at most max_rows.  Successive calls continue
 * the output schedule. */
int mmxd_run_table(mmxd_sim* s, double seconds, float period, float* rows, int max_rows, int* nrows);

#ifdef __cplusplus
}
#endif
#endif
