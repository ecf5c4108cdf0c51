// Common definitions for the B200 LLG engine (libgpukern drop-in + mmx_*).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

// Error handling of the drop-in ABI follows the reference's convention:
// print and abort on any CUDA failure (src/gpukern/gpu_safe.h:36-57).
#define MMX_ABORT_ON(cond, ...)                                 \
  do {                                                          \
    if (cond) {                                                 \
      fprintf(stderr, "libgpukern(b200): " __VA_ARGS__);        \
      fprintf(stderr, "\n");                                    \
      abort();                                                  \
    }                                                           \
  } while (0)

#define GK_CHECK(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    MMX_ABORT_ON(e_ != cudaSuccess, "CUDA error %s at %s:%d", cudaGetErrorString(e_),  \
                 __FILE__, __LINE__);                                                   \
  } while (0)

// The ABI is synchronous: every entry point waits for its work
// (gpu_safe.h:41 gpu_sync after each launch).
// The reference synchronises the device after every primitive (gpu_sync,
// gpu_safe.h:40-44).  Here a drop-in primitive returns once its work is
// queued on the legacy default stream, which orders it before every later
// primitive and every cudaMemcpy of the caller; a failure surfaces, and
// aborts, at the next synchronising call (a host copy, a reduction, a free).
// MMX_GPUKERN_SYNC=1 in the environment restores a device synchronisation
// after every primitive.
bool gk_sync_each_call();
#define GK_SYNC()                                                    \
  do {                                                               \
    if (gk_sync_each_call()) GK_CHECK(cudaDeviceSynchronize());      \
  } while (0)
#define GK_LAUNCHED() GK_CHECK(cudaGetLastError())

// Status codes of the extended (mmx_*) ABI; it never aborts.
enum {
  MMX_OK = 0,
  MMX_ERR_ARG = 1,
  MMX_ERR_CUDA = 2,
  MMX_ERR_SIZE = 3,
  MMX_ERR_NAN = 4,
  MMX_ERR_MEM = 5,
  MMX_ERR_STATE = 6,
};

#define MMX_TRY(call)                          \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) {                   \
      mmx_set_error(cudaGetErrorString(e_));   \
      return MMX_ERR_CUDA;                     \
    }                                          \
  } while (0)

// Propagates a non-zero MMX_* status of an mmx_* call.
#define MMX_CHECK_RC(call)       \
  do {                           \
    int rc_ = (call);            \
    if (rc_ != 0) return rc_;    \
  } while (0)

void mmx_set_error(const char* msg);

static inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (cached per process).
int mmx_sm_count();
