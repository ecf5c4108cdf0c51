// Transforms of any padded size for the drop-in FFT plan (fft_generic.cu).
#pragma once
#include "fft_engine.cuh"

struct GenericAxis {
  int L;            // line length (the padded size of the axis)
  int bluestein;    // 1: a prime factor above 7, Bluestein convolution
  int len;          // transformed length: L, or the Bluestein length M
  LineFFT f;        // transform of length len
  float2* chirp;    // exp(-i pi n^2 / L), n < L (Bluestein)
  float2* B;        // transform of the conjugate chirp, length M (Bluestein)
};

struct GenericPlan {
  int N[3], P[3];
  GenericAxis ax[3];
  float2* work;     // the complex box (P0,P1,P2)
  float2* T;        // scratch tile of gathered lines
  int64_t tcap;     // its capacity in complex elements
};

// true when the zero-aware engine cannot plan these sizes: a padded size
// with a prime factor above 7, or an odd padded Z size
bool generic_plan_needed(const int N[3], const int P[3]);
int generic_plan_init(GenericPlan* g, const int N[3], const int P[3]);
void generic_plan_free(GenericPlan* g);
// real (N0,N1,N2) -> half spectrum in rows of P2 + 2 floats, and back
// (unnormalised); the input of the inverse is left unchanged
cudaError_t generic_forward(GenericPlan* g, const float* in, float* out, cudaStream_t st);
cudaError_t generic_inverse(GenericPlan* g, const float* in, float* out, cudaStream_t st);
