/*
 * libgpukern C ABI of the B200 LLG engine -- drop-in for the reference's
 * libgpukern.so (MuMax 1.1, src/gpukern/gpukern.h:24-43).
 *
 * Same symbols, argument meaning, data layout and error behaviour as the
 * reference, so src/go/sim/gpu.go (cgo, #include "../../gpukern/gpukern.h")
 * links against this library unchanged:
 *  - device arrays are raw float*, vector fields component-major
 *    [3][N0][N1][N2] with N2 contiguous;
 *  - FFT buffers are (P0, P1, P2+2) floats holding the interleaved half
 *    spectrum of an in-place real-to-complex transform;
 *  - every entry point is synchronous and aborts the process with a message
 *    on a CUDA failure or an invalid argument (gpu_safe.h:36-57);
 *  - Hext, anisK, anisAxes, size, periodic, cellSize, u are HOST pointers.
 * Each declaration names the reference declaration it replaces.
 */
#ifndef GPUKERN_B200_H
#define GPUKERN_B200_H

#include <stdio.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- gpu_init.h / gpu_conf.h / gpu_properties.h / gpu_stream.h ---- */
void gpu_init(int threads, int options);                  /* gpu_init.h:27 */
void gpu_set_device(int devid);                           /* gpu_init.h:34 */
int gpu_maxthreads(void);                                 /* gpu_conf.h:27 */
void gpu_setmaxthreads(int max);                          /* gpu_conf.h:30 */
void check3dconf(dim3 gridsize, dim3 blocksize);          /* gpu_conf.h:53 */
void check1dconf(int gridsize, int blocksize);            /* gpu_conf.h:62 */
void make1dconf(int N, dim3* gridSize, dim3* blockSize);  /* gpu_conf.h:89 */
void* gpu_getproperties(void);                            /* gpu_properties.h:69 */
void gpu_print_properties(FILE* out);                     /* gpu_properties.h:73 */
void gpu_print_properties_stdout(void);                   /* gpu_properties.h:79 */
cudaStream_t gpu_getstream(void);                         /* gpu_stream.h:30 */
void gpu_init_stream(void);                               /* gpu_stream.h:33 */

/* ---- gpu_mem.h ---- */
#define DIR_TO 1
#define DIR_ON 2
#define DIR_FROM 3
float* new_gpu_array(int size);                           /* gpu_mem.h:30 */
void free_gpu_array(float* ptr);                          /* gpu_mem.h:34 */
unsigned long long int gpu_usedmem(void);                 /* gpu_mem.h:37 */
int gpu_stride_float(void);                               /* gpu_mem.h:52 */
void gpu_override_stride(int nFloats);                    /* gpu_mem.h:60 */
void memcpy_gpu_dir(float* source, float* dest, int nElements, int direction); /* gpu_mem.h:89 */
void memcpy_to_gpu(float* source, float* dest, int nElements);                /* gpu_mem.h:95 */
void memcpy_from_gpu(float* source, float* dest, int nElements);              /* gpu_mem.h:104 */
void memcpy_on_gpu(float* source, float* dest, int nElements);                /* gpu_mem.h:113 */
void memcpy_on_gpu_async(float* source, float* dest, int nElements);          /* gpu_mem.h:118 */
float gpu_array_get(float* dataptr, int index);           /* gpu_mem.h:124 */
void gpu_array_set(float* dataptr, int index, float value); /* gpu_mem.h:127 */
void gpu_zero(float* data, int nElements);                /* gpu_mem.h:134 */
void gpu_zero_async(float* data, int nElements);          /* gpu_mem.h:141 */
void assertHost(float* pointer);                          /* gpu_mem.h:150 */
void assertDevice(float* pointer);                        /* gpu_mem.h:158 */
float* new_ram_array(int size);                           /* gpu_mem.cu:43 */

/* ---- gpu_linalg.h ---- */
void gpu_add(float* a, float* b, int N);                                  /* gpu_linalg.h:26 */
void gpu_madd(float* a, float cnst, float* b, int N);                     /* gpu_linalg.h:29 */
void gpu_madd2(float* a, float* b, float* c, int N);                      /* gpu_linalg.h:32 */
void gpu_add_constant(float* a, float cnst, int N);                       /* gpu_linalg.h:35 */
void gpu_linear_combination(float* a, float* b, float weightA, float weightB, int N); /* gpu_linalg.h:38 */
void gpu_linear_combination_many(float* result, float** vectors, float* weights, int NVectors,
                                 int NElem);                              /* gpu_linalg.h:44 */
void gpu_scale_dot_product(float* result, float* vector1, float* vector2, float a, int N); /* gpu_linalg.h:47 */

/* ---- gpu_normalize.h / gpu_torque.h ---- */
void gpu_normalize_uniform(float* m, int N);              /* gpu_normalize.h:26 */
void gpu_normalize_map(float* m, float* map, int N);      /* gpu_normalize.h:31 */
void gpu_deltaM(float* m, float* h, float alpha_mul, float* alpha_map, float dt_gilb, int N); /* gpu_torque.h:27 */

/* ---- gpu_local_contr3.h (anisType: 0 none, 1 uniaxial, 2 cubic) ---- */
void gpu_add_local_fields(float* m, float* h, int N, float* Hext, float* hmap, int anisType, float* anisK,
                          float* anisAxes);               /* gpu_local_contr3.h:33 */
void gpu_add_local_fields_H_and_phi(float* m, float* h, float* phi, int N, float* Hext, float* hmap, int anisType,
                                    float* anisK, float* anisAxes); /* gpu_local_contr3.h:39 */

/* ---- gpu_kernmul.h ---- */
void gpu_kernelmul6(float* fftMx, float* fftMy, float* fftMz, float* fftKxx, float* fftKyy, float* fftKzz,
                    float* fftKyz, float* fftKxz, float* fftKxy, int nRealNumbers); /* gpu_kernmul.h:37 */
void gpu_kernelmul4(float* fftMx, float* fftMy, float* fftMz, float* fftKxx, float* fftKyy, float* fftKzz,
                    float* fftKyz, int nRealNumbers);     /* gpu_kernmul.h:42 */
void gpu_kernelmul3(float* fftMy, float* fftMz, float* fftKyy, float* fftKzz, float* fftKyz,
                    int nRealNumbers);                    /* gpu_kernmul.h:48 */
void gpu_kernelmul_biot_savart3D(float* fftJx, float* fftJy, float* fftJz, float* fftKx, float* fftKy,
                                 float* fftKz, int nRealNumbers); /* gpu_kernmul.h:54 */
void gpu_kernelmul_biot_savart3DNx1(float* fftJx, float* fftJy, float* fftJz, float* fftKy, float* fftKz,
                                    int nRealNumbers);    /* gpu_kernmul.h:58 */
void gpu_kernelmul_biot_savart2D(float* fftJx, float* fftJy, float* fftJz, float* fftKy, float* fftKz,
                                 int nRealNumbers);       /* gpu_kernmul.h:62 */

/* ---- gpu_zeropad.h ---- */
void gpu_copy_pad(float* source, float* dest, int S0, int S1, int S2, int D0, int D1, int D2);   /* gpu_zeropad.h:25 */
void gpu_copy_unpad(float* source, float* dest, int S0, int S1, int S2, int D0, int D1, int D2); /* gpu_zeropad.h:31 */
void gpu_copy_pad2D(float* source, float* dest, int S1, int S2, int D1, int D2);                 /* gpu_zeropad.h:36 */
void gpu_copy_unpad2D(float* source, float* dest, int S1, int S2, int D1, int D2);     /* gpu_zeropad.cu:76 */
void gpu_copy_pad2D_async(float* source, float* dest, int S1, int S2, int D1, int D2); /* gpu_zeropad.cu:41 */
void gpu_copy_unpad2D_async(float* source, float* dest, int S1, int S2, int D1, int D2); /* gpu_zeropad.cu:64 */

/* ---- gpu_fft0.h: padded real-to-complex 3D transform ---- */
typedef struct gpuFFT3dPlan {
  int* size;          /* logical size of the real, unpadded data */
  int* paddedSize;    /* size after zero padding */
  int paddedN;        /* P0*P1*P2 */
  int paddedComplexN; /* P0*P1*(P2+2) */
  void* engine;       /* B200 transform plan (opaque) */
} gpuFFT3dPlan;       /* gpu_fft0.h:30-42 */
gpuFFT3dPlan* new_gpuFFT3dPlan_padded(int* size, int* paddedSize); /* gpu_fft0.h:51 */
gpuFFT3dPlan* new_gpuFFT3dPlan(int* size);                        /* gpu_fft0.cu:92-94 */
void delete_gpuFFT3dPlan(gpuFFT3dPlan* plan);                     /* gpu_fft0.h:56 */
void gpuFFT3dPlan_forward(gpuFFT3dPlan* plan, float* input, float* output); /* gpu_fft0.h:64 */
void gpuFFT3dPlan_inverse(gpuFFT3dPlan* plan, float* input, float* output); /* gpu_fft0.h:75 */
int gpuFFT3dPlan_normalization(gpuFFT3dPlan* plan);               /* gpu_fft0.cu:112-114 */

/* ---- gpu_reduction.h ---- */
#define REDUCE_ADD 1
#define REDUCE_MAX 2
#define REDUCE_MAXABS 3
#define REDUCE_MIN 4
#define REDUCE_SUMABS 5
float gpu_reduce(int operation, float* input, float* devbuffer, float* hostbuffer, int blocks, int threadsPerBlock,
                 int N);                                  /* gpu_reduction.h:31 */
void gpu_partial_sums(float* input, float* output, int blocks, int threadsPerBlock, int N); /* gpu_reduction.h:43 */
void gpu_partial_sumabs(float* input, float* output, int blocks, int threads, int N); /* gpu_reduction.cu:400 */
void gpu_partial_max(float* input, float* output, int blocks, int threads, int N);    /* gpu_reduction.cu:444 */
void gpu_partial_min(float* input, float* output, int blocks, int threads, int N);    /* gpu_reduction.cu:488 */
void gpu_partial_maxabs(float* input, float* output, int blocks, int threads, int N); /* gpu_reduction.cu:532 */
int isPow2(unsigned int x);                               /* gpu_reduction.cu:52 */

/* ---- gpu_exch.h (type: 6 or 12 neighbours) ---- */
void gpu_add_exch(float* m, float* h, int* size, int* periodic, int* exchInConv, float* cellSize, int type); /* gpu_exch.h:23 */
void gpu_add_6NGBR_exchange_3D_geometry(float* m, float* h, int* size, int* periodic, float* cellSize);  /* gpu_exch.h:34 */
void gpu_add_6NGBR_exchange_2D_geometry(float* m, float* h, int* size, int* periodic, float* cellSize);  /* gpu_exch.h:44 */
void gpu_add_12NGBR_exchange_3D_geometry(float* m, float* h, int* size, int* periodic, float* cellSize); /* gpu_exch.h:53 */
void gpu_add_12NGBR_exchange_2D_geometry(float* m, float* h, int* size, int* periodic, float* cellSize); /* gpu_exch.h:63 */

/* ---- gpu_anis.h / gpu_anal.h / gpu_spintorque.h / gpu_temperature.h ---- */
void gpu_add_lin_anisotropy(float* hx, float* hy, float* hz, float* mx, float* my, float* mz, float* kxx, float* kyy,
                            float* kzz, float* kyz, float* kxz, float* kxy, int N); /* gpu_anis.h:27 */
void gpu_anal_fw_step(float dt, float alpha, int Ntot, float* m_in, float* m_out, float* h); /* gpu_anal.h:34 */
void gpu_anal_pc_mean_h(float* h1, float* h2, int Ntot);  /* gpu_anal.h:46 */
void gpu_spintorque_deltaM(float* m, float* h, float alpha, float beta, float epsillon, float* u, float* jmap,
                           float dt_gilb, int N0, int N1, int N2); /* gpu_spintorque.h:23 */
void gpu_directionial_diff(float ux, float uy, float uz, float* in, float* out, int N0, int N1, int N2); /* gpu_spintorque.cu:254 */
void gpu_gaussian_noise(float* devData, float mean, float stddev, int n); /* gpu_temperature.h:25 */

/* ---- gpu_transpose.h ---- */
void gpu_transpose_complex_YZ(float* input, float* output, int N1, int N2, int N0); /* gpu_transpose.h:30 */
void gpu_transpose_complex_XZ(float* input, float* output, int N0, int N1, int N2); /* gpu_transpose.h:33 */

#ifdef __cplusplus
}
#endif
#endif
