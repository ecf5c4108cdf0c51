// Split-BF16 DFT-matrix GEMMs on the 5th-generation tensor cores (tcgen05).
//
// A length-32 (or any multiple-of-8 length) complex DFT applied to many
// vectors is the real GEMM D[64 x N] = W[64 x K] . X[K x N], with complex
// numbers interleaved (row 2j = real part, row 2j+1 = imaginary part of
// output j; likewise for the K inputs), so W holds the 2x2 blocks
// [[c, -s], [s, c]] of the DFT matrix.  Both operands are split into a
// bfloat16 "hi" part and the bfloat16 rounding of the remainder, "lo", and
// D = Whi.Xhi + Whi.Xlo + Wlo.Xhi is accumulated in FP32 in tensor memory
// (the Wlo.Xlo term, ~2^-16 relative, is dropped): a compensated product
// with about 16 significant bits per operand.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8 x 8 "core matrices" of 16-byte rows stored contiguously (128 bytes),
// the K-direction neighbour of a core matrix 128 bytes further and the next
// group of 8 rows K/8*128 bytes further.  Matrix descriptor fields (start
// address, leading/stride byte offsets >> 4, version 1, no swizzle) and the
// instruction descriptor (BF16 x BF16 -> F32, K-major A and B, N >> 3,
// M >> 4) follow the PTX ISA's tcgen05 descriptor formats.  For M = 64 the
// accumulator row m lives in TMEM lane (m % 16) + 32 (m / 16): warp w of
// the CTA reads rows 16w..16w+15 in its lanes 0..15.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace dtc {

// byte offset of element (row r, k) in a K-major canonical tile with K columns
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
  return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (no swizzle, K-major)
__host__ __device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  // base offset 0, leading-byte-offset mode 0, layout type 0 (no swizzle)
  return d;
}

// instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// whole warp: allocate ncols TMEM columns, address written to *slot (smem)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes visible to the tensor core's reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bounded wait for the phase with the given parity; false if it never came
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_iter) {
  uint32_t a = smem_u32(bar);
  for (int i = 0; i < max_iter; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// one thread: D(tmem) (+)= A(smem) . B(smem)
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
// one thread: arrive on bar when every MMA issued so far has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// whole warp: 8 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
// whole warp: 32 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + lo, both bfloat16 (lo the rounding of the remainder)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// The GEMM D[64 x N] (+)= A[64 x K] . B[K x N] with split operands, issued
// by the calling thread: for each 16-wide K slice, hi.hi, hi.lo, lo.hi.
// a_hi/a_lo: 64 x K tiles, b_hi/b_lo: N x K tiles (canonical K-major).
template <int K, int N>
__device__ __forceinline__ void gemm_split(uint32_t tmem_d, const void* a_hi, const void* a_lo, const void* b_hi,
                                           const void* b_lo) {
  constexpr uint32_t idesc = idesc_bf16(64, N);
  constexpr uint32_t LBO = 128, SBO_A = (K / 8) * 128, SBO_B = (K / 8) * 128;
  const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
  for (int kk = 0; kk < K; kk += 16) {
    const uint32_t off = (kk / 8) * 128;
    mma_bf16(tmem_d, smem_desc(ah + off, LBO, SBO_A), smem_desc(bh + off, LBO, SBO_B), idesc, kk > 0 ? 1u : 0u);
    mma_bf16(tmem_d, smem_desc(ah + off, LBO, SBO_A), smem_desc(bl + off, LBO, SBO_B), idesc, 1u);
    mma_bf16(tmem_d, smem_desc(al + off, LBO, SBO_A), smem_desc(bh + off, LBO, SBO_B), idesc, 1u);
  }
}

}  // namespace dtc
