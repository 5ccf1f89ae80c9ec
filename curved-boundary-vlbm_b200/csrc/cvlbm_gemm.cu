// BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in TMEM)
// for the warm-start surrogate:
//
//   C[M x N] (fp32, row-major, ldc) = A[M x K] . B[N x K]^T  (+ C if accumulate)
//
// A and B are bf16, K-major (row-major with K contiguous).  M % 128 == 0,
// N % 64 == 0, K % 64 == 0, lda/ldb % 8 == 0 (16-byte rows of 8 elements).
//
// One CTA (4 warps) computes a 128 x 64 tile of C.  For every 64-wide slice
// of K the CTA copies the A (128 x 64) and B (64 x 64) tiles into shared
// memory in the canonical no-swizzle K-major layout of the tensor core: core
// matrices of 8 rows x 16 bytes, the two 8-element halves of a 16-element K
// step LBO = 128 bytes apart and consecutive 8-row groups SBO = 256 bytes
// apart.  Thread 0 issues four 128x64x16 MMAs (kind::f16, bf16 inputs, fp32
// accumulation in 64 TMEM columns) and commits them to an mbarrier; the CTA
// waits on it (bounded) before refilling shared memory.  The epilogue reads
// the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows)
// and stores fp32 rows.
//
// Every wait is bounded: a CTA whose MMAs do not complete within about a
// second raises the error word, waits once more (bounded), frees its TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "cvlbm_common.cuh"

using namespace cv;

namespace {

constexpr int kBM = 128, kBN = 64, kBK = 64;
constexpr int kTmemCols = 64;
constexpr long long kWaitCycles = 2000000000LL;  // about one second at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: no swizzle, K-major, start address,
// leading byte offset (between the K halves) and stride byte offset (between
// 8-row groups), version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both
// K-major, N and M encoded as N/8 and M/16.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  uint32_t done = 0;
  while (true) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(128)
    k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                float* __restrict__ C, int M, int N, int K, int lda, int ldb, int ldc,
                int accumulate, int* __restrict__ error) {
  __shared__ __align__(1024) uint8_t sA[kBM * kBK * 2];  // 16 KB, 4 slabs of 128x16
  __shared__ __align__(1024) uint8_t sB[kBN * kBK * 2];  //  8 KB, 4 slabs of 64x16
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t bar_a = smem_u32(&bar);
  const uint32_t idesc = instr_desc_bf16(kBM, kBN);
  bool ok = true;
  int kb_last = 0;
  const int nk = K / kBK;
  for (int kb = 0; kb < nk; ++kb) {
    // A tile: 128 rows x 8 chunks of 8 elements (16 bytes)
    for (int c = tid; c < kBM * 8; c += 128) {
      const int m = c >> 3, kc = c & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + m) * lda + kb * kBK + kc * 8);
      const int off = (kc >> 1) * (kBM * 32) + (m >> 3) * 256 + (kc & 1) * 128 + (m & 7) * 16;
      *reinterpret_cast<uint4*>(sA + off) = v;
    }
    for (int c = tid; c < kBN * 8; c += 128) {
      const int n = c >> 3, kc = c & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + n) * ldb + kb * kBK + kc * 8);
      const int off = (kc >> 1) * (kBN * 32) + (n >> 3) * 256 + (kc & 1) * 128 + (n & 7) * 16;
      *reinterpret_cast<uint4*>(sB + off) = v;
    }
    // make the generic-proxy stores visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int s = 0; s < kBK / 16; ++s) {
        const uint64_t ad = smem_desc(smem_u32(sA + s * kBM * 32), 128, 256);
        const uint64_t bd = smem_desc(smem_u32(sB + s * kBN * 32), 128, 256);
        const uint32_t acc = (kb > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              bar_a)
          : "memory");
    }
    // shared memory is reused only after the MMAs that read it completed;
    // the outcome of the bounded wait is made block-uniform
    kb_last = kb;
    const int got = mbar_wait(bar_a, (uint32_t)(kb & 1)) ? 1 : 0;
    if (!__syncthreads_and(got)) {
      ok = false;
      break;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicExch(error, 1);
    // give outstanding MMAs one more bounded wait before the TMEM is freed
    mbar_wait(bar_a, (uint32_t)(kb_last & 1));
  } else {
    const int row = m0 + warp * 32 + (tid & 31);
#pragma unroll
    for (int c0 = 0; c0 < kBN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < M) {
        float* dst = C + (size_t)row * ldc + n0 + c0;
#pragma unroll
        for (int i = 0; i < 16; ++i) dst[i] = accumulate ? dst[i] + v[i] : v[i];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols));
}

}  // namespace

extern "C" int cvlbm_gemm_bf16(const void* A, const void* B, float* C, int32_t M, int32_t N,
                               int32_t K, int32_t lda, int32_t ldb, int32_t ldc,
                               int32_t accumulate, int32_t* error, void* stream) {
  if (!A || !B || !C || !error) return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: null pointer");
  if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % kBN || K % kBK)
    return fail(CVLBM_ERR_INVALID_ARG,
                "cvlbm_gemm_bf16: M must be a multiple of 128, N of 64 and K of 64");
  if (lda < K || ldb < K || ldc < N || lda % 8 || ldb % 8)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: bad leading dimensions");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: A and B must be 16-byte aligned");
  dim3 grid(M / kBM, N / kBN);
  k_gemm_bf16<<<grid, 128, 0, (cudaStream_t)stream>>>(
      static_cast<const __nv_bfloat16*>(A), static_cast<const __nv_bfloat16*>(B), C, M, N, K,
      lda, ldb, ldc, accumulate, error);
  cv::count_launches(1);
  return check_launch("cvlbm_gemm_bf16");
}
