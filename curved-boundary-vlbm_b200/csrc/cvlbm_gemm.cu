// BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in TMEM)
// for the warm-start surrogate:
//
//   C[M x N] (fp32, row-major, ldc) = A[M x K] . B[N x K]^T  (+ C if accumulate)
//
// A and B are bf16, K-major (row-major with K contiguous).  M % 128 == 0,
// N % 64 == 0, K % 64 == 0, lda/ldb % 8 == 0 (16-byte rows of 8 elements).
//
// Two kernels compute the same product.  k_gemm_tma (the default, further
// down) has the operand tiles brought in by TMA tensor copies; k_gemm_bf16,
// described here, loads them with threads and is the fallback when no tensor
// map can be encoded (or CVLBM_GEMM_LOADER=threads).
//
// One CTA (4 warps) computes a 128 x BN tile of C (BN = 128 when N allows,
// else 64).  For every 64-wide slice of K the CTA stages the A (128 x 64) and
// B (BN x 64) tiles in shared memory in the canonical no-swizzle K-major
// layout of the tensor core: core matrices of 8 rows x 16 bytes, the two
// 8-element halves of a 16-element K step LBO = 128 bytes apart and
// consecutive 8-row groups SBO = 256 bytes apart.  Two stages: while thread 0
// has the four 128xBNx16 MMAs of one slice in flight (kind::f16, bf16 inputs,
// fp32 accumulation in BN TMEM columns, committed to that stage's mbarrier),
// all threads load the next slice from global memory into registers.  Long
// K with few output tiles is split over gridDim.z into fp32 partials that a
// second kernel adds in a fixed order.  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows).
//
// Every wait is bounded: a CTA whose MMAs do not complete within about a
// second raises the error word, waits once more (bounded), frees its TMEM and
// returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "cvlbm_common.cuh"

using namespace cv;

namespace {

constexpr int kBM = 128, kBN = 64, kBK = 64;
constexpr long long kWaitCycles = 2000000000LL;  // about one second at 2 GHz
constexpr int kMaxSplits = 64;                    // K splits of one product

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

// One CTA computes a 128 x BN tile of C over the K range
// [blockIdx.z * kchunk, (blockIdx.z + 1) * kchunk): two shared-memory stages,
// the global loads of slice k+1 in flight while the MMAs of slice k run.
// With gridDim.z > 1 the tile goes to partial[blockIdx.z] (reduced later in
// a fixed order), else to C.
template <int BN>
__global__ void __launch_bounds__(128)
    k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                float* __restrict__ C, float* __restrict__ partial, int M, int N, int kchunk,
                int lda, int ldb, int ldc, int accumulate, int* __restrict__ error) {
  extern __shared__ __align__(1024) uint8_t smem_g[];
  uint8_t* sA[2] = {smem_g, smem_g + kBM * kBK * 2};
  uint8_t* sB[2] = {smem_g + 2 * kBM * kBK * 2, smem_g + 2 * kBM * kBK * 2 + BN * kBK * 2};
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int kbeg = blockIdx.z * kchunk, nk = kchunk / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = instr_desc_bf16(kBM, BN);

  // 16-byte chunk c of a tile: a warp covers 8 rows x 4 consecutive chunks,
  // so 8 lanes store one core matrix (128 contiguous bytes, no bank conflict)
  // and lanes l, l+8 read adjacent halves of one 32-byte sector
  auto chunk_pos = [](int c, int& row, int& kc) {
    const int w = c >> 5, l = c & 31;
    row = (w >> 1) * 8 + (l & 7);
    kc = (w & 1) * 4 + (l >> 3);
  };
  constexpr int kAChunks = kBM * 8 / 128, kBChunks = BN * 8 / 128;
  uint4 ra[kAChunks], rb[kBChunks];
  auto load_slice = [&](int kb) {
    const int kk = kbeg + kb * kBK;
#pragma unroll
    for (int t = 0; t < kAChunks; ++t) {
      int row, kc;
      chunk_pos(tid + t * 128, row, kc);
      ra[t] = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + row) * lda + kk + kc * 8);
    }
#pragma unroll
    for (int t = 0; t < kBChunks; ++t) {
      int row, kc;
      chunk_pos(tid + t * 128, row, kc);
      rb[t] = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + row) * ldb + kk + kc * 8);
    }
  };
  auto store_slice = [&](int s) {
#pragma unroll
    for (int t = 0; t < kAChunks; ++t) {
      int row, kc;
      chunk_pos(tid + t * 128, row, kc);
      const int off = (kc >> 1) * (kBM * 32) + (row >> 3) * 256 + (kc & 1) * 128 + (row & 7) * 16;
      *reinterpret_cast<uint4*>(sA[s] + off) = ra[t];
    }
#pragma unroll
    for (int t = 0; t < kBChunks; ++t) {
      int row, kc;
      chunk_pos(tid + t * 128, row, kc);
      const int off = (kc >> 1) * (BN * 32) + (row >> 3) * 256 + (kc & 1) * 128 + (row & 7) * 16;
      *reinterpret_cast<uint4*>(sB[s] + off) = rb[t];
    }
  };

  bool ok = true;
  load_slice(0);
  for (int kb = 0; kb < nk; ++kb) {
    const int s = kb & 1;
    if (kb >= 2) {  // stage s is free once the MMAs of slice kb-2 completed
      const int got = mbar_wait(smem_u32(&bar[s]), (uint32_t)(((kb - 2) >> 1) & 1)) ? 1 : 0;
      if (!__syncthreads_and(got)) {
        ok = false;
        break;
      }
    }
    store_slice(s);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (kb + 1 < nk) load_slice(kb + 1);
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int k16 = 0; k16 < kBK / 16; ++k16) {
        const uint64_t ad = smem_desc(smem_u32(sA[s] + k16 * kBM * 32), 128, 256);
        const uint64_t bd = smem_desc(smem_u32(sB[s] + k16 * BN * 32), 128, 256);
        const uint32_t acc = (kb > 0 || k16 > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(&bar[s]))
          : "memory");
    }
  }
  if (ok && nk > 0) {  // the last commit covers every earlier MMA
    const int last = nk - 1;
    const int got =
        mbar_wait(smem_u32(&bar[last & 1]), (uint32_t)((last >> 1) & 1)) ? 1 : 0;
    ok = __syncthreads_and(got) != 0;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicExch(error, 1);
    // one more bounded wait on both stages before the TMEM is freed
    mbar_wait(smem_u32(&bar[0]), 0u);
    mbar_wait(smem_u32(&bar[1]), 0u);
  } else {
    const int row = m0 + warp * 32 + lane;
    float* dst = partial ? partial + (size_t)blockIdx.z * M * N + (size_t)row * N + n0
                         : C + (size_t)row * ldc + n0;
    const bool acc = partial == nullptr && accumulate;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) dst[c0 + i] = acc ? dst[c0 + i] + v[i] : v[i];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN));
}

// -- TMA-fed form ------------------------------------------------------------
// The same product with the operand tiles brought in by the tensor memory
// accelerator: a 2-D tensor map per operand (K innermost, box 64 x rows,
// 128-byte swizzle), so every 64-wide K slice of a 128-row tile is one
// cp.async.bulk.tensor that lands in the canonical SWIZZLE_128B K-major
// layout of the tensor core (rows of 128 bytes, 8-row atoms of 1024 bytes,
// 16-byte chunks permuted by row).  Three stages: one thread issues the TMA
// loads of slice k + 2 while another has the MMAs of slice k in flight;
// stage s is refilled once the MMAs that read it have committed to empty[s].
constexpr int kStagesT = 3;

// Shared-memory descriptor of a SWIZZLE_128B K-major tile: start address,
// stride between 8-row atoms 1024 bytes, leading offset unused (1), version
// 1, layout type 2 (128-byte swizzle).  The K step of 16 elements advances
// the start address by 32 bytes inside the atom.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
      : "memory");
}

// One CTA computes a 128 x BN tile of C over the K range of blockIdx.z (as
// k_gemm_bf16).  Thread 0 issues the TMA loads, thread 32 the MMAs; every
// wait is bounded, and a CTA that gives up raises the error word, waits
// (bounded) for the copies and MMAs it started, frees its TMEM and returns.
template <int BN>
__global__ void __launch_bounds__(128)
    k_gemm_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
               float* __restrict__ C, float* __restrict__ partial, int M, int N, int kchunk,
               int ldc, int accumulate, int* __restrict__ error) {
  extern __shared__ uint8_t smem_t[];
  constexpr uint32_t kATile = kBM * kBK * 2, kBTile = BN * kBK * 2;
  __shared__ __align__(8) uint64_t full[kStagesT], empty[kStagesT], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail, s_issued, s_consumed;
  const uint32_t base = (smem_u32(smem_t) + 1023u) & ~1023u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int kbeg = blockIdx.z * kchunk, nk = kchunk / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 32) {
    for (int s = 0; s < kStagesT; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&done)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = instr_desc_bf16(kBM, BN);

  if (tid == 0) {
    int kb = 0;
    for (; kb < nk; ++kb) {
      const int s = kb % kStagesT, j = kb / kStagesT;
      if (kb >= kStagesT && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((j - 1) & 1))) {
        s_fail = 1;
        break;
      }
      const uint32_t a = base + (uint32_t)s * (kATile + kBTile);
      mbar_expect(smem_u32(&full[s]), kATile + kBTile);
      tma_load_2d(a, &mapA, kbeg + kb * kBK, m0, smem_u32(&full[s]));
      tma_load_2d(a + kATile, &mapB, kbeg + kb * kBK, n0, smem_u32(&full[s]));
    }
    s_issued = kb;
  } else if (tid == 32) {
    int kb = 0;
    for (; kb < nk; ++kb) {
      const int s = kb % kStagesT, j = kb / kStagesT;
      if (!mbar_wait(smem_u32(&full[s]), (uint32_t)(j & 1))) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a = base + (uint32_t)s * (kATile + kBTile);
#pragma unroll
      for (int k16 = 0; k16 < kBK / 16; ++k16) {
        const uint64_t ad = smem_desc_sw128(a + k16 * 32);
        const uint64_t bd = smem_desc_sw128(a + kATile + k16 * 32);
        const uint32_t acc = (kb > 0 || k16 > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
      }
      mma_commit(smem_u32(&empty[s]));
    }
    s_consumed = kb;
    mma_commit(smem_u32(&done));  // tracks every MMA issued, also after a failure
  }
  __syncthreads();
  const int got = mbar_wait(smem_u32(&done), 0u) ? 1 : 0;
  const bool ok = __syncthreads_and(got && s_fail == 0) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) {
      atomicExch(error, 1);
      // loads issued but not consumed still target this CTA's shared memory
      for (int kb = s_consumed; kb < s_issued; ++kb)
        mbar_wait(smem_u32(&full[kb % kStagesT]), (uint32_t)((kb / kStagesT) & 1));
    }
  } else {
    const int row = m0 + warp * 32 + lane;
    float* dst = partial ? partial + (size_t)blockIdx.z * M * N + (size_t)row * N + n0
                         : C + (size_t)row * ldc + n0;
    const bool acc = partial == nullptr && accumulate;
    // 16-byte stores when the row start allows them (partials always do)
    const bool vec = (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (vec) {
        float4* d4 = reinterpret_cast<float4*>(dst + c0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          float4 o = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
          if (acc) {
            const float4 c = d4[i];
            o.x = c.x + o.x;
            o.y = c.y + o.y;
            o.z = c.z + o.z;
            o.w = c.w + o.w;
          }
          d4[i] = o;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) dst[c0 + i] = acc ? dst[c0 + i] + v[i] : v[i];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN));
}

// C (+)= sum_z partial[z] in z order.
__global__ void k_gemm_reduce(int splits, long long MN, int M, int N, int ldc,
                              const float* __restrict__ partial, float* __restrict__ C,
                              int accumulate) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= MN) return;
  const int m = (int)(t / N), n = (int)(t - (long long)m * N);
  float acc = accumulate ? C[(size_t)m * ldc + n] : 0.0f;
  for (int z = 0; z < splits; ++z) acc += partial[(size_t)z * MN + t];
  C[(size_t)m * ldc + n] = acc;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver API); null if unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of a K-major bf16 operand (rows x K, leading dimension ld):
// boxes of 64 K-elements (128 bytes) x box_rows rows, 128-byte swizzle.
bool operand_map(CUtensorMap* map, const void* ptr, int rows, int K, int ld, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
             elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// CVLBM_GEMM_LOADER=threads selects the thread-loaded kernel (comparison).
bool tma_allowed() {
  const char* e = std::getenv("CVLBM_GEMM_LOADER");
  return !(e && std::strcmp(e, "threads") == 0);
}

}  // namespace

extern "C" int64_t cvlbm_gemm_bf16_workspace(int32_t M, int32_t N, int32_t K) {
  return (int64_t)kMaxSplits * M * N * (int64_t)sizeof(float);
}

extern "C" int cvlbm_gemm_bf16(const void* A, const void* B, float* C, int32_t M, int32_t N,
                               int32_t K, int32_t lda, int32_t ldb, int32_t ldc,
                               int32_t accumulate, int32_t* error, void* workspace,
                               int64_t workspace_bytes, void* stream) {
  if (!A || !B || !C || !error) return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: null pointer");
  if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % kBN || K % kBK)
    return fail(CVLBM_ERR_INVALID_ARG,
                "cvlbm_gemm_bf16: M must be a multiple of 128, N of 64 and K of 64");
  if (lda < K || ldb < K || ldc < N || lda % 8 || ldb % 8)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: bad leading dimensions");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_gemm_bf16: A and B must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  const int bn = (N % 128 == 0) ? 128 : 64;
  const int tiles = (M / kBM) * (N / bn);
  // split K until about two CTAs per SM, keeping at least 4 slices per split
  int splits = 1;
  const long long nkb = K / kBK;
  while (splits < kMaxSplits && tiles * splits < 296 && nkb % (2 * splits) == 0 &&
         nkb / (2 * splits) >= 4 &&
         (long long)(2 * splits) * M * N * (long long)sizeof(float) <= workspace_bytes)
    splits *= 2;
  float* part = splits > 1 ? static_cast<float*>(workspace) : nullptr;
  dim3 grid(M / kBM, N / bn, splits);
  const int kchunk = K / splits;
  CUtensorMap mapA, mapB;
  if (tma_allowed() && operand_map(&mapA, A, M, K, lda, kBM) &&
      operand_map(&mapB, B, N, K, ldb, bn)) {
    const size_t smem = (size_t)kStagesT * (kBM + bn) * kBK * 2 + 1024;
    if (bn == 128) {
      cudaFuncSetAttribute(k_gemm_tma<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      k_gemm_tma<128><<<grid, 128, smem, s>>>(mapA, mapB, C, part, M, N, kchunk, ldc, accumulate,
                                              error);
    } else {
      cudaFuncSetAttribute(k_gemm_tma<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      k_gemm_tma<64><<<grid, 128, smem, s>>>(mapA, mapB, C, part, M, N, kchunk, ldc, accumulate,
                                             error);
    }
  } else if (bn == 128) {
    const size_t smem = 2 * (kBM + 128) * kBK * 2;
    cudaFuncSetAttribute(k_gemm_bf16<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_gemm_bf16<128><<<grid, 128, smem, s>>>(static_cast<const __nv_bfloat16*>(A),
                                             static_cast<const __nv_bfloat16*>(B), C, part, M, N,
                                             kchunk, lda, ldb, ldc, accumulate, error);
  } else {
    const size_t smem = 2 * (kBM + 64) * kBK * 2;
    cudaFuncSetAttribute(k_gemm_bf16<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_gemm_bf16<64><<<grid, 128, smem, s>>>(static_cast<const __nv_bfloat16*>(A),
                                            static_cast<const __nv_bfloat16*>(B), C, part, M, N,
                                            kchunk, lda, ldb, ldc, accumulate, error);
  }
  cv::count_launches(1);
  if (splits > 1) {
    const long long MN = (long long)M * N;
    k_gemm_reduce<<<(unsigned)((MN + 255) / 256), 256, 0, s>>>(splits, MN, M, N, ldc, part, C,
                                                               accumulate);
    cv::count_launches(1);
  }
  return check_launch("cvlbm_gemm_bf16");
}
