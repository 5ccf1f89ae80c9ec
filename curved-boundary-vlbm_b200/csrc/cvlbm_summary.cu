// Field reductions of the solvers' summary() on the device: max |u|, max |v|,
// min J, max J and the finite flag over the active nodes, from the refreshed
// U and u (two_d/curved_boundary_warp.py:4343-4415,
// three_d/curved_boundary_warp3d.py summary).  Each node's values are formed
// with the reference's NumPy expressions in their order; max / min are exact,
// so the results equal the host reductions of the downloaded fields.
#include <cuda_runtime.h>

#include <cstdint>

#include "cvlbm_common.cuh"

using namespace cv;

namespace {

struct SummaryAcc {
  unsigned long long max_u, max_v;  // bit patterns of non-negative doubles (NaN above +inf)
  unsigned long long min_j, max_j;  // order-preserving keys of J
  int32_t nan_j, not_finite, count, pad;
};

__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__host__ __device__ inline double from_key(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double d;
  static_assert(sizeof(d) == sizeof(b), "double size");
  __builtin_memcpy(&d, &b, sizeof(d));
  return d;
#endif
}

template <int D>
__global__ void __launch_bounds__(256)
    k_summary(const double* __restrict__ U, const double* __restrict__ u,
              const int32_t* __restrict__ active, int64_t n_nodes, SummaryAcc* acc) {
  const int64_t N = n_nodes;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool use = n < N && (!active || active[n] != 0);
  double au = 0.0, av = 0.0, J = 0.0;
  bool finite = true;
  if (use) {
    if (D == 2) {
      const double u0 = u[n], u1 = u[N + n];
      const double v0 = U[n], v1 = U[N + n];
      const double F11 = U[2 * N + n], F12 = U[3 * N + n], F21 = U[4 * N + n],
                   F22 = U[5 * N + n];
      au = sqrt(u0 * u0 + u1 * u1);
      av = sqrt(v0 * v0 + v1 * v1);
      J = F11 * F22 - F12 * F21;
      finite = isfinite(u0) && isfinite(u1) && isfinite(v0) && isfinite(v1) && isfinite(F11) &&
               isfinite(F12) && isfinite(F21) && isfinite(F22);
    } else {
      const double u0 = u[n], u1 = u[N + n], u2 = u[2 * N + n];
      const double v0 = U[n], v1 = U[N + n], v2 = U[2 * N + n];
      double F[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) F[k] = U[(3 + k) * N + n];
      au = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
      av = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
          F[2] * (F[3] * F[7] - F[4] * F[6]);
      finite = isfinite(v0) && isfinite(v1) && isfinite(v2);
#pragma unroll
      for (int k = 0; k < 9; ++k) finite = finite && isfinite(F[k]);
    }
    finite = finite && J > 0.0;
  }
  // warp reductions, one atomic per warp and quantity
  unsigned long long bu = use ? (unsigned long long)__double_as_longlong(fabs(au)) : 0ull;
  unsigned long long bv = use ? (unsigned long long)__double_as_longlong(fabs(av)) : 0ull;
  unsigned long long kmin = use && !isnan(J) ? order_key(J) : ~0ull;
  unsigned long long kmax = use && !isnan(J) ? order_key(J) : 0ull;
  int nanj = use && isnan(J), bad = use && !finite, cnt = use;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a1 = __shfl_xor_sync(0xffffffffu, bu, o);
    const unsigned long long a2 = __shfl_xor_sync(0xffffffffu, bv, o);
    const unsigned long long a3 = __shfl_xor_sync(0xffffffffu, kmin, o);
    const unsigned long long a4 = __shfl_xor_sync(0xffffffffu, kmax, o);
    bu = a1 > bu ? a1 : bu;
    bv = a2 > bv ? a2 : bv;
    kmin = a3 < kmin ? a3 : kmin;
    kmax = a4 > kmax ? a4 : kmax;
    nanj |= __shfl_xor_sync(0xffffffffu, nanj, o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0 && cnt > 0) {
    atomicMax(&acc->max_u, bu);
    atomicMax(&acc->max_v, bv);
    atomicMin(&acc->min_j, kmin);
    atomicMax(&acc->max_j, kmax);
    if (nanj) atomicOr(&acc->nan_j, 1);
    if (bad) atomicOr(&acc->not_finite, 1);
    atomicAdd(&acc->count, cnt);
  }
}

}  // namespace

extern "C" int64_t cvlbm_field_summary_work_bytes(void) { return (int64_t)sizeof(SummaryAcc); }

extern "C" int cvlbm_field_summary(int32_t dim, int64_t n_nodes, const double* U, const double* u,
                                   const int32_t* active, void* work, double* out, void* stream) {
  if ((dim != 2 && dim != 3) || n_nodes < 0 || !work || !out || (n_nodes > 0 && (!U || !u)))
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_field_summary: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  SummaryAcc init{0ull, 0ull, ~0ull, 0ull, 0, 0, 0, 0};
  auto* acc = static_cast<SummaryAcc*>(work);
  cudaMemcpyAsync(acc, &init, sizeof(init), cudaMemcpyHostToDevice, s);
  if (n_nodes > 0) {
    const unsigned nb = (unsigned)((n_nodes + 255) / 256);
    if (dim == 2)
      k_summary<2><<<nb, 256, 0, s>>>(U, u, active, n_nodes, acc);
    else
      k_summary<3><<<nb, 256, 0, s>>>(U, u, active, n_nodes, acc);
    cv::count_launches(1);
  }
  SummaryAcc h{};
  cudaMemcpyAsync(&h, acc, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_launch("cvlbm_field_summary");
  const double qnan = __builtin_nan("");
  double bu, bv;
  __builtin_memcpy(&bu, &h.max_u, sizeof(bu));
  __builtin_memcpy(&bv, &h.max_v, sizeof(bv));
  out[0] = bu;
  out[1] = bv;
  out[2] = h.nan_j ? qnan : (h.count ? from_key(h.min_j) : 0.0);
  out[3] = h.nan_j ? qnan : (h.count ? from_key(h.max_j) : 0.0);
  out[4] = (h.count > 0 && !h.not_finite) ? 1.0 : 0.0;
  out[5] = (double)h.count;
  return check_launch("cvlbm_field_summary");
}
