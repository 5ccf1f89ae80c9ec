// Forward and backward kernels of the warm-start surrogate, a Fourier neural
// operator (FNO) on the solver lattice.  The spectral transforms run on the
// tensor cores through cvlbm_gemm_bf16; this file holds the CUDA-core parts.
//
// Layouts (fp32 unless stated): activations channel-major per sample,
// X[b][c][g] with g the lattice node (k fastest); spectral coefficients
// A[b][c][k] with k the retained real Fourier mode; weights W[o][i] (pointwise
// channel mixing), R[k][i][o] (per-mode channel mixing).
//
// Reductions over samples and nodes (weight gradients, the loss) go through
// fixed-size per-block partials and a second pass, so every result is
// deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "cvlbm_common.cuh"

using namespace cv;

namespace {

constexpr int kMaxC = 32;  // channel limit of the pointwise kernels

__device__ __forceinline__ float gelu_f(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// z[b][o][g] = bias[o] + sum_i W[o][i] x[b][i][g] (+ s[b][o][g]);
// y = gelu(z) if act else z.  One thread per (b, g).
__global__ void k_pointwise_fwd(int B, int G, int Cin, int Cout, const float* __restrict__ x,
                                const float* __restrict__ W, const float* __restrict__ bias,
                                const float* __restrict__ s, int act, float* __restrict__ z,
                                float* __restrict__ y) {
  __shared__ float sW[kMaxC * kMaxC], sb[kMaxC];
  for (int t = threadIdx.x; t < Cout * Cin; t += blockDim.x) sW[t] = W[t];
  for (int t = threadIdx.x; t < Cout; t += blockDim.x) sb[t] = bias[t];
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * G) return;
  const int b = (int)(t / G), g = (int)(t - (long long)b * G);
  float xi[kMaxC];
  for (int i = 0; i < Cin; ++i) xi[i] = x[((size_t)b * Cin + i) * G + g];
  for (int o = 0; o < Cout; ++o) {
    float acc = sb[o];
    for (int i = 0; i < Cin; ++i) acc += sW[o * Cin + i] * xi[i];
    const size_t k = ((size_t)b * Cout + o) * G + g;
    if (s) acc += s[k];
    if (z) z[k] = acc;
    y[k] = act ? gelu_f(acc) : acc;
  }
}

// dz = dy * gelu'(z)
__global__ void k_gelu_bwd(long long n, const float* __restrict__ z, const float* __restrict__ dy,
                           float* __restrict__ dz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dz[t] = dy[t] * gelu_grad(z[t]);
}

// dx[b][i][g] (+)= sum_o W[o][i] dz[b][o][g].  One thread per (b, g).
__global__ void k_pointwise_bwd_x(int B, int G, int Cin, int Cout, const float* __restrict__ dz,
                                  const float* __restrict__ W, int accumulate,
                                  float* __restrict__ dx) {
  __shared__ float sW[kMaxC * kMaxC];
  for (int t = threadIdx.x; t < Cout * Cin; t += blockDim.x) sW[t] = W[t];
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * G) return;
  const int b = (int)(t / G), g = (int)(t - (long long)b * G);
  float d[kMaxC];
  for (int o = 0; o < Cout; ++o) d[o] = dz[((size_t)b * Cout + o) * G + g];
  for (int i = 0; i < Cin; ++i) {
    float acc = 0.0f;
    for (int o = 0; o < Cout; ++o) acc += sW[o * Cin + i] * d[o];
    const size_t k = ((size_t)b * Cin + i) * G + g;
    dx[k] = accumulate ? dx[k] + acc : acc;
  }
}

// Partial weight gradients over a chunk of 128 nodes of one sample:
// part[c][o*Cin+i] = sum_g dz[b][o][g] x[b][i][g], part[c][Cout*Cin+o] = sum_g dz.
constexpr int kChunkG = 128;
__global__ void __launch_bounds__(256)
    k_pointwise_bwd_w_part(int B, int G, int Cin, int Cout, const float* __restrict__ dz,
                           const float* __restrict__ x, float* __restrict__ part) {
  __shared__ float sdz[kMaxC][kChunkG], sx[kMaxC][kChunkG];
  const int chunks = (G + kChunkG - 1) / kChunkG;
  const int c = blockIdx.x, b = c / chunks, g0 = (c % chunks) * kChunkG;
  for (int t = threadIdx.x; t < kMaxC * kChunkG; t += blockDim.x) {
    const int ch = t / kChunkG, gg = t % kChunkG, g = g0 + gg;
    const bool ok = g < G;
    sdz[ch][gg] = (ch < Cout && ok) ? dz[((size_t)b * Cout + ch) * G + g] : 0.0f;
    sx[ch][gg] = (ch < Cin && ok) ? x[((size_t)b * Cin + ch) * G + g] : 0.0f;
  }
  __syncthreads();
  const int nw = Cout * Cin + Cout;
  float* out = part + (size_t)c * nw;
  for (int t = threadIdx.x; t < nw; t += blockDim.x) {
    float acc = 0.0f;
    if (t < Cout * Cin) {
      const int o = t / Cin, i = t % Cin;
      for (int gg = 0; gg < kChunkG; ++gg) acc += sdz[o][gg] * sx[i][gg];
    } else {
      const int o = t - Cout * Cin;
      for (int gg = 0; gg < kChunkG; ++gg) acc += sdz[o][gg];
    }
    out[t] = acc;
  }
}

// out[t] = sum_c part[c][t] in chunk order.
__global__ void k_sum_parts(int n_parts, int width, const float* __restrict__ part,
                            float* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= width) return;
  float acc = 0.0f;
  for (int c = 0; c < n_parts; ++c) acc += part[(size_t)c * width + t];
  out[t] = acc;
}

// Per-mode channel mixing: bh[b][o][k] = sum_i a[b][i][k] R[k][i][o], written
// as bf16 for the inverse transform.  One thread per (b, k).
__global__ void k_spec_mix_fwd(int B, int C, int M, const float* __restrict__ a,
                               const float* __restrict__ R, __nv_bfloat16* __restrict__ bh) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * M) return;
  const int b = (int)(t / M), k = (int)(t - (long long)b * M);
  float acc[kMaxC];
  for (int o = 0; o < C; ++o) acc[o] = 0.0f;
  const float* Rk = R + (size_t)k * C * C;
  for (int i = 0; i < C; ++i) {
    const float ai = a[((size_t)b * C + i) * M + k];
    for (int o = 0; o < C; ++o) acc[o] += ai * Rk[i * C + o];
  }
  for (int o = 0; o < C; ++o) bh[((size_t)b * C + o) * M + k] = __float2bfloat16_rn(acc[o]);
}

// da[b][i][k] = sum_o R[k][i][o] dbh[b][o][k] (bf16 out, for the inverse of
// the transform in the backward pass).  One thread per (b, k).
__global__ void k_spec_mix_bwd_a(int B, int C, int M, const float* __restrict__ dbh,
                                 const float* __restrict__ R, __nv_bfloat16* __restrict__ da) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * M) return;
  const int b = (int)(t / M), k = (int)(t - (long long)b * M);
  float d[kMaxC];
  for (int o = 0; o < C; ++o) d[o] = dbh[((size_t)b * C + o) * M + k];
  const float* Rk = R + (size_t)k * C * C;
  for (int i = 0; i < C; ++i) {
    float acc = 0.0f;
    for (int o = 0; o < C; ++o) acc += Rk[i * C + o] * d[o];
    da[((size_t)b * C + i) * M + k] = __float2bfloat16_rn(acc);
  }
}

// dR[k][i][o] = sum_b a[b][i][k] dbh[b][o][k].  One thread per (k, i, o).
__global__ void k_spec_mix_bwd_r(int B, int C, int M, const float* __restrict__ a,
                                 const float* __restrict__ dbh, float* __restrict__ dR) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)M * C * C) return;
  const int k = (int)(t / (C * C)), r = (int)(t - (long long)k * C * C), i = r / C, o = r % C;
  float acc = 0.0f;
  for (int b = 0; b < B; ++b)
    acc += a[((size_t)b * C + i) * M + k] * dbh[((size_t)b * C + o) * M + k];
  dR[t] = acc;
}

__global__ void k_to_bf16(long long n, const float* __restrict__ src,
                          __nv_bfloat16* __restrict__ dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = __float2bfloat16_rn(src[t]);
}

// Masked mean-squared error: loss = sum w_o mask (y - t)^2 / count,
// dy = 2 w_o mask (y - t) / count; per-block loss partials.
__global__ void __launch_bounds__(256)
    k_mse(int B, int C, int G, const float* __restrict__ y, const float* __restrict__ tgt,
          const float* __restrict__ mask, const float* __restrict__ w, float inv_count,
          float* __restrict__ dy, float* __restrict__ part) {
  __shared__ float red[256];
  const long long n = (long long)B * C * G;
  float acc = 0.0f;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long bc = t / G;
    const int g = (int)(t - bc * G), b = (int)(bc / C), o = (int)(bc % C);
    const float m = mask[(size_t)b * G + g] * w[o];
    const float e = y[t] - tgt[t];
    acc += m * e * e;
    dy[t] = 2.0f * m * e * inv_count;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0] * inv_count;
}

// Adam with bias correction (lr already includes it).
__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2,
                       float eps) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * mt / (sqrtf(vt) + eps);
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" int cvlbm_fno_pointwise_fwd(int32_t B, int32_t G, int32_t Cin, int32_t Cout,
                                       const float* x, const float* W, const float* bias,
                                       const float* s, int32_t act, float* z, float* y,
                                       void* stream) {
  if (Cin > kMaxC || Cout > kMaxC || Cin <= 0 || Cout <= 0)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_fno_pointwise_fwd: 1..32 channels");
  k_pointwise_fwd<<<nblk((long long)B * G, 128), 128, 0, (cudaStream_t)stream>>>(
      B, G, Cin, Cout, x, W, bias, s, act, z, y);
  cv::count_launches(1);
  return check_launch("cvlbm_fno_pointwise_fwd");
}

extern "C" int cvlbm_fno_gelu_bwd(int64_t n, const float* z, const float* dy, float* dz,
                                  void* stream) {
  k_gelu_bwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, z, dy, dz);
  cv::count_launches(1);
  return check_launch("cvlbm_fno_gelu_bwd");
}

extern "C" int cvlbm_fno_pointwise_bwd(int32_t B, int32_t G, int32_t Cin, int32_t Cout,
                                       const float* dz, const float* x, const float* W,
                                       float* dx, int32_t accumulate_dx, float* dW, float* db,
                                       float* scratch, void* stream) {
  if (Cin > kMaxC || Cout > kMaxC || Cin <= 0 || Cout <= 0)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_fno_pointwise_bwd: 1..32 channels");
  cudaStream_t s = (cudaStream_t)stream;
  if (dx) {
    k_pointwise_bwd_x<<<nblk((long long)B * G, 128), 128, 0, s>>>(B, G, Cin, Cout, dz, W,
                                                                  accumulate_dx, dx);
    cv::count_launches(1);
  }
  const int chunks = (G + kChunkG - 1) / kChunkG;
  const int nparts = B * chunks, width = Cout * Cin + Cout;
  k_pointwise_bwd_w_part<<<nparts, 256, 0, s>>>(B, G, Cin, Cout, dz, x, scratch);
  cv::count_launches(1);
  // scratch holds nparts x width partials; the sums land behind them
  float* sums = scratch + (size_t)nparts * width;
  k_sum_parts<<<nblk(width, 128), 128, 0, s>>>(nparts, width, scratch, sums);
  cv::count_launches(1);
  cudaMemcpyAsync(dW, sums, sizeof(float) * Cout * Cin, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(db, sums + Cout * Cin, sizeof(float) * Cout, cudaMemcpyDeviceToDevice, s);
  return check_launch("cvlbm_fno_pointwise_bwd");
}

extern "C" int64_t cvlbm_fno_pointwise_scratch(int32_t B, int32_t G, int32_t Cin,
                                               int32_t Cout) {
  const long long chunks = (G + kChunkG - 1) / kChunkG;
  return ((long long)B * chunks + 1) * ((long long)Cout * Cin + Cout);
}

extern "C" int cvlbm_fno_spec_mix_fwd(int32_t B, int32_t C, int32_t M, const float* a,
                                      const float* R, void* bh_bf16, void* stream) {
  if (C > kMaxC) return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_fno_spec_mix_fwd: C <= 32");
  k_spec_mix_fwd<<<nblk((long long)B * M, 128), 128, 0, (cudaStream_t)stream>>>(
      B, C, M, a, R, static_cast<__nv_bfloat16*>(bh_bf16));
  cv::count_launches(1);
  return check_launch("cvlbm_fno_spec_mix_fwd");
}

extern "C" int cvlbm_fno_spec_mix_bwd(int32_t B, int32_t C, int32_t M, const float* a,
                                      const float* dbh, const float* R, void* da_bf16,
                                      float* dR, void* stream) {
  if (C > kMaxC) return fail(CVLBM_ERR_INVALID_ARG, "cvlbm_fno_spec_mix_bwd: C <= 32");
  cudaStream_t s = (cudaStream_t)stream;
  k_spec_mix_bwd_a<<<nblk((long long)B * M, 128), 128, 0, s>>>(
      B, C, M, dbh, R, static_cast<__nv_bfloat16*>(da_bf16));
  cv::count_launches(1);
  k_spec_mix_bwd_r<<<nblk((long long)M * C * C, 256), 256, 0, s>>>(B, C, M, a, dbh, dR);
  cv::count_launches(1);
  return check_launch("cvlbm_fno_spec_mix_bwd");
}

extern "C" int cvlbm_fno_to_bf16(int64_t n, const float* src, void* dst, void* stream) {
  k_to_bf16<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, src,
                                                           static_cast<__nv_bfloat16*>(dst));
  cv::count_launches(1);
  return check_launch("cvlbm_fno_to_bf16");
}

extern "C" int cvlbm_fno_mse(int32_t B, int32_t C, int32_t G, const float* y, const float* t,
                             const float* mask, const float* w, float inv_count, float* dy,
                             float* part, int32_t n_parts, void* stream) {
  k_mse<<<n_parts, 256, 0, (cudaStream_t)stream>>>(B, C, G, y, t, mask, w, inv_count, dy, part);
  cv::count_launches(1);
  return check_launch("cvlbm_fno_mse");
}

extern "C" int cvlbm_fno_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr,
                              float b1, float b2, float eps, void* stream) {
  k_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2, eps);
  cv::count_launches(1);
  return check_launch("cvlbm_fno_adam");
}
