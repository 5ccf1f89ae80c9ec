// Initial populations of initialize_from_numpy on the device.  Included at
// the end of cvlbm2d.cu (shares Ctx2 and the material helpers).
//
// The reference forms them on the host with NumPy
// (two_d/vector_nonlinear_elastic_warp.py:595-847):
//   order 1  f = feq(U) - (0.5 dt / 4) B(U)
//   order 2  f = feq(U) - 0.5 dt corr,  corr_q = 0.25 (W_q + (2/c) c_q.A W_q),
//            W_q = U_t + c (c_qx U_x + c_qy U_y),  U_t = B(U) - (A_x U_x + A_y U_y),
//            U_x, U_y centred differences (second-order one-sided at the edges)
//   order 3  order 2 on U with inactive nodes replaced by the undeformed state
//            and derivatives from active neighbours only
// A_axis W is a centred difference of the flux with one step
// eps = 1e-6 / max(1, max|W|) for the WHOLE field, so the step needs three
// launches with two global maxima between them:
//   k_init_deriv2  U_x, U_y (12 rows) and max|U_x|, max|U_y|
//   k_init_w2      A_x U_x, A_y U_y, U_t, the four W_q (24 rows), max|W_q|
//   k_init_f2      feq, A_x W_q, A_y W_q, the populations (zero at inactive nodes)
// Every expression keeps the operand order of the NumPy code, so with the
// library's --fmad=false the populations are the host's doubles (the laws
// with log/exp differ by the two libm's rounding).  The host code raises
// FloatingPointError (and retries a flux tangent with a smaller step) where
// a flux evaluation meets J <= 0 or the Gent chain limit; the kernels raise
// *status instead and the caller repeats the host computation, which then
// takes its own course.
#pragma once

namespace {

constexpr int kInitMax = 6;  // |U_x|, |U_y|, |W_0| .. |W_3|

// P(F) as _first_piola_np evaluates it, or bad = true where the NumPy code
// raises or where piola2's Jacobian / chain-limit floors would change a value
// the NumPy code uses unclamped.
__device__ __forceinline__ P2 piola2_np(double F11, double F12, double F21, double F22,
                                        const Mat& m, bool& bad) {
  if (m.model != kMatSVK) {
    const double J = F11 * F22 - F12 * F21;
    if (!(J > 0.0) || J < m.jf) bad = true;
    if (m.model == kMatGent && J > 0.0) {
      const double logJ = log(J);
      const double jm23 = exp((-2.0 / 3.0) * logJ);
      const double I1 = (F11 * F11 + F12 * F12 + F21 * F21 + F22 * F22) + 1.0;
      const double den = 1.0 - (jm23 * I1 - 3.0) / m.p0;
      if (!(den > 0.0) || den < m.jf) bad = true;
    }
  }
  return piola2(F11, F12, F21, F22, m);
}

// _flux_np of one node, axis 1 (x) or 2 (y).
__device__ __forceinline__ void flux2_np(const double* u, int axis, const Mat& m, double* out,
                                         bool& bad) {
  const P2 P = piola2_np(u[2], u[3], u[4], u[5], m, bad);
  if (axis == 1) {
    out[0] = -P.a;
    out[1] = -P.c;
    out[2] = -u[0];
    out[3] = 0.0;
    out[4] = -u[1];
    out[5] = 0.0;
  } else {
    out[0] = -P.b;
    out[1] = -P.d;
    out[2] = 0.0;
    out[3] = -u[0];
    out[4] = 0.0;
    out[5] = -u[1];
  }
}

// _flux_jvp_np of one node for the field maximum `scale` = max|W|.
__device__ __forceinline__ void flux2_jvp_np(const double* u, const double* w, double scale,
                                             int axis, const Mat& m, double* out, bool& bad) {
  if (scale == 0.0 || !isfinite(scale)) {
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    return;
  }
  const double eps = 1.0e-6 / (scale > 1.0 ? scale : 1.0);
  double up[6], um[6], fp[6], fm[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    up[k] = u[k] + eps * w[k];
    um[k] = u[k] - eps * w[k];
  }
  flux2_np(up, axis, m, fp, bad);
  flux2_np(um, axis, m, fm, bad);
  const double den = 2.0 * eps;
#pragma unroll
  for (int k = 0; k < 6; ++k) out[k] = (fp[k] - fm[k]) / den;
}

// U of node n as the init uses it (order 3: the undeformed state at inactive nodes).
__device__ __forceinline__ void init_u2(const Ctx2& c, const double* __restrict__ U, int order,
                                        int n, double* u) {
  const int N = c.N;
  if (order == 3 && c.p.active[n] == 0) {
    u[0] = u[1] = u[3] = u[4] = 0.0;
    u[2] = u[5] = 1.0;
    return;
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) u[a] = U[(size_t)a * N + n];
}

__device__ __forceinline__ double init_uc2(const Ctx2& c, const double* __restrict__ U,
                                           int order, int a, int n) {
  if (order == 3 && c.p.active[n] == 0) return (a == 2 || a == 5) ? 1.0 : 0.0;
  return U[(size_t)a * c.N + n];
}

// d/d(axis) of component a at node (i, j): _spatial_derivative (order 2) or
// _active_derivative_first_spatial (order 3), non-periodic.
__device__ __forceinline__ double init_deriv2(const Ctx2& c, const double* __restrict__ U,
                                              int order, int a, int i, int j, int axis) {
  const cvlbm2d_problem& p = c.p;
  const int len = axis == 1 ? p.nx : p.ny;
  const int k = axis == 1 ? i : j;
  const int st = axis == 1 ? p.ny : 1;
  const int n = i * p.ny + j;
  const double h = axis == 1 ? p.dx : p.dy;
  auto val = [&](int off) { return init_uc2(c, U, order, a, n + off * st); };
  if (order != 3) {
    const double h2 = 2.0 * h;
    if (len < 3) return 0.0;
    if (k == 0) return (-3.0 * val(0) + 4.0 * val(1) - val(2)) / h2;
    if (k == len - 1) return (3.0 * val(0) - 4.0 * val(-1) + val(-2)) / h2;
    return (val(1) - val(-1)) / h2;
  }
  if (len < 2) return 0.0;
  auto act = [&](int off) {
    const int kk = k + off;
    return kk >= 0 && kk < len && p.active[n + off * st] != 0;
  };
  if (len >= 3) {
    if (k >= 1 && k <= len - 2 && act(0) && act(1) && act(-1))
      return (val(1) - val(-1)) / (2.0 * h);
    if (k <= len - 3 && act(0) && act(1) && act(2))
      return (-3.0 * val(0) + 4.0 * val(1) - val(2)) / (2.0 * h);
    if (k >= 2 && act(0) && act(-1) && act(-2))
      return (3.0 * val(0) - 4.0 * val(-1) + val(-2)) / (2.0 * h);
  }
  if (k <= len - 2 && act(0) && act(1)) return (val(1) - val(0)) / h;
  if (k >= 1 && act(0) && act(-1)) return (val(0) - val(-1)) / h;
  return 0.0;
}

// Block maximum of non-negative doubles (or NaN) into *gmax: the bit patterns
// of non-negative doubles order like their values, and a NaN's pattern sits
// above +inf, so the maximum is NaN when any input is (as numpy's max).
__device__ __forceinline__ void block_max_abs(double v, unsigned long long* gmax) {
  unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
    b = ob > b ? ob : b;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(gmax, b);
}

__device__ __forceinline__ double max_of(const unsigned long long* gmax, int k) {
  return __longlong_as_double((long long)gmax[k]);
}

__global__ void __launch_bounds__(256) k_init_deriv2(Ctx2 c, const double* __restrict__ U,
                                                     int order, double* __restrict__ D,
                                                     unsigned long long* __restrict__ gmax) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  double mx = 0.0, my = 0.0;
  if (n < N) {
    const int i = n / c.p.ny, j = n - i * c.p.ny;
#pragma unroll 1
    for (int a = 0; a < 6; ++a) {
      const double dxv = init_deriv2(c, U, order, a, i, j, 1);
      const double dyv = init_deriv2(c, U, order, a, i, j, 2);
      D[(size_t)a * N + n] = dxv;
      D[(size_t)(6 + a) * N + n] = dyv;
      // NaN-propagating maxima (fmax would drop a NaN)
      mx = (fabs(dxv) > mx || isnan(dxv)) ? fabs(dxv) : mx;
      my = (fabs(dyv) > my || isnan(dyv)) ? fabs(dyv) : my;
    }
  }
  block_max_abs(mx, gmax + 0);
  block_max_abs(my, gmax + 1);
}

__global__ void __launch_bounds__(256) k_init_w2(Ctx2 c, const double* __restrict__ U,
                                                 int order, const double* __restrict__ D,
                                                 double* __restrict__ W,
                                                 unsigned long long* __restrict__ gmax,
                                                 int32_t* __restrict__ status) {
  const cvlbm2d_problem& p = c.p;
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  double mq[4] = {0.0, 0.0, 0.0, 0.0};
  if (n < N) {
    bool bad = false;
    double u[6], ux[6], uy[6], ax[6], ay[6], ut[6];
    init_u2(c, U, order, n, u);
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      ux[a] = D[(size_t)a * N + n];
      uy[a] = D[(size_t)(6 + a) * N + n];
    }
    flux2_jvp_np(u, ux, max_of(gmax, 0), 1, c.m, ax, bad);
    flux2_jvp_np(u, uy, max_of(gmax, 1), 2, c.m, ay, bad);
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      double src = 0.0;
      if (p.source_mode == kSrcConstant) src = p.source[a];
      else if (p.source_mode == kSrcDamping && a < 2) src = -p.source[0] * u[a];
      ut[a] = src - (ax[a] + ay[a]);
    }
    const double cc = p.c;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double cx = (double)cx2(q), cy = (double)cy2(q);
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        const double w = ut[a] + cc * (cx * ux[a] + cy * uy[a]);
        W[(size_t)(q * 6 + a) * N + n] = w;
        mq[q] = (fabs(w) > mq[q] || isnan(w)) ? fabs(w) : mq[q];
      }
    }
    if (bad) *status = 1;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) block_max_abs(mq[q], gmax + 2 + q);
}

__global__ void __launch_bounds__(256) k_init_f2(Ctx2 c, const double* __restrict__ U,
                                                 int order, const double* __restrict__ W,
                                                 const unsigned long long* __restrict__ gmax,
                                                 double* __restrict__ f0,
                                                 int32_t* __restrict__ status) {
  const cvlbm2d_problem& p = c.p;
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  bool bad = false;
  double u[6], phx[6], phy[6];
  init_u2(c, U, order, n, u);
  flux2_np(u, 1, c.m, phx, bad);
  flux2_np(u, 2, c.m, phy, bad);
  const bool act = p.active[n] != 0;
  const double k = 2.0 / p.c;
  const double hdt = 0.5 * p.dt;
  const double hdtq = 0.5 * p.dt / 4.0;
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const double cx = (double)cx2(q), cy = (double)cy2(q);
    double w[6], axw[6], ayw[6];
    if (order != 1) {
#pragma unroll
      for (int a = 0; a < 6; ++a) w[a] = W[(size_t)(q * 6 + a) * N + n];
      flux2_jvp_np(u, w, max_of(gmax, 2 + q), 1, c.m, axw, bad);
      flux2_jvp_np(u, w, max_of(gmax, 2 + q), 2, c.m, ayw, bad);
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      const double feq = 0.25 * (u[a] + k * (cx * phx[a] + cy * phy[a]));
      double v;
      if (order == 1) {
        double src = 0.0;
        if (p.source_mode == kSrcConstant) src = p.source[a];
        else if (p.source_mode == kSrcDamping && a < 2) src = -p.source[0] * u[a];
        v = feq - hdtq * src;
      } else {
        const double corr = 0.25 * (w[a] + (2.0 / p.c) * (cx * axw[a] + cy * ayw[a]));
        v = feq - hdt * corr;
      }
      f0[(size_t)(q * 6 + a) * N + n] = act ? v : 0.0;
    }
  }
  if (bad) *status = 1;
}

}  // namespace

extern "C" int64_t cvlbm2d_init_work_bytes(int32_t nx, int32_t ny) {
  if (nx <= 0 || ny <= 0) return 0;
  const int64_t N = (int64_t)nx * ny;
  return (int64_t)sizeof(double) * 36 * N + (int64_t)sizeof(unsigned long long) * 8;
}

extern "C" int cvlbm2d_init_populations(const cvlbm2d_problem* p, const double* U, int32_t order,
                                        double* f0, void* work, int32_t* status, void* stream) {
  if (!p || !U || !f0 || !work || !status)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm2d_init_populations: null argument");
  if (order < 1 || order > 3)
    return fail(CVLBM_ERR_INVALID_ARG, "init_order must be 1, 2, or 3");
  if (p->nx <= 0 || p->ny <= 0 || !p->active)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm2d_init_populations: bad lattice");
  if ((int64_t)p->nx * p->ny * 36 >= ((int64_t)1 << 31))
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm2d_init_populations: lattice too large");
  cudaStream_t s = (cudaStream_t)stream;
  Ctx2 c = make_ctx(p);
  const int N = c.N;
  double* D = static_cast<double*>(work);                 // [12][N]
  double* Wq = D + 12 * (size_t)N;                        // [24][N]
  auto* gmax = reinterpret_cast<unsigned long long*>(Wq + 24 * (size_t)N);  // [kInitMax]
  cudaMemsetAsync(status, 0, sizeof(int32_t), s);
  cudaMemsetAsync(gmax, 0, sizeof(unsigned long long) * kInitMax, s);
  const int nb = blocks(N, 256);
  if (order != 1) {
    k_init_deriv2<<<nb, 256, 0, s>>>(c, U, order, D, gmax);
    k_init_w2<<<nb, 256, 0, s>>>(c, U, order, D, Wq, gmax, status);
    cv::count_launches(2);
  }
  k_init_f2<<<nb, 256, 0, s>>>(c, U, order, Wq, gmax, f0, status);
  cv::count_launches(1);
  return check_launch("cvlbm2d_init_populations");
}
