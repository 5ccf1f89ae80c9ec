// D2Q4x6 curved-boundary VLBM time step for sm_100a.
//
// Layout: dense SoA, component-major, j fastest: f[(q*6+a)*N + i*ny + j],
// N = nx*ny.  One thread per node (a warp covers 32 consecutive j, so every
// population load and store is a coalesced 256-byte segment) and one thread
// per cut link.
//
// Step pipeline (one launch each, all on one stream):
//   collide  f0 -> fpost, U, u, u*            _collide_masked_kernel
//   sweep    U, u -> u_next, u* (+ anchors)    _local_displacement_bc/relax
//   commit   u <- u_next                       _local_displacement_commit
//   repair   fpost, U <- blend(F, I+grad u)    _local_compatibility_repair
//   stream   f1[q](x) = fpost[q](x - c_q)      _stream_masked_kernel (pull form)
//   links    f1[q_in] at cut nodes             _apply_curved_boundary_links
// Anchors are gathered per node from a CSR of its links in ascending link
// order, the order in which the reference's serial atomics add them.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>
#include <string>

#include "cvlbm_common.cuh"
#include "cvlbm_math.cuh"

using namespace cv;

namespace {

constexpr int kQ2 = 4;
constexpr int kC2 = 6;
constexpr int kMaxLsq2 = 24;
constexpr int kMaxIds2 = 8;

struct Ctx2 {
  cvlbm2d_problem p;
  Mat m;
  int N;
  // per-problem constants of the collision, formed once on the host with the
  // same IEEE operations the kernels would otherwise repeat per node
  double k2c;   // 2 / c
  double ff;    // 0.5 / c
  double hdt;   // 0.5 dt
  double den;   // damping: 1 + 0.5 dt gamma (else 1)
  double dt_om; // dt / omega
  double src_w; // dt (1/omega - 0.5) * 0.25, the source weight of a characteristic row
};

// Boundary time: the step's start time (host value, or the device clock in
// graph mode) plus `offset`, evaluated as the reference's time + 0.5*dt.
__device__ __forceinline__ double time_of(const double* clock, double t, double offset) {
  return (clock ? clock[0] : t) + offset;
}

// ---------------------------------------------------------------------------
// Collision, two_d/curved_boundary_warp.py:1691-1843.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_collide2(Ctx2 c, const double* __restrict__ f0,
                                                  double* __restrict__ fpost,
                                                  double* __restrict__ U, double* __restrict__ u,
                                                  double* __restrict__ ustar,
                                                  int* __restrict__ invalid) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) {
    for (int k = 0; k < kQ2 * kC2; ++k) fpost[(size_t)k * N + n] = 0.0;
    for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = 0.0;
    u[n] = 0.0;
    u[N + n] = 0.0;
    return;
  }
  double f[kQ2 * kC2];
#pragma unroll
  for (int k = 0; k < kQ2 * kC2; ++k) f[k] = f0[(size_t)k * N + n];
  double S[kC2];
#pragma unroll
  for (int a = 0; a < kC2; ++a) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kQ2; ++q) s += f[q * kC2 + a];
    S[a] = s;
  }
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
#pragma unroll
    for (int a = 0; a < kC2; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
  double B[kC2];
#pragma unroll
  for (int a = 0; a < kC2; ++a) B[a] = source_comp(a, p.source_mode, p.source, S);
#pragma unroll
  for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = S[a];
  double ux = ustar[n] + 0.5 * p.dt * S[0];
  double uy = ustar[N + n] + 0.5 * p.dt * S[1];
  u[n] = ux;
  u[N + n] = uy;
  ustar[n] = ux + 0.5 * p.dt * S[0];
  ustar[N + n] = uy + 0.5 * p.dt * S[1];
  double J = S[2] * S[5] - S[3] * S[4];
  if (J <= c.m.jf) *invalid = 1;
  P2 P = piola2(S[2], S[3], S[4], S[5], c.m);
  const double k2c = 2.0 / p.c;
  const double om = p.omega;
  const double sw = p.dt * (2.0 - om) * 0.125;
#pragma unroll
  for (int q = 0; q < kQ2; ++q) {
#pragma unroll
    for (int a = 0; a < kC2; ++a) {
      double fe = feq2(q, a, S, P, k2c);
      double old = f[q * kC2 + a];
      fpost[(size_t)(q * kC2 + a) * N + n] = old + om * (fe - old) + sw * B[a];
    }
  }
}

// ---------------------------------------------------------------------------
// Moment-space collision with ghost damping, two_d/curved_boundary_warp.py
// :1846-2040 (collision_model "mrt_ghost"): the D2Q4 moments m0 (sum), m1,
// m2 (fluxes) relax with omega, the ghost m3 = fE - fN + fW - fS with
// ghost_omega; omega_ghost = omega is the BGK collision.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_collide2_mrt(Ctx2 c, const double* __restrict__ f0,
                                                      double* __restrict__ fpost,
                                                      double* __restrict__ U,
                                                      double* __restrict__ u,
                                                      double* __restrict__ ustar,
                                                      int* __restrict__ invalid) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) {
    for (int k = 0; k < kQ2 * kC2; ++k) fpost[(size_t)k * N + n] = 0.0;
    for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = 0.0;
    u[n] = 0.0;
    u[N + n] = 0.0;
    return;
  }
  double f[kQ2 * kC2];
#pragma unroll
  for (int k = 0; k < kQ2 * kC2; ++k) f[k] = f0[(size_t)k * N + n];
  double S[kC2];
#pragma unroll
  for (int a = 0; a < kC2; ++a) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kQ2; ++q) s += f[q * kC2 + a];
    S[a] = s;
  }
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
#pragma unroll
    for (int a = 0; a < kC2; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
#pragma unroll
  for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = S[a];
  double ux = ustar[n] + 0.5 * p.dt * S[0];
  double uy = ustar[N + n] + 0.5 * p.dt * S[1];
  u[n] = ux;
  u[N + n] = uy;
  ustar[n] = ux + 0.5 * p.dt * S[0];
  ustar[N + n] = uy + 0.5 * p.dt * S[1];
  if (S[2] * S[5] - S[3] * S[4] <= c.m.jf) *invalid = 1;
  const P2 P = piola2(S[2], S[3], S[4], S[5], c.m);
  const double phx[kC2] = {-P.a, -P.c, -S[0], 0.0, -S[1], 0.0};
  const double phy[kC2] = {-P.b, -P.d, 0.0, -S[0], 0.0, -S[1]};
  const double om = p.omega, og = p.ghost_omega;
#pragma unroll
  for (int a = 0; a < kC2; ++a) {
    const double fE = f[a], fN = f[kC2 + a], fW = f[2 * kC2 + a], fS = f[3 * kC2 + a];
    const double m0 = fE + fN + fW + fS;
    const double m1 = fE - fW;
    const double m2 = fN - fS;
    const double m3 = fE - fN + fW - fS;
    const double b = source_comp(a, p.source_mode, p.source, S);
    const double m0p = m0 + om * (S[a] - m0) + p.dt * (2.0 - om) * 0.5 * b;
    const double m1p = m1 + om * (phx[a] / p.c - m1);
    const double m2p = m2 + om * (phy[a] / p.c - m2);
    const double m3p = (1.0 - og) * m3;
    fpost[(size_t)(0 * kC2 + a) * N + n] = 0.25 * (m0p + m3p + 2.0 * m1p);
    fpost[(size_t)(1 * kC2 + a) * N + n] = 0.25 * (m0p - m3p + 2.0 * m2p);
    fpost[(size_t)(2 * kC2 + a) * N + n] = 0.25 * (m0p + m3p - 2.0 * m1p);
    fpost[(size_t)(3 * kC2 + a) * N + n] = 0.25 * (m0p - m3p - 2.0 * m2p);
  }
}

// Kinetic ghost filter, two_d/curved_boundary_warp.py:3101-3124: the ghost
// moment of each component damped by `strength`, U and the fluxes unchanged.
__global__ void __launch_bounds__(256) k_ghost_filter2(Ctx2 c, double* __restrict__ f) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N || c.p.active[n] == 0) return;
  const double str = c.p.kinetic_filter;
  if (str <= 0.0) return;
#pragma unroll
  for (int a = 0; a < kC2; ++a) {
    double* fE = f + (size_t)(0 * kC2 + a) * N + n;
    double* fN = f + (size_t)(1 * kC2 + a) * N + n;
    double* fW = f + (size_t)(2 * kC2 + a) * N + n;
    double* fS = f + (size_t)(3 * kC2 + a) * N + n;
    const double m3 = *fE - *fN + *fW - *fS;
    const double delta = -str * m3;
    const double quarter = 0.25 * delta;
    *fE = *fE + quarter;
    *fW = *fW + quarter;
    *fN = *fN - quarter;
    *fS = *fS - quarter;
  }
}

// ---------------------------------------------------------------------------
// Local displacement sweep, two_d/curved_boundary_warp.py:3275-3490, with the
// link anchors (:3287-3417) gathered per node.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void anchor2(const Ctx2& c, const double* U, int ell, int n, int i, int j,
                                        double time, double& diag, double& r0, double& r1) {
  const cvlbm2d_problem& p = c.p;
  int bid = p.link_bid[ell];
  if (p.disp_bid >= 0) {
    if (bid != p.disp_bid) return;
  } else if (p.bc_kind[bid] != kDirichlet) {
    return;
  }
  const double* pp = p.bc_params + bid * 8;
  int mode = p.bc_mode[bid];
  double xb = p.link_xb[ell], yb = p.link_yb[ell];
  double nxb = p.link_nx[ell], nyb = p.link_ny[ell];
  double ub0 = 0.0, ub1 = 0.0;
  if (mode == 1) {
    ub0 = time * value2(0, mode, pp, xb, yb, nxb, nyb, 0.0);
    ub1 = time * value2(1, mode, pp, xb, yb, nxb, nyb, 0.0);
  } else if (mode == 6) {
    double at = time;
    if (pp[6] > 0.0 && at > pp[6]) at = pp[6];
    ub0 = at * value2(0, mode, pp, xb, yb, nxb, nyb, 0.0);
    ub1 = at * value2(1, mode, pp, xb, yb, nxb, nyb, 0.0);
  }
  const int N = c.N;
  double dbx = xb - ((double)i + 0.5) * p.dx;
  double dby = yb - ((double)j + 0.5) * p.dy;
  double tx = ub0 - ((U[2 * N + n] - 1.0) * dbx + U[3 * N + n] * dby);
  double ty = ub1 - (U[4 * N + n] * dbx + (U[5 * N + n] - 1.0) * dby);
  double w2 = p.weight * p.weight;
  diag = diag + w2;
  r0 = r0 + w2 * tx;
  r1 = r1 + w2 * ty;
}

__global__ void __launch_bounds__(256) k_sweep2(Ctx2 c, const double* __restrict__ U,
                                                const double* __restrict__ u,
                                                double* __restrict__ unext,
                                                double* __restrict__ ustar, const double* clock,
                                                double time_host) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) {
    unext[n] = 0.0;
    unext[N + n] = 0.0;
    return;
  }
  const int nx = p.nx, ny = p.ny;
  const int i = n / ny, j = n - i * ny;
  double diag = 0.0, rx = 0.0, ry = 0.0;
  const double time = time_of(clock, time_host, 0.5 * p.dt);
  for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k)
    anchor2(c, U, p.node_link_list[k], n, i, j, time, diag, rx, ry);
  const double* U2 = U + 2 * N;
  const double* U3 = U + 3 * N;
  const double* U4 = U + 4 * N;
  const double* U5 = U + 5 * N;
  const double hx = 0.5 * p.dx, hy = 0.5 * p.dy;
  if (i + 1 < nx && p.active[n + ny] != 0) {
    int m = n + ny;
    double gx = hx * ((U2[n] - 1.0) + (U2[m] - 1.0));
    double gy = hx * (U4[n] + U4[m]);
    rx += u[m] - gx;
    ry += u[N + m] - gy;
    diag += 1.0;
  }
  if (i > 0 && p.active[n - ny] != 0) {
    int m = n - ny;
    double gx = hx * ((U2[m] - 1.0) + (U2[n] - 1.0));
    double gy = hx * (U4[m] + U4[n]);
    rx += u[m] + gx;
    ry += u[N + m] + gy;
    diag += 1.0;
  }
  if (j + 1 < ny && p.active[n + 1] != 0) {
    int m = n + 1;
    double gx = hy * (U3[n] + U3[m]);
    double gy = hy * ((U5[n] - 1.0) + (U5[m] - 1.0));
    rx += u[m] - gx;
    ry += u[N + m] - gy;
    diag += 1.0;
  }
  if (j > 0 && p.active[n - 1] != 0) {
    int m = n - 1;
    double gx = hy * (U3[m] + U3[n]);
    double gy = hy * ((U5[m] - 1.0) + (U5[n] - 1.0));
    rx += u[m] + gx;
    ry += u[N + m] + gy;
    diag += 1.0;
  }
  double u0 = u[n], u1 = u[N + n];
  double n0 = u0, n1 = u1;
  if (diag > 0.0) {
    n0 = u0 + p.relax * (rx / diag - u0);
    n1 = u1 + p.relax * (ry / diag - u1);
  }
  unext[n] = n0;
  unext[N + n] = n1;
  // commit (two_d/curved_boundary_warp.py:3493-3518): u* follows the same shift
  ustar[n] = ustar[n] + (n0 - u0);
  ustar[N + n] = ustar[N + n] + (n1 - u1);
}

__global__ void k_commit2(int N2, const double* __restrict__ src, double* __restrict__ dst) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < N2) dst[n] = src[n];
}

// ---------------------------------------------------------------------------
// Local deformation-gradient repair, two_d/curved_boundary_warp.py:3213-3272
// (_local_dudx/_local_dudy) and :3521-3615.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dudx2(const double* uc, const int* act, int n, int i, int nx,
                                        int stride, double h) {
  // stride = ny for d/dx, 1 for d/dy; i is the index along that axis
  bool am = i > 0 && act[n - stride] != 0;
  bool ap = i + 1 < nx && act[n + stride] != 0;
  if (am && ap) return (uc[n + stride] - uc[n - stride]) / (2.0 * h);
  if (ap) {
    if (i + 2 < nx && act[n + 2 * stride] != 0)
      return (-3.0 * uc[n] + 4.0 * uc[n + stride] - uc[n + 2 * stride]) / (2.0 * h);
    return (uc[n + stride] - uc[n]) / h;
  }
  if (am) {
    if (i > 1 && act[n - 2 * stride] != 0)
      return (3.0 * uc[n] - 4.0 * uc[n - stride] + uc[n - 2 * stride]) / (2.0 * h);
    return (uc[n] - uc[n - stride]) / h;
  }
  return 0.0;
}

__global__ void __launch_bounds__(256) k_repair2(Ctx2 c, double* __restrict__ f,
                                                 double* __restrict__ U,
                                                 const double* __restrict__ u) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  const int* act = p.active;
  if (act[n] == 0) return;
  const int nx = p.nx, ny = p.ny;
  const int i = n / ny, j = n - i * ny;
  if (p.interior_only != 0) {
    if (i == 0 || i + 1 >= nx || j == 0 || j + 1 >= ny) return;
    if (act[n - ny] == 0 || act[n + ny] == 0 || act[n - 1] == 0 || act[n + 1] == 0) return;
  }
  double o11 = U[2 * N + n], o12 = U[3 * N + n], o21 = U[4 * N + n], o22 = U[5 * N + n];
  double t11 = 1.0 + dudx2(u, act, n, i, nx, ny, p.dx);
  double t12 = dudx2(u, act, n, j, ny, 1, p.dy);
  double t21 = dudx2(u + N, act, n, i, nx, ny, p.dx);
  double t22 = 1.0 + dudx2(u + N, act, n, j, ny, 1, p.dy);
  double alpha = fmax(0.0, fmin(1.0, p.blend));
  double n11 = o11, n12 = o12, n21 = o21, n22 = o22;
  for (int g = 0; g < 10; ++g) {
    n11 = o11 + alpha * (t11 - o11);
    n12 = o12 + alpha * (t12 - o12);
    n21 = o21 + alpha * (t21 - o21);
    n22 = o22 + alpha * (t22 - o22);
    if (n11 * n22 - n12 * n21 > c.m.jf) break;
    alpha = 0.5 * alpha;
  }
  P2 Po = piola2(o11, o12, o21, o22, c.m);
  P2 Pn = piola2(n11, n12, n21, n22, c.m);
  double dP11 = Pn.a - Po.a, dP12 = Pn.b - Po.b, dP21 = Pn.c - Po.c, dP22 = Pn.d - Po.d;
  const double ff = 0.5 / p.c;
  const double qt = 0.25;
#pragma unroll
  for (int q = 0; q < kQ2; ++q) {
    double cx = (double)cx2(q), cy = (double)cy2(q);
    size_t b = (size_t)(q * kC2) * N + n;
    f[b] = f[b] - ff * (cx * dP11 + cy * dP12);
    f[b + N] = f[b + N] - ff * (cx * dP21 + cy * dP22);
    f[b + 2 * (size_t)N] = f[b + 2 * (size_t)N] + qt * (n11 - o11);
    f[b + 3 * (size_t)N] = f[b + 3 * (size_t)N] + qt * (n12 - o12);
    f[b + 4 * (size_t)N] = f[b + 4 * (size_t)N] + qt * (n21 - o21);
    f[b + 5 * (size_t)N] = f[b + 5 * (size_t)N] + qt * (n22 - o22);
  }
  U[2 * N + n] = n11;
  U[3 * N + n] = n12;
  U[4 * N + n] = n21;
  U[5 * N + n] = n22;
}

// ---------------------------------------------------------------------------
// Streaming in pull form, equivalent to the push of
// two_d/curved_boundary_warp.py:2043-2060 after the clear of f1.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_stream2(Ctx2 c, const double* __restrict__ fpost,
                                                 double* __restrict__ f1) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  const int nx = p.nx, ny = p.ny;
  const int i = n / ny, j = n - i * ny;
  if (p.active[n] == 0) {
    for (int k = 0; k < kQ2 * kC2; ++k) f1[(size_t)k * N + n] = 0.0;
    return;
  }
#pragma unroll
  for (int q = 0; q < kQ2; ++q) {
    int si = i - cx2(q), sj = j - cy2(q);
    bool ok = si >= 0 && si < nx && sj >= 0 && sj < ny && p.active[si * ny + sj] != 0;
    int s = si * ny + sj;
#pragma unroll
    for (int a = 0; a < kC2; ++a) {
      size_t k = (size_t)(q * kC2 + a) * N;
      f1[k + n] = ok ? fpost[k + s] : 0.0;
    }
  }
}

// ---------------------------------------------------------------------------
// Cut-link reconstruction, two_d/curved_boundary_warp.py:2063-3098, for the
// bfl / lsq_bfl / compat_bfl / local_char2 / local_f / local_f_bfl closures.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double interp_link(const double* Uc, const int* act, int i, int j,
                                              int qo, double s, int nx, int ny) {
  // two_d/curved_boundary_warp.py:1443-1480 (_interp_U_link)
  double v0 = Uc[i * ny + j];
  int i1 = i - cx2(qo), j1 = j - cy2(qo);
  if (i1 >= 0 && i1 < nx && j1 >= 0 && j1 < ny && act[i1 * ny + j1] != 0) {
    double v1 = Uc[i1 * ny + j1];
    int i2 = i - 2 * cx2(qo), j2 = j - 2 * cy2(qo);
    if (i2 >= 0 && i2 < nx && j2 >= 0 && j2 < ny && act[i2 * ny + j2] != 0) {
      double v2 = Uc[i2 * ny + j2];
      double l0 = 0.5 * (s + 1.0) * (s + 2.0);
      double l1 = -s * (s + 2.0);
      double l2 = 0.5 * s * (s + 1.0);
      return l0 * v0 + l1 * v1 + l2 * v2;
    }
    return (s + 1.0) * v0 - s * v1;
  }
  return v0;
}


}  // namespace

#include "cvlbm2d_fused.cuh"
#include "cvlbm2d_split.cuh"

namespace {

// ---------------------------------------------------------------------------
// Field refresh, two_d/curved_boundary_warp.py:3127-3210.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_refresh2(Ctx2 c, const double* __restrict__ f0,
                                                  double* __restrict__ U, double* __restrict__ u,
                                                  const double* __restrict__ ustar,
                                                  double* __restrict__ Pf,
                                                  double* __restrict__ sg,
                                                  int* __restrict__ invalid) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) {
    for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = 0.0;
    u[n] = 0.0;
    u[N + n] = 0.0;
    for (int a = 0; a < 4; ++a) {
      Pf[(size_t)a * N + n] = 0.0;
      sg[(size_t)a * N + n] = 0.0;
    }
    return;
  }
  double S[kC2];
  for (int a = 0; a < kC2; ++a) {
    double s = 0.0;
    for (int q = 0; q < kQ2; ++q) s += f0[(size_t)(q * kC2 + a) * N + n];
    S[a] = s;
  }
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
    for (int a = 0; a < kC2; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
  for (int a = 0; a < kC2; ++a) U[(size_t)a * N + n] = S[a];
  u[n] = ustar[n] + 0.5 * p.dt * S[0];
  u[N + n] = ustar[N + n] + 0.5 * p.dt * S[1];
  double J = S[2] * S[5] - S[3] * S[4];
  if (J <= c.m.jf) *invalid = 1;
  double Js = clamp_j(J, c.m.jf);
  P2 P = piola2(S[2], S[3], S[4], S[5], c.m);
  Pf[n] = P.a;
  Pf[(size_t)N + n] = P.b;
  Pf[2 * (size_t)N + n] = P.c;
  Pf[3 * (size_t)N + n] = P.d;
  sg[n] = (P.a * S[2] + P.b * S[3]) / Js;
  sg[(size_t)N + n] = (P.a * S[4] + P.b * S[5]) / Js;
  sg[2 * (size_t)N + n] = (P.c * S[2] + P.d * S[3]) / Js;
  sg[3 * (size_t)N + n] = (P.c * S[4] + P.d * S[5]) / Js;
}

// P and sigma from U, as stored by the collision (two_d/curved_boundary_warp.py:1791-1803)
__global__ void __launch_bounds__(256) k_stress2(Ctx2 c, const double* __restrict__ U,
                                                 double* __restrict__ Pf,
                                                 double* __restrict__ sg) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N || c.p.active[n] == 0) return;
  double F11 = U[2 * (size_t)N + n], F12 = U[3 * (size_t)N + n];
  double F21 = U[4 * (size_t)N + n], F22 = U[5 * (size_t)N + n];
  double Js = clamp_j(F11 * F22 - F12 * F21, c.m.jf);
  P2 P = piola2(F11, F12, F21, F22, c.m);
  Pf[n] = P.a;
  Pf[(size_t)N + n] = P.b;
  Pf[2 * (size_t)N + n] = P.c;
  Pf[3 * (size_t)N + n] = P.d;
  sg[n] = (P.a * F11 + P.b * F12) / Js;
  sg[(size_t)N + n] = (P.a * F21 + P.b * F22) / Js;
  sg[2 * (size_t)N + n] = (P.c * F11 + P.d * F12) / Js;
  sg[3 * (size_t)N + n] = (P.c * F21 + P.d * F22) / Js;
}

__global__ void k_tick(const double* clock, double* next, double dt) { next[0] = clock[0] + dt; }

__global__ void k_zero_flag(int* flag) { *flag = 0; }

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

bool due(int interval, long long step) { return interval > 0 && step % interval == 0; }

int check_problem(const cvlbm2d_problem* p, const cvlbm2d_fields* f) {
  if (!p || !f) return fail(CVLBM_ERR_INVALID_ARG, "null problem or fields");
  if (p->nx < 1 || p->ny < 1) return fail(CVLBM_ERR_INVALID_ARG, "empty lattice");
  if ((long long)p->nx * p->ny > 0x7fffffffLL / 24)
    return fail(CVLBM_ERR_INVALID_ARG, "lattice too large for 32-bit node indexing");
  if (!f->f0 || !f->f1 || !f->fpost || !f->U || !f->u || !f->u_next || !f->u_star ||
      !f->invalid)
    return fail(CVLBM_ERR_INVALID_ARG, "missing field buffer");
  if (!p->active || !p->node_link_start || !p->bc_kind || !p->bc_mode || !p->bc_params)
    return fail(CVLBM_ERR_INVALID_ARG, "missing geometry table");
  switch (p->recon) {
    case 0: case 2: case 9: case 11: case 12: case 13: break;
    default: return fail(CVLBM_ERR_UNSUPPORTED, "unsupported 2-D boundary reconstruction id");
  }
  if (p->disp_interval > 0 && (p->disp_sweeps < 1 || p->disp_sweeps > 8))
    return fail(CVLBM_ERR_INVALID_ARG, "displacement sweeps must be in [1,8]");
  return CVLBM_OK;
}

Ctx2 make_ctx(const cvlbm2d_problem* p) {
  Ctx2 c;
  c.p = *p;
  c.m = Mat{p->mat.model, p->mat.lam, p->mat.mu, p->mat.p0, p->mat.p1, p->mat.p2, p->mat.j_floor};
  c.N = p->nx * p->ny;
  c.k2c = 2.0 / p->c;
  c.ff = 0.5 / p->c;
  c.hdt = 0.5 * p->dt;
  c.den = p->source_mode == kSrcDamping ? 1.0 + c.hdt * p->source[0] : 1.0;
  c.dt_om = p->dt / p->omega;
  c.src_w = p->dt * (1.0 / p->omega - 0.5) * 0.25;
  return c;
}

// The link kernel is a set of long dependent chains (one per link) that
// gates the next step: it is launched at the device's highest priority, so
// that with the inner tiles of the next step in flight on another stream its
// blocks are placed first (graphs keep the priority, see capture_graph).
int link_priority() {
  static int prio = [] {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) return 0;
    return greatest;
  }();
  return prio;
}

void launch_links(const Ctx2& c, const double* src, double* dst, const double* U,
                  const double* u, const double* clock, double t, double offset,
                  cudaStream_t s, int fused = 0, const double* scratch = nullptr,
                  const int32_t* partner = nullptr, double* clock_next = nullptr) {
  if (c.p.n_links <= 0) return;
  const int per = kLinksPerBlock2;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks(c.p.n_links, per));
  cfg.blockDim = dim3(kLinkThreads2);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = link_priority();
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // builds for the neo-Hooke law with the local_f closure and each Neumann
  // solver hold only that path's code (fewer instruction-cache misses along
  // the link's chain); other problems take the generic builds
  auto kern = k_links2g<-1>;
  if (c.m.model == kMatNeoHooke) {
    kern = k_links2g<kMatNeoHooke>;
    if (c.p.recon == 12 && c.p.normal_solver == kSolverFD)
      kern = k_links2g<kMatNeoHooke, 12, kSolverFD>;
    else if (c.p.recon == 12 && c.p.normal_solver == kSolverAcoustic)
      kern = k_links2g<kMatNeoHooke, 12, kSolverAcoustic>;
    else if (c.p.recon == 12 && c.p.normal_solver == kSolverEnergy)
      kern = k_links2g<kMatNeoHooke, 12, kSolverEnergy>;
  }
  const int tk = link_timer_begin(s);
  cudaLaunchKernelEx(&cfg, kern, c, src, dst, U, u, clock, t, offset, fused, scratch, partner,
                     clock_next);
  link_timer_end(tk, s);
  cv::count_launches(1);
}

// Second stream and the two events of the overlapped fused step, one set per
// device and caller stream (runs on one stream are ordered, so they can share
// a set; runs on different streams get different sets), created on first use
// and kept for the life of the process.
struct Overlap2 {
  cudaStream_t inner;          // inner tiles
  cudaEvent_t inner_done;      // last inner-tile launch issued
  cudaEvent_t boundary_done;   // last boundary-tile launch issued
};
std::mutex g_overlap_mu;
std::map<std::pair<int, cudaStream_t>, Overlap2> g_overlap;  // (device, caller stream)

Overlap2* overlap_resources(cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_overlap_mu);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  const auto key = std::make_pair(dev, s);  // the default stream's handle is shared by devices
  auto it = g_overlap.find(key);
  if (it != g_overlap.end()) return &it->second;
  Overlap2 o{};
  if (cudaStreamCreateWithFlags(&o.inner, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&o.inner_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&o.boundary_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaStreamDestroy(o.inner);
    return nullptr;
  }
  return &(g_overlap[key] = o);
}

using FusedFn2 = void (*)(Ctx2, Fused2, const double*, double*, double*, double*, const double*,
                          double*, int*, const double*, double, int, int, const double*);
using MomFn2 = void (*)(Ctx2, Fused2, const double*, const double*, double*);

struct FusedLaunch2 {
  FusedFn2 fn;
  int threads;
  size_t smem;
  int tile_i;
  MomFn2 mom;  // PRE form: moments kernel launched before the tile kernel, else null
};

// Compiled tile variants: (tile rows, resident blocks per SM, PRE).  The tile
// list in the problem must have been built for the variant's tile height.
// Variant 5 selects the split form (cvlbm2d_split.cuh) instead of a tile
// shape; variants 6 and 7 are the PRE form (moments of every active node
// written once per step by k_mom2 into fields->fpost, halo moments read from
// there instead of recomputed), which runs without the link overlap;
// variants 8-10 keep the owned nodes' populations in shared memory from the
// moments to the collision (STAGE) instead of reloading them.
constexpr int kSplitVariant = 5;
constexpr int kMaxVariant = 10;

FusedLaunch2 fused_variant(int v) {
  switch (v) {
    case 1: return {k_fused2<8, 2, false>, kTX * 8, fused_smem2<8>(), 8, nullptr};
    case 2: return {k_fused2<8, 3, false>, kTX * 8, fused_smem2<8>(), 8, nullptr};
    case 3: return {k_fused2<16, 2, false>, kTX * 16, fused_smem2<16>(), 16, nullptr};
    case 4: return {k_fused2<4, 4, false>, kTX * 4, fused_smem2<4>(), 4, nullptr};
    case kSplitVariant: return {nullptr, 0, 0, 16, nullptr};  // split kernels, no tiles used
    case 6: return {k_fused2<16, 1, true>, kTX * 16, fused_smem2<16>(), 16, k_mom2<16>};
    case 7: return {k_fused2<8, 3, true>, kTX * 8, fused_smem2<8>(), 8, k_mom2<8>};
    case 8: return {k_fused2<8, 2, false, true>, kTX * 8, fused_smem2<8, true>(), 8, nullptr};
    case 9: return {k_fused2<16, 1, false, true>, kTX * 16, fused_smem2<16, true>(), 16, nullptr};
    case 10: return {k_fused2<4, 4, false, true>, kTX * 4, fused_smem2<4, true>(), 4, nullptr};
    default: return {k_fused2<16, 1, false>, kTX * 16, fused_smem2<16>(), 16, nullptr};
  }
}

bool fused_ok(const cvlbm2d_problem* p, const cvlbm2d_fields* f) {
  const FusedLaunch2 fl = fused_variant(p->tile_variant);
  return p->tiles && p->need_fields && p->link_partner && f->link_scratch && p->lsq_node &&
         p->disp_sweeps <= 1 && fl.tile_i == p->tile_i && (!fl.mom || f->fpost) &&
         p->collision_model == 0 && !(p->kinetic_filter > 0.0) &&
         // the fused node kernel indexes populations with 32-bit offsets
         24LL * p->nx * p->ny < 2147483647LL;
}

}  // namespace

extern "C" int cvlbm2d_run(const cvlbm2d_problem* p, cvlbm2d_fields* f, double time0,
                           int64_t step0, int32_t nsteps, int32_t graph_mode, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (nsteps < 0) return fail(CVLBM_ERR_INVALID_ARG, "negative step count");
  if (graph_mode && !f->clock) return fail(CVLBM_ERR_INVALID_ARG, "graph mode needs a clock");
  cudaStream_t s = (cudaStream_t)stream;
  Ctx2 c = make_ctx(p);
  const int N = c.N;
  const unsigned nb = blocks(N, 256);
  k_zero_flag<<<1, 1, 0, s>>>(f->invalid); cv::count_launches(1);
  double t = time0;
  const bool fused = fused_ok(p, f);
  FusedLaunch2 fl = fused_variant(p->tile_variant);
  const bool split = fused && p->tile_variant == kSplitVariant;
  if (fused && !split)
    cudaFuncSetAttribute(fl.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fl.smem);
  // the fused kernel reads u* in the halo of its tile, so it ping-pongs
  // between u_star and u_next; an odd count ends with one copy back
  double* us_cur = f->u_star;
  double* us_nxt = f->u_next;
  Overlap2* ov = nullptr;
  if (fused && !split && !fl.mom && p->overlap && p->n_tiles_inner > 0 &&
      p->n_tiles_inner < p->n_tiles && nsteps > 0) {
    ov = overlap_resources(s);
    if (ov) {
      cudaEventRecord(ov->boundary_done, s);  // the inner stream starts after prior work
      cudaStreamWaitEvent(ov->inner, ov->boundary_done, 0);
    }
  }
  for (int k = 0; k < nsteps; ++k) {
    const long long step = step0 + k;
    const int sweep = due(p->disp_interval, step), repair = due(p->rep_interval, step);
    // graph mode: step k reads the device time from clock[k&1] and the link
    // kernel writes clock[(k+1)&1] (no separate tick launch)
    const double* clock = graph_mode ? f->clock + (k & 1) : nullptr;
    double* clock_next = graph_mode ? f->clock + ((k + 1) & 1) : nullptr;
    if (split) {
      int tk = timer_begin(s);
      k2s_moments<<<blocks(N, 256), 256, 0, s>>>(c, f->f0, f->U, sweep ? f->u_next : f->u,
                                                 f->u_star, f->invalid, sweep);
      cv::count_launches(1);
      if (sweep) {
        k2s_sweep<<<blocks(N, 256), 256, 0, s>>>(c, f->U, f->u_next, f->u, f->u_star, clock, t);
        cv::count_launches(1);
      }
      k2s_collide<<<blocks(N, 128), 128, 0, s>>>(c, f->f0, f->f1, f->U, f->u, p->need_fields,
                                                 f->link_scratch, repair, k == nsteps - 1);
      cv::count_launches(1);
      timer_end(tk, s);
      launch_links(c, f->f1, f->f1, f->U, f->u, clock, t, 0.5 * p->dt, s, 1, f->link_scratch,
                   p->link_partner, clock_next);
    } else if (ov) {
      // step k: boundary tiles after the links of step k-1 (stream order) and
      // the inner tiles of step k-1; inner tiles after the boundary tiles of
      // step k-1 only, so they run while the link kernel of step k-1 does.
      // The inner tiles hold no cut-link node in their halo and no node a
      // link reads, so neither kernel touches what the other one reads.
      const int n_in = p->n_tiles_inner, n_bd = p->n_tiles - n_in;
      Fused2 fz_in{p->tiles, n_in, p->tiles_j, p->need_fields, p->link_partner,
                   f->link_scratch, k == nsteps - 1};
      Fused2 fz_bd{p->tiles + n_in, n_bd, p->tiles_j, p->need_fields, p->link_partner,
                   f->link_scratch, k == nsteps - 1};
      if (k > 0) {
        cudaStreamWaitEvent(s, ov->inner_done, 0);
        cudaStreamWaitEvent(ov->inner, ov->boundary_done, 0);
      }
      fl.fn<<<n_bd, fl.threads, fl.smem, s>>>(c, fz_bd, f->f0, f->f1, f->U, f->u, us_cur,
                                              us_nxt, f->invalid, clock, t, sweep, repair,
                                              nullptr);
      cudaEventRecord(ov->boundary_done, s);
      // inner tiles read no time (they have no cut-point anchors)
      fl.fn<<<n_in, fl.threads, fl.smem, ov->inner>>>(c, fz_in, f->f0, f->f1, f->U, f->u, us_cur,
                                                      us_nxt, f->invalid, nullptr, t, sweep,
                                                      repair, nullptr);
      cudaEventRecord(ov->inner_done, ov->inner);
      cv::count_launches(2);
      double* us = us_cur;
      us_cur = us_nxt;
      us_nxt = us;
      launch_links(c, f->f1, f->f1, f->U, f->u, clock, t, 0.5 * p->dt, s, 1, f->link_scratch,
                   p->link_partner, clock_next);
    } else if (fused) {
      Fused2 fz{p->tiles, p->n_tiles, p->tiles_j, p->need_fields, p->link_partner,
                f->link_scratch, k == nsteps - 1};
      int tk = timer_begin(s);
      if (p->n_tiles > 0) {
        if (fl.mom) {
          fl.mom<<<p->n_tiles, fl.threads, 0, s>>>(c, fz, f->f0, us_cur, f->fpost);
          cv::count_launches(1);
        }
        fl.fn<<<p->n_tiles, fl.threads, fl.smem, s>>>(c, fz, f->f0, f->f1, f->U, f->u, us_cur,
                                                      us_nxt, f->invalid, clock, t, sweep, repair,
                                                      f->fpost);
        cv::count_launches(1);
      }
      double* us = us_cur;
      us_cur = us_nxt;
      us_nxt = us;
      timer_end(tk, s);
      launch_links(c, f->f1, f->f1, f->U, f->u, clock, t, 0.5 * p->dt, s, 1, f->link_scratch,
                   p->link_partner, clock_next);
    } else {
      int tk = timer_begin(s);
      if (p->collision_model == 1)
        k_collide2_mrt<<<nb, 256, 0, s>>>(c, f->f0, f->fpost, f->U, f->u, f->u_star, f->invalid);
      else
        k_collide2<<<nb, 256, 0, s>>>(c, f->f0, f->fpost, f->U, f->u, f->u_star, f->invalid);
      cv::count_launches(1);
      timer_end(tk, s);
      if (sweep) {
        for (int sw = 0; sw < p->disp_sweeps; ++sw) {
          k_sweep2<<<nb, 256, 0, s>>>(c, f->U, f->u, f->u_next, f->u_star, clock, t);
          cv::count_launches(1);
          k_commit2<<<blocks(2LL * N, 256), 256, 0, s>>>(2 * N, f->u_next, f->u);
          cv::count_launches(1);
        }
      }
      if (repair) {
        k_repair2<<<nb, 256, 0, s>>>(c, f->fpost, f->U, f->u);
        cv::count_launches(1);
      }
      k_stream2<<<nb, 256, 0, s>>>(c, f->fpost, f->f1);
      cv::count_launches(1);
      launch_links(c, f->fpost, f->f1, f->U, f->u, clock, t, 0.5 * p->dt, s, 0, nullptr, nullptr,
                   clock_next);
      if (p->kinetic_filter > 0.0) {
        k_ghost_filter2<<<nb, 256, 0, s>>>(c, f->f1);
        cv::count_launches(1);
      }
    }
    if (graph_mode && p->n_links <= 0) {
      k_tick<<<1, 1, 0, s>>>(f->clock + (k & 1), f->clock + ((k + 1) & 1), p->dt);
      cv::count_launches(1);
    }
    double* tmp = f->f0;
    f->f0 = f->f1;
    f->f1 = tmp;
    t += p->dt;
  }
  if (ov) cudaStreamWaitEvent(s, ov->inner_done, 0);  // join: the run ends on `s`
  if (us_cur != f->u_star)
    cudaMemcpyAsync(f->u_star, us_cur, sizeof(double) * 2 * (size_t)N, cudaMemcpyDeviceToDevice, s);
  return check_launch("cvlbm2d_run");
}

extern "C" int cvlbm2d_kinetic_filter(const cvlbm2d_problem* p, cvlbm2d_fields* f,
                                      void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  Ctx2 c = make_ctx(p);
  if (!(p->kinetic_filter > 0.0) || c.N == 0) return CVLBM_OK;
  k_ghost_filter2<<<blocks(c.N, 256), 256, 0, (cudaStream_t)stream>>>(c, f->f0);
  cv::count_launches(1);
  return check_launch("cvlbm2d_kinetic_filter");
}

extern "C" int cvlbm2d_apply_boundary(const cvlbm2d_problem* p, cvlbm2d_fields* f, double t,
                                      int32_t in_place, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx2 c = make_ctx(p);
  if (p->n_links == 0) return CVLBM_OK;
  if (in_place) {
    // opposing cut links must read one frozen state
    cudaMemcpyAsync(f->fpost, f->f0, sizeof(double) * 24 * (size_t)c.N, cudaMemcpyDeviceToDevice,
                    s);
    launch_links(c, f->fpost, f->f0, f->U, f->u, nullptr, t, 0.0, s);
  } else {
    launch_links(c, f->fpost, f->f1, f->U, f->u, nullptr, t, 0.0, s);
  }
  return check_launch("cvlbm2d_apply_boundary");
}

extern "C" int cvlbm2d_refresh(const cvlbm2d_problem* p, cvlbm2d_fields* f, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (!f->P || !f->sigma) return fail(CVLBM_ERR_INVALID_ARG, "missing stress buffers");
  cudaStream_t s = (cudaStream_t)stream;
  Ctx2 c = make_ctx(p);
  k_zero_flag<<<1, 1, 0, s>>>(f->invalid); cv::count_launches(1);
  k_refresh2<<<blocks(c.N, 256), 256, 0, s>>>(c, f->f0, f->U, f->u, f->u_star, f->P, f->sigma,
                                               f->invalid); cv::count_launches(1);
  return check_launch("cvlbm2d_refresh");
}

extern "C" int cvlbm2d_tile_variant(int32_t v) {
  if (v < 0 || v > kMaxVariant) return 0;
  return fused_variant(v).tile_i;
}

extern "C" int cvlbm2d_stress(const cvlbm2d_problem* p, cvlbm2d_fields* f, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (!f->P || !f->sigma) return fail(CVLBM_ERR_INVALID_ARG, "missing stress buffers");
  Ctx2 c = make_ctx(p);
  k_stress2<<<blocks(c.N, 256), 256, 0, (cudaStream_t)stream>>>(c, f->U, f->P, f->sigma); cv::count_launches(1);
  return check_launch("cvlbm2d_stress");
}

extern "C" int cvlbm2d_graph_create(const cvlbm2d_problem* p, const cvlbm2d_fields* f,
                                    int64_t step0, int32_t nsteps, cvlbm_graph** out) {
  if (!out) return fail(CVLBM_ERR_INVALID_ARG, "null output");
  if (nsteps <= 0 || (nsteps & 1)) return fail(CVLBM_ERR_INVALID_ARG, "nsteps must be even");
  cvlbm2d_fields local = *f;
  return capture_graph(
      [&](cudaStream_t s) { return cvlbm2d_run(p, &local, 0.0, step0, nsteps, 1, s); }, out);
}

// ---------------------------------------------------------------------------
// Allocation-free step: link scratch in a fixed array compiled into the library.
//
// The fused step parks the post-collision populations that leave through cut
// links in a per-link scratch buffer (6 doubles per link) that cvlbm2d_run
// takes from the caller.  Some hosts cannot hand one over: an application that
// has carved all device memory into its own pool before this library is
// loaded, or a fixed-rate driver loop that must not enter an allocator between
// steps (cudaMalloc/cudaFree may synchronise the whole device).  For them the
// scratch lives here instead, in a static device array sized for
// CVLBM2D_STATIC_SCRATCH_MAX_LINKS cut links (6 * 16384 doubles = 768 KiB per
// device).  Nothing is allocated on any call: the array's address is looked
// up once per device context (cudaGetSymbolAddress) and cached.
//
// Contents: no element has to start at zero.  Within every step the node
// kernel writes the entry of each cut link before the link kernel reads it.
// One array per device is shared by all callers: two calls in flight at the
// same time on one device (different streams or threads) overwrite each
// other's scratch and give wrong results; the caller serialises them.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) double g_static_link_scratch[6 * CVLBM2D_STATIC_SCRATCH_MAX_LINKS];

// The current context, through the runtime's driver entry point (the library
// does not link the driver API); null when that entry point is unavailable.
typedef int (*CtxGetCurrentFn)(void**);
void* current_context() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrentFn) nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kMaxDevices] = {};
void* g_static_ctx[kMaxDevices] = {};

// Address of g_static_link_scratch on the current device.  It is looked up
// (cudaGetSymbolAddress) on the first call on a device and kept for that
// device's context; a new context (after cudaDeviceReset the runtime creates
// one and loads the module again) gets a fresh lookup.
int static_scratch(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(CVLBM_ERR_CUDA, (std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
  if (dev < 0 || dev >= kMaxDevices) return fail(CVLBM_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mu);
  void* ctx = current_context();
  if (!g_static_ptr[dev] || !ctx || ctx != g_static_ctx[dev]) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_static_link_scratch);
    if (e != cudaSuccess || !addr)
      return fail(CVLBM_ERR_CUDA, (std::string("cudaGetSymbolAddress(static link scratch): ") +
                                   cudaGetErrorString(e)).c_str());
    g_static_ptr[dev] = static_cast<double*>(addr);
    g_static_ctx[dev] = current_context();  // the lookup made the context current
  }
  *out = g_static_ptr[dev];
  return CVLBM_OK;
}

}  // namespace

extern "C" int cvlbm2d_run_static_scratch(const cvlbm2d_problem* p, cvlbm2d_fields* f,
                                          double time0, int64_t step0, int32_t nsteps,
                                          void* stream) {
  if (!p || !f) return fail(CVLBM_ERR_INVALID_ARG, "null problem or fields");
  if (p->n_links > CVLBM2D_STATIC_SCRATCH_MAX_LINKS)
    return fail(CVLBM_ERR_INVALID_ARG,
                ("cvlbm2d_run_static_scratch: " + std::to_string(p->n_links) +
                    " cut links exceed the static scratch of " +
                    std::to_string(CVLBM2D_STATIC_SCRATCH_MAX_LINKS) +
                    "; use cvlbm2d_run with a caller-owned link_scratch")
                       .c_str());
  if (f->f0) {  // the fields must live on the current device
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, f->f0) == cudaSuccess && attr.type == cudaMemoryTypeDevice) {
      int dev = -1;
      cudaGetDevice(&dev);
      if (attr.device != dev)
        return fail(CVLBM_ERR_INVALID_ARG,
                    ("cvlbm2d_run_static_scratch: fields are on device " +
                     std::to_string(attr.device) + " but device " + std::to_string(dev) +
                     " is current")
                        .c_str());
    }
  }
  double* scratch = nullptr;
  int rc = static_scratch(&scratch);
  if (rc) return rc;
  cvlbm2d_fields local = *f;
  local.link_scratch = scratch;
  // the serial step: no second stream or events are created for this call
  cvlbm2d_problem serial = *p;
  serial.overlap = 0;
  rc = cvlbm2d_run(&serial, &local, time0, step0, nsteps, 0, stream);
  // hand back the f0/f1 exchange cvlbm2d_run made, keep the caller's scratch field
  f->f0 = local.f0;
  f->f1 = local.f1;
  return rc;
}

// ---------------------------------------------------------------------------
// Batched step of many independent 2-D problems (see cvlbm2d_batch.cuh).
// ---------------------------------------------------------------------------
#include "cvlbm2d_batch.cuh"

// ---------------------------------------------------------------------------
// Initial populations on the device (see cvlbm2d_init.cuh).
// ---------------------------------------------------------------------------
#include "cvlbm2d_init.cuh"
