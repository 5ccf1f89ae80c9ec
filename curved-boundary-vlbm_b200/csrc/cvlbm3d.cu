// D3Q6x12 curved-boundary VLBM time step on compacted active nodes, sm_100a.
//
// Layout: f[(q*12+a)*N + p], N = n_active, nodes in (i,j,k) raster order with
// k fastest, so +-z neighbours are adjacent ids and +-x/+-y neighbours are
// contiguous runs: the pull through the 6-neighbour table stays coalesced.
//
// Step pipeline:
//   collide  f0 in place, U, u, u*              _sparse_collide_inplace_kernel
//   sweep    u -> u_next, u* (+ anchors)         _sparse_local_build_bc/sweep
//   commit   u <- u_next                         _sparse_local_displacement_commit
//   repair   f0, U <- blend(F, I+grad u)         _sparse_local_repair_F
//   stream   f1[q](p) = f0[q](nbr(p, -c_q))      _sparse_stream_kernel (pull form)
//   links    gather + prepare + BFL + characteristic, one thread per link
//            (_sparse_characteristic_gather, _sparse_prepare_links_gpu,
//             _sparse_apply_links, _sparse_apply_characteristic)
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "cvlbm_common.cuh"
#include "cvlbm_math.cuh"

using namespace cv;

namespace {

constexpr int kQ3 = 6;
constexpr int kC3 = 12;
constexpr int kF3 = 72;
constexpr int kMaxLsq3 = 32;
constexpr int kChar = 64;
constexpr int kMaxIds3 = 16;

struct Ctx3 {
  cvlbm3d_problem p;
  Mat m;
  int N;
};

__device__ __forceinline__ double time_of(const double* clock, double t, double offset) {
  return (clock ? clock[0] : t) + offset;
}

// ---------------------------------------------------------------------------
// Collision in place, three_d/curved_boundary_warp3d.py:2192-2316.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_collide3(Ctx3 c, double* __restrict__ f,
                                                  double* __restrict__ U, double* __restrict__ u,
                                                  double* __restrict__ ustar,
                                                  int* __restrict__ invalid) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm3d_problem& p = c.p;
  double S[kC3];
#pragma unroll
  for (int a = 0; a < kC3; ++a) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kQ3; ++q) s += f[(size_t)(q * kC3 + a) * N + n];
    S[a] = s;
  }
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
#pragma unroll
    for (int a = 0; a < kC3; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
    S[2] = S[2] / den;
  }
#pragma unroll
  for (int a = 0; a < kC3; ++a) U[(size_t)a * N + n] = S[a];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double uu = ustar[(size_t)d * N + n] + hdt * S[d];
    u[(size_t)d * N + n] = uu;
    ustar[(size_t)d * N + n] = uu + hdt * S[d];
  }
  if (det3(S[3], S[4], S[5], S[6], S[7], S[8], S[9], S[10], S[11]) <= c.m.jf) *invalid = 1;
  M3 P = piola3(S + 3, c.m);
  const double k3c = 3.0 / p.c;
  const double sixth = 1.0 / 6.0;
  const double om = p.omega;
  const double sw = p.dt * (2.0 - om) * (1.0 / 12.0);
#pragma unroll
  for (int q = 0; q < kQ3; ++q) {
#pragma unroll
    for (int a = 0; a < kC3; ++a) {
      double fe = feq3(q, a, S, P, k3c, sixth);
      size_t k = (size_t)(q * kC3 + a) * N + n;
      double old = f[k];
      f[k] = old + om * (fe - old) + sw * source_comp3(a, p.source_mode, p.source, S);
    }
  }
}

// ---------------------------------------------------------------------------
// Local displacement sweep, three_d/curved_boundary_warp3d.py:2402-2540.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sweep3(Ctx3 c, const double* __restrict__ U,
                                                const double* __restrict__ u,
                                                double* __restrict__ unext,
                                                double* __restrict__ ustar, const double* clock,
                                                double t_host) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm3d_problem& p = c.p;
  double d[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
  const double time = time_of(clock, t_host, 0.5 * p.dt);
  const double w2 = p.weight * p.weight;
  // anchors in ascending link order (_sparse_local_build_bc, :2412-2469)
  for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
    int ell = p.node_link_list[k];
    int bid = p.link_bid[ell];
    bool force_all = false;
    if (p.disp_bid >= 0) {
      if (bid != p.disp_bid) continue;
      force_all = true;
    }
    double x = p.link_xb[ell], y = p.link_yb[ell], z = p.link_zb[ell];
    double dbx = x - ((double)p.active_i[n] + 0.5) * p.dx;
    double dby = y - ((double)p.active_j[n] + 0.5) * p.dy;
    double dbz = z - ((double)p.active_k[n] + 0.5) * p.dz;
    int mode = p.bc_mode[bid];
    const double* pp = p.bc_params + bid * 16;
    for (int comp = 0; comp < 3; ++comp) {
      if (!(force_all || p.bc_comp_kind[comp * kMaxIds3 + bid] == kDirichlet)) continue;
      double ub = disp3(mode, pp, comp, x, y, z, time);
      const double* F = U + (size_t)(3 + 3 * comp) * N;
      double e0 = F[n], e1 = F[(size_t)N + n], e2 = F[2 * (size_t)N + n];
      if (comp == 0) e0 = e0 - 1.0;
      if (comp == 1) e1 = e1 - 1.0;
      if (comp == 2) e2 = e2 - 1.0;
      double rhs = ub - (e0 * dbx + e1 * dby + e2 * dbz);
      d[comp] = d[comp] + w2;
      r[comp] = r[comp] + w2 * rhs;
    }
  }
  for (int q = 0; q < kQ3; ++q) {
    int m = p.neighbor[(size_t)q * N + n];
    if (m < 0) continue;
    double ddx = (double)dx3(q) * p.dx, ddy = (double)dy3(q) * p.dy, ddz = (double)dz3(q) * p.dz;
    const double* Ub = U + 3 * (size_t)N;
    double g0 = 0.5 * ((Ub[n] + Ub[m] - 2.0) * ddx + (Ub[N + n] + Ub[N + m]) * ddy +
                       (Ub[2 * (size_t)N + n] + Ub[2 * (size_t)N + m]) * ddz);
    double g1 = 0.5 * ((Ub[3 * (size_t)N + n] + Ub[3 * (size_t)N + m]) * ddx +
                       (Ub[4 * (size_t)N + n] + Ub[4 * (size_t)N + m] - 2.0) * ddy +
                       (Ub[5 * (size_t)N + n] + Ub[5 * (size_t)N + m]) * ddz);
    double g2 = 0.5 * ((Ub[6 * (size_t)N + n] + Ub[6 * (size_t)N + m]) * ddx +
                       (Ub[7 * (size_t)N + n] + Ub[7 * (size_t)N + m]) * ddy +
                       (Ub[8 * (size_t)N + n] + Ub[8 * (size_t)N + m] - 2.0) * ddz);
    r[0] += u[m] - g0;
    r[1] += u[(size_t)N + m] - g1;
    r[2] += u[2 * (size_t)N + m] - g2;
    d[0] += 1.0;
    d[1] += 1.0;
    d[2] += 1.0;
  }
  for (int comp = 0; comp < 3; ++comp) {
    double uo = u[(size_t)comp * N + n];
    double un = uo;
    if (d[comp] > 0.0) un = uo + p.relax * (r[comp] / d[comp] - uo);
    unext[(size_t)comp * N + n] = un;
    ustar[(size_t)comp * N + n] = ustar[(size_t)comp * N + n] + (un - uo);
  }
}

__global__ void k_copy3(long long n3, const double* __restrict__ src, double* __restrict__ dst) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < n3) dst[n] = src[n];
}

// ---------------------------------------------------------------------------
// Local F repair on all active nodes, three_d/curved_boundary_warp3d.py:2543-2672.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double du_axis3(const double* uc, const int* nbr, int N, int n,
                                           int qp, int qm, double h) {
  int pp = nbr[(size_t)qp * N + n];
  int pm = nbr[(size_t)qm * N + n];
  if (pp >= 0 && pm >= 0) return (uc[pp] - uc[pm]) / (2.0 * h);
  if (pp >= 0) {
    int pp2 = nbr[(size_t)qp * N + pp];
    if (pp2 >= 0) return (-3.0 * uc[n] + 4.0 * uc[pp] - uc[pp2]) / (2.0 * h);
    return (uc[pp] - uc[n]) / h;
  }
  if (pm >= 0) {
    int pm2 = nbr[(size_t)qm * N + pm];
    if (pm2 >= 0) return (3.0 * uc[n] - 4.0 * uc[pm] + uc[pm2]) / (2.0 * h);
    return (uc[n] - uc[pm]) / h;
  }
  return 0.0;
}

__global__ void __launch_bounds__(128) k_repair3(Ctx3 c, double* __restrict__ f,
                                                 double* __restrict__ U,
                                                 const double* __restrict__ u) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm3d_problem& p = c.p;
  double beta = fmax(0.0, fmin(1.0, p.blend));
  double o[9], t[9], nn[9];
  for (int k = 0; k < 9; ++k) o[k] = U[(size_t)(3 + k) * N + n];
  const double h[3] = {p.dx, p.dy, p.dz};
  for (int comp = 0; comp < 3; ++comp)
    for (int ax = 0; ax < 3; ++ax) {
      double g = du_axis3(u + (size_t)comp * N, p.neighbor, N, n, ax, ax + 3, h[ax]);
      t[3 * comp + ax] = comp == ax ? 1.0 + g : g;
    }
  for (int k = 0; k < 9; ++k) nn[k] = o[k] + beta * (t[k] - o[k]);
  if (det3v(nn) <= c.m.jf) return;
  M3 Po = piola3(o, c.m);
  M3 Pn = piola3(nn, c.m);
  const double ff = 0.5 / p.c;
  const double sixth = 1.0 / 6.0;
  for (int q = 0; q < kQ3; ++q) {
    double sx = (double)dx3(q), sy = (double)dy3(q), sz = (double)dz3(q);
    size_t b = (size_t)(q * kC3) * N + n;
    for (int i = 0; i < 3; ++i) {
      size_t k = b + (size_t)i * N;
      f[k] = f[k] - ff * (sx * (Pn.v[3 * i] - Po.v[3 * i]) + sy * (Pn.v[3 * i + 1] - Po.v[3 * i + 1]) +
                          sz * (Pn.v[3 * i + 2] - Po.v[3 * i + 2]));
    }
    for (int k9 = 0; k9 < 9; ++k9) {
      size_t k = b + (size_t)(3 + k9) * N;
      f[k] = f[k] + sixth * (nn[k9] - o[k9]);
    }
  }
  for (int k = 0; k < 9; ++k) U[(size_t)(3 + k) * N + n] = nn[k];
}

// ---------------------------------------------------------------------------
// Streaming in pull form, equivalent to three_d/curved_boundary_warp3d.py:2319-2330
// after the clear of f1.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_stream3(Ctx3 c, const double* __restrict__ fpost,
                                                 double* __restrict__ f1) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int* nbr = c.p.neighbor;
#pragma unroll
  for (int q = 0; q < kQ3; ++q) {
    int s = nbr[(size_t)opp3(q) * N + n];
#pragma unroll
    for (int a = 0; a < kC3; ++a) {
      size_t k = (size_t)(q * kC3 + a) * N;
      f1[k + n] = s >= 0 ? fpost[k + s] : 0.0;
    }
  }
}

// ---------------------------------------------------------------------------
// Cut links: gather, prepare, BFL rows, characteristic rows.
// ---------------------------------------------------------------------------
// three_d/curved_boundary_warp3d.py:2755-2809 (_local_characteristic_population3)
__device__ void char_population3(const double* Ub, const double* Gx, const double* Gy,
                                 const double* Gz, const double* d, double eta, double dt,
                                 double c, const cvlbm3d_problem& p, const Mat& m, double omega,
                                 double* out) {
  double dG[12], shift[12];
  const double k = eta * dt * c;
  for (int a = 0; a < 12; ++a) {
    dG[a] = d[0] * Gx[a] + d[1] * Gy[a] + d[2] * Gz[a];
    shift[a] = k * dG[a];
  }
  double chi = 1.0;
  double Uc[12];
  for (int g = 0; g < 10; ++g) {
    for (int a = 0; a < 12; ++a) Uc[a] = Ub[a] + chi * shift[a];
    if (state_det3(Uc) > 10.0 * m.jf) break;
    chi = 0.5 * chi;
  }
  for (int a = 0; a < 12; ++a) Uc[a] = Ub[a] + chi * shift[a];
  double B[12];
  for (int a = 0; a < 12; ++a) B[a] = source_comp3(a, p.source_mode, p.source, Uc);
  double j0[12], j1[12], j2[12], w[12];
  jvp3(0, Uc, Gx, m, j0);
  jvp3(1, Uc, Gy, m, j1);
  jvp3(2, Uc, Gz, m, j2);
  for (int a = 0; a < 12; ++a) w[a] = B[a] - j0[a] - j1[a] - j2[a] + c * dG[a];
  int axis = 0;
  if (fabs(d[1]) > 0.5) axis = 1;
  if (fabs(d[2]) > 0.5) axis = 2;
  double Aw[12];
  jvp3(axis, Uc, w, m, Aw);
  M3 P = piola3(Uc + 3, m);
  double fl[12];
  for (int a = 0; a < 12; ++a) fl[a] = 0.0;
  for (int i = 0; i < 3; ++i) {
    fl[i] = -P.v[3 * i + axis];
    fl[3 + 3 * i + axis] = -Uc[i];
  }
  const double s3 = 3.0 * d[axis];
  const double kk = dt / omega;
  const double kb = dt * (1.0 / omega - 0.5);
  for (int a = 0; a < 12; ++a)
    out[a] = (Uc[a] + s3 * fl[a] / c - kk * (w[a] + s3 * Aw[a] / c) + kb * B[a]) / 6.0;
}

__device__ void link3(const Ctx3& c, int ell, const double* __restrict__ src,
                      double* __restrict__ dst, const double* __restrict__ U,
                      const double* __restrict__ u, const cvlbm3d_fields& fl, double t,
                      int* invalid) {
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
  const int N = c.N, L = p.n_links;
  const int bid = p.link_bid[ell];
  const int kind = p.bc_kind[bid], mode = p.bc_mode[bid];
  int ck[3];
  for (int r = 0; r < 3; ++r) ck[r] = p.bc_comp_kind[r * kMaxIds3 + bid];
  const double* pp = p.bc_params + bid * 16;
  const double x = p.link_xb[ell], y = p.link_yb[ell], z = p.link_zb[ell];
  const double nx = p.link_nx[ell], ny = p.link_ny[ell], nz = p.link_nz[ell];
  const int n = p.link_p[ell];
  const int upid = p.link_up[ell];
  const int qo = p.link_q[ell];
  const int qi = opp3(qo);
  double eta = p.link_eta[ell];

  // characteristic gather (_sparse_characteristic_gather, :2675-2700)
  double G[4][12] = {};
  const bool gather = p.has_char && p.char_idx[ell] >= 0;
  if (gather) {
    for (int a = 0; a < 12; ++a) {
      double v0 = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
      const double* Ua = U + (size_t)a * N;
      for (int mm = 0; mm < kChar; ++mm) {
        int q = p.char_idx[(size_t)mm * L + ell];
        if (q >= 0) {
          double uv = Ua[q];
          v0 += p.char_w[((size_t)0 * kChar + mm) * L + ell] * uv;
          gx += p.char_w[((size_t)1 * kChar + mm) * L + ell] * uv;
          gy += p.char_w[((size_t)2 * kChar + mm) * L + ell] * uv;
          gz += p.char_w[((size_t)3 * kChar + mm) * L + ell] * uv;
        }
      }
      G[0][a] = v0;
      G[1][a] = gx;
      G[2][a] = gy;
      G[3][a] = gz;
      if (fl.char_state)
        for (int k = 0; k < 4; ++k) fl.char_state[((size_t)k * 12 + a) * L + ell] = G[k][a];
    }
  }

  // preparation (_sparse_prepare_links_gpu, :2887-3151)
  double T[3];
  for (int r = 0; r < 3; ++r) T[r] = value3(r, mode, pp, x, y, z, nx, ny, nz, t, m.jf);
  if (p.dyn_enabled && p.dyn_enabled[ell] != 0)
    for (int r = 0; r < 3; ++r) T[r] = p.dyn_traction[(size_t)r * L + ell];
  double Fb[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double Pb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const bool anyN = ck[0] == kNeumann || ck[1] == kNeumann || ck[2] == kNeumann;
  if (anyN) {
    double F[9];
    for (int k = 0; k < 9; ++k) F[k] = U[(size_t)(3 + k) * N + n];
    if (p.recon == 2 || p.recon == 4) {
      if (upid >= 0)
        for (int k = 0; k < 9; ++k) {
          const double* Uk = U + (size_t)(3 + k) * N;
          F[k] = Uk[n] + eta * (Uk[n] - Uk[upid]);
        }
      if (p.recon == 2 && p.has_tangent_lsq && p.lsq_valid[ell] != 0) {
        Frame3 fr = frame3(nx, ny, nz);
        double du1[3] = {0, 0, 0}, du2[3] = {0, 0, 0}, wt_abs = 0.0;
        for (int mm = 0; mm < kMaxLsq3; ++mm) {
          int q = p.lsq_p[(size_t)ell * kMaxLsq3 + mm];
          if (q >= 0) {
            double w1 = p.lsq_wt1[(size_t)ell * kMaxLsq3 + mm];
            double w2 = p.lsq_wt2[(size_t)ell * kMaxLsq3 + mm];
            for (int r = 0; r < 3; ++r) {
              du1[r] += w1 * u[(size_t)r * N + q];
              du2[r] += w2 * u[(size_t)r * N + q];
            }
            wt_abs += fabs(w1) + fabs(w2);
          }
        }
        if (wt_abs > 0.0) {
          double h[3], g1[3], g2[3];
          for (int r = 0; r < 3; ++r) {
            h[r] = F[3 * r] * fr.n[0] + F[3 * r + 1] * fr.n[1] + F[3 * r + 2] * fr.n[2];
            g1[r] = fr.t1[r] + du1[r];
            g2[r] = fr.t2[r] + du2[r];
          }
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s)
              F[3 * r + s] = h[r] * fr.n[s] + g1[r] * fr.t1[s] + g2[r] * fr.t2[s];
        }
      }
    }
    if (p.recon == 3)
      for (int k = 0; k < 9; ++k) F[k] = G[0][3 + k];
    for (int k = 0; k < 9; ++k) Fb[k] = F[k];
    if (ck[0] == kNeumann && ck[1] == kNeumann && ck[2] == kNeumann)
      solve_Fb3(F, nx, ny, nz, T, m, p.normal_solver, Fb);
    else if (ck[0] == kNeumann || ck[1] == kNeumann || ck[2] == kNeumann)
      solve_Fb3_mixed(F, nx, ny, nz, T, ck, m, p.normal_solver, Fb);
    M3 P = piola3(Fb, m);
    for (int k = 0; k < 9; ++k) Pb[k] = P.v[k];
  }
  if (fl.link_kind) {
    fl.link_kind[ell] = kind;
    for (int r = 0; r < 3; ++r) {
      fl.link_comp_kind[(size_t)r * L + ell] = ck[r];
      fl.link_bv[(size_t)r * L + ell] = T[r];
    }
    for (int k = 0; k < 9; ++k) {
      fl.link_Fb[(size_t)k * L + ell] = Fb[k];
      fl.link_Pb[(size_t)k * L + ell] = Pb[k];
    }
  }

  // BFL rows (_sparse_apply_links, :3154-3241)
  if (p.recon == 1) eta = 0.5;
  const double din[3] = {(double)dx3(qi), (double)dy3(qi), (double)dz3(qi)};
  const double cc = p.c;
  for (int a = 0; a < 12; ++a) {
    int row = a < 3 ? a : (a - 3) / 3;
    double D = 1.0, S = 0.0;
    if (ck[row] == kDirichlet) {
      if (a < 3) {
        D = -1.0;
        S = T[a] / 3.0;
      } else {
        int col = (a - 3) - row * 3;
        S = -din[col] * T[row] / cc;
      }
    } else {
      if (a < 3) {
        S = -(din[0] * Pb[3 * a] + din[1] * Pb[3 * a + 1] + din[2] * Pb[3 * a + 2]) / cc;
      } else {
        D = -1.0;
        S = Fb[a - 3] / 3.0;
      }
    }
    double fo = src[(size_t)(qo * 12 + a) * N + n];
    double fi = src[(size_t)(qi * 12 + a) * N + n];
    double val;
    if (eta >= 0.5) {
      double al = 1.0 / (2.0 * eta);
      val = al * (D * fo + S) + (1.0 - al) * fi;
    } else {
      double up = fo;
      if (upid >= 0) up = src[(size_t)(qo * 12 + a) * N + upid];
      val = D * (2.0 * eta * fo + (1.0 - 2.0 * eta) * up) + S;
    }
    dst[(size_t)(qi * 12 + a) * N + n] = val;
  }

  // characteristic rows (_sparse_apply_characteristic, :2812-2884)
  if (gather && anyN) {
    double Ub[12];
    for (int a = 0; a < 3; ++a) Ub[a] = ck[a] == kDirichlet ? T[a] : U[(size_t)a * N + n];
    for (int k = 0; k < 9; ++k) Ub[3 + k] = Fb[k];
    if (state_det3(Ub) <= m.jf) *invalid = 1;
    double out[12];
    char_population3(Ub, G[1], G[2], G[3], din, p.link_eta[ell], p.dt, cc, p, m, p.omega, out);
    for (int a = 0; a < 12; ++a) {
      int row = a < 3 ? a : (a - 3) / 3;
      if (ck[row] == kNeumann) dst[(size_t)(qi * 12 + a) * N + n] = out[a];
    }
  }
}

__global__ void __launch_bounds__(64) k_links3(Ctx3 c, const double* __restrict__ src,
                                               double* __restrict__ dst,
                                               const double* __restrict__ U,
                                               const double* __restrict__ u, cvlbm3d_fields fl,
                                               const double* clock, double t_host, double offset) {
  int ell = blockIdx.x * blockDim.x + threadIdx.x;
  if (ell >= c.p.n_links) return;
  link3(c, ell, src, dst, U, u, fl, time_of(clock, t_host, offset), fl.invalid);
}

// ---------------------------------------------------------------------------
// Refresh, three_d/curved_boundary_warp3d.py:2109-2189.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_refresh3(Ctx3 c, const double* __restrict__ f,
                                                  double* __restrict__ U, double* __restrict__ u,
                                                  const double* __restrict__ ustar,
                                                  int* __restrict__ invalid) {
  const int N = c.N;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm3d_problem& p = c.p;
  double S[kC3];
  for (int a = 0; a < kC3; ++a) {
    double s = 0.0;
    for (int q = 0; q < kQ3; ++q) s += f[(size_t)(q * kC3 + a) * N + n];
    S[a] = s;
  }
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
    for (int a = 0; a < kC3; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
    S[2] = S[2] / den;
  }
  for (int a = 0; a < kC3; ++a) U[(size_t)a * N + n] = S[a];
  for (int d = 0; d < 3; ++d) u[(size_t)d * N + n] = ustar[(size_t)d * N + n] + hdt * S[d];
  if (det3(S[3], S[4], S[5], S[6], S[7], S[8], S[9], S[10], S[11]) <= c.m.jf) *invalid = 1;
}

__global__ void k_set_ustar3(int N, const double* __restrict__ disp, const double* __restrict__ U,
                             double* __restrict__ ustar, double dt) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  for (int d = 0; d < 3; ++d)
    ustar[(size_t)d * N + n] = disp[(size_t)d * N + n] - 0.5 * dt * U[(size_t)d * N + n];
}

}  // namespace

#include "cvlbm3d_fused.cuh"

namespace {

__global__ void k_tick3(double* clock, double dt) { clock[0] = clock[0] + dt; }
__global__ void k_zero_flag3(int* flag) { *flag = 0; }

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }
bool due(int interval, long long step) { return interval > 0 && step % interval == 0; }

int check_problem(const cvlbm3d_problem* p, const cvlbm3d_fields* f) {
  if (!p || !f) return fail(CVLBM_ERR_INVALID_ARG, "null problem or fields");
  if (p->n_active < 0 || p->n_links < 0) return fail(CVLBM_ERR_INVALID_ARG, "negative sizes");
  if ((long long)p->n_active * 72 > 0x7fffffffffffLL)
    return fail(CVLBM_ERR_INVALID_ARG, "too many active nodes");
  if (!f->f0 || !f->f1 || !f->U || !f->u || !f->u_next || !f->u_star || !f->invalid)
    return fail(CVLBM_ERR_INVALID_ARG, "missing field buffer");
  if (!p->neighbor || !p->node_link_start || !p->bc_kind || !p->bc_comp_kind || !p->bc_params)
    return fail(CVLBM_ERR_INVALID_ARG, "missing geometry table");
  if (p->recon < 0 || p->recon > 4)
    return fail(CVLBM_ERR_UNSUPPORTED, "unsupported 3-D boundary reconstruction id");
  if (p->has_char && (!p->char_idx || !p->char_w))
    return fail(CVLBM_ERR_INVALID_ARG, "characteristic stencil tables missing");
  return CVLBM_OK;
}

// The fused pipeline needs its link tables and scratch, and one sweep per
// due step (several sweeps per step take the per-phase pipeline).
bool fused_ok3(const cvlbm3d_problem* p, const cvlbm3d_fields* f) {
  if (!p->need_slot || p->disp_sweeps > 1) return false;
  if (p->n_links > 0) {
    if (!p->link_partner || !f->link_scratch || !f->U_need || p->n_need <= 0 ||
        !f->link_kind || !f->link_comp_kind || !f->link_bv || !f->link_Fb || !f->link_Pb)
      return false;
    if (p->has_char && (!f->char_state || !p->char_slot)) return false;
  }
  return true;
}

// Second stream and two events of the overlapped fused step, one set per
// device and caller stream, created on first use and kept for the life of the
// process.
struct Overlap3 {
  cudaStream_t inner;         // moments of the nodes without a cut link
  cudaEvent_t inner_done;     // last such launch issued
  cudaEvent_t collide_done;   // last collide launch issued
};
std::mutex g_overlap3_mu;
std::map<std::pair<int, cudaStream_t>, Overlap3> g_overlap3;  // (device, caller stream)

Overlap3* overlap3_resources(cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_overlap3_mu);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  const auto key = std::make_pair(dev, s);  // the default stream's handle is shared by devices
  auto it = g_overlap3.find(key);
  if (it != g_overlap3.end()) return &it->second;
  Overlap3 o{};
  if (cudaStreamCreateWithFlags(&o.inner, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&o.inner_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&o.collide_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaStreamDestroy(o.inner);
    return nullptr;
  }
  return &(g_overlap3[key] = o);
}

// Persistent grid of the wavefront kernel: the blocks one device holds at
// once (all resident, each taking items until none are left).
template <int MINB>
int wave_grid() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int sms = 0, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k3_wave<MINB>, 128, 0);
  if (per < 1) per = 1;
  if (sms < 1) sms = 1;
  return cache[dev] = sms * per;
}

bool wave_ok3(const cvlbm3d_problem* p, const cvlbm3d_fields* f) {
  return (p->node_variant == 3 || p->node_variant == 4) && p->wave_items && p->n_wave_items > 0 && p->n_planes > 0 &&
         p->wave_plane_chunks && f->wave_sync;
}

Ctx3 make_ctx(const cvlbm3d_problem* p) {
  Ctx3 c;
  c.p = *p;
  c.m = Mat{p->mat.model, p->mat.lam, p->mat.mu, p->mat.p0, p->mat.p1, p->mat.p2, p->mat.j_floor};
  c.N = p->n_active;
  return c;
}

}  // namespace

extern "C" int cvlbm3d_run(const cvlbm3d_problem* p, cvlbm3d_fields* f, double time0,
                           int64_t step0, int32_t nsteps, int32_t graph_mode, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (nsteps < 0) return fail(CVLBM_ERR_INVALID_ARG, "negative step count");
  if (graph_mode && !f->clock) return fail(CVLBM_ERR_INVALID_ARG, "graph mode needs a clock");
  cudaStream_t s = (cudaStream_t)stream;
  Ctx3 c = make_ctx(p);
  const int N = c.N;
  const double* clock = graph_mode ? f->clock : nullptr;
  k_zero_flag3<<<1, 1, 0, s>>>(f->invalid); cv::count_launches(1);
  double t = time0;
  if (fused_ok3(p, f)) {
    Fused3 fz{p->need_slot, p->char_slot, p->link_partner, p->link_order, f->link_scratch,
              f->U_need};
    const int L = p->n_links;
    // Overlap: the links of step k read f1 only at link nodes and their
    // upstream nodes, and U_need, the swept u and link_scratch; the moments
    // of step k + 1 at nodes without a cut link read f1 elsewhere and write
    // U and u_next.  So they run on a second stream after the collide of step
    // k, while the links do; the moments of the link nodes follow the links.
    const bool wave = wave_ok3(p, f) && N > 0;
    Overlap3* ov = nullptr;
    if (!wave && p->overlap && p->disp_interval == 1 && N > 0 && L > 0 && p->link_nodes &&
        p->n_link_nodes > 0 && nsteps > 1)
      ov = overlap3_resources(s);
    const Wave3 wv{reinterpret_cast<const int4*>(p->wave_items), p->n_wave_items, p->n_planes,
                   p->wave_plane_chunks, f->wave_sync};
    for (int k = 0; k < nsteps; ++k) {
      const long long step = step0 + k;
      const int sweep = N > 0 && due(p->disp_interval, step);
      const int repair = due(p->rep_interval, step);
      int tk = ov ? -1 : timer_begin(s);
      if (wave) {
        cudaMemsetAsync(f->wave_sync, 0, sizeof(int32_t) * (2 + 3 * (size_t)p->n_planes), s);
        if (p->node_variant == 4)
          k3_wave<3><<<wave_grid<3>(), 128, 0, s>>>(c, fz, wv, f->f0, f->f1, f->U, f->u_next,
                                                     f->u, f->u_star, f->invalid, clock, t,
                                                     sweep, repair, k == nsteps - 1);
        else
          k3_wave<4><<<wave_grid<4>(), 128, 0, s>>>(c, fz, wv, f->f0, f->f1, f->U, f->u_next,
                                                     f->u, f->u_star, f->invalid, clock, t,
                                                     sweep, repair, k == nsteps - 1);
        cv::count_launches(1);
      } else if (N > 0 && ov && k > 0) {
        cudaStreamWaitEvent(s, ov->inner_done, 0);
        k3_moments_part<1><<<blocks(p->n_link_nodes, 256), 256, 0, s>>>(
            c, f->f0, f->U, f->u_next, f->u_star, f->invalid, sweep);
        cv::count_launches(1);
      } else if (N > 0) {
        k3_moments<<<blocks(N, 256), 256, 0, s>>>(c, f->f0, f->U, sweep ? f->u_next : f->u,
                                                  f->u_star, f->invalid, sweep);
        cv::count_launches(1);
      }
      if (N > 0 && !wave) {
        if (sweep) {
          k3_sweep<<<blocks(N, 256), 256, 0, s>>>(c, f->U, f->u_next, f->u, f->u_star, clock, t);
          cv::count_launches(1);
        }
        if (p->node_variant == 1)
          k3_collide<<<blocks(N, kCN), kQ3 * kCN, 0, s>>>(c, fz, f->f0, f->f1, f->U, f->u,
                                                          repair, k == nsteps - 1);
        else if (p->node_variant == 2)
          k3_collide_node<3><<<blocks(N, 128), 128, 0, s>>>(c, fz, f->f0, f->f1, f->U, f->u,
                                                            repair, k == nsteps - 1);
        else
          k3_collide_node<4><<<blocks(N, 128), 128, 0, s>>>(c, fz, f->f0, f->f1, f->U, f->u,
                                                            repair, k == nsteps - 1);
        cv::count_launches(1);
        if (ov && k + 1 < nsteps) {
          // a sweep is due every step, so these moments write u_next
          cudaEventRecord(ov->collide_done, s);
          cudaStreamWaitEvent(ov->inner, ov->collide_done, 0);
          k3_moments_part<0><<<blocks(N, 256), 256, 0, ov->inner>>>(
              c, f->f1, f->U, f->u_next, f->u_star, f->invalid, 1);
          cudaEventRecord(ov->inner_done, ov->inner);
          cv::count_launches(1);
        }
      }
      timer_end(tk, s);
      if (L > 0) {
        if (p->has_char) {
          if (p->char_slot_lm && p->char_w_lm)
            k3_link_gather4<<<blocks(L, kGather4Links), 128, 0, s>>>(c, fz, f->char_state);
          else
            k3_link_gather<<<blocks(L, kGatherLinks), 128, 0, s>>>(c, fz, f->char_state);
          cv::count_launches(1);
        }
        k3_link_prepare<<<blocks(L, 128), 128, 0, s>>>(c, fz, f->u, *f, clock, t, 0.5 * p->dt);
        cv::count_launches(1);
        k3_link_rows<<<blocks((long long)L * kC3, 128), 128, 0, s>>>(c, fz, f->f1, *f);
        cv::count_launches(1);
        if (p->has_char) {
          k3_link_char<<<blocks(L, 64), 64, 0, s>>>(c, fz, f->f1, *f);
          cv::count_launches(1);
        }
      }
      if (graph_mode) {
        k_tick3<<<1, 1, 0, s>>>(f->clock, p->dt);
        cv::count_launches(1);
      }
      double* tmp = f->f0;
      f->f0 = f->f1;
      f->f1 = tmp;
      t += p->dt;
    }
    return check_launch("cvlbm3d_run");
  }
  for (int k = 0; k < nsteps; ++k) {
    const long long step = step0 + k;
    int tk = timer_begin(s);
    if (N > 0) k_collide3<<<blocks(N, 128), 128, 0, s>>>(c, f->f0, f->U, f->u, f->u_star, f->invalid); cv::count_launches(1);
    timer_end(tk, s);
    if (N > 0 && due(p->disp_interval, step)) {
      for (int sw = 0; sw < p->disp_sweeps; ++sw) {
        k_sweep3<<<blocks(N, 256), 256, 0, s>>>(c, f->U, f->u, f->u_next, f->u_star, clock, t); cv::count_launches(1);
        k_copy3<<<blocks(3LL * N, 256), 256, 0, s>>>(3LL * N, f->u_next, f->u); cv::count_launches(1);
      }
    }
    if (N > 0 && due(p->rep_interval, step))
      k_repair3<<<blocks(N, 128), 128, 0, s>>>(c, f->f0, f->U, f->u); cv::count_launches(1);
    if (N > 0) k_stream3<<<blocks(N, 256), 256, 0, s>>>(c, f->f0, f->f1); cv::count_launches(1);
    if (p->n_links > 0)
      k_links3<<<blocks(p->n_links, 64), 64, 0, s>>>(c, f->f0, f->f1, f->U, f->u, *f, clock, t,
                                                     0.5 * p->dt); cv::count_launches(1);
    if (graph_mode) k_tick3<<<1, 1, 0, s>>>(f->clock, p->dt); cv::count_launches(1);
    double* tmp = f->f0;
    f->f0 = f->f1;
    f->f1 = tmp;
    t += p->dt;
  }
  return check_launch("cvlbm3d_run");
}

extern "C" int cvlbm3d_apply_boundary(const cvlbm3d_problem* p, cvlbm3d_fields* f, double t,
                                      int32_t in_place, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (p->n_links == 0) return CVLBM_OK;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx3 c = make_ctx(p);
  if (in_place) {
    // f1 is scratch until the next streaming step: links read the copy
    cudaMemcpyAsync(f->f1, f->f0, sizeof(double) * kF3 * (size_t)c.N, cudaMemcpyDeviceToDevice, s);
    k_links3<<<blocks(p->n_links, 64), 64, 0, s>>>(c, f->f1, f->f0, f->U, f->u, *f, nullptr, t,
                                                   0.0); cv::count_launches(1);
  } else {
    k_links3<<<blocks(p->n_links, 64), 64, 0, s>>>(c, f->f0, f->f1, f->U, f->u, *f, nullptr, t,
                                                   0.0); cv::count_launches(1);
  }
  return check_launch("cvlbm3d_apply_boundary");
}

extern "C" int cvlbm3d_refresh(const cvlbm3d_problem* p, cvlbm3d_fields* f, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx3 c = make_ctx(p);
  k_zero_flag3<<<1, 1, 0, s>>>(f->invalid); cv::count_launches(1);
  if (c.N > 0)
    k_refresh3<<<blocks(c.N, 256), 256, 0, s>>>(c, f->f0, f->U, f->u, f->u_star, f->invalid); cv::count_launches(1);
  return check_launch("cvlbm3d_refresh");
}

extern "C" int cvlbm3d_set_ustar(const cvlbm3d_problem* p, cvlbm3d_fields* f,
                                 const double* displacement, void* stream) {
  int rc = check_problem(p, f);
  if (rc) return rc;
  if (!displacement) return fail(CVLBM_ERR_INVALID_ARG, "null displacement");
  cudaStream_t s = (cudaStream_t)stream;
  if (p->n_active > 0)
    k_set_ustar3<<<blocks(p->n_active, 256), 256, 0, s>>>(p->n_active, displacement, f->U,
                                                          f->u_star, p->dt); cv::count_launches(1);
  return check_launch("cvlbm3d_set_ustar");
}

extern "C" int cvlbm3d_graph_create(const cvlbm3d_problem* p, const cvlbm3d_fields* f,
                                    int64_t step0, int32_t nsteps, cvlbm_graph** out) {
  if (!out) return fail(CVLBM_ERR_INVALID_ARG, "null output");
  if (nsteps <= 0 || (nsteps & 1)) return fail(CVLBM_ERR_INVALID_ARG, "nsteps must be even");
  cvlbm3d_fields local = *f;
  return capture_graph(
      [&](cudaStream_t s) { return cvlbm3d_run(p, &local, 0.0, step0, nsteps, 1, s); }, out);
}
