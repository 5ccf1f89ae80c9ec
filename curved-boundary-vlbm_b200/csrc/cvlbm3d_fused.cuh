// D3Q6x12 step, fused form.  Included by cvlbm3d.cu (shares Ctx3 and the
// per-link helpers).
//
// Node kernels (reference raster order of the active nodes):
//   k3_moments   f0 -> U (all 12 components), collide-time u into `ucol`
//                (u_next), invalid flag; when no sweep is due, u and u* too
//   k3_sweep     u_swept -> u and the trapezoidal u* update, from U and ucol
//                of the node and its six neighbours plus cut-point anchors
//   k3_collide_node (default; one thread per node) or k3_collide (six
//                warps per 32 nodes, one per direction; shared memory):
//                f0 again, F repair from the swept u (+-2 star stencil), BGK
//                collision with damping/source, repair delta and push
//                streaming to f1; a population whose neighbour is not active
//                leaves through a cut link and is kept per link
//                (link_scratch) for the link kernels; the post-step U of
//                nodes that links read goes to U_need, one 96-byte row each
//   k3_moments_part  the moments of the nodes without / with a cut link,
//                for the optional overlap of the next step with the links
// Per active node this reads f0 twice and writes f1 once (the f0 re-read of
// the collide is what a single-pass 3-D fusion would save; its 3-deep halo
// does not fit shared memory), plus U, u and u* (about 2.1 KB per node
// against the algorithmic 1.2 KB).
//
// Link kernels (the four phases of apply_boundary_reconstruction,
// three_d/curved_boundary_warp3d.py:4339-4399):
//   k3_link_gather   16 lanes per link, one per component: value and
//                    gradient of the characteristic stencil (:2675-2700)
//   k3_link_prepare  one thread per link: boundary value, F predictor, Newton
//                    normal solve, P(F_b) (:2887-3151)
//   k3_link_rows     one thread per (link, row): BFL rows (:3154-3241) that
//                    the characteristic closure does not overwrite
//   k3_link_char     one thread per link: characteristic rows (:2812-2884)
// In the fused step they read the outgoing populations from link_scratch and
// the post-stream f1 instead of a stored post-collision field.
#pragma once

namespace {

struct Fused3 {
  const int32_t* need_slot;  // [N] row of Uneed of a node some link reads, or -1
  const int32_t* char_slot;  // [64*n_links] characteristic samples as Uneed rows
  const int32_t* partner;    // [n_links] link at the same node in direction q_in, or -1
  const int32_t* order;      // [n_links] processing order of one-thread-per-link kernels
  double* scratch;           // [12*n_links] post-collision population leaving through a link
  double* Uneed;             // [n_need*12] post-step U, one 96-byte row per node
};

// Moments with the collision's damping/source half step
// (three_d/curved_boundary_warp3d.py:2192-2260), summed over q in order.
__device__ __forceinline__ void moments3(const cvlbm3d_problem& p, const double* __restrict__ f,
                                         int N, int n, double* S) {
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
    const double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
    S[2] = S[2] / den;
  }
}

__device__ __forceinline__ void moments_node3(const Ctx3& c, const double* __restrict__ f0,
                                              double* __restrict__ U,
                                              double* __restrict__ ucol,
                                              double* __restrict__ ustar,
                                              int* __restrict__ invalid, int sweep_due, int n);

__global__ void __launch_bounds__(256) k3_moments(Ctx3 c, const double* __restrict__ f0,
                                                  double* __restrict__ U,
                                                  double* __restrict__ ucol,
                                                  double* __restrict__ ustar,
                                                  int* __restrict__ invalid, int sweep_due) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.N) return;
  moments_node3(c, f0, U, ucol, ustar, invalid, sweep_due, n);
}

// The moments of part of the nodes: LINKED = 0 the nodes without a cut link
// (one thread per node, the others return), LINKED = 1 the nodes of
// p.link_nodes (one thread per listed node).
template <int LINKED>
__global__ void __launch_bounds__(256) k3_moments_part(Ctx3 c, const double* __restrict__ f0,
                                                       double* __restrict__ U,
                                                       double* __restrict__ ucol,
                                                       double* __restrict__ ustar,
                                                       int* __restrict__ invalid,
                                                       int sweep_due) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const cvlbm3d_problem& p = c.p;
  int n;
  if (LINKED) {
    if (t >= p.n_link_nodes) return;
    n = p.link_nodes[t];
  } else {
    if (t >= c.N || p.node_link_start[t + 1] > p.node_link_start[t]) return;
    n = t;
  }
  moments_node3(c, f0, U, ucol, ustar, invalid, sweep_due, n);
}

__device__ __forceinline__ void moments_node3(const Ctx3& c, const double* __restrict__ f0,
                                              double* __restrict__ U,
                                              double* __restrict__ ucol,
                                              double* __restrict__ ustar,
                                              int* __restrict__ invalid, int sweep_due, int n) {
  const int N = c.N;
  const cvlbm3d_problem& p = c.p;
  double S[kC3];
  moments3(p, f0, N, n, S);
#pragma unroll
  for (int a = 0; a < kC3; ++a) U[(size_t)a * N + n] = S[a];
  const double hdt = 0.5 * p.dt;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double uu = ustar[(size_t)d * N + n] + hdt * S[d];
    ucol[(size_t)d * N + n] = uu;
    // with a sweep due, k3_sweep writes u* = (uu + hdt v) + (u_swept - uu)
    if (!sweep_due) ustar[(size_t)d * N + n] = uu + hdt * S[d];
  }
  if (det3(S[3], S[4], S[5], S[6], S[7], S[8], S[9], S[10], S[11]) <= c.m.jf) *invalid = 1;
}

// One Jacobi sweep (three_d/curved_boundary_warp3d.py:2402-2540); ucol holds
// the collide-time u of every node, the swept u goes to `u`.
// Loads of values that other blocks of the same launch write (the wavefront
// kernel): through L2 only, so that no stale L1 line is read.
template <bool CG>
__device__ __forceinline__ double ldx(const double* q) {
  if constexpr (CG)
    return __ldcg(q);
  else
    return *q;
}

template <bool CG>
__device__ __forceinline__ void sweep_node3(const Ctx3& c, const double* U, const double* ucol,
                                            double* __restrict__ u, double* __restrict__ ustar,
                                            const double* clock, double t_host, int n) {
  const int N = c.N;
  const cvlbm3d_problem& p = c.p;
  double d[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
  const double time = time_of(clock, t_host, 0.5 * p.dt);
  const double w2 = p.weight * p.weight;
  for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
    const int ell = p.node_link_list[k];
    const int bid = p.link_bid[ell];
    bool force_all = false;
    if (p.disp_bid >= 0) {
      if (bid != p.disp_bid) continue;
      force_all = true;
    }
    const double x = p.link_xb[ell], y = p.link_yb[ell], z = p.link_zb[ell];
    const double dbx = x - ((double)p.active_i[n] + 0.5) * p.dx;
    const double dby = y - ((double)p.active_j[n] + 0.5) * p.dy;
    const double dbz = z - ((double)p.active_k[n] + 0.5) * p.dz;
    const int mode = p.bc_mode[bid];
    const double* pp = p.bc_params + bid * 16;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      if (!(force_all || p.bc_comp_kind[comp * kMaxIds3 + bid] == kDirichlet)) continue;
      const double ub = disp3(mode, pp, comp, x, y, z, time);
      const double* F = U + (size_t)(3 + 3 * comp) * N;
      double e0 = ldx<CG>(F + n), e1 = ldx<CG>(F + (size_t)N + n),
             e2 = ldx<CG>(F + 2 * (size_t)N + n);
      if (comp == 0) e0 = e0 - 1.0;
      if (comp == 1) e1 = e1 - 1.0;
      if (comp == 2) e2 = e2 - 1.0;
      const double rhs = ub - (e0 * dbx + e1 * dby + e2 * dbz);
      d[comp] = d[comp] + w2;
      r[comp] = r[comp] + w2 * rhs;
    }
  }
  const double* Ub = U + 3 * (size_t)N;
  double Fs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Fs[k] = ldx<CG>(Ub + (size_t)k * N + n);
#pragma unroll
  for (int q = 0; q < kQ3; ++q) {
    const int m = p.neighbor[(size_t)q * N + n];
    if (m < 0) continue;
    const double ddx = (double)dx3(q) * p.dx, ddy = (double)dy3(q) * p.dy,
                 ddz = (double)dz3(q) * p.dz;
    const double* Um = Ub + m;
    const size_t NN = (size_t)N;
    const double g0 = 0.5 * ((Fs[0] + ldx<CG>(Um) - 2.0) * ddx + (Fs[1] + ldx<CG>(Um + NN)) * ddy +
                             (Fs[2] + ldx<CG>(Um + 2 * NN)) * ddz);
    const double g1 = 0.5 * ((Fs[3] + ldx<CG>(Um + 3 * NN)) * ddx +
                             (Fs[4] + ldx<CG>(Um + 4 * NN) - 2.0) * ddy +
                             (Fs[5] + ldx<CG>(Um + 5 * NN)) * ddz);
    const double g2 = 0.5 * ((Fs[6] + ldx<CG>(Um + 6 * NN)) * ddx +
                             (Fs[7] + ldx<CG>(Um + 7 * NN)) * ddy +
                             (Fs[8] + ldx<CG>(Um + 8 * NN) - 2.0) * ddz);
    r[0] += ldx<CG>(ucol + m) - g0;
    r[1] += ldx<CG>(ucol + (size_t)N + m) - g1;
    r[2] += ldx<CG>(ucol + 2 * (size_t)N + m) - g2;
    d[0] += 1.0;
    d[1] += 1.0;
    d[2] += 1.0;
  }
  const double hdt = 0.5 * p.dt;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const double uo = ldx<CG>(ucol + (size_t)comp * N + n);
    double un = uo;
    if (d[comp] > 0.0) un = uo + p.relax * (r[comp] / d[comp] - uo);
    u[(size_t)comp * N + n] = un;
    ustar[(size_t)comp * N + n] = (uo + hdt * ldx<CG>(U + (size_t)comp * N + n)) + (un - uo);
  }
}

__global__ void __launch_bounds__(256) k3_sweep(Ctx3 c, const double* __restrict__ U,
                                                const double* __restrict__ ucol,
                                                double* __restrict__ u,
                                                double* __restrict__ ustar, const double* clock,
                                                double t_host) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.N) return;
  sweep_node3<false>(c, U, ucol, u, ustar, clock, t_host, n);
}

// Collision + F repair + push streaming (three_d/curved_boundary_warp3d.py
// :2192-2330, 2543-2672).  `u` is the swept displacement of every node.
//
// A block takes 32 consecutive active nodes with six warps, warp q owning
// direction q (lane = node), so every population load and store is one
// coalesced 256-byte row:
//   1  warp q loads f0[q][0..11] of its 32 nodes (kept in registers, copied
//      to shared memory for the moments)
//   2  moments (summed over q in order) and the nine targets of I + grad u
//      (+-2 star stencil of the swept u), spread over the block
//   3  P(F) and P(F_repaired), one row per warp (six rows), U / U_need rows
//   4  warp q: collision, repair delta and push of direction q
constexpr int kCN = 32;  // nodes per collide block (one per lane)

struct CollideSmem3 {
  double f[kQ3][kC3][kCN];
  double un[kQ3][3][kCN];  // swept u of the neighbour in direction q
  double u0[3][kCN];       // swept u of the node
  int nb[kQ3][kCN];        // neighbour in direction q, -1 if not active
  double S[kC3][kCN];
  double T[9][kCN];   // I + grad u
  double Po[9][kCN];  // P(F)
  double Pn[9][kCN];  // P(F_repaired)
  double dF[9][kCN];  // F_repaired - F
  int rep[kCN];
};

// feq of (q, a) with the moments and P(F) of lane `l` in shared memory; the
// same operations as feq3 (zero-weight axes included).
__device__ __forceinline__ double feq3_smem(int q, int a, const CollideSmem3& sm, int l,
                                            double three_over_c, double sixth) {
  const double sx = (double)dx3(q), sy = (double)dy3(q), sz = (double)dz3(q);
  double f0, f1, f2;
  if (a < 3) {
    f0 = -sm.Po[3 * a][l];
    f1 = -sm.Po[3 * a + 1][l];
    f2 = -sm.Po[3 * a + 2][l];
  } else {
    const int r = a - 3, ax = r % 3;
    const double v = -sm.S[r / 3][l];
    f0 = ax == 0 ? v : 0.0;
    f1 = ax == 1 ? v : 0.0;
    f2 = ax == 2 ? v : 0.0;
  }
  return sixth * (sm.S[a][l] + three_over_c * (sx * f0 + sy * f1 + sz * f2));
}

__global__ void __launch_bounds__(kQ3 * kCN, 4)
    k3_collide(Ctx3 c, Fused3 fz, const double* __restrict__ f0, double* __restrict__ f1,
               double* __restrict__ U, const double* __restrict__ u, int do_repair,
               int store_all) {
  __shared__ CollideSmem3 sm;
  const int N = c.N;
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n0 = blockIdx.x * kCN;
  const int n = n0 + lane;
  const bool live = n < N;

  // 1: populations of direction `warp`, its neighbour and (for the repair)
  // the neighbour's swept u
  double v[kC3];
  const int q = warp;
#pragma unroll
  for (int a = 0; a < kC3; ++a) v[a] = live ? f0[(size_t)(q * kC3 + a) * N + n] : 0.0;
  const int nq = live ? p.neighbor[(size_t)q * N + n] : -1;
  if (do_repair) {
#pragma unroll
    for (int comp = 0; comp < 3; ++comp)
      sm.un[q][comp][lane] = nq >= 0 ? u[(size_t)comp * N + nq] : 0.0;
    if (warp < 3) sm.u0[warp][lane] = live ? u[(size_t)warp * N + n] : 0.0;
  }
#pragma unroll
  for (int a = 0; a < kC3; ++a) sm.f[q][a][lane] = v[a];
  sm.nb[q][lane] = nq;
  __syncthreads();

  // 2: moments (12 x 32 sums) and I + grad u (9 x 32 targets)
  const double hdt = 0.5 * p.dt;
  for (int t = threadIdx.x; t < kC3 * kCN; t += blockDim.x) {
    const int a = t / kCN, l = t % kCN;
    double sacc = 0.0;
#pragma unroll
    for (int qq = 0; qq < kQ3; ++qq) sacc += sm.f[qq][a][l];
    if (p.source_mode == kSrcConstant) {
      sacc += hdt * p.source[a];
    } else if (p.source_mode == kSrcDamping && a < 3) {
      const double den = 1.0 + hdt * p.source[0];
      sacc = sacc / den;
    }
    sm.S[a][l] = sacc;
  }
  if (do_repair) {
    // derivative of the swept u along each axis, as du_axis3: centred with
    // both neighbours, second-order one-sided with two on one side, first
    // order with one, zero with none
    const double h[3] = {p.dx, p.dy, p.dz};
    for (int t = threadIdx.x; t < 9 * kCN; t += blockDim.x) {
      const int k = t / kCN, l = t % kCN, comp = k / 3, ax = k % 3;
      const int pp = sm.nb[ax][l], pm = sm.nb[ax + 3][l];
      const double* uc = u + (size_t)comp * N;
      const double hh = h[ax];
      double g = 0.0;
      if (n0 + l < N) {
        if (pp >= 0 && pm >= 0) {
          g = (sm.un[ax][comp][l] - sm.un[ax + 3][comp][l]) / (2.0 * hh);
        } else if (pp >= 0) {
          const int pp2 = p.neighbor[(size_t)ax * N + pp];
          if (pp2 >= 0)
            g = (-3.0 * sm.u0[comp][l] + 4.0 * sm.un[ax][comp][l] - uc[pp2]) / (2.0 * hh);
          else
            g = (sm.un[ax][comp][l] - sm.u0[comp][l]) / hh;
        } else if (pm >= 0) {
          const int pm2 = p.neighbor[(size_t)(ax + 3) * N + pm];
          if (pm2 >= 0)
            g = (3.0 * sm.u0[comp][l] - 4.0 * sm.un[ax + 3][comp][l] + uc[pm2]) / (2.0 * hh);
          else
            g = (sm.u0[comp][l] - sm.un[ax + 3][comp][l]) / hh;
        }
      }
      sm.T[k][l] = comp == ax ? 1.0 + g : g;
    }
  }
  __syncthreads();

  // 3: P(F) and P(F_repaired), one row of each per warp: warps 0-2 row
  // `warp` of P(F), warps 3-5 row `warp - 3` of the repaired F and its Piola;
  // warp 3 also writes the repaired flag and the U / U_need rows
  {
    const int row = warp < 3 ? warp : warp - 3;
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = sm.S[3 + k][lane];
    if (warp < 3) {
      double Pr[3];
      piola3_row(F, m, row, Pr);
#pragma unroll
      for (int c2 = 0; c2 < 3; ++c2) sm.Po[3 * row + c2][lane] = Pr[c2];
    } else {
      bool repaired = false;
      double nn[9];
      if (do_repair) {
        const double beta = fmax(0.0, fmin(1.0, p.blend));
#pragma unroll
        for (int k = 0; k < 9; ++k) nn[k] = F[k] + beta * (sm.T[k][lane] - F[k]);
        if (det3v(nn) > m.jf) {
          repaired = true;
          double Pr[3];
          piola3_row(nn, m, row, Pr);
#pragma unroll
          for (int c2 = 0; c2 < 3; ++c2) {
            sm.Pn[3 * row + c2][lane] = Pr[c2];
            sm.dF[3 * row + c2][lane] = nn[3 * row + c2] - F[3 * row + c2];
          }
        }
      }
      if (warp == 3) {
        sm.rep[lane] = repaired ? 1 : 0;
        if (repaired && store_all && live) {
#pragma unroll
          for (int k = 0; k < 9; ++k) U[(size_t)(3 + k) * N + n] = nn[k];
        }
        const int slot = live ? fz.need_slot[n] : -1;
        if (slot >= 0) {
          double* rowp = fz.Uneed + (size_t)slot * kC3;
          rowp[0] = sm.S[0][lane];
          rowp[1] = sm.S[1][lane];
          rowp[2] = sm.S[2][lane];
#pragma unroll
          for (int k = 0; k < 9; ++k) rowp[3 + k] = repaired ? nn[k] : F[k];
        }
      }
    }
  }
  __syncthreads();
  if (!live) return;

  // 4: collision, repair delta, push of direction q
  const double k3c = 3.0 / p.c, sixth = 1.0 / 6.0, om = p.omega;
  const double sw = p.dt * (2.0 - om) * (1.0 / 12.0);
  const double ff = 0.5 / p.c;
  const bool repaired = sm.rep[lane] != 0;
  int ell = -1;
  if (nq < 0) {
    for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
      const int e = p.node_link_list[k];
      if (p.link_q[e] == q) ell = e;
    }
  }
  const double sx = (double)dx3(q), sy = (double)dy3(q), sz = (double)dz3(q);
  const double vel[3] = {sm.S[0][lane], sm.S[1][lane], sm.S[2][lane]};
#pragma unroll
  for (int a = 0; a < kC3; ++a) {
    const double old = v[a];
    const double fe = feq3_smem(q, a, sm, lane, k3c, sixth);
    double val = old + om * (fe - old) + sw * source_comp3(a, p.source_mode, p.source, vel);
    if (repaired) {
      if (a < 3)
        val = val - ff * (sx * (sm.Pn[3 * a][lane] - sm.Po[3 * a][lane]) +
                          sy * (sm.Pn[3 * a + 1][lane] - sm.Po[3 * a + 1][lane]) +
                          sz * (sm.Pn[3 * a + 2][lane] - sm.Po[3 * a + 2][lane]));
      else
        val = val + sixth * sm.dF[a - 3][lane];
    }
    if (nq >= 0)
      f1[(size_t)(q * kC3 + a) * N + nq] = val;
    else if (ell >= 0)
      fz.scratch[(size_t)ell * kC3 + a] = val;
  }
}

// Collision + F repair + push streaming, one thread per node.
//
// The moments come from U, which k3_moments wrote this step with the same
// sums (so they equal the shared-memory sums of k3_collide bit for bit), and
// P(F), P(F_repaired) are evaluated once per node.  Each direction is then 12
// coalesced loads of f0 and 12 stores to f1 at the neighbour, with the
// direction a compile-time constant: of the three terms s_x f_x + s_y f_y +
// s_z f_z of the equilibrium flux only the one on the direction's axis is
// formed (the others are products with an exact zero, which change no finite
// sum), so the arithmetic is that of k3_collide without its 0 * x products.
struct NodeState3 {
  double S[kC3];
  double Po[9];  // P(F)
  double dP[9];  // P(F_repaired) - P(F)
  double dF[9];  // F_repaired - F
  int nb[kQ3];
  bool repaired;
};

// Moments, neighbours, P(F), the F repair and its Piola difference; the U
// and U_need rows of the node.
template <bool CG = false>
__device__ __forceinline__ void node_prologue3(const Ctx3& c, const Fused3& fz, double* U,
                                               const double* u, int do_repair, int store_all,
                                               int n, NodeState3& st) {
  const int N = c.N;
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
#pragma unroll
  for (int a = 0; a < kC3; ++a) st.S[a] = ldx<CG>(U + (size_t)a * N + n);
#pragma unroll
  for (int q = 0; q < kQ3; ++q) st.nb[q] = p.neighbor[(size_t)q * N + n];
  const double* F = st.S + 3;
#pragma unroll
  for (int r = 0; r < 3; ++r) piola3_row(F, m, r, st.Po + 3 * r);

  st.repaired = false;
  double nn[9];
  if (do_repair) {
    // I + grad u of the swept u, as du_axis3: centred with both neighbours,
    // second-order one-sided with two on one side, first order with one,
    // zero with none
    const double h[3] = {p.dx, p.dy, p.dz};
    double T[9];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      const double* uc = u + (size_t)comp * N;
      const double u0 = ldx<CG>(uc + n);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int pp = st.nb[ax], pm = st.nb[ax + 3];
        const double hh = h[ax];
        double g = 0.0;
        if (pp >= 0 && pm >= 0) {
          g = (ldx<CG>(uc + pp) - ldx<CG>(uc + pm)) / (2.0 * hh);
        } else if (pp >= 0) {
          const int pp2 = p.neighbor[(size_t)ax * N + pp];
          if (pp2 >= 0)
            g = (-3.0 * u0 + 4.0 * ldx<CG>(uc + pp) - ldx<CG>(uc + pp2)) / (2.0 * hh);
          else
            g = (ldx<CG>(uc + pp) - u0) / hh;
        } else if (pm >= 0) {
          const int pm2 = p.neighbor[(size_t)(ax + 3) * N + pm];
          if (pm2 >= 0)
            g = (3.0 * u0 - 4.0 * ldx<CG>(uc + pm) + ldx<CG>(uc + pm2)) / (2.0 * hh);
          else
            g = (u0 - ldx<CG>(uc + pm)) / hh;
        }
        T[3 * comp + ax] = comp == ax ? 1.0 + g : g;
      }
    }
    const double beta = fmax(0.0, fmin(1.0, p.blend));
#pragma unroll
    for (int k = 0; k < 9; ++k) nn[k] = F[k] + beta * (T[k] - F[k]);
    if (det3v(nn) > m.jf) {
      st.repaired = true;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        double Pr[3];
        piola3_row(nn, m, r, Pr);
#pragma unroll
        for (int c2 = 0; c2 < 3; ++c2) st.dP[3 * r + c2] = Pr[c2] - st.Po[3 * r + c2];
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) st.dF[k] = nn[k] - F[k];
    }
  }
  if (st.repaired && store_all) {
#pragma unroll
    for (int k = 0; k < 9; ++k) U[(size_t)(3 + k) * N + n] = nn[k];
  }
  const int slot = fz.need_slot[n];
  if (slot >= 0) {
    double* rowp = fz.Uneed + (size_t)slot * kC3;
    rowp[0] = st.S[0];
    rowp[1] = st.S[1];
    rowp[2] = st.S[2];
#pragma unroll
    for (int k = 0; k < 9; ++k) rowp[3 + k] = st.repaired ? nn[k] : F[k];
  }
}

template <int Q>
__device__ __forceinline__ void collide_dir3(const cvlbm3d_problem& p, const Fused3& fz,
                                             const NodeState3& st,
                                             const double* __restrict__ f0,
                                             double* __restrict__ f1, int N, int n) {
  constexpr int ax = Q % 3;
  constexpr double s = Q < 3 ? 1.0 : -1.0;
  const double k3c = 3.0 / p.c, sixth = 1.0 / 6.0, om = p.omega;
  const double sw = p.dt * (2.0 - om) * (1.0 / 12.0);
  const double ff = 0.5 / p.c;
  const int nq = st.nb[Q];
  double* dst;
  size_t stride;
  if (nq >= 0) {
    dst = f1 + (size_t)(Q * kC3) * N + nq;
    stride = (size_t)N;
  } else {
    int ell = -1;
    for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
      const int e = p.node_link_list[k];
      if (p.link_q[e] == Q) ell = e;
    }
    if (ell < 0) return;
    dst = fz.scratch + (size_t)ell * kC3;
    stride = 1;
  }
  double old[kC3];
#pragma unroll
  for (int a = 0; a < kC3; ++a) old[a] = f0[(size_t)(Q * kC3 + a) * N + n];
#pragma unroll
  for (int a = 0; a < kC3; ++a) {
    double fe;
    if (a < 3) {
      fe = sixth * (st.S[a] + k3c * (s * -st.Po[3 * a + ax]));
    } else if ((a - 3) % 3 == ax) {
      fe = sixth * (st.S[a] + k3c * (s * -st.S[(a - 3) / 3]));
    } else {
      fe = sixth * st.S[a];
    }
    double val = old[a] + om * (fe - old[a]) + sw * source_comp3(a, p.source_mode, p.source, st.S);
    if (st.repaired) {
      if (a < 3)
        val = val - ff * (s * st.dP[3 * a + ax]);
      else
        val = val + sixth * st.dF[a - 3];
    }
    dst[a * stride] = val;
  }
}

// MINB resident blocks of 128 threads per SM bound the registers per thread
// (4: 128 registers, 3: 168).
template <int MINB>
__global__ void __launch_bounds__(128, MINB)
    k3_collide_node(Ctx3 c, Fused3 fz, const double* __restrict__ f0, double* __restrict__ f1,
                    double* __restrict__ U, const double* __restrict__ u, int do_repair,
                    int store_all) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  NodeState3 st;
  node_prologue3(c, fz, U, u, do_repair, store_all, n, st);
  const cvlbm3d_problem& p = c.p;
  collide_dir3<0>(p, fz, st, f0, f1, N, n);
  collide_dir3<1>(p, fz, st, f0, f1, N, n);
  collide_dir3<2>(p, fz, st, f0, f1, N, n);
  collide_dir3<3>(p, fz, st, f0, f1, N, n);
  collide_dir3<4>(p, fz, st, f0, f1, N, n);
  collide_dir3<5>(p, fz, st, f0, f1, N, n);
}

// ---------------------------------------------------------------------------
// Wavefront form of the node work (node_variant 3): the moments, sweep and
// collide of chunks of one x-plane (the slowest index of the active order)
// in ONE persistent launch.  Blocks take work items from a ticket counter in
// the order  moments(w), sweep(w-1), collide(w-3)  for w = 0, 1, ..., so the
// collide of a plane re-reads f0 a few planes after the moments read it,
// while it is still in L2: f0 crosses HBM once per step instead of twice.
// Dependencies (whole planes): the sweep of plane i needs the moments of
// planes i-1..i+1 (+-x neighbours, same-plane +-y/z); the collide of plane i
// needs the sweep of planes i-2..i+2 (repair stencil +-2) - which also
// orders it after every read of its U by a neighbouring sweep.  A block
// waits only on items with lower tickets, which are held by running blocks,
// so the order cannot deadlock; every wait is bounded all the same, and a
// wait that runs out sets the timeout flag and the invalid flag and goes on
// (a wrong step, never a hung device).  Values other blocks of the launch
// write (U, collide-time u, swept u) are read through L2 only (ldx<true>).
// ---------------------------------------------------------------------------
struct Wave3 {
  const int4* items;         // [n_items] (stage, plane, first active id, end active id)
  int n_items, n_planes;
  const int32_t* chunks;     // [n_planes] items of one stage per plane
  int32_t* sync;             // [2 + 3*n_planes] ticket, timeout flag, done counters
};

// A wait gives up after this many polls (about a quarter of a second); the
// first wait that gives up makes every later wait of the launch return at
// once, so a broken dependency costs one bound, not one per item.
constexpr long long kWaveMaxSpins = 1LL << 20;

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
    k3_wave(Ctx3 c, Fused3 fz, Wave3 wv, const double* __restrict__ f0, double* __restrict__ f1,
            double* U, double* ucol, double* u, double* ustar, int* __restrict__ invalid,
            const double* clock, double t_host, int sweep_due, int do_repair, int store_all) {
  __shared__ int s_item;
  int* ticket = wv.sync;
  int* timeout = wv.sync + 1;
  int* done = wv.sync + 2;
  const cvlbm3d_problem& p = c.p;
  const int N = c.N;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // s_item is rewritten only after every thread has read it
    if (it >= wv.n_items) return;
    const int4 w = wv.items[it];
    const int stage = w.x, plane = w.y;
    if (stage > 0 && threadIdx.x == 0) {
      const int dep = stage - 1;
      const int r = stage == 1 ? 1 : 2;
      const int lo = plane - r < 0 ? 0 : plane - r;
      const int hi = plane + r >= wv.n_planes ? wv.n_planes - 1 : plane + r;
      const volatile int* gave_up = timeout;
      for (int pl = lo; pl <= hi && !*gave_up; ++pl) {
        const int want = wv.chunks[pl];
        const volatile int* d = done + dep * wv.n_planes + pl;
        long long spins = 0;
        while (*d < want && !*gave_up) {
          if (++spins > kWaveMaxSpins) {
            atomicExch(timeout, 1);
            atomicExch(invalid, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    __syncthreads();
    const int n = w.z + (int)threadIdx.x;
    if (n < w.w) {
      if (stage == 0) {
        moments_node3(c, f0, U, sweep_due ? ucol : u, ustar, invalid, sweep_due, n);
      } else if (stage == 1) {
        if (sweep_due) sweep_node3<true>(c, U, ucol, u, ustar, clock, t_host, n);
      } else {
        NodeState3 st;
        node_prologue3<true>(c, fz, U, u, do_repair, store_all, n, st);
        collide_dir3<0>(p, fz, st, f0, f1, N, n);
        collide_dir3<1>(p, fz, st, f0, f1, N, n);
        collide_dir3<2>(p, fz, st, f0, f1, N, n);
        collide_dir3<3>(p, fz, st, f0, f1, N, n);
        collide_dir3<4>(p, fz, st, f0, f1, N, n);
        collide_dir3<5>(p, fz, st, f0, f1, N, n);
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(done + stage * wv.n_planes + plane, 1);
  }
}

// -- link kernels -------------------------------------------------------------
constexpr int kGatherLanes = 16;  // lanes per link in the gather (12 components used)

// Value and gradients of the 12 components at a link from its <= 64
// characteristic samples, in slot order (_sparse_characteristic_gather,
// :2675-2700).  A block takes 8 consecutive links: their sample slots and
// weights are staged in shared memory with coalesced loads, then the 12
// lanes of a link read one 96-byte U_need row per sample, 16 samples per
// batch of independent loads.
constexpr int kGatherLinks = 128 / kGatherLanes;

__global__ void __launch_bounds__(128)
    k3_link_gather(Ctx3 c, Fused3 fz, double* __restrict__ char_state) {
  __shared__ int s_slot[kGatherLinks][kChar];
  __shared__ double s_w[kGatherLinks][4][kChar];
  const cvlbm3d_problem& p = c.p;
  const int L = p.n_links;
  const int ell0 = blockIdx.x * kGatherLinks;
  for (int t = threadIdx.x; t < kChar * kGatherLinks; t += blockDim.x) {
    const int mm = t / kGatherLinks, g = t % kGatherLinks;
    const int ell = ell0 + g;
    s_slot[g][mm] = ell < L ? fz.char_slot[(size_t)mm * L + ell] : -1;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      s_w[g][k][mm] = ell < L ? p.char_w[((size_t)k * kChar + mm) * L + ell] : 0.0;
  }
  __syncthreads();
  const int a = threadIdx.x % kGatherLanes;
  const int g = threadIdx.x / kGatherLanes;
  const int ell = ell0 + g;
  if (ell >= L || a >= kC3 || p.char_idx[ell] < 0) return;
  double v0 = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  constexpr int kChunk = 16;
#pragma unroll 1
  for (int m0 = 0; m0 < kChar; m0 += kChunk) {
    double uv[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      const int q = s_slot[g][m0 + k];
      uv[k] = q >= 0 ? fz.Uneed[(size_t)q * kC3 + a] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      const int mm = m0 + k;
      if (s_slot[g][mm] >= 0) {
        v0 += s_w[g][0][mm] * uv[k];
        gx += s_w[g][1][mm] * uv[k];
        gy += s_w[g][2][mm] * uv[k];
        gz += s_w[g][3][mm] * uv[k];
      }
    }
  }
  char_state[((size_t)0 * 12 + a) * L + ell] = v0;
  char_state[((size_t)1 * 12 + a) * L + ell] = gx;
  char_state[((size_t)2 * 12 + a) * L + ell] = gy;
  char_state[((size_t)3 * 12 + a) * L + ell] = gz;
}

// The same gather with 4 lanes per link, 3 components per lane and 32 links
// per block, from the link-major copies of the tables (char_slot_lm
// [n_links][64], char_w_lm [n_links][64][4]): a sample's slot and four
// weights are one 4-byte and two 16-byte loads shared by the link's lanes,
// every lane does useful work (the 16-lane form leaves 4 of 16 idle), and
// each lane runs 12 independent accumulations.  Each of the 48 sums runs
// over the samples in slot order, as in k3_link_gather (the same doubles).
constexpr int kGather4Lanes = 4;
constexpr int kGather4Links = 128 / kGather4Lanes;

__global__ void __launch_bounds__(128)
    k3_link_gather4(Ctx3 c, Fused3 fz, double* __restrict__ char_state) {
  // the block's 32 x 64 sample slots, staged with coalesced 16-byte loads so
  // that each chunk of samples waits for one load level (weights and U rows
  // together) instead of two (the slot, then its U row)
  __shared__ int4 s_slot4[kGather4Links * kChar / 4];
  const cvlbm3d_problem& p = c.p;
  const int L = p.n_links;
  const int ell0 = blockIdx.x * kGather4Links;
  const int nl = L - ell0 < kGather4Links ? L - ell0 : kGather4Links;
  const int4* src = reinterpret_cast<const int4*>(p.char_slot_lm + (size_t)ell0 * kChar);
  for (int t = threadIdx.x; t < kGather4Links * kChar / 4; t += blockDim.x)
    s_slot4[t] = t < nl * (kChar / 4) ? src[t] : make_int4(-1, -1, -1, -1);
  __syncthreads();
  const int lane = threadIdx.x % kGather4Lanes;
  const int g = threadIdx.x / kGather4Lanes;
  const int ell = ell0 + g;
  if (ell >= L || p.char_idx[ell] < 0) return;
  const int a0 = 3 * lane;
  const int* slot = reinterpret_cast<const int*>(s_slot4) + g * kChar;
  const double2* w2 = reinterpret_cast<const double2*>(p.char_w_lm + (size_t)ell * kChar * 4);
  double acc[3][4];
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[cc][k] = 0.0;
  constexpr int kChunk = 8;
#pragma unroll 1
  for (int m0 = 0; m0 < kChar; m0 += kChunk) {
    int q[kChunk];
    double2 wa[kChunk], wb[kChunk];
    double uv[kChunk][3];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      q[k] = slot[m0 + k];
      wa[k] = w2[2 * (m0 + k)];
      wb[k] = w2[2 * (m0 + k) + 1];
    }
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      const double* row = fz.Uneed + (size_t)(q[k] >= 0 ? q[k] : 0) * kC3 + a0;
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) uv[k][cc] = q[k] >= 0 ? row[cc] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      if (q[k] >= 0) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          acc[cc][0] += wa[k].x * uv[k][cc];
          acc[cc][1] += wa[k].y * uv[k][cc];
          acc[cc][2] += wb[k].x * uv[k][cc];
          acc[cc][3] += wb[k].y * uv[k][cc];
        }
      }
    }
  }
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int k = 0; k < 4; ++k) char_state[((size_t)k * 12 + a0 + cc) * L + ell] = acc[cc][k];
}

// Boundary value, F predictor, Newton normal solve and P(F_b) of one link;
// the results go to the link buffers (link_kind .. link_Pb), which the
// reference also exposes (three_d/curved_boundary_warp3d.py:4281-4337).
__global__ void __launch_bounds__(128)
    k3_link_prepare(Ctx3 c, Fused3 fz, const double* __restrict__ u, cvlbm3d_fields fl,
                    const double* clock, double t_host, double offset) {
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
  const int L = p.n_links, N = c.N;
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= L) return;
  const int ell = fz.order ? fz.order[slot] : slot;
  const double t = time_of(clock, t_host, offset);
  const int bid = p.link_bid[ell];
  const int kind = p.bc_kind[bid], mode = p.bc_mode[bid];
  int ck[3];
  for (int r = 0; r < 3; ++r) ck[r] = p.bc_comp_kind[r * kMaxIds3 + bid];
  const double* pp = p.bc_params + bid * 16;
  const double x = p.link_xb[ell], y = p.link_yb[ell], z = p.link_zb[ell];
  const double nx = p.link_nx[ell], ny = p.link_ny[ell], nz = p.link_nz[ell];
  const int n = p.link_p[ell];
  const int upid = p.link_up[ell];
  const double eta = p.link_eta[ell];
  double T[3];
  for (int r = 0; r < 3; ++r) T[r] = value3(r, mode, pp, x, y, z, nx, ny, nz, t, m.jf);
  if (p.dyn_enabled && p.dyn_enabled[ell] != 0)
    for (int r = 0; r < 3; ++r) T[r] = p.dyn_traction[(size_t)r * L + ell];
  double Fb[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double Pb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const bool anyN = ck[0] == kNeumann || ck[1] == kNeumann || ck[2] == kNeumann;
  if (anyN) {
    const double* Un = fz.Uneed + (size_t)fz.need_slot[n] * kC3;
    double F[9];
    for (int k = 0; k < 9; ++k) F[k] = Un[3 + k];
    if (p.recon == 2 || p.recon == 4) {
      if (upid >= 0) {
        const double* Uu = fz.Uneed + (size_t)fz.need_slot[upid] * kC3;
        for (int k = 0; k < 9; ++k) F[k] = Un[3 + k] + eta * (Un[3 + k] - Uu[3 + k]);
      }
      if (p.recon == 2 && p.has_tangent_lsq && p.lsq_valid[ell] != 0) {
        Frame3 fr = frame3(nx, ny, nz);
        double du1[3] = {0, 0, 0}, du2[3] = {0, 0, 0}, wt_abs = 0.0;
        for (int mm = 0; mm < kMaxLsq3; ++mm) {
          const int q = p.lsq_p[(size_t)ell * kMaxLsq3 + mm];
          if (q >= 0) {
            const double w1 = p.lsq_wt1[(size_t)ell * kMaxLsq3 + mm];
            const double w2 = p.lsq_wt2[(size_t)ell * kMaxLsq3 + mm];
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
    if (p.recon == 3 && p.has_char && p.char_idx[ell] >= 0)
      for (int k = 0; k < 9; ++k) F[k] = fl.char_state[((size_t)0 * 12 + 3 + k) * L + ell];
    else if (p.recon == 3)
      for (int k = 0; k < 9; ++k) F[k] = 0.0;
    for (int k = 0; k < 9; ++k) Fb[k] = F[k];
    if (ck[0] == kNeumann && ck[1] == kNeumann && ck[2] == kNeumann)
      solve_Fb3(F, nx, ny, nz, T, m, p.normal_solver, Fb);
    else if (ck[0] == kNeumann || ck[1] == kNeumann || ck[2] == kNeumann)
      solve_Fb3_mixed(F, nx, ny, nz, T, ck, m, p.normal_solver, Fb);
    const M3 P = piola3(Fb, m);
    for (int k = 0; k < 9; ++k) Pb[k] = P.v[k];
  }
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

__device__ __forceinline__ bool char_rows3(const cvlbm3d_problem& p, int ell) {
  return p.has_char && p.char_idx[ell] >= 0;
}

// BFL value of row `a` of one link (:3154-3241) with the outgoing populations
// taken from link_scratch and the post-stream f1.
__global__ void __launch_bounds__(128)
    k3_link_rows(Ctx3 c, Fused3 fz, double* __restrict__ f1, cvlbm3d_fields fl) {
  const cvlbm3d_problem& p = c.p;
  const int L = p.n_links, N = c.N;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)L * kC3) return;
  const int ell = (int)(t / kC3), a = (int)(t - (long long)ell * kC3);
  const int row = a < 3 ? a : (a - 3) / 3;
  const int ckr = fl.link_comp_kind[(size_t)row * L + ell];
  const bool anyN = fl.link_comp_kind[ell] == kNeumann ||
                    fl.link_comp_kind[(size_t)L + ell] == kNeumann ||
                    fl.link_comp_kind[2 * (size_t)L + ell] == kNeumann;
  // rows the characteristic closure overwrites are written by k3_link_char
  if (anyN && ckr == kNeumann && char_rows3(p, ell)) return;
  const int n = p.link_p[ell], upid = p.link_up[ell], qo = p.link_q[ell];
  const int qi = opp3(qo);
  double eta = p.link_eta[ell];
  if (p.recon == 1) eta = 0.5;
  const double din[3] = {(double)dx3(qi), (double)dy3(qi), (double)dz3(qi)};
  const double cc = p.c;
  double D = 1.0, S = 0.0;
  if (ckr == kDirichlet) {
    const double Tr = fl.link_bv[(size_t)row * L + ell];
    if (a < 3) {
      D = -1.0;
      S = fl.link_bv[(size_t)a * L + ell] / 3.0;
    } else {
      const int col = (a - 3) - row * 3;
      S = -din[col] * Tr / cc;
    }
  } else {
    if (a < 3) {
      const double* Pb = fl.link_Pb;
      S = -(din[0] * Pb[(size_t)(3 * a) * L + ell] + din[1] * Pb[(size_t)(3 * a + 1) * L + ell] +
            din[2] * Pb[(size_t)(3 * a + 2) * L + ell]) / cc;
    } else {
      D = -1.0;
      S = fl.link_Fb[(size_t)(a - 3) * L + ell] / 3.0;
    }
  }
  const double fo = fz.scratch[(size_t)ell * kC3 + a];
  double val;
  if (eta >= 0.5) {
    const double fi = upid >= 0 ? f1[(size_t)(qi * kC3 + a) * N + upid]
                                : fz.scratch[(size_t)fz.partner[ell] * kC3 + a];
    const double al = 1.0 / (2.0 * eta);
    val = al * (D * fo + S) + (1.0 - al) * fi;
  } else {
    const double up = upid >= 0 ? f1[(size_t)(qo * kC3 + a) * N + n] : fo;
    val = D * (2.0 * eta * fo + (1.0 - 2.0 * eta) * up) + S;
  }
  f1[(size_t)(qi * kC3 + a) * N + n] = val;
}

// Characteristic rows (:2812-2884) of links with a Neumann row.
__global__ void __launch_bounds__(64)
    k3_link_char(Ctx3 c, Fused3 fz, double* __restrict__ f1, cvlbm3d_fields fl) {
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
  const int L = p.n_links, N = c.N;
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= L) return;
  const int ell = fz.order ? fz.order[slot] : slot;
  if (!char_rows3(p, ell)) return;
  int ck[3];
  for (int r = 0; r < 3; ++r) ck[r] = fl.link_comp_kind[(size_t)r * L + ell];
  if (!(ck[0] == kNeumann || ck[1] == kNeumann || ck[2] == kNeumann)) return;
  const int n = p.link_p[ell], qi = opp3(p.link_q[ell]);
  const double din[3] = {(double)dx3(qi), (double)dy3(qi), (double)dz3(qi)};
  double Ub[12], G[3][12];
  const double* Un = fz.Uneed + (size_t)fz.need_slot[n] * kC3;
  for (int a = 0; a < 3; ++a)
    Ub[a] = ck[a] == kDirichlet ? fl.link_bv[(size_t)a * L + ell] : Un[a];
  for (int k = 0; k < 9; ++k) Ub[3 + k] = fl.link_Fb[(size_t)k * L + ell];
  if (state_det3(Ub) <= m.jf) *fl.invalid = 1;
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 12; ++a) G[d][a] = fl.char_state[((size_t)(1 + d) * 12 + a) * L + ell];
  double out[12];
  char_population3(Ub, G[0], G[1], G[2], din, p.link_eta[ell], p.dt, p.c, p, m, p.omega, out);
  for (int a = 0; a < 12; ++a) {
    const int row = a < 3 ? a : (a - 3) / 3;
    if (ck[row] == kNeumann) f1[(size_t)(qi * kC3 + a) * N + n] = out[a];
  }
}

}  // namespace
