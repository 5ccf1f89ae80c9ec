// D3Q6x12 step, fused form.  Included by cvlbm3d.cu (shares Ctx3 and the
// per-link helpers).
//
// Node kernels (reference raster order of the active nodes):
//   k3_moments   f0 -> U (all 12 components), collide-time u into `ucol`
//                (u_next), invalid flag; when no sweep is due, u and u* too
//   k3_sweep     u_swept -> u and the trapezoidal u* update, from U and ucol
//                of the node and its six neighbours plus cut-point anchors
//   k3_prep      F repair preparation from U and the swept u (+-2 star
//                stencil): P(F), and where the repair applies the deltas of
//                P and F; the post-step U of nodes that links read goes to
//                U_need, one 96-byte row each
//   k3_collide   f0 again (six warps per 32 nodes, one per direction, no
//                barriers): BGK collision with damping/source and the repair
//                delta, push streaming to f1; a population whose neighbour is
//                not active leaves through a cut link and is kept per link
//                (link_scratch) for the link kernels
// Per active node this reads f0 twice and writes f1 once (the f0 re-read of
// k3_collide is what a single-pass 3-D fusion would save; its 3-deep halo
// does not fit shared memory), plus U, u, u* and the 27 repair doubles:
// about 2.8 KB per node against the algorithmic 1.2 KB, every kernel a
// stream of independent coalesced loads.
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

__global__ void __launch_bounds__(256) k3_moments(Ctx3 c, const double* __restrict__ f0,
                                                  double* __restrict__ U,
                                                  double* __restrict__ ucol,
                                                  double* __restrict__ ustar,
                                                  int* __restrict__ invalid, int sweep_due) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
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
__global__ void __launch_bounds__(256) k3_sweep(Ctx3 c, const double* __restrict__ U,
                                                const double* __restrict__ ucol,
                                                double* __restrict__ u,
                                                double* __restrict__ ustar, const double* clock,
                                                double t_host) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
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
    for (int comp = 0; comp < 3; ++comp) {
      if (!(force_all || p.bc_comp_kind[comp * kMaxIds3 + bid] == kDirichlet)) continue;
      const double ub = disp3(mode, pp, comp, x, y, z, time);
      const double* F = U + (size_t)(3 + 3 * comp) * N;
      double e0 = F[n], e1 = F[(size_t)N + n], e2 = F[2 * (size_t)N + n];
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
  for (int k = 0; k < 9; ++k) Fs[k] = Ub[(size_t)k * N + n];
#pragma unroll
  for (int q = 0; q < kQ3; ++q) {
    const int m = p.neighbor[(size_t)q * N + n];
    if (m < 0) continue;
    const double ddx = (double)dx3(q) * p.dx, ddy = (double)dy3(q) * p.dy,
                 ddz = (double)dz3(q) * p.dz;
    const double g0 = 0.5 * ((Fs[0] + Ub[m] - 2.0) * ddx + (Fs[1] + Ub[N + m]) * ddy +
                             (Fs[2] + Ub[2 * (size_t)N + m]) * ddz);
    const double g1 = 0.5 * ((Fs[3] + Ub[3 * (size_t)N + m]) * ddx +
                             (Fs[4] + Ub[4 * (size_t)N + m] - 2.0) * ddy +
                             (Fs[5] + Ub[5 * (size_t)N + m]) * ddz);
    const double g2 = 0.5 * ((Fs[6] + Ub[6 * (size_t)N + m]) * ddx +
                             (Fs[7] + Ub[7 * (size_t)N + m]) * ddy +
                             (Fs[8] + Ub[8 * (size_t)N + m] - 2.0) * ddz);
    r[0] += ucol[m] - g0;
    r[1] += ucol[(size_t)N + m] - g1;
    r[2] += ucol[2 * (size_t)N + m] - g2;
    d[0] += 1.0;
    d[1] += 1.0;
    d[2] += 1.0;
  }
  const double hdt = 0.5 * p.dt;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const double uo = ucol[(size_t)comp * N + n];
    double un = uo;
    if (d[comp] > 0.0) un = uo + p.relax * (r[comp] / d[comp] - uo);
    u[(size_t)comp * N + n] = un;
    ustar[(size_t)comp * N + n] = (uo + hdt * U[(size_t)comp * N + n]) + (un - uo);
  }
}

// F repair preparation (three_d/curved_boundary_warp3d.py:2543-2672), one
// thread per node, from U (the moments k3_moments stored) and the swept u:
// P(F), and where the repair applies (det of the repaired F above the floor)
// P(F_repaired) - P(F) and F_repaired - F.  rs holds Po[9][N], dP[9][N],
// dF[9][N] followed by one flag byte per node.  Also writes the U_need row
// and, on the last step of a run, the repaired F into U.
__global__ void __launch_bounds__(128)
    k3_prep(Ctx3 c, Fused3 fz, double* __restrict__ U, const double* __restrict__ u,
            double* __restrict__ rs, int do_repair, int store_all) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm3d_problem& p = c.p;
  const Mat& m = c.m;
  double F[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) F[k] = U[(size_t)(3 + k) * N + n];
  const M3 Po = piola3(F, m);
  double* Pog = rs;
  double* dPg = rs + 9 * (size_t)N;
  double* dFg = rs + 18 * (size_t)N;
  uint8_t* flag = reinterpret_cast<uint8_t*>(rs + 27 * (size_t)N);
#pragma unroll
  for (int k = 0; k < 9; ++k) Pog[(size_t)k * N + n] = Po.v[k];
  bool repaired = false;
  double nn[9];
  if (do_repair) {
    const double beta = fmax(0.0, fmin(1.0, p.blend));
    const double h[3] = {p.dx, p.dy, p.dz};
#pragma unroll
    for (int comp = 0; comp < 3; ++comp)
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const double g = du_axis3(u + (size_t)comp * N, p.neighbor, N, n, ax, ax + 3, h[ax]);
        const double t = comp == ax ? 1.0 + g : g;
        nn[3 * comp + ax] = F[3 * comp + ax] + beta * (t - F[3 * comp + ax]);
      }
    if (det3v(nn) > m.jf) {
      repaired = true;
      const M3 Pn = piola3(nn, m);
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        dPg[(size_t)k * N + n] = Pn.v[k] - Po.v[k];
        dFg[(size_t)k * N + n] = nn[k] - F[k];
      }
      if (store_all) {
#pragma unroll
        for (int k = 0; k < 9; ++k) U[(size_t)(3 + k) * N + n] = nn[k];
      }
    }
  }
  flag[n] = repaired ? 1 : 0;
  const int slot = fz.need_slot[n];
  if (slot >= 0) {
    double* row = fz.Uneed + (size_t)slot * kC3;
    row[0] = U[n];
    row[1] = U[(size_t)N + n];
    row[2] = U[2 * (size_t)N + n];
#pragma unroll
    for (int k = 0; k < 9; ++k) row[3 + k] = repaired ? nn[k] : F[k];
  }
}

// Collision + repair delta + push streaming (three_d/curved_boundary_warp3d.py
// :2192-2330).  32 consecutive nodes x 6 warps, warp q = direction q (lane =
// node), so every population load and store is a coalesced 256-byte row; the
// moments come from U (bitwise the sums k3_moments stored), P(F) and the
// repair deltas from k3_prep.  No shared memory and no block barrier.
constexpr int kCN = 32;  // nodes per collide block (one per lane)

__global__ void __launch_bounds__(kQ3 * kCN)
    k3_collide(Ctx3 c, Fused3 fz, const double* __restrict__ f0, double* __restrict__ f1,
               const double* __restrict__ U, const double* __restrict__ rs) {
  const int N = c.N;
  const cvlbm3d_problem& p = c.p;
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  const int n = blockIdx.x * kCN + lane;
  if (n >= N) return;
  double v[kC3], S[kC3];
#pragma unroll
  for (int a = 0; a < kC3; ++a) v[a] = f0[(size_t)(q * kC3 + a) * N + n];
#pragma unroll
  for (int a = 0; a < kC3; ++a) S[a] = U[(size_t)a * N + n];
  const int nq = p.neighbor[(size_t)q * N + n];
  const bool repaired = reinterpret_cast<const uint8_t*>(rs + 27 * (size_t)N)[n] != 0;
  M3 Po;
#pragma unroll
  for (int k = 0; k < 9; ++k) Po.v[k] = rs[(size_t)k * N + n];
  int ell = -1;
  if (nq < 0) {
    for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
      const int e = p.node_link_list[k];
      if (p.link_q[e] == q) ell = e;
    }
  }
  const double k3c = 3.0 / p.c, sixth = 1.0 / 6.0, om = p.omega;
  const double sw = p.dt * (2.0 - om) * (1.0 / 12.0);
  const double ff = 0.5 / p.c;
  const double sx = (double)dx3(q), sy = (double)dy3(q), sz = (double)dz3(q);
  const double* dP = rs + 9 * (size_t)N;
  const double* dF = rs + 18 * (size_t)N;
#pragma unroll
  for (int a = 0; a < kC3; ++a) {
    const double old = v[a];
    const double fe = feq3(q, a, S, Po, k3c, sixth);
    double val = old + om * (fe - old) + sw * source_comp3(a, p.source_mode, p.source, S);
    if (repaired) {
      if (a < 3)
        val = val - ff * (sx * dP[(size_t)(3 * a) * N + n] + sy * dP[(size_t)(3 * a + 1) * N + n] +
                          sz * dP[(size_t)(3 * a + 2) * N + n]);
      else
        val = val + sixth * dF[(size_t)(a - 3) * N + n];
    }
    if (nq >= 0)
      f1[(size_t)(q * kC3 + a) * N + nq] = val;
    else if (ell >= 0)
      fz.scratch[(size_t)ell * kC3 + a] = val;
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
  __shared__ double s_w[4][kChar][kGatherLinks];
  const cvlbm3d_problem& p = c.p;
  const int L = p.n_links;
  const int ell0 = blockIdx.x * kGatherLinks;
  for (int t = threadIdx.x; t < kChar * kGatherLinks; t += blockDim.x) {
    const int mm = t / kGatherLinks, g = t % kGatherLinks;
    const int ell = ell0 + g;
    s_slot[g][mm] = ell < L ? fz.char_slot[(size_t)mm * L + ell] : -1;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      s_w[k][mm][g] = ell < L ? p.char_w[((size_t)k * kChar + mm) * L + ell] : 0.0;
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
        v0 += s_w[0][mm][g] * uv[k];
        gx += s_w[1][mm][g] * uv[k];
        gy += s_w[2][mm][g] * uv[k];
        gz += s_w[3][mm][g] * uv[k];
      }
    }
  }
  char_state[((size_t)0 * 12 + a) * L + ell] = v0;
  char_state[((size_t)1 * 12 + a) * L + ell] = gx;
  char_state[((size_t)2 * 12 + a) * L + ell] = gy;
  char_state[((size_t)3 * 12 + a) * L + ell] = gz;
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
