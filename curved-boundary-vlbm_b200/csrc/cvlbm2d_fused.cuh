// D2Q4x6 step, fused form: one tiled node kernel plus one cooperative link
// kernel per time step.  Included by cvlbm2d.cu (shares Ctx2 and helpers).
//
// Node kernel (k_fused2): a 32x16 tile of nodes per 512-thread block.
//   A  every node of the tile plus a 3-node halo: moments and collide-time
//      displacement u from f0, u* into shared memory (halo moments are
//      recomputed from f0 through L2 instead of being exchanged);
//   B  displacement sweep with cut-point anchors on tile+2;
//   C  owner nodes: F repair (needs swept u at +-2), BGK collision, repair
//      delta, push-streaming of f_post to active neighbours.  A population
//      whose neighbour is not active leaves through a cut link: it is stored
//      per link (link_scratch) for the link kernel.
// Per active node and step the node kernel reads f0 and u* once and writes
// f1 and u* once (416 bytes), plus the fields the link stencils read.
//
// Link kernel (k_links2g): 16 lanes cooperate on one cut link: component-wise
// stencil gathers in parallel, Newton on one lane, flux tangents split over
// two lanes, one population row per lane.  With `fused` set the link reads
// the populations it needs from link_scratch and f1 (post-stream) instead of
// fpost.
#pragma once

namespace {

constexpr int kTX = 32, kH = 3;
constexpr int kRX = kTX + 2 * kH;  // region row length (tile + halo 3)
constexpr int kSX = kTX + 4;       // sweep-region row length (tile + 2)

struct Fused2 {
  const int32_t* tiles;        // [n_tiles] tile ids with at least one active node
  int32_t n_tiles, tiles_j;    // tiles along j
  const uint8_t* need;         // [N] node fields read by some link stencil
  const int32_t* partner;      // [n_links] link at the same node in direction q_in, or -1
  double* scratch;             // [6*n_links] f_post leaving through each link
  int32_t store_all;           // write U and u for every active node
};

// Moments of node n (reference order: for q: for a) with the collision's
// source / damping half step (two_d/curved_boundary_warp.py:1735-1756).
__device__ __forceinline__ void moments2(const cvlbm2d_problem& p, const double* __restrict__ f0,
                                         int N, int n, double* S) {
#pragma unroll
  for (int a = 0; a < 6; ++a) S[a] = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int a = 0; a < 6; ++a) S[a] += f0[(size_t)(q * 6 + a) * N + n];
  const double hdt = 0.5 * p.dt;
  if (p.source_mode == kSrcConstant) {
#pragma unroll
    for (int a = 0; a < 6; ++a) S[a] += hdt * p.source[a];
  } else if (p.source_mode == kSrcDamping) {
    double den = 1.0 + hdt * p.source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
}

// moments2 with the per-problem constants of Ctx2 (the same doubles)
__device__ __forceinline__ void moments2c(const Ctx2& c, const double* __restrict__ f0, int n,
                                          double* S) {
  const int N = c.N;
#pragma unroll
  for (int a = 0; a < 6; ++a) S[a] = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int a = 0; a < 6; ++a) S[a] += f0[(size_t)(q * 6 + a) * N + n];
  if (c.p.source_mode == kSrcConstant) {
#pragma unroll
    for (int a = 0; a < 6; ++a) S[a] += c.hdt * c.p.source[a];
  } else if (c.p.source_mode == kSrcDamping) {
    S[0] = S[0] / c.den;
    S[1] = S[1] / c.den;
  }
}

// Region flags in shared memory: bit 0 active, bit 1 holds a cut link
constexpr int kFlagLinks = 2;

template <int TY, bool STAGE = false>
constexpr size_t fused_smem2() {
  return sizeof(double) * (6 * kRX * (TY + 2 * kH) + 2 * kSX * (TY + 4)) +
         sizeof(double) * ((kRX * (TY + 2 * kH) + 1) / 2) +  // int flags, padded to 8 bytes
         (STAGE ? sizeof(double) * 24 * kTX * TY : 0);
}

// One tile of the fused step (phases A-C above); `tile` is a tile id of the
// problem's tile list.  Every thread of the block calls it; it returns
// early only after the last block-wide barrier.  PRE: the collide-time
// moments of every active node were written by k_mom2 into `mom` this step
// ([8][N]: U (6), collide-time u (2)), so phase A reads them instead of
// summing populations (the same doubles: k_mom2 evaluates the same sums).
template <int TY, bool PRE = false, bool STAGE = false>
__device__ __forceinline__ void fused2_tile(
    const Ctx2& c, const Fused2& fz, int tile, const double* __restrict__ f0,
    double* __restrict__ f1, double* __restrict__ Ug, double* __restrict__ ug,
    const double* __restrict__ ustar, double* __restrict__ ustar_out, int* __restrict__ invalid,
    const double* clock, double t_host, int do_sweep, int do_repair, double* smem2,
    const double* __restrict__ mom = nullptr) {
  constexpr int kTY = TY;
  constexpr int kRN = kRX * (TY + 2 * kH);
  constexpr int kSN = kSX * (TY + 4);
  double(*sF)[kRN] = reinterpret_cast<double(*)[kRN]>(smem2);            // collide-time F
  double(*sU)[kRN] = reinterpret_cast<double(*)[kRN]>(smem2 + 4 * kRN);  // collide-time u
  double(*sN)[kSN] = reinterpret_cast<double(*)[kSN]>(smem2 + 6 * kRN);  // swept u, tile+2
  int* sA = reinterpret_cast<int*>(smem2 + 6 * kRN + 2 * kSN);           // active flags
  // STAGE: the owned nodes' populations, kept from phase A for phase C
  double* sfo = smem2 + 6 * kRN + 2 * kSN + (kRN + 1) / 2;  // [24][kTX*TY]
  constexpr int kTN = kTX * TY;

  const cvlbm2d_problem& p = c.p;
  const int N = c.N, nx = p.nx, ny = p.ny;
  const int i0 = (tile / fz.tiles_j) * kTY, j0 = (tile % fz.tiles_j) * kTX;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i = i0 + ty, j = j0 + tx;
  const bool own = i < nx && j < ny;
  const int n = i * ny + j;
  const bool own_act = own && p.active[n] != 0;
  const int r_own = (ty + kH) * kRX + tx + kH;

  // -- A: region moments -----------------------------------------------------
  // (loads whose latency would otherwise sit in phase B or C start here)
  const double time_mid = time_of(clock, t_host, c.hdt);
  double S[6];
  double ucol0 = 0.0, ucol1 = 0.0;
  int own_flag = 0;
  bool own_need = false;
  if (own_act) {
    own_flag = 1 | (p.node_link_start[n + 1] > p.node_link_start[n] ? kFlagLinks : 0);
    own_need = fz.store_all || fz.need[n];
    if constexpr (PRE) {
#pragma unroll
      for (int a = 0; a < 6; ++a) S[a] = mom[(size_t)a * N + n];
      ucol0 = mom[6 * (size_t)N + n];
      ucol1 = mom[7 * (size_t)N + n];
    } else if constexpr (STAGE) {
      // moments2c with every population also kept in shared memory
#pragma unroll
      for (int a = 0; a < 6; ++a) S[a] = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          const double v = f0[(size_t)(q * 6 + a) * N + n];
          sfo[(q * 6 + a) * kTN + threadIdx.x] = v;
          S[a] += v;
        }
      if (p.source_mode == kSrcConstant) {
#pragma unroll
        for (int a = 0; a < 6; ++a) S[a] += c.hdt * p.source[a];
      } else if (p.source_mode == kSrcDamping) {
        S[0] = S[0] / c.den;
        S[1] = S[1] / c.den;
      }
      ucol0 = ustar[n] + c.hdt * S[0];
      ucol1 = ustar[N + n] + c.hdt * S[1];
    } else {
      moments2c(c, f0, n, S);
      ucol0 = ustar[n] + c.hdt * S[0];
      ucol1 = ustar[N + n] + c.hdt * S[1];
    }
  }
  for (int r = threadIdx.x; r < kRN; r += blockDim.x) {
    const int ri = r / kRX, rj = r - ri * kRX;
    const bool interior = ri >= kH && ri < kH + kTY && rj >= kH && rj < kH + kTX;
    if (interior) continue;
    const int gi = i0 - kH + ri, gj = j0 - kH + rj;
    const bool inb = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
    const int m = gi * ny + gj;
    const int act = inb ? p.active[m] : 0;
    sA[r] = act ? 1 | (p.node_link_start[m + 1] > p.node_link_start[m] ? kFlagLinks : 0) : 0;
    if (act) {
      if constexpr (PRE) {
#pragma unroll
        for (int k = 0; k < 4; ++k) sF[k][r] = mom[(size_t)(2 + k) * N + m];
        sU[0][r] = mom[6 * (size_t)N + m];
        sU[1][r] = mom[7 * (size_t)N + m];
      } else {
        double Sh[6];
        moments2c(c, f0, m, Sh);
        sF[0][r] = Sh[2];
        sF[1][r] = Sh[3];
        sF[2][r] = Sh[4];
        sF[3][r] = Sh[5];
        sU[0][r] = ustar[m] + c.hdt * Sh[0];
        sU[1][r] = ustar[N + m] + c.hdt * Sh[1];
      }
    } else {
      sF[0][r] = sF[1][r] = sF[2][r] = sF[3][r] = 0.0;
      sU[0][r] = sU[1][r] = 0.0;
    }
  }
  sA[r_own] = own_flag;
  if (own_act) {
    sF[0][r_own] = S[2];
    sF[1][r_own] = S[3];
    sF[2][r_own] = S[4];
    sF[3][r_own] = S[5];
    sU[0][r_own] = ucol0;
    sU[1][r_own] = ucol1;
  } else {
    sF[0][r_own] = sF[1][r_own] = sF[2][r_own] = sF[3][r_own] = 0.0;
    sU[0][r_own] = sU[1][r_own] = 0.0;
  }
  __syncthreads();

  // -- B: displacement sweep on tile+2 (two_d/curved_boundary_warp.py:3275-3518)
  for (int s = threadIdx.x; s < kSN; s += blockDim.x) {
    const int si = s / kSX, sj = s - si * kSX;
    const int r = (si + 1) * kRX + sj + 1;
    if (!sA[r]) {
      sN[0][s] = 0.0;
      sN[1][s] = 0.0;
      continue;
    }
    if (!do_sweep) {
      sN[0][s] = sU[0][r];
      sN[1][s] = sU[1][r];
      continue;
    }
    const int gi = i0 - 2 + si, gj = j0 - 2 + sj;
    const int m = gi * ny + gj;
    double diag = 0.0, rx = 0.0, ry = 0.0;
    const int k0 = (sA[r] & kFlagLinks) ? p.node_link_start[m] : 0;
    const int k1 = (sA[r] & kFlagLinks) ? p.node_link_start[m + 1] : 0;
    for (int k = k0; k < k1; ++k) {
      const int ell = p.node_link_list[k];
      const int bid = p.link_bid[ell];
      if (p.disp_bid >= 0) {
        if (bid != p.disp_bid) continue;
      } else if (p.bc_kind[bid] != kDirichlet) {
        continue;
      }
      const double* pp = p.bc_params + bid * 8;
      const int mode = p.bc_mode[bid];
      const double xb = p.link_xb[ell], yb = p.link_yb[ell];
      const double nxb = p.link_nx[ell], nyb = p.link_ny[ell];
      double ub0 = 0.0, ub1 = 0.0;
      if (mode == 1) {
        ub0 = time_mid * value2(0, mode, pp, xb, yb, nxb, nyb, 0.0);
        ub1 = time_mid * value2(1, mode, pp, xb, yb, nxb, nyb, 0.0);
      } else if (mode == 6) {
        double at = time_mid;
        if (pp[6] > 0.0 && at > pp[6]) at = pp[6];
        ub0 = at * value2(0, mode, pp, xb, yb, nxb, nyb, 0.0);
        ub1 = at * value2(1, mode, pp, xb, yb, nxb, nyb, 0.0);
      }
      const double dbx = xb - ((double)gi + 0.5) * p.dx;
      const double dby = yb - ((double)gj + 0.5) * p.dy;
      const double tx_ = ub0 - ((sF[0][r] - 1.0) * dbx + sF[1][r] * dby);
      const double ty_ = ub1 - (sF[2][r] * dbx + (sF[3][r] - 1.0) * dby);
      const double w2 = p.weight * p.weight;
      diag = diag + w2;
      rx = rx + w2 * tx_;
      ry = ry + w2 * ty_;
    }
    const double hx = 0.5 * p.dx, hy = 0.5 * p.dy;
    if (sA[r + kRX]) {  // +x (i+1)
      const int o = r + kRX;
      rx += sU[0][o] - hx * ((sF[0][r] - 1.0) + (sF[0][o] - 1.0));
      ry += sU[1][o] - hx * (sF[2][r] + sF[2][o]);
      diag += 1.0;
    }
    if (sA[r - kRX]) {  // -x
      const int o = r - kRX;
      rx += sU[0][o] + hx * ((sF[0][o] - 1.0) + (sF[0][r] - 1.0));
      ry += sU[1][o] + hx * (sF[2][o] + sF[2][r]);
      diag += 1.0;
    }
    if (sA[r + 1]) {  // +y
      const int o = r + 1;
      rx += sU[0][o] - hy * (sF[1][r] + sF[1][o]);
      ry += sU[1][o] - hy * ((sF[3][r] - 1.0) + (sF[3][o] - 1.0));
      diag += 1.0;
    }
    if (sA[r - 1]) {  // -y
      const int o = r - 1;
      rx += sU[0][o] + hy * (sF[1][o] + sF[1][r]);
      ry += sU[1][o] + hy * ((sF[3][o] - 1.0) + (sF[3][r] - 1.0));
      diag += 1.0;
    }
    double u0 = sU[0][r], u1 = sU[1][r];
    if (diag > 0.0) {
      u0 = u0 + p.relax * (rx / diag - u0);
      u1 = u1 + p.relax * (ry / diag - u1);
    }
    sN[0][s] = u0;
    sN[1][s] = u1;
  }
  __syncthreads();
  if (!own_act) return;

  // -- C: repair, collision, streaming (owner) -------------------------------
  const int s_own = (ty + 2) * kSX + tx + 2;
  const double un0 = sN[0][s_own], un1 = sN[1][s_own];
  const Mat& m = c.m;
  double Fn[4] = {S[2], S[3], S[4], S[5]};
  bool repaired = false;
  if (do_repair) {
    bool ok = true;
    if (p.interior_only) {
      ok = i > 0 && i + 1 < nx && j > 0 && j + 1 < ny && sA[r_own - kRX] && sA[r_own + kRX] &&
           sA[r_own - 1] && sA[r_own + 1];
    }
    if (ok) {
      // one-sided / centred derivatives of the swept displacement
      // (two_d/curved_boundary_warp.py:3213-3272) on the shared tile+2 window
      double g[2][2];
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        const int rs = ax == 0 ? kRX : 1, ss = ax == 0 ? kSX : 1;
        const int ii = ax == 0 ? i : j, nn = ax == 0 ? nx : ny;
        const double h = ax == 0 ? p.dx : p.dy;
        const bool am = ii > 0 && sA[r_own - rs], ap = ii + 1 < nn && sA[r_own + rs];
#pragma unroll
        for (int comp = 0; comp < 2; ++comp) {
          const double* w = sN[comp];
          double d;
          if (am && ap) {
            d = (w[s_own + ss] - w[s_own - ss]) / (2.0 * h);
          } else if (ap) {
            if (ii + 2 < nn && sA[r_own + 2 * rs])
              d = (-3.0 * w[s_own] + 4.0 * w[s_own + ss] - w[s_own + 2 * ss]) / (2.0 * h);
            else
              d = (w[s_own + ss] - w[s_own]) / h;
          } else if (am) {
            if (ii > 1 && sA[r_own - 2 * rs])
              d = (3.0 * w[s_own] - 4.0 * w[s_own - ss] + w[s_own - 2 * ss]) / (2.0 * h);
            else
              d = (w[s_own] - w[s_own - ss]) / h;
          } else {
            d = 0.0;
          }
          g[comp][ax] = d;
        }
      }
      const double t11 = 1.0 + g[0][0], t12 = g[0][1], t21 = g[1][0], t22 = 1.0 + g[1][1];
      double alpha = fmax(0.0, fmin(1.0, p.blend));
      for (int it = 0; it < 10; ++it) {
        Fn[0] = S[2] + alpha * (t11 - S[2]);
        Fn[1] = S[3] + alpha * (t12 - S[3]);
        Fn[2] = S[4] + alpha * (t21 - S[4]);
        Fn[3] = S[5] + alpha * (t22 - S[5]);
        if (Fn[0] * Fn[3] - Fn[1] * Fn[2] > m.jf) break;
        alpha = 0.5 * alpha;
      }
      repaired = true;
    }
  }
  const double J = S[2] * S[5] - S[3] * S[4];
  if (J <= m.jf) *invalid = 1;
  const P2 Po = piola2(S[2], S[3], S[4], S[5], m);
  const double k2c = c.k2c, om = p.omega, sw = p.dt * (2.0 - om) * 0.125;
  const double ff = c.ff, qt = 0.25;
  // Per-node constants of the collision.  The reference's equilibrium
  // 0.25*(U_a + (2/c)*(cx*phix_a + cy*phiy_a)) has cx, cy in {0, +-1}: a
  // product with an exact zero adds nothing to a finite sum and a product
  // with -1 is a negation, so with g = (2/c)*phi along the direction's axis
  // it is 0.25*(U_a +- g_a), the same double (up to the sign of an exact
  // zero).  The source and repair terms do not depend on q and are formed
  // once per component.
  P2 dP{0.0, 0.0, 0.0, 0.0};
  if (repaired) {
    const P2 Pn = piola2(Fn[0], Fn[1], Fn[2], Fn[3], m);
    dP = {Pn.a - Po.a, Pn.b - Po.b, Pn.c - Po.c, Pn.d - Po.d};
  }
  // destinations of the four directions: a neighbour node, a cut link's
  // scratch row, or nowhere (a cut link without scratch)
  int dst[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int cq = cx2(q), cy = cy2(q);
    if (sA[r_own + cq * kRX + cy] != 0) {
      dst[q] = n + cq * ny + cy;
    } else {
      int ell_out = -1;
      for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
        const int e = p.node_link_list[k];
        if (p.link_q[e] == q) ell_out = e;
      }
      dst[q] = ell_out >= 0 ? -2 - ell_out : -1;
    }
  }
  const bool add_src = p.source_mode != kSrcNone;
  const bool add_src_f = p.source_mode == kSrcConstant;  // damping: rows 2-5 get +0
  // collision, repair delta and push-streaming, component by component
  // (f0 of the owner is re-read from L1: the tile loaded it in phase A)
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    // g along x and y for this component (zero rows: 3, 5 along x; 2, 4 along y)
    const double gx = a == 0 ? k2c * -Po.a : a == 1 ? k2c * -Po.c : a == 2 ? k2c * -S[0]
                    : a == 4 ? k2c * -S[1] : 0.0;
    const double gy = a == 0 ? k2c * -Po.b : a == 1 ? k2c * -Po.d : a == 3 ? k2c * -S[0]
                    : a == 5 ? k2c * -S[1] : 0.0;
    const bool hx = a == 0 || a == 1 || a == 2 || a == 4;
    const bool hy = a == 0 || a == 1 || a == 3 || a == 5;
    const double swB = (add_src && (a < 2 || add_src_f))
                           ? sw * source_comp(a, p.source_mode, p.source, S) : 0.0;
    // repair: ff*(cx*dP_a1 + cy*dP_a2) for the velocity rows, qt*(Fn - F) for the F rows
    const double tx = a == 0 ? ff * dP.a : a == 1 ? ff * dP.c : 0.0;
    const double ty = a == 0 ? ff * dP.b : a == 1 ? ff * dP.d : 0.0;
    const double rF = a >= 2 ? qt * (Fn[a - 2] - S[a]) : 0.0;
    const double Ua = S[a];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int cq = cx2(q), cy = cy2(q);
      const bool neg = cq < 0 || cy < 0;
      const bool has_g = cq != 0 ? hx : hy;
      const double g = cq != 0 ? gx : gy;
      double old;
      if constexpr (STAGE)
        old = sfo[(q * 6 + a) * kTN + threadIdx.x];
      else
        old = f0[(size_t)(q * 6 + a) * N + n];
      const double fe = 0.25 * (has_g ? (neg ? Ua - g : Ua + g) : Ua);
      double v = old + om * (fe - old);
      if (add_src && (a < 2 || add_src_f)) v = v + swB;
      if (repaired) {
        if (a < 2) {
          const double t = cq != 0 ? tx : ty;
          v = neg ? v + t : v - t;
        } else {
          v = v + rF;
        }
      }
      const int d = dst[q];
      if (d >= 0)
        f1[(size_t)(q * 6 + a) * N + d] = v;
      else if (d <= -2)
        fz.scratch[(size_t)(-2 - d) * 6 + a] = v;
    }
  }
  const double dt = p.dt;
  // u* goes to the other buffer: neighbouring tiles read this node's old u*
  // in their halo during the same launch
  ustar_out[n] = (ucol0 + 0.5 * dt * S[0]) + (un0 - ucol0);
  ustar_out[N + n] = (ucol1 + 0.5 * dt * S[1]) + (un1 - ucol1);
  if (own_need) {
    Ug[n] = S[0];
    Ug[(size_t)N + n] = S[1];
    Ug[2 * (size_t)N + n] = Fn[0];
    Ug[3 * (size_t)N + n] = Fn[1];
    Ug[4 * (size_t)N + n] = Fn[2];
    Ug[5 * (size_t)N + n] = Fn[3];
    ug[n] = un0;
    ug[N + n] = un1;
  }
}

// Tile kTX x TY, one node per thread; MINB resident blocks per SM bounds the
// registers per thread (tuned per problem, see curved_lbm autotune).
template <int TY, int MINB, bool PRE, bool STAGE = false>
__global__ void __launch_bounds__(kTX * TY, MINB)
    k_fused2(Ctx2 c, Fused2 fz, const double* __restrict__ f0, double* __restrict__ f1,
             double* __restrict__ Ug, double* __restrict__ ug,
             const double* __restrict__ ustar, double* __restrict__ ustar_out,
             int* __restrict__ invalid, const double* clock, double t_host, int do_sweep,
             int do_repair, const double* __restrict__ mom) {
  extern __shared__ double smem2[];
  fused2_tile<TY, PRE, STAGE>(c, fz, fz.tiles[blockIdx.x], f0, f1, Ug, ug, ustar, ustar_out,
                              invalid, clock, t_host, do_sweep, do_repair, smem2, mom);
}

// Collide-time moments of the active nodes of the listed tiles, for the PRE
// form of the tile kernel: mom[0..5] = U with the damping half step
// (moments2), mom[6..7] = u* + dt/2 v.  One thread per node, coalesced rows.
template <int TY>
__global__ void __launch_bounds__(kTX * TY)
    k_mom2(Ctx2 c, Fused2 fz, const double* __restrict__ f0, const double* __restrict__ ustar,
           double* __restrict__ mom) {
  const cvlbm2d_problem& p = c.p;
  const int N = c.N;
  const int tile = fz.tiles[blockIdx.x];
  const int i = (tile / fz.tiles_j) * TY + (threadIdx.x >> 5);
  const int j = (tile % fz.tiles_j) * kTX + (threadIdx.x & 31);
  if (i >= p.nx || j >= p.ny) return;
  const int n = i * p.ny + j;
  if (p.active[n] == 0) return;
  double S[6];
  moments2(p, f0, N, n, S);
#pragma unroll
  for (int a = 0; a < 6; ++a) mom[(size_t)a * N + n] = S[a];
  mom[6 * (size_t)N + n] = ustar[n] + 0.5 * p.dt * S[0];
  mom[7 * (size_t)N + n] = ustar[N + n] + 0.5 * p.dt * S[1];
}

// ---------------------------------------------------------------------------
// Cut-link kernel: 8 links per 64-thread block, in two stages.
//   gather  8 lanes per link, 16 gathered quantities: q < 6 sums d/dx of
//           component q over the link's 24-node stencil, 6 <= q < 12 d/dy of
//           component q - 6, 12 <= q < 16 the F predictor component q - 12;
//           lane l takes q = l and l + 8 (one code path for every lane on
//           characteristic links); lanes 0/1 then the tangential image of u
//           (compatible predictors on a traction wall).
//   finish  one thread per link: predictor, normal-image solve,
//           characteristic state and flux tangents, the six population rows.
//           In one thread the independent chains (the two flux tangents, the
//           six rows, the BFL population loads) overlap instead of running
//           lane after lane, and a warp carries 8 links, not 2.
// Links are visited in `order` (traction links first) so neighbouring links
// take the same branches.
// ---------------------------------------------------------------------------
constexpr int kLG = 8;
constexpr int kLinksPerBlock2 = 8;
constexpr int kLinkThreads2 = kLG * kLinksPerBlock2;

struct LinkShared2 {
  double g[16];  // ux[6], uy[6], Fg[4]
  double dut[2], wt_abs;
};

// Per-link inputs: the link row when the host built rows, else the link tables.
struct LinkIn2 {
  const double* pp;
  double eta, xb, yb, nxb, nyb;
  int ell, i, j, qo, qi, kind, mode, n, nu;
  bool live, rowed, up_ok, lsq_ok;
};

__device__ __forceinline__ LinkIn2 link2_in(const Ctx2& c, int slot) {
  const cvlbm2d_problem& p = c.p;
  LinkIn2 L;
  L.live = slot < p.n_links;
  L.rowed = p.link_rows != nullptr;
  L.pp = p.bc_params;
  L.eta = 0.5;
  L.xb = L.yb = L.nyb = 0.0;
  L.nxb = 1.0;
  L.ell = L.i = L.j = L.qo = L.n = L.nu = L.mode = 0;
  L.qi = 2;
  L.kind = kDirichlet;
  L.up_ok = L.lsq_ok = false;
  if (!L.live) return L;
  int bid;
  if (L.rowed) {
    // every per-link input is one load away from the slot (no link_order /
    // link-table / stencil-id indirection)
    const cvlbm2d_link_row* row = p.link_rows + slot;
    L.ell = row->ell;
    L.i = row->i;
    L.j = row->j;
    L.qo = row->q;
    bid = row->bid;
    L.eta = row->eta;
    L.xb = row->xb;
    L.yb = row->yb;
    L.nxb = row->nx;
    L.nyb = row->ny;
    L.n = row->node;
    L.up_ok = row->upstream >= 0;
    L.nu = L.up_ok ? row->upstream : L.n;
    L.lsq_ok = row->lsq_valid != 0;
  } else {
    const int ell = p.link_order ? p.link_order[slot] : slot;
    L.ell = ell;
    L.i = p.link_i[ell];
    L.j = p.link_j[ell];
    L.qo = p.link_q[ell];
    bid = p.link_bid[ell];
    L.eta = p.link_eta[ell];
    L.xb = p.link_xb[ell];
    L.yb = p.link_yb[ell];
    L.nxb = p.link_nx[ell];
    L.nyb = p.link_ny[ell];
    L.n = L.i * p.ny + L.j;
    const int iu = L.i - cx2(L.qo), ju = L.j - cy2(L.qo);
    L.up_ok = iu >= 0 && iu < p.nx && ju >= 0 && ju < p.ny && p.active[iu * p.ny + ju] != 0;
    L.nu = L.up_ok ? iu * p.ny + ju : L.n;
    L.lsq_ok = p.lsq_valid[ell] != 0;
  }
  if (bid < 0 || bid >= kMaxIds2) bid = 0;
  L.kind = p.bc_kind[bid];
  L.mode = p.bc_mode[bid];
  L.pp = p.bc_params + bid * 8;
  L.qi = L.qo + 2;
  if (L.qi >= 4) L.qi -= 4;
  return L;
}

// sum_m w[m] * Uc[node[m]] over the 24 stencil slots in slot order (as
// _lsq_U_at_boundary, two_d/curved_boundary_warp.py:1213-1221), with all
// loads issued before the sequential sum.
__device__ __forceinline__ double lsq_sum(const int* __restrict__ node, const double* __restrict__ w,
                                          const double* __restrict__ Uc) {
  int nd[kMaxLsq2];
  double wv[kMaxLsq2], uv[kMaxLsq2];
#pragma unroll
  for (int m = 0; m < kMaxLsq2; ++m) {
    nd[m] = node[m];
    wv[m] = w[m];
  }
#pragma unroll
  for (int m = 0; m < kMaxLsq2; ++m) uv[m] = nd[m] >= 0 ? Uc[nd[m]] : 0.0;
  double out = 0.0;
#pragma unroll
  for (int m = 0; m < kMaxLsq2; ++m)
    if (nd[m] >= 0) out += wv[m] * uv[m];
  return out;
}

// Gather stage of one link (slot `slot`) on lane `lane` of its 8-lane group.
__device__ __forceinline__ void link2_gather(const Ctx2& c, LinkShared2& S, int lane, int slot,
                                             const double* __restrict__ U,
                                             const double* __restrict__ u) {
  const cvlbm2d_problem& p = c.p;
  const LinkIn2 L = link2_in(c, slot);
  if (!L.live) return;
  const int N = c.N, recon = p.recon;
  // stencil ids and weights of this link (slot order when rows are given)
  const size_t sl = (size_t)(L.rowed ? slot : L.ell) * kMaxLsq2;
  const int* lnode = (L.rowed ? p.lsq_node_slot : p.lsq_node) + sl;
  const bool lsq_recon = (recon == 11 || recon == 12) && L.lsq_ok;
  const bool use_char = lsq_recon && L.kind == kNeumann;
  const bool compat = (recon == 9 || recon == 11) && L.lsq_ok;
#pragma unroll
  for (int q = lane; q < 16; q += kLG) {
    if (q < 12 ? use_char : lsq_recon) {
      const double* w = q < 6 ? (L.rowed ? p.lsq_wx_slot : p.lsq_wx)
                      : q < 12 ? (L.rowed ? p.lsq_wy_slot : p.lsq_wy)
                               : (L.rowed ? p.lsq_wb_slot : p.lsq_wb);
      const int comp = q < 6 ? q : q < 12 ? q - 6 : q - 10;
      S.g[q] = lsq_sum(lnode, w + sl, U + (size_t)comp * N);
    } else if (q >= 12) {
      const double* Uk = U + (size_t)(q - 10) * N;
      double fg;
      if (recon == 0 || recon == 2 || recon == 13) {
        fg = L.up_ok ? Uk[L.n] + L.eta * (Uk[L.n] - Uk[L.nu]) : Uk[L.n];
        if (recon == 2 && L.lsq_ok)
          fg = lsq_sum(lnode, (L.rowed ? p.lsq_wb_slot : p.lsq_wb) + sl, Uk);
      } else {
        fg = interp_link(Uk, p.active, L.i, L.j, L.qo, L.eta, p.nx, p.ny);
      }
      S.g[q] = fg;
    }
  }
  if (compat && L.kind == kNeumann && lane < 2) {
    // tangential image of u along the wall, component `lane`
    const double* wt = (L.rowed ? p.lsq_wt_slot : p.lsq_wt) + sl;
    double d = 0.0, wa = 0.0;
    for (int mm = 0; mm < kMaxLsq2; ++mm) {
      const int nd = lnode[mm];
      if (nd >= 0) {
        d += wt[mm] * u[(size_t)lane * N + nd];
        wa += fabs(wt[mm]);
      }
    }
    S.dut[lane] = d;
    if (lane == 0) S.wt_abs = wa;
  }
}

// BFL inputs of population row a of a link: the outgoing post-collision value
// fo, the incoming fi and the upstream value upv.
__device__ __forceinline__ void link2_bfl_in(const LinkIn2& L, int a, int N,
                                             const double* __restrict__ fpost, int fused,
                                             const double* __restrict__ scratch,
                                             const int32_t* __restrict__ partner, double& fo,
                                             double& fi, double& upv) {
  if (fused) {
    fo = scratch[(size_t)L.ell * 6 + a];
    fi = L.up_ok ? fpost[(size_t)(L.qi * 6 + a) * N + L.nu]
                 : scratch[(size_t)partner[L.ell] * 6 + a];
    upv = L.up_ok ? fpost[(size_t)(L.qo * 6 + a) * N + L.n] : fo;
  } else {
    fo = fpost[(size_t)(L.qo * 6 + a) * N + L.n];
    fi = fpost[(size_t)(L.qi * 6 + a) * N + L.n];
    upv = L.up_ok ? fpost[(size_t)(L.qo * 6 + a) * N + L.nu] : fo;
  }
}

// Finish stage of one link, on one thread.
__device__ __forceinline__ void link2_finish(
    const Ctx2& c, const LinkShared2& S, int slot, const double* __restrict__ fpost,
    double* __restrict__ fout, const double* __restrict__ U, const double* clock, double t_host,
    double offset, int fused, const double* __restrict__ scratch,
    const int32_t* __restrict__ partner) {
  const cvlbm2d_problem& p = c.p;
  const Mat& m = c.m;
  const LinkIn2 L = link2_in(c, slot);
  if (!L.live) return;
  const int N = c.N, recon = p.recon, kind = L.kind, mode = L.mode, n = L.n, qi = L.qi;
  const double* pp = L.pp;
  const double nxb = L.nxb, nyb = L.nyb, eta = L.eta;
  const bool lsq_recon = (recon == 11 || recon == 12) && L.lsq_ok;
  const bool use_char = lsq_recon && kind == kNeumann;
  const bool compat = (recon == 9 || recon == 11) && L.lsq_ok;
  // loads that do not depend on the chain below go first
  const double Un0 = U[n], Un1 = U[(size_t)N + n];
  double fo[6], fi[6], upv[6];
  if (!use_char) {
#pragma unroll
    for (int a = 0; a < 6; ++a) link2_bfl_in(L, a, N, fpost, fused, scratch, partner, fo[a],
                                             fi[a], upv[a]);
  }
  const double tmid = time_of(clock, t_host, offset);
  double bv0 = value2(0, mode, pp, L.xb, L.yb, nxb, nyb, tmid);
  double bv1 = value2(1, mode, pp, L.xb, L.yb, nxb, nyb, tmid);
  if (kind == kNeumann && p.use_dynamic_traction != 0) {
    bv0 = p.traction_x[L.ell];
    bv1 = p.traction_y[L.ell];
  }
  const double dt = p.dt, cc = p.c, om = p.omega;
  const double dxin = (double)cx2(qi), dyin = (double)cy2(qi);

  // -- predictor finalisation and the normal-image solve ---------------------
  double Fg[4] = {S.g[12], S.g[13], S.g[14], S.g[15]};
  if (compat) {
    const double tanx = -nyb, tany = nxb;
    double dut0 = 0.0, dut1 = 0.0, wt_abs = 0.0;
    if (kind == kNeumann) {
      dut0 = S.dut[0];
      dut1 = S.dut[1];
      wt_abs = S.wt_abs;
    } else {
      if (mode == 6) {
        double at = tmid;
        if (pp[6] > 0.0 && at > pp[6]) at = pp[6];
        dut0 = at * (pp[0] * tanx + pp[1] * tany);
        dut1 = at * (pp[3] * tanx + pp[4] * tany);
      }
      wt_abs = 1.0;
    }
    if (wt_abs > 0.0) {
      const double hn0 = Fg[0] * nxb + Fg[1] * nyb, hn1 = Fg[2] * nxb + Fg[3] * nyb;
      const double gt0 = tanx + dut0, gt1 = tany + dut1;
      Fg[0] = hn0 * nxb + gt0 * tanx;
      Fg[1] = hn0 * nyb + gt0 * tany;
      Fg[2] = hn1 * nxb + gt1 * tanx;
      Fg[3] = hn1 * nyb + gt1 * tany;
    }
  }
  double Fb[4] = {Fg[0], Fg[1], Fg[2], Fg[3]};
  if (kind == kNeumann) solve_normal_image2(Fg, nxb, nyb, bv0, bv1, m, p.normal_solver, Fb);
  const P2 Pb = piola2(Fb[0], Fb[1], Fb[2], Fb[3], m);

  // -- characteristic state, flux tangents and equilibrium flux --------------
  double cv[6] = {Un0, Un1, Fb[0], Fb[1], Fb[2], Fb[3]};
  if (kind == kDirichlet) {
    cv[0] = bv0;
    cv[1] = bv1;
  }
  double cw[6], eqx[6], eqy[6];
  P2 Pc{0.0, 0.0, 0.0, 0.0};
  bool char_ok = false;
  if (use_char) {
    double ux[6], uy[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      ux[a] = S.g[a];
      uy[a] = S.g[6 + a];
    }
    const double sx = -eta * dt * cc * (double)cx2(L.qo);
    const double sy = -eta * dt * cc * (double)cy2(L.qo);
    double dv[6];
    for (int a = 0; a < 6; ++a) dv[a] = sx * ux[a] + sy * uy[a];
    double sc = 1.0;
    for (int g = 0; g < 10; ++g) {
      const double t11 = cv[2] + sc * dv[2], t12 = cv[3] + sc * dv[3];
      const double t21 = cv[4] + sc * dv[4], t22 = cv[5] + sc * dv[5];
      if (t11 * t22 - t12 * t21 > 10.0 * m.jf) break;
      sc = 0.5 * sc;
    }
    for (int a = 0; a < 6; ++a) cv[a] = cv[a] + sc * dv[a];
    double Ax[6], Ay[6], unused[6];
    flux2_jvp(cv, ux, m, Ax, unused);  // A_x U_x
    flux2_jvp(cv, uy, m, unused, Ay);  // A_y U_y
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      const double b = source_comp(a, p.source_mode, p.source, cv);
      cw[a] = b - Ax[a] - Ay[a] + cc * (dxin * ux[a] + dyin * uy[a]);
    }
    char_ok = cv[2] * cv[5] - cv[3] * cv[4] > m.jf;
    if (char_ok) {
      flux2_jvp(cv, cw, m, eqx, eqy);
      Pc = piola2(cv[2], cv[3], cv[4], cv[5], m);
    } else {
#pragma unroll
      for (int a = 0; a < 6; ++a) link2_bfl_in(L, a, N, fpost, fused, scratch, partner, fo[a],
                                               fi[a], upv[a]);
    }
  }

  // -- the six population rows ----------------------------------------------
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    double D = 1.0, Sv = 0.0;
    if (kind == kDirichlet) {
      switch (a) {
        case 0: D = -1.0; Sv = 0.5 * bv0; break;
        case 1: D = -1.0; Sv = 0.5 * bv1; break;
        case 2: Sv = -dxin * bv0 / cc; break;
        case 3: Sv = -dyin * bv0 / cc; break;
        case 4: Sv = -dxin * bv1 / cc; break;
        default: Sv = -dyin * bv1 / cc; break;
      }
    } else {
      switch (a) {
        case 0: Sv = -(dxin * Pb.a + dyin * Pb.b) / cc; break;
        case 1: Sv = -(dxin * Pb.c + dyin * Pb.d) / cc; break;
        default: D = -1.0; Sv = 0.5 * Fb[a - 2]; break;
      }
    }
    double val;
    if (char_ok) {
      const double jv = 0.25 * (cw[a] + (2.0 / cc) * (dxin * eqx[a] + dyin * eqy[a]));
      const double ge = feq2(qi, a, cv, Pc, 2.0 / cc);
      const double sa = source_comp(a, p.source_mode, p.source, cv);
      val = ge - dt / om * jv + dt * (1.0 / om - 0.5) * 0.25 * sa;
    } else if (eta >= 0.5) {
      const double al = 1.0 / (2.0 * eta);
      val = al * (D * fo[a] + Sv) + (1.0 - al) * fi[a];
    } else {
      val = D * (2.0 * eta * fo[a] + (1.0 - 2.0 * eta) * upv[a]) + Sv;
    }
    fout[(size_t)(qi * 6 + a) * N + n] = val;
  }
}

// Links [slot0, slot0 + 8) on the 64 threads of a block (every thread calls
// it; contains block barriers).
__device__ __forceinline__ void link2_block(
    const Ctx2& c, LinkShared2* sh, int slot0, const double* __restrict__ fpost,
    double* __restrict__ fout, const double* __restrict__ U, const double* __restrict__ u,
    const double* clock, double t_host, double offset, int fused,
    const double* __restrict__ scratch, const int32_t* __restrict__ partner) {
  const int lane = threadIdx.x & (kLG - 1);
  const int grp = threadIdx.x / kLG;
  link2_gather(c, sh[grp], lane, slot0 + grp, U, u);
  __syncthreads();
  if (threadIdx.x < kLinksPerBlock2)
    link2_finish(c, sh[threadIdx.x], slot0 + threadIdx.x, fpost, fout, U, clock, t_host, offset,
                 fused, scratch, partner);
  __syncthreads();
}

__global__ void __launch_bounds__(kLinkThreads2, 4)
    k_links2g(Ctx2 c, const double* __restrict__ fpost, double* __restrict__ fout,
              const double* __restrict__ U, const double* __restrict__ u, const double* clock,
              double t_host, double offset, int fused, const double* __restrict__ scratch,
              const int32_t* __restrict__ partner, double* clock_next) {
  __shared__ LinkShared2 sh[kLinksPerBlock2];
  if (clock_next && blockIdx.x == 0 && threadIdx.x == 0) *clock_next = clock[0] + c.p.dt;
  link2_block(c, sh, blockIdx.x * kLinksPerBlock2, fpost, fout, U, u, clock, t_host, offset,
              fused, scratch, partner);
}

}  // namespace
