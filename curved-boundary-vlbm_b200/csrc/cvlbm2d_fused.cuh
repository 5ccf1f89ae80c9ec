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
    for (int a = 0; a < 6; ++a) S[a] += f0[(q * 6 + a) * N + n];
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
          const double v = f0[(q * 6 + a) * N + n];
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
  // the halo ring only (3 rows above and below the tile, 3 columns either
  // side of its rows), enumerated so that every lane of a warp takes a halo
  // node (a loop over the whole region would leave the lanes over interior
  // nodes idle in most warps)
  constexpr int kHalo = 2 * kH * kRX + 2 * kH * kTY;
  for (int h = threadIdx.x; h < kHalo; h += blockDim.x) {
    int ri, rj;
    if (h < 2 * kH * kRX) {
      const int hr = h / kRX;  // 0..5: rows 0..2 and TY+3..TY+5
      rj = h - hr * kRX;
      ri = hr < kH ? hr : kTY + hr;
    } else {
      const int h3 = h - 2 * kH * kRX;
      const int row = h3 / (2 * kH), col = h3 - row * (2 * kH);
      ri = kH + row;
      rj = col < kH ? col : kTX + col;
    }
    const int r = ri * kRX + rj;
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
        old = f0[(q * 6 + a) * N + n];
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
        f1[(q * 6 + a) * N + d] = v;
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
    Ug[N + n] = S[1];
    Ug[2 * N + n] = Fn[0];
    Ug[3 * N + n] = Fn[1];
    Ug[4 * N + n] = Fn[2];
    Ug[5 * N + n] = Fn[3];
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
// Cut-link kernel: 16 lanes per link, 8 links per 128-thread block.
// The kernel is a chain of dependent steps per link, so its length is set by
// the number of dependent global-load levels and by the serial math.  Loads
// are therefore issued as early as their addresses are known:
//   level 1  the link row, the stencil node ids and this lane's stencil
//            weights (all indexed by the processing slot alone); the
//            boundary tables are staged in shared memory per block
//   level 2  the stencil values U[node] of this lane's quantity, U at the
//            node, the dynamic traction and the BFL populations of the row
//            this lane writes
// then: lane q < 6 sums d/dx of component q, 6 <= q < 12 d/dy of component
// q - 6, 12 <= q < 16 the F predictor component q - 12 (one code path for
// every lane on characteristic links), lanes 0/1 the tangential image of u;
// lane 0 the predictor and the normal-image solve; lanes 0/1 the two flux
// tangents (the same code path, the lane picks the direction) while lane 2
// evaluates P at the characteristic state; lanes 0-5 one population row each.
// Links are visited in `order` (traction links first) so a warp's two links
// take the same branches.  MAT >= 0 compiles the kernel for that material
// law only (smaller code: fewer instruction-cache misses on the chain).
// ---------------------------------------------------------------------------
constexpr int kLG = 16;
constexpr int kLinksPerBlock2 = 8;
constexpr int kLinkThreads2 = kLG * kLinksPerBlock2;

struct LinkShared2 {
  double g[16];  // ux[6], uy[6], Fg[4]
  double dut[2], wt_abs;
  double Fb[4], cv[6], cw[6], Ax[6], Ay[6], eqx[6], eqy[6], Pb[4], Pc[4];
};

// boundary tables of one problem, staged per block
struct LinkBC2 {
  int32_t kind[kMaxIds2], mode[kMaxIds2];
  double params[kMaxIds2 * 8];
};

__device__ __forceinline__ void stage_bc2(const cvlbm2d_problem& p, LinkBC2& B) {
  for (int t = threadIdx.x; t < kMaxIds2 * 8; t += blockDim.x) {
    B.params[t] = p.bc_params[t];
    if (t < kMaxIds2) {
      B.kind[t] = p.bc_kind[t];
      B.mode[t] = p.bc_mode[t];
    }
  }
}

// Per-link inputs: the link row when the host built rows, else the link tables.
struct LinkIn2 {
  const double* pp;
  double eta, xb, yb, nxb, nyb;
  int ell, i, j, qo, qi, kind, mode, n, nu;
  bool live, rowed, up_ok, lsq_ok;
};

// The row part (no boundary tables needed: these loads can be issued before
// the block's boundary tables are staged), then link2_in_bc.
__device__ __forceinline__ LinkIn2 link2_in_row(const Ctx2& c, int slot, int& bid) {
  const cvlbm2d_problem& p = c.p;
  LinkIn2 L;
  L.live = slot < p.n_links;
  L.rowed = p.link_rows != nullptr;
  L.pp = nullptr;
  bid = 0;
  L.eta = 0.5;
  L.xb = L.yb = L.nyb = 0.0;
  L.nxb = 1.0;
  L.ell = L.i = L.j = L.qo = L.n = L.nu = L.mode = 0;
  L.qi = 2;
  L.kind = kDirichlet;
  L.up_ok = L.lsq_ok = false;
  if (!L.live) return L;
  if (L.rowed) {
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
  L.qi = L.qo + 2;
  if (L.qi >= 4) L.qi -= 4;
  return L;
}

// The boundary-table part of a link's inputs (after the tables are staged).
__device__ __forceinline__ void link2_in_bc(LinkIn2& L, const LinkBC2& B, int bid) {
  L.pp = B.params + bid * 8;
  if (!L.live) return;
  L.kind = B.kind[bid];
  L.mode = B.mode[bid];
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

// One cut link (processing slot `slot`) on the 16 lanes of a group; every
// lane of the group calls it (only __syncwarp inside).  RECON / SOLVER >= 0
// fix the reconstruction and the Neumann solver at compile time (they must
// equal the problem's), so that the kernel holds only that path's code.
// LG (16 or 8) lanes per link: with 8, lane l gathers quantities l and l + 8
// one after the other (twice the links in flight per SM for the same
// registers, a longer gather per link: the batched solve's throughput form).
template <int RECON = -1, int SOLVER = -1, int LG = kLG>
__device__ __forceinline__ void link2_group(
    const Ctx2& c, const Mat& m, LinkBC2& B, LinkShared2& S, int lane, int slot,
    const double* __restrict__ fpost, double* __restrict__ fout, const double* __restrict__ U,
    const double* __restrict__ u, const double* clock, double t_host, double offset, int fused,
    const double* __restrict__ scratch, const int32_t* __restrict__ partner) {
  const cvlbm2d_problem& p = c.p;
  const int N = c.N, recon = RECON >= 0 ? RECON : p.recon;
  const int solver = SOLVER >= 0 ? SOLVER : p.normal_solver;
  const bool live = slot < p.n_links;
  const bool rowed = p.link_rows != nullptr;
  // this lane's quantity: d/dx (q < 6), d/dy (6 <= q < 12) of component
  // comp, or the predictor of F component q - 12
  const int q = lane;
  const int comp = q < 6 ? q : q < 12 ? q - 6 : q - 10;
  const bool lsq_tables = recon == 2 || recon == 9 || recon == 11 || recon == 12;
  // -- level 1: slot-indexed stencil tables (slot order) and the link row ----
  int nd[kMaxLsq2];
  double wv[kMaxLsq2];
  const bool early = live && rowed && lsq_tables;
  if (early) {
    const size_t sl = (size_t)slot * kMaxLsq2;
    const double* w = q < 6 ? p.lsq_wx_slot : q < 12 ? p.lsq_wy_slot : p.lsq_wb_slot;
#pragma unroll
    for (int k = 0; k < kMaxLsq2; ++k) {
      nd[k] = p.lsq_node_slot[sl + k];
      wv[k] = w[sl + k];
    }
  }
  int bid;
  LinkIn2 L = link2_in_row(c, slot, bid);
  // the block's boundary tables, staged while the loads above are in flight
  // (every thread of the block reaches this barrier)
  stage_bc2(p, B);
  __syncthreads();
  link2_in_bc(L, B, bid);
  const size_t sl = (size_t)(L.rowed ? slot : L.ell) * kMaxLsq2;
  if (live && !early && lsq_tables) {
    const int* lnode = (L.rowed ? p.lsq_node_slot : p.lsq_node) + sl;
    const double* w = q < 6 ? (L.rowed ? p.lsq_wx_slot : p.lsq_wx)
                    : q < 12 ? (L.rowed ? p.lsq_wy_slot : p.lsq_wy)
                             : (L.rowed ? p.lsq_wb_slot : p.lsq_wb);
#pragma unroll
    for (int k = 0; k < kMaxLsq2; ++k) {
      nd[k] = lnode[k];
      wv[k] = w[sl + k];
    }
  }
  const bool lsq_recon = (recon == 11 || recon == 12) && L.lsq_ok;
  const bool use_char = lsq_recon && L.kind == kNeumann;
  const bool compat = (recon == 9 || recon == 11) && L.lsq_ok;
  const bool tang = compat && L.kind == kNeumann && lane < 2;
  // -- level 2: stencil values, node values, traction, BFL populations -------
  const bool mine = live && (q < 12 ? use_char : (lsq_recon || (recon == 2 && L.lsq_ok)));
  double uv[kMaxLsq2];
  if (mine) {
    const double* Uq = U + (size_t)comp * N;
#pragma unroll
    for (int k = 0; k < kMaxLsq2; ++k) uv[k] = nd[k] >= 0 ? Uq[nd[k]] : 0.0;
  }
  double Un0 = 0.0, Un1 = 0.0, trx = 0.0, try_ = 0.0;
  if (live && lane == 0) {
    Un0 = U[L.n];
    Un1 = U[(size_t)N + L.n];
    if (L.kind == kNeumann && p.use_dynamic_traction != 0) {
      trx = p.traction_x[L.ell];
      try_ = p.traction_y[L.ell];
    }
  }
  double fo = 0.0, fi = 0.0, upv = 0.0;
  if (live && lane < 6 && !use_char) link2_bfl_in(L, lane, N, fpost, fused, scratch, partner, fo, fi, upv);

  // -- gathered quantities ----------------------------------------------------
  if (live) {
    if (mine) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < kMaxLsq2; ++k)
        if (nd[k] >= 0) acc += wv[k] * uv[k];
      S.g[q] = acc;
    } else if (q >= 12) {
      const double* Uk = U + (size_t)comp * N;
      double fg;
      if (recon == 0 || recon == 2 || recon == 13) {
        fg = L.up_ok ? Uk[L.n] + L.eta * (Uk[L.n] - Uk[L.nu]) : Uk[L.n];
      } else {
        fg = interp_link(Uk, p.active, L.i, L.j, L.qo, L.eta, p.nx, p.ny);
      }
      S.g[q] = fg;
    }
    if (tang) {
      // tangential image of u along the wall, component `lane`
      const double* wt = (L.rowed ? p.lsq_wt_slot : p.lsq_wt) + sl;
      const double* uc = u + (size_t)lane * N;
      double d = 0.0, wa = 0.0;
#pragma unroll
      for (int k = 0; k < kMaxLsq2; ++k) {
        if (nd[k] >= 0) {
          d += wt[k] * uc[nd[k]];
          wa += fabs(wt[k]);
        }
      }
      S.dut[lane] = d;
      if (lane == 0) S.wt_abs = wa;
    }
    if constexpr (LG == 8) {
      // the second quantity of this lane: d/dy of components 2-5 or a
      // predictor component
      const int q2 = lane + 8;
      const int comp2 = q2 < 12 ? q2 - 6 : q2 - 10;
      const bool mine2 = q2 < 12 ? use_char : (lsq_recon || (recon == 2 && L.lsq_ok));
      if (mine2) {
        const double* w = (q2 < 12 ? (L.rowed ? p.lsq_wy_slot : p.lsq_wy)
                                   : (L.rowed ? p.lsq_wb_slot : p.lsq_wb)) + sl;
        const double* Uq = U + (size_t)comp2 * N;
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < kMaxLsq2; ++k)
          if (nd[k] >= 0) acc += w[k] * Uq[nd[k]];
        S.g[q2] = acc;
      } else if (q2 >= 12) {
        const double* Uk = U + (size_t)comp2 * N;
        double fg;
        if (recon == 0 || recon == 2 || recon == 13) {
          fg = L.up_ok ? Uk[L.n] + L.eta * (Uk[L.n] - Uk[L.nu]) : Uk[L.n];
        } else {
          fg = interp_link(Uk, p.active, L.i, L.j, L.qo, L.eta, p.nx, p.ny);
        }
        S.g[q2] = fg;
      }
    }
  }
  __syncwarp();

  const int qi = L.qi, kind = L.kind, mode = L.mode;
  const double* pp = L.pp;
  const double nxb = L.nxb, nyb = L.nyb, eta = L.eta;
  const double dt = p.dt, cc = p.c;
  const double dxin = (double)cx2(qi), dyin = (double)cy2(qi);
  const double tmid = time_of(clock, t_host, offset);
  // lane 0 of the group loaded the dynamic traction; every lane needs bv for
  // its row (all 32 lanes of the warp take part in the shuffles)
  const int lane0 = (threadIdx.x & 31) & ~(LG - 1);
  const double trx_g = __shfl_sync(0xffffffffu, trx, lane0);
  const double try_g = __shfl_sync(0xffffffffu, try_, lane0);
  double bv0 = 0.0, bv1 = 0.0;
  if (live) {
    bv0 = value2(0, mode, pp, L.xb, L.yb, nxb, nyb, tmid);
    bv1 = value2(1, mode, pp, L.xb, L.yb, nxb, nyb, tmid);
    if (kind == kNeumann && p.use_dynamic_traction != 0) {
      bv0 = trx_g;
      bv1 = try_g;
    }
  }

  // -- predictor finalisation, normal-image solve, characteristic state -------
  if (live && lane == 0) {
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
    if (kind == kNeumann) solve_normal_image2(Fg, nxb, nyb, bv0, bv1, m, solver, Fb);
    const P2 Pb = piola2(Fb[0], Fb[1], Fb[2], Fb[3], m);
    S.Pb[0] = Pb.a;
    S.Pb[1] = Pb.b;
    S.Pb[2] = Pb.c;
    S.Pb[3] = Pb.d;
    for (int k = 0; k < 4; ++k) S.Fb[k] = Fb[k];
    double cv[6] = {Un0, Un1, Fb[0], Fb[1], Fb[2], Fb[3]};
    if (kind == kDirichlet) {
      cv[0] = bv0;
      cv[1] = bv1;
    }
    if (use_char) {
      const double sx = -eta * dt * cc * (double)cx2(L.qo);
      const double sy = -eta * dt * cc * (double)cy2(L.qo);
      double dv[6];
      for (int a = 0; a < 6; ++a) dv[a] = sx * S.g[a] + sy * S.g[6 + a];
      double sc = 1.0;
      for (int g = 0; g < 10; ++g) {
        const double t11 = cv[2] + sc * dv[2], t12 = cv[3] + sc * dv[3];
        const double t21 = cv[4] + sc * dv[4], t22 = cv[5] + sc * dv[5];
        if (t11 * t22 - t12 * t21 > 10.0 * m.jf) break;
        sc = 0.5 * sc;
      }
      for (int a = 0; a < 6; ++a) cv[a] = cv[a] + sc * dv[a];
    }
    for (int a = 0; a < 6; ++a) S.cv[a] = cv[a];
  }
  __syncwarp();

  // -- flux tangents (lanes 0/1, one code path) and P at the state (lane 2) ---
  if (use_char && lane < 2) {
    double ax[6], ay[6];
    flux2_jvp(S.cv, S.g + 6 * lane, m, ax, ay);  // lane 0: A_x U_x, lane 1: A_y U_y
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      if (lane == 0)
        S.Ax[a] = ax[a];
      else
        S.Ay[a] = ay[a];
    }
  } else if (use_char && lane == 2) {
    const P2 Pc = piola2(S.cv[2], S.cv[3], S.cv[4], S.cv[5], m);
    S.Pc[0] = Pc.a;
    S.Pc[1] = Pc.b;
    S.Pc[2] = Pc.c;
    S.Pc[3] = Pc.d;
  }
  __syncwarp();
  if (use_char && lane < 6) {
    const int a = lane;
    const double b = source_comp(a, p.source_mode, p.source, S.cv);
    S.cw[a] = b - S.Ax[a] - S.Ay[a] + cc * (dxin * S.g[a] + dyin * S.g[6 + a]);
  }
  __syncwarp();
  const bool char_ok = use_char && S.cv[2] * S.cv[5] - S.cv[3] * S.cv[4] > m.jf;
  if (char_ok && lane == 0) flux2_jvp(S.cv, S.cw, m, S.eqx, S.eqy);
  __syncwarp();

  // -- one population row per lane -----------------------------------------
  if (live && lane < 6) {
    const int a = lane;
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
        case 0: Sv = -(dxin * S.Pb[0] + dyin * S.Pb[1]) / cc; break;
        case 1: Sv = -(dxin * S.Pb[2] + dyin * S.Pb[3]) / cc; break;
        default: D = -1.0; Sv = 0.5 * S.Fb[a - 2]; break;
      }
    }
    double val;
    if (char_ok) {
      const P2 Pc{S.Pc[0], S.Pc[1], S.Pc[2], S.Pc[3]};
      // 2/c, dt/omega and dt (1/omega - 1/2) / 4 are per-problem constants
      // formed once on the host with the same IEEE operations (Ctx2)
      const double jv = 0.25 * (S.cw[a] + c.k2c * (dxin * S.eqx[a] + dyin * S.eqy[a]));
      const double ge = feq2(qi, a, S.cv, Pc, c.k2c);
      const double sa = source_comp(a, p.source_mode, p.source, S.cv);
      val = ge - c.dt_om * jv + c.src_w * sa;
    } else {
      if (use_char) link2_bfl_in(L, a, N, fpost, fused, scratch, partner, fo, fi, upv);
      if (eta >= 0.5) {
        const double al = 1.0 / (2.0 * eta);
        val = al * (D * fo + Sv) + (1.0 - al) * fi;
      } else {
        val = D * (2.0 * eta * fo + (1.0 - 2.0 * eta) * upv) + Sv;
      }
    }
    fout[(size_t)(qi * 6 + a) * N + L.n] = val;
  }
}

// The material of the kernel: the problem's, or MAT when it is compiled for one.
template <int MAT>
__device__ __forceinline__ Mat link_mat2(const Ctx2& c) {
  Mat m = c.m;
  if (MAT >= 0) m.model = MAT;
  return m;
}

template <int MAT, int RECON = -1, int SOLVER = -1>
__global__ void __launch_bounds__(kLinkThreads2, 3)
    k_links2g(Ctx2 c, const double* __restrict__ fpost, double* __restrict__ fout,
              const double* __restrict__ U, const double* __restrict__ u, const double* clock,
              double t_host, double offset, int fused, const double* __restrict__ scratch,
              const int32_t* __restrict__ partner, double* clock_next) {
  __shared__ LinkShared2 sh[kLinksPerBlock2];
  __shared__ LinkBC2 bc;  // staged inside link2_group
  const int lane = threadIdx.x & (kLG - 1);
  const int grp = threadIdx.x / kLG;
  const int slot = blockIdx.x * kLinksPerBlock2 + grp;
  if (clock_next && blockIdx.x == 0 && threadIdx.x == 0) *clock_next = clock[0] + c.p.dt;
  const Mat m = link_mat2<MAT>(c);
  link2_group<RECON, SOLVER>(c, m, bc, sh[grp], lane, slot, fpost, fout, U, u, clock, t_host,
                             offset, fused, scratch, partner);
}

}  // namespace
