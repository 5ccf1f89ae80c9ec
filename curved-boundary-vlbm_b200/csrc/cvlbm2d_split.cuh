// D2Q4x6 step, split form: three node kernels without halo recomputation.
// Included by cvlbm2d.cu (shares Ctx2, moments2 and the link kernel).
//
//   k2s_moments  moments with the damping half step, U of every active node,
//                the collide-time u (into u_next when a sweep is due, else
//                into u together with the u* update), invalid flag
//   k2s_sweep    one displacement sweep from U and the collide-time u of the
//                four neighbours plus cut-point anchors: swept u into u, u*
//   k2s_collide  f0 again, F repair from the swept u, BGK collision, repair
//                delta, push to f1; populations leaving through cut links go
//                to link_scratch; U at link-stencil nodes (every node on the
//                last step of a run) gets the repaired F
// followed by the cooperative link kernel in its fused mode.  Per active node
// this moves about 770 B (f0 twice, f1, U, u, u*) against the 416 B of the
// halo-tiled kernel, but every load is a plain coalesced row and no node's
// moments are recomputed: on lattices far larger than L2 it runs closer to
// the memory bandwidth.  The arithmetic is the per-phase kernels' (same
// operations in the same order), so results are bitwise equal.
#pragma once

namespace {

__global__ void __launch_bounds__(256)
    k2s_moments(Ctx2 c, const double* __restrict__ f0, double* __restrict__ U,
                double* __restrict__ ucol, double* __restrict__ ustar,
                int* __restrict__ invalid, int sweep_due) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) return;
  double S[6];
  moments2(p, f0, N, n, S);
#pragma unroll
  for (int a = 0; a < 6; ++a) U[(size_t)a * N + n] = S[a];
  const double u0 = ustar[n] + 0.5 * p.dt * S[0];
  const double u1 = ustar[N + n] + 0.5 * p.dt * S[1];
  ucol[n] = u0;
  ucol[N + n] = u1;
  if (!sweep_due) {
    ustar[n] = u0 + 0.5 * p.dt * S[0];
    ustar[N + n] = u1 + 0.5 * p.dt * S[1];
  }
  if (S[2] * S[5] - S[3] * S[4] <= c.m.jf) *invalid = 1;
}

__global__ void __launch_bounds__(256)
    k2s_sweep(Ctx2 c, const double* __restrict__ U, const double* __restrict__ ucol,
              double* __restrict__ u, double* __restrict__ ustar, const double* clock,
              double t_host) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  if (p.active[n] == 0) return;
  const int nx = p.nx, ny = p.ny;
  const int i = n / ny, j = n - i * ny;
  double diag = 0.0, rx = 0.0, ry = 0.0;
  const double time = time_of(clock, t_host, 0.5 * p.dt);
  for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k)
    anchor2(c, U, p.node_link_list[k], n, i, j, time, diag, rx, ry);
  const double* U2 = U + 2 * N;
  const double* U3 = U + 3 * N;
  const double* U4 = U + 4 * N;
  const double* U5 = U + 5 * N;
  const double hx = 0.5 * p.dx, hy = 0.5 * p.dy;
  if (i + 1 < nx && p.active[n + ny] != 0) {
    const int m = n + ny;
    rx += ucol[m] - hx * ((U2[n] - 1.0) + (U2[m] - 1.0));
    ry += ucol[N + m] - hx * (U4[n] + U4[m]);
    diag += 1.0;
  }
  if (i > 0 && p.active[n - ny] != 0) {
    const int m = n - ny;
    rx += ucol[m] + hx * ((U2[m] - 1.0) + (U2[n] - 1.0));
    ry += ucol[N + m] + hx * (U4[m] + U4[n]);
    diag += 1.0;
  }
  if (j + 1 < ny && p.active[n + 1] != 0) {
    const int m = n + 1;
    rx += ucol[m] - hy * (U3[n] + U3[m]);
    ry += ucol[N + m] - hy * ((U5[n] - 1.0) + (U5[m] - 1.0));
    diag += 1.0;
  }
  if (j > 0 && p.active[n - 1] != 0) {
    const int m = n - 1;
    rx += ucol[m] + hy * (U3[m] + U3[n]);
    ry += ucol[N + m] + hy * ((U5[m] - 1.0) + (U5[n] - 1.0));
    diag += 1.0;
  }
  const double u0 = ucol[n], u1 = ucol[N + n];
  double n0 = u0, n1 = u1;
  if (diag > 0.0) {
    n0 = u0 + p.relax * (rx / diag - u0);
    n1 = u1 + p.relax * (ry / diag - u1);
  }
  u[n] = n0;
  u[N + n] = n1;
  ustar[n] = (u0 + 0.5 * p.dt * U[n]) + (n0 - u0);
  ustar[N + n] = (u1 + 0.5 * p.dt * U[N + n]) + (n1 - u1);
}

__global__ void __launch_bounds__(128)
    k2s_collide(Ctx2 c, const double* __restrict__ f0, double* __restrict__ f1,
                double* __restrict__ U, const double* __restrict__ u,
                const uint8_t* __restrict__ need, double* __restrict__ scratch, int do_repair,
                int store_all) {
  const int N = c.N;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const cvlbm2d_problem& p = c.p;
  const int* act = p.active;
  if (act[n] == 0) return;
  const int nx = p.nx, ny = p.ny;
  const int i = n / ny, j = n - i * ny;
  const Mat& m = c.m;
  double S[6];
  moments2(p, f0, N, n, S);
  double Fn[4] = {S[2], S[3], S[4], S[5]};
  bool repaired = false;
  if (do_repair) {
    bool ok = true;
    if (p.interior_only != 0)
      ok = i > 0 && i + 1 < nx && j > 0 && j + 1 < ny && act[n - ny] && act[n + ny] &&
           act[n - 1] && act[n + 1];
    if (ok) {
      const double t11 = 1.0 + dudx2(u, act, n, i, nx, ny, p.dx);
      const double t12 = dudx2(u, act, n, j, ny, 1, p.dy);
      const double t21 = dudx2(u + N, act, n, i, nx, ny, p.dx);
      const double t22 = 1.0 + dudx2(u + N, act, n, j, ny, 1, p.dy);
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
  const P2 Po = piola2(S[2], S[3], S[4], S[5], m);
  double d11 = 0.0, d12 = 0.0, d21 = 0.0, d22 = 0.0;
  if (repaired) {
    const P2 Pn = piola2(Fn[0], Fn[1], Fn[2], Fn[3], m);
    d11 = Pn.a - Po.a;
    d12 = Pn.b - Po.b;
    d21 = Pn.c - Po.c;
    d22 = Pn.d - Po.d;
  }
  const double k2c = 2.0 / p.c, om = p.omega, sw = p.dt * (2.0 - om) * 0.125;
  const double ff = 0.5 / p.c, qt = 0.25;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int cq = cx2(q), cy = cy2(q);
    const double cxd = (double)cq, cyd = (double)cy;
    const int ii = i + cq, jj = j + cy;
    const int d = n + cq * ny + cy;
    const bool to_node = ii >= 0 && ii < nx && jj >= 0 && jj < ny && act[d] != 0;
    int ell_out = -1;
    if (!to_node) {
      for (int k = p.node_link_start[n]; k < p.node_link_start[n + 1]; ++k) {
        const int e = p.node_link_list[k];
        if (p.link_q[e] == q) ell_out = e;
      }
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      const double old = f0[(size_t)(q * 6 + a) * N + n];
      const double fe = feq2(q, a, S, Po, k2c);
      double v = old + om * (fe - old) + sw * source_comp(a, p.source_mode, p.source, S);
      if (repaired) {
        switch (a) {
          case 0: v = v - ff * (cxd * d11 + cyd * d12); break;
          case 1: v = v - ff * (cxd * d21 + cyd * d22); break;
          default: v = v + qt * (Fn[a - 2] - S[a]); break;
        }
      }
      if (to_node)
        f1[(size_t)(q * 6 + a) * N + d] = v;
      else if (ell_out >= 0)
        scratch[(size_t)ell_out * 6 + a] = v;
    }
  }
  if (repaired && (store_all || need[n])) {
    U[2 * (size_t)N + n] = Fn[0];
    U[3 * (size_t)N + n] = Fn[1];
    U[4 * (size_t)N + n] = Fn[2];
    U[5 * (size_t)N + n] = Fn[3];
  }
}

}  // namespace
