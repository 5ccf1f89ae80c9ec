// D3Q6 geometry preprocessing on the device: the local characteristic
// stencil of every traction cut link (the 3-D local_f closure's fixed
// geometry weights).  Reference: build_characteristic_weights,
// three_d/characteristic_stencil3d.py:18-171.
//
// One warp per cut link (k3_char_stencil):
//   1. the 343 nodes of the 7^3 cube around the link node, squared distance
//      to the cut point (lattice units), kept when active and r^2 <= 9.5;
//   2. the 48 nearest, ties broken in cube order: every lane ranks its
//      candidates against all 343 (the reference's stable argsort);
//   3. quadratic basis rows A (1, x, y, z, x^2/2, xy, xz, y^2/2, yz, z^2/2)
//      and Gaussian weights exp(-r^2 / 4.5) + 1e-4; the 55 entries of the
//      symmetric normal matrix M = A^T W A spread over the lanes, each summed
//      over the samples in order;
//   4. lane 0: 2-norm condition number of M from cyclic Jacobi eigenvalues
//      (must be <= 1e8 with >= 10 samples), LU with partial pivoting of
//      M + 1e-12 I; then every lane solves its samples' right-hand sides
//      A_m W_m, the gradient rows of the solution divided by dx being the
//      gradient weights; lane 0 checks them (row sums ~ 0, |w| sums <= 12/dx);
//   5. lane 0: the probe weights - trilinear interpolation at the cut point
//      minus h times the normal, an extrapolating pair of depths if both
//      probes' corners are active within 3 cells, else one depth, else up to
//      three nodes upstream along the link with Lagrange weights.
// Output in the reference's layout: indices [64][L] (48 gradient samples then
// 16 probe samples), weights [4][64][L] (row 0 probe weights, rows 1-3 the
// x, y, z gradient weights), probe modes [L] (2 pair, 1 single, -k upstream
// nodes) and a status per link (0 ok, 1 no full-rank fit, 2 inconsistent
// gradient weights); the host raises the reference's ValueError on a
// nonzero status.  Round-off: the reference solves with LAPACK, so the
// gradient weights agree to ~1e-14 of each link's largest weight; sample
// choice, probe weights and modes agree exactly.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "cvlbm_common.cuh"

namespace {

constexpr int kGrad = 48, kProbe = 16, kMax = 64, kCube = 343;
constexpr int kWarpsPerBlock = 4;

struct StencilWarp {
  double r2[kCube];
  int32_t id[kCube];
  int32_t sel[kGrad];
  double A[kGrad][10];
  double W[kGrad];
  double M[10][10];
  double E[10][10];
  double G[3][kGrad];
  int32_t piv[10];
  int32_t nsel, status;
};

__device__ int32_t grid_id3(const cvlbm3d_stencil_input& in, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= in.nx || j >= in.ny || k >= in.nz) return -2;
  return in.active_id[((size_t)i * in.ny + j) * in.nz + k];
}

// Eigenvalues of the symmetric 10x10 matrix a (overwritten), cyclic Jacobi.
__device__ void jacobi_eigen10(double (*a)[10], double* ev) {
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < 10; ++i)
      for (int j = 0; j < 10; ++j) {
        tot += a[i][j] * a[i][j];
        if (i != j) off += a[i][j] * a[i][j];
      }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < 9; ++p)
      for (int q = p + 1; q < 10; ++q) {
        if (a[p][q] == 0.0) continue;
        const double tau = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < 10; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 10; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
      }
  }
  for (int i = 0; i < 10; ++i) ev[i] = a[i][i];
}

// In-place LU with partial pivoting (first largest pivot); false if singular.
__device__ bool lu10(double (*a)[10], int32_t* piv) {
  for (int k = 0; k < 10; ++k) {
    int p = k;
    for (int i = k + 1; i < 10; ++i)
      if (fabs(a[i][k]) > fabs(a[p][k])) p = i;
    piv[k] = p;
    if (a[p][k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < 10; ++j) {
        const double t = a[k][j];
        a[k][j] = a[p][j];
        a[p][j] = t;
      }
    const double r = 1.0 / a[k][k];
    for (int i = k + 1; i < 10; ++i) {
      a[i][k] *= r;
      for (int j = k + 1; j < 10; ++j) a[i][j] -= a[i][k] * a[k][j];
    }
  }
  return true;
}

__device__ void lu10_solve(const double (*a)[10], const int32_t* piv, double* b) {
  for (int k = 0; k < 10; ++k) {
    const int p = piv[k];
    if (p != k) {
      const double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
  for (int i = 1; i < 10; ++i)
    for (int j = 0; j < i; ++j) b[i] -= a[i][j] * b[j];
  for (int i = 9; i >= 0; --i) {
    for (int j = i + 1; j < 10; ++j) b[i] -= a[i][j] * b[j];
    b[i] /= a[i][i];
  }
}

// Trilinear probe at `pt`: true when all 8 corners are active nodes within
// 3 cells of the link node (reference :94-109).
__device__ bool probe3(const cvlbm3d_stencil_input& in, const int* ctr, const double* pt,
                       int32_t* pp, double* ww) {
  int lo[3];
  double fr[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = (int)floor(pt[d]);
    fr[d] = pt[d] - (double)lo[d];
  }
  bool ok = true;
  for (int c = 0; c < 8; ++c) {
    const int cb[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    int nd[3];
    double w = 1.0;
    for (int d = 0; d < 3; ++d) {
      nd[d] = lo[d] + cb[d];
      const double f = cb[d] ? fr[d] : 1.0 - fr[d];
      w = d == 0 ? f : w * f;
      if (abs(nd[d] - ctr[d]) > 3) ok = false;
    }
    const int32_t id = grid_id3(in, nd[0], nd[1], nd[2]);
    if (id < 0) ok = false;
    pp[c] = id;
    ww[c] = w;
  }
  return ok;
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock)
    k3_char_stencil(cvlbm3d_stencil_input in, int32_t* __restrict__ indices,
                    double* __restrict__ weights, int32_t* __restrict__ modes,
                    int32_t* __restrict__ status) {
  __shared__ StencilWarp shw[kWarpsPerBlock];
  StencilWarp& S = shw[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int ell = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (ell >= in.n_links) return;
  const size_t L = (size_t)in.n_links;
  for (int m = lane; m < kMax; m += 32) {
    indices[m * L + ell] = -1;
    for (int r = 0; r < 4; ++r) weights[(r * kMax + m) * L + ell] = 0.0;
  }
  if (lane == 0) {
    modes[ell] = 0;
    status[ell] = 0;
  }
  if (in.link_mask && !in.link_mask[ell]) return;
  const int ctr[3] = {in.link_i[ell], in.link_j[ell], in.link_k[ell]};
  const double dx = in.dx;
  const double xr[3] = {in.link_xb[ell] / dx - 0.5, in.link_yb[ell] / dx - 0.5,
                        in.link_zb[ell] / dx - 0.5};

  // 1. candidates of the cube, (-3..3)^3 order
  int nfin = 0;
  for (int t = lane; t < kCube; t += 32) {
    const int o0 = t / 49 - 3, o1 = (t / 7) % 7 - 3, o2 = t % 7 - 3;
    const double x = (double)(ctr[0] + o0) - xr[0];
    const double y = (double)(ctr[1] + o1) - xr[1];
    const double z = (double)(ctr[2] + o2) - xr[2];
    const double r2 = x * x + y * y + z * z;
    const int32_t id = grid_id3(in, ctr[0] + o0, ctr[1] + o1, ctr[2] + o2);
    S.id[t] = id;
    const bool fin = id >= 0 && r2 <= 9.5;
    S.r2[t] = fin ? r2 : INFINITY;
    nfin += fin ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) nfin += __shfl_xor_sync(0xffffffffu, nfin, o);
  __syncwarp();
  // 2. the 48 nearest, ties in cube order
  for (int t = lane; t < kCube; t += 32) {
    const double r = S.r2[t];
    if (!(r < INFINITY)) continue;
    int rank = 0;
    for (int u = 0; u < kCube; ++u) {
      const double ru = S.r2[u];
      rank += (ru < r || (ru == r && u < t)) ? 1 : 0;
    }
    if (rank < kGrad) S.sel[rank] = t;
  }
  const int nsel = nfin < kGrad ? nfin : kGrad;
  __syncwarp();
  // 3. basis rows, weights, normal matrix
  for (int m = lane; m < nsel; m += 32) {
    const int t = S.sel[m];
    const double x = (double)(ctr[0] + t / 49 - 3) - xr[0];
    const double y = (double)(ctr[1] + (t / 7) % 7 - 3) - xr[1];
    const double z = (double)(ctr[2] + t % 7 - 3) - xr[2];
    const double row[10] = {1.0, x, y, z, 0.5 * x * x, x * y, x * z, 0.5 * y * y, y * z,
                            0.5 * z * z};
    for (int i = 0; i < 10; ++i) S.A[m][i] = row[i];
    S.W[m] = exp(-S.r2[t] / (2.0 * 1.5 * 1.5)) + 1e-4;
  }
  __syncwarp();
  for (int e = lane; e < 55; e += 32) {
    int i = 0, rem = e;
    while (rem >= 10 - i) {
      rem -= 10 - i;
      ++i;
    }
    const int j = i + rem;
    double s = 0.0;
    for (int m = 0; m < nsel; ++m) s += S.A[m][i] * S.W[m] * S.A[m][j];
    S.M[i][j] = s;
    S.M[j][i] = s;
  }
  __syncwarp();
  // 4. condition number and factorisation (lane 0)
  if (lane == 0) {
    for (int i = 0; i < 10; ++i)
      for (int j = 0; j < 10; ++j) S.E[i][j] = S.M[i][j];
    double ev[10];
    jacobi_eigen10(S.E, ev);
    double emax = 0.0, emin = INFINITY;
    for (int i = 0; i < 10; ++i) {
      const double a = fabs(ev[i]);
      emax = a > emax ? a : emax;
      emin = a < emin ? a : emin;
    }
    const double cond = emax / emin;
    int st = (nsel < 10 || !isfinite(cond) || cond > 1e8) ? 1 : 0;
    if (!st) {
      for (int i = 0; i < 10; ++i) S.M[i][i] += 1e-12;
      if (!lu10(S.M, S.piv)) st = 1;
    }
    S.status = st;
  }
  __syncwarp();
  if (S.status) {
    if (lane == 0) status[ell] = S.status;
    return;
  }
  for (int m = lane; m < nsel; m += 32) {
    double b[10];
    for (int i = 0; i < 10; ++i) b[i] = S.A[m][i] * S.W[m];
    lu10_solve(S.M, S.piv, b);
    for (int r = 0; r < 3; ++r) S.G[r][m] = b[1 + r] / dx;
  }
  __syncwarp();
  if (lane == 0) {
    bool good = true;
    for (int r = 0; r < 3; ++r) {
      double s = 0.0, sa = 0.0;
      for (int m = 0; m < nsel; ++m) {
        if (!isfinite(S.G[r][m])) good = false;
        s += S.G[r][m];
        sa += fabs(S.G[r][m]);
      }
      if (!(fabs(s) * dx < 1e-6) || !(sa * dx <= 12.0)) good = false;
    }
    S.status = good ? 0 : 2;
  }
  __syncwarp();
  if (S.status) {
    if (lane == 0) status[ell] = S.status;
    return;
  }
  for (int m = lane; m < nsel; m += 32) {
    indices[m * L + ell] = S.id[S.sel[m]];
    for (int r = 0; r < 3; ++r) weights[((1 + r) * kMax + m) * L + ell] = S.G[r][m];
  }
  // 5. probes (lane 0)
  if (lane != 0) return;
  const double nrm[3] = {in.link_nx[ell], in.link_ny[ell], in.link_nz[ell]};
  int32_t pp[kProbe];
  double pw[kProbe];
  for (int c = 0; c < kProbe; ++c) {
    pp[c] = -1;
    pw[c] = 0.0;
  }
  int mode = 0;
  const double pairs[4][2] = {{0.75, 1.75}, {1.0, 2.0}, {1.25, 2.5}, {1.5, 3.0}};
  for (int k = 0; k < 4 && !mode; ++k) {
    const double h1 = pairs[k][0], h2 = pairs[k][1];
    double p1[3], p2[3];
    for (int d = 0; d < 3; ++d) {
      p1[d] = xr[d] - h1 * nrm[d];
      p2[d] = xr[d] - h2 * nrm[d];
    }
    int32_t i1[8], i2[8];
    double w1[8], w2[8];
    const bool ok1 = probe3(in, ctr, p1, i1, w1);
    const bool ok2 = probe3(in, ctr, p2, i2, w2);
    if (ok1 && ok2) {
      for (int c = 0; c < 8; ++c) {
        pp[c] = i1[c];
        pp[8 + c] = i2[c];
        pw[c] = h2 / (h2 - h1) * w1[c];
        pw[8 + c] = -h1 / (h2 - h1) * w2[c];
      }
      mode = 2;
    }
  }
  const double singles[5] = {0.75, 1.0, 1.25, 1.5, 2.0};
  for (int k = 0; k < 5 && !mode; ++k) {
    double p1[3];
    for (int d = 0; d < 3; ++d) p1[d] = xr[d] - singles[k] * nrm[d];
    int32_t i1[8];
    double w1[8];
    if (probe3(in, ctr, p1, i1, w1)) {
      for (int c = 0; c < 8; ++c) {
        pp[c] = i1[c];
        pw[c] = w1[c];
      }
      mode = 1;
    }
  }
  if (!mode) {
    const int q = in.link_q[ell];
    const int dir[3] = {q == 0 ? 1 : (q == 3 ? -1 : 0), q == 1 ? 1 : (q == 4 ? -1 : 0),
                        q == 2 ? 1 : (q == 5 ? -1 : 0)};
    int cnt = 0;
    for (int k = 0; k < 3; ++k) {
      const int32_t id = grid_id3(in, ctr[0] - k * dir[0], ctr[1] - k * dir[1],
                                  ctr[2] - k * dir[2]);
      if (id < 0) break;
      pp[cnt++] = id;
    }
    const double e = in.link_eta[ell];
    if (cnt == 3) {
      pw[0] = 0.5 * (e + 1) * (e + 2);
      pw[1] = -e * (e + 2);
      pw[2] = 0.5 * e * (e + 1);
    } else if (cnt == 2) {
      pw[0] = 1 + e;
      pw[1] = -e;
    } else if (cnt == 1) {
      pw[0] = 1.0;
    }
    mode = -cnt;
  }
  for (int c = 0; c < kProbe; ++c) {
    indices[(kGrad + c) * L + ell] = pp[c];
    weights[(kGrad + c) * L + ell] = pw[c];
  }
  modes[ell] = mode;
}

}  // namespace

extern "C" int cvlbm3d_build_char_stencil(const cvlbm3d_stencil_input* in, int32_t* indices,
                                          double* weights, int32_t* modes, int32_t* status,
                                          void* stream) {
  if (!in || !indices || !weights || !modes || !status)
    return cv::fail(CVLBM_ERR_INVALID_ARG, "cvlbm3d_build_char_stencil: null argument");
  if (in->n_links < 0 || in->nx <= 0 || in->ny <= 0 || in->nz <= 0 || !(in->dx > 0.0))
    return cv::fail(CVLBM_ERR_INVALID_ARG, "cvlbm3d_build_char_stencil: bad sizes");
  if (in->n_links == 0) return CVLBM_OK;
  if (!in->active_id || !in->link_i || !in->link_j || !in->link_k || !in->link_q ||
      !in->link_eta || !in->link_xb || !in->link_yb || !in->link_zb || !in->link_nx ||
      !in->link_ny || !in->link_nz)
    return cv::fail(CVLBM_ERR_INVALID_ARG, "cvlbm3d_build_char_stencil: null table");
  const unsigned grid = (unsigned)((in->n_links + kWarpsPerBlock - 1) / kWarpsPerBlock);
  k3_char_stencil<<<grid, 32 * kWarpsPerBlock, 0, (cudaStream_t)stream>>>(*in, indices, weights,
                                                                          modes, status);
  cv::count_launches(1);
  return cv::check_launch("cvlbm3d_build_char_stencil");
}
