/*
 * CPU restatement of the D3Q6 local characteristic stencil builder --
 * TEST INFRASTRUCTURE (checker of the CUDA builder; never on the product path).
 *
 * Follows build_characteristic_weights (three_d/characteristic_stencil3d.py:18-171
 * of the reference) for one cut link at a time:
 *   gradient fit  (:56-92)   the <= 48 active nodes of the 7^3 cube around the
 *                            link node nearest to the cut point (r^2 <= 9.5,
 *                            ties in cube order), quadratic basis, Gaussian
 *                            weights exp(-r^2 / 4.5) + 1e-4, normal matrix M,
 *                            2-norm condition number <= 1e8, weights
 *                            C = (M + 1e-12 I)^-1 (A W)^T, gradient rows / dx,
 *                            consistency checks;
 *   probes        (:94-131)  trilinear probes at the cut point minus h times
 *                            the normal: an extrapolating pair, else a single
 *                            probe, else up to three nodes upstream along the
 *                            link with Lagrange weights (:132-155).
 * The reference solves with LAPACK (numpy.linalg.solve / cond); here the
 * condition number comes from cyclic Jacobi eigenvalues of the symmetric
 * matrix and the solve from an LU factorisation with partial pivoting, so the
 * weights agree to round-off (the tests state the tolerance), the sample
 * choice, probe weights and modes exactly.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define CS_GRAD 48
#define CS_PROBE 16
#define CS_MAX 64
#define CS_CUBE 343

/* Eigenvalues of the symmetric 10x10 matrix a (overwritten) by cyclic Jacobi. */
static void jacobi_eigen10(double a[10][10], double ev[10]) {
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
        double tau = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < 10; ++k) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 10; ++k) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
      }
  }
  for (int i = 0; i < 10; ++i) ev[i] = a[i][i];
}

/* In-place LU with partial pivoting (first largest pivot); 0 if singular. */
static int lu10(double a[10][10], int piv[10]) {
  for (int k = 0; k < 10; ++k) {
    int p = k;
    for (int i = k + 1; i < 10; ++i)
      if (fabs(a[i][k]) > fabs(a[p][k])) p = i;
    piv[k] = p;
    if (a[p][k] == 0.0) return 0;
    if (p != k)
      for (int j = 0; j < 10; ++j) {
        double t = a[k][j];
        a[k][j] = a[p][j];
        a[p][j] = t;
      }
    double r = 1.0 / a[k][k];
    for (int i = k + 1; i < 10; ++i) {
      a[i][k] *= r;
      for (int j = k + 1; j < 10; ++j) a[i][j] -= a[i][k] * a[k][j];
    }
  }
  return 1;
}

static void lu10_solve(double a[10][10], const int piv[10], double b[10]) {
  for (int k = 0; k < 10; ++k) {
    int p = piv[k];
    if (p != k) {
      double t = b[k];
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

typedef struct {
  int nx, ny, nz;
  const int32_t* active_id; /* [nx][ny][nz], -1 outside */
} Grid3;

static int32_t grid_id(const Grid3* g, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= g->nx || j >= g->ny || k >= g->nz) return -2;
  return g->active_id[((size_t)i * g->ny + j) * g->nz + k];
}

/* Trilinear probe at `pt` (lattice units); 1 when all 8 corners are active
 * nodes within 3 cells of the link node (reference :94-109). */
static int probe(const Grid3* g, const int ctr[3], const double pt[3], int32_t pp[8], double ww[8]) {
  int lo[3];
  double fr[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = (int)floor(pt[d]);
    fr[d] = pt[d] - (double)lo[d];
  }
  int ok = 1;
  for (int c = 0; c < 8; ++c) {
    int cb[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    int nd[3];
    double w = 1.0;
    for (int d = 0; d < 3; ++d) {
      nd[d] = lo[d] + cb[d];
      w = (d == 0) ? (cb[d] ? fr[d] : 1.0 - fr[d]) : w * (cb[d] ? fr[d] : 1.0 - fr[d]);
      if (abs(nd[d] - ctr[d]) > 3) ok = 0;
    }
    int32_t id = grid_id(g, nd[0], nd[1], nd[2]);
    if (id < 0) ok = 0;
    pp[c] = id;
    ww[c] = w;
  }
  return ok;
}

/* Status per link: 0 ok, 1 no full-rank fit, 2 inconsistent gradient weights. */
int oracle3d_char_stencil(int nx, int ny, int nz, const int32_t* active_id, int n_links,
                          const int32_t* li, const int32_t* lj, const int32_t* lk,
                          const int32_t* lq, const double* eta, const double* xb,
                          const double* yb, const double* zb, const double* nxv,
                          const double* nyv, const double* nzv, double dx,
                          const uint8_t* mask, int32_t* indices, double* weights,
                          int32_t* modes, int32_t* status) {
  const Grid3 g = {nx, ny, nz, active_id};
  const size_t L = (size_t)n_links;
  static const int dirs[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
  int first_bad = -1;
  for (int ell = 0; ell < n_links; ++ell) {
    for (int m = 0; m < CS_MAX; ++m) {
      indices[m * L + ell] = -1;
      for (int r = 0; r < 4; ++r) weights[(r * CS_MAX + m) * L + ell] = 0.0;
    }
    modes[ell] = 0;
    status[ell] = 0;
    if (mask && !mask[ell]) continue;
    const int ctr[3] = {li[ell], lj[ell], lk[ell]};
    const double xr[3] = {xb[ell] / dx - 0.5, yb[ell] / dx - 0.5, zb[ell] / dx - 0.5};
    const double nrm[3] = {nxv[ell], nyv[ell], nzv[ell]};
    /* candidates of the 7^3 cube in its (-3..3)^3 order */
    double r2c[CS_CUBE];
    int32_t idc[CS_CUBE];
    for (int t = 0; t < CS_CUBE; ++t) {
      int o[3] = {t / 49 - 3, (t / 7) % 7 - 3, t % 7 - 3};
      double x = (double)(ctr[0] + o[0]) - xr[0];
      double y = (double)(ctr[1] + o[1]) - xr[1];
      double z = (double)(ctr[2] + o[2]) - xr[2];
      double r2 = x * x + y * y + z * z;
      int32_t id = grid_id(&g, ctr[0] + o[0], ctr[1] + o[1], ctr[2] + o[2]);
      idc[t] = id;
      r2c[t] = (id >= 0 && r2 <= 9.5) ? r2 : INFINITY;
    }
    /* the 48 nearest, ties in cube order */
    int sel[CS_GRAD];
    int nsel = 0;
    for (int t = 0; t < CS_CUBE; ++t) {
      if (!isfinite(r2c[t])) continue;
      int rank = 0;
      for (int u = 0; u < CS_CUBE; ++u)
        if (r2c[u] < r2c[t] || (r2c[u] == r2c[t] && u < t)) ++rank;
      if (rank < CS_GRAD) {
        sel[rank] = t;
        ++nsel;
      }
    }
    if (nsel > CS_GRAD) nsel = CS_GRAD;
    double A[CS_GRAD][10], W[CS_GRAD];
    for (int m = 0; m < nsel; ++m) {
      int t = sel[m];
      double x = (double)(ctr[0] + t / 49 - 3) - xr[0];
      double y = (double)(ctr[1] + (t / 7) % 7 - 3) - xr[1];
      double z = (double)(ctr[2] + t % 7 - 3) - xr[2];
      double row[10] = {1.0, x, y, z, 0.5 * x * x, x * y, x * z, 0.5 * y * y, y * z, 0.5 * z * z};
      memcpy(A[m], row, sizeof(row));
      W[m] = exp(-r2c[t] / (2.0 * 1.5 * 1.5)) + 1e-4;
    }
    double M[10][10];
    for (int i = 0; i < 10; ++i)
      for (int j = i; j < 10; ++j) {
        double s = 0.0;
        for (int m = 0; m < nsel; ++m) s += A[m][i] * W[m] * A[m][j];
        M[i][j] = M[j][i] = s;
      }
    double E[10][10], ev[10];
    memcpy(E, M, sizeof(M));
    jacobi_eigen10(E, ev);
    double emax = 0.0, emin = INFINITY;
    for (int i = 0; i < 10; ++i) {
      double a = fabs(ev[i]);
      if (a > emax) emax = a;
      if (a < emin) emin = a;
    }
    double cond = emax / emin;
    if (nsel < 10 || !isfinite(cond) || cond > 1e8) {
      status[ell] = 1;
      if (first_bad < 0) first_bad = ell;
      continue;
    }
    for (int i = 0; i < 10; ++i) M[i][i] += 1e-12;
    int piv[10];
    if (!lu10(M, piv)) {
      status[ell] = 1;
      if (first_bad < 0) first_bad = ell;
      continue;
    }
    double G[3][CS_GRAD];
    for (int m = 0; m < nsel; ++m) {
      double b[10];
      for (int i = 0; i < 10; ++i) b[i] = A[m][i] * W[m];
      lu10_solve(M, piv, b);
      for (int r = 0; r < 3; ++r) G[r][m] = b[1 + r] / dx;
    }
    int good = 1;
    for (int r = 0; r < 3; ++r) {
      double s = 0.0, sa = 0.0;
      for (int m = 0; m < nsel; ++m) {
        if (!isfinite(G[r][m])) good = 0;
        s += G[r][m];
        sa += fabs(G[r][m]);
      }
      if (!(fabs(s) * dx < 1e-6) || !(sa * dx <= 12.0)) good = 0;
    }
    if (!good) {
      status[ell] = 2;
      if (first_bad < 0) first_bad = ell;
      continue;
    }
    for (int m = 0; m < nsel; ++m) {
      indices[m * L + ell] = idc[sel[m]];
      for (int r = 0; r < 3; ++r) weights[((1 + r) * CS_MAX + m) * L + ell] = G[r][m];
    }
    /* probes */
    int32_t pp[CS_PROBE];
    double pw[CS_PROBE];
    int mode = 0;
    static const double pairs[4][2] = {{0.75, 1.75}, {1.0, 2.0}, {1.25, 2.5}, {1.5, 3.0}};
    for (int k = 0; k < 4 && !mode; ++k) {
      double h1 = pairs[k][0], h2 = pairs[k][1];
      double p1[3], p2[3];
      for (int d = 0; d < 3; ++d) {
        p1[d] = xr[d] - h1 * nrm[d];
        p2[d] = xr[d] - h2 * nrm[d];
      }
      int32_t i1[8], i2[8];
      double w1[8], w2[8];
      int ok1 = probe(&g, ctr, p1, i1, w1);
      int ok2 = probe(&g, ctr, p2, i2, w2);
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
    static const double singles[5] = {0.75, 1.0, 1.25, 1.5, 2.0};
    for (int k = 0; k < 5 && !mode; ++k) {
      double p1[3];
      for (int d = 0; d < 3; ++d) p1[d] = xr[d] - singles[k] * nrm[d];
      int32_t i1[8];
      double w1[8];
      if (probe(&g, ctr, p1, i1, w1)) {
        for (int c = 0; c < 8; ++c) {
          pp[c] = i1[c];
          pw[c] = w1[c];
          pp[8 + c] = -1;
          pw[8 + c] = 0.0;
        }
        mode = 1;
      }
    }
    if (!mode) {
      const int* dir = dirs[lq[ell]];
      int cnt = 0;
      for (int c = 0; c < CS_PROBE; ++c) {
        pp[c] = -1;
        pw[c] = 0.0;
      }
      for (int k = 0; k < 3; ++k) {
        int32_t id = grid_id(&g, ctr[0] - k * dir[0], ctr[1] - k * dir[1], ctr[2] - k * dir[2]);
        if (id < 0) break;
        pp[cnt++] = id;
      }
      double e = eta[ell];
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
    for (int c = 0; c < CS_PROBE; ++c) {
      indices[(CS_GRAD + c) * L + ell] = pp[c];
      weights[(0 * CS_MAX + CS_GRAD + c) * L + ell] = pw[c];
    }
    modes[ell] = mode;
  }
  return first_bad;
}
