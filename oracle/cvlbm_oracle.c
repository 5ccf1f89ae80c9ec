/*
 * CPU oracle: plain-C restatement of the reference's curved-boundary VLBM
 * kernels -- TEST INFRASTRUCTURE, see cvlbm_oracle.h.
 *
 * Reference files (curved_lbm 1.0.0):
 *   V2 = src/curved_lbm/two_d/vector_nonlinear_elastic_warp.py
 *   C2 = src/curved_lbm/two_d/curved_boundary_warp.py
 *   V3 = src/curved_lbm/three_d/vector_nonlinear_elastic_warp3d.py
 *   C3 = src/curved_lbm/three_d/curved_boundary_warp3d.py
 * Build with -ffp-contract=off so every product and sum rounds separately,
 * as the reference's float64 arithmetic does.
 */
#include "cvlbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI_ = 3.141592653589793238462643383279502884;
enum { DIR_ = 1, NEU_ = 2 };

typedef struct {
  int model;
  double lam, mu, p0, p1, p2, jf;
} mat_t;

static mat_t mat_of(const cvlbm_material *m) {
  mat_t r = {m->model, m->lam, m->mu, m->p0, m->p1, m->p2, m->j_floor};
  return r;
}

static double clamp_j(double j, double fl) { return j < fl ? fl : j; }

/* ---------------------------------------------------------------------- */
/* Constitutive maps                                                       */
/* ---------------------------------------------------------------------- */

/* V2:938-1052 _piola_vec; out = (P11, P12, P21, P22) */
static void piola_vec(double F11, double F12, double F21, double F22, const mat_t *m, double *P) {
  double lam = m->lam, mu = m->mu;
  if (m->model == 0) {
    double C00 = F11 * F11 + F21 * F21, C01 = F11 * F12 + F21 * F22, C11 = F12 * F12 + F22 * F22;
    double E00 = 0.5 * (C00 - 1.0), E01 = 0.5 * C01, E11 = 0.5 * (C11 - 1.0);
    double trE = E00 + E11;
    double S00 = lam * trE + 2.0 * mu * E00, S01 = 2.0 * mu * E01, S11 = lam * trE + 2.0 * mu * E11;
    P[0] = F11 * S00 + F12 * S01;
    P[1] = F11 * S01 + F12 * S11;
    P[2] = F21 * S00 + F22 * S01;
    P[3] = F21 * S01 + F22 * S11;
    return;
  }
  double J = clamp_j(F11 * F22 - F12 * F21, m->jf);
  double H00 = F22 / J, H01 = -F21 / J, H10 = -F12 / J, H11 = F11 / J;
  double logJ = log(J);
  double vol = lam * logJ;
  if (m->model == 1) {
    vol = 0.5 * lam * (J * J - 1.0);
    P[0] = mu * (F11 - H00) + vol * H00;
    P[1] = mu * (F12 - H01) + vol * H01;
    P[2] = mu * (F21 - H10) + vol * H10;
    P[3] = mu * (F22 - H11) + vol * H11;
    return;
  }
  if (m->model == 2) {
    P[0] = mu * (F11 - H00) + vol * H00;
    P[1] = mu * (F12 - H01) + vol * H01;
    P[2] = mu * (F21 - H10) + vol * H10;
    P[3] = mu * (F22 - H11) + vol * H11;
    return;
  }
  double F2 = F11 * F11 + F12 * F12 + F21 * F21 + F22 * F22;
  double I1 = F2 + 1.0, I2 = J * J + F2;
  double jm23 = exp((-2.0 / 3.0) * logJ), jm43 = exp((-4.0 / 3.0) * logJ);
  double hs1 = (-2.0 / 3.0) * I1, hs2 = 2.0 * J * J - (4.0 / 3.0) * I2;
  double G1[4] = {jm23 * (2.0 * F11 + hs1 * H00), jm23 * (2.0 * F12 + hs1 * H01),
                  jm23 * (2.0 * F21 + hs1 * H10), jm23 * (2.0 * F22 + hs1 * H11)};
  double Hv[4] = {H00, H01, H10, H11};
  if (m->model == 3 || m->model == 6) {
    double G2[4] = {jm43 * (2.0 * F11 + hs2 * H00), jm43 * (2.0 * F12 + hs2 * H01),
                    jm43 * (2.0 * F21 + hs2 * H10), jm43 * (2.0 * F22 + hs2 * H11)};
    if (m->model == 6) {
      double A = jm23 * I1 - 3.0, c2 = -0.5 * mu, c3 = (m->p0 + 2.0 * mu) / 8.0;
      double sc = mu + 2.0 * c3 * A;
      for (int k = 0; k < 4; ++k) P[k] = sc * G1[k] + c2 * G2[k] + vol * Hv[k];
      return;
    }
    for (int k = 0; k < 4; ++k) P[k] = m->p0 * G1[k] + m->p1 * G2[k] + vol * Hv[k];
    return;
  }
  if (m->model == 4) {
    double A = jm23 * I1 - 3.0;
    double sc = m->p0 + 2.0 * m->p1 * A + 3.0 * m->p2 * A * A;
    for (int k = 0; k < 4; ++k) P[k] = sc * G1[k] + vol * Hv[k];
    return;
  }
  if (m->model == 5) {
    double A = jm23 * I1 - 3.0, den = 1.0 - A / m->p0;
    if (den < m->jf) den = m->jf;
    double sc = 0.5 * mu / den;
    for (int k = 0; k < 4; ++k) P[k] = sc * G1[k] + vol * Hv[k];
    return;
  }
  P[0] = mu * (F11 - H00) + vol * H00;
  P[1] = mu * (F12 - H01) + vol * H01;
  P[2] = mu * (F21 - H10) + vol * H10;
  P[3] = mu * (F22 - H11) + vol * H11;
}

/* V3:774-789 _det3 */
static double det3(const double *F) {
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

/* V3:792-1022 _piola_mat; F, P row-major 3x3 */
static void piola_mat(const double *F, const mat_t *m, double *P) {
  double lam = m->lam, mu = m->mu;
  double F11 = F[0], F12 = F[1], F13 = F[2], F21 = F[3], F22 = F[4], F23 = F[5], F31 = F[6],
         F32 = F[7], F33 = F[8];
  if (m->model == 0) {
    double C00 = F11 * F11 + F21 * F21 + F31 * F31, C01 = F11 * F12 + F21 * F22 + F31 * F32;
    double C02 = F11 * F13 + F21 * F23 + F31 * F33, C11 = F12 * F12 + F22 * F22 + F32 * F32;
    double C12 = F12 * F13 + F22 * F23 + F32 * F33, C22 = F13 * F13 + F23 * F23 + F33 * F33;
    double E00 = 0.5 * (C00 - 1.0), E01 = 0.5 * C01, E02 = 0.5 * C02, E11 = 0.5 * (C11 - 1.0),
           E12 = 0.5 * C12, E22 = 0.5 * (C22 - 1.0);
    double trE = E00 + E11 + E22;
    double S00 = lam * trE + 2.0 * mu * E00, S01 = 2.0 * mu * E01, S02 = 2.0 * mu * E02;
    double S11 = lam * trE + 2.0 * mu * E11, S12 = 2.0 * mu * E12, S22 = lam * trE + 2.0 * mu * E22;
    P[0] = F11 * S00 + F12 * S01 + F13 * S02;
    P[1] = F11 * S01 + F12 * S11 + F13 * S12;
    P[2] = F11 * S02 + F12 * S12 + F13 * S22;
    P[3] = F21 * S00 + F22 * S01 + F23 * S02;
    P[4] = F21 * S01 + F22 * S11 + F23 * S12;
    P[5] = F21 * S02 + F22 * S12 + F23 * S22;
    P[6] = F31 * S00 + F32 * S01 + F33 * S02;
    P[7] = F31 * S01 + F32 * S11 + F33 * S12;
    P[8] = F31 * S02 + F32 * S12 + F33 * S22;
    return;
  }
  double J = clamp_j(det3(F), m->jf);
  double H[9] = {(F22 * F33 - F23 * F32) / J, (F23 * F31 - F21 * F33) / J,
                 (F21 * F32 - F22 * F31) / J, (F13 * F32 - F12 * F33) / J,
                 (F11 * F33 - F13 * F31) / J, (F12 * F31 - F11 * F32) / J,
                 (F12 * F23 - F13 * F22) / J, (F13 * F21 - F11 * F23) / J,
                 (F11 * F22 - F12 * F21) / J};
  double logJ = log(J);
  if (m->model == 1) {
    double vol = 0.5 * lam * (J * J - 1.0);
    for (int k = 0; k < 9; ++k) P[k] = mu * (F[k] - H[k]) + vol * H[k];
    return;
  }
  if (m->model == 2) {
    double vol = lam * logJ;
    for (int k = 0; k < 9; ++k) P[k] = mu * (F[k] - H[k]) + vol * H[k];
    return;
  }
  double C00 = F11 * F11 + F21 * F21 + F31 * F31, C01 = F11 * F12 + F21 * F22 + F31 * F32;
  double C02 = F11 * F13 + F21 * F23 + F31 * F33, C11 = F12 * F12 + F22 * F22 + F32 * F32;
  double C12 = F12 * F13 + F22 * F23 + F32 * F33, C22 = F13 * F13 + F23 * F23 + F33 * F33;
  double I1 = C00 + C11 + C22;
  double jm23 = exp((-2.0 / 3.0) * logJ);
  double G1[9];
  for (int k = 0; k < 9; ++k) G1[k] = jm23 * (2.0 * F[k] - (2.0 / 3.0) * I1 * H[k]);
  if (m->model == 6) {
    double vol = 0.5 * lam * (J * J - 1.0), sc = 0.5 * mu;
    for (int k = 0; k < 9; ++k) P[k] = sc * G1[k] + vol * H[k];
    return;
  }
  double trC2 = C00 * C00 + C11 * C11 + C22 * C22 + 2.0 * (C01 * C01 + C02 * C02 + C12 * C12);
  double I2 = 0.5 * (I1 * I1 - trC2);
  double jm43 = exp((-4.0 / 3.0) * logJ);
  double vol = lam * logJ;
  if (m->model == 3) {
    double FC[9] = {F11 * C00 + F12 * C01 + F13 * C02, F11 * C01 + F12 * C11 + F13 * C12,
                    F11 * C02 + F12 * C12 + F13 * C22, F21 * C00 + F22 * C01 + F23 * C02,
                    F21 * C01 + F22 * C11 + F23 * C12, F21 * C02 + F22 * C12 + F23 * C22,
                    F31 * C00 + F32 * C01 + F33 * C02, F31 * C01 + F32 * C11 + F33 * C12,
                    F31 * C02 + F32 * C12 + F33 * C22};
    for (int k = 0; k < 9; ++k) {
      double G2 = jm43 * (2.0 * (I1 * F[k] - FC[k]) - (4.0 / 3.0) * I2 * H[k]);
      P[k] = m->p0 * G1[k] + m->p1 * G2 + vol * H[k];
    }
    return;
  }
  if (m->model == 4 || m->model == 5) {
    double A = jm23 * I1 - 3.0, sc;
    if (m->model == 4) {
      sc = m->p0 + 2.0 * m->p1 * A + 3.0 * m->p2 * A * A;
    } else {
      double den = 1.0 - A / m->p0;
      if (den < m->jf) den = m->jf;
      sc = 0.5 * mu / den;
    }
    for (int k = 0; k < 9; ++k) P[k] = sc * G1[k] + vol * H[k];
    return;
  }
  for (int k = 0; k < 9; ++k) P[k] = 0.0;
}

/* ---------------------------------------------------------------------- */
/* 2-D lattice primitives                                                  */
/* ---------------------------------------------------------------------- */
static const int CX[4] = {1, 0, -1, 0};
static const int CY[4] = {0, 1, 0, -1};

/* V2:1078-1137 _flux_x_comp/_flux_y_comp given P */
static double flux_x_comp(int a, const double *U, const double *P) {
  switch (a) {
    case 0: return -P[0];
    case 1: return -P[2];
    case 2: return -U[0];
    case 4: return -U[1];
    default: return 0.0;
  }
}
static double flux_y_comp(int a, const double *U, const double *P) {
  switch (a) {
    case 0: return -P[1];
    case 1: return -P[3];
    case 3: return -U[0];
    case 5: return -U[1];
    default: return 0.0;
  }
}

/* V2:1140-1168 _equilibrium_comp */
static double equilibrium_comp(int q, int a, const double *U, const double *P, double c) {
  double cx = (double)CX[q], cy = (double)CY[q];
  return 0.25 * (U[a] + (2.0 / c) * (cx * flux_x_comp(a, U, P) + cy * flux_y_comp(a, U, P)));
}

/* V2:1250-1280 _source_comp */
static double source_comp(int a, int mode, const double *sp, double vx, double vy) {
  if (mode == 1) return sp[a];
  if (mode == 2) {
    if (a == 0) return -sp[0] * vx;
    if (a == 1) return -sp[0] * vy;
  }
  return 0.0;
}

static double smoothstep5(double e) {
  double z = e < 0.0 ? 0.0 : (e > 1.0 ? 1.0 : e);
  return z * z * z * (10.0 - 15.0 * z + 6.0 * z * z);
}

/* V2:1180-1247 _boundary_value_comp */
static double boundary_value_comp(int comp, int mode, const double *p, double x, double y, double t) {
  if (mode == 0) return 0.0;
  if (mode == 1) return comp == 0 ? p[0] : p[1];
  if (mode == 2) {
    double sc = 1.0;
    if (p[2] > 0.0 && t < p[2]) {
      double s = sin(PI_ * t / p[2]);
      sc = s * s;
    }
    return comp == 0 ? p[0] * sc : p[1] * sc;
  }
  if (mode == 5) {
    double sc = 1.0;
    if (p[2] > 0.0 && t < p[2]) {
      double den = p[3];
      if (den <= 0.0) den = 2.0 * p[2];
      double s = sin(PI_ * t / den);
      sc = s * s;
    }
    return comp == 0 ? p[0] * sc : p[1] * sc;
  }
  if (mode == 3) {
    if (comp == 0 && t < p[1]) return p[0] * sin(PI_ * t / p[1]);
    return 0.0;
  }
  if (mode == 4) {
    if (comp != 1 || t > p[3]) return 0.0;
    double z = (t - p[2]) / p[1];
    double pref = 2.0 * p[0] / (sqrt(3.0 * p[1]) * sqrt(sqrt(PI_)));
    double v = pref * (1.0 - z * z) * exp(-0.5 * z * z);
    if (p[6] > 0.0) {
      double layer = p[6] * p[5];
      if (layer < 1.0e-30) layer = 1.0e-30;
      double w = smoothstep5(y / layer) * smoothstep5((p[4] - y) / layer);
      if (p[7] > 1.0e-14) w = w / p[7];
      v = v * w;
    }
    return v;
  }
  if (mode == 6) {
    if (p[6] > 0.0 && t > p[6]) return 0.0;
    return comp == 0 ? p[0] * x + p[1] * y + p[2] : p[3] * x + p[4] * y + p[5];
  }
  return 0.0;
}

/* C2:935-984 _curved_boundary_value_comp (+ mode 105, linear ramp then hold) */
static double curved_boundary_value_comp(int comp, int mode, const double *p, double x, double y,
                                         double nx, double ny, double t) {
  if (mode == 101) return comp == 0 ? p[0] * nx + p[1] * ny : p[2] * nx + p[3] * ny;
  if (mode == 102) return comp == 0 ? p[0] * nx : p[0] * ny;
  if (mode == 103) {
    double sc = 1.0;
    if (p[1] > 0.0 && t < p[1]) {
      double den = p[2];
      if (den <= 0.0) den = 2.0 * p[1];
      double s = sin(PI_ * t / den);
      sc = s * s;
    }
    return comp == 0 ? p[0] * sc * nx : p[0] * sc * ny;
  }
  if (mode == 104) {
    double sc = 0.0;
    if (p[1] > 0.0 && t < p[1]) {
      double s = sin(PI_ * t / p[1]);
      sc = s * s;
    }
    return comp == 0 ? p[0] * sc * nx : p[0] * sc * ny;
  }
  if (mode == 105) {
    double sc = 1.0;
    if (p[1] > 0.0 && t < p[1]) sc = t / p[1];
    return comp == 0 ? p[0] * sc * nx : p[0] * sc * ny;
  }
  return boundary_value_comp(comp, mode, p, x, y, t);
}

/* C2:987-1013 _normal_traction_residual_arbitrary */
static void normal_traction_residual(double hn0, double hn1, double gt0, double gt1, double nx,
                                     double ny, double tx, double ty, const mat_t *m, double *r) {
  double tx1 = -ny, tx2 = nx;
  double P[4];
  piola_vec(hn0 * nx + gt0 * tx1, hn0 * ny + gt0 * tx2, hn1 * nx + gt1 * tx1, hn1 * ny + gt1 * tx2,
            m, P);
  r[0] = P[0] * nx + P[1] * ny - tx;
  r[1] = P[2] * nx + P[3] * ny - ty;
}

/* C2:1046-1192 _solve_normal_image_arbitrary (with :1016-1043 acoustic Jacobian) */
static void solve_normal_image(const double *Fg, double nx, double ny, double tx, double ty,
                               const mat_t *m, int nj, double *out) {
  double lam = m->lam, mu = m->mu, jf = m->jf;
  if (nj == 2 && m->model == 1) {
    double a0 = Fg[3] * nx - Fg[2] * ny, a1 = -Fg[1] * nx + Fg[0] * ny;
    double a2 = a0 * a0 + a1 * a1;
    if (a2 > 1.0e-28) {
      double area = sqrt(a2), e0 = a0 / area, e1 = a1 / area;
      double tau = tx * e0 + ty * e1;
      double aa = mu + 0.5 * lam * a2, bb = mu + 0.5 * lam;
      double disc = sqrt(tau * tau + 4.0 * aa * bb);
      double s = (tau + disc) / (2.0 * aa);
      if (tau < 0.0) s = 2.0 * bb / (disc - tau);
      if (area * s > jf) {
        double h0 = (tx - tau * e0) / mu + s * e0, h1 = (ty - tau * e1) / mu + s * e1;
        double d0 = h0 - (Fg[0] * nx + Fg[1] * ny), d1 = h1 - (Fg[2] * nx + Fg[3] * ny);
        out[0] = Fg[0] + d0 * nx;
        out[1] = Fg[1] + d0 * ny;
        out[2] = Fg[2] + d1 * nx;
        out[3] = Fg[3] + d1 * ny;
        return;
      }
    }
  }
  double tanx = -ny, tany = nx;
  double hn0 = Fg[0] * nx + Fg[1] * ny, hn1 = Fg[2] * nx + Fg[3] * ny;
  double gt0 = Fg[0] * tanx + Fg[1] * tany, gt1 = Fg[2] * tanx + Fg[3] * tany;
  double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r[2];
    normal_traction_residual(hn0, hn1, gt0, gt1, nx, ny, tx, ty, m, r);
    if (sqrt(r[0] * r[0] + r[1] * r[1]) < 1.0e-11) break;
    double a, b, c, d;
    if (nj != 0 && m->model == 1) {
      double F11 = hn0 * nx + gt0 * tanx, F12 = hn0 * ny + gt0 * tany;
      double F21 = hn1 * nx + gt1 * tanx, F22 = hn1 * ny + gt1 * tany;
      double J = clamp_j(F11 * F22 - F12 * F21, jf);
      double H00 = F22 / J, H01 = -F21 / J, H10 = -F12 / J, H11 = F11 / J;
      double beta = 0.5 * lam * (J * J - 1.0) - mu;
      double coeff = lam * J * J - beta;
      double n2 = nx * nx + ny * ny;
      double v0 = H00 * nx + H01 * ny, v1 = H10 * nx + H11 * ny;
      a = mu * n2 + coeff * v0 * v0;
      b = coeff * v0 * v1;
      c = coeff * v1 * v0;
      d = mu * n2 + coeff * v1 * v1;
    } else {
      double rp0[2], rp1[2];
      normal_traction_residual(hn0 + eps, hn1, gt0, gt1, nx, ny, tx, ty, m, rp0);
      normal_traction_residual(hn0, hn1 + eps, gt0, gt1, nx, ny, tx, ty, m, rp1);
      a = (rp0[0] - r[0]) / eps;
      c = (rp0[1] - r[1]) / eps;
      b = (rp1[0] - r[0]) / eps;
      d = (rp1[1] - r[1]) / eps;
    }
    double det = a * d - b * c;
    if (fabs(det) < 1.0e-14) break;
    double d0 = (-r[0] * d + b * r[1]) / det, d1 = (c * r[0] - a * r[1]) / det;
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double c0 = hn0 + step * d0, c1 = hn1 + step * d1;
      double F11 = c0 * nx + gt0 * tanx, F12 = c0 * ny + gt0 * tany;
      double F21 = c1 * nx + gt1 * tanx, F22 = c1 * ny + gt1 * tany;
      if (F11 * F22 - F12 * F21 > jf) {
        hn0 = c0;
        hn1 = c1;
        break;
      }
      step = 0.5 * step;
    }
  }
  out[0] = hn0 * nx + gt0 * tanx;
  out[1] = hn0 * ny + gt0 * tany;
  out[2] = hn1 * nx + gt1 * tanx;
  out[3] = hn1 * ny + gt1 * tany;
}

/* C2:1224-1247 _jvp_eps6 */
static double jvp_eps6(const double *w) {
  double s = fabs(w[0]);
  for (int k = 1; k < 6; ++k)
    if (fabs(w[k]) > s) s = fabs(w[k]);
  double eps = 1.0e-6;
  if (s > 1.0) eps = eps / s;
  return eps;
}

/* C2:1250-1365 _flux_x_jvp_comp (axis 0) / _flux_y_jvp_comp (axis 1) */
static double flux_jvp_comp(int axis, int a, const double *U, const double *W, const mat_t *m) {
  double eps = jvp_eps6(W);
  double Up[6], Um[6], Pp[4], Pm[4];
  for (int k = 0; k < 6; ++k) {
    Up[k] = U[k] + eps * W[k];
    Um[k] = U[k] - eps * W[k];
  }
  piola_vec(Up[2], Up[3], Up[4], Up[5], m, Pp);
  piola_vec(Um[2], Um[3], Um[4], Um[5], m, Pm);
  double fp = axis == 0 ? flux_x_comp(a, Up, Pp) : flux_y_comp(a, Up, Pp);
  double fm = axis == 0 ? flux_x_comp(a, Um, Pm) : flux_y_comp(a, Um, Pm);
  return (fp - fm) / (2.0 * eps);
}

/* C2:1368-1440 _equilibrium_jvp_comp */
static double equilibrium_jvp_comp(int q, int a, const double *U, const double *W, const mat_t *m,
                                   double c) {
  double AxW = flux_jvp_comp(0, a, U, W, m), AyW = flux_jvp_comp(1, a, U, W, m);
  return 0.25 * (W[a] + (2.0 / c) * ((double)CX[q] * AxW + (double)CY[q] * AyW));
}

#define IDX2(k, i, j) ((size_t)(k) * N + (size_t)(i) * ny + (size_t)(j))

/* C2:1443-1480 _interp_U_link */
static double interp_U_link(const double *U, const int *act, int comp, int i, int j, int qo,
                            double s, int nx, int ny) {
  size_t N = (size_t)nx * ny;
  double v0 = U[IDX2(comp, i, j)];
  int i1 = i - CX[qo], j1 = j - CY[qo];
  if (i1 >= 0 && i1 < nx && j1 >= 0 && j1 < ny && act[i1 * ny + j1] != 0) {
    double v1 = U[IDX2(comp, i1, j1)];
    int i2 = i - 2 * CX[qo], j2 = j - 2 * CY[qo];
    if (i2 >= 0 && i2 < nx && j2 >= 0 && j2 < ny && act[i2 * ny + j2] != 0) {
      double v2 = U[IDX2(comp, i2, j2)];
      double l0 = 0.5 * (s + 1.0) * (s + 2.0), l1 = -s * (s + 2.0), l2 = 0.5 * s * (s + 1.0);
      return l0 * v0 + l1 * v1 + l2 * v2;
    }
    return (s + 1.0) * v0 - s * v1;
  }
  return v0;
}

/* C2:1202-1221 _lsq_U_at_boundary */
static double lsq_U_at_boundary(const cvlbm2d_problem *p, const double *U, const double *w, int ell,
                                int comp, double fallback) {
  if (p->lsq_valid[ell] == 0) return fallback;
  size_t N = (size_t)p->nx * p->ny;
  int ny = p->ny;
  double out = 0.0;
  for (int m = 0; m < 24; ++m) {
    int ii = p->lsq_i[ell * 24 + m], jj = p->lsq_j[ell * 24 + m];
    if (ii >= 0 && jj >= 0) out += w[ell * 24 + m] * U[IDX2(comp, ii, jj)];
  }
  return out;
}

/* ---------------------------------------------------------------------- */
/* 2-D kernels                                                             */
/* ---------------------------------------------------------------------- */

/* C2:1691-1843 _collide_masked_kernel (P and sigma stored as the reference does) */
static void collide_masked(const cvlbm2d_problem *p, const mat_t *m, cvlbm2d_fields *f, size_t n,
                           int *invalid) {
  size_t N = (size_t)p->nx * p->ny;
  if (p->active[n] == 0) {
    for (int k = 0; k < 24; ++k) f->fpost[k * N + n] = 0.0;
    for (int a = 0; a < 6; ++a) f->U[a * N + n] = 0.0;
    f->u[n] = 0.0;
    f->u[N + n] = 0.0;
    return;
  }
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 4; ++q)
    for (int a = 0; a < 6; ++a) S[a] += f->f0[(q * 6 + a) * N + n];
  double hdt = 0.5 * p->dt;
  if (p->source_mode == 1) {
    for (int a = 0; a < 6; ++a) S[a] += hdt * p->source[a];
  } else if (p->source_mode == 2) {
    double den = 1.0 + hdt * p->source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
  double b[6];
  for (int a = 0; a < 6; ++a) b[a] = source_comp(a, p->source_mode, p->source, S[0], S[1]);
  for (int a = 0; a < 6; ++a) f->U[a * N + n] = S[a];
  double ux = f->u_star[n] + 0.5 * p->dt * S[0], uy = f->u_star[N + n] + 0.5 * p->dt * S[1];
  f->u[n] = ux;
  f->u[N + n] = uy;
  f->u_star[n] = ux + 0.5 * p->dt * S[0];
  f->u_star[N + n] = uy + 0.5 * p->dt * S[1];
  double J = S[2] * S[5] - S[3] * S[4];
  if (J <= m->jf) *invalid = 1;
  double Js = clamp_j(J, m->jf), P[4];
  piola_vec(S[2], S[3], S[4], S[5], m, P);
  if (f->P) {
    for (int k = 0; k < 4; ++k) f->P[k * N + n] = P[k];
    f->sigma[n] = (P[0] * S[2] + P[1] * S[3]) / Js;
    f->sigma[N + n] = (P[0] * S[4] + P[1] * S[5]) / Js;
    f->sigma[2 * N + n] = (P[2] * S[2] + P[3] * S[3]) / Js;
    f->sigma[3 * N + n] = (P[2] * S[4] + P[3] * S[5]) / Js;
  }
  for (int q = 0; q < 4; ++q)
    for (int a = 0; a < 6; ++a) {
      double feq = equilibrium_comp(q, a, S, P, p->c);
      double old = f->f0[(q * 6 + a) * N + n];
      f->fpost[(q * 6 + a) * N + n] =
          old + p->omega * (feq - old) + p->dt * (2.0 - p->omega) * 0.125 * b[a];
    }
}

/* C2:1846-2040 _collide_masked_mrt_ghost_kernel: moment-space collision,
 * flux moments relaxed with omega, the D2Q4 ghost moment with ghost_omega */
static void collide_masked_mrt(const cvlbm2d_problem *p, const mat_t *m, cvlbm2d_fields *f,
                               size_t n, int *invalid) {
  size_t N = (size_t)p->nx * p->ny;
  if (p->active[n] == 0) {
    for (int k = 0; k < 24; ++k) f->fpost[k * N + n] = 0.0;
    for (int a = 0; a < 6; ++a) f->U[a * N + n] = 0.0;
    f->u[n] = 0.0;
    f->u[N + n] = 0.0;
    return;
  }
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 4; ++q)
    for (int a = 0; a < 6; ++a) S[a] += f->f0[(q * 6 + a) * N + n];
  double hdt = 0.5 * p->dt;
  if (p->source_mode == 1) {
    for (int a = 0; a < 6; ++a) S[a] += hdt * p->source[a];
  } else if (p->source_mode == 2) {
    double den = 1.0 + hdt * p->source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
  double b[6];
  for (int a = 0; a < 6; ++a) b[a] = source_comp(a, p->source_mode, p->source, S[0], S[1]);
  for (int a = 0; a < 6; ++a) f->U[a * N + n] = S[a];
  double ux = f->u_star[n] + 0.5 * p->dt * S[0], uy = f->u_star[N + n] + 0.5 * p->dt * S[1];
  f->u[n] = ux;
  f->u[N + n] = uy;
  f->u_star[n] = ux + 0.5 * p->dt * S[0];
  f->u_star[N + n] = uy + 0.5 * p->dt * S[1];
  double J = S[2] * S[5] - S[3] * S[4];
  if (J <= m->jf) *invalid = 1;
  double Js = clamp_j(J, m->jf), P[4];
  piola_vec(S[2], S[3], S[4], S[5], m, P);
  if (f->P) {
    for (int k = 0; k < 4; ++k) f->P[k * N + n] = P[k];
    f->sigma[n] = (P[0] * S[2] + P[1] * S[3]) / Js;
    f->sigma[N + n] = (P[0] * S[4] + P[1] * S[5]) / Js;
    f->sigma[2 * N + n] = (P[2] * S[2] + P[3] * S[3]) / Js;
    f->sigma[3 * N + n] = (P[2] * S[4] + P[3] * S[5]) / Js;
  }
  const double phx[6] = {-P[0], -P[2], -S[0], 0.0, -S[1], 0.0};
  const double phy[6] = {-P[1], -P[3], 0.0, -S[0], 0.0, -S[1]};
  const double om = p->omega, og = p->ghost_omega;
  for (int a = 0; a < 6; ++a) {
    double fE = f->f0[(0 * 6 + a) * N + n], fN = f->f0[(1 * 6 + a) * N + n];
    double fW = f->f0[(2 * 6 + a) * N + n], fS = f->f0[(3 * 6 + a) * N + n];
    double m0 = fE + fN + fW + fS;
    double m1 = fE - fW;
    double m2 = fN - fS;
    double m3 = fE - fN + fW - fS;
    double m0p = m0 + om * (S[a] - m0) + p->dt * (2.0 - om) * 0.5 * b[a];
    double m1p = m1 + om * (phx[a] / p->c - m1);
    double m2p = m2 + om * (phy[a] / p->c - m2);
    double m3p = (1.0 - og) * m3;
    f->fpost[(0 * 6 + a) * N + n] = 0.25 * (m0p + m3p + 2.0 * m1p);
    f->fpost[(1 * 6 + a) * N + n] = 0.25 * (m0p - m3p + 2.0 * m2p);
    f->fpost[(2 * 6 + a) * N + n] = 0.25 * (m0p + m3p - 2.0 * m1p);
    f->fpost[(3 * 6 + a) * N + n] = 0.25 * (m0p - m3p - 2.0 * m2p);
  }
}

/* C2:3101-3124 _kinetic_ghost_filter_kernel: damp the ghost moment in place */
static void kinetic_filter(const cvlbm2d_problem *p, double *fld, size_t n) {
  size_t N = (size_t)p->nx * p->ny;
  double str = p->kinetic_filter;
  if (p->active[n] == 0 || str <= 0.0) return;
  for (int a = 0; a < 6; ++a) {
    size_t iE = (0 * 6 + a) * N + n, iN = (1 * 6 + a) * N + n;
    size_t iW = (2 * 6 + a) * N + n, iS = (3 * 6 + a) * N + n;
    double m3 = fld[iE] - fld[iN] + fld[iW] - fld[iS];
    double delta = -str * m3;
    double quarter = 0.25 * delta;
    fld[iE] = fld[iE] + quarter;
    fld[iW] = fld[iW] + quarter;
    fld[iN] = fld[iN] - quarter;
    fld[iS] = fld[iS] - quarter;
  }
}

int oracle2d_kinetic_filter(const cvlbm2d_problem *p, cvlbm2d_fields *f) {
  long N = (long)p->nx * p->ny;
  for (long n = 0; n < N; ++n) kinetic_filter(p, f->f0, (size_t)n);
  return 0;
}

/* C2:3287-3417 _local_displacement_bc_kernel, serial in link order */
static void displacement_bc(const cvlbm2d_problem *p, const cvlbm2d_fields *f, oracle2d_scratch *s,
                            double time) {
  size_t N = (size_t)p->nx * p->ny;
  int ny = p->ny;
  for (int ell = 0; ell < p->n_links; ++ell) {
    int bid = p->link_bid[ell];
    if (p->disp_bid >= 0) {
      if (bid != p->disp_bid) continue;
    } else if (p->bc_kind[bid] != DIR_) {
      continue;
    }
    int i = p->link_i[ell], j = p->link_j[ell];
    if (p->active[i * ny + j] == 0) continue;
    const double *pp = p->bc_params + bid * 8;
    int mode = p->bc_mode[bid];
    double xb = p->link_xb[ell], yb = p->link_yb[ell], nxb = p->link_nx[ell], nyb = p->link_ny[ell];
    double ub0 = 0.0, ub1 = 0.0;
    if (mode == 1) {
      ub0 = time * curved_boundary_value_comp(0, mode, pp, xb, yb, nxb, nyb, 0.0);
      ub1 = time * curved_boundary_value_comp(1, mode, pp, xb, yb, nxb, nyb, 0.0);
    } else if (mode == 6) {
      double at = time;
      if (pp[6] > 0.0 && at > pp[6]) at = pp[6];
      ub0 = at * curved_boundary_value_comp(0, mode, pp, xb, yb, nxb, nyb, 0.0);
      ub1 = at * curved_boundary_value_comp(1, mode, pp, xb, yb, nxb, nyb, 0.0);
    }
    double dbx = xb - ((double)i + 0.5) * p->dx, dby = yb - ((double)j + 0.5) * p->dy;
    size_t n = (size_t)i * ny + j;
    double tx = ub0 - ((f->U[2 * N + n] - 1.0) * dbx + f->U[3 * N + n] * dby);
    double ty = ub1 - (f->U[4 * N + n] * dbx + (f->U[5 * N + n] - 1.0) * dby);
    double w2 = p->weight * p->weight;
    s->bc_diag[n] = s->bc_diag[n] + w2;
    s->bc_rhs[n] = s->bc_rhs[n] + w2 * tx;
    s->bc_rhs[N + n] = s->bc_rhs[N + n] + w2 * ty;
  }
}

/* C2:3420-3490 _local_displacement_relax_kernel */
static void displacement_relax(const cvlbm2d_problem *p, const cvlbm2d_fields *f,
                               const oracle2d_scratch *s, size_t n) {
  size_t N = (size_t)p->nx * p->ny;
  int nx = p->nx, ny = p->ny, i = (int)(n / ny), j = (int)(n % ny);
  double *un = f->u_next;
  const double *U = f->U, *u = f->u;
  const int *act = p->active;
  if (act[n] == 0) {
    un[n] = 0.0;
    un[N + n] = 0.0;
    return;
  }
  double diag = s->bc_diag[n], rx = s->bc_rhs[n], ry = s->bc_rhs[N + n];
  double dx = p->dx, dy = p->dy;
  if (i + 1 < nx && act[n + ny] != 0) {
    size_t mm = n + ny;
    double gx = 0.5 * dx * ((U[2 * N + n] - 1.0) + (U[2 * N + mm] - 1.0));
    double gy = 0.5 * dx * (U[4 * N + n] + U[4 * N + mm]);
    rx += u[mm] - gx;
    ry += u[N + mm] - gy;
    diag += 1.0;
  }
  if (i > 0 && act[n - ny] != 0) {
    size_t mm = n - ny;
    double gx = 0.5 * dx * ((U[2 * N + mm] - 1.0) + (U[2 * N + n] - 1.0));
    double gy = 0.5 * dx * (U[4 * N + mm] + U[4 * N + n]);
    rx += u[mm] + gx;
    ry += u[N + mm] + gy;
    diag += 1.0;
  }
  if (j + 1 < ny && act[n + 1] != 0) {
    size_t mm = n + 1;
    double gx = 0.5 * dy * (U[3 * N + n] + U[3 * N + mm]);
    double gy = 0.5 * dy * ((U[5 * N + n] - 1.0) + (U[5 * N + mm] - 1.0));
    rx += u[mm] - gx;
    ry += u[N + mm] - gy;
    diag += 1.0;
  }
  if (j > 0 && act[n - 1] != 0) {
    size_t mm = n - 1;
    double gx = 0.5 * dy * (U[3 * N + mm] + U[3 * N + n]);
    double gy = 0.5 * dy * ((U[5 * N + mm] - 1.0) + (U[5 * N + n] - 1.0));
    rx += u[mm] + gx;
    ry += u[N + mm] + gy;
    diag += 1.0;
  }
  if (diag > 0.0) {
    un[n] = u[n] + p->relax * (rx / diag - u[n]);
    un[N + n] = u[N + n] + p->relax * (ry / diag - u[N + n]);
  } else {
    un[n] = u[n];
    un[N + n] = u[N + n];
  }
}

/* C2:3493-3518 _local_displacement_commit_kernel */
static void displacement_commit(const cvlbm2d_problem *p, cvlbm2d_fields *f, size_t n) {
  size_t N = (size_t)p->nx * p->ny;
  if (p->active[n] == 0) {
    f->u[n] = f->u[N + n] = f->u_star[n] = f->u_star[N + n] = 0.0;
    return;
  }
  double d0 = f->u_next[n] - f->u[n], d1 = f->u_next[N + n] - f->u[N + n];
  f->u[n] = f->u_next[n];
  f->u[N + n] = f->u_next[N + n];
  f->u_star[n] = f->u_star[n] + d0;
  f->u_star[N + n] = f->u_star[N + n] + d1;
}

/* C2:3213-3272 _local_dudx / _local_dudy (stride = ny along x, 1 along y) */
static double local_du(const double *uc, const int *act, size_t n, int i, int nax, size_t stride,
                       double h) {
  if (i > 0 && i + 1 < nax && act[n - stride] != 0 && act[n + stride] != 0)
    return (uc[n + stride] - uc[n - stride]) / (2.0 * h);
  if (i + 1 < nax && act[n + stride] != 0) {
    if (i + 2 < nax && act[n + 2 * stride] != 0)
      return (-3.0 * uc[n] + 4.0 * uc[n + stride] - uc[n + 2 * stride]) / (2.0 * h);
    return (uc[n + stride] - uc[n]) / h;
  }
  if (i > 0 && act[n - stride] != 0) {
    if (i > 1 && act[n - 2 * stride] != 0)
      return (3.0 * uc[n] - 4.0 * uc[n - stride] + uc[n - 2 * stride]) / (2.0 * h);
    return (uc[n] - uc[n - stride]) / h;
  }
  return 0.0;
}

/* C2:3521-3615 _local_compatibility_repair_kernel */
static void compatibility_repair(const cvlbm2d_problem *p, const mat_t *m, cvlbm2d_fields *f,
                                 size_t n) {
  size_t N = (size_t)p->nx * p->ny;
  int nx = p->nx, ny = p->ny, i = (int)(n / ny), j = (int)(n % ny);
  const int *act = p->active;
  if (act[n] == 0) return;
  if (p->interior_only) {
    if (i == 0 || i + 1 >= nx || j == 0 || j + 1 >= ny) return;
    if (act[n - ny] == 0 || act[n + ny] == 0 || act[n - 1] == 0 || act[n + 1] == 0) return;
  }
  double *U = f->U;
  double o11 = U[2 * N + n], o12 = U[3 * N + n], o21 = U[4 * N + n], o22 = U[5 * N + n];
  double t11 = 1.0 + local_du(f->u, act, n, i, nx, ny, p->dx);
  double t12 = local_du(f->u, act, n, j, ny, 1, p->dy);
  double t21 = local_du(f->u + N, act, n, i, nx, ny, p->dx);
  double t22 = 1.0 + local_du(f->u + N, act, n, j, ny, 1, p->dy);
  double alpha = fmax(0.0, fmin(1.0, p->blend));
  double n11 = o11, n12 = o12, n21 = o21, n22 = o22;
  for (int g = 0; g < 10; ++g) {
    n11 = o11 + alpha * (t11 - o11);
    n12 = o12 + alpha * (t12 - o12);
    n21 = o21 + alpha * (t21 - o21);
    n22 = o22 + alpha * (t22 - o22);
    if (n11 * n22 - n12 * n21 > m->jf) break;
    alpha = 0.5 * alpha;
  }
  double Po[4], Pn[4];
  piola_vec(o11, o12, o21, o22, m, Po);
  piola_vec(n11, n12, n21, n22, m, Pn);
  double d11 = Pn[0] - Po[0], d12 = Pn[1] - Po[1], d21 = Pn[2] - Po[2], d22 = Pn[3] - Po[3];
  double ff = 0.5 / p->c, qt = 0.25;
  double *fp = f->fpost;
  for (int q = 0; q < 4; ++q) {
    double cx = (double)CX[q], cy = (double)CY[q];
    size_t b = (size_t)(q * 6) * N + n;
    fp[b] = fp[b] - ff * (cx * d11 + cy * d12);
    fp[b + N] = fp[b + N] - ff * (cx * d21 + cy * d22);
    fp[b + 2 * N] = fp[b + 2 * N] + qt * (n11 - o11);
    fp[b + 3 * N] = fp[b + 3 * N] + qt * (n12 - o12);
    fp[b + 4 * N] = fp[b + 4 * N] + qt * (n21 - o21);
    fp[b + 5 * N] = fp[b + 5 * N] + qt * (n22 - o22);
  }
  U[2 * N + n] = n11;
  U[3 * N + n] = n12;
  U[4 * N + n] = n21;
  U[5 * N + n] = n22;
  if (f->P) {
    double Js = clamp_j(n11 * n22 - n12 * n21, m->jf);
    for (int k = 0; k < 4; ++k) f->P[k * N + n] = Pn[k];
    f->sigma[n] = (Pn[0] * n11 + Pn[1] * n12) / Js;
    f->sigma[N + n] = (Pn[0] * n21 + Pn[1] * n22) / Js;
    f->sigma[2 * N + n] = (Pn[2] * n11 + Pn[3] * n12) / Js;
    f->sigma[3 * N + n] = (Pn[2] * n21 + Pn[3] * n22) / Js;
  }
}

/* C2:2043-2060 _stream_masked_kernel (push) after V2:1482-1485 _clear_kernel */
static void stream_masked(const cvlbm2d_problem *p, const double *fpost, double *f1, size_t n) {
  size_t N = (size_t)p->nx * p->ny;
  int nx = p->nx, ny = p->ny, i = (int)(n / ny), j = (int)(n % ny);
  if (p->active[n] == 0) return;
  for (int q = 0; q < 4; ++q) {
    int ii = i + CX[q], jj = j + CY[q];
    if (ii >= 0 && ii < nx && jj >= 0 && jj < ny && p->active[ii * ny + jj] != 0)
      for (int a = 0; a < 6; ++a) f1[(q * 6 + a) * N + (size_t)ii * ny + jj] = fpost[(q * 6 + a) * N + n];
  }
}

/* C2:2063-3098 _apply_curved_boundary_links_kernel (closures bfl, lsq_bfl,
 * compat_bfl, local_char2, local_f, local_f_bfl) */
static void apply_links(const cvlbm2d_problem *p, const mat_t *m, const double *fpost, double *f1,
                        const double *U, const double *u, int ell, double tmid) {
  size_t N = (size_t)p->nx * p->ny;
  int nx = p->nx, ny = p->ny, recon = p->recon;
  int i = p->link_i[ell], j = p->link_j[ell], qo = p->link_q[ell];
  int bid = p->link_bid[ell];
  if (bid < 0 || bid >= 8) bid = 0;
  int kind = p->bc_kind[bid], mode = p->bc_mode[bid];
  const double *pp = p->bc_params + bid * 8;
  int qi = qo + 2;
  if (qi >= 4) qi -= 4;
  double eta = p->link_eta[ell], xb = p->link_xb[ell], yb = p->link_yb[ell];
  double nxb = p->link_nx[ell], nyb = p->link_ny[ell];
  double dxin = (double)CX[qi], dyin = (double)CY[qi];
  size_t n = (size_t)i * ny + j;
  double bv0 = curved_boundary_value_comp(0, mode, pp, xb, yb, nxb, nyb, tmid);
  double bv1 = curved_boundary_value_comp(1, mode, pp, xb, yb, nxb, nyb, tmid);
  if (kind == NEU_ && p->use_dynamic_traction) {
    bv0 = p->traction_x[ell];
    bv1 = p->traction_y[ell];
  }
  double Fg[4] = {U[2 * N + n], U[3 * N + n], U[4 * N + n], U[5 * N + n]};
  int iu = i - CX[qo], ju = j - CY[qo];
  int up_ok = iu >= 0 && iu < nx && ju >= 0 && ju < ny && p->active[iu * ny + ju] != 0;
  size_t nu = up_ok ? (size_t)iu * ny + ju : 0;
  if (recon == 0 || recon == 3 || recon == 2 || recon == 13) {
    if (up_ok)
      for (int k = 0; k < 4; ++k)
        Fg[k] = U[(2 + k) * N + n] + eta * (U[(2 + k) * N + n] - U[(2 + k) * N + nu]);
    if (recon == 2)
      for (int k = 0; k < 4; ++k) Fg[k] = lsq_U_at_boundary(p, U, p->lsq_wb, ell, 2 + k, Fg[k]);
  } else {
    for (int k = 0; k < 4; ++k) Fg[k] = interp_U_link(U, p->active, 2 + k, i, j, qo, eta, nx, ny);
  }
  if (recon == 11 || recon == 12)
    for (int k = 0; k < 4; ++k) Fg[k] = lsq_U_at_boundary(p, U, p->lsq_wb, ell, 2 + k, Fg[k]);
  if ((recon == 9 || recon == 10 || recon == 11) && p->lsq_valid[ell] != 0) {
    double tanx = -nyb, tany = nxb, dut0 = 0.0, dut1 = 0.0, wt_abs = 0.0;
    if (kind == NEU_) {
      for (int mm = 0; mm < 24; ++mm) {
        int ii = p->lsq_i[ell * 24 + mm], jj = p->lsq_j[ell * 24 + mm];
        if (ii >= 0 && jj >= 0) {
          double ww = p->lsq_wt[ell * 24 + mm];
          dut0 += ww * u[(size_t)ii * ny + jj];
          dut1 += ww * u[N + (size_t)ii * ny + jj];
          wt_abs += fabs(ww);
        }
      }
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
      double hn0 = Fg[0] * nxb + Fg[1] * nyb, hn1 = Fg[2] * nxb + Fg[3] * nyb;
      double gt0 = tanx + dut0, gt1 = tany + dut1;
      Fg[0] = hn0 * nxb + gt0 * tanx;
      Fg[1] = hn0 * nyb + gt0 * tany;
      Fg[2] = hn1 * nxb + gt1 * tanx;
      Fg[3] = hn1 * nyb + gt1 * tany;
    }
  }
  double Fb[4] = {Fg[0], Fg[1], Fg[2], Fg[3]};
  if (kind == NEU_) solve_normal_image(Fg, nxb, nyb, bv0, bv1, m, p->normal_solver, Fb);
  double Pb[4];
  piola_vec(Fb[0], Fb[1], Fb[2], Fb[3], m, Pb);
  int use_char = (recon == 11 || recon == 12) && kind == NEU_ && p->lsq_valid[ell] != 0;
  double cv[6] = {U[n], U[N + n], Fb[0], Fb[1], Fb[2], Fb[3]};
  if (kind == DIR_) {
    cv[0] = bv0;
    cv[1] = bv1;
  }
  double cw[6] = {0, 0, 0, 0, 0, 0};
  double dt = p->dt, c = p->c, om = p->omega;
  if (use_char) {
    double ux[6], uy[6], dv[6];
    for (int a = 0; a < 6; ++a) {
      ux[a] = lsq_U_at_boundary(p, U, p->lsq_wx, ell, a, 0.0);
      uy[a] = lsq_U_at_boundary(p, U, p->lsq_wy, ell, a, 0.0);
    }
    double sx = -eta * dt * c * (double)CX[qo], sy = -eta * dt * c * (double)CY[qo];
    for (int a = 0; a < 6; ++a) dv[a] = sx * ux[a] + sy * uy[a];
    double sc = 1.0;
    for (int g = 0; g < 10; ++g) {
      double t11 = cv[2] + sc * dv[2], t12 = cv[3] + sc * dv[3], t21 = cv[4] + sc * dv[4],
             t22 = cv[5] + sc * dv[5];
      if (t11 * t22 - t12 * t21 > 10.0 * m->jf) break;
      sc = 0.5 * sc;
    }
    for (int a = 0; a < 6; ++a) cv[a] = cv[a] + sc * dv[a];
    for (int a = 0; a < 6; ++a) {
      double b = source_comp(a, p->source_mode, p->source, cv[0], cv[1]);
      cw[a] = b - flux_jvp_comp(0, a, cv, ux, m) - flux_jvp_comp(1, a, cv, uy, m) +
              c * (dxin * ux[a] + dyin * uy[a]);
    }
  }
  for (int a = 0; a < 6; ++a) {
    double D = 1.0, S = 0.0;
    if (kind == DIR_) {
      if (a == 0) { D = -1.0; S = 0.5 * bv0; }
      else if (a == 1) { D = -1.0; S = 0.5 * bv1; }
      else if (a == 2) S = -dxin * bv0 / c;
      else if (a == 3) S = -dyin * bv0 / c;
      else if (a == 4) S = -dxin * bv1 / c;
      else S = -dyin * bv1 / c;
    } else {
      if (a == 0) S = -(dxin * Pb[0] + dyin * Pb[1]) / c;
      else if (a == 1) S = -(dxin * Pb[2] + dyin * Pb[3]) / c;
      else { D = -1.0; S = 0.5 * Fb[a - 2]; }
    }
    double fo = fpost[(size_t)(qo * 6 + a) * N + n], fi = fpost[(size_t)(qi * 6 + a) * N + n];
    double val;
    if (eta >= 0.5) {
      double al = 1.0 / (2.0 * eta);
      val = al * (D * fo + S) + (1.0 - al) * fi;
    } else {
      double up = fo;
      if (up_ok) up = fpost[(size_t)(qo * 6 + a) * N + nu];
      val = D * (2.0 * eta * fo + (1.0 - 2.0 * eta) * up) + S;
    }
    if (use_char && cv[2] * cv[5] - cv[3] * cv[4] > m->jf) {
      double Pc[4];
      piola_vec(cv[2], cv[3], cv[4], cv[5], m, Pc);
      double eq_jvp = equilibrium_jvp_comp(qi, a, cv, cw, m, c);
      double geq = equilibrium_comp(qi, a, cv, Pc, c);
      double sa = source_comp(a, p->source_mode, p->source, cv[0], cv[1]);
      val = geq - dt / om * eq_jvp + dt * (1.0 / om - 0.5) * 0.25 * sa;
    }
    f1[(size_t)(qi * 6 + a) * N + n] = val;
  }
}

/* C2:3127-3210 _refresh_masked_kernel */
static void refresh_masked(const cvlbm2d_problem *p, const mat_t *m, cvlbm2d_fields *f, size_t n,
                           int *invalid) {
  size_t N = (size_t)p->nx * p->ny;
  if (p->active[n] == 0) {
    for (int a = 0; a < 6; ++a) f->U[a * N + n] = 0.0;
    f->u[n] = f->u[N + n] = 0.0;
    if (f->P)
      for (int a = 0; a < 4; ++a) f->P[a * N + n] = f->sigma[a * N + n] = 0.0;
    return;
  }
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 4; ++q)
    for (int a = 0; a < 6; ++a) S[a] += f->f0[(q * 6 + a) * N + n];
  double hdt = 0.5 * p->dt;
  if (p->source_mode == 1) {
    for (int a = 0; a < 6; ++a) S[a] += hdt * p->source[a];
  } else if (p->source_mode == 2) {
    double den = 1.0 + hdt * p->source[0];
    S[0] = S[0] / den;
    S[1] = S[1] / den;
  }
  for (int a = 0; a < 6; ++a) f->U[a * N + n] = S[a];
  f->u[n] = f->u_star[n] + 0.5 * p->dt * S[0];
  f->u[N + n] = f->u_star[N + n] + 0.5 * p->dt * S[1];
  double J = S[2] * S[5] - S[3] * S[4];
  if (J <= m->jf) *invalid = 1;
  if (f->P) {
    double Js = clamp_j(J, m->jf), P[4];
    piola_vec(S[2], S[3], S[4], S[5], m, P);
    for (int k = 0; k < 4; ++k) f->P[k * N + n] = P[k];
    f->sigma[n] = (P[0] * S[2] + P[1] * S[3]) / Js;
    f->sigma[N + n] = (P[0] * S[4] + P[1] * S[5]) / Js;
    f->sigma[2 * N + n] = (P[2] * S[2] + P[3] * S[3]) / Js;
    f->sigma[3 * N + n] = (P[2] * S[4] + P[3] * S[5]) / Js;
  }
}

static int due(int interval, int64_t step) { return interval > 0 && step % interval == 0; }

/* C2:4163-4258 WarpCurvedBoundaryLBM2D.step */
int oracle2d_step(const cvlbm2d_problem *p, cvlbm2d_fields *f, oracle2d_scratch *s, double time,
                  int64_t step, int threads) {
  mat_t m = mat_of(&p->mat);
  long N = (long)p->nx * p->ny;
  int invalid = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  if (p->collision_model == 1) {
#pragma omp parallel for schedule(static) reduction(| : invalid)
    for (long n = 0; n < N; ++n) collide_masked_mrt(p, &m, f, (size_t)n, &invalid);
  } else {
#pragma omp parallel for schedule(static) reduction(| : invalid)
    for (long n = 0; n < N; ++n) collide_masked(p, &m, f, (size_t)n, &invalid);
  }
  if (due(p->disp_interval, step)) {
    for (int sw = 0; sw < p->disp_sweeps; ++sw) {
      memset(s->bc_diag, 0, sizeof(double) * N);
      memset(s->bc_rhs, 0, sizeof(double) * 2 * N);
      displacement_bc(p, f, s, time + 0.5 * p->dt);
#pragma omp parallel for schedule(static)
      for (long n = 0; n < N; ++n) displacement_relax(p, f, s, (size_t)n);
#pragma omp parallel for schedule(static)
      for (long n = 0; n < N; ++n) displacement_commit(p, f, (size_t)n);
    }
  }
  if (due(p->rep_interval, step)) {
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) compatibility_repair(p, &m, f, (size_t)n);
  }
  memset(f->f1, 0, sizeof(double) * 24 * N);
#pragma omp parallel for schedule(static)
  for (long n = 0; n < N; ++n) stream_masked(p, f->fpost, f->f1, (size_t)n);
  double tmid = time + 0.5 * p->dt;
#pragma omp parallel for schedule(static)
  for (int ell = 0; ell < p->n_links; ++ell)
    apply_links(p, &m, f->fpost, f->f1, f->U, f->u, ell, tmid);
  if (p->kinetic_filter > 0.0) {
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) kinetic_filter(p, f->f1, (size_t)n);
  }
  double *tmp = f->f0;
  f->f0 = f->f1;
  f->f1 = tmp;
  if (f->invalid) *f->invalid = invalid;
  return 0;
}

/* C2:4020-4035 apply_boundary_reconstruction */
int oracle2d_apply_boundary(const cvlbm2d_problem *p, cvlbm2d_fields *f, double t, int in_place) {
  mat_t m = mat_of(&p->mat);
  size_t N = (size_t)p->nx * p->ny;
  if (p->n_links == 0) return 0;
  if (in_place) memcpy(f->fpost, f->f0, sizeof(double) * 24 * N);
  double *target = in_place ? f->f0 : f->f1;
  for (int ell = 0; ell < p->n_links; ++ell) apply_links(p, &m, f->fpost, target, f->U, f->u, ell, t);
  return 0;
}

/* C2:4260-4291 refresh_current */
int oracle2d_refresh(const cvlbm2d_problem *p, cvlbm2d_fields *f) {
  mat_t m = mat_of(&p->mat);
  long N = (long)p->nx * p->ny;
  int invalid = 0;
  for (long n = 0; n < N; ++n) refresh_masked(p, &m, f, (size_t)n, &invalid);
  if (f->invalid) *f->invalid = invalid;
  return 0;
}

/* ---------------------------------------------------------------------- */
/* 3-D                                                                      */
/* ---------------------------------------------------------------------- */
static const int D3X[6] = {1, 0, 0, -1, 0, 0};
static const int D3Y[6] = {0, 1, 0, 0, -1, 0};
static const int D3Z[6] = {0, 0, 1, 0, 0, -1};
static int opp3(int q) { return q < 3 ? q + 3 : q - 3; }

/* V3:1066-1133 _flux_comp given P */
static double flux_comp3(int axis, int a, const double *U, const double *P) {
  if (a < 3) return -P[3 * a + axis];
  int r = a - 3;
  if (r % 3 == axis) return -U[r / 3];
  return 0.0;
}

/* V3:1136-1236 _equilibrium_comp */
static double equilibrium_comp3(int q, int a, const double *U, const double *P, double c) {
  double sx = (double)D3X[q], sy = (double)D3Y[q], sz = (double)D3Z[q];
  return (1.0 / 6.0) * (U[a] + (3.0 / c) * (sx * flux_comp3(0, a, U, P) + sy * flux_comp3(1, a, U, P) +
                                            sz * flux_comp3(2, a, U, P)));
}

/* V3:1371-1389 _source_comp */
static double source_comp3(int a, int mode, const double *sp, const double *v) {
  if (mode == 1) return sp[a];
  if (mode == 2 && a < 3) return -sp[0] * v[a];
  return 0.0;
}

/* C3:995-1133 _curved_value_comp (+ mode 208, linear ramp then hold) */
static double curved_value_comp3(int mode, const double *p, int comp, double x, double y, double z,
                                 double nx, double ny, double nz, double t, double jf) {
  double nn[3] = {nx, ny, nz};
  if (mode == 0) return 0.0;
  if (mode == 1) return p[comp];
  if (mode == 200) {
    double sc = 1.0;
    if (p[3] > 0.0 && t < p[3]) sc = sin(PI_ * t / p[3]) * sin(PI_ * t / p[3]);
    return p[comp] * sc;
  }
  if (mode == 4) {
    if (p[12] > 0.0 && t > p[12]) return 0.0;
    if (comp == 0) return p[0] * x + p[1] * y + p[2] * z + p[9];
    if (comp == 1) return p[3] * x + p[4] * y + p[5] * z + p[10];
    return p[6] * x + p[7] * y + p[8] * z + p[11];
  }
  if (mode == 204) {
    double act = p[3], den = p[4], sc = 1.0;
    if (den <= 0.0) den = 2.0 * act;
    if (act > 0.0 && t < act) sc = sin(PI_ * t / den) * sin(PI_ * t / den);
    return p[comp] * sc;
  }
  if (mode == 201) return p[3 * comp] * nx + p[3 * comp + 1] * ny + p[3 * comp + 2] * nz;
  if (mode == 205) {
    double tt = t;
    if (p[11] > 0.0 && tt > p[11]) tt = p[11];
    double F[9] = {1.0 + tt * p[0], tt * p[1], tt * p[2], tt * p[3], 1.0 + tt * p[4],
                   tt * p[5], tt * p[6], tt * p[7], 1.0 + tt * p[8]};
    mat_t nh = {1, p[9], p[10], 0.0, 0.0, 0.0, jf};
    double P[9];
    piola_mat(F, &nh, P);
    return P[3 * comp] * nx + P[3 * comp + 1] * ny + P[3 * comp + 2] * nz;
  }
  if (mode == 202) return p[0] * nn[comp];
  if (mode == 203 || mode == 208) {
    double sc = 1.0;
    if (mode == 203) {
      double act = p[1], den = p[2];
      if (den <= 0.0) den = 2.0 * act;
      if (act > 0.0 && t < act) sc = sin(PI_ * t / den) * sin(PI_ * t / den);
    } else if (p[1] > 0.0 && t < p[1]) {
      sc = t / p[1];
    }
    return p[0] * sc * nn[comp];
  }
  if (mode == 206) {
    double act = p[4], den = p[5], sc = 1.0;
    if (den <= 0.0) den = 2.0 * act;
    if (act > 0.0 && t < act) sc = sin(PI_ * t / den) * sin(PI_ * t / den);
    double dx = x - p[0], dy = y - p[1];
    if (comp == 0) return -sc * p[3] * dy;
    if (comp == 1) return sc * p[3] * dx;
    return sc * p[2];
  }
  if (mode == 207) {
    double act = p[4];
    if (act <= 0.0 || t >= act) return 0.0;
    double ph = PI_ * t / act;
    double s = 0.5 * (1.0 - cos(ph)), sdot = 0.5 * PI_ / act * sin(ph);
    double th = p[3] * s, thd = p[3] * sdot, dx = x - p[0], dy = y - p[1];
    if (comp == 0) return thd * (-sin(th) * dx - cos(th) * dy);
    if (comp == 1) return thd * (cos(th) * dx - sin(th) * dy);
    return p[2] * sdot;
  }
  return 0.0;
}

/* C3:2333-2347 _local_sine2_integral */
static double sine2_integral(double time, double act, double den) {
  if (act <= 0.0) return time;
  if (den <= 0.0) den = act;
  double t = time > 0.0 ? time : 0.0;
  if (t < act) return 0.5 * t - den * sin(2.0 * PI_ * t / den) / (4.0 * PI_);
  return 0.5 * act - den * sin(2.0 * PI_ * act / den) / (4.0 * PI_) + (t - act);
}

/* C3:2350-2399 _local_dirichlet_displacement_comp */
static double dirichlet_displacement3(int mode, const double *p, int comp, double x, double y,
                                      double z, double time) {
  if (mode == 0) return 0.0;
  if (mode == 1) return time * p[comp];
  if (mode == 200) return p[comp] * sine2_integral(time, p[3], p[3]);
  if (mode == 204) {
    double den = p[4];
    if (den <= 0.0) den = 2.0 * p[3];
    return p[comp] * sine2_integral(time, p[3], den);
  }
  if (mode == 4) {
    double at = time;
    if (p[12] > 0.0 && at > p[12]) at = p[12];
    double out = p[0] * x + p[1] * y + p[2] * z + p[9];
    if (comp == 1) out = p[3] * x + p[4] * y + p[5] * z + p[10];
    if (comp == 2) out = p[6] * x + p[7] * y + p[8] * z + p[11];
    return at * out;
  }
  if (mode == 207) {
    double s = 1.0;
    if (p[4] > 0.0 && time < p[4]) s = 0.5 * (1.0 - cos(PI_ * time / p[4]));
    double th = p[3] * s, dx = x - p[0], dy = y - p[1], c = cos(th), ss = sin(th);
    if (comp == 0) return (c - 1.0) * dx - ss * dy;
    if (comp == 1) return ss * dx + (c - 1.0) * dy;
    return p[2] * s;
  }
  return 0.0;
}

static void normalize3(double *v) {
  double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (r < 1.0e-30) r = 1.0e-30;
  v[0] = v[0] / r;
  v[1] = v[1] / r;
  v[2] = v[2] / r;
}
static void cross3(const double *a, const double *b, double *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* C3:1137-1157 _make_F_from_h */
static void make_F_from_h(const double *h, const double *n, const double *t1, const double *t2,
                          const double *g1, const double *g2, double *F) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[3 * i + j] = h[i] * n[j] + g1[i] * t1[j] + g2[i] * t2[j];
}

/* C3:1161-1202 _normal_residual_h */
static void normal_residual_h(const double *h, const double *n, const double *t1, const double *t2,
                              const double *g1, const double *g2, const double *T, const mat_t *m,
                              double *r) {
  double F[9], P[9];
  make_F_from_h(h, n, t1, t2, g1, g2, F);
  piola_mat(F, m, P);
  for (int i = 0; i < 3; ++i) r[i] = P[3 * i] * n[0] + P[3 * i + 1] * n[1] + P[3 * i + 2] * n[2] - T[i];
}

/* C3:1249-1329 _energy_Fb_neo_hooke_3d, all rows Neumann; returns 0 when degenerate */
static int energy_Fb3(const double *F, const double *n, const double *T, double lam, double mu,
                      double jf, double *Fb) {
  double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                   F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                   F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  double a[3], ho[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = cof[3 * i] * n[0] + cof[3 * i + 1] * n[1] + cof[3 * i + 2] * n[2];
    ho[i] = F[3 * i] * n[0] + F[3 * i + 1] * n[1] + F[3 * i + 2] * n[2];
  }
  double a2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  if (!(a2 > 1.0e-28)) return 0;
  double area = sqrt(a2), e[3] = {a[0] / area, a[1] / area, a[2] / area};
  double tau = T[0] * e[0] + T[1] * e[1] + T[2] * e[2];
  double aa = mu + 0.5 * lam * a2, bb = mu + 0.5 * lam;
  double disc = sqrt(tau * tau + 4.0 * aa * bb);
  double s = (tau + disc) / (2.0 * aa);
  if (tau < 0.0) s = 2.0 * bb / (disc - tau);
  if (!(area * s > jf)) return 0;
  for (int i = 0; i < 3; ++i) {
    double dh = ((T[i] - tau * e[i]) / mu + s * e[i]) - ho[i];
    for (int j = 0; j < 3; ++j) Fb[3 * i + j] = F[3 * i + j] + dh * n[j];
  }
  return 1;
}

/* C3:1332-1515 _solve_Fb_arbitrary_normal (with :1205-1246 acoustic Jacobian) */
static void solve_Fb_arbitrary_normal(const double *Fg, double nx, double ny, double nz,
                                      const double *T, const mat_t *m, int nj, double *out) {
  double n[3] = {nx, ny, nz};
  normalize3(n);
  if (nj == 2 && m->model == 1) {
    double Fb[9];
    if (energy_Fb3(Fg, n, T, m->lam, m->mu, m->jf, Fb) && det3(Fb) > m->jf) {
      memcpy(out, Fb, sizeof Fb);
      return;
    }
  }
  double ref[3] = {1.0, 0.0, 0.0};
  if (fabs(n[0]) >= 0.75) {
    ref[0] = 0.0;
    ref[1] = 1.0;
  }
  double t1[3], t2[3];
  cross3(n, ref, t1);
  normalize3(t1);
  cross3(n, t1, t2);
  double h[3], g1[3], g2[3];
  for (int i = 0; i < 3; ++i) {
    h[i] = Fg[3 * i] * n[0] + Fg[3 * i + 1] * n[1] + Fg[3 * i + 2] * n[2];
    g1[i] = Fg[3 * i] * t1[0] + Fg[3 * i + 1] * t1[1] + Fg[3 * i + 2] * t1[2];
    g2[i] = Fg[3 * i] * t2[0] + Fg[3 * i + 1] * t2[1] + Fg[3 * i + 2] * t2[2];
  }
  double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r[3];
    normal_residual_h(h, n, t1, t2, g1, g2, T, m, r);
    if (sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) < 1.0e-10) break;
    double A[9];
    if (nj != 0 && m->model == 1) {
      double F[9];
      make_F_from_h(h, n, t1, t2, g1, g2, F);
      double J = det3(F);
      if (J < m->jf) J = m->jf;
      double H[9] = {(F[4] * F[8] - F[5] * F[7]) / J, (F[5] * F[6] - F[3] * F[8]) / J,
                     (F[3] * F[7] - F[4] * F[6]) / J, (F[2] * F[7] - F[1] * F[8]) / J,
                     (F[0] * F[8] - F[2] * F[6]) / J, (F[1] * F[6] - F[0] * F[7]) / J,
                     (F[1] * F[5] - F[2] * F[4]) / J, (F[2] * F[3] - F[0] * F[5]) / J,
                     (F[0] * F[4] - F[1] * F[3]) / J};
      double beta = 0.5 * m->lam * (J * J - 1.0) - m->mu, coeff = m->lam * J * J - beta;
      double n2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2], v[3];
      for (int i = 0; i < 3; ++i) v[i] = H[3 * i] * n[0] + H[3 * i + 1] * n[1] + H[3 * i + 2] * n[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          A[3 * i + j] = i == j ? m->mu * n2 + coeff * v[i] * v[j] : coeff * v[i] * v[j];
    } else {
      for (int k = 0; k < 3; ++k) {
        double hp[3] = {h[0], h[1], h[2]}, rp[3];
        hp[k] = hp[k] + eps;
        normal_residual_h(hp, n, t1, t2, g1, g2, T, m, rp);
        for (int i = 0; i < 3; ++i) A[3 * i + k] = (rp[i] - r[i]) / eps;
      }
    }
    double a = A[0], b = A[1], c = A[2], d = A[3], e = A[4], ff = A[5], g = A[6], hh = A[7], ii = A[8];
    double det = a * (e * ii - ff * hh) - b * (d * ii - ff * g) + c * (d * hh - e * g);
    if (fabs(det) < 1.0e-14) break;
    double inv[9] = {(e * ii - ff * hh) / det, (c * hh - b * ii) / det, (b * ff - c * e) / det,
                     (ff * g - d * ii) / det,  (a * ii - c * g) / det,  (c * d - a * ff) / det,
                     (d * hh - e * g) / det,   (b * g - a * hh) / det,  (a * e - b * d) / det};
    double dl[3];
    for (int i = 0; i < 3; ++i) dl[i] = -(inv[3 * i] * r[0] + inv[3 * i + 1] * r[1] + inv[3 * i + 2] * r[2]);
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double cand[3] = {h[0] + step * dl[0], h[1] + step * dl[1], h[2] + step * dl[2]}, F[9];
      make_F_from_h(cand, n, t1, t2, g1, g2, F);
      if (det3(F) > m->jf) {
        h[0] = cand[0];
        h[1] = cand[1];
        h[2] = cand[2];
        break;
      }
      step = 0.5 * step;
    }
  }
  make_F_from_h(h, n, t1, t2, g1, g2, out);
}

/* C3:1249-1329 _energy_Fb_neo_hooke_3d, branch with Dirichlet rows */
static int energy_Fb3_mixed(const double *F, const double *n, const double *T, const int *ck,
                            double lam, double mu, double jf, double *Fb) {
  double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                   F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                   F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  double a[3], ho[3], an[3] = {0, 0, 0}, tn[3] = {0, 0, 0}, fx[3], h[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = cof[3 * i] * n[0] + cof[3 * i + 1] * n[1] + cof[3 * i + 2] * n[2];
    ho[i] = F[3 * i] * n[0] + F[3 * i + 1] * n[1] + F[3 * i + 2] * n[2];
    fx[i] = ho[i];
    if (ck[i] == NEU_) {
      an[i] = a[i];
      tn[i] = T[i];
      fx[i] = 0.0;
    }
  }
  double a2 = an[0] * an[0] + an[1] * an[1] + an[2] * an[2];
  double d = a[0] * fx[0] + a[1] * fx[1] + a[2] * fx[2];
  if (a2 > 1.0e-28) {
    double aa = mu + 0.5 * lam * a2, bb = (mu + 0.5 * lam) * a2;
    double cc = mu * d + (an[0] * tn[0] + an[1] * tn[1] + an[2] * tn[2]);
    double disc = sqrt(cc * cc + 4.0 * aa * bb);
    double J = (cc + disc) / (2.0 * aa);
    if (cc < 0.0) J = 2.0 * bb / (disc - cc);
    if (!(J > jf)) return 0;
    double area = sqrt(a2), e[3] = {an[0] / area, an[1] / area, an[2] / area};
    double te = tn[0] * e[0] + tn[1] * e[1] + tn[2] * e[2];
    for (int i = 0; i < 3; ++i) h[i] = fx[i] + (tn[i] - te * e[i]) / mu + ((J - d) / area) * e[i];
  } else if (a2 == 0.0 && d > jf) {
    for (int i = 0; i < 3; ++i) h[i] = fx[i] + tn[i] / mu;
  } else {
    return 0;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Fb[3 * i + j] = F[3 * i + j] + (h[i] - ho[i]) * n[j];
  return 1;
}

/* C3:1518-1737 _solve_Fb_componentwise_normal: Newton on the Neumann rows only */
static void solve_Fb_componentwise_normal(const double *Fg, double nx, double ny, double nz,
                                          const double *T, const int *ck, const mat_t *m, int nj,
                                          double *out) {
  double n[3] = {nx, ny, nz};
  normalize3(n);
  if (nj == 2 && m->model == 1) {
    double Fb[9];
    if (energy_Fb3_mixed(Fg, n, T, ck, m->lam, m->mu, m->jf, Fb) && det3(Fb) > m->jf) {
      memcpy(out, Fb, sizeof Fb);
      return;
    }
  }
  double ref[3] = {1.0, 0.0, 0.0};
  if (fabs(n[0]) >= 0.75) {
    ref[0] = 0.0;
    ref[1] = 1.0;
  }
  double t1[3], t2[3];
  cross3(n, ref, t1);
  normalize3(t1);
  cross3(n, t1, t2);
  double h[3], g1[3], g2[3];
  for (int i = 0; i < 3; ++i) {
    h[i] = Fg[3 * i] * n[0] + Fg[3 * i + 1] * n[1] + Fg[3 * i + 2] * n[2];
    g1[i] = Fg[3 * i] * t1[0] + Fg[3 * i + 1] * t1[1] + Fg[3 * i + 2] * t1[2];
    g2[i] = Fg[3 * i] * t2[0] + Fg[3 * i + 1] * t2[1] + Fg[3 * i + 2] * t2[2];
  }
  double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r[3], rm[3];
    normal_residual_h(h, n, t1, t2, g1, g2, T, m, r);
    for (int i = 0; i < 3; ++i) rm[i] = ck[i] == NEU_ ? r[i] : 0.0;
    if (sqrt(rm[0] * rm[0] + rm[1] * rm[1] + rm[2] * rm[2]) < 1.0e-10) break;
    double A[9];
    if (nj != 0 && m->model == 1) {
      double F[9];
      make_F_from_h(h, n, t1, t2, g1, g2, F);
      double J = det3(F);
      if (J < m->jf) J = m->jf;
      double H[9] = {(F[4] * F[8] - F[5] * F[7]) / J, (F[5] * F[6] - F[3] * F[8]) / J,
                     (F[3] * F[7] - F[4] * F[6]) / J, (F[2] * F[7] - F[1] * F[8]) / J,
                     (F[0] * F[8] - F[2] * F[6]) / J, (F[1] * F[6] - F[0] * F[7]) / J,
                     (F[1] * F[5] - F[2] * F[4]) / J, (F[2] * F[3] - F[0] * F[5]) / J,
                     (F[0] * F[4] - F[1] * F[3]) / J};
      double beta = 0.5 * m->lam * (J * J - 1.0) - m->mu, coeff = m->lam * J * J - beta;
      double n2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2], v[3];
      for (int i = 0; i < 3; ++i) v[i] = H[3 * i] * n[0] + H[3 * i + 1] * n[1] + H[3 * i + 2] * n[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          A[3 * i + j] = i == j ? m->mu * n2 + coeff * v[i] * v[j] : coeff * v[i] * v[j];
    } else {
      for (int k = 0; k < 3; ++k) {
        double hp[3] = {h[0], h[1], h[2]}, rp[3];
        hp[k] = hp[k] + eps;
        normal_residual_h(hp, n, t1, t2, g1, g2, T, m, rp);
        for (int i = 0; i < 3; ++i) A[3 * i + k] = (rp[i] - r[i]) / eps;
      }
    }
    for (int i = 0; i < 3; ++i)
      if (ck[i] != NEU_)
        for (int k = 0; k < 3; ++k) A[3 * i + k] = i == k ? 1.0 : 0.0;
    double a = A[0], b = A[1], c = A[2], d = A[3], e = A[4], ff = A[5], g = A[6], hh = A[7], ii = A[8];
    double det = a * (e * ii - ff * hh) - b * (d * ii - ff * g) + c * (d * hh - e * g);
    if (fabs(det) < 1.0e-14) break;
    double inv[9] = {(e * ii - ff * hh) / det, (c * hh - b * ii) / det, (b * ff - c * e) / det,
                     (ff * g - d * ii) / det,  (a * ii - c * g) / det,  (c * d - a * ff) / det,
                     (d * hh - e * g) / det,   (b * g - a * hh) / det,  (a * e - b * d) / det};
    double dl[3];
    for (int i = 0; i < 3; ++i)
      dl[i] = -(inv[3 * i] * rm[0] + inv[3 * i + 1] * rm[1] + inv[3 * i + 2] * rm[2]);
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double cand[3], F[9];
      for (int i = 0; i < 3; ++i) cand[i] = ck[i] == NEU_ ? h[i] + step * dl[i] : h[i];
      make_F_from_h(cand, n, t1, t2, g1, g2, F);
      if (det3(F) > m->jf) {
        h[0] = cand[0];
        h[1] = cand[1];
        h[2] = cand[2];
        break;
      }
      step = 0.5 * step;
    }
  }
  make_F_from_h(h, n, t1, t2, g1, g2, out);
}

/* C3:2719-2725 _state_det3 */
static double state_det3(const double *U) {
  return U[3] * (U[7] * U[11] - U[8] * U[10]) - U[4] * (U[6] * U[11] - U[8] * U[9]) +
         U[5] * (U[6] * U[10] - U[7] * U[9]);
}

/* C3:2728-2752 _state_flux_jvp3 */
static void state_flux_jvp3(int axis, const double *U, const double *W, const mat_t *m, double *out) {
  double sc = 1.0;
  for (int a = 0; a < 12; ++a) sc = fmax(sc, fabs(W[a]));
  double eps = 1.0e-6 / sc, Up[12], Um[12], Pp[9], Pm[9];
  for (int a = 0; a < 12; ++a) {
    Up[a] = U[a] + eps * W[a];
    Um[a] = U[a] - eps * W[a];
  }
  piola_mat(Up + 3, m, Pp);
  piola_mat(Um + 3, m, Pm);
  for (int a = 0; a < 12; ++a) out[a] = 0.0;
  for (int i = 0; i < 3; ++i) {
    out[i] = -(Pp[3 * i + axis] - Pm[3 * i + axis]) / (2.0 * eps);
    out[3 + 3 * i + axis] = -W[i];
  }
}

/* C3:2755-2809 _local_characteristic_population3 */
static void local_characteristic_population3(const double *Ub, const double *Gx, const double *Gy,
                                             const double *Gz, const double *d, double eta, double dt,
                                             double c, const cvlbm3d_problem *p, const mat_t *m,
                                             double omega, double *out) {
  double shift[12], dG[12], Uc[12];
  for (int a = 0; a < 12; ++a) {
    dG[a] = d[0] * Gx[a] + d[1] * Gy[a] + d[2] * Gz[a];
    shift[a] = eta * dt * c * dG[a];
  }
  double chi = 1.0;
  for (int g = 0; g < 10; ++g) {
    double t[12];
    for (int a = 0; a < 12; ++a) t[a] = Ub[a] + chi * shift[a];
    if (state_det3(t) > 10.0 * m->jf) break;
    chi = 0.5 * chi;
  }
  for (int a = 0; a < 12; ++a) Uc[a] = Ub[a] + chi * shift[a];
  double B[12], j0[12], j1[12], j2[12], w[12], Aw[12], P[9], fl[12];
  for (int a = 0; a < 12; ++a) B[a] = source_comp3(a, p->source_mode, p->source, Uc);
  state_flux_jvp3(0, Uc, Gx, m, j0);
  state_flux_jvp3(1, Uc, Gy, m, j1);
  state_flux_jvp3(2, Uc, Gz, m, j2);
  for (int a = 0; a < 12; ++a) w[a] = B[a] - j0[a] - j1[a] - j2[a] + c * dG[a];
  int axis = 0;
  if (fabs(d[1]) > 0.5) axis = 1;
  if (fabs(d[2]) > 0.5) axis = 2;
  state_flux_jvp3(axis, Uc, w, m, Aw);
  piola_mat(Uc + 3, m, P);
  for (int a = 0; a < 12; ++a) fl[a] = 0.0;
  for (int i = 0; i < 3; ++i) {
    fl[i] = -P[3 * i + axis];
    fl[3 + 3 * i + axis] = -Uc[i];
  }
  for (int a = 0; a < 12; ++a)
    out[a] = (Uc[a] + 3.0 * d[axis] * fl[a] / c - dt / omega * (w[a] + 3.0 * d[axis] * Aw[a] / c) +
              dt * (1.0 / omega - 0.5) * B[a]) / 6.0;
}

/* C3:2192-2316 _sparse_collide_inplace_kernel */
static void sparse_collide(const cvlbm3d_problem *p, const mat_t *m, cvlbm3d_fields *f, size_t n,
                           int *invalid) {
  size_t N = (size_t)p->n_active;
  double S[12] = {0};
  for (int q = 0; q < 6; ++q)
    for (int a = 0; a < 12; ++a) S[a] += f->f0[(q * 12 + a) * N + n];
  double hdt = 0.5 * p->dt;
  if (p->source_mode == 1) {
    for (int a = 0; a < 12; ++a) S[a] += hdt * p->source[a];
  } else if (p->source_mode == 2) {
    double den = 1.0 + hdt * p->source[0];
    for (int a = 0; a < 3; ++a) S[a] = S[a] / den;
  }
  for (int a = 0; a < 12; ++a) f->U[a * N + n] = S[a];
  for (int d = 0; d < 3; ++d) {
    double uu = f->u_star[d * N + n] + hdt * S[d];
    f->u[d * N + n] = uu;
    f->u_star[d * N + n] = uu + hdt * S[d];
  }
  if (det3(S + 3) <= m->jf) *invalid = 1;
  double P[9];
  piola_mat(S + 3, m, P);
  for (int q = 0; q < 6; ++q)
    for (int a = 0; a < 12; ++a) {
      double feq = equilibrium_comp3(q, a, S, P, p->c);
      double old = f->f0[(q * 12 + a) * N + n];
      f->f0[(q * 12 + a) * N + n] = old + p->omega * (feq - old) +
                                    p->dt * (2.0 - p->omega) * (1.0 / 12.0) *
                                        source_comp3(a, p->source_mode, p->source, S);
    }
}

/* C3:2412-2469 _sparse_local_build_bc, serial in link order */
static void sparse_build_bc(const cvlbm3d_problem *p, const cvlbm3d_fields *f, oracle3d_scratch *s,
                            double time) {
  size_t N = (size_t)p->n_active;
  double w2 = p->weight * p->weight;
  for (int ell = 0; ell < p->n_links; ++ell) {
    int bid = p->link_bid[ell], force_all = 0;
    if (p->disp_bid >= 0) {
      if (bid != p->disp_bid) continue;
      force_all = 1;
    }
    int pn = p->link_p[ell];
    if (pn < 0) continue;
    double x = p->link_xb[ell], y = p->link_yb[ell], z = p->link_zb[ell];
    double db[3] = {x - ((double)p->active_i[pn] + 0.5) * p->dx,
                    y - ((double)p->active_j[pn] + 0.5) * p->dy,
                    z - ((double)p->active_k[pn] + 0.5) * p->dz};
    const double *pp = p->bc_params + bid * 16;
    int mode = p->bc_mode[bid];
    for (int comp = 0; comp < 3; ++comp) {
      double ub = dirichlet_displacement3(mode, pp, comp, x, y, z, time);
      if (force_all || p->bc_comp_kind[comp * 16 + bid] == DIR_) {
        const double *U = f->U;
        double e[3];
        for (int k = 0; k < 3; ++k) e[k] = U[(3 + 3 * comp + k) * N + pn] - (k == comp ? 1.0 : 0.0);
        double rhs = ub - (e[0] * db[0] + e[1] * db[1] + e[2] * db[2]);
        s->bc_diag[comp * N + pn] += w2;
        s->bc_rhs[comp * N + pn] += w2 * rhs;
      }
    }
  }
}

/* C3:2472-2540 _sparse_local_displacement_sweep + _commit */
static void sparse_sweep(const cvlbm3d_problem *p, const cvlbm3d_fields *f, const oracle3d_scratch *s,
                         size_t n) {
  size_t N = (size_t)p->n_active;
  const double *U = f->U, *u = f->u;
  double d[3], r[3];
  for (int c = 0; c < 3; ++c) {
    d[c] = s->bc_diag[c * N + n];
    r[c] = s->bc_rhs[c * N + n];
  }
  for (int q = 0; q < 6; ++q) {
    int pn = p->neighbor[q * N + n];
    if (pn < 0) continue;
    double ddx = (double)D3X[q] * p->dx, ddy = (double)D3Y[q] * p->dy, ddz = (double)D3Z[q] * p->dz;
    double g0 = 0.5 * ((U[3 * N + n] + U[3 * N + pn] - 2.0) * ddx + (U[4 * N + n] + U[4 * N + pn]) * ddy +
                       (U[5 * N + n] + U[5 * N + pn]) * ddz);
    double g1 = 0.5 * ((U[6 * N + n] + U[6 * N + pn]) * ddx + (U[7 * N + n] + U[7 * N + pn] - 2.0) * ddy +
                       (U[8 * N + n] + U[8 * N + pn]) * ddz);
    double g2 = 0.5 * ((U[9 * N + n] + U[9 * N + pn]) * ddx + (U[10 * N + n] + U[10 * N + pn]) * ddy +
                       (U[11 * N + n] + U[11 * N + pn] - 2.0) * ddz);
    r[0] += u[pn] - g0;
    r[1] += u[N + pn] - g1;
    r[2] += u[2 * N + pn] - g2;
    d[0] += 1.0;
    d[1] += 1.0;
    d[2] += 1.0;
  }
  for (int c = 0; c < 3; ++c) {
    f->u_next[c * N + n] = u[c * N + n];
    if (d[c] > 0.0) f->u_next[c * N + n] = u[c * N + n] + p->relax * (r[c] / d[c] - u[c * N + n]);
  }
}

/* C3:2543-2571 _sparse_local_du_axis */
static double sparse_du_axis(const double *uc, const int *nbr, size_t N, size_t n, int qp, int qm,
                             double h) {
  int pp = nbr[qp * N + n], pm = nbr[qm * N + n];
  if (pp >= 0 && pm >= 0) return (uc[pp] - uc[pm]) / (2.0 * h);
  if (pp >= 0) {
    int pp2 = nbr[qp * N + pp];
    if (pp2 >= 0) return (-3.0 * uc[n] + 4.0 * uc[pp] - uc[pp2]) / (2.0 * h);
    return (uc[pp] - uc[n]) / h;
  }
  if (pm >= 0) {
    int pm2 = nbr[qm * N + pm];
    if (pm2 >= 0) return (3.0 * uc[n] - 4.0 * uc[pm] + uc[pm2]) / (2.0 * h);
    return (uc[n] - uc[pm]) / h;
  }
  return 0.0;
}

/* C3:2574-2672 _sparse_local_repair_F */
static void sparse_repair(const cvlbm3d_problem *p, const mat_t *m, cvlbm3d_fields *f, size_t n) {
  size_t N = (size_t)p->n_active;
  double beta = fmax(0.0, fmin(1.0, p->blend)), o[9], t[9], nn[9], h[3] = {p->dx, p->dy, p->dz};
  for (int k = 0; k < 9; ++k) o[k] = f->U[(3 + k) * N + n];
  for (int c = 0; c < 3; ++c)
    for (int ax = 0; ax < 3; ++ax) {
      double g = sparse_du_axis(f->u + c * N, p->neighbor, N, n, ax, ax + 3, h[ax]);
      t[3 * c + ax] = c == ax ? 1.0 + g : g;
    }
  for (int k = 0; k < 9; ++k) nn[k] = o[k] + beta * (t[k] - o[k]);
  if (det3(nn) <= m->jf) return;
  double Po[9], Pn[9];
  piola_mat(o, m, Po);
  piola_mat(nn, m, Pn);
  double ff = 0.5 / p->c, sixth = 1.0 / 6.0;
  for (int q = 0; q < 6; ++q) {
    double sx = (double)D3X[q], sy = (double)D3Y[q], sz = (double)D3Z[q];
    size_t b = (size_t)(q * 12) * N + n;
    for (int i = 0; i < 3; ++i)
      f->f0[b + i * N] = f->f0[b + i * N] - ff * (sx * (Pn[3 * i] - Po[3 * i]) + sy * (Pn[3 * i + 1] - Po[3 * i + 1]) +
                                                  sz * (Pn[3 * i + 2] - Po[3 * i + 2]));
    for (int k = 0; k < 9; ++k) f->f0[b + (3 + k) * N] = f->f0[b + (3 + k) * N] + sixth * (nn[k] - o[k]);
  }
  for (int k = 0; k < 9; ++k) f->U[(3 + k) * N + n] = nn[k];
}

/* C3:2675-2700 gather, :2887-3151 prepare, :3154-3241 BFL, :2812-2884 characteristic */
static void sparse_link(const cvlbm3d_problem *p, const mat_t *m, const cvlbm3d_fields *f,
                        const double *src, double *dst, int ell, double t, int *invalid) {
  size_t N = (size_t)p->n_active, L = (size_t)p->n_links;
  int bid = p->link_bid[ell], kind = p->bc_kind[bid], mode = p->bc_mode[bid];
  int ck[3] = {p->bc_comp_kind[bid], p->bc_comp_kind[16 + bid], p->bc_comp_kind[32 + bid]};
  const double *pp = p->bc_params + bid * 16;
  double x = p->link_xb[ell], y = p->link_yb[ell], z = p->link_zb[ell];
  double nx = p->link_nx[ell], ny = p->link_ny[ell], nz = p->link_nz[ell];
  int n = p->link_p[ell], up = p->link_up[ell], qo = p->link_q[ell], qi = opp3(qo);
  double eta = p->link_eta[ell];
  double G[4][12];
  memset(G, 0, sizeof G);
  int gathered = p->has_char && p->char_idx[ell] >= 0;
  if (gathered) {
    for (int a = 0; a < 12; ++a) {
      double acc[4] = {0, 0, 0, 0};
      for (int mm = 0; mm < 64; ++mm) {
        int q = p->char_idx[mm * L + ell];
        if (q >= 0) {
          double uv = f->U[a * N + q];
          for (int k = 0; k < 4; ++k) acc[k] += p->char_w[(k * 64 + mm) * L + ell] * uv;
        }
      }
      for (int k = 0; k < 4; ++k) {
        G[k][a] = acc[k];
        if (f->char_state) f->char_state[(k * 12 + a) * L + ell] = acc[k];
      }
    }
  }
  double T[3];
  for (int r = 0; r < 3; ++r) T[r] = curved_value_comp3(mode, pp, r, x, y, z, nx, ny, nz, t, m->jf);
  if (p->dyn_enabled && p->dyn_enabled[ell] != 0)
    for (int r = 0; r < 3; ++r) T[r] = p->dyn_traction[r * L + ell];
  double Fb[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Pb[9] = {0};
  int anyN = ck[0] == NEU_ || ck[1] == NEU_ || ck[2] == NEU_;
  if (anyN) {
    double F[9];
    for (int k = 0; k < 9; ++k) F[k] = f->U[(3 + k) * N + n];
    if (p->recon == 2 || p->recon == 4) {
      if (up >= 0)
        for (int k = 0; k < 9; ++k) F[k] = f->U[(3 + k) * N + n] + eta * (f->U[(3 + k) * N + n] - f->U[(3 + k) * N + up]);
      if (p->recon == 2 && p->has_tangent_lsq && p->lsq_valid[ell] != 0) {
        double nv[3] = {nx, ny, nz}, ref[3] = {1.0, 0.0, 0.0}, t1[3], t2[3];
        normalize3(nv);
        if (fabs(nv[0]) >= 0.75) {
          ref[0] = 0.0;
          ref[1] = 1.0;
        }
        cross3(nv, ref, t1);
        normalize3(t1);
        cross3(nv, t1, t2);
        double du1[3] = {0, 0, 0}, du2[3] = {0, 0, 0}, wt_abs = 0.0;
        for (int mm = 0; mm < 32; ++mm) {
          int q = p->lsq_p[ell * 32 + mm];
          if (q >= 0) {
            double w1 = p->lsq_wt1[ell * 32 + mm], w2 = p->lsq_wt2[ell * 32 + mm];
            for (int r = 0; r < 3; ++r) {
              du1[r] += w1 * f->u[r * N + q];
              du2[r] += w2 * f->u[r * N + q];
            }
            wt_abs += fabs(w1) + fabs(w2);
          }
        }
        if (wt_abs > 0.0) {
          double h[3], g1[3], g2[3];
          for (int r = 0; r < 3; ++r) {
            h[r] = F[3 * r] * nv[0] + F[3 * r + 1] * nv[1] + F[3 * r + 2] * nv[2];
            g1[r] = t1[r] + du1[r];
            g2[r] = t2[r] + du2[r];
          }
          make_F_from_h(h, nv, t1, t2, g1, g2, F);
        }
      }
    }
    if (p->recon == 3)
      for (int k = 0; k < 9; ++k) F[k] = G[0][3 + k];
    memcpy(Fb, F, sizeof F);
    if (ck[0] == NEU_ && ck[1] == NEU_ && ck[2] == NEU_)
      solve_Fb_arbitrary_normal(F, nx, ny, nz, T, m, p->normal_solver, Fb);
    else if (ck[0] == NEU_ || ck[1] == NEU_ || ck[2] == NEU_)
      solve_Fb_componentwise_normal(F, nx, ny, nz, T, ck, m, p->normal_solver, Fb);
    piola_mat(Fb, m, Pb);
  }
  if (f->link_kind) {
    f->link_kind[ell] = kind;
    for (int r = 0; r < 3; ++r) {
      f->link_comp_kind[r * L + ell] = ck[r];
      f->link_bv[r * L + ell] = T[r];
    }
    for (int k = 0; k < 9; ++k) {
      f->link_Fb[k * L + ell] = Fb[k];
      f->link_Pb[k * L + ell] = Pb[k];
    }
  }
  double e_bfl = p->recon == 1 ? 0.5 : eta;
  double din[3] = {(double)D3X[qi], (double)D3Y[qi], (double)D3Z[qi]}, c = p->c;
  for (int a = 0; a < 12; ++a) {
    int row = a < 3 ? a : (a - 3) / 3;
    double D = 1.0, S = 0.0;
    if (ck[row] == DIR_) {
      if (a < 3) {
        D = -1.0;
        S = T[a] / 3.0;
      } else {
        S = -din[(a - 3) - row * 3] * T[row] / c;
      }
    } else if (a < 3) {
      S = -(din[0] * Pb[3 * a] + din[1] * Pb[3 * a + 1] + din[2] * Pb[3 * a + 2]) / c;
    } else {
      D = -1.0;
      S = Fb[a - 3] / 3.0;
    }
    double fo = src[(qo * 12 + a) * N + n], fi = src[(qi * 12 + a) * N + n], val;
    if (e_bfl >= 0.5) {
      double al = 1.0 / (2.0 * e_bfl);
      val = al * (D * fo + S) + (1.0 - al) * fi;
    } else {
      double upv = fo;
      if (up >= 0) upv = src[(qo * 12 + a) * N + up];
      val = D * (2.0 * e_bfl * fo + (1.0 - 2.0 * e_bfl) * upv) + S;
    }
    dst[(qi * 12 + a) * N + n] = val;
  }
  if (gathered && anyN) {
    double Ub[12], out[12];
    for (int a = 0; a < 3; ++a) Ub[a] = ck[a] == DIR_ ? T[a] : f->U[a * N + n];
    for (int k = 0; k < 9; ++k) Ub[3 + k] = Fb[k];
    if (state_det3(Ub) <= m->jf) *invalid = 1;
    local_characteristic_population3(Ub, G[1], G[2], G[3], din, eta, p->dt, c, p, m, p->omega, out);
    for (int a = 0; a < 12; ++a) {
      int row = a < 3 ? a : (a - 3) / 3;
      if (ck[row] == NEU_) dst[(qi * 12 + a) * N + n] = out[a];
    }
  }
}

/* C3:4549-4589 WarpSparseCurvedBoundaryLBM3D.step */
int oracle3d_step(const cvlbm3d_problem *p, cvlbm3d_fields *f, oracle3d_scratch *s, double time,
                  int64_t step, int threads) {
  mat_t m = mat_of(&p->mat);
  long N = p->n_active;
  int invalid = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(static) reduction(| : invalid)
  for (long n = 0; n < N; ++n) sparse_collide(p, &m, f, (size_t)n, &invalid);
  if (due(p->disp_interval, step)) {
    memset(s->bc_diag, 0, sizeof(double) * 3 * N);
    memset(s->bc_rhs, 0, sizeof(double) * 3 * N);
    sparse_build_bc(p, f, s, time + 0.5 * p->dt);
    for (int sw = 0; sw < p->disp_sweeps; ++sw) {
#pragma omp parallel for schedule(static)
      for (long n = 0; n < N; ++n) sparse_sweep(p, f, s, (size_t)n);
#pragma omp parallel for schedule(static)
      for (long k = 0; k < 3 * N; ++k) {
        double dl = f->u_next[k] - f->u[k];
        f->u[k] = f->u_next[k];
        f->u_star[k] = f->u_star[k] + dl;
      }
    }
  }
  if (due(p->rep_interval, step)) {
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) sparse_repair(p, &m, f, (size_t)n);
  }
  memset(f->f1, 0, sizeof(double) * 72 * N);
#pragma omp parallel for schedule(static)
  for (long n = 0; n < N; ++n)
    for (int q = 0; q < 6; ++q) {
      int nid = p->neighbor[q * N + n];
      if (nid >= 0)
        for (int a = 0; a < 12; ++a) f->f1[(q * 12 + a) * (size_t)N + nid] = f->f0[(q * 12 + a) * (size_t)N + n];
    }
  double tmid = time + 0.5 * p->dt;
  int inv2 = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : inv2)
  for (int ell = 0; ell < p->n_links; ++ell) sparse_link(p, &m, f, f->f0, f->f1, ell, tmid, &inv2);
  double *tmp = f->f0;
  f->f0 = f->f1;
  f->f1 = tmp;
  if (f->invalid) *f->invalid = invalid | inv2;
  return 0;
}

/* C3:4339-4399 apply_boundary_reconstruction */
int oracle3d_apply_boundary(const cvlbm3d_problem *p, cvlbm3d_fields *f, double t, int in_place) {
  mat_t m = mat_of(&p->mat);
  size_t N = (size_t)p->n_active;
  if (p->n_links == 0) return 0;
  int inv = 0;
  if (in_place) memcpy(f->f1, f->f0, sizeof(double) * 72 * N);
  const double *src = in_place ? f->f1 : f->f0;
  double *dst = in_place ? f->f0 : f->f1;
  for (int ell = 0; ell < p->n_links; ++ell) sparse_link(p, &m, f, src, dst, ell, t, &inv);
  if (f->invalid && inv) *f->invalid = 1;
  return 0;
}

/* C3:2109-2189 _sparse_refresh_kernel */
int oracle3d_refresh(const cvlbm3d_problem *p, cvlbm3d_fields *f) {
  mat_t m = mat_of(&p->mat);
  size_t N = (size_t)p->n_active;
  int invalid = 0;
  for (size_t n = 0; n < N; ++n) {
    double S[12] = {0};
    for (int q = 0; q < 6; ++q)
      for (int a = 0; a < 12; ++a) S[a] += f->f0[(q * 12 + a) * N + n];
    double hdt = 0.5 * p->dt;
    if (p->source_mode == 1) {
      for (int a = 0; a < 12; ++a) S[a] += hdt * p->source[a];
    } else if (p->source_mode == 2) {
      double den = 1.0 + hdt * p->source[0];
      for (int a = 0; a < 3; ++a) S[a] = S[a] / den;
    }
    for (int a = 0; a < 12; ++a) f->U[a * N + n] = S[a];
    for (int d = 0; d < 3; ++d) f->u[d * N + n] = f->u_star[d * N + n] + hdt * S[d];
    if (det3(S + 3) <= m.jf) invalid = 1;
  }
  if (f->invalid) *f->invalid = invalid;
  return 0;
}
