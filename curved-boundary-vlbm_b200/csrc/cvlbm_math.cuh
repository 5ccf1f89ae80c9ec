// Device math shared by the D2Q4x6 and D3Q6x12 kernels.
//
// Every function states the reference routine it evaluates.  Expressions keep
// the reference's association order (Python/Warp evaluate a*b*c as (a*b)*c and
// a+b+c as (a+b)+c); together with --fmad=false this makes the kernels
// reproduce the reference's float64 arithmetic operation for operation.  The
// only deviation is the count of constitutive evaluations: the reference
// re-evaluates the Piola map inside every flux call (48 times per 2-D node and
// 216 times per 3-D node in one collision); the map is a pure function, so it
// is evaluated once here and the identical value reused.
#pragma once

#include <math.h>
#include <stdint.h>

#define CV_DEV __device__ __forceinline__

namespace cv {

constexpr double kPi = 3.141592653589793238462643383279502884;

enum : int { kDirichlet = 1, kNeumann = 2 };
enum : int { kSrcNone = 0, kSrcConstant = 1, kSrcDamping = 2 };
enum : int { kSolverFD = 0, kSolverAcoustic = 1, kSolverEnergy = 2 };
enum : int {
  kMatSVK = 0,
  kMatNeoHooke = 1,
  kMatLogNeoHooke = 2,
  kMatMooneyRivlin = 3,
  kMatYeoh = 4,
  kMatGent = 5,
  kMatSix = 6  // 2-D: Sugiyama SVK; 3-D: SPH neo-Hooke
};

struct Mat {
  int model;
  double lam, mu, p0, p1, p2, jf;
};

CV_DEV double clamp_j(double j, double fl) { return j < fl ? fl : j; }

// ---------------------------------------------------------------------------
// 2-D first Piola stress, row-major (P11, P12, P21, P22).
// two_d/vector_nonlinear_elastic_warp.py:938-1052 (_piola_vec).
// ---------------------------------------------------------------------------
struct P2 {
  double a, b, c, d;
};

CV_DEV P2 piola2(double F11, double F12, double F21, double F22, const Mat& m) {
  const double lam = m.lam, mu = m.mu;
  if (m.model == kMatSVK) {
    double C00 = F11 * F11 + F21 * F21;
    double C01 = F11 * F12 + F21 * F22;
    double C11 = F12 * F12 + F22 * F22;
    double E00 = 0.5 * (C00 - 1.0);
    double E01 = 0.5 * C01;
    double E11 = 0.5 * (C11 - 1.0);
    double trE = E00 + E11;
    double S00 = lam * trE + 2.0 * mu * E00;
    double S01 = 2.0 * mu * E01;
    double S11 = lam * trE + 2.0 * mu * E11;
    return {F11 * S00 + F12 * S01, F11 * S01 + F12 * S11, F21 * S00 + F22 * S01,
            F21 * S01 + F22 * S11};
  }
  double J = clamp_j(F11 * F22 - F12 * F21, m.jf);
  double H00 = F22 / J;
  double H01 = -F21 / J;
  double H10 = -F12 / J;
  double H11 = F11 / J;
  if (m.model == kMatNeoHooke) {
    double vol = 0.5 * lam * (J * J - 1.0);
    return {mu * (F11 - H00) + vol * H00, mu * (F12 - H01) + vol * H01,
            mu * (F21 - H10) + vol * H10, mu * (F22 - H11) + vol * H11};
  }
  double logJ = log(J);
  double vol = lam * logJ;
  if (m.model == kMatLogNeoHooke) {
    return {mu * (F11 - H00) + vol * H00, mu * (F12 - H01) + vol * H01,
            mu * (F21 - H10) + vol * H10, mu * (F22 - H11) + vol * H11};
  }
  double F2 = F11 * F11 + F12 * F12 + F21 * F21 + F22 * F22;
  double I1 = F2 + 1.0;
  double I2 = J * J + F2;
  double jm23 = exp((-2.0 / 3.0) * logJ);
  double jm43 = exp((-4.0 / 3.0) * logJ);
  double hs1 = (-2.0 / 3.0) * I1;
  double hs2 = 2.0 * J * J - (4.0 / 3.0) * I2;
  double G100 = jm23 * (2.0 * F11 + hs1 * H00);
  double G101 = jm23 * (2.0 * F12 + hs1 * H01);
  double G110 = jm23 * (2.0 * F21 + hs1 * H10);
  double G111 = jm23 * (2.0 * F22 + hs1 * H11);
  if (m.model == kMatMooneyRivlin || m.model == kMatSix) {
    double G200 = jm43 * (2.0 * F11 + hs2 * H00);
    double G201 = jm43 * (2.0 * F12 + hs2 * H01);
    double G210 = jm43 * (2.0 * F21 + hs2 * H10);
    double G211 = jm43 * (2.0 * F22 + hs2 * H11);
    if (m.model == kMatSix) {
      double A = jm23 * I1 - 3.0;
      double c2 = -0.5 * mu;
      double c3 = (m.p0 + 2.0 * mu) / 8.0;
      double s = mu + 2.0 * c3 * A;
      return {s * G100 + c2 * G200 + vol * H00, s * G101 + c2 * G201 + vol * H01,
              s * G110 + c2 * G210 + vol * H10, s * G111 + c2 * G211 + vol * H11};
    }
    return {m.p0 * G100 + m.p1 * G200 + vol * H00, m.p0 * G101 + m.p1 * G201 + vol * H01,
            m.p0 * G110 + m.p1 * G210 + vol * H10, m.p0 * G111 + m.p1 * G211 + vol * H11};
  }
  if (m.model == kMatYeoh) {
    double A = jm23 * I1 - 3.0;
    double s = m.p0 + 2.0 * m.p1 * A + 3.0 * m.p2 * A * A;
    return {s * G100 + vol * H00, s * G101 + vol * H01, s * G110 + vol * H10,
            s * G111 + vol * H11};
  }
  if (m.model == kMatGent) {
    double A = jm23 * I1 - 3.0;
    double den = 1.0 - A / m.p0;
    if (den < m.jf) den = m.jf;
    double s = 0.5 * mu / den;
    return {s * G100 + vol * H00, s * G101 + vol * H01, s * G110 + vol * H10,
            s * G111 + vol * H11};
  }
  return {mu * (F11 - H00) + vol * H00, mu * (F12 - H01) + vol * H01,
          mu * (F21 - H10) + vol * H10, mu * (F22 - H11) + vol * H11};
}

// ---------------------------------------------------------------------------
// 3-D first Piola stress, row-major p[3*i+j].
// three_d/vector_nonlinear_elastic_warp3d.py:792-1022 (_piola_mat).
// ---------------------------------------------------------------------------
struct M3 {
  double v[9];
};

CV_DEV double det3(double F11, double F12, double F13, double F21, double F22, double F23,
                   double F31, double F32, double F33) {
  // three_d/vector_nonlinear_elastic_warp3d.py:774-789 (_det3)
  return F11 * (F22 * F33 - F23 * F32) - F12 * (F21 * F33 - F23 * F31) +
         F13 * (F21 * F32 - F22 * F31);
}

CV_DEV M3 piola3(const double* F, const Mat& m) {
  const double F11 = F[0], F12 = F[1], F13 = F[2], F21 = F[3], F22 = F[4], F23 = F[5],
               F31 = F[6], F32 = F[7], F33 = F[8];
  const double lam = m.lam, mu = m.mu;
  M3 P;
  if (m.model == kMatSVK) {
    double C00 = F11 * F11 + F21 * F21 + F31 * F31;
    double C01 = F11 * F12 + F21 * F22 + F31 * F32;
    double C02 = F11 * F13 + F21 * F23 + F31 * F33;
    double C11 = F12 * F12 + F22 * F22 + F32 * F32;
    double C12 = F12 * F13 + F22 * F23 + F32 * F33;
    double C22 = F13 * F13 + F23 * F23 + F33 * F33;
    double E00 = 0.5 * (C00 - 1.0), E01 = 0.5 * C01, E02 = 0.5 * C02;
    double E11 = 0.5 * (C11 - 1.0), E12 = 0.5 * C12, E22 = 0.5 * (C22 - 1.0);
    double trE = E00 + E11 + E22;
    double S00 = lam * trE + 2.0 * mu * E00, S01 = 2.0 * mu * E01, S02 = 2.0 * mu * E02;
    double S11 = lam * trE + 2.0 * mu * E11, S12 = 2.0 * mu * E12;
    double S22 = lam * trE + 2.0 * mu * E22;
    P.v[0] = F11 * S00 + F12 * S01 + F13 * S02;
    P.v[1] = F11 * S01 + F12 * S11 + F13 * S12;
    P.v[2] = F11 * S02 + F12 * S12 + F13 * S22;
    P.v[3] = F21 * S00 + F22 * S01 + F23 * S02;
    P.v[4] = F21 * S01 + F22 * S11 + F23 * S12;
    P.v[5] = F21 * S02 + F22 * S12 + F23 * S22;
    P.v[6] = F31 * S00 + F32 * S01 + F33 * S02;
    P.v[7] = F31 * S01 + F32 * S11 + F33 * S12;
    P.v[8] = F31 * S02 + F32 * S12 + F33 * S22;
    return P;
  }
  double J = clamp_j(det3(F11, F12, F13, F21, F22, F23, F31, F32, F33), m.jf);
  double H[9];
  H[0] = (F22 * F33 - F23 * F32) / J;
  H[1] = (F23 * F31 - F21 * F33) / J;
  H[2] = (F21 * F32 - F22 * F31) / J;
  H[3] = (F13 * F32 - F12 * F33) / J;
  H[4] = (F11 * F33 - F13 * F31) / J;
  H[5] = (F12 * F31 - F11 * F32) / J;
  H[6] = (F12 * F23 - F13 * F22) / J;
  H[7] = (F13 * F21 - F11 * F23) / J;
  H[8] = (F11 * F22 - F12 * F21) / J;
  if (m.model == kMatNeoHooke) {
    double vol = 0.5 * lam * (J * J - 1.0);
#pragma unroll
    for (int k = 0; k < 9; ++k) P.v[k] = mu * (F[k] - H[k]) + vol * H[k];
    return P;
  }
  double logJ = log(J);
  if (m.model == kMatLogNeoHooke) {
    double vol = lam * logJ;
#pragma unroll
    for (int k = 0; k < 9; ++k) P.v[k] = mu * (F[k] - H[k]) + vol * H[k];
    return P;
  }
  double C00 = F11 * F11 + F21 * F21 + F31 * F31;
  double C01 = F11 * F12 + F21 * F22 + F31 * F32;
  double C02 = F11 * F13 + F21 * F23 + F31 * F33;
  double C11 = F12 * F12 + F22 * F22 + F32 * F32;
  double C12 = F12 * F13 + F22 * F23 + F32 * F33;
  double C22 = F13 * F13 + F23 * F23 + F33 * F33;
  double I1 = C00 + C11 + C22;
  double jm23 = exp((-2.0 / 3.0) * logJ);
  const double two3 = 2.0 / 3.0;
  double G1[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) G1[k] = jm23 * (2.0 * F[k] - two3 * I1 * H[k]);
  if (m.model == kMatSix) {  // SPH neo-Hooke, lam carries the bulk modulus
    double vol = 0.5 * lam * (J * J - 1.0);
    double s = 0.5 * mu;
#pragma unroll
    for (int k = 0; k < 9; ++k) P.v[k] = s * G1[k] + vol * H[k];
    return P;
  }
  double trC2 = C00 * C00 + C11 * C11 + C22 * C22 + 2.0 * (C01 * C01 + C02 * C02 + C12 * C12);
  double I2 = 0.5 * (I1 * I1 - trC2);
  double jm43 = exp((-4.0 / 3.0) * logJ);
  double vol = lam * logJ;
  if (m.model == kMatMooneyRivlin) {
    double FC[9];
    FC[0] = F11 * C00 + F12 * C01 + F13 * C02;
    FC[1] = F11 * C01 + F12 * C11 + F13 * C12;
    FC[2] = F11 * C02 + F12 * C12 + F13 * C22;
    FC[3] = F21 * C00 + F22 * C01 + F23 * C02;
    FC[4] = F21 * C01 + F22 * C11 + F23 * C12;
    FC[5] = F21 * C02 + F22 * C12 + F23 * C22;
    FC[6] = F31 * C00 + F32 * C01 + F33 * C02;
    FC[7] = F31 * C01 + F32 * C11 + F33 * C12;
    FC[8] = F31 * C02 + F32 * C12 + F33 * C22;
    const double four3 = 4.0 / 3.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double G2 = jm43 * (2.0 * (I1 * F[k] - FC[k]) - four3 * I2 * H[k]);
      P.v[k] = m.p0 * G1[k] + m.p1 * G2 + vol * H[k];
    }
    return P;
  }
  if (m.model == kMatYeoh) {
    double A = jm23 * I1 - 3.0;
    double s = m.p0 + 2.0 * m.p1 * A + 3.0 * m.p2 * A * A;
#pragma unroll
    for (int k = 0; k < 9; ++k) P.v[k] = s * G1[k] + vol * H[k];
    return P;
  }
  if (m.model == kMatGent) {
    double A = jm23 * I1 - 3.0;
    double den = 1.0 - A / m.p0;
    if (den < m.jf) den = m.jf;
    double s = 0.5 * mu / den;
#pragma unroll
    for (int k = 0; k < 9; ++k) P.v[k] = s * G1[k] + vol * H[k];
    return P;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) P.v[k] = 0.0;
  return P;
}

// Row r (entries 3r..3r+2) of piola3(F, m), with the same operations for the
// neo-Hooke law (cofactor / J per entry); other laws evaluate the full tensor.
CV_DEV void piola3_row(const double* F, const Mat& m, int r, double* out) {
  if (m.model != kMatNeoHooke) {
    const M3 P = piola3(F, m);
    out[0] = P.v[3 * r];
    out[1] = P.v[3 * r + 1];
    out[2] = P.v[3 * r + 2];
    return;
  }
  const double F11 = F[0], F12 = F[1], F13 = F[2], F21 = F[3], F22 = F[4], F23 = F[5],
               F31 = F[6], F32 = F[7], F33 = F[8];
  const double J = clamp_j(det3(F11, F12, F13, F21, F22, F23, F31, F32, F33), m.jf);
  double c0, c1, c2;
  if (r == 0) {
    c0 = F22 * F33 - F23 * F32;
    c1 = F23 * F31 - F21 * F33;
    c2 = F21 * F32 - F22 * F31;
  } else if (r == 1) {
    c0 = F13 * F32 - F12 * F33;
    c1 = F11 * F33 - F13 * F31;
    c2 = F12 * F31 - F11 * F32;
  } else {
    c0 = F12 * F23 - F13 * F22;
    c1 = F13 * F21 - F11 * F23;
    c2 = F11 * F22 - F12 * F21;
  }
  const double h0 = c0 / J, h1 = c1 / J, h2 = c2 / J;
  const double vol = 0.5 * m.lam * (J * J - 1.0);
  out[0] = m.mu * (F[3 * r] - h0) + vol * h0;
  out[1] = m.mu * (F[3 * r + 1] - h1) + vol * h1;
  out[2] = m.mu * (F[3 * r + 2] - h2) + vol * h2;
}

// ---------------------------------------------------------------------------
// Lattice helpers.
// ---------------------------------------------------------------------------
// D2Q4 directions E, N, W, S (two_d/vector_nonlinear_elastic_warp.py:68-71).
CV_DEV int cx2(int q) { return q == 0 ? 1 : (q == 2 ? -1 : 0); }
CV_DEV int cy2(int q) { return q == 1 ? 1 : (q == 3 ? -1 : 0); }
// D3Q6 directions +x +y +z -x -y -z (three_d/curved_boundary_warp3d.py:944-974).
CV_DEV int dx3(int q) { return q == 0 ? 1 : (q == 3 ? -1 : 0); }
CV_DEV int dy3(int q) { return q == 1 ? 1 : (q == 4 ? -1 : 0); }
CV_DEV int dz3(int q) { return q == 2 ? 1 : (q == 5 ? -1 : 0); }
CV_DEV int opp3(int q) { return q < 3 ? q + 3 : q - 3; }

// 2-D flux components for state U=(vx,vy,F11,F12,F21,F22) given P.
// two_d/vector_nonlinear_elastic_warp.py:1078-1137 (_flux_x_comp/_flux_y_comp).
CV_DEV double flux2x(int a, const double* U, const P2& P) {
  switch (a) {
    case 0: return -P.a;
    case 1: return -P.c;
    case 2: return -U[0];
    case 4: return -U[1];
    default: return 0.0;
  }
}
CV_DEV double flux2y(int a, const double* U, const P2& P) {
  switch (a) {
    case 0: return -P.b;
    case 1: return -P.d;
    case 3: return -U[0];
    case 5: return -U[1];
    default: return 0.0;
  }
}

// 2-D equilibrium, two_d/vector_nonlinear_elastic_warp.py:1140-1168:
// feq_qa = 0.25*(U_a + (2/c)*(cx*phix_a + cy*phiy_a)).
CV_DEV double feq2(int q, int a, const double* U, const P2& P, double two_over_c) {
  double cx = (double)cx2(q), cy = (double)cy2(q);
  return 0.25 * (U[a] + two_over_c * (cx * flux2x(a, U, P) + cy * flux2y(a, U, P)));
}

// 3-D flux component along `axis`, three_d/vector_nonlinear_elastic_warp3d.py:1066-1133.
CV_DEV double flux3(int axis, int a, const double* U, const M3& P) {
  if (a < 3) return -P.v[3 * a + axis];
  int r = a - 3;
  if (r % 3 == axis) return -U[r / 3];
  return 0.0;
}

// 3-D equilibrium, three_d/vector_nonlinear_elastic_warp3d.py:1136-1236.
CV_DEV double feq3(int q, int a, const double* U, const M3& P, double three_over_c,
                   double sixth) {
  double sx = (double)dx3(q), sy = (double)dy3(q), sz = (double)dz3(q);
  return sixth * (U[a] + three_over_c * (sx * flux3(0, a, U, P) + sy * flux3(1, a, U, P) +
                                         sz * flux3(2, a, U, P)));
}

// ---------------------------------------------------------------------------
// Boundary value functions.
// ---------------------------------------------------------------------------
// two_d/vector_nonlinear_elastic_warp.py:1171-1247 (_ricker_wavelet,
// _boundary_value_comp) and two_d/curved_boundary_warp.py:935-984
// (_curved_boundary_value_comp).  Mode 105 (linear ramp then hold of a
// radial traction, params amp, ramp_time) is an addition of this project.
CV_DEV double smoothstep5(double e) {
  double z = e;
  if (z < 0.0) z = 0.0;
  if (z > 1.0) z = 1.0;
  return z * z * z * (10.0 - 15.0 * z + 6.0 * z * z);
}

CV_DEV double value2(int comp, int mode, const double* p, double x, double y, double nx,
                     double ny, double t) {
  switch (mode) {
    case 101: return comp == 0 ? p[0] * nx + p[1] * ny : p[2] * nx + p[3] * ny;
    case 102: return comp == 0 ? p[0] * nx : p[0] * ny;
    case 103: {
      double act = p[1], den = p[2], s2 = 1.0;
      if (act > 0.0 && t < act) {
        if (den <= 0.0) den = 2.0 * act;
        double s = sin(kPi * t / den);
        s2 = s * s;
      }
      return comp == 0 ? p[0] * s2 * nx : p[0] * s2 * ny;
    }
    case 104: {
      double pt = p[1], s2 = 0.0;
      if (pt > 0.0 && t < pt) {
        double s = sin(kPi * t / pt);
        s2 = s * s;
      }
      return comp == 0 ? p[0] * s2 * nx : p[0] * s2 * ny;
    }
    case 105: {
      double rt = p[1], s = 1.0;
      if (rt > 0.0 && t < rt) s = t / rt;
      return comp == 0 ? p[0] * s * nx : p[0] * s * ny;
    }
    case 0: return 0.0;
    case 1: return comp == 0 ? p[0] : p[1];
    case 2: {
      double rt = p[2], s2 = 1.0;
      if (rt > 0.0 && t < rt) {
        double s = sin(kPi * t / rt);
        s2 = s * s;
      }
      return comp == 0 ? p[0] * s2 : p[1] * s2;
    }
    case 5: {
      double act = p[2], den = p[3], s2 = 1.0;
      if (act > 0.0 && t < act) {
        if (den <= 0.0) den = 2.0 * act;
        double s = sin(kPi * t / den);
        s2 = s * s;
      }
      return comp == 0 ? p[0] * s2 : p[1] * s2;
    }
    case 3:
      if (comp == 0 && t < p[1]) return p[0] * sin(kPi * t / p[1]);
      return 0.0;
    case 4: {
      if (comp != 1 || t > p[3]) return 0.0;
      double z = (t - p[2]) / p[1];
      double pref = 2.0 * p[0] / (sqrt(3.0 * p[1]) * sqrt(sqrt(kPi)));
      double val = pref * (1.0 - z * z) * exp(-0.5 * z * z);
      if (p[6] > 0.0) {
        double layer = p[6] * p[5];
        if (layer < 1.0e-30) layer = 1.0e-30;
        double w = smoothstep5(y / layer) * smoothstep5((p[4] - y) / layer);
        if (p[7] > 1.0e-14) w = w / p[7];
        val = val * w;
      }
      return val;
    }
    case 6:
      if (p[6] > 0.0 && t > p[6]) return 0.0;
      return comp == 0 ? p[0] * x + p[1] * y + p[2] : p[3] * x + p[4] * y + p[5];
    default: return 0.0;
  }
}

// 3-D curved boundary values, three_d/curved_boundary_warp3d.py:995-1133.
// Mode 208 (linear ramp then hold of a normal traction, params amp, ramp_time)
// is an addition of this project.
CV_DEV M3 piola3_nh(const double* F, double lam, double mu, double jf) {
  Mat m{kMatNeoHooke, lam, mu, 0.0, 0.0, 0.0, jf};
  return piola3(F, m);
}

CV_DEV double value3(int comp, int mode, const double* p, double x, double y, double z,
                     double nx, double ny, double nz, double t, double jf) {
  switch (mode) {
    case 0: return 0.0;
    case 1: return p[comp];
    case 200: {
      double act = p[3], s2 = 1.0;
      if (act > 0.0 && t < act) s2 = sin(kPi * t / act) * sin(kPi * t / act);
      return p[comp] * s2;
    }
    case 4: {
      double act = p[12];
      if (act > 0.0 && t > act) return 0.0;
      if (comp == 0) return p[0] * x + p[1] * y + p[2] * z + p[9];
      if (comp == 1) return p[3] * x + p[4] * y + p[5] * z + p[10];
      return p[6] * x + p[7] * y + p[8] * z + p[11];
    }
    case 204: {
      double act = p[3], den = p[4];
      if (den <= 0.0) den = 2.0 * act;
      double s2 = 1.0;
      if (act > 0.0 && t < act) s2 = sin(kPi * t / den) * sin(kPi * t / den);
      return p[comp] * s2;
    }
    case 201: return p[3 * comp + 0] * nx + p[3 * comp + 1] * ny + p[3 * comp + 2] * nz;
    case 205: {
      double tt = t, act = p[11];
      if (act > 0.0 && tt > act) tt = act;
      double F[9] = {1.0 + tt * p[0], tt * p[1],       tt * p[2],
                     tt * p[3],       1.0 + tt * p[4], tt * p[5],
                     tt * p[6],       tt * p[7],       1.0 + tt * p[8]};
      M3 P = piola3_nh(F, p[9], p[10], jf);
      return P.v[3 * comp] * nx + P.v[3 * comp + 1] * ny + P.v[3 * comp + 2] * nz;
    }
    case 202: return comp == 0 ? p[0] * nx : (comp == 1 ? p[0] * ny : p[0] * nz);
    case 203: {
      double amp = p[0], act = p[1], den = p[2];
      if (den <= 0.0) den = 2.0 * act;
      double s2 = 1.0;
      if (act > 0.0 && t < act) s2 = sin(kPi * t / den) * sin(kPi * t / den);
      return comp == 0 ? amp * s2 * nx : (comp == 1 ? amp * s2 * ny : amp * s2 * nz);
    }
    case 208: {
      double amp = p[0], rt = p[1], s = 1.0;
      if (rt > 0.0 && t < rt) s = t / rt;
      return comp == 0 ? amp * s * nx : (comp == 1 ? amp * s * ny : amp * s * nz);
    }
    case 206: {
      double act = p[4], den = p[5];
      if (den <= 0.0) den = 2.0 * act;
      double s2 = 1.0;
      if (act > 0.0 && t < act) s2 = sin(kPi * t / den) * sin(kPi * t / den);
      double ddx = x - p[0], ddy = y - p[1];
      if (comp == 0) return -s2 * p[3] * ddy;
      if (comp == 1) return s2 * p[3] * ddx;
      return s2 * p[2];
    }
    case 207: {
      double act = p[4];
      if (act <= 0.0 || t >= act) return 0.0;
      double phase = kPi * t / act;
      double s = 0.5 * (1.0 - cos(phase));
      double sdot = 0.5 * kPi / act * sin(phase);
      double th = p[3] * s, thd = p[3] * sdot;
      double ddx = x - p[0], ddy = y - p[1];
      if (comp == 0) return thd * (-sin(th) * ddx - cos(th) * ddy);
      if (comp == 1) return thd * (cos(th) * ddx - sin(th) * ddy);
      return p[2] * sdot;
    }
    default: return 0.0;
  }
}

// Prescribed boundary displacement used by the 3-D cut-point anchors,
// three_d/curved_boundary_warp3d.py:2333-2399.
CV_DEV double sine2_integral(double time, double act, double den) {
  if (act <= 0.0) return time;
  if (den <= 0.0) den = act;
  double t = time > 0.0 ? time : 0.0;
  if (t < act) return 0.5 * t - den * sin(2.0 * kPi * t / den) / (4.0 * kPi);
  double pre = 0.5 * act - den * sin(2.0 * kPi * act / den) / (4.0 * kPi);
  return pre + (t - act);
}

CV_DEV double disp3(int mode, const double* p, int comp, double x, double y, double z,
                    double time) {
  switch (mode) {
    case 0: return 0.0;
    case 1: return time * p[comp];
    case 200: return p[comp] * sine2_integral(time, p[3], p[3]);
    case 204: {
      double act = p[3], den = p[4];
      if (den <= 0.0) den = 2.0 * act;
      return p[comp] * sine2_integral(time, act, den);
    }
    case 4: {
      double at = time, act = p[12];
      if (act > 0.0 && at > act) at = act;
      double out;
      if (comp == 0) out = p[0] * x + p[1] * y + p[2] * z + p[9];
      else if (comp == 1) out = p[3] * x + p[4] * y + p[5] * z + p[10];
      else out = p[6] * x + p[7] * y + p[8] * z + p[11];
      return at * out;
    }
    case 207: {
      double act = p[4], s = 1.0;
      if (act > 0.0 && time < act) s = 0.5 * (1.0 - cos(kPi * time / act));
      double th = p[3] * s, ddx = x - p[0], ddy = y - p[1];
      double c = cos(th), ss = sin(th);
      if (comp == 0) return (c - 1.0) * ddx - ss * ddy;
      if (comp == 1) return ss * ddx + (c - 1.0) * ddy;
      return p[2] * s;
    }
    default: return 0.0;
  }
}

// Source term B_a(U), two_d/vector_nonlinear_elastic_warp.py:1250-1280 and
// three_d/vector_nonlinear_elastic_warp3d.py:1371-1389.
CV_DEV double source_comp(int a, int mode, const double* sp, const double* v) {
  if (mode == kSrcConstant) return sp[a];
  if (mode == kSrcDamping) {
    if (a == 0) return -sp[0] * v[0];
    if (a == 1) return -sp[0] * v[1];
  }
  return 0.0;
}
CV_DEV double source_comp3(int a, int mode, const double* sp, const double* v) {
  if (mode == kSrcConstant) return sp[a];
  if (mode == kSrcDamping && a < 3) return -sp[0] * v[a];
  return 0.0;
}

// ---------------------------------------------------------------------------
// 2-D normal-image solve P(F_b) n = T with the tangential image fixed.
// two_d/curved_boundary_warp.py:987-1192.
// ---------------------------------------------------------------------------
CV_DEV void residual2(double hn0, double hn1, double gt0, double gt1, double nx, double ny,
                      double tx, double ty, const Mat& m, double& r0, double& r1) {
  double t1 = -ny, t2 = nx;
  double F11 = hn0 * nx + gt0 * t1;
  double F12 = hn0 * ny + gt0 * t2;
  double F21 = hn1 * nx + gt1 * t1;
  double F22 = hn1 * ny + gt1 * t2;
  P2 P = piola2(F11, F12, F21, F22, m);
  r0 = P.a * nx + P.b * ny - tx;
  r1 = P.c * nx + P.d * ny - ty;
}

CV_DEV void solve_normal_image2(const double* Fg, double nx, double ny, double tx, double ty,
                                const Mat& m, int solver, double* Fout) {
  const double lam = m.lam, mu = m.mu, jf = m.jf;
  if (solver == kSolverEnergy && m.model == kMatNeoHooke) {
    double a0 = Fg[3] * nx - Fg[2] * ny;
    double a1 = -Fg[1] * nx + Fg[0] * ny;
    double a2 = a0 * a0 + a1 * a1;
    if (a2 > 1.0e-28) {
      double area = sqrt(a2);
      double e0 = a0 / area, e1 = a1 / area;
      double tau = tx * e0 + ty * e1;
      double aa = mu + 0.5 * lam * a2;
      double bb = mu + 0.5 * lam;
      double disc = sqrt(tau * tau + 4.0 * aa * bb);
      double s = (tau + disc) / (2.0 * aa);
      if (tau < 0.0) s = 2.0 * bb / (disc - tau);
      if (area * s > jf) {
        double h0 = (tx - tau * e0) / mu + s * e0;
        double h1 = (ty - tau * e1) / mu + s * e1;
        double d0 = h0 - (Fg[0] * nx + Fg[1] * ny);
        double d1 = h1 - (Fg[2] * nx + Fg[3] * ny);
        Fout[0] = Fg[0] + d0 * nx;
        Fout[1] = Fg[1] + d0 * ny;
        Fout[2] = Fg[2] + d1 * nx;
        Fout[3] = Fg[3] + d1 * ny;
        return;
      }
    }
  }
  const double tanx = -ny, tany = nx;
  double hn0 = Fg[0] * nx + Fg[1] * ny;
  double hn1 = Fg[2] * nx + Fg[3] * ny;
  const double gt0 = Fg[0] * tanx + Fg[1] * tany;
  const double gt1 = Fg[2] * tanx + Fg[3] * tany;
  const double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r0, r1;
    residual2(hn0, hn1, gt0, gt1, nx, ny, tx, ty, m, r0, r1);
    double rn = sqrt(r0 * r0 + r1 * r1);
    if (rn < 1.0e-11) break;
    double a, b, c, d;
    if (solver != kSolverFD && m.model == kMatNeoHooke) {
      // two_d/curved_boundary_warp.py:1016-1043 (_neo_hooke_acoustic_normal_2d)
      double F11 = hn0 * nx + gt0 * tanx;
      double F12 = hn0 * ny + gt0 * tany;
      double F21 = hn1 * nx + gt1 * tanx;
      double F22 = hn1 * ny + gt1 * tany;
      double J = clamp_j(F11 * F22 - F12 * F21, jf);
      double H00 = F22 / J, H01 = -F21 / J, H10 = -F12 / J, H11 = F11 / J;
      double beta = 0.5 * lam * (J * J - 1.0) - mu;
      double coeff = lam * J * J - beta;
      double n2 = nx * nx + ny * ny;
      double v0 = H00 * nx + H01 * ny;
      double v1 = H10 * nx + H11 * ny;
      a = mu * n2 + coeff * v0 * v0;
      b = coeff * v0 * v1;
      c = coeff * v1 * v0;
      d = mu * n2 + coeff * v1 * v1;
    } else {
      double p00, p01, p10, p11;
      residual2(hn0 + eps, hn1, gt0, gt1, nx, ny, tx, ty, m, p00, p01);
      residual2(hn0, hn1 + eps, gt0, gt1, nx, ny, tx, ty, m, p10, p11);
      a = (p00 - r0) / eps;
      c = (p01 - r1) / eps;
      b = (p10 - r0) / eps;
      d = (p11 - r1) / eps;
    }
    double det = a * d - b * c;
    if (fabs(det) < 1.0e-14) break;
    double d0 = (-r0 * d + b * r1) / det;
    double d1 = (c * r0 - a * r1) / det;
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double c0 = hn0 + step * d0, c1 = hn1 + step * d1;
      double F11 = c0 * nx + gt0 * tanx;
      double F12 = c0 * ny + gt0 * tany;
      double F21 = c1 * nx + gt1 * tanx;
      double F22 = c1 * ny + gt1 * tany;
      double J = F11 * F22 - F12 * F21;
      if (J > jf) {
        hn0 = c0;
        hn1 = c1;
        break;
      }
      step = 0.5 * step;
    }
  }
  Fout[0] = hn0 * nx + gt0 * tanx;
  Fout[1] = hn0 * ny + gt0 * tany;
  Fout[2] = hn1 * nx + gt1 * tanx;
  Fout[3] = hn1 * ny + gt1 * tany;
}

// Centred finite-difference directional derivative of the 2-D fluxes,
// two_d/curved_boundary_warp.py:1224-1365 (_jvp_eps6, _flux_x/_flux_y_jvp_comp).
// Computes all six components of A_x W and A_y W from one pair of Piola
// evaluations (the reference evaluates the same pair once per component).
CV_DEV double jvp_eps6(const double* w) {
  double s = fabs(w[0]);
  for (int k = 1; k < 6; ++k)
    if (fabs(w[k]) > s) s = fabs(w[k]);
  double eps = 1.0e-6;
  if (s > 1.0) eps = eps / s;
  return eps;
}

CV_DEV void flux2_jvp(const double* U, const double* W, const Mat& m, double* AxW, double* AyW) {
  double eps = jvp_eps6(W);
  double Up[6], Um[6];
  for (int k = 0; k < 6; ++k) {
    Up[k] = U[k] + eps * W[k];
    Um[k] = U[k] - eps * W[k];
  }
  P2 Pp = piola2(Up[2], Up[3], Up[4], Up[5], m);
  P2 Pm = piola2(Um[2], Um[3], Um[4], Um[5], m);
  double den = 2.0 * eps;
  for (int a = 0; a < 6; ++a) {
    AxW[a] = (flux2x(a, Up, Pp) - flux2x(a, Um, Pm)) / den;
    AyW[a] = (flux2y(a, Up, Pp) - flux2y(a, Um, Pm)) / den;
  }
}

// ---------------------------------------------------------------------------
// 3-D traction solve, three_d/curved_boundary_warp3d.py:977-1515.
// ---------------------------------------------------------------------------
CV_DEV void normalize3(double* v) {
  double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (r < 1.0e-30) r = 1.0e-30;
  v[0] = v[0] / r;
  v[1] = v[1] / r;
  v[2] = v[2] / r;
}
CV_DEV void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

struct Frame3 {
  double n[3], t1[3], t2[3];
};

// Orthonormal frame of the cut-point normal, three_d/curved_boundary_warp3d.py:1358-1364.
CV_DEV Frame3 frame3(double nx, double ny, double nz) {
  Frame3 f;
  f.n[0] = nx;
  f.n[1] = ny;
  f.n[2] = nz;
  normalize3(f.n);
  double ref[3] = {1.0, 0.0, 0.0};
  if (fabs(f.n[0]) >= 0.75) {
    ref[0] = 0.0;
    ref[1] = 1.0;
  }
  cross3(f.n, ref, f.t1);
  normalize3(f.t1);
  cross3(f.n, f.t1, f.t2);
  return f;
}

CV_DEV void make_F_h(const double* h, const Frame3& fr, const double* g1, const double* g2,
                     double* F) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[3 * i + j] = h[i] * fr.n[j] + g1[i] * fr.t1[j] + g2[i] * fr.t2[j];
}

CV_DEV void residual3(const double* h, const Frame3& fr, const double* g1, const double* g2,
                      const double* T, const Mat& m, double* r) {
  double F[9];
  make_F_h(h, fr, g1, g2, F);
  M3 P = piola3(F, m);
  for (int i = 0; i < 3; ++i)
    r[i] = P.v[3 * i] * fr.n[0] + P.v[3 * i + 1] * fr.n[1] + P.v[3 * i + 2] * fr.n[2] - T[i];
}

CV_DEV double det3v(const double* F) {
  return det3(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8]);
}

// Closed-form minimiser for quadratic-volumetric neo-Hooke with all three
// components Neumann, three_d/curved_boundary_warp3d.py:1249-1329.
// Returns false for the degenerate branch (caller falls back to Newton).
CV_DEV bool energy_Fb3(const double* F, const double* n, const double* T, double lam, double mu,
                       double jf, double* Fb) {
  double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                   F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                   F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  double a[3], ho[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = cof[3 * i] * n[0] + cof[3 * i + 1] * n[1] + cof[3 * i + 2] * n[2];
    ho[i] = F[3 * i] * n[0] + F[3 * i + 1] * n[1] + F[3 * i + 2] * n[2];
  }
  double a2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  if (!(a2 > 1.0e-28)) return false;
  double area = sqrt(a2);
  double e[3] = {a[0] / area, a[1] / area, a[2] / area};
  double tau = T[0] * e[0] + T[1] * e[1] + T[2] * e[2];
  double aa = mu + 0.5 * lam * a2;
  double bb = mu + 0.5 * lam;
  double disc = sqrt(tau * tau + 4.0 * aa * bb);
  double s = (tau + disc) / (2.0 * aa);
  if (tau < 0.0) s = 2.0 * bb / (disc - tau);
  if (!(area * s > jf)) return false;
  for (int i = 0; i < 3; ++i) {
    double h = (T[i] - tau * e[i]) / mu + s * e[i];
    double dh = h - ho[i];
    for (int j = 0; j < 3; ++j) Fb[3 * i + j] = F[3 * i + j] + dh * n[j];
  }
  return true;
}

CV_DEV void solve_Fb3(const double* Fg, double nx, double ny, double nz, const double* T,
                      const Mat& m, int solver, double* Fout) {
  Frame3 fr = frame3(nx, ny, nz);
  if (solver == kSolverEnergy && m.model == kMatNeoHooke) {
    double Fb[9];
    if (energy_Fb3(Fg, fr.n, T, m.lam, m.mu, m.jf, Fb) && det3v(Fb) > m.jf) {
      for (int k = 0; k < 9; ++k) Fout[k] = Fb[k];
      return;
    }
  }
  double h[3], g1[3], g2[3];
  for (int i = 0; i < 3; ++i) {
    h[i] = Fg[3 * i] * fr.n[0] + Fg[3 * i + 1] * fr.n[1] + Fg[3 * i + 2] * fr.n[2];
    g1[i] = Fg[3 * i] * fr.t1[0] + Fg[3 * i + 1] * fr.t1[1] + Fg[3 * i + 2] * fr.t1[2];
    g2[i] = Fg[3 * i] * fr.t2[0] + Fg[3 * i + 1] * fr.t2[1] + Fg[3 * i + 2] * fr.t2[2];
  }
  const double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r[3];
    residual3(h, fr, g1, g2, T, m, r);
    double rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (rn < 1.0e-10) break;
    double A[9];
    if (solver != kSolverFD && m.model == kMatNeoHooke) {
      // three_d/curved_boundary_warp3d.py:1205-1246 (_neo_hooke_acoustic_normal_3d)
      double F[9];
      make_F_h(h, fr, g1, g2, F);
      double J = det3v(F);
      if (J < m.jf) J = m.jf;
      double H[9];
      H[0] = (F[4] * F[8] - F[5] * F[7]) / J;
      H[1] = (F[5] * F[6] - F[3] * F[8]) / J;
      H[2] = (F[3] * F[7] - F[4] * F[6]) / J;
      H[3] = (F[2] * F[7] - F[1] * F[8]) / J;
      H[4] = (F[0] * F[8] - F[2] * F[6]) / J;
      H[5] = (F[1] * F[6] - F[0] * F[7]) / J;
      H[6] = (F[1] * F[5] - F[2] * F[4]) / J;
      H[7] = (F[2] * F[3] - F[0] * F[5]) / J;
      H[8] = (F[0] * F[4] - F[1] * F[3]) / J;
      double beta = 0.5 * m.lam * (J * J - 1.0) - m.mu;
      double coeff = m.lam * J * J - beta;
      double n2 = fr.n[0] * fr.n[0] + fr.n[1] * fr.n[1] + fr.n[2] * fr.n[2];
      double v[3];
      for (int i = 0; i < 3; ++i)
        v[i] = H[3 * i] * fr.n[0] + H[3 * i + 1] * fr.n[1] + H[3 * i + 2] * fr.n[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          A[3 * i + j] = (i == j) ? m.mu * n2 + coeff * v[i] * v[j] : coeff * v[i] * v[j];
    } else {
      double rp[3][3];
      for (int k = 0; k < 3; ++k) {
        double hp[3] = {h[0], h[1], h[2]};
        hp[k] = hp[k] + eps;
        residual3(hp, fr, g1, g2, T, m, rp[k]);
      }
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) A[3 * i + k] = (rp[k][i] - r[i]) / eps;
    }
    const double a = A[0], b = A[1], c = A[2], d = A[3], e = A[4], f = A[5], g = A[6],
                 hh = A[7], ii = A[8];
    double det = a * (e * ii - f * hh) - b * (d * ii - f * g) + c * (d * hh - e * g);
    if (fabs(det) < 1.0e-14) break;
    double i00 = (e * ii - f * hh) / det, i01 = (c * hh - b * ii) / det,
           i02 = (b * f - c * e) / det;
    double i10 = (f * g - d * ii) / det, i11 = (a * ii - c * g) / det,
           i12 = (c * d - a * f) / det;
    double i20 = (d * hh - e * g) / det, i21 = (b * g - a * hh) / det,
           i22 = (a * e - b * d) / det;
    double dl[3] = {-(i00 * r[0] + i01 * r[1] + i02 * r[2]),
                    -(i10 * r[0] + i11 * r[1] + i12 * r[2]),
                    -(i20 * r[0] + i21 * r[1] + i22 * r[2])};
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double cand[3] = {h[0] + step * dl[0], h[1] + step * dl[1], h[2] + step * dl[2]};
      double F[9];
      make_F_h(cand, fr, g1, g2, F);
      if (det3v(F) > m.jf) {
        h[0] = cand[0];
        h[1] = cand[1];
        h[2] = cand[2];
        break;
      }
      step = 0.5 * step;
    }
  }
  make_F_h(h, fr, g1, g2, Fout);
}

// Closed-form minimiser over the Neumann rows only, quadratic-volumetric
// neo-Hooke, mixed rows (three_d/curved_boundary_warp3d.py:1249-1329, branch
// with a Dirichlet row): J = d + a_N.h_N with d from the fixed rows.
CV_DEV bool energy_Fb3_mixed(const double* F, const double* n, const double* T, const int* ck,
                             double lam, double mu, double jf, double* Fb) {
  double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                   F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                   F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  double a[3], ho[3], an[3] = {0.0, 0.0, 0.0}, tn[3] = {0.0, 0.0, 0.0}, fixed[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = cof[3 * i] * n[0] + cof[3 * i + 1] * n[1] + cof[3 * i + 2] * n[2];
    ho[i] = F[3 * i] * n[0] + F[3 * i + 1] * n[1] + F[3 * i + 2] * n[2];
    fixed[i] = ho[i];
    if (ck[i] == kNeumann) {
      an[i] = a[i];
      tn[i] = T[i];
      fixed[i] = 0.0;
    }
  }
  const double a2 = an[0] * an[0] + an[1] * an[1] + an[2] * an[2];
  const double d = a[0] * fixed[0] + a[1] * fixed[1] + a[2] * fixed[2];
  double h[3];
  if (a2 > 1.0e-28) {
    const double aa = mu + 0.5 * lam * a2;
    const double bb = (mu + 0.5 * lam) * a2;
    const double cc = mu * d + (an[0] * tn[0] + an[1] * tn[1] + an[2] * tn[2]);
    const double disc = sqrt(cc * cc + 4.0 * aa * bb);
    double J = (cc + disc) / (2.0 * aa);
    if (cc < 0.0) J = 2.0 * bb / (disc - cc);
    if (!(J > jf)) return false;
    const double area = sqrt(a2);
    const double e[3] = {an[0] / area, an[1] / area, an[2] / area};
    const double te = tn[0] * e[0] + tn[1] * e[1] + tn[2] * e[2];
    for (int i = 0; i < 3; ++i) h[i] = fixed[i] + (tn[i] - te * e[i]) / mu + ((J - d) / area) * e[i];
  } else if (a2 == 0.0 && d > jf) {
    for (int i = 0; i < 3; ++i) h[i] = fixed[i] + tn[i] / mu;
  } else {
    return false;
  }
  for (int i = 0; i < 3; ++i) {
    const double dh = h[i] - ho[i];
    for (int j = 0; j < 3; ++j) Fb[3 * i + j] = F[3 * i + j] + dh * n[j];
  }
  return true;
}

// Normal solve of the Neumann rows only, three_d/curved_boundary_warp3d.py
// :1518-1737 (_solve_Fb_componentwise_normal): a Dirichlet row keeps its
// extrapolated normal derivative (its residual and Jacobian row are replaced
// by the identity), so its traction is not prescribed but retained in
// P(F_b) n as the boundary reaction.
CV_DEV void solve_Fb3_mixed(const double* Fg, double nx, double ny, double nz, const double* T,
                            const int* ck, const Mat& m, int solver, double* Fout) {
  Frame3 fr = frame3(nx, ny, nz);
  if (solver == kSolverEnergy && m.model == kMatNeoHooke) {
    double Fb[9];
    if (energy_Fb3_mixed(Fg, fr.n, T, ck, m.lam, m.mu, m.jf, Fb) && det3v(Fb) > m.jf) {
      for (int k = 0; k < 9; ++k) Fout[k] = Fb[k];
      return;
    }
  }
  double h[3], g1[3], g2[3];
  for (int i = 0; i < 3; ++i) {
    h[i] = Fg[3 * i] * fr.n[0] + Fg[3 * i + 1] * fr.n[1] + Fg[3 * i + 2] * fr.n[2];
    g1[i] = Fg[3 * i] * fr.t1[0] + Fg[3 * i + 1] * fr.t1[1] + Fg[3 * i + 2] * fr.t1[2];
    g2[i] = Fg[3 * i] * fr.t2[0] + Fg[3 * i + 1] * fr.t2[1] + Fg[3 * i + 2] * fr.t2[2];
  }
  const double eps = 1.0e-6;
  for (int it = 0; it < 16; ++it) {
    double r[3];
    residual3(h, fr, g1, g2, T, m, r);
    double rm[3];
    for (int i = 0; i < 3; ++i) rm[i] = ck[i] == kNeumann ? r[i] : 0.0;
    const double rn = sqrt(rm[0] * rm[0] + rm[1] * rm[1] + rm[2] * rm[2]);
    if (rn < 1.0e-10) break;
    double A[9];
    if (solver != kSolverFD && m.model == kMatNeoHooke) {
      double F[9];
      make_F_h(h, fr, g1, g2, F);
      double J = det3v(F);
      if (J < m.jf) J = m.jf;
      double H[9];
      H[0] = (F[4] * F[8] - F[5] * F[7]) / J;
      H[1] = (F[5] * F[6] - F[3] * F[8]) / J;
      H[2] = (F[3] * F[7] - F[4] * F[6]) / J;
      H[3] = (F[2] * F[7] - F[1] * F[8]) / J;
      H[4] = (F[0] * F[8] - F[2] * F[6]) / J;
      H[5] = (F[1] * F[6] - F[0] * F[7]) / J;
      H[6] = (F[1] * F[5] - F[2] * F[4]) / J;
      H[7] = (F[2] * F[3] - F[0] * F[5]) / J;
      H[8] = (F[0] * F[4] - F[1] * F[3]) / J;
      const double beta = 0.5 * m.lam * (J * J - 1.0) - m.mu;
      const double coeff = m.lam * J * J - beta;
      const double n2 = fr.n[0] * fr.n[0] + fr.n[1] * fr.n[1] + fr.n[2] * fr.n[2];
      double v[3];
      for (int i = 0; i < 3; ++i)
        v[i] = H[3 * i] * fr.n[0] + H[3 * i + 1] * fr.n[1] + H[3 * i + 2] * fr.n[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          A[3 * i + j] = (i == j) ? m.mu * n2 + coeff * v[i] * v[j] : coeff * v[i] * v[j];
    } else {
      double rp[3][3];
      for (int k = 0; k < 3; ++k) {
        double hp[3] = {h[0], h[1], h[2]};
        hp[k] = hp[k] + eps;
        residual3(hp, fr, g1, g2, T, m, rp[k]);
      }
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) A[3 * i + k] = (rp[k][i] - r[i]) / eps;
    }
    for (int i = 0; i < 3; ++i)
      if (ck[i] != kNeumann)
        for (int k = 0; k < 3; ++k) A[3 * i + k] = i == k ? 1.0 : 0.0;
    const double a = A[0], b = A[1], c = A[2], d = A[3], e = A[4], f = A[5], g = A[6],
                 hh = A[7], ii = A[8];
    const double det = a * (e * ii - f * hh) - b * (d * ii - f * g) + c * (d * hh - e * g);
    if (fabs(det) < 1.0e-14) break;
    const double i00 = (e * ii - f * hh) / det, i01 = (c * hh - b * ii) / det,
                 i02 = (b * f - c * e) / det;
    const double i10 = (f * g - d * ii) / det, i11 = (a * ii - c * g) / det,
                 i12 = (c * d - a * f) / det;
    const double i20 = (d * hh - e * g) / det, i21 = (b * g - a * hh) / det,
                 i22 = (a * e - b * d) / det;
    const double dl[3] = {-(i00 * rm[0] + i01 * rm[1] + i02 * rm[2]),
                          -(i10 * rm[0] + i11 * rm[1] + i12 * rm[2]),
                          -(i20 * rm[0] + i21 * rm[1] + i22 * rm[2])};
    double step = 1.0;
    for (int ls = 0; ls < 12; ++ls) {
      double cand[3];
      for (int i = 0; i < 3; ++i) cand[i] = ck[i] == kNeumann ? h[i] + step * dl[i] : h[i];
      double F[9];
      make_F_h(cand, fr, g1, g2, F);
      if (det3v(F) > m.jf) {
        h[0] = cand[0];
        h[1] = cand[1];
        h[2] = cand[2];
        break;
      }
      step = 0.5 * step;
    }
  }
  make_F_h(h, fr, g1, g2, Fout);
}

// Flux directional derivative for the 12-component state,
// three_d/curved_boundary_warp3d.py:2728-2752 (_state_flux_jvp3).
CV_DEV void jvp3(int axis, const double* U, const double* W, const Mat& m, double* out) {
  double s = 1.0;
  for (int a = 0; a < 12; ++a) s = fmax(s, fabs(W[a]));
  double eps = 1.0e-6 / s;
  double Fp[9], Fm[9];
  for (int k = 0; k < 9; ++k) {
    Fp[k] = U[3 + k] + eps * W[3 + k];
    Fm[k] = U[3 + k] - eps * W[3 + k];
  }
  M3 Pp = piola3(Fp, m);
  M3 Pm = piola3(Fm, m);
  for (int a = 0; a < 12; ++a) out[a] = 0.0;
  for (int i = 0; i < 3; ++i) {
    out[i] = -(Pp.v[3 * i + axis] - Pm.v[3 * i + axis]) / (2.0 * eps);
    out[3 + 3 * i + axis] = -W[i];
  }
}

CV_DEV double state_det3(const double* U) {
  // three_d/curved_boundary_warp3d.py:2719-2725
  return U[3] * (U[7] * U[11] - U[8] * U[10]) - U[4] * (U[6] * U[11] - U[8] * U[9]) +
         U[5] * (U[6] * U[10] - U[7] * U[9]);
}

}  // namespace cv
