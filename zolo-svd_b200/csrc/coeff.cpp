// Host scalar code of the polar iterations: Zolotarev coefficients
// (Auxil_Zolo.f90:36-200), the Zolo FONE / CON recursion (pzolopd1.f90:459-472)
// and the QDWH dynamical weights (hfunc.f90:2-42, pqdwhfacs.f90:361-368).
// Written in double precision with the same operation order as the reference
// so that the iteration control (branch choice, stopping test) matches it.
#include "coeff.h"

#include <cfloat>
#include <cmath>
#include <vector>

namespace zolo {

double eps_precision() { return DBL_EPSILON; }  // DLAMCH('Precision') = 2^-52

void mellipke(double alpha, double tol, double* k, double* e) {
  const double m = std::sin(alpha) * std::sin(alpha);
  double a0 = 1.0, b0 = std::cos(alpha), s0 = m, mm = 1.0, a1 = a0;
  int i1 = 0;
  while (mm > tol) {
    a1 = (a0 + b0) / 2.0;
    const double b1 = std::sqrt(a0 * b0);
    const double c1 = (a0 - b0) / 2.0;
    ++i1;
    const double w1 = std::ldexp(1.0, i1) * (c1 * c1);
    mm = w1;
    s0 = s0 + w1;
    a0 = a1;
    b0 = b1;
  }
  *k = M_PI / (2.0 * a1);
  *e = *k * (1.0 - s0 / 2.0);
}

void mellipj(double u, double alpha, double tol, double* sn, double* cn, double* dn) {
  const int mchunk = 1000;
  const double m = std::sin(alpha) * std::sin(alpha);
  // work arrays reused across calls (every entry read is written first)
  thread_local std::vector<double> a(mchunk + 2), b(mchunk + 2), c(mchunk + 2), phin(mchunk + 2);
  c[1] = std::sin(alpha);
  b[1] = std::cos(alpha);
  a[1] = 1.0;
  int i = 1, nin = 0;
  while (std::fabs(c[i]) > tol && i < mchunk) {
    ++i;
    a[i] = (a[i - 1] + b[i - 1]) * 0.5;
    b[i] = std::sqrt(a[i - 1] * b[i - 1]);
    c[i] = (a[i - 1] - b[i - 1]) * 0.5;
    if (std::fabs(c[i]) <= tol && std::fabs(c[i - 1]) > tol) nin = i - 1;
  }
  phin[1] = u;
  phin[i] = std::ldexp(1.0, nin) * a[i] * u;
  while (i > 1) {
    --i;
    phin[i] = phin[i + 1];
    if (nin >= i) phin[i] = 0.5 * (std::asin(c[i + 1] * std::sin(phin[i + 1]) / a[i + 1]) + phin[i + 1]);
  }
  *sn = std::sin(phin[1]);
  *cn = std::cos(phin[1]);
  *dn = std::sqrt(1.0 - m * (*sn) * (*sn));
}

int choosem(double con) {
  if (con < 1.001) return 2;
  if (con <= 1.01) return 3;
  if (con <= 1.1) return 4;
  if (con <= 1.2) return 5;
  if (con <= 1.5) return 6;
  if (con <= 2) return 8;
  if (con < 6.5) return 2;
  if (con < 180) return 3;
  if (con < 1.5e4) return 4;
  if (con < 2e6) return 5;
  if (con < 1e9) return 6;
  if (con < 3e12) return 7;
  return 8;
}

void compute_coeff(double con, double tol, int rk, double* coeff) {
  const double kappa = 1.0 / con;
  const double alpha = std::acos(kappa);
  double kk, e;
  mellipke(alpha, tol, &kk, &e);
  const int rk2 = 2 * rk;
  for (int i = 1; i <= rk2; ++i) {
    const double t = static_cast<double>(i) * kk / (rk2 + 1.0);
    double sn, cn, dn;
    mellipj(t, alpha, tol, &sn, &cn, &dn);
    coeff[i - 1] = (sn * sn) / (cn * cn);
  }
  for (int i = 1; i <= rk; ++i) {
    double v = 1.0;
    for (int j = 1; j <= rk; ++j) {
      v = v * (coeff[2 * i - 2] - coeff[2 * j - 1]);
      if (i != j) v = v / (coeff[2 * i - 2] - coeff[2 * j - 2]);
    }
    coeff[rk2 + i - 1] = v;
  }
}

// Jacobi sn, cn for the modulus k = sqrt(1 - kp^2) given by its complement kp: the
// descending Landen / AGM scheme of mellipj started from (a, b, c) = (1, kp, k), so kp
// enters exactly (no acos of 1/CON, whose rounding near pi/2 is an absolute error of
// ~1e-16 in kp).
static void jacobi_sn_cn_kp(double u, double kp, double tol, double* sn, double* cn) {
  double a[64], c[64], phin[64];
  double b = kp;
  a[1] = 1.0;
  c[1] = std::sqrt((1.0 - kp) * (1.0 + kp));
  int i = 1;
  while (std::fabs(c[i]) > tol && i < 62) {
    const double an = (a[i] + b) * 0.5;
    const double bn = std::sqrt(a[i] * b);
    c[i + 1] = (a[i] - b) * 0.5;
    a[i + 1] = an;
    b = bn;
    ++i;
  }
  phin[i] = std::ldexp(1.0, i - 1) * a[i] * u;
  for (int j = i; j > 1; --j) phin[j - 1] = 0.5 * (std::asin(c[j] * std::sin(phin[j]) / a[j]) + phin[j]);
  *sn = std::sin(phin[1]);
  *cn = std::cos(phin[1]);
}

// sn, cn for a modulus near one (kp <= 1e-6): the hyperbolic expansions in m1 = kp^2
// (Abramowitz & Stegun 16.15.1-2), whose next terms are O(m1^2 e^{4u}) <= 16 kp^2 relative
// for u <= K/2 (e^{2u} <= 4/kp there).  The AGM scheme above loses ~1e-16/kp relative
// accuracy in this range (checked against 80-digit mpmath: 4e-11 at CON = 1e6).
static void jacobi_sn_cn_near1(double u, double kp, double* sn, double* cn) {
  const double m1 = kp * kp;
  const double th = std::tanh(u), sh = 1.0 / std::cosh(u);
  const double w = 0.25 * m1 * (std::sinh(u) * std::cosh(u) - u);
  *sn = th + w * sh * sh;
  *cn = sh - w * th * sh;
}

void compute_coeff_kp(double con, double tol, int rk, double* coeff) {
  const double kp = 1.0 / con;
  const bool near1 = kp <= 1e-6;
  // K(k) = pi / (2 AGM(1, kp))
  double a0 = 1.0, b0 = kp;
  for (int i = 0; i < 64 && std::fabs(a0 - b0) > tol * a0; ++i) {
    const double a1 = (a0 + b0) * 0.5;
    b0 = std::sqrt(a0 * b0);
    a0 = a1;
  }
  const double kk = M_PI / (2.0 * a0);
  const int rk2 = 2 * rk;
  for (int i = 1; i <= rk2; ++i) {
    const double u = static_cast<double>(i) * kk / (rk2 + 1.0);
    double sn, cn;
    if (2 * i <= rk2 + 1) {
      if (near1) jacobi_sn_cn_near1(u, kp, &sn, &cn);
      else jacobi_sn_cn_kp(u, kp, tol, &sn, &cn);
      coeff[i - 1] = (sn * sn) / (cn * cn);
    } else {
      // sn(u)/cn(u) = cn(K - u) / (kp sn(K - u)): no cancellation in cn(u) -> 0
      const double v = static_cast<double>(rk2 + 1 - i) * kk / (rk2 + 1.0);
      if (near1) jacobi_sn_cn_near1(v, kp, &sn, &cn);
      else jacobi_sn_cn_kp(v, kp, tol, &sn, &cn);
      const double sc = cn / (kp * sn);
      coeff[i - 1] = sc * sc;
    }
  }
  for (int i = 1; i <= rk; ++i) {
    double v = 1.0;
    for (int j = 1; j <= rk; ++j) {
      v = v * (coeff[2 * i - 2] - coeff[2 * j - 1]);
      if (i != j) v = v / (coeff[2 * i - 2] - coeff[2 * j - 2]);
    }
    coeff[rk2 + i - 1] = v;
  }
}

double zolo_fone(const double* coeff, int rk) {
  double f = 1.0;
  for (int i = 1; i <= rk; ++i) f = f * (1.0 + coeff[2 * i - 1]) / (1.0 + coeff[2 * i - 2]);
  return f;
}

double zolo_next_con(double con, const double* coeff, int rk, double fone) {
  double fcon = con;
  for (int i = 1; i <= rk; ++i) fcon = fcon * (con * con + coeff[2 * i - 1]) / (con * con + coeff[2 * i - 2]);
  const double v = fcon / fone;
  return v > 1.0 ? v : 1.0;
}

double hfunc(double x) {
  const double tol = 30.0 * eps_precision();
  const double x2 = x * x;
  double ww;
  if (std::fabs(x - 1.0) <= tol) {
    ww = 0.0;
  } else {
    const double tmp = 4.0 * (1.0 - x2) / (x2 * x2);
    ww = std::exp(std::log(tmp) / 3.0);
  }
  const double sum1 = std::sqrt(1.0 + ww);
  const double h = std::sqrt(8.0 - 4.0 * ww + 8.0 * (2.0 - x2) / (x2 * sum1));
  return sum1 + h / 2.0;
}

void qdwh_weights(double lowk, double* ak, double* bk, double* ck, double* lnext) {
  *ak = hfunc(lowk);
  *bk = (*ak - 1.0) * (*ak - 1.0) / 4.0;
  *ck = *ak + *bk - 1.0;
  const double l2 = lowk * lowk;
  *lnext = lowk * (*ak + *bk * l2) / (1.0 + *ck * l2);
}

}  // namespace zolo
