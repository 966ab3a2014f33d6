// Host FP64 numerics for the WPCD path.  See tt_math.h.
#include "tt_math.h"

#include <cmath>
#include <cstdlib>
#include <vector>

namespace tt {

void gauss_legendre(double* x, double* w, int n) {
  // Newton on P_n with the Bonnet recurrence; operation order kept equal to
  // CPP/General_functions/gauss_legendre.cpp:47-77 so the points are
  // bit-identical (they define the x-mesh of every P123 cell integral).
  const double eps = 3.e-16;
  const int half = (n + 1) / 2;
  for (int i = 1; i < half + 1; i++) {
    double t = std::cos(M_PI * (i - 0.25) / (n + 0.5));
    double t_old = 1;
    double dp = 0;
    while (std::abs(t - t_old) >= eps) {
      double pa = 1, pb = 0, pc = 0;
      for (int j = 1; j < n + 1; j++) {
        pc = pb;
        pb = pa;
        pa = ((2 * j - 1) * t * pb - (j - 1) * pc) / j;
      }
      dp = n * (t * pa - pb) / (t * t - 1);
      t_old = t;
      t = t_old - pa / dp;
    }
    x[i - 1] = -t;
    x[n - i] = t;
    w[i - 1] = 2. / ((1 - t * t) * dp * dp);
    w[n - i] = w[i - 1];
  }
}

void rescale_rule(double* x, double* w, double a, double b, int n) {
  for (int i = 0; i < n; i++) {
    x[i] = 0.5 * (b - a) * x[i] + 0.5 * (b + a);
    w[i] = 0.5 * (b - a) * w[i];
  }
}

double legendre_P(int l, double x) {
  if (l == 0) return 1.0;
  if (l == 1) return x;
  if (l == 2) return 0.5 * (3.0 * x * x - 1.0);
  if (x == 1.0) return 1.0;
  if (x == -1.0) return (l % 2 == 0) ? 1.0 : -1.0;
  double p_lm2 = 1.0, p_lm1 = x, p_l = x;
  for (int ell = 2; ell <= l; ell++) {
    p_l = (x * (2 * ell - 1) * p_lm1 - (ell - 1) * p_lm2) / ell;
    p_lm2 = p_lm1;
    p_lm1 = p_l;
  }
  return p_l;
}

double legendre_dP(int l, double x) {
  return (l * x * legendre_P(l, x) - l * legendre_P(l - 1, x)) / (x * x - 1);
}

void legendre_roots_newton(double* x, int n) {
  std::vector<double> q(n);
  for (int i = 0; i <= n - 1; i++) q[n - 1 - i] = std::cos(3.14159 * (i + 1 - 0.25) / (n + 0.5));
  for (int i = 0; i <= n - 1; i++) {
    // Newton: r <- r - f(r)/f'(r), f and f' evaluated at the current root.
    double r = q[i];
    double f = legendre_P(n, r);
    double df = legendre_dP(n, r);
    int iter = 0;
    bool more = true;
    while (more && iter < 100) {
      iter++;
      double r_new = r - (f / df);
      r = r_new;
      f = legendre_P(n, r);
      df = legendre_dP(n, r);
      double r_prev = q[i];
      q[i] = r;
      // convergence when |x1 - x0| < epsabs + epsrel |x1| (epsabs 0, epsrel 1e-9)
      more = !(std::fabs(q[i] - r_prev) < 1e-9 * std::fabs(q[i]));
    }
  }
  for (int i = 0; i < n; i++) x[i] = q[i];
}

void gauss_points_newton(double* q, double* w, double a, double b, int n) {
  std::vector<double> t(n);
  legendre_roots_newton(t.data(), n);
  for (int j = 0; j <= n - 1; j++) {
    w[j] = 2.0 / (1 - t[j] * t[j]) * 1.0 / (legendre_dP(n, t[j]) * legendre_dP(n, t[j])) * (b - a) / 2.0;
    q[j] = (b - a) * (t[j] + 1) / 2.0 + a;
  }
}

void legendre_spharm_array(int lmax, double x, double* out) {
  // Normalised associated Legendre functions by the standard stable
  // recurrences: diagonal m=l, first off-diagonal l=m+1, then upward in l.
  const double s = std::sqrt((1.0 - x) * (1.0 + x));
  double ymm = 1.0 / std::sqrt(4.0 * M_PI);
  for (int m = 0; m <= lmax; m++) {
    if (m > 0) ymm = -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * ymm;
    out[spharm_index(m, m)] = ymm;
    if (m + 1 > lmax) continue;
    double y_lm1 = ymm;
    double y_l = x * std::sqrt(2.0 * m + 3.0) * ymm;
    out[spharm_index(m + 1, m)] = y_l;
    for (int l = m + 2; l <= lmax; l++) {
      double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      double b = std::sqrt(((double)(l - 1) * (l - 1) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
      double y_new = a * (x * y_l - b * y_lm1);
      y_lm1 = y_l;
      y_l = y_new;
      out[spharm_index(l, m)] = y_l;
    }
  }
}

// ---------------------------------------------------------------------------
// Wigner symbols (Racah formulae), extended-precision sums.
namespace {

struct FactTable {
  std::vector<long double> f;
  FactTable() : f(401) {
    f[0] = 1.0L;
    for (int i = 1; i < 401; i++) f[i] = f[i - 1] * (long double)i;
  }
};

const FactTable& facts() {
  static FactTable t;
  return t;
}

inline long double fct(int k) { return facts().f[k]; }

// doubled-argument triangle test including integer-sum parity
inline bool triangle(int ta, int tb, int tc) {
  if (ta < 0 || tb < 0 || tc < 0) return false;
  if ((ta + tb + tc) % 2 != 0) return false;
  return tc <= ta + tb && tc >= std::abs(ta - tb);
}

// Delta(abc)^2 = (a+b-c)!(a-b+c)!(-a+b+c)!/(a+b+c+1)!  (doubled arguments)
inline long double delta_sq(int ta, int tb, int tc) {
  return fct((ta + tb - tc) / 2) * fct((ta - tb + tc) / 2) * fct((-ta + tb + tc) / 2) /
         fct((ta + tb + tc) / 2 + 1);
}

long double sixj_ld(int tj1, int tj2, int tj3, int tj4, int tj5, int tj6) {
  if (!triangle(tj1, tj2, tj3) || !triangle(tj1, tj5, tj6) || !triangle(tj4, tj2, tj6) ||
      !triangle(tj4, tj5, tj3))
    return 0.0L;
  const int a1 = (tj1 + tj2 + tj3) / 2, a2 = (tj1 + tj5 + tj6) / 2;
  const int a3 = (tj4 + tj2 + tj6) / 2, a4 = (tj4 + tj5 + tj3) / 2;
  const int b1 = (tj1 + tj2 + tj4 + tj5) / 2, b2 = (tj2 + tj3 + tj5 + tj6) / 2;
  const int b3 = (tj3 + tj1 + tj6 + tj4) / 2;
  int tmin = a1;
  if (a2 > tmin) tmin = a2;
  if (a3 > tmin) tmin = a3;
  if (a4 > tmin) tmin = a4;
  int tmax = b1;
  if (b2 < tmax) tmax = b2;
  if (b3 < tmax) tmax = b3;
  long double sum = 0.0L;
  for (int t = tmin; t <= tmax; t++) {
    long double term = fct(t + 1) / (fct(t - a1) * fct(t - a2) * fct(t - a3) * fct(t - a4) *
                                     fct(b1 - t) * fct(b2 - t) * fct(b3 - t));
    sum += (t % 2 == 0) ? term : -term;
  }
  if (sum == 0.0L) return 0.0L;
  long double pre = std::sqrt(delta_sq(tj1, tj2, tj3) * delta_sq(tj1, tj5, tj6) *
                              delta_sq(tj4, tj2, tj6) * delta_sq(tj4, tj5, tj3));
  return pre * sum;
}

}  // namespace

double wigner3j(int tj1, int tj2, int tj3, int tm1, int tm2, int tm3) {
  if (tj1 < 0 || tj2 < 0 || tj3 < 0) return 0.0;
  if (tm1 + tm2 + tm3 != 0) return 0.0;
  if (std::abs(tm1) > tj1 || std::abs(tm2) > tj2 || std::abs(tm3) > tj3) return 0.0;
  if ((tj1 + tm1) % 2 != 0 || (tj2 + tm2) % 2 != 0 || (tj3 + tm3) % 2 != 0) return 0.0;
  if (!triangle(tj1, tj2, tj3)) return 0.0;
  const int c1 = (tj3 - tj2 + tm1) / 2;  // j3 - j2 + m1
  const int c2 = (tj3 - tj1 - tm2) / 2;  // j3 - j1 - m2
  const int c3 = (tj1 + tj2 - tj3) / 2;  // j1 + j2 - j3
  const int c4 = (tj1 - tm1) / 2;        // j1 - m1
  const int c5 = (tj2 + tm2) / 2;        // j2 + m2
  int kmin = 0;
  if (-c1 > kmin) kmin = -c1;
  if (-c2 > kmin) kmin = -c2;
  int kmax = c3;
  if (c4 < kmax) kmax = c4;
  if (c5 < kmax) kmax = c5;
  long double sum = 0.0L;
  for (int k = kmin; k <= kmax; k++) {
    long double term = 1.0L / (fct(k) * fct(c1 + k) * fct(c2 + k) * fct(c3 - k) * fct(c4 - k) * fct(c5 - k));
    sum += (k % 2 == 0) ? term : -term;
  }
  if (sum == 0.0L) return 0.0;
  long double pre = std::sqrt(delta_sq(tj1, tj2, tj3) * fct((tj1 + tm1) / 2) * fct((tj1 - tm1) / 2) *
                              fct((tj2 + tm2) / 2) * fct((tj2 - tm2) / 2) * fct((tj3 + tm3) / 2) *
                              fct((tj3 - tm3) / 2));
  const int phase = (tj1 - tj2 - tm3) / 2;
  long double v = pre * sum;
  return (double)((phase % 2 == 0) ? v : -v);
}

double wigner6j(int tj1, int tj2, int tj3, int tj4, int tj5, int tj6) {
  return (double)sixj_ld(tj1, tj2, tj3, tj4, tj5, tj6);
}

double wigner9j(int tj1, int tj2, int tj3, int tj4, int tj5, int tj6, int tj7, int tj8, int tj9) {
  if (!triangle(tj1, tj2, tj3) || !triangle(tj4, tj5, tj6) || !triangle(tj7, tj8, tj9) ||
      !triangle(tj1, tj4, tj7) || !triangle(tj2, tj5, tj8) || !triangle(tj3, tj6, tj9))
    return 0.0;
  int xmin = std::abs(tj1 - tj9);
  if (std::abs(tj4 - tj8) > xmin) xmin = std::abs(tj4 - tj8);
  if (std::abs(tj2 - tj6) > xmin) xmin = std::abs(tj2 - tj6);
  int xmax = tj1 + tj9;
  if (tj4 + tj8 < xmax) xmax = tj4 + tj8;
  if (tj2 + tj6 < xmax) xmax = tj2 + tj6;
  long double sum = 0.0L;
  for (int tx = xmin; tx <= xmax; tx += 2) {
    long double t = sixj_ld(tj1, tj4, tj7, tj8, tj9, tx) * sixj_ld(tj2, tj5, tj8, tj4, tx, tj6) *
                    sixj_ld(tj3, tj6, tj9, tx, tj1, tj2);
    t *= (long double)(tx + 1);
    sum += (tx % 2 == 0) ? t : -t;
  }
  return (double)sum;
}

double clebsch_gordan(int tj1, int tj2, int tj3, int tm1, int tm2, int tm3) {
  double result = 0.0;
  if ((std::abs(tm1) <= tj1) && (std::abs(tm2) <= tj2)) {
    result = sign_pow((tj1 - tj2 + tm3) / 2) * std::sqrt((double)(tj3 + 1)) *
             wigner3j(tj1, tj2, tj3, tm1, tm2, -tm3);
  }
  return result;
}

}  // namespace tt
