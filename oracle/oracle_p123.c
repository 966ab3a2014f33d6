/* CPU oracle: P123 of one 3N channel.  Test infrastructure only (see oracle.h).
 * Restates, loop for loop, CPP/make_permutation_matrix.cpp:160-943 and
 * CPP/auxiliary.cpp:35-88, 127-135, 453-462, 660-746, 863-884, 950-1067, with
 * GSL's coupling coefficients, Legendre functions and Newton root finder
 * (GSL 2.x, not present here) restated from their published formulae. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- numerics ---------------------------------------------------------- */

/* CPP/General_functions/gauss_legendre.cpp:36-66 */
static void gauss(double* x, double* w, int N) {
  double eps = 3.e-16;
  int m = (N + 1) / 2;
  for (int i = 1; i < m + 1; i++) {
    double t = cos(M_PI * (i - 0.25) / (N + 0.5)), t1 = 1, pp = 0;
    while (fabs(t - t1) >= eps) {
      double p1 = 1, p2 = 0, p3;
      for (int j = 1; j < N + 1; j++) {
        p3 = p2;
        p2 = p1;
        p1 = ((2 * j - 1) * t * p2 - (j - 1) * p3) / j;
      }
      pp = N * (t * p1 - p2) / (t * t - 1);
      t1 = t;
      t = t1 - p1 / pp;
    }
    x[i - 1] = -t;
    x[N - i] = t;
    w[i - 1] = 2. / ((1 - t * t) * pp * pp);
    w[N - i] = w[i - 1];
  }
}

/* Bonnet upward recurrence (GSL gsl_sf_legendre_Pl) */
static double legP(int l, double x) {
  if (l == 0) return 1.0;
  if (l == 1) return x;
  if (l == 2) return 0.5 * (3.0 * x * x - 1.0);
  if (x == 1.0) return 1.0;
  if (x == -1.0) return (l % 2 == 0) ? 1.0 : -1.0;
  double a = 1.0, b = x, c = x;
  for (int ell = 2; ell <= l; ell++) {
    c = (x * (2 * ell - 1) * b - (ell - 1) * a) / ell;
    a = b;
    b = c;
  }
  return c;
}
static double dlegP(int n, double x) { return (n * x * legP(n, x) - n * legP(n - 1, x)) / (x * x - 1); }

/* auxiliary.cpp:35-88: Newton roots with GSL's relative delta test 1e-9 */
static void calc_gauss_points(double* q, double* w, double pmin, double pmax, int N) {
  double* t = (double*)malloc(sizeof(double) * N);
  for (int i = 0; i <= N - 1; i++) t[N - 1 - i] = cos(3.14159 * (i + 1 - 0.25) / (N + 0.5));
  for (int i = 0; i <= N - 1; i++) {
    double r = t[i], f = legP(N, r), df = dlegP(N, r);
    int iter = 0, more = 1;
    while (more && iter < 100) {
      iter++;
      r = r - (f / df);
      f = legP(N, r);
      df = dlegP(N, r);
      double prev = t[i];
      t[i] = r;
      more = !(fabs(t[i] - prev) < 1e-9 * fabs(t[i]));
    }
  }
  for (int j = 0; j <= N - 1; j++) {
    w[j] = 2.0 / (1 - t[j] * t[j]) * 1.0 / (dlegP(N, t[j]) * dlegP(N, t[j])) * (pmax - pmin) / 2.0;
    q[j] = (pmax - pmin) * (t[j] + 1) / 2.0 + pmin;
  }
  free(t);
}

static long double fct(int k) {
  static long double tab[401];
  static int init = 0;
  if (!init) {
    tab[0] = 1.0L;
    for (int i = 1; i < 401; i++) tab[i] = tab[i - 1] * (long double)i;
    init = 1;
  }
  return tab[k];
}
static int tri(int a, int b, int c) {
  if (a < 0 || b < 0 || c < 0 || (a + b + c) % 2) return 0;
  return c <= a + b && c >= abs(a - b);
}
static long double dsq(int a, int b, int c) {
  return fct((a + b - c) / 2) * fct((a - b + c) / 2) * fct((-a + b + c) / 2) / fct((a + b + c) / 2 + 1);
}
/* Racah formula, doubled arguments */
static double w3j(int j1, int j2, int j3, int m1, int m2, int m3) {
  if (m1 + m2 + m3 != 0 || abs(m1) > j1 || abs(m2) > j2 || abs(m3) > j3) return 0;
  if ((j1 + m1) % 2 || (j2 + m2) % 2 || (j3 + m3) % 2 || !tri(j1, j2, j3)) return 0;
  int c1 = (j3 - j2 + m1) / 2, c2 = (j3 - j1 - m2) / 2, c3 = (j1 + j2 - j3) / 2, c4 = (j1 - m1) / 2,
      c5 = (j2 + m2) / 2;
  int kmin = 0, kmax = c3;
  if (-c1 > kmin) kmin = -c1;
  if (-c2 > kmin) kmin = -c2;
  if (c4 < kmax) kmax = c4;
  if (c5 < kmax) kmax = c5;
  long double s = 0;
  for (int k = kmin; k <= kmax; k++) {
    long double t = 1.0L / (fct(k) * fct(c1 + k) * fct(c2 + k) * fct(c3 - k) * fct(c4 - k) * fct(c5 - k));
    s += (k % 2) ? -t : t;
  }
  if (s == 0) return 0;
  long double pre = sqrtl(dsq(j1, j2, j3) * fct((j1 + m1) / 2) * fct((j1 - m1) / 2) * fct((j2 + m2) / 2) *
                          fct((j2 - m2) / 2) * fct((j3 + m3) / 2) * fct((j3 - m3) / 2));
  long double v = pre * s;
  return (double)((((j1 - j2 - m3) / 2) % 2) ? -v : v);
}
static long double w6j_ld(int j1, int j2, int j3, int j4, int j5, int j6) {
  if (!tri(j1, j2, j3) || !tri(j1, j5, j6) || !tri(j4, j2, j6) || !tri(j4, j5, j3)) return 0;
  int a1 = (j1 + j2 + j3) / 2, a2 = (j1 + j5 + j6) / 2, a3 = (j4 + j2 + j6) / 2, a4 = (j4 + j5 + j3) / 2;
  int b1 = (j1 + j2 + j4 + j5) / 2, b2 = (j2 + j3 + j5 + j6) / 2, b3 = (j3 + j1 + j6 + j4) / 2;
  int tmin = a1, tmax = b1;
  if (a2 > tmin) tmin = a2;
  if (a3 > tmin) tmin = a3;
  if (a4 > tmin) tmin = a4;
  if (b2 < tmax) tmax = b2;
  if (b3 < tmax) tmax = b3;
  long double s = 0;
  for (int t = tmin; t <= tmax; t++) {
    long double v = fct(t + 1) / (fct(t - a1) * fct(t - a2) * fct(t - a3) * fct(t - a4) * fct(b1 - t) * fct(b2 - t) *
                                  fct(b3 - t));
    s += (t % 2) ? -v : v;
  }
  if (s == 0) return 0;
  return sqrtl(dsq(j1, j2, j3) * dsq(j1, j5, j6) * dsq(j4, j2, j6) * dsq(j4, j5, j3)) * s;
}
static double w6j(int a, int b, int c, int d, int e, int f) { return (double)w6j_ld(a, b, c, d, e, f); }
static double w9j(int j1, int j2, int j3, int j4, int j5, int j6, int j7, int j8, int j9) {
  if (!tri(j1, j2, j3) || !tri(j4, j5, j6) || !tri(j7, j8, j9) || !tri(j1, j4, j7) || !tri(j2, j5, j8) ||
      !tri(j3, j6, j9))
    return 0;
  int xmin = abs(j1 - j9), xmax = j1 + j9;
  if (abs(j4 - j8) > xmin) xmin = abs(j4 - j8);
  if (abs(j2 - j6) > xmin) xmin = abs(j2 - j6);
  if (j4 + j8 < xmax) xmax = j4 + j8;
  if (j2 + j6 < xmax) xmax = j2 + j6;
  long double s = 0;
  for (int x = xmin; x <= xmax; x += 2) {
    long double t = w6j_ld(j1, j4, j7, j8, j9, x) * w6j_ld(j2, j5, j8, j4, x, j6) * w6j_ld(j3, j6, j9, x, j1, j2) *
                    (long double)(x + 1);
    s += (x % 2) ? -t : t;
  }
  return (double)s;
}
static double sgn(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }
static double clebsch(int j1, int j2, int j3, int m1, int m2, int m3) {
  if (abs(m1) <= j1 && abs(m2) <= j2) return sgn((j1 - j2 + m3) / 2) * sqrt(j3 + 1) * w3j(j1, j2, j3, m1, m2, -m3);
  return 0;
}
/* Y_l^m(theta,0), m >= 0, Condon-Shortley phase, index l(l+1)/2+m */
static void spharm(int lmax, double x, double* out) {
  double s = sqrt((1.0 - x) * (1.0 + x)), ymm = 1.0 / sqrt(4.0 * M_PI);
  for (int m = 0; m <= lmax; m++) {
    if (m > 0) ymm = -sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * ymm;
    out[m * (m + 1) / 2 + m] = ymm;
    if (m + 1 > lmax) continue;
    double y1 = ymm, y = x * sqrt(2.0 * m + 3.0) * ymm;
    out[(m + 1) * (m + 2) / 2 + m] = y;
    for (int l = m + 2; l <= lmax; l++) {
      double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      double b = sqrt(((double)(l - 1) * (l - 1) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
      double yn = a * (x * y - b * y1);
      y1 = y;
      y = yn;
      out[l * (l + 1) / 2 + m] = y;
    }
  }
}
static double pi1t(double p, double q, double x) { return sqrt(0.25 * p * p + 9.0 / 16.0 * q * q + 0.75 * p * q * x); }
static double pi2t(double p, double q, double x) { return sqrt(p * p + 0.25 * q * q - p * q * x); }
static double dmax(double a, double b) { return (a < b) ? b : a; }
static double dmin(double a, double b) { return (b < a) ? b : a; }

/* ---- P123 ---------------------------------------------------------------- */

typedef struct {
  int64_t key;
  double val;
} coo_t;
static int cmp_coo(const void* a, const void* b) {
  int64_t x = ((const coo_t*)a)->key, y = ((const coo_t*)b)->key;
  return (x > y) - (x < y);
}

int to_p123(int Np, int Nq, const double* pb, const double* qb, int Nphi, int Nx, int Na, const int* pw,
            int64_t* nnz_out, int32_t** row_out, int32_t** col_out, double** val_out) {
#define L12(a) pw[9 * (a) + 0]
#define S12(a) pw[9 * (a) + 1]
#define J12(a) pw[9 * (a) + 2]
#define T12(a) pw[9 * (a) + 3]
#define l3(a) pw[9 * (a) + 4]
#define j3(a) pw[9 * (a) + 5]
#define TT3(a) pw[9 * (a) + 7]
  const int two_J = pw[6];
  const size_t nrow = (size_t)Nq * Np;
  double* x = malloc(sizeof(double) * Nx);
  double* wx = malloc(sizeof(double) * Nx);
  gauss(x, wx, Nx);
  double* phi = malloc(sizeof(double) * nrow * Nphi);
  double* wphi = malloc(sizeof(double) * nrow * Nphi);
  unsigned char* mask = malloc(nrow * nrow);
  /* calculate_WP_overlap, make_permutation_matrix.cpp:160-255 */
#pragma omp parallel for schedule(dynamic)
  for (int qp = 0; qp < Nq; qp++) {
    double qp_l = qb[qp], qp_u = qb[qp + 1];
    for (int pp = 0; pp < Np; pp++) {
      double pp_l = pb[pp], pp_u = pb[pp + 1];
      double phi_lo = atan(pp_l / qp_u), phi_hi = atan(pp_u / qp_l);
      size_t r = (size_t)qp * Np + pp;
      calc_gauss_points(&phi[r * Nphi], &wphi[r * Nphi], phi_lo, phi_hi, Nphi);
      for (int q = 0; q < Nq; q++)
        for (int p = 0; p < Np; p++) {
          double q_l = qb[q], q_u = qb[q + 1], p_l = pb[p], p_u = pb[p + 1];
          int hit = 0;
          if (phi_lo < phi_hi) {
            for (int ip = 0; ip < Nphi && !hit; ip++) {
              double ph = phi[r * Nphi + ip], s = sin(ph), c = cos(ph);
              double kmin = dmax(pp_l / s, qp_l / c), kmax = dmin(pp_u / s, qp_u / c);
              if (kmin < kmax)
                for (int ix = 0; ix < Nx; ix++) {
                  double z1 = pi1t(s, c, x[ix]), z2 = pi2t(s, c, x[ix]);
                  double hl = dmax(p_l / z1, q_l / z2), hu = dmin(p_u / z1, q_u / z2);
                  if (hl < hu) {
                    if (dmax(kmin, hl) < dmin(kmax, hu)) {
                      hit = 1;
                      break;
                    }
                  }
                }
            }
          }
          mask[r * nrow + (size_t)q * Np + p] = (unsigned char)hit;
        }
    }
  }
  int maxL = 0, maxl = 0;
  for (int a = 0; a < Na; a++) {
    if (L12(a) > maxL) maxL = L12(a);
    if (l3(a) > maxl) maxl = l3(a);
  }
  const int Lmax = maxL + maxl, lenL = (maxL + 1) * (maxL + 2) / 2, lenl = (maxl + 1) * (maxl + 2) / 2;
  double* At = calloc((size_t)Na * Na * (Lmax + 1), sizeof(double));
  for (int a = 0; a < Na; a++)
    for (int ap = 0; ap < Na; ap++) {
      if (TT3(a) != TT3(ap)) continue;
      const int two_T = TT3(a);
      for (int Lt = 0; Lt <= Lmax; Lt++) {
        double ret = 0;
        for (int tS = 1; tS <= 3; tS += 2)
          ret += sqrt((double)((2 * J12(a) + 1) * (j3(a) + 1) * (2 * S12(a) + 1) * (2 * T12(a) + 1) *
                               (2 * J12(ap) + 1) * (j3(ap) + 1) * (2 * S12(ap) + 1) * (2 * T12(ap) + 1))) *
                 sgn(S12(ap) + T12(ap)) * (tS + 1) *
                 w9j(2 * L12(a), 2 * S12(a), 2 * J12(a), 2 * l3(a), 1, j3(a), 2 * Lt, tS, two_J) *
                 w9j(2 * L12(ap), 2 * S12(ap), 2 * J12(ap), 2 * l3(ap), 1, j3(ap), 2 * Lt, tS, two_J) *
                 w6j(1, 1, 2 * S12(a), 1, tS, 2 * S12(ap)) * w6j(1, 1, 2 * T12(a), 1, two_T, 2 * T12(ap));
        At[((size_t)a * Na + ap) * (Lmax + 1) + Lt] = ret;
      }
    }
  double* sn = malloc(sizeof(double) * nrow * Nphi);
  double* cs = malloc(sizeof(double) * nrow * Nphi);
  for (size_t i = 0; i < nrow * Nphi; i++) {
    sn[i] = sin(phi[i]);
    cs[i] = cos(phi[i]);
  }
  double* P1 = malloc(sizeof(double) * Nx * lenl);
  for (int ix = 0; ix < Nx; ix++) spharm(maxl, x[ix], &P1[ix * lenl]);
  const int n = Na * Nq * Np;
  size_t cap = 1 << 20, cnt = 0;
  coo_t* out = malloc(sizeof(coo_t) * cap);
  const int K = Nphi * Nx;
#pragma omp parallel
  {
    double* G = malloc(sizeof(double) * K);
    double* P2 = malloc(sizeof(double) * K * lenL);
    double* P3 = malloc(sizeof(double) * K * lenl);
#pragma omp for schedule(dynamic)
    for (long r = 0; r < (long)nrow; r++) {
      const int qp = (int)(r / Np), pp = (int)(r % Np);
      const double* s = &sn[r * Nphi];
      const double* c = &cs[r * Nphi];
      for (int ip = 0; ip < Nphi; ip++)
        for (int ix = 0; ix < Nx; ix++) {
          double p = s[ip], q = c[ip], xv = x[ix];
          double ct1 = -(0.5 * p + 0.75 * q * xv) / pi1t(p, q, xv), ct2 = (p - 0.5 * q * xv) / pi2t(p, q, xv);
          ct1 = ct1 > 1 ? 1 : (ct1 < -1 ? -1 : ct1);
          ct2 = ct2 > 1 ? 1 : (ct2 < -1 ? -1 : ct2);
          spharm(maxL, ct1, &P2[(ip * Nx + ix) * lenL]);
          spharm(maxl, ct2, &P3[(ip * Nx + ix) * lenl]);
        }
      for (int ap = 0; ap < Na; ap++)
        for (int a = 0; a < Na; a++) {
          /* Gtilde_subarray_new with L12 = L(alpha'), L12' = L(alpha) (auxiliary.cpp:950-1067) */
          const int L1 = L12(ap), s3 = l3(ap), L1p = L12(a), s3p = l3(a);
          const double* Ar = &At[((size_t)ap * Na + a) * (Lmax + 1)];
          int lo = abs(L1 - s3), hi = (two_J + 5) / 2;
          if (abs(L1p - s3p) > lo) lo = abs(L1p - s3p);
          if (L1 + s3 < hi) hi = L1 + s3;
          if (L1p + s3p < hi) hi = L1p + s3p;
          for (int k = 0; k < K; k++) {
            const int ix = k % Nx;
            double ret = 0;
            for (int Lt = lo; Lt <= hi; Lt++) {
              double fac1 = 8.0 * M_PI * M_PI * Ar[Lt];
              if (fac1 == 0) continue;
              int Ml = s3 < Lt ? s3 : Lt;
              for (int M = -Ml; M <= Ml; M++) {
                double v1 = P1[ix * lenl + s3 * (s3 + 1) / 2 + abs(M)];
                if (M < 0 && M % 2 == -1) v1 = -v1;
                double fac2 = clebsch(2 * L1, 2 * s3, 2 * Lt, 0, 2 * M, 2 * M) * sgn(M) * v1;
                if (fac2 == 0) continue;
                for (int Mp = -L1p; Mp <= L1p; Mp++) {
                  if (abs(M - Mp) > s3p) continue;
                  double v2 = P2[k * lenL + L1p * (L1p + 1) / 2 + abs(Mp)];
                  if (Mp < 0 && Mp % 2 == -1) v2 = -v2;
                  int Md = M - Mp;
                  double v3 = P3[k * lenl + s3p * (s3p + 1) / 2 + abs(Md)];
                  if (Md < 0 && Md % 2 == -1) v3 = -v3;
                  ret += fac1 * fac2 * clebsch(2 * L1p, 2 * s3p, 2 * Lt, 2 * Mp, 2 * M - 2 * Mp, 2 * M) * v2 * v3;
                }
              }
            }
            G[k] = ret * sqrt((2.0 * L1 + 1) / (4 * M_PI));
          }
          for (int q = 0; q < Nq; q++)
            for (int p = 0; p < Np; p++) {
              if (!mask[r * nrow + (size_t)q * Np + p]) continue;
              /* calculate_P123_element_in_WP_basis_mod, auxiliary.cpp:660-746 */
              double p_l = pb[p], p_u = pb[p + 1], q_l = qb[q], q_u = qb[q + 1];
              double pp_l = pb[pp], pp_u = pb[pp + 1], qp_l = qb[qp], qp_u = qb[qp + 1];
              double sum = 0;
              for (int ix = 0; ix < Nx; ix++)
                for (int ip = 0; ip < Nphi; ip++) {
                  double si = s[ip], co = c[ip], z1 = pi1t(si, co, x[ix]), z2 = pi2t(si, co, x[ix]);
                  double kmin = dmax(dmax(dmax(pp_l / si, qp_l / co), p_l / z1), q_l / z2);
                  double kmax = dmin(dmin(dmin(pp_u / si, qp_u / co), p_u / z1), q_u / z2);
                  if (kmin > kmax) continue;
                  sum += wx[ix] * wphi[r * Nphi + ip] * co * si * G[ip * Nx + ix] * (kmax * kmax - kmin * kmin) /
                         (2 * z1 * z2);
                }
              double nw = sqrt(q_u - q_l) * sqrt(p_u - p_l) * sqrt(qp_u - qp_l) * sqrt(pp_u - pp_l);
              double v = sum / nw;
              if (v != 0) {
                int64_t row = (int64_t)ap * Nq * Np + (int64_t)qp * Np + pp;
                int64_t col = (int64_t)a * Nq * Np + (int64_t)q * Np + p;
#pragma omp critical
                {
                  if (cnt == cap) {
                    cap *= 2;
                    out = realloc(out, sizeof(coo_t) * cap);
                  }
                  out[cnt].key = row * n + col;
                  out[cnt].val = v;
                  cnt++;
                }
              }
            }
        }
    }
    free(G);
    free(P2);
    free(P3);
  }
  qsort(out, cnt, sizeof(coo_t), cmp_coo);
  *nnz_out = (int64_t)cnt;
  *row_out = malloc(sizeof(int32_t) * (cnt ? cnt : 1));
  *col_out = malloc(sizeof(int32_t) * (cnt ? cnt : 1));
  *val_out = malloc(sizeof(double) * (cnt ? cnt : 1));
  for (size_t i = 0; i < cnt; i++) {
    (*row_out)[i] = (int32_t)(out[i].key / n);
    (*col_out)[i] = (int32_t)(out[i].key % n);
    (*val_out)[i] = out[i].val;
  }
  free(out);
  free(x);
  free(wx);
  free(phi);
  free(wphi);
  free(mask);
  free(At);
  free(sn);
  free(cs);
  free(P1);
  return 0;
}

void to_free(void* p) { free(p); }
