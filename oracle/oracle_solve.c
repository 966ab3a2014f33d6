/* CPU oracle: resolvent, A = C^T (2 P123) (V C) and the dense Faddeev solve.
 * Test infrastructure only (see oracle.h).  Restates CPP/make_resolvent.cpp:14-211,
 * CPP/solve_faddeev.cpp:4-181 and 305-438 (with LAPACK's zgetrf/zgetrs replaced
 * by an LU with partial pivoting written out here). */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static const double kMp = 938.272, kMn = 939.565;

static double heav(double v) { return v < 0 ? 0.0 : 1.0; }

void to_resolvent(int Na, int Nq, int Np, const int32_t* e_off, const double* e_swp, const double* qb, double E,
                  double* G) {
  for (int a = 0; a < Na; a++)
    for (int p = 0; p < Np; p++) {
      const double el = e_swp[e_off[a] + p], eu = e_swp[e_off[a] + p + 1];
      const int bound = el < 0;
      const double Eb = bound ? el : 0;
      for (int q = 0; q < Nq; q++) {
        const double ql = qb[q], qu = qb[q + 1];
        const double mu1 = kMn * (kMn + kMp + Eb) / (kMn + kMn + kMp + Eb);
        const double Eql = ql * ql / (2 * mu1), Equ = qu * qu / (2 * mu1), Dq = Equ - Eql;
        double re, im;
        if (bound) {
          re = log(fabs((Eql + Eb - E) / (Equ + Eb - E))) / (Dq);
          im = (heav(Equ + Eb - E) - heav(Eql + Eb - E)) * (-M_PI) / (Dq);
        } else {
          const double Ep = 0.5 * (el + eu), Eq = 0.5 * (Eql + Equ), Dp = eu - el;
          const double DM = 0.5 * (Dp - Dq), DP = 0.5 * (Dp + Dq), D = Ep + Eq - E;
          re = ((D + DM) * log(fabs(D + DM)) + (D - DM) * log(fabs(D - DM)) - (D + DP) * log(fabs(D + DP)) -
                (D - DP) * log(fabs(D - DP))) /
               (Dp * Dq);
          im = ((D + DM) * heav(D + DM) + (D - DM) * heav(D - DM) - (D + DP) * heav(D + DP) - (D - DP) * heav(D - DP)) *
               M_PI / (Dp * Dq);
        }
        const size_t i = (size_t)a * Nq * Np + (size_t)q * Np + p;
        G[2 * i] = re;
        G[2 * i + 1] = im;
      }
    }
}

void to_build_A(int Na, int Nq, int Np, const int64_t* colptr, const int32_t* row, const double* val,
                const int32_t* blk, const int32_t* part, const int32_t* cpl_off, const int32_t* cpl,
                const int64_t* blk_off, const int32_t* blk_dim, const double* C, const double* VC, double* A) {
  const size_t n = (size_t)Na * Nq * Np;
#pragma omp parallel
  {
    double* pvc = malloc(sizeof(double) * n);
#pragma omp for schedule(dynamic)
    for (long c = 0; c < (long)n; c++) {
      const int ac = (int)(c / ((size_t)Nq * Np)), qc = (int)((c / Np) % Nq), pc = (int)(c % Np);
      memset(pvc, 0, sizeof(double) * n);
      /* calculate_PVC_col: column (ac,qc,pc) of (2 P123)(VC), CSC walk */
      const int b = blk[ac], d = blk_dim[b];
      const double* VCb = VC + blk_off[b];
      for (int t = cpl_off[ac]; t < cpl_off[ac + 1]; t++) {
        const int aj = cpl[t];
        for (int pj = 0; pj < Np; pj++) {
          const double vc = VCb[(size_t)(part[aj] * Np + pj) * d + part[ac] * Np + pc];
          const size_t j = (size_t)aj * Nq * Np + (size_t)qc * Np + pj;
          for (int64_t e = colptr[j]; e < colptr[j + 1]; e++) pvc[row[e]] += (2 * val[e]) * vc;
        }
      }
      /* calculate_CPVC_col: C^T blocks applied per (alpha_r, q) */
      for (int ar = 0; ar < Na; ar++) {
        const int br = blk[ar], dr = blk_dim[br];
        const double* Cb = C + blk_off[br];
        for (int q = 0; q < Nq; q++)
          for (int pr = 0; pr < Np; pr++) {
            double s = 0;
            for (int t = cpl_off[ar]; t < cpl_off[ar + 1]; t++) {
              const int ai = cpl[t];
              for (int pi = 0; pi < Np; pi++)
                s += Cb[(size_t)(part[ai] * Np + pi) * dr + part[ar] * Np + pr] *
                     pvc[(size_t)ai * Nq * Np + (size_t)q * Np + pi];
            }
            A[((size_t)ar * Nq * Np + (size_t)q * Np + pr) * n + c] = s;
          }
      }
    }
    free(pvc);
  }
}

int to_dense_solve(int n, const double* A, int nE, const double* G, const int32_t* q_idx, int nd, const int32_t* deut,
                   int Nq, int Np, double* U) {
  double complex* L = malloc(sizeof(double complex) * (size_t)n * n);
  double complex* X = malloc(sizeof(double complex) * (size_t)n * (nd ? nd : 1));
  int* piv = malloc(sizeof(int) * n);
  int status = 0;
  for (int j = 0; j < nE && !status; j++) {
    const double complex* Gj = (const double complex*)(G + 2 * (size_t)j * n);
    for (size_t r = 0; r < (size_t)n; r++)
      for (size_t c = 0; c < (size_t)n; c++) L[r * n + c] = (r == c ? 1.0 : 0.0) - A[r * n + c] * Gj[c];
    /* LU with partial pivoting (largest |re|+|im|, as izamax) */
    for (int k = 0; k < n; k++) {
      int p = k;
      double best = -1;
      for (int i = k; i < n; i++) {
        const double a = fabs(creal(L[(size_t)i * n + k])) + fabs(cimag(L[(size_t)i * n + k]));
        if (a > best) {
          best = a;
          p = i;
        }
      }
      piv[k] = p;
      if (best == 0) {
        status = k + 1;
        break;
      }
      if (p != k)
        for (int c = 0; c < n; c++) {
          const double complex t = L[(size_t)k * n + c];
          L[(size_t)k * n + c] = L[(size_t)p * n + c];
          L[(size_t)p * n + c] = t;
        }
      const double complex d = L[(size_t)k * n + k];
#pragma omp parallel for
      for (int i = k + 1; i < n; i++) {
        const double complex l = L[(size_t)i * n + k] / d;
        L[(size_t)i * n + k] = l;
        for (int c = k + 1; c < n; c++) L[(size_t)i * n + c] -= l * L[(size_t)k * n + c];
      }
    }
    if (status) break;
    /* right-hand sides: the on-shell columns of A */
    for (int dd = 0; dd < nd; dd++) {
      const size_t col = (size_t)deut[dd] * Nq * Np + (size_t)q_idx[j] * Np;
      double complex* x = X + (size_t)dd * n;
      for (int r = 0; r < n; r++) x[r] = A[(size_t)r * n + col];
      for (int k = 0; k < n; k++)
        if (piv[k] != k) {
          const double complex t = x[k];
          x[k] = x[piv[k]];
          x[piv[k]] = t;
        }
      for (int r = 0; r < n; r++)
        for (int c = 0; c < r; c++) x[r] -= L[(size_t)r * n + c] * x[c];
      for (int r = n - 1; r >= 0; r--) {
        for (int c = r + 1; c < n; c++) x[r] -= L[(size_t)r * n + c] * x[c];
        x[r] /= L[(size_t)r * n + r];
      }
    }
    for (int dr = 0; dr < nd; dr++)
      for (int dc = 0; dc < nd; dc++) {
        const size_t rr = (size_t)deut[dr] * Nq * Np + (size_t)q_idx[j] * Np;
        const size_t u = (size_t)dr * nd * nE + (size_t)dc * nE + j;
        U[2 * u] = creal(X[(size_t)dc * n + rr]);
        U[2 * u + 1] = cimag(X[(size_t)dc * n + rr]);
      }
  }
  free(L);
  free(X);
  free(piv);
  return status;
}
