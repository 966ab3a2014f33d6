/* GSL subset used by the reference's P123 and kinematics code, restated for
 * the reference build used as the parity oracle (GSL is not installed here).
 * Wigner symbols and Legendre functions come from the mathematics (Racah
 * sums, normalised Legendre recurrences); the root solver is Newton's method
 * with GSL's documented delta test.  Test infrastructure only. */
#ifndef TT_GSL_SHIM_H
#define TT_GSL_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define GSL_SUCCESS 0
#define GSL_CONTINUE (-2)
#define GSL_MAX_INT(a, b) ((a) > (b) ? (a) : (b))
#define GSL_MIN_INT(a, b) ((a) < (b) ? (a) : (b))
typedef enum { GSL_SF_LEGENDRE_SCHMIDT, GSL_SF_LEGENDRE_SPHARM, GSL_SF_LEGENDRE_FULL, GSL_SF_LEGENDRE_NONE } gsl_sf_legendre_t;
double gsl_sf_coupling_3j(int two_ja, int two_jb, int two_jc, int two_ma, int two_mb, int two_mc);
double gsl_sf_coupling_6j(int two_ja, int two_jb, int two_jc, int two_jd, int two_je, int two_jf);
double gsl_sf_coupling_9j(int two_ja, int two_jb, int two_jc, int two_jd, int two_je, int two_jf, int two_jg, int two_jh, int two_ji);
double gsl_sf_legendre_Pl(int l, double x);
double gsl_sf_legendre_sphPlm(int l, int m, double x);
int gsl_sf_legendre_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase, double* result_array);
size_t gsl_sf_legendre_array_n(size_t lmax);
size_t gsl_sf_legendre_array_index(size_t l, size_t m);
double gsl_sf_pow_int(double x, int n);

typedef struct { double dat[2]; } gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) do { (zp)->dat[0] = (x); (zp)->dat[1] = (y); } while (0)
gsl_complex gsl_complex_exp(gsl_complex a);
gsl_complex gsl_complex_mul_real(gsl_complex a, double x);
gsl_complex gsl_complex_conjugate(gsl_complex a);

typedef struct {
  double (*f)(double x, void* params);
  double (*df)(double x, void* params);
  void (*fdf)(double x, void* params, double* f, double* df);
  void* params;
} gsl_function_fdf;
typedef struct { const char* name; } gsl_root_fdfsolver_type;
typedef struct {
  const gsl_root_fdfsolver_type* type;
  gsl_function_fdf* fdf;
  double root, f, df;
} gsl_root_fdfsolver;
extern const gsl_root_fdfsolver_type* gsl_root_fdfsolver_newton;
gsl_root_fdfsolver* gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type* T);
int gsl_root_fdfsolver_set(gsl_root_fdfsolver* s, gsl_function_fdf* fdf, double root);
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver* s);
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver* s);
void gsl_root_fdfsolver_free(gsl_root_fdfsolver* s);
int gsl_root_test_delta(double x1, double x0, double epsabs, double epsrel);
#ifdef __cplusplus
}
#endif
#endif
