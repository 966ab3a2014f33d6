// Host-side FP64 numerics shared by the WPCD path: Gauss-Legendre meshes,
// Legendre functions and Wigner coupling symbols.
//
// Where the reference's result bits feed a geometric decision (wave-packet
// boundaries, quadrature meshes of the P123 cell integrals) the arithmetic is
// written with the same operation order as the reference so that both sides
// produce identical doubles.  Compile with -ffp-contract=off.
#pragma once
#include <cstddef>

namespace tt {

// Gauss-Legendre points/weights on [-1,1] by Newton iteration on the Bonnet
// recurrence with the stopping rule |t - t_old| < 3e-16, following
// CPP/General_functions/gauss_legendre.cpp:36-66 (double overload).
void gauss_legendre(double* x, double* w, int n);

// Affine map of a [-1,1] rule onto [a,b]; gauss_legendre.cpp:85-90.
void rescale_rule(double* x, double* w, double a, double b, int n);

// Legendre polynomial P_l(x) by the upward Bonnet recurrence (the published
// method of GSL's gsl_sf_legendre_Pl, GSL 2.x, used by the reference).
double legendre_P(int l, double x);

// dP_l/dx = l (x P_l - P_{l-1}) / (x^2 - 1); auxiliary.cpp:30-33.
double legendre_dP(int l, double x);

// Roots of P_n by Newton's method from the reference's starting guesses
// cos(3.14159 (i + 0.75) / (n + 0.5)) with the relative step test 1e-9
// (auxiliary.cpp:35-75, GSL root_fdfsolver_newton + root_test_delta).
void legendre_roots_newton(double* x, int n);

// Gauss points on [a,b] built on legendre_roots_newton; auxiliary.cpp:77-88.
void gauss_points_newton(double* q, double* w, double a, double b, int n);

// Number of entries of a spherical-harmonic Legendre table up to lmax,
// (lmax+1)(lmax+2)/2, and the index of (l,m), l(l+1)/2+m (GSL layout).
inline int spharm_len(int lmax) { return (lmax + 1) * (lmax + 2) / 2; }
inline int spharm_index(int l, int m) { return l * (l + 1) / 2 + m; }

// Y_l^m(theta, 0) for 0 <= m <= l <= lmax at x = cos(theta), Condon-Shortley
// phase included: the values GSL's gsl_sf_legendre_array_e returns for
// GSL_SF_LEGENDRE_SPHARM with csphase = -1 (make_permutation_matrix.cpp:549-589).
void legendre_spharm_array(int lmax, double x, double* out);

// Wigner symbols with doubled (2j, 2m) integer arguments, same argument order
// as gsl_sf_coupling_3j/6j/9j.  Racah sums evaluated in extended precision;
// every selection-rule violation returns exactly 0.
double wigner3j(int tj1, int tj2, int tj3, int tm1, int tm2, int tm3);
double wigner6j(int tj1, int tj2, int tj3, int tj4, int tj5, int tj6);
double wigner9j(int tj1, int tj2, int tj3, int tj4, int tj5, int tj6,
                int tj7, int tj8, int tj9);

// <j1 m1 j2 m2 | j3 m3> through the 3j symbol; auxiliary.cpp:127-135.
double clebsch_gordan(int tj1, int tj2, int tj3, int tm1, int tm2, int tm3);

// (-1)^n for any integer n.
inline double sign_pow(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }

}  // namespace tt
