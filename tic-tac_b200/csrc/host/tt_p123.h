// Host preparation of the per-channel tables the device P123 builder consumes.
// Everything that decides *which* permutation-matrix entries exist (meshes,
// sin/cos of the phi mesh, recoupling coefficients) is computed here in FP64
// with the reference's arithmetic; the device only does +,-,*,/,sqrt,min,max on
// these tables (compiled without FMA contraction), so the overlap decisions are
// bit-identical to the reference's host loops.
#pragma once
#include <cstdint>
#include <vector>

#include "tt_host.h"

namespace tt {

// One term of the geometric function Gtilde_{alpha' alpha}(phi, x) in the
// order of the reference's loops (auxiliary.cpp:991-1061): L_total outer,
// M_total, then M12'.  fac1 = 8 pi^2 Atilde, cgm = CG(L12 l3 Lt; 0 M) (-1)^M,
// cg2 = CG(L12' l3' Lt; M' M-M').  i1/i2/i3 index the spharm tables of
// x, cos(theta1), cos(theta2); s1/s2/s3 are the (-1)^m factors for m < 0.
struct GTerm {
  double fac1, cgm, cg2;
  int32_t i1, i2, i3;
  int32_t signs;  // bit0: s1 = -1, bit1: s2 = -1, bit2: s3 = -1, bit3: first term of an (Lt,M) group
};

struct P123Tables {
  int Np = 0, Nq = 0, Nalpha = 0, Nphi = 0, Nx = 0;
  int two_J_3N = 0, P_3N = 0;
  bool production_run = true;
  std::vector<double> p_WP, q_WP;     // boundaries
  std::vector<double> x, wx;          // [Nx], gauss_legendre
  std::vector<double> phi, wphi;      // [Nq*Np*Nphi], per (q',p') mesh
  std::vector<double> sinphi, cosphi; // host libm values of the phi mesh
  int max_L12 = 0, max_l3 = 0, lenL = 0, lenl = 0;
  std::vector<double> plm1;           // [Nx][lenl] spharm(l3max, x)
  // active (alpha', alpha) pairs: those with at least one term
  std::vector<int32_t> pair_ap, pair_a;
  std::vector<int32_t> pair_term_off; // [npairs+1]
  std::vector<GTerm> terms;
  std::vector<double> pair_norm;      // sqrt((2 L12 + 1)/(4 pi)) of alpha'
  std::vector<int32_t> L12, l3;       // per alpha, for the device Legendre indexing
};

// Builds all tables for one 3N channel (make_permutation_matrix.cpp:324-611).
bool p123_prepare(const RunParams& rp, const FWPStates& fwp, const PWChannel& ch, P123Tables& t,
                  std::string* err);

// Atilde(alpha, alpha', L_total), auxiliary.cpp:863-884.
double atilde(const PWChannel& ch, int a, int ap, int Ltot, int two_J, int two_T);

}  // namespace tt
