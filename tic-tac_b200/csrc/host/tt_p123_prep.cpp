// Host tables for the device P123 builder.  See tt_p123.h.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <unordered_map>

#include "tt_math.h"
#include "tt_p123.h"

namespace tt {

namespace {

// 9j(L12 S12 J12; l3 1/2 j3; Lt S J) of alpha for total spin S = tS/2.
double ninej(const PWChannel& ch, int a, int Ltot, int tS, int two_J) {
  return wigner9j(2 * ch.L_2N[a], 2 * ch.S_2N[a], 2 * ch.J_2N[a], 2 * ch.L_1N[a], 1, ch.two_J_1N[a], 2 * Ltot, tS,
                  two_J);
}

// The spin and isospin 6j symbols of a pair: 6j(1/2 1/2 S12; 1/2 S S12') for
// tS = 1, 3 in s6[0..1] and 6j(1/2 1/2 T12; 1/2 T T12') in s6[2].
void sixj_pair(const PWChannel& ch, int a, int ap, int two_T, double* s6) {
  s6[0] = wigner6j(1, 1, 2 * ch.S_2N[a], 1, 1, 2 * ch.S_2N[ap]);
  s6[1] = wigner6j(1, 1, 2 * ch.S_2N[a], 1, 3, 2 * ch.S_2N[ap]);
  s6[2] = wigner6j(1, 1, 2 * ch.T_2N[a], 1, two_T, 2 * ch.T_2N[ap]);
}

// Atilde from the two states' 9j symbols n9a[s], n9ap[s] for tS = 1, 3 and
// the pair's 6j symbols s6 (sixj_pair).
double atilde_from(const PWChannel& ch, int a, int ap, const double* n9a, const double* n9ap, const double* s6) {
  // auxiliary.cpp:863-884: sum over total spin S = 1/2, 3/2 of
  // sqrt(hats) (-1)^(S'+T') (2S+1) 9j 9j 6j(spin) 6j(isospin)
  double ret = 0.0;
  for (int tS = 1, s = 0; tS <= 3; tS += 2, s++) {
    ret += std::sqrt((double)((2 * ch.J_2N[a] + 1) * (ch.two_J_1N[a] + 1) * (2 * ch.S_2N[a] + 1) *
                              (2 * ch.T_2N[a] + 1) * (2 * ch.J_2N[ap] + 1) * (ch.two_J_1N[ap] + 1) *
                              (2 * ch.S_2N[ap] + 1) * (2 * ch.T_2N[ap] + 1))) *
           sign_pow(ch.S_2N[ap] + ch.T_2N[ap]) * (tS + 1) * n9a[s] * n9ap[s] * s6[s] * s6[2];
  }
  return ret;
}

}  // namespace

double atilde(const PWChannel& ch, int a, int ap, int Ltot, int two_J, int two_T) {
  const double n9a[2] = {ninej(ch, a, Ltot, 1, two_J), ninej(ch, a, Ltot, 3, two_J)};
  const double n9ap[2] = {ninej(ch, ap, Ltot, 1, two_J), ninej(ch, ap, Ltot, 3, two_J)};
  double s6[3];
  sixj_pair(ch, a, ap, two_T, s6);
  return atilde_from(ch, a, ap, n9a, n9ap, s6);
}

bool p123_prepare(const RunParams& rp, const FWPStates& fwp, const PWChannel& ch, P123Tables& t,
                  std::string* err) {
  t = P123Tables();
  t.Np = fwp.Np_WP;
  t.Nq = fwp.Nq_WP;
  t.Nalpha = ch.Nalpha;
  t.Nphi = rp.Nphi;
  t.Nx = rp.Nx;
  t.two_J_3N = ch.two_J_3N[0];
  t.P_3N = ch.P_3N[0];
  t.production_run = rp.production_run;
  t.p_WP = fwp.p_WP;
  t.q_WP = fwp.q_WP;
  if (t.Nphi < 2 || t.Nx < 2) {
    if (err) *err = "Nphi and Nx must be >= 2";
    return false;
  }
  // x mesh (fill_P123_arrays, make_permutation_matrix.cpp:1330-1332)
  t.x.resize(t.Nx);
  t.wx.resize(t.Nx);
  gauss_legendre(t.x.data(), t.wx.data(), t.Nx);
  // phi mesh per (q',p') cell row (calculate_WP_overlap, :169-183)
  // The reference recomputes the Legendre roots on [-1, 1] for every cell
  // (gauss_points_newton); they and the weights' cell-independent factor are
  // computed once here, and each cell maps them with gauss_points_newton's
  // own expressions, so the meshes are the same bit for bit.
  const size_t nrow = (size_t)t.Nq * t.Np;
  t.phi.resize(nrow * t.Nphi);
  t.wphi.resize(nrow * t.Nphi);
  std::vector<double> root(t.Nphi), wfac(t.Nphi);
  legendre_roots_newton(root.data(), t.Nphi);
  for (int j = 0; j < t.Nphi; j++)
    wfac[j] = 2.0 / (1 - root[j] * root[j]) * 1.0 / (legendre_dP(t.Nphi, root[j]) * legendre_dP(t.Nphi, root[j]));
  for (int qp = 0; qp < t.Nq; qp++) {
    const double qp_l = t.q_WP[qp], qp_u = t.q_WP[qp + 1];
    for (int pp = 0; pp < t.Np; pp++) {
      const double pp_l = t.p_WP[pp], pp_u = t.p_WP[pp + 1];
      const double a = std::atan(pp_l / qp_u);
      const double b = std::atan(pp_u / qp_l);
      const size_t off = ((size_t)qp * t.Np + pp) * t.Nphi;
      for (int j = 0; j < t.Nphi; j++) {
        t.wphi[off + j] = wfac[j] * (b - a) / 2.0;
        t.phi[off + j] = (b - a) * (root[j] + 1) / 2.0 + a;
      }
    }
  }
  t.sinphi.resize(t.phi.size());
  t.cosphi.resize(t.phi.size());
  for (size_t i = 0; i < t.phi.size(); i++) {
    t.sinphi[i] = std::sin(t.phi[i]);
    t.cosphi[i] = std::cos(t.phi[i]);
  }
  // angular-momentum maxima (make_permutation_matrix.cpp:371-390)
  int max_L12 = 0, max_l3 = 0;
  for (int a = 0; a < ch.Nalpha; a++) {
    max_L12 = std::max(max_L12, ch.L_2N[a]);
    max_l3 = std::max(max_l3, ch.L_1N[a]);
  }
  t.max_L12 = max_L12;
  t.max_l3 = max_l3;
  t.lenL = spharm_len(max_L12);
  t.lenl = spharm_len(max_l3);
  const int Lmax = max_L12 + max_l3;
  t.plm1.resize((size_t)t.Nx * t.lenl);
  for (int ix = 0; ix < t.Nx; ix++) legendre_spharm_array(max_l3, t.x[ix], &t.plm1[(size_t)ix * t.lenl]);
  t.L12.assign(ch.L_2N, ch.L_2N + ch.Nalpha);
  t.l3.assign(ch.L_1N, ch.L_1N + ch.Nalpha);

  // Atilde[ap][a][Lt] for equal 2T_3N (make_permutation_matrix.cpp:444-462);
  // each state's 9j symbols are evaluated once per (Lt, S) instead of once per pair
  const int Na = ch.Nalpha;
  std::vector<double> n9((size_t)Na * (Lmax + 1) * 2);
  for (int a = 0; a < Na; a++)
    for (int Lt = 0; Lt <= Lmax; Lt++)
      for (int s = 0; s < 2; s++) n9[((size_t)a * (Lmax + 1) + Lt) * 2 + s] = ninej(ch, a, Lt, 2 * s + 1, t.two_J_3N);
  std::vector<double> At((size_t)Na * Na * (Lmax + 1), 0.0);
  for (int a = 0; a < Na; a++)
    for (int ap = 0; ap < Na; ap++)
      if (ch.two_T_3N[a] == ch.two_T_3N[ap]) {
        double s6[3];
        sixj_pair(ch, a, ap, ch.two_T_3N[a], s6);
        for (int Lt = 0; Lt <= Lmax; Lt++)
          At[((size_t)a * Na + ap) * (Lmax + 1) + Lt] = atilde_from(
              ch, a, ap, &n9[((size_t)a * (Lmax + 1) + Lt) * 2], &n9[((size_t)ap * (Lmax + 1) + Lt) * 2], s6);
      }

  // Term lists.  The reference evaluates Gtilde for (row alpha' = alphap_idx,
  // column alpha = alpha_idx) with Atilde_store[alphap][alpha] and
  // L12 = L(alpha'), l3 = l(alpha'), L12' = L(alpha), l3' = l(alpha)
  // (make_permutation_matrix.cpp:755-787, auxiliary.cpp:950-1067).
  // Clebsch-Gordan values recur across pairs: each argument set is evaluated once
  std::unordered_map<uint64_t, double> cg_memo;
  auto cg = [&](int j1, int j2, int j3, int m1, int m2, int m3) {
    uint64_t key = 0;
    for (int v : {j1, j2, j3, m1, m2, m3}) key = (key << 10) | (uint64_t)(v + 512);
    auto it = cg_memo.find(key);
    if (it != cg_memo.end()) return it->second;
    const double c = clebsch_gordan(j1, j2, j3, m1, m2, m3);
    cg_memo.emplace(key, c);
    return c;
  };
  t.pair_term_off.push_back(0);
  for (int ap = 0; ap < Na; ap++) {
    for (int a = 0; a < Na; a++) {
      const int L12 = ch.L_2N[ap], l3 = ch.L_1N[ap];
      const int L12p = ch.L_2N[a], l3p = ch.L_1N[a];
      const double* A = &At[((size_t)ap * Na + a) * (Lmax + 1)];
      const int Lt_lo = std::max(std::abs(L12 - l3), std::abs(L12p - l3p));
      const int Lt_hi = std::min((t.two_J_3N + 5) / 2, std::min(L12 + l3, L12p + l3p));
      size_t n_before = t.terms.size();
      for (int Lt = Lt_lo; Lt <= Lt_hi; Lt++) {
        const double fac1 = 8.0 * M_PI * M_PI * A[Lt];
        if (fac1 == 0) continue;
        const int Mlim = std::min(l3, Lt);
        for (int M = -Mlim; M <= Mlim; M++) {
          const double cgm = cg(2 * L12, 2 * l3, 2 * Lt, 0, 2 * M, 2 * M) * sign_pow(M);
          bool first = true;
          for (int Mp = -L12p; Mp <= L12p; Mp++) {
            if (std::abs(M - Mp) > l3p) continue;
            GTerm g;
            g.fac1 = fac1;
            g.cgm = cgm;
            g.cg2 = cg(2 * L12p, 2 * l3p, 2 * Lt, 2 * Mp, 2 * M - 2 * Mp, 2 * M);
            g.i1 = spharm_index(l3, std::abs(M));
            g.i2 = spharm_index(L12p, std::abs(Mp));
            g.i3 = spharm_index(l3p, std::abs(M - Mp));
            g.signs = 0;
            if (M < 0 && (M % 2) == -1) g.signs |= 1;
            if (Mp < 0 && (Mp % 2) == -1) g.signs |= 2;
            if ((M - Mp) < 0 && ((M - Mp) % 2) == -1) g.signs |= 4;
            if (first) g.signs |= 8;
            first = false;
            t.terms.push_back(g);
          }
        }
      }
      if (t.terms.size() > n_before) {
        t.pair_ap.push_back(ap);
        t.pair_a.push_back(a);
        t.pair_term_off.push_back((int32_t)t.terms.size());
        t.pair_norm.push_back(std::sqrt((2.0 * L12 + 1) / (4 * M_PI)));
      }
    }
  }
  return true;
}

}  // namespace tt
