// Two-nucleon input of the WPCD path: potential models, potential matrices in
// the free wave-packet basis and scattering wave packets (SWP).  Each routine
// restates the reference routine named in tt_host.h with the same arithmetic.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <numeric>
#include <system_error>
#include <thread>

#include "tt_host.h"
#include "tt_math.h"

namespace tt {

// ---------------------------------------------------------------------------
// Malfliet-Tjon I-III (Interactions/malfliet_tjon.cpp:27-66): pure S-wave.
class MalflietTjon : public Potential {
 public:
  void V(double qi, double qo, bool, int, int J, int, int, double* Varray) override {
    for (int k = 0; k < 6; k++) Varray[k] = 0;
    const double VA_I = 513.968, VA_III = 626.885, VR = 1438.720;
    double muA = 1.550, muR = 3.110;
    muA *= kHbarc;
    muR *= kHbarc;
    if (J == 0 || J == 1) {
      const double num_A = (qo + qi) * (qo + qi) + muA * muA;
      const double num_R = (qo + qi) * (qo + qi) + muR * muR;
      const double den_A = (qo - qi) * (qo - qi) + muA * muA;
      const double den_R = (qo - qi) * (qo - qi) + muR * muR;
      const double VA = (J == 0) ? VA_I : VA_III;
      const double v = ((VR / kHbarc) * std::log(num_R / den_R) - (VA / kHbarc) * std::log(num_A / den_A)) /
                       (2 * M_PI * qi * qo);
      Varray[J == 0 ? 0 : 2] = v;
    }
  }
};

// One-pion exchange with a 150-point angular quadrature (Interactions/OPEP.cpp)
// and the chiral LO contact terms (Interactions/chiral_LO_internal.cpp:27-68).
class ChiralLO : public Potential {
 public:
  explicit ChiralLO(double c1s0 = kC1S0, double c3s1 = kC3S1) : c1s0_(c1s0), c3s1_(c3s1), z_(kNz), wz_(kNz) {
    gauss_legendre(z_.data(), wz_.data(), kNz);
    // Legendre values P_l(z_i) for l = 0..kJmax+1 by the Bonnet recurrence
    // (General_functions/legendre.cpp:155-178).
    pl_.assign((kJmax + 2) * kNz, 0.0);
    for (int i = 0; i < kNz; i++) {
      pl_[0 * kNz + i] = 1;
      pl_[1 * kNz + i] = z_[i];
    }
    for (int l = 1; l < kJmax + 1; l++)
      for (int i = 0; i < kNz; i++)
        pl_[(l + 1) * kNz + i] = ((2 * l + 1) * z_[i] * pl_[l * kNz + i] - l * pl_[(l - 1) * kNz + i]) / (l + 1);
  }
  void V(double qi, double qo, bool, int, int J, int, int, double* Varray) override {
    for (int k = 0; k < 6; k++) Varray[k] = 0;
    opep(qi, qo, J, Varray);
    if (J == 0) Varray[0] += c1s0_;
    else if (J == 1) Varray[2] += c3s1_;
    const double M = kMN;
    const double Epi = std::sqrt(M * M + qi * qi);
    const double Epo = std::sqrt(M * M + qo * qo);
    const double rel_i = std::sqrt(M / Epi);
    const double rel_o = std::sqrt(M / Epo);
    double t1 = qi / kLambdaLO;
    double t2 = t1 * t1 * t1 * t1 * t1 * t1;
    const double f1 = std::exp(-t2);
    t1 = qo / kLambdaLO;
    t2 = t1 * t1 * t1 * t1 * t1 * t1;
    const double f2 = std::exp(-t2);
    const double coeff = f1 * f2 * rel_i * rel_o / (8 * M_PI * M_PI * M_PI);
    for (int k = 0; k < 6; k++) Varray[k] *= coeff;
  }

 private:
  static constexpr int kNz = 150;
  static constexpr int kJmax = 100;
  double c1s0_, c3s1_;  // contact LECs of the 1S0 and 3S1 waves
  std::vector<double> z_, wz_, pl_;

  static int iso_fac(int L, int S) {
    const int T = ((1 - L - S) & 1);
    return -3 * (1 - T) + 1 * T;
  }
  static double pot_mom(double qi, double qo, double z) {
    const double q2 = qi * qi + qo * qo - 2 * qi * qo * z;
    return -(kGA * kGA / (4 * kFpi * kFpi)) * (1. / (q2 + kMpi * kMpi));
  }
  double ang_integral(double qi, double qo, int J, int l) const {
    double integral = 0;
    if (l == 0) {
      for (int i = 0; i < kNz; i++) integral += wz_[i] * pot_mom(qi, qo, z_[i]) * pl_[J * kNz + i];
    } else {
      for (int i = 0; i < kNz; i++) integral += wz_[i] * pot_mom(qi, qo, z_[i]) * z_[i] * pl_[J * kNz + i];
    }
    return M_PI * integral;
  }
  void opep(double qi, double qo, int J, double* Varray) const {
    const double i0 = ang_integral(qi, qo, J, 0);
    const double i1 = ang_integral(qi, qo, J, 1);
    const double iP = ang_integral(qi, qo, J + 1, 0);
    double s0 = 0, s1 = 0, mm = 0, pm = 0, mp = 0, pp = 0;
    s0 = 2 * (-(qo * qo + qi * qi) * i0 + 2 * qo * qi * i1);
    pp = (2. / (2 * J + 1)) * (-(qo * qo + qi * qi) * iP + 2 * qo * qi * i0);
    s0 *= iso_fac(J, 0);
    pp *= iso_fac(J + 1, 1);
    if (J != 0) {
      const double iM = ang_integral(qi, qo, J - 1, 0);
      s1 = 2 * ((qo * qo + qi * qi) * i0 - 2 * qo * qi * (1. / (2 * J + 1)) * (J * iP + (J + 1) * iM));
      mm = (2. / (2 * J + 1)) * ((qo * qo + qi * qi) * iM - 2 * qo * qi * i0);
      pm = (4 * std::sqrt(J * (J + 1)) / (2 * J + 1)) * (qi * qi * iP + qo * qo * iM - 2 * qo * qi * i0);
      mp = (4 * std::sqrt(J * (J + 1)) / (2 * J + 1)) * (qi * qi * iM + qo * qo * iP - 2 * qo * qi * i0);
      s1 *= iso_fac(J, 1);
      mm *= iso_fac(J - 1, 1);
      pm *= iso_fac(J - 1, 1);
      mp *= iso_fac(J + 1, 1);
    }
    Varray[0] = s0;
    Varray[1] = s1;
    Varray[2] = mm;
    Varray[3] = pm;
    Varray[4] = mp;
    Varray[5] = pp;
  }
};

int num_lecs(const std::string& name) { return name == "LO_internal" ? 2 : 0; }

std::vector<double> nominal_lecs(const std::string& name) {
  if (name == "LO_internal") return {kC1S0, kC3S1};
  return {};
}

Potential* make_potential(const std::string& name, std::string* err, const std::vector<double>& lec_offsets) {
  if ((int)lec_offsets.size() > num_lecs(name)) {
    if (err) *err = "potential model '" + name + "' has " + std::to_string(num_lecs(name)) + " adjustable constants, " +
                    std::to_string(lec_offsets.size()) + " offsets given";
    return nullptr;
  }
  if (name == "malfliet_tjon") return new MalflietTjon();
  if (name == "LO_internal") {
    const double d0 = lec_offsets.size() > 0 ? lec_offsets[0] : 0.0;
    const double d1 = lec_offsets.size() > 1 ? lec_offsets[1] : 0.0;
    return new ChiralLO(kC1S0 + d0, kC3S1 + d1);
  }
  if (err)
    *err = "potential model '" + name +
           "' is not available: the chiral N2LOopt/Idaho_N3LO and Nijmegen models exist only as Fortran in the "
           "reference (no Fortran compiler on this platform); use malfliet_tjon or LO_internal";
  return nullptr;
}

// ---------------------------------------------------------------------------
// extract_potential_element_from_array, make_potential_matrix.cpp:4-48
static double extract_element(int L, int Lp, int J, int S, bool coupled, const double* V) {
  const double sgn = -1;
  if (coupled) {
    if (L == Lp && L < J) return V[2];
    if (L == Lp && L > J) return V[5];
    if (L < Lp) return sgn * V[4];
    return sgn * V[3];
  }
  if (L == J + 1) return V[5];
  if (L == J - 1) return V[2];
  if (S == 0) return V[0];
  if (S == 1 && L == J) return V[1];
  return 0;
}

namespace {

// One 2N matrix of potential_matrices: the (alpha_r, alpha_c) pair that first
// touches it and how its elements are formed.
struct VTask {
  int L_r, L_c, S_r, J_r, T_r;
  int iso_type;  // 0 np (T = 0), 1 nn/np average (T = 1), 2 / 3 isospin-breaking 1S0 blocks
  bool via_L, via_T, coupled_matrix, coupled_model;
  int idx;       // 2N slot in V_coup (coupled_matrix) or V_unco
};

// Isoscalar potential Vis[6] at (p_in, p_out) for one task
// (make_potential_matrix.cpp:215-300).
void isoscalar(Potential& pot, const RunParams& rp, const VTask& t, double p_in, double p_out, double* Vis) {
  const int Tz_nn = -1, Tz_np = 0;
  double Vnn[6], Vnp[6];
  const bool np_only = rp.midpoint_approx ? t.iso_type == 0 : (!t.via_T && t.iso_type == 0);
  const bool average = rp.midpoint_approx ? t.iso_type == 1 : (!t.via_T && t.iso_type == 1);
  if (np_only) {
    pot.V(p_in, p_out, t.coupled_model, t.S_r, t.J_r, t.T_r, Tz_np, Vis);
  } else if (average) {
    pot.V(p_in, p_out, t.coupled_model, t.S_r, t.J_r, t.T_r, Tz_nn, Vnn);
    pot.V(p_in, p_out, t.coupled_model, t.S_r, t.J_r, t.T_r, Tz_np, Vnp);
    for (int k = 0; k < 6; k++) Vis[k] = (2. / 3) * Vnn[k] + (1. / 3) * Vnp[k];
  } else {  // the 1S0 block coupled through T_3N
    pot.V(p_in, p_out, t.coupled_model, t.S_r, t.J_r, t.T_r, Tz_nn, Vnn);
    pot.V(p_in, p_out, t.coupled_model, t.S_r, t.J_r, t.T_r, Tz_np, Vnp);
    const double e_nn = extract_element(t.L_r, t.L_c, t.J_r, t.S_r, false, Vnn);
    const double e_np = extract_element(t.L_r, t.L_c, t.J_r, t.S_r, false, Vnp);
    Vis[2] = (2. / 3) * e_nn + (1. / 3) * e_np;
    Vis[3] = (std::sqrt(2) / 3.) * (e_nn - e_np);
    Vis[4] = (std::sqrt(2) / 3.) * (e_nn - e_np);
    Vis[5] = (1. / 3) * e_nn + (2. / 3) * e_np;
  }
}

// Row br of a task's matrix: every element is a quadrature double sum over
// the two bins' points (or the bin mid-points), summed in the same order for
// any thread count, so V does not depend on how rows are shared out.
void potential_row(Potential& pot, const RunParams& rp, const FWPStates& fwp, const VTask& t, int br,
                   std::vector<double>& V_unco, std::vector<double>& V_coup) {
  const int Np = fwp.Np_WP;
  const double N_r = fwp.norm_p[br];
  double Vwp[6], Vis[6] = {0, 0, 0, 0, 0, 0};
  for (int bc = 0; bc < Np; bc++) {
    const double N_c = fwp.norm_p[bc];
    for (int k = 0; k < 6; k++) Vwp[k] = 0;
    if (rp.midpoint_approx) {
      const double p_in = fwp.p[bc], p_out = fwp.p[br];
      const double f_in = fwp.fp[bc], f_out = fwp.fp[br];
      const double d_c = fwp.p_WP[bc + 1] - fwp.p_WP[bc];
      const double d_r = fwp.p_WP[br + 1] - fwp.p_WP[br];
      for (int k = 0; k < 6; k++) Vis[k] = 0;
      isoscalar(pot, rp, t, p_in, p_out, Vis);
      for (int k = 0; k < 6; k++) Vwp[k] += p_in * p_out * f_in * f_out * d_r * d_c * Vis[k] / (N_r * N_c);
    } else {
      const int npw = fwp.Np_per_WP;
      for (int ir = 0; ir < npw; ir++) {
        const double p_r = fwp.p[br * npw + ir];
        const double wp_r = fwp.wp[br * npw + ir];
        const double wpf_r = fwp.fp[br * npw + ir] * wp_r * p_r;
        for (int ic = 0; ic < npw; ic++) {
          const double p_c = fwp.p[bc * npw + ic];
          const double wp_c = fwp.wp[bc * npw + ic];
          const double wpf_c = fwp.fp[bc * npw + ic] * wp_c * p_c;
          const double fac = wpf_r * wpf_c;
          isoscalar(pot, rp, t, p_c, p_r, Vis);
          for (int k = 0; k < 6; k++) Vwp[k] += fac * Vis[k] / (N_r * N_c);
        }
      }
    }
    if (t.coupled_matrix) {
      double* M = &V_coup[(size_t)t.idx * 4 * Np * Np];
      const size_t ul = (size_t)br * 2 * Np + bc, ur = ul + Np;
      const size_t ll = (size_t)(br + Np) * 2 * Np + bc, lr = ll + Np;
      if (t.via_L) {
        M[ul] = extract_element(t.J_r - 1, t.J_r - 1, t.J_r, t.S_r, true, Vwp);
        M[ur] = extract_element(t.J_r - 1, t.J_r + 1, t.J_r, t.S_r, true, Vwp);
        M[ll] = extract_element(t.J_r + 1, t.J_r - 1, t.J_r, t.S_r, true, Vwp);
        M[lr] = extract_element(t.J_r + 1, t.J_r + 1, t.J_r, t.S_r, true, Vwp);
      } else {
        M[ul] = Vwp[2];
        M[ur] = Vwp[3];
        M[ll] = Vwp[4];
        M[lr] = Vwp[5];
      }
    } else {
      V_unco[(size_t)t.idx * Np * Np + (size_t)br * Np + bc] = extract_element(t.L_r, t.L_c, t.J_r, t.S_r, false, Vwp);
    }
  }
}

}  // namespace

bool potential_matrices(const RunParams& rp, const FWPStates& fwp, const PWStates& pw,
                        std::vector<double>& V_unco, std::vector<double>& V_coup, std::string* err) {
  std::unique_ptr<Potential> pot(make_potential(rp.potential_model, err, rp.lec_offsets));
  if (!pot) return false;
  int n_unco = 0, n_coup = 0;
  count_2N_channels(rp, n_unco, n_coup);
  const int Np = fwp.Np_WP;
  V_unco.assign((size_t)Np * Np * n_unco, 0.0);
  V_coup.assign((size_t)Np * Np * 4 * n_coup, 0.0);
  // the 2N matrices in the reference's discovery order (every (alpha_r,
  // alpha_c) pair of equal T, J, S and allowed L; a matrix once), with the
  // reference's errors in that order (make_potential_matrix.cpp:51-214)
  std::vector<char> done_unco(n_unco, 0), done_coup(n_coup, 0);
  std::vector<VTask> tasks;
  const bool tf = rp.tensor_force;
  for (int r = 0; r < pw.Nalpha; r++) {
    const int L_r = pw.L_2N[r], S_r = pw.S_2N[r], J_r = pw.J_2N[r], T_r = pw.T_2N[r];
    const int tT_r = pw.two_T_3N[r];
    for (int c = 0; c < pw.Nalpha; c++) {
      const int L_c = pw.L_2N[c], S_c = pw.S_2N[c], J_c = pw.J_2N[c], T_c = pw.T_2N[c];
      const int tT_c = pw.two_T_3N[c];
      const bool check_L = ((tf && std::abs(L_r - L_c) <= 2) || L_r == L_c);
      if (!(T_r == T_c && J_r == J_c && S_r == S_c && check_L)) continue;
      const bool state_1S0 = (S_r == 0 && J_r == 0 && L_r == 0);
      VTask t;
      t.iso_type = -1;
      if (state_1S0 && tT_r == 3 && tT_c == 3) t.iso_type = 2;
      else if ((state_1S0 && (tT_r == 3 && tT_c == 1)) || (tT_r == 1 && tT_c == 3)) t.iso_type = 3;
      else if (T_r == 0 && tT_r == tT_c && tT_r == 1) t.iso_type = 0;
      else if (T_r == 1 && tT_r == tT_c && tT_r == 1) t.iso_type = 1;
      else {
        if (err) *err = "Unknown isoscalar-potential encountered in potential-matrix construction";
        return false;
      }
      t.via_L = (tf && (L_r != L_c || (L_r == L_c && L_r != J_r && J_r != 0)));
      t.via_T = (state_1S0 && rp.isospin_breaking_1S0);
      if (t.via_L && t.via_T) {
        if (err) *err = "isospin-breaking in coupled channels is not supported";
        return false;
      }
      t.coupled_matrix = t.via_L || t.via_T;
      t.coupled_model = (L_r != L_c || (L_r == L_c && L_r != J_r));
      t.L_r = L_r;
      t.L_c = L_c;
      t.S_r = S_r;
      t.J_r = J_r;
      t.T_r = T_r;
      t.idx = unique_2N_idx(L_r, S_r, J_r, T_r, t.coupled_matrix, rp);
      std::vector<char>& done = t.coupled_matrix ? done_coup : done_unco;
      if (t.idx < 0 || t.idx >= (int)done.size()) {
        if (err) *err = "partial wave maps to a 2N channel outside the potential arrays";
        return false;
      }
      if (done[t.idx]) continue;
      done[t.idx] = 1;
      // outside the mid-point approximation an isospin-breaking block needs T_3N coupling
      if (!rp.midpoint_approx && !t.via_T && (t.iso_type == 2 || t.iso_type == 3)) {
        if (err) *err = "Unknown isoscalar potential encountered";
        return false;
      }
      tasks.push_back(t);
    }
  }
  // rows of all matrices shared out over the host's cores
  const size_t items = tasks.size() * (size_t)Np;
  auto work = [&](std::atomic<size_t>* next) {
    for (size_t it = next->fetch_add(1); it < items; it = next->fetch_add(1))
      potential_row(*pot, rp, fwp, tasks[it / Np], (int)(it % Np), V_unco, V_coup);
  };
  std::atomic<size_t> next{0};
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nthreads = std::min<size_t>({hw, (size_t)64, std::max<size_t>(1, items / 4)});
  std::vector<std::thread> pool;
  try {
    for (size_t k = 1; k < nthreads; k++) pool.emplace_back(work, &next);
  } catch (const std::system_error&) {
    // fewer threads than asked for: the ones running (and this one) take all rows
  }
  work(&next);
  for (auto& th : pool) th.join();
  return true;
}

// ---------------------------------------------------------------------------
void symmetric_eigen(const double* A, int n, double* w, double* z) {
  // Cyclic Jacobi rotations (Rutishauser's formulation) on a copy of A,
  // accumulating the rotations in V; converged when the off-diagonal mass
  // underflows relative to the diagonal.
  std::vector<double> a(A, A + (size_t)n * n), v((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; i++) {
      diag += a[(size_t)i * n + i] * a[(size_t)i * n + i];
      for (int j = i + 1; j < n; j++) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
    }
    if (off <= 1e-36 * diag || off == 0.0) break;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) {
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
    }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int i, int j) { return a[(size_t)i * n + i] < a[(size_t)j * n + j]; });
  for (int k = 0; k < n; k++) {
    const int src = order[k];
    w[k] = a[(size_t)src * n + src];
    // fixed sign convention: largest-magnitude component positive
    int imax = 0;
    for (int i = 1; i < n; i++)
      if (std::fabs(v[(size_t)i * n + src]) > std::fabs(v[(size_t)imax * n + src])) imax = i;
    const double sg = v[(size_t)imax * n + src] < 0 ? -1.0 : 1.0;
    for (int i = 0; i < n; i++) z[(size_t)i * n + k] = sg * v[(size_t)i * n + src];
  }
}

bool make_swp_states(const RunParams& rp, const FWPStates& fwp, const PWStates& pw,
                     const std::vector<double>& V_unco, const std::vector<double>& V_coup,
                     SWPStates& swp, std::string* err) {
  const int Np = fwp.Np_WP;
  swp = SWPStates();
  swp.Np_WP = fwp.Np_WP;
  swp.Nq_WP = fwp.Nq_WP;
  swp.q_WP = fwp.q_WP;
  count_2N_channels(rp, swp.n_unco, swp.n_coup);
  swp.e_unco.assign((size_t)(Np + 1) * swp.n_unco, 0.0);
  swp.e_coup.assign((size_t)2 * (Np + 1) * swp.n_coup, 0.0);
  swp.C_unco.assign(V_unco.size(), 0.0);
  swp.C_coup.assign(V_coup.size(), 0.0);
  std::vector<char> done_unco(swp.n_unco, 0), done_coup(swp.n_coup, 0);
  // free Hamiltonian of momentum wave packets, make_swp_states.cpp:28-42
  std::vector<double> H0(Np);
  for (int i = 0; i < Np; i++) {
    const double p1 = fwp.p_WP[i], p2 = fwp.p_WP[i + 1];
    H0[i] = (p2 * p2 + p2 * p1 + p1 * p1) / (6 * kMu23);
  }
  const bool tf = rp.tensor_force;
  double E_bound = 0;
  for (int r = 0; r < pw.Nalpha; r++) {
    const int L_r = pw.L_2N[r], S_r = pw.S_2N[r], J_r = pw.J_2N[r], T_r = pw.T_2N[r];
    for (int c = 0; c < pw.Nalpha; c++) {
      const int L_c = pw.L_2N[c], S_c = pw.S_2N[c], J_c = pw.J_2N[c], T_c = pw.T_2N[c];
      if (!(T_r == T_c && J_r == J_c && S_r == S_c && std::abs(L_r - L_c) <= 2)) continue;
      const bool state_1S0 = (S_r == 0 && J_r == 0 && L_r == 0);
      const bool via_L = (tf && (L_r != L_c || (L_r == L_c && L_r != J_r && J_r != 0)));
      const bool via_T = (state_1S0 && rp.isospin_breaking_1S0);
      if (via_L && via_T) {
        if (err) *err = "isospin-breaking in coupled channels is not supported";
        return false;
      }
      const bool coupled = via_L || via_T;
      int dim, chn;
      const double* V;
      double *C, *e;
      if (coupled) {
        dim = 2 * Np;
        chn = unique_2N_idx(L_r, S_r, J_r, T_r, true, rp);
        if (done_coup[chn]) continue;
        done_coup[chn] = 1;
        V = &V_coup[(size_t)chn * dim * dim];
        C = &swp.C_coup[(size_t)chn * dim * dim];
        e = &swp.e_coup[(size_t)chn * 2 * (Np + 1)];
      } else {
        dim = Np;
        chn = unique_2N_idx(L_r, S_r, J_r, T_r, false, rp);
        if (done_unco[chn]) continue;
        done_unco[chn] = 1;
        V = &V_unco[(size_t)chn * dim * dim];
        C = &swp.C_unco[(size_t)chn * dim * dim];
        e = &swp.e_unco[(size_t)chn * (Np + 1)];
      }
      // H = H0 + V from the upper triangle (construct_full_hamiltonian, :45-81)
      std::vector<double> H((size_t)dim * dim, 0.0), ev(dim);
      for (int i = 0; i < dim; i++) {
        for (int j = i; j < dim; j++) {
          double h = V[(size_t)i * dim + j];
          if (i == j) h = H0[i % Np] + h;
          H[(size_t)i * dim + j] = h;
          H[(size_t)j * dim + i] = h;
        }
      }
      symmetric_eigen(H.data(), dim, ev.data(), C);
      const bool chn_3S1 = (L_r == 0 && S_r == 1 && J_r == 1 && T_r == 0);
      int n_bound = 0;
      for (int i = 0; i < dim; i++) {
        if (ev[i] < 0) {
          n_bound += 1;
          E_bound = ev[i];
        }
      }
      if (!((n_bound == 0 && !chn_3S1) || (n_bound == 1 && chn_3S1))) {
        if (err)
          *err = n_bound != 0 ? "Found unphysical bound states in NN-pair Hamiltonian eigenspectrum"
                              : "Didn't find any bound states in NN-pair Hamiltonian eigenspectrum";
        return false;
      }
      if (coupled) {
        // reorder_coupled_eigenspectrum, :85-112
        std::vector<double> vals(2 * Np), vecs((size_t)4 * Np * Np);
        for (int i = 0; i < Np; i++) {
          vals[i] = ev[2 * i];
          vals[i + Np] = ev[2 * i + 1];
          for (int j = 0; j < 2 * Np; j++) {
            vecs[(size_t)j * 2 * Np + i] = C[(size_t)j * 2 * Np + 2 * i];
            vecs[(size_t)j * 2 * Np + i + Np] = C[(size_t)j * 2 * Np + 2 * i + 1];
          }
        }
        std::copy(vals.begin(), vals.end(), ev.begin());
        std::copy(vecs.begin(), vecs.end(), C);
      }
      // make_swp_bin_boundaries, :146-183
      e[0] = 0;
      if (coupled) e[Np + 1] = 0;
      for (int i = 0; i < Np - 1; i++) {
        e[i + 1] = 0.5 * (ev[i + 1] + ev[i]);
        if (coupled) e[i + 1 + Np + 1] = 0.5 * (ev[i + 1 + Np] + ev[i + Np]);
      }
      e[Np] = ev[Np - 1] + 0.5 * (e[Np - 1] - e[Np - 2]);
      if (coupled) e[2 * Np + 1] = ev[2 * Np - 1] + 0.5 * (e[2 * Np] - e[2 * Np - 1]);
      if (chn_3S1) {
        e[0] = ev[0];
        e[1] = 0;
      }
    }
  }
  swp.E_bound = E_bound;
  return true;
}

void swp_derivative(const FWPStates& fwp, const std::vector<double>& V_unco, const std::vector<double>& V_coup,
                    const SWPStates& swp, const double* dV_unco, const double* dV_coup, SWPStates& d) {
  const int Np = swp.Np_WP;
  d = swp;
  d.E_bound = 0;
  std::fill(d.e_unco.begin(), d.e_unco.end(), 0.0);
  std::fill(d.e_coup.begin(), d.e_coup.end(), 0.0);
  std::vector<double> H0(Np);
  for (int i = 0; i < Np; i++) {
    const double p1 = fwp.p_WP[i], p2 = fwp.p_WP[i + 1];
    H0[i] = (p2 * p2 + p2 * p1 + p1 * p1) / (6 * kMu23);
  }
  auto block = [&](int dim, bool coupled, const double* V, const double* dV, const double* C, double* dC, double* de) {
    // H and dH symmetric from their upper triangles, as make_swp_states builds H
    std::vector<double> H((size_t)dim * dim), dH((size_t)dim * dim);
    for (int i = 0; i < dim; i++)
      for (int j = i; j < dim; j++) {
        double h = V[(size_t)i * dim + j];
        if (i == j) h += H0[i % Np];
        H[(size_t)i * dim + j] = H[(size_t)j * dim + i] = h;
        dH[(size_t)i * dim + j] = dH[(size_t)j * dim + i] = dV[(size_t)i * dim + j];
      }
    // eps_m (Rayleigh quotients of the stored eigenvectors) and M = C^T dH C
    std::vector<double> HC((size_t)dim * dim, 0.0), dHC((size_t)dim * dim, 0.0), eps(dim), M((size_t)dim * dim);
    for (int i = 0; i < dim; i++)
      for (int k = 0; k < dim; k++) {
        const double h = H[(size_t)i * dim + k], dh = dH[(size_t)i * dim + k];
        for (int m = 0; m < dim; m++) {
          HC[(size_t)i * dim + m] += h * C[(size_t)k * dim + m];
          dHC[(size_t)i * dim + m] += dh * C[(size_t)k * dim + m];
        }
      }
    for (int l = 0; l < dim; l++)
      for (int m = 0; m < dim; m++) {
        double s = 0, sh = 0;
        for (int i = 0; i < dim; i++) {
          s += C[(size_t)i * dim + l] * dHC[(size_t)i * dim + m];
          if (l == m) sh += C[(size_t)i * dim + l] * HC[(size_t)i * dim + m];
        }
        M[(size_t)l * dim + m] = s;
        if (l == m) eps[m] = sh;
      }
    for (int m = 0; m < dim; m++)
      for (int i = 0; i < dim; i++) {
        double v = 0;
        for (int l = 0; l < dim; l++) {
          if (l == m) continue;
          const double gap = eps[m] - eps[l];
          if (std::fabs(gap) <= 1e-12 * (std::fabs(eps[m]) + std::fabs(eps[l]) + 1.0)) continue;
          v += C[(size_t)i * dim + l] * M[(size_t)l * dim + m] / gap;
        }
        dC[(size_t)i * dim + m] = v;
      }
    // bin boundaries (make_swp_bin_boundaries): mid-points of consecutive
    // eigenvalues per half, the last bin as wide again as half the one before,
    // the bound state's bin [E_bound, 0]
    for (int h = 0; h < (coupled ? 2 : 1); h++) {
      double* e = de + h * (Np + 1);
      const int off = h * Np;
      e[0] = 0;
      for (int i = 0; i < Np - 1; i++) e[i + 1] = 0.5 * (M[(size_t)(off + i + 1) * dim + off + i + 1] +
                                                      M[(size_t)(off + i) * dim + off + i]);
      e[Np] = M[(size_t)(off + Np - 1) * dim + off + Np - 1] + 0.5 * (e[Np - 1] - e[Np - 2]);
    }
    if (eps[0] < 0) {
      de[0] = M[0];
      de[1] = 0;
      d.E_bound = M[0];
    }
  };
  const size_t nu = (size_t)Np * Np, nc = (size_t)4 * Np * Np;
  for (int b = 0; b < swp.n_unco; b++)
    block(Np, false, &V_unco[b * nu], dV_unco + b * nu, &swp.C_unco[b * nu], &d.C_unco[b * nu],
          &d.e_unco[(size_t)b * (Np + 1)]);
  for (int b = 0; b < swp.n_coup; b++)
    block(2 * Np, true, &V_coup[b * nc], dV_coup + b * nc, &swp.C_coup[b * nc], &d.C_coup[b * nc],
          &d.e_coup[(size_t)b * 2 * (Np + 1)]);
}

}  // namespace tt
