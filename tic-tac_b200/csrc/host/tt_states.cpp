// Host state-space setup: run parameters, partial waves, WP grids, on-shell
// indexing and kinematics.  See tt_host.h for the reference routine each
// function restates.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "tt_host.h"
#include "tt_math.h"

namespace tt {

static bool parse_bool(const std::string& v, bool& out) {
  if (v == "true") { out = true; return true; }
  if (v == "false") { out = false; return true; }
  return false;
}

bool set_run_parameter(RunParams& rp, const std::string& key, const std::string& value, std::string* err) {
  auto bad = [&](const char* what) {
    if (err) *err = std::string("invalid value for ") + what + ": " + value;
    return false;
  };
  try {
    if (key == "two_J_3N_max") rp.two_J_3N_max = std::stoi(value);
    else if (key == "Np_WP") rp.Np_WP = std::stoi(value);
    else if (key == "Nq_WP") rp.Nq_WP = std::stoi(value);
    else if (key == "J_2N_max") rp.J_2N_max = std::stoi(value);
    else if (key == "Nphi") rp.Nphi = std::stoi(value);
    else if (key == "Nx") rp.Nx = std::stoi(value);
    else if (key == "chebyshev_t") rp.chebyshev_t = std::stod(value);
    else if (key == "chebyshev_s") rp.chebyshev_s = std::stod(value);
    else if (key == "Np_per_WP") rp.Np_per_WP = std::stoi(value);
    else if (key == "Nq_per_WP") rp.Nq_per_WP = std::stoi(value);
    else if (key == "channel_idx") rp.channel_idx = std::stoi(value);
    else if (key == "parallel_run") { if (!parse_bool(value, rp.parallel_run)) return bad("parallel_run"); }
    else if (key == "tensor_force") { if (!parse_bool(value, rp.tensor_force)) return bad("tensor_force"); }
    else if (key == "isospin_breaking_1S0") { if (!parse_bool(value, rp.isospin_breaking_1S0)) return bad("isospin_breaking_1S0"); }
    else if (key == "midpoint_approx") { if (!parse_bool(value, rp.midpoint_approx)) return bad("midpoint_approx"); }
    else if (key == "calculate_and_store_P123") { if (!parse_bool(value, rp.calculate_and_store_P123)) return bad("calculate_and_store_P123"); }
    else if (key == "solve_faddeev") { if (!parse_bool(value, rp.solve_faddeev)) return bad("solve_faddeev"); }
    else if (key == "solve_dense") { if (!parse_bool(value, rp.solve_dense)) return bad("solve_dense"); }
    else if (key == "production_run") { if (!parse_bool(value, rp.production_run)) return bad("production_run"); }
    else if (key == "swave_only") { if (!parse_bool(value, rp.swave_only)) return bad("swave_only"); }
    else if (key == "include_breakup_channels") {
      if (!parse_bool(value, rp.include_breakup_channels)) return bad("include_breakup_channels");
    }
    else if (key == "potential_model") rp.potential_model = value;
    else if (key == "energy_input_file") rp.energy_input_file = value;
    else if (key == "output_folder") rp.output_folder = value;
    else if (key == "P123_folder") rp.P123_folder = value;
    else if (key == "p_grid_type") rp.p_grid_type = value;
    else if (key == "q_grid_type") rp.q_grid_type = value;
    else if (key == "p_grid_filename") rp.p_grid_filename = value;
    else if (key == "q_grid_filename") rp.q_grid_filename = value;
    else if (key == "precision") {
      if (value != "fp64" && value != "mixed") return bad("precision");
      rp.precision = value;
    } else if (key == "refine_tol") rp.refine_tol = std::stod(value);
    else if (key == "refine_max_iter") rp.refine_max_iter = std::stoi(value);
    else if (key == "adjoint_basis") {
      if (value == "total") rp.adjoint_total = true;
      else if (value == "fixed") rp.adjoint_total = false;
      else return bad("adjoint_basis (total or fixed)");
    } else if (key == "panel_width") {
      rp.panel_width = std::stoi(value);
      if (rp.panel_width < 0 || rp.panel_width > 512 || rp.panel_width % 32) return bad("panel_width (0 or 32..512)");
    } else if (key == "inverse_block") {
      rp.inverse_block = std::stoi(value);
      if (rp.inverse_block < 0 || rp.inverse_block > 512 || rp.inverse_block % 32)
        return bad("inverse_block (0 or 32..512)");
    } else if (key == "mid_panel") {
      rp.mid_panel = std::stoi(value);
      if (rp.mid_panel < 0 || rp.mid_panel > 512 || rp.mid_panel % 32) return bad("mid_panel (0 or 32..512)");
    } else if (key == "cta_pairs") {
      if (!parse_bool(value, rp.cta_pairs)) return bad("cta_pairs (true or false)");
    } else if (key == "panel_order") {
      if (value == "blocked") rp.panel_blocked = true;
      else if (value == "recursive") rp.panel_blocked = false;
      else return bad("panel_order (recursive or blocked)");
    } else if (key == "tc_product") {
      if (value == "bf16x3_n128") rp.tc_product = 1;
      else if (value == "tf32") rp.tc_product = 2;
      else if (value == "bf16x3") rp.tc_product = 3;
      else return bad("tc_product (tf32, bf16x3 or bf16x3_n128)");
    } else if (key == "energy_batch") {
      rp.energy_batch = std::stoi(value);
      if (rp.energy_batch < 1 || rp.energy_batch > 4) return bad("energy_batch (1..4)");
    }
    else if (key == "lab_energies") {
      rp.lab_energies.clear();
      std::stringstream ss(value);
      std::string tok;
      while (std::getline(ss, tok, ',')) if (!tok.empty()) rp.lab_energies.push_back(std::stod(tok));
    } else if (key == "lec_offsets") {
      rp.lec_offsets.clear();
      std::stringstream ss(value);
      std::string tok;
      while (std::getline(ss, tok, ',')) if (!tok.empty()) rp.lec_offsets.push_back(std::stod(tok));
    } else if (key == "subfolder" || key == "P123_omp_num_threads" || key == "P123_recovery" ||
               key == "parameter_walk" || key == "parameter_file" ||
               key == "PSI_start" || key == "PSI_end") {
      // accepted for argument-surface compatibility; no effect on this path
    } else {
      if (err) *err = "unrecognised run option: " + key;
      return false;
    }
  } catch (...) {
    if (err) *err = "could not parse value for " + key + ": " + value;
    return false;
  }
  return true;
}

bool read_input_energies(const std::string& path, std::vector<double>& out, std::string* err) {
  if (path.size() < 4 || path.substr(path.size() - 4) != ".txt") {
    if (err) *err = "Input energy file must be .txt";
    return false;
  }
  std::ifstream f(path);
  if (!f) {
    if (err) *err = "cannot open energy file " + path;
    return false;
  }
  out.clear();
  double e;
  while (f >> e) out.push_back(e);
  return true;
}

// ---------------------------------------------------------------------------
int unique_2N_idx(int L, int S, int J, int T, bool coupled, const RunParams& rp) {
  const bool state_1S0 = (S == 0 && J == 0 && L == 0 && T == 1);
  int idx = -1;
  if (rp.tensor_force) {
    if (coupled) {
      idx = J - 1;
      if (!state_1S0 && rp.isospin_breaking_1S0) idx += 1;
      if (state_1S0 && rp.isospin_breaking_1S0) idx = 0;
    } else {
      idx = 2 * J + S;
      if (rp.isospin_breaking_1S0) idx -= 1;
    }
  } else {
    if (coupled) {
      if (rp.isospin_breaking_1S0) idx = 0;
    } else {
      idx = J * (4 * (J > 1) + 2) + (S == 1) + (S == 1 && J != 0) * (J - L + 1);
      if (rp.isospin_breaking_1S0) idx -= 1;
    }
  }
  return idx;
}

bool construct_pw_states(const RunParams& rp, PWStates& pw, std::string* err) {
  if (rp.J_2N_max < 0) {
    if (err) *err = "Cannot have negative J_2N!";
    return false;
  }
  if (rp.two_J_3N_max % 2 == 0 || rp.two_J_3N_max <= 0) {
    if (err) *err = "Cannot have even two_J_3N_max!";
    return false;
  }
  pw = PWStates();
  pw.J_2N_max = rp.J_2N_max;
  const int two_T_3N_max = rp.isospin_breaking_1S0 ? 3 : 1;
  int n_prev = 0;
  for (int two_J_3N = 1; two_J_3N < rp.two_J_3N_max + 1; two_J_3N += 2) {
    for (int par_rem = 0; par_rem < 2; par_rem++) {
      int n_in_chn = 0;
      for (int two_T_3N = 1; two_T_3N < two_T_3N_max + 1; two_T_3N += 2) {
        for (int J = 0; J < rp.J_2N_max + 1; J++) {
          for (int S = 0; S < 2; S++) {
            const int Lmin = std::abs(J - S), Lmax = J + S;
            for (int L = Lmin; L < Lmax + 1; L++) {
              const int Tmin = std::abs(two_T_3N - 1) / 2;
              int Tmax = (two_T_3N + 1) / 2;
              if (Tmax > 1) Tmax = 1;
              for (int T = Tmin; T < Tmax + 1; T++) {
                if (!((L + S + T) % 2)) continue;  // generalised Pauli principle
                const int tj_min = std::abs(two_J_3N - 2 * J), tj_max = two_J_3N + 2 * J;
                for (int tj = tj_min; tj < tj_max + 1; tj += 2) {
                  const int lmin = std::abs(tj - 1) / 2, lmax = (tj + 1) / 2;
                  for (int l = lmin; l < lmax + 1; l++) {
                    if (((L + l) % 2) != par_rem) continue;
                    if (two_T_3N == 3 && !(S == 0 && L == 0 && J == 0)) continue;
                    if (rp.swave_only && (L != 0 || l != 0)) continue;
                    pw.L_2N.push_back(L);
                    pw.S_2N.push_back(S);
                    pw.J_2N.push_back(J);
                    pw.T_2N.push_back(T);
                    pw.L_1N.push_back(l);
                    pw.two_J_1N.push_back(tj);
                    pw.two_J_3N.push_back(two_J_3N);
                    pw.two_T_3N.push_back(two_T_3N);
                    pw.P_3N.push_back(1 - 2 * par_rem);
                    pw.Nalpha += 1;
                    n_in_chn += 1;
                  }
                }
              }
            }
          }
        }
      }
      if (n_in_chn != 0) {
        pw.N_chn_3N += 1;
        pw.chn_3N_idx.push_back(n_prev);
      }
      n_prev = pw.Nalpha;
    }
  }
  pw.chn_3N_idx.push_back(pw.Nalpha);
  return true;
}

PWChannel channel_view(const PWStates& pw, int chn) {
  PWChannel c;
  const int lo = pw.chn_3N_idx[chn], hi = pw.chn_3N_idx[chn + 1];
  c.Nalpha = hi - lo;
  c.J_2N_max = pw.J_2N_max;
  c.L_2N = &pw.L_2N[lo];
  c.S_2N = &pw.S_2N[lo];
  c.J_2N = &pw.J_2N[lo];
  c.T_2N = &pw.T_2N[lo];
  c.L_1N = &pw.L_1N[lo];
  c.two_J_1N = &pw.two_J_1N[lo];
  c.two_J_3N = &pw.two_J_3N[lo];
  c.two_T_3N = &pw.two_T_3N[lo];
  c.P_3N = &pw.P_3N[lo];
  return c;
}

// ---------------------------------------------------------------------------
void chebyshev_boundaries(int n, double* b, double scale, double t) {
  for (int i = 1; i < n + 1; i++) {
    double tan_term = std::tan((2 * i - 1) * M_PI / (4 * n));
    b[i] = scale * std::pow(tan_term, t);
  }
  b[0] = 0.0;
}

bool read_input_list(const std::string& path, RunParams& rp, std::string* err) {
  std::ifstream in(path);
  if (!in) {
    if (err) *err = "cannot open input list " + path;
    return false;
  }
  std::string line;
  while (std::getline(in, line)) {
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;  // lines without '=' are comments
    const std::string key = line.substr(0, eq);
    std::string value = line.substr(eq + 1);
    if (value.find_first_not_of(' ') == std::string::npos) continue;  // empty value: keep the default
    value.erase(std::remove_if(value.begin(), value.end(), [](unsigned char ch) { return std::isspace(ch); }),
                value.end());
    if (!set_run_parameter(rp, key, value, err)) return false;
  }
  return true;
}

// read_WP_boundaries_from_txt (CPP/disk_io_routines.cpp:977-994): one
// boundary per line (the first number of the line), exactly N + 1 lines
static bool read_wp_boundaries(const std::string& path, int N, double* out, std::string* err) {
  std::ifstream in(path);
  if (!in) {
    if (err) *err = "cannot open WP-boundary file " + path;
    return false;
  }
  std::string line;
  int k = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    double v;
    if (!(ls >> v)) {
      if (err) *err = "Unknown format in input WP-boundary file:" + path;
      return false;
    }
    if (k <= N) out[k] = v;
    k++;
  }
  if (k != N + 1) {
    if (err) *err = "Program mismatch with number of wave-packets in input WP-boundaries file";
    return false;
  }
  return true;
}

// make_p_bin_grid / make_q_bin_grid (CPP/make_wp_states.cpp:46-75): Chebyshev
// boundaries or a file; the q grid is read from its file when the P grid
// type is "custom", as there
static bool wp_boundaries(const RunParams& rp, bool is_p, int N, double* b, std::string* err) {
  const std::string& type = is_p ? rp.p_grid_type : rp.q_grid_type;
  if (type == "chebyshev") {
    chebyshev_boundaries(N, b, rp.chebyshev_s, rp.chebyshev_t);
    return true;
  }
  if (rp.p_grid_type == "custom")
    return read_wp_boundaries(is_p ? rp.p_grid_filename : rp.q_grid_filename, N, b, err);
  if (err) *err = is_p ? "Unknown p-momentum gridtype specified." : "Unknown q-momentum gridtype specified.";
  return false;
}

bool make_fwp_states(const RunParams& rp, FWPStates& f, std::string* err) {
  if (rp.Np_WP < 2 || rp.Nq_WP < 2) {
    if (err) *err = "Np_WP and Nq_WP must be >= 2";
    return false;
  }
  f = FWPStates();
  f.Np_WP = rp.Np_WP;
  f.Nq_WP = rp.Nq_WP;
  f.Np_per_WP = rp.Np_per_WP;
  f.Nq_per_WP = rp.Nq_per_WP;
  const int Np = rp.midpoint_approx ? f.Np_WP : f.Np_per_WP * f.Np_WP;
  const int Nq = rp.midpoint_approx ? f.Nq_WP : f.Nq_per_WP * f.Nq_WP;
  f.p_WP.resize(f.Np_WP + 1);
  f.q_WP.resize(f.Nq_WP + 1);
  if (!wp_boundaries(rp, true, f.Np_WP, f.p_WP.data(), err)) return false;
  if (!wp_boundaries(rp, false, f.Nq_WP, f.q_WP.data(), err)) return false;
  f.p.resize(Np);
  f.q.resize(Nq);
  if (rp.midpoint_approx) {
    for (int i = 0; i < Np; i++) f.p[i] = 0.5 * (f.p_WP[i] + f.p_WP[i + 1]);
    for (int i = 0; i < Nq; i++) f.q[i] = 0.5 * (f.q_WP[i] + f.q_WP[i + 1]);
  } else {
    f.wp.resize(Np);
    f.wq.resize(Nq);
    for (int b = 0; b < f.Np_WP; b++) {
      gauss_legendre(&f.p[b * f.Np_per_WP], &f.wp[b * f.Np_per_WP], f.Np_per_WP);
      rescale_rule(&f.p[b * f.Np_per_WP], &f.wp[b * f.Np_per_WP], f.p_WP[b], f.p_WP[b + 1], f.Np_per_WP);
    }
    for (int b = 0; b < f.Nq_WP; b++) {
      gauss_legendre(&f.q[b * f.Nq_per_WP], &f.wq[b * f.Nq_per_WP], f.Nq_per_WP);
      rescale_rule(&f.q[b * f.Nq_per_WP], &f.wq[b * f.Nq_per_WP], f.q_WP[b], f.q_WP[b + 1], f.Nq_per_WP);
    }
  }
  f.fp.assign(Np, 1.0);  // momentum wave packets: weight function 1
  f.fq.assign(Nq, 1.0);
  f.norm_p.resize(f.Np_WP);
  f.norm_q.resize(f.Nq_WP);
  for (int i = 0; i < f.Np_WP; i++) f.norm_p[i] = std::sqrt(f.p_WP[i + 1] - f.p_WP[i]);
  for (int i = 0; i < f.Nq_WP; i++) f.norm_q[i] = std::sqrt(f.q_WP[i + 1] - f.q_WP[i]);
  return true;
}

void count_2N_channels(const RunParams& rp, int& n_unco, int& n_coup) {
  n_unco = 0;
  n_coup = 0;
  if (rp.tensor_force) {
    n_unco = 2 * (rp.J_2N_max + 1);
    n_coup = rp.J_2N_max;
    if (rp.isospin_breaking_1S0) {
      n_unco -= 1;
      n_coup += 1;
    }
  } else {
    n_unco = 4 * rp.J_2N_max + 2;
    if (rp.isospin_breaking_1S0) {
      n_unco -= 1;
      n_coup = 1;
    }
  }
}

// ---------------------------------------------------------------------------
double mu1(double Eb) {
  const double Md = kMn + kMp + Eb;
  return kMn * Md / (kMn + Md);
}
double com_momentum_to_lab_energy(double q_com, double Eb) {
  const double Md = kMn + kMp + Eb;
  const double b = 2 * (kMp - q_com * q_com / Md);
  const double c = -q_com * q_com * (kMp + Md) * (kMp + Md) / (Md * Md);
  return 0.5 * (-b + std::sqrt(b * b - 4 * c));
}
double lab_energy_to_com_momentum(double T_lab, double Eb) {
  const double Md = kMn + kMp + Eb;
  return std::sqrt(Md * Md * T_lab * (T_lab + 2 * kMp) / ((kMp + Md) * (kMp + Md) + 2 * T_lab * Md));
}
double com_energy_to_com_q_momentum(double E_com) { return std::sqrt(4 * E_com * kMN / 3); }
double com_q_momentum_to_com_energy(double q_com) { return 3 * q_com * q_com / (4 * kMN); }

bool find_on_shell_bins(const RunParams& rp, const SWPStates& swp, OnShell& os, std::string* err) {
  const int Nq = swp.Nq_WP;
  const double Eb = swp.E_bound;
  const double* qb = swp.q_WP.data();
  std::vector<double> energies = rp.lab_energies;
  if (energies.empty()) {
    if (!read_input_energies(rp.energy_input_file, energies, err)) return false;
  }
  std::vector<double> T_mid(Nq);
  for (int i = 0; i < Nq; i++) {
    const double El = 0.5 * (qb[i] * qb[i]) / mu1(Eb);
    const double Eu = 0.5 * (qb[i + 1] * qb[i + 1]) / mu1(Eb);
    const double Ec = 0.5 * (Eu + El);
    T_mid[i] = com_momentum_to_lab_energy(com_energy_to_com_q_momentum(Ec), Eb);
  }
  std::vector<bool> mid_hit(Nq - 1, false);
  for (int i = 0; i < Nq - 1; i++)
    for (double T : energies)
      if (T_mid[i] <= T && T <= T_mid[i + 1]) mid_hit[i] = true;
  std::vector<bool> bin_hit(Nq, false);
  for (int i = 0; i < Nq - 1; i++)
    if (mid_hit[i]) bin_hit[i] = bin_hit[i + 1] = true;
  os = OnShell();
  std::vector<int> bins;
  for (int i = 0; i < Nq; i++)
    if (bin_hit[i]) bins.push_back(i);
  for (int b : bins) {
    const double El = 0.5 * (qb[b] * qb[b]) / mu1(Eb);
    const double Eu = 0.5 * (qb[b + 1] * qb[b + 1]) / mu1(Eb);
    const double Ec = 0.5 * (Eu + El);
    os.T_lab.push_back(com_momentum_to_lab_energy(com_energy_to_com_q_momentum(Ec), Eb));
  }
  for (double T : os.T_lab) {
    const double q = lab_energy_to_com_momentum(T, Eb);
    os.q_com.push_back(q);
    os.E_com.push_back(com_q_momentum_to_com_energy(q));
  }
  for (size_t k = 0; k < os.q_com.size(); k++) {
    int idx = -1;
    for (int i = 0; i < Nq; i++) {
      if (qb[i] < os.q_com[k] && os.q_com[k] < qb[i + 1]) {
        idx = i;
        break;
      }
    }
    if (idx == -1) {
      if (err) *err = "Invalid Tlab entered: on-shell energy outside the WP state space";
      return false;
    }
    os.q_com_idx.push_back(idx);
  }
  return true;
}

std::vector<int> deuteron_indices(const PWChannel& ch) {
  std::vector<int> d;
  for (int a = 0; a < ch.Nalpha; a++)
    if (ch.L_2N[a] == 0 && ch.S_2N[a] == 1 && ch.J_2N[a] == 1 && ch.T_2N[a] == 0) d.push_back(a);
  return d;
}

}  // namespace tt
