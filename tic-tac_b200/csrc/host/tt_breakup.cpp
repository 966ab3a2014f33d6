// Breakup channels of the elastic solve: the on-shell (alpha, q, p) cells of
// each energy (CPP/run_organizer.cpp:134-339) and the text table of their
// U elements (restructure_breakup_data + store_U_BU_matrix_elements_txt,
// CPP/disk_io_routines.cpp:341-706).  The amplitudes themselves come from
// the Pade solve on the device (ChannelSolver::solve_pade).
#include <algorithm>
#include <cmath>
#include <iomanip>
#include <map>
#include <sstream>

#include "tt_breakup.h"
#include "tt_solver.h"

namespace tt {

double mu1_free() {
  const double M12 = kMp + kMn;
  return kMn * M12 / (kMn + M12);
}

double com_energy_to_com_p_momentum(double Ep) { return std::sqrt(2 * Ep * kMu23); }

bool find_breakup_cells(const RunParams& rp, const PWChannel& ch, const SWPStates& swp,
                        const std::vector<double>& E_com, BreakupCells& bu, std::string* err) {
  const int Na = ch.Nalpha, Np = swp.Np_WP, Nq = swp.Nq_WP;
  bu = BreakupCells();
  bu.start.push_back(0);
  if (Na == 0) {
    bu.start.assign(E_com.size() + 1, 0);
    return true;
  }
  // each alpha's SWP energy boundaries: the pair's own 2N block, the part of a
  // coupled block chosen as for the resolvent (run_organizer.cpp:161-203)
  std::vector<int32_t> e_off(Na);
  if (!channel_energy_offsets(rp, ch, Np, swp.n_unco, swp.n_coup, e_off.data(), err)) return false;
  std::vector<double> e_swp = swp.e_unco;
  e_swp.insert(e_swp.end(), swp.e_coup.begin(), swp.e_coup.end());
  const double* q = swp.q_WP.data();
  const double mu = mu1_free();
  auto push = [&](int a, int qb, int pb) {
    bu.cells.push_back(a);
    bu.cells.push_back(qb);
    bu.cells.push_back(pb);
  };
  for (const double E : E_com) {
    if (E + swp.E_bound < 0) {  // below the breakup threshold
      bu.start.push_back((int32_t)bu.count());
      continue;
    }
    bool found = false;
    for (int a = 0; a < Na; a++) {
      const double* e = &e_swp[e_off[a]];
      for (int qi = 0; qi < Nq; qi++) {
        const double Eql = 0.5 * (q[qi] * q[qi]) / mu;
        const double Equ = 0.5 * (q[qi + 1] * q[qi + 1]) / mu;
        for (int pi = 0; pi < Np; pi++) {
          const double Epl = e[pi], Epu = e[pi + 1];
          const double Ecl = Epl + Eql, Ecu = Epu + Equ;
          if (!(Ecl <= E && E <= Ecu && Epl >= 0 && Epu >= 0)) continue;
          found = true;
          push(a, qi, pi);
          // the cell's quadrants by its mid-point energies; the first whose
          // energy range holds E picks the three neighbours (p, q) to add
          const double Ep = 0.5 * (Epu + Epl), Eq = 0.5 * (Equ + Eql);
          int p0, q0;
          if (Eq + Ep <= E && E <= Ecu) {
            p0 = pi;
            q0 = qi;
          } else if (Eq + Epl <= E && E <= Ep + Equ) {
            p0 = pi - 1;
            q0 = qi;
          } else if (Ecl <= E && E <= Eq + Ep) {
            p0 = pi - 1;
            q0 = qi - 1;
          } else if (Eql + Ep <= E && E <= Epu + Eq) {
            p0 = pi;
            q0 = qi - 1;
          } else {
            continue;
          }
          for (int p2 = p0; p2 <= p0 + 1; p2++)
            for (int q2 = q0; q2 <= q0 + 1; q2++)
              if (p2 != pi || q2 != qi) push(a, q2, p2);
        }
      }
    }
    if (!found) {
      if (err) *err = "Invalid Tlab entered: breakup on-shell energy " + std::to_string(E) +
                      " MeV outside the WP state space";
      return false;
    }
    bu.start.push_back((int32_t)bu.count());
  }
  return true;
}

std::string signed_scientific(double v) {
  std::ostringstream o;
  o.precision(16);
  if (v >= 0) o << "+";
  o << std::scientific << v;
  return o.str();
}

bool write_breakup_table(std::ostream& f, const BreakupTableInput& in, std::string* err) {
  const PWChannel& c = in.ch;
  const int Na = c.Nalpha, Np = in.swp->Np_WP, Nq = in.swp->Nq_WP;
  const BreakupCells& bu = *in.bu;
  const size_t nE = in.os->q_com_idx.size(), nd = in.deut.size(), nb = (size_t)bu.count();
  if (bu.start.size() != nE + 1) {
    if (err) *err = "breakup cells do not match the run's energies";
    return false;
  }
  std::vector<int32_t> e_off(std::max(Na, 1));
  if (Na && !channel_energy_offsets(*in.rp, c, Np, in.swp->n_unco, in.swp->n_coup, e_off.data(), err)) return false;
  std::vector<double> e_swp = in.swp->e_unco;
  e_swp.insert(e_swp.end(), in.swp->e_coup.begin(), in.swp->e_coup.end());
  const std::vector<double>& qWP = in.swp->q_WP;

  // columns: five per energy row, then five per (alpha', alpha) pair in order
  // of first appearance; rows: per energy, one per cell of each pair
  // (disk_io_routines.cpp:387-459)
  struct Col {
    bool comp;
    std::string name;
  };
  std::vector<Col> head = {{false, "Tlab [MeV]"},
                           {false, "Ecm [MeV]"},
                           {false, "qcm [MeV] (init.)"},
                           {false, "qlo [MeV] (init.)"},
                           {false, "qup [MeV] (init.)"}};
  std::map<long long, int> alpha_col;  // alpha' * Nalpha + alpha -> pair index
  std::map<long long, int> row_of;     // cell * Nalpha + alpha -> row
  std::vector<int> rows_at = {0};      // first row of each energy; the last entry is the row count
  for (size_t j = 0; j < nE; j++) {
    std::map<long long, int> next_row;  // pair -> next row of this energy
    for (size_t d = 0; d < nd; d++) {
      const int ar = in.deut[d];
      for (int b = bu.start[j]; b < bu.start[j + 1]; b++) {
        const int ac = bu.cells[(size_t)3 * b];
        const long long key = (long long)ac * Na + ar, key_row = (long long)b * Na + ar;
        if (!alpha_col.count(key)) {
          const std::string label = "<" + std::to_string(c.L_2N[ac]) + "," + std::to_string(c.S_2N[ac]) + "," +
                                    std::to_string(c.J_2N[ac]) + "," + std::to_string(c.L_1N[ac]) + "," +
                                    std::to_string(c.two_J_1N[ac]) + "|U|" + std::to_string(c.L_1N[ar]) + "," +
                                    std::to_string(c.two_J_1N[ar]) + ">";
          head.push_back({true, label});
          head.push_back({false, "qlo [MeV]"});
          head.push_back({false, "qup [MeV]"});
          head.push_back({false, "plo [MeV]"});
          head.push_back({false, "pup [MeV]"});
          const int k = (int)alpha_col.size();
          alpha_col[key] = k;
        }
        auto it = next_row.find(key);
        if (it == next_row.end()) {
          row_of[key_row] = rows_at[j];
          next_row[key] = rows_at[j] + 1;
        } else {
          row_of[key_row] = it->second;
          it->second += 1;
        }
      }
    }
    // the energy's last row; an energy without cells reports 0, as there
    int last = 0;
    for (const auto& kv : next_row) last = std::max(last, kv.second);
    rows_at.push_back(last);
  }
  // rows_at is non-decreasing here (energies ascend, so those below the
  // threshold come first); the maximum keeps every row index in the table
  const int n_rows = *std::max_element(rows_at.begin(), rows_at.end()), n_cols = (int)head.size();
  std::vector<double> re((size_t)n_rows * n_cols, 0.0), im((size_t)n_rows * n_cols, 0.0);
  const double nan = std::nan("");
  auto at = [&](int r, int col) -> size_t { return (size_t)r * n_cols + col; };
  for (size_t j = 0; j < nE; j++) {
    const int qj = in.os->q_com_idx[j];
    for (int r = rows_at[j]; r < rows_at[j + 1]; r++) {
      re[at(r, 0)] = in.os->T_lab[j];
      re[at(r, 1)] = in.os->E_com[j];
      re[at(r, 2)] = in.os->q_com[j];
      re[at(r, 3)] = qWP[qj];
      re[at(r, 4)] = qWP[qj + 1];
    }
    for (size_t d = 0; d < nd; d++) {
      const int ar = in.deut[d];
      for (int b = bu.start[j]; b < bu.start[j + 1]; b++) {
        const int ac = bu.cells[(size_t)3 * b], qb = bu.cells[(size_t)3 * b + 1], pb = bu.cells[(size_t)3 * b + 2];
        const long long key = (long long)ac * Na + ar, key_row = (long long)b * Na + ar;
        const int col = 5 * alpha_col[key] + 5, r = row_of[key_row];
        const double* e = &e_swp[e_off[ac]];
        // boundaries outside the grid (an edge cell's neighbour) have no value
        auto qv = [&](int i) { return i >= 0 && i <= Nq ? qWP[i] : nan; };
        auto pv = [&](int i) { return i >= 0 && i <= Np ? com_energy_to_com_p_momentum(e[i]) : nan; };
        const size_t u = d * nb + (size_t)b;
        re[at(r, col)] = in.U_BU[2 * u];
        im[at(r, col)] = in.U_BU[2 * u + 1];
        re[at(r, col + 1)] = qv(qb);
        re[at(r, col + 2)] = qv(qb + 1);
        re[at(r, col + 3)] = pv(pb);
        re[at(r, col + 4)] = pv(pb + 1);
      }
    }
  }

  // store_U_BU_matrix_elements_txt (disk_io_routines.cpp:566-706)
  f << std::setprecision(8);
  f << "# Breakup Nd-scattering U-matrix elements in a wave-packet, Jj-scheme representation. \n";
  f << "# \n";
  f << "# The calculations below were done for: \n";
  f << "# JP:          " << c.two_J_3N[0] << "/2" << (c.P_3N[0] == 1 ? "+" : "-") << "\n";
  f << "# Potential:   " << in.rp->potential_model << "\n";
  f << "# Np:          " << Np << " \n";
  f << "# Nq:          " << Nq << " \n";
  f << "# Particles:   nd-scattering\n";
  f << "# Deuteron BE: " << in.swp->E_bound << " MeV \n";
  f << "# \n";
  f << "# Symbol definitions: \n";
  f << "# <L,S,J,2*l,2*j|U|2*l,2*j>:   U-matrix element in MeV with for channel <L S J l j|U|L=0 S=1 J=1 l j> "
       "(NOTE in wave-packet representation!)  \n";
  static const char* const kSymbols[][2] = {
      {"L:", "Pair orbital angular momentum"},
      {"S:", "Pair spin"},
      {"J:", "Pair total angular momentum"},
      {"l:", "Spectator orbital angular momentum"},
      {"j:", "Spectator total angular momentum"},
      {"Tlab:", "Laboratory scattering/kinetic energy"},
      {"Ecm:", "Centre-of-mass scattering/kinetic energy"},
      {"qcm:", "Spectator centre-of-mass momentum bin midpoint "},
      {"qlo:", "Spectator centre-of-mass momentum bin lower boundary "},
      {"qup:", "Spectator centre-of-mass momentum bin upper boundary "},
      {"plo:", "Pair centre-of-mass momentum bin lower boundary "},
      {"pup:", "Pair centre-of-mass momentum bin upper boundary "},
      {"init.:", "Pre-scattering "}};
  for (const auto& s : kSymbols) {
    std::string tag = s[0];
    tag.resize(29, ' ');
    std::string text = s[1];
    if (text.back() != ' ') text += "  ";
    f << "# " << tag << text << "\n";
  }
  f << "# \n";
  f << "# ################################################################################################### \n";
  f << std::right << std::scientific << std::setprecision(16);
  f << "#";
  for (const Col& h : head) f << std::right << std::setw(h.comp ? 50 : 24) << h.name;
  f << "\n";
  for (int r = 0; r < n_rows; r++) {
    f << " ";
    for (int col = 0; col < n_cols; col++) {
      if (head[col].comp)
        f << std::right << std::setw(50) << (signed_scientific(re[at(r, col)]) + signed_scientific(im[at(r, col)]) + "j");
      else
        f << std::right << std::setw(24) << re[at(r, col)];
    }
    f << "\n";
  }
  f << "# ################################################################################################### \n";
  f << std::endl;
  return true;
}

}  // namespace tt
