// Driver for the reference build (oracle/_ref/tictac_ref).  Replaces
// CPP/main.cpp: runs the reference's own routines for state-space setup,
// P123, resolvent and the dense LAPACK Faddeev solve, and writes every stage
// as raw binary arrays so the tests can compare them with the GPU path.
//
//   tictac_ref dump <outdir> [--solver=reference|replica|pade] key=value ...
//   tictac_ref time <outdir> [--channel=k] [--sample_cols=m] [--repeat=r] key=value ...
//
// --channel=k also restricts dump to channel k.
//   tictac_ref info <outdir> key=value ...
//
// time: the dense solve of the selected channel (A columns once, then per
// energy L = 1 - A G, R = A and zgetrf + zgetrs with nrhs = n) repeated r
// times after one set-up, one "step" line per repetition in meta.txt; the
// first repetition also times the fair variant (zgetrs on the on-shell
// right-hand sides only).  info: the channels' sizes, energies and deuteron
// states from the state-space set-up alone (no P123, no solve).
//
// Extra keys understood here (stripped before the reference's parser sees them):
//   swave_only=true   apply the reference's commented-out s-wave filter
//                     (make_pw_symm_states.cpp:176-179) to the basis
//   lab_energies=a,b  write the energies to <outdir>/lab_energies.txt
//
// Parity-oracle infrastructure only.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "General_functions/kinetic_conversion.h"
#include "General_functions/matrix_routines.h"
#include "Interactions/potential_model.h"
#include "constants.h"
#include "disk_io_routines.h"
#include "make_permutation_matrix.h"
#include "make_potential_matrix.h"
#include "make_pw_symm_states.h"
#include "make_resolvent.h"
#include "make_swp_states.h"
#include "make_wp_states.h"
#include "run_organizer.h"
#include "set_run_parameters.h"
#include "solve_faddeev.h"

// defined in CPP/solve_faddeev.cpp without a header declaration
void calculate_CPVC_col(double* col_array, int* row_to_nnz_array, int* nnz_to_row_array, size_t& num_nnz,
                        size_t idx_alpha_c, size_t idx_p_c, size_t idx_q_c, size_t Nalpha, size_t Nq_WP,
                        size_t Np_WP, double** CT_RM_array, double** VC_CM_array, double* P123_val_array,
                        int* P123_row_array, size_t* P123_col_array, size_t P123_dim);

static std::string g_out;

template <typename T>
static void dump(const std::string& name, const T* data, size_t count) {
  std::ofstream o(g_out + "/" + name + ".bin", std::ios::binary | std::ios::trunc);
  o.write((const char*)data, sizeof(T) * count);
}

static void filter_swave(pw_3N_statespace& pw) {
  // the reference's s-wave filter, applied after enumeration
  std::vector<int> keep;
  for (int a = 0; a < pw.Nalpha; a++)
    if (pw.L_2N_array[a] == 0 && pw.L_1N_array[a] == 0) keep.push_back(a);
  std::vector<int> chn_new;
  std::vector<int> chn_of(pw.Nalpha);
  for (int c = 0; c < pw.N_chn_3N; c++)
    for (int a = pw.chn_3N_idx_array[c]; a < pw.chn_3N_idx_array[c + 1]; a++) chn_of[a] = c;
  int* arrays[9] = {pw.L_2N_array, pw.S_2N_array, pw.J_2N_array, pw.T_2N_array, pw.L_1N_array,
                    pw.two_J_1N_array, pw.two_J_3N_array, pw.two_T_3N_array, pw.P_3N_array};
  int prev_chn = -1, count = 0;
  for (size_t i = 0; i < keep.size(); i++) {
    const int a = keep[i];
    for (int k = 0; k < 9; k++) arrays[k][i] = arrays[k][a];
    if (chn_of[a] != prev_chn) {
      chn_new.push_back((int)i);
      prev_chn = chn_of[a];
    }
    count++;
  }
  chn_new.push_back(count);
  pw.Nalpha = count;
  pw.N_chn_3N = (int)chn_new.size() - 1;
  for (size_t i = 0; i < chn_new.size(); i++) pw.chn_3N_idx_array[i] = chn_new[i];
}

static pw_3N_statespace substates(const pw_3N_statespace& pw, int chn) {
  const int lo = pw.chn_3N_idx_array[chn], hi = pw.chn_3N_idx_array[chn + 1];
  pw_3N_statespace s = pw;
  s.Nalpha = hi - lo;
  s.L_2N_array = &pw.L_2N_array[lo];
  s.S_2N_array = &pw.S_2N_array[lo];
  s.J_2N_array = &pw.J_2N_array[lo];
  s.T_2N_array = &pw.T_2N_array[lo];
  s.L_1N_array = &pw.L_1N_array[lo];
  s.two_J_1N_array = &pw.two_J_1N_array[lo];
  s.two_T_3N_array = &pw.two_T_3N_array[lo];
  s.two_J_3N_array = &pw.two_J_3N_array[lo];
  s.P_3N_array = &pw.P_3N_array[lo];
  return s;
}

// Dense A = C^T (2 P123) (V C) column by column with the reference's own
// calculate_CPVC_col (solve_faddeev.cpp:50-181); row-major n x n.
static void build_A(std::vector<double>& A, size_t Nalpha, size_t Nq, size_t Np, double** CT, double** VC,
                    double* val, int* row, size_t* colptr, size_t nnz) {
  const size_t n = Nalpha * Nq * Np;
  A.assign(n * n, 0.0);
#pragma omp parallel
  {
    std::vector<double> col(n);
    std::vector<int> r2n(n), n2r(n);
#pragma omp for schedule(dynamic)
    for (size_t c = 0; c < n; c++) {
      const size_t ac = c / (Nq * Np), qc = (c / Np) % Nq, pc = c % Np;
      std::fill(col.begin(), col.end(), 0.0);
      size_t nn = 0;
      calculate_CPVC_col(col.data(), r2n.data(), n2r.data(), nn, ac, pc, qc, Nalpha, Nq, Np, CT, VC, val, row, colptr,
                         nnz);
      for (size_t r = 0; r < n; r++) A[r * n + c] = col[r];
    }
  }
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: tictac_ref dump|time <outdir> [options] key=value ...\n");
    return 2;
  }
  const std::string mode = argv[1];
  g_out = argv[2];
  std::string solver = "reference";
  int time_channel = -1;
  long sample_cols = -1;
  int repeat = 1;
  bool swave = false;
  std::vector<std::string> keep_args = {"tictac_ref"};
  std::string energies;
  for (int i = 3; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--solver=", 0) == 0) solver = a.substr(9);
    else if (a.rfind("--channel=", 0) == 0) time_channel = std::atoi(a.c_str() + 10);
    else if (a.rfind("--sample_cols=", 0) == 0) sample_cols = std::atol(a.c_str() + 14);
    else if (a.rfind("--repeat=", 0) == 0) repeat = std::max(1, std::atoi(a.c_str() + 9));
    else if (a == "swave_only=true") swave = true;
    else if (a == "swave_only=false") swave = false;
    else if (a.rfind("lab_energies=", 0) == 0) energies = a.substr(13);
    else keep_args.push_back(a);
  }
  if (!energies.empty()) {
    std::ofstream e(g_out + "/lab_energies.txt");
    for (char& ch : energies)
      if (ch == ',') ch = '\n';
    e << energies << "\n";
    keep_args.push_back("energy_input_file=" + g_out + "/lab_energies.txt");
  }
  keep_args.push_back("output_folder=" + g_out);
  keep_args.push_back("P123_folder=" + g_out);
  // --solver=pade runs the reference's default production path (Pade-resummed
  // Neumann series, solve_faddeev.cpp:440-1444) through its own dispatcher
  keep_args.push_back(solver == "pade" ? "solve_dense=false" : "solve_dense=true");
  std::vector<char*> av;
  for (auto& s : keep_args) av.push_back(&s[0]);
  int ac = (int)av.size();
  run_params rp;
  set_run_parameters(ac, av.data(), rp);

  pw_3N_statespace pw;
  construct_symmetric_pw_states(pw, rp);
  if (swave) filter_swave(pw);
  fwp_statespace fwp;
  make_fwp_statespace(fwp, rp);
  potential_model* pot = potential_model::fetch_potential_ptr(rp);

  int n_unco = 0, n_coup = 0;  // CPP/main.cpp:273-289
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
  const int Np = rp.Np_WP, Nq = rp.Nq_WP;
  const size_t Vu_n = (size_t)Np * Np * n_unco, Vc_n = rp.tensor_force ? (size_t)Np * Np * 4 * n_coup : 0;
  std::vector<double> Vu(Vu_n + 1), Vc(Vc_n + 1), Cu(Vu_n + 1), Cc(Vc_n + 1);
  std::vector<double> eu((size_t)(Np + 1) * n_unco + 1), ec((size_t)2 * (Np + 1) * n_coup + 1);
  calculate_potential_matrices_array_in_WP_basis(Vu.data(), n_unco, Vc.data(), n_coup, fwp, pw, pot, rp);
  double E_bound = 0;
  swp_statespace swp;
  make_swp_states(eu.data(), ec.data(), Cu.data(), Cc.data(), Vu.data(), Vc.data(), n_unco, n_coup, E_bound, fwp, swp,
                  pw, rp);

  dump("p_WP", fwp.p_WP_array, Np + 1);
  dump("q_WP", fwp.q_WP_array, Nq + 1);
  dump("V_unco", Vu.data(), Vu_n);
  dump("V_coup", Vc.data(), Vc_n);
  dump("C_unco", Cu.data(), Vu_n);
  dump("C_coup", Cc.data(), Vc_n);
  dump("e_unco", eu.data(), (size_t)(Np + 1) * n_unco);
  dump("e_coup", ec.data(), (size_t)2 * (Np + 1) * n_coup);

  solution_configuration cfg;
  cfg.deuteron_idx_arrays = new int*[pw.N_chn_3N];
  cfg.deuteron_num_array = new int[pw.N_chn_3N];
  std::ofstream meta(g_out + "/meta.txt");
  meta.precision(17);
  meta << "E_bound " << swp.E_bound << "\nn_chn " << pw.N_chn_3N << "\n";

  for (int chn = 0; chn < pw.N_chn_3N; chn++) {
    if ((mode == "time" || mode == "dump") && time_channel >= 0 && chn != time_channel) continue;
    pw_3N_statespace sub = substates(pw, chn);
    const size_t n = (size_t)sub.Nalpha * Nq * Np;
    std::vector<int> pwtab;
    for (int a = 0; a < sub.Nalpha; a++) {
      const int v[9] = {sub.L_2N_array[a], sub.S_2N_array[a], sub.J_2N_array[a], sub.T_2N_array[a],
                        sub.L_1N_array[a], sub.two_J_1N_array[a], sub.two_J_3N_array[a], sub.two_T_3N_array[a],
                        sub.P_3N_array[a]};
      pwtab.insert(pwtab.end(), v, v + 9);
    }
    const std::string tag = "_c" + std::to_string(chn);
    if (mode == "info") {
      channel_os_indexing os;
      find_on_shell_bins(cfg, os, sub, fwp, swp, rp);
      find_deuteron_channels(cfg, pw);
      meta << "chn " << chn << " Nalpha " << sub.Nalpha << " n " << n << " nE " << cfg.num_T_lab << " nd "
           << cfg.deuteron_num_array[chn] << "\n";
      continue;
    }
    dump("pw" + tag, pwtab.data(), pwtab.size());

    auto t0 = std::chrono::steady_clock::now();
    double* val = nullptr;
    int *row = nullptr, *col = nullptr;
    size_t nnz = 0;
    fill_P123_arrays(&val, &row, &col, nnz, rp.production_run, fwp, sub, rp, rp.P123_folder);
    const double t_p123 = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    dump("p123_row" + tag, row, nnz);
    dump("p123_col" + tag, col, nnz);
    dump("p123_val" + tag, val, nnz);
    unsorted_sparse_to_coo_col_major_sorter(&val, &row, &col, nnz, n);
    std::vector<size_t> colptr(n + 1);
    coo_to_csc_format_converter(col, colptr.data(), nnz, n);

    channel_os_indexing os;
    find_on_shell_bins(cfg, os, sub, fwp, swp, rp);
    find_deuteron_channels(cfg, pw);
    os.num_T_lab = cfg.num_T_lab;
    os.q_com_idx_array = cfg.q_com_idx_array;
    os.num_deuteron_states = cfg.deuteron_num_array[chn];
    os.deuteron_idx_array = cfg.deuteron_idx_arrays[chn];
    const size_t nE = os.num_T_lab, nd = os.num_deuteron_states;
    meta << "chn " << chn << " Nalpha " << sub.Nalpha << " n " << n << " nnz " << nnz << " nE " << nE << " nd " << nd
         << " t_p123 " << t_p123 << "\n";
    if (chn == 0 || (mode == "time")) {
      meta << "energies";
      for (size_t j = 0; j < nE; j++)
        meta << " " << cfg.T_lab_array[j] << " " << cfg.E_com_array[j] << " " << cfg.q_com_idx_array[j];
      meta << "\n";
    }
    std::vector<cdouble> G(n * nE);
    for (size_t j = 0; j < nE; j++)
      calculate_resolvent_array_in_SWP_basis(&G[j * n], cfg.E_com_array[j] + swp.E_bound, swp, sub, rp);
    dump("G" + tag, G.data(), G.size());

    std::vector<cdouble> U(nE * nd * nd + 1);
    if (mode == "dump" && (solver == "reference" || solver == "pade")) {
      // include_breakup_channels=true: the breakup cells find_on_shell_bins
      // located (run_organizer.cpp:136-339) and their Pade amplitudes
      // (solve_faddeev.cpp:867-890, 1176-1205, 1299-1407), U_BU[d*num_BU + b];
      // main.cpp:416-419 allocates num_T_lab * num_BU, the larger size is taken here
      std::vector<cdouble> U_BU;
      const size_t nbu = rp.include_breakup_channels ? (size_t)os.num_BU_chns : 0;
      if (rp.include_breakup_channels) U_BU.assign(std::max(nE, nd) * nbu + 1, cdouble(0.0, 0.0));
      solve_faddeev_equations(U.data(), rp.include_breakup_channels ? U_BU.data() : nullptr, G.data(), val, row,
                              colptr.data(), nnz, Vu.data(), Vc.data(), swp, os, sub, "_ref", rp);
      if (rp.include_breakup_channels) {
        dump("bu_start" + tag, os.q_com_BU_idx_array, nE + 1);
        dump("bu_cells" + tag, os.alphapq_idx_array, 3 * nbu);
        dump("U_BU" + tag, U_BU.data(), nd * nbu);
        store_U_BU_matrix_elements_txt(U_BU.data(), cfg, os, rp, fwp, swp, sub, g_out + "/U_BU" + tag + ".txt");
      }
    } else {
      // the dense solver's steps (solve_faddeev.cpp:305-438) without its text dumps
      double** CT = new double*[sub.Nalpha * sub.Nalpha];
      double** VC = new double*[sub.Nalpha * sub.Nalpha];
      create_CT_row_maj_3N_pointer_array(CT, Cu.data(), Cc.data(), n_unco, n_coup, Np, sub, rp);
      create_VC_col_maj_3N_pointer_array(VC, Cu.data(), Cc.data(), Vu.data(), Vc.data(), n_unco, n_coup, Np, sub, rp);
      std::vector<double> A;
      auto ta = std::chrono::steady_clock::now();
      if (mode == "time" && sample_cols > 0 && (size_t)sample_cols < n) {
        // bounded sample of the A-column generation
        std::vector<double> colv(n);
        std::vector<int> r2n(n), n2r(n);
        for (long c = 0; c < sample_cols; c++) {
          size_t cc = (size_t)c * (n / sample_cols), nn = 0;
          std::fill(colv.begin(), colv.end(), 0.0);
          calculate_CPVC_col(colv.data(), r2n.data(), n2r.data(), nn, cc / (Nq * Np), cc % Np, (cc / Np) % Nq,
                             sub.Nalpha, Nq, Np, CT, VC, val, row, colptr.data(), nnz);
        }
        const double t_cols = std::chrono::duration<double>(std::chrono::steady_clock::now() - ta).count();
        meta << "timing chn " << chn << " n " << n << " sample_cols " << sample_cols << " t_cols " << t_cols << "\n";
        continue;
      }
      build_A(A, sub.Nalpha, Nq, Np, CT, VC, val, row, colptr.data(), nnz);
      const double t_A = std::chrono::duration<double>(std::chrono::steady_clock::now() - ta).count();
      if (mode == "dump" && n <= 4096) dump("A" + tag, A.data(), A.size());
      std::vector<cdouble> L(n * n), R(n * n);
      double t_lu = 0, t_fair = 0;
      for (int rep = 0; rep < (mode == "time" ? repeat : 1); rep++) {
      const auto ts = std::chrono::steady_clock::now();
      const double t_lu0 = t_lu;
      for (size_t j = 0; j < nE; j++) {
        for (size_t r = 0; r < n; r++)
          for (size_t c = 0; c < n; c++) {
            L[r * n + c] = -A[r * n + c] * G[j * n + c];
            R[r * n + c] = A[r * n + c];
          }
        for (size_t c = 0; c < n; c++) L[c * n + c] += 1;
        std::vector<cdouble> Lcopy;
        if (mode == "time") Lcopy = L;
        auto tl = std::chrono::steady_clock::now();
        solve_MM(L.data(), R.data(), (int)n);  // zgetrf + zgetrs(nrhs = n), matrix_routines.cpp:73-80
        t_lu += std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
        if (mode == "time" && rep == 0) {
          // fair variant: zgetrf + zgetrs with only the on-shell right-hand sides
          std::vector<cdouble> B(n * nd);
          std::vector<long long> piv(n);
          auto tf = std::chrono::steady_clock::now();
          LAPACKE_zgetrf(LAPACK_ROW_MAJOR, n, n, Lcopy.data(), n, piv.data());
          for (size_t r = 0; r < n; r++)
            for (size_t d = 0; d < nd; d++)
              B[r * nd + d] = A[r * n + os.deuteron_idx_array[d] * Nq * Np + os.q_com_idx_array[j] * Np];
          LAPACKE_zgetrs(LAPACK_ROW_MAJOR, 'N', n, nd, Lcopy.data(), n, piv.data(), B.data(), nd);
          t_fair += std::chrono::duration<double>(std::chrono::steady_clock::now() - tf).count();
        }
        for (size_t dr = 0; dr < nd; dr++)
          for (size_t dc = 0; dc < nd; dc++) {
            const size_t rr = os.deuteron_idx_array[dr] * Nq * Np + os.q_com_idx_array[j] * Np;
            const size_t cc = os.deuteron_idx_array[dc] * Nq * Np + os.q_com_idx_array[j] * Np;
            U[dr * nd * nE + dc * nE + j] = R[rr * n + cc];
          }
      }
      if (mode == "time") {
        // one step: every energy's L/R formation and solve (the fair variant's time excluded)
        const double t_step =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count() - (rep == 0 ? t_fair : 0.0);
        meta << "step " << rep << " t " << t_step << " t_lu " << (t_lu - t_lu0) << "\n";
        meta.flush();
      }
      }
      meta << "timing chn " << chn << " n " << n << " t_A " << t_A << " t_getrf_getrs " << t_lu << " t_fair " << t_fair
           << " threads " << omp_get_max_threads() << "\n";
      delete[] CT;
      delete[] VC;
    }
    dump("U" + tag, U.data(), nE * nd * nd);
    if (mode == "dump")  // the reference's own elastic table of this U (disk_io_routines.cpp:759-913)
      store_U_matrix_elements_txt(U.data(), cfg, os, rp, swp, sub, g_out + "/U_table" + tag + ".txt");
    meta.flush();
    delete[] val;
    delete[] row;
    delete[] col;
  }
  meta.close();
  return 0;
}
