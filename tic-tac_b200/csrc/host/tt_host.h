// Host-side (FP64) state-space setup for the WPCD solve: run parameters,
// 3N partial-wave basis, free wave-packet grids, 2N potential in the WP basis,
// scattering wave packets and on-shell indexing.  These are the inputs the
// three device stages (P123, resolvent, Faddeev solve) consume; parity of the
// device stages depends on them bit-for-bit, so each function restates the
// reference routine it cites with the same arithmetic.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace tt {

// Physical constants, CPP/constants.h:13-35.
constexpr double kMp = 938.272;
constexpr double kMn = 939.565;
constexpr double kMN = 0.5 * (kMp + kMn);
constexpr double kMu23 = kMp * kMn / (kMn + kMp);
constexpr double kHbarc = 197.327;
constexpr double kLambdaLO = 450;
constexpr double kGA = 1.289;
constexpr double kFpi = 92.2;
constexpr double kMpi = 138.039;
constexpr double kC1S0 = -0.112927 / 100.;
constexpr double kC3S1 = -0.087340 / 100.;

// Argument surface of CPP/set_run_parameters.cpp (defaults :577-615) plus the
// keys this implementation adds (swave_only, precision, tolerances).
struct RunParams {
  int two_J_3N_max = 1;
  int Np_WP = 50;
  int Nq_WP = 50;
  int J_2N_max = 3;
  int Nphi = 48;
  int Nx = 48;
  int Np_per_WP = 8;
  int Nq_per_WP = 8;
  int channel_idx = -1;
  double chebyshev_t = 1;
  double chebyshev_s = 100;
  bool parallel_run = false;
  bool tensor_force = true;
  bool isospin_breaking_1S0 = true;
  bool midpoint_approx = false;
  bool calculate_and_store_P123 = true;
  bool solve_faddeev = true;
  bool solve_dense = false;
  bool production_run = true;
  bool swave_only = false;          // the reference's commented-out s-wave filter (make_pw_symm_states.cpp:176-179)
  bool include_breakup_channels = false;  // breakup cells located per channel, amplitudes from the Pade solve
  std::string potential_model = "LO_internal";
  std::string energy_input_file = "lab_energies.txt";
  std::string output_folder = "Output";
  std::string P123_folder = "Output";
  std::string p_grid_type = "chebyshev";
  std::string q_grid_type = "chebyshev";
  std::string p_grid_filename, q_grid_filename;  // boundaries of a "custom" grid, one per line
  std::string precision = "mixed";  // "fp64" | "mixed"
  int precision_code = 1;           // TT_PRECISION_*
  double refine_tol = 1e-12;
  int refine_max_iter = 30;
  int energy_batch = 4;  // complex64 LUs of a channel's energies factored together (1..4)
  int tc_product = 2;          // tensor-core product of the complex64 LU: 1 bf16x3_n128, 2 tf32, 3 bf16x3
  bool panel_blocked = true;   // LU panels in 32-column steps (else recursive halving)
  int panel_width = 0;         // complex64 LU panel width, 0 = the tuning table's choice
  int inverse_block = 0;       // explicit unit-lower inverses up to this many rows, 0 = 512
  bool cta_pairs = true;       // tensor-core updates on CTA pairs
  int mid_panel = 128;         // blocked panels in mid-panels of this many columns, 0 = one level
  bool adjoint_total = true;   // run-handle adjoint: total derivative (basis and resolvent move with V)
  std::vector<double> lab_energies; // set directly or read from energy_input_file
  // additive offsets to the potential's low-energy constants, in the model's
  // order (LO_internal: C_1S0, C_3S1 in MeV^-2; malfliet_tjon has none)
  std::vector<double> lec_offsets;
};

// Sets one key=value option. Returns false (with message) on unknown key or bad value.
bool set_run_parameter(RunParams& rp, const std::string& key, const std::string& value, std::string* err);
// Applies an input-list file (read_input_list_and_set_parameters,
// CPP/set_run_parameters.cpp:247-279): every line "key=value" in order, the
// value's whitespace removed, lines without '=' and empty values skipped.
bool read_input_list(const std::string& path, RunParams& rp, std::string* err);
// Reads whitespace-separated lab energies (disk_io_routines.cpp:80-108).
bool read_input_energies(const std::string& path, std::vector<double>& out, std::string* err);

// 3N partial-wave basis (pw_3N_statespace, CPP/type_defs.h:15-29).
struct PWStates {
  int Nalpha = 0;
  int J_2N_max = 0;
  std::vector<int> L_2N, S_2N, J_2N, T_2N, L_1N, two_J_1N, two_J_3N, two_T_3N, P_3N;
  std::vector<int> chn_3N_idx;  // N_chn_3N + 1 entries
  int N_chn_3N = 0;
};

// A view of one 3N channel (contiguous alpha range of PWStates).
struct PWChannel {
  int Nalpha = 0;
  int J_2N_max = 0;
  const int *L_2N, *S_2N, *J_2N, *T_2N, *L_1N, *two_J_1N, *two_J_3N, *two_T_3N, *P_3N;
};

// construct_symmetric_pw_states, CPP/make_pw_symm_states.cpp:62-284.
bool construct_pw_states(const RunParams& rp, PWStates& pw, std::string* err);
PWChannel channel_view(const PWStates& pw, int chn);
// unique_2N_idx, CPP/make_pw_symm_states.cpp:4-60.
int unique_2N_idx(int L, int S, int J, int T, bool coupled, const RunParams& rp);

// Free wave-packet grids (fwp_statespace, CPP/type_defs.h:32-47).
struct FWPStates {
  int Np_WP = 0, Nq_WP = 0, Np_per_WP = 0, Nq_per_WP = 0;
  std::vector<double> p_WP, q_WP;        // boundaries [N+1]
  std::vector<double> p, wp, fp, q, wq, fq;
  std::vector<double> norm_p, norm_q;    // [N]
};
// make_fwp_statespace, CPP/make_wp_states.cpp:116-212 (Chebyshev grid :26-44).
bool make_fwp_states(const RunParams& rp, FWPStates& fwp, std::string* err);
void chebyshev_boundaries(int n, double* b, double scale, double t);

// 2N channel counts (CPP/main.cpp:273-289).
void count_2N_channels(const RunParams& rp, int& n_unco, int& n_coup);

// Potential matrices in the WP basis for all 2N channels touched by pw
// (calculate_potential_matrices_array_in_WP_basis, make_potential_matrix.cpp:51-429).
// V_unco: [n_unco][Np][Np] row-major; V_coup: [n_coup][2Np][2Np].
bool potential_matrices(const RunParams& rp, const FWPStates& fwp, const PWStates& pw,
                        std::vector<double>& V_unco, std::vector<double>& V_coup, std::string* err);

// Scattering wave packets (swp_statespace, CPP/type_defs.h:50-61).
struct SWPStates {
  int Np_WP = 0, Nq_WP = 0;
  int n_unco = 0, n_coup = 0;
  double E_bound = 0;
  std::vector<double> e_unco, e_coup;    // [(Np+1) n_unco], [2 (Np+1) n_coup]
  std::vector<double> C_unco, C_coup;    // eigenvector matrices (row-major, columns = states)
  std::vector<double> q_WP;              // [Nq+1]
};
// make_swp_states, CPP/make_swp_states.cpp:221-472 (eigenproblem by cyclic Jacobi).
bool make_swp_states(const RunParams& rp, const FWPStates& fwp, const PWStates& pw,
                     const std::vector<double>& V_unco, const std::vector<double>& V_coup,
                     SWPStates& swp, std::string* err);
// Symmetric eigenproblem, eigenvalues ascending, eigenvectors as columns of z (row-major n x n).
void symmetric_eigen(const double* A, int n, double* w, double* z);
// First-order change d of the SWP states (C, e_SWP boundaries, E_bound) of
// make_swp_states for a change (dV_unco, dV_coup) of the WP potential
// matrices, by perturbation theory of each 2N block's eigenproblem
// (H0 + V) C = C diag(eps): d eps_m = c_m^T dV c_m and
// d c_m = sum_{l != m} c_l (c_l^T dV c_m) / (eps_m - eps_l), carried through
// the bin-boundary rule of CPP/make_swp_states.cpp:146-183.  d has swp's
// sizes; d.C_* = dC, d.e_* = de, d.E_bound = dE_bound.  Pairs of eigenvalues
// closer than 1e-12 of their scale (degenerate) contribute nothing.
void swp_derivative(const FWPStates& fwp, const std::vector<double>& V_unco, const std::vector<double>& V_coup,
                    const SWPStates& swp, const double* dV_unco, const double* dV_coup, SWPStates& d);

// On-shell indexing (find_on_shell_bins / find_deuteron_channels,
// CPP/run_organizer.cpp:4-131, 342-378).
struct OnShell {
  std::vector<double> T_lab, q_com, E_com;
  std::vector<int> q_com_idx;
};
bool find_on_shell_bins(const RunParams& rp, const SWPStates& swp, OnShell& os, std::string* err);
std::vector<int> deuteron_indices(const PWChannel& ch);

// Breakup on-shell cells of one channel (the include_breakup_channels part of
// find_on_shell_bins, CPP/run_organizer.cpp:134-339): for every on-shell
// energy at or above the breakup threshold (E_com + E_bound >= 0), each
// (alpha, q, p) wave-packet cell whose energy range [e_p + E_q, e_{p+1} +
// E_{q+1}] (E_q = q^2 / (2 mu1_free)) holds E_com with both p boundaries
// >= 0, followed by the three neighbours on the side of the cell's quadrant
// that holds E_com.  The order and the repeats are the reference's; a
// neighbour of an edge cell can lie outside the grid (bin -1 or N).
struct BreakupCells {
  std::vector<int32_t> start;  // [nE + 1]: energy j owns cells start[j] .. start[j+1]-1
  std::vector<int32_t> cells;  // 3 per cell: alpha, q bin, p bin
  int count() const { return (int)(cells.size() / 3); }
  bool inside(int b, int Nalpha, int Nq, int Np) const {
    const int32_t* c = &cells[(size_t)3 * b];
    return c[0] >= 0 && c[0] < Nalpha && c[1] >= 0 && c[1] < Nq && c[2] >= 0 && c[2] < Np;
  }
};
bool find_breakup_cells(const RunParams& rp, const PWChannel& ch, const SWPStates& swp,
                        const std::vector<double>& E_com, BreakupCells& bu, std::string* err);

// Kinematics, CPP/General_functions/kinetic_conversion.cpp:5-54.
double mu1(double Eb);
double mu1_free();
double com_energy_to_com_p_momentum(double Ep);
double com_momentum_to_lab_energy(double q_com, double Eb);
double lab_energy_to_com_momentum(double T_lab, double Eb);
double com_energy_to_com_q_momentum(double E_com);
double com_q_momentum_to_com_energy(double q_com);

// Nucleon-nucleon potential models available without a Fortran compiler:
// Malfliet-Tjon I-III (Interactions/malfliet_tjon.cpp) and chiral LO with
// one-pion exchange (Interactions/chiral_LO_internal.cpp + OPEP.cpp).
class Potential {
 public:
  virtual ~Potential() {}
  // Varray[6] as in Interactions/potential_model.h:21
  virtual void V(double qi, double qo, bool coupled, int S, int J, int T, int Tz, double* Varray) = 0;
};
Potential* make_potential(const std::string& name, std::string* err,
                          const std::vector<double>& lec_offsets = std::vector<double>());
// Number of low-energy constants of a model that lec_offsets can move.
int num_lecs(const std::string& name);
// Nominal values of those constants (same order).
std::vector<double> nominal_lecs(const std::string& name);

}  // namespace tt
