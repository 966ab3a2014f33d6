// C-ABI of tictac_b200 (include/tictac_b200.h).
#include "tictac_b200.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../cuda/tt_kernels.h"
#include "../host/tt_breakup.h"
#include "../host/tt_h5.h"
#include "../host/tt_host.h"
#include "../host/tt_math.h"
#include "../host/tt_p123.h"
#include "../host/tt_solver.h"

namespace tt {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

}  // namespace tt

using namespace tt;

namespace {

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

struct ChannelState {
  std::unique_ptr<ChannelSolver> solver;
  bool have_P = false, have_A = false, have_G = false;
  int fwd_precision = -1;  // precision of the last tt_run_adjoint_forward
};

// Per-thread stream for the drop-in entry points.
cudaStream_t default_stream() {
  static thread_local cudaStream_t s = nullptr;
  if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  return s;
}

PWChannel view_of(const tt_pw_states* pw) {
  PWChannel c;
  c.Nalpha = pw->Nalpha;
  c.J_2N_max = pw->J_2N_max;
  c.L_2N = pw->L_2N_array;
  c.S_2N = pw->S_2N_array;
  c.J_2N = pw->J_2N_array;
  c.T_2N = pw->T_2N_array;
  c.L_1N = pw->L_1N_array;
  c.two_J_1N = pw->two_J_1N_array;
  c.two_J_3N = pw->two_J_3N_array;
  c.two_T_3N = pw->two_T_3N_array;
  c.P_3N = pw->P_3N_array;
  return c;
}

RunParams params_of(const tt_run_params* rp) {
  RunParams r;
  if (rp) {
    r.Nphi = rp->Nphi;
    r.Nx = rp->Nx;
    r.tensor_force = rp->tensor_force != 0;
    r.isospin_breaking_1S0 = rp->isospin_breaking_1S0 != 0;
    r.production_run = rp->production_run != 0;
    r.precision = rp->precision == TT_PRECISION_FP64 ? "fp64" : "mixed";
    r.precision_code = rp->precision;
    r.refine_tol = rp->refine_tol;
    r.refine_max_iter = rp->refine_max_iter;
  }
  return r;
}

SWPStates swp_of(const tt_swp_states* s) {
  SWPStates w;
  w.Np_WP = s->Np_WP;
  w.Nq_WP = s->Nq_WP;
  w.n_unco = s->num_2N_unco_states;
  w.n_coup = s->num_2N_coup_states;
  w.E_bound = s->E_bound;
  const size_t Np = s->Np_WP;
  if (s->e_SWP_unco_array) w.e_unco.assign(s->e_SWP_unco_array, s->e_SWP_unco_array + (Np + 1) * w.n_unco);
  if (s->e_SWP_coup_array) w.e_coup.assign(s->e_SWP_coup_array, s->e_SWP_coup_array + 2 * (Np + 1) * w.n_coup);
  if (s->C_SWP_unco_array) w.C_unco.assign(s->C_SWP_unco_array, s->C_SWP_unco_array + Np * Np * w.n_unco);
  if (s->C_SWP_coup_array) w.C_coup.assign(s->C_SWP_coup_array, s->C_SWP_coup_array + 4 * Np * Np * w.n_coup);
  w.q_WP.assign(s->q_WP_array, s->q_WP_array + s->Nq_WP + 1);
  return w;
}

SolveOptions options_of(const RunParams& rp, int precision) {
  SolveOptions o;
  o.mixed = precision == TT_PRECISION_MIXED || precision == TT_PRECISION_MIXED_SIMT;
  o.tensor_cores = precision == TT_PRECISION_MIXED;
  o.pade = precision == TT_PRECISION_PADE;
  o.refine_tol = rp.refine_tol;
  o.refine_max_iter = rp.refine_max_iter;
  o.energy_batch = rp.energy_batch;
  o.tc_product = rp.tc_product;
  o.panel_blocked = rp.panel_blocked;
  o.panel_width = rp.panel_width;
  o.inverse_block = rp.inverse_block;
  o.cta_pairs = rp.cta_pairs;
  o.mid_panel = rp.mid_panel;
  return o;
}

void fill_report(const SolveReport& r, double ms_A, tt_solve_report* out) {
  if (!out) return;
  out->ms_A = ms_A;
  out->ms_form = r.ms_form;
  out->ms_factor = r.ms_factor;
  out->ms_solve = r.ms_solve;
  out->ms_refine = r.ms_refine;
  out->refine_iters = r.refine_iters;
  out->final_correction = r.final_correction;
  out->info = r.info;
  out->ms_adjoint = r.ms_adjoint;
  out->adjoint_refine_iters = r.adjoint_refine_iters;
  out->product_fallbacks = r.product_fallbacks;
}

// dV_k C blocks (layout of ChannelLayout::VC) of n_theta potential derivatives
int dvc_blocks(const RunParams& rp, const PWChannel& ch, const SWPStates& w, int n_theta, const double* dVu,
               const double* dVc, std::vector<double>& out, size_t& per) {
  const size_t Np = w.Np_WP, nu = Np * Np * w.n_unco, nc = 4 * Np * Np * w.n_coup;
  out.clear();
  per = 0;
  for (int k = 0; k < n_theta; k++) {
    std::vector<double> Vu(dVu + k * nu, dVu + (k + 1) * nu), Vc;
    if (nc) Vc.assign(dVc + k * nc, dVc + (k + 1) * nc);
    ChannelLayout Lk;
    std::string err;
    if (!build_channel_layout(rp, ch, w, Vu, Vc, Lk, &err)) return fail(TT_ERR_BADARG, err);
    per = Lk.VC.size();
    out.insert(out.end(), Lk.VC.begin(), Lk.VC.end());
  }
  return TT_OK;
}

// tt_solve_faddeev_equations, with the adjoint when n_theta > 0
int dropin_solve(tt_complex* U, tt_complex* dU, int n_theta, const double* dVu, const double* dVc,
                 const tt_complex* G, const double* P_val, const int* P_row, const size_t* P_colptr, size_t P_nnz,
                 const double* V_unco, const double* V_coup, const tt_swp_states* swp, const tt_os_indexing* os,
                 const tt_pw_states* pw, const tt_run_params* rpp, tt_solve_report* report,
                 const tt_bu_indexing* bui = nullptr, tt_complex* U_BU = nullptr) {
  if (!U || !G || !P_colptr || !swp || !os || !pw || !rpp) return fail(TT_ERR_BADARG, "null argument");
  BreakupCells cells;
  if (bui) {
    if (rpp->precision != TT_PRECISION_PADE)
      return fail(TT_ERR_UNSUPPORTED, "breakup amplitudes come from the Pade path (TT_PRECISION_PADE), as in the reference");
    if (bui->num_BU_chns < 0 || !bui->q_com_BU_idx_array || (bui->num_BU_chns > 0 && (!bui->alphapq_idx_array || !U_BU)))
      return fail(TT_ERR_BADARG, "null or negative breakup indexing");
    cells.start.assign(bui->q_com_BU_idx_array, bui->q_com_BU_idx_array + os->num_T_lab + 1);
    cells.cells.assign(bui->alphapq_idx_array, bui->alphapq_idx_array + (size_t)3 * bui->num_BU_chns);
  }
  if (P_nnz && (!P_val || !P_row)) return fail(TT_ERR_BADARG, "null P123 arrays");
  if (n_theta < 0 || (n_theta > 0 && (!dU || !dVu || (swp->num_2N_coup_states && !dVc))))
    return fail(TT_ERR_BADARG, "null or negative adjoint arguments");
  RunParams rp = params_of(rpp);
  SWPStates w = swp_of(swp);
  const size_t Np = w.Np_WP;
  std::vector<double> Vu(V_unco, V_unco + Np * Np * w.n_unco);
  std::vector<double> Vc;
  if (w.n_coup) Vc.assign(V_coup, V_coup + 4 * Np * Np * w.n_coup);
  ChannelLayout L;
  std::string err;
  const PWChannel ch = view_of(pw);
  if (!build_channel_layout(rp, ch, w, Vu, Vc, L, &err)) return fail(TT_ERR_BADARG, err);
  const int n = ch.Nalpha * w.Np_WP * w.Nq_WP;
  if (P_colptr[n] != P_nnz) return fail(TT_ERR_BADARG, "P123 column pointers do not end at nnz");
  cudaStream_t st = default_stream();
  ChannelSolver cs;
  int s = cs.setup(L, w.q_WP, st);
  if (s != TT_OK) return s;
  // CSC -> CSR on the device
  static_assert(sizeof(size_t) == sizeof(uint64_t), "size_t column pointers");
  s = cs.set_P_host_csc(P_val, P_row, reinterpret_cast<const uint64_t*>(P_colptr), (int64_t)P_nnz, st);
  if (s != TT_OK) return s;
  double msA = 0;
  s = cs.build_A(st, &msA);
  if (s != TT_OK) return s;
  // G supplied by the caller: upload into the solver through resolvent-shaped storage
  std::vector<double> dummyE(os->num_T_lab, 0.0);
  s = cs.resolvent(dummyE, st);
  if (s != TT_OK) return s;
  if (cudaMemcpy((void*)cs.G(), G, sizeof(tt_complex) * (size_t)n * os->num_T_lab, cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return fail(TT_ERR_CUDA, "upload of G failed");
  std::vector<int> q_idx(os->q_com_idx_array, os->q_com_idx_array + os->num_T_lab);
  std::vector<int> deut(os->deuteron_idx_array, os->deuteron_idx_array + os->num_deuteron_states);
  std::vector<double> Uh, dUh, dvc;
  SolveReport rep;
  if (rpp->precision < TT_PRECISION_FP64 || rpp->precision > TT_PRECISION_PADE)
    return fail(TT_ERR_BADARG, "unknown precision");
  AdjointRequest adj;
  DevBuf<double> d_dvc;
  if (n_theta > 0) {
    size_t per = 0;
    TT_TRY(dvc_blocks(rp, ch, w, n_theta, dVu, dVc, dvc, per));
    TT_TRY(d_dvc.upload(dvc, st));
    adj.n_theta = n_theta;
    adj.d_dVC = d_dvc.ptr;
    adj.vc_count = per;
    adj.dU = &dUh;
  }
  std::vector<double> UBh;
  BreakupRequest bq;
  bq.cells = &cells;
  bq.U_BU = &UBh;
  s = cs.solve(q_idx, deut, options_of(rp, rpp->precision), Uh, &rep, st, n_theta > 0 ? &adj : nullptr,
               bui ? &bq : nullptr);
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  if (n_theta > 0) std::memcpy(dU, dUh.data(), sizeof(double) * dUh.size());
  if (bui && !UBh.empty()) std::memcpy(U_BU, UBh.data(), sizeof(double) * UBh.size());
  return TT_OK;
}

}  // namespace

struct tt_run {
  RunParams rp;
  PWStates pw;
  FWPStates fwp;
  std::vector<double> V_unco, V_coup;
  SWPStates swp;
  OnShell os;
  std::vector<BreakupCells> bu;  // per channel, when include_breakup_channels=true
  std::vector<ChannelState> chn;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

extern "C" {

void tt_run_params_default(tt_run_params* rp) {
  if (!rp) return;
  rp->Nphi = 48;
  rp->Nx = 48;
  rp->tensor_force = 1;
  rp->isospin_breaking_1S0 = 1;
  rp->production_run = 1;
  rp->precision = TT_PRECISION_MIXED;
  rp->refine_tol = 1e-12;
  rp->refine_max_iter = 30;
}

void tt_free(void* p) { std::free(p); }

unsigned long long tt_kernel_launches(void) { return g_launches.load(); }

double tt_wigner_3j(int a, int b, int c, int ma, int mb, int mc) { return wigner3j(a, b, c, ma, mb, mc); }
double tt_wigner_6j(int a, int b, int c, int d, int e, int f) { return wigner6j(a, b, c, d, e, f); }
double tt_wigner_9j(int a, int b, int c, int d, int e, int f, int g, int h, int i) {
  return wigner9j(a, b, c, d, e, f, g, h, i);
}
double tt_clebsch_gordan(int j1, int j2, int j3, int m1, int m2, int m3) {
  return clebsch_gordan(j1, j2, j3, m1, m2, m3);
}
int tt_legendre_spharm_array(int lmax, double x, double* out) {
  if (lmax < 0 || !out) return fail(TT_ERR_BADARG, "bad argument");
  legendre_spharm_array(lmax, x, out);
  return TT_OK;
}
int tt_gauss_legendre(int n, double* x, double* w) {
  if (n < 1 || !x || !w) return fail(TT_ERR_BADARG, "bad argument");
  gauss_legendre(x, w, n);
  return TT_OK;
}
const char* tt_last_error_string(void) { return last_error(); }

int tt_device_count(int* count) {
  if (!count) return fail(TT_ERR_BADARG, "null count");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return fail(TT_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = c;
  return TT_OK;
}

int tt_fill_P123_arrays(double** val, int** row, int** col, size_t* nnz, int production_run, const tt_fwp_states* fwp,
                        const tt_pw_states* pw, const tt_run_params* rpp) {
  if (!val || !row || !col || !nnz || !fwp || !pw || !rpp) return fail(TT_ERR_BADARG, "null argument");
  RunParams rp = params_of(rpp);
  rp.production_run = production_run != 0;
  FWPStates f;
  f.Np_WP = fwp->Np_WP;
  f.Nq_WP = fwp->Nq_WP;
  f.p_WP.assign(fwp->p_WP_array, fwp->p_WP_array + fwp->Np_WP + 1);
  f.q_WP.assign(fwp->q_WP_array, fwp->q_WP_array + fwp->Nq_WP + 1);
  P123Tables t;
  std::string err;
  if (!p123_prepare(rp, f, view_of(pw), t, &err)) return fail(TT_ERR_BADARG, err);
  cudaStream_t st = default_stream();
  DeviceCSR P;
  int s = p123_build_device(t, P, st, nullptr);
  if (s != TT_OK) return s;
  const int n = P.n;
  std::vector<int64_t> rowptr(n + 1);
  if (cudaMemcpy(rowptr.data(), P.rowptr.ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy of P123 row pointers failed");
  const size_t m = (size_t)P.nnz;
  *val = (double*)std::malloc(sizeof(double) * std::max<size_t>(m, 1));
  *row = (int*)std::malloc(sizeof(int) * std::max<size_t>(m, 1));
  *col = (int*)std::malloc(sizeof(int) * std::max<size_t>(m, 1));
  if (!*val || !*row || !*col) return fail(TT_ERR_NOMEM, "host allocation for P123 failed");
  if (m) {
    if (cudaMemcpy(*val, P.val.ptr, sizeof(double) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(*col, P.col.ptr, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(TT_ERR_CUDA, "copy of P123 failed");
  }
  for (int r = 0; r < n; r++)
    for (int64_t e = rowptr[r]; e < rowptr[r + 1]; e++) (*row)[e] = r;
  *nnz = m;
  return TT_OK;
}

int tt_calculate_resolvent_array_in_SWP_basis(tt_complex* G, double E, const tt_swp_states* swp,
                                              const tt_pw_states* pw, const tt_run_params* rpp) {
  if (!G || !swp || !pw || !rpp) return fail(TT_ERR_BADARG, "null argument");
  RunParams rp = params_of(rpp);
  SWPStates w = swp_of(swp);
  // only the SWP energy boundaries are needed; give the layout builder
  // identity C/V blocks of the right size
  if (w.C_unco.empty()) w.C_unco.assign((size_t)w.Np_WP * w.Np_WP * w.n_unco, 0.0);
  if (w.C_coup.empty()) w.C_coup.assign((size_t)4 * w.Np_WP * w.Np_WP * w.n_coup, 0.0);
  std::vector<double> Vu(w.C_unco.size(), 0.0), Vc(w.C_coup.size(), 0.0);
  ChannelLayout L;
  std::string err;
  if (!build_channel_layout(rp, view_of(pw), w, Vu, Vc, L, &err)) return fail(TT_ERR_BADARG, err);
  cudaStream_t st = default_stream();
  ChannelSolver cs;
  int s = cs.setup(L, w.q_WP, st);
  if (s != TT_OK) return s;
  s = cs.resolvent({E}, st);
  if (s != TT_OK) return s;
  if (cudaMemcpy(G, cs.G(), sizeof(tt_complex) * cs.n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy of G failed");
  return TT_OK;
}

int tt_calculate_resolvent_array_in_SWP_basis_noalloc(tt_complex* G_dev, const double* E, int nE,
                                                      const tt_swp_states* swp, const tt_pw_states* pw,
                                                      const tt_run_params* rpp, void* stream) {
  if (!G_dev || !swp || !pw || !rpp || (nE > 0 && !E) || !swp->q_WP_array) return fail(TT_ERR_BADARG, "null argument");
  if (nE < 0 || swp->Np_WP < 1 || swp->Nq_WP < 1 || pw->Nalpha < 0 || swp->num_2N_unco_states < 0 ||
      swp->num_2N_coup_states < 0)
    return fail(TT_ERR_BADARG, "negative or empty size");
  if ((swp->num_2N_unco_states && !swp->e_SWP_unco_array) || (swp->num_2N_coup_states && !swp->e_SWP_coup_array))
    return fail(TT_ERR_BADARG, "null SWP energy array");
  const RunParams rp = params_of(rpp);
  return resolvent_noalloc(rp, view_of(pw), swp->Np_WP, swp->Nq_WP, swp->num_2N_unco_states, swp->num_2N_coup_states,
                           swp->e_SWP_unco_array, swp->e_SWP_coup_array, swp->q_WP_array, E, nE,
                           reinterpret_cast<double*>(G_dev), static_cast<cudaStream_t>(stream));
}

int tt_solve_faddeev_equations(tt_complex* U, const tt_complex* G, const double* P_val, const int* P_row,
                               const size_t* P_colptr, size_t P_nnz, const double* V_unco, const double* V_coup,
                               const tt_swp_states* swp, const tt_os_indexing* os, const tt_pw_states* pw,
                               const tt_run_params* rpp, tt_solve_report* report) {
  return dropin_solve(U, nullptr, 0, nullptr, nullptr, G, P_val, P_row, P_colptr, P_nnz, V_unco, V_coup, swp, os, pw,
                      rpp, report);
}

int tt_solve_faddeev_equations_breakup(tt_complex* U, tt_complex* U_BU, const tt_bu_indexing* bu, const tt_complex* G,
                                       const double* P_val, const int* P_row, const size_t* P_colptr, size_t P_nnz,
                                       const double* V_unco, const double* V_coup, const tt_swp_states* swp,
                                       const tt_os_indexing* os, const tt_pw_states* pw, const tt_run_params* rp,
                                       tt_solve_report* report) {
  if (!bu) return fail(TT_ERR_BADARG, "null breakup indexing");
  return dropin_solve(U, nullptr, 0, nullptr, nullptr, G, P_val, P_row, P_colptr, P_nnz, V_unco, V_coup, swp, os, pw,
                      rp, report, bu, U_BU);
}

int tt_solve_faddeev_adjoint(tt_complex* U, tt_complex* dU, int n_theta, const double* dVu, const double* dVc,
                             const tt_complex* G, const double* P_val, const int* P_row, const size_t* P_colptr,
                             size_t P_nnz, const double* V_unco, const double* V_coup, const tt_swp_states* swp,
                             const tt_os_indexing* os, const tt_pw_states* pw, const tt_run_params* rpp,
                             tt_solve_report* report) {
  return dropin_solve(U, dU, n_theta, dVu, dVc, G, P_val, P_row, P_colptr, P_nnz, V_unco, V_coup, swp, os, pw, rpp,
                      report);
}

// ---------------------------------------------------------------------------
int tt_run_create(tt_run** out, int nopt, const char* const* opts) {
  if (!out) return fail(TT_ERR_BADARG, "null run pointer");
  *out = nullptr;
  std::unique_ptr<tt_run> r(new tt_run());
  std::string err;
  for (int i = 0; i < nopt; i++) {
    const std::string a = opts[i] ? opts[i] : "";
    const size_t eq = a.find('=');
    // an input-list file, applied in argument order (CPP/set_run_parameters.cpp:641-644)
    if (eq == std::string::npos && a.size() > 4 && a.compare(a.size() - 4, 4, ".txt") == 0) {
      if (!read_input_list(a, r->rp, &err)) return fail(TT_ERR_BADARG, err);
      continue;
    }
    if (eq == std::string::npos) return fail(TT_ERR_BADARG, "option without '=': " + a);
    const std::string v = a.substr(eq + 1);
    if (v.empty()) continue;  // the reference skips empty values
    if (!set_run_parameter(r->rp, a.substr(0, eq), v, &err)) return fail(TT_ERR_BADARG, err);
  }
  // set_run_parameters' and main's consistency checks (CPP/set_run_parameters.cpp:666-668, main.cpp:162-164)
  if (r->rp.parallel_run && r->rp.channel_idx == -1)
    return fail(TT_ERR_BADARG, "Parallel run specified in input but no channel index (i.e. channel_idx=<int>) given!");
  if (!r->rp.solve_faddeev && !r->rp.calculate_and_store_P123)
    return fail(TT_ERR_BADARG,
                "Both solve_faddeev=false and calculate_and_store_P123==false so code has nothing to do!");
  if (!construct_pw_states(r->rp, r->pw, &err)) return fail(TT_ERR_BADARG, err);
  if (!make_fwp_states(r->rp, r->fwp, &err)) return fail(TT_ERR_BADARG, err);
  if (!potential_matrices(r->rp, r->fwp, r->pw, r->V_unco, r->V_coup, &err)) return fail(TT_ERR_BADARG, err);
  if (!make_swp_states(r->rp, r->fwp, r->pw, r->V_unco, r->V_coup, r->swp, &err)) return fail(TT_ERR_BADARG, err);
  if (!find_on_shell_bins(r->rp, r->swp, r->os, &err)) return fail(TT_ERR_BADARG, err);
  if (r->rp.include_breakup_channels) {  // located with the elastic bins, as in the reference
    r->bu.resize(r->pw.N_chn_3N);
    for (int c = 0; c < r->pw.N_chn_3N; c++)
      if (!find_breakup_cells(r->rp, channel_view(r->pw, c), r->swp, r->os.E_com, r->bu[c], &err))
        return fail(TT_ERR_BADARG, err);
  }
  r->chn.resize(r->pw.N_chn_3N);
  *out = r.release();
  return TT_OK;
}

int tt_release_cached_device_memory(void) {
  device_cache_trim();
  return TT_OK;
}

int tt_cached_device_memory(size_t* bytes) {
  if (!bytes) return fail(TT_ERR_BADARG, "null bytes");
  *bytes = device_cache_bytes();
  return TT_OK;
}

int tt_run_set_solve_option(tt_run* run, const char* key, const char* value) {
  if (!run || !key || !value) return fail(TT_ERR_BADARG, "null run, key or value");
  static const char* const kSolveKeys[] = {"tc_product", "panel_width", "panel_order", "energy_batch",
                                           "refine_tol", "refine_max_iter", "inverse_block", "cta_pairs", "mid_panel"};
  bool ok = false;
  for (const char* k : kSolveKeys) ok = ok || std::strcmp(k, key) == 0;
  if (!ok) return fail(TT_ERR_BADARG, std::string("not a solve option: ") + key);
  std::string err;
  RunParams rp = run->rp;
  if (!set_run_parameter(rp, key, value, &err)) return fail(TT_ERR_BADARG, err);
  run->rp = rp;
  return TT_OK;
}

void tt_run_destroy(tt_run* run) {
  if (!run) return;
  run->chn.clear();
  device_cache_trim();
  if (run->ev0) cudaEventDestroy(run->ev0);
  if (run->ev1) cudaEventDestroy(run->ev1);
  if (run->stream) cudaStreamDestroy(run->stream);
  delete run;
}

static int check_chn(const tt_run* run, int chn) {
  if (!run) return fail(TT_ERR_BADARG, "null run");
  if (chn < 0 || chn >= run->pw.N_chn_3N) return fail(TT_ERR_BADARG, "channel index out of range");
  return TT_OK;
}

static cudaStream_t run_stream(tt_run* run) {
  if (!run->stream) cudaStreamCreateWithFlags(&run->stream, cudaStreamNonBlocking);
  return run->stream;
}

// Device blocks of an adjoint request for n_theta potential derivatives of a
// run: d(V C) (and, for the total derivative, dC, de_SWP and dE_bound from the
// SWP eigenproblem's first-order perturbation).
struct AdjointBuffers {
  DevBuf<double> dvc, dc, de;
};

static int adjoint_request(tt_run* run, const PWChannel& ch, int n_theta, const double* dVu, const double* dVc,
                    AdjointRequest& adj, AdjointBuffers& ab) {
  std::vector<double> dvc;
  size_t per = 0;
  TT_TRY(dvc_blocks(run->rp, ch, run->swp, n_theta, dVu, dVc, dvc, per));
  adj.n_theta = n_theta;
  adj.vc_count = per;
  if (run->rp.adjoint_total) {
    // the SWP basis moves with the potential: dC, de_SWP, dE_bound per
    // parameter, and d(V C) = dV C + V dC
    const size_t Np = run->swp.Np_WP, nu = Np * Np * run->swp.n_unco, nc = 4 * Np * Np * run->swp.n_coup;
    std::vector<double> dcb, deb;
    for (int k = 0; k < n_theta; k++) {
      SWPStates dswp;
      swp_derivative(run->fwp, run->V_unco, run->V_coup, run->swp, dVu + k * nu, nc ? dVc + k * nc : nullptr, dswp);
      ChannelLayout Ld;
      std::string err;
      if (!build_channel_layout(run->rp, ch, dswp, run->V_unco, run->V_coup, Ld, &err)) return fail(TT_ERR_BADARG, err);
      if (Ld.VC.size() != per) return fail(TT_ERR_BADARG, "derivative blocks do not match the channel layout");
      for (size_t i = 0; i < per; i++) dvc[(size_t)k * per + i] += Ld.VC[i];  // + V dC
      adj.c_count = Ld.C.size();
      adj.e_count = Ld.e_swp.size();
      dcb.insert(dcb.end(), Ld.C.begin(), Ld.C.end());
      deb.insert(deb.end(), Ld.e_swp.begin(), Ld.e_swp.end());
      adj.dEb.push_back(dswp.E_bound);
    }
    TT_TRY(ab.dc.upload(dcb, run_stream(run)));
    TT_TRY(ab.de.upload(deb, run_stream(run)));
    adj.total = true;
    // mu1 = Mn Md / (Mn + Md), Md = Mn + Mp + E_bound (CPP/General_functions/kinetic_conversion.cpp:10-13)
    const double Md = kMn + kMp + run->swp.E_bound;
    adj.E_bound = run->swp.E_bound;
    adj.dlnmu1_dEb = 1.0 / Md - 1.0 / (kMn + Md);
    adj.d_dC = ab.dc.ptr;
    adj.d_de = ab.de.ptr;
  }
  TT_TRY(ab.dvc.upload(dvc, run_stream(run)));
  adj.d_dVC = ab.dvc.ptr;
  return TT_OK;
}


int tt_run_num_channels(const tt_run* run, int* n) {
  if (!run || !n) return fail(TT_ERR_BADARG, "null argument");
  *n = run->pw.N_chn_3N;
  return TT_OK;
}

int tt_run_channel_info(const tt_run* run, int chn, int* Nalpha, int* dense_dim, int* two_J, int* P, int* nd) {
  int s = check_chn(run, chn);
  if (s) return s;
  const PWChannel c = channel_view(run->pw, chn);
  if (Nalpha) *Nalpha = c.Nalpha;
  if (dense_dim) *dense_dim = c.Nalpha * run->fwp.Np_WP * run->fwp.Nq_WP;
  if (two_J) *two_J = c.two_J_3N[0];
  if (P) *P = c.P_3N[0];
  if (nd) *nd = (int)deuteron_indices(c).size();
  return TT_OK;
}

int tt_run_num_energies(const tt_run* run, int* nE) {
  if (!run || !nE) return fail(TT_ERR_BADARG, "null argument");
  *nE = (int)run->os.q_com_idx.size();
  return TT_OK;
}

int tt_run_energies(const tt_run* run, double* T_lab, double* E_com, int* q_idx) {
  if (!run) return fail(TT_ERR_BADARG, "null run");
  for (size_t i = 0; i < run->os.q_com_idx.size(); i++) {
    if (T_lab) T_lab[i] = run->os.T_lab[i];
    if (E_com) E_com[i] = run->os.E_com[i];
    if (q_idx) q_idx[i] = run->os.q_com_idx[i];
  }
  return TT_OK;
}

int tt_run_E_bound(const tt_run* run, double* Eb) {
  if (!run || !Eb) return fail(TT_ERR_BADARG, "null argument");
  *Eb = run->swp.E_bound;
  return TT_OK;
}

static int ensure_solver(tt_run* run, int chn) {
  ChannelState& cs = run->chn[chn];
  if (cs.solver) return TT_OK;
  ChannelLayout L;
  std::string err;
  if (!build_channel_layout(run->rp, channel_view(run->pw, chn), run->swp, run->V_unco, run->V_coup, L, &err))
    return fail(TT_ERR_BADARG, err);
  cs.solver.reset(new ChannelSolver());
  return cs.solver->setup(L, run->swp.q_WP, run_stream(run));
}

int tt_run_build_P123(tt_run* run, int chn, int64_t* nnz) {
  int s = check_chn(run, chn);
  if (s) return s;
  // calculate_and_store_P123 = false: the reference reads the channel's file
  // instead of computing P123 (CPP/make_permutation_matrix.cpp:1387-1403)
  if (!run->rp.calculate_and_store_P123) return tt_run_load_P123_h5(run, chn, nullptr, nnz);
  TT_TRY(ensure_solver(run, chn));
  P123Tables t;
  std::string err;
  if (!p123_prepare(run->rp, run->fwp, channel_view(run->pw, chn), t, &err)) return fail(TT_ERR_BADARG, err);
  DeviceCSR P;
  TT_TRY(p123_build_device(t, P, run_stream(run), nullptr));
  if (nnz) *nnz = P.nnz;
  TT_TRY(run->chn[chn].solver->set_P_device(std::move(P)));
  run->chn[chn].have_P = true;
  return TT_OK;
}

int tt_run_build_A(tt_run* run, int chn, double* ms) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!run->chn[chn].have_P) TT_TRY(tt_run_build_P123(run, chn, nullptr));
  TT_TRY(run->chn[chn].solver->build_A(run_stream(run), ms));
  run->chn[chn].have_A = true;
  return TT_OK;
}

int tt_run_build_resolvent(tt_run* run, int chn) {
  int s = check_chn(run, chn);
  if (s) return s;
  TT_TRY(ensure_solver(run, chn));
  std::vector<double> E;
  for (double e : run->os.E_com) E.push_back(e + run->swp.E_bound);  // CPP/main.cpp:391
  TT_TRY(run->chn[chn].solver->resolvent(E, run_stream(run)));
  run->chn[chn].have_G = true;
  return TT_OK;
}

int tt_run_solve(tt_run* run, int chn, int precision, tt_complex* U, tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U) return fail(TT_ERR_BADARG, "null U");
  if (precision < TT_PRECISION_FP64 || precision > TT_PRECISION_PADE) return fail(TT_ERR_BADARG, "unknown precision");
  double msA = 0;
  if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
  if (!run->chn[chn].have_G) TT_TRY(tt_run_build_resolvent(run, chn));
  const std::vector<int> deut = deuteron_indices(channel_view(run->pw, chn));
  std::vector<double> Uh;
  SolveReport rep;
  s = run->chn[chn].solver->solve(run->os.q_com_idx, deut, options_of(run->rp, precision), Uh, &rep,
                                  run_stream(run));
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  return TT_OK;
}

int tt_run_solve_energies(tt_run* run, int chn, int precision, int n_sel, const int* energy_idx, tt_complex* U,
                          tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U || n_sel < 0 || (n_sel > 0 && !energy_idx)) return fail(TT_ERR_BADARG, "null or negative argument");
  if (precision < TT_PRECISION_FP64 || precision > TT_PRECISION_PADE) return fail(TT_ERR_BADARG, "unknown precision");
  const int nE = (int)run->os.E_com.size();
  std::vector<double> E;
  std::vector<int> q;
  for (int k = 0; k < n_sel; k++) {
    const int j = energy_idx[k];
    if (j < 0 || j >= nE) return fail(TT_ERR_BADARG, "energy index " + std::to_string(j) + " outside the run's bins");
    for (int k2 = 0; k2 < k; k2++)
      if (energy_idx[k2] == j) return fail(TT_ERR_BADARG, "energy index listed twice");
    E.push_back(run->os.E_com[j] + run->swp.E_bound);  // CPP/main.cpp:391
    q.push_back(run->os.q_com_idx[j]);
  }
  double msA = 0;
  if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
  // the channel's resolvents now hold the selected energies only
  run->chn[chn].have_G = false;
  TT_TRY(run->chn[chn].solver->resolvent(E, run_stream(run)));
  const std::vector<int> deut = deuteron_indices(channel_view(run->pw, chn));
  std::vector<double> Uh;
  SolveReport rep;
  s = run->chn[chn].solver->solve(q, deut, options_of(run->rp, precision), Uh, &rep, run_stream(run));
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  return TT_OK;
}

int tt_run_solve_adjoint(tt_run* run, int chn, int precision, int n_theta, const double* dVu, const double* dVc,
                         tt_complex* U, tt_complex* dU, tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U || n_theta < 0 || (n_theta > 0 && (!dU || !dVu || (run->swp.n_coup && !dVc))))
    return fail(TT_ERR_BADARG, "null or negative argument");
  if (precision < TT_PRECISION_FP64 || precision > TT_PRECISION_PADE) return fail(TT_ERR_BADARG, "unknown precision");
  double msA = 0;
  if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
  if (!run->chn[chn].have_G) TT_TRY(tt_run_build_resolvent(run, chn));
  const PWChannel ch = channel_view(run->pw, chn);
  const std::vector<int> deut = deuteron_indices(ch);
  std::vector<double> Uh, dUh;
  AdjointRequest adj;
  AdjointBuffers ab;
  if (n_theta > 0) {
    TT_TRY(adjoint_request(run, ch, n_theta, dVu, dVc, adj, ab));
    adj.dU = &dUh;
  }
  SolveReport rep;
  s = run->chn[chn].solver->solve(run->os.q_com_idx, deut, options_of(run->rp, precision), Uh, &rep,
                                  run_stream(run), n_theta > 0 ? &adj : nullptr);
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  if (n_theta > 0) std::memcpy(dU, dUh.data(), sizeof(double) * dUh.size());
  return TT_OK;
}

int tt_run_adjoint_forward(tt_run* run, int chn, int precision, tt_complex* U, tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U) return fail(TT_ERR_BADARG, "null U");
  if (precision != TT_PRECISION_FP64 && precision != TT_PRECISION_MIXED && precision != TT_PRECISION_MIXED_SIMT)
    return fail(TT_ERR_UNSUPPORTED, "the adjoint needs an LU precision");
  double msA = 0;
  if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
  if (!run->chn[chn].have_G) TT_TRY(tt_run_build_resolvent(run, chn));
  const std::vector<int> deut = deuteron_indices(channel_view(run->pw, chn));
  SolveOptions o = options_of(run->rp, precision);
  o.keep_factors = true;
  std::vector<double> Uh;
  SolveReport rep;
  s = run->chn[chn].solver->solve(run->os.q_com_idx, deut, o, Uh, &rep, run_stream(run));
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  run->chn[chn].fwd_precision = precision;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  return TT_OK;
}

int tt_run_adjoint_backward(tt_run* run, int chn, int n_theta, const double* dVu, const double* dVc,
                            const tt_complex* U_bar, double* theta_bar, tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (n_theta < 0 || (n_theta > 0 && (!U_bar || !theta_bar || !dVu || (run->swp.n_coup && !dVc))))
    return fail(TT_ERR_BADARG, "null or negative argument");
  const int precision = run->chn[chn].fwd_precision;
  if (precision < 0) return fail(TT_ERR_BADARG, "no forward solve of this channel (tt_run_adjoint_forward)");
  if (n_theta == 0) return TT_OK;
  const PWChannel ch = channel_view(run->pw, chn);
  const std::vector<int> deut = deuteron_indices(ch);
  AdjointRequest adj;
  AdjointBuffers ab;
  TT_TRY(adjoint_request(run, ch, n_theta, dVu, dVc, adj, ab));
  std::vector<double> dUh, Uh;
  SolveReport rep;
  double msA = 0;
  if (run->chn[chn].solver->kept()) {
    s = run->chn[chn].solver->backward(adj, dUh, &rep, run_stream(run));
  } else {
    // the forward factors were not kept (HBM): factor again with the request
    if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
    if (!run->chn[chn].have_G) TT_TRY(tt_run_build_resolvent(run, chn));
    adj.dU = &dUh;
    s = run->chn[chn].solver->solve(run->os.q_com_idx, deut, options_of(run->rp, precision), Uh, &rep,
                                    run_stream(run), &adj);
  }
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  run->chn[chn].fwd_precision = -1;
  // theta_bar_k = Re sum_e conj(U_bar_e) dU_e / dtheta_k
  const size_t ne = dUh.size() / 2 / (size_t)n_theta;
  for (int k = 0; k < n_theta; k++) {
    double acc = 0;
    for (size_t e = 0; e < ne; e++) {
      const double dr = dUh[2 * ((size_t)k * ne + e)], di = dUh[2 * ((size_t)k * ne + e) + 1];
      acc += U_bar[e].re * dr + U_bar[e].im * di;
    }
    theta_bar[k] = acc;
  }
  return TT_OK;
}

int tt_run_swp_derivative(const tt_run* run, const double* dVu, const double* dVc, double* dC_unco, double* dC_coup,
                          double* de_unco, double* de_coup, double* dE_bound) {
  if (!run || !dVu || (run->swp.n_coup && !dVc)) return fail(TT_ERR_BADARG, "null argument");
  SWPStates d;
  swp_derivative(run->fwp, run->V_unco, run->V_coup, run->swp, dVu, dVc, d);
  if (dC_unco) std::memcpy(dC_unco, d.C_unco.data(), sizeof(double) * d.C_unco.size());
  if (dC_coup) std::memcpy(dC_coup, d.C_coup.data(), sizeof(double) * d.C_coup.size());
  if (de_unco) std::memcpy(de_unco, d.e_unco.data(), sizeof(double) * d.e_unco.size());
  if (de_coup) std::memcpy(de_coup, d.e_coup.data(), sizeof(double) * d.e_coup.size());
  if (dE_bound) *dE_bound = d.E_bound;
  return TT_OK;
}

int tt_run_num_lecs(const tt_run* run, int* n_lecs, double* values) {
  if (!run || !n_lecs) return fail(TT_ERR_BADARG, "null argument");
  *n_lecs = num_lecs(run->rp.potential_model);
  if (values) {
    const std::vector<double> v = nominal_lecs(run->rp.potential_model);
    for (int k = 0; k < *n_lecs; k++)
      values[k] = v[k] + (k < (int)run->rp.lec_offsets.size() ? run->rp.lec_offsets[k] : 0.0);
  }
  return TT_OK;
}

int tt_run_lec_derivative(const tt_run* run, int k, double* dVu, double* dVc) {
  if (!run || !dVu || (run->swp.n_coup && !dVc)) return fail(TT_ERR_BADARG, "null argument");
  const int nl = num_lecs(run->rp.potential_model);
  if (k < 0 || k >= nl) return fail(TT_ERR_BADARG, "LEC index out of range");
  const std::vector<double> nom = nominal_lecs(run->rp.potential_model);
  // V is linear in the contact constants: any step gives the exact derivative
  const double h = std::max(std::fabs(nom[k]), 1e-6);
  std::vector<double> up[2], uc[2];
  for (int sgn = 0; sgn < 2; sgn++) {
    RunParams rp = run->rp;
    rp.lec_offsets.resize(nl, 0.0);
    rp.lec_offsets[k] += sgn == 0 ? h : -h;
    std::string err;
    if (!potential_matrices(rp, run->fwp, run->pw, up[sgn], uc[sgn], &err)) return fail(TT_ERR_BADARG, err);
  }
  for (size_t i = 0; i < up[0].size(); i++) dVu[i] = (up[0][i] - up[1][i]) / (2 * h);
  for (size_t i = 0; i < uc[0].size(); i++) dVc[i] = (uc[0][i] - uc[1][i]) / (2 * h);
  return TT_OK;
}

int tt_run_release_channel(tt_run* run, int chn) {
  int s = check_chn(run, chn);
  if (s) return s;
  run->chn[chn] = ChannelState();
  return TT_OK;
}

int tt_run_release_A(tt_run* run, int chn) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (run->chn[chn].solver) run->chn[chn].solver->release_A();
  run->chn[chn].have_A = false;
  run->chn[chn].have_G = false;
  return TT_OK;
}

int tt_run_timer_start(tt_run* run) {
  if (!run) return fail(TT_ERR_BADARG, "null run");
  cudaStream_t st = run_stream(run);
  if (!run->ev0) TT_CUDA_TRY(cudaEventCreate(&run->ev0));
  if (!run->ev1) TT_CUDA_TRY(cudaEventCreate(&run->ev1));
  TT_CUDA_TRY(cudaEventRecord(run->ev0, st));
  return TT_OK;
}

int tt_run_timer_stop(tt_run* run, double* ms) {
  if (!run || !ms || !run->ev0) return fail(TT_ERR_BADARG, "timer not started");
  TT_CUDA_TRY(cudaEventRecord(run->ev1, run_stream(run)));
  TT_CUDA_TRY(cudaEventSynchronize(run->ev1));
  float f = 0;
  TT_CUDA_TRY(cudaEventElapsedTime(&f, run->ev0, run->ev1));
  *ms = f;
  return TT_OK;
}

int tt_run_get_P123_csr(const tt_run* run, int chn, int64_t* rowptr, int32_t* col, double* val) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!run->chn[chn].have_P) return fail(TT_ERR_BADARG, "P123 not built");
  const DeviceCSR& P = run->chn[chn].solver->P();
  if (rowptr && cudaMemcpy(rowptr, P.rowptr.ptr, sizeof(int64_t) * (P.n + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy failed");
  if (P.nnz && col && cudaMemcpy(col, P.col.ptr, sizeof(int32_t) * P.nnz, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy failed");
  if (P.nnz && val && cudaMemcpy(val, P.val.ptr, sizeof(double) * P.nnz, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy failed");
  return TT_OK;
}

int tt_run_get_A(const tt_run* run, int chn, double* A) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!run->chn[chn].have_A || !A) return fail(TT_ERR_BADARG, "A not built");
  const size_t n = run->chn[chn].solver->n;
  if (cudaMemcpy(A, run->chn[chn].solver->A(), sizeof(double) * n * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy failed");
  return TT_OK;
}

int tt_run_get_G(const tt_run* run, int chn, tt_complex* G) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!run->chn[chn].have_G || !G) return fail(TT_ERR_BADARG, "resolvent not built");
  const size_t n = run->chn[chn].solver->n, nE = run->chn[chn].solver->nE();
  if (cudaMemcpy(G, run->chn[chn].solver->G(), sizeof(tt_complex) * n * nE, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(TT_ERR_CUDA, "copy failed");
  return TT_OK;
}

int tt_run_get_host_array(const tt_run* run, int chn, int which, void* buf, size_t* count) {
  if (!run || !count) return fail(TT_ERR_BADARG, "null argument");
  auto put_d = [&](const std::vector<double>& v) {
    *count = v.size();
    if (buf) std::memcpy(buf, v.data(), sizeof(double) * v.size());
    return TT_OK;
  };
  switch (which) {
    case 0: {
      int s = check_chn(run, chn);
      if (s) return s;
      const PWChannel c = channel_view(run->pw, chn);
      *count = (size_t)c.Nalpha * 9;
      if (buf) {
        int* o = (int*)buf;
        for (int a = 0; a < c.Nalpha; a++) {
          const int v[9] = {c.L_2N[a], c.S_2N[a], c.J_2N[a], c.T_2N[a], c.L_1N[a],
                            c.two_J_1N[a], c.two_J_3N[a], c.two_T_3N[a], c.P_3N[a]};
          std::memcpy(o + 9 * a, v, sizeof(v));
        }
      }
      return TT_OK;
    }
    case 1: return put_d(run->fwp.p_WP);
    case 2: return put_d(run->fwp.q_WP);
    case 3: return put_d(run->V_unco);
    case 4: return put_d(run->V_coup);
    case 5: return put_d(run->swp.C_unco);
    case 6: return put_d(run->swp.C_coup);
    case 7: return put_d(run->swp.e_unco);
    case 8: return put_d(run->swp.e_coup);
    default: return fail(TT_ERR_BADARG, "unknown host array");
  }
}

int tt_run_write_U_table(const tt_run* run, int chn, const tt_complex* U, const char* path) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U || !path) return fail(TT_ERR_BADARG, "null argument");
  const PWChannel c = channel_view(run->pw, chn);
  const std::vector<int> deut = deuteron_indices(c);
  const size_t nd = deut.size(), nE = run->os.q_com_idx.size();
  std::ofstream f(path);
  if (!f) return fail(TT_ERR_IO, std::string("cannot open ") + path);
  // layout of store_U_matrix_elements_txt, disk_io_routines.cpp:759-913
  f << std::setprecision(8);
  f << "# Elastic Nd-scattering U-matrix elements in a wave-packet, Jj-scheme representation. \n# \n";
  f << "# The calculations below were done for: \n";
  f << "# JP:          " << c.two_J_3N[0] << "/2" << (c.P_3N[0] == 1 ? "+" : "-") << "\n";
  f << "# Potential:   " << run->rp.potential_model << "\n";
  f << "# Np:          " << run->fwp.Np_WP << " \n";
  f << "# Nq:          " << run->fwp.Nq_WP << " \n";
  f << "# Particles:   nd-scattering\n";
  f << "# Deuteron BE: " << run->swp.E_bound << " MeV \n# \n";
  f << "# Symbol definitions: \n";
  static const char* const kSymbols[][2] = {
      {"Uij:", "U-matrix element in MeV with row-idx i and col-idx j (NOTE in wave-packet representation!)"},
      {"l:", "Spectator nucleon orbital angular momentum"},
      {"j:", "Spectator nucleon total angular momentum"},
      {"Tlab:", "Laboratory scattering/kinetic energy"},
      {"Ecm:", "Centre-of-mass scattering/kinetic energy"},
      {"q_idx:", "Index of on-shell q-momentum bin correponding to Tlab/Ecm"}};
  for (const auto& sym : kSymbols) {
    std::string tag = sym[0];
    tag.resize(7, ' ');
    f << "# " << tag << sym[1] << "  \n";
  }
  f << "# \n";
  f << "# ################################################################################################### \n";
  f << std::right << std::scientific << std::setprecision(16);
  const char* h1[] = {"Name", "row-idx", "col-idx", "l'", "2*j'", "l", "2*j"};
  f << "#";
  for (const char* h : h1) f << std::setw(10) << h;
  f << "\n";
  for (size_t r = 0; r < nd; r++)
    for (size_t cc = 0; cc < nd; cc++) {
      f << " " << std::setw(10) << ("U" + std::to_string(r) + std::to_string(cc)) << std::setw(10) << r
        << std::setw(10) << cc << std::setw(10) << c.L_1N[deut[r]] << std::setw(10) << c.two_J_1N[deut[r]]
        << std::setw(10) << c.L_1N[deut[cc]] << std::setw(10) << c.two_J_1N[deut[cc]] << "\n";
    }
  f << "# ################################################################################################### \n";
  // the second table's header names nine U columns whatever nd is, as there
  f << "#" << std::setw(24) << "Tlab [MeV]" << std::setw(24) << "Ecm [MeV]" << std::setw(10) << "q_idx";
  for (int r = 0; r < 3; r++)
    for (int cc = 0; cc < 3; cc++) f << std::setw(50) << ("U" + std::to_string(r) + std::to_string(cc) + " [MeV]");
  f << "\n";
  const auto fmt = signed_scientific;
  for (size_t j = 0; j < nE; j++) {
    f << " " << std::setw(24) << run->os.T_lab[j] << std::setw(24) << run->os.E_com[j] << std::setw(10)
      << run->os.q_com_idx[j];
    for (size_t r = 0; r < nd; r++)
      for (size_t cc = 0; cc < nd; cc++) {
        const tt_complex u = U[r * nd * nE + cc * nE + j];
        f << std::setw(50) << (fmt(u.re) + fmt(u.im) + "j");
      }
    f << "\n";
  }
  f << "# ################################################################################################### \n";
  f << std::endl;
  return TT_OK;
}


// ---- breakup channels ----

// the channel's breakup cells: those located at creation, else located now
static int run_breakup_cells(const tt_run* run, int chn, BreakupCells& out, const BreakupCells** cells) {
  if (!run->bu.empty()) {
    *cells = &run->bu[chn];
    return TT_OK;
  }
  std::string err;
  if (!find_breakup_cells(run->rp, channel_view(run->pw, chn), run->swp, run->os.E_com, out, &err))
    return fail(TT_ERR_BADARG, err);
  *cells = &out;
  return TT_OK;
}

int tt_run_breakup_cells(const tt_run* run, int chn, int* num_cells, int* start, int* cells) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!num_cells) return fail(TT_ERR_BADARG, "null num_cells");
  BreakupCells local;
  const BreakupCells* bu = nullptr;
  TT_TRY(run_breakup_cells(run, chn, local, &bu));
  *num_cells = bu->count();
  if (start) std::memcpy(start, bu->start.data(), sizeof(int) * bu->start.size());
  if (cells) std::memcpy(cells, bu->cells.data(), sizeof(int) * bu->cells.size());
  return TT_OK;
}

int tt_run_solve_breakup(tt_run* run, int chn, tt_complex* U, tt_complex* U_BU, tt_solve_report* report) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!U || !U_BU) return fail(TT_ERR_BADARG, "null U or U_BU");
  BreakupCells local;
  const BreakupCells* bu = nullptr;
  TT_TRY(run_breakup_cells(run, chn, local, &bu));
  double msA = 0;
  if (!run->chn[chn].have_A) TT_TRY(tt_run_build_A(run, chn, &msA));
  if (!run->chn[chn].have_G) TT_TRY(tt_run_build_resolvent(run, chn));
  const std::vector<int> deut = deuteron_indices(channel_view(run->pw, chn));
  std::vector<double> Uh, UBh;
  BreakupRequest bq;
  bq.cells = bu;
  bq.U_BU = &UBh;
  SolveReport rep;
  s = run->chn[chn].solver->solve(run->os.q_com_idx, deut, options_of(run->rp, TT_PRECISION_PADE), Uh, &rep,
                                  run_stream(run), nullptr, &bq);
  fill_report(rep, msA, report);
  if (s != TT_OK) return s;
  std::memcpy(U, Uh.data(), sizeof(double) * Uh.size());
  if (!UBh.empty()) std::memcpy(U_BU, UBh.data(), sizeof(double) * UBh.size());
  return TT_OK;
}

int tt_run_write_U_BU_table(const tt_run* run, int chn, const tt_complex* U_BU, const char* path) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!path) return fail(TT_ERR_BADARG, "null path");
  BreakupCells local;
  const BreakupCells* bu = nullptr;
  TT_TRY(run_breakup_cells(run, chn, local, &bu));
  BreakupTableInput in;
  in.rp = &run->rp;
  in.ch = channel_view(run->pw, chn);
  in.swp = &run->swp;
  in.os = &run->os;
  in.deut = deuteron_indices(in.ch);
  in.bu = bu;
  if (!U_BU && !in.deut.empty() && bu->count() > 0) return fail(TT_ERR_BADARG, "null U_BU");
  in.U_BU = reinterpret_cast<const double*>(U_BU);
  std::ofstream f(path);
  if (!f) return fail(TT_ERR_IO, std::string("cannot open ") + path);
  std::string err;
  if (!write_breakup_table(f, in, &err)) return fail(TT_ERR_BADARG, err);
  return f ? TT_OK : fail(TT_ERR_IO, std::string("write failed: ") + path);
}

// ---- P123 files in the reference's HDF5 layout ----

static int p123_file_header(const PWChannel& c, int Np_WP, const double* p_WP, int Nq_WP, const double* q_WP,
                            P123H5& f) {
  if (c.Nalpha <= 0 || Np_WP <= 0 || Nq_WP <= 0 || !p_WP || !q_WP) return fail(TT_ERR_BADARG, "empty state space");
  f.Nalpha = c.Nalpha;
  f.Np_WP = Np_WP;
  f.Nq_WP = Nq_WP;
  f.p_WP.assign(p_WP, p_WP + Np_WP + 1);
  f.q_WP.assign(q_WP, q_WP + Nq_WP + 1);
  // write_PW_statespace_to_h5 (CPP/disk_io_routines.cpp:1474-1545): the
  // channel's J and parity in every record
  f.pw.resize((size_t)c.Nalpha * kPwFields);
  for (int a = 0; a < c.Nalpha; a++) {
    const int32_t rec[kPwFields] = {a,           c.L_2N[a],     c.S_2N[a],        c.J_2N[a],        c.T_2N[a],
                                    c.L_1N[a],   c.two_J_1N[a], c.two_T_3N[a],    c.two_J_3N[0],    c.P_3N[0]};
    std::memcpy(&f.pw[(size_t)a * kPwFields], rec, sizeof rec);
  }
  return TT_OK;
}

// the reference's integrity checks on a read file (CPP/disk_io_routines.cpp:1209-1270)
static int p123_file_matches(const P123H5& want, const P123H5& got) {
  if (got.Nalpha != want.Nalpha || got.Np_WP != want.Np_WP || got.Nq_WP != want.Nq_WP)
    return fail(TT_ERR_BADARG, "File-read P123 state-space dimensions (Nalpha, Nq_WP, Np_WP) mismatch.");
  if (got.p_WP != want.p_WP) return fail(TT_ERR_BADARG, "File-read P123 p-momentum boundaries mismatch.");
  if (got.q_WP != want.q_WP) return fail(TT_ERR_BADARG, "File-read P123 q-momentum boundaries mismatch.");
  for (size_t e = 0; e < want.pw.size(); e++)  // every field but the record index
    if (e % kPwFields != 0 && got.pw[e] != want.pw[e])
      return fail(TT_ERR_BADARG, "File-read P123 PW state-space mismatch.");
  return TT_OK;
}

int tt_store_P123_h5(const char* filename, const double* val, const int* row, const int* col, size_t nnz,
                     const tt_fwp_states* fwp, const tt_pw_states* pw) {
  if (!filename || !fwp || !pw || (nnz && (!val || !row || !col))) return fail(TT_ERR_BADARG, "null argument");
  P123H5 f;
  int s = p123_file_header(view_of(pw), fwp->Np_WP, fwp->p_WP_array, fwp->Nq_WP, fwp->q_WP_array, f);
  if (s) return s;
  f.nnz = nnz;
  std::string err;
  if (!h5_write_p123(filename, f, row, col, val, &err)) return fail(TT_ERR_IO, err);
  return TT_OK;
}

int tt_read_P123_h5(const char* filename, double** val, int** row, int** col, size_t* nnz, const tt_fwp_states* fwp,
                    const tt_pw_states* pw) {
  if (!filename || !val || !row || !col || !nnz || !fwp || !pw) return fail(TT_ERR_BADARG, "null argument");
  P123H5 want, got;
  int s = p123_file_header(view_of(pw), fwp->Np_WP, fwp->p_WP_array, fwp->Nq_WP, fwp->q_WP_array, want);
  if (s) return s;
  std::string err;
  if (!h5_read_p123(filename, got, &err)) return fail(TT_ERR_IO, err);
  s = p123_file_matches(want, got);
  if (s) return s;
  const size_t m = (size_t)got.nnz;
  *val = (double*)std::malloc(sizeof(double) * std::max<size_t>(m, 1));
  *row = (int*)std::malloc(sizeof(int) * std::max<size_t>(m, 1));
  *col = (int*)std::malloc(sizeof(int) * std::max<size_t>(m, 1));
  if (!*val || !*row || !*col) {
    std::free(*val);
    std::free(*row);
    std::free(*col);
    *val = nullptr;
    *row = *col = nullptr;
    return fail(TT_ERR_NOMEM, "host allocation for P123 failed");
  }
  if (m) {
    std::memcpy(*val, got.val.data(), sizeof(double) * m);
    std::memcpy(*row, got.row.data(), sizeof(int) * m);
    std::memcpy(*col, got.col.data(), sizeof(int) * m);
  }
  *nnz = m;
  return TT_OK;
}

int tt_P123_h5_filename(char* buf, size_t cap, const char* folder, const tt_pw_states* pw, int Np_WP, int Nq_WP) {
  if (!buf || !folder || !pw || !pw->two_J_3N_array || !pw->P_3N_array) return fail(TT_ERR_BADARG, "null argument");
  const std::string name =
      p123_h5_filename(folder, pw->two_J_3N_array[0], pw->P_3N_array[0], Np_WP, Nq_WP, pw->J_2N_max);
  if (name.size() + 1 > cap) return fail(TT_ERR_BADARG, "file name buffer too small");
  std::memcpy(buf, name.c_str(), name.size() + 1);
  return TT_OK;
}

int tt_run_store_P123_h5(const tt_run* run, int chn, const char* filename) {
  int s = check_chn(run, chn);
  if (s) return s;
  if (!run->chn[chn].have_P) return fail(TT_ERR_BADARG, "P123 not built");
  const PWChannel c = channel_view(run->pw, chn);
  P123H5 f;
  s = p123_file_header(c, run->fwp.Np_WP, run->fwp.p_WP.data(), run->fwp.Nq_WP, run->fwp.q_WP.data(), f);
  if (s) return s;
  const DeviceCSR& P = run->chn[chn].solver->P();
  std::vector<int64_t> rowptr(P.n + 1);
  f.nnz = (uint64_t)P.nnz;
  f.row.resize(f.nnz);
  f.col.resize(f.nnz);
  f.val.resize(f.nnz);
  if (cudaMemcpy(rowptr.data(), P.rowptr.ptr, sizeof(int64_t) * (P.n + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
      (f.nnz && (cudaMemcpy(f.col.data(), P.col.ptr, sizeof(int32_t) * f.nnz, cudaMemcpyDeviceToHost) != cudaSuccess ||
                 cudaMemcpy(f.val.data(), P.val.ptr, sizeof(double) * f.nnz, cudaMemcpyDeviceToHost) != cudaSuccess)))
    return fail(TT_ERR_CUDA, "copy of P123 failed");
  for (int r = 0; r < P.n; r++)
    for (int64_t e = rowptr[r]; e < rowptr[r + 1]; e++) f.row[e] = r;
  const std::string path = filename ? std::string(filename)
                                    : p123_h5_filename(run->rp.P123_folder, c.two_J_3N[0], c.P_3N[0], run->fwp.Np_WP,
                                                       run->fwp.Nq_WP, c.J_2N_max);
  std::string err;
  if (!h5_write_p123(path, f, nullptr, nullptr, nullptr, &err)) return fail(TT_ERR_IO, err);
  return TT_OK;
}

int tt_run_load_P123_h5(tt_run* run, int chn, const char* filename, int64_t* nnz) {
  int s = check_chn(run, chn);
  if (s) return s;
  const PWChannel c = channel_view(run->pw, chn);
  P123H5 want, got;
  s = p123_file_header(c, run->fwp.Np_WP, run->fwp.p_WP.data(), run->fwp.Nq_WP, run->fwp.q_WP.data(), want);
  if (s) return s;
  const std::string path = filename ? std::string(filename)
                                    : p123_h5_filename(run->rp.P123_folder, c.two_J_3N[0], c.P_3N[0], run->fwp.Np_WP,
                                                       run->fwp.Nq_WP, c.J_2N_max);
  std::string err;
  if (!h5_read_p123(path, got, &err)) return fail(TT_ERR_IO, err);
  s = p123_file_matches(want, got);
  if (s) return s;
  // the file holds the reference's row-major sorted COO; rebuild the row pointers
  const int64_t n = (int64_t)want.Nalpha * want.Np_WP * want.Nq_WP;
  const int64_t m = (int64_t)got.nnz;
  std::vector<int64_t> rowptr(n + 1, 0);
  for (int64_t e = 0; e < m; e++) {
    const int32_t r = got.row[e], cc = got.col[e];
    if (r < 0 || r >= n || cc < 0 || cc >= n) return fail(TT_ERR_BADARG, path + ": P123 index out of range");
    if (e > 0 && (r < got.row[e - 1] || (r == got.row[e - 1] && cc <= got.col[e - 1])))
      return fail(TT_ERR_BADARG, path + ": P123 entries are not in row-major order");
    rowptr[r + 1]++;
  }
  for (int64_t r = 0; r < n; r++) rowptr[r + 1] += rowptr[r];
  TT_TRY(ensure_solver(run, chn));
  cudaStream_t st = run_stream(run);
  TT_TRY(run->chn[chn].solver->set_P_host_csr(rowptr.data(), got.col.data(), got.val.data(), m, st));
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(TT_ERR_CUDA, "upload of P123 failed");
  run->chn[chn].have_P = true;
  run->chn[chn].have_A = false;
  if (nnz) *nnz = m;
  return TT_OK;
}

}  // extern "C"
