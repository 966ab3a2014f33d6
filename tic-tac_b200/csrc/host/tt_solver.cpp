// Host orchestration of the per-channel Faddeev solve.  See tt_solver.h.
#include "tt_solver.h"

#include <chrono>
#include <complex>
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <map>

#include "../cuda/tt_lu_internal.h"
#include "tt_panel_table.h"

namespace tt {

namespace {

struct AlphaBlock {
  bool coupled;
  int chn;
  int part;
};

// 2N block and part of one partial wave (make_resolvent.cpp:118-156).
bool alpha_block(const RunParams& rp, const PWChannel& ch, int a, AlphaBlock& out, std::string* err) {
  const int L = ch.L_2N[a], S = ch.S_2N[a], J = ch.J_2N[a], T = ch.T_2N[a];
  const bool state_1S0 = (S == 0 && J == 0 && L == 0);
  const bool via_L = (rp.tensor_force && L != J && J != 0);
  const bool via_T = (state_1S0 && rp.isospin_breaking_1S0);
  if (via_L && via_T) {
    if (err) *err = "isospin-breaking in coupled channels is not supported";
    return false;
  }
  out.coupled = via_L || via_T;
  out.chn = unique_2N_idx(L, S, J, T, out.coupled, rp);
  if (via_L) out.part = (L < J) ? 0 : 1;
  else if (via_T) out.part = (ch.two_T_3N[a] == 1) ? 0 : 1;
  else out.part = 0;
  return true;
}

// Remaining relative error after a refinement step, per right-hand side: the
// last correction |dx|/|x| = c, or, once two corrections contract by
// rho = c / c_prev < 1/2, the rest of the geometric series c rho / (1 - rho).
// Returns the worst over the right-hand sides.
double refine_error_estimate(const std::vector<double>& cur, std::vector<double>& prev, bool have_prev) {
  double worst = 0;
  for (size_t k = 0; k < cur.size(); k++) {
    double e = cur[k];
    if (have_prev && prev[k] > 0 && cur[k] < 0.5 * prev[k]) {
      const double rho = cur[k] / prev[k];
      e = std::min(e, cur[k] * rho / (1 - rho));
    }
    if (!(cur[k] == cur[k])) e = cur[k];  // NaN stays NaN
    worst = std::max(worst, e);
    if (!(e == e)) worst = e;
  }
  prev = cur;
  return worst;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

bool channel_energy_offsets(const RunParams& rp, const PWChannel& ch, int Np, int n_unco, int n_coup,
                            int32_t* e_off, std::string* err) {
  for (int a = 0; a < ch.Nalpha; a++) {
    AlphaBlock ab;
    if (!alpha_block(rp, ch, a, ab, err)) return false;
    if (ab.chn < 0 || ab.chn >= (ab.coupled ? n_coup : n_unco)) {
      if (err) *err = "partial wave maps to a 2N channel outside the SWP state arrays";
      return false;
    }
    e_off[a] = ab.coupled ? n_unco * (Np + 1) + ab.chn * 2 * (Np + 1) + ab.part * (Np + 1) : ab.chn * (Np + 1);
  }
  return true;
}

bool build_channel_layout(const RunParams& rp, const PWChannel& ch, const SWPStates& swp,
                          const std::vector<double>& V_unco, const std::vector<double>& V_coup, ChannelLayout& L,
                          std::string* err) {
  const int Na = ch.Nalpha, Np = swp.Np_WP;
  L = ChannelLayout();
  L.Nalpha = Na;
  L.Np = Np;
  L.Nq = swp.Nq_WP;
  L.e_swp = swp.e_unco;
  L.e_swp.insert(L.e_swp.end(), swp.e_coup.begin(), swp.e_coup.end());
  const int e_coup_base = (int)swp.e_unco.size();
  std::map<std::pair<int, int>, int> blocks;  // (coupled, chn) -> block index
  for (int a = 0; a < Na; a++) {
    AlphaBlock ab;
    if (!alpha_block(rp, ch, a, ab, err)) return false;
    const auto key = std::make_pair(ab.coupled ? 1 : 0, ab.chn);
    auto it = blocks.find(key);
    int b;
    if (it == blocks.end()) {
      b = (int)L.blk_dim.size();
      blocks[key] = b;
      const int dim = ab.coupled ? 2 * Np : Np;
      const double* Cs = ab.coupled ? &swp.C_coup[(size_t)ab.chn * dim * dim] : &swp.C_unco[(size_t)ab.chn * dim * dim];
      const double* Vs = ab.coupled ? &V_coup[(size_t)ab.chn * dim * dim] : &V_unco[(size_t)ab.chn * dim * dim];
      L.blk_dim.push_back(dim);
      L.blk_off.push_back((int64_t)L.C.size());
      L.C.insert(L.C.end(), Cs, Cs + (size_t)dim * dim);
      // VC = V . C (row-major), the dot_MM products of solve_faddeev.cpp:1818-1846
      std::vector<double> vc((size_t)dim * dim, 0.0);
      for (int i = 0; i < dim; i++)
        for (int k = 0; k < dim; k++) {
          const double v = Vs[(size_t)i * dim + k];
          if (v == 0.0) continue;
          for (int j = 0; j < dim; j++) vc[(size_t)i * dim + j] += v * Cs[(size_t)k * dim + j];
        }
      L.VC.insert(L.VC.end(), vc.begin(), vc.end());
    } else {
      b = it->second;
    }
    L.blk.push_back(b);
    L.part.push_back(ab.part);
    L.dim.push_back(L.blk_dim[b]);
    L.e_off.push_back(ab.coupled ? e_coup_base + ab.chn * 2 * (Np + 1) + ab.part * (Np + 1) : ab.chn * (Np + 1));
  }
  // coupling partners (non-NULL entries of the C^T / VC pointer tables,
  // solve_faddeev.cpp:1690-1699)
  L.cpl_off.push_back(0);
  for (int r = 0; r < Na; r++) {
    int cnt = 0;
    for (int c = 0; c < Na; c++) {
      const bool check_T = ch.T_2N[r] == ch.T_2N[c];
      const bool check_J = ch.J_2N[r] == ch.J_2N[c];
      const bool check_S = ch.S_2N[r] == ch.S_2N[c];
      const bool check_L = (rp.tensor_force && std::abs(ch.L_2N[r] - ch.L_2N[c]) <= 2) || ch.L_2N[r] == ch.L_2N[c];
      const bool check_l = ch.L_1N[r] == ch.L_1N[c];
      const bool check_j = ch.two_J_1N[r] == ch.two_J_1N[c];
      if (check_T && check_J && check_S && check_L && check_l && check_j) {
        if (L.blk[r] != L.blk[c]) {
          if (err) *err = "inconsistent 2N block structure between coupled partial waves";
          return false;
        }
        L.cpl.push_back(c);
        cnt++;
      }
    }
    if (cnt > 2) {
      if (err) *err = "more than two coupled partial waves per 2N block";
      return false;
    }
    L.cpl_off.push_back((int32_t)L.cpl.size());
  }
  return true;
}

int ChannelSolver::setup(const ChannelLayout& L, const std::vector<double>& q_WP, cudaStream_t st) {
  n = L.Nalpha * L.Np * L.Nq;
  return L_.upload(L, q_WP, st);
}

int ChannelSolver::set_P_device(DeviceCSR&& P) {
  if (P.n != n) {
    set_error("P123 dimension does not match the channel");
    return TT_ERR_BADARG;
  }
  P_ = std::move(P);
  aoff_.release();
  return TT_OK;
}

int ChannelSolver::set_P_host_csr(const int64_t* rowptr, const int32_t* col, const double* val, int64_t nnz,
                                  cudaStream_t st) {
  P_.n = n;
  P_.nnz = nnz;
  aoff_.release();
  TT_TRY(P_.rowptr.upload(rowptr, (size_t)n + 1, st));
  TT_TRY(P_.col.upload(col, (size_t)std::max<int64_t>(nnz, 0), st));
  TT_TRY(P_.val.upload(val, (size_t)std::max<int64_t>(nnz, 0), st));
  return TT_OK;
}

int ChannelSolver::set_P_host_csc(const double* val, const int32_t* row, const uint64_t* colptr, int64_t nnz,
                                  cudaStream_t st) {
  aoff_.release();
  return csc_to_csr_device(val, row, colptr, nnz, n, P_, st);
}

int ChannelSolver::build_A(cudaStream_t st, double* ms) {
  auto t0 = std::chrono::steady_clock::now();
  TT_TRY(A_.alloc((size_t)n * n));
  if (!aoff_.ptr && n > 0) {
    TT_TRY(aoff_.alloc((size_t)n * (L_.Nalpha + 1)));
    TT_TRY(alpha_offsets_device(L_, P_, aoff_.ptr, st));
  }
  TT_TRY(build_A_device(L_, P_, aoff_.ptr, A_.ptr, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  if (ms) *ms = ms_since(t0);
  return TT_OK;
}

int ChannelSolver::resolvent(const std::vector<double>& E, cudaStream_t st) {
  nE_ = (int)E.size();
  Eh_ = E;
  TT_TRY(E_.upload(E, st));
  TT_TRY(G_.alloc((size_t)2 * n * std::max(1, nE_)));
  TT_TRY(resolvent_device(L_, E_.ptr, nE_, G_.ptr, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  return TT_OK;
}

namespace {

using cd = std::complex<double>;

// Panel width of the complex64 LU for order n and tensor-core product.
int tuned_panel_width(int n, int product) {
  for (const PanelWidthRow& r : kPanelWidthTable)
    if (r.product == product && n <= r.n_max) return r.width;
  return 512;
}

// Determinant by LU with partial pivoting, pivots chosen by |re| + |im| as
// LAPACK's zgetrf does (determinant, CPP/General_functions/matrix_routines.cpp:82-101).
cd determinant(std::vector<cd> a, int n) {
  cd det = 1.0;
  for (int k = 0; k < n; k++) {
    int p = k;
    double best = -1;
    for (int i = k; i < n; i++) {
      const double v = std::fabs(a[i * n + k].real()) + std::fabs(a[i * n + k].imag());
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (a[p * n + k] == cd(0.0)) return 0.0;
    if (p != k) {
      for (int c = 0; c < n; c++) std::swap(a[k * n + c], a[p * n + c]);
      det = -det;
    }
    det *= a[k * n + k];
    for (int i = k + 1; i < n; i++) {
      const cd l = a[i * n + k] / a[k * n + k];
      for (int c = k + 1; c < n; c++) a[i * n + c] -= l * a[k * n + c];
    }
  }
  return det;
}

// [N/M] Pade approximant at z of the series with coefficients a[0 .. N+M]
// (pade_approximant, CPP/solve_faddeev.cpp:271-296)
cd pade_approximant(const cd* a, int N, int M, cd z) {
  std::vector<cd> P((M + 1) * (M + 1)), Q((M + 1) * (M + 1));
  for (int r = 0; r < M; r++)
    for (int c = 0; c < M + 1; c++) P[r * (M + 1) + c] = Q[r * (M + 1) + c] = a[N - M + 1 + r + c];
  for (int c = 0; c < M + 1; c++) {
    Q[M * (M + 1) + c] = std::pow(z, M - c);
    cd s = 0.0;
    for (int j = M - c; j < N + 1; j++) s += a[j - (M - c)] * std::pow(z, j);
    P[M * (M + 1) + c] = s;
  }
  return determinant(P, M + 1) / determinant(Q, M + 1);
}

}  // namespace

// The reference's production solver (pade_method_solve,
// CPP/solve_faddeev.cpp:440-1444): on-shell rows r_0 = A[row, :] and
// r_{n+1} = (r_n o G_j) A give the Neumann coefficients a_n of
// U = sum_n A (G A)^n; [N/N] Pade approximants at z = 1 for N = 0 .. 14 are
// formed as two new terms arrive, and an element stops at the first of the
// reference's criteria (N = 14; no better difference in the last 4 orders;
// smallest difference of consecutive approximants < 1e-6 |best| or < 1e-7).
int ChannelSolver::solve_pade(const std::vector<int>& q_idx, const std::vector<int>& deut, std::vector<double>& U,
                              SolveReport& r, cudaStream_t st, const BreakupRequest* bu) {
  constexpr int NM_MAX = 14, NTERMS = 2 * NM_MAX + 1;
  auto t0 = std::chrono::steady_clock::now();
  const int nE = (int)q_idx.size(), nd = (int)deut.size();
  const int Nq = L_.Nq, Np = L_.Np;
  const int nrows = nd * nE, nel_el = nd * nd * nE;
  // breakup elements (d, cell) of the cells inside the grid follow the
  // elastic ones; bu_slot maps them to U_BU's [d][cell] index
  const BreakupCells* cells = bu ? bu->cells : nullptr;
  const int nb = cells ? cells->count() : 0;
  std::vector<int32_t> bu_row, bu_col, bu_slot;
  for (int d = 0; d < nd && nb; d++)
    for (int j = 0; j < nE; j++)
      for (int b = cells->start[j]; b < cells->start[j + 1]; b++) {
        if (!cells->inside(b, L_.Nalpha, Nq, Np)) continue;
        const int32_t* c = &cells->cells[(size_t)3 * b];
        bu_row.push_back(d * nE + j);
        bu_col.push_back(c[0] * Nq * Np + c[1] * Np + c[2]);
        bu_slot.push_back(d * nb + b);
      }
  const int nel = nel_el + (int)bu_slot.size();
  std::vector<int32_t> rows(nrows), erow(nrows), prow(nel), pcol(nel);
  for (int d = 0; d < nd; d++)
    for (int j = 0; j < nE; j++) {
      rows[d * nE + j] = deut[d] * Nq * Np + q_idx[j] * Np;
      erow[d * nE + j] = j;
    }
  for (int dr = 0; dr < nd; dr++)
    for (int dc = 0; dc < nd; dc++)
      for (int j = 0; j < nE; j++) {
        const int e = dr * nd * nE + dc * nE + j;
        prow[e] = dr * nE + j;
        pcol[e] = deut[dc] * Nq * Np + q_idx[j] * Np;
      }
  for (size_t k = 0; k < bu_slot.size(); k++) {
    prow[nel_el + k] = bu_row[k];
    pcol[nel_el + k] = bu_col[k];
  }
  for (int e = 0; e < nel; e++)  // every picked element inside the on-shell rows of R
    if (prow[e] < 0 || prow[e] >= nrows || pcol[e] < 0 || pcol[e] >= n) {
      set_error("Pade element outside the on-shell rows");
      return TT_ERR_BADARG;
    }
  DevBuf<int32_t> d_rows, d_erow, d_prow, d_pcol;
  DevBuf<double> R, V, picked;
  TT_TRY(d_rows.upload(rows, st));
  TT_TRY(d_erow.upload(erow, st));
  TT_TRY(d_prow.upload(prow, st));
  TT_TRY(d_pcol.upload(pcol, st));
  TT_TRY(R.alloc((size_t)2 * n * nrows));
  TT_TRY(V.alloc((size_t)2 * n * nrows));
  TT_TRY(picked.alloc((size_t)2 * nel));
  std::vector<cd> a((size_t)nel * NTERMS, 0.0), pa((size_t)nel * (NM_MAX + 1), 0.0), hv(nel);
  std::vector<char> conv(nel, 0);
  std::vector<int> best(nel, 0);
  auto extract = [&](int term) -> int {
    TT_TRY(pick_device(R.ptr, n, d_prow.ptr, d_pcol.ptr, nel, picked.ptr, st));
    TT_CUDA_TRY(cudaMemcpyAsync(hv.data(), picked.ptr, sizeof(cd) * nel, cudaMemcpyDeviceToHost, st));
    TT_CUDA_TRY(cudaStreamSynchronize(st));
    for (int e = 0; e < nel; e++)
      if (!conv[e]) a[(size_t)e * NTERMS + term] = hv[e];
    return TT_OK;
  };
  TT_TRY(gather_rows_device(A_.ptr, n, d_rows.ptr, nrows, R.ptr, st));
  TT_TRY(extract(0));
  int nconv = 0, top = 0;
  double worst_diff = 0;
  for (int NM = 0; NM <= NM_MAX && nconv < nel; NM++) {
    top = NM;
    for (int term = 2 * NM - 1; term <= 2 * NM; term++) {
      if (term <= 0) continue;
      TT_TRY(scale_rows_device(R.ptr, G_.ptr, d_erow.ptr, n, nrows, V.ptr, st));
      for (int k0 = 0; k0 < nrows; k0 += 8)
        TT_TRY(gemv_t_device(A_.ptr, n, V.ptr + (size_t)2 * n * k0, std::min(8, nrows - k0),
                             R.ptr + (size_t)2 * n * k0, st));
      TT_TRY(extract(term));
    }
    for (int e = 0; e < nel; e++) {
      if (conv[e]) continue;
      cd* p = &pa[(size_t)e * (NM_MAX + 1)];
      p[NM] = pade_approximant(&a[(size_t)e * NTERMS], NM, NM, 1.0);
      int idx_best = 0;
      double min_diff = 1;
      for (int prev = 0; prev < NM; prev++) {
        // the reference compares approximant 0 with the slot before it, zero here
        const double d = std::abs(p[prev] - (prev > 0 ? p[prev - 1] : cd(0.0)));
        if (d < min_diff && d > 1e-15) {
          idx_best = prev;
          min_diff = d;
        }
      }
      const double d = std::abs(p[NM] - (NM > 0 ? p[NM - 1] : cd(0.0)));
      if (d < min_diff && d > 1e-15) {
        idx_best = NM;
        min_diff = d;
      }
      if (NM == NM_MAX || NM - idx_best > 4 || min_diff < 1e-6 * std::abs(p[idx_best]) || min_diff < 1e-7) {
        conv[e] = 1;
        best[e] = idx_best;
        nconv++;
        worst_diff = std::max(worst_diff, min_diff / std::max(1e-300, std::abs(p[idx_best])));
      }
    }
  }
  for (int e = 0; e < nel; e++) {
    const cd v = pa[(size_t)e * (NM_MAX + 1) + best[e]];
    double* out = e < nel_el ? &U[2 * (size_t)e] : &(*bu->U_BU)[2 * (size_t)bu_slot[e - nel_el]];
    out[0] = v.real();
    out[1] = v.imag();
  }
  r.ms_solve += ms_since(t0);
  r.refine_iters = top;           // highest [N/N] order formed
  r.final_correction = worst_diff;  // largest relative difference of consecutive approximants at the choice
  return TT_OK;
}

int ChannelSolver::adjoint_energy(int j, int nE, int nd, const double* Gj, const int32_t* d_rows, const int32_t* d_perm,
                                  double* tmp, const double* x, const SolveOptions& opt, void* F,
                                  TrsvBlocks<float2>& tbT32, TrsvBlocks<double2>& tbT64, double* lam, double* yT,
                                  double* rT, double* u, double* g, double* w, double* h, double* dots,
                                  const AdjointRequest& adj, SolveReport& r, cudaStream_t st) {
  auto t0 = std::chrono::steady_clock::now();
  // lambda_d' = (1 - A G)^{-T} e_d' with the factor transposed in place: the
  // forward solve and its refinement are done, and the next energy forms a new
  // L, so the adjoint needs no second n x n buffer
  auto solve_t = [&](double* v) -> int {
    if (opt.mixed)
      return lu_solve_transposed_device<float2>(static_cast<const float2*>(F), n, tbT32, d_perm, v, tmp, nd, st);
    return lu_solve_transposed_device<double2>(static_cast<const double2*>(F), n, tbT64, d_perm, v, tmp, nd, st);
  };
  if (opt.mixed) {
    TT_TRY(transpose_inplace_device<float2>(static_cast<float2*>(F), n, st));
    TT_TRY(lu_trsv_prepare<float2>(static_cast<const float2*>(F), n, tbT32, st, true));
  } else {
    TT_TRY(transpose_inplace_device<double2>(static_cast<double2*>(F), n, st));
    TT_TRY(lu_trsv_prepare<double2>(static_cast<const double2*>(F), n, tbT64, st, true));
  }
  TT_TRY(unit_rhs_device(d_rows, n, nd, lam, st));
  TT_TRY(solve_t(lam));
  if (opt.mixed) {
    // FP64 refinement: r = e - (lambda - G o (A^T lambda)), solve, lambda += r
    bool converged = false;
    int it = 0;
    double worst = 0;
    std::vector<double> ratio(nd), prev(nd, 0.0);
    for (it = 1; it <= opt.refine_max_iter; it++) {
      TT_TRY(gemv_t_device(A_.ptr, n, lam, nd, yT, st));
      TT_TRY(residual_t_device(lam, yT, Gj, d_rows, n, nd, rT, st));
      TT_TRY(solve_t(rT));
      TT_TRY(axpy_norms_device(lam, rT, n, nd, ratio.data(), st));
      worst = refine_error_estimate(ratio, prev, it > 1);
      if (!(worst == worst)) break;
      if (worst <= opt.refine_tol) {
        converged = true;
        break;
      }
    }
    r.adjoint_refine_iters = std::max(r.adjoint_refine_iters, std::min(it, opt.refine_max_iter));
    if (!converged) {
      set_error("refinement of the adjoint solve did not converge (last |dx|/|x| = " + std::to_string(worst) + ")");
      return TT_ERR_NOCONVERGE;
    }
  }
  // g = 2 P123^T OP(C) lambda, w = e + G o x
  TT_TRY(block_apply_device(L_, L_.C.ptr, lam, nd, u, st));
  TT_TRY(spmv_t_device(P_, u, nd, g, st));
  TT_TRY(make_w_device(x, Gj, d_rows, n, nd, w, st));
  // total derivative: with dA = OP(dC)^T (2P) OP(VC) + OP(C)^T (2P) OP(d(VC)) and
  // dU = lambda^T dA w + lambda^T A (dG o x), the extra pieces are
  // u2 = 2 P OP(VC) w and A^T lambda, once per energy
  DevBuf<double> u2, t2, dG;
  DevBuf<int32_t> zero_e;
  if (adj.total) {
    const size_t vec = (size_t)2 * n * nd;
    TT_TRY(u2.alloc(vec));
    TT_TRY(t2.alloc(vec));
    TT_TRY(dG.alloc((size_t)2 * n));
    TT_TRY(zero_e.upload(std::vector<int32_t>(nd, 0), st));
    TT_TRY(block_apply_device(L_, L_.VC.ptr, w, nd, t2.ptr, st));
    TT_TRY(spmv_device(P_, t2.ptr, nd, u2.ptr, st));
    TT_TRY(gemv_t_device(A_.ptr, n, lam, nd, yT, st));
  }
  std::vector<double> hd((size_t)2 * nd * nd), acc((size_t)2 * nd * nd);
  auto add_dots = [&]() -> int {
    TT_CUDA_TRY(cudaMemcpyAsync(hd.data(), dots, sizeof(double) * hd.size(), cudaMemcpyDeviceToHost, st));
    TT_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < acc.size(); i++) acc[i] += hd[i];
    return TT_OK;
  };
  for (int k = 0; k < adj.n_theta; k++) {
    std::fill(acc.begin(), acc.end(), 0.0);
    // lambda^T OP(C)^T (2P) OP(d(VC)) w = g^T h
    TT_TRY(block_apply_device(L_, adj.d_dVC + (size_t)k * adj.vc_count, w, nd, h, st));
    TT_TRY(bilinear_device(n, g, nd, h, nd, dots, st));
    TT_TRY(add_dots());
    if (adj.total) {
      // (OP(dC) lambda)^T u2
      TT_TRY(block_apply_device(L_, adj.d_dC + (size_t)k * adj.c_count, lam, nd, u, st));
      TT_TRY(bilinear_device(n, u, nd, u2.ptr, nd, dots, st));
      TT_TRY(add_dots());
      // (A^T lambda)^T (dG o x)
      const double dEj = adj.dEb[k] * (1.0 - (Eh_[j] - adj.E_bound) * adj.dlnmu1_dEb);
      TT_TRY(dresolvent_device(L_, adj.d_de + (size_t)k * adj.e_count, dEj, E_.ptr + j, 1, dG.ptr, st));
      TT_TRY(hadamard_device(dG.ptr, zero_e.ptr, n, x, nd, t2.ptr, st));
      TT_TRY(bilinear_device(n, yT, nd, t2.ptr, nd, dots, st));
      TT_TRY(add_dots());
    }
    for (int dr = 0; dr < nd; dr++)
      for (int dc = 0; dc < nd; dc++) {
        const size_t o = (size_t)k * nd * nd * nE + (size_t)dr * nd * nE + (size_t)dc * nE + j;
        (*adj.dU)[2 * o + 0] = acc[2 * (dr * nd + dc) + 0];
        (*adj.dU)[2 * o + 1] = acc[2 * (dr * nd + dc) + 1];
      }
  }
  r.ms_adjoint += ms_since(t0);
  return TT_OK;
}

int ChannelSolver::solve(const std::vector<int>& q_idx, const std::vector<int>& deut, const SolveOptions& opt,
                         std::vector<double>& U, SolveReport* rep, cudaStream_t st, const AdjointRequest* adj,
                         const BreakupRequest* bu) {
  const int nE = (int)q_idx.size(), nd = (int)deut.size();
  if (bu) {
    if (!opt.pade) {
      set_error("breakup amplitudes come from the Pade path, as in the reference");
      return TT_ERR_UNSUPPORTED;
    }
    const BreakupCells* c = bu->cells;
    if (!c || !bu->U_BU || c->start.size() != (size_t)nE + 1 || c->cells.size() % 3 || c->start[0] != 0 ||
        c->start[nE] != c->count()) {
      set_error("breakup cells do not match the solve's energies");
      return TT_ERR_BADARG;
    }
    for (int j = 0; j < nE; j++)
      if (c->start[j + 1] < c->start[j]) {
        set_error("breakup cell offsets decrease");
        return TT_ERR_BADARG;
      }
    bu->U_BU->assign((size_t)2 * nd * c->count(), std::nan(""));
  }
  if (nE != nE_) {
    set_error("number of on-shell bins does not match the resolvent energies");
    return TT_ERR_BADARG;
  }
  if (!A_.ptr) {
    set_error("A has not been built");
    return TT_ERR_BADARG;
  }
  U.assign((size_t)2 * nd * nd * nE, 0.0);
  drop_kept();
  if (adj) {
    if (!adj->dU || (adj->n_theta > 0 && !adj->d_dVC)) {
      set_error("adjoint request without output or derivative blocks");
      return TT_ERR_BADARG;
    }
    if (nd > 4) {
      set_error("the adjoint handles at most 4 deuteron states per channel");
      return TT_ERR_UNSUPPORTED;
    }
    adj->dU->assign((size_t)adj->n_theta * 2 * nd * nd * nE, 0.0);
  }
  SolveReport r;
  if (nd == 0 || nE == 0) {
    if (rep) *rep = r;
    return TT_OK;
  }
  if (opt.pade) {
    if (adj) {
      set_error("the adjoint needs the LU path; the Pade series has no stored factors");
      return TT_ERR_UNSUPPORTED;
    }
    const int s = solve_pade(q_idx, deut, U, r, st, bu);
    if (rep) *rep = r;
    return s;
  }
  const int Nq = L_.Nq, Np = L_.Np;
  // complex64: up to opt.energy_batch (<= 4) energies' matrices formed and
  // factored together (their sub-panels share each grid barrier), as many as
  // free HBM holds
  int B = 1;
  if (opt.mixed && nE > 1 && opt.energy_batch > 1) {
    size_t free_b = 0, total_b = 0;
    TT_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    free_b += device_cache_bytes();  // cached blocks are freed when an allocation needs them
    const size_t per = (size_t)n * n * sizeof(float2), reserve = (size_t)2 << 30;
    const size_t fit = free_b > reserve + per ? (free_b - reserve) / per : 1;
    B = (int)std::max<size_t>(1, std::min<size_t>(std::min<size_t>((size_t)nE, std::min(opt.energy_batch, 4)), fit));
  }
  DevBuf<int32_t> ipiv_all, cols, rhs_e;
  TT_TRY(ipiv_all.alloc((size_t)n * B));
  DevBuf<double2> L64;
  DevBuf<float2> L32all;
  if (opt.mixed) {
    // the batch was sized from free HBM before the per-solve buffers: fewer
    // matrices when their allocation still does not fit
    for (;;) {
      const int s = L32all.alloc((size_t)B * n * n);
      if (s == TT_OK) break;
      if (s != TT_ERR_NOMEM || B == 1) return s;
      B--;
    }
  } else {
    TT_TRY(L64.alloc((size_t)n * n));
  }
  // right-hand sides, solutions and refinement vectors of a group's energies:
  // [q][d][n] complex128, energy q of the group, deuteron column d
  const size_t vec = (size_t)2 * n * nd;
  DevBuf<double> b, x, y, res, tmp;
  TT_TRY(tmp.alloc(vec));
  TT_TRY(b.alloc(vec * B));
  TT_TRY(x.alloc(vec * B));
  if (opt.mixed) {
    TT_TRY(y.alloc(vec * B));
    TT_TRY(res.alloc(vec * B));
  }
  std::vector<DevBuf<int32_t>> perm_d(B);
  std::vector<TrsvBlocks<float2>> tb32(B);
  TrsvBlocks<double2> tb64, tbT64;
  TrsvBlocks<float2> tbT32;
  // adjoint: the vectors of lambda, its refinement and the products
  DevBuf<double> lam, yT, rT, u, g, w, h, dots;
  if (adj && adj->n_theta > 0) {
    for (DevBuf<double>* v : {&lam, &yT, &rT, &u, &g, &w, &h}) TT_TRY(v->alloc(vec));
    TT_TRY(dots.alloc((size_t)2 * nd * nd));
  }
  // a TF32 factor whose refinement does not converge is made again with BF16x3
  const int product0 = opt.tensor_cores ? opt.tc_product : 0;
  int product = product0;
  for (int g0 = 0; g0 < nE;) {
    const int nb = std::min(B, nE - g0);
    // ---- form and factor the group's matrices
    auto t0 = std::chrono::steady_clock::now();
    int info[4] = {0, 0, 0, 0};
    if (opt.mixed) {
      float2* Ls[4];
      int32_t* ps[4];
      for (int q = 0; q < nb; q++) {
        Ls[q] = L32all.ptr + (size_t)q * n * n;
        ps[q] = ipiv_all.ptr + (size_t)q * n;
        TT_TRY(form_L_device<float2>(A_.ptr, G_.ptr + (size_t)2 * n * (g0 + q), n, Ls[q], st));
      }
      TT_CUDA_TRY(cudaStreamSynchronize(st));
      r.ms_form += ms_since(t0);
      t0 = std::chrono::steady_clock::now();
      TT_TRY(lu_factor_batched_device<float2>(Ls, nb, n, ps, st, product, info, opt.panel_blocked,
                                              opt.panel_width ? opt.panel_width : tuned_panel_width(n, product),
                                              opt.inverse_block, opt.cta_pairs, opt.mid_panel));
      r.ms_factor += ms_since(t0);
    } else {
      TT_TRY(form_L_device<double2>(A_.ptr, G_.ptr + (size_t)2 * n * g0, n, L64.ptr, st));
      TT_CUDA_TRY(cudaStreamSynchronize(st));
      r.ms_form += ms_since(t0);
      t0 = std::chrono::steady_clock::now();
      double2* L64p = L64.ptr;
      int32_t* piv0 = ipiv_all.ptr;
      TT_TRY(lu_factor_batched_device<double2>(&L64p, 1, n, &piv0, st, 0, &info[0], opt.panel_blocked));
      r.ms_factor += ms_since(t0);
    }
    for (int q = 0; q < nb; q++)
      if (info[q] != 0) {
        r.info = info[q];
        set_error("zero pivot at column " + std::to_string(info[q]) + " of the Faddeev kernel matrix");
        if (rep) *rep = r;
        return TT_ERR_SINGULAR;
      }
    // on-shell rows (= the columns of A taken as right-hand sides) of every
    // (energy, deuteron) of the group, and each vector's energy in the group
    std::vector<int32_t> hc((size_t)nb * nd), he((size_t)nb * nd);
    for (int q = 0; q < nb; q++)
      for (int k = 0; k < nd; k++) {
        hc[(size_t)q * nd + k] = deut[k] * Nq * Np + q_idx[g0 + q] * Np + 0;
        he[(size_t)q * nd + k] = q;
      }
    TT_TRY(cols.upload(hc, st));
    TT_TRY(rhs_e.upload(he, st));
    const double* Gg = G_.ptr + (size_t)2 * n * g0;  // the group's resolvents [q][n]
    auto factor_of = [&](int q) -> float2* { return L32all.ptr + (size_t)q * n * n; };
    // ---- per energy: right-hand sides and the first solve with its factor
    t0 = std::chrono::steady_clock::now();
    TT_TRY(gather_rhs_device(A_.ptr, n, cols.ptr, nb * nd, b.ptr, st));
    TT_CUDA_TRY(cudaMemcpyAsync(x.ptr, b.ptr, sizeof(double) * vec * nb, cudaMemcpyDeviceToDevice, st));
    // the group's complex64 factors solved together (one sweep launch for all)
    auto solve_group = [&](const std::vector<int>& qs, double* v) -> int {
      const float2* F[4];
      const TrsvBlocks<float2>* TB[4];
      const int32_t* PD[4];
      double* X[4];
      for (size_t i = 0; i < qs.size(); i++) {
        F[i] = factor_of(qs[i]);
        TB[i] = &tb32[qs[i]];
        PD[i] = perm_d[qs[i]].ptr;
        X[i] = v + vec * qs[i];
      }
      return lu_solve_batched_device<float2>((int)qs.size(), F, n, TB, PD, X, tmp.ptr, nd, st);
    };
    std::vector<int> all_q;
    for (int q = 0; q < nb; q++) {
      std::vector<int32_t> perm;
      TT_TRY(lu_permutation(ipiv_all.ptr + (size_t)q * n, n, perm, st));
      TT_TRY(perm_d[q].upload(perm, st));
      if (opt.mixed) {
        TT_TRY(lu_trsv_prepare<float2>(factor_of(q), n, tb32[q], st));
        all_q.push_back(q);
      } else {
        TT_TRY(lu_trsv_prepare<double2>(L64.ptr, n, tb64, st));
        TT_TRY(lu_solve_device<double2>(L64.ptr, n, tb64, perm_d[q].ptr, x.ptr + vec * q, tmp.ptr, nd, st));
      }
    }
    if (opt.mixed) TT_TRY(solve_group(all_q, x.ptr));
    TT_CUDA_TRY(cudaStreamSynchronize(st));
    r.ms_solve += ms_since(t0);
    if (opt.mixed) {
      // FP64 iterative refinement of the group's energies together: one
      // residual pass over A for all their columns, r = b - (x - A (G o x)),
      // then each energy's correction L d = r with its own factor, x += d.
      // An energy stops when the estimated remaining relative error of every
      // on-shell entry (the U elements: rows cols[] of each column) is below
      // the tolerance, with the whole column's max|dx|/max|x| as a floor (the
      // adjoint reads all of x).
      t0 = std::chrono::steady_clock::now();
      std::vector<char> done(nb, 0);
      std::vector<int> iters(nb, 0);
      std::vector<double> worst(nb, 0.0);
      std::vector<std::vector<double>> prev(nb, std::vector<double>((size_t)nd + (size_t)nd * nd, 0.0));
      std::vector<double> ratio((size_t)nd + (size_t)nd * nd);
      int left = nb;
      // TF32 factors refine in about 4 steps here; one that needs more than 12
      // is made again with BF16x3 rather than iterated to the limit
      const int max_it = product == TC_TF32 ? std::min(opt.refine_max_iter, 12) : opt.refine_max_iter;
      for (int it = 1; it <= max_it && left > 0; it++) {
        TT_TRY(hadamard_device(Gg, rhs_e.ptr, n, x.ptr, nb * nd, y.ptr, st));
        TT_TRY(residual_multi_device(A_.ptr, n, y.ptr, b.ptr, x.ptr, nb * nd, res.ptr, st));
        std::vector<int> active;
        for (int q = 0; q < nb; q++)
          if (!done[q]) active.push_back(q);
        TT_TRY(solve_group(active, res.ptr));
        for (int q = 0; q < nb; q++) {
          if (done[q]) continue;
          TT_TRY(axpy_norms_device(x.ptr + vec * q, res.ptr + vec * q, n, nd, ratio.data(), st,
                                   cols.ptr + (size_t)q * nd, nd, ratio.data() + nd));
          worst[q] = refine_error_estimate(ratio, prev[q], it > 1);
          iters[q] = it;
          if (!(worst[q] == worst[q])) {  // NaN: no convergence
            left = 0;
            break;
          }
          if (worst[q] <= opt.refine_tol) {
            done[q] = 1;
            left--;
          }
        }
      }
      r.ms_refine += ms_since(t0);
      for (int q = 0; q < nb; q++) {
        r.refine_iters = std::max(r.refine_iters, iters[q]);
        r.final_correction = std::max(r.final_correction, worst[q]);
        if (!(worst[q] == worst[q])) r.final_correction = worst[q];
      }
      if (std::find(done.begin(), done.end(), 0) != done.end()) {
        if (product == TC_TF32) {
          // the same group again with the BF16x3 product
          product = TC_BF16X3;
          r.product_fallbacks++;
          continue;
        }
        int q = 0;
        while (done[q]) q++;
        set_error("iterative refinement did not converge (last |dx|/|x| = " + std::to_string(worst[q]) + ")");
        if (rep) *rep = r;
        return TT_ERR_NOCONVERGE;
      }
    }
    // ---- per energy: adjoint, on-shell read-out (solve_faddeev.cpp:407-431)
    for (int q = 0; q < nb; q++) {
      const int j = g0 + q;
      const double* Gj = G_.ptr + (size_t)2 * n * j;
      double* xq = x.ptr + vec * q;
      if (adj && adj->n_theta > 0)
        TT_TRY(adjoint_energy(j, nE, nd, Gj, cols.ptr + (size_t)q * nd, perm_d[q].ptr, tmp.ptr, xq, opt,
                              opt.mixed ? (void*)factor_of(q) : (void*)L64.ptr, tbT32, tbT64, lam.ptr, yT.ptr, rT.ptr,
                              u.ptr, g.ptr, w.ptr, h.ptr, dots.ptr, *adj, r, st));
      std::vector<double> hx(vec);
      TT_CUDA_TRY(cudaMemcpyAsync(hx.data(), xq, sizeof(double) * hx.size(), cudaMemcpyDeviceToHost, st));
      TT_CUDA_TRY(cudaStreamSynchronize(st));
      for (int dr = 0; dr < nd; dr++)
        for (int dc = 0; dc < nd; dc++) {
          const size_t row = (size_t)deut[dr] * Nq * Np + (size_t)q_idx[j] * Np + 0;
          const size_t uu = (size_t)dr * nd * nE + (size_t)dc * nE + j;
          U[2 * uu + 0] = hx[2 * ((size_t)dc * n + row) + 0];
          U[2 * uu + 1] = hx[2 * ((size_t)dc * n + row) + 1];
        }
    }
    if (opt.keep_factors && !adj && nb == nE) {
      // one group held every energy: its factors stay for backward()
      kept_.valid = true;
      kept_.opt = opt;
      kept_.nE = nE;
      kept_.nd = nd;
      kept_.L32 = std::move(L32all);
      kept_.L64 = std::move(L64);
      kept_.perm.clear();
      for (int q = 0; q < nb; q++) kept_.perm.push_back(std::move(perm_d[q]));
      kept_.x = std::move(x);
      kept_.cols = std::move(cols);
      TT_CUDA_TRY(cudaStreamSynchronize(st));
    }
    g0 += nb;
    product = product0;
  }
  if (rep) *rep = r;
  return TT_OK;
}

int ChannelSolver::backward(const AdjointRequest& adj, std::vector<double>& dU, SolveReport* rep, cudaStream_t st) {
  if (!kept_.valid) {
    set_error("no factors kept from a forward solve");
    return TT_ERR_UNSUPPORTED;
  }
  const int nE = kept_.nE, nd = kept_.nd;
  if (nE != nE_) {
    set_error("the resolvents changed since the forward solve");
    return TT_ERR_BADARG;
  }
  if (nd > 4) {
    set_error("the adjoint handles at most 4 deuteron states per channel");
    return TT_ERR_UNSUPPORTED;
  }
  dU.assign((size_t)adj.n_theta * 2 * nd * nd * nE, 0.0);
  SolveReport r;
  const size_t vec = (size_t)2 * n * nd;
  DevBuf<double> tmp, lam, yT, rT, u, g, w, h, dots;
  for (DevBuf<double>* v : {&tmp, &lam, &yT, &rT, &u, &g, &w, &h}) TT_TRY(v->alloc(vec));
  TT_TRY(dots.alloc((size_t)2 * nd * nd));
  TrsvBlocks<float2> tbT32;
  TrsvBlocks<double2> tbT64;
  AdjointRequest a = adj;
  a.dU = &dU;
  for (int j = 0; j < nE; j++) {
    void* F = kept_.opt.mixed ? (void*)(kept_.L32.ptr + (size_t)j * n * n) : (void*)kept_.L64.ptr;
    TT_TRY(adjoint_energy(j, nE, nd, G_.ptr + (size_t)2 * n * j, kept_.cols.ptr + (size_t)j * nd, kept_.perm[j].ptr,
                          tmp.ptr, kept_.x.ptr + vec * j, kept_.opt, F, tbT32, tbT64, lam.ptr, yT.ptr, rT.ptr, u.ptr,
                          g.ptr, w.ptr, h.ptr, dots.ptr, a, r, st));
  }
  // the factors were transposed in place by the adjoint solves
  drop_kept();
  if (rep) *rep = r;
  return TT_OK;
}

}  // namespace tt
