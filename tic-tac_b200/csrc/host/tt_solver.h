// Per-channel device solver of the elastic AGS/Faddeev equations in the WPCD
// basis: U = (1 - A G)^{-1} A on the on-shell deuteron columns, A = C^T (2 P123) (V C).
#pragma once
#include <string>
#include <vector>

#include "../cuda/tt_kernels.h"
#include "tt_host.h"

namespace tt {

// 2N block structure of one channel (solve_faddeev.cpp:1588-1927, make_resolvent.cpp:109-156).
bool build_channel_layout(const RunParams& rp, const PWChannel& ch, const SWPStates& swp,
                          const std::vector<double>& V_unco, const std::vector<double>& V_coup, ChannelLayout& L,
                          std::string* err);

// Per-alpha offsets into the SWP energy table e_unco ++ e_coup (the e_off of
// build_channel_layout), written to e_off[Nalpha]; checks each 2N index
// against the n_unco / n_coup slots.  Allocates nothing.
bool channel_energy_offsets(const RunParams& rp, const PWChannel& ch, int Np, int n_unco, int n_coup,
                            int32_t* e_off, std::string* err);

// Resolvent for nE energies into caller-owned device memory d_G [nE][n] with
// the tables staged in a static device array (no device allocation); defined
// in the CUDA sources.  TT_ERR_UNSUPPORTED when the tables exceed it.
int resolvent_noalloc(const RunParams& rp, const PWChannel& ch, int Np, int Nq, int n_unco, int n_coup,
                      const double* e_unco, const double* e_coup, const double* q_WP, const double* E, int nE,
                      double* d_G, cudaStream_t st);

struct SolveOptions {
  bool mixed = true;        // complex64 LU on tensor cores + FP64 refinement; false: complex128 LU
  bool tensor_cores = true; // trailing update on tcgen05 (mixed only)
  bool panel_blocked = true;  // LU panels in 32-column steps instead of recursive halving
  int panel_width = 0;        // complex64 LU panel width (0: the tuning table's choice for n, else 512)
  int inverse_block = 0;      // unit-lower blocks solved by explicit inverse up to this size (0: 512)
  bool cta_pairs = true;      // tensor-core updates on CTA pairs (cta_group::2, 256-row tiles)
  int mid_panel = 128;        // blocked panels in mid-panels of this many columns (0: one level)
  int tc_product = 2;        // product mode of the tensor-core updates: 1 BF16x3 with N = 128 tiles,
                             // 2 TF32 (a group whose refinement does not converge is factored
                             // again with 3), 3 BF16x3 (real-row form, N = 256)
  bool pade = false;        // Pade-resummed Neumann series on the resident A instead of an LU
  double refine_tol = 1e-12;
  int refine_max_iter = 30;
  int energy_batch = 4;     // complex64: energies factored together at most (1..4; fewer if HBM is short)
  bool keep_factors = false;  // keep every energy's factor and solution for backward() (when they fit)
};

struct SolveReport {
  double ms_A = 0, ms_form = 0, ms_factor = 0, ms_solve = 0, ms_refine = 0;
  int refine_iters = 0;          // max over energies
  double final_correction = 0;   // max over rhs of |dx|/|x| at exit
  int info = 0;                  // first zero pivot (1-based) if any
  double ms_adjoint = 0;         // transposed solves, their refinement and the parameter products
  int adjoint_refine_iters = 0;  // max over energies
  int product_fallbacks = 0;     // energy groups factored again with BF16x3 after TF32 did not refine
};

// Parameter derivatives wanted from a solve: dV/dtheta_k C for k < n_theta,
// each in the layout of ChannelLayout::VC (one block per 2N channel), on the
// device.  dU receives [n_theta][nd][nd][nE] interleaved complex.
struct AdjointRequest {
  int n_theta = 0;
  const double* d_dVC = nullptr;  // n_theta * vc_count doubles: d(V C) blocks (dV C, plus V dC when total)
  size_t vc_count = 0;
  std::vector<double>* dU = nullptr;
  // total derivative: the SWP basis and the resolvent move with the potential
  bool total = false;
  const double* d_dC = nullptr;   // n_theta * c_count doubles: dC blocks (layout of C)
  size_t c_count = 0;
  const double* d_de = nullptr;   // n_theta * e_count doubles: d e_SWP (layout of the channel's e_swp)
  size_t e_count = 0;
  std::vector<double> dEb;        // n_theta: d E_bound
  // the on-shell energies E_j = E_com,j + E_bound move with E_bound also
  // through E_com,j = (q_j^2 + q_{j+1}^2) / (4 mu1(E_bound)) (the bin mid-point
  // energy of CPP/run_organizer.cpp:92-110): dE_j = dEb (1 - E_com,j dln mu1/dEb)
  double E_bound = 0;
  double dlnmu1_dEb = 0;
};

// Breakup amplitudes wanted from a Pade solve (the reference computes them on
// that path only, CPP/solve_faddeev.cpp:867-890, 1176-1205, 1299-1407): the
// on-shell rows of A (G A)^n read at each cell's column alpha Nq Np + q Np + p
// and resummed with the elastic criteria.  U_BU receives [nd][cells]
// interleaved complex; a cell outside the grid gets NaN.
struct BreakupRequest {
  const BreakupCells* cells = nullptr;  // the cells of the solve's energies
  std::vector<double>* U_BU = nullptr;
};

class ChannelSolver {
 public:
  int n = 0;
  int setup(const ChannelLayout& L, const std::vector<double>& q_WP, cudaStream_t st);
  // P123 built on the device, or uploaded from host CSR arrays
  int set_P_device(DeviceCSR&& P);
  int set_P_host_csr(const int64_t* rowptr, const int32_t* col, const double* val, int64_t nnz, cudaStream_t st);
  // the reference's CSC form, converted on the device
  int set_P_host_csc(const double* val, const int32_t* row, const uint64_t* colptr, int64_t nnz, cudaStream_t st);
  int build_A(cudaStream_t st, double* ms = nullptr);
  // resolvent for energies E (= E_com + E_bound) into device G [nE][n]
  int resolvent(const std::vector<double>& E, cudaStream_t st);
  // U[d'*nd*nE + d*nE + j] for each on-shell q bin j and deuteron states
  int solve(const std::vector<int>& q_idx, const std::vector<int>& deut, const SolveOptions& opt,
            std::vector<double>& U_interleaved, SolveReport* rep, cudaStream_t st,
            const AdjointRequest* adj = nullptr, const BreakupRequest* bu = nullptr);
  // Adjoint of the last solve(keep_factors) from the factors it kept:
  // dU/dtheta of adj for its energies.  TT_ERR_UNSUPPORTED when nothing was
  // kept (the energies' factors did not fit at once): the caller then runs
  // solve() with the request, which factors again.
  int backward(const AdjointRequest& adj, std::vector<double>& dU, SolveReport* rep, cudaStream_t st);
  bool kept() const { return kept_.valid; }
  void drop_kept() { kept_ = Kept(); }
  void release_A() {
    A_.release();
    G_.release();
    nE_ = 0;
    drop_kept();
  }
  const DeviceCSR& P() const { return P_; }
  const double* A() const { return A_.ptr; }
  const DeviceLayout& layout() const { return L_; }
  const double* G() const { return G_.ptr; }
  int nE() const { return nE_; }

 private:
  int solve_pade(const std::vector<int>& q_idx, const std::vector<int>& deut, std::vector<double>& U,
                 SolveReport& r, cudaStream_t st, const BreakupRequest* bu);
  int adjoint_energy(int j, int nE, int nd, const double* Gj, const int32_t* d_rows, const int32_t* d_perm,
                     double* tmp, const double* x, const SolveOptions& opt, void* F,
                     TrsvBlocks<float2>& tbT32, TrsvBlocks<double2>& tbT64, double* lam, double* yT, double* rT,
                     double* u, double* g, double* w, double* h, double* dots, const AdjointRequest& adj,
                     SolveReport& r, cudaStream_t st);
  // state a solve(keep_factors) leaves for backward(): each energy's factor,
  // row permutation and refined solution
  struct Kept {
    bool valid = false;
    SolveOptions opt;
    int nE = 0, nd = 0;
    DevBuf<float2> L32;
    DevBuf<double2> L64;
    std::vector<DevBuf<int32_t>> perm;
    DevBuf<double> x;
    DevBuf<int32_t> cols;
  };
  Kept kept_;
  DeviceLayout L_;
  DeviceCSR P_;
  DevBuf<double> A_, G_, E_;
  DevBuf<int32_t> aoff_;  // per P123 row, the start of each alpha's column range
  std::vector<double> Eh_;  // host copy of E_  // E_: the energies of the resolvents in G_
  int nE_ = 0;
};

}  // namespace tt
