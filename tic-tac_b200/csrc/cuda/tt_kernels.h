// Device stages of the WPCD path (host-callable launchers).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "tt_device.h"

namespace tt {

struct P123Tables;

struct P123Stats {
  int64_t n_cells = 0;
  int64_t n_pairs = 0;
};

// P123 of one channel in CSR on the device (p123.cu).
int p123_build_device(const P123Tables& t, DeviceCSR& out, cudaStream_t st, P123Stats* stats);

// Per-channel description of the 2N structure used by the resolvent and the
// A = C^T (2 P123) (V C) build (host-prepared, see tt_solve_prep.cpp).
struct ChannelLayout {
  int Nalpha = 0, Np = 0, Nq = 0;
  // per alpha: index of its 2N block, its part (0 = L=J-1 / T3=1/2, 1 = L=J+1 / T3=3/2), block dim (Np or 2Np)
  std::vector<int32_t> blk, part, dim;
  // per alpha: partners alpha' coupled through the 2N interaction (CSR)
  std::vector<int32_t> cpl_off, cpl;
  // per 2N block: offset (in doubles) into the C and VC arrays; dim
  std::vector<int64_t> blk_off;
  std::vector<int32_t> blk_dim;
  std::vector<double> C, VC;  // row-major blocks, VC = V.C
  // per alpha: offset into e_swp (Np+1 boundaries of its SWP energies)
  std::vector<int32_t> e_off;
  std::vector<double> e_swp;
};

struct DeviceLayout {
  int Nalpha = 0, Np = 0, Nq = 0, n = 0;
  DevBuf<int32_t> blk, part, dim, cpl_off, cpl, blk_dim, e_off;
  DevBuf<int64_t> blk_off;
  DevBuf<double> C, VC, e_swp;
  DevBuf<double> q_WP;
  int upload(const ChannelLayout& L, const std::vector<double>& q_WP, cudaStream_t st);
};

// G[j*n + i] (complex128 interleaved) for energies E[j]; make_resolvent.cpp:82-211.
int resolvent_device(const DeviceLayout& L, const double* d_E, int nE, double* d_G, cudaStream_t st);

// Same kernel on tables the caller placed in device memory: e_off[Na],
// e_swp (SWP energy boundaries), q_WP[Nq+1], E[nE].
int resolvent_device_tables(int Na, int Nq, int Np, const int32_t* e_off, const double* e_swp, const double* q_WP,
                            const double* d_E, int nE, double* d_G, cudaStream_t st);

// Dense A (n x n, row-major FP64) = C^T (2 P123) (V C); solve_faddeev.cpp:4-181.
// d_aoff: the table of alpha_offsets_device for P.
int build_A_device(const DeviceLayout& L, const DeviceCSR& P, const int32_t* d_aoff, double* d_A, cudaStream_t st);
// d_aoff[r (Nalpha + 1) + a]: first nonzero of CSR row r with column >= a Nq Np,
// relative to rowptr[r] (n (Nalpha + 1) int32).
int alpha_offsets_device(const DeviceLayout& L, const DeviceCSR& P, int32_t* d_aoff, cudaStream_t st);

// L = 1 - A diag(G), complex, row-major; T = double2 (complex128) or float2 (complex64).
template <typename T>
int form_L_device(const double* d_A, const double* d_G, int n, T* d_L, cudaStream_t st);

// RHS columns b_k = A[:, cols[k]] as complex128, stored column-by-column [k][n].
int gather_rhs_device(const double* d_A, int n, const int32_t* d_cols, int nrhs, double* d_b, cudaStream_t st);

// y_k = G_{e(k)} o x_k (complex128) for nrhs right-hand sides, G stored [nE][n].
int hadamard_device(const double* d_G, const int32_t* d_rhs_e, int n, const double* d_x, int nrhs, double* d_y,
                    cudaStream_t st);
// r_k = b_k - x_k + A y_k: the FP64 residual of (1 - A G) x = b, one read of A for all rhs.
int residual_multi_device(const double* d_A, int n, const double* d_y, const double* d_b, const double* d_x, int nrhs,
                          double* d_r, cudaStream_t st);

// LU with partial pivoting, in place, row-major (lu.cu).  ipiv[k] = row swapped with k.
template <typename T>
int lu_factor_device(T* d_L, int n, int32_t* d_ipiv, cudaStream_t st, int use_tensor_cores, int* info);
// B <= 4 matrices of equal n factored together (each sub-panel of all of them
// in one cooperative launch, one grid barrier per column for the batch);
// info[B] receives each matrix's first zero pivot (1-based) or 0.
// blocked: the panel in 32-column steps, each followed by its rank-32 update
// (otherwise recursive halving of the panel and of the U12 solve).
// panel: the outer panel width (a multiple of 32 up to 512; 0 = 512 for
// complex64, 128 for complex128).  inv_block: in the tensor-core modes a block
// row is solved through the explicit inverses of unit-lower diagonal blocks of
// at most this many rows (a multiple of 32 up to 512; 0 = 512), larger blocks
// by halving with tensor-core updates between the halves.  cta_pairs: the
// tensor-core updates run on CTA pairs (256-row tiles, cta_group::2).  mid: the
// blocked panel in mid-panels of this many columns (a multiple of 32; 0 = one
// level): sub-panel updates stay inside the mid-panel and the rest of the
// panel is updated once per mid-panel, with depth mid.
template <typename T>
int lu_factor_batched_device(T* const* d_L, int B, int n, int32_t* const* d_ipiv, cudaStream_t st,
                             int use_tensor_cores, int* info, bool blocked = false, int panel = 0,
                             int inv_block = 0, bool cta_pairs = false, int mid = 0);
// Row permutation of the interchange sequence ipiv (host, once per factorisation).
int lu_permutation(const int32_t* d_ipiv, int n, std::vector<int32_t>& perm, cudaStream_t st);
// Inverted diagonal blocks of one LU factor (unit lower and upper) and their
// products with the neighbouring off-diagonal blocks, made by lu_trsv_prepare
// after each factorisation and read by every solve with it.
template <typename T>
struct TrsvBlocks {
  DevBuf<T> invL, invU;  // inverted 64 x 64 diagonal blocks
  DevBuf<T> mL, mU;      // inv[b] times the block that carries the previous solved block into b
  int n = 0;
};
// transposed = true: d_LU holds the transpose of a factor (non-unit lower,
// unit upper), for lu_solve_transposed_device.
template <typename T>
int lu_trsv_prepare(const T* d_LU, int n, TrsvBlocks<T>& blk, cudaStream_t st, bool transposed = false);
// Solve L U x = P b for nrhs complex128 columns [k][n] in place using the factor
// of type T; d_perm from lu_permutation (uploaded), d_tmp scratch of 2 n nrhs doubles.
template <typename T>
int lu_solve_device(const T* d_LU, int n, const TrsvBlocks<T>& blk, const int32_t* d_perm, double* d_x,
                    double* d_tmp, int nrhs, cudaStream_t st);
// The same for B <= 4 factors of order n at once (their substitution sweeps
// share each cooperative launch and grid barrier): x_b with factor b.
template <typename T>
int lu_solve_batched_device(int B, const T* const* d_LU, int n, const TrsvBlocks<T>* const* blk,
                            const int32_t* const* d_perm, double* const* d_x, double* d_tmp, int nrhs,
                            cudaStream_t st);

// Solve (P^T L U)^T x = b, i.e. transposed systems of the same factor, for
// nrhs complex128 columns [k][n] in place: d_LUt is the transpose of the
// factor (transpose_inplace_device) with blkT from lu_trsv_prepare(..., true).
template <typename T>
int lu_solve_transposed_device(const T* d_LUt, int n, const TrsvBlocks<T>& blkT, const int32_t* d_perm, double* d_x,
                               double* d_tmp, int nrhs, cudaStream_t st);

// P123 from the reference's host CSC (values, int rows, size_t column pointers)
// to device CSR with ascending columns per row (csr_build.cu).
int csc_to_csr_device(const double* h_val, const int32_t* h_row, const uint64_t* h_colptr, int64_t nnz, int n,
                      DeviceCSR& out, cudaStream_t st);

// Adjoint pieces (adjoint.cu); vectors are complex128 [k][n].
// the factor transposed in place (it is not needed in row form afterwards)
template <typename T>
int transpose_inplace_device(T* a, int n, cudaStream_t st);
// y_k = A^T v_k, k < nrhs <= 8
int gemv_t_device(const double* d_A, int n, const double* d_v, int nrhs, double* d_y, cudaStream_t st);
// Pade path (adjoint.cu): R[k] = A[rows[k], :] as complex; V[k] = R[k] o G[e[k]];
// out[i] = R[row[i]][col[i]]
int gather_rows_device(const double* d_A, int n, const int32_t* d_rows, int nrows, double* d_R, cudaStream_t st);
int scale_rows_device(const double* d_R, const double* d_G, const int32_t* d_e, int n, int nrows, double* d_V,
                      cudaStream_t st);
int pick_device(const double* d_R, int n, const int32_t* d_row, const int32_t* d_col, int m, double* d_out,
                cudaStream_t st);
// r_k = e_{rows[k]} - lam_k + G o y_k
int residual_t_device(const double* d_lam, const double* d_y, const double* d_G, const int32_t* d_rows, int n,
                      int nrhs, double* d_r, cudaStream_t st);
int unit_rhs_device(const int32_t* d_rows, int n, int nrhs, double* d_x, cudaStream_t st);
// w_k = e_{rows[k]} + G o x_k
int make_w_device(const double* d_x, const double* d_G, const int32_t* d_rows, int n, int nrhs, double* d_w,
                  cudaStream_t st);
// out_k = OP(X) in_k with X in the layout of C / VC (one block per 2N channel)
int block_apply_device(const DeviceLayout& L, const double* d_X, const double* d_in, int nrhs, double* d_out,
                       cudaStream_t st);
// out_k = 2 P u_k
int spmv_device(const DeviceCSR& P, const double* d_u, int nrhs, double* d_out, cudaStream_t st);
// dG[j*n + i]: first-order change of the resolvents for a change de of the SWP
// energy boundaries (layout of the layout's e_swp; the bound state's lower
// boundary is E_bound, which also moves the n-d reduced mass of its
// bound-continuum bins) and dE of the energies E[j] = E_com,j + E_bound (the
// same dE for the nE energies given)
int dresolvent_device(const DeviceLayout& L, const double* d_de, double dE, const double* d_E, int nE, double* d_dG,
                      cudaStream_t st);
// g_k = 2 P^T u_k
int spmv_t_device(const DeviceCSR& P, const double* d_u, int nrhs, double* d_g, cudaStream_t st);
// out[a nb + b] = sum_i g_a[i] h_b[i], complex, na, nb <= 4
int bilinear_device(int n, const double* d_g, int na, const double* d_h, int nb, double* d_out, cudaStream_t st);

// On-shell U elements smaller than this fraction of the largest one of their
// column are zero by symmetry up to rounding: their relative change is taken
// against the fraction instead of their own magnitude.
constexpr double kOnshellZeroFloor = 1e-6;
// x += d ; returns max |d| / max |x| per rhs in h_ratio (host, synchronises).
// With d_rows (nrows entries), also each on-shell entry's relative change
// |d_k[rows[r]]| / max(|x_k[rows[r]]|, kOnshellZeroFloor max_r |x_k[rows[r]]|)
// in h_elem[k nrows + r].
int axpy_norms_device(double* d_x, const double* d_d, int n, int nrhs, double* h_dx_over_x, cudaStream_t st,
                      const int32_t* d_rows = nullptr, int nrows = 0, double* h_elem = nullptr);

// Device count of SMs, cached.
int device_sm_count();

}  // namespace tt
