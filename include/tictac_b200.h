/* tictac_b200 — B200-native WPCD solve of the elastic nucleon-deuteron
 * AGS/Faddeev equations (the P123 / resolvent / Faddeev-solve path of Tic-tac).
 *
 * C-ABI: plain structs of pointers and sizes, status codes, no exceptions and
 * no process exit.  Every entry point returns TT_OK (0) or an error code; the
 * message of the last error on the calling thread is tt_last_error_string().
 *
 * Two layers:
 *   1. drop-in entry points with the argument meaning of the reference's
 *      three hot-path functions (host buffers in and out);
 *   2. a run handle (tt_run_*) that performs the reference main loop's
 *      state-space setup from key=value options and keeps each channel's
 *      P123, A and factorisations resident in HBM for repeated solves.
 */
#ifndef TICTAC_B200_H
#define TICTAC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TT_OK 0
#define TT_ERR_BADARG 1
#define TT_ERR_NOMEM 2       /* HBM admission failed; nothing was left allocated */
#define TT_ERR_CUDA 3
#define TT_ERR_NOCONVERGE 4  /* iterative refinement hit refine_max_iter */
#define TT_ERR_IO 5
#define TT_ERR_UNSUPPORTED 6
#define TT_ERR_SINGULAR 7    /* zero pivot in the LU of 1 - A G */

/* ---- precision of the dense solve ---- */
#define TT_PRECISION_FP64 0   /* complex128 LU, FP64 throughout */
#define TT_PRECISION_MIXED 1  /* complex64 LU, BF16x3 tcgen05 trailing updates, FP64 refinement */
#define TT_PRECISION_MIXED_SIMT 2  /* complex64 LU, FP32 CUDA-core trailing updates, FP64 refinement */
#define TT_PRECISION_PADE 3   /* the reference's production default (solve_dense = false): Pade-resummed Neumann
                                 series A (G A)^n on the resident FP64 A, stopped by the reference's criteria
                                 (about 1e-6 relative); report.refine_iters = highest [N/N] order formed */

/* complex128, layout-compatible with std::complex<double> */
typedef struct tt_complex {
  double re, im;
} tt_complex;

/* One 3N channel of the partial-wave basis.  Same fields and order as
 * pw_3N_statespace (CPP/type_defs.h:15-29) restricted to one channel
 * (the reference passes pw_substates, CPP/main.cpp:181-192). */
typedef struct tt_pw_states {
  int Nalpha;
  int J_2N_max;
  const int* L_2N_array;
  const int* S_2N_array;
  const int* J_2N_array;
  const int* T_2N_array;
  const int* L_1N_array;
  const int* two_J_1N_array;
  const int* two_J_3N_array;
  const int* two_T_3N_array;
  const int* P_3N_array;
} tt_pw_states;

/* Free wave-packet grid: the fields of fwp_statespace (CPP/type_defs.h:32-47)
 * the path reads (bin boundaries). */
typedef struct tt_fwp_states {
  int Np_WP;
  int Nq_WP;
  const double* p_WP_array; /* [Np_WP+1] */
  const double* q_WP_array; /* [Nq_WP+1] */
} tt_fwp_states;

/* Scattering wave packets, swp_statespace (CPP/type_defs.h:50-61). */
typedef struct tt_swp_states {
  int Np_WP;
  int Nq_WP;
  int num_2N_unco_states;
  int num_2N_coup_states;
  double E_bound;
  const double* e_SWP_unco_array; /* [(Np+1) num_unco] */
  const double* e_SWP_coup_array; /* [2 (Np+1) num_coup] */
  const double* C_SWP_unco_array; /* [Np Np num_unco] row-major */
  const double* C_SWP_coup_array; /* [4 Np Np num_coup] row-major */
  const double* q_WP_array;       /* [Nq+1] */
} tt_swp_states;

/* Elastic on-shell indexing, channel_os_indexing (CPP/type_defs.h:77-85). */
typedef struct tt_os_indexing {
  int num_T_lab;
  const int* q_com_idx_array;     /* [num_T_lab] */
  const int* deuteron_idx_array;  /* [num_deuteron_states] */
  int num_deuteron_states;
} tt_os_indexing;

/* Breakup indexing, the include_breakup_channels fields of
 * channel_os_indexing (CPP/type_defs.h:82-84) as find_on_shell_bins fills
 * them (CPP/run_organizer.cpp:134-339): the cells of energy j are
 * q_com_BU_idx_array[j] .. q_com_BU_idx_array[j+1]-1, cell b is
 * (alpha, q bin, p bin) = alphapq_idx_array[3b .. 3b+2]. */
typedef struct tt_bu_indexing {
  int num_BU_chns;
  const int* q_com_BU_idx_array; /* [num_T_lab + 1] */
  const int* alphapq_idx_array;  /* [3 num_BU_chns] */
} tt_bu_indexing;

/* The run_params fields (CPP/type_defs.h:87-123) the three functions read,
 * plus the precision controls of this implementation. */
typedef struct tt_run_params {
  int Nphi;                 /* default 48 */
  int Nx;                   /* default 48 */
  int tensor_force;         /* default 1 */
  int isospin_breaking_1S0; /* default 1 */
  int production_run;       /* default 1 */
  int precision;            /* TT_PRECISION_* (replaces solve_dense/Pade selection) */
  double refine_tol;        /* refinement stop (default 1e-12): estimated remaining relative error of every
                               on-shell entry (each U element's own |dx|/|x|; elements below 1e-6 of the
                               largest in their column, zero by symmetry up to rounding, against that
                               fraction) and of the whole column (max |dx| / max |x|) */
  int refine_max_iter;      /* default 30 */
} tt_run_params;

void tt_run_params_default(tt_run_params* rp);

typedef struct tt_solve_report {
  double ms_A;          /* building A = C^T (2 P123) (V C) */
  double ms_form;       /* forming 1 - A G for all energies */
  double ms_factor;     /* LU factorisations */
  double ms_solve;      /* triangular solves */
  double ms_refine;     /* FP64 refinement */
  int refine_iters;     /* max over energies */
  double final_correction; /* estimated remaining relative error at exit, the worst of the on-shell entries'
                              and the columns' measures of refine_tol: the last relative change, or, once two
                              corrections contract by rho < 1/2, that times rho / (1 - rho); max over energies */
  int info;             /* first zero pivot (1-based), 0 if none */
  double ms_adjoint;    /* adjoint: transposed solves, their refinement, parameter products */
  int adjoint_refine_iters;
  int product_fallbacks; /* energy groups factored again with BF16x3 because their TF32 factors did not refine */
} tt_solve_report;

/* ---- layer 1: drop-in entry points ---------------------------------- */

/* Replaces fill_P123_arrays (CPP/make_permutation_matrix.h:79-87,
 * make_permutation_matrix.cpp:1297-1403) for one channel: builds P123 on the
 * GPU and returns it in the reference's row-major COO order (sorted by
 * row*n+col).  Callee allocates *val, *row, *col (free with tt_free).
 * No TFC/HDF5 side files are written. */
int tt_fill_P123_arrays(double** val, int** row, int** col, size_t* nnz, int production_run,
                        const tt_fwp_states* fwp, const tt_pw_states* pw, const tt_run_params* rp);

/* Replaces calculate_resolvent_array_in_SWP_basis (CPP/make_resolvent.h:36-40):
 * caller-allocated G[n], n = Nalpha Nq Np, index alpha*Nq*Np + q*Np + p. */
int tt_calculate_resolvent_array_in_SWP_basis(tt_complex* G, double E, const tt_swp_states* swp,
                                              const tt_pw_states* pw, const tt_run_params* rp);

/* No counterpart in the reference.  The resolvent of
 * tt_calculate_resolvent_array_in_SWP_basis for nE energies E[j] (host array),
 * written to G_dev[j*n + i] in DEVICE memory the caller owns, on `stream`
 * (a cudaStream_t; NULL = the legacy default stream), without any device
 * allocation: for callers whose device memory is all held by their own pool
 * (a caching allocator, a pre-reserved arena) and that cannot let a library
 * cudaMalloc.  The lookup tables are staged in a fixed static device scratch
 * of TT_RESOLVENT_NOALLOC_SCRATCH_BYTES:
 *   4 Nalpha + 8 [(Np+1)(num_unco + 2 num_coup)] + 8 (Nq+1) + 8 nE bytes,
 *   each part rounded up to 256,
 * and larger inputs are rejected with TT_ERR_UNSUPPORTED before any device work.
 * The first call on each device looks up the scratch address with
 * cudaGetSymbolAddress (that device current) and loads the module there.
 * Nothing has to be zeroed beforehand;
 * every call rewrites the tables it reads.  Calls that overlap in time on one
 * device (other streams or host threads) share the scratch and race:
 * serialise them.  Returns when the work is queued on `stream`; a call first
 * waits until the previous call's copy of its tables to the device has read
 * the library's host staging buffer. */
#define TT_RESOLVENT_NOALLOC_SCRATCH_BYTES (256u * 1024u)
int tt_calculate_resolvent_array_in_SWP_basis_noalloc(tt_complex* G_dev, const double* E, int nE,
                                                      const tt_swp_states* swp, const tt_pw_states* pw,
                                                      const tt_run_params* rp, void* stream);

/* Replaces solve_faddeev_equations (CPP/solve_faddeev.h:25-38) for the
 * elastic on-shell U-matrix: U[d'*nd*nE + d*nE + j] (caller allocates
 * nE*nd*nd), G[j*n + i] the resolvents of the nE on-shell energies, P123 in
 * the reference's CSC form (values, int row indices, size_t column pointers
 * [n+1]), V in the WP basis.  rp->precision selects FP64 or mixed+refined. */
int tt_solve_faddeev_equations(tt_complex* U, const tt_complex* G, const double* P123_val, const int* P123_row,
                               const size_t* P123_colptr_csc, size_t P123_nnz, const double* V_WP_unco,
                               const double* V_WP_coup, const tt_swp_states* swp, const tt_os_indexing* os,
                               const tt_pw_states* pw, const tt_run_params* rp, tt_solve_report* report);

/* solve_faddeev_equations with its breakup output U_BU (CPP/solve_faddeev.h:25-38
 * with include_breakup_channels=true): U as tt_solve_faddeev_equations, and
 * U_BU[d*num_BU_chns + b] (caller allocates nd*num_BU_chns) for deuteron state
 * d and breakup cell b of bu, read off the on-shell rows of A (G A)^n at the
 * cell's column and Pade-resummed with the elastic criteria
 * (CPP/solve_faddeev.cpp:867-890, 1176-1205, 1299-1407).  The reference
 * computes breakup amplitudes on its Pade path only: rp->precision must be
 * TT_PRECISION_PADE, else TT_ERR_UNSUPPORTED.  A cell outside the grid (the
 * neighbour of an edge cell, bin -1 or N) gets NaN; the reference reads a
 * neighbouring element of its row storage there. */
int tt_solve_faddeev_equations_breakup(tt_complex* U, tt_complex* U_BU, const tt_bu_indexing* bu, const tt_complex* G,
                                       const double* P123_val, const int* P123_row, const size_t* P123_colptr_csc,
                                       size_t P123_nnz, const double* V_WP_unco, const double* V_WP_coup,
                                       const tt_swp_states* swp, const tt_os_indexing* os, const tt_pw_states* pw,
                                       const tt_run_params* rp, tt_solve_report* report);

/* Adjoint of tt_solve_faddeev_equations (no counterpart in the reference):
 * besides U, the derivatives dU/dtheta_k for n_theta perturbations of the
 * potential, given as dV/dtheta_k in the layout of V_WP_unco / V_WP_coup
 * ([n_theta][Np Np num_unco] and [n_theta][4 Np Np num_coup]).  Per energy
 * one transposed solve with the same LU factors gives lambda = (1 - A G)^-T e
 * for the on-shell rows, and dU[d'][d] = lambda_d'^T dA (e_d + G x_d) with
 * dA = C^T (2 P123)(dV C); the mixed-precision path refines lambda in FP64.
 * dU_dtheta[k*nE*nd*nd + d'*nd*nE + d*nE + j] (caller allocates).
 * At most 4 deuteron states per channel. */
int tt_solve_faddeev_adjoint(tt_complex* U, tt_complex* dU_dtheta, int n_theta, const double* dV_WP_unco_dtheta,
                             const double* dV_WP_coup_dtheta, const tt_complex* G, const double* P123_val,
                             const int* P123_row, const size_t* P123_colptr_csc, size_t P123_nnz,
                             const double* V_WP_unco, const double* V_WP_coup, const tt_swp_states* swp,
                             const tt_os_indexing* os, const tt_pw_states* pw, const tt_run_params* rp,
                             tt_solve_report* report);

/* P123 files in the reference's HDF5 layout, written and read by this
 * library without libhdf5 (file format subset: superblock version 0,
 * version-1 object headers, symbol-table root group, contiguous datasets;
 * the reader also takes chunked tables as H5TBmake_table writes them).
 *
 * Replaces store_sparse_permutation_matrix_for_3N_channel_h5
 * (CPP/disk_io_routines.cpp:1078-1164): datasets "Nalpha", "Np_WP", "Nq_WP"
 * (int32[1]), "P123_sparse_dim" (uint64[1]), tables "p boundaries" /
 * "q boundaries" {int32 index, float64 mesh point} and "pw channels" (10 int32
 * fields), "row indices" / "column indices" (int32[nnz]) and "values"
 * (float64[nnz]).  val/row/col are the COO arrays of tt_fill_P123_arrays. */
int tt_store_P123_h5(const char* filename, const double* val, const int* row, const int* col, size_t nnz,
                     const tt_fwp_states* fwp, const tt_pw_states* pw);
/* Replaces read_sparse_permutation_matrix_for_3N_channel_h5
 * (CPP/disk_io_routines.cpp:1166-1284) with its checks: Nalpha, Np_WP, Nq_WP,
 * the boundaries (bit-equal) and the pw table must match fwp/pw, else
 * TT_ERR_BADARG with the reference's message.  Callee allocates *val, *row,
 * *col (free with tt_free). */
int tt_read_P123_h5(const char* filename, double** val, int** row, int** col, size_t* nnz,
                    const tt_fwp_states* fwp, const tt_pw_states* pw);
/* The reference's P123 file name for a channel, folder + "/P123_sparse_JP_<2J>_<P>_Np_<Np>_Nq_<Nq>_J2max_<j>.h5"
 * (CPP/make_permutation_matrix.cpp:1320-1323), into buf[cap]. */
int tt_P123_h5_filename(char* buf, size_t cap, const char* folder, const tt_pw_states* pw, int Np_WP, int Nq_WP);

void tt_free(void* p);
const char* tt_last_error_string(void);
int tt_device_count(int* count);
/* Large device blocks (256 MB and up) that the library releases are kept for
 * its next allocations of about the same size (cudaMalloc / cudaFree of tens
 * of GB cost milliseconds each); this returns the current device's cached
 * blocks to the driver.  tt_run_destroy does the same. */
int tt_release_cached_device_memory(void);
/* Bytes of those blocks currently held for the current device. */
int tt_cached_device_memory(size_t* bytes);
/* Kernels launched by this library since load (diagnostic). */
unsigned long long tt_kernel_launches(void);

/* Kernel timing over a region (diagnostic; no counterpart in the reference).
 * Between tt_profile_begin and tt_profile_end every launch of the kernel
 * classes below is bracketed by CUDA events on its own stream; end waits for
 * them and tt_profile_read returns, per class, the launches, the summed event
 * time and the algorithmic flops and bytes booked for those launches:
 *   TC_UPDATE  trailing update C -= L U of the complex64 LU on tcgen05, 8 M N K flops
 *   SUBPANEL   pivoted factorisation of an m x w sub-panel (w <= 32): 4 m w^2 flops,
 *              2 m w sizeof(elem) bytes (panel read and written once)
 *   TRSV       forward + backward substitution, LU read once: n^2 sizeof(elem) bytes
 *   RESIDUAL   FP64 refinement residual b - x + A (G o x), A read once: 8 n^2 bytes
 *   A_BUILD    A = C^T (2 P123)(V C) */
#define TT_PROF_TC_UPDATE 0
#define TT_PROF_SUBPANEL 1
#define TT_PROF_TRSV 2
#define TT_PROF_RESIDUAL 3
#define TT_PROF_A_BUILD 4
/*   PANEL_TRSM  U = L^-1 X for the 32-wide unit-lower blocks of the panels: 4 w^2 cols flops
 *   OPERANDS    packing the tensor-core operands (splits, real-row planes): bytes read + written
 *   LASWP       row interchanges: 4 swaps cols sizeof(elem) bytes
 *   FORM_L      L = 1 - A G: 8 n^2 bytes read + n^2 sizeof(elem) written
 *   SUBST_PREP  inverted diagonal blocks of the substitutions and their neighbour products
 *   SIMT_UPDATE C -= L U on the CUDA cores (complex64 without tensor cores): 8 M N K flops */
#define TT_PROF_PANEL_TRSM 5
#define TT_PROF_OPERANDS 6
#define TT_PROF_LASWP 7
#define TT_PROF_FORM_L 8
#define TT_PROF_SUBST_PREP 9
#define TT_PROF_SIMT_UPDATE 10
/*   TC_PANEL    the tensor-core updates inside a panel and of its U block row (K below 256),
 *               booked apart from TC_UPDATE (the trailing updates, K >= 256): 8 M N K flops */
#define TT_PROF_TC_PANEL 11
/*   FP64_UPDATE C -= L U of the complex128 factorisation on the FP64 tensor cores (DMMA): 8 M N K flops */
#define TT_PROF_FP64_UPDATE 12
/*   VECTOR      O(n k) kernels of the solve: resolvents, right-hand sides, G o x,
 *               the refinement's axpy and norms (bytes read + written) */
#define TT_PROF_VECTOR 13
#define TT_PROF_COUNT 14
typedef struct tt_kernel_profile {
  unsigned long long launches;
  double ms;
  double flops;
  double bytes;
} tt_kernel_profile;
int tt_profile_begin(void);
/* Classes recorded by the next regions, bit k = class k (default all): a
 * region that times only the classes it reports keeps the event records of the
 * other launches off the host path. */
int tt_profile_select(unsigned long long class_mask);
int tt_profile_end(void);
int tt_profile_read(int kernel_class, tt_kernel_profile* out);

/* Host numerics the P123 tables are built from, doubled (2j, 2m) arguments:
 * replace gsl_sf_coupling_3j/6j/9j as wrapped by wigner_3j/6j/9j and
 * clebsch_gordan (CPP/General_functions/coupling_coefficients.h:12-24,
 * CPP/auxiliary.cpp:127-135). */
double tt_wigner_3j(int two_j1, int two_j2, int two_j3, int two_m1, int two_m2, int two_m3);
double tt_wigner_6j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6);
double tt_wigner_9j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6, int two_j7, int two_j8,
                    int two_j9);
double tt_clebsch_gordan(int two_j1, int two_j2, int two_j3, int two_m1, int two_m2, int two_m3);
/* Y_l^m(theta,0), 0 <= m <= l <= lmax at x = cos(theta), index l(l+1)/2+m: the
 * gsl_sf_legendre_array_e(GSL_SF_LEGENDRE_SPHARM, lmax, x, -1, out) table the
 * reference uses (CPP/make_permutation_matrix.cpp:549-589). */
int tt_legendre_spharm_array(int lmax, double x, double* out);
/* Gauss-Legendre rule on [-1,1] (gauss, CPP/General_functions/gauss_legendre.cpp:36-66). */
int tt_gauss_legendre(int n, double* x, double* w);

/* ---- layer 2: run handle -------------------------------------------- */

typedef struct tt_run tt_run;

/* Configure a run from key=value options with the reference's keys and
 * defaults (CPP/set_run_parameters.cpp:76-280, 577-615), e.g.
 * "Np_WP=16", "potential_model=malfliet_tjon", "lab_energies=13".  An option
 * without '=' that ends in ".txt" names an input-list file of key=value lines
 * (CPP/set_run_parameters.cpp:247-279, 641-644); options and files apply in
 * order, the last setting wins.  Builds the partial-wave basis, WP grids
 * (Chebyshev, or p_grid_type=custom with the boundaries read from
 * p_grid_filename / q_grid_filename), potential matrices, SWP states and
 * on-shell bins on the host (CPP/main.cpp:98-378). */
int tt_run_create(tt_run** run, int nopt, const char* const* opts);
void tt_run_destroy(tt_run* run);
/* Change one option of the linear solve (tc_product, panel_width, panel_order,
 * inverse_block, cta_pairs, mid_panel, energy_batch, refine_tol, refine_max_iter) for the run's next
 * solves; the states, grids and built operators stay.  Other keys: TT_ERR_BADARG. */
int tt_run_set_solve_option(tt_run* run, const char* key, const char* value);

/* Counts and per-channel facts. */
int tt_run_num_channels(const tt_run* run, int* n_chn);
int tt_run_channel_info(const tt_run* run, int chn, int* Nalpha, int* dense_dim, int* two_J_3N, int* P_3N,
                        int* n_deuteron);
int tt_run_num_energies(const tt_run* run, int* nE);
int tt_run_energies(const tt_run* run, double* T_lab, double* E_com, int* q_com_idx);
int tt_run_E_bound(const tt_run* run, double* E_bound);

/* Device stages for one channel: P123 in HBM, A in HBM, resolvents.
 * tt_run_build_P123 builds P123 on the device, or, when the run has
 * calculate_and_store_P123=false, reads the channel's P123 file from
 * P123_folder (tt_run_load_P123_h5) as the reference does.  Storing is
 * explicit (tt_run_store_P123_h5): the files reach GBs at Np = Nq = 30. */
int tt_run_build_P123(tt_run* run, int chn, int64_t* nnz);
int tt_run_build_A(tt_run* run, int chn, double* ms);
int tt_run_build_resolvent(tt_run* run, int chn);
/* Solve all on-shell energies of the channel; U as in tt_solve_faddeev_equations. */
int tt_run_solve(tt_run* run, int chn, int precision, tt_complex* U, tt_solve_report* report);
/* tt_run_solve for a subset of the run's on-shell energies: energy_idx[n_sel]
 * indexes tt_run_energies (distinct); U[d'*nd*n_sel + d*n_sel + s] for energy
 * energy_idx[s].  The unit of work a scan is sharded by across GPUs, one
 * (channel, energy) item or a group of them (the reference shards whole
 * channels across processes, CPP/main.cpp:168-170).  The channel's resident
 * resolvents afterwards hold the selected energies; tt_run_solve rebuilds them. */
int tt_run_solve_energies(tt_run* run, int chn, int precision, int n_sel, const int* energy_idx, tt_complex* U,
                          tt_solve_report* report);
/* tt_run_solve plus dU/dtheta (see tt_solve_faddeev_adjoint), for dV/dtheta
 * arrays over all 2N channels of the run (sizes as tt_run_get_host_array
 * which = 3 and 4).  With the run option adjoint_basis=total (default) this is
 * the total derivative: the SWP eigenvectors C, bin energies e_SWP and the
 * deuteron energy move with the potential (first-order perturbation of each
 * 2N block's eigenproblem, CPP/make_swp_states.cpp:114-183), and with them the
 * resolvent (CPP/make_resolvent.cpp:14-80, energies E_com + E_bound):
 *   dU = lambda^T dA (e + G o x) + (A^T lambda)^T (dG o x),
 *   dA = OP(dC)^T (2P) OP(V C) + OP(C)^T (2P) OP(dV C + V dC).
 * adjoint_basis=fixed keeps the basis and G, as tt_solve_faddeev_adjoint. */
int tt_run_solve_adjoint(tt_run* run, int chn, int precision, int n_theta, const double* dV_WP_unco_dtheta,
                         const double* dV_WP_coup_dtheta, tt_complex* U, tt_complex* dU_dtheta,
                         tt_solve_report* report);
/* The same derivative as a forward/backward pair, the contract of an
 * autograd function (no counterpart in the reference):
 * tt_run_adjoint_forward solves (as tt_run_solve) and keeps every energy's LU
 * factor, row interchanges and refined solution in the run handle when they
 * fit in HBM together (one energy group); tt_run_adjoint_backward takes a
 * cotangent U_bar (layout of U) and returns
 *   theta_bar[k] = Re sum_e conj(U_bar[e]) dU[e]/dtheta_k
 * for n_theta derivatives dV/dtheta (as tt_run_solve_adjoint), with the kept
 * factors (transposed solves only), or, when they were not kept, by factoring
 * again.  One backward per forward; the kept factors are released by it. */
int tt_run_adjoint_forward(tt_run* run, int chn, int precision, tt_complex* U, tt_solve_report* report);
int tt_run_adjoint_backward(tt_run* run, int chn, int n_theta, const double* dV_WP_unco_dtheta,
                            const double* dV_WP_coup_dtheta, const tt_complex* U_bar, double* theta_bar,
                            tt_solve_report* report);
/* First-order change of the run's SWP states for a change dV (layout of
 * tt_run_get_host_array which = 3, 4) of the WP potential matrices: dC (which =
 * 5, 6), the bin boundaries de_SWP (which = 7, 8) and dE_bound, from the
 * perturbation of each 2N block's eigenproblem (host FP64; the adjoint's
 * basis derivative).  Any output may be NULL. */
int tt_run_swp_derivative(const tt_run* run, const double* dV_WP_unco, const double* dV_WP_coup, double* dC_unco,
                          double* dC_coup, double* de_unco, double* de_coup, double* dE_bound);
/* Low-energy constants of the run's potential that the option lec_offsets
 * moves (LO_internal: C_1S0, C_3S1; none for malfliet_tjon), their values,
 * and dV/dLEC_k in the WP basis for all 2N channels (the potential is linear
 * in these contacts, so the central difference is exact up to rounding). */
int tt_run_num_lecs(const tt_run* run, int* n_lecs, double* values);
int tt_run_lec_derivative(const tt_run* run, int k, double* dV_WP_unco, double* dV_WP_coup);
/* Writes channel chn's resident P123 (after tt_run_build_P123) with
 * tt_store_P123_h5 to filename, or, if NULL, to the reference's file name in
 * the run's P123_folder (what fill_P123_arrays stores when
 * calculate_and_store_P123 is set, CPP/make_permutation_matrix.cpp:1364-1375). */
int tt_run_store_P123_h5(const tt_run* run, int chn, const char* filename);
/* Makes a P123 file the channel's resident P123 instead of building it, as
 * the reference reads its file when calculate_and_store_P123 is false
 * (CPP/make_permutation_matrix.cpp:1387-1403), with tt_read_P123_h5's checks
 * against the run's state space; filename NULL = the reference's name in the
 * run's P123_folder. */
int tt_run_load_P123_h5(tt_run* run, int chn, const char* filename, int64_t* nnz);
/* Release the channel's device data (all of it, or only A and the resolvents,
 * keeping P123 resident for the next parameter set or energy scan). */
int tt_run_release_channel(tt_run* run, int chn);
int tt_run_release_A(tt_run* run, int chn);

/* CUDA-event timer on the run's stream: start records an event, stop records
 * another, waits for it and returns the elapsed device time in ms. */
int tt_run_timer_start(tt_run* run);
int tt_run_timer_stop(tt_run* run, double* ms);

/* Host copies for checking (sizes from tt_run_channel_info / build results). */
int tt_run_get_P123_csr(const tt_run* run, int chn, int64_t* rowptr, int32_t* col, double* val);
int tt_run_get_A(const tt_run* run, int chn, double* A);
int tt_run_get_G(const tt_run* run, int chn, tt_complex* G);
/* which: 0 pw states (9 ints per alpha: L S J T l 2j 2J 2T P), 1 p_WP, 2 q_WP,
 * 3 V_unco, 4 V_coup, 5 C_unco, 6 C_coup, 7 e_unco, 8 e_coup.  With buf NULL
 * only *count is returned. */
int tt_run_get_host_array(const tt_run* run, int chn, int which, void* buf, size_t* count);

/* U-matrix text table in the reference's format (disk_io_routines.cpp:759-913). */
int tt_run_write_U_table(const tt_run* run, int chn, const tt_complex* U, const char* path);

/* Breakup cells of channel chn for the run's energies (the
 * include_breakup_channels part of find_on_shell_bins,
 * CPP/run_organizer.cpp:134-339; located at tt_run_create when the run was
 * made with include_breakup_channels=true, else on this call).  *num_cells
 * always; start[num_energies + 1] and cells[3 num_cells] = (alpha, q bin,
 * p bin) in the reference's order when not NULL.  Host work only. */
int tt_run_breakup_cells(const tt_run* run, int chn, int* num_cells, int* start, int* cells);

/* Pade solve (TT_PRECISION_PADE) of all the run's energies of channel chn
 * with the breakup amplitudes: U as tt_run_solve, U_BU[d*num_cells + b] as
 * tt_solve_faddeev_equations_breakup (caller allocates nd*num_cells). */
int tt_run_solve_breakup(tt_run* run, int chn, tt_complex* U, tt_complex* U_BU, tt_solve_report* report);

/* Breakup U-matrix text table in the reference's format
 * (restructure_breakup_data + store_U_BU_matrix_elements_txt,
 * disk_io_routines.cpp:341-706); boundaries of a cell outside the grid are
 * written as nan.  Host work only. */
int tt_run_write_U_BU_table(const tt_run* run, int chn, const tt_complex* U_BU, const char* path);

#ifdef __cplusplus
}
#endif

#endif /* TICTAC_B200_H */
