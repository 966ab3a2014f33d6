/* CPU oracle of the WPCD hot path: a plain-C restatement of the reference's
 * algorithm, used ONLY as the checker in tests/, by __graft_entry__.smoke() and
 * as bench.py's cpu_baseline.  Never linked into or called by the product.
 *
 * Parity pinning: tests/test_oracle_golden.py checks every function here against the
 * golden fixtures produced by the reference's own code (tests/golden/). */
#ifndef TT_ORACLE_H
#define TT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

/* P123 of one channel in the reference's row-major COO order; arrays are
 * malloc'ed (free with to_free).  pw: Nalpha x 9 ints (L S J T l 2j 2J 2T P).
 * Follows calculate_WP_overlap and calculate_permutation_elements_for_3N_channel
 * (CPP/make_permutation_matrix.cpp:160-255, 324-943), calculate_P123_element_in_WP_basis_mod
 * and Gtilde_subarray_new (CPP/auxiliary.cpp:660-746, 950-1067). */
int to_p123(int Np, int Nq, const double* p_WP, const double* q_WP, int Nphi, int Nx, int Nalpha, const int* pw,
            int64_t* nnz, int32_t** row, int32_t** col, double** val);

/* Resolvent diagonal for one energy E (calculate_resolvent_array_in_SWP_basis,
 * CPP/make_resolvent.cpp:14-211).  e_off[alpha] indexes the Np+1 SWP energy
 * boundaries of alpha in e_swp.  G interleaved complex [2n]. */
void to_resolvent(int Nalpha, int Nq, int Np, const int32_t* e_off, const double* e_swp, const double* q_WP,
                  double E, double* G);

/* Dense A = C^T (2 P123) (V C) (row-major n x n) from P123 in CSC
 * (calculate_PVC_col / calculate_CPVC_col, CPP/solve_faddeev.cpp:4-181).
 * The 2N block structure is given per alpha: blk, part, and per block the
 * offset/dim into C and VC (row-major), plus the coupling lists cpl_off/cpl. */
void to_build_A(int Nalpha, int Nq, int Np, const int64_t* colptr, const int32_t* row, const double* val,
                const int32_t* blk, const int32_t* part, const int32_t* cpl_off, const int32_t* cpl,
                const int64_t* blk_off, const int32_t* blk_dim, const double* C, const double* VC, double* A);

/* U[d'*nd*nE + d*nE + j] (interleaved complex) of the dense solve of
 * (1 - A G_j) U = A for each energy j on the on-shell deuteron columns
 * (faddeev_dense_solver, CPP/solve_faddeev.cpp:305-438), by LU with partial
 * pivoting.  G: nE x n interleaved complex.  Returns 0, or k+1 on a zero pivot. */
int to_dense_solve(int n, const double* A, int nE, const double* G, const int32_t* q_idx, int nd,
                   const int32_t* deut, int Nq, int Np, double* U);

void to_free(void* p);

#endif
