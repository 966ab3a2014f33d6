/* MKL subset used by the reference, forwarded to the OpenBLAS/LAPACKE build
 * bundled with scipy (LP64).  ILP64 integer arguments are narrowed, pivots
 * widened.  Test infrastructure only. */
#ifndef TT_MKL_SHIM_H
#define TT_MKL_SHIM_H
#include <complex>
typedef long long MKL_INT;
typedef long long MKL_INT64;
typedef long long _INTEGER_t;
enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
void cblas_sgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, float, const float*, MKL_INT,
                 const float*, MKL_INT, float, float*, MKL_INT);
void cblas_dgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, double, const double*,
                 MKL_INT, const double*, MKL_INT, double, double*, MKL_INT);
void cblas_cgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, const void*, const void*,
                 MKL_INT, const void*, MKL_INT, const void*, void*, MKL_INT);
void cblas_zgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, const void*, const void*,
                 MKL_INT, const void*, MKL_INT, const void*, void*, MKL_INT);
void cblas_cdotu_sub(MKL_INT, const void*, MKL_INT, const void*, MKL_INT, void*);
void cblas_zdotu_sub(MKL_INT, const void*, MKL_INT, const void*, MKL_INT, void*);
void dgemv(const char*, const MKL_INT*, const MKL_INT*, const double*, const double*, const MKL_INT*, const double*,
           const MKL_INT*, const double*, double*, const MKL_INT*);
MKL_INT LAPACKE_sgetrf(int, MKL_INT, MKL_INT, float*, MKL_INT, MKL_INT*);
MKL_INT LAPACKE_dgetrf(int, MKL_INT, MKL_INT, double*, MKL_INT, MKL_INT*);
MKL_INT LAPACKE_cgetrf(int, MKL_INT, MKL_INT, std::complex<float>*, MKL_INT, MKL_INT*);
MKL_INT LAPACKE_zgetrf(int, MKL_INT, MKL_INT, std::complex<double>*, MKL_INT, MKL_INT*);
MKL_INT LAPACKE_sgetrs(int, char, MKL_INT, MKL_INT, const float*, MKL_INT, const MKL_INT*, float*, MKL_INT);
MKL_INT LAPACKE_dgetrs(int, char, MKL_INT, MKL_INT, const double*, MKL_INT, const MKL_INT*, double*, MKL_INT);
MKL_INT LAPACKE_cgetrs(int, char, MKL_INT, MKL_INT, const std::complex<float>*, MKL_INT, const MKL_INT*,
                       std::complex<float>*, MKL_INT);
MKL_INT LAPACKE_zgetrs(int, char, MKL_INT, MKL_INT, const std::complex<double>*, MKL_INT, const MKL_INT*,
                       std::complex<double>*, MKL_INT);
MKL_INT LAPACKE_sspevd(int, char, char, MKL_INT, float*, float*, float*, MKL_INT);
MKL_INT LAPACKE_dspevd(int, char, char, MKL_INT, double*, double*, double*, MKL_INT);
void mkl_set_num_threads(int);
void mkl_dimatcopy(char, char, size_t, size_t, double, double*, size_t, size_t);
#endif
