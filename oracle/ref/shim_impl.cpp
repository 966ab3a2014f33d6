// Implementations of the GSL / HDF5 / MKL subsets declared in shim/.
// Parity-oracle infrastructure: linked only into the reference build.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tt_math.h"
#include "shim/mkl.h"
#include "shim/tt_gsl_shim.h"
#include "shim/tt_hdf5_shim.h"

// ------------------------------------------------------------------ GSL
extern "C" {
double gsl_sf_coupling_3j(int a, int b, int c, int ma, int mb, int mc) { return tt::wigner3j(a, b, c, ma, mb, mc); }
double gsl_sf_coupling_6j(int a, int b, int c, int d, int e, int f) { return tt::wigner6j(a, b, c, d, e, f); }
double gsl_sf_coupling_9j(int a, int b, int c, int d, int e, int f, int g, int h, int i) {
  return tt::wigner9j(a, b, c, d, e, f, g, h, i);
}
double gsl_sf_legendre_Pl(int l, double x) { return tt::legendre_P(l, x); }
size_t gsl_sf_legendre_array_n(size_t lmax) { return (lmax + 1) * (lmax + 2) / 2 + 2 * lmax + 2; }
size_t gsl_sf_legendre_array_index(size_t l, size_t m) { return l * (l + 1) / 2 + m; }
int gsl_sf_legendre_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase, double* out) {
  if (norm != GSL_SF_LEGENDRE_SPHARM) {
    std::fprintf(stderr, "shim: only GSL_SF_LEGENDRE_SPHARM is provided\n");
    std::abort();
  }
  tt::legendre_spharm_array((int)lmax, x, out);
  if (csphase > 0)  // remove the Condon-Shortley phase
    for (size_t l = 0; l <= lmax; l++)
      for (size_t m = 1; m <= l; m += 2) out[l * (l + 1) / 2 + m] = -out[l * (l + 1) / 2 + m];
  return GSL_SUCCESS;
}
double gsl_sf_legendre_sphPlm(int l, int m, double x) {
  std::vector<double> t((size_t)(l + 1) * (l + 2) / 2);
  tt::legendre_spharm_array(l, x, t.data());
  return t[(size_t)l * (l + 1) / 2 + m];
}
double gsl_sf_pow_int(double x, int n) {
  if (n < 0) {
    x = 1.0 / x;
    n = -n;
  }
  double value = 1.0;
  do {
    if (n & 1) value *= x;
    n >>= 1;
    x *= x;
  } while (n);
  return value;
}
gsl_complex gsl_complex_exp(gsl_complex a) {
  std::complex<double> z = std::exp(std::complex<double>(a.dat[0], a.dat[1]));
  gsl_complex r;
  r.dat[0] = z.real();
  r.dat[1] = z.imag();
  return r;
}
gsl_complex gsl_complex_mul_real(gsl_complex a, double x) {
  a.dat[0] *= x;
  a.dat[1] *= x;
  return a;
}
gsl_complex gsl_complex_conjugate(gsl_complex a) {
  a.dat[1] = -a.dat[1];
  return a;
}
static const gsl_root_fdfsolver_type tt_newton_type = {"newton"};
const gsl_root_fdfsolver_type* gsl_root_fdfsolver_newton = &tt_newton_type;
gsl_root_fdfsolver* gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type* T) {
  gsl_root_fdfsolver* s = new gsl_root_fdfsolver();
  s->type = T;
  return s;
}
int gsl_root_fdfsolver_set(gsl_root_fdfsolver* s, gsl_function_fdf* fdf, double root) {
  s->fdf = fdf;
  s->root = root;
  fdf->fdf(root, fdf->params, &s->f, &s->df);
  return GSL_SUCCESS;
}
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver* s) {
  // Newton step x <- x - f(x)/f'(x), then f and f' at the new point
  const double r = s->root - (s->f / s->df);
  s->root = r;
  s->fdf->fdf(r, s->fdf->params, &s->f, &s->df);
  return GSL_SUCCESS;
}
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver* s) { return s->root; }
void gsl_root_fdfsolver_free(gsl_root_fdfsolver* s) { delete s; }
int gsl_root_test_delta(double x1, double x0, double epsabs, double epsrel) {
  return (std::fabs(x1 - x0) < epsabs + epsrel * std::fabs(x1)) ? GSL_SUCCESS : GSL_CONTINUE;
}
}  // extern "C"

// ------------------------------------------------------------------ HDF5
namespace {
struct H5Dataset {
  std::string name;
  std::vector<unsigned char> bytes;
  size_t elem = 0;
};
struct H5File {
  std::string path;
  bool writable = false;
  std::map<std::string, H5Dataset> ds;
};
struct H5Handle {
  int kind;  // 1 file, 2 space, 3 dataset, 4 type
  int64_t file = 0;
  std::string name;
  size_t count = 0;
  size_t elem = 0;
};
std::mutex g_h5_mu;
std::map<int64_t, H5File> g_files;
std::map<int64_t, H5Handle> g_handles;
int64_t g_next = 1000;
const char kMagic[8] = {'T', 'T', 'H', '5', 'C', 'N', 'T', '1'};

void save_file(const H5File& f) {
  std::ofstream o(f.path, std::ios::binary | std::ios::trunc);
  o.write(kMagic, 8);
  uint64_t nds = f.ds.size();
  o.write((const char*)&nds, 8);
  for (auto& kv : f.ds) {
    uint64_t nl = kv.first.size(), nb = kv.second.bytes.size(), el = kv.second.elem;
    o.write((const char*)&nl, 8);
    o.write(kv.first.data(), nl);
    o.write((const char*)&el, 8);
    o.write((const char*)&nb, 8);
    o.write((const char*)kv.second.bytes.data(), nb);
  }
}
bool load_file(const std::string& path, H5File& f) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  char m[8];
  in.read(m, 8);
  if (!in || std::memcmp(m, kMagic, 8) != 0) return false;
  uint64_t nds = 0;
  in.read((char*)&nds, 8);
  for (uint64_t i = 0; i < nds; i++) {
    uint64_t nl, el, nb;
    in.read((char*)&nl, 8);
    std::string name(nl, '\0');
    in.read(&name[0], nl);
    in.read((char*)&el, 8);
    in.read((char*)&nb, 8);
    H5Dataset d;
    d.name = name;
    d.elem = el;
    d.bytes.resize(nb);
    in.read((char*)d.bytes.data(), nb);
    if (!in) return false;
    f.ds[name] = std::move(d);
  }
  f.path = path;
  return true;
}
size_t type_size(hid_t t) {
  auto it = g_handles.find(t);
  if (it != g_handles.end() && it->second.kind == 4) return it->second.elem;
  return 0;
}
hid_t make_type(size_t sz) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  const int64_t h = g_next++;
  H5Handle hh;
  hh.kind = 4;
  hh.elem = sz;
  g_handles[h] = hh;
  return h;
}
}  // namespace

extern "C" {
hid_t tt_h5_native_int = make_type(sizeof(int));
hid_t tt_h5_native_double = make_type(sizeof(double));
hid_t tt_h5_native_ullong = make_type(sizeof(unsigned long long));

hid_t H5Fcreate(const char* name, unsigned, hid_t, hid_t) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  const int64_t h = g_next++;
  H5File f;
  f.path = name;
  f.writable = true;
  g_files[h] = f;
  H5Handle hh;
  hh.kind = 1;
  hh.file = h;
  g_handles[h] = hh;
  return h;
}
hid_t H5Fopen(const char* name, unsigned, hid_t) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  H5File f;
  if (!load_file(name, f)) return -1;
  const int64_t h = g_next++;
  g_files[h] = f;
  H5Handle hh;
  hh.kind = 1;
  hh.file = h;
  g_handles[h] = hh;
  return h;
}
herr_t H5Fclose(hid_t fh) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto it = g_files.find(fh);
  if (it == g_files.end()) return -1;
  if (it->second.writable) save_file(it->second);
  g_files.erase(it);
  g_handles.erase(fh);
  return 0;
}
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t*) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  size_t c = 1;
  for (int i = 0; i < rank; i++) c *= dims[i];
  const int64_t h = g_next++;
  H5Handle hh;
  hh.kind = 2;
  hh.count = c;
  g_handles[h] = hh;
  return h;
}
herr_t H5Sclose(hid_t s) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  g_handles.erase(s);
  return 0;
}
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t, hid_t, hid_t) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto sp = g_handles.find(space);
  if (sp == g_handles.end() || g_files.find(loc) == g_files.end()) return -1;
  const int64_t h = g_next++;
  H5Handle hh;
  hh.kind = 3;
  hh.file = loc;
  hh.name = name;
  hh.count = sp->second.count;
  hh.elem = type_size(type);
  g_handles[h] = hh;
  H5Dataset d;
  d.name = name;
  d.elem = hh.elem;
  d.bytes.assign(hh.count * hh.elem, 0);
  g_files[loc].ds[name] = d;
  return h;
}
hid_t H5Dopen(hid_t loc, const char* name, hid_t) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto f = g_files.find(loc);
  if (f == g_files.end()) return -1;
  auto d = f->second.ds.find(name);
  if (d == f->second.ds.end()) return -1;
  const int64_t h = g_next++;
  H5Handle hh;
  hh.kind = 3;
  hh.file = loc;
  hh.name = name;
  hh.elem = d->second.elem;
  hh.count = hh.elem ? d->second.bytes.size() / hh.elem : 0;
  g_handles[h] = hh;
  return h;
}
herr_t H5Dwrite(hid_t d, hid_t, hid_t, hid_t, hid_t, const void* buf) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto h = g_handles.find(d);
  if (h == g_handles.end()) return -1;
  H5Dataset& ds = g_files[h->second.file].ds[h->second.name];
  std::memcpy(ds.bytes.data(), buf, ds.bytes.size());
  return 0;
}
herr_t H5Dread(hid_t d, hid_t, hid_t, hid_t, hid_t, void* buf) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto h = g_handles.find(d);
  if (h == g_handles.end()) return -1;
  const H5Dataset& ds = g_files[h->second.file].ds[h->second.name];
  std::memcpy(buf, ds.bytes.data(), ds.bytes.size());
  return 0;
}
herr_t H5Dclose(hid_t d) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  g_handles.erase(d);
  return 0;
}
hid_t H5Tcopy(hid_t t) { return make_type(type_size(t)); }
herr_t H5Tset_order(hid_t, H5T_order_t) { return 0; }
herr_t H5Tclose(hid_t) { return 0; }
hid_t H5Gopen(hid_t loc, const char*, hid_t) { return loc; }
herr_t H5Gclose(hid_t) { return 0; }
herr_t H5TBmake_table(const char*, hid_t loc, const char* name, hsize_t, hsize_t nrecords, size_t type_size_,
                      const char*[], const size_t*, const hid_t*, hsize_t, void*, int, const void* buf) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto f = g_files.find(loc);
  if (f == g_files.end()) return -1;
  H5Dataset d;
  d.name = name;
  d.elem = type_size_;
  d.bytes.resize(nrecords * type_size_);
  std::memcpy(d.bytes.data(), buf, d.bytes.size());
  f->second.ds[name] = d;
  return 0;
}
herr_t H5TBread_table(hid_t loc, const char* name, size_t, const size_t*, const size_t*, void* dst) {
  std::lock_guard<std::mutex> g(g_h5_mu);
  auto f = g_files.find(loc);
  if (f == g_files.end()) return -1;
  auto d = f->second.ds.find(name);
  if (d == f->second.ds.end()) return -1;
  std::memcpy(dst, d->second.bytes.data(), d->second.bytes.size());
  return 0;
}
}  // extern "C"

// ------------------------------------------------------------------ MKL -> scipy OpenBLAS
extern "C" {
void scipy_cblas_sgemm(int, int, int, int, int, int, float, const float*, int, const float*, int, float, float*, int);
void scipy_cblas_dgemm(int, int, int, int, int, int, double, const double*, int, const double*, int, double, double*,
                       int);
void scipy_cblas_cgemm(int, int, int, int, int, int, const void*, const void*, int, const void*, int, const void*,
                       void*, int);
void scipy_cblas_zgemm(int, int, int, int, int, int, const void*, const void*, int, const void*, int, const void*,
                       void*, int);
void scipy_cblas_cdotu_sub(int, const void*, int, const void*, int, void*);
void scipy_cblas_zdotu_sub(int, const void*, int, const void*, int, void*);
void scipy_dgemv_(const char*, const int*, const int*, const double*, const double*, const int*, const double*,
                  const int*, const double*, double*, const int*);
int scipy_LAPACKE_sgetrf(int, int, int, float*, int, int*);
int scipy_LAPACKE_dgetrf(int, int, int, double*, int, int*);
int scipy_LAPACKE_cgetrf(int, int, int, void*, int, int*);
int scipy_LAPACKE_zgetrf(int, int, int, void*, int, int*);
int scipy_LAPACKE_sgetrs(int, char, int, int, const float*, int, const int*, float*, int);
int scipy_LAPACKE_dgetrs(int, char, int, int, const double*, int, const int*, double*, int);
int scipy_LAPACKE_cgetrs(int, char, int, int, const void*, int, const int*, void*, int);
int scipy_LAPACKE_zgetrs(int, char, int, int, const void*, int, const int*, void*, int);
int scipy_LAPACKE_sspevd(int, char, char, int, float*, float*, float*, int);
int scipy_LAPACKE_dspevd(int, char, char, int, double*, double*, double*, int);
void scipy_openblas_set_num_threads(int);
}

void cblas_sgemm(CBLAS_LAYOUT l, CBLAS_TRANSPOSE a, CBLAS_TRANSPOSE b, MKL_INT m, MKL_INT n, MKL_INT k, float al,
                 const float* A, MKL_INT lda, const float* B, MKL_INT ldb, float be, float* C, MKL_INT ldc) {
  scipy_cblas_sgemm(l, a, b, (int)m, (int)n, (int)k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
}
void cblas_dgemm(CBLAS_LAYOUT l, CBLAS_TRANSPOSE a, CBLAS_TRANSPOSE b, MKL_INT m, MKL_INT n, MKL_INT k, double al,
                 const double* A, MKL_INT lda, const double* B, MKL_INT ldb, double be, double* C, MKL_INT ldc) {
  scipy_cblas_dgemm(l, a, b, (int)m, (int)n, (int)k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
}
void cblas_cgemm(CBLAS_LAYOUT l, CBLAS_TRANSPOSE a, CBLAS_TRANSPOSE b, MKL_INT m, MKL_INT n, MKL_INT k, const void* al,
                 const void* A, MKL_INT lda, const void* B, MKL_INT ldb, const void* be, void* C, MKL_INT ldc) {
  scipy_cblas_cgemm(l, a, b, (int)m, (int)n, (int)k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
}
void cblas_zgemm(CBLAS_LAYOUT l, CBLAS_TRANSPOSE a, CBLAS_TRANSPOSE b, MKL_INT m, MKL_INT n, MKL_INT k, const void* al,
                 const void* A, MKL_INT lda, const void* B, MKL_INT ldb, const void* be, void* C, MKL_INT ldc) {
  scipy_cblas_zgemm(l, a, b, (int)m, (int)n, (int)k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
}
void cblas_cdotu_sub(MKL_INT n, const void* x, MKL_INT ix, const void* y, MKL_INT iy, void* r) {
  scipy_cblas_cdotu_sub((int)n, x, (int)ix, y, (int)iy, r);
}
void cblas_zdotu_sub(MKL_INT n, const void* x, MKL_INT ix, const void* y, MKL_INT iy, void* r) {
  scipy_cblas_zdotu_sub((int)n, x, (int)ix, y, (int)iy, r);
}
void dgemv(const char* t, const MKL_INT* m, const MKL_INT* n, const double* al, const double* a, const MKL_INT* lda,
           const double* x, const MKL_INT* ix, const double* be, double* y, const MKL_INT* iy) {
  int mm = (int)*m, nn = (int)*n, ll = (int)*lda, xi = (int)*ix, yi = (int)*iy;
  scipy_dgemv_(t, &mm, &nn, al, a, &ll, x, &xi, be, y, &yi);
}
template <typename F>
static MKL_INT getrf_widen(MKL_INT m, MKL_INT n, MKL_INT* ipiv, F call) {
  std::vector<int> p((size_t)std::min(m, n));
  const int info = call(p.data());
  for (size_t i = 0; i < p.size(); i++) ipiv[i] = p[i];
  return info;
}
template <typename F>
static MKL_INT getrs_narrow(MKL_INT n, const MKL_INT* ipiv, F call) {
  std::vector<int> p((size_t)n);
  for (size_t i = 0; i < p.size(); i++) p[i] = (int)ipiv[i];
  return call(p.data());
}
MKL_INT LAPACKE_sgetrf(int l, MKL_INT m, MKL_INT n, float* a, MKL_INT lda, MKL_INT* ipiv) {
  return getrf_widen(m, n, ipiv, [&](int* p) { return scipy_LAPACKE_sgetrf(l, (int)m, (int)n, a, (int)lda, p); });
}
MKL_INT LAPACKE_dgetrf(int l, MKL_INT m, MKL_INT n, double* a, MKL_INT lda, MKL_INT* ipiv) {
  return getrf_widen(m, n, ipiv, [&](int* p) { return scipy_LAPACKE_dgetrf(l, (int)m, (int)n, a, (int)lda, p); });
}
MKL_INT LAPACKE_cgetrf(int l, MKL_INT m, MKL_INT n, std::complex<float>* a, MKL_INT lda, MKL_INT* ipiv) {
  return getrf_widen(m, n, ipiv, [&](int* p) { return scipy_LAPACKE_cgetrf(l, (int)m, (int)n, a, (int)lda, p); });
}
MKL_INT LAPACKE_zgetrf(int l, MKL_INT m, MKL_INT n, std::complex<double>* a, MKL_INT lda, MKL_INT* ipiv) {
  return getrf_widen(m, n, ipiv, [&](int* p) { return scipy_LAPACKE_zgetrf(l, (int)m, (int)n, a, (int)lda, p); });
}
MKL_INT LAPACKE_sgetrs(int l, char t, MKL_INT n, MKL_INT nr, const float* a, MKL_INT lda, const MKL_INT* ipiv, float* b,
                       MKL_INT ldb) {
  return getrs_narrow(n, ipiv, [&](const int* p) {
    return scipy_LAPACKE_sgetrs(l, t, (int)n, (int)nr, a, (int)lda, p, b, (int)ldb);
  });
}
MKL_INT LAPACKE_dgetrs(int l, char t, MKL_INT n, MKL_INT nr, const double* a, MKL_INT lda, const MKL_INT* ipiv,
                       double* b, MKL_INT ldb) {
  return getrs_narrow(n, ipiv, [&](const int* p) {
    return scipy_LAPACKE_dgetrs(l, t, (int)n, (int)nr, a, (int)lda, p, b, (int)ldb);
  });
}
MKL_INT LAPACKE_cgetrs(int l, char t, MKL_INT n, MKL_INT nr, const std::complex<float>* a, MKL_INT lda,
                       const MKL_INT* ipiv, std::complex<float>* b, MKL_INT ldb) {
  return getrs_narrow(n, ipiv, [&](const int* p) {
    return scipy_LAPACKE_cgetrs(l, t, (int)n, (int)nr, a, (int)lda, p, b, (int)ldb);
  });
}
MKL_INT LAPACKE_zgetrs(int l, char t, MKL_INT n, MKL_INT nr, const std::complex<double>* a, MKL_INT lda,
                       const MKL_INT* ipiv, std::complex<double>* b, MKL_INT ldb) {
  return getrs_narrow(n, ipiv, [&](const int* p) {
    return scipy_LAPACKE_zgetrs(l, t, (int)n, (int)nr, a, (int)lda, p, b, (int)ldb);
  });
}
MKL_INT LAPACKE_sspevd(int l, char j, char u, MKL_INT n, float* ap, float* w, float* z, MKL_INT ldz) {
  return scipy_LAPACKE_sspevd(l, j, u, (int)n, ap, w, z, (int)ldz);
}
MKL_INT LAPACKE_dspevd(int l, char j, char u, MKL_INT n, double* ap, double* w, double* z, MKL_INT ldz) {
  return scipy_LAPACKE_dspevd(l, j, u, (int)n, ap, w, z, (int)ldz);
}
void mkl_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }
void mkl_dimatcopy(char, char, size_t, size_t, double, double*, size_t, size_t) {
  std::fprintf(stderr, "shim: mkl_dimatcopy is not provided (keep_CPVC_in_mem path)\n");
  std::abort();
}

// ------------------------------------------------------------------ Fortran potentials (not compilable here)
extern "C" {
static void no_fortran(const char* what) {
  std::fprintf(stderr, "reference build: %s needs the Fortran potential library (no Fortran compiler)\n", what);
  std::abort();
}
void chp_set_Idaho_N3LO(double*) { no_fortran("Idaho_N3LO"); }
void chp_set_N2LOopt(double*) { no_fortran("N2LOopt"); }
void chp_set_ispot_lo(double*) { no_fortran("IS_LO"); }
void chp_set_ispot_nlo(double*) { no_fortran("IS_NLO"); }
void chp_set_ispot_n2lo(double*) { no_fortran("IS_N2LO"); }
void chp_set_ispot_n3lo(double*) { no_fortran("IS_N3LO"); }
void __idaho_chiral_potential_MOD_chp(double*, double*, int*, int*, int*, int*, int*, double*) { no_fortran("chp"); }
void nijmegen_fort_interface(double*, double*, int*, int*, int*, int*, int*, double*) { no_fortran("nijmegen"); }
}
