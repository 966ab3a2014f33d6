/* HDF5 subset used by the reference's P123 storage (disk_io_routines.cpp),
 * backed by a private one-file container so the reference can read back what
 * it wrote.  Not the HDF5 file format.  Test infrastructure only. */
#ifndef TT_HDF5_SHIM_H
#define TT_HDF5_SHIM_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef int H5T_order_t;
#define HOFFSET(S, M) (offsetof(S, M))
#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u
#define H5T_ORDER_LE 0
extern hid_t tt_h5_native_int, tt_h5_native_double, tt_h5_native_ullong;
#define H5T_NATIVE_INT tt_h5_native_int
#define H5T_NATIVE_DOUBLE tt_h5_native_double
#define H5T_NATIVE_ULLONG tt_h5_native_ullong
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
herr_t H5Fclose(hid_t f);
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
herr_t H5Sclose(hid_t s);
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
hid_t H5Dopen(hid_t loc, const char* name, hid_t dapl);
herr_t H5Dwrite(hid_t d, hid_t memtype, hid_t mspace, hid_t fspace, hid_t xfer, const void* buf);
herr_t H5Dread(hid_t d, hid_t memtype, hid_t mspace, hid_t fspace, hid_t xfer, void* buf);
herr_t H5Dclose(hid_t d);
hid_t H5Tcopy(hid_t t);
herr_t H5Tset_order(hid_t t, H5T_order_t order);
herr_t H5Tclose(hid_t t);
hid_t H5Gopen(hid_t loc, const char* name, hid_t gapl);
herr_t H5Gclose(hid_t g);
herr_t H5TBmake_table(const char* title, hid_t loc, const char* name, hsize_t nfields, hsize_t nrecords,
                      size_t type_size, const char* field_names[], const size_t* field_offset,
                      const hid_t* field_types, hsize_t chunk_size, void* fill_data, int compress, const void* buf);
herr_t H5TBread_table(hid_t loc, const char* name, size_t dst_size, const size_t* dst_offset,
                      const size_t* dst_sizes, void* dst_buf);
#ifdef __cplusplus
}
#endif
#endif
