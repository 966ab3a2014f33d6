// P123 files in the reference's HDF5 layout, written and read without libhdf5.
//
// The reference stores one channel's permutation matrix with
// store_sparse_permutation_matrix_for_3N_channel_h5 and reads it back with
// read_sparse_permutation_matrix_for_3N_channel_h5
// (CPP/disk_io_routines.cpp:1078-1164, 1166-1284): root-group datasets
//   "Nalpha", "Np_WP", "Nq_WP"   int32[1]            (write_integer_to_h5, :1286-1302)
//   "P123_sparse_dim"            uint64[1]           (write_ULL_integer_to_h5, :1336-1352)
//   "p boundaries", "q boundaries"  tables {int32 "index", float64 "mesh point"}, N+1 records
//                                (write_WP_boundaries_to_h5 via H5TBmake_table, :1386-1432)
//   "pw channels"                table of 10 int32 fields, Nalpha records
//                                (write_PW_statespace_to_h5, :1474-1545)
//   "row indices", "column indices" int32[nnz], "values" float64[nnz], little endian
//                                (write_sparse_permutation_matrix_h5, :1625-1672)
// This file format subset: superblock version 0, version-1 object headers,
// the root group as a symbol table (v1 B-tree + local heap), contiguous
// storage, little-endian fixed-point / IEEE double / compound / fixed-length
// string datatypes.  The reader also follows object-header continuation
// messages and reads chunked datasets indexed by a version-1 B-tree without
// filters, which is how H5TBmake_table stores its tables.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tt {

// One pw-channels record in the reference's field order ("index", "L_12",
// "S_12", "J_12", "T_12", "l_3", "2*j_3", "2*T_total", "2*J_total",
// "PAR_total"), whatever the byte offsets in the file's compound type.
constexpr int kPwFields = 10;
extern const char* const kPwFieldNames[kPwFields];

struct P123H5 {
  int Nalpha = 0, Np_WP = 0, Nq_WP = 0;
  uint64_t nnz = 0;
  std::vector<double> p_WP, q_WP;  // [Np_WP+1], [Nq_WP+1]
  std::vector<int32_t> pw;         // [Nalpha][kPwFields]
  std::vector<int32_t> row, col;   // [nnz]
  std::vector<double> val;         // [nnz]
};

// Writes the file; row/col/val may be passed as external pointers of length
// f.nnz (the vectors in f are then ignored) to avoid copying large arrays.
bool h5_write_p123(const std::string& path, const P123H5& f, const int32_t* row, const int32_t* col,
                   const double* val, std::string* err);
bool h5_read_p123(const std::string& path, P123H5& f, std::string* err);

// The reference's file name (CPP/make_permutation_matrix.cpp:1320-1323).
std::string p123_h5_filename(const std::string& folder, int two_J_3N, int P_3N, int Np_WP, int Nq_WP, int J_2N_max);

}  // namespace tt
