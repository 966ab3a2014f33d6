// The reference's U-matrix text tables: the breakup table of one channel
// (find_breakup_cells is declared in tt_host.h) and the number format of both.
#pragma once
#include <ostream>
#include <string>
#include <vector>

#include "tt_host.h"

namespace tt {

struct BreakupTableInput {
  const RunParams* rp = nullptr;
  PWChannel ch;
  const SWPStates* swp = nullptr;
  const OnShell* os = nullptr;
  std::vector<int> deut;            // the channel's deuteron states
  const BreakupCells* bu = nullptr;
  const double* U_BU = nullptr;     // interleaved complex, [nd][cells]
};

// The table of store_U_BU_matrix_elements_txt (CPP/disk_io_routines.cpp:
// 341-706): a row per (energy, cell of a pair), five columns per energy
// (T_lab, E_com, q_com and the on-shell q bin) and five per (alpha', alpha)
// pair (U, the cell's q and p boundaries as momenta).  Boundaries of a cell
// outside the grid are written as nan.
bool write_breakup_table(std::ostream& f, const BreakupTableInput& in, std::string* err);

// A U element part as the reference's tables write it
// (to_string_with_precision_and_sign, CPP/disk_io_routines.cpp:3-12): "+" in
// front of values >= 0, then 16 digits in scientific form.
std::string signed_scientific(double v);

}  // namespace tt
