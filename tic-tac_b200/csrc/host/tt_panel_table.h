// Complex64 LU panel width by matrix order and tensor-core product, measured
// on a B200 by tictac_b200.autotune (python -m tictac_b200.autotune --write):
// the first row whose product matches and whose n_max >= n gives the width.
// Products: 1 BF16x3 N=128 tiles, 2 TF32, 3 BF16x3 real-row.
// Tuned on J_2N_max=3, two_J_3N_max=7, Np=Nq=24, 2 energies, widths 256,384,512 (fastest of 3 repetitions).
#pragma once

namespace tt {

struct PanelWidthRow {
  int product;
  int n_max;
  int width;
};

constexpr PanelWidthRow kPanelWidthTable[] = {
    {2, 1 << 30, 512},
    {3, 30528, 512},
    {3, 35136, 384},
    {3, 1 << 30, 512},
    {1, 1 << 30, 512},
};

}  // namespace tt
