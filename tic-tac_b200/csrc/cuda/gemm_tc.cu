// Tensor-core (tcgen05) trailing update of the complex64 LU.  Placeholder
// until the tcgen05 kernel lands: reports UNSUPPORTED so no caller silently
// runs another path.
#include "tt_lu_internal.h"

namespace tt {

int lu_update_tc(float2*, int, int, int, cudaStream_t) {
  set_error("tcgen05 trailing update not built");
  return TT_ERR_UNSUPPORTED;
}

}  // namespace tt
