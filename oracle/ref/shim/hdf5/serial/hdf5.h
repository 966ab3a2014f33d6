#include "../../tt_hdf5_shim.h"
