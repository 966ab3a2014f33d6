#include "../tt_gsl_shim.h"
