#include "mkl.h"
