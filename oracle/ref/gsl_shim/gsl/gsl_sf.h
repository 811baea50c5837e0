/* GSL stand-in header: see gsl_shim_types.h */
#include "gsl_shim_types.h"
