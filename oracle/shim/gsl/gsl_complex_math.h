/* GSL header subset for the oracle build (test infrastructure only); see gsl_shim_types.h. */
#include "gsl_shim_types.h"
