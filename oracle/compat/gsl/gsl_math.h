/* Oracle-only stand-in header; see gsl_compat.h. */
#include "gsl_compat.h"
