/* Forwarding header of the oracle's GSL subset (test infrastructure only). */
#include "ipg_gsl_shim.h"
