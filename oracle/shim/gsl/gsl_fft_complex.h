/* Forwarding header: see gsl_shim.h (oracle test infrastructure). */
#include "gsl_shim.h"
