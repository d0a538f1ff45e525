/* test-only stand-in: see psi4_shim_core.h */
#ifndef V2B_SHIM_PSI4_LIBPSIO_PSIO_HPP
#define V2B_SHIM_PSI4_LIBPSIO_PSIO_HPP
#include "../../psi4_shim_core.h"
#endif
