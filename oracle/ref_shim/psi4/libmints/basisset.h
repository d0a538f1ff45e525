/* test-only stand-in: see psi4_shim_core.h */
#ifndef V2B_SHIM_PSI4_LIBMINTS_BASISSET_H
#define V2B_SHIM_PSI4_LIBMINTS_BASISSET_H
#include "../../psi4_shim_core.h"
#endif
