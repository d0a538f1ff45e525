/* test-only stand-in: see psi4_shim_core.h */
#ifndef V2B_SHIM_PSI4_LIBPSI4UTIL_PSIOUTSTREAM_H
#define V2B_SHIM_PSI4_LIBPSI4UTIL_PSIOUTSTREAM_H
#include "../../psi4_shim_core.h"
#endif
