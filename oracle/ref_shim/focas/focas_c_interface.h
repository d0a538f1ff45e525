/* test-only stand-in for hilbert's focas C interface header: the oracle never
 * calls the Fortran orbital optimizer, it only needs the namespace import. */
#ifndef V2B_SHIM_FOCAS_C_INTERFACE_H
#define V2B_SHIM_FOCAS_C_INTERFACE_H
#include "../psi4_shim_core.h"
using namespace psi;
#endif
