/* test-only stand-in: the oracle holds the optimizer pointer but never creates one */
#ifndef V2B_SHIM_ORBITAL_OPTIMIZER_H
#define V2B_SHIM_ORBITAL_OPTIMIZER_H
#include "../psi4_shim_core.h"
namespace hilbert { class OrbitalOptimizer; }
#endif
