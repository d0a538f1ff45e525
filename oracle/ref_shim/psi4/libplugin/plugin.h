/* test-only stand-in: see psi4_shim_core.h */
#ifndef V2B_SHIM_PSI4_LIBPLUGIN_PLUGIN_H
#define V2B_SHIM_PSI4_LIBPLUGIN_PLUGIN_H
#include "../../psi4_shim_core.h"
#endif
