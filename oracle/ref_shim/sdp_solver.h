/* test-only stand-in for libsdp's header: the oracle only stores the pointer */
#ifndef V2B_SHIM_SDP_SOLVER_H
#define V2B_SHIM_SDP_SOLVER_H
namespace libsdp { class SDPSolver; }
#endif
