// Spin-summed active densities for the orbital optimiser (see v2b_orbital.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace v2b {

struct PackArgs {
    int n;                            // active orbitals
    int64_t d2ab, d2aa, d2bb, d1a, d1b;   // block offsets in x
    const int *ibas_aa;               // n x n aa geminal numbers (device)
};

// d2: (g00 (g00 + 1) / 2) packed elements, g00 = n (n + 1) / 2; d1: g00
__global__ void pack_spatial_density_kernel(const double *__restrict__ x, PackArgs a,
                                            double *__restrict__ d2, double *__restrict__ d1);

}  // namespace v2b
