// focas's density-fitted integral transform and its adjoint (see v2b_transform.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace v2b {

// largest orbital count of the shared-memory transform (four padded 80 x 80
// matrices fill 207 KB of the 227 KB a CTA can hold)
constexpr int kTransformMaxDim = 80;

// Bp_Q = U^T B_Q U for Q = 0 .. count-1 (n x n row-major, device memory)
cudaError_t launch_df_transform(const double *U, const double *B, double *Bp, int n, int count,
                                cudaStream_t s);
// dU = sum_Q (B_Q U M_Q^T + B_Q^T U M_Q); slab: count * n * n doubles of scratch
cudaError_t launch_df_transform_adjoint(const double *U, const double *B, const double *M, double *dU,
                                        double *slab, int n, int count, cudaStream_t s);

}  // namespace v2b
