// Warm eigen-refinement of the PSD projection (see v2b_refine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "v2b_device.cuh"

namespace v2b {

// per-block state during one projection call
constexpr int kStWork = 0;     // refinement passes continue
constexpr int kStDone = 1;     // T passed the acceptance test; P written
constexpr int kStJacobi = 2;   // handed to the selective Jacobi kernels

constexpr int kRefineMaxCluster = 64;    // largest cluster diagonalised in place
constexpr int kRefineEdgeCap = 8192;     // non-separable pairs recorded per block and pass
constexpr int kRefinePasses = 3;         // Newton passes before the Jacobi fallback
constexpr int kRefineMinDim = 24;        // smaller blocks always take the Jacobi kernel
constexpr int kRefineThreads = 512;
constexpr double kRefineRho = 1e-2;      // separable: |t_pq| <= rho |d_p - d_q|
constexpr double kRefineKappa = 1e-5;    // accepted pairs still take Newton steps up to this size
// max |Vt Vt^T - I| before the last Newton-Schulz step; the step leaves about
// 3/4 of its square (3e-14)
constexpr double kRefineOrthDone = 2e-7;

// one cluster of one block: rows mem[moff .. moff+k) of block blk
struct ClusterJob {
    int blk, k, moff, qoff;
};

// acceptance test, pair classification and, for accepted blocks, P = Gamma o T
__global__ void refine_classify_kernel(const double *__restrict__ T, double *__restrict__ P,
                                       const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                       int *__restrict__ bstate,
                                       const unsigned long long *__restrict__ orth, int force,
                                       double gap_tol, double abs_tol, double *__restrict__ bnorm,
                                       int *h_state, int *h_nbad, int *h_nedge, int2 *h_edges);

// exact eigen-decomposition of each cluster's T[C, C]: rows of Qt (k x k) are
// the eigenvectors, lam the eigenvalues
__global__ void cluster_eig_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                                   const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                                   const int *__restrict__ mem, double *__restrict__ Qt,
                                   double *__restrict__ lam);

// new cluster rows: W[C_i, :] = sum_l Qt[i][l] T[C_l, :],  Vt2[C_i, :] = sum_l Qt[i][l] Vt[C_l, :]
__global__ void cluster_rows_kernel(const double *__restrict__ T, const double *__restrict__ Vt,
                                    double *__restrict__ W, double *__restrict__ Vt2,
                                    const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                    const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                                    const double *__restrict__ Qt);

// cluster columns of every row: T[a, C_i] = sum_l R(a)[C_l] Qt[i][l], with
// R(a) = W[a, :] for cluster rows and T[a, :] otherwise; T[C, C] = diag(lam)
__global__ void cluster_cols_kernel(double *__restrict__ T, const double *__restrict__ W,
                                    const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                    const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                                    const int *__restrict__ rowclus, const int *__restrict__ rowbase,
                                    const double *__restrict__ Qt, const double *__restrict__ lam);

// cluster rows outside cluster columns: T[C_i, b] = W[C_i, b]; Vt[C_i, :] = Vt2[C_i, :]
__global__ void cluster_commit_kernel(double *__restrict__ T, const double *__restrict__ W,
                                      double *__restrict__ Vt, const double *__restrict__ Vt2,
                                      const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                      const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                                      const int *__restrict__ rowclus, const int *__restrict__ rowbase);

// M = I - K, K_pq = t_pq / (d_q - d_p) for separable pairs that fail the
// acceptance test or whose step is at most kRefineKappa, 0 otherwise (GEMM tile grid)
__global__ void newton_m_kernel(const double *__restrict__ T, double *__restrict__ M,
                                const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                                const int *__restrict__ bdim, const int *__restrict__ bstate,
                                const double *__restrict__ bnorm, double gap_tol, double abs_tol);

}  // namespace v2b
