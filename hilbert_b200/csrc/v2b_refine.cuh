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
constexpr int kStBlockJacobi = 3;   // block-Jacobi sweeps over pairs of row groups
constexpr int kStFp32 = 4;     // mixed mode: an FP32 eigensolve, then FP64 Rayleigh-Ritz + Newton

constexpr int kBJGroup = 32;           // rows per block-Jacobi group (pairs: 64-row subproblems)
constexpr int kBJMaxSweeps = 24;
constexpr int kBJInnerSweeps = 2;      // Jacobi sweeps per 64-row subproblem and step
constexpr int kClusterSweeps = 40;     // cap of the exact cluster diagonalisation

constexpr int kRefineSmallCluster = 64;  // clusters up to this size: cluster_eig_kernel
constexpr int kRefineEdgeCap = 32768;    // non-separable pairs recorded per block and pass
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

constexpr int kClassifySplit = 16;   // CTAs per block in the acceptance test

// Frobenius norms of the symmetrised blocks as kClassifySplit partial sums each
__global__ void block_norm_kernel(const double *__restrict__ Us, const int64_t *__restrict__ boff,
                                  const int *__restrict__ bdim, double *__restrict__ part);
// acceptance test and pair classification (grid nblk x kClassifySplit)
__global__ void refine_classify_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                                       const int *__restrict__ bdim, int *__restrict__ bstate,
                                       const unsigned long long *__restrict__ orth,
                                       const double *__restrict__ part, double gap_tol, double abs_tol,
                                       double *__restrict__ bnorm, int *__restrict__ counts,
                                       int *__restrict__ done_stamp, int stamp, int *h_state,
                                       int *h_nbad, int *h_nedge, int2 *h_edges);
// P = Gamma o T for the blocks accepted under this stamp (GEMM tile grid)
__global__ void write_p_kernel(const double *__restrict__ T, double *__restrict__ P,
                               const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                               const int *__restrict__ bdim, const int *__restrict__ done_stamp,
                               int stamp);

// cyclic Jacobi on each cluster's T[C, C] (at most max_sweeps sweeps; enough
// sweeps diagonalise it exactly): rows of Qt (k x k) are the eigenvectors,
// lam the diagonal left
__global__ void cluster_eig_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                                   const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                                   const int *__restrict__ mem, double *__restrict__ Qt,
                                   double *__restrict__ lam, const int *__restrict__ only,
                                   int max_sweeps);

// gathered GEMM tiles of the cluster transform; ctiles = (job, tile row, tile col).
// With `only` non-null, jobs of blocks b with only[b] == 0 are skipped.
__global__ void cluster_rows_kernel(const double *__restrict__ T, const double *__restrict__ Vt,
                                    double *__restrict__ W, double *__restrict__ Vt2,
                                    const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                    const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                                    const double *__restrict__ Qt, const int4 *__restrict__ ctiles,
                                    const int *__restrict__ only);
__global__ void cluster_cols_kernel(const double *__restrict__ T, const double *__restrict__ W,
                                    double *__restrict__ P, const int64_t *__restrict__ boff,
                                    const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                                    const int *__restrict__ mem, const int *__restrict__ rowclus,
                                    const int *__restrict__ rowbase, const double *__restrict__ Qt,
                                    const double *__restrict__ lam, const int4 *__restrict__ ctiles,
                                    const int *__restrict__ only);
__global__ void cluster_commit_kernel(double *__restrict__ T, const double *__restrict__ W,
                                      const double *__restrict__ P, double *__restrict__ Vt,
                                      const double *__restrict__ Vt2, const int64_t *__restrict__ boff,
                                      const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                                      const int *__restrict__ mem, const int *__restrict__ rowclus,
                                      const int *__restrict__ rowbase, const int4 *__restrict__ ctiles,
                                      const int *__restrict__ only);
// one block-Jacobi step in place: tiles (I, J, 0) T[C_I, C_J] <- Qt_I T Qt_J^T,
// (I, t, 1) Vt[C_I, 64 t ..] <- Qt_I Vt[C_I, ..]; dynamic shared memory
// 3 x 64 x 65 doubles
__global__ void bj_apply_kernel(double *__restrict__ T, double *__restrict__ Vt,
                                const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                                const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                                const double *__restrict__ Qt, const int4 *__restrict__ tiles,
                                const int *__restrict__ only);
// compact sym(T[C, C]) and identity for the clusters in jlist
__global__ void cluster_gather_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                                      const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                                      const int *__restrict__ mem, const int *__restrict__ jlist,
                                      double *__restrict__ Tc, double *__restrict__ Vc);
// eigenvalues of Jacobi-diagonalised clusters: jlist[0 .. big_from) read Dsmall, the rest Dbig
__global__ void cluster_lam_kernel(const ClusterJob *__restrict__ jobs, const int *__restrict__ jlist,
                                   int njobs, const double *__restrict__ Dsmall,
                                   const double *__restrict__ Dbig, int big_from,
                                   double *__restrict__ lam);

// M = I - K, K_pq = t_pq / (d_q - d_p) for separable pairs that fail the
// acceptance test or whose step is at most kRefineKappa, 0 otherwise (GEMM tile grid)
__global__ void newton_m_kernel(const double *__restrict__ T, double *__restrict__ M,
                                const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                                const int *__restrict__ bdim, const int *__restrict__ bstate,
                                const double *__restrict__ bnorm, double gap_tol, double abs_tol);

}  // namespace v2b
