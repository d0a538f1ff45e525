// Cluster-parallel selective Jacobi for large PSD blocks (see v2b_bigjacobi.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "v2b_device.cuh"

namespace v2b {

constexpr int kBigCluster = 8;    // CTAs per block (portable cluster size)
constexpr int kBigThreads = 512;

struct BigJacobiArgs {
    double *T;                   // V^T U V per block (updated in place)
    double *P;                   // middle factor of U+ (out)
    double *Vt;                  // eigenvector rows (in / out)
    const int64_t *boff;         // matrix offset of each block
    const int *bdim;
    double *diag;                // per-index work arrays, offset ioff[b]
    int *partner;
    int *act;
    double2 *acs;
    const int64_t *ioff;
    int2 *log_pq;                // rotation log, offset loff[b], capacity lcap[b]
    double2 *log_cs;
    const int64_t *loff;
    const int64_t *lcap;
    int *round_cnt;              // max_rounds ints per block
    double *norm_part;           // kBigCluster doubles per block
    int max_rounds;
    double abs_tol, gap_tol;
    int *counters;               // [0] blocks that stopped early, [1] rotations
};

__global__ void jacobi_big_kernel(BigJacobiArgs a);

}  // namespace v2b
