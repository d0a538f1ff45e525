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
    double2 *rot;                // rotation record + step counters, offset roff[b]
    const int64_t *roff;
    int max_sweeps;
    double *norm_part;           // kBigCluster doubles per block
    double abs_tol, gap_tol;
    int *counters;               // [0] blocks that hit max_sweeps, [1] rotations
};

// double2 slots of one block's record: sweeps x steps x pairs rotations,
// then sweeps x (steps + 1) int counters
inline int64_t big_record_slots(int n, int max_sweeps) {
    const int np = n + (n & 1), nsteps = np - 1, m = np / 2;
    return (int64_t)max_sweeps * nsteps * m + ((int64_t)max_sweeps * (nsteps + 1) + 3) / 4 + 1;
}

__global__ void jacobi_big_kernel(BigJacobiArgs a);
// the same selective Jacobi with T held in FP32 (T32: a working copy laid
// out like a.T, filled from a.T's symmetric part); the rotations and the
// replay onto Vt stay FP64, P is written from the FP32 result
__global__ void jacobi_big32_kernel(BigJacobiArgs a, float *T32);

}  // namespace v2b
