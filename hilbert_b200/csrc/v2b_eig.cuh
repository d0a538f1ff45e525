// Batched GEMM tiles of the warm-started PSD projection (see v2b_eig.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "v2b_device.cuh"

namespace v2b {

constexpr int kEpiStore = 0;     // C = op(A) op(B)
constexpr int kEpiAdd = 1;       // C = Cin + op(A) op(B)
constexpr int kEpiProject = 2;   // x = (op(A) op(B)) / mu, z = op(A) op(B) - Us
constexpr int kEpiNS = 3;        // C = 3/2 I - 1/2 op(A) op(B); orth[b] = max |op(A) op(B) - I|
constexpr int kGemmTile = 64;
constexpr int kGemmMaxSplit = 4;   // K parts of one output tile at most

#define GEMM_ARGS                                                                           \
    const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C,     \
        const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,                    \
        const int *__restrict__ bdim, const double *__restrict__ Cin,                        \
        const double *__restrict__ Us, double inv_mu, double *__restrict__ xo,               \
        double *__restrict__ zo, const int *__restrict__ bstate,                             \
        unsigned long long *__restrict__ orth

// Host launcher of gemm_tiles_kernel<TA, TB, EPI> (defined, with the kernel
// instantiations, in v2b_eig.cu).  variant: 0 <N,T,store>, 1 <N,N,store>,
// 2 <T,N,store>, 3 <N,N,project>, 4 <N,N,add>, 5 <N,T,Newton-Schulz>.
// With bstate non-null, tiles of blocks whose state is not 0 (refinement in
// progress) are skipped.  sched: two ints, zero before the first launch, that
// make the grid persistent (tiles taken in list order; the kernel leaves them
// zero again); null launches one CTA per tile.  Launches that share a sched
// pair must be ordered (one stream).  Tiles split along K (tile word bits
// 8-11 above 1) need split_ws (kGemmMaxSplit x 64 x 64 doubles per group) and split_cnt
// (one int per group, zero before the first launch, left zero).
enum GemmVariant { kGemmNTStore = 0, kGemmNNStore = 1, kGemmTNStore = 2, kGemmNNProject = 3,
                   kGemmNNAdd = 4, kGemmNTNewtonSchulz = 5 };
cudaError_t launch_gemm_tiles(GemmVariant v, int ntiles, cudaStream_t s, GEMM_ARGS,
                              int *sched = nullptr, double *split_ws = nullptr, int *split_cnt = nullptr);
// CTA slots of the persistent GEMM grid on the current device (SMs x
// resident CTAs)
cudaError_t gemm_slots(int *slots);

}  // namespace v2b

#include <string>
namespace v2b {
// message returned by v2b_last_error() on the calling thread
void set_last_error(const std::string &msg);

__global__ void symmetrize_kernel(const double *__restrict__ U, double *__restrict__ Us,
                                  const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                                  const int *__restrict__ bdim);

}  // namespace v2b
