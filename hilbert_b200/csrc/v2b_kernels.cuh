// Kernel declarations and launch parameters for the B200 v2RDM path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "v2b_device.cuh"

namespace v2b {

constexpr int kSpmvThreads = 256;
constexpr int kCgThreads = 512;
constexpr uint32_t kCgLongRow = 32;   // rows with more entries get a whole warp inside CG

// Sliced ELL copy of an operator for the CG kernel (SELL-C-sigma, C = 32):
// rows of at most kCgLongRow entries, sorted by length inside windows of
// kSellSigma rows, in slices of 32 rows stored column-major (entry k of the
// slice's lane l at off[s] + 32 k + l), perm = original row (0xffffffff on
// padding lanes), len = its entry count.  A warp handles a slice: its loads
// are coalesced and independent of one another.
constexpr int kSellSigma = 8192;
struct SellOp {
    const uint32_t *ent, *perm, *off;
    const uint8_t *len;
    int64_t nslices;
    const uint32_t *split;   // CG warp w takes slices split[w] .. split[w + 1] - 1
};
constexpr int kJacobiThreads = 512;
constexpr int kJacobiMaxDim = 160;     // np*np doubles + rotations must fit in 227 KB
constexpr int kStatsBlocks = 256;

struct Palette {
    double v[16];
};

struct CgParams {
    const uint32_t *a_rp, *a_ent;   // A   (rows = dual constraints)
    const uint32_t *t_rp, *t_ent;   // A^T (rows = primal variables)
    const int64_t *long_a, *long_t; // rows longer than kCgLongRow (warp per row)
    int64_t n_long_a, n_long_t;
    SellOp sa, st;                  // the other rows of A and A^T
    Palette palA, palT;
    int64_t np, nd;
    const double *Ax, *Acz, *b;     // rhs = Acz + mu (b - Ax)
    double mu;
    double *y, *r, *p0, *p1, *t;
    double *partials;               // >= 2 * gridDim.x (t.t partials, then r.r partials)
    GridBarrier *bar;
    int *status;
    long long spin_limit;
    double tol;
    int maxit;
    double *out;                    // out[0] = iterations, out[1] = final ||r||
    unsigned long long *phase_ns;   // null, or 4 sums of ns: initial residual, pass 1 (A^T p),
                                    // pass 2 (A t and the update), and a slot left at zero
};

__global__ void spmv_kernel(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ent,
                            int64_t nrows, const double *__restrict__ x, double *__restrict__ y,
                            Palette pal);
__global__ void spmv_A2_kernel(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ent,
                               int64_t nrows, const double *__restrict__ x,
                               const double *__restrict__ c, const double *__restrict__ z,
                               double *__restrict__ Ax, double *__restrict__ Acz, Palette pal);
__global__ void spmv_AT_U_kernel(const uint32_t *__restrict__ rp,
                                 const uint32_t *__restrict__ ent, int64_t nrows,
                                 const double *__restrict__ y, const double *__restrict__ x,
                                 const double *__restrict__ c, double mu,
                                 double *__restrict__ ATy, double *__restrict__ U, Palette pal);
__global__ void cg_kernel(CgParams P);
// the CG starting point of the next outer iteration from the last dual
// solutions (order 0: y itself, 1: 2y - y1, 2: 3y - 3y1 + y2); y1, y2 shift
__global__ void extrapolate_y_kernel(double *__restrict__ y, double *__restrict__ y1,
                                     double *__restrict__ y2, int64_t n, int order);
__global__ void stats_kernel(const double *__restrict__ Ax, const double *__restrict__ b,
                             const double *__restrict__ ATy, const double *__restrict__ z,
                             const double *__restrict__ c, const double *__restrict__ x,
                             const double *__restrict__ y, int64_t np, int64_t nd,
                             double *__restrict__ partials, unsigned int *counter,
                             double *__restrict__ out, int *status);
__global__ void jacobi_warm_kernel(const double *__restrict__ T0, double *__restrict__ Pout,
                                   double *__restrict__ Vt, const int64_t *__restrict__ boff,
                                   const int *__restrict__ bdim, double2 *__restrict__ rot,
                                   const int64_t *__restrict__ rot_off, int max_sweeps,
                                   double abs_tol, double gap_tol, int *status, int *rot_count,
                                   int raw = 0);
__global__ void identity_blocks_kernel(double *__restrict__ Vt, const int64_t *__restrict__ boff,
                                       const int *__restrict__ bdim);
__global__ void half_residual_kernel(const double *__restrict__ G, double *__restrict__ H,
                                     const int64_t *__restrict__ boff, const int *__restrict__ bdim);

// Raise func's dynamic shared-memory limit on the current device to at least
// bytes, under one process-wide lock; never lowers it, because several
// problems (and the allocation-free entry point) share the attribute.
cudaError_t raise_dynamic_smem(const void *func, int bytes);
// Unique id of the current CUDA context, 0 when there is none.  A new
// context (after cudaDeviceReset) gets a new id, so per-device caches of
// symbol addresses and function attributes can tell that they are stale.
unsigned long long current_context_id();

inline size_t jacobi_smem_bytes(int n) {
    const int np = n + (n & 1);
    return (size_t)np * np * sizeof(double) + (size_t)(np / 2) * (sizeof(double2) + 2 * sizeof(int));
}

}  // namespace v2b
