// Device building blocks for the B200 v2RDM path (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace v2b {

constexpr uint32_t kDevColMask = (1u << 27) - 1u;
constexpr int kStatusTimeout = 4;   // V2B_DEVICE_TIMEOUT
constexpr int kStatusNan = 3;       // V2B_NAN

// One packed sparse row: sum of coef * x[col] in stored order, with separate
// multiply and add roundings (no FMA contraction), so that the result equals
// hilbert's own left-to-right accumulation.  Entries flagged with bit 31 are
// summed into a second partial that is added at the end (rows the reference
// assembles as "(D2 - Q2) + (sum of delta terms)", q2.cc:218-318).
__device__ __forceinline__ double packed_row(const uint32_t *__restrict__ ent, uint32_t b,
                                             uint32_t e, const double *__restrict__ x,
                                             const double *pal) {
    double acc0 = 0.0, acc1 = 0.0;
    bool grp = false;
#pragma unroll 4
    for (uint32_t k = b; k < e; k++) {
        const uint32_t w = __ldg(ent + k);
        const double v = __dmul_rn(pal[(w >> 27) & 15u], __ldg(x + (w & kDevColMask)));
        grp = grp || (w >> 31);
        if (grp) acc1 = __dadd_rn(acc1, v);
        else acc0 = __dadd_rn(acc0, v);
    }
    return grp ? __dadd_rn(acc0, acc1) : acc0;
}

// Same row applied to (r + beta * p) without materialising it: each operand is
// formed as __dadd_rn(r, __dmul_rn(beta, p)), identical to the stored update.
__device__ __forceinline__ double packed_row_rbp(const uint32_t *__restrict__ ent, uint32_t b,
                                                 uint32_t e, const double *__restrict__ r,
                                                 const double *__restrict__ p, double beta,
                                                 const double *pal) {
    double acc0 = 0.0, acc1 = 0.0;
    bool grp = false;
#pragma unroll 4
    for (uint32_t k = b; k < e; k++) {
        const uint32_t w = __ldg(ent + k);
        const uint32_t c = w & kDevColMask;
        const double xv = __dadd_rn(__ldg(r + c), __dmul_rn(beta, __ldg(p + c)));
        const double v = __dmul_rn(pal[(w >> 27) & 15u], xv);
        grp = grp || (w >> 31);
        if (grp) acc1 = __dadd_rn(acc1, v);
        else acc0 = __dadd_rn(acc0, v);
    }
    return grp ? __dadd_rn(acc0, acc1) : acc0;
}

// the GPU's nanosecond clock (PTX %globaltimer)
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block reduction (fixed tree); result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *red /* >= 32 */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block max; result valid in thread 0.
__device__ __forceinline__ double block_max(double v, double *red /* >= 32 */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? red[lane] : 0.0;
        s = warp_max(s);
    }
    return s;
}

// Deterministic sum of n partials, every thread of the block gets the result.
// Called right after a grid barrier (whose acquire orders these loads); the
// loads bypass L1 (__ldcg) and are independent, so they pipeline.
__device__ __forceinline__ double sum_partials(const double *part, int n, double *bcast) {
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += 32) s += __ldcg(part + i);
        s = warp_sum(s);
        if (threadIdx.x == 0) *bcast = s;
    }
    __syncthreads();
    const double r = *bcast;
    __syncthreads();
    return r;
}

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int *p) {
    return *((volatile const unsigned int *)p);
}
__device__ __forceinline__ int ld_volatile_i32(const int *p) { return *((volatile const int *)p); }
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid-wide barrier for a cooperatively launched kernel.  Every wait is
// bounded: after spin_limit polls the waiting block records
// kStatusTimeout in *status and all blocks leave at their next barrier.
// Returns false when the kernel must stop (timeout or an error status).
__device__ __forceinline__ bool grid_sync(GridBarrier *bar, int *status, long long spin_limit,
                                          int *s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int fail = 0;
        const unsigned int g = ld_acquire_u32(&bar->gen);
        const unsigned int arrived = atom_add_acq_rel_u32(&bar->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&bar->count, 0u);
            atom_add_acq_rel_u32(&bar->gen, 1u);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(&bar->gen) == g) {
                if ((spins & 63) == 0 && ld_volatile_i32(status) != 0) { fail = 1; break; }
                if (++spins > spin_limit) {
                    atomicExch(status, kStatusTimeout);
                    fail = 1;
                    break;
                }
                if (spins > 256) __nanosleep(32);
            }
        }
        *s_flag = fail || (ld_volatile_i32(status) != 0);
    }
    __syncthreads();
    return *s_flag == 0;
}

// Round-robin ("circle method") pairing of np (even) indices: in step s the
// fixed index np-1 meets s and, for k >= 1, (s+k) meets (s-k) mod (np-1).
__device__ __forceinline__ void rr_pair(int s, int k, int np, int &p, int &q) {
    const int m1 = np - 1;
    int a, b;
    if (k == 0) {
        a = m1;
        b = s;
    } else {
        a = (s + k) % m1;
        b = (s - k + m1) % m1;
    }
    p = a < b ? a : b;
    q = a < b ? b : a;
}

}  // namespace v2b
