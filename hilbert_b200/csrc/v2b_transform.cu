// focas's density-fitted integral transform and its adjoint on FP64 tensor
// cores (sm_100a).
//
// focas rotates the orbitals of the three-index integrals one auxiliary
// index at a time (OrbitalOptimizer::TransformTei_Q,
// src/focas/C_files/orbopt_integraltransform_cpu.cc:235-261: two DGEMMs per
// Q, scr2 = B_Q U, then B'_Q = U^T scr2), and the one-electron integrals the
// same way (TransformOei, :263-285).  Here one CTA owns one matrix: U and B_Q
// are staged in shared memory, both products run as m8n8k4 FP64 MMAs
// (mma.sync .f64, the tensor-core path for FP64 on sm_100a; tcgen05 has no
// FP64 kind) and B'_Q goes back to global memory.  The adjoint gives the
// U-gradient of E = sum_Q <M_Q, U^T B_Q U> for given M_Q = dE/dB'_Q:
//   dE/dU = sum_Q (B_Q U M_Q^T + B_Q^T U M_Q),
// one CTA per Q into a per-Q slab, then a fixed-order sum over Q
// (deterministic, no atomics).
//
// Matrices are n x n, row-major, n <= kTransformMaxDim; in shared memory they
// are zero-padded to a multiple of 8 with a row stride of that plus one
// double (the fragment reads of a warp then fall on distinct banks).
#include "v2b_transform.cuh"

#include <algorithm>

#include "v2b_kernels.cuh"

namespace v2b {

namespace {

constexpr int kTransformThreads = 256;

__device__ __forceinline__ void dmma8x8x4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

struct Pad {
    int n, m, ld;   // dimension, padded dimension (multiple of 8), row stride
    __device__ Pad(int n_) : n(n_), m((n_ + 7) & ~7), ld(((n_ + 7) & ~7) + 1) {}
};

// global n x n (row-major) -> shared, zero-padded
__device__ __forceinline__ void stage(double *s, const double *__restrict__ g, const Pad &P) {
    for (int e = threadIdx.x; e < P.m * P.m; e += blockDim.x) {
        const int r = e / P.m, c = e % P.m;
        s[r * P.ld + c] = (r < P.n && c < P.n) ? g[(int64_t)r * P.n + c] : 0.0;
    }
}

// element (r, c) of op(X) for a shared matrix X
template <bool T>
__device__ __forceinline__ double at(const double *X, int r, int c, int ld) {
    return T ? X[c * ld + r] : X[r * ld + c];
}

// the 8 x 8 tile (tr, tc) of op(A) op(B) added into (d0, d1), all of K = P.m
template <bool TA, bool TB>
__device__ __forceinline__ void tile_mma(const double *A, const double *B, int tr, int tc, const Pad &P,
                                         double &d0, double &d1) {
    const int lane = threadIdx.x & 31;
    const int fr = lane >> 2, fk = lane & 3;
    for (int k0 = 0; k0 < P.m; k0 += 4) {
        const double a = at<TA>(A, tr * 8 + fr, k0 + fk, P.ld);
        const double b = at<TB>(B, k0 + fk, tc * 8 + fr, P.ld);
        dmma8x8x4(d0, d1, a, b);
    }
}

// C = op(A) op(B) into shared C (tiles spread over the warps)
template <bool TA, bool TB>
__device__ void smem_gemm(const double *A, const double *B, double *C, const Pad &P) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nt = P.m / 8;
    for (int t = warp; t < nt * nt; t += nw) {
        const int tr = t / nt, tc = t % nt;
        double d0 = 0.0, d1 = 0.0;
        tile_mma<TA, TB>(A, B, tr, tc, P, d0, d1);
        const int r = tr * 8 + (lane >> 2), c = tc * 8 + 2 * (lane & 3);
        C[r * P.ld + c] = d0;
        C[r * P.ld + c + 1] = d1;
    }
}

__global__ void __launch_bounds__(kTransformThreads)
    df_transform_kernel(const double *__restrict__ U, const double *__restrict__ B, double *__restrict__ Bp,
                        int n) {
    extern __shared__ double sm[];
    const Pad P(n);
    const int sz = P.m * P.ld;
    double *sU = sm, *sB = sm + sz, *sW = sm + 2 * sz;
    const int64_t q = blockIdx.x;
    stage(sU, U, P);
    stage(sB, B + q * n * n, P);
    __syncthreads();
    smem_gemm<false, false>(sB, sU, sW, P);   // W = B_Q U
    __syncthreads();
    // B'_Q = U^T W, straight from the fragments to global memory
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nt = P.m / 8;
    double *out = Bp + q * n * n;
    for (int t = warp; t < nt * nt; t += nw) {
        const int tr = t / nt, tc = t % nt;
        double d0 = 0.0, d1 = 0.0;
        tile_mma<true, false>(sU, sW, tr, tc, P, d0, d1);
        const int r = tr * 8 + (lane >> 2), c = tc * 8 + 2 * (lane & 3);
        if (r < n && c < n) out[(int64_t)r * n + c] = d0;
        if (r < n && c + 1 < n) out[(int64_t)r * n + c + 1] = d1;
    }
}

// slab_Q = B_Q U M_Q^T + B_Q^T U M_Q; the output tiles stay in registers
// while the shared buffer changes from X = B_Q U to Y = B_Q^T U
__global__ void __launch_bounds__(kTransformThreads)
    df_transform_adjoint_kernel(const double *__restrict__ U, const double *__restrict__ B,
                                const double *__restrict__ M, double *__restrict__ slab, int n) {
    extern __shared__ double sm[];
    const Pad P(n);
    const int sz = P.m * P.ld;
    double *sU = sm, *sB = sm + sz, *sM = sm + 2 * sz, *sX = sm + 3 * sz;
    const int64_t q = blockIdx.x;
    stage(sU, U, P);
    stage(sB, B + q * n * n, P);
    stage(sM, M + q * n * n, P);
    __syncthreads();
    smem_gemm<false, false>(sB, sU, sX, P);   // X = B_Q U
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nt = P.m / 8;
    constexpr int kWarps = kTransformThreads / 32;
    constexpr int kMaxTilesPerWarp = ((kTransformMaxDim / 8) * (kTransformMaxDim / 8) + kWarps - 1) / kWarps;
    double acc[kMaxTilesPerWarp][2];
#pragma unroll
    for (int i = 0; i < kMaxTilesPerWarp; i++) acc[i][0] = acc[i][1] = 0.0;
#pragma unroll
    for (int i = 0; i < kMaxTilesPerWarp; i++) {
        const int t = warp + i * nw;
        if (t < nt * nt) tile_mma<false, true>(sX, sM, t / nt, t % nt, P, acc[i][0], acc[i][1]);   // X M^T
    }
    __syncthreads();
    smem_gemm<true, false>(sB, sU, sX, P);    // Y = B_Q^T U
    __syncthreads();
    double *out = slab + q * n * n;
#pragma unroll
    for (int i = 0; i < kMaxTilesPerWarp; i++) {
        const int t = warp + i * nw;
        if (t < nt * nt) {
            const int tr = t / nt, tc = t % nt;
            tile_mma<false, false>(sX, sM, tr, tc, P, acc[i][0], acc[i][1]);   // + Y M
            const int r = tr * 8 + (lane >> 2), c = tc * 8 + 2 * (lane & 3);
            if (r < n && c < n) out[(int64_t)r * n + c] = acc[i][0];
            if (r < n && c + 1 < n) out[(int64_t)r * n + c + 1] = acc[i][1];
        }
    }
}

// dU[e] = sum over Q of slab_Q[e], Q in order
__global__ void sum_slabs_kernel(const double *__restrict__ slab, double *__restrict__ dU, int64_t nn,
                                 int count) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < count; q++) s += slab[(int64_t)q * nn + e];
        dU[e] = s;
    }
}

size_t transform_smem(int n, int mats) {
    const int m = (n + 7) & ~7;
    return (size_t)mats * m * (m + 1) * sizeof(double);
}

}  // namespace

cudaError_t launch_df_transform(const double *U, const double *B, double *Bp, int n, int count,
                                cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const size_t smem = transform_smem(n, 3);
    cudaError_t e = raise_dynamic_smem((const void *)df_transform_kernel, (int)smem);
    if (e != cudaSuccess) return e;
    df_transform_kernel<<<count, kTransformThreads, smem, s>>>(U, B, Bp, n);
    return cudaGetLastError();
}

cudaError_t launch_df_transform_adjoint(const double *U, const double *B, const double *M, double *dU,
                                        double *slab, int n, int count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const size_t smem = transform_smem(n, 4);
    cudaError_t e = raise_dynamic_smem((const void *)df_transform_adjoint_kernel, (int)smem);
    if (e != cudaSuccess) return e;
    df_transform_adjoint_kernel<<<count, kTransformThreads, smem, s>>>(U, B, M, slab, n);
    const int64_t nn = (int64_t)n * n;
    sum_slabs_kernel<<<(int)std::min<int64_t>((nn + 255) / 256, 1024), 256, 0, s>>>(slab, dU, nn, count);
    return cudaGetLastError();
}

}  // namespace v2b

// --------------------------------------------------------------- C ABI
#include <string>

#include "v2b_eig.cuh"
#include "v2rdm_b200.h"

namespace {

int transform_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return V2B_OK;
    v2b::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return V2B_CUDA_ERROR;
}

int transform_args(const void *a, const void *b, const void *c, int n, int count, const char *what) {
    if (!a || !b || !c || n < 1 || count < 0) {
        v2b::set_last_error(std::string(what) + ": NULL pointer or bad size");
        return V2B_BAD_ARG;
    }
    if (n > v2b::kTransformMaxDim) {
        v2b::set_last_error(std::string(what) + ": " + std::to_string(n) + " orbitals, at most " +
                            std::to_string(v2b::kTransformMaxDim));
        return V2B_BAD_ARG;
    }
    return V2B_OK;
}

}  // namespace

extern "C" int v2b_df_transform(const double *d_U, const double *d_B, double *d_Bp, int n, int count,
                                void *stream) {
    const int rc = transform_args(d_U, d_B, d_Bp, n, count, "df_transform");
    if (rc != V2B_OK) return rc;
    return transform_status(v2b::launch_df_transform(d_U, d_B, d_Bp, n, count, (cudaStream_t)stream),
                            "df_transform");
}

extern "C" int v2b_df_transform_adjoint(const double *d_U, const double *d_B, const double *d_M, double *d_dU,
                                        double *d_work, int n, int count, void *stream) {
    int rc = transform_args(d_U, d_B, d_M, n, count, "df_transform_adjoint");
    if (rc == V2B_OK && (!d_dU || !d_work)) {
        v2b::set_last_error("df_transform_adjoint: NULL pointer");
        rc = V2B_BAD_ARG;
    }
    if (rc != V2B_OK) return rc;
    return transform_status(
        v2b::launch_df_transform_adjoint(d_U, d_B, d_M, d_dU, d_work, n, count, (cudaStream_t)stream),
        "df_transform_adjoint");
}
