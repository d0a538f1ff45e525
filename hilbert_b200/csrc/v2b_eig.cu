// Batched FP64 GEMM tiles for the warm-started PSD projection (sm_100a).
//
// Between outer iterations U = mu x + A^T y - c changes little, so the
// eigenvectors of the previous iteration (rows of Vt) nearly diagonalise the
// new block: per iteration
//   W  = sym(U) Vt^T          gemm<N,T>
//   T0 = Vt W                 gemm<N,N>      (= V^T U V, nearly diagonal)
//   selective Jacobi on T0    jacobi_warm_kernel (shared memory, one CTA per block)
//   Y  = Vt^T P               gemm<T,N>
//   U+ = Y Vt                 gemm<N,N> with the projection epilogue
//                             x = U+ / mu,  z = U+ - sym(U)
// Every gemm launch covers all blocks of the problem: the grid is the list of
// 64 x 64 output tiles of every block.
#include "v2b_eig.cuh"

namespace v2b {

// ---------------------------------------------------------------------------
// batched FP64 GEMM over square blocks: C_b = op(A_b) op(B_b) [+ epilogue]
// 64 x 64 output tile per CTA, 256 threads, 4 x 4 outputs per thread, K in
// chunks of 16 staged through shared memory.
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256)
    gemm_tiles_kernel(const double *__restrict__ A, const double *__restrict__ B,
                      double *__restrict__ C, const int4 *__restrict__ tiles,
                      const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                      const double *__restrict__ Cin, const double *__restrict__ Us, double inv_mu,
                      double *__restrict__ xo, double *__restrict__ zo,
                      const int *__restrict__ bstate, unsigned long long *__restrict__ orth) {
    constexpr int BM = 64, BK = 16;
    __shared__ double As[BK][BM + 2];
    __shared__ double Bs[BK][BM + 2];
    const int4 t = tiles[blockIdx.x];
    const int blk = t.x, n = bdim[blk];
    if (bstate && bstate[blk] != 0) return;   // uniform over the CTA
    const int64_t off = boff[blk];
    const int r0 = t.y * BM, c0 = t.z * BM;
    const double *Ab = A + off, *Bb = B + off;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;

    for (int k0 = 0; k0 < n; k0 += BK) {
        // op(A)[r][k] for r in [r0, r0+64), k in [k0, k0+16)
        for (int e = threadIdx.x; e < BM * BK; e += 256) {
            int rr, kk;
            if (TA) { kk = e / BM; rr = e % BM; }   // A[k][r]: contiguous in r
            else { rr = e / BK; kk = e % BK; }      // A[r][k]: contiguous in k
            const int r = r0 + rr, k = k0 + kk;
            double v = 0.0;
            if (r < n && k < n) v = TA ? Ab[(int64_t)k * n + r] : Ab[(int64_t)r * n + k];
            As[kk][rr] = v;
        }
        // op(B)[k][c] for k in [k0, k0+16), c in [c0, c0+64)
        for (int e = threadIdx.x; e < BM * BK; e += 256) {
            int cc, kk;
            if (TB) { cc = e / BK; kk = e % BK; }   // B[c][k]: contiguous in k
            else { kk = e / BM; cc = e % BM; }      // B[k][c]: contiguous in c
            const int c = c0 + cc, k = k0 + kk;
            double v = 0.0;
            if (c < n && k < n) v = TB ? Bb[(int64_t)c * n + k] : Bb[(int64_t)k * n + c];
            Bs[kk][cc] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    double dev = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = r0 + ty * 4 + i;
        if (r >= n) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = c0 + tx * 4 + j;
            if (c >= n) continue;
            const int64_t e = off + (int64_t)r * n + c;
            if (EPI == kEpiStore) {
                C[e] = acc[i][j];
            } else if (EPI == kEpiAdd) {
                C[e] = Cin[e] + acc[i][j];
            } else if (EPI == kEpiNS) {   // acc = Vt Vt^T
                const double id = (r == c) ? 1.0 : 0.0;
                C[e] = 1.5 * id - 0.5 * acc[i][j];
                dev = fmax(dev, fabs(acc[i][j] - id));
            } else {   // kEpiProject: acc = U+
                xo[e] = acc[i][j] * inv_mu;
                zo[e] = acc[i][j] - Us[e];
            }
        }
    }
    if (EPI == kEpiNS) {
        // non-negative doubles order like their bit patterns
        dev = warp_max(dev);
        if ((threadIdx.x & 31) == 0 && dev > 0.0)
            atomicMax(orth + blk, (unsigned long long)__double_as_longlong(dev));
    }
}

cudaError_t launch_gemm_tiles(GemmVariant v, int ntiles, cudaStream_t s, GEMM_ARGS) {
    if (ntiles <= 0) return cudaSuccess;
    switch (v) {
        case kGemmNTNewtonSchulz:
            gemm_tiles_kernel<false, true, kEpiNS><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
        case kGemmNTStore:
            gemm_tiles_kernel<false, true, kEpiStore><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
        case kGemmNNStore:
            gemm_tiles_kernel<false, false, kEpiStore><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
        case kGemmTNStore:
            gemm_tiles_kernel<true, false, kEpiStore><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
        case kGemmNNProject:
            gemm_tiles_kernel<false, false, kEpiProject><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
        case kGemmNNAdd:
            gemm_tiles_kernel<false, false, kEpiAdd><<<ntiles, 256, 0, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth);
            break;
    }
    return cudaGetLastError();
}

// Us = (U + U^T) / 2 per block, tile by tile
__global__ void symmetrize_kernel(const double *__restrict__ U, double *__restrict__ Us,
                                  const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                                  const int *__restrict__ bdim) {
    const int4 t = tiles[blockIdx.x];
    const int n = bdim[t.x];
    const int64_t off = boff[t.x];
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int r = t.y * 64 + e / 64, c = t.z * 64 + e % 64;
        if (r < n && c < n)
            Us[off + (int64_t)r * n + c] = 0.5 * (U[off + (int64_t)r * n + c] + U[off + (int64_t)c * n + r]);
    }
}

}  // namespace v2b
