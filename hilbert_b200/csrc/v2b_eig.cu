// Warm-started PSD projection of the BPSDP blocks (sm_100a, FP64).
//
// Between outer iterations U = mu x + A^T y - c changes little, so the
// previous eigenvectors V are an excellent basis.  Each iteration refines V
// by one Newton step for the symmetric eigenproblem (Ogita & Aishima,
// "Iterative refinement for symmetric eigenvalue problems", Japan J. Indust.
// Appl. Math. 35, 1007 (2018)) and then projects in the refined basis:
//
//   round 1:  W = U V0,  S = V0^T W,  G = V0^T V0,  R = I - G
//             lam_i = S_ii / G_ii,  delta = 2 (||S - diag(lam)||_F + ||S||_F ||R||_F)
//             E_ij = (S_ij + lam_j R_ij) / (lam_j - lam_i)   if |lam_j - lam_i| > delta
//                  = R_ij / 2                                 otherwise (and i = j)
//             V1 = V0 + V0 E
//   round 2:  S, G, R for V1; M = S + (R o (lam_i + lam_j)/2)  (basis re-orthonormalised
//             to first order), M+ from the first-order (Daleckii-Krein) formula
//             M+_ij = Gamma_ij M_ij, Gamma_ij = (m_i+ - m_j+) / (m_i - m_j),
//             P = M+ + R o (m_i+ + m_j+)/2,   U+ = V1 P V1^T,   x = U+/mu,  z = U+ - U.
//
// All n^3 work is batched GEMM tiles over every block of the problem
// (gemm_tiles_kernel); the elementwise steps run one CTA per block
// (refine_kernel).  Round 2 estimates the relative error of U+ it leaves,
//   max over pairs straddling zero of corr_ij^2 |lam_i - lam_j| / ||U||_F + max |R_ij|^2,
// and flags the block when it exceeds the tolerance; the caller then repeats
// the warm step from the refined basis (one more Newton round) and falls back
// to the Jacobi kernel if that is still not enough.
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
                      double *__restrict__ xo, double *__restrict__ zo) {
    constexpr int BM = 64, BK = 16;
    __shared__ double As[BK][BM + 2];
    __shared__ double Bs[BK][BM + 2];
    const int4 t = tiles[blockIdx.x];
    const int blk = t.x, n = bdim[blk];
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
            } else {   // kEpiProject: acc = U+
                xo[e] = acc[i][j] * inv_mu;
                zo[e] = acc[i][j] - Us[e];
            }
        }
    }
}

template __global__ void gemm_tiles_kernel<false, false, kEpiStore>(GEMM_ARGS);
template __global__ void gemm_tiles_kernel<true, false, kEpiStore>(GEMM_ARGS);
template __global__ void gemm_tiles_kernel<false, false, kEpiAdd>(GEMM_ARGS);
template __global__ void gemm_tiles_kernel<false, true, kEpiProject>(GEMM_ARGS);

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

// ---------------------------------------------------------------------------
// One CTA per block.  mode 0: Newton correction E (written to Eo).
// mode 1: projected middle factor P (written to Eo) for U+ = V P V^T, and the
// size of the correction that was not applied (block flagged when large).
__global__ void __launch_bounds__(kRefineThreads)
    refine_kernel(const double *__restrict__ S, const double *__restrict__ G,
                  double *__restrict__ Eo, double *__restrict__ lam_buf,
                  const int64_t *__restrict__ loff, const int64_t *__restrict__ boff,
                  const int *__restrict__ bdim, int mode, double flag_tol,
                  int *__restrict__ flags) {
    const int blk = blockIdx.x, n = bdim[blk];
    if (n <= 0) return;
    const int64_t off = boff[blk];
    double *lam = lam_buf + loff[blk];
    __shared__ double red[32];
    __shared__ double s_delta, s_max;
    // lam_i = S_ii / G_ii
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        lam[i] = S[off + (int64_t)i * n + i] / G[off + (int64_t)i * n + i];
    __syncthreads();
    double off2 = 0.0, r2 = 0.0, s2 = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        const double s = 0.5 * (S[off + e] + S[off + (int64_t)j * n + i]);
        const double r = (i == j ? 1.0 : 0.0) - G[off + e];
        const double d = (i == j) ? s - lam[i] : s;
        off2 += d * d;
        r2 += r * r;
        s2 += s * s;
    }
    off2 = block_sum(off2, red);
    r2 = block_sum(r2, red);
    s2 = block_sum(s2, red);
    if (threadIdx.x == 0) {
        s_delta = 2.0 * (sqrt(off2) + sqrt(s2) * sqrt(r2));
        s_max = 0.0;
    }
    __syncthreads();
    const double delta = s_delta;
    double m_straddle = 0.0, m_orth = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        const double s = 0.5 * (S[off + e] + S[off + (int64_t)j * n + i]);
        const double r = (i == j ? 1.0 : 0.0) - G[off + e];
        const double li = lam[i], lj = lam[j];
        double corr;
        if (i != j && fabs(lj - li) > delta) corr = (s + lj * r) / (lj - li);
        else corr = 0.5 * r;
        if (mode == 0) {
            Eo[off + e] = corr;
        } else {
            // second-order error of leaving (i, j) unresolved matters only when
            // the pair straddles zero; non-orthonormality enters squared
            if (li * lj < 0.0) m_straddle = fmax(m_straddle, corr * corr * fabs(lj - li));
            m_orth = fmax(m_orth, fabs(r));
            // middle factor in an orthonormal basis, to first order in R
            const double m = (i == j) ? li : s + r * 0.5 * (li + lj);
            const double pi = fmax(li, 0.0), pj = fmax(lj, 0.0);
            double p;
            if (i == j) {
                p = pi + r * pi;
            } else {
                double gam;
                if (li != lj) gam = (pi - pj) / (li - lj);
                else gam = li > 0.0 ? 1.0 : 0.0;
                p = gam * m + r * 0.5 * (pi + pj);
            }
            Eo[off + e] = p;
        }
    }
    if (mode == 1) {
        m_straddle = block_max(m_straddle, red);
        m_orth = block_max(m_orth, red);
        if (threadIdx.x == 0) {
            const double est = m_straddle / fmax(sqrt(s2), 1e-300) + m_orth * m_orth;
            if (!(est <= flag_tol)) flags[blk] = 1;
        }
    }
}

}  // namespace v2b
