// Warm eigen-refinement of the per-block PSD projection (sm_100a).
//
// The projection needs U+ = V f(L) V^T with f(l) = max(l, 0).  The rows of
// Vt from the previous outer iteration nearly diagonalise the new block, so
// T = Vt U Vt^T = D + E with E small, and to first order
//     f(T) = Gamma o T,   Gamma_pq = (f(d_p) - f(d_q)) / (d_p - d_q)
// (Daleckii-Krein).  f is linear on each side of zero, so the first-order
// formula loses accuracy only through couplings between the two sides, and
// through couplings that blur the sign of a diagonal entry.  A pair (p, q) is
// accepted when
//     t_pq^2 <= gap_tol ||T||_F Delta_pq   or   |t_pq| <= abs_tol ||T||_F,
//     Delta_pq = |d_p - d_q|            (d_p, d_q of opposite sign)
//              = min(|d_p|, |d_q|)      (same sign: distance to zero)
// (the same tolerances as the Jacobi kernels' rotation test, with the gap
// replaced by the distance that governs f's second divided differences).
// A block whose pairs all pass takes P = Gamma o T directly.  Otherwise one
// pass refines Vt:
//   * non-separable failing pairs (|t_pq| > rho |d_p - d_q|) form a graph; its
//     connected components ("clusters", found on the host from the recorded
//     edges) are diagonalised exactly -- up to kRefineSmallCluster rows by
//     cluster_eig_kernel, larger ones gathered into compact matrices for the
//     selective Jacobi kernels with the gap test off -- and the rotation G
//     (identity outside the clusters) is applied as T <- G T G^T, Vt <- G Vt
//     with gathered GEMM tiles;
//   * every remaining separable failing pair takes one Newton step of the
//     eigenvector equation, Vt <- (I - K) Vt with K_pq = t_pq / (d_q - d_p),
//     followed by one Newton-Schulz orthonormalisation
//     Vt <- (3/2 I - 1/2 Vt Vt^T) Vt (GEMMs).  Accepted pairs take the step only
//     when it is tiny: inside a near-degenerate same-sign cluster t/(d_q - d_p)
//     is large and meaningless (f is linear there) and would only cost
//     orthogonality;
// and T is recomputed.  Blocks that still fail after kRefinePasses passes, or
// record more than kRefineEdgeCap non-separable pairs, fall back to the
// selective Jacobi kernels, restarted from the basis and T the call began with.
#include "v2b_kernels.cuh"
#include "v2b_refine.cuh"

namespace v2b {

__device__ __forceinline__ double gamma_pq(double li, double lj) {
    const double pi = fmax(li, 0.0), pj = fmax(lj, 0.0);
    return (li != lj) ? (pi - pj) / (li - lj) : (li > 0.0 ? 1.0 : 0.0);
}

// Row pairs (r, n-1-r) hold n-1 upper-triangle pairs together: CTA s of a
// block takes row pairs [s R, (s+1) R), R = ceil(ceil(n/2) / kClassifySplit).
__device__ __forceinline__ void split_rows(int n, int s, int &r0, int &r1) {
    const int half = (n + 1) / 2, R = (half + kClassifySplit - 1) / kClassifySplit;
    r0 = min(half, s * R);
    r1 = min(half, (s + 1) * R);
}

// Frobenius norms of the symmetrised blocks, in kClassifySplit partial sums per
// block (summed in a fixed order by the readers: the result is deterministic)
__global__ void __launch_bounds__(256)
    block_norm_kernel(const double *__restrict__ Us, const int64_t *__restrict__ boff,
                      const int *__restrict__ bdim, double *__restrict__ part) {
    const int blk = blockIdx.x, sidx = blockIdx.y, n = bdim[blk];
    __shared__ double red[32];
    int r0, r1;
    split_rows(n, sidx, r0, r1);
    const double *Ub = Us + boff[blk];
    double acc = 0.0;
    for (int r = r0; r < r1; r++)
        for (int side = 0; side < 2; side++) {
            const int row = side ? n - 1 - r : r;
            if (side && row == r) continue;   // the middle row of an odd block
            for (int c = threadIdx.x; c < n; c += blockDim.x) {
                const double v = Ub[(int64_t)row * n + c];
                acc += v * v;
            }
        }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[blk * kClassifySplit + sidx] = acc;
}

__device__ __forceinline__ double block_norm(const double *part, int blk) {
    double s = 0.0;
    for (int k = 0; k < kClassifySplit; k++) s += part[blk * kClassifySplit + k];
    return sqrt(s);
}

// Acceptance test, kClassifySplit CTAs per block.  Failing pairs are counted
// and non-separable ones recorded as edges; the last CTA of a block to finish
// sets its state (done -> done_stamp = stamp, for write_p_kernel).
__global__ void __launch_bounds__(kRefineThreads)
    refine_classify_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                           const int *__restrict__ bdim, int *__restrict__ bstate,
                           const unsigned long long *__restrict__ orth, const double *__restrict__ part,
                           double gap_tol, double abs_tol, double *__restrict__ bnorm,
                           int *__restrict__ counts, int *__restrict__ done_stamp, int stamp,
                           int *h_state, int *h_nbad, int *h_nedge, int2 *h_edges) {
    const int blk = blockIdx.x, sidx = blockIdx.y;
    const int st_in = bstate[blk];
    if (st_in != kStWork && st_in != kStBlockJacobi) return;   // uniform over the CTA
    const int n = bdim[blk];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    int *cnt = counts + 3 * blk;   // [0] failing pairs, [1] edges, [2] finished CTAs
    __shared__ int s_last;
    extern __shared__ double dg[];   // n diagonal entries
    const int64_t off = boff[blk];
    const double *Tb = T + off;
    const double nrm = block_norm(part, blk);
    const double atol = abs_tol * nrm, gtol = gap_tol * nrm;
    for (int i = tid; i < n; i += blockDim.x) dg[i] = Tb[(int64_t)i * n + i];
    __syncthreads();
    int r0, r1;
    split_rows(n, sidx, r0, r1);
    int bad = 0;
    int2 *eb = h_edges + (int64_t)blk * kRefineEdgeCap;
    // rows r0..r1-1 and their partners n-1-r, one warp per row
    for (int w = warp; w < 2 * (r1 - r0); w += nwarp) {
        const int r = r0 + (w >> 1);
        const int i = (w & 1) ? n - 1 - r : r;
        if ((w & 1) && i == r) continue;
        const double di = dg[i];
        for (int j = i + 1 + lane; j < n; j += 32) {
            const double t = 0.5 * (Tb[(int64_t)i * n + j] + Tb[(int64_t)j * n + i]);
            const double at = fabs(t);
            if (at <= atol) continue;
            const double dj = dg[j];
            const double g = fabs(di - dj);
            const bool cross = (di >= 0.0) != (dj >= 0.0);
            const double delta = cross ? g : fmin(fabs(di), fabs(dj));
            if (t * t > gtol * delta) {
                bad++;
                if (at > kRefineRho * g) {
                    const int e = atomicAdd(cnt + 1, 1);
                    if (e < kRefineEdgeCap) eb[e] = make_int2(i, j);
                }
            }
        }
    }
    bad = __reduce_add_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicAdd(cnt, bad);
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(cnt + 2, 1) == kClassifySplit - 1);
    __syncthreads();
    if (!s_last) return;
    if (tid == 0) {
        __threadfence();
        const int nbad = atomicAdd(cnt, 0), ne = atomicAdd(cnt + 1, 0);
        const bool done = nbad == 0 && __longlong_as_double((long long)orth[blk]) <= kRefineOrthDone;
        const int st = done ? kStDone : st_in;
        if (done) done_stamp[blk] = stamp;
        bstate[blk] = st;
        bnorm[blk] = nrm;
        h_state[blk] = st;
        h_nbad[blk] = nbad;
        h_nedge[blk] = ne;
        cnt[0] = cnt[1] = cnt[2] = 0;   // ready for the next launch
    }
}

// P = Gamma o T on the tiles of the blocks accepted by the classify launch
// with this stamp
__global__ void __launch_bounds__(256)
    write_p_kernel(const double *__restrict__ T, double *__restrict__ P,
                   const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                   const int *__restrict__ bdim, const int *__restrict__ done_stamp, int stamp) {
    const int4 t = tiles[blockIdx.x];
    if (done_stamp[t.x] != stamp) return;
    const int n = bdim[t.x];
    const int64_t off = boff[t.x];
    const double *Tb = T + off;
    double *Pb = P + off;
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int i = t.y * 64 + e / 64, j = t.z * 64 + e % 64;
        if (i >= n || j >= n) continue;
        const double di = Tb[(int64_t)i * n + i];
        double v;
        if (i == j) {
            v = fmax(di, 0.0);
        } else {
            const double dj = Tb[(int64_t)j * n + j];
            v = gamma_pq(di, dj) * 0.5 * (Tb[(int64_t)i * n + j] + Tb[(int64_t)j * n + i]);
        }
        Pb[(int64_t)i * n + j] = v;
    }
}

// ---------------------------------------------------------------- clusters
// Cyclic Jacobi on one cluster per CTA (k <= kRefineSmallCluster), A and the
// eigenvector rows Q in shared memory.  The round-robin pairs of every step
// are tabulated once; a step computes the rotations of its m = kp/2 disjoint
// pairs (sym.schur2), then applies all of them at once, each thread updating
// whole 2 x 2 blocks (rows of pair P, columns of pair Q) two-sidedly and the
// rows p, q of Q: two barriers per step.
__global__ void __launch_bounds__(256)
    cluster_eig_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                       const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                       const int *__restrict__ mem, double *__restrict__ Qt,
                       double *__restrict__ lam, const int *__restrict__ only, int max_sweeps) {
    const ClusterJob jb = jobs[blockIdx.x];
    if (only && !only[jb.blk]) return;   // uniform over the CTA
    const int k = jb.k, n = bdim[jb.blk];
    const int kp = k + (k & 1), ld = kp + 1, m = kp / 2, nst = kp - 1;
    const int *C = mem + jb.moff;
    const double *Tb = T + boff[jb.blk];
    extern __shared__ double sm[];
    double *A = sm;              // kp x ld
    double *Q = A + kp * ld;     // kp x ld, rows = eigenvectors
    constexpr int KM = kRefineSmallCluster;
    __shared__ unsigned char pr[KM - 1][KM / 2], qr[KM - 1][KM / 2];
    __shared__ double2 cs[KM / 2];
    __shared__ double red[32];
    __shared__ double s_thr;
    __shared__ int s_nrot;
    const int tid = threadIdx.x;
    for (int e = tid; e < nst * m; e += blockDim.x) {
        int p, q;
        rr_pair(e / m, e % m, kp, p, q);
        pr[e / m][e % m] = (unsigned char)p;
        qr[e / m][e % m] = (unsigned char)q;
    }
    double fro = 0.0;
    for (int e = tid; e < kp * kp; e += blockDim.x) {
        const int i = e / kp, j = e % kp;
        double v = 0.0;
        if (i < k && j < k) {
            const int64_t a = C[i], b = C[j];
            v = 0.5 * (Tb[a * n + b] + Tb[b * n + a]);
        }
        A[i * ld + j] = v;
        Q[i * ld + j] = (i == j) ? 1.0 : 0.0;
        fro += v * v;
    }
    fro = block_sum(fro, red);
    // rotate down to 1e-14 of the cluster's norm: below the acceptance test's
    // floor (1e-14 of the block's norm) and above the rounding noise the
    // rotations themselves leave, so the sweeps end
    if (tid == 0) s_thr = 1e-14 * sqrt(fro) + 1e-300;
    __syncthreads();
    const double thr = s_thr;
    const int P = tid >> 3, sub = tid & 7;   // 32 pair rows x 8 lanes
    for (int sweep = 0; sweep < max_sweeps; sweep++) {
        if (tid == 0) s_nrot = 0;
        __syncthreads();
        for (int st = 0; st < nst; st++) {
            if (tid < m) {
                const int p = pr[st][tid], q = qr[st][tid];
                double c = 1.0, s = 0.0;
                if (q < k) {
                    const double apq = A[p * ld + q];
                    if (fabs(apq) > thr) {
                        const double app = A[p * ld + p], aqq = A[q * ld + q];
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        atomicAdd(&s_nrot, 1);
                    }
                }
                cs[tid] = make_double2(c, s);
            }
            __syncthreads();
            if (P < m) {
                const double2 cp = cs[P];
                const int pP = pr[st][P], qP = qr[st][P];
                // A <- G A G^T on the 2 x 2 blocks (P, Q2)
                for (int Q2 = sub; Q2 < m; Q2 += 8) {
                    const double2 cq = cs[Q2];
                    if (cp.y == 0.0 && cq.y == 0.0) continue;
                    const int pQ = pr[st][Q2], qQ = qr[st][Q2];
                    const double b11 = A[pP * ld + pQ], b12 = A[pP * ld + qQ];
                    const double b21 = A[qP * ld + pQ], b22 = A[qP * ld + qQ];
                    const double m11 = b11 * cq.x - b12 * cq.y, m12 = b11 * cq.y + b12 * cq.x;
                    const double m21 = b21 * cq.x - b22 * cq.y, m22 = b21 * cq.y + b22 * cq.x;
                    double n11 = cp.x * m11 - cp.y * m21, n12 = cp.x * m12 - cp.y * m22;
                    double n21 = cp.y * m11 + cp.x * m21, n22 = cp.y * m12 + cp.x * m22;
                    if (Q2 == P) n12 = n21 = 0.0;   // the pair's own coupling, annihilated
                    A[pP * ld + pQ] = n11;
                    A[pP * ld + qQ] = n12;
                    A[qP * ld + pQ] = n21;
                    A[qP * ld + qQ] = n22;
                }
                // Q <- G Q on rows p, q
                if (cp.y != 0.0)
                    for (int jc = sub; jc < kp; jc += 8) {
                        const double qp = Q[pP * ld + jc], qq = Q[qP * ld + jc];
                        Q[pP * ld + jc] = cp.x * qp - cp.y * qq;
                        Q[qP * ld + jc] = cp.y * qp + cp.x * qq;
                    }
            }
            __syncthreads();
        }
        const int nrot = s_nrot;   // read by all before thread 0 resets it
        __syncthreads();
        if (nrot == 0) break;
    }
    double *Qo = Qt + jb.qoff;
    for (int e = tid; e < k * k; e += blockDim.x) Qo[e] = Q[(e / k) * ld + e % k];
    for (int i = tid; i < k; i += blockDim.x) lam[jb.moff + i] = A[i * ld + i];
}

// One block-Jacobi step applied in place.  The step's jobs partition each
// block's rows, so T splits into job tiles T[C_I, C_J] that only their own
// CTA reads and writes:  tile kind 0 (I, J):  T[C_I, C_J] <- Qt_I T[C_I, C_J] Qt_J^T;
// kind 1 (I, t):  Vt[C_I, 64 t .. 64 t + 64) <- Qt_I Vt[C_I, ...].
__global__ void __launch_bounds__(256)
    bj_apply_kernel(double *__restrict__ T, double *__restrict__ Vt, const int64_t *__restrict__ boff,
                    const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                    const int *__restrict__ mem, const double *__restrict__ Qt,
                    const int4 *__restrict__ tiles, const int *__restrict__ only) {
    const int4 tl = tiles[blockIdx.x];
    const ClusterJob jI = jobs[tl.x];
    if (only && !only[jI.blk]) return;   // uniform over the CTA
    const int n = bdim[jI.blk];
    const int64_t off = boff[jI.blk];
    constexpr int KM = kRefineSmallCluster, LD = KM + 1;
    extern __shared__ double sm[];
    double *sQ = sm;              // KM x LD: Qt_I
    double *sX = sQ + KM * LD;    // KM x LD: the tile, then Qt_I x tile
    double *sR = sX + KM * LD;    // KM x LD: Qt_J (kind 0)
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    const int kI = jI.k;
    const int *CI = mem + jI.moff;
    for (int e = tid; e < kI * kI; e += blockDim.x) sQ[(e / kI) * LD + e % kI] = Qt[jI.qoff + e];
    if (tl.z == 0) {
        const ClusterJob jJ = jobs[tl.y];
        const int kJ = jJ.k;
        const int *CJ = mem + jJ.moff;
        for (int e = tid; e < kJ * kJ; e += blockDim.x) sR[(e / kJ) * LD + e % kJ] = Qt[jJ.qoff + e];
        for (int e = tid; e < kI * kJ; e += blockDim.x) {
            const int i = e / kJ, j = e % kJ;
            sX[i * LD + j] = T[off + (int64_t)CI[i] * n + CJ[j]];
        }
        __syncthreads();
        // Y = Qt_I X (rows 4 ty .., cols 4 tx ..)
        double y[4][4] = {};
        for (int l = 0; l < kI; l++) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = (4 * ty + r < kI) ? sQ[(4 * ty + r) * LD + l] : 0.0;
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = (4 * tx + c < kJ) ? sX[l * LD + 4 * tx + c] : 0.0;
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) y[r][c] = fma(a[r], b[c], y[r][c]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) sX[(4 * ty + r) * LD + 4 * tx + c] = y[r][c];
        __syncthreads();
        // Z = Y Qt_J^T
        double z[4][4] = {};
        for (int l = 0; l < kJ; l++) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = sX[(4 * ty + r) * LD + l];
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = (4 * tx + c < kJ) ? sR[(4 * tx + c) * LD + l] : 0.0;
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) z[r][c] = fma(a[r], b[c], z[r][c]);
        }
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = 4 * ty + r;
            if (i >= kI) continue;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int j = 4 * tx + c;
                if (j < kJ) T[off + (int64_t)CI[i] * n + CJ[j]] = z[r][c];
            }
        }
    } else {
        const int c0 = tl.y * 64;
        for (int e = tid; e < kI * 64; e += blockDim.x) {
            const int i = e >> 6, c = c0 + (e & 63);
            sX[i * LD + (e & 63)] = (c < n) ? Vt[off + (int64_t)CI[i] * n + c] : 0.0;
        }
        __syncthreads();
        double y[4][4] = {};
        for (int l = 0; l < kI; l++) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = (4 * ty + r < kI) ? sQ[(4 * ty + r) * LD + l] : 0.0;
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = sX[l * LD + 4 * tx + c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) y[r][c] = fma(a[r], b[c], y[r][c]);
        }
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = 4 * ty + r;
            if (i >= kI) continue;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int cc = c0 + 4 * tx + c;
                if (cc < n) Vt[off + (int64_t)CI[i] * n + cc] = y[r][c];
            }
        }
    }
}

// Gathered GEMM tiles of the cluster transform G (identity outside the
// clusters, Qt on each cluster): tile (job, ti, tc) of
//     W[C_i, c]   = sum_l Qt[i][l] T[C_l, c],   Vt2[C_i, c] = sum_l Qt[i][l] Vt[C_l, c]
// for i in [32 ti, 32 ti + 32), c in [64 tc, 64 tc + 64).
__global__ void __launch_bounds__(256)
    cluster_rows_kernel(const double *__restrict__ T, const double *__restrict__ Vt,
                        double *__restrict__ W, double *__restrict__ Vt2,
                        const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                        const ClusterJob *__restrict__ jobs, const int *__restrict__ mem,
                        const double *__restrict__ Qt, const int4 *__restrict__ ctiles,
                        const int *__restrict__ only) {
    const int4 ct = ctiles[blockIdx.x];
    const ClusterJob jb = jobs[ct.x];
    if (only && !only[jb.blk]) return;
    const int k = jb.k, n = bdim[jb.blk];
    const int i0 = ct.y * 32, c0 = ct.z * 64;
    const int64_t off = boff[jb.blk];
    const int *C = mem + jb.moff;
    const double *Q = Qt + jb.qoff;
    __shared__ double sQ[32][17];
    __shared__ double sT[16][65], sV[16][65];
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    double aT[2][4] = {}, aV[2][4] = {};
    for (int l0 = 0; l0 < k; l0 += 16) {
        for (int e = tid; e < 32 * 16; e += 256) {
            const int ii = e >> 4, ll = e & 15;
            const int i = i0 + ii, l = l0 + ll;
            sQ[ii][ll] = (i < k && l < k) ? Q[(int64_t)i * k + l] : 0.0;
        }
        for (int e = tid; e < 16 * 64; e += 256) {
            const int ll = e >> 6, cc = e & 63;
            const int l = l0 + ll, c = c0 + cc;
            double vt = 0.0, vv = 0.0;
            if (l < k && c < n) {
                const int64_t idx = off + (int64_t)C[l] * n + c;
                vt = T[idx];
                vv = Vt[idx];
            }
            sT[ll][cc] = vt;
            sV[ll][cc] = vv;
        }
        __syncthreads();
#pragma unroll
        for (int ll = 0; ll < 16; ll++) {
            const double q0 = sQ[ty * 2][ll], q1 = sQ[ty * 2 + 1][ll];
#pragma unroll
            for (int jj = 0; jj < 4; jj++) {
                const double bt = sT[ll][tx * 4 + jj], bv = sV[ll][tx * 4 + jj];
                aT[0][jj] = fma(q0, bt, aT[0][jj]);
                aT[1][jj] = fma(q1, bt, aT[1][jj]);
                aV[0][jj] = fma(q0, bv, aV[0][jj]);
                aV[1][jj] = fma(q1, bv, aV[1][jj]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = i0 + ty * 2 + r;
        if (i >= k) continue;
#pragma unroll
        for (int jj = 0; jj < 4; jj++) {
            const int c = c0 + tx * 4 + jj;
            if (c >= n) continue;
            const int64_t idx = off + (int64_t)C[i] * n + c;
            W[idx] = aT[r][jj];
            Vt2[idx] = aV[r][jj];
        }
    }
}

// tile (job, ta, ti): P[a, C_i] = sum_l R(a)[C_l] Qt[i][l] for a in [64 ta, 64 ta + 64),
// i in [32 ti, 32 ti + 32), with R(a) = W[a, :] on cluster rows (already
// rotated by their own cluster) and T[a, :] elsewhere.  The cluster's own
// block comes out as Qt T[C, C] Qt^T: diagonal when the cluster solve was
// exact, and still the rotated block when its sweeps were capped.  P is free
// scratch for blocks in refinement.
__global__ void __launch_bounds__(256)
    cluster_cols_kernel(const double *__restrict__ T, const double *__restrict__ W,
                        double *__restrict__ P, const int64_t *__restrict__ boff,
                        const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                        const int *__restrict__ mem, const int *__restrict__ rowclus,
                        const int *__restrict__ rowbase, const double *__restrict__ Qt,
                        const double *__restrict__ lam, const int4 *__restrict__ ctiles,
                        const int *__restrict__ only) {
    const int4 ct = ctiles[blockIdx.x];
    const int jid = ct.x;
    const ClusterJob jb = jobs[jid];
    if (only && !only[jb.blk]) return;
    const int k = jb.k, n = bdim[jb.blk];
    const int a0 = ct.y * 64, i0 = ct.z * 32;
    const int64_t off = boff[jb.blk];
    const int *C = mem + jb.moff;
    const int *rc = rowclus + rowbase[jb.blk];
    const double *Q = Qt + jb.qoff;
    __shared__ double sR[64][17];
    __shared__ double sQ[32][17];
    const int tid = threadIdx.x, ta = tid >> 3, ti = tid & 7;
    double acc[2][4] = {};
    for (int l0 = 0; l0 < k; l0 += 16) {
        for (int e = tid; e < 64 * 16; e += 256) {
            const int aa = e >> 4, ll = e & 15;
            const int a = a0 + aa, l = l0 + ll;
            double v = 0.0;
            if (a < n && l < k) v = (rc[a] >= 0 ? W : T)[off + (int64_t)a * n + C[l]];
            sR[aa][ll] = v;
        }
        for (int e = tid; e < 32 * 16; e += 256) {
            const int ii = e >> 4, ll = e & 15;
            const int i = i0 + ii, l = l0 + ll;
            sQ[ii][ll] = (i < k && l < k) ? Q[(int64_t)i * k + l] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int ll = 0; ll < 16; ll++) {
            const double r0 = sR[ta * 2][ll], r1 = sR[ta * 2 + 1][ll];
#pragma unroll
            for (int jj = 0; jj < 4; jj++) {
                const double q = sQ[ti * 4 + jj][ll];
                acc[0][jj] = fma(r0, q, acc[0][jj]);
                acc[1][jj] = fma(r1, q, acc[1][jj]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int a = a0 + ta * 2 + r;
        if (a >= n) continue;
#pragma unroll
        for (int jj = 0; jj < 4; jj++) {
            const int i = i0 + ti * 4 + jj;
            if (i >= k) continue;
            P[off + (int64_t)a * n + C[i]] = acc[r][jj];
        }
    }
}

// tile (job, t): T[a, C_i] = P[a, C_i] for rows a in [64 t, 64 t + 64), and
// for columns b in that range outside every cluster T[C_i, b] = W[C_i, b];
// Vt[C_i, b] = Vt2[C_i, b] for every b in the range.
__global__ void __launch_bounds__(256)
    cluster_commit_kernel(double *__restrict__ T, const double *__restrict__ W,
                          const double *__restrict__ P, double *__restrict__ Vt,
                          const double *__restrict__ Vt2, const int64_t *__restrict__ boff,
                          const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                          const int *__restrict__ mem, const int *__restrict__ rowclus,
                          const int *__restrict__ rowbase, const int4 *__restrict__ ctiles,
                          const int *__restrict__ only) {
    const int4 ct = ctiles[blockIdx.x];
    const ClusterJob jb = jobs[ct.x];
    if (only && !only[jb.blk]) return;
    const int k = jb.k, n = bdim[jb.blk];
    const int t0 = ct.y * 64;
    const int64_t off = boff[jb.blk];
    const int *C = mem + jb.moff;
    const int *rc = rowclus + rowbase[jb.blk];
    for (int e = threadIdx.x; e < 64 * k; e += blockDim.x) {
        const int i = e / 64, x = t0 + e % 64;
        if (x >= n) continue;
        const int64_t col = off + (int64_t)x * n + C[i];   // (row x, cluster column C_i)
        T[col] = P[col];
        const int64_t row = off + (int64_t)C[i] * n + x;   // (cluster row C_i, column x)
        if (rc[x] < 0) T[row] = W[row];
        Vt[row] = Vt2[row];
    }
}

// Tc = sym(T[C, C]) and Vc = I in compact k x k storage at qoff, for clusters
// diagonalised by the Jacobi kernels (grid: jobs x 16, grid-stride inside)
__global__ void __launch_bounds__(256)
    cluster_gather_kernel(const double *__restrict__ T, const int64_t *__restrict__ boff,
                          const int *__restrict__ bdim, const ClusterJob *__restrict__ jobs,
                          const int *__restrict__ mem, const int *__restrict__ jlist,
                          double *__restrict__ Tc, double *__restrict__ Vc) {
    const ClusterJob jb = jobs[jlist[blockIdx.x]];
    const int k = jb.k, n = bdim[jb.blk];
    const int *C = mem + jb.moff;
    const double *Tb = T + boff[jb.blk];
    const int64_t kk = (int64_t)k * k;
    for (int64_t e = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; e < kk;
         e += (int64_t)gridDim.y * blockDim.x) {
        const int i = (int)(e / k), j = (int)(e % k);
        const int64_t a = C[i], b = C[j];
        Tc[jb.qoff + e] = 0.5 * (Tb[a * n + b] + Tb[b * n + a]);
        Vc[jb.qoff + e] = (i == j) ? 1.0 : 0.0;
    }
}

// lam[moff + i] = D[qoff + i k + i]: the eigenvalues left on the diagonal of
// the rotated compact matrix D by the Jacobi kernels
__global__ void cluster_lam_kernel(const ClusterJob *__restrict__ jobs, const int *__restrict__ jlist,
                                   int njobs, const double *__restrict__ Dsmall,
                                   const double *__restrict__ Dbig, int big_from,
                                   double *__restrict__ lam) {
    for (int q = blockIdx.x; q < njobs; q += gridDim.x) {
        const ClusterJob jb = jobs[jlist[q]];
        const double *D = (q >= big_from ? Dbig : Dsmall) + jb.qoff;
        for (int i = threadIdx.x; i < jb.k; i += blockDim.x) lam[jb.moff + i] = D[(int64_t)i * jb.k + i];
    }
}

// ---------------------------------------------------------------- Newton
__global__ void __launch_bounds__(256)
    newton_m_kernel(const double *__restrict__ T, double *__restrict__ M,
                    const int4 *__restrict__ tiles, const int64_t *__restrict__ boff,
                    const int *__restrict__ bdim, const int *__restrict__ bstate,
                    const double *__restrict__ bnorm, double gap_tol, double abs_tol) {
    const int4 t = tiles[blockIdx.x];
    if (bstate[t.x] != kStWork) return;
    const int n = bdim[t.x];
    const int64_t off = boff[t.x];
    const double *Tb = T + off;
    const double nrm = bnorm[t.x];
    const double atol = abs_tol * nrm, gtol = gap_tol * nrm;
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int r = t.y * 64 + e / 64, c = t.z * 64 + e % 64;
        if (r >= n || c >= n) continue;
        double v;
        if (r == c) {
            v = 1.0;
        } else {
            const double tv = 0.5 * (Tb[(int64_t)r * n + c] + Tb[(int64_t)c * n + r]);
            const double dr = Tb[(int64_t)r * n + r], dc = Tb[(int64_t)c * n + c];
            const double g = dc - dr;
            v = 0.0;
            if (tv != 0.0 && fabs(tv) <= kRefineRho * fabs(g)) {
                const double k = tv / g;
                const bool cross = (dr >= 0.0) != (dc >= 0.0);
                const double delta = cross ? fabs(g) : fmin(fabs(dr), fabs(dc));
                const bool bad = fabs(tv) > atol && tv * tv > gtol * delta;
                if (bad || fabs(k) <= kRefineKappa) v = -k;
            }
        }
        M[off + (int64_t)r * n + c] = v;
    }
}

}  // namespace v2b
