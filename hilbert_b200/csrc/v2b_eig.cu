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
#include "v2b_kernels.cuh"

#include <mutex>

#include <algorithm>

namespace v2b {

// ---------------------------------------------------------------------------
// batched FP64 GEMM over square blocks: C_b = op(A_b) op(B_b) [+ epilogue]
//
// FP64 tensor cores (mma.sync m8n8k4 .f64): a 64 x 64 output tile per CTA of
// 4 warps, each warp a 32 x 32 sub-tile of 4 x 4 m8n8 fragments (32
// accumulators per thread).  K runs in chunks of 16 through a 3-stage
// cp.async pipeline (8-byte copies: a block of odd dimension starts at an
// odd double, so 16-byte alignment is not available; out-of-range elements
// are zero-filled by the copy itself).  Each operand tile is stored with its
// global contiguous index innermost (k-major when the matrix is read down
// its columns), padded so that both the copies and the fragment reads are
// free of bank conflicts.
//
// With a scheduler counter the grid is persistent (the SM count times the
// CTAs an SM holds) and CTAs take tiles in list order, the tile list sorted
// by block dimension (its K) descending: the longest tiles start first and
// the short ones fill in behind them.  Without one, CTA i computes tile i.
//
// Split K: when a launch has fewer tiles than the grid has CTA slots, the
// plan cuts the K range of the large blocks' tiles into S parts (tile word w:
// bit 0 mirror, bits 4-7 the part s, bits 8-11 S, bits 12+ the output tile's
// group; S <= kGemmMaxSplit).  Each part stores its 64 x 64 partial product
// in the group's slot s of split_ws and counts itself in split_cnt[group]; the part that arrives
// last sums the slots in the order s = 0 .. S-1 (the same bits whichever
// part arrives last), re-arms the counter and runs the epilogue.
constexpr int kGemmBK = 16;
constexpr int kGemmStages = 3;
constexpr int kGemmThreads = 128;
constexpr int kPadM = kGemmTile + 4;    // k-major rows: 64 + 4 doubles
constexpr int kPadK = kGemmBK + 4;      // m-major rows: 16 + 4 doubles
constexpr int kOpDoubles = (kGemmTile * kPadK > kGemmBK * kPadM) ? kGemmTile * kPadK : kGemmBK * kPadM;
constexpr int kGemmSmem = kGemmStages * 2 * kOpDoubles * (int)sizeof(double);

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int bytes = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D (8 x 8) += A (8 x 4, row) B (4 x 8, col); per lane: A[l/4][l%4],
// B[l%4][l/4], D[l/4][2 (l%4) + {0, 1}]
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// shared-memory index of element (m, k) of a 64 x 16 operand tile
template <bool KMAJOR>
__device__ __forceinline__ int op_idx(int m, int k) {
    return KMAJOR ? k * kPadM + m : m * kPadK + k;
}

// one 64 x 16 operand tile: rows m of the operand (rows of op(A) or columns of
// op(B)) from m0, k from k0.  KMAJOR: the global matrix is contiguous in m
// (element (m, k) at X[k n + m]), else in k (X[m n + k]).
template <bool KMAJOR>
__device__ __forceinline__ void load_op(double *sm, const double *__restrict__ X, int n, int m0, int k0) {
#pragma unroll
    for (int it = 0; it < kGemmTile * kGemmBK / kGemmThreads; it++) {
        const int e = it * kGemmThreads + threadIdx.x;
        const int m = KMAJOR ? e % kGemmTile : e / kGemmBK;
        const int k = KMAJOR ? e / kGemmTile : e % kGemmBK;
        const int gm = m0 + m, gk = k0 + k;
        const bool ok = gm < n && gk < n;
        const double *src = ok ? (KMAJOR ? X + (int64_t)gk * n + gm : X + (int64_t)gm * n + gk) : X;
        cp_async8(sm + op_idx<KMAJOR>(m, k), src, ok);
    }
}

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 3)
    gemm_tiles_kernel(const double *__restrict__ A, const double *__restrict__ B,
                      double *__restrict__ C, const int4 *__restrict__ tiles,
                      const int64_t *__restrict__ boff, const int *__restrict__ bdim,
                      const double *__restrict__ Cin, const double *__restrict__ Us, double inv_mu,
                      double *__restrict__ xo, double *__restrict__ zo,
                      const int *__restrict__ bstate, unsigned long long *__restrict__ orth,
                      int ntiles, int *__restrict__ sched, double *__restrict__ split_ws,
                      int *__restrict__ split_cnt) {
    // op(A) rows are m-contiguous in memory when A is read transposed;
    // op(B) columns are m-contiguous when B is read as stored
    constexpr bool AK = TA, BKM = !TB;
    extern __shared__ double gsm[];
    __shared__ int s_tile, s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int fr = lane >> 2, fk = lane & 3;
    for (int iter = 0;; iter++) {
        int ti;
        if (sched) {
            if (threadIdx.x == 0) {
                int t = atomicAdd(sched, 1);
                if (t >= ntiles) {
                    // the last CTA to run out re-arms the counter for the next launch
                    if (atomicAdd(sched + 1, 1) == (int)gridDim.x - 1) {
                        sched[0] = 0;
                        sched[1] = 0;
                    }
                    t = -1;
                }
                s_tile = t;
            }
            __syncthreads();
            ti = s_tile;
            __syncthreads();
        } else {
            ti = iter == 0 ? (int)blockIdx.x : -1;
        }
        if (ti < 0) break;
        const int4 t = tiles[ti];
        const int blk = t.x, n = bdim[blk];
        if (bstate && bstate[blk] != 0) continue;   // uniform over the CTA
        const int64_t off = boff[blk];
        const int r0 = t.y * kGemmTile, c0 = t.z * kGemmTile;
        const double *Ab = A + off, *Bb = B + off;
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

        const int split = (t.w >> 8) & 15, part = (t.w >> 4) & 15;
        const int nk_all = (n + kGemmBK - 1) / kGemmBK;
        // this part's K chunks: kb .. kb + nk - 1
        const int per = split > 1 ? (nk_all + split - 1) / split : nk_all;
        const int kb = split > 1 ? min(part * per, nk_all) : 0;
        const int nk = min(nk_all - kb, per);
#pragma unroll
        for (int st = 0; st < kGemmStages - 1; st++) {
            if (st < nk) {
                double *sa = gsm + st * 2 * kOpDoubles;
                load_op<AK>(sa, Ab, n, r0, (kb + st) * kGemmBK);
                load_op<BKM>(sa + kOpDoubles, Bb, n, c0, (kb + st) * kGemmBK);
            }
            cp_async_commit();
        }
        for (int kt = 0; kt < nk; kt++) {
            cp_async_wait<kGemmStages - 2>();
            __syncthreads();
            // refill the stage consumed one step ago (every warp is past it)
            const int kn = kt + kGemmStages - 1;
            if (kn < nk) {
                double *sa = gsm + (kn % kGemmStages) * 2 * kOpDoubles;
                load_op<AK>(sa, Ab, n, r0, (kb + kn) * kGemmBK);
                load_op<BKM>(sa + kOpDoubles, Bb, n, c0, (kb + kn) * kGemmBK);
            }
            cp_async_commit();
            const double *sa = gsm + (kt % kGemmStages) * 2 * kOpDoubles;
            const double *sb = sa + kOpDoubles;
#pragma unroll
            for (int k4 = 0; k4 < kGemmBK; k4 += 4) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = sa[op_idx<AK>(wm + i * 8 + fr, k4 + fk)];
#pragma unroll
                for (int j = 0; j < 4; j++) b[j] = sb[op_idx<BKM>(wn + j * 8 + fr, k4 + fk)];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
            }
        }
        cp_async_wait<0>();
        __syncthreads();   // the next tile's copies reuse the stages

        if (split > 1) {
            const unsigned group = (unsigned)t.w >> 12;
            double *slot = split_ws + ((int64_t)group * kGemmMaxSplit + part) * (kGemmTile * kGemmTile);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
                        __stcg(slot + (wm + i * 8 + fr) * kGemmTile + wn + j * 8 + 2 * fk + h, acc[i][j][h]);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) s_last = atomicAdd(split_cnt + group, 1) == split - 1;
            __syncthreads();
            if (!s_last) continue;
            __threadfence();
            const double *slots = split_ws + (int64_t)group * kGemmMaxSplit * (kGemmTile * kGemmTile);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int e = (wm + i * 8 + fr) * kGemmTile + wn + j * 8 + 2 * fk + h;
                        double v = __ldcg(slots + e);
                        for (int q = 1; q < split; q++) v += __ldcg(slots + q * (kGemmTile * kGemmTile) + e);
                        acc[i][j][h] = v;
                    }
            if (threadIdx.x == 0) split_cnt[group] = 0;   // every part has arrived: re-arm
        }

        double dev = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = r0 + wm + i * 8 + fr;
            if (r >= n) continue;
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int c = c0 + wn + j * 8 + 2 * fk + h;
                    if (c >= n) continue;
                    const double v = acc[i][j][h];
                    // t.w: an off-diagonal tile of a symmetric product, stored
                    // at (r, c) and at its mirror image (c, r)
                    for (int m = 0; m <= (t.w & 1); m++) {
                        const int64_t e = m ? off + (int64_t)c * n + r : off + (int64_t)r * n + c;
                        if (EPI == kEpiStore) {
                            C[e] = v;
                        } else if (EPI == kEpiAdd) {
                            C[e] = Cin[e] + v;
                        } else if (EPI == kEpiNS) {   // v = (Vt Vt^T)[r][c]
                            const double id = (r == c) ? 1.0 : 0.0;
                            C[e] = 1.5 * id - 0.5 * v;
                            dev = fmax(dev, fabs(v - id));
                        } else {   // kEpiProject: v = U+
                            xo[e] = v * inv_mu;
                            zo[e] = v - Us[e];
                        }
                    }
                }
        }
        if (EPI == kEpiNS) {
            // non-negative doubles order like their bit patterns
            dev = warp_max(dev);
            if (lane == 0 && dev > 0.0)
                atomicMax(orth + blk, (unsigned long long)__double_as_longlong(dev));
        }
    }
}

template <bool TA, bool TB, int EPI>
static cudaError_t launch_variant(int ntiles, cudaStream_t s, GEMM_ARGS, int *sched, double *split_ws,
                                  int *split_cnt) {
    auto kern = gemm_tiles_kernel<TA, TB, EPI>;
    // opt in to the pipeline's shared memory and size the persistent grid,
    // once per variant, device and context (function attributes are per
    // device and do not survive a cudaDeviceReset)
    struct Cfg {
        unsigned long long ctx = 0;
        int slots = 0;
    };
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static Cfg cache[kMaxDevices];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    Cfg cfg;
    {
        std::lock_guard<std::mutex> lock(mu);
        const unsigned long long ctx = current_context_id();
        if (cache[dev].slots == 0 || cache[dev].ctx != ctx) {
            int sms = 0, occ = 0;
            err = raise_dynamic_smem((const void *)kern, kGemmSmem);
            if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (err == cudaSuccess)
                err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kGemmThreads, kGemmSmem);
            if (err != cudaSuccess) return err;
            // the context id is read after the calls above, which create the context if needed
            cache[dev].ctx = current_context_id();
            cache[dev].slots = std::max(1, sms * occ);
        }
        cfg = cache[dev];
    }
    const int grid = sched ? std::min(ntiles, cfg.slots) : ntiles;
    kern<<<grid, kGemmThreads, kGemmSmem, s>>>(A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate,
                                               orth, ntiles, sched, split_ws, split_cnt);
    return cudaGetLastError();
}

cudaError_t gemm_slots(int *slots) {
    int dev = 0, sms = 0, occ = 0;
    const void *kern = (const void *)gemm_tiles_kernel<false, false, kEpiStore>;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = raise_dynamic_smem(kern, kGemmSmem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kGemmThreads, kGemmSmem);
    if (e == cudaSuccess) *slots = std::max(1, sms * occ);
    return e;
}

cudaError_t launch_gemm_tiles(GemmVariant v, int ntiles, cudaStream_t s, GEMM_ARGS, int *sched, double *split_ws,
                              int *split_cnt) {
    if (ntiles <= 0) return cudaSuccess;
#define V2B_GEMM_CASE(NAME, TA, TB, EPI) \
    case NAME:                           \
        return launch_variant<TA, TB, EPI>(ntiles, s, A, B, C, tiles, boff, bdim, Cin, Us, inv_mu, xo, zo, bstate, orth, \
                                           sched, split_ws, split_cnt);
    switch (v) {
        V2B_GEMM_CASE(kGemmNTNewtonSchulz, false, true, kEpiNS)
        V2B_GEMM_CASE(kGemmNTStore, false, true, kEpiStore)
        V2B_GEMM_CASE(kGemmNNStore, false, false, kEpiStore)
        V2B_GEMM_CASE(kGemmTNStore, true, false, kEpiStore)
        V2B_GEMM_CASE(kGemmNNProject, false, false, kEpiProject)
        V2B_GEMM_CASE(kGemmNNAdd, false, false, kEpiAdd)
    }
#undef V2B_GEMM_CASE
    return cudaErrorInvalidValue;
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
