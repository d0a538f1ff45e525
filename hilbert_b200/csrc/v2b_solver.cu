// Host orchestration of the B200 boundary-point iteration and the C ABI
// declared in include/v2rdm_b200.h.
//
// Outer protocol (hilbert v2rdm_solver.cc:1296-1361 with libsdp's BPSDP):
//   mu0 = 0.1; each solve() call runs up to MU_UPDATE_FREQUENCY iterations
//   with mu fixed, then mu <- mu * eps_p / eps_d.
// One iteration on the device:
//   cg_kernel          (A A^T) y = A(c - z) + mu (b - A x)       [cooperative]
//   spmv_AT_U_kernel   A^T y, U = mu x + A^T y - c
//   jacobi_project     x = U+ / mu, z = U+ - U   per PSD block
//   spmv_A2_kernel     A x, A (c - z)  (reused by the next iteration's rhs)
//   stats_kernel       eps_p, eps_d, c.x, b.y  -> pinned host readback
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "v2b_bigjacobi.cuh"
#include "v2b_eig.cuh"
#include "v2b_kernels.cuh"
#include "v2b_orbital.cuh"
#include "v2b_refine.cuh"
#include "v2rdm_b200.h"
#include "v2rdm_problem.h"
#include "rdm_records.h"
#include "doci_problem.h"

namespace {

thread_local std::string g_last_error;

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define V2B_CK(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw Failure(V2B_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const Failure &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::invalid_argument &e) {
        g_last_error = e.what();
        return V2B_BAD_ARG;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return V2B_INTERNAL;
    }
}

template <class T>
T *dalloc(size_t n) {
    void *p = nullptr;
    V2B_CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    return (T *)p;
}

// first index of a non-finite value in v[0..n), or -1 (host arrays)
int64_t first_nonfinite(const double *v, int64_t n) {
    for (int64_t i = 0; i < n; i++)
        if (!std::isfinite(v[i])) return i;
    return -1;
}

// lowest index of a non-finite value in each of up to three device vectors
__global__ void nonfinite_kernel(const double *__restrict__ a, int64_t na, const double *__restrict__ b,
                                 int64_t nb, const double *__restrict__ c, int64_t nc,
                                 unsigned long long *first) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na + nb + nc; i += stride) {
        const int which = i < na ? 0 : (i < na + nb ? 1 : 2);
        const int64_t k = i - (which > 0 ? na : 0) - (which > 1 ? nb : 0);
        const double v = which == 0 ? a[k] : (which == 1 ? b[k] : c[k]);
        if (!isfinite(v)) atomicMin(first + which, (unsigned long long)k);
    }
}

void ensure_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        throw Failure(V2B_NO_DEVICE, "no CUDA device available");
}

struct DeviceOp {
    uint32_t *rp = nullptr, *ent = nullptr;
    int64_t *long_rows = nullptr;   // rows longer than kCgLongRow
    int64_t nrows = 0, n_long = 0;
    size_t nnz = 0;
    v2b::Palette pal{};
    // sliced-ELL copy of the other rows, for the CG kernel
    uint32_t *sell_ent = nullptr, *sell_perm = nullptr, *sell_off = nullptr;
    uint8_t *sell_len = nullptr;
    int64_t nslices = 0;
    std::vector<uint32_t> host_off;   // slice offsets (entries), for the work split
    uint32_t *sell_split = nullptr;   // per CG warp: its first slice (nwarps + 1 entries)

    void upload(const v2b::PackedOperator &op) {
        nrows = op.nrows;
        nnz = op.entries.size();
        rp = dalloc<uint32_t>(op.row_ptr.size());
        ent = dalloc<uint32_t>(nnz);
        V2B_CK(cudaMemcpy(rp, op.row_ptr.data(), op.row_ptr.size() * 4, cudaMemcpyHostToDevice));
        V2B_CK(cudaMemcpy(ent, op.entries.data(), nnz * 4, cudaMemcpyHostToDevice));
        for (int i = 0; i < 16; i++) pal.v[i] = i < (int)op.palette.size() ? op.palette[i] : 0.0;
        std::vector<int64_t> lr;
        for (int64_t r = 0; r < nrows; r++)
            if (op.row_ptr[r + 1] - op.row_ptr[r] > v2b::kCgLongRow) lr.push_back(r);
        n_long = (int64_t)lr.size();
        long_rows = dalloc<int64_t>(lr.size());
        if (n_long) V2B_CK(cudaMemcpy(long_rows, lr.data(), lr.size() * 8, cudaMemcpyHostToDevice));
        build_sell(op);
    }

    // SELL-C-sigma with C = 32: inside each window of kSellSigma rows the
    // short rows are sorted by length (longest first, stable), cut into
    // slices of 32 (the window's last slice padded with empty lanes) and
    // stored column-major at the slice's width
    void build_sell(const v2b::PackedOperator &op) {
        std::vector<uint32_t> e, perm, off;
        std::vector<uint8_t> len;
        std::vector<std::pair<uint32_t, uint32_t>> w;   // (length, row)
        for (int64_t w0 = 0; w0 < nrows; w0 += v2b::kSellSigma) {
            const int64_t w1 = std::min<int64_t>(nrows, w0 + v2b::kSellSigma);
            w.clear();
            for (int64_t r = w0; r < w1; r++) {
                const uint32_t L = op.row_ptr[r + 1] - op.row_ptr[r];
                if (L <= v2b::kCgLongRow) w.push_back({L, (uint32_t)r});
            }
            std::stable_sort(w.begin(), w.end(), [](const std::pair<uint32_t, uint32_t> &a,
                                                    const std::pair<uint32_t, uint32_t> &b) {
                return a.first > b.first;
            });
            for (size_t s0 = 0; s0 < w.size(); s0 += 32) {
                const size_t cnt = std::min<size_t>(32, w.size() - s0);
                const uint32_t width = w[s0].first;
                off.push_back((uint32_t)e.size());
                for (uint32_t k = 0; k < width; k++)
                    for (size_t l = 0; l < 32; l++) {
                        uint32_t v = 0;
                        if (l < cnt && k < w[s0 + l].first) v = op.entries[op.row_ptr[w[s0 + l].second] + k];
                        e.push_back(v);
                    }
                for (size_t l = 0; l < 32; l++) {
                    perm.push_back(l < cnt ? w[s0 + l].second : 0xffffffffu);
                    len.push_back(l < cnt ? (uint8_t)w[s0 + l].first : 0);
                }
            }
        }
        nslices = (int64_t)off.size();
        off.push_back((uint32_t)e.size());
        host_off = off;
        sell_ent = dalloc<uint32_t>(e.size());
        sell_perm = dalloc<uint32_t>(perm.size());
        sell_len = dalloc<uint8_t>(len.size());
        sell_off = dalloc<uint32_t>(off.size());
        if (!e.empty()) V2B_CK(cudaMemcpy(sell_ent, e.data(), e.size() * 4, cudaMemcpyHostToDevice));
        if (!perm.empty()) {
            V2B_CK(cudaMemcpy(sell_perm, perm.data(), perm.size() * 4, cudaMemcpyHostToDevice));
            V2B_CK(cudaMemcpy(sell_len, len.data(), len.size(), cudaMemcpyHostToDevice));
        }
        V2B_CK(cudaMemcpy(sell_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
    }
    // Contiguous runs of slices, one per CG warp, of about equal work: a
    // slice costs its stored entries (32 x its width) plus a fixed share for
    // its row indices and the write of its results; the long rows, which
    // warps take round-robin (row k: warp k mod nwarps), count toward their
    // warp's share.  Warp w's run ends where the cumulative slice work comes
    // nearest to (w + 1) x the average less the long-row work of warps 0..w
    // (cumulative targets: the rounding of one warp does not carry into the
    // next).
    void split_slices(int64_t nwarps, const v2b::PackedOperator &op) {
        const double fixed = 32.0 * 3.0;
        std::vector<double> extra(nwarps, 0.0);
        int64_t k = 0;
        double total = 0.0;
        for (int64_t r = 0; r < op.nrows; r++) {
            const uint32_t L = op.row_ptr[r + 1] - op.row_ptr[r];
            if (L <= v2b::kCgLongRow) continue;
            const double c = 32.0 * (double)((L + 31) / 32) + fixed;
            extra[k % nwarps] += c;
            total += c;
            k++;
        }
        std::vector<double> cum(nslices + 1, 0.0);
        for (int64_t s = 0; s < nslices; s++) cum[s + 1] = cum[s] + (double)(host_off[s + 1] - host_off[s]) + fixed;
        total += cum[nslices];
        const double avg = total / (double)nwarps;
        std::vector<uint32_t> first(nwarps + 1, 0);
        double ce = 0.0;
        for (int64_t w = 0; w < nwarps; w++) {
            ce += extra[w];
            const double target = (double)(w + 1) * avg - ce;
            int64_t s = std::lower_bound(cum.begin(), cum.end(), target) - cum.begin();
            if (s > 0 && s <= nslices && target - cum[s - 1] < cum[s] - target) s--;
            s = std::min<int64_t>(std::max<int64_t>(s, first[w]), nslices);
            first[w + 1] = (uint32_t)s;
        }
        first[nwarps] = (uint32_t)nslices;
        if (sell_split) cudaFree(sell_split);
        sell_split = dalloc<uint32_t>(first.size());
        V2B_CK(cudaMemcpy(sell_split, first.data(), first.size() * 4, cudaMemcpyHostToDevice));
    }
    v2b::SellOp sell() const {
        v2b::SellOp s;
        s.ent = sell_ent;
        s.perm = sell_perm;
        s.off = sell_off;
        s.len = sell_len;
        s.nslices = nslices;
        s.split = sell_split;
        return s;
    }
    void release() {
        for (void *p : {(void *)rp, (void *)ent, (void *)long_rows, (void *)sell_ent, (void *)sell_perm,
                        (void *)sell_off, (void *)sell_len, (void *)sell_split})
            cudaFree(p);
        sell_split = nullptr;
        rp = ent = sell_ent = sell_perm = sell_off = nullptr;
        sell_len = nullptr;
        long_rows = nullptr;
    }
};

// Per-block PSD projection for a fixed list of block sizes.  The rows of Vt
// hold each block's eigenvector basis from the previous call (the identity
// before the first), so every call starts with
//   symmetrize; W = Us Vt^T; T = Vt W                        (GEMM tiles, all blocks)
// and then, per block, either
//   warm refinement (v2b_refine.cu): accept T when its remaining couplings
//     leave the first-order formula P = Gamma o T exact to the tolerances;
//     else diagonalise the non-separable clusters exactly, take one Newton
//     step for the separable pairs, re-orthonormalise and recompute T (up to
//     kRefinePasses times), or
//   selective Jacobi on T (blocks below kRefineMinDim, the first call after a
//   reset, and blocks the refinement hands over):
//     blocks <= kJacobiMaxDim  jacobi_warm_kernel (one CTA, T in shared memory)
//     larger blocks            jacobi_big_kernel  (one 8-CTA cluster, T in L2)
// and finally Y = Vt^T P; U+ = Y Vt -> x = U+/mu, z = U+ - Us.   (GEMM tiles)
// Every kReorthEvery calls Vt is re-orthonormalised, Vt <- Vt + (I - Vt Vt^T) Vt / 2.
struct ProjectPlan {
    static constexpr int kReorthEvery = 64;
    std::vector<int> dims;
    std::vector<int64_t> h_off;
    std::vector<int64_t> h_roff_small, h_roff_big;   // per block, -1 if not of that kind
    int nblk = 0, nsmall = 0, nbig = 0;
    int64_t total = 0, rows_total = 0;
    int64_t *boff = nullptr, *rot_off = nullptr;
    int *bdim = nullptr, *counters = nullptr;
    int4 *tiles = nullptr;
    int ntiles = 0;
    // the upper tiles (row tile <= column tile) of every block, w = 1 on the
    // off-diagonal ones: for products that are symmetric, whose kernel then
    // stores each off-diagonal tile and its mirror image
    int4 *stiles = nullptr;
    int nstiles = 0;
    // both lists with the tiles of blocks of kSplitMinDim rows or more cut
    // along K into the number of parts the tuner found fastest
    // (gemm_tiles_kernel); the parts' partial products meet in split_ws,
    // counted in split_cnt
    static constexpr int kSplitMinDim = 256;
    int4 *ktiles = nullptr, *kstiles = nullptr;
    int nktiles = 0, nkstiles = 0;
    double *split_ws = nullptr;
    int *split_cnt = nullptr;
    bool split_k = true;
    int split_full = 1, split_sym = 1;   // the tuner's choices
    int *gemm_sched = nullptr;   // persistent-grid tile counter of the GEMM launches
    double2 *rot = nullptr;
    double *Vt = nullptr, *Vt2 = nullptr, *Us = nullptr, *W = nullptr, *T = nullptr, *P = nullptr;
    // large-block work arrays
    static constexpr int kBigSweeps = 16;
    double *norm_b = nullptr;
    double2 *rec_b = nullptr;
    int max_big = 0;
    size_t smem = 0;
    int max_sweeps = 30;
    // Jacobi block lists of one call (subsets), device copies and pinned staging
    int64_t *sub_boff = nullptr, *sub_roff = nullptr;
    int *sub_bdim = nullptr;
    int64_t *sub32_boff = nullptr, *sub32_roff = nullptr;   // mode 2's FP32 eigensolve list
    int *sub32_bdim = nullptr;
    int64_t *h_sub = nullptr;   // pinned: 3 x nblk int64 (boff, roff, bdim) for small then big
    // refinement state
    int *bstate = nullptr, *h_bstate_up = nullptr;   // device / pinned staging
    unsigned long long *orth = nullptr;
    double *bnorm = nullptr;
    double *norm_part = nullptr;     // kClassifySplit partial squared norms per block
    int *cls_counts = nullptr;       // per block: failing pairs, edges, finished CTAs
    int *done_stamp = nullptr;       // classify launch that accepted the block
    int stamp = 0;
    double *Vsave = nullptr, *Tsave = nullptr;   // the call's starting basis and T
    int *h_state = nullptr, *h_nbad = nullptr, *h_nedge = nullptr;   // mapped host memory
    int2 *h_edges = nullptr;
    int *d_state = nullptr, *d_nbad = nullptr, *d_nedge = nullptr;   // their device aliases
    int2 *d_edges = nullptr;
    int *rowbase = nullptr;
    double *Qt = nullptr, *lam = nullptr;     // cluster eigenvectors (rows) and eigenvalues
    double *Tc = nullptr, *Pc = nullptr;      // compact clusters for the Jacobi kernels
    // per-pass cluster lists: one device arena filled from one pinned staging
    // buffer (jobs, members, row -> cluster, tile lists, Jacobi lists); both grow
    unsigned char *arena = nullptr, *h_arena = nullptr;
    size_t arena_bytes = 0;
    double2 *crec = nullptr;                  // rotation records of Jacobi-diagonalised clusters
    int64_t crec_slots = 0;
    double *cnorm = nullptr;
    int cnorm_n = 0;
    size_t mid_smem = 0;
    // block-Jacobi schedule (fixed by the block sizes): per step, the pairs of
    // kBJGroup-row groups of every block of at least kRefineMinDim rows, as
    // cluster jobs with their tile lists, device-resident
    struct BJStep {
        size_t o_jobs = 0, o_mem = 0, o_tiles = 0;
        int njobs = 0, ntiles = 0;
    };
    std::vector<BJStep> bj_steps;
    std::vector<int> bj_nsteps;   // steps per sweep of each block (0: not scheduled)
    unsigned char *bj_dev = nullptr;
    int *bj_on = nullptr, *h_bjon = nullptr;
    long refine_bj_sweeps = 0;
    size_t classify_smem = 0;
    // recorded after a call's last upload from the pinned staging buffers; the
    // next call waits for it before writing them again
    cudaEvent_t staged = nullptr;
    bool staged_pending = false;
    // host-side counters
    long refine_accepted = 0, refine_jacobi = 0, refine_passes = 0, refine_clusters = 0;
    long refine_large_clusters = 0;   // clusters diagonalised by the Jacobi kernels
    long fb_edges = 0, fb_passes = 0;  // why refined blocks went to Jacobi
    // optional CUDA-event timing of the projection's phases (with the
    // problem's profiling): 0 GEMM tiles, 1 acceptance test (norms, test,
    // P), 2 clusters + Newton step, 3 block-Jacobi sweeps, 4 Jacobi kernels
    static constexpr int kPhases = 5;
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pev_phase;
    int pev_used = 0;
    double ph_ms[kPhases] = {};
    long ph_n[kPhases] = {};
    void ph_begin(int ph, cudaStream_t s) {
        if (!prof) return;
        if ((size_t)(2 * pev_used + 2) > pev.size()) {
            for (int k = 0; k < 64; k++) {
                cudaEvent_t e;
                V2B_CK(cudaEventCreate(&e));
                pev.push_back(e);
            }
            pev_phase.resize(pev.size() / 2);
        }
        pev_phase[pev_used] = ph;
        V2B_CK(cudaEventRecord(pev[2 * pev_used], s));
    }
    void ph_end(cudaStream_t s) {
        if (!prof) return;
        V2B_CK(cudaEventRecord(pev[2 * pev_used + 1], s));
        pev_used++;
    }
    // after the stream has been synchronised
    void ph_collect() {
        for (int k = 0; k < pev_used; k++) {
            float ms = 0.f;
            V2B_CK(cudaEventElapsedTime(&ms, pev[2 * k], pev[2 * k + 1]));
            ph_ms[pev_phase[k]] += ms;
            ph_n[pev_phase[k]]++;
        }
        pev_used = 0;
    }
    bool fresh = true;
    bool built = false;
    // 0: warm refinement; 1: selective Jacobi on every block, every call;
    // 2: warm refinement where the blocks above kJacobiMaxDim rows that
    //    would change to block-Jacobi sweeps take an FP32 selective Jacobi
    //    eigensolve instead, followed by the FP64 Rayleigh-Ritz step
    //    (T recomputed in the new basis) and the FP64 acceptance test and
    //    Newton passes; block-Jacobi only if that fails
    int mode = 0;
    float *T32 = nullptr;          // mode 2: FP32 working copy of T (total elements)
    long fp32_solves = 0;          // blocks given the FP32 eigensolve
    static constexpr double kFp32AbsTol = 3e-6, kFp32GapTol = 3e-5;
    long calls = 0, since_reset = 0;
    double abs_tol = 1e-14, gap_tol = 1e-13;

    // K-split tile list: the tiles of blocks of kSplitMinDim rows or more cut
    // into S parts (tile word: bits 4-7 part, 8-11 S, 12+ group), the others
    // as they are
    static std::vector<int4> split_tiles(const std::vector<int> &d, const std::vector<int4> &L, int S,
                                         int &groups) {
        std::vector<int4> out;
        groups = 0;
        for (const int4 &t : L) {
            if (S < 2 || d[t.x] < kSplitMinDim || groups >= (1 << 19)) {
                out.push_back(t);
                continue;
            }
            for (int q = 0; q < S; q++)
                out.push_back(make_int4(t.x, t.y, t.z, (t.w & 1) | (q << 4) | (S << 8) | (groups << 12)));
            groups++;
        }
        return out;
    }

    // The split autotuner: for the full and the symmetric tile list, the part
    // count S in {1, 2, kGemmMaxSplit} whose GEMM launch over every block is
    // fastest on this GPU (CUDA events, one warm-up and three timed launches
    // each, on the zeroed work arrays, when the plan is built).  The launches
    // are the per-iteration products W = Us Vt^T (full list) and
    // T = Vt W (symmetric list).
    void tune_split(const std::vector<int> &d, const std::vector<int4> &tl, const std::vector<int4> &stl) {
        using namespace v2b;
        int groups = 0;
        split_tiles(d, tl, 2, groups);
        split_ws = dalloc<double>((size_t)std::max(groups, 1) * kGemmMaxSplit * kGemmTile * kGemmTile);
        split_cnt = dalloc<int>(std::max(groups, 1));
        V2B_CK(cudaMemset(split_cnt, 0, std::max(groups, 1) * sizeof(int)));
        for (double *b : {Vt, Us, W, T}) V2B_CK(cudaMemset(b, 0, total * sizeof(double)));
        // the uploads and fills above ran on the legacy stream, the timed
        // launches run on a non-blocking one
        V2B_CK(cudaDeviceSynchronize());
        cudaStream_t s = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        V2B_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        V2B_CK(cudaEventCreate(&e0));
        V2B_CK(cudaEventCreate(&e1));
        int4 *buf = dalloc<int4>(std::max<size_t>(1, (size_t)kGemmMaxSplit * std::max(tl.size(), stl.size())));
        auto pick = [&](const std::vector<int4> &L, bool sym, int &n_out) {
            int best_s = 1;
            float best = 0.0f;
            for (int S : {1, 2, kGemmMaxSplit}) {
                int g = 0;
                const std::vector<int4> k = split_tiles(d, L, S, g);
                if (k.empty()) break;
                V2B_CK(cudaMemcpy(buf, k.data(), k.size() * sizeof(int4), cudaMemcpyHostToDevice));
                float ms = 0.0f;
                for (int rep = 0; rep < 4; rep++) {
                    if (rep == 1) V2B_CK(cudaEventRecord(e0, s));
                    if (sym)
                        V2B_CK(launch_gemm_tiles(kGemmNNStore, (int)k.size(), s, Vt, W, T, buf, boff, bdim, nullptr,
                                                 Us, 0.0, nullptr, nullptr, nullptr, orth, gemm_sched, split_ws,
                                                 split_cnt));
                    else
                        V2B_CK(launch_gemm_tiles(kGemmNTStore, (int)k.size(), s, Us, Vt, W, buf, boff, bdim, nullptr,
                                                 Us, 0.0, nullptr, nullptr, nullptr, orth, gemm_sched, split_ws,
                                                 split_cnt));
                }
                V2B_CK(cudaEventRecord(e1, s));
                V2B_CK(cudaEventSynchronize(e1));
                V2B_CK(cudaEventElapsedTime(&ms, e0, e1));
                if (S == 1 || ms < best) {
                    best = ms;
                    best_s = S;
                }
            }
            int g = 0;
            const std::vector<int4> k = split_tiles(d, L, best_s, g);
            n_out = (int)k.size();
            int4 *dev = dalloc<int4>(std::max(n_out, 1));
            if (n_out) V2B_CK(cudaMemcpy(dev, k.data(), n_out * sizeof(int4), cudaMemcpyHostToDevice));
            return std::make_pair(dev, best_s);
        };
        auto full = pick(tl, false, nktiles);
        auto upper = pick(stl, true, nkstiles);
        ktiles = full.first;
        kstiles = upper.first;
        split_full = full.second;
        split_sym = upper.second;
        V2B_CK(cudaDeviceSynchronize());   // the chosen lists' uploads complete before any launch
        cudaFree(buf);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(s);
    }

    void build(const std::vector<int> &d) {
        dims = d;
        nblk = (int)d.size();
        h_off.assign(nblk, 0);
        h_roff_small.assign(nblk, -1);
        h_roff_big.assign(nblk, -1);
        std::vector<int4> tl;
        std::vector<int> rb_host(nblk, 0);
        int64_t o = 0, ro = 0, rb = 0, rows = 0;
        smem = 0;
        int maxn = 0;
        for (int i = 0; i < nblk; i++) {
            if (d[i] < 0) throw std::invalid_argument("negative block dimension");
            h_off[i] = o;
            rb_host[i] = (int)rows;
            rows += d[i];
            maxn = std::max(maxn, d[i]);
            const int nt = (d[i] + v2b::kGemmTile - 1) / v2b::kGemmTile;
            for (int a = 0; a < nt; a++)
                for (int b = 0; b < nt; b++) tl.push_back(make_int4(i, a, b, 0));
            if (d[i] <= v2b::kJacobiMaxDim) {
                const int np = d[i] + (d[i] & 1);
                h_roff_small[i] = ro;
                nsmall++;
                // rotation record (max_sweeps x steps x pairs) + per-step counts
                ro += (int64_t)max_sweeps * std::max(np - 1, 0) * (np / 2) +
                      ((int64_t)max_sweeps * std::max(np - 1, 0) + 3) / 4 + 1;
                smem = std::max(smem, v2b::jacobi_smem_bytes(d[i]));
            } else {
                h_roff_big[i] = rb;
                nbig++;
                rb += v2b::big_record_slots(d[i], kBigSweeps);
                max_big = std::max(max_big, d[i]);
            }
            o += (int64_t)d[i] * d[i];
        }
        total = o;
        rows_total = rows;
        // longest K first: the persistent GEMM grid takes tiles in this order
        std::stable_sort(tl.begin(), tl.end(), [&](const int4 &a, const int4 &b) { return d[a.x] > d[b.x]; });
        ntiles = (int)tl.size();
        std::vector<int4> stl;
        for (const int4 &t : tl)
            if (t.y <= t.z) stl.push_back(make_int4(t.x, t.y, t.z, t.y < t.z ? 1 : 0));
        nstiles = (int)stl.size();
        stiles = dalloc<int4>(std::max(nstiles, 1));
        if (nstiles) V2B_CK(cudaMemcpy(stiles, stl.data(), nstiles * sizeof(int4), cudaMemcpyHostToDevice));
        boff = dalloc<int64_t>(nblk);
        gemm_sched = dalloc<int>(2);
        V2B_CK(cudaMemset(gemm_sched, 0, 2 * sizeof(int)));
        bdim = dalloc<int>(nblk);
        counters = dalloc<int>(4);
        tiles = dalloc<int4>(std::max(ntiles, 1));
        for (double **b : {&Vt, &Vt2, &Us, &W, &T, &P}) *b = dalloc<double>(total);
        V2B_CK(cudaMemcpy(boff, h_off.data(), nblk * 8, cudaMemcpyHostToDevice));
        V2B_CK(cudaMemcpy(bdim, d.data(), nblk * 4, cudaMemcpyHostToDevice));
        V2B_CK(cudaMemset(counters, 0, 16));
        if (ntiles) V2B_CK(cudaMemcpy(tiles, tl.data(), ntiles * sizeof(int4), cudaMemcpyHostToDevice));
        tune_split(d, tl, stl);
        if (nsmall) rot = dalloc<double2>(ro);
        if (smem)
            V2B_CK(v2b::raise_dynamic_smem((const void *)v2b::jacobi_warm_kernel, (int)smem));
        if (nbig) {
            rec_b = dalloc<double2>(rb);
            norm_b = dalloc<double>((size_t)nbig * v2b::kBigCluster);
        }
        sub_boff = dalloc<int64_t>(nblk);
        sub_roff = dalloc<int64_t>(nblk);
        sub_bdim = dalloc<int>(nblk);
        sub32_boff = dalloc<int64_t>(nblk);
        sub32_roff = dalloc<int64_t>(nblk);
        sub32_bdim = dalloc<int>(nblk);
        V2B_CK(cudaMallocHost(&h_sub, std::max(nblk, 1) * 3 * sizeof(int64_t)));
        // refinement
        bstate = dalloc<int>(nblk);
        orth = dalloc<unsigned long long>(nblk);
        bnorm = dalloc<double>(nblk);
        norm_part = dalloc<double>((size_t)nblk * v2b::kClassifySplit);
        cls_counts = dalloc<int>(3 * (size_t)nblk);
        done_stamp = dalloc<int>(nblk);
        V2B_CK(cudaMemset(cls_counts, 0, 3 * sizeof(int) * nblk));
        V2B_CK(cudaMemset(done_stamp, 0xff, sizeof(int) * nblk));
        Vsave = dalloc<double>(total);
        Tsave = dalloc<double>(total);
        V2B_CK(cudaMallocHost(&h_bstate_up, std::max(nblk, 1) * sizeof(int)));
        V2B_CK(cudaHostAlloc(&h_state, std::max(nblk, 1) * 3 * sizeof(int), cudaHostAllocMapped));
        h_nbad = h_state + nblk;
        h_nedge = h_nbad + nblk;
        V2B_CK(cudaHostAlloc(&h_edges, std::max<size_t>(nblk, 1) * v2b::kRefineEdgeCap * sizeof(int2),
                             cudaHostAllocMapped));
        V2B_CK(cudaHostGetDevicePointer((void **)&d_state, h_state, 0));
        d_nbad = d_state + nblk;
        d_nedge = d_nbad + nblk;
        V2B_CK(cudaHostGetDevicePointer((void **)&d_edges, h_edges, 0));
        rowbase = dalloc<int>(nblk);
        lam = dalloc<double>(rows_total);
        Qt = dalloc<double>(total);   // sum of k^2 over the clusters of a block is at most n^2
        Tc = dalloc<double>(total);
        Pc = dalloc<double>(total);
        V2B_CK(cudaMemcpy(rowbase, rb_host.data(), nblk * 4, cudaMemcpyHostToDevice));
        classify_smem = (size_t)maxn * sizeof(double);
        if (classify_smem > 48 * 1024)
            V2B_CK(v2b::raise_dynamic_smem((const void *)v2b::refine_classify_kernel, (int)classify_smem));
        const int kc = v2b::kRefineSmallCluster;
        V2B_CK(v2b::raise_dynamic_smem((const void *)v2b::cluster_eig_kernel, (int)(2 * kc * (kc + 1) * sizeof(double))));
        V2B_CK(v2b::raise_dynamic_smem((const void *)v2b::bj_apply_kernel, (int)(3 * kc * (kc + 1) * sizeof(double))));
        // clusters of kRefineSmallCluster+1 .. kJacobiMaxDim rows use jacobi_warm_kernel
        mid_smem = v2b::jacobi_smem_bytes(v2b::kJacobiMaxDim);
        V2B_CK(v2b::raise_dynamic_smem((const void *)v2b::jacobi_warm_kernel, (int)std::max(smem, mid_smem)));
        build_block_jacobi();
        V2B_CK(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
        fresh = true;
        built = true;
    }
    void release() {
        if (!built) return;
        for (auto e : pev) cudaEventDestroy(e);
        pev.clear();
        if (staged) cudaEventDestroy(staged);
        staged = nullptr;
        staged_pending = false;
        for (void *q : {(void *)boff, (void *)rot_off, (void *)bdim, (void *)counters, (void *)tiles, (void *)stiles,
                        (void *)ktiles, (void *)kstiles, (void *)split_ws, (void *)split_cnt, (void *)gemm_sched, (void *)rot, (void *)Vt, (void *)Vt2, (void *)Us, (void *)W, (void *)T,
                        (void *)P, (void *)rec_b, (void *)norm_b, (void *)sub_boff, (void *)sub_roff,
                        (void *)sub_bdim, (void *)bstate, (void *)orth, (void *)bnorm, (void *)norm_part,
                        (void *)cls_counts, (void *)done_stamp, (void *)Vsave,
                        (void *)Tsave, (void *)arena, (void *)crec, (void *)cnorm, (void *)Tc,
                        (void *)Pc, (void *)bj_dev, (void *)bj_on,
                        (void *)rowbase, (void *)lam, (void *)Qt, (void *)sub32_boff, (void *)sub32_roff,
                        (void *)sub32_bdim, (void *)T32})
            cudaFree(q);
        T32 = nullptr;
        for (void *q : {(void *)h_sub, (void *)h_bstate_up, (void *)h_state, (void *)h_edges,
                        (void *)h_arena, (void *)h_bjon})
            if (q) cudaFreeHost(q);
        built = false;
    }

    // sym: the product is symmetric (Vt W with W = Us Vt^T, Vt^T P Vt, Vt Vt^T):
    // the upper tiles are computed and mirrored
    void gemm(v2b::GemmVariant v, const double *A, const double *B, double *C, const double *Cin,
              double inv_mu, double *x, double *z, cudaStream_t s, long &launches,
              const int *only_work = nullptr, bool sym = false) {
        ph_begin(0, s);
        const int nt = sym ? (split_k ? nkstiles : nstiles) : (split_k ? nktiles : ntiles);
        const int4 *tl = sym ? (split_k ? kstiles : stiles) : (split_k ? ktiles : tiles);
        V2B_CK(v2b::launch_gemm_tiles(v, nt, s, A, B, C, tl, boff, bdim, Cin, Us, inv_mu, x, z, only_work, orth,
                                      gemm_sched, split_ws, split_cnt));
        ph_end(s);
        launches++;
    }

    // forget the eigenvector basis: the next projection starts from V = I
    // (and the re-orthonormalisation schedule restarts, so solves repeat exactly)
    void reset() {
        fresh = true;
        since_reset = 0;
    }

    // connected components of one block's recorded non-separable pairs
    void clusters_of(int b, std::vector<std::vector<int>> &out) const {
        const int n = dims[b];
        const int ne = h_nedge[b];
        std::vector<int> parent(n);
        for (int i = 0; i < n; i++) parent[i] = i;
        auto find = [&](int a) {
            while (parent[a] != a) {
                parent[a] = parent[parent[a]];
                a = parent[a];
            }
            return a;
        };
        const volatile int2 *eb = h_edges + (int64_t)b * v2b::kRefineEdgeCap;
        std::vector<char> touched(n, 0);
        for (int e = 0; e < ne; e++) {
            const int i = eb[e].x, j = eb[e].y;
            if (i < 0 || j < 0 || i >= n || j >= n) throw Failure(V2B_INTERNAL, "bad cluster edge");
            touched[i] = touched[j] = 1;
            const int ri = find(i), rj = find(j);
            if (ri != rj) parent[std::max(ri, rj)] = std::min(ri, rj);
        }
        std::vector<int> id(n, -1);
        for (int i = 0; i < n; i++) {
            if (!touched[i]) continue;
            const int r = find(i);
            if (id[r] < 0) {
                id[r] = (int)out.size();
                out.emplace_back();
            }
            out[id[r]].push_back(i);   // ascending: rows are visited in order
        }
    }

    // Round-robin pairing of the kBJGroup-row groups of each block (the
    // circle method over an even number of groups, a padding group when the
    // count is odd): one sweep of ng_even - 1 steps meets every pair of groups
    // once.  A step's pairs are disjoint and cover the block, so each step
    // runs kBJInnerSweeps Jacobi sweeps on every paired 2 x kBJGroup sub-block
    // (cluster_eig_kernel) and applies all rotations at once, in place, tile
    // by tile (bj_apply_kernel).
    void build_block_jacobi() {
        using namespace v2b;
        bj_nsteps.assign(nblk, 0);
        int S = 0;
        std::vector<int> ng(nblk, 0);
        for (int b = 0; b < nblk; b++) {
            if (dims[b] < kRefineMinDim) continue;
            ng[b] = (dims[b] + kBJGroup - 1) / kBJGroup;
            const int ge = ng[b] + (ng[b] & 1);
            bj_nsteps[b] = std::max(ge - 1, 1);
            S = std::max(S, bj_nsteps[b]);
        }
        std::vector<unsigned char> buf;
        auto sect = [&](const void *src, size_t bytes) {
            const size_t o = buf.size();
            buf.resize(o + ((bytes + 15) & ~(size_t)15));
            if (bytes) std::memcpy(buf.data() + o, src, bytes);
            return o;
        };
        bj_steps.assign(S, BJStep());
        for (int st = 0; st < S; st++) {
            std::vector<ClusterJob> jl;
            std::vector<int> ml;
            std::vector<int4> tl;
            int qoff = 0;
            for (int b = 0; b < nblk; b++) {
                if (st >= bj_nsteps[b]) continue;
                const int n = dims[b], ge = ng[b] + (ng[b] & 1);
                const int first = (int)jl.size();
                for (int kk = 0; kk < std::max(ge / 2, 1); kk++) {
                    int ga = 0, gb = 1;
                    if (ge >= 2) {
                        const int m1 = ge - 1;
                        int a, c;
                        if (kk == 0) {
                            a = m1;
                            c = st;
                        } else {
                            a = (st + kk) % m1;
                            c = (st - kk + m1) % m1;
                        }
                        ga = std::min(a, c);
                        gb = std::max(a, c);
                    }
                    ClusterJob j;
                    j.blk = b;
                    j.moff = (int)ml.size();
                    j.qoff = qoff;
                    for (int g : {ga, gb}) {
                        if (g >= ng[b]) continue;   // the padding group
                        for (int r = g * kBJGroup; r < std::min(n, (g + 1) * kBJGroup); r++) ml.push_back(r);
                    }
                    j.k = (int)ml.size() - j.moff;
                    if (j.k == 0) continue;
                    qoff += j.k * j.k;
                    jl.push_back(j);
                }
                // every row of the block is in exactly one job of this step
                const int last = (int)jl.size(), ntc = (n + 63) / 64;
                for (int I = first; I < last; I++) {
                    for (int J = first; J < last; J++) tl.push_back(make_int4(I, J, 0, 0));
                    for (int t = 0; t < ntc; t++) tl.push_back(make_int4(I, t, 1, 0));
                }
            }
            BJStep &bs = bj_steps[st];
            bs.njobs = (int)jl.size();
            bs.ntiles = (int)tl.size();
            bs.o_jobs = sect(jl.data(), jl.size() * sizeof(ClusterJob));
            bs.o_mem = sect(ml.data(), ml.size() * 4);
            bs.o_tiles = sect(tl.data(), tl.size() * 16);
        }
        bj_dev = dalloc<unsigned char>(std::max<size_t>(buf.size(), 16));
        if (!buf.empty()) V2B_CK(cudaMemcpy(bj_dev, buf.data(), buf.size(), cudaMemcpyHostToDevice));
        bj_on = dalloc<int>(nblk);
        V2B_CK(cudaMallocHost(&h_bjon, std::max(nblk, 1) * sizeof(int)));
    }

    // one block-Jacobi sweep of the blocks with st == kStBlockJacobi
    void block_jacobi_sweep(const std::vector<int> &st, cudaStream_t s, long &launches) {
        using namespace v2b;
        int S = 0;
        for (int b = 0; b < nblk; b++) {
            h_bjon[b] = st[b] == kStBlockJacobi;
            if (h_bjon[b]) S = std::max(S, bj_nsteps[b]);
        }
        if (S == 0) return;
        V2B_CK(cudaMemcpyAsync(bj_on, h_bjon, nblk * sizeof(int), cudaMemcpyHostToDevice, s));
        refine_bj_sweeps++;
        const int kc = kRefineSmallCluster;
        for (int i = 0; i < S; i++) {
            const BJStep &bs = bj_steps[i];
            if (bs.njobs == 0) continue;
            const ClusterJob *jobs = (const ClusterJob *)(bj_dev + bs.o_jobs);
            const int *mem = (const int *)(bj_dev + bs.o_mem);
            cluster_eig_kernel<<<bs.njobs, 256, 2 * kc * (kc + 1) * sizeof(double), s>>>(T, boff, bdim, jobs,
                                                                                      mem, Qt, lam, bj_on,
                                                                                      kBJInnerSweeps);
            bj_apply_kernel<<<bs.ntiles, 256, 3 * kc * (kc + 1) * sizeof(double), s>>>(
                T, Vt, boff, bdim, jobs, mem, Qt, (const int4 *)(bj_dev + bs.o_tiles), bj_on);
            V2B_CK(cudaGetLastError());
            launches += 2;
        }
    }

    // grow-only device buffers of the cluster pass (called with the stream idle)
    void ensure_arena(size_t bytes) {
        if (bytes <= arena_bytes) return;
        bytes = std::max(bytes, arena_bytes * 2);
        if (arena) cudaFree(arena);
        if (h_arena) cudaFreeHost(h_arena);
        arena = nullptr;
        h_arena = nullptr;
        arena_bytes = 0;
        arena = dalloc<unsigned char>(bytes);
        V2B_CK(cudaMallocHost(&h_arena, bytes));
        arena_bytes = bytes;
    }
    void ensure_crec(int64_t slots, int nbig_jobs) {
        if (slots > crec_slots) {
            if (crec) cudaFree(crec);
            crec = nullptr;
            crec = dalloc<double2>(slots);
            crec_slots = slots;
        }
        if (nbig_jobs > cnorm_n) {
            if (cnorm) cudaFree(cnorm);
            cnorm = nullptr;
            cnorm = dalloc<double>((size_t)nbig_jobs * v2b::kBigCluster);
            cnorm_n = nbig_jobs;
        }
    }

    void upload_states(cudaStream_t s, const std::vector<int> &st) {
        std::copy(st.begin(), st.end(), h_bstate_up);
        V2B_CK(cudaMemcpyAsync(bstate, h_bstate_up, nblk * sizeof(int), cudaMemcpyHostToDevice, s));
    }

    // Diagonalise every cluster exactly and apply the rotation G (identity
    // outside the clusters): T <- G T G^T, Vt <- G Vt.  Jobs are ordered by
    // size class: up to kRefineSmallCluster rows (cluster_eig_kernel), up to
    // kJacobiMaxDim (jacobi_warm_kernel on a compact copy), larger
    // (jacobi_big_kernel on a compact copy).
    void cluster_pass(const std::vector<std::vector<int>> &members, const std::vector<int> &jblk,
                      cudaStream_t s, long &launches) {
        using namespace v2b;
        const int nj_all = (int)members.size();
        std::vector<int> order(nj_all);
        for (int q = 0; q < nj_all; q++) order[q] = q;
        auto cls = [&](int q) {
            const int k = (int)members[q].size();
            return k <= kRefineSmallCluster ? 0 : (k <= kJacobiMaxDim ? 1 : 2);
        };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cls(a) < cls(b); });
        std::vector<ClusterJob> jl(nj_all);
        std::vector<int> ml, rc((size_t)rows_total, -1), jlist;
        std::vector<int4> trows, tcols, tcommit;
        std::vector<int64_t> cboff, croff;
        std::vector<int> cdim;
        std::vector<int> base(nblk, 0);
        for (int b = 1; b < nblk; b++) base[b] = base[b - 1] + dims[b - 1];
        int64_t qoff = 0, roff = 0;
        int nsm = 0, nmid = 0, nbg = 0, kmax_big = 0;
        for (int q = 0; q < nj_all; q++) {
            const auto &c = members[order[q]];
            ClusterJob &j = jl[q];
            j.blk = jblk[order[q]];
            j.k = (int)c.size();
            j.moff = (int)ml.size();
            j.qoff = (int)qoff;
            qoff += (int64_t)j.k * j.k;
            for (int r : c) {
                rc[base[j.blk] + r] = q;
                ml.push_back(r);
            }
            const int n = dims[j.blk];
            const int nti = (j.k + 31) / 32, ntc = (n + 63) / 64;
            for (int a = 0; a < nti; a++)
                for (int b = 0; b < ntc; b++) trows.push_back(make_int4(q, a, b, 0));
            for (int a = 0; a < ntc; a++)
                for (int b = 0; b < nti; b++) tcols.push_back(make_int4(q, a, b, 0));
            for (int a = 0; a < ntc; a++) tcommit.push_back(make_int4(q, a, 0, 0));
            const int kind = cls(order[q]);
            if (kind == 0) {
                nsm++;
                continue;
            }
            jlist.push_back(q);
            cboff.push_back(j.qoff);
            cdim.push_back(j.k);
            croff.push_back(roff);
            if (kind == 1) {
                const int np = j.k + (j.k & 1);
                roff += (int64_t)max_sweeps * (np - 1) * (np / 2) + ((int64_t)max_sweeps * (np - 1) + 3) / 4 + 1;
                nmid++;
            } else {
                roff += big_record_slots(j.k, kBigSweeps);
                kmax_big = std::max(kmax_big, j.k);
                nbg++;
            }
        }
        refine_clusters += nj_all;
        refine_large_clusters += nmid + nbg;
        // pack the lists into the arena (16-byte aligned sections)
        size_t off = 0;
        auto sect = [&](size_t bytes) {
            const size_t o = off;
            off += (bytes + 15) & ~(size_t)15;
            return o;
        };
        const size_t o_jobs = sect(jl.size() * sizeof(ClusterJob)), o_mem = sect(ml.size() * 4),
                     o_rc = sect(rc.size() * 4), o_tr = sect(trows.size() * 16),
                     o_tc = sect(tcols.size() * 16), o_tm = sect(tcommit.size() * 16),
                     o_jl = sect(jlist.size() * 4), o_cb = sect(cboff.size() * 8),
                     o_cd = sect(cdim.size() * 4), o_cr = sect(croff.size() * 8);
        ensure_arena(off);
        ensure_crec(std::max<int64_t>(roff, 1), nbg);
        auto put = [&](size_t o, const void *src, size_t bytes) {
            if (bytes) std::memcpy(h_arena + o, src, bytes);
        };
        put(o_jobs, jl.data(), jl.size() * sizeof(ClusterJob));
        put(o_mem, ml.data(), ml.size() * 4);
        put(o_rc, rc.data(), rc.size() * 4);
        put(o_tr, trows.data(), trows.size() * 16);
        put(o_tc, tcols.data(), tcols.size() * 16);
        put(o_tm, tcommit.data(), tcommit.size() * 16);
        put(o_jl, jlist.data(), jlist.size() * 4);
        put(o_cb, cboff.data(), cboff.size() * 8);
        put(o_cd, cdim.data(), cdim.size() * 4);
        put(o_cr, croff.data(), croff.size() * 8);
        V2B_CK(cudaMemcpyAsync(arena, h_arena, off, cudaMemcpyHostToDevice, s));
        const ClusterJob *d_jobs = (const ClusterJob *)(arena + o_jobs);
        const int *d_mem = (const int *)(arena + o_mem), *d_rc = (const int *)(arena + o_rc);
        const int4 *d_tr = (const int4 *)(arena + o_tr), *d_tc = (const int4 *)(arena + o_tc),
                   *d_tm = (const int4 *)(arena + o_tm);
        const int *d_jl = (const int *)(arena + o_jl);
        const int64_t *d_cb = (const int64_t *)(arena + o_cb), *d_cr = (const int64_t *)(arena + o_cr);
        const int *d_cd = (const int *)(arena + o_cd);
        if (nsm) {
            const int kc = kRefineSmallCluster;
            cluster_eig_kernel<<<nsm, 256, 2 * kc * (kc + 1) * sizeof(double), s>>>(T, boff, bdim, d_jobs,
                                                                                 d_mem, Qt, lam, nullptr,
                                                                                 kClusterSweeps);
            V2B_CK(cudaGetLastError());
            launches++;
        }
        if (nmid + nbg) {
            cluster_gather_kernel<<<dim3(nmid + nbg, 16), 256, 0, s>>>(T, boff, bdim, d_jobs, d_mem, d_jl,
                                                                       Tc, Qt);
            V2B_CK(cudaGetLastError());
            launches++;
            // gap test off (gap_tol 0): the cluster is diagonalised to 1e-15 of its norm
            if (nmid) {
                jacobi_warm_kernel<<<nmid, kJacobiThreads, mid_smem, s>>>(
                    Tc, Pc, Qt, d_cb, d_cd, crec, d_cr, max_sweeps, 1e-15, 0.0, counters, counters + 1, 1);
                V2B_CK(cudaGetLastError());
                launches++;
            }
            if (nbg) {
                BigJacobiArgs a;
                a.T = Tc; a.P = Pc; a.Vt = Qt; a.boff = d_cb + nmid; a.bdim = d_cd + nmid;
                a.rot = crec; a.roff = d_cr + nmid; a.max_sweeps = kBigSweeps; a.norm_part = cnorm;
                a.abs_tol = 1e-15; a.gap_tol = 0.0; a.counters = counters + 2;
                const size_t alist_bytes = (size_t)((kmax_big + 1) / 2 + 1) * sizeof(int);
                jacobi_big_kernel<<<nbg * kBigCluster, kBigThreads, alist_bytes, s>>>(a);
                V2B_CK(cudaGetLastError());
                launches++;
            }
            cluster_lam_kernel<<<std::min(nmid + nbg, 148), 256, 0, s>>>(d_jobs, d_jl, nmid + nbg, Pc, Tc,
                                                                          nmid, lam);
            V2B_CK(cudaGetLastError());
            launches++;
        }
        cluster_rows_kernel<<<(int)trows.size(), 256, 0, s>>>(T, Vt, W, Vt2, boff, bdim, d_jobs, d_mem, Qt,
                                                               d_tr, nullptr);
        cluster_cols_kernel<<<(int)tcols.size(), 256, 0, s>>>(T, W, P, boff, bdim, d_jobs, d_mem, d_rc,
                                                               rowbase, Qt, lam, d_tc, nullptr);
        cluster_commit_kernel<<<(int)tcommit.size(), 256, 0, s>>>(T, W, P, Vt, Vt2, boff, bdim, d_jobs,
                                                                   d_mem, d_rc, rowbase, d_tm, nullptr);
        V2B_CK(cudaGetLastError());
        launches += 3;
    }

    // The refinement passes; leaves every block Done or Jacobi.  Per pass,
    // after the acceptance test, a block in Newton mode (kStWork) takes the
    // cluster diagonalisation and one Newton step; it changes to block-Jacobi
    // mode (kStBlockJacobi) when it records too many non-separable pairs, has
    // a cluster above kRefineSmallCluster rows or runs out of Newton passes,
    // restarting from the call's saved basis and T (block-Jacobi keeps Vt
    // orthonormal by construction, the Newton steps only to the accepted
    // tolerance).  A block in block-Jacobi mode takes one sweep per pass, and
    // after kBJMaxSweeps goes to the selective Jacobi kernels.  In the mixed
    // mode a block above kJacobiMaxDim rows takes the FP32 eigensolve before
    // block-Jacobi; from then on its clusters of every size take the cluster
    // kernels, and a later restart begins from the FP32-solved basis.
    void refine(std::vector<int> &st, cudaStream_t s, long &launches) {
        using namespace v2b;
        bool any = false;
        for (int b = 0; b < nblk; b++) any = any || st[b] == kStWork || st[b] == kStBlockJacobi || st[b] == kStFp32;
        if (!any) return;
        V2B_CK(cudaMemsetAsync(orth, 0, nblk * sizeof(unsigned long long), s));
        V2B_CK(cudaMemcpyAsync(Vsave, Vt, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
        V2B_CK(cudaMemcpyAsync(Tsave, T, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
        // ||T||_F = ||sym(U)||_F for an orthonormal Vt: the tests use the block norms of Us
        ph_begin(1, s);
        block_norm_kernel<<<dim3(nblk, kClassifySplit), 256, 0, s>>>(Us, boff, bdim, norm_part);
        ph_end(s);
        V2B_CK(cudaGetLastError());
        launches++;
        std::vector<char> changed(nblk, 0);
        std::vector<int> newton(nblk, 0), sweeps(nblk, 0);
        auto restore = [&](int b) {
            if (!changed[b]) return;
            const size_t bytes = (size_t)dims[b] * dims[b] * sizeof(double);
            V2B_CK(cudaMemcpyAsync(Vt + h_off[b], Vsave + h_off[b], bytes, cudaMemcpyDeviceToDevice, s));
            V2B_CK(cudaMemcpyAsync(T + h_off[b], Tsave + h_off[b], bytes, cudaMemcpyDeviceToDevice, s));
            V2B_CK(cudaMemsetAsync(orth + b, 0, sizeof(unsigned long long), s));
            changed[b] = 0;
        };
        // fp32_done: the block took the FP32 eigensolve in this call; snap:
        // its FP64 T in the new basis is computed at the top of the next
        // pass, and the basis and T are then kept as the block's restart
        // point in place of the call's saved ones
        std::vector<char> fp32_done(nblk, 0), snap(nblk, 0);
        auto to_block_jacobi = [&](int b) {
            restore(b);
            st[b] = (mode == 2 && !fp32_done[b] && dims[b] > kJacobiMaxDim) ? kStFp32 : kStBlockJacobi;
        };
        for (int pass = 0;; pass++) {
            if (pass > 0) {   // T of the blocks that took a Newton step (bstate == kStWork)
                bool nw = false;
                for (int b = 0; b < nblk; b++) nw = nw || st[b] == kStWork;
                if (nw) {
                    gemm(kGemmNTStore, Us, Vt, W, nullptr, 0.0, nullptr, nullptr, s, launches, bstate);
                    gemm(kGemmNNStore, Vt, W, T, nullptr, 0.0, nullptr, nullptr, s, launches, bstate, true);
                }
                for (int b = 0; b < nblk; b++) {
                    if (!snap[b]) continue;
                    const size_t bytes = (size_t)dims[b] * dims[b] * sizeof(double);
                    V2B_CK(cudaMemcpyAsync(Vsave + h_off[b], Vt + h_off[b], bytes, cudaMemcpyDeviceToDevice, s));
                    V2B_CK(cudaMemcpyAsync(Tsave + h_off[b], T + h_off[b], bytes, cudaMemcpyDeviceToDevice, s));
                    snap[b] = 0;
                    changed[b] = 0;
                }
            }
            ++stamp;
            ph_begin(1, s);
            refine_classify_kernel<<<dim3(nblk, kClassifySplit), kRefineThreads, classify_smem, s>>>(
                T, boff, bdim, bstate, orth, norm_part, gap_tol, abs_tol, bnorm, cls_counts, done_stamp,
                stamp, d_state, d_nbad, d_nedge, d_edges);
            write_p_kernel<<<ntiles, 256, 0, s>>>(T, P, tiles, boff, bdim, done_stamp, stamp);
            ph_end(s);
            V2B_CK(cudaGetLastError());
            launches += 2;
            V2B_CK(cudaStreamSynchronize(s));
            refine_passes++;
            std::vector<std::vector<int>> members;   // clusters of the Newton-mode blocks
            std::vector<int> jblk;
            int nwork = 0, nbj = 0;
            for (int b = 0; b < nblk; b++) {
                if (st[b] != kStWork && st[b] != kStBlockJacobi) continue;
                if (h_state[b] == kStDone) {
                    st[b] = kStDone;
                    refine_accepted++;
                    continue;
                }
                if (st[b] == kStBlockJacobi) {
                    if (sweeps[b] >= kBJMaxSweeps) {
                        fb_passes++;
                        st[b] = kStJacobi;
                    } else {
                        nbj++;
                    }
                    continue;
                }
                // Newton mode
                if (newton[b] >= kRefinePasses) {
                    to_block_jacobi(b);
                    nbj++;
                    continue;
                }
                if (h_nedge[b] > kRefineEdgeCap) {
                    fb_edges++;
                    to_block_jacobi(b);
                    nbj++;
                    continue;
                }
                std::vector<std::vector<int>> cl;
                clusters_of(b, cl);
                size_t kmax = 0;
                for (const auto &c : cl) kmax = std::max(kmax, c.size());
                // after the FP32 eigensolve the clusters are those of an
                // almost diagonal T: any size goes to the cluster kernels
                if ((int)kmax > kRefineSmallCluster && !fp32_done[b]) {
                    refine_large_clusters++;
                    to_block_jacobi(b);
                    nbj++;
                    continue;
                }
                changed[b] = 1;
                newton[b]++;
                nwork++;
                for (auto &c : cl) {
                    members.push_back(std::move(c));
                    jblk.push_back(b);
                }
            }
            int nfp = 0;
            for (int b = 0; b < nblk; b++) nfp += st[b] == kStFp32;
            if (nwork == 0 && nbj == 0 && nfp == 0) break;
            upload_states(s, st);
            if (nfp) {
                // FP32 eigensolve; the next pass recomputes T in the new basis
                // (the FP64 Rayleigh-Ritz step) and tests / polishes it in FP64
                ph_begin(3, s);
                fp32_solve(st, s, launches);
                ph_end(s);
                for (int b = 0; b < nblk; b++)
                    if (st[b] == kStFp32) {
                        st[b] = kStWork;
                        fp32_done[b] = 1;
                        snap[b] = 1;
                        changed[b] = 1;
                        newton[b] = 0;
                    }
            }
            if (nbj) {
                ph_begin(3, s);
                block_jacobi_sweep(st, s, launches);
                ph_end(s);
                for (int b = 0; b < nblk; b++)
                    if (st[b] == kStBlockJacobi) sweeps[b]++;
            }
            if (nwork) {
                ph_begin(2, s);
                if (!members.empty()) cluster_pass(members, jblk, s, launches);
                newton_m_kernel<<<ntiles, 256, 0, s>>>(T, W, tiles, boff, bdim, bstate, bnorm, gap_tol,
                                                       abs_tol);
                ph_end(s);
                V2B_CK(cudaGetLastError());
                launches++;
                V2B_CK(cudaMemsetAsync(orth, 0, nblk * sizeof(unsigned long long), s));
                gemm(kGemmNNStore, W, Vt, Vt2, nullptr, 0.0, nullptr, nullptr, s, launches, bstate);
                gemm(kGemmNTNewtonSchulz, Vt2, Vt2, W, nullptr, 0.0, nullptr, nullptr, s, launches, bstate, true);
                gemm(kGemmNNStore, W, Vt2, Vt, nullptr, 0.0, nullptr, nullptr, s, launches, bstate);
            }
            if (nfp) upload_states(s, st);   // the solved blocks are Newton-mode blocks from the next pass on
        }
        upload_states(s, st);
    }

    // mode 2: FP32 selective Jacobi (jacobi_big32_kernel) on the blocks in
    // state kStFp32, each warm-started from the call's basis: T is read from
    // the FP64 T, the rotations are replayed onto Vt in FP64
    void fp32_solve(const std::vector<int> &st, cudaStream_t s, long &launches) {
        using namespace v2b;
        std::vector<int64_t> hb, hr;
        std::vector<int> hd;
        for (int b = 0; b < nblk; b++)
            if (st[b] == kStFp32) {
                hb.push_back(h_off[b]);
                hr.push_back(h_roff_big[b]);
                hd.push_back(dims[b]);
            }
        const int nb = (int)hb.size();
        if (nb == 0) return;
        if (!T32) T32 = dalloc<float>(total);
        V2B_CK(cudaMemcpyAsync(sub32_boff, hb.data(), nb * 8, cudaMemcpyHostToDevice, s));
        V2B_CK(cudaMemcpyAsync(sub32_roff, hr.data(), nb * 8, cudaMemcpyHostToDevice, s));
        V2B_CK(cudaMemcpyAsync(sub32_bdim, hd.data(), nb * 4, cudaMemcpyHostToDevice, s));
        BigJacobiArgs a;
        a.T = T; a.P = P; a.Vt = Vt; a.boff = sub32_boff; a.bdim = sub32_bdim;
        a.rot = rec_b; a.roff = sub32_roff; a.max_sweeps = kBigSweeps; a.norm_part = norm_b;
        a.abs_tol = kFp32AbsTol; a.gap_tol = kFp32GapTol; a.counters = counters + 2;
        const size_t alist_bytes = (size_t)((max_big + 1) / 2 + 1) * sizeof(int);
        jacobi_big32_kernel<<<nb * kBigCluster, kBigThreads, alist_bytes, s>>>(a, T32);
        V2B_CK(cudaGetLastError());
        // the copied lists stay valid until the kernel has read them
        V2B_CK(cudaStreamSynchronize(s));
        launches++;
        fp32_solves += nb;
    }

    // selective Jacobi on the blocks in state kStJacobi
    void jacobi(const std::vector<int> &st, cudaStream_t s, long &launches) {
        using namespace v2b;
        int ns = 0, nb = 0;
        int64_t *hb = h_sub, *hr = h_sub + nblk, *hd = h_sub + 2 * nblk;
        for (int pass = 0; pass < 2; pass++)
            for (int b = 0; b < nblk; b++) {
                if (st[b] != kStJacobi) continue;
                const bool small = h_roff_small[b] >= 0;
                if ((pass == 0) != small) continue;
                const int k = ns + nb;
                hb[k] = h_off[b];
                hr[k] = small ? h_roff_small[b] : h_roff_big[b];
                hd[k] = dims[b];
                (small ? ns : nb)++;
            }
        const int m = ns + nb;
        if (m == 0) return;
        refine_jacobi += m;
        std::vector<int> dd(m);
        for (int k = 0; k < m; k++) dd[k] = (int)hd[k];
        std::memcpy(hd, dd.data(), m * sizeof(int));
        V2B_CK(cudaMemcpyAsync(sub_boff, hb, m * 8, cudaMemcpyHostToDevice, s));
        V2B_CK(cudaMemcpyAsync(sub_roff, hr, m * 8, cudaMemcpyHostToDevice, s));
        V2B_CK(cudaMemcpyAsync(sub_bdim, hd, m * 4, cudaMemcpyHostToDevice, s));
        if (ns) {
            jacobi_warm_kernel<<<ns, kJacobiThreads, smem, s>>>(T, P, Vt, sub_boff, sub_bdim, rot, sub_roff,
                                                                max_sweeps, abs_tol, gap_tol, counters,
                                                                counters + 1);
            V2B_CK(cudaGetLastError());
            launches++;
        }
        if (nb) {
            BigJacobiArgs a;
            a.T = T; a.P = P; a.Vt = Vt; a.boff = sub_boff + ns; a.bdim = sub_bdim + ns;
            a.rot = rec_b; a.roff = sub_roff + ns; a.max_sweeps = kBigSweeps; a.norm_part = norm_b;
            a.abs_tol = abs_tol; a.gap_tol = gap_tol; a.counters = counters + 2;
            const size_t alist_bytes = (size_t)((max_big + 1) / 2 + 1) * sizeof(int);
            jacobi_big_kernel<<<nb * kBigCluster, kBigThreads, alist_bytes, s>>>(a);
            V2B_CK(cudaGetLastError());
            launches++;
        }
    }

    void project(const double *U, double mu, double *x, double *z, cudaStream_t s, long &launches) {
        using namespace v2b;
        if (nblk == 0 || ntiles == 0) return;
        const bool cold = fresh;
        if (fresh) {
            identity_blocks_kernel<<<nblk, 256, 0, s>>>(Vt, boff, bdim);
            V2B_CK(cudaGetLastError());
            launches++;
            fresh = false;
        } else if (++calls, ++since_reset % kReorthEvery == 0) {
            gemm(kGemmNTStore, Vt, Vt, W, nullptr, 0.0, nullptr, nullptr, s, launches, nullptr, true);
            half_residual_kernel<<<nblk, 256, 0, s>>>(W, T, boff, bdim);
            V2B_CK(cudaGetLastError());
            launches++;
            gemm(kGemmNNAdd, T, Vt, Vt2, Vt, 0.0, nullptr, nullptr, s, launches);
            std::swap(Vt, Vt2);
        }
        symmetrize_kernel<<<ntiles, 256, 0, s>>>(U, Us, tiles, boff, bdim);
        V2B_CK(cudaGetLastError());
        launches++;
        gemm(kGemmNTStore, Us, Vt, W, nullptr, 0.0, nullptr, nullptr, s, launches);
        gemm(kGemmNNStore, Vt, W, T, nullptr, 0.0, nullptr, nullptr, s, launches, nullptr, true);
        std::vector<int> st(nblk);
        for (int b = 0; b < nblk; b++)
            st[b] = dims[b] == 0 ? kStDone
                    : (mode == 1 || dims[b] < kRefineMinDim) ? kStJacobi
                    : !cold ? kStWork
                    : (mode == 2 && dims[b] > kJacobiMaxDim) ? kStFp32 : kStBlockJacobi;
        if (staged_pending) V2B_CK(cudaEventSynchronize(staged));
        upload_states(s, st);
        refine(st, s, launches);
        ph_begin(4, s);
        jacobi(st, s, launches);
        ph_end(s);
        V2B_CK(cudaEventRecord(staged, s));
        staged_pending = true;
        gemm(kGemmTNStore, Vt, P, W, nullptr, 0.0, nullptr, nullptr, s, launches);
        gemm(kGemmNNProject, W, Vt, nullptr, nullptr, 1.0 / mu, x, z, s, launches, nullptr, true);
    }
};

int sm_count() {
    int dev = 0, n = 0;
    V2B_CK(cudaGetDevice(&dev));
    V2B_CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

}  // namespace

void v2b::set_last_error(const std::string &msg) { g_last_error = msg; }

// ====================================================================
// device-map problem
// ====================================================================
struct v2b_problem {
    v2b::Problem prob;
    DeviceOp A, AT;
    ProjectPlan plan;
    cudaStream_t stream = nullptr;
    double *x = nullptr, *b = nullptr, *c = nullptr, *y = nullptr, *z = nullptr;
    double *Ax = nullptr, *Acz = nullptr, *ATy = nullptr, *U = nullptr;
    double *r = nullptr, *p0 = nullptr, *p1 = nullptr, *t = nullptr;
    double *y1 = nullptr, *y2 = nullptr;   // the last two dual solutions, for the CG start
    double *partials = nullptr, *cg_out = nullptr, *stats = nullptr, *stats_partials = nullptr;
    unsigned int *stats_counter = nullptr;
    v2b::GridBarrier *bar = nullptr;
    int *ibas_aa_dev = nullptr;   // n x n aa geminal numbers, for the density packing
    double *pack_layout = nullptr;   // DOCI: x in the v2RDM layout, for the density packing
    int *status = nullptr;   // [0] fatal device status, [1] projection sweeps exhausted
    double *h_readback = nullptr;   // pinned: stats[4], cg_out[2], status[2]
    int cg_grid = 0;
    double mu = 0.1;
    long launches = 0;
    long cur_oiter = 0;

    // optional per-kernel-class CUDA-event timing on the launching stream
    // classes: 0 cg_kernel, 1 spmv_AT_U, 2 jacobi_project, 3 spmv_A2, 4 stats
    static constexpr int kClasses = 5;
    bool profiling = false;
    cudaEvent_t ev[2 * kClasses] = {};
    double prof_ms[kClasses] = {};
    long prof_n[kClasses] = {};
    // CG phases, summed by the kernel's own clock: initial residual, A^T p, A t, update
    static constexpr int kCgPhases = 4;
    unsigned long long *cg_phase = nullptr;
    bool phases = false;   // profiling level 2
    void mark(int cls, int edge) {
        if (profiling) V2B_CK(cudaEventRecord(ev[2 * cls + edge], stream));
    }
    void collect() {
        if (!profiling) return;
        if (plan.built) plan.ph_collect();
        for (int k = 0; k < kClasses; k++) {
            float ms = 0.f;
            V2B_CK(cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]));
            prof_ms[k] += ms;
            prof_n[k] += 1;
        }
    }
    // level 0 off; 1 CUDA events around each kernel class; 2 also the
    // projection's phases and the CG kernel's own phase clock
    void set_profiling(int level) {
        const bool on = level > 0;
        if (on && !ev[0])
            for (auto &e : ev) V2B_CK(cudaEventCreate(&e));
        if (level > 1 && !cg_phase) cg_phase = dalloc<unsigned long long>(kCgPhases);
        if (cg_phase) V2B_CK(cudaMemset(cg_phase, 0, kCgPhases * sizeof(unsigned long long)));
        profiling = on;
        phases = level > 1;
        for (int k = 0; k < kClasses; k++) { prof_ms[k] = 0.0; prof_n[k] = 0; }
        plan.prof = level > 1;
        plan.pev_used = 0;
        for (int k = 0; k < ProjectPlan::kPhases; k++) { plan.ph_ms[k] = 0.0; plan.ph_n[k] = 0; }
    }

    ~v2b_problem() {
        if (!on_device) return;
        A.release();
        AT.release();
        plan.release();
        for (double *p : {x, b, c, y, z, Ax, Acz, ATy, U, r, p0, p1, t, y1, y2, partials, cg_out, stats,
                          stats_partials})
            cudaFree(p);
        if (cg_phase) cudaFree(cg_phase);
        if (pack_layout) cudaFree(pack_layout);
        cudaFree(stats_counter);
        cudaFree(bar);
        cudaFree(ibas_aa_dev);
        cudaFree(status);
        if (nonfinite) cudaFree(nonfinite);
        if (h_readback) cudaFreeHost(h_readback);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }

    // host operator tables, built once at creation
    v2b::PackedOperator hostA, hostAT;
    bool on_device = false;
    // a restart state (v2b_problem_set_state) that the next solve starts from
    bool resume = false;
    // v2b_problem_continue: the next solve keeps mu, y, z and the projection's
    // bases of the last device solve (libsdp's state across solve() calls)
    bool keep_state = false;
    bool solved = false;   // a device solve has run (its state can be continued)
    // polls of a CG grid-barrier wait before it gives up (a few seconds of 32 ns sleeps)
    static constexpr long long kDefaultWaitLimit = 40000000LL;
    long long wait_limit = kDefaultWaitLimit;
    unsigned long long *nonfinite = nullptr;   // nonfinite_kernel's three results
    std::vector<double> resume_y, resume_z;

    // device resources are created on first device use, so that the host-side
    // problem (sizes, b, c, guesses, operator tables) needs no GPU
    void setup() {
        if (on_device) return;
        ensure_device();
        V2B_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        A.upload(hostA);
        AT.upload(hostAT);
        const int64_t np = prob.n_primal, nd = prob.n_dual;
        x = dalloc<double>(np); c = dalloc<double>(np); z = dalloc<double>(np);
        ATy = dalloc<double>(np); U = dalloc<double>(np); t = dalloc<double>(np);
        b = dalloc<double>(nd); y = dalloc<double>(nd); Ax = dalloc<double>(nd);
        Acz = dalloc<double>(nd); r = dalloc<double>(nd); p0 = dalloc<double>(nd);
        p1 = dalloc<double>(nd);
        y1 = dalloc<double>(nd); y2 = dalloc<double>(nd);
        int per_sm = 0;
        V2B_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v2b::cg_kernel,
                                                             v2b::kCgThreads, 0));
        if (per_sm < 1) throw Failure(V2B_INTERNAL, "cg_kernel cannot be resident");
        // small problems: fewer CTAs make the grid barrier cheaper
        const int64_t rows = std::max(prob.n_primal, prob.n_dual);
        const int64_t want = (rows + (int64_t)v2b::kCgThreads - 1) / (int64_t)v2b::kCgThreads;
        cg_grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count() * per_sm));
        A.split_slices((int64_t)cg_grid * (v2b::kCgThreads / 32), hostA);
        AT.split_slices((int64_t)cg_grid * (v2b::kCgThreads / 32), hostAT);
        partials = dalloc<double>(2 * (size_t)cg_grid);
        stats_partials = dalloc<double>(4 * v2b::kStatsBlocks);
        cg_out = dalloc<double>(2);
        stats = dalloc<double>(4);
        stats_counter = dalloc<unsigned int>(1);
        bar = dalloc<v2b::GridBarrier>(1);
        status = dalloc<int>(2);
        V2B_CK(cudaMemset(stats_counter, 0, 4));
        V2B_CK(cudaMemset(status, 0, 8));
        V2B_CK(cudaMallocHost(&h_readback, 8 * sizeof(double)));
        on_device = true;
    }

    void ensure_plan() {
        if (!plan.built) plan.build(prob.dims);
    }

    int grid_for(int64_t rows, int threads) const {
        const int64_t g = (rows + threads - 1) / threads;
        return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
    }

    void Au(const double *in, double *out, cudaStream_t s) {
        v2b::spmv_kernel<<<grid_for(A.nrows, v2b::kSpmvThreads), v2b::kSpmvThreads, 0, s>>>(
            A.rp, A.ent, A.nrows, in, out, A.pal);
        V2B_CK(cudaGetLastError());
        launches++;
    }
    void ATu(const double *in, double *out, cudaStream_t s) {
        v2b::spmv_kernel<<<grid_for(AT.nrows, v2b::kSpmvThreads), v2b::kSpmvThreads, 0, s>>>(
            AT.rp, AT.ent, AT.nrows, in, out, AT.pal);
        V2B_CK(cudaGetLastError());
        launches++;
    }

    void launch_cg(double tol, int maxit) {
        V2B_CK(cudaMemsetAsync(bar, 0, sizeof(v2b::GridBarrier), stream));
        v2b::CgParams P;
        P.a_rp = A.rp; P.a_ent = A.ent; P.t_rp = AT.rp; P.t_ent = AT.ent;
        P.long_a = A.long_rows; P.long_t = AT.long_rows;
        P.n_long_a = A.n_long; P.n_long_t = AT.n_long;
        P.sa = A.sell(); P.st = AT.sell();
        P.palA = A.pal; P.palT = AT.pal;
        P.np = prob.n_primal; P.nd = prob.n_dual;
        P.Ax = Ax; P.Acz = Acz; P.b = b; P.mu = mu;
        P.y = y; P.r = r; P.p0 = p0; P.p1 = p1; P.t = t;
        P.partials = partials; P.bar = bar; P.status = status;
        P.spin_limit = wait_limit;
        P.tol = tol; P.maxit = maxit; P.out = cg_out;
        P.phase_ns = (profiling && phases) ? cg_phase : nullptr;
        void *args[] = {&P};
        V2B_CK(cudaLaunchCooperativeKernel((const void *)v2b::cg_kernel, dim3(cg_grid),
                                           dim3(v2b::kCgThreads), args, 0, stream));
        launches++;
    }

    // one boundary-point iteration; returns {iters, eps_p, eps_d, E_p, E_d}
    void iterate(const v2b_sdp_options &o, double out[5], int order) {
        const int64_t np = prob.n_primal, nd = prob.n_dual;
        mark(0, 0);
        v2b::extrapolate_y_kernel<<<grid_for(nd, 256), 256, 0, stream>>>(y, y1, y2, nd, order);
        V2B_CK(cudaGetLastError());
        launches++;
        launch_cg(o.cg_convergence, o.cg_maxiter);
        mark(0, 1);
        mark(1, 0);
        v2b::spmv_AT_U_kernel<<<grid_for(np, v2b::kSpmvThreads), v2b::kSpmvThreads, 0, stream>>>(
            AT.rp, AT.ent, np, y, x, c, mu, ATy, U, AT.pal);
        V2B_CK(cudaGetLastError());
        launches++;
        mark(1, 1);
        mark(2, 0);
        ensure_plan();
        plan.project(U, mu, x, z, stream, launches);
        mark(2, 1);
        mark(3, 0);
        v2b::spmv_A2_kernel<<<grid_for(nd, v2b::kSpmvThreads), v2b::kSpmvThreads, 0, stream>>>(
            A.rp, A.ent, nd, x, c, z, Ax, Acz, A.pal);
        V2B_CK(cudaGetLastError());
        launches++;
        mark(3, 1);
        mark(4, 0);
        v2b::stats_kernel<<<v2b::kStatsBlocks, 256, 0, stream>>>(Ax, b, ATy, z, c, x, y, np, nd,
                                                                 stats_partials, stats_counter,
                                                                 stats, status);
        V2B_CK(cudaGetLastError());
        launches++;
        mark(4, 1);
        V2B_CK(cudaMemcpyAsync(h_readback, stats, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        V2B_CK(cudaMemcpyAsync(h_readback + 4, cg_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        V2B_CK(cudaMemcpyAsync(h_readback + 6, status, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
        V2B_CK(cudaStreamSynchronize(stream));
        collect();
        const int *st = (const int *)(h_readback + 6);
        if (st[0] == V2B_DEVICE_TIMEOUT)
            throw Failure(V2B_DEVICE_TIMEOUT, "grid barrier wait gave up in cg_kernel");
        if (st[0] == V2B_NAN) {
            char msg[256];
            snprintf(msg, sizeof msg,
                     "non-finite value at outer iteration %ld: cg iterations %g |r| %g, "
                     "|Ax-b|^2 %g |ATy+z-c|^2 %g cx %g by %g, mu %g",
                     cur_oiter, h_readback[4], h_readback[5], h_readback[0], h_readback[1],
                     h_readback[2], h_readback[3], mu);
            throw Failure(V2B_NAN, msg);
        }
        out[0] = h_readback[4];
        out[1] = std::sqrt(h_readback[0]);
        out[2] = std::sqrt(h_readback[1]);
        out[3] = h_readback[2];
        out[4] = h_readback[3];
    }

    // x, b, c on the device must be finite: a NaN there would only surface
    // after a whole iteration, inside the projection
    void check_inputs_finite() {
        if (!nonfinite) nonfinite = dalloc<unsigned long long>(3);
        V2B_CK(cudaMemsetAsync(nonfinite, 0xff, 3 * sizeof(unsigned long long), stream));
        const int64_t tot = 2 * prob.n_primal + prob.n_dual;
        nonfinite_kernel<<<grid_for(tot, 256), 256, 0, stream>>>(x, prob.n_primal, b, prob.n_dual, c,
                                                                  prob.n_primal, nonfinite);
        V2B_CK(cudaGetLastError());
        launches++;
        unsigned long long first[3];
        V2B_CK(cudaMemcpyAsync(first, nonfinite, sizeof first, cudaMemcpyDeviceToHost, stream));
        V2B_CK(cudaStreamSynchronize(stream));
        const char *names[3] = {"x", "b", "c"};
        for (int k = 0; k < 3; k++)
            if (first[k] != ~0ull)
                throw Failure(V2B_NAN, std::string("non-finite value in ") + names[k] + " at index " +
                                           std::to_string(first[k]));
    }

    int solve_device(const v2b_sdp_options &o, int muf, v2b_sdp_monitor monitor, int print_level,
                     void *data, long *oiter_out, long *iiter_out, double *energy) {
        if (muf < 1) throw std::invalid_argument("mu_update_frequency must be >= 1");
        check_inputs_finite();
        const int64_t np = prob.n_primal, nd = prob.n_dual;
        ensure_plan();
        if (keep_state) {   // continue where the last device solve stopped
            keep_state = false;
        } else if (resume) {   // mu was set with the state
            plan.reset();
            V2B_CK(cudaMemcpyAsync(y, resume_y.data(), nd * 8, cudaMemcpyHostToDevice, stream));
            V2B_CK(cudaMemcpyAsync(z, resume_z.data(), np * 8, cudaMemcpyHostToDevice, stream));
            V2B_CK(cudaStreamSynchronize(stream));
            resume = false;
            std::vector<double>().swap(resume_y);
            std::vector<double>().swap(resume_z);
        } else {
            plan.reset();
            mu = 0.1;
            V2B_CK(cudaMemsetAsync(y, 0, nd * 8, stream));
            V2B_CK(cudaMemsetAsync(z, 0, np * 8, stream));
        }
        V2B_CK(cudaMemsetAsync(status, 0, 8, stream));
        v2b::spmv_A2_kernel<<<grid_for(nd, v2b::kSpmvThreads), v2b::kSpmvThreads, 0, stream>>>(
            A.rp, A.ent, nd, x, c, z, Ax, Acz, A.pal);
        V2B_CK(cudaGetLastError());
        launches++;
        long oiter = 0, iiter = 0;
        bool converged = false;
        double res[5] = {0, 0, 0, 0, 0};
        while (!converged && oiter < o.maxiter) {
            const long budget = std::min<long>(muf, o.maxiter - oiter);
            for (long k = 0; k < budget; k++) {
                cur_oiter = oiter;
                // mu is fixed inside this block: extrapolate the CG start through
                // the block's previous solutions (none at its first iteration)
                iterate(o, res, (int)std::min<long>(k, 2));
                const int it = (int)res[0];
                if (monitor) monitor(print_level, (int)oiter, it, res[3], res[4], mu, res[1], res[2], data);
                oiter++;
                iiter += it;
                converged = res[1] < o.sdp_error_convergence && res[2] < o.sdp_error_convergence &&
                            std::fabs(res[3] - res[4]) < o.sdp_objective_convergence;
                if (converged) break;
            }
            if (!converged && res[2] > 0.0) mu = mu * res[1] / res[2];
        }
        solved = true;
        if (oiter_out) *oiter_out = oiter;
        if (iiter_out) *iiter_out = iiter;
        if (energy) *energy = res[3];
        return converged ? V2B_OK : V2B_NOT_CONVERGED;
    }
};

// ====================================================================
// libsdp-shaped solver with host callbacks
// ====================================================================
struct v2b_bpsdp {
    long np = 0, nd = 0;
    v2b_sdp_options opt{};
    double mu = 0.1;
    std::vector<double> y, z;
    long iiter = 0, oiter = 0;
    bool converged = false;
    ProjectPlan plan;
    cudaStream_t stream = nullptr;
    double *dU = nullptr, *dx = nullptr, *dz = nullptr;
    int *status = nullptr;
    long launches = 0;

    ~v2b_bpsdp() {
        if (!stream) return;
        plan.release();
        cudaFree(dU); cudaFree(dx); cudaFree(dz); cudaFree(status);
        if (stream) cudaStreamDestroy(stream);
    }

    void ensure_plan(const std::vector<int> &dims) {
        if (dims == plan.dims && dU) return;
        int64_t tot = 0;
        for (int d : dims) tot += (int64_t)d * d;
        if (tot != np) throw std::invalid_argument("sum of squared block dimensions != n_primal");
        plan.release();
        plan.build(dims);
        if (!dU) {
            dU = dalloc<double>(np); dx = dalloc<double>(np); dz = dalloc<double>(np);
            status = dalloc<int>(2);
            V2B_CK(cudaMemset(status, 0, 8));
        }
    }

    int solve(double *x, const double *b, const double *c, const std::vector<int> &dims, int maxiter,
              v2b_sdp_callback Au, v2b_sdp_callback ATu, v2b_sdp_monitor monitor, int print_level,
              void *data) {
        ensure_plan(dims);
        std::vector<double> Ax(nd), Acz(nd), rhs(nd), r(nd), p(nd), Ap(nd), tmp_p(np), w(np);
        std::vector<double> ATy(np), U(np);
        auto dot = [](const std::vector<double> &a, const std::vector<double> &bb) {
            double s = 0.0;
            for (size_t i = 0; i < a.size(); i++) s += a[i] * bb[i];
            return s;
        };
        auto AAT = [&](std::vector<double> &in, std::vector<double> &out) {
            ATu(tmp_p.data(), in.data(), data);
            Au(out.data(), tmp_p.data(), data);
        };
        double ep = 0, ed = 0;
        converged = false;
        for (int it = 0; it < maxiter; it++) {
            Au(Ax.data(), x, data);
            for (long i = 0; i < np; i++) w[i] = c[i] - z[i];
            Au(Acz.data(), w.data(), data);
            for (long j = 0; j < nd; j++) rhs[j] = Acz[j] + mu * (b[j] - Ax[j]);
            // conjugate gradients on A A^T, warm start from y
            AAT(y, Ap);
            for (long j = 0; j < nd; j++) { r[j] = rhs[j] - Ap[j]; p[j] = r[j]; }
            double rs = dot(r, r);
            int cg_it = 0;
            while (std::sqrt(rs) >= opt.cg_convergence && cg_it < opt.cg_maxiter) {
                AAT(p, Ap);
                const double pAp = dot(p, Ap);
                if (!(pAp > 0.0)) break;
                const double alpha = rs / pAp;
                for (long j = 0; j < nd; j++) { y[j] += alpha * p[j]; r[j] -= alpha * Ap[j]; }
                const double rs_new = dot(r, r);
                cg_it++;
                if (std::sqrt(rs_new) < opt.cg_convergence) { rs = rs_new; break; }
                const double beta = rs_new / rs;
                for (long j = 0; j < nd; j++) p[j] = r[j] + beta * p[j];
                rs = rs_new;
            }
            ATu(ATy.data(), y.data(), data);
            for (long i = 0; i < np; i++) U[i] = mu * x[i] + ATy[i] - c[i];
            V2B_CK(cudaMemcpyAsync(dU, U.data(), np * 8, cudaMemcpyHostToDevice, stream));
            plan.project(dU, mu, dx, dz, stream, launches);
            V2B_CK(cudaMemcpyAsync(x, dx, np * 8, cudaMemcpyDeviceToHost, stream));
            V2B_CK(cudaMemcpyAsync(z.data(), dz, np * 8, cudaMemcpyDeviceToHost, stream));
            V2B_CK(cudaStreamSynchronize(stream));
            Au(Ax.data(), x, data);
            double s0 = 0.0, s1 = 0.0, Ep = 0.0, Ed = 0.0;
            for (long j = 0; j < nd; j++) { const double d = Ax[j] - b[j]; s0 += d * d; Ed += b[j] * y[j]; }
            for (long i = 0; i < np; i++) { const double d = ATy[i] + z[i] - c[i]; s1 += d * d; Ep += c[i] * x[i]; }
            ep = std::sqrt(s0);
            ed = std::sqrt(s1);
            if (!std::isfinite(ep) || !std::isfinite(ed)) throw Failure(V2B_NAN, "non-finite error norm");
            iiter += cg_it;
            if (monitor) monitor(print_level, (int)oiter, cg_it, Ep, Ed, mu, ep, ed, data);
            oiter++;
            converged = ep < opt.sdp_error_convergence && ed < opt.sdp_error_convergence &&
                        std::fabs(Ep - Ed) < opt.sdp_objective_convergence;
            if (converged) break;
        }
        if (!converged && ed > 0.0) mu = mu * ep / ed;
        return converged ? V2B_OK : V2B_NOT_CONVERGED;
    }
};

// ====================================================================
// C ABI
// ====================================================================
extern "C" {

const char *v2b_last_error(void) { return g_last_error.c_str(); }
int v2b_version(void) { return 1; }

int v2b_bpsdp_create(long n_primal, long n_dual, const v2b_sdp_options *options, v2b_bpsdp **out) {
    return guarded([&] {
        if (!out || !options || n_primal <= 0 || n_dual <= 0)
            throw std::invalid_argument("v2b_bpsdp_create: bad arguments");
        ensure_device();
        std::unique_ptr<v2b_bpsdp> s(new v2b_bpsdp());
        s->np = n_primal;
        s->nd = n_dual;
        s->opt = *options;
        s->y.assign(n_dual, 0.0);
        s->z.assign(n_primal, 0.0);
        V2B_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        *out = s.release();
        return V2B_OK;
    });
}

int v2b_bpsdp_solve(v2b_bpsdp *s, double *x, const double *b, const double *c,
                    const int *primal_block_dims, int n_blocks, int maxiter, v2b_sdp_callback Au,
                    v2b_sdp_callback ATu, v2b_sdp_monitor monitor, int print_level, void *data) {
    return guarded([&] {
        if (!s || !x || !b || !c || !primal_block_dims || n_blocks <= 0 || !Au || !ATu || maxiter < 0)
            throw std::invalid_argument("v2b_bpsdp_solve: bad arguments");
        std::vector<int> dims(primal_block_dims, primal_block_dims + n_blocks);
        return s->solve(x, b, c, dims, maxiter, Au, ATu, monitor, print_level, data);
    });
}

int v2b_bpsdp_is_converged(const v2b_bpsdp *s) { return s && s->converged ? 1 : 0; }
double v2b_bpsdp_get_mu(const v2b_bpsdp *s) { return s ? s->mu : NAN; }
int v2b_bpsdp_set_mu(v2b_bpsdp *s, double mu) {
    if (!s || !(mu > 0.0)) { g_last_error = "set_mu: mu must be positive"; return V2B_BAD_ARG; }
    s->mu = mu;
    return V2B_OK;
}
int v2b_bpsdp_get_y(const v2b_bpsdp *s, double *y) {
    if (!s || !y) return V2B_BAD_ARG;
    std::memcpy(y, s->y.data(), s->nd * 8);
    return V2B_OK;
}
int v2b_bpsdp_get_z(const v2b_bpsdp *s, double *z) {
    if (!s || !z) return V2B_BAD_ARG;
    std::memcpy(z, s->z.data(), s->np * 8);
    return V2B_OK;
}
int v2b_bpsdp_set_y(v2b_bpsdp *s, const double *y) {
    if (!s || !y) return V2B_BAD_ARG;
    std::memcpy(s->y.data(), y, s->nd * 8);
    return V2B_OK;
}
int v2b_bpsdp_set_z(v2b_bpsdp *s, const double *z) {
    if (!s || !z) return V2B_BAD_ARG;
    std::memcpy(s->z.data(), z, s->np * 8);
    return V2B_OK;
}
long v2b_bpsdp_iiter_total(const v2b_bpsdp *s) { return s ? s->iiter : -1; }
long v2b_bpsdp_oiter_total(const v2b_bpsdp *s) { return s ? s->oiter : -1; }
void v2b_bpsdp_destroy(v2b_bpsdp *s) { delete s; }

int v2b_problem_create(int nmo, int nalpha, int nbeta, int positivity, int constrain_spin,
                       int constrain_sz, int hubbard_multiplicity, v2b_problem **out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("v2b_problem_create: out is NULL");
        v2b::ProblemSpec spec;
        spec.nmo = nmo;
        spec.nalpha = nalpha;
        spec.nbeta = nbeta;
        if (positivity < 0 ||
            (positivity & ~(15 | V2B_CONSTRAIN_D3 | V2B_CONSTRAIN_Q3 | V2B_CONSTRAIN_E3 | V2B_CONSTRAIN_F3 |
                            V2B_CONSTRAIN_D4)))
            throw std::invalid_argument("v2b_problem_create: unknown POSITIVITY bits");
        spec.positivity = positivity & 15;
        spec.constrain_d3 = (positivity & V2B_CONSTRAIN_D3) != 0;
        spec.constrain_q3 = (positivity & V2B_CONSTRAIN_Q3) != 0;
        spec.constrain_e3 = (positivity & V2B_CONSTRAIN_E3) != 0;
        spec.constrain_f3 = (positivity & V2B_CONSTRAIN_F3) != 0;
        spec.constrain_d4 = (positivity & V2B_CONSTRAIN_D4) != 0;
        spec.constrain_spin = constrain_spin != 0;
        spec.constrain_sz = constrain_sz != 0;
        spec.hubbard_multiplicity = hubbard_multiplicity != 0;
        std::unique_ptr<v2b_problem> p(new v2b_problem());
        p->prob = v2b::make_problem(spec);
        p->hostA = v2b::build_A(p->prob);
        p->hostAT = v2b::build_AT(p->prob);
        *out = p.release();
        return V2B_OK;
    });
}

int v2b_doci_problem_create(int nmo, int nalpha, int nbeta, int positivity, v2b_problem **out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("v2b_doci_problem_create: out is NULL");
        if (positivity < 0 || (positivity & ~(15 | V2B_CONSTRAIN_D3)))
            throw std::invalid_argument("v2b_doci_problem_create: DOCI takes POSITIVITY and CONSTRAIN_D3 only");
        v2b::ProblemSpec spec;
        spec.doci = true;
        spec.nmo = nmo;
        spec.nalpha = nalpha;
        spec.nbeta = nbeta;
        spec.positivity = positivity & 15;
        spec.constrain_d3 = (positivity & V2B_CONSTRAIN_D3) != 0;
        std::unique_ptr<v2b_problem> p(new v2b_problem());
        p->prob = v2b::make_problem(spec);
        p->hostA = v2b::build_A(p->prob);
        p->hostAT = v2b::build_AT(p->prob);
        *out = p.release();
        return V2B_OK;
    });
}

int v2b_problem_palette(const v2b_problem *p, int transposed, double *out, int *count) {
    return guarded([&] {
        if (!p || !count) throw std::invalid_argument("palette: NULL argument");
        const std::vector<double> &pal = transposed ? p->hostAT.palette : p->hostA.palette;
        *count = (int)pal.size();
        if (out) std::copy(pal.begin(), pal.end(), out);
        return V2B_OK;
    });
}
int v2b_batch_problem_create(const v2b_problem *const *parts, int count, v2b_problem **out) {
    return guarded([&] {
        if (!out || !parts || count < 1) throw std::invalid_argument("v2b_batch_problem_create: bad argument");
        std::vector<const v2b::Problem *> probs;
        std::vector<const v2b::PackedOperator *> A, AT;
        for (int k = 0; k < count; k++) {
            if (!parts[k]) throw std::invalid_argument("v2b_batch_problem_create: NULL part");
            probs.push_back(&parts[k]->prob);
            A.push_back(&parts[k]->hostA);
            AT.push_back(&parts[k]->hostAT);
        }
        std::unique_ptr<v2b_problem> p(new v2b_problem());
        v2b::make_batch(probs, A, AT, p->prob, p->hostA, p->hostAT);
        *out = p.release();
        return V2B_OK;
    });
}

void v2b_problem_destroy(v2b_problem *p) { delete p; }
long v2b_problem_n_primal(const v2b_problem *p) { return p ? p->prob.n_primal : -1; }
long v2b_problem_n_dual(const v2b_problem *p) { return p ? p->prob.n_dual : -1; }
int v2b_problem_n_blocks(const v2b_problem *p) { return p ? (int)p->prob.dims.size() : -1; }
int v2b_problem_block_dims(const v2b_problem *p, int *dims) {
    if (!p || !dims) return V2B_BAD_ARG;
    std::copy(p->prob.dims.begin(), p->prob.dims.end(), dims);
    return V2B_OK;
}
int v2b_problem_build_b(const v2b_problem *p, double *b) {
    return guarded([&] {
        if (!p || !b) throw std::invalid_argument("build_b: NULL argument");
        v2b::build_b(p->prob, b);
        return V2B_OK;
    });
}
int v2b_problem_build_c_hubbard(const v2b_problem *p, double t, double U, double *c) {
    return guarded([&] {
        if (!p || !c) throw std::invalid_argument("build_c_hubbard: NULL argument");
        v2b::build_c_hubbard(p->prob, t, U, c);
        return V2B_OK;
    });
}
int v2b_problem_build_c_external(const v2b_problem *p, const double *h, const double *g, double *c) {
    return guarded([&] {
        if (!p || !h || !g || !c) throw std::invalid_argument("build_c_external: NULL argument");
        v2b::build_c_external(p->prob, h, g, c);
        return V2B_OK;
    });
}
int v2b_problem_guess(const v2b_problem *p, int hf, double *x) {
    return guarded([&] {
        if (!p || !x) throw std::invalid_argument("guess: NULL argument");
        if (hf) v2b::guess_hf(p->prob, x);
        else v2b::guess_random(p->prob, x);
        return V2B_OK;
    });
}
int v2b_problem_Au(v2b_problem *p, const double *d_in, double *d_out, void *stream) {
    return guarded([&] {
        if (!p || !d_in || !d_out) throw std::invalid_argument("Au: NULL argument");
        p->setup();
        p->Au(d_in, d_out, (cudaStream_t)stream);
        return V2B_OK;
    });
}
int v2b_problem_ATu(v2b_problem *p, const double *d_in, double *d_out, void *stream) {
    return guarded([&] {
        if (!p || !d_in || !d_out) throw std::invalid_argument("ATu: NULL argument");
        p->setup();
        p->ATu(d_in, d_out, (cudaStream_t)stream);
        return V2B_OK;
    });
}
int v2b_problem_project(v2b_problem *p, const double *d_U, double mu, double *d_x, double *d_z,
                        void *stream) {
    return guarded([&] {
        if (!p || !d_U || !d_x || !d_z || !(mu > 0.0)) throw std::invalid_argument("project: bad argument");
        p->setup();
        p->ensure_plan();
        // a stand-alone projection has no previous basis: solve each block from scratch
        p->plan.reset();
        p->plan.project(d_U, mu, d_x, d_z, (cudaStream_t)stream, p->launches);
        p->plan.reset();
        return V2B_OK;
    });
}
int v2b_problem_project_warm(v2b_problem *p, const double *d_U, double mu, double *d_x, double *d_z,
                             void *stream) {
    return guarded([&] {
        if (!p || !d_U || !d_x || !d_z || !(mu > 0.0))
            throw std::invalid_argument("project_warm: bad argument");
        p->setup();
        p->ensure_plan();
        p->plan.project(d_U, mu, d_x, d_z, (cudaStream_t)stream, p->launches);
        return V2B_OK;
    });
}
int v2b_problem_solve_device(v2b_problem *p, double *d_x, const double *d_b, const double *d_c,
                             const v2b_sdp_options *options, int mu_update_frequency,
                             v2b_sdp_monitor monitor, int print_level, void *data, long *oiter,
                             long *iiter, double *energy) {
    return guarded([&] {
        if (!p || !d_x || !d_b || !d_c || !options) throw std::invalid_argument("solve_device: NULL argument");
        p->setup();
        const int64_t np = p->prob.n_primal, nd = p->prob.n_dual;
        V2B_CK(cudaMemcpyAsync(p->x, d_x, np * 8, cudaMemcpyDeviceToDevice, p->stream));
        V2B_CK(cudaMemcpyAsync(p->b, d_b, nd * 8, cudaMemcpyDeviceToDevice, p->stream));
        V2B_CK(cudaMemcpyAsync(p->c, d_c, np * 8, cudaMemcpyDeviceToDevice, p->stream));
        const int rc = p->solve_device(*options, mu_update_frequency, monitor, print_level, data, oiter,
                                       iiter, energy);
        V2B_CK(cudaMemcpyAsync(d_x, p->x, np * 8, cudaMemcpyDeviceToDevice, p->stream));
        V2B_CK(cudaStreamSynchronize(p->stream));
        return rc;
    });
}
int v2b_problem_solve(v2b_problem *p, double *x, const double *b, const double *c,
                      const v2b_sdp_options *options, int mu_update_frequency,
                      v2b_sdp_monitor monitor, int print_level, void *data, long *oiter, long *iiter,
                      double *energy) {
    return guarded([&] {
        if (!p || !x || !b || !c || !options) throw std::invalid_argument("solve: NULL argument");
        const double *in[3] = {x, b, c};
        const int64_t len[3] = {p->prob.n_primal, p->prob.n_dual, p->prob.n_primal};
        const char *names[3] = {"x", "b", "c"};
        for (int k = 0; k < 3; k++) {
            const int64_t i = first_nonfinite(in[k], len[k]);
            if (i >= 0)
                throw Failure(V2B_NAN, std::string("non-finite value in ") + names[k] + " at index " +
                                           std::to_string(i));
        }
        p->setup();
        const int64_t np = p->prob.n_primal, nd = p->prob.n_dual;
        V2B_CK(cudaMemcpyAsync(p->x, x, np * 8, cudaMemcpyHostToDevice, p->stream));
        V2B_CK(cudaMemcpyAsync(p->b, b, nd * 8, cudaMemcpyHostToDevice, p->stream));
        V2B_CK(cudaMemcpyAsync(p->c, c, np * 8, cudaMemcpyHostToDevice, p->stream));
        const int rc = p->solve_device(*options, mu_update_frequency, monitor, print_level, data, oiter,
                                       iiter, energy);
        V2B_CK(cudaMemcpyAsync(x, p->x, np * 8, cudaMemcpyDeviceToHost, p->stream));
        V2B_CK(cudaStreamSynchronize(p->stream));
        return rc;
    });
}
int v2b_problem_get_y(const v2b_problem *p, double *y) {
    return guarded([&] {
        if (!p || !y) throw std::invalid_argument("get_y: NULL argument");
        if (!p->on_device) throw std::invalid_argument("get_y: no device solve has run");
        V2B_CK(cudaMemcpy(y, p->y, p->prob.n_dual * 8, cudaMemcpyDeviceToHost));
        return V2B_OK;
    });
}
int v2b_problem_set_state(v2b_problem *p, double mu, const double *y, const double *z) {
    return guarded([&] {
        if (!p || !y || !z) throw std::invalid_argument("set_state: NULL argument");
        if (!(mu > 0.0) || !std::isfinite(mu)) throw std::invalid_argument("set_state: mu must be positive");
        p->resume_y.assign(y, y + p->prob.n_dual);
        p->resume_z.assign(z, z + p->prob.n_primal);
        p->mu = mu;
        p->resume = true;
        p->keep_state = false;
        return V2B_OK;
    });
}
int v2b_problem_set_wait_limit(v2b_problem *p, long long polls) {
    return guarded([&] {
        if (!p || polls < 0) throw std::invalid_argument("set_wait_limit: bad argument");
        p->wait_limit = polls ? polls : v2b_problem::kDefaultWaitLimit;
        return V2B_OK;
    });
}
int v2b_problem_continue(v2b_problem *p) {
    return guarded([&] {
        if (!p) throw std::invalid_argument("continue: NULL argument");
        if (!p->on_device || !p->solved) throw std::invalid_argument("continue: no device solve has run");
        p->resume = false;
        std::vector<double>().swap(p->resume_y);
        std::vector<double>().swap(p->resume_z);
        p->keep_state = true;
        return V2B_OK;
    });
}
int v2b_problem_get_z(const v2b_problem *p, double *z) {
    return guarded([&] {
        if (!p || !z) throw std::invalid_argument("get_z: NULL argument");
        if (!p->on_device) throw std::invalid_argument("get_z: no device solve has run");
        V2B_CK(cudaMemcpy(z, p->z, p->prob.n_primal * 8, cudaMemcpyDeviceToHost));
        return V2B_OK;
    });
}
int v2b_problem_operator_size(const v2b_problem *p, int transposed, long *nrows, long *nnz,
                              int *npalette) {
    if (!p || !nrows || !nnz || !npalette) return V2B_BAD_ARG;
    const v2b::PackedOperator &op = transposed ? p->hostAT : p->hostA;
    *nrows = op.nrows;
    *nnz = (long)op.entries.size();
    *npalette = (int)op.palette.size();
    return V2B_OK;
}
int v2b_problem_operator(const v2b_problem *p, int transposed, uint32_t *row_ptr, uint32_t *entries,
                         double *palette) {
    if (!p || !row_ptr || !entries || !palette) return V2B_BAD_ARG;
    const v2b::PackedOperator &op = transposed ? p->hostAT : p->hostA;
    std::copy(op.row_ptr.begin(), op.row_ptr.end(), row_ptr);
    std::copy(op.entries.begin(), op.entries.end(), entries);
    std::copy(op.palette.begin(), op.palette.end(), palette);
    return V2B_OK;
}
double v2b_problem_get_mu(const v2b_problem *p) { return p ? p->mu : NAN; }
long v2b_problem_kernel_launches(const v2b_problem *p) { return p ? p->launches : -1; }
int v2b_problem_set_profiling(v2b_problem *p, int on) {
    return guarded([&] {
        if (!p) throw std::invalid_argument("set_profiling: NULL problem");
        p->setup();
        p->set_profiling(on < 0 ? 0 : on);
        return V2B_OK;
    });
}
int v2b_problem_profile(const v2b_problem *p, double *ms, long *launches) {
    if (!p || !ms || !launches) return V2B_BAD_ARG;
    for (int k = 0; k < v2b_problem::kClasses; k++) {
        ms[k] = p->prof_ms[k];
        launches[k] = p->prof_n[k];
    }
    return V2B_OK;
}
void *v2b_problem_stream(const v2b_problem *p) { return p ? (void *)p->stream : nullptr; }
int v2b_problem_projection_counts(const v2b_problem *p, long *calls, long *rotations,
                                  long *sweep_overruns) {
    return guarded([&] {
        if (!p || !calls || !rotations || !sweep_overruns)
            throw std::invalid_argument("projection_counts: NULL argument");
        *calls = p->plan.calls;
        int h[4] = {0, 0, 0, 0};
        if (p->plan.built) V2B_CK(cudaMemcpy(h, p->plan.counters, 16, cudaMemcpyDeviceToHost));
        *rotations = (long)h[1] + h[3];
        *sweep_overruns = (long)h[0] + h[2];
        return V2B_OK;
    });
}

int v2b_problem_cg_profile(const v2b_problem *p, double *ms, int count) {
    return guarded([&] {
        if (!p || !ms || count < 0) throw std::invalid_argument("cg_profile: bad argument");
        unsigned long long h[v2b_problem::kCgPhases] = {};
        if (p->cg_phase) {
            V2B_CK(cudaStreamSynchronize(p->stream));
            V2B_CK(cudaMemcpy(h, p->cg_phase, sizeof(h), cudaMemcpyDeviceToHost));
        }
        for (int k = 0; k < count && k < v2b_problem::kCgPhases; k++) ms[k] = 1e-6 * (double)h[k];
        return V2B_OK;
    });
}

int v2b_problem_set_projection_mode(v2b_problem *p, int mode) {
    return guarded([&] {
        if (!p || mode < 0 || mode > 2) throw std::invalid_argument("set_projection_mode: bad argument");
        p->plan.mode = mode;
        return V2B_OK;
    });
}

int v2b_problem_set_gemm_split(v2b_problem *p, int on) {
    return guarded([&] {
        if (!p) throw std::invalid_argument("set_gemm_split: NULL problem");
        p->plan.split_k = on != 0;
        return V2B_OK;
    });
}

int v2b_problem_gemm_split_choice(const v2b_problem *p, int *full, int *upper) {
    return guarded([&] {
        if (!p || !full || !upper) throw std::invalid_argument("gemm_split_choice: NULL argument");
        *full = p->plan.built ? p->plan.split_full : 0;
        *upper = p->plan.built ? p->plan.split_sym : 0;
        return V2B_OK;
    });
}
int v2b_problem_projection_profile(const v2b_problem *p, double *ms, long *n, int count) {
    return guarded([&] {
        if (!p || !ms || !n || count < 0) throw std::invalid_argument("projection_profile: bad argument");
        for (int k = 0; k < count && k < ProjectPlan::kPhases; k++) {
            ms[k] = p->plan.ph_ms[k];
            n[k] = p->plan.ph_n[k];
        }
        return V2B_OK;
    });
}
int v2b_doci_v2rdm_layout(const v2b_problem *p, const double *x, double *out, long *size) {
    return guarded([&] {
        if (!p || !size) throw std::invalid_argument("doci_v2rdm_layout: NULL argument");
        if (!p->prob.spec.doci) throw std::invalid_argument("doci_v2rdm_layout: not a DOCI problem");
        *size = (long)v2b::doci_v2rdm_layout_size(p->prob);
        if (out) {
            if (!x) throw std::invalid_argument("doci_v2rdm_layout: NULL x");
            v2b::doci_v2rdm_layout(p->prob, x, out);
        }
        return V2B_OK;
    });
}
int v2b_problem_rdm_counts(const v2b_problem *p, int ncore, long *counts) {
    return guarded([&] {
        if (!p || !counts) throw std::invalid_argument("rdm_counts: NULL argument");
        const v2b::RdmCounts c = v2b::rdm_counts(p->prob, ncore);
        const long v[6] = {(long)c.d2aa, (long)c.d2bb, (long)c.d2ab, (long)c.d2, (long)c.d1a, (long)c.d1b};
        std::copy(v, v + 6, counts);
        return V2B_OK;
    });
}
int v2b_problem_rdm_records(const v2b_problem *p, int ncore, const double *x, v2b_tpdm_record *d2aa,
                            v2b_tpdm_record *d2bb, v2b_tpdm_record *d2ab, v2b_tpdm_record *d2,
                            v2b_opdm_record *d1a, v2b_opdm_record *d1b) {
    static_assert(sizeof(v2b_tpdm_record) == sizeof(v2b::TpdmRecord), "record layout");
    static_assert(sizeof(v2b_opdm_record) == sizeof(v2b::OpdmRecord), "record layout");
    return guarded([&] {
        if (!p || !x) throw std::invalid_argument("rdm_records: NULL argument");
        v2b::rdm_records(p->prob, x, ncore, (v2b::TpdmRecord *)d2aa, (v2b::TpdmRecord *)d2bb,
                         (v2b::TpdmRecord *)d2ab, (v2b::TpdmRecord *)d2, (v2b::OpdmRecord *)d1a,
                         (v2b::OpdmRecord *)d1b);
        return V2B_OK;
    });
}
int v2b_problem_tpdm_iwl_records(const v2b_problem *p, int ncore, const double *x, v2b_tpdm_record *d2aa,
                                 v2b_tpdm_record *d2ab, v2b_tpdm_record *d2bb) {
    return guarded([&] {
        if (!p || !x) throw std::invalid_argument("tpdm_iwl_records: NULL argument");
        v2b::iwl_records(p->prob, x, ncore, (v2b::TpdmRecord *)d2aa, (v2b::TpdmRecord *)d2ab,
                         (v2b::TpdmRecord *)d2bb);
        return V2B_OK;
    });
}
int v2b_problem_d3_counts(const v2b_problem *p, long *counts) {
    return guarded([&] {
        if (!p || !counts) throw std::invalid_argument("d3_counts: NULL argument");
        int64_t c[2];
        v2b::d3_counts(p->prob, c);
        counts[0] = (long)c[0];
        counts[1] = (long)c[1];
        return V2B_OK;
    });
}
int v2b_problem_d3_records(const v2b_problem *p, int ncore, const double *x, v2b_dm3_record *d3aaa,
                           v2b_dm3_record *d3aab, v2b_dm3_record *d3bba, v2b_dm3_record *d3bbb) {
    static_assert(sizeof(v2b_dm3_record) == sizeof(v2b::Dm3Record), "record layout");
    return guarded([&] {
        if (!p || !x) throw std::invalid_argument("d3_records: NULL argument");
        v2b::d3_records(p->prob, x, ncore, (v2b::Dm3Record *)d3aaa, (v2b::Dm3Record *)d3aab,
                        (v2b::Dm3Record *)d3bba, (v2b::Dm3Record *)d3bbb);
        return V2B_OK;
    });
}
int v2b_problem_pack_dims(const v2b_problem *p, long *d2_size, long *d1_size) {
    return guarded([&] {
        if (!p || !d2_size || !d1_size) throw std::invalid_argument("pack_dims: NULL argument");
        if (p->prob.spec.batch_parts) throw std::invalid_argument("pack_dims: pack each part of a batch");
        const long g00 = (long)p->prob.n * (p->prob.n + 1) / 2;
        *d2_size = g00 * (g00 + 1) / 2;
        *d1_size = g00;
        return V2B_OK;
    });
}
int v2b_problem_pack_spatial_density(v2b_problem *p, const double *d_x, double *d_d2, double *d_d1,
                                     void *stream) {
    return guarded([&] {
        if (!p || !d_x || !d_d2 || !d_d1) throw std::invalid_argument("pack_spatial_density: NULL argument");
        if (p->prob.spec.batch_parts) throw std::invalid_argument("pack_spatial_density: pack each part of a batch");
        p->setup();
        const v2b::Problem &q = p->prob;
        if (!p->ibas_aa_dev) {
            p->ibas_aa_dev = dalloc<int>((size_t)q.n * q.n);
            V2B_CK(cudaMemcpy(p->ibas_aa_dev, q.ibas_aa.data(), sizeof(int) * q.n * q.n,
                              cudaMemcpyHostToDevice));
        }
        v2b::PackArgs a;
        a.n = q.n;
        a.d2ab = q.d2ab; a.d2aa = q.d2aa; a.d2bb = q.d2bb; a.d1a = q.d1a; a.d1b = q.d1b;
        a.ibas_aa = p->ibas_aa_dev;
        if (q.spec.doci) {
            // hilbert's DOCI packing (v2rdm_doci_solver.cc:1568-1703) is the
            // v2RDM packing of D2ab, D2aa = D2bb and D1a = D1b expanded from
            // the seniority blocks; D2s2, D2s0 and D1 lead the primal vector
            const int64_t n = q.n, lead = 2 * n * n + n, size = v2b::doci_v2rdm_layout_size(q);
            if (q.doci.d2s2 != 0 || q.doci.d2s0 != n * n || q.doci.d1 != 2 * n * n)
                throw std::logic_error("DOCI block layout");
            std::vector<double> blocks(lead), layout(size);
            V2B_CK(cudaMemcpyAsync(blocks.data(), d_x, lead * 8, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
            V2B_CK(cudaStreamSynchronize((cudaStream_t)stream));
            v2b::doci_v2rdm_layout(q, blocks.data(), layout.data());
            if (!p->pack_layout) p->pack_layout = dalloc<double>(size);
            V2B_CK(cudaMemcpyAsync(p->pack_layout, layout.data(), size * 8, cudaMemcpyHostToDevice,
                                   (cudaStream_t)stream));
            V2B_CK(cudaStreamSynchronize((cudaStream_t)stream));   // layout is a host temporary
            const int64_t gab2 = (int64_t)q.gab * q.gab, gaa2 = (int64_t)q.gaa * q.gaa;
            a.d2ab = 0; a.d2aa = gab2; a.d2bb = gab2 + gaa2; a.d1a = gab2 + 2 * gaa2; a.d1b = a.d1a + n * n;
            d_x = p->pack_layout;
        }
        const int64_t g00 = (int64_t)q.n * (q.n + 1) / 2, total = g00 * (g00 + 1) / 2 + g00;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 8));
        v2b::pack_spatial_density_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(d_x, a, d_d2, d_d1);
        V2B_CK(cudaGetLastError());
        p->launches++;
        return V2B_OK;
    });
}
int v2b_problem_refine_counts(const v2b_problem *p, long *counts, int n) {
    return guarded([&] {
        if (!p || !counts || n < 0) throw std::invalid_argument("refine_counts: bad argument");
        const ProjectPlan &q = p->plan;
        const long v[9] = {q.refine_accepted, q.refine_jacobi, q.refine_passes, q.refine_clusters,
                           q.refine_large_clusters, q.fb_edges, q.fb_passes, q.refine_bj_sweeps,
                           q.fp32_solves};
        for (int i = 0; i < n && i < 9; i++) counts[i] = v[i];
        return V2B_OK;
    });
}

}  // extern "C"
