// CUDA kernels of the B200 boundary-point iteration (sm_100a).
//
//   spmv_kernel          y = A.x or A^T.y over packed rows (bit-exact to hilbert's maps)
//   spmv_A2_kernel       A.x and A.(c - z) in one pass over A's rows
//   spmv_AT_U_kernel     A^T.y and U = mu x + A^T y - c in one pass over A^T's rows
//   cg_kernel            persistent conjugate-gradient solve of (A A^T) y = rhs
//   stats_kernel         eps_p^2, eps_d^2, c.x, b.y (deterministic reductions)
//   jacobi_warm_kernel   per-block selective Jacobi on V^T U V in shared memory,
//                        middle factor of U+ and the refined eigenvectors
#include "v2b_kernels.cuh"

#include <cuda.h>

#include <mutex>

namespace v2b {

__global__ void spmv_kernel(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ent,
                            int64_t nrows, const double *__restrict__ x, double *__restrict__ y,
                            Palette pal) {
    __shared__ double spal[16];
    if (threadIdx.x < 16) spal[threadIdx.x] = pal.v[threadIdx.x];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
         r += (int64_t)gridDim.x * blockDim.x)
        y[r] = packed_row(ent, __ldg(rp + r), __ldg(rp + r + 1), x, spal);
}

__global__ void spmv_A2_kernel(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ent,
                               int64_t nrows, const double *__restrict__ x,
                               const double *__restrict__ c, const double *__restrict__ z,
                               double *__restrict__ Ax, double *__restrict__ Acz, Palette pal) {
    __shared__ double spal[16];
    if (threadIdx.x < 16) spal[threadIdx.x] = pal.v[threadIdx.x];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
         r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        double a0 = 0.0, a1 = 0.0, w0 = 0.0, w1 = 0.0;
        bool grp = false;
        for (uint32_t k = b; k < e; k++) {
            const uint32_t w = __ldg(ent + k);
            const uint32_t col = w & kDevColMask;
            const double cf = spal[(w >> 27) & 15u];
            const double vx = __dmul_rn(cf, __ldg(x + col));
            const double vw = __dmul_rn(cf, __dsub_rn(__ldg(c + col), __ldg(z + col)));
            grp = grp || (w >> 31);
            if (grp) { a1 = __dadd_rn(a1, vx); w1 = __dadd_rn(w1, vw); }
            else { a0 = __dadd_rn(a0, vx); w0 = __dadd_rn(w0, vw); }
        }
        Ax[r] = grp ? __dadd_rn(a0, a1) : a0;
        Acz[r] = grp ? __dadd_rn(w0, w1) : w0;
    }
}

__global__ void spmv_AT_U_kernel(const uint32_t *__restrict__ rp,
                                 const uint32_t *__restrict__ ent, int64_t nrows,
                                 const double *__restrict__ y, const double *__restrict__ x,
                                 const double *__restrict__ c, double mu,
                                 double *__restrict__ ATy, double *__restrict__ U, Palette pal) {
    __shared__ double spal[16];
    if (threadIdx.x < 16) spal[threadIdx.x] = pal.v[threadIdx.x];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
         r += (int64_t)gridDim.x * blockDim.x) {
        const double a = packed_row(ent, __ldg(rp + r), __ldg(rp + r + 1), y, spal);
        ATy[r] = a;
        U[r] = mu * x[r] + a - c[r];
    }
}

// Long rows inside CG: one warp per row, lanes stride over the entries and the
// partial sums meet in a shuffle tree (order differs from hilbert's left-to-
// right sum; the bit-exact kernels above are the ones the map API uses).
__device__ __forceinline__ double warp_row(const uint32_t *__restrict__ ent, uint32_t b, uint32_t e,
                                           const double *__restrict__ x, const double *__restrict__ p,
                                           double beta, const double *pal, int lane) {
    double acc = 0.0;
    for (uint32_t k = b + lane; k < e; k += 32) {
        const uint32_t w = __ldg(ent + k);
        const uint32_t c = w & kDevColMask;
        double v = __ldg(x + c);
        if (p) v = __dadd_rn(v, __dmul_rn(beta, __ldg(p + c)));
        acc += pal[(w >> 27) & 15u] * v;
    }
    return warp_sum(acc);
}

// One SELL slice per warp: lane l forms row perm[32 s + l] of the operator
// applied to x (RBP: to r + beta p, formed per operand as in the stored
// update), summing its entries in stored order (the group flag splits the
// sum as packed_row does).  Table loads stream (evict first) so the vectors
// stay in L2.
template <bool RBP>
__device__ __forceinline__ double sell_row(const SellOp &S, int64_t sl, int lane,
                                           const double *__restrict__ x, const double *__restrict__ p,
                                           double beta, const double *pal, uint32_t &row) {
    const int64_t pos = sl * 32 + lane;
    row = __ldcs(S.perm + pos);
    const int len = __ldcs(S.len + pos);
    const uint32_t base = __ldcs(S.off + sl) + lane;
    double acc0 = 0.0, acc1 = 0.0;
    bool grp = false;
#pragma unroll 4
    for (int k = 0; k < len; k++) {
        const uint32_t w = __ldcs(S.ent + base + 32u * k);
        const uint32_t c = w & kDevColMask;
        double xv = __ldg(x + c);
        if (RBP) xv = __dadd_rn(xv, __dmul_rn(beta, __ldg(p + c)));
        const double v = __dmul_rn(pal[(w >> 27) & 15u], xv);
        grp = grp || (w >> 31);
        if (grp) acc1 = __dadd_rn(acc1, v);
        else acc0 = __dadd_rn(acc0, v);
    }
    return grp ? __dadd_rn(acc0, acc1) : acc0;
}

// ------------------------------------------------------------------ CG
// Solves (A A^T) y = rhs with rhs = A(c - z) + mu (b - A x), warm-started from
// y, in the form CG takes on normal equations: with t = A^T p the step
// length's denominator p.(A A^T p) is ||t||^2, which the pass that forms t
// sums as it goes, so the update of y and r joins the pass that forms A t.
// Two grid barriers per iteration:
//   1. p_new = r + beta p_old, t = A^T p_new, partial ||t||^2
//      -> alpha = r.r / ||t||^2
//   2. per row j of A: q_j = (A t)_j, y_j += alpha p_new_j,
//      r_j -= alpha q_j, partial r.r  -> beta, convergence
// The t.t and r.r partials live in separate arrays: a block that has passed
// one barrier writes its next partial while slower blocks may still be
// summing the other.  Operator rows of up to kCgLongRow entries are applied
// from the sliced-ELL copies (one warp per 32-row slice), longer rows by a
// warp each from the CSR tables; every row of A is in exactly one of the
// two, so the row update of pass 2 covers every dual index once.
// 3 CTAs per SM: the gathers are latency-bound and gain more from resident
// warps than from registers (2 CTAs per SM measured 10-15% slower)
__global__ void __launch_bounds__(kCgThreads, 3) cg_kernel(CgParams P) {
    __shared__ double palA[16], palT[16];
    __shared__ double red[32];
    __shared__ double bcast;
    __shared__ int flag;
    __shared__ unsigned long long tmark;   // phase clock (CTA 0, thread 0)
    if (threadIdx.x < 16) {
        palA[threadIdx.x] = P.palA.v[threadIdx.x];
        palT[threadIdx.x] = P.palT.v[threadIdx.x];
    }
    __syncthreads();
    // 32-bit thread indices (a grid holds far fewer than 2^31 threads);
    // the kernel runs at the 40-register limit of 3 CTAs per SM
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned stride = gridDim.x * blockDim.x;
    const int nb = gridDim.x;

    const int lane = threadIdx.x & 31;
    const unsigned gwarp = gtid >> 5, nwarps = stride >> 5;
    // optional phase clock: CTA 0 adds the time from barrier to barrier
    if (gtid == 0) tmark = global_ns();
    auto lap = [&](int k) {
        if (P.phase_ns != nullptr && gtid == 0) {
            const unsigned long long now = global_ns();
            P.phase_ns[k] += now - tmark;
            tmark = now;
        }
    };

    // r = rhs - A A^T y
    for (int64_t sl = P.st.split[gwarp], se = P.st.split[gwarp + 1]; sl < se; sl++) {
        uint32_t row;
        const double v = sell_row<false>(P.st, sl, lane, P.y, nullptr, 0.0, palT, row);
        if (row != 0xffffffffu) P.t[row] = v;
    }
    for (int64_t w = gwarp; w < P.n_long_t; w += nwarps) {
        const int64_t i = __ldg(P.long_t + w);
        const double v = warp_row(P.t_ent, __ldg(P.t_rp + i), __ldg(P.t_rp + i + 1), P.y, nullptr, 0.0,
                                  palT, lane);
        if (lane == 0) P.t[i] = v;
    }
    if (!grid_sync(P.bar, P.status, P.spin_limit, &flag)) return;
    double loc = 0.0;
    for (int64_t sl = P.sa.split[gwarp], se = P.sa.split[gwarp + 1]; sl < se; sl++) {
        uint32_t row;
        const double av = sell_row<false>(P.sa, sl, lane, P.t, nullptr, 0.0, palA, row);
        if (row != 0xffffffffu) {
            const double v = P.Acz[row] + P.mu * (P.b[row] - P.Ax[row]) - av;
            P.r[row] = v;
            loc += v * v;
        }
    }
    for (int64_t w = gwarp; w < P.n_long_a; w += nwarps) {
        const int64_t j = __ldg(P.long_a + w);
        const double av = warp_row(P.a_ent, __ldg(P.a_rp + j), __ldg(P.a_rp + j + 1), P.t, nullptr, 0.0,
                                   palA, lane);
        if (lane == 0) {
            const double v = P.Acz[j] + P.mu * (P.b[j] - P.Ax[j]) - av;
            P.r[j] = v;
            loc += v * v;
        }
    }
    double s = block_sum(loc, red);
    if (threadIdx.x == 0) P.partials[nb + blockIdx.x] = s;
    if (!grid_sync(P.bar, P.status, P.spin_limit, &flag)) return;
    lap(0);
    double rs = sum_partials(P.partials + nb, nb, &bcast);

    int it = 0;
    double beta = 0.0;
    // p_old is r on the first iteration (beta = 0), then p0 and p1 alternate
    // as p_new and p_old
    bool done = !(sqrt(rs) >= P.tol);
    while (!done && it < P.maxit) {
        // pass 1: t = A^T (r + beta p_old), ||t||^2; p_new = r + beta p_old
        const double *pold = it == 0 ? P.r : ((it & 1) ? P.p0 : P.p1);
        double *pnew = (it & 1) ? P.p1 : P.p0;
        loc = 0.0;
        for (int64_t sl = P.st.split[gwarp], se = P.st.split[gwarp + 1]; sl < se; sl++) {
            uint32_t row;
            const double v = sell_row<true>(P.st, sl, lane, P.r, pold, beta, palT, row);
            if (row != 0xffffffffu) {
                P.t[row] = v;
                loc += v * v;
            }
        }
        for (int64_t w = gwarp; w < P.n_long_t; w += nwarps) {
            const int64_t i = __ldg(P.long_t + w);
            const double v = warp_row(P.t_ent, __ldg(P.t_rp + i), __ldg(P.t_rp + i + 1), P.r, pold,
                                      beta, palT, lane);
            if (lane == 0) {
                P.t[i] = v;
                loc += v * v;
            }
        }
        for (int64_t j = gtid; j < P.nd; j += stride)
            pnew[j] = __dadd_rn(P.r[j], __dmul_rn(beta, pold[j]));
        s = block_sum(loc, red);
        if (threadIdx.x == 0) P.partials[blockIdx.x] = s;
        if (!grid_sync(P.bar, P.status, P.spin_limit, &flag)) return;
        lap(1);
        const double tt = sum_partials(P.partials, nb, &bcast);
        if (!(tt > 0.0)) break;   // range of A A^T exhausted (or non-finite)
        const double alpha = rs / tt;

        // pass 2: q = A t row by row, y += alpha p_new, r -= alpha q, r.r
        loc = 0.0;
        for (int64_t w = gwarp; w < P.n_long_a; w += nwarps) {
            const int64_t j = __ldg(P.long_a + w);
            const double q = warp_row(P.a_ent, __ldg(P.a_rp + j), __ldg(P.a_rp + j + 1), P.t, nullptr,
                                      0.0, palA, lane);
            if (lane == 0) {
                P.y[j] += alpha * pnew[j];
                const double rv = P.r[j] - alpha * q;
                P.r[j] = rv;
                loc += rv * rv;
            }
        }
        for (int64_t sl = P.sa.split[gwarp], se = P.sa.split[gwarp + 1]; sl < se; sl++) {
            uint32_t row;
            const double q = sell_row<false>(P.sa, sl, lane, P.t, nullptr, 0.0, palA, row);
            if (row != 0xffffffffu) {
                P.y[row] += alpha * pnew[row];
                const double rv = P.r[row] - alpha * q;
                P.r[row] = rv;
                loc += rv * rv;
            }
        }
        s = block_sum(loc, red);
        if (threadIdx.x == 0) P.partials[nb + blockIdx.x] = s;
        if (!grid_sync(P.bar, P.status, P.spin_limit, &flag)) return;
        lap(2);
        const double rs_new = sum_partials(P.partials + nb, nb, &bcast);
        it++;
        if (!(rs_new == rs_new)) {   // NaN
            if (gtid == 0) atomicExch(P.status, kStatusNan);
            break;
        }
        done = sqrt(rs_new) < P.tol;
        beta = rs_new / rs;
        rs = rs_new;
    }
    if (gtid == 0) {
        P.out[0] = (double)it;
        P.out[1] = sqrt(rs);
    }
}

// ------------------------------------------------------- CG start
// The dual solution moves smoothly from one outer iteration to the next
// while mu stays fixed, so the conjugate gradients start from its polynomial
// extrapolation through the last solutions (linear after one, quadratic
// after two) instead of the last one.  The CG still runs to the same
// residual tolerance: only the number of its iterations changes (about half
// on the benchmark problems, the same outer iterations and energies to
// 1e-8 Eh).
__global__ void extrapolate_y_kernel(double *__restrict__ y, double *__restrict__ y1,
                                     double *__restrict__ y2, int64_t n, int order) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const double v = y[j], v1 = y1[j];
        if (order == 1) y[j] = 2.0 * v - v1;
        else if (order == 2) y[j] = 3.0 * (v - v1) + y2[j];
        y2[j] = v1;
        y1[j] = v;
    }
}

// --------------------------------------------------------------- stats
// out[0] = ||A x - b||^2, out[1] = ||A^T y + z - c||^2, out[2] = c.x, out[3] = b.y
__global__ void stats_kernel(const double *__restrict__ Ax, const double *__restrict__ b,
                             const double *__restrict__ ATy, const double *__restrict__ z,
                             const double *__restrict__ c, const double *__restrict__ x,
                             const double *__restrict__ y, int64_t np, int64_t nd,
                             double *__restrict__ partials, unsigned int *counter,
                             double *__restrict__ out, int *status) {
    __shared__ double red[32];
    __shared__ bool last;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = gtid; j < nd; j += stride) {
        const double d = Ax[j] - b[j];
        s[0] += d * d;
        s[3] += b[j] * y[j];
    }
    for (int64_t i = gtid; i < np; i += stride) {
        const double d = ATy[i] + z[i] - c[i];
        s[1] += d * d;
        s[2] += c[i] * x[i];
    }
    for (int k = 0; k < 4; k++) {
        const double v = block_sum(s[k], red);
        if (threadIdx.x == 0) partials[k * gridDim.x + blockIdx.x] = v;
    }
    __threadfence();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = 0; k < 4; k++) {
        double v = 0.0;
        if (threadIdx.x < 32) {
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32)
                v += *((volatile double *)(partials + k * gridDim.x + i));
            v = warp_sum(v);
        }
        if (threadIdx.x == 0) {
            out[k] = v;
            if (!(v == v) || v - v != 0.0) atomicExch(status, kStatusNan);
        }
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// --------------------------------------------------------- projection

// One CTA per PSD block (n <= kJacobiMaxDim): selective parallel cyclic
// Jacobi on T = V^T U V, where the rows of Vt (= V^T) are the previous
// iteration's eigenvectors (the identity on a cold start).
//
// A pair (p, q) is rotated (sym.schur2, Golub & Van Loan sec. 8.5) only when
// the first-order (Daleckii-Krein) projection formula could not settle it:
//     t_pq^2 > gap_tol * ||T||_F * |t_pp - t_qq|   and   |t_pq| > abs_tol * ||T||_F.
// Sweeps repeat until a sweep rotates nothing.  The kernel then writes the
// middle factor of U+ = V P V^T,
//     P_ii = max(t_ii, 0),   P_ij = t_ij (t_ii+ - t_jj+) / (t_ii - t_jj)   (i != j),
// (with raw != 0: the rotated T itself, for callers that want eigenvalues)
// and replays the recorded rotations on Vt (rows p, q of Vt per rotation),
// leaving the refined eigenvectors for the next iteration.
__global__ void __launch_bounds__(kJacobiThreads)
    jacobi_warm_kernel(const double *__restrict__ T0, double *__restrict__ Pout,
                       double *__restrict__ Vt, const int64_t *__restrict__ boff,
                       const int *__restrict__ bdim, double2 *__restrict__ rot,
                       const int64_t *__restrict__ rot_off, int max_sweeps, double abs_tol,
                       double gap_tol, int *status, int *rot_count, int raw) {
    extern __shared__ double sm[];
    const int blk = blockIdx.x;
    const int n = bdim[blk];
    if (n <= 0) return;
    const int64_t off = boff[blk];
    const int np = n + (n & 1);
    const int m = np / 2;
    double *T = sm;                                   // np*np (later: Vt)
    double2 *cs = (double2 *)(T + (size_t)np * np);   // m
    int *act = (int *)(cs + m);                       // m
    int *alist = act + m;                             // m
    __shared__ double red[32];
    __shared__ int nrot, nstep;
    __shared__ double s_nrm;

    const double *Tb = T0 + off;
    double fro = 0.0;
    for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int i = e / np, j = e % np;
        double v = 0.0;
        if (i < n && j < n) v = 0.5 * (Tb[(int64_t)i * n + j] + Tb[(int64_t)j * n + i]);
        T[e] = v;
        fro += v * v;
    }
    fro = block_sum(fro, red);
    if (threadIdx.x == 0) s_nrm = sqrt(fro);
    __syncthreads();
    const double nrm = s_nrm;
    const double atol = abs_tol * nrm + 1e-300, gtol = gap_tol * nrm;

    double2 *rb = rot + rot_off[blk];
    // per-step rotation counts live after the block's rotation record
    int *scount = (int *)(rb + (int64_t)max_sweeps * (np - 1) * m);
    int sweep = 0, total = 0;
    for (; sweep < max_sweeps; sweep++) {
        if (threadIdx.x == 0) nrot = 0;
        __syncthreads();
        for (int st = 0; st < np - 1; st++) {
            if (threadIdx.x == 0) nstep = 0;
            __syncthreads();
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                int p, q;
                rr_pair(st, k, np, p, q);
                double c = 1.0, s = 0.0;
                int a = 0;
                if (q < n) {
                    const double apq = T[p * np + q];
                    const double app = T[p * np + p], aqq = T[q * np + q];
                    if (fabs(apq) > atol && apq * apq > gtol * fabs(aqq - app)) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        a = 1;
                        atomicAdd(&nstep, 1);
                    }
                }
                cs[k] = make_double2(c, s);
                act[k] = a;
                rb[((int64_t)sweep * (np - 1) + st) * m + k] = make_double2(c, s);
            }
            __syncthreads();
            const int active = nstep;
            if (threadIdx.x == 0) nrot += active;
            if (active) {
                // compact list of the rotated pairs of this step (warp 0, ballots)
                if (threadIdx.x < 32) {
                    const int lane = threadIdx.x;
                    int base = 0;
                    for (int k0 = 0; k0 < m; k0 += 32) {
                        const int k = k0 + lane;
                        const int a = (k < m) ? act[k] : 0;
                        const unsigned bal = __ballot_sync(0xffffffffu, a);
                        if (a) alist[base + __popc(bal & ((1u << lane) - 1u))] = k;
                        base += __popc(bal);
                    }
                }
                __syncthreads();
                // 2x2 blocks (P, Q) with P rotated; a block with both P and Q
                // rotated is handled once, by the smaller of the two
                for (int it = threadIdx.x; it < active * m; it += blockDim.x) {
                    const int P = alist[it / m], Q = it % m;
                    if (act[Q] && Q < P) continue;
                    const double2 cp = cs[P], cq = cs[Q];
                    int pP, qP, pQ, qQ;
                    rr_pair(st, P, np, pP, qP);
                    rr_pair(st, Q, np, pQ, qQ);
                    const double b11 = T[pP * np + pQ], b12 = T[pP * np + qQ];
                    const double b21 = T[qP * np + pQ], b22 = T[qP * np + qQ];
                    const double m11 = b11 * cq.x - b12 * cq.y, m12 = b11 * cq.y + b12 * cq.x;
                    const double m21 = b21 * cq.x - b22 * cq.y, m22 = b21 * cq.y + b22 * cq.x;
                    double n11 = cp.x * m11 - cp.y * m21, n12 = cp.x * m12 - cp.y * m22;
                    double n21 = cp.y * m11 + cp.x * m21, n22 = cp.y * m12 + cp.x * m22;
                    if (P == Q) {
                        n12 = 0.0;
                        n21 = 0.0;
                        T[pP * np + pP] = n11;
                        T[pP * np + qP] = n12;
                        T[qP * np + pP] = n21;
                        T[qP * np + qP] = n22;
                    } else {
                        T[pP * np + pQ] = n11; T[pQ * np + pP] = n11;
                        T[pP * np + qQ] = n12; T[qQ * np + pP] = n12;
                        T[qP * np + pQ] = n21; T[pQ * np + qP] = n21;
                        T[qP * np + qQ] = n22; T[qQ * np + qP] = n22;
                    }
                }
            }
            if (threadIdx.x == 0) scount[(int64_t)sweep * (np - 1) + st] = active;
            __syncthreads();
        }
        total += nrot;
        const int done = (nrot == 0);
        __syncthreads();
        if (done) {
            sweep++;
            break;
        }
    }
    if (threadIdx.x == 0) {
        if (rot_count) atomicAdd(rot_count, total);
        if (sweep >= max_sweeps && nrot != 0) atomicAdd(status, 1);   // sweeps exhausted
    }

    // middle factor P of U+ = V P V^T (first-order in the remaining couplings)
    double *Pb = Pout + off;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e % n;
        const double li = T[i * np + i];
        double pv;
        if (raw) {
            pv = T[i * np + j];   // the rotated matrix itself (its diagonal: the eigenvalues)
        } else if (i == j) {
            pv = fmax(li, 0.0);
        } else {
            const double lj = T[j * np + j];
            const double pi = fmax(li, 0.0), pj = fmax(lj, 0.0);
            const double gam = (li != lj) ? (pi - pj) / (li - lj) : (li > 0.0 ? 1.0 : 0.0);
            pv = gam * T[i * np + j];
        }
        Pb[e] = pv;
    }
    __syncthreads();

    // replay the rotations on Vt (rows = eigenvectors)
    double *V = T;
    double *Vb = Vt + off;
    for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int i = e / np, j = e % np;
        V[e] = (i < n && j < n) ? Vb[(int64_t)i * n + j] : (i == j ? 1.0 : 0.0);
    }
    __syncthreads();
    for (int sw = 0; sw < sweep; sw++) {
        for (int st = 0; st < np - 1; st++) {
            if (scount[(int64_t)sw * (np - 1) + st] == 0) continue;   // uniform across the CTA
            const double2 *rs = rb + ((int64_t)sw * (np - 1) + st) * m;
            if (threadIdx.x < 32) {
                const int lane = threadIdx.x;
                int base = 0;
                for (int k0 = 0; k0 < m; k0 += 32) {
                    const int k = k0 + lane;
                    const int a = (k < m) ? (rs[k].y != 0.0) : 0;
                    const unsigned bal = __ballot_sync(0xffffffffu, a);
                    if (a) alist[base + __popc(bal & ((1u << lane) - 1u))] = k;
                    base += __popc(bal);
                }
                if (lane == 0) nstep = base;
            }
            __syncthreads();
            const int active = nstep;
            for (int it = threadIdx.x; it < active * np; it += blockDim.x) {
                const int k = alist[it / np], j = it % np;
                const double2 r = rs[k];
                int p, q;
                rr_pair(st, k, np, p, q);
                const double vp = V[p * np + j], vq = V[q * np + j];
                V[p * np + j] = r.x * vp - r.y * vq;
                V[q * np + j] = r.y * vp + r.x * vq;
            }
            __syncthreads();
        }
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e % n;
        Vb[e] = V[i * np + j];
    }
}

// Vt <- identity on every block (cold start of the warm path)
__global__ void identity_blocks_kernel(double *__restrict__ Vt, const int64_t *__restrict__ boff,
                                       const int *__restrict__ bdim) {
    const int n = bdim[blockIdx.x];
    const int64_t off = boff[blockIdx.x];
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x)
        Vt[off + e] = (e / n == e % n) ? 1.0 : 0.0;
}

// H = (I - G) / 2 for the re-orthonormalisation Vt <- Vt + H Vt
__global__ void half_residual_kernel(const double *__restrict__ G, double *__restrict__ H,
                                     const int64_t *__restrict__ boff, const int *__restrict__ bdim) {
    const int n = bdim[blockIdx.x];
    const int64_t off = boff[blockIdx.x];
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x)
        H[off + e] = 0.5 * (((e / n == e % n) ? 1.0 : 0.0) - G[off + e]);
}

cudaError_t raise_dynamic_smem(const void *func, int bytes) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, func);
    if (e == cudaSuccess && fa.maxDynamicSharedSizeBytes < bytes)
        e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

unsigned long long current_context_id() {
    // driver entry points through the runtime: no link-time libcuda dependency
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static const std::pair<GetCurrent, GetId> fn = [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess)
            a = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qb != cudaDriverEntryPointSuccess)
            b = nullptr;
        return std::make_pair((GetCurrent)a, (GetId)b);
    }();
    if (!fn.first || !fn.second) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (fn.first(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (fn.second(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

}  // namespace v2b
