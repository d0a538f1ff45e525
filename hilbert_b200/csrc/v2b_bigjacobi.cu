// Selective Jacobi for PSD blocks too large for one CTA's shared memory
// (n > kJacobiMaxDim), e.g. the 190 / 400 / 800-row blocks of a (20e,20o)
// active space.  One thread-block cluster of kBigCluster CTAs works on one
// block; T = V^T U V stays in global memory (L2-resident).
//
// The schedule is the shared-memory kernel's: parallel cyclic Jacobi with the
// round-robin pairing (every index once per step, every pair once per sweep),
// rotating only the pairs the first-order projection formula cannot settle
//     t_pq^2 > gap_tol ||T||_F |t_pp - t_qq|   and   |t_pq| > abs_tol ||T||_F,
// with sym.schur2 rotations (Golub & Van Loan sec. 8.5).  Per step:
//   A. the pairs' rotations are computed (spread over the cluster's CTAs) and
//      recorded; B. every 2 x 2 block touched by a rotation is updated
//      two-sided, each element once.  The cluster's hardware barrier separates
//      A, B and the next step.
// Sweeps repeat until one rotates nothing.  Then the middle factor P of
// U+ = V P V^T is written and the recorded rotations are replayed onto Vt.
// Data other CTAs wrote in an earlier phase are read with __ldcg (L2), as the
// per-SM L1 is not coherent across the cluster.
#include <cooperative_groups.h>

#include "v2b_bigjacobi.cuh"

namespace cg = cooperative_groups;

namespace v2b {

// The body, for T stored as R: double (jacobi_big_kernel, in place in a.T)
// or float (jacobi_big32_kernel: T32 is the working copy, filled from a.T).
// Rotation parameters are computed in double from the stored elements and
// recorded as double pairs (exactly orthogonal to double rounding), so the
// replay keeps the rows of Vt orthonormal whatever R is; the two-sided
// updates of T run in R.
template <typename R>
__device__ __forceinline__ void jacobi_big_body(const BigJacobiArgs &a, R *Tall) {
    cg::cluster_group cl = cg::this_cluster();
    const int blk = blockIdx.x / kBigCluster;
    const int rank = (int)cl.block_rank();
    const int n = a.bdim[blk];
    if (n <= 0) return;   // uniform over the cluster
    const int np = n + (n & 1), m = np / 2, nsteps = np - 1;
    R *T = Tall + a.boff[blk];
    const double *T0 = a.T + a.boff[blk];
    double *P = a.P + a.boff[blk];
    double *Vt = a.Vt + a.boff[blk];
    double2 *rec = a.rot + a.roff[blk];                          // sweeps x steps x m
    int *scount = (int *)(rec + (int64_t)a.max_sweeps * nsteps * m);  // sweeps x steps
    int *sweep_total = scount + (int64_t)a.max_sweeps * nsteps;      // sweeps
    double *npart = a.norm_part + (int64_t)blk * kBigCluster;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    const int r0 = (int)((int64_t)rank * n / kBigCluster), r1 = (int)((int64_t)(rank + 1) * n / kBigCluster);
    const int64_t ctid = (int64_t)rank * blockDim.x + tid, cstride = (int64_t)kBigCluster * blockDim.x;
    extern __shared__ int alist[];   // m entries
    __shared__ double red[32];
    __shared__ int s_cnt;

    // symmetrise (the owner of row i averages (i, j) with (j, i) for j > i),
    // clear the step counters, Frobenius norm
    double fro = 0.0;
    for (int i = r0 + warp; i < r1; i += nwarp) {
        for (int j = i + 1 + lane; j < n; j += 32) {
            const R v = (R)(0.5 * (T0[(int64_t)i * n + j] + T0[(int64_t)j * n + i]));
            T[(int64_t)i * n + j] = v;
            T[(int64_t)j * n + i] = v;
            fro += 2.0 * (double)v * (double)v;
        }
        if (lane == 0) {
            const R d = (R)T0[(int64_t)i * n + i];
            T[(int64_t)i * n + i] = d;
            fro += (double)d * (double)d;
        }
    }
    for (int64_t r = ctid; r < (int64_t)a.max_sweeps * (nsteps + 1); r += cstride) scount[r] = 0;
    fro = block_sum(fro, red);
    if (tid == 0) npart[rank] = fro;
    cl.sync();
    double nrm2 = 0.0;
    for (int k = 0; k < kBigCluster; k++) nrm2 += __ldcg(npart + k);
    const double nrm = sqrt(nrm2);
    const double atol = a.abs_tol * nrm + 1e-300, gtol = a.gap_tol * nrm;

    int sweep = 0;
    bool done = false;
    for (; sweep < a.max_sweeps && !done; sweep++) {
        for (int st = 0; st < nsteps; st++) {
            double2 *rs = rec + ((int64_t)sweep * nsteps + st) * m;
            int *cnt = scount + (int64_t)sweep * nsteps + st;
            // A: rotations of this step's pairs
            for (int64_t k = ctid; k < m; k += cstride) {
                int p, q;
                rr_pair(st, (int)k, np, p, q);
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = (double)__ldcg(T + (int64_t)p * n + q);
                    const double app = (double)__ldcg(T + (int64_t)p * n + p);
                    const double aqq = (double)__ldcg(T + (int64_t)q * n + q);
                    if (fabs(apq) > atol && apq * apq > gtol * fabs(aqq - app)) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        atomicAdd(cnt, 1);
                        atomicAdd(sweep_total + sweep, 1);
                    }
                }
                rs[k] = make_double2(c, s);
            }
            cl.sync();
            if (__ldcg(cnt) == 0) continue;   // uniform: nothing to apply, next step
            // active list of this step (every CTA builds its own copy)
            if (warp == 0) {
                int base = 0;
                for (int k0 = 0; k0 < m; k0 += 32) {
                    const int k = k0 + lane;
                    const int act = (k < m) ? (__ldcg(&rs[k].y) != 0.0) : 0;
                    const unsigned bal = __ballot_sync(0xffffffffu, act);
                    if (act) alist[base + __popc(bal & ((1u << lane) - 1u))] = k;
                    base += __popc(bal);
                }
                if (lane == 0) s_cnt = base;
            }
            __syncthreads();
            const int active = s_cnt;
            // B: 2x2 blocks (P, Q) with P rotated; both rotated -> handled by the smaller
            for (int64_t it = ctid; it < (int64_t)active * m; it += cstride) {
                const int Pk = alist[it / m], Qk = (int)(it % m);
                const double2 cq = __ldcg(rs + Qk);
                if (cq.y != 0.0 && Qk < Pk) continue;
                const double2 cp = __ldcg(rs + Pk);
                int pP, qP, pQ, qQ;
                rr_pair(st, Pk, np, pP, qP);
                rr_pair(st, Qk, np, pQ, qQ);
                const bool qPin = qP < n, qQin = qQ < n;   // n odd: index n is padding
                const R cqx = (R)cq.x, cqy = (R)cq.y, cpx = (R)cp.x, cpy = (R)cp.y;
                const R b11 = __ldcg(T + (int64_t)pP * n + pQ);
                const R b12 = qQin ? __ldcg(T + (int64_t)pP * n + qQ) : (R)0;
                const R b21 = qPin ? __ldcg(T + (int64_t)qP * n + pQ) : (R)0;
                const R b22 = (qPin && qQin) ? __ldcg(T + (int64_t)qP * n + qQ) : (R)0;
                const R m11 = b11 * cqx - b12 * cqy, m12 = b11 * cqy + b12 * cqx;
                const R m21 = b21 * cqx - b22 * cqy, m22 = b21 * cqy + b22 * cqx;
                const R n11 = cpx * m11 - cpy * m21, n12 = cpx * m12 - cpy * m22;
                const R n21 = cpy * m11 + cpx * m21, n22 = cpy * m12 + cpx * m22;
                if (Pk == Qk) {
                    T[(int64_t)pP * n + pP] = n11;
                    T[(int64_t)qP * n + qP] = n22;
                    T[(int64_t)pP * n + qP] = (R)0;
                    T[(int64_t)qP * n + pP] = (R)0;
                } else {
                    T[(int64_t)pP * n + pQ] = n11; T[(int64_t)pQ * n + pP] = n11;
                    if (qQin) { T[(int64_t)pP * n + qQ] = n12; T[(int64_t)qQ * n + pP] = n12; }
                    if (qPin) { T[(int64_t)qP * n + pQ] = n21; T[(int64_t)pQ * n + qP] = n21; }
                    if (qPin && qQin) { T[(int64_t)qP * n + qQ] = n22; T[(int64_t)qQ * n + qP] = n22; }
                }
            }
            cl.sync();
        }
        done = (__ldcg(sweep_total + sweep) == 0);
        cl.sync();
    }
    if (rank == 0 && tid == 0) {
        int tot = 0;
        for (int sw = 0; sw < sweep; sw++) tot += sweep_total[sw];
        atomicAdd(a.counters + 1, tot);
        if (!done) atomicAdd(a.counters, 1);
    }

    // middle factor P of U+ = V P V^T
    for (int64_t e = ctid; e < (int64_t)n * n; e += cstride) {
        const int i = (int)(e / n), j = (int)(e % n);
        const double li = (double)__ldcg(T + (int64_t)i * n + i);
        double pv;
        if (i == j) {
            pv = fmax(li, 0.0);
        } else {
            const double lj = (double)__ldcg(T + (int64_t)j * n + j);
            const double pi = fmax(li, 0.0), pj = fmax(lj, 0.0);
            const double gam = (li != lj) ? (pi - pj) / (li - lj) : (li > 0.0 ? 1.0 : 0.0);
            pv = gam * (double)__ldcg(T + e);
        }
        P[e] = pv;
    }
    // replay the recorded rotations onto the rows of Vt
    for (int sw = 0; sw < sweep; sw++) {
        for (int st = 0; st < nsteps; st++) {
            if (__ldcg(scount + (int64_t)sw * nsteps + st) == 0) continue;
            const double2 *rs = rec + ((int64_t)sw * nsteps + st) * m;
            if (warp == 0) {
                int base = 0;
                for (int k0 = 0; k0 < m; k0 += 32) {
                    const int k = k0 + lane;
                    const int act = (k < m) ? (__ldcg(&rs[k].y) != 0.0) : 0;
                    const unsigned bal = __ballot_sync(0xffffffffu, act);
                    if (act) alist[base + __popc(bal & ((1u << lane) - 1u))] = k;
                    base += __popc(bal);
                }
                if (lane == 0) s_cnt = base;
            }
            __syncthreads();
            const int active = s_cnt;
            for (int64_t it = ctid; it < (int64_t)active * n; it += cstride) {
                const int k = alist[it / n], j = (int)(it % n);
                int p, q;
                rr_pair(st, k, np, p, q);
                const double2 r2 = __ldcg(rs + k);
                const double vp = __ldcg(Vt + (int64_t)p * n + j), vq = __ldcg(Vt + (int64_t)q * n + j);
                Vt[(int64_t)p * n + j] = r2.x * vp - r2.y * vq;
                Vt[(int64_t)q * n + j] = r2.y * vp + r2.x * vq;
            }
            cl.sync();
        }
    }
}

__global__ void __cluster_dims__(kBigCluster, 1, 1) __launch_bounds__(kBigThreads)
    jacobi_big_kernel(BigJacobiArgs a) {
    jacobi_big_body<double>(a, a.T);
}

__global__ void __cluster_dims__(kBigCluster, 1, 1) __launch_bounds__(kBigThreads)
    jacobi_big32_kernel(BigJacobiArgs a, float *T32) {
    jacobi_big_body<float>(a, T32);
}

}  // namespace v2b
