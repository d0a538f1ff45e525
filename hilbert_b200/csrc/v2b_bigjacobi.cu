// Selective Jacobi for PSD blocks too large for one CTA's shared memory
// (n > kJacobiMaxDim), e.g. the 190 / 400 / 800-row blocks of a (20e,20o)
// active space.  One thread-block cluster of kBigCluster CTAs works on one
// block; T = V^T U V stays in global memory (L2-resident) and the cluster's
// hardware barrier separates the phases of each round:
//
//   A. every row i picks its best partner j: the largest |t_ij| among the
//      pairs the first-order projection formula cannot settle
//      (t_ij^2 > gap_tol ||T||_F |t_ii - t_jj| and |t_ij| > abs_tol ||T||_F);
//   B. mutual best pairs (partner[partner[i]] == i) form a matching; each
//      gets a sym.schur2 rotation (Golub & Van Loan sec. 8.5), appended to the
//      block's rotation log;
//   C. all rotations of the round are applied two-sided to T (each element
//      touched once: 2 x 2 blocks between rotated pairs, row pairs against
//      unrotated indices, with mirrored writes);
//
// until a round finds no pair (the global largest needed |t_ij| is always a
// mutual pair, so every round makes progress).  Then the middle factor P of
// U+ = V P V^T is written, and the log is replayed onto Vt round by round.
// A block whose log fills up stops early and is counted in counters[0]; its
// basis is still orthogonal, so the next call continues from it.  Data other
// CTAs of the cluster wrote in an earlier phase are read with __ldcg (L2), as
// the per-SM L1 is not coherent across the cluster.
#include <cooperative_groups.h>

#include "v2b_bigjacobi.cuh"

namespace cg = cooperative_groups;

namespace v2b {

__device__ __forceinline__ bool needed_pair(double t, double tii, double tjj, double atol,
                                            double gtol) {
    return fabs(t) > atol && t * t > gtol * fabs(tii - tjj);
}

__global__ void __cluster_dims__(kBigCluster, 1, 1) __launch_bounds__(kBigThreads)
    jacobi_big_kernel(BigJacobiArgs a) {
    cg::cluster_group cl = cg::this_cluster();
    const int blk = blockIdx.x / kBigCluster;
    const int rank = (int)cl.block_rank();
    const int n = a.bdim[blk];
    if (n <= 0) return;   // uniform over the cluster
    double *T = a.T + a.boff[blk];
    double *P = a.P + a.boff[blk];
    double *Vt = a.Vt + a.boff[blk];
    double *dg = a.diag + a.ioff[blk];
    int *partner = a.partner + a.ioff[blk];
    int *act = a.act + a.ioff[blk];
    double2 *acs = a.acs + a.ioff[blk];
    int2 *log_pq = a.log_pq + a.loff[blk];
    double2 *log_cs = a.log_cs + a.loff[blk];
    int *rcnt = a.round_cnt + (int64_t)blk * a.max_rounds;
    double *npart = a.norm_part + (int64_t)blk * kBigCluster;
    const int64_t cap = a.lcap[blk];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    const int r0 = (int)((int64_t)rank * n / kBigCluster), r1 = (int)((int64_t)(rank + 1) * n / kBigCluster);
    const int64_t ctid = (int64_t)rank * blockDim.x + tid, cstride = (int64_t)kBigCluster * blockDim.x;
    __shared__ double red[32];

    // symmetrise (the owner of row i averages (i, j) with (j, i) for j > i),
    // copy the diagonal, clear the round counters, Frobenius norm
    double fro = 0.0;
    for (int i = r0 + warp; i < r1; i += nwarp) {
        for (int j = i + 1 + lane; j < n; j += 32) {
            const double v = 0.5 * (T[(int64_t)i * n + j] + T[(int64_t)j * n + i]);
            T[(int64_t)i * n + j] = v;
            T[(int64_t)j * n + i] = v;
            fro += 2.0 * v * v;
        }
        if (lane == 0) {
            const double d = T[(int64_t)i * n + i];
            dg[i] = d;
            fro += d * d;
        }
    }
    for (int64_t r = ctid; r < a.max_rounds; r += cstride) rcnt[r] = 0;
    fro = block_sum(fro, red);
    if (tid == 0) npart[rank] = fro;
    cl.sync();
    double nrm2 = 0.0;
    for (int k = 0; k < kBigCluster; k++) nrm2 += __ldcg(npart + k);
    const double nrm = sqrt(nrm2);
    const double atol = a.abs_tol * nrm + 1e-300, gtol = a.gap_tol * nrm;

    int64_t logpos = 0;
    int round = 0;
    bool overrun = false;
    for (; round < a.max_rounds; round++) {
        if (logpos + n / 2 + 1 > cap) {
            overrun = true;
            break;
        }
        // A: best partner of every row
        for (int i = r0 + warp; i < r1; i += nwarp) {
            const double tii = __ldcg(dg + i);
            double bv = 0.0;
            int bj = -1;
            for (int j = lane; j < n; j += 32) {
                if (j == i) continue;
                const double t = __ldcg(T + (int64_t)i * n + j);
                if (needed_pair(t, tii, __ldcg(dg + j), atol, gtol) && fabs(t) > bv) {
                    bv = fabs(t);
                    bj = j;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, o);
                const int oj = __shfl_down_sync(0xffffffffu, bj, o);
                if (oj >= 0 && (ov > bv || (ov == bv && (bj < 0 || oj < bj)))) {
                    bv = ov;
                    bj = oj;
                }
            }
            if (lane == 0) partner[i] = bj;
        }
        cl.sync();
        // B: mutual pairs; both rows store the pair's rotation, the smaller logs it
        for (int i = r0 + tid; i < r1; i += blockDim.x) {
            const int j = __ldcg(partner + i);
            int pj = -1;
            if (j >= 0 && __ldcg(partner + j) == i) {
                pj = j;
                const int p = i < j ? i : j, q = i < j ? j : i;
                const double app = __ldcg(dg + p), aqq = __ldcg(dg + q);
                const double apq = __ldcg(T + (int64_t)p * n + q);
                const double tau = (aqq - app) / (2.0 * apq);
                const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
                const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                acs[i] = make_double2(c, s);
                if (i == p) {
                    const int slot = atomicAdd(rcnt + round, 1);
                    log_pq[logpos + slot] = make_int2(p, q);
                    log_cs[logpos + slot] = make_double2(c, s);
                }
            }
            act[i] = pj;
        }
        cl.sync();
        const int na = __ldcg(rcnt + round);
        if (na == 0) break;
        // C: two-sided update of T by every rotation of the round
        for (int64_t it = ctid; it < (int64_t)na * n; it += cstride) {
            const int k = (int)(it / n), j = (int)(it % n);
            const int2 pq = __ldcg(log_pq + logpos + k);
            const double2 cp = __ldcg(log_cs + logpos + k);
            const int p = pq.x, q = pq.y;
            const int pj = __ldcg(act + j);
            if (pj >= 0) {
                const int p2 = j < pj ? j : pj, q2 = j < pj ? pj : j;
                if (j != p2 || p > p2) continue;   // each 2x2 block once
                const double2 cq = __ldcg(acs + p2);
                const double b11 = __ldcg(T + (int64_t)p * n + p2), b12 = __ldcg(T + (int64_t)p * n + q2);
                const double b21 = __ldcg(T + (int64_t)q * n + p2), b22 = __ldcg(T + (int64_t)q * n + q2);
                const double m11 = b11 * cq.x - b12 * cq.y, m12 = b11 * cq.y + b12 * cq.x;
                const double m21 = b21 * cq.x - b22 * cq.y, m22 = b21 * cq.y + b22 * cq.x;
                double n11 = cp.x * m11 - cp.y * m21, n12 = cp.x * m12 - cp.y * m22;
                double n21 = cp.y * m11 + cp.x * m21, n22 = cp.y * m12 + cp.x * m22;
                if (p == p2) {
                    T[(int64_t)p * n + p] = n11;
                    T[(int64_t)q * n + q] = n22;
                    T[(int64_t)p * n + q] = 0.0;
                    T[(int64_t)q * n + p] = 0.0;
                    dg[p] = n11;
                    dg[q] = n22;
                } else {
                    T[(int64_t)p * n + p2] = n11; T[(int64_t)p2 * n + p] = n11;
                    T[(int64_t)p * n + q2] = n12; T[(int64_t)q2 * n + p] = n12;
                    T[(int64_t)q * n + p2] = n21; T[(int64_t)p2 * n + q] = n21;
                    T[(int64_t)q * n + q2] = n22; T[(int64_t)q2 * n + q] = n22;
                }
            } else {
                const double tp = __ldcg(T + (int64_t)p * n + j), tq = __ldcg(T + (int64_t)q * n + j);
                const double np_ = cp.x * tp - cp.y * tq, nq = cp.y * tp + cp.x * tq;
                T[(int64_t)p * n + j] = np_; T[(int64_t)j * n + p] = np_;
                T[(int64_t)q * n + j] = nq; T[(int64_t)j * n + q] = nq;
            }
        }
        logpos += na;
        cl.sync();
    }
    if (rank == 0 && tid == 0) {
        atomicAdd(a.counters + 1, (int)logpos);
        if (overrun || round >= a.max_rounds) atomicAdd(a.counters, 1);
    }

    // middle factor P of U+ = V P V^T
    for (int64_t e = ctid; e < (int64_t)n * n; e += cstride) {
        const int i = (int)(e / n), j = (int)(e % n);
        const double li = __ldcg(dg + i);
        double pv;
        if (i == j) {
            pv = fmax(li, 0.0);
        } else {
            const double lj = __ldcg(dg + j);
            const double pi = fmax(li, 0.0), pj = fmax(lj, 0.0);
            const double gam = (li != lj) ? (pi - pj) / (li - lj) : (li > 0.0 ? 1.0 : 0.0);
            pv = gam * __ldcg(T + e);
        }
        P[e] = pv;
    }
    // replay the log onto the rows of Vt, round by round
    int64_t pos = 0;
    for (int r = 0; r < round; r++) {
        const int na = __ldcg(rcnt + r);
        for (int64_t it = ctid; it < (int64_t)na * n; it += cstride) {
            const int k = (int)(it / n), j = (int)(it % n);
            const int2 pq = __ldcg(log_pq + pos + k);
            const double2 r2 = __ldcg(log_cs + pos + k);
            const double vp = __ldcg(Vt + (int64_t)pq.x * n + j), vq = __ldcg(Vt + (int64_t)pq.y * n + j);
            Vt[(int64_t)pq.x * n + j] = r2.x * vp - r2.y * vq;
            Vt[(int64_t)pq.y * n + j] = r2.y * vp + r2.x * vq;
        }
        pos += na;
        cl.sync();
    }
}

}  // namespace v2b
