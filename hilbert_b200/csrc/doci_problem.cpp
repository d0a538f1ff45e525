// v2RDM-DOCI sizes, b and c (see doci_problem.h for the rows of A).
#include "doci_problem.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace v2b {

Problem make_doci_problem(const ProblemSpec &spec) {
    if (spec.nmo < 1 || spec.nalpha < 0 || spec.nbeta < 0 || spec.nalpha > spec.nmo ||
        spec.nbeta > spec.nmo)
        throw std::invalid_argument("invalid orbital / electron counts");
    if (spec.positivity < POS_D || spec.positivity > POS_DQGT1T2)
        throw std::invalid_argument("unsupported POSITIVITY");
    if (spec.constrain_q3 || spec.constrain_e3 || spec.constrain_f3 || spec.constrain_d4)
        throw std::invalid_argument("v2RDM-DOCI has no Q3, E3, F3 or D4 conditions");
    Problem p;
    p.spec = spec;
    const int64_t n = spec.nmo;
    p.n = (int)n;
    // v2rdm_doci_solver.cc:427-494.  The second "DQGT2" branch there is never
    // reached: DQGT2 is D, Q, G and T2.
    p.q2 = spec.positivity == POS_DQ || spec.positivity >= POS_DQG;
    p.g2 = spec.positivity == POS_DG || spec.positivity >= POS_DQG;
    p.t1 = spec.positivity == POS_DQGT1 || spec.positivity == POS_DQGT1T2;
    p.t2 = spec.positivity == POS_DQGT2 || spec.positivity == POS_DQGT1T2;
    p.d3 = spec.constrain_d3;
    if ((p.d3 || p.t1) && n < 2)
        throw std::invalid_argument("DOCI D3 and T1 need at least two orbitals (blocks of n - 1)");
    const int64_t pairs = n * (n - 1) / 2, trip = n * (n - 1) * (n - 2) / 6, w = 2 * n - 1;

    // offsets and blocks, v2rdm_doci_solver.cc:542-600 and 649-700
    DociOffsets &o = p.doci;
    int64_t off = 0;
    auto blocks = [&](int64_t count, int dim) {
        for (int64_t k = 0; k < count; k++) {
            p.dims.push_back(dim);
            p.block_off.push_back(off);
            off += (int64_t)dim * dim;
        }
    };
    o.d2s2 = off; blocks(n * n, 1);
    o.d2s0 = off; blocks(1, (int)n);
    o.d1 = off;   blocks(n, 1);
    if (p.q2) {
        o.q2s2 = off; blocks(pairs, 1);
        o.q2s0 = off; blocks(1, (int)n);
    }
    if (p.g2) {
        o.g2s2 = off; blocks(pairs, 2);
        o.g2s0 = off; blocks(1, (int)n);
    }
    if (p.d3) {
        o.d3s3 = off; blocks(n * n * n, 1);
        o.d3s1 = off; blocks(n, (int)n - 1);
    }
    if (p.t1) {
        o.t1aaa = off; blocks(trip, 1);
        o.t1aab = off; blocks(n * pairs, 1);
        o.t1s1 = off;  blocks(n, (int)n - 1);
    }
    if (p.t2) {
        o.t2s1 = off; blocks(n, (int)w);
        o.t2 = off;   blocks(trip, 3);
    }
    p.n_primal = off;

    // constraints, v2rdm_doci_solver.cc:602-646
    int64_t d = 3 + 3 * n + n * n;
    if (p.q2) d += pairs + n * n;
    if (p.g2) d += 4 * pairs + n * n;
    if (p.d3) d += 3 * n * (n - 1) + n * n;
    if (p.t1) d += trip + n * pairs + n * (n - 1) * (n - 1);
    if (p.t2) d += n * w * w + 9 * trip;
    p.n_dual = d;
    if (p.n_primal > (int64_t)kColMask || p.n_dual > (int64_t)kColMask)
        throw std::invalid_argument("problem too large for 27-bit packed column indices");
    // the ab / aa geminal tables: DOCI's BuildBasis numbers them with the same
    // loops as the v2RDM basis (src/v2rdm_doci/basis.cc:425-535)
    ProblemSpec t;
    t.nmo = (int)n;
    t.positivity = POS_D;
    const Problem tab = make_problem(t);
    p.gab = tab.gab;
    p.gaa = tab.gaa;
    p.bas_ab = tab.bas_ab;
    p.ibas_ab = tab.ibas_ab;
    p.bas_aa = tab.bas_aa;
    p.ibas_aa = tab.ibas_aa;
    return p;
}

int64_t doci_v2rdm_layout_size(const Problem &p) {
    return (int64_t)p.gab * p.gab + 2 * (int64_t)p.gaa * p.gaa + 2 * (int64_t)p.n * p.n;
}

void doci_v2rdm_layout(const Problem &p, const double *x, double *out) {
    // v2rdm_doci_solver.cc:1570-1597 builds D2aa (= D2bb) and D2ab from the
    // seniority blocks; D1 is diagonal, the same for both spins (:1693-1700)
    const int64_t n = p.n, gab = p.gab, gaa = p.gaa;
    const int64_t ab = 0, aa = gab * gab, bb = aa + gaa * gaa, d1a = bb + gaa * gaa, d1b = d1a + n * n;
    const DociOffsets &o = p.doci;
    std::memset(out, 0, sizeof(double) * doci_v2rdm_layout_size(p));
    for (int64_t g = 0; g < gaa; g++) {
        // the reference's aa pair (i, j) has i > j (basis.cc:520-526)
        const int64_t i = std::max(p.bas_aa[2 * g], p.bas_aa[2 * g + 1]);
        const int64_t j = std::min(p.bas_aa[2 * g], p.bas_aa[2 * g + 1]);
        out[aa + g * gaa + g] = x[o.d2s2 + i * n + j];
        out[bb + g * gaa + g] = x[o.d2s2 + i * n + j];
    }
    for (int64_t g = 0; g < gab; g++) {
        const int64_t i = p.bas_ab[2 * g], j = p.bas_ab[2 * g + 1];
        if (i != j) out[ab + g * gab + g] = x[o.d2s2 + i * n + j];
    }
    for (int64_t i = 0; i < n; i++)
        for (int64_t j = 0; j < n; j++)
            out[ab + (int64_t)p.iab((int)i, (int)i) * gab + p.iab((int)j, (int)j)] = x[o.d2s0 + i * n + j];
    for (int64_t i = 0; i < n; i++) {
        out[d1a + i * n + i] = x[o.d1 + i];
        out[d1b + i * n + i] = x[o.d1 + i];
    }
}

void doci_build_b(const Problem &p, double *b) {
    // v2rdm_doci_solver.cc:1338-1507
    const int n = p.n;
    const double na = p.spec.nalpha;
    std::memset(b, 0, sizeof(double) * p.n_dual);
    int64_t off = 0;
    b[off++] = na * (na - 1.0);
    b[off++] = na;
    b[off++] = na;
    off += 3 * (int64_t)n + (int64_t)n * n;
    if (p.q2) {
        for (int64_t k = 0; k < (int64_t)n * (n - 1) / 2; k++) b[off++] = -1.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) b[off++] = -1.0 * (double)(i == j);
    }
    if (p.g2) off += 2 * (int64_t)n * (n - 1) + (int64_t)n * n;
    if (p.d3) off += 3 * (int64_t)n * (n - 1) + (int64_t)n * n;
    if (p.t1) {
        const int64_t ones = (int64_t)n * (n - 1) * (n - 2) / 6 + (int64_t)n * n * (n - 1) / 2;
        for (int64_t k = 0; k < ones; k++) b[off++] = 1.0;
        for (int bb = 0; bb < n; bb++)
            for (int a = 0; a < n; a++) {
                if (a == bb) continue;
                for (int c = 0; c < n; c++) {
                    if (c == bb) continue;
                    b[off++] = (double)(a == c);
                }
            }
    }
}

void doci_build_c_external(const Problem &p, const double *h, const double *g, double *c) {
    // RepackIntegrals, tei.cc:127-153: TEI(i,j,k,l) = (ij|kl) and the diagonal
    // of h (the packed buffer's INDEX(i,i), tei.cc:98-106)
    const int64_t n = p.n;
    const DociOffsets &o = p.doci;
    std::memset(c, 0, sizeof(double) * p.n_primal);
    const double f = 2.0 / ((double)(p.spec.nalpha + p.spec.nbeta) - 1.0);
    auto tei = [&](int64_t i, int64_t j, int64_t k, int64_t l) { return g[((i * n + j) * n + k) * n + l]; };
    for (int64_t i = 0; i < n; i++)
        for (int64_t j = 0; j < n; j++) {
            double &s2 = c[o.d2s2 + i * n + j];
            if (i != j) {
                s2 = 2.0 * tei(i, i, j, j);
                s2 -= tei(i, j, i, j);
                s2 += f * (h[i * n + i] + h[j * n + j]);
            }
            double &s0 = c[o.d2s0 + i * n + j];
            s0 = tei(i, j, i, j);
            s0 += f * (double)(i == j) * h[i * n + i];
        }
}

}  // namespace v2b
