// The density-matrix records hilbert writes after a v2RDM solve, built from
// the primal vector on the host: the same records, in the same order, with
// the same values as
//   WriteTPDM          src/v2rdm_casscf/write_tpdm.cc:40-310   (D2aa, D2bb, D2ab)
//   WriteTPDMSpinFree  src/v2rdm_casscf/write_tpdm.cc:312-519  (D2)
//   WriteOPDM          src/v2rdm_casscf/write_opdm.cc:40-114   (D1a, D1b)
//   WriteTPDM_IWL      src/v2rdm_casscf/write_tpdm_iwl.cc:45-205 (IWL labels)
//   WriteActive3PDM    src/v2rdm_casscf/write_3pdm.cc:50-206   (D3aaa, D3aab, D3bba, D3bbb)
// for C1 with ncore doubly occupied (restricted) orbitals numbered 0 ..
// ncore-1 ahead of the active ones (active orbital i is ncore + i); and as
// v2RDM-DOCI's WriteTPDM (src/v2rdm_doci/write_tpdm.cc:47-176) for a DOCI
// problem (no core).
#include "rdm_records.h"

#include <stdexcept>
#include <vector>

#include "doci_problem.h"

namespace v2b {

namespace {
void check(const Problem &p, int ncore) {
    if (p.spec.batch_parts) throw std::invalid_argument("density records of a batch: ask each part");
    if (ncore < 0) throw std::invalid_argument("ncore must be >= 0");
    if (p.spec.doci && ncore) throw std::invalid_argument("v2RDM-DOCI writes no core records");
}

struct Blocks {   // where the spin blocks sit in the vector the records read
    int64_t d2ab, d2aa, d2bb, d1a, d1b;
};

// a record sink that counts when given no array
struct Out {
    TpdmRecord *r;
    int64_t n = 0;
    void put(int i, int j, int k, int l, double v) {
        if (r) r[n] = TpdmRecord{i, j, k, l, v};
        n++;
    }
};

void records(const Problem &p, const double *x, const Blocks &o, int ncore, TpdmRecord *d2aa,
             TpdmRecord *d2bb, TpdmRecord *d2ab, TpdmRecord *d2, OpdmRecord *d1a, OpdmRecord *d1b) {
    const int n = p.n, gab = p.gab, gaa = p.gaa, c0 = ncore;
    Out aa{d2aa}, bb{d2bb}, ab{d2ab}, sf{d2};
    // active-active (write_tpdm.cc:55-108, 320-372)
    for (int ij = 0; ij < gab; ij++) {
        const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
            const double vab = x[o.d2ab + (int64_t)ij * gab + kl];
            ab.put(c0 + i, c0 + j, c0 + k, c0 + l, vab);
            if (i != j && k != l) {   // signed by the order of both pairs
                const int64_t e = (int64_t)p.iaa(i, j) * gaa + p.iaa(k, l);
                const double s = (double)((i < j ? 1 : -1) * (k < l ? 1 : -1));
                aa.put(c0 + i, c0 + j, c0 + k, c0 + l, s * x[o.d2aa + e]);
                bb.put(c0 + i, c0 + j, c0 + k, c0 + l, s * x[o.d2bb + e]);
            }
            if (d2) {
                double v = 0.0;
                v += vab;
                v += x[o.d2ab + (int64_t)p.iab(j, i) * gab + p.iab(l, k)];
                if (i != j && k != l) {
                    // the reference's sign is -1 when either pair is reversed
                    // (not the product of the two signs)
                    const int sg = (i > j || k > l) ? -1 : 1;
                    const int64_t e = (int64_t)p.iaa(i, j) * gaa + p.iaa(k, l);
                    v += sg * x[o.d2aa + e];
                    v += sg * x[o.d2bb + e];
                }
                sf.put(c0 + i, c0 + j, c0 + k, c0 + l, v);
            } else {
                sf.n++;
            }
        }
    }
    // core-core (write_tpdm.cc:110-147, 374-405)
    for (int i = 0; i < c0; i++)
        for (int j = 0; j < c0; j++) {
            ab.put(i, j, i, j, 1.0);
            if (i != j) {
                aa.put(i, j, i, j, 1.0);
                bb.put(i, j, i, j, 1.0);
                aa.put(i, j, j, i, -1.0);
                bb.put(i, j, j, i, -1.0);
            }
            sf.put(i, j, i, j, i != j ? 2.0 + 2.0 : 2.0);
            if (i != j) sf.put(i, j, j, i, -2.0);
        }
    // core-active, from D1 (write_tpdm.cc:149-224, 407-462)
    for (int i = 0; i < c0; i++)
        for (int j = 0; j < n; j++)
            for (int l = 0; l < n; l++) {
                const int jf = c0 + j, lf = c0 + l;
                const double va = x[o.d1a + (int64_t)j * n + l], vb = x[o.d1b + (int64_t)j * n + l];
                aa.put(i, jf, i, lf, va);
                bb.put(i, jf, i, lf, vb);
                aa.put(i, jf, lf, i, -va);
                bb.put(i, jf, lf, i, -vb);
                aa.put(jf, i, lf, i, va);
                bb.put(jf, i, lf, i, vb);
                aa.put(jf, i, i, lf, -va);
                bb.put(jf, i, i, lf, -vb);
                ab.put(i, jf, i, lf, vb);    // valab: the beta D1
                ab.put(jf, i, lf, i, va);    // valba: the alpha D1
                const double sum = va + vb + vb + va, neg = -va - vb;
                sf.put(i, jf, i, lf, sum);
                sf.put(i, jf, lf, i, neg);
                sf.put(jf, i, lf, i, sum);
                sf.put(jf, i, i, lf, neg);
            }
    // D1 (write_opdm.cc:50-106): active, then core
    int64_t c1 = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++, c1++) {
            if (d1a) d1a[c1] = OpdmRecord{c0 + i, c0 + j, x[o.d1a + (int64_t)i * n + j]};
            if (d1b) d1b[c1] = OpdmRecord{c0 + i, c0 + j, x[o.d1b + (int64_t)i * n + j]};
        }
    for (int i = 0; i < c0; i++, c1++) {
        if (d1a) d1a[c1] = OpdmRecord{i, i, 1.0};
        if (d1b) d1b[c1] = OpdmRecord{i, i, 1.0};
    }
}
}  // namespace

RdmCounts rdm_counts(const Problem &p, int ncore) {
    check(p, ncore);
    const int64_t n = p.n, gab = p.gab, c = ncore, same = n * (n - 1) * n * (n - 1);
    if (p.spec.doci)   // src/v2rdm_doci/write_tpdm.cc writes the three spin blocks only
        return RdmCounts{same, same, gab * gab, -1, -1, -1};
    const int64_t aa = same + 2 * c * (c - 1) + 4 * c * n * n;
    return RdmCounts{aa, aa, gab * gab + c * c + 2 * c * n * n, gab * gab + c * c + c * (c - 1) + 4 * c * n * n,
                     n * n + c, n * n + c};
}

void rdm_records(const Problem &p, const double *x, int ncore, TpdmRecord *d2aa, TpdmRecord *d2bb,
                 TpdmRecord *d2ab, TpdmRecord *d2, OpdmRecord *d1a, OpdmRecord *d1b) {
    check(p, ncore);
    if (p.spec.doci) {
        // DOCI's WriteTPDM (src/v2rdm_doci/write_tpdm.cc:47-176) writes the
        // spin blocks its PackSpatialDensity expands, D2bb from D2aa
        std::vector<double> layout(doci_v2rdm_layout_size(p));
        doci_v2rdm_layout(p, x, layout.data());
        const int64_t gab2 = (int64_t)p.gab * p.gab, gaa2 = (int64_t)p.gaa * p.gaa, nn = (int64_t)p.n * p.n;
        const Blocks o{0, gab2, gab2 + gaa2, gab2 + 2 * gaa2, gab2 + 2 * gaa2 + nn};
        records(p, layout.data(), o, 0, d2aa, d2bb, d2ab, nullptr, nullptr, nullptr);
        return;
    }
    records(p, x, Blocks{p.d2ab, p.d2aa, p.d2bb, p.d1a, p.d1b}, ncore, d2aa, d2bb, d2ab, d2, d1a, d1b);
}

void iwl_records(const Problem &p, const double *x, int ncore, TpdmRecord *aa_out, TpdmRecord *ab_out,
                 TpdmRecord *bb_out) {
    // WriteTPDM_IWL (src/v2rdm_casscf/write_tpdm_iwl.cc:45-205): the calls it
    // makes to IWL::write_value, labels (i, k, j, l) for the element D2(ij, kl),
    // aa and bb values scaled by 1/4
    check(p, ncore);
    if (p.spec.doci) throw std::invalid_argument("the IWL 2-RDM of v2RDM problems");
    const int n = p.n, gab = p.gab, gaa = p.gaa, c0 = ncore;
    Out aa{aa_out}, ab{ab_out}, bb{bb_out};
    for (int ij = 0; ij < gab; ij++) {
        const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
            ab.put(c0 + i, c0 + k, c0 + j, c0 + l, x[p.d2ab + (int64_t)ij * gab + kl]);
            if (i != j && k != l) {
                const int64_t e = (int64_t)p.iaa(i, j) * gaa + p.iaa(k, l);
                const double s = 0.25 * (double)((i < j ? 1 : -1) * (k < l ? 1 : -1));
                aa.put(c0 + i, c0 + k, c0 + j, c0 + l, s * x[p.d2aa + e]);
                bb.put(c0 + i, c0 + k, c0 + j, c0 + l, s * x[p.d2bb + e]);
            }
        }
    }
    for (int i = 0; i < c0; i++)   // core-core (:84-107)
        for (int j = 0; j < c0; j++) {
            ab.put(i, i, j, j, 1.0);
            if (i != j) {
                aa.put(i, i, j, j, 0.25);
                bb.put(i, i, j, j, 0.25);
                aa.put(i, j, j, i, -0.25);
                bb.put(i, j, j, i, -0.25);
            }
        }
    for (int i = 0; i < c0; i++)   // core-active, from D1 (:109-190)
        for (int j = 0; j < n; j++)
            for (int l = 0; l < n; l++) {
                const int jf = c0 + j, lf = c0 + l;
                const double va = 0.25 * x[p.d1a + (int64_t)j * n + l], vb = 0.25 * x[p.d1b + (int64_t)j * n + l];
                aa.put(i, i, jf, lf, va);
                bb.put(i, i, jf, lf, vb);
                aa.put(i, lf, jf, i, -va);
                bb.put(i, lf, jf, i, -vb);
                aa.put(jf, lf, i, i, va);
                bb.put(jf, lf, i, i, vb);
                aa.put(jf, i, i, lf, -va);
                bb.put(jf, i, i, lf, -vb);
                ab.put(i, i, jf, lf, x[p.d1b + (int64_t)j * n + l]);
                ab.put(jf, lf, i, i, x[p.d1a + (int64_t)j * n + l]);
            }
}

void d3_counts(const Problem &p, int64_t *counts) {
    check(p, 0);
    if (p.spec.doci || !p.d3) throw std::invalid_argument("3-RDM records need the v2RDM D3 blocks (CONSTRAIN_D3)");
    const int64_t n = p.n, distinct = n * (n - 1) * (n - 2), pair_first = n * n * (n - 1);
    counts[0] = distinct * distinct;
    counts[1] = pair_first * pair_first;
}

void d3_records(const Problem &p, const double *x, int ncore, Dm3Record *aaa, Dm3Record *aab,
                Dm3Record *bba, Dm3Record *bbb) {
    // every ordered triple (i, j, k) in the aba order, i n^2 + j n + k
    // (basis.cc:640-727); the sign is the parity of the order within the
    // alpha pair (aab) or the whole triple (aaa)
    int64_t counts[2];
    d3_counts(p, counts);
    if (ncore < 0) throw std::invalid_argument("ncore must be >= 0");
    const int n = p.n, c0 = ncore;
    const int64_t taab = p.trip_aab, taaa = p.trip_aaa;
    auto put = [](Dm3Record *r, int64_t k, int a, int b, int c, int d, int e, int f, double v) {
        if (r) r[k] = Dm3Record{a, b, c, d, e, f, v};
    };
    int64_t q = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                if (i == j) continue;
                const int64_t ijk = p.ibas_aab[((int64_t)i * n + j) * n + k];
                for (int l = 0; l < n; l++)
                    for (int m = 0; m < n; m++)
                        for (int o = 0; o < n; o++) {
                            if (l == m) continue;
                            const int64_t lmo = p.ibas_aab[((int64_t)l * n + m) * n + o];
                            const int s = (i > j ? -1 : 1) * (l > m ? -1 : 1);
                            put(aab, q, c0 + i, c0 + j, c0 + k, c0 + l, c0 + m, c0 + o, s * x[p.d3aab + ijk * taab + lmo]);
                            put(bba, q, c0 + i, c0 + j, c0 + k, c0 + l, c0 + m, c0 + o, s * x[p.d3bba + ijk * taab + lmo]);
                            q++;
                        }
            }
    auto parity = [](int a, int b, int c) {
        int s = 1;
        if (a > b) s = -s;
        if (a > c) s = -s;
        if (b > c) s = -s;
        return s;
    };
    q = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                if (i == j || i == k || j == k) continue;
                const int64_t ijk = p.ibas_aaa[((int64_t)i * n + j) * n + k];
                for (int l = 0; l < n; l++)
                    for (int m = 0; m < n; m++)
                        for (int o = 0; o < n; o++) {
                            if (l == m || l == o || m == o) continue;
                            const int64_t lmo = p.ibas_aaa[((int64_t)l * n + m) * n + o];
                            const int s = parity(i, j, k) * parity(l, m, o);
                            put(aaa, q, c0 + i, c0 + j, c0 + k, c0 + l, c0 + m, c0 + o, s * x[p.d3aaa + ijk * taaa + lmo]);
                            put(bbb, q, c0 + i, c0 + j, c0 + k, c0 + l, c0 + m, c0 + o, s * x[p.d3bbb + ijk * taaa + lmo]);
                            q++;
                        }
            }
}

}  // namespace v2b
