// The density-matrix records hilbert writes after a v2RDM solve, built from
// the primal vector on the host: the same records, in the same order, with
// the same values as
//   WriteTPDM          src/v2rdm_casscf/write_tpdm.cc:40-310   (D2aa, D2bb, D2ab)
//   WriteTPDMSpinFree  src/v2rdm_casscf/write_tpdm.cc:312-519  (D2)
//   WriteOPDM          src/v2rdm_casscf/write_opdm.cc:40-114   (D1a, D1b)
// for the C1 active space (no frozen or restricted core, so the core
// records of those functions are empty; orbital numbers are active indices),
// and as v2RDM-DOCI's WriteTPDM (src/v2rdm_doci/write_tpdm.cc:47-176) for a
// DOCI problem.
#include "rdm_records.h"

#include <stdexcept>
#include <vector>

#include "doci_problem.h"

namespace v2b {

namespace {
void check(const Problem &p) {
    if (p.spec.batch_parts) throw std::invalid_argument("density records of a batch: ask each part");
}

struct Blocks {   // where the spin blocks sit in the vector the records read
    int64_t d2ab, d2aa, d2bb, d1a, d1b;
};

void records(const Problem &p, const double *x, const Blocks &o, TpdmRecord *d2aa, TpdmRecord *d2bb,
             TpdmRecord *d2ab, TpdmRecord *d2, OpdmRecord *d1a, OpdmRecord *d1b) {
    const int n = p.n, gab = p.gab, gaa = p.gaa;
    int64_t caa = 0, cab = 0, csf = 0;
    for (int ij = 0; ij < gab; ij++) {
        const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
            const double vab = x[o.d2ab + (int64_t)ij * gab + kl];
            if (d2ab) d2ab[cab] = TpdmRecord{i, j, k, l, vab};
            cab++;
            if (i != j && k != l) {   // write_tpdm.cc:86-105: signed by the order of both pairs
                const int64_t e = (int64_t)p.iaa(i, j) * gaa + p.iaa(k, l);
                const double s = (double)((i < j ? 1 : -1) * (k < l ? 1 : -1));
                if (d2aa) d2aa[caa] = TpdmRecord{i, j, k, l, s * x[o.d2aa + e]};
                if (d2bb) d2bb[caa] = TpdmRecord{i, j, k, l, s * x[o.d2bb + e]};
                caa++;
            }
            if (d2) {   // write_tpdm.cc:320-372
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
                d2[csf] = TpdmRecord{i, j, k, l, v};
            }
            csf++;
        }
    }
    int64_t c1 = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++, c1++) {
            if (d1a) d1a[c1] = OpdmRecord{i, j, x[o.d1a + (int64_t)i * n + j]};
            if (d1b) d1b[c1] = OpdmRecord{i, j, x[o.d1b + (int64_t)i * n + j]};
        }
}
}  // namespace

RdmCounts rdm_counts(const Problem &p) {
    check(p);
    const int64_t n = p.n, gab = p.gab, same = n * (n - 1) * n * (n - 1);
    if (p.spec.doci)   // src/v2rdm_doci/write_tpdm.cc writes the three spin blocks only
        return RdmCounts{same, same, gab * gab, -1, -1, -1};
    return RdmCounts{same, same, gab * gab, gab * gab, n * n, n * n};
}

void rdm_records(const Problem &p, const double *x, TpdmRecord *d2aa, TpdmRecord *d2bb,
                 TpdmRecord *d2ab, TpdmRecord *d2, OpdmRecord *d1a, OpdmRecord *d1b) {
    check(p);
    if (p.spec.doci) {
        // DOCI's WriteTPDM (src/v2rdm_doci/write_tpdm.cc:47-176) writes the
        // spin blocks its PackSpatialDensity expands, D2bb from D2aa
        std::vector<double> layout(doci_v2rdm_layout_size(p));
        doci_v2rdm_layout(p, x, layout.data());
        const int64_t gab2 = (int64_t)p.gab * p.gab, gaa2 = (int64_t)p.gaa * p.gaa, nn = (int64_t)p.n * p.n;
        const Blocks o{0, gab2, gab2 + gaa2, gab2 + 2 * gaa2, gab2 + 2 * gaa2 + nn};
        records(p, layout.data(), o, d2aa, d2bb, d2ab, nullptr, nullptr, nullptr);
        return;
    }
    records(p, x, Blocks{p.d2ab, p.d2aa, p.d2bb, p.d1a, p.d1b}, d2aa, d2bb, d2ab, d2, d1a, d1b);
}

void iwl_records(const Problem &p, const double *x, TpdmRecord *aa, TpdmRecord *ab, TpdmRecord *bb) {
    // WriteTPDM_IWL (src/v2rdm_casscf/write_tpdm_iwl.cc:45-205): the calls it
    // makes to IWL::write_value, labels in (i, k, j, l) order for the element
    // D2(ij, kl); aa and bb scaled by 1/4; no core orbitals, so no core calls
    check(p);
    if (p.spec.doci) throw std::invalid_argument("the IWL 2-RDM of v2RDM problems");
    const int gab = p.gab, gaa = p.gaa;
    int64_t caa = 0, cab = 0;
    for (int ij = 0; ij < gab; ij++) {
        const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
            if (ab) ab[cab] = TpdmRecord{i, k, j, l, x[p.d2ab + (int64_t)ij * gab + kl]};
            cab++;
            if (i != j && k != l) {
                const int64_t e = (int64_t)p.iaa(i, j) * gaa + p.iaa(k, l);
                const double s = 0.25 * (double)((i < j ? 1 : -1) * (k < l ? 1 : -1));
                if (aa) aa[caa] = TpdmRecord{i, k, j, l, s * x[p.d2aa + e]};
                if (bb) bb[caa] = TpdmRecord{i, k, j, l, s * x[p.d2bb + e]};
                caa++;
            }
        }
    }
}

}  // namespace v2b
