// Density-matrix records of hilbert's RDM writers (see rdm_records.cpp).
#pragma once

#include "v2rdm_problem.h"

namespace v2b {

// struct tpdm / struct opdm, src/v2rdm_casscf/v2rdm_solver.h:53-65
struct TpdmRecord {
    int i, j, k, l;
    double value;
};
struct OpdmRecord {
    int i, j;
    double value;
};

// struct dm3, src/v2rdm_casscf/write_3pdm.cc:39-47
struct Dm3Record {
    int i, j, k, l, m, n;
    double value;
};

struct RdmCounts {
    int64_t d2aa, d2bb, d2ab, d2, d1a, d1b;
};

// ncore doubly occupied orbitals come first (0 .. ncore-1), active orbital
// i is ncore + i; x is the host primal vector; any output may be null
RdmCounts rdm_counts(const Problem &p, int ncore);
void rdm_records(const Problem &p, const double *x, int ncore, TpdmRecord *d2aa, TpdmRecord *d2bb,
                 TpdmRecord *d2ab, TpdmRecord *d2, OpdmRecord *d1a, OpdmRecord *d1b);

// the IWL::write_value calls of WriteTPDM_IWL (v2RDM problems), as records
// (i, j, k, l) = its labels; counts are rdm_counts' d2aa (aa, bb) and d2ab
void iwl_records(const Problem &p, const double *x, int ncore, TpdmRecord *aa, TpdmRecord *ab,
                 TpdmRecord *bb);

// WriteActive3PDM (src/v2rdm_casscf/write_3pdm.cc:50-206), problems with the
// D3 blocks: counts[0] records each in D3aaa and D3bbb, counts[1] in D3aab
// and D3bba
void d3_counts(const Problem &p, int64_t *counts);
void d3_records(const Problem &p, const double *x, int ncore, Dm3Record *aaa, Dm3Record *aab,
                Dm3Record *bba, Dm3Record *bbb);

}  // namespace v2b
