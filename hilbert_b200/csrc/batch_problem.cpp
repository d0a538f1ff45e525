// Independent problems solved as one block-diagonal problem: every launch of
// the device iteration (CG, projection, norms) then covers all of them.  The
// joint boundary-point SDP separates into the parts, so its optimum is the
// parts' optima side by side; the penalty mu and the CG scalars are shared.
#include <cstring>
#include <stdexcept>
#include <string>

#include "v2rdm_problem.h"

namespace v2b {

namespace {
// concatenate packed operators along the diagonal; pal is the merged palette
void join(const std::vector<const PackedOperator *> &ops, const std::vector<int64_t> &col_shift,
          std::vector<double> &pal, PackedOperator &out) {
    out = PackedOperator();
    uint64_t nnz = 0;
    for (const PackedOperator *op : ops) {
        out.nrows += op->nrows;
        out.ncols += op->ncols;
        nnz += op->entries.size();
    }
    if (nnz >= (1ull << 32)) throw std::invalid_argument("batch has more than 2^32 operator entries");
    out.row_ptr.reserve(out.nrows + 1);
    out.entries.reserve(nnz);
    for (size_t k = 0; k < ops.size(); k++) {
        const PackedOperator &op = *ops[k];
        uint32_t code_map[16];
        for (size_t c = 0; c < op.palette.size(); c++) {
            size_t m = 0;
            while (m < pal.size() && std::memcmp(&pal[m], &op.palette[c], sizeof(double)) != 0) m++;
            if (m == pal.size()) {
                if (pal.size() == 16)
                    throw std::invalid_argument("batch: the parts' coefficients do not fit one 16-entry palette "
                                                "(part " + std::to_string(k) + ")");
                pal.push_back(op.palette[c]);
            }
            code_map[c] = (uint32_t)m;
        }
        const uint32_t base = (uint32_t)out.entries.size();
        for (int64_t r = 0; r < op.nrows; r++) out.row_ptr.push_back(base + op.row_ptr[r]);
        for (uint32_t w : op.entries) {
            const uint64_t col = (uint64_t)(w & kColMask) + (uint64_t)col_shift[k];
            const uint32_t code = (w >> kColBits) & 15u;
            out.entries.push_back((uint32_t)col | (code_map[code] << kColBits) | (w & kGroupFlag));
        }
    }
    out.row_ptr.push_back((uint32_t)out.entries.size());
}
}  // namespace

void make_batch(const std::vector<const Problem *> &parts, const std::vector<const PackedOperator *> &A,
                const std::vector<const PackedOperator *> &AT, Problem &out, PackedOperator &outA,
                PackedOperator &outAT) {
    if (parts.empty()) throw std::invalid_argument("batch: no parts");
    Problem b;
    b.spec.batch_parts = (int)parts.size();
    std::vector<int64_t> primal_shift, dual_shift;
    for (const Problem *p : parts) {
        if (p->spec.batch_parts) throw std::invalid_argument("batch: a part is itself a batch");
        primal_shift.push_back(b.n_primal);
        dual_shift.push_back(b.n_dual);
        for (size_t k = 0; k < p->dims.size(); k++) {
            b.dims.push_back(p->dims[k]);
            b.block_off.push_back(b.n_primal + p->block_off[k]);
        }
        b.n_primal += p->n_primal;
        b.n_dual += p->n_dual;
    }
    if (b.n_primal > (int64_t)kColMask || b.n_dual > (int64_t)kColMask)
        throw std::invalid_argument("batch too large for 27-bit packed column indices");
    std::vector<double> palA, palAT;
    join(A, primal_shift, palA, outA);    // A's columns are primal elements
    join(AT, dual_shift, palAT, outAT);   // A^T's columns are dual rows
    outA.palette = palA;
    outAT.palette = palAT;
    out = std::move(b);
}

}  // namespace v2b
