// Host-side v2RDM-DOCI problem: hilbert's seniority-zero 2-RDM program
// (src/v2rdm_doci) on the same packed-operator path as the v2RDM problem.
//
// The primal vector holds, in order (v2rdm_doci_solver.cc:542-600):
//   D2s2 (n x n, n^2 blocks of 1), D2s0 (one n x n block), D1 (n blocks of 1),
//   [Q2s2 (n(n-1)/2 blocks of 1), Q2s0 (n x n)], [G2s2 (n(n-1)/2 blocks of
//   2 x 2), G2s0 (n x n)], [D3s3 (n^3 blocks of 1), D3s1 (n blocks of n-1)],
//   [T1 aaa, aab (blocks of 1), T1s1 (n blocks of n-1)],
//   [T2s1 (n blocks of 2n-1), T2 (C(n,3) blocks of 3)].
// The dual rows follow bpsdp_Au (v2rdm_doci_solver.cc:1509-1537).
#pragma once

#include <stdexcept>
#include <vector>

#include "v2rdm_problem.h"

namespace v2b {

Problem make_doci_problem(const ProblemSpec &spec);
void doci_build_b(const Problem &p, double *b);
void doci_build_c_external(const Problem &p, const double *h, const double *g, double *c);
// x in the v2RDM layout (D2ab gab^2, D2aa gaa^2, D2bb gaa^2, D1a n^2, D1b n^2)
// that hilbert's DOCI PackSpatialDensity builds before packing
int64_t doci_v2rdm_layout_size(const Problem &p);
void doci_v2rdm_layout(const Problem &p, const double *x, double *out);

struct DociTerm {
    int64_t col;
    double coef;
    bool tail;   // summed separately and added at the end of the row
};

// Every dual row of hilbert's DOCI A, as f(row, terms, count), in the order
// bpsdp_Au writes them; the terms of a row in the order the reference adds
// them.  bpsdp_ATu visits the rows in the same order and scatters the same
// terms, so the same list also orders every column of A^T.
//
// One family is not reproduced bit for bit in A.x: the seniority-3 D3 rows
// (d3.cc:131-145) scale the partial sum, (1/6) * sum(D3) - (N/2 - 2) D2,
// and are emitted as sum((1/6) D3) - (N/2 - 2) D2, which rounds differently.
// Their A^T.y scatter (d3.cc:37-54) multiplies term by term and is exact.
template <class F>
void doci_rows(const Problem &p, F &&f) {
    const int n = p.n;
    const int64_t nm = n - 1, nm2 = nm * nm;
    const DociOffsets &o = p.doci;
    const double na = p.spec.nalpha;
    const int ntot = p.spec.nalpha + p.spec.nbeta;
    std::vector<DociTerm> t;
    t.reserve(8 * (size_t)n + 16);
    int64_t row = 0;
    auto add = [&](int64_t col, double c) { t.push_back({col, c, false}); };
    auto tail = [&](int64_t col, double c) { t.push_back({col, c, true}); };
    auto emit = [&](int64_t r) {
        f(r, t.data(), (int)t.size());
        t.clear();
    };
    auto shift = [](int a, int b) { return a > b ? a - 1 : a; };   // index without b

    // d2.cc:114-186: traces, contractions to D1, D2s2 symmetry
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (i != j) add(o.d2s2 + i * n + j, 1.0);
    emit(row++);
    for (int i = 0; i < n; i++) add(o.d2s0 + (int64_t)i * n + i, 1.0);
    emit(row++);
    for (int i = 0; i < n; i++) add(o.d1 + i, 1.0);
    emit(row++);
    for (int sp = 0; sp < 2; sp++)
        for (int i = 0; i < n; i++) {
            add(o.d1 + i, na - 1.0);
            for (int j = 0; j < n; j++)
                if (j != i) add(o.d2s2 + (sp ? (int64_t)j * n + i : (int64_t)i * n + j), -1.0);
            emit(row++);
        }
    for (int i = 0; i < n; i++) {
        add(o.d1 + i, 1.0);
        add(o.d2s0 + (int64_t)i * n + i, -1.0);
        emit(row++);
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            if (i == j) {
                add(o.d2s2 + (int64_t)i * n + i, 1.0);
            } else {
                add(o.d2s2 + (int64_t)i * n + j, 1.0);
                add(o.d2s2 + (int64_t)j * n + i, -1.0);
            }
            emit(row++);
        }

    // q2.cc:45-85
    if (p.q2) {
        int64_t ij = 0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++, ij++) {
                add(o.d2s2 + (int64_t)i * n + j, 0.5);
                add(o.d2s2 + (int64_t)j * n + i, 0.5);
                add(o.q2s2 + ij, -1.0);
                add(o.d1 + i, -1.0);
                add(o.d1 + j, -1.0);
                emit(row++);
            }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                add(o.d2s0 + (int64_t)i * n + j, 1.0);
                add(o.q2s0 + (int64_t)i * n + j, -1.0);
                if (i == j) {   // the diagonal's D1 terms, summed apart (q2.cc:75-81)
                    tail(o.d1 + i, -1.0);
                    tail(o.d1 + i, -1.0);
                }
                emit(row++);
            }
    }

    // g2.cc:45-103
    if (p.g2) {
        int64_t aux = 0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++, aux += 4) {
                const int64_t ij = (int64_t)i * n + j, ji = (int64_t)j * n + i;
                add(o.g2s2 + aux + 0, -1.0);
                add(o.d1 + i, 1.0);
                add(o.d2s2 + ij, -0.5);
                add(o.d2s2 + ji, -0.5);
                emit(row++);
                for (int q = 1; q <= 2; q++) {
                    add(o.g2s2 + aux + q, -1.0);
                    add(o.d2s0 + ij, 0.5);
                    add(o.d2s0 + ji, 0.5);
                    emit(row++);
                }
                add(o.g2s2 + aux + 3, -1.0);
                add(o.d1 + j, 1.0);
                add(o.d2s2 + ij, -0.5);
                add(o.d2s2 + ji, -0.5);
                emit(row++);
            }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                add(o.g2s0 + (int64_t)i * n + j, -1.0);
                if (i != j) {
                    add(o.d2s2 + (int64_t)i * n + j, 0.5);
                    add(o.d2s2 + (int64_t)j * n + i, 0.5);
                } else {
                    add(o.d1 + i, 1.0);
                }
                emit(row++);
            }
    }

    // d3.cc:128-215
    if (p.d3) {
        const double sixth = 1.0 / 6.0;
        const double s3 = -(0.5 * ntot - 2.0);
        const double s1 = -(0.5 * (0.5 * ntot - 1.0));
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) {
                if (a == b) continue;
                for (int c = 0; c < n; c++) {
                    if (c == a || c == b) continue;
                    add(o.d3s3 + ((int64_t)c * n + a) * n + b, sixth);
                    add(o.d3s3 + ((int64_t)c * n + b) * n + a, sixth);
                    add(o.d3s3 + ((int64_t)a * n + c) * n + b, sixth);
                    add(o.d3s3 + ((int64_t)b * n + c) * n + a, sixth);
                    add(o.d3s3 + ((int64_t)a * n + b) * n + c, sixth);
                    add(o.d3s3 + ((int64_t)b * n + a) * n + c, sixth);
                }
                add(o.d2s2 + (int64_t)a * n + b, s3);
                emit(row++);
            }
        for (int twin = 0; twin < 2; twin++)
            for (int a = 0; a < n; a++)
                for (int b = 0; b < n; b++) {
                    if (a == b) continue;
                    if (twin == 0) {
                        const int myb = shift(b, a);
                        add(o.d3s1 + a * nm2 + myb * nm + myb, 1.0);
                    } else {
                        const int mya = shift(a, b);
                        add(o.d3s1 + b * nm2 + mya * nm + mya, 1.0);
                    }
                    add(o.d2s2 + (int64_t)a * n + b, -0.5);
                    add(o.d2s2 + (int64_t)b * n + a, -0.5);
                    emit(row++);
                }
        for (int a = 0; a < n; a++)
            for (int c = 0; c < n; c++) {
                for (int b = 0; b < n; b++) {
                    if (b == a || b == c) continue;
                    const int mya = shift(a, b), myc = shift(c, b);
                    add(o.d3s1 + b * nm2 + mya * nm + myc, 0.5);
                    add(o.d3s1 + b * nm2 + myc * nm + mya, 0.5);
                }
                add(o.d2s0 + (int64_t)a * n + c, s1);
                add(o.d2s0 + (int64_t)c * n + a, s1);
                emit(row++);
            }
    }

    // t1.cc:45-144
    if (p.t1) {
        auto pair = [&](int a, int b, int64_t blk) {
            add(blk + (int64_t)a * n + b, -0.5);
            add(blk + (int64_t)b * n + a, -0.5);
        };
        int64_t abc = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                for (int c = b + 1; c < n; c++, abc++) {
                    add(o.t1aaa + abc, 1.0);
                    add(o.d1 + a, 1.0);
                    add(o.d1 + b, 1.0);
                    add(o.d1 + c, 1.0);
                    pair(a, b, o.d2s2);
                    pair(b, c, o.d2s2);
                    pair(a, c, o.d2s2);
                    emit(row++);
                }
        abc = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                for (int c = 0; c < n; c++, abc++) {
                    add(o.t1aab + abc, 1.0);
                    add(o.d1 + a, 1.0);
                    add(o.d1 + b, 1.0);
                    add(o.d1 + c, 1.0);
                    pair(a, b, o.d2s2);
                    pair(b, c, b != c ? o.d2s2 : o.d2s0);
                    pair(a, c, a != c ? o.d2s2 : o.d2s0);
                    emit(row++);
                }
        for (int b = 0; b < n; b++)
            for (int a = 0; a < n; a++) {
                if (a == b) continue;
                for (int c = 0; c < n; c++) {
                    if (c == b) continue;
                    const int mya = shift(a, b), myc = shift(c, b);
                    add(o.t1s1 + b * nm2 + mya * nm + myc, 1.0);
                    if (a == c) {
                        add(o.d1 + a, 2.0);
                        add(o.d1 + b, 1.0);
                        add(o.d2s2 + (int64_t)a * n + b, -1.0);
                        add(o.d2s2 + (int64_t)b * n + a, -1.0);
                    }
                    pair(a, c, o.d2s0);
                    emit(row++);
                }
            }
    }

    // t2.cc:45-211 (Rubio-Garcia et al., JCTC 2018, eq. 33): one (2n-1)^2
    // block per i, written at row (block + id) in nine sub-blocks
    if (p.t2) {
        const int64_t w = 2 * (int64_t)n - 1, bs = w * w;
        auto sym = [&](int64_t blk, int a, int b, double c) {
            add(blk + (int64_t)a * n + b, c);
            add(blk + (int64_t)b * n + a, c);
        };
        for (int i = 0; i < n; i++) {
            const int64_t base = row + i * bs, aux = o.t2s1 + i * bs;
            for (int j = 0; j < n; j++) {   // D(jk)
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    const int64_t id = shift(k, i) * w + shift(j, i);
                    add(aux + id, -1.0);
                    if (j == k) add(o.d1 + j, 1.0);
                    else sym(o.d2s2, j, k, 0.5);
                    emit(base + id);
                }
            }
            for (int j = 0; j < n; j++) {   // -djk Pi(ik)
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    const int64_t id = shift(k, i) * w + shift(j, i) + n - 1;
                    add(aux + id, -1.0);
                    if (j == k) sym(o.d2s0, i, k, -0.5);
                    emit(base + id);
                }
            }
            for (int k = 0; k < n; k++) {   // D(ik)
                if (k == i) continue;
                const int64_t id = shift(k, i) * w + 2 * n - 2;
                add(aux + id, -1.0);
                sym(o.d2s2, i, k, 0.5);
                emit(base + id);
            }
            for (int j = 0; j < n; j++) {   // -djk Pi(ki)
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    const int64_t id = (shift(k, i) + n - 1) * w + shift(j, i);
                    add(aux + id, -1.0);
                    if (j == k) sym(o.d2s0, i, k, -0.5);
                    emit(base + id);
                }
            }
            for (int j = 0; j < n; j++) {   // Pi(jk) + djk (-D(ik) - D(ki) + p(i))
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    const int64_t id = (shift(k, i) + n - 1) * w + shift(j, i) + n - 1;
                    add(aux + id, -1.0);
                    if (j == k) {
                        add(o.d1 + i, 1.0);
                        sym(o.d2s2, i, k, -1.0);
                    }
                    sym(o.d2s0, j, k, 0.5);
                    emit(base + id);
                }
            }
            for (int k = 0; k < n; k++) {   // Pi(ik)
                if (k == i) continue;
                const int64_t id = (shift(k, i) + n - 1) * w + 2 * n - 2;
                add(aux + id, -1.0);
                sym(o.d2s0, i, k, 0.5);
                emit(base + id);
            }
            for (int j = 0; j < n; j++) {   // D(ji)
                if (j == i) continue;
                const int64_t id = (2 * (int64_t)n - 2) * w + shift(j, i);
                add(aux + id, -1.0);
                sym(o.d2s2, j, i, 0.5);
                emit(base + id);
            }
            for (int j = 0; j < n; j++) {   // Pi(ji)
                if (j == i) continue;
                const int64_t id = (2 * (int64_t)n - 2) * w + shift(j, i) + n - 1;
                add(aux + id, -1.0);
                sym(o.d2s0, j, i, 0.5);
                emit(base + id);
            }
            const int64_t id = (2 * (int64_t)n - 2) * w + 2 * n - 2;   // p(i)
            add(aux + id, -1.0);
            add(o.d1 + i, 1.0);
            emit(base + id);
        }
        row += n * bs;
        // t2.cc:560-657: one 3 x 3 block per i < k < m
        int64_t aux = o.t2;
        for (int i = 0; i < n; i++)
            for (int k = i + 1; k < n; k++)
                for (int m = k + 1; m < n; m++, aux += 9) {
                    add(aux + 0, -1.0);
                    sym(o.d2s2, i, k, 0.5);
                    sym(o.d2s2, i, m, -0.5);
                    sym(o.d2s2, k, m, -0.5);
                    add(o.d1 + m, 1.0);
                    emit(row++);
                    add(aux + 1, -1.0);
                    sym(o.d2s0, m, k, 0.5);
                    emit(row++);
                    add(aux + 2, -1.0);
                    sym(o.d2s0, m, i, 0.5);
                    emit(row++);
                    add(aux + 3, -1.0);
                    sym(o.d2s0, k, m, 0.5);
                    emit(row++);
                    add(aux + 4, -1.0);
                    sym(o.d2s2, i, k, -0.5);
                    sym(o.d2s2, i, m, 0.5);
                    sym(o.d2s2, m, k, -0.5);
                    add(o.d1 + k, 1.0);
                    emit(row++);
                    add(aux + 5, -1.0);
                    sym(o.d2s0, k, i, 0.5);
                    emit(row++);
                    add(aux + 6, -1.0);
                    sym(o.d2s0, i, m, 0.5);
                    emit(row++);
                    add(aux + 7, -1.0);
                    sym(o.d2s0, i, k, 0.5);
                    emit(row++);
                    add(aux + 8, -1.0);
                    sym(o.d2s2, i, k, -0.5);
                    sym(o.d2s2, i, m, -0.5);
                    sym(o.d2s2, k, m, 0.5);
                    add(o.d1 + i, 1.0);
                    emit(row++);
                }
    }
    if (row != p.n_dual) throw std::logic_error("DOCI row count mismatch");
}

}  // namespace v2b
