// Host problem builder for the B200 v2RDM path (see v2rdm_problem.h).
//
// The operator emitters walk the constraint families in the order of
// hilbert's bpsdp_Au / bpsdp_ATu and record, for every dual row (A) or
// primal element (A^T), its terms in the order the reference accumulates
// them.  A gather that sums each row left to right with separate multiply
// and add roundings therefore reproduces the reference's A.x and A^T.y.
#include "v2rdm_problem.h"
#include "doci_problem.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace v2b {

Problem make_problem(const ProblemSpec &spec) {
    if (spec.doci) return make_doci_problem(spec);
    if (spec.nmo < 1 || spec.nalpha < 0 || spec.nbeta < 0 || spec.nalpha > spec.nmo ||
        spec.nbeta > spec.nmo)
        throw std::invalid_argument("invalid orbital / electron counts");
    if (spec.positivity < POS_D || spec.positivity > POS_DQGT1T2)
        throw std::invalid_argument("unsupported POSITIVITY");
    Problem p;
    p.spec = spec;
    const int n = spec.nmo;
    p.n = n;
    p.gab = n * n;
    p.gaa = n * (n - 1) / 2;
    // v2rdm_solver.cc:4081-4118: every T option keeps Q2 and G2
    p.q2 = spec.positivity == POS_DQ || spec.positivity >= POS_DQG;
    p.g2 = spec.positivity == POS_DG || spec.positivity >= POS_DQG;
    p.t1 = spec.positivity == POS_DQGT1 || spec.positivity == POS_DQGT1T2;
    p.t2 = spec.positivity == POS_DQGT2 || spec.positivity == POS_DQGT1T2;
    p.q3 = spec.constrain_q3;
    p.e3 = spec.constrain_e3;
    p.f3 = spec.constrain_f3;
    p.d4 = spec.constrain_d4;
    p.d3 = spec.constrain_d3 || p.q3 || p.e3 || p.f3 || p.d4;
    if (p.q3 && !(p.q2 && p.g2))
        throw std::invalid_argument("CONSTRAIN_Q3 needs the Q2 and G2 conditions (POSITIVITY DQG or a T option)");
    p.mult = spec.hubbard_multiplicity ? 2 * (spec.nalpha - spec.nbeta) + 1
                                       : (spec.nalpha - spec.nbeta) + 1;

    // basis.cc:426-533 for one irrep: geminal number i*n + j holds the
    // ordered pair (j, i); aa geminals are the pairs with first < second,
    // numbered in the same sweep.
    p.bas_ab.assign(2 * p.gab, -999);
    p.bas_aa.assign(2 * (p.gaa > 0 ? p.gaa : 1), -999);
    p.ibas_ab.assign(n * n, -999);
    p.ibas_aa.assign(n * n, -999);
    int count_aa = 0;
    for (int second = 0; second < n; second++) {
        for (int first = 0; first < n; first++) {
            const int g = second * n + first;
            p.ibas_ab[first * n + second] = g;
            p.bas_ab[2 * g] = first;
            p.bas_ab[2 * g + 1] = second;
            if (first < second) {
                p.ibas_aa[first * n + second] = count_aa;
                p.ibas_aa[second * n + first] = count_aa;
                p.bas_aa[2 * count_aa] = first;
                p.bas_aa[2 * count_aa + 1] = second;
                count_aa++;
            }
        }
    }

    int64_t off = 0;
    auto add_block = [&](int64_t &where, int dim) {
        where = off;
        off += (int64_t)dim * dim;
        p.dims.push_back(dim);
        p.block_off.push_back(where);
    };
    const bool singlet = spec.nalpha == spec.nbeta;
    add_block(p.d2ab, p.gab);
    add_block(p.d2aa, p.gaa);
    add_block(p.d2bb, p.gaa);
    if (spec.constrain_spin) add_block(p.d200, singlet ? p.gab : 2 * p.gab);
    add_block(p.d1a, n);
    add_block(p.d1b, n);
    add_block(p.q1a, n);
    add_block(p.q1b, n);
    if (p.q2) {
        add_block(p.q2ab, p.gab);
        add_block(p.q2aa, p.gaa);
        add_block(p.q2bb, p.gaa);
    }
    if (p.g2) {
        add_block(p.g2ab, p.gab);
        add_block(p.g2ba, p.gab);
        add_block(p.g2aa, 2 * p.gab);
    }
    if (p.t1 || p.t2 || p.d3) {   // basis.cc:640-745: lexicographic triplets
        p.trip_aba = n * n * n;
        p.ibas_aaa.assign((size_t)n * n * n, -999);
        p.ibas_aab.assign((size_t)n * n * n, -999);
        auto at = [&](int a, int b, int c) { return ((size_t)a * n + b) * n + c; };
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
                for (int k = 0; k < n; k++) {
                    const int ta = (int)(p.bas_aab.size() / 3);
                    p.ibas_aab[at(i, j, k)] = p.ibas_aab[at(j, i, k)] = ta;
                    p.bas_aab.push_back(i);
                    p.bas_aab.push_back(j);
                    p.bas_aab.push_back(k);
                    if (k > j) {
                        const int t3 = (int)(p.bas_aaa.size() / 3);
                        for (size_t e : {at(i, j, k), at(i, k, j), at(j, i, k), at(j, k, i), at(k, i, j), at(k, j, i)})
                            p.ibas_aaa[e] = t3;
                        p.bas_aaa.push_back(i);
                        p.bas_aaa.push_back(j);
                        p.bas_aaa.push_back(k);
                    }
                }
        p.trip_aab = (int)(p.bas_aab.size() / 3);
        p.trip_aaa = (int)(p.bas_aaa.size() / 3);
    }
    if (p.d4) {   // basis.cc:747-900
        const size_t n4 = (size_t)n * n * n * n;
        p.ibas_aaaa.assign(n4, -999);
        p.ibas_aaab.assign(n4, -999);
        p.ibas_aabb.assign(n4, -999);
        auto at = [&](int a, int b, int c, int d) { return (((size_t)a * n + b) * n + c) * n + d; };
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++)
                    for (int l = 0; l < n; l++) {
                        if (i < j && k < l) {
                            for (size_t e : {at(i, j, k, l), at(j, i, k, l), at(i, j, l, k), at(j, i, l, k)})
                                p.ibas_aabb[e] = p.quad_aabb;
                            p.quad_aabb++;
                        }
                        if (i < j && j < k) {
                            const int t[3] = {i, j, k};
                            for (int a = 0; a < 3; a++)
                                for (int b = 0; b < 3; b++)
                                    if (a != b) p.ibas_aaab[at(t[a], t[b], t[3 - a - b], l)] = p.quad_aaab;
                            p.quad_aaab++;
                        }
                        if (i < j && j < k && k < l) {
                            const int t[4] = {i, j, k, l};
                            for (int a = 0; a < 4; a++)
                                for (int b = 0; b < 4; b++)
                                    for (int c = 0; c < 4; c++)
                                        if (a != b && a != c && b != c)
                                            p.ibas_aaaa[at(t[a], t[b], t[c], t[6 - a - b - c])] = p.quad_aaaa;
                            p.quad_aaaa++;
                        }
                    }
    }
    if (p.t1) {   // v2rdm_solver.cc:3848-3877
        add_block(p.t1aaa, p.trip_aaa);
        add_block(p.t1bbb, p.trip_aaa);
        add_block(p.t1aab, p.trip_aab);
        add_block(p.t1bba, p.trip_aab);
    }
    if (p.t2) {   // v2rdm_solver.cc:3879-3906
        add_block(p.t2aaa, p.trip_aab + p.trip_aba);
        add_block(p.t2bbb, p.trip_aab + p.trip_aba);
        add_block(p.t2aab, p.trip_aab);
        add_block(p.t2bba, p.trip_aab);
    }
    if (p.e3) {   // v2rdm_solver.cc:3909-3938
        add_block(p.e3aaa, p.trip_aab + p.trip_aba);
        add_block(p.e3bbb, p.trip_aab + p.trip_aba);
        add_block(p.e3aab, p.trip_aab);
        add_block(p.e3bba, p.trip_aab);
    }
    if (p.f3) {   // v2rdm_solver.cc:3940-3968
        add_block(p.f3aaa, p.trip_aab + p.trip_aba);
        add_block(p.f3bbb, p.trip_aab + p.trip_aba);
        add_block(p.f3aab, p.trip_aab);
        add_block(p.f3bba, p.trip_aab);
    }
    if (p.q3) {   // v2rdm_solver.cc:3970-3998
        add_block(p.q3aaa, p.trip_aaa);
        add_block(p.q3bbb, p.trip_aaa);
        add_block(p.q3aab, p.trip_aab);
        add_block(p.q3bba, p.trip_aab);
    }
    if (p.d3) {   // v2rdm_solver.cc:4000-4029
        add_block(p.d3aaa, p.trip_aaa);
        add_block(p.d3bbb, p.trip_aaa);
        add_block(p.d3aab, p.trip_aab);
        add_block(p.d3bba, p.trip_aab);
    }
    if (p.d4) {   // v2rdm_solver.cc:4030-4061
        add_block(p.d4aaaa, p.quad_aaaa);
        add_block(p.d4aaab, p.quad_aaab);
        add_block(p.d4aabb, p.quad_aabb);
        add_block(p.d4bbba, p.quad_aaab);
        add_block(p.d4bbbb, p.quad_aaaa);
    }
    p.n_primal = off;

    const int64_t gab2 = (int64_t)p.gab * p.gab, gaa2 = (int64_t)p.gaa * p.gaa, n2 = (int64_t)n * n;
    int64_t d = spec.constrain_sz ? 3 : 1;
    d += 2 * gaa2 + gab2 + 2 * n2 + (spec.constrain_sz ? 4 : 2) * n2;
    if (spec.constrain_spin) {
        d += 1 + (singlet ? n2 + 3 * gaa2 + 2 * gab2 : 4 * gab2);
        if (p.g2) d += 2 * (int64_t)p.gab;
    }
    if (p.q2) d += gab2 + 2 * gaa2;
    if (p.g2) d += 6 * gab2;
    if (p.t1) d += 2 * (int64_t)p.trip_aaa * p.trip_aaa + 2 * (int64_t)p.trip_aab * p.trip_aab;
    if (p.t2) {
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        d += 2 * aab * aab + 2 * big * big;
    }
    if (p.e3) {
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        d += 2 * aab * aab + 2 * big * big;
    }
    if (p.f3) {
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        d += 2 * aab * aab + 2 * big * big;
    }
    if (p.q3) d += 2 * (int64_t)p.trip_aaa * p.trip_aaa + 2 * (int64_t)p.trip_aab * p.trip_aab;
    if (p.d3) {   // v2rdm_solver.cc:3624-3660
        d += spec.constrain_sz ? 4 * gaa2 + 2 * gab2 : 2 * gaa2 + gab2;
        if (spec.constrain_spin && singlet)
            d += (int64_t)p.trip_aab * p.trip_aab + 2 * (int64_t)p.trip_aaa * p.trip_aaa;
    }
    if (p.d4) {   // v2rdm_solver.cc:3678-3720
        const int64_t t3 = p.trip_aaa, ta = p.trip_aab;
        const int na = spec.nalpha, nb = spec.nbeta;
        if (na > 3) d += t3 * t3;
        if (na > 2 && nb > 0) d += t3 * t3 + ta * ta;
        // the reference counts the aabb family twice and writes it once: the
        // second 2 aab^2 rows are empty, at the end of the dual vector
        if (na > 1 && nb > 1) d += 4 * ta * ta;
        if (na > 0 && nb > 2) d += t3 * t3 + ta * ta;
        if (nb > 3) d += t3 * t3;
    }
    p.n_dual = d;
    if (p.n_primal > (int64_t)kColMask || p.n_dual > (int64_t)kColMask)
        throw std::invalid_argument("problem too large for 27-bit packed column indices");
    return p;
}

// ------------------------------------------------------------------ b, c, x
void build_b(const Problem &p, double *b) {
    if (p.spec.batch_parts) throw std::invalid_argument("a batch's b is its parts' b, concatenated");
    if (p.spec.doci) return doci_build_b(p, b);
    const int n = p.n, gab = p.gab, gaa = p.gaa;
    const double na = p.spec.nalpha, nb = p.spec.nbeta;
    std::memset(b, 0, sizeof(double) * p.n_dual);
    int64_t off = 0;
    if (p.spec.constrain_sz) {
        b[off++] = na * nb;
        b[off++] = na * (na - 1.0);
        b[off++] = nb * (nb - 1.0);
    } else {
        const double nt = na + nb;
        b[off++] = nt * (nt - 1.0);
    }
    off += 2 * (int64_t)gaa * gaa + (int64_t)gab * gab;
    for (int s = 0; s < 2; s++) {
        for (int i = 0; i < n; i++) b[off + i * n + i] = 1.0;
        off += (int64_t)n * n;
    }
    off += (p.spec.constrain_sz ? 4 : 2) * (int64_t)n * n;
    if (p.spec.constrain_spin) {
        const double ms = (p.mult - 1.0) / 2.0;
        b[off++] = 0.5 * (na + nb) + ms * ms - ms * (ms + 1.0);
        if (p.spec.nalpha == p.spec.nbeta)
            off += (int64_t)n * n + 3 * (int64_t)gaa * gaa + 2 * (int64_t)gab * gab;
        else
            off += 4 * (int64_t)gab * gab;
        if (p.g2) off += 2 * (int64_t)gab;
    }
    if (p.q2) {
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            b[off + (int64_t)ij * gab + p.iab(i, j)] = -1.0;  // -d_ik d_jl
        }
        off += (int64_t)gab * gab;
        for (int s = 0; s < 2; s++) {
            for (int ij = 0; ij < gaa; ij++) {
                const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                    b[off + (int64_t)ij * gaa + kl] = -(double)((i == k) && (j == l)) + (double)((i == l) && (j == k));
                }
            }
            off += (int64_t)gaa * gaa;
        }
    }
}

namespace {
// D1 from the upper triangle of h, as the packed one-electron buffer of
// tei.cc:96-120 leaves it, plus the (zero) core contribution of tei.cc:236-270.
void fill_d1(const Problem &p, const double *hsym, double *c) {
    const int n = p.n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            const double v = hsym[(i < j ? i : j) * n + (i < j ? j : i)];
            c[p.d1a + i * n + j] = v + 0.0;
            c[p.d1b + i * n + j] = v + 0.0;
        }
}
}  // namespace

void build_c_hubbard(const Problem &p, double t, double U, double *c) {
    if (p.spec.batch_parts) throw std::invalid_argument("a batch's c is its parts' c, concatenated");
    if (p.spec.doci) throw std::invalid_argument("v2RDM-DOCI has no Hubbard Hamiltonian: pass h and g");
    const int n = p.n, gab = p.gab;
    std::memset(c, 0, sizeof(double) * p.n_primal);
    std::vector<double> h((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            const int d = std::abs(i - j);
            if (d == 1 || d == n - 1) h[i * n + j] = -t;   // oei.cc:83-88
        }
    fill_d1(p, h.data(), c);
    for (int i = 0; i < n; i++) {
        const int ii = p.iab(i, i);
        c[p.d2ab + (int64_t)ii * gab + ii] = U;             // tei.cc:285-292
    }
}

void build_c_external(const Problem &p, const double *h, const double *g, double *c) {
    if (p.spec.batch_parts) throw std::invalid_argument("a batch's c is its parts' c, concatenated");
    if (p.spec.doci) return doci_build_c_external(p, h, g, c);
    const int64_t n = p.n;
    const int gab = p.gab, gaa = p.gaa;
    std::memset(c, 0, sizeof(double) * p.n_primal);
    fill_d1(p, h, c);
    for (int ij = 0; ij < gab; ij++) {
        const int64_t i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            const int64_t k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
            c[p.d2ab + (int64_t)ij * gab + kl] = g[((i * n + k) * n + j) * n + l];
        }
    }
    for (int ij = 0; ij < gaa; ij++) {
        const int64_t i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
        for (int kl = 0; kl < gaa; kl++) {
            const int64_t k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
            const double v = g[((i * n + k) * n + j) * n + l] - g[((i * n + l) * n + j) * n + k];
            c[p.d2aa + (int64_t)ij * gaa + kl] = v;
            c[p.d2bb + (int64_t)ij * gaa + kl] = v;
        }
    }
}

// ------------------------------------------------------------------ T2
// The T2 rows (t2.cc:1236-1843, T2_constraints_Au_slow, C1): one row per
// element (I, J) of the T2aab, T2bba, T2aaa and T2bbb blocks, in that order of
// dual rows, each -T2(I, J) + delta-masked D2 and D1 terms with coefficients
// +-1.  f(dual_row, t2_col, sub, cols, coefs, nterms) receives a row's D terms
// in the order the reference adds them, rows in the reference's loop order
// (which is also the order T2_constraints_ATu_slow scatters them, t2.cc:3376).
// sub numbers the sub-blocks 0 aab, 1 bba, 2-5 aaa (aaa/aaa, aaa/abb, abb/aaa,
// abb/abb), 6-9 bbb (bbb/bbb, bbb/baa, baa/bbb, baa/baa).
namespace {
constexpr int kT2AaaAbb = 3;

// ------------------------------------------------------------------ T1
// The T1 rows (t1.cc:419-795, T1_constraints_Au, C1): one row per element
// of T1aab, T1bba (aab triplets) and T1aaa, T1bbb (aaa triplets, i < j < k),
// in that order of dual rows, each -T1(I, J) + delta-masked Q2, D2, G2 and
// D1 terms with coefficients +-1.  f(dual_row, t1_col, sub, cols, coefs,
// nterms) receives them in the reference's order; T1_constraints_ATu
// (t1.cc:795-1200) scatters the same terms in the same order, and the guess
// (t1.cc:45-419) sums them from zero.
// The Q3 rows (q3.cc:45-423, scatter :425-803) carry the same terms with
// -Q3 - D3 in front: t1_rows(p, off, f, true) hands f the Q3 element as the
// leading column (its D3 twin sits at the same place in the D3 block).
template <class F>
void t1_rows(const Problem &p, int64_t off, F &&f, bool q3 = false) {
    const int N = p.n, gab = p.gab, gaa = p.gaa;
    int64_t cols[12];
    double coef[12];
    int nt = 0;
    auto add = [&](int64_t c, double v) {
        cols[nt] = c;
        coef[nt] = v;
        nt++;
    };
    auto aa = [&](int64_t base, int a, int b, int c, int d) { return base + (int64_t)p.iaa(a, b) * gaa + p.iaa(c, d); };
    auto ab = [&](int64_t base, int a, int b, int c, int d) { return base + (int64_t)p.iab(a, b) * gab + p.iab(c, d); };
    for (int sub = 0; sub < 4; sub++) {
        const bool aab = sub < 2, beta = (sub % 2) == 1;
        const std::vector<int> &tb = aab ? p.bas_aab : p.bas_aaa;
        const int nr = aab ? p.trip_aab : p.trip_aaa;
        const int64_t t1 = q3 ? (sub == 0 ? p.q3aab : sub == 1 ? p.q3bba : sub == 2 ? p.q3aaa : p.q3bbb)
                              : (sub == 0 ? p.t1aab : sub == 1 ? p.t1bba : sub == 2 ? p.t1aaa : p.t1bbb);
        const int64_t q2 = beta ? p.q2bb : p.q2aa;
        for (int r = 0; r < nr; r++) {
            const int i = tb[3 * r], j = tb[3 * r + 1], k = tb[3 * r + 2];
            for (int c = 0; c < nr; c++) {
                const int l = tb[3 * c], m = tb[3 * c + 1], n = tb[3 * c + 2];
                nt = 0;
                if (aab) {   // t1.cc:421-515
                    const int64_t g2 = beta ? p.g2ab : p.g2ba;
                    if (k == n) add(aa(q2, i, j, l, m), 1.0);
                    if (j == l) add(beta ? ab(p.d2ab, n, m, k, i) : ab(p.d2ab, m, n, i, k), -1.0);
                    if (l == i) add(beta ? ab(p.d2ab, n, m, k, j) : ab(p.d2ab, m, n, j, k), 1.0);
                    if (j == m) add(ab(g2, n, i, k, l), -1.0);
                    if (i == m) add(ab(g2, n, j, k, l), 1.0);
                } else {     // t1.cc:517-793
                    const int64_t d2 = beta ? p.d2bb : p.d2aa, d1 = beta ? p.d1b : p.d1a;
                    const int64_t sh = beta ? gab : 0, w = 2 * (int64_t)gab;
                    auto g2 = [&](int a, int b, int cc, int d) {
                        return p.g2aa + (p.iab(a, b) + sh) * w + (p.iab(cc, d) + sh);
                    };
                    if (k == n) add(aa(q2, i, j, l, m), 1.0);
                    if (j == n) add(aa(q2, i, k, l, m), -1.0);
                    if (i == n) add(aa(q2, j, k, l, m), 1.0);
                    if (l == k) add(aa(d2, n, m, j, i), 1.0);
                    if (j == l) add(aa(d2, n, m, k, i), -1.0);
                    if (l == i) add(aa(d2, n, m, k, j), 1.0);
                    if (k == m) {
                        if (j == l) add(d1 + (int64_t)n * N + i, -1.0);
                        add(g2(n, i, j, l), 1.0);
                    }
                    if (j == m) {
                        if (k == l) add(d1 + (int64_t)n * N + i, 1.0);
                        add(g2(n, i, k, l), -1.0);
                    }
                    if (i == m) {
                        if (k == l) add(d1 + (int64_t)n * N + j, -1.0);
                        add(g2(n, j, k, l), 1.0);
                    }
                }
                const int64_t e = (int64_t)r * nr + c;
                f(off + e, t1 + e, sub, cols, coef, nt);
            }
        }
        off += (int64_t)nr * nr;
    }
}

// the D3 element at the place of a Q3 element (blocks of equal shape)
int64_t d3_twin(const Problem &p, int64_t q3col) {
    if (q3col >= p.q3bba) return p.d3bba + (q3col - p.q3bba);
    if (q3col >= p.q3aab) return p.d3aab + (q3col - p.q3aab);
    if (q3col >= p.q3bbb) return p.d3bbb + (q3col - p.q3bbb);
    return p.d3aaa + (q3col - p.q3aaa);
}

// ------------------------------------------------------------------ D3
// CONSTRAIN_D3 rows (d3.cc:45-406, D3_constraints_Au, C1): plain term lists,
// first a D2 element times an electron count, then D3 elements with
// coefficients -+1 (contractions D3 -> D2, with CONSTRAIN_SZ six families,
// d3.cc:49-212, without it three, :213-330) and, for singlets with
// CONSTRAIN_SPIN, D3aab - D3bba and D3aaa (D3bbb) minus a third of nine D3aab
// (D3bba) elements (:332-404).  D3_constraints_ATu (d3.cc:408-766) scatters
// the same terms in the same order.  f(dual_row, cols, coefs, nterms).
template <class F>
void d3_rows(const Problem &p, int64_t off, F &&f) {
    const int N = p.n, gab = p.gab, gaa = p.gaa;
    const int64_t t3 = p.trip_aaa, ta = p.trip_aab;
    const double na = p.spec.nalpha, nb = p.spec.nbeta;
    const bool sz = p.spec.constrain_sz;
    std::vector<int64_t> cols;
    std::vector<double> coef;
    auto add = [&](int64_t c, double v) {
        cols.push_back(c);
        coef.push_back(v);
    };
    auto emit = [&]() {
        f(off++, cols.data(), coef.data(), (int)cols.size());
        cols.clear();
        coef.clear();
    };
    auto aaa = [&](int a, int b, int c) { return (int64_t)p.ibas_aaa[((size_t)a * N + b) * N + c]; };
    auto aab = [&](int a, int b, int c) { return (int64_t)p.ibas_aab[((size_t)a * N + b) * N + c]; };
    // parity of sorting (a, b, q) with a < b into triplet order: odd when a < q < b
    auto mid = [](int a, int q, int b) { return (a < q && q < b) ? -1.0 : 1.0; };
    for (int fam = 0; fam < (sz ? 4 : 2); fam++) {
        const bool beta = fam % 2 == 1;
        const int64_t d2 = beta ? p.d2bb : p.d2aa;
        const int64_t same = beta ? p.d3bbb : p.d3aaa, mixed = beta ? p.d3bba : p.d3aab;
        for (int ij = 0; ij < gaa; ij++) {
            const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
            for (int kl = 0; kl < gaa; kl++) {
                const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                const int64_t d2e = d2 + (int64_t)ij * gaa + kl;
                if (sz && fam < 2) {
                    add(d2e, (beta ? nb : na) - 2.0);
                    for (int q = 0; q < N; q++) {
                        if (q == i || q == j || q == k || q == l) continue;
                        add(same + aaa(i, j, q) * t3 + aaa(k, l, q), -mid(i, q, j) * mid(k, q, l));
                    }
                } else if (sz) {
                    add(d2e, beta ? na : nb);
                    for (int q = 0; q < N; q++) add(mixed + aab(i, j, q) * ta + aab(k, l, q), -1.0);
                } else {
                    add(d2e, na + nb - 2.0);
                    for (int q = 0; q < N; q++) {
                        add(mixed + aab(i, j, q) * ta + aab(k, l, q), -1.0);
                        if (q == i || q == j || q == k || q == l) continue;
                        add(same + aaa(i, j, q) * t3 + aaa(k, l, q), -mid(i, q, j) * mid(k, q, l));
                    }
                }
                emit();
            }
        }
    }
    for (int fam = 0; fam < (sz ? 2 : 1); fam++) {
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                add(p.d2ab + (int64_t)ij * gab + kl, !sz ? na + nb - 2.0 : (fam ? nb - 1.0 : na - 1.0));
                for (int q = 0; q < N; q++) {
                    if ((!sz || fam == 0) && q != i && q != k)
                        add(p.d3aab + aab(i, q, j) * ta + aab(k, q, l), -((q < i ? -1.0 : 1.0) * (q < k ? -1.0 : 1.0)));
                    if ((!sz || fam == 1) && q != j && q != l)
                        add(p.d3bba + aab(j, q, i) * ta + aab(l, q, k), -((q < j ? -1.0 : 1.0) * (q < l ? -1.0 : 1.0)));
                }
                emit();
            }
        }
    }
    if (p.spec.constrain_spin && p.spec.nalpha == p.spec.nbeta) {
        for (int64_t e = 0; e < ta * ta; e++) {
            add(p.d3aab + e, 1.0);
            add(p.d3bba + e, -1.0);
            emit();
        }
        const double third = 1.0 / 3.0;
        for (int beta = 0; beta < 2; beta++) {
            const int64_t same = beta ? p.d3bbb : p.d3aaa, mixed = beta ? p.d3bba : p.d3aab;
            for (int64_t r = 0; r < t3; r++) {
                const int a = p.bas_aaa[3 * r], b = p.bas_aaa[3 * r + 1], c = p.bas_aaa[3 * r + 2];
                const int64_t rr[3] = {aab(a, b, c), aab(a, c, b), aab(b, c, a)};
                for (int64_t s = 0; s < t3; s++) {
                    const int x = p.bas_aaa[3 * s], y = p.bas_aaa[3 * s + 1], z = p.bas_aaa[3 * s + 2];
                    const int64_t cc[3] = {aab(x, y, z), aab(x, z, y), aab(y, z, x)};
                    add(same + r * t3 + s, 1.0);
                    for (int u = 0; u < 3; u++)
                        for (int v = 0; v < 3; v++) add(mixed + rr[u] * ta + cc[v], (u + v) % 2 ? third : -third);
                    emit();
                }
            }
        }
    }
}

// ------------------------------------------------------------------ E3
// CONSTRAIN_E3 rows (e3.cc:45-566, E3_constraints_Au, C1) in the T2 layout
// (sub-blocks 0 aab, 1 bba, 2-5 aaa, 6-9 bbb as for T2): -E3(I, J), one D3
// element whose third index is exchanged between row and column,
// (i j n | l m k), with the sign that reorders it, and d_kn times a D2
// element.  E3_constraints_ATu (e3.cc:570-1082) scatters the same terms in
// the same order.  f(dual_row, e3_col, sub, cols, coefs, nterms).
template <class F>
void e3_rows(const Problem &p, int64_t off, F &&f) {
    const int N = p.n, gab = p.gab, gaa = p.gaa, aab = p.trip_aab, aba = p.trip_aba;
    const int64_t big = (int64_t)aab + aba, t3 = p.trip_aaa;
    int64_t cols[4];
    double coef[4];
    int nt = 0;
    auto add = [&](int64_t c, double v) {
        cols[nt] = c;
        coef[nt] = v;
        nt++;
    };
    auto trip = [&](int idx, bool is_aab, int &i, int &j, int &k) {
        if (is_aab) {
            i = p.bas_aab[3 * idx];
            j = p.bas_aab[3 * idx + 1];
            k = p.bas_aab[3 * idx + 2];
        } else {
            i = idx / (N * N);
            j = (idx / N) % N;
            k = idx % N;
        }
    };
    auto x3 = [&](int a, int b, int c) { return (int64_t)p.ibas_aab[((size_t)a * N + b) * N + c]; };
    auto y3 = [&](int a, int b, int c) { return (int64_t)p.ibas_aaa[((size_t)a * N + b) * N + c]; };
    auto mixed = [&](int64_t base, int a, int b, int c, int d, int e, int g) { return base + x3(a, b, c) * aab + x3(d, e, g); };
    auto same = [&](int64_t base, int a, int b, int c, int d, int e, int g) { return base + y3(a, b, c) * t3 + y3(d, e, g); };
    auto aa2 = [&](int64_t base, int a, int b, int c, int d) { return base + (int64_t)p.iaa(a, b) * gaa + p.iaa(c, d); };
    auto ab2 = [&](int a, int b, int c, int d) { return p.d2ab + (int64_t)p.iab(a, b) * gab + p.iab(c, d); };
    auto neg = [](bool flip) { return flip ? -1.0 : 1.0; };

    for (int spin = 0; spin < 2; spin++) {   // E3aab (e3.cc:47-92), E3bba (:94-139)
        const int64_t e3 = spin ? p.e3bba : p.e3aab;
        for (int ijk = 0; ijk < aab; ijk++) {
            int i, j, k;
            trip(ijk, true, i, j, k);
            for (int lmn = 0; lmn < aab; lmn++) {
                int l, m, n;
                trip(lmn, true, l, m, n);
                nt = 0;
                add(mixed(spin ? p.d3bba : p.d3aab, i, j, n, l, m, k), -1.0);
                if (k == n) add(aa2(spin ? p.d2bb : p.d2aa, i, j, l, m), 1.0);
                const int64_t e = (int64_t)ijk * aab + lmn;
                f(off + e, e3 + e, spin, cols, coef, nt);
            }
        }
        off += (int64_t)aab * aab;
    }
    for (int spin = 0; spin < 2; spin++) {   // E3aaa (e3.cc:142-355), E3bbb (:359-564)
        const int64_t e3 = spin ? p.e3bbb : p.e3aaa;
        for (int sb = 0; sb < 4; sb++) {
            const bool rowaab = sb < 2, colaab = (sb % 2) == 0;
            const int nr = rowaab ? aab : aba, nc = colaab ? aab : aba;
            for (int ijk = 0; ijk < nr; ijk++) {
                int i, j, k;
                trip(ijk, rowaab, i, j, k);
                for (int lmn = 0; lmn < nc; lmn++) {
                    int l, m, n;
                    trip(lmn, colaab, l, m, n);
                    nt = 0;
                    if (sb == 0) {
                        if (i != n && j != n && l != k && m != k)
                            add(same(spin ? p.d3bbb : p.d3aaa, i, j, n, l, m, k),
                                -(neg(i < n && n < j) * neg(l < k && k < m)));
                        if (k == n) add(aa2(spin ? p.d2bb : p.d2aa, i, j, l, m), 1.0);
                    } else if (sb == 1) {
                        if (i != j && l != k)
                            add(mixed(spin ? p.d3bba : p.d3aab, i, j, n, l, k, m),
                                spin ? neg(i > j) * neg(l > k) : neg(l > k));
                    } else if (sb == 2) {
                        if (i != n && l != m)
                            add(mixed(spin ? p.d3bba : p.d3aab, i, n, j, l, m, k),
                                spin ? neg(i > n) * neg(l > m) : neg(i > n));
                    } else {
                        if (j != n && m != k)
                            add(mixed(spin ? p.d3aab : p.d3bba, j, n, i, m, k, l), -(neg(j > n) * neg(m > k)));
                        if (k == n) add(spin ? ab2(j, i, m, l) : ab2(i, j, l, m), 1.0);
                    }
                    const int64_t I = rowaab ? ijk : aab + ijk, J = colaab ? lmn : aab + lmn;
                    const int64_t e = I * big + J;
                    f(off + e, e3 + e, 2 + 4 * spin + sb, cols, coef, nt);
                }
            }
        }
        off += big * big;
    }
}

// f3 = true gives the CONSTRAIN_F3 rows (f3.cc:45-836, scatter :842-1623):
// led by F3, then the D3 element of the E3 row with the opposite sign, then
// the T2 terms without the d_kn D2 term (T2 = E3 + F3).
// ------------------------------------------------------------------ D4
// CONSTRAIN_D4 rows (d4.cc:44-297, scatter :300-557): contractions of the
// 4-RDM to the 3-RDM, families gated on the electron counts, in the
// reference's order: aaaa->aaa (na > 3); aaab->aaa, aaab->aab (na > 2,
// nb > 0); aabb->aab, aabb->bba (na, nb > 1); bbba->bbb, bbba->bba (na > 0,
// nb > 2); bbbb->bbb (nb > 3).  A row: count x D3 element - sum_p (sign) D4
// element; the sign is the parity of the positions p passes.  f(dual_row,
// cols, coefs, nterms); returns the rows written.
template <class F>
int64_t d4_rows(const Problem &p, int64_t off, F &&f) {
    const int N = p.n, na = p.spec.nalpha, nb = p.spec.nbeta;
    const int64_t t3 = p.trip_aaa, ta = p.trip_aab;
    const int64_t q4 = p.quad_aaaa, q31 = p.quad_aaab, q22 = p.quad_aabb;
    const int64_t first = off;
    std::vector<int64_t> cols;
    std::vector<double> coef;
    auto at = [&](int a, int b, int c, int d) { return (((size_t)a * N + b) * N + c) * N + d; };
    auto lt = [](int q, int x) { return q < x ? -1.0 : 1.0; };
    for (int fam = 0; fam < 8; fam++) {
        bool on;
        switch (fam) {
            case 0: on = na > 3; break;
            case 1: case 2: on = na > 2 && nb > 0; break;
            case 3: case 4: on = na > 1 && nb > 1; break;
            case 5: case 6: on = na > 0 && nb > 2; break;
            default: on = nb > 3; break;
        }
        if (!on) continue;
        const bool aaa_rows = fam == 0 || fam == 1 || fam == 5 || fam == 7;
        const int64_t nr = aaa_rows ? t3 : ta;
        const std::vector<int> &tb = aaa_rows ? p.bas_aaa : p.bas_aab;
        for (int64_t x = 0; x < nr; x++) {
            const int i = tb[3 * x], j = tb[3 * x + 1], k = tb[3 * x + 2];
            for (int64_t y = 0; y < nr; y++) {
                const int l = tb[3 * y], m = tb[3 * y + 1], n = tb[3 * y + 2];
                const int64_t e = x * nr + y;
                cols.clear();
                coef.clear();
                auto add = [&](int64_t c, double v) {
                    cols.push_back(c);
                    coef.push_back(v);
                };
                if (fam == 0 || fam == 7) {
                    add((fam ? p.d3bbb : p.d3aaa) + e, fam ? nb - 3.0 : na - 3.0);
                    for (int q = 0; q < N; q++) {
                        if (q == i || q == j || q == k || q == l || q == m || q == n) continue;
                        const double sg = lt(q, i) * lt(q, j) * lt(q, k) * lt(q, l) * lt(q, m) * lt(q, n);
                        add((fam ? p.d4bbbb : p.d4aaaa) + (int64_t)p.ibas_aaaa[at(i, j, k, q)] * q4 +
                                p.ibas_aaaa[at(l, m, n, q)], -sg);
                    }
                } else if (fam == 1 || fam == 5) {
                    add((fam == 5 ? p.d3bbb : p.d3aaa) + e, fam == 5 ? (double)na : (double)nb);
                    for (int q = 0; q < N; q++)
                        add((fam == 5 ? p.d4bbba : p.d4aaab) + (int64_t)p.ibas_aaab[at(i, j, k, q)] * q31 +
                                p.ibas_aaab[at(l, m, n, q)], -1.0);
                } else if (fam == 2 || fam == 6) {
                    add((fam == 6 ? p.d3bba : p.d3aab) + e, fam == 6 ? nb - 2.0 : na - 2.0);
                    for (int q = 0; q < N; q++) {
                        if (q == i || q == j || q == l || q == m) continue;
                        const double sg = lt(q, i) * lt(q, j) * lt(q, l) * lt(q, m);
                        add((fam == 6 ? p.d4bbba : p.d4aaab) + (int64_t)p.ibas_aaab[at(i, j, q, k)] * q31 +
                                p.ibas_aaab[at(l, m, q, n)], -sg);
                    }
                } else if (fam == 3) {
                    add(p.d3aab + e, nb - 1.0);
                    for (int q = 0; q < N; q++) {
                        if (q == k || q == n) continue;
                        add(p.d4aabb + (int64_t)p.ibas_aabb[at(i, j, k, q)] * q22 + p.ibas_aabb[at(l, m, n, q)],
                            -(lt(q, k) * lt(q, n)));
                    }
                } else {   // fam == 4
                    add(p.d3bba + e, na - 1.0);
                    for (int q = 0; q < N; q++) {
                        if (q == k || q == n) continue;
                        add(p.d4aabb + (int64_t)p.ibas_aabb[at(k, q, i, j)] * q22 + p.ibas_aabb[at(n, q, l, m)],
                            -(lt(q, k) * lt(q, n)));
                    }
                }
                f(off++, cols.data(), coef.data(), (int)cols.size());
            }
        }
    }
    return off - first;
}

template <class F>
void t2_rows(const Problem &p, int64_t off, F &&f, bool f3 = false) {
    const int N = p.n, gab = p.gab, gaa = p.gaa, aab = p.trip_aab, aba = p.trip_aba;
    const int64_t big = (int64_t)aab + aba, t3 = p.trip_aaa;
    int64_t cols[9];
    double coef[9];
    int nt = 0;
    auto add = [&](int64_t c, double v) {
        cols[nt] = c;
        coef[nt] = v;
        nt++;
    };
    auto trip = [&](int idx, bool is_aab, int &i, int &j, int &k) {
        if (is_aab) {
            i = p.bas_aab[3 * idx];
            j = p.bas_aab[3 * idx + 1];
            k = p.bas_aab[3 * idx + 2];
        } else {
            i = idx / (N * N);
            j = (idx / N) % N;
            k = idx % N;
        }
    };
    auto d2aa_t = [&](int64_t base, int a, int b, int c, int d) { return base + (int64_t)p.iaa(a, b) * gaa + p.iaa(c, d); };
    auto d2ab_t = [&](int a, int b, int c, int d) { return p.d2ab + (int64_t)p.iab(a, b) * gab + p.iab(c, d); };
    // sign of the aa geminal terms: s = (n > j ? -1 : 1) (k > m ? -1 : 1)
    auto sgn = [](int a, int b, int c, int d) { return (a > b ? -1.0 : 1.0) * (c > d ? -1.0 : 1.0); };
    auto x3 = [&](int a, int b, int c) { return (int64_t)p.ibas_aab[((size_t)a * N + b) * N + c]; };
    auto y3 = [&](int a, int b, int c) { return (int64_t)p.ibas_aaa[((size_t)a * N + b) * N + c]; };
    auto mixed = [&](int64_t base, int a, int b, int c, int d, int e, int g) { return base + x3(a, b, c) * aab + x3(d, e, g); };
    auto neg = [](bool flip) { return flip ? -1.0 : 1.0; };

    // T2aab (t2.cc:1239-1302) and T2bba (t2.cc:1305-1368)
    for (int spin = 0; spin < 2; spin++) {
        const int64_t t2 = f3 ? (spin ? p.f3bba : p.f3aab) : (spin ? p.t2bba : p.t2aab);
        const int64_t d2same = spin ? p.d2bb : p.d2aa, d1other = spin ? p.d1a : p.d1b;
        for (int ijk = 0; ijk < aab; ijk++) {
            int i, j, k;
            trip(ijk, true, i, j, k);
            for (int lmn = 0; lmn < aab; lmn++) {
                int l, m, n;
                trip(lmn, true, l, m, n);
                nt = 0;
                if (f3) add(mixed(spin ? p.d3bba : p.d3aab, i, j, n, l, m, k), 1.0);
                else if (k == n) add(d2aa_t(d2same, i, j, l, m), 1.0);
                if (j == m && i == l) add(d1other + (int64_t)n * N + k, 1.0);
                if (j == l && i == m) add(d1other + (int64_t)n * N + k, -1.0);
                if (spin == 0) {
                    if (i == l) add(d2ab_t(j, n, m, k), -1.0);
                    if (j == l) add(d2ab_t(i, n, m, k), 1.0);
                    if (i == m) add(d2ab_t(j, n, l, k), 1.0);
                    if (j == m) add(d2ab_t(i, n, l, k), -1.0);
                } else {
                    if (i == l) add(d2ab_t(n, j, k, m), -1.0);
                    if (j == l) add(d2ab_t(n, i, k, m), 1.0);
                    if (i == m) add(d2ab_t(n, j, k, l), 1.0);
                    if (j == m) add(d2ab_t(n, i, k, l), -1.0);
                }
                const int64_t e = (int64_t)ijk * aab + lmn;
                f(off + e, t2 + e, spin, cols, coef, nt);
            }
        }
        off += (int64_t)aab * aab;
    }
    // big blocks T2aaa (t2.cc:1371-1601) and T2bbb (t2.cc:1604-1840)
    for (int spin = 0; spin < 2; spin++) {
        const int64_t t2 = f3 ? (spin ? p.f3bbb : p.f3aaa) : (spin ? p.t2bbb : p.t2aaa);
        const int64_t d2s = spin ? p.d2bb : p.d2aa, d2o = spin ? p.d2aa : p.d2bb;
        const int64_t d1s = spin ? p.d1b : p.d1a, d1o = spin ? p.d1a : p.d1b;
        for (int sb = 0; sb < 4; sb++) {
            const bool rowaab = sb < 2, colaab = (sb % 2) == 0;
            const int nr = rowaab ? aab : aba, nc = colaab ? aab : aba;
            for (int ijk = 0; ijk < nr; ijk++) {
                int i, j, k;
                trip(ijk, rowaab, i, j, k);
                for (int lmn = 0; lmn < nc; lmn++) {
                    int l, m, n;
                    trip(lmn, colaab, l, m, n);
                    nt = 0;
                    if (sb == 0) {   // aaa/aaa, bbb/bbb
                        if (f3) {
                            if (i != n && j != n && l != k && m != k)
                                add((spin ? p.d3bbb : p.d3aaa) + y3(i, j, n) * t3 + y3(l, m, k),
                                    neg(i < n && n < j) * neg(l < k && k < m));
                        } else if (k == n) {
                            add(d2aa_t(d2s, i, j, l, m), 1.0);
                        }
                        if (j == m && i == l) add(d1s + (int64_t)n * N + k, 1.0);
                        if (j == l && i == m) add(d1s + (int64_t)n * N + k, -1.0);
                        if (i == l && n != j && k != m) add(d2aa_t(d2s, n, j, k, m), -sgn(n, j, k, m));
                        if (j == l && n != i && k != m) add(d2aa_t(d2s, n, i, k, m), sgn(n, i, k, m));
                        if (i == m && n != j && k != l) add(d2aa_t(d2s, n, j, k, l), sgn(n, j, k, l));
                        if (j == m && n != i && k != l) add(d2aa_t(d2s, n, i, k, l), -sgn(n, i, k, l));
                    } else if (sb == 1) {   // aaa/abb, bbb/baa
                        if (f3 && i != j && l != k)
                            add(mixed(spin ? p.d3bba : p.d3aab, i, j, n, l, k, m),
                                -(spin ? neg(i > j) * neg(l > k) : neg(l > k)));
                        if (spin == 0) {
                            if (i == l) add(d2ab_t(j, n, k, m), 1.0);
                            if (j == l) add(d2ab_t(i, n, k, m), -1.0);
                        } else {
                            if (i == l) add(d2ab_t(n, j, m, k), 1.0);
                            if (j == l) add(d2ab_t(n, i, m, k), -1.0);
                        }
                    } else if (sb == 2) {   // abb/aaa, baa/bbb
                        if (f3 && i != n && l != m)
                            add(mixed(spin ? p.d3bba : p.d3aab, i, n, j, l, m, k),
                                -(spin ? neg(i > n) * neg(l > m) : neg(i > n)));
                        if (spin == 0) {
                            if (i == l) add(d2ab_t(n, j, m, k), 1.0);
                            if (i == m) add(d2ab_t(n, j, l, k), -1.0);
                        } else {
                            if (i == l) add(d2ab_t(j, n, k, m), 1.0);
                            if (i == m) add(d2ab_t(j, n, k, l), -1.0);
                        }
                    } else {   // abb/abb, baa/baa
                        if (f3 && j != n && m != k)
                            add(mixed(spin ? p.d3aab : p.d3bba, j, n, i, m, k, l), neg(j > n) * neg(m > k));
                        if (spin == 0) {
                            if (!f3 && k == n) add(d2ab_t(i, j, l, m), 1.0);
                            if (j == m && i == l) add(d1o + (int64_t)n * N + k, 1.0);
                            if (i == l && n != j && k != m) add(d2aa_t(d2o, n, j, k, m), -sgn(n, j, k, m));
                            if (j == m) add(d2ab_t(i, n, l, k), -1.0);
                        } else {
                            if (!f3 && k == n) add(d2ab_t(j, i, m, l), 1.0);
                            if (j == m && i == l) add(d1o + (int64_t)n * N + k, 1.0);
                            if (i == l && n != j && k != m) add(d2aa_t(d2o, n, j, k, m), -sgn(n, j, k, m));
                            if (j == m) add(d2ab_t(n, i, k, l), -1.0);
                        }
                    }
                    const int64_t I = rowaab ? ijk : aab + ijk, J = colaab ? lmn : aab + lmn;
                    const int64_t e = I * big + J;
                    f(off + e, t2 + e, 2 + 4 * spin + sb, cols, coef, nt);
                }
            }
        }
        off += big * big;
    }
}
}  // namespace

void guess_random(const Problem &p, double *x) {
    if (p.spec.batch_parts) throw std::invalid_argument("a batch's guess is its parts' guesses, concatenated");
    // v2rdm_solver.cc:1799-1806 (C library rand() seeded with 0)
    srand(0);
    for (int64_t i = 0; i < p.n_primal; i++) x[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
}

void guess_hf(const Problem &p, double *x) {
    if (p.spec.batch_parts) throw std::invalid_argument("a batch's guess is its parts' guesses, concatenated");
    if (p.spec.doci)
        throw std::invalid_argument("v2RDM-DOCI starts from the random guess (v2rdm_doci_solver.cc:1325-1336)");
    // v2rdm_solver.cc:1713-1823; the reference stores doccpi = nalpha for
    // Hubbard / external problems, so both spins fill nalpha orbitals.
    const int n = p.n, gab = p.gab, gaa = p.gaa, occ = p.spec.nalpha;
    std::memset(x, 0, sizeof(double) * p.n_primal);
    for (int i = 0; i < occ; i++)
        for (int j = 0; j < occ; j++) {
            const int ij = p.iab(i, j);
            x[p.d2ab + (int64_t)ij * gab + ij] = 1.0;
        }
    for (int i = 0; i < occ; i++)
        for (int j = 0; j < i; j++) {
            const int ij = p.iaa(i, j);
            x[p.d2aa + (int64_t)ij * gaa + ij] = 1.0;
            x[p.d2bb + (int64_t)ij * gaa + ij] = 1.0;
        }
    for (int i = 0; i < occ; i++) {
        x[p.d1a + i * n + i] = 1.0;
        x[p.d1b + i * n + i] = 1.0;
    }
    for (int i = occ; i < n; i++) {
        x[p.q1a + i * n + i] = 1.0;
        x[p.q1b + i * n + i] = 1.0;
    }
    if (p.q2) {  // q2.cc:45-167
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                double dum = 0.0;
                dum += x[p.d2ab + (int64_t)kl * gab + ij];
                if (j == l) dum += x[p.q1a + i * n + k];
                if (i == k) dum -= x[p.d1b + l * n + j];
                x[p.q2ab + (int64_t)ij * gab + kl] = dum;
            }
        }
        for (int s = 0; s < 2; s++) {
            const int64_t d2 = s ? p.d2bb : p.d2aa, q2 = s ? p.q2bb : p.q2aa;
            const int64_t q1 = s ? p.q1b : p.q1a, d1 = s ? p.d1b : p.d1a;
            for (int ij = 0; ij < gaa; ij++) {
                const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                    double dum = 0.0;
                    dum += x[d2 + (int64_t)kl * gaa + ij];
                    if (j == l) dum += x[q1 + i * n + k];
                    if (j == k) dum += x[d1 + l * n + i];
                    if (i == l) dum -= x[q1 + j * n + k];
                    if (i == k) dum -= x[d1 + l * n + j];
                    x[q2 + (int64_t)ij * gaa + kl] = dum;
                }
            }
        }
    }
    if (p.g2) {  // g2.cc:44-242
        for (int s = 0; s < 2; s++) {
            const int64_t g = s ? p.g2ba : p.g2ab, d1 = s ? p.d1b : p.d1a;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    double dum = 0.0;
                    if (j == l) dum += x[d1 + i * n + k];
                    dum -= s ? x[p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(j, k)]
                             : x[p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(k, j)];
                    x[g + (int64_t)ij * gab + kl] = dum;
                }
            }
        }
        const int64_t w = 2 * (int64_t)gab;
        for (int s = 0; s < 2; s++) {
            const int64_t d1 = s ? p.d1b : p.d1a, d2 = s ? p.d2bb : p.d2aa, sh = s ? gab : 0;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    double dum = 0.0;
                    if (j == l) dum += x[d1 + i * n + k];
                    if (i != l && k != j) {
                        const int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                        dum -= x[d2 + (int64_t)p.iaa(i, l) * gaa + p.iaa(k, j)] * sil * skj;
                    }
                    x[p.g2aa + (sh + ij) * w + (sh + kl)] = dum;
                }
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                x[p.g2aa + (int64_t)ij * w + (gab + kl)] = 0.0 + x[p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(j, k)];
                x[p.g2aa + (gab + ij) * w + kl] = 0.0 + x[p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(k, j)];
            }
        }
    }
    if (p.t1) {   // t1.cc:45-419: each element from its row's terms
        t1_rows(p, 0, [&](int64_t, int64_t t1c, int, const int64_t *cols, const double *coef, int nt) {
            double dum = 0.0;
            for (int q = 0; q < nt; q++) dum += coef[q] * x[cols[q]];
            x[t1c] = dum;
        });
    }
    if (p.t2) {   // t2.cc:1845-2452: each element from its row's D terms (the aaa/abb part zero)
        t2_rows(p, 0, [&](int64_t, int64_t t2c, int sub, const int64_t *cols, const double *coef, int nt) {
            double dum = 0.0;
            for (int q = 0; q < nt; q++) dum += coef[q] * x[cols[q]];
            x[t2c] = sub == kT2AaaAbb ? 0.0 : dum;
        });
    }
}

// ------------------------------------------------------------ emitters
namespace {

const double kSqrt2 = std::sqrt(2.0);

// A (rows = dual constraints).  S::t(row, col, coef) appends a term to row's
// running sum; S::g(row, col, coef) appends to the row's second partial sum
// (rows the reference assembles as "first part + separately summed tail").
template <class S>
void visit_A(const Problem &p, S &s) {
    if (p.spec.doci) {
        doci_rows(p, [&](int64_t row, const DociTerm *t, int nt) {
            for (int q = 0; q < nt; q++) {
                if (t[q].tail) s.g(row, t[q].col, t[q].coef);
                else s.t(row, t[q].col, t[q].coef);
            }
        });
        return;
    }
    const int n = p.n, gab = p.gab, gaa = p.gaa;
    const double na = p.spec.nalpha, nb = p.spec.nbeta;
    int64_t off = 0;
    // d2.cc:316-378 traces
    if (p.spec.constrain_sz) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) { const int ij = p.iab(i, j); s.t(off, p.d2ab + (int64_t)ij * gab + ij, 1.0); }
        off++;
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d2 = sp ? p.d2bb : p.d2aa;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    if (i == j || gaa == 0) continue;
                    const int ij = p.iaa(i, j);
                    s.t(off, d2 + (int64_t)ij * gaa + ij, 1.0);
                }
            off++;
        }
    } else {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int ij = p.iab(i, j);
                s.t(off, p.d2ab + (int64_t)ij * gab + ij, 2.0);
                if (i == j || gaa == 0) continue;
                ij = p.iaa(i, j);
                s.t(off, p.d2aa + (int64_t)ij * gaa + ij, 1.0);
                s.t(off, p.d2bb + (int64_t)ij * gaa + ij, 1.0);
            }
        off++;
    }
    // d2.cc:380-414 hermiticity
    const int64_t hb[3] = {p.d2aa, p.d2bb, p.d2ab};
    const int hg[3] = {gaa, gaa, gab};
    for (int sp = 0; sp < 3; sp++)
        for (int64_t ij = 0; ij < hg[sp]; ij++)
            for (int64_t kl = 0; kl < hg[sp]; kl++) {
                s.t(off, hb[sp] + ij * hg[sp] + kl, 1.0);
                s.t(off, hb[sp] + kl * hg[sp] + ij, -1.0);
                off++;
            }
    // d2.cc:416-435 D1^T + Q1 = I
    for (int sp = 0; sp < 2; sp++) {
        const int64_t d1 = sp ? p.d1b : p.d1a, q1 = sp ? p.q1b : p.q1a;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                s.t(off + i * n + j, d1 + j * n + i, 1.0);
                s.t(off + i * n + j, q1 + i * n + j, 1.0);
            }
        off += (int64_t)n * n;
    }
    // d2.cc:441-591 partial traces
    auto contract_ab = [&](int sp, double f, int64_t d1) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const int64_t row = off + i * n + j;
                s.t(row, d1 + i * n + j, f);
                for (int k = 0; k < n; k++) {
                    const int ik = sp ? p.iab(k, i) : p.iab(i, k);
                    const int jk = sp ? p.iab(k, j) : p.iab(j, k);
                    s.t(row, p.d2ab + (int64_t)ik * gab + jk, -1.0);
                }
            }
    };
    auto contract_aa = [&](int64_t d2, bool with_ab, int sp, double f, int64_t d1) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const int64_t row = off + i * n + j;
                s.t(row, d1 + i * n + j, f);
                if (with_ab)
                    for (int k = 0; k < n; k++) {
                        const int ik = sp ? p.iab(k, i) : p.iab(i, k);
                        const int jk = sp ? p.iab(k, j) : p.iab(j, k);
                        s.t(row, p.d2ab + (int64_t)ik * gab + jk, -1.0);
                    }
                for (int k = 0; k < n; k++) {
                    if (i == k || j == k) continue;
                    const int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                    s.t(row, d2 + (int64_t)p.iaa(i, k) * gaa + p.iaa(j, k), -(double)(sik * sjk));
                }
            }
    };
    if (!p.spec.constrain_sz) {
        contract_aa(p.d2aa, true, 0, na + nb - 1.0, p.d1a); off += (int64_t)n * n;
        contract_aa(p.d2bb, true, 1, na + nb - 1.0, p.d1b); off += (int64_t)n * n;
    } else {
        contract_ab(0, nb, p.d1a); off += (int64_t)n * n;
        contract_ab(1, na, p.d1b); off += (int64_t)n * n;
        contract_aa(p.d2aa, false, 0, na - 1.0, p.d1a); off += (int64_t)n * n;
        contract_aa(p.d2bb, false, 1, nb - 1.0, p.d1b); off += (int64_t)n * n;
    }

    if (p.spec.constrain_spin) {
        // spin.cc:279-290 <S^2>
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) s.t(off, p.d2ab + (int64_t)p.iab(i, j) * gab + p.iab(j, i), 1.0);
        off++;
        if (p.spec.nalpha == p.spec.nbeta) {
            // spin.cc:320-393
            for (int64_t r = 0; r < (int64_t)n * n; r++) { s.t(off + r, p.d1a + r, 1.0); s.t(off + r, p.d1b + r, -1.0); }
            off += (int64_t)n * n;
            for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) { s.t(off + r, p.d2aa + r, 1.0); s.t(off + r, p.d2bb + r, -1.0); }
            off += (int64_t)gaa * gaa;
            for (int sp = 0; sp < 2; sp++) {
                const int64_t d2 = sp ? p.d2bb : p.d2aa;
                for (int ij = 0; ij < gaa; ij++) {
                    const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                    const int64_t ijb = p.iab(i, j), jib = p.iab(j, i);
                    for (int kl = 0; kl < gaa; kl++) {
                        const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                        const int64_t klb = p.iab(k, l), lkb = p.iab(l, k);
                        const int64_t row = off + (int64_t)ij * gaa + kl;
                        s.t(row, d2 + (int64_t)ij * gaa + kl, 1.0);
                        s.t(row, p.d2ab + ijb * gab + klb, -0.5);
                        s.t(row, p.d2ab + jib * gab + klb, 0.5);
                        s.t(row, p.d2ab + ijb * gab + lkb, 0.5);
                        s.t(row, p.d2ab + jib * gab + lkb, -0.5);
                    }
                }
                off += (int64_t)gaa * gaa;
            }
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                const int64_t ji = p.iab(j, i);
                const double dij = (i == j) ? kSqrt2 : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t lk = p.iab(l, k);
                    const double dkl = (k == l) ? kSqrt2 : 1.0;
                    const double f = -(0.5 / (dij * dkl));
                    const int64_t row = off + (int64_t)ij * gab + kl;
                    s.t(row, p.d200 + (int64_t)ij * gab + kl, 1.0);
                    s.t(row, p.d2ab + (int64_t)ij * gab + kl, f);
                    s.t(row, p.d2ab + ji * gab + kl, f);
                    s.t(row, p.d2ab + (int64_t)ij * gab + lk, f);
                    s.t(row, p.d2ab + ji * gab + lk, f);
                }
            }
            off += (int64_t)gab * gab;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                const int64_t ji = p.iab(j, i);
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t row = off + (int64_t)ij * gab + kl;
                    s.t(row, p.d2ab + (int64_t)ij * gab + kl, 1.0);
                    s.t(row, p.d2ab + ji * gab + p.iab(l, k), -1.0);
                }
            }
            off += (int64_t)gab * gab;
        } else {
            // spin.cc:411-485 (non-singlet 2gab x 2gab block)
            const int64_t w = 2 * (int64_t)gab;
            for (int q = 0; q < 4; q++) {
                const int rs = q >> 1, cs = q & 1;   // (row half, column half)
                for (int ij = 0; ij < gab; ij++) {
                    const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                    const int64_t ji = p.iab(j, i);
                    const double dij = (i == j) ? kSqrt2 : 1.0;
                    for (int kl = 0; kl < gab; kl++) {
                        const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                        const int64_t lk = p.iab(l, k);
                        const double dkl = (k == l) ? kSqrt2 : 1.0;
                        const int64_t e = (ij + rs * gab) * w + (kl + cs * gab);
                        const int64_t row = off + e;
                        const int64_t ab_ijkl = (int64_t)ij * gab + kl, ab_jikl = ji * gab + kl;
                        const int64_t ab_ijlk = (int64_t)ij * gab + lk, ab_jilk = ji * gab + lk;
                        s.t(row, p.d200 + e, 1.0);
                        if (q == 0) {
                            const double f = -(0.5 / (dij * dkl));
                            s.t(row, p.d2ab + ab_ijkl, f); s.t(row, p.d2ab + ab_jikl, f);
                            s.t(row, p.d2ab + ab_ijlk, f); s.t(row, p.d2ab + ab_jilk, f);
                        } else if (q == 1) {
                            const double f = 0.5 / dij;
                            s.t(row, p.d2ab + ab_ijkl, -f); s.t(row, p.d2ab + ab_ijlk, f);
                            s.t(row, p.d2ab + ab_jikl, -f); s.t(row, p.d2ab + ab_jilk, f);
                        } else if (q == 2) {
                            const double f = 0.5 / dkl;
                            s.t(row, p.d2ab + ab_ijkl, -f); s.t(row, p.d2ab + ab_ijlk, -f);
                            s.t(row, p.d2ab + ab_jikl, f); s.t(row, p.d2ab + ab_jilk, f);
                        } else {
                            s.t(row, p.d2ab + ab_ijkl, -0.5); s.t(row, p.d2ab + ab_jikl, 0.5);
                            s.t(row, p.d2ab + ab_ijlk, 0.5); s.t(row, p.d2ab + ab_jilk, -0.5);
                        }
                    }
                }
            }
            off += 4 * (int64_t)gab * gab;
        }
        if (p.g2) {
            // spin.cc:487-507
            for (int kl = 0; kl < gab; kl++)
                for (int i = 0; i < n; i++) s.t(off + kl, p.g2ba + (int64_t)kl * gab + p.iab(i, i), 1.0);
            off += gab;
            for (int kl = 0; kl < gab; kl++)
                for (int i = 0; i < n; i++) s.t(off + kl, p.g2ba + (int64_t)p.iab(i, i) * gab + kl, 1.0);
            off += gab;
        }
    }

    if (p.q2) {
        // q2.cc:170-216
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t row = off + (int64_t)ij * gab + kl;
                s.t(row, p.d2ab + (int64_t)ij * gab + kl, 1.0);
                s.t(row, p.q2ab + (int64_t)ij * gab + kl, -1.0);
                if (j == l) s.t(row, p.d1a + k * n + i, -1.0);
                if (i == k) s.t(row, p.d1b + l * n + j, -1.0);
            }
        }
        off += (int64_t)gab * gab;
        // q2.cc:218-318: (D2 - Q2) + (separately summed delta terms)
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d2 = sp ? p.d2bb : p.d2aa, q2 = sp ? p.q2bb : p.q2aa, d1 = sp ? p.d1b : p.d1a;
            for (int ij = 0; ij < gaa; ij++) {
                const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                    const int64_t row = off + (int64_t)ij * gaa + kl;
                    s.t(row, d2 + (int64_t)ij * gaa + kl, 1.0);
                    s.t(row, q2 + (int64_t)ij * gaa + kl, -1.0);
                    if (j == l) s.g(row, d1 + k * n + i, -1.0);
                    if (j == k) s.g(row, d1 + l * n + i, 1.0);
                    if (i == l) s.g(row, d1 + k * n + j, 1.0);
                    if (i == k) s.g(row, d1 + l * n + j, -1.0);
                }
            }
            off += (int64_t)gaa * gaa;
        }
    }

    if (p.g2) {
        // g2.cc:245-312
        for (int sp = 0; sp < 2; sp++) {
            const int64_t g = sp ? p.g2ba : p.g2ab, d1 = sp ? p.d1b : p.d1a;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t row = off + (int64_t)ij * gab + kl;
                    s.t(row, g + (int64_t)ij * gab + kl, -1.0);
                    if (j == l) s.t(row, d1 + i * n + k, 1.0);
                    const int64_t col = sp ? p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(j, k)
                                           : p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(k, j);
                    s.t(row, col, -1.0);
                }
            }
            off += (int64_t)gab * gab;
        }
        // g2.cc:313-440
        const int64_t w = 2 * (int64_t)gab;
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d1 = sp ? p.d1b : p.d1a, d2 = sp ? p.d2bb : p.d2aa, sh = sp ? gab : 0;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t e = (sh + ij) * w + (sh + kl);
                    s.t(off + e, p.g2aa + e, -1.0);
                    if (j == l) s.t(off + e, d1 + i * n + k, 1.0);
                    if (i != l && k != j) {
                        const int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                        s.t(off + e, d2 + (int64_t)p.iaa(i, l) * gaa + p.iaa(k, j), -(double)(sil * skj));
                    }
                }
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t e = (int64_t)ij * w + (gab + kl);
                s.t(off + e, p.g2aa + e, -1.0);
                s.t(off + e, p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(j, k), 1.0);
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t e = (gab + ij) * w + kl;
                s.t(off + e, p.g2aa + e, -1.0);
                s.t(off + e, p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(k, j), 1.0);
            }
        }
        off += 4 * (int64_t)gab * gab;
    }
    if (p.t1) {   // t1.cc:419-795
        t1_rows(p, off, [&](int64_t row, int64_t t1c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(row, t1c, -1.0);
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        });
        off += 2 * (int64_t)p.trip_aab * p.trip_aab + 2 * (int64_t)p.trip_aaa * p.trip_aaa;
    }
    if (p.t2) {   // t2.cc:1236-1843
        t2_rows(p, off, [&](int64_t row, int64_t t2c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(row, t2c, -1.0);
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        });
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.e3) {   // e3.cc:45-566
        e3_rows(p, off, [&](int64_t row, int64_t e3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(row, e3c, -1.0);
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        });
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.f3) {   // f3.cc:45-836
        t2_rows(p, off, [&](int64_t row, int64_t f3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(row, f3c, -1.0);
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        }, true);
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.q3) {   // q3.cc:45-423
        t1_rows(p, off, [&](int64_t row, int64_t q3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(row, q3c, -1.0);
            s.t(row, d3_twin(p, q3c), -1.0);
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        }, true);
        off += 2 * (int64_t)p.trip_aab * p.trip_aab + 2 * (int64_t)p.trip_aaa * p.trip_aaa;
    }
    if (p.d3) {   // d3.cc:45-406
        d3_rows(p, off, [&](int64_t row, const int64_t *cols, const double *coef, int nt) {
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
            off++;
        });
    }
    if (p.d4) {   // d4.cc:44-297, then the empty rows of the reference's double count
        off += d4_rows(p, off, [&](int64_t row, const int64_t *cols, const double *coef, int nt) {
            for (int q = 0; q < nt; q++) s.t(row, cols[q], coef[q]);
        });
        if (p.spec.nalpha > 1 && p.spec.nbeta > 1) off += 2 * (int64_t)p.trip_aab * p.trip_aab;
    }
    if (off != p.n_dual) throw std::logic_error("A emitter row count mismatch");
}

// A^T (rows = primal elements).  S::t(primal, dual_row, coef) appends one
// contribution in the order hilbert's bpsdp_ATu scatters it.
template <class S>
void visit_AT(const Problem &p, S &s) {
    if (p.spec.doci) {   // bpsdp_ATu scatters the rows in bpsdp_Au's order
        doci_rows(p, [&](int64_t row, const DociTerm *t, int nt) {
            for (int q = 0; q < nt; q++) s.t(t[q].col, row, t[q].coef);
        });
        return;
    }
    const int n = p.n, gab = p.gab, gaa = p.gaa;
    const double na = p.spec.nalpha, nb = p.spec.nbeta;
    int64_t off = 0;
    // d2.cc:48-100
    if (p.spec.constrain_sz) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) { const int ij = p.iab(i, j); s.t(p.d2ab + (int64_t)ij * gab + ij, off, 1.0); }
        off++;
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d2 = sp ? p.d2bb : p.d2aa;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    if (i == j || gaa == 0) continue;
                    const int ij = p.iaa(i, j);
                    s.t(d2 + (int64_t)ij * gaa + ij, off, 1.0);
                }
            off++;
        }
    } else {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int ij = p.iab(i, j);
                s.t(p.d2ab + (int64_t)ij * gab + ij, off, 2.0);
                if (i == j || gaa == 0) continue;
                ij = p.iaa(i, j);
                s.t(p.d2aa + (int64_t)ij * gaa + ij, off, 1.0);
                s.t(p.d2bb + (int64_t)ij * gaa + ij, off, 1.0);
            }
        off++;
    }
    // d2.cc:102-134
    const int64_t hb[3] = {p.d2aa, p.d2bb, p.d2ab};
    const int hg[3] = {gaa, gaa, gab};
    for (int sp = 0; sp < 3; sp++)
        for (int64_t ij = 0; ij < hg[sp]; ij++)
            for (int64_t kl = 0; kl < hg[sp]; kl++) {
                s.t(hb[sp] + ij * hg[sp] + kl, off, 1.0);
                s.t(hb[sp] + kl * hg[sp] + ij, off, -1.0);
                off++;
            }
    // d2.cc:136-158
    for (int sp = 0; sp < 2; sp++) {
        const int64_t d1 = sp ? p.d1b : p.d1a, q1 = sp ? p.q1b : p.q1a;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                s.t(d1 + j * n + i, off + i * n + j, 1.0);
                s.t(q1 + i * n + j, off + i * n + j, 1.0);
            }
        off += (int64_t)n * n;
    }
    // d2.cc:160-309
    auto contract = [&](int sp, double f, int64_t d1, bool with_ab, bool with_aa, int64_t d2) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const int64_t row = off + i * n + j;
                s.t(d1 + i * n + j, row, f);
                if (with_ab)
                    for (int k = 0; k < n; k++) {
                        const int ik = sp ? p.iab(k, i) : p.iab(i, k);
                        const int jk = sp ? p.iab(k, j) : p.iab(j, k);
                        s.t(p.d2ab + (int64_t)ik * gab + jk, row, -1.0);
                    }
                if (with_aa)
                    for (int k = 0; k < n; k++) {
                        if (i == k || j == k) continue;
                        const int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                        s.t(d2 + (int64_t)p.iaa(i, k) * gaa + p.iaa(j, k), row, -(double)(sik * sjk));
                    }
            }
        off += (int64_t)n * n;
    };
    if (!p.spec.constrain_sz) {
        contract(0, na + nb - 1.0, p.d1a, true, true, p.d2aa);
        contract(1, na + nb - 1.0, p.d1b, true, true, p.d2bb);
    } else {
        contract(0, nb, p.d1a, true, false, p.d2aa);
        contract(1, na, p.d1b, true, false, p.d2bb);
        contract(0, na - 1.0, p.d1a, false, true, p.d2aa);
        contract(1, nb - 1.0, p.d1b, false, true, p.d2bb);
    }

    if (p.spec.constrain_spin) {
        // spin.cc:48-60
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) s.t(p.d2ab + (int64_t)p.iab(i, j) * gab + p.iab(j, i), off, 1.0);
        off++;
        if (p.spec.nalpha == p.spec.nbeta) {
            // spin.cc:88-170
            for (int64_t r = 0; r < (int64_t)n * n; r++) s.t(p.d1a + r, off + r, 1.0);
            for (int64_t r = 0; r < (int64_t)n * n; r++) s.t(p.d1b + r, off + r, -1.0);
            off += (int64_t)n * n;
            for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) s.t(p.d2aa + r, off + r, 1.0);
            for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) s.t(p.d2bb + r, off + r, -1.0);
            off += (int64_t)gaa * gaa;
            for (int sp = 0; sp < 2; sp++) {
                const int64_t d2 = sp ? p.d2bb : p.d2aa;
                for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) s.t(d2 + r, off + r, 1.0);
                for (int ij = 0; ij < gaa; ij++) {
                    const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                    const int64_t ijb = p.iab(i, j), jib = p.iab(j, i);
                    for (int kl = 0; kl < gaa; kl++) {
                        const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                        const int64_t klb = p.iab(k, l), lkb = p.iab(l, k);
                        const int64_t row = off + (int64_t)ij * gaa + kl;
                        s.t(p.d2ab + ijb * gab + klb, row, -0.5);
                        s.t(p.d2ab + jib * gab + klb, row, 0.5);
                        s.t(p.d2ab + ijb * gab + lkb, row, 0.5);
                        s.t(p.d2ab + jib * gab + lkb, row, -0.5);
                    }
                }
                off += (int64_t)gaa * gaa;
            }
            for (int64_t r = 0; r < (int64_t)gab * gab; r++) s.t(p.d200 + r, off + r, 1.0);
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                const int64_t ji = p.iab(j, i);
                const double dij = (i == j) ? kSqrt2 : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t lk = p.iab(l, k);
                    const double dkl = (k == l) ? kSqrt2 : 1.0;
                    const double f = -(0.5 / (dij * dkl));
                    const int64_t row = off + (int64_t)ij * gab + kl;
                    s.t(p.d2ab + (int64_t)ij * gab + kl, row, f);
                    s.t(p.d2ab + ji * gab + kl, row, f);
                    s.t(p.d2ab + (int64_t)ij * gab + lk, row, f);
                    s.t(p.d2ab + ji * gab + lk, row, f);
                }
            }
            off += (int64_t)gab * gab;
            for (int64_t r = 0; r < (int64_t)gab * gab; r++) s.t(p.d2ab + r, off + r, 1.0);
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                const int64_t ji = p.iab(j, i);
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    s.t(p.d2ab + ji * gab + p.iab(l, k), off + (int64_t)ij * gab + kl, -1.0);
                }
            }
            off += (int64_t)gab * gab;
        } else {
            // spin.cc:171-251
            const int64_t w = 2 * (int64_t)gab;
            for (int q = 0; q < 4; q++) {
                const int rs = q >> 1, cs = q & 1;
                for (int ij = 0; ij < gab; ij++) {
                    const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                    const int64_t ji = p.iab(j, i);
                    const double dij = (i == j) ? kSqrt2 : 1.0;
                    for (int kl = 0; kl < gab; kl++) {
                        const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                        const int64_t lk = p.iab(l, k);
                        const double dkl = (k == l) ? kSqrt2 : 1.0;
                        const int64_t e = (ij + rs * gab) * w + (kl + cs * gab);
                        const int64_t row = off + e;
                        const int64_t ab_ijkl = (int64_t)ij * gab + kl, ab_jikl = ji * gab + kl;
                        const int64_t ab_ijlk = (int64_t)ij * gab + lk, ab_jilk = ji * gab + lk;
                        s.t(p.d200 + e, row, 1.0);
                        if (q == 0) {
                            const double f = -(0.5 / (dij * dkl));
                            s.t(p.d2ab + ab_ijkl, row, f); s.t(p.d2ab + ab_jikl, row, f);
                            s.t(p.d2ab + ab_ijlk, row, f); s.t(p.d2ab + ab_jilk, row, f);
                        } else if (q == 1) {
                            const double f = 0.5 / dij;
                            s.t(p.d2ab + ab_ijkl, row, -f); s.t(p.d2ab + ab_ijlk, row, f);
                            s.t(p.d2ab + ab_jikl, row, -f); s.t(p.d2ab + ab_jilk, row, f);
                        } else if (q == 2) {
                            const double f = 0.5 / dkl;
                            s.t(p.d2ab + ab_ijkl, row, -f); s.t(p.d2ab + ab_ijlk, row, -f);
                            s.t(p.d2ab + ab_jikl, row, f); s.t(p.d2ab + ab_jilk, row, f);
                        } else {
                            s.t(p.d2ab + ab_ijkl, row, -0.5); s.t(p.d2ab + ab_jikl, row, 0.5);
                            s.t(p.d2ab + ab_ijlk, row, 0.5); s.t(p.d2ab + ab_jilk, row, -0.5);
                        }
                    }
                }
            }
            off += 4 * (int64_t)gab * gab;
        }
        if (p.g2) {
            // spin.cc:253-271
            for (int kl = 0; kl < gab; kl++)
                for (int i = 0; i < n; i++) s.t(p.g2ba + (int64_t)kl * gab + p.iab(i, i), off + kl, 1.0);
            off += gab;
            for (int kl = 0; kl < gab; kl++)
                for (int i = 0; i < n; i++) s.t(p.g2ba + (int64_t)p.iab(i, i) * gab + kl, off + kl, 1.0);
            off += gab;
        }
    }

    if (p.q2) {
        // q2.cc:320-354
        for (int64_t r = 0; r < (int64_t)gab * gab; r++) s.t(p.d2ab + r, off + r, 1.0);
        for (int64_t r = 0; r < (int64_t)gab * gab; r++) s.t(p.q2ab + r, off + r, -1.0);
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t row = off + (int64_t)ij * gab + kl;
                if (j == l) s.t(p.d1a + k * n + i, row, -1.0);
                if (i == k) s.t(p.d1b + l * n + j, row, -1.0);
            }
        }
        off += (int64_t)gab * gab;
        // q2.cc:356-436
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d2 = sp ? p.d2bb : p.d2aa, q2 = sp ? p.q2bb : p.q2aa, d1 = sp ? p.d1b : p.d1a;
            for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) s.t(d2 + r, off + r, 1.0);
            for (int64_t r = 0; r < (int64_t)gaa * gaa; r++) s.t(q2 + r, off + r, -1.0);
            for (int ij = 0; ij < gaa; ij++) {
                const int i = p.bas_aa[2 * ij], j = p.bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    const int k = p.bas_aa[2 * kl], l = p.bas_aa[2 * kl + 1];
                    const int64_t row = off + (int64_t)ij * gaa + kl;
                    if (j == l) s.t(d1 + k * n + i, row, -1.0);
                    if (j == k) s.t(d1 + l * n + i, row, 1.0);
                    if (i == l) s.t(d1 + k * n + j, row, 1.0);
                    if (i == k) s.t(d1 + l * n + j, row, -1.0);
                }
            }
            off += (int64_t)gaa * gaa;
        }
    }

    if (p.g2) {
        // g2.cc:445-510
        for (int sp = 0; sp < 2; sp++) {
            const int64_t g = sp ? p.g2ba : p.g2ab, d1 = sp ? p.d1b : p.d1a;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t row = off + (int64_t)ij * gab + kl;
                    s.t(g + (int64_t)ij * gab + kl, row, -1.0);
                    if (j == l) s.t(d1 + i * n + k, row, 1.0);
                    const int64_t col = sp ? p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(j, k)
                                           : p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(k, j);
                    s.t(col, row, -1.0);
                }
            }
            off += (int64_t)gab * gab;
        }
        // g2.cc:511-631
        const int64_t w = 2 * (int64_t)gab;
        for (int sp = 0; sp < 2; sp++) {
            const int64_t d1 = sp ? p.d1b : p.d1a, d2 = sp ? p.d2bb : p.d2aa, sh = sp ? gab : 0;
            for (int ij = 0; ij < gab; ij++) {
                const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                    const int64_t e = (sh + ij) * w + (sh + kl);
                    s.t(p.g2aa + e, off + e, -1.0);
                    if (j == l) s.t(d1 + i * n + k, off + e, 1.0);
                    if (i != l && k != j) {
                        const int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                        s.t(d2 + (int64_t)p.iaa(i, l) * gaa + p.iaa(k, j), off + e, -(double)(sil * skj));
                    }
                }
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t e = (int64_t)ij * w + (gab + kl);
                s.t(p.g2aa + e, off + e, -1.0);
                s.t(p.d2ab + (int64_t)p.iab(i, l) * gab + p.iab(j, k), off + e, 1.0);
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            const int i = p.bas_ab[2 * ij], j = p.bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p.bas_ab[2 * kl], l = p.bas_ab[2 * kl + 1];
                const int64_t e = (gab + ij) * w + kl;
                s.t(p.g2aa + e, off + e, -1.0);
                s.t(p.d2ab + (int64_t)p.iab(l, i) * gab + p.iab(k, j), off + e, 1.0);
            }
        }
        off += 4 * (int64_t)gab * gab;
    }
    if (p.t1) {   // t1.cc:795-1200 scatters in the same loop order as the A rows
        t1_rows(p, off, [&](int64_t row, int64_t t1c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(t1c, row, -1.0);
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        });
        off += 2 * (int64_t)p.trip_aab * p.trip_aab + 2 * (int64_t)p.trip_aaa * p.trip_aaa;
    }
    if (p.t2) {   // t2.cc:3376-3966 scatters in the same loop order as the A rows
        t2_rows(p, off, [&](int64_t row, int64_t t2c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(t2c, row, -1.0);
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        });
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.e3) {   // e3.cc:570-1082 scatters in the same order as the A rows
        e3_rows(p, off, [&](int64_t row, int64_t e3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(e3c, row, -1.0);
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        });
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.f3) {   // f3.cc:842-1623 scatters in the same order as the A rows
        t2_rows(p, off, [&](int64_t row, int64_t f3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(f3c, row, -1.0);
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        }, true);
        const int64_t aab = p.trip_aab, big = (int64_t)p.trip_aab + p.trip_aba;
        off += 2 * aab * aab + 2 * big * big;
    }
    if (p.q3) {   // q3.cc:425-803 scatters in the same order as the A rows
        t1_rows(p, off, [&](int64_t row, int64_t q3c, int, const int64_t *cols, const double *coef, int nt) {
            s.t(q3c, row, -1.0);
            s.t(d3_twin(p, q3c), row, -1.0);
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        }, true);
        off += 2 * (int64_t)p.trip_aab * p.trip_aab + 2 * (int64_t)p.trip_aaa * p.trip_aaa;
    }
    if (p.d3) {   // d3.cc:408-766 scatters in the same order as the A rows
        d3_rows(p, off, [&](int64_t row, const int64_t *cols, const double *coef, int nt) {
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
            off++;
        });
    }
    if (p.d4) {   // d4.cc:300-557 scatters in the same order as the A rows
        off += d4_rows(p, off, [&](int64_t row, const int64_t *cols, const double *coef, int nt) {
            for (int q = 0; q < nt; q++) s.t(cols[q], row, coef[q]);
        });
        if (p.spec.nalpha > 1 && p.spec.nbeta > 1) off += 2 * (int64_t)p.trip_aab * p.trip_aab;
    }
    if (off != p.n_dual) throw std::logic_error("A^T emitter row count mismatch");
}

struct Palette {
    std::vector<double> v;
    uint32_t code(double c) {
        for (size_t i = 0; i < v.size(); i++)
            if (std::memcmp(&v[i], &c, sizeof(double)) == 0) return (uint32_t)i;
        if (v.size() >= 16) throw std::logic_error("more than 16 distinct coefficients");
        v.push_back(c);
        return (uint32_t)(v.size() - 1);
    }
};

struct CountSink {
    std::vector<uint64_t> &cnt;
    Palette &pal;
    void t(int64_t row, int64_t, double c) { cnt[row]++; pal.code(c); }
    void g(int64_t row, int64_t, double c) { cnt[row]++; pal.code(c); }
};

struct FillSink {
    std::vector<uint64_t> &cursor;
    std::vector<uint32_t> &ent;
    Palette &pal;
    void t(int64_t row, int64_t col, double c) {
        ent[cursor[row]++] = (uint32_t)col | (pal.code(c) << kColBits);
    }
    void g(int64_t row, int64_t col, double c) {
        ent[cursor[row]++] = (uint32_t)col | (pal.code(c) << kColBits) | kGroupFlag;
    }
};

template <bool Transposed>
PackedOperator build_op(const Problem &p) {
    PackedOperator op;
    op.nrows = Transposed ? p.n_primal : p.n_dual;
    op.ncols = Transposed ? p.n_dual : p.n_primal;
    std::vector<uint64_t> cnt(op.nrows + 1, 0);
    Palette pal;
    CountSink cs{cnt, pal};
    if (Transposed) visit_AT(p, cs); else visit_A(p, cs);
    std::vector<uint64_t> cursor(op.nrows + 1, 0);
    uint64_t nnz = 0;
    for (int64_t r = 0; r < op.nrows; r++) { cursor[r] = nnz; nnz += cnt[r]; }
    if (nnz >= (1ull << 32)) throw std::invalid_argument("operator has more than 2^32 entries");
    op.row_ptr.resize(op.nrows + 1);
    for (int64_t r = 0; r < op.nrows; r++) op.row_ptr[r] = (uint32_t)cursor[r];
    op.row_ptr[op.nrows] = (uint32_t)nnz;
    op.entries.resize(nnz);
    FillSink fs{cursor, op.entries, pal};
    if (Transposed) visit_AT(p, fs); else visit_A(p, fs);
    op.palette = pal.v;
    return op;
}

}  // namespace

PackedOperator build_A(const Problem &p) { return build_op<false>(p); }
PackedOperator build_AT(const Problem &p) { return build_op<true>(p); }

}  // namespace v2b
