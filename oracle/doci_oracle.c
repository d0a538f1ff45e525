/*
 * ORACLE -- test infrastructure only; the product never links it.
 *
 * C restatement of hilbert's v2RDM-DOCI program (src/v2rdm_doci): primal
 * layout, constraint count, b, c, the random guess, A.x and A^T.y, with the
 * reference's own accumulation order and roundings (compiled without FMA
 * contraction).  Pinned bit for bit against the reference's compiled DOCI
 * code (oracle/build_ref.sh -> _ref/libdoci_ref.so) by tests/test_doci.py.
 *
 *   layout, counts, blocks   v2rdm_doci_solver.cc:427-700 (common_init)
 *   b                        v2rdm_doci_solver.cc:1338-1507 (BuildConstraints)
 *   guess                    v2rdm_doci_solver.cc:1325-1336
 *   c                        tei.cc:127-153 (RepackIntegrals)
 *   A.x / A^T.y              v2rdm_doci_solver.cc:1509-1566 calling
 *                            d2.cc, q2.cc, g2.cc, d3.cc, t1.cc, t2.cc
 */
#include <stdlib.h>
#include <string.h>

typedef struct {
    int n, na, nb;
    int q2, g2, t1, t2, d3;
    long d2s2, d2s0, d1, q2s2, q2s0, g2s2, g2s0, d3s3, d3s1, t1aaa, t1aab, t1s1, t2s1, t2blk;
    long n_primal, n_dual;
    int nblocks;
    int *dims;
} doci_t;

/* ---- one row at a time: AU sums terms into the row, ATU scatters them ---- */
enum { AU = 0, ATU = 1 };
typedef struct {
    int mode;
    const double *in;
    double *out;
    long row;         /* current dual row */
    double acc, tail; /* AU partial sums */
    int has_tail;
} visit_t;

static void begin(visit_t *v, long row) { v->row = row; v->acc = 0.0; v->tail = 0.0; v->has_tail = 0; }
static void term(visit_t *v, long col, double coef) {
    if (v->mode == AU) v->acc += coef * v->in[col];
    else v->out[col] += coef * v->in[v->row];
}
static void tail_term(visit_t *v, long col, double coef) {
    if (v->mode == AU) { v->tail += coef * v->in[col]; v->has_tail = 1; }
    else v->out[col] += coef * v->in[v->row];
}
static void end(visit_t *v) {
    if (v->mode == AU) v->out[v->row] = v->has_tail ? v->acc + v->tail : v->acc;
}
static int without(int a, int b) { return a > b ? a - 1 : a; }

/* the seniority-3 D3 row (d3.cc:131-145): the D3 sum is scaled by 1/6 as a
   whole before the D2 term; its A^T side (d3.cc:37-54) is term by term */
static void d3s3_row(visit_t *v, const doci_t *p, int a, int b) {
    const int n = p->n;
    double sum = 0.0;
    for (int c = 0; c < n; c++) {
        if (c == a || c == b) continue;
        long idx[6] = {((long)c * n + a) * n + b, ((long)c * n + b) * n + a, ((long)a * n + c) * n + b,
                       ((long)b * n + c) * n + a, ((long)a * n + b) * n + c, ((long)b * n + a) * n + c};
        for (int q = 0; q < 6; q++) {
            if (v->mode == AU) sum += v->in[p->d3s3 + idx[q]];
            else v->out[p->d3s3 + idx[q]] += 1.0 / 6.0 * v->in[v->row];
        }
    }
    const double x = 0.5 * (p->na + p->nb) - 2.0;
    if (v->mode == AU) v->out[v->row] = 1.0 / 6.0 * sum - x * v->in[p->d2s2 + (long)a * n + b];
    else v->out[p->d2s2 + (long)a * n + b] -= x * v->in[v->row];
}

static void visit(const doci_t *p, visit_t *v) {
    const int n = p->n;
    const long nm = n - 1, nm2 = nm * nm, w = 2L * n - 1, bs = w * w;
    long row = 0;
#define ROW(r) begin(v, (r))
#define T(col, coef) term(v, (col), (coef))
#define S(blk, a, b, coef) (T((blk) + (long)(a) * n + (b), coef), T((blk) + (long)(b) * n + (a), coef))
    /* d2.cc: Tr D2s2, Tr D2s0, Tr D1 */
    ROW(row++); for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) if (i != j) T(p->d2s2 + (long)i * n + j, 1.0); end(v);
    ROW(row++); for (int i = 0; i < n; i++) T(p->d2s0 + (long)i * n + i, 1.0); end(v);
    ROW(row++); for (int i = 0; i < n; i++) T(p->d1 + i, 1.0); end(v);
    /* D2s2 -> D1, over the first index, then the second */
    for (int second = 0; second < 2; second++)
        for (int i = 0; i < n; i++) {
            ROW(row++);
            T(p->d1 + i, p->na - 1.0);
            for (int j = 0; j < n; j++)
                if (j != i) T(p->d2s2 + (second ? (long)j * n + i : (long)i * n + j), -1.0);
            end(v);
        }
    /* D2s0 -> D1 */
    for (int i = 0; i < n; i++) { ROW(row++); T(p->d1 + i, 1.0); T(p->d2s0 + (long)i * n + i, -1.0); end(v); }
    /* D2s2 antisymmetric part vanishes, diagonal vanishes */
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            ROW(row++);
            T(p->d2s2 + (long)i * n + j, 1.0);
            if (i != j) T(p->d2s2 + (long)j * n + i, -1.0);
            end(v);
        }
    if (p->q2) {   /* q2.cc */
        long ij = 0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++, ij++) {
                ROW(row++);
                S(p->d2s2, i, j, 0.5);
                T(p->q2s2 + ij, -1.0);
                T(p->d1 + i, -1.0);
                T(p->d1 + j, -1.0);
                end(v);
            }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                ROW(row++);
                T(p->d2s0 + (long)i * n + j, 1.0);
                T(p->q2s0 + (long)i * n + j, -1.0);
                if (i == j) { tail_term(v, p->d1 + i, -1.0); tail_term(v, p->d1 + i, -1.0); }
                end(v);
            }
    }
    if (p->g2) {   /* g2.cc */
        long aux = 0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++, aux += 4) {
                ROW(row++); T(p->g2s2 + aux, -1.0); T(p->d1 + i, 1.0); S(p->d2s2, i, j, -0.5); end(v);
                ROW(row++); T(p->g2s2 + aux + 1, -1.0); S(p->d2s0, i, j, 0.5); end(v);
                ROW(row++); T(p->g2s2 + aux + 2, -1.0); S(p->d2s0, i, j, 0.5); end(v);
                ROW(row++); T(p->g2s2 + aux + 3, -1.0); T(p->d1 + j, 1.0); S(p->d2s2, i, j, -0.5); end(v);
            }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                ROW(row++);
                T(p->g2s0 + (long)i * n + j, -1.0);
                if (i != j) S(p->d2s2, i, j, 0.5);
                else T(p->d1 + i, 1.0);
                end(v);
            }
    }
    if (p->d3) {   /* d3.cc */
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++)
                if (a != b) { ROW(row++); d3s3_row(v, p, a, b); }
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) {
                if (a == b) continue;
                const int myb = without(b, a);
                ROW(row++); T(p->d3s1 + a * nm2 + myb * nm + myb, 1.0); S(p->d2s2, a, b, -0.5); end(v);
            }
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) {
                if (a == b) continue;
                const int mya = without(a, b);
                ROW(row++); T(p->d3s1 + b * nm2 + mya * nm + mya, 1.0); S(p->d2s2, a, b, -0.5); end(v);
            }
        const double y = 0.5 * (0.5 * (p->na + p->nb) - 1.0);
        for (int a = 0; a < n; a++)
            for (int c = 0; c < n; c++) {
                ROW(row++);
                for (int b = 0; b < n; b++) {
                    if (b == a || b == c) continue;
                    const int mya = without(a, b), myc = without(c, b);
                    T(p->d3s1 + b * nm2 + mya * nm + myc, 0.5);
                    T(p->d3s1 + b * nm2 + myc * nm + mya, 0.5);
                }
                S(p->d2s0, a, c, -y);
                end(v);
            }
    }
    if (p->t1) {   /* t1.cc */
        long abc = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                for (int c = b + 1; c < n; c++, abc++) {
                    ROW(row++);
                    T(p->t1aaa + abc, 1.0);
                    T(p->d1 + a, 1.0); T(p->d1 + b, 1.0); T(p->d1 + c, 1.0);
                    S(p->d2s2, a, b, -0.5); S(p->d2s2, b, c, -0.5); S(p->d2s2, a, c, -0.5);
                    end(v);
                }
        abc = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                for (int c = 0; c < n; c++, abc++) {
                    ROW(row++);
                    T(p->t1aab + abc, 1.0);
                    T(p->d1 + a, 1.0); T(p->d1 + b, 1.0); T(p->d1 + c, 1.0);
                    S(p->d2s2, a, b, -0.5);
                    S(b != c ? p->d2s2 : p->d2s0, b, c, -0.5);
                    S(a != c ? p->d2s2 : p->d2s0, a, c, -0.5);
                    end(v);
                }
        for (int b = 0; b < n; b++)
            for (int a = 0; a < n; a++) {
                if (a == b) continue;
                for (int c = 0; c < n; c++) {
                    if (c == b) continue;
                    ROW(row++);
                    T(p->t1s1 + b * nm2 + without(a, b) * nm + without(c, b), 1.0);
                    if (a == c) { T(p->d1 + a, 2.0); T(p->d1 + b, 1.0); S(p->d2s2, a, b, -1.0); }
                    S(p->d2s0, a, c, -0.5);
                    end(v);
                }
            }
    }
    if (p->t2) {   /* t2.cc: the (2n-1)^2 block of orbital i, rows at base + (r, c) */
        for (int i = 0; i < n; i++) {
            const long base = row + i * bs, t = p->t2s1 + i * bs, last = 2L * n - 2;
#define R2(r, c) ROW(base + (r) * w + (c)); T(t + (r) * w + (c), -1.0)
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    R2(without(k, i), without(j, i));
                    if (j == k) T(p->d1 + j, 1.0); else S(p->d2s2, j, k, 0.5);
                    end(v);
                }
            }
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    R2(without(k, i), without(j, i) + n - 1);
                    if (j == k) S(p->d2s0, i, k, -0.5);
                    end(v);
                }
            }
            for (int k = 0; k < n; k++) {
                if (k == i) continue;
                R2(without(k, i), last); S(p->d2s2, i, k, 0.5); end(v);
            }
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    R2(without(k, i) + n - 1, without(j, i));
                    if (j == k) S(p->d2s0, i, k, -0.5);
                    end(v);
                }
            }
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                for (int k = 0; k < n; k++) {
                    if (k == i) continue;
                    R2(without(k, i) + n - 1, without(j, i) + n - 1);
                    if (j == k) { T(p->d1 + i, 1.0); S(p->d2s2, i, k, -1.0); }
                    S(p->d2s0, j, k, 0.5);
                    end(v);
                }
            }
            for (int k = 0; k < n; k++) {
                if (k == i) continue;
                R2(without(k, i) + n - 1, last); S(p->d2s0, i, k, 0.5); end(v);
            }
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                R2(last, without(j, i)); S(p->d2s2, j, i, 0.5); end(v);
            }
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                R2(last, without(j, i) + n - 1); S(p->d2s0, j, i, 0.5); end(v);
            }
            R2(last, last); T(p->d1 + i, 1.0); end(v);
#undef R2
        }
        row += n * bs;
        long aux = p->t2blk;
        for (int i = 0; i < n; i++)
            for (int k = i + 1; k < n; k++)
                for (int m = k + 1; m < n; m++, aux += 9) {
                    ROW(row++); T(aux, -1.0); S(p->d2s2, i, k, 0.5); S(p->d2s2, i, m, -0.5);
                    S(p->d2s2, k, m, -0.5); T(p->d1 + m, 1.0); end(v);
                    ROW(row++); T(aux + 1, -1.0); S(p->d2s0, m, k, 0.5); end(v);
                    ROW(row++); T(aux + 2, -1.0); S(p->d2s0, m, i, 0.5); end(v);
                    ROW(row++); T(aux + 3, -1.0); S(p->d2s0, k, m, 0.5); end(v);
                    ROW(row++); T(aux + 4, -1.0); S(p->d2s2, i, k, -0.5); S(p->d2s2, i, m, 0.5);
                    S(p->d2s2, m, k, -0.5); T(p->d1 + k, 1.0); end(v);
                    ROW(row++); T(aux + 5, -1.0); S(p->d2s0, k, i, 0.5); end(v);
                    ROW(row++); T(aux + 6, -1.0); S(p->d2s0, i, m, 0.5); end(v);
                    ROW(row++); T(aux + 7, -1.0); S(p->d2s0, i, k, 0.5); end(v);
                    ROW(row++); T(aux + 8, -1.0); S(p->d2s2, i, k, -0.5); S(p->d2s2, i, m, -0.5);
                    S(p->d2s2, k, m, 0.5); T(p->d1 + i, 1.0); end(v);
                }
    }
#undef ROW
#undef T
#undef S
    if (row != p->n_dual) abort();   /* layout and rows disagree: a bug in this file */
}

/* ---------------------------------------------------------------- interface */
/* positivity: 0 D, 1 DQ, 2 DG, 3 DQG, 4 DQGT2 (D, Q, G, T2), 5 DQGT1, 6 DQGT1T2 */
void *dco_create(int n, int na, int nb, int positivity, int d3) {
    if (n < 1 || na < 0 || nb < 0 || na > n || nb > n || positivity < 0 || positivity > 6) return NULL;
    if ((d3 || positivity == 5 || positivity == 6) && n < 2) return NULL;
    doci_t *p = calloc(1, sizeof(doci_t));
    p->n = n; p->na = na; p->nb = nb;
    p->q2 = positivity == 1 || positivity >= 3;
    p->g2 = positivity == 2 || positivity >= 3;
    p->t1 = positivity == 5 || positivity == 6;
    p->t2 = positivity == 4 || positivity == 6;
    p->d3 = d3 != 0;
    const long ln = n, pairs = ln * (ln - 1) / 2, trip = ln * (ln - 1) * (ln - 2) / 6, w = 2 * ln - 1;
    long cap = ln * ln + 1 + ln + pairs + 1 + pairs + 1 + ln * ln * ln + ln + trip + ln * pairs + ln + ln + trip;
    p->dims = malloc(sizeof(int) * (size_t)cap);
    long off = 0;
    int nb_ = 0;
#define BLOCKS(field, count, dim) do { p->field = off; for (long k_ = 0; k_ < (count); k_++) { \
        p->dims[nb_++] = (int)(dim); off += (long)(dim) * (dim); } } while (0)
    BLOCKS(d2s2, ln * ln, 1);
    BLOCKS(d2s0, 1, ln);
    BLOCKS(d1, ln, 1);
    if (p->q2) { BLOCKS(q2s2, pairs, 1); BLOCKS(q2s0, 1, ln); }
    if (p->g2) { BLOCKS(g2s2, pairs, 2); BLOCKS(g2s0, 1, ln); }
    if (p->d3) { BLOCKS(d3s3, ln * ln * ln, 1); BLOCKS(d3s1, ln, ln - 1); }
    if (p->t1) { BLOCKS(t1aaa, trip, 1); BLOCKS(t1aab, ln * pairs, 1); BLOCKS(t1s1, ln, ln - 1); }
    if (p->t2) { BLOCKS(t2s1, ln, w); BLOCKS(t2blk, trip, 3); }
#undef BLOCKS
    p->nblocks = nb_;
    p->n_primal = off;
    long d = 3 + 3 * ln + ln * ln;
    if (p->q2) d += pairs + ln * ln;
    if (p->g2) d += 4 * pairs + ln * ln;
    if (p->d3) d += 3 * ln * (ln - 1) + ln * ln;
    if (p->t1) d += trip + ln * pairs + ln * (ln - 1) * (ln - 1);
    if (p->t2) d += ln * w * w + 9 * trip;
    p->n_dual = d;
    return p;
}
void dco_destroy(void *h) {
    doci_t *p = h;
    if (p) free(p->dims);
    free(p);
}
long dco_n_primal(void *h) { return ((doci_t *)h)->n_primal; }
long dco_n_dual(void *h) { return ((doci_t *)h)->n_dual; }
int dco_n_blocks(void *h) { return ((doci_t *)h)->nblocks; }
void dco_block_dims(void *h, int *out) { memcpy(out, ((doci_t *)h)->dims, sizeof(int) * ((doci_t *)h)->nblocks); }

void dco_build_b(void *h, double *b) {
    const doci_t *p = h;
    const int n = p->n;
    memset(b, 0, sizeof(double) * p->n_dual);
    b[0] = p->na * (p->na - 1.0);
    b[1] = p->na;
    b[2] = p->na;
    long off = 3 + 3L * n + (long)n * n;
    if (p->q2) {
        for (long k = 0; k < (long)n * (n - 1) / 2; k++) b[off++] = -1.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) b[off++] = i == j ? -1.0 : -0.0;
    }
    if (p->g2) off += 2L * n * (n - 1) + (long)n * n;
    if (p->d3) off += 3L * n * (n - 1) + (long)n * n;
    if (p->t1) {
        long ones = (long)n * (n - 1) * (n - 2) / 6 + (long)n * n * (n - 1) / 2;
        while (ones--) b[off++] = 1.0;
        for (int bb = 0; bb < n; bb++)
            for (int a = 0; a < n; a++)
                for (int c = 0; c < n; c++)
                    if (a != bb && c != bb) b[off++] = a == c ? 1.0 : 0.0;
    }
}

/* h[i*n+j], g[((i*n+j)*n+k)*n+l] = (ij|kl) */
void dco_build_c(void *hp, const double *h, const double *g, double *c) {
    const doci_t *p = hp;
    const long n = p->n;
    memset(c, 0, sizeof(double) * p->n_primal);
    const double f = 2.0 / (p->na + p->nb - 1.0);
    for (long i = 0; i < n; i++)
        for (long j = 0; j < n; j++) {
            const double coulomb = g[((i * n + i) * n + j) * n + j], exchange = g[((i * n + j) * n + i) * n + j];
            if (i != j) {
                double v = 2.0 * coulomb;
                v -= exchange;
                v += f * (h[i * n + i] + h[j * n + j]);
                c[p->d2s2 + i * n + j] = v;
            }
            double s = exchange;
            s += f * (double)(i == j) * h[i * n + i];
            c[p->d2s0 + i * n + j] = s;
        }
}

void dco_guess(void *h, double *x) {
    const doci_t *p = h;
    srand(0);
    for (long i = 0; i < p->n_primal; i++) x[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
}

void dco_Au(void *h, const double *x, double *out) {
    visit_t v = {AU, x, out, 0, 0.0, 0.0, 0};
    memset(out, 0, sizeof(double) * ((doci_t *)h)->n_dual);
    visit(h, &v);
}
void dco_ATu(void *h, const double *y, double *out) {
    visit_t v = {ATU, y, out, 0, 0.0, 0.0, 0};
    memset(out, 0, sizeof(double) * ((doci_t *)h)->n_primal);
    visit(h, &v);
}
