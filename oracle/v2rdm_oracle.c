/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Not part of the product: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Plain-C restatement of hilbert's v2RDM constraint maps for C1 symmetry
 * (one irrep, no frozen/restricted orbitals), written to follow the
 * reference's loop and accumulation order so that A.x and A^T.y agree with
 * the reference bit for bit.  Each function cites the reference code it
 * restates (paths relative to the hilbert source tree).
 *
 * Supported constraint sets: POSITIVITY D / DQ / DG / DQG / DQGT1 / DQGT2 /
 * DQGT1T2, each optionally with CONSTRAIN_D3, _Q3, _E3, _F3 and _D4, with
 * CONSTRAIN_SPIN and CONSTRAIN_SZ on or off, singlet and non-singlet.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int n;            /* active orbitals (amo_) */
    int na, nb;       /* alpha / beta electrons */
    int q2, g2, t1, t2, d3, q3, e3, f3, d4, spin, sz;
    int mult;         /* 2S+1 as the reference stores it */
    int gab, gaa;
    int *bas_ab, *ibas_ab, *bas_aa, *ibas_aa;
    long d2ab, d2aa, d2bb, d200, d1a, d1b, q1a, q1b, q2ab, q2aa, q2bb, g2ab, g2ba, g2aa;
    long t1aaa, t1bbb, t1aab, t1bba, t2aaa, t2bbb, t2aab, t2bba, d3aaa, d3bbb, d3aab, d3bba;
    long q3aaa, q3bbb, q3aab, q3bba, e3aaa, e3bbb, e3aab, e3bba, f3aaa, f3bbb, f3aab, f3bba;
    long d4aaaa, d4aaab, d4aabb, d4bbba, d4bbbb;
    int quad_aaaa, quad_aaab, quad_aabb;            /* quartets: i<j<k<l; i<j<k, l; i<j, k<l */
    int *ibas_aaaa, *ibas_aaab, *ibas_aabb;         /* n^4 each */
    int trip_aaa, trip_aab, trip_aba;   /* triplets (i<j<k), (i<j, k) and (i, j, k) */
    int *bas_aaa, *bas_aab, *bas_aba;   /* 3 ints per triplet */
    int *ibas_aaa, *ibas_aab;           /* n^3: any order of an aaa set / of the aa pair */
    long n_primal, n_dual;
    int nblocks;
    int dims[64];     /* at most 51 blocks: every family of the reference on */
} v2o_problem;

/* basis.cc:426-533 (C1): geminal (j,i) is pushed for i outer, j inner, so
 * geminal n = i*amo + j holds (first, second) = (j, i); aa geminals keep
 * first < second and are numbered in the same sweep. */
static void build_tables(v2o_problem *p) {
    int n = p->n;
    p->gab = n * n;
    p->gaa = n * (n - 1) / 2;
    p->bas_ab = (int *)malloc(sizeof(int) * 2 * (p->gab > 0 ? p->gab : 1));
    p->ibas_ab = (int *)malloc(sizeof(int) * (n * n > 0 ? n * n : 1));
    p->bas_aa = (int *)malloc(sizeof(int) * 2 * (p->gaa > 0 ? p->gaa : 1));
    p->ibas_aa = (int *)malloc(sizeof(int) * (n * n > 0 ? n * n : 1));
    for (int i = 0; i < n * n; i++) { p->ibas_ab[i] = -999; p->ibas_aa[i] = -999; }
    int count_ab = 0, count_aa = 0;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) {
            int first = j, second = i;
            p->ibas_ab[first * n + second] = count_ab;
            p->bas_ab[2 * count_ab] = first;
            p->bas_ab[2 * count_ab + 1] = second;
            count_ab++;
            if (first >= second) continue;
            p->ibas_aa[first * n + second] = count_aa;
            p->ibas_aa[second * n + first] = count_aa;
            p->bas_aa[2 * count_aa] = first;
            p->bas_aa[2 * count_aa + 1] = second;
            count_aa++;
        }
    }
}

#define IAB(p, i, j) ((p)->ibas_ab[(i) * (p)->n + (j)])
#define IAA(p, i, j) ((p)->ibas_aa[(i) * (p)->n + (j)])
#define D3_AAA(a, b, c) (p->ibas_aaa[((long)(a) * p->n + (b)) * p->n + (c)])
#define D3_AAB(a, b, c) (p->ibas_aab[((long)(a) * p->n + (b)) * p->n + (c)])

enum { MODE_AU = 0, MODE_ATU = 1, MODE_GUESS = 2 };
static void t1_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                     double *x);
static void t1_like_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                          double *x, int q3);
static void t2_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                     double *x);
static void d3_visit(const v2o_problem *p, long off, int mode, const double *u, double *A);
static void d4_visit(const v2o_problem *p, long off, int mode, const double *u, double *A);
/* number of D3 rows (v2rdm_solver.cc:3624-3660) */
static long d3_rows_count(const v2o_problem *p) {
    const long gaa = p->gaa, gab = p->gab, t3 = p->trip_aaa, ta = p->trip_aab;
    long d = p->sz ? 4 * gaa * gaa + 2 * gab * gab : 2 * gaa * gaa + gab * gab;
    if (p->spin && p->na == p->nb) d += ta * ta + 2 * t3 * t3;
    return d;
}

/* v2rdm_solver.cc:3729-4079 (set_primal_offsets) and 3294-3727 (sizes) */
static void set_offsets(v2o_problem *p) {
    long off = 0;
    int gab = p->gab, gaa = p->gaa, n = p->n, nb = 0;
    p->d2ab = off; off += (long)gab * gab; p->dims[nb++] = gab;
    p->d2aa = off; off += (long)gaa * gaa; p->dims[nb++] = gaa;
    p->d2bb = off; off += (long)gaa * gaa; p->dims[nb++] = gaa;
    p->d200 = -1;
    if (p->spin && p->na == p->nb) {
        p->d200 = off; off += (long)gab * gab; p->dims[nb++] = gab;
    } else if (p->spin) {
        p->d200 = off; off += 4L * gab * gab; p->dims[nb++] = 2 * gab;
    }
    p->d1a = off; off += (long)n * n; p->dims[nb++] = n;
    p->d1b = off; off += (long)n * n; p->dims[nb++] = n;
    p->q1a = off; off += (long)n * n; p->dims[nb++] = n;
    p->q1b = off; off += (long)n * n; p->dims[nb++] = n;
    p->q2ab = p->q2aa = p->q2bb = -1;
    if (p->q2) {
        p->q2ab = off; off += (long)gab * gab; p->dims[nb++] = gab;
        p->q2aa = off; off += (long)gaa * gaa; p->dims[nb++] = gaa;
        p->q2bb = off; off += (long)gaa * gaa; p->dims[nb++] = gaa;
    }
    p->g2ab = p->g2ba = p->g2aa = -1;
    if (p->g2) {
        p->g2ab = off; off += (long)gab * gab; p->dims[nb++] = gab;
        p->g2ba = off; off += (long)gab * gab; p->dims[nb++] = gab;
        p->g2aa = off; off += 4L * gab * gab; p->dims[nb++] = 2 * gab;
    }
    /* v2rdm_solver.cc:3848-3877: T1aaa, T1bbb (dim aaa), T1aab, T1bba (dim aab) */
    p->t1aaa = p->t1bbb = p->t1aab = p->t1bba = -1;
    if (p->t1) {
        long t3 = p->trip_aaa, ta = p->trip_aab;
        p->t1aaa = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->t1bbb = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->t1aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->t1bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:3879-3906: T2aaa, T2bbb (dim aab + aba), T2aab, T2bba (dim aab) */
    p->t2aaa = p->t2bbb = p->t2aab = p->t2bba = -1;
    if (p->t2) {
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        p->t2aaa = off; off += w * w; p->dims[nb++] = (int)w;
        p->t2bbb = off; off += w * w; p->dims[nb++] = (int)w;
        p->t2aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->t2bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:3909-3938: E3aaa, E3bbb (dim aab + aba), E3aab, E3bba (dim aab) */
    p->e3aaa = p->e3bbb = p->e3aab = p->e3bba = -1;
    if (p->e3) {
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        p->e3aaa = off; off += w * w; p->dims[nb++] = (int)w;
        p->e3bbb = off; off += w * w; p->dims[nb++] = (int)w;
        p->e3aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->e3bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:3940-3968: F3aaa, F3bbb (dim aab + aba), F3aab, F3bba (dim aab) */
    p->f3aaa = p->f3bbb = p->f3aab = p->f3bba = -1;
    if (p->f3) {
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        p->f3aaa = off; off += w * w; p->dims[nb++] = (int)w;
        p->f3bbb = off; off += w * w; p->dims[nb++] = (int)w;
        p->f3aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->f3bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:3970-3998: Q3aaa, Q3bbb (dim aaa), Q3aab, Q3bba (dim aab) */
    p->q3aaa = p->q3bbb = p->q3aab = p->q3bba = -1;
    if (p->q3) {
        long t3 = p->trip_aaa, ta = p->trip_aab;
        p->q3aaa = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->q3bbb = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->q3aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->q3bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:4000-4029: D3aaa, D3bbb (dim aaa), D3aab, D3bba (dim aab) */
    p->d3aaa = p->d3bbb = p->d3aab = p->d3bba = -1;
    if (p->d3) {
        long t3 = p->trip_aaa, ta = p->trip_aab;
        p->d3aaa = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->d3bbb = off; off += t3 * t3; p->dims[nb++] = (int)t3;
        p->d3aab = off; off += ta * ta; p->dims[nb++] = (int)ta;
        p->d3bba = off; off += ta * ta; p->dims[nb++] = (int)ta;
    }
    /* v2rdm_solver.cc:4030-4061: D4aaaa, D4aaab, D4aabb, D4bbba, D4bbbb */
    p->d4aaaa = p->d4aaab = p->d4aabb = p->d4bbba = p->d4bbbb = -1;
    if (p->d4) {
        long q4 = p->quad_aaaa, q31 = p->quad_aaab, q22 = p->quad_aabb;
        p->d4aaaa = off; off += q4 * q4; p->dims[nb++] = (int)q4;
        p->d4aaab = off; off += q31 * q31; p->dims[nb++] = (int)q31;
        p->d4aabb = off; off += q22 * q22; p->dims[nb++] = (int)q22;
        p->d4bbba = off; off += q31 * q31; p->dims[nb++] = (int)q31;
        p->d4bbbb = off; off += q4 * q4; p->dims[nb++] = (int)q4;
    }
    p->n_primal = off;
    p->nblocks = nb;
    if (nb > (int)(sizeof(p->dims) / sizeof(p->dims[0]))) abort();

    long d = 0;
    d += p->sz ? 3 : 1;
    d += 2L * gaa * gaa + (long)gab * gab;          /* hermiticity */
    d += 2L * n * n;                                 /* D1 + Q1 = I */
    d += (p->sz ? 4L : 2L) * n * n;                  /* partial traces */
    if (p->spin) {
        d += 1;
        if (p->na == p->nb) d += (long)n * n + 3L * gaa * gaa + 2L * gab * gab;
        else d += 4L * gab * gab;
        if (p->g2) d += 2L * gab;
    }
    if (p->q2) d += (long)gab * gab + 2L * gaa * gaa;
    if (p->g2) d += 6L * gab * gab;
    if (p->t1) {   /* v2rdm_solver.cc:3554-3567 */
        long t3 = p->trip_aaa, ta = p->trip_aab;
        d += 2 * t3 * t3 + 2 * ta * ta;
    }
    if (p->t2) {   /* v2rdm_solver.cc:3568-3580 */
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        d += 2 * w * w + 2 * ta * ta;
    }
    if (p->e3) {   /* v2rdm_solver.cc:3582-3595 */
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        d += 2 * ta * ta + 2 * w * w;
    }
    if (p->f3) {   /* v2rdm_solver.cc:3596-3609 */
        long w = (long)p->trip_aab + p->trip_aba, ta = p->trip_aab;
        d += 2 * ta * ta + 2 * w * w;
    }
    if (p->q3) {   /* v2rdm_solver.cc:3610-3623 */
        long t3 = p->trip_aaa, ta = p->trip_aab;
        d += 2 * t3 * t3 + 2 * ta * ta;
    }
    if (p->d3) {   /* v2rdm_solver.cc:3624-3660 */
        long t3 = p->trip_aaa, ta = p->trip_aab;
        d += p->sz ? 4L * gaa * gaa + 2L * gab * gab : 2L * gaa * gaa + (long)gab * gab;
        if (p->spin && p->na == p->nb) d += ta * ta + 2 * t3 * t3;
    }
    if (p->d4) {   /* v2rdm_solver.cc:3678-3707 */
        long t3 = p->trip_aaa, ta = p->trip_aab;
        if (p->na > 3) d += t3 * t3;
        if (p->na > 2 && p->nb > 0) d += t3 * t3 + ta * ta;
        /* counted twice by the reference (v2rdm_solver.cc:3692-3707) but written
         * once by D4_constraints_Au: the second 2 aab^2 rows stay empty, at the
         * end of the dual vector, and the dual vector keeps the reference's length */
        if (p->na > 1 && p->nb > 1) d += 4 * ta * ta;
        if (p->na > 0 && p->nb > 2) d += t3 * t3 + ta * ta;
        if (p->nb > 3) d += t3 * t3;
    }
    p->n_dual = d;
}

/* basis.cc:640-745 (C1): every (i, j, k) in i, j, k order is an aba triplet;
 * those with i < j are also aab triplets, and those with i < j < k aaa
 * triplets, each numbered in the same sweep. */
static void build_triplets(v2o_problem *p) {
    int n = p->n;
    long n3 = (long)n * n * n;
    p->bas_aba = (int *)malloc(sizeof(int) * 3 * (n3 > 0 ? n3 : 1));
    p->bas_aab = (int *)malloc(sizeof(int) * 3 * (n3 > 0 ? n3 : 1));
    p->bas_aaa = (int *)malloc(sizeof(int) * 3 * (n3 > 0 ? n3 : 1));
    p->ibas_aaa = (int *)malloc(sizeof(int) * (n3 > 0 ? n3 : 1));
    p->ibas_aab = (int *)malloc(sizeof(int) * (n3 > 0 ? n3 : 1));
    for (long e = 0; e < n3; e++) p->ibas_aaa[e] = p->ibas_aab[e] = -999;
#define TRIP(a, b, c) (((long)(a) * n + (b)) * n + (c))
    int c3 = 0, ca = 0, cb = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                int *t = p->bas_aba + 3 * cb++;
                t[0] = i; t[1] = j; t[2] = k;
                if (i >= j) continue;
                p->ibas_aab[TRIP(i, j, k)] = p->ibas_aab[TRIP(j, i, k)] = ca;
                t = p->bas_aab + 3 * ca++;
                t[0] = i; t[1] = j; t[2] = k;
                if (j >= k) continue;
                p->ibas_aaa[TRIP(i, j, k)] = p->ibas_aaa[TRIP(i, k, j)] = p->ibas_aaa[TRIP(j, i, k)] = c3;
                p->ibas_aaa[TRIP(j, k, i)] = p->ibas_aaa[TRIP(k, i, j)] = p->ibas_aaa[TRIP(k, j, i)] = c3;
                t = p->bas_aaa + 3 * c3++;
                t[0] = i; t[1] = j; t[2] = k;
            }
#undef TRIP
    p->trip_aaa = c3;
    p->trip_aab = ca;
    p->trip_aba = cb;
}

/* basis.cc:747-900 (C1): quartets (i, j, k, l) in lexicographic order; aabb
 * those with i < j and k < l (either order within each pair maps to it),
 * aaab those with i < j < k (any order of the first three), aaaa those with
 * i < j < k < l (any order). */
static void build_quartets(v2o_problem *p) {
    const int n = p->n;
    const long n4 = (long)n * n * n * n;
    p->ibas_aaaa = (int *)malloc(sizeof(int) * (n4 > 0 ? n4 : 1));
    p->ibas_aaab = (int *)malloc(sizeof(int) * (n4 > 0 ? n4 : 1));
    p->ibas_aabb = (int *)malloc(sizeof(int) * (n4 > 0 ? n4 : 1));
    for (long e = 0; e < n4; e++) p->ibas_aaaa[e] = p->ibas_aaab[e] = p->ibas_aabb[e] = -999;
#define Q4(a, b, c, d) ((((long)(a) * n + (b)) * n + (c)) * n + (d))
    int c4 = 0, c31 = 0, c22 = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++)
                for (int l = 0; l < n; l++) {
                    if (i < j && k < l) {
                        p->ibas_aabb[Q4(i, j, k, l)] = p->ibas_aabb[Q4(j, i, k, l)] = c22;
                        p->ibas_aabb[Q4(i, j, l, k)] = p->ibas_aabb[Q4(j, i, l, k)] = c22;
                        c22++;
                    }
                    if (i < j && j < k) {
                        const int t[3] = {i, j, k};
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                if (b != a) p->ibas_aaab[Q4(t[a], t[b], t[3 - a - b], l)] = c31;
                        c31++;
                    }
                    if (i < j && j < k && k < l) {
                        const int t[4] = {i, j, k, l};
                        for (int a = 0; a < 4; a++)
                            for (int b = 0; b < 4; b++)
                                for (int c = 0; c < 4; c++) {
                                    if (b == a || c == a || c == b) continue;
                                    p->ibas_aaaa[Q4(t[a], t[b], t[c], t[6 - a - b - c])] = c4;
                                }
                        c4++;
                    }
                }
#undef Q4
    p->quad_aaaa = c4;
    p->quad_aaab = c31;
    p->quad_aabb = c22;
}

/* positivity: 0 D, 1 DQ, 2 DG, 3 DQG, 4 DQGT2, 5 DQGT1, 6 DQGT1T2 (= DQGT)
 * (v2rdm_solver.cc:4081-4118), plus 16 for CONSTRAIN_D3 (:4120-4122) and 32 for
 * CONSTRAIN_Q3 (which implies D3, :4132-4135), 64 for CONSTRAIN_E3 (implies D3,
 * :4124-4127), 128 for CONSTRAIN_F3 (implies D3, :4128-4131) and 256 for
 * CONSTRAIN_D4 (implies D3, :4144-4149).
 * hubbard selects the multiplicity convention of
 * v2rdm_solver.cc:862-863 (Hubbard) versus :983-984 (external). */
v2o_problem *v2o_create(int n, int na, int nb, int positivity, int spin, int sz, int hubbard) {
    const int q3 = (positivity >> 5) & 1, e3 = (positivity >> 6) & 1, f3 = (positivity >> 7) & 1;
    const int d4 = (positivity >> 8) & 1;
    const int d3 = ((positivity >> 4) & 1) | q3 | e3 | f3 | d4;
    positivity &= 15;
    if (n < 1 || na < 0 || nb < 0 || na > n || nb > n || positivity < 0 || positivity > 6) return NULL;
    v2o_problem *p = (v2o_problem *)calloc(1, sizeof(v2o_problem));
    p->n = n; p->na = na; p->nb = nb;
    p->d3 = d3;
    p->q3 = q3;
    p->e3 = e3;
    p->f3 = f3;
    p->d4 = d4;
    p->q2 = (positivity == 1 || positivity >= 3);
    p->g2 = (positivity >= 2);
    p->t1 = (positivity == 5 || positivity == 6);
    p->t2 = (positivity == 4 || positivity == 6);
    if (p->q3 && !(p->q2 && p->g2)) {   /* the Q3 rows read Q2 and G2 elements */
        free(p);
        return NULL;
    }
    p->spin = spin != 0; p->sz = sz != 0;
    p->mult = hubbard ? 2 * (na - nb) + 1 : (na - nb) + 1;
    build_tables(p);
    if (p->t1 || p->t2 || p->d3) build_triplets(p);
    if (p->d4) build_quartets(p);
    set_offsets(p);
    return p;
}

void v2o_destroy(v2o_problem *p) {
    if (!p) return;
    free(p->bas_ab); free(p->ibas_ab); free(p->bas_aa); free(p->ibas_aa);
    free(p->bas_aaa); free(p->bas_aab); free(p->bas_aba); free(p->ibas_aaa); free(p->ibas_aab);
    free(p->ibas_aaaa); free(p->ibas_aaab); free(p->ibas_aabb);
    free(p);
}

long v2o_n_primal(const v2o_problem *p) { return p->n_primal; }
long v2o_n_dual(const v2o_problem *p) { return p->n_dual; }
int v2o_n_blocks(const v2o_problem *p) { return p->nblocks; }
void v2o_block_dims(const v2o_problem *p, int *out) { memcpy(out, p->dims, sizeof(int) * p->nblocks); }
void v2o_gems(const v2o_problem *p, int *gab, int *gaa) { *gab = p->gab; *gaa = p->gaa; }
void v2o_tables(const v2o_problem *p, int *bas_ab, int *ibas_ab, int *bas_aa, int *ibas_aa) {
    memcpy(bas_ab, p->bas_ab, sizeof(int) * 2 * p->gab);
    memcpy(bas_aa, p->bas_aa, sizeof(int) * 2 * p->gaa);
    memcpy(ibas_ab, p->ibas_ab, sizeof(int) * p->n * p->n);
    memcpy(ibas_aa, p->ibas_aa, sizeof(int) * p->n * p->n);
}
/* block offsets in the order d2ab d2aa d2bb d200 d1a d1b q1a q1b q2ab q2aa q2bb g2ab g2ba g2aa */
void v2o_offsets(const v2o_problem *p, long *o) {
    long v[43] = {p->d2ab, p->d2aa, p->d2bb, p->d200, p->d1a, p->d1b, p->q1a,
                  p->q1b,  p->q2ab, p->q2aa, p->q2bb, p->g2ab, p->g2ba, p->g2aa,
                  p->t2aaa, p->t2bbb, p->t2aab, p->t2bba,
                  p->t1aaa, p->t1bbb, p->t1aab, p->t1bba, p->d3aaa, p->d3bbb, p->d3aab, p->d3bba,
                  p->q3aaa, p->q3bbb, p->q3aab, p->q3bba, p->e3aaa, p->e3bbb, p->e3aab, p->e3bba,
                  p->f3aaa, p->f3bbb, p->f3aab, p->f3bba, p->d4aaaa, p->d4aaab, p->d4aabb,
                  p->d4bbba, p->d4bbbb};
    memcpy(o, v, sizeof(v));
}

/* ---------------------------------------------------------------- b ---- */
/* v2rdm_solver.cc:1826-2070 (BuildConstraints) */
void v2o_build_b(const v2o_problem *p, double *b) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    double na = p->na, nb = p->nb;
    memset(b, 0, sizeof(double) * p->n_dual);
    long off = 0;
    if (p->sz) {
        b[off++] = na * nb;
        b[off++] = na * (na - 1.0);
        b[off++] = nb * (nb - 1.0);
    } else {
        double nt = na + nb;
        b[off++] = nt * (nt - 1.0);
    }
    off += 2L * gaa * gaa + (long)gab * gab;
    for (int s = 0; s < 2; s++) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) b[off + i * n + j] = (double)(i == j);
        off += (long)n * n;
    }
    off += (p->sz ? 4L : 2L) * n * n;
    if (p->spin) {
        double ms = (p->mult - 1.0) / 2.0;
        b[off++] = 0.5 * (na + nb) + ms * ms - ms * (ms + 1.0);
        if (p->na == p->nb) off += (long)n * n + 3L * gaa * gaa + 2L * gab * gab;
        else off += 4L * gab * gab;
        if (p->g2) off += 2L * gab;
    }
    if (p->q2) {
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                b[off + (long)ij * gab + kl] = -(i == k) * (j == l);
            }
        }
        off += (long)gab * gab;
        for (int s = 0; s < 2; s++) {
            for (int ij = 0; ij < gaa; ij++) {
                int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                    b[off + (long)ij * gaa + kl] = -(i == k) * (j == l) + (i == l) * (j == k);
                }
            }
            off += (long)gaa * gaa;
        }
    }
}

/* ---------------------------------------------------------------- c ---- */
/* Hubbard ring: oei.cc:76-95 (h), tei.cc:285-292 ((ii|ii) = U), repacked
 * through tei.cc:139-199 / 201-275 (RepackIntegrals, FrozenCoreEnergy). */
void v2o_build_c_hubbard(const v2o_problem *p, double t, double U, double *c) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    memset(c, 0, sizeof(double) * p->n_primal);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            /* only the upper triangle survives the packed oei buffer */
            int lo = i < j ? i : j, hi = i < j ? j : i;
            double h = 0.0;
            if (abs(lo - hi) == 1) h = -t;
            else if (abs(lo - hi) == n - 1) h = -t;
            c[p->d1a + i * n + j] = h;
            c[p->d1b + i * n + j] = h;
            c[p->d1a + i * n + j] += 0.0;
            c[p->d1b + i * n + j] += 0.0;
        }
    for (int ij = 0; ij < gab; ij++) {
        int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
            /* TEI(i,k,j,l) */
            c[p->d2ab + (long)ij * gab + kl] = (i == k && j == l && i == j) ? U : 0.0;
        }
    }
    for (int ij = 0; ij < gaa; ij++) {
        int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
        for (int kl = 0; kl < gaa; kl++) {
            int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
            double d1 = (i == k && j == l && i == j) ? U : 0.0;
            double d2 = (i == l && j == k && i == j) ? U : 0.0;
            c[p->d2aa + (long)ij * gaa + kl] = d1 - d2;
            c[p->d2bb + (long)ij * gaa + kl] = d1 - d2;
        }
    }
}

/* external Hamiltonian: v2rdm_solver.cc:164-193 (h -> D1, (ik|jl) -> D2ab,
 * (ik|jl)-(il|jk) -> D2aa/bb), then GetOEI_external (oei.cc:59-74) and
 * RepackIntegrals: D1 is rebuilt from the upper triangle of h. */
void v2o_build_c_external(const v2o_problem *p, const double *h, const double *g, double *c) {
    long n = p->n;
    int gab = p->gab, gaa = p->gaa;
    memset(c, 0, sizeof(double) * p->n_primal);
    for (long i = 0; i < n; i++)
        for (long j = 0; j < n; j++) {
            long lo = i < j ? i : j, hi = i < j ? j : i;
            double v = h[lo * n + hi];
            c[p->d1a + i * n + j] = v;
            c[p->d1b + i * n + j] = v;
            c[p->d1a + i * n + j] += 0.0;
            c[p->d1b + i * n + j] += 0.0;
        }
    for (int ij = 0; ij < gab; ij++) {
        long i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            long k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
            c[p->d2ab + (long)ij * gab + kl] = g[i * n * n * n + k * n * n + j * n + l];
        }
    }
    for (int ij = 0; ij < gaa; ij++) {
        long i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
        for (int kl = 0; kl < gaa; kl++) {
            long k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
            double v = g[i * n * n * n + k * n * n + j * n + l] - g[i * n * n * n + l * n * n + j * n + k];
            c[p->d2aa + (long)ij * gaa + kl] = v;
            c[p->d2bb + (long)ij * gaa + kl] = v;
        }
    }
}

/* ------------------------------------------------------------ guess ---- */
/* v2rdm_solver.cc:1799-1806: srand(0); x = (rand()/RAND_MAX - 1) * 2 */
void v2o_guess_random(const v2o_problem *p, double *x) {
    srand(0);
    for (long i = 0; i < p->n_primal; i++) x[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
}

/* q2.cc:45-167 (Q2 guess) */
static void q2_guess(const v2o_problem *p, double *u) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    for (int ij = 0; ij < gab; ij++) {
        int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
            double dum = 0.0;
            dum += u[p->d2ab + (long)kl * gab + ij];
            if (j == l) dum += u[p->q1a + i * n + k];
            if (i == k) dum -= u[p->d1b + l * n + j];
            u[p->q2ab + (long)ij * gab + kl] = dum;
        }
    }
    for (int s = 0; s < 2; s++) {
        long d2 = s ? p->d2bb : p->d2aa, q2 = s ? p->q2bb : p->q2aa;
        long q1 = s ? p->q1b : p->q1a, d1 = s ? p->d1b : p->d1a;
        for (int ij = 0; ij < gaa; ij++) {
            int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
            for (int kl = 0; kl < gaa; kl++) {
                int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                double dum = 0.0;
                dum += u[d2 + (long)kl * gaa + ij];
                if (j == l) dum += u[q1 + i * n + k];
                if (j == k) dum += u[d1 + l * n + i];
                if (i == l) dum -= u[q1 + j * n + k];
                if (i == k) dum -= u[d1 + l * n + j];
                u[q2 + (long)ij * gaa + kl] = dum;
            }
        }
    }
}

/* g2.cc:44-242 (G2 guess) */
static void g2_guess(const v2o_problem *p, double *u) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    for (int s = 0; s < 2; s++) {
        long g2 = s ? p->g2ba : p->g2ab, d1 = s ? p->d1b : p->d1a;
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = 0.0;
                if (j == l) dum += u[d1 + i * n + k];
                if (s == 0) dum -= u[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, k, j)];
                else dum -= u[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, j, k)];
                u[g2 + (long)ij * gab + kl] = dum;
            }
        }
    }
    long g = p->g2aa;
    long w = 2L * gab;
    for (int s = 0; s < 2; s++) {
        long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa, sh = s ? gab : 0;
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = 0.0;
                if (j == l) dum += u[d1 + i * n + k];
                if (i != l && k != j) {
                    int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                    dum -= u[d2 + (long)IAA(p, i, l) * gaa + IAA(p, k, j)] * sil * skj;
                }
                u[g + (sh + ij) * w + (sh + kl)] = dum;
            }
        }
    }
    for (int ij = 0; ij < gab; ij++) {
        int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
            double dum = 0.0;
            dum += u[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, j, k)];
            u[g + (long)ij * w + (gab + kl)] = dum;
        }
    }
    for (int ij = 0; ij < gab; ij++) {
        int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
        for (int kl = 0; kl < gab; kl++) {
            int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
            double dum = 0.0;
            dum += u[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, k, j)];
            u[g + (gab + ij) * w + kl] = dum;
        }
    }
}

/* v2rdm_solver.cc:1713-1823 (TPDM_GUESS HF).  The reference stores
 * doccpi = nalpha and soccpi = 0 for Hubbard/external problems
 * (v2rdm_solver.cc:881-882, 1003-1004), so both spins occupy nalpha orbitals. */
void v2o_guess_hf(const v2o_problem *p, double *x) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    int occ = p->na;
    memset(x, 0, sizeof(double) * p->n_primal);
    for (int i = 0; i < occ; i++)
        for (int j = 0; j < occ; j++) {
            int ij = IAB(p, i, j);
            x[p->d2ab + (long)ij * gab + ij] = 1.0;
        }
    for (int i = 0; i < occ; i++)
        for (int j = 0; j < i; j++) {
            int ij = IAA(p, i, j);
            x[p->d2aa + (long)ij * gaa + ij] = 1.0;
        }
    for (int i = 0; i < occ; i++)
        for (int j = 0; j < i; j++) {
            int ij = IAA(p, i, j);
            x[p->d2bb + (long)ij * gaa + ij] = 1.0;
        }
    for (int i = 0; i < occ; i++) x[p->d1a + i * n + i] = 1.0;
    for (int i = 0; i < occ; i++) x[p->d1b + i * n + i] = 1.0;
    for (int i = occ; i < n; i++) x[p->q1a + i * n + i] = 1.0;
    for (int i = occ; i < n; i++) x[p->q1b + i * n + i] = 1.0;
    if (p->q2) q2_guess(p, x);
    if (p->g2) g2_guess(p, x);
    if (p->t1) t1_visit(p, 0, MODE_GUESS, NULL, NULL, x);   /* v2rdm_solver.cc:1817-1819 */
    if (p->t2) t2_visit(p, 0, MODE_GUESS, NULL, NULL, x);   /* v2rdm_solver.cc:1820-1822 */
}

/* ------------------------------------------------------------- T2 ---- */
/* The T2 rows of t2.cc:1236-1843 (T2_constraints_Au_slow, C1).  Each dual
 * row belongs to one element (r, c) of a T2 block and reads
 *     -T2(r, c) + sum of conditional D2 / D1 terms with coefficients +-1,
 * the terms added left to right in the order the reference adds them.  The
 * ten sub-blocks, in the reference's order of dual rows:
 *   0 T2aab (rows, cols: aab triplets)            t2.cc:1239-1302
 *   1 T2bba                                        t2.cc:1305-1368
 *   2-5 T2aaa: aaa/aaa, aaa/abb, abb/aaa, abb/abb t2.cc:1371-1601
 *   6-9 T2bbb: bbb/bbb, bbb/baa, baa/bbb, baa/baa t2.cc:1604-1840
 * ("aaa" rows/cols are the aab triplets, "abb" / "baa" the aba triplets,
 * placed after them in the big blocks). */
typedef struct { long col; double coef; } map_term;

#define T2_D2AA(a, b, c, d) (p->d2aa + (long)IAA(p, a, b) * p->gaa + IAA(p, c, d))
#define T2_D2BB(a, b, c, d) (p->d2bb + (long)IAA(p, a, b) * p->gaa + IAA(p, c, d))
#define T2_D2AB(a, b, c, d) (p->d2ab + (long)IAB(p, a, b) * p->gab + IAB(p, c, d))
#define T2_D1A(a, b) (p->d1a + (long)(a) * p->n + (b))
#define T2_D1B(a, b) (p->d1b + (long)(a) * p->n + (b))
#define ADD_TERM(c, v) do { t[nt].col = (c); t[nt].coef = (v); nt++; } while (0)

/* sign of an aa geminal read as (a, b): -1 when a > b (the reference's s) */
static double pair_sign(int a, int b) { return a > b ? -1.0 : 1.0; }

/* terms of row (i, j, k) x column (l, m, q) of sub-block sb, at most 7 */
static int t2_terms(const v2o_problem *p, int sb, int i, int j, int k, int l, int m, int q,
                    map_term *t) {
    int nt = 0;
    switch (sb) {
    case 0:   /* T2aab */
    case 1: { /* T2bba: the same terms with alpha and beta exchanged */
        const int b = sb == 1;
        if (k == q) ADD_TERM(b ? T2_D2BB(i, j, l, m) : T2_D2AA(i, j, l, m), 1.0);
        if (j == m && i == l) ADD_TERM(b ? T2_D1A(q, k) : T2_D1B(q, k), 1.0);
        if (j == l && i == m) ADD_TERM(b ? T2_D1A(q, k) : T2_D1B(q, k), -1.0);
        if (i == l) ADD_TERM(b ? T2_D2AB(q, j, k, m) : T2_D2AB(j, q, m, k), -1.0);
        if (j == l) ADD_TERM(b ? T2_D2AB(q, i, k, m) : T2_D2AB(i, q, m, k), 1.0);
        if (i == m) ADD_TERM(b ? T2_D2AB(q, j, k, l) : T2_D2AB(j, q, l, k), 1.0);
        if (j == m) ADD_TERM(b ? T2_D2AB(q, i, k, l) : T2_D2AB(i, q, l, k), -1.0);
        break;
    }
    case 2:   /* aaa/aaa */
    case 6: { /* bbb/bbb */
        const int b = sb == 6;
        if (k == q) ADD_TERM(b ? T2_D2BB(i, j, l, m) : T2_D2AA(i, j, l, m), 1.0);
        if (j == m && i == l) ADD_TERM(b ? T2_D1B(q, k) : T2_D1A(q, k), 1.0);
        if (j == l && i == m) ADD_TERM(b ? T2_D1B(q, k) : T2_D1A(q, k), -1.0);
        if (i == l && q != j && k != m)
            ADD_TERM(b ? T2_D2BB(q, j, k, m) : T2_D2AA(q, j, k, m), -pair_sign(q, j) * pair_sign(k, m));
        if (j == l && q != i && k != m)
            ADD_TERM(b ? T2_D2BB(q, i, k, m) : T2_D2AA(q, i, k, m), pair_sign(q, i) * pair_sign(k, m));
        if (i == m && q != j && k != l)
            ADD_TERM(b ? T2_D2BB(q, j, k, l) : T2_D2AA(q, j, k, l), pair_sign(q, j) * pair_sign(k, l));
        if (j == m && q != i && k != l)
            ADD_TERM(b ? T2_D2BB(q, i, k, l) : T2_D2AA(q, i, k, l), -pair_sign(q, i) * pair_sign(k, l));
        break;
    }
    case 3:   /* aaa/abb */
        if (i == l) ADD_TERM(T2_D2AB(j, q, k, m), 1.0);
        if (j == l) ADD_TERM(T2_D2AB(i, q, k, m), -1.0);
        break;
    case 7:   /* bbb/baa */
        if (i == l) ADD_TERM(T2_D2AB(q, j, m, k), 1.0);
        if (j == l) ADD_TERM(T2_D2AB(q, i, m, k), -1.0);
        break;
    case 4:   /* abb/aaa */
        if (i == l) ADD_TERM(T2_D2AB(q, j, m, k), 1.0);
        if (i == m) ADD_TERM(T2_D2AB(q, j, l, k), -1.0);
        break;
    case 8:   /* baa/bbb */
        if (i == l) ADD_TERM(T2_D2AB(j, q, k, m), 1.0);
        if (i == m) ADD_TERM(T2_D2AB(j, q, k, l), -1.0);
        break;
    case 5:   /* abb/abb */
        if (k == q) ADD_TERM(T2_D2AB(i, j, l, m), 1.0);
        if (j == m && i == l) ADD_TERM(T2_D1B(q, k), 1.0);
        if (i == l && q != j && k != m) ADD_TERM(T2_D2BB(q, j, k, m), -pair_sign(q, j) * pair_sign(k, m));
        if (j == m) ADD_TERM(T2_D2AB(i, q, l, k), -1.0);
        break;
    case 9:   /* baa/baa */
        if (k == q) ADD_TERM(T2_D2AB(j, i, m, l), 1.0);
        if (j == m && i == l) ADD_TERM(T2_D1A(q, k), 1.0);
        if (i == l && q != j && k != m) ADD_TERM(T2_D2AA(q, j, k, m), -pair_sign(q, j) * pair_sign(k, m));
        if (j == m) ADD_TERM(T2_D2AB(q, i, k, l), -1.0);
        break;
    }
    return nt;
}

/* Visit every T2 row in the reference's order, dual rows from off.
 *  MODE_AU:    A[row] = -u[t2] + terms                       (t2.cc:1236-1843)
 *  MODE_ATU:   A[t2] -= u[row], A[col] += coef u[row]         (t2.cc:3376-3966,
 *            the scatter of the same terms in the same order)
 *  MODE_GUESS: u[t2] = 0 + terms, zero on aaa/abb             (t2.cc:1845-2452) */
typedef int (*big_terms_fn)(const v2o_problem *, int, int, int, int, int, int, int, map_term *);

/* the T2 block layout (aab, bba, then the aab+aba blocks), rows led by
 * -X(r, c) for X in lead = {aab, bba, aaa, bbb} */
static void big_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                      double *x, big_terms_fn terms, const long lead[4]) {
    const long ta = p->trip_aab, tb = p->trip_aba, w = ta + tb;
    const long dual[4] = {off, off + ta * ta, off + 2 * ta * ta, off + 2 * ta * ta + w * w};
    const long *prim = lead;
    for (int sb = 0; sb < 10; sb++) {
        const int blk = sb < 2 ? sb : (sb < 6 ? 2 : 3);
        const long width = sb < 2 ? ta : w;
        const int rows_aba = (sb == 4 || sb == 5 || sb == 8 || sb == 9);
        const int cols_aba = (sb == 3 || sb == 5 || sb == 7 || sb == 9);
        const long nr = rows_aba ? tb : ta, nc = cols_aba ? tb : ta;
        const long r0 = rows_aba ? ta : 0, c0 = cols_aba ? ta : 0;
        const int *rb = rows_aba ? p->bas_aba : p->bas_aab, *cb = cols_aba ? p->bas_aba : p->bas_aab;
        for (long r = 0; r < nr; r++) {
            const int i = rb[3 * r], j = rb[3 * r + 1], k = rb[3 * r + 2];
            for (long c = 0; c < nc; c++) {
                const int l = cb[3 * c], m = cb[3 * c + 1], q = cb[3 * c + 2];
                const long id = (r0 + r) * width + (c0 + c);
                map_term t[8];
                const int nt = terms(p, sb, i, j, k, l, m, q, t);
                if (mode == MODE_AU) {
                    double dum = -u[prim[blk] + id];
                    for (int e = 0; e < nt; e++) dum += t[e].coef * u[t[e].col];
                    A[dual[blk] + id] = dum;
                } else if (mode == MODE_ATU) {
                    const double dum = u[dual[blk] + id];
                    A[prim[blk] + id] -= dum;
                    for (int e = 0; e < nt; e++) A[t[e].col] += t[e].coef * dum;
                } else {
                    double dum = 0.0;
                    for (int e = 0; e < nt; e++) dum += t[e].coef * x[t[e].col];
                    x[prim[blk] + id] = sb == 3 ? 0.0 : dum;
                }
            }
        }
    }
}

static void t2_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                     double *x) {
    const long lead[4] = {p->t2aab, p->t2bba, p->t2aaa, p->t2bbb};
    big_visit(p, off, mode, u, A, x, t2_terms, lead);
}

/* ------------------------------------------------------------- E3 ---- */
/* CONSTRAIN_E3 rows of e3.cc:45-566 (scatter :570-1082) in T2's layout:
 * -E3(r, c), then one D3 element (the row's third index swapped with the
 * column's: (i j n | l m k)) with a sign, then d_kn times a D2 element.
 * Sub-blocks as for T2. */
static int e3_terms(const v2o_problem *p, int sb, int i, int j, int k, int l, int m, int q,
                    map_term *t) {
    int nt = 0;
    const long ta = p->trip_aab, t3 = p->trip_aaa;
#define E3_AB(base, a, b, c, d, e, f) ((base) + (long)D3_AAB(a, b, c) * ta + D3_AAB(d, e, f))
#define E3_AA3(base, a, b, c, d, e, f) ((base) + (long)D3_AAA(a, b, c) * t3 + D3_AAA(d, e, f))
    switch (sb) {
    case 0:
    case 1: {
        const int b = sb == 1;
        ADD_TERM(E3_AB(b ? p->d3bba : p->d3aab, i, j, q, l, m, k), -1.0);
        if (k == q) ADD_TERM(b ? T2_D2BB(i, j, l, m) : T2_D2AA(i, j, l, m), 1.0);
        break;
    }
    case 2:
    case 6: {
        const int b = sb == 6;
        if (i != q && j != q && l != k && m != k) {
            const double sg = ((i < q && q < j) ? -1.0 : 1.0) * ((l < k && k < m) ? -1.0 : 1.0);
            ADD_TERM(E3_AA3(b ? p->d3bbb : p->d3aaa, i, j, q, l, m, k), -sg);
        }
        if (k == q) ADD_TERM(b ? T2_D2BB(i, j, l, m) : T2_D2AA(i, j, l, m), 1.0);
        break;
    }
    case 3:
        if (i != j && l != k) ADD_TERM(E3_AB(p->d3aab, i, j, q, l, k, m), l > k ? -1.0 : 1.0);
        break;
    case 7:
        if (i != j && l != k)
            ADD_TERM(E3_AB(p->d3bba, i, j, q, l, k, m), (i > j ? -1.0 : 1.0) * (l > k ? -1.0 : 1.0));
        break;
    case 4:
        if (i != q && l != m) ADD_TERM(E3_AB(p->d3aab, i, q, j, l, m, k), i > q ? -1.0 : 1.0);
        break;
    case 8:
        if (i != q && l != m)
            ADD_TERM(E3_AB(p->d3bba, i, q, j, l, m, k), (i > q ? -1.0 : 1.0) * (l > m ? -1.0 : 1.0));
        break;
    case 5:
    case 9: {
        const int b = sb == 9;
        if (j != q && m != k) {
            const double sg = (j > q ? -1.0 : 1.0) * (m > k ? -1.0 : 1.0);
            ADD_TERM(E3_AB(b ? p->d3aab : p->d3bba, j, q, i, m, k, l), -sg);
        }
        if (k == q) ADD_TERM(b ? T2_D2AB(j, i, m, l) : T2_D2AB(i, j, l, m), 1.0);
        break;
    }
    }
#undef E3_AB
#undef E3_AA3
    return nt;
}

static void e3_visit(const v2o_problem *p, long off, int mode, const double *u, double *A) {
    const long lead[4] = {p->e3aab, p->e3bba, p->e3aaa, p->e3bbb};
    big_visit(p, off, mode, u, A, NULL, e3_terms, lead);
}


/* ------------------------------------------------------------- F3 ---- */
/* CONSTRAIN_F3 rows of f3.cc:45-836 (scatter :842-1623), T2's layout: -F3,
 * then E3's D3 element with the opposite sign, then T2's terms without the
 * d_kn D2 term that E3 carries (T2 = E3 + F3), all in the reference's order. */
static int f3_terms(const v2o_problem *p, int sb, int i, int j, int k, int l, int m, int q,
                    map_term *t) {
    map_term e[8], w[8];
    const int ne = e3_terms(p, sb, i, j, k, l, m, q, e);
    const int nw = t2_terms(p, sb, i, j, k, l, m, q, w);
    int nt = 0;
    if (ne > 0 && e[0].col >= p->d3aaa) {   /* the D3 element, when the row has one */
        t[nt] = e[0];
        t[nt].coef = -e[0].coef;
        nt++;
    }
    const int skip = (k == q && (sb == 0 || sb == 1 || sb == 2 || sb == 5 || sb == 6 || sb == 9));
    for (int x = skip; x < nw; x++) t[nt++] = w[x];
    return nt;
}

static void f3_visit(const v2o_problem *p, long off, int mode, const double *u, double *A) {
    const long lead[4] = {p->f3aab, p->f3bba, p->f3aaa, p->f3bbb};
    big_visit(p, off, mode, u, A, NULL, f3_terms, lead);
}

/* ------------------------------------------------------------- T1 ---- */
/* The T1 rows of t1.cc:419-795 (T1_constraints_Au, C1): each dual row is
 *     -T1(r, c) + conditional Q2 / D2 / G2 / D1 terms (coefficients +-1),
 * added in the reference's order, four sub-blocks in the order of dual rows:
 *   0 T1aab (rows, cols: aab triplets)   t1.cc:421-467
 *   1 T1bba                              t1.cc:469-515
 *   2 T1aaa (aaa triplets, i<j<k)        t1.cc:517-650
 *   3 T1bbb                              t1.cc:652-793
 * A^T.y scatters the same terms in the same order (t1.cc:795-1200) and the
 * guess sums them from zero (t1.cc:45-419). */
#define T1_G2S(r, c, sh) (p->g2aa + ((long)(r) + (sh)) * 2 * p->gab + ((c) + (sh)))
#define T1_G2H(base, r, c) ((base) + (long)(r) * p->gab + (c))

static int t1_terms(const v2o_problem *p, int sb, int i, int j, int k, int l, int m, int q,
                    map_term *t) {
    int nt = 0;
    if (sb < 2) {   /* aab, bba */
        const int b = sb == 1;
        const long q2 = b ? p->q2bb : p->q2aa, g2 = b ? p->g2ab : p->g2ba;
        if (k == q) ADD_TERM(q2 + (long)IAA(p, i, j) * p->gaa + IAA(p, l, m), 1.0);
        if (b) {
            if (j == l) ADD_TERM(T2_D2AB(q, m, k, i), -1.0);
            if (l == i) ADD_TERM(T2_D2AB(q, m, k, j), 1.0);
        } else {
            if (j == l) ADD_TERM(T2_D2AB(m, q, i, k), -1.0);
            if (l == i) ADD_TERM(T2_D2AB(m, q, j, k), 1.0);
        }
        if (j == m) ADD_TERM(T1_G2H(g2, IAB(p, q, i), IAB(p, k, l)), -1.0);
        if (i == m) ADD_TERM(T1_G2H(g2, IAB(p, q, j), IAB(p, k, l)), 1.0);
        return nt;
    }
    /* aaa, bbb */
    const int b = sb == 3;
    const long q2 = b ? p->q2bb : p->q2aa, d2 = b ? p->d2bb : p->d2aa, d1 = b ? p->d1b : p->d1a;
    const int sh = b ? p->gab : 0;
#define T1_AA(base, a, bb, c, d) ((base) + (long)IAA(p, a, bb) * p->gaa + IAA(p, c, d))
    if (k == q) ADD_TERM(T1_AA(q2, i, j, l, m), 1.0);
    if (j == q) ADD_TERM(T1_AA(q2, i, k, l, m), -1.0);
    if (i == q) ADD_TERM(T1_AA(q2, j, k, l, m), 1.0);
    if (l == k) ADD_TERM(T1_AA(d2, q, m, j, i), 1.0);
    if (j == l) ADD_TERM(T1_AA(d2, q, m, k, i), -1.0);
    if (l == i) ADD_TERM(T1_AA(d2, q, m, k, j), 1.0);
    if (k == m) {
        if (j == l) ADD_TERM(d1 + (long)q * p->n + i, -1.0);
        ADD_TERM(T1_G2S(IAB(p, q, i), IAB(p, j, l), sh), 1.0);
    }
    if (j == m) {
        if (k == l) ADD_TERM(d1 + (long)q * p->n + i, 1.0);
        ADD_TERM(T1_G2S(IAB(p, q, i), IAB(p, k, l), sh), -1.0);
    }
    if (i == m) {
        if (k == l) ADD_TERM(d1 + (long)q * p->n + j, -1.0);
        ADD_TERM(T1_G2S(IAB(p, q, j), IAB(p, k, l), sh), 1.0);
    }
#undef T1_AA
    return nt;
}

/* T1 rows lead with -T1; the Q3 rows of q3.cc:45-423 (scatter :425-803)
 * lead with -Q3 - D3 and continue with the same terms as T1. */
static void t1_like_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                          double *x, int q3) {
    const long ta = p->trip_aab, t3 = p->trip_aaa;
    const long dual[4] = {off, off + ta * ta, off + 2 * ta * ta, off + 2 * ta * ta + t3 * t3};
    const long prim[4] = {q3 ? p->q3aab : p->t1aab, q3 ? p->q3bba : p->t1bba,
                          q3 ? p->q3aaa : p->t1aaa, q3 ? p->q3bbb : p->t1bbb};
    const long prim2[4] = {p->d3aab, p->d3bba, p->d3aaa, p->d3bbb};
    for (int sb = 0; sb < 4; sb++) {
        const long nr = sb < 2 ? ta : t3;
        const int *tb = sb < 2 ? p->bas_aab : p->bas_aaa;
        for (long r = 0; r < nr; r++) {
            const int i = tb[3 * r], j = tb[3 * r + 1], k = tb[3 * r + 2];
            for (long c = 0; c < nr; c++) {
                const int l = tb[3 * c], m = tb[3 * c + 1], q = tb[3 * c + 2];
                const long id = r * nr + c;
                map_term t[12];
                const int nt = t1_terms(p, sb, i, j, k, l, m, q, t);
                if (mode == MODE_AU) {
                    double dum = -u[prim[sb] + id];
                    if (q3) dum -= u[prim2[sb] + id];
                    for (int e = 0; e < nt; e++) dum += t[e].coef * u[t[e].col];
                    A[dual[sb] + id] = dum;
                } else if (mode == MODE_ATU) {
                    const double dum = u[dual[sb] + id];
                    A[prim[sb] + id] -= dum;
                    if (q3) A[prim2[sb] + id] -= dum;
                    for (int e = 0; e < nt; e++) A[t[e].col] += t[e].coef * dum;
                } else {
                    double dum = 0.0;
                    for (int e = 0; e < nt; e++) dum += t[e].coef * x[t[e].col];
                    x[prim[sb] + id] = dum;
                }
            }
        }
    }
}

static void t1_visit(const v2o_problem *p, long off, int mode, const double *u, double *A,
                     double *x) {
    t1_like_visit(p, off, mode, u, A, x, 0);
}

/* ------------------------------------------------------------- D3 ---- */
/* CONSTRAIN_D3 rows of d3.cc:45-406 (D3_constraints_Au, C1), each a plain
 * list of terms summed left to right (the first one a D2 element times an
 * electron count), and their scatter in the same order (d3.cc:408-766):
 *  with CONSTRAIN_SZ (d3.cc:49-212)
 *    (na-2) D2aa(ij,kl) - sum_p s D3aaa(ijp,klp)      p not in {i,j,k,l}
 *    (nb-2) D2bb(ij,kl) - sum_p s D3bbb(ijp,klp)
 *    nb D2aa(ij,kl)     - sum_p D3aab(ij p, kl p)
 *    na D2bb(ij,kl)     - sum_p D3bba(ij p, kl p)
 *    (na-1) D2ab(ij,kl) - sum_p s D3aab(ip j, kp l)   p != i, k
 *    (nb-1) D2ab(ij,kl) - sum_p s D3bba(jp i, lp k)   p != j, l
 *  without it (d3.cc:213-330): (na+nb-2) D2 - the D3 terms of both spins;
 *  singlets with CONSTRAIN_SPIN (d3.cc:332-404): D3aab - D3bba, and D3aaa
 *  (D3bbb) minus a third of nine D3aab (D3bba) elements.
 * s: the parity that sorts (i, j, p) (resp. (p, i)) into triplet order. */
typedef struct {
    const v2o_problem *p;
    int mode;
    const double *u;
    double *A;
    long row;
    int nt;
    map_term t[64];
} d3_row;

static void d3_add(d3_row *r, long col, double coef) {
    r->t[r->nt].col = col;
    r->t[r->nt].coef = coef;
    r->nt++;
}

static void d3_emit(d3_row *r) {
    if (r->mode == MODE_AU) {
        double dum = 0.0;
        for (int e = 0; e < r->nt; e++) dum += r->t[e].coef * r->u[r->t[e].col];
        r->A[r->row] = dum;
    } else {
        const double dum = r->u[r->row];
        for (int e = 0; e < r->nt; e++) r->A[r->t[e].col] += r->t[e].coef * dum;
    }
    r->row++;
    r->nt = 0;
}


static void d3_visit(const v2o_problem *p, long off, int mode, const double *u, double *A) {
    const int n = p->n, gaa = p->gaa, gab = p->gab;
    const long t3 = p->trip_aaa, ta = p->trip_aab;
    const double na = p->na, nb = p->nb;
    d3_row r;
    r.p = p; r.mode = mode; r.u = u; r.A = A; r.row = off; r.nt = 0;
    /* aa rows against D3aaa (and D3aab) for one spin */
    for (int fam = 0; fam < (p->sz ? 4 : 2); fam++) {
        const int beta = fam % 2;
        const long d2 = beta ? p->d2bb : p->d2aa;
        const long d3s = beta ? p->d3bbb : p->d3aaa, d3m = beta ? p->d3bba : p->d3aab;
        for (int ij = 0; ij < gaa; ij++) {
            const int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
            for (int kl = 0; kl < gaa; kl++) {
                const int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                if (p->sz && fam < 2) {          /* same-spin triples */
                    d3_add(&r, d2 + (long)ij * gaa + kl, (beta ? nb : na) - 2.0);
                    for (int q = 0; q < n; q++) {
                        if (i == q || j == q || k == q || l == q) continue;
                        const double sg = ((i < q && q < j) ? -1.0 : 1.0) * ((k < q && q < l) ? -1.0 : 1.0);
                        d3_add(&r, d3s + (long)D3_AAA(i, j, q) * t3 + D3_AAA(k, l, q), -sg);
                    }
                } else if (p->sz) {              /* mixed triples */
                    d3_add(&r, d2 + (long)ij * gaa + kl, beta ? na : nb);
                    for (int q = 0; q < n; q++)
                        d3_add(&r, d3m + (long)D3_AAB(i, j, q) * ta + D3_AAB(k, l, q), -1.0);
                } else {                         /* both */
                    d3_add(&r, d2 + (long)ij * gaa + kl, na + nb - 2.0);
                    for (int q = 0; q < n; q++) {
                        d3_add(&r, d3m + (long)D3_AAB(i, j, q) * ta + D3_AAB(k, l, q), -1.0);
                        if (i == q || j == q || k == q || l == q) continue;
                        const double sg = ((i < q && q < j) ? -1.0 : 1.0) * ((k < q && q < l) ? -1.0 : 1.0);
                        d3_add(&r, d3s + (long)D3_AAA(i, j, q) * t3 + D3_AAA(k, l, q), -sg);
                    }
                }
                d3_emit(&r);
            }
        }
    }
    /* ab rows */
    for (int fam = 0; fam < (p->sz ? 2 : 1); fam++) {
        for (int ij = 0; ij < gab; ij++) {
            const int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                const int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                const double c0 = !p->sz ? na + nb - 2.0 : (fam ? nb - 1.0 : na - 1.0);
                d3_add(&r, p->d2ab + (long)ij * gab + kl, c0);
                for (int q = 0; q < n; q++) {
                    if ((!p->sz || fam == 0) && i != q && k != q) {
                        const double sg = (q < i ? -1.0 : 1.0) * (q < k ? -1.0 : 1.0);
                        d3_add(&r, p->d3aab + (long)D3_AAB(i, q, j) * ta + D3_AAB(k, q, l), -sg);
                    }
                    if ((!p->sz || fam == 1) && j != q && l != q) {
                        const double sg = (q < j ? -1.0 : 1.0) * (q < l ? -1.0 : 1.0);
                        d3_add(&r, p->d3bba + (long)D3_AAB(j, q, i) * ta + D3_AAB(l, q, k), -sg);
                    }
                }
                d3_emit(&r);
            }
        }
    }
    if (p->spin && p->na == p->nb) {
        for (long e = 0; e < ta * ta; e++) {
            d3_add(&r, p->d3aab + e, 1.0);
            d3_add(&r, p->d3bba + e, -1.0);
            d3_emit(&r);
        }
        const double third = 1.0 / 3.0;
        for (int beta = 0; beta < 2; beta++) {
            const long d3s = beta ? p->d3bbb : p->d3aaa, d3m = beta ? p->d3bba : p->d3aab;
            for (long pqr = 0; pqr < t3; pqr++) {
                const int a = p->bas_aaa[3 * pqr], b = p->bas_aaa[3 * pqr + 1], c = p->bas_aaa[3 * pqr + 2];
                const long rows3[3] = {D3_AAB(a, b, c), D3_AAB(a, c, b), D3_AAB(b, c, a)};
                for (long stv = 0; stv < t3; stv++) {
                    const int s_ = p->bas_aaa[3 * stv], t_ = p->bas_aaa[3 * stv + 1], v_ = p->bas_aaa[3 * stv + 2];
                    const long cols3[3] = {D3_AAB(s_, t_, v_), D3_AAB(s_, v_, t_), D3_AAB(t_, v_, s_)};
                    d3_add(&r, d3s + pqr * t3 + stv, 1.0);
                    for (int x = 0; x < 3; x++)
                        for (int y = 0; y < 3; y++)
                            d3_add(&r, d3m + rows3[x] * ta + cols3[y], ((x + y) % 2) ? third : -third);
                    d3_emit(&r);
                }
            }
        }
    }
}

/* ------------------------------------------------------------- D4 ---- */
/* CONSTRAIN_D4 rows of d4.cc:44-297 (scatter :300-557): contractions of the
 * 4-RDM to the 3-RDM, each family present only when the electron counts
 * allow it.  A row: count x D3 element - sum_p (sign) D4 element, the sign
 * the parity of the positions p passes when inserted into the sets. */
static void d4_visit(const v2o_problem *p, long off, int mode, const double *u, double *A) {
    const int n = p->n;
    const long t3 = p->trip_aaa, ta = p->trip_aab;
    const long q4 = p->quad_aaaa, q31 = p->quad_aaab, q22 = p->quad_aabb;
    const double na = p->na, nb = p->nb;
    d3_row r;
    r.p = p; r.mode = mode; r.u = u; r.A = A; r.row = off; r.nt = 0;
#define I4(tab, a, b, c, d) (p->tab[(((long)(a) * n + (b)) * n + (c)) * n + (d)])
#define LT(q, x) ((q) < (x) ? -1.0 : 1.0)
    /* families in the reference's order: aaaa->aaa (d4.cc:48-85); aaab->aaa,
     * aaab->aab (:86-148); aabb->aab, aabb->bba (:149-199); bbba->bbb,
     * bbba->bba (:200-257); bbbb->bbb (:258-295) */
    for (int fam = 0; fam < 8; fam++) {
        int on;
        switch (fam) {
        case 0: on = p->na > 3; break;
        case 1: case 2: on = p->na > 2 && p->nb > 0; break;
        case 3: case 4: on = p->na > 1 && p->nb > 1; break;
        case 5: case 6: on = p->na > 0 && p->nb > 2; break;
        default: on = p->nb > 3; break;
        }
        if (!on) continue;
        const int rows_aaa = (fam == 0 || fam == 1 || fam == 5 || fam == 7);
        const long nr = rows_aaa ? t3 : ta;
        const int *tb = rows_aaa ? p->bas_aaa : p->bas_aab;
        for (long x = 0; x < nr; x++) {
            const int i = tb[3 * x], j = tb[3 * x + 1], k = tb[3 * x + 2];
            for (long y = 0; y < nr; y++) {
                const int l = tb[3 * y], m = tb[3 * y + 1], q = tb[3 * y + 2];
                const long e = x * nr + y;
                switch (fam) {
                case 0:
                case 7: {
                    d3_add(&r, (fam ? p->d3bbb : p->d3aaa) + e, fam ? nb - 3.0 : na - 3.0);
                    for (int s = 0; s < n; s++) {
                        if (s == i || s == j || s == k || s == l || s == m || s == q) continue;
                        const double sg = LT(s, i) * LT(s, j) * LT(s, k) * LT(s, l) * LT(s, m) * LT(s, q);
                        d3_add(&r, (fam ? p->d4bbbb : p->d4aaaa) + (long)I4(ibas_aaaa, i, j, k, s) * q4
                                   + I4(ibas_aaaa, l, m, q, s), -sg);
                    }
                    break;
                }
                case 1:
                case 5:
                    d3_add(&r, (fam == 5 ? p->d3bbb : p->d3aaa) + e, fam == 5 ? na : nb);
                    for (int s = 0; s < n; s++)
                        d3_add(&r, (fam == 5 ? p->d4bbba : p->d4aaab) + (long)I4(ibas_aaab, i, j, k, s) * q31
                                   + I4(ibas_aaab, l, m, q, s), -1.0);
                    break;
                case 2:
                case 6:
                    d3_add(&r, (fam == 6 ? p->d3bba : p->d3aab) + e, fam == 6 ? nb - 2.0 : na - 2.0);
                    for (int s = 0; s < n; s++) {
                        if (s == i || s == j || s == l || s == m) continue;
                        const double sg = LT(s, i) * LT(s, j) * LT(s, l) * LT(s, m);
                        d3_add(&r, (fam == 6 ? p->d4bbba : p->d4aaab) + (long)I4(ibas_aaab, i, j, s, k) * q31
                                   + I4(ibas_aaab, l, m, s, q), -sg);
                    }
                    break;
                case 3:
                    d3_add(&r, p->d3aab + e, nb - 1.0);
                    for (int s = 0; s < n; s++) {
                        if (s == k || s == q) continue;
                        d3_add(&r, p->d4aabb + (long)I4(ibas_aabb, i, j, k, s) * q22 + I4(ibas_aabb, l, m, q, s),
                               -(LT(s, k) * LT(s, q)));
                    }
                    break;
                case 4:
                    d3_add(&r, p->d3bba + e, na - 1.0);
                    for (int s = 0; s < n; s++) {
                        if (s == k || s == q) continue;
                        d3_add(&r, p->d4aabb + (long)I4(ibas_aabb, k, s, i, j) * q22 + I4(ibas_aabb, q, s, l, m),
                               -(LT(s, k) * LT(s, q)));
                    }
                    break;
                }
                d3_emit(&r);
            }
        }
    }
#undef I4
#undef LT
}

/* ------------------------------------------------------------- A.x ---- */
/* v2rdm_solver.cc:2995-3050 (bpsdp_Au) -> d2.cc:314-594, spin.cc:276-508,
 * q2.cc:170-318, g2.cc:245-442 */
void v2o_Au(const v2o_problem *p, const double *u, double *A) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    double na = p->na, nb = p->nb;
    long off = 0;
    memset(A, 0, sizeof(double) * p->n_dual);

    /* d2.cc:314-378 traces */
    if (p->sz) {
        double s = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) { int ij = IAB(p, i, j); s += u[p->d2ab + (long)ij * gab + ij]; }
        A[off++] = s;
        s = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (i == j || gaa == 0) continue;
                int ij = IAA(p, i, j); s += u[p->d2aa + (long)ij * gaa + ij];
            }
        A[off++] = s;
        s = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (i == j || gaa == 0) continue;
                int ij = IAA(p, i, j); s += u[p->d2bb + (long)ij * gaa + ij];
            }
        A[off++] = s;
    } else {
        double s = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int ij = IAB(p, i, j);
                s += 2.0 * u[p->d2ab + (long)ij * gab + ij];
                if (i == j || gaa == 0) continue;
                ij = IAA(p, i, j);
                s += u[p->d2aa + (long)ij * gaa + ij];
                s += u[p->d2bb + (long)ij * gaa + ij];
            }
        A[off++] = s;
    }
    /* d2.cc:380-414 hermiticity */
    const long hb[3] = {p->d2aa, p->d2bb, p->d2ab};
    const int hg[3] = {gaa, gaa, gab};
    for (int s = 0; s < 3; s++)
        for (long ij = 0; ij < hg[s]; ij++)
            for (long kl = 0; kl < hg[s]; kl++) {
                double dum = u[hb[s] + ij * hg[s] + kl];
                dum -= u[hb[s] + kl * hg[s] + ij];
                A[off++] = dum;
            }
    /* d2.cc:416-435 D1 + Q1 */
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) A[off + i * n + j] = u[p->d1a + j * n + i] + u[p->q1a + i * n + j];
    off += (long)n * n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) A[off + i * n + j] = u[p->d1b + j * n + i] + u[p->q1b + i * n + j];
    off += (long)n * n;
    /* d2.cc:441-591 partial traces */
    if (!p->sz) {
        double nt = na + nb;
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    double sum = (nt - 1.0) * u[d1 + i * n + j];
                    for (int k = 0; k < n; k++) {
                        int ik = s ? IAB(p, k, i) : IAB(p, i, k);
                        int jk = s ? IAB(p, k, j) : IAB(p, j, k);
                        sum -= u[p->d2ab + (long)ik * gab + jk];
                    }
                    for (int k = 0; k < n; k++) {
                        if (i == k || j == k) continue;
                        int ik = IAA(p, i, k), jk = IAA(p, j, k);
                        int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                        sum -= sik * sjk * u[d2 + (long)ik * gaa + jk];
                    }
                    A[off + i * n + j] = sum;
                }
            off += (long)n * n;
        }
    } else {
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a;
            double f = s ? na : nb;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    double sum = f * u[d1 + i * n + j];
                    for (int k = 0; k < n; k++) {
                        int ik = s ? IAB(p, k, i) : IAB(p, i, k);
                        int jk = s ? IAB(p, k, j) : IAB(p, j, k);
                        sum -= u[p->d2ab + (long)ik * gab + jk];
                    }
                    A[off + i * n + j] = sum;
                }
            off += (long)n * n;
        }
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa;
            double f = s ? (nb - 1.0) : (na - 1.0);
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    double sum = f * u[d1 + i * n + j];
                    for (int k = 0; k < n; k++) {
                        if (i == k || j == k) continue;
                        int ik = IAA(p, i, k), jk = IAA(p, j, k);
                        int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                        sum -= sik * sjk * u[d2 + (long)ik * gaa + jk];
                    }
                    A[off + i * n + j] = sum;
                }
            off += (long)n * n;
        }
    }

    if (p->spin) {
        /* spin.cc:279-290  <S^2> row */
        double s2 = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) s2 += u[p->d2ab + (long)IAB(p, i, j) * gab + IAB(p, j, i)];
        A[off++] = s2;
        if (p->na == p->nb) {
            /* spin.cc:320-393 singlet rows */
            for (long r = 0; r < (long)n * n; r++) { A[off + r] = u[p->d1a + r]; A[off + r] += -1.0 * u[p->d1b + r]; }
            off += (long)n * n;
            for (long r = 0; r < (long)gaa * gaa; r++) { A[off + r] = u[p->d2aa + r]; A[off + r] += -1.0 * u[p->d2bb + r]; }
            off += (long)gaa * gaa;
            for (int s = 0; s < 2; s++) {
                long d2 = s ? p->d2bb : p->d2aa;
                for (long r = 0; r < (long)gaa * gaa; r++) A[off + r] = u[d2 + r];
                for (int ij = 0; ij < gaa; ij++) {
                    int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
                    long ijb = IAB(p, i, j), jib = IAB(p, j, i);
                    for (int kl = 0; kl < gaa; kl++) {
                        int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                        long klb = IAB(p, k, l), lkb = IAB(p, l, k);
                        double *a = &A[off + (long)ij * gaa + kl];
                        *a -= 0.5 * u[p->d2ab + ijb * gab + klb];
                        *a += 0.5 * u[p->d2ab + jib * gab + klb];
                        *a += 0.5 * u[p->d2ab + ijb * gab + lkb];
                        *a -= 0.5 * u[p->d2ab + jib * gab + lkb];
                    }
                }
                off += (long)gaa * gaa;
            }
            for (long r = 0; r < (long)gab * gab; r++) A[off + r] = u[p->d200 + r];
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double *a = &A[off + (long)ij * gab + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + (long)ij * gab + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + ji * gab + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + (long)ij * gab + lk];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + ji * gab + lk];
                }
            }
            off += (long)gab * gab;
            for (long r = 0; r < (long)gab * gab; r++) A[off + r] += 1.0 * u[p->d2ab + r];
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    A[off + (long)ij * gab + kl] -= u[p->d2ab + ji * gab + lk];
                }
            }
            off += (long)gab * gab;
        } else {
            /* spin.cc:411-485 non-singlet 2gab x 2gab block */
            long w = 2L * gab;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double *a = &A[off + (long)ij * w + kl];
                    *a += u[p->d200 + (long)ij * w + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + (long)ij * gab + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + ji * gab + kl];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + (long)ij * gab + lk];
                    *a -= 0.5 / (dij * dkl) * u[p->d2ab + ji * gab + lk];
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double *a = &A[off + (long)ij * w + (kl + gab)];
                    *a += u[p->d200 + (long)ij * w + (kl + gab)];
                    *a -= 0.5 / dij * u[p->d2ab + (long)ij * gab + kl];
                    *a += 0.5 / dij * u[p->d2ab + (long)ij * gab + lk];
                    *a -= 0.5 / dij * u[p->d2ab + ji * gab + kl];
                    *a += 0.5 / dij * u[p->d2ab + ji * gab + lk];
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double *a = &A[off + (ij + gab) * w + kl];
                    *a += u[p->d200 + (ij + gab) * w + kl];
                    *a -= 0.5 / dkl * u[p->d2ab + (long)ij * gab + kl];
                    *a -= 0.5 / dkl * u[p->d2ab + (long)ij * gab + lk];
                    *a += 0.5 / dkl * u[p->d2ab + ji * gab + kl];
                    *a += 0.5 / dkl * u[p->d2ab + ji * gab + lk];
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double *a = &A[off + (ij + gab) * w + (kl + gab)];
                    *a += u[p->d200 + (ij + gab) * w + (kl + gab)];
                    *a -= 0.5 * u[p->d2ab + (long)ij * gab + kl];
                    *a += 0.5 * u[p->d2ab + ji * gab + kl];
                    *a += 0.5 * u[p->d2ab + (long)ij * gab + lk];
                    *a -= 0.5 * u[p->d2ab + ji * gab + lk];
                }
            }
            off += 4L * gab * gab;
        }
        if (p->g2) {
            /* spin.cc:487-507 maximal-spin rows on G2ba */
            for (int kl = 0; kl < gab; kl++) {
                double dum = 0.0;
                for (int i = 0; i < n; i++) dum += u[p->g2ba + (long)kl * gab + IAB(p, i, i)];
                A[off + kl] = dum;
            }
            off += gab;
            for (int kl = 0; kl < gab; kl++) {
                double dum = 0.0;
                for (int i = 0; i < n; i++) dum += u[p->g2ba + (long)IAB(p, i, i) * gab + kl];
                A[off + kl] = dum;
            }
            off += gab;
        }
    }

    if (p->q2) {
        /* q2.cc:170-216 Q2ab */
        for (long r = 0; r < (long)gab * gab; r++) { A[off + r] = u[p->d2ab + r]; A[off + r] += -1.0 * u[p->q2ab + r]; }
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int k = 0; k < n; k++) A[off + (long)ij * gab + IAB(p, k, j)] -= u[p->d1a + k * n + i];
            for (int l = 0; l < n; l++) A[off + (long)ij * gab + IAB(p, i, l)] -= u[p->d1b + l * n + j];
        }
        off += (long)gab * gab;
        /* q2.cc:218-318 Q2aa / Q2bb */
        for (int s = 0; s < 2; s++) {
            long d2 = s ? p->d2bb : p->d2aa, q2 = s ? p->q2bb : p->q2aa, d1 = s ? p->d1b : p->d1a;
            for (long r = 0; r < (long)gaa * gaa; r++) { A[off + r] = u[d2 + r]; A[off + r] += -1.0 * u[q2 + r]; }
            for (int ij = 0; ij < gaa; ij++) {
                int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                    double dum = 0.0;
                    if (j == l) dum -= u[d1 + k * n + i];
                    if (j == k) dum += u[d1 + l * n + i];
                    if (i == l) dum += u[d1 + k * n + j];
                    if (i == k) dum -= u[d1 + l * n + j];
                    A[off + (long)ij * gaa + kl] += dum;
                }
            }
            off += (long)gaa * gaa;
        }
    }

    if (p->g2) {
        /* g2.cc:245-312 G2ab / G2ba */
        for (int s = 0; s < 2; s++) {
            long g = s ? p->g2ba : p->g2ab, d1 = s ? p->d1b : p->d1a;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    double dum = -u[g + (long)ij * gab + kl];
                    if (j == l) dum += u[d1 + i * n + k];
                    if (s == 0) dum -= u[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, k, j)];
                    else dum -= u[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, j, k)];
                    A[off + (long)ij * gab + kl] = dum;
                }
            }
            off += (long)gab * gab;
        }
        /* g2.cc:313-440 G2 aaaa / bbbb / aabb / bbaa */
        long g = p->g2aa, w = 2L * gab;
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa, sh = s ? gab : 0;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    double dum = -u[g + (sh + ij) * w + (sh + kl)];
                    if (j == l) dum += u[d1 + i * n + k];
                    if (i != l && k != j) {
                        int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                        dum -= u[d2 + (long)IAA(p, i, l) * gaa + IAA(p, k, j)] * sil * skj;
                    }
                    A[off + (sh + ij) * w + (sh + kl)] = dum;
                }
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = -u[g + (long)ij * w + (gab + kl)];
                dum += u[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, j, k)];
                A[off + (long)ij * w + (gab + kl)] = dum;
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = -u[g + (gab + ij) * w + kl];
                dum += u[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, k, j)];
                A[off + (gab + ij) * w + kl] = dum;
            }
        }
        off += 4L * gab * gab;
    }
    if (p->t1) {   /* v2rdm_solver.cc:3015-3017 */
        t1_visit(p, off, MODE_AU, u, A, NULL);
        off += 2L * p->trip_aab * p->trip_aab + 2L * p->trip_aaa * p->trip_aaa;
    }
    if (p->t2) {   /* v2rdm_solver.cc:3019-3022 */
        t2_visit(p, off, MODE_AU, u, A, NULL);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->e3) {   /* v2rdm_solver.cc:3024-3026 */
        e3_visit(p, off, MODE_AU, u, A);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->f3) {   /* v2rdm_solver.cc:3028-3030 */
        f3_visit(p, off, MODE_AU, u, A);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->q3) {   /* v2rdm_solver.cc:3032-3034 */
        t1_like_visit(p, off, MODE_AU, u, A, NULL, 1);
        off += 2L * p->trip_aab * p->trip_aab + 2L * p->trip_aaa * p->trip_aaa;
    }
    if (p->d3) {   /* v2rdm_solver.cc:3036-3038 */
        d3_visit(p, off, MODE_AU, u, A);
        off += d3_rows_count(p);
    }
    if (p->d4) d4_visit(p, off, MODE_AU, u, A);   /* v2rdm_solver.cc:3040-3042 */
}

/* ----------------------------------------------------------- A^T.y ---- */
/* v2rdm_solver.cc:3054-3108 (bpsdp_ATu) -> d2.cc:46-311, spin.cc:46-273,
 * q2.cc:320-438, g2.cc:444-634; same scatter order as the reference */
void v2o_ATu(const v2o_problem *p, const double *u, double *A) {
    int n = p->n, gab = p->gab, gaa = p->gaa;
    double na = p->na, nb = p->nb;
    long off = 0;
    memset(A, 0, sizeof(double) * p->n_primal);

    if (p->sz) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) { int ij = IAB(p, i, j); A[p->d2ab + (long)ij * gab + ij] += u[off]; }
        off++;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (i == j || gaa == 0) continue;
                int ij = IAA(p, i, j); A[p->d2aa + (long)ij * gaa + ij] += u[off];
            }
        off++;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (i == j || gaa == 0) continue;
                int ij = IAA(p, i, j); A[p->d2bb + (long)ij * gaa + ij] += u[off];
            }
        off++;
    } else {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int ij = IAB(p, i, j);
                A[p->d2ab + (long)ij * gab + ij] += 2.0 * u[off];
                if (i == j || gaa == 0) continue;
                ij = IAA(p, i, j);
                A[p->d2aa + (long)ij * gaa + ij] += u[off];
                A[p->d2bb + (long)ij * gaa + ij] += u[off];
            }
        off++;
    }
    const long hb[3] = {p->d2aa, p->d2bb, p->d2ab};
    const int hg[3] = {gaa, gaa, gab};
    for (int s = 0; s < 3; s++)
        for (long ij = 0; ij < hg[s]; ij++)
            for (long kl = 0; kl < hg[s]; kl++) {
                double dum = u[off];
                A[hb[s] + ij * hg[s] + kl] += dum;
                A[hb[s] + kl * hg[s] + ij] -= dum;
                off++;
            }
    for (int s = 0; s < 2; s++) {
        long d1 = s ? p->d1b : p->d1a, q1 = s ? p->q1b : p->q1a;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double dum = u[off + i * n + j];
                A[d1 + j * n + i] += dum;
                A[q1 + i * n + j] += dum;
            }
        off += (long)n * n;
    }
    if (!p->sz) {
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    A[d1 + i * n + j] += (na + nb - 1.0) * u[off + i * n + j];
                    for (int k = 0; k < n; k++) {
                        int ik = s ? IAB(p, k, i) : IAB(p, i, k);
                        int jk = s ? IAB(p, k, j) : IAB(p, j, k);
                        A[p->d2ab + (long)ik * gab + jk] -= u[off + i * n + j];
                    }
                    for (int k = 0; k < n; k++) {
                        if (i == k || j == k) continue;
                        int ik = IAA(p, i, k), jk = IAA(p, j, k);
                        int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                        A[d2 + (long)ik * gaa + jk] -= sik * sjk * u[off + i * n + j];
                    }
                }
            off += (long)n * n;
        }
    } else {
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a;
            double f = s ? na : nb;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    A[d1 + i * n + j] += f * u[off + i * n + j];
                    for (int k = 0; k < n; k++) {
                        int ik = s ? IAB(p, k, i) : IAB(p, i, k);
                        int jk = s ? IAB(p, k, j) : IAB(p, j, k);
                        A[p->d2ab + (long)ik * gab + jk] -= u[off + i * n + j];
                    }
                }
            off += (long)n * n;
        }
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa;
            double f = s ? (nb - 1.0) : (na - 1.0);
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    A[d1 + i * n + j] += f * u[off + i * n + j];
                    for (int k = 0; k < n; k++) {
                        if (i == k || j == k) continue;
                        int ik = IAA(p, i, k), jk = IAA(p, j, k);
                        int sik = i < k ? 1 : -1, sjk = j < k ? 1 : -1;
                        A[d2 + (long)ik * gaa + jk] -= sik * sjk * u[off + i * n + j];
                    }
                }
            off += (long)n * n;
        }
    }

    if (p->spin) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) A[p->d2ab + (long)IAB(p, i, j) * gab + IAB(p, j, i)] += u[off];
        off++;
        if (p->na == p->nb) {
            for (long r = 0; r < (long)n * n; r++) A[p->d1a + r] += 1.0 * u[off + r];
            for (long r = 0; r < (long)n * n; r++) A[p->d1b + r] += -1.0 * u[off + r];
            off += (long)n * n;
            for (long r = 0; r < (long)gaa * gaa; r++) A[p->d2aa + r] += 1.0 * u[off + r];
            for (long r = 0; r < (long)gaa * gaa; r++) A[p->d2bb + r] += -1.0 * u[off + r];
            off += (long)gaa * gaa;
            for (int s = 0; s < 2; s++) {
                long d2 = s ? p->d2bb : p->d2aa;
                for (long r = 0; r < (long)gaa * gaa; r++) A[d2 + r] += 1.0 * u[off + r];
                for (int ij = 0; ij < gaa; ij++) {
                    int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
                    long ijb = IAB(p, i, j), jib = IAB(p, j, i);
                    for (int kl = 0; kl < gaa; kl++) {
                        int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                        long klb = IAB(p, k, l), lkb = IAB(p, l, k);
                        double v = u[off + (long)ij * gaa + kl];
                        A[p->d2ab + ijb * gab + klb] -= 0.5 * v;
                        A[p->d2ab + jib * gab + klb] += 0.5 * v;
                        A[p->d2ab + ijb * gab + lkb] += 0.5 * v;
                        A[p->d2ab + jib * gab + lkb] -= 0.5 * v;
                    }
                }
                off += (long)gaa * gaa;
            }
            for (long r = 0; r < (long)gab * gab; r++) A[p->d200 + r] += 1.0 * u[off + r];
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double v = u[off + (long)ij * gab + kl];
                    A[p->d2ab + (long)ij * gab + kl] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + ji * gab + kl] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + (long)ij * gab + lk] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + ji * gab + lk] -= 0.5 / (dij * dkl) * v;
                }
            }
            off += (long)gab * gab;
            for (long r = 0; r < (long)gab * gab; r++) A[p->d2ab + r] += 1.0 * u[off + r];
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    A[p->d2ab + ji * gab + lk] -= u[off + (long)ij * gab + kl];
                }
            }
            off += (long)gab * gab;
        } else {
            long w = 2L * gab;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double v = u[off + (long)ij * w + kl];
                    A[p->d200 + (long)ij * w + kl] += v;
                    A[p->d2ab + (long)ij * gab + kl] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + ji * gab + kl] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + (long)ij * gab + lk] -= 0.5 / (dij * dkl) * v;
                    A[p->d2ab + ji * gab + lk] -= 0.5 / (dij * dkl) * v;
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                double dij = (i == j) ? sqrt(2.0) : 1.0;
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double v = u[off + (long)ij * w + (kl + gab)];
                    A[p->d200 + (long)ij * w + (kl + gab)] += v;
                    A[p->d2ab + (long)ij * gab + kl] -= 0.5 / dij * v;
                    A[p->d2ab + (long)ij * gab + lk] += 0.5 / dij * v;
                    A[p->d2ab + ji * gab + kl] -= 0.5 / dij * v;
                    A[p->d2ab + ji * gab + lk] += 0.5 / dij * v;
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double dkl = (k == l) ? sqrt(2.0) : 1.0;
                    double v = u[off + (ij + gab) * w + kl];
                    A[p->d200 + (ij + gab) * w + kl] += v;
                    A[p->d2ab + (long)ij * gab + kl] -= 0.5 / dkl * v;
                    A[p->d2ab + (long)ij * gab + lk] -= 0.5 / dkl * v;
                    A[p->d2ab + ji * gab + kl] += 0.5 / dkl * v;
                    A[p->d2ab + ji * gab + lk] += 0.5 / dkl * v;
                }
            }
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                long ji = IAB(p, j, i);
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    long lk = IAB(p, l, k);
                    double v = u[off + (ij + gab) * w + (kl + gab)];
                    A[p->d200 + (ij + gab) * w + (kl + gab)] += v;
                    A[p->d2ab + (long)ij * gab + kl] -= 0.5 * v;
                    A[p->d2ab + ji * gab + kl] += 0.5 * v;
                    A[p->d2ab + (long)ij * gab + lk] += 0.5 * v;
                    A[p->d2ab + ji * gab + lk] -= 0.5 * v;
                }
            }
            off += 4L * gab * gab;
        }
        if (p->g2) {
            for (int kl = 0; kl < gab; kl++) {
                double dum = u[off + kl];
                for (int i = 0; i < n; i++) A[p->g2ba + (long)kl * gab + IAB(p, i, i)] += dum;
            }
            off += gab;
            for (int kl = 0; kl < gab; kl++) {
                double dum = u[off + kl];
                for (int i = 0; i < n; i++) A[p->g2ba + (long)IAB(p, i, i) * gab + kl] += dum;
            }
            off += gab;
        }
    }

    if (p->q2) {
        for (long r = 0; r < (long)gab * gab; r++) A[p->d2ab + r] += 1.0 * u[off + r];
        for (long r = 0; r < (long)gab * gab; r++) A[p->q2ab + r] += -1.0 * u[off + r];
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double v = u[off + (long)ij * gab + kl];
                if (j == l) A[p->d1a + k * n + i] -= v;
                if (i == k) A[p->d1b + l * n + j] -= v;
            }
        }
        off += (long)gab * gab;
        for (int s = 0; s < 2; s++) {
            long d2 = s ? p->d2bb : p->d2aa, q2 = s ? p->q2bb : p->q2aa, d1 = s ? p->d1b : p->d1a;
            for (long r = 0; r < (long)gaa * gaa; r++) A[d2 + r] += 1.0 * u[off + r];
            for (long r = 0; r < (long)gaa * gaa; r++) A[q2 + r] += -1.0 * u[off + r];
            for (int ij = 0; ij < gaa; ij++) {
                int i = p->bas_aa[2 * ij], j = p->bas_aa[2 * ij + 1];
                for (int kl = 0; kl < gaa; kl++) {
                    int k = p->bas_aa[2 * kl], l = p->bas_aa[2 * kl + 1];
                    double v = u[off + (long)ij * gaa + kl];
                    if (j == l) A[d1 + k * n + i] -= v;
                    if (j == k) A[d1 + l * n + i] += v;
                    if (i == l) A[d1 + k * n + j] += v;
                    if (i == k) A[d1 + l * n + j] -= v;
                }
            }
            off += (long)gaa * gaa;
        }
    }

    if (p->g2) {
        for (int s = 0; s < 2; s++) {
            long g = s ? p->g2ba : p->g2ab, d1 = s ? p->d1b : p->d1a;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    double dum = u[off + (long)ij * gab + kl];
                    A[g + (long)ij * gab + kl] -= dum;
                    if (j == l) A[d1 + i * n + k] += dum;
                    if (s == 0) A[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, k, j)] -= dum;
                    else A[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, j, k)] -= dum;
                }
            }
            off += (long)gab * gab;
        }
        long g = p->g2aa, w = 2L * gab;
        for (int s = 0; s < 2; s++) {
            long d1 = s ? p->d1b : p->d1a, d2 = s ? p->d2bb : p->d2aa, sh = s ? gab : 0;
            for (int ij = 0; ij < gab; ij++) {
                int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
                for (int kl = 0; kl < gab; kl++) {
                    int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                    double dum = u[off + (sh + ij) * w + (sh + kl)];
                    A[g + (sh + ij) * w + (sh + kl)] -= dum;
                    if (j == l) A[d1 + i * n + k] += dum;
                    if (i != l && k != j) {
                        int sil = i < l ? 1 : -1, skj = k < j ? 1 : -1;
                        A[d2 + (long)IAA(p, i, l) * gaa + IAA(p, k, j)] -= dum * sil * skj;
                    }
                }
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = u[off + (long)ij * w + (kl + gab)];
                A[g + (long)ij * w + (kl + gab)] -= dum;
                A[p->d2ab + (long)IAB(p, i, l) * gab + IAB(p, j, k)] += dum;
            }
        }
        for (int ij = 0; ij < gab; ij++) {
            int i = p->bas_ab[2 * ij], j = p->bas_ab[2 * ij + 1];
            for (int kl = 0; kl < gab; kl++) {
                int k = p->bas_ab[2 * kl], l = p->bas_ab[2 * kl + 1];
                double dum = u[off + (gab + ij) * w + kl];
                A[g + (gab + ij) * w + kl] -= dum;
                A[p->d2ab + (long)IAB(p, l, i) * gab + IAB(p, k, j)] += dum;
            }
        }
        off += 4L * gab * gab;
    }
    if (p->t1) {   /* v2rdm_solver.cc:3073-3075 */
        t1_visit(p, off, MODE_ATU, u, A, NULL);
        off += 2L * p->trip_aab * p->trip_aab + 2L * p->trip_aaa * p->trip_aaa;
    }
    if (p->t2) {   /* v2rdm_solver.cc:3077-3080 */
        t2_visit(p, off, MODE_ATU, u, A, NULL);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->e3) {   /* v2rdm_solver.cc:3082-3084 */
        e3_visit(p, off, MODE_ATU, u, A);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->f3) {   /* v2rdm_solver.cc:3086-3088 */
        f3_visit(p, off, MODE_ATU, u, A);
        const long w = (long)p->trip_aab + p->trip_aba;
        off += 2L * p->trip_aab * p->trip_aab + 2 * w * w;
    }
    if (p->q3) {   /* v2rdm_solver.cc:3090-3092 */
        t1_like_visit(p, off, MODE_ATU, u, A, NULL, 1);
        off += 2L * p->trip_aab * p->trip_aab + 2L * p->trip_aaa * p->trip_aaa;
    }
    if (p->d3) {   /* v2rdm_solver.cc:3094-3096 */
        d3_visit(p, off, MODE_ATU, u, A);
        off += d3_rows_count(p);
    }
    if (p->d4) d4_visit(p, off, MODE_ATU, u, A);   /* v2rdm_solver.cc:3098-3100 */
}
