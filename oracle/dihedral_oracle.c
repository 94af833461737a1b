/*
 * dihedral_oracle.c -- CPU restatement of the dihedral (8-fold) task
 * decomposition that n_queens_b200's nq_count_dihedral runs on the GPU.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/ through oracle/__init__.py; the
 * product library never links, calls or falls back to it.
 *
 * The reference counts only the left-right mirror (row 0 restricted to the
 * left half, every prefix counted twice: src/n_queens.cpp:74-113 and the x2 of
 * src/n_queens_cuda.cu:181-183).  This decomposition uses all eight
 * symmetries of the square.  Its totals are checked against the reference's
 * own totals (README.md:16-25, logs/5090.log, and oracle/_ref), so the
 * restatement below is pinned by the reference's outputs, not by its code.
 *
 * Every solution falls in exactly one family:
 *
 *  corner   a queen at (0,0).  Transposition maps such a solution to another
 *           one (never to itself: a transposed pair (i,j),(j,i) shares an
 *           anti-diagonal), rotations move the corner.  Keep the one whose
 *           row-1 queen column B1 is below the row of its column-1 queen:
 *           with B1 < k the prefix forbids column 1 in rows 2..B1-1 (weight
 *           8); with B1 >= k both the solution and its transpose have B1 and
 *           that row >= k, the prefix forbids column 1 in rows 2..k-1 and
 *           each is counted with weight 4.
 *  class m  (1 <= m <= k-1, m < (N-1)/2) the border queen nearest to a
 *           corner is at distance m, and the queen (0,m) represents it: rows
 *           1..m-1 hold no queen in column 0 or N-1, rows below B2 = N-1-m
 *           neither, and the row N-1 queen lies in [m, N-1-m].  Ties: the
 *           other cells at distance m that (0,m) does not attack are
 *           X1=(m,N-1), X2=(B2,0), X3=(N-1,N-1-m); a quarter turn cycles
 *           (0,m) -> X1 -> X3 -> X2.  Among the nearest border queens pick
 *           those whose quarter-turn successor cell is empty (all four when
 *           every cell is taken); the canonical ones then have X1 empty
 *           (or all four taken), and the weight is 8/(number picked):
 *             X1 empty:  8, or 4 when X3 is taken and X2 empty;
 *             all four:  2.
 *           The half turn pairs {X1 empty, X2, X3 taken} with {X1, X3 taken,
 *           X2 empty}, which turns the X2-dependent part into two counts of
 *           X1-taken prefixes, so no solution needs X2 at all:
 *             x1=0 prefixes: weight 8, or 4 when the row N-1 queen is at X3;
 *             x1=1 prefixes, copy A (side columns barred below B2, row N-1
 *               queen at X3): weight 2;
 *             x1=1 prefixes, copy B (side columns barred from row B2 on,
 *               row N-1 queen at X3): weight 2.
 *  rest     every border queen at distance >= k.  Only the left-right mirror
 *           and the top-bottom flip are used: the top queen (0,a), a in
 *           [k, (N-1)/2), no side-column queen in rows 1..k-1 or below
 *           N-1-k, the row N-1 queen in [a, N-1-a]; weight 4, or 2 when the
 *           row N-1 queen is at N-1-a (same distance as the top one).
 *
 * Below the prefix a task's search follows three rules only: rows beyond
 * `side_row` may not use column 0 or N-1, row N-1 is masked by `last_mask`,
 * and a completion weighs `w_tie` when its row N-1 queen is `tie_bit`, else
 * `w`.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t side_row;
    uint32_t last_mask, tie_bit, w, w_tie;
} dih_class_t;

typedef struct {
    int N, k;
    uint32_t full, side;
    dih_class_t *cls;
    int ncls, cap_cls;
    uint32_t *c, *l, *r;
    uint8_t *t;
    int64_t n, cap;
} dih_ctx_t;

enum { FAM_CORNER_LOW, FAM_CORNER_HIGH, FAM_M0, FAM_M1, FAM_REST };

typedef struct {
    int fam, m, b1;
    int cls;
} dih_walk_t;

/* Columns row `row` (1 <= row <= k-1) of a prefix may use in family `fam`. */
static uint32_t prefix_allowed(const dih_ctx_t *x, const dih_walk_t *w, int row) {
    uint32_t a = x->full;
    const dih_class_t *c = &x->cls[w->cls];
    switch (w->fam) {
        case FAM_CORNER_LOW:
            if (row == 1) a &= ((1u << x->k) - 1u) & ~3u; /* B1 in [2, k-1] */
            else if (row < w->b1) a &= ~2u;
            break;
        case FAM_CORNER_HIGH:
            if (row == 1) a &= ~((1u << x->k) - 1u); /* B1 >= k */
            else a &= ~2u;
            break;
        case FAM_M0:
            if (row <= w->m) a &= ~x->side;
            break;
        case FAM_M1:
            if (row < w->m) a &= ~x->side;
            else if (row == w->m) a &= 1u << (x->N - 1);
            break;
        case FAM_REST:
            a &= ~x->side;
            break;
    }
    if (row > c->side_row) a &= ~x->side;
    return a;
}

static void emit(dih_ctx_t *x, uint32_t c, uint32_t l, uint32_t r, int cls) {
    if (x->n < x->cap) {
        x->c[x->n] = c;
        x->l[x->n] = l;
        x->r[x->n] = r;
        x->t[x->n] = (uint8_t)cls;
    }
    x->n++;
}

static void walk(dih_ctx_t *x, dih_walk_t *w, uint32_t c, uint32_t l, uint32_t r, int row) {
    if (row == x->k) {
        emit(x, c, l, r, w->cls);
        return;
    }
    uint32_t f = prefix_allowed(x, w, row) & ~(c | l | r);
    while (f) {
        uint32_t p = f & (0u - f);
        f ^= p;
        const int save = w->b1;
        if (row == 1) w->b1 = __builtin_ctz(p);
        walk(x, w, c | p, (l | p) << 1, (r | p) >> 1, row + 1);
        w->b1 = save;
    }
}

static int add_class(dih_ctx_t *x, int side_row, uint32_t last_mask, uint32_t tie_bit, uint32_t wt, uint32_t wt_tie) {
    if (x->ncls < x->cap_cls) {
        dih_class_t *c = &x->cls[x->ncls];
        c->side_row = side_row;
        c->last_mask = last_mask;
        c->tie_bit = tie_bit;
        c->w = wt;
        c->w_tie = wt_tie;
    }
    return x->ncls++;
}

static uint32_t middle(int N, int a) { /* columns [a, N-1-a] */
    return ((1u << (N - a)) - 1u) & ~((1u << a) - 1u);
}

static void root(dih_ctx_t *x, dih_walk_t *w, int col) {
    const uint32_t p = 1u << col;
    w->b1 = 0;
    walk(x, w, p, p << 1, p >> 1, 1);
}

/* Expands the decomposition for (N, k); returns the task count (at most cap
 * tasks and cap_cls classes are written), -1 for a bad argument.  Classes are
 * numbered in creation order; every class is created even when it gets no
 * task, so the class table depends on (N, k) only. */
int64_t nq_oracle_dihedral_expand(int N, int k, uint32_t *cols, uint32_t *ld, uint32_t *rd, uint8_t *cls,
                                  int64_t cap, dih_class_t *table, int cap_cls, int *n_cls) {
    if (N < 4 || N > 31 || k < 2 || k > N - 2) return -1;
    dih_ctx_t x;
    memset(&x, 0, sizeof(x));
    x.N = N;
    x.k = k;
    x.full = (1u << N) - 1u;
    x.side = 1u | (1u << (N - 1));
    x.c = cols;
    x.l = ld;
    x.r = rd;
    x.t = cls;
    x.cap = cap;
    dih_class_t scratch[64];
    x.cls = scratch;
    x.cap_cls = 64;
    const int M = (N - 2) / 2; /* largest m with 2m < N-1 */
    dih_walk_t w;
    memset(&w, 0, sizeof(w));

    w.fam = FAM_CORNER_LOW;
    w.cls = add_class(&x, N, x.full, 0, 8, 8);
    root(&x, &w, 0);
    w.fam = FAM_CORNER_HIGH;
    w.cls = add_class(&x, N, x.full, 0, 4, 4);
    root(&x, &w, 0);
    for (int m = 1; m <= k - 1 && m <= M; ++m) {
        const int b2 = N - 1 - m;
        const uint32_t x3 = 1u << (N - 1 - m);
        w.m = m;
        w.fam = FAM_M0;
        w.cls = add_class(&x, b2, middle(N, m) & ~x.side, x3, 8, 4);
        root(&x, &w, m);
        w.fam = FAM_M1;
        w.cls = add_class(&x, b2, x3, x3, 2, 2);
        root(&x, &w, m);
        w.cls = add_class(&x, b2 - 1, x3, x3, 2, 2);
        root(&x, &w, m);
    }
    for (int a = k; a <= M; ++a) {
        w.fam = FAM_REST;
        w.cls = add_class(&x, N - 1 - k, middle(N, a) & ~x.side, 1u << (N - 1 - a), 4, 2);
        root(&x, &w, a);
    }
    if (table) memcpy(table, scratch, sizeof(dih_class_t) * (size_t)(x.ncls < cap_cls ? x.ncls : cap_cls));
    if (n_cls) *n_cls = x.ncls;
    return x.n;
}

/* Weighted completions of one task under its class's rules. */
static uint64_t count_rec(int N, const dih_class_t *c, uint32_t side, uint32_t cur, uint32_t left, uint32_t right,
                          int row) {
    const uint32_t full = (1u << N) - 1u;
    uint32_t f = full & ~(cur | left | right);
    if (row > c->side_row) f &= ~side;
    if (row == N - 1) f &= c->last_mask;
    uint64_t s = 0;
    while (f) {
        const uint32_t p = f & (0u - f);
        f ^= p;
        if (row == N - 1)
            s += (p == c->tie_bit) ? c->w_tie : c->w;
        else
            s += count_rec(N, c, side, cur | p, (left | p) << 1, (right | p) >> 1, row + 1);
    }
    return s;
}

uint64_t nq_oracle_dihedral_count_task(int N, const dih_class_t *c, uint32_t cur, uint32_t left, uint32_t right) {
    const uint32_t side = 1u | (1u << (N - 1));
    return count_rec(N, c, side, cur, left, right, __builtin_popcount(cur));
}

void nq_oracle_dihedral_count_tasks(int N, int64_t n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                                    const uint8_t *cls, const dih_class_t *table, uint64_t *out, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t i = 0; i < n; i++) out[i] = nq_oracle_dihedral_count_task(N, &table[cls[i]], cols[i], ld[i], rd[i]);
    (void)threads;
}

/* Whole-board total through the decomposition (-1 for a bad argument). */
int64_t nq_oracle_dihedral_total(int N, int k, int threads) {
    int ncls = 0;
    const int64_t n = nq_oracle_dihedral_expand(N, k, NULL, NULL, NULL, NULL, 0, NULL, 0, &ncls);
    if (n < 0) return -1;
    const size_t m = (size_t)(n ? n : 1);
    uint32_t *c = malloc(4 * m), *l = malloc(4 * m), *r = malloc(4 * m);
    uint8_t *t = malloc(m);
    uint64_t *o = malloc(8 * m);
    dih_class_t table[64];
    nq_oracle_dihedral_expand(N, k, c, l, r, t, n, table, 64, &ncls);
    nq_oracle_dihedral_count_tasks(N, n, c, l, r, t, table, o, threads);
    uint64_t s = 0;
    for (int64_t i = 0; i < n; i++) s += o[i];
    free(c); free(l); free(r); free(t); free(o);
    return (int64_t)s;
}
