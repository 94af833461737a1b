/*
 * nq_oracle.c -- CPU restatement of the ygch/n_queens counting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the
 * n_queens_b200 GPU path: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product library never links,
 * calls or falls back to it.
 *
 * Parity is pinned two ways (tests/test_oracle.py):
 *   - against the reference's own functions compiled from its sources into
 *     oracle/_ref/libnq_ref.so (per-task counts, expander output byte for
 *     byte, serial totals), through fixtures in tests/golden/;
 *   - against the published totals in README.md:16-25 and logs/5090.log.
 *
 * Every function cites the reference file:line it restates.  All masks are
 * 32-bit; shifts follow the reference's `int` arithmetic (left shift drops
 * bits past 31, right shift of `right` is arithmetic), so results agree with
 * the reference for every 32-bit input, not only for well-formed boards.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SHL1(x) ((int32_t)((uint32_t)(x) << 1))
#define SAR1(x) ((int32_t)(x) >> 1)

/* Recursive completion count from one partial board.
 * Restates n_queens() in src/n_queens.cpp:8-21: a board whose column mask
 * equals `last` counts 1; otherwise every free column of the next row is
 * tried, lowest bit first. */
static uint64_t count_rec(int32_t last, int32_t cur, int32_t left, int32_t right) {
    if (cur == last) return 1;
    uint64_t sum = 0;
    int32_t valid = last & ~(cur | left | right);
    while (valid) {
        int32_t p = valid & -valid;
        valid -= p;
        sum += count_rec(last, cur | p, SHL1(left | p), SAR1(right | p));
    }
    return sum;
}

uint64_t nq_oracle_count_task(int N, uint32_t cur, uint32_t left, uint32_t right) {
    int32_t last = (int32_t)((N >= 32) ? 0xFFFFFFFFu : ((1u << N) - 1u));
    return count_rec(last, (int32_t)cur, (int32_t)left, (int32_t)right);
}

/* DFS node count of one task, with the node defined by the reference GPU
 * loop in src/n_queens_cuda.cu:39-72: one node is one placement taken from
 * the valid mask of a stacked entry.  The root is stacked when its valid mask
 * is non-zero (:19-24,36); a child is stacked only when it is not dead and
 * popc(cur) != N-1 (:59-71); a child with popc(cur) == N-1 is a leaf whose
 * completions are added by popcount and which is never expanded.  So nodes
 * are the placements in rows k..N-2 of a task rooted at row k. */
static uint64_t nodes_rec(int N, int32_t last, int32_t cur, int32_t left, int32_t right) {
    int32_t valid = last & ~(cur | left | right);
    uint64_t n = 0;
    while (valid) {
        int32_t p = valid & -valid;
        valid -= p;
        n += 1;
        int32_t c = cur | p;
        int32_t l = SHL1(left | p);
        int32_t r = SAR1(right | p);
        int32_t v = last & ~(c | l | r);
        if (v != 0 && __builtin_popcount((uint32_t)c) != N - 1) n += nodes_rec(N, last, c, l, r);
    }
    return n;
}

uint64_t nq_oracle_nodes_task(int N, uint32_t cur, uint32_t left, uint32_t right) {
    int32_t last = (int32_t)((N >= 32) ? 0xFFFFFFFFu : ((1u << N) - 1u));
    /* A root that already holds N-1 queens has only board-completing
     * placements left, which are not nodes (the reference never builds such
     * a task: src/main.cpp:21-24 keeps N - rows >= 2). */
    if (__builtin_popcount(cur) >= N - 1) return 0;
    return nodes_rec(N, last, (int32_t)cur, (int32_t)left, (int32_t)right);
}

/* Prefix expander.  Restates partial_n_queens (src/n_queens.cpp:74-91) and
 * partial_n_queens_for_odd (:93-113): all non-attacking placements of rows
 * 0..rows-1, row 0 restricted to columns [0, N/2); for odd N a second pass
 * puts row 0 on the middle column and restricts row 1 to columns
 * [0, (N-2)/2).  Each leaf emits (cur|p, (left|p)<<1, (right|p)>>1), in the
 * reference's order (lowest bit first, even pass then odd pass). */
typedef struct {
    uint32_t *cols, *ld, *rd;
    int64_t n, cap;
} emit_t;

static void emit(emit_t *e, int32_t c, int32_t l, int32_t r) {
    if (e->n < e->cap) {
        e->cols[e->n] = (uint32_t)c;
        e->ld[e->n] = (uint32_t)l;
        e->rd[e->n] = (uint32_t)r;
    }
    e->n++;
}

static void expand_even(int N, int32_t cur, int32_t left, int32_t right, int rows, emit_t *e) {
    int32_t last = (int32_t)((1u << N) - 1u);
    if (cur == 0) last = (int32_t)((1u << (N / 2)) - 1u);
    int32_t valid = last & ~(cur | left | right);
    while (valid) {
        int32_t p = valid & -valid;
        valid -= p;
        if (rows == 1) {
            emit(e, cur | p, SHL1(left | p), SAR1(right | p));
            continue;
        }
        expand_even(N, cur | p, SHL1(left | p), SAR1(right | p), rows - 1, e);
    }
}

static void expand_odd(int N, int32_t cur, int32_t left, int32_t right, int rows, emit_t *e) {
    int32_t last = (int32_t)((1u << N) - 1u);
    if (cur == 0)
        last = (int32_t)(1u << (N / 2));
    else if ((cur & (cur - 1)) == 0)
        last = (int32_t)((1u << ((N - 2) / 2)) - 1u);
    int32_t valid = last & ~(cur | left | right);
    while (valid) {
        int32_t p = valid & -valid;
        valid -= p;
        if (rows == 1) {
            emit(e, cur | p, SHL1(left | p), SAR1(right | p));
            continue;
        }
        expand_odd(N, cur | p, SHL1(left | p), SAR1(right | p), rows - 1, e);
    }
}

/* Returns the number of tasks; writes at most `cap` of them (pass cap = 0 and
 * NULL arrays to only count).  rows must be >= 1. */
int64_t nq_oracle_expand(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, int64_t cap) {
    emit_t e = {cols, ld, rd, 0, cap};
    if (N < 2 || N > 31 || rows < 1) return -1;
    expand_even(N, 0, 0, 0, rows, &e);
    if (N & 1) expand_odd(N, 0, 0, 0, rows, &e);
    return e.n;
}

/* Per-task counts and nodes for a task list (either output may be NULL).
 * The loop is the body of serial_n_queens / parallel_n_queens
 * (src/n_queens.cpp:128-130,152-157), with the thread count a parameter
 * instead of the hard-coded 32 and a dynamic schedule. */
void nq_oracle_count_tasks(int N, int64_t n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                           uint64_t *counts, uint64_t *nodes, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t i = 0; i < n; i++) {
        if (counts) counts[i] = nq_oracle_count_task(N, cols[i], ld[i], rd[i]);
        if (nodes) nodes[i] = nq_oracle_nodes_task(N, cols[i], ld[i], rd[i]);
    }
    (void)threads;
}

/* Whole-board count: expand, count every task, sum x2.  Restates
 * serial_n_queens (src/n_queens.cpp:115-137) and the x2 reduction of
 * cuda_n_queens (src/n_queens_cuda.cu:181-183).  Optionally returns the DFS
 * node total of the same decomposition. */
int64_t nq_oracle_total(int N, int rows, int threads, uint64_t *nodes_out) {
    int64_t n = nq_oracle_expand(N, rows, NULL, NULL, NULL, 0);
    if (n < 0) return -1;
    uint32_t *c = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t *l = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t *r = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1));
    uint64_t *nd = nodes_out ? (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1)) : NULL;
    nq_oracle_expand(N, rows, c, l, r, n);
    nq_oracle_count_tasks(N, n, c, l, r, cnt, nd, threads);
    uint64_t s = 0, ns = 0;
    for (int64_t i = 0; i < n; i++) {
        s += cnt[i] * 2;
        if (nd) ns += nd[i];
    }
    if (nodes_out) *nodes_out = ns;
    free(c); free(l); free(r); free(cnt); free(nd);
    return (int64_t)s;
}
