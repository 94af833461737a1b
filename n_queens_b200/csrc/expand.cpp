// expand.cpp -- host prefix expander.
//
// Produces the task list of cuda_n_queens (src/n_queens_cuda.cu:91-95):
// partial_n_queens (src/n_queens.cpp:74-91) followed, for odd N, by
// partial_n_queens_for_odd (:93-113).  The rule set and the output order are
// the reference's (lowest free column first, even pass then odd pass), so
// task i here is task i there; the representation is SoA uint32 instead of an
// AoS vector<int>, and the work is spread over host threads:
//
//   1. enumerate the "seeds" (placements of the first s rows, s <= 3) in
//      order, serially -- there are at most a few thousand;
//   2. expand every seed to `rows` rows twice in parallel: first to count its
//      tasks, then (after a prefix sum) to write them at their final offsets.
//
// Row masks: row 0 of the even pass takes columns [0, N/2); row 0 of the odd
// pass takes only the middle column N/2 and row 1 of the odd pass columns
// [0, (N-2)/2).  Every other row takes all N columns.
#include "expand.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace nqb {

namespace {

struct Pass {
    int N;
    bool odd;
    uint32_t full;
    uint32_t row_mask(int row) const {
        if (row == 0) return odd ? (1u << (N / 2)) : ((1u << (N / 2)) - 1u);
        if (row == 1 && odd) return (1u << ((N - 2) / 2)) - 1u;
        return full;
    }
};

struct State {
    uint32_t c, l, r;
};

inline State child(const State &s, uint32_t p) {
    // (cur|p, (left|p)<<1, (right|p)>>1) with the reference's int arithmetic:
    // the right shift is arithmetic (right never has bit 31 set here).
    return State{s.c | p, (s.l | p) << 1, (uint32_t)((int32_t)(s.r | p) >> 1)};
}

// Depth-first enumeration of rows [row0, rows) from state s, calling
// emit(State) for each complete prefix in the reference's order.
template <class F>
void dfs(const Pass &ps, State s, int row0, int rows, F &&emit) {
    if (row0 == rows) {
        emit(s);
        return;
    }
    struct Lv {
        State s;
        uint32_t avail;
    };
    Lv st[32];
    int d = 0;
    st[0].s = s;
    st[0].avail = ps.row_mask(row0) & ~(s.c | s.l | s.r);
    while (d >= 0) {
        uint32_t a = st[d].avail;
        if (a == 0) {
            --d;
            continue;
        }
        const uint32_t p = a & (0u - a);
        st[d].avail = a ^ p;
        const State cs = child(st[d].s, p);
        const int row = row0 + d + 1;
        if (row == rows) {
            emit(cs);
        } else {
            ++d;
            st[d].s = cs;
            st[d].avail = ps.row_mask(row) & ~(cs.c | cs.l | cs.r);
        }
    }
}

int pick_threads(int threads) {
    if (threads > 0) return threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

template <class F>
void parallel_for(int nthreads, int64_t n, F &&f) {
    if (nthreads <= 1 || n <= 1) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= n) break;
            f(i);
        }
    };
    const int nt = (int)std::min<int64_t>(nthreads, n);
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}

}  // namespace

int64_t expand_prefixes(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, int64_t cap, int threads) {
    return expand_prefixes_to(
        N, rows,
        [&](int64_t, uint32_t **c, uint32_t **l, uint32_t **r, int64_t *k) {
            *c = cols;
            *l = ld;
            *r = rd;
            *k = (cols && ld && rd) ? cap : 0;
            return true;
        },
        threads);
}

int64_t expand_prefixes_to(int N, int rows, const PrefixSink &sink, int threads) {
    if (N < 2 || N > 31 || rows < 1 || rows > N) return -1;
    const uint32_t full = (1u << N) - 1u;
    const int nthreads = pick_threads(threads);

    struct Seed {
        State s;
        bool odd;
    };
    std::vector<Seed> seeds;
    const int seed_rows = std::min(rows, 3);
    for (int pass = 0; pass < ((N & 1) ? 2 : 1); ++pass) {
        const Pass ps{N, pass == 1, full};
        dfs(ps, State{0, 0, 0}, 0, seed_rows, [&](const State &s) { seeds.push_back(Seed{s, ps.odd}); });
    }
    const int64_t ns = (int64_t)seeds.size();
    std::vector<int64_t> off(ns + 1, 0);
    parallel_for(nthreads, ns, [&](int64_t i) {
        const Pass ps{N, seeds[i].odd, full};
        int64_t c = 0;
        dfs(ps, seeds[i].s, seed_rows, rows, [&](const State &) { ++c; });
        off[i + 1] = c;
    });
    for (int64_t i = 0; i < ns; ++i) off[i + 1] += off[i];
    const int64_t total = off[ns];
    uint32_t *cols = nullptr, *ld = nullptr, *rd = nullptr;
    int64_t cap = 0;
    if (!sink(total, &cols, &ld, &rd, &cap)) return -2;
    if (cap > 0 && cols && ld && rd) {
        parallel_for(nthreads, ns, [&](int64_t i) {
            if (off[i] >= cap) return;
            const Pass ps{N, seeds[i].odd, full};
            int64_t k = off[i];
            dfs(ps, seeds[i].s, seed_rows, rows, [&](const State &s) {
                if (k < cap) {
                    cols[k] = s.c;
                    ld[k] = s.l;
                    rd[k] = s.r;
                }
                ++k;
            });
        });
    }
    return total;
}

int64_t expand_board(int N, uint32_t c0, uint32_t l0, uint32_t r0, int rows, std::vector<uint32_t> &cols,
                     std::vector<uint32_t> &ld, std::vector<uint32_t> &rd) {
    // Splits one partial board into subtasks `rows` rows deeper.  The sum of
    // n_queens() over the subtasks equals n_queens() of the board
    // (src/n_queens.cpp:8-21): a board that is complete, malformed (columns
    // off the board) or already at the split depth is kept as it is.
    const uint32_t last = (N >= 32) ? 0xffffffffu : ((1u << N) - 1u);
    int64_t n = 0;
    if (rows <= 0 || (c0 & ~last) || c0 == last) {
        cols.push_back(c0);
        ld.push_back(l0);
        rd.push_back(r0);
        return 1;
    }
    struct Lv {
        State s;
        uint32_t avail;
    };
    Lv st[33];
    int d = 0;
    st[0].s = State{c0, l0, r0};
    st[0].avail = last & ~(c0 | l0 | r0);
    while (d >= 0) {
        const uint32_t a = st[d].avail;
        if (a == 0) {
            --d;
            continue;
        }
        const uint32_t p = a & (0u - a);
        st[d].avail = a ^ p;
        const State cs = child(st[d].s, p);
        if (d + 1 == rows || cs.c == last) {
            cols.push_back(cs.c);
            ld.push_back(cs.l);
            rd.push_back(cs.r);
            ++n;
        } else {
            ++d;
            st[d].s = cs;
            st[d].avail = last & ~(cs.c | cs.l | cs.r);
        }
    }
    return n;
}

}  // namespace nqb
