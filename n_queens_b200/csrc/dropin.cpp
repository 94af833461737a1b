// dropin.cpp -- the reference's C++ entry points (include/n_queens.h) over the
// C ABI.  Output lines keep the reference's text so existing log parsers work:
// "Use %.2fms to generate %lld subproblems!" (src/n_queens_cuda.cu:101),
// "Failed to find any gpu!" (:106), "gpu [%d] start job, with %lld(%.2f)
// subproblems." (:154) and "gpu [%d] finish job." (:178).
#include <stdint.h>
#include <stdio.h>

#include <vector>

#include "n_queens.h"
#include "n_queens_b200.h"
#include "timefmt.h"

long long cuda_n_queens(int N, int rows) {
    nq_stats st;
    uint64_t total = 0;
    int rc = nq_count(N, rows, nullptr, &total, nullptr, &st);
    nqb::print_with_time("Use %.2fms to generate %lld subproblems!\n", st.expand_ms, (long long)st.tasks);
    if (rc == NQ_ERR_NO_DEVICE) {
        printf("Failed to find any gpu!\n");
        return -1;
    }
    nqb::print_with_time("gpu [%d] start job, with %lld(%.2f) subproblems.\n", 0, (long long)st.tasks, 1.0);
    if (rc != NQ_OK) {
        fprintf(stderr, "n_queens_b200: %s (%s)\n", nq_status_string(rc), nq_last_error());
        return -1;
    }
    nqb::print_with_time("gpu [%d] finish job.\n", 0);
    return (long long)total;
}

void n_queens(int N, int cur, int left, int right, long long &sum) {
    nq_instance in;
    in.N = N;
    in.cols = (uint32_t)cur;
    in.ld = (uint32_t)left;
    in.rd = (uint32_t)right;
    uint64_t out = 0;
    int rc = nq_count_batch(&in, 1, 0, &out, nullptr, nullptr);
    if (rc != NQ_OK) {
        fprintf(stderr, "n_queens_b200: %s (%s)\n", nq_status_string(rc), nq_last_error());
        return;
    }
    sum += (long long)out;
}

namespace {

// Generic-start expander with the reference's row rules: the first-row rule
// applies while cur == 0 and, in the odd pass, the second-row rule while cur
// holds a single queen (src/n_queens.cpp:76-78,95-98).
void expand_from(int N, int cur, int left, int right, std::vector<int> &tot, int rows, bool odd) {
    int last = (int)((1u << N) - 1u);
    if (!odd) {
        if (cur == 0) last = (int)((1u << (N / 2)) - 1u);
    } else {
        if (cur == 0)
            last = (int)(1u << (N / 2));
        else if ((cur & (cur - 1)) == 0)
            last = (int)((1u << ((N - 2) / 2)) - 1u);
    }
    unsigned valid = (unsigned)(last & ~(cur | left | right));
    while (valid) {
        const unsigned p = valid & (0u - valid);
        valid ^= p;
        const int c = cur | (int)p;
        const int l = (int)((unsigned)(left | (int)p) << 1);
        const int r = (right | (int)p) >> 1;
        if (rows == 1) {
            tot.push_back(c);
            tot.push_back(l);
            tot.push_back(r);
            continue;
        }
        expand_from(N, c, l, r, tot, rows - 1, odd);
    }
}

}  // namespace

void partial_n_queens(int N, int cur, int left, int right, std::vector<int> &tot, int rows) {
    if (cur == 0 && left == 0 && right == 0 && rows >= 1 && N >= 2 && N <= NQ_MAX_N) {
        // The common call: the threaded expander writes straight into tot.
        int64_t n = 0;
        if (nq_expand(N, rows, nullptr, nullptr, nullptr, 0, &n, 0) != NQ_OK) return;
        // nq_expand covers both passes for odd N; this entry is the even pass
        // only, so fall through to the generic path for odd N.
        if ((N & 1) == 0) {
            std::vector<uint32_t> c((size_t)n), l((size_t)n), r((size_t)n);
            nq_expand(N, rows, c.data(), l.data(), r.data(), n, &n, 0);
            const size_t base = tot.size();
            tot.resize(base + 3 * (size_t)n);
            for (int64_t i = 0; i < n; ++i) {
                tot[base + 3 * i] = (int)c[i];
                tot[base + 3 * i + 1] = (int)l[i];
                tot[base + 3 * i + 2] = (int)r[i];
            }
            return;
        }
    }
    expand_from(N, cur, left, right, tot, rows, false);
}

void partial_n_queens_for_odd(int N, int cur, int left, int right, std::vector<int> &tot, int rows) {
    expand_from(N, cur, left, right, tot, rows, true);
}
