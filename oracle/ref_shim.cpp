// ref_shim.cpp -- extern "C" entry points over the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified src/n_queens.cpp and src/utils.cpp (read where
// they lie; nothing is copied) into oracle/_ref/libnq_ref.so.  Python loads it
// through ctypes to pin the restated oracle (nq_oracle.c), to generate the
// golden fixtures in tests/golden/, and as the timed CPU baseline of bench.py.
#include <stdint.h>
#include <string.h>

#include <vector>

#include <omp.h>

#include "n_queens.h"  // reference header: src/n_queens.h

extern "C" {

// One task through the reference recursion n_queens() (src/n_queens.cpp:8-21).
long long nqref_n_queens(int N, int cur, int left, int right) {
    long long s = 0;
    n_queens(N, cur, left, right, s);
    return s;
}

// The reference expander (src/n_queens.cpp:74-113) exactly as cuda_n_queens
// calls it (src/n_queens_cuda.cu:91-95).  Writes up to cap triples in the
// reference's AoS int layout and returns the task count.
long long nqref_expand(int N, int rows, int *out_aos, long long cap) {
    vector<int> tot;
    partial_n_queens(N, 0, 0, 0, tot, rows);
    if (N & 0x1) partial_n_queens_for_odd(N, 0, 0, 0, tot, rows);
    long long cnt = (long long)tot.size() / 3;
    long long m = cnt < cap ? cnt : cap;
    if (out_aos && m > 0) memcpy(out_aos, tot.data(), sizeof(int) * 3 * (size_t)m);
    return cnt;
}

long long nqref_serial(int N, int rows) { return serial_n_queens(N, rows); }

long long nqref_parallel(int N, int rows) { return parallel_n_queens(N, rows); }

// The per-task loop of parallel_n_queens (src/n_queens.cpp:152-157) over a
// caller-given task list (AoS int triples), with the thread count a parameter
// instead of the hard-coded 32.  Returns the x2 sum as the reference does
// (:158-160); per-task counts go to out when it is not NULL.
long long nqref_count_tasks(int N, long long n, const int *tot, long long *out, int threads) {
    vector<long long> partial(n > 0 ? n : 1, 0);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (long long i = 0; i < n; i++) {
        n_queens(N, tot[3 * i], tot[3 * i + 1], tot[3 * i + 2], partial[i]);
    }
    long long sum = 0;
    for (long long i = 0; i < n; i++) {
        sum += partial[i] * 2;
        if (out) out[i] = partial[i];
    }
    return sum;
}

}  // extern "C"
