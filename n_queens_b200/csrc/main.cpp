// main.cpp -- the `n_queens N k` command line of the reference (src/main.cpp),
// same checks, same messages, same result line, over libnqueens_b200.so.
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include "n_queens.h"
#include "timefmt.h"

// Deepest per-lane stack the library accepts for the CLI's range of N (the
// reference's STACKSIZE, src/macro.h:25-35, fixed at build time to 16..24).
static const int kStackLevels = 30;

int main(int argc, char *argv[]) {
    if (argc < 3) {
        printf("usage: %s N rows\n", argv[0]);
        return -1;
    }
    int N = atoi(argv[1]);
    if (N < 2 || N > 28) {
        printf("Not allowed %d queens problem!\n", N);
        return -1;
    }

    int rows = atoi(argv[2]);
    if (kStackLevels + 1 + rows < N) {
        printf("This configure cannot process %d-queens with pre-placing %d rows. Pre-placed rows should be >= %d.\n",
               N, rows, N - kStackLevels - 1);
        return -1;
    }

    if (N - rows < 2) {
        printf("Pre-placed rows should be <= %d.\n", N - 2);
        return -1;
    }

    if (rows < 2) {
        printf("Pre-placed rows shold be at least 2, so set to 2!\n");
        rows = 2;
    }

    struct timeval start, end;
    nqb::print_with_time("===============================================================\n");
    gettimeofday(&start, NULL);
    long long sum = cuda_n_queens(N, rows);
    gettimeofday(&end, NULL);
    nqb::print_with_time("cuda %d queens result %lld, calc time: [%.2fms]\n", N, sum, nqb::time_diff_ms(start, end));
    nqb::print_with_time("===============================================================\n");
    return 0;
}
