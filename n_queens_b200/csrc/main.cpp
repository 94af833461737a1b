// main.cpp -- the `n_queens N k` command line of the reference (src/main.cpp),
// same checks, same messages, same result line, over libnqueens_b200.so.
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include <string.h>

#include "n_queens.h"
#include "n_queens_b200.h"
#include "timefmt.h"

// Deepest per-lane stack the library accepts for the CLI's range of N (the
// reference's STACKSIZE, src/macro.h:25-35, fixed at build time to 16..24).
static const int kStackLevels = 30;

int main(int argc, char *argv[]) {
    if (argc < 3) {
        printf("usage: %s N rows [--checkpoint PATH [--slice-ms MS]] [--dihedral]\n", argv[0]);
        return -1;
    }
    // Optional resumable mode (not in the reference): the count runs in
    // slices of MS milliseconds and saves its state to PATH after each one, so
    // an interrupted run continues where it stopped when started again.
    // --dihedral (not in the reference) counts through the 8-fold
    // decomposition (nq_count_dihedral, or nq_count_dihedral_resumable with
    // --checkpoint): same total, fewer DFS nodes.
    const char *ckpt = nullptr;
    unsigned slice_ms = 600000;
    bool dihedral = false;
    for (int a = 3; a < argc; ++a) {
        if (!strcmp(argv[a], "--dihedral")) {
            dihedral = true;
        } else if (a + 1 < argc) {
            if (!strcmp(argv[a], "--checkpoint")) ckpt = argv[a + 1];
            else if (!strcmp(argv[a], "--slice-ms")) slice_ms = (unsigned)strtoul(argv[a + 1], nullptr, 10);
            ++a;
        }
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
    long long sum = 0;
    if (ckpt) {
        nq_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.time_limit_ms = slice_ms;
        for (int slice = 1;; ++slice) {
            uint64_t total = 0;
            int done = 0;
            const int rc = dihedral ? (N < 4 ? NQ_OK : nq_count_dihedral_resumable(N, rows, &cfg, ckpt, &total, &done,
                                                                                    nullptr))
                                    : nq_count_resumable(N, rows, &cfg, ckpt, &total, &done, nullptr);
            if (dihedral && N < 4) done = 1;  // N = 2, 3: no solutions
            if (rc != NQ_OK) {
                printf("n_queens_b200: %s (%s)\n", nq_status_string(rc), nq_last_error());
                sum = -1;
                break;
            }
            if (done) {
                sum = (long long)total;
                break;
            }
            nqb::print_with_time("slice %d saved to %s\n", slice, ckpt);
        }
    } else if (dihedral) {
        uint64_t total = 0;
        const int rc = N < 4 ? NQ_OK : nq_count_dihedral(N, rows, nullptr, &total, nullptr);
        if (rc != NQ_OK) printf("n_queens_b200: %s (%s)\n", nq_status_string(rc), nq_last_error());
        sum = rc == NQ_OK ? (long long)total : -1;  // N = 2, 3: no solutions
    } else {
        sum = cuda_n_queens(N, rows);
    }
    gettimeofday(&end, NULL);
    nqb::print_with_time("cuda %d queens result %lld, calc time: [%.2fms]\n", N, sum, nqb::time_diff_ms(start, end));
    nqb::print_with_time("===============================================================\n");
    return 0;
}
