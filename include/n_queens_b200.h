/*
 * n_queens_b200.h -- C ABI of the B200 (sm_100a) N-Queens solution counter.
 *
 * This is the drop-in boundary for the counting path of ygch/n_queens:
 *
 *   host prefix expander  ->  device task queue  ->  persistent DFS kernel
 *   (src/n_queens.cpp:74-113)  (src/n_queens_cuda.cu:8)  (src/n_queens_cuda.cu:9-82)
 *   -> uint64 reduction (src/n_queens_cuda.cu:181-183)
 *
 * Plain pointers and sizes only.  The caller owns every host buffer; the
 * library owns its device buffers (kept per device and reused between calls)
 * except in the *_device entry, where the caller passes device pointers.
 * Every entry returns an nq_status; nothing here calls exit() (the reference's
 * CU_SAFE_CALL in src/macro.h:40-49 does).  Calls on one device must come from
 * one host thread at a time; a per-device mutex serialises them.
 *
 * Semantics of one task (cols, ld, rd, N): exactly the reference recursion
 * n_queens(N, cur, left, right) of src/n_queens.cpp:8-21 -- a task whose
 * column mask equals (1<<N)-1 counts 1; otherwise every free column
 * last & ~(cur|left|right) is tried, left shifts left (bits past 31 drop) and
 * right shifts right arithmetically, as the reference's `int` arithmetic does.
 */
#ifndef N_QUEENS_B200_H
#define N_QUEENS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NQ_ABI_VERSION 1

/* Largest board.  The reference CLI stops at 28 (src/main.cpp:10); the
 * library takes any N < 32, since masks are 32-bit. */
#define NQ_MAX_N 31

/* Largest nq_config.inner_steps.  A lane's 32-bit counter is folded into its
 * 64-bit total every inner_steps steps and a step adds at most 32, so any
 * bound below 2^27 keeps it exact; this one is far above the useful range
 * (256..4096). */
#define NQ_MAX_INNER_STEPS (1 << 20)

/* Largest nq_config.stack_levels.  No task of a board of at most NQ_MAX_N
 * columns needs more than N-1 <= 30 slots per lane; larger values are
 * NQ_ERR_ARG. */
#define NQ_MAX_STACK_LEVELS 32

typedef enum nq_status {
    NQ_OK = 0,
    NQ_ERR_ARG = -1,       /* an argument is out of range or a pointer is NULL */
    NQ_ERR_NO_DEVICE = -2, /* no CUDA device (cuda_n_queens then returns -1, src/n_queens_cuda.cu:105-108) */
    NQ_ERR_CUDA = -3,      /* a CUDA runtime call failed; see nq_last_error() */
    NQ_ERR_OOM = -4,       /* device, pinned-host or host allocation failed */
    NQ_ERR_DEPTH = -5,     /* a task needs more stack levels than the launch provides */
    NQ_ERR_TIMEOUT = -6,   /* the kernel reached cfg->time_limit_ms and stopped; the counts are partial */
    NQ_ERR_NO_KERNEL = -7  /* the library has no sm_100a image for this device */
} nq_status;

/* Task order.  NQ_ORDER_PLAIN hands tasks out in expander order through one
 * atomic ticket (the reference's dynamic fetch, src/n_queens_cuda.cu:10,80);
 * NQ_ORDER_GIVEN uses the caller's permutation (nq_config.order), e.g. a
 * longest-first schedule from the learned cost model. */
enum { NQ_ORDER_PLAIN = 0, NQ_ORDER_GIVEN = 1 };

/* Shared-memory stack layouts.  INTERLEAVED puts slot s of lane l at
 * s*512 + l*16 inside the warp's block: the eight lanes of a quarter-warp
 * always cover the 32 banks once, whatever the lanes' depths, so no stack
 * access needs more wavefronts than a dense 16-byte access of the warp.
 * LANE_MAJOR keeps each lane's slots contiguous (conflicts depend on the
 * depths); it exists for the autotuner's comparison. */
enum { NQ_LAYOUT_INTERLEAVED = 0, NQ_LAYOUT_LANE_MAJOR = 1 };

/* Launch parameters; zero-initialise and set what you need.  Zero means
 * "default" (the autotuned or built-in choice) for every field. */
typedef struct nq_config {
    int block_threads;      /* threads per CTA: 32..1024, multiple of 32; 0 = the size (64..512) that keeps
                               the most warps resident per SM for the launch's stack depth */
    int blocks_per_sm;      /* resident CTAs per SM for the persistent grid */
    int stack_levels;       /* per-lane DFS stack slots (>= nq_stack_levels(N, rows, nodes), at most
                               NQ_MAX_STACK_LEVELS) */
    int steal;              /* 0 = default (on), 1 = on, -1 = off: in-warp work donation */
    int inner_steps;        /* DFS steps between warp refill checks: 1..NQ_MAX_INNER_STEPS (larger values
                               are NQ_ERR_ARG), rounded up to a multiple of the kernel's steps per warp
                               vote (16 for counts, 8 for node counts and the dihedral kernels) */
    int order_kind;         /* NQ_ORDER_PLAIN or NQ_ORDER_GIVEN */
    const uint32_t *order;  /* NQ_ORDER_GIVEN: queue position -> task index (host or device
                               pointer, matching the entry's other task arrays) */
    uint32_t time_limit_ms; /* 0 = none; else the kernel stops after this long (NQ_ERR_TIMEOUT) */
    int device;             /* CUDA device ordinal (default 0) */
    int timing;             /* non-zero: host entries record per-CTA start/end times and fill the
                               makespan / tail fields of nq_stats */
    int layout;             /* NQ_LAYOUT_INTERLEAVED (default) or NQ_LAYOUT_LANE_MAJOR */
    int device_expand;      /* nq_count: non-zero builds the prefix tasks on the device (nq_expand_device)
                               instead of on the host + H2D copy */
    uint32_t queue_len;     /* queue positions to run, 0 = all n (must be <= n): the count covers only the
                               tasks at positions 0 .. queue_len-1 (order[i] with NQ_ORDER_GIVEN, else i) */
    int reserved[2];
} nq_config;

/* Timings and sizes of one call (all optional outputs). */
typedef struct nq_stats {
    double expand_ms;   /* host prefix expansion */
    double h2d_ms;      /* task upload (event-timed) */
    double kernel_ms;   /* queue reset + DFS kernel + reduction (event-timed) */
    double d2h_ms;      /* result download (event-timed) */
    double total_ms;    /* wall time of the whole call */
    int64_t tasks;      /* number of tasks */
    uint64_t nodes;     /* DFS nodes, when the entry was asked to count them */
    int grid;           /* CTAs launched */
    int block_threads;  /* threads per CTA */
    int stack_levels;   /* stack slots per lane */
    int smem_bytes;     /* dynamic shared memory per CTA */
    int reserved[5];
    /* With nq_config.timing: kernel span from the first CTA start to the last
     * CTA end, the mean CTA busy time, and the idle fraction of the grid
     * (1 - sum of CTA busy times / (CTAs x span)) -- the tail left by uneven
     * tasks. */
    double makespan_ms;
    double cta_busy_mean_ms;
    double tail_idle_frac;
    double schedule_ms; /* nq_count_learned: prediction + longest-first sort */
} nq_stats;

/* One independent completion-counting problem of the batched entry. */
typedef struct nq_instance {
    int32_t N;     /* board size, 1..NQ_MAX_N */
    uint32_t cols; /* columns taken by the pre-placed rows */
    uint32_t ld;   /* left-diagonal attacks on the next row */
    uint32_t rd;   /* right-diagonal attacks on the next row */
} nq_instance;

/* Library and error reporting. */
int nq_abi_version(void);
const char *nq_status_string(int status);
/* Text of the last CUDA error seen by this thread (empty if none). */
const char *nq_last_error(void);
/* Number of CUDA devices (0 when none); returns NQ_OK or NQ_ERR_CUDA. */
int nq_device_count(int *count);
/* Stack slots per lane (nq_config.stack_levels) that tasks with `rows`
 * queens placed need: N-1-rows when the count also reports DFS nodes
 * (nodes != 0), N-3-rows otherwise (the count step never enters rows N-2 and
 * N-1), at least 1.  The reference fixes this depth at compile time
 * (STACKSIZE, src/macro.h:25-35).  Returns NQ_ERR_ARG for an invalid (N, rows). */
int nq_stack_levels(int N, int rows, int nodes);

/* Host prefix expander.  Replaces partial_n_queens + partial_n_queens_for_odd
 * (src/n_queens.cpp:74-113) as cuda_n_queens calls them
 * (src/n_queens_cuda.cu:91-95): every non-attacking placement of rows
 * 0..rows-1 with row 0 in columns [0, N/2), then for odd N the middle-column
 * pass, in the reference's order, as SoA uint32 triples.  Writes at most cap
 * tasks and stores the full count in *n_tasks (call with cap = 0 to size).
 * threads <= 0 uses every host core. */
int nq_expand(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, int64_t cap, int64_t *n_tasks,
              int threads);

/* The same expansion on the device (no counterpart in the reference): the
 * host enumerates the reference-ordered placements of the first min(rows, 4)
 * rows, then a count pass, a scan and a write pass on `device` produce the
 * prefixes into the caller's device arrays, in the same order as nq_expand.
 * Writes at most cap tasks, *n_tasks receives the full count; synchronises
 * `stream` (NULL = legacy default) once, to learn that count. */
int nq_expand_device(int N, int rows, uint32_t *d_cols, uint32_t *d_ld, uint32_t *d_rd, int64_t cap,
                     int64_t *n_tasks, int device, void *stream);

/* Whole-board count.  Replaces cuda_n_queens (src/n_queens_cuda.cu:84-186)
 * on one device: expand, upload, count, and return 2 x the sum of the
 * per-prefix counts in *total (the reference's x2 mirror reduction,
 * src/n_queens_cuda.cu:181-183).  Requires 2 <= N <= NQ_MAX_N and
 * 1 <= rows <= N-2 (src/main.cpp:21-24).  If nodes is not NULL the DFS
 * node total of the same decomposition is counted as well (slower).
 * As in the reference, odd N with rows == 1 overcounts (the middle-column
 * task is doubled without the second-row restriction); the reference CLI
 * raises rows to 2 (src/main.cpp:26-29) and so does this library's CLI. */
int nq_count(int N, int rows, const nq_config *cfg, uint64_t *total, uint64_t *nodes, nq_stats *stats);

/* Time-sliced, resumable whole-board count (no counterpart in the reference,
 * whose N=26/27 runs took 2.5 and 28.4 days with no way to stop and resume,
 * README.md:41-48).  Same total as nq_count.  If checkpoint_path exists the
 * count resumes from it (it must be for the same N and rows).  With
 * cfg->time_limit_ms > 0 the kernel stops after that long: every lane saves
 * its unfinished DFS levels, and the queue cursor, the partial sum and those
 * levels are written to checkpoint_path (atomically, via a .tmp file);
 * *done = 0 and NQ_OK are returned.  Once the count finishes, *done = 1,
 * *total holds it and the checkpoint file is removed.  Call again until done.
 * Saved work is never counted twice or lost: each level is either finished
 * (and in the partial sum) or saved with only its untried columns. */
int nq_count_resumable(int N, int rows, const nq_config *cfg, const char *checkpoint_path, uint64_t *total,
                       int *done, nq_stats *stats);

/* Counts over a caller-built task list in host memory.  Replaces the
 * per-GPU upload / launch / download of src/n_queens_cuda.cu:156-177 with
 * the per-task semantics of n_queens() (src/n_queens.cpp:8-21).
 * per_task[i] (optional) receives task i's completions, nodes_per_task[i]
 * (optional) its DFS nodes; *sum receives the plain sum of the counts
 * (no x2).  n may be 0. */
int nq_count_tasks(int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                   uint64_t *per_task, uint64_t *nodes_per_task, uint64_t *sum, const nq_config *cfg,
                   nq_stats *stats);

/* The same over device-resident tasks (device pointers, already in HBM),
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream).
 * d_per_task / d_nodes are optional device arrays of n uint64 (overwritten;
 * d_nodes needs d_per_task).  d_sum is a device array of 2 uint64: [0]
 * receives the plain sum of the counts, [1] status bits (1: a task needed
 * more stack levels than the launch had and was skipped; 2: the time limit
 * stopped the kernel).  Without a host view of the tasks the stack covers
 * the deepest possible task (nq_stack_levels(N, 0, d_nodes != NULL) levels)
 * unless cfg->stack_levels says otherwise.  Returns after enqueueing;
 * the caller synchronises the stream.  Uses the library's device scratch for the
 * queue and the per-CTA partials, so calls on one device must not overlap. */
int nq_count_tasks_device(int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd, int64_t n,
                          uint64_t *d_per_task, uint64_t *d_nodes, uint64_t *d_sum, const nq_config *cfg,
                          void *stream);

/* Device-resident count that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot let a library call cudaMalloc
 * -- a host framework whose caching allocator has reserved the GPU's memory,
 * or a service that forbids device allocation after start-up.  Same inputs,
 * outputs and meaning as nq_count_tasks_device without per-task outputs:
 * d_sum (2 device uint64) receives the plain sum and the status bits.  The
 * queue/flag words and per-CTA partials live in a fixed array inside the
 * library image (about 64 KiB, held on every GPU that loads the library until
 * exit) with room for 8192 CTAs; a cfg->blocks_per_sm that would launch more
 * is rejected with NQ_ERR_ARG.  Every call shares that array and clears its
 * control words first, so calls whose kernels overlap on the GPU race and
 * must be serialised by the caller.  The first call on a device performs the
 * device's set-up (the array's device address, the kernel's shared-memory
 * opt-in); make it before any stream capture.  The launch shape (CTA size,
 * DFS steps between queue visits, stack layout) is chosen from cfg exactly as
 * nq_count_tasks_device chooses it, with the grid bounded by the array.  The
 * caller's current device is the same after the call as before it. */
int nq_count_tasks_device_noalloc(int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd,
                                  int64_t n, uint64_t *d_sum, const nq_config *cfg, void *stream);

/* Batched independent instances of uneven N and partial boards in one
 * persistent launch (no counterpart in the reference).  out[i] receives
 * n_queens() of instance i (src/n_queens.cpp:8-21, no symmetry factor).
 * Identical instances, and instances equal up to their mirror image, are
 * counted once; a mirror-symmetric board counts its left-half children twice
 * (the reference's half-board rule, src/n_queens.cpp:74-113, applied to any
 * symmetric board).  Every distinct board is split split_rows rows deeper
 * (0 = 3).  nq_count_batch = nq_batch_create + nq_batch_run + destroy. */
int nq_count_batch(const nq_instance *inst, int64_t n, int split_rows, uint64_t *out, const nq_config *cfg,
                   nq_stats *stats);

/* A reusable batch plan: the subtasks are built and uploaded once, and the
 * queue reset + count + result copy are captured in one CUDA graph that
 * nq_batch_run replays.  A plan keeps its device buffers until destroyed and
 * uses its device's shared library scratch, so runs on one device are
 * serialised. */
typedef struct nq_batch nq_batch;
int nq_batch_create(const nq_instance *inst, int64_t n, int split_rows, const nq_config *cfg, nq_batch **out);
int nq_batch_run(nq_batch *b, uint64_t *out, nq_stats *stats);
int nq_batch_destroy(nq_batch *b);

/* One measured configuration of the batch autotuner. */
typedef struct nq_tune_entry {
    int split_rows;
    int block_threads;
    int layout;
    int inner_steps; /* DFS steps a warp runs between queue refills */
    double ms;       /* mean graph replay time over `repeats` runs after one warm-up */
} nq_tune_entry;

/* Sweeps split depth 3..7, CTA size 64/128/256/512 and both stack layouts on
 * the given instances (other launch fields from `base`), then queue chunking
 * -- 256, 1024 (the default) and 4096 DFS steps between a warp's queue
 * refills -- at the fastest of those; replays each plan's graph and writes up
 * to table_cap measured entries (40 + 2), their number and the fastest.  Each
 * plan's stack depth is the least its subtasks need (a deeper split needs
 * fewer slots), so the split sweep also sweeps the stack depth and the
 * resident warps it allows; a deeper stack than that only costs occupancy. */
int nq_batch_autotune(const nq_instance *inst, int64_t n, int repeats, const nq_config *base, nq_tune_entry *table,
                      int table_cap, int *n_entries, nq_tune_entry *best);

/* ---- Learned subtree-cost scheduler (no counterpart in the reference) ----
 *
 * The reference hands tasks out in expander order (src/n_queens_cuda.cu:10,80).
 * These entries build and use a small cost model so the queue can run the
 * most expensive prefixes first.  Model: the three masks of a task as 96 bits
 * (cols, ld, rd, 32 bits each, columns >= N cleared) -> 128 ReLU -> 128 ReLU
 * -> predicted log2(1 + DFS nodes).  BF16 weights for compute, FP32 master
 * weights and Adam, FP32 accumulation; every kernel is this library's own.
 * A model lives on one device; calls on one model are serialised. */
typedef struct nq_mlp nq_mlp;

/* Number of FP32 parameters (29057).  Flat layout: W1[128][96], b1[128],
 * W2[128][128], b2[128], W3[128], b3. */
int nq_mlp_num_params(void);
/* New model on `device`, weights ~ U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from
 * SplitMix64(seed). */
int nq_mlp_create(int device, uint64_t seed, nq_mlp **out);
int nq_mlp_destroy(nq_mlp *m);
/* FP32 master weights in the flat layout; set also resets Adam's moments. */
int nq_mlp_get_params(nq_mlp *m, float *out);
int nq_mlp_set_params(nq_mlp *m, const float *in);
/* Predicted log2(1 + nodes) of n tasks of board size N (host arrays). */
int nq_mlp_predict(nq_mlp *m, int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                   float *out);
/* The same forward on the tensor cores (tcgen05.mma, BF16 operands, FP32
 * accumulators in TMEM), as nq_schedule_device runs it: the layer-1 outputs
 * are rounded to BF16 before layer 2, so results differ from nq_mlp_predict
 * by that rounding. */
int nq_mlp_predict_tensor(nq_mlp *m, int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                          float *out);
/* Gradient of the mean squared error over n tasks (per-task board sizes in
 * task_n, targets in log2(1 + nodes)) with respect to the BF16 compute
 * weights, in the flat layout, and the loss.  Changes nothing. */
int nq_mlp_grad(nq_mlp *m, const uint8_t *task_n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                const float *target, int64_t n, float *grad_out, float *loss_out);
/* Adam (beta 0.9/0.999, eps 1e-8) over `epochs` shuffled passes (SplitMix64
 * seed) in minibatches of `batch`; epoch_loss (optional, `epochs` floats)
 * receives each pass's mean squared error. */
int nq_mlp_train(nq_mlp *m, const uint8_t *task_n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                 const float *target, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                 float *epoch_loss);
/* Longest-first order of device-resident tasks: d_order (n u32) receives the
 * task indices sorted by predicted cost, descending, in bins of 1/8 log2 unit
 * and stable inside a bin; d_pred (optional, n floats) the predictions.
 * Stream-ordered on `stream` (a cudaStream_t; NULL = legacy default stream).
 * The model's prediction scratch is in use until that work completes: call no
 * other entry of the same model before it has. */
int nq_schedule_device(nq_mlp *m, int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd,
                       int64_t n, uint32_t *d_order, float *d_pred, void *stream);
/* nq_schedule_device with the n_last tasks listed in d_last (device u32 task
 * indices) placed behind every other task, in index order; an order run with
 * nq_config.queue_len = n - n_last then skips exactly those tasks.  Indices
 * at or beyond n are ignored.  No counterpart in the reference. */
int nq_schedule_device_last(nq_mlp *m, int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd,
                            int64_t n, const uint32_t *d_last, int64_t n_last, uint32_t *d_order, float *d_pred,
                            void *stream);
/* nq_count with the queue ordered by the model: expand, upload, schedule on
 * the device, count.  The same total as nq_count; stats->schedule_ms holds the
 * prediction + sort time.  The model must live on cfg->device. */
int nq_count_learned(int N, int rows, nq_mlp *m, const nq_config *cfg, uint64_t *total, nq_stats *stats);
/* nq_count_learned for a board part of whose tasks was already counted --
 * typically the cost model's fine-tuning and hold-out samples, which the
 * model build counts exactly to label them.  done_idx lists those task
 * indices (expander order, ascending, distinct; n_done of them) and done_sum
 * is the plain sum of their counts.  The queue holds only the other tasks,
 * longest first, and *total = 2 x (done_sum + their sum), the same total as
 * nq_count.  No counterpart in the reference. */
int nq_count_learned_reuse(int N, int rows, nq_mlp *m, const int64_t *done_idx, int64_t n_done, uint64_t done_sum,
                           const nq_config *cfg, uint64_t *total, nq_stats *stats);

/* ---- Dihedral (8-fold) decomposition (no counterpart in the reference) ----
 * The reference counts only the left-right mirror: row 0 in the left half,
 * every prefix x2 (src/n_queens.cpp:74-113, src/n_queens_cuda.cu:181-183).
 * These entries use all eight symmetries of the square: the tasks fall into
 * classes (a corner queen; the border queen nearest a corner at distance m;
 * all border queens at distance >= rows) whose searches follow the class's
 * rules and whose completions carry the class's weights, so the weighted sum
 * is the whole-board total with ~1.75x fewer DFS nodes than the reference's
 * decomposition.  rows (the prefix depth) must be in [2, N-2], 4 <= N <= 31. */

/* Rules of one class: rows beyond side_row may not use column 0 or N-1;
 * row N-1 may use only last_mask's columns; a completion weighs weight_tie
 * when its row N-1 queen is at tie_bit, else weight. */
typedef struct {
    int32_t side_row;
    uint32_t last_mask;
    uint32_t tie_bit;
    uint32_t weight;
    uint32_t weight_tie;
} nq_dihedral_class;

/* The task list of (N, rows) in host memory: cols (on-board bits), ld, rd as
 * the reference packs prefixes, cls[i] the class index of task i.  Writes at
 * most cap tasks (cap 0 and NULL arrays: count only) and at most cap_classes
 * classes; *n_tasks and *n_classes receive the full counts.  Host only. */
int nq_dihedral_expand(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, uint8_t *cls, int64_t cap,
                       int64_t *n_tasks, nq_dihedral_class *classes, int cap_classes, int *n_classes);
/* Whole-board total through the dihedral decomposition (the same total as
 * nq_count / cuda_n_queens).  stats->tasks counts the dihedral tasks.  cfg's
 * launch fields apply; device_expand does not (the tasks are built on the
 * host). */
int nq_count_dihedral(int N, int rows, const nq_config *cfg, uint64_t *total, nq_stats *stats);
/* nq_count_resumable through the dihedral decomposition: the same slices,
 * checkpoint file and guarantees (every saved level keeps its class); a
 * checkpoint of the other decomposition is rejected with NQ_ERR_ARG.
 * CLI: n_queens N rows --dihedral --checkpoint PATH [--slice-ms MS]. */
int nq_count_dihedral_resumable(int N, int rows, const nq_config *cfg, const char *checkpoint_path, uint64_t *total,
                                int *done, nq_stats *stats);
/* Weighted counts of a caller's dihedral tasks (host arrays, the classes of
 * (N, rows)): per_task[i] (optional) receives task i's weighted count, *sum
 * their sum.  The tasks are meant to come from nq_dihedral_expand (any subset
 * or order): on-board masks, ld/rd as the expander packs them. */
int nq_count_dihedral_tasks(int N, int rows, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                            const uint8_t *cls, int64_t n, uint64_t *per_task, uint64_t *sum, const nq_config *cfg,
                            nq_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* N_QUEENS_B200_H */
