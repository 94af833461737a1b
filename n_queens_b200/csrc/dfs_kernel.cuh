// dfs_kernel.cuh -- persistent iterative-DFS kernel for sm_100a.
//
// Replaces the reference kernel n_queens() of src/n_queens_cuda.cu:9-82 and
// its ticket counter global_counter (:8).  Same per-task arithmetic
// (n_queens() of src/n_queens.cpp:8-21); different machine organisation:
//
//  * One lane runs one DFS.  The current level lives in registers
//    (cols, ld, rd, avail); only levels that still have untried columns are
//    pushed to the lane's shared-memory stack, so a pop always resumes a level
//    with work and every DFS step places exactly one queen.
//  * The count kernels' step (VAR 4) lists only a level's alive columns --
//    those whose child still has a free column in the next row -- and counts
//    the completions of a row N-2 level from its alive columns instead of
//    stepping rows N-2 and N-1 (37 % fewer steps at N=18).
//  * cols carries the off-board bits (~last) pre-set.  Then the free mask is
//    one LOP3 (~(cols|ld|rd)) with no `& last`, a completed board is
//    cols == 0xffffffff, and no depth counter is kept at all.
//  * Stack layout: slot s of lane l in warp w is the 16-byte entry at
//    w*levels*512 + s*512 + l*16.  Every stack access is a 128-bit LDS/STS and
//    the eight lanes of a quarter-warp always cover the 32 banks once,
//    whatever the per-lane depths are, so no access needs more wavefronts
//    than a dense 16-byte access of the warp (the reference mixes in a
//    32-bit store, src/n_queens_cuda.cu:47, which is 4-way conflicted).
//  * Tasks come from a device queue: one atomicAdd per warp refill hands a
//    block of consecutive queue positions to the idle lanes (the reference
//    takes one atomic per task per thread, :10,80).  An optional permutation
//    maps queue positions to tasks (longest-first schedules).
//  * Once the queue is empty, idle lanes take the bottom (shallowest, hence
//    largest) stacked level of a busy lane in the same warp: __ballot_sync
//    finds donors and receivers, __shfl_sync moves the donor's slot address,
//    and the receiver loads the entry straight from the donor's stack.
//  * Counts are uint32 per lane inside a bounded inner loop, folded into
//    uint64 per lane, reduced per warp (shuffles) and per CTA, and the last
//    CTA to finish sums the per-CTA partials in a fixed order.
//
// The kernel has no spin-wait of any kind: a lane never waits for another
// CTA or for host memory.  An optional %globaltimer deadline bounds its run.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nqb {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kSlotBytes = 512;  // one stack level of one warp: 32 lanes x 16 B
constexpr uint32_t kNoOwner = 0xffffffffu;

enum CtlWord : int {
    kCtlHead = 0,      // next queue position
    kCtlDone = 1,      // CTAs finished
    kCtlError = 2,     // error bits (kErr*)
    kCtlTimeout = 3,   // set when the deadline stopped the kernel
    kCtlCont = 4,      // continuation entries written at a deadline stop
    kCtlWords = 5,
};
enum : unsigned long long { kErrDepth = 1ull, kErrContOverflow = 2ull };
// Bits of *status_out: a task needed more stack levels than the launch had
// (it was skipped), and/or the run-time limit stopped the kernel early.
enum : unsigned long long { kStatDepth = 1ull, kStatTimeout = 2ull, kStatContOverflow = 4ull };

struct DfsParams {
    const uint32_t *cols;      // task column masks (reference `cur`)
    const uint32_t *ld;        // task left-diagonal masks (reference `left`)
    const uint32_t *rd;        // task right-diagonal masks (reference `right`)
    const uint8_t *task_n;     // per-task board size, or nullptr (use N)
    const uint32_t *owner_of;  // per-task output slot, or nullptr (slot = task index)
    const uint32_t *order;     // queue position -> task index, or nullptr (identity)
    long long ntasks;
    long long nqueue;          // queue positions to run (<= ntasks; 0 = ntasks)
    int N;                     // board size when task_n is nullptr
    int levels;                // stack slots per lane
    int inner;                 // DFS steps per outer trip (multiple of 4)
    int steal;                 // in-warp donation on/off
    unsigned long long limit_ns;     // run-time limit from the CTA's start, 0 = none
    unsigned long long *ctl;         // kCtlWords control words (zeroed before launch)
    unsigned long long *block_cnt;   // [gridDim.x] per-CTA count partials
    unsigned long long *block_nodes; // [gridDim.x] per-CTA node partials (NODES)
    unsigned long long *out_cnt;     // per-owner counts (PER_OWNER), zeroed by the host
    unsigned long long *out_nodes;   // per-owner nodes (PER_OWNER && NODES), zeroed by the host
    unsigned long long *sum_out;     // total count (device word)
    unsigned long long *nodes_out;   // total nodes (device word, NODES)
    unsigned long long *status_out;  // kStat* bits of this launch (device word)
    uint32_t k_one, k_two, k_mone;   // 1, 2, -1 (see dfs_step)
    unsigned long long *cta_times;   // optional [2*gridDim.x]: %globaltimer at CTA start and end
    int layout;                      // stack layout: 0 interleaved (default), 1 lane-major
    // Resumable runs.  Queue positions [0, n_cont_in) are continuation entries
    // (a lane's saved level: cols with the off-board bits set, ld, rd, untried
    // columns); position n_cont_in + j is task list position task_base + j.
    const uint4 *cont_in;
    const uint32_t *cont_in_owner;   // optional owners of the continuation entries
    long long n_cont_in;
    long long task_base;
    // At a deadline stop every lane writes its unfinished levels here (if not
    // null): the current level and each stacked level, in kCtlCont order.
    uint4 *cont_out;
    uint32_t *cont_out_owner;        // optional
    long long cont_cap;
    // Dihedral decomposition (DIH kernels only): class index per task and the
    // class table {popc threshold, row N-1 mask, tie column bit,
    // weight | tie weight << 16}; a child whose column mask (off-board bits
    // set) has more bits than the threshold may not use column 0 or N-1.
    const uint8_t *task_cls;
    const uint4 *cls_tab;
    uint32_t noside;                 // ~(column 0 | column N-1)
    // Resumable dihedral runs: the class index of each continuation entry
    // (in) and of each saved level (out).
    const uint8_t *cont_in_cls;
    uint8_t *cont_out_cls;
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ void lds128(uint32_t a, uint32_t &x, uint32_t &y, uint32_t &z, uint32_t &w) {
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(x), "=r"(y), "=r"(z), "=r"(w) : "r"(a) : "memory");
}

// One DFS step of one lane, branch-free.  State: (cols, ld, rd, avail) of the
// level being enumerated; sp/bot are the lane's stack top/bottom addresses.
//   bit   = lowest free column;  avail -= bit
//   child = (cols|bit, (ld|bit)<<1, (rd|bit)>>1),  free = ~(c|l|r)
//   child cols == ~0            -> one completed board: cnt += 1
//   free != 0 (and bit != 0)    -> descend; the parent is pushed only if
//                                  it still has untried columns
//   otherwise, level exhausted  -> pop a stacked level if there is one
// An idle lane (avail == 0, empty stack) passes through with no effect.
// Right shift is arithmetic, as in the reference's `int` arithmetic.
//
// Operands: %0 cols, %1 ld, %2 rd, %3 avail, %4 sp, %5 cnt, %6 placements
// (node statistics), %7 bot, %8 = 1, %9 = 2, %10 = -1, %11 the slot stride
// (512 B interleaved, 16 B lane-major).  The constants arrive as kernel
// parameters, so the compiler cannot fold the multiply-adds below back into
// ALU adds/moves.
//
// VAR 1 issues the adds, the left shift and the four register moves in
// multiply-add form (the FMA pipe), leaving the LOP3/shift/compare work on the
// ALU pipe: about 11 instructions on each pipe per step (an all-ALU form ran
// ~17 ALU + 7 FMA and was 20 % slower).
#define NQB_STEP_HEAD                                                                 \
    "{\n\t"                                                                           \
    ".reg .pred pb, pd, pp, pe, pq;\n\t"                                              \
    ".reg .b32 t, bit, nc, nl, nr, na;\n\t"

#define NQB_STEP_CHILD_VAR1                                                           \
    "mul.lo.s32 t, %3, %10;\n\t"                                                      \
    "and.b32 bit, t, %3;\n\t"                                                         \
    "setp.ne.u32 pb, bit, 0;\n\t"                                                     \
    "mad.lo.s32 %3, bit, %10, %3;\n\t"                                                \
    "mad.lo.s32 nc, bit, %8, %0;\n\t"                                                 \
    "or.b32 nl, %1, bit;\n\t"                                                         \
    "mul.lo.s32 nl, nl, %9;\n\t"                                                      \
    "or.b32 nr, %2, bit;\n\t"                                                         \
    "shr.s32 nr, nr, 1;\n\t"                                                          \
    "lop3.b32 na, nc, nl, nr, 0x01;\n\t"                                              \
    "setp.eq.u32 pe, nc, 0xffffffff;\n\t"                                             \
    "@pe mad.lo.s32 %5, %8, %8, %5;\n\t"

#define NQB_STEP_NODES_VAR1 "@pb mad.lo.s32 %6, %8, %8, %6;\n\t"

#define NQB_STEP_TAIL_VAR1                                                            \
    "setp.ne.and.u32 pd, na, 0, pb;\n\t"                                              \
    "setp.ne.and.u32 pp, %3, 0, pd;\n\t"                                              \
    "@pp st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"                                \
    "@pp mad.lo.s32 %4, %8, %11, %4;\n\t"                                             \
    "@pd mul.lo.s32 %0, nc, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %1, nl, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %2, nr, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %3, na, %8;\n\t"                                                  \
    "setp.eq.u32 pq, %3, 0;\n\t"                                                      \
    "setp.ne.and.u32 pq, %4, %7, pq;\n\t"                                             \
    "@pq mad.lo.s32 %4, %10, %11, %4;\n\t"                                            \
    "@pq ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"                                \
    "}\n\t"

// VAR 3 keeps a level's left-diagonal mask pre-shifted for its children
// (register ld holds left << 1), so a child's left mask is one multiply-add,
// (left | bit) << 1 = ld + 2*bit (bit is free, so | equals +), and the shift
// for the grandchildren rides on the descend move (x 2 instead of x 1).  The
// right diagonal stays in the reference's form: a right shift has no
// multiply-add form, and a multiply-high in its place loaded the FMA pipe
// more than the two ALU operations it saved (measured 5-7 % slower).  The
// predicates come from LOP3's predicate output (p = (result != 0) op q)
// instead of separate compares:
//   lop3.and bit|pb      bit = avail & -avail,  pb = bit != 0
//   lop3.and na|pd       na = ~(c|l|r),         pd = na != 0 && pb    (descend)
//   lop3.or  avail|pk    avail ^= bit,          pk = avail != 0 || pd (level goes on)
//   setp pp = avail != 0 && pd (push),  setp pq = sp != bot && !pk (pop)
// 20 instructions per step (9 ALU, 9 FMA pipe, 2 shared) against VAR 1's 24,
// same stack traffic.  Four steps share one asm block, whose head sets the
// constant predicate `pt1` (true) once.  Operands as in VAR 1.
#define NQB_STEP3_HEAD                                                                \
    "{\n\t"                                                                           \
    ".reg .pred pt1, pb, pd, pk, pp, pe, pq;\n\t"                                     \
    ".reg .b32 t, bit, nc, nl, nr, na;\n\t"                                           \
    "setp.ne.u32 pt1, %8, 0;\n\t"

#define NQB_STEP3_CHILD                                                               \
    "mul.lo.s32 t, %3, %10;\n\t"                                                      \
    "lop3.and.b32 bit|pb, t, %3, 0, 0xC0, pt1;\n\t"                                   \
    "mad.lo.s32 nc, bit, %8, %0;\n\t"                                                 \
    "mad.lo.s32 nl, bit, %9, %1;\n\t"                                                 \
    "or.b32 nr, %2, bit;\n\t"                                                         \
    "shr.s32 nr, nr, 1;\n\t"                                                          \
    "lop3.and.b32 na|pd, nc, nl, nr, 0x01, pb;\n\t"                                   \
    "lop3.or.b32 %3|pk, %3, bit, 0, 0x3C, pd;\n\t"                                    \
    "setp.eq.u32 pe, nc, 0xffffffff;\n\t"                                             \
    "@pe add.u32 %5, %5, 1;\n\t"

#define NQB_STEP3_TAIL                                                                \
    "setp.ne.and.u32 pp, %3, 0, pd;\n\t"                                              \
    "@pp st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"                                \
    "@pp mad.lo.s32 %4, %8, %11, %4;\n\t"                                             \
    "@pd mul.lo.s32 %0, nc, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %1, nl, %9;\n\t"                                                  \
    "@pd mul.lo.s32 %2, nr, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %3, na, %8;\n\t"                                                  \
    "setp.ne.and.u32 pq, %4, %7, !pk;\n\t"                                            \
    "@pq mad.lo.s32 %4, %10, %11, %4;\n\t"                                            \
    "@pq ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"

#define NQB_STEP3 NQB_STEP3_CHILD NQB_STEP3_TAIL
#define NQB_STEP3_NODES NQB_STEP3_CHILD NQB_STEP_NODES_VAR1 NQB_STEP3_TAIL
#define NQB_STEP3_X4 NQB_STEP3 NQB_STEP3 NQB_STEP3 NQB_STEP3
#define NQB_STEP3_NODES_X4 NQB_STEP3_NODES NQB_STEP3_NODES NQB_STEP3_NODES NQB_STEP3_NODES

// VAR 4 ("filtered") enumerates only children that have a future.  A child C
// of the level (placed at column `bit`) lists the columns of the next row it
// may try (free = ~(c|l|r)); such a column b is dead when the row after it
// would have no free column at all.  With F0 = the free columns of that row
// before b is placed (~(c | l<<1 | r>>1)), b is dead exactly when F0 lies
// inside {b-1, b, b+1}, i.e. when no column of F0 is two or more away from
// b.  The alive columns are therefore
//   (columns >= lowest(F0) + 2) | (columns <= highest(F0) - 2)
//   = -(lo << 2) | (0x3fffffff >> bfind.shiftamt(F0))       (empty when F0 = 0)
// (bfind.shiftamt is 31 - the highest set bit's position, all ones for 0, and a
// shift by 32 or more gives 0).
// and the child's list becomes free & that mask.  A child on row N-2 (its
// column mask has 30 bits set, off-board bits included) is not entered: every
// alive column of it completes the board on row N-1, so the step adds the
// popcount of its filtered list.  Rows N-2 and N-1 are never stepped and dead
// children never cost a step or a stack push: at N=18, k=6 the steps fall from
// 29.7e9 to 18.6e9 and the pushes from 7.8e9 to 5.0e9, for 32 instructions per
// step instead of 20.  Tasks and saved levels on rows N-2 and N-1 are counted
// when they are loaded.  Lane registers as in VAR 3.  Operands as in VAR 1
// plus %12 = 0x3fffffff, %13 = -4, %14 = 30.  Pipe balance (N=21, measured):
// taking the highest bit's mask from bfind's shift amount instead of a
// multiply-add saved 4.2 %, negating F0 on the ALU instead of the FMA pipe
// 0.3 %; moving the count or the first negation to the ALU pipe did not help.
#define NQB_STEP4_HEAD                                                                \
    "{\n\t"                                                                           \
    ".reg .pred pt1, pb, pg, p2, pd, pk, pp, pq;\n\t"                                 \
    ".reg .b32 t, bit, nc, nl, nr, na, xl, xr, f0, lo, ma, mb, pos, pc, naf;\n\t"     \
    "setp.ne.u32 pt1, %8, 0;\n\t"

#define NQB_STEP4                                                                     \
    "mul.lo.s32 t, %3, %10;\n\t"                                                      \
    "lop3.and.b32 bit|pb, t, %3, 0, 0xC0, pt1;\n\t"                                   \
    "mad.lo.s32 nc, bit, %8, %0;\n\t"                                                 \
    "mad.lo.s32 nl, bit, %9, %1;\n\t"                                                 \
    "or.b32 nr, %2, bit;\n\t"                                                         \
    "shr.s32 nr, nr, 1;\n\t"                                                          \
    "lop3.b32 na, nc, nl, nr, 0x01;\n\t"                                              \
    "mul.lo.s32 xl, nl, %9;\n\t"                                                      \
    "shr.s32 xr, nr, 1;\n\t"                                                          \
    "lop3.b32 f0, nc, xl, xr, 0x01;\n\t"                                              \
    "neg.s32 t, f0;\n\t"                                                              \
    "and.b32 lo, t, f0;\n\t"                                                          \
    "mul.lo.s32 ma, lo, %13;\n\t"                                                     \
    "bfind.shiftamt.u32 pos, f0;\n\t"                                                 \
    "shr.b32 mb, %12, pos;\n\t"                                                       \
    "popc.b32 pc, nc;\n\t"                                                            \
    "setp.ne.and.u32 pg, pc, %14, pb;\n\t"                                            \
    "setp.eq.and.u32 p2, pc, %14, pb;\n\t"                                            \
    "lop3.and.b32 naf|pd, na, ma, mb, 0xE0, pg;\n\t"                                  \
    "popc.b32 t, naf;\n\t"                                                            \
    "@p2 mad.lo.s32 %5, t, %8, %5;\n\t"                                               \
    "lop3.or.b32 %3|pk, %3, bit, 0, 0x3C, pd;\n\t"                                    \
    "setp.ne.and.u32 pp, %3, 0, pd;\n\t"                                              \
    "@pp st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"                                \
    "@pp mad.lo.s32 %4, %8, %11, %4;\n\t"                                             \
    "@pd mul.lo.s32 %0, nc, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %1, xl, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %2, nr, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %3, naf, %8;\n\t"                                                 \
    "setp.ne.and.u32 pq, %4, %7, !pk;\n\t"                                            \
    "@pq mad.lo.s32 %4, %10, %11, %4;\n\t"                                            \
    "@pq ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"

#define NQB_STEP4_X4 NQB_STEP4 NQB_STEP4 NQB_STEP4 NQB_STEP4

// Dihedral step: the VAR 1 step plus the class rules of the lane's task.
//   pc = popc(child cols) = 32 - N + child row
//   pc > %12            -> the child row may not use the side columns, and
//                          when it is row N-1 (pc == 31) only %13's columns
//   child cols == ~0    -> one completion of weight %16 if the row N-1 queen
//                          is at %14, else %15
// Operands %0-%11 as in the plain step; %12 popc threshold, %13 row N-1
// mask, %14 tie column bit, %15 weight, %16 tie weight, %17 ~side columns.
#define NQB_STEP_HEAD_DIH                                                             \
    "{\n\t"                                                                           \
    ".reg .pred pb, pd, pp, pe, pq, ps, pl, px;\n\t"                                  \
    ".reg .b32 t, bit, nc, nl, nr, na, pc, msk, w;\n\t"

#define NQB_STEP_CHILD_DIH                                                            \
    "mul.lo.s32 t, %3, %10;\n\t"                                                      \
    "and.b32 bit, t, %3;\n\t"                                                         \
    "setp.ne.u32 pb, bit, 0;\n\t"                                                     \
    "mad.lo.s32 %3, bit, %10, %3;\n\t"                                                \
    "mad.lo.s32 nc, bit, %8, %0;\n\t"                                                 \
    "or.b32 nl, %1, bit;\n\t"                                                         \
    "mul.lo.s32 nl, nl, %9;\n\t"                                                      \
    "or.b32 nr, %2, bit;\n\t"                                                         \
    "shr.s32 nr, nr, 1;\n\t"                                                          \
    "lop3.b32 na, nc, nl, nr, 0x01;\n\t"                                              \
    "popc.b32 pc, nc;\n\t"                                                            \
    "setp.gt.u32 ps, pc, %12;\n\t"                                                    \
    "setp.eq.u32 pl, pc, 31;\n\t"                                                     \
    "selp.b32 msk, %13, %17, pl;\n\t"                                                 \
    "@ps and.b32 na, na, msk;\n\t"                                                    \
    "setp.eq.u32 pe, nc, 0xffffffff;\n\t"                                             \
    "setp.eq.u32 px, bit, %14;\n\t"                                                   \
    "selp.b32 w, %16, %15, px;\n\t"                                                   \
    "@pe add.u32 %5, %5, w;\n\t"

// The dihedral step in the filtered form (the dihedral kernels' default when
// the count kernels run VAR 4): the left diagonal pre-shifted as in VAR 3, and
// each child's list cut to its alive columns (those whose next row keeps a free
// column, ignoring the class rules -- the rules only remove columns, so this
// drops dead children only) except on row N-1, whose columns complete the
// board.  Rows N-2 and N-1 are still stepped, because the class rules and the
// tie weight decide what their completions count.  Operands as in the
// dihedral step above.
#define NQB_STEP_HEAD_DIH4                                                            \
    "{\n\t"                                                                           \
    ".reg .pred pb, pd, pp, pe, pq, pq0, ps, pl, px;\n\t"                              \
    ".reg .b32 t, bit, nc, nl, nr, na, pc, msk, w, xl, xr, f0, lo, ma, mb, pos;\n\t"  \

#define NQB_STEP_DIH4                                                                 \
    "mul.lo.s32 t, %3, %10;\n\t"                                                      \
    "and.b32 bit, t, %3;\n\t"                                                         \
    "setp.ne.u32 pb, bit, 0;\n\t"                                                     \
    "mad.lo.s32 %3, bit, %10, %3;\n\t"                                                \
    "mad.lo.s32 nc, bit, %8, %0;\n\t"                                                 \
    "mad.lo.s32 nl, bit, %9, %1;\n\t"                                                 \
    "or.b32 nr, %2, bit;\n\t"                                                         \
    "shr.s32 nr, nr, 1;\n\t"                                                          \
    "lop3.b32 na, nc, nl, nr, 0x01;\n\t"                                              \
    "popc.b32 pc, nc;\n\t"                                                            \
    "setp.gt.u32 ps, pc, %12;\n\t"                                                    \
    "setp.eq.u32 pl, pc, 31;\n\t"                                                     \
    "selp.b32 msk, %13, %17, pl;\n\t"                                                 \
    "@ps and.b32 na, na, msk;\n\t"                                                    \
    "mul.lo.s32 xl, nl, %9;\n\t"                                                      \
    "shr.s32 xr, nr, 1;\n\t"                                                          \
    "lop3.b32 f0, nc, xl, xr, 0x01;\n\t"                                              \
    "mul.lo.s32 t, f0, %10;\n\t"                                                      \
    "and.b32 lo, t, f0;\n\t"                                                          \
    "mul.lo.s32 ma, lo, -4;\n\t"                                                      \
    "bfind.u32 pos, f0;\n\t"                                                          \
    "mad.lo.s32 pos, pos, %10, 33;\n\t"                                               \
    "shr.b32 mb, %10, pos;\n\t"                                                       \
    "@!pl lop3.b32 na, na, ma, mb, 0xE0;\n\t"                                         \
    "setp.ne.and.u32 pd, na, 0, pb;\n\t"                                              \
    "setp.eq.u32 pe, nc, 0xffffffff;\n\t"                                             \
    "setp.eq.u32 px, bit, %14;\n\t"                                                   \
    "selp.b32 w, %16, %15, px;\n\t"                                                   \
    "@pe mad.lo.s32 %5, w, %8, %5;\n\t"                                               \
    "setp.ne.and.u32 pp, %3, 0, pd;\n\t"                                              \
    "setp.eq.and.u32 pq0, %3, 0, !pd;\n\t"                                            \
    "@pp st.shared.v4.u32 [%4], {%0, %1, %2, %3};\n\t"                                \
    "@pp mad.lo.s32 %4, %8, %11, %4;\n\t"                                             \
    "@pd mul.lo.s32 %0, nc, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %1, xl, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %2, nr, %8;\n\t"                                                  \
    "@pd mul.lo.s32 %3, na, %8;\n\t"                                                  \
    "setp.ne.and.u32 pq, %4, %7, pq0;\n\t"                                            \
    "@pq mad.lo.s32 %4, %10, %11, %4;\n\t"                                            \
    "@pq ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n\t"                                \
    "}\n\t"

// Class registers of a lane in a DIH kernel (cls: the class index, kept for
// the deadline dump of resumable runs).
struct DihLane {
    uint32_t side_popc = 64u, last_mask = ~0u, tie_bit = 0u, w = 0u, w_tie = 0u, cls = 0u;
};

struct StepConsts {
    uint32_t one, two, mone, stride;  // stride: bytes between a lane's consecutive stack slots
};

// Step variant of the count kernels: 4 = filtered children (default), 3 =
// pre-shifted left diagonal with LOP3 predicate outputs, 1 = the reference's
// mask form with IMAD-form moves.  Kernels that count DFS nodes (NODES) step
// every placement, so they run variant 3 when 4 is chosen; the dihedral
// kernels run their own filtered step (NQB_STEP_DIH4) with 4, else variant 1.
#ifndef NQB_STEP_VAR
#define NQB_STEP_VAR 4
#endif
constexpr int kStepVar = NQB_STEP_VAR;
static_assert(kStepVar == 1 || kStepVar == 3 || kStepVar == 4, "step variant");
constexpr int kNodesStepVar = kStepVar == 4 ? 3 : kStepVar;
constexpr int kDihStepVar = kStepVar == 4 ? 4 : 1;

// Stack rows a step variant never pushes beyond the reference's N-1-rows: the
// filtered step enters no level on row N-2 or N-1, so the deepest level it
// pushes is on row N-4.
template <int VAR>
constexpr int kStackRowsSpared = VAR == 4 ? 2 : 0;

// Lane registers (ld, rd) from the reference's (left, right) masks of the row
// a level enumerates, and back (for the checkpoint file, which stores the
// reference's form).  Going back loses left's bit 31, which no later row can
// see (a left bit only moves further left).
template <int VAR>
__device__ __forceinline__ uint32_t lane_ld(uint32_t left) { return VAR >= 3 ? left << 1 : left; }
template <int VAR>
__device__ __forceinline__ uint32_t ref_ld(uint32_t ld) { return VAR >= 3 ? ld >> 1 : ld; }

// The alive part of a level's untried columns (VAR 4): drops every column
// whose child would leave the next row without a free column.  ld in lane
// form (pre-shifted), rd in the reference's form.
__device__ __forceinline__ uint32_t alive_columns(uint32_t cols, uint32_t ld, uint32_t rd, uint32_t avail) {
    const uint32_t f0 = ~(cols | ld | (uint32_t)((int32_t)rd >> 1));
    if (f0 == 0) return 0;
    const uint32_t lo = f0 & (0u - f0);
    const int hi = 31 - __clz(f0);
    const uint32_t above = 0u - (lo << 2);                              // columns >= lowest + 2
    const uint32_t below = hi >= 2 ? (0xffffffffu >> (33 - hi)) : 0u;  // columns <= highest - 2
    return avail & (above | below);
}

template <bool NODES, int VAR>
__device__ __forceinline__ void dfs_step(uint32_t &cols, uint32_t &ld, uint32_t &rd, uint32_t &avail, uint32_t &sp,
                                         uint32_t &cnt, uint32_t &it, uint32_t bot, const StepConsts &k) {
    static_assert(VAR == 1, "VAR 3 and 4 run in groups (dfs_steps3, dfs_steps4)");
    if (NODES)
        asm volatile(NQB_STEP_HEAD NQB_STEP_CHILD_VAR1 NQB_STEP_NODES_VAR1 NQB_STEP_TAIL_VAR1
                     : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                     : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride)
                     : "memory");
    else
        asm volatile(NQB_STEP_HEAD NQB_STEP_CHILD_VAR1 NQB_STEP_TAIL_VAR1
                     : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                     : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride)
                     : "memory");
}

template <int VAR>
__device__ __forceinline__ void dfs_step_dih(uint32_t &cols, uint32_t &ld, uint32_t &rd, uint32_t &avail, uint32_t &sp,
                                             uint32_t &cnt, uint32_t &it, uint32_t bot, const StepConsts &k,
                                             const DihLane &d, uint32_t noside) {
    static_assert(VAR == 1 || VAR == 4, "dihedral step variants: 1 (reference form) and 4 (filtered)");
    if constexpr (VAR == 4)
        asm volatile(NQB_STEP_HEAD_DIH4 NQB_STEP_DIH4
                     : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                     : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride), "r"(d.side_popc),
                       "r"(d.last_mask), "r"(d.tie_bit), "r"(d.w), "r"(d.w_tie), "r"(noside)
                     : "memory");
    else
        asm volatile(NQB_STEP_HEAD_DIH NQB_STEP_CHILD_DIH NQB_STEP_TAIL_VAR1
                     : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                     : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride), "r"(d.side_popc),
                       "r"(d.last_mask), "r"(d.tie_bit), "r"(d.w), "r"(d.w_tie), "r"(noside)
                     : "memory");
}

// UNROLL steps of VAR 3 (UNROLL a multiple of 4), four per asm block.
template <bool NODES, int UNROLL>
__device__ __forceinline__ void dfs_steps3(uint32_t &cols, uint32_t &ld, uint32_t &rd, uint32_t &avail, uint32_t &sp,
                                           uint32_t &cnt, uint32_t &it, uint32_t bot, const StepConsts &k) {
    static_assert(UNROLL % 4 == 0, "VAR 3 unrolls in groups of 4");
#pragma unroll
    for (int g = 0; g < UNROLL / 4; ++g) {
        if (NODES)
            asm volatile(NQB_STEP3_HEAD NQB_STEP3_NODES_X4 "}\n\t"
                         : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                         : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride)
                         : "memory");
        else
            asm volatile(NQB_STEP3_HEAD NQB_STEP3_X4 "}\n\t"
                         : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt), "+r"(it)
                         : "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride)
                         : "memory");
    }
}

// UNROLL steps of VAR 4 (no NODES form), four per asm block.  Operand %6 is
// unused (it stands where the node counter sits in the other forms).
template <int UNROLL>
__device__ __forceinline__ void dfs_steps4(uint32_t &cols, uint32_t &ld, uint32_t &rd, uint32_t &avail, uint32_t &sp,
                                           uint32_t &cnt, uint32_t bot, const StepConsts &k) {
    static_assert(UNROLL % 4 == 0, "VAR 4 unrolls in groups of 4");
#pragma unroll
    for (int g = 0; g < UNROLL / 4; ++g)
        asm volatile(NQB_STEP4_HEAD NQB_STEP4_X4 "}\n\t"
                     : "+r"(cols), "+r"(ld), "+r"(rd), "+r"(avail), "+r"(sp), "+r"(cnt)
                     : "r"(0u), "r"(bot), "r"(k.one), "r"(k.two), "r"(k.mone), "r"(k.stride), "r"(0x3fffffffu),
                       "r"(0xfffffffcu), "r"(30u)
                     : "memory");
}

__device__ __forceinline__ void load_class_index(const DfsParams &p, uint32_t idx, DihLane &d) {
    const uint4 c = __ldg(p.cls_tab + idx);
    d.cls = idx;
    d.side_popc = c.x;
    d.last_mask = c.y;
    d.tie_bit = c.z;
    d.w = c.w & 0xffffu;
    d.w_tie = c.w >> 16;
}

__device__ __forceinline__ void load_class(const DfsParams &p, long long t, DihLane &d) {
    load_class_index(p, __ldg(p.task_cls + t), d);
}

// VAR 4 keeps only levels on rows 0..N-3, with their alive columns.  A level
// on row N-1 (one column left) completes once per free column; on row N-2
// once per alive column.  Returns those completions and leaves avail = 0 for
// such levels; otherwise filters avail and returns 0.
__device__ __forceinline__ uint32_t settle_level(int n, uint32_t cols, uint32_t ld, uint32_t rd, uint32_t &avail) {
    const int row = __popc(cols) - (32 - n);
    if (row >= n - 1) {
        const uint32_t done = __popc(avail);
        avail = 0;
        return done;
    }
    avail = alive_columns(cols, ld, rd, avail);
    if (row == n - 2) {
        const uint32_t done = __popc(avail);
        avail = 0;
        return done;
    }
    return 0;
}

// Loads task t into a lane.  Returns the completions credited immediately
// (1 for an already-complete board) and leaves avail == 0 when the task has
// no free column.  A column mask with off-board bits can never equal `last`,
// so such a task counts 0, exactly as the reference recursion does.
template <int VAR>
__device__ __forceinline__ uint32_t load_task(const DfsParams &p, long long t, uint32_t &cols, uint32_t &ld,
                                              uint32_t &rd, uint32_t &avail) {
    const int n = p.task_n ? (int)p.task_n[t] : p.N;
    const uint32_t last = (n >= 32) ? kFull : ((1u << n) - 1u);
    const uint32_t c = __ldg(p.cols + t);
    const uint32_t l = __ldg(p.ld + t);
    const uint32_t r = __ldg(p.rd + t);
    avail = 0;
    if (c & ~last) return 0;
    if (c == last) return 1;
    // Stack slots this task can use: one per level that still has a sibling,
    // at most N-1-popc(cols) -- N-3-popc(cols) for the filtered step, which
    // never enters rows N-2 and N-1.
    const int need = n - 1 - __popc(c) - kStackRowsSpared<VAR>;
    if (need > p.levels) {
        atomicOr(p.ctl + kCtlError, kErrDepth);
        return 0;
    }
    cols = c | ~last;
    ld = lane_ld<VAR>(l);
    rd = r;
    avail = ~(cols | l | r);
    if (VAR == 4) return settle_level(n, cols, ld, rd, avail);
    return 0;
}

// RESUME adds the continuation queue and the deadline dump; it is a separate
// instantiation so that the plain count kernel carries none of that code
// (it measurably changed the code generated for the DFS loop).
// DIH runs the dihedral decomposition: every task carries a class (rules and
// weights, see DfsParams::cls_tab) and the step is dfs_step_dih.
template <bool PER_OWNER, bool NODES, int VAR, int UNROLL, bool RESUME = false, bool DIH = false>
__global__ void __launch_bounds__(1024) dfs_kernel(DfsParams p) {
    static_assert(!(VAR == 4 && NODES), "the filtered step counts no nodes");
    static_assert(!DIH || VAR == 1 || VAR == 4, "dihedral step variants: 1 and 4");
    // Lane registers and task loading of the step: the dihedral filtered step
    // keeps VAR 3's lane form and steps rows N-2 and N-1 (no settling).
    constexpr int LVAR = (DIH && VAR == 4) ? 3 : VAR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long red_cnt[32];
    __shared__ unsigned long long red_nodes[32];
    __shared__ int s_is_last;

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t smem_base = (uint32_t)__cvta_generic_to_shared(smem_raw);
    // Stack layout 0 (interleaved): slot s of lane l at warp_base + s*512 + l*16,
    // conflict-free for every mix of depths.  Layout 1 (lane-major): each
    // lane's slots contiguous, lane_base + s*16 (kept for the autotuner).
    const uint32_t stride = p.layout == 1 ? 16u : kSlotBytes;
    const uint32_t my_base = p.layout == 1
                                 ? smem_base + (warp * 32u + lane) * (uint32_t)p.levels * 16u
                                 : smem_base + warp * (uint32_t)p.levels * kSlotBytes + lane * 16u;

    if (p.cta_times && threadIdx.x == 0) p.cta_times[2 * blockIdx.x] = globaltimer_ns();
    const StepConsts kc{p.k_one, p.k_two, p.k_mone, stride};
    uint32_t cols = 0, ld = 0, rd = 0, avail = 0;
    uint32_t sp = my_base, bot = my_base;
    uint32_t cnt = 0, it = 0;
    uint32_t owner = kNoOwner;
    DihLane dih;
    unsigned long long tot = 0, tot_nodes = 0;
    const long long qlen = RESUME ? p.n_cont_in + p.ntasks - p.task_base : (p.nqueue > 0 ? p.nqueue : p.ntasks);
    bool queue_live = qlen > 0;
    bool timed_out = false;
    unsigned long long deadline = 0;
    if (p.limit_ns) {
        unsigned long long t0 = 0;
        if (lane == 0) t0 = globaltimer_ns();
        deadline = __shfl_sync(kFull, t0, 0) + p.limit_ns;
    }

    for (;;) {
        // ---- fold the per-lane 32-bit counters (bounded inner loop keeps them < 2^32)
        if (PER_OWNER) {
            if (avail == 0 && owner != kNoOwner) {
                if (cnt) atomicAdd(p.out_cnt + owner, (unsigned long long)cnt);
                if (NODES && it) atomicAdd(p.out_nodes + owner, (unsigned long long)(it - cnt));
                tot += cnt;
                if (NODES) tot_nodes += it - cnt;
                cnt = 0;
                it = 0;
                owner = kNoOwner;
            }
        } else {
            tot += cnt;
            if (NODES) tot_nodes += it - cnt;
            cnt = 0;
            it = 0;
        }

        // ---- deadline (lane 0 reads the timer; the decision is warp-uniform)
        if (deadline) {
            unsigned long long now = 0;
            if (lane == 0) now = globaltimer_ns();
            now = __shfl_sync(kFull, now, 0);
            if (now > deadline) {
                if (lane == 0) atomicExch(p.ctl + kCtlTimeout, 1ull);
                if (RESUME) timed_out = true;
                break;
            }
        }

        unsigned idle = __ballot_sync(kFull, avail == 0);
        bool check_idle = true;
        if (idle) {
            if (queue_live) {
                // ---- refill from the queue: one atomic per warp
                const int nidle = __popc(idle);
                const int leader = __ffs(idle) - 1;
                unsigned long long b = 0;
                if ((int)lane == leader) b = atomicAdd(p.ctl + kCtlHead, (unsigned long long)nidle);
                b = __shfl_sync(kFull, b, leader);
                if (b + (unsigned long long)nidle >= (unsigned long long)qlen) queue_live = false;
                if (avail == 0) {
                    const unsigned long long q = b + (unsigned long long)__popc(idle & lanemask_lt());
                    if (RESUME && q < (unsigned long long)p.n_cont_in) {
                        // a level saved by an earlier, interrupted run
                        sp = bot = my_base;
                        const uint4 e = p.cont_in[q];
                        const int need = __popc(~e.x) - 1 - kStackRowsSpared<LVAR>;
                        if (need > p.levels) {
                            atomicOr(p.ctl + kCtlError, kErrDepth);
                        } else {
                            cols = e.x;
                            ld = lane_ld<LVAR>(e.y);
                            rd = e.z;
                            avail = e.w;
                            // a level saved on row N-2 or N-1 (by a kernel that steps those rows)
                            if (VAR == 4 && !DIH) tot += settle_level(p.N, cols, ld, rd, avail);
                            // a saved level already carries its class's rules in avail
                            if (DIH) load_class_index(p, p.cont_in_cls[q], dih);
                            if (PER_OWNER && avail) owner = p.cont_in_owner ? p.cont_in_owner[q] : 0u;
                        }
                    } else if (q < (unsigned long long)qlen) {
                        const long long pos =
                            RESUME ? p.task_base + (long long)(q - (unsigned long long)p.n_cont_in) : (long long)q;
                        const long long t = p.order ? (long long)__ldg(p.order + pos) : pos;
                        // A permutation entry out of range is skipped, never dereferenced.
                        if (t >= 0 && t < p.ntasks) {
                            sp = bot = my_base;
                            uint32_t done = load_task<LVAR>(p, t, cols, ld, rd, avail);
                            if (DIH) {
                                load_class(p, t, dih);
                                done *= dih.w;
                                // The task's own row follows the class rules too
                                // (the step applies them to children only).
                                const uint32_t pc = (uint32_t)__popc(cols);
                                if (avail && pc > dih.side_popc) avail &= pc == 31u ? dih.last_mask : p.noside;
                            }
                            const uint32_t own = p.owner_of ? __ldg(p.owner_of + t) : (uint32_t)t;
                            if (PER_OWNER) {
                                if (done) atomicAdd(p.out_cnt + own, (unsigned long long)done);
                                if (avail) owner = own;
                            }
                            tot += done;
                        }
                    }
                }
                // Lanes whose task was empty are still idle: refill again.
                if (queue_live) continue;
                idle = __ballot_sync(kFull, avail == 0);
            }
            if (idle && !queue_live) {
                if (p.steal) {
                    // ---- in-warp donation: k-th idle lane takes the bottom
                    // stacked level of the k-th lane that has one.
                    const unsigned rich = __ballot_sync(kFull, sp != bot);
                    __syncwarp();  // order the donors' earlier stack stores before the reads below
                    const int npair = min(__popc(idle), __popc(rich));
                    if (npair > 0) {
                        int donor = -1;
                        if (avail == 0) {
                            const int k = __popc(idle & lanemask_lt());
                            if (k < npair) {
                                unsigned m = rich;
                                for (int i = 0; i < k; ++i) m &= m - 1;
                                donor = __ffs(m) - 1;
                            }
                        }
                        const uint32_t src_addr = __shfl_sync(kFull, bot, donor < 0 ? lane : donor);
                        const uint32_t src_owner = __shfl_sync(kFull, owner, donor < 0 ? lane : donor);
                        DihLane src_dih;
                        if (DIH) {
                            const int src = donor < 0 ? (int)lane : donor;
                            src_dih.side_popc = __shfl_sync(kFull, dih.side_popc, src);
                            src_dih.last_mask = __shfl_sync(kFull, dih.last_mask, src);
                            src_dih.tie_bit = __shfl_sync(kFull, dih.tie_bit, src);
                            src_dih.w = __shfl_sync(kFull, dih.w, src);
                            src_dih.w_tie = __shfl_sync(kFull, dih.w_tie, src);
                            if (RESUME) src_dih.cls = __shfl_sync(kFull, dih.cls, src);
                        }
                        if (donor >= 0) {
                            lds128(src_addr, cols, ld, rd, avail);
                            sp = bot = my_base;
                            owner = src_owner;
                            if (DIH) dih = src_dih;
                        }
                        __syncwarp();
                        if (sp != bot && __popc(rich & lanemask_lt()) < npair) bot += stride;
                        __syncwarp();
                    } else {
                        // Nobody can donate right now: run a full trip
                        // without idle checks, then look again.
                        if (idle == kFull) break;  // whole warp idle, queue empty: done
                        check_idle = false;
                    }
                } else {
                    if (idle == kFull) break;
                    check_idle = false;
                }
            }
        }

        // ---- DFS steps
        if (check_idle) {
            for (int s = 0; s < p.inner; s += UNROLL) {
#pragma unroll
                for (int u = 0; u < (VAR >= 3 && !DIH ? 1 : UNROLL); ++u) {
                    if constexpr (DIH)
                        dfs_step_dih<VAR>(cols, ld, rd, avail, sp, cnt, it, bot, kc, dih, p.noside);
                    else if constexpr (VAR == 4)
                        dfs_steps4<UNROLL>(cols, ld, rd, avail, sp, cnt, bot, kc);
                    else if constexpr (VAR == 3)
                        dfs_steps3<NODES, UNROLL>(cols, ld, rd, avail, sp, cnt, it, bot, kc);
                    else
                        dfs_step<NODES, VAR>(cols, ld, rd, avail, sp, cnt, it, bot, kc);
                }
                if (__any_sync(kFull, avail == 0)) break;
            }
        } else {
            for (int s = 0; s < p.inner; s += UNROLL) {
#pragma unroll
                for (int u = 0; u < (VAR >= 3 && !DIH ? 1 : UNROLL); ++u) {
                    if constexpr (DIH)
                        dfs_step_dih<VAR>(cols, ld, rd, avail, sp, cnt, it, bot, kc, dih, p.noside);
                    else if constexpr (VAR == 4)
                        dfs_steps4<UNROLL>(cols, ld, rd, avail, sp, cnt, bot, kc);
                    else if constexpr (VAR == 3)
                        dfs_steps3<NODES, UNROLL>(cols, ld, rd, avail, sp, cnt, it, bot, kc);
                    else
                        dfs_step<NODES, VAR>(cols, ld, rd, avail, sp, cnt, it, bot, kc);
                }
                if (__all_sync(kFull, avail == 0)) break;
            }
        }
    }

    // Deadline stop: save every unfinished level so a later run can resume.
    // The current level keeps its untried columns; every stacked level does
    // too (only levels with untried columns are ever pushed).
    if (RESUME && timed_out && p.cont_out) {
        const uint32_t nstk = (sp - bot) / stride;
        const uint32_t mine = (avail != 0 ? 1u : 0u) + nstk;
        unsigned long long at = 0;
        if (mine) at = atomicAdd(p.ctl + kCtlCont, (unsigned long long)mine);
        if (mine && at + mine > (unsigned long long)p.cont_cap) {
            atomicOr(p.ctl + kCtlError, kErrContOverflow);
        } else if (mine) {
            if (avail) {
                p.cont_out[at] = make_uint4(cols, ref_ld<LVAR>(ld), rd, avail);
                if (p.cont_out_owner) p.cont_out_owner[at] = owner;
                if (DIH) p.cont_out_cls[at] = (uint8_t)dih.cls;
                ++at;
            }
            for (uint32_t a = bot; a != sp; a += stride, ++at) {
                uint32_t x, y, z, w;
                lds128(a, x, y, z, w);
                p.cont_out[at] = make_uint4(x, ref_ld<LVAR>(y), z, w);
                if (p.cont_out_owner) p.cont_out_owner[at] = owner;
                if (DIH) p.cont_out_cls[at] = (uint8_t)dih.cls;
            }
        }
    }

    // CTA finish time: the last warp of the CTA to leave the DFS loop.
    if (p.cta_times) atomicMax(p.cta_times + 2 * blockIdx.x + 1, globaltimer_ns());

    // Flush what the last trip left (deadline exit, or the final fold).
    if (PER_OWNER) {
        if (owner != kNoOwner) {
            if (cnt) atomicAdd(p.out_cnt + owner, (unsigned long long)cnt);
            if (NODES && it) atomicAdd(p.out_nodes + owner, (unsigned long long)(it - cnt));
        }
    }
    tot += cnt;
    if (NODES) tot_nodes += it - cnt;

    // ---- per-warp, per-CTA reduction
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tot += __shfl_xor_sync(kFull, tot, o);
        if (NODES) tot_nodes += __shfl_xor_sync(kFull, tot_nodes, o);
    }
    if (lane == 0) {
        red_cnt[warp] = tot;
        red_nodes[warp] = tot_nodes;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0, sn = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
            s += red_cnt[w];
            sn += red_nodes[w];
        }
        p.block_cnt[blockIdx.x] = s;
        if (NODES) p.block_nodes[blockIdx.x] = sn;
        __threadfence();
        const unsigned long long ticket = atomicAdd(p.ctl + kCtlDone, 1ull);
        s_is_last = (ticket == (unsigned long long)gridDim.x - 1ull);
    }
    __syncthreads();
    // ---- the last CTA sums the per-CTA partials in CTA order
    if (s_is_last) {
        __threadfence();
        unsigned long long s = 0, sn = 0;
        for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            s += *((volatile unsigned long long *)(p.block_cnt + b));
            if (NODES) sn += *((volatile unsigned long long *)(p.block_nodes + b));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(kFull, s, o);
            if (NODES) sn += __shfl_xor_sync(kFull, sn, o);
        }
        __syncthreads();
        if (lane == 0) {
            red_cnt[warp] = s;
            red_nodes[warp] = sn;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long a = 0, an = 0;
            for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
                a += red_cnt[w];
                an += red_nodes[w];
            }
            *p.sum_out = a;
            if (NODES) *p.nodes_out = an;
            const unsigned long long err = *((volatile unsigned long long *)(p.ctl + kCtlError));
            const unsigned long long tmo = *((volatile unsigned long long *)(p.ctl + kCtlTimeout));
            *p.status_out = ((err & kErrDepth) ? kStatDepth : 0ull) | (tmo ? kStatTimeout : 0ull) |
                            ((err & kErrContOverflow) ? kStatContOverflow : 0ull);
        }
    }
}

}  // namespace nqb
