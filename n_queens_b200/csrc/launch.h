// launch.h -- launch-shape choices shared by every entry that starts the DFS
// kernel (capi.cu and the allocation-free entry in noalloc.cu).
//
// The reference fixes its CTA size and stack depth at compile time
// (CU1DBLOCK / STACKSIZE, src/macro.h:25-35).  Here both are chosen per launch
// from the stack depth the tasks need: a warp's stack takes levels x 512 B of
// shared memory, so the CTA size decides how much of the SM's shared memory
// can hold stacks, and with it how many warps stay resident.
#pragma once

#include <cuda_runtime.h>

#include "dfs_kernel.cuh"

namespace nqb {

// DFS steps per warp vote (the unroll of the kernel's inner loop), a
// compile-time choice.  The filtered count step runs 16 between votes: fewer
// votes and loop branches per step, for lanes that wait up to 15 steps for a
// refill (1.1 % faster than 8 at N=21, k=6).  The node-count and dihedral
// steps keep 8; the node-count step spills registers at 16.  A trip of the
// inner loop runs inner_steps rounded up to a multiple of the unroll.
#ifndef NQB_UNROLL
#define NQB_UNROLL 8
#endif
#ifndef NQB_COUNT_UNROLL
#define NQB_COUNT_UNROLL 16
#endif
constexpr int kUnroll = NQB_UNROLL;
constexpr int kCountUnroll = kStepVar == 4 ? NQB_COUNT_UNROLL : NQB_UNROLL;
static_assert(kUnroll % 4 == 0 && kCountUnroll % 4 == 0, "inner_steps are rounded to multiples of 4");

// DFS steps a warp runs between visits to the queue (the fold of its 32-bit
// counters happens at the same point).
constexpr int kDefaultInner = 1024;
// Static shared memory of dfs_kernel: two 32-entry reduction arrays + a flag.
constexpr int kDfsStaticSmem = 2 * 32 * 8 + 16;
// Search range of the default CTA size.  One 1024-thread CTA per SM holds as
// many warps as two 512-thread CTAs at 14 stack levels (32) but ran an N=21
// count 2.9 % slower (13.97 s against 13.57 s), so the search stops at 512.
constexpr int kMinAutoThreads = 64;
constexpr int kMaxAutoThreads = 512;

// Stack slots per lane that a launch over prefixes with `placed` queens needs:
// N-1-placed for the kernels that step every row (node counts, the dihedral
// decomposition), two fewer for the filtered count step.  At least 1.
inline int stack_need(int N, int placed, bool filtered) {
    const int need = N - 1 - placed - (filtered && kStepVar == 4 ? kStackRowsSpared<4> : 0);
    return need < 1 ? 1 : need;
}

// The CTA size (a multiple of 32 in [64, 512]) that keeps the most warps
// resident per SM for `levels` stack slots per lane, the larger CTA on a tie;
// at most cap_per_sm CTAs per SM are counted.  Returns 0 when no size fits.
// Uses only occupancy queries (no allocation, no launch).
template <typename Kernel>
int resident_warp_threads(Kernel fn, int levels, int smem_optin, int cap_per_sm) {
    int best = 0, best_warps = 0;
    for (int t = kMaxAutoThreads; t >= kMinAutoThreads; t -= 32) {
        const long long smem = (long long)(t / 32) * levels * kSlotBytes;
        if (smem + kDfsStaticSmem > smem_optin) continue;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, t, (size_t)smem) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        per_sm = per_sm < cap_per_sm ? per_sm : cap_per_sm;
        if (per_sm * (t / 32) > best_warps) {
            best_warps = per_sm * (t / 32);
            best = t;
        }
    }
    return best;
}

}  // namespace nqb
