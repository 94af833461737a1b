// capi.cu -- the C ABI (include/n_queens_b200.h) over the persistent DFS kernel.
//
// Host-side replacement for cuda_n_queens (src/n_queens_cuda.cu:84-186) on one
// device.  Differences from the reference driver, all deliberate:
//  * one device per call (no ratio split, :110-143);
//  * device buffers and pinned staging are cached per device and grown on
//    demand instead of cudaMalloc/cudaFree per call (:157-177);
//  * the queue word is reset on every launch (the reference's global_counter,
//    :8, is never reset, so its second call in a process counts nothing);
//  * no cudaDeviceSynchronize after every call (src/macro.h:48): one stream,
//    events for timing, one synchronisation per entry;
//  * errors come back as nq_status codes; the library never exits.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <functional>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "dfs_kernel.cuh"
#include "dihedral.h"
#include "expand.h"
#include "launch.h"
#include "n_queens_b200.h"

namespace nqb {

namespace {

constexpr int kMaxDevices = 64;
constexpr int kMaxBlocksPerSm = 32;
// d_ctl layout (uint64 words): control words, results, per-CTA partials.
constexpr int kWordSum = kCtlWords + 0;
constexpr int kWordNodes = kCtlWords + 1;
constexpr int kWordStatus = kCtlWords + 2;
constexpr int kWordBlocks = 8;

thread_local std::string g_last_error;

int fail_cuda(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? NQ_ERR_OOM : NQ_ERR_CUDA;
}

#define NQ_CUDA(call)                                         \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call);   \
    } while (0)

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

typedef void (*KernelFn)(DfsParams);

KernelFn pick_kernel(bool per_owner, bool nodes, bool dih = false) {
    if (dih) return per_owner ? dfs_kernel<true, false, kDihStepVar, kUnroll, false, true>
                              : dfs_kernel<false, false, kDihStepVar, kUnroll, false, true>;
    if (per_owner)
        return nodes ? dfs_kernel<true, true, kNodesStepVar, kUnroll> : dfs_kernel<true, false, kStepVar, kCountUnroll>;
    return nodes ? dfs_kernel<false, true, kNodesStepVar, kUnroll> : dfs_kernel<false, false, kStepVar, kCountUnroll>;
}

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int grow(size_t need) {
        if (need <= cap) return NQ_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(need + need / 4, 1 << 20);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc");
        cap = want;
        return NQ_OK;
    }
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    int grow(size_t need) {
        if (need <= cap) return NQ_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(need + need / 4, 1 << 20);
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e != cudaSuccess) return fail_cuda(e, "cudaHostAlloc");
        cap = want;
        return NQ_OK;
    }
};

struct Ctx {
    std::mutex mu;
    bool ready = false;
    int dev = 0;
    int sms = 0;
    int smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    unsigned long long *d_ctl = nullptr;  // control words + results + per-CTA partials
    DevBuf tasks;                         // cols | ld | rd (uint32 SoA)
    DevBuf aux;                           // order, owners, task_n, per-task outputs
    HostBuf h_tasks;                      // pinned staging for the expander
    DevBuf expand_scratch;                // seeds, counts, offsets of the device expander
};

Ctx g_ctx[kMaxDevices];

int ensure_ready(Ctx &c, int dev) {
    if (c.ready) {
        NQ_CUDA(cudaSetDevice(dev));
        return NQ_OK;
    }
    NQ_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    NQ_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10 || prop.minor != 0) {
        g_last_error = std::string("device is sm_") + std::to_string(prop.major) + std::to_string(prop.minor) +
                       "; this library carries only an sm_100a image";
        return NQ_ERR_NO_KERNEL;
    }
    c.dev = dev;
    c.sms = prop.multiProcessorCount;
    c.smem_optin = (int)prop.sharedMemPerBlockOptin;
    NQ_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    for (auto &e : c.ev) NQ_CUDA(cudaEventCreate(&e));
    const size_t ctl_words = kWordBlocks + 4 * (size_t)c.sms * kMaxBlocksPerSm;
    NQ_CUDA(cudaMalloc(&c.d_ctl, ctl_words * sizeof(unsigned long long)));
    NQ_CUDA(cudaMemset(c.d_ctl, 0, ctl_words * sizeof(unsigned long long)));
    // Dynamic shared memory above 48 KiB needs an opt-in per kernel.
    const int static_smem = kDfsStaticSmem;
    for (int po = 0; po < 2; ++po)
        for (int nd = 0; nd < 2; ++nd)
            NQ_CUDA(cudaFuncSetAttribute(pick_kernel(po, nd), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         c.smem_optin - static_smem));
    NQ_CUDA(cudaFuncSetAttribute(dfs_kernel<false, false, kStepVar, kCountUnroll, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, c.smem_optin - static_smem));
    NQ_CUDA(cudaFuncSetAttribute(dfs_kernel<false, false, kDihStepVar, kUnroll, true, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, c.smem_optin - static_smem));
    for (int po = 0; po < 2; ++po)
        NQ_CUDA(cudaFuncSetAttribute(pick_kernel(po, false, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     c.smem_optin - static_smem));
    c.ready = true;
    return NQ_OK;
}

int device_of(const nq_config *cfg) { return cfg ? cfg->device : 0; }

int lock_device(int dev, Ctx *&out) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        g_last_error = "no CUDA device";
        return NQ_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= n || dev >= kMaxDevices) {
        g_last_error = "device ordinal out of range";
        return NQ_ERR_ARG;
    }
    out = &g_ctx[dev];
    return NQ_OK;
}

struct Launch {
    int threads = 0, levels = 0, smem = 0, grid = 0, inner = 0, steal = 1, layout = 0;
    bool dih = false;  // dihedral-decomposition kernel
};

// Chooses the persistent grid: CTA size, stack slots per lane and as many
// resident CTAs per SM as shared memory and registers allow.  Default CTA
// size: resident_warp_threads (launch.h), the one that keeps the most warps
// resident per SM for this stack depth.
int plan_launch(Ctx &c, const nq_config *cfg, int levels_needed, bool per_owner, bool nodes, Launch &L,
                bool dih = false) {
    L.dih = dih;
    L.levels = std::max(1, levels_needed);
    if (cfg && cfg->stack_levels > NQ_MAX_STACK_LEVELS) {
        g_last_error = "stack_levels is above NQ_MAX_STACK_LEVELS";
        return NQ_ERR_ARG;
    }
    if (cfg && cfg->stack_levels > 0) {
        if (cfg->stack_levels < levels_needed) {
            g_last_error = "stack_levels is below what the tasks need";
            return NQ_ERR_DEPTH;
        }
        L.levels = cfg->stack_levels;
    }
    const int cap_per_sm = (cfg && cfg->blocks_per_sm > 0) ? std::min(cfg->blocks_per_sm, kMaxBlocksPerSm)
                                                           : kMaxBlocksPerSm;
    L.threads = (cfg && cfg->block_threads)
                    ? cfg->block_threads
                    : resident_warp_threads(pick_kernel(per_owner, nodes, dih), L.levels, c.smem_optin, cap_per_sm);
    if (!(cfg && cfg->block_threads) && L.threads == 0) {
        g_last_error = "no CTA size of 64 or more threads fits this stack depth in shared memory";
        return NQ_ERR_DEPTH;
    }
    if (L.threads < 32 || L.threads > 1024 || (L.threads & 31)) {
        g_last_error = "block_threads must be a multiple of 32 in [32, 1024]";
        return NQ_ERR_ARG;
    }
    const long long smem = (long long)(L.threads / 32) * L.levels * kSlotBytes;
    if (smem + kDfsStaticSmem > c.smem_optin) {
        g_last_error = "per-CTA stack does not fit in shared memory: lower block_threads";
        return NQ_ERR_DEPTH;
    }
    L.smem = (int)smem;
    int per_sm = 0;
    NQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_kernel(per_owner, nodes, dih),
                                                          L.threads, L.smem));
    if (per_sm <= 0) {
        g_last_error = "launch configuration cannot be resident";
        return NQ_ERR_ARG;
    }
    per_sm = std::min(per_sm, kMaxBlocksPerSm);
    if (cfg && cfg->blocks_per_sm > 0) per_sm = std::min(per_sm, cfg->blocks_per_sm);
    L.grid = c.sms * per_sm;
    if (cfg && cfg->inner_steps > NQ_MAX_INNER_STEPS) {
        g_last_error = "inner_steps is above NQ_MAX_INNER_STEPS";
        return NQ_ERR_ARG;
    }
    L.inner = (cfg && cfg->inner_steps > 0) ? ((cfg->inner_steps + 3) & ~3) : kDefaultInner;
    L.steal = (cfg && cfg->steal < 0) ? 0 : 1;
    L.layout = (cfg && cfg->layout == NQ_LAYOUT_LANE_MAJOR) ? 1 : 0;
    return NQ_OK;
}

void fill_stats_launch(nq_stats *st, const Launch &L) {
    if (!st) return;
    st->grid = L.grid;
    st->block_threads = L.threads;
    st->stack_levels = L.levels;
    st->smem_bytes = L.smem;
}

// Enqueues queue reset + kernel on stream s.
int enqueue_dfs(Ctx &c, DfsParams p, const Launch &L, bool per_owner, bool nodes, cudaStream_t s) {
    p.levels = L.levels;
    p.inner = L.inner;
    p.steal = L.steal;
    p.layout = L.layout;
    NQ_CUDA(cudaMemsetAsync(p.ctl, 0, kCtlWords * sizeof(unsigned long long), s));
    if (p.cta_times) NQ_CUDA(cudaMemsetAsync(p.cta_times, 0, 2 * (size_t)L.grid * sizeof(unsigned long long), s));
    pick_kernel(per_owner, nodes, L.dih)<<<L.grid, L.threads, L.smem, s>>>(p);
    NQ_CUDA(cudaGetLastError());
    return NQ_OK;
}

DfsParams base_params(Ctx &c, int N, int64_t n, const nq_config *cfg) {
    DfsParams p;
    memset(&p, 0, sizeof(p));
    p.N = N;
    p.ntasks = n;
    p.limit_ns = cfg ? (unsigned long long)cfg->time_limit_ms * 1000000ull : 0ull;
    p.ctl = c.d_ctl;
    p.sum_out = c.d_ctl + kWordSum;
    p.nodes_out = c.d_ctl + kWordNodes;
    p.status_out = c.d_ctl + kWordStatus;
    p.block_cnt = c.d_ctl + kWordBlocks;
    p.k_one = 1;
    p.k_two = 2;
    p.k_mone = 0xffffffffu;
    p.block_nodes = c.d_ctl + kWordBlocks + (size_t)c.sms * kMaxBlocksPerSm;
    if (cfg && cfg->timing) p.cta_times = c.d_ctl + kWordBlocks + 2 * (size_t)c.sms * kMaxBlocksPerSm;
    return p;
}

// Queue length of a launch over n tasks: cfg->queue_len positions, or all.
int queue_len_of(const nq_config *cfg, int64_t n, long long &q) {
    q = n;
    if (cfg && cfg->queue_len) {
        if ((int64_t)cfg->queue_len > n) {
            g_last_error = "queue_len exceeds the number of tasks";
            return NQ_ERR_ARG;
        }
        q = (long long)cfg->queue_len;
    }
    return NQ_OK;
}

int status_from_bits(unsigned long long bits) {
    if (bits & kStatDepth) {
        g_last_error = "a task needed more stack levels than the launch provided";
        return NQ_ERR_DEPTH;
    }
    if (bits & kStatTimeout) {
        g_last_error = "the kernel reached its time limit; counts are partial";
        return NQ_ERR_TIMEOUT;
    }
    return NQ_OK;
}

int levels_for_tasks(int N, const uint32_t *cols, int64_t n, bool filtered) {
    const uint32_t last = (N >= 32) ? 0xffffffffu : ((1u << N) - 1u);
    int need = 1;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t c = cols[i];
        if ((c & ~last) || c == last) continue;
        need = std::max(need, stack_need(N, __builtin_popcount(c), filtered));
    }
    return need;
}

// Per-CTA start/end stamps -> makespan, mean busy time, idle fraction.
int timing_stats(const unsigned long long *d_times, int grid, nq_stats *st) {
    std::vector<unsigned long long> t(2 * (size_t)grid);
    NQ_CUDA(cudaMemcpy(t.data(), d_times, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    unsigned long long t0 = ~0ull, t1 = 0;
    double busy = 0;
    for (int b = 0; b < grid; ++b) {
        t0 = std::min(t0, t[2 * b]);
        t1 = std::max(t1, t[2 * b + 1]);
        busy += (double)(t[2 * b + 1] - t[2 * b]);
    }
    const double span = (double)(t1 - t0);
    st->makespan_ms = span / 1e6;
    st->cta_busy_mean_ms = busy / grid / 1e6;
    st->tail_idle_frac = span > 0 ? 1.0 - busy / (span * grid) : 0.0;
    return NQ_OK;
}

// Counts tasks that are already in device memory (d_cols, d_ld, d_rd) and
// downloads the results.  Used by nq_count and nq_count_tasks.
// Class data of a dihedral launch (device pointers).
struct DihArgs {
    const uint8_t *task_cls = nullptr;
    const uint4 *cls_tab = nullptr;
    uint32_t noside = 0;
};

int count_resident(Ctx &c, int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd, int64_t n,
                   int levels_needed, const nq_config *cfg, bool per_owner, bool nodes, uint64_t *h_per_task,
                   uint64_t *h_nodes_task, uint64_t *sum, uint64_t *nodes_total, nq_stats *st, bool timed_h2d,
                   const uint32_t *d_order = nullptr, const DihArgs *dih = nullptr, int64_t nqueue = -1) {
    if (dih) nodes = false;
    Launch L;
    int rc = plan_launch(c, cfg, levels_needed, per_owner, nodes, L, dih != nullptr);
    if (rc) return rc;
    fill_stats_launch(st, L);
    DfsParams p = base_params(c, N, n, cfg);
    long long qlen = n;
    if (nqueue >= 0) {
        qlen = nqueue;  // the caller's internal order decides the queue
    } else {
        rc = queue_len_of(cfg, n, qlen);
        if (rc) return rc;
    }
    p.nqueue = qlen;
    if (qlen == 0 && n > 0) {
        // nothing queued: no launch, the sum is 0
        if (sum) *sum = 0;
        if (nodes_total) *nodes_total = 0;
        if (per_owner && h_per_task) memset(h_per_task, 0, (size_t)n * 8);
        if (per_owner && nodes && h_nodes_task) memset(h_nodes_task, 0, (size_t)n * 8);
        if (st) st->kernel_ms = 0;
        return NQ_OK;
    }
    p.cols = d_cols;
    p.ld = d_ld;
    p.rd = d_rd;
    if (dih) {
        p.task_cls = dih->task_cls;
        p.cls_tab = dih->cls_tab;
        p.noside = dih->noside;
    }
    // aux layout: [order u32 n] [out_cnt u64 n] [out_nodes u64 n]
    size_t off_order = 0, off_cnt = 0, off_nodes = 0, need = 0;
    const bool given = !d_order && cfg && cfg->order_kind == NQ_ORDER_GIVEN && cfg->order;
    if (given) {
        off_order = need;
        need += ((size_t)n * 4 + 255) & ~(size_t)255;
    }
    if (per_owner) {
        off_cnt = need;
        need += (size_t)n * 8;
        if (nodes) {
            off_nodes = need;
            need += (size_t)n * 8;
        }
    }
    if (need) {
        rc = c.aux.grow(need);
        if (rc) return rc;
    }
    char *aux = (char *)c.aux.p;
    if (given) {
        NQ_CUDA(cudaMemcpyAsync(aux + off_order, cfg->order, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
        p.order = (const uint32_t *)(aux + off_order);
    }
    if (d_order) p.order = d_order;
    if (per_owner) {
        p.out_cnt = (unsigned long long *)(aux + off_cnt);
        NQ_CUDA(cudaMemsetAsync(p.out_cnt, 0, (size_t)n * 8, c.stream));
        if (nodes) {
            p.out_nodes = (unsigned long long *)(aux + off_nodes);
            NQ_CUDA(cudaMemsetAsync(p.out_nodes, 0, (size_t)n * 8, c.stream));
        }
    }
    NQ_CUDA(cudaEventRecord(c.ev[1], c.stream));
    rc = enqueue_dfs(c, p, L, per_owner, nodes, c.stream);
    if (rc) return rc;
    NQ_CUDA(cudaEventRecord(c.ev[2], c.stream));
    unsigned long long res[3] = {0, 0, 0};
    NQ_CUDA(cudaMemcpyAsync(res, c.d_ctl + kWordSum, sizeof(res), cudaMemcpyDeviceToHost, c.stream));
    if (per_owner && h_per_task)
        NQ_CUDA(cudaMemcpyAsync(h_per_task, p.out_cnt, (size_t)n * 8, cudaMemcpyDeviceToHost, c.stream));
    if (per_owner && nodes && h_nodes_task)
        NQ_CUDA(cudaMemcpyAsync(h_nodes_task, p.out_nodes, (size_t)n * 8, cudaMemcpyDeviceToHost, c.stream));
    NQ_CUDA(cudaEventRecord(c.ev[3], c.stream));
    NQ_CUDA(cudaStreamSynchronize(c.stream));
    if (st && p.cta_times) {
        rc = timing_stats(p.cta_times, L.grid, st);
        if (rc) return rc;
    }
    if (st) {
        float ms = 0;
        if (timed_h2d) {
            cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]);
            st->h2d_ms = ms;
        }
        cudaEventElapsedTime(&ms, c.ev[1], c.ev[2]);
        st->kernel_ms = ms;
        cudaEventElapsedTime(&ms, c.ev[2], c.ev[3]);
        st->d2h_ms = ms;
        if (nodes) st->nodes = res[1];
    }
    if (sum) *sum = res[0];
    if (nodes_total) *nodes_total = res[1];
    return status_from_bits(res[2]);
}



// Uploads the class table of (N, rows) behind `used` bytes of c.tasks and
// fills the launch's class arguments.  The caller has grown c.tasks.
int dih_upload_classes(Ctx &c, int N, int rows, size_t used, DihArgs &a) {
    std::vector<DihClass> tab;
    if (!dihedral_classes(N, rows, tab) || tab.size() > (size_t)kMaxDihClasses) return NQ_ERR_ARG;
    uint4 h[kMaxDihClasses];  // synchronous copy below: the array may go out of scope after it
    for (size_t i = 0; i < tab.size(); ++i) {
        const DihClass &t = tab[i];
        // popc of a child's column mask (off-board bits set) is 32 - N + its
        // row; rows beyond side_row are popc values beyond this threshold.
        const int thr = 32 - N + t.side_row;
        h[i] = make_uint4((uint32_t)std::min(thr, 64), t.last_mask, t.tie_bit, t.w | (t.w_tie << 16));
    }
    const size_t off = (used + 255) & ~(size_t)255;
    uint4 *d = (uint4 *)((char *)c.tasks.p + off);
    NQ_CUDA(cudaMemcpy(d, h, tab.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    a.cls_tab = d;
    a.noside = ~(1u | (1u << (N - 1)));
    return NQ_OK;
}

size_t dih_bytes(int64_t n) {
    return (((size_t)std::max<int64_t>(n, 1) * 13 + 255) & ~(size_t)255) + kMaxDihClasses * sizeof(uint4);
}

// Checkpoint of a resumable whole-board count (little-endian file):
//   "NQB200CK" | u32 version=1 | i32 N | i32 rows | i32 mode | i64 ntasks |
//   i64 cursor | u64 partial (plain sum so far) | u64 slices | i64 n_cont |
//   n_cont x 16-byte continuation entries (cols|~last, ld, rd, untried) |
//   mode 1 only: n_cont class-index bytes
// mode 0 is the reference's decomposition (the partial sum is doubled at the
// end), mode 1 the dihedral one (the partial sum is weighted already).
struct Checkpoint {
    int N = 0, rows = 0;
    int mode = 0;  // 0: the reference's decomposition, 1: the dihedral one
    int64_t ntasks = 0, cursor = 0;
    uint64_t partial = 0, slices = 0;
    std::vector<uint4> cont;
    std::vector<uint8_t> cls;  // mode 1: class index of each continuation entry
};

const char kCkMagic[8] = {'N', 'Q', 'B', '2', '0', '0', 'C', 'K'};

int read_checkpoint(const char *path, int N, int rows, int mode, Checkpoint &ck, bool &have) {
    have = false;
    FILE *f = std::fopen(path, "rb");
    if (!f) return NQ_OK;  // no checkpoint yet: start from the beginning
    char magic[8];
    uint32_t version = 0;
    int32_t hN = 0, hrows = 0, hmode = 0;
    int64_t n_cont = -1;
    bool ok = std::fread(magic, 1, 8, f) == 8 && memcmp(magic, kCkMagic, 8) == 0 &&
              std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(&hN, 4, 1, f) == 1 &&
              std::fread(&hrows, 4, 1, f) == 1 && std::fread(&hmode, 4, 1, f) == 1 && (hmode == 0 || hmode == 1) &&
              std::fread(&ck.ntasks, 8, 1, f) == 1 && std::fread(&ck.cursor, 8, 1, f) == 1 &&
              std::fread(&ck.partial, 8, 1, f) == 1 && std::fread(&ck.slices, 8, 1, f) == 1 &&
              std::fread(&n_cont, 8, 1, f) == 1 && n_cont >= 0 && n_cont < (int64_t)1 << 32;
    if (ok) {
        // The entries must fill the rest of the file exactly; checking that
        // before sizing the buffers keeps a corrupt count from asking for
        // gigabytes.
        const long here = std::ftell(f);
        ok = here >= 0 && std::fseek(f, 0, SEEK_END) == 0;
        const long end = ok ? std::ftell(f) : -1;
        ok = ok && end >= here && std::fseek(f, here, SEEK_SET) == 0 &&
             (int64_t)(end - here) == n_cont * (hmode == 1 ? 17 : 16);
    }
    if (ok) {
        ck.cont.resize((size_t)n_cont);
        ok = n_cont == 0 || std::fread(ck.cont.data(), 16, (size_t)n_cont, f) == (size_t)n_cont;
        if (ok && hmode == 1) {
            ck.cls.resize((size_t)n_cont);
            ok = n_cont == 0 || std::fread(ck.cls.data(), 1, (size_t)n_cont, f) == (size_t)n_cont;
        }
        char extra;
        ok = ok && std::fread(&extra, 1, 1, f) == 0;  // nothing after the entries
    }
    std::fclose(f);
    if (!ok) {
        g_last_error = std::string("not a valid checkpoint file: ") + path;
        return NQ_ERR_ARG;
    }
    if (hN != N || hrows != rows) {
        g_last_error = "checkpoint is for N=" + std::to_string(hN) + " rows=" + std::to_string(hrows);
        return NQ_ERR_ARG;
    }
    if (hmode != mode) {
        g_last_error = hmode ? "checkpoint is of a dihedral count" : "checkpoint is of a plain (mirror) count";
        return NQ_ERR_ARG;
    }
    // Every continuation entry must be a level the kernel could have saved:
    // its column mask carries the off-board columns and its untried columns
    // are free (no column, no diagonal).  The kernel's stack bound rests on
    // the second: a step on a column already in the mask would add no queen.
    const uint32_t last = (N >= 32) ? 0xffffffffu : ((1u << N) - 1u);
    for (const uint4 &e : ck.cont)
        if ((e.x & ~last) != ~last || (e.w & (e.x | e.y | e.z)) != 0) {
            g_last_error = "checkpoint holds a continuation entry that no count could have saved";
            return NQ_ERR_ARG;
        }
    ck.N = hN;
    ck.rows = hrows;
    ck.mode = hmode;
    have = true;
    return NQ_OK;
}

int write_checkpoint(const char *path, const Checkpoint &ck) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) {
        g_last_error = "cannot write " + tmp;
        return NQ_ERR_ARG;
    }
    const uint32_t version = 1;
    const int32_t hN = ck.N, hrows = ck.rows, hmode = ck.mode;
    const int64_t n_cont = (int64_t)ck.cont.size();
    bool ok = std::fwrite(kCkMagic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
              std::fwrite(&hN, 4, 1, f) == 1 && std::fwrite(&hrows, 4, 1, f) == 1 &&
              std::fwrite(&hmode, 4, 1, f) == 1 && std::fwrite(&ck.ntasks, 8, 1, f) == 1 &&
              std::fwrite(&ck.cursor, 8, 1, f) == 1 && std::fwrite(&ck.partial, 8, 1, f) == 1 &&
              std::fwrite(&ck.slices, 8, 1, f) == 1 && std::fwrite(&n_cont, 8, 1, f) == 1 &&
              (n_cont == 0 || std::fwrite(ck.cont.data(), 16, (size_t)n_cont, f) == (size_t)n_cont) &&
              (ck.mode == 0 || n_cont == 0 || std::fwrite(ck.cls.data(), 1, (size_t)n_cont, f) == (size_t)n_cont);
    ok = (std::fflush(f) == 0) && ok;
    std::fclose(f);
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        g_last_error = "cannot write checkpoint " + std::string(path);
        return NQ_ERR_ARG;
    }
    return NQ_OK;
}

constexpr int kDefaultSplit = 3;

}  // namespace
}  // namespace nqb

// A batch plan: the deduplicated, split and uploaded subtasks of a set of
// partial boards, and a CUDA graph that resets the queue, counts and copies
// the results back.
struct nq_batch {
    int device = 0;
    int64_t n_inst = 0, n_unique = 0, m_tasks = 0;
    std::vector<int64_t> inst_to_u;
    void *d_buf = nullptr;                 // tasks (cols | ld | rd | owner u32, task_n u8) + results
    unsigned long long *h_res = nullptr;   // pinned: [sum, nodes, status, 2 words per unique board]
    unsigned long long *d_out = nullptr;   // 2 words per unique board: weight-1 and weight-2 sums
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    nqb::Launch L;
    int levels = 0;
};

namespace nqb {
namespace {

// Reverses the low N bits (column j -> N-1-j).
uint32_t rev_bits(uint32_t x, int N) {
    uint32_t y = 0;
    for (int j = 0; j < N; ++j)
        if (x >> j & 1u) y |= 1u << (N - 1 - j);
    return y;
}

struct Board {
    int N;
    uint32_t c, l, r;
    bool operator==(const Board &o) const { return N == o.N && c == o.c && l == o.l && r == o.r; }
};
struct BoardHash {
    size_t operator()(const Board &b) const {
        uint64_t h = (uint64_t)b.N * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)b.c + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h ^= (uint64_t)b.l + 0x8CB92BA72F3D8DD7ull + (h << 6) + (h >> 2);
        h ^= (uint64_t)b.r + 0xAEF17502108EF2D9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

// The left-right mirror of a board has the same completion count.  It is
// used only for boards whose column and right-diagonal masks lie on the
// board (then no attack outside the board can shift back onto it, and the
// left-diagonal bits beyond the board, which only move further out, can be
// dropped).
bool mirror_safe(const Board &b) {
    const uint32_t last = (b.N >= 32) ? 0xffffffffu : ((1u << b.N) - 1u);
    return b.N < 32 && !(b.c & ~last) && !(b.r & ~last) && b.c != last;
}

Board mirror(const Board &b) {
    const uint32_t last = (1u << b.N) - 1u;
    return Board{b.N, rev_bits(b.c, b.N), rev_bits(b.r & last, b.N), rev_bits(b.l & last, b.N)};
}

bool board_less(const Board &a, const Board &b) {
    if (a.c != b.c) return a.c < b.c;
    if (a.l != b.l) return a.l < b.l;
    return a.r < b.r;
}

// Splits board b `rows` rows deeper into (subtask, weight) pairs whose
// weighted counts add up to b's count.  A mirror-symmetric board keeps only
// its left-half children at weight 2 and recurses into the middle column's
// child (itself symmetric) -- the reference's half-board rule
// (src/n_queens.cpp:74-113) applied to any symmetric board.
void split_board(const Board &b, int rows, bool symmetric, std::vector<uint32_t> &tc, std::vector<uint32_t> &tl,
                 std::vector<uint32_t> &tr, std::vector<uint8_t> &tw) {
    if (!symmetric || rows <= 0) {
        expand_board(b.N, b.c, b.l, b.r, rows, tc, tl, tr);
        tw.resize(tc.size(), 1);
        return;
    }
    const uint32_t last = (1u << b.N) - 1u;
    uint32_t avail = last & ~(b.c | b.l | b.r);
    while (avail) {
        const uint32_t p = avail & (0u - avail);
        avail ^= p;
        const uint32_t q = rev_bits(p, b.N);
        if (q < p) continue;  // right half: the mirror of a left-half child
        const Board ch{b.N, b.c | p, (b.l | p) << 1, (uint32_t)((int32_t)(b.r | p) >> 1)};
        if (q == p) {
            split_board(ch, rows - 1, ch.c != last, tc, tl, tr, tw);
        } else {
            expand_board(ch.N, ch.c, ch.l, ch.r, rows - 1, tc, tl, tr);
            tw.resize(tc.size(), 2);
        }
    }
}

void destroy_batch(nq_batch &b) {
    if (b.exec) cudaGraphExecDestroy(b.exec);
    if (b.graph) cudaGraphDestroy(b.graph);
    if (b.d_buf) cudaFree(b.d_buf);
    if (b.h_res) cudaFreeHost(b.h_res);
    b.exec = nullptr;
    b.graph = nullptr;
    b.d_buf = nullptr;
    b.h_res = nullptr;
}

int build_batch(Ctx &c, const nq_instance *inst, int64_t n, int split, const nq_config *cfg, nq_batch &B) {
    B.device = device_of(cfg);
    B.n_inst = n;
    B.inst_to_u.resize((size_t)n);
    // 1. exact dedup: identical boards, and boards equal up to mirror image
    std::unordered_map<Board, int64_t, BoardHash> index;
    std::vector<Board> uniq;
    for (int64_t i = 0; i < n; ++i) {
        Board b{inst[i].N, inst[i].cols, inst[i].ld, inst[i].rd};
        if (mirror_safe(b)) {
            const uint32_t last = (1u << b.N) - 1u;
            b.l &= last;  // bits beyond the board never return
            const Board m = mirror(b);
            if (board_less(m, b)) b = m;
        }
        auto it = index.find(b);
        if (it == index.end()) {
            it = index.emplace(b, (int64_t)uniq.size()).first;
            uniq.push_back(b);
        }
        B.inst_to_u[i] = it->second;
    }
    B.n_unique = (int64_t)uniq.size();
    // 2. split every distinct board; owner = 2u + (weight == 2)
    std::vector<uint32_t> tc, tl, tr, own;
    std::vector<uint8_t> tw, tn;
    int need = 1;
    for (int64_t u = 0; u < B.n_unique; ++u) {
        const Board &b = uniq[u];
        const bool sym = mirror_safe(b) && mirror(b) == b;
        const size_t before = tc.size();
        split_board(b, split, sym, tc, tl, tr, tw);
        const uint32_t last = (b.N >= 32) ? 0xffffffffu : ((1u << b.N) - 1u);
        for (size_t k = before; k < tc.size(); ++k) {
            own.push_back((uint32_t)(2 * u + (tw[k] == 2 ? 1 : 0)));
            tn.push_back((uint8_t)b.N);
            if (!(tc[k] & ~last) && tc[k] != last)
                need = std::max(need, stack_need(b.N, __builtin_popcount(tc[k]), true));
        }
    }
    const int64_t m = (int64_t)tc.size();
    B.m_tasks = m;
    B.levels = need;
    int rc = plan_launch(c, cfg, need, true, false, B.L);
    if (rc) return rc;
    // 3. device buffer: tasks, owners, sizes, per-owner sums
    const size_t task_bytes = ((size_t)m * 17 + 255) & ~(size_t)255;
    const size_t out_bytes = (size_t)B.n_unique * 2 * 8;
    NQ_CUDA(cudaMalloc(&B.d_buf, task_bytes + out_bytes + 256));
    NQ_CUDA(cudaHostAlloc((void **)&B.h_res, (3 + 2 * (size_t)B.n_unique) * 8, cudaHostAllocDefault));
    uint32_t *d = (uint32_t *)B.d_buf;
    B.d_out = (unsigned long long *)((char *)B.d_buf + task_bytes);
    if (m) {
        NQ_CUDA(cudaMemcpyAsync(d, tc.data(), (size_t)m * 4, cudaMemcpyHostToDevice, c.stream));
        NQ_CUDA(cudaMemcpyAsync(d + m, tl.data(), (size_t)m * 4, cudaMemcpyHostToDevice, c.stream));
        NQ_CUDA(cudaMemcpyAsync(d + 2 * m, tr.data(), (size_t)m * 4, cudaMemcpyHostToDevice, c.stream));
        NQ_CUDA(cudaMemcpyAsync(d + 3 * m, own.data(), (size_t)m * 4, cudaMemcpyHostToDevice, c.stream));
        NQ_CUDA(cudaMemcpyAsync(d + 4 * m, tn.data(), (size_t)m, cudaMemcpyHostToDevice, c.stream));
    }
    NQ_CUDA(cudaStreamSynchronize(c.stream));
    DfsParams p = base_params(c, 0, m, cfg);
    p.cols = d;
    p.ld = d + m;
    p.rd = d + 2 * m;
    p.owner_of = d + 3 * m;
    p.task_n = (const uint8_t *)(d + 4 * m);
    p.out_cnt = B.d_out;
    p.cta_times = nullptr;
    // 4. one graph: reset, count, copy back (result words and per-owner sums)
    NQ_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(B.d_out, 0, out_bytes, c.stream);
    int krc = NQ_OK;
    if (e == cudaSuccess) krc = enqueue_dfs(c, p, B.L, true, false, c.stream);
    if (e == cudaSuccess && krc == NQ_OK)
        e = cudaMemcpyAsync(B.h_res, c.d_ctl + kWordSum, 3 * 8, cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess && krc == NQ_OK)
        e = cudaMemcpyAsync(B.h_res + 3, B.d_out, out_bytes, cudaMemcpyDeviceToHost, c.stream);
    cudaError_t e2 = cudaStreamEndCapture(c.stream, &B.graph);
    if (krc) return krc;
    if (e != cudaSuccess) return fail_cuda(e, "batch graph capture");
    if (e2 != cudaSuccess) return fail_cuda(e2, "cudaStreamEndCapture");
    NQ_CUDA(cudaGraphInstantiate(&B.exec, B.graph, 0));
    return NQ_OK;
}

int run_batch(Ctx &c, nq_batch &B, nq_stats *st) {
    NQ_CUDA(cudaEventRecord(c.ev[1], c.stream));
    NQ_CUDA(cudaGraphLaunch(B.exec, c.stream));
    NQ_CUDA(cudaEventRecord(c.ev[2], c.stream));
    NQ_CUDA(cudaStreamSynchronize(c.stream));
    if (st) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c.ev[1], c.ev[2]);
        st->kernel_ms = ms;
        st->tasks = B.m_tasks;
        fill_stats_launch(st, B.L);
    }
    return NQ_OK;
}
}  // namespace

void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

// No exception may cross the C ABI: every exported entry ends in a
// function-try-block whose handler returns this status for the exception in
// flight (a host allocation that failed is NQ_ERR_OOM).
int status_of_exception() noexcept {
    try {
        throw;
    } catch (const std::bad_alloc &) {
        g_last_error = "out of host memory";
        return NQ_ERR_OOM;
    } catch (const std::exception &e) {
        g_last_error = std::string("internal error: ") + e.what();
    } catch (...) {
        g_last_error = "internal error";
    }
    return NQ_ERR_ARG;
}

}  // namespace nqb

namespace nqb {
namespace {

// One slice of a resumable whole-board count, in the reference's
// decomposition (dih false) or the dihedral one (dih true).
int count_resumable_impl(int N, int rows, const nq_config *cfg, const char *checkpoint_path, bool dih,
                         uint64_t *total, int *done, nq_stats *stats) {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    *done = 0;
    *total = 0;
    Checkpoint ck;
    bool have = false;
    int rc = read_checkpoint(checkpoint_path, N, rows, dih ? 1 : 0, ck, have);
    if (rc) return rc;
    Ctx *cp = nullptr;
    rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    const double te = now_ms();
    const int64_t n = dih ? dihedral_expand(N, rows, nullptr, nullptr, nullptr, nullptr, 0)
                          : expand_prefixes(N, rows, nullptr, nullptr, nullptr, 0, 0);
    if (n < 0 || n > 0xffffffffll) return NQ_ERR_ARG;
    if (have && (ck.ntasks != n || ck.cursor < 0 || ck.cursor > n)) {
        g_last_error = "checkpoint does not match this board's task list";
        return NQ_ERR_ARG;
    }
    const size_t ncont = have ? ck.cont.size() : 0;
    const size_t per_task = dih ? 13 : 12;  // cols | ld | rd (u32) [| class (u8)]
    rc = c.h_tasks.grow((size_t)std::max<int64_t>(n, 1) * per_task);
    if (rc) return rc;
    uint32_t *h = (uint32_t *)c.h_tasks.p;
    if (dih)
        dihedral_expand(N, rows, h, h + n, h + 2 * n, (uint8_t *)(h + 3 * n), n);
    else
        expand_prefixes(N, rows, h, h + n, h + 2 * n, n, 0);
    if (stats) {
        stats->expand_ms = now_ms() - te;
        stats->tasks = n;
    }
    // tasks [+ classes + class table], then the continuation entries to resume
    // [and their class indices]
    const size_t task_bytes = dih ? dih_bytes(n) : (((size_t)std::max<int64_t>(n, 1) * 12 + 255) & ~(size_t)255);
    rc = c.tasks.grow(task_bytes + ncont * 17 + 512);
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    uint4 *d_cont_in = (uint4 *)((char *)c.tasks.p + task_bytes);
    uint8_t *d_cont_cls = (uint8_t *)(d_cont_in + ncont);
    DihArgs a;
    if (dih) {
        a.task_cls = (const uint8_t *)(d + 3 * n);
        rc = dih_upload_classes(c, N, rows, (size_t)n * 13, a);
        if (rc) return rc;
        std::vector<DihClass> tab;
        dihedral_classes(N, rows, tab);
        for (size_t i = 0; i < ncont; ++i)
            if (ck.cls[i] >= tab.size()) {
                g_last_error = "checkpoint holds a class index out of range";
                return NQ_ERR_ARG;
            }
    }
    NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    if (n) NQ_CUDA(cudaMemcpyAsync(d, h, (size_t)n * per_task, cudaMemcpyHostToDevice, c.stream));
    if (ncont) {
        NQ_CUDA(cudaMemcpyAsync(d_cont_in, ck.cont.data(), ncont * 16, cudaMemcpyHostToDevice, c.stream));
        if (dih) NQ_CUDA(cudaMemcpyAsync(d_cont_cls, ck.cls.data(), ncont, cudaMemcpyHostToDevice, c.stream));
    }
    KernelFn fn = dih ? dfs_kernel<false, false, kDihStepVar, kUnroll, true, true> : dfs_kernel<false, false, kStepVar, kCountUnroll, true>;
    Launch L;
    rc = plan_launch(c, cfg, stack_need(N, rows, !dih), false, false, L, dih);
    if (rc) return rc;
    {
        // the resumable instantiation may fit fewer CTAs per SM
        int per_sm = 0;
        NQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, L.threads, L.smem));
        if (per_sm <= 0) return NQ_ERR_ARG;
        L.grid = std::min(L.grid, c.sms * std::min(per_sm, kMaxBlocksPerSm));
    }
    fill_stats_launch(stats, L);
    // room for every lane's unfinished levels: the current one + one per slot
    const size_t cap = (size_t)L.grid * L.threads * (L.levels + 1);
    rc = c.aux.grow(cap * (dih ? 17 : 16));
    if (rc) return rc;
    DfsParams p = base_params(c, N, n, cfg);
    p.cols = d;
    p.ld = d + n;
    p.rd = d + 2 * n;
    p.cont_in = d_cont_in;
    p.n_cont_in = (long long)ncont;
    p.task_base = have ? ck.cursor : 0;
    p.cont_out = (uint4 *)c.aux.p;
    p.cont_cap = (long long)cap;
    if (dih) {
        p.task_cls = a.task_cls;
        p.cls_tab = a.cls_tab;
        p.noside = a.noside;
        p.cont_in_cls = d_cont_cls;
        p.cont_out_cls = (uint8_t *)((uint4 *)c.aux.p + cap);
    }
    p.levels = L.levels;
    p.inner = L.inner;
    p.steal = L.steal;
    p.layout = L.layout;
    NQ_CUDA(cudaEventRecord(c.ev[1], c.stream));
    NQ_CUDA(cudaMemsetAsync(p.ctl, 0, kCtlWords * sizeof(unsigned long long), c.stream));
    fn<<<L.grid, L.threads, L.smem, c.stream>>>(p);
    NQ_CUDA(cudaGetLastError());
    NQ_CUDA(cudaEventRecord(c.ev[2], c.stream));
    unsigned long long words[kWordBlocks];
    NQ_CUDA(cudaMemcpyAsync(words, c.d_ctl, sizeof(words), cudaMemcpyDeviceToHost, c.stream));
    NQ_CUDA(cudaStreamSynchronize(c.stream));
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]);
        stats->h2d_ms = ms;
        cudaEventElapsedTime(&ms, c.ev[1], c.ev[2]);
        stats->kernel_ms = ms;
    }
    const unsigned long long bits = words[kWordStatus];
    if (bits & kStatContOverflow) {
        g_last_error = "continuation buffer overflow";
        return NQ_ERR_CUDA;
    }
    if (bits & kStatDepth) return status_from_bits(bits);
    const uint64_t partial = (have ? ck.partial : 0) + words[kWordSum];
    if (bits & kStatTimeout) {
        // Positions taken from the queue were either finished or saved.
        const long long qlen = (long long)ncont + n - p.task_base;
        const long long taken = std::min<long long>((long long)words[kCtlHead], qlen);
        Checkpoint out;
        out.N = N;
        out.rows = rows;
        out.mode = dih ? 1 : 0;
        out.ntasks = n;
        out.cursor = p.task_base + std::max<long long>(0, taken - (long long)ncont);
        out.partial = partial;
        out.slices = (have ? ck.slices : 0) + 1;
        // Saved levels of an earlier slice that no lane picked up this time
        // carry over unchanged, then come the levels this slice saved.
        const size_t untaken = (size_t)std::max<long long>(0, (long long)ncont - taken);
        const size_t fresh = (size_t)words[kCtlCont];
        out.cont.resize(untaken + fresh);
        for (size_t i = 0; i < untaken; ++i) out.cont[i] = ck.cont[ncont - untaken + i];
        if (fresh)
            NQ_CUDA(cudaMemcpy(out.cont.data() + untaken, c.aux.p, fresh * 16, cudaMemcpyDeviceToHost));
        if (dih) {
            out.cls.resize(untaken + fresh);
            for (size_t i = 0; i < untaken; ++i) out.cls[i] = ck.cls[ncont - untaken + i];
            if (fresh)
                NQ_CUDA(cudaMemcpy(out.cls.data() + untaken, p.cont_out_cls, fresh, cudaMemcpyDeviceToHost));
        }
        rc = write_checkpoint(checkpoint_path, out);
        if (rc) return rc;
        if (stats) stats->total_ms = now_ms() - t0;
        return NQ_OK;
    }
    // The reference doubles the half-board sum (src/n_queens_cuda.cu:181-183);
    // dihedral weights already carry every symmetry factor.
    *total = dih ? partial : 2 * partial;
    *done = 1;
    if (have) std::remove(checkpoint_path);
    if (stats) stats->total_ms = now_ms() - t0;
    return NQ_OK;
}

}  // namespace
}  // namespace nqb

using namespace nqb;

extern "C" {

int nq_abi_version(void) { return NQ_ABI_VERSION; }

const char *nq_status_string(int status) {
    switch (status) {
        case NQ_OK: return "ok";
        case NQ_ERR_ARG: return "invalid argument";
        case NQ_ERR_NO_DEVICE: return "no CUDA device";
        case NQ_ERR_CUDA: return "CUDA runtime error";
        case NQ_ERR_OOM: return "out of memory";
        case NQ_ERR_DEPTH: return "stack depth exceeds the launch's stack";
        case NQ_ERR_TIMEOUT: return "time limit reached; counts are partial";
        case NQ_ERR_NO_KERNEL: return "no kernel image for this device";
        default: return "unknown status";
    }
}

const char *nq_last_error(void) { return g_last_error.c_str(); }

int nq_stack_levels(int N, int rows, int nodes) try {
    if (N < 1 || N > NQ_MAX_N || rows < 0 || rows > N) return NQ_ERR_ARG;
    return stack_need(N, rows, nodes == 0);
} catch (...) {
    return status_of_exception();
}

int nq_device_count(int *count) try {
    if (!count) return NQ_ERR_ARG;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
        (void)cudaGetLastError();
        *count = 0;
        return NQ_OK;
    }
    if (e != cudaSuccess) {
        *count = 0;
        return fail_cuda(e, "cudaGetDeviceCount");
    }
    *count = n;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_expand(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, int64_t cap, int64_t *n_tasks,
              int threads) try {
    if (N < 2 || N > NQ_MAX_N || rows < 1 || rows > N || !n_tasks || cap < 0) return NQ_ERR_ARG;
    if (cap > 0 && (!cols || !ld || !rd)) return NQ_ERR_ARG;
    const int64_t n = expand_prefixes(N, rows, cols, ld, rd, cap, threads);
    if (n < 0) return NQ_ERR_ARG;
    *n_tasks = n;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_expand_device(int N, int rows, uint32_t *d_cols, uint32_t *d_ld, uint32_t *d_rd, int64_t cap,
                     int64_t *n_tasks, int device, void *stream) try {
    if (N < 2 || N > NQ_MAX_N || rows < 1 || rows > N || !n_tasks || cap < 0) return NQ_ERR_ARG;
    if (cap > 0 && (!d_cols || !d_ld || !d_rd)) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device, cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device);
    if (rc) return rc;
    NQ_CUDA(expand_prefixes_device(N, rows, d_cols, d_ld, d_rd, cap, n_tasks, &c.expand_scratch.p,
                                   &c.expand_scratch.cap, (cudaStream_t)stream));
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

// Expands (N, rows) into the context's task buffer on the device.
int device_expand_into_ctx(Ctx &c, int N, int rows, int64_t &n) {
    NQ_CUDA(expand_prefixes_device(N, rows, nullptr, nullptr, nullptr, 0, &n, &c.expand_scratch.p,
                                   &c.expand_scratch.cap, c.stream));
    int rc = c.tasks.grow((size_t)std::max<int64_t>(n, 1) * 16 + 256);
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    int64_t n2 = 0;
    NQ_CUDA(expand_prefixes_device(N, rows, d, d + n, d + 2 * n, n, &n2, &c.expand_scratch.p, &c.expand_scratch.cap,
                                   c.stream));
    return n2 == n ? NQ_OK : NQ_ERR_CUDA;
}

int nq_count(int N, int rows, const nq_config *cfg, uint64_t *total, uint64_t *nodes, nq_stats *stats) try {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (N < 2 || N > NQ_MAX_N || rows < 1 || rows > N - 2 || !total) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc == NQ_ERR_NO_DEVICE) {
        // Mirror the reference: the prefixes are generated before the GPU
        // count is checked (src/n_queens_cuda.cu:91-108).
        const double te = now_ms();
        const int64_t n = expand_prefixes(N, rows, nullptr, nullptr, nullptr, 0, 0);
        if (stats) {
            stats->expand_ms = now_ms() - te;
            stats->tasks = n;
            stats->total_ms = now_ms() - t0;
        }
        return rc;
    }
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;

    const double te = now_ms();
    int64_t n = 0;
    if (cfg && cfg->device_expand) {
        rc = device_expand_into_ctx(c, N, rows, n);
        if (rc) return rc;
        if (stats) {
            stats->expand_ms = now_ms() - te;
            stats->tasks = n;
        }
        NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    } else {
        uint32_t *h = nullptr;
        int grow_rc = NQ_OK;
        n = expand_prefixes_to(
            N, rows,
            [&](int64_t total_tasks, uint32_t **pc, uint32_t **pl, uint32_t **pr, int64_t *cap) {
                grow_rc = c.h_tasks.grow((size_t)std::max<int64_t>(total_tasks, 1) * 12);
                if (grow_rc) return false;
                h = (uint32_t *)c.h_tasks.p;
                *pc = h;
                *pl = h + total_tasks;
                *pr = h + 2 * total_tasks;
                *cap = total_tasks;
                return true;
            },
            0);
        if (grow_rc) return grow_rc;
        if (n < 0) return NQ_ERR_ARG;
        if (stats) {
            stats->expand_ms = now_ms() - te;
            stats->tasks = n;
        }
        rc = c.tasks.grow((size_t)std::max<int64_t>(n, 1) * 12);
        if (rc) return rc;
        NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
        if (n) NQ_CUDA(cudaMemcpyAsync(c.tasks.p, h, (size_t)n * 12, cudaMemcpyHostToDevice, c.stream));
    }
    uint32_t *d = (uint32_t *)c.tasks.p;
    uint64_t sum = 0, nd = 0;
    rc = count_resident(c, N, d, d + n, d + 2 * n, n, stack_need(N, rows, nodes == nullptr), cfg, false,
                        nodes != nullptr, nullptr, nullptr,
                        &sum, &nd, stats, true);
    // The reference doubles every per-prefix sum for the mirror image
    // (src/n_queens_cuda.cu:181-183).
    *total = 2 * sum;
    if (nodes) *nodes = nd;
    if (stats) stats->total_ms = now_ms() - t0;
    return rc;
} catch (...) {
    return status_of_exception();
}

int nq_count_resumable(int N, int rows, const nq_config *cfg, const char *checkpoint_path, uint64_t *total,
                       int *done, nq_stats *stats) try {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (N < 2 || N > NQ_MAX_N || rows < 1 || rows > N - 2 || !total || !done || !checkpoint_path) return NQ_ERR_ARG;
    return count_resumable_impl(N, rows, cfg, checkpoint_path, false, total, done, stats);
} catch (...) {
    return status_of_exception();
}

int nq_count_dihedral_resumable(int N, int rows, const nq_config *cfg, const char *checkpoint_path, uint64_t *total,
                                int *done, nq_stats *stats) try {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (N < 4 || N > NQ_MAX_N || rows < 2 || rows > N - 2 || !total || !done || !checkpoint_path) return NQ_ERR_ARG;
    return count_resumable_impl(N, rows, cfg, checkpoint_path, true, total, done, stats);
} catch (...) {
    return status_of_exception();
}

}  // extern "C"

namespace nqb {
namespace {

// nq_count_learned and nq_count_learned_reuse: expand, upload, order the
// queue longest-first on the device (the listed already-counted tasks last,
// outside the queue), count.
int count_learned_impl(int N, int rows, nq_mlp *m, const int64_t *done_idx, int64_t n_done, uint64_t done_sum,
                       const nq_config *cfg, uint64_t *total, nq_stats *stats) {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (N < 2 || N > NQ_MAX_N || rows < 1 || rows > N - 2 || !total || !m) return NQ_ERR_ARG;
    if (n_done < 0 || (n_done > 0 && !done_idx)) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    const double te = now_ms();
    uint32_t *h = nullptr;
    int grow_rc = NQ_OK;
    const int64_t n = expand_prefixes_to(
        N, rows,
        [&](int64_t total_tasks, uint32_t **pc, uint32_t **pl, uint32_t **pr, int64_t *cap) {
            // tasks (12 B each), then the already-counted indices (4 B each)
            grow_rc = c.h_tasks.grow((size_t)std::max<int64_t>(total_tasks, 1) * 12 + (size_t)n_done * 4 + 256);
            if (grow_rc) return false;
            h = (uint32_t *)c.h_tasks.p;
            *pc = h;
            *pl = h + total_tasks;
            *pr = h + 2 * total_tasks;
            *cap = total_tasks;
            return true;
        },
        0);
    if (grow_rc) return grow_rc;
    if (n < 0 || n > 0xffffffffll) return NQ_ERR_ARG;
    if (n_done > n) {
        g_last_error = "more already-counted tasks than the board has";
        return NQ_ERR_ARG;
    }
    // The listed indices must be distinct and in range: ascending order is
    // required, so one pass checks both.
    uint32_t *h_done = h + 3 * n;
    for (int64_t i = 0; i < n_done; ++i) {
        if (done_idx[i] < 0 || done_idx[i] >= n || (i > 0 && done_idx[i] <= done_idx[i - 1])) {
            g_last_error = "already-counted task indices must be ascending, distinct and below the task count";
            return NQ_ERR_ARG;
        }
        h_done[i] = (uint32_t)done_idx[i];
    }
    if (stats) {
        stats->expand_ms = now_ms() - te;
        stats->tasks = n;
    }
    // tasks (12 B each), the order (4 B each), the already-counted indices
    rc = c.tasks.grow((size_t)std::max<int64_t>(n, 1) * 16 + (size_t)n_done * 4 + 256);
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    uint32_t *d_order = d + 3 * n;
    uint32_t *d_done = d + 4 * n;
    NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    if (n) NQ_CUDA(cudaMemcpyAsync(d, h, (size_t)n * 12, cudaMemcpyHostToDevice, c.stream));
    if (n_done) NQ_CUDA(cudaMemcpyAsync(d_done, h_done, (size_t)n_done * 4, cudaMemcpyHostToDevice, c.stream));
    cudaEvent_t e_sched0 = nullptr, e_sched1 = nullptr;
    NQ_CUDA(cudaEventCreate(&e_sched0));
    NQ_CUDA(cudaEventCreate(&e_sched1));
    NQ_CUDA(cudaEventRecord(e_sched0, c.stream));
    rc = nq_schedule_device_last(m, N, d, d + n, d + 2 * n, n, d_done, n_done, d_order, nullptr, c.stream);
    if (rc) {
        cudaEventDestroy(e_sched0);
        cudaEventDestroy(e_sched1);
        return rc;
    }
    NQ_CUDA(cudaEventRecord(e_sched1, c.stream));
    uint64_t sum = 0;
    rc = count_resident(c, N, d, d + n, d + 2 * n, n, stack_need(N, rows, true), cfg, false, false, nullptr, nullptr, &sum,
                        nullptr, stats, true, d_order, nullptr, n - n_done);
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e_sched0, e_sched1);
        stats->schedule_ms = ms;
        cudaEventElapsedTime(&ms, c.ev[0], e_sched0);
        stats->h2d_ms = ms;
        stats->total_ms = now_ms() - t0;
    }
    cudaEventDestroy(e_sched0);
    cudaEventDestroy(e_sched1);
    // The reference doubles every per-prefix sum for the mirror image
    // (src/n_queens_cuda.cu:181-183).
    *total = 2 * (sum + done_sum);
    return rc;
}

}  // namespace
}  // namespace nqb

extern "C" {

int nq_count_learned(int N, int rows, nq_mlp *m, const nq_config *cfg, uint64_t *total, nq_stats *stats) try {
    return count_learned_impl(N, rows, m, nullptr, 0, 0, cfg, total, stats);
} catch (...) {
    return status_of_exception();
}

int nq_count_learned_reuse(int N, int rows, nq_mlp *m, const int64_t *done_idx, int64_t n_done, uint64_t done_sum,
                           const nq_config *cfg, uint64_t *total, nq_stats *stats) try {
    return count_learned_impl(N, rows, m, done_idx, n_done, done_sum, cfg, total, stats);
} catch (...) {
    return status_of_exception();
}

int nq_count_tasks(int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                   uint64_t *per_task, uint64_t *nodes_per_task, uint64_t *sum, const nq_config *cfg,
                   nq_stats *stats) try {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (N < 1 || N > NQ_MAX_N || n < 0 || !sum) return NQ_ERR_ARG;
    if (n > 0 && (!cols || !ld || !rd)) return NQ_ERR_ARG;
    if (n > 0xffffffffll) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    if (stats) stats->tasks = n;
    if (n == 0) {
        *sum = 0;
        if (stats) stats->total_ms = now_ms() - t0;
        return NQ_OK;
    }
    const int need = levels_for_tasks(N, cols, n, nodes_per_task == nullptr);
    rc = c.tasks.grow((size_t)n * 12);
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    NQ_CUDA(cudaMemcpyAsync(d, cols, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    NQ_CUDA(cudaMemcpyAsync(d + n, ld, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    NQ_CUDA(cudaMemcpyAsync(d + 2 * n, rd, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    const bool per_owner = per_task != nullptr || nodes_per_task != nullptr;
    const bool want_nodes = nodes_per_task != nullptr;
    std::vector<uint64_t> tmp;
    uint64_t *pt = per_task;
    if (per_owner && !pt) {
        tmp.resize((size_t)n);
        pt = tmp.data();
    }
    rc = count_resident(c, N, d, d + n, d + 2 * n, n, need, cfg, per_owner, want_nodes, pt, nodes_per_task, sum,
                        nullptr, stats, true);
    if (stats) stats->total_ms = now_ms() - t0;
    return rc;
} catch (...) {
    return status_of_exception();
}

int nq_count_tasks_device(int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd, int64_t n,
                          uint64_t *d_per_task, uint64_t *d_nodes, uint64_t *d_sum, const nq_config *cfg,
                          void *stream) try {
    if (N < 1 || N > NQ_MAX_N || n < 0 || !d_sum) return NQ_ERR_ARG;
    if (n > 0 && (!d_cols || !d_ld || !d_rd)) return NQ_ERR_ARG;
    if (n > 0xffffffffll) return NQ_ERR_ARG;
    if (d_nodes && !d_per_task) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // Without a host view of the tasks the stack must cover the deepest
    // possible task (an empty board) unless the caller states the depth.
    const bool per_owner = d_per_task != nullptr;
    const bool want_nodes = d_nodes != nullptr;
    const int need = (cfg && cfg->stack_levels > 0) ? cfg->stack_levels : stack_need(N, 0, !want_nodes);
    Launch L;
    rc = plan_launch(c, cfg, need, per_owner, want_nodes, L);
    if (rc) return rc;
    DfsParams p = base_params(c, N, n, cfg);
    long long qlen = n;
    rc = queue_len_of(cfg, n, qlen);
    if (rc) return rc;
    p.nqueue = qlen;
    p.cols = d_cols;
    p.ld = d_ld;
    p.rd = d_rd;
    p.sum_out = (unsigned long long *)d_sum;
    p.status_out = (unsigned long long *)d_sum + 1;
    if (cfg && cfg->order_kind == NQ_ORDER_GIVEN && cfg->order) p.order = cfg->order;
    if (per_owner) {
        p.out_cnt = (unsigned long long *)d_per_task;
        NQ_CUDA(cudaMemsetAsync(d_per_task, 0, (size_t)n * 8, s));
        if (want_nodes) {
            p.out_nodes = (unsigned long long *)d_nodes;
            NQ_CUDA(cudaMemsetAsync(d_nodes, 0, (size_t)n * 8, s));
        }
    }
    return enqueue_dfs(c, p, L, per_owner, want_nodes, s);
} catch (...) {
    return status_of_exception();
}

int nq_batch_create(const nq_instance *inst, int64_t n, int split_rows, const nq_config *cfg, nq_batch **out) try {
    if (!out) return NQ_ERR_ARG;
    *out = nullptr;
    if (n < 0 || (n > 0 && !inst) || split_rows < 0 || split_rows > 8) return NQ_ERR_ARG;
    if (n > 0x7fffffffll) return NQ_ERR_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (inst[i].N < 1 || inst[i].N > NQ_MAX_N) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    nq_batch *b = new nq_batch();
    rc = build_batch(c, inst, n, split_rows ? split_rows : kDefaultSplit, cfg, *b);
    if (rc) {
        destroy_batch(*b);
        delete b;
        return rc;
    }
    *out = b;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_batch_run(nq_batch *b, uint64_t *out, nq_stats *stats) try {
    if (!b || (b->n_inst > 0 && !out)) return NQ_ERR_ARG;
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    Ctx &c = g_ctx[b->device];
    std::lock_guard<std::mutex> lock(c.mu);
    NQ_CUDA(cudaSetDevice(b->device));
    int rc = run_batch(c, *b, stats);
    if (rc) return rc;
    for (int64_t i = 0; i < b->n_inst; ++i) {
        const int64_t u = b->inst_to_u[i];
        out[i] = b->h_res[3 + 2 * u] + 2 * b->h_res[3 + 2 * u + 1];
    }
    if (stats) stats->total_ms = now_ms() - t0;
    return status_from_bits(b->h_res[2]);
} catch (...) {
    return status_of_exception();
}

int nq_batch_destroy(nq_batch *b) try {
    if (!b) return NQ_OK;
    {
        Ctx &c = g_ctx[b->device];
        std::lock_guard<std::mutex> lock(c.mu);
        cudaSetDevice(b->device);
        destroy_batch(*b);
    }
    delete b;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_batch_autotune(const nq_instance *inst, int64_t n, int repeats, const nq_config *base, nq_tune_entry *table,
                      int table_cap, int *n_entries, nq_tune_entry *best) try {
    if (!inst || n <= 0 || repeats < 1 || !best || table_cap < 0 || (table_cap > 0 && !table)) return NQ_ERR_ARG;
    if (base && base->inner_steps > NQ_MAX_INNER_STEPS) return NQ_ERR_ARG;
    static const int kSplits[] = {3, 4, 5, 6, 7};
    static const int kThreads[] = {64, 128, 256, 512};
    static const int kLayouts[] = {NQ_LAYOUT_INTERLEAVED, NQ_LAYOUT_LANE_MAJOR};
    static const int kInner[] = {256, 4096};  // queue chunking tried beside the default
    nq_config cfg;
    if (base)
        cfg = *base;
    else
        memset(&cfg, 0, sizeof(cfg));
    const int inner0 = cfg.inner_steps > 0 ? ((cfg.inner_steps + 3) & ~3) : kDefaultInner;
    int count = 0;
    best->ms = -1.0;
    // Measures one configuration; NQ_ERR_DEPTH (the CTA cannot hold the
    // stacks) skips it.
    auto measure = [&](int split, int threads, int layout, int inner) -> int {
        cfg.block_threads = threads;
        cfg.layout = layout;
        cfg.inner_steps = inner;
        nq_batch *b = nullptr;
        int rc = nq_batch_create(inst, n, split, &cfg, &b);
        if (rc == NQ_ERR_DEPTH) return NQ_OK;
        if (rc) return rc;
        std::vector<uint64_t> outv((size_t)n);
        nq_stats st;
        rc = nq_batch_run(b, outv.data(), &st);  // warm-up
        double sum_ms = 0;
        for (int r = 0; r < repeats && rc == NQ_OK; ++r) {
            rc = nq_batch_run(b, outv.data(), &st);
            sum_ms += st.kernel_ms;
        }
        nq_batch_destroy(b);
        if (rc) return rc;
        nq_tune_entry e;
        e.split_rows = split;
        e.block_threads = threads;
        e.layout = layout;
        e.inner_steps = inner;
        e.ms = sum_ms / repeats;
        if (count < table_cap) table[count] = e;
        ++count;
        if (best->ms < 0 || e.ms < best->ms) *best = e;
        return NQ_OK;
    };
    for (int split : kSplits)
        for (int threads : kThreads)
            for (int layout : kLayouts) {
                const int rc = measure(split, threads, layout, inner0);
                if (rc) return rc;
            }
    if (best->ms < 0) return NQ_ERR_ARG;
    const nq_tune_entry first = *best;
    for (int inner : kInner) {
        if (inner == inner0) continue;
        const int rc = measure(first.split_rows, first.block_threads, first.layout, inner);
        if (rc) return rc;
    }
    if (n_entries) *n_entries = count;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_dihedral_expand(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, uint8_t *cls, int64_t cap,
                       int64_t *n_tasks, nq_dihedral_class *classes, int cap_classes, int *n_classes) try {
    std::vector<DihClass> tab;
    if (!dihedral_classes(N, rows, tab) || cap < 0 || cap_classes < 0) return NQ_ERR_ARG;
    if (cap > 0 && (!cols || !ld || !rd || !cls)) return NQ_ERR_ARG;
    static_assert(sizeof(DihClass) == sizeof(nq_dihedral_class), "class layout");
    if (classes)
        for (int i = 0; i < (int)tab.size() && i < cap_classes; ++i) memcpy(&classes[i], &tab[i], sizeof(DihClass));
    if (n_classes) *n_classes = (int)tab.size();
    const int64_t n = dihedral_expand(N, rows, cols, ld, rd, cls, cap);
    if (n < 0) return NQ_ERR_ARG;
    if (n_tasks) *n_tasks = n;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_count_dihedral(int N, int rows, const nq_config *cfg, uint64_t *total, nq_stats *stats) try {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!total || N < 4 || N > NQ_MAX_N || rows < 2 || rows > N - 2) return NQ_ERR_ARG;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    const double te = now_ms();
    const int64_t n = dihedral_expand(N, rows, nullptr, nullptr, nullptr, nullptr, 0);
    if (n < 0 || n > 0xffffffffll) return NQ_ERR_ARG;
    // host staging: cols | ld | rd (u32) | cls (u8)
    rc = c.h_tasks.grow((size_t)std::max<int64_t>(n, 1) * 13);
    if (rc) return rc;
    uint32_t *h = (uint32_t *)c.h_tasks.p;
    uint8_t *hc = (uint8_t *)(h + 3 * n);
    dihedral_expand(N, rows, h, h + n, h + 2 * n, hc, n);
    if (stats) {
        stats->expand_ms = now_ms() - te;
        stats->tasks = n;
    }
    rc = c.tasks.grow(dih_bytes(n));
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    DihArgs a;
    a.task_cls = (const uint8_t *)(d + 3 * n);
    rc = dih_upload_classes(c, N, rows, (size_t)n * 13, a);
    if (rc) return rc;
    NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    if (n) NQ_CUDA(cudaMemcpyAsync(d, h, (size_t)n * 13, cudaMemcpyHostToDevice, c.stream));
    uint64_t sum = 0;
    rc = count_resident(c, N, d, d + n, d + 2 * n, n, stack_need(N, rows, false), cfg, false, false, nullptr, nullptr, &sum,
                        nullptr, stats, true, nullptr, &a);
    *total = sum;  // the class weights already carry every symmetry factor
    if (stats) stats->total_ms = now_ms() - t0;
    return rc;
} catch (...) {
    return status_of_exception();
}

int nq_count_dihedral_tasks(int N, int rows, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                            const uint8_t *cls, int64_t n, uint64_t *per_task, uint64_t *sum, const nq_config *cfg,
                            nq_stats *stats) try {
    const double t0 = now_ms();
    if (stats) memset(stats, 0, sizeof(*stats));
    std::vector<DihClass> tab;
    if (!sum || n < 0 || n > 0xffffffffll || !dihedral_classes(N, rows, tab)) return NQ_ERR_ARG;
    if (n > 0 && (!cols || !ld || !rd || !cls)) return NQ_ERR_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (cls[i] >= tab.size()) return NQ_ERR_ARG;
    *sum = 0;
    if (n == 0) return NQ_OK;
    Ctx *cp = nullptr;
    int rc = lock_device(device_of(cfg), cp);
    if (rc) return rc;
    Ctx &c = *cp;
    std::lock_guard<std::mutex> lock(c.mu);
    rc = ensure_ready(c, device_of(cfg));
    if (rc) return rc;
    rc = c.tasks.grow(dih_bytes(n));
    if (rc) return rc;
    uint32_t *d = (uint32_t *)c.tasks.p;
    DihArgs a;
    a.task_cls = (const uint8_t *)(d + 3 * n);
    rc = dih_upload_classes(c, N, rows, (size_t)n * 13, a);
    if (rc) return rc;
    NQ_CUDA(cudaEventRecord(c.ev[0], c.stream));
    NQ_CUDA(cudaMemcpyAsync(d, cols, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    NQ_CUDA(cudaMemcpyAsync(d + n, ld, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    NQ_CUDA(cudaMemcpyAsync(d + 2 * n, rd, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    NQ_CUDA(cudaMemcpyAsync(d + 3 * n, cls, (size_t)n, cudaMemcpyHostToDevice, c.stream));
    const int need = levels_for_tasks(N, cols, n, false);
    rc = count_resident(c, N, d, d + n, d + 2 * n, n, need, cfg, per_task != nullptr, false, per_task, nullptr, sum,
                        nullptr, stats, true, nullptr, &a);
    if (stats) stats->total_ms = now_ms() - t0;
    return rc;
} catch (...) {
    return status_of_exception();
}

int nq_count_batch(const nq_instance *inst, int64_t n, int split_rows, uint64_t *out, const nq_config *cfg,
                   nq_stats *stats) try {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n == 0) return (n < 0 || split_rows < 0 || split_rows > 8) ? NQ_ERR_ARG : NQ_OK;
    nq_batch *b = nullptr;
    int rc = nq_batch_create(inst, n, split_rows, cfg, &b);
    if (rc) return rc;
    rc = nq_batch_run(b, out, stats);
    nq_batch_destroy(b);
    return rc;
} catch (...) {
    return status_of_exception();
}

}  // extern "C"
