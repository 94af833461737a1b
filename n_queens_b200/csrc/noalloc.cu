// noalloc.cu -- a device-resident count that allocates no memory at all.
//
// Every other entry of this library keeps its own device scratch (the task
// queue word, the completion/error flags and one partial sum per CTA) in
// memory it obtains with cudaMalloc the first time a device is used.  Some
// callers cannot let a library do that: a host framework whose caching
// allocator has already reserved the GPU's memory and wants every byte to go
// through it, or a service that forbids device allocation after start-up
// because an allocation can stall or fail mid-run.  For them this file keeps
// the same scratch in a fixed-size array that is part of the loaded library
// image, so counting needs no allocation from anyone.  The caller still owns
// and passes the task arrays and the two-word result.
//
// Limits and sharing rules (also stated in include/n_queens_b200.h):
//  * the array holds the control words and one partial per CTA for at most
//    kNoAllocMaxCtas CTAs (about 64 KiB); every GPU that loads the library
//    holds this array until the process exits;
//  * all calls share the one array: the control words are cleared at the
//    start of every call, and calls whose kernels overlap on the GPU (two
//    streams, or two host threads) race on it and must be serialised;
//  * the first call on a device does that device's set-up
//    (cudaGetSymbolAddress of the array, the shared-memory opt-in of the
//    kernel); make that first call before any stream capture begins.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "dfs_kernel.cuh"
#include "launch.h"
#include "n_queens_b200.h"

namespace nqb {

// Sets the text returned by nq_last_error() (defined in capi.cu).
void set_last_error(const char *msg);
// Status of the exception in flight, for the entry's handler (defined in capi.cu).
int status_of_exception() noexcept;

namespace {

constexpr int kNoAllocMaxCtas = 8192;
constexpr int kNoAllocWords = 8 + kNoAllocMaxCtas;  // control + results + per-CTA partials
constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxBlocksPerSm = 32;

// The scratch itself.  In host code `g_noalloc_scratch` is only a host-side
// stand-in for the device symbol: its device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

struct NoAllocDev {
    bool ready = false;
    unsigned long long *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
    int smem_optin = 0;
};

std::mutex g_noalloc_mu;
NoAllocDev g_noalloc_dev[kNoAllocMaxDevices];

typedef void (*NoAllocKernel)(DfsParams);
// The same instantiation the allocating device entry runs for a plain count.
NoAllocKernel noalloc_kernel() { return dfs_kernel<false, false, kStepVar, kCountUnroll>; }

int noalloc_fail(cudaError_t e, const char *what) {
    set_last_error((std::string(what) + ": " + cudaGetErrorString(e)).c_str());
    (void)cudaGetLastError();
    return NQ_ERR_CUDA;
}

// Puts the caller's current device back when the entry returns, so a host
// framework that keeps its own notion of the current device never sees it
// change.
struct CurrentDeviceGuard {
    int saved = -1;
    ~CurrentDeviceGuard() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

// The device checks of the other entries: a device must exist, the ordinal
// must be in range, and the device must be an sm_100 part (the library
// carries only an sm_100a image).
int noalloc_check_device(int dev) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        set_last_error("no CUDA device");
        return NQ_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= n || dev >= kNoAllocMaxDevices) {
        set_last_error("device ordinal out of range");
        return NQ_ERR_ARG;
    }
    int major = 0, minor = 0;
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaDeviceGetAttribute");
    e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaDeviceGetAttribute");
    if (major != 10 || minor != 0) {
        set_last_error(("device is sm_" + std::to_string(major) + std::to_string(minor) +
                        "; this library carries only an sm_100a image")
                           .c_str());
        return NQ_ERR_NO_KERNEL;
    }
    return NQ_OK;
}

// Once per device, with that device current.
int noalloc_setup(int dev, NoAllocDev &d) {
    if (d.ready) return NQ_OK;
    cudaError_t e = cudaGetSymbolAddress((void **)&d.scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaDeviceGetAttribute");
    e = cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaDeviceGetAttribute");
    e = cudaFuncSetAttribute(noalloc_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             d.smem_optin - kDfsStaticSmem);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaFuncSetAttribute");
    d.ready = true;
    return NQ_OK;
}

}  // namespace
}  // namespace nqb

using namespace nqb;

extern "C" int nq_count_tasks_device_noalloc(int N, const uint32_t *d_cols, const uint32_t *d_ld,
                                             const uint32_t *d_rd, int64_t n, uint64_t *d_sum,
                                             const nq_config *cfg, void *stream) try {
    if (N < 1 || N > NQ_MAX_N || n < 0 || n > 0xffffffffll || !d_sum) return NQ_ERR_ARG;
    if (n > 0 && (!d_cols || !d_ld || !d_rd)) return NQ_ERR_ARG;
    const int dev = cfg ? cfg->device : 0;
    int rc = noalloc_check_device(dev);
    if (rc) return rc;
    CurrentDeviceGuard guard;
    cudaError_t e = cudaGetDevice(&guard.saved);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaGetDevice");
    if (guard.saved != dev) {
        e = cudaSetDevice(dev);
        if (e != cudaSuccess) return noalloc_fail(e, "cudaSetDevice");
    } else {
        guard.saved = -1;  // nothing to restore
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDev &d = g_noalloc_dev[dev];
    rc = noalloc_setup(dev, d);
    if (rc) return rc;
    if (d.sms > kNoAllocMaxCtas) {
        set_last_error("this GPU has more SMs than the fixed scratch array has CTA slots");
        return NQ_ERR_ARG;
    }
    if (cfg && cfg->blocks_per_sm > 0 && (long long)cfg->blocks_per_sm * d.sms > kNoAllocMaxCtas) {
        set_last_error(("blocks_per_sm x SMs exceeds the " + std::to_string(kNoAllocMaxCtas) +
                        " CTAs that the fixed scratch array can hold")
                           .c_str());
        return NQ_ERR_ARG;
    }

    // Launch shape: chosen exactly as the allocating entries choose it (the
    // CTA size that keeps the most warps resident for the stack depth, 1024
    // DFS steps between queue visits), with the grid bounded by the array's
    // per-CTA partials.
    if (cfg && cfg->stack_levels > NQ_MAX_STACK_LEVELS) {
        set_last_error("stack_levels is above NQ_MAX_STACK_LEVELS");
        return NQ_ERR_ARG;
    }
    const int levels = (cfg && cfg->stack_levels > 0) ? cfg->stack_levels : stack_need(N, 0, true);
    int cap_per_sm = std::min(kNoAllocMaxBlocksPerSm, std::max(1, kNoAllocMaxCtas / d.sms));
    if (cfg && cfg->blocks_per_sm > 0) cap_per_sm = std::min(cap_per_sm, cfg->blocks_per_sm);
    const int threads = (cfg && cfg->block_threads)
                            ? cfg->block_threads
                            : resident_warp_threads(noalloc_kernel(), levels, d.smem_optin, cap_per_sm);
    if (threads == 0) {
        set_last_error("no CTA size of 64 or more threads fits this stack depth in shared memory");
        return NQ_ERR_DEPTH;
    }
    if (threads < 32 || threads > 1024 || (threads & 31)) return NQ_ERR_ARG;
    const long long smem64 = (long long)(threads / 32) * levels * kSlotBytes;
    if (smem64 + kDfsStaticSmem > d.smem_optin) {
        set_last_error("per-CTA stack does not fit in shared memory: lower block_threads or stack_levels");
        return NQ_ERR_DEPTH;
    }
    const int smem = (int)smem64;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_kernel(), threads, smem);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm <= 0) {
        set_last_error("launch configuration cannot be resident");
        return NQ_ERR_ARG;
    }
    per_sm = std::min(per_sm, cap_per_sm);
    const int grid = d.sms * per_sm;

    DfsParams p;
    memset(&p, 0, sizeof(p));
    p.cols = d_cols;
    p.ld = d_ld;
    p.rd = d_rd;
    p.ntasks = n;
    if (cfg && cfg->queue_len) {
        if ((int64_t)cfg->queue_len > n) {
            set_last_error("queue_len exceeds the number of tasks");
            return NQ_ERR_ARG;
        }
        p.nqueue = (long long)cfg->queue_len;
    }
    p.N = N;
    p.levels = levels;
    if (cfg && cfg->inner_steps > NQ_MAX_INNER_STEPS) {
        set_last_error("inner_steps is above NQ_MAX_INNER_STEPS");
        return NQ_ERR_ARG;
    }
    p.inner = (cfg && cfg->inner_steps > 0) ? ((cfg->inner_steps + 3) & ~3) : kDefaultInner;
    p.steal = (cfg && cfg->steal < 0) ? 0 : 1;
    p.layout = (cfg && cfg->layout == NQ_LAYOUT_LANE_MAJOR) ? 1 : 0;
    p.limit_ns = cfg ? (unsigned long long)cfg->time_limit_ms * 1000000ull : 0ull;
    p.order = (cfg && cfg->order_kind == NQ_ORDER_GIVEN) ? cfg->order : nullptr;
    p.ctl = d.scratch;  // words 0..4: queue head, CTAs done, error bits, timeout flag, continuation count
    p.block_cnt = d.scratch + 8;
    p.block_nodes = d.scratch + 8;  // unused: this variant counts no nodes
    p.sum_out = (unsigned long long *)d_sum;
    p.nodes_out = d.scratch + 5;
    p.status_out = (unsigned long long *)d_sum + 1;
    p.k_one = 1;
    p.k_two = 2;
    p.k_mone = 0xffffffffu;

    cudaStream_t s = (cudaStream_t)stream;
    // The previous call left its control words behind (queue head, done
    // ticket, error and timeout words): clear all of them.
    e = cudaMemsetAsync(d.scratch, 0, kCtlWords * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return noalloc_fail(e, "cudaMemsetAsync");
    noalloc_kernel()<<<grid, threads, smem, s>>>(p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(e, "dfs_kernel launch");
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}
