// mlp.cu -- the learned subtree-cost model and the longest-first scheduler.
//
// No counterpart in the reference (its tasks run in expander order through
// one atomic ticket, src/n_queens_cuda.cu:10,80).  A small MLP predicts
// log2(1 + DFS nodes) of a prefix task from its three masks; the predictions
// order the task queue longest-first (binned to 1/8 of a log2 unit, stable
// inside a bin).  The order only changes which lane runs which task, never a
// count.
//
// Model: x (96 bits: cols, ld, rd, each as 32 bits with the columns >= N
// cleared) -> 128 ReLU -> 128 ReLU -> 1.  Weights are BF16 for compute with
// FP32 master copies for Adam; biases are FP32; every sum accumulates in
// FP32.  Kernels (all hand-written, CUDA cores; at 29k parameters the model
// is far too small for tensor-core tiles to pay):
//   mlp_predict_kernel  forward for many tasks, 32 tasks per group per CTA
//   mlp_train_kernel    forward + backward of a minibatch slice; per-CTA
//                       partial gradients (no atomics: deterministic)
//   mlp_adam_kernel     sums the partials in CTA order, Adam step, refreshes
//                       the BF16 copies
// The first layer exploits binary inputs: h1 = b1 + sum of the W1 columns of
// the set bits (about 3k of them for a k-row prefix), so no feature matrix
// is ever materialised.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <cmath>
#include <cub/device/device_radix_sort.cuh>
#include <mutex>
#include <string>
#include <vector>

#include "dfs_kernel.cuh"
#include "expand.h"
#include "n_queens_b200.h"

namespace nqb {

void set_last_error(const char *msg);
// Status of the exception in flight, for the entries' handlers (defined in capi.cu).
int status_of_exception() noexcept;

namespace {

constexpr int kIn = 96, kH1 = 128, kH2 = 128;
// Flat FP32 parameter layout (also the layout of gradients and of
// nq_mlp_get_params): W1[H1][IN], b1[H1], W2[H2][H1], b2[H2], W3[H2], b3.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH1 * kIn;
constexpr int kOffW2 = kOffB1 + kH1;
constexpr int kOffB2 = kOffW2 + kH2 * kH1;
constexpr int kOffW3 = kOffB2 + kH2;
constexpr int kOffB3 = kOffW3 + kH2;
constexpr int kParams = kOffB3 + 1;
constexpr int kGroup = 32;  // tasks per group (one per lane of the layer-3 reduction)

// Compute copy of the weights in device memory.
struct Weights {
    __nv_bfloat16 w1t[kIn * kH1];  // [input bit][hidden unit]
    __nv_bfloat16 w2[kH2 * kH1];   // [unit of layer 2][unit of layer 1]
    __nv_bfloat16 w3[kH2];
    float b1[kH1];
    float b2[kH2];
    float b3;
};

struct TaskView {
    const uint32_t *cols, *ld, *rd;
    const uint8_t *task_n;  // per-task board size or nullptr
    const uint32_t *index;  // optional indirection (training permutation)
    int N;
};

__device__ __forceinline__ void load_masks(const TaskView &tv, long long t, uint32_t &m0, uint32_t &m1,
                                           uint32_t &m2) {
    const long long i = tv.index ? (long long)tv.index[t] : t;
    const int n = tv.task_n ? (int)tv.task_n[i] : tv.N;
    const uint32_t last = (n >= 32) ? 0xffffffffu : ((1u << n) - 1u);
    m0 = tv.cols[i] & last;
    m1 = tv.ld[i] & last;
    m2 = tv.rd[i] & last;
}

// Layer 1 for one task and hidden unit j: b1[j] + sum of W1 columns of the
// set input bits.  Every thread of the CTA walks the same bits (uniform).
__device__ __forceinline__ float layer1(const __nv_bfloat16 *w1t, float b, uint32_t m0, uint32_t m1, uint32_t m2,
                                        int j) {
    float acc = b;
    while (m0) {
        const int f = __ffs(m0) - 1;
        m0 &= m0 - 1;
        acc += __bfloat162float(w1t[f * kH1 + j]);
    }
    while (m1) {
        const int f = __ffs(m1) - 1 + 32;
        m1 &= m1 - 1;
        acc += __bfloat162float(w1t[f * kH1 + j]);
    }
    while (m2) {
        const int f = __ffs(m2) - 1 + 64;
        m2 &= m2 - 1;
        acc += __bfloat162float(w1t[f * kH1 + j]);
    }
    return acc;
}

// Layer 2 pre-activation of unit j for one task: w2row holds W2[j][:] as
// 64 packed BF16 pairs, h1 the task's 128 layer-1 outputs (broadcast reads).
__device__ __forceinline__ float layer2(const uint32_t (&w2row)[kH1 / 2], float b, const float *h1) {
    float acc = b;
#pragma unroll
    for (int i = 0; i < kH1; i += 4) {
        const float4 h = *reinterpret_cast<const float4 *>(h1 + i);
        const __nv_bfloat162 wa = *reinterpret_cast<const __nv_bfloat162 *>(&w2row[i / 2]);
        const __nv_bfloat162 wb = *reinterpret_cast<const __nv_bfloat162 *>(&w2row[i / 2 + 1]);
        acc = fmaf(__low2float(wa), h.x, acc);
        acc = fmaf(__high2float(wa), h.y, acc);
        acc = fmaf(__low2float(wb), h.z, acc);
        acc = fmaf(__high2float(wb), h.w, acc);
    }
    return acc;
}

__device__ __forceinline__ void load_w2row(const Weights *w, int j, uint32_t (&w2row)[kH1 / 2]) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(w->w2 + j * kH1);
#pragma unroll
    for (int i = 0; i < kH1 / 2; ++i) w2row[i] = src[i];
}

// Forward over n tasks: out[t] = predicted log2(1 + nodes).  128 threads,
// thread j = hidden unit j.
__global__ void __launch_bounds__(128) mlp_predict_kernel(TaskView tv, long long n, const Weights *w, float *out) {
    __shared__ __align__(16) __nv_bfloat16 s_w1t[kIn * kH1];
    __shared__ __align__(16) float s_h[kGroup * kH1];
    __shared__ uint32_t s_m[3][kGroup];
    const int j = threadIdx.x;
    for (int i = j; i < kIn * kH1 / 8; i += blockDim.x)
        reinterpret_cast<uint4 *>(s_w1t)[i] = reinterpret_cast<const uint4 *>(w->w1t)[i];
    uint32_t w2row[kH1 / 2];
    load_w2row(w, j, w2row);
    const float b1 = w->b1[j], b2 = w->b2[j], w3 = __bfloat162float(w->w3[j]), b3 = w->b3;
    const int warp = j >> 5, lane = j & 31;
    __syncthreads();
    for (long long g0 = (long long)blockIdx.x * kGroup; g0 < n; g0 += (long long)gridDim.x * kGroup) {
        const int gn = (int)min((long long)kGroup, n - g0);
        if (j < gn) load_masks(tv, g0 + j, s_m[0][j], s_m[1][j], s_m[2][j]);
        __syncthreads();
        for (int s = 0; s < gn; ++s)
            s_h[s * kH1 + j] = fmaxf(layer1(s_w1t, b1, s_m[0][s], s_m[1][s], s_m[2][s], j), 0.f);
        __syncthreads();
        float v[kGroup];
#pragma unroll
        for (int s = 0; s < kGroup; ++s) v[s] = (s < gn) ? fmaxf(layer2(w2row, b2, s_h + s * kH1), 0.f) * w3 : 0.f;
        __syncthreads();
#pragma unroll
        for (int s = 0; s < kGroup; ++s) s_h[s * kH1 + j] = v[s];
        __syncthreads();
        // layer 3: warp w reduces tasks 8w..8w+7, each lane summing 4 units
        for (int s = warp * 8; s < warp * 8 + 8; ++s) {
            const float4 q = *reinterpret_cast<const float4 *>(s_h + s * kH1 + lane * 4);
            float a = (q.x + q.y) + (q.z + q.w);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == 0 && s < gn) out[g0 + s] = a + b3;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Tensor-core inference (tcgen05).  Per tile of 128 tasks, one CTA of 128
// threads (thread t = task row t = TMEM lane t):
//   X (128 x 96 binary, BF16) --tcgen05.mma--> D1 (TMEM, FP32) --relu+b1,
//   BF16--> H1 (128 x 128, smem) --tcgen05.mma--> D2 (TMEM) --relu+b2, dot W3,
//   +b3--> out.
// Operands use the SM100 K-major canonical layout without swizzle: 8-row x
// 16-byte core matrices, LBO = 128 B between the two core matrices of one
// K=16 step, SBO = K/8 * 128 B between 8-row groups.  One thread issues the
// MMAs; completion is signalled through an mbarrier (tcgen05.commit) and every
// wait on it is bounded (on expiry the kernel sets *err and stops).
namespace tc {

constexpr uint32_t kSbo1 = (kIn / 8) * 128;   // 1536 B
constexpr uint32_t kSbo2 = (kH1 / 8) * 128;   // 2048 B
constexpr uint32_t kOffB1 = 0;                 // W1: 128 units x 96  (24 KiB)
constexpr uint32_t kOffB2 = kOffB1 + kH1 * kSbo1 / 8;  // 24576: W2: 128 x 128 (32 KiB)
constexpr uint32_t kOffA = kOffB2 + kH2 * kSbo2 / 8;   // 57344: X / H1 tile (32 KiB)
constexpr uint32_t kOffBias = kOffA + 128 * kSbo2 / 8;  // 90112: b1, b2, w3 (fp32)
constexpr uint32_t kOffBar = kOffBias + 3 * 128 * 4;    // 91648: mbarrier (8 B)
constexpr uint32_t kOffTmem = kOffBar + 8;              // TMEM base address word
constexpr uint32_t kSmemBytes = kOffTmem + 8;
constexpr uint32_t kTmemCols = 256;  // D1 at column 0, D2 at column 128
// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major,
// N = 128 (N>>3 at bit 17), M = 128 (M>>4 at bit 24).
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
constexpr unsigned long long kWaitLimit = 1ull << 22;  // a few seconds at most

__host__ __device__ constexpr uint32_t off_kmajor(uint32_t row, uint32_t k, uint32_t sbo) {
    return (row >> 3) * sbo + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}
static_assert(off_kmajor(127, 95, kSbo1) < kOffB2 - kOffB1, "W1 tile bounds");
static_assert(off_kmajor(127, 127, kSbo2) < kOffA - kOffB2, "W2 tile bounds");
static_assert(off_kmajor(127, 127, kSbo2) < kOffBias - kOffA, "A tile bounds");

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1; base offset 0; no swizzle
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false on expiry.
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity) {
    for (unsigned long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a -> low half
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void sts128(uint32_t addr, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}

}  // namespace tc

__global__ void __launch_bounds__(128, 1)
    mlp_predict_tc_kernel(TaskView tv, long long n, const Weights *w, float *out, int *err) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(tc_smem);
    const uint32_t t = threadIdx.x, warp = t >> 5;
    float *bias = reinterpret_cast<float *>(tc_smem + tc::kOffBias);
    const uint32_t bar = base + tc::kOffBar;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tc_smem + tc::kOffTmem);

    // Weights into the canonical operand layouts (BF16 copies as stored).
    for (uint32_t i = t; i < (uint32_t)(kH1 * kIn); i += blockDim.x) {
        const uint32_t unit = i / kIn, k = i % kIn;
        *reinterpret_cast<__nv_bfloat16 *>(tc_smem + tc::kOffB1 + tc::off_kmajor(unit, k, tc::kSbo1)) =
            w->w1t[k * kH1 + unit];
    }
    for (uint32_t i = t; i < (uint32_t)(kH2 * kH1); i += blockDim.x) {
        const uint32_t unit = i / kH1, k = i % kH1;
        *reinterpret_cast<__nv_bfloat16 *>(tc_smem + tc::kOffB2 + tc::off_kmajor(unit, k, tc::kSbo2)) =
            w->w2[unit * kH1 + k];
    }
    bias[t] = w->b1[t];
    bias[128 + t] = w->b2[t];
    bias[256 + t] = __bfloat162float(w->w3[t]);
    const float b3 = w->b3;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + tc::kOffTmem),
                     "r"(tc::kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_off = (warp * 32u) << 16;  // this warp's TMEM lanes
    const uint32_t d1 = tmem, d2 = tmem + 128;
    uint32_t phase = 0;
    __shared__ int s_fail;
    if (t == 0) s_fail = 0;
    __syncthreads();

    for (long long g0 = (long long)blockIdx.x * 128; g0 < n; g0 += (long long)gridDim.x * 128) {
        // ---- X row of this thread's task (zeros past the end)
        uint32_t m0 = 0, m1 = 0, m2 = 0;
        if (g0 + t < n) load_masks(tv, g0 + t, m0, m1, m2);
        const uint32_t masks[3] = {m0, m1, m2};
#pragma unroll
        for (int c = 0; c < kIn / 8; ++c) {
            const uint32_t byte = (masks[c >> 2] >> ((c & 3) * 8)) & 0xFFu;
            uint32_t q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                q[j] = ((byte >> (2 * j)) & 1u ? 0x3F80u : 0u) | ((byte >> (2 * j + 1)) & 1u ? 0x3F800000u : 0u);
            tc::sts128(base + tc::kOffA + tc::off_kmajor(t, 8 * c, tc::kSbo1), q[0], q[1], q[2], q[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // ---- layer 1 on the tensor cores: D1 = X * W1^T, K = 96 in 6 steps
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kIn / 16; ++kk)
                tc::mma(d1, tc::smem_desc(base + tc::kOffA + kk * 256, 128, tc::kSbo1),
                        tc::smem_desc(base + tc::kOffB1 + kk * 256, 128, tc::kSbo1), kk > 0);
            tc::commit(bar);
        }
        if (!tc::wait_phase(bar, phase)) s_fail = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (s_fail) break;
        // ---- relu(D1 + b1) -> BF16 -> H1 rows (the A operand of layer 2)
#pragma unroll 1
        for (int c = 0; c < kH1 / 16; ++c) {
            float v[16];
            tc::ld16(d1 + lane_off + 16 * c, v);
            uint32_t q[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                q[j] = tc::pack_bf16(fmaxf(v[2 * j] + bias[16 * c + 2 * j], 0.f),
                                     fmaxf(v[2 * j + 1] + bias[16 * c + 2 * j + 1], 0.f));
            tc::sts128(base + tc::kOffA + tc::off_kmajor(t, 16 * c, tc::kSbo2), q[0], q[1], q[2], q[3]);
            tc::sts128(base + tc::kOffA + tc::off_kmajor(t, 16 * c + 8, tc::kSbo2), q[4], q[5], q[6], q[7]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // ---- layer 2: D2 = H1 * W2^T, K = 128 in 8 steps
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kH1 / 16; ++kk)
                tc::mma(d2, tc::smem_desc(base + tc::kOffA + kk * 256, 128, tc::kSbo2),
                        tc::smem_desc(base + tc::kOffB2 + kk * 256, 128, tc::kSbo2), kk > 0);
            tc::commit(bar);
        }
        if (!tc::wait_phase(bar, phase)) s_fail = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (s_fail) break;
        // ---- layer 3: sum_j relu(D2 + b2)_j * w3_j + b3
        float acc = 0.f;
#pragma unroll 1
        for (int c = 0; c < kH2 / 16; ++c) {
            float v[16];
            tc::ld16(d2 + lane_off + 16 * c, v);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                acc = fmaf(fmaxf(v[j] + bias[128 + 16 * c + j], 0.f), bias[256 + 16 * c + j], acc);
        }
        if (g0 + t < n) out[g0 + t] = acc + b3;
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (s_fail && t == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols));
}

// Shared memory of the training kernel (about 216 KiB; one CTA per SM).
struct TrainSmem {
    __nv_bfloat16 w1t[kIn * kH1];    // 24 KiB
    __nv_bfloat162 w2p[kH2 / 2 * kH1];  // 32 KiB: w2p[(j/2)*H1 + i] = (W2[j][i], W2[j+1][i])
    float h1[kGroup * kH1];          // 16 KiB: relu(layer 1), [task][unit]
    float h2[kGroup * kH1];          // 16 KiB: relu(layer 2), then dL/d(pre-act 2)
    float dh1[kGroup * kH1];         // 16 KiB: dL/d(pre-act 1)
    float dw1[kIn * kH1];            // 48 KiB: [input bit][unit]
    float dw2[kH1 * kH2];            // 64 KiB: [unit of layer 1][unit of layer 2]
    float dout[kGroup];
    float y[kGroup];
    uint32_t m[3][kGroup];
};

// Forward + backward of tasks [begin, end) of the view (mean-squared-error
// loss with gradient scale `scale` = 2/batch), one partial gradient per CTA.
__global__ void __launch_bounds__(128, 1)
    mlp_train_kernel(TaskView tv, const float *target, long long begin, long long end, float scale,
                     const Weights *w, float *grad_part, float *loss_part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
    const int j = threadIdx.x;  // unit index in every layer (H1 == H2 == blockDim.x)
    const int warp = j >> 5, lane = j & 31;
    for (int i = j; i < kIn * kH1 / 8; i += blockDim.x)
        reinterpret_cast<uint4 *>(S.w1t)[i] = reinterpret_cast<const uint4 *>(w->w1t)[i];
    for (int jj = 0; jj < kH2; jj += 2)
        S.w2p[(jj / 2) * kH1 + j] = __halves2bfloat162(w->w2[jj * kH1 + j], w->w2[(jj + 1) * kH1 + j]);
    for (int i = j; i < kIn * kH1; i += blockDim.x) S.dw1[i] = 0.f;
    for (int i = j; i < kH1 * kH2; i += blockDim.x) S.dw2[i] = 0.f;
    uint32_t w2row[kH1 / 2];
    load_w2row(w, j, w2row);
    const float b1 = w->b1[j], b2 = w->b2[j], w3 = __bfloat162float(w->w3[j]), b3 = w->b3;
    float w3q[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) w3q[k] = __bfloat162float(w->w3[lane * 4 + k]);
    float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, loss = 0.f;
    __syncthreads();

    for (long long g0 = begin + (long long)blockIdx.x * kGroup; g0 < end; g0 += (long long)gridDim.x * kGroup) {
        const int gn = (int)min((long long)kGroup, end - g0);
        if (j < kGroup) {
            if (j < gn) {
                load_masks(tv, g0 + j, S.m[0][j], S.m[1][j], S.m[2][j]);
                const long long i = tv.index ? (long long)tv.index[g0 + j] : g0 + j;
                S.y[j] = target[i];
            } else {
                S.m[0][j] = S.m[1][j] = S.m[2][j] = 0;
                S.y[j] = 0.f;
            }
        }
        __syncthreads();
        // forward
        for (int s = 0; s < gn; ++s)
            S.h1[s * kH1 + j] = fmaxf(layer1(S.w1t, b1, S.m[0][s], S.m[1][s], S.m[2][s], j), 0.f);
        __syncthreads();
        for (int s = 0; s < gn; ++s) S.h2[s * kH1 + j] = fmaxf(layer2(w2row, b2, S.h1 + s * kH1), 0.f);
        __syncthreads();
        for (int s = warp * 8; s < warp * 8 + 8; ++s) {
            const float4 q = *reinterpret_cast<const float4 *>(S.h2 + s * kH1 + lane * 4);
            float a = q.x * w3q[0];
            a = fmaf(q.y, w3q[1], a);
            a = fmaf(q.z, w3q[2], a);
            a = fmaf(q.w, w3q[3], a);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == 0) {
                const float e = (s < gn) ? (a + b3 - S.y[s]) : 0.f;
                S.dout[s] = scale * e;
                loss += e * e;
            }
        }
        __syncthreads();
        // layer 3 and layer 2 backward (thread j = unit of layer 2)
        for (int s = 0; s < gn; ++s) {
            const float h = S.h2[s * kH1 + j];
            const float d = S.dout[s];
            gw3 = fmaf(d, h, gw3);
            const float dh = (h > 0.f) ? d * w3 : 0.f;
            S.h2[s * kH1 + j] = dh;
            gb2 += dh;
        }
        if (j == 0)
            for (int s = 0; s < gn; ++s) gb3 += S.dout[s];
        __syncthreads();
        // dW2[j][i] += sum_s dh2[s][j] * h1[s][i]   (accumulated as dw2[i][j])
        for (int i0 = 0; i0 < kH1; i0 += 32) {
            float acc[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) acc[k] = 0.f;
            for (int s = 0; s < gn; ++s) {
                const float d = S.h2[s * kH1 + j];
#pragma unroll
                for (int k = 0; k < 32; k += 4) {
                    const float4 h = *reinterpret_cast<const float4 *>(S.h1 + s * kH1 + i0 + k);
                    acc[k] = fmaf(d, h.x, acc[k]);
                    acc[k + 1] = fmaf(d, h.y, acc[k + 1]);
                    acc[k + 2] = fmaf(d, h.z, acc[k + 2]);
                    acc[k + 3] = fmaf(d, h.w, acc[k + 3]);
                }
            }
#pragma unroll
            for (int k = 0; k < 32; ++k) S.dw2[(i0 + k) * kH2 + j] += acc[k];
        }
        // dh1[s][i] = relu'(h1) * sum_j W2[j][i] dh2[s][j]   (thread j acts as unit i of layer 1)
        for (int s = 0; s < gn; ++s) {
            float acc = 0.f;
            const float *dh2 = S.h2 + s * kH1;
#pragma unroll 8
            for (int jj = 0; jj < kH2; jj += 4) {
                const float4 d = *reinterpret_cast<const float4 *>(dh2 + jj);
                const __nv_bfloat162 wa = S.w2p[(jj / 2) * kH1 + j];
                const __nv_bfloat162 wb = S.w2p[(jj / 2 + 1) * kH1 + j];
                acc = fmaf(__low2float(wa), d.x, acc);
                acc = fmaf(__high2float(wa), d.y, acc);
                acc = fmaf(__low2float(wb), d.z, acc);
                acc = fmaf(__high2float(wb), d.w, acc);
            }
            const float dh = (S.h1[s * kH1 + j] > 0.f) ? acc : 0.f;
            S.dh1[s * kH1 + j] = dh;
            gb1 += dh;
        }
        __syncthreads();
        // dW1[i][f] += sum_s dh1[s][i] over the set bits f of task s
        for (int s = 0; s < gn; ++s) {
            const float d = S.dh1[s * kH1 + j];
            uint32_t m0 = S.m[0][s], m1 = S.m[1][s], m2 = S.m[2][s];
            while (m0) {
                const int f = __ffs(m0) - 1;
                m0 &= m0 - 1;
                S.dw1[f * kH1 + j] += d;
            }
            while (m1) {
                const int f = __ffs(m1) - 1 + 32;
                m1 &= m1 - 1;
                S.dw1[f * kH1 + j] += d;
            }
            while (m2) {
                const int f = __ffs(m2) - 1 + 64;
                m2 &= m2 - 1;
                S.dw1[f * kH1 + j] += d;
            }
        }
        __syncthreads();
    }

    // Partial gradient of this CTA in the flat parameter layout.
    float *g = grad_part + (size_t)blockIdx.x * kParams;
    for (int f = 0; f < kIn; ++f) g[kOffW1 + j * kIn + f] = S.dw1[f * kH1 + j];
    g[kOffB1 + j] = gb1;
    for (int i = 0; i < kH1; ++i) g[kOffW2 + j * kH1 + i] = S.dw2[i * kH2 + j];
    g[kOffB2 + j] = gb2;
    g[kOffW3 + j] = gw3;
    if (j == 0) g[kOffB3] = gb3;
    // loss: lanes 0 of each warp hold partial sums
    __shared__ float s_loss[4];
    if (lane == 0) s_loss[warp] = loss;
    __syncthreads();
    if (j == 0) loss_part[blockIdx.x] = (s_loss[0] + s_loss[1]) + (s_loss[2] + s_loss[3]);
}

// Master weights -> compute copy (round to nearest even BF16).
__device__ __forceinline__ void refresh_one(int p, float v, Weights *w) {
    if (p < kOffB1) {
        const int i = (p - kOffW1) / kIn, f = (p - kOffW1) % kIn;
        w->w1t[f * kH1 + i] = __float2bfloat16_rn(v);
    } else if (p < kOffW2) {
        w->b1[p - kOffB1] = v;
    } else if (p < kOffB2) {
        w->w2[p - kOffW2] = __float2bfloat16_rn(v);
    } else if (p < kOffW3) {
        w->b2[p - kOffB2] = v;
    } else if (p < kOffB3) {
        w->w3[p - kOffW3] = __float2bfloat16_rn(v);
    } else {
        w->b3 = v;
    }
}

__global__ void mlp_refresh_kernel(const float *master, Weights *w) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x)
        refresh_one(p, master[p], w);
}

// Sums the per-CTA partial gradients in CTA order (deterministic), applies
// one Adam step to the master weights and refreshes the compute copy.
// nparts == 0 only sums (gradient check): grad_out receives the gradient.
__global__ void mlp_adam_kernel(float *master, float *m1, float *m2, const float *grad_part, int nparts,
                                float lr, float beta1, float beta2, float eps, float bc1, float bc2, Weights *w,
                                float *grad_out, int apply) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (int b = 0; b < nparts; ++b) g += grad_part[(size_t)b * kParams + p];
        if (grad_out) grad_out[p] = g;
        if (!apply) continue;
        const float a = beta1 * m1[p] + (1.f - beta1) * g;
        const float v = beta2 * m2[p] + (1.f - beta2) * g * g;
        m1[p] = a;
        m2[p] = v;
        const float upd = (a / bc1) / (sqrtf(v / bc2) + eps);
        const float nw = master[p] - lr * upd;
        master[p] = nw;
        refresh_one(p, nw, w);
    }
}

// Sort keys for the longest-first order: 1 + predicted log2 cost in 1/8
// units (key 0 is kept for tasks that must go last, mlp_last_kernel).
__global__ void mlp_bin_kernel(const float *pred, long long n, uint16_t *key, uint32_t *idx) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float v = fminf(fmaxf(pred[t] * 8.f + 0.5f, 0.f), 65534.f);
        key[t] = (uint16_t)(1.f + v);
        idx[t] = (uint32_t)t;
    }
}

// Moves the listed tasks behind every other task of the order (key 0).
// Indices at or beyond n are ignored.
__global__ void mlp_last_kernel(const uint32_t *last, long long n_last, long long n, uint16_t *key) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_last;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t t = last[i];
        if ((long long)t < n) key[t] = 0;
    }
}

}  // namespace
}  // namespace nqb

using namespace nqb;

struct nq_mlp {
    std::mutex mu;
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    float *master = nullptr, *adam1 = nullptr, *adam2 = nullptr;
    Weights *w = nullptr;
    long long steps = 0;
    // scratch
    float *grad_part = nullptr;
    int grad_parts_cap = 0;
    float *gsum = nullptr;  // summed gradient (nq_mlp_grad)
    int *tc_err = nullptr;  // set by the tensor-core kernel when an MMA wait expires
    float *loss_part = nullptr;
    void *data = nullptr;
    size_t data_cap = 0;
    void *sort_tmp = nullptr;
    size_t sort_tmp_cap = 0;
};

namespace {

int mlp_fail(cudaError_t e, const char *what) {
    set_last_error((std::string(what) + ": " + cudaGetErrorString(e)).c_str());
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? NQ_ERR_OOM : NQ_ERR_CUDA;
}

#define MLP_CUDA(call)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return mlp_fail(e_, #call);      \
    } while (0)

int grow(void *&p, size_t &cap, size_t need) {
    if (need <= cap) return NQ_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = need + need / 4 + 256;
    MLP_CUDA(cudaMalloc(&p, want));
    cap = want;
    return NQ_OK;
}

int train_blocks(nq_mlp *m) { return m->sms; }

uint64_t splitmix(uint64_t &s) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uploads a task list (+ per-task N and targets) into the model's scratch:
// [cols | ld | rd | index] u32, [target] f32, [task_n] u8.
struct Staged {
    uint32_t *cols, *ld, *rd, *index;
    float *target;
    uint8_t *task_n;
};

int stage(nq_mlp *m, const uint8_t *task_n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
          const float *target, int64_t n, Staged &st) {
    const size_t need = (size_t)n * (4 * 4 + 4 + 1) + 1024;
    int rc = grow(m->data, m->data_cap, need);
    if (rc) return rc;
    char *b = (char *)m->data;
    st.cols = (uint32_t *)b;
    st.ld = st.cols + n;
    st.rd = st.ld + n;
    st.index = st.rd + n;
    st.target = (float *)(st.index + n);
    st.task_n = (uint8_t *)(st.target + n);
    MLP_CUDA(cudaMemcpyAsync(st.cols, cols, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(cudaMemcpyAsync(st.ld, ld, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(cudaMemcpyAsync(st.rd, rd, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    if (target) MLP_CUDA(cudaMemcpyAsync(st.target, target, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    if (task_n) MLP_CUDA(cudaMemcpyAsync(st.task_n, task_n, (size_t)n, cudaMemcpyHostToDevice, m->stream));
    return NQ_OK;
}

int ensure_grad_parts(nq_mlp *m, int parts) {
    if (parts <= m->grad_parts_cap) return NQ_OK;
    if (m->grad_part) cudaFree(m->grad_part);
    if (m->loss_part) cudaFree(m->loss_part);
    m->grad_part = nullptr;
    m->loss_part = nullptr;
    MLP_CUDA(cudaMalloc(&m->grad_part, (size_t)parts * kParams * sizeof(float)));
    MLP_CUDA(cudaMalloc(&m->loss_part, (size_t)parts * sizeof(float)));
    m->grad_parts_cap = parts;
    return NQ_OK;
}

// One forward+backward over [begin, end) into the partials; returns #parts.
int launch_train(nq_mlp *m, const TaskView &tv, const float *target, long long begin, long long end, float scale,
                 int &parts) {
    // Two groups of 32 tasks per CTA amortise the CTA's weight load and its
    // partial-gradient write; at most one CTA per SM (the kernel takes ~216 KiB).
    const long long groups = (end - begin + kGroup - 1) / kGroup;
    parts = (int)std::min<long long>(train_blocks(m), std::max<long long>((groups + 1) / 2, 1));
    int rc = ensure_grad_parts(m, parts);
    if (rc) return rc;
    mlp_train_kernel<<<parts, kH1, sizeof(TrainSmem), m->stream>>>(tv, target, begin, end, scale, m->w,
                                                                    m->grad_part, m->loss_part);
    MLP_CUDA(cudaGetLastError());
    return NQ_OK;
}

// Tensor-core forward over n device-resident tasks of board size N.
int launch_predict_tc(nq_mlp *m, const TaskView &tv, long long n, float *d_out, cudaStream_t s) {
    const long long tiles = (n + 127) / 128;
    const int grid = (int)std::min<long long>(tiles, (long long)m->sms * 2);
    mlp_predict_tc_kernel<<<grid, 128, tc::kSmemBytes, s>>>(tv, n, m->w, d_out, m->tc_err);
    MLP_CUDA(cudaGetLastError());
    return NQ_OK;
}

int check_model(nq_mlp *m) {
    if (!m) return NQ_ERR_ARG;
    MLP_CUDA(cudaSetDevice(m->device));
    return NQ_OK;
}

}  // namespace

extern "C" {

int nq_mlp_num_params(void) { return kParams; }

int nq_mlp_create(int device, uint64_t seed, nq_mlp **out) try {
    if (!out) return NQ_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        set_last_error("no CUDA device");
        return NQ_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return NQ_ERR_ARG;
    MLP_CUDA(cudaSetDevice(device));
    nq_mlp *m = new nq_mlp();
    m->device = device;
    cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&m->master, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->adam1, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->adam2, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->w, sizeof(Weights));
    if (e == cudaSuccess) e = cudaMalloc(&m->gsum, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->tc_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->tc_err, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp_predict_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(TrainSmem));
    if (e != cudaSuccess) {
        nq_mlp_destroy(m);
        return mlp_fail(e, "nq_mlp_create");
    }
    // Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) for every weight and bias,
    // from SplitMix64(seed).
    std::vector<float> p(kParams);
    uint64_t s = seed;
    auto uni = [&](float bound) {
        const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2.0 * u - 1.0) * bound);
    };
    for (int i = kOffW1; i < kOffB1; ++i) p[i] = uni(1.f / std::sqrt((float)kIn));
    for (int i = kOffB1; i < kOffW2; ++i) p[i] = uni(1.f / std::sqrt((float)kIn));
    for (int i = kOffW2; i < kOffB2; ++i) p[i] = uni(1.f / std::sqrt((float)kH1));
    for (int i = kOffB2; i < kOffW3; ++i) p[i] = uni(1.f / std::sqrt((float)kH1));
    for (int i = kOffW3; i < kOffB3; ++i) p[i] = uni(1.f / std::sqrt((float)kH2));
    p[kOffB3] = uni(1.f / std::sqrt((float)kH2));
    *out = m;
    return nq_mlp_set_params(m, p.data());
} catch (...) {
    return status_of_exception();
}

int nq_mlp_destroy(nq_mlp *m) try {
    if (!m) return NQ_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    cudaFree(m->master);
    cudaFree(m->adam1);
    cudaFree(m->adam2);
    cudaFree(m->w);
    cudaFree(m->gsum);
    cudaFree(m->tc_err);
    cudaFree(m->grad_part);
    cudaFree(m->loss_part);
    cudaFree(m->data);
    cudaFree(m->sort_tmp);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_get_params(nq_mlp *m, float *out) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (!out) return NQ_ERR_ARG;
    std::lock_guard<std::mutex> lock(m->mu);
    MLP_CUDA(cudaMemcpyAsync(out, m->master, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_set_params(nq_mlp *m, const float *in) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (!in) return NQ_ERR_ARG;
    std::lock_guard<std::mutex> lock(m->mu);
    MLP_CUDA(cudaMemcpyAsync(m->master, in, kParams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(cudaMemsetAsync(m->adam1, 0, kParams * sizeof(float), m->stream));
    MLP_CUDA(cudaMemsetAsync(m->adam2, 0, kParams * sizeof(float), m->stream));
    mlp_refresh_kernel<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->master, m->w);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    m->steps = 0;
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_predict(nq_mlp *m, int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                   float *out) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (N < 1 || N > NQ_MAX_N || n < 0 || (n > 0 && (!cols || !ld || !rd || !out))) return NQ_ERR_ARG;
    if (n == 0) return NQ_OK;
    std::lock_guard<std::mutex> lock(m->mu);
    Staged st;
    rc = stage(m, nullptr, cols, ld, rd, nullptr, n, st);
    if (rc) return rc;
    TaskView tv{st.cols, st.ld, st.rd, nullptr, nullptr, N};
    float *d_out = st.target;
    const int grid = (int)std::min<long long>((n + kGroup - 1) / kGroup, (long long)m->sms * 8);
    mlp_predict_kernel<<<grid, kH1, 0, m->stream>>>(tv, n, m->w, d_out);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpyAsync(out, d_out, (size_t)n * 4, cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_predict_tensor(nq_mlp *m, int N, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd, int64_t n,
                          float *out) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (N < 1 || N > NQ_MAX_N || n < 0 || (n > 0 && (!cols || !ld || !rd || !out))) return NQ_ERR_ARG;
    if (n == 0) return NQ_OK;
    std::lock_guard<std::mutex> lock(m->mu);
    Staged st;
    rc = stage(m, nullptr, cols, ld, rd, nullptr, n, st);
    if (rc) return rc;
    TaskView tv{st.cols, st.ld, st.rd, nullptr, nullptr, N};
    MLP_CUDA(cudaMemsetAsync(m->tc_err, 0, sizeof(int), m->stream));
    rc = launch_predict_tc(m, tv, n, st.target, m->stream);
    if (rc) return rc;
    int err = 0;
    MLP_CUDA(cudaMemcpyAsync(out, st.target, (size_t)n * 4, cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaMemcpyAsync(&err, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    if (err) {
        set_last_error("tensor-core MMA completion wait expired");
        return NQ_ERR_TIMEOUT;
    }
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_grad(nq_mlp *m, const uint8_t *task_n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                const float *target, int64_t n, float *grad_out, float *loss_out) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (n <= 0 || !task_n || !cols || !ld || !rd || !target || !grad_out) return NQ_ERR_ARG;
    std::lock_guard<std::mutex> lock(m->mu);
    Staged st;
    rc = stage(m, task_n, cols, ld, rd, target, n, st);
    if (rc) return rc;
    TaskView tv{st.cols, st.ld, st.rd, st.task_n, nullptr, 0};
    int parts = 0;
    rc = launch_train(m, tv, st.target, 0, n, 2.f / (float)n, parts);
    if (rc) return rc;
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->master, m->adam1, m->adam2, m->grad_part,
                                                                  parts, 0.f, 0.f, 0.f, 0.f, 1.f, 1.f, m->w, m->gsum, 0);
    cudaError_t e = cudaGetLastError();
    std::vector<float> lp(parts);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(grad_out, m->gsum, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(lp.data(), m->loss_part, parts * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return mlp_fail(e, "nq_mlp_grad");
    if (loss_out) {
        double l = 0;
        for (float v : lp) l += v;
        *loss_out = (float)(l / (double)n);
    }
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_mlp_train(nq_mlp *m, const uint8_t *task_n, const uint32_t *cols, const uint32_t *ld, const uint32_t *rd,
                 const float *target, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                 float *epoch_loss) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (n <= 0 || !task_n || !cols || !ld || !rd || !target || epochs < 0 || batch < kGroup || lr <= 0.f)
        return NQ_ERR_ARG;
    if (n > 0xffffffffll) return NQ_ERR_ARG;
    std::lock_guard<std::mutex> lock(m->mu);
    Staged st;
    rc = stage(m, task_n, cols, ld, rd, target, n, st);
    if (rc) return rc;
    std::vector<uint32_t> perm((size_t)n);
    uint64_t s = seed;
    const int parts_max = train_blocks(m);
    rc = ensure_grad_parts(m, parts_max);
    if (rc) return rc;
    const long long nsteps_epoch = (n + batch - 1) / batch;
    std::vector<float> lp((size_t)parts_max * nsteps_epoch);
    for (int ep = 0; ep < epochs; ++ep) {
        // Fisher-Yates shuffle from SplitMix64(seed), one per epoch.
        for (int64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        for (int64_t i = n - 1; i > 0; --i) {
            const int64_t k = (int64_t)(splitmix(s) % (uint64_t)(i + 1));
            std::swap(perm[i], perm[k]);
        }
        MLP_CUDA(cudaMemcpyAsync(st.index, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
        TaskView tv{st.cols, st.ld, st.rd, st.task_n, st.index, 0};
        double eloss = 0;
        for (long long b0 = 0, stepi = 0; b0 < n; b0 += batch, ++stepi) {
            const long long b1 = std::min<long long>(n, b0 + batch);
            int parts = 0;
            rc = launch_train(m, tv, st.target, b0, b1, 2.f / (float)(b1 - b0), parts);
            if (rc) return rc;
            m->steps += 1;
            const float bc1 = 1.f - std::pow(0.9f, (float)m->steps);
            const float bc2 = 1.f - std::pow(0.999f, (float)m->steps);
            mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->master, m->adam1, m->adam2,
                                                                          m->grad_part, parts, lr, 0.9f, 0.999f,
                                                                          1e-8f, bc1, bc2, m->w, nullptr, 1);
            MLP_CUDA(cudaGetLastError());
            if (epoch_loss)
                MLP_CUDA(cudaMemcpyAsync(lp.data() + (size_t)stepi * parts_max, m->loss_part, parts * sizeof(float),
                                         cudaMemcpyDeviceToHost, m->stream));
            if (epoch_loss && parts < parts_max)
                for (int q = parts; q < parts_max; ++q) lp[(size_t)stepi * parts_max + q] = 0.f;
        }
        if (epoch_loss) {
            MLP_CUDA(cudaStreamSynchronize(m->stream));
            for (float v : lp) eloss += v;
            epoch_loss[ep] = (float)(eloss / (double)n);
        }
    }
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

// Longest-first order of device-resident tasks: predictions -> keys in
// 1/8-log2 bins -> stable descending radix sort of task indices.
int nq_schedule_device_last(nq_mlp *m, int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd,
                            int64_t n, const uint32_t *d_last, int64_t n_last, uint32_t *d_order, float *d_pred,
                            void *stream) try {
    int rc = check_model(m);
    if (rc) return rc;
    if (N < 1 || N > NQ_MAX_N || n < 0 || n > 0xffffffffll || (n > 0 && (!d_cols || !d_ld || !d_rd || !d_order)))
        return NQ_ERR_ARG;
    if (n_last < 0 || (n_last > 0 && !d_last)) return NQ_ERR_ARG;
    if (n == 0) return NQ_OK;
    std::lock_guard<std::mutex> lock(m->mu);
    cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream, as in every device entry
    // scratch: pred f32 | key u16 | key_out u16 | idx u32
    const size_t need = (size_t)n * (4 + 2 + 2 + 4) + 1024;
    rc = grow(m->data, m->data_cap, need);
    if (rc) return rc;
    float *pred = d_pred ? d_pred : (float *)m->data;
    uint16_t *key = (uint16_t *)((char *)m->data + (size_t)n * 4);
    uint16_t *key2 = key + n;
    uint32_t *idx = (uint32_t *)(((uintptr_t)(key2 + n) + 15) & ~(uintptr_t)15);
    TaskView tv{d_cols, d_ld, d_rd, nullptr, nullptr, N};
    rc = launch_predict_tc(m, tv, n, pred, s);
    if (rc) return rc;
    mlp_bin_kernel<<<m->sms * 4, 256, 0, s>>>(pred, n, key, idx);
    MLP_CUDA(cudaGetLastError());
    if (n_last > 0) {
        mlp_last_kernel<<<m->sms * 4, 256, 0, s>>>(d_last, n_last, n, key);
        MLP_CUDA(cudaGetLastError());
    }
    size_t tmp = 0;
    MLP_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, key, key2, idx, d_order, (int)n, 0, 16, s));
    rc = grow(m->sort_tmp, m->sort_tmp_cap, tmp);
    if (rc) return rc;
    MLP_CUDA(cub::DeviceRadixSort::SortPairsDescending(m->sort_tmp, tmp, key, key2, idx, d_order, (int)n, 0, 16, s));
    return NQ_OK;
} catch (...) {
    return status_of_exception();
}

int nq_schedule_device(nq_mlp *m, int N, const uint32_t *d_cols, const uint32_t *d_ld, const uint32_t *d_rd,
                       int64_t n, uint32_t *d_order, float *d_pred, void *stream) try {
    return nq_schedule_device_last(m, N, d_cols, d_ld, d_rd, n, nullptr, 0, d_order, d_pred, stream);
} catch (...) {
    return status_of_exception();
}

}  // extern "C"
