// expand_dev.cu -- prefix expansion on the device.
//
// Produces exactly the task list of the host expander (expand.cpp), i.e. the
// reference's partial_n_queens + partial_n_queens_for_odd output
// (src/n_queens.cpp:74-113) in the reference's order, without building it on
// the host or copying it over PCIe:
//
//   1. the host enumerates the seeds -- placements of the first s rows
//      (s = min(rows, 4)), the only rows with the half-board / middle-column
//      rules -- in order (a few thousand; tens of kilobytes to upload);
//   2. count pass: one thread per seed walks its subtree down to `rows` rows
//      and counts the prefixes;
//   3. an exclusive scan turns the counts into output offsets;
//   4. write pass: the same walk writes every prefix at its offset.
// Below row 1 every row admits all N columns, so a seed's subtree needs no
// rule but the masks.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/device/device_scan.cuh>
#include <vector>

#include "expand.h"

namespace nqb {

namespace {

constexpr int kSeedRows = 4;

// Depth-first walk of one seed's subtree from row r0 to `rows`, lowest free
// column first; emit(k, c, l, r) for the k-th prefix of the seed.
template <bool WRITE>
__device__ __forceinline__ long long walk(uint32_t c0, uint32_t l0, uint32_t r0, int depth, uint32_t full,
                                          long long base, long long cap, uint32_t *cols, uint32_t *ld,
                                          uint32_t *rd) {
    if (depth == 0) {
        if (WRITE && base < cap) {
            cols[base] = c0;
            ld[base] = l0;
            rd[base] = r0;
        }
        return 1;
    }
    uint32_t sc[32], sl[32], sr[32], sa[32];
    int d = 0;
    sc[0] = c0;
    sl[0] = l0;
    sr[0] = r0;
    sa[0] = full & ~(c0 | l0 | r0);
    long long k = 0;
    while (d >= 0) {
        const uint32_t a = sa[d];
        if (a == 0) {
            --d;
            continue;
        }
        const uint32_t p = a & (0u - a);
        sa[d] = a ^ p;
        const uint32_t c = sc[d] | p;
        const uint32_t l = (sl[d] | p) << 1;
        const uint32_t r = (uint32_t)((int32_t)(sr[d] | p) >> 1);
        if (d + 1 == depth) {
            if (WRITE && base + k < cap) {
                cols[base + k] = c;
                ld[base + k] = l;
                rd[base + k] = r;
            }
            ++k;
        } else {
            ++d;
            sc[d] = c;
            sl[d] = l;
            sr[d] = r;
            sa[d] = full & ~(c | l | r);
        }
    }
    return k;
}

__global__ void expand_count_kernel(const uint4 *seeds, int nseeds, int depth, uint32_t full,
                                    unsigned long long *counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseeds) return;
    const uint4 s = seeds[i];
    counts[i] = (unsigned long long)walk<false>(s.x, s.y, s.z, depth, full, 0, 0, nullptr, nullptr, nullptr);
}

__global__ void expand_write_kernel(const uint4 *seeds, int nseeds, int depth, uint32_t full,
                                    const unsigned long long *offsets, long long cap, uint32_t *cols, uint32_t *ld,
                                    uint32_t *rd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseeds) return;
    const uint4 s = seeds[i];
    walk<true>(s.x, s.y, s.z, depth, full, (long long)offsets[i], cap, cols, ld, rd);
}

}  // namespace

// Device expansion into caller-provided device arrays (at most cap tasks);
// `scratch` is grown as needed (seeds, counts, offsets, scan temp).  Returns
// the task count through *n_tasks; synchronises `stream` once (to learn it).
cudaError_t expand_prefixes_device(int N, int rows, uint32_t *d_cols, uint32_t *d_ld, uint32_t *d_rd, int64_t cap,
                                   int64_t *n_tasks, void **scratch, size_t *scratch_cap, cudaStream_t stream) {
    const int s = rows < kSeedRows ? rows : kSeedRows;
    std::vector<uint32_t> sc, sl, sr;
    const int64_t ns = expand_prefixes_to(
        N, s,
        [&](int64_t total, uint32_t **c, uint32_t **l, uint32_t **r, int64_t *k) {
            sc.resize((size_t)total);
            sl.resize((size_t)total);
            sr.resize((size_t)total);
            *c = sc.data();
            *l = sl.data();
            *r = sr.data();
            *k = total;
            return true;
        },
        1);
    if (ns < 0) return cudaErrorInvalidValue;
    if (ns == 0) {
        *n_tasks = 0;
        return cudaSuccess;
    }
    std::vector<uint4> seeds((size_t)ns);
    for (int64_t i = 0; i < ns; ++i) seeds[i] = make_uint4(sc[i], sl[i], sr[i], 0);
    size_t scan_tmp = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (unsigned long long *)nullptr,
                                                  (unsigned long long *)nullptr, (int)ns, stream);
    if (e != cudaSuccess) return e;
    const size_t need = (size_t)ns * 16 + 2 * (size_t)ns * 8 + scan_tmp + 1024;
    if (need > *scratch_cap) {
        if (*scratch) cudaFree(*scratch);
        *scratch = nullptr;
        *scratch_cap = 0;
        e = cudaMalloc(scratch, need + need / 4);
        if (e != cudaSuccess) return e;
        *scratch_cap = need + need / 4;
    }
    char *b = (char *)*scratch;
    uint4 *d_seeds = (uint4 *)b;
    unsigned long long *d_counts = (unsigned long long *)(b + (size_t)ns * 16);
    unsigned long long *d_offsets = d_counts + ns;
    void *d_tmp = (void *)(((uintptr_t)(d_offsets + ns) + 255) & ~(uintptr_t)255);
    e = cudaMemcpyAsync(d_seeds, seeds.data(), (size_t)ns * 16, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    const uint32_t full = (1u << N) - 1u;
    const int depth = rows - s;
    const int threads = 128, blocks = (int)((ns + threads - 1) / threads);
    expand_count_kernel<<<blocks, threads, 0, stream>>>(d_seeds, (int)ns, depth, full, d_counts);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(d_tmp, scan_tmp, d_counts, d_offsets, (int)ns, stream);
    if (e != cudaSuccess) return e;
    unsigned long long last[2];
    e = cudaMemcpyAsync(&last[0], d_offsets + ns - 1, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last[1], d_counts + ns - 1, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    *n_tasks = (int64_t)(last[0] + last[1]);
    if (cap > 0 && d_cols && d_ld && d_rd) {
        expand_write_kernel<<<blocks, threads, 0, stream>>>(d_seeds, (int)ns, depth, full, d_offsets, cap, d_cols,
                                                            d_ld, d_rd);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace nqb
