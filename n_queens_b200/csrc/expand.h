// expand.h -- host prefix expansion (see expand.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <vector>

namespace nqb {

// Reference-ordered half-board prefixes of `rows` rows as SoA triples.
// Returns the task count (or -1 on bad arguments); writes at most cap tasks.
int64_t expand_prefixes(int N, int rows, uint32_t *cols, uint32_t *ld, uint32_t *rd, int64_t cap, int threads);

// Same, but the output buffers are asked for once the task count is known:
// sink(total, &cols, &ld, &rd, &cap) returns false to abort (-2 is returned).
typedef std::function<bool(int64_t, uint32_t **, uint32_t **, uint32_t **, int64_t *)> PrefixSink;
int64_t expand_prefixes_to(int N, int rows, const PrefixSink &sink, int threads);

// Splits one partial board `rows` rows deeper (no symmetry), appending the
// subtasks; returns how many were appended.
int64_t expand_board(int N, uint32_t c0, uint32_t l0, uint32_t r0, int rows, std::vector<uint32_t> &cols,
                     std::vector<uint32_t> &ld, std::vector<uint32_t> &rd);

// Device expansion into caller device arrays (expand_dev.cu); `scratch` is a
// device buffer the function grows as needed.  Same output and order as
// expand_prefixes.
cudaError_t expand_prefixes_device(int N, int rows, uint32_t *d_cols, uint32_t *d_ld, uint32_t *d_rd, int64_t cap,
                                   int64_t *n_tasks, void **scratch, size_t *scratch_cap, cudaStream_t stream);

}  // namespace nqb
