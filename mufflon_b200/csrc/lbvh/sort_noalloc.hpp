// Allocation-free pair sort (see sort_noalloc.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mb {

constexpr uint32_t NOALLOC_MAX_PAIRS = 1u << 20;

// Sorts n <= NOALLOC_MAX_PAIRS device-resident pairs in place on `stream`
// and returns after they are sorted. Allocates nothing.
cudaError_t sort_pairs_noalloc(uint64_t* keys, int32_t* values, uint32_t n, cudaStream_t stream, bool* waitExpired);

// The per-device set-up of sort_pairs_noalloc (the scratch array's address and
// the sort kernels loaded), done now for the current device; idempotent.
cudaError_t noalloc_prepare_current_device();

// Size of the library-resident scratch array in bytes.
size_t noalloc_scratch_bytes();

} // namespace mb
