// Stable (uint64 key, int32 value) radix sort that allocates no device memory.
//
// Some callers cannot call cudaMalloc: an engine that reserves all device
// memory for its own allocator up front has nothing left to hand out, and a
// frame loop that must not stall cannot afford cudaMalloc/cudaFree, which may
// synchronise the device. For them this variant of the LBVH builder's sort
// keeps its scratch (the ping-pong key/value buffers, the digit histograms,
// the look-back tile status and the tile counters) in one file-scope device
// array of a fixed size, so a call only launches kernels and clears memory.
//
// Limits and sharing:
//   * at most NOALLOC_MAX_PAIRS pairs per call; larger sizes are rejected;
//   * the array (about 12.5 MiB) is part of the library's device image: every
//     GPU on which the library is loaded holds it until the process exits;
//   * all calls share the array and it keeps the previous call's contents, so
//     every region that must start at zero is cleared at the start of a call,
//     and calls that overlap on the GPU (different streams, or threads) race;
//   * host code cannot use the array's name as a device address; the address
//     is looked up with cudaGetSymbolAddress once per device, with that device
//     current. mufflon_initialize does this for the device it selects (through
//     noalloc_prepare_current_device); on any other device the first call does
//     it. The look-up, and loading the sort's kernels with it, loads this
//     file's device code onto the device, which takes device memory under
//     CUDA's lazy module loading: so the set-up must come before the caller
//     reserves its device memory, and before any stream capture.
#include "radix_sort.cuh"
#include "sort_noalloc.hpp"

#include <mutex>

namespace mb {
namespace {

constexpr size_t NA_KEYS = 0;
constexpr size_t NA_VALS = NA_KEYS + size_t(NOALLOC_MAX_PAIRS) * sizeof(u64);
constexpr size_t NA_TILES = (size_t(NOALLOC_MAX_PAIRS) + SORT_TILE - 1) / SORT_TILE;
constexpr size_t NA_STATUS = NA_VALS + size_t(NOALLOC_MAX_PAIRS) * sizeof(int32_t);
constexpr size_t NA_HIST = NA_STATUS + NA_TILES * 256 * sizeof(uint32_t);
constexpr size_t NA_COUNTERS = NA_HIST + 8 * 256 * sizeof(uint32_t);
constexpr size_t NA_ERROR = NA_COUNTERS + 8 * sizeof(unsigned int);
constexpr size_t NA_BYTES = (NA_ERROR + sizeof(unsigned int) + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_sortScratch[NA_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setupMutex;
unsigned char* g_scratchAddress[MAX_DEVICES] = {};

// Once per device, with that device current.
cudaError_t scratch_for_current_device(unsigned char** base) {
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if(e != cudaSuccess) return e;
	if(dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
	std::lock_guard<std::mutex> lock(g_setupMutex);
	if(!g_scratchAddress[dev]) {
		void* p = nullptr;
		if((e = cudaGetSymbolAddress(&p, g_sortScratch)) != cudaSuccess) return e;
		if((e = cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SORT_SMEM))) != cudaSuccess)
			return e;
		// Load the other two kernels now as well: under lazy loading their
		// first launch would otherwise load their code into device memory.
		cudaFuncAttributes attr;
		if((e = cudaFuncGetAttributes(&attr, k_sort_hist)) != cudaSuccess) return e;
		if((e = cudaFuncGetAttributes(&attr, k_sort_scan)) != cudaSuccess) return e;
		g_scratchAddress[dev] = static_cast<unsigned char*>(p);
	}
	*base = g_scratchAddress[dev];
	return cudaSuccess;
}

} // namespace

size_t noalloc_scratch_bytes() { return NA_BYTES; }

cudaError_t noalloc_prepare_current_device() {
	unsigned char* base = nullptr;
	return scratch_for_current_device(&base);
}

cudaError_t sort_pairs_noalloc(uint64_t* keys, int32_t* values, uint32_t n, cudaStream_t stream, bool* waitExpired) {
	if(waitExpired) *waitExpired = false;
	if(n > NOALLOC_MAX_PAIRS) return cudaErrorInvalidValue;
	if(n <= 1) return cudaSuccess;
	unsigned char* base = nullptr;
	cudaError_t e = scratch_for_current_device(&base);
	if(e != cudaSuccess) return e;
	u64* spareKeys = reinterpret_cast<u64*>(base + NA_KEYS);
	int32_t* spareVals = reinterpret_cast<int32_t*>(base + NA_VALS);
	uint32_t* status = reinterpret_cast<uint32_t*>(base + NA_STATUS);
	uint32_t* hist = reinterpret_cast<uint32_t*>(base + NA_HIST);
	unsigned int* counters = reinterpret_cast<unsigned int*>(base + NA_COUNTERS);
	unsigned int* error = reinterpret_cast<unsigned int*>(base + NA_ERROR);
	const uint32_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
	// the previous call's histogram, counters and error word are still there
	if((e = cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
	if((e = cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned int), stream)) != cudaSuccess) return e;
	if((e = cudaMemsetAsync(error, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
	const unsigned hb = std::min<unsigned>((n + 255) / 256, 148u * 8u);
	k_sort_hist<<<hb, 256, 0, stream>>>(keys, n, hist);
	k_sort_scan<<<8, 256, 0, stream>>>(hist);
	u64* kin = keys; u64* kout = spareKeys;
	int32_t* vin = values; int32_t* vout = spareVals;
	for(int pass = 0; pass < 8; ++pass) {
		if((e = cudaMemsetAsync(status, 0, size_t(tiles) * 256 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
		k_onesweep<<<tiles, SORT_THREADS, SORT_SMEM, stream>>>(kin, vin, kout, vout, n, 8 * pass, hist + 256 * pass,
		                                                      status, counters + pass, error);
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	if((e = cudaGetLastError()) != cudaSuccess) return e;
	// 8 passes: the sorted pairs are back in (keys, values)
	unsigned int err = 0;
	if((e = cudaMemcpyAsync(&err, error, sizeof(err), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
	if((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
	if(err && waitExpired) *waitExpired = true;
	return err ? cudaErrorLaunchTimeout : cudaSuccess;
}

} // namespace mb
