// Onesweep LSD radix sort of (uint64 key, int32 value) pairs: the kernels
// shared by the LBVH builder (lbvh.cu) and the allocation-free sort entry
// point (sort_noalloc.cu). Each including translation unit gets its own copy
// in an anonymous namespace.
//
// One pass sorts by 8 key bits: a tile of SORT_TILE keys is ranked with
// __match_any_sync inside each warp, per-warp digit histograms in shared
// memory give block-local ranks, and the tile's global digit offsets come from
// decoupled look-back over the preceding tiles' published counts. Every wait in
// the look-back is bounded; an expired wait sets *error instead of spinning.
// Passes are stable, so 8 passes sort 64-bit keys.
#pragma once

#include "../trace/dmath.cuh"

namespace mb {
namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr size_t SORT_SMEM = size_t(SORT_TILE) * 8 + size_t(SORT_TILE) * 4 + size_t(SORT_WARPS) * 256 * 4;
constexpr unsigned SPIN_LIMIT = 1u << 22;

// ---------------------------------------------------------------- radix sort
__global__ void k_sort_hist(const u64* keys, uint32_t n, uint32_t* hist) {
	__shared__ uint32_t h[8 * 256];
	for(int i = threadIdx.x; i < 8 * 256; i += blockDim.x) h[i] = 0;
	__syncthreads();
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const u64 k = keys[i];
#pragma unroll
		for(int p = 0; p < 8; ++p) atomicAdd(&h[p * 256 + ((k >> (8 * p)) & 255u)], 1u);
	}
	__syncthreads();
	for(int i = threadIdx.x; i < 8 * 256; i += blockDim.x)
		if(h[i]) atomicAdd(&hist[i], h[i]);
}

// Exclusive scan of each pass's 256-bin histogram (one block per pass).
__global__ void k_sort_scan(uint32_t* hist) {
	__shared__ uint32_t s[256];
	const int t = threadIdx.x;
	uint32_t* h = hist + blockIdx.x * 256;
	const uint32_t own = h[t];
	s[t] = own;
	__syncthreads();
	for(int off = 1; off < 256; off <<= 1) {
		const uint32_t v = t >= off ? s[t - off] : 0u;
		__syncthreads();
		s[t] += v;
		__syncthreads();
	}
	h[t] = s[t] - own;
}

MBD unsigned lanemask_lt() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

// One onesweep pass over 8 key bits starting at `shift`.
__global__ void __launch_bounds__(SORT_THREADS)
k_onesweep(const u64* __restrict__ keysIn, const int32_t* __restrict__ valsIn, u64* __restrict__ keysOut,
           int32_t* __restrict__ valsOut, uint32_t n, int shift, const uint32_t* __restrict__ digitStart,
           uint32_t* status, unsigned int* tileCounter, unsigned int* error) {
	extern __shared__ __align__(16) unsigned char smem[];
	u64* sKeys = reinterpret_cast<u64*>(smem);
	int32_t* sVals = reinterpret_cast<int32_t*>(sKeys + SORT_TILE);
	uint32_t* sWarpHist = reinterpret_cast<uint32_t*>(sVals + SORT_TILE);
	__shared__ uint32_t sBlockStart[256];
	__shared__ uint32_t sGlobal[256];
	__shared__ uint32_t sTile;

	const int tid = threadIdx.x;
	const unsigned lane = tid & 31u;
	const int warp = tid >> 5;
	if(tid == 0) sTile = atomicAdd(tileCounter, 1u);
	for(int i = tid; i < SORT_WARPS * 256; i += SORT_THREADS) sWarpHist[i] = 0;
	__syncthreads();
	const uint32_t tile = sTile;
	const uint32_t base = tile * SORT_TILE + uint32_t(warp) * (32 * SORT_ITEMS);

	u64 k[SORT_ITEMS];
	int32_t v[SORT_ITEMS];
	uint32_t rank[SORT_ITEMS];
#pragma unroll
	for(int i = 0; i < SORT_ITEMS; ++i) {
		const uint32_t idx = base + uint32_t(i) * 32 + lane;
		if(idx < n) { k[i] = keysIn[idx]; v[i] = valsIn[idx]; }
		else { k[i] = ~0ull; v[i] = 0; }
	}
	const unsigned lt = lanemask_lt();
#pragma unroll
	for(int i = 0; i < SORT_ITEMS; ++i) {
		const bool valid = base + uint32_t(i) * 32 + lane < n;
		const uint32_t d = uint32_t(k[i] >> shift) & 255u;
		const unsigned vm = __ballot_sync(0xffffffffu, valid);
		rank[i] = 0;
		if(valid) {
			const unsigned peers = __match_any_sync(vm, d);
			const int leader = __ffs(peers) - 1;
			uint32_t prev = 0;
			if(int(lane) == leader) {
				prev = sWarpHist[warp * 256 + d];
				sWarpHist[warp * 256 + d] = prev + __popc(peers);
			}
			prev = __shfl_sync(peers, prev, leader);
			rank[i] = prev + __popc(peers & lt);
		}
		__syncwarp();
	}
	__syncthreads();
	// per digit: exclusive prefix over warps, block total
	const uint32_t d = uint32_t(tid);
	uint32_t total = 0;
#pragma unroll
	for(int w = 0; w < SORT_WARPS; ++w) {
		const uint32_t c = sWarpHist[w * 256 + d];
		sWarpHist[w * 256 + d] = total;
		total += c;
	}
	sBlockStart[d] = total;
	__syncthreads();
	for(int off = 1; off < 256; off <<= 1) {
		const uint32_t x = d >= uint32_t(off) ? sBlockStart[d - off] : 0u;
		__syncthreads();
		sBlockStart[d] += x;
		__syncthreads();
	}
	const uint32_t blockStart = sBlockStart[d] - total;
	__syncthreads();
	sBlockStart[d] = blockStart;
	// decoupled look-back across tiles; status = (flag << 30) | count,
	// flag 1 = tile aggregate, 2 = inclusive prefix
	uint32_t excl = 0;
	if(tile == 0) {
		atomicExch(&status[d], (2u << 30) | total);
	} else {
		atomicExch(&status[tile * 256 + d], (1u << 30) | total);
		int j = int(tile) - 1;
		unsigned spins = 0;
		while(j >= 0) {
			const uint32_t s = *reinterpret_cast<volatile uint32_t*>(&status[uint32_t(j) * 256 + d]);
			const uint32_t flag = s >> 30;
			if(flag == 0) {
				if(++spins > SPIN_LIMIT) { atomicOr(error, 1u); break; }
				__nanosleep(32);
				continue;
			}
			excl += s & 0x3FFFFFFFu;
			if(flag == 2) break;
			--j;
		}
		atomicExch(&status[tile * 256 + d], (2u << 30) | (excl + total));
	}
	sGlobal[d] = digitStart[d] + excl;
	__syncthreads();
#pragma unroll
	for(int i = 0; i < SORT_ITEMS; ++i) {
		if(base + uint32_t(i) * 32 + lane < n) {
			const uint32_t dd = uint32_t(k[i] >> shift) & 255u;
			const uint32_t pos = sBlockStart[dd] + sWarpHist[warp * 256 + dd] + rank[i];
			sKeys[pos] = k[i];
			sVals[pos] = v[i];
		}
	}
	__syncthreads();
	const uint32_t tileBase = tile * SORT_TILE;
	const uint32_t count = n - tileBase < uint32_t(SORT_TILE) ? n - tileBase : uint32_t(SORT_TILE);
	for(uint32_t j = tid; j < count; j += SORT_THREADS) {
		const u64 key = sKeys[j];
		const uint32_t dd = uint32_t(key >> shift) & 255u;
		const uint32_t dest = sGlobal[dd] + (j - sBlockStart[dd]);
		keysOut[dest] = key;
		valsOut[dest] = sVals[j];
	}
}


} // namespace
} // namespace mb
