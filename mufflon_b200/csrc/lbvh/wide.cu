// GPU conversion of a binary Karras hierarchy into the compressed 8-wide
// format of wide.hpp, one kernel launch per level of the wide tree.
//
// Each thread turns one queued binary node into one wide node:
//   1. gather up to eight children by repeatedly opening the gathered binary
//      internal node with the largest surface area,
//   2. children with more than leafMax primitives become wide internal nodes
//      (queued for the next level), the others become leaves,
//   3. children are assigned to slots by direction octant: slot s prefers the
//      child whose centroid offset points along (s&4 ? -x : +x, s&2 ? -y : +y,
//      s&1 ? -z : +z); a greedy maximum of centroid-offset . octant vector,
//   4. boxes are quantised conservatively (see wide.hpp) and the node is
//      written; leaf primitives are copied into the node's primitive block.
#include "wide.hpp"
#include "../trace/dmath.cuh"

namespace mb {
namespace {

enum { CNT_NODES = 0, CNT_PRIMS = 1, CNT_QUEUE = 2 /* 3 rotating counts */, CNT_ERROR = 5 };
constexpr int MAX_WIDE_LEVELS = 512;
constexpr float INV_252 = 1.0f / 252.0f;

__global__ void k_wide_init(uint32_t* counters, int2* queueA) {
	counters[CNT_NODES] = 1;
	counters[CNT_PRIMS] = 0;
	counters[CNT_QUEUE + 0] = 1;
	counters[CNT_QUEUE + 1] = 0;
	counters[CNT_QUEUE + 2] = 0;
	counters[CNT_ERROR] = 0;
	queueA[0] = make_int2(0, 0);
}

MBD void bin_box(const float4* nd, int b, f3& mn, f3& mx) {
	const float4 a = nd[2 * size_t(b)], c = nd[2 * size_t(b) + 1];
	mn = make3(a.x, a.y, a.z);
	mx = make3(c.x, c.y, c.z);
}
MBD float half_area(f3 mn, f3 mx) {
	const f3 d = mx - mn;
	return d.x * d.y + d.y * d.z + d.z * d.x;
}
MBD float comp(f3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
MBD float pow2f(int e) { return __int_as_float((e + 127) << 23); }

__global__ void __launch_bounds__(128) k_wide_level(WideBuildArgs A, const int2* __restrict__ qin,
                                                    const uint32_t* inCount, int2* qout, uint32_t* outCount,
                                                    uint32_t* zeroCount) {
	if(blockIdx.x == 0 && threadIdx.x == 0) *zeroCount = 0;
	const uint32_t count = *inCount;
	const int nI = A.numInternal;
	const uint32_t lane = threadIdx.x & 31u;
	// Warp-uniform loop: the node, primitive and queue allocations of a warp's
	// nodes are one atomic each per warp (per-node atomics on these three
	// counters serialised in L2 at the wide levels).
	for(uint32_t first0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; first0 < count; first0 += gridDim.x * blockDim.x) {
		const uint32_t item = first0 + lane;
		const bool valid = item < count;
		const int2 e = valid ? qin[item] : make_int2(0, 0);
		const int b = e.x;
		const uint32_t w = uint32_t(e.y);
		// 1. gather
		int ch[8];
		float area[8];
		f3 cmn[8], cmx[8];
		int nc = 2;
		ch[0] = A.children[2 * b];
		ch[1] = A.children[2 * b + 1];
		for(int i = 0; i < 2; ++i) {
			bin_box(A.nodeData, ch[i], cmn[i], cmx[i]);
			area[i] = ch[i] < nI ? half_area(cmn[i], cmx[i]) : -1.0f;
		}
		while(nc < 8) {
			int best = -1;
			float ba = -1.0f;
			for(int i = 0; i < nc; ++i)
				if(area[i] > ba) { ba = area[i]; best = i; }
			if(best < 0) break;
			const int c = ch[best];
			ch[best] = A.children[2 * c];
			ch[nc] = A.children[2 * c + 1];
			bin_box(A.nodeData, ch[best], cmn[best], cmx[best]);
			bin_box(A.nodeData, ch[nc], cmn[nc], cmx[nc]);
			area[best] = ch[best] < nI ? half_area(cmn[best], cmx[best]) : -1.0f;
			area[nc] = ch[nc] < nI ? half_area(cmn[nc], cmx[nc]) : -1.0f;
			++nc;
		}
		// 2. classify
		int first[8], cnt[8];
		bool inner[8];
		int nInner = 0, nPrims = 0;
		for(int i = 0; i < nc; ++i) {
			if(ch[i] >= nI) { first[i] = ch[i] - nI; cnt[i] = 1; }
			else { const int2 r = A.ranges[ch[i]]; first[i] = r.x; cnt[i] = r.y - r.x + 1; }
			inner[i] = cnt[i] > A.leafMax;
			if(inner[i]) ++nInner; else nPrims += cnt[i];
		}
		if(!valid) { nInner = 0; nPrims = 0; }
		uint32_t incN = uint32_t(nInner), incP = uint32_t(nPrims);
		for(int off = 1; off < 32; off <<= 1) {
			const uint32_t tn = __shfl_up_sync(0xffffffffu, incN, off), tp = __shfl_up_sync(0xffffffffu, incP, off);
			if(lane >= uint32_t(off)) { incN += tn; incP += tp; }
		}
		const uint32_t totN = __shfl_sync(0xffffffffu, incN, 31), totP = __shfl_sync(0xffffffffu, incP, 31);
		uint32_t bn = 0, bp = 0, bq = 0;
		if(lane == 0) {
			if(totN) { bn = atomicAdd(A.counters + CNT_NODES, totN); bq = atomicAdd(outCount, totN); }
			if(totP) bp = atomicAdd(A.counters + CNT_PRIMS, totP);
		}
		bn = __shfl_sync(0xffffffffu, bn, 0);
		bp = __shfl_sync(0xffffffffu, bp, 0);
		bq = __shfl_sync(0xffffffffu, bq, 0);
		if(!valid) continue;
		const uint32_t childBase = bn + incN - uint32_t(nInner);
		const uint32_t primBase = bp + incP - uint32_t(nPrims);
		const uint32_t queueBase = bq + incN - uint32_t(nInner);
		if(childBase + nInner > A.nodeCapacity || primBase + nPrims > uint32_t(A.n) || w >= A.nodeCapacity) {
			atomicOr(A.counters + CNT_ERROR, 1u);
			continue;
		}
		// 3. octant slots
		f3 pmn, pmx;
		bin_box(A.nodeData, b, pmn, pmx);
		const f3 pc = (pmn + pmx) * 0.5f;
		int slotChild[8];
		for(int s = 0; s < 8; ++s) slotChild[s] = -1;
		unsigned assigned = 0;
		for(int round = 0; round < nc; ++round) {
			float bestScore = -INFINITY;
			int bi = -1, bs = -1;
			for(int i = 0; i < nc; ++i) {
				if(assigned & (1u << i)) continue;
				const f3 off = (cmn[i] + cmx[i]) * 0.5f - pc;
				for(int s = 0; s < 8; ++s) {
					if(slotChild[s] >= 0) continue;
					const float sc = ((s & 4) ? -off.x : off.x) + ((s & 2) ? -off.y : off.y) + ((s & 1) ? -off.z : off.z);
					if(sc > bestScore || bi < 0) { bestScore = sc; bi = i; bs = s; }
				}
			}
			assigned |= 1u << bi;
			slotChild[bs] = bi;
		}
		// 4. quantisation grid per axis
		WideNode N;
		float pgrid[3], inv[3];
		uint32_t ebytes = 0;
		for(int a = 0; a < 3; ++a) {
			const float lo = comp(pmn, a), hi = comp(pmx, a);
			const float ext = __fsub_ru(hi, lo);
			const float amax = fmaxf(fabsf(lo), fabsf(hi));
			float need = fmaxf(__fmul_ru(ext, INV_252), amax * (1.0f / 1048576.0f));
			int ex = -100;
			if(need > 0.0f) { frexpf(need, &ex); }
			ex = max(-100, min(100, ex));
			const float scale = pow2f(ex);
			pgrid[a] = __fsub_rd(lo, scale);
			inv[a] = pow2f(-ex);
			N.p[a] = pgrid[a];
			ebytes |= uint32_t(ex + 127) << (8 * a);
		}
		uint32_t imask = 0;
		uint32_t meta[2] = { 0u, 0u };
		uint32_t qlo[3][2] = { { 0xFFFFFFFFu, 0xFFFFFFFFu }, { 0xFFFFFFFFu, 0xFFFFFFFFu }, { 0xFFFFFFFFu, 0xFFFFFFFFu } };
		uint32_t qhi[3][2] = { { 0u, 0u }, { 0u, 0u }, { 0u, 0u } };
		int innerRank = 0, primOffset = 0;
		bool bad = false;
		for(int s = 0; s < 8; ++s) {
			const int i = slotChild[s];
			if(i < 0) continue;
			for(int a = 0; a < 3; ++a) {
				const float l = floorf(__fsub_rd(comp(cmn[i], a), pgrid[a]) * inv[a]) - 1.0f;
				const float h = ceilf(__fsub_ru(comp(cmx[i], a), pgrid[a]) * inv[a]) + 1.0f;
				if(l < 0.0f || h > 255.0f) bad = true; // (NaN boxes of degenerate primitives quantise to slot 0)
				const uint32_t ql = uint32_t(fminf(fmaxf(l, 0.0f), 255.0f));
				const uint32_t qh = uint32_t(fminf(fmaxf(h, 0.0f), 255.0f));
				const int sh = 8 * (s & 3);
				qlo[a][s >> 2] = (qlo[a][s >> 2] & ~(0xFFu << sh)) | (ql << sh);
				qhi[a][s >> 2] = (qhi[a][s >> 2] & ~(0xFFu << sh)) | (qh << sh);
			}
			if(inner[i]) {
				imask |= 1u << s;
				const uint32_t q = queueBase + uint32_t(innerRank);
				const uint32_t idx = childBase + uint32_t(innerRank++);
				if(q < A.nodeCapacity) qout[q] = make_int2(ch[i], int(idx));
				else bad = true;
			} else {
				meta[s >> 2] |= uint32_t((cnt[i] << 5) | primOffset) << (8 * (s & 3));
				for(int j = 0; j < cnt[i]; ++j) A.prims[primBase + uint32_t(primOffset + j)] = A.sortedIds[first[i] + j];
				primOffset += cnt[i];
			}
		}
		if(bad) atomicOr(A.counters + CNT_ERROR, 2u);
		N.eimask = ebytes | (imask << 24);
		N.childBase = childBase;
		N.primBase = primBase;
		N.meta[0] = meta[0]; N.meta[1] = meta[1];
		for(int a = 0; a < 3; ++a) {
			N.qlo[a][0] = qlo[a][0]; N.qlo[a][1] = qlo[a][1];
			N.qhi[a][0] = qhi[a][0]; N.qhi[a][1] = qhi[a][1];
		}
		const float4* src = reinterpret_cast<const float4*>(&N);
		float4* dst = reinterpret_cast<float4*>(A.nodes + w);
#pragma unroll
		for(int k = 0; k < 5; ++k) dst[k] = src[k];
	}
}

} // namespace

cudaError_t build_wide(const WideBuildArgs& a, int32_t* numNodesOut, cudaStream_t stream) {
	*numNodesOut = 0;
	if(a.n < 2) return cudaSuccess;
	k_wide_init<<<1, 1, 0, stream>>>(a.counters, a.queueA);
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const unsigned grid = unsigned(std::max(1, std::min(sms * 8, int((a.nodeCapacity + 127) / 128))));
	constexpr int LEVELS_PER_CHECK = 12;
	uint32_t host[WIDE_COUNTERS];
	for(int level = 0; level < MAX_WIDE_LEVELS;) {
		for(int k = 0; k < LEVELS_PER_CHECK; ++k, ++level) {
			const int2* qin = (level & 1) ? a.queueB : a.queueA;
			int2* qout = (level & 1) ? a.queueA : a.queueB;
			uint32_t* cin = a.counters + CNT_QUEUE + level % 3;
			uint32_t* cout = a.counters + CNT_QUEUE + (level + 1) % 3;
			uint32_t* czero = a.counters + CNT_QUEUE + (level + 2) % 3;
			k_wide_level<<<grid, 128, 0, stream>>>(a, qin, cin, qout, cout, czero);
		}
		cudaError_t e = cudaMemcpyAsync(host, a.counters, sizeof(host), cudaMemcpyDeviceToHost, stream);
		if(e == cudaSuccess) e = cudaStreamSynchronize(stream);
		if(e != cudaSuccess) return e;
		if(host[CNT_ERROR]) return cudaErrorInvalidValue;
		if(host[CNT_QUEUE + level % 3] == 0) {
			if(host[CNT_PRIMS] != uint32_t(a.n)) return cudaErrorInvalidValue;
			*numNodesOut = int32_t(host[CNT_NODES]);
			return cudaSuccess;
		}
	}
	return cudaErrorInvalidValue;
}

} // namespace mb
