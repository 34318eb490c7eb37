// The trace stage of the renderers that run in stages per path length (the
// light tracer's and the bidirectional path tracer's staged schedules): one
// launch traces one generation's queued rays, segments (closest hit, stored
// for the next shade stage) and connections (any hit, handed to the
// renderer's visibility handler), and nothing else. Persistent warps take 32
// items at a time from a counter once all their lanes are idle, so the warp
// refills in one step and the traversal loop is the only code in the kernel.
#pragma once

#include "wide_traverse.cuh"

#include <cooperative_groups.h>

namespace mb {

// One generation's rays. Segments come first in the item order, then the
// connections.
struct RayQueue {
	const float4* org;  // segments: origin (xyz)
	const float4* dir;  // direction (xyz)
	float4* hit;        // out: t, instance bits (-1: miss), primitive bits, surface u
	float* hitV;        // out: surface v
	const float4* sOrg; // connections: origin, length
	const float4* sDir; // direction (xyz)
	unsigned nExt, nSh;
	unsigned* work;     // item counter of this launch (zero before it)
};

// A slot in a queue for every calling lane, one atomic per group of
// converged lanes.
MBD unsigned queue_reserve(unsigned* counter) {
	namespace cg = cooperative_groups;
	cg::coalesced_group g = cg::coalesced_threads();
	unsigned base = 0;
	if(g.thread_rank() == 0) base = atomicAdd(counter, g.size());
	base = g.shfl(base, 0);
	return base + g.thread_rank();
}

// Traces the queue; visible(s, occluded) is called for connection s once its
// shadow ray ends. The traversal statistics go to `counters`.
template < int AM, class Visibility >
MBD void trace_ray_queue(const DScene& S, const RayQueue& Q, TraceCounters* counters, Visibility&& visible) {
	const unsigned total = Q.nExt + Q.nSh;
	if(total == 0) return;
	LocalStack stack;
	LocalCounters cnt;
	const unsigned lane = threadIdx.x & 31u;
	WideTracerT<AM> t;
	bool active = false, exhausted = false;
	unsigned item = 0;
	for(;;) {
		const unsigned busy = __ballot_sync(0xffffffffu, active);
		const unsigned idle = __ballot_sync(0xffffffffu, !active && !exhausted);
		if(idle && !busy) {
			unsigned base = 0;
			if(lane == unsigned(__ffs(int(idle)) - 1)) base = atomicAdd(Q.work, unsigned(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, __ffs(int(idle)) - 1);
			if(idle & (1u << lane)) {
				item = base + unsigned(__popc(idle & ((1u << lane) - 1u)));
				if(item >= total) exhausted = true;
				else {
					++cnt.rays;
					if(item < Q.nExt) {
						t.init(S, f4to3(__ldcs(Q.org + item)), f4to3(__ldcs(Q.dir + item)), MAX_SCENE_SIZE, false, cnt);
					} else {
						++cnt.shadow;
						const float4 o = __ldcs(Q.sOrg + (item - Q.nExt));
						t.init(S, f4to3(o), f4to3(__ldcs(Q.sDir + (item - Q.nExt))), o.w, true, cnt);
					}
					active = true;
				}
			}
		}
		if(__all_sync(0xffffffffu, exhausted)) break;
		if(active && t.step(S, cnt, stack)) {
			active = false;
			if(item < Q.nExt) {
				const HitRec& h = t.best;
				__stcs(Q.hit + item, make_float4(h.t, __int_as_float(h.has ? h.inst : -1), __int_as_float(h.has ? h.prim : -1), h.sp.x));
				__stcs(Q.hitV + item, h.sp.y);
			} else {
				visible(item - Q.nExt, t.occluded);
			}
		}
	}
	unsigned long long rays = cnt.rays, shadowRays = cnt.shadow, nodes = cnt.nodes, prims = cnt.prims, inst = cnt.instances;
	unsigned errs = cnt.errors;
	for(int o = 16; o > 0; o >>= 1) {
		rays += __shfl_down_sync(0xffffffffu, rays, o);
		shadowRays += __shfl_down_sync(0xffffffffu, shadowRays, o);
		nodes += __shfl_down_sync(0xffffffffu, nodes, o);
		prims += __shfl_down_sync(0xffffffffu, prims, o);
		inst += __shfl_down_sync(0xffffffffu, inst, o);
		errs += __shfl_down_sync(0xffffffffu, errs, o);
	}
	if(lane == 0 && rays) {
		atomicAdd(&counters->rays, rays);
		atomicAdd(&counters->shadowRays, shadowRays);
		atomicAdd(&counters->nodeVisits, nodes);
		atomicAdd(&counters->primTests, prims);
		atomicAdd(&counters->instanceVisits, inst);
		if(errs) atomicAdd(&counters->errors, errs);
	}
}

} // namespace mb
