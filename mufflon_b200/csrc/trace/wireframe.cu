// Wireframe renderer (the CUDA "Wireframe" of the C API): per pixel and
// iteration one camera ray, walked through the surfaces it meets until it
// passes within "Line width" pixels of a triangle or quad edge (or of a
// sphere's rim), which paints the pixel white; a ray that leaves the scene
// shows the background (src/core/renderer/wireframe/wireframe_common.hpp:
// 93-180, cpu_wireframe.cpp:18-38: a persistent generator per pixel seeded
// with the pixel index). One thread per pixel; the rays are coherent camera
// rays, traced over the 8-wide hierarchies.
#include "accumulate.cuh"
#include "shading.cuh"
#include "wide_traverse.cuh"
#include "lt_api.hpp"

namespace mb {
namespace {

MBD f3 xform34(const float* m, f3 p) {
	return make3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
	             m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
	             m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}

// wireframe_common.hpp:15-41 (triangle) and 43-78 (quad): the point on the
// closest edge line. Edge k is chosen if its distance is <= every other
// edge's, tried in order, else the last edge (the reference's comparison
// chain, :36-41 and :70-77): a NaN distance from a zero-length edge never
// wins a comparison, so such a triangle falls through to its last edge.
MBD f3 closest_line_point(const f3* c, int n, f3 hit) {
	// edges: triangle AB, AC, BC; quad AB, AC, BD, CD with (A, B, C, D) = (v0, v1, v3, v2)
	const int e0[4] = { 0, 0, 1, 2 };
	const int e1[4] = { 1, 2, n == 3 ? 2 : 3, 3 };
	const int ne = n == 3 ? 3 : 4;
	f3 on[4];
	float d[4];
	for(int k = 0; k < ne; ++k) {
		const f3 a = c[e0[k]], e = c[e1[k]] - a, ap = hit - a;
		on[k] = a + e * __fdiv_rn(dot(ap, e), lensq(e));
		d[k] = lensq(on[k] - hit);
	}
	for(int k = 0; k + 1 < ne; ++k) {
		bool closest = true;
		for(int j = 0; j < ne; ++j)
			if(j != k && !(d[k] <= d[j])) closest = false;
		if(closest) return on[k];
	}
	return on[ne - 1];
}

__global__ void k_wireframe(const DScene S, const float* instToWorld, WireParams P, uint64_t* rngState, float4* iter,
                            uint32_t width, uint32_t height, TraceCounters* counters) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	LocalStack stack;
	LocalCounters cnt;
	if(p < width * height) {
		const int px = int(p % width), py = int(p / width);
		u64 rng = rngState[p];
		(void)pcg_next(rng); // create_camera consumes one number (unused by the pinhole camera)
		const u64 x0 = pcg_next(rng);
		(void)pcg_next(rng);
		float pdf;
		f3 dir = pinhole_ray(S.camera, px, py, sample_uniform(uint32_t(x0)), sample_uniform(uint32_t(x0 >> 32)), pdf);
		const f3 cam = lv(S.camera.position);
		f3 origin = cam;
		float total = 0.0f;
		float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		for(int i = 0; i < P.maxTraceDepth; ++i) {
			const HitRec hr = closest_hit_wide<ALPHA_NEVER>(S, origin, dir, MAX_SCENE_SIZE, cnt, stack);
			if(!hr.has) {
				// evaluate_background (light_sampling.hpp:467-471)
				if(S.hasBackground) {
					const f3 bg = lv(S.bgColor) * lv(S.bgScale);
					if(any_pos(bg)) out = make_float4(bg.x, bg.y, bg.z, 0.0f);
				}
				break;
			}
			const float hitDist = hr.t < 0.001f ? 0.001f : hr.t;
			const f3 hit = origin + dir * hitDist;
			total += hitDist;
			const float pixelSize = __fdiv_rn(total * S.camera.tanVFov, float(S.camera.resY));
			const float* m = instToWorld + 12 * size_t(hr.inst);
			const DLod& l = S.lods[__ldg(S.instanceLod + hr.inst)];
			float rim;
			if(uint32_t(hr.prim) < l.numTriangles + l.numQuads) {
				f3 c[4];
				int n;
				if(uint32_t(hr.prim) < l.numTriangles) {
					const uint32_t o = 3u * uint32_t(hr.prim);
					for(int k = 0; k < 3; ++k) c[k] = xform34(m, vert(l, __ldg(l.indices + o + k)));
					n = 3;
				} else {
					const uint32_t o = 3u * l.numTriangles + 4u * (uint32_t(hr.prim) - l.numTriangles);
					// (A, B, C, D) = (v0, v1, v3, v2)
					c[0] = xform34(m, vert(l, __ldg(l.indices + o)));
					c[1] = xform34(m, vert(l, __ldg(l.indices + o + 1)));
					c[2] = xform34(m, vert(l, __ldg(l.indices + o + 3)));
					c[3] = xform34(m, vert(l, __ldg(l.indices + o + 2)));
					n = 4;
				}
				const f3 seg = closest_line_point(c, n, hit) - cam;
				const f3 proj = seg - dir * dot(seg, dir);
				rim = len(proj);
			} else {
				// wireframe_common.hpp:79-89 and 166-172
				const float4 s = __ldg(l.spheres + (hr.prim - int(l.numTriangles + l.numQuads)));
				const f3 center = xform34(m, f4to3(s));
				const f3 toCenter = normalize(center - hit);
				rim = 0.05f * (s.w * dot(toCenter, dir));
			}
			if(rim > P.lineWidth * pixelSize) origin = origin + dir * hitDist;
			else { out = make_float4(1.0f, 1.0f, 1.0f, 0.0f); break; }
		}
		rngState[p] = rng;
		iter[p] = out;
	}
	unsigned long long rays = cnt.rays, nodes = cnt.nodes, prims = cnt.prims, inst = cnt.instances;
	unsigned errs = cnt.errors;
	for(int o = 16; o > 0; o >>= 1) {
		rays += __shfl_down_sync(0xffffffffu, rays, o);
		nodes += __shfl_down_sync(0xffffffffu, nodes, o);
		prims += __shfl_down_sync(0xffffffffu, prims, o);
		inst += __shfl_down_sync(0xffffffffu, inst, o);
		errs += __shfl_down_sync(0xffffffffu, errs, o);
	}
	if((threadIdx.x & 31u) == 0) {
		atomicAdd(&counters->rays, rays);
		atomicAdd(&counters->nodeVisits, nodes);
		atomicAdd(&counters->primTests, prims);
		atomicAdd(&counters->instanceVisits, inst);
		if(errs) atomicAdd(&counters->errors, errs);
	}
}

// output_handler_variance.hpp:7-31, into the radiance buffers (the "Border"
// target and its variance)
__global__ void k_wireframe_finalize(LtTargets T) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if(p >= T.width * T.height || !T.radiance) return;
	const float4 it = T.iter[p];
	float* cr = T.radiance + 3 * size_t(p);
	float* vr = T.radianceVar ? T.radianceVar + 3 * size_t(p) : nullptr;
	const float v[3] = { it.x, it.y, it.z };
	for(int c = 0; c < 3; ++c) update_moments(v[c], cr + c, vr ? vr + c : nullptr, T.iteration);
}

} // namespace

cudaError_t launch_wireframe(const DScene& S, const float* instToWorld, const WireParams& P, const LtTargets& T,
                             TraceCounters* counters, cudaStream_t stream) {
	const uint32_t n = T.width * T.height;
	if(n == 0) return cudaSuccess;
	k_wireframe<<<(n + 127) / 128, 128, 0, stream>>>(S, instToWorld, P, T.rngState, T.iter, T.width, T.height, counters);
	cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) return e;
	k_wireframe_finalize<<<(n + 255) / 256, 256, 0, stream>>>(T);
	return cudaGetLastError();
}

} // namespace mb
