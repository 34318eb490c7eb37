// Path-tracing kernel (the CUDA "Pathtracer" of the C API).
//
// One thread traces one path (one sample of one pixel) per iteration, as the
// reference's pt_sample does (src/core/renderer/pt/pt_common.hpp:75-156,
// random_walk.hpp:38-113). Work is distributed by persistent warps: the grid
// is sized to fill every SM of the B200 and each warp claims 32 consecutive
// pixels from a global atomic counter, so long and short paths balance across
// SMs (the reference's gpu_pt.cu:54-99 uses the same persistent-warp idea
// with 8x4 tiles). A pixel is written only by its own thread, so the running
// mean of output_handler_variance.hpp:7-31 is updated in place, without
// atomics and without a separate accumulation kernel.
#include "accumulate.cuh"
#include "aux_targets.cuh"
#include "shading.cuh"
#include "pt_api.hpp"

#include <cstdio>

namespace mb {

enum VType { V_CAMERA = 0, V_SURFACE = 1, V_VOID = 2 };

struct Vertex {
	int type;
	f3 position;
	f3 incidentEncoded;
	float incidentPdf;
	TangentSpace ts;
	int inst, prim;
	f2 surfaceParams;
	Params mat;
};

MBD f3 incident_direction(const Vertex& v) {
	const f3 e = v.incidentEncoded;
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = fminf(fmaxf(t, 0.0f), 1.0f);
	return make3(e.x, e.y, sgn(e.z) * sqrt_(t));
}

MBD float nan_to_zero(float x) { return isnan(x) ? 0.0f : x; }
MBD f3 contribute(f3 acc, f3 c) {
	return make3(acc.x + nan_to_zero(c.x), acc.y + nan_to_zero(c.y), acc.z + nan_to_zero(c.z));
}

// pt_common.hpp:75-156
MBD void pt_sample(const DScene& S, const PtParams& P, int px, int py, u64& rng, f3& radianceOut, f2& hitOut,
                   LocalCounters& cnt, int2* bstack, int2* tstack, float* aux) {
	f3 throughput = make3(1.0f, 1.0f, 1.0f);
	f3 radiance = make3(0.0f, 0.0f, 0.0f);
	f2 hitAcc = make2(0.0f, 0.0f);
	Vertex v;
	v.type = V_CAMERA;
	v.position = lv(S.camera.position);
	v.incidentEncoded = make3(float(px), float(py), 0.0f);
	v.incidentPdf = 1.0f;
	v.inst = v.prim = -1;
	(void)pcg_next(rng); // create_camera consumes one number
	int pathLen = 0;
	float guideA = 0.0f, guideWeight = 1.0f;
	auto aux_add = [&](int c, float x) { aux[c] += nan_to_zero(x); };
	do {
		if(pathLen > 0 && pathLen + 1 >= P.minPathLength && pathLen + 1 <= P.maxPathLength) {
			const u64 neeSeed = pcg_next(rng);
			for(int i = 0; i < P.neeCount; ++i) {
				const u64 r = pcg_next(rng);
				const float nu0 = sample_uniform(uint32_t(r)), nu1 = sample_uniform(uint32_t(r >> 32));
				const Nee nee = lights_connect(S, u64(i), u64(P.neeCount), neeSeed, v.position, nu0, nu1);
				if(!nee.valid) continue;
				EvalValue val = material_evaluate(v.ts, v.mat, incident_direction(v), nee.dir);
				if(nee.cosOut != 0.0f) val.cosOut *= nee.cosOut;
				const f3 rad = val.value * nee.diffIrradiance;
				if(any_pos(rad) && val.cosOut > 0.0f) {
					const bool occ = any_intersection(S, v.position, nee.position, v.ts.geoN, nee.geoNormal, nee.dir, cnt, bstack, tstack);
					if(!occ) {
						const float hitPdf = __fdiv_rn(val.pdfF * fabsf(nee.cosOut), nee.distSq);
						const float mis = __fdiv_rn(1.0f, float(P.neeCount) + __fdiv_rn(hitPdf, nee.creationPdf));
						radiance = contribute(radiance, ((throughput * val.cosOut) * rad) * mis);
						if(aux) aux_add(AUX_LIGHT, __fmul_rn(guideWeight, val.cosOut));
					}
				}
			}
		}
		const u64 x0 = pcg_next(rng), x1 = pcg_next(rng);
		const float ru0 = sample_uniform(uint32_t(x0)), ru1 = sample_uniform(uint32_t(x0 >> 32));
		const float rr = sample_uniform(uint32_t(pcg_next(rng)));
		f3 origin, excident, sThroughput;
		float pdfF;
		if(v.type == V_CAMERA) {
			excident = pinhole_ray(S.camera, px, py, ru0, ru1, pdfF);
			sThroughput = make3(1.0f, 1.0f, 1.0f);
			origin = v.position;
		} else {
			const PathSample s = material_sample(v.ts, v.mat, incident_direction(v), ru0, ru1, x1);
			if(!s.valid) break;
			excident = s.excident;
			sThroughput = s.throughput;
			pdfF = s.pdfF;
			origin = v.position;
		}
		throughput = throughput * sThroughput;
		if(pathLen >= P.rrStartDepth) {
			const float cp = fmin_(maxc(throughput) + 0.1f, 1.0f);
			if(rr >= cp) break;
			throughput = throughput / cp;
		}
		const f3 geoN = (v.type == V_SURFACE) ? v.ts.geoN : make3(0.0f, 0.0f, 0.0f);
		const f3 lastPosition = v.position; // pt_common.hpp:126
		const Intersection hit = first_intersection(S, origin, excident, geoN, MAX_SCENE_SIZE, cnt, bstack, tstack);
		if(hit.inst < 0) {
			v.type = V_VOID;
			v.incidentEncoded = excident;
			v.position = make3(0.0f, 0.0f, 0.0f);
			v.incidentPdf = pdfF * 1.0f;
		} else {
			const f3 position = origin + excident * hit.distance;
			v.ts = tangent_space(S, hit);
			v.type = V_SURFACE;
			v.position = position;
			v.incidentEncoded = make3(excident.x, excident.y, hit.distance * sgn(excident.z));
			v.inst = hit.inst;
			v.prim = hit.prim;
			v.surfaceParams = hit.sp;
			v.mat = fetch_material(S, material_index(S, hit.inst, hit.prim), hit.uv);
			const float inCosAbs = fabsf(dot(excident, v.ts.shadingN));
			v.incidentPdf = __fdiv_rn(pdfF * fabsf(inCosAbs), hit.distance * hit.distance);
		}
		if(pathLen == 0)
			hitAcc = make2(float(v.type == V_SURFACE ? v.inst : -1), float(v.type == V_SURFACE ? v.prim : -1));
		if(aux) guideWeight = guide_after_segment(guideA, pdfF);
		++pathLen;
		if(pathLen >= P.minPathLength) {
			f3 emission = make3(0.0f, 0.0f, 0.0f);
			float connectPdf = 0.0f;
			if(v.type == V_VOID) {
				if(S.hasBackground) {
					emission = lv(S.bgColor) * lv(S.bgScale);
					if(nonzero(emission)) {
						const float bgFlux = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
						const float p = __fdiv_rn(bgFlux, (S.dirFlux + S.rootFlux) + bgFlux);
						connectPdf = __fdiv_rn(1.0f, 4.0f * PI) * p;
					}
				}
			} else if(v.mat.type == MAT_EMISSIVE) {
				const f3 ex = -incident_direction(v);
				const float cosOut = dot(v.ts.geoN, ex);
				if(cosOut > 0.0f) {
					emission = v.mat.radiance;
					if(nonzero(emission)) connectPdf = light_pdfs(S, v.inst, v.prim, v.surfaceParams, lastPosition).connect;
				}
			}
			if(nonzero(emission) && pathLen > 1) {
				const float misWeight = __fdiv_rn(1.0f, 1.0f + float(P.neeCount) * __fdiv_rn(connectPdf, v.incidentPdf));
				emission = emission * misWeight;
			}
			radiance = contribute(radiance, throughput * emission);
			if(aux) {
				const bool surf = v.type == V_SURFACE;
				const f3 zero = make3(0.0f, 0.0f, 0.0f);
				aux_vertex(aux_add, guideWeight, surf ? v.position : zero, surf ? fabsf(v.incidentEncoded.z) : 0.0f,
				           surf ? v.ts.shadingN : zero, surf ? hit.uv : make2(0.0f, 0.0f),
				           surf && v.mat.type != MAT_EMISSIVE ? v.mat.albedo : zero, emission);
			}
		}
		if(v.type != V_SURFACE) break;
	} while(pathLen < P.maxPathLength);
	radianceOut = radiance;
	hitOut = hitAcc;
}

__global__ void seed_rng_kernel(u64* states, uint32_t numPixels, int32_t seed) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= numPixels) return;
	// cpu_pt.cpp:40-45 / gpu_pt.cu:140-145: Rng(pixel + seed * (numPixels + 1))
	const int32_t s = int32_t(uint32_t(seed) * (numPixels + 1u));
	states[i] = pcg_seed(uint32_t(int32_t(i + uint32_t(s))));
}

__launch_bounds__(128)
__global__ void pt_megakernel(const DScene S, const PtParams P, RenderState R, unsigned int* workCounter,
                              TraceCounters* counters, uint32_t pixelBegin, uint32_t pixelEnd) {
	int2 bstack[BLAS_STACK];
	int2 tstack[TLAS_STACK];
	LocalCounters cnt;
	const unsigned lane = threadIdx.x & 31u;
	for(;;) {
		unsigned base = 0;
		if(lane == 0) base = atomicAdd(workCounter, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		const uint32_t pixel = pixelBegin + base + lane;
		if(pixelBegin + base >= pixelEnd) break;
		if(pixel < pixelEnd) {
			const int px = int(pixel % R.width), py = int(pixel / R.width);
			u64 rng = R.rngState[pixel];
			f3 rad; f2 hid;
			float aux[AUX_CHANNELS];
			for(int c = 0; c < AUX_CHANNELS; ++c) aux[c] = 0.0f;
			pt_sample(S, P, px, py, rng, rad, hid, cnt, bstack, tstack, R.auxOn ? aux : nullptr);
			R.rngState[pixel] = rng;
			if(R.auxOn)
				for(int a = 0; a < AUX_TARGETS; ++a) {
					if(!R.aux[a]) continue;
					float* cum = R.aux[a] + size_t(aux_count(a)) * pixel;
					float* var = R.auxVar[a] ? R.auxVar[a] + size_t(aux_count(a)) * pixel : nullptr;
					for(int c = 0; c < aux_count(a); ++c)
						update_moments(aux[aux_first(a) + c], cum + c, var ? var + c : nullptr, R.iteration);
				}
			if(R.radiance) {
				float* cr = R.radiance + 3 * size_t(pixel);
				float* vr = R.radianceVar ? R.radianceVar + 3 * size_t(pixel) : nullptr;
				const float it[3] = { rad.x, rad.y, rad.z };
				for(int c = 0; c < 3; ++c) update_moments(it[c], cr + c, vr ? vr + c : nullptr, R.iteration);
			}
			if(R.hitId) {
				float* ch = R.hitId + 2 * size_t(pixel);
				float* vh = R.hitIdVar ? R.hitIdVar + 2 * size_t(pixel) : nullptr;
				const float it[2] = { hid.x, hid.y };
				for(int c = 0; c < 2; ++c) update_moments(it[c], ch + c, vh ? vh + c : nullptr, R.iteration);
			}
			if(R.iterRadiance) {
				float* o = R.iterRadiance + 3 * size_t(pixel);
				o[0] = rad.x; o[1] = rad.y; o[2] = rad.z;
			}
		}
	}
	// one atomic per warp for the counters
	unsigned long long rays = cnt.rays, shadow = cnt.shadow, nodes = cnt.nodes, prims = cnt.prims, inst = cnt.instances;
	unsigned errs = cnt.errors;
	for(int o = 16; o > 0; o >>= 1) {
		rays += __shfl_down_sync(0xffffffffu, rays, o);
		shadow += __shfl_down_sync(0xffffffffu, shadow, o);
		nodes += __shfl_down_sync(0xffffffffu, nodes, o);
		prims += __shfl_down_sync(0xffffffffu, prims, o);
		inst += __shfl_down_sync(0xffffffffu, inst, o);
		errs += __shfl_down_sync(0xffffffffu, errs, o);
	}
	if(lane == 0) {
		atomicAdd(&counters->rays, rays);
		atomicAdd(&counters->shadowRays, shadow);
		atomicAdd(&counters->nodeVisits, nodes);
		atomicAdd(&counters->primTests, prims);
		atomicAdd(&counters->instanceVisits, inst);
		if(errs) atomicAdd(&counters->errors, errs);
	}
}

// Ray-query kernel used by the trace extension of the C API.
__global__ void trace_rays_kernel(const DScene S, const float* rays, const float* geoNormals, float tmax, uint32_t n,
                                  float* tOut, int32_t* instOut, int32_t* primOut, float* spOut) {
	int2 bstack[BLAS_STACK];
	int2 tstack[TLAS_STACK];
	LocalCounters cnt;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		f3 o = make3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
		const f3 d = make3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
		const f3 g = geoNormals ? make3(geoNormals[3 * i], geoNormals[3 * i + 1], geoNormals[3 * i + 2]) : make3(0, 0, 0);
		const Intersection h = first_intersection(S, o, d, g, tmax, cnt, bstack, tstack);
		tOut[i] = h.distance; instOut[i] = h.inst; primOut[i] = h.prim;
		if(spOut) { spOut[2 * i] = h.sp.x; spOut[2 * i + 1] = h.sp.y; }
	}
}

__global__ void occlusion_kernel(const DScene S, const float* a, const float* b, uint32_t n, uint8_t* out) {
	int2 bstack[BLAS_STACK];
	int2 tstack[TLAS_STACK];
	LocalCounters cnt;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const f3 pa = make3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
		const f3 pb = make3(b[3 * i], b[3 * i + 1], b[3 * i + 2]);
		const f3 dv = pb - pa;
		const f3 dir = dv / len(dv);
		out[i] = any_intersection(S, pa, pb, make3(0, 0, 0), make3(0, 0, 0), dir, cnt, bstack, tstack) ? 1 : 0;
	}
}

// Streaming read of an L2-resident buffer: the measured L2 read bandwidth is
// the roofline denominator of the traversal kernel.
__global__ void l2_read_kernel(const float4* __restrict__ buf, size_t n, int reps, float* sink) {
	float acc = 0.0f;
	for(int r = 0; r < reps; ++r)
		for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
			const float4 v = __ldcg(buf + i);
			acc += v.x + v.y + v.z + v.w;
		}
	if(acc == 1234.5f) *sink = acc;
}

// ------------------------------------------------------------ host wrappers
static int sm_count() {
	static int n = 0;
	if(n == 0) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		if(n <= 0) n = 148;
	}
	return n;
}

cudaError_t launch_seed_rng(uint64_t* states, uint32_t numPixels, int32_t seed, cudaStream_t stream) {
	seed_rng_kernel<<<(numPixels + 255) / 256, 256, 0, stream>>>(states, numPixels, seed);
	return cudaGetLastError();
}

cudaError_t launch_pt(const DScene& S, const PtParams& P, const RenderState& R, unsigned int* workCounter,
                      TraceCounters* counters, uint32_t pixelBegin, uint32_t pixelEnd, int blocksPerSm,
                      cudaStream_t stream) {
	cudaError_t e = cudaMemsetAsync(workCounter, 0, sizeof(unsigned int), stream);
	if(e != cudaSuccess) return e;
	const int blocks = sm_count() * (blocksPerSm > 0 ? blocksPerSm : 8);
	pt_megakernel<<<blocks, 128, 0, stream>>>(S, P, R, workCounter, counters, pixelBegin, pixelEnd);
	return cudaGetLastError();
}

cudaError_t launch_trace_rays(const DScene& S, const float* rays, const float* geoNormals, float tmax, uint32_t n,
                              float* t, int32_t* inst, int32_t* prim, float* sp, cudaStream_t stream) {
	const int blocks = (int)std::min<uint32_t>((n + 127) / 128, uint32_t(sm_count() * 16));
	if(n == 0) return cudaSuccess;
	trace_rays_kernel<<<blocks, 128, 0, stream>>>(S, rays, geoNormals, tmax, n, t, inst, prim, sp);
	return cudaGetLastError();
}

cudaError_t measure_l2_bandwidth(size_t bytes, int reps, float* gbs) {
	float4* buf = nullptr;
	float* sink = nullptr;
	cudaError_t e = cudaMalloc(&buf, bytes);
	if(e != cudaSuccess) return e;
	if((e = cudaMalloc(&sink, sizeof(float))) != cudaSuccess) { cudaFree(buf); return e; }
	cudaMemset(buf, 0, bytes);
	const size_t n = bytes / sizeof(float4);
	const int blocks = sm_count() * 8;
	cudaEvent_t a, b;
	cudaEventCreate(&a); cudaEventCreate(&b);
	l2_read_kernel<<<blocks, 256>>>(buf, n, 2, sink); // warm the L2
	cudaEventRecord(a);
	l2_read_kernel<<<blocks, 256>>>(buf, n, reps, sink);
	cudaEventRecord(b);
	e = cudaEventSynchronize(b);
	float ms = 0.0f;
	cudaEventElapsedTime(&ms, a, b);
	*gbs = float(double(bytes) * reps / (double(ms) * 1e-3) / 1e9);
	cudaEventDestroy(a); cudaEventDestroy(b);
	cudaFree(buf); cudaFree(sink);
	return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_occlusion(const DScene& S, const float* a, const float* b, uint32_t n, uint8_t* out,
                             cudaStream_t stream) {
	const int blocks = (int)std::min<uint32_t>((n + 127) / 128, uint32_t(sm_count() * 16));
	if(n == 0) return cudaSuccess;
	occlusion_kernel<<<blocks, 128, 0, stream>>>(S, a, b, n, out);
	return cudaGetLastError();
}

} // namespace mb
