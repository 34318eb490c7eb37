// Materials, light sampling and the pinhole camera on the device.
//
// Follows src/core/scene/materials/{material_sampling,lambert,
// microfacet_base,microfacet_specular,emissive}.hpp,
// src/core/scene/lights/{light_tree_sampling,light_sampling,lights}.hpp and
// src/core/cameras/pinhole.hpp:53-81, restricted to the models the
// workloads use (Lambert, Torrance with GGX + Smith, emissive; quad area
// lights, point lights, monochrome environment).
#pragma once

#include "intersect.cuh"

namespace mb {

struct Params { int type; f3 albedo; f2 roughness; f3 radiance; int shadowing; };

MBD Params fetch_material(const DScene& S, uint16_t idx, f2 uv) {
	const DMaterial& m = S.materials[idx];
	Params p;
	p.type = m.type;
	p.albedo = (m.albedoTex >= 0) ? sample_texture(S.textures[m.albedoTex], uv) : load3(m.albedo);
	p.roughness = make2(m.roughness[0], m.roughness[1]);
	p.radiance = load3(m.radiance);
	p.shadowing = m.shadowing;
	return p;
}

MBD uint16_t material_index(const DScene& S, int inst, int prim) {
	const DLod& l = S.lods[__ldg(S.instanceLod + inst)];
	const uint32_t faces = l.numTriangles + l.numQuads;
	if(uint32_t(prim) < faces) return __ldg(l.faceMaterials + prim);
	return __ldg(l.sphereMaterials + (uint32_t(prim) - faces));
}

struct PathSample { f3 throughput; bool valid; f3 excident; float pdfF, pdfB; };
struct EvalValue { f3 value; float cosOut; float pdfF, pdfB; };

MBD f3 sample_dir_cosine(float u0, float u1) {
	const float cosTheta = sqrt_(u0);
	const float sinTheta = sqrt_(1.0f - u0);
	const float phi = u1 * 2.0f * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	return make3(sinTheta * s, sinTheta * c, cosTheta);
}
MBD f3 sample_dir_sphere_uniform(float u0, float u1) {
	const float cosTheta = u0 * 2.0f - 1.0f;
	const float sinTheta = sqrt_((1.0f - cosTheta) * (1.0f + cosTheta));
	const float phi = u1 * 2.0f * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	return make3(sinTheta * s, sinTheta * c, cosTheta);
}
MBD float projected_area(f3 dir, const float* mn, const float* mx) {
	const f3 sides = make3(mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]);
	const float ax = sides.y * sides.z * fabsf(dir.x);
	const float ay = sides.x * sides.z * fabsf(dir.y);
	const float az = sides.x * sides.y * fabsf(dir.z);
	return ax + ay + az;
}

MBD float geo_smith(float wDotH, f3 w, f2 r) {
	if(wDotH * w.z <= 0.0f) return 0.0f;
	const float a = w.x * r.x, b = w.y * r.y;
	const float oneOverASq = sdiv(a * a + b * b, w.z * w.z);
	return __fdiv_rn(2.0f, 1.0f + sqrt_(1.0f + oneOverASq));
}
MBD float eval_ggx(f2 r, f3 h) {
	const float norm = fmax_(PI * r.x * r.y, 1e-30f);
	const float cosThetaSq = h.z * h.z;
	const float rx = sdiv(h.x, r.x), ry = sdiv(h.y, r.y);
	const float tmp = rx * rx + ry * ry + cosThetaSq;
	return sdiv(1.0f, norm * tmp * tmp);
}
MBD f2 sample_slopes_ggx(float tanTheta, float u0, float u1, u64& rnd2) {
	// The reference compares against the double 0.0001; for a float x,
	// x < 0.0001 (double) <=> x <= 0.0001f.
	if(tanTheta <= 0.0001f) {
		const float r = sqrt_(sdiv(u0, 1.0f - u0));
		const float phi = 6.28318530718f * u1;
		float s, c;
		mbmath::sincos(phi, s, c);
		return make2(r * c, r * s);
	}
	const float a1 = __fdiv_rn(1.0f, tanTheta);
	const float g1 = __fdiv_rn(2.0f, 1.0f + sqrt_(1.0f + __fdiv_rn(1.0f, a1 * a1)));
	const float a = __fdiv_rn(2.0f * u0, g1) - 1.0f;
	const float tmp = sdiv(1.0f, a * a - 1.0f);
	const float d = tmp * sqrt_(tanTheta * tanTheta - __fdiv_rn(a * a - tanTheta * tanTheta, tmp));
	const float sx1 = tanTheta * tmp - d;
	const float sx2 = tanTheta * tmp + d;
	const float slopeX = (a < 0.0f || sx2 > __fdiv_rn(1.0f, tanTheta)) ? sx1 : sx2;
	float s;
	if(rnd2 & (1ull << 63)) { rnd2 *= 2; s = 1.0f; } else { rnd2 *= 2; s = -1.0f; }
	const float z = sdiv(u1 * (u1 * (u1 * 0.27385f - 0.73369f) + 0.46341f),
	                     u1 * (u1 * (u1 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
	const float slopeY = s * z * sqrt_(1.0f + slopeX * slopeX);
	return make2(slopeX, slopeY);
}
MBD f3 sample_visible_normal_smith(f3 inc, f2 r, float u0, float u1, u64& rnd2) {
	f3 st = normalize(inc * make3(r.x, r.y, 1.0f));
	if(inc.z < 0.0f) st = -st;
	const float sinTheta = sqrt_((1.0f - st.z) * (1.0f + st.z));
	const float tanTheta = __fdiv_rn(sinTheta, st.z);
	const float cosPhi = sinTheta > 1e-5f ? __fdiv_rn(st.x, sinTheta) : 0.0f;
	const float sinPhi = sinTheta > 1e-5f ? __fdiv_rn(st.y, sinTheta) : 0.0f;
	f2 sl = sample_slopes_ggx(tanTheta, u0, u1, rnd2);
	const float tmp = cosPhi * sl.x - sinPhi * sl.y;
	sl.y = sinPhi * sl.x + cosPhi * sl.y;
	sl.x = tmp;
	sl.x *= r.x;
	sl.y *= r.y;
	return normalize(make3(-sl.x, -sl.y, 1.0f));
}
// microfacet_base.hpp:73-81: V-cavity shadowing of one direction
MBD float geo_vcavity(float wDotH, float wDotN, float hDotN) {
	if(wDotH * wDotN <= 0.0f) return 0.0f;
	return fmin_(1.0f, 2.0f * fabsf(sdiv(hDotN * wDotN, wDotH)));
}
// microfacet_base.hpp:116-142: the multi-bounce compensation applied to
// min(Gi, Ge) for reflection. The eighth power is three squarings.
MBD float vcavity_reflection(float gi, float ge) {
	const float g = fmin_(gi, ge);
	if(g < 0.11f) {
		const float x = g + 0.74299714456847f;
		const float x2 = x * x, x4 = x2 * x2;
		return x4 * x4 - 0.092874643071059f;
	}
	return ((1.139400367544197f * g - 3.317658394008854f) * g + 3.317115685385115f) * g - 0.13885765892046f;
}
// microfacet_base.hpp:323-343: a microfacet normal drawn from the GGX
// distribution itself (slope space), with its pdf
MBD f3 sample_ndf_ggx(f2 r, float u0, float u1, float& pdf) {
	const float phi = 2.0f * PI * u0;
	const float e = sqrt_(__fdiv_rn(u1, 1.0f - u1));
	float s, c;
	mbmath::sincos(phi, s, c);
	float slopeX = e * c, slopeY = e * s;
	const float norm = PI * r.x * r.y;
	const float tmp = 1.0f + slopeX * slopeX + slopeY * slopeY;
	slopeX *= r.x;
	slopeY *= r.y;
	const f3 dir = normalize(make3(-slopeX, -slopeY, 1.0f));
	pdf = __fdiv_rn(1.0f, fmax_(norm * tmp * tmp * dir.z * dir.z * dir.z, 1e-20f));
	return dir;
}
// microfacet_base.hpp:149-170: the cavity normal or its mirror image, chosen
// in proportion to their visibility from the incident direction
MBD f3 sample_visible_normal_vcavity(f3 inc, f3 cav, u64 rnd, float& iDotH) {
	const f3 adj = make3(-cav.x, -cav.y, cav.z);
	const float dOut = dot(inc, cav), dAdj = dot(inc, adj);
	const float t = inc.z > 0.0f ? __fdiv_rn(fmax_(0.0f, dAdj), fmax_(0.0f, dOut) + fmax_(0.0f, dAdj))
	                             : __fdiv_rn(fmax_(0.0f, -dAdj), fmax_(0.0f, -dOut) + fmax_(0.0f, -dAdj));
	if(rnd < percentage_of(~0ull, t)) { iDotH = dAdj; return adj; }
	iDotH = dOut;
	return cav;
}

MBD f3 half_vector(f3 inTS, f3 exTS) {
	const f3 h = 1.0f * inTS + 1.0f * exTS;
	const float l = len(h) * sgn(h.z);
	return make3(sdiv(h.x, l), sdiv(h.y, l), sdiv(h.z, l));
}

constexpr float SHADING_NORMAL_EPS = 1e-3f; // material_sampling.hpp:56

// material_sampling.hpp:77-141. adjoint: a vertex of a light sub-path; the
// throughput gets the shading-normal correction of :132-135.
MBD PathSample material_sample(const TangentSpace& ts, const Params& p, f3 incident, float u0, float u1, u64 i0,
                               bool adjoint = false) {
	PathSample none; none.valid = false; none.throughput = make3(0, 0, 0); none.excident = make3(0, 0, 0); none.pdfF = none.pdfB = 0.0f;
	const float iDotG = -dot(incident, ts.geoN);
	const float iDotN = -dot(incident, ts.shadingN);
	if(iDotG * iDotN <= 0.0f) return none;
	const f3 inTS = make3(-dot(incident, ts.shadingTX), -dot(incident, ts.shadingTY), iDotN);
	PathSample res;
	if(p.type == MAT_LAMBERT) {
		const f3 e = sample_dir_cosine(u0, u1);
		res.throughput = p.albedo; res.valid = true; res.excident = e * sgn(inTS.z);
		res.pdfF = __fdiv_rn(e.z, PI);
		res.pdfB = __fdiv_rn(fabsf(inTS.z), PI);
	} else if(p.type == MAT_TORRANCE) {
		// microfacet_specular.hpp:26-79
		u64 rnd = i0;
		f3 h;
		float cavityPdf, iDotH;
		if(p.shadowing == SHADOW_SMITH) {
			h = sample_visible_normal_smith(inTS, p.roughness, u0, u1, rnd);
			cavityPdf = eval_ggx(p.roughness, h);
			cavityPdf *= h.z;
			iDotH = dot(inTS, h);
		} else {
			const f3 cav = sample_ndf_ggx(p.roughness, u0, u1, cavityPdf);
			h = sample_visible_normal_vcavity(inTS, cav, rnd, iDotH);
		}
		const f3 exTS = (2.0f * iDotH) * h - inTS;
		float ge, gi, g;
		if(p.shadowing == SHADOW_SMITH) {
			ge = geo_smith(iDotH, exTS, p.roughness);
			gi = geo_smith(iDotH, inTS, p.roughness);
			g = gi * ge;
		} else {
			ge = geo_vcavity(iDotH, exTS.z, h.z);
			gi = geo_vcavity(iDotH, inTS.z, h.z);
			g = vcavity_reflection(gi, ge);
		}
		if(ge == 0.0f || gi == 0.0f) return none;
		res.throughput = p.albedo * sdiv(g, gi); res.valid = true; res.excident = exTS;
		res.pdfF = cavityPdf * sdiv(gi, fabsf(4.0f * inTS.z * h.z));
		res.pdfB = cavityPdf * sdiv(ge, fabsf(4.0f * exTS.z * h.z));
	} else {
		return none;
	}
	if(!nonzero(res.throughput)) return none;
	f3 g = (res.excident.x * ts.shadingTX + res.excident.y * ts.shadingTY) + res.excident.z * ts.shadingN;
	g = normalize(g);
	const float eDotG = dot(g, ts.geoN);
	const float eDotN = res.excident.z;
	if(eDotG * eDotN <= 0.0f) return none;
	res.excident = g;
	res.pdfF = fmin_(res.pdfF, 1e9f);
	res.pdfB = fmin_(res.pdfB, 1e9f);
	if(adjoint)
		res.throughput = res.throughput * __fdiv_rn(SHADING_NORMAL_EPS + fabsf(iDotN * eDotG),
		                                            SHADING_NORMAL_EPS + fabsf(iDotG * eDotN));
	return res;
}

// material_sampling.hpp:156-237 (no merge normal). adjoint: a light sub-path
// vertex; the tangent-space directions are swapped for the BSDF, the value
// gets the shading-normal correction and the pdfs are swapped back.
// lightNormal (material_sampling.hpp:173, 217-220): a merge evaluates the view
// vertex's material with the photon's geometric normal in the shadow-masking
// test and corrects the value by |cos| at the shading over the geometric normal.
MBD EvalValue material_evaluate(const TangentSpace& ts, const Params& p, f3 incident, f3 excident,
                                bool adjoint = false, const f3* lightNormal = nullptr) {
	EvalValue none; none.value = make3(0, 0, 0); none.cosOut = 0.0f; none.pdfF = none.pdfB = 0.0f;
	const float iDotN = -dot(incident, ts.shadingN);
	const float eDotN = dot(excident, ts.shadingN);
	if(p.type == MAT_EMISSIVE) {
		if(iDotN * eDotN > 0.0f) return none;
		if(iDotN * eDotN < 0.0f) return none;
	} else {
		if(iDotN * eDotN < 0.0f) return none;
	}
	const f3 geoN = lightNormal ? *lightNormal : ts.geoN;
	const float iDotG = -dot(incident, geoN);
	const float eDotG = dot(excident, geoN);
	if(eDotG * eDotN <= 0.0f || iDotG * iDotN <= 0.0f) return none;
	f3 inTS = make3(-dot(incident, ts.shadingTX), -dot(incident, ts.shadingTY), iDotN);
	f3 exTS = make3(dot(excident, ts.shadingTX), dot(excident, ts.shadingTY), eDotN);
	if(adjoint) { const f3 t = inTS; inTS = exTS; exTS = t; }
	f3 value; float pf, pb;
	if(p.type == MAT_LAMBERT) {
		if(inTS.z * exTS.z < 0.0f) return none;
		value = p.albedo / PI;
		pf = __fdiv_rn(fabsf(exTS.z), PI);
		pb = __fdiv_rn(fabsf(inTS.z), PI);
	} else if(p.type == MAT_TORRANCE) {
		const f3 h = half_vector(inTS, exTS);
		if(inTS.z * exTS.z < 0.0f) return none;
		const float iDotH = dot(inTS, h);
		float ge, gi, g;
		if(p.shadowing == SHADOW_SMITH) {
			ge = geo_smith(iDotH, exTS, p.roughness);
			gi = geo_smith(iDotH, inTS, p.roughness);
			g = gi * ge;
		} else {
			ge = geo_vcavity(iDotH, exTS.z, h.z);
			gi = geo_vcavity(iDotH, inTS.z, h.z);
			g = vcavity_reflection(gi, ge);
		}
		if(ge == 0.0f || gi == 0.0f) return none;
		const float dd = eval_ggx(p.roughness, h);
		value = p.albedo * sdiv(g * dd, fabsf(4.0f * inTS.z * exTS.z));
		pf = sdiv(gi * dd, fabsf(4.0f * inTS.z));
		pb = sdiv(ge * dd, fabsf(4.0f * exTS.z));
	} else {
		return none;
	}
	if(!nonzero(value)) return none;
	EvalValue r; r.value = value; r.cosOut = fabsf(eDotN); r.pdfF = fmin_(pf, 1e9f); r.pdfB = fmin_(pb, 1e9f);
	if(lightNormal) {
		r.value = value * __fdiv_rn(SHADING_NORMAL_EPS + fabsf(eDotN), SHADING_NORMAL_EPS + fabsf(eDotG));
	} else if(adjoint) {
		r.value = value * __fdiv_rn(SHADING_NORMAL_EPS + fabsf(iDotN * eDotG), SHADING_NORMAL_EPS + fabsf(iDotG * eDotN));
		r.pdfF = fmin_(pb, 1e9f); r.pdfB = fmin_(pf, 1e9f);
	}
	return r;
}

struct Nee {
	f3 position;
	float creationPdf;
	f3 dir;
	float cosOut;
	f3 diffIrradiance;
	f3 geoNormal;
	float distSq;
	bool valid;
	int emitMat;      // material of the sampled area light; -1 for point lights and the background
};

MBD f3 lv(const float* p) { return make3(p[0], p[1], p[2]); }

MBD Nee connect_quad(const DScene& S, const DLight& l, f3 pos, float u0, float u1) {
	const f3 tx = lv(l.posV[1]) + u0 * lv(l.posV[3]);
	const f3 ty = lv(l.posV[2]) + u1 * lv(l.posV[3]);
	f3 normal = cross(ty, tx);
	const float area = len(normal);
	normal = normal / area;
	const f3 position = (lv(l.posV[0]) + tx * u1) + lv(l.posV[2]) * u0;
	const DMaterial& m = S.materials[l.material];
	const f3 radiance = m.type == MAT_EMISSIVE ? load3(m.radiance) : make3(0, 0, 0);
	const f3 intensity = radiance * area;
	const float pdf = __fdiv_rn(1.0f, area);
	f3 direction = position - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = sqrt_(distSq);
	direction = direction / dist;
	const float cosOut = dot(normal, -direction);
	f3 value = make3(0, 0, 0); float vcos = 0.0f;
	if(cosOut > 0.0f) { value = intensity; vcos = cosOut; }
	Nee n;
	n.position = position; n.creationPdf = pdf; n.dir = direction; n.cosOut = vcos;
	n.diffIrradiance = value / distSq; n.geoNormal = normal; n.distSq = distSq; n.valid = true;
	n.emitMat = int(l.material);
	return n;
}

// light_sampling.hpp:117-140 + 347-368; sampling.hpp:123-128 (barycentric sample)
MBD Nee connect_tri(const DScene& S, const DLight& l, f3 pos, float u0, float u1) {
	f3 normal = cross(lv(l.posV[1]), lv(l.posV[2]));
	const float area2 = len(normal);
	normal = normal / area2;
	const float area = area2 * 0.5f;
	const float bs = 1.0f - sqrt_(1.0f - u0);
	const float bt = (1.0f - bs) * u1;
	const f3 position = (lv(l.posV[0]) + lv(l.posV[1]) * bs) + lv(l.posV[2]) * bt;
	const DMaterial& m = S.materials[l.material];
	const f3 radiance = m.type == MAT_EMISSIVE ? load3(m.radiance) : make3(0, 0, 0);
	const f3 intensity = radiance * area;
	const float pdf = __fdiv_rn(1.0f, area);
	f3 direction = position - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = sqrt_(distSq);
	direction = direction / dist;
	const float cosOut = dot(normal, -direction);
	f3 value = make3(0, 0, 0); float vcos = 0.0f;
	if(cosOut > 0.0f) { value = intensity; vcos = cosOut; }
	Nee n;
	n.position = position; n.creationPdf = pdf; n.dir = direction; n.cosOut = vcos;
	n.diffIrradiance = value / distSq; n.geoNormal = normal; n.distSq = distSq; n.valid = true;
	n.emitMat = int(l.material);
	return n;
}

// A vector perpendicular to n (not normalised): n crossed with the coordinate
// axis of n's smallest component. The reference takes `perpendicular` from
// its math library (epsilon, absent); the lobes and cones it orients are
// rotationally symmetric about n, so the choice of axis changes which
// direction a random number pair maps to, not the image's expectation.
MBD f3 perpendicular(f3 n) {
	const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
	if(ax <= ay && ax <= az) return make3(0.0f, n.z, -n.y);
	if(ay <= az) return make3(-n.z, 0.0f, n.x);
	return make3(n.y, -n.x, 0.0f);
}

// sampling.hpp:112-119: a direction in the cone cos theta >= maxCos about +z
MBD f3 sample_cone_uniform(float maxCos, float u0, float u1, float& pdf) {
	const float cosTheta = (1.0f - u0) + u0 * maxCos;
	const float sinTheta = sqrt_(1.0f - cosTheta * cosTheta);
	const float phi = (2.0f * u1) * PI;
	float s, c;
	mbmath::sincos(phi, s, c);
	pdf = __fdiv_rn(1.0f, (2.0f * PI) * (1.0f - maxCos));
	return make3(c * sinTheta, s * sinTheta, cosTheta);
}

// light_sampling.hpp:389-430: the cap of the sphere seen from pos, sampled
// uniformly by solid angle; no sample from inside the sphere (an empty NEE,
// valid but without irradiance)
MBD Nee connect_sphere(const DScene& S, const DLight& l, f3 pos, float u0, float u1) {
	Nee n;
	n.valid = true;
	n.emitMat = int(l.material);
	n.position = make3(0.0f, 0.0f, 0.0f); n.creationPdf = 0.0f; n.dir = make3(0.0f, 0.0f, 0.0f); n.cosOut = 0.0f;
	n.diffIrradiance = make3(0.0f, 0.0f, 0.0f); n.geoNormal = make3(0.0f, 0.0f, 0.0f); n.distSq = 0.0f;
	const f3 center = lv(l.position);
	const float r = l.radius;
	f3 centerDir = pos - center;
	const float dist = len(centerDir);
	if(dist <= r) return n;
	centerDir = centerDir / dist;
	const float cosSphere = __fdiv_rn(r, dist);
	float conePdf;
	const f3 d = sample_cone_uniform(cosSphere, u0, u1, conePdf);
	const f3 tx = normalize(perpendicular(centerDir));
	const f3 ty = cross(centerDir, tx);
	const f3 globalDir = (tx * d.x + ty * d.y) + centerDir * d.z;
	const f3 surfPos = center + globalDir * r;
	f3 connection = surfPos - pos;
	const float cDistSq = lensq(connection) + DISTANCESQ_EPSILON;
	const float cDist = sqrt_(cDistSq);
	connection = connection / cDist;
	const DMaterial& m = S.materials[l.material];
	const f3 radiance = m.type == MAT_EMISSIVE ? load3(m.radiance) : make3(0, 0, 0);
	const float sampleArea = __fdiv_rn(r * r, conePdf);
	const float cosOut = fmax_(0.0f, -dot(globalDir, connection));
	n.position = surfPos;
	n.creationPdf = __fdiv_rn(1.0f, sampleArea);
	n.dir = connection;
	n.cosOut = cosOut;
	n.diffIrradiance = radiance * __fdiv_rn(sampleArea, cDistSq);
	n.geoNormal = globalDir;
	n.distSq = cDistSq;
	return n;
}

MBD Nee connect_point(const DLight& l, f3 pos) {
	f3 direction = lv(l.position) - pos;
	const float distSq = lensq(direction) + DISTANCESQ_EPSILON;
	const float dist = sqrt_(distSq);
	direction = direction / dist;
	Nee n;
	n.position = lv(l.position); n.creationPdf = INF_PDF; n.dir = direction; n.cosOut = 0.0f;
	n.diffIrradiance = lv(l.intensity) / distSq; n.geoNormal = make3(0, 0, 0); n.distSq = distSq; n.valid = true;
	n.emitMat = -1;
	return n;
}

MBD Nee connect_background(const DScene& S, f3 pos, float u0, float u1) {
	const f3 dir = sample_dir_sphere_uniform(u0, u1);
	const float dirPdf = __fdiv_rn(1.0f, 4.0f * PI);
	const f3 radiance = lv(S.bgColor) * lv(S.bgScale);
	const f3 diff = radiance / dirPdf;
	const float creation = __fdiv_rn(dirPdf * fabsf(1.0f), MAX_SCENE_SIZE * MAX_SCENE_SIZE);
	const f3 diag = make3(S.aabbMax[0] - S.aabbMin[0], S.aabbMax[1] - S.aabbMin[1], S.aabbMax[2] - S.aabbMin[2]);
	Nee n;
	n.position = pos + dir * len(diag); n.creationPdf = creation; n.dir = dir; n.cosOut = 1.0f;
	n.diffIrradiance = diff; n.geoNormal = make3(0, 0, 0); n.distSq = MAX_SCENE_SIZE * MAX_SCENE_SIZE; n.valid = true;
	n.emitMat = -1;
	return n;
}

MBD Nee adjust(Nee n, float chance) {
	n.creationPdf *= chance;
	n.diffIrradiance = n.diffIrradiance / chance;
	return n;
}

// light_tree_sampling.hpp:278-329 with the positional sub-tree walk of :195-259
MBD Nee lights_connect(const DScene& S, u64 index, u64 numIndices, u64 seed, f3 position, float u0, float u1) {
	u64 rndChoice = numIndices > 0 ? seed + index * (~0ull / numIndices) : seed;
	if(rndChoice == ~0ull) --rndChoice;
	const float bgSum = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
	const float fluxSum = (bgSum + S.dirFlux) + S.rootFlux;
	Nee none; none.valid = false;
	if(!(fluxSum > 0.0f)) return none;
	const float envProb = __fdiv_rn(bgSum, fluxSum);
	const float dirProb = __fdiv_rn(S.dirFlux, fluxSum);
	const float posProb = __fdiv_rn(S.rootFlux, fluxSum);
	const u64 rightEnv = percentage_of(~0ull, envProb);
	if(rndChoice < rightEnv) return adjust(connect_background(S, position, u0, u1), envProb);
	u64 right = percentage_of(~0ull, envProb + dirProb);
	if(rndChoice < right) return none;
	u64 iL = right, iR = ~0ull;
	float lightProb = posProb;
	uint16_t type = S.rootType;
	int idx = S.rootIndex;
	int nodeIdx = 0;
	while(type == LT_INTERNAL) {
		const DLightNode& nd = S.lightNodes[nodeIdx];
		const float probLeft = __fdiv_rn(nd.leftFlux, nd.leftFlux + nd.rightFlux);
		const u64 boundary = iL + percentage_of(iR - iL, probLeft);
		if(rndChoice < boundary) { type = nd.leftType; idx = nd.leftIndex; iR = boundary; lightProb *= probLeft; }
		else { type = nd.rightType; idx = nd.rightIndex; iL = boundary; lightProb *= (1.0f - probLeft); }
		nodeIdx = idx;
	}
	const DLight& l = S.lights[idx];
	if(l.type == LT_QUAD) return adjust(connect_quad(S, l, position, u0, u1), lightProb);
	if(l.type == LT_TRI) return adjust(connect_tri(S, l, position, u0, u1), lightProb);
	if(l.type == LT_SPHERE) return adjust(connect_sphere(S, l, position, u0, u1), lightProb);
	return adjust(connect_point(l, position), lightProb);
}

// light_tree_sampling.hpp:340-412: the area pdfs of a hit on an area light,
// for starting a light path there (emit: what the bidirectional path tracer
// weighs) and for a next-event sample of it from refPos (connect: what the
// path tracer weighs); they differ for spheres, whose next-event samples
// cover only the cap seen from refPos.
struct LightPdfs { float emit, connect; };
MBD LightPdfs light_pdfs(const DScene& S, int inst, int prim, f2 sp, f3 refPos) {
	LightPdfs out; out.emit = 0.0f; out.connect = 0.0f;
	const float bgSum = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
	float p = __fdiv_rn(S.rootFlux, (S.dirFlux + S.rootFlux) + bgSum);
	const u64 key = (u64(uint32_t(inst)) << 32) | uint32_t(prim);
	int lo = 0, hi = int(S.numLightPrims) - 1, found = -1;
	while(lo <= hi) {
		const int mid = (lo + hi) >> 1;
		const u64 k = S.lightPrimKeys[mid];
		if(k == key) { found = mid; break; }
		if(k < key) lo = mid + 1; else hi = mid - 1;
	}
	if(found < 0) return out;
	uint32_t code = S.lightPrimCodes[found];
	uint16_t type = S.rootType;
	int idx = S.rootIndex;
	int nodeIdx = 0;
	while(type == LT_INTERNAL) {
		const DLightNode& nd = S.lightNodes[nodeIdx];
		const float pLeft = __fdiv_rn(nd.leftFlux, nd.leftFlux + nd.rightFlux);
		if(code & 0x80000000u) { p *= (1.0f - pLeft); type = nd.rightType; idx = nd.rightIndex; }
		else { p *= pLeft; type = nd.leftType; idx = nd.leftIndex; }
		nodeIdx = idx;
		code <<= 1;
	}
	const DLight& l = S.lights[idx];
	if(l.type == LT_QUAD) {
		const f3 tx = lv(l.posV[1]) + sp.x * lv(l.posV[3]);
		const f3 ty = lv(l.posV[2]) + sp.y * lv(l.posV[3]);
		out.emit = out.connect = __fdiv_rn(p, len(cross(ty, tx)));
	} else if(l.type == LT_TRI) {
		out.emit = out.connect = __fdiv_rn(p, __fdiv_rn(len(cross(lv(l.posV[1]), lv(l.posV[2]))), 2.0f));
	} else if(l.type == LT_SPHERE) {
		const float cosSphere = __fdiv_rn(l.radius, len(refPos - lv(l.position)));
		const float solidAngle = (2.0f * PI) * (1.0f - cosSphere);
		const float rsq = l.radius * l.radius;
		out.connect = __fdiv_rn(p, solidAngle * rsq);
		out.emit = __fdiv_rn(p, (4.0f * PI) * rsq);
	}
	return out;
}

MBD f3 pinhole_ray(const DCamera& c, int px, int py, float u0, float u1, float& pdf) {
	const f2 sub = make2(float(px) + u0, float(py) + u1);
	f2 cp = make2(__fdiv_rn(sub.x, float(c.resX)), __fdiv_rn(sub.y, float(c.resY)));
	cp = make2(cp.x * 2.0f - 1.0f, cp.y * 2.0f - 1.0f);
	cp = make2(cp.x * c.tanVFov, cp.y * c.tanVFov);
	const float aspect = __fdiv_rn(float(c.resX), float(c.resY));
	const f3 nPos = make3(cp.x * aspect, cp.y, 1.0f);
	const f3 view = lv(c.viewDir), up = lv(c.up);
	const f3 xAxis = cross(view, up);
	const f3 dir = normalize((xAxis * nPos.x + up * nPos.y) + view * nPos.z);
	const float t2 = 2.0f * c.tanVFov;
	const float pixelArea = (t2 * t2) * aspect;
	const float cosOut = dot(view, dir);
	pdf = __fdiv_rn(1.0f, ((pixelArea * cosOut) * cosOut) * cosOut);
	return dir;
}

} // namespace mb
