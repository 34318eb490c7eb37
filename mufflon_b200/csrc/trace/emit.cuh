// Photon emission and camera projection shared by the light tracer (lt.cu)
// and the bidirectional path tracer (bpt.cu): starting points on point,
// triangle and quad lights and the colored background chosen through the
// light tree (light_tree_sampling.hpp:81-188, light_sampling.hpp:80-306), the
// start points of environment photons on the scene box (sampling.hpp:132-158)
// and the pinhole projection of a direction to a pixel (pinhole.hpp:86-116).
#pragma once

#include "shading.cuh"

namespace mb {

enum LtKind { LV_POINT = 0, LV_AREA = 1, LV_SURFACE = 2, LV_ENV = 3 };

// A photon's start on a light (light_sampling.hpp:20-49 Emitter): the
// position, the intensity divided by the probability of choosing the light
// (light_tree_sampling.hpp:12-16) and, for an area light, its normal; for
// the environment, the direction the photon travels (in `normal`) and the
// irradiance.
struct Emitter { f3 position, intensity, normal; int kind; bool valid; float pChoice, pdf; };

// render_target.hpp:64-75: a NaN channel of a contribution is added as 0
MBD float nan_to_zero(float x) { return isnan(x) ? 0.0f : x; }

// light_sampling.hpp:80-84 (point), 117-140 (triangle), 143-171 (quad), 173-194 (sphere)
MBD Emitter sample_light_pos(const DScene& S, const DLight& l, float u0, float u1, float lightProb) {
	Emitter e;
	e.valid = true;
	if(l.type == LT_POINT) {
		e.position = lv(l.position);
		e.intensity = lv(l.intensity) / lightProb;
		e.normal = make3(0.0f, 0.0f, 0.0f);
		e.kind = LV_POINT;
		e.pChoice = lightProb;
		e.pdf = INF_PDF;
		return e;
	}
	const DMaterial& m = S.materials[l.material];
	const f3 radiance = m.type == MAT_EMISSIVE ? load3(m.radiance) : make3(0, 0, 0);
	if(l.type == LT_SPHERE) {
		// light_sampling.hpp:173-194: a uniformly chosen point of the sphere,
		// its area pdf the direction pdf 1 / (4 pi) over r^2
		const float r = l.radius;
		const f3 normal = sample_dir_sphere_uniform(u0, u1);
		const float area = ((4.0f * PI) * r) * r;
		e.position = lv(l.position) + normal * r;
		e.intensity = (radiance * area) / lightProb;
		e.normal = normal;
		e.kind = LV_AREA;
		e.pChoice = lightProb;
		e.pdf = __fdiv_rn(__fdiv_rn(1.0f, 4.0f * PI) * 1.0f, r * r);
		return e;
	}
	f3 normal, position;
	float area;
	if(l.type == LT_TRI) {
		normal = cross(lv(l.posV[1]), lv(l.posV[2]));
		const float area2 = len(normal);
		normal = normal / area2;
		area = area2 * 0.5f;
		const float bs = 1.0f - sqrt_(1.0f - u0);
		const float bt = (1.0f - bs) * u1;
		position = (lv(l.posV[0]) + lv(l.posV[1]) * bs) + lv(l.posV[2]) * bt;
	} else {
		const f3 tx = lv(l.posV[1]) + u0 * lv(l.posV[3]);
		const f3 ty = lv(l.posV[2]) + u1 * lv(l.posV[3]);
		normal = cross(ty, tx);
		area = len(normal);
		normal = normal / area;
		position = (lv(l.posV[0]) + tx * u1) + lv(l.posV[2]) * u0;
	}
	e.position = position;
	e.intensity = (radiance * area) / lightProb;
	e.normal = normal;
	e.kind = LV_AREA;
	e.pChoice = lightProb;
	e.pdf = __fdiv_rn(1.0f, area);
	return e;
}

// light_sampling.hpp:226-232 and 292-306 (a colored background), scaled by
// the environment's choice probability (light_tree_sampling.hpp:158-167): a
// direction drawn uniformly on the sphere; the photon travels against it.
MBD Emitter sample_background(const DScene& S, float u0, float u1, float envProb) {
	const f3 dir = sample_dir_sphere_uniform(u0, u1);
	const float dirPdf = __fdiv_rn(1.0f, 4.0f * PI);
	const f3 irradiance = (lv(S.bgColor) * lv(S.bgScale)) / dirPdf;
	Emitter e;
	e.valid = true;
	e.kind = LV_ENV;
	e.position = make3(0.0f, 0.0f, 0.0f);
	e.normal = -dir;
	e.intensity = irradiance / envProb;
	e.pChoice = envProb;
	e.pdf = dirPdf;
	return e;
}

// light_tree_sampling.hpp:141-188 with the sub-tree descent of :81-131: the
// photon index spreads the photons evenly over the flux interval before the
// seed's random offset. There are no directional lights.
MBD Emitter lights_emit(const DScene& S, u64 index, u64 numIndices, u64 seed, float u0, float u1) {
	u64 rndChoice = numIndices > 0 ? seed + index * (~0ull / numIndices) : seed;
	if(rndChoice == ~0ull) --rndChoice;
	const float bgSum = (S.bgFlux[0] + S.bgFlux[1]) + S.bgFlux[2];
	const float fluxSum = (bgSum + S.dirFlux) + S.rootFlux;
	Emitter none;
	none.valid = false;
	if(!(fluxSum > 0.0f)) return none;
	const float envProb = __fdiv_rn(bgSum, fluxSum);
	const float dirProb = __fdiv_rn(S.dirFlux, fluxSum);
	const float posProb = __fdiv_rn(S.rootFlux, fluxSum);
	if(rndChoice < percentage_of(~0ull, envProb)) return sample_background(S, u0, u1, envProb);
	const u64 right = percentage_of(~0ull, envProb + dirProb);
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
	return sample_light_pos(S, S.lights[idx], u0, u1, lightProb);
}

// pinhole.hpp:86-116: the pixel a direction leaving the camera falls in and
// the sensor response w (equal to the sampling pdf); false when the direction
// points behind the camera or off the image.
MBD bool pinhole_project(const DCamera& c, f3 excident, int& px, int& py, float& w) {
	const f3 view = lv(c.viewDir), up = lv(c.up);
	const float cosOut = dot(view, excident);
	if(cosOut < 0.0f) return false;
	const f3 xAxis = cross(view, up);
	const float d = cosOut * c.tanVFov;
	float ux = __fdiv_rn(dot(xAxis, excident), d);
	const float uy = __fdiv_rn(dot(up, excident), d);
	const float aspect = __fdiv_rn(float(c.resX), float(c.resY));
	ux = __fdiv_rn(ux, aspect);
	if(!(ux > -1.0f && ux <= 1.0f && uy > -1.0f && uy <= 1.0f)) return false;
	px = int(floorf((ux * 0.5f + 0.5f) * float(c.resX)));
	py = int(floorf((uy * 0.5f + 0.5f) * float(c.resY)));
	if(px >= int(c.resX)) px = int(c.resX) - 1;
	if(py >= int(c.resY)) py = int(c.resY) - 1;
	const float t2 = 2.0f * c.tanVFov;
	const float pixelArea = (t2 * t2) * aspect;
	w = __fdiv_rn(1.0f, ((pixelArea * cosOut) * cosOut) * cosOut);
	return true;
}

MBD f3 decode_incident(f3 e) {
	float t = 1.0f - e.x * e.x - e.y * e.y;
	t = fminf(fmaxf(t, 0.0f), 1.0f);
	return make3(e.x, e.y, sgn(e.z) * sqrt_(t));
}

// math/sampling.hpp:132-158: a start point for a photon of direction dir on
// the faces of the scene box it enters through, and the inverse of the
// box's projected area (the position pdf).
MBD f3 sample_position(const DScene& S, f3 dir, float u0, float u1, float& pdf) {
	const f3 mn = lv(S.aabbMin);
	const f3 sides = lv(S.aabbMax) - mn;
	const float projAx = (sides.y * sides.z) * fabsf(dir.x);
	const float projAy = (sides.x * sides.z) * fabsf(dir.y);
	const float projAz = (sides.x * sides.y) * fabsf(dir.z);
	const float area = (projAx + projAy) + projAz;
	float x = u0 * area;
	f3 p;
	if(x < projAx) {
		x = __fdiv_rn(x - 0.0f, projAx - 0.0f);
		p = make3(dir.x < 0.0f ? 1.0f : 0.0f, u1, x);
	} else if(x < projAx + projAy) {
		x = __fdiv_rn(x - projAx, (projAx + projAy) - projAx);
		p = make3(u1, dir.y < 0.0f ? 1.0f : 0.0f, x);
	} else {
		x = __fdiv_rn(x - (projAx + projAy), area - (projAx + projAy));
		p = make3(u1, x, dir.z < 0.0f ? 1.0f : 0.0f);
	}
	pdf = __fdiv_rn(1.0f, area);
	return (mn + p * sides) - dir * 1e-3f;
}

} // namespace mb
