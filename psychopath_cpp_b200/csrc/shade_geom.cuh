/*
 * Hit-point geometry and closure selection, evaluated once per ray after the
 * traversal found the closest hit:
 *   - Sphere::intersect_ray's differential geometry (object/sphere.cpp:126-186);
 *   - Bilinear/Bicubic::differential_geometry at the leaf's cell centre
 *     (object/bilinear.hpp:92-125, object/bicubic.hpp:133-177) and the
 *     leaf's offset (object/patch_utils.hpp:82-131);
 *   - SphereLight::intersect_ray's emission and light pdf
 *     (lights/sphere_light.hpp:124-141, 226-242);
 *   - the shader's closure (shading/surface_shader.hpp:28-72, and the
 *     magenta emitter used when no shader is bound, tracer/tracer.cpp:245-250).
 */
#ifndef PSY_SHADE_GEOM_CUH
#define PSY_SHADE_GEOM_CUH

#include "trace_device.cuh"
#include "psy_libm.cuh"

namespace psy {

#define PSY_PI_D 3.14159265358979323846

struct Geo {
	float u, v;
	V3 p, dpdu, dpdv, n, dndu, dndv;
};

struct HitInfo {
	Geo geo;
	bool backfacing;
	float light_pdf;
	V3 offset;
	int closure;      // CLOSURE_*
	float col[3];     // closure colour
};

__device__ __forceinline__ void normal_derivs(const V3& n, const V3& dpdu, const V3& dpdv, const V3& d2pduu,
                                              const V3& d2pduv, const V3& d2pdvv, V3* dndu, V3* dndv) {
	const float E = dot(dpdu, dpdu);
	const float F = dot(dpdu, dpdv);
	const float G = dot(dpdv, dpdv);
	const float e = dot(n, d2pduu);
	const float f = dot(n, d2pduv);
	const float g = dot(n, d2pdvv);
	const float invEGF2 = 1.0f / ((E * G) - (F * F));
	*dndu = ((((f * F) - (e * G)) * invEGF2) * dpdu) + ((((e * F) - (f * E)) * invEGF2) * dpdv);
	*dndv = ((((g * F) - (f * G)) * invEGF2) * dpdu) + ((((f * F) - (g * E)) * invEGF2) * dpdv);
}

__device__ __forceinline__ V3 bl_eval_p(float u, V3 p0, V3 p1) { return (p0 * (1.0f - u)) + (p1 * u); }
__device__ __forceinline__ V3 bl_eval_pd(V3 p0, V3 p1) { return (p0 * -1.0f) + (p1 * 1.0f); }

__device__ __forceinline__ void bilinear_geo(const Patch<4>& p, float u, float v, Geo* g) {
	g->dpdu = bl_eval_pd(bl_eval_p(v, p.p[0], p.p[2]), bl_eval_p(v, p.p[1], p.p[3]));
	g->dpdv = bl_eval_pd(bl_eval_p(u, p.p[0], p.p[1]), bl_eval_p(u, p.p[2], p.p[3]));
	g->n = normalized(cross(g->dpdv, g->dpdu));
	const V3 zero(0.0f);
	const V3 d2pduv = bl_eval_pd(bl_eval_pd(p.p[0], p.p[1]), bl_eval_pd(p.p[2], p.p[3]));
	normal_derivs(g->n, g->dpdu, g->dpdv, zero, d2pduv, zero, &g->dndu, &g->dndv);
}

__device__ __forceinline__ V3 bc_eval_p(float u, V3 p0, V3 p1, V3 p2, V3 p3) {
	const float iu = 1.0f - u;
	const float b0 = iu * iu * iu;
	const float b1 = 3.0f * u * iu * iu;
	const float b2 = 3.0f * u * u * iu;
	const float b3 = u * u * u;
	return (p0 * b0) + (p1 * b1) + (p2 * b2) + (p3 * b3);
}
__device__ __forceinline__ V3 bc_eval_pd(float u, V3 p0, V3 p1, V3 p2, V3 p3) {
	const float iu = 1.0f - u;
	const float d0 = -3.0f * iu * iu;
	const float d1 = (3.0f * iu * iu) - (6.0f * iu * u);
	const float d2 = (6.0f * iu * u) - (3.0f * u * u);
	const float d3 = 3.0f * u * u;
	return (p0 * d0) + (p1 * d1) + (p2 * d2) + (p3 * d3);
}
__device__ __forceinline__ V3 bc_eval_pdd(float u, V3 p0, V3 p1, V3 p2, V3 p3) {
	const float iu = 1.0f - u;
	const float dd0 = 6.0f * iu;
	const float dd1 = (6.0f * u) - (12.0f * iu);
	const float dd2 = (6.0f * iu) - (12.0f * u);
	const float dd3 = 6.0f * u;
	return (p0 * dd0) + (p1 * dd1) + (p2 * dd2) + (p3 * dd3);
}

__device__ __forceinline__ void bicubic_geo(const Patch<16>& p, float u, float v, Geo* g) {
	V3 pu[4], pv[4], pdv[4];
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		pu[i] = bc_eval_p(v, p.p[i], p.p[i + 4], p.p[i + 8], p.p[i + 12]);
		pv[i] = bc_eval_p(u, p.p[i * 4], p.p[i * 4 + 1], p.p[i * 4 + 2], p.p[i * 4 + 3]);
		pdv[i] = bc_eval_pd(u, p.p[i * 4], p.p[i * 4 + 1], p.p[i * 4 + 2], p.p[i * 4 + 3]);
	}
	g->dpdu = bc_eval_pd(u, pu[0], pu[1], pu[2], pu[3]);
	g->dpdv = bc_eval_pd(v, pv[0], pv[1], pv[2], pv[3]);
	g->n = normalized(cross(g->dpdv, g->dpdu));
	const V3 d2pduu = bc_eval_pdd(u, pu[0], pu[1], pu[2], pu[3]);
	const V3 d2pduv = bc_eval_pd(v, pdv[0], pdv[1], pdv[2], pdv[3]);
	const V3 d2pdvv = bc_eval_pdd(v, pv[0], pv[1], pv[2], pv[3]);
	normal_derivs(g->n, g->dpdu, g->dpdv, d2pduu, d2pduv, d2pdvv, &g->dndu, &g->dndv);
}

// Patch at the ray time (the `ipatch` of object/patch_utils.hpp:92-101).
template <int NV>
__device__ __forceinline__ void patch_at(const float* verts, int tsc, float time, Patch<NV>* q) {
	if (tsc == 1) {
		patch_load<NV>(verts, q);
		return;
	}
	const float t_time = time * (float)(tsc - 1);
	int t_index = (int)t_time;
	const float t_nalpha = t_time - (float)t_index;
	if (t_index > tsc - 2) t_index = tsc - 2;
	Patch<NV> a, b;
	patch_load<NV>(verts + t_index * NV * 3, &a);
	patch_load<NV>(verts + (t_index + 1) * NV * 3, &b);
#pragma unroll
	for (int i = 0; i < NV; ++i) q->p[i] = lerp3(t_nalpha, a.p[i], b.p[i]);
}

// SphereLight::sample_pdf (lights/sphere_light.hpp:124-141): the pdf of
// sampling the light from `arr` (position and radius at the ray time).
__device__ __forceinline__ float sphere_light_pdf(V3 pos, float radius_f, V3 arr) {
	const double radius = (double)radius_f;
	const double d2 = (double)length2(pos - arr);
	const double d = sqrt(d2);
	if (d > radius) {
		const double r2d2 = (radius * radius) / d2;
		const double sin_theta_max2 = r2d2 < 1.0 ? r2d2 : 1.0;
		const double cos_theta_max2 = 1.0 - sin_theta_max2;
		const double cos_theta_max = sqrt(cos_theta_max2);
		return (float)(1.0 / (2.0 * PSY_PI_D * (1.0 - cos_theta_max)));
	}
	return (float)(1.0f / (4.0f * PSY_PI_D));
}

// spherical_triangle_solid_angle (utils/monte_carlo.hpp:110-137), in double
// as there.
__device__ __forceinline__ float spherical_triangle_solid_angle(V3 A, V3 B, V3 C) {
	auto clampd = [](double v) { return fmin(1.0, fmax(-1.0, v)); };
	const double cos_a = clampd((double)dot(B, C));
	const double cos_b = clampd((double)dot(C, A));
	const double cos_c = clampd((double)dot(A, B));
	const double sin_a = sqrt(1.0 - (cos_a * cos_a));
	const double sin_b = sqrt(1.0 - (cos_b * cos_b));
	const double sin_c = sqrt(1.0 - (cos_c * cos_c));
	if (cos_a == 1.0 || cos_b == 1.0 || cos_c == 1.0) return 0.0f;
	const double cos_A = clampd((cos_a - (cos_b * cos_c)) / (sin_b * sin_c));
	const double cos_B = clampd((cos_b - (cos_c * cos_a)) / (sin_c * sin_a));
	const double cos_C = clampd((cos_c - (cos_a * cos_b)) / (sin_a * sin_b));
	return (float)(((acos(cos_A) + acos(cos_B)) + acos(cos_C)) - PSY_PI_D);
}

// The four corners of a rectangle light (dimensions dx, dy), seen from
// `arr` and projected on the unit sphere around it, and the solid angles of
// its two triangles (lights/rectangle_light.hpp:48-57).
__device__ __forceinline__ void rect_light_corners(float dx, float dy, V3 arr, V3 p[4], float* area_1, float* area_2) {
	p[0] = normalized(V3(dx * 0.5f, dy * 0.5f, 0.0f) - arr);
	p[1] = normalized(V3(dx * -0.5f, dy * 0.5f, 0.0f) - arr);
	p[2] = normalized(V3(dx * -0.5f, dy * -0.5f, 0.0f) - arr);
	p[3] = normalized(V3(dx * 0.5f, dy * -0.5f, 0.0f) - arr);
	*area_1 = spherical_triangle_solid_angle(p[1], p[0], p[2]);
	*area_2 = spherical_triangle_solid_angle(p[3], p[0], p[2]);
}

// RectangleLight::sample_pdf (lights/rectangle_light.hpp:73-88).
__device__ __forceinline__ float rect_light_pdf(float dx, float dy, V3 arr) {
	V3 p[4];
	float a1, a2;
	rect_light_corners(dx, dy, arr, p, &a1, &a2);
	return 1.0f / (a1 + a2);
}

__device__ __forceinline__ void closure_of_shader(const DevScene& sc, int shader, HitInfo* h) {
	if (shader < 0) {
		h->closure = CLOSURE_EMIT;
		h->col[0] = 1.0f; h->col[1] = 0.0f; h->col[2] = 1.0f;
		return;
	}
	const DevShader s = sc.shaders[shader];
	h->closure = s.kind == SHADER_LAMBERT ? CLOSURE_LAMBERT : (s.kind == SHADER_EMIT ? CLOSURE_EMIT : CLOSURE_GTR);
	h->col[0] = s.col[0];
	h->col[1] = s.col[1];
	h->col[2] = s.col[2];
}

// Fills the Intersection data of a closest hit. `lo`, `ld` are the ray
// origin and direction in the hit object's space.
static __device__ void hit_geometry(const DevScene& sc, const HitRec& rec, float time, V3 lo, V3 ld, HitInfo* h) {
	const DevObject ob = sc.objects[rec.obj];
	const float t = rec.t;
	h->light_pdf = 9999.0f;
	if (ob.kind == OBJ_SPHERE) {
		V3 cent;
		float radi;
		sphere_at(sc, ob, time, &cent, &radi);
		Geo& g = h->geo;
		g.p = lo + (ld * t);
		g.n = normalized(g.p - cent);
		h->backfacing = dot(g.n, normalized(ld)) > 0.0f;
		const V3 unit_p = g.n;
		const V3 p = unit_p * radi;
		const float lat_cos = unit_p.z;
		const float lat_sin = sqrtf((unit_p.x * unit_p.x) + (unit_p.y * unit_p.y));
		const float long_cos = unit_p.x / lat_sin;
		const float long_sin = unit_p.y / lat_sin;
		const float latitude = lm_acosf(lat_cos);
		float longitude = 0.0f;
		if (unit_p.x != 0.0f || unit_p.y != 0.0f) {
			longitude = lm_acosf(long_cos);
			if (unit_p.y < 0.0f) longitude = (float)((double)(2.0f * (float)1.0f) * PSY_PI_D - (double)longitude);
		}
		const float pi2 = (float)(PSY_PI_D * 2);
		const float pif = (float)PSY_PI_D;
		g.u = longitude / pi2;
		g.v = (float)((double)latitude / PSY_PI_D);
		g.dpdu = V3(p.y * -1.0f, p.x, 0.0f) * pi2;
		g.dpdv = V3(p.z * long_cos, p.z * long_sin, -radi * lat_sin) * pif;
		const V3 d2pduu = V3(p.x, p.y, 0.0f) * (-pi2 * pi2);
		const V3 d2pduv = ((V3(-long_sin, long_cos, 0.0f) * pif) * p.z) * pi2;
		const V3 d2pdvv = V3(p.x, p.y, p.z) * (float)(-PSY_PI_D * PSY_PI_D);
		normal_derivs(g.n, g.dpdu, g.dpdv, d2pduu, d2pduv, d2pdvv, &g.dndu, &g.dndv);
		h->offset = g.n * 0.000001f;
		closure_of_shader(sc, rec.shader, h);
	} else if (ob.kind == OBJ_SPHERE_LIGHT) {
		V3 cent;
		float radi;
		float col[3];
		light_at(sc, ob, time, &cent, &radi, col);
		const double surface_area = 4.0 * PSY_PI_D * (double)radi * (double)radi;
		Geo& g = h->geo;
		g.p = lo + (ld * t);
		g.n = normalized(g.p - cent);
		g.u = g.v = 0.0f;
		g.dpdu = g.dpdv = g.dndu = g.dndv = V3(0.0f);
		h->backfacing = dot(g.n, normalized(ld)) > 0.0f;
		h->light_pdf = sphere_light_pdf(cent, radi, lo);
		h->offset = g.n * 0.000001f;
		h->closure = CLOSURE_EMIT;
		const float sa = (float)surface_area;
		h->col[0] = col[0] / sa;
		h->col[1] = col[1] / sa;
		h->col[2] = col[2] / sa;
	} else if (ob.kind == OBJ_RECT_LIGHT) {
		// RectangleLight::intersect_ray's Intersection (lights/rectangle_light.hpp:122-135)
		float dx, dy, col[3];
		rect_light_at(sc, ob, time, &dx, &dy, col);
		Geo& g = h->geo;
		const float x = lo.x + (ld.x * t);
		const float y = lo.y + (ld.y * t);
		g.p = V3(x, y, 0.0f);
		g.n = V3(0.0f, 0.0f, 1.0f);
		g.u = g.v = 0.0f;
		g.dpdu = g.dpdv = g.dndu = g.dndv = V3(0.0f);
		h->backfacing = ld.z > 0.0f;
		h->light_pdf = rect_light_pdf(dx, dy, lo);
		h->offset = g.n * 0.000001f;
		h->closure = CLOSURE_EMIT;
		const float sa = (float)((double)(dx * dy));
		h->col[0] = (col[0] * 0.5f) / sa;
		h->col[1] = (col[1] * 0.5f) / sa;
		h->col[2] = (col[2] * 0.5f) / sa;
	} else {
		Geo& g = h->geo;
		g.p = lo + (ld * t);
		g.u = rec.u;
		g.v = rec.v;
		const float* verts = sc.fpool + ob.data;
		if (ob.kind == OBJ_BILINEAR) {
			Patch<4> q;
			patch_at<4>(verts, ob.n0, time, &q);
			bilinear_geo(q, rec.u, rec.v, &g);
		} else {
			Patch<16> q;
			patch_at<16>(verts, ob.n0, time, &q);
			bicubic_geo(q, rec.u, rec.v, &g);
		}
		h->backfacing = dot(g.n, normalized(ld)) > 0.0f;
		h->offset = g.n * (rec.max_dim * 1.74f);
		closure_of_shader(sc, rec.shader, h);
	}
}

}  // namespace psy

#endif
