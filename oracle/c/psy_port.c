/*
 * Test infrastructure: a plain-C restatement of the reference renderer's
 * ray tracing (the checker; never part of the product).  Built into
 * oracle/_build/libpsyoracle.so by oracle/Makefile and loaded only by
 * tests/, the smoke check and the benchmark's CPU-baseline leg.
 *
 * It reads the same flattened scene description as the C ABI
 * (include/psy_b200.h) and traces each ray by testing every instance of
 * every assembly in order (no acceleration structure), keeping the
 * reference's per-object tests and max_t updates:
 *   WorldRay -> Ray widths           basics/ray.hpp:207-305, utils/utils.hpp:443-456
 *   instance transforms, element ids tracer/tracer.cpp:125-219, math/transform.hpp:241-272,
 *                                    basics/instance_id.hpp:18-23
 *   sphere / sphere light            object/sphere.cpp:67-124, lights/sphere_light.hpp:159-221
 *   patch bisection (bilinear, bicubic) object/patch_utils.hpp:18-200,
 *                                    object/bilinear.hpp:44-141, object/bicubic.hpp:55-189
 *   slab test                        basics/bbox.hpp:138-177
 * Closest hits equal the reference's except exact t ties, whose winner
 * depends on visiting order.  Float evaluation order follows the
 * reference; compile without FMA contraction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#include "../../include/psy_b200.h"

typedef struct { float x, y, z; } v3;
typedef struct { float m[4][4]; } m44;

static v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static float fmin_std(float a, float b) { return (b < a) ? b : a; }  /* std::min */
static float fmax_std(float a, float b) { return (a < b) ? b : a; }  /* std::max */
static float vmin_(float a, float b) { return (a < b) ? a : b; }
static float vmax_(float a, float b) { return (a > b) ? a : b; }

/* Imath Vec3<float>::length */
static float len3(v3 a) {
	float l2 = dot3(a, a);
	if (l2 < 2.0f * FLT_MIN) {
		float ax = fabsf(a.x), ay = fabsf(a.y), az = fabsf(a.z), m = ax;
		if (m < ay) m = ay;
		if (m < az) m = az;
		if (m == 0.0f) return 0.0f;
		ax /= m; ay /= m; az /= m;
		return m * sqrtf(ax * ax + ay * ay + az * az);
	}
	return sqrtf(l2);
}

static float longest(v3 v) { return fmax_std(fmax_std(fabsf(v.x), fabsf(v.y)), fabsf(v.z)); }

/* lerp of float sequences and structs (utils/utils.hpp:53-91) */
static void seqpos(float alpha, int n, int* i0, int* single, float* na) {
	if (n <= 1) { *i0 = 0; *single = 1; *na = 0.0f; return; }
	if (alpha >= 1.0f) { *i0 = n - 1; *single = 1; *na = 0.0f; return; }
	{
		float t = alpha * (float)(n - 1);
		int i = (int)t;
		*i0 = i; *single = 0; *na = t - (float)i;
	}
}
static float lerpf(float a, float x, float y) { return (float)((double)x * (1.0 - (double)a) + (double)(y * a)); }

static m44 mload(const float* p) { m44 r; memcpy(r.m, p, 64); return r; }
static m44 mmul(const m44* a, const m44* b) {
	m44 r; int i, j;
	for (i = 0; i < 4; ++i)
		for (j = 0; j < 4; ++j)
			r.m[i][j] = (((b->m[0][j] * a->m[i][0]) + (b->m[1][j] * a->m[i][1])) + (b->m[2][j] * a->m[i][2])) + (b->m[3][j] * a->m[i][3]);
	return r;
}
static m44 mlerp(float al, const m44* a, const m44* b) {
	m44 r; int i, j; float ia = 1.0f - al;
	for (i = 0; i < 4; ++i)
		for (j = 0; j < 4; ++j) r.m[i][j] = (a->m[i][j] * ia) + (b->m[i][j] * al);
	return r;
}
static v3 xpos(const m44* t, v3 v) {
	float r[4]; int j;
	for (j = 0; j < 4; ++j) r[j] = (((t->m[0][j] * v.x) + (t->m[1][j] * v.y)) + (t->m[2][j] * v.z)) + t->m[3][j];
	return V(r[0] / r[3], r[1] / r[3], r[2] / r[3]);
}
static v3 xdir(const m44* t, v3 v) {
	float r[3]; int j;
	for (j = 0; j < 3; ++j) r[j] = ((t->m[0][j] * v.x) + (t->m[1][j] * v.y)) + (t->m[2][j] * v.z);
	return V(r[0], r[1], r[2]);
}

/* ------------------------------------------------------------------ */
typedef struct {
	v3 o, d, dinv;
	float owx, owy, dwx, dwy, fwx, fwy;
} ray_t;

typedef struct {
	v3 o, d, odx, ody, ddx, ddy;
	float time;
	int occl;
} wray_t;

static void closest_t2(v3 o1, v3 d1, v3 o2, v3 d2, float* t, float* dist) {
	v3 dd = sub(d1, d2);
	float dd2 = dot3(dd, dd);
	v3 w;
	if (dd2 < 0.00001f) { *t = -1.0f; *dist = -1.0f; return; }
	w = sub(o1, o2);
	*t = -dot3(w, dd) / dd2;
	*dist = len3(sub(add(o1, mul(d1, *t)), add(o2, mul(d2, *t))));
}

static void setup_ray(ray_t* r, v3 o, v3 d, v3 odx, v3 ody, v3 ddx, v3 ddy) {
	float tdx, lx, tdy, ly;
	r->o = o; r->d = d;
	closest_t2(o, d, add(o, odx), add(d, ddx), &tdx, &lx);
	closest_t2(o, d, add(o, ody), add(d, ddy), &tdy, &ly);
	r->owx = len3(odx);
	if (tdx <= 0.0f) { r->dwx = len3(ddx); r->fwx = 0.0f; } else { r->dwx = (lx - r->owx) / tdx; r->fwx = lx; }
	r->owy = len3(ody);
	if (tdy <= 0.0f) { r->dwy = len3(ddy); r->fwy = 0.0f; } else { r->dwy = (ly - r->owy) / tdy; r->fwy = ly; }
	r->dinv = V(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
}

static void ray_in(ray_t* r, const wray_t* w, const m44* x) {
	if (!x) { setup_ray(r, w->o, w->d, w->odx, w->ody, w->ddx, w->ddy); return; }
	setup_ray(r, xpos(x, w->o), xdir(x, w->d), xdir(x, w->odx), xdir(x, w->ody), xdir(x, w->ddx), xdir(x, w->ddy));
}

static float min_width(const ray_t* r, float tn, float tf) {
	float fx = (r->owx - r->fwx) / r->dwx, fy = (r->owy - r->fwy) / r->dwy, mx, my;
	if (tn < fx && tf > fx) mx = r->fwx;
	else mx = fmin_std(fabsf((r->owx - r->fwx) + (r->dwx * tn)) + r->fwx, fabsf((r->owx - r->fwx) + (r->dwx * tf)) + r->fwx);
	if (tn < fy && tf > fy) my = r->fwy;
	else my = fmin_std(fabsf((r->owy - r->fwy) + (r->dwy * tn)) + r->fwy, fabsf((r->owy - r->fwy) + (r->dwy * tf)) + r->fwy);
	return fmin_std(mx, my);
}

static int box_hit(v3 lo, v3 hi, const ray_t* r, float tmax, float* t0, float* t1) {
	float tx1 = (lo.x - r->o.x) * r->dinv.x, tx2 = (hi.x - r->o.x) * r->dinv.x;
	float h0 = fmin_std(tx1, tx2), h1 = fmax_std(tx1, tx2);
	float ty1 = (lo.y - r->o.y) * r->dinv.y, ty2 = (hi.y - r->o.y) * r->dinv.y;
	float tz1, tz2;
	h0 = fmax_std(h0, fmin_std(ty1, ty2));
	h1 = fmin_std(h1, fmax_std(ty1, ty2));
	tz1 = (lo.z - r->o.z) * r->dinv.z; tz2 = (hi.z - r->o.z) * r->dinv.z;
	h0 = fmax_std(0.0f, fmax_std(h0, fmin_std(tz1, tz2)));
	h1 = fmin_std(h1, fmax_std(tz1, tz2)) * 1.00000024f;
	*t0 = h0; *t1 = h1;
	return h0 <= fmin_std(tmax, h1);
}

/* quadratic of Sphere::intersect_ray / SphereLight::intersect_ray; -1 = miss */
static float sphere_t(const ray_t* r, v3 c, float radi, float max_t) {
	v3 o = sub(r->o, c), d = r->d;
	float a = dot3(d, d), b = 2.0f * dot3(d, o), cc = dot3(o, o) - radi * radi, disc, q, t0, t1, tmp;
	disc = b * b - 4.0f * a * cc;
	if (disc < 0.0f) return -1.0f;
	disc = sqrtf(disc);
	q = (b < 0.0f) ? -0.5f * (b - disc) : -0.5f * (b + disc);
	t0 = q / a;
	t1 = (q != 0.0f) ? cc / q : max_t;
	if (t0 > t1) { tmp = t1; t1 = t0; t0 = tmp; }
	if (t0 >= max_t || t1 < 0.0001f) return -1.0f;
	if (t0 >= 0.0001f) return t0;
	if (t1 < max_t) return t1;
	return -1.0f;
}

/* ------------------------------------------------------------------ */
/* Patches: one routine for 4 (bilinear) or 16 (bicubic) control points. */
typedef struct { v3 p[16]; } patch_t;

static void pbound(const patch_t* q, int nv, v3* lo, v3* hi) {
	int i;
	*lo = q->p[0]; *hi = q->p[0];
	for (i = 1; i < nv; ++i) {
		lo->x = vmin_(lo->x, q->p[i].x); lo->y = vmin_(lo->y, q->p[i].y); lo->z = vmin_(lo->z, q->p[i].z);
		hi->x = vmax_(hi->x, q->p[i].x); hi->y = vmax_(hi->y, q->p[i].y); hi->z = vmax_(hi->z, q->p[i].z);
	}
}
static v3 half(v3 a, v3 b) { return mul(add(a, b), 0.5f); }

/* split along u (first half stays in *p) */
static void split_u(patch_t* p, patch_t* s, int nv) {
	if (nv == 4) {
		v3 m01 = half(p->p[0], p->p[1]), m23 = half(p->p[2], p->p[3]);
		s->p[0] = m01; s->p[1] = p->p[1]; s->p[2] = m23; s->p[3] = p->p[3];
		p->p[1] = m01; p->p[3] = m23;
	} else {
		int r;
		for (r = 0; r < 4; ++r) {
			int k = r * 4;
			v3 tmp = half(p->p[k + 1], p->p[k + 2]);
			v3 q3 = p->p[k + 3], q2 = half(p->p[k + 3], p->p[k + 2]), q1 = half(tmp, q2);
			v3 a0 = p->p[k], a1 = half(p->p[k], p->p[k + 1]), a2 = half(tmp, a1), a3 = half(a2, q1);
			s->p[k + 3] = q3; s->p[k + 2] = q2; s->p[k + 1] = q1; s->p[k] = a3;
			p->p[k] = a0; p->p[k + 1] = a1; p->p[k + 2] = a2; p->p[k + 3] = a3;
		}
	}
}
static void split_v(patch_t* p, patch_t* s, int nv) {
	if (nv == 4) {
		v3 m02 = half(p->p[0], p->p[2]), m13 = half(p->p[1], p->p[3]);
		s->p[0] = m02; s->p[1] = m13; s->p[2] = p->p[2]; s->p[3] = p->p[3];
		p->p[2] = m02; p->p[3] = m13;
	} else {
		int c;
		for (c = 0; c < 4; ++c) {
			v3 tmp = half(p->p[c + 4], p->p[c + 8]);
			v3 q3 = p->p[c + 12], q2 = half(p->p[c + 12], p->p[c + 8]), q1 = half(tmp, q2);
			v3 a0 = p->p[c], a1 = half(p->p[c], p->p[c + 4]), a2 = half(tmp, a1), a3 = half(a2, q1);
			s->p[c + 12] = q3; s->p[c + 8] = q2; s->p[c + 4] = q1; s->p[c] = a3;
			p->p[c] = a0; p->p[c + 4] = a1; p->p[c + 8] = a2; p->p[c + 12] = a3;
		}
	}
}

typedef struct { patch_t q[2]; float u0, u1, v0, v1; int depth; } pentry;

/* intersect_rays_with_patch for one ray; returns 1 when a leaf hit was taken */
static int patch_hit(const float* verts, int nv, int tsc, float time, const ray_t* r, float* max_t, int occl,
                     float dice, float minup, float* ht, float* hu, float* hv) {
	pentry* stack = (pentry*)malloc(sizeof(pentry) * 64);
	pentry cur, second;
	int sp = 0, k, found = 0, t_index = 0;
	float t_nalpha = 0.0f;
	for (k = 0; k < tsc && k < 2; ++k) {
		int i;
		for (i = 0; i < nv; ++i) cur.q[k].p[i] = V(verts[(k * nv + i) * 3], verts[(k * nv + i) * 3 + 1], verts[(k * nv + i) * 3 + 2]);
	}
	cur.u0 = 0.0f; cur.u1 = 1.0f; cur.v0 = 0.0f; cur.v1 = 1.0f; cur.depth = 0;
	if (tsc > 1) {
		float tt = time * (float)(tsc - 1);
		t_index = (int)tt;
		t_nalpha = tt - (float)t_index;
		if (t_index > tsc - 2) t_index = tsc - 2;
	}
	for (;;) {
		v3 lo[2], hi[2], blo, bhi;
		float max_dim = 0.0f, h0, h1;
		int h, descend = 0;
		for (k = 0; k < tsc; ++k) {
			float ld;
			pbound(&cur.q[k], nv, &lo[k], &hi[k]);
			ld = longest(sub(hi[k], lo[k]));
			max_dim = (k == 0) ? ld : fmax_std(max_dim, ld);
		}
		if (tsc == 1) { blo = lo[0]; bhi = hi[0]; }
		else {
			float ia = 1.0f - t_nalpha;
			blo = add(mul(lo[t_index], ia), mul(lo[t_index + 1], t_nalpha));
			bhi = add(mul(hi[t_index], ia), mul(hi[t_index + 1], t_nalpha));
		}
		h = box_hit(blo, bhi, r, *max_t, &h0, &h1);
		if (h) {
			float width = fmax_std(min_width(r, h0, h1) * dice, minup);
			if (max_dim <= width || cur.depth == 63) {
				float tt = (h0 + h1) * 0.5f;
				if (tt > 0.0f && tt < *max_t) {
					found = 1;
					if (occl) { free(stack); return 1; }
					*max_t = tt; *ht = tt;
					*hu = (cur.u0 + cur.u1) * 0.5f;
					*hv = (cur.v0 + cur.v1) * 0.5f;
				}
			} else descend = 1;
		}
		if (descend) {
			float ul, vl;
			if (nv == 4) { ul = longest(sub(cur.q[0].p[0], cur.q[0].p[1])); vl = longest(sub(cur.q[0].p[0], cur.q[0].p[2])); }
			else { ul = longest(sub(cur.q[0].p[0], cur.q[0].p[3])); vl = longest(sub(cur.q[0].p[0], cur.q[0].p[12])); }
			if (ul > vl) {
				float um = (cur.u0 + cur.u1) * 0.5f;
				for (k = 0; k < tsc; ++k) split_u(&cur.q[k], &second.q[k], nv);
				second.u0 = um; second.u1 = cur.u1; second.v0 = cur.v0; second.v1 = cur.v1;
				cur.u1 = um;
			} else {
				float vm = (cur.v0 + cur.v1) * 0.5f;
				for (k = 0; k < tsc; ++k) split_v(&cur.q[k], &second.q[k], nv);
				second.u0 = cur.u0; second.u1 = cur.u1; second.v0 = vm; second.v1 = cur.v1;
				cur.v1 = vm;
			}
			second.depth = cur.depth + 1;
			stack[sp++] = cur;
			cur = second;
		} else {
			if (sp == 0) break;
			cur = stack[--sp];
		}
	}
	free(stack);
	return found;
}

/* ------------------------------------------------------------------ */
/* Scene traversal: every instance, recursively, in order. */
#define MAXM 4
typedef struct { int n; m44 m[MAXM]; } frame_t;

typedef struct {
	const psy_scene_desc* sc;
	float dice, minup;
	/* result */
	int hit;
	uint64_t id;
	float t, u, v;
	float max_t;
} tracer_t;

static m44 frame_at(const frame_t* f, float time) {
	int i0, single; float na;
	seqpos(time, f->n, &i0, &single, &na);
	if (single) return f->m[i0];
	return mlerp(na, &f->m[i0], &f->m[i0 + 1]);
}

static m44 seq_at(const float* xs, int n, float time) {
	int i0, single; float na;
	m44 a, b;
	seqpos(time, n, &i0, &single, &na);
	a = mload(xs + 16 * i0);
	if (single) return a;
	b = mload(xs + 16 * (i0 + 1));
	return mlerp(na, &a, &b);
}

/* merge(parent, instance transforms) (math/transform.hpp:241-272) */
static int merge(const frame_t* a, const float* b, int nb, frame_t* d) {
	int na = a->n, i;
	if (na > MAXM || nb > MAXM) return 0;
	if (na == nb) {
		for (i = 0; i < na; ++i) { m44 bb = mload(b + 16 * i); d->m[i] = mmul(&a->m[i], &bb); }
		d->n = na;
	} else if (na > nb) {
		if (nb == 0) for (i = 0; i < na; ++i) d->m[i] = a->m[i];
		else {
			float inv_s = 1.0f / (float)(na - 1);
			for (i = 0; i < na; ++i) { m44 bb = seq_at(b, nb, (float)i * inv_s); d->m[i] = mmul(&a->m[i], &bb); }
		}
		d->n = na;
	} else {
		if (na == 0) for (i = 0; i < nb; ++i) d->m[i] = mload(b + 16 * i);
		else {
			float inv_s = 1.0f / (float)(nb - 1);
			for (i = 0; i < nb; ++i) { m44 bb = mload(b + 16 * i); m44 aa = frame_at(a, (float)i * inv_s); d->m[i] = mmul(&bb, &aa); }
		}
		d->n = nb;
	}
	return 1;
}

static uint32_t upow2(uint32_t v) { v--; v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16; return v + 1; }
static uint32_t ilog2(uint32_t v) { uint32_t r = 0; while (v > 1) { v >>= 1; ++r; } return r; }

static void trace_assembly(tracer_t* T, uint32_t ai, const frame_t* fr, uint64_t idp, const wray_t* w, int depth) {
	const psy_assembly_desc* a = &T->sc->assemblies[ai];
	const int bits = (int)ilog2(upow2(a->instance_count));
	uint32_t i;
	if (depth > 16) return;
	for (i = 0; i < a->instance_count; ++i) {
		const psy_instance_desc* in = &a->instances[i];
		uint64_t id = (idp << bits) | ((uint64_t)i & (uint64_t)(int64_t)((1 << bits) - 1));
		frame_t nf;
		const frame_t* f = fr;
		ray_t r;
		if (in->transform_count > 0) {
			if (!merge(fr, a->transforms + 16 * in->transform_index, (int)in->transform_count, &nf)) continue;
			f = &nf;
		}
		if (in->kind == PSY_INSTANCE_ASSEMBLY) {
			trace_assembly(T, a->children[in->data_index], f, id, w, depth + 1);
			if (T->hit && w->occl) return;
			continue;
		}
		{
			m44 x;
			if (f->n > 0) { x = frame_at(f, w->time); ray_in(&r, w, &x); }
			else ray_in(&r, w, NULL);
		}
		{
			const psy_object_desc* ob = &a->objects[in->data_index];
			const float* p = ob->data;
			int hit = 0;
			float th = 0.0f, hu = 0.0f, hv = 0.0f;
			if (ob->kind == PSY_OBJ_SPHERE || ob->kind == PSY_OBJ_SPHERE_LIGHT) {
				int i0, single; float na, radi, t;
				v3 c;
				if (ob->kind == PSY_OBJ_SPHERE) {
					seqpos(w->time, (int)ob->n0, &i0, &single, &na);
					if (single) { c = V(p[i0 * 4], p[i0 * 4 + 1], p[i0 * 4 + 2]); radi = p[i0 * 4 + 3]; }
					else {
						const float* x0 = p + i0 * 4; const float* x1 = x0 + 4; float ia = 1.0f - na;
						c = add(mul(V(x0[0], x0[1], x0[2]), ia), mul(V(x1[0], x1[1], x1[2]), na));
						radi = lerpf(na, x0[3], x1[3]);
					}
				} else {
					seqpos(w->time, (int)ob->n0, &i0, &single, &na);
					if (single) c = V(p[i0 * 3], p[i0 * 3 + 1], p[i0 * 3 + 2]);
					else { float ia = 1.0f - na; c = add(mul(V(p[i0 * 3], p[i0 * 3 + 1], p[i0 * 3 + 2]), ia), mul(V(p[i0 * 3 + 3], p[i0 * 3 + 4], p[i0 * 3 + 5]), na)); }
					seqpos(w->time, (int)ob->n1, &i0, &single, &na);
					radi = single ? p[ob->n0 * 3 + i0] : lerpf(na, p[ob->n0 * 3 + i0], p[ob->n0 * 3 + i0 + 1]);
				}
				t = sphere_t(&r, c, radi, T->max_t);
				if (t >= 0.0f) { hit = 1; th = t; if (!w->occl) T->max_t = t; }
			} else {
				int nv = ob->kind == PSY_OBJ_BILINEAR ? 4 : 16;
				hit = patch_hit(p, nv, (int)ob->n0, w->time, &r, &T->max_t, w->occl, T->dice, T->minup, &th, &hu, &hv);
			}
			if (hit) {
				T->hit = 1;
				T->id = id;
				if (w->occl) return;
				T->t = th; T->u = hu; T->v = hv;
			}
		}
	}
}

/* Traces n rays (SoA host arrays, psy_ray_soa layout).  Writes hit, id, t, uv. */
int psyport_trace(const psy_scene_desc* sc, const psy_ray_soa* rays, uint32_t n, uint8_t* hit, uint64_t* id,
                  float* t, float* uv) {
	uint32_t i;
	for (i = 0; i < n; ++i) {
		tracer_t T;
		wray_t w;
		frame_t root;
		int k;
		memset(&T, 0, sizeof(T));
		T.sc = sc;
		T.dice = sc->dice_rate;
		T.minup = sc->min_upoly_size;
		for (k = 0; k < 3; ++k) {
			(&w.o.x)[k] = rays->o[3 * i + k]; (&w.d.x)[k] = rays->d[3 * i + k];
			(&w.odx.x)[k] = rays->odx[3 * i + k]; (&w.ody.x)[k] = rays->ody[3 * i + k];
			(&w.ddx.x)[k] = rays->ddx[3 * i + k]; (&w.ddy.x)[k] = rays->ddy[3 * i + k];
		}
		w.time = rays->time[i];
		w.occl = rays->type ? (rays->type[i] == 32) : 0;
		T.max_t = w.occl ? 1.0f : INFINITY;
		T.t = INFINITY;
		root.n = 0;
		trace_assembly(&T, 0, &root, 0, &w, 0);
		hit[i] = (uint8_t)T.hit;
		id[i] = T.hit ? T.id : 0;
		t[i] = (T.hit && !w.occl) ? T.t : INFINITY;
		if (uv) { uv[2 * i] = T.hit ? T.u : 0.0f; uv[2 * i + 1] = T.hit ? T.v : 0.0f; }
	}
	return 0;
}

/* BBox::intersect_ray for one box and ray (inverse direction from 1/d). */
int psyport_box_hit(const float* lo, const float* hi, const float* o, const float* d, float tmax, float* t0, float* t1) {
	ray_t r;
	memset(&r, 0, sizeof(r));
	r.o = V(o[0], o[1], o[2]);
	r.d = V(d[0], d[1], d[2]);
	r.dinv = V(1.0f / d[0], 1.0f / d[1], 1.0f / d[2]);
	return box_hit(V(lo[0], lo[1], lo[2]), V(hi[0], hi[1], hi[2]), &r, tmax, t0, t1);
}

/* InstanceID::push_back (basics/instance_id.hpp:18-23). */
uint64_t psyport_id_push(uint64_t id, uint64_t sub, int bits) {
	return (id << bits) | (sub & (uint64_t)(int64_t)((1 << bits) - 1));
}

/*
 * The host C library's float math as the reference calls it (std::sin and
 * std::cos of one float become sincosf under GCC; std::acos, std::asin and
 * std::exp of a float become acosf, asinf and expf), evaluated over an
 * array: fn 0 sin, 1 cos, 2 acos, 3 asin, 4 exp.
 */
void sincosf(float x, float* s, float* c);
int psyport_libm(int fn, uint32_t n, const float* x, float* out) {
	for (uint32_t i = 0; i < n; ++i) {
		float s, c;
		switch (fn) {
			case 0: sincosf(x[i], &s, &c); out[i] = s; break;
			case 1: sincosf(x[i], &s, &c); out[i] = c; break;
			case 2: out[i] = acosf(x[i]); break;
			case 3: out[i] = asinf(x[i]); break;
			case 4: out[i] = expf(x[i]); break;
			default: return -1;
		}
	}
	return 0;
}
