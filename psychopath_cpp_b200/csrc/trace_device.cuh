/*
 * Device-side ray traversal of the uploaded scene: one ray per thread.
 *
 * The reference traces ray *streams* breadth-first (accel/bvh4.cpp:163-236,
 * object/patch_utils.hpp:18-200); every per-ray decision there depends only
 * on that ray's own state, so a depth-first per-ray walk that keeps the
 * reference's tests and its max_t updates returns the same closest hit.  The
 * one order-dependent case, two candidates at exactly the same t, resolves
 * to whichever is found first; child boxes are visited nearest-first here.
 *
 * Per-ray state: the ray in the current instance space, a node stack,
 * a level stack for nested assemblies (element id prefix, inherited shader,
 * merged motion transforms, as the reference's xform_stack /
 * surface_shader_stack / element_id, tracer/tracer.cpp:125-219), and the
 * path bits of the patch bisection (PatchWork, patch_run).
 */
#ifndef PSY_TRACE_DEVICE_CUH
#define PSY_TRACE_DEVICE_CUH

#include "psy_math.h"
#include "psy_scene.h"

namespace psy {

#define PSY_NODE_STACK 64
#define PSY_MAX_LEVELS 8
#define PSY_MAX_MOTION 4
#define PSY_SPLIT_STACK 64


struct WorldRayD {
	V3 o, d, odx, ody, ddx, ddy;
	float time;
	bool occl;
};

// Ray in the current instance space (Ray, basics/ray.hpp:24-37).  Its
// width parameters are kept apart (ray_width_of): only patch leaves need
// them, so they are computed on first use in each space.
struct LocalRay {
	V3 o, d, dinv;
};

__device__ __forceinline__ M44 load_m44_dev(const float* p) {
	M44 m;
	const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
	for (int r = 0; r < 4; ++r) {
		const float4 v = __ldg(q + r);
		m.m[r][0] = v.x;
		m.m[r][1] = v.y;
		m.m[r][2] = v.z;
		m.m[r][3] = v.w;
	}
	return m;
}

// WorldRay::update_ray (basics/ray.hpp:207-305): with and without transform.
__device__ __forceinline__ LocalRay make_local(const WorldRayD& wr) {
	LocalRay r;
	r.o = wr.o;
	r.d = wr.d;
	r.dinv = recip3(r.d);
	return r;
}

__device__ __forceinline__ LocalRay make_local_x(const WorldRayD& wr, const M44& t) {
	LocalRay r;
	r.o = pos_to(t, wr.o);
	r.d = dir_to(t, wr.d);
	r.dinv = recip3(r.d);
	return r;
}

// The width parameters update_ray computes beside the local ray `r` (made
// from wr with transform t, or none).  Computed once per space a ray meets
// a patch in.
__device__ __forceinline__ RayWidth ray_width_of(const WorldRayD& wr, const LocalRay& r, const M44* t) {
	if (!t) return ray_width_params(r.o, r.d, wr.odx, wr.ody, wr.ddx, wr.ddy);
	return ray_width_params(r.o, r.d, dir_to(*t, wr.odx), dir_to(*t, wr.ody), dir_to(*t, wr.ddx), dir_to(*t, wr.ddy));
}

// Merged motion-transform sequence of a level (the reference's xform_stack frame).
struct Frame {
	int count;  // 0 = no transform (identity)
	M44 m[PSY_MAX_MOTION];
};

__device__ __forceinline__ M44 frame_at_index_lerp(const Frame& f, float alpha) {
	const SeqPos sp = seq_pos(alpha, f.count);
	if (sp.single) return f.m[sp.i0];
	return m44_lerp(sp.nalpha, f.m[sp.i0], f.m[sp.i0 + 1]);
}

__device__ __forceinline__ M44 seq_lerp_global(const float* xs, int count, float alpha) {
	const SeqPos sp = seq_pos(alpha, count);
	if (sp.single) return load_m44_dev(xs + 16 * sp.i0);
	return m44_lerp(sp.nalpha, load_m44_dev(xs + 16 * sp.i0), load_m44_dev(xs + 16 * (sp.i0 + 1)));
}

// merge() of transform sequences (math/transform.hpp:241-272): parent `a`
// with instance transforms `b` (global, count nb), written into `dst`.
// Returns false if the result needs more than PSY_MAX_MOTION samples.  The
// three cases of the reference (equal counts, more parent samples, more
// instance samples) share one loop with one matrix product.  (Outlined, so
// that its frames pass through memory, this and the other traversal helpers
// cost 11% of the many-light render's traversal time.)
__device__ __forceinline__ bool frame_merge(const Frame& a, const float* b, int nb, Frame* dst) {
	const int na = a.count;
	if (na > PSY_MAX_MOTION || nb > PSY_MAX_MOTION) return false;
	const int n = na > nb ? na : nb;
	const float inv_s = n > 1 ? 1.0f / (float)(n - 1) : 0.0f;
#pragma unroll 1
	for (int i = 0; i < n; ++i) {
		M44 r;
		if (na == nb) {
			r = m44_mul(a.m[i], load_m44_dev(b + 16 * i));
		} else if (na > nb) {
			if (nb == 0) r = a.m[i];
			else r = m44_mul(a.m[i], seq_lerp_global(b, nb, (float)i * inv_s));
		} else {
			// the reference multiplies instance * lerped-parent in this case
			if (na == 0) r = load_m44_dev(b + 16 * i);
			else r = m44_mul(load_m44_dev(b + 16 * i), frame_at_index_lerp(a, (float)i * inv_s));
		}
		dst->m[i] = r;
	}
	dst->count = n;
	return true;
}

// ---------------------------------------------------------------------
// Sphere / sphere light intersection (object/sphere.cpp:67-189,
// lights/sphere_light.hpp:159-246): returns the hit t or -1.
// ---------------------------------------------------------------------
__device__ __forceinline__ float sphere_t(V3 ro, V3 rd, V3 cent, float radi, float max_t) {
	const V3 o = ro - cent;
	const V3 d = rd;
	const float a = length2(d);
	const float b = 2.0f * dot(d, o);
	const float c = length2(o) - radi * radi;
	float disc = b * b - 4.0f * a * c;
	if (disc < 0.0f) return -1.0f;
	disc = sqrtf(disc);
	float q;
	if (b < 0.0f) q = -0.5f * (b - disc);
	else q = -0.5f * (b + disc);
	float t0 = q / a;
	float t1;
	if (q != 0.0f) t1 = c / q;
	else t1 = max_t;
	if (t0 > t1) {
		const float tmp = t1;
		t1 = t0;
		t0 = tmp;
	}
	if (t0 >= max_t || t1 < 0.0001f) return -1.0f;
	if (t0 >= 0.0001f) return t0;
	if (t1 < max_t) return t1;
	return -1.0f;
}

__device__ __forceinline__ void sphere_at(const DevScene& sc, const DevObject& ob, float time, V3* cent, float* radi) {
	const float* p = sc.fpool + ob.data;
	const SeqPos sp = seq_pos(time, ob.n0);
	if (sp.single) {
		*cent = V3(p[sp.i0 * 4], p[sp.i0 * 4 + 1], p[sp.i0 * 4 + 2]);
		*radi = p[sp.i0 * 4 + 3];
	} else {
		const float* a = p + sp.i0 * 4;
		const float* b = a + 4;
		*cent = lerp3(sp.nalpha, V3(a[0], a[1], a[2]), V3(b[0], b[1], b[2]));
		*radi = lerp1(sp.nalpha, a[3], b[3]);
	}
}

__device__ __forceinline__ void light_at(const DevScene& sc, const DevObject& ob, float time, V3* pos, float* radi,
                                         float col[3]) {
	const float* p = sc.fpool + ob.data;
	{
		const SeqPos sp = seq_pos(time, ob.n0);
		const float* a = p + sp.i0 * 3;
		if (sp.single) *pos = V3(a[0], a[1], a[2]);
		else *pos = lerp3(sp.nalpha, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]));
	}
	const float* rp = p + ob.n0 * 3;
	{
		const SeqPos sp = seq_pos(time, ob.n1);
		if (sp.single) *radi = rp[sp.i0];
		else *radi = lerp1(sp.nalpha, rp[sp.i0], rp[sp.i0 + 1]);
	}
	const float* cp = rp + ob.n1;
	{
		const SeqPos sp = seq_pos(time, ob.n2);
		const float* a = cp + sp.i0 * 3;
		if (sp.single) {
			col[0] = a[0]; col[1] = a[1]; col[2] = a[2];
		} else {
			const float ia = one_minus(sp.nalpha);
			for (int k = 0; k < 3; ++k) col[k] = (a[k] * ia) + (a[3 + k] * sp.nalpha);
		}
	}
}

// RectangleLight's dimensions and colour at `time` (lerp_seq over each
// sequence, lights/rectangle_light.hpp:44-46).
__device__ __forceinline__ void rect_light_at(const DevScene& sc, const DevObject& ob, float time, float* dx, float* dy,
                                              float col[3]) {
	const float* p = sc.fpool + ob.data;
	{
		const SeqPos sp = seq_pos(time, ob.n0);
		const float* a = p + sp.i0 * 2;
		if (sp.single) {
			*dx = a[0];
			*dy = a[1];
		} else {
			// std::pair's operator* takes a float: (1 - alpha) is narrowed first
			const float ia = one_minus(sp.nalpha);
			*dx = (a[0] * ia) + (a[2] * sp.nalpha);
			*dy = (a[1] * ia) + (a[3] * sp.nalpha);
		}
	}
	if (col) {
		const float* cp = p + ob.n0 * 2;
		const SeqPos sp = seq_pos(time, ob.n1);
		const float* a = cp + sp.i0 * 3;
		if (sp.single) {
			col[0] = a[0]; col[1] = a[1]; col[2] = a[2];
		} else {
			const float ia = one_minus(sp.nalpha);
			for (int k = 0; k < 3; ++k) col[k] = (a[k] * ia) + (a[3 + k] * sp.nalpha);
		}
	}
}

// RectangleLight::intersect_ray's hit test (lights/rectangle_light.hpp:
// 106-121): the plane z = 0 of the light's space, inside the rectangle.
// The upper y bound is dimension x / 2, as the reference has it.  Returns t
// or -1.
__device__ __forceinline__ float rect_light_t(V3 o, V3 d, V3 dinv, float dx, float dy, float max_t) {
	if (d.z == 0.0f) return -1.0f;
	const float t = -o.z * dinv.z;
	if (t <= 0.0f || t > max_t) return -1.0f;
	const float x = o.x + (d.x * t);
	const float y = o.y + (d.y * t);
	if (x >= (dx * -0.5f) && x <= (dx * 0.5f) && y >= (dy * -0.5f) && y <= (dx * 0.5f)) return t;
	return -1.0f;
}

// ---------------------------------------------------------------------
// Patches (object/bilinear.hpp, object/bicubic.hpp)
// ---------------------------------------------------------------------
template <int NV>
struct Patch {
	V3 p[NV];
};

template <int NV>
__device__ __forceinline__ Box patch_bound(const Patch<NV>& q) {
	Box b;
	b.lo = q.p[0];
	b.hi = q.p[0];
#pragma unroll
	for (int i = 1; i < NV; ++i) {
		b.lo = vmin3(b.lo, q.p[i]);
		b.hi = vmax3(b.hi, q.p[i]);
	}
	return b;
}

__device__ __forceinline__ float patch_ulen(const Patch<4>& q) { return longest_axis(q.p[0] - q.p[1]); }
__device__ __forceinline__ float patch_vlen(const Patch<4>& q) { return longest_axis(q.p[0] - q.p[2]); }
__device__ __forceinline__ float patch_ulen(const Patch<16>& q) { return longest_axis(q.p[0] - q.p[3]); }
__device__ __forceinline__ float patch_vlen(const Patch<16>& q) { return longest_axis(q.p[0] - q.p[12]); }

template <int NV>
__device__ __forceinline__ void patch_load(const float* src, Patch<NV>* q) {
#pragma unroll
	for (int i = 0; i < NV; ++i) q->p[i] = V3(__ldg(src + i * 3), __ldg(src + i * 3 + 1), __ldg(src + i * 3 + 2));
}

// Result of a patch leaf hit, consumed by the shading epilogue.
struct PatchHit {
	float t, u, v, max_dim;
};

// Splits of a patch at the middle of u or v (Bilinear::split_u / split_v,
// object/bilinear.hpp:59-82; Bicubic::split_u / split_v, de Casteljau at 0.5
// per row or column, object/bicubic.hpp:74-108), with the reference's float
// operations.  patch_split leaves the second half in `p` and writes the
// first half to `f`; patch_half_u / patch_half_v keep one half in place and
// give the same values for it.
__device__ __forceinline__ void patch_split(Patch<4>& p, Patch<4>& f, bool along_u) {
	if (along_u) {
		const V3 m01 = (p.p[0] + p.p[1]) * 0.5f;
		const V3 m23 = (p.p[2] + p.p[3]) * 0.5f;
		f.p[0] = p.p[0];
		f.p[1] = m01;
		f.p[2] = p.p[2];
		f.p[3] = m23;
		p.p[0] = m01;
		p.p[2] = m23;
	} else {
		const V3 m02 = (p.p[0] + p.p[2]) * 0.5f;
		const V3 m13 = (p.p[1] + p.p[3]) * 0.5f;
		f.p[0] = p.p[0];
		f.p[1] = p.p[1];
		f.p[2] = m02;
		f.p[3] = m13;
		p.p[0] = m02;
		p.p[1] = m13;
	}
}
__device__ __forceinline__ void patch_half_u(Patch<4>& p, bool second) {
	const V3 m01 = (p.p[0] + p.p[1]) * 0.5f;
	const V3 m23 = (p.p[2] + p.p[3]) * 0.5f;
	if (second) {
		p.p[0] = m01;
		p.p[2] = m23;
	} else {
		p.p[1] = m01;
		p.p[3] = m23;
	}
}
__device__ __forceinline__ void patch_half_v(Patch<4>& p, bool second) {
	const V3 m02 = (p.p[0] + p.p[2]) * 0.5f;
	const V3 m13 = (p.p[1] + p.p[3]) * 0.5f;
	if (second) {
		p.p[0] = m02;
		p.p[1] = m13;
	} else {
		p.p[2] = m02;
		p.p[3] = m13;
	}
}

// One de Casteljau split at 0.5 of the control points a,b,c,d of a row or a
// column: a..d become the second half, fa..fd the first.
__device__ __forceinline__ void bezier_split(V3& a, V3& b, V3& c, V3& d, V3& fa, V3& fb, V3& fc, V3& fd) {
	const V3 tmp = (b + c) * 0.5f;
	const V3 q2 = (d + c) * 0.5f;
	const V3 q1 = (tmp + q2) * 0.5f;
	const V3 a1 = (a + b) * 0.5f;
	const V3 a2 = (tmp + a1) * 0.5f;
	const V3 a3 = (a2 + q1) * 0.5f;
	fa = a;
	fb = a1;
	fc = a2;
	fd = a3;
	a = a3;
	b = q1;
	c = q2;
}
// The same split keeping one half in place.
__device__ __forceinline__ void bezier_half(V3& a, V3& b, V3& c, V3& d, bool second) {
	const V3 tmp = (b + c) * 0.5f;
	const V3 q2 = (d + c) * 0.5f;
	const V3 q1 = (tmp + q2) * 0.5f;
	const V3 a1 = (a + b) * 0.5f;
	const V3 a2 = (tmp + a1) * 0.5f;
	const V3 a3 = (a2 + q1) * 0.5f;
	if (second) {
		a = a3;
		b = q1;
		c = q2;
	} else {
		b = a1;
		c = a2;
		d = a3;
	}
}
__device__ __forceinline__ void patch_split(Patch<16>& p, Patch<16>& f, bool along_u) {
	if (along_u) {
#pragma unroll
		for (int r = 0; r < 4; ++r)
			bezier_split(p.p[r * 4], p.p[r * 4 + 1], p.p[r * 4 + 2], p.p[r * 4 + 3], f.p[r * 4], f.p[r * 4 + 1],
			             f.p[r * 4 + 2], f.p[r * 4 + 3]);
	} else {
#pragma unroll
		for (int c = 0; c < 4; ++c)
			bezier_split(p.p[c], p.p[c + 4], p.p[c + 8], p.p[c + 12], f.p[c], f.p[c + 4], f.p[c + 8], f.p[c + 12]);
	}
}
__device__ __forceinline__ void patch_half_u(Patch<16>& p, bool second) {
#pragma unroll
	for (int r = 0; r < 4; ++r) bezier_half(p.p[r * 4], p.p[r * 4 + 1], p.p[r * 4 + 2], p.p[r * 4 + 3], second);
}
__device__ __forceinline__ void patch_half_v(Patch<16>& p, bool second) {
#pragma unroll
	for (int c = 0; c < 4; ++c) bezier_half(p.p[c], p.p[c + 4], p.p[c + 8], p.p[c + 12], second);
}

// The 24 floats of a BBox4 record (six 128-bit loads).
__device__ __forceinline__ void load_box4(const float4* q, float* b) {
#pragma unroll
	for (int i = 0; i < 6; ++i) {
		const float4 v = __ldg(q + i);
		b[i * 4 + 0] = v.x;
		b[i * 4 + 1] = v.y;
		b[i * 4 + 2] = v.z;
		b[i * 4 + 3] = v.w;
	}
}

// Path of a node in the bisection tree: one bit per split level.
struct Bits128 {
	uint64_t lo, hi;
	__device__ __forceinline__ bool get(int i) const { return i < 64 ? ((lo >> i) & 1ull) : ((hi >> (i - 64)) & 1ull); }
	__device__ __forceinline__ void set(int i, bool v) {
		if (i < 64) lo = v ? (lo | (1ull << i)) : (lo & ~(1ull << i));
		else hi = v ? (hi | (1ull << (i - 64))) : (hi & ~(1ull << (i - 64)));
	}
	// keep bits [0, n)
	__device__ __forceinline__ void truncate(int n) {
		if (n <= 0) { lo = 0; hi = 0; }
		else if (n < 64) { lo &= (1ull << n) - 1ull; hi = 0; }
		else if (n < 128) { hi &= (1ull << (n - 64)) - 1ull; }
	}
	// highest set bit below n, or -1
	__device__ __forceinline__ int highest_below(int n) const {
		Bits128 t = *this;
		t.truncate(n);
		if (t.hi) return 64 + 63 - __clzll((long long)t.hi);
		if (t.lo) return 63 - __clzll((long long)t.lo);
		return -1;
	}
	__device__ __forceinline__ int popc() const { return __popcll(lo) + __popcll(hi); }
};

// Bounds of a sub-patch (each time sample) and the ray's test against them:
// the top of the loop of intersect_rays_with_patch (object/patch_utils.hpp).
template <int NV, int TSC>
__device__ __forceinline__ bool patch_node_test(const Patch<NV> (&q)[TSC], float t_nalpha, const LocalRay& r,
                                                float max_t, float* max_dim, float* h0, float* h1) {
	Box bb[TSC];
	float md = 0.0f;
#pragma unroll
	for (int k = 0; k < TSC; ++k) {
		bb[k] = patch_bound<NV>(q[k]);
		const float ld = longest_axis(bb[k].hi - bb[k].lo);
		md = (k == 0) ? ld : smax(md, ld);
	}
	*max_dim = md;
	const bool h = (TSC == 1) ? box_hit(bb[0], r.o, r.dinv, max_t, h0, h1)
	                          : box_hit(box_lerp(t_nalpha, bb[0], bb[TSC - 1]), r.o, r.dinv, max_t, h0, h1);
	// A NaN far distance comes from 0 * inf: the ray runs exactly along a
	// box face (a zero direction component, the origin on the face).  The
	// reference's std::min/max slab test then reports a hit with h0 = 0 and
	// h1 = NaN, and every sub-box is again NaN or a plain miss, so none of
	// the subtree's leaves can be taken (their t = (h0 + h1) / 2 is NaN)
	// while the reference still walks all of it, millions of nodes deep
	// for a camera ray through the image centre.  Treating it as a miss
	// gives the same hits.
	return h && !(*h1 != *h1);
}

// Pending first halves a bisection can hold: at most one per second half
// on the path, and the path has at most PSY_SPLIT_STACK - 1 of those.
#define PSY_PATCH_PEND PSY_SPLIT_STACK

// Per-ray bisection of one patch with TSC time samples (TSC = 1 or 2):
// intersect_rays_with_patch for a single ray (object/patch_utils.hpp:18-200).
//
// The reference walks the split tree depth first with a stack of sub-patches:
// a split pushes the first half, then the second, and the second half is
// processed first.  Here both halves are tested against the ray when they
// are made.  The second half is entered if its box is hit; the first half
// is entered at once if only its box is hit, pushed on a stack of pending
// first halves (control points and uv range) if both are, and dropped if
// its box is missed (box_hit only gets stricter as the ray's max t
// shrinks, so the reference would find it missed later as well).  When a
// subtree ends, the deepest pending first half is popped and tested again
// with the current max t.  The stack holds only the halves that are
// pending, so it is written once per split that hits both halves; the path
// bits (1 = second half) give the reference's stack index (its forced leaf
// at 63: the population count of the path) and the depth to resume at.
// Control points and uv ranges are those of the reference's walk, so the
// visiting order and the leaf results are the same.
//
// The bisection can stop after any number of loop iterations and resume
// later from its cursor (the node at the top of the loop, whose box the ray
// hits, with its path bits and uv range) and its stack, so that a lane can
// leave a long bisection to run with the other lanes of its warp.
// patch_run works on a cursor the caller holds as a local (kept in
// registers) and copies back only when it stops short of the end.
template <int NV, int TSC>
struct PatchCursor {
	Patch<NV> cur[TSC];        // the node at the top of the loop
	Bits128 path, dirs, pend;  // dirs bit: 1 = split along u
	int depth;                 // splits from the root
	float u0, u1, v0, v1;
	float t_nalpha, max_dim, h0, h1;
	bool found;
	unsigned steps;  // loop iterations taken (bounded: PSY_PATCH_MAX_STEPS)
	int sp;          // pending first halves on the stack
};

// A bisection ends with an error (ERRF_BISECT) after this many loop
// iterations.  The walk is finite (a leaf is forced at 63 second halves or
// depth 127), but a ray the reference would bisect for hours must not hold
// a wave: far above any bisection of a real scene.
#define PSY_PATCH_MAX_STEPS (1u << 24)

// Sub-patches stored on the current path (with their uv ranges).
template <int NV, int TSC>
struct PatchStore {
	Patch<NV> pend[PSY_PATCH_PEND][TSC];
	float penduv[PSY_PATCH_PEND][4];
};

// A suspended bisection in a lane's traversal state.
template <int NV, int TSC>
struct PatchWork {
	PatchCursor<NV, TSC> c;
	PatchStore<NV, TSC> st;
};

// The root's test: sets up `pc` and returns true when the ray hits the
// patch's box.
template <int NV, int TSC>
__device__ __forceinline__ bool patch_begin(PatchCursor<NV, TSC>& pc, const float* verts, float time,
                                            const LocalRay& r, float max_t) {
#pragma unroll
	for (int k = 0; k < TSC; ++k) patch_load<NV>(verts + k * NV * 3, &pc.cur[k]);
	pc.t_nalpha = 0.0f;
	if (TSC > 1) {
		// bounds are lerped between the two samples; time == 1.0 would index
		// past the last sample in the reference (undefined) and gives the
		// first sample's bounds here
		const float t_time = time * (float)(TSC - 1);
		pc.t_nalpha = t_time - (float)(int)t_time;
	}
	if (!patch_node_test<NV, TSC>(pc.cur, pc.t_nalpha, r, max_t, &pc.max_dim, &pc.h0, &pc.h1)) return false;
	pc.path = Bits128{0, 0};
	pc.dirs = Bits128{0, 0};
	pc.pend = Bits128{0, 0};
	pc.depth = 0;
	pc.u0 = 0.0f;
	pc.u1 = 1.0f;
	pc.v0 = 0.0f;
	pc.v1 = 1.0f;
	pc.found = false;
	pc.steps = 0;
	pc.sp = 0;
	return true;
}

// Runs up to `units` iterations of the bisection loop (a leaf test or a
// split, with the resume that follows it).  Returns true when the
// bisection has ended; pc.found then says whether a leaf was taken (the
// closest one in *hit, with *max_t lowered to it; for occlusion rays the
// first one).  Otherwise `pc` is the node to carry on from.  A bisection
// that exceeds PSY_PATCH_MAX_STEPS iterations ends without a hit and sets
// ERRF_BISECT in *err.
template <int NV, int TSC>
__device__ __forceinline__ bool patch_run(PatchCursor<NV, TSC>& pc, PatchStore<NV, TSC>& ps, const float* verts,
                                          const LocalRay& r, const RayWidth& rw, float* max_t, bool occl,
                                          float dice_rate, float min_upoly, PatchHit* hit, int& units,
                                          unsigned* err) {
	Patch<NV>(&cur)[TSC] = pc.cur;
	const float t_nalpha = pc.t_nalpha;
	float &max_dim = pc.max_dim, &h0 = pc.h0, &h1 = pc.h1;
	Bits128 &path = pc.path, &dirs = pc.dirs, &pend = pc.pend;
	int& depth = pc.depth;
	float &u0 = pc.u0, &u1 = pc.u1, &v0 = pc.v0, &v1 = pc.v1;
	bool& found = pc.found;
	while (true) {
		if (units == 0) return false;
		--units;
		if (++pc.steps > PSY_PATCH_MAX_STEPS) {
			found = false;
			*err |= ERRF_BISECT;
			return true;
		}
		// `cur` is a node whose box the ray hits; max_dim, h0, h1 are its test
		// A NaN width (from NaN ray differentials: a grazing hit makes the
		// next ray's origin differentials 0/0 in transfer_ray_origin_
		// differential, basics/differential_geometry.hpp:85-98) survives the
		// reference's std::max, no sub-patch is ever small enough, and its
		// bisection does not end.  Here it counts as zero width: the leaves
		// stop at min_upoly, as for a ray with zero differentials.
		const float wm = ray_min_width(rw, h0, h1) * dice_rate;
		const float width = (wm != wm) ? min_upoly : smax(wm, min_upoly);
		bool entered = false;
		if (max_dim <= width || path.popc() == PSY_SPLIT_STACK - 1 || depth == 127) {
			const float tt = (h0 + h1) * 0.5f;
			if (tt > 0.0f && tt < *max_t) {
				found = true;
				if (occl) return true;
				*max_t = tt;
				hit->t = tt;
				hit->u = (u0 + u1) * 0.5f;
				hit->v = (v0 + v1) * 0.5f;
				hit->max_dim = max_dim;
			}
		} else {
			const bool along_u = patch_ulen(cur[0]) > patch_vlen(cur[0]);
			Patch<NV> first[TSC];
#pragma unroll
			for (int k = 0; k < TSC; ++k) patch_split(cur[k], first[k], along_u);
			float smd, sh0, sh1, fmd, fh0, fh1;
			const bool s_hit = patch_node_test<NV, TSC>(cur, t_nalpha, r, *max_t, &smd, &sh0, &sh1);
			const bool f_hit = patch_node_test<NV, TSC>(first, t_nalpha, r, *max_t, &fmd, &fh0, &fh1);
			dirs.set(depth, along_u);
			const float mid = along_u ? (u0 + u1) * 0.5f : (v0 + v1) * 0.5f;
			if (s_hit) {
				path.set(depth, true);
				pend.set(depth, f_hit);
				if (f_hit) {
					// the first half waits on the stack with its uv range
					const int q = pc.sp++;
#pragma unroll
					for (int k = 0; k < TSC; ++k) ps.pend[q][k] = first[k];
					ps.penduv[q][0] = u0;
					ps.penduv[q][1] = along_u ? mid : u1;
					ps.penduv[q][2] = v0;
					ps.penduv[q][3] = along_u ? v1 : mid;
				}
				if (along_u) u0 = mid; else v0 = mid;
				max_dim = smd;
				h0 = sh0;
				h1 = sh1;
				entered = true;
			} else if (f_hit) {
				path.set(depth, false);
#pragma unroll
				for (int k = 0; k < TSC; ++k) cur[k] = first[k];
				if (along_u) u1 = mid; else v1 = mid;
				max_dim = fmd;
				h0 = fh0;
				h1 = fh1;
				entered = true;
			}
			if (entered) {
				++depth;
				continue;
			}
		}
		// resume at the deepest pending first half (the top of the stack)
		// whose box is still hit
		while (true) {
			const int j = pend.highest_below(depth);
			if (j < 0) return true;
			pend.set(j, false);
			path.set(j, false);
			depth = j + 1;
			path.truncate(depth);
			dirs.truncate(depth);
			pend.truncate(depth);
			const int q = --pc.sp;
#pragma unroll
			for (int k = 0; k < TSC; ++k) cur[k] = ps.pend[q][k];
			u0 = ps.penduv[q][0]; u1 = ps.penduv[q][1]; v0 = ps.penduv[q][2]; v1 = ps.penduv[q][3];
			if (patch_node_test<NV, TSC>(cur, t_nalpha, r, *max_t, &max_dim, &h0, &h1)) break;
		}
	}
}

// The whole bisection of one patch in one call, its state in the caller's
// frame.  Returns true when a leaf was taken.
template <int NV, int TSC>
__device__ bool patch_whole(const float* verts, float time, const LocalRay& r, const RayWidth& rw,
                                            float* max_t, bool occl, float dice_rate, float min_upoly,
                                            PatchHit* hit, unsigned* err) {
	PatchCursor<NV, TSC> pc;
	PatchStore<NV, TSC> ps;
	if (!patch_begin<NV, TSC>(pc, verts, time, r, *max_t)) return false;
	int units = 0x7fffffff;
	patch_run<NV, TSC>(pc, ps, verts, r, rw, max_t, occl, dice_rate, min_upoly, hit, units, err);
	return pc.found;
}

// ---------------------------------------------------------------------
// Whole-scene traversal
// ---------------------------------------------------------------------
struct HitRec {
	float t;
	float u, v, max_dim;
	int obj;          // global object index, -1 = miss
	int kind;
	int shader;       // innermost bound shader, -1 = none
	uint64_t id;
	int depth;        // number of instances on the path
	int path[PSY_MAX_LEVELS];  // global instance indices, root first
};

struct Level {
	int asmb;
	int stack_base;
	int shader;
	int inst;         // global instance that entered this level (-1 for the root)
	uint64_t id;
	int id_bits;      // id bits of this level's assembly
	int inst_base;
};

// Patch kind of a bisection in progress: bilinear or bicubic, one or two
// time samples.
enum : int { PM_NONE = 0, PM_BILINEAR1, PM_BILINEAR2, PM_BICUBIC1, PM_BICUBIC2 };

// Bytes of the bisection state for the patch kinds of feature set F.
template <unsigned F>
struct PatchBuf {
	static constexpr int TS = (F & FEAT_PATCH_MOTION) ? 2 : 1;
	static constexpr size_t b4 = (F & FEAT_BILINEAR) ? sizeof(PatchWork<4, TS>) : 0;
	static constexpr size_t b16 = (F & FEAT_BICUBIC) ? sizeof(PatchWork<16, TS>) : 0;
	static constexpr size_t m = b4 > b16 ? b4 : b16;
	static constexpr size_t bytes = m > 16 ? m : 16;
};

// Traversal state of one ray.  trace_init sets it up.  A lane that runs
// its ray alone calls trace_step (to the next object leaf and its test)
// until it returns false; the wave kernels advance it in pieces instead
// (walk_nodes, leaf_visit, patch_step, each returning false once the ray
// is finished).  rec and err then hold the result.  Kernels can refill a
// lane with a new ray between pieces.
template <unsigned F>
struct TraceState {
	WorldRayD wr;
	float max_t;
	unsigned err;
	HitRec rec;
	Level lv[PSY_MAX_LEVELS];
	Frame frames[PSY_MAX_LEVELS];   // merged frames of transformed levels
	int lvl_frame[PSY_MAX_LEVELS];  // frame used by each level, -1 = none
	LocalRay lvr[PSY_MAX_LEVELS];   // ray of each enclosing level, kept while a transformed child is traversed
	int node_stack[PSY_NODE_STACK];
	int nsp, L;
	int leaf;                       // leaf popped by walk_nodes, for leaf_visit
	LocalRay r;                     // the ray in the current level's space
	RayWidth rw;                    // width parameters of r, valid when rw_ok
	bool rw_ok;
	// a patch leaf whose bisection is in progress (pmode != PM_NONE): its
	// vertices, ray and widths, the hit record's fields, the bisection
	int pmode;
	int p_obj, p_kind, p_shader, p_gi;
	uint64_t p_id;
	const float* pverts;
	LocalRay pr;
	RayWidth prw;
	PatchHit ph;
	alignas(16) unsigned char pbuf[PatchBuf<F>::bytes];
	template <int NV, int TSC>
	__device__ __forceinline__ PatchWork<NV, TSC>& work() {
		static_assert(sizeof(PatchWork<NV, TSC>) <= sizeof(pbuf), "patch work buffer");
		return *reinterpret_cast<PatchWork<NV, TSC>*>(pbuf);
	}
};

// F is a mask of FEAT_* scene features; code for absent features is not
// compiled into the variant, which keeps the flat-scene kernels small.
template <unsigned F>
__device__ __forceinline__ void trace_init(const DevScene& sc, TraceState<F>& s, const WorldRayD& wr) {
	s.wr = wr;
	s.err = 0;
	s.max_t = wr.occl ? 1.0f : INFINITY;
	s.rec.obj = -1;
	s.rec.t = INFINITY;
	s.rec.depth = 0;
	s.nsp = 0;
	s.L = 0;
	s.lv[0].asmb = 0;
	s.lv[0].stack_base = 0;
	s.lv[0].shader = -1;
	s.lv[0].inst = -1;
	s.lv[0].id = 0;
	s.lv[0].id_bits = sc.assemblies[0].id_bits;
	s.lv[0].inst_base = sc.assemblies[0].inst_base;
	s.lvl_frame[0] = -1;
	s.r = make_local(wr);
	s.rw_ok = false;
	s.pmode = PM_NONE;
	const int root = sc.assemblies[0].root;
	if (root != REF_EMPTY) s.node_stack[s.nsp++] = root;
}

// Records the hit on an object of the current level (Intersection fields
// the traversal knows).  Returns false when the ray is finished: an
// occlusion ray stops at its first hit.
template <unsigned F>
__device__ __forceinline__ bool trace_record(TraceState<F>& s, int obj, int kind, uint64_t id, int shader, int gi,
                                             const PatchHit& ph) {
	HitRec& rec = s.rec;
	rec.obj = obj;
	rec.kind = kind;
	rec.id = id;
	rec.shader = shader;
	if (s.wr.occl) return false;
	rec.t = ph.t;
	rec.u = ph.u;
	rec.v = ph.v;
	rec.max_dim = ph.max_dim;
	const int L = s.L;
	rec.depth = L + 1;
	for (int k = 1; k <= L; ++k) rec.path[k - 1] = s.lv[k].inst;
	rec.path[L] = gi;
	return true;
}

// An inner node: tests the child boxes (BBox4::intersect_ray,
// basics/bbox.hpp:566-595) and pushes the hit children, nearest on top.
// Returns false when the node stack overflows (the ray ends with an error).
template <unsigned F>
__device__ __forceinline__ bool node_visit(const DevScene& sc, TraceState<F>& s, int ref) {
	const WorldRayD& wr = s.wr;
	const DevNode* nd = sc.nodes + ref;
	float b[24];
	load_box4(reinterpret_cast<const float4*>(nd->b), b);
	const int4 ch = __ldg(reinterpret_cast<const int4*>(nd->child));
	const int4 meta = __ldg(reinterpret_cast<const int4*>(&nd->nchild));
	const int nch = meta.x;
	const int ts = meta.y;
	if (ts > 1) {
		// motion: lerp the boxes of the two time samples around the ray
		// time (sample 0 is in the node, later ones in node_extra)
		const SeqPos sp = seq_pos(wr.time, ts);
		auto extra = [&](int k) {
			return reinterpret_cast<const float4*>(sc.node_extra + (size_t)(meta.z + k - 1) * 24);
		};
		if (sp.single) {
			if (sp.i0 != 0) load_box4(extra(sp.i0), b);
		} else {
			float e1[24];
			load_box4(extra(sp.i0 + 1), e1);
			if (sp.i0 != 0) load_box4(extra(sp.i0), b);
			const float ia = one_minus(sp.nalpha);
#pragma unroll
			for (int i = 0; i < 24; ++i) b[i] = (b[i] * ia) + (e1[i] * sp.nalpha);
		}
	}
	// slab tests of the four children; every array index below is a
	// compile-time constant so the node stays in registers
	const bool ds0 = s.r.dinv.x < 0.0f, ds1 = s.r.dinv.y < 0.0f, ds2 = s.r.dinv.z < 0.0f;
	const int chv[4] = {ch.x, ch.y, ch.z, ch.w};
	float tk[4];
	int ck[4], sk[4];
	int nhit = 0;
#pragma unroll
	for (int c = 0; c < 4; ++c) {
		const float x0 = b[0 * 4 + c], x1 = b[1 * 4 + c];
		const float y0 = b[2 * 4 + c], y1 = b[3 * 4 + c];
		const float z0 = b[4 * 4 + c], z1 = b[5 * 4 + c];
		const float xlo = ((ds0 ? x1 : x0) - s.r.o.x) * s.r.dinv.x;
		const float xhi = ((ds0 ? x0 : x1) - s.r.o.x) * s.r.dinv.x;
		const float ylo = ((ds1 ? y1 : y0) - s.r.o.y) * s.r.dinv.y;
		const float yhi = ((ds1 ? y0 : y1) - s.r.o.y) * s.r.dinv.y;
		const float zlo = ((ds2 ? z1 : z0) - s.r.o.z) * s.r.dinv.z;
		const float zhi = ((ds2 ? z0 : z1) - s.r.o.z) * s.r.dinv.z;
		const float mins = vmax(vmax(xlo, ylo), vmax(zlo, 0.0f));
		const float maxs = vmax(vmin(vmin(xhi, yhi), zhi), -INFINITY) * BBOX_MAXT_ADJUST;
		const bool h = c < nch && mins < s.max_t && mins <= maxs;
		// a hit has mins < max_t <= inf, so inf marks the misses
		tk[c] = h ? mins : INFINITY;
		ck[c] = chv[c];
		sk[c] = c;
		nhit += h ? 1 : 0;
	}
	// nearest first, ties in child order (a stable sort by distance)
	auto cswap = [&](int a, int bb) {
		if (tk[bb] < tk[a] || (tk[bb] == tk[a] && sk[bb] < sk[a])) {
			const float t = tk[a]; tk[a] = tk[bb]; tk[bb] = t;
			const int c = ck[a]; ck[a] = ck[bb]; ck[bb] = c;
			const int q = sk[a]; sk[a] = sk[bb]; sk[bb] = q;
		}
	};
	if (s.nsp + nhit > PSY_NODE_STACK) {
		s.err |= ERRF_STACK;
		return false;
	}
	if (wr.occl) {
		// an occlusion ray stops at any hit, so the order it meets the
		// children in does not matter: push the hit ones unsorted
#pragma unroll
		for (int c = 3; c >= 0; --c)
			if (tk[c] != INFINITY) s.node_stack[s.nsp++] = ck[c];
		return true;
	}
	cswap(0, 1);
	cswap(2, 3);
	cswap(0, 2);
	cswap(1, 3);
	cswap(1, 2);
	if (nhit > 3) s.node_stack[s.nsp++] = ck[3];
	if (nhit > 2) s.node_stack[s.nsp++] = ck[2];
	if (nhit > 1) s.node_stack[s.nsp++] = ck[1];
	if (nhit > 0) s.node_stack[s.nsp++] = ck[0];
	return true;
}

// Leaves the finished levels, restoring the ray of the enclosing level.
template <unsigned F>
__device__ __forceinline__ void leave_levels(TraceState<F>& s) {
	constexpr bool NESTED = (F & FEAT_NESTED) != 0;
	while (NESTED && s.L > 0 && s.nsp == s.lv[s.L].stack_base) {
		const bool changed = s.lvl_frame[s.L] != s.lvl_frame[s.L - 1];
		--s.L;
		if (changed) {
			s.r = s.lvr[s.L];
			s.rw_ok = false;
		}
	}
}

// Enters the assembly of instance `inst` (global index gi, element id
// `id`, inherited shader): merges its transforms into the level's frame,
// moves the ray into its space and pushes its root.  Returns false when the
// node stack overflows.
template <unsigned F>
__device__ __forceinline__ bool enter_assembly(const DevScene& sc, TraceState<F>& s, const DevInstance& inst, int gi,
                                               uint64_t id, int shader) {
	constexpr bool XFORM = (F & FEAT_XFORM) != 0;
	const WorldRayD& wr = s.wr;
	Frame none;
	none.count = 0;
	const int L = s.L;
	const Frame& parent = s.lvl_frame[L] >= 0 ? s.frames[s.lvl_frame[L]] : none;
	if (L + 1 >= PSY_MAX_LEVELS) {
		s.err |= ERRF_LEVELS;
		return true;
	}
	const DevAssembly as = sc.assemblies[inst.data];
	if (as.root == REF_EMPTY) return true;
	if (XFORM && inst.xform_count > 0) {
		if (!frame_merge(parent, sc.xforms + (size_t)inst.xform * 16, inst.xform_count, &s.frames[L + 1])) {
			s.err |= ERRF_MOTION;
			return true;
		}
		s.lvl_frame[L + 1] = L + 1;
		s.lvr[L] = s.r;
		s.r = make_local_x(wr, frame_at_index_lerp(s.frames[L + 1], wr.time));
		s.rw_ok = false;
	} else {
		s.lvl_frame[L + 1] = s.lvl_frame[L];
	}
	s.L = L + 1;
	Level& nl = s.lv[L + 1];
	nl.asmb = inst.data;
	nl.stack_base = s.nsp;
	nl.shader = shader;
	nl.inst = gi;
	nl.id = id;
	nl.id_bits = as.id_bits;
	nl.inst_base = as.inst_base;
	if (s.nsp + 1 > PSY_NODE_STACK) {
		s.err |= ERRF_STACK;
		return false;
	}
	s.node_stack[s.nsp++] = as.root;
	return true;
}

// The test of object instance `inst` of the current level (global index
// gi, element id `id`, bound shader).  With RESUME a patch whose box the
// ray hits only starts its bisection (patch_step carries it on); without,
// the bisection runs here.  Returns false when the ray is finished (an
// occlusion ray's hit).
template <unsigned F, bool RESUME>
__device__ __forceinline__ bool object_test(const DevScene& sc, TraceState<F>& s, const DevInstance& inst, int gi,
                                            uint64_t id, int shader) {
	constexpr bool XFORM = (F & FEAT_XFORM) != 0;
	const WorldRayD& wr = s.wr;
	Frame none;
	none.count = 0;
	const int L = s.L;
	LocalRay lr = s.r;
	M44 om;  // the object's own transform at the ray time
	const bool oxf = XFORM && inst.xform_count > 0;
	if (oxf) {
		const Frame& parent = s.lvl_frame[L] >= 0 ? s.frames[s.lvl_frame[L]] : none;
		Frame nf;
		if (!frame_merge(parent, sc.xforms + (size_t)inst.xform * 16, inst.xform_count, &nf)) {
			s.err |= ERRF_MOTION;
			return true;
		}
		om = frame_at_index_lerp(nf, wr.time);
		lr = make_local_x(wr, om);
	}
	const DevObject ob = sc.objects[inst.data];
	// width parameters for patches: the object's own, or the level's (cached)
	auto width = [&]() -> RayWidth {
		if (oxf) return ray_width_of(wr, lr, &om);
		if (!s.rw_ok) {
			if (XFORM && s.lvl_frame[L] >= 0) {
				const M44 lm = frame_at_index_lerp(s.frames[s.lvl_frame[L]], wr.time);
				s.rw = ray_width_of(wr, s.r, &lm);
			} else {
				s.rw = ray_width_of(wr, s.r, nullptr);
			}
			s.rw_ok = true;
		}
		return s.rw;
	};
	// a patch with RESUME: test the root box here, bisect in patch_step
	auto begin_patch = [&](const float* v) {
		int pm = PM_NONE;
		if constexpr ((F & FEAT_BILINEAR) != 0) {
			if (ob.kind == OBJ_BILINEAR) {
				if constexpr ((F & FEAT_PATCH_MOTION) != 0) {
					if (ob.n0 != 1)
						pm = patch_begin<4, 2>(s.template work<4, 2>().c, v, wr.time, lr, s.max_t) ? PM_BILINEAR2 : -1;
				}
				if (pm == PM_NONE) pm = patch_begin<4, 1>(s.template work<4, 1>().c, v, wr.time, lr, s.max_t) ? PM_BILINEAR1 : -1;
			}
		}
		if constexpr ((F & FEAT_BICUBIC) != 0) {
			if (ob.kind == OBJ_BICUBIC) {
				if constexpr ((F & FEAT_PATCH_MOTION) != 0) {
					if (ob.n0 != 1)
						pm = patch_begin<16, 2>(s.template work<16, 2>().c, v, wr.time, lr, s.max_t) ? PM_BICUBIC2 : -1;
				}
				if (pm == PM_NONE) pm = patch_begin<16, 1>(s.template work<16, 1>().c, v, wr.time, lr, s.max_t) ? PM_BICUBIC1 : -1;
			}
		}
		if (pm > PM_NONE) {
			s.pmode = pm;
			s.pverts = v;
			s.pr = lr;
			s.prw = width();
			s.p_obj = inst.data;
			s.p_kind = ob.kind;
			s.p_id = id;
			s.p_shader = shader;
			s.p_gi = gi;
		}
	};
	bool hit = false;
	PatchHit ph;
	ph.u = ph.v = ph.max_dim = 0.0f;
	float max_t = s.max_t;
	const float* v = sc.fpool + ob.data;
	if (ob.kind == OBJ_SPHERE || ob.kind == OBJ_SPHERE_LIGHT) {
		V3 cent;
		float radi;
		if (ob.kind == OBJ_SPHERE) {
			sphere_at(sc, ob, wr.time, &cent, &radi);
		} else {
			float col[3];
			light_at(sc, ob, wr.time, &cent, &radi, col);
		}
		const float t = sphere_t(lr.o, lr.d, cent, radi, max_t);
		if (t >= 0.0f) {
			hit = true;
			ph.t = t;
			if (!wr.occl) max_t = t;
		}
	} else if (ob.kind == OBJ_RECT_LIGHT) {
		float dx, dy;
		rect_light_at(sc, ob, wr.time, &dx, &dy, nullptr);
		const float t = rect_light_t(lr.o, lr.d, lr.dinv, dx, dy, max_t);
		if (t >= 0.0f) {
			hit = true;
			ph.t = t;
			if (!wr.occl) max_t = t;
		}
	} else if constexpr (!RESUME) {
		// the bisection runs here, to its end
		if ((F & FEAT_BILINEAR) && ob.kind == OBJ_BILINEAR) {
			const RayWidth w = width();
			if ((F & FEAT_PATCH_MOTION) && ob.n0 != 1)
				hit = patch_whole<4, 2>(v, wr.time, lr, w, &max_t, wr.occl, sc.dice_rate, sc.min_upoly_size, &ph,
				                             &s.err);
			else
				hit = patch_whole<4, 1>(v, wr.time, lr, w, &max_t, wr.occl, sc.dice_rate, sc.min_upoly_size, &ph,
				                             &s.err);
		} else if ((F & FEAT_BICUBIC) && ob.kind == OBJ_BICUBIC) {
			const RayWidth w = width();
			if ((F & FEAT_PATCH_MOTION) && ob.n0 != 1)
				hit = patch_whole<16, 2>(v, wr.time, lr, w, &max_t, wr.occl, sc.dice_rate, sc.min_upoly_size, &ph,
				                             &s.err);
			else
				hit = patch_whole<16, 1>(v, wr.time, lr, w, &max_t, wr.occl, sc.dice_rate, sc.min_upoly_size, &ph,
				                             &s.err);
		}
	} else {
		begin_patch(v);
	}
	s.max_t = max_t;
	if (hit) return trace_record<F>(s, inst.data, ob.kind, id, shader, gi, ph);
	return true;
}

// One step of a lane that runs its ray alone: traverse to the next object
// leaf and test it, a patch's whole bisection included.  The closest hit
// does not depend on the order objects are tested in (a sub-patch's box
// lies inside its parent's, so max_t pruning only drops leaves that could
// not be closer), except for exact ties.  Returns false when the ray is
// finished.
template <unsigned F>
__device__ __forceinline__ bool trace_step(const DevScene& sc, TraceState<F>& s) {
	constexpr bool NESTED = (F & FEAT_NESTED) != 0;
	while (true) {
		leave_levels<F>(s);
		if (s.nsp == 0) return false;
		const int ref = s.node_stack[--s.nsp];
		if (ref >= 0) {
			if (!node_visit<F>(sc, s, ref)) return false;
			continue;
		}
		// leaf: one instance of the current level's assembly
		const int local = leaf_instance(ref);
		const int gi = s.lv[s.L].inst_base + local;
		const DevInstance inst = sc.instances[gi];
		const uint64_t id = id_push(s.lv[s.L].id, (uint64_t)local, s.lv[s.L].id_bits);
		const int shader = inst.shader >= 0 ? inst.shader : s.lv[s.L].shader;
		if (NESTED && inst.kind == INST_ASSEMBLY) {
			if (!enter_assembly<F>(sc, s, inst, gi, id, shader)) return false;
			continue;
		}
		return object_test<F, false>(sc, s, inst, gi, id, shader);
	}
}

// The walk cut into pieces for kernels that group their lanes by the work
// they do next: up to `nodes` inner-node visits, stopping at a leaf, which
// is popped into s.leaf for leaf_visit.  Returns WALK_DONE when the ray is
// finished, WALK_LEAF at a leaf, WALK_MORE when the visits ran out; `nodes`
// is left at the visits not used.
enum : int { WALK_DONE = 0, WALK_LEAF = 1, WALK_MORE = 2 };

template <unsigned F>
__device__ __forceinline__ int walk_nodes(const DevScene& sc, TraceState<F>& s, int& nodes) {
	while (true) {
		leave_levels<F>(s);
		if (s.nsp == 0) return WALK_DONE;
		const int ref = s.node_stack[s.nsp - 1];
		if (ref < 0) {
			--s.nsp;
			s.leaf = ref;
			return WALK_LEAF;
		}
		if (nodes == 0) return WALK_MORE;
		--nodes;
		--s.nsp;
		if (!node_visit<F>(sc, s, ref)) return WALK_DONE;
	}
}

// The leaf popped by walk_nodes: an assembly instance is entered, an object
// instance tested (a patch starts its bisection).  Returns false when the
// ray is finished.
template <unsigned F>
__device__ __forceinline__ bool leaf_visit(const DevScene& sc, TraceState<F>& s) {
	constexpr bool NESTED = (F & FEAT_NESTED) != 0;
	const int local = leaf_instance(s.leaf);
	const int gi = s.lv[s.L].inst_base + local;
	const DevInstance inst = sc.instances[gi];
	const uint64_t id = id_push(s.lv[s.L].id, (uint64_t)local, s.lv[s.L].id_bits);
	const int shader = inst.shader >= 0 ? inst.shader : s.lv[s.L].shader;
	if (NESTED && inst.kind == INST_ASSEMBLY) return enter_assembly<F>(sc, s, inst, gi, id, shader);
	return object_test<F, true>(sc, s, inst, gi, id, shader);
}

// Work kinds of the wave kernels' lanes: idle, node visits, a leaf visit of
// one of three classes, a bisection in progress.  Leaf visits are told
// apart by class so that the lanes of a warp step run one branch of
// leaf_visit together: assembly entries (transform merge, ray transform),
// simple objects (spheres, sphere and rectangle lights), patches (root box,
// ray widths, bisection set-up).
enum : int { KIND_IDLE = 0, KIND_NODES = 1, LEAF_ENTER = 2, LEAF_SIMPLE = 3, LEAF_PATCH = 4, KIND_PATCH = 5 };

// The class of the leaf walk_nodes stopped at (s.leaf).
template <unsigned F>
__device__ __forceinline__ int leaf_class(const DevScene& sc, const TraceState<F>& s) {
	constexpr bool NESTED = (F & FEAT_NESTED) != 0;
	const int gi = s.lv[s.L].inst_base + leaf_instance(s.leaf);
	const int2 kd = __ldg(reinterpret_cast<const int2*>(sc.instances + gi));  // kind, data
	if (NESTED && kd.x == INST_ASSEMBLY) return LEAF_ENTER;
	const int ok = __ldg(&sc.objects[kd.y].kind);
	return (ok == OBJ_BICUBIC || ok == OBJ_BILINEAR) ? LEAF_PATCH : LEAF_SIMPLE;
}

// Carries the bisection in progress on for up to `units` iterations of its
// loop (`units` is left at the iterations not used).  Returns false when
// the ray is finished (an occlusion ray's hit).
template <unsigned F>
__device__ __forceinline__ bool patch_step(const DevScene& sc, TraceState<F>& s, int& units) {
	constexpr int TS = PatchBuf<F>::TS;
	bool done = false, found = false;
	float max_t = s.max_t;
	const bool occl = s.wr.occl;
	const float dr = sc.dice_rate, mu = sc.min_upoly_size;
	// the cursor runs as a local copy (registers) and goes back to the
	// state only when the bisection stops short of its end
	auto run = [&](auto& pw) {
		auto pc = pw.c;
		done = patch_run(pc, pw.st, s.pverts, s.pr, s.prw, &max_t, occl, dr, mu, &s.ph, units, &s.err);
		if (!done) pw.c = pc;
		found = pc.found;
	};
	if constexpr ((F & FEAT_BILINEAR) != 0) {
		if (s.pmode == PM_BILINEAR1) run(s.template work<4, 1>());
		else if (TS == 2 && s.pmode == PM_BILINEAR2) run(s.template work<4, TS>());
	}
	if constexpr ((F & FEAT_BICUBIC) != 0) {
		if (s.pmode == PM_BICUBIC1) run(s.template work<16, 1>());
		else if (TS == 2 && s.pmode == PM_BICUBIC2) run(s.template work<16, TS>());
	}
	s.max_t = max_t;
	if (!done) return true;
	s.pmode = PM_NONE;
	if (found) return trace_record<F>(s, s.p_obj, s.p_kind, s.p_id, s.p_shader, s.p_gi, s.ph);
	return true;
}

// Traces one ray through the scene. Returns the device error flags.
template <unsigned F>
__device__ unsigned trace_ray(const DevScene& sc, const WorldRayD& wr, HitRec* rec) {
	TraceState<F> s;
	trace_init<F>(sc, s, wr);
	while (trace_step<F>(sc, s)) {
	}
	*rec = s.rec;
	return s.err;
}

// Transform from world space into the hit object's space at the ray time
// (the Intersection::space of the reference), rebuilt from the hit path.
// Returns false when the path carries no transform (identity).
template <unsigned F>
__device__ bool hit_space(const DevScene& sc, const HitRec& rec, float time, M44* out, unsigned* err) {
	if (!(F & FEAT_XFORM)) return false;
	Frame f;
	f.count = 0;
	for (int k = 0; k < rec.depth; ++k) {
		const DevInstance inst = sc.instances[rec.path[k]];
		if (inst.xform_count > 0) {
			Frame g;
			if (!frame_merge(f, sc.xforms + (size_t)inst.xform * 16, inst.xform_count, &g)) {
				*err |= ERRF_MOTION;
				return false;
			}
			f = g;
		}
	}
	if (f.count == 0) return false;
	*out = frame_at_index_lerp(f, time);
	return true;
}

}  // namespace psy

#endif
