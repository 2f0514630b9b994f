/*
 * Wavefront path tracer: PathTraceIntegrator::integrate restated for the
 * GPU (reference integrator/path_trace_integrator.cpp:91-384).
 *
 * The reference renders a bucket as a stream of paths and loops
 *   generate one ray per live path -> Tracer::trace -> update -> partition.
 * Here a wave of paths lives in HBM as SoA state and the loop is split into
 * kernels that each do one kind of work, so the traversal kernels carry no
 * shading state and the shading kernels no traversal state:
 *
 *   camera_gen            camera rays of every path of the wave
 *   trace<closest>        Tracer::trace of the ray buffer (closest hits)
 *   shade_hit             update_path after a camera / bounce ray, then
 *                         next_ray_for_path's shadow step: light-tree sample
 *                         and shadow ray; live paths are compacted into the
 *                         next queue (ballot + popc, one atomic per warp)
 *   trace<occlusion>      Tracer::trace of the shadow rays
 *   shade_shadow          update_path after the shadow ray, then the bounce
 *                         ray (the path stays at its queue position)
 *   ... trace<closest> -> shade_hit -> ... for path_length bounces.
 *
 * Rays and hits are stored by queue position (coalesced), path state by
 * path slot.  Finished paths write their film sample
 * (Color_XYZ(col) * XYZ_NORM_FAC); a per-wave reduction adds each pixel's
 * samples in sample order.
 *
 * The same kernels serve two modes.  PlainWave renders one scene and takes
 * the scene and render parameters as kernel parameters.  BatchWave renders
 * many scenes at once: a wave covers consecutive global paths of several
 * renders, each path carries its render index, and scenes and parameters
 * are read from device arrays.
 */
#include "kernels.h"
#include "render_device.cuh"

namespace psy {

__device__ __forceinline__ float4 f4(const Spec& s) { return make_float4(s.e[0], s.e[1], s.e[2], s.e[3]); }
__device__ __forceinline__ Spec sp(float4 v) {
	Spec s;
	s.e[0] = v.x; s.e[1] = v.y; s.e[2] = v.z; s.e[3] = v.w;
	return s;
}

// ---------------------------------------------------------------------
// Ray and hit records by queue position
// ---------------------------------------------------------------------
// Ray planes (5 x float4 per position):
//   0: o.xyz, time   1: d.xyz, odx.x   2: odx.yz, ody.xy   3: ody.z, ddx.xyz
//   4: ddy.xyz, tag = render index << 1 | 1 when there is no ray (the shadow
//      step found no light sample)
__device__ __forceinline__ void store_ray(float4* rb, int cap, int i, const WorldRayD& r, int tag) {
	rb[i] = make_float4(r.o.x, r.o.y, r.o.z, r.time);
	rb[cap + i] = make_float4(r.d.x, r.d.y, r.d.z, r.odx.x);
	rb[2 * cap + i] = make_float4(r.odx.y, r.odx.z, r.ody.x, r.ody.y);
	rb[3 * cap + i] = make_float4(r.ody.z, r.ddx.x, r.ddx.y, r.ddx.z);
	rb[4 * cap + i] = make_float4(r.ddy.x, r.ddy.y, r.ddy.z, __int_as_float(tag));
}
__device__ __forceinline__ int load_ray(const float4* rb, int cap, int i, WorldRayD* r) {
	const float4 a = rb[i], b = rb[cap + i], c = rb[2 * cap + i], d = rb[3 * cap + i], e = rb[4 * cap + i];
	r->o = V3(a.x, a.y, a.z);
	r->time = a.w;
	r->d = V3(b.x, b.y, b.z);
	r->odx = V3(b.w, c.x, c.y);
	r->ody = V3(c.z, c.w, d.x);
	r->ddx = V3(d.y, d.z, d.w);
	r->ddy = V3(e.x, e.y, e.z);
	return __float_as_int(e.w);
}

// Hit planes: 0: t, u, v, max_dim (float4)   1: obj, kind | depth << 8,
// shader, path[0]   2: path[1..4]   3: path[5..7] (int4).  The path planes
// beyond the hit's depth are neither written nor read.
__device__ __forceinline__ void store_rec(const WaveBufs& wb, int i, const HitRec& h) {
	wb.hit_f[i] = make_float4(h.t, h.u, h.v, h.max_dim);
	const int cap = wb.cap;
	if (h.obj < 0) {
		wb.hit_i[i] = make_int4(-1, 0, -1, 0);
		return;
	}
	wb.hit_i[i] = make_int4(h.obj, h.kind | (h.depth << 8), h.shader, h.path[0]);
	if (h.depth > 1) wb.hit_i[cap + i] = make_int4(h.path[1], h.path[2], h.path[3], h.path[4]);
	if (h.depth > 5) wb.hit_i[2 * cap + i] = make_int4(h.path[5], h.path[6], h.path[7], 0);
}
__device__ __forceinline__ void load_rec(const WaveBufs& wb, int i, HitRec* h) {
	const float4 f = wb.hit_f[i];
	h->t = f.x; h->u = f.y; h->v = f.z; h->max_dim = f.w;
	const int4 a = wb.hit_i[i];
	h->obj = a.x;
	h->kind = a.y & 0xff;
	h->depth = a.y >> 8;
	h->shader = a.z;
	h->path[0] = a.w;
	h->id = 0;
	const int cap = wb.cap;
	if (h->depth > 1) {
		const int4 b = wb.hit_i[cap + i];
		h->path[1] = b.x; h->path[2] = b.y; h->path[3] = b.z; h->path[4] = b.w;
	}
	if (h->depth > 5) {
		const int4 c = wb.hit_i[2 * cap + i];
		h->path[5] = c.x; h->path[6] = c.y; h->path[7] = c.z;
	}
}

// World-space shading data of the stored intersection (the PTState::inter
// and prev_ray the reference keeps per path).
struct StoredHit {
	V3 p, n, off;       // geo.p, geo.n (after transformed_from), signed ray-origin offset
	float t;
	float bf;           // 1 when the hit was back-facing
	float col[3];       // closure colour (Lambert)
	int pid;            // differentiable renders: the shader's first albedo weight (>= 0), -2 - q when its
	                    // RGB albedo is scaled by params[q], or -1 (not parameterised)
	int gtr;            // the GTR shader of the hit, or -1 (Lambert)
	V3 d, odx, ody, ddx, ddy;  // previous ray
	V3 dpdu, dpdv, dndu, dndv; // GTR hits: geo's derivatives in world space (transformed_from)
};

__device__ __forceinline__ void load_hit(const PathSoA& ps, int s, StoredHit* h) {
	const float4* g = reinterpret_cast<const float4*>(ps.hit) + (size_t)s * 4;
	const float4 a = g[0], b = g[1], c = g[2], d = g[3];
	h->p = V3(a.x, a.y, a.z);
	h->n = V3(a.w, b.x, b.y);
	h->off = V3(b.z, b.w, c.x);
	h->t = c.y;
	h->col[0] = c.z; h->col[1] = c.w; h->col[2] = d.x;
	h->bf = d.y;
	h->pid = __float_as_int(d.z);
	h->gtr = __float_as_int(d.w);
	if (h->gtr >= 0) {
		const float4* x = reinterpret_cast<const float4*>(ps.hitx) + (size_t)s * 3;
		const float4 u = x[0], v = x[1], w = x[2];
		h->dpdu = V3(u.x, u.y, u.z);
		h->dpdv = V3(u.w, v.x, v.y);
		h->dndu = V3(v.z, v.w, w.x);
		h->dndv = V3(w.y, w.z, w.w);
	}
	const float4* r = reinterpret_cast<const float4*>(ps.pray) + (size_t)s * 4;
	const float4 e = r[0], f = r[1], gg = r[2], hh = r[3];
	h->d = V3(e.x, e.y, e.z);
	h->odx = V3(e.w, f.x, f.y);
	h->ody = V3(f.z, f.w, gg.x);
	h->ddx = V3(gg.y, gg.z, gg.w);
	h->ddy = V3(hh.x, hh.y, hh.z);
}

__device__ __forceinline__ void store_hit(const PathSoA& ps, int s, const StoredHit& h) {
	float4* g = reinterpret_cast<float4*>(ps.hit) + (size_t)s * 4;
	g[0] = make_float4(h.p.x, h.p.y, h.p.z, h.n.x);
	g[1] = make_float4(h.n.y, h.n.z, h.off.x, h.off.y);
	g[2] = make_float4(h.off.z, h.t, h.col[0], h.col[1]);
	g[3] = make_float4(h.col[2], h.bf, __int_as_float(h.pid), __int_as_float(h.gtr));
	if (h.gtr >= 0) {
		float4* x = reinterpret_cast<float4*>(ps.hitx) + (size_t)s * 3;
		x[0] = make_float4(h.dpdu.x, h.dpdu.y, h.dpdu.z, h.dpdv.x);
		x[1] = make_float4(h.dpdv.y, h.dpdv.z, h.dndu.x, h.dndu.y);
		x[2] = make_float4(h.dndu.z, h.dndv.x, h.dndv.y, h.dndv.z);
	}
	float4* r = reinterpret_cast<float4*>(ps.pray) + (size_t)s * 4;
	r[0] = make_float4(h.d.x, h.d.y, h.d.z, h.odx.x);
	r[1] = make_float4(h.odx.y, h.odx.z, h.ody.x, h.ody.y);
	r[2] = make_float4(h.ody.z, h.ddx.x, h.ddx.y, h.ddx.z);
	r[3] = make_float4(h.ddy.x, h.ddy.y, h.ddy.z, 0.0f);
}

// Intersection -> stored hit: DifferentialGeometry::transformed_from(space)
// (basics/differential_geometry.hpp:20-40) and the offset of
// path_trace_integrator.cpp:141-145.
template <unsigned F>
__device__ void make_stored(const DevScene& sc, const HitRec& rec, const WorldRayD& wr, float ident_inv,
                            StoredHit* sh, int* closure, float* emit_col, float* light_pdf, unsigned* err) {
	M44 space;
	const bool xf = hit_space<F>(sc, rec, wr.time, &space, err);
	V3 lo = wr.o, ld = wr.d;
	if (xf) {
		lo = pos_to(space, wr.o);
		ld = dir_to(space, wr.d);
	}
	HitInfo h;
	hit_geometry(sc, rec, wr.time, lo, ld, &h);
	*closure = h.closure;
	emit_col[0] = h.col[0]; emit_col[1] = h.col[1]; emit_col[2] = h.col[2];
	*light_pdf = h.light_pdf;
	if (h.closure != CLOSURE_LAMBERT && h.closure != CLOSURE_GTR) return;
	M44 inv;
	if (xf) {
		inv = m44_inverse_dev(space, sc.rcp);
	} else {
		inv = m44_identity();
		for (int i = 0; i < 4; ++i) inv.m[i][i] = ident_inv;
	}
	sh->p = pos_to(inv, h.geo.p);
	const M44 nx = xf ? space : m44_identity();
	const V3 n = nor_from(nx, h.geo.n);
	const float il = 1.0f / length(n);
	sh->n = n * il;
	sh->gtr = -1;
	if (h.closure == CLOSURE_GTR) {
		// the rest of DifferentialGeometry::transformed_from (basics/differential_geometry.hpp:20-40)
		sh->gtr = rec.shader;
		sh->dpdu = dir_to(inv, h.geo.dpdu);
		sh->dpdv = dir_to(inv, h.geo.dpdv);
		sh->dndu = nor_from(nx, h.geo.dndu) * il;
		sh->dndv = nor_from(nx, h.geo.dndv) * il;
	}
	V3 off = dir_to(inv, h.offset);
	if (h.backfacing) off = off * -1.0f;
	sh->off = off;
	sh->bf = h.backfacing ? 1.0f : 0.0f;
	sh->t = rec.t;
	sh->col[0] = h.col[0]; sh->col[1] = h.col[1]; sh->col[2] = h.col[2];
	sh->d = wr.d;
	sh->odx = wr.odx;
	sh->ody = wr.ody;
	sh->ddx = wr.ddx;
	sh->ddy = wr.ddy;
}

// LambertClosure::propagate_differentials (shading/surface_closure.hpp:306-320).
__device__ __forceinline__ void propagate_differentials(const StoredHit& h, WorldRayD* out) {
	const float len = length(out->d);
	const V3 nn = normalized(h.n);
	V3 x, y;
	coordinate_system(out->d, &x, &y);
	x = normalized(x);
	y = normalized(y);
	out->odx = transfer_origin_differential(h.t, nn, h.d, h.odx, h.ddx);
	out->ody = transfer_origin_differential(h.t, nn, h.d, h.ody, h.ddy);
	out->ddx = (x * 0.15f) / len;
	out->ddy = (y * 0.15f) / len;
}

// GTRClosure::propagate_differentials (shading/surface_closure.hpp:574-607):
// origin differentials transferred to the hit, normal differentials turned
// into half-vector differentials, direction differentials reflected about
// the half vector, then clamped (clamp_dd).
static __device__ __noinline__ void gtr_propagate_differentials(const StoredHit& h, WorldRayD* out) {
	V3 nn = normalized(h.n);
	const V3 hh = normalized(normalized(h.d * -1.0f) + normalized(out->d));
	out->odx = transfer_origin_differential(h.t, nn, h.d, h.odx, h.ddx);
	out->ody = transfer_origin_differential(h.t, nn, h.d, h.ody, h.ddy);
	float dux, dvx, duy, dvy;
	uv_differentials(out->odx, h.dpdu, h.dpdv, &dux, &dvx);
	uv_differentials(out->ody, h.dpdu, h.dpdv, &duy, &dvy);
	V3 dndx = (h.dndu * dux) + (h.dndv * dvx);
	V3 dndy = (h.dndu * duy) + (h.dndv * dvy);
	if (dot(nn, hh) < 0.0f) {
		nn = nn * -1.0f;
		dndx = dndx * -1.0f;
		dndy = dndy * -1.0f;
	}
	const V3 axis = normalized(cross(nn, hh));
	const float angle = lm_acosf(clampf(dot(nn, hh), 0.0f, 1.0f));
	const M44 xf = axis_angle(axis, angle);
	const V3 dhdx = dir_to(xf, dndx);
	const V3 dhdy = dir_to(xf, dndy);
	out->ddx = reflect_dd(hh, dhdx, h.d, h.ddx);
	out->ddy = reflect_dd(hh, dhdy, h.d, h.ddy);
	const float len_d = length(out->d);
	const float len_dx = length(out->ddx);
	const float len_dy = length(out->ddy);
	if ((len_dx / len_d) > 0.9f) out->ddx = out->ddx * ((0.9f * len_d) / len_dx);
	if ((len_dy / len_d) > 0.9f) out->ddy = out->ddy * ((0.9f * len_d) / len_dy);
}

__device__ __forceinline__ void finish_path(const PathSoA& ps, int slot, const Spec& col, float wl) {
	float xyz[3];
	spec_to_xyz(col, wl, xyz);
	float3 o;
	o.x = xyz[0] * XYZ_NORM_FAC;
	o.y = xyz[1] * XYZ_NORM_FAC;
	o.z = xyz[2] * XYZ_NORM_FAC;
	reinterpret_cast<float3*>(ps.sample)[slot] = o;
}

// ---------------------------------------------------------------------
// Wave modes: where a kernel finds the scene and parameters of render r
// ---------------------------------------------------------------------
struct PlainWave {
	static constexpr bool BATCH = false;
	DevScene sc;
	RenderParams rp;
	__device__ __forceinline__ const DevScene& scene(int) const { return sc; }
	__device__ __forceinline__ const RenderParams& render(int) const { return rp; }
	__device__ __forceinline__ int render_of_path(uint64_t) const { return 0; }
	__device__ __forceinline__ int render_of_pixel(uint64_t) const { return 0; }
};

struct BatchWave {
	static constexpr bool BATCH = true;
	const DevScene* scenes;
	const RenderParams* renders;
	int count;
	__device__ __forceinline__ const DevScene& scene(int r) const { return scenes[r]; }
	__device__ __forceinline__ const RenderParams& render(int r) const { return renders[r]; }
	// the last render whose first path (pixel) is at or before g
	__device__ __forceinline__ int render_of_path(uint64_t g) const {
		int lo = 0, hi = count - 1;
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if (renders[mid].path_base <= g) lo = mid; else hi = mid - 1;
		}
		return lo;
	}
	__device__ __forceinline__ int render_of_pixel(uint64_t q) const {
		int lo = 0, hi = count - 1;
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if (renders[mid].pixel_base <= q) lo = mid; else hi = mid - 1;
		}
		return lo;
	}
};

// ---------------------------------------------------------------------
// Differentiable rendering (no reference counterpart)
// ---------------------------------------------------------------------
// Emission scale parameter of object `obj`, or -1.
__device__ __forceinline__ int emission_param(const RenderParams& rp, int obj) {
	return (rp.params && obj >= 0) ? rp.object_param[obj] : -1;
}

// lambert_eval with the albedo taken from parameters when the stored hit's
// shader has them.
__device__ __forceinline__ Spec lambert_eval_p(const RenderParams& rp, const StoredHit& sh, V3 out, float wl) {
	if (sh.pid == -1) return lambert_eval(sh.col, sh.d, out, sh.n, wl);
	if (sh.pid < -1) {
		Spec f = lambert_eval(sh.col, sh.d, out, sh.n, wl);
		const float q = rp.params[-2 - sh.pid];
		for (int k = 0; k < 4; ++k) f.e[k] *= q;
		return f;
	}
	const float c = lambert_cos(sh.d, out, sh.n);
	const Spec a = albedo_spec(rp.params + sh.pid, wl);
	Spec f;
	for (int k = 0; k < 4; ++k) f.e[k] = c * a.e[k];
	return f;
}

// Adjoint: adds u . dC/dparams for a radiance contribution C (hero
// wavelengths) whose albedo factors come from vertices 0..nv-1 of the path
// and whose emission is scaled by params[lp] (lp < 0: none).  C is the
// product of B (the contribution with every parameterised albedo and the
// emission scale left out), the parameterised vertices' albedos (each
// linear in its four weights) and the scale, so the derivative for one
// factor is the product of all the others: no division, so a factor that
// is zero (a black albedo, a light scaled to 0) still gets its gradient.
__device__ void grad_add(const RenderParams& rp, float* sg, const PathSoA& ps, int slot, int nv, const Spec& B,
                         int lp, float wl) {
	const float4 u4 = ps.adj[slot];
	const float ub[4] = {u4.x * B.e[0], u4.y * B.e[1], u4.z * B.e[2], u4.w * B.e[3]};
	float* g = rp.grad_in_smem ? sg : rp.grad;
	const float scale = lp >= 0 ? rp.params[lp] : 1.0f;
	if (nv > PSY_ADJ_MAX_VERTS) nv = PSY_ADJ_MAX_VERTS;
	float a[PSY_ADJ_MAX_VERTS][4];
	int pid[PSY_ADJ_MAX_VERTS];
	for (int v = 0; v < nv; ++v) {
		pid[v] = ps.vpid[slot * PSY_ADJ_MAX_VERTS + v];
		const float4 a4 = ps.valb[slot * PSY_ADJ_MAX_VERTS + v];
		a[v][0] = a4.x; a[v][1] = a4.y; a[v][2] = a4.z; a[v][3] = a4.w;
	}
	if (lp >= 0) {
		float d = 0.0f;
		for (int j = 0; j < 4; ++j) {
			float q = ub[j];
			for (int v = 0; v < nv; ++v)
				if (pid[v] != -1) q *= a[v][j];
			d += q;
		}
		atomicAdd(g + lp, d);
	}
	for (int v = 0; v < nv; ++v) {
		if (pid[v] == -1) continue;
		float q[4];
		for (int j = 0; j < 4; ++j) {
			q[j] = ub[j] * scale;
			for (int o = 0; o < nv; ++o)
				if (o != v && pid[o] != -1) q[j] *= a[o][j];
		}
		if (pid[v] < -1) {
			// scaled RGB albedo: its derivative is the upsampled colour
			const float4 u = ps.vdsc[slot * PSY_ADJ_MAX_VERTS + v];
			atomicAdd(g + (-2 - pid[v]), ((q[0] * u.x + q[1] * u.y) + q[2] * u.z) + q[3] * u.w);
			continue;
		}
		for (int k = 0; k < 4; ++k) {
			float d = 0.0f;
			for (int j = 0; j < 4; ++j) d += q[j] * albedo_basis(k, wavelength_n(wl, j));
			atomicAdd(g + pid[v] + k, d);
		}
	}
}

// Per-block gradient accumulators: cleared at kernel start, added to the
// global gradient at the end.
__device__ __forceinline__ void grad_begin(const RenderParams& rp, float* sg) {
	if (!rp.grad || !rp.grad_in_smem) return;
	for (int i = threadIdx.x; i < rp.param_count; i += blockDim.x) sg[i] = 0.0f;
	__syncthreads();
}
__device__ __forceinline__ void grad_end(const RenderParams& rp, float* sg) {
	if (!rp.grad || !rp.grad_in_smem) return;
	__syncthreads();
	for (int i = threadIdx.x; i < rp.param_count; i += blockDim.x)
		if (sg[i] != 0.0f) atomicAdd(rp.grad + i, sg[i]);
}

// Warp-wide work fetch: lane 0 takes the next 32 queue positions.
__device__ __forceinline__ int fetch32(int* work) {
	int base = 0;
	if ((threadIdx.x & 31) == 0) base = atomicAdd(work, 32);
	return __shfl_sync(0xffffffffu, base, 0);
}

// ---------------------------------------------------------------------
// Camera rays (next_ray_for_path, step 0: path_trace_integrator.cpp:109-125)
// ---------------------------------------------------------------------
template <class W>
__global__ void __launch_bounds__(256) camera_gen_kernel(W w, HaltonDev hd, WaveRange wv, PathSoA ps, WaveBufs wb) {
	const int slot = blockIdx.x * blockDim.x + threadIdx.x;
	if (slot >= wv.paths) return;
	const uint64_t gidx = wv.base + (uint64_t)slot;
	const int rid = w.render_of_path(gidx);
	const RenderParams& rp = w.render(rid);
	const uint64_t local = gidx - rp.path_base;
	const uint64_t pixel = local / rp.spp;
	const uint32_t px = (uint32_t)(pixel % rp.width);
	const uint32_t py = (uint32_t)(pixel / rp.width);
	const uint32_t s = (uint32_t)(local % rp.spp);
	const uint32_t smp = sampler_offset(px, py, s, rp.seed);
	uint32_t dim = 0;
	const float wl = (sampler_get(hd, smp, dim++) * (WAVELENGTH_MAX - WAVELENGTH_MIN)) + WAVELENGTH_MIN;
	const float samp_x = (fast_logit(sampler_get(hd, smp, dim++), 1.5f) + 0.5f + (float)px) / (float)rp.width;
	const float samp_y = (fast_logit(sampler_get(hd, smp, dim++), 1.5f) + 0.5f + (float)py) / (float)rp.height;
	const float rx = (float)(((double)samp_x - 0.5) * (double)(rp.max_x - rp.min_x));
	const float ry = (float)((0.5 - (double)samp_y) * (double)(rp.max_y - rp.min_y));
	const float dx = (rp.max_x - rp.min_x) / (float)rp.width;
	const float dy = (rp.max_y - rp.min_y) / (float)rp.height;
	const float samp_a = sampler_get(hd, smp, dim++);
	const float samp_b = sampler_get(hd, smp, dim++);
	const float samp_c = sampler_get(hd, smp, dim++);
	WorldRayD wr;
	camera_ray(w.scene(rid), rx, ry, dx, dy, samp_c, samp_a, samp_b, &wr);
	store_ray(wb.ray[0], wb.cap, slot, wr, rid << 1);
	if (W::BATCH) ps.rid[slot] = (uint16_t)rid;
	ps.smp[slot] = smp;
	ps.dimstep[slot] = dim;  // step 0
	ps.wl[slot] = wl;
	ps.time[slot] = wr.time;
	ps.last_pdf[slot] = 0.0f;
	ps.col[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	ps.fcol[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
	if (!W::BATCH && rp.dl_dxyz) {
		// d(film sum)/d(col) of finish_path: XYZ_NORM_FAC / 4 * CIE(lambda_j)
		const float* g = rp.dl_dxyz + 3 * pixel;
		float u[4];
		for (int j = 0; j < 4; ++j) {
			const float lw = wavelength_n(wl, j);
			u[j] = ((g[0] * X_1931(lw) + g[1] * Y_1931(lw)) + g[2] * Z_1931(lw)) * (0.25f * XYZ_NORM_FAC);
		}
		ps.adj[slot] = make_float4(u[0], u[1], u[2], u[3]);
		ps.fexcl[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
	}
}

// ---------------------------------------------------------------------
// Traversal of a ray buffer (Tracer::trace, tracer/tracer.cpp:38-121)
// ---------------------------------------------------------------------
// n_dev == nullptr: n_host rays.  OCCL: occlusion rays, the result (1 =
// blocked or no ray) goes to wb.occl by position.
//
// Persistent warps with per-lane ray replacement: a lane whose ray is
// finished takes the next ray of the queue between traversal steps instead
// of idling until the slowest ray of its warp is done.  128 registers a
// thread (16 resident warps an SM) hide more latency than the
// register-unbounded variant's 8 warps (measured: +13% on the many-light
// scene, no change on flat scenes).
//
// Scenes with instance levels (the large traversal kernels): one block of
// 512 threads per SM, whose warps run the same kind of work while they
// can.  The kernel is bound by instruction fetch (the lanes of 16 warps
// spread over more code than an SM's instruction cache holds), so a warp
// that has lanes for the kind the block is running runs that kind, and
// only a warp without any takes its own most common kind, which the block
// then follows.  The preference is a shared word read and written without
// synchronisation (a stale value only costs time).  A warp also refills
// its lanes from 4 idle lanes instead of 8.  Measured on the many-light
// render: 11% off the traversal time against blocks of 128 threads that
// each vote alone.  Flat scenes (a small kernel) keep the render's block
// size and the per-warp vote, which are 3-4% faster there.
template <unsigned F>
struct TraceCfg {
	static constexpr bool NESTED = (F & FEAT_NESTED) != 0;
	static constexpr int BLOCK = NESTED ? 512 : 256;      // launch bound (flat: the render's block size)
	static constexpr int MIN_BLOCKS = NESTED ? 1 : 2;
	static constexpr bool FOLLOW = NESTED;                // warps follow the block's kind of work
	static constexpr int REFILL_MIN = NESTED ? 4 : 8;     // idle lanes that trigger a refill while rays remain
	static int launch_block(int render_block) { return NESTED ? BLOCK : render_block; }
};
// Each lane's traversal is cut into kinds of work: node visits (up to
// PSY_WALK_NODES at a time, stopping at a leaf), leaf visits of three
// classes (entering an assembly instance, testing a simple object, starting
// a patch bisection) and bisection iterations (PSY_PATCH_UNITS at a time).
// Each loop iteration of a warp runs the kind that most of its lanes have
// next (leaf visits counted PSY_LEAF_WEIGHT times, bisections
// PSY_PATCH_WEIGHT times), so that the lanes doing the same work run
// together instead of one lane's long bisection or transformed-instance
// entry holding up the others.  (Measured on the many-light render: 4 node
// visits a step 1.4% faster than 8 and 16; 16 bisection iterations and a
// refill threshold of 16 slower than 8.)
#ifndef PSY_WALK_NODES
#define PSY_WALK_NODES 4
#endif
#ifndef PSY_PATCH_UNITS
#define PSY_PATCH_UNITS 8
#endif
#ifndef PSY_PATCH_WEIGHT
#define PSY_PATCH_WEIGHT 1
#endif
#ifndef PSY_LEAF_WEIGHT
#define PSY_LEAF_WEIGHT 1
#endif

template <class W, unsigned F, bool OCCL>
__global__ void __launch_bounds__(TraceCfg<F>::BLOCK, TraceCfg<F>::MIN_BLOCKS) trace_wave_kernel(W w, WaveBufs wb, const float4* __restrict__ rb,
                                                         const int* n_dev, int n_host, int* work,
                                                         unsigned long long* counts, unsigned* status) {
	const int n = n_dev ? *n_dev : n_host;
	const int lane = threadIdx.x & 31;
	const unsigned lt_mask = (1u << lane) - 1u;
	unsigned err = 0;
	// per-lane work counters (TC_*), and the warp's own (lane 0 keeps them)
	unsigned rays = 0, c_nodes = 0, c_leaves = 0, c_iters = 0, c_warp = 0, c_lanes = 0;
	TraceState<F> st;
	int my = -1;    // queue position of this lane's ray, -1 = idle
	int leaf = 0;   // walk_nodes stopped at a leaf (st.leaf): its LEAF_* class, else 0
	int rid = 0;
	bool more = true;  // the queue may still hold rays (warp-uniform)
	__shared__ int s_kind;  // the kind of work the block's warps run
	if (threadIdx.x == 0) s_kind = KIND_NODES;
	__syncthreads();
	while (true) {
		const unsigned idle = __ballot_sync(0xffffffffu, my < 0);
		if (more && (__popc(idle) >= TraceCfg<F>::REFILL_MIN || idle == 0xffffffffu)) {
			int base = 0;
			if (lane == 0) base = atomicAdd(work, __popc(idle));
			base = __shfl_sync(0xffffffffu, base, 0);
			if (base + __popc(idle) >= n) more = false;
			if (my < 0) {
				const int k = base + __popc(idle & lt_mask);
				if (k < n) {
					WorldRayD wr;
					const int tag = load_ray(rb, wb.cap, k, &wr);
					wr.occl = OCCL;
					if (tag & 1) {
						// no ray: a shadow step without a light sample, or a
						// path of a shorter render in a batch that has ended
						if (OCCL) wb.occl[k] = 1;
					} else {
						rid = tag >> 1;
						trace_init<F>(w.scene(rid), st, wr);
						my = k;
						leaf = 0;
						++rays;
					}
				}
			}
		}
		// KIND_IDLE, KIND_NODES (node visits), a leaf visit of one of the
		// LEAF_* classes, or KIND_PATCH (bisection)
		const int kind = my < 0 ? KIND_IDLE : st.pmode != PM_NONE ? KIND_PATCH : leaf ? leaf : KIND_NODES;
		unsigned m[KIND_PATCH + 1];
#pragma unroll
		for (int k = KIND_NODES; k <= KIND_PATCH; ++k) m[k] = __ballot_sync(0xffffffffu, kind == k);
		if ((m[KIND_NODES] | m[LEAF_ENTER] | m[LEAF_SIMPLE] | m[LEAF_PATCH] | m[KIND_PATCH]) == 0u) {
			if (!more) break;
			continue;
		}
		// the block's kind if this warp has lanes for it, else the kind most
		// of its lanes have next (later kinds win ties), which the block takes
		int run = *(volatile int*)&s_kind;
		bool has = false;
		if (TraceCfg<F>::FOLLOW) {
#pragma unroll
			for (int k = KIND_NODES; k <= KIND_PATCH; ++k)
				if (run == k) has = m[k] != 0u;
		}
		if (!has) {
			run = KIND_NODES;
			int best = __popc(m[KIND_NODES]);
#pragma unroll
			for (int k = LEAF_ENTER; k <= KIND_PATCH; ++k) {
				const int c = __popc(m[k]) * (k == KIND_PATCH ? PSY_PATCH_WEIGHT : PSY_LEAF_WEIGHT);
				if (c >= best && c > 0) {
					best = c;
					run = k;
				}
			}
			if (TraceCfg<F>::FOLLOW && lane == 0) *(volatile int*)&s_kind = run;
		}
		++c_warp;
		unsigned runmask = m[KIND_NODES];
#pragma unroll
		for (int k = LEAF_ENTER; k <= KIND_PATCH; ++k)
			if (run == k) runmask = m[k];
		c_lanes += __popc(runmask);
		bool live = true;
		if (kind == run) {
			const DevScene& sc = w.scene(rid);
			if (run == KIND_PATCH) {
				int left = PSY_PATCH_UNITS;
				live = patch_step<F>(sc, st, left);
				c_iters += PSY_PATCH_UNITS - left;
			} else if (run == KIND_NODES) {
				int left = PSY_WALK_NODES;
				const int r = walk_nodes<F>(sc, st, left);
				c_nodes += PSY_WALK_NODES - left;
				live = r != WALK_DONE;
				leaf = r == WALK_LEAF ? leaf_class<F>(sc, st) : 0;
			} else {
				leaf = 0;
				++c_leaves;
				live = leaf_visit<F>(sc, st);
			}
		}
		if (!live) {
			err |= st.err;
			if (OCCL) wb.occl[my] = st.rec.obj >= 0 ? 1 : 0;
			else store_rec(wb, my, st.rec);
			my = -1;
		}
	}
	unsigned long long c[4] = {rays, c_nodes, c_leaves, c_iters};
#pragma unroll
	for (int k = 0; k < 4; ++k)
		for (int o = 16; o > 0; o >>= 1) c[k] += __shfl_down_sync(0xffffffffu, c[k], o);
	if (lane == 0) {
		if (c[0]) atomicAdd(counts + TC_RAYS, c[0]);
		if (c[1]) atomicAdd(counts + TC_NODES, c[1]);
		if (c[2]) atomicAdd(counts + TC_LEAVES, c[2]);
		if (c[3]) atomicAdd(counts + TC_PATCH_ITERS, c[3]);
		if (c_warp) atomicAdd(counts + TC_WARP_STEPS, (unsigned long long)c_warp);
		if (c_lanes) atomicAdd(counts + TC_LANE_STEPS, (unsigned long long)c_lanes);
	}
	if (err) atomicOr(status, err);
}

// ---------------------------------------------------------------------
// After a camera (CAMERA) or bounce ray: update_path
// (path_trace_integrator.cpp:251-272 and 273-302), then the shadow step of
// next_ray_for_path (path_trace_integrator.cpp:126-184).
//
// Registers are capped at PSY_SHADE_MAXNREG a thread.  The kernel waits on
// memory (path state, light-tree nodes, light and shader records) through
// long dependent chains, and with the compiler's choice of about 225
// registers only 8 warps fit an SM; at 32 registers 64 fit, and the spills
// stay in L1.  Measured (640x360x4 many-light frame / flat 20,000- and
// 50,000-primitive renders): 95.2 -> 84.4 ms and 45.2 -> 23.1 and
// 96.5 -> 47.5 ms for the whole render, with caps of 168, 128, 96, 64, 48
// and 40 registers in between.
// ---------------------------------------------------------------------
#ifndef PSY_SHADE_MAXNREG
#define PSY_SHADE_MAXNREG 32
#endif
template <class W, bool CAMERA, unsigned F>
__global__ void __maxnreg__(PSY_SHADE_MAXNREG) shade_hit_kernel(W w, HaltonDev hd, PathSoA ps, WaveBufs wb,
                                                        const int* __restrict__ q_in, const int* n_dev, int n_host,
                                                        int* q_out, int* n_out, int* work, unsigned* status) {
	extern __shared__ float sgrad[];
	if (!W::BATCH) grad_begin(w.render(0), sgrad);
	const int lane = threadIdx.x & 31;
	const int n = n_dev ? *n_dev : n_host;
	unsigned err = 0;
	while (true) {
		const int base = fetch32(work);
		if (base >= n) break;
		const int i = base + lane;
		bool live = false;
		int slot = -1;
		WorldRayD sray;
		int stag = 1;
		WorldRayD wr;
		const int tag = i < n ? load_ray(wb.ray[0], wb.cap, i, &wr) : 1;
		// (tag & 1): the path ended at its own path length before this step
		// (a shorter render of a batch) and is only waiting in the queue
		if (i < n && !(tag & 1)) {
			slot = q_in ? q_in[i] : i;
			const int rid = tag >> 1;
			const DevScene& sc = w.scene(rid);
			const RenderParams& rp = w.render(rid);
			const uint32_t smp = ps.smp[slot];
			const uint32_t ds = ps.dimstep[slot];
			uint32_t dim = ds & 0xffffu;
			uint32_t step = ds >> 16;
			const float wl = ps.wl[slot];
			const float time = ps.time[slot];
			const float last_pdf = ps.last_pdf[slot];
			Spec col = sp(ps.col[slot]);
			const Spec fcol = sp(ps.fcol[slot]);
			HitRec rec;
			load_rec(wb, i, &rec);
			bool done = false;
			StoredHit sh;
			if (rec.obj >= 0) {
				int closure;
				float ecol[3], lpdf;
				make_stored<F>(sc, rec, wr, rp.ident_inv, &sh, &closure, ecol, &lpdf, &err);
				const int vtx = (int)(step >> 1);  // index of this path vertex
				if (closure == CLOSURE_EMIT) {
					done = true;
					Spec e = rgb_to_spec(ecol, wl);
					const int lp = emission_param(rp, rec.obj);
					if (lp >= 0)
						for (int k = 0; k < 4; ++k) e.e[k] *= rp.params[lp];
					Spec C;
					if (!CAMERA && last_pdf != 0.0f) {
						const float mis_inv_pdf = power_heuristic(last_pdf, lpdf) / last_pdf;
						for (int k = 0; k < 4; ++k) C.e[k] = ((fcol.e[k] * last_pdf) * e.e[k]) * mis_inv_pdf;
					} else {
						for (int k = 0; k < 4; ++k) C.e[k] = fcol.e[k] * e.e[k];
					}
					for (int k = 0; k < 4; ++k) col.e[k] += C.e[k];
					if (!W::BATCH && rp.grad) {
						// the same contribution without its parameterised factors
						const Spec e0 = rgb_to_spec(ecol, wl);
						const Spec fx = sp(ps.fexcl[slot]);
						Spec B;
						if (!CAMERA && last_pdf != 0.0f) {
							const float mis_inv_pdf = power_heuristic(last_pdf, lpdf) / last_pdf;
							for (int k = 0; k < 4; ++k) B.e[k] = ((fx.e[k] * last_pdf) * e0.e[k]) * mis_inv_pdf;
						} else {
							for (int k = 0; k < 4; ++k) B.e[k] = fx.e[k] * e0.e[k];
						}
						grad_add(rp, sgrad, ps, slot, vtx, B, lp, wl);
					}
				} else if (closure != CLOSURE_LAMBERT && closure != CLOSURE_GTR) {
					done = true;  // closures outside the supported set end the path
				} else {
					sh.pid = (rp.params && rec.shader >= 0) ? rp.shader_param[rec.shader] : -1;
					if (!W::BATCH && rp.grad && vtx < PSY_ADJ_MAX_VERTS) {
						Spec a = Spec{};
						if (sh.pid >= 0) {
							a = albedo_spec(rp.params + sh.pid, wl);
						} else if (sh.pid < -1) {
							const Spec up = rgb_to_spec(sh.col, wl);
							const float q = rp.params[-2 - sh.pid];
							for (int k = 0; k < 4; ++k) a.e[k] = up.e[k] * q;
							ps.vdsc[slot * PSY_ADJ_MAX_VERTS + vtx] = f4(up);
						}
						ps.vpid[slot * PSY_ADJ_MAX_VERTS + vtx] = sh.pid;
						ps.valb[slot * PSY_ADJ_MAX_VERTS + vtx] = f4(a);
					}
				}
			} else {
				done = true;
				const Spec bg = rgb_to_spec(sc.background, wl);
				for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * bg.e[k];
			}
			step++;
			if (step == rp.path_length * 2) done = true;
			const bool gtr = !done && sh.gtr >= 0;
			const Gtr gp = gtr ? gtr_of(sc.shaders[sh.gtr]) : Gtr{};
			if (done) {
				finish_path(ps, slot, col, wl);
			} else if (gtr && gtr_is_delta(gp)) {
				// a delta closure takes no light sample and no sampler draws;
				// the reference traces the step's ray again, and its result
				// adds nothing (path_trace_integrator.cpp:131-184, 235-249)
				sray = wr;
				sray.occl = true;
				stag = rid << 1;
				ps.dimstep[slot] = (dim & 0xffffu) | (step << 16);
				ps.col[slot] = f4(col);
				ps.lcol[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
				if (!W::BATCH && rp.grad) {
					ps.nee_param[slot] = -1;
					ps.nee_base[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
				}
				store_hit(ps, slot, sh);
				live = true;
			} else {
				// shadow step: light-tree sample and shadow ray
				LightQuery q;
				q.n = sampler_get(hd, smp, dim++);
				q.u = sampler_get(hd, smp, dim++);
				q.v = sampler_get(hd, smp, dim++);
				q.pos = sh.p;
				// lq_nor = geo.n, flipped for back-facing hits
				q.nor = (sh.bf != 0.0f) ? sh.n * -1.0f : sh.n;
				q.d = sh.d;
				q.wavelength = wl;
				q.time = time;
				q.has_xform = false;
				q.id = 0;
				q.obj = -1;
				q.selection_pdf = 1.0f;
				q.light_sample_pdf = 1.0f;
				q.gtr = gtr;
				q.gp = gp;
				light_tree_sample(sc, &q, rp.ident_inv);
				float4 contrib = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
				if (q.valid) {
					const float bsdf_pdf = gtr ? gtr_pdf(gp, sh.d, q.to_light, sh.n) : lambert_pdf(sh.d, q.to_light, sh.n);
					const float mis_inv_pdf = power_heuristic(q.light_sample_pdf, bsdf_pdf) / q.light_sample_pdf;
					const float lc = (float)rp.light_count;
					Spec lcol;
					for (int k = 0; k < 4; ++k) lcol.e[k] = ((q.spec.e[k] * mis_inv_pdf) * lc) / q.selection_pdf;
					const int lp = emission_param(rp, q.obj);
					if (lp >= 0)
						for (int k = 0; k < 4; ++k) lcol.e[k] *= rp.params[lp];
					if (!W::BATCH && rp.grad) ps.nee_param[slot] = lp;
					sray.o = sh.p + sh.off;
					sray.d = (q.to_light - sh.off) * 0.9995f;
					sray.time = time;
					sray.occl = true;
					if (gtr) gtr_propagate_differentials(sh, &sray);
					else propagate_differentials(sh, &sray);
					// the light's contribution if the shadow ray is not blocked
					// (update_path, shadow result: path_trace_integrator.cpp:235-249)
					const Spec fac = gtr ? gtr_eval(gp, sh.d, sray.d, sh.n, wl) : lambert_eval_p(rp, sh, sray.d, wl);
					Spec c;
					for (int k = 0; k < 4; ++k) c.e[k] = (fcol.e[k] * lcol.e[k]) * fac.e[k];
					contrib = f4(c);
					if (!W::BATCH && rp.grad) {
						// without the light's scale and the albedos of parameterised vertices
						const Spec fx = sp(ps.fexcl[slot]);
						const float cs = gtr ? 0.0f : lambert_cos(sh.d, sray.d, sh.n);
						const Spec f0 = sh.pid != -1 ? Spec{{cs, cs, cs, cs}} : fac;
						Spec b;
						for (int k = 0; k < 4; ++k)
							b.e[k] = (fx.e[k] * (((q.spec.e[k] * mis_inv_pdf) * lc) / q.selection_pdf)) * f0.e[k];
						ps.nee_base[slot] = f4(b);
					}
					stag = rid << 1;
				} else {
					err |= ERRF_NOLIGHT;
					sray.o = V3(0.0f); sray.d = V3(0.0f, 0.0f, 1.0f); sray.time = time;
					sray.odx = sray.ody = sray.ddx = sray.ddy = V3(0.0f);
					stag = (rid << 1) | 1;
				}
				ps.dimstep[slot] = (dim & 0xffffu) | (step << 16);
				ps.col[slot] = f4(col);
				ps.lcol[slot] = contrib;
				store_hit(ps, slot, sh);
				live = true;
			}
		}
		// ballot compaction of the live paths into the next queue
		const unsigned m = __ballot_sync(0xffffffffu, live);
		int out_base = 0;
		if (lane == 0 && m) out_base = atomicAdd(n_out, __popc(m));
		out_base = __shfl_sync(0xffffffffu, out_base, 0);
		if (live) {
			const int j = out_base + __popc(m & ((1u << lane) - 1u));
			q_out[j] = slot;
			store_ray(wb.ray[1], wb.cap, j, sray, stag);
		}
	}
	if (!W::BATCH) grad_end(w.render(0), sgrad);
	if (err) atomicOr(status, err);
}

// ---------------------------------------------------------------------
// After the shadow ray: update_path (path_trace_integrator.cpp:235-249),
// then the bounce step of next_ray_for_path (path_trace_integrator.cpp:185-223).
// Paths keep their queue position.
// ---------------------------------------------------------------------
template <class W>
__global__ void __launch_bounds__(256) shade_shadow_kernel(W w, HaltonDev hd, PathSoA ps, WaveBufs wb,
                                                           const int* __restrict__ q_in, const int* n_dev, int* work) {
	extern __shared__ float sgrad[];
	if (!W::BATCH) grad_begin(w.render(0), sgrad);
	const int n = *n_dev;
	while (true) {
		const int base = fetch32(work);
		if (base >= n) break;
		const int i = base + (threadIdx.x & 31);
		if (i >= n) continue;
		const int slot = q_in[i];
		const int rid = W::BATCH ? (int)ps.rid[slot] : 0;
		const uint32_t smp = ps.smp[slot];
		const uint32_t ds = ps.dimstep[slot];
		uint32_t dim = ds & 0xffffu;
		uint32_t step = ds >> 16;
		const float wl = ps.wl[slot];
		Spec col = sp(ps.col[slot]);
		const RenderParams& rp = w.render(rid);
		if (wb.occl[i] == 0) {
			const Spec c = sp(ps.lcol[slot]);
			for (int k = 0; k < 4; ++k) col.e[k] += c.e[k];
			if (!W::BATCH && rp.grad)
				grad_add(rp, sgrad, ps, slot, (int)(step >> 1) + 1, sp(ps.nee_base[slot]), ps.nee_param[slot], wl);
		}
		step++;
		if (step == rp.path_length * 2) {
			finish_path(ps, slot, col, wl);
			// paths of longer renders in the same batch keep going: leave a
			// "no ray" mark so later steps pass over this queue position
			WorldRayD none;
			none.o = none.d = none.odx = none.ody = none.ddx = none.ddy = V3(0.0f);
			none.time = 0.0f;
			store_ray(wb.ray[0], wb.cap, i, none, (rid << 1) | 1);
			continue;
		}
		StoredHit sh;
		load_hit(ps, slot, &sh);
		Spec fcol = sp(ps.fcol[slot]);
		// The reference passes two sampler.next() calls as arguments; g++
		// evaluates them right to left, so the second draw is `si` and the
		// first `sj`.
		const float sj = sampler_get(hd, smp, dim++);
		const float si = sampler_get(hd, smp, dim++);
		WorldRayD wr;
		wr.o = sh.p + sh.off;
		wr.time = ps.time[slot];
		wr.occl = false;
		V3 out;
		float pdf;
		Spec filter;
		bool delta = false;
		if (sh.gtr >= 0) {
			const Gtr gp = gtr_of(w.scene(rid).shaders[sh.gtr]);
			gtr_sample(gp, sh.d, sh.n, si, sj, wl, &out, &filter, &pdf);
			delta = gtr_is_delta(gp);
			wr.d = out;
			gtr_propagate_differentials(sh, &wr);
		} else {
			V3 nn = normalized(sh.n);
			if (dot(nn, sh.d) > 0.0f) nn = nn * -1.0f;
			const V3 dir = cosine_sample_hemisphere(si, sj);
			pdf = dir.z * (float)PSY_INV_PI_D;
			out = zup_to_vec(dir, nn);
			filter = lambert_eval_p(rp, sh, out, wl);
			wr.d = out;
			propagate_differentials(sh, &wr);
		}
		if (!delta) {
			if (pdf < 0.00001f) pdf = 0.00001f;
			for (int k = 0; k < 4; ++k) fcol.e[k] *= filter.e[k] / pdf;
		} else {
			for (int k = 0; k < 4; ++k) fcol.e[k] *= filter.e[k];
			pdf = 0.0f;  // last_pdf 0: the next emitter hit takes no MIS weight
		}
		if (!W::BATCH && rp.grad) {
			// the path weight without the parameterised albedos
			Spec fx = sp(ps.fexcl[slot]);
			const float cs = sh.gtr >= 0 ? 0.0f : lambert_cos(sh.d, out, sh.n);
			for (int k = 0; k < 4; ++k) fx.e[k] *= (sh.pid != -1 ? cs : filter.e[k]) / (delta ? 1.0f : pdf);
			ps.fexcl[slot] = f4(fx);
		}
		store_ray(wb.ray[0], wb.cap, i, wr, rid << 1);
		ps.dimstep[slot] = (dim & 0xffffu) | (step << 16);
		ps.col[slot] = f4(col);
		ps.fcol[slot] = f4(fcol);
		ps.last_pdf[slot] = pdf;
	}
	if (!W::BATCH) grad_end(w.render(0), sgrad);
}

// Adds each pixel's samples, in sample order, to its render's film; rejects
// non-finite samples as Film::add_sample does (film/film.hpp:135-153).
template <class W>
__global__ void film_reduce_kernel(W w, WaveRange wv, PathSoA ps) {
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= wv.pixels) return;
	const uint64_t q = wv.pix_base + (uint64_t)p;
	const RenderParams& rp = w.render(w.render_of_pixel(q));
	const uint64_t pixel = q - rp.pixel_base;
	const uint64_t first = rp.path_base + pixel * rp.spp - wv.base;  // slot of the pixel's first sample
	const float3* s = reinterpret_cast<const float3*>(ps.sample) + first;
	float* xyz = rp.xyz;
	float ax = xyz[pixel * 3], ay = xyz[pixel * 3 + 1], az = xyz[pixel * 3 + 2];
	uint32_t c = 0;
	for (uint32_t k = 0; k < rp.spp; ++k) {
		const float3 v = s[k];
		if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) continue;
		ax += v.x;
		ay += v.y;
		az += v.z;
		++c;
	}
	xyz[pixel * 3] = ax;
	xyz[pixel * 3 + 1] = ay;
	xyz[pixel * 3 + 2] = az;
	if (rp.counts) rp.counts[pixel] += c;
}

// ---------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------
// Persistent grid: resident blocks of `kernel` at `block` threads x SMs.
template <typename K>
static int persistent_grid(K kernel, int block) {
	int dev = 0, sms = 0, b = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, block, 0);
	return sms * (b < 1 ? 1 : b);
}

struct WaveGrids {
	int block = 0;
	int trace_b = 0;  // traversal block size
	int trace_c, trace_o, shade_c, shade_b, shadow;
};

template <class W, unsigned F>
static const WaveGrids& grids_for(int block) {
	// one entry per block size, filled on first use (block sizes 64..256)
	static WaveGrids g[5];
	const int k = block == 64 ? 0 : block == 128 ? 1 : block == 256 ? 2 : 3;
	if (g[k].block != block) {
		WaveGrids n;
		n.block = block;
		n.trace_b = TraceCfg<F>::launch_block(block);
		n.trace_c = persistent_grid(trace_wave_kernel<W, F, false>, n.trace_b);
		n.trace_o = persistent_grid(trace_wave_kernel<W, F, true>, n.trace_b);
		n.shade_c = persistent_grid(shade_hit_kernel<W, true, F>, block);
		n.shade_b = persistent_grid(shade_hit_kernel<W, false, F>, block);
		n.shadow = persistent_grid(shade_shadow_kernel<W>, block);
		g[k] = n;
	}
	return g[k];
}

// Counters per wave: [0] camera trace work, [1] camera shade work, [2]
// live paths after the camera step; then per bounce eight: [0] shadow trace
// work, [1] shadow shade work, [2] bounce trace work, [3] bounce shade work,
// [4] live paths after the bounce.
int render_counter_count(uint32_t path_length) { return 4 + 8 * (int)path_length; }

template <class W, unsigned F>
static void launch_wave(const W& w, uint32_t path_length, const HaltonDev& hd, const WaveRange& wv,
                        const PathSoA& ps, const WaveBufs& wb, const WaveQueues& wq, unsigned* status, int block,
                        size_t gsmem, cudaStream_t st, uint32_t* launches, const LaunchTimer* tm = nullptr) {
	const WaveGrids& g = grids_for<W, F>(block);
	auto tstart = [&]() {
		if (tm && *tm->used < tm->capacity) cudaEventRecord(tm->events[2 * *tm->used], st);
	};
	auto tstop = [&]() {
		if (tm && *tm->used < tm->capacity) cudaEventRecord(tm->events[2 * (*tm->used)++ + 1], st);
	};
	const int P = wv.paths;
	int* c = wq.counters;
	cudaMemsetAsync(c, 0, sizeof(int) * render_counter_count(path_length), st);
	camera_gen_kernel<W><<<(P + block - 1) / block, block, 0, st>>>(w, hd, wv, ps, wb);
	tstart();
	trace_wave_kernel<W, F, false><<<g.trace_c, g.trace_b, 0, st>>>(w, wb, wb.ray[0], nullptr, P, c + 0, wq.rays, status);
	tstop();
	// camera hit -> shadow rays of the live paths into queue 0
	int* q = wq.q0;
	int* n = c + 2;
	shade_hit_kernel<W, true, F><<<g.shade_c, block, gsmem, st>>>(w, hd, ps, wb, nullptr, nullptr, P, q, n, c + 1,
	                                                             status);
	*launches += 3;
	c += 4;
	for (uint32_t b = 0; b < path_length; ++b) {
		tstart();
		trace_wave_kernel<W, F, true><<<g.trace_o, g.trace_b, 0, st>>>(w, wb, wb.ray[1], n, 0, c + 0, wq.rays + TC_COUNT,
		                                                          status);
		tstop();
		shade_shadow_kernel<W><<<g.shadow, block, gsmem, st>>>(w, hd, ps, wb, q, n, c + 1);
		*launches += 2;
		if (b + 1 == path_length) break;  // the last shadow step ends every path
		tstart();
		trace_wave_kernel<W, F, false><<<g.trace_c, g.trace_b, 0, st>>>(w, wb, wb.ray[0], n, 0, c + 2, wq.rays, status);
		tstop();
		int* q2 = (q == wq.q0) ? wq.q1 : wq.q0;
		int* n2 = c + 4;
		shade_hit_kernel<W, false, F><<<g.shade_b, block, gsmem, st>>>(w, hd, ps, wb, q, n, 0, q2, n2, c + 3, status);
		*launches += 2;
		q = q2;
		n = n2;
		c += 8;
	}
	film_reduce_kernel<W><<<(wv.pixels + 127) / 128, 128, 0, st>>>(w, wv, ps);
	++*launches;
}

static int valid_block(int block) { return (block == 64 || block == 128 || block == 256) ? block : 128; }

cudaError_t launch_render_wave(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const WaveRange& wv,
                               const PathSoA& ps, const WaveBufs& wb, const WaveQueues& wq, unsigned* status,
                               int block, cudaStream_t st, uint32_t* launches, const LaunchTimer* timer) {
	PlainWave w;
	w.sc = sc;
	w.rp = rp;
	block = valid_block(block);
	const size_t gsmem = (rp.grad && rp.grad_in_smem) ? sizeof(float) * (size_t)rp.param_count : 0;
	const uint32_t L = rp.path_length;
	switch (feature_variant(sc.features)) {
		case FEAT_FLAT: launch_wave<PlainWave, FEAT_FLAT>(w, L, hd, wv, ps, wb, wq, status, block, gsmem, st, launches, timer); break;
		case FEAT_STILL_BICUBIC: launch_wave<PlainWave, FEAT_STILL_BICUBIC>(w, L, hd, wv, ps, wb, wq, status, block, gsmem, st, launches, timer); break;
		case FEAT_STILL: launch_wave<PlainWave, FEAT_STILL>(w, L, hd, wv, ps, wb, wq, status, block, gsmem, st, launches, timer); break;
		default: launch_wave<PlainWave, FEAT_ALL>(w, L, hd, wv, ps, wb, wq, status, block, gsmem, st, launches, timer); break;
	}
	return cudaGetLastError();
}

cudaError_t launch_batch_wave(const DevScene* scenes, const RenderParams* renders, int count, unsigned features,
                              uint32_t max_path_length, const HaltonDev& hd, const WaveRange& wv, const PathSoA& ps,
                              const WaveBufs& wb, const WaveQueues& wq, unsigned* status, int block,
                              cudaStream_t st, uint32_t* launches) {
	BatchWave w;
	w.scenes = scenes;
	w.renders = renders;
	w.count = count;
	block = valid_block(block);
	if (feature_variant(features) == FEAT_FLAT)
		launch_wave<BatchWave, FEAT_FLAT>(w, max_path_length, hd, wv, ps, wb, wq, status, block, 0, st, launches);
	else
		launch_wave<BatchWave, FEAT_ALL>(w, max_path_length, hd, wv, ps, wb, wq, status, block, 0, st, launches);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------
// Batched LightTree::sample queries (psy_light_sample)
// ---------------------------------------------------------------------
__global__ void light_sample_kernel(DevScene sc, LightQuerySoADev q, LightSampleSoADev o, uint32_t n, float ident_inv,
                                    unsigned* status) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	LightQuery lq;
	lq.n = q.n[i];
	lq.u = q.u[i];
	lq.v = q.v[i];
	lq.pos = V3(q.pos[3 * i], q.pos[3 * i + 1], q.pos[3 * i + 2]);
	lq.nor = V3(q.nor[3 * i], q.nor[3 * i + 1], q.nor[3 * i + 2]);
	lq.d = V3(q.d[3 * i], q.d[3 * i + 1], q.d[3 * i + 2]);
	lq.wavelength = q.wavelength[i];
	lq.time = q.time[i];
	lq.has_xform = false;
	lq.gtr = false;
	lq.id = 0;
	lq.selection_pdf = 1.0f;
	lq.light_sample_pdf = 1.0f;
	light_tree_sample(sc, &lq, ident_inv);
	if (!lq.valid) {
		atomicOr(status, ERRF_NOLIGHT);
		return;
	}
	if (o.to_light) {
		o.to_light[3 * i] = lq.to_light.x;
		o.to_light[3 * i + 1] = lq.to_light.y;
		o.to_light[3 * i + 2] = lq.to_light.z;
	}
	if (o.spec)
		for (int k = 0; k < 4; ++k) o.spec[4 * i + k] = lq.spec.e[k];
	if (o.selection_pdf) o.selection_pdf[i] = lq.selection_pdf;
	if (o.light_pdf) o.light_pdf[i] = lq.light_sample_pdf;
	if (o.id) o.id[i] = lq.id;
}

cudaError_t launch_light_sample(const DevScene& sc, const LightQuerySoADev& q, const LightSampleSoADev& o, uint32_t n,
                                float ident_inv, unsigned* status, cudaStream_t st) {
	if (n == 0) return cudaSuccess;
	light_sample_kernel<<<(n + 127) / 128, 128, 0, st>>>(sc, q, o, n, ident_inv, status);
	return cudaGetLastError();
}

}  // namespace psy
