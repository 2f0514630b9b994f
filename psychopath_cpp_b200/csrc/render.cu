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
//   4: ddy.xyz, flag (1 = no ray: the shadow step found no light sample)
__device__ __forceinline__ void store_ray(float4* rb, int cap, int i, const WorldRayD& r, float flag) {
	rb[i] = make_float4(r.o.x, r.o.y, r.o.z, r.time);
	rb[cap + i] = make_float4(r.d.x, r.d.y, r.d.z, r.odx.x);
	rb[2 * cap + i] = make_float4(r.odx.y, r.odx.z, r.ody.x, r.ody.y);
	rb[3 * cap + i] = make_float4(r.ody.z, r.ddx.x, r.ddx.y, r.ddx.z);
	rb[4 * cap + i] = make_float4(r.ddy.x, r.ddy.y, r.ddy.z, flag);
}
__device__ __forceinline__ float load_ray(const float4* rb, int cap, int i, WorldRayD* r) {
	const float4 a = rb[i], b = rb[cap + i], c = rb[2 * cap + i], d = rb[3 * cap + i], e = rb[4 * cap + i];
	r->o = V3(a.x, a.y, a.z);
	r->time = a.w;
	r->d = V3(b.x, b.y, b.z);
	r->odx = V3(b.w, c.x, c.y);
	r->ody = V3(c.z, c.w, d.x);
	r->ddx = V3(d.y, d.z, d.w);
	r->ddy = V3(e.x, e.y, e.z);
	return e.w;
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
	V3 d, odx, ody, ddx, ddy;  // previous ray
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
	g[3] = make_float4(h.col[2], h.bf, 0.0f, 0.0f);
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
	if (h.closure != CLOSURE_LAMBERT) return;
	M44 inv;
	if (xf) {
		inv = m44_inverse(space);
	} else {
		inv = m44_identity();
		for (int i = 0; i < 4; ++i) inv.m[i][i] = ident_inv;
	}
	sh->p = pos_to(inv, h.geo.p);
	const V3 n = xf ? nor_from(space, h.geo.n) : nor_from(m44_identity(), h.geo.n);
	const float il = 1.0f / length(n);
	sh->n = n * il;
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

__device__ __forceinline__ void finish_path(const PathSoA& ps, int slot, const Spec& col, float wl) {
	float xyz[3];
	spec_to_xyz(col, wl, xyz);
	float3 o;
	o.x = xyz[0] * XYZ_NORM_FAC;
	o.y = xyz[1] * XYZ_NORM_FAC;
	o.z = xyz[2] * XYZ_NORM_FAC;
	reinterpret_cast<float3*>(ps.sample)[slot] = o;
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
__global__ void __launch_bounds__(128) camera_gen_kernel(DevScene sc, HaltonDev hd, RenderParams rp, PathSoA ps,
                                                         WaveBufs wb) {
	const int slot = blockIdx.x * blockDim.x + threadIdx.x;
	if (slot >= rp.wave_paths) return;
	const uint64_t gidx = rp.wave_base + (uint64_t)slot;
	const uint64_t pixel = gidx / rp.spp;
	const uint32_t px = (uint32_t)(pixel % rp.width);
	const uint32_t py = (uint32_t)(pixel / rp.width);
	const uint32_t s = (uint32_t)(gidx % rp.spp);
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
	camera_ray(sc, rx, ry, dx, dy, samp_c, samp_a, samp_b, &wr);
	store_ray(wb.ray[0], wb.cap, slot, wr, 0.0f);
	ps.smp[slot] = smp;
	ps.dimstep[slot] = dim;  // step 0
	ps.wl[slot] = wl;
	ps.time[slot] = wr.time;
	ps.last_pdf[slot] = 0.0f;
	ps.col[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	ps.fcol[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
}

// ---------------------------------------------------------------------
// Traversal of a ray buffer (Tracer::trace, tracer/tracer.cpp:38-121)
// ---------------------------------------------------------------------
// n_dev == nullptr: n_host rays.  OCCL: occlusion rays, the result (1 =
// blocked or no ray) goes to wb.occl by position.
template <unsigned F, bool OCCL>
__global__ void __launch_bounds__(128) trace_wave_kernel(DevScene sc, WaveBufs wb, const float4* __restrict__ rb,
                                                         const int* n_dev, int n_host, int* work,
                                                         unsigned long long* ray_count, unsigned* status) {
	const int n = n_dev ? *n_dev : n_host;
	unsigned err = 0;
	unsigned long long rays = 0;
	while (true) {
		const int base = fetch32(work);
		if (base >= n) break;
		const int i = base + (threadIdx.x & 31);
		if (i < n) {
			WorldRayD wr;
			const float flag = load_ray(rb, wb.cap, i, &wr);
			wr.occl = OCCL;
			if (OCCL && flag != 0.0f) {
				wb.occl[i] = 1;
			} else {
				HitRec rec;
				err |= trace_ray<F>(sc, wr, &rec);
				++rays;
				if (OCCL) wb.occl[i] = rec.obj >= 0 ? 1 : 0;
				else store_rec(wb, i, rec);
			}
		}
	}
	for (int o = 16; o > 0; o >>= 1) rays += __shfl_down_sync(0xffffffffu, rays, o);
	if ((threadIdx.x & 31) == 0 && rays) atomicAdd(ray_count, rays);
	if (err) atomicOr(status, err);
}

// ---------------------------------------------------------------------
// After a camera (CAMERA) or bounce ray: update_path
// (path_trace_integrator.cpp:251-272 and 273-302), then the shadow step of
// next_ray_for_path (path_trace_integrator.cpp:126-184).
// ---------------------------------------------------------------------
template <bool CAMERA, unsigned F>
__global__ void __launch_bounds__(128) shade_hit_kernel(DevScene sc, HaltonDev hd, RenderParams rp, PathSoA ps,
                                                        WaveBufs wb, const int* __restrict__ q_in, const int* n_dev,
                                                        int n_host, int* q_out, int* n_out, int* work,
                                                        unsigned* status) {
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
		float sflag = 1.0f;
		if (i < n) {
			slot = q_in ? q_in[i] : i;
			const uint32_t smp = ps.smp[slot];
			const uint32_t ds = ps.dimstep[slot];
			uint32_t dim = ds & 0xffffu;
			uint32_t step = ds >> 16;
			const float wl = ps.wl[slot];
			const float time = ps.time[slot];
			const float last_pdf = ps.last_pdf[slot];
			Spec col = sp(ps.col[slot]);
			const Spec fcol = sp(ps.fcol[slot]);
			WorldRayD wr;
			load_ray(wb.ray[0], wb.cap, i, &wr);
			HitRec rec;
			load_rec(wb, i, &rec);
			bool done = false;
			StoredHit sh;
			if (rec.obj >= 0) {
				int closure;
				float ecol[3], lpdf;
				make_stored<F>(sc, rec, wr, rp.ident_inv, &sh, &closure, ecol, &lpdf, &err);
				if (closure == CLOSURE_EMIT) {
					done = true;
					const Spec e = rgb_to_spec(ecol, wl);
					if (!CAMERA && last_pdf != 0.0f) {
						const float mis_inv_pdf = power_heuristic(last_pdf, lpdf) / last_pdf;
						for (int k = 0; k < 4; ++k) col.e[k] += ((fcol.e[k] * last_pdf) * e.e[k]) * mis_inv_pdf;
					} else {
						for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * e.e[k];
					}
				} else if (closure != CLOSURE_LAMBERT) {
					done = true;  // closures outside the supported set end the path
				}
			} else {
				done = true;
				const Spec bg = rgb_to_spec(sc.background, wl);
				for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * bg.e[k];
			}
			step++;
			if (step == rp.path_length * 2) done = true;
			if (done) {
				finish_path(ps, slot, col, wl);
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
				q.selection_pdf = 1.0f;
				q.light_sample_pdf = 1.0f;
				light_tree_sample(sc, &q, rp.ident_inv);
				float4 contrib = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
				if (q.valid) {
					const float bsdf_pdf = lambert_pdf(sh.d, q.to_light, sh.n);
					const float mis_inv_pdf = power_heuristic(q.light_sample_pdf, bsdf_pdf) / q.light_sample_pdf;
					const float lc = (float)rp.light_count;
					Spec lcol;
					for (int k = 0; k < 4; ++k) lcol.e[k] = ((q.spec.e[k] * mis_inv_pdf) * lc) / q.selection_pdf;
					sray.o = sh.p + sh.off;
					sray.d = (q.to_light - sh.off) * 0.9995f;
					sray.time = time;
					sray.occl = true;
					propagate_differentials(sh, &sray);
					// the light's contribution if the shadow ray is not blocked
					// (update_path, shadow result: path_trace_integrator.cpp:235-249)
					const Spec fac = lambert_eval(sh.col, sh.d, sray.d, sh.n, wl);
					Spec c;
					for (int k = 0; k < 4; ++k) c.e[k] = (fcol.e[k] * lcol.e[k]) * fac.e[k];
					contrib = f4(c);
					sflag = 0.0f;
				} else {
					err |= ERRF_NOLIGHT;
					sray.o = V3(0.0f); sray.d = V3(0.0f, 0.0f, 1.0f); sray.time = time;
					sray.odx = sray.ody = sray.ddx = sray.ddy = V3(0.0f);
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
			store_ray(wb.ray[1], wb.cap, j, sray, sflag);
		}
	}
	if (err) atomicOr(status, err);
}

// ---------------------------------------------------------------------
// After the shadow ray: update_path (path_trace_integrator.cpp:235-249),
// then the bounce step of next_ray_for_path (path_trace_integrator.cpp:185-223).
// Paths keep their queue position.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(128) shade_shadow_kernel(HaltonDev hd, RenderParams rp, PathSoA ps, WaveBufs wb,
                                                           const int* __restrict__ q_in, const int* n_dev, int* work) {
	const int n = *n_dev;
	while (true) {
		const int base = fetch32(work);
		if (base >= n) break;
		const int i = base + (threadIdx.x & 31);
		if (i >= n) continue;
		const int slot = q_in[i];
		const uint32_t smp = ps.smp[slot];
		const uint32_t ds = ps.dimstep[slot];
		uint32_t dim = ds & 0xffffu;
		uint32_t step = ds >> 16;
		const float wl = ps.wl[slot];
		Spec col = sp(ps.col[slot]);
		if (wb.occl[i] == 0) {
			const Spec c = sp(ps.lcol[slot]);
			for (int k = 0; k < 4; ++k) col.e[k] += c.e[k];
		}
		step++;
		if (step == rp.path_length * 2) {
			finish_path(ps, slot, col, wl);
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
		V3 nn = normalized(sh.n);
		if (dot(nn, sh.d) > 0.0f) nn = nn * -1.0f;
		const V3 dir = cosine_sample_hemisphere(si, sj);
		float pdf = dir.z * (float)PSY_INV_PI_D;
		const V3 out = zup_to_vec(dir, nn);
		const Spec filter = lambert_eval(sh.col, sh.d, out, sh.n, wl);
		WorldRayD wr;
		wr.o = sh.p + sh.off;
		wr.d = out;
		wr.time = ps.time[slot];
		wr.occl = false;
		propagate_differentials(sh, &wr);
		if (pdf < 0.00001f) pdf = 0.00001f;
		for (int k = 0; k < 4; ++k) fcol.e[k] *= filter.e[k] / pdf;
		store_ray(wb.ray[0], wb.cap, i, wr, 0.0f);
		ps.dimstep[slot] = (dim & 0xffffu) | (step << 16);
		ps.col[slot] = f4(col);
		ps.fcol[slot] = f4(fcol);
		ps.last_pdf[slot] = pdf;
	}
}

// Adds each pixel's samples, in sample order, to the film; rejects
// non-finite samples as Film::add_sample does (film/film.hpp:135-153).
__global__ void film_reduce_kernel(RenderParams rp, PathSoA ps, float* xyz, uint32_t* counts) {
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	const int npix = rp.wave_paths / rp.spp;
	if (p >= npix) return;
	const uint64_t pixel = rp.wave_base / rp.spp + (uint64_t)p;
	const float3* s = reinterpret_cast<const float3*>(ps.sample) + (size_t)p * rp.spp;
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
	if (counts) counts[pixel] += c;
}

// ---------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------
template <typename K>
static int resident_blocks(K kernel) {
	int b = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 128, 0);
	return b < 1 ? 1 : b;
}

struct WaveGrids {
	int trace_c, trace_o, shade_c, shade_b, shadow;
};

template <unsigned F>
static WaveGrids grids_for() {
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	WaveGrids g;
	g.trace_c = sms * resident_blocks(trace_wave_kernel<F, false>);
	g.trace_o = sms * resident_blocks(trace_wave_kernel<F, true>);
	g.shade_c = sms * resident_blocks(shade_hit_kernel<true, F>);
	g.shade_b = sms * resident_blocks(shade_hit_kernel<false, F>);
	g.shadow = sms * resident_blocks(shade_shadow_kernel);
	return g;
}

// Counters per wave: [0] camera trace work, [1] camera shade work; per step
// s >= 1 (shadow and bounce pairs) four more; see launch_wave.
int render_counter_count(uint32_t path_length) { return 4 + 8 * (int)path_length; }

template <unsigned F>
static void launch_wave(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const PathSoA& ps,
                        const WaveBufs& wb, const WaveQueues& wq, unsigned* status, cudaStream_t st,
                        uint32_t* launches) {
	static const WaveGrids g = grids_for<F>();
	const int P = rp.wave_paths;
	int* c = wq.counters;
	camera_gen_kernel<<<(P + 127) / 128, 128, 0, st>>>(sc, hd, rp, ps, wb);
	trace_wave_kernel<F, false><<<g.trace_c, 128, 0, st>>>(sc, wb, wb.ray[0], nullptr, P, c + 0, wq.rays, status);
	// camera hit -> shadow rays of the live paths into queue 0
	int* q = wq.q0;
	int* n = c + 2;
	shade_hit_kernel<true, F><<<g.shade_c, 128, 0, st>>>(sc, hd, rp, ps, wb, nullptr, nullptr, P, q, n, c + 1, status);
	*launches += 3;
	c += 4;
	for (uint32_t b = 0; b < rp.path_length; ++b) {
		trace_wave_kernel<F, true><<<g.trace_o, 128, 0, st>>>(sc, wb, wb.ray[1], n, 0, c + 0, wq.rays, status);
		shade_shadow_kernel<<<g.shadow, 128, 0, st>>>(hd, rp, ps, wb, q, n, c + 1);
		*launches += 2;
		if (b + 1 == rp.path_length) break;  // the last shadow step ends every path
		trace_wave_kernel<F, false><<<g.trace_c, 128, 0, st>>>(sc, wb, wb.ray[0], n, 0, c + 2, wq.rays, status);
		int* q2 = (q == wq.q0) ? wq.q1 : wq.q0;
		int* n2 = c + 4;
		shade_hit_kernel<false, F><<<g.shade_b, 128, 0, st>>>(sc, hd, rp, ps, wb, q, n, 0, q2, n2, c + 3, status);
		*launches += 2;
		q = q2;
		n = n2;
		c += 8;
	}
}

cudaError_t launch_render_wave(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const PathSoA& ps,
                               const WaveBufs& wb, const WaveQueues& wq, float* xyz, uint32_t* counts,
                               unsigned* status, cudaStream_t st, uint32_t* launches) {
	cudaMemsetAsync(wq.counters, 0, sizeof(int) * render_counter_count(rp.path_length), st);
	switch (feature_variant(sc.features)) {
		case FEAT_FLAT: launch_wave<FEAT_FLAT>(sc, hd, rp, ps, wb, wq, status, st, launches); break;
		case FEAT_STILL: launch_wave<FEAT_STILL>(sc, hd, rp, ps, wb, wq, status, st, launches); break;
		default: launch_wave<FEAT_ALL>(sc, hd, rp, ps, wb, wq, status, st, launches); break;
	}
	film_reduce_kernel<<<(rp.wave_paths / rp.spp + 127) / 128, 128, 0, st>>>(rp, ps, xyz, counts);
	++*launches;
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
