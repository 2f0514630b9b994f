/*
 * Wavefront path tracer: PathTraceIntegrator::integrate restated for the
 * GPU (reference integrator/path_trace_integrator.cpp:91-384).
 *
 * The reference renders a bucket as a stream of paths and loops
 *   generate one ray per live path -> Tracer::trace -> update -> partition.
 * Here a wave of paths lives in HBM as SoA state; each step of the loop is
 * one persistent kernel over the wave's live-path queue that generates the
 * path's ray (camera / shadow / bounce), traces it, updates the path, and
 * appends still-live paths to the next queue with one atomic per warp
 * (ballot + popc compaction).  Finished paths write their film sample
 * (Color_XYZ(col) * XYZ_NORM_FAC); a per-wave reduction adds each pixel's
 * samples in sample order.
 */
#include "kernels.h"
#include "render_device.cuh"

namespace psy {

enum : int { STEP_CAMERA = 0, STEP_SHADOW = 1, STEP_BOUNCE = 2 };

__device__ __forceinline__ float4 f4(const Spec& s) { return make_float4(s.e[0], s.e[1], s.e[2], s.e[3]); }
__device__ __forceinline__ Spec sp(float4 v) {
	Spec s;
	s.e[0] = v.x; s.e[1] = v.y; s.e[2] = v.z; s.e[3] = v.w;
	return s;
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

__device__ __forceinline__ void finish_path(const RenderParams& rp, const PathSoA& ps, int slot, const Spec& col,
                                            float wl) {
	float xyz[3];
	spec_to_xyz(col, wl, xyz);
	float3 o;
	o.x = xyz[0] * XYZ_NORM_FAC;
	o.y = xyz[1] * XYZ_NORM_FAC;
	o.z = xyz[2] * XYZ_NORM_FAC;
	reinterpret_cast<float3*>(ps.sample)[slot] = o;
}

template <int KIND, unsigned F>
__global__ void __launch_bounds__(128) step_kernel(DevScene sc, HaltonDev hd, RenderParams rp, PathSoA ps,
                                                  const int* __restrict__ q_in, const int* n_in, int* q_out,
                                                  int* n_out, int* work, unsigned long long* ray_count,
                                                  unsigned* status) {
	const int lane = threadIdx.x & 31;
	const int n = (KIND == STEP_CAMERA) ? rp.wave_paths : *n_in;
	unsigned err = 0;
	unsigned long long rays = 0;
	while (true) {
		int base;
		if (lane == 0) base = atomicAdd(work, 32);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n) break;
		const int i = base + lane;
		bool live = false;
		int slot = -1;
		if (i < n) {
			slot = (KIND == STEP_CAMERA) ? i : q_in[i];
			// ---- load path state
			uint32_t smp, dim, step;
			float wl, time, last_pdf;
			Spec col, fcol, lcol;
			const uint32_t pix = ps.pix[slot];
			const uint32_t px = pix & 0xffffu, py = pix >> 16;
			if (KIND == STEP_CAMERA) {
				const uint64_t gidx = rp.wave_base + (uint64_t)slot;
				const uint32_t s = (uint32_t)(gidx % rp.spp);
				smp = sampler_offset(px, py, s, rp.seed);
				dim = 0;
				step = 0;
				wl = (sampler_get(hd, smp, dim++) * (WAVELENGTH_MAX - WAVELENGTH_MIN)) + WAVELENGTH_MIN;
				time = 0.0f;
				last_pdf = 0.0f;
				for (int k = 0; k < 4; ++k) {
					col.e[k] = 0.0f;
					fcol.e[k] = 1.0f;
					lcol.e[k] = 0.0f;
				}
			} else {
				smp = ps.smp[slot];
				const uint32_t ds = ps.dimstep[slot];
				dim = ds & 0xffffu;
				step = ds >> 16;
				wl = ps.wl[slot];
				time = ps.time[slot];
				last_pdf = ps.last_pdf[slot];
				col = sp(ps.col[slot]);
				fcol = sp(ps.fcol[slot]);
				lcol = sp(ps.lcol[slot]);
			}
			StoredHit sh;
			if (KIND != STEP_CAMERA) load_hit(ps, slot, &sh);
			bool done = false;

			if (KIND == STEP_CAMERA) {
				// next_ray_for_path, step 0 (path_trace_integrator.cpp:109-125)
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
				time = wr.time;
				HitRec rec;
				err |= trace_ray<F>(sc, wr, &rec);
				++rays;
				// update_path for a camera ray (path_trace_integrator.cpp:251-272)
				if (rec.obj >= 0) {
					int closure;
					float ecol[3], lpdf;
					make_stored<F>(sc, rec, wr, rp.ident_inv, &sh, &closure, ecol, &lpdf, &err);
					if (closure == CLOSURE_EMIT) {
						done = true;
						const Spec e = rgb_to_spec(ecol, wl);
						for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * e.e[k];
					} else if (closure != CLOSURE_LAMBERT) {
						done = true;  // closures outside the supported set end the path
					}
				} else {
					done = true;
					const Spec bg = rgb_to_spec(sc.background, wl);
					for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * bg.e[k];
				}
			} else if (KIND == STEP_SHADOW) {
				// next_ray_for_path, shadow step (path_trace_integrator.cpp:126-184)
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
				if (q.valid) {
					const float bsdf_pdf = lambert_pdf(sh.d, q.to_light, sh.n);
					const float mis_inv_pdf = power_heuristic(q.light_sample_pdf, bsdf_pdf) / q.light_sample_pdf;
					const float lc = (float)rp.light_count;
					for (int k = 0; k < 4; ++k) lcol.e[k] = ((q.spec.e[k] * mis_inv_pdf) * lc) / q.selection_pdf;
					WorldRayD wr;
					wr.o = sh.p + sh.off;
					wr.d = (q.to_light - sh.off) * 0.9995f;
					wr.time = time;
					wr.occl = true;
					propagate_differentials(sh, &wr);
					HitRec rec;
					err |= trace_ray<F>(sc, wr, &rec);
					++rays;
					// update_path, shadow result (path_trace_integrator.cpp:235-249)
					if (rec.obj < 0) {
						const Spec fac = lambert_eval(sh.col, sh.d, wr.d, sh.n, wl);
						for (int k = 0; k < 4; ++k) col.e[k] += (fcol.e[k] * lcol.e[k]) * fac.e[k];
					}
				} else {
					err |= ERRF_NOLIGHT;
				}
			} else {
				// next_ray_for_path, bounce step (path_trace_integrator.cpp:185-223).  The
				// reference passes two sampler.next() calls as arguments; g++ evaluates
				// them right to left, so the second draw is `si` and the first `sj`.
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
				wr.time = time;
				wr.occl = false;
				propagate_differentials(sh, &wr);
				if (pdf < 0.00001f) pdf = 0.00001f;
				for (int k = 0; k < 4; ++k) fcol.e[k] *= filter.e[k] / pdf;
				last_pdf = pdf;
				HitRec rec;
				err |= trace_ray<F>(sc, wr, &rec);
				++rays;
				if (rec.obj >= 0) {
					int closure;
					float ecol[3], lpdf;
					StoredHit nh;
					make_stored<F>(sc, rec, wr, rp.ident_inv, &nh, &closure, ecol, &lpdf, &err);
					if (closure == CLOSURE_EMIT) {
						done = true;
						const Spec e = rgb_to_spec(ecol, wl);
						if (last_pdf != 0.0f) {
							const float mis_inv_pdf = power_heuristic(last_pdf, lpdf) / last_pdf;
							for (int k = 0; k < 4; ++k) col.e[k] += ((fcol.e[k] * last_pdf) * e.e[k]) * mis_inv_pdf;
						} else {
							for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * e.e[k];
						}
					} else if (closure == CLOSURE_LAMBERT) {
						sh = nh;
					} else {
						done = true;
					}
				} else {
					done = true;
					const Spec bg = rgb_to_spec(sc.background, wl);
					for (int k = 0; k < 4; ++k) col.e[k] += fcol.e[k] * bg.e[k];
				}
			}
			step++;
			if (step == rp.path_length * 2) done = true;

			if (done) {
				finish_path(rp, ps, slot, col, wl);
			} else {
				ps.smp[slot] = smp;
				ps.dimstep[slot] = (dim & 0xffffu) | (step << 16);
				ps.wl[slot] = wl;
				ps.time[slot] = time;
				ps.last_pdf[slot] = last_pdf;
				ps.col[slot] = f4(col);
				ps.fcol[slot] = f4(fcol);
				ps.lcol[slot] = f4(lcol);
				if (KIND != STEP_SHADOW) {
					store_hit(ps, slot, sh);
				}
				live = true;
			}
		}
		// ballot compaction of the live paths into the next queue
		const unsigned m = __ballot_sync(0xffffffffu, live);
		int out_base = 0;
		if (lane == 0 && m) out_base = atomicAdd(n_out, __popc(m));
		out_base = __shfl_sync(0xffffffffu, out_base, 0);
		if (live) q_out[out_base + __popc(m & ((1u << lane) - 1u))] = slot;
	}
	// warp-aggregated ray count
	for (int o = 16; o > 0; o >>= 1) rays += __shfl_down_sync(0xffffffffu, rays, o);
	if (lane == 0 && rays) atomicAdd(ray_count, rays);
	if (err) atomicOr(status, err);
}

// Pixel coordinates of every path slot of a wave (paths are ordered pixel
// by pixel, samples innermost).
__global__ void pix_init_kernel(RenderParams rp, PathSoA ps) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= rp.wave_paths) return;
	const uint64_t gidx = rp.wave_base + (uint64_t)i;
	const uint64_t pixel = gidx / rp.spp;
	const uint32_t x = (uint32_t)(pixel % rp.width);
	const uint32_t y = (uint32_t)(pixel / rp.width);
	ps.pix[i] = x | (y << 16);
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

template <unsigned F>
static int grid_for() {
	int dev = 0, sms = 0, b0 = 0, b1 = 0, b2 = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, step_kernel<STEP_CAMERA, F>, 128, 0);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, step_kernel<STEP_SHADOW, F>, 128, 0);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, step_kernel<STEP_BOUNCE, F>, 128, 0);
	int b = b0;
	if (b1 > 0 && b1 < b) b = b1;
	if (b2 > 0 && b2 < b) b = b2;
	if (b < 1) b = 1;
	return sms * b;
}

int render_grid(unsigned features) { return features == FEAT_FLAT ? grid_for<FEAT_FLAT>() : grid_for<FEAT_ALL>(); }

template <unsigned F>
static void launch_steps(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const PathSoA& ps,
                         const WaveQueues& wq, unsigned* status, int grid, cudaStream_t st, uint32_t* launches) {
	int* n_prev = nullptr;
	const int* q_prev = nullptr;
	for (int s = 0; s < (int)rp.path_length * 2; ++s) {
		int* q_out = (s & 1) ? wq.q1 : wq.q0;
		int* n_out = wq.counters + 2 * s;
		int* work = wq.counters + 2 * s + 1;
		if (s == 0)
			step_kernel<STEP_CAMERA, F><<<grid, 128, 0, st>>>(sc, hd, rp, ps, nullptr, nullptr, q_out, n_out, work,
			                                                   wq.rays, status);
		else if (s & 1)
			step_kernel<STEP_SHADOW, F><<<grid, 128, 0, st>>>(sc, hd, rp, ps, q_prev, n_prev, q_out, n_out, work,
			                                                   wq.rays, status);
		else
			step_kernel<STEP_BOUNCE, F><<<grid, 128, 0, st>>>(sc, hd, rp, ps, q_prev, n_prev, q_out, n_out, work,
			                                                   wq.rays, status);
		++*launches;
		q_prev = q_out;
		n_prev = n_out;
	}
}

cudaError_t launch_render_wave(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const PathSoA& ps,
                               const WaveQueues& wq, float* xyz, uint32_t* counts, unsigned* status, int grid,
                               cudaStream_t st, uint32_t* launches) {
	pix_init_kernel<<<(rp.wave_paths + 255) / 256, 256, 0, st>>>(rp, ps);
	++*launches;
	cudaMemsetAsync(wq.counters, 0, sizeof(int) * 2 * (rp.path_length * 2 + 1), st);
	if (sc.features == FEAT_FLAT) launch_steps<FEAT_FLAT>(sc, hd, rp, ps, wq, status, grid, st, launches);
	else launch_steps<FEAT_ALL>(sc, hd, rp, ps, wq, status, grid, st, launches);
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
