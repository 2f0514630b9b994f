/*
 * Test infrastructure: a C entry surface over the reference renderer's own
 * code, compiled unchanged from the reference sources into
 * oracle/_ref/libpsyref.so by oracle/Makefile.  Only tests/, the smoke check
 * and the benchmark's CPU-baseline leg load it, and only as the checker.
 *
 * Every function wraps a reference call site:
 *   psyref_load       Parser::parse_next_frame + Scene::finalize (parser/parser.cpp:37, scene/scene.hpp:50)
 *   psyref_render     PathTraceIntegrator::integrate (integrator/path_trace_integrator.cpp:28)
 *   psyref_trace      Tracer::trace (tracer/tracer.cpp:38)
 *   psyref_light_sample  LightTree::sample (accel/light_tree.cpp:30)
 *   psyref_camera_ray Camera::generate_ray (basics/camera.hpp:72)
 *   psyref_halton / psyref_sampler  Halton::sample, Sampler::get_sample (sampling/)
 *   psyref_eval       small scalar helpers (spectral upsampling, CIE curves, ...)
 *   psyref_bvh4_* / psyref_lighttree_*  dumps of the built acceleration structures
 */
#include <atomic>
#include <cassert>
#include <chrono>
#include <deque>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <mutex>
#include <random>
#include <regex>
#include <tuple>
#include <unordered_map>
#include <fcntl.h>
#include <unistd.h>

// The oracle reads private members of the reference classes (render settings
// held by Renderer, built BVH4/LightTree nodes) without modifying them.
#define private public
#define protected public
#include "parser.hpp"
#include "renderer.hpp"
#include "scene.hpp"
#include "film.hpp"
#include "tracer.hpp"
#include "path_trace_integrator.hpp"
#include "light_tree.hpp"
#include "bvh4.hpp"
#include "halton.hpp"
#include "image_sampler.hpp"
#include "color.hpp"
#include "monte_carlo.hpp"
#include "surface_closure.hpp"
#include "config.hpp"
#include "global.hpp"
#undef private
#undef protected

namespace {

struct RefScene {
	std::unique_ptr<Renderer> renderer;
	Scene* scene = nullptr;
	std::vector<const Assembly*> assemblies;  // depth-first pre-order, root first
};

void collect_assemblies(const Assembly* a, std::vector<const Assembly*>* out) {
	out->push_back(a);
	for (const auto& sub : a->assemblies) {
		collect_assemblies(sub.get(), out);
	}
}

// Temporarily silences stdout (the integrator prints progress per bucket).
struct QuietStdout {
	int saved = -1;
	QuietStdout() {
		std::cout.flush();
		fflush(stdout);
		saved = dup(1);
		int devnull = open("/dev/null", O_WRONLY);
		if (devnull >= 0) {
			dup2(devnull, 1);
			close(devnull);
		}
	}
	~QuietStdout() {
		std::cout.flush();
		fflush(stdout);
		if (saved >= 0) {
			dup2(saved, 1);
			close(saved);
		}
	}
};

// The closures keep their colour as the first (class-private) member, right
// after the vtable pointer (reference shading/surface_closure.hpp:186,233,339).
void closure_colour(const SurfaceClosure* c, float* col) {
	std::memcpy(col, reinterpret_cast<const char*>(c) + sizeof(void*), 3 * sizeof(float));
}

// Closure kind codes shared with the tests: 0 none, 1 Lambert, 2 Emit, 3 GTR.
int closure_kind(const SurfaceClosure* c, float* col) {
	int kind = 0;
	if (dynamic_cast<const LambertClosure*>(c)) kind = 1;
	else if (dynamic_cast<const EmitClosure*>(c)) kind = 2;
	else if (dynamic_cast<const GTRClosure*>(c)) kind = 3;
	if (kind) closure_colour(c, col);
	else col[0] = col[1] = col[2] = 0.0f;
	return kind;
}

// Layout mirror of LightTree (reference accel/light_tree.hpp:7-31), whose
// data members are class-private by default.
struct LightTreeNodeMirror {
	std::vector<BBox> bounds;
	float energy;
	size_t index1;
	size_t index2;
	bool is_leaf;
	size_t instance_index;
};
struct LightTreeBuildNodeMirror {
	size_t instance_index;
	Vec3 center;
	BBox bbox;
	float energy;
};
struct LightTreeMirror {
	void* vptr;
	const Assembly* assembly;
	std::vector<LightTreeBuildNodeMirror> build_nodes;
	std::vector<LightTreeNodeMirror> nodes;
	std::vector<BBox> bounds_;
	float total_energy;
	size_t total_lights;
};
static_assert(sizeof(LightTreeMirror) == sizeof(LightTree), "LightTree layout changed");

const LightTreeMirror& lt_view(const LightTree& lt) {
	return *reinterpret_cast<const LightTreeMirror*>(&lt);
}

} // namespace

extern "C" {

/* Number of floats written per intersection by psyref_trace. */
int psyref_hit_floats() { return 48; }

void* psyref_load(const char* path) {
	RefScene* rs = new RefScene();
	{
		QuietStdout q;
		Parser parser(path);
		rs->renderer = parser.parse_next_frame();
	}
	if (!rs->renderer) {
		delete rs;
		return nullptr;
	}
	rs->scene = rs->renderer->scene.get();
	rs->scene->finalize();
	collect_assemblies(rs->scene->root.get(), &rs->assemblies);
	return rs;
}

void psyref_free(void* h) {
	delete static_cast<RefScene*>(h);
}

void psyref_info(void* h, int* res_x, int* res_y, int* spp, int* seed) {
	RefScene* rs = static_cast<RefScene*>(h);
	*res_x = (int)rs->renderer->res_x;
	*res_y = (int)rs->renderer->res_y;
	*spp = (int)rs->renderer->spp;
	*seed = (int)rs->renderer->seed;
}

float psyref_get_dice_rate() { return Config::dice_rate; }
void psyref_set_dice_rate(float r) { Config::dice_rate = r; }

/*
 * Renders the scene with the reference integrator.  xyz receives the film's
 * per-pixel XYZ sums (w*h*3, row-major, each sample already scaled by
 * XYZ_NORM_FAC), counts the per-pixel sample counts.
 */
int psyref_render(void* h, int threads, int spp, int path_length, int seed,
                  float* xyz, uint32_t* counts, uint64_t* rays_shot, double* seconds) {
	RefScene* rs = static_cast<RefScene*>(h);
	const int w = (int)rs->renderer->res_x;
	const int ht = (int)rs->renderer->res_y;
	if (spp <= 0) spp = (int)rs->renderer->spp;
	if (seed < 0) seed = (int)rs->renderer->seed;
	Film film(w, ht, -1.0, -((static_cast<float>(ht)) / w), 1.0, ((static_cast<float>(ht)) / w));
	Global::Stats::clear();
	PathTraceIntegrator integrator(rs->scene, &film, spp, spp, 0.0f, (uint)seed, threads, std::function<void()>());
	if (path_length > 0) integrator.path_length = path_length;
	auto t0 = std::chrono::steady_clock::now();
	{
		QuietStdout q;
		integrator.integrate();
	}
	auto t1 = std::chrono::steady_clock::now();
	if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
	if (rays_shot) *rays_shot = Global::Stats::rays_shot;
	for (int y = 0; y < ht; ++y) {
		for (int x = 0; x < w; ++x) {
			const Color_XYZ c = film.pixels(x, y);
			const size_t i = (size_t)y * w + x;
			if (xyz) {
				xyz[i * 3 + 0] = c.x;
				xyz[i * 3 + 1] = c.y;
				xyz[i * 3 + 2] = c.z;
			}
			if (counts) counts[i] = film.accum(x, y);
		}
	}
	return 0;
}

/*
 * Film::scanline_image_8bbc (film/film.hpp:173-225) of a film holding the
 * given per-pixel XYZ sums and sample counts (w*h*3 floats, w*h counts,
 * scanline order), with the film's own dither; out: w*h*3 bytes.
 */
void psyref_film_srgb8(const float* xyz, const uint32_t* counts, int w, int ht, uint8_t* out) {
	Film film(w, ht, -1.0, -((static_cast<float>(ht)) / w), 1.0, ((static_cast<float>(ht)) / w));
	for (int y = 0; y < ht; ++y) {
		for (int x = 0; x < w; ++x) {
			const size_t i = (size_t)y * w + x;
			film.pixels(x, y) = Color_XYZ();
			film.pixels(x, y).x = xyz[3 * i];
			film.pixels(x, y).y = xyz[3 * i + 1];
			film.pixels(x, y).z = xyz[3 * i + 2];
			film.accum(x, y) = counts[i];
		}
	}
	const std::vector<uint8_t> im = film.scanline_image_8bbc();
	std::copy(im.begin(), im.end(), out);
}

/*
 * Traces n world rays through Tracer::trace, in chunks of `chunk` rays (the
 * reference's own streams are about 65,536 long), on `threads` threads with
 * one Tracer each.
 *   rays:  n*19 floats: o(3) d(3) odx(3) ody(3) ddx(3) ddy(3) time
 *   types: n WorldRay::Type values (1 camera, 2 diffuse, 32 occlusion, ...)
 *   hit:   n bytes; id: n uint64 instance ids; out: n*48 floats (see below)
 * out layout: 0 t, 1 u, 2 v, 3-5 p, 6-8 n, 9-11 dpdu, 12-14 dpdv, 15-17 dndu,
 * 18-20 dndv, 21 backfacing, 22 light_pdf, 23-25 offset, 26-41 space matrix
 * (row-major), 42 closure kind, 43-45 closure colour, 46 closure_prob.
 * Returns seconds spent inside Tracer::trace (max over threads).
 */
double psyref_trace(void* h, size_t n, const float* rays, const uint16_t* types, int threads, size_t chunk,
                    uint8_t* hit, uint64_t* id, float* out) {
	RefScene* rs = static_cast<RefScene*>(h);
	if (threads < 1) threads = 1;
	if (chunk == 0) chunk = 65536;
	const size_t nchunks = (n + chunk - 1) / chunk;
	std::atomic<size_t> next_chunk(0);
	std::vector<double> secs(threads, 0.0);
	auto worker = [&](int ti) {
		Tracer tracer(rs->scene);
		std::vector<WorldRay> wr;
		std::vector<Intersection> inter;
		while (true) {
			const size_t c = next_chunk.fetch_add(1);
			if (c >= nchunks) break;
			const size_t b = c * chunk;
			const size_t e = std::min(n, b + chunk);
			wr.resize(e - b);
			inter.resize(e - b);
			for (size_t i = b; i < e; ++i) {
				const float* r = rays + i * 19;
				WorldRay& w = wr[i - b];
				w.o = Vec3(r[0], r[1], r[2]);
				w.d = Vec3(r[3], r[4], r[5]);
				w.odx = Vec3(r[6], r[7], r[8]);
				w.ody = Vec3(r[9], r[10], r[11]);
				w.ddx = Vec3(r[12], r[13], r[14]);
				w.ddy = Vec3(r[15], r[16], r[17]);
				w.time = r[18];
				w.type = static_cast<WorldRay::Type>(types[i]);
			}
			auto t0 = std::chrono::steady_clock::now();
			tracer.trace(&(*wr.begin()), &(*wr.begin()) + wr.size(), &(*inter.begin()), &(*inter.begin()) + inter.size());
			auto t1 = std::chrono::steady_clock::now();
			secs[ti] += std::chrono::duration<double>(t1 - t0).count();
			for (size_t i = b; i < e; ++i) {
				const Intersection& it = inter[i - b];
				if (hit) hit[i] = it.hit ? 1 : 0;
				if (id) id[i] = it.hit ? it.id.id : 0;
				if (!out) continue;
				float* o = out + i * 48;
				std::fill(o, o + 48, 0.0f);
				o[0] = it.t;
				if (!it.hit || types[i] == WorldRay::OCCLUSION) continue;
				const DifferentialGeometry& g = it.geo;
				o[1] = g.u; o[2] = g.v;
				for (int k = 0; k < 3; ++k) {
					o[3 + k] = g.p[k]; o[6 + k] = g.n[k];
					o[9 + k] = g.dpdu[k]; o[12 + k] = g.dpdv[k];
					o[15 + k] = g.dndu[k]; o[18 + k] = g.dndv[k];
					o[23 + k] = it.offset[k];
				}
				o[21] = it.backfacing ? 1.0f : 0.0f;
				o[22] = it.light_pdf;
				for (int r = 0; r < 4; ++r)
					for (int cc = 0; cc < 4; ++cc) o[26 + r * 4 + cc] = it.space.to[r][cc];
				o[42] = (float)closure_kind(it.surface_closure.get(), o + 43);
				o[46] = it.closure_prob;
			}
		}
	};
	std::vector<std::thread> pool;
	for (int t = 0; t < threads; ++t) pool.emplace_back(worker, t);
	for (auto& t : pool) t.join();
	return *std::max_element(secs.begin(), secs.end());
}

/*
 * LightTree::sample of the root assembly for n queries.
 *   q:   n*15 floats: n u v pos(3) nor(3) d(3) wavelength time, lambert_flag
 *   out: n*14 floats: to_light(3) spec_samp e(4) hero selection_pdf
 *        light_sample_pdf, light_count, pad(3)
 *   ids: n uint64
 */
void psyref_light_sample(void* h, size_t n, const float* q, float* out, uint64_t* ids) {
	RefScene* rs = static_cast<RefScene*>(h);
	LambertClosure lambert(Color(0.5f));
	for (size_t i = 0; i < n; ++i) {
		const float* a = q + i * 15;
		LightQuery lq {a[0], a[1], a[2], 0.0f,
		               Vec3(a[3], a[4], a[5]), Vec3(a[6], a[7], a[8]), Vec3(a[9], a[10], a[11]),
		               &lambert, a[12], a[13], Transform()};
		lq.selection_pdf = 1.0f;
		lq.light_sample_pdf = 1.0f;
		lq.id.clear();
		rs->scene->root->light_accel.sample(&lq);
		float* o = out + i * 14;
		for (int k = 0; k < 3; ++k) o[k] = lq.to_light[k];
		for (int k = 0; k < 4; ++k) o[3 + k] = lq.spec_samp.e[k];
		o[7] = lq.spec_samp.hero_wavelength;
		o[8] = lq.selection_pdf;
		o[9] = lq.light_sample_pdf;
		o[10] = (float)rs->scene->root->light_accel.light_count();
		o[11] = o[12] = o[13] = 0.0f;
		if (ids) ids[i] = lq.id.id;
	}
}

/*
 * Camera::generate_ray for n argument tuples (x y dx dy time u v);
 * writes n*19 floats in the psyref_trace ray layout.
 */
void psyref_camera_ray(void* h, size_t n, const float* args, float* rays) {
	RefScene* rs = static_cast<RefScene*>(h);
	for (size_t i = 0; i < n; ++i) {
		const float* a = args + i * 7;
		WorldRay w = rs->scene->camera->generate_ray(a[0], a[1], a[2], a[3], a[4], a[5], a[6]);
		float* r = rays + i * 19;
		for (int k = 0; k < 3; ++k) {
			r[k] = w.o[k]; r[3 + k] = w.d[k]; r[6 + k] = w.odx[k];
			r[9 + k] = w.ody[k]; r[12 + k] = w.ddx[k]; r[15 + k] = w.ddy[k];
		}
		r[18] = w.time;
	}
}

void psyref_halton(size_t n, const uint32_t* dims, const uint32_t* idx, float* out) {
	for (size_t i = 0; i < n; ++i) out[i] = Halton::sample(dims[i], idx[i]);
}

/* Sampler(x, y, s, seed) then `count` calls of next(). */
void psyref_sampler(uint32_t x, uint32_t y, uint32_t s, uint32_t seed, int count, float* out, uint32_t* offset) {
	Sampler smp(x, y, s, seed);
	if (offset) *offset = smp.offset;
	for (int i = 0; i < count; ++i) out[i] = smp.next();
}

/*
 * Scalar helpers, one function id per reference routine:
 *   0 Color_to_SpectralSample(rgb, wavelength) -> e(4)     in: r g b wl
 *   1 Color_XYZ(SpectralSample)                -> xyz(3)   in: e0..e3 wl
 *   2 fast_logit(p, 1.5)                       -> 1        in: p
 *   3 square_to_circle(x, y)                   -> 2        in: x y
 *   4 cosine_sample_hemisphere(u, v)           -> 3        in: u v
 *   5 sphere_lambert(nlcos, rcos)              -> 1        in: nlcos rcos
 *   6 wavelength_n(hero, i) for i=0..3         -> 4        in: hero
 *   7 zup_to_vec(from, toz)                    -> 3        in: from(3) toz(3)
 *   8 Matrix44::inverse                        -> 16       in: m(16)
 *   9 XYZ_to_sRGB_E(xyz)                       -> 3        in: x y z
 * `in_stride`/`out_stride` are the per-item float counts.
 */
void psyref_eval(int fn, size_t n, const float* in, int in_stride, float* out, int out_stride) {
	for (size_t i = 0; i < n; ++i) {
		const float* a = in + i * in_stride;
		float* o = out + i * out_stride;
		switch (fn) {
			case 0: {
				SpectralSample s = Color_to_SpectralSample(Color(a[0], a[1], a[2]), a[3]);
				for (int k = 0; k < 4; ++k) o[k] = s.e[k];
				break;
			}
			case 1: {
				SpectralSample s(a[4]);
				for (int k = 0; k < 4; ++k) s.e[k] = a[k];
				Color_XYZ c(s);
				o[0] = c.x; o[1] = c.y; o[2] = c.z;
				break;
			}
			case 2: o[0] = fast_logit(a[0], 1.5f); break;
			case 3: {
				float x = a[0], y = a[1];
				square_to_circle(&x, &y);
				o[0] = x; o[1] = y;
				break;
			}
			case 4: {
				Vec3 v = cosine_sample_hemisphere(a[0], a[1]);
				o[0] = v.x; o[1] = v.y; o[2] = v.z;
				break;
			}
			case 5: o[0] = sphere_lambert(a[0], a[1]); break;
			case 6: for (int k = 0; k < 4; ++k) o[k] = wavelength_n(a[0], k); break;
			case 7: {
				Vec3 v = zup_to_vec(Vec3(a[0], a[1], a[2]), Vec3(a[3], a[4], a[5]));
				o[0] = v.x; o[1] = v.y; o[2] = v.z;
				break;
			}
			case 8: {
				Matrix44 m;
				for (int r = 0; r < 4; ++r)
					for (int c = 0; c < 4; ++c) m[r][c] = a[r * 4 + c];
				Matrix44 inv = m.inverse();
				for (int r = 0; r < 4; ++r)
					for (int c = 0; c < 4; ++c) o[r * 4 + c] = inv[r][c];
				break;
			}
			case 9: {
				Color_XYZ c;
				c.x = a[0]; c.y = a[1]; c.z = a[2];
				std::tie(o[0], o[1], o[2]) = XYZ_to_sRGB_E(c);
				break;
			}
			default: break;
		}
	}
}

/* Assemblies are numbered depth-first, pre-order, root = 0. */
int psyref_assembly_count(void* h) {
	return (int)static_cast<RefScene*>(h)->assemblies.size();
}

/* Number of BVH4::Node records (time samples counted separately). */
size_t psyref_bvh4_node_count(void* h, int assembly) {
	return static_cast<RefScene*>(h)->assemblies[assembly]->object_accel.nodes.size();
}

/*
 * Raw BVH4 node records: bounds n*24 floats (BBox4 SoA, as stored), child
 * n*3 uint64 (children 2-4), ts n uint32, data_index n uint64 (the union's
 * integer view, meaningful for leaves).
 */
void psyref_bvh4_nodes(void* h, int assembly, float* bounds, uint64_t* child, uint32_t* ts, uint64_t* data_index) {
	const auto& nodes = static_cast<RefScene*>(h)->assemblies[assembly]->object_accel.nodes;
	for (size_t i = 0; i < nodes.size(); ++i) {
		const auto& nd = nodes[i];
		for (int b = 0; b < 6; ++b)
			for (int k = 0; k < 4; ++k) bounds[i * 24 + b * 4 + k] = nd.bounds.bounds[b][k];
		for (int k = 0; k < 3; ++k) child[i * 3 + k] = nd.child_indices[k];
		ts[i] = nd.ts;
		data_index[i] = nd.data_index;
	}
}

size_t psyref_lighttree_node_count(void* h, int assembly) {
	return lt_view(static_cast<RefScene*>(h)->assemblies[assembly]->light_accel).nodes.size();
}

/*
 * Light tree nodes: meta n*6 uint64 (is_leaf, index1, index2,
 * instance_index, bounds count, first bounds record), energy n floats,
 * bounds written as 6 floats per BBox (min xyz, max xyz) into `bounds`
 * (caller sizes it with psyref_lighttree_bounds_count).
 */
size_t psyref_lighttree_bounds_count(void* h, int assembly) {
	size_t c = 0;
	for (const auto& nd : lt_view(static_cast<RefScene*>(h)->assemblies[assembly]->light_accel).nodes) c += nd.bounds.size();
	return c;
}

void psyref_lighttree_nodes(void* h, int assembly, uint64_t* meta, float* energy, float* bounds) {
	const auto& lt = lt_view(static_cast<RefScene*>(h)->assemblies[assembly]->light_accel);
	size_t bi = 0;
	for (size_t i = 0; i < lt.nodes.size(); ++i) {
		const auto& nd = lt.nodes[i];
		meta[i * 6 + 0] = nd.is_leaf ? 1 : 0;
		meta[i * 6 + 1] = nd.is_leaf ? 0 : nd.index1;
		meta[i * 6 + 2] = nd.is_leaf ? 0 : nd.index2;
		meta[i * 6 + 3] = nd.is_leaf ? nd.instance_index : 0;
		meta[i * 6 + 4] = nd.bounds.size();
		meta[i * 6 + 5] = bi;
		energy[i] = nd.energy;
		for (const auto& b : nd.bounds) {
			for (int k = 0; k < 3; ++k) {
				bounds[bi * 6 + k] = b.min[k];
				bounds[bi * 6 + 3 + k] = b.max[k];
			}
			++bi;
		}
	}
}

/* LightTree totals of one assembly: light_count, total energy. */
void psyref_lighttree_totals(void* h, int assembly, uint64_t* count, float* energy) {
	const auto& lt = static_cast<RefScene*>(h)->assemblies[assembly]->light_accel;
	*count = lt.light_count();
	*energy = lt_view(lt).total_energy;
}

} // extern "C"
