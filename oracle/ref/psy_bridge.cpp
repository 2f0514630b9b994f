/*
 * The reference-side bridge to libpsy_b200: what a maintainer of the
 * reference adds so that its own PathTraceIntegrator traces through the B200
 * library.  Compiled by oracle/Makefile against the reference's headers into
 * oracle/_ref/libpsyref_bridged.so, which links every reference source of
 * libpsyref.so except tracer/tracer.cpp: this file defines Tracer::trace
 * (reference tracer/tracer.hpp:76, tracer/tracer.cpp:38-121) in its place.
 *
 *   psy_bridge_upload(scene)        flattens the reference Scene after
 *                                   Scene::finalize() into a psy_scene_desc
 *                                   and uploads it (psy_scene_upload);
 *   Tracer::trace(...)              WorldRay stream -> psy_trace_host ->
 *                                   psy_hits_to_intersections;
 *   psy_hits_to_intersections(...)  rebuilds each Intersection
 *                                   (basics/intersection.hpp:22-49) from the
 *                                   hit arrays, with the closure a shader's
 *                                   shade() would give (tracer/tracer.cpp:
 *                                   245-250; lights set their own emission
 *                                   closure, lights/sphere_light.hpp:159-246).
 *
 * libpsy_b200.so is opened at run time (psy_bridge_set_library, or the
 * PSY_B200_LIB environment variable), so the reference build itself needs
 * no CUDA toolchain.  A context is single-threaded, so the integrator's
 * tracer threads take turns on it.  Test infrastructure here: only tests
 * load the bridged library, to run the reference's integrator on the B200
 * trace.
 */
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#define private public
#define protected public
#include "bicubic.hpp"
#include "bilinear.hpp"
#include "camera.hpp"
#include "config.hpp"
#include "global.hpp"
#include "scene.hpp"
#include "sphere.hpp"
#include "sphere_light.hpp"
#include "surface_closure.hpp"
#include "surface_shader.hpp"
#include "tracer.hpp"
#undef private
#undef protected

#include "psy_b200.h"

namespace {

// ---------------------------------------------------------------------
// libpsy_b200 entry points, resolved with dlsym
// ---------------------------------------------------------------------
struct PsyLib {
	void* handle = nullptr;
	int (*ctx_create)(int, psy_ctx**) = nullptr;
	const char* (*last_error)(const psy_ctx*) = nullptr;
	int (*scene_upload)(psy_ctx*, const psy_scene_desc*) = nullptr;
	int (*trace_host)(psy_ctx*, const psy_ray_soa*, uint32_t, const psy_hit_soa*) = nullptr;
};

std::mutex g_mu;
std::string g_lib_path;
PsyLib g_lib;
std::map<const Scene*, psy_ctx*> g_ctx;
std::string g_error;

bool load_library() {
	if (g_lib.handle) return true;
	std::string path = g_lib_path;
	if (path.empty()) {
		const char* e = std::getenv("PSY_B200_LIB");
		if (e) path = e;
	}
	if (path.empty()) {
		g_error = "no libpsy_b200.so given (psy_bridge_set_library or PSY_B200_LIB)";
		return false;
	}
	void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
	if (!h) {
		g_error = std::string("dlopen: ") + dlerror();
		return false;
	}
	g_lib.ctx_create = reinterpret_cast<int (*)(int, psy_ctx**)>(dlsym(h, "psy_ctx_create"));
	g_lib.last_error = reinterpret_cast<const char* (*)(const psy_ctx*)>(dlsym(h, "psy_last_error"));
	g_lib.scene_upload = reinterpret_cast<int (*)(psy_ctx*, const psy_scene_desc*)>(dlsym(h, "psy_scene_upload"));
	g_lib.trace_host = reinterpret_cast<int (*)(psy_ctx*, const psy_ray_soa*, uint32_t, const psy_hit_soa*)>(
	    dlsym(h, "psy_trace_host"));
	if (!g_lib.ctx_create || !g_lib.last_error || !g_lib.scene_upload || !g_lib.trace_host) {
		g_error = "libpsy_b200.so lacks an entry point";
		return false;
	}
	g_lib.handle = h;
	return true;
}

// ---------------------------------------------------------------------
// SphereLight keeps its data in implicitly private members and has no
// accessors; an explicit instantiation may name them (access checks do not
// apply to its template arguments), which gives the bridge member pointers
// without editing the reference's header.
// ---------------------------------------------------------------------
template <typename Tag, typename Tag::type M>
struct MemberOf {
	friend typename Tag::type member(Tag) { return M; }
};
struct LightPositions {
	typedef std::vector<Vec3> SphereLight::*type;
	friend type member(LightPositions);
};
struct LightRadii {
	typedef std::vector<float> SphereLight::*type;
	friend type member(LightRadii);
};
struct LightColors {
	typedef std::vector<Color> SphereLight::*type;
	friend type member(LightColors);
};
template struct MemberOf<LightPositions, &SphereLight::positions>;
template struct MemberOf<LightRadii, &SphereLight::radii>;
template struct MemberOf<LightColors, &SphereLight::colors>;

// ---------------------------------------------------------------------
// Scene flattening (the reference's Scene -> psy_scene_desc)
// ---------------------------------------------------------------------
struct Flat {
	std::vector<psy_assembly_desc> assemblies;
	std::vector<std::vector<psy_object_desc>> objects;
	std::vector<std::vector<psy_instance_desc>> instances;
	std::vector<std::vector<float>> xforms;
	std::vector<std::vector<uint32_t>> children;
	std::vector<std::unique_ptr<std::vector<float>>> data;
	std::vector<psy_shader_desc> shaders;
	std::unordered_map<const SurfaceShader*, int> shader_ids;
	std::string error;
};

void put_matrix(std::vector<float>* out, const Transform& t) {
	for (int r = 0; r < 4; ++r)
		for (int c = 0; c < 4; ++c) out->push_back(t.to[r][c]);
}

int shader_id(Flat& f, const SurfaceShader* sh) {
	if (!sh) return -1;
	auto it = f.shader_ids.find(sh);
	if (it != f.shader_ids.end()) return it->second;
	psy_shader_desc d{};
	Color c(0.0f);
	if (auto l = dynamic_cast<const LambertShader*>(sh)) {
		d.kind = PSY_SHADER_LAMBERT;
		c = l->col;
	} else if (auto e = dynamic_cast<const EmitShader*>(sh)) {
		d.kind = PSY_SHADER_EMIT;
		c = e->col;
	} else if (auto g = dynamic_cast<const GTRShader*>(sh)) {
		d.kind = PSY_SHADER_GTR;
		c = g->col;
		d.roughness = g->roughness;
		d.tail_shape = g->tail_shape;
		d.fresnel = g->fresnel;
	}
	for (int k = 0; k < 3; ++k) d.color[k] = c[k];
	f.shaders.push_back(d);
	return f.shader_ids[sh] = (int)f.shaders.size() - 1;
}

// Depth-first, pre-order: the root gets index 0 and every assembly's
// sub-assemblies follow it, as psy_assembly_desc::children expects.
uint32_t flatten(Flat& f, const Assembly& a) {
	const uint32_t me = (uint32_t)f.assemblies.size();
	f.assemblies.emplace_back();
	f.objects.emplace_back();
	f.instances.emplace_back();
	f.xforms.emplace_back();
	f.children.emplace_back();
	std::vector<uint32_t> kids;
	for (const auto& sub : a.assemblies) kids.push_back(flatten(f, *sub));
	f.children[me] = kids;
	for (const auto& obj : a.objects) {
		f.data.emplace_back(new std::vector<float>());
		std::vector<float>& d = *f.data.back();
		psy_object_desc od{};
		if (auto sp = dynamic_cast<const Sphere*>(obj.get())) {
			od.kind = PSY_OBJ_SPHERE;
			od.n0 = (uint32_t)sp->center.size();
			for (size_t t = 0; t < sp->center.size(); ++t)
				d.insert(d.end(), {sp->center[t].x, sp->center[t].y, sp->center[t].z, sp->radius[t]});
		} else if (auto bl = dynamic_cast<const Bilinear*>(obj.get())) {
			od.kind = PSY_OBJ_BILINEAR;
			od.n0 = (uint32_t)bl->verts.size();
			for (const auto& ts : bl->verts)
				for (const auto& v : ts) d.insert(d.end(), {v.x, v.y, v.z});
		} else if (auto bc = dynamic_cast<const Bicubic*>(obj.get())) {
			od.kind = PSY_OBJ_BICUBIC;
			od.n0 = (uint32_t)bc->verts.size();
			for (const auto& ts : bc->verts)
				for (const auto& v : ts) d.insert(d.end(), {v.x, v.y, v.z});
		} else if (auto sl = dynamic_cast<const SphereLight*>(obj.get())) {
			const std::vector<Vec3>& pos = sl->*member(LightPositions());
			const std::vector<float>& rad = sl->*member(LightRadii());
			const std::vector<Color>& col = sl->*member(LightColors());
			od.kind = PSY_OBJ_SPHERE_LIGHT;
			od.n0 = (uint32_t)pos.size();
			od.n1 = (uint32_t)rad.size();
			od.n2 = (uint32_t)col.size();
			for (const auto& p : pos) d.insert(d.end(), {p.x, p.y, p.z});
			d.insert(d.end(), rad.begin(), rad.end());
			for (const auto& c : col) d.insert(d.end(), {c[0], c[1], c[2]});
		} else {
			f.error = "an object kind the B200 trace does not support (subdivision surface, rectangle light)";
		}
		od.data = d.data();
		f.objects[me].push_back(od);
	}
	for (const auto& inst : a.instances) {
		psy_instance_desc id{};
		id.kind = inst.type == Instance::OBJECT ? PSY_INSTANCE_OBJECT : PSY_INSTANCE_ASSEMBLY;
		id.data_index = (uint32_t)inst.data_index;
		id.transform_index = (uint32_t)inst.transform_index;
		id.transform_count = (uint32_t)inst.transform_count;
		id.shader = shader_id(f, inst.surface_shader);
		f.instances[me].push_back(id);
	}
	for (const auto& x : a.xforms) put_matrix(&f.xforms[me], x);
	return me;
}

psy_ctx* upload(const Scene* scene) {
	auto it = g_ctx.find(scene);
	if (it != g_ctx.end()) return it->second;
	if (!load_library()) return nullptr;
	Flat f;
	flatten(f, *scene->root);
	if (!f.error.empty()) {
		g_error = f.error;
		return nullptr;
	}
	for (size_t i = 0; i < f.assemblies.size(); ++i) {
		psy_assembly_desc& ad = f.assemblies[i];
		ad.object_count = (uint32_t)f.objects[i].size();
		ad.objects = f.objects[i].data();
		ad.instance_count = (uint32_t)f.instances[i].size();
		ad.instances = f.instances[i].data();
		ad.transform_count = (uint32_t)(f.xforms[i].size() / 16);
		ad.transforms = f.xforms[i].data();
		ad.child_count = (uint32_t)f.children[i].size();
		ad.children = f.children[i].data();
	}
	// The camera is the reference's own here (its integrator makes the
	// camera rays); the description carries it for completeness, with the
	// field of view recovered from Camera's tan(fov / 2).
	std::vector<float> cx, fov, ap, fd;
	const Camera* cam = scene->camera.get();
	for (const auto& t : cam->transforms) put_matrix(&cx, t);
	for (float tf : cam->tfovs) fov.push_back(2.0f * std::atan(tf));
	ap = cam->aperture_radii;
	fd = cam->focus_distances;
	psy_scene_desc d{};
	d.cam_transform_count = (uint32_t)cam->transforms.size();
	d.cam_transforms = cx.data();
	d.cam_fov_count = (uint32_t)fov.size();
	d.cam_fovs = fov.data();
	d.cam_aperture_count = (uint32_t)ap.size();
	d.cam_aperture_radii = ap.data();
	d.cam_focus_count = (uint32_t)fd.size();
	d.cam_focus_distances = fd.data();
	for (int k = 0; k < 3; ++k) d.background[k] = scene->background_color[k];
	d.dice_rate = Config::dice_rate;
	d.min_upoly_size = Config::min_upoly_size;
	d.assembly_count = (uint32_t)f.assemblies.size();
	d.assemblies = f.assemblies.data();
	d.shader_count = (uint32_t)f.shaders.size();
	d.shaders = f.shaders.data();
	psy_ctx* ctx = nullptr;
	if (g_lib.ctx_create(0, &ctx) != PSY_OK) {
		g_error = "psy_ctx_create failed";
		return nullptr;
	}
	if (g_lib.scene_upload(ctx, &d) != PSY_OK) {
		g_error = std::string("psy_scene_upload: ") + g_lib.last_error(ctx);
		return nullptr;
	}
	g_ctx[scene] = ctx;
	return ctx;
}

// The hit arrays of one trace call, in host memory.
struct Hits {
	std::vector<uint8_t> hit, backfacing, closure;
	std::vector<uint64_t> id;
	std::vector<float> t, uv, p, n, dpdu, dpdv, dndu, dndv, light_pdf, offset, space, closure_color;
	psy_hit_soa soa{};
	void resize(size_t k) {
		hit.resize(k); backfacing.resize(k); closure.resize(k); id.resize(k); t.resize(k); uv.resize(2 * k);
		p.resize(3 * k); n.resize(3 * k); dpdu.resize(3 * k); dpdv.resize(3 * k); dndu.resize(3 * k);
		dndv.resize(3 * k); light_pdf.resize(k); offset.resize(3 * k); space.resize(16 * k);
		closure_color.resize(3 * k);
		soa = psy_hit_soa{hit.data(),  id.data(),   t.data(),    uv.data(),         p.data(),
		                  n.data(),    dpdu.data(), dpdv.data(), dndu.data(),       dndv.data(),
		                  backfacing.data(), light_pdf.data(), offset.data(), space.data(), closure.data(),
		                  closure_color.data()};
	}
};

Vec3 v3(const float* a) { return Vec3(a[0], a[1], a[2]); }

}  // namespace

// Rebuilds n Intersections from psy_trace_host's hit arrays (host memory),
// as Tracer::trace leaves them: every Intersection reset, then for a hit
// the fields the reference writes (occlusion rays: hit and id only).
void psy_hits_to_intersections(const psy_hit_soa& h, uint32_t n, const WorldRay* rays, Intersection* out) {
	for (uint32_t i = 0; i < n; ++i) {
		Intersection& in = out[i];
		in = Intersection();
		if (!h.hit[i]) continue;
		in.hit = true;
		in.id.id = h.id[i];
		if (rays[i].type & WorldRay::OCCLUSION) continue;
		in.t = h.t[i];
		in.backfacing = h.backfacing[i] != 0;
		in.light_pdf = h.light_pdf[i];
		const float* m = h.space + 16 * (size_t)i;
		in.space = Transform(Matrix44(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9], m[10], m[11], m[12],
		                              m[13], m[14], m[15]));
		in.geo.u = h.uv[2 * i];
		in.geo.v = h.uv[2 * i + 1];
		in.geo.p = v3(h.p + 3 * i);
		in.geo.n = v3(h.n + 3 * i);
		in.geo.dpdu = v3(h.dpdu + 3 * i);
		in.geo.dpdv = v3(h.dpdv + 3 * i);
		in.geo.dndu = v3(h.dndu + 3 * i);
		in.geo.dndv = v3(h.dndv + 3 * i);
		in.offset = v3(h.offset + 3 * i);
		const float* c = h.closure_color + 3 * i;
		const Color col(c[0], c[1], c[2]);
		if (h.closure[i] == 1) in.surface_closure.init(LambertClosure(col));
		else in.surface_closure.init(EmitClosure(col));  // emission, lights, and no-shader magenta
		in.closure_prob = 1.0f;
	}
}

uint32_t Tracer::trace(const WorldRay* w_rays_begin, const WorldRay* w_rays_end, Intersection* intersections_begin,
                       Intersection* intersections_end) {
	const uint32_t n = (uint32_t)(w_rays_end - w_rays_begin);
	Global::Stats::rays_shot += n;
	std::vector<float> o(3 * (size_t)n), d(3 * (size_t)n), odx(3 * (size_t)n), ody(3 * (size_t)n),
	    ddx(3 * (size_t)n), ddy(3 * (size_t)n), time(n);
	std::vector<uint16_t> type(n);
	for (uint32_t i = 0; i < n; ++i) {
		const WorldRay& r = w_rays_begin[i];
		const Vec3* src[6] = {&r.o, &r.d, &r.odx, &r.ody, &r.ddx, &r.ddy};
		std::vector<float>* dst[6] = {&o, &d, &odx, &ody, &ddx, &ddy};
		for (int k = 0; k < 6; ++k) {
			(*dst[k])[3 * i] = src[k]->x;
			(*dst[k])[3 * i + 1] = src[k]->y;
			(*dst[k])[3 * i + 2] = src[k]->z;
		}
		time[i] = r.time;
		type[i] = (uint16_t)r.type;
	}
	const psy_ray_soa rays{o.data(), d.data(), odx.data(), ody.data(), ddx.data(), ddy.data(), time.data(), type.data()};
	Hits h;
	h.resize(n);
	{
		std::lock_guard<std::mutex> lock(g_mu);
		psy_ctx* ctx = upload(scene);
		if (!ctx || g_lib.trace_host(ctx, &rays, n, &h.soa) != PSY_OK) {
			std::fprintf(stderr, "psy bridge: %s\n", ctx ? g_lib.last_error(ctx) : g_error.c_str());
			std::abort();
		}
	}
	psy_hits_to_intersections(h.soa, n, w_rays_begin, intersections_begin);
	(void)intersections_end;
	return n;
}

extern "C" {

// Which libpsy_b200.so the bridge opens (before the first trace).
void psy_bridge_set_library(const char* path) {
	std::lock_guard<std::mutex> lock(g_mu);
	g_lib_path = path ? path : "";
}

}  // extern "C"
