/*
 * C ABI implementation (include/psy_b200.h): contexts, scene upload, ray
 * tracing entry points, status reporting.
 */
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/psy_b200.h"
#include "host_cpu.h"
#include "kernels.h"
#include "psy_ctx.h"
#include "sampler_tables.h"
#include "scene_build.h"

using namespace psy;

#define PSY_VERSION "psy_b200 0.1"

int ctx_fail(psy_ctx* ctx, int code, const char* fmt, ...) {
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	if (ctx) ctx->last_error = buf;
	return code;
}

int ctx_cuda(psy_ctx* ctx, cudaError_t e, const char* what) {
	if (e == cudaSuccess) return PSY_OK;
	const int code = (e == cudaErrorMemoryAllocation) ? PSY_ERR_OOM : PSY_ERR_DEVICE;
	return ctx_fail(ctx, code, "%s: %s", what, cudaGetErrorString(e));
}

psy_ctx::~psy_ctx() {
	cudaSetDevice(device);
	free_scene();
	for (auto& kv : scratch) cudaFree(kv.second.ptr);
	for (void* p : const_allocs) cudaFree(p);
	if (d_status) cudaFree(d_status);
	if (h_status) cudaFreeHost(h_status);
}

void psy_ctx::free_scene() {
	for (void* p : scene_allocs) cudaFree(p);
	scene_allocs.clear();
	has_scene = false;
	device_bytes = 0;
	std::memset(&dev, 0, sizeof(dev));
}

int psy_ctx::upload(const void* src, size_t bytes, void** dst) {
	*dst = nullptr;
	if (bytes == 0) return PSY_OK;
	cudaError_t e = cudaMalloc(dst, bytes);
	if (e != cudaSuccess) return ctx_cuda(this, e, "cudaMalloc(scene)");
	scene_allocs.push_back(*dst);
	device_bytes += bytes;
	e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
	return ctx_cuda(this, e, "cudaMemcpy(scene)");
}

void* psy_ctx::scratch_buffer(const char* name, size_t bytes, int* rc) {
	*rc = PSY_OK;
	Scratch& s = scratch[name];
	if (s.bytes >= bytes && s.ptr) return s.ptr;
	if (s.ptr) cudaFree(s.ptr);
	s.ptr = nullptr;
	s.bytes = 0;
	cudaError_t e = cudaMalloc(&s.ptr, bytes < 256 ? 256 : bytes);
	if (e != cudaSuccess) {
		*rc = ctx_cuda(this, e, "cudaMalloc(scratch)");
		s.ptr = nullptr;
		return nullptr;
	}
	s.bytes = bytes < 256 ? 256 : bytes;
	return s.ptr;
}

int psy_ctx::check_status(cudaStream_t stream) {
	cudaError_t e = cudaMemcpyAsync(h_status, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
	if (e != cudaSuccess) return ctx_cuda(this, e, "status read");
	e = cudaStreamSynchronize(stream);
	if (e != cudaSuccess) return ctx_cuda(this, e, "stream synchronize");
	const unsigned st = *h_status;
	if (st) {
		cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream);
		cudaStreamSynchronize(stream);
		if (st & ERRF_STACK) return ctx_fail(this, PSY_ERR_STACK_OVERFLOW, "a traversal stack overflowed (flags %#x)", st);
		if (st & ERRF_LEVELS)
			return ctx_fail(this, PSY_ERR_STACK_OVERFLOW, "assembly nesting deeper than supported (flags %#x)", st);
		if (st & ERRF_MOTION)
			return ctx_fail(this, PSY_ERR_ARG, "more motion samples than supported (flags %#x)", st);
		return ctx_fail(this, PSY_ERR_DEVICE, "device error flags %#x", st);
	}
	return PSY_OK;
}

extern "C" {

const char* psy_version(void) { return PSY_VERSION; }

int psy_ctx_create(int device, psy_ctx** out) {
	if (!out) return PSY_ERR_ARG;
	*out = nullptr;
	int count = 0;
	cudaError_t e = cudaGetDeviceCount(&count);
	if (e != cudaSuccess || count == 0) return PSY_ERR_DEVICE;
	if (device < 0 || device >= count) return PSY_ERR_ARG;
	e = cudaSetDevice(device);
	if (e != cudaSuccess) return PSY_ERR_DEVICE;
	std::unique_ptr<psy_ctx> ctx(new psy_ctx());
	ctx->device = device;
	if (cudaMalloc(&ctx->d_status, sizeof(unsigned)) != cudaSuccess) return PSY_ERR_OOM;
	if (cudaMemset(ctx->d_status, 0, sizeof(unsigned)) != cudaSuccess) return PSY_ERR_DEVICE;
	if (cudaMallocHost(&ctx->h_status, sizeof(unsigned)) != cudaSuccess) return PSY_ERR_OOM;
	// sampler tables, uploaded once per context
	{
		const HaltonTables ht = build_halton_tables();
		std::vector<uint4> dims;
		for (const HaltonDim& d : ht.dims) dims.push_back(make_uint4(d.base, d.pow_base, d.groups, d.perm_offset));
		void *p0, *p1, *p2;
		if (cudaMalloc(&p0, ht.perm.size() * sizeof(uint16_t)) != cudaSuccess) return PSY_ERR_OOM;
		ctx->const_allocs.push_back(p0);
		if (cudaMalloc(&p1, dims.size() * sizeof(uint4)) != cudaSuccess) return PSY_ERR_OOM;
		ctx->const_allocs.push_back(p1);
		if (cudaMalloc(&p2, ht.cmul.size() * sizeof(double)) != cudaSuccess) return PSY_ERR_OOM;
		ctx->const_allocs.push_back(p2);
		if (cudaMemcpy(p0, ht.perm.data(), ht.perm.size() * sizeof(uint16_t), cudaMemcpyHostToDevice) != cudaSuccess ||
		    cudaMemcpy(p1, dims.data(), dims.size() * sizeof(uint4), cudaMemcpyHostToDevice) != cudaSuccess ||
		    cudaMemcpy(p2, ht.cmul.data(), ht.cmul.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
			return PSY_ERR_DEVICE;
		ctx->halton.perm = static_cast<const uint16_t*>(p0);
		ctx->halton.dims = static_cast<const uint4*>(p1);
		ctx->halton.cmul = static_cast<const double*>(p2);
	}
	ctx->ident_inv = reference_identity_inverse_scale();
	*out = ctx.release();
	return PSY_OK;
}

void psy_ctx_destroy(psy_ctx* ctx) { delete ctx; }

const char* psy_last_error(const psy_ctx* ctx) {
	if (!ctx) return "no context";
	return ctx->last_error.c_str();
}

int psy_scene_upload(psy_ctx* ctx, const psy_scene_desc* desc) {
	if (!ctx) return PSY_ERR_ARG;
	cudaSetDevice(ctx->device);
	std::unique_ptr<BuiltScene> b(new BuiltScene());
	std::string err;
	int rc = build_scene(desc, b.get(), &err);
	if (rc != PSY_OK) return ctx_fail(ctx, rc, "scene: %s", err.c_str());
	ctx->free_scene();
	DevScene& d = ctx->dev;
	void* p;
#define UP(field, vec)                                                                        \
	if ((rc = ctx->upload(vec.data(), vec.size() * sizeof(vec[0]), &p)) != PSY_OK) return rc; \
	d.field = static_cast<decltype(d.field)>(p);
	UP(assemblies, b->assemblies);
	UP(instances, b->instances);
	UP(objects, b->objects);
	UP(nodes, b->nodes);
	UP(node_extra, b->node_extra);
	UP(xforms, b->xforms);
	UP(fpool, b->fpool);
	UP(light_nodes, b->light_nodes);
	UP(light_extra, b->light_extra);
	UP(shaders, b->shaders);
	UP(cam_xforms, b->cam_xforms);
	UP(cam_tfovs, b->cam_tfovs);
	UP(cam_apertures, b->cam_apertures);
	UP(cam_focus, b->cam_focus);
#undef UP
	d.assembly_count = (int)b->assemblies.size();
	d.max_depth = b->max_depth;
	d.features = b->features;
	d.dice_rate = b->dice_rate;
	d.min_upoly_size = b->min_upoly_size;
	d.cam_xform_count = (int)b->cam_xforms.size() / 16;
	d.cam_tfov_count = (int)b->cam_tfovs.size();
	d.cam_aperture_count = (int)b->cam_apertures.size();
	d.cam_focus_count = (int)b->cam_focus.size();
	for (int k = 0; k < 3; ++k) d.background[k] = b->background[k];
	if (b->max_depth > PSY_MAX_LEVELS_HOST) {
		ctx->free_scene();
		return ctx_fail(ctx, PSY_ERR_ARG, "assembly nesting %d deeper than %d", b->max_depth, PSY_MAX_LEVELS_HOST);
	}
	ctx->host = std::move(b);
	ctx->has_scene = true;
	return PSY_OK;
}

int psy_scene_stats_get(const psy_ctx* ctx, psy_scene_stats* out) {
	if (!ctx || !out) return PSY_ERR_ARG;
	if (!ctx->has_scene) return PSY_ERR_NO_SCENE;
	out->assemblies = (uint32_t)ctx->host->assemblies.size();
	out->instances = (uint32_t)ctx->host->instances.size();
	out->objects = (uint32_t)ctx->host->objects.size();
	out->bvh4_nodes = (uint32_t)ctx->host->nodes.size();
	out->light_nodes = (uint32_t)ctx->host->light_nodes.size();
	out->lights = ctx->host->total_lights;
	out->device_bytes = ctx->device_bytes;
	return PSY_OK;
}

int psy_build_bvh4(const psy_scene_desc* desc, uint32_t assembly, uint64_t* count, float* bounds, uint64_t* child,
                   uint32_t* ts, uint64_t* data_index) {
	if (!count) return PSY_ERR_ARG;
	BuiltScene b;
	std::string err;
	const int rc = build_scene(desc, &b, &err);
	if (rc != PSY_OK) return rc;
	if (assembly >= b.ref_bvh4.size()) return PSY_ERR_ARG;
	const RefBVH4& r = b.ref_bvh4[assembly];
	*count = r.ts.size();
	if (bounds) std::memcpy(bounds, r.bounds.data(), r.bounds.size() * sizeof(float));
	if (child) std::memcpy(child, r.child.data(), r.child.size() * sizeof(uint64_t));
	if (ts) std::memcpy(ts, r.ts.data(), r.ts.size() * sizeof(uint32_t));
	if (data_index) std::memcpy(data_index, r.data_index.data(), r.data_index.size() * sizeof(uint64_t));
	return PSY_OK;
}

int psy_build_light_tree(const psy_scene_desc* desc, uint32_t assembly, uint64_t* count, uint64_t* nbounds,
                         uint64_t* meta, float* energy, float* bounds, uint64_t* light_count, float* total_energy) {
	if (!count || !nbounds) return PSY_ERR_ARG;
	BuiltScene b;
	std::string err;
	const int rc = build_scene(desc, &b, &err);
	if (rc != PSY_OK) return rc;
	if (assembly >= b.assemblies.size()) return PSY_ERR_ARG;
	const DevAssembly& a = b.assemblies[assembly];
	if (light_count) *light_count = (uint64_t)a.light_count;
	if (total_energy) *total_energy = a.light_energy;
	// the assembly's nodes are contiguous from light_root up to the next assembly's root
	size_t first = 0, last = 0;
	if (a.light_root >= 0) {
		first = (size_t)a.light_root;
		last = b.light_nodes.size();
		for (const DevAssembly& o : b.assemblies)
			if (o.light_root > a.light_root && (size_t)o.light_root < last) last = (size_t)o.light_root;
	}
	*count = last - first;
	uint64_t nb = 0;
	for (size_t i = first; i < last; ++i) {
		const DevLightNode& n = b.light_nodes[i];
		const size_t k = i - first;
		if (meta) {
			meta[k * 6 + 0] = (uint64_t)n.is_leaf;
			meta[k * 6 + 1] = n.is_leaf ? 0 : (uint64_t)(n.c1 - a.light_root);
			meta[k * 6 + 2] = n.is_leaf ? 0 : (uint64_t)(n.c2 - a.light_root);
			meta[k * 6 + 3] = n.is_leaf ? (uint64_t)n.c1 : 0;
			meta[k * 6 + 4] = (uint64_t)n.ts;
			meta[k * 6 + 5] = nb;
		}
		if (energy) energy[k] = n.energy;
		for (int t = 0; t < n.ts; ++t) {
			if (bounds) {
				float* o = bounds + (nb + t) * 6;
				if (t == 0) {
					for (int c = 0; c < 3; ++c) {
						o[c] = n.lo[c];
						o[3 + c] = n.hi[c];
					}
				} else {
					std::memcpy(o, b.light_extra.data() + (size_t)(n.extra + t - 1) * 6, 6 * sizeof(float));
				}
			}
		}
		nb += (uint64_t)n.ts;
	}
	*nbounds = nb;
	return PSY_OK;
}

static int make_hit_soa(const psy_hit_soa* h, HitSoA* o) {
	std::memset(o, 0, sizeof(*o));
	if (!h) return PSY_OK;
	o->hit = h->hit;
	o->id = h->id;
	o->t = h->t;
	o->uv = h->uv;
	o->p = h->p;
	o->n = h->n;
	o->dpdu = h->dpdu;
	o->dpdv = h->dpdv;
	o->dndu = h->dndu;
	o->dndv = h->dndv;
	o->backfacing = h->backfacing;
	o->light_pdf = h->light_pdf;
	o->offset = h->offset;
	o->space = h->space;
	o->closure = h->closure;
	o->closure_color = h->closure_color;
	o->want_geometry = (h->uv || h->p || h->n || h->dpdu || h->dpdv || h->dndu || h->dndv || h->backfacing ||
	                    h->light_pdf || h->offset || h->space || h->closure || h->closure_color)
	                       ? 1
	                       : 0;
	return PSY_OK;
}

static bool rays_complete(const psy_ray_soa* r) {
	return r && r->o && r->d && r->odx && r->ody && r->ddx && r->ddy && r->time;
}

int psy_trace(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits, void* stream) {
	if (!ctx) return PSY_ERR_ARG;
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "psy_trace: no scene uploaded");
	if (n == 0) return PSY_OK;
	if (!rays_complete(rays)) return ctx_fail(ctx, PSY_ERR_ARG, "psy_trace: incomplete ray arrays");
	cudaSetDevice(ctx->device);
	RaySoA rs{rays->o, rays->d, rays->odx, rays->ody, rays->ddx, rays->ddy, rays->time, rays->type};
	HitSoA hs;
	make_hit_soa(hits, &hs);
	return ctx_cuda(ctx, launch_trace(ctx->dev, rs, hs, n, ctx->d_status, (cudaStream_t)stream), "trace launch");
}

int psy_sync(psy_ctx* ctx, void* stream) {
	if (!ctx) return PSY_ERR_ARG;
	cudaSetDevice(ctx->device);
	return ctx->check_status((cudaStream_t)stream);
}

int psy_trace_host(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits) {
	if (!ctx) return PSY_ERR_ARG;
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "psy_trace_host: no scene uploaded");
	if (n == 0) return PSY_OK;
	if (!rays_complete(rays)) return ctx_fail(ctx, PSY_ERR_ARG, "psy_trace_host: incomplete ray arrays");
	cudaSetDevice(ctx->device);
	int rc;
	const size_t f3 = (size_t)n * 3 * sizeof(float);
	const size_t f1 = (size_t)n * sizeof(float);
	const size_t ray_bytes = 6 * f3 + f1 + (size_t)n * sizeof(uint16_t);
	char* dr = static_cast<char*>(ctx->scratch_buffer("host_rays", ray_bytes + 64, &rc));
	if (!dr) return rc;
	cudaStream_t st = ctx->host_stream();
	float* d_o = reinterpret_cast<float*>(dr);
	float* d_d = d_o + 3 * (size_t)n;
	float* d_odx = d_d + 3 * (size_t)n;
	float* d_ody = d_odx + 3 * (size_t)n;
	float* d_ddx = d_ody + 3 * (size_t)n;
	float* d_ddy = d_ddx + 3 * (size_t)n;
	float* d_time = d_ddy + 3 * (size_t)n;
	uint16_t* d_type = reinterpret_cast<uint16_t*>(d_time + n);
	const float* srcs[6] = {rays->o, rays->d, rays->odx, rays->ody, rays->ddx, rays->ddy};
	float* dsts[6] = {d_o, d_d, d_odx, d_ody, d_ddx, d_ddy};
	for (int k = 0; k < 6; ++k)
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(dsts[k], srcs[k], f3, cudaMemcpyHostToDevice, st), "H2D rays")))
			return rc;
	if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(d_time, rays->time, f1, cudaMemcpyHostToDevice, st), "H2D rays")))
		return rc;
	if (rays->type) {
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(d_type, rays->type, (size_t)n * 2, cudaMemcpyHostToDevice, st),
		                   "H2D rays")))
			return rc;
	}
	// device hit buffers for the requested fields
	struct F {
		void* host;
		size_t per;
	};
	const F fields[16] = {{hits ? hits->hit : nullptr, 1},       {hits ? hits->id : nullptr, 8},
	                      {hits ? hits->t : nullptr, 4},         {hits ? hits->uv : nullptr, 8},
	                      {hits ? hits->p : nullptr, 12},        {hits ? hits->n : nullptr, 12},
	                      {hits ? hits->dpdu : nullptr, 12},     {hits ? hits->dpdv : nullptr, 12},
	                      {hits ? hits->dndu : nullptr, 12},     {hits ? hits->dndv : nullptr, 12},
	                      {hits ? hits->backfacing : nullptr, 1}, {hits ? hits->light_pdf : nullptr, 4},
	                      {hits ? hits->offset : nullptr, 12},   {hits ? hits->space : nullptr, 64},
	                      {hits ? hits->closure : nullptr, 1},   {hits ? hits->closure_color : nullptr, 12}};
	size_t total = 0;
	size_t offs[16];
	for (int k = 0; k < 16; ++k) {
		offs[k] = total;
		if (fields[k].host) total += ((fields[k].per * n + 255) / 256) * 256;
	}
	char* dh = static_cast<char*>(ctx->scratch_buffer("host_hits", total + 256, &rc));
	if (!dh) return rc;
	void* dptr[16];
	for (int k = 0; k < 16; ++k) dptr[k] = fields[k].host ? (void*)(dh + offs[k]) : nullptr;
	psy_hit_soa dhits;
	dhits.hit = (uint8_t*)dptr[0];
	dhits.id = (uint64_t*)dptr[1];
	dhits.t = (float*)dptr[2];
	dhits.uv = (float*)dptr[3];
	dhits.p = (float*)dptr[4];
	dhits.n = (float*)dptr[5];
	dhits.dpdu = (float*)dptr[6];
	dhits.dpdv = (float*)dptr[7];
	dhits.dndu = (float*)dptr[8];
	dhits.dndv = (float*)dptr[9];
	dhits.backfacing = (uint8_t*)dptr[10];
	dhits.light_pdf = (float*)dptr[11];
	dhits.offset = (float*)dptr[12];
	dhits.space = (float*)dptr[13];
	dhits.closure = (uint8_t*)dptr[14];
	dhits.closure_color = (float*)dptr[15];
	psy_ray_soa drays{d_o, d_d, d_odx, d_ody, d_ddx, d_ddy, d_time, rays->type ? d_type : nullptr};
	if ((rc = psy_trace(ctx, &drays, n, &dhits, st))) return rc;
	for (int k = 0; k < 16; ++k) {
		if (!fields[k].host) continue;
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(fields[k].host, dptr[k], fields[k].per * n, cudaMemcpyDeviceToHost, st),
		                   "D2H hits")))
			return rc;
	}
	return ctx->check_status(st);
}


int psy_light_sample(psy_ctx* ctx, const psy_light_query_soa* q, uint32_t n, const psy_light_sample_soa* out,
                     void* stream) {
	if (!ctx || !q || !out) return PSY_ERR_ARG;
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "psy_light_sample: no scene uploaded");
	if (n == 0) return PSY_OK;
	if (!q->n || !q->u || !q->v || !q->pos || !q->nor || !q->d || !q->wavelength || !q->time)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_light_sample: incomplete query arrays");
	if (ctx->dev.assemblies == nullptr || ctx->host->assemblies[0].light_root < 0)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_light_sample: the scene has no lights");
	cudaSetDevice(ctx->device);
	LightQuerySoADev qd{q->n, q->u, q->v, q->pos, q->nor, q->d, q->wavelength, q->time};
	LightSampleSoADev od{out->to_light, out->spec, out->selection_pdf, out->light_pdf, out->id};
	return ctx_cuda(ctx, launch_light_sample(ctx->dev, qd, od, n, ctx->ident_inv, ctx->d_status, (cudaStream_t)stream),
	                "light sample launch");
}

int psy_render(psy_ctx* ctx, const psy_render_desc* desc, float* xyz, uint32_t* counts, psy_render_stats* stats,
               void* stream) {
	if (!ctx || !desc || !xyz) return PSY_ERR_ARG;
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "psy_render: no scene uploaded");
	if (desc->width == 0 || desc->height == 0 || desc->width > 65535 || desc->height > 65535)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_render: resolution must be 1..65535 per axis");
	if (desc->spp == 0 || desc->spp > 65535) return ctx_fail(ctx, PSY_ERR_ARG, "psy_render: spp must be 1..65535");
	const uint32_t path_length = desc->path_length ? desc->path_length : 4;
	if (path_length > 40) return ctx_fail(ctx, PSY_ERR_ARG, "psy_render: path_length must be at most 40");
	if (ctx->host->assemblies[0].light_root < 0)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_render: the scene has no lights (the reference integrator needs one)");
	cudaSetDevice(ctx->device);
	cudaStream_t st = (cudaStream_t)stream;
	const uint64_t total = (uint64_t)desc->width * desc->height * desc->spp;
	uint64_t want = desc->stream_paths ? desc->stream_paths : (1ull << 21);
	if (want > (1ull << 26)) want = 1ull << 26;
	uint64_t P = (want / desc->spp) * desc->spp;
	if (P < desc->spp) P = desc->spp;
	if (P > total) P = total;
	int rc;
	auto buf = [&](const char* name, size_t bytes) -> void* { return ctx->scratch_buffer(name, bytes, &rc); };
	PathSoA ps;
	ps.smp = (uint32_t*)buf("r_smp", P * 4);
	ps.dimstep = (uint32_t*)buf("r_dimstep", P * 4);
	ps.wl = (float*)buf("r_wl", P * 4);
	ps.time = (float*)buf("r_time", P * 4);
	ps.last_pdf = (float*)buf("r_lpdf", P * 4);
	ps.col = (float4*)buf("r_col", P * 16);
	ps.fcol = (float4*)buf("r_fcol", P * 16);
	ps.lcol = (float4*)buf("r_lcol", P * 16);
	ps.hit = (float*)buf("r_hit", P * 64);
	ps.pray = (float*)buf("r_pray", P * 64);
	ps.sample = (float*)buf("r_sample", P * 12);
	WaveQueues wq;
	wq.q0 = (int*)buf("r_q0", P * 4);
	wq.q1 = (int*)buf("r_q1", P * 4);
	wq.counters = (int*)buf("r_counters", sizeof(int) * render_counter_count(path_length));
	wq.rays = (unsigned long long*)buf("r_rays", sizeof(unsigned long long));
	WaveBufs wb;
	wb.cap = (int)P;
	wb.ray[0] = (float4*)buf("r_ray0", P * 80);
	wb.ray[1] = (float4*)buf("r_ray1", P * 80);
	wb.hit_f = (float4*)buf("r_hitf", P * 16);
	wb.hit_i = (int4*)buf("r_hiti", P * 48);
	wb.occl = (uint8_t*)buf("r_occl", P);
	if (!wb.ray[0] || !wb.ray[1] || !wb.hit_f || !wb.hit_i || !wb.occl) return rc ? rc : PSY_ERR_OOM;
	if (!ps.smp || !ps.dimstep || !ps.wl || !ps.time || !ps.last_pdf || !ps.col || !ps.fcol || !ps.lcol ||
	    !ps.hit || !ps.pray || !ps.sample || !wq.q0 || !wq.q1 || !wq.counters || !wq.rays)
		return rc ? rc : PSY_ERR_OOM;
	if ((rc = ctx_cuda(ctx, cudaMemsetAsync(wq.rays, 0, sizeof(unsigned long long), st), "memset"))) return rc;
	RenderParams rp;
	rp.width = desc->width;
	rp.height = desc->height;
	rp.spp = desc->spp;
	rp.seed = desc->seed;
	rp.path_length = path_length;
	rp.light_count = (uint32_t)ctx->host->assemblies[0].light_count;
	rp.min_x = -1.0f;
	rp.max_x = 1.0f;
	rp.max_y = (float)desc->height / (float)desc->width;
	rp.min_y = -rp.max_y;
	rp.ident_inv = ctx->ident_inv;
	uint32_t launches = 0, waves = 0;
	for (uint64_t base = 0; base < total; base += P) {
		rp.wave_base = base;
		rp.wave_paths = (int)((total - base) < P ? (total - base) : P);
		if ((rc = ctx_cuda(ctx,
		                   launch_render_wave(ctx->dev, ctx->halton, rp, ps, wb, wq, xyz, counts, ctx->d_status, st,
		                                      &launches),
		                   "render launch")))
			return rc;
		++waves;
	}
	if (stats) {
		unsigned long long rays = 0;
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(&rays, wq.rays, sizeof(rays), cudaMemcpyDeviceToHost, st), "D2H")))
			return rc;
		if ((rc = ctx->check_status(st))) return rc;
		stats->paths = total;
		stats->rays = rays;
		stats->launches = launches;
		stats->waves = waves;
	}
	return PSY_OK;
}

}  // extern "C"
