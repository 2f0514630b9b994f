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
	if (batch_graph) cudaGraphExecDestroy(batch_graph);
	for (cudaEvent_t e : timer_events) cudaEventDestroy(e);
	if (capture_stream) cudaStreamDestroy(capture_stream);
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
		if (st & ERRF_BISECT)
			return ctx_fail(this, PSY_ERR_TIMEOUT, "a patch bisection exceeded its step bound (flags %#x)", st);
		return ctx_fail(this, PSY_ERR_DEVICE, "device error flags %#x", st);
	}
	return PSY_OK;
}

// ---------------------------------------------------------------------
// Rendering helpers
// ---------------------------------------------------------------------
static int check_render(psy_ctx* ctx, const psy_render_desc* desc, const char* who) {
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "%s: no scene uploaded", who);
	if (desc->width == 0 || desc->height == 0 || desc->width > 65535 || desc->height > 65535)
		return ctx_fail(ctx, PSY_ERR_ARG, "%s: resolution must be 1..65535 per axis", who);
	if (desc->spp == 0 || desc->spp > 65535) return ctx_fail(ctx, PSY_ERR_ARG, "%s: spp must be 1..65535", who);
	if (desc->path_length > 40) return ctx_fail(ctx, PSY_ERR_ARG, "%s: path_length must be at most 40", who);
	if (ctx->host->assemblies[0].light_root < 0)
		return ctx_fail(ctx, PSY_ERR_ARG, "%s: the scene has no lights (the reference integrator needs one)", who);
	return PSY_OK;
}

static RenderParams render_params(const psy_ctx* ctx, const psy_render_desc* desc, float* xyz, uint32_t* counts) {
	RenderParams rp;
	rp.width = desc->width;
	rp.height = desc->height;
	rp.spp = desc->spp;
	rp.seed = desc->seed;
	rp.path_length = desc->path_length ? desc->path_length : 4;
	rp.light_count = (uint32_t)ctx->host->assemblies[0].light_count;
	rp.min_x = -1.0f;
	rp.max_x = 1.0f;
	rp.max_y = (float)desc->height / (float)desc->width;
	rp.min_y = -rp.max_y;
	rp.ident_inv = ctx->ident_inv;
	rp.path_base = 0;
	rp.pixel_base = 0;
	rp.xyz = xyz;
	rp.counts = counts;
	rp.params = nullptr;
	rp.shader_param = nullptr;
	rp.object_param = nullptr;
	rp.dl_dxyz = nullptr;
	rp.grad = nullptr;
	rp.param_count = 0;
	rp.grad_in_smem = 0;
	return rp;
}

// Path state, ray / hit buffers and queues for waves of P paths, in the
// context's scratch buffers named with `prefix`.
struct WaveSet {
	PathSoA ps;
	WaveBufs wb;
	WaveQueues wq;
};

static int wave_set(psy_ctx* ctx, const char* prefix, uint64_t P, uint32_t path_length, WaveSet* ws,
                    bool adjoint = false) {
	int rc = PSY_OK;
	std::string pre(prefix);
	auto buf = [&](const char* name, size_t bytes) -> void* {
		return ctx->scratch_buffer((pre + name).c_str(), bytes, &rc);
	};
	PathSoA& ps = ws->ps;
	ps.smp = (uint32_t*)buf("smp", P * 4);
	ps.dimstep = (uint32_t*)buf("dimstep", P * 4);
	ps.wl = (float*)buf("wl", P * 4);
	ps.time = (float*)buf("time", P * 4);
	ps.last_pdf = (float*)buf("lpdf", P * 4);
	ps.col = (float4*)buf("col", P * 16);
	ps.fcol = (float4*)buf("fcol", P * 16);
	ps.lcol = (float4*)buf("lcol", P * 16);
	ps.hit = (float*)buf("hit", P * 64);
	ps.pray = (float*)buf("pray", P * 64);
	ps.hitx = (float*)buf("hitx", P * 48);
	ps.sample = (float*)buf("sample", P * 12);
	ps.rid = (uint16_t*)buf("rid", P * 2);
	ps.adj = nullptr;
	ps.valb = nullptr;
	ps.vpid = nullptr;
	ps.nee_param = nullptr;
	ps.vdsc = nullptr;
	ps.fexcl = nullptr;
	ps.nee_base = nullptr;
	if (adjoint) {
		ps.adj = (float4*)buf("adj", P * 16);
		ps.valb = (float4*)buf("valb", P * 16 * PSY_ADJ_MAX_VERTS);
		ps.vpid = (int*)buf("vpid", P * 4 * PSY_ADJ_MAX_VERTS);
		ps.nee_param = (int*)buf("neep", P * 4);
		ps.vdsc = (float4*)buf("vdsc", P * 16 * PSY_ADJ_MAX_VERTS);
		ps.fexcl = (float4*)buf("fexcl", P * 16);
		ps.nee_base = (float4*)buf("neeb", P * 16);
		if (!ps.adj || !ps.valb || !ps.vpid || !ps.nee_param || !ps.vdsc || !ps.fexcl || !ps.nee_base)
			return rc ? rc : PSY_ERR_OOM;
	}
	WaveQueues& wq = ws->wq;
	wq.q0 = (int*)buf("q0", P * 4);
	wq.q1 = (int*)buf("q1", P * 4);
	wq.counters = (int*)buf("counters", sizeof(int) * render_counter_count(path_length));
	wq.rays = (unsigned long long*)buf("rays", 2 * TC_COUNT * sizeof(unsigned long long));
	WaveBufs& wb = ws->wb;
	wb.cap = (int)P;
	wb.ray[0] = (float4*)buf("ray0", P * 80);
	wb.ray[1] = (float4*)buf("ray1", P * 80);
	wb.hit_f = (float4*)buf("hitf", P * 16);
	wb.hit_i = (int4*)buf("hiti", P * 48);
	wb.occl = (uint8_t*)buf("occl", P);
	if (!ps.smp || !ps.dimstep || !ps.wl || !ps.time || !ps.last_pdf || !ps.col || !ps.fcol || !ps.lcol ||
	    !ps.hit || !ps.pray || !ps.hitx || !ps.sample || !ps.rid || !wq.q0 || !wq.q1 || !wq.counters || !wq.rays || !wb.ray[0] ||
	    !wb.ray[1] || !wb.hit_f || !wb.hit_i || !wb.occl)
		return rc ? rc : PSY_ERR_OOM;
	return PSY_OK;
}

// Profiling: makes room for `pairs` more traversal-launch timings.  The
// event pool grows as needed, so every launch of the profiled region is
// timed.
static int timer_reserve(psy_ctx* ctx, int pairs) {
	const size_t need = 2 * (size_t)(ctx->timer_used + pairs);
	if (ctx->timer_events.size() < need) {
		size_t n = ctx->timer_events.size();
		size_t cap = n ? n : 2 * (size_t)PSY_PROFILE_MAX_LAUNCHES;
		while (cap < need) cap *= 2;
		ctx->timer_events.resize(cap, nullptr);
		for (size_t k = n; k < cap; ++k) {
			const int rc = ctx_cuda(ctx, cudaEventCreate(&ctx->timer_events[k]), "profiling: event");
			if (rc) {
				ctx->timer_events.resize(k);
				return rc;
			}
		}
	}
	ctx->timer.events = ctx->timer_events.data();
	ctx->timer.capacity = (int)(ctx->timer_events.size() / 2);
	ctx->timer.used = &ctx->timer_used;
	return PSY_OK;
}

// One render in waves of P paths (a multiple of spp), on the context's
// "r_" scratch buffers.
static int render_single(psy_ctx* ctx, const psy_render_desc* desc, const RenderParams& rp, bool adjoint,
                         psy_render_stats* stats, cudaStream_t st) {
	cudaSetDevice(ctx->device);
	int rc;
	const uint64_t total = (uint64_t)desc->width * desc->height * desc->spp;
	uint64_t want = desc->stream_paths ? desc->stream_paths : (1ull << 21);
	if (want > (1ull << 26)) want = 1ull << 26;
	uint64_t P = (want / desc->spp) * desc->spp;
	if (P < desc->spp) P = desc->spp;
	if (P > total) P = total;
	WaveSet ws;
	if ((rc = wave_set(ctx, "r_", P, rp.path_length, &ws, adjoint))) return rc;
	if ((rc = ctx_cuda(ctx, cudaMemsetAsync(ws.wq.rays, 0, 2 * TC_COUNT * sizeof(unsigned long long), st), "memset")))
		return rc;
	ctx->last_counts = ws.wq.rays;
	uint32_t launches = 0, waves = 0;
	for (uint64_t base = 0; base < total; base += P) {
		// each wave launches 2 * path_length traversal kernels
		if (ctx->profiling && (rc = timer_reserve(ctx, 2 * (int)rp.path_length))) return rc;
		WaveRange wv;
		wv.base = base;
		wv.paths = (int)((total - base) < P ? (total - base) : P);
		wv.pix_base = base / desc->spp;
		wv.pixels = wv.paths / (int)desc->spp;
		if ((rc = ctx_cuda(ctx,
		                   launch_render_wave(ctx->dev, ctx->halton, rp, wv, ws.ps, ws.wb, ws.wq, ctx->d_status,
		                                      (int)desc->block_size, st, &launches,
		                                      ctx->profiling ? &ctx->timer : nullptr),
		                   "render launch")))
			return rc;
		++waves;
	}
	if (stats) {
		unsigned long long cnt[2 * TC_COUNT] = {};
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(cnt, ws.wq.rays, sizeof(cnt), cudaMemcpyDeviceToHost, st), "D2H")))
			return rc;
		if ((rc = ctx->check_status(st))) return rc;
		stats->paths = total;
		stats->rays = cnt[TC_RAYS] + cnt[TC_COUNT + TC_RAYS];
		stats->occlusion_rays = cnt[TC_COUNT + TC_RAYS];
		stats->launches = launches;
		stats->waves = waves;
	}
	return PSY_OK;
}

// Validates a parameter description against the scene and uploads its
// index tables into rp.
static int diff_params(psy_ctx* ctx, const psy_diff_desc* d, const char* who, RenderParams* rp) {
	const size_t ns = ctx->host->shaders.size(), no = ctx->host->objects.size();
	if (!d->params && d->param_count) return ctx_fail(ctx, PSY_ERR_ARG, "%s: params is NULL", who);
	if (d->shader_count != ns || (ns && !d->shader_param))
		return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader_param must have one entry per scene shader (%zu)", who, ns);
	if (d->object_count != no || (no && !d->object_param))
		return ctx_fail(ctx, PSY_ERR_ARG, "%s: object_param must have one entry per scene object (%zu)", who, no);
	if (d->shader_scale_count != 0 && (d->shader_scale_count != ns || !d->shader_scale_param))
		return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader_scale_param must be empty or have one entry per scene shader (%zu)",
		                who, ns);
	const int pc = (int)d->param_count;
	// one device entry per shader: weights (>= 0), a scale q (-2 - q), or none (-1)
	std::vector<int> code(ns, -1);
	for (size_t i = 0; i < ns; ++i) {
		const int p = d->shader_param[i];
		const int q = d->shader_scale_count ? d->shader_scale_param[i] : -1;
		if (p < -1 || (p >= 0 && p + 3 >= pc))
			return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader %zu's albedo weights %d..%d are outside the %d parameters", who,
			                i, p, p + 3, pc);
		if (q < -1 || q >= pc)
			return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader %zu's albedo scale %d is out of range", who, i, q);
		if (p >= 0 && q >= 0)
			return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader %zu has both basis weights and a scale", who, i);
		if ((p >= 0 || q >= 0) && ctx->host->shaders[i].kind != SHADER_LAMBERT)
			return ctx_fail(ctx, PSY_ERR_ARG, "%s: shader %zu is not Lambert", who, i);
		code[i] = p >= 0 ? p : (q >= 0 ? -2 - q : -1);
	}
	for (size_t i = 0; i < no; ++i) {
		const int p = d->object_param[i];
		if (p < -1 || p >= pc) return ctx_fail(ctx, PSY_ERR_ARG, "%s: object %zu's parameter %d is out of range", who, i, p);
		if (p >= 0 && ctx->host->objects[i].kind != OBJ_SPHERE_LIGHT && ctx->host->objects[i].kind != OBJ_RECT_LIGHT)
			return ctx_fail(ctx, PSY_ERR_ARG, "%s: object %zu is not a light", who, i);
	}
	int rc;
	int* sp = static_cast<int*>(ctx->scratch_buffer("d_spar", sizeof(int) * (ns ? ns : 1), &rc));
	if (!sp) return rc;
	int* op = static_cast<int*>(ctx->scratch_buffer("d_opar", sizeof(int) * (no ? no : 1), &rc));
	if (!op) return rc;
	if (ns && (rc = ctx_cuda(ctx, cudaMemcpy(sp, code.data(), sizeof(int) * ns, cudaMemcpyHostToDevice), who)))
		return rc;
	if (no && (rc = ctx_cuda(ctx, cudaMemcpy(op, d->object_param, sizeof(int) * no, cudaMemcpyHostToDevice), who)))
		return rc;
	rp->params = d->params;
	rp->shader_param = sp;
	rp->object_param = op;
	rp->param_count = pc;
	return PSY_OK;
}

// The batch: renders laid end to end in one global path space, rendered in
// waves of at most P paths that end on pixel boundaries.
static int render_batch(psy_ctx* ctx, const psy_batch_desc* b, psy_render_stats* stats, cudaStream_t st) {
	if (b->count == 0) return PSY_OK;
	if (!b->scenes || !b->renders || !b->xyz)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_batch: scenes, renders and xyz are required");
	if (b->count > 65535) return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_batch: at most 65535 renders");
	cudaSetDevice(ctx->device);
	std::vector<RenderParams> rps(b->count);
	std::vector<DevScene> scs(b->count);
	uint64_t total = 0, pixels = 0;
	uint32_t max_len = 1, max_spp = 1;
	unsigned features = 0;
	int rc;
	for (uint32_t i = 0; i < b->count; ++i) {
		psy_ctx* sc = b->scenes[i];
		if (!sc) return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_batch: render %u has no scene context", i);
		if (sc->device != ctx->device)
			return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_batch: render %u's scene is on another device", i);
		if ((rc = check_render(sc, &b->renders[i], "psy_render_batch")))
			return ctx_fail(ctx, rc, "render %u: %s", i, sc->last_error.c_str());
		if (!b->xyz[i]) return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_batch: render %u has no film", i);
		rps[i] = render_params(sc, &b->renders[i], b->xyz[i], b->counts ? b->counts[i] : nullptr);
		rps[i].path_base = total;
		rps[i].pixel_base = pixels;
		scs[i] = sc->dev;
		const uint64_t px = (uint64_t)b->renders[i].width * b->renders[i].height;
		pixels += px;
		total += px * b->renders[i].spp;
		if (rps[i].path_length > max_len) max_len = rps[i].path_length;
		if (rps[i].spp > max_spp) max_spp = rps[i].spp;
		features |= sc->dev.features;
	}
	uint64_t P = b->stream_paths ? b->stream_paths : (ctx->tuned_stream_paths ? ctx->tuned_stream_paths : (1u << 21));
	if (P > (1ull << 26)) P = 1ull << 26;
	if (P < max_spp) P = max_spp;
	if (P > total) P = total;
	const int block = (int)(b->block_size ? b->block_size : (ctx->tuned_block ? ctx->tuned_block : 128));
	WaveSet ws;
	if ((rc = wave_set(ctx, "b_", P, max_len, &ws))) return rc;
	DevScene* d_scs = static_cast<DevScene*>(ctx->scratch_buffer("b_scenes", sizeof(DevScene) * b->count, &rc));
	if (!d_scs) return rc;
	RenderParams* d_rps = static_cast<RenderParams*>(ctx->scratch_buffer("b_renders", sizeof(RenderParams) * b->count, &rc));
	if (!d_rps) return rc;
	if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(d_scs, scs.data(), sizeof(DevScene) * b->count, cudaMemcpyHostToDevice, st),
	                   "psy_render_batch: scene table")))
		return rc;
	if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(d_rps, rps.data(), sizeof(RenderParams) * b->count, cudaMemcpyHostToDevice,
	                                        st),
	                   "psy_render_batch: render table")))
		return rc;
	if ((rc = ctx_cuda(ctx, cudaMemsetAsync(ws.wq.rays, 0, 2 * TC_COUNT * sizeof(unsigned long long), st), "memset")))
		return rc;
	// waves on pixel boundaries
	std::vector<WaveRange> waves;
	{
		uint64_t base = 0, pix = 0;
		uint32_t r = 0;
		while (base < total) {
			uint64_t end = base + P < total ? base + P : total;
			// the render containing path end - 1, and the end of its last whole pixel
			while (r + 1 < b->count && rps[r + 1].path_base < end) ++r;
			uint32_t rr = r;
			uint64_t local = end - rps[rr].path_base;
			uint64_t cut = rps[rr].path_base + (local / rps[rr].spp) * rps[rr].spp;
			if (cut <= base) cut = end;  // cannot happen with P >= max spp
			end = cut;
			WaveRange wv;
			wv.base = base;
			wv.paths = (int)(end - base);
			wv.pix_base = pix;
			// pixels of the wave
			uint64_t np = 0;
			for (uint32_t k = 0; k < b->count; ++k) {
				const uint64_t lo = rps[k].path_base, hi = lo + (uint64_t)rps[k].width * rps[k].height * rps[k].spp;
				const uint64_t a = base > lo ? base : lo, c = end < hi ? end : hi;
				if (c > a) np += (c - a) / rps[k].spp;
			}
			wv.pixels = (int)np;
			waves.push_back(wv);
			pix += np;
			base = end;
		}
	}
	uint32_t launches = 0;
	auto launch_all = [&](cudaStream_t s) -> int {
		for (const WaveRange& wv : waves) {
			const cudaError_t e = launch_batch_wave(d_scs, d_rps, (int)b->count, features, max_len, ctx->halton, wv,
			                                        ws.ps, ws.wb, ws.wq, ctx->d_status, block, s, &launches);
			if (e != cudaSuccess) return ctx_cuda(ctx, e, "psy_render_batch: launch");
		}
		return PSY_OK;
	};
	if (b->use_graph) {
		// the graph is valid while the launch parameters are the same
		std::vector<uint8_t> key;
		auto put = [&](const void* p, size_t n) {
			const uint8_t* c = static_cast<const uint8_t*>(p);
			key.insert(key.end(), c, c + n);
		};
		put(&P, sizeof(P));
		put(&block, sizeof(block));
		put(&features, sizeof(features));
		put(&max_len, sizeof(max_len));
		put(&ws, sizeof(ws));
		put(&d_scs, sizeof(d_scs));
		put(&d_rps, sizeof(d_rps));
		const uint32_t cnt = b->count;
		put(&cnt, sizeof(cnt));
		for (const WaveRange& wv : waves) put(&wv, sizeof(wv));
		if (!ctx->batch_graph || key != ctx->batch_graph_key) {
			if (ctx->batch_graph) {
				cudaGraphExecDestroy(ctx->batch_graph);
				ctx->batch_graph = nullptr;
			}
			if (!ctx->capture_stream &&
			    (rc = ctx_cuda(ctx, cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking),
			                   "psy_render_batch: stream")))
				return rc;
			if ((rc = ctx_cuda(ctx, cudaStreamBeginCapture(ctx->capture_stream, cudaStreamCaptureModeThreadLocal),
			                   "psy_render_batch: begin capture")))
				return rc;
			const int lrc = launch_all(ctx->capture_stream);
			cudaGraph_t graph = nullptr;
			const cudaError_t ee = cudaStreamEndCapture(ctx->capture_stream, &graph);
			if (lrc) {
				if (graph) cudaGraphDestroy(graph);
				return lrc;
			}
			if ((rc = ctx_cuda(ctx, ee, "psy_render_batch: end capture"))) return rc;
			const cudaError_t ie = cudaGraphInstantiate(&ctx->batch_graph, graph, 0);
			cudaGraphDestroy(graph);
			if ((rc = ctx_cuda(ctx, ie, "psy_render_batch: instantiate"))) {
				ctx->batch_graph = nullptr;
				return rc;
			}
			ctx->batch_graph_key = key;
		} else {
			// the launch count of the captured sequence
			for (size_t i = 0; i < waves.size(); ++i) launches += 2 + 4 * max_len;
		}
		if ((rc = ctx_cuda(ctx, cudaGraphLaunch(ctx->batch_graph, st), "psy_render_batch: graph launch"))) return rc;
	} else {
		if ((rc = launch_all(st))) return rc;
	}
	if (stats) {
		unsigned long long cnt[2 * TC_COUNT] = {};
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(cnt, ws.wq.rays, sizeof(cnt), cudaMemcpyDeviceToHost, st), "D2H")))
			return rc;
		if ((rc = ctx->check_status(st))) return rc;
		stats->paths = total;
		stats->rays = cnt[TC_RAYS] + cnt[TC_COUNT + TC_RAYS];
		stats->occlusion_rays = cnt[TC_COUNT + TC_RAYS];
		stats->launches = launches;
		stats->waves = (uint32_t)waves.size();
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
	{
		const HostRcp& hr = host_rcp();
		void* p = nullptr;
		const size_t bytes = hr.entries.size() * sizeof(uint32_t);
		if (cudaMalloc(&p, bytes) != cudaSuccess) return PSY_ERR_OOM;
		ctx->const_allocs.push_back(p);
		if (cudaMemcpy(p, hr.entries.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return PSY_ERR_DEVICE;
		ctx->rcp = RcpTable{static_cast<const uint32_t*>(p), hr.shift};
	}
	// the fixed array of psy_trace_host_noalloc is reserved now, so that its
	// first call allocates nothing
	if (noalloc_reserve(ctx.get()) != PSY_OK) return PSY_ERR_OOM;
	*out = ctx.release();
	return PSY_OK;
}

void psy_ctx_destroy(psy_ctx* ctx) { delete ctx; }

const char* psy_last_error(const psy_ctx* ctx) {
	if (!ctx) return "no context";
	return ctx->last_error.c_str();
}

int psy_scene_upload(psy_ctx* ctx, const psy_scene_desc* desc) { return psy_scene_upload_ex(ctx, desc, 0u); }

int psy_scene_upload_ex(psy_ctx* ctx, const psy_scene_desc* desc, uint32_t flags) {
	if (!ctx) return PSY_ERR_ARG;
	if (flags & ~PSY_UPLOAD_GPU_BVH) return ctx_fail(ctx, PSY_ERR_ARG, "psy_scene_upload_ex: unknown flags %#x", flags);
	cudaSetDevice(ctx->device);
	std::unique_ptr<BuiltScene> b(new BuiltScene());
	std::string err;
	int rc = build_scene(desc, b.get(), &err, (flags & PSY_UPLOAD_GPU_BVH) != 0);
	if (rc != PSY_OK) return ctx_fail(ctx, rc, "scene: %s", err.c_str());
	ctx->free_scene();
	DevScene& d = ctx->dev;
	void* p;
#define UP(field, vec)                                                                        \
	if ((rc = ctx->upload(vec.data(), vec.size() * sizeof(vec[0]), &p)) != PSY_OK) return rc; \
	d.field = static_cast<decltype(d.field)>(p);
	ctx->gpu_bvh_nodes = -1;
	if (b->gpu_root_pending) {
		// the host-built nodes, then room for the root's device-built ones
		const int n = (int)b->gpu_leaf_first.size() - 1;
		const size_t host_nodes = b->nodes.size();
		const size_t cap = host_nodes + (size_t)(n > 1 ? n - 1 : 0);
		void* np = nullptr;
		if ((rc = ctx_cuda(ctx, cudaMalloc(&np, (cap ? cap : 1) * sizeof(DevNode)), "cudaMalloc(nodes)"))) return rc;
		ctx->scene_allocs.push_back(np);
		ctx->device_bytes += cap * sizeof(DevNode);
		if (host_nodes && (rc = ctx_cuda(ctx, cudaMemcpy(np, b->nodes.data(), host_nodes * sizeof(DevNode),
		                                                 cudaMemcpyHostToDevice), "cudaMemcpy(nodes)")))
			return rc;
		// the host-built nodes' later time samples, then room for the device
		// nodes' (at most one record per sample after the first)
		int most = 1;
		for (int i = 0; i < n; ++i) most = std::max(most, b->gpu_leaf_first[i + 1] - b->gpu_leaf_first[i]);
		const size_t host_extra = b->node_extra.size();
		const size_t extra_cap = host_extra + (size_t)(n > 1 ? n - 1 : 0) * (size_t)(most - 1) * 24;
		void* ep = nullptr;
		if ((rc = ctx_cuda(ctx, cudaMalloc(&ep, (extra_cap ? extra_cap : 1) * sizeof(float)), "cudaMalloc(node_extra)")))
			return rc;
		ctx->scene_allocs.push_back(ep);
		ctx->device_bytes += extra_cap * sizeof(float);
		if (host_extra && (rc = ctx_cuda(ctx, cudaMemcpy(ep, b->node_extra.data(), host_extra * sizeof(float),
		                                                 cudaMemcpyHostToDevice), "cudaMemcpy(node_extra)")))
			return rc;
		int root = REF_EMPTY, count = 0, extras = 0;
		if ((rc = ctx_cuda(ctx, build_bvh4_gpu(b->gpu_leaf_boxes.data(), b->gpu_leaf_first.data(),
		                                       b->gpu_leaf_centres.data(), n, (int)host_nodes,
		                                       static_cast<DevNode*>(np) + host_nodes,
		                                       static_cast<float*>(ep) + host_extra, (int)(host_extra / 24), &root,
		                                       &count, &extras, nullptr),
		                   "psy_scene_upload_ex: device BVH build")))
			return rc;
		b->assemblies[0].root = root;
		ctx->gpu_bvh_nodes = count;
		d.nodes = static_cast<const DevNode*>(np);
		d.node_extra = static_cast<const float*>(ep);
	} else {
		UP(nodes, b->nodes);
		UP(node_extra, b->node_extra);
	}
	ctx->gpu_light_nodes = -1;
	if (b->gpu_light_pending) {
		// the host-built light nodes, then the root's device-built tree
		const int n = (int)b->gpu_light_first.size() - 1;
		const size_t host_nodes = b->light_nodes.size();
		const size_t cap = host_nodes + 2 * (size_t)n - 1;
		void* lp = nullptr;
		if ((rc = ctx_cuda(ctx, cudaMalloc(&lp, cap * sizeof(DevLightNode)), "cudaMalloc(light_nodes)"))) return rc;
		ctx->scene_allocs.push_back(lp);
		ctx->device_bytes += cap * sizeof(DevLightNode);
		if (host_nodes && (rc = ctx_cuda(ctx, cudaMemcpy(lp, b->light_nodes.data(), host_nodes * sizeof(DevLightNode),
		                                                 cudaMemcpyHostToDevice), "cudaMemcpy(light_nodes)")))
			return rc;
		// the host-built nodes' later bounds samples, then room for the device
		// nodes' (at most one record per sample after the first)
		int most = 1;
		for (int i = 0; i < n; ++i) most = std::max(most, b->gpu_light_first[i + 1] - b->gpu_light_first[i]);
		const size_t host_extra = b->light_extra.size();
		const size_t extra_cap = host_extra + (2 * (size_t)n - 1) * (size_t)(most - 1) * 6;
		void* xp = nullptr;
		if ((rc = ctx_cuda(ctx, cudaMalloc(&xp, (extra_cap ? extra_cap : 1) * sizeof(float)),
		                   "cudaMalloc(light_extra)")))
			return rc;
		ctx->scene_allocs.push_back(xp);
		ctx->device_bytes += extra_cap * sizeof(float);
		if (host_extra && (rc = ctx_cuda(ctx, cudaMemcpy(xp, b->light_extra.data(), host_extra * sizeof(float),
		                                                 cudaMemcpyHostToDevice), "cudaMemcpy(light_extra)")))
			return rc;
		float energy = 0.0f;
		int extras = 0;
		if ((rc = ctx_cuda(ctx, build_light_tree_gpu(b->gpu_light_elems.data(), b->gpu_light_samples.data(),
		                                             b->gpu_light_first.data(), n, (int)host_nodes,
		                                             static_cast<DevLightNode*>(lp) + host_nodes,
		                                             static_cast<float*>(xp) + host_extra, (int)(host_extra / 6),
		                                             &energy, &extras, nullptr),
		                   "psy_scene_upload_ex: device light tree build")))
			return rc;
		d.light_extra = static_cast<const float*>(xp);
		b->assemblies[0].light_root = (int)host_nodes;
		b->assemblies[0].light_energy = energy;
		ctx->gpu_light_nodes = 2 * n - 1;
		d.light_nodes = static_cast<const DevLightNode*>(lp);
	} else {
		UP(light_nodes, b->light_nodes);
		UP(light_extra, b->light_extra);
	}
	UP(assemblies, b->assemblies);
	UP(instances, b->instances);
	UP(objects, b->objects);
	UP(xforms, b->xforms);
	UP(fpool, b->fpool);
	UP(shaders, b->shaders);
	UP(cam_xforms, b->cam_xforms);
	UP(cam_tfovs, b->cam_tfovs);
	UP(cam_apertures, b->cam_apertures);
	UP(cam_focus, b->cam_focus);
#undef UP
	d.assembly_count = (int)b->assemblies.size();
	d.light_node_count = (int)b->light_nodes.size() + (ctx->gpu_light_nodes > 0 ? ctx->gpu_light_nodes : 0);
	d.rcp = ctx->rcp;
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
	out->bvh4_nodes = (uint32_t)ctx->host->nodes.size() + (uint32_t)(ctx->gpu_bvh_nodes > 0 ? ctx->gpu_bvh_nodes : 0);
	out->light_nodes =
	    (uint32_t)ctx->host->light_nodes.size() + (uint32_t)(ctx->gpu_light_nodes > 0 ? ctx->gpu_light_nodes : 0);
	out->lights = ctx->host->total_lights;
	out->device_bytes = ctx->device_bytes;
	out->gpu_bvh4_nodes = (uint32_t)(ctx->gpu_bvh_nodes > 0 ? ctx->gpu_bvh_nodes : 0);
	out->gpu_light_nodes = (uint32_t)(ctx->gpu_light_nodes > 0 ? ctx->gpu_light_nodes : 0);
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
	int rc = check_render(ctx, desc, "psy_render");
	if (rc) return rc;
	return render_single(ctx, desc, render_params(ctx, desc, xyz, counts), false, stats, (cudaStream_t)stream);
}

int psy_render_diff(psy_ctx* ctx, const psy_render_desc* desc, const psy_diff_desc* diff, float* xyz,
                    uint32_t* counts, psy_render_stats* stats, void* stream) {
	if (!ctx || !desc || !diff || !xyz) return PSY_ERR_ARG;
	int rc = check_render(ctx, desc, "psy_render_diff");
	if (rc) return rc;
	RenderParams rp = render_params(ctx, desc, xyz, counts);
	if ((rc = diff_params(ctx, diff, "psy_render_diff", &rp))) return rc;
	return render_single(ctx, desc, rp, false, stats, (cudaStream_t)stream);
}

int psy_render_adjoint(psy_ctx* ctx, const psy_render_desc* desc, const psy_diff_desc* diff, const float* dl_dxyz,
                       float* grad, psy_render_stats* stats, void* stream) {
	if (!ctx || !desc || !diff || !dl_dxyz || !grad) return PSY_ERR_ARG;
	int rc = check_render(ctx, desc, "psy_render_adjoint");
	if (rc) return rc;
	if ((desc->path_length ? desc->path_length : 4) > PSY_ADJOINT_MAX_PATH)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_render_adjoint: path_length must be at most %d", PSY_ADJOINT_MAX_PATH);
	// the replay renders into a scratch film: only the gradient is kept
	const size_t npx = (size_t)desc->width * desc->height;
	float* film = static_cast<float*>(ctx->scratch_buffer("a_film", npx * 3 * sizeof(float), &rc));
	if (!film) return rc;
	RenderParams rp = render_params(ctx, desc, film, nullptr);
	if ((rc = diff_params(ctx, diff, "psy_render_adjoint", &rp))) return rc;
	rp.dl_dxyz = dl_dxyz;
	rp.grad = grad;
	rp.grad_in_smem = (size_t)rp.param_count * sizeof(float) <= 32768 ? 1 : 0;
	return render_single(ctx, desc, rp, true, stats, (cudaStream_t)stream);
}

int psy_render_batch(psy_ctx* ctx, const psy_batch_desc* b, psy_render_stats* stats, void* stream) {
	if (!ctx || !b) return PSY_ERR_ARG;
	return render_batch(ctx, b, stats, (cudaStream_t)stream);
}

int psy_batch_autotune(psy_ctx* ctx, const psy_batch_desc* b, uint32_t spp_divisor, psy_batch_tuning* out) {
	if (!ctx || !b || !out) return PSY_ERR_ARG;
	if (b->count == 0 || !b->scenes || !b->renders)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_batch_autotune: empty batch");
	cudaSetDevice(ctx->device);
	if (spp_divisor == 0) spp_divisor = 1;
	// the tuning batch: the same renders with fewer samples, on scratch films
	std::vector<psy_render_desc> descs(b->renders, b->renders + b->count);
	size_t film = 0;
	std::vector<size_t> offs(b->count);
	for (uint32_t i = 0; i < b->count; ++i) {
		descs[i].spp = descs[i].spp / spp_divisor ? descs[i].spp / spp_divisor : 1;
		offs[i] = film;
		film += (size_t)descs[i].width * descs[i].height * 3;
	}
	int rc;
	float* tfilm = static_cast<float*>(ctx->scratch_buffer("t_film", film * sizeof(float), &rc));
	if (!tfilm) return rc;
	std::vector<float*> films(b->count);
	for (uint32_t i = 0; i < b->count; ++i) films[i] = tfilm + offs[i];
	psy_batch_desc t = *b;
	t.renders = descs.data();
	t.xyz = films.data();
	t.counts = nullptr;
	cudaStream_t st = nullptr;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	const uint32_t blocks[3] = {64, 128, 256};
	psy_batch_tuning best{};
	best.ms = -1.0f;
	uint32_t trials = 0;
	for (uint32_t lg = 14; lg <= 22 && rc == PSY_OK; ++lg) {
		for (uint32_t bi = 0; bi < 3; ++bi) {
			t.stream_paths = 1u << lg;
			t.block_size = blocks[bi];
			if (trials == 0 && (rc = render_batch(ctx, &t, nullptr, st))) break;  // warm-up
			cudaEventRecord(e0, st);
			if ((rc = render_batch(ctx, &t, nullptr, st))) break;
			cudaEventRecord(e1, st);
			if ((rc = ctx_cuda(ctx, cudaEventSynchronize(e1), "psy_batch_autotune: synchronize"))) break;
			float ms = 0.0f;
			cudaEventElapsedTime(&ms, e0, e1);
			++trials;
			if (best.ms < 0.0f || ms < best.ms) {
				best.ms = ms;
				best.stream_paths = t.stream_paths;
				best.block_size = t.block_size;
			}
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (rc) return rc;
	if ((rc = ctx->check_status(st))) return rc;
	best.trials = trials;
	ctx->tuned_stream_paths = best.stream_paths;
	ctx->tuned_block = best.block_size;
	*out = best;
	return PSY_OK;
}

int psy_profile_enable(psy_ctx* ctx, int on) {
	if (!ctx) return PSY_ERR_ARG;
	cudaSetDevice(ctx->device);
	ctx->timer_used = 0;
	if (on) {
		const int rc = timer_reserve(ctx, PSY_PROFILE_MAX_LAUNCHES);
		if (rc) return rc;
	}
	ctx->profiling = on != 0;
	return PSY_OK;
}

int psy_profile_counters(psy_ctx* ctx, psy_trace_counters* closest, psy_trace_counters* occlusion) {
	if (!ctx) return PSY_ERR_ARG;
	if (!ctx->last_counts) return ctx_fail(ctx, PSY_ERR_ARG, "psy_profile_counters: no render on this context yet");
	cudaSetDevice(ctx->device);
	int rc = ctx_cuda(ctx, cudaDeviceSynchronize(), "psy_profile_counters: synchronize");
	if (rc) return rc;
	unsigned long long cnt[2 * TC_COUNT] = {};
	if ((rc = ctx_cuda(ctx, cudaMemcpy(cnt, ctx->last_counts, sizeof(cnt), cudaMemcpyDeviceToHost),
	                   "psy_profile_counters: read")))
		return rc;
	psy_trace_counters* outs[2] = {closest, occlusion};
	for (int k = 0; k < 2; ++k) {
		if (!outs[k]) continue;
		const unsigned long long* c = cnt + k * TC_COUNT;
		outs[k]->rays = c[TC_RAYS];
		outs[k]->node_visits = c[TC_NODES];
		outs[k]->leaf_visits = c[TC_LEAVES];
		outs[k]->patch_iterations = c[TC_PATCH_ITERS];
		outs[k]->warp_steps = c[TC_WARP_STEPS];
		outs[k]->lane_steps = c[TC_LANE_STEPS];
	}
	return PSY_OK;
}

int psy_profile_read(psy_ctx* ctx, double* trace_ms, uint32_t* launches) {
	if (!ctx || !trace_ms || !launches) return PSY_ERR_ARG;
	cudaSetDevice(ctx->device);
	double ms = 0.0;
	for (int k = 0; k < ctx->timer_used; ++k) {
		int rc = ctx_cuda(ctx, cudaEventSynchronize(ctx->timer_events[2 * k + 1]), "psy_profile_read: synchronize");
		if (rc) return rc;
		float e = 0.0f;
		if ((rc = ctx_cuda(ctx, cudaEventElapsedTime(&e, ctx->timer_events[2 * k], ctx->timer_events[2 * k + 1]),
		                   "psy_profile_read: elapsed")))
			return rc;
		ms += e;
	}
	*trace_ms = ms;
	*launches = (uint32_t)ctx->timer_used;
	ctx->timer_used = 0;
	return PSY_OK;
}

}  // extern "C"
