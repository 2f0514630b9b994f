/*
 * psy_trace_host_noalloc: psy_trace_host without any allocation.
 *
 * psy_trace_host keeps its device copies of the rays and hits in per-context
 * scratch buffers that grow with cudaMalloc on demand.  Some callers cannot
 * let a call allocate: a renderer that has already handed all free device
 * memory to its own pool allocator (a fresh cudaMalloc would fail there), or
 * one that keeps other streams busy while it traces small batches
 * (cudaMalloc / cudaFree may synchronise the whole device and stall them).
 * This variant stages everything in one file-scope device array of fixed
 * size instead.
 *
 * Limits, stated in the header as well:
 *  - at most PSY_NOALLOC_MAX_RAYS rays per call; larger requests fail with
 *    PSY_ERR_ARG before any device work;
 *  - the array is one per device and shared by every context on it, so two
 *    calls that overlap in time on the same device (other threads, other
 *    contexts) race on it: callers serialise them;
 *  - the array's address is resolved once per device (cudaGetSymbolAddress).
 *    With CUDA's lazy module loading that is also when the module holding
 *    the array is loaded and the array's device memory is reserved, so
 *    psy_ctx_create does it for its device (noalloc_reserve); a call with
 *    n == 0 does it as well, as an explicit warm-up.  Either must come before
 *    the caller's pool allocator takes the free device memory and before any
 *    stream capture begins on that device.
 * The only part of the array that must start at zero is the status word the
 * kernel ORs its error flags into; each call clears it on its stream before
 * the launch.
 */
#include <cstring>
#include <mutex>

#include "psy_ctx.h"

namespace {

constexpr size_t kMaxRays = PSY_NOALLOC_MAX_RAYS;
constexpr size_t kAlign = 256;

constexpr size_t region(size_t per_ray) { return ((per_ray * kMaxRays + kAlign - 1) / kAlign) * kAlign; }

// Fixed layout: status word, the ray arrays, then one region per hit field.
constexpr size_t kStatusOff = 0;
constexpr size_t kRaysOff = kAlign;
constexpr size_t kRayF3 = region(3 * sizeof(float));
constexpr size_t kRayBytes = 6 * kRayF3 + region(sizeof(float)) + region(sizeof(uint16_t));
constexpr size_t kHitPer[16] = {1, 8, 4, 8, 12, 12, 12, 12, 12, 12, 1, 4, 12, 64, 1, 12};
constexpr size_t hit_bytes() {
	size_t s = 0;
	for (size_t k = 0; k < 16; ++k) s += region(kHitPer[k]);
	return s;
}
constexpr size_t kHitsOff = kRaysOff + kRayBytes;
constexpr size_t kScratchBytes = kHitsOff + hit_bytes();
static_assert(kScratchBytes <= (size_t)18 << 20, "static trace scratch larger than intended");

constexpr int kMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned char psy_noalloc_scratch[kScratchBytes];

static std::mutex g_sym_mu;
static char* g_sym_addr[kMaxDevices];

// Address of psy_noalloc_scratch on `device` (current), resolved once.
static int scratch_address(psy_ctx* ctx, char** out) {
	if (ctx->device < 0 || ctx->device >= kMaxDevices)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_trace_host_noalloc: device %d out of range", ctx->device);
	std::lock_guard<std::mutex> lock(g_sym_mu);
	if (!g_sym_addr[ctx->device]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, psy_noalloc_scratch);
		if (e != cudaSuccess) return ctx_cuda(ctx, e, "psy_trace_host_noalloc: cudaGetSymbolAddress");
		if (!p) return ctx_fail(ctx, PSY_ERR_DEVICE, "psy_trace_host_noalloc: null scratch address");
		g_sym_addr[ctx->device] = static_cast<char*>(p);
	}
	*out = g_sym_addr[ctx->device];
	return PSY_OK;
}

// Resolves the array on ctx's device (current): loads its module, which
// reserves the array, once per device.  psy_ctx_create calls it.
int noalloc_reserve(psy_ctx* ctx) {
	char* base = nullptr;
	return scratch_address(ctx, &base);
}

extern "C" int psy_trace_host_noalloc(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits,
                                      void* stream) {
	if (!ctx) return PSY_ERR_ARG;
	if (n > kMaxRays)
		return ctx_fail(ctx, PSY_ERR_ARG,
		                "psy_trace_host_noalloc: %u rays exceed the static scratch capacity of %u rays per call",
		                n, (unsigned)kMaxRays);
	if (n == 0) {
		// warm-up form: only makes sure the array is resident on this device
		const int rc = ctx_cuda(ctx, cudaSetDevice(ctx->device), "psy_trace_host_noalloc: cudaSetDevice");
		return rc ? rc : noalloc_reserve(ctx);
	}
	if (!ctx->has_scene) return ctx_fail(ctx, PSY_ERR_NO_SCENE, "psy_trace_host_noalloc: no scene uploaded");
	if (!rays || !rays->o || !rays->d || !rays->odx || !rays->ody || !rays->ddx || !rays->ddy || !rays->time)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_trace_host_noalloc: incomplete ray arrays");
	int rc = ctx_cuda(ctx, cudaSetDevice(ctx->device), "psy_trace_host_noalloc: cudaSetDevice");
	if (rc) return rc;
	char* base = nullptr;
	if ((rc = scratch_address(ctx, &base))) return rc;
	cudaStream_t st = static_cast<cudaStream_t>(stream);

	unsigned* d_status = reinterpret_cast<unsigned*>(base + kStatusOff);
	if ((rc = ctx_cuda(ctx, cudaMemsetAsync(d_status, 0, sizeof(unsigned), st), "psy_trace_host_noalloc: clear status")))
		return rc;

	const size_t f3 = (size_t)n * 3 * sizeof(float);
	char* rp = base + kRaysOff;
	float* dr[6];
	for (int k = 0; k < 6; ++k) dr[k] = reinterpret_cast<float*>(rp + k * kRayF3);
	float* d_time = reinterpret_cast<float*>(rp + 6 * kRayF3);
	uint16_t* d_type = reinterpret_cast<uint16_t*>(rp + 6 * kRayF3 + region(sizeof(float)));
	const float* srcs[6] = {rays->o, rays->d, rays->odx, rays->ody, rays->ddx, rays->ddy};
	for (int k = 0; k < 6; ++k)
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(dr[k], srcs[k], f3, cudaMemcpyHostToDevice, st), "H2D rays")))
			return rc;
	if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(d_time, rays->time, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st),
	                   "H2D rays")))
		return rc;
	if (rays->type &&
	    (rc = ctx_cuda(ctx, cudaMemcpyAsync(d_type, rays->type, (size_t)n * sizeof(uint16_t), cudaMemcpyHostToDevice, st),
	                   "H2D rays")))
		return rc;

	void* host[16] = {};
	if (hits) {
		void* h[16] = {hits->hit,  hits->id,   hits->t,          hits->uv,        hits->p,      hits->n,
		               hits->dpdu, hits->dpdv, hits->dndu,       hits->dndv,      hits->backfacing,
		               hits->light_pdf, hits->offset, hits->space, hits->closure, hits->closure_color};
		std::memcpy(host, h, sizeof(h));
	}
	void* dev[16];
	size_t off = kHitsOff;
	for (int k = 0; k < 16; ++k) {
		dev[k] = host[k] ? static_cast<void*>(base + off) : nullptr;
		off += region(kHitPer[k]);
	}
	psy::HitSoA hs;
	hs.hit = static_cast<uint8_t*>(dev[0]);
	hs.id = static_cast<uint64_t*>(dev[1]);
	hs.t = static_cast<float*>(dev[2]);
	hs.uv = static_cast<float*>(dev[3]);
	hs.p = static_cast<float*>(dev[4]);
	hs.n = static_cast<float*>(dev[5]);
	hs.dpdu = static_cast<float*>(dev[6]);
	hs.dpdv = static_cast<float*>(dev[7]);
	hs.dndu = static_cast<float*>(dev[8]);
	hs.dndv = static_cast<float*>(dev[9]);
	hs.backfacing = static_cast<uint8_t*>(dev[10]);
	hs.light_pdf = static_cast<float*>(dev[11]);
	hs.offset = static_cast<float*>(dev[12]);
	hs.space = static_cast<float*>(dev[13]);
	hs.closure = static_cast<uint8_t*>(dev[14]);
	hs.closure_color = static_cast<float*>(dev[15]);
	hs.want_geometry = 0;
	for (int k = 3; k < 16; ++k)
		if (dev[k]) hs.want_geometry = 1;

	const psy::RaySoA rs{dr[0], dr[1], dr[2], dr[3], dr[4], dr[5], d_time, rays->type ? d_type : nullptr};
	if ((rc = ctx_cuda(ctx, psy::launch_trace(ctx->dev, rs, hs, n, d_status, st), "psy_trace_host_noalloc: launch")))
		return rc;
	for (int k = 0; k < 16; ++k) {
		if (!host[k]) continue;
		if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(host[k], dev[k], kHitPer[k] * n, cudaMemcpyDeviceToHost, st),
		                   "D2H hits")))
			return rc;
	}
	unsigned flags = 0;
	if ((rc = ctx_cuda(ctx, cudaMemcpyAsync(&flags, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st),
	                   "status read")))
		return rc;
	if ((rc = ctx_cuda(ctx, cudaStreamSynchronize(st), "stream synchronize"))) return rc;
	if (flags & (psy::ERRF_STACK | psy::ERRF_LEVELS))
		return ctx_fail(ctx, PSY_ERR_STACK_OVERFLOW, "psy_trace_host_noalloc: traversal limits exceeded (flags %#x)",
		                flags);
	if (flags & psy::ERRF_MOTION)
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_trace_host_noalloc: more motion samples than supported (flags %#x)",
		                flags);
	if (flags) return ctx_fail(ctx, PSY_ERR_DEVICE, "psy_trace_host_noalloc: device error flags %#x", flags);
	return PSY_OK;
}
