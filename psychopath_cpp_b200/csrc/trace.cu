/*
 * psy_trace kernel: Tracer::trace for a device ray stream
 * (reference tracer/tracer.cpp:38-121).  One thread per ray; rays are read
 * as SoA float streams and the requested Intersection fields are written as
 * SoA streams.
 */
#include "kernels.h"
#include "shade_geom.cuh"

namespace psy {

__device__ __forceinline__ V3 ld3(const float* p, uint32_t i) {
	return V3(__ldg(p + 3 * (size_t)i), __ldg(p + 3 * (size_t)i + 1), __ldg(p + 3 * (size_t)i + 2));
}
__device__ __forceinline__ void st3(float* p, uint32_t i, V3 v) {
	p[3 * (size_t)i] = v.x;
	p[3 * (size_t)i + 1] = v.y;
	p[3 * (size_t)i + 2] = v.z;
}

// Register cap of the kernel: flat scenes (spheres, lights, bilinear
// patches in one level) run at 64 registers, where more resident warps hide
// the walk's memory latency (the 4M-ray heightfield stream: 1.92 -> 2.15 G
// rays/s against the compiler's 127; 96 and 48 are slower); the larger
// variants keep the compiler's choice.
template <unsigned F>
struct TraceKernelRegs {
	static constexpr int value = F == FEAT_FLAT ? 64 : 255;
};

template <unsigned F>
__global__ void __maxnreg__(TraceKernelRegs<F>::value) trace_kernel(DevScene sc, RaySoA rays, HitSoA hits,
                                                                   uint32_t n, unsigned* status) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	WorldRayD wr;
	wr.o = ld3(rays.o, i);
	wr.d = ld3(rays.d, i);
	wr.odx = ld3(rays.odx, i);
	wr.ody = ld3(rays.ody, i);
	wr.ddx = ld3(rays.ddx, i);
	wr.ddy = ld3(rays.ddy, i);
	wr.time = __ldg(rays.time + i);
	wr.occl = rays.type ? (__ldg(rays.type + i) == 32) : false;

	HitRec rec;
	unsigned err = trace_ray<F>(sc, wr, &rec);
	const bool hit = rec.obj >= 0;
	if (hits.hit) hits.hit[i] = hit ? 1 : 0;
	if (hits.id) hits.id[i] = hit ? rec.id : 0ull;
	if (hits.t) hits.t[i] = (hit && !wr.occl) ? rec.t : INFINITY;
	if (hit && !wr.occl && hits.want_geometry) {
		M44 space;
		const bool xf = hit_space<F>(sc, rec, wr.time, &space, &err);
		V3 lo = wr.o, ld = wr.d;
		if (xf) {
			lo = pos_to(space, wr.o);
			ld = dir_to(space, wr.d);
		} else {
			space = m44_identity();
		}
		HitInfo h;
		hit_geometry(sc, rec, wr.time, lo, ld, &h);
		if (hits.uv) {
			hits.uv[2 * (size_t)i] = h.geo.u;
			hits.uv[2 * (size_t)i + 1] = h.geo.v;
		}
		if (hits.p) st3(hits.p, i, h.geo.p);
		if (hits.n) st3(hits.n, i, h.geo.n);
		if (hits.dpdu) st3(hits.dpdu, i, h.geo.dpdu);
		if (hits.dpdv) st3(hits.dpdv, i, h.geo.dpdv);
		if (hits.dndu) st3(hits.dndu, i, h.geo.dndu);
		if (hits.dndv) st3(hits.dndv, i, h.geo.dndv);
		if (hits.backfacing) hits.backfacing[i] = h.backfacing ? 1 : 0;
		if (hits.light_pdf) hits.light_pdf[i] = h.light_pdf;
		if (hits.offset) st3(hits.offset, i, h.offset);
		if (hits.space)
			for (int k = 0; k < 16; ++k) hits.space[16 * (size_t)i + k] = space.m[k / 4][k % 4];
		if (hits.closure) hits.closure[i] = (uint8_t)h.closure;
		if (hits.closure_color) {
			hits.closure_color[3 * (size_t)i] = h.col[0];
			hits.closure_color[3 * (size_t)i + 1] = h.col[1];
			hits.closure_color[3 * (size_t)i + 2] = h.col[2];
		}
	} else if (hits.want_geometry) {
		if (hits.uv) {
			hits.uv[2 * (size_t)i] = 0.0f;
			hits.uv[2 * (size_t)i + 1] = 0.0f;
		}
		const V3 z(0.0f);
		if (hits.p) st3(hits.p, i, z);
		if (hits.n) st3(hits.n, i, z);
		if (hits.dpdu) st3(hits.dpdu, i, z);
		if (hits.dpdv) st3(hits.dpdv, i, z);
		if (hits.dndu) st3(hits.dndu, i, z);
		if (hits.dndv) st3(hits.dndv, i, z);
		if (hits.backfacing) hits.backfacing[i] = 0;
		if (hits.light_pdf) hits.light_pdf[i] = 9999.0f;
		if (hits.offset) st3(hits.offset, i, z);
		if (hits.space)
			for (int k = 0; k < 16; ++k) hits.space[16 * (size_t)i + k] = (k % 5 == 0) ? 1.0f : 0.0f;
		if (hits.closure) hits.closure[i] = 0;
		if (hits.closure_color) st3(hits.closure_color, i, z);
	}
	if (err) atomicOr(status, err);
}

cudaError_t launch_trace(const DevScene& sc, const RaySoA& rays, const HitSoA& hits, uint32_t n, unsigned* status,
                         cudaStream_t stream) {
	if (n == 0) return cudaSuccess;
	const int block = 128;
	const uint32_t grid = (n + block - 1) / block;
	switch (feature_variant(sc.features)) {
		case FEAT_FLAT: trace_kernel<FEAT_FLAT><<<grid, block, 0, stream>>>(sc, rays, hits, n, status); break;
		case FEAT_STILL_BICUBIC: trace_kernel<FEAT_STILL_BICUBIC><<<grid, block, 0, stream>>>(sc, rays, hits, n, status); break;
		case FEAT_STILL: trace_kernel<FEAT_STILL><<<grid, block, 0, stream>>>(sc, rays, hits, n, status); break;
		default: trace_kernel<FEAT_ALL><<<grid, block, 0, stream>>>(sc, rays, hits, n, status); break;
	}
	return cudaGetLastError();
}

}  // namespace psy
