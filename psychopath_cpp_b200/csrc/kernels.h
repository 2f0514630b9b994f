/*
 * Internal interface between the C ABI layer and the CUDA kernels.
 */
#ifndef PSY_KERNELS_H
#define PSY_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "psy_scene.h"

namespace psy {

struct RaySoA {
	const float *o, *d, *odx, *ody, *ddx, *ddy, *time;
	const uint16_t* type;
};

struct HitSoA {
	uint8_t* hit;
	uint64_t* id;
	float *t, *uv, *p, *n, *dpdu, *dpdv, *dndu, *dndv;
	uint8_t* backfacing;
	float* light_pdf;
	float* offset;
	float* space;
	uint8_t* closure;
	float* closure_color;
	int want_geometry;  // any geometry field requested
};

cudaError_t launch_trace(const DevScene& sc, const RaySoA& rays, const HitSoA& hits, uint32_t n, unsigned* status,
                         cudaStream_t stream);

}  // namespace psy

#endif
