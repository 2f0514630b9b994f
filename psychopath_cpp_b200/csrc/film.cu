/*
 * Film output: the per-pixel XYZ sums and sample counts that psy_render
 * accumulates, converted to 8-bit sRGB scanlines as
 * Film::scanline_image_8bbc does (reference film/film.hpp:173-225, with
 * XYZ_to_sRGB_E and sRGB_gamma from color/color.hpp:384-439):
 *   - a pixel without samples shows the grey checkerboard (0.5 / 0.35 in
 *     16-pixel squares);
 *   - otherwise the mean XYZ goes through the whitepoint-E sRGB matrix,
 *     clamped to [0, 1], then the sRGB transfer curve;
 *   - each channel is scaled to [0, 255], dithered, clamped and truncated.
 * The reference dithers with its film's RNG, seeded from the clock
 * (utils/rng.hpp), so its dither is not reproducible; here the dither of a
 * channel is a hash of (seed, pixel, channel) in [-0.5, 0.5), the same
 * distribution, or 0 when the caller asks for none.
 */
#include "../../include/psy_b200.h"
#include "kernels.h"
#include "psy_ctx.h"

namespace psy {

__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float clamp01(float v) { return std_min(1.0f, std_max(0.0f, v)); }

__device__ __forceinline__ float srgb_gamma(float n) {
	return n < 0.0031308f ? (n * 12.92f) : ((1.055f * powf(n, 1.0f / 2.4f)) - 0.055f);
}

// A uniform float in [-0.5, 0.5) from a 32-bit hash (the integer finaliser
// of MurmurHash3, applied twice over the inputs).
__device__ __forceinline__ float dither(uint32_t seed, uint32_t pixel, uint32_t channel) {
	uint32_t h = seed ^ (pixel * 0x9e3779b9u) ^ (channel * 0x85ebca6bu);
	for (int k = 0; k < 2; ++k) {
		h ^= h >> 16;
		h *= 0x85ebca6bu;
		h ^= h >> 13;
		h *= 0xc2b2ae35u;
		h ^= h >> 16;
	}
	return (float)(h >> 8) * (1.0f / 16777216.0f) - 0.5f;
}

__global__ void film_srgb8_kernel(const float* __restrict__ xyz, const uint32_t* __restrict__ counts, uint32_t width,
                                  uint32_t height, int dithered, uint32_t seed, uint8_t* __restrict__ out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= width * height) return;
	const uint32_t x = i % width, y = i / width;
	float c[3];
	if (((y % 32) < 16) ^ ((x % 32) < 16)) c[0] = c[1] = c[2] = 0.5f;
	else c[0] = c[1] = c[2] = 0.35f;
	const uint32_t n = counts[i];
	if (n != 0) {
		const float fn = (float)n;
		const float X = xyz[3 * i] / fn, Y = xyz[3 * i + 1] / fn, Z = xyz[3 * i + 2] / fn;
		c[0] = srgb_gamma(clamp01(((X * 2.6897f) + (Y * -1.2759f)) + (Z * -0.4138f)));
		c[1] = srgb_gamma(clamp01(((X * -1.0216f) + (Y * 1.9778f)) + (Z * 0.0438f)));
		c[2] = srgb_gamma(clamp01(((X * 0.0613f) + (Y * -0.2245f)) + (Z * 1.1632f)));
	}
	for (int k = 0; k < 3; ++k) {
		float v = c[k] * 255.0f;
		if (dithered) v += dither(seed, i, (uint32_t)k);
		v = std_min(255.0f, std_max(0.0f, v));
		out[3 * i + k] = (uint8_t)v;
	}
}

}  // namespace psy

extern "C" int psy_film_srgb8(psy_ctx* ctx, const float* xyz, const uint32_t* counts, uint32_t width, uint32_t height,
                              int dithered, uint32_t seed, uint8_t* rgb, void* stream) {
	if (!ctx || !xyz || !counts || !rgb) return PSY_ERR_ARG;
	if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 31))
		return ctx_fail(ctx, PSY_ERR_ARG, "psy_film_srgb8: bad film size %ux%u", width, height);
	cudaSetDevice(ctx->device);
	const uint32_t n = width * height;
	psy::film_srgb8_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(xyz, counts, width, height,
	                                                                                      dithered ? 1 : 0, seed, rgb);
	return ctx_cuda(ctx, cudaGetLastError(), "psy_film_srgb8: launch");
}
