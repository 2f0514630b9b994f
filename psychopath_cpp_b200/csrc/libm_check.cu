/*
 * Self-check of the device restatements of the host C library's float math
 * (psy_libm.cuh): evaluates one of them on the device over caller-given
 * arguments, so that a test can hold the device's bits against the host
 * library's (sincosf, acosf, asinf, expf) on the same machine.
 */
#include "../../include/psy_b200.h"
#include "psy_ctx.h"
#include "psy_libm.cuh"

namespace psy {

__global__ void libm_check_kernel(uint32_t fn, uint32_t n, const float* __restrict__ x, float* __restrict__ out) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const float v = x[i];
		float r;
		switch (fn) {
			case PSY_MATH_SIN: r = lm_sinf(v); break;
			case PSY_MATH_COS: r = lm_cosf(v); break;
			case PSY_MATH_ACOS: r = lm_acosf(v); break;
			case PSY_MATH_ASIN: r = lm_asinf(v); break;
			default: r = lm_expf(v); break;
		}
		out[i] = r;
	}
}

}  // namespace psy

extern "C" int psy_math_check(psy_ctx* ctx, uint32_t fn, uint32_t n, const float* x, float* out) {
	if (!ctx || (n && (!x || !out))) return PSY_ERR_ARG;
	if (fn > PSY_MATH_EXP) return ctx_fail(ctx, PSY_ERR_ARG, "psy_math_check: unknown function %u", fn);
	if (n == 0) return PSY_OK;
	cudaSetDevice(ctx->device);
	float* d = nullptr;
	cudaError_t e = cudaMalloc(&d, sizeof(float) * 2 * (size_t)n);
	if (e != cudaSuccess) return ctx_cuda(ctx, e, "psy_math_check: device buffer");
	e = cudaMemcpy(d, x, sizeof(float) * n, cudaMemcpyHostToDevice);
	if (e == cudaSuccess) {
		const uint32_t blocks = (n + 255) / 256 < 4096u ? (n + 255) / 256 : 4096u;
		psy::libm_check_kernel<<<blocks, 256>>>(fn, n, d, d + n);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = cudaMemcpy(out, d + n, sizeof(float) * n, cudaMemcpyDeviceToHost);
	cudaFree(d);
	return ctx_cuda(ctx, e, "psy_math_check");
}
