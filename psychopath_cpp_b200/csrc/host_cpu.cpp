/*
 * Host-CPU properties the reference's arithmetic depends on.
 *
 * The reference inverts matrices with an SSE cofactor routine that
 * starts from the approximate reciprocal instruction and refines it with
 * one Newton step (utils/simd.hpp:110-205).  The instruction's result is
 * specified only to 1.5 * 2^-12 relative error; its exact bits come from a
 * table in the core and differ between CPU models.  For the identity
 * matrix, which is what Transform() holds when no instance transform
 * applies, the result is diag(k) with k = newton(rcp(1)) (0.99999994 on
 * current Intel cores); for any other matrix the reciprocal of its
 * determinant enters every element.  So the instruction is measured here,
 * on the host that also runs the reference, and the device looks its
 * results up (psy_math.h approx_rcp).
 */
#include "host_cpu.h"

#include <mutex>

#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#endif

namespace psy {

float reference_identity_inverse_scale() {
#if defined(__x86_64__) || defined(__i386__)
	const __m128 one = _mm_set_ss(1.0f);
	const __m128 r = _mm_rcp_ss(one);
	const __m128 k = _mm_sub_ss(_mm_add_ss(r, r), _mm_mul_ss(one, _mm_mul_ss(r, r)));
	float out;
	_mm_store_ss(&out, k);
	return out;
#else
	return 1.0f;
#endif
}

namespace {

uint32_t rcp_bits(uint32_t xb) {
#if defined(__x86_64__) || defined(__i386__)
	const __m128 r = _mm_rcp_ss(_mm_set_ss(u2f(xb)));
	return f2u(_mm_cvtss_f32(r));
#else
	return f2u(1.0f / u2f(xb));
#endif
}

// Fills the table at `shift` and checks it against the instruction for
// every mantissa at exponents from 2^-40 to 2^40 (both signs at 2^0).
bool build(int shift, std::vector<uint32_t>* out) {
	const uint32_t n = 1u << (23 - shift);
	out->assign(n, 0u);
	for (uint32_t k = 0; k < n; ++k) (*out)[k] = rcp_bits(0x3f800000u | (k << shift));
	const RcpTable t{out->data(), shift};
	for (uint32_t m = 0; m < (1u << 23); ++m) {
		const uint32_t xb = 0x3f800000u | m;
		if (f2u(approx_rcp(u2f(xb), t)) != rcp_bits(xb)) return false;
		if (f2u(approx_rcp(u2f(xb | 0x80000000u), t)) != rcp_bits(xb | 0x80000000u)) return false;
	}
	for (int e = -40; e <= 40; e += 8) {
		for (uint32_t m = 0; m < (1u << 23); m += 4093) {
			const uint32_t xb = ((uint32_t)(127 + e) << 23) | m;
			if (f2u(approx_rcp(u2f(xb), t)) != rcp_bits(xb)) return false;
		}
	}
	return true;
}

}  // namespace

const HostRcp& host_rcp() {
	static HostRcp h;
	static std::once_flag once;
	std::call_once(once, [] {
		if (!build(12, &h.entries)) {
			// the result depends on more mantissa bits on this core: tabulate all
			build(0, &h.entries);
			h.shift = 0;
		} else {
			h.shift = 12;
		}
	});
	return h;
}

}  // namespace psy
