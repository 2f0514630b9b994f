/*
 * Host-CPU properties the reference's arithmetic depends on.
 *
 * The reference inverts matrices with an SSE cofactor routine that
 * starts from the approximate reciprocal instruction and refines it with
 * one Newton step (utils/simd.hpp:110-205).  For the identity matrix, which
 * is what Transform() holds when no instance transform applies, the result
 * is diag(k) with k = newton(rcp(1)), a value that depends on the CPU's
 * reciprocal table (0.99999994 on current Intel cores).  The reference then
 * uses that matrix for every world-space hit position, offset and light
 * direction of untransformed geometry, so the same k is measured here, on
 * the host that also runs the reference, and used on the device.
 */
#include "host_cpu.h"

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

}  // namespace psy
