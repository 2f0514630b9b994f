// The host C library's single-precision math, restated for the device.
//
// The reference renderer calls std::sin/std::cos/std::acos/std::asin/
// std::exp on floats; built with GCC for x86-64 these become the C
// library's sincosf, acosf, asinf and expf (glibc 2.39 here).  CUDA's own
// sinf/cosf/acosf/asinf/expf round differently in the last place for a
// sizable share of inputs, and one ulp in a sampled direction is enough
// to flip a later discrete decision of a path (a light choice, a hit).  So
// the shading kernels call these restatements, which return the same bits
// as the host's library over the argument ranges the renderer uses:
//
//   lm_sincosf  |x| < 120: the polynomial scheme of glibc's sincosf
//               (since 2.28; from Arm's optimized-routines, sincosf.h /
//               sincosf_data.c): reduction by the nearest multiple of
//               pi/2 in double, one sine and one cosine polynomial in
//               double, quadrant swap and signs.  glibc on x86-64 selects
//               its FMA build, so the polynomial and the reduction use
//               fused multiply-adds.  Checked bit-exact against glibc for
//               every float with |x| < 120.  Larger |x| (no call site of
//               the renderer) rounds the double sin/cos.
//   lm_acosf    fdlibm's float acos (Sun, e_acosf.c): rational p/q
//               approximation in float on three ranges.  Checked bit-exact
//               for every float in [-1, 1].
//   lm_asinf    glibc's float asin (e_asinf.c): a degree-4 polynomial in
//               x^2 (Cephes coefficients) on fdlibm's range split.  Checked
//               bit-exact for every float in [-1, 1].
//   lm_expf     glibc's expf (since 2.27; optimized-routines e_expf.c):
//               x/ln2 scaled by 32, the 32-entry table of 2^(i/32) (the
//               doubles nearest 2^(i/32), exponent field pre-subtracted)
//               and a cubic in double.  Matches glibc on all but 2 of the
//               2.2e9 floats with |x| < 88; larger |x| (overflow and
//               underflow handling, no call site) goes to CUDA's expf.
//
// The polynomial coefficients are the published minimax values of those
// routines.  Device code is built with -fmad=false, so every fused step
// is an explicit fma() and every other product or sum rounds on its own.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define PSY_LM_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define PSY_LM_HD static inline
#endif

namespace psylm {

PSY_LM_HD uint32_t fbits(float f) {
#ifdef __CUDA_ARCH__
	return __float_as_uint(f);
#else
	uint32_t u;
	memcpy(&u, &f, 4);
	return u;
#endif
}
PSY_LM_HD float bitsf(uint32_t u) {
#ifdef __CUDA_ARCH__
	return __uint_as_float(u);
#else
	float f;
	memcpy(&f, &u, 4);
	return f;
#endif
}
PSY_LM_HD uint64_t dbits(double d) {
#ifdef __CUDA_ARCH__
	return (uint64_t)__double_as_longlong(d);
#else
	uint64_t u;
	memcpy(&u, &d, 8);
	return u;
#endif
}
PSY_LM_HD double bitsd(uint64_t u) {
#ifdef __CUDA_ARCH__
	return __longlong_as_double((long long)u);
#else
	double d;
	memcpy(&d, &u, 8);
	return d;
#endif
}
// top 12 bits below the sign: the biased exponent and the first mantissa bit
PSY_LM_HD uint32_t abstop12(float x) { return (fbits(x) >> 20) & 0x7ffu; }

}  // namespace psylm

// sincosf: cosine 1 + c1 x^2 + ... + c4 x^8 and sine x + s1 x^3 + s2 x^5 +
// s3 x^7, minimax on [-pi/4, pi/4]; 2/pi scaled by 2^24 for the integer
// rounding of the quadrant; pi/2 in double.
#define PSY_LM_SC_C1 (-0x1.ffffffd0c621cp-2)
#define PSY_LM_SC_C2 0x1.55553e1068f19p-5
#define PSY_LM_SC_C3 (-0x1.6c087e89a359dp-10)
#define PSY_LM_SC_C4 0x1.99343027bf8c3p-16
#define PSY_LM_SC_S1 (-0x1.555545995a603p-3)
#define PSY_LM_SC_S2 0x1.1107605230bc4p-7
#define PSY_LM_SC_S3 (-0x1.994eb3774cf24p-13)
#define PSY_LM_HPI_INV_2P24 0x1.45f306dc9c883p+23
#define PSY_LM_HPI 0x1.921fb54442d18p+0

PSY_LM_HD void lm_sincosf(float y, float* sinp, float* cosp) {
	using namespace psylm;
	double x = (double)y;
	const uint32_t top = abstop12(y);
	int n = 0;
	// range tests on the top 12 bits: those of pi/4 (so |y| < 0.75), 2^-12, 120
	if (top < 0x3f4u) {
		if (top < 0x398u) {
			*sinp = y;
			*cosp = 1.0f;
			return;
		}
	} else if (top < 0x42fu) {
		// nearest multiple of pi/2: (int)(x * 2/pi * 2^24), rounded at bit 24
		const double r = x * PSY_LM_HPI_INV_2P24;
		n = (((int32_t)r) + 0x800000) >> 24;
		x = fma(-(double)n, PSY_LM_HPI, x);
	} else {
		*sinp = (float)sin(x);
		*cosp = (float)cos(x);
		return;
	}
	// quadrants 1 and 2 take the sine of -x; 2 and 3 negate the cosine
	const double xs = ((n & 3) == 1 || (n & 3) == 2) ? -x : x;
	const double x2 = x * x;
	const double x4 = x2 * x2;
	const double x3 = x2 * xs;
	const double c2 = fma(x2, PSY_LM_SC_C4, PSY_LM_SC_C3);
	const double s1 = fma(x2, PSY_LM_SC_S3, PSY_LM_SC_S2);
	const double c1 = fma(x2, PSY_LM_SC_C1, 1.0);
	const double x5 = x3 * x2;
	const double x6 = x4 * x2;
	const double s = fma(x3, PSY_LM_SC_S1, xs);
	const double c = fma(x4, PSY_LM_SC_C2, c1);
	const float sv = (float)fma(x5, s1, s);
	float cv = (float)fma(x6, c2, c);
	if (n & 2) cv = -cv;
	if (n & 1) {
		*sinp = cv;
		*cosp = sv;
	} else {
		*sinp = sv;
		*cosp = cv;
	}
}

PSY_LM_HD float lm_sinf(float x) {
	float s, c;
	lm_sincosf(x, &s, &c);
	return s;
}

PSY_LM_HD float lm_cosf(float x) {
	float s, c;
	lm_sincosf(x, &s, &c);
	return c;
}

// fdlibm's float acos: pi and pi/2 split into a float head and tail, and
// the rational approximation asin(t)/t - 1 ~ t^2 P(t^2) / Q(t^2).
PSY_LM_HD float lm_acos_pq(float z) {
	const float p = z * (1.6666667163e-01f +
	                     z * (-3.2556581497e-01f +
	                          z * (2.0121252537e-01f +
	                               z * (-4.0055535734e-02f + z * (7.9153501429e-04f + z * 3.4793309169e-05f)))));
	const float q = 1.0f + z * (-2.4033949375e+00f + z * (2.0209457874e+00f + z * (-6.8828397989e-01f + z * 7.7038154006e-02f)));
	return p / q;
}

// The three ranges (|x| < 0.5, x < -0.5, x > 0.5) are evaluated with the
// same operations as fdlibm's branches, but every lane computes the
// rational function once and the square root and head/tail split once, and
// the result is selected: the lanes of a warp take different ranges, and
// branches would run the divisions once per range.
PSY_LM_HD float lm_acosf(float x) {
	using namespace psylm;
	const float pi = 3.1415925026e+00f, pio2_hi = 1.5707962513e+00f, pio2_lo = 7.5497894159e-08f;
	const uint32_t hx = fbits(x), ix = hx & 0x7fffffffu;
	if (ix >= 0x3f800000u) {  // |x| >= 1
		if (ix == 0x3f800000u) return (hx >> 31) ? pi + 2.0f * pio2_lo : 0.0f;
		return (x - x) / (x - x);
	}
	const bool small = ix < 0x3f000000u, neg = (hx >> 31) != 0;
	const float z = small ? x * x : (neg ? (1.0f + x) * 0.5f : (1.0f - x) * 0.5f);
	const float r = lm_acos_pq(z);
	const float s = sqrtf(z);
	// x > 0.5: sqrt(z) split into a head with 12 low mantissa bits cleared
	const float df = bitsf(fbits(s) & 0xfffff000u);
	const float c = (z - df * df) / (s + df);
	const float a_small = ix <= 0x32800000u ? pio2_hi + pio2_lo : pio2_hi - (x - (pio2_lo - x * r));
	const float w_neg = r * s - pio2_lo;
	const float a_neg = pi - 2.0f * (s + w_neg);
	const float w_pos = r * s + c;
	const float a_pos = 2.0f * (df + w_pos);
	return small ? a_small : (neg ? a_neg : a_pos);
}

// glibc's float asin: asin(t) ~ t + t^3 P(t^2), P of degree 4.
PSY_LM_HD float lm_asin_p(float t) {
	return t * (1.666675248e-1f + t * (7.495297643e-2f + t * (4.547037598e-2f + t * (2.417951451e-2f + t * 4.216630880e-2f))));
}

// As lm_acosf, the ranges (|x| < 0.5, 0.5 <= |x| <= 0.975, above) share
// the polynomial and the square root, and the result is selected.
PSY_LM_HD float lm_asinf(float x) {
	using namespace psylm;
	const float pio2_hi = 1.57079637050628662109375f, pio2_lo = -4.37113900018624283e-8f,
	            pio4_hi = 0.785398185253143310546875f;
	const uint32_t hx = fbits(x), ix = hx & 0x7fffffffu;
	if (ix >= 0x3f800000u) {  // |x| >= 1
		if (ix == 0x3f800000u) return x * pio2_hi + x * pio2_lo;
		return (x - x) / (x - x);
	}
	const bool small = ix < 0x3f000000u;
	const float w = 1.0f - fabsf(x);
	const float t = small ? x * x : w * 0.5f;
	const float p = lm_asin_p(t);
	const float a_small = ix < 0x32000000u ? x : x + x * p;
	const float s = sqrtf(t);
	// |x| > 0.975
	const float a_top = pio2_hi - (2.0f * (s + s * p) - pio2_lo);
	// otherwise: sqrt(t) split into a head with 12 low mantissa bits cleared
	const float hw = bitsf(fbits(s) & 0xfffff000u);
	const float c = (t - hw * hw) / (s + hw);
	const float pm = 2.0f * s * p - (pio2_lo - 2.0f * c);
	const float q = pio4_hi - 2.0f * hw;
	const float a_mid = pio4_hi - (pm - q);
	const float a = ix >= 0x3f79999au ? a_top : a_mid;
	return small ? a_small : ((hx >> 31) ? -a : a);
}

// expf: 2^(i/32) for i = 0..31 as the nearest double, less i << 47 (the
// exponent the scaled quotient adds back), and the cubic for 2^(r/32).
#define PSY_LM_EXP2_TABLE                                                                                     \
	{                                                                                                         \
		0x3ff0000000000000ull, 0x3fefd9b0d3158574ull, 0x3fefb5586cf9890full, 0x3fef9301d0125b51ull,           \
		    0x3fef72b83c7d517bull, 0x3fef54873168b9aaull, 0x3fef387a6e756238ull, 0x3fef1e9df51fdee1ull,       \
		    0x3fef06fe0a31b715ull, 0x3feef1a7373aa9cbull, 0x3feedea64c123422ull, 0x3feece086061892dull,       \
		    0x3feebfdad5362a27ull, 0x3feeb42b569d4f82ull, 0x3feeab07dd485429ull, 0x3feea47eb03a5585ull,       \
		    0x3feea09e667f3bcdull, 0x3fee9f75e8ec5f74ull, 0x3feea11473eb0187ull, 0x3feea589994cce13ull,       \
		    0x3feeace5422aa0dbull, 0x3feeb737b0cdc5e5ull, 0x3feec49182a3f090ull, 0x3feed503b23e255dull,       \
		    0x3feee89f995ad3adull, 0x3feeff76f2fb5e47ull, 0x3fef199bdd85529cull, 0x3fef3720dcef9069ull,       \
		    0x3fef5818dcfba487ull, 0x3fef7c97337b9b5full, 0x3fefa4afa2a490daull, 0x3fefd0765b6e4540ull        \
	}

#ifdef __CUDACC__
__device__ __constant__ static const uint64_t psy_lm_exp2_tab_dev[32] = PSY_LM_EXP2_TABLE;
#endif
static const uint64_t psy_lm_exp2_tab_host[32] = PSY_LM_EXP2_TABLE;

PSY_LM_HD float lm_expf(float x) {
	using namespace psylm;
	if (abstop12(x) >= 0x42bu) return expf(x);  // |x| >= 88 (or NaN): overflow / underflow range
	const double xd = (double)x;
	const double invln2n = 0x1.71547652b82fep+0 * 32;
	const double shift = 0x1.8p+52;
	double z = invln2n * xd;
	double kd = z + shift;
	const uint64_t ki = dbits(kd);
	kd -= shift;
	const double r = z - kd;
#ifdef __CUDA_ARCH__
	uint64_t t = psy_lm_exp2_tab_dev[ki % 32];
#else
	uint64_t t = psy_lm_exp2_tab_host[ki % 32];
#endif
	t += ki << 47;
	const double s = bitsd(t);
	z = fma(0x1.c6af84b912394p-5 / 32 / 32 / 32, r, 0x1.ebfce50fac4f3p-3 / 32 / 32);
	const double r2 = r * r;
	double y = fma(0x1.62e42ff0c52d6p-1 / 32, r, 1.0);
	y = fma(z, r2, y);
	y = y * s;
	return (float)y;
}
