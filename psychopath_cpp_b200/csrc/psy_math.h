/*
 * Float arithmetic of the hot path, host + device.
 *
 * Every operation keeps the reference's evaluation order so that the GPU
 * (compiled with -fmad=false, IEEE division and square root) reproduces
 * the reference's single-precision results bit for bit:
 *   - Vec3 follows Imath::Vec3<float> (dot = (x*x'+y*y')+z*z', length with
 *     the tiny-vector rescale, normalize divides by length);
 *   - Matrix44 follows reference math/matrix.hpp (row-vector convention,
 *     left-to-right sums, multVecMatrix divides by w);
 *   - min/max follow std::min/std::max ("first wins") or SSE minps/maxps
 *     ("a op b ? a : b") exactly where the reference uses each;
 *   - lerp(alpha, a, b) = a*(1-alpha) + b*alpha (reference utils/utils.hpp:53-56),
 *     lerp_seq as utils/utils.hpp:76-91.
 *   - Matrix44::inverse follows the reference's SSE cofactor routine
 *     (utils/simd.hpp:110-205, after Intel's application note AP-928,
 *     "Streaming SIMD Extensions - Inverse of 4x4 Matrix") lane for lane, and
 *     its approximate reciprocal of the determinant is the host CPU's own
 *     rcpss, tabulated on the host (host_cpu.cpp) and looked up here.
 */
#ifndef PSY_MATH_H
#define PSY_MATH_H

#include <cfloat>
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define PSY_HD __host__ __device__ __forceinline__
#else
#define PSY_HD inline
#endif

namespace psy {

static constexpr float BBOX_MAXT_ADJUST = 1.00000024f;  // reference basics/bbox.hpp:20

// std::min / std::max: the first argument is kept unless the second is strictly better.
PSY_HD float smin(float a, float b) { return (b < a) ? b : a; }
PSY_HD float smax(float a, float b) { return (a < b) ? b : a; }
// SSE minps / maxps and the reference's component-wise Vec3 min/max
// (math/vector.hpp:156-168): a op b ? a : b.
PSY_HD float vmin(float a, float b) { return (a < b) ? a : b; }
PSY_HD float vmax(float a, float b) { return (a > b) ? a : b; }
PSY_HD float fabs_(float a) { return fabsf(a); }

struct V3 {
	float x, y, z;
	PSY_HD V3() {}
	PSY_HD V3(float a, float b, float c): x(a), y(b), z(c) {}
	PSY_HD explicit V3(float a): x(a), y(a), z(a) {}
	PSY_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
	PSY_HD float& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

PSY_HD V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
PSY_HD V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
PSY_HD V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
PSY_HD V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
PSY_HD V3 operator*(float s, V3 a) { return V3(s * a.x, s * a.y, s * a.z); }
PSY_HD V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
PSY_HD V3 operator/(V3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
PSY_HD V3 operator/(V3 a, V3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }

PSY_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PSY_HD V3 cross(V3 a, V3 b) {
	return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PSY_HD float length2(V3 a) { return dot(a, a); }

// Imath::Vec3<float>::length() including its tiny-vector branch.
PSY_HD float length(V3 a) {
	const float l2 = dot(a, a);
	if (l2 < 2.0f * FLT_MIN) {
		float ax = fabsf(a.x), ay = fabsf(a.y), az = fabsf(a.z);
		float m = ax;
		if (m < ay) m = ay;
		if (m < az) m = az;
		if (m == 0.0f) return 0.0f;
		ax /= m;
		ay /= m;
		az /= m;
		return m * sqrtf(ax * ax + ay * ay + az * az);
	}
	return sqrtf(l2);
}

PSY_HD V3 normalized(V3 a) {
	const float l = length(a);
	if (l != 0.0f) return V3(a.x / l, a.y / l, a.z / l);
	return a;
}

// Component-wise min/max of reference math/vector.hpp:156-168.
PSY_HD V3 vmin3(V3 a, V3 b) { return V3(vmin(a.x, b.x), vmin(a.y, b.y), vmin(a.z, b.z)); }
PSY_HD V3 vmax3(V3 a, V3 b) { return V3(vmax(a.x, b.x), vmax(a.y, b.y), vmax(a.z, b.z)); }

// longest_axis (reference math/vector.hpp:170-172)
PSY_HD float longest_axis(V3 v) { return smax(smax(fabsf(v.x), fabsf(v.y)), fabsf(v.z)); }

// lerp for struct types: the (1.0 - alpha) double is narrowed to float
// before the multiply, which equals the float subtraction for alpha in [0,1].
PSY_HD float one_minus(float alpha) { return 1.0f - alpha; }
PSY_HD V3 lerp3(float alpha, V3 a, V3 b) {
	const float ia = one_minus(alpha);
	return (a * ia) + (b * alpha);
}
// lerp<float>: a * (1.0 - alpha) in double, plus the float product b*alpha,
// summed in double and narrowed (reference utils/utils.hpp:53-56 with T=float).
PSY_HD float lerp1(float alpha, float a, float b) {
	const double t = (double)a * (1.0 - (double)alpha);
	const float u = b * alpha;
	return (float)(t + (double)u);
}

// lerp_seq index selection (reference utils/utils.hpp:76-91). Returns the
// first index and the local alpha; count==1 or alpha>=1 select one sample.
struct SeqPos {
	int i0;
	int single;  // 1 when a single element is returned (no interpolation)
	float nalpha;
};
PSY_HD SeqPos seq_pos(float alpha, int count) {
	SeqPos p;
	if (count <= 1) {
		p.i0 = 0; p.single = 1; p.nalpha = 0.0f;
	} else if (alpha >= 1.0f) {
		p.i0 = count - 1; p.single = 1; p.nalpha = 0.0f;
	} else {
		const float temp = alpha * (float)(count - 1);
		const int index = (int)temp;
		p.i0 = index; p.single = 0; p.nalpha = temp - (float)index;
	}
	return p;
}

// ---------------------------------------------------------------------
// 4x4 matrices (row-major, row-vector convention)
// ---------------------------------------------------------------------
struct M44 {
	float m[4][4];
};

PSY_HD M44 m44_identity() {
	M44 r;
	for (int i = 0; i < 4; ++i)
		for (int j = 0; j < 4; ++j) r.m[i][j] = (i == j) ? 1.0f : 0.0f;
	return r;
}

PSY_HD M44 m44_nan() {
	M44 r;
	for (int i = 0; i < 4; ++i)
		for (int j = 0; j < 4; ++j) r.m[i][j] = NAN;
	return r;
}

// Matrix44::operator* (reference math/matrix.hpp:148-155): r = this * b.
PSY_HD M44 m44_mul(const M44& a, const M44& b) {
	M44 r;
	for (int i = 0; i < 4; ++i)
		for (int j = 0; j < 4; ++j)
			r.m[i][j] = (((b.m[0][j] * a.m[i][0]) + (b.m[1][j] * a.m[i][1])) + (b.m[2][j] * a.m[i][2])) +
			            (b.m[3][j] * a.m[i][3]);
	return r;
}

PSY_HD M44 m44_lerp(float alpha, const M44& a, const M44& b) {
	const float ia = one_minus(alpha);
	M44 r;
	for (int i = 0; i < 4; ++i)
		for (int j = 0; j < 4; ++j) r.m[i][j] = (a.m[i][j] * ia) + (b.m[i][j] * alpha);
	return r;
}

// multVecMatrix: r = row0*x + row1*y + row2*z + row3, divided by r.w.
PSY_HD V3 pos_to(const M44& t, V3 v) {
	float r[4];
	for (int j = 0; j < 4; ++j)
		r[j] = (((t.m[0][j] * v.x) + (t.m[1][j] * v.y)) + (t.m[2][j] * v.z)) + t.m[3][j];
	return V3(r[0] / r[3], r[1] / r[3], r[2] / r[3]);
}

// multDirMatrix.
PSY_HD V3 dir_to(const M44& t, V3 v) {
	float r[3];
	for (int j = 0; j < 3; ++j) r[j] = ((t.m[0][j] * v.x) + (t.m[1][j] * v.y)) + (t.m[2][j] * v.z);
	return V3(r[0], r[1], r[2]);
}

// dir_transform_transpose (reference math/matrix.hpp:418-421): each row
// dotted with (x, y, z, 0) and reduced as SSE hadd pairs.
PSY_HD V3 dir_transpose(const M44& t, V3 v) {
	float r[3];
	for (int i = 0; i < 3; ++i) {
		const float p0 = t.m[i][0] * v.x, p1 = t.m[i][1] * v.y, p2 = t.m[i][2] * v.z, p3 = t.m[i][3] * 0.0f;
		r[i] = (p0 + p1) + (p2 + p3);
	}
	return V3(r[0], r[1], r[2]);
}

// The host CPU's approximate reciprocal instruction (rcpss) as a table.
// On the x86 cores measured so far its result for a normal input x =
// m * 2^e depends only on the leading bits of the mantissa m and scales
// exactly with 2^-e, so `bits[k]` holds the result bits for the input
// 1 + k / 2^(23 - shift) (shift = 12: 2048 entries); host_cpu.cpp verifies
// that against the instruction for every mantissa and falls back to the
// full table (shift 0) on a core where it does not hold.
struct RcpTable {
	const uint32_t* bits;
	int shift;
};

PSY_HD uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
	return __float_as_uint(f);
#else
	uint32_t u;
	__builtin_memcpy(&u, &f, 4);
	return u;
#endif
}
PSY_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
	return __uint_as_float(u);
#else
	float f;
	__builtin_memcpy(&f, &u, 4);
	return f;
#endif
}

// rcpss of x: denormal inputs count as zero (signed infinity), infinities
// give signed zero, NaN stays NaN, and results below the normal range
// flush to signed zero, as the instruction does.
PSY_HD float approx_rcp(float x, const RcpTable& t) {
	const uint32_t b = f2u(x);
	const uint32_t sign = b & 0x80000000u;
	const int e = (int)((b >> 23) & 0xffu);
	const uint32_t m = b & 0x7fffffu;
	if (e == 0) return u2f(sign | 0x7f800000u);
	if (e == 255) return m ? u2f(b | 0x400000u) : u2f(sign);
	const uint32_t r = t.bits[m >> t.shift];
	const int re = (int)((r >> 23) & 0xffu) - (e - 127);
	if (re <= 0) return u2f(sign);
	return u2f(sign | ((uint32_t)re << 23) | (r & 0x7fffffu));
}

// Four SSE lanes and the shuffles the inverse uses (_mm_shuffle_ps(a, b,
// imm): lanes 0, 1 from a, lanes 2, 3 from b, two bits of imm each).
struct L4 {
	float v[4];
};
PSY_HD L4 l4(float a, float b, float c, float d) {
	L4 r;
	r.v[0] = a; r.v[1] = b; r.v[2] = c; r.v[3] = d;
	return r;
}
PSY_HD L4 operator*(const L4& a, const L4& b) { return l4(a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]); }
PSY_HD L4 operator+(const L4& a, const L4& b) { return l4(a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]); }
PSY_HD L4 operator-(const L4& a, const L4& b) { return l4(a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2], a.v[3] - b.v[3]); }
template <int IMM>
PSY_HD L4 shuf(const L4& a, const L4& b) {
	return l4(a.v[IMM & 3], a.v[(IMM >> 2) & 3], b.v[(IMM >> 4) & 3], b.v[(IMM >> 6) & 3]);
}

// Matrix44::inverse (reference math/matrix.hpp:319-329 over
// utils/simd.hpp:110-205): the cofactors of the transposed rows in the
// routine's lane order, the determinant summed as its shuffles pair the
// lanes, its reciprocal from rcpss refined by one Newton step, every
// cofactor times that.  A singular matrix comes out all NaN, as there.
PSY_HD M44 m44_inverse(const M44& a, const RcpTable& rt) {
	const float* s = &a.m[0][0];
	L4 row0 = l4(s[0], s[4], s[8], s[12]);
	L4 row1 = l4(s[9], s[13], s[1], s[5]);
	L4 row2 = l4(s[2], s[6], s[10], s[14]);
	L4 row3 = l4(s[11], s[15], s[3], s[7]);
	L4 tmp1, minor0, minor1, minor2, minor3;
	tmp1 = row2 * row3;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	minor0 = row1 * tmp1;
	minor1 = row0 * tmp1;
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor0 = (row1 * tmp1) - minor0;
	minor1 = (row0 * tmp1) - minor1;
	minor1 = shuf<0x4E>(minor1, minor1);

	tmp1 = row1 * row2;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	minor0 = (row3 * tmp1) + minor0;
	minor3 = row0 * tmp1;
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor0 = minor0 - (row3 * tmp1);
	minor3 = (row0 * tmp1) - minor3;
	minor3 = shuf<0x4E>(minor3, minor3);

	tmp1 = shuf<0x4E>(row1, row1) * row3;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	row2 = shuf<0x4E>(row2, row2);
	minor0 = (row2 * tmp1) + minor0;
	minor2 = row0 * tmp1;
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor0 = minor0 - (row2 * tmp1);
	minor2 = (row0 * tmp1) - minor2;
	minor2 = shuf<0x4E>(minor2, minor2);

	tmp1 = row0 * row1;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	minor2 = (row3 * tmp1) + minor2;
	minor3 = (row2 * tmp1) - minor3;
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor2 = (row3 * tmp1) - minor2;
	minor3 = minor3 - (row2 * tmp1);

	tmp1 = row0 * row3;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	minor1 = minor1 - (row2 * tmp1);
	minor2 = (row1 * tmp1) + minor2;
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor1 = (row2 * tmp1) + minor1;
	minor2 = minor2 - (row1 * tmp1);

	tmp1 = row0 * row2;
	tmp1 = shuf<0xB1>(tmp1, tmp1);
	minor1 = (row3 * tmp1) + minor1;
	minor3 = minor3 - (row1 * tmp1);
	tmp1 = shuf<0x4E>(tmp1, tmp1);
	minor1 = minor1 - (row3 * tmp1);
	minor3 = (row1 * tmp1) + minor3;

	L4 det = row0 * minor0;
	det = shuf<0x4E>(det, det) + det;
	const float d = det.v[1] + det.v[0];
	const float r = approx_rcp(d, rt);
	const float k = (r + r) - (d * (r * r));
	M44 out;
	const L4* mi[4] = {&minor0, &minor1, &minor2, &minor3};
	for (int i = 0; i < 4; ++i)
		for (int j = 0; j < 4; ++j) out.m[i][j] = k * mi[i]->v[j];
	if (k == 0.0f) return m44_nan();
	return out;
}

PSY_HD V3 pos_from(const M44& t, V3 v, const RcpTable& rt) { return pos_to(m44_inverse(t, rt), v); }
PSY_HD V3 dir_from(const M44& t, V3 v, const RcpTable& rt) { return dir_to(m44_inverse(t, rt), v); }
PSY_HD V3 nor_to(const M44& t, V3 v, const RcpTable& rt) { return dir_transpose(m44_inverse(t, rt), v); }
PSY_HD V3 nor_from(const M44& t, V3 v) { return dir_transpose(t, v); }

// Transform::get_inv_scale (reference math/transform.hpp:108-114).
PSY_HD V3 inv_scale(const M44& t) {
	V3 s;
	s.x = sqrtf(((t.m[0][0] * t.m[0][0]) + (t.m[0][1] * t.m[0][1])) + (t.m[0][2] * t.m[0][2]));
	s.y = sqrtf(((t.m[1][0] * t.m[1][0]) + (t.m[1][1] * t.m[1][1])) + (t.m[1][2] * t.m[1][2]));
	s.z = sqrtf(((t.m[2][0] * t.m[2][0]) + (t.m[2][1] * t.m[2][1])) + (t.m[2][2] * t.m[2][2]));
	return s;
}

// ---------------------------------------------------------------------
// Axis-aligned boxes
// ---------------------------------------------------------------------
struct Box {
	V3 lo, hi;
};

PSY_HD Box box_empty() {
	Box b;
	b.lo = V3(INFINITY);
	b.hi = V3(-INFINITY);
	return b;
}

PSY_HD Box box_lerp(float alpha, const Box& a, const Box& b) {
	Box r;
	r.lo = lerp3(alpha, a.lo, b.lo);
	r.hi = lerp3(alpha, a.hi, b.hi);
	return r;
}

// BBox::operator| / merge_with (basics/bbox.hpp:80-119): a[i] < b[i] ? a : b.
PSY_HD Box box_union(const Box& a, const Box& b) {
	Box r;
	r.lo = V3(a.lo.x < b.lo.x ? a.lo.x : b.lo.x, a.lo.y < b.lo.y ? a.lo.y : b.lo.y,
	          a.lo.z < b.lo.z ? a.lo.z : b.lo.z);
	r.hi = V3(a.hi.x > b.hi.x ? a.hi.x : b.hi.x, a.hi.y > b.hi.y ? a.hi.y : b.hi.y,
	          a.hi.z > b.hi.z ? a.hi.z : b.hi.z);
	return r;
}

PSY_HD V3 box_center(const Box& b) { return (b.lo + b.hi) * 0.5f; }

PSY_HD float box_diagonal(const Box& b) { return length(b.hi - b.lo); }

// BBox::intersect_ray (basics/bbox.hpp:138-177), scalar slab test with the
// std::min/std::max semantics of the reference.
PSY_HD bool box_hit(const Box& b, V3 o, V3 dinv, float tmax, float* t0, float* t1) {
	const float tx1 = (b.lo.x - o.x) * dinv.x;
	const float tx2 = (b.hi.x - o.x) * dinv.x;
	float h0 = smin(tx1, tx2);
	float h1 = smax(tx1, tx2);
	const float ty1 = (b.lo.y - o.y) * dinv.y;
	const float ty2 = (b.hi.y - o.y) * dinv.y;
	h0 = smax(h0, smin(ty1, ty2));
	h1 = smin(h1, smax(ty1, ty2));
	const float tz1 = (b.lo.z - o.z) * dinv.z;
	const float tz2 = (b.hi.z - o.z) * dinv.z;
	h0 = smax(0.0f, smax(h0, smin(tz1, tz2)));
	h1 = smin(h1, smax(tz1, tz2)) * BBOX_MAXT_ADJUST;
	*t0 = h0;
	*t1 = h1;
	return h0 <= smin(tmax, h1);
}

// Box corners transformed with pos_to of the inverse (BBox::inverse_transformed,
// basics/bbox.hpp:227-258).
PSY_HD Box box_inverse_transformed(const Box& b, const M44& t, const RcpTable& rt) {
	const M44 inv = m44_inverse(t, rt);
	Box r = box_empty();
	for (int c = 0; c < 8; ++c) {
		const V3 v((c & 4) ? b.hi.x : b.lo.x, (c & 2) ? b.hi.y : b.lo.y, (c & 1) ? b.hi.z : b.lo.z);
		const V3 p = pos_to(inv, v);
		for (int i = 0; i < 3; ++i) {
			const float pi = p[i];
			float& lo = r.lo.at(i);
			float& hi = r.hi.at(i);
			lo = pi < lo ? pi : lo;
			hi = pi > hi ? pi : hi;
		}
	}
	return r;
}

// ---------------------------------------------------------------------
// Ray widths (basics/ray.hpp:118-153, 207-252; utils/utils.hpp:443-456)
// ---------------------------------------------------------------------
PSY_HD void closest_ray_t2(V3 o1, V3 d1, V3 o2, V3 d2, float* t_out, float* dist_out) {
	const V3 dd = d1 - d2;
	const float dd2 = dot(dd, dd);
	if (dd2 < 0.00001f) {
		*t_out = -1.0f;
		*dist_out = -1.0f;
		return;
	}
	const V3 w = o1 - o2;
	const float t = -dot(w, dd) / dd2;
	*t_out = t;
	*dist_out = length((o1 + (d1 * t)) - (o2 + (d2 * t)));
}

struct RayWidth {
	float owx, owy, dwx, dwy, fwx, fwy;
};

// Width parameters of a ray with origin o, direction d and the (already
// transformed) differentials.
PSY_HD RayWidth ray_width_params(V3 o, V3 d, V3 odx, V3 ody, V3 ddx, V3 ddy) {
	RayWidth w;
	float tdx, lx, tdy, ly;
	closest_ray_t2(o, d, o + odx, d + ddx, &tdx, &lx);
	closest_ray_t2(o, d, o + ody, d + ddy, &tdy, &ly);
	w.owx = length(odx);
	if (tdx <= 0.0f) {
		w.dwx = length(ddx);
		w.fwx = 0.0f;
	} else {
		w.dwx = (lx - w.owx) / tdx;
		w.fwx = lx;
	}
	w.owy = length(ody);
	if (tdy <= 0.0f) {
		w.dwy = length(ddy);
		w.fwy = 0.0f;
	} else {
		w.dwy = (ly - w.owy) / tdy;
		w.fwy = ly;
	}
	return w;
}

// Ray::min_width (basics/ray.hpp:132-153).
PSY_HD float ray_min_width(const RayWidth& w, float tnear, float tfar) {
	const float tflipx = (w.owx - w.fwx) / w.dwx;
	const float tflipy = (w.owy - w.fwy) / w.dwy;
	float minx, miny;
	if (tnear < tflipx && tfar > tflipx) {
		minx = w.fwx;
	} else {
		minx = smin(fabsf((w.owx - w.fwx) + (w.dwx * tnear)) + w.fwx, fabsf((w.owx - w.fwx) + (w.dwx * tfar)) + w.fwx);
	}
	if (tnear < tflipy && tfar > tflipy) {
		miny = w.fwy;
	} else {
		miny = smin(fabsf((w.owy - w.fwy) + (w.dwy * tnear)) + w.fwy, fabsf((w.owy - w.fwy) + (w.dwy * tfar)) + w.fwy);
	}
	return smin(minx, miny);
}

PSY_HD V3 recip3(V3 d) { return V3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z); }

// InstanceID::push_back bit mask (basics/instance_id.hpp:18-23): the mask
// is computed in int, so widths of 31+ bits follow the int arithmetic.
PSY_HD uint64_t id_push(uint64_t id, uint64_t sub, int bits) {
	id <<= bits;
	id |= sub & (uint64_t)(int64_t)((1 << bits) - 1);
	return id;
}

// intlog2(upper_power_of_two(n)) (reference utils/utils.hpp:254-287).
PSY_HD uint32_t upper_power_of_two(uint32_t v) {
	v--;
	v |= v >> 1;
	v |= v >> 2;
	v |= v >> 4;
	v |= v >> 8;
	v |= v >> 16;
	v++;
	return v;
}
PSY_HD uint32_t intlog2(uint32_t v) {
	uint32_t r, shift;
	r = (v > 0xFFFF) << 4;
	v >>= r;
	shift = (v > 0xFF) << 3;
	v >>= shift;
	r |= shift;
	shift = (v > 0xF) << 2;
	v >>= shift;
	r |= shift;
	shift = (v > 0x3) << 1;
	v >>= shift;
	r |= shift;
	r |= (v >> 1);
	return r;
}

}  // namespace psy

#endif
