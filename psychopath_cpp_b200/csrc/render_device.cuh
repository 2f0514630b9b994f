/*
 * Device functions of the path-tracing integrator.  Each restates a
 * reference routine with its evaluation order and precision (float, or
 * double where the reference computes in double):
 *   Sampler / Halton           sampling/image_sampler.hpp:16-38, sampling/halton.cpp, utils/hash.hpp:6-16
 *   fast_logit, square_to_circle, cosine_sample_hemisphere, uniform cone /
 *   sphere sampling, sphere_lambert           utils/monte_carlo.hpp, utils/utils.hpp:214-343
 *   spectral upsampling and CIE curves        color/color.hpp:15-188,490-511, color/spectrum_grid.h:21-135
 *   Camera::generate_ray                      basics/camera.hpp:72-104
 *   LightTree::sample / node_prob             accel/light_tree.cpp:6-96
 *   SphereLight::sample                       lights/sphere_light.hpp:58-122
 *   LambertClosure                            shading/surface_closure.hpp:233-331
 *   transfer_ray_origin_differential          basics/differential_geometry.hpp:85-98
 */
#ifndef PSY_RENDER_DEVICE_CUH
#define PSY_RENDER_DEVICE_CUH

#include "kernels.h"
#include "shade_geom.cuh"
#include "psy_libm.cuh"

#define PSY_SPEC_QUAL __device__
#include "spectral_table.inc"

namespace psy {

#define PSY_HPI_D (PSY_PI_D / 2.0)
#define PSY_QPI_D (PSY_PI_D / 4.0)
#define PSY_INV_PI_D (1.0 / PSY_PI_D)

static constexpr float WAVELENGTH_MIN = 380.0f;
static constexpr float WAVELENGTH_MAX = 700.0f;
static constexpr float WAVELENGTH_RANGE = WAVELENGTH_MAX - WAVELENGTH_MIN;
static constexpr float INV_XYZ_INTEGRAL = 0.009358239977091027f;
static constexpr float XYZ_NORM_FAC = INV_XYZ_INTEGRAL * (WAVELENGTH_MAX - WAVELENGTH_MIN);

// ---------------------------------------------------------------------
// Sampler
// ---------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash_u32(uint32_t n, uint32_t seed) {
	uint32_t h = n;
#pragma unroll
	for (int i = 0; i < 3; ++i) {
		h *= 1936502639u;
		h ^= h >> 16;
		h += seed;
	}
	return h;
}

__device__ __forceinline__ float halton_sample(const HaltonDev& hd, uint32_t dim, uint32_t index) {
	if (dim == 0) {
		const uint32_t r = __brev(index);
		return __uint2float_rn(r) * (1.0f / 4294967296.0f);
	}
	const uint4 d = __ldg(hd.dims + dim);
	const uint32_t pb = d.y;
	uint32_t q = index;
	uint32_t sum = 0;
	uint32_t mult = 1;
	for (uint32_t g = 1; g < d.z; ++g) mult *= pb;
	for (uint32_t g = 0; g < d.z; ++g) {
		sum += (uint32_t)__ldg(hd.perm + d.w + q % pb) * mult;
		q /= pb;
		mult /= pb;
	}
	return (float)((double)sum * __ldg(hd.cmul + dim));
}

// Sampler::get_sample with the reordered first 11 dimensions.
__device__ __forceinline__ float sampler_get(const HaltonDev& hd, uint32_t offset, uint32_t dimension) {
	uint32_t d;
	switch (dimension) {
		case 0: d = 10; break;
		case 1: d = 7; break;
		case 2: d = 6; break;
		case 3: d = 5; break;
		case 4: d = 4; break;
		case 5: d = 2; break;
		case 6: d = 9; break;
		case 7: d = 8; break;
		case 8: d = 3; break;
		case 9: d = 1; break;
		case 10: d = 0; break;
		default: d = dimension; break;
	}
	return halton_sample(hd, d, offset);
}

__device__ __forceinline__ uint32_t sampler_offset(uint32_t x, uint32_t y, uint32_t n, uint32_t seed) {
	return hash_u32(x ^ ((y >> 16) | (y << 16)), seed) + n;
}

// ---------------------------------------------------------------------
// Monte Carlo helpers
// ---------------------------------------------------------------------
__device__ __forceinline__ float faster_ln(float x) {
	float y = (float)__float_as_uint(x);
	y *= 8.2629582881927490e-8f;
	return y - 87.989971088f;
}

__device__ __forceinline__ float fast_logit(float p, float width) {
	const float n = 0.001f + (p * 0.998f);
	return faster_ln((n / (1.0f - n))) * width * (0.6266f / 4.0f);
}

__device__ __forceinline__ void square_to_circle(float* x, float* y) {
	if (*x == 0.0f && *y == 0.0f) return;
	float radius, angle;
	if (*x > fabsf(*y)) {
		radius = *x;
		angle = (float)(PSY_QPI_D * (double)(*y / *x));
	} else if (*y > fabsf(*x)) {
		radius = *y;
		angle = (float)(PSY_QPI_D * (double)(2.0f - (*x / *y)));
	} else if (*x < -fabsf(*y)) {
		radius = -*x;
		angle = (float)(PSY_QPI_D * (double)(4.0f + (*y / *x)));
	} else {
		radius = -*y;
		angle = (float)(PSY_QPI_D * (double)(6.0f - (*x / *y)));
	}
	float sine, cosine;
	lm_sincosf(angle, &sine, &cosine);
	*x = radius * cosine;
	*y = radius * sine;
}

__device__ __forceinline__ V3 cosine_sample_hemisphere(float u, float v) {
	u = (u * 2) - 1;
	v = (v * 2) - 1;
	square_to_circle(&u, &v);
	const double t = 1.0 - (double)((u * u) + (v * v));
	const float z = (float)sqrt(t > 0.0 ? t : 0.0);
	return V3(u, v, z);
}

__device__ __forceinline__ void coordinate_system(V3 v1, V3* v2, V3* v3) {
	if (fabsf(v1.x) > fabsf(v1.y)) {
		const float invlen = 1.f / sqrtf(v1.x * v1.x + v1.z * v1.z);
		*v2 = V3(-v1.z * invlen, 0.f, v1.x * invlen);
	} else {
		const float invlen = 1.f / sqrtf(v1.y * v1.y + v1.z * v1.z);
		*v2 = V3(0.f, v1.z * invlen, -v1.y * invlen);
	}
	*v3 = cross(v1, *v2);
}

__device__ __forceinline__ V3 zup_to_vec(V3 from, V3 toz) {
	V3 tox, toy;
	toz = normalized(toz);
	coordinate_system(toz, &tox, &toy);
	return (tox * from.x) + (toy * from.y) + (toz * from.z);
}

__device__ __forceinline__ V3 uniform_sample_sphere(float u, float v) {
	const float z = 1.f - (2.f * u);
	const float t = 1.f - z * z;
	const float r = sqrtf(0.f < t ? t : 0.f);
	const float phi = (float)((2.0 * PSY_PI_D) * (double)v);
	float sine, cosine;
	lm_sincosf(phi, &sine, &cosine);
	return V3(r * cosine, r * sine, z);
}

// sphere_lambert (utils/monte_carlo.hpp:207-233).
__device__ __forceinline__ float sphere_lambert(float nlcos, float rcos) {
	const float nlsin = (float)sqrt(1.0 - (double)(nlcos * nlcos));
	const float rsin2 = (float)(1.0 - (double)(rcos * rcos));
	const float rsin = sqrtf(rsin2);
	const float ysin = rcos / nlsin;
	const float ycos2 = (float)(1.0 - (double)(ysin * ysin));
	const float ycos = sqrtf(ycos2);
	const float g = (float)(((((-2.0 * (double)nlsin) * (double)rcos) * (double)ycos) + PSY_HPI_D) -
	                        (double)lm_asinf(ysin) + (double)(ysin * ycos));
	const float h = nlcos * ((ycos * sqrtf(rsin2 - ycos2)) + (rsin2 * lm_asinf(ycos / rsin)));
	const float nl = lm_acosf(nlcos);
	const float r = lm_acosf(rcos);
	if ((double)nl < (PSY_HPI_D - (double)r)) return nlcos * rsin2;
	if ((double)nl < PSY_HPI_D) return (nlcos * rsin2) + g - h;
	if ((double)nl < (PSY_HPI_D + (double)r)) return (float)((double)(g + h) * PSY_INV_PI_D);
	return 0.0f;
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
	const float a2 = a * a;
	const float b2 = b * b;
	return a2 / (a2 + b2);
}

// ---------------------------------------------------------------------
// Spectral
// ---------------------------------------------------------------------
struct Spec {
	float e[4];
};

__device__ __forceinline__ float wavelength_n(float hero, int n) {
	hero += (float)n * (WAVELENGTH_RANGE / 4);
	if (hero > WAVELENGTH_MAX) hero -= WAVELENGTH_RANGE;
	return hero;
}

__device__ __forceinline__ float X_1931(float w) {
	const float t1 = (w - 442.0f) * ((w < 442.0f) ? 0.0624f : 0.0374f);
	const float t2 = (w - 599.8f) * ((w < 599.8f) ? 0.0264f : 0.0323f);
	const float t3 = (w - 501.1f) * ((w < 501.1f) ? 0.0490f : 0.0382f);
	return (0.362f * lm_expf(-0.5f * t1 * t1)) + (1.056f * lm_expf(-0.5f * t2 * t2)) - (0.065f * lm_expf(-0.5f * t3 * t3));
}
__device__ __forceinline__ float Y_1931(float w) {
	const float t1 = (w - 568.8f) * ((w < 568.8f) ? 0.0213f : 0.0247f);
	const float t2 = (w - 530.9f) * ((w < 530.9f) ? 0.0613f : 0.0322f);
	return (0.821f * lm_expf(-0.5f * t1 * t1)) + (0.286f * lm_expf(-0.5f * t2 * t2));
}
__device__ __forceinline__ float Z_1931(float w) {
	const float t1 = (w - 437.0f) * ((w < 437.0f) ? 0.0845f : 0.0278f);
	const float t2 = (w - 459.0f) * ((w < 459.0f) ? 0.0385f : 0.0725f);
	return (1.217f * lm_expf(-0.5f * t1 * t1)) + (0.681f * lm_expf(-0.5f * t2 * t2));
}

// spectrum_xyz_to_p (color/spectrum_grid.h:21-135).
static __device__ float spectrum_xyz_to_p(float lambda, const float* xyz) {
	const float norm = (float)(1.0 / (double)(xyz[0] + xyz[1] + xyz[2]));
	if (!(norm < FLT_MAX)) return 0.0f;
	float xyY[2], uv[2];
	xyY[0] = xyz[0] * norm;
	xyY[1] = xyz[1] * norm;
	uv[0] = psy_spec_xy_to_uv[0] * xyY[0] + psy_spec_xy_to_uv[1] * xyY[1] + psy_spec_xy_to_uv[2];
	uv[1] = psy_spec_xy_to_uv[3] * xyY[0] + psy_spec_xy_to_uv[4] * xyY[1] + psy_spec_xy_to_uv[5];
	if (uv[0] < 0.0f || uv[0] >= PSY_SPEC_GRID_W || uv[1] < 0.0f || uv[1] >= PSY_SPEC_GRID_H) return 0.f;
	const int uvi0 = (int)uv[0], uvi1 = (int)uv[1];
	const int cell = uvi0 + PSY_SPEC_GRID_W * uvi1;
	const int inside = psy_spec_cells[cell][0];
	const int num = psy_spec_cells[cell][1];
	const int* idx = &psy_spec_cells[cell][2];
	const float sb = (lambda - 380.0f) / (780.0f - 380.0f) * (float)(PSY_SPEC_SAMPLES - 1);
	const int sb0 = (int)sb;
	const int sb1 = (sb + 1 < (float)PSY_SPEC_SAMPLES) ? (int)(sb + 1) : PSY_SPEC_SAMPLES - 1;
	const float sbf = sb - (float)sb0;
	float p[6];
	for (int i = 0; i < num; ++i) {
		const float* spectrum = psy_spec_point_spectrum[idx[i]];
		p[i] = spectrum[sb0] * (1.0f - sbf) + spectrum[sb1] * sbf;
	}
	float interpolated_p = 0.0f;
	if (inside) {
		const float u0 = uv[0] - (float)uvi0;
		const float u1 = uv[1] - (float)uvi1;
		interpolated_p = p[0] * (1.0f - u0) * (1.0f - u1) + p[2] * (1.0f - u0) * u1 + p[3] * u0 * u1 +
		                 p[1] * u0 * (1.0f - u1);
	} else {
		const float ex = uv[0] - psy_spec_point_uv[idx[0]][0];
		const float ey = uv[1] - psy_spec_point_uv[idx[0]][1];
		float e0x = psy_spec_point_uv[idx[1]][0] - psy_spec_point_uv[idx[0]][0];
		float e0y = psy_spec_point_uv[idx[1]][1] - psy_spec_point_uv[idx[0]][1];
		float uu = e0x * ey - ex * e0y;
		for (int i = 0; i < num - 1; i++) {
			float e1x, e1y;
			if (i == num - 2) {
				e1x = psy_spec_point_uv[idx[1]][0] - psy_spec_point_uv[idx[0]][0];
				e1y = psy_spec_point_uv[idx[1]][1] - psy_spec_point_uv[idx[0]][1];
			} else {
				e1x = psy_spec_point_uv[idx[i + 2]][0] - psy_spec_point_uv[idx[0]][0];
				e1y = psy_spec_point_uv[idx[i + 2]][1] - psy_spec_point_uv[idx[0]][1];
			}
			const float vv = ex * e1y - e1x * ey;
			const float area = e0x * e1y - e1x * e0y;
			const float u = uu / area;
			const float v = vv / area;
			const float w = 1.0f - u - v;
			if (u < 0.0f || v < 0.0f || w < 0.0f) {
				uu = -vv;
				e0x = e1x;
				e0y = e1y;
				continue;
			}
			interpolated_p = p[0] * w + p[i + 1] * v + p[(i == num - 2) ? 1 : (i + 2)] * u;
			break;
		}
	}
	return interpolated_p / norm;
}

// Color_to_XYZ (color/color.hpp:476-487) then XYZ_to_SpectralSample.
// Not inlined: called several times per path step, one copy of its code
// keeps the shading kernels small.
static __device__ __noinline__ Spec rgb_to_spec(const float* col, float hero) {
	float xyz[3];
	xyz[0] = (col[0] * 0.4339f) + (col[1] * 0.3762f) + (col[2] * 0.1899f);
	xyz[1] = (col[0] * 0.2126f) + (col[1] * 0.7152f) + (col[2] * 0.0722f);
	xyz[2] = (col[0] * 0.0177f) + (col[1] * 0.1095f) + (col[2] * 0.8728f);
	const float inv_eer = 1.0f / 0.009358239977091027f;
	Spec s;
#pragma unroll
	for (int i = 0; i < 4; ++i) s.e[i] = spectrum_xyz_to_p(wavelength_n(hero, i), xyz) * inv_eer;
	return s;
}

// Color_XYZ(SpectralSample) (color/color.hpp:179-188).
__device__ __forceinline__ void spec_to_xyz(const Spec& s, float hero, float* out) {
	float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		const float w = wavelength_n(hero, i);
		x += X_1931(w) * s.e[i];
		y += Y_1931(w) * s.e[i];
		z += Z_1931(w) * s.e[i];
	}
	out[0] = x * (1.0f / 4);
	out[1] = y * (1.0f / 4);
	out[2] = z * (1.0f / 4);
}

// ---------------------------------------------------------------------
// Lambert closure
// ---------------------------------------------------------------------
__device__ __forceinline__ Spec lambert_eval(const float* col, V3 in, V3 out, V3 n, float wl) {
	V3 nn = normalized(n);
	const V3 v = normalized(out);
	if (dot(nn, in) > 0.0f) nn = nn * -1.0f;
	const float d = dot(nn, v);
	const float fac = (d > 0.0f ? d : 0.0f) * (float)PSY_INV_PI_D;
	const float c[3] = {col[0] * fac, col[1] * fac, col[2] * fac};
	return rgb_to_spec(c, wl);
}

// The cosine factor lambert_eval scales the colour by.
__device__ __forceinline__ float lambert_cos(V3 in, V3 out, V3 n) {
	V3 nn = normalized(n);
	const V3 v = normalized(out);
	if (dot(nn, in) > 0.0f) nn = nn * -1.0f;
	const float d = dot(nn, v);
	return (d > 0.0f ? d : 0.0f) * (float)PSY_INV_PI_D;
}

// ---------------------------------------------------------------------
// GTR microfacet closure (GTRClosure, shading/surface_closure.hpp:339-608)
// ---------------------------------------------------------------------
// The closure's parameters at a hit (from its validated shader).
struct Gtr {
	float col[3];
	float rough, tail, fres, norm, pow_r2_1mt;
};

__device__ __forceinline__ Gtr gtr_of(const DevShader& s) {
	Gtr g;
	g.col[0] = s.col[0]; g.col[1] = s.col[1]; g.col[2] = s.col[2];
	g.rough = s.roughness;
	g.tail = s.tail_shape;
	g.fres = s.fresnel;
	g.norm = s.norm;
	g.pow_r2_1mt = s.pow_r2_1mt;
	return g;
}

__device__ __forceinline__ bool gtr_is_delta(const Gtr& g) { return g.rough == 0.0f; }

__device__ __forceinline__ float clampf(float v, float a, float b) { return smin(b, smax(a, v)); }

// GTRClosure::normalization (:374-380): top in float, the division in double.
__device__ __forceinline__ float gtr_normalization(float r, float t) {
	const float r2 = r * r;
	const float top = (t - 1.0f) * (r2 - 1.0f);
	const double bottom = PSY_PI_D * (double)(1.0f - powf(r2, 1.0f - t));
	return (float)((double)top / bottom);
}

// GTRClosure::dist (:397-409) with the normalisation factor `norm` of `rough`.
__device__ __forceinline__ float gtr_dist(float nh, float rough, float tail, float norm) {
	const float r2 = rough * rough;
	float D = 0.0f;
	if (nh > 0.0f) {
		const float nh2 = nh * nh;
		D = norm / powf(1.0f + ((r2 - 1.0f) * nh2), tail);
	}
	return D;
}

// GTRClosure::half_theta_sample (:383-395).
__device__ __forceinline__ float gtr_half_theta_sample(const Gtr& g, float u) {
	const float r2 = g.rough * g.rough;
	const float top = 1.0f - powf((g.pow_r2_1mt * (1.0f - u)) + u, 1.0f / (1.0f - g.tail));
	const float bottom = 1.0f - r2;
	return sqrtf(top / bottom);
}

// schlick_fresnel_from_fac (:173-177).
__device__ __forceinline__ float schlick_fresnel_from_fac(float f, float c) {
	const float c1 = 1.0f - c;
	const float c2 = c1 * c1;
	return f + ((((1.0f - f) * c1) * c2) * c2);
}

// GTRClosure::evaluate (:452-516).
static __device__ __noinline__ Spec gtr_eval(const Gtr& g, V3 in, V3 out, V3 n, float wl) {
	V3 nn = normalized(n);
	const V3 aa = normalized(in) * -1.0f;
	const V3 bb = normalized(out);
	const V3 hh = normalized(aa + bb);
	if (dot(nn, hh) < 0.0f) nn = nn * -1.0f;
	const float na = clampf(dot(nn, aa), -1.0f, 1.0f);
	const float nb = clampf(dot(nn, bb), -1.0f, 1.0f);
	const float ha = clampf(dot(hh, aa), -1.0f, 1.0f);
	const float hb = clampf(dot(hh, bb), -1.0f, 1.0f);
	const float nh = clampf(dot(nn, hh), -1.0f, 1.0f);
	const float r2 = g.rough * g.rough;
	float D = 1.0f, G1 = 1.0f, G2 = 1.0f;
	Spec col_f = rgb_to_spec(g.col, wl);
	for (int i = 0; i < 4; ++i) col_f.e[i] = lerp1(1.0f - g.fres, schlick_fresnel_from_fac(col_f.e[i], hb), col_f.e[i]);
	if (g.rough == 0.0f) return col_f;
	if (nh > 0.0f) {
		const float nh2 = nh * nh;
		D = g.norm / powf(1.0f + ((r2 - 1.0f) * nh2), g.tail);
	}
	const float na2 = na * na;
	const float tan_na = sqrtf((1.0f - na2) / na2);
	const float g1_pos_char = (ha * na) > 0.0f ? 1.0f : 0.0f;
	const float g1_a = r2 * tan_na;
	const float g1_b = (sqrtf(1.0f + (g1_a * g1_a)) - 1.0f) * 0.5f;
	G1 = g1_pos_char / (1.0f + g1_b);
	const float nb2 = nb * nb;
	const float tan_nb = sqrtf((1.0f - nb2) / nb2);
	const float g2_pos_char = (hb * nb) > 0.0f ? 1.0f : 0.0f;
	const float g2_a = r2 * tan_nb;
	const float g2_b = (sqrtf(1.0f + (g2_a * g2_a)) - 1.0f) * 0.5f;
	G2 = g2_pos_char / (1.0f + g2_b);
	const float f = (D * G1) * G2;
	for (int i = 0; i < 4; ++i) col_f.e[i] = (col_f.e[i] * f) * (float)PSY_INV_PI_D;
	return col_f;
}

// GTRClosure::sample_pdf (:556-571).
static __device__ __noinline__ float gtr_pdf(const Gtr& g, V3 in, V3 out, V3 n) {
	V3 nn = normalized(n);
	const V3 aa = normalized(in) * -1.0f;
	const V3 bb = normalized(out);
	const V3 hh = normalized((aa + bb) * 0.5f);
	if (dot(nn, hh) < 0.0f) nn = nn * -1.0f;
	const float nh = clampf(dot(nn, hh), -1.0f, 1.0f);
	return gtr_dist(nh, g.rough, g.tail, g.norm) * (float)PSY_INV_PI_D;
}

// GTRClosure::sample (:428-449): a half vector from the distribution, the
// mirror direction about it, its pdf and the closure's value.
static __device__ __noinline__ void gtr_sample(const Gtr& g, V3 in, V3 n, float si, float sj, float wl, V3* out,
                                           Spec* filter, float* pdf) {
	V3 nn = normalized(n);
	if (dot(nn, in) > 0.0f) nn = nn * -1.0f;
	const float theta_cos = gtr_half_theta_sample(g, si);
	const float theta_sin = sqrtf(1.0f - (theta_cos * theta_cos));
	const float angle = (float)(((double)sj * PSY_PI_D) * 2.0);
	float sine, cosine;
	lm_sincosf(angle, &sine, &cosine);
	V3 half_dir(cosine * theta_sin, sine * theta_sin, theta_cos);
	half_dir = normalized(zup_to_vec(half_dir, nn));
	*out = in - ((half_dir * 2.0f) * dot(in, half_dir));
	*pdf = gtr_pdf(g, in, *out, n);
	*filter = gtr_eval(g, in, *out, n, wl);
}

// GTRClosure::estimate_eval_over_solid_angle (:519-553).
static __device__ __noinline__ float gtr_estimate(const Gtr& g, V3 in, V3 cent, float cos_theta, V3 nor) {
	V3 nn = normalized(nor);
	const V3 aa = normalized(in) * -1.0f;
	const V3 bb = normalized(cent);
	if (dot(nn, in) > 0.0f) nn = nn * -1.0f;
	const float theta = lm_acosf(cos_theta);
	const V3 hh = normalized(aa + bb);
	const float nh = clampf(dot(nn, hh), -1.0f, 1.0f);
	const float rough = smin(1.0f, sqrtf(g.rough) + ((2.0f * theta) / (float)PSY_PI_D));
	const float fac = gtr_dist(nh, rough, g.tail, gtr_normalization(rough, g.tail));
	return (fac * smin(1.0f - cos_theta, 1.0f)) * (float)PSY_INV_PI_D;
}

// Matrix44::setAxisAngle (math/matrix.hpp:345-372, after ImathMatrix.h) with
// make_axis_angle_transform (math/transform.hpp:221-226).
__device__ __forceinline__ M44 axis_angle(V3 axis, float angle) {
	const V3 u = normalized(axis);
	float sine, cosine;
	lm_sincosf(angle, &sine, &cosine);
	const float c1 = 1.0f - cosine;
	M44 m;
	m.m[0][0] = ((u.x * u.x) * c1) + cosine;
	m.m[0][1] = ((u.x * u.y) * c1) + (u.z * sine);
	m.m[0][2] = ((u.x * u.z) * c1) - (u.y * sine);
	m.m[0][3] = 0.0f;
	m.m[1][0] = ((u.x * u.y) * c1) - (u.z * sine);
	m.m[1][1] = ((u.y * u.y) * c1) + cosine;
	m.m[1][2] = ((u.y * u.z) * c1) + (u.x * sine);
	m.m[1][3] = 0.0f;
	m.m[2][0] = ((u.x * u.z) * c1) + (u.y * sine);
	m.m[2][1] = ((u.y * u.z) * c1) - (u.x * sine);
	m.m[2][2] = ((u.z * u.z) * c1) + cosine;
	m.m[2][3] = 0.0f;
	m.m[3][0] = 0.0f;
	m.m[3][1] = 0.0f;
	m.m[3][2] = 0.0f;
	m.m[3][3] = 1.0f;
	return m;
}

// reflect_ray_direction_differential and calc_uv_differentials
// (basics/differential_geometry.hpp:113-156), clamp_dd (:125-135).
__device__ __forceinline__ V3 reflect_dd(V3 normal, V3 normal_d, V3 d, V3 dd) {
	const float ddn = dot(dd, normal) + dot(d, normal_d);
	const V3 tmp = (normal_d * dot(d, normal)) + (normal * ddn);
	return dd - (tmp * 2.0f);
}
__device__ __forceinline__ void uv_differentials(V3 dp, V3 dpdu, V3 dpdv, float* du, float* dv) {
	const float dpdu_ilen = 1.0f / length(dpdu);
	const V3 dpdu_n = dpdu * dpdu_ilen;
	const float dpdv_ilen = 1.0f / length(dpdv);
	const V3 dpdv_n = dpdv * dpdv_ilen;
	*du = dot(dp, dpdu_n) * dpdu_ilen;
	*dv = dot(dp, dpdv_n) * dpdv_ilen;
}

// ---------------------------------------------------------------------
// Parameterised albedo (differentiable rendering; no reference counterpart)
// ---------------------------------------------------------------------
// Gaussian basis function k at wavelength w (nm).
__device__ __forceinline__ float albedo_basis(int k, float w) {
	const float c = PSY_ALBEDO_BASIS_C0 + (float)k * PSY_ALBEDO_BASIS_STEP;
	const float x = (w - c) * (1.0f / PSY_ALBEDO_BASIS_SIGMA);
	return expf(-0.5f * x * x);
}

// Albedo spectrum at the four hero wavelengths from weights p[0..3].
__device__ __forceinline__ Spec albedo_spec(const float* p, float hero) {
	Spec a;
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		const float w = wavelength_n(hero, i);
		float v = 0.0f;
#pragma unroll
		for (int k = 0; k < 4; ++k) v += p[k] * albedo_basis(k, w);
		a.e[i] = v;
	}
	return a;
}

__device__ __forceinline__ float lambert_pdf(V3 in, V3 out, V3 n) {
	V3 nn = normalized(n);
	const V3 v = normalized(out);
	if (dot(nn, normalized(in)) > 0.0f) nn = nn * -1.0f;
	const float p = dot(nn, v) * (float)PSY_INV_PI_D;
	return p > 0.0f ? p : 0.0f;
}

__device__ __forceinline__ float lambert_estimate(V3 in, V3 out, float cos_theta, V3 nor) {
	if (cos_theta < 0.0f) return 1.0f;
	V3 nn = normalized(nor);
	const V3 v = normalized(out);
	if (dot(nn, in) > 0.0f) nn = nn * -1.0f;
	return sphere_lambert(dot(nn, v), cos_theta);
}

__device__ __forceinline__ V3 transfer_origin_differential(float t, V3 normal, V3 d, V3 od, V3 dd) {
	const V3 temp = od + (dd * t);
	const float td = -dot(temp, normal) / dot(d, normal);
	const V3 real_projected = temp + (d * td);
	return normalized(real_projected) * length(temp);
}

// ---------------------------------------------------------------------
// Light tree and sphere lights
// ---------------------------------------------------------------------
struct LightQuery {
	float n, u, v;
	V3 pos, nor, d;
	float wavelength, time;
	bool gtr;             // the query's BSDF: GTR (gp) or Lambert
	Gtr gp;
	// out
	M44 xform;
	bool has_xform;
	uint64_t id;
	int obj;              // global object index of the sampled light
	V3 to_light;
	Spec spec;
	float selection_pdf;
	float light_sample_pdf;
	bool valid;
};

__device__ __forceinline__ Box light_node_box(const DevScene& sc, const DevLightNode& nd, float time) {
	Box b0;
	b0.lo = V3(nd.lo[0], nd.lo[1], nd.lo[2]);
	b0.hi = V3(nd.hi[0], nd.hi[1], nd.hi[2]);
	if (nd.ts <= 1) return b0;
	const SeqPos sp = seq_pos(time, nd.ts);
	auto sample = [&](int k) -> Box {
		if (k == 0) return b0;
		const float* e = sc.light_extra + (size_t)(nd.extra + k - 1) * 6;
		Box b;
		b.lo = V3(e[0], e[1], e[2]);
		b.hi = V3(e[3], e[4], e[5]);
		return b;
	};
	if (sp.single) return sample(sp.i0);
	return box_lerp(sp.nalpha, sample(sp.i0), sample(sp.i0 + 1));
}

static __device__ __noinline__ float light_node_prob(const DevScene& sc, const LightQuery& q, int index) {
	const DevLightNode nd = sc.light_nodes[index];
	const Box bbox = light_node_box(sc, nd, q.time);
	const V3 d = box_center(bbox) - q.pos;
	const float dist2 = length2(d);
	const float r = box_diagonal(bbox) * 0.5f;
	const float r2 = r * r;
	const float inv_surface_area = 1.0f / r2;
	float cos_theta_max;
	if (dist2 <= r2) {
		cos_theta_max = -1.0f;
	} else {
		const float q2 = r2 / dist2;
		const float sin_theta_max2 = q2 < 1.0f ? q2 : 1.0f;
		cos_theta_max = sqrtf(1.0f - sin_theta_max2);
	}
	const float est = q.gtr ? gtr_estimate(q.gp, q.d, d, cos_theta_max, q.nor) : lambert_estimate(q.d, d, cos_theta_max, q.nor);
	const float approx_contrib = 0.0f < est ? est : 0.0f;
	return nd.energy * inv_surface_area * approx_contrib;
}

// SphereLight::sample; returns the colour scale and writes the shadow vector and pdf.
static __device__ __noinline__ void sphere_light_sample(const DevScene& sc, const DevObject& ob, V3 arr, float u, float v, float wl,
                                    float time, V3* shadow_vec, float* pdf, Spec* spec) {
	V3 pos;
	float radius_f;
	float col[3];
	light_at(sc, ob, time, &pos, &radius_f, col);
	const double radius = (double)radius_f;
	const double surface_area_inv = 1.0 / (4.0 * PSY_PI_D * radius * radius);
	V3 x, y;
	V3 z = pos - arr;
	const double d2 = (double)length2(z);
	const double d = sqrt(d2);
	coordinate_system(z, &x, &y);
	x = normalized(x);
	y = normalized(y);
	z = normalized(z);
	if (d > radius) {
		const double s2 = (radius * radius) / d2;
		const double sin_theta_max2 = s2 < 1.0 ? s2 : 1.0;
		const double cos_theta_max2 = 1.0 - sin_theta_max2;
		const double sin_theta_max = sqrt(sin_theta_max2);
		const double cos_theta_max = sqrt(cos_theta_max2);
		// uniform_sample_cone<double>
		const double du = (double)u, dv = (double)v;
		const double ct = (1.0 - du) + (du * cos_theta_max);
		const double st = sqrt(1.0 - (ct * ct));
		const double phi0 = dv * 2.0 * PSY_PI_D;
		V3 sample = normalized(V3((float)(cos(phi0) * st), (float)(sin(phi0) * st), (float)ct));
		const double cos_theta = (double)sample.z;
		const double cos_theta2 = cos_theta * cos_theta;
		const double t2 = 1.0 - cos_theta2;
		const double sin_theta2 = 0.0 < t2 ? t2 : 0.0;
		const double sin_theta = sqrt(sin_theta2);
		const double D = 1.0 - (d2 * sin_theta * sin_theta / (radius * radius));
		double cos_a;
		if (D <= 0.0) cos_a = sin_theta_max;
		else cos_a = ((d / radius) * sin_theta2) + (cos_theta * sqrt(D));
		const double t3 = 1.0 - (cos_a * cos_a);
		const double sin_a = sqrt(0.0 < t3 ? t3 : 0.0);
		const double phi = dv * 2.0 * PSY_PI_D;
		sample.x = (float)(cos(phi) * sin_a * radius);
		sample.y = (float)(sin(phi) * sin_a * radius);
		sample.z = (float)(d - (cos_a * radius));
		*shadow_vec = (x * sample.x) + (y * sample.y) + (z * sample.z);
		*pdf = (float)(1.0 / (2.0 * PSY_PI_D * (1.0 - cos_theta_max)));
	} else {
		*shadow_vec = uniform_sample_sphere(u, v);
		*pdf = (float)(1.0f / (4.0f * PSY_PI_D));
	}
	const float sai = (float)surface_area_inv;
	const float c[3] = {col[0] * sai, col[1] * sai, col[2] * sai};
	*spec = rgb_to_spec(c, wl);
}

// uniform_sample_spherical_triangle (utils/monte_carlo.hpp:143-196, after
// Arvo, "Stratified Sampling of Spherical Triangles", 1995): the angles in
// double as there; the vector arithmetic is Vec3's float arithmetic, each
// double factor rounded to float where it scales a Vec3.
static __device__ __noinline__ V3 uniform_sample_spherical_triangle(V3 A, V3 B, V3 C, float i, float j) {
	auto clampd = [](double v) { return fmin(1.0, fmax(-1.0, v)); };
	const double cos_a = clampd((double)dot(B, C));
	const double cos_b = clampd((double)dot(C, A));
	const double cos_c = clampd((double)dot(A, B));
	const double sin_a = sqrt(1.0 - (cos_a * cos_a));
	const double sin_b = sqrt(1.0 - (cos_b * cos_b));
	const double sin_c = sqrt(1.0 - (cos_c * cos_c));
	if (cos_a == 1.0 || cos_b == 1.0 || cos_c == 1.0) return A;
	const double cos_A = clampd((cos_a - (cos_b * cos_c)) / (sin_b * sin_c));
	const double cos_B = clampd((cos_b - (cos_c * cos_a)) / (sin_c * sin_a));
	const double cos_C = clampd((cos_c - (cos_a * cos_b)) / (sin_a * sin_b));
	const double sin_A = sqrt(1.0 - (cos_A * cos_A));
	const double ang_A = acos(cos_A);
	const double ang_B = acos(cos_B);
	const double ang_C = acos(cos_C);
	const double area = ((ang_A + ang_B) + ang_C) - PSY_PI_D;
	const double area_2 = area * (double)i;
	const double s = sin(area_2 - ang_A);
	const double t = cos(area_2 - ang_A);
	const double u = t - cos_A;
	const double v = s + (sin_A * cos_c);
	const double q_top = (((v * t) - (u * s)) * cos_A) - v;
	const double q_bottom = ((v * s) + (u * t)) * sin_A;
	const double q = q_top / q_bottom;
	const V3 C_2 = (A * (float)q) + (normalized(C - (A * dot(C, A))) * (float)sqrt(1.0 - (q * q)));
	const double z = 1.0 - ((double)j * (1.0 - (double)dot(C_2, B)));
	return (B * (float)z) + (normalized(C_2 - (B * dot(C_2, B))) * (float)sqrt(1.0 - (z * z)));
}

// RectangleLight::sample (lights/rectangle_light.hpp:40-71): one of the
// rectangle's two spherical triangles, chosen by solid angle, sampled
// uniformly and projected back onto the rectangle.
static __device__ __noinline__ void rect_light_sample(const DevScene& sc, const DevObject& ob, V3 arr, float u, float v, float wl,
                                         float time, V3* shadow_vec, float* pdf, Spec* spec) {
	float dx, dy, col[3];
	rect_light_at(sc, ob, time, &dx, &dy, col);
	const double inv_surface_area = 1.0 / (double)(dx * dy);
	V3 p[4];
	float area_1, area_2;
	rect_light_corners(dx, dy, arr, p, &area_1, &area_2);
	const float prob_1 = area_1 / (area_1 + area_2);
	const float prob_2 = 1.0f - prob_1;
	V3 sv;
	if (u < prob_1) sv = uniform_sample_spherical_triangle(p[1], p[0], p[2], v, u / prob_1);
	else sv = uniform_sample_spherical_triangle(p[3], p[0], p[2], v, 1.0f - ((u - prob_1) / prob_2));
	sv = sv * (-arr.z / sv.z);
	*shadow_vec = sv;
	*pdf = 1.0f / (area_1 + area_2);
	const float isa = (float)inv_surface_area;
	const float c[3] = {(col[0] * isa) * 0.5f, (col[1] * isa) * 0.5f, (col[2] * isa) * 0.5f};
	*spec = rgb_to_spec(c, wl);
}

// Matrix44::inverse on the device, not inlined: only transformed hits and
// instanced lights need it, and one copy keeps the shading kernels' code
// small.
static __device__ __noinline__ M44 m44_inverse_dev(const M44& a, const RcpTable& rt) { return m44_inverse(a, rt); }

// LightTree::sample starting at the root assembly's tree.
static __device__ void light_tree_sample(const DevScene& sc, LightQuery* q, float ident_inv) {
	q->valid = false;
	int asmb = 0;
	for (int level = 0; level < 16; ++level) {
		const DevAssembly as = sc.assemblies[asmb];
		if (as.light_root < 0) return;
		int node = as.light_root;
		float tot_prob = 1.0f;
		// a tree is never deeper than its node count: the bound only stops a
		// walk over a malformed tree
		for (int guard = 0; guard < sc.light_node_count; ++guard) {
			const DevLightNode nd = sc.light_nodes[node];
			if (nd.is_leaf) break;
			float p1 = light_node_prob(sc, *q, nd.c1);
			float p2 = light_node_prob(sc, *q, nd.c2);
			const float total = p1 + p2;
			if (total <= 0.0f) {
				p1 = 0.5f;
				p2 = 0.5f;
			} else {
				p1 /= total;
				p2 /= total;
			}
			if (q->n <= p1) {
				tot_prob *= p1;
				node = nd.c1;
				q->n /= p1;
			} else {
				tot_prob *= p2;
				node = nd.c2;
				q->n = (q->n - p1) / p2;
			}
		}
		const DevLightNode leaf = sc.light_nodes[node];
		if (!leaf.is_leaf || leaf.c1 < 0 || leaf.c1 >= as.inst_count) return;  // malformed tree: no sample
		const int local = leaf.c1;
		const DevInstance inst = sc.instances[as.inst_base + local];
		q->id = id_push(q->id, (uint64_t)local, as.id_bits);
		if (inst.xform_count > 0) {
			const M44 X = seq_lerp_global(sc.xforms + (size_t)inst.xform * 16, inst.xform_count, q->time);
			q->pos = pos_to(X, q->pos);
			q->nor = normalized(dir_transpose(m44_inverse_dev(X, sc.rcp), q->nor));
			q->xform = q->has_xform ? m44_mul(q->xform, X) : m44_mul(m44_identity(), X);
			q->has_xform = true;
		}
		if (inst.kind == INST_OBJECT) {
			const DevObject ob = sc.objects[inst.data];
			if (ob.kind != OBJ_SPHERE_LIGHT && ob.kind != OBJ_RECT_LIGHT) return;
			q->obj = inst.data;
			float p = 1.0f;
			V3 tl;
			if (ob.kind == OBJ_SPHERE_LIGHT)
				sphere_light_sample(sc, ob, q->pos, q->u, q->v, q->wavelength, q->time, &tl, &p, &q->spec);
			else
				rect_light_sample(sc, ob, q->pos, q->u, q->v, q->wavelength, q->time, &tl, &p, &q->spec);
			// xform.dir_from: the reference inverts the accumulated transform,
			// which is the identity when no instance carried one
			if (q->has_xform) q->to_light = dir_to(m44_inverse_dev(q->xform, sc.rcp), tl);
			else q->to_light = tl * ident_inv;
			q->selection_pdf *= (tot_prob * (float)as.light_count);
			q->light_sample_pdf = p;
			q->valid = true;
			return;
		}
		const DevAssembly sub = sc.assemblies[inst.data];
		q->selection_pdf *= (tot_prob * (float)as.light_count) / (float)sub.light_count;
		asmb = inst.data;
	}
}

// ---------------------------------------------------------------------
// Camera (basics/camera.hpp:72-104)
// ---------------------------------------------------------------------
__device__ __forceinline__ float seq_lerp_f(const float* p, int count, float alpha) {
	const SeqPos sp = seq_pos(alpha, count);
	if (sp.single) return p[sp.i0];
	return lerp1(sp.nalpha, p[sp.i0], p[sp.i0 + 1]);
}

static __device__ void camera_ray(const DevScene& sc, float x, float y, float dx, float dy, float time, float u, float v,
                           WorldRayD* r) {
	const M44 T = seq_lerp_global(sc.cam_xforms, sc.cam_xform_count, time);
	const float tfov = seq_lerp_f(sc.cam_tfovs, sc.cam_tfov_count, time);
	const float aperture = seq_lerp_f(sc.cam_apertures, sc.cam_aperture_count, time);
	const float focus = seq_lerp_f(sc.cam_focus, sc.cam_focus_count, time);
	V3 o, d;
	o.x = aperture * ((u * 2) - 1);
	o.y = aperture * ((v * 2) - 1);
	o.z = 0.0f;
	square_to_circle(&o.x, &o.y);
	d.x = (x * tfov) - (o.x / focus);
	d.y = (y * tfov) - (o.y / focus);
	d.z = 1.0f;
	d = normalized(d);
	r->time = time;
	r->o = pos_to(T, o);
	r->d = dir_to(T, d);
	r->odx = dir_to(T, V3(0.0f));
	r->ody = dir_to(T, V3(0.0f));
	r->ddx = dir_to(T, V3(dx * tfov, 0.0f, 0.0f));
	r->ddy = dir_to(T, V3(0.0f, dy * tfov, 0.0f));
	r->occl = false;
}

}  // namespace psy

#endif
