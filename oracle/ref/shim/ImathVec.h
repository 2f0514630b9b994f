/*
 * Test infrastructure: part of the oracle build only.  Nothing in the
 * product links or includes this file.
 *
 * A project-written stand-in for the subset of IlmBase's Imath::Vec3<T>
 * (the "ImathVec.h" header of IlmBase 2.x) that the reference renderer uses
 * through its `Vec3` typedef (reference math/vector.hpp:9,12,186).  IlmBase
 * is not vendored in the reference and is absent from this machine, so its
 * published semantics are restated here:
 *
 *   - length()    = sqrt(x*x + y*y + z*z), with Imath's rescaling branch for
 *                   vectors whose squared length is below 2*FLT_MIN;
 *   - normalize() divides each component by length() when length() != 0;
 *   - scalar * vector with a scalar of another type S computes (S * T) per
 *     component and converts the result back to T.
 */
#ifndef PSY_ORACLE_IMATHVEC_SHIM_H
#define PSY_ORACLE_IMATHVEC_SHIM_H

#include <cmath>
#include <limits>

namespace Imath {

template <class T>
class Vec3 {
public:
	T x, y, z;

	Vec3() {}
	explicit Vec3(T a): x(a), y(a), z(a) {}
	Vec3(T a, T b, T c): x(a), y(b), z(c) {}
	template <class S> Vec3(const Vec3<S>& v): x(T(v.x)), y(T(v.y)), z(T(v.z)) {}

	T& operator[](int i) { return (&x)[i]; }
	const T& operator[](int i) const { return (&x)[i]; }

	bool operator==(const Vec3& v) const { return x == v.x && y == v.y && z == v.z; }
	bool operator!=(const Vec3& v) const { return !(*this == v); }

	T dot(const Vec3& v) const { return x * v.x + y * v.y + z * v.z; }
	T operator^(const Vec3& v) const { return dot(v); }

	Vec3 cross(const Vec3& v) const {
		return Vec3(y * v.z - z * v.y, z * v.x - x * v.z, x * v.y - y * v.x);
	}
	Vec3 operator%(const Vec3& v) const { return cross(v); }

	const Vec3& operator+=(const Vec3& v) { x += v.x; y += v.y; z += v.z; return *this; }
	Vec3 operator+(const Vec3& v) const { return Vec3(x + v.x, y + v.y, z + v.z); }
	const Vec3& operator-=(const Vec3& v) { x -= v.x; y -= v.y; z -= v.z; return *this; }
	Vec3 operator-(const Vec3& v) const { return Vec3(x - v.x, y - v.y, z - v.z); }
	Vec3 operator-() const { return Vec3(-x, -y, -z); }

	const Vec3& operator*=(const Vec3& v) { x *= v.x; y *= v.y; z *= v.z; return *this; }
	const Vec3& operator*=(T a) { x *= a; y *= a; z *= a; return *this; }
	Vec3 operator*(const Vec3& v) const { return Vec3(x * v.x, y * v.y, z * v.z); }
	Vec3 operator*(T a) const { return Vec3(x * a, y * a, z * a); }

	const Vec3& operator/=(const Vec3& v) { x /= v.x; y /= v.y; z /= v.z; return *this; }
	const Vec3& operator/=(T a) { x /= a; y /= a; z /= a; return *this; }
	Vec3 operator/(const Vec3& v) const { return Vec3(x / v.x, y / v.y, z / v.z); }
	Vec3 operator/(T a) const { return Vec3(x / a, y / a, z / a); }

	T length2() const { return dot(*this); }

	T length() const {
		const T l2 = dot(*this);
		if (l2 < T(2) * std::numeric_limits<T>::min()) {
			return length_tiny();
		}
		return std::sqrt(l2);
	}

	const Vec3& normalize() {
		const T l = length();
		if (l != T(0)) {
			x /= l;
			y /= l;
			z /= l;
		}
		return *this;
	}

	Vec3 normalized() const {
		Vec3 v(*this);
		v.normalize();
		return v;
	}

private:
	// Rescaled length for vectors whose squared length would underflow.
	T length_tiny() const {
		T ax = std::abs(x), ay = std::abs(y), az = std::abs(z);
		T m = ax;
		if (m < ay) m = ay;
		if (m < az) m = az;
		if (m == T(0)) return T(0);
		ax /= m;
		ay /= m;
		az /= m;
		return m * std::sqrt(ax * ax + ay * ay + az * az);
	}
};

template <class S, class T>
inline Vec3<T> operator*(S a, const Vec3<T>& v) {
	return Vec3<T>(a * v.x, a * v.y, a * v.z);
}

typedef Vec3<float> V3f;

} // namespace Imath

#endif
