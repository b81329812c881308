// vec.hpp -- double3 arithmetic under the names reference-style scene code
// uses (the reference keeps them in DEMSPH/kernel/myUtility/myVec.h:13-125:
// pi(), the +, -, *, / operators, dot, cross, length, lengthSquared,
// normalize).  Host-only, in the global namespace, so that a scene main()
// written for the reference compiles against include/demsph_compat.  Code
// that uses the library directly does not need this header.
#pragma once
#include <vector_functions.h>
#include <vector_types.h>

#include <cmath>

constexpr double pi() { return 3.14159265358979323846; }

inline double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline double3 operator-(double3 a) { return make_double3(-a.x, -a.y, -a.z); }
inline double3 operator*(double3 a, double s) { return make_double3(a.x * s, a.y * s, a.z * s); }
inline double3 operator*(double s, double3 a) { return make_double3(a.x * s, a.y * s, a.z * s); }
inline double3 operator/(double3 a, double s) { return make_double3(a.x / s, a.y / s, a.z / s); }
inline double3& operator+=(double3& a, double3 b) { a = a + b; return a; }
inline double3& operator-=(double3& a, double3 b) { a = a - b; return a; }
inline double3& operator*=(double3& a, double s) { a = a * s; return a; }
inline double3& operator/=(double3& a, double s) { a = a / s; return a; }

inline double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double3 cross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline double lengthSquared(double3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline double length(double3 v) { return std::sqrt(lengthSquared(v)); }
// The zero vector for |v|^2 < 1e-20, as the reference's normalize.
inline double3 normalize(double3 v) {
    const double l2 = lengthSquared(v);
    if (l2 < 1.0e-20) return make_double3(0.0, 0.0, 0.0);
    const double inv = 1.0 / std::sqrt(l2);
    return make_double3(v.x * inv, v.y * inv, v.z * inv);
}
