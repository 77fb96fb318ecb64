// glsl_compat.hpp -- TEST INFRASTRUCTURE ONLY.
//
// The GLSL 4.50 subset that the reference's MPM compute shaders use, as C++
// types and functions, so that those shaders compile unchanged in meaning with
// g++ and run on the CPU (oracle/build_ref.py drives that build; the result
// lives in oracle/_ref/ and is only ever a checker for the CPU restatement in
// oracle/mpm_oracle.cpp, never part of the product).
//
// Semantics follow the GLSL 4.50 specification: column-major mat3 (m[c][r]),
// float arithmetic in float, min(x, y) = y < x ? y : x, max(x, y) = x < y ? y
// : x, clamp = min(max(x, lo), hi), mix(x, y, a) = x (1 - a) + y a, sign(0) =
// 0.  Where GLSL leaves the result to the implementation (inversesqrt,
// normalize, exp, log, pow, the order of a matrix product's sums) this header
// makes the same choice as oracle/mpm_oracle.cpp: correctly rounded sqrt,
// 1 / sqrt, v / length(v), the C library's expf / logf / powf / sinf, and sums
// taken in index order.  Only <cstdint> is included, so no C library overload
// of sqrt / abs / min competes with the float ones declared here.
#pragma once
#include <cstdint>

#include "glsl_env.hpp"

typedef uint32_t uint;

// ------------------------------------------------------------------ scalars
inline float abs(float x) { return __builtin_fabsf(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float floor(float x) { return __builtin_floorf(x); }
inline float fract(float x) { return x - __builtin_floorf(x); }
inline float sqrt(float x) { return __builtin_sqrtf(x); }
inline float inversesqrt(float x) { return 1.0f / __builtin_sqrtf(x); }
inline float exp(float x) { return __builtin_expf(x); }
inline float log(float x) { return __builtin_logf(x); }
inline float pow(float x, float y) { return __builtin_powf(x, y); }
inline float sin(float x) { return __builtin_sinf(x); }
inline float min(float x, float y) { return y < x ? y : x; }
inline float max(float x, float y) { return x < y ? y : x; }
inline int min(int x, int y) { return y < x ? y : x; }
inline int max(int x, int y) { return x < y ? y : x; }
inline uint min(uint x, uint y) { return y < x ? y : x; }
inline uint max(uint x, uint y) { return x < y ? y : x; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float uintBitsToFloat(uint u) {
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
}
inline uint floatBitsToUint(float f) {
  uint u;
  __builtin_memcpy(&u, &f, 4);
  return u;
}
// The shaders' only atomics are integer counters (hash count / hash sort).
inline uint atomicAdd(uint& mem, uint v) { return __atomic_fetch_add(&mem, v, __ATOMIC_RELAXED); }

// ------------------------------------------------------------------ vectors
struct bvec3 {
  bool x, y, z;
};
inline bool any(bvec3 b) { return b.x || b.y || b.z; }

template <class T> struct tvec3 {
  // x, y, z name the three elements of v (a GNU anonymous struct in a union).
  union {
    struct {
      T x, y, z;
    };
    T v[3];
  };
  tvec3() : x(0), y(0), z(0) {}
  template <class S> explicit tvec3(S s) : x(T(s)), y(T(s)), z(T(s)) {}
  template <class A, class B, class C> tvec3(A a, B b, C c) : x(T(a)), y(T(b)), z(T(c)) {}
  template <class U> explicit tvec3(const tvec3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
  T& operator[](uint i) { return v[i]; }
  const T& operator[](uint i) const { return v[i]; }
  tvec3& xyz() { return *this; }
  const tvec3& xyz() const { return *this; }
};
using vec3 = tvec3<float>;
using ivec3 = tvec3<int>;
using uvec3 = tvec3<uint>;

template <class T> inline tvec3<T> operator-(tvec3<T> a) { return tvec3<T>(-a.x, -a.y, -a.z); }
#define NEBULA_GLSL_VEC_OP(op)                                                                              \
  template <class T> inline tvec3<T> operator op(tvec3<T> a, tvec3<T> b) {                                  \
    return tvec3<T>(a.x op b.x, a.y op b.y, a.z op b.z);                                                     \
  }                                                                                                          \
  template <class T, class S> inline tvec3<T> operator op(tvec3<T> a, S s) {                                \
    return tvec3<T>(a.x op T(s), a.y op T(s), a.z op T(s));                                                  \
  }                                                                                                          \
  template <class T, class S> inline tvec3<T> operator op(S s, tvec3<T> a) {                                \
    return tvec3<T>(T(s) op a.x, T(s) op a.y, T(s) op a.z);                                                  \
  }                                                                                                          \
  template <class T> inline tvec3<T>& operator op##=(tvec3<T>& a, tvec3<T> b) { return a = a op b; }        \
  template <class T, class S> inline tvec3<T>& operator op##=(tvec3<T>& a, S s) { return a = a op T(s); }
NEBULA_GLSL_VEC_OP(+)
NEBULA_GLSL_VEC_OP(-)
NEBULA_GLSL_VEC_OP(*)
NEBULA_GLSL_VEC_OP(/)
#undef NEBULA_GLSL_VEC_OP

template <class T> inline bvec3 lessThan(tvec3<T> a, tvec3<T> b) { return bvec3{a.x < b.x, a.y < b.y, a.z < b.z}; }
template <class T> inline bvec3 greaterThanEqual(tvec3<T> a, tvec3<T> b) {
  return bvec3{a.x >= b.x, a.y >= b.y, a.z >= b.z};
}
template <class T> inline tvec3<T> min(tvec3<T> a, tvec3<T> b) { return tvec3<T>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
template <class T> inline tvec3<T> max(tvec3<T> a, tvec3<T> b) { return tvec3<T>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 min(vec3 a, float s) { return min(a, vec3(s)); }
inline vec3 max(vec3 a, float s) { return max(a, vec3(s)); }
template <class T> inline tvec3<T> clamp(tvec3<T> x, tvec3<T> lo, tvec3<T> hi) { return min(max(x, lo), hi); }
inline vec3 abs(vec3 a) { return vec3(abs(a.x), abs(a.y), abs(a.z)); }
inline vec3 sign(vec3 a) { return vec3(sign(a.x), sign(a.y), sign(a.z)); }
inline vec3 floor(vec3 a) { return vec3(floor(a.x), floor(a.y), floor(a.z)); }
inline vec3 fract(vec3 a) { return vec3(fract(a.x), fract(a.y), fract(a.z)); }
inline vec3 sqrt(vec3 a) { return vec3(sqrt(a.x), sqrt(a.y), sqrt(a.z)); }
inline vec3 exp(vec3 a) { return vec3(exp(a.x), exp(a.y), exp(a.z)); }
inline vec3 log(vec3 a) { return vec3(log(a.x), log(a.y), log(a.z)); }
inline vec3 sin(vec3 a) { return vec3(sin(a.x), sin(a.y), sin(a.z)); }
inline vec3 mix(vec3 x, vec3 y, float a) { return x * (1.0f - a) + y * a; }
inline float dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(vec3 a) { return sqrt(dot(a, a)); }
inline vec3 normalize(vec3 a) { return a / length(a); }
inline vec3 cross(vec3 a, vec3 b) { return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

struct vec4 {
  float x, y, z, w;
  vec4() : x(0), y(0), z(0), w(0) {}
  explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  vec4(vec3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
  // .xyz of a vec4 names its first three components (read and write).
  vec3& xyz() { return *reinterpret_cast<vec3*>(this); }
  vec3 xyz() const { return vec3(x, y, z); }
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
static_assert(sizeof(vec3) == 12 && sizeof(vec4) == 16, "GLSL vector sizes");

// ------------------------------------------------------------------ mat3 (column-major)
struct mat3 {
  vec3 c[3];
  mat3() {}
  explicit mat3(float s) {
    c[0] = vec3(s, 0.0f, 0.0f);
    c[1] = vec3(0.0f, s, 0.0f);
    c[2] = vec3(0.0f, 0.0f, s);
  }
  mat3(vec3 a, vec3 b, vec3 d) {
    c[0] = a;
    c[1] = b;
    c[2] = d;
  }
  template <class A0, class A1, class A2, class A3, class A4, class A5, class A6, class A7, class A8>
  mat3(A0 a0, A1 a1, A2 a2, A3 a3, A4 a4, A5 a5, A6 a6, A7 a7, A8 a8) {
    c[0] = vec3(float(a0), float(a1), float(a2));
    c[1] = vec3(float(a3), float(a4), float(a5));
    c[2] = vec3(float(a6), float(a7), float(a8));
  }
  vec3& operator[](int i) { return c[i]; }
  const vec3& operator[](int i) const { return c[i]; }
};
inline mat3 operator+(const mat3& a, const mat3& b) { return mat3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline mat3 operator-(const mat3& a, const mat3& b) { return mat3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline mat3 operator*(float s, const mat3& a) { return mat3(s * a[0], s * a[1], s * a[2]); }
inline mat3 operator*(const mat3& a, float s) { return mat3(a[0] * s, a[1] * s, a[2] * s); }
inline vec3 operator*(const mat3& A, vec3 v) {
  vec3 r;
  for (int i = 0; i < 3; ++i) r[i] = A[0][i] * v[0] + A[1][i] * v[1] + A[2][i] * v[2];
  return r;
}
inline mat3 operator*(const mat3& A, const mat3& B) {
  mat3 C;
  for (int j = 0; j < 3; ++j) C[j] = A * B[j];
  return C;
}
inline mat3& operator+=(mat3& a, const mat3& b) { return a = a + b; }
inline mat3& operator-=(mat3& a, const mat3& b) { return a = a - b; }
inline mat3 transpose(const mat3& A) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) r[c][k] = A[k][c];
  return r;
}
inline float determinant(const mat3& A) {
  const vec3& a = A[0];
  const vec3& b = A[1];
  const vec3& c = A[2];
  return a[0] * (b[1] * c[2] - c[1] * b[2]) - b[0] * (a[1] * c[2] - c[1] * a[2]) + c[0] * (a[1] * b[2] - b[1] * a[2]);
}
// outerProduct(c, r): column j is c * r[j].
inline mat3 outerProduct(vec3 c, vec3 r) { return mat3(c * r.x, c * r.y, c * r.z); }

