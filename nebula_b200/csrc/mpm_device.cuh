// mpm_device.cuh -- device math shared by every MPM kernel (sm_100a).
//
// Restates, for CUDA, the math of the reference's shader library:
//   Morton codes              shaders/mpm_common.glsl:161-195
//   quadratic B-spline        shaders/mpm_common.glsl:198-210
//   Jacobi eigen / svd3       shaders/mpm_common.glsl:213-281
//   Hencky / fluid stress     shaders/mpm_common.glsl:284-302
//   Von Mises / Drucker-Prager return maps  shaders/mpm_g2p.comp:19-68
//   analytic collider SDFs + Coulomb BC     shaders/collider_common.glsl:22-85
//
// Matrices use GLSL's column-major indexing, m[c][r] = column c, row r, so the
// products below compute exactly what the shaders' `U * diag * transpose(U)`
// and `U * diag * transpose(V)` compute with svd3's layout (singular vectors
// stored as U[.][i], i.e. as rows of the GLSL matrix).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nebula_mpm.h"

namespace nebula {

// ------------------------------------------------------------------ records
struct Material {  // MaterialParams, 64 B
  float mu, lambda, rho0;
  uint32_t model;
  float M_friction, q_cohesion, q_max, bulkK, fluidGamma, viscosity, hardening, xi, pad[4];
};
struct Collider {  // ColliderPrimitive, 64 B
  uint32_t type;
  float px, py, pz, nx, ny, nz, radius, vx, vy, vz, restitution, friction, pad[3];
};
struct Force {  // ForceGPU, 32 B
  uint16_t type, affectMask;
  float data[7];
};
static_assert(sizeof(Material) == 64, "Material");
static_assert(sizeof(Collider) == 64, "Collider");
static_assert(sizeof(Force) == 32, "Force");

enum : uint32_t {
  MAT_ELASTIC = 0, MAT_VON_MISES = 1, MAT_DRUCKER_PRAGER = 2, MAT_GRANULAR_POWDER = 3, MAT_FLUID = 4, MAT_VISCOPLASTIC_MUD = 5,
  MAT_FIXED_COROTATED = 6  // not in the reference's shaders: see fixedCorotatedStress
};
enum : uint32_t { COLL_PLANE = 0, COLL_SPHERE = 1, COLL_BOX = 2, COLL_CAPSULE = 3 };
enum : uint32_t { FORCE_GRAVITY = 0, FORCE_CONSTANT_WIND = 1 };

constexpr int kMaxMaterials = 16;
constexpr int kMaxColliders = 64;
constexpr int kMaxForces = 16;

// Every scalar a substep kernel reads (the MPMSimPC fields, MPMSimPC.h:14-77),
// passed by value.  Tables live in device memory.
struct SubstepParams {
  float dt;
  float cellSize;
  int gridRes[3];
  uint32_t cubeRes;
  uint32_t hashCells;
  float worldMin[3];
  float worldMax[3];
  float flip_ratio;
  uint32_t materialCount;
  uint32_t colliderCount;
  uint32_t forceCount;
  float mu_lame, lambda_lame, rho0, M_friction, q_cohesion, q_max;
  uint32_t plasticModel;
  const Material* materials;
  const Collider* colliders;
  const Force* forces;
  const float* sdf;  // dense Morton-ordered SDF or nullptr
};

// ------------------------------------------------------------------ Morton
__host__ __device__ __forceinline__ uint32_t mortonExpand(uint32_t v) {
  v = (v | (v << 16u)) & 0x030000FFu;
  v = (v | (v << 8u)) & 0x0300F00Fu;
  v = (v | (v << 4u)) & 0x030C30C3u;
  v = (v | (v << 2u)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ uint32_t mortonCompact(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2u)) & 0x030C30C3u;
  v = (v | (v >> 4u)) & 0x0300F00Fu;
  v = (v | (v >> 8u)) & 0x030000FFu;
  v = (v | (v >> 16u)) & 0x000003FFu;
  return v;
}
__host__ __device__ __forceinline__ uint32_t mortonEncode(int x, int y, int z) {
  return mortonExpand(uint32_t(x)) | (mortonExpand(uint32_t(y)) << 1u) | (mortonExpand(uint32_t(z)) << 2u);
}
__host__ __device__ __forceinline__ void mortonDecode(uint32_t c, int& x, int& y, int& z) {
  x = int(mortonCompact(c));
  y = int(mortonCompact(c >> 1u));
  z = int(mortonCompact(c >> 2u));
}

// cellIdFromPos (mpm_common.glsl:190-195): clamp((p - worldMin)/h, 0, gridRes-1), truncate.
__device__ __forceinline__ void cellCoords(const SubstepParams& P, float x, float y, float z, int& cx, int& cy, int& cz) {
  float lx = fminf(fmaxf(__fdiv_rn(x - P.worldMin[0], P.cellSize), 0.0f), float(P.gridRes[0]) - 1.0f);
  float ly = fminf(fmaxf(__fdiv_rn(y - P.worldMin[1], P.cellSize), 0.0f), float(P.gridRes[1]) - 1.0f);
  float lz = fminf(fmaxf(__fdiv_rn(z - P.worldMin[2], P.cellSize), 0.0f), float(P.gridRes[2]) - 1.0f);
  cx = int(uint32_t(lx));
  cy = int(uint32_t(ly));
  cz = int(uint32_t(lz));
}

// One vector reduction of 4 floats into global memory (sm_90+).
__device__ __forceinline__ void redAddV4(float4* addr, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

// ------------------------------------------------------------------ B-spline
__device__ __forceinline__ float gsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ double gsign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

__device__ __forceinline__ float bspline2(float d) {
  float ad = fabsf(d);
  if (ad < 0.5f) return 0.75f - ad * ad;
  if (ad < 1.5f) { float t = 1.5f - ad; return 0.5f * t * t; }
  return 0.0f;
}
__device__ __forceinline__ float bspline2g(float d) {
  float ad = fabsf(d);
  if (ad < 0.5f) return -2.0f * d;
  if (ad < 1.5f) return -gsign(d) * (1.5f - ad);
  return 0.0f;
}

// N(d_k) and N'(d_k) of one axis' three stencil nodes, d_k = (x_p - x_k) / h
// with the nodes at base, base + 1, base + 2: d_0 lies in [0.5, 1.5], d_1 in
// [-0.5, 0.5], d_2 in [-1.5, -0.5] up to rounding, so each node takes the
// branch of bspline2 / bspline2g its interval selects, with the same
// operations (equal results inside the intervals, and at their ends, where
// the branches meet).  A particle outside its cell (a clamped cell index)
// falls back to the general functions.
__device__ __forceinline__ void bsplineStencil(float d0, float d1, float d2, float W[3], float G[3]) {
  if (fabsf(d1) <= 0.5009765625f) {
    const float t0 = fmaxf(1.5f - d0, 0.0f), t2 = fmaxf(1.5f + d2, 0.0f);
    W[0] = 0.5f * t0 * t0;
    G[0] = -t0;
    W[1] = 0.75f - d1 * d1;
    G[1] = -2.0f * d1;
    W[2] = 0.5f * t2 * t2;
    G[2] = t2;
  } else {
    W[0] = bspline2(d0); G[0] = bspline2g(d0);
    W[1] = bspline2(d1); G[1] = bspline2g(d1);
    W[2] = bspline2(d2); G[2] = bspline2g(d2);
  }
}

// ------------------------------------------------------------------ small matrices (GLSL indexing)
template <class T> struct m3 {
  T m[3][3];
};
template <class T> __device__ __forceinline__ m3<T> m3zero() {
  m3<T> r;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; k < 3; ++k) r.m[c][k] = T(0);
  return r;
}
template <class T> __device__ __forceinline__ m3<T> m3ident() {
  m3<T> r = m3zero<T>();
  r.m[0][0] = r.m[1][1] = r.m[2][2] = T(1);
  return r;
}
// GLSL A * B
template <class T> __device__ __forceinline__ m3<T> m3mul(const m3<T>& A, const m3<T>& B) {
  m3<T> C;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) C.m[j][i] = A.m[0][i] * B.m[j][0] + A.m[1][i] * B.m[j][1] + A.m[2][i] * B.m[j][2];
  return C;
}
template <class T> __device__ __forceinline__ T m3det(const m3<T>& A) {
  const T* a = A.m[0];
  const T* b = A.m[1];
  const T* c = A.m[2];
  return a[0] * (b[1] * c[2] - c[1] * b[2]) - b[0] * (a[1] * c[2] - c[1] * a[2]) + c[0] * (a[1] * b[2] - b[1] * a[2]);
}
template <class A, class B> __device__ __forceinline__ m3<A> m3cast(const m3<B>& s) {
  m3<A> r;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; k < 3; ++k) r.m[c][k] = A(s.m[c][k]);
  return r;
}

template <class T> __device__ __forceinline__ T dsqrt(T x);
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <class T> __device__ __forceinline__ T rcpsqrt(T x);
template <> __device__ __forceinline__ float rcpsqrt<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rcpsqrt<double>(double x) { return rsqrt(x); }
template <class T> __device__ __forceinline__ T dlog(T x);
template <> __device__ __forceinline__ float dlog<float>(float x) { return logf(x); }
template <> __device__ __forceinline__ double dlog<double>(double x) { return log(x); }
template <class T> __device__ __forceinline__ T dexp(T x);
template <> __device__ __forceinline__ float dexp<float>(float x) { return expf(x); }
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }

// One Jacobi rotation zeroing A[P][Q] (P < Q), as mpm_common.glsl:224-244; the
// pivot pair is a template argument so every index is static.
template <class T, int P0, int P1>
__device__ __forceinline__ void jacobiRotate(m3<T>& A, m3<T>& V) {
  constexpr int R = 3 - P0 - P1;
  const T apq = A.m[P0][P1];
  const T app = A.m[P0][P0], aqq = A.m[P1][P1];
  const T tau = (aqq - app) / (T(2) * apq);
  const T t = gsign(tau) / (fabs(tau) + dsqrt<T>(T(1) + tau * tau));
  const T c = rcpsqrt<T>(T(1) + t * t);
  const T s = t * c;
  A.m[P0][P0] = app - t * apq;
  A.m[P1][P1] = aqq + t * apq;
  A.m[P0][P1] = T(0);
  A.m[P1][P0] = T(0);
  const T arp = A.m[R][P0], arq = A.m[R][P1];
  A.m[R][P0] = c * arp - s * arq;
  A.m[P0][R] = A.m[R][P0];
  A.m[R][P1] = s * arp + c * arq;
  A.m[P1][R] = A.m[R][P1];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const T vrp = V.m[q][P0], vrq = V.m[q][P1];
    V.m[q][P0] = c * vrp - s * vrq;
    V.m[q][P1] = s * vrp + c * vrq;
  }
}

// jacobiEigen3 (mpm_common.glsl:213-247): cyclic-max Jacobi, <= 20 rotations,
// stop when every off-diagonal of A is below 1e-8.
template <class T> __device__ __forceinline__ void jacobiEigen3(m3<T> A, T D[3], m3<T>& V) {
  V = m3ident<T>();
#pragma unroll 1
  for (int iter = 0; iter < 20; iter++) {
    const T b01 = fabs(A.m[0][1]), b02 = fabs(A.m[0][2]), b12 = fabs(A.m[1][2]);
    if (fmax(b01, fmax(b02, b12)) < T(1e-8)) break;
    if (b01 >= fmax(b02, b12)) jacobiRotate<T, 0, 1>(A, V);
    else if (b02 >= b12) jacobiRotate<T, 0, 2>(A, V);
    else jacobiRotate<T, 1, 2>(A, V);
  }
  D[0] = A.m[0][0];
  D[1] = A.m[1][1];
  D[2] = A.m[2][2];
}

// svd3 (mpm_common.glsl:250-281) on F^T F; sigma sorted descending.
template <class T> __device__ __forceinline__ void svd3(const m3<T>& F, m3<T>& U, T sigma[3], m3<T>& V) {
  m3<T> FtF;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) FtF.m[j][i] = F.m[i][0] * F.m[j][0] + F.m[i][1] * F.m[j][1] + F.m[i][2] * F.m[j][2];
  T sig2[3];
  jacobiEigen3(FtF, sig2, V);
#pragma unroll
  for (int i = 0; i < 3; ++i) sigma[i] = dsqrt<T>(fmax(sig2[i], T(0)));
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = i + 1; j < 3; j++) {
      if (sigma[j] > sigma[i]) {
        T tmp = sigma[i]; sigma[i] = sigma[j]; sigma[j] = tmp;
#pragma unroll
        for (int k = 0; k < 3; ++k) { T v = V.m[k][i]; V.m[k][i] = V.m[k][j]; V.m[k][j] = v; }
      }
    }
  U = m3zero<T>();
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (sigma[i] > T(1e-8)) {
      T v0 = V.m[0][i], v1 = V.m[1][i], v2 = V.m[2][i];
      const T inv = T(1) / sigma[i];
#pragma unroll
      for (int k = 0; k < 3; ++k) U.m[k][i] = (F.m[0][k] * v0 + F.m[1][k] * v1 + F.m[2][k] * v2) * inv;
    } else {
      U.m[i][i] = T(1);
    }
  }
  if (m3det(U) < T(0)) {
    U.m[0][2] = -U.m[0][2];
    U.m[1][2] = -U.m[1][2];
    U.m[2][2] = -U.m[2][2];
    sigma[2] = -sigma[2];
  }
}

// ---- float64 decomposition of the return maps.
// One Jacobi rotation zeroing A[P0][P1] with the update of
// mpm_common.glsl:224-244 (A[p][p] -= t apq, A[q][q] += t apq, A[p][q] = 0,
// the third row and column rotated, V rotated), in float64.  The tangent t is
// the small root of apq t^2 + (aqq - app) t - apq = 0, i.e. the shader's
// sign(tau) / (|tau| + sqrt(1 + tau^2)) with tau = (aqq - app) / (2 apq): it
// is first evaluated in float and then refined by one Newton step in double
// whose reciprocal derivative is taken in float, so t carries ~1e-14 relative
// error without a float64 division or square root.  tau's sign is taken from
// the double operands; sign(0) = 0 gives t = 0, for which the shader's update
// only zeroes A[p][q] (equal diagonals).
template <int P0, int P1>
__device__ __forceinline__ void jacobiRotateF64(m3<double>& A, m3<double>& V) {
  constexpr int R = 3 - P0 - P1;
  const double apq = A.m[P0][P1], app = A.m[P0][P0], aqq = A.m[P1][P1];
  const double d = aqq - app;
  if (d == 0.0) {
    A.m[P0][P1] = 0.0;
    A.m[P1][P0] = 0.0;
    return;
  }
  const float sg = (d > 0.0) == (apq > 0.0) ? 1.0f : -1.0f;
  const float tau = float(d) / (2.0f * float(apq));
  const float at = fabsf(tau);
  const float t0 = at < 1e18f ? sg / (at + sqrtf(1.0f + tau * tau)) : 0.5f / tau;
  const double tf = double(t0);
  const double f = apq * (tf * tf - 1.0) + d * tf;
  const double fp = 2.0 * apq * tf + d;
  const double t = tf - f * double(__frcp_rn(float(fp)));
  const double c = rsqrt(1.0 + t * t);
  const double sn = t * c;
  A.m[P0][P0] = app - t * apq;
  A.m[P1][P1] = aqq + t * apq;
  A.m[P0][P1] = 0.0;
  A.m[P1][P0] = 0.0;
  const double arp = A.m[R][P0], arq = A.m[R][P1];
  A.m[R][P0] = c * arp - sn * arq;
  A.m[P0][R] = A.m[R][P0];
  A.m[R][P1] = sn * arp + c * arq;
  A.m[P1][R] = A.m[R][P1];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double vrp = V.m[q][P0], vrq = V.m[q][P1];
    V.m[q][P0] = c * vrp - sn * vrq;
    V.m[q][P1] = sn * vrp + c * vrq;
  }
}

// svd3 of the return maps: same eigen-decomposition of F^T F (<= 20 rotations,
// stop below 1e-8), descending sort, U columns F v_i / sigma_i and the sign
// fix-up; sigma_i and 1/sigma_i come from one rsqrt of the eigenvalue.
__device__ __forceinline__ void svd3F64(const m3<double>& F, m3<double>& U, double sigma[3], m3<double>& V) {
  m3<double> A;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) A.m[j][i] = F.m[i][0] * F.m[j][0] + F.m[i][1] * F.m[j][1] + F.m[i][2] * F.m[j][2];
  V = m3ident<double>();
#pragma unroll 1
  for (int iter = 0; iter < 20; iter++) {
    const double b01 = fabs(A.m[0][1]), b02 = fabs(A.m[0][2]), b12 = fabs(A.m[1][2]);
    if (fmax(b01, fmax(b02, b12)) < 1e-8) break;
    if (b01 >= fmax(b02, b12)) jacobiRotateF64<0, 1>(A, V);
    else if (b02 >= b12) jacobiRotateF64<0, 2>(A, V);
    else jacobiRotateF64<1, 2>(A, V);
  }
  double inv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double l = fmax(A.m[i][i], 0.0);
    const double r = l > 0.0 ? rsqrt(l) : 0.0;
    sigma[i] = l * r;
    inv[i] = r;
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = i + 1; j < 3; j++) {
      if (sigma[j] > sigma[i]) {
        double tmp = sigma[i]; sigma[i] = sigma[j]; sigma[j] = tmp;
        tmp = inv[i]; inv[i] = inv[j]; inv[j] = tmp;
#pragma unroll
        for (int k = 0; k < 3; ++k) { double v = V.m[k][i]; V.m[k][i] = V.m[k][j]; V.m[k][j] = v; }
      }
    }
  U = m3zero<double>();
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (sigma[i] > 1e-8) {
      const double v0 = V.m[0][i], v1 = V.m[1][i], v2 = V.m[2][i];
#pragma unroll
      for (int k = 0; k < 3; ++k) U.m[k][i] = (F.m[0][k] * v0 + F.m[1][k] * v1 + F.m[2][k] * v2) * inv[i];
    } else {
      U.m[i][i] = 1.0;
    }
  }
  if (m3det(U) < 0.0) {
    U.m[0][2] = -U.m[0][2];
    U.m[1][2] = -U.m[1][2];
    U.m[2][2] = -U.m[2][2];
    sigma[2] = -sigma[2];
  }
}

// Hencky principal stresses from log-strains e_i = log(max(|sigma_i|, 1e-6)).
__device__ __forceinline__ void henckyFromLogStrain(const double e[3], double mu, double lam, double k[3]) {
  const double tr = e[0] + e[1] + e[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) k[i] = lam * tr + 2.0 * mu * e[i];
}

// Hencky principal Kirchhoff stresses k_i = lam*tr(eps) + 2 mu eps_i with
// eps = log(max(|sigma|, 1e-6)).
template <class T> __device__ __forceinline__ void henckyPrincipal(const T sigma[3], T mu, T lam, T k[3]) {
  T e[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) e[i] = dlog<T>(fmax(fabs(sigma[i]), T(1e-6)));
  T tr = e[0] + e[1] + e[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) k[i] = lam * tr + T(2) * mu * e[i];
}

// The shaders' `U * diag(k) * transpose(U)` with svd3's U layout:
//   tau[c][r] = sum_m k_m U[m][r] U[m][c]
template <class T> __device__ __forceinline__ m3<T> stressUDUt(const m3<T>& U, const T k[3]) {
  m3<T> t;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) t.m[c][r] = k[0] * U.m[0][r] * U.m[0][c] + k[1] * U.m[1][r] * U.m[1][c] + k[2] * U.m[2][r] * U.m[2][c];
  return t;
}

// The textbook stress sum_i k_i u_i u_i^T from svd3's row-stored vectors:
//   tau[c][r] = sum_i k_i U[r][i] U[c][i]
template <class T> __device__ __forceinline__ m3<T> stressTextbook(const m3<T>& U, const T k[3]) {
  m3<T> t;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) t.m[c][r] = k[0] * U.m[r][0] * U.m[c][0] + k[1] * U.m[r][1] * U.m[c][1] + k[2] * U.m[r][2] * U.m[c][2];
  return t;
}

// `U * diag(s) * transpose(V)` (GLSL): F[c][r] = sum_m s_m U[m][r] V[m][c]
template <class T> __device__ __forceinline__ m3<T> rebuildUSVt(const m3<T>& U, const T s[3], const m3<T>& V) {
  m3<T> F;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) F.m[c][r] = s[0] * U.m[0][r] * V.m[0][c] + s[1] * U.m[1][r] * V.m[1][c] + s[2] * U.m[2][r] * V.m[2][c];
  return F;
}

// henckyStress (mpm_common.glsl:284-293)
template <class T> __device__ __forceinline__ m3<T> henckyStress(const m3<T>& F, T mu, T lam) {
  m3<T> U, V;
  T s[3], k[3];
  svd3(F, U, s, V);
  henckyPrincipal(s, mu, lam, k);
  return stressUDUt(U, k);
}

// Fixed-corotated elasticity (Stomakhin et al. 2012), the model the
// reference's README names beside Hencky for ELASTIC (README.md:78) without
// implementing it; here model 6.  tau = 2 mu (F - R) F^T + lam (J - 1) J I
// with R = U V^T a rotation; for F = U S V^T with det U = det V = +1 (S
// signed) that is U diag(2 mu s_i (s_i - 1) + lam J (J - 1)) U^T, J = s0 s1 s2
// = det F.  svd3's sign fix makes det U = +1 but its eigenvector sort can
// leave det V = -1, with s2 of the wrong sign: flipping V's last column with
// s2 leaves U S V^T and U unchanged.  Same float svd3 as ELASTIC.  svd3 keeps
// the singular vectors in the rows of its matrices (the reference's layout,
// which its own models multiply as columns); this model is not the
// reference's, so its stress is the textbook sum of k_i u_i u_i^T:
// tau[c][r] = sum_i k_i U[r][i] U[c][i] (stressTextbook).
template <class T> __device__ __forceinline__ m3<T> fixedCorotatedStress(const m3<T>& F, T mu, T lam) {
  m3<T> U, V;
  T s[3], k[3];
  svd3(F, U, s, V);
  if (s[0] * s[1] * s[2] * m3det(F) < T(0)) s[2] = -s[2];
  const T J = s[0] * s[1] * s[2];
  const T c = lam * J * (J - T(1));
#pragma unroll
  for (int i = 0; i < 3; ++i) k[i] = T(2) * mu * s[i] * (s[i] - T(1)) + c;
  return stressTextbook(U, k);
}

// Plastic return maps + Kirchhoff stress, decompositions in float64.
// model VON_MISES: mpm_g2p.comp:19-38 then henckyStress; DRUCKER_PRAGER /
// POWDER / MUD: mpm_g2p.comp:41-68 then henckyStress, as mpm_g2p.comp:150-181
// calls them.  The return maps rebuild F as the shaders' `U * diag(s') *
// transpose(V)` from svd3's row-stored vectors, which is not F's own
// orientation, and the shaders then take the stress of the rebuilt matrix
// from a second svd3.  That stress, `U' * diag(k) * transpose(U')` in the
// same layout, depends on the signs the second decomposition gives its
// singular vectors (the layout turns them into signs of rows and columns of
// tau), so the second decomposition is run here too; its log-strains equal
// the returned ones (k_i from e_i below) up to rounding.  Without a rebuild
// (Von Mises inside the yield surface) the shader's second svd3 decomposes
// the unchanged F again, which is the first decomposition.

// Drucker-Prager (and POWDER / MUD) after the first decomposition.  The map
// from log-strains to returned log-strains is continuous (the apex branch and
// the deviatoric scaling meet where q_yield and delta reach zero), so the
// log-strains, the projection and the exponentials are float: a log-strain
// is formed as log1p of |sigma| - 1 taken in float64 (relative error of a
// few float ulps even for strains of 1e-4, where log of a float sigma near 1
// would lose three digits), and sigma' - 1 as expm1, so the rebuilt F in
// float64 carries the float rounding of F itself.
__device__ __forceinline__ float logStrain(double sigma) {
  const double a = fabs(sigma);
  if (a > 0.5 && a < 2.0) return log1pf(float(a - 1.0));
  return logf(float(fmax(a, 1e-6)));
}
__device__ __forceinline__ double expStrain(float e) { return fabsf(e) < 0.5f ? 1.0 + double(expm1f(e)) : double(expf(e)); }

__device__ __forceinline__ void druckerPragerFromSvd(m3<float>& F, m3<float>& tau, m3<double>& U, const double s[3], m3<double>& V, float mu,
                                                     float lam, float M, float qc) {
  constexpr float kThird = 1.0f / 3.0f;
  float eps[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eps[i] = logStrain(s[i]);
  const float trEps = eps[0] + eps[1] + eps[2];
  const float mean = trEps * kThird;
  float dev[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) dev[i] = eps[i] - mean;
  const float normDev = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const float K = lam + 2.0f * mu * kThird;
  const float q_yield = M * (-K * trEps) + qc;
  const bool apex = q_yield <= 1e-8f;
  if (apex) {
    const float tr = (qc / fmaxf(M, 1e-8f)) / K;  // -p_proj / K with p_proj = -qc / max(M, 1e-8)
#pragma unroll
    for (int i = 0; i < 3; ++i) eps[i] = tr * kThird;
  } else {
    const float delta = normDev - q_yield / (2.0f * mu);
    if (delta > 0.0f && normDev > 1e-8f) {
      const float r = delta / normDev;
#pragma unroll
      for (int i = 0; i < 3; ++i) eps[i] = (dev[i] - r * dev[i]) + mean;
    }
  }
  // the second decomposition's log-strains: log(max(exp(eps), 1e-6)) = max(eps, log 1e-6)
  double sp[3];
  float e[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    sp[i] = expStrain(eps[i]);
    e[i] = fmaxf(eps[i], -13.815510557964274f);
  }
  const float te = e[0] + e[1] + e[2];
  float k[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) k[i] = lam * te + 2.0f * mu * e[i];
  const m3<double> Fn = rebuildUSVt(U, sp, V);
  F = m3cast<float>(Fn);
  if (apex) {
    // three equal log-strains: the rebuilt F is a multiple of an orthogonal
    // matrix, whose decomposition finds orthonormal singular vectors in any
    // order and orientation, so its stress is k I (to the float64 rounding of
    // those vectors' orthonormality, below float precision): the second
    // decomposition is not needed
    tau = m3zero<float>();
    tau.m[0][0] = tau.m[1][1] = tau.m[2][2] = k[0];
    return;
  }
  double s2[3];
  svd3F64(Fn, U, s2, V);
  const double kd[3] = {double(k[0]), double(k[1]), double(k[2])};
  tau = m3cast<float>(stressUDUt(U, kd));
}

// Von Mises, all in float64 after the decomposition as well: a particle on
// the yield surface (where the last return left it) decides yield or not by
// the sign of ||dev eps|| - q_max / (2 mu), a difference at the rounding of F
// itself, and float logarithms there change the decision (and, through the
// rebuild, F's orientation) against the float64 oracle.
__device__ __forceinline__ void plasticReturn(uint32_t model, m3<float>& F, m3<float>& tau, float mu_f, float lam_f, float M_f, float qc_f,
                                              float qmax_f) {
  m3<double> U, V;
  double s[3];
  svd3F64(m3cast<double>(F), U, s, V);
  if (model != MAT_VON_MISES) {
    druckerPragerFromSvd(F, tau, U, s, V, mu_f, lam_f, M_f, qc_f);
    return;
  }
  const double mu = mu_f, lam = lam_f;
  // (divisions by constants and by 2 mu are multiplications by reciprocals:
  // within an ulp of float64 of the shaders' quotients)
  constexpr double kThird = 1.0 / 3.0;
  const double inv2mu = 1.0 / (2.0 * mu);
  double eps[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eps[i] = log(fmax(fabs(s[i]), 1e-6));
  const double trEps = eps[0] + eps[1] + eps[2];
  const double mean = trEps * kThird;
  double dev[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) dev[i] = eps[i] - mean;
  const double normDev = sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double delta = normDev - double(qmax_f) * inv2mu;
  double k[3];
  if (delta > 0.0 && normDev > 1e-8) {
    const double r = delta / normDev;
#pragma unroll
    for (int i = 0; i < 3; ++i) eps[i] = (dev[i] - r * dev[i]) + mean;
    double sp[3], e[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      sp[i] = exp(eps[i]);
      e[i] = fmax(eps[i], -13.815510557964274);  // log(max(exp(eps), 1e-6)) = max(eps, log 1e-6)
    }
    const m3<double> Fn = rebuildUSVt(U, sp, V);
    F = m3cast<float>(Fn);
    double s2[3];
    svd3F64(Fn, U, s2, V);
    henckyFromLogStrain(e, mu, lam, k);
  } else {
    henckyFromLogStrain(eps, mu, lam, k);  // eps = log(max(|s|, 1e-6)) already
  }
  tau = m3cast<float>(stressUDUt(U, k));
}

// ------------------------------------------------------------------ colliders
struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 mkf3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(f3 a) { return sqrtf(dot3(a, a)); }

__device__ __forceinline__ float colliderSDF(const Collider& c, f3 p, f3& n) {
  if (c.type == COLL_SPHERE) {
    f3 d = mkf3(p.x - c.px, p.y - c.py, p.z - c.pz);
    float dist = len3(d);
    n = dist > 1e-8f ? mkf3(d.x / dist, d.y / dist, d.z / dist) : mkf3(0.f, 1.f, 0.f);
    return dist - c.radius;
  }
  if (c.type == COLL_BOX) {
    f3 rel = mkf3(p.x - c.px, p.y - c.py, p.z - c.pz);
    f3 q = mkf3(fabsf(rel.x) - c.nx, fabsf(rel.y) - c.ny, fabsf(rel.z) - c.nz);
    f3 qp = mkf3(fmaxf(q.x, 0.f), fmaxf(q.y, 0.f), fmaxf(q.z, 0.f));
    float sdf = len3(qp) + fminf(fmaxf(q.x, fmaxf(q.y, q.z)), 0.f);
    if (sdf < 0.f) {
      f3 diff = mkf3(c.nx - fabsf(rel.x), c.ny - fabsf(rel.y), c.nz - fabsf(rel.z));
      if (diff.x < diff.y && diff.x < diff.z) n = mkf3(gsign(rel.x + 1e-8f), 0.f, 0.f);
      else if (diff.y < diff.z) n = mkf3(0.f, gsign(rel.y + 1e-8f), 0.f);
      else n = mkf3(0.f, 0.f, gsign(rel.z + 1e-8f));
    } else {
      float qLen = len3(qp);
      f3 sg = mkf3(gsign(rel.x + 1e-8f), gsign(rel.y + 1e-8f), gsign(rel.z + 1e-8f));
      f3 a = qLen > 1e-8f ? mkf3(qp.x * sg.x, qp.y * sg.y, qp.z * sg.z) : sg;
      float l = len3(a);
      n = mkf3(a.x / l, a.y / l, a.z / l);
    }
    return sdf;
  }
  if (c.type == COLL_CAPSULE) {
    f3 ax = mkf3(c.nx, c.ny, c.nz);
    float axisLen = len3(ax);
    f3 dir = axisLen > 1e-8f ? mkf3(ax.x / axisLen, ax.y / axisLen, ax.z / axisLen) : mkf3(0.f, 1.f, 0.f);
    float t = fminf(fmaxf(dot3(mkf3(p.x - c.px, p.y - c.py, p.z - c.pz), dir), 0.f), axisLen);
    f3 d = mkf3(p.x - (c.px + t * dir.x), p.y - (c.py + t * dir.y), p.z - (c.pz + t * dir.z));
    float dist = len3(d);
    n = dist > 1e-8f ? mkf3(d.x / dist, d.y / dist, d.z / dist) : mkf3(0.f, 1.f, 0.f);
    return dist - c.radius;
  }
  // plane (default)
  f3 nn = mkf3(c.nx, c.ny, c.nz);
  float l = len3(nn);
  n = mkf3(nn.x / l, nn.y / l, nn.z / l);
  return dot3(mkf3(p.x - c.px, p.y - c.py, p.z - c.pz), n);
}

__device__ __forceinline__ void applyColliderBC(f3& v, f3 n, f3 vc, float restitution, float friction) {
  f3 vr = mkf3(v.x - vc.x, v.y - vc.y, v.z - vc.z);
  float vn = dot3(vr, n);
  if (vn < 0.f) {
    f3 vnv = mkf3(vn * n.x, vn * n.y, vn * n.z);
    f3 vt = mkf3(vr.x - vnv.x, vr.y - vnv.y, vr.z - vnv.z);
    float vtLen = len3(vt);
    if (vtLen > 1e-8f) {
      float s = fmaxf(0.f, 1.f - friction * fabsf(vn) / vtLen);
      vt = mkf3(s * vt.x, s * vt.y, s * vt.z);
    }
    v = mkf3(vc.x + vt.x - restitution * vnv.x, vc.y + vt.y - restitution * vnv.y, vc.z + vt.z - restitution * vnv.z);
  }
}

// ------------------------------------------------------------------ per-particle material
struct MatSample {
  float mu, lam, rho0, M, qc, qmax, bulkK, visc;
  uint32_t model;
};
__device__ __forceinline__ MatSample fetchMaterial(const SubstepParams& P, uint32_t id) {
  MatSample s;
  if (P.materialCount > 0u) {
    id = min(id, P.materialCount - 1u);
    const Material& m = P.materials[id];
    s.mu = m.mu; s.lam = m.lambda; s.rho0 = m.rho0; s.model = m.model;
    s.M = m.M_friction; s.qc = m.q_cohesion; s.qmax = m.q_max; s.bulkK = m.bulkK; s.visc = m.viscosity;
  } else {
    s.mu = P.mu_lame; s.lam = P.lambda_lame; s.rho0 = P.rho0; s.model = P.plasticModel;
    s.M = P.M_friction; s.qc = P.q_cohesion; s.qmax = P.q_max; s.bulkK = 0.f; s.visc = 0.f;
  }
  return s;
}
__device__ __forceinline__ float fetchRho0(const SubstepParams& P, uint32_t id) {
  if (P.materialCount > 0u) return P.materials[min(id, P.materialCount - 1u)].rho0;
  return P.rho0;
}

}  // namespace nebula
