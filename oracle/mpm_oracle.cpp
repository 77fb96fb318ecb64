// mpm_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the nebula MPMEngine substep, used as the parity checker
// for the CUDA path and as the timed CPU baseline.  Only tests/, bench.py's
// cpu_baseline leg and __graft_entry__.smoke() load it; the product never does.
//
// It follows the reference shaders pass by pass (paths relative to the nebula
// source tree):
//   cell id / Morton         shaders/mpm_common.glsl:161-195
//   B-spline weights          shaders/mpm_common.glsl:198-210
//   Jacobi eigen / svd3       shaders/mpm_common.glsl:213-281
//   Hencky / fluid stress     shaders/mpm_common.glsl:284-302
//   zero grid / zero cells    shaders/mpm_zero_grid.comp:12-19, zero_cells.comp:11-15
//   binning                   shaders/mpm_hash_count.comp:7-14, hash_scan_local.comp,
//                             hash_scan_global.comp, hash_add_base.comp,
//                             mpm_hash_sort.comp:7-15 (intended exclusive scan; the
//                             shaders' single-workgroup global scan is only correct
//                             for hashCells <= 262,144, and within-cell order is
//                             canonical: ascending particle index, as the CPU
//                             binning of tests/helpers/MPMHarness.cpp:132-178)
//   P2G (per-node gather)     shaders/mpm_p2g.comp:17-87
//   grid update + forces      shaders/mpm_grid_update.comp:17-102,
//                             src/core/Force.h:136-141 (gravity / wind: v += dir*s*dt)
//   analytic colliders        shaders/collider_common.glsl:22-85
//   dense SDF boundary        shaders/mpm_nanovdb_bc.comp:23-54
//   G2P + return maps         shaders/mpm_g2p.comp:19-272
//   substep loop              src/engine/MPMEngine.cpp:404-474
//
// GLSL matrices are column-major: M[c][r] is column c, row r.  M3 below stores
// exactly that indexing so every expression reads like the shader it restates
// (including svd3 writing singular vectors into U[.][i]/V[.][i], i.e. as rows of
// the GLSL matrix, which the Hencky and return-map products then consume).
//
// In "ref32" mode every pass reproduces, bit for bit, the reference's own shaders
// compiled for the CPU by oracle/build_ref.py (tests/test_ref_shaders.py; golden
// vectors from that build in tests/golden/ref_shader_fixtures.npz), with the one
// intended difference named above: the exclusive scan over any number of cells.
//
// Precision modes (template parameters R = state/arithmetic type, RP = type of
// the SVD + stress inside the VON_MISES / DRUCKER_PRAGER / MUD return maps):
//   0 "ref32"  R=float,  RP=float   -- the shaders' own precision
//   1 "mixed"  R=float,  RP=double  -- the CUDA path's precision policy
//   2 "fp64"   R=double, RP=double  -- error statements / finite differences
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- small types
template <class T> struct V3 {
  T v[3];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};
template <class T> inline V3<T> mk(T a, T b, T c) { return V3<T>{{a, b, c}}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return mk(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return mk(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return mk(s * a[0], s * a[1], s * a[2]); }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return mk(a[0] * s, a[1] * s, a[2] * s); }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return mk(a[0] / s, a[1] / s, a[2] / s); }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline T gsign(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0)); }
template <class T> inline V3<T> vsign(V3<T> a) { return mk(gsign(a[0]), gsign(a[1]), gsign(a[2])); }
template <class T> inline V3<T> vabs(V3<T> a) { return mk(std::abs(a[0]), std::abs(a[1]), std::abs(a[2])); }
template <class T> inline V3<T> vmax(V3<T> a, T s) { return mk(std::max(a[0], s), std::max(a[1], s), std::max(a[2], s)); }
template <class T> inline V3<T> normalize(V3<T> a) { return a / length(a); }
template <class T> inline V3<T> mulc(V3<T> a, V3<T> b) { return mk(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }

// GLSL mat3: m[c][r]
template <class T> struct M3 {
  T m[3][3];
  T* operator[](int c) { return m[c]; }
  const T* operator[](int c) const { return m[c]; }
};
template <class T> inline M3<T> mdiag(T a, T b, T c) {
  M3<T> r{};
  r.m[0][0] = a; r.m[1][1] = b; r.m[2][2] = c;
  return r;
}
template <class T> inline M3<T> mident() { return mdiag(T(1), T(1), T(1)); }
template <class T> inline M3<T> mzero() { return M3<T>{}; }
template <class T> inline M3<T> mmul(const M3<T>& A, const M3<T>& B) {
  M3<T> C{};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) C.m[j][i] = A.m[0][i] * B.m[j][0] + A.m[1][i] * B.m[j][1] + A.m[2][i] * B.m[j][2];
  return C;
}
template <class T> inline V3<T> mmulv(const M3<T>& A, V3<T> v) {
  V3<T> r;
  for (int i = 0; i < 3; ++i) r[i] = A.m[0][i] * v[0] + A.m[1][i] * v[1] + A.m[2][i] * v[2];
  return r;
}
template <class T> inline M3<T> mtrans(const M3<T>& A) {
  M3<T> r;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) r.m[c][k] = A.m[k][c];
  return r;
}
template <class T> inline M3<T> madd(const M3<T>& A, const M3<T>& B) {
  M3<T> r;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) r.m[c][k] = A.m[c][k] + B.m[c][k];
  return r;
}
template <class T> inline M3<T> mscale(T s, const M3<T>& A) {
  M3<T> r;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) r.m[c][k] = s * A.m[c][k];
  return r;
}
// outerProduct(a, b)[j] = a * b[j]
template <class T> inline M3<T> outer(V3<T> a, V3<T> b) {
  M3<T> r;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) r.m[j][i] = a[i] * b[j];
  return r;
}
template <class T> inline T mdet(const M3<T>& A) {
  const T* a = A.m[0]; const T* b = A.m[1]; const T* c = A.m[2];
  return a[0] * (b[1] * c[2] - c[1] * b[2]) - b[0] * (a[1] * c[2] - c[1] * a[2]) + c[0] * (a[1] * b[2] - b[1] * a[2]);
}
template <class A, class B> inline M3<A> mcast(const M3<B>& s) {
  M3<A> r;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) r.m[c][k] = A(s.m[c][k]);
  return r;
}

// ---------------------------------------------------------------- records
// MaterialParams (src/core/MaterialParams.h:16-38), 64 bytes
struct Material {
  float mu, lambda, rho0;
  uint32_t model;
  float M_friction, q_cohesion, q_max, bulkK, fluidGamma, viscosity, hardening, xi, pad[4];
};
static_assert(sizeof(Material) == 64, "material record");
// ColliderPrimitive (src/core/Collider.h:19-29), 64 bytes
struct Collider {
  uint32_t type;
  float px, py, pz, nx, ny, nz, radius, vx, vy, vz, restitution, friction, pad[3];
};
static_assert(sizeof(Collider) == 64, "collider record");
// ForceGPU (src/core/Force.h:27-32), 32 bytes
struct Force {
  uint16_t type, affectMask;
  float data[7];
};
static_assert(sizeof(Force) == 32, "force record");

enum { MAT_ELASTIC = 0, MAT_VON_MISES = 1, MAT_DRUCKER_PRAGER = 2, MAT_GRANULAR_POWDER = 3, MAT_FLUID = 4, MAT_VISCOPLASTIC_MUD = 5,
       MAT_FIXED_COROTATED = 6 };
enum { COLL_PLANE = 0, COLL_SPHERE = 1, COLL_BOX = 2, COLL_CAPSULE = 3 };

}  // namespace

// Scalar parameters of one substep: the fields of MPMSimPC (src/core/MPMSimPC.h:14-77)
// that an MPM shader reads.
struct orc_params {
  float dt;
  float cellSize;
  uint32_t gridRes[3];
  uint32_t hashCells;
  float worldMin[3];
  float worldMax[3];
  float flip_ratio;
  uint32_t materialCount;
  float mu_lame, lambda_lame, rho0, M_friction, q_cohesion, q_max;
  uint32_t plasticModel;
  uint32_t colliderCount;
  uint32_t forceCount;
};

namespace {

// ---------------------------------------------------------------- Morton
inline uint32_t mortonExpand(uint32_t v) {
  v = (v | (v << 16u)) & 0x030000FFu;
  v = (v | (v << 8u)) & 0x0300F00Fu;
  v = (v | (v << 4u)) & 0x030C30C3u;
  v = (v | (v << 2u)) & 0x09249249u;
  return v;
}
inline uint32_t mortonCompact(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2u)) & 0x030C30C3u;
  v = (v | (v >> 4u)) & 0x0300F00Fu;
  v = (v | (v >> 8u)) & 0x030000FFu;
  v = (v | (v >> 16u)) & 0x000003FFu;
  return v;
}
inline uint32_t mortonEncodeI(int x, int y, int z) {
  return mortonExpand(uint32_t(x)) | (mortonExpand(uint32_t(y)) << 1u) | (mortonExpand(uint32_t(z)) << 2u);
}
inline void mortonDecodeI(uint32_t code, int& x, int& y, int& z) {
  x = int(mortonCompact(code));
  y = int(mortonCompact(code >> 1u));
  z = int(mortonCompact(code >> 2u));
}

// ---------------------------------------------------------------- B-spline
template <class T> inline T bspline2(T d) {
  T ad = std::abs(d);
  if (ad < T(0.5)) return T(0.75) - ad * ad;
  if (ad < T(1.5)) { T t = T(1.5) - ad; return T(0.5) * t * t; }
  return T(0);
}
template <class T> inline T bspline2g(T d) {
  T ad = std::abs(d);
  if (ad < T(0.5)) return T(-2) * d;
  if (ad < T(1.5)) return -gsign(d) * (T(1.5) - ad);
  return T(0);
}

// ---------------------------------------------------------------- SVD (mpm_common.glsl:213-281)
template <class T> void jacobiEigen3(M3<T> A, V3<T>& D, M3<T>& V) {
  V = mident<T>();
  for (int iter = 0; iter < 20; iter++) {
    T a01 = A[0][1], a02 = A[0][2], a12 = A[1][2];
    if (std::max(std::abs(a01), std::max(std::abs(a02), std::abs(a12))) < T(1e-8)) break;
    int p0, p1;
    T apq;
    if (std::abs(a01) >= std::max(std::abs(a02), std::abs(a12))) { p0 = 0; p1 = 1; apq = a01; }
    else if (std::abs(a02) >= std::abs(a12)) { p0 = 0; p1 = 2; apq = a02; }
    else { p0 = 1; p1 = 2; apq = a12; }
    T app = A[p0][p0], aqq = A[p1][p1];
    T tau = (aqq - app) / (T(2) * apq);
    T t = gsign(tau) / (std::abs(tau) + std::sqrt(T(1) + tau * tau));
    T c = T(1) / std::sqrt(T(1) + t * t);
    T s = t * c;
    A[p0][p0] = app - t * apq;
    A[p1][p1] = aqq + t * apq;
    A[p0][p1] = T(0); A[p1][p0] = T(0);
    for (int r = 0; r < 3; r++) {
      if (r == p0 || r == p1) continue;
      T arp = A[r][p0], arq = A[r][p1];
      A[r][p0] = c * arp - s * arq; A[p0][r] = A[r][p0];
      A[r][p1] = s * arp + c * arq; A[p1][r] = A[r][p1];
    }
    for (int r = 0; r < 3; r++) {
      T vrp = V[r][p0], vrq = V[r][p1];
      V[r][p0] = c * vrp - s * vrq;
      V[r][p1] = s * vrp + c * vrq;
    }
  }
  D = mk(A[0][0], A[1][1], A[2][2]);
}

template <class T> void svd3(const M3<T>& F, M3<T>& U, V3<T>& sigma, M3<T>& V) {
  M3<T> FtF = mmul(mtrans(F), F);
  V3<T> sig2;
  jacobiEigen3(FtF, sig2, V);
  sigma = mk(std::sqrt(std::max(sig2[0], T(0))), std::sqrt(std::max(sig2[1], T(0))), std::sqrt(std::max(sig2[2], T(0))));
  for (int i = 0; i < 2; i++)
    for (int j = i + 1; j < 3; j++) {
      if (sigma[j] > sigma[i]) {
        std::swap(sigma[i], sigma[j]);
        for (int k = 0; k < 3; ++k) std::swap(V[k][i], V[k][j]);
      }
    }
  U = mzero<T>();
  for (int i = 0; i < 3; i++) {
    V3<T> vi = mk(V[0][i], V[1][i], V[2][i]);
    if (sigma[i] > T(1e-8)) {
      V3<T> Fv = mmulv(F, vi);
      U[0][i] = Fv[0] / sigma[i];
      U[1][i] = Fv[1] / sigma[i];
      U[2][i] = Fv[2] / sigma[i];
    } else {
      U[i][i] = T(1);
    }
  }
  if (mdet(U) < T(0)) {
    U[0][2] = -U[0][2]; U[1][2] = -U[1][2]; U[2][2] = -U[2][2];
    sigma[2] = -sigma[2];
  }
}

template <class T> M3<T> henckyStress(const M3<T>& F, T mu, T lam) {
  M3<T> U, V;
  V3<T> sigma;
  svd3(F, U, sigma, V);
  sigma = vmax(vabs(sigma), T(1e-6));
  V3<T> eps = mk(std::log(sigma[0]), std::log(sigma[1]), std::log(sigma[2]));
  T trEps = eps[0] + eps[1] + eps[2];
  V3<T> kp = lam * trEps * mk(T(1), T(1), T(1)) + T(2) * mu * eps;
  M3<T> dg = mdiag(kp[0], kp[1], kp[2]);
  return mmul(mmul(U, dg), mtrans(U));
}

// Fixed-corotated elasticity (Stomakhin et al. 2012, "Energetically consistent
// invertible elasticity"): the model the reference's README names beside
// Hencky for ELASTIC (README.md:78; MaterialParams.h:6) but does not
// implement, added as its own model number 6.  Kirchhoff stress
//   tau = 2 mu (F - R) F^T + lam (J - 1) J I,  R = U V^T a rotation,
// and with F = U S V^T, det U = det V = +1 (S signed):
//   tau = U diag(2 mu s_i (s_i - 1) + lam J (J - 1)) U^T,  J = s0 s1 s2 = det F.
// svd3's sign fix makes det U = +1, but its sort of the eigenvectors can
// leave det V = -1; then s2 carries the wrong sign, and flipping V's last
// column with s2 (which leaves U S V^T and U unchanged) restores det V = +1.
// svd3 stores the singular vectors as the rows of its GLSL matrices (the
// reference's layout, kept for its own models); this model is not the
// reference's, so its stress is the textbook sum of k_i u_i u_i^T, which in
// that storage is transpose(U) * diag(k) * U.
template <class T> M3<T> fixedCorotatedStress(const M3<T>& F, T mu, T lam) {
  M3<T> U, V;
  V3<T> s;
  svd3(F, U, s, V);
  const T detF = mdet(F);
  if (s[0] * s[1] * s[2] * detF < T(0)) s[2] = -s[2];
  T J = s[0] * s[1] * s[2];
  T c = lam * J * (J - T(1));
  M3<T> dg = mdiag(T(2) * mu * s[0] * (s[0] - T(1)) + c, T(2) * mu * s[1] * (s[1] - T(1)) + c, T(2) * mu * s[2] * (s[2] - T(1)) + c);
  return mmul(mmul(mtrans(U), dg), U);
}

template <class T> M3<T> fluidStressJ(T J, T bulkK) { return mscale(bulkK * (J - T(1)), mident<T>()); }

// mpm_g2p.comp:19-38
template <class T> M3<T> projectVonMises(M3<T> F, T mu, T lam, T q_max) {
  (void)lam;
  M3<T> U, V;
  V3<T> sigma;
  svd3(F, U, sigma, V);
  sigma = vmax(vabs(sigma), T(1e-6));
  V3<T> eps = mk(std::log(sigma[0]), std::log(sigma[1]), std::log(sigma[2]));
  T trEps = eps[0] + eps[1] + eps[2];
  V3<T> devEps = eps - (trEps / T(3)) * mk(T(1), T(1), T(1));
  T normDev = length(devEps);
  T e_mu = T(2) * mu;
  T delta = normDev - q_max / e_mu;
  if (delta > T(0) && normDev > T(1e-8)) {
    devEps = devEps - (delta / normDev) * devEps;
    eps = devEps + (trEps / T(3)) * mk(T(1), T(1), T(1));
    sigma = mk(std::exp(eps[0]), std::exp(eps[1]), std::exp(eps[2]));
    F = mmul(mmul(U, mdiag(sigma[0], sigma[1], sigma[2])), mtrans(V));
  }
  return F;
}

// mpm_g2p.comp:41-68
template <class T> M3<T> projectDruckerPrager(M3<T> F, T mu, T lam, T M, T q_c) {
  M3<T> U, V;
  V3<T> sigma;
  svd3(F, U, sigma, V);
  sigma = vmax(vabs(sigma), T(1e-6));
  V3<T> eps = mk(std::log(sigma[0]), std::log(sigma[1]), std::log(sigma[2]));
  T trEps = eps[0] + eps[1] + eps[2];
  V3<T> devEps = eps - (trEps / T(3)) * mk(T(1), T(1), T(1));
  T normDev = length(devEps);
  T K = lam + T(2) * mu / T(3);
  T p = -K * trEps;
  T q_yield = M * p + q_c;
  if (q_yield <= T(1e-8)) {
    T p_proj = -q_c / std::max(M, T(1e-8));
    trEps = -p_proj / K;
    eps = (trEps / T(3)) * mk(T(1), T(1), T(1));
  } else {
    T delta = normDev - q_yield / (T(2) * mu);
    if (delta > T(0) && normDev > T(1e-8)) {
      devEps = devEps - (delta / normDev) * devEps;
      eps = devEps + (trEps / T(3)) * mk(T(1), T(1), T(1));
    }
  }
  sigma = mk(std::exp(eps[0]), std::exp(eps[1]), std::exp(eps[2]));
  return mmul(mmul(U, mdiag(sigma[0], sigma[1], sigma[2])), mtrans(V));
}

// ---------------------------------------------------------------- colliders (collider_common.glsl:22-85)
template <class T> T planeSDF(V3<T> p, V3<T> cpos, V3<T> cnrm, V3<T>& n) {
  n = normalize(cnrm);
  return dot(p - cpos, n);
}
template <class T> T sphereSDF(V3<T> p, V3<T> cpos, T cr, V3<T>& n) {
  V3<T> d = p - cpos;
  T dist = length(d);
  n = (dist > T(1e-8)) ? (d / dist) : mk(T(0), T(1), T(0));
  return dist - cr;
}
template <class T> T boxSDF(V3<T> p, V3<T> cpos, V3<T> halfExt, V3<T>& n) {
  V3<T> rel = p - cpos;
  V3<T> q = vabs(rel) - halfExt;
  V3<T> qp = vmax(q, T(0));
  T sdf = length(qp) + std::min(std::max(q[0], std::max(q[1], q[2])), T(0));
  if (sdf < T(0)) {
    V3<T> diff = halfExt - vabs(rel);
    if (diff[0] < diff[1] && diff[0] < diff[2]) n = mk(gsign(rel[0] + T(1e-8)), T(0), T(0));
    else if (diff[1] < diff[2]) n = mk(T(0), gsign(rel[1] + T(1e-8)), T(0));
    else n = mk(T(0), T(0), gsign(rel[2] + T(1e-8)));
  } else {
    T qLen = length(qp);
    V3<T> sgn = vsign(rel + mk(T(1e-8), T(1e-8), T(1e-8)));
    n = (qLen > T(1e-8)) ? normalize(mulc(qp, sgn)) : normalize(sgn);
  }
  return sdf;
}
template <class T> T capsuleSDF(V3<T> p, V3<T> cpos, V3<T> axisVec, T cr, V3<T>& n) {
  T axisLen = length(axisVec);
  V3<T> axisDir = (axisLen > T(1e-8)) ? (axisVec / axisLen) : mk(T(0), T(1), T(0));
  T t = std::min(std::max(dot(p - cpos, axisDir), T(0)), axisLen);
  V3<T> closest = cpos + t * axisDir;
  V3<T> d = p - closest;
  T dist = length(d);
  n = (dist > T(1e-8)) ? (d / dist) : mk(T(0), T(1), T(0));
  return dist - cr;
}
template <class T> void applyColliderBC(V3<T>& v, V3<T> n, V3<T> v_coll, T restitution, T friction) {
  V3<T> v_rel = v - v_coll;
  T v_n = dot(v_rel, n);
  if (v_n < T(0)) {
    V3<T> v_n_vec = v_n * n;
    V3<T> v_t = v_rel - v_n_vec;
    T vtLen = length(v_t);
    if (vtLen > T(1e-8)) v_t = std::max(T(0), T(1) - friction * std::abs(v_n) / vtLen) * v_t;
    v = v_coll + v_t - restitution * v_n_vec;
  }
}

// ---------------------------------------------------------------- engine
struct SimBase {
  virtual ~SimBase() = default;
  virtual void setParams(const orc_params& p) = 0;
  virtual void setTables(const void* mats, uint32_t nm, const void* cols, uint32_t nc, const void* forces, uint32_t nf) = 0;
  virtual void setSdf(const float* sdf) = 0;
  virtual void setState(const float* const* f4, uint32_t n) = 0;
  virtual void getState(double* const* f4) const = 0;
  virtual void getMatIds(uint32_t* ids) const = 0;
  virtual void setGrid(const float* mom, const float* mass) = 0;
  virtual void getGrid(double* mom, double* mass) const = 0;
  virtual void setBins(const uint32_t* cnt, const uint32_t* off, const uint32_t* sorted) = 0;
  virtual void getBins(uint32_t* cnt, uint32_t* off, uint32_t* sorted) const = 0;
  virtual void zeroGrid() = 0;
  virtual void bin() = 0;
  virtual void p2g() = 0;
  virtual void gridUpdate() = 0;
  virtual void sdfBC() = 0;
  virtual void g2p() = 0;
  virtual void substep() = 0;
};

template <class R, class RP> struct Sim final : SimBase {
  orc_params pc{};
  std::vector<Material> mats;
  std::vector<Collider> cols;
  std::vector<Force> forces;
  std::vector<float> sdf;
  bool hasSdf = false;
  uint32_t N = 0;
  // particle state, reference layout: 8 x vec4 per particle; v.w keeps the
  // material id bits in `mat`
  std::vector<R> P, Vv, F0, F1, F2, B0, B1, B2;
  std::vector<uint32_t> mat;
  std::vector<R> gridMom;  // 4 x 2*NC
  std::vector<R> gridMass; // NC
  std::vector<uint32_t> cellCount, cellOffset, sorted;

  void setParams(const orc_params& p) override {
    uint32_t oldNC = pc.hashCells;
    pc = p;
    if (pc.hashCells != oldNC || gridMass.size() != pc.hashCells) {
      gridMom.assign(size_t(pc.hashCells) * 8, R(0));
      gridMass.assign(pc.hashCells, R(0));
      cellCount.assign(pc.hashCells, 0);
      cellOffset.assign(pc.hashCells, 0);
    }
  }
  void setTables(const void* m, uint32_t nm, const void* c, uint32_t nc, const void* f, uint32_t nf) override {
    mats.assign(nm, Material{});
    if (nm) std::memcpy(mats.data(), m, nm * sizeof(Material));
    cols.assign(nc, Collider{});
    if (nc) std::memcpy(cols.data(), c, nc * sizeof(Collider));
    forces.assign(nf, Force{});
    if (nf) std::memcpy(forces.data(), f, nf * sizeof(Force));
  }
  void setSdf(const float* s) override {
    hasSdf = s != nullptr;
    if (hasSdf) sdf.assign(s, s + pc.hashCells);
    else sdf.clear();
  }
  void setState(const float* const* f4, uint32_t n) override {
    N = n;
    std::vector<R>* fl[8] = {&P, &Vv, &F0, &F1, &F2, &B0, &B1, &B2};
    for (int k = 0; k < 8; ++k) {
      fl[k]->resize(size_t(n) * 4);
      for (size_t i = 0; i < size_t(n) * 4; ++i) (*fl[k])[i] = R(f4[k][i]);
    }
    mat.resize(n);
    for (uint32_t i = 0; i < n; ++i) std::memcpy(&mat[i], &f4[1][size_t(i) * 4 + 3], 4);
    for (uint32_t i = 0; i < n; ++i) Vv[size_t(i) * 4 + 3] = R(0);
    sorted.assign(n, 0);
  }
  void getState(double* const* f4) const override {
    const std::vector<R>* fl[8] = {&P, &Vv, &F0, &F1, &F2, &B0, &B1, &B2};
    for (int k = 0; k < 8; ++k)
      for (size_t i = 0; i < size_t(N) * 4; ++i) f4[k][i] = double((*fl[k])[i]);
  }
  void getMatIds(uint32_t* ids) const override { std::memcpy(ids, mat.data(), N * sizeof(uint32_t)); }
  void setGrid(const float* mom, const float* mass) override {
    for (size_t i = 0; i < gridMom.size(); ++i) gridMom[i] = R(mom[i]);
    for (size_t i = 0; i < gridMass.size(); ++i) gridMass[i] = R(mass[i]);
  }
  void getGrid(double* mom, double* mass) const override {
    for (size_t i = 0; i < gridMom.size(); ++i) mom[i] = double(gridMom[i]);
    for (size_t i = 0; i < gridMass.size(); ++i) mass[i] = double(gridMass[i]);
  }
  void setBins(const uint32_t* cnt, const uint32_t* off, const uint32_t* s) override {
    std::memcpy(cellCount.data(), cnt, pc.hashCells * 4);
    std::memcpy(cellOffset.data(), off, pc.hashCells * 4);
    std::memcpy(sorted.data(), s, N * 4);
  }
  void getBins(uint32_t* cnt, uint32_t* off, uint32_t* s) const override {
    std::memcpy(cnt, cellCount.data(), pc.hashCells * 4);
    std::memcpy(off, cellOffset.data(), pc.hashCells * 4);
    std::memcpy(s, sorted.data(), N * 4);
  }

  V3<R> wmin() const { return mk(R(pc.worldMin[0]), R(pc.worldMin[1]), R(pc.worldMin[2])); }
  V3<R> wmax() const { return mk(R(pc.worldMax[0]), R(pc.worldMax[1]), R(pc.worldMax[2])); }
  V3<R> pos(uint32_t p) const { return mk(P[4 * size_t(p)], P[4 * size_t(p) + 1], P[4 * size_t(p) + 2]); }

  // cellIdFromPos (mpm_common.glsl:190-195)
  uint32_t cellId(V3<R> p) const {
    const R h = R(pc.cellSize);
    V3<R> w0 = wmin();
    uint32_t g[3];
    for (int a = 0; a < 3; ++a) {
      R l = (p[a] - w0[a]) / h;
      l = std::min(std::max(l, R(0)), R(pc.gridRes[a]) - R(1));
      g[a] = uint32_t(l);
    }
    return mortonExpand(g[0]) | (mortonExpand(g[1]) << 1u) | (mortonExpand(g[2]) << 2u);
  }

  void zeroGrid() override {
    std::fill(gridMom.begin(), gridMom.end(), R(0));
    std::fill(gridMass.begin(), gridMass.end(), R(0));
  }

  // zero_cells + mpm_hash_count + exclusive scan + mpm_hash_sort.  After the
  // sort cellOffset[c] holds the END of cell c's range, as the shaders leave it.
  void bin() override {
    const uint32_t NC = pc.hashCells;
    std::fill(cellCount.begin(), cellCount.end(), 0u);
    std::vector<uint32_t> key(N);
    for (uint32_t i = 0; i < N; ++i) {
      key[i] = cellId(pos(i));
      cellCount[key[i]]++;
    }
    uint32_t acc = 0;
    for (uint32_t c = 0; c < NC; ++c) {
      cellOffset[c] = acc;
      acc += cellCount[c];
    }
    for (uint32_t i = 0; i < N; ++i) sorted[cellOffset[key[i]]++] = i;
  }

  void material(uint32_t id, R& mu, R& lam, R& rho0, uint32_t& model, R& M, R& qc, R& qmax, R& bulkK, R& visc) const {
    if (pc.materialCount > 0u) {
      id = std::min(id, pc.materialCount - 1u);
      const Material& m = mats[id];
      mu = R(m.mu); lam = R(m.lambda); rho0 = R(m.rho0); model = m.model;
      M = R(m.M_friction); qc = R(m.q_cohesion); qmax = R(m.q_max); bulkK = R(m.bulkK); visc = R(m.viscosity);
    } else {
      mu = R(pc.mu_lame); lam = R(pc.lambda_lame); rho0 = R(pc.rho0); model = pc.plasticModel;
      M = R(pc.M_friction); qc = R(pc.q_cohesion); qmax = R(pc.q_max); bulkK = R(0); visc = R(0);
    }
  }

  M3<R> readMat3(const std::vector<R>& c0, const std::vector<R>& c1, const std::vector<R>& c2, uint32_t p) const {
    M3<R> m;
    for (int k = 0; k < 3; ++k) {
      m.m[0][k] = c0[4 * size_t(p) + k];
      m.m[1][k] = c1[4 * size_t(p) + k];
      m.m[2][k] = c2[4 * size_t(p) + k];
    }
    return m;
  }
  // readStressW (mpm_common.glsl:104-113)
  M3<R> readStressW(uint32_t p) const {
    size_t w = 4 * size_t(p) + 3;
    M3<R> t;
    t.m[0][0] = F0[w]; t.m[0][1] = B0[w]; t.m[0][2] = B1[w];
    t.m[1][0] = B0[w]; t.m[1][1] = F1[w]; t.m[1][2] = B2[w];
    t.m[2][0] = B1[w]; t.m[2][1] = B2[w]; t.m[2][2] = F2[w];
    return t;
  }

  // mpm_p2g.comp:17-87 -- one node per iteration, gathering the particles of the
  // 27 neighbour cells in (dz, dy, dx) order and in sorted order inside a cell.
  void p2g() override {
    const int64_t NC = pc.hashCells;
    const R h = R(pc.cellSize);
    const R dt = R(pc.dt);
    const V3<R> w0 = wmin();
    const bool apic = pc.flip_ratio < -0.5f;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t gid = 0; gid < NC; ++gid) {
      int nx, ny, nz;
      mortonDecodeI(uint32_t(gid), nx, ny, nz);
      V3<R> xi = (mk(R(nx), R(ny), R(nz)) + mk(R(0.5), R(0.5), R(0.5))) * h + w0;
      R totalMass = R(0);
      V3<R> totalMom = mk(R(0), R(0), R(0));
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            int cx = nx + dx, cy = ny + dy, cz = nz + dz;
            if (cx < 0 || cy < 0 || cz < 0 || cx >= int(pc.gridRes[0]) || cy >= int(pc.gridRes[1]) || cz >= int(pc.gridRes[2])) continue;
            uint32_t cid = mortonEncodeI(cx, cy, cz);
            uint32_t cnt = cellCount[cid];
            uint32_t start = cellOffset[cid] - cnt;
            for (uint32_t k = start; k < start + cnt; k++) {
              uint32_t p = sorted[k];
              V3<R> xp = pos(p);
              R Vp = P[4 * size_t(p) + 3];
              V3<R> vp = mk(Vv[4 * size_t(p)], Vv[4 * size_t(p) + 1], Vv[4 * size_t(p) + 2]);
              R mu, lam, rho0, M, qc, qmax, bulkK, visc;
              uint32_t model;
              material(mat[p], mu, lam, rho0, model, M, qc, qmax, bulkK, visc);
              R mp = rho0 * Vp;
              V3<R> d = (xp - xi) / h;
              R wx = bspline2(d[0]), wy = bspline2(d[1]), wz = bspline2(d[2]);
              R w = wx * wy * wz;
              if (w < R(1e-12)) continue;
              V3<R> dw = mk(bspline2g(d[0]) * wy * wz, wx * bspline2g(d[1]) * wz, wx * wy * bspline2g(d[2])) / h;
              M3<R> Bp = mzero<R>();
              if (apic) Bp = readMat3(B0, B1, B2, p);
              R D_inv = R(4) / (h * h);
              V3<R> v_eff = vp + D_inv * mmulv(Bp, xi - xp);
              M3<R> tau = readStressW(p);
              totalMass += w * mp;
              totalMom = totalMom + (w * mp) * v_eff;
              totalMom = totalMom - (dt * Vp) * mmulv(tau, dw);
            }
          }
      gridMom[4 * gid + 0] = totalMom[0];
      gridMom[4 * gid + 1] = totalMom[1];
      gridMom[4 * gid + 2] = totalMom[2];
      gridMom[4 * gid + 3] = R(0);
      gridMass[gid] = totalMass;
    }
  }

  // mpm_grid_update.comp:17-102
  void gridUpdate() override {
    const int64_t NC = pc.hashCells;
    const R h = R(pc.cellSize);
    const R dt = R(pc.dt);
    const V3<R> w0 = wmin();
#pragma omp parallel for schedule(static, 4096)
    for (int64_t gid = 0; gid < NC; ++gid) {
      R mass = gridMass[gid];
      if (mass < R(1e-10)) continue;
      V3<R> mom = mk(gridMom[4 * gid], gridMom[4 * gid + 1], gridMom[4 * gid + 2]);
      V3<R> v = mom / mass;
      {
        R vspeed = length(v);
        R vmax_grid = R(15);
        if (vspeed > vmax_grid) v = v * (vmax_grid / vspeed);
      }
      size_t o = 4 * size_t(gid + NC);
      gridMom[o] = v[0]; gridMom[o + 1] = v[1]; gridMom[o + 2] = v[2]; gridMom[o + 3] = R(0);
      int ix, iy, iz;
      mortonDecodeI(uint32_t(gid), ix, iy, iz);
      V3<R> forcePos = (mk(R(ix), R(iy), R(iz)) + mk(R(0.5), R(0.5), R(0.5))) * h + w0;
      for (uint32_t fi = 0; fi < pc.forceCount; ++fi) {
        const Force& f = forces[fi];
        uint32_t fmask = f.affectMask;
        if (fmask != 0u && ((fmask >> 0u) & 1u) == 0u) continue;
        if (f.type == 0u || f.type == 1u) {  // GRAVITY / CONSTANT_WIND
          V3<R> dir = mk(R(f.data[0]), R(f.data[1]), R(f.data[2]));
          v = v + (dir * R(f.data[3])) * dt;
        }
      }
      int Nx = int(pc.gridRes[0]) - 1, Ny = int(pc.gridRes[1]) - 1, Nz = int(pc.gridRes[2]) - 1;
      if (ix <= 1 && v[0] < R(0)) v[0] = R(0);
      if (ix >= Nx - 1 && v[0] > R(0)) v[0] = R(0);
      if (iy <= 1 && v[1] < R(0)) v[1] = R(0);
      if (iy >= Ny - 1 && v[1] > R(0)) v[1] = R(0);
      if (iz <= 1 && v[2] < R(0)) v[2] = R(0);
      if (iz >= Nz - 1 && v[2] > R(0)) v[2] = R(0);
      for (uint32_t ci = 0; ci < pc.colliderCount; ++ci) {
        const Collider& c = cols[ci];
        V3<R> cpos = mk(R(c.px), R(c.py), R(c.pz));
        V3<R> cnrm = mk(R(c.nx), R(c.ny), R(c.nz));
        V3<R> cvel = mk(R(c.vx), R(c.vy), R(c.vz));
        V3<R> col_n;
        R s;
        if (c.type == COLL_SPHERE) s = sphereSDF(forcePos, cpos, R(c.radius), col_n);
        else if (c.type == COLL_BOX) s = boxSDF(forcePos, cpos, cnrm, col_n);
        else if (c.type == COLL_CAPSULE) s = capsuleSDF(forcePos, cpos, cnrm, R(c.radius), col_n);
        else s = planeSDF(forcePos, cpos, cnrm, col_n);
        if (s <= R(0)) applyColliderBC(v, col_n, cvel, R(c.restitution), R(c.friction));
      }
      gridMom[4 * gid] = v[0]; gridMom[4 * gid + 1] = v[1]; gridMom[4 * gid + 2] = v[2]; gridMom[4 * gid + 3] = R(0);
    }
  }

  R sampleSdf(int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= int(pc.gridRes[0]) || y >= int(pc.gridRes[1]) || z >= int(pc.gridRes[2])) return R(1e6);
    return R(sdf[mortonEncodeI(x, y, z)]);
  }

  // mpm_nanovdb_bc.comp:23-54
  void sdfBC() override {
    if (!hasSdf) return;
    const int64_t NC = pc.hashCells;
    const R h = R(pc.cellSize);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t gid = 0; gid < NC; ++gid) {
      R mass = gridMass[gid];
      if (mass < R(1e-10)) continue;
      int x, y, z;
      mortonDecodeI(uint32_t(gid), x, y, z);
      R s = sampleSdf(x, y, z);
      if (s < R(0)) {
        for (int k = 0; k < 4; ++k) gridMom[4 * gid + k] = R(0);
      } else if (s < h * R(1.5)) {
        V3<R> v = mk(gridMom[4 * gid], gridMom[4 * gid + 1], gridMom[4 * gid + 2]);
        R sdx = sampleSdf(x + 1, y, z) - sampleSdf(x - 1, y, z);
        R sdy = sampleSdf(x, y + 1, z) - sampleSdf(x, y - 1, z);
        R sdz = sampleSdf(x, y, z + 1) - sampleSdf(x, y, z - 1);
        V3<R> gn = mk(sdx, sdy, sdz);
        R gl = length(gn);
        if (gl > R(1e-6)) {
          V3<R> n = gn / gl;
          R vn = dot(v, n);
          if (vn < R(0)) v = v - vn * n;
        }
        gridMom[4 * gid] = v[0]; gridMom[4 * gid + 1] = v[1]; gridMom[4 * gid + 2] = v[2]; gridMom[4 * gid + 3] = R(0);
      }
    }
  }

  R sdfAt(int x, int y, int z) const { return R(sdf[mortonEncodeI(x, y, z)]); }

  // mpm_g2p.comp:70-272
  void g2p() override {
    const R h = R(pc.cellSize);
    const R dt = R(pc.dt);
    const V3<R> w0 = wmin();
    const V3<R> w1 = wmax();
    const int64_t NC = pc.hashCells;
    const float flip = pc.flip_ratio;
#pragma omp parallel for schedule(static, 1024)
    for (int64_t pi = 0; pi < int64_t(N); ++pi) {
      const uint32_t p = uint32_t(pi);
      V3<R> xp = pos(p);
      int base[3];
      for (int a = 0; a < 3; ++a) base[a] = int(std::floor((xp[a] - w0[a]) / h)) - 1;
      V3<R> vpic = mk(R(0), R(0), R(0)), vpic_old = vpic;
      M3<R> vgrad = mzero<R>(), B_new = mzero<R>();
      for (int iz = 0; iz < 3; iz++)
        for (int iy = 0; iy < 3; iy++)
          for (int ix = 0; ix < 3; ix++) {
            int nx = base[0] + ix, ny = base[1] + iy, nz = base[2] + iz;
            if (nx < 0 || ny < 0 || nz < 0 || nx >= int(pc.gridRes[0]) || ny >= int(pc.gridRes[1]) || nz >= int(pc.gridRes[2])) continue;
            uint32_t nid = mortonEncodeI(nx, ny, nz);
            R mass = gridMass[nid];
            if (mass < R(1e-10)) continue;
            V3<R> xi = (mk(R(nx), R(ny), R(nz)) + mk(R(0.5), R(0.5), R(0.5))) * h + w0;
            V3<R> d = (xp - xi) / h;
            R wx = bspline2(d[0]), wy = bspline2(d[1]), wz = bspline2(d[2]);
            R w = wx * wy * wz;
            if (w < R(1e-12)) continue;
            V3<R> dw = mk(bspline2g(d[0]) * wy * wz, wx * bspline2g(d[1]) * wz, wx * wy * bspline2g(d[2])) / h;
            V3<R> vi = mk(gridMom[4 * size_t(nid)], gridMom[4 * size_t(nid) + 1], gridMom[4 * size_t(nid) + 2]);
            vpic = vpic + w * vi;
            vgrad = madd(vgrad, outer(vi, dw));
            B_new = madd(B_new, mscale(w, outer(vi, xi - xp)));
            if (flip > 0.01f) {
              size_t o = 4 * size_t(nid + NC);
              vpic_old = vpic_old + w * mk(gridMom[o], gridMom[o + 1], gridMom[o + 2]);
            }
          }
      V3<R> vold = mk(Vv[4 * size_t(p)], Vv[4 * size_t(p) + 1], Vv[4 * size_t(p) + 2]);
      R mu, lam, rho0, M, qc, qmax, bulkK, visc;
      uint32_t model;
      material(mat[p], mu, lam, rho0, model, M, qc, qmax, bulkK, visc);

      M3<R> F = readMat3(F0, F1, F2, p);
      M3<R> F_new = mmul(madd(mident<R>(), mscale(dt, vgrad)), F);
      M3<R> tau_new;
      if (model == MAT_FLUID) {
        R J = mdet(F_new);
        J = std::max(J, R(1e-4));
        F_new = mscale(R(std::pow(J, R(1) / R(3))), mident<R>());
        tau_new = fluidStressJ(J, bulkK);
      } else if (model == MAT_VON_MISES) {
        M3<RP> Fp = projectVonMises(mcast<RP>(F_new), RP(mu), RP(lam), RP(qmax));
        F_new = mcast<R>(Fp);
        tau_new = mcast<R>(henckyStress(Fp, RP(mu), RP(lam)));
      } else if (model == MAT_DRUCKER_PRAGER || model == MAT_GRANULAR_POWDER) {
        M3<RP> Fp = projectDruckerPrager(mcast<RP>(F_new), RP(mu), RP(lam), RP(M), RP(qc));
        F_new = mcast<R>(Fp);
        tau_new = mcast<R>(henckyStress(Fp, RP(mu), RP(lam)));
      } else if (model == MAT_VISCOPLASTIC_MUD) {
        M3<RP> Fp = projectDruckerPrager(mcast<RP>(F_new), RP(mu), RP(lam), RP(M), RP(qc));
        F_new = mcast<R>(Fp);
        tau_new = mcast<R>(henckyStress(Fp, RP(mu), RP(lam)));
        M3<R> D = mscale(R(0.5), madd(vgrad, mtrans(vgrad)));
        R trD = D[0][0] + D[1][1] + D[2][2];
        M3<R> devD = madd(D, mscale(-(trD / R(3)), mident<R>()));
        tau_new = madd(tau_new, mscale(R(2) * visc, devD));
      } else if (model == MAT_FIXED_COROTATED) {
        tau_new = fixedCorotatedStress(F_new, mu, lam);
      } else {
        tau_new = henckyStress(F_new, mu, lam);
      }
      bool j_reset = false;
      {
        R J_det = std::abs(mdet(F_new));
        if (J_det < R(0.15) || J_det > R(10)) {
          F_new = mident<R>();
          tau_new = mzero<R>();
          j_reset = true;
        }
      }
      if (flip > -0.5f) B_new = mzero<R>();
      V3<R> v_new;
      if (flip > 0.01f) {
        V3<R> v_flip = vold + (vpic - vpic_old);
        R fr = R(flip);
        v_new = vpic * (R(1) - fr) + v_flip * fr;
      } else {
        v_new = vpic;
      }
      if (j_reset) v_new = v_new * R(0.1);
      V3<R> x_new = xp + dt * v_new;

      if (hasSdf) {
        int gres[3] = {int(pc.gridRes[0]), int(pc.gridRes[1]), int(pc.gridRes[2])};
        int pijk[3];
        for (int a = 0; a < 3; ++a) pijk[a] = std::min(std::max(int(std::floor((x_new[a] - w0[a]) / h)), 0), gres[a] - 1);
        R psdf = sdfAt(pijk[0], pijk[1], pijk[2]);
        if (psdf < R(0)) {
          auto cl = [&](int a, int v) { return std::min(std::max(v, 0), gres[a] - 1); };
          V3<R> gn = mk(sdfAt(cl(0, pijk[0] + 1), pijk[1], pijk[2]) - sdfAt(cl(0, pijk[0] - 1), pijk[1], pijk[2]),
                        sdfAt(pijk[0], cl(1, pijk[1] + 1), pijk[2]) - sdfAt(pijk[0], cl(1, pijk[1] - 1), pijk[2]),
                        sdfAt(pijk[0], pijk[1], cl(2, pijk[2] + 1)) - sdfAt(pijk[0], pijk[1], cl(2, pijk[2] - 1)));
          R gl = length(gn);
          if (gl > R(1e-6)) {
            V3<R> n = gn / gl;
            x_new = x_new - psdf * n;
            R vn = dot(v_new, n);
            if (vn < R(0)) v_new = v_new - vn * n;
          } else {
            x_new = xp;
            v_new = mk(R(0), R(0), R(0));
          }
          F_new = mident<R>();
          tau_new = mzero<R>();
        }
      }
      R margin = h * R(1.5);
      V3<R> lo = w0 + mk(margin, margin, margin);
      V3<R> hi = w1 - mk(margin, margin, margin);
      for (int a = 0; a < 3; ++a) {
        if (x_new[a] < lo[a]) { x_new[a] = lo[a]; v_new[a] = std::max(v_new[a], R(0)); }
        if (x_new[a] > hi[a]) { x_new[a] = hi[a]; v_new[a] = std::min(v_new[a], R(0)); }
      }
      size_t b = 4 * size_t(p);
      P[b] = x_new[0]; P[b + 1] = x_new[1]; P[b + 2] = x_new[2];
      Vv[b] = v_new[0]; Vv[b + 1] = v_new[1]; Vv[b + 2] = v_new[2];
      for (int k = 0; k < 3; ++k) {
        F0[b + k] = F_new[0][k]; F1[b + k] = F_new[1][k]; F2[b + k] = F_new[2][k];
        B0[b + k] = B_new[0][k]; B1[b + k] = B_new[1][k]; B2[b + k] = B_new[2][k];
      }
      // writeStressW (mpm_common.glsl:116-122)
      F0[b + 3] = tau_new[0][0]; F1[b + 3] = tau_new[1][1]; F2[b + 3] = tau_new[2][2];
      B0[b + 3] = tau_new[0][1]; B1[b + 3] = tau_new[0][2]; B2[b + 3] = tau_new[1][2];
    }
  }

  // MPMEngine::step body for one substep (MPMEngine.cpp:419-472)
  void substep() override {
    zeroGrid();
    bin();
    p2g();
    gridUpdate();
    sdfBC();
    g2p();
  }
};

thread_local std::string g_err;

}  // namespace

extern "C" {

// mode: 0 ref32, 1 mixed, 2 fp64
void* orc_create(int mode) {
  switch (mode) {
    case 0: return new Sim<float, float>();
    case 1: return new Sim<float, double>();
    case 2: return new Sim<double, double>();
    default: return nullptr;
  }
}
void orc_destroy(void* h) { delete static_cast<SimBase*>(h); }
void orc_set_params(void* h, const orc_params* p) { static_cast<SimBase*>(h)->setParams(*p); }
void orc_set_tables(void* h, const void* mats, uint32_t nm, const void* cols, uint32_t nc, const void* forces, uint32_t nf) {
  static_cast<SimBase*>(h)->setTables(mats, nm, cols, nc, forces, nf);
}
void orc_set_sdf(void* h, const float* sdf) { static_cast<SimBase*>(h)->setSdf(sdf); }
// fields: P, v, F0, F1, F2, B0, B1, B2 as float4 x n each (v.w = material id bits)
void orc_set_state(void* h, const float* P, const float* v, const float* F0, const float* F1, const float* F2, const float* B0,
                   const float* B1, const float* B2, uint32_t n) {
  const float* f[8] = {P, v, F0, F1, F2, B0, B1, B2};
  static_cast<SimBase*>(h)->setState(f, n);
}
void orc_get_state(void* h, double* P, double* v, double* F0, double* F1, double* F2, double* B0, double* B1, double* B2) {
  double* f[8] = {P, v, F0, F1, F2, B0, B1, B2};
  static_cast<SimBase*>(h)->getState(f);
}
void orc_get_mat_ids(void* h, uint32_t* ids) { static_cast<SimBase*>(h)->getMatIds(ids); }
void orc_set_grid(void* h, const float* mom, const float* mass) { static_cast<SimBase*>(h)->setGrid(mom, mass); }
void orc_get_grid(void* h, double* mom, double* mass) { static_cast<SimBase*>(h)->getGrid(mom, mass); }
void orc_set_bins(void* h, const uint32_t* cnt, const uint32_t* off, const uint32_t* sorted) {
  static_cast<SimBase*>(h)->setBins(cnt, off, sorted);
}
void orc_get_bins(void* h, uint32_t* cnt, uint32_t* off, uint32_t* sorted) { static_cast<SimBase*>(h)->getBins(cnt, off, sorted); }
void orc_zero_grid(void* h) { static_cast<SimBase*>(h)->zeroGrid(); }
void orc_bin(void* h) { static_cast<SimBase*>(h)->bin(); }
void orc_p2g(void* h) { static_cast<SimBase*>(h)->p2g(); }
void orc_grid_update(void* h) { static_cast<SimBase*>(h)->gridUpdate(); }
void orc_sdf_bc(void* h) { static_cast<SimBase*>(h)->sdfBC(); }
void orc_g2p(void* h) { static_cast<SimBase*>(h)->g2p(); }
void orc_substep(void* h) { static_cast<SimBase*>(h)->substep(); }
void orc_run(void* h, uint32_t nsub) {
  for (uint32_t s = 0; s < nsub; ++s) static_cast<SimBase*>(h)->substep();
}
int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Small pure helpers exposed for the known-answer tests.
float orc_bspline2(float d) { return bspline2(d); }
float orc_bspline2g(float d) { return bspline2g(d); }
uint32_t orc_morton_encode(uint32_t x, uint32_t y, uint32_t z) { return mortonEncodeI(int(x), int(y), int(z)); }
void orc_morton_decode(uint32_t c, uint32_t* xyz) {
  int x, y, z;
  mortonDecodeI(c, x, y, z);
  xyz[0] = uint32_t(x); xyz[1] = uint32_t(y); xyz[2] = uint32_t(z);
}
// F, tau: 9 floats each in GLSL column-major order (m[c][r] at 3*c+r)
void orc_hencky(const float* F, float mu, float lam, float* tau, int fp64) {
  if (fp64) {
    M3<double> f;
    for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
    M3<double> t = henckyStress(f, double(mu), double(lam));
    for (int i = 0; i < 9; ++i) tau[i] = float(t.m[i / 3][i % 3]);
  } else {
    M3<float> f;
    for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
    M3<float> t = henckyStress(f, mu, lam);
    for (int i = 0; i < 9; ++i) tau[i] = t.m[i / 3][i % 3];
  }
}
void orc_fixed_corotated(const float* F, float mu, float lam, float* tau, int fp64) {
  if (fp64) {
    M3<double> f;
    for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
    M3<double> t = fixedCorotatedStress(f, double(mu), double(lam));
    for (int i = 0; i < 9; ++i) tau[i] = float(t.m[i / 3][i % 3]);
  } else {
    M3<float> f;
    for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
    M3<float> t = fixedCorotatedStress(f, mu, lam);
    for (int i = 0; i < 9; ++i) tau[i] = t.m[i / 3][i % 3];
  }
}
// svd3 outputs in GLSL layout: U, V as m[c][r] at 3*c+r
void orc_svd3(const double* F, double* U, double* sigma, double* V) {
  M3<double> f, u, v;
  V3<double> s;
  for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
  svd3(f, u, s, v);
  for (int i = 0; i < 9; ++i) { U[i] = u.m[i / 3][i % 3]; V[i] = v.m[i / 3][i % 3]; }
  for (int i = 0; i < 3; ++i) sigma[i] = s[i];
}
void orc_project(const double* F, int model, double mu, double lam, double M, double qc, double qmax, double* Fout) {
  M3<double> f;
  for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
  M3<double> r = model == MAT_VON_MISES ? projectVonMises(f, mu, lam, qmax) : projectDruckerPrager(f, mu, lam, M, qc);
  for (int i = 0; i < 9; ++i) Fout[i] = r.m[i / 3][i % 3];
}

}  // extern "C"
