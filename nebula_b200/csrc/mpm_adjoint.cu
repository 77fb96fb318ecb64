// mpm_adjoint.cu -- differentiable rollout: forward with checkpoints and the
// hand-written reverse pass of P2G, grid update and G2P (sm_100a).
//
// Matrices in the adjoint are mathematical (row, column).  The engine's
// state stores GLSL columns: F0..F2 / B0..B2 hold columns of F / B, so
// F[r][c] = F<c>.<r>; the Kirchhoff stress lives in the w lanes.
//
// Per substep (forward):  P2G   m_i = sum w m_p,  p_i = sum w m_p (v_p + D^-1 B_p r) - dt V_p tau_p grad w
//                         grid  v_i = walls(cap(p_i / m_i) + g dt)
//                         G2P   v_p' = sum w v_i,  B_p' = sum w v_i r^T,  G = sum v_i grad w^T,
//                               F' = (I + dt G) F,  tau' = hencky(F'),  x' = x + dt v_p'
// with r = x_i - x_p and D^-1 = 4/h^2.  The reverse pass applies the
// transposed Jacobians in the opposite order: G2P adjoint (a scatter to the
// grid), grid adjoint (per node), P2G adjoint (a gather from the grid).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>

#include "mpm_adjoint.h"
#include "mpm_particle.cuh"

namespace nebula {
namespace {

constexpr int kT = 256;
inline uint32_t blocks(uint64_t n) { return uint32_t((n + kT - 1) / kT); }

// Adjoint of the particle state; B, F, T are three float4 rows per particle.
struct AdjPtrs {
  float4* x;
  float4* v;
  float4* B;
  float4* F;
  float4* T;
};

AdjPtrs adjPtrs(DevBuf& b, uint32_t n) {
  float4* base = static_cast<float4*>(b.ptr);
  return AdjPtrs{base, base + n, base + 2 * size_t(n), base + 5 * size_t(n), base + 8 * size_t(n)};
}

struct St {
  float4* f[8];
};
St stPtrs(DevBuf& b, uint32_t n) {
  St s;
  for (int k = 0; k < 8; ++k) s.f[k] = static_cast<float4*>(b.ptr) + size_t(k) * n;
  return s;
}

// Second derivative of the quadratic B-spline.
__device__ __forceinline__ float bspline2h(float d) {
  const float a = fabsf(d);
  if (a < 0.5f) return -2.0f;
  if (a < 1.5f) return 1.0f;
  return 0.0f;
}

// Grid accessor for g2pParticle over the dense velocity grid (w = mass).
struct VelGrid {
  const float4* vel;
  __device__ __forceinline__ bool node(int x, int y, int z, float& m, float3& v, float3& vo) const {
    const float4 a = __ldg(vel + mortonEncode(x, y, z));
    m = a.w;
    if (m < 1e-10f) return false;
    v = make_float3(a.x, a.y, a.z);
    vo = v;
    return true;
  }
};

// Node box of one substep's P2G: every node a particle stencil touched lies in
// [lo, hi] (per axis, inclusive).  lo is stored complemented (~lo), so both
// halves grow with atomicMax from a zeroed record.
struct NodeBox {
  uint32_t loInv[3];
  uint32_t hi[3];
  uint32_t pad[2];
};
static_assert(sizeof(NodeBox) == 32, "NodeBox");

// Fold the stencil of every particle of the block into box `b` (one atomic
// per bound per CTA).
__device__ __forceinline__ void boxAdd(NodeBox* b, bool valid, int cx, int cy, int cz, int cube) {
  __shared__ uint32_t red[6][kT / 32];
  uint32_t v[6];
  v[0] = valid ? ~uint32_t(max(cx - 1, 0)) : 0u;
  v[1] = valid ? ~uint32_t(max(cy - 1, 0)) : 0u;
  v[2] = valid ? ~uint32_t(max(cz - 1, 0)) : 0u;
  v[3] = valid ? uint32_t(min(cx + 1, cube - 1)) : 0u;
  v[4] = valid ? uint32_t(min(cy + 1, cube - 1)) : 0u;
  v[5] = valid ? uint32_t(min(cz + 1, cube - 1)) : 0u;
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = max(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k][warp] = v[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    uint32_t m = 0;
    for (int w = 0; w < kT / 32; ++w) m = max(m, red[threadIdx.x][w]);
    if (m) atomicMax(threadIdx.x < 3 ? &b->loInv[threadIdx.x] : &b->hi[threadIdx.x - 3], m);
  }
}

// The cells of box `b` (an empty box when no particle folded in), visited
// with a grid-stride loop: fn(Morton code).
template <class Fn>
__device__ __forceinline__ void forBox(const NodeBox& b, Fn&& fn) {
  const int lo[3] = {int(~b.loInv[0]), int(~b.loInv[1]), int(~b.loInv[2])};
  const int n[3] = {int(b.hi[0]) - lo[0] + 1, int(b.hi[1]) - lo[1] + 1, int(b.hi[2]) - lo[2] + 1};
  if (b.loInv[0] == 0u || n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return;
  const uint32_t total = uint32_t(n[0]) * uint32_t(n[1]) * uint32_t(n[2]);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int x = lo[0] + int(i % uint32_t(n[0])), y = lo[1] + int((i / uint32_t(n[0])) % uint32_t(n[1])), z = lo[2] + int(i / (uint32_t(n[0]) * uint32_t(n[1])));
    fn(mortonEncode(x, y, z));
  }
}

// ------------------------------------------------------------------ forward
__global__ void __launch_bounds__(kT) k_init(const float4* __restrict__ x0, const float4* __restrict__ v0, const float* __restrict__ E, float nu,
                                             uint32_t n, St st, float2* lame) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  st.f[0][p] = x0[p];
  const float4 v = v0[p];
  st.f[1][p] = make_float4(v.x, v.y, v.z, 0.f);
  st.f[2][p] = make_float4(1.f, 0.f, 0.f, 0.f);
  st.f[3][p] = make_float4(0.f, 1.f, 0.f, 0.f);
  st.f[4][p] = make_float4(0.f, 0.f, 1.f, 0.f);
  st.f[5][p] = st.f[6][p] = st.f[7][p] = make_float4(0.f, 0.f, 0.f, 0.f);
  const float e = E[p];
  lame[p] = make_float2(e / (2.0f * (1.0f + nu)), e * nu / ((1.0f + nu) * (1.0f - 2.0f * nu)));
}

__global__ void __launch_bounds__(kT) k_fwd_p2g(SubstepParams P, St st, uint32_t n, float4* acc, NodeBox* box) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  int c[3] = {0, 0, 0};
  if (p < n) {
    const PState s = loadState(st.f, p);
    cellCoords(P, s.P.x, s.P.y, s.P.z, c[0], c[1], c[2]);
    p2gParticle(P, s, P.dt, [&](int nx, int ny, int nz, float mx, float my, float mz, float m) {
      redAddV4(acc + mortonEncode(nx, ny, nz), mx, my, mz, m);
    });
  }
  boxAdd(box, p < n, c[0], c[1], c[2], int(P.cubeRes));
}

// Grid update over the substep's node box (G2P reads no node outside it);
// `clear` zeroes acc behind the read for the next substep's P2G.
__global__ void __launch_bounds__(kT) k_fwd_grid(SubstepParams P, float4* acc, float4* vel, AdjScalars* sc, const NodeBox* box, int clear) {
  forBox(*box, [&](uint32_t c) {
    const float4 a = acc[c];
    if (clear) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    int ix, iy, iz;
    mortonDecode(c, ix, iy, iz);
    float3 v, vo;
    const bool ok = gridNode(P, ix, iy, iz, a.w, a.x, a.y, a.z, v, vo);
    vel[c] = ok ? make_float4(v.x, v.y, v.z, a.w) : make_float4(0.f, 0.f, 0.f, a.w);
    if (ok) {
      const float ux = a.x / a.w, uy = a.y / a.w, uz = a.z / a.w;
      if (sqrtf(ux * ux + uy * uy + uz * uz) > 15.0f) atomicOr(&sc->events, 4u);
    }
  });
}

__global__ void __launch_bounds__(kT) k_fwd_g2p(SubstepParams P, St in, St out, const float2* __restrict__ lame, uint32_t n,
                                                const float4* __restrict__ vel, AdjScalars* sc) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  PState s = loadState(in.f, p);
  SubstepParams Pp = P;  // the particle's own Lame parameters through the global-material path
  const float2 l = lame[p];
  Pp.mu_lame = l.x;
  Pp.lambda_lame = l.y;
  const uint32_t ev = g2pParticle(Pp, s, VelGrid{vel}, P.dt);
  const float lo = 1.5f * P.cellSize;
  uint32_t flags = (ev & 1u) ? 1u : 0u;
  const float xn[3] = {s.P.x, s.P.y, s.P.z};
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (xn[a] <= P.worldMin[a] + lo || xn[a] >= P.worldMax[a] - lo) flags |= 2u;
  if (flags) atomicOr(&sc->events, flags);
  storeState(out.f, p, s);
}

// sum m_p x_p and sum m_p, accumulated in double
__global__ void __launch_bounds__(kT) k_com(const float4* __restrict__ pos, const float4* __restrict__ x0, float rho0, uint32_t n, AdjScalars* sc) {
  __shared__ double red[4][kT / 32];
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  if (p < n) {
    const float4 x = pos[p];
    const double m = double(rho0 * x0[p].w);
    a[0] = m * x.x;
    a[1] = m * x.y;
    a[2] = m * x.z;
    a[3] = m;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) red[k][warp] = a[k];
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int w = 0; w < kT / 32; ++w) s += red[threadIdx.x][w];
    atomicAdd(&sc->com[threadIdx.x], s);
  }
}

__global__ void k_loss(AdjScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double L = 0;
  for (int a = 0; a < 3; ++a) {
    const double d = sc->com[a] / sc->com[3] - sc->target[a];
    L += d * d;
  }
  sc->loss = float(L);
}

// ------------------------------------------------------------------ adjoint of the Hencky stress (double)
// tau = sum_m k_m u_m u_m^T in svd3's layout (U[q][m] = U.m[q][m], the
// shaders' U * diag(k) * transpose(U)), k = lam tr(e) + 2 mu e, e = log|s|.
// Given tbar (symmetrised here) adds dL/dF to Fb and dL/dmu, dL/dlam.
// Singular-vector derivative: dU = U Omega with
//   Omega_ij = (s_j P_ij + s_i P_ji) / (s_j^2 - s_i^2),  P = U^T dF V,
// which turns the skew part A = tau tbar - tbar tau into off-diagonal terms.
__device__ __forceinline__ void henckyAdj(const double Fm[3][3], double mu, double lam, const double tbIn[3][3], double Fb[3][3], double& mub,
                                          double& lamb) {
  m3<double> F, Ug, Vg;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) F.m[c][r] = Fm[r][c];
  double s[3];
  svd3F64(F, Ug, s, Vg);
  double tb[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) tb[i][j] = 0.5 * (tbIn[i][j] + tbIn[j][i]);
  double e[3], k[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) e[m] = log(fmax(fabs(s[m]), 1e-6));
  const double tr = e[0] + e[1] + e[2];
#pragma unroll
  for (int m = 0; m < 3; ++m) k[m] = lam * tr + 2.0 * mu * e[m];
  double tau[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) tau[i][j] = k[0] * Ug.m[0][i] * Ug.m[0][j] + k[1] * Ug.m[1][i] * Ug.m[1][j] + k[2] * Ug.m[2][i] * Ug.m[2][j];
  double kb[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double acc = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc += Ug.m[m][i] * tb[i][j] * Ug.m[m][j];
    kb[m] = acc;
  }
  const double ksum = kb[0] + kb[1] + kb[2];
  mub += 2.0 * (kb[0] * e[0] + kb[1] * e[1] + kb[2] * e[2]);
  lamb += ksum * tr;
  double A[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double a = 0;
#pragma unroll
      for (int q = 0; q < 3; ++q) a += tau[i][q] * tb[q][j] - tb[i][q] * tau[q][j];
      A[i][j] = a;
    }
  double Pb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double eb = lam * ksum + 2.0 * mu * kb[m];
    Pb[m][m] = fabs(s[m]) > 1e-6 ? eb / s[m] : 0.0;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i + 1; j < 3; ++j) {
      const double den = s[j] * s[j] - s[i] * s[i];
      if (fabs(den) < 1e-14) continue;
      const double c = 2.0 * A[i][j] / den;
      Pb[i][j] += c * s[j];
      Pb[j][i] += c * s[i];
    }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double acc = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc += Ug.m[a][i] * Pb[i][j] * Vg.m[b][j];
      Fb[a][b] += acc;
    }
}

// ------------------------------------------------------------------ reverse kernels
// Per-axis stencil data of one particle: N, N', N'' and node centres.
struct Stencil {
  int base[3];
  float w[3][3], g[3][3], hh[3][3], xi[3][3];
};

__device__ __forceinline__ void stencilAt(const SubstepParams& P, const float xp[3], const int base[3], Stencil& S) {
  const float invH = 1.0f / P.cellSize;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    S.base[a] = base[a];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      S.xi[a][k] = nodeCentre(P, a, base[a] + k);
      const float d = (xp[a] - S.xi[a][k]) * invH;
      S.w[a][k] = bspline2(d);
      S.g[a][k] = bspline2g(d);
      S.hh[a][k] = bspline2h(d);
    }
  }
}

struct NodeTerms {
  float w, dw[3], H[3][3], r[3];
};

__device__ __forceinline__ void nodeTerms(const SubstepParams& P, const Stencil& S, const float xp[3], int ix, int iy, int iz, NodeTerms& t) {
  const float h = P.cellSize, invH = 1.0f / h, ih2 = 1.0f / (h * h);
  const float wx = S.w[0][ix], wy = S.w[1][iy], wz = S.w[2][iz];
  const float gx = S.g[0][ix], gy = S.g[1][iy], gz = S.g[2][iz];
  t.w = wx * wy * wz;
  t.dw[0] = gx * wy * wz * invH;
  t.dw[1] = wx * gy * wz * invH;
  t.dw[2] = wx * wy * gz * invH;
  t.H[0][0] = S.hh[0][ix] * wy * wz * ih2;
  t.H[1][1] = wx * S.hh[1][iy] * wz * ih2;
  t.H[2][2] = wx * wy * S.hh[2][iz] * ih2;
  t.H[0][1] = t.H[1][0] = gx * gy * wz * ih2;
  t.H[0][2] = t.H[2][0] = gx * wy * gz * ih2;
  t.H[1][2] = t.H[2][1] = wx * gy * gz * ih2;
  t.r[0] = S.xi[0][ix] - xp[0];
  t.r[1] = S.xi[1][iy] - xp[1];
  t.r[2] = S.xi[2][iz] - xp[2];
}

__device__ __forceinline__ void loadRows(const float4* rows, uint32_t p, float M[3][3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float4 a = rows[3 * size_t(p) + r];
    M[r][0] = a.x;
    M[r][1] = a.y;
    M[r][2] = a.z;
  }
}
__device__ __forceinline__ void storeRows(float4* rows, uint32_t p, const float M[3][3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) rows[3 * size_t(p) + r] = make_float4(M[r][0], M[r][1], M[r][2], 0.f);
}

// G2P adjoint: adjoints of (x', v', B', F', tau') -> adjoint of x (partial), F,
// mu, lambda, and the grid-velocity adjoint (scattered).
__global__ void __launch_bounds__(kT) k_adj_g2p(SubstepParams P, St st, const float2* __restrict__ lame, uint32_t n, const float4* __restrict__ vel,
                                                AdjPtrs ob, AdjPtrs ib, float4* gadj, float* mub, float* lamb) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float dt = P.dt, h = P.cellSize, invH = 1.0f / h;
  const float4 P4 = st.f[0][p];
  const float xp[3] = {P4.x, P4.y, P4.z};
  float F[3][3];
  {
    const float4 c0 = st.f[2][p], c1 = st.f[3][p], c2 = st.f[4][p];
    F[0][0] = c0.x; F[1][0] = c0.y; F[2][0] = c0.z;
    F[0][1] = c1.x; F[1][1] = c1.y; F[2][1] = c1.z;
    F[0][2] = c2.x; F[1][2] = c2.y; F[2][2] = c2.z;
  }
  int base[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) base[a] = int(floorf(__fdiv_rn(xp[a] - P.worldMin[a], h))) - 1;
  Stencil S;
  stencilAt(P, xp, base, S);
  // pass 1: velocity gradient G = sum v_i grad w^T
  float G[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
  for (int iy = 0; iy < 3; ++iy)
#pragma unroll
  for (int ix = 0; ix < 3; ++ix) {
    const int nx = base[0] + ix, ny = base[1] + iy, nz = base[2] + iz;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= P.gridRes[0] || ny >= P.gridRes[1] || nz >= P.gridRes[2]) continue;
    const float4 vi = __ldg(vel + mortonEncode(nx, ny, nz));
    if (vi.w < 1e-10f) continue;
    const float w = S.w[0][ix] * S.w[1][iy] * S.w[2][iz];
    if (w < 1e-12f) continue;
    const float dw[3] = {S.g[0][ix] * S.w[1][iy] * S.w[2][iz] * invH, S.w[0][ix] * S.g[1][iy] * S.w[2][iz] * invH,
                         S.w[0][ix] * S.w[1][iy] * S.g[2][iz] * invH};
    const float v[3] = {vi.x, vi.y, vi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) G[a][b] += v[a] * dw[b];
  }
  // F' = (I + dt G) F
  double Fn[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      float acc = F[a][b];
#pragma unroll
      for (int q = 0; q < 3; ++q) acc += dt * G[a][q] * F[q][b];
      Fn[a][b] = acc;
    }
  float Fnbf[3][3], tbf[3][3];
  loadRows(ob.F, p, Fnbf);
  loadRows(ob.T, p, tbf);
  double Fnb[3][3], tb[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Fnb[a][b] = Fnbf[a][b];
      tb[a][b] = tbf[a][b];
    }
  const float2 l = lame[p];
  double mb = 0, lb = 0;
  henckyAdj(Fn, double(l.x), double(l.y), tb, Fnb, mb, lb);
  mub[p] += float(mb);
  lamb[p] += float(lb);
  // x' = x + dt v'
  const float4 xb4 = ob.x[p], vb4 = ob.v[p];
  float xb[3] = {xb4.x, xb4.y, xb4.z};
  const float vb[3] = {vb4.x + dt * xb4.x, vb4.y + dt * xb4.y, vb4.z + dt * xb4.z};
  // F' = (I + dt G) F:  Fbar = (I + dt G)^T F'bar,  Gbar = dt F'bar F^T
  float Fb[3][3], Gb[3][3], Fnf[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) Fnf[a][b] = float(Fnb[a][b]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      float fb = Fnf[a][b], gb = 0.f;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        fb += dt * G[q][a] * Fnf[q][b];
        gb += Fnf[a][q] * F[b][q];
      }
      Fb[a][b] = fb;
      Gb[a][b] = dt * gb;
    }
  float Bb[3][3];
  loadRows(ob.B, p, Bb);
  // pass 2: scatter to the grid-velocity adjoint; gather the x adjoint
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
  for (int iy = 0; iy < 3; ++iy)
#pragma unroll
  for (int ix = 0; ix < 3; ++ix) {
    const int nx = base[0] + ix, ny = base[1] + iy, nz = base[2] + iz;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= P.gridRes[0] || ny >= P.gridRes[1] || nz >= P.gridRes[2]) continue;
    const uint32_t id = mortonEncode(nx, ny, nz);
    const float4 vi4 = __ldg(vel + id);
    if (vi4.w < 1e-10f) continue;
    NodeTerms t;
    nodeTerms(P, S, xp, ix, iy, iz, t);
    if (t.w < 1e-12f) continue;
    const float vi[3] = {vi4.x, vi4.y, vi4.z};
    float gadd[3], Bbr[3];
    float viVb = 0.f, viBbr = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      Bbr[a] = Bb[a][0] * t.r[0] + Bb[a][1] * t.r[1] + Bb[a][2] * t.r[2];
      const float Gbdw = Gb[a][0] * t.dw[0] + Gb[a][1] * t.dw[1] + Gb[a][2] * t.dw[2];
      gadd[a] = t.w * vb[a] + t.w * Bbr[a] + Gbdw;
      viVb += vi[a] * vb[a];
      viBbr += vi[a] * Bbr[a];
    }
    redAddV4(gadj + id, gadd[0], gadd[1], gadd[2], 0.f);
    float GtV[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) GtV[c] = Gb[0][c] * vi[0] + Gb[1][c] * vi[1] + Gb[2][c] * vi[2];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const float BtV = Bb[0][b] * vi[0] + Bb[1][b] * vi[1] + Bb[2][b] * vi[2];
      const float HGtv = t.H[b][0] * GtV[0] + t.H[b][1] * GtV[1] + t.H[b][2] * GtV[2];
      xb[b] += t.dw[b] * (viVb + viBbr) - t.w * BtV + HGtv;
    }
  }
  ib.x[p] = make_float4(xb[0], xb[1], xb[2], 0.f);
  storeRows(ib.F, p, Fb);
}

// Grid adjoint: v = walls(cap(p/m) + g dt); turns the grid-velocity adjoint
// into momentum and mass adjoints (p_bar, m_bar), in place.
// Over the substep's node box (the G2P adjoint scattered into no node outside
// it, and the P2G adjoint gathers from none).  acc is read for the last time
// here and cleared behind the read (the segment's next recomputation
// accumulates into it again); `other` -- the grid adjoint of the next substep
// back -- is cleared over the box where the substep after this one left it.
__device__ __forceinline__ void adjGridNode(const SubstepParams& P, float4* acc, float4* gadj, uint32_t c);
__global__ void __launch_bounds__(kT) k_adj_grid(SubstepParams P, float4* acc, float4* gadj, const NodeBox* box, float4* other,
                                                 const NodeBox* otherBox) {
  forBox(*box, [&](uint32_t c) { adjGridNode(P, acc, gadj, c); });
  if (otherBox) forBox(*otherBox, [&](uint32_t c) { other[c] = make_float4(0.f, 0.f, 0.f, 0.f); });
}
__device__ __forceinline__ void adjGridNode(const SubstepParams& P, float4* acc, float4* gadj, uint32_t c) {
  const float4 a = acc[c];
  acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
  const float m = a.w;
  if (m < 1e-10f) {
    gadj[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  const float4 g = gadj[c];
  int idx[3];
  mortonDecode(c, idx[0], idx[1], idx[2]);
  float3 vo3, vc3;
  gridNode(P, idx[0], idx[1], idx[2], m, a.x, a.y, a.z, vo3, vc3);
  const float vout[3] = {vo3.x, vo3.y, vo3.z};
  const float gi[3] = {g.x, g.y, g.z};
  float vcb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const bool band = idx[k] <= 1 || idx[k] >= P.gridRes[k] - 2;
    vcb[k] = (band && vout[k] == 0.f) ? 0.f : gi[k];  // a component the wall band zeroed
  }
  const float v[3] = {a.x / m, a.y / m, a.z / m};
  const float speed = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  float v0b[3];
  if (speed > 15.0f) {
    // v_c = 15 v / |v|:  dv_c = (15/|v|) (I - u u^T) dv,  u = v_c / 15
    const float sc = 15.0f / speed;
    const float u[3] = {vc3.x / 15.0f, vc3.y / 15.0f, vc3.z / 15.0f};
    const float ud = u[0] * vcb[0] + u[1] * vcb[1] + u[2] * vcb[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) v0b[k] = sc * (vcb[k] - u[k] * ud);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) v0b[k] = vcb[k];
  }
  const float mb = -(v0b[0] * v[0] + v0b[1] * v[1] + v0b[2] * v[2]) / m;
  gadj[c] = make_float4(v0b[0] / m, v0b[1] / m, v0b[2] / m, mb);
}

// P2G adjoint: gathers (p_bar, m_bar) -> adjoints of v, B, tau and x (added).
__global__ void __launch_bounds__(kT) k_adj_p2g(SubstepParams P, St st, uint32_t n, const float4* __restrict__ gadj, AdjPtrs ib) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float dt = P.dt, h = P.cellSize, Dinv = 4.0f / (h * h);
  const PState s = loadState(st.f, p);
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  const float Vp = s.P.w;
  const float mp = fetchRho0(P, __float_as_uint(s.v.w)) * Vp;
  const float vp[3] = {s.v.x, s.v.y, s.v.z};
  float Bm[3][3];  // math rows from the GLSL columns
  Bm[0][0] = s.B0.x; Bm[1][0] = s.B0.y; Bm[2][0] = s.B0.z;
  Bm[0][1] = s.B1.x; Bm[1][1] = s.B1.y; Bm[2][1] = s.B1.z;
  Bm[0][2] = s.B2.x; Bm[1][2] = s.B2.y; Bm[2][2] = s.B2.z;
  const float T[3][3] = {{s.F0.w, s.B0.w, s.B1.w}, {s.B0.w, s.F1.w, s.B2.w}, {s.B1.w, s.B2.w, s.F2.w}};
  int c[3];
  cellCoords(P, xp[0], xp[1], xp[2], c[0], c[1], c[2]);
  const int base[3] = {c[0] - 1, c[1] - 1, c[2] - 1};
  Stencil S;
  stencilAt(P, xp, base, S);
  float xb[3] = {0.f, 0.f, 0.f}, vb[3] = {0.f, 0.f, 0.f};
  float Bb[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, Tb[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  const int cr = int(P.cubeRes);
#pragma unroll
  for (int iz = 0; iz < 3; ++iz)
#pragma unroll
  for (int iy = 0; iy < 3; ++iy)
#pragma unroll
  for (int ix = 0; ix < 3; ++ix) {
    const int nx = base[0] + ix, ny = base[1] + iy, nz = base[2] + iz;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= cr || ny >= cr || nz >= cr) continue;
    NodeTerms t;
    nodeTerms(P, S, xp, ix, iy, iz, t);
    if (t.w < 1e-12f) continue;
    const float4 g4 = __ldg(gadj + mortonEncode(nx, ny, nz));
    const float Pb[3] = {g4.x, g4.y, g4.z};
    const float mb = g4.w;
    float ve[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ve[a] = vp[a] + Dinv * (Bm[a][0] * t.r[0] + Bm[a][1] * t.r[1] + Bm[a][2] * t.r[2]);
    const float vePb = ve[0] * Pb[0] + ve[1] * Pb[1] + ve[2] * Pb[2];
    const float wm = t.w * mp;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      vb[a] += wm * Pb[a];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        Bb[a][b] += wm * Dinv * Pb[a] * t.r[b];
        Tb[a][b] -= dt * Vp * Pb[a] * t.dw[b];
      }
    }
    float TP[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) TP[k] = T[0][k] * Pb[0] + T[1][k] * Pb[1] + T[2][k] * Pb[2];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const float BtP = Bm[0][b] * Pb[0] + Bm[1][b] * Pb[1] + Bm[2][b] * Pb[2];
      const float HTP = t.H[b][0] * TP[0] + t.H[b][1] * TP[1] + t.H[b][2] * TP[2];
      xb[b] += mb * mp * t.dw[b] + t.dw[b] * mp * vePb - wm * Dinv * BtP - dt * Vp * HTP;
    }
  }
  const float4 x0 = ib.x[p];
  ib.x[p] = make_float4(x0.x + xb[0], x0.y + xb[1], x0.z + xb[2], 0.f);
  ib.v[p] = make_float4(vb[0], vb[1], vb[2], 0.f);
  storeRows(ib.B, p, Bb);
  storeRows(ib.T, p, Tb);
}

// Adjoint of the final state: dL/dx_p = lossGrad * 2 (COM - target) m_p / M.
__global__ void __launch_bounds__(kT) k_adj_seed(const float4* __restrict__ x0, float rho0, uint32_t n, const AdjScalars* sc, AdjPtrs ob) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double M = sc->com[3];
  const double m = double(rho0 * x0[p].w);
  float g[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) g[a] = float(double(sc->lossGrad) * 2.0 * (sc->com[a] / M - sc->target[a]) * m / M);
  ob.x[p] = make_float4(g[0], g[1], g[2], 0.f);
}

__global__ void __launch_bounds__(kT) k_adj_out(AdjPtrs ob, const float* __restrict__ mub, const float* __restrict__ lamb, float nu, uint32_t n,
                                                float4* gv, float* gE, float4* gx) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  gv[p] = ob.v[p];
  gx[p] = ob.x[p];
  const float dmu = 1.0f / (2.0f * (1.0f + nu)), dlam = nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  gE[p] = mub[p] * dmu + lamb[p] * dlam;
}

}  // namespace

// ====================================================================== host
AdjointEngine::AdjointEngine(const nebula_mpm_adjoint_config& cfg) : cfg_(cfg) {
  if (!(cfg.cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  if (cfg.particles == 0 || cfg.substeps == 0) throw Error(NEBULA_MPM_ERR_INVALID, "particles and substeps must be > 0");
  if (!(cfg.dt > 0.f) || !(cfg.nu > -1.f && cfg.nu < 0.5f) || !(cfg.rho0 > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "bad dt, nu or rho0");
  check(cudaGetDevice(&device_), "cudaGetDevice");
  n_ = cfg.particles;
  every_ = std::max(1u, std::min(cfg.checkpointEvery, cfg.substeps));
  segs_ = (cfg.substeps + every_ - 1) / every_;
  uint32_t res[3];
  domainGridRes(cfg.domainSize, cfg.cellSize, res);
  const uint32_t cube = domainCubeRes(res);
  if (cube > 512u) throw Error(NEBULA_MPM_ERR_INVALID, "adjoint grid above 512 per axis");
  nc_ = cube * cube * cube;
  // substep parameters: APIC, global-material path (per-particle Lame set per thread), gravity as one force
  P_.dt = cfg.dt;
  P_.cellSize = cfg.cellSize;
  for (int a = 0; a < 3; ++a) {
    P_.gridRes[a] = int(res[a]);
    P_.worldMin[a] = 0.f;
    P_.worldMax[a] = cfg.domainSize[a];
  }
  P_.cubeRes = cube;
  P_.hashCells = nc_;
  P_.flip_ratio = -1.0f;
  P_.materialCount = 0;
  P_.colliderCount = 0;
  P_.rho0 = cfg.rho0;
  P_.plasticModel = MAT_ELASTIC;
  P_.q_max = 1e5f;
  Force f{};
  const float g = std::sqrt(cfg.gravity[0] * cfg.gravity[0] + cfg.gravity[1] * cfg.gravity[1] + cfg.gravity[2] * cfg.gravity[2]);
  f.type = FORCE_GRAVITY;
  for (int a = 0; a < 3; ++a) f.data[a] = g > 0.f ? cfg.gravity[a] / g : 0.f;
  f.data[3] = g;
  forces_.alloc(sizeof(Force));
  check(cudaMemcpy(forces_.ptr, &f, sizeof(Force), cudaMemcpyHostToDevice), "upload forces");
  P_.forceCount = g > 0.f ? 1u : 0u;
  P_.forces = static_cast<const Force*>(forces_.ptr);

  const size_t stBytes = size_t(8) * n_ * sizeof(float4);
  const size_t gBytes = size_t(nc_) * sizeof(float4);
  lame_.alloc(size_t(n_) * sizeof(float2));
  scal_.alloc(sizeof(AdjScalars));
  check(cudaMemset(scal_.ptr, 0, sizeof(AdjScalars)), "cudaMemset");
  x0_.alloc(size_t(n_) * sizeof(float4));
  v0_.alloc(size_t(n_) * sizeof(float4));
  E_.alloc(size_t(n_) * sizeof(float));
  gradV_.alloc(size_t(n_) * sizeof(float4));
  gradX_.alloc(size_t(n_) * sizeof(float4));
  gradE_.alloc(size_t(n_) * sizeof(float));
  for (auto& b : ping_) b.alloc(stBytes);
  ck_.resize(segs_);
  for (auto& b : ck_) b.alloc(stBytes);
  segState_.resize(every_);
  for (uint32_t j = 1; j < every_; ++j) segState_[j].alloc(stBytes);
  // grids start zeroed and are left so by the grid passes that read them last
  segAcc_.resize(every_);
  segVel_.resize(every_);
  for (uint32_t j = 0; j < every_; ++j) {
    segAcc_[j].alloc(gBytes);
    segVel_[j].alloc(gBytes);
    check(cudaMemset(segAcc_[j].ptr, 0, gBytes), "cudaMemset");
  }
  acc_.alloc(gBytes);
  vel_.alloc(gBytes);
  check(cudaMemset(acc_.ptr, 0, gBytes), "cudaMemset");
  for (auto& b : adj_) b.alloc(size_t(11) * n_ * sizeof(float4));
  for (auto& g : gadj_) g.alloc(gBytes);
  boxes_.alloc(size_t(std::max(cfg.substeps, 1u)) * sizeof(NodeBox));
  check(cudaMemset(boxes_.ptr, 0, boxes_.bytes), "cudaMemset");
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");
  gridBlocks_ = uint32_t(std::max(sms, 1)) * 2u;  // grid-stride over a node box
  mub_.alloc(size_t(n_) * sizeof(float));
  lamb_.alloc(size_t(n_) * sizeof(float));
  finalBuf_ = int(cfg.substeps & 1u);
}

AdjointEngine::~AdjointEngine() {
  cudaDeviceSynchronize();
  for (auto& g : graph_)
    if (g) cudaGraphExecDestroy(g);
}

void AdjointEngine::bindDevice() const { check(cudaSetDevice(device_), "cudaSetDevice"); }

void AdjointEngine::setGraphs(bool on) {
  bindDevice();
  if (!on) {
    check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    for (auto& g : graph_)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  useGraphs_ = on;
}

// One forward substep into grid buffers acc (zero on entry) and vel; the P2G's
// node box goes to box[k].  clear: zero acc behind the grid update's read.
void AdjointEngine::substepForward(const float4* const* in, float4* const* out, float4* acc, float4* vel, uint32_t k, bool clear, cudaStream_t s) {
  St si, so;
  for (int q = 0; q < 8; ++q) {
    si.f[q] = const_cast<float4*>(in[q]);
    so.f[q] = out ? out[q] : nullptr;
  }
  AdjScalars* sc = static_cast<AdjScalars*>(scal_.ptr);
  NodeBox* box = static_cast<NodeBox*>(boxes_.ptr) + k;
  k_fwd_p2g<<<blocks(n_), kT, 0, s>>>(P_, si, n_, acc, box);
  k_fwd_grid<<<gridBlocks_, kT, 0, s>>>(P_, acc, vel, sc, box, clear ? 1 : 0);
  launches_ += 2;
  if (out) {
    k_fwd_g2p<<<blocks(n_), kT, 0, s>>>(P_, si, so, static_cast<const float2*>(lame_.ptr), n_, vel, sc);
    ++launches_;
  }
  check(cudaGetLastError(), "forward substep");
}

// Forward rollout from x0_/v0_/E_: checkpoints, final state, loss.
void AdjointEngine::forwardBody(cudaStream_t s) {
  AdjScalars* sc = static_cast<AdjScalars*>(scal_.ptr);
  check(cudaMemsetAsync(sc, 0, offsetof(AdjScalars, target), s), "memset com");
  check(cudaMemsetAsync(&sc->events, 0, sizeof(uint32_t), s), "memset events");
  check(cudaMemsetAsync(boxes_.ptr, 0, size_t(cfg_.substeps) * sizeof(NodeBox), s), "memset boxes");
  St s0 = stPtrs(ping_[0], n_);
  k_init<<<blocks(n_), kT, 0, s>>>(static_cast<const float4*>(x0_.ptr), static_cast<const float4*>(v0_.ptr), static_cast<const float*>(E_.ptr),
                                   cfg_.nu, n_, s0, static_cast<float2*>(lame_.ptr));
  ++launches_;
  int cur = 0;
  const size_t stBytes = size_t(8) * n_ * sizeof(float4);
  for (uint32_t k = 0; k < cfg_.substeps; ++k) {
    if (k % every_ == 0) check(cudaMemcpyAsync(ck_[k / every_].ptr, ping_[cur].ptr, stBytes, cudaMemcpyDeviceToDevice, s), "checkpoint");
    St a = stPtrs(ping_[cur], n_), b = stPtrs(ping_[cur ^ 1], n_);
    substepForward(a.f, b.f, static_cast<float4*>(acc_.ptr), static_cast<float4*>(vel_.ptr), k, true, s);
    cur ^= 1;
  }
  St fin = stPtrs(ping_[cur], n_);
  k_com<<<blocks(n_), kT, 0, s>>>(fin.f[0], static_cast<const float4*>(x0_.ptr), cfg_.rho0, n_, sc);
  k_loss<<<1, 32, 0, s>>>(sc);
  launches_ += 2;
  check(cudaGetLastError(), "forward");
}

void AdjointEngine::backwardBody(cudaStream_t s) {
  AdjScalars* sc = static_cast<AdjScalars*>(scal_.ptr);
  const size_t adjBytes = size_t(11) * n_ * sizeof(float4);
  check(cudaMemsetAsync(mub_.ptr, 0, size_t(n_) * sizeof(float), s), "memset");
  check(cudaMemsetAsync(lamb_.ptr, 0, size_t(n_) * sizeof(float), s), "memset");
  check(cudaMemsetAsync(adj_[0].ptr, 0, adjBytes, s), "memset");
  // the grid adjoints start zeroed; each reverse substep then clears the other
  // buffer over the box the substep after it left dirty
  for (auto& g : gadj_) check(cudaMemsetAsync(g.ptr, 0, size_t(nc_) * sizeof(float4), s), "memset grid adjoint");
  NodeBox* boxes = static_cast<NodeBox*>(boxes_.ptr);
  int o = 0;
  k_adj_seed<<<blocks(n_), kT, 0, s>>>(static_cast<const float4*>(x0_.ptr), cfg_.rho0, n_, sc, adjPtrs(adj_[o], n_));
  ++launches_;
  const float2* lame = static_cast<const float2*>(lame_.ptr);
  float* mub = static_cast<float*>(mub_.ptr);
  float* lamb = static_cast<float*>(lamb_.ptr);
  for (int seg = int(segs_) - 1; seg >= 0; --seg) {
    const uint32_t k0 = uint32_t(seg) * every_, k1 = std::min(cfg_.substeps, k0 + every_), len = k1 - k0;
    auto stateOf = [&](uint32_t j) { return j == 0 ? stPtrs(ck_[seg], n_) : stPtrs(segState_[j], n_); };
    // recompute the segment, keeping every substep's input state, grid and node box
    check(cudaMemsetAsync(boxes + k0, 0, size_t(len) * sizeof(NodeBox), s), "memset boxes");
    for (uint32_t j = 0; j < len; ++j) {
      St in = stateOf(j);
      St out = j + 1 < len ? stateOf(j + 1) : St{};
      substepForward(in.f, j + 1 < len ? out.f : nullptr, static_cast<float4*>(segAcc_[j].ptr), static_cast<float4*>(segVel_[j].ptr), k0 + j,
                     false, s);
    }
    // reverse the segment
    for (int j = int(len) - 1; j >= 0; --j) {
      St st = stateOf(uint32_t(j));
      AdjPtrs ob = adjPtrs(adj_[o], n_), ib = adjPtrs(adj_[o ^ 1], n_);
      const uint32_t k = k0 + uint32_t(j);
      float4* gadj = static_cast<float4*>(gadj_[k & 1u].ptr);
      float4* other = static_cast<float4*>(gadj_[(k + 1u) & 1u].ptr);
      const NodeBox* otherBox = k + 1u < cfg_.substeps ? boxes + k + 1u : nullptr;
      k_adj_g2p<<<blocks(n_), kT, 0, s>>>(P_, st, lame, n_, static_cast<const float4*>(segVel_[j].ptr), ob, ib, gadj, mub, lamb);
      k_adj_grid<<<gridBlocks_, kT, 0, s>>>(P_, static_cast<float4*>(segAcc_[j].ptr), gadj, boxes + k, other, otherBox);
      k_adj_p2g<<<blocks(n_), kT, 0, s>>>(P_, st, n_, gadj, ib);
      launches_ += 3;
      o ^= 1;
    }
  }
  k_adj_out<<<blocks(n_), kT, 0, s>>>(adjPtrs(adj_[o], n_), mub, lamb, cfg_.nu, n_, static_cast<float4*>(gradV_.ptr),
                                      static_cast<float*>(gradE_.ptr), static_cast<float4*>(gradX_.ptr));
  ++launches_;
  check(cudaGetLastError(), "backward");
}

// Run the forward (fwd) or backward body, from a graph captured on first use
// when the stream is not the legacy default stream.
void AdjointEngine::run(bool fwd, cudaStream_t s) {
  const int g = fwd ? 0 : 1;
  if (!useGraphs_ || s == nullptr) {
    fwd ? forwardBody(s) : backwardBody(s);
    return;
  }
  if (!graph_[g]) {
    const uint64_t l0 = launches_;
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      fwd ? forwardBody(s) : backwardBody(s);
    } catch (...) {
      cudaStreamEndCapture(s, &graph);
      if (graph) cudaGraphDestroy(graph);
      launches_ = l0;
      throw;
    }
    check(cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture");
    const cudaError_t e = cudaGraphInstantiate(&graph_[g], graph, 0);
    cudaGraphDestroy(graph);
    check(e, "cudaGraphInstantiate");
    graphLaunches_[g] = launches_ - l0;
    launches_ = l0;
  }
  check(cudaGraphLaunch(graph_[g], s), "cudaGraphLaunch");
  launches_ += graphLaunches_[g];
}

void AdjointEngine::forward(const float* dPos4, const float* dVel4, const float* dE, const float target[3], float* dLoss, cudaStream_t s) {
  bindDevice();
  if (!dPos4 || !dVel4 || !dE || !target) throw Error(NEBULA_MPM_ERR_INVALID, "null input");
  AdjScalars* sc = static_cast<AdjScalars*>(scal_.ptr);
  const double t[3] = {target[0], target[1], target[2]};
  check(cudaMemcpyAsync(sc->target, t, sizeof(t), cudaMemcpyHostToDevice, s), "upload target");
  check(cudaMemcpyAsync(x0_.ptr, dPos4, size_t(n_) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "copy input");
  check(cudaMemcpyAsync(v0_.ptr, dVel4, size_t(n_) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "copy input");
  check(cudaMemcpyAsync(E_.ptr, dE, size_t(n_) * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy input");
  run(true, s);
  if (dLoss) check(cudaMemcpyAsync(dLoss, &sc->loss, sizeof(float), cudaMemcpyDeviceToDevice, s), "copy loss");
  haveForward_ = true;
}

void AdjointEngine::backward(float lossGrad, float* dGradVel4, float* dGradE, float* dGradPos4, cudaStream_t s) {
  bindDevice();
  if (!haveForward_) throw Error(NEBULA_MPM_ERR_INVALID, "backward needs a forward first");
  AdjScalars* sc = static_cast<AdjScalars*>(scal_.ptr);
  check(cudaMemcpyAsync(&sc->lossGrad, &lossGrad, sizeof(float), cudaMemcpyHostToDevice, s), "upload loss gradient");
  run(false, s);
  if (dGradVel4) check(cudaMemcpyAsync(dGradVel4, gradV_.ptr, size_t(n_) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "copy gradient");
  if (dGradE) check(cudaMemcpyAsync(dGradE, gradE_.ptr, size_t(n_) * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy gradient");
  if (dGradPos4) check(cudaMemcpyAsync(dGradPos4, gradX_.ptr, size_t(n_) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "copy gradient");
}

void AdjointEngine::download(int field, float* host, uint64_t count) {
  bindDevice();
  if (field < 0 || field > 7) throw Error(NEBULA_MPM_ERR_INVALID, "field index out of range");
  if (count != uint64_t(n_) * 4 || !host) throw Error(NEBULA_MPM_ERR_INVALID, "count must be 4 * particles");
  if (!haveForward_) throw Error(NEBULA_MPM_ERR_INVALID, "no forward run yet");
  check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  const float4* src = static_cast<const float4*>(ping_[finalBuf_].ptr) + size_t(field) * n_;
  check(cudaMemcpy(host, src, count * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

uint32_t AdjointEngine::events() {
  bindDevice();
  check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  AdjScalars h;
  check(cudaMemcpy(&h, scal_.ptr, sizeof(h), cudaMemcpyDeviceToHost), "read events");
  return h.events;
}

}  // namespace nebula

// ====================================================================== C ABI
using nebula::Error;
using nebula::g_last_error;

struct nebula_mpm_adjoint {
  std::unique_ptr<nebula::AdjointEngine> eng;
};

namespace {
template <class F> int guardedA(F&& f) {
  try {
    f();
    return NEBULA_MPM_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return NEBULA_MPM_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return NEBULA_MPM_ERR_INVALID;
  }
}
nebula::AdjointEngine& A(nebula_mpm_adjoint* a) {
  if (!a || !a->eng) throw Error(NEBULA_MPM_ERR_INVALID, "null adjoint engine");
  return *a->eng;
}
}  // namespace

extern "C" {

int nebula_mpm_adjoint_create(const nebula_mpm_adjoint_config* cfg, nebula_mpm_adjoint** out) {
  return guardedA([&] {
    if (!cfg || !out) throw Error(NEBULA_MPM_ERR_INVALID, "null argument");
    *out = nullptr;
    auto h = std::make_unique<nebula_mpm_adjoint>();
    h->eng = std::make_unique<nebula::AdjointEngine>(*cfg);
    *out = h.release();
  });
}
int nebula_mpm_adjoint_destroy(nebula_mpm_adjoint* a) {
  return guardedA([&] { delete a; });
}
int nebula_mpm_adjoint_forward(nebula_mpm_adjoint* a, const float* dPos4, const float* dVel4, const float* dE, const float target[3], float* dLoss,
                               void* stream) {
  return guardedA([&] { A(a).forward(dPos4, dVel4, dE, target, dLoss, static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_adjoint_backward(nebula_mpm_adjoint* a, float lossGrad, float* dGradVel4, float* dGradE, float* dGradPos4, void* stream) {
  return guardedA([&] { A(a).backward(lossGrad, dGradVel4, dGradE, dGradPos4, static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_adjoint_download(nebula_mpm_adjoint* a, int field, float* host, uint64_t count) {
  return guardedA([&] { A(a).download(field, host, count); });
}
int nebula_mpm_adjoint_events(nebula_mpm_adjoint* a, uint32_t* events) {
  return guardedA([&] {
    if (!events) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *events = A(a).events();
  });
}
int nebula_mpm_adjoint_set_graphs(nebula_mpm_adjoint* a, int enable) {
  return guardedA([&] { A(a).setGraphs(enable != 0); });
}
int nebula_mpm_adjoint_launches(nebula_mpm_adjoint* a, uint64_t* launches) {
  return guardedA([&] {
    if (!launches) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *launches = A(a).launches();
  });
}

}  // extern "C"
