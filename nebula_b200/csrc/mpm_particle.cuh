// mpm_particle.cuh -- per-particle halves of the substep (sm_100a device code).
//
//   g2pParticle   gather, F update, return map, stress, advection, SDF
//                 push-out and world clamp of one particle: mpm_g2p.comp:70-272
//   p2gParticle   the contributions of one particle to its 27 stencil nodes:
//                 the terms the per-node gather of mpm_p2g.comp:40-82 sums
//   gridNode      velocity, cap, forces, walls, colliders and dense-SDF
//                 boundary of one node: mpm_grid_update.comp:17-102 followed
//                 by mpm_nanovdb_bc.comp:23-54
//
// Grid storage differs between callers (the reference's dense float4 arrays
// for the single-pass API, brick-sparse arrays for the engine), so the gather
// and scatter take accessor objects.
#pragma once
#include "mpm_device.cuh"

namespace nebula {

// One particle in the reference layout (8 float4, MPMEngine.cpp:46-53).
struct PState {
  float4 P, v, F0, F1, F2, B0, B1, B2;
};

__device__ __forceinline__ PState loadState(const float4* const* f, uint32_t i) {
  PState s;
  s.P = f[0][i]; s.v = f[1][i];
  s.F0 = f[2][i]; s.F1 = f[3][i]; s.F2 = f[4][i];
  s.B0 = f[5][i]; s.B1 = f[6][i]; s.B2 = f[7][i];
  return s;
}
__device__ __forceinline__ void storeState(float4* const* f, uint32_t i, const PState& s) {
  f[0][i] = s.P; f[1][i] = s.v;
  f[2][i] = s.F0; f[3][i] = s.F1; f[4][i] = s.F2;
  f[5][i] = s.B0; f[6][i] = s.B1; f[7][i] = s.B2;
}

// Node centre (ix + 0.5) h + worldMin, per axis.
__device__ __forceinline__ float nodeCentre(const SubstepParams& P, int a, int i) { return (float(i) + 0.5f) * P.cellSize + P.worldMin[a]; }

// ---------------------------------------------------------------- P2G terms
// For each of the 27 nodes n = cell + (dx,dy,dz) that exist in the Morton
// grid (coords in [0, cubeRes)) and get weight >= 1e-12, calls
// emit(nx, ny, nz, mom_x, mom_y, mom_z, mass) with
//   mass = w m_p,
//   mom  = w m_p (v_p + (4/h^2) B_p (x_i - x_p)) - dt V_p tau_p grad w.
template <class Emit>
__device__ __forceinline__ void p2gParticle(const SubstepParams& P, const PState& s, float dtStress, Emit&& emit) {
  const float h = P.cellSize;
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  const float Vp = s.P.w;
  const float vp[3] = {s.v.x, s.v.y, s.v.z};
  const float mp = fetchRho0(P, __float_as_uint(s.v.w)) * Vp;
  int c[3];
  cellCoords(P, xp[0], xp[1], xp[2], c[0], c[1], c[2]);
  const bool apic = P.flip_ratio < -0.5f;
  // B (GLSL columns B0..B2) and the symmetric stress from the w lanes
  float Bm[3][3];
  Bm[0][0] = s.B0.x; Bm[0][1] = s.B0.y; Bm[0][2] = s.B0.z;
  Bm[1][0] = s.B1.x; Bm[1][1] = s.B1.y; Bm[1][2] = s.B1.z;
  Bm[2][0] = s.B2.x; Bm[2][1] = s.B2.y; Bm[2][2] = s.B2.z;
  if (!apic) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) Bm[a][b] = 0.f;
  }
  // tau[c][r]: col0=(xx,xy,xz) col1=(xy,yy,yz) col2=(xz,yz,zz)
  const float t[3][3] = {{s.F0.w, s.B0.w, s.B1.w}, {s.B0.w, s.F1.w, s.B2.w}, {s.B1.w, s.B2.w, s.F2.w}};
  const float D_inv = 4.0f / (h * h);
  const float sdt = dtStress * Vp;
  float wa[3][3], ga[3][3];  // per axis, per offset: N(d), N'(d)
  float xi[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      xi[a][k] = nodeCentre(P, a, c[a] + k - 1);
      float d = __fdiv_rn(xp[a] - xi[a][k], h);
      wa[a][k] = bspline2(d);
      ga[a][k] = bspline2g(d);
    }
#pragma unroll
  for (int dz = 0; dz < 3; ++dz)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const int nx = c[0] + dx - 1, ny = c[1] + dy - 1, nz = c[2] + dz - 1;
        if (nx < 0 || ny < 0 || nz < 0 || nx >= int(P.cubeRes) || ny >= int(P.cubeRes) || nz >= int(P.cubeRes)) continue;
        const float wx = wa[0][dx], wy = wa[1][dy], wz = wa[2][dz];
        const float w = wx * wy * wz;
        if (w < 1e-12f) continue;
        const float dw0 = __fdiv_rn(ga[0][dx] * wy * wz, h);
        const float dw1 = __fdiv_rn(wx * ga[1][dy] * wz, h);
        const float dw2 = __fdiv_rn(wx * wy * ga[2][dz], h);
        const float r0 = xi[0][dx] - xp[0], r1 = xi[1][dy] - xp[1], r2 = xi[2][dz] - xp[2];
        const float wm = w * mp;
        float m[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const float ve = vp[i] + D_inv * (Bm[0][i] * r0 + Bm[1][i] * r1 + Bm[2][i] * r2);
          const float td = t[0][i] * dw0 + t[1][i] * dw1 + t[2][i] * dw2;
          m[i] = wm * ve - sdt * td;
        }
        emit(nx, ny, nz, m[0], m[1], m[2], wm);
      }
}

// ---------------------------------------------------------------- grid node
// Returns false when the node is skipped (mass < 1e-10).  On true, v is the
// boundary-conditioned velocity and vold the pre-force velocity (FLIP).
__device__ __forceinline__ bool gridNode(const SubstepParams& P, int ix, int iy, int iz, float mass, float mx, float my, float mz, float3& vout,
                                         float3& vold) {
  if (mass < 1e-10f) return false;
  f3 v = mkf3(mx / mass, my / mass, mz / mass);
  {
    float vs = len3(v);
    const float vmax_grid = 15.0f;
    if (vs > vmax_grid) {
      float s = vmax_grid / vs;
      v = mkf3(v.x * s, v.y * s, v.z * s);
    }
  }
  vold = make_float3(v.x, v.y, v.z);
  const f3 xi = mkf3(nodeCentre(P, 0, ix), nodeCentre(P, 1, iy), nodeCentre(P, 2, iz));
  for (uint32_t fi = 0; fi < P.forceCount; ++fi) {
    const Force& f = P.forces[fi];
    uint32_t fm = f.affectMask;
    if (fm != 0u && (fm & 1u) == 0u) continue;
    if (f.type == FORCE_GRAVITY || f.type == FORCE_CONSTANT_WIND) {
      const float s = f.data[3];
      v.x += (f.data[0] * s) * P.dt;
      v.y += (f.data[1] * s) * P.dt;
      v.z += (f.data[2] * s) * P.dt;
    }
  }
  const int Nx = P.gridRes[0] - 1, Ny = P.gridRes[1] - 1, Nz = P.gridRes[2] - 1;
  if (ix <= 1 && v.x < 0.f) v.x = 0.f;
  if (ix >= Nx - 1 && v.x > 0.f) v.x = 0.f;
  if (iy <= 1 && v.y < 0.f) v.y = 0.f;
  if (iy >= Ny - 1 && v.y > 0.f) v.y = 0.f;
  if (iz <= 1 && v.z < 0.f) v.z = 0.f;
  if (iz >= Nz - 1 && v.z > 0.f) v.z = 0.f;
  for (uint32_t ci = 0; ci < P.colliderCount; ++ci) {
    const Collider& c = P.colliders[ci];
    f3 n;
    float s = colliderSDF(c, xi, n);
    if (s <= 0.f) applyColliderBC(v, n, mkf3(c.vx, c.vy, c.vz), c.restitution, c.friction);
  }
  if (P.sdf) {
    auto sample = [&](int x, int y, int z) -> float {
      if (x < 0 || y < 0 || z < 0 || x >= P.gridRes[0] || y >= P.gridRes[1] || z >= P.gridRes[2]) return 1e6f;
      return __ldg(P.sdf + mortonEncode(x, y, z));
    };
    float s = sample(ix, iy, iz);
    if (s < 0.f) {
      v = mkf3(0.f, 0.f, 0.f);
    } else if (s < P.cellSize * 1.5f) {
      f3 gn = mkf3(sample(ix + 1, iy, iz) - sample(ix - 1, iy, iz), sample(ix, iy + 1, iz) - sample(ix, iy - 1, iz),
                   sample(ix, iy, iz + 1) - sample(ix, iy, iz - 1));
      float gl = len3(gn);
      if (gl > 1e-6f) {
        f3 n = mkf3(gn.x / gl, gn.y / gl, gn.z / gl);
        float vn = dot3(v, n);
        if (vn < 0.f) v = mkf3(v.x - vn * n.x, v.y - vn * n.y, v.z - vn * n.z);
      }
    }
  }
  vout = make_float3(v.x, v.y, v.z);
  return true;
}

// ---------------------------------------------------------------- G2P
// Gather of mpm_g2p.comp:87-118 through a node accessor: vpic, vpic_old,
// grad v (G) and the APIC B (both GLSL [col][row]).
template <class Grid>
__device__ __forceinline__ void g2pGather(const SubstepParams& P, const PState& s, const Grid& grid, float vpic[3], float vpo[3], float G[3][3],
                                          float Bn[3][3]) {
  const float h = P.cellSize;
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  int base[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) base[a] = int(floorf(__fdiv_rn(xp[a] - P.worldMin[a], h))) - 1;
  const bool flip = P.flip_ratio > 0.01f;
#pragma unroll
  for (int i = 0; i < 3; ++i) vpic[i] = vpo[i] = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) { G[a][b] = 0.f; Bn[a][b] = 0.f; }
  float wa[3][3], ga[3][3], xi[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      xi[a][k] = nodeCentre(P, a, base[a] + k);
      float d = __fdiv_rn(xp[a] - xi[a][k], h);
      wa[a][k] = bspline2(d);
      ga[a][k] = bspline2g(d);
    }
#pragma unroll
  for (int iz = 0; iz < 3; iz++)
#pragma unroll
    for (int iy = 0; iy < 3; iy++)
#pragma unroll
      for (int ix = 0; ix < 3; ix++) {
        const int nx = base[0] + ix, ny = base[1] + iy, nz = base[2] + iz;
        if (nx < 0 || ny < 0 || nz < 0 || nx >= P.gridRes[0] || ny >= P.gridRes[1] || nz >= P.gridRes[2]) continue;
        float mass;
        float3 vi, vo;
        if (!grid.node(nx, ny, nz, mass, vi, vo)) continue;
        if (mass < 1e-10f) continue;
        const float wx = wa[0][ix], wy = wa[1][iy], wz = wa[2][iz];
        const float w = wx * wy * wz;
        if (w < 1e-12f) continue;
        const float dw[3] = {__fdiv_rn(ga[0][ix] * wy * wz, h), __fdiv_rn(wx * ga[1][iy] * wz, h), __fdiv_rn(wx * wy * ga[2][iz], h)};
        const float r[3] = {xi[0][ix] - xp[0], xi[1][iy] - xp[1], xi[2][iz] - xp[2]};
        const float v3[3] = {vi.x, vi.y, vi.z};
#pragma unroll
        for (int i = 0; i < 3; ++i) vpic[i] += w * v3[i];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            G[j][i] += v3[i] * dw[j];
            Bn[j][i] += w * (v3[i] * r[j]);
          }
        if (flip) {
          vpo[0] += w * vo.x;
          vpo[1] += w * vo.y;
          vpo[2] += w * vo.z;
        }
      }
}

// The same gather from a brick's staged 6^3 node block (origin sx,sy,sz) whose
// velocities are zero where the node is outside [0, gridRes) or lighter than
// 1e-10 -- exactly the nodes the shader skips.  The B-spline weights are
// products of 1D factors, so sums run along x first for each (dy, dz) and are
// then scaled by the y/z factors.  Returns false when the particle's stencil
// is not inside the block (the caller then uses g2pGather).
template <bool FLIP>
__device__ __forceinline__ bool g2pGatherStaged(const SubstepParams& P, const PState& s, const float4* __restrict__ sv, const float4* __restrict__ svo,
                                                int sx, int sy, int sz, float vpic[3], float vpo[3], float G[3][3], float Bn[3][3]) {
  const float h = P.cellSize, invH = 1.0f / P.cellSize;
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  int base[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) base[a] = int(floorf(__fdiv_rn(xp[a] - P.worldMin[a], h))) - 1;
  const int lx = base[0] - sx, ly = base[1] - sy, lz = base[2] - sz;
  if ((unsigned)lx > 3u || (unsigned)ly > 3u || (unsigned)lz > 3u) return false;
  float W[3][3], Gd[3][3], R[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float xi = nodeCentre(P, a, base[a] + k);
      d[k] = (xp[a] - xi) * invH;
      R[a][k] = xi - xp[a];
    }
    bsplineStencil(d[0], d[1], d[2], W[a], Gd[a]);
#pragma unroll
    for (int k = 0; k < 3; ++k) Gd[a][k] *= invH;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) vpic[i] = vpo[i] = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) { G[a][b] = 0.f; Bn[a][b] = 0.f; }
#pragma unroll
  for (int dz = 0; dz < 3; ++dz)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
      float Sw[3] = {0.f, 0.f, 0.f}, Sr[3] = {0.f, 0.f, 0.f}, Sg[3] = {0.f, 0.f, 0.f}, So[3] = {0.f, 0.f, 0.f};
      const int q0 = ((lz + dz) * 6 + (ly + dy)) * 6 + lx;
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const float4 a = sv[q0 + dx];
        const float wx = W[0][dx], wr = W[0][dx] * R[0][dx], gx = Gd[0][dx];
        Sw[0] += wx * a.x; Sw[1] += wx * a.y; Sw[2] += wx * a.z;
        Sr[0] += wr * a.x; Sr[1] += wr * a.y; Sr[2] += wr * a.z;
        Sg[0] += gx * a.x; Sg[1] += gx * a.y; Sg[2] += gx * a.z;
        if (FLIP) {
          const float4 o = svo[q0 + dx];
          So[0] += wx * o.x; So[1] += wx * o.y; So[2] += wx * o.z;
        }
      }
      const float wyz = W[1][dy] * W[2][dz];
      const float byy = W[1][dy] * R[1][dy] * W[2][dz];
      const float bzz = wyz * R[2][dz];
      const float gyy = Gd[1][dy] * W[2][dz];
      const float gzz = W[1][dy] * Gd[2][dz];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        vpic[i] += wyz * Sw[i];
        Bn[0][i] += wyz * Sr[i];
        Bn[1][i] += byy * Sw[i];
        Bn[2][i] += bzz * Sw[i];
        G[0][i] += wyz * Sg[i];
        G[1][i] += gyy * Sw[i];
        G[2][i] += gzz * Sw[i];
        if (FLIP) vpo[i] += wyz * So[i];
      }
    }
  return true;
}

// Material-model sets the particle update is compiled for: any model
// (dispatched per particle), or a scene whose every material is of one family,
// for which the update holds only that family's code (a smaller kernel with
// fewer values live across the stress; chosen by the host from the material
// table).
enum ModelSet : int {
  kModelsAny = 0,
  kModelsElastic = 1,        // ELASTIC (Hencky) only
  kModelsDruckerPrager = 2,  // DRUCKER_PRAGER and GRANULAR_POWDER (the same return map, no viscosity)
  kModelsElasticVonMises = 3,  // ELASTIC and VON_MISES
  kModelsElasticDruckerPrager = 4,  // ELASTIC and the Drucker-Prager family
};

// Everything of mpm_g2p.comp after the gather (lines 120-271): material,
// F update, return map, stress, J reset, transfer, advection, SDF push-out,
// world clamp, write-back.  Returns event bits (1 J reset, 2 SDF push-out).
template <int MS = kModelsAny>
__device__ __forceinline__ uint32_t g2pUpdate(const SubstepParams& P, PState& s, float dt, const float vpic[3], const float vpo[3],
                                              const float G[3][3], float Bn[3][3]) {
  const float h = P.cellSize;
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  const bool flip = P.flip_ratio > 0.01f;
  const MatSample mat = fetchMaterial(P, __float_as_uint(s.v.w));
  // F_new = (I + dt grad v) F
  m3<float> F, A;
  F.m[0][0] = s.F0.x; F.m[0][1] = s.F0.y; F.m[0][2] = s.F0.z;
  F.m[1][0] = s.F1.x; F.m[1][1] = s.F1.y; F.m[1][2] = s.F1.z;
  F.m[2][0] = s.F2.x; F.m[2][1] = s.F2.y; F.m[2][2] = s.F2.z;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) A.m[a][b] = (a == b ? 1.f : 0.f) + dt * G[a][b];
  m3<float> Fn = m3mul(A, F);
  m3<float> tau;
  if constexpr (MS == kModelsDruckerPrager) {
    plasticReturn(MAT_DRUCKER_PRAGER, Fn, tau, mat.mu, mat.lam, mat.M, mat.qc, mat.qmax);
  } else if constexpr (MS == kModelsElastic) {
    tau = henckyStress<float>(Fn, mat.mu, mat.lam);
  } else if constexpr (MS == kModelsElasticVonMises) {
    if (mat.model == MAT_VON_MISES) plasticReturn(MAT_VON_MISES, Fn, tau, mat.mu, mat.lam, mat.M, mat.qc, mat.qmax);
    else tau = henckyStress<float>(Fn, mat.mu, mat.lam);
  } else if constexpr (MS == kModelsElasticDruckerPrager) {
    if (mat.model == MAT_ELASTIC) tau = henckyStress<float>(Fn, mat.mu, mat.lam);
    else plasticReturn(MAT_DRUCKER_PRAGER, Fn, tau, mat.mu, mat.lam, mat.M, mat.qc, mat.qmax);
  } else if (mat.model == MAT_FLUID) {
    float J = fmaxf(m3det(Fn), 1e-4f);
    float c = powf(J, 1.0f / 3.0f);
    Fn = m3zero<float>();
    Fn.m[0][0] = Fn.m[1][1] = Fn.m[2][2] = c;
    float pr = mat.bulkK * (J - 1.0f);
    tau = m3zero<float>();
    tau.m[0][0] = tau.m[1][1] = tau.m[2][2] = pr;
  } else if (mat.model == MAT_VON_MISES || mat.model == MAT_DRUCKER_PRAGER || mat.model == MAT_GRANULAR_POWDER ||
             mat.model == MAT_VISCOPLASTIC_MUD) {
    const uint32_t rm = mat.model == MAT_VON_MISES ? MAT_VON_MISES : MAT_DRUCKER_PRAGER;
    plasticReturn(rm, Fn, tau, mat.mu, mat.lam, mat.M, mat.qc, mat.qmax);
    if (mat.model == MAT_VISCOPLASTIC_MUD) {
      float D[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) D[a][b] = 0.5f * (G[a][b] + G[b][a]);
      float trD = D[0][0] + D[1][1] + D[2][2];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) tau.m[a][b] += (2.0f * mat.visc) * (D[a][b] - (a == b ? trD / 3.0f : 0.f));
    }
  } else if (mat.model == MAT_FIXED_COROTATED) {
    tau = fixedCorotatedStress<float>(Fn, mat.mu, mat.lam);
  } else {
    tau = henckyStress<float>(Fn, mat.mu, mat.lam);
  }
  uint32_t events = 0;
  bool j_reset = false;
  {
    float Jd = fabsf(m3det(Fn));
    if (Jd < 0.15f || Jd > 10.0f) {
      Fn = m3ident<float>();
      tau = m3zero<float>();
      j_reset = true;
      events |= 1u;
    }
  }
  if (P.flip_ratio > -0.5f) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) Bn[a][b] = 0.f;
  }
  float vn[3];
  if (flip) {
    const float vo[3] = {s.v.x, s.v.y, s.v.z};
    const float fr = P.flip_ratio;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float vf = vo[i] + (vpic[i] - vpo[i]);
      vn[i] = vpic[i] * (1.0f - fr) + vf * fr;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) vn[i] = vpic[i];
  }
  if (j_reset) {
#pragma unroll
    for (int i = 0; i < 3; ++i) vn[i] *= 0.1f;
  }
  float xn[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) xn[i] = xp[i] + dt * vn[i];

  if (P.sdf) {
    int pijk[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) pijk[a] = min(max(int(floorf(__fdiv_rn(xn[a] - P.worldMin[a], h))), 0), P.gridRes[a] - 1);
    auto at = [&](int x, int y, int z) { return __ldg(P.sdf + mortonEncode(x, y, z)); };
    float psdf = at(pijk[0], pijk[1], pijk[2]);
    if (psdf < 0.f) {
      auto cl = [&](int a, int v) { return min(max(v, 0), P.gridRes[a] - 1); };
      f3 gn = mkf3(at(cl(0, pijk[0] + 1), pijk[1], pijk[2]) - at(cl(0, pijk[0] - 1), pijk[1], pijk[2]),
                   at(pijk[0], cl(1, pijk[1] + 1), pijk[2]) - at(pijk[0], cl(1, pijk[1] - 1), pijk[2]),
                   at(pijk[0], pijk[1], cl(2, pijk[2] + 1)) - at(pijk[0], pijk[1], cl(2, pijk[2] - 1)));
      float gl = len3(gn);
      if (gl > 1e-6f) {
        f3 n = mkf3(gn.x / gl, gn.y / gl, gn.z / gl);
        xn[0] -= psdf * n.x; xn[1] -= psdf * n.y; xn[2] -= psdf * n.z;
        float vdn = vn[0] * n.x + vn[1] * n.y + vn[2] * n.z;
        if (vdn < 0.f) { vn[0] -= vdn * n.x; vn[1] -= vdn * n.y; vn[2] -= vdn * n.z; }
      } else {
        xn[0] = xp[0]; xn[1] = xp[1]; xn[2] = xp[2];
        vn[0] = vn[1] = vn[2] = 0.f;
      }
      Fn = m3ident<float>();
      tau = m3zero<float>();
      events |= 2u;
    }
  }
  const float margin = h * 1.5f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = P.worldMin[a] + margin, hi = P.worldMax[a] - margin;
    if (xn[a] < lo) { xn[a] = lo; vn[a] = fmaxf(vn[a], 0.f); }
    if (xn[a] > hi) { xn[a] = hi; vn[a] = fminf(vn[a], 0.f); }
  }
  s.P = make_float4(xn[0], xn[1], xn[2], s.P.w);
  s.v = make_float4(vn[0], vn[1], vn[2], s.v.w);
  s.F0 = make_float4(Fn.m[0][0], Fn.m[0][1], Fn.m[0][2], tau.m[0][0]);
  s.F1 = make_float4(Fn.m[1][0], Fn.m[1][1], Fn.m[1][2], tau.m[1][1]);
  s.F2 = make_float4(Fn.m[2][0], Fn.m[2][1], Fn.m[2][2], tau.m[2][2]);
  s.B0 = make_float4(Bn[0][0], Bn[0][1], Bn[0][2], tau.m[0][1]);
  s.B1 = make_float4(Bn[1][0], Bn[1][1], Bn[1][2], tau.m[0][2]);
  s.B2 = make_float4(Bn[2][0], Bn[2][1], Bn[2][2], tau.m[1][2]);
  return events;
}

// grid.node(nx, ny, nz, mass, vel, vold) returns false for nodes to skip.
template <class Grid>
__device__ __forceinline__ uint32_t g2pParticle(const SubstepParams& P, PState& s, const Grid& grid, float dt) {
  float vpic[3], vpo[3], G[3][3], Bn[3][3];
  g2pGather(P, s, grid, vpic, vpo, G, Bn);
  return g2pUpdate(P, s, dt, vpic, vpo, G, Bn);
}

}  // namespace nebula
