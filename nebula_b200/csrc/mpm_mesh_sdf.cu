// mpm_mesh_sdf.cu -- mesh -> Morton-ordered SDF on the GPU (buildMeshSDF,
// src/core/MeshSDF.h:98-132, with transformTriangles, MeshSDF.h:134-141,
// applied on the device).
//
// Same definition as the reference: for every cell centre (ix+0.5, iy+0.5,
// iz+0.5) * cellSize inside gridRes, the distance to the closest triangle,
// signed by that triangle's normal (outside when dot(p - cp, n) >= 0); the
// first triangle wins ties (strict <); cells of the Morton cube beyond gridRes
// hold 1e9.  The closest point is Ericson's complete region test: the
// reference's closestPtOnTriangle (MeshSDF.h:48-78) leaves out the edge-BC
// region and then returns a point outside the triangle (too short, wrongly
// signed distances); that case is added here.
//
// The reference loops over all cells x all triangles on the host.  Here a CTA
// owns 256 consecutive Morton codes (an 8 x 8 x 4 box of cells), one per
// thread, and culls the triangle list for the whole box before any thread
// computes a closest point:
//   1. U = min over triangles and their vertices of the distance from the
//      vertex to the farthest cell centre of the box.  Every cell of the box
//      has a triangle within U, so its closest distance is <= U.
//   2. The triangles are staged through shared memory in tiles of 256, in
//      list order.  A triangle whose bounding sphere is farther than U from
//      the box cannot be any cell's closest and is dropped from the tile; the
//      survivors are compacted in list order.
//   3. Each thread walks the survivors, skipping a triangle whose bounding
//      sphere is no closer than min(its best so far, U).
// Every skipped triangle is strictly farther than the cell's closest one (the
// bounds carry a margin above float rounding), so the distances and the
// winning triangle are those of the brute-force loop.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "mpm_device.cuh"
#include "mpm_engine.h"

namespace nebula {
namespace {

constexpr int kThreads = 256;  // = the Morton codes of one 8 x 8 x 4 box

struct TriS {  // a, b - a, c - a, normal, bounding sphere (centre, radius)
  float ax, ay, az, bx, by, bz, cx, cy, cz, nx, ny, nz, sx, sy, sz, sr;
};

__device__ __forceinline__ float dot3f(float ax, float ay, float az, float bx, float by, float bz) { return ax * bx + ay * by + az * bz; }

// glm::quat * vec3 for a unit quaternion (w, u): v + 2 (w (u x v) + u x (u x v)).
__device__ __forceinline__ void rotate(const MeshPose& q, float& vx, float& vy, float& vz) {
  const float cx = q.q[2] * vz - q.q[3] * vy, cy = q.q[3] * vx - q.q[1] * vz, cz = q.q[1] * vy - q.q[2] * vx;
  const float dx = q.q[2] * cz - q.q[3] * cy, dy = q.q[3] * cx - q.q[1] * cz, dz = q.q[1] * cy - q.q[2] * cx;
  vx += (cx * q.q[0] + dx) * 2.0f;
  vy += (cy * q.q[0] + dy) * 2.0f;
  vz += (cz * q.q[0] + dz) * 2.0f;
}

// Triangle k as (normal, v0, v1, v2), the binary STL order, after the pose.
__device__ __forceinline__ void loadTri(const float4* __restrict__ t4, uint32_t k, const MeshPose& p, float (&v)[12]) {
  const float4 r0 = __ldg(t4 + 3 * size_t(k)), r1 = __ldg(t4 + 3 * size_t(k) + 1), r2 = __ldg(t4 + 3 * size_t(k) + 2);
  v[0] = r0.x; v[1] = r0.y; v[2] = r0.z; v[3] = r0.w;
  v[4] = r1.x; v[5] = r1.y; v[6] = r1.z; v[7] = r1.w;
  v[8] = r2.x; v[9] = r2.y; v[10] = r2.z; v[11] = r2.w;
  if (p.posed) {
#pragma unroll
    for (int j = 0; j < 4; ++j) rotate(p, v[3 * j], v[3 * j + 1], v[3 * j + 2]);
#pragma unroll
    for (int j = 1; j < 4; ++j) {
      v[3 * j] += p.t[0];
      v[3 * j + 1] += p.t[1];
      v[3 * j + 2] += p.t[2];
    }
  }
}

// Closest point of triangle (a, a + ab, a + ac) to p (MeshSDF.h:48-78).
__device__ __forceinline__ void closestOnTriangle(const TriS& t, float px, float py, float pz, float& qx, float& qy, float& qz) {
  const float apx = px - t.ax, apy = py - t.ay, apz = pz - t.az;
  const float d1 = dot3f(t.bx, t.by, t.bz, apx, apy, apz), d2 = dot3f(t.cx, t.cy, t.cz, apx, apy, apz);
  if (d1 <= 0.f && d2 <= 0.f) {
    qx = t.ax; qy = t.ay; qz = t.az;
    return;
  }
  const float bpx = apx - t.bx, bpy = apy - t.by, bpz = apz - t.bz;  // p - b
  const float d3 = dot3f(t.bx, t.by, t.bz, bpx, bpy, bpz), d4 = dot3f(t.cx, t.cy, t.cz, bpx, bpy, bpz);
  if (d3 >= 0.f && d4 <= d3) {
    qx = t.ax + t.bx; qy = t.ay + t.by; qz = t.az + t.bz;
    return;
  }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    const float v = d1 / (d1 - d3);
    qx = t.ax + v * t.bx; qy = t.ay + v * t.by; qz = t.az + v * t.bz;
    return;
  }
  const float cpx = apx - t.cx, cpy = apy - t.cy, cpz = apz - t.cz;  // p - c
  const float d5 = dot3f(t.bx, t.by, t.bz, cpx, cpy, cpz), d6 = dot3f(t.cx, t.cy, t.cz, cpx, cpy, cpz);
  if (d6 >= 0.f && d5 <= d6) {
    qx = t.ax + t.cx; qy = t.ay + t.cy; qz = t.az + t.cz;
    return;
  }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    const float w = d2 / (d2 - d6);
    qx = t.ax + w * t.cx; qy = t.ay + w * t.cy; qz = t.az + w * t.cz;
    return;
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {  // edge BC (Ericson 5.1.5; left out by MeshSDF.h:76-78)
    const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    qx = t.ax + t.bx + w * (t.cx - t.bx); qy = t.ay + t.by + w * (t.cy - t.by); qz = t.az + t.bz + w * (t.cz - t.bz);
    return;
  }
  const float sum = va + vb + vc;
  const float v = vb / sum, w = vc / sum;
  qx = t.ax + v * t.bx + w * t.cx;
  qy = t.ay + v * t.by + w * t.cy;
  qz = t.az + v * t.bz + w * t.cz;
}

__global__ void __launch_bounds__(kThreads) k_mesh_sdf(const float4* __restrict__ tris, uint32_t n, MeshPose pose, int rx, int ry, int rz,
                                                       uint32_t totalCells, float cs, float eps, float* __restrict__ sdf) {
  __shared__ TriS tile[kThreads];
  __shared__ uint32_t warpCount[kThreads / 32];
  __shared__ uint32_t boundBits;
  const uint32_t base = blockIdx.x * kThreads;
  const uint32_t code = base + threadIdx.x;
  int bx0, by0, bz0;
  mortonDecode(base, bx0, by0, bz0);
  if (bx0 >= rx || by0 >= ry || bz0 >= rz) {  // the whole box lies in the padding of the Morton cube
    if (code < totalCells) sdf[code] = 1e9f;
    return;
  }
  int bx1, by1, bz1;
  mortonDecode(base | uint32_t(kThreads - 1), bx1, by1, bz1);
  const float lox = (float(bx0) + 0.5f) * cs, loy = (float(by0) + 0.5f) * cs, loz = (float(bz0) + 0.5f) * cs;
  const float hix = (float(min(bx1, rx - 1)) + 0.5f) * cs, hiy = (float(min(by1, ry - 1)) + 0.5f) * cs, hiz = (float(min(bz1, rz - 1)) + 0.5f) * cs;

  // 1. U^2 over the box
  if (threadIdx.x == 0) boundBits = __float_as_uint(INFINITY);
  __syncthreads();
  float u2 = INFINITY;
  for (uint32_t k = threadIdx.x; k < n; k += kThreads) {
    float v[12];
    loadTri(tris, k, pose, v);
#pragma unroll
    for (int j = 1; j < 4; ++j) {
      const float ex = fmaxf(v[3 * j] - lox, hix - v[3 * j]);
      const float ey = fmaxf(v[3 * j + 1] - loy, hiy - v[3 * j + 1]);
      const float ez = fmaxf(v[3 * j + 2] - loz, hiz - v[3 * j + 2]);
      u2 = fminf(u2, ex * ex + ey * ey + ez * ez);
    }
  }
  u2 = __uint_as_float(__reduce_min_sync(0xffffffffu, __float_as_uint(u2)));  // non-negative floats order as their bits
  if ((threadIdx.x & 31) == 0) atomicMin(&boundBits, __float_as_uint(u2));
  __syncthreads();
  const float U = sqrtf(__uint_as_float(boundBits)) * (1.0f + 1e-5f) + eps;

  int ix = 0, iy = 0, iz = 0;
  if (code < totalCells) mortonDecode(code, ix, iy, iz);
  const bool inside = code < totalCells && ix < rx && iy < ry && iz < rz;
  const float px = (float(ix) + 0.5f) * cs, py = (float(iy) + 0.5f) * cs, pz = (float(iz) + 0.5f) * cs;
  float best = 1e9f;
  bool outer = true;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t t0 = 0; t0 < n; t0 += kThreads) {
    // 2. stage the tile's triangles that can be closest to some cell of the box
    const uint32_t k = t0 + threadIdx.x;
    TriS t;
    bool keep = false;
    if (k < n) {
      float v[12];
      loadTri(tris, k, pose, v);
      t.nx = v[0]; t.ny = v[1]; t.nz = v[2];
      t.ax = v[3]; t.ay = v[4]; t.az = v[5];
      t.bx = v[6] - v[3]; t.by = v[7] - v[4]; t.bz = v[8] - v[5];
      t.cx = v[9] - v[3]; t.cy = v[10] - v[4]; t.cz = v[11] - v[5];
      t.sx = (v[3] + v[6] + v[9]) * (1.0f / 3.0f);
      t.sy = (v[4] + v[7] + v[10]) * (1.0f / 3.0f);
      t.sz = (v[5] + v[8] + v[11]) * (1.0f / 3.0f);
      float rr = 0.f;
#pragma unroll
      for (int j = 1; j < 4; ++j) {
        const float dx = v[3 * j] - t.sx, dy = v[3 * j + 1] - t.sy, dz = v[3 * j + 2] - t.sz;
        rr = fmaxf(rr, dx * dx + dy * dy + dz * dz);
      }
      t.sr = sqrtf(rr) * 1.0001f + eps;  // covers the triangle despite rounding
      const float gx = fmaxf(fmaxf(lox - t.sx, t.sx - hix), 0.f), gy = fmaxf(fmaxf(loy - t.sy, t.sy - hiy), 0.f),
                  gz = fmaxf(fmaxf(loz - t.sz, t.sz - hiz), 0.f);
      keep = sqrtf(gx * gx + gy * gy + gz * gz) - t.sr <= U;
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, keep);
    __syncthreads();  // the previous tile has been consumed
    if (lane == 0) warpCount[warp] = __popc(mask);
    __syncthreads();
    uint32_t off = 0, m = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      const uint32_t c = warpCount[w];
      off += uint32_t(w) < warp ? c : 0u;
      m += c;
    }
    if (keep) tile[off + __popc(mask & ((1u << lane) - 1u))] = t;
    __syncthreads();
    if (!inside) continue;
    // 3. closest points against the survivors, in list order
    for (uint32_t j = 0; j < m; ++j) {
      const TriS& s = tile[j];
      const float ex = px - s.sx, ey = py - s.sy, ez = pz - s.sz;
      const float dc = sqrtf(ex * ex + ey * ey + ez * ez);
      if (dc - s.sr >= fminf(best, U)) continue;  // every point of the triangle is at least this far
      float qx, qy, qz;
      closestOnTriangle(s, px, py, pz, qx, qy, qz);
      const float dx = px - qx, dy = py - qy, dz = pz - qz;
      const float d = sqrtf(dx * dx + dy * dy + dz * dz);
      if (d < best) {
        best = d;
        outer = dot3f(dx, dy, dz, s.nx, s.ny, s.nz) >= 0.f;
      }
    }
  }
  if (code < totalCells) sdf[code] = inside ? (outer ? best : -best) : 1e9f;
}

// ---------------------------------------------------------------- prepared meshes
// The same SDF from a prepared mesh: triangles sorted by the Morton code of
// their centroids and grouped in clusters of 32 with a bounding sphere each,
// so culling works on clusters before triangles.  Per CTA (the 256 cells of an
// 8 x 8 x 4 box):
//   1. U from one vertex of every cluster (a point on the mesh).
//   2. Clusters in tiles of 256: those whose sphere comes within U of the box
//      are compacted; eight at a time, warp w stages the 32 triangles of one
//      of them and keeps those whose own sphere comes within U of the box.
//   3. Each thread first tests the triangles of the cluster that gave U (near
//      every cell of the box), then skips any cluster whose sphere is no
//      closer than min(its best so far, U) and tests the kept triangles of
//      the others as before.
// Triangles are visited out of list order, so a tie in distance goes to the
// smaller list index: the first triangle of the list reaching the minimum,
// as in the brute-force loop.
__device__ __forceinline__ void loadTriS(const float4* __restrict__ t4, uint32_t k, const MeshPose& pose, float eps, TriS& t) {
  float v[12];
  loadTri(t4, k, pose, v);
  t.nx = v[0]; t.ny = v[1]; t.nz = v[2];
  t.ax = v[3]; t.ay = v[4]; t.az = v[5];
  t.bx = v[6] - v[3]; t.by = v[7] - v[4]; t.bz = v[8] - v[5];
  t.cx = v[9] - v[3]; t.cy = v[10] - v[4]; t.cz = v[11] - v[5];
  t.sx = (v[3] + v[6] + v[9]) * (1.0f / 3.0f);
  t.sy = (v[4] + v[7] + v[10]) * (1.0f / 3.0f);
  t.sz = (v[5] + v[8] + v[11]) * (1.0f / 3.0f);
  float rr = 0.f;
#pragma unroll
  for (int j = 1; j < 4; ++j) {
    const float dx = v[3 * j] - t.sx, dy = v[3 * j + 1] - t.sy, dz = v[3 * j + 2] - t.sz;
    rr = fmaxf(rr, dx * dx + dy * dy + dz * dz);
  }
  t.sr = sqrtf(rr) * 1.0001f + eps;
}

// Distance from point s to the box [lo, hi] (0 inside).
__device__ __forceinline__ float boxDistance(float lox, float loy, float loz, float hix, float hiy, float hiz, float sx, float sy, float sz) {
  const float gx = fmaxf(fmaxf(lox - sx, sx - hix), 0.f), gy = fmaxf(fmaxf(loy - sy, sy - hiy), 0.f), gz = fmaxf(fmaxf(loz - sz, sz - hiz), 0.f);
  return sqrtf(gx * gx + gy * gy + gz * gz);
}

__global__ void __launch_bounds__(kThreads) k_mesh_sdf_clusters(const float4* __restrict__ tris, const uint32_t* __restrict__ index,
                                                                const float4* __restrict__ spheres, uint32_t n, uint32_t nClusters, MeshPose pose,
                                                                int rx, int ry, int rz, uint32_t totalCells, float cs, float eps,
                                                                float* __restrict__ sdf) {
  constexpr int kWarps = kThreads / 32;
  __shared__ TriS tile[kThreads];
  __shared__ uint32_t tileIdx[kThreads];
  __shared__ float4 clus[kThreads];       // surviving clusters of the current cluster tile: posed centre, radius
  __shared__ uint32_t clusId[kThreads];
  __shared__ uint32_t warpCount[kWarps];
  __shared__ uint32_t runStart[kWarps + 1];  // kept triangles of the staged clusters: [runStart[w], runStart[w + 1])
  __shared__ unsigned long long boundKey;    // (U^2 bits, cluster): the bound and the cluster that gave it
  const uint32_t base = blockIdx.x * kThreads;
  const uint32_t code = base + threadIdx.x;
  int bx0, by0, bz0;
  mortonDecode(base, bx0, by0, bz0);
  if (bx0 >= rx || by0 >= ry || bz0 >= rz) {
    if (code < totalCells) sdf[code] = 1e9f;
    return;
  }
  int bx1, by1, bz1;
  mortonDecode(base | uint32_t(kThreads - 1), bx1, by1, bz1);
  const float lox = (float(bx0) + 0.5f) * cs, loy = (float(by0) + 0.5f) * cs, loz = (float(bz0) + 0.5f) * cs;
  const float hix = (float(min(bx1, rx - 1)) + 0.5f) * cs, hiy = (float(min(by1, ry - 1)) + 0.5f) * cs, hiz = (float(min(bz1, rz - 1)) + 0.5f) * cs;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // 1. U^2 over the box from the first vertex of every cluster, and the
  //    cluster that gives it (non-negative floats order as their bits)
  if (threadIdx.x == 0) boundKey = ~0ull;
  __syncthreads();
  unsigned long long key = ~0ull;
  for (uint32_t c = threadIdx.x; c < nClusters; c += kThreads) {
    float v[12];
    loadTri(tris, c * kMeshCluster, pose, v);
    const float ex = fmaxf(v[3] - lox, hix - v[3]), ey = fmaxf(v[4] - loy, hiy - v[4]), ez = fmaxf(v[5] - loz, hiz - v[5]);
    const unsigned long long k = (static_cast<unsigned long long>(__float_as_uint(ex * ex + ey * ey + ez * ez)) << 32) | c;
    key = k < key ? k : key;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  if (lane == 0) atomicMin(&boundKey, key);
  __syncthreads();
  const unsigned long long bk = boundKey;
  const float U = nClusters ? sqrtf(__uint_as_float(uint32_t(bk >> 32))) * (1.0f + 1e-5f) + eps : INFINITY;
  const uint32_t firstCluster = uint32_t(bk & 0xffffffffu);

  int ix = 0, iy = 0, iz = 0;
  if (code < totalCells) mortonDecode(code, ix, iy, iz);
  const bool inside = code < totalCells && ix < rx && iy < ry && iz < rz;
  const float px = (float(ix) + 0.5f) * cs, py = (float(iy) + 0.5f) * cs, pz = (float(iz) + 0.5f) * cs;
  float best = 1e9f;
  uint32_t bestIdx = 0xffffffffu;
  bool outer = true;
  auto visit = [&](const TriS& s, uint32_t id) {
    const float fx = px - s.sx, fy = py - s.sy, fz = pz - s.sz;
    const float dt = sqrtf(fx * fx + fy * fy + fz * fz);
    if (dt - s.sr >= fminf(best, U)) return;  // every point of the triangle is at least this far
    float qx, qy, qz;
    closestOnTriangle(s, px, py, pz, qx, qy, qz);
    const float dx = px - qx, dy = py - qy, dz = pz - qz;
    const float d = sqrtf(dx * dx + dy * dy + dz * dz);
    if (d < best || (d == best && id < bestIdx)) {
      best = d;
      bestIdx = id;
      outer = dot3f(dx, dy, dz, s.nx, s.ny, s.nz) >= 0.f;
    }
  };
  // the cluster that gave U first: near every cell of the box, it makes each
  // thread's bound tight before the other clusters are tested
  if (nClusters) {
    if (warp == 0) {
      const uint32_t t = firstCluster * kMeshCluster + lane;
      if (t < n) {
        loadTriS(tris, t, pose, eps, tile[lane]);
        tileIdx[lane] = index[t];
      }
    }
    __syncthreads();
    if (inside) {
      const uint32_t m = min(kMeshCluster, n - firstCluster * kMeshCluster);
      for (uint32_t j = 0; j < m; ++j) visit(tile[j], tileIdx[j]);
    }
  }
  for (uint32_t c0 = 0; c0 < nClusters; c0 += kThreads) {
    // 2a. the tile's clusters that can hold the closest triangle of some cell of the box
    const uint32_t c = c0 + threadIdx.x;
    bool keep = false;
    float4 sph = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c < nClusters) {
      sph = spheres[c];
      if (pose.posed) {
        rotate(pose, sph.x, sph.y, sph.z);
        sph.x += pose.t[0];
        sph.y += pose.t[1];
        sph.z += pose.t[2];
      }
      keep = boxDistance(lox, loy, loz, hix, hiy, hiz, sph.x, sph.y, sph.z) - sph.w <= U;
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, keep);
    __syncthreads();  // the previous cluster tile is consumed
    if (lane == 0) warpCount[warp] = __popc(mask);
    __syncthreads();
    uint32_t off = 0, mC = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t k = warpCount[w];
      off += uint32_t(w) < warp ? k : 0u;
      mC += k;
    }
    if (keep) {
      const uint32_t at = off + __popc(mask & ((1u << lane) - 1u));
      clus[at] = sph;
      clusId[at] = c;
    }
    __syncthreads();
    for (uint32_t k0 = 0; k0 < mC; k0 += kWarps) {
      // 2b. warp w stages the triangles of surviving cluster k0 + w
      const uint32_t kc = k0 + warp;
      const uint32_t t = kc < mC ? clusId[kc] * kMeshCluster + lane : n;
      TriS tri;
      bool keepT = false;
      if (t < n) {
        loadTriS(tris, t, pose, eps, tri);
        keepT = boxDistance(lox, loy, loz, hix, hiy, hiz, tri.sx, tri.sy, tri.sz) - tri.sr <= U;
      }
      const uint32_t tm = __ballot_sync(0xffffffffu, keepT);
      __syncthreads();  // the previous staging is consumed
      if (lane == 0) warpCount[warp] = __popc(tm);
      __syncthreads();
      if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int w = 0; w < kWarps; ++w) {
          runStart[w] = acc;
          acc += warpCount[w];
        }
        runStart[kWarps] = acc;
      }
      uint32_t toff = 0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) toff += uint32_t(w) < warp ? warpCount[w] : 0u;
      if (keepT) {
        const uint32_t at = toff + __popc(tm & ((1u << lane) - 1u));
        tile[at] = tri;
        tileIdx[at] = index[t];
      }
      __syncthreads();
      if (!inside) continue;
      // 3. per cell: clusters first, then their kept triangles
      const uint32_t nk = min(uint32_t(kWarps), mC - k0);
      for (uint32_t w = 0; w < nk; ++w) {
        const float4 cw = clus[k0 + w];
        const float ex = px - cw.x, ey = py - cw.y, ez = pz - cw.z;
        const float dc = sqrtf(ex * ex + ey * ey + ez * ez);
        if (dc - cw.w >= fminf(best, U)) continue;  // every point of the cluster is at least this far
        for (uint32_t j = runStart[w]; j < runStart[w + 1]; ++j) visit(tile[j], tileIdx[j]);
      }
    }
  }
  if (code < totalCells) sdf[code] = inside ? (outer ? best : -best) : 1e9f;
}

// ------------------------------------------------------------------ the reference's closest point
// closestPtOnTriangle (MeshSDF.h:48-78) step for step, including its gap: a
// point whose closest feature is edge BC falls through to the barycentric
// face case and gets the projection onto the triangle's plane, outside the
// triangle.  That point can be nearer than any point of the triangle, so no
// distance bound culls triangles here: every cell visits every triangle, as
// buildMeshSDF's loop does (MeshSDF.h:113-126).
struct TriRef {  // posed vertices and normal
  float ax, ay, az, bx, by, bz, cx, cy, cz, nx, ny, nz;
};

// Float operations rounded one at a time, in the reference's order (no fused
// multiply-add): the missing region makes the result jump where a region test
// flips, so its arithmetic is kept operation for operation.
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float subr(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dotr(float ax, float ay, float az, float bx, float by, float bz) {
  return addr(addr(mulr(ax, bx), mulr(ay, by)), mulr(az, bz));
}

__device__ __forceinline__ void closestRef(const TriRef& t, float px, float py, float pz, float& qx, float& qy, float& qz) {
  const float abx = subr(t.bx, t.ax), aby = subr(t.by, t.ay), abz = subr(t.bz, t.az);
  const float acx = subr(t.cx, t.ax), acy = subr(t.cy, t.ay), acz = subr(t.cz, t.az);
  const float apx = subr(px, t.ax), apy = subr(py, t.ay), apz = subr(pz, t.az);
  const float d1 = dotr(abx, aby, abz, apx, apy, apz), d2 = dotr(acx, acy, acz, apx, apy, apz);
  if (d1 <= 0.f && d2 <= 0.f) {
    qx = t.ax; qy = t.ay; qz = t.az;
    return;
  }
  const float bpx = subr(px, t.bx), bpy = subr(py, t.by), bpz = subr(pz, t.bz);
  const float d3 = dotr(abx, aby, abz, bpx, bpy, bpz), d4 = dotr(acx, acy, acz, bpx, bpy, bpz);
  if (d3 >= 0.f && d4 <= d3) {
    qx = t.bx; qy = t.by; qz = t.bz;
    return;
  }
  const float vc = subr(mulr(d1, d4), mulr(d3, d2));
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    const float v = __fdiv_rn(d1, subr(d1, d3));
    qx = addr(t.ax, mulr(v, abx)); qy = addr(t.ay, mulr(v, aby)); qz = addr(t.az, mulr(v, abz));
    return;
  }
  const float cpx = subr(px, t.cx), cpy = subr(py, t.cy), cpz = subr(pz, t.cz);
  const float d5 = dotr(abx, aby, abz, cpx, cpy, cpz), d6 = dotr(acx, acy, acz, cpx, cpy, cpz);
  if (d6 >= 0.f && d5 <= d6) {
    qx = t.cx; qy = t.cy; qz = t.cz;
    return;
  }
  const float vb = subr(mulr(d5, d2), mulr(d1, d6));
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    const float w = __fdiv_rn(d2, subr(d2, d6));
    qx = addr(t.ax, mulr(w, acx)); qy = addr(t.ay, mulr(w, acy)); qz = addr(t.az, mulr(w, acz));
    return;
  }
  const float va = subr(mulr(d3, d6), mulr(d5, d4));
  const float sum = addr(addr(va, vb), vc);
  const float v = __fdiv_rn(vb, sum), w = __fdiv_rn(vc, sum);
  qx = addr(addr(t.ax, mulr(v, abx)), mulr(w, acx));
  qy = addr(addr(t.ay, mulr(v, aby)), mulr(w, acy));
  qz = addr(addr(t.az, mulr(v, abz)), mulr(w, acz));
}

// One thread per Morton code; the (posed) triangles pass through shared
// memory in tiles of kThreads.  `index` (may be null: list order) gives each
// triangle's place in the caller's list, so a list in another order still
// resolves equal distances to the first triangle of the caller's list, as
// the strict < of the reference's loop does.
__global__ void __launch_bounds__(kThreads) k_mesh_sdf_ref(const float4* __restrict__ tris, const uint32_t* __restrict__ index, uint32_t n,
                                                           MeshPose pose, int rx, int ry, int rz, uint32_t totalCells, float cs,
                                                           float* __restrict__ sdf) {
  __shared__ TriRef tile[kThreads];
  __shared__ uint32_t tileIdx[kThreads];
  const uint32_t code = blockIdx.x * kThreads + threadIdx.x;
  int ix, iy, iz;
  mortonDecode(code, ix, iy, iz);
  const bool inside = code < totalCells && ix < rx && iy < ry && iz < rz;
  const float px = mulr(addr(float(ix), 0.5f), cs), py = mulr(addr(float(iy), 0.5f), cs), pz = mulr(addr(float(iz), 0.5f), cs);
  float best = 1e9f;
  uint32_t bestIdx = 0xffffffffu;
  bool outer = true;
  for (uint32_t t0 = 0; t0 < n; t0 += kThreads) {
    __syncthreads();  // the previous tile is consumed
    const uint32_t t = t0 + threadIdx.x;
    if (t < n) {
      float v[12];
      loadTri(tris, t, pose, v);
      tile[threadIdx.x] = TriRef{v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11], v[0], v[1], v[2]};
      tileIdx[threadIdx.x] = index ? __ldg(index + t) : t;
    }
    __syncthreads();
    if (!inside) continue;
    const uint32_t m = min(uint32_t(kThreads), n - t0);
    for (uint32_t j = 0; j < m; ++j) {
      const TriRef& tr = tile[j];
      float qx, qy, qz;
      closestRef(tr, px, py, pz, qx, qy, qz);
      const float dx = subr(px, qx), dy = subr(py, qy), dz = subr(pz, qz);
      const float d = __fsqrt_rn(dotr(dx, dy, dz, dx, dy, dz));
      const uint32_t id = tileIdx[j];
      if (d < best || (d == best && id < bestIdx)) {
        best = d;
        bestIdx = id;
        outer = dotr(dx, dy, dz, tr.nx, tr.ny, tr.nz) >= 0.f;
      }
    }
  }
  if (code < totalCells) sdf[code] = inside ? (outer ? best : -best) : 1e9f;
}

}  // namespace

cudaError_t launchMeshSdfReference(const float* dTris, const uint32_t* dIndex, uint32_t n, const MeshPose& pose, const uint32_t res[3],
                                   uint32_t totalCells, float cellSize, float* dSdf, cudaStream_t s, uint64_t* launches) {
  if (totalCells == 0) return cudaSuccess;
  k_mesh_sdf_ref<<<(totalCells + kThreads - 1) / kThreads, kThreads, 0, s>>>(reinterpret_cast<const float4*>(dTris), dIndex, n, pose, int(res[0]),
                                                                             int(res[1]), int(res[2]), totalCells, cellSize, dSdf);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchMeshSdf(const float* dTris, uint32_t n, const MeshPose& pose, const uint32_t res[3], uint32_t totalCells, float cellSize,
                          float* dSdf, cudaStream_t s, uint64_t* launches) {
  if (totalCells == 0) return cudaSuccess;
  // Margin of the culling bounds over float rounding: distances within the
  // domain are O(cellSize * cubeRes).
  const float extent = cellSize * float(domainCubeRes(res));
  const float eps = 1e-5f * fmaxf(extent, 1.0f);
  k_mesh_sdf<<<(totalCells + kThreads - 1) / kThreads, kThreads, 0, s>>>(reinterpret_cast<const float4*>(dTris), n, pose, int(res[0]),
                                                                         int(res[1]), int(res[2]), totalCells, cellSize, eps, dSdf);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchMeshSdfPrepared(const PreparedMesh& m, const MeshPose& pose, const uint32_t res[3], uint32_t totalCells, float cellSize,
                                  float* dSdf, cudaStream_t s, uint64_t* launches) {
  if (totalCells == 0) return cudaSuccess;
  const float extent = cellSize * float(domainCubeRes(res));
  const float eps = 1e-5f * fmaxf(extent, 1.0f);
  k_mesh_sdf_clusters<<<(totalCells + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      static_cast<const float4*>(m.tris.ptr), static_cast<const uint32_t*>(m.index.ptr), static_cast<const float4*>(m.spheres.ptr), m.n, m.clusters,
      pose, int(res[0]), int(res[1]), int(res[2]), totalCells, cellSize, eps, dSdf);
  ++*launches;
  return cudaGetLastError();
}

// Sort by the Morton code of the centroid (10 bits per axis over the mesh's
// bounding box; ties by list index), group runs of kMeshCluster, and bound
// each run by the sphere around its vertices' bounding box.
void PreparedMesh::build(const float* h, uint32_t count) {
  checkMeshArgs(h, count);
  n = count;
  clusters = (count + kMeshCluster - 1) / kMeshCluster;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  std::vector<float> cen(size_t(count) * 3);
  for (uint32_t k = 0; k < count; ++k)
    for (int a = 0; a < 3; ++a) {
      const float c = (h[12 * size_t(k) + 3 + a] + h[12 * size_t(k) + 6 + a] + h[12 * size_t(k) + 9 + a]) / 3.0f;
      cen[3 * size_t(k) + a] = c;
      if (std::isfinite(c)) {
        lo[a] = std::min(lo[a], c);
        hi[a] = std::max(hi[a], c);
      }
    }
  std::vector<uint64_t> key(count);
  for (uint32_t k = 0; k < count; ++k) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
      const float ext = hi[a] > lo[a] ? hi[a] - lo[a] : 1.0f;
      float u = (cen[3 * size_t(k) + a] - lo[a]) / ext * 1023.0f;
      u = std::isfinite(u) ? std::min(std::max(u, 0.0f), 1023.0f) : 0.0f;
      q[a] = uint32_t(u);
    }
    key[k] = (uint64_t(mortonEncode(int(q[0]), int(q[1]), int(q[2]))) << 32) | k;
  }
  std::sort(key.begin(), key.end());
  std::vector<float> sorted(size_t(count) * 12);
  std::vector<uint32_t> idx(count);
  for (uint32_t i = 0; i < count; ++i) {
    idx[i] = uint32_t(key[i] & 0xffffffffu);
    std::memcpy(&sorted[12 * size_t(i)], h + 12 * size_t(idx[i]), 12 * sizeof(float));
  }
  std::vector<float4> sph(std::max(clusters, 1u));
  for (uint32_t c = 0; c < clusters; ++c) {
    const uint32_t t0 = c * kMeshCluster, t1 = std::min(count, t0 + kMeshCluster);
    float l[3] = {INFINITY, INFINITY, INFINITY}, u[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = t0; t < t1; ++t)
      for (int v = 1; v < 4; ++v)
        for (int a = 0; a < 3; ++a) {
          l[a] = std::min(l[a], sorted[12 * size_t(t) + 3 * v + a]);
          u[a] = std::max(u[a], sorted[12 * size_t(t) + 3 * v + a]);
        }
    const float cx = 0.5f * (l[0] + u[0]), cy = 0.5f * (l[1] + u[1]), cz = 0.5f * (l[2] + u[2]);
    double r2 = 0.0;
    for (uint32_t t = t0; t < t1; ++t)
      for (int v = 1; v < 4; ++v) {
        const double dx = double(sorted[12 * size_t(t) + 3 * v]) - cx, dy = double(sorted[12 * size_t(t) + 3 * v + 1]) - cy,
                     dz = double(sorted[12 * size_t(t) + 3 * v + 2]) - cz;
        r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
      }
    // covers the cluster despite the device's float rounding of posed points
    sph[c] = make_float4(cx, cy, cz, float(std::sqrt(r2)) * 1.0001f + 1e-6f * std::max(1.0f, std::fabs(cx) + std::fabs(cy) + std::fabs(cz)));
  }
  tris.ensure(std::max<size_t>(sorted.size() * sizeof(float), 16));
  index.ensure(std::max<size_t>(idx.size() * sizeof(uint32_t), 16));
  spheres.ensure(sph.size() * sizeof(float4));
  if (count) {
    check(cudaMemcpy(tris.ptr, sorted.data(), sorted.size() * sizeof(float), cudaMemcpyHostToDevice), "upload mesh");
    check(cudaMemcpy(index.ptr, idx.data(), idx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload mesh");
    check(cudaMemcpy(spheres.ptr, sph.data(), size_t(clusters) * sizeof(float4), cudaMemcpyHostToDevice), "upload mesh");
  }
}

MeshPose meshPose(const float* translation, const float* rotationWxyz) {
  MeshPose p{};
  p.q[0] = 1.0f;
  if (translation)
    for (int i = 0; i < 3; ++i) p.t[i] = translation[i];
  if (rotationWxyz)
    for (int i = 0; i < 4; ++i) p.q[i] = rotationWxyz[i];
  p.posed = translation != nullptr || rotationWxyz != nullptr;
  return p;
}

void checkMeshArgs(const float* tris, uint32_t nTris) {
  if (nTris && !tris) throw Error(NEBULA_MPM_ERR_INVALID, "null triangles");
  if (nTris > (1u << 26)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 2^26 triangles");
}

}  // namespace nebula

using namespace nebula;

struct nebula_mpm_mesh {
  nebula::PreparedMesh mesh;
};

namespace {
template <class F> int guardedMesh(F&& f) {
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
void checkGrid(const uint32_t realRes[3], uint32_t totalCells, float cellSize, const float* dSdf) {
  if (!realRes || !dSdf) throw Error(NEBULA_MPM_ERR_INVALID, "null argument");
  if (!(cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  if (!realRes[0] || !realRes[1] || !realRes[2]) throw Error(NEBULA_MPM_ERR_INVALID, "realRes must be >= 1");
  const uint32_t cube = domainCubeRes(realRes);
  if (cube > 1024u || uint64_t(totalCells) < uint64_t(cube) * cube * cube)
    throw Error(NEBULA_MPM_ERR_INVALID, "totalCells must hold the Morton cube of realRes (cubeRes <= 1024)");
}
}  // namespace

extern "C" {

int nebula_mpm_mesh_create(const float* tris, uint32_t n, nebula_mpm_mesh** out) {
  return guardedMesh([&] {
    if (!out) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    auto m = std::make_unique<nebula_mpm_mesh>();
    m->mesh.build(tris, n);
    *out = m.release();
  });
}

int nebula_mpm_mesh_destroy(nebula_mpm_mesh* m) {
  delete m;
  return NEBULA_MPM_OK;
}

int nebula_mpm_mesh_build_sdf(const nebula_mpm_mesh* m, const float translation[3], const float rotation_wxyz[4], const uint32_t realRes[3],
                              uint32_t totalCells, float cellSize, float* dSdf, void* stream) {
  return guardedMesh([&] {
    if (!m) throw Error(NEBULA_MPM_ERR_INVALID, "null mesh");
    checkGrid(realRes, totalCells, cellSize, dSdf);
    uint64_t l = 0;
    check(launchMeshSdfPrepared(m->mesh, meshPose(translation, rotation_wxyz), realRes, totalCells, cellSize, dSdf, static_cast<cudaStream_t>(stream),
                                &l),
          "mesh sdf");
  });
}

int nebula_mpm_mesh_build_sdf_reference(const nebula_mpm_mesh* m, const float translation[3], const float rotation_wxyz[4],
                                        const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream) {
  return guardedMesh([&] {
    if (!m) throw Error(NEBULA_MPM_ERR_INVALID, "null mesh");
    checkGrid(realRes, totalCells, cellSize, dSdf);
    uint64_t l = 0;
    check(launchMeshSdfReference(static_cast<const float*>(m->mesh.tris.ptr), static_cast<const uint32_t*>(m->mesh.index.ptr), m->mesh.n,
                                 meshPose(translation, rotation_wxyz), realRes, totalCells, cellSize, dSdf, static_cast<cudaStream_t>(stream), &l),
          "mesh sdf (reference closest point)");
  });
}

int nebula_mpm_mesh_sdf_reference(const float* dTris, uint32_t nTris, const float translation[3], const float rotation_wxyz[4],
                                  const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream) {
  return guardedMesh([&] {
    checkGrid(realRes, totalCells, cellSize, dSdf);
    checkMeshArgs(dTris, nTris);
    if (reinterpret_cast<uintptr_t>(dTris) % 16u) throw Error(NEBULA_MPM_ERR_INVALID, "triangles must be 16-byte aligned");
    uint64_t l = 0;
    check(launchMeshSdfReference(dTris, nullptr, nTris, meshPose(translation, rotation_wxyz), realRes, totalCells, cellSize, dSdf,
                                 static_cast<cudaStream_t>(stream), &l),
          "mesh sdf (reference closest point)");
  });
}

int nebula_mpm_mesh_sdf(const float* dTris, uint32_t nTris, const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf,
                        void* stream) {
  return nebula_mpm_mesh_sdf_posed(dTris, nTris, nullptr, nullptr, realRes, totalCells, cellSize, dSdf, stream);
}

int nebula_mpm_mesh_sdf_posed(const float* dTris, uint32_t nTris, const float translation[3], const float rotationWxyz[4],
                              const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream) {
  return guardedMesh([&] {
    checkGrid(realRes, totalCells, cellSize, dSdf);
    checkMeshArgs(dTris, nTris);
    if (reinterpret_cast<uintptr_t>(dTris) % 16u) throw Error(NEBULA_MPM_ERR_INVALID, "triangles must be 16-byte aligned");
    uint64_t l = 0;
    check(launchMeshSdf(dTris, nTris, meshPose(translation, rotationWxyz), realRes, totalCells, cellSize, dSdf,
                        static_cast<cudaStream_t>(stream), &l),
          "mesh sdf");
  });
}

}  // extern "C"
