// mpm_mesh_sdf_oracle.cpp -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
// reference's mesh -> SDF builder, the checker of the CUDA kernel.
//
// buildMeshSDF (src/core/MeshSDF.h:98-132): for every cell centre inside
// realRes, the distance to the closest triangle (first triangle wins ties),
// negative when dot(p - closest, triangle normal) < 0; cells of the Morton
// cube outside realRes hold 1e9.  A plain brute force over all cells and
// triangles.  Closest point on a triangle by the region test of Ericson's
// "Real-Time Collision Detection" (5.1.5), which closestPtOnTriangle
// (MeshSDF.h:48-78) follows except that it leaves out the edge-BC region:
// a point whose closest feature is edge BC gets the plane projection,
// extrapolated outside the triangle.  complete = 0 reproduces the reference's
// steps; complete = 1 adds the edge-BC case (the CUDA kernel's definition).
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct V3 {
  float x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scl(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

V3 closestPt(V3 p, V3 a, V3 b, V3 c, bool complete) {
  const V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) return a;
  const V3 bp = sub(p, b);
  const float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.f && d4 <= d3) return b;
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) return add(a, scl(d1 / (d1 - d3), ab));
  const V3 cp = sub(p, c);
  const float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.f && d5 <= d6) return c;
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) return add(a, scl(d2 / (d2 - d6), ac));
  const float va = d3 * d6 - d5 * d4;
  if (complete && va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) return add(b, scl((d4 - d3) / ((d4 - d3) + (d5 - d6)), sub(c, b)));
  const float sum = va + vb + vc;
  return add(add(a, scl(vb / sum, ab)), scl(vc / sum, ac));  // a + (vb/sum) ab + (vc/sum) ac, left to right
}

uint32_t expand(uint32_t v) {
  v = (v | (v << 16u)) & 0x030000FFu;
  v = (v | (v << 8u)) & 0x0300F00Fu;
  v = (v | (v << 4u)) & 0x030C30C3u;
  v = (v | (v << 2u)) & 0x09249249u;
  return v;
}

}  // namespace

extern "C" {

// tris: n x 12 floats (normal, v0, v1, v2); sdf: totalCells floats.
void orc_mesh_sdf(const float* tris, uint32_t n, const uint32_t* res, uint32_t totalCells, float cs, float* sdf, int complete) {
  for (uint32_t i = 0; i < totalCells; ++i) sdf[i] = 1e9f;
#pragma omp parallel for schedule(dynamic, 1)
  for (int iz = 0; iz < int(res[2]); ++iz)
    for (uint32_t iy = 0; iy < res[1]; ++iy)
      for (uint32_t ix = 0; ix < res[0]; ++ix) {
        const V3 p = {(ix + 0.5f) * cs, (iy + 0.5f) * cs, (iz + 0.5f) * cs};
        float minD = 1e9f;
        bool outer = true;
        for (uint32_t t = 0; t < n; ++t) {
          const float* r = tris + 12 * size_t(t);
          const V3 q = closestPt(p, {r[3], r[4], r[5]}, {r[6], r[7], r[8]}, {r[9], r[10], r[11]}, complete != 0);
          const V3 d = sub(p, q);
          const float len = std::sqrt(dot(d, d));
          if (len < minD) {
            minD = len;
            outer = dot(d, {r[0], r[1], r[2]}) >= 0.f;
          }
        }
        sdf[expand(ix) | (expand(iy) << 1) | (expand(uint32_t(iz)) << 2)] = outer ? minD : -minD;
      }
}

}  // extern "C"
