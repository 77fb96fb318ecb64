// mpm_emit.cu -- the emission kernel (see mpm_emit.cuh).
#include "mpm_emit.cuh"

namespace nebula {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform in [0, 1) with 24 bits: draw k of particle j of emission `event`.
__device__ __forceinline__ float draw(uint64_t h, uint64_t seed, uint32_t k) {
  const uint64_t x = mix64(h + seed + uint64_t(k) * 0x9E3779B97F4A7C15ull);
  return float(uint32_t(x >> 40)) * (1.0f / 16777216.0f);
}

__global__ void __launch_bounds__(kThreads) k_emit(EmitterRec em, float Vp, uint64_t seed, uint64_t event, uint32_t n, StatePtrs st,
                                                   uint32_t* pid, uint32_t offset) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint64_t h = mix64((event << 32) | j);
  const float cx = em.center[0], cy = em.center[1], cz = em.center[2];
  float px, py, pz;
  if (em.shape == EMIT_SPHERE) {
    // AABB/Sphere/Ellipse::sample (Emitter.h:106-112, 160-169, 206-217)
    const float r = em.size[0] * cbrtf(draw(h, seed, 0));
    const float th = 3.14159265f * draw(h, seed, 1);
    const float ph = 6.28318530f * draw(h, seed, 2);
    px = cx + r * sinf(th) * cosf(ph);
    py = cy + r * sinf(th) * sinf(ph);
    pz = cz + r * cosf(th);
  } else if (em.shape == EMIT_ELLIPSE) {
    const float a = em.size[0], b = em.size[1];
    float ex = 0.f, ey = 0.f;
    for (uint32_t t = 0; t < 64; ++t) {
      const float x = a * (2.0f * draw(h, seed, 2 * t) - 1.0f);
      const float y = b * (2.0f * draw(h, seed, 2 * t + 1) - 1.0f);
      if ((x * x) / (a * a) + (y * y) / (b * b) <= 1.0f) {
        ex = x;
        ey = y;
        break;
      }
    }
    px = cx + ex;
    py = cy + ey;
    pz = cz;
  } else {
    const float hx = 0.5f * em.size[0], hy = 0.5f * em.size[1], hz = 0.5f * em.size[2];
    px = cx + hx * (2.0f * draw(h, seed, 0) - 1.0f);
    py = cy + hy * (2.0f * draw(h, seed, 1) - 1.0f);
    pz = cz + hz * (2.0f * draw(h, seed, 2) - 1.0f);
  }
  // Emitter::sample_velocity (Emitter.h:72-80)
  float vx = em.vel[0], vy = em.vel[1], vz = em.vel[2];
  if (em.emitAlongNormal) {
    const float speed = sqrtf(vx * vx + vy * vy + vz * vz);
    float nx = 0.f, ny = 0.f, nz = 1.f;
    if (em.shape == EMIT_AABB) {  // AABBEmitter::surface_normal (Emitter.h:115-122)
      const float dx = (px - cx) / fmaxf(0.5f * em.size[0], 1e-6f), dy = (py - cy) / fmaxf(0.5f * em.size[1], 1e-6f),
                  dz = (pz - cz) / fmaxf(0.5f * em.size[2], 1e-6f);
      const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
      nz = 0.f;
      if (ax >= ay && ax >= az) nx = dx >= 0.f ? 1.f : -1.f;
      else if (ay >= az) ny = dy >= 0.f ? 1.f : -1.f;
      else nz = dz >= 0.f ? 1.f : -1.f;
    } else {  // Emitter::surface_normal (Emitter.h:64-68)
      const float dx = px - cx, dy = py - cy, dz = pz - cz;
      const float len = sqrtf(dx * dx + dy * dy + dz * dz);
      if (len > 1e-6f) {
        nx = dx / len;
        ny = dy / len;
        nz = dz / len;
      }
    }
    vx = nx * speed;
    vy = ny * speed;
    vz = nz * speed;
  }
  if (em.velocityRandomness > 0.f) {
    const float r = em.velocityRandomness;
    vx += r * (2.0f * draw(h, seed, 128) - 1.0f);
    vy += r * (2.0f * draw(h, seed, 129) - 1.0f);
    vz += r * (2.0f * draw(h, seed, 130) - 1.0f);
  }
  const uint32_t slot = offset + j;
  st.f[0][slot] = make_float4(px, py, pz, Vp);
  st.f[1][slot] = make_float4(vx, vy, vz, __uint_as_float(em.particleType));
  st.f[2][slot] = make_float4(1.f, 0.f, 0.f, 0.f);
  st.f[3][slot] = make_float4(0.f, 1.f, 0.f, 0.f);
  st.f[4][slot] = make_float4(0.f, 0.f, 1.f, 0.f);
  st.f[5][slot] = st.f[6][slot] = st.f[7][slot] = make_float4(0.f, 0.f, 0.f, 0.f);
  pid[slot] = slot;
}

}  // namespace

cudaError_t launchEmit(const EmitterRec& em, float Vp, uint64_t seed, uint64_t event, uint32_t n, StatePtrs st, uint32_t* pid,
                       uint32_t offset, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_emit<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(em, Vp, seed, event, n, st, pid, offset);
  ++*launches;
  return cudaGetLastError();
}

}  // namespace nebula
