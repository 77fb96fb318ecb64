// mpm_emit_oracle.cpp -- TEST INFRASTRUCTURE ONLY: CPU restatement of particle
// emission, the checker of the CUDA emission kernel.
//
// Shapes, normals and the velocity rule follow src/core/Emitter.h:64-80
// (sample_velocity, surface_normal), :106-122 (AABBEmitter), :160-169
// (SphereEmitter) and :206-217 (EllipseEmitter), with the schedule of
// MPMEngine::emitFromEmitters (MPMEngine.cpp:289-352) applied by the caller.
// The reference draws its uniforms from std::mt19937 on the host; the CUDA
// path draws them from a counter-based hash so that every particle is
// generated independently on the device.  This restatement uses the same
// published hash (the SplitMix64 finalizer, Steele, Lea & Flood 2014) from
// its own code: draw k of particle j of emission e is the top 24 bits of
// mix(mix((e << 32) | j) + seed + k * 0x9E3779B97F4A7C15) / 2^24; position
// draws 0..2 (ellipse rejection: draws 2a, 2a+1 of attempt a < 64),
// velocity draws 128..130.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

struct Rec {
  uint32_t shape;
  float center[3], size[3], vel[3], center_vel[3];
  int32_t particles_per_step;
  uint32_t particleType, emitAlongNormal;
  float velocityRandomness;
  int32_t step_count;
  float particleVolume;
  uint32_t pad;
};
static_assert(sizeof(Rec) == 80, "emitter record");

uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

float uniform24(uint64_t h, uint64_t seed, uint32_t k) {
  const uint64_t x = splitmix(h + seed + uint64_t(k) * 0x9E3779B97F4A7C15ull);
  return float(uint32_t(x >> 40)) * (1.0f / 16777216.0f);
}

}  // namespace

extern "C" {

// n particles of emission `event`: pos4 = (x, Vp), vel4 = (v, material id bits).
void orc_emit(const void* record, float Vp, uint64_t seed, uint64_t event, uint32_t n, float* pos4, float* vel4) {
  Rec em;
  std::memcpy(&em, record, sizeof(em));
  for (uint32_t j = 0; j < n; ++j) {
    const uint64_t h = splitmix((event << 32) | j);
    const float c[3] = {em.center[0], em.center[1], em.center[2]};
    float p[3];
    if (em.shape == 1u) {
      const float r = em.size[0] * std::cbrt(uniform24(h, seed, 0));
      const float th = 3.14159265f * uniform24(h, seed, 1);
      const float ph = 6.28318530f * uniform24(h, seed, 2);
      p[0] = c[0] + r * std::sin(th) * std::cos(ph);
      p[1] = c[1] + r * std::sin(th) * std::sin(ph);
      p[2] = c[2] + r * std::cos(th);
    } else if (em.shape == 2u) {
      const float a = em.size[0], b = em.size[1];
      float ex = 0.f, ey = 0.f;
      for (uint32_t t = 0; t < 64; ++t) {
        const float x = a * (2.0f * uniform24(h, seed, 2 * t) - 1.0f);
        const float y = b * (2.0f * uniform24(h, seed, 2 * t + 1) - 1.0f);
        if ((x * x) / (a * a) + (y * y) / (b * b) <= 1.0f) {
          ex = x;
          ey = y;
          break;
        }
      }
      p[0] = c[0] + ex;
      p[1] = c[1] + ey;
      p[2] = c[2];
    } else {
      for (int k = 0; k < 3; ++k) p[k] = c[k] + 0.5f * em.size[k] * (2.0f * uniform24(h, seed, k) - 1.0f);
    }
    float v[3] = {em.vel[0], em.vel[1], em.vel[2]};
    if (em.emitAlongNormal) {
      const float speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      float nrm[3] = {0.f, 0.f, 1.f};
      if (em.shape == 0u) {
        float d[3], ad[3];
        for (int k = 0; k < 3; ++k) {
          d[k] = (p[k] - c[k]) / std::fmax(0.5f * em.size[k], 1e-6f);
          ad[k] = std::fabs(d[k]);
        }
        nrm[2] = 0.f;
        if (ad[0] >= ad[1] && ad[0] >= ad[2]) nrm[0] = d[0] >= 0.f ? 1.f : -1.f;
        else if (ad[1] >= ad[2]) nrm[1] = d[1] >= 0.f ? 1.f : -1.f;
        else nrm[2] = d[2] >= 0.f ? 1.f : -1.f;
      } else {
        const float d[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
        const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (len > 1e-6f)
          for (int k = 0; k < 3; ++k) nrm[k] = d[k] / len;
      }
      for (int k = 0; k < 3; ++k) v[k] = nrm[k] * speed;
    }
    if (em.velocityRandomness > 0.f)
      for (int k = 0; k < 3; ++k) v[k] += em.velocityRandomness * (2.0f * uniform24(h, seed, 128 + k) - 1.0f);
    float idf;
    std::memcpy(&idf, &em.particleType, 4);
    for (int k = 0; k < 3; ++k) {
      pos4[4 * size_t(j) + k] = p[k];
      vel4[4 * size_t(j) + k] = v[k];
    }
    pos4[4 * size_t(j) + 3] = Vp;
    vel4[4 * size_t(j) + 3] = idf;
  }
}

}  // extern "C"
