// mpm_emit.cuh -- device-side particle emission (MPMEngine::emitFromEmitters,
// MPMEngine.cpp:289-352, with the shapes of src/core/Emitter.h:95-224).
//
// The reference samples every new particle on the host with std::mt19937 and
// uploads the eight arrays with a blocking copy each step.  Here one kernel
// writes the new particles in place: particle j of emission `event` draws its
// uniforms from a counter-based hash, u_k = top 24 bits of
// mix(mix((event << 32) | j) + seed + k * golden), mix = the SplitMix64
// finalizer (Steele, Lea & Flood 2014).  Draws 0..2 place the particle
// (ellipse rejection uses draws 2a and 2a+1 of attempt a < 64), draws
// 128..130 perturb its velocity.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_internal.h"

namespace nebula {

struct EmitterRec {  // nebula_mpm_emitter, 80 B
  uint32_t shape;
  float center[3];
  float size[3];
  float vel[3];
  float center_vel[3];
  int32_t particles_per_step;
  uint32_t particleType;
  uint32_t emitAlongNormal;
  float velocityRandomness;
  int32_t step_count;
  float particleVolume;
  uint32_t pad;
};
static_assert(sizeof(EmitterRec) == 80, "EmitterRec");

enum : uint32_t { EMIT_AABB = 0, EMIT_SPHERE = 1, EMIT_ELLIPSE = 2 };

// Append n particles of emitter `em` (volume Vp) at buffer slots
// [offset, offset + n): original ids offset + j.
cudaError_t launchEmit(const EmitterRec& em, float Vp, uint64_t seed, uint64_t event, uint32_t n, StatePtrs st, uint32_t* pid,
                       uint32_t offset, cudaStream_t s, uint64_t* launches);

}  // namespace nebula
