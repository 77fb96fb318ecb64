// glsl_env.hpp -- TEST INFRASTRUCTURE ONLY.
//
// The bindless storage-buffer table (set 0, binding 0) that the reference's MPM
// shaders index as buffers[slot].data[word]; shared by the shaders compiled for
// the CPU (through glsl_compat.hpp) and their dispatcher (ref_dispatch.cpp).
#pragma once
#include <cstdint>

struct StorageBuffer {
  uint32_t* data;
};
inline StorageBuffer buffers[32];
