/* nebula_mpm.hpp -- header-only C++ facade over the C ABI of nebula_mpm.h
 * with the method names and public tunables of the reference's MPMEngine
 * (src/engine/MPMEngine.h:59-186, EngineBase force table EngineBase.cpp:22-40),
 * so that callers written against it (examples/mpm_*.cpp, tests/test_mpm.cpp)
 * keep their code: init / step / setMaterials / setColliders / setColliderSDF
 * / setColliderSphere / appendParticles / resetParticles / addForce ... and the
 * fields restitution, wall_friction, numSubsteps, plasticModel, q_max,
 * M_friction, q_cohesion, flip_ratio, pushed to the engine before every step.
 *
 * Differences the type system makes visible: step takes a cudaStream_t
 * (passed as void*) instead of a VkCommandBuffer; buffers are device
 * pointers instead of VkBuffers; failures throw std::runtime_error with
 * nebula_mpm_last_error() where the reference throws its own exceptions.
 * Record types are the C ABI's (nebula_mpm_material, nebula_mpm_collider,
 * nebula_mpm_force, nebula_mpm_emitter), byte-compatible with MaterialParams,
 * ColliderPrimitive and ForceGPU; a std::vector of the reference's records can
 * be passed through the pointer overloads.
 *
 * The class lives in namespace nebula_b200 (the library's own C++ classes are
 * in namespace nebula and are not part of its interface). */
#ifndef NEBULA_MPM_HPP
#define NEBULA_MPM_HPP

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "nebula_mpm.h"

namespace nebula_b200 {

struct MPMConfig {  // MPMEngine.h:22-55, same defaults
  uint32_t nx = 32, ny = 32, nz = 32;                 // particle lattice
  float domainSize[3] = {10.0f, 10.0f, 10.0f};       // [m]
  float cellSize = 10.0f / 64.0f;                     // [m]
  uint32_t maxParticles = 0;                          // 0 = nx * ny * nz
  float E = 1e4f, nu = 0.3f, rho0 = 1000.0f;
};

enum class Field : int { P = 0, v = 1, F0 = 2, F1 = 3, F2 = 4, B0 = 5, B1 = 6, B2 = 7 };

class MPMEngine {
 public:
  MPMEngine() = default;
  explicit MPMEngine(const MPMConfig& c) { init(c); }
  ~MPMEngine() { cleanup(); }
  MPMEngine(const MPMEngine&) = delete;
  MPMEngine& operator=(const MPMEngine&) = delete;
  MPMEngine(MPMEngine&& o) noexcept { *this = std::move(o); }
  MPMEngine& operator=(MPMEngine&& o) noexcept {
    if (this != &o) {
      cleanup();
      e_ = o.e_;
      cfg_ = o.cfg_;
      forces_ = std::move(o.forces_);
      restitution = o.restitution;
      wall_friction = o.wall_friction;
      numSubsteps = o.numSubsteps;
      plasticModel = o.plasticModel;
      q_max = o.q_max;
      M_friction = o.M_friction;
      q_cohesion = o.q_cohesion;
      flip_ratio = o.flip_ratio;
      o.e_ = nullptr;
    }
    return *this;
  }

  // MPMEngine::init (MPMEngine.cpp:34-156): places the nx*ny*nz lattice
  void init(const MPMConfig& c) {
    cleanup();
    cfg_ = c;
    nebula_mpm_config cc{c.nx, c.ny, c.nz, {c.domainSize[0], c.domainSize[1], c.domainSize[2]}, c.cellSize, c.maxParticles, c.E, c.nu, c.rho0};
    ok(nebula_mpm_create(&cc, &e_));
    pull();
  }
  void cleanup() {
    if (e_) nebula_mpm_destroy(e_);
    e_ = nullptr;
  }
  const MPMConfig& config() const { return cfg_; }

  // MPMEngine::step (MPMEngine.cpp:404-474), stream-ordered on `stream` (a cudaStream_t)
  void step(void* stream, float dt) {
    push();
    ok(nebula_mpm_step(e_, dt, stream));
  }
  void sync() { ok(nebula_mpm_sync(e_)); }
  // replays of the substep loop from the engine's own CUDA graphs (on by default)
  void setGraphs(bool enable) { ok(nebula_mpm_set_graphs(e_, enable ? 1 : 0)); }
  uint32_t liveParticleCount() const {
    uint32_t n = 0;
    ok(nebula_mpm_live_count(e_, &n));
    return n;
  }

  // materials and colliders (MPMEngine.cpp:180-267)
  void setMaterials(const nebula_mpm_material* m, uint32_t n) { ok(nebula_mpm_set_materials(e_, m, n)); }
  void setMaterials(const std::vector<nebula_mpm_material>& m) { setMaterials(m.data(), uint32_t(m.size())); }
  void setParticleMaterialIds(const std::vector<uint32_t>& ids) { ok(nebula_mpm_set_particle_material_ids(e_, ids.data(), uint32_t(ids.size()))); }
  void setColliders(const nebula_mpm_collider* c, uint32_t n) { ok(nebula_mpm_set_colliders(e_, c, n)); }
  void setColliders(const std::vector<nebula_mpm_collider>& c) { setColliders(c.data(), uint32_t(c.size())); }
  void clearAnalyticColliders() { ok(nebula_mpm_clear_analytic_colliders(e_)); }
  void setColliderSDF(const std::vector<float>& sdf) { ok(nebula_mpm_set_collider_sdf(e_, sdf.data(), sdf.size())); }
  void setColliderSphere(float radius, float cx, float cy, float cz) { ok(nebula_mpm_set_collider_sphere(e_, radius, cx, cy, cz)); }
  void clearCollider() { ok(nebula_mpm_clear_collider(e_)); }
  // setColliderSDF(buildMeshSDF(tris, ...)) built on the device; tris: 12 floats each (normal, v0, v1, v2)
  void setColliderMesh(const float* tris, uint32_t n) { ok(nebula_mpm_set_collider_mesh(e_, tris, n)); }
  void setColliderMeshPose(const float translation[3], const float rotationWxyz[4]) {
    ok(nebula_mpm_set_collider_mesh_pose(e_, translation, rotationWxyz));
  }
  // true: later mesh builds take the reference's closestPtOnTriangle (its exact SDF)
  void setColliderMeshClosestPoint(bool reference) {
    ok(nebula_mpm_set_collider_mesh_closest_point(e_, reference ? NEBULA_MPM_CLOSEST_POINT_REFERENCE : NEBULA_MPM_CLOSEST_POINT_COMPLETE));
  }

  // the force table of EngineBase (EngineBase.cpp:22-40)
  void addForce(const nebula_mpm_force& f) {
    forces_.push_back(f);
    uploadForces();
  }
  void removeForce(size_t index) {
    if (index >= forces_.size()) throw std::out_of_range("removeForce: index out of range");
    forces_.erase(forces_.begin() + std::ptrdiff_t(index));
    uploadForces();
  }
  void setForces(const std::vector<nebula_mpm_force>& f) {
    forces_ = f;
    uploadForces();
  }
  void clearForces() {
    forces_.clear();
    uploadForces();
  }
  const std::vector<nebula_mpm_force>& forces() const { return forces_; }

  // particles (MPMEngine.cpp:211-235, 281-287)
  uint32_t appendParticles(const float* pos4, const float* vel4, uint32_t n) {
    uint32_t appended = 0;
    ok(nebula_mpm_append_particles(e_, pos4, vel4, n, &appended));
    return appended;
  }
  void resetParticles() { ok(nebula_mpm_reset_particles(e_)); }
  // the seeded jittered lattice of the measurement configurations
  uint32_t appendLattice(const nebula_mpm_lattice& L) {
    uint32_t appended = 0;
    ok(nebula_mpm_append_lattice(e_, &L, &appended));
    return appended;
  }
  uint32_t addEmitter(const nebula_mpm_emitter& em) {
    uint32_t index = 0;
    ok(nebula_mpm_add_emitter(e_, &em, &index));
    return index;
  }
  void clearEmitters() { ok(nebula_mpm_clear_emitters(e_)); }

  // getPositionBuffer / getVelocityBuffer (MPMEngine.cpp:165-166): device
  // arrays in the original particle order, valid until the next step
  float* getPositionBuffer() { return devicePointer(Field::P); }
  float* getVelocityBuffer() { return devicePointer(Field::v); }
  float* devicePointer(Field f) {
    float* p = nullptr;
    ok(nebula_mpm_device_ptr(e_, int(f), &p));
    return p;
  }
  // a field copied to the host, 4 floats per live particle
  std::vector<float> download(Field f) const {
    std::vector<float> out(size_t(liveParticleCount()) * 4);
    ok(nebula_mpm_download(e_, int(f), out.data(), out.size()));
    return out;
  }

  nebula_mpm* handle() { return e_; }

  // public tunables (MPMEngine.h:72-80), applied at every step
  float restitution = 0.3f;
  float wall_friction = 0.0f;
  int numSubsteps = 20;
  uint32_t plasticModel = 0;
  float q_max = 1e5f;
  float M_friction = 0.577f;
  float q_cohesion = 0.0f;
  float flip_ratio = 0.0f;

 private:
  static void ok(int rc) {
    if (rc != NEBULA_MPM_OK) {
      const char* m = nebula_mpm_last_error();
      throw std::runtime_error(std::string("nebula_mpm: ") + (m ? m : "error"));
    }
  }
  void pull() {
    nebula_mpm_params p{};
    ok(nebula_mpm_get_params(e_, &p));
    restitution = p.restitution;
    wall_friction = p.wall_friction;
    numSubsteps = p.numSubsteps;
    plasticModel = p.plasticModel;
    q_max = p.q_max;
    M_friction = p.M_friction;
    q_cohesion = p.q_cohesion;
    flip_ratio = p.flip_ratio;
  }
  void push() {
    nebula_mpm_params p{restitution, wall_friction, numSubsteps, plasticModel, q_max, M_friction, q_cohesion, flip_ratio};
    ok(nebula_mpm_set_params(e_, &p));
  }
  void uploadForces() { ok(nebula_mpm_set_forces(e_, forces_.data(), uint32_t(forces_.size()))); }

  nebula_mpm* e_ = nullptr;
  MPMConfig cfg_;
  std::vector<nebula_mpm_force> forces_;
};

}  // namespace nebula_b200

#endif /* NEBULA_MPM_HPP */
