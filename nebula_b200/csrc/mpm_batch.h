// mpm_batch.h -- nebula::BatchEngine: many independent MPM scenes stepped by
// one set of launches per substep (no counterpart in the reference, whose
// MPMEngine holds one scene).
//
// Every scene keeps the plain engine's parameter surface (MPMConfig domain,
// MPMEngine tunables, material table, colliders, SDF, forces).  All scenes
// share one brick space and one particle array (see SceneTable), so a substep
// is the plain fused pipeline run once over the union: batched grid update,
// batched fused G2P+P2G, brick scan, permutation.  A step of K substeps is
// captured once into a CUDA graph and replayed.
#pragma once
#include <map>
#include <tuple>
#include <vector>

#include "mpm_engine.h"

namespace nebula {

class BatchEngine {
 public:
  explicit BatchEngine(const nebula_mpm_batch_config& cfg);
  ~BatchEngine();

  uint32_t addScene(const nebula_mpm_config& cfg, const float* pos4, const float* vel4, uint32_t n);
  void setParams(uint32_t s, const nebula_mpm_params& p);
  void getParams(uint32_t s, nebula_mpm_params* p) const;
  void setMaterials(uint32_t s, const nebula_mpm_material* m, uint32_t n);
  void setParticleMaterialIds(uint32_t s, const uint32_t* ids, uint32_t n);
  void setColliders(uint32_t s, const nebula_mpm_collider* c, uint32_t n);
  void setColliderTrack(uint32_t s, const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps);
  void setColliderSDF(uint32_t s, const float* sdf, uint64_t n);
  void clearColliderSDF(uint32_t s);
  void setForces(uint32_t s, const nebula_mpm_force* f, uint32_t n);
  void uploadState(uint32_t s, const float* const f[8], uint32_t n);
  void download(uint32_t s, int field, float* host, uint64_t count);
  void step(float dt, uint32_t substeps, cudaStream_t st);
  void setGraphs(bool on);
  void setLaunchConfig(const LaunchConfig& c);
  const LaunchConfig& launchConfig() const { return launchCfg_; }
  uint32_t syncAndCheck();
  void stats(nebula_mpm_batch_stats* out);
  void sceneInfo(uint32_t s, nebula_mpm_scene_info* out) const;
  uint32_t sceneCount() const { return uint32_t(scenes_.size()); }

 private:
  struct Scene {
    nebula_mpm_config cfg;
    nebula_mpm_params params;
    uint32_t gridRes[3];
    uint32_t cubeRes, hashCells, nb;
    uint32_t brickBase, partBase, n;
    std::vector<Material> materials;
    std::vector<Collider> track;  // trackLen * colliderCount
    uint32_t colliderCount = 0, trackLen = 1;
    std::vector<Force> forces;
    DevBuf sdf;
    bool hasSdf = false;
  };

  void bindDevice() const;
  void quiesce();
  void seal();
  Scene& scene(uint32_t s);
  const Scene& scene(uint32_t s) const;
  void beforeHostEdit(bool particles);
  void normalizeOrder(cudaStream_t st);
  void discardPending(cudaStream_t st);
  void uploadTables(float subDt, uint32_t substeps, cudaStream_t st);
  void buildPending(cudaStream_t st);
  void substep(uint32_t k, cudaStream_t st);
  bool anyFlip() const;
  StatePtrs statePtrs(int buf);
  BrickBuffers brickBuffers(int q);
  int modelSet() const;
  GridBuffers gridBuffers();
  SceneTable table() const;
  void clearGraphs();

  nebula_mpm_batch_config cfg_;
  int device_ = 0;
  int numSMs_ = 148;
  LaunchConfig launchCfg_;
  std::vector<Scene> scenes_;
  uint32_t live_ = 0;
  uint32_t nbTotal_ = 0;
  bool sealed_ = false;
  cudaStream_t lastStream_ = nullptr;

  DevBuf state_[8], stateB_[8], pid_[2];
  int cur_ = 0;
  bool permuted_ = false;
  DevBuf gridAcc_, gridVel_, gridVold_;
  DevBuf bCount_, bFlag_, bStart_, cCount_[2], pbBrick_, pbStart_, gbBrick_, counters_, scanState_, scanTile_, binKey_, binRank_, perm_, err_;
  uint32_t tiles_ = 1;
  // device tables
  DevBuf tParams_, tBrickBase_, tPartBase_, tMaterials_, tForces_, tTrack_;
  // pinned staging for table uploads; reused once the previous upload's copy finished
  void* staging_ = nullptr;
  size_t stagingBytes_ = 0;
  cudaEvent_t stagingFree_ = nullptr;
  bool tablesDirty_ = true;
  float tableDt_ = -1.f;
  uint32_t tableSubsteps_ = 0;

  bool pending_ = false;
  float pendingDt_ = 0.f;

  bool useGraphs_ = true;
  std::map<std::tuple<uint32_t, int, bool, int>, cudaGraphExec_t> graphs_;  // by substeps, buffer parity, FLIP, model set
  std::map<std::tuple<uint32_t, int, bool, int>, uint64_t> launchesPerGraph_;

  uint64_t substeps_ = 0;
  uint64_t launches_ = 0;
  uint64_t graphLaunches_ = 0;
  uint32_t overflow_ = 0, activeBricks_ = 0, particleBricks_ = 0, errorFlags_ = 0;
};

}  // namespace nebula
