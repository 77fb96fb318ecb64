// mpm_engine.h -- nebula::MPMEngine, the C++ host engine behind include/nebula_mpm.h.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/nebula_mpm.h"
#include "mpm_bricks.cuh"
#include "mpm_device.cuh"
#include "mpm_emit.cuh"
#include "mpm_internal.h"

namespace nebula {

// Rejects launch shapes outside the compiled variants (NEBULA_MPM_ERR_INVALID).
void validateLaunchConfig(const LaunchConfig& c);
LaunchConfig fromAbi(const nebula_mpm_launch_config& c);
nebula_mpm_launch_config toAbi(const LaunchConfig& c);

struct Error : std::runtime_error {
  int code;
  Error(int code, const std::string& msg);
};
void check(cudaError_t e, const char* what);
extern thread_local std::string g_last_error;
// Throws NEBULA_MPM_ERR_DEVICE naming the error bits of a single-pass binning call (none: returns).
void throwBinErrors(uint32_t bits);

// Rigid pose applied to a mesh on the device (transformTriangles, MeshSDF.h:134-141):
// v -> q * v + t, n -> q * n; q a unit quaternion (w, x, y, z).
struct MeshPose {
  float q[4];
  float t[3];
  bool posed;  // false: the triangles as given
};
MeshPose meshPose(const float* translation, const float* rotationWxyz);  // null pointers: identity parts
void checkMeshArgs(const float* tris, uint32_t nTris);  // null with n > 0, count

// Morton-ordered SDF of a triangle mesh (12 floats per triangle: normal, v0, v1, v2;
// 16-byte aligned), posed by `pose`.
cudaError_t launchMeshSdf(const float* dTris, uint32_t n, const MeshPose& pose, const uint32_t res[3], uint32_t totalCells, float cellSize,
                          float* dSdf, cudaStream_t s, uint64_t* launches);

void domainGridRes(const float size[3], float h, uint32_t out[3]);
uint32_t domainCubeRes(const uint32_t res[3]);
uint32_t domainHashCells(const uint32_t res[3]);

// Owning device allocation.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf();
  void alloc(size_t n);
  void ensure(size_t n);
  void reset();
};

// A triangle mesh prepared for repeated SDF builds: triangles sorted by the
// Morton code of their centroids (device, 12 floats each), their indices in
// the caller's list, and the bounding sphere of every run of kMeshCluster
// sorted triangles (centre, radius).  Built on the host from a host list.
constexpr uint32_t kMeshCluster = 32;
struct PreparedMesh {
  uint32_t n = 0, clusters = 0;
  DevBuf tris, index, spheres;
  void build(const float* hostTris, uint32_t n);
};
// SDF of a prepared mesh, posed by `pose` (same result as launchMeshSdf on
// the caller's list).
cudaError_t launchMeshSdfPrepared(const PreparedMesh& m, const MeshPose& pose, const uint32_t res[3], uint32_t totalCells, float cellSize,
                                  float* dSdf, cudaStream_t s, uint64_t* launches);
// SDF with the reference's closest-point steps (no edge-BC region) by brute
// force over the triangles; `dIndex` (may be null: list order) is each
// triangle's index in the caller's list, for the first-in-list tie rule.
cudaError_t launchMeshSdfReference(const float* dTris, const uint32_t* dIndex, uint32_t n, const MeshPose& pose, const uint32_t res[3],
                                   uint32_t totalCells, float cellSize, float* dSdf, cudaStream_t s, uint64_t* launches);


class MPMEngine {
 public:
  explicit MPMEngine(const nebula_mpm_config& cfg);
  ~MPMEngine();

  void setParams(const nebula_mpm_params& p);
  const nebula_mpm_params& params() const { return params_; }
  void setMaterials(const nebula_mpm_material* mats, uint32_t n);
  void setParticleMaterialIds(const uint32_t* ids, uint32_t n);
  void setColliders(const nebula_mpm_collider* c, uint32_t n);
  void setColliderTrack(const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps);
  void clearAnalyticColliders();
  void setColliderSDF(const float* sdf, uint64_t n);
  void setColliderSphere(float radius, float cx, float cy, float cz);
  void setColliderMesh(const float* tris, uint32_t n);
  void setColliderMeshPose(const float* translation, const float* rotationWxyz);
  // NEBULA_MPM_CLOSEST_POINT_COMPLETE (default) or _REFERENCE; applies to the
  // next setColliderMesh / setColliderMeshPose
  void setColliderMeshClosestPoint(int mode);
  void clearCollider();
  void setForces(const nebula_mpm_force* f, uint32_t n);
  uint32_t appendParticles(const float* pos4, const float* vel4, uint32_t n);
  uint32_t addEmitter(const nebula_mpm_emitter& em);
  void clearEmitters();
  void getEmitter(uint32_t i, nebula_mpm_emitter* em, int32_t* done) const;
  void resetParticles();
  void uploadState(const float* const f[8], uint32_t n);
  void download(int field, float* host, uint64_t count);
  void downloadState(float* const host[8], uint64_t count);
  // Stream-ordered state exchange through device staging buffers and
  // engine-owned copy streams (overlaps the transfers with the steps).
  void uploadStateAsync(const float* const f[8], uint32_t n, cudaStream_t s);
  void downloadStateAsync(float* const host[8], uint64_t count, cudaStream_t s);
  void waitDownloads(cudaStream_t s);
  float* devicePointer(int field);
  void setGravity(float gx, float gy, float gz);
  StatePtrs originalOrder();
  void step(float dt, cudaStream_t s);
  uint32_t liveCount() const { return live_; }
  void stats(nebula_mpm_stats* s);
  uint32_t syncAndCheck();
  void exportBins(uint32_t* cnt, uint32_t* off, uint32_t* srt);
  void exportGrid(float dt, float* mom, float* mass);
  void profileEnable(bool on);
  void profileRead(double* ms, uint64_t* launches, bool reset);
  void setPipeline(int p);
  int pipeline() const { return pipeline_; }
  void setLaunchConfig(const LaunchConfig& c);
  const LaunchConfig& launchConfig() const { return launchCfg_; }
  // Replays of the fused substep loop from CUDA graphs (on by default).
  void setGraphs(bool on);
  void exportBrickBins(uint32_t* numBricks, uint32_t* brickIds, uint32_t* brickStarts, uint32_t* sortedPids);

 private:
  // phase timing
  void phaseBegin(int phase, cudaStream_t s);
  void phaseEnd(int phase, cudaStream_t s, uint64_t launchesBefore);
  cudaEvent_t takeEvent();
  struct Timed {
    int phase;
    cudaEvent_t a, b;
    uint64_t launches;
  };
  bool profile_ = false;
  std::vector<cudaEvent_t> freeEvents_;
  std::vector<Timed> timed_;
  cudaEvent_t openEvent_ = nullptr;
  double phaseMs_[NEBULA_MPM_PHASES] = {};
  uint64_t phaseLaunches_[NEBULA_MPM_PHASES] = {};

  void bindDevice() const;
  void quiesce();
  SubstepParams buildParams(float subDt) const;
  StatePtrs statePtrs();
  BinBuffers binBuffers();
  void substepDense(const SubstepParams& P, cudaStream_t s);
  // brick-sparse fused pipeline
  StatePtrs statePtrs(int buf);
  BrickBuffers brickBuffers(int q);
  GridBuffers gridBuffers();
  void ensureDense();
  void normalizeOrder(cudaStream_t s);
  void discardPending(cudaStream_t s);
  void buildPending(const SubstepParams& P, cudaStream_t s);
  void substepFused(const SubstepParams& P, cudaStream_t s);
  void runFused(const SubstepParams& P, cudaStream_t s);
  SubstepParams atSubstep(const SubstepParams& P, int k) const;
  // Fused substep loops replayed from CUDA graphs.  A graph holds the kernels
  // of one step with their arguments, so it is keyed by every argument the
  // launches take (the substep parameters, buffer pointers, live count,
  // substep count, buffer parity and launch shape): a replay under an equal
  // key launches exactly what the uncaptured loop would.  One slot per buffer
  // parity; a key is captured the second step in a row that its slot sees it.
  struct StepGraph {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
  };
  bool graphsUsable(cudaStream_t s) const;
  std::vector<unsigned char> graphKey(const SubstepParams& P);
  void clearGraphs();
  bool useGraphs_ = true;
  StepGraph graphs_[2];
  cudaStream_t captureStream_ = nullptr;
  uint64_t graphLaunches_ = 0;
  // asynchronous state exchange: staging buffers (8 fields x capacity float4
  // each), one copy stream per direction, and the events ordering their reuse
  void ensureStaging();
  void switchStream(cudaStream_t s);
  DevBuf inStage_, outStage_;
  cudaStream_t copyIn_ = nullptr, copyOut_ = nullptr;
  cudaEvent_t inReady_ = nullptr, inFree_ = nullptr, outReady_ = nullptr, outFree_ = nullptr;
  void prepareHostAccess(bool modifiesParticles);
  bool pendingMatches(float subDt) const;
  bool emitFromEmitters(float dt, cudaStream_t s);

  nebula_mpm_config cfg_;
  nebula_mpm_params params_{0.3f, 0.0f, 20, 0u, 1e5f, 0.577f, 0.0f, 0.0f};  // MPMEngine.h:72-80
  int device_ = 0;
  uint32_t gridRes_[3] = {1, 1, 1};
  uint32_t cubeRes_ = 1;
  uint32_t hashCells_ = 1;
  uint32_t capacity_ = 0;
  uint32_t live_ = 0;
  cudaStream_t lastStream_ = nullptr;

  DevBuf state_[8];
  DevBuf stateB_[8];
  DevBuf pid_[2];
  int cur_ = 0;
  bool permuted_ = false;
  // Bumped by every change of the particle state; the idle state buffer holds
  // the original-order copy of version unpermutedVersion_ (downloads reuse it).
  uint64_t stateVersion_ = 0;
  uint64_t unpermutedVersion_ = ~uint64_t(0);
  int pipeline_ = NEBULA_MPM_PIPELINE_FUSED;
  LaunchConfig launchCfg_;
  int numSMs_ = 148;
  // brick-sparse grid + binning
  uint32_t ncPad_ = 64, nb_ = 1, tiles_ = 1;
  DevBuf gridAcc_, gridVel_, gridVold_;
  DevBuf bCount_, bFlag_, bStart_, cCount_[2], pbBrick_, pbStart_, gbBrick_, counters_, scanState_, scanTile_, binKey_, binRank_, perm_;
  bool pending_ = false;
  float pendingDt_ = 0.f;
  bool pendingApic_ = false;
  bool denseReady_ = false;
  DevBuf gridMom_, gridMass_;
  DevBuf cellCount_, cellStart_, cellEnd_, key_, rank_, sortedTmp_, sorted_, scanWs_;
  DevBuf materials_, colliders_, forces_, sdf_, err_;
  PreparedMesh mesh_;
  bool hasMesh_ = false;
  bool meshReferenceClosest_ = false;
  void buildMeshSdf(const MeshPose& pose);
  std::vector<Material> hostMaterials_;
  uint32_t colliderCount_ = 0;
  uint32_t colliderTrackLen_ = 1;
  std::vector<EmitterRec> emitters_;
  std::vector<int32_t> emitterDone_;
  uint64_t emitEvents_ = 0;  // emissions since create / reset: the counter of the sampling hash
  static constexpr uint64_t kEmitSeed = 12345;
  uint32_t forceCount_ = 0;
  std::vector<Force> hostForces_;  // the table last uploaded (setGravity edits it)
  bool hasSdf_ = false;

  uint64_t substeps_ = 0;
  uint64_t launches_ = 0;
  uint32_t activeBricks_ = 0;
  uint32_t particleBricks_ = 0;
  uint32_t overflow_ = 0;
  uint32_t errorFlags_ = 0;
};

}  // namespace nebula
