// mpm_engine.cu -- nebula::MPMEngine: the C++ host side of the substep and the
// C ABI declared in include/nebula_mpm.h.
//
// The class keeps the reference's parameter surface (src/engine/MPMEngine.h:59-186):
// config, public tunables, material / collider / SDF / force tables, particle
// append / reset, and step(dt) running numSubsteps substeps
// (src/engine/MPMEngine.cpp:404-474).  Device memory is owned here; the caller
// owns the stream.  Errors are C++ exceptions inside and status codes at the ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpm_engine.h"
#include "mpm_internal.h"
#include "mpm_scan.cuh"

namespace nebula {

// ------------------------------------------------------------------ errors
thread_local std::string g_last_error;

Error::Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}

void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  int code = e == cudaErrorMemoryAllocation ? NEBULA_MPM_ERR_OOM : NEBULA_MPM_ERR_CUDA;
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ domain (src/core/Domain.h:14-39)
void domainGridRes(const float size[3], float h, uint32_t out[3]) {
  const float hh = std::max(h, 1e-6f);
  for (int a = 0; a < 3; ++a) {
    float r = std::ceil(size[a] / hh);
    out[a] = r < 1.0f ? 1u : uint32_t(r);
  }
}
uint32_t domainCubeRes(const uint32_t res[3]) {
  uint32_t m = std::max({res[0], res[1], res[2], 1u});
  uint32_t p = 1;
  while (p < m) p <<= 1u;
  return p;
}
uint32_t domainHashCells(const uint32_t res[3]) {
  uint32_t c = domainCubeRes(res);
  return c * c * c;
}

// ------------------------------------------------------------------ device buffer
DevBuf::~DevBuf() { reset(); }
void DevBuf::reset() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}
void DevBuf::alloc(size_t n) {
  reset();
  if (n == 0) return;
  check(cudaMalloc(&ptr, n), "cudaMalloc");
  bytes = n;
}
void DevBuf::ensure(size_t n) {
  if (n > bytes) alloc(n);
}

// ------------------------------------------------------------------ engine
MPMEngine::MPMEngine(const nebula_mpm_config& cfg) : cfg_(cfg) {
  if (!(cfg.cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  for (int a = 0; a < 3; ++a)
    if (!(cfg.domainSize[a] >= 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "domainSize must be >= 0");
  check(cudaGetDevice(&device_), "cudaGetDevice");
  domainGridRes(cfg.domainSize, cfg.cellSize, gridRes_);
  cubeRes_ = domainCubeRes(gridRes_);
  if (cubeRes_ > 1024u) throw Error(NEBULA_MPM_ERR_INVALID, "grid resolution above 1024 per axis (10-bit Morton code)");
  hashCells_ = cubeRes_ * cubeRes_ * cubeRes_;
  const uint64_t lattice = uint64_t(cfg.nx) * cfg.ny * cfg.nz;
  capacity_ = cfg.maxParticles > 0 ? cfg.maxParticles : uint32_t(lattice);
  if (lattice > capacity_) throw Error(NEBULA_MPM_ERR_INVALID, "nx*ny*nz exceeds maxParticles");

  const size_t capN = size_t(std::max(capacity_, 1u));
  for (int k = 0; k < 8; ++k) {
    state_[k].alloc(capN * sizeof(float4));
    stateB_[k].alloc(capN * sizeof(float4));
  }
  for (auto& p : pid_) p.alloc(capN * sizeof(uint32_t));
  materials_.alloc(kMaxMaterials * sizeof(Material));
  colliders_.alloc(kMaxColliders * sizeof(Collider));
  forces_.alloc(kMaxForces * sizeof(Force));
  err_.alloc(sizeof(uint32_t));
  check(cudaMemset(err_.ptr, 0, sizeof(uint32_t)), "cudaMemset");
  check(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");

  // brick-sparse grid: dense arrays over hashCells (padded to one brick), touched per brick
  ncPad_ = std::max(hashCells_, 64u);
  nb_ = ncPad_ / 64u;
  tiles_ = (nb_ + kBrickScanTile - 1) / kBrickScanTile;
  gridAcc_.alloc(size_t(ncPad_) * sizeof(float4));
  gridVel_.alloc(size_t(ncPad_) * sizeof(float4));
  check(cudaMemset(gridAcc_.ptr, 0, gridAcc_.bytes), "cudaMemset");
  check(cudaMemset(gridVel_.ptr, 0, gridVel_.bytes), "cudaMemset");
  for (DevBuf* b : {&bCount_, &bFlag_, &bStart_, &pbBrick_, &gbBrick_}) {
    b->alloc(size_t(nb_) * sizeof(uint32_t));
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  // per-cell counts of two binnings (each cleared by the fused kernel after the one that follows it)
  for (DevBuf* b : {&cCount_[0], &cCount_[1]}) {
    b->alloc(size_t(nb_) * 64u * sizeof(uint32_t));
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  pbStart_.alloc(size_t(nb_ + 1) * sizeof(uint32_t));
  counters_.alloc(kCntSlots * sizeof(uint32_t));
  scanState_.alloc(size_t(3) * tiles_ * sizeof(unsigned long long));
  scanTile_.alloc(sizeof(unsigned long long));
  for (DevBuf* b : {&pbStart_, &counters_, &scanState_, &scanTile_}) check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  for (DevBuf* b : {&binKey_, &binRank_, &perm_}) {
    b->alloc(capN * sizeof(uint32_t));
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  uint64_t l = 0;
  check(launchIota(static_cast<uint32_t*>(pid_[0].ptr), capacity_, nullptr, &l), "iota");

  // default material: presetJelly(E, nu, rho0) with model ELASTIC and the
  // public DP/VM defaults (MPMEngine.cpp:67-78)
  Material m{};
  m.mu = cfg.E / (2.0f * (1.0f + cfg.nu));
  m.lambda = cfg.E * cfg.nu / ((1.0f + cfg.nu) * (1.0f - 2.0f * cfg.nu));
  m.rho0 = cfg.rho0;
  m.model = MAT_ELASTIC;
  m.M_friction = params_.M_friction;
  m.q_cohesion = params_.q_cohesion;
  m.q_max = params_.q_max;
  hostMaterials_.assign(1, m);
  check(cudaMemcpy(materials_.ptr, &m, sizeof(m), cudaMemcpyHostToDevice), "upload materials");

  // default lattice (MPMEngine.cpp:86-137)
  live_ = uint32_t(lattice);
  if (live_ > 0) {
    const float blockFrac = 0.40f;
    const float minDomain = std::min({cfg.domainSize[0], cfg.domainSize[1], cfg.domainSize[2]});
    const float sp = minDomain * blockFrac / float(std::max({cfg.nx, cfg.ny, cfg.nz}));
    const float Vp = sp * sp * sp;
    const float cx = cfg.domainSize[0] * 0.5f, cz = cfg.domainSize[2] * 0.5f, cy = cfg.domainSize[1] * 0.70f;
    const float halfX = sp * float(cfg.nx - 1) / 2.0f, halfY = sp * float(cfg.ny - 1) / 2.0f, halfZ = sp * float(cfg.nz - 1) / 2.0f;
    std::vector<float4> host[8];
    for (auto& h : host) h.assign(live_, make_float4(0.f, 0.f, 0.f, 0.f));
    uint32_t idx = 0;
    for (uint32_t iz = 0; iz < cfg.nz; iz++)
      for (uint32_t iy = 0; iy < cfg.ny; iy++)
        for (uint32_t ix = 0; ix < cfg.nx; ix++, idx++) {
          host[0][idx] = make_float4(cx - halfX + ix * sp, cy - halfY + iy * sp, cz - halfZ + iz * sp, Vp);
          host[2][idx] = make_float4(1.f, 0.f, 0.f, 0.f);
          host[3][idx] = make_float4(0.f, 1.f, 0.f, 0.f);
          host[4][idx] = make_float4(0.f, 0.f, 1.f, 0.f);
        }
    for (int k = 0; k < 8; ++k) check(cudaMemcpy(state_[k].ptr, host[k].data(), live_ * sizeof(float4), cudaMemcpyHostToDevice), "upload state");
  }
}

MPMEngine::~MPMEngine() {
  if (lastStream_) cudaStreamSynchronize(lastStream_);
  else cudaDeviceSynchronize();
  for (auto& t : timed_) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto ev : freeEvents_) cudaEventDestroy(ev);
  if (openEvent_) cudaEventDestroy(openEvent_);
  clearGraphs();
  if (captureStream_) cudaStreamDestroy(captureStream_);
  if (copyIn_) {
    cudaStreamSynchronize(copyIn_);
    cudaStreamSynchronize(copyOut_);
    cudaStreamDestroy(copyIn_);
    cudaStreamDestroy(copyOut_);
    for (cudaEvent_t ev : {inReady_, inFree_, outReady_, outFree_}) cudaEventDestroy(ev);
  }
}

// ------------------------------------------------------------------ phase timing
cudaEvent_t MPMEngine::takeEvent() {
  if (!freeEvents_.empty()) {
    cudaEvent_t e = freeEvents_.back();
    freeEvents_.pop_back();
    return e;
  }
  cudaEvent_t e;
  check(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

void MPMEngine::phaseBegin(int phase, cudaStream_t s) {
  (void)phase;
  if (!profile_) return;
  openEvent_ = takeEvent();
  check(cudaEventRecord(openEvent_, s), "cudaEventRecord");
}

void MPMEngine::phaseEnd(int phase, cudaStream_t s, uint64_t launchesBefore) {
  if (!profile_ || !openEvent_) return;
  cudaEvent_t b = takeEvent();
  check(cudaEventRecord(b, s), "cudaEventRecord");
  timed_.push_back(Timed{phase, openEvent_, b, launches_ - launchesBefore});
  openEvent_ = nullptr;
}

void MPMEngine::profileEnable(bool on) { profile_ = on; }

void MPMEngine::profileRead(double* ms, uint64_t* launches, bool reset) {
  quiesce();
  for (auto& t : timed_) {
    float m = 0.f;
    check(cudaEventElapsedTime(&m, t.a, t.b), "cudaEventElapsedTime");
    phaseMs_[t.phase] += m;
    phaseLaunches_[t.phase] += t.launches;
    freeEvents_.push_back(t.a);
    freeEvents_.push_back(t.b);
  }
  timed_.clear();
  for (int i = 0; i < NEBULA_MPM_PHASES; ++i) {
    ms[i] = phaseMs_[i];
    launches[i] = phaseLaunches_[i];
  }
  if (reset)
    for (int i = 0; i < NEBULA_MPM_PHASES; ++i) {
      phaseMs_[i] = 0.0;
      phaseLaunches_[i] = 0;
    }
}

void MPMEngine::bindDevice() const { check(cudaSetDevice(device_), "cudaSetDevice"); }

void MPMEngine::quiesce() {
  bindDevice();
  check(lastStream_ ? cudaStreamSynchronize(lastStream_) : cudaDeviceSynchronize(), "synchronize");
  if (copyIn_) check(cudaStreamSynchronize(copyIn_), "synchronize uploads");
  if (copyOut_) check(cudaStreamSynchronize(copyOut_), "synchronize downloads");
}

void MPMEngine::switchStream(cudaStream_t s) {
  if (s != lastStream_) {
    quiesce();  // work queued on the previous stream must finish first
    lastStream_ = s;
  }
}

void MPMEngine::ensureStaging() {
  const size_t bytes = size_t(8) * std::max<uint32_t>(capacity_, 1u) * sizeof(float4);
  if (inStage_.bytes < bytes) {
    inStage_.alloc(bytes);
    outStage_.alloc(bytes);
  }
  if (!copyIn_) {
    check(cudaStreamCreateWithFlags(&copyIn_, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaStreamCreateWithFlags(&copyOut_, cudaStreamNonBlocking), "cudaStreamCreate");
    for (cudaEvent_t* ev : {&inReady_, &inFree_, &outReady_, &outFree_}) check(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "cudaEventCreate");
  }
}

// H2D of the new state into the input staging buffer on the upload stream
// (after the previous upload's staging copy was consumed); then, in `s`'s
// order, the staged state becomes the current one (device copy, identity
// particle order, no pending P2G).  The transfer runs while earlier work on
// `s` (a step) still computes.
void MPMEngine::uploadStateAsync(const float* const f[8], uint32_t n, cudaStream_t s) {
  if (n > capacity_) throw Error(NEBULA_MPM_ERR_INVALID, "more particles than capacity");
  for (int k = 0; k < 8; ++k)
    if (n && !f[k]) throw Error(NEBULA_MPM_ERR_INVALID, "null field");
  bindDevice();
  switchStream(s);
  ensureStaging();
  float4* stage = static_cast<float4*>(inStage_.ptr);
  const size_t cap = capacity_;
  check(cudaStreamWaitEvent(copyIn_, inFree_, 0), "cudaStreamWaitEvent");
  for (int k = 0; k < 8 && n; ++k)
    check(cudaMemcpyAsync(stage + k * cap, f[k], size_t(n) * sizeof(float4), cudaMemcpyHostToDevice, copyIn_), "upload state");
  check(cudaEventRecord(inReady_, copyIn_), "cudaEventRecord");
  check(cudaStreamWaitEvent(s, inReady_, 0), "cudaStreamWaitEvent");
  discardPending(s);
  const StatePtrs st = statePtrs(cur_);
  for (int k = 0; k < 8 && n; ++k)
    check(cudaMemcpyAsync(st.f[k], stage + k * cap, size_t(n) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "stage state");
  check(cudaEventRecord(inFree_, s), "cudaEventRecord");
  check(launchIota(static_cast<uint32_t*>(pid_[cur_].ptr), capacity_, s, &launches_), "iota");
  permuted_ = false;
  live_ = n;
  ++stateVersion_;
}

// In `s`'s order the current state goes, in original particle order, to the
// output staging buffer (after the previous download's transfer left it); the
// D2H then runs on the download stream while later work on `s` computes.
void MPMEngine::downloadStateAsync(float* const host[8], uint64_t count, cudaStream_t s) {
  if (count != uint64_t(live_) * 4) throw Error(NEBULA_MPM_ERR_INVALID, "count must be 4 * live particles");
  for (int k = 0; k < 8; ++k)
    if (count && (!host || !host[k])) throw Error(NEBULA_MPM_ERR_INVALID, "null host buffer");
  bindDevice();
  switchStream(s);
  ensureStaging();
  float4* stage = static_cast<float4*>(outStage_.ptr);
  const size_t cap = capacity_;
  StatePtrs out;
  for (int k = 0; k < 8; ++k) out.f[k] = stage + k * cap;
  check(cudaStreamWaitEvent(s, outFree_, 0), "cudaStreamWaitEvent");
  if (live_) {
    if (permuted_) {
      check(launchUnpermute(statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), out, live_, s, &launches_), "unpermute");
    } else {
      const StatePtrs st = statePtrs(cur_);
      for (int k = 0; k < 8; ++k)
        check(cudaMemcpyAsync(out.f[k], st.f[k], size_t(live_) * sizeof(float4), cudaMemcpyDeviceToDevice, s), "stage state");
    }
  }
  check(cudaEventRecord(outReady_, s), "cudaEventRecord");
  check(cudaStreamWaitEvent(copyOut_, outReady_, 0), "cudaStreamWaitEvent");
  for (int k = 0; k < 8 && count; ++k)
    check(cudaMemcpyAsync(host[k], out.f[k], count * sizeof(float), cudaMemcpyDeviceToHost, copyOut_), "download state");
  check(cudaEventRecord(outFree_, copyOut_), "cudaEventRecord");
}

void MPMEngine::waitDownloads(cudaStream_t s) {
  bindDevice();
  if (outFree_) check(cudaStreamWaitEvent(s, outFree_, 0), "cudaStreamWaitEvent");
}

void MPMEngine::setParams(const nebula_mpm_params& p) {
  if (p.numSubsteps < 0) throw Error(NEBULA_MPM_ERR_INVALID, "numSubsteps must be >= 0");
  params_ = p;
}

void validateLaunchConfig(const LaunchConfig& c) {
  if (c.fusedThreads != 0 && c.fusedThreads != 192 && c.fusedThreads != 256)
    throw Error(NEBULA_MPM_ERR_INVALID, "fused_threads must be 192 or 256 (0 = by scene size)");
  if (c.gridBatch != 2 && c.gridBatch != 4) throw Error(NEBULA_MPM_ERR_INVALID, "grid_batch must be 2 or 4");
  if (c.fusedCtasPerSm > 64 || c.gridCtasPerSm > 64) throw Error(NEBULA_MPM_ERR_INVALID, "CTAs per SM must be <= 64 (0 = as many as fit)");
  if (c.fusedSplit > 4) throw Error(NEBULA_MPM_ERR_INVALID, "fused_split must be 0-4 (0 = by scene size)");
}

LaunchConfig fromAbi(const nebula_mpm_launch_config& c) {
  LaunchConfig l;
  l.fusedThreads = c.fused_threads;
  l.fusedCtasPerSm = c.fused_ctas_per_sm;
  l.gridCtasPerSm = c.grid_ctas_per_sm;
  l.gridBatch = c.grid_batch;
  l.fusedSplit = c.fused_split;
  return l;
}

nebula_mpm_launch_config toAbi(const LaunchConfig& l) {
  nebula_mpm_launch_config c;
  c.fused_threads = l.fusedThreads;
  c.fused_ctas_per_sm = l.fusedCtasPerSm;
  c.grid_ctas_per_sm = l.gridCtasPerSm;
  c.grid_batch = l.gridBatch;
  c.fused_split = l.fusedSplit;
  return c;
}

// Takes effect at the next launch; kernels already queued keep their shape.
void MPMEngine::setLaunchConfig(const LaunchConfig& c) {
  validateLaunchConfig(c);
  launchCfg_ = c;
}

void MPMEngine::setPipeline(int p) {
  if (p != NEBULA_MPM_PIPELINE_DENSE && p != NEBULA_MPM_PIPELINE_FUSED) throw Error(NEBULA_MPM_ERR_INVALID, "unknown pipeline");
  if (p == pipeline_) return;
  bindDevice();
  prepareHostAccess(true);
  pipeline_ = p;
}

// Before the host reads or writes particle arrays: a write needs the particles
// back in their original order and any pending P2G discarded; both need the
// engine's stream drained.
void MPMEngine::prepareHostAccess(bool modifiesParticles) {
  bindDevice();
  if (modifiesParticles) {
    normalizeOrder(lastStream_);
    discardPending(lastStream_);
  }
  quiesce();
}

void MPMEngine::setMaterials(const nebula_mpm_material* mats, uint32_t n) {
  if (n == 0) return;  // MPMEngine.cpp:240
  if (n > uint32_t(kMaxMaterials)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 16 materials");
  if (!mats) throw Error(NEBULA_MPM_ERR_INVALID, "null materials");
  prepareHostAccess(true);  // rho0 enters P2G
  hostMaterials_.assign(reinterpret_cast<const Material*>(mats), reinterpret_cast<const Material*>(mats) + n);
  check(cudaMemcpy(materials_.ptr, mats, n * sizeof(Material), cudaMemcpyHostToDevice), "upload materials");
}

void MPMEngine::setParticleMaterialIds(const uint32_t* ids, uint32_t n) {
  if (n > capacity_) throw Error(NEBULA_MPM_ERR_INVALID, "more ids than particle capacity");
  if (n && !ids) throw Error(NEBULA_MPM_ERR_INVALID, "null ids");
  prepareHostAccess(true);
  std::vector<float4> v(n);
  for (uint32_t i = 0; i < n; ++i) {
    float w;
    std::memcpy(&w, ids + i, 4);
    v[i] = make_float4(0.f, 0.f, 0.f, w);
  }
  if (n) check(cudaMemcpy(statePtrs(cur_).f[1], v.data(), n * sizeof(float4), cudaMemcpyHostToDevice), "upload ids");
  ++stateVersion_;
}

void MPMEngine::setColliders(const nebula_mpm_collider* c, uint32_t n) {
  if (n > uint32_t(kMaxColliders)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 64 colliders");
  if (n && !c) throw Error(NEBULA_MPM_ERR_INVALID, "null colliders");
  prepareHostAccess(false);
  colliderCount_ = n;
  colliderTrackLen_ = 1;
  if (n) check(cudaMemcpy(colliders_.ptr, c, n * sizeof(Collider), cudaMemcpyHostToDevice), "upload colliders");
}

void MPMEngine::setColliderTrack(const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps) {
  if (perSubstep > uint32_t(kMaxColliders)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 64 colliders per substep");
  if (substeps == 0) throw Error(NEBULA_MPM_ERR_INVALID, "a collider track needs at least one substep");
  const size_t total = size_t(perSubstep) * substeps;
  if (total && !c) throw Error(NEBULA_MPM_ERR_INVALID, "null colliders");
  prepareHostAccess(false);
  colliders_.ensure(std::max(total, size_t(kMaxColliders)) * sizeof(Collider));
  colliderCount_ = perSubstep;
  colliderTrackLen_ = substeps;
  if (total) check(cudaMemcpy(colliders_.ptr, c, total * sizeof(Collider), cudaMemcpyHostToDevice), "upload collider track");
}

void MPMEngine::clearAnalyticColliders() { colliderCount_ = 0; }

void MPMEngine::setColliderSDF(const float* sdf, uint64_t n) {
  if (!sdf || n != hashCells_) throw Error(NEBULA_MPM_ERR_INVALID, "SDF must hold hashCells floats");
  prepareHostAccess(false);
  sdf_.ensure(size_t(hashCells_) * sizeof(float));
  check(cudaMemcpy(sdf_.ptr, sdf, size_t(hashCells_) * sizeof(float), cudaMemcpyHostToDevice), "upload sdf");
  hasSdf_ = true;
}

// MPMEngine::setColliderSphere (MPMEngine.cpp:180-200): cell-centre distances on the gridRes box
void MPMEngine::setColliderSphere(float radius, float cx, float cy, float cz) {
  std::vector<float> s(hashCells_, 0.0f);
  const float h = cfg_.cellSize;
  for (uint32_t iz = 0; iz < gridRes_[2]; iz++)
    for (uint32_t iy = 0; iy < gridRes_[1]; iy++)
      for (uint32_t ix = 0; ix < gridRes_[0]; ix++) {
        float wx = (ix + 0.5f) * h, wy = (iy + 0.5f) * h, wz = (iz + 0.5f) * h;
        float d = std::sqrt((wx - cx) * (wx - cx) + (wy - cy) * (wy - cy) + (wz - cz) * (wz - cz));
        s[mortonEncode(int(ix), int(iy), int(iz))] = d - radius;
      }
  setColliderSDF(s.data(), s.size());
}

void MPMEngine::clearCollider() { hasSdf_ = false; }

// setColliderSDF(buildMeshSDF(tris, gridRes, hashCells, cellSize)) (MeshSDF.h:98-132),
// the SDF built on the GPU straight into the engine's SDF buffer.  The mesh
// stays on the device, prepared (clustered), for setColliderMeshPose.
void MPMEngine::setColliderMesh(const float* tris, uint32_t n) {
  checkMeshArgs(tris, n);
  prepareHostAccess(false);  // a queued substep or rebuild may still read the old SDF or mesh
  mesh_.build(tris, n);
  hasMesh_ = true;
  sdf_.ensure(size_t(hashCells_) * sizeof(float));
  buildMeshSdf(meshPose(nullptr, nullptr));
}

// The collider mesh's SDF into the engine's SDF buffer, with the closest-point
// definition the engine is set to (setColliderMeshClosestPoint).
void MPMEngine::buildMeshSdf(const MeshPose& pose) {
  float* out = static_cast<float*>(sdf_.ptr);
  if (meshReferenceClosest_)
    check(launchMeshSdfReference(static_cast<const float*>(mesh_.tris.ptr), static_cast<const uint32_t*>(mesh_.index.ptr), mesh_.n, pose, gridRes_,
                                 hashCells_, cfg_.cellSize, out, lastStream_, &launches_),
          "mesh sdf (reference closest point)");
  else
    check(launchMeshSdfPrepared(mesh_, pose, gridRes_, hashCells_, cfg_.cellSize, out, lastStream_, &launches_), "mesh sdf");
  hasSdf_ = true;
}

void MPMEngine::setColliderMeshClosestPoint(int mode) {
  if (mode != NEBULA_MPM_CLOSEST_POINT_COMPLETE && mode != NEBULA_MPM_CLOSEST_POINT_REFERENCE)
    throw Error(NEBULA_MPM_ERR_INVALID, "closest-point mode must be NEBULA_MPM_CLOSEST_POINT_COMPLETE or _REFERENCE");
  meshReferenceClosest_ = mode == NEBULA_MPM_CLOSEST_POINT_REFERENCE;
}

// The moving-obstacle rebuild (examples/pyro_basic.cpp:130-134:
// setColliderSDF(buildMeshSDF(transformTriangles(base, t, q), ...))) from the
// mesh of the last setColliderMesh, posed and rebuilt on the device.
// Ordered on the engine's stream after the substeps already queued.
void MPMEngine::setColliderMeshPose(const float* translation, const float* rotationWxyz) {
  if (!hasMesh_) throw Error(NEBULA_MPM_ERR_INVALID, "no collider mesh: call setColliderMesh first");
  if (!translation || !rotationWxyz) throw Error(NEBULA_MPM_ERR_INVALID, "null pose");
  buildMeshSdf(meshPose(translation, rotationWxyz));
}

void MPMEngine::setForces(const nebula_mpm_force* f, uint32_t n) {
  if (n > uint32_t(kMaxForces)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 16 forces");
  if (n && !f) throw Error(NEBULA_MPM_ERR_INVALID, "null forces");
  for (uint32_t i = 0; i < n; ++i)
    if (f[i].type != FORCE_GRAVITY && f[i].type != FORCE_CONSTANT_WIND)
      throw Error(NEBULA_MPM_ERR_UNSUPPORTED, "only GRAVITY and CONSTANT_WIND forces act on the MPM grid in this build");
  prepareHostAccess(false);
  forceCount_ = n;
  hostForces_.assign(reinterpret_cast<const Force*>(f), reinterpret_cast<const Force*>(f) + n);
  if (n) check(cudaMemcpy(forces_.ptr, f, n * sizeof(Force), cudaMemcpyHostToDevice), "upload forces");
}

// The gravity entry of the force table: every GRAVITY force is replaced by one
// of vector g (direction g/|g|, strength |g|, all engines), appended if there
// was none; the other forces stay.  A zero vector removes gravity.
void MPMEngine::setGravity(float gx, float gy, float gz) {
  if (!std::isfinite(gx) || !std::isfinite(gy) || !std::isfinite(gz)) throw Error(NEBULA_MPM_ERR_INVALID, "gravity must be finite");
  std::vector<Force> t;
  for (const Force& f : hostForces_)
    if (f.type != FORCE_GRAVITY) t.push_back(f);
  const float s = std::sqrt(gx * gx + gy * gy + gz * gz);
  if (s > 0.f) {
    Force g{};
    g.type = FORCE_GRAVITY;
    g.affectMask = 0;
    g.data[0] = gx / s;
    g.data[1] = gy / s;
    g.data[2] = gz / s;
    g.data[3] = s;
    t.push_back(g);
  }
  if (t.size() > size_t(kMaxForces)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 16 forces");
  setForces(reinterpret_cast<const nebula_mpm_force*>(t.data()), uint32_t(t.size()));
}

// A field's device array in the original particle order (getPositionBuffer /
// getVelocityBuffer, MPMEngine.cpp:165-166): the particles are put back in
// that order first (a step reorders them again, so query after each step).
// Writes through the pointer are seen by the next step.
float* MPMEngine::devicePointer(int field) {
  if (field < 0 || field > 7) throw Error(NEBULA_MPM_ERR_INVALID, "field index out of range");
  prepareHostAccess(true);
  ++stateVersion_;  // the caller may write through the pointer
  return reinterpret_cast<float*>(statePtrs(cur_).f[field]);
}

uint32_t MPMEngine::appendParticles(const float* pos4, const float* vel4, uint32_t n) {
  const uint32_t nNew = std::min(n, capacity_ - live_);  // MPMEngine.cpp:212-214
  if (nNew == 0) return 0;
  if (!pos4 || !vel4) throw Error(NEBULA_MPM_ERR_INVALID, "null particle arrays");
  prepareHostAccess(true);
  std::vector<float4> F0(nNew, make_float4(1, 0, 0, 0)), F1(nNew, make_float4(0, 1, 0, 0)), F2(nNew, make_float4(0, 0, 1, 0)),
      Z(nNew, make_float4(0, 0, 0, 0));
  StatePtrs st = statePtrs(cur_);
  const size_t bytes = size_t(nNew) * sizeof(float4);
  auto up = [&](int k, const void* src) { check(cudaMemcpy(st.f[k] + live_, src, bytes, cudaMemcpyHostToDevice), "append"); };
  up(0, pos4);
  up(1, vel4);
  up(2, F0.data());
  up(3, F1.data());
  up(4, F2.data());
  up(5, Z.data());
  up(6, Z.data());
  up(7, Z.data());
  live_ += nNew;
  ++stateVersion_;
  return nNew;
}

void MPMEngine::resetParticles() {
  prepareHostAccess(true);
  live_ = 0;
  ++stateVersion_;
  std::fill(emitterDone_.begin(), emitterDone_.end(), 0);  // MPMEngine.cpp:285-286
  emitEvents_ = 0;
}

uint32_t MPMEngine::addEmitter(const nebula_mpm_emitter& em) {
  if (em.shape > 2u) throw Error(NEBULA_MPM_ERR_INVALID, "emitter shape must be 0 (AABB), 1 (SPHERE) or 2 (ELLIPSE)");
  if (em.particles_per_step < 0) throw Error(NEBULA_MPM_ERR_INVALID, "particles_per_step must be >= 0");
  if (em.step_count < -1) throw Error(NEBULA_MPM_ERR_INVALID, "step_count must be -1, 0 or positive");
  for (int a = 0; a < 3; ++a)
    if (!(em.size[a] >= 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "emitter size must be >= 0");
  if (!(em.particleVolume > 0.f) && (cfg_.nx == 0 || cfg_.ny == 0 || cfg_.nz == 0))
    throw Error(NEBULA_MPM_ERR_INVALID, "emitter particleVolume <= 0 needs the config's nx, ny, nz (MPMConfig::particleVolume)");
  EmitterRec r;
  static_assert(sizeof(r) == sizeof(em), "emitter record");
  std::memcpy(&r, &em, sizeof(r));
  emitters_.push_back(r);
  emitterDone_.push_back(0);
  return uint32_t(emitters_.size() - 1);
}

void MPMEngine::clearEmitters() {
  emitters_.clear();
  emitterDone_.clear();
}

void MPMEngine::getEmitter(uint32_t i, nebula_mpm_emitter* em, int32_t* done) const {
  if (i >= emitters_.size()) throw Error(NEBULA_MPM_ERR_INVALID, "emitter index out of range");
  std::memcpy(em, &emitters_[i], sizeof(*em));
  if (done) *done = emitterDone_[i];
}

// MPMEngine::emitFromEmitters (MPMEngine.cpp:289-352): the same schedule,
// count, truncation and centre motion; the particles are written by a kernel
// on the step's stream.  Returns whether any particle was added.
bool MPMEngine::emitFromEmitters(float dt, cudaStream_t s) {
  bool added = false;
  for (size_t si = 0; si < emitters_.size(); ++si) {
    EmitterRec& em = emitters_[si];
    int32_t& done = emitterDone_[si];
    const bool due = em.step_count == -1 ? done == 0 : (em.step_count == 0 ? true : done < em.step_count);
    if (!due) continue;
    const int64_t available = int64_t(capacity_) - int64_t(live_);
    const int64_t nNew = std::min<int64_t>(em.particles_per_step, available);
    if (nNew <= 0) {
      ++done;
      continue;
    }
    const float Vp = em.particleVolume > 0.f ? em.particleVolume
                                             : (cfg_.domainSize[0] / float(cfg_.nx)) * (cfg_.domainSize[1] / float(cfg_.ny)) *
                                                   (cfg_.domainSize[2] / float(cfg_.nz));
    check(launchEmit(em, Vp, kEmitSeed, emitEvents_++, uint32_t(nNew), statePtrs(cur_), static_cast<uint32_t*>(pid_[cur_].ptr), live_, s,
                     &launches_),
          "emit");
    live_ += uint32_t(nNew);
    ++done;
    for (int a = 0; a < 3; ++a) em.center[a] += em.center_vel[a] * dt;
    added = true;
  }
  return added;
}

void MPMEngine::uploadState(const float* const f[8], uint32_t n) {
  if (n > capacity_) throw Error(NEBULA_MPM_ERR_INVALID, "more particles than capacity");
  for (int k = 0; k < 8; ++k)
    if (n && !f[k]) throw Error(NEBULA_MPM_ERR_INVALID, "null field");
  prepareHostAccess(true);
  StatePtrs st = statePtrs(cur_);
  for (int k = 0; k < 8; ++k)
    if (n) check(cudaMemcpyAsync(st.f[k], f[k], size_t(n) * sizeof(float4), cudaMemcpyHostToDevice, lastStream_), "upload state");
  quiesce();  // the host arrays may be reused as soon as this returns
  live_ = n;
  ++stateVersion_;
}

// The state buffer holding the current particles in their original order:
// the current buffer, or the idle one after an unpermute (once per state version).
StatePtrs MPMEngine::originalOrder() {
  if (!permuted_ || !live_) return statePtrs(cur_);
  StatePtrs tmp = statePtrs(cur_ ^ 1);  // free between substeps
  if (unpermutedVersion_ != stateVersion_) {
    check(launchUnpermute(statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), tmp, live_, lastStream_, &launches_), "unpermute");
    unpermutedVersion_ = stateVersion_;
  }
  return tmp;
}

void MPMEngine::download(int field, float* host, uint64_t count) {
  if (field < 0 || field > 7) throw Error(NEBULA_MPM_ERR_INVALID, "field index out of range");
  if (count != uint64_t(live_) * 4) throw Error(NEBULA_MPM_ERR_INVALID, "count must be 4 * live particles");
  if (count && !host) throw Error(NEBULA_MPM_ERR_INVALID, "null host buffer");
  bindDevice();
  const float4* src = originalOrder().f[field];
  quiesce();
  if (count) check(cudaMemcpy(host, src, count * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

void MPMEngine::downloadState(float* const host[8], uint64_t count) {
  if (count != uint64_t(live_) * 4) throw Error(NEBULA_MPM_ERR_INVALID, "count must be 4 * live particles");
  for (int k = 0; k < 8; ++k)
    if (count && (!host || !host[k])) throw Error(NEBULA_MPM_ERR_INVALID, "null host buffer");
  bindDevice();
  const StatePtrs src = originalOrder();
  for (int k = 0; k < 8 && count; ++k)
    check(cudaMemcpyAsync(host[k], src.f[k], count * sizeof(float), cudaMemcpyDeviceToHost, lastStream_), "download");
  quiesce();
}

SubstepParams MPMEngine::buildParams(float subDt) const {
  SubstepParams P{};
  P.dt = subDt;
  P.cellSize = cfg_.cellSize;
  for (int a = 0; a < 3; ++a) {
    P.gridRes[a] = int(gridRes_[a]);
    P.worldMin[a] = 0.0f;
    P.worldMax[a] = cfg_.domainSize[a];
  }
  P.cubeRes = cubeRes_;
  P.hashCells = hashCells_;
  P.flip_ratio = params_.flip_ratio;
  P.materialCount = uint32_t(hostMaterials_.size());
  P.colliderCount = colliderCount_;
  P.forceCount = forceCount_;
  P.mu_lame = cfg_.E / (2.0f * (1.0f + cfg_.nu));
  P.lambda_lame = cfg_.E * cfg_.nu / ((1.0f + cfg_.nu) * (1.0f - 2.0f * cfg_.nu));
  P.rho0 = cfg_.rho0;
  P.M_friction = params_.M_friction;
  P.q_cohesion = params_.q_cohesion;
  P.q_max = params_.q_max;
  P.plasticModel = params_.plasticModel;
  P.materials = static_cast<const Material*>(materials_.ptr);
  P.colliders = static_cast<const Collider*>(colliders_.ptr);
  P.forces = static_cast<const Force*>(forces_.ptr);
  P.sdf = hasSdf_ ? static_cast<const float*>(sdf_.ptr) : nullptr;
  return P;
}

StatePtrs MPMEngine::statePtrs(int buf) {
  StatePtrs s;
  for (int k = 0; k < 8; ++k) s.f[k] = static_cast<float4*>(buf == 0 ? state_[k].ptr : stateB_[k].ptr);
  return s;
}
StatePtrs MPMEngine::statePtrs() { return statePtrs(cur_); }

// q: the buffer whose state the binning describes (its counts are array q).
BrickBuffers MPMEngine::brickBuffers(int q) {
  BrickBuffers b;
  b.nb = nb_;
  b.tiles = tiles_;
  b.brickCount = static_cast<uint32_t*>(bCount_.ptr);
  b.brickFlag = static_cast<uint32_t*>(bFlag_.ptr);
  b.brickStart = static_cast<uint32_t*>(bStart_.ptr);
  b.cellCount = static_cast<uint32_t*>(cCount_[q & 1].ptr);
  b.cellPrev = static_cast<uint32_t*>(cCount_[(q & 1) ^ 1].ptr);
  b.pbBrick = static_cast<uint32_t*>(pbBrick_.ptr);
  b.pbStart = static_cast<uint32_t*>(pbStart_.ptr);
  b.gbBrick = static_cast<uint32_t*>(gbBrick_.ptr);
  b.counters = static_cast<uint32_t*>(counters_.ptr);
  b.scanState = static_cast<unsigned long long*>(scanState_.ptr);
  b.scanTile = static_cast<unsigned long long*>(scanTile_.ptr);
  b.binKey = static_cast<uint32_t*>(binKey_.ptr);
  b.binRank = static_cast<uint32_t*>(binRank_.ptr);
  b.perm = static_cast<uint32_t*>(perm_.ptr);
  return b;
}

GridBuffers MPMEngine::gridBuffers() {
  GridBuffers g;
  g.acc = static_cast<float4*>(gridAcc_.ptr);
  g.vel = static_cast<float4*>(gridVel_.ptr);
  g.vold = nullptr;
  if (params_.flip_ratio > 0.01f) {
    if (!gridVold_.ptr) {
      gridVold_.alloc(size_t(ncPad_) * sizeof(float4));
      check(cudaMemset(gridVold_.ptr, 0, gridVold_.bytes), "cudaMemset");
    }
    g.vold = static_cast<float4*>(gridVold_.ptr);
  }
  return g;
}

// Buffers of the dense pipeline (and of the reference-format binning export),
// allocated on first use.
void MPMEngine::ensureDense() {
  if (denseReady_) return;
  const size_t nc = hashCells_;
  const size_t pc = size_t(std::max(capacity_, 1u)) * sizeof(uint32_t);
  gridMom_.alloc(nc * 2 * sizeof(float4));
  gridMass_.alloc(nc * sizeof(float));
  check(cudaMemset(gridMom_.ptr, 0, gridMom_.bytes), "cudaMemset");
  check(cudaMemset(gridMass_.ptr, 0, gridMass_.bytes), "cudaMemset");
  cellCount_.alloc(nc * sizeof(uint32_t));
  cellStart_.alloc(nc * sizeof(uint32_t));
  cellEnd_.alloc(nc * sizeof(uint32_t));
  key_.alloc(pc);
  rank_.alloc(pc);
  sortedTmp_.alloc(pc);
  sorted_.alloc(pc);
  scanWs_.alloc(scanWorkspaceBytes(nc));
  denseReady_ = true;
}

BinBuffers MPMEngine::binBuffers() {
  ensureDense();
  BinBuffers b;
  b.cellCount = static_cast<uint32_t*>(cellCount_.ptr);
  b.cellStart = static_cast<uint32_t*>(cellStart_.ptr);
  b.cellEnd = static_cast<uint32_t*>(cellEnd_.ptr);
  b.key = static_cast<uint32_t*>(key_.ptr);
  b.rank = static_cast<uint32_t*>(rank_.ptr);
  b.sortedTmp = static_cast<uint32_t*>(sortedTmp_.ptr);
  b.sorted = static_cast<uint32_t*>(sorted_.ptr);
  b.tileState = static_cast<unsigned long long*>(scanWs_.ptr);
  b.tileCounter = reinterpret_cast<uint32_t*>(b.tileState + scanTiles(hashCells_));
  b.err = static_cast<uint32_t*>(err_.ptr);
  return b;
}

// Put the particles back in original order (buffer index == particle index).
void MPMEngine::normalizeOrder(cudaStream_t s) {
  if (!permuted_) return;
  StatePtrs src = statePtrs(cur_), dst = statePtrs(cur_ ^ 1);
  check(launchUnpermute(src, static_cast<const uint32_t*>(pid_[cur_].ptr), dst, live_, s, &launches_), "unpermute");
  cur_ ^= 1;
  ++stateVersion_;
  check(launchIota(static_cast<uint32_t*>(pid_[cur_].ptr), capacity_, s, &launches_), "iota");
  permuted_ = false;
  // the pending bins index the old order
  discardPending(s);
}

void MPMEngine::discardPending(cudaStream_t s) {
  if (!pending_) return;
  check(launchClearBricks(brickBuffers(cur_), gridBuffers(), numSMs_, s, &launches_), "clear bricks");
  pending_ = false;
}

bool MPMEngine::pendingMatches(float subDt) const {
  return pending_ && pendingDt_ == subDt && pendingApic_ == (params_.flip_ratio < -0.5f);
}

// Bin the current particles (buffer order), then P2G them into the brick grid.
void MPMEngine::buildPending(const SubstepParams& P, cudaStream_t s) {
  BrickBuffers B = brickBuffers(cur_);
  GridBuffers G = gridBuffers();
  uint32_t* err = static_cast<uint32_t*>(err_.ptr);
  uint64_t l0 = launches_;
  phaseBegin(kPhaseBin, s);
  // a binning from scratch: neither count array may hold an earlier binning's counts
  for (DevBuf& c : cCount_) check(cudaMemsetAsync(c.ptr, 0, c.bytes, s), "clear cell counts");
  check(launchBrickCount(P, statePtrs(cur_).f[0], live_, B, err, s, &launches_), "brick count");
  check(launchBrickScan(B, err, s, &launches_), "brick scan");
  check(launchPermScatter(B, live_, err, s, &launches_), "perm scatter");
  phaseEnd(kPhaseBin, s, l0);
  l0 = launches_;
  phaseBegin(kPhaseP2G, s);
  check(launchP2GBricks(P, statePtrs(cur_), live_, B, G, P.dt, numSMs_, s, &launches_), "p2g bricks");
  phaseEnd(kPhaseP2G, s, l0);
  pending_ = true;
  pendingDt_ = P.dt;
  pendingApic_ = P.flip_ratio < -0.5f;
}

// One substep on the pending grid: grid update, fused G2P + P2G (+ binning
// count), brick scan, permutation.  Leaves the next substep's grid pending.
void MPMEngine::substepFused(const SubstepParams& P, cudaStream_t s) {
  // the binning of the state read (buffer cur_) and of the state written
  const BrickBuffers B = brickBuffers(cur_), Bn = brickBuffers(cur_ ^ 1);
  GridBuffers G = gridBuffers();
  uint32_t* err = static_cast<uint32_t*>(err_.ptr);
  uint64_t l0 = launches_;
  phaseBegin(kPhaseGrid, s);
  const bool fold = live_ < kFoldScatterMax;
  check(launchGridBricks(P, B, G, fold ? live_ : 0u, err, launchCfg_, numSMs_, s, &launches_), "grid bricks");
  phaseEnd(kPhaseGrid, s, l0);
  l0 = launches_;
  phaseBegin(kPhaseFused, s);
  check(launchG2P2G(P, modelSetOf(hostMaterials_.data(), uint32_t(hostMaterials_.size())), statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), statePtrs(cur_ ^ 1),
                    static_cast<uint32_t*>(pid_[cur_ ^ 1].ptr), live_, Bn, G, P.dt, err, launchCfg_, numSMs_, s, &launches_),
        "g2p2g");
  phaseEnd(kPhaseFused, s, l0);
  l0 = launches_;
  phaseBegin(kPhaseBin, s);
  check(launchBrickScan(Bn, err, s, &launches_), "brick scan");
  // the permutation of this binning: here, or by the next grid launch
  if (!fold) check(launchPermScatter(Bn, live_, err, s, &launches_), "perm scatter");
  phaseEnd(kPhaseBin, s, l0);
  cur_ ^= 1;
  permuted_ = true;
  ++substeps_;
}

// One substep in the reference's pass order (MPMEngine.cpp:419-472): bin,
// zero the grid, P2G, grid update (+ SDF boundary fused per node), G2P.
void MPMEngine::substepDense(const SubstepParams& P, cudaStream_t s) {
  BinBuffers b = binBuffers();
  StatePtrs st = statePtrs(cur_);
  uint64_t l0 = launches_;
  phaseBegin(kPhaseBin, s);
  check(launchBin(P, st.f[0], live_, b, s, &launches_), "bin");
  phaseEnd(kPhaseBin, s, l0);
  check(cudaMemsetAsync(gridMom_.ptr, 0, gridMom_.bytes, s), "zero grid");
  check(cudaMemsetAsync(gridMass_.ptr, 0, gridMass_.bytes, s), "zero grid");
  l0 = launches_;
  phaseBegin(kPhaseP2G, s);
  check(launchP2GDense(P, st, b.sorted, live_, static_cast<float4*>(gridMom_.ptr), static_cast<float*>(gridMass_.ptr), s, &launches_), "p2g");
  phaseEnd(kPhaseP2G, s, l0);
  l0 = launches_;
  phaseBegin(kPhaseGrid, s);
  check(launchGridDense(P, static_cast<float4*>(gridMom_.ptr), static_cast<const float*>(gridMass_.ptr), s, &launches_), "grid");
  phaseEnd(kPhaseGrid, s, l0);
  l0 = launches_;
  phaseBegin(kPhaseG2P, s);
  check(launchG2PDense(P, st, live_, static_cast<const float4*>(gridMom_.ptr), static_cast<const float*>(gridMass_.ptr), b.err, s, &launches_),
        "g2p");
  phaseEnd(kPhaseG2P, s, l0);
  ++substeps_;
}

void MPMEngine::step(float dt, cudaStream_t s) {
  bindDevice();
  if (!(dt >= 0.f) || !std::isfinite(dt)) throw Error(NEBULA_MPM_ERR_INVALID, "dt must be finite and >= 0");
  ++stateVersion_;
  if (s != lastStream_) {
    // work queued on the previous stream must finish first
    quiesce();
    lastStream_ = s;
  }
  // the emitters run first (MPMEngine.cpp:406); new particles invalidate the pending P2G
  if (!emitters_.empty() && emitFromEmitters(dt, s)) discardPending(s);
  const int n = std::max(1, params_.numSubsteps);
  const float subDt = dt / float(n);  // MPMEngine.cpp:413
  const SubstepParams P = buildParams(subDt);
  if (params_.numSubsteps <= 0 || live_ == 0) return;
  if (pipeline_ == NEBULA_MPM_PIPELINE_DENSE) {
    normalizeOrder(s);
    discardPending(s);
    for (int k = 0; k < params_.numSubsteps; ++k) substepDense(atSubstep(P, k), s);
    return;
  }
  if (!pendingMatches(subDt)) {
    discardPending(s);
    buildPending(P, s);
  }
  runFused(P, s);
}

// substep k reads collider set min(k, trackLen - 1) of the track
SubstepParams MPMEngine::atSubstep(const SubstepParams& P, int k) const {
  SubstepParams Pk = P;
  Pk.colliders += size_t(std::min(uint32_t(k), colliderTrackLen_ - 1)) * colliderCount_;
  return Pk;
}

namespace {
template <class T>
void putKey(std::vector<unsigned char>& k, const T& v) {
  const auto* p = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), p, p + sizeof(T));
}
}  // namespace
// graph keys compare these records as bytes, so none of them may have padding
static_assert(sizeof(SubstepParams) == 24 * 4 + 4 * sizeof(void*), "SubstepParams has padding");
static_assert(sizeof(BrickBuffers) == 2 * 4 + 14 * sizeof(void*), "BrickBuffers has padding");
static_assert(sizeof(StatePtrs) == 8 * sizeof(void*), "StatePtrs has padding");
static_assert(sizeof(GridBuffers) == 3 * sizeof(void*), "GridBuffers has padding");
static_assert(sizeof(LaunchConfig) == 5 * 4, "LaunchConfig has padding");

std::vector<unsigned char> MPMEngine::graphKey(const SubstepParams& P) {
  std::vector<unsigned char> k;
  k.reserve(512);
  putKey(k, P);
  putKey(k, colliderTrackLen_);
  putKey(k, params_.numSubsteps);
  putKey(k, live_);
  putKey(k, cur_);
  putKey(k, statePtrs(0));
  putKey(k, statePtrs(1));
  putKey(k, pid_[0].ptr);
  putKey(k, pid_[1].ptr);
  putKey(k, brickBuffers(cur_));
  putKey(k, gridBuffers());
  putKey(k, err_.ptr);
  putKey(k, launchCfg_);
  putKey(k, numSMs_);
  putKey(k, modelSetOf(hostMaterials_.data(), uint32_t(hostMaterials_.size())));  // the fused kernel's instantiation
  return k;
}

bool MPMEngine::graphsUsable(cudaStream_t s) const {
  if (!useGraphs_ || profile_) return false;
  // inside a capture of the caller's the launches go into the caller's graph
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return st == cudaStreamCaptureStatusNone;
}

void MPMEngine::clearGraphs() {
  for (auto& g : graphs_) {
    if (g.exec) cudaGraphExecDestroy(g.exec);  // an in-flight replay completes first
    g = StepGraph{};
  }
}

void MPMEngine::setGraphs(bool on) {
  bindDevice();
  if (!on) clearGraphs();
  useGraphs_ = on;
}

// The fused substep loop of one step, uncaptured or replayed from a graph.
// Graphs are captured on an engine-owned stream (capture only records) and
// launched on `s`, which may be the legacy default stream.
void MPMEngine::runFused(const SubstepParams& P, cudaStream_t s) {
  const int n = params_.numSubsteps;
  auto loop = [&](cudaStream_t q) {
    for (int k = 0; k < n; ++k) substepFused(atSubstep(P, k), q);
  };
  if (!graphsUsable(s)) {
    loop(s);
    return;
  }
  StepGraph& g = graphs_[cur_];
  std::vector<unsigned char> key = graphKey(P);
  if (g.key != key) {
    // not what the last step of this parity ran: run it uncaptured, remember it
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = StepGraph{};
    g.key = std::move(key);
    loop(s);
    return;
  }
  if (!g.exec) {
    if (!captureStream_) check(cudaStreamCreateWithFlags(&captureStream_, cudaStreamNonBlocking), "cudaStreamCreate");
    // the host-side counters advance during the capture as for one run; they
    // are put back and advanced below as for every replay
    const int cur0 = cur_;
    const bool perm0 = permuted_;
    const uint64_t sub0 = substeps_, l0 = launches_;
    auto restore = [&] {
      cur_ = cur0;
      permuted_ = perm0;
      substeps_ = sub0;
      launches_ = l0;
    };
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(captureStream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      loop(captureStream_);
    } catch (...) {
      cudaStreamEndCapture(captureStream_, &graph);
      if (graph) cudaGraphDestroy(graph);
      restore();
      throw;
    }
    const cudaError_t ec = cudaStreamEndCapture(captureStream_, &graph);
    const uint64_t launched = launches_ - l0;
    restore();
    check(ec, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    check(ei, "cudaGraphInstantiate");
    g.exec = exec;
    g.launches = launched;
  }
  check(cudaGraphLaunch(g.exec, s), "cudaGraphLaunch");
  ++graphLaunches_;
  launches_ += g.launches;
  substeps_ += uint64_t(n);
  if (n & 1) cur_ ^= 1;
  permuted_ = true;
}

void MPMEngine::exportBins(uint32_t* cnt, uint32_t* off, uint32_t* srt) {
  bindDevice();
  const SubstepParams P = buildParams(0.f);
  BinBuffers b = binBuffers();
  const float4* pos = originalOrder().f[0];
  check(launchBin(P, pos, live_, b, lastStream_, &launches_), "bin");
  quiesce();
  check(cudaMemcpy(cnt, b.cellCount, size_t(hashCells_) * 4, cudaMemcpyDeviceToHost), "download bins");
  check(cudaMemcpy(off, b.cellEnd, size_t(hashCells_) * 4, cudaMemcpyDeviceToHost), "download bins");
  if (live_) check(cudaMemcpy(srt, b.sorted, size_t(live_) * 4, cudaMemcpyDeviceToHost), "download bins");
}

void MPMEngine::exportBrickBins(uint32_t* numBricks, uint32_t* brickIds, uint32_t* brickStarts, uint32_t* sortedPids) {
  bindDevice();
  if (pipeline_ != NEBULA_MPM_PIPELINE_FUSED) throw Error(NEBULA_MPM_ERR_INVALID, "brick bins exist in the FUSED pipeline only");
  cudaStream_t s = lastStream_;
  // binning does not depend on dt; a grid built here is rebuilt by a step with dt != 0
  if (!pending_) buildPending(buildParams(0.f), s);
  // after a step the last binning's permutation waits for the next grid
  // launch, which reads the bin keys again: scatter it here (the same
  // values) and keep the keys intact
  check(launchPermScatter(brickBuffers(cur_), live_, static_cast<uint32_t*>(err_.ptr), s, &launches_), "perm scatter");
  DevBuf sortedTmp;
  sortedTmp.alloc(size_t(std::max<uint32_t>(live_, 1u)) * sizeof(uint32_t));
  uint32_t* tmp = static_cast<uint32_t*>(sortedTmp.ptr);
  check(launchSortedPid(static_cast<const uint32_t*>(perm_.ptr), static_cast<const uint32_t*>(pid_[cur_].ptr), tmp, live_, s, &launches_),
        "sorted pid");
  quiesce();
  uint32_t cnt[kCntSlots];
  check(cudaMemcpy(cnt, counters_.ptr, sizeof(cnt), cudaMemcpyDeviceToHost), "download counters");
  *numBricks = cnt[kCntNumPB];
  if (cnt[kCntNumPB] > nb_) throw Error(NEBULA_MPM_ERR_DEVICE, "brick count exceeds the brick grid");
  check(cudaMemcpy(brickIds, pbBrick_.ptr, size_t(cnt[kCntNumPB]) * 4, cudaMemcpyDeviceToHost), "download bricks");
  check(cudaMemcpy(brickStarts, pbStart_.ptr, size_t(cnt[kCntNumPB] + 1) * 4, cudaMemcpyDeviceToHost), "download bricks");
  if (live_) check(cudaMemcpy(sortedPids, tmp, size_t(live_) * 4, cudaMemcpyDeviceToHost), "download bricks");
  // the bin keys and the pending grid stay valid for the next step
}

void MPMEngine::exportGrid(float dt, float* mom, float* mass) {
  bindDevice();
  const SubstepParams P = buildParams(dt);
  cudaStream_t s = lastStream_;
  std::vector<float4> acc(hashCells_);
  if (pipeline_ == NEBULA_MPM_PIPELINE_FUSED) {
    if (!pendingMatches(dt)) {
      discardPending(s);
      buildPending(P, s);
    }
    quiesce();
    check(cudaMemcpy(acc.data(), gridAcc_.ptr, size_t(hashCells_) * sizeof(float4), cudaMemcpyDeviceToHost), "download grid");
    for (uint32_t i = 0; i < hashCells_; ++i) {
      mom[4 * size_t(i)] = acc[i].x;
      mom[4 * size_t(i) + 1] = acc[i].y;
      mom[4 * size_t(i) + 2] = acc[i].z;
      mom[4 * size_t(i) + 3] = 0.f;
      mass[i] = acc[i].w;
    }
    return;
  }
  normalizeOrder(s);
  BinBuffers b = binBuffers();
  StatePtrs st = statePtrs(cur_);
  check(cudaMemsetAsync(gridMom_.ptr, 0, gridMom_.bytes, s), "zero grid");
  check(cudaMemsetAsync(gridMass_.ptr, 0, gridMass_.bytes, s), "zero grid");
  check(launchBin(P, st.f[0], live_, b, s, &launches_), "bin");
  check(launchP2GDense(P, st, b.sorted, live_, static_cast<float4*>(gridMom_.ptr), static_cast<float*>(gridMass_.ptr), s, &launches_), "p2g");
  quiesce();
  check(cudaMemcpy(mom, gridMom_.ptr, size_t(hashCells_) * sizeof(float4), cudaMemcpyDeviceToHost), "download grid");
  check(cudaMemcpy(mass, gridMass_.ptr, size_t(hashCells_) * sizeof(float), cudaMemcpyDeviceToHost), "download grid");
}

uint32_t MPMEngine::syncAndCheck() {
  quiesce();
  uint32_t e = 0;
  check(cudaMemcpy(&e, err_.ptr, 4, cudaMemcpyDeviceToHost), "read error flags");
  errorFlags_ = e;
  return e;
}

void MPMEngine::stats(nebula_mpm_stats* s) {
  std::memset(s, 0, sizeof(*s));
  if (pipeline_ == NEBULA_MPM_PIPELINE_FUSED && counters_.ptr) {
    quiesce();
    uint32_t cnt[kCntSlots];
    check(cudaMemcpy(cnt, counters_.ptr, sizeof(cnt), cudaMemcpyDeviceToHost), "download counters");
    particleBricks_ = cnt[kCntNumPB];
    activeBricks_ = cnt[kCntNumGB];
    overflow_ = cnt[kCntOverflow];
  }
  s->substeps = substeps_;
  s->live_particles = live_;
  s->active_bricks = activeBricks_;
  s->particle_bricks = particleBricks_;
  for (int a = 0; a < 3; ++a) s->grid_res[a] = gridRes_[a];
  s->cube_res = cubeRes_;
  s->hash_cells = hashCells_;
  s->kernel_launches = launches_;
  s->overflow_particles = overflow_;
  s->error_flags = errorFlags_;
  s->graph_launches = graphLaunches_;
}

}  // namespace nebula

// ====================================================================== C ABI
using nebula::Error;
using nebula::g_last_error;

struct nebula_mpm {
  std::unique_ptr<nebula::MPMEngine> eng;
};

namespace {
template <class F> int guarded(F&& f) {
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
nebula::MPMEngine& E(nebula_mpm* e) {
  if (!e || !e->eng) throw Error(NEBULA_MPM_ERR_INVALID, "null engine handle");
  return *e->eng;
}
const nebula::MPMEngine& E(const nebula_mpm* e) {
  if (!e || !e->eng) throw Error(NEBULA_MPM_ERR_INVALID, "null engine handle");
  return *e->eng;
}
}  // namespace

extern "C" {

const char* nebula_mpm_last_error(void) { return g_last_error.c_str(); }

int nebula_mpm_create(const nebula_mpm_config* cfg, nebula_mpm** out) {
  return guarded([&] {
    if (!cfg || !out) throw Error(NEBULA_MPM_ERR_INVALID, "null argument");
    *out = nullptr;
    auto h = std::make_unique<nebula_mpm>();
    h->eng = std::make_unique<nebula::MPMEngine>(*cfg);
    *out = h.release();
  });
}
int nebula_mpm_destroy(nebula_mpm* e) {
  return guarded([&] { delete e; });
}
int nebula_mpm_set_params(nebula_mpm* e, const nebula_mpm_params* p) {
  return guarded([&] {
    if (!p) throw Error(NEBULA_MPM_ERR_INVALID, "null params");
    E(e).setParams(*p);
  });
}
int nebula_mpm_get_params(const nebula_mpm* e, nebula_mpm_params* p) {
  return guarded([&] {
    if (!p) throw Error(NEBULA_MPM_ERR_INVALID, "null params");
    *p = E(e).params();
  });
}
int nebula_mpm_set_materials(nebula_mpm* e, const nebula_mpm_material* m, uint32_t n) {
  return guarded([&] { E(e).setMaterials(m, n); });
}
int nebula_mpm_set_particle_material_ids(nebula_mpm* e, const uint32_t* ids, uint32_t n) {
  return guarded([&] { E(e).setParticleMaterialIds(ids, n); });
}
int nebula_mpm_set_colliders(nebula_mpm* e, const nebula_mpm_collider* c, uint32_t n) {
  return guarded([&] { E(e).setColliders(c, n); });
}
int nebula_mpm_set_collider_track(nebula_mpm* e, const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps) {
  return guarded([&] { E(e).setColliderTrack(c, perSubstep, substeps); });
}
int nebula_mpm_clear_analytic_colliders(nebula_mpm* e) {
  return guarded([&] { E(e).clearAnalyticColliders(); });
}
int nebula_mpm_set_collider_sdf(nebula_mpm* e, const float* sdf, uint64_t n) {
  return guarded([&] { E(e).setColliderSDF(sdf, n); });
}
int nebula_mpm_set_collider_sphere(nebula_mpm* e, float r, float cx, float cy, float cz) {
  return guarded([&] { E(e).setColliderSphere(r, cx, cy, cz); });
}
int nebula_mpm_set_collider_mesh(nebula_mpm* e, const float* tris, uint32_t n) {
  return guarded([&] { E(e).setColliderMesh(tris, n); });
}
int nebula_mpm_set_collider_mesh_pose(nebula_mpm* e, const float translation[3], const float rotation_wxyz[4]) {
  return guarded([&] { E(e).setColliderMeshPose(translation, rotation_wxyz); });
}
int nebula_mpm_set_collider_mesh_closest_point(nebula_mpm* e, int mode) {
  return guarded([&] { E(e).setColliderMeshClosestPoint(mode); });
}
int nebula_mpm_clear_collider(nebula_mpm* e) {
  return guarded([&] { E(e).clearCollider(); });
}
int nebula_mpm_set_forces(nebula_mpm* e, const nebula_mpm_force* f, uint32_t n) {
  return guarded([&] { E(e).setForces(f, n); });
}
int nebula_mpm_append_particles(nebula_mpm* e, const float* pos4, const float* vel4, uint32_t n, uint32_t* appended) {
  return guarded([&] {
    uint32_t k = E(e).appendParticles(pos4, vel4, n);
    if (appended) *appended = k;
  });
}
namespace {
// SplitMix64 at counter i (1-based) of the stream (seed, stream): the base
// seed * 0x100000001B3 + stream * 0xD1B54A32D192ED03 plus i golden-ratio
// increments, then the SplitMix64 finaliser (Steele, Lea, Flood 2014).
uint64_t splitmix64At(uint64_t base, uint64_t i) {
  uint64_t z = base + i * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t latticeCount(const nebula_mpm_lattice& L) { return uint64_t(L.counts[0]) * L.counts[1] * L.counts[2]; }

void latticePoints(const nebula_mpm_lattice& L, float* pos4, float* vel4) {
  const uint64_t base = L.seed * 0x100000001B3ull + L.stream * 0xD1B54A32D192ED03ull;
  const uint32_t nx = L.counts[0], ny = L.counts[1], nz = L.counts[2];
  float idBits;
  std::memcpy(&idBits, &L.materialId, 4);
  uint64_t p = 0;
  for (uint32_t iy = 0; iy < ny; ++iy)
    for (uint32_t iz = 0; iz < nz; ++iz)
      for (uint32_t ix = 0; ix < nx; ++ix, ++p) {
        const uint32_t idx[3] = {ix, iy, iz};
        for (int a = 0; a < 3; ++a) {
          // top 53 bits as a double in [0, 1), then lo + (hi - lo) * u; the
          // products are kept apart from the sums (no fused multiply-add), so
          // the points are the same on every host
          const double u = double(splitmix64At(base, 3 * p + a + 1) >> 11) * (1.0 / 9007199254740992.0);
          const volatile double ju = (2.0 * L.jitter) * u;
          const volatile double at = double(idx[a]) * L.spacing;
          pos4[4 * p + a] = float((at + L.origin[a]) + (-L.jitter + ju));
          vel4[4 * p + a] = L.vel[a];
        }
        pos4[4 * p + 3] = L.particleVolume;
        vel4[4 * p + 3] = idBits;
      }
}
}  // namespace

int nebula_mpm_lattice_points(const nebula_mpm_lattice* L, float* pos4, float* vel4, uint64_t n) {
  return guarded([&] {
    if (!L) throw Error(NEBULA_MPM_ERR_INVALID, "null lattice");
    if (n != latticeCount(*L)) throw Error(NEBULA_MPM_ERR_INVALID, "n must be counts[0] * counts[1] * counts[2]");
    if (n && (!pos4 || !vel4)) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    latticePoints(*L, pos4, vel4);
  });
}
int nebula_mpm_append_lattice(nebula_mpm* e, const nebula_mpm_lattice* L, uint32_t* appended) {
  return guarded([&] {
    if (!L) throw Error(NEBULA_MPM_ERR_INVALID, "null lattice");
    const uint64_t n = latticeCount(*L);
    if (n > 0xFFFFFFFFull) throw Error(NEBULA_MPM_ERR_INVALID, "lattice larger than 2^32 points");
    std::vector<float> pos(4 * n), vel(4 * n);
    latticePoints(*L, pos.data(), vel.data());
    const uint32_t k = E(e).appendParticles(pos.data(), vel.data(), uint32_t(n));
    if (appended) *appended = k;
  });
}
int nebula_mpm_add_emitter(nebula_mpm* e, const nebula_mpm_emitter* em, uint32_t* index) {
  return guarded([&] {
    if (!em) throw Error(NEBULA_MPM_ERR_INVALID, "null emitter");
    const uint32_t i = E(e).addEmitter(*em);
    if (index) *index = i;
  });
}
int nebula_mpm_clear_emitters(nebula_mpm* e) {
  return guarded([&] { E(e).clearEmitters(); });
}
int nebula_mpm_get_emitter(const nebula_mpm* e, uint32_t index, nebula_mpm_emitter* em, int32_t* stepsDone) {
  return guarded([&] {
    if (!em) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).getEmitter(index, em, stepsDone);
  });
}
int nebula_mpm_reset_particles(nebula_mpm* e) {
  return guarded([&] { E(e).resetParticles(); });
}
int nebula_mpm_upload_state(nebula_mpm* e, const float* const fields[8], uint32_t n) {
  return guarded([&] {
    if (!fields) throw Error(NEBULA_MPM_ERR_INVALID, "null fields");
    E(e).uploadState(fields, n);
  });
}
int nebula_mpm_upload_state_async(nebula_mpm* e, const float* const fields[8], uint32_t n, void* stream) {
  return guarded([&] {
    if (!fields) throw Error(NEBULA_MPM_ERR_INVALID, "null fields");
    E(e).uploadStateAsync(fields, n, static_cast<cudaStream_t>(stream));
  });
}
int nebula_mpm_download_state_async(nebula_mpm* e, float* const host[8], uint64_t count, void* stream) {
  return guarded([&] { E(e).downloadStateAsync(host, count, static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_wait_downloads(nebula_mpm* e, void* stream) {
  return guarded([&] { E(e).waitDownloads(static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_download(nebula_mpm* e, int field, float* host, uint64_t count) {
  return guarded([&] { E(e).download(field, host, count); });
}
int nebula_mpm_download_state(nebula_mpm* e, float* const host[8], uint64_t count) {
  return guarded([&] { E(e).downloadState(host, count); });
}
int nebula_mpm_device_ptr(nebula_mpm* e, int field, float** out) {
  return guarded([&] {
    if (!out) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *out = E(e).devicePointer(field);
  });
}
int nebula_mpm_probe_wait_expiry(uint32_t* error_bits) {
  return guarded([&] {
    if (!error_bits) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    nebula::check(nebula::probeWaitExpiry(error_bits), "wait-expiry probe");
  });
}
int nebula_mpm_set_gravity(nebula_mpm* e, float gx, float gy, float gz) {
  return guarded([&] { E(e).setGravity(gx, gy, gz); });
}
int nebula_mpm_step(nebula_mpm* e, float dt, void* stream) {
  return guarded([&] { E(e).step(dt, static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_live_count(const nebula_mpm* e, uint32_t* n) {
  return guarded([&] {
    if (!n) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *n = E(e).liveCount();
  });
}
int nebula_mpm_get_stats(nebula_mpm* e, nebula_mpm_stats* s) {
  return guarded([&] {
    if (!s) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).stats(s);
  });
}
int nebula_mpm_sync(nebula_mpm* e) {
  return guarded([&] {
    uint32_t f = E(e).syncAndCheck();
    if (f & ~nebula::kErrTileOverflow) {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "device error flags 0x%x (1: bounded wait expired, 2: non-finite particle state)", f);
      throw Error(NEBULA_MPM_ERR_DEVICE, buf);
    }
  });
}
int nebula_mpm_profile_enable(nebula_mpm* e, int enable) {
  return guarded([&] { E(e).profileEnable(enable != 0); });
}
int nebula_mpm_profile_read(nebula_mpm* e, double ms[NEBULA_MPM_PHASES], uint64_t launches[NEBULA_MPM_PHASES], int reset) {
  return guarded([&] {
    if (!ms || !launches) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).profileRead(ms, launches, reset != 0);
  });
}
int nebula_mpm_set_pipeline(nebula_mpm* e, int pipeline) {
  return guarded([&] { E(e).setPipeline(pipeline); });
}
int nebula_mpm_set_launch_config(nebula_mpm* e, const nebula_mpm_launch_config* c) {
  return guarded([&] {
    if (!c) throw Error(NEBULA_MPM_ERR_INVALID, "null launch config");
    E(e).setLaunchConfig(nebula::fromAbi(*c));
  });
}
int nebula_mpm_set_graphs(nebula_mpm* e, int enable) {
  return guarded([&] { E(e).setGraphs(enable != 0); });
}
int nebula_mpm_get_launch_config(nebula_mpm* e, nebula_mpm_launch_config* c) {
  return guarded([&] {
    if (!c) throw Error(NEBULA_MPM_ERR_INVALID, "null launch config");
    *c = nebula::toAbi(E(e).launchConfig());
  });
}
int nebula_mpm_launch_limits(int flip, int batch, uint32_t fused_ctas_per_sm[2], uint32_t grid_ctas_per_sm[2]) {
  return guarded([&] {
    if (!fused_ctas_per_sm || !grid_ctas_per_sm) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    int dev = 0;
    nebula::check(cudaGetDevice(&dev), "device");
    const nebula::LaunchLimits l = nebula::launchLimits(flip != 0, batch != 0);
    for (int i = 0; i < 2; ++i) {
      fused_ctas_per_sm[i] = l.fusedCtasPerSm[i];
      grid_ctas_per_sm[i] = l.gridCtasPerSm[i];
    }
  });
}
int nebula_mpm_export_brick_bins(nebula_mpm* e, uint32_t* numBricks, uint32_t* brickIds, uint32_t* brickStarts, uint32_t* sortedPids) {
  return guarded([&] {
    if (!numBricks || !brickIds || !brickStarts || (!sortedPids && E(e).liveCount())) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).exportBrickBins(numBricks, brickIds, brickStarts, sortedPids);
  });
}
int nebula_mpm_export_bins(nebula_mpm* e, uint32_t* cnt, uint32_t* off, uint32_t* srt) {
  return guarded([&] {
    if (!cnt || !off || (!srt && E(e).liveCount())) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).exportBins(cnt, off, srt);
  });
}
int nebula_mpm_export_grid(nebula_mpm* e, float dt, float* mom, float* mass) {
  return guarded([&] {
    if (!mom || !mass) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    E(e).exportGrid(dt, mom, mass);
  });
}

void nebula_mpm_domain_grid_res(const float domainSize[3], float cellSize, uint32_t out[3]) {
  nebula::domainGridRes(domainSize, cellSize, out);
}
uint32_t nebula_mpm_domain_cube_res(const uint32_t res[3]) { return nebula::domainCubeRes(res); }
uint32_t nebula_mpm_domain_hash_cells(const uint32_t res[3]) { return nebula::domainHashCells(res); }
uint32_t nebula_mpm_domain_n_groups(uint32_t cells) { return (cells + 255u) / 256u; }

}  // extern "C"
