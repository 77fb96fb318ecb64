// mpm_batch.cu -- BatchEngine: many scenes, one set of launches per substep.
//
// Scene s owns bricks [brickBase_s, brickBase_s + nb_s) of one shared brick
// space and particle slots [partBase_s, partBase_s + n_s) of one particle
// array.  Because the brick sort is scene-major, the slot range of a scene is
// the same in every brick-ordered buffer, so the batched kernels find a
// particle's scene from its slot and an item's scene from its brick (binary
// search over the base tables) and read that scene's SubstepParams from a
// device table.  Per-substep physics is exactly the single-scene engine's.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "mpm_batch.h"

namespace nebula {

namespace {
constexpr uint32_t kMaxBatchScenes = 65536;
constexpr uint32_t kMaxBatchBricks = 1u << 26;  // 64 * bricks must fit a u32 cell code
inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
}  // namespace

BatchEngine::BatchEngine(const nebula_mpm_batch_config& cfg) : cfg_(cfg) {
  if (cfg.maxScenes == 0 || cfg.maxScenes > kMaxBatchScenes) throw Error(NEBULA_MPM_ERR_INVALID, "maxScenes must be in [1, 65536]");
  check(cudaGetDevice(&device_), "cudaGetDevice");
  check(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");
  const size_t capN = size_t(std::max(cfg.maxParticles, 1u));
  for (int k = 0; k < 8; ++k) {
    state_[k].alloc(capN * sizeof(float4));
    stateB_[k].alloc(capN * sizeof(float4));
  }
  for (auto& p : pid_) p.alloc(capN * sizeof(uint32_t));
  err_.alloc(sizeof(uint32_t));
  check(cudaMemset(err_.ptr, 0, sizeof(uint32_t)), "cudaMemset");
  uint64_t l = 0;
  check(launchIota(static_cast<uint32_t*>(pid_[0].ptr), uint32_t(capN), nullptr, &l), "iota");
  check(cudaEventCreateWithFlags(&stagingFree_, cudaEventDisableTiming), "cudaEventCreate");
}

BatchEngine::~BatchEngine() {
  if (lastStream_) cudaStreamSynchronize(lastStream_);
  else cudaDeviceSynchronize();
  clearGraphs();
  if (stagingFree_) cudaEventDestroy(stagingFree_);
  if (staging_) cudaFreeHost(staging_);
}

void BatchEngine::bindDevice() const { check(cudaSetDevice(device_), "cudaSetDevice"); }

void BatchEngine::quiesce() {
  if (lastStream_) check(cudaStreamSynchronize(lastStream_), "cudaStreamSynchronize");
  else check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
}

BatchEngine::Scene& BatchEngine::scene(uint32_t s) {
  if (s >= scenes_.size()) throw Error(NEBULA_MPM_ERR_INVALID, "scene index out of range");
  return scenes_[s];
}
const BatchEngine::Scene& BatchEngine::scene(uint32_t s) const {
  if (s >= scenes_.size()) throw Error(NEBULA_MPM_ERR_INVALID, "scene index out of range");
  return scenes_[s];
}

void BatchEngine::clearGraphs() {
  for (auto& g : graphs_) cudaGraphExecDestroy(g.second);
  graphs_.clear();
}

bool BatchEngine::anyFlip() const {
  for (const Scene& sc : scenes_)
    if (sc.params.flip_ratio > 0.01f) return true;
  return false;
}

// ------------------------------------------------------------------ scenes
uint32_t BatchEngine::addScene(const nebula_mpm_config& cfg, const float* pos4, const float* vel4, uint32_t n) {
  bindDevice();
  if (sealed_) throw Error(NEBULA_MPM_ERR_INVALID, "scenes are added before the first step of a batch");
  if (scenes_.size() >= cfg_.maxScenes) throw Error(NEBULA_MPM_ERR_INVALID, "scene table full (maxScenes)");
  if (!(cfg.cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  for (int a = 0; a < 3; ++a)
    if (!(cfg.domainSize[a] >= 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "domainSize must be >= 0");
  if (uint64_t(live_) + n > std::max(cfg_.maxParticles, 0u)) throw Error(NEBULA_MPM_ERR_INVALID, "batch particle capacity exceeded");
  if (n && (!pos4 || !vel4)) throw Error(NEBULA_MPM_ERR_INVALID, "null particle arrays");
  Scene sc;
  sc.cfg = cfg;
  sc.params = nebula_mpm_params{0.3f, 0.0f, 20, 0u, 1e5f, 0.577f, 0.0f, 0.0f};  // MPMEngine.h:72-80
  domainGridRes(cfg.domainSize, cfg.cellSize, sc.gridRes);
  sc.cubeRes = domainCubeRes(sc.gridRes);
  if (sc.cubeRes > 1024u) throw Error(NEBULA_MPM_ERR_INVALID, "grid resolution above 1024 per axis (10-bit Morton code)");
  sc.hashCells = sc.cubeRes * sc.cubeRes * sc.cubeRes;
  sc.nb = std::max(sc.hashCells / 64u, 1u);
  if (uint64_t(nbTotal_) + sc.nb > kMaxBatchBricks) throw Error(NEBULA_MPM_ERR_INVALID, "batch grid exceeds 2^26 bricks");
  sc.brickBase = nbTotal_;
  sc.partBase = live_;
  sc.n = n;
  // presetJelly(E, nu, rho0) with the public DP/VM defaults (MPMEngine.cpp:67-78)
  Material m{};
  m.mu = cfg.E / (2.0f * (1.0f + cfg.nu));
  m.lambda = cfg.E * cfg.nu / ((1.0f + cfg.nu) * (1.0f - 2.0f * cfg.nu));
  m.rho0 = cfg.rho0;
  m.model = MAT_ELASTIC;
  m.M_friction = sc.params.M_friction;
  m.q_cohesion = sc.params.q_cohesion;
  m.q_max = sc.params.q_max;
  sc.materials.assign(1, m);
  if (n) {
    std::vector<float4> F0(n, make_float4(1, 0, 0, 0)), F1(n, make_float4(0, 1, 0, 0)), F2(n, make_float4(0, 0, 1, 0)), Z(n, make_float4(0, 0, 0, 0));
    StatePtrs st = statePtrs(cur_);
    const size_t bytes = size_t(n) * sizeof(float4);
    const void* src[8] = {pos4, vel4, F0.data(), F1.data(), F2.data(), Z.data(), Z.data(), Z.data()};
    for (int k = 0; k < 8; ++k) check(cudaMemcpy(st.f[k] + live_, src[k], bytes, cudaMemcpyHostToDevice), "upload scene particles");
  }
  live_ += n;
  nbTotal_ += sc.nb;
  scenes_.push_back(std::move(sc));
  tablesDirty_ = true;
  return uint32_t(scenes_.size() - 1);
}

void BatchEngine::setParams(uint32_t s, const nebula_mpm_params& p) {
  Scene& sc = scene(s);
  bindDevice();
  discardPending(lastStream_);  // APIC mode and stress scaling enter the pending P2G
  const bool hadFlip = anyFlip();
  sc.params = p;
  if (sealed_ && anyFlip() != hadFlip) clearGraphs();
  tablesDirty_ = true;
}

void BatchEngine::getParams(uint32_t s, nebula_mpm_params* p) const { *p = scene(s).params; }

// The material-model set of every scene's table together (the fused kernel's instantiation).
int BatchEngine::modelSet() const {
  std::vector<Material> all;
  for (const Scene& sc : scenes_) all.insert(all.end(), sc.materials.begin(), sc.materials.end());
  return modelSetOf(all.data(), uint32_t(all.size()));
}

void BatchEngine::setMaterials(uint32_t s, const nebula_mpm_material* mats, uint32_t n) {
  Scene& sc = scene(s);
  if (n == 0) return;  // MPMEngine.cpp:240
  if (n > uint32_t(kMaxMaterials)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 16 materials");
  if (!mats) throw Error(NEBULA_MPM_ERR_INVALID, "null materials");
  bindDevice();
  discardPending(lastStream_);  // rho0 enters P2G
  sc.materials.assign(reinterpret_cast<const Material*>(mats), reinterpret_cast<const Material*>(mats) + n);
  tablesDirty_ = true;
}

void BatchEngine::setColliders(uint32_t s, const nebula_mpm_collider* c, uint32_t n) {
  if (n > uint32_t(kMaxColliders)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 64 colliders");
  if (n && !c) throw Error(NEBULA_MPM_ERR_INVALID, "null colliders");
  Scene& sc = scene(s);
  sc.track.assign(reinterpret_cast<const Collider*>(c), reinterpret_cast<const Collider*>(c) + n);
  sc.colliderCount = n;
  sc.trackLen = 1;
  tablesDirty_ = true;
}

void BatchEngine::setColliderTrack(uint32_t s, const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps) {
  if (perSubstep > uint32_t(kMaxColliders)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 64 colliders per substep");
  if (substeps == 0) throw Error(NEBULA_MPM_ERR_INVALID, "a collider track needs at least one substep");
  const size_t total = size_t(perSubstep) * substeps;
  if (total && !c) throw Error(NEBULA_MPM_ERR_INVALID, "null colliders");
  Scene& sc = scene(s);
  sc.track.assign(reinterpret_cast<const Collider*>(c), reinterpret_cast<const Collider*>(c) + total);
  sc.colliderCount = perSubstep;
  sc.trackLen = substeps;
  tablesDirty_ = true;
}

void BatchEngine::setColliderSDF(uint32_t s, const float* sdf, uint64_t n) {
  Scene& sc = scene(s);
  if (!sdf || n != sc.hashCells) throw Error(NEBULA_MPM_ERR_INVALID, "SDF must hold the scene's hashCells floats");
  bindDevice();
  quiesce();  // a running step may read the old values
  sc.sdf.ensure(size_t(sc.hashCells) * sizeof(float));
  check(cudaMemcpy(sc.sdf.ptr, sdf, size_t(sc.hashCells) * sizeof(float), cudaMemcpyHostToDevice), "upload sdf");
  sc.hasSdf = true;
  tablesDirty_ = true;
}

void BatchEngine::clearColliderSDF(uint32_t s) {
  scene(s).hasSdf = false;
  tablesDirty_ = true;
}

void BatchEngine::setForces(uint32_t s, const nebula_mpm_force* f, uint32_t n) {
  if (n > uint32_t(kMaxForces)) throw Error(NEBULA_MPM_ERR_INVALID, "at most 16 forces");
  if (n && !f) throw Error(NEBULA_MPM_ERR_INVALID, "null forces");
  for (uint32_t i = 0; i < n; ++i)
    if (f[i].type != FORCE_GRAVITY && f[i].type != FORCE_CONSTANT_WIND)
      throw Error(NEBULA_MPM_ERR_UNSUPPORTED, "only GRAVITY and CONSTANT_WIND forces act on the MPM grid in this build");
  Scene& sc = scene(s);
  sc.forces.assign(reinterpret_cast<const Force*>(f), reinterpret_cast<const Force*>(f) + n);
  tablesDirty_ = true;
}

// ------------------------------------------------------------------ particles
StatePtrs BatchEngine::statePtrs(int buf) {
  StatePtrs s;
  for (int k = 0; k < 8; ++k) s.f[k] = static_cast<float4*>(buf == 0 ? state_[k].ptr : stateB_[k].ptr);
  return s;
}

void BatchEngine::normalizeOrder(cudaStream_t st) {
  if (!permuted_) return;
  check(launchUnpermute(statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), statePtrs(cur_ ^ 1), live_, st, &launches_), "unpermute");
  cur_ ^= 1;
  check(launchIota(static_cast<uint32_t*>(pid_[cur_].ptr), std::max(cfg_.maxParticles, 1u), st, &launches_), "iota");
  permuted_ = false;
  discardPending(st);  // the pending bins index the old order
}

void BatchEngine::discardPending(cudaStream_t st) {
  if (!pending_) return;
  check(launchClearBricks(brickBuffers(cur_), gridBuffers(), numSMs_, st, &launches_), "clear bricks");
  pending_ = false;
}

void BatchEngine::beforeHostEdit(bool particles) {
  bindDevice();
  if (particles) {
    normalizeOrder(lastStream_);
    discardPending(lastStream_);
  }
  quiesce();
}

void BatchEngine::setParticleMaterialIds(uint32_t s, const uint32_t* ids, uint32_t n) {
  Scene& sc = scene(s);
  if (n > sc.n) throw Error(NEBULA_MPM_ERR_INVALID, "more ids than scene particles");
  if (n && !ids) throw Error(NEBULA_MPM_ERR_INVALID, "null ids");
  beforeHostEdit(true);
  std::vector<float4> v(n);
  for (uint32_t i = 0; i < n; ++i) {
    float w;
    std::memcpy(&w, ids + i, 4);
    v[i] = make_float4(0.f, 0.f, 0.f, w);
  }
  if (n) check(cudaMemcpy(statePtrs(cur_).f[1] + sc.partBase, v.data(), n * sizeof(float4), cudaMemcpyHostToDevice), "upload ids");
}

void BatchEngine::uploadState(uint32_t s, const float* const f[8], uint32_t n) {
  Scene& sc = scene(s);
  if (n != sc.n) throw Error(NEBULA_MPM_ERR_INVALID, "upload_state must replace all of the scene's particles");
  for (int k = 0; k < 8; ++k)
    if (n && !f[k]) throw Error(NEBULA_MPM_ERR_INVALID, "null field");
  beforeHostEdit(true);
  StatePtrs st = statePtrs(cur_);
  for (int k = 0; k < 8; ++k)
    if (n) check(cudaMemcpy(st.f[k] + sc.partBase, f[k], size_t(n) * sizeof(float4), cudaMemcpyHostToDevice), "upload state");
}

void BatchEngine::download(uint32_t s, int field, float* host, uint64_t count) {
  const Scene& sc = scene(s);
  if (field < 0 || field > 7) throw Error(NEBULA_MPM_ERR_INVALID, "field index out of range");
  if (count != uint64_t(sc.n) * 4) throw Error(NEBULA_MPM_ERR_INVALID, "count must be 4 * scene particles");
  if (count && !host) throw Error(NEBULA_MPM_ERR_INVALID, "null host buffer");
  bindDevice();
  const float4* src = statePtrs(cur_).f[field];
  if (permuted_ && live_) {
    StatePtrs tmp = statePtrs(cur_ ^ 1);  // idle between substeps
    check(launchUnpermute(statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), tmp, live_, lastStream_, &launches_), "unpermute");
    src = tmp.f[field];
  }
  quiesce();
  if (count) check(cudaMemcpy(host, src + sc.partBase, count * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

// ------------------------------------------------------------------ layout
void BatchEngine::seal() {
  if (sealed_) return;
  if (scenes_.empty()) throw Error(NEBULA_MPM_ERR_INVALID, "batch has no scenes");
  const size_t cells = size_t(nbTotal_) * 64u;
  gridAcc_.alloc(cells * sizeof(float4));
  gridVel_.alloc(cells * sizeof(float4));
  check(cudaMemset(gridAcc_.ptr, 0, gridAcc_.bytes), "cudaMemset");
  check(cudaMemset(gridVel_.ptr, 0, gridVel_.bytes), "cudaMemset");
  tiles_ = (nbTotal_ + kBrickScanTile - 1) / kBrickScanTile;
  for (DevBuf* b : {&bCount_, &bFlag_, &bStart_, &pbBrick_, &gbBrick_}) {
    b->alloc(size_t(nbTotal_) * sizeof(uint32_t));
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  // per-cell counts of two binnings (each cleared by the fused kernel after the one that follows it)
  for (DevBuf* b : {&cCount_[0], &cCount_[1]}) {
    b->alloc(size_t(nbTotal_) * 64u * sizeof(uint32_t));
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  pbStart_.alloc(size_t(nbTotal_ + 1) * sizeof(uint32_t));
  counters_.alloc(kCntSlots * sizeof(uint32_t));
  scanState_.alloc(size_t(3) * tiles_ * sizeof(unsigned long long));
  scanTile_.alloc(sizeof(unsigned long long));
  for (DevBuf* b : {&pbStart_, &counters_, &scanState_, &scanTile_}) check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  const size_t capN = size_t(std::max(cfg_.maxParticles, 1u)) * sizeof(uint32_t);
  for (DevBuf* b : {&binKey_, &binRank_, &perm_}) {
    b->alloc(capN);
    check(cudaMemset(b->ptr, 0, b->bytes), "cudaMemset");
  }
  const size_t S = scenes_.size();
  tParams_.alloc(S * sizeof(SubstepParams));
  tBrickBase_.alloc((S + 1) * sizeof(uint32_t));
  tPartBase_.alloc((S + 1) * sizeof(uint32_t));
  tMaterials_.alloc(S * kMaxMaterials * sizeof(Material));
  tForces_.alloc(S * kMaxForces * sizeof(Force));
  prepareBrickKernels(numSMs_);
  sealed_ = true;
  tablesDirty_ = true;
}

// q: the buffer whose state the binning describes (its counts are array q).
BrickBuffers BatchEngine::brickBuffers(int q) {
  BrickBuffers b;
  b.nb = nbTotal_;
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

GridBuffers BatchEngine::gridBuffers() {
  GridBuffers g;
  g.acc = static_cast<float4*>(gridAcc_.ptr);
  g.vel = static_cast<float4*>(gridVel_.ptr);
  g.vold = nullptr;
  if (anyFlip()) {
    if (!gridVold_.ptr) {
      gridVold_.alloc(size_t(nbTotal_) * 64u * sizeof(float4));
      check(cudaMemset(gridVold_.ptr, 0, gridVold_.bytes), "cudaMemset");
    }
    g.vold = static_cast<float4*>(gridVold_.ptr);
  }
  return g;
}

SceneTable BatchEngine::table() const {
  SceneTable T;
  T.params = static_cast<const SubstepParams*>(tParams_.ptr);
  T.brickBase = static_cast<const uint32_t*>(tBrickBase_.ptr);
  T.partBase = static_cast<const uint32_t*>(tPartBase_.ptr);
  T.count = uint32_t(scenes_.size());
  return T;
}

// Device tables for a step of `substeps` substeps of length subDt: per-scene
// SubstepParams, base tables, materials, forces, and every scene's collider
// track expanded to one set per substep.  Uploaded on the stream from pinned
// staging (reused once the previous upload's copies finished).
void BatchEngine::uploadTables(float subDt, uint32_t substeps, cudaStream_t st) {
  if (!tablesDirty_ && tableDt_ == subDt && tableSubsteps_ == substeps) return;
  const size_t S = scenes_.size();
  size_t trackTotal = 0;
  for (const Scene& sc : scenes_) trackTotal += size_t(sc.colliderCount) * substeps;
  const size_t trackBytes = std::max<size_t>(trackTotal, 1) * sizeof(Collider);
  if (tTrack_.bytes < trackBytes) {
    quiesce();  // kernels of an earlier step may still read the old track
    tTrack_.alloc(trackBytes);
  }
  const size_t oParams = 0;
  const size_t oBB = al256(oParams + S * sizeof(SubstepParams));
  const size_t oPB = al256(oBB + (S + 1) * 4);
  const size_t oMat = al256(oPB + (S + 1) * 4);
  const size_t oFor = al256(oMat + S * kMaxMaterials * sizeof(Material));
  const size_t oTrk = al256(oFor + S * kMaxForces * sizeof(Force));
  const size_t total = al256(oTrk + trackBytes);
  check(cudaEventSynchronize(stagingFree_), "cudaEventSynchronize");
  if (stagingBytes_ < total) {
    if (staging_) check(cudaFreeHost(staging_), "cudaFreeHost");
    staging_ = nullptr;
    check(cudaHostAlloc(&staging_, total, cudaHostAllocDefault), "cudaHostAlloc");
    stagingBytes_ = total;
  }
  char* h = static_cast<char*>(staging_);
  std::memset(h, 0, total);
  SubstepParams* P = reinterpret_cast<SubstepParams*>(h + oParams);
  uint32_t* bb = reinterpret_cast<uint32_t*>(h + oBB);
  uint32_t* pb = reinterpret_cast<uint32_t*>(h + oPB);
  Material* mats = reinterpret_cast<Material*>(h + oMat);
  Force* forces = reinterpret_cast<Force*>(h + oFor);
  Collider* trk = reinterpret_cast<Collider*>(h + oTrk);
  const Material* dMat = static_cast<const Material*>(tMaterials_.ptr);
  const Force* dFor = static_cast<const Force*>(tForces_.ptr);
  const Collider* dTrk = static_cast<const Collider*>(tTrack_.ptr);
  size_t trkOff = 0;
  for (size_t s = 0; s < S; ++s) {
    const Scene& sc = scenes_[s];
    SubstepParams& p = P[s];
    p.dt = subDt;
    p.cellSize = sc.cfg.cellSize;
    for (int a = 0; a < 3; ++a) {
      p.gridRes[a] = int(sc.gridRes[a]);
      p.worldMin[a] = 0.0f;
      p.worldMax[a] = sc.cfg.domainSize[a];
    }
    p.cubeRes = sc.cubeRes;
    p.hashCells = sc.hashCells;
    p.flip_ratio = sc.params.flip_ratio;
    p.materialCount = uint32_t(sc.materials.size());
    p.colliderCount = sc.colliderCount;
    p.forceCount = uint32_t(sc.forces.size());
    p.mu_lame = sc.cfg.E / (2.0f * (1.0f + sc.cfg.nu));
    p.lambda_lame = sc.cfg.E * sc.cfg.nu / ((1.0f + sc.cfg.nu) * (1.0f - 2.0f * sc.cfg.nu));
    p.rho0 = sc.cfg.rho0;
    p.M_friction = sc.params.M_friction;
    p.q_cohesion = sc.params.q_cohesion;
    p.q_max = sc.params.q_max;
    p.plasticModel = sc.params.plasticModel;
    p.materials = dMat + s * kMaxMaterials;
    p.forces = dFor + s * kMaxForces;
    p.colliders = dTrk + trkOff;
    p.sdf = sc.hasSdf ? static_cast<const float*>(sc.sdf.ptr) : nullptr;
    bb[s] = sc.brickBase;
    pb[s] = sc.partBase;
    std::copy(sc.materials.begin(), sc.materials.end(), mats + s * kMaxMaterials);
    std::copy(sc.forces.begin(), sc.forces.end(), forces + s * kMaxForces);
    for (uint32_t k = 0; k < substeps && sc.colliderCount; ++k) {
      const size_t set = std::min(k, sc.trackLen - 1);
      std::copy(sc.track.begin() + set * sc.colliderCount, sc.track.begin() + (set + 1) * sc.colliderCount, trk + trkOff);
      trkOff += sc.colliderCount;
    }
  }
  bb[S] = nbTotal_;
  pb[S] = live_;
  auto up = [&](void* dst, size_t off, size_t bytes) {
    if (bytes) check(cudaMemcpyAsync(dst, h + off, bytes, cudaMemcpyHostToDevice, st), "upload batch tables");
  };
  up(tParams_.ptr, oParams, S * sizeof(SubstepParams));
  up(tBrickBase_.ptr, oBB, (S + 1) * 4);
  up(tPartBase_.ptr, oPB, (S + 1) * 4);
  up(tMaterials_.ptr, oMat, S * kMaxMaterials * sizeof(Material));
  up(tForces_.ptr, oFor, S * kMaxForces * sizeof(Force));
  up(tTrack_.ptr, oTrk, trackTotal * sizeof(Collider));
  check(cudaEventRecord(stagingFree_, st), "cudaEventRecord");
  tablesDirty_ = false;
  tableDt_ = subDt;
  tableSubsteps_ = substeps;
}

// ------------------------------------------------------------------ substeps
void BatchEngine::buildPending(cudaStream_t st) {
  const SceneTable T = table();
  BrickBuffers B = brickBuffers(cur_);
  GridBuffers G = gridBuffers();
  uint32_t* err = static_cast<uint32_t*>(err_.ptr);
  // a binning from scratch: neither count array may hold an earlier binning's counts
  for (DevBuf& c : cCount_) check(cudaMemsetAsync(c.ptr, 0, c.bytes, st), "clear cell counts");
  check(launchBrickCountBatch(T, statePtrs(cur_).f[0], live_, B, st, &launches_), "brick count");
  check(launchBrickScan(B, err, st, &launches_), "brick scan");
  check(launchPermScatter(B, live_, err, st, &launches_), "perm scatter");
  check(launchP2GBricksBatch(T, statePtrs(cur_), live_, B, G, numSMs_, st, &launches_), "p2g bricks");
  pending_ = true;
}

void BatchEngine::substep(uint32_t k, cudaStream_t st) {
  const SceneTable T = table();
  // the binning of the state read (buffer cur_) and of the state written
  const BrickBuffers B = brickBuffers(cur_), Bn = brickBuffers(cur_ ^ 1);
  GridBuffers G = gridBuffers();
  uint32_t* err = static_cast<uint32_t*>(err_.ptr);
  const bool fold = live_ < kFoldScatterMax;
  check(launchGridBricksBatch(T, k, B, G, fold ? live_ : 0u, err, launchCfg_, numSMs_, st, &launches_), "grid bricks");
  check(launchG2P2GBatch(T, modelSet(), G.vold != nullptr, statePtrs(cur_), static_cast<const uint32_t*>(pid_[cur_].ptr), statePtrs(cur_ ^ 1),
                         static_cast<uint32_t*>(pid_[cur_ ^ 1].ptr), live_, Bn, G, err, launchCfg_, numSMs_, st, &launches_),
        "g2p2g");
  check(launchBrickScan(Bn, err, st, &launches_), "brick scan");
  // the permutation of this binning: here, or by the next grid launch
  if (!fold) check(launchPermScatter(Bn, live_, err, st, &launches_), "perm scatter");
  cur_ ^= 1;
  permuted_ = true;
}

// Captured graphs hold the old shape: drop them (after the queued work).
void BatchEngine::setLaunchConfig(const LaunchConfig& c) {
  validateLaunchConfig(c);
  bindDevice();
  quiesce();
  clearGraphs();
  launchCfg_ = c;
}

void BatchEngine::setGraphs(bool on) {
  bindDevice();
  if (!on) {
    quiesce();
    clearGraphs();
  }
  useGraphs_ = on;
}

void BatchEngine::step(float dt, uint32_t substeps, cudaStream_t st) {
  bindDevice();
  if (!(dt >= 0.f) || !std::isfinite(dt)) throw Error(NEBULA_MPM_ERR_INVALID, "dt must be finite and >= 0");
  seal();
  if (st != lastStream_) {
    quiesce();  // work queued on the previous stream must finish first
    lastStream_ = st;
  }
  if (substeps == 0 || live_ == 0) return;
  const float subDt = dt / float(substeps);
  if (pending_ && pendingDt_ != subDt) discardPending(st);
  uploadTables(subDt, substeps, st);
  if (!pending_) buildPending(st);
  const bool flip = gridBuffers().vold != nullptr;
  if (useGraphs_ && st != nullptr) {
    const auto key = std::make_tuple(substeps, cur_, flip, modelSet());
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
      // capture: the launchers record their kernels into the graph, and the
      // host-side state (buffer parity, counters) advances as for one run
      cudaGraph_t graph = nullptr;
      check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      const int cur0 = cur_;
      const uint64_t l0 = launches_;
      try {
        for (uint32_t k = 0; k < substeps; ++k) substep(k, st);
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        cur_ = cur0;
        launches_ = l0;
        throw;
      }
      check(cudaStreamEndCapture(st, &graph), "cudaStreamEndCapture");
      cudaGraphExec_t exec = nullptr;
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      cur_ = cur0;
      launchesPerGraph_[key] = launches_ - l0;
      launches_ = l0;
      check(e, "cudaGraphInstantiate");
      it = graphs_.emplace(key, exec).first;
    }
    check(cudaGraphLaunch(it->second, st), "cudaGraphLaunch");
    ++graphLaunches_;
    launches_ += launchesPerGraph_[key];
    if (substeps & 1u) cur_ ^= 1;
    permuted_ = true;
  } else {
    for (uint32_t k = 0; k < substeps; ++k) substep(k, st);
  }
  substeps_ += substeps;
  pending_ = true;
  pendingDt_ = subDt;
}

uint32_t BatchEngine::syncAndCheck() {
  bindDevice();
  quiesce();
  uint32_t e = 0;
  check(cudaMemcpy(&e, err_.ptr, 4, cudaMemcpyDeviceToHost), "read error flags");
  errorFlags_ = e;
  return e;
}

void BatchEngine::stats(nebula_mpm_batch_stats* s) {
  bindDevice();
  std::memset(s, 0, sizeof(*s));
  if (sealed_) {
    quiesce();
    uint32_t cnt[kCntSlots];
    check(cudaMemcpy(cnt, counters_.ptr, sizeof(cnt), cudaMemcpyDeviceToHost), "download counters");
    particleBricks_ = cnt[kCntNumPB];
    activeBricks_ = cnt[kCntNumGB];
    overflow_ = cnt[kCntOverflow];
  }
  s->substeps = substeps_;
  s->scenes = uint32_t(scenes_.size());
  s->live_particles = live_;
  s->total_bricks = nbTotal_;
  s->active_bricks = activeBricks_;
  s->particle_bricks = particleBricks_;
  s->overflow_particles = overflow_;
  s->kernel_launches = launches_;
  s->graph_launches = graphLaunches_;
  s->error_flags = errorFlags_;
}

void BatchEngine::sceneInfo(uint32_t s, nebula_mpm_scene_info* out) const {
  const Scene& sc = scene(s);
  for (int a = 0; a < 3; ++a) out->grid_res[a] = sc.gridRes[a];
  out->cube_res = sc.cubeRes;
  out->hash_cells = sc.hashCells;
  out->particles = sc.n;
  out->first_brick = sc.brickBase;
  out->bricks = sc.nb;
}

}  // namespace nebula

// ====================================================================== C ABI
using nebula::Error;
using nebula::g_last_error;

struct nebula_mpm_batch {
  std::unique_ptr<nebula::BatchEngine> eng;
};

namespace {
template <class F> int guardedB(F&& f) {
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

nebula::BatchEngine& B(nebula_mpm_batch* b) {
  if (!b || !b->eng) throw Error(NEBULA_MPM_ERR_INVALID, "null batch");
  return *b->eng;
}
const nebula::BatchEngine& B(const nebula_mpm_batch* b) {
  if (!b || !b->eng) throw Error(NEBULA_MPM_ERR_INVALID, "null batch");
  return *b->eng;
}
}  // namespace

extern "C" {

int nebula_mpm_batch_create(const nebula_mpm_batch_config* cfg, nebula_mpm_batch** out) {
  return guardedB([&] {
    if (!cfg || !out) throw Error(NEBULA_MPM_ERR_INVALID, "null argument");
    *out = nullptr;
    auto h = std::make_unique<nebula_mpm_batch>();
    h->eng = std::make_unique<nebula::BatchEngine>(*cfg);
    *out = h.release();
  });
}
int nebula_mpm_batch_destroy(nebula_mpm_batch* b) {
  return guardedB([&] { delete b; });
}
int nebula_mpm_batch_add_scene(nebula_mpm_batch* b, const nebula_mpm_config* cfg, const float* pos4, const float* vel4, uint32_t n,
                               uint32_t* scene) {
  return guardedB([&] {
    if (!cfg) throw Error(NEBULA_MPM_ERR_INVALID, "null config");
    const uint32_t s = B(b).addScene(*cfg, pos4, vel4, n);
    if (scene) *scene = s;
  });
}
int nebula_mpm_batch_set_params(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_params* p) {
  return guardedB([&] {
    if (!p) throw Error(NEBULA_MPM_ERR_INVALID, "null params");
    B(b).setParams(scene, *p);
  });
}
int nebula_mpm_batch_get_params(const nebula_mpm_batch* b, uint32_t scene, nebula_mpm_params* p) {
  return guardedB([&] {
    if (!p) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    B(b).getParams(scene, p);
  });
}
int nebula_mpm_batch_set_materials(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_material* mats, uint32_t n) {
  return guardedB([&] { B(b).setMaterials(scene, mats, n); });
}
int nebula_mpm_batch_set_particle_material_ids(nebula_mpm_batch* b, uint32_t scene, const uint32_t* ids, uint32_t n) {
  return guardedB([&] { B(b).setParticleMaterialIds(scene, ids, n); });
}
int nebula_mpm_batch_set_colliders(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_collider* c, uint32_t n) {
  return guardedB([&] { B(b).setColliders(scene, c, n); });
}
int nebula_mpm_batch_set_collider_track(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_collider* c, uint32_t perSubstep,
                                        uint32_t substeps) {
  return guardedB([&] { B(b).setColliderTrack(scene, c, perSubstep, substeps); });
}
int nebula_mpm_batch_set_collider_sdf(nebula_mpm_batch* b, uint32_t scene, const float* sdf, uint64_t n) {
  return guardedB([&] { B(b).setColliderSDF(scene, sdf, n); });
}
int nebula_mpm_batch_clear_collider_sdf(nebula_mpm_batch* b, uint32_t scene) {
  return guardedB([&] { B(b).clearColliderSDF(scene); });
}
int nebula_mpm_batch_set_forces(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_force* f, uint32_t n) {
  return guardedB([&] { B(b).setForces(scene, f, n); });
}
int nebula_mpm_batch_upload_state(nebula_mpm_batch* b, uint32_t scene, const float* const fields[8], uint32_t n) {
  return guardedB([&] {
    if (!fields) throw Error(NEBULA_MPM_ERR_INVALID, "null fields");
    B(b).uploadState(scene, fields, n);
  });
}
int nebula_mpm_batch_download(nebula_mpm_batch* b, uint32_t scene, int field, float* host, uint64_t count) {
  return guardedB([&] { B(b).download(scene, field, host, count); });
}
int nebula_mpm_batch_step(nebula_mpm_batch* b, float dt, uint32_t substeps, void* stream) {
  return guardedB([&] { B(b).step(dt, substeps, static_cast<cudaStream_t>(stream)); });
}
int nebula_mpm_batch_set_graphs(nebula_mpm_batch* b, int enable) {
  return guardedB([&] { B(b).setGraphs(enable != 0); });
}
int nebula_mpm_batch_set_launch_config(nebula_mpm_batch* b, const nebula_mpm_launch_config* c) {
  return guardedB([&] {
    if (!c) throw Error(NEBULA_MPM_ERR_INVALID, "null launch config");
    B(b).setLaunchConfig(nebula::fromAbi(*c));
  });
}
int nebula_mpm_batch_get_launch_config(nebula_mpm_batch* b, nebula_mpm_launch_config* c) {
  return guardedB([&] {
    if (!c) throw Error(NEBULA_MPM_ERR_INVALID, "null launch config");
    *c = nebula::toAbi(B(b).launchConfig());
  });
}
int nebula_mpm_batch_sync(nebula_mpm_batch* b) {
  return guardedB([&] {
    const uint32_t f = B(b).syncAndCheck();
    if (f & ~nebula::kErrTileOverflow) {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "device error flags 0x%x (1: bounded wait expired, 2: non-finite particle state)", f);
      throw Error(NEBULA_MPM_ERR_DEVICE, buf);
    }
  });
}
int nebula_mpm_batch_get_stats(nebula_mpm_batch* b, nebula_mpm_batch_stats* s) {
  return guardedB([&] {
    if (!s) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    B(b).stats(s);
  });
}
int nebula_mpm_batch_scene_info(const nebula_mpm_batch* b, uint32_t scene, nebula_mpm_scene_info* info) {
  return guardedB([&] {
    if (!info) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    B(b).sceneInfo(scene, info);
  });
}

}  // extern "C"
