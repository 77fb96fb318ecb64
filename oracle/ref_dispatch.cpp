// ref_dispatch.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's MPM compute shaders, compiled for the CPU by
// oracle/build_ref.py, the way MPMEngine drives them on the GPU: one storage
// buffer per attribute in a bindless table, the MPMSimPC push constants of
// MPMEngine::buildPC (src/engine/MPMEngine.cpp:355-396), and the passes of
// MPMEngine::step (src/engine/MPMEngine.cpp:404-474) in order:
//   zero grid, zero cells, hash count, scan local / global / add base, hash
//   sort, P2G, grid update, dense-SDF boundary, G2P.
// Each dispatch runs its invocations in index order (the per-invocation
// shaders whose invocations are independent may be spread over threads; the
// hash count and hash sort always run in order, so within a cell the sorted
// list is in ascending particle index).
//
// The PBF engine's spatial hash (hash_count.comp, hash_sort.comp) runs through
// ref_hash_bin with the same scan.
//
// Two passes are restated here rather than compiled, because they use
// workgroup shared memory and barriers: zero_cells.comp:11-15 (a fill) and the
// three hash-scan shaders (hash_scan_local.comp:12-43, hash_scan_global.comp:
// 14-34, hash_add_base.comp:12-22).  The restatement keeps their behaviour
// exactly, including the single 1024-invocation global scan: for more than
// 1024 groups (hashCells > 262,144) the groups from 1024 on keep their own
// inclusive total as their base, so the reference's offsets are not a prefix
// sum there.
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#include "glsl_env.hpp"

extern "C" {
void ref_run_mpm_zero_grid(const void*, uint32_t, int);
void ref_run_mpm_hash_count(const void*, uint32_t, int);
void ref_run_mpm_hash_sort(const void*, uint32_t, int);
void ref_run_mpm_p2g(const void*, uint32_t, int);
void ref_run_mpm_grid_update(const void*, uint32_t, int);
void ref_run_mpm_nanovdb_bc(const void*, uint32_t, int);
void ref_run_mpm_g2p(const void*, uint32_t, int);
void ref_run_hash_count(const void*, uint32_t, int);
void ref_run_hash_sort(const void*, uint32_t, int);
}

namespace {

// MPMSimPC (src/core/MPMSimPC.h), 188 bytes; the shaders' push-constant block.
struct SimPC {
  uint32_t posIdx, velIdx, F0Idx, F1Idx, typeFlagIdx, cellCountIdx, cellOffsetIdx, sortedIdxIdx, particleCount,
      hashCells, F2Idx, materialsIdx;
  float dt, cellSize;
  uint32_t forceBufIdx;
  float mu_lame;
  uint32_t gridRes[3];
  float lambda_lame;
  float worldMin[3];
  float particleVolume;
  float worldMax[3];
  float M_friction, q_cohesion, q_max, flip_ratio;
  uint32_t colliderIdx, colliderCount, B0Idx, B1Idx, B2Idx, nanoVDBIdx, gridMomIdx, gridMassIdx;
  float restitution, wall_friction;
  uint32_t plasticModel, materialCount;
  float rho0, p0_mcc, xi_hard;
  uint32_t forceCount;
};
static_assert(sizeof(SimPC) == 188, "MPMSimPC layout");
static_assert(offsetof(SimPC, gridRes) == 64 && offsetof(SimPC, worldMax) == 96 && offsetof(SimPC, forceCount) == 184,
              "MPMSimPC offsets");

// SimPC (common.glsl:11-65), 200 bytes: the PBF engine's push constants, of
// which the spatial hash reads the words set in hashPC() below.
struct HashPC {
  uint32_t w[50];
};

// hash_scan_local.comp:12-43, hash_scan_global.comp:14-34 and
// hash_add_base.comp:12-22 over `NC` cells: offset[0, NC) gets each cell's
// exclusive prefix inside its group of 256 plus the group's base, where the
// bases are the exclusive prefix of the first 1024 group totals and, for any
// later group, its own total (the single 1024-invocation global scan);
// offset[NC, NC + groups) holds the bases.
// With `intended`, every group's base is the exclusive prefix of all group
// totals: the plain exclusive scan the three passes mean to compute, which
// they give for up to 1024 groups.
void scanCells(const uint32_t* count, uint32_t* offset, uint32_t NC, bool intended = false) {
  const uint32_t NG = (NC + 255u) / 256u;
  for (uint32_t g = 0; g < NG; ++g) {
    uint32_t acc = 0;
    for (uint32_t l = 0; l < 256u; ++l) {
      const uint32_t gid = g * 256u + l;
      const uint32_t val = gid < NC ? count[gid] : 0u;
      if (gid < NC) offset[gid] = acc;
      acc += val;
    }
    offset[NC + g] = acc;
  }
  uint32_t acc = 0;
  for (uint32_t l = 0; l < NG && (intended || l < 1024u); ++l) {
    const uint32_t t = offset[NC + l];
    offset[NC + l] = acc;
    acc += t;
  }
  for (uint32_t c = 0; c < NC; ++c) offset[c] += offset[NC + c / 256u];
}

// Bindless slots (index 0 stays unbound: a 0 index means "none" to the shaders).
enum Slot : uint32_t {
  kPos = 1, kVel, kF0, kF1, kF2, kB0, kB1, kB2, kCellCount, kCellOffset, kSorted, kMaterials, kColliders, kForces,
  kSdf, kGridMom, kGridMass
};

}  // namespace

// The scene scalars; same layout as the CPU restatement's orc_params.
struct ref_params {
  float dt;
  float cellSize;
  uint32_t gridRes[3];
  uint32_t hashCells;
  float worldMin[3];
  float worldMax[3];
  float flip_ratio;
  uint32_t materialCount;
  float mu_lame, lambda_lame, rho0, M_friction, q_cohesion, q_max;
  uint32_t plasticModel;
  uint32_t colliderCount;
  uint32_t forceCount;
};

namespace {

struct RefScene {
  ref_params p{};
  uint32_t N = 0;
  int threads = 1;
  bool intendedScan = false;
  bool hasSdf = false;
  std::vector<uint32_t> attr[8];  // pos, vel, F0, F1, F2, B0, B1, B2: 4 words per particle
  std::vector<uint32_t> cellCount, cellOffset, sorted, materials, colliders, forces, sdf, gridMom, gridMass;

  uint32_t nGroups() const { return (p.hashCells + 255u) / 256u; }

  void bind() {
    for (int a = 0; a < 8; ++a) buffers[kPos + a].data = attr[a].data();
    buffers[kCellCount].data = cellCount.data();
    buffers[kCellOffset].data = cellOffset.data();
    buffers[kSorted].data = sorted.data();
    buffers[kMaterials].data = materials.data();
    buffers[kColliders].data = colliders.data();
    buffers[kForces].data = forces.data();
    buffers[kSdf].data = sdf.data();
    buffers[kGridMom].data = gridMom.data();
    buffers[kGridMass].data = gridMass.data();
  }

  // MPMEngine::buildPC (src/engine/MPMEngine.cpp:355-396) for this scene.
  SimPC pc() const {
    SimPC c{};
    c.posIdx = kPos;
    c.velIdx = kVel;
    c.F0Idx = kF0;
    c.F1Idx = kF1;
    c.F2Idx = kF2;
    c.typeFlagIdx = 0;
    c.cellCountIdx = kCellCount;
    c.cellOffsetIdx = kCellOffset;
    c.sortedIdxIdx = kSorted;
    c.particleCount = N;
    c.hashCells = p.hashCells;
    c.materialsIdx = p.materialCount ? kMaterials : 0u;
    c.dt = p.dt;
    c.cellSize = p.cellSize;
    std::memcpy(c.gridRes, p.gridRes, sizeof c.gridRes);
    std::memcpy(c.worldMin, p.worldMin, sizeof c.worldMin);
    std::memcpy(c.worldMax, p.worldMax, sizeof c.worldMax);
    c.forceBufIdx = kForces;
    c.mu_lame = p.mu_lame;
    c.lambda_lame = p.lambda_lame;
    c.M_friction = p.M_friction;
    c.q_cohesion = p.q_cohesion;
    c.q_max = p.q_max;
    c.flip_ratio = p.flip_ratio;
    c.colliderIdx = kColliders;
    c.colliderCount = p.colliderCount;
    c.B0Idx = kB0;
    c.B1Idx = kB1;
    c.B2Idx = kB2;
    c.nanoVDBIdx = hasSdf ? kSdf : 0u;
    c.gridMomIdx = kGridMom;
    c.gridMassIdx = kGridMass;
    c.plasticModel = p.plasticModel;
    c.materialCount = p.materialCount;
    c.rho0 = p.rho0;
    c.forceCount = p.forceCount;
    return c;
  }

  void resizeGrid() {
    const size_t NC = p.hashCells;
    gridMom.assign(NC * 8, 0u);
    gridMass.assign(NC, 0u);
    cellCount.assign(NC, 0u);
    cellOffset.assign(NC + nGroups(), 0u);
    sdf.resize(NC, 0u);
  }

  void zeroGrid() {
    bind();
    SimPC c = pc();
    ref_run_mpm_zero_grid(&c, p.hashCells, threads);
  }

  // zero cells, hash count, the three scan passes, hash sort
  // (src/engine/MPMEngine.cpp:423-456).
  void bin() {
    bind();
    SimPC c = pc();
    std::fill(cellCount.begin(), cellCount.end(), 0u);  // zero_cells.comp:11-15
    ref_run_mpm_hash_count(&c, N, 1);
    scanCells(cellCount.data(), cellOffset.data(), p.hashCells, intendedScan);
    ref_run_mpm_hash_sort(&c, N, 1);
  }

  void p2g() {
    bind();
    SimPC c = pc();
    ref_run_mpm_p2g(&c, p.hashCells, threads);
  }
  void gridUpdate() {
    bind();
    SimPC c = pc();
    ref_run_mpm_grid_update(&c, p.hashCells, threads);
  }
  void sdfBC() {
    bind();
    SimPC c = pc();
    ref_run_mpm_nanovdb_bc(&c, p.hashCells, threads);
  }
  void g2p() {
    bind();
    SimPC c = pc();
    ref_run_mpm_g2p(&c, N, threads);
  }
  void substep() {
    zeroGrid();
    bin();
    p2g();
    gridUpdate();
    sdfBC();
    g2p();
  }
};

}  // namespace

extern "C" {

void* ref_create(void) { return new RefScene(); }
void ref_destroy(void* h) { delete static_cast<RefScene*>(h); }
void ref_set_threads(void* h, int n) { static_cast<RefScene*>(h)->threads = n > 0 ? n : 1; }
// 1: the scan passes give the plain exclusive prefix over any number of
// groups (their intended result; the MPM binning of the oracle and of the
// CUDA path); 0 (default): exactly the reference's single 1024-wide global scan.
void ref_set_intended_scan(void* h, int on) { static_cast<RefScene*>(h)->intendedScan = on != 0; }

void ref_set_params(void* h, const ref_params* p) {
  RefScene& s = *static_cast<RefScene*>(h);
  const bool regrid = p->hashCells != s.p.hashCells || s.gridMass.size() != p->hashCells;
  s.p = *p;
  if (regrid) s.resizeGrid();
}

void ref_set_tables(void* h, const void* mats, uint32_t nm, const void* cols, uint32_t nc, const void* forces,
                    uint32_t nf) {
  RefScene& s = *static_cast<RefScene*>(h);
  s.materials.assign(size_t(nm) * 16 + 16, 0u);
  if (nm) std::memcpy(s.materials.data(), mats, size_t(nm) * 64);
  s.colliders.assign(size_t(nc) * 16 + 16, 0u);
  if (nc) std::memcpy(s.colliders.data(), cols, size_t(nc) * 64);
  s.forces.assign(size_t(nf) * 8 + 8, 0u);
  if (nf) std::memcpy(s.forces.data(), forces, size_t(nf) * 32);
}

// Morton-ordered dense SDF (hashCells floats), or null for none.
void ref_set_sdf(void* h, const float* sdf) {
  RefScene& s = *static_cast<RefScene*>(h);
  s.hasSdf = sdf != nullptr;
  s.sdf.assign(s.p.hashCells, 0u);
  if (sdf) std::memcpy(s.sdf.data(), sdf, size_t(s.p.hashCells) * 4);
}

// Eight float4 arrays of n particles each: pos, vel (w = material id bits),
// F0, F1, F2, B0, B1, B2 (w lanes = the packed stress).
void ref_set_state(void* h, const float* const* arrays, uint32_t n) {
  RefScene& s = *static_cast<RefScene*>(h);
  s.N = n;
  for (int a = 0; a < 8; ++a) {
    s.attr[a].assign(size_t(n) * 4 + 4, 0u);
    std::memcpy(s.attr[a].data(), arrays[a], size_t(n) * 16);
  }
  // With more than 1024 scan groups the reference's offsets are not a prefix
  // sum and the hash sort's slots reach up to twice the particle count (a
  // cell's base is at most its group's total, its slots at most twice that):
  // the list is sized so those writes stay inside it.
  s.sorted.assign(size_t(n) * 2 + 1, 0u);
}
void ref_get_state(void* h, float* const* arrays) {
  RefScene& s = *static_cast<RefScene*>(h);
  for (int a = 0; a < 8; ++a) std::memcpy(arrays[a], s.attr[a].data(), size_t(s.N) * 16);
}

// gridMom: 2 * hashCells float4 (second half: pre-force velocities for FLIP);
// gridMass: hashCells floats.
void ref_set_grid(void* h, const float* mom, const float* mass) {
  RefScene& s = *static_cast<RefScene*>(h);
  std::memcpy(s.gridMom.data(), mom, s.gridMom.size() * 4);
  std::memcpy(s.gridMass.data(), mass, s.gridMass.size() * 4);
}
void ref_get_grid(void* h, float* mom, float* mass) {
  RefScene& s = *static_cast<RefScene*>(h);
  std::memcpy(mom, s.gridMom.data(), s.gridMom.size() * 4);
  std::memcpy(mass, s.gridMass.data(), s.gridMass.size() * 4);
}

// cellCount (hashCells), cellOffset (hashCells: after the sort each holds its
// cell's end), sortedIdx (n).
void ref_set_bins(void* h, const uint32_t* cnt, const uint32_t* off, const uint32_t* sorted) {
  RefScene& s = *static_cast<RefScene*>(h);
  std::memcpy(s.cellCount.data(), cnt, size_t(s.p.hashCells) * 4);
  std::memcpy(s.cellOffset.data(), off, size_t(s.p.hashCells) * 4);
  std::memcpy(s.sorted.data(), sorted, size_t(s.N) * 4);
}
void ref_get_bins(void* h, uint32_t* cnt, uint32_t* off, uint32_t* sorted) {
  RefScene& s = *static_cast<RefScene*>(h);
  std::memcpy(cnt, s.cellCount.data(), size_t(s.p.hashCells) * 4);
  std::memcpy(off, s.cellOffset.data(), size_t(s.p.hashCells) * 4);
  std::memcpy(sorted, s.sorted.data(), size_t(s.N) * 4);
}

void ref_zero_grid(void* h) { static_cast<RefScene*>(h)->zeroGrid(); }
void ref_bin(void* h) { static_cast<RefScene*>(h)->bin(); }
void ref_p2g(void* h) { static_cast<RefScene*>(h)->p2g(); }
void ref_grid_update(void* h) { static_cast<RefScene*>(h)->gridUpdate(); }
void ref_sdf_bc(void* h) { static_cast<RefScene*>(h)->sdfBC(); }
void ref_g2p(void* h) { static_cast<RefScene*>(h)->g2p(); }
void ref_substep(void* h) { static_cast<RefScene*>(h)->substep(); }
void ref_run(void* h, uint32_t nsub) {
  for (uint32_t i = 0; i < nsub; ++i) static_cast<RefScene*>(h)->substep();
}

// The PBF engine's spatial hash over predicted positions (n float4; typeFlag
// n words or null for all 0): zero cells, hash_count.comp, the three scan
// passes, hash_sort.comp.  cellCount / cellOffset get hashCells words
// (offsets: range ends, as the sort leaves them); sortedIdx comes in with the
// caller's fill and gets the sorted list in its first n words.
void ref_hash_bin(const float* predP4, const uint32_t* typeFlag, uint32_t n, const float* worldMin, float cellSize,
                  const uint32_t* gridRes, uint32_t hashCells, uint32_t* cellCount, uint32_t* cellOffset,
                  uint32_t* sortedIdx) {
  const uint32_t NG = (hashCells + 255u) / 256u;
  std::vector<uint32_t> pred(size_t(n) * 4 + 4, 0u), flags(size_t(n) + 1, 0u), cnt(size_t(hashCells) + 1, 0u),
      off(size_t(hashCells) + NG + 1, 0u), srt(size_t(n) * 2 + 1, 0u);
  std::memcpy(pred.data(), predP4, size_t(n) * 16);
  if (typeFlag) std::memcpy(flags.data(), typeFlag, size_t(n) * 4);
  std::memcpy(srt.data(), sortedIdx, size_t(n) * 4);
  enum : uint32_t { kPred = 1, kFlags, kCount, kOffset, kSortedIdx };
  buffers[kPred].data = pred.data();
  buffers[kFlags].data = flags.data();
  buffers[kCount].data = cnt.data();
  buffers[kOffset].data = off.data();
  buffers[kSortedIdx].data = srt.data();
  HashPC c{};
  c.w[2] = kPred;        // predPIdx
  c.w[4] = kFlags;       // typeFlagIdx
  c.w[5] = kCount;       // cellCountIdx
  c.w[6] = kOffset;      // cellOffsetIdx
  c.w[7] = kSortedIdx;   // sortedIdxIdx
  c.w[8] = n;            // particleCount
  c.w[9] = hashCells;    // hashCells
  std::memcpy(&c.w[13], &cellSize, 4);
  std::memcpy(&c.w[16], gridRes, 12);
  std::memcpy(&c.w[20], worldMin, 12);
  ref_run_hash_count(&c, n, 1);
  scanCells(cnt.data(), off.data(), hashCells);
  ref_run_hash_sort(&c, n, 1);
  std::memcpy(cellCount, cnt.data(), size_t(hashCells) * 4);
  std::memcpy(cellOffset, off.data(), size_t(hashCells) * 4);
  std::memcpy(sortedIdx, srt.data(), size_t(n) * 4);
}

}  // extern "C"
