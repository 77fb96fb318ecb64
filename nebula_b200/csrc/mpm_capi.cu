// mpm_capi.cu -- single-pass entry points of include/nebula_mpm.h.
//
// Each call runs one reference dispatch on caller-owned device buffers in the
// reference layout, the per-pass surface of the reference's test harness
// (MPMHarness::runZeroGrid / runP2G / runGridUpdate / runG2P and
// buildHashGridCPU, tests/helpers/MPMHarness.cpp:132-178, 260-282), plus the
// PBF engine's spatial hash on the same counting sort (nebula_hash_bin).
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mpm_engine.h"
#include "mpm_internal.h"
#include "mpm_scan.cuh"

namespace nebula {
namespace {

SubstepParams fromPass(const nebula_mpm_pass& p, const nebula_mpm_material* mats, const nebula_mpm_collider* cols, const nebula_mpm_force* forces,
                       const float* sdf) {
  SubstepParams P{};
  P.dt = p.dt;
  P.cellSize = p.cellSize;
  for (int a = 0; a < 3; ++a) {
    P.gridRes[a] = int(p.gridRes[a]);
    P.worldMin[a] = p.worldMin[a];
    P.worldMax[a] = p.worldMax[a];
  }
  P.cubeRes = domainCubeRes(p.gridRes);
  P.hashCells = p.hashCells;
  P.flip_ratio = p.flip_ratio;
  P.materialCount = p.materialCount;
  P.colliderCount = p.colliderCount;
  P.forceCount = p.forceCount;
  P.mu_lame = p.mu_lame;
  P.lambda_lame = p.lambda_lame;
  P.rho0 = p.rho0;
  P.M_friction = p.M_friction;
  P.q_cohesion = p.q_cohesion;
  P.q_max = p.q_max;
  P.plasticModel = p.plasticModel;
  P.materials = reinterpret_cast<const Material*>(mats);
  P.colliders = reinterpret_cast<const Collider*>(cols);
  P.forces = reinterpret_cast<const Force*>(forces);
  P.sdf = sdf;
  return P;
}

void validate(const nebula_mpm_pass* p) {
  if (!p) throw Error(NEBULA_MPM_ERR_INVALID, "null pass parameters");
  if (!(p->cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  uint32_t c = domainCubeRes(p->gridRes);
  if (c > 1024u) throw Error(NEBULA_MPM_ERR_INVALID, "grid resolution above 1024 per axis");
  if (p->hashCells != c * c * c) throw Error(NEBULA_MPM_ERR_INVALID, "hashCells must equal cubeRes^3 of gridRes");
  if (p->materialCount > uint32_t(kMaxMaterials) || p->colliderCount > uint32_t(kMaxColliders) || p->forceCount > uint32_t(kMaxForces))
    throw Error(NEBULA_MPM_ERR_INVALID, "table size out of range");
}

StatePtrs statePtrs(const nebula_mpm_particles* parts) {
  if (!parts) throw Error(NEBULA_MPM_ERR_INVALID, "null particles");
  StatePtrs s;
  for (int k = 0; k < 8; ++k) {
    if (!parts->f[k]) throw Error(NEBULA_MPM_ERR_INVALID, "null particle field");
    s.f[k] = reinterpret_cast<float4*>(parts->f[k]);
  }
  return s;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct BinWorkspaceLayout {
  size_t cellStart, key, rank, sortedTmp, tiles, err, total;
};
BinWorkspaceLayout binLayout(uint32_t nc, uint32_t n) {
  BinWorkspaceLayout L;
  size_t o = 0;
  L.cellStart = o; o = align256(o + size_t(nc) * 4);
  L.key = o; o = align256(o + size_t(n) * 4);
  L.rank = o; o = align256(o + size_t(n) * 4);
  L.sortedTmp = o; o = align256(o + size_t(n) * 4);
  L.tiles = o; o = align256(o + scanWorkspaceBytes(nc));
  L.err = o; o = align256(o + 4);
  L.total = o;
  return L;
}

// The counting sort's buffers inside a caller workspace laid out by binLayout.
BinBuffers workspaceBins(const BinWorkspaceLayout& L, void* dWorkspace, uint32_t hashCells) {
  char* ws = static_cast<char*>(dWorkspace);
  BinBuffers b{};
  b.cellStart = reinterpret_cast<uint32_t*>(ws + L.cellStart);
  b.key = reinterpret_cast<uint32_t*>(ws + L.key);
  b.rank = reinterpret_cast<uint32_t*>(ws + L.rank);
  b.sortedTmp = reinterpret_cast<uint32_t*>(ws + L.sortedTmp);
  b.tileState = reinterpret_cast<unsigned long long*>(ws + L.tiles);
  b.tileCounter = reinterpret_cast<uint32_t*>(b.tileState + scanTiles(hashCells));
  b.err = reinterpret_cast<uint32_t*>(ws + L.err);
  return b;
}

}  // namespace

void throwBinErrors(uint32_t bits) {
  if (!bits) return;
  char buf[192];
  std::snprintf(buf, sizeof(buf), "binning error bits 0x%x (1: a scan look-back wait expired, 8: a binning index fell outside [0, n))", bits);
  throw Error(NEBULA_MPM_ERR_DEVICE, buf);
}

namespace {

template <class F> int guarded(F&& f) {
  try {
    f();
    return NEBULA_MPM_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return NEBULA_MPM_ERR_INVALID;
  }
}

}  // namespace
}  // namespace nebula

using namespace nebula;

extern "C" {

size_t nebula_mpm_bin_workspace_size(uint32_t hashCells, uint32_t particleCount) { return binLayout(hashCells, particleCount).total; }

int nebula_mpm_bin(const nebula_mpm_pass* pass, const float* dPos4, uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSorted,
                   void* dWorkspace, size_t workspaceBytes, void* stream) {
  return guarded([&] {
    validate(pass);
    const uint32_t n = pass->particleCount;
    BinWorkspaceLayout L = binLayout(pass->hashCells, n);
    if (!dWorkspace || workspaceBytes < L.total) throw Error(NEBULA_MPM_ERR_INVALID, "bin workspace too small");
    if (!dCellCount || !dCellOffset || (n && (!dPos4 || !dSorted))) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BinBuffers b = workspaceBins(L, dWorkspace, pass->hashCells);
    b.cellCount = dCellCount;
    b.cellEnd = dCellOffset;
    b.sorted = dSorted;
    check(cudaMemsetAsync(b.err, 0, 4, s), "memset");
    uint64_t launches = 0;
    SubstepParams P = fromPass(*pass, nullptr, nullptr, nullptr, nullptr);
    check(launchBin(P, reinterpret_cast<const float4*>(dPos4), n, b, s, &launches), "bin");
  });
}

int nebula_mpm_bin_status(const void* dWorkspace, size_t workspaceBytes, uint32_t hashCells, uint32_t particleCount, uint32_t* errorBits,
                          void* stream) {
  return guarded([&] {
    if (!errorBits) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *errorBits = 0;
    const BinWorkspaceLayout L = binLayout(hashCells, particleCount);
    if (!dWorkspace || workspaceBytes < L.total) throw Error(NEBULA_MPM_ERR_INVALID, "bin workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t bits = 0;
    check(cudaMemcpyAsync(&bits, static_cast<const char*>(dWorkspace) + L.err, sizeof(bits), cudaMemcpyDeviceToHost, s), "read error word");
    check(cudaStreamSynchronize(s), "stream synchronize");
    *errorBits = bits;
    throwBinErrors(bits);
  });
}

int nebula_mpm_bin_probe_wait_expiry(const nebula_mpm_pass* pass, const uint32_t* dCellCount, void* dWorkspace, size_t workspaceBytes,
                                     void* stream) {
  return guarded([&] {
    validate(pass);
    if (pass->hashCells < 2u * uint32_t(kScanTile)) throw Error(NEBULA_MPM_ERR_INVALID, "the probe needs hashCells >= 4096");
    const BinWorkspaceLayout L = binLayout(pass->hashCells, pass->particleCount);
    if (!dWorkspace || workspaceBytes < L.total) throw Error(NEBULA_MPM_ERR_INVALID, "bin workspace too small");
    if (!dCellCount) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");
    BinBuffers b = workspaceBins(L, dWorkspace, pass->hashCells);
    b.cellCount = const_cast<uint32_t*>(dCellCount);
    uint64_t launches = 0;
    SubstepParams P = fromPass(*pass, nullptr, nullptr, nullptr, nullptr);
    check(launchBinScanExpiryProbe(P, b, static_cast<cudaStream_t>(stream), &launches), "bin scan probe");
  });
}

size_t nebula_hash_bin_workspace_size(uint32_t hashCells, uint32_t particleCount) { return binLayout(hashCells, particleCount).total; }

int nebula_hash_bin(const nebula_hash_grid* grid, const float* dPredP4, const uint32_t* dTypeFlag, uint32_t particleCount,
                    uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSortedIdx, void* dWorkspace, size_t workspaceBytes, void* stream) {
  return guarded([&] {
    if (!grid) throw Error(NEBULA_MPM_ERR_INVALID, "null grid");
    if (!(grid->cellSize > 0.f) || !std::isfinite(grid->cellSize)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be finite and > 0");
    for (int a = 0; a < 3; ++a) {
      if (grid->gridRes[a] == 0) throw Error(NEBULA_MPM_ERR_INVALID, "gridRes must be >= 1");
      if (!std::isfinite(grid->worldMin[a])) throw Error(NEBULA_MPM_ERR_INVALID, "worldMin must be finite");
    }
    const uint32_t cube = domainCubeRes(grid->gridRes);
    if (cube > 1024u || uint64_t(grid->hashCells) < uint64_t(cube) * cube * cube)
      throw Error(NEBULA_MPM_ERR_INVALID, "hashCells must hold the Morton cube of gridRes (cubeRes <= 1024)");
    const uint32_t n = particleCount;
    BinWorkspaceLayout L = binLayout(grid->hashCells, n);
    if (!dWorkspace || workspaceBytes < L.total) throw Error(NEBULA_MPM_ERR_INVALID, "hash workspace too small");
    if (!dCellCount || !dCellOffset || (n && (!dPredP4 || !dSortedIdx))) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BinBuffers b = workspaceBins(L, dWorkspace, grid->hashCells);
    b.cellCount = dCellCount;
    b.cellEnd = dCellOffset;
    b.sorted = dSortedIdx;
    b.typeFlag = dTypeFlag;
    check(cudaMemsetAsync(b.err, 0, 4, s), "memset");
    SubstepParams P{};
    P.cellSize = grid->cellSize;
    for (int a = 0; a < 3; ++a) {
      P.gridRes[a] = int(grid->gridRes[a]);
      P.worldMin[a] = grid->worldMin[a];
    }
    P.cubeRes = cube;
    P.hashCells = grid->hashCells;
    uint64_t launches = 0;
    check(launchBin(P, reinterpret_cast<const float4*>(dPredP4), n, b, s, &launches), "hash bin");
  });
}

int nebula_mpm_p2g(const nebula_mpm_pass* pass, const nebula_mpm_particles* parts, const uint32_t* dCellCount, const uint32_t* dCellOffset,
                   const uint32_t* dSorted, const nebula_mpm_material* dMaterials, float* dGridMom, float* dGridMass, void* stream) {
  return guarded([&] {
    validate(pass);
    (void)dCellCount;
    (void)dCellOffset;
    if (!dGridMom || !dGridMass) throw Error(NEBULA_MPM_ERR_INVALID, "null grid");
    if (pass->materialCount && !dMaterials) throw Error(NEBULA_MPM_ERR_INVALID, "null materials");
    StatePtrs st = statePtrs(parts);
    const uint32_t n = pass->particleCount;
    if (n && !dSorted) throw Error(NEBULA_MPM_ERR_INVALID, "null sorted indices");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemsetAsync(dGridMom, 0, size_t(pass->hashCells) * 2 * sizeof(float4), s), "zero grid");
    check(cudaMemsetAsync(dGridMass, 0, size_t(pass->hashCells) * sizeof(float), s), "zero grid");
    uint64_t launches = 0;
    SubstepParams P = fromPass(*pass, dMaterials, nullptr, nullptr, nullptr);
    check(launchP2GDense(P, st, dSorted, n, reinterpret_cast<float4*>(dGridMom), dGridMass, s, &launches), "p2g");
  });
}

int nebula_mpm_grid_update(const nebula_mpm_pass* pass, float* dGridMom, const float* dGridMass, const nebula_mpm_collider* dColliders,
                           const nebula_mpm_force* dForces, const float* dSdf, void* stream) {
  return guarded([&] {
    validate(pass);
    if (!dGridMom || !dGridMass) throw Error(NEBULA_MPM_ERR_INVALID, "null grid");
    if ((pass->colliderCount && !dColliders) || (pass->forceCount && !dForces)) throw Error(NEBULA_MPM_ERR_INVALID, "null table");
    uint64_t launches = 0;
    SubstepParams P = fromPass(*pass, nullptr, dColliders, dForces, dSdf);
    check(launchGridDense(P, reinterpret_cast<float4*>(dGridMom), dGridMass, static_cast<cudaStream_t>(stream), &launches), "grid update");
  });
}

int nebula_mpm_g2p(const nebula_mpm_pass* pass, const nebula_mpm_particles* parts, const float* dGridMom, const float* dGridMass,
                   const nebula_mpm_material* dMaterials, const float* dSdf, void* stream) {
  return guarded([&] {
    validate(pass);
    if (!dGridMom || !dGridMass) throw Error(NEBULA_MPM_ERR_INVALID, "null grid");
    if (pass->materialCount && !dMaterials) throw Error(NEBULA_MPM_ERR_INVALID, "null materials");
    StatePtrs st = statePtrs(parts);
    uint64_t launches = 0;
    SubstepParams P = fromPass(*pass, dMaterials, nullptr, nullptr, dSdf);
    check(launchG2PDense(P, st, pass->particleCount, reinterpret_cast<const float4*>(dGridMom), dGridMass, nullptr,
                         static_cast<cudaStream_t>(stream), &launches),
          "g2p");
  });
}

}  // extern "C"
