// mpm_internal.h -- launch helpers shared by the engine and the C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_device.cuh"

namespace nebula {

constexpr uint32_t kErrNonFinite = 1u << 1;   // a particle left G2P with a non-finite position
constexpr uint32_t kErrTileOverflow = 1u << 2; // informational: a particle scattered outside its block tile
constexpr uint32_t kErrBinRange = 1u << 3;     // a binning index fell outside [0, n) (follows an expired scan wait)

enum : int { kPhaseBin = 0, kPhaseP2G = 1, kPhaseGrid = 2, kPhaseG2P = 3, kPhaseFused = 4, kPhaseOther = 5 };

struct StatePtrs {
  float4* f[8];  // P, v, F0, F1, F2, B0, B1, B2
};

// Buffers of the counting sort.  cellStart / cellEnd / cellCount are dense
// over hashCells; key / rank / sortedTmp / sorted over particles.
struct BinBuffers {
  uint32_t* cellCount;
  uint32_t* cellStart;
  uint32_t* cellEnd;
  uint32_t* key;
  uint32_t* rank;
  uint32_t* sortedTmp;
  uint32_t* sorted;
  unsigned long long* tileState;  // scanTiles(hashCells) words
  uint32_t* tileCounter;
  uint32_t* err;
  // Optional per-particle type flags: particles flagged kTypeFlagUnused stay
  // out of the bins (the PBF binning, hash_count.comp:9-16).
  const uint32_t* typeFlag = nullptr;
};
constexpr uint32_t kTypeFlagUnused = 6u;

// Bytes of scan workspace (tile status words + counter) for `n` items.
size_t scanWorkspaceBytes(uint64_t n);

// Counting sort of particles by Morton cell: counts, exclusive scan, scatter,
// then in-cell ordering by ascending particle index.  `launches` counts kernels.
cudaError_t launchBin(const SubstepParams& P, const float4* pos, uint32_t n, const BinBuffers& b, cudaStream_t s, uint64_t* launches);
// Failure-path self-test of launchBin's scan on the same buffers: one CTA of
// the cell scan runs as tile 1 against a tile 0 that never publishes, so its
// bounded look-back gives up, sets kErrScanTimeout in *b.err and returns
// (about a second).  Reads cellCount[0, hashCells), writes only workspace
// words (cellStart of tile 1, the status words, the ticket, the error word).
// Needs hashCells >= 2 scan tiles (4,096 cells).
cudaError_t launchBinScanExpiryProbe(const SubstepParams& P, const BinBuffers& b, cudaStream_t s, uint64_t* launches);
// Particle-major P2G into the reference's dense grid layout (grid must be zeroed).
cudaError_t launchP2GDense(const SubstepParams& P, StatePtrs st, const uint32_t* sorted, uint32_t n, float4* gridMom, float* gridMass,
                           cudaStream_t s, uint64_t* launches);
// Grid update + dense-SDF boundary per node over all hashCells.
cudaError_t launchGridDense(const SubstepParams& P, float4* gridMom, const float* gridMass, cudaStream_t s, uint64_t* launches);
// G2P over particles [0, n) against the dense grid.
cudaError_t launchG2PDense(const SubstepParams& P, StatePtrs st, uint32_t n, const float4* gridMom, const float* gridMass, uint32_t* err,
                           cudaStream_t s, uint64_t* launches);

}  // namespace nebula
