// mpm_bricks.cuh -- buffers and launchers of the brick-sparse fused substep.
//
// The grid is split into bricks of 4x4x4 cells; a brick is 64 consecutive
// Morton codes, so brick id = cell Morton code >> 6.  Per substep:
//   grid     sparse grid update over the bricks the last P2G touched
//   g2p2g    per particle brick: G2P from the staged grid, particle update,
//            P2G of the updated particle into a shared tile, binning count
//   scan     brick counts / marks -> particle-brick list, grid-brick list,
//            brick starts (single pass, decoupled look-back, compaction)
//   perm     (cell, rank) -> sorted slot of every particle: its brick's start
//            plus the counts of the brick's lower cells plus its rank
// Particles are physically reordered by cell every substep (bricks in Morton
// order, the 64 cells of a brick in Morton order; ping-pong state buffers
// plus the original particle id).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_internal.h"

namespace nebula {

constexpr int kBrickScanThreads = 256;
constexpr int kBrickScanItems = 8;
constexpr int kBrickScanTile = kBrickScanThreads * kBrickScanItems;

// counters[] slots
enum : int { kCntNumPB = 0, kCntNumGB = 1, kCntTotal = 2, kCntQueueP2G = 3, kCntQueueFused = 4, kCntOverflow = 5, kCntSlots = 8 };

struct BrickBuffers {
  uint32_t nb;                // number of bricks (>= 1)
  uint32_t tiles;             // scan tiles over nb
  uint32_t* brickCount;       // [nb] particles per brick (zeroed by the scan)
  uint32_t* brickFlag;        // [nb] grid-active marks (zeroed by the scan)
  uint32_t* brickStart;       // [nb] first sorted slot of each brick
  // Per-cell particle counts, two arrays used in turn: the binning of the
  // state in buffer q counts into array q, the fused kernel that reads that
  // state (and counts its output into the other array) clears array q brick
  // by brick as it takes the bricks' items, after the permutation has read it.
  uint32_t* cellCount;        // [64 nb] the counts of this binning
  uint32_t* cellPrev;         // [64 nb] the counts of the binning before it (cleared by the fused kernel)
  uint32_t* pbBrick;          // [nb] particle-brick list
  uint32_t* pbStart;          // [nb + 1] first slot of each listed brick; pbStart[numPB] = total
  uint32_t* gbBrick;          // [nb] grid-brick list, ascending (k_brick_scan writes it in brick order)
  uint32_t* counters;         // [kCntSlots]
  unsigned long long* scanState;  // [3 * tiles] status words (epoch-tagged)
  unsigned long long* scanTile;   // monotone tile counter
  uint32_t* binKey;           // [cap] cell (global code: 64 x brick + Morton code in the brick) of each particle (by buffer index)
  uint32_t* binRank;          // [cap] rank inside its cell
  uint32_t* perm;             // [cap] sorted slot -> buffer index
};

// The scenes of a batch share one brick space: scene s owns the global bricks
// [brickBase[s], brickBase[s+1]) and the particle slots [partBase[s],
// partBase[s+1]) of every brick-ordered buffer (a sort by global brick keeps
// each scene's particles together).  Grid arrays are indexed by global cell
// code = 64 * brickBase[s] + the scene's own Morton code.
struct SceneTable {
  const SubstepParams* params;  // [count] per-scene substep parameters
  const uint32_t* brickBase;    // [count + 1]
  const uint32_t* partBase;     // [count + 1]
  uint32_t count;
};

struct GridBuffers {
  float4* acc;   // [ncPad] (mom.xyz, mass) accumulated by P2G
  float4* vel;   // [ncPad] (v.xyz, mass) after the grid update
  float4* vold;  // [ncPad] pre-force velocity (FLIP), may be null
};

// Launch shape of the per-substep kernels, picked per GPU and workload by the
// autotuner (nebula_b200/autotune.py); 0 CTAs per SM = as many as fit.
struct LaunchConfig {
  uint32_t fusedThreads = 0;    // k_g2p2g CTA size: 192 or 256 (a warp takes 32 slots per round); 0 = by scene size
  uint32_t fusedCtasPerSm = 0;  // persistent k_g2p2g CTAs per SM
  uint32_t gridCtasPerSm = 0;   // persistent grid-update CTAs per SM
  uint32_t gridBatch = 4;       // k_grid_bricks nodes per thread per round: 2 or 4
  uint32_t fusedSplit = 0;      // k_g2p2g items per particle brick (1-4): contiguous parts of a brick's slots; 0 = by scene size
};
// Most CTAs per SM (occupancy) of each variant: [fusedThreads == 256], [gridBatch == 4].
struct LaunchLimits {
  uint32_t fusedCtasPerSm[2];
  uint32_t gridCtasPerSm[2];
};
LaunchLimits launchLimits(bool flip, bool batch);

// Standalone binning of the particles in buffer order: counts + stencil marks.
cudaError_t launchBrickCount(const SubstepParams& P, const float4* pos, uint32_t n, const BrickBuffers& b, uint32_t* err, cudaStream_t s,
                             uint64_t* launches);
// Compaction scan (tile numbering and status epochs come from a device ticket).
cudaError_t launchBrickScan(const BrickBuffers& b, uint32_t* err, cudaStream_t s, uint64_t* launches);
cudaError_t launchPermScatter(const BrickBuffers& b, uint32_t n, uint32_t* err, cudaStream_t s, uint64_t* launches);
// P2G of the particles of every listed brick (no binning, no marks).
cudaError_t launchP2GBricks(const SubstepParams& P, StatePtrs cur, uint32_t n, const BrickBuffers& b, GridBuffers g, float dtStress,
                            int numSMs, cudaStream_t s, uint64_t* launches);
// Sparse grid update over the listed grid bricks; clears acc as it reads.
// Also scatters the permutation (sorted slot -> buffer index of the n
// particles) of the binning before it, which the next fused kernel reads
// (n = 0: none).  Below kFoldScatterMax particles the scatter rides on the
// grid launch (one launch fewer per substep: -3.4% per substep at 8,000
// particles, -1.4% at 80,000); above it the separate k_perm_scatter launch,
// all of whose threads issue their loads at once, is faster (+0.3% folded
// at 1M).
constexpr uint32_t kFoldScatterMax = 1u << 19;
cudaError_t launchGridBricks(const SubstepParams& P, const BrickBuffers& b, GridBuffers g, uint32_t n, uint32_t* err, const LaunchConfig& lc,
                             int numSMs, cudaStream_t s, uint64_t* launches);
// Zero acc over the listed grid bricks (discarding a pending P2G).
cudaError_t launchClearBricks(const BrickBuffers& b, GridBuffers g, int numSMs, cudaStream_t s, uint64_t* launches);
// The material-model set (ModelSet, mpm_particle.cuh) a fused kernel may be
// specialised for: that of every material of the table.
int modelSetOf(const Material* mats, uint32_t count);
// The fused G2P -> particle update -> P2G + binning count, specialised for
// `modelSet` where an instantiation exists.
cudaError_t launchG2P2G(const SubstepParams& P, int modelSet, StatePtrs cur, const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt, uint32_t n,
                        const BrickBuffers& b, GridBuffers g, float dtStress, uint32_t* err, const LaunchConfig& lc, int numSMs, cudaStream_t s,
                        uint64_t* launches);
// Batched forms: every scene of `T` in one launch.  `substep` selects the
// colliders of this substep on each scene's collider track
// (params.colliders + substep * params.colliderCount).
cudaError_t launchBrickCountBatch(const SceneTable& T, const float4* pos, uint32_t n, const BrickBuffers& b, cudaStream_t s, uint64_t* launches);
cudaError_t launchP2GBricksBatch(const SceneTable& T, StatePtrs cur, uint32_t n, const BrickBuffers& b, GridBuffers g, int numSMs,
                                 cudaStream_t s, uint64_t* launches);
cudaError_t launchGridBricksBatch(const SceneTable& T, uint32_t substep, const BrickBuffers& b, GridBuffers g, uint32_t n, uint32_t* err,
                                  const LaunchConfig& lc, int numSMs, cudaStream_t s, uint64_t* launches);
cudaError_t launchG2P2GBatch(const SceneTable& T, int modelSet, bool flip, StatePtrs cur, const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt,
                             uint32_t n, const BrickBuffers& b, GridBuffers g, uint32_t* err, const LaunchConfig& lc, int numSMs, cudaStream_t s,
                             uint64_t* launches);
// Run the brick scan's bounded look-back against a predecessor that never
// publishes; *errorBits receives the device error word (kErrScanTimeout set
// when the wait gave up as designed).
cudaError_t probeWaitExpiry(uint32_t* errorBits);
// Resolve every launcher's one-time set-up (shared-memory limits, persistent
// block counts) outside any stream capture.
void prepareBrickKernels(int numSMs);
// out[pid[i]] = in[i] for the 8 fields (original particle order).
cudaError_t launchUnpermute(StatePtrs in, const uint32_t* pid, StatePtrs out, uint32_t n, cudaStream_t s, uint64_t* launches);
cudaError_t launchIota(uint32_t* pid, uint32_t n, cudaStream_t s, uint64_t* launches);
// out[t] = pid[perm[t]]: original particle ids in brick order.
cudaError_t launchSortedPid(const uint32_t* perm, const uint32_t* pid, uint32_t* out, uint32_t n, cudaStream_t s, uint64_t* launches);

}  // namespace nebula
