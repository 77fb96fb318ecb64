// mpm_scan.cuh -- single-pass exclusive scan of u32 counts (decoupled look-back).
//
// Replaces the reference's three-dispatch scan (hash_scan_local.comp:10-43,
// hash_scan_global.comp:10-35, hash_add_base.comp:11-22), which is only correct
// while hashCells <= 256*1024; this one is correct for any length.
//
// Each CTA takes the next tile index from a global counter (so every tile it
// waits on belongs to a CTA that is already running), scans its 2048 items,
// publishes its aggregate, then walks back over earlier tiles' published
// values.  Every wait is bounded: after kScanSpinLimit polls the CTA records
// an error bit and continues with what it has, so a fault can never hang the
// GPU.  Workspace: one u64 status word per tile plus one u32 tile counter,
// zeroed before the launch.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nebula {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kScanSpinLimit = 1u << 22;
constexpr unsigned long long kFlagAggregate = 1ull << 32;
constexpr unsigned long long kFlagPrefix = 2ull << 32;
constexpr uint32_t kErrScanTimeout = 1u << 0;

__host__ __device__ inline uint32_t scanTiles(uint64_t n) { return uint32_t((n + kScanTile - 1) / kScanTile); }

}  // namespace nebula
