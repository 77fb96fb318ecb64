// mpm_scan_kernel.cuh -- the scan kernel itself (included by one translation unit).
#pragma once
#include "mpm_scan.cuh"

namespace nebula {

__device__ __forceinline__ unsigned long long ldVolatile64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

// out_start[i] = sum_{j<i} in[j]; out_end[i] = out_start[i] + in[i] (either may be null).
// *total (if non-null) receives the sum of all items.
__global__ void __launch_bounds__(kScanThreads) k_scan_exclusive(const uint32_t* __restrict__ in, uint32_t* __restrict__ out_start,
                                                                 uint32_t* __restrict__ out_end, uint64_t n, unsigned long long* tile_state,
                                                                 uint32_t* tile_counter, uint32_t* err, uint32_t* total) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t i0 = uint64_t(tile) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
  uint32_t v[kScanItems];
  uint32_t tsum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (i0 + k < n) ? __ldg(in + i0 + k) : 0u;
    tsum += v[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t block_total = s_warp[kScanThreads / 32 - 1];
  const uint32_t excl = (warp > 0 ? s_warp[warp - 1] : 0u) + incl - tsum;
  if (threadIdx.x == 0) {
    uint32_t prefix = 0;
    if (tile == 0) {
      atomicExch(tile_state, kFlagPrefix | block_total);
    } else {
      atomicExch(tile_state + tile, kFlagAggregate | block_total);
      int64_t j = int64_t(tile) - 1;
      uint32_t spins = 0;
      while (j >= 0) {
        unsigned long long s = ldVolatile64(tile_state + j);
        unsigned long long flag = s & (3ull << 32);
        if (flag == 0) {
          if (++spins > kScanSpinLimit) {
            atomicOr(err, kErrScanTimeout);
            break;
          }
          __nanosleep(32);
          continue;
        }
        prefix += uint32_t(s & 0xffffffffull);
        if (flag == kFlagPrefix) break;
        --j;
      }
      atomicExch(tile_state + tile, kFlagPrefix | uint32_t(prefix + block_total));
    }
    s_prefix = prefix;
    if (total && tile == scanTiles(n) - 1) *total = prefix + block_total;
  }
  __syncthreads();
  uint32_t run = s_prefix + excl;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (i0 + k < n) {
      if (out_start) out_start[i0 + k] = run;
      if (out_end) out_end[i0 + k] = run + v[k];
    }
    run += v[k];
  }
}

}  // namespace nebula
