// mpm_bricks.cu -- brick-sparse fused substep kernels (sm_100a).
//
// Same per-particle and per-node math as the single-pass kernels
// (mpm_particle.cuh, restating mpm_p2g.comp, mpm_grid_update.comp,
// mpm_nanovdb_bc.comp and mpm_g2p.comp), organised for HBM:
//   * particles live in brick order, read once and written once per substep;
//   * G2P reads a brick's 6^3 node neighbourhood staged in shared memory;
//   * P2G accumulates into an 8^3 shared tile and flushes each non-zero node
//     with one vector reduction to global memory;
//   * only bricks some particle stencil touched are updated or cleared.
#include "mpm_bricks.cuh"
#include "mpm_particle.cuh"
#include "mpm_scan.cuh"

#include <algorithm>
#include <atomic>
#include <mutex>

namespace nebula {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kBrickScanSpinLimit = 1u << 22;
constexpr unsigned long long kStFlagAgg = 1ull << 48;
constexpr unsigned long long kStFlagPre = 2ull << 48;
constexpr unsigned long long kStValue = (1ull << 48) - 1;

inline uint32_t blocksFor(uint64_t n, int t = kThreads) { return uint32_t((n + t - 1) / t); }

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }

// Programmatic dependent launch: the per-substep kernels are launched with
// programmatic stream serialization, so a kernel's CTAs may be scheduled as
// soon as the previous kernel's CTAs have all exited (no kernel triggers
// earlier), hiding the launch latency between them.  Every such kernel waits
// here, before its first memory access, until the previous grid has
// completed and its writes are visible; without the launch attribute the
// wait returns at once.
__device__ __forceinline__ void waitForPredecessorGrid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class... KArgs, class... Args>
cudaError_t launchSerialized(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Lanes in `mask` holding the same key take consecutive slots of counter[key].
__device__ __forceinline__ uint32_t warpAggInc(uint32_t mask, uint32_t* counter, uint32_t key) {
  const uint32_t peers = __match_any_sync(mask, key);
  const int leader = __ffs(peers) - 1;
  const uint32_t lane = laneId();
  uint32_t base = 0;
  if (int(lane) == leader) base = atomicAdd(counter + key, uint32_t(__popc(peers)));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

// The same for lanes whose keys come in a few runs (particles in cell order),
// in two halves so the atomic's round trip overlaps other work: the claim
// finds the groups with one ballot per distinct key instead of a match, and
// every group leader issues its atomic at once; the rank reads the leader's
// result later.  Every lane of `mask` calls both with the same mask.
struct GroupTicket {
  uint32_t peers;  // lanes of this lane's key
  uint32_t base;   // the leader's atomic result (in the leader)
};
__device__ __forceinline__ GroupTicket warpGroupClaim(uint32_t mask, uint32_t* counter, uint32_t key) {
  uint32_t pending = mask, mine = 0;
  while (pending) {
    const int leader = __ffs(pending) - 1;
    const uint32_t k = __shfl_sync(mask, key, leader);
    const uint32_t peers = __ballot_sync(mask, key == k);
    if (key == k) mine = peers;
    pending &= ~peers;
  }
  GroupTicket g{mine, 0u};
  if (int(laneId()) == __ffs(mine) - 1) g.base = atomicAdd(counter + key, uint32_t(__popc(mine)));
  return g;
}
__device__ __forceinline__ uint32_t warpGroupRank(uint32_t mask, const GroupTicket& g) {
  const uint32_t base = __shfl_sync(mask, g.base, __ffs(g.peers) - 1);
  return base + __popc(g.peers & ((1u << laneId()) - 1u));
}

// counter[key] += number of lanes of `mask` holding key (keys in a few runs).
__device__ __forceinline__ void warpGroupAdd(uint32_t mask, uint32_t* counter, uint32_t key) {
  uint32_t pending = mask;
  while (pending) {
    const int leader = __ffs(pending) - 1;
    const uint32_t k = __shfl_sync(mask, key, leader);
    const uint32_t peers = __ballot_sync(mask, key == k);
    if (int(laneId()) == leader) atomicAdd(counter + k, uint32_t(__popc(peers)));
    pending &= ~peers;
  }
}

// Mark every brick holding a node of the 3x3x3 stencil around cell (cx,cy,cz).
__device__ __forceinline__ void markStencilBricks(const SubstepParams& P, int cx, int cy, int cz, uint32_t* flag) {
  const int cr = int(P.cubeRes) - 1;
  const int x0 = max(cx - 1, 0) >> 2, x1 = min(cx + 1, cr) >> 2;
  const int y0 = max(cy - 1, 0) >> 2, y1 = min(cy + 1, cr) >> 2;
  const int z0 = max(cz - 1, 0) >> 2, z1 = min(cz + 1, cr) >> 2;
  for (int bz = z0; bz <= z1; ++bz)
    for (int by = y0; by <= y1; ++by)
      for (int bx = x0; bx <= x1; ++bx) flag[mortonEncode(bx, by, bz)] = 1u;
}

// Bit (dz*9 + dy*3 + dx) of the 3^3 bricks around brick (bx, by, bz) for every
// brick the stencil of cell (cx,cy,cz) touches; false when one lies outside
// that neighbourhood (the caller then marks globally).
__device__ __forceinline__ bool stencilBrickMask(const SubstepParams& P, int cx, int cy, int cz, int bx, int by, int bz, uint32_t& mask) {
  const int cr = int(P.cubeRes) - 1;
  const int x0 = max(cx - 1, 0) >> 2, x1 = min(cx + 1, cr) >> 2;
  const int y0 = max(cy - 1, 0) >> 2, y1 = min(cy + 1, cr) >> 2;
  const int z0 = max(cz - 1, 0) >> 2, z1 = min(cz + 1, cr) >> 2;
  if (x0 < bx - 1 || x1 > bx + 1 || y0 < by - 1 || y1 > by + 1 || z0 < bz - 1 || z1 > bz + 1) return false;
  // per axis the 3-bit set of touched neighbour offsets; their product set is
  // the bits z*9 + y*3 + x: spreading y's bits to 0/3/6 and z's to 0/9/18
  // makes it two multiplications (the partial products never overlap)
  const uint32_t mx = ((2u << (x1 - x0)) - 1u) << (x0 - bx + 1);
  const uint32_t my = ((2u << (y1 - y0)) - 1u) << (y0 - by + 1);
  const uint32_t mz = ((2u << (z1 - z0)) - 1u) << (z0 - bz + 1);
  const uint32_t ys = (my & 1u) | ((my & 2u) << 2) | ((my & 4u) << 4);
  const uint32_t zs = (mz & 1u) | ((mz & 2u) << 8) | ((mz & 4u) << 16);
  mask |= (mx * ys) * zs;
  return true;
}

// Flags of the marked neighbour bricks of item brick (bx, by, bz); run by threads 0..26.
__device__ __forceinline__ void flushBrickMarks(const SubstepParams& P, uint32_t mask, int bx, int by, int bz, uint32_t* flag) {
  const int t = threadIdx.x;
  if (t >= 27 || !((mask >> t) & 1u)) return;
  const int x = bx + t % 3 - 1, y = by + (t / 3) % 3 - 1, z = bz + t / 9 - 1;
  const int bmax = (int(P.cubeRes) - 1) >> 2;
  if (x < 0 || y < 0 || z < 0 || x > bmax || y > bmax || z > bmax) return;
  flag[mortonEncode(x, y, z)] = 1u;
}

// ------------------------------------------------------------------ batch scenes
// The scene s with base[s] <= x < base[s+1] (base non-decreasing, x < base[count]).
__device__ __forceinline__ uint32_t findScene(const uint32_t* __restrict__ base, uint32_t count, uint32_t x) {
  uint32_t lo = 0, hi = count;
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

static_assert(sizeof(SubstepParams) % 4 == 0, "SubstepParams is copied as 32-bit words");
constexpr int kParamWords = int(sizeof(SubstepParams) / 4);

// Word copy of one scene's parameters by threads t = 0..nthreads-1.
__device__ __forceinline__ void copyParams(SubstepParams* dst, const SubstepParams* src, int t, int nthreads) {
  const uint32_t* a = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  for (int q = t; q < kParamWords; q += nthreads) d[q] = a[q];
}

__device__ __forceinline__ GridBuffers offsetGrid(const GridBuffers& G, uint32_t brickBase) {
  const size_t c = size_t(brickBase) << 6;
  return GridBuffers{G.acc + c, G.vel + c, G.vold ? G.vold + c : nullptr};
}

// ------------------------------------------------------------------ binning count (standalone)
template <bool BATCH>
__global__ void __launch_bounds__(kThreads) k_brick_count(SubstepParams P0, SceneTable T, const float4* __restrict__ pos, uint32_t n,
                                                          BrickBuffers B) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < n;
  const uint32_t mask = __ballot_sync(0xffffffffu, act);
  if (!act) return;
  const float4 p = pos[i];
  auto body = [&](const SubstepParams& P, uint32_t base) {
    int cx, cy, cz;
    cellCoords(P, p.x, p.y, p.z, cx, cy, cz);
    const uint32_t c = (base << 6) + mortonEncode(cx, cy, cz);
    B.binKey[i] = c;
    B.binRank[i] = warpAggInc(mask, B.cellCount, c);
    (void)warpAggInc(mask, B.brickCount, c >> 6);
    markStencilBricks(P, cx, cy, cz, B.brickFlag + base);
  };
  if constexpr (BATCH) {
    const uint32_t sc = findScene(T.partBase, T.count, i);
    body(T.params[sc], T.brickBase[sc]);
  } else {
    body(P0, 0u);
  }
}

// ------------------------------------------------------------------ compaction scan
__device__ __forceinline__ unsigned long long ldv64(const unsigned long long* p) { return *reinterpret_cast<const volatile unsigned long long*>(p); }

// One chain of the decoupled look-back, run by a whole warp: returns the
// exclusive prefix of `tile` (in every lane).  The warp reads 32 predecessor
// status words at once; it may add them up to the nearest published prefix
// once every tile in between has published its aggregate, and otherwise
// takes all 32 aggregates and moves 32 tiles back.  Waits are bounded.
__device__ uint32_t lookBackWarp(unsigned long long* st, uint32_t tile, uint32_t aggregate, unsigned long long tag, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) atomicExch(st, tag | kStFlagPre | aggregate);
    return 0;
  }
  if (lane == 0) atomicExch(st + tile, tag | kStFlagAgg | aggregate);
  uint32_t prefix = 0;
  int64_t j = int64_t(tile) - 1;  // nearest predecessor not yet added
  uint32_t spins = 0;
  for (;;) {
    const int64_t idx = j - lane;
    bool ready = true, isPre = true;  // before tile 0: an empty prefix
    uint32_t val = 0;
    if (idx >= 0) {
      const unsigned long long s = ldv64(st + idx);
      const bool mine = (s & ~((1ull << 50) - 1)) == tag;
      const unsigned long long flag = s & (3ull << 48);
      ready = mine && flag != 0;
      isPre = ready && flag == kStFlagPre;
      val = uint32_t(s & kStValue);
    }
    const uint32_t preMask = __ballot_sync(0xffffffffu, isPre);
    const uint32_t notReady = __ballot_sync(0xffffffffu, !ready);
    const int last = preMask ? __ffs(preMask) - 1 : 31;  // lanes 0..last are consumed
    const uint32_t need = last == 31 ? 0xffffffffu : ((2u << last) - 1u);
    if ((notReady & need) == 0u) {
      uint32_t v = lane <= last ? val : 0u;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      prefix += v;
      if (preMask) break;
      j -= 32;
      continue;
    }
    if (++spins > kBrickScanSpinLimit) {
      if (lane == 0) atomicOr(err, kErrScanTimeout);
      break;
    }
    __nanosleep(32);
  }
  if (lane == 0) atomicExch(st + tile, tag | kStFlagPre | uint32_t(prefix + aggregate));
  return prefix;
}

// One warp waits as tile 1 on a tile 0 that never publishes: the bounded
// look-back must give up after kBrickScanSpinLimit polls (a second or two),
// set kErrScanTimeout and return.
__global__ void k_wait_expiry_probe(unsigned long long* st, uint32_t* err) { (void)lookBackWarp(st, 1u, 0u, 0ull, err); }

// Tickets from the monotone counter number every tile of every launch: tile =
// ticket % tiles, launch = ticket / tiles.  Launches are stream-ordered, so one
// launch's tickets are contiguous, and no host-side value changes between
// launches (the kernel can be replayed from a CUDA graph).
__global__ void __launch_bounds__(kBrickScanThreads) k_brick_scan(BrickBuffers B, uint32_t* err) {
  __shared__ unsigned long long s_ticket;
  __shared__ uint32_t s_warp[3][kBrickScanThreads / 32];
  __shared__ uint32_t s_prefix[3];
  waitForPredecessorGrid();
  if (threadIdx.x == 0) s_ticket = atomicAdd(B.scanTile, 1ull);
  __syncthreads();
  const uint32_t tile = uint32_t(s_ticket % B.tiles);
  const uint32_t epoch = uint32_t(s_ticket / B.tiles);
  const unsigned long long tag = (unsigned long long)(epoch & 0x3fffu) << 50;
  const uint32_t b0 = tile * kBrickScanTile + threadIdx.x * kBrickScanItems;
  static_assert(kBrickScanItems == 8, "the vector path moves 8 bricks as two uint4");
  uint32_t cnt[kBrickScanItems];
  uint32_t flg = 0;  // bit k: grid-active
  uint32_t sc = 0, sp = 0, sg = 0;
  const bool full = b0 + kBrickScanItems <= B.nb;  // b0 is a multiple of 8: 32-byte aligned
  if (full) {
    uint4* pc = reinterpret_cast<uint4*>(B.brickCount + b0);
    uint4* pf = reinterpret_cast<uint4*>(B.brickFlag + b0);
    const uint4 c0 = pc[0], c1 = pc[1], f0 = pf[0], f1 = pf[1];
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    pc[0] = z; pc[1] = z; pf[0] = z; pf[1] = z;
    cnt[0] = c0.x; cnt[1] = c0.y; cnt[2] = c0.z; cnt[3] = c0.w;
    cnt[4] = c1.x; cnt[5] = c1.y; cnt[6] = c1.z; cnt[7] = c1.w;
    const uint32_t fv[8] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
#pragma unroll
    for (int k = 0; k < kBrickScanItems; ++k)
      if (fv[k]) flg |= 1u << k;
  } else {
#pragma unroll
    for (int k = 0; k < kBrickScanItems; ++k) {
      const uint32_t b = b0 + k;
      cnt[k] = 0;
      if (b < B.nb) {
        cnt[k] = B.brickCount[b];
        const uint32_t f = B.brickFlag[b];
        B.brickCount[b] = 0;
        B.brickFlag[b] = 0;
        if (f) flg |= 1u << k;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kBrickScanItems; ++k) {
    sc += cnt[k];
    sp += cnt[k] ? 1u : 0u;
  }
  sg = __popc(flg);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t ic = sc, ip = sp, ig = sg;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yc = __shfl_up_sync(0xffffffffu, ic, o), yp = __shfl_up_sync(0xffffffffu, ip, o), yg = __shfl_up_sync(0xffffffffu, ig, o);
    if (lane >= o) {
      ic += yc;
      ip += yp;
      ig += yg;
    }
  }
  if (lane == 31) {
    s_warp[0][warp] = ic;
    s_warp[1][warp] = ip;
    s_warp[2][warp] = ig;
  }
  __syncthreads();
  if (warp == 0) {
    constexpr int W = kBrickScanThreads / 32;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uint32_t w = lane < W ? s_warp[c][lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < W) s_warp[c][lane] = w;
    }
  }
  __syncthreads();
  constexpr int WL = kBrickScanThreads / 32 - 1;
  // chains run in three different warps
  if (warp < 3) {
    const int c = warp;
    const uint32_t agg = s_warp[c][WL];
    const uint32_t pre = lookBackWarp(B.scanState + size_t(c) * B.tiles, tile, agg, tag, err);
    if (lane == 0) s_prefix[c] = pre;
    if (lane == 0 && tile == B.tiles - 1) {
      const uint32_t total = pre + agg;
      if (c == 0) {
        B.counters[kCntTotal] = total;
      } else if (c == 1) {
        B.counters[kCntNumPB] = total;
      } else {
        B.counters[kCntNumGB] = total;
      }
    }
  }
  __syncthreads();
  uint32_t rc = s_prefix[0] + (warp > 0 ? s_warp[0][warp - 1] : 0u) + ic - sc;
  uint32_t rp = s_prefix[1] + (warp > 0 ? s_warp[1][warp - 1] : 0u) + ip - sp;
  uint32_t rg = s_prefix[2] + (warp > 0 ? s_warp[2][warp - 1] : 0u) + ig - sg;
  uint32_t starts[kBrickScanItems];
#pragma unroll
  for (int k = 0; k < kBrickScanItems; ++k) {
    const uint32_t b = b0 + k;
    starts[k] = rc;
    if (b < B.nb) {
      if (!full) B.brickStart[b] = rc;
      if (cnt[k]) {
        B.pbBrick[rp] = b;
        B.pbStart[rp] = rc;
        ++rp;
      }
      if (flg & (1u << k)) {
        B.gbBrick[rg] = b;
        ++rg;
      }
    }
    rc += cnt[k];
  }
  if (full) {
    uint4* ps = reinterpret_cast<uint4*>(B.brickStart + b0);
    ps[0] = make_uint4(starts[0], starts[1], starts[2], starts[3]);
    ps[1] = make_uint4(starts[4], starts[5], starts[6], starts[7]);
  }
  if (tile == B.tiles - 1 && threadIdx.x == 0) {
    // the last tile's look-back finished, so all three totals are final
    const uint32_t npb = s_prefix[1] + s_warp[1][WL];
    B.pbStart[npb] = s_prefix[0] + s_warp[0][WL];
    B.counters[kCntQueueP2G] = 0;
    B.counters[kCntQueueFused] = 0;
  }
}

// Sorted slots of the buffer indices t of one warp (every lane calls it; `valid`
// per lane): the start of the particle's brick, plus the counts of the cells
// of the brick below its cell, plus its rank in its cell.  The lanes' keys
// come in a few bricks (the buffer holds particles in cell order), and for
// each distinct brick the warp reads its 64 counts once (two per lane) and
// scans them.
__device__ __forceinline__ void permScatterWarp(const BrickBuffers& B, uint32_t n, uint32_t* err, uint32_t t, bool valid) {
  const uint32_t lane = laneId();
  const uint32_t key = valid ? B.binKey[t] : 0u;
  const uint32_t rank = valid ? B.binRank[t] : 0u;
  const uint32_t brick = key >> 6, cell = key & 63u;
  const uint32_t start = valid ? B.brickStart[brick] : 0u;
  uint32_t below = 0;
  uint32_t pending = __ballot_sync(0xffffffffu, valid);
  while (pending) {
    const uint32_t b = __shfl_sync(0xffffffffu, brick, __ffs(pending) - 1);
    const uint2 c = reinterpret_cast<const uint2*>(B.cellCount + (size_t(b) << 6))[lane];
    uint32_t incl = c.x + c.y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= uint32_t(o)) incl += y;
    }
    const uint32_t pairBelow = __shfl_sync(0xffffffffu, incl - c.x - c.y, cell >> 1);
    const uint32_t evenCount = __shfl_sync(0xffffffffu, c.x, cell >> 1);
    const bool mine = valid && brick == b;
    if (mine) below = pairBelow + ((cell & 1u) ? evenCount : 0u);
    pending &= ~__ballot_sync(0xffffffffu, mine);
  }
  if (valid) {
    const uint32_t slot = start + below + rank;
    if (slot < n) B.perm[slot] = t;
    else atomicOr(err, kErrBinRange);
  }
}

// The same over buffer indices t0, t0 + stride, ... < n (t0 - lane and stride
// multiples of 32, so the warp's lanes stay together).
__device__ __forceinline__ void permScatterStrided(const BrickBuffers& B, uint32_t n, uint32_t* err, uint64_t t0, uint64_t stride) {
  for (uint64_t w = t0 - laneId(); w < n; w += stride) {
    const uint64_t t = w + laneId();
    permScatterWarp(B, n, err, uint32_t(t < n ? t : 0u), t < n);
  }
}

// The separate permutation launch: each warp takes kPermRounds groups of 32
// buffer indices and issues the loads of all groups before their sums (the
// key -> brick start / counts -> slot chain is the kernel's latency); a group
// whose lanes hold more than one brick finishes the other bricks one by one.
constexpr int kPermRounds = 4;
__global__ void __launch_bounds__(kThreads) k_perm_scatter(BrickBuffers B, uint32_t n, uint32_t* err) {
  waitForPredecessorGrid();
  const uint32_t lane = laneId();
  const uint32_t base = (blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)) * (32u * kPermRounds);
  uint32_t t[kPermRounds], key[kPermRounds], rank[kPermRounds], start[kPermRounds], lead[kPermRounds];
  uint2 c[kPermRounds];
#pragma unroll
  for (int r = 0; r < kPermRounds; ++r) {
    t[r] = base + uint32_t(r) * 32u + lane;
    const bool v = t[r] < n;
    key[r] = v ? B.binKey[t[r]] : 0u;
    rank[r] = v ? B.binRank[t[r]] : 0u;
  }
#pragma unroll
  for (int r = 0; r < kPermRounds; ++r) {
    const bool v = t[r] < n;
    start[r] = v ? B.brickStart[key[r] >> 6] : 0u;
    lead[r] = __shfl_sync(0xffffffffu, key[r] >> 6, 0);  // the brick of the group's first lane (lane 0 is valid whenever any lane is)
    c[r] = reinterpret_cast<const uint2*>(B.cellCount + (size_t(lead[r]) << 6))[lane];
  }
#pragma unroll
  for (int r = 0; r < kPermRounds; ++r) {
    const bool v = t[r] < n;
    const uint32_t brick = key[r] >> 6, cell = key[r] & 63u;
    uint32_t incl = c[r].x + c[r].y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= uint32_t(o)) incl += y;
    }
    const uint32_t pairBelow = __shfl_sync(0xffffffffu, incl - c[r].x - c[r].y, cell >> 1);
    const uint32_t evenCount = __shfl_sync(0xffffffffu, c[r].x, cell >> 1);
    const bool first = v && brick == lead[r];
    uint32_t below = first ? pairBelow + ((cell & 1u) ? evenCount : 0u) : 0u;
    if (__ballot_sync(0xffffffffu, v && !first)) {
      // lanes of other bricks: the general per-brick walk
      uint32_t pending = __ballot_sync(0xffffffffu, v && !first);
      while (pending) {
        const uint32_t b = __shfl_sync(0xffffffffu, brick, __ffs(pending) - 1);
        const uint2 cb = reinterpret_cast<const uint2*>(B.cellCount + (size_t(b) << 6))[lane];
        uint32_t in2 = cb.x + cb.y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, in2, o);
          if (lane >= uint32_t(o)) in2 += y;
        }
        const uint32_t pb = __shfl_sync(0xffffffffu, in2 - cb.x - cb.y, cell >> 1);
        const uint32_t ec = __shfl_sync(0xffffffffu, cb.x, cell >> 1);
        const bool mine = v && !first && brick == b;
        if (mine) below = pb + ((cell & 1u) ? ec : 0u);
        pending &= ~__ballot_sync(0xffffffffu, mine);
      }
    }
    if (v) {
      const uint32_t slot = start[r] + below + rank[r];
      if (slot < n) B.perm[slot] = t[r];
      else atomicOr(err, kErrBinRange);
    }
  }
}

// ------------------------------------------------------------------ shared-memory P2G
// A CTA handles one particle brick at a time.  Each particle's P2G inputs go
// to its lane's row in shared memory in separable form (p2gRow); the lanes of
// a warp are grouped by the cell their stencils are centred on, and for each
// group lanes 0..26 take the cell's 27 nodes, sum the group's rows and add the
// sums into the brick's 8^3 accumulation tile with shared-memory float
// reductions (p2gWarpGroups).  The item ends with one barrier and one vector
// reduction to global memory per non-zero node of the tile (p2gFlush).
constexpr int kRow = 9;         // float4 per input row: 3 axes x 3 offsets (see p2gRow)
constexpr int kTileNodes = 512; // 8^3
// A tile plane (one of mass, mom.x, mom.y, mom.z) stores node (x, y, z) at
// x + 11 y + 89 z: with strides 11 and 89 (3 and 25 modulo the 32 banks) the
// 27 nodes of any 3x3x3 stencil in the tile fall into 27 different banks, so
// a warp's shared-memory reductions over a stencil never conflict (with the
// dense 8 / 64 strides the three z-layers of a stencil share 9 banks).
constexpr int kTileSy = 11, kTileSz = 89;
constexpr int kTilePlane = 7 * kTileSz + 7 * kTileSy + 8;  // 708 floats
__device__ __forceinline__ int tileIndex(int x, int y, int z) { return x + kTileSy * y + kTileSz * z; }
constexpr uint32_t kNoKey = 0xFFFFFFFFu;  // a lane with no row for the warp's P2G

// Shared memory of the standalone P2G kernel.
struct P2GSmem {
  float4 rows[kThreads * kRow];  // P2G input rows; warp w owns rows [32 w, 32 w + 32)
  float tiles[4 * kTilePlane];   // the item's 8^3 accumulation tile
  float mass[kThreads];          // the particle mass of an exact-form row
  uint32_t item;
};

// Shared memory of the fused kernel (THREADS = the CTA size, 192 or 256).

template <bool FLIP, int THREADS>
struct FusedSmem {
  float4 rows[THREADS * kRow];  // P2G input rows; warp w owns rows [32 w, 32 w + 32)
  float tiles[4 * kTilePlane];  // the item's 8^3 accumulation tile (mass, mom.x, mom.y, mom.z planes; tileIndex)
  float mass[THREADS];          // the particle mass of an exact-form row
  float4 v[216];                // staged 6^3 node block (v, mass)
  float4 vo[FLIP ? 216 : 1];
  uint32_t markMask[2];         // grid-active marks of the item brick's 3^3 neighbour bricks, by item parity
  uint32_t items[2];            // claimed items by item parity
};

// P2G inputs of one particle in separable form.  The quadratic B-spline weight
// of node (dx,dy,dz) is W_x[dx] W_y[dy] W_z[dz], so the particle's momentum
// term  w (m v + m (4/h^2) B r) - dt Vp tau grad w  equals
//   W_y W_z A_x[dx] + W_x W_z A_y[dy] + W_x W_y A_z[dz]
// with, per axis c and offset d (r_c = x_i,c - x_p,c, G = N'/h):
//   A_c[d] = [c == x] m v W_c + (m 4/h^2 B)[:, c] W_c r_c - (dt Vp tau)[:, c] G_c
// and the mass term is m W_x W_y W_z.  The usual form folds the mass into the
// x factors:
//   row[d]     = (A_x[d],     m W_x[d])
//   row[3 + d] = (A_y[d] / m, W_y[d])
//   row[6 + d] = (A_z[d] / m, W_z[d])
// so a node term is  wyz X.xyz + (X.w Z.w) Y.xyz + (X.w Y.w) Z.xyz  and its
// mass X.w wyz: three vector loads, no per-particle scalar, and no weight
// test.  The shader skips a node whose weight is below 1e-12
// (mpm_p2g.comp:47); the smallest of the 27 weights is the product of the
// three axis minima, so when that product is below 1e-12 (0.15% of the slope
// scene's particles: near a cell face in all three axes, or very near one),
// or the mass is not positive, the row is written in the exact form instead,
// (A_c[d], W_c[d]) for every axis with the mass in `mass`, whose terms carry
// the shader's test (p2gNodeTermExact).  Returns true for the exact form.
__device__ __forceinline__ bool p2gRow(const SubstepParams& P, const PState& s, float dtStress, int cx, int cy, int cz, float4* row, float& m) {
  const float invH = 1.0f / P.cellSize;
  m = fetchRho0(P, __float_as_uint(s.v.w)) * s.P.w;
  const float av[3] = {m * s.v.x, m * s.v.y, m * s.v.z};
  float Q[3][3];  // GLSL [col][row]
  if (P.flip_ratio < -0.5f) {
    const float k = m * (4.0f / (P.cellSize * P.cellSize));
    Q[0][0] = k * s.B0.x; Q[0][1] = k * s.B0.y; Q[0][2] = k * s.B0.z;
    Q[1][0] = k * s.B1.x; Q[1][1] = k * s.B1.y; Q[1][2] = k * s.B1.z;
    Q[2][0] = k * s.B2.x; Q[2][1] = k * s.B2.y; Q[2][2] = k * s.B2.z;
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 3; ++q) Q[c][q] = 0.f;
  }
  const float sdt = dtStress * s.P.w;
  const float T[3][3] = {{sdt * s.F0.w, sdt * s.B0.w, sdt * s.B1.w},
                         {sdt * s.B0.w, sdt * s.F1.w, sdt * s.B2.w},
                         {sdt * s.B1.w, sdt * s.B2.w, sdt * s.F2.w}};
  const float xp[3] = {s.P.x, s.P.y, s.P.z};
  const int cc[3] = {cx, cy, cz};
  float xs[3][3], W[3][3], G[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float ds[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xs[c][d] = nodeCentre(P, c, cc[c] - 1 + d);
      ds[d] = (xp[c] - xs[c][d]) * invH;
    }
    bsplineStencil(ds[0], ds[1], ds[2], W[c], G[c]);
  }
  const float wmin = (fminf(W[0][0], fminf(W[0][1], W[0][2])) * fminf(W[1][0], fminf(W[1][1], W[1][2]))) * fminf(W[2][0], fminf(W[2][1], W[2][2]));
  const bool exact = !(m > 0.f && wmin >= 1e-12f);
  const float sx = exact ? 1.0f : m, sa = exact ? 1.0f : 1.0f / m;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float Wc = W[c][d], Gc = G[c][d] * invH;
      const float Rw = Wc * (xs[c][d] - xp[c]);
      float A[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) A[q] = (c == 0 ? av[q] * Wc : 0.f) + Q[c][q] * Rw - T[c][q] * Gc;
      if (c == 0) row[d] = make_float4(A[0], A[1], A[2], sx * Wc);
      else row[3 * c + d] = make_float4(A[0] * sa, A[1] * sa, A[2] * sa, Wc);
    }
  return exact;
}

// Contribution of a usual-form row's three factors to its stencil node.
__device__ __forceinline__ void p2gNodeTermXYZ(const float4 X, const float4 Y, const float4 Z, float acc[4]) {
  const float wyz = Y.w * Z.w;
  const float wxz = X.w * Z.w, wxy = X.w * Y.w;
  acc[0] += wyz * X.x + wxz * Y.x + wxy * Z.x;
  acc[1] += wyz * X.y + wxz * Y.y + wxy * Z.y;
  acc[2] += wyz * X.z + wxz * Y.z + wxy * Z.z;
  acc[3] += X.w * wyz;
}

// Contribution of a usual-form row to its stencil node (dx, dy, dz).
__device__ __forceinline__ void p2gNodeTerm(const float4* __restrict__ row, int dx, int dy, int dz, float acc[4]) {
  const float4 X = row[dx], Y = row[3 + dy], Z = row[6 + dz];
  const float wyz = Y.w * Z.w;
  const float wxz = X.w * Z.w, wxy = X.w * Y.w;
  acc[0] += wyz * X.x + wxz * Y.x + wxy * Z.x;
  acc[1] += wyz * X.y + wxz * Y.y + wxy * Z.y;
  acc[2] += wyz * X.z + wxz * Y.z + wxy * Z.z;
  acc[3] += X.w * wyz;
}

// Contribution of an exact-form row (mass m) to its stencil node, skipped
// below w = 1e-12.
__device__ __forceinline__ void p2gNodeTermExact(const float4* __restrict__ row, float m, int dx, int dy, int dz, float acc[4]) {
  const float4 X = row[dx], Y = row[3 + dy], Z = row[6 + dz];
  const float wyz = Y.w * Z.w;
  const float w = X.w * wyz;
  if (w < 1e-12f) return;
  const float wxz = X.w * Z.w, wxy = X.w * Y.w;
  acc[0] += wyz * X.x + wxz * Y.x + wxy * Z.x;
  acc[1] += wyz * X.y + wxz * Y.y + wxy * Z.y;
  acc[2] += wyz * X.z + wxz * Y.z + wxy * Z.z;
  acc[3] += w * m;
}

// Direct scatter of one row (either form) to global memory: particles whose
// stencil leaves the brick's block.
__device__ __noinline__ void p2gRowGlobal(const SubstepParams& P, const float4* row, float m, bool exact, int cx, int cy, int cz, float4* acc) {
  const int cr = int(P.cubeRes);
  for (int dz = 0; dz < 3; ++dz)
    for (int dy = 0; dy < 3; ++dy)
      for (int dx = 0; dx < 3; ++dx) {
        const int nx = cx + dx - 1, ny = cy + dy - 1, nz = cz + dz - 1;
        if (nx < 0 || ny < 0 || nz < 0 || nx >= cr || ny >= cr || nz >= cr) continue;
        float a[4] = {0.f, 0.f, 0.f, 0.f};
        if (exact) p2gNodeTermExact(row, m, dx, dy, dz, a);
        else p2gNodeTerm(row, dx, dy, dz, a);
        if (a[3] != 0.f || a[0] != 0.f || a[1] != 0.f || a[2] != 0.f) redAddV4(acc + mortonEncode(nx, ny, nz), a[0], a[1], a[2], a[3]);
      }
}

// Add every non-zero node of the tile to the global grid and leave the tile
// zeroed (each node is read and cleared by the one thread that owns it) for
// the CTA's next item.
template <class SM>
__device__ __forceinline__ void p2gFlush(const SubstepParams& P, SM& sm, int tx, int ty, int tz, float4* acc) {
  const int cr = int(P.cubeRes);
  for (int q = threadIdx.x; q < kTileNodes; q += blockDim.x) {
    float* t = sm.tiles + tileIndex(q & 7, (q >> 3) & 7, q >> 6);
    const float m = t[0], mx = t[kTilePlane], my = t[2 * kTilePlane], mz = t[3 * kTilePlane];
    t[0] = 0.f;
    t[kTilePlane] = 0.f;
    t[2 * kTilePlane] = 0.f;
    t[3 * kTilePlane] = 0.f;
    if (m == 0.f && mx == 0.f && my == 0.f && mz == 0.f) continue;
    const int nx = tx + (q & 7), ny = ty + ((q >> 3) & 7), nz = tz + (q >> 6);
    if (nx < 0 || ny < 0 || nz < 0 || nx >= cr || ny >= cr || nz >= cr) continue;
    redAddV4(acc + mortonEncode(nx, ny, nz), mx, my, mz, m);
  }
}

// G2P node source: the brick's 6^3 staged neighbourhood, global memory outside it.
template <bool FLIP>
struct StagedGrid {
  const float4* sv;
  const float4* svo;
  const float4* gvel;
  const float4* gvold;
  int ox, oy, oz;
  __device__ __forceinline__ bool node(int x, int y, int z, float& m, float3& v, float3& vo) const {
    const int lx = x - ox, ly = y - oy, lz = z - oz;
    float4 a, b = make_float4(0.f, 0.f, 0.f, 0.f);
    if ((unsigned)lx < 6u && (unsigned)ly < 6u && (unsigned)lz < 6u) {
      const int q = (lz * 6 + ly) * 6 + lx;
      a = sv[q];
      if (FLIP) b = svo[q];
    } else {
      const uint32_t c = mortonEncode(x, y, z);
      a = gvel[c];
      if (FLIP) b = gvold[c];
    }
    m = a.w;
    if (m < 1e-10f) return false;
    v = make_float3(a.x, a.y, a.z);
    vo = make_float3(b.x, b.y, b.z);
    return true;
  }
};

// A particle's stencil centre among the brick's 6^3 cells (block origin ox,
// oy, oz), packed as rx | ry << 3 | rz << 6, or -1.
__device__ __forceinline__ int cellPacked(int cx, int cy, int cz, int ox, int oy, int oz) {
  const int rx = cx - ox, ry = cy - oy, rz = cz - oz;
  if ((unsigned)rx < 6u && (unsigned)ry < 6u && (unsigned)rz < 6u) return rx | (ry << 3) | (rz << 6);
  return -1;
}

// ------------------------------------------------------------------ P2G over particle bricks (standalone)
// P2G of one warp's rows (written by the lanes holding a row, key = packed
// stencil-centre cell, kNoKey for none): the lanes of equal key form a group,
// and for each group lanes 0..26 take the cell's 27 stencil nodes, sum the
// group's rows (each read at a known address, no list to follow) and add the
// sums into the tile with shared-memory float reductions.  Warps do not wait
// for one another.
__device__ __forceinline__ void p2gWarpGroups(const SubstepParams& P, const float4* __restrict__ wrows, const float* __restrict__ wmass, float* tile,
                                              uint32_t key, uint32_t exactMask, int tx, int ty, int tz) {
  const int lane = threadIdx.x & 31;
  const int dx = lane % 3, dy = (lane / 3) % 3, dz = lane / 9;
  const int cr = int(P.cubeRes);
  // a tile wholly inside the grid needs no per-node bounds test
  const bool inside = tx >= 0 && ty >= 0 && tz >= 0 && tx + 8 <= cr && ty + 8 <= cr && tz + 8 <= cr;
  __syncwarp();  // the rows are visible to every lane
  uint32_t pending = __ballot_sync(0xffffffffu, key != kNoKey);
  while (pending) {
    const int leader = __ffs(pending) - 1;
    const uint32_t k = __shfl_sync(0xffffffffu, key, leader);
    const uint32_t peers = __ballot_sync(0xffffffffu, key == k);
    pending &= ~peers;
    const int lx = int(k & 7u) + dx, ly = int((k >> 3) & 7u) + dy, lz = int(k >> 6) + dz;  // tile-local node
    const int nx = tx + lx, ny = ty + ly, nz = tz + lz;
    if (lane < 27 && (inside || (nx >= 0 && ny >= 0 && nz >= 0 && nx < cr && ny < cr && nz < cr))) {
      float a[4] = {0.f, 0.f, 0.f, 0.f};
      if (!(peers & exactMask)) {
        // usual-form rows: two per step, loads of both issued before their sums
        uint32_t m = peers;
        while (m) {
          const int j0 = __ffs(m) - 1;
          m &= m - 1u;
          const int j1 = m ? __ffs(m) - 1 : -1;
          m &= m - 1u;
          const float4* r0 = wrows + j0 * kRow;
          const float4 X0 = r0[dx], Y0 = r0[3 + dy], Z0 = r0[6 + dz];
          float4 X1 = make_float4(0.f, 0.f, 0.f, 0.f), Y1 = X1, Z1 = X1;
          if (j1 >= 0) {
            const float4* r1 = wrows + j1 * kRow;
            X1 = r1[dx]; Y1 = r1[3 + dy]; Z1 = r1[6 + dz];
          }
          p2gNodeTermXYZ(X0, Y0, Z0, a);
          p2gNodeTermXYZ(X1, Y1, Z1, a);  // a missing second row adds zeros
        }
      } else {
        uint32_t m = peers;
        while (m) {
          const int j = __ffs(m) - 1;
          m &= m - 1u;
          if ((exactMask >> j) & 1u) p2gNodeTermExact(wrows + j * kRow, wmass[j], dx, dy, dz, a);
          else p2gNodeTerm(wrows + j * kRow, dx, dy, dz, a);
        }
      }
      const int t = tileIndex(lx, ly, lz);
      atomicAdd(tile + t, a[3]);
      atomicAdd(tile + kTilePlane + t, a[0]);
      atomicAdd(tile + 2 * kTilePlane + t, a[1]);
      atomicAdd(tile + 3 * kTilePlane + t, a[2]);
    }
  }
  __syncwarp();  // every lane has read the rows before they are written again
}

// P2G of the particles in sorted slots [start, end) of brick `b` (the scene's
// own brick id): warps take rounds of 32 slots, each lane writes its
// particle's row, each warp adds its groups into the tile; one barrier, then
// the flush.
__device__ __forceinline__ void p2gBrickItem(const SubstepParams& P, P2GSmem& sm, uint32_t b, uint32_t start, uint32_t end, StatePtrs cur,
                                             uint32_t n, const BrickBuffers& B, const GridBuffers& G, float dtStress) {
  int bx, by, bz;
  mortonDecode(b, bx, by, bz);
  const int tx = 4 * bx - 2, ty = 4 * by - 2, tz = 4 * bz - 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* wrows = sm.rows + warp * 32 * kRow;
  float* wmass = sm.mass + warp * 32;
#pragma unroll 1
  for (uint32_t t0 = start + uint32_t(warp) * 32u; t0 < end; t0 += kThreads) {
    const uint32_t t = t0 + uint32_t(lane);
    uint32_t key = kNoKey;
    bool exact = false;
    if (t < end) {
      const uint32_t s = B.perm[t];
      if (s < n) {
        const PState st = loadState(cur.f, s);
        int cx, cy, cz;
        cellCoords(P, st.P.x, st.P.y, st.P.z, cx, cy, cz);
        float m;
        exact = p2gRow(P, st, dtStress, cx, cy, cz, wrows + lane * kRow, m);
        wmass[lane] = m;
        const int pk = cellPacked(cx, cy, cz, tx + 1, ty + 1, tz + 1);
        if (pk >= 0) key = uint32_t(pk);
        else p2gRowGlobal(P, wrows + lane * kRow, m, exact, cx, cy, cz, G.acc);
      }
    }
    p2gWarpGroups(P, wrows, wmass, sm.tiles, key, __ballot_sync(0xffffffffu, exact), tx, ty, tz);
  }
  __syncthreads();  // the tile is complete
  p2gFlush(P, sm, tx, ty, tz, G.acc);
}

template <bool BATCH>
__global__ void __launch_bounds__(kThreads) k_p2g_bricks(SubstepParams P0, SceneTable T, StatePtrs cur, uint32_t n, BrickBuffers B,
                                                         GridBuffers G, float dtStress) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  P2GSmem& sm = *reinterpret_cast<P2GSmem*>(smem_raw);
  const uint32_t numPB = B.counters[kCntNumPB];
  // the tile starts zeroed here and is left so by every item's flush
  for (int q = threadIdx.x; q < 4 * kTilePlane; q += blockDim.x) sm.tiles[q] = 0.f;
  for (;;) {
    if (threadIdx.x == 0) sm.item = atomicAdd(B.counters + kCntQueueP2G, 1u);
    __syncthreads();
    const uint32_t i = sm.item;
    if (i >= numPB) break;
    const uint32_t b = B.pbBrick[i], end = min(B.pbStart[i + 1], n), start = min(B.pbStart[i], end);
    if constexpr (BATCH) {
      __shared__ SubstepParams sP;
      __shared__ uint32_t sBase;
      if (threadIdx.x < 32) {
        const uint32_t sc = findScene(T.brickBase, T.count, b);
        copyParams(&sP, T.params + sc, threadIdx.x, 32);
        if (threadIdx.x == 0) sBase = T.brickBase[sc];
      }
      __syncthreads();
      p2gBrickItem(sP, sm, b - sBase, start, end, cur, n, B, offsetGrid(G, sBase), sP.dt);
    } else {
      p2gBrickItem(P0, sm, b, start, end, cur, n, B, G, dtStress);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ sparse grid update
// Per thread, kGridBatch nodes per round (2 or 4, picked by the launch
// configuration): their brick ids, then their accumulators (and an L1
// prefetch of their SDF samples) are loaded before any node is updated, so
// one round costs about the memory round trips of one node.
// The kernel also scatters the permutation of the binning that precedes it
// (the scan's brick starts, the fused kernel's keys and ranks) when n > 0:
// the grid update does not read it and the next fused kernel does, so the
// scatter needs no launch of its own.  Scattering the same binning twice
// writes the same values.
template <int kGridBatch>
__global__ void __launch_bounds__(kThreads) k_grid_bricks(SubstepParams P, BrickBuffers B, GridBuffers G, uint32_t n, uint32_t* err) {
  waitForPredecessorGrid();
  const uint64_t total = uint64_t(B.counters[kCntNumGB]) * 64u;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  permScatterStrided(B, n, err, uint64_t(blockIdx.x) * blockDim.x + threadIdx.x, stride);
  for (uint64_t g0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g0 < total; g0 += stride * kGridBatch) {
    uint32_t code[kGridBatch];
    bool live[kGridBatch];
#pragma unroll
    for (int k = 0; k < kGridBatch; ++k) {
      const uint64_t g = g0 + uint64_t(k) * stride;
      live[k] = g < total;
      code[k] = live[k] ? ((B.gbBrick[g >> 6] << 6) | uint32_t(g & 63u)) : 0u;
      live[k] = live[k] && code[k] < P.hashCells;
    }
    float4 a[kGridBatch];
#pragma unroll
    for (int k = 0; k < kGridBatch; ++k) {
      a[k] = live[k] ? G.acc[code[k]] : make_float4(0.f, 0.f, 0.f, 0.f);
      if (live[k] && P.sdf) {
        // the node's SDF sample and its six neighbours (read when the node is
        // within 1.5 h of the surface): the second read hits L1 (-7% per launch)
        int ix, iy, iz;
        mortonDecode(code[k], ix, iy, iz);
        const int cm = int(P.cubeRes) - 1;
        const float* f = P.sdf;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + code[k]));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(min(ix + 1, cm), iy, iz)));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(max(ix - 1, 0), iy, iz)));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(ix, min(iy + 1, cm), iz)));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(ix, max(iy - 1, 0), iz)));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(ix, iy, min(iz + 1, cm))));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(f + mortonEncode(ix, iy, max(iz - 1, 0))));
      }
    }
#pragma unroll
    for (int k = 0; k < kGridBatch; ++k) {
      if (!live[k]) continue;
      const uint32_t c = code[k];
      G.acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
      int ix, iy, iz;
      mortonDecode(c, ix, iy, iz);
      float3 v, vo;
      const bool ok = gridNode(P, ix, iy, iz, a[k].w, a[k].x, a[k].y, a[k].z, v, vo);
      G.vel[c] = ok ? make_float4(v.x, v.y, v.z, a[k].w) : make_float4(0.f, 0.f, 0.f, a[k].w);
      if (G.vold) G.vold[c] = ok ? make_float4(vo.x, vo.y, vo.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

// Batched grid update: one warp per listed grid brick, two nodes per lane, the
// brick's scene parameters in a warp-private shared copy.
// Also scatters the permutation of the preceding binning (as k_grid_bricks).
__global__ void __launch_bounds__(kThreads) k_grid_bricks_batch(SceneTable T, uint32_t substep, BrickBuffers B, GridBuffers G, uint32_t n,
                                                                uint32_t* err) {
  __shared__ SubstepParams sP[kThreads / 32];
  waitForPredecessorGrid();
  permScatterStrided(B, n, err, uint64_t(blockIdx.x) * blockDim.x + threadIdx.x, uint64_t(gridDim.x) * blockDim.x);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t numGB = B.counters[kCntNumGB];
  // Each warp takes a contiguous run of the (ascending) grid-brick list, so
  // consecutive bricks mostly share a scene: the scene is searched once and
  // then advanced, and its parameters are copied only when it changes.
  const uint32_t warps = gridDim.x * (kThreads / 32), gw = blockIdx.x * (kThreads / 32) + warp;
  const uint32_t per = (numGB + warps - 1) / warps;
  const uint32_t g0 = min(gw * per, numGB), g1 = min(g0 + per, numGB);
  uint32_t sc = g0 < g1 ? findScene(T.brickBase, T.count, B.gbBrick[g0]) : 0u;
  uint32_t loaded = 0xFFFFFFFFu;
  for (uint32_t gb = g0; gb < g1; ++gb) {
    const uint32_t bg = B.gbBrick[gb];
    // k_brick_scan lists grid bricks in ascending order, so the scene only
    // moves forward; a brick below the current scene's base (a list built
    // otherwise) is searched for again instead of taking the wrong scene
    if (bg < T.brickBase[sc]) sc = findScene(T.brickBase, T.count, bg);
    while (sc + 1u < T.count && T.brickBase[sc + 1u] <= bg) ++sc;
    const uint32_t base = T.brickBase[sc];
    if (sc != loaded) {
      __syncwarp();
      copyParams(&sP[warp], T.params + sc, lane, 32);
      __syncwarp();
      if (lane == 0) sP[warp].colliders += size_t(substep) * sP[warp].colliderCount;
      __syncwarp();
      loaded = sc;
    }
    const SubstepParams& P = sP[warp];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t sub = uint32_t(lane + 32 * h);
      const uint32_t local = ((bg - base) << 6) | sub;
      if (local >= P.hashCells) continue;
      const size_t code = (size_t(bg) << 6) | sub;
      const float4 a = G.acc[code];
      G.acc[code] = make_float4(0.f, 0.f, 0.f, 0.f);
      int ix, iy, iz;
      mortonDecode(local, ix, iy, iz);
      float3 v, vo;
      const bool ok = gridNode(P, ix, iy, iz, a.w, a.x, a.y, a.z, v, vo);
      G.vel[code] = ok ? make_float4(v.x, v.y, v.z, a.w) : make_float4(0.f, 0.f, 0.f, a.w);
      if (G.vold) G.vold[code] = ok ? make_float4(vo.x, vo.y, vo.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_clear_bricks(BrickBuffers B, GridBuffers G) {
  const uint64_t total = uint64_t(B.counters[kCntNumGB]) * 64u;
  for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t code = (B.gbBrick[g >> 6] << 6) | uint32_t(g & 63u);
    G.acc[code] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// ------------------------------------------------------------------ fused G2P -> update -> P2G
// One work item: the sorted slots [start, end) of particle brick `b` (the
// scene's own brick id).  The binning orders a brick's particles by cell
// (the brick's 64 cells in Morton order), so a warp's 32 consecutive slots
// hold the particles of a few neighbouring cells: the G2P reads of the staged
// 6^3 block are mostly broadcasts, the binning counts group into a few runs,
// and the warp's P2G groups its lanes by stencil-centre cell
// (p2gWarpGroups).  Per particle: G2P from the staged grid, particle update,
// write to its slot in the next buffer, binning count under the global cell
// key 64 brickBase + Morton code, stencil brick marks, and P2G into the
// item's tile.  Warps take the item's rounds of 32 slots without waiting for
// one another; the item ends with one barrier and the tile flush (one vector
// reduction per non-zero node).  `mp` selects the item's marks.
template <bool FLIP, int THREADS, int MS>
__device__ __forceinline__ void g2p2gPart(const SubstepParams& P, FusedSmem<FLIP, THREADS>& S, uint32_t b, uint32_t start, uint32_t end,
                                          uint32_t brickBase, StatePtrs cur, const uint32_t* __restrict__ pidCur, StatePtrs nxt,
                                          uint32_t* __restrict__ pidNxt, uint32_t n, const BrickBuffers& B, const GridBuffers& G, float dtStress,
                                          uint32_t* err, uint32_t mp) {
  int bx, by, bz;
  mortonDecode(b, bx, by, bz);
  // stage the 6^3 nodes [4b-1, 4b+4]^3 (nodes outside [0, gridRes) read as empty)
  const int sx = 4 * bx - 1, sy = 4 * by - 1, sz = 4 * bz - 1;
  for (int q = threadIdx.x; q < 216; q += THREADS) {
    const int x = sx + q % 6, y = sy + (q / 6) % 6, z = sz + q / 36;
    const bool valid = x >= 0 && y >= 0 && z >= 0 && x < P.gridRes[0] && y < P.gridRes[1] && z < P.gridRes[2];
    const uint32_t c = valid ? mortonEncode(x, y, z) : 0u;
    float4 v = valid ? G.vel[c] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool live = v.w >= 1e-10f;  // the nodes the shader gathers from
    if (!live) v = make_float4(0.f, 0.f, 0.f, v.w);
    S.v[q] = v;
    if (FLIP) S.vo[q] = live ? G.vold[c] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const StagedGrid<FLIP> grid{S.v, S.vo, G.vel, G.vold, sx, sy, sz};
  const int tx = sx - 1, ty = sy - 1, tz = sz - 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* wrows = S.rows + warp * 32 * kRow;
  float* wmass = S.mass + warp * 32;
  const uint32_t cellBase = brickBase << 6;
  uint32_t marks = 0;
#pragma unroll 1
  for (uint32_t t0 = start + uint32_t(warp) * 32u; t0 < end; t0 += THREADS) {
    const uint32_t t = t0 + uint32_t(lane);  // the particle's slot in the next buffer
    const bool act = t < end;
    const uint32_t mask = __ballot_sync(0xffffffffu, act);
    uint32_t key = kNoKey;
    bool exact = false;
    GroupTicket ticket{0u, 0u};
    if (act) {
      const uint32_t s = B.perm[t];
      const bool valid = s < n;
      PState st;
      int cx = 0, cy = 0, cz = 0;
      uint32_t nc = 0;
      if (valid) {
        st = loadState(cur.f, s);
        const uint32_t pid = pidCur[s];
        float vpic[3], vpo[3], Gv[3][3], Bn[3][3];
        if (!g2pGatherStaged<FLIP>(P, st, S.v, S.vo, sx, sy, sz, vpic, vpo, Gv, Bn)) g2pGather(P, st, grid, vpic, vpo, Gv, Bn);
        g2pUpdate<MS>(P, st, P.dt, vpic, vpo, Gv, Bn);
        storeState(nxt.f, t, st);
        pidNxt[t] = pid;
        if (!(isfinite(st.P.x) && isfinite(st.P.y) && isfinite(st.P.z))) atomicOr(err, kErrNonFinite);
        cellCoords(P, st.P.x, st.P.y, st.P.z, cx, cy, cz);
        nc = cellBase + mortonEncode(cx, cy, cz);
      } else {
        atomicOr(err, kErrBinRange);  // a slot that maps nowhere: only after an expired scan wait
      }
      // every active lane reaches these call sites
      ticket = warpGroupClaim(mask, B.cellCount, nc);
      B.binKey[t] = nc;
      warpGroupAdd(mask, B.brickCount, nc >> 6);
      if (valid) {
        if (!stencilBrickMask(P, cx, cy, cz, bx, by, bz, marks)) markStencilBricks(P, cx, cy, cz, B.brickFlag + brickBase);
        float m;
        exact = p2gRow(P, st, dtStress, cx, cy, cz, wrows + lane * kRow, m);
        wmass[lane] = m;
        const int pk = cellPacked(cx, cy, cz, sx, sy, sz);
        if (pk >= 0) {
          key = uint32_t(pk);
        } else {
          p2gRowGlobal(P, wrows + lane * kRow, m, exact, cx, cy, cz, G.acc);
          atomicAdd(B.counters + kCntOverflow, 1u);
        }
      }
    }
    p2gWarpGroups(P, wrows, wmass, S.tiles, key, __ballot_sync(0xffffffffu, exact), tx, ty, tz);
    if (act) B.binRank[t] = warpGroupRank(mask, ticket);  // the count's atomic has returned by now
  }
  marks = __reduce_or_sync(0xffffffffu, marks);
  if (lane == 0 && marks) atomicOr(&S.markMask[mp], marks);
  __syncthreads();  // the tile and the marks are complete
  flushBrickMarks(P, S.markMask[mp], bx, by, bz, B.brickFlag + brickBase);
  p2gFlush(P, S, tx, ty, tz, G.acc);
}

// Persistent CTAs pull work items from the queue: item i is part i / numPB of
// particle brick i % numPB, whose sorted slots are cut into `split`
// contiguous parts of near-equal size (empty parts are skipped).  split = 1
// keeps a brick in one CTA (one staging and one tile flush per brick); more
// parts shorten the longest item, which bounds small scenes.  768 / THREADS
// CTAs per SM (4 of 192 threads, 3 of 256): 80 registers with some spills to
// L1-cached local memory.  MS: the material-model set compiled in.
template <bool FLIP, bool BATCH, int THREADS, int MS>
__global__ void __launch_bounds__(THREADS, 768 / THREADS) k_g2p2g(SubstepParams P0, SceneTable T, StatePtrs cur, const uint32_t* __restrict__ pidCur,
                                                      StatePtrs nxt, uint32_t* __restrict__ pidNxt, uint32_t n, BrickBuffers B, GridBuffers G,
                                                      float dtStress, uint32_t* err, uint32_t split) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FusedSmem<FLIP, THREADS>& S = *reinterpret_cast<FusedSmem<FLIP, THREADS>*>(smem_raw);
  waitForPredecessorGrid();
  const uint32_t numPB = B.counters[kCntNumPB];
  const uint32_t numItems = numPB * split;
  // The tile starts zeroed here and is left so by every item's flush.
  for (int q = threadIdx.x; q < 4 * kTilePlane; q += THREADS) S.tiles[q] = 0.f;
  // the claim alternates between two slots: a thread may claim the next item
  // while others still read this one, never two ahead (one barrier per claim)
  for (uint32_t it = 0;; it ^= 1u) {
    if (threadIdx.x == 0) {
      S.items[it] = atomicAdd(B.counters + kCntQueueFused, 1u);
      S.markMask[it] = 0u;  // last read by the item two back, before the previous claim's barrier
    }
    __syncthreads();
    const uint32_t i = S.items[it];
    if (i >= numItems) break;
    const uint32_t part = i / numPB, bi = i - part * numPB;
    const uint32_t b = B.pbBrick[bi], bend = min(B.pbStart[bi + 1], n), bstart = min(B.pbStart[bi], bend);
    // the permutation has read the previous binning's counts of this brick:
    // clear them for the binning after this one (every part writes the same zeros)
    if (threadIdx.x < 32) reinterpret_cast<uint2*>(B.cellPrev + (size_t(b) << 6))[threadIdx.x] = make_uint2(0u, 0u);
    const uint32_t len = (bend - bstart + split - 1u) / split;
    const uint32_t start = min(bstart + part * len, bend), end = min(start + len, bend);
    if (start >= end) continue;  // the brick has no particles for this part
    if constexpr (BATCH) {
      __shared__ SubstepParams sP;
      __shared__ uint32_t sBase;
      if (threadIdx.x < 32) {
        const uint32_t sc = findScene(T.brickBase, T.count, b);
        copyParams(&sP, T.params + sc, threadIdx.x, 32);
        if (threadIdx.x == 0) sBase = T.brickBase[sc];
      }
      __syncthreads();
      const uint32_t base = sBase;
      g2p2gPart<FLIP, THREADS, MS>(sP, S, b - base, start, end, base, cur, pidCur, nxt, pidNxt, n, B, offsetGrid(G, base), sP.dt, err, it);
    } else {
      g2p2gPart<FLIP, THREADS, MS>(P0, S, b, start, end, 0u, cur, pidCur, nxt, pidNxt, n, B, G, dtStress, err, it);
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_unpermute(StatePtrs in, const uint32_t* __restrict__ pid, StatePtrs out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t d = pid[i];
  if (d >= n) return;
#pragma unroll
  for (int k = 0; k < 8; ++k) out.f[k][d] = in.f[k][i];
}

__global__ void __launch_bounds__(kThreads) k_sorted_pid(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ pid, uint32_t* out,
                                                         uint32_t n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t s = perm[t];
  out[t] = s < n ? pid[s] : 0xffffffffu;
}

__global__ void __launch_bounds__(kThreads) k_iota(uint32_t* pid, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pid[i] = i;
}

template <class K> int ctasPerSm(K kernel, int threads, size_t smem = 0) {
  int perSM = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, threads, smem) != cudaSuccess || perSM < 1) perSM = 1;
  return perSM;
}

template <class K> int bigSmemCtasPerSm(K kernel, int threads, size_t smem) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  return ctasPerSm(kernel, threads, smem);
}

// Most CTAs per SM of every kernel variant, resolved once per device (kernel
// attributes are per device; the queries stay outside stream capture).
struct LaunchShapes {
  std::atomic<bool> ready{false};
  int p2g[2] = {0, 0};                          // [BATCH]
  int grid[2] = {0, 0};                         // [gridBatch == 4]
  int gridBatch = 0;                            // batched grid kernel
  int fused[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};  // [FLIP][BATCH][THREADS == 256]
};
constexpr int kShapeSlots = 64;  // device ordinals beyond this share slots modulo 64
LaunchShapes g_shapes[kShapeSlots];
std::mutex g_shapesMutex;

template <bool FLIP, bool BATCH, int THREADS, int MS> void setupFused(LaunchShapes& L) {
  // every model set of one shape has the same shared memory and register bound
  L.fused[FLIP][BATCH][THREADS == 256] = bigSmemCtasPerSm(k_g2p2g<FLIP, BATCH, THREADS, MS>, THREADS, sizeof(FusedSmem<FLIP, THREADS>));
}
template <int THREADS> void setupFusedShape(LaunchShapes& L) {
  setupFused<false, false, THREADS, kModelsElastic>(L);
  setupFused<false, false, THREADS, kModelsDruckerPrager>(L);
  setupFused<false, false, THREADS, kModelsElasticVonMises>(L);
  setupFused<false, false, THREADS, kModelsElasticDruckerPrager>(L);
  setupFused<false, false, THREADS, kModelsAny>(L);
  setupFused<false, true, THREADS, kModelsElasticVonMises>(L);
  setupFused<false, true, THREADS, kModelsAny>(L);
  setupFused<true, false, THREADS, kModelsAny>(L);
  setupFused<true, true, THREADS, kModelsAny>(L);
}

const LaunchShapes& shapes() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  LaunchShapes& L = g_shapes[dev % kShapeSlots];
  if (L.ready.load(std::memory_order_acquire)) return L;
  std::lock_guard<std::mutex> lock(g_shapesMutex);
  if (L.ready.load(std::memory_order_relaxed)) return L;
  L.p2g[0] = bigSmemCtasPerSm(k_p2g_bricks<false>, kThreads, sizeof(P2GSmem));
  L.p2g[1] = bigSmemCtasPerSm(k_p2g_bricks<true>, kThreads, sizeof(P2GSmem));
  L.grid[0] = ctasPerSm(k_grid_bricks<2>, kThreads);
  L.grid[1] = ctasPerSm(k_grid_bricks<4>, kThreads);
  L.gridBatch = ctasPerSm(k_grid_bricks_batch, kThreads);
  setupFusedShape<192>(L);
  setupFusedShape<256>(L);
  L.ready.store(true, std::memory_order_release);
  return L;
}

// Blocks of a persistent launch: the requested CTAs per SM (0 = most that fit), capped by occupancy.
int persistentGrid(uint32_t requested, int most, int numSMs) {
  const int per = requested == 0 ? most : std::min(int(requested), most);
  return std::max(per, 1) * numSMs;
}

}  // namespace

LaunchLimits launchLimits(bool flip, bool batch) {
  const LaunchShapes& L = shapes();
  LaunchLimits out;
  out.fusedCtasPerSm[0] = uint32_t(L.fused[flip][batch][0]);
  out.fusedCtasPerSm[1] = uint32_t(L.fused[flip][batch][1]);
  out.gridCtasPerSm[0] = uint32_t(L.grid[0]);
  out.gridCtasPerSm[1] = uint32_t(L.grid[1]);
  return out;
}

cudaError_t probeWaitExpiry(uint32_t* errorBits) {
  unsigned long long* st = nullptr;
  uint32_t* err = nullptr;
  cudaError_t e = cudaMalloc(&st, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(st, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(uint32_t));
  if (e == cudaSuccess) {
    k_wait_expiry_probe<<<1, 32>>>(st, err);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(errorBits, err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(st);
  cudaFree(err);
  return e;
}

void prepareBrickKernels(int numSMs) {
  (void)numSMs;
  (void)shapes();
}

cudaError_t launchBrickCount(const SubstepParams& P, const float4* pos, uint32_t n, const BrickBuffers& b, uint32_t* err, cudaStream_t s,
                             uint64_t* launches) {
  (void)err;
  if (n == 0) return cudaSuccess;
  k_brick_count<false><<<blocksFor(n), kThreads, 0, s>>>(P, SceneTable{}, pos, n, b);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchBrickCountBatch(const SceneTable& T, const float4* pos, uint32_t n, const BrickBuffers& b, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_brick_count<true><<<blocksFor(n), kThreads, 0, s>>>(SubstepParams{}, T, pos, n, b);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchBrickScan(const BrickBuffers& b, uint32_t* err, cudaStream_t s, uint64_t* launches) {
  const cudaError_t e = launchSerialized(k_brick_scan, dim3(b.tiles), dim3(kBrickScanThreads), 0, s, b, err);
  ++*launches;
  return e;
}

cudaError_t launchPermScatter(const BrickBuffers& b, uint32_t n, uint32_t* err, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  const cudaError_t e = launchSerialized(k_perm_scatter, dim3(blocksFor(n, kThreads * kPermRounds)), dim3(kThreads), 0, s, b, n, err);
  ++*launches;
  return e;
}

cudaError_t launchP2GBricks(const SubstepParams& P, StatePtrs cur, uint32_t n, const BrickBuffers& b, GridBuffers g, float dtStress,
                            int numSMs, cudaStream_t s, uint64_t* launches) {
  k_p2g_bricks<false><<<shapes().p2g[0] * numSMs, kThreads, sizeof(P2GSmem), s>>>(P, SceneTable{}, cur, n, b, g, dtStress);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchP2GBricksBatch(const SceneTable& T, StatePtrs cur, uint32_t n, const BrickBuffers& b, GridBuffers g, int numSMs,
                                 cudaStream_t s, uint64_t* launches) {
  k_p2g_bricks<true><<<shapes().p2g[1] * numSMs, kThreads, sizeof(P2GSmem), s>>>(SubstepParams{}, T, cur, n, b, g, 0.f);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchGridBricks(const SubstepParams& P, const BrickBuffers& b, GridBuffers g, uint32_t n, uint32_t* err, const LaunchConfig& lc,
                             int numSMs, cudaStream_t s, uint64_t* launches) {
  const LaunchShapes& L = shapes();
  const cudaError_t e = lc.gridBatch == 2
                            ? launchSerialized(k_grid_bricks<2>, dim3(persistentGrid(lc.gridCtasPerSm, L.grid[0], numSMs)), dim3(kThreads), 0, s,
                                               P, b, g, n, err)
                            : launchSerialized(k_grid_bricks<4>, dim3(persistentGrid(lc.gridCtasPerSm, L.grid[1], numSMs)), dim3(kThreads), 0, s,
                                               P, b, g, n, err);
  ++*launches;
  return e;
}

cudaError_t launchGridBricksBatch(const SceneTable& T, uint32_t substep, const BrickBuffers& b, GridBuffers g, uint32_t n, uint32_t* err,
                                  const LaunchConfig& lc, int numSMs, cudaStream_t s, uint64_t* launches) {
  const cudaError_t e = launchSerialized(k_grid_bricks_batch, dim3(persistentGrid(lc.gridCtasPerSm, shapes().gridBatch, numSMs)), dim3(kThreads), 0,
                                         s, T, substep, b, g, n, err);
  ++*launches;
  return e;
}

cudaError_t launchClearBricks(const BrickBuffers& b, GridBuffers g, int numSMs, cudaStream_t s, uint64_t* launches) {
  k_clear_bricks<<<numSMs * 4, kThreads, 0, s>>>(b, g);
  ++*launches;
  return cudaGetLastError();
}

namespace {

template <bool FLIP, bool BATCH, int THREADS, int MS>
cudaError_t launchFused(const SubstepParams& P, const SceneTable& T, StatePtrs cur, const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt,
                        uint32_t n, const BrickBuffers& b, GridBuffers g, float dtStress, uint32_t* err, uint32_t ctasPerSm, uint32_t split,
                        int numSMs, cudaStream_t s) {
  const int blocks = persistentGrid(ctasPerSm, shapes().fused[FLIP][BATCH][THREADS == 256], numSMs);
  return launchSerialized(k_g2p2g<FLIP, BATCH, THREADS, MS>, dim3(blocks), dim3(THREADS), sizeof(FusedSmem<FLIP, THREADS>), s, P, T, cur, pidCur,
                          nxt, pidNxt, n, b, g, dtStress, err, split);
}

// The instantiation for the launch shape and the model set: model-specialised
// kernels exist for APIC or PIC transfer (batches: the elastic / Von Mises set).
template <bool BATCH, int THREADS>
cudaError_t launchFusedShape(bool flip, int modelSet, const LaunchConfig& lc, const SubstepParams& P, const SceneTable& T, StatePtrs cur,
                             const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt, uint32_t n, const BrickBuffers& b, GridBuffers g,
                             float dtStress, uint32_t* err, int numSMs, cudaStream_t s) {
  // parts per brick by scene size when not set: scenes of up to 2^16 particles
  // have too few bricks to fill the GPU with one item per brick (50,000
  // particles on 64^3: 40.8 us per substep with two parts, 51.9 with one),
  // larger ones lose to the second staging and flush (80,000 particles: 71.6 /
  // 95.8 us; 1M: 292 / 390 us per launch)
  const uint32_t k = lc.fusedCtasPerSm, sp = lc.fusedSplit ? lc.fusedSplit : (n <= (1u << 16) ? 2u : 1u);
  if (flip) return launchFused<true, BATCH, THREADS, kModelsAny>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs, s);
  if (modelSet == kModelsElasticVonMises)
    return launchFused<false, BATCH, THREADS, kModelsElasticVonMises>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs, s);
  if constexpr (!BATCH) {
    if (modelSet == kModelsElastic)
      return launchFused<false, false, THREADS, kModelsElastic>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs, s);
    if (modelSet == kModelsDruckerPrager)
      return launchFused<false, false, THREADS, kModelsDruckerPrager>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs, s);
    if (modelSet == kModelsElasticDruckerPrager)
      return launchFused<false, false, THREADS, kModelsElasticDruckerPrager>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs,
                                                                              s);
  }
  return launchFused<false, BATCH, THREADS, kModelsAny>(P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, k, sp, numSMs, s);
}

template <bool BATCH>
cudaError_t launchFusedFor(bool flip, int modelSet, const LaunchConfig& lc, const SubstepParams& P, const SceneTable& T, StatePtrs cur,
                           const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt, uint32_t n, const BrickBuffers& b, GridBuffers g, float dtStress,
                           uint32_t* err, int numSMs, cudaStream_t s) {
  // CTA size by scene size when not set: 192 threads between 2^16 and 2^19
  // particles (80,000-particle mix: 65.2 against 70.0 us per substep), 256
  // otherwise (50,000 particles: 39.3 against 45.3; 1M: 292 against 296)
  const uint32_t threads = lc.fusedThreads ? lc.fusedThreads : (n > (1u << 16) && n < (1u << 19) ? 192u : 256u);
  if (threads == 192)
    return launchFusedShape<BATCH, 192>(flip, modelSet, lc, P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, numSMs, s);
  return launchFusedShape<BATCH, 256>(flip, modelSet, lc, P, T, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, numSMs, s);
}

}  // namespace

int modelSetOf(const Material* mats, uint32_t count) {
  bool elastic = count > 0, dp = count > 0, evm = count > 0, edp = count > 0;
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t m = mats[i].model;
    const bool isDp = m == MAT_DRUCKER_PRAGER || m == MAT_GRANULAR_POWDER;
    elastic = elastic && m == MAT_ELASTIC;
    dp = dp && isDp;
    evm = evm && (m == MAT_ELASTIC || m == MAT_VON_MISES);
    edp = edp && (m == MAT_ELASTIC || isDp);
  }
  return elastic ? kModelsElastic : dp ? kModelsDruckerPrager : evm ? kModelsElasticVonMises : edp ? kModelsElasticDruckerPrager : kModelsAny;
}

cudaError_t launchG2P2G(const SubstepParams& P, int modelSet, StatePtrs cur, const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt, uint32_t n,
                        const BrickBuffers& b, GridBuffers g, float dtStress, uint32_t* err, const LaunchConfig& lc, int numSMs, cudaStream_t s,
                        uint64_t* launches) {
  const cudaError_t e =
      launchFusedFor<false>(P.flip_ratio > 0.01f, modelSet, lc, P, SceneTable{}, cur, pidCur, nxt, pidNxt, n, b, g, dtStress, err, numSMs, s);
  ++*launches;
  return e;
}

cudaError_t launchG2P2GBatch(const SceneTable& T, int modelSet, bool flip, StatePtrs cur, const uint32_t* pidCur, StatePtrs nxt, uint32_t* pidNxt,
                             uint32_t n, const BrickBuffers& b, GridBuffers g, uint32_t* err, const LaunchConfig& lc, int numSMs, cudaStream_t s,
                             uint64_t* launches) {
  const cudaError_t e = launchFusedFor<true>(flip, modelSet == kModelsElasticVonMises || modelSet == kModelsElastic ? kModelsElasticVonMises : kModelsAny,
                                             lc, SubstepParams{}, T, cur, pidCur, nxt, pidNxt, n, b, g, 0.f, err, numSMs, s);
  ++*launches;
  return e;
}

cudaError_t launchUnpermute(StatePtrs in, const uint32_t* pid, StatePtrs out, uint32_t n, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_unpermute<<<blocksFor(n), kThreads, 0, s>>>(in, pid, out, n);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchSortedPid(const uint32_t* perm, const uint32_t* pid, uint32_t* out, uint32_t n, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_sorted_pid<<<blocksFor(n), kThreads, 0, s>>>(perm, pid, out, n);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchIota(uint32_t* pid, uint32_t n, cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_iota<<<blocksFor(n), kThreads, 0, s>>>(pid, n);
  ++*launches;
  return cudaGetLastError();
}

}  // namespace nebula
