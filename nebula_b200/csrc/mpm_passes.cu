// mpm_passes.cu -- single-pass kernels on the reference's dense grid layout.
//
// These run one reference dispatch each (binning, P2G, grid update + SDF
// boundary, G2P) on gridMom (float4 x 2 hashCells: [0,NC) momentum/velocity,
// [NC,2NC) pre-force velocity) and gridMass (float x NC), as the shaders do.
// They back the single-pass C ABI and the dense engine path.
#include "mpm_internal.h"
#include "mpm_particle.cuh"
#include "mpm_scan_kernel.cuh"

namespace nebula {

namespace {

constexpr int kThreads = 256;

inline uint32_t blocksFor(uint64_t n, int t = kThreads) { return uint32_t((n + t - 1) / t); }

constexpr uint32_t kKeyExcluded = 0xffffffffu;

// mpm_hash_count.comp:7-14 / hash_count.comp:7-20 (+ the slot the sort would take).
// Runs of equal keys in neighbouring lanes (particles stored in cell order, or
// lattice order along x) take their slots with one atomic per run; the whole
// warp stays converged for the shuffles, lanes without a particle carrying
// the excluded key.
__global__ void __launch_bounds__(kThreads) k_bin_count(SubstepParams P, const float4* __restrict__ pos, const uint32_t* __restrict__ typeFlag,
                                                        uint32_t n, uint32_t* cellCount, uint32_t* key, uint32_t* rank) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t c = kKeyExcluded;
  if (i < n && !(typeFlag && typeFlag[i] == kTypeFlagUnused)) {
    const float4 p = pos[i];
    int cx, cy, cz;
    cellCoords(P, p.x, p.y, p.z, cx, cy, cz);
    c = mortonEncode(cx, cy, cz);
  }
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t up = __shfl_up_sync(0xffffffffu, c, 1);
  const uint32_t heads = __ballot_sync(0xffffffffu, lane == 0 || up != c);
  const uint32_t le = 0xffffffffu >> (31u - lane);  // lanes 0..lane
  const uint32_t head = 31u - __clz(heads & le);     // first lane of this lane's run
  const uint32_t after = heads & ~le;
  const uint32_t runEnd = after ? uint32_t(__ffs(after) - 1) : 32u;
  uint32_t base = 0;
  if (lane == head && c != kKeyExcluded) base = atomicAdd(cellCount + c, runEnd - lane);
  base = __shfl_sync(0xffffffffu, base, head);
  if (i < n) {
    key[i] = c;
    rank[i] = base + (lane - head);
  }
}

// mpm_hash_sort.comp:7-15 with the slot taken at count time
__global__ void __launch_bounds__(kThreads) k_bin_scatter(uint32_t n, const uint32_t* __restrict__ key, const uint32_t* __restrict__ rank,
                                                          const uint32_t* __restrict__ cellStart, uint32_t* sortedTmp, uint32_t* err) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = key[i];
  if (c == kKeyExcluded) return;
  const uint32_t slot = cellStart[c] + rank[i];
  if (slot < n) sortedTmp[slot] = i;
  else atomicOr(err, kErrBinRange);  // only after an expired scan wait
}

// In-cell canonical order (ascending particle index).  Cells of at most
// kCanonCellMax particles: one thread per cell loads the cell's slots (the
// warp reads one contiguous span) and ranks them in registers.  Larger cells:
// one thread per particle counts the smaller indices of its cell.
constexpr uint32_t kCanonCellMax = 16;

__global__ void __launch_bounds__(kThreads) k_bin_canon_cells(uint32_t nc, uint32_t n, const uint32_t* __restrict__ cellStart,
                                                              const uint32_t* __restrict__ cellCount, const uint32_t* __restrict__ sortedTmp,
                                                              uint32_t* sorted, uint32_t* err) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const uint32_t cnt = cellCount[c];
  if (cnt == 0 || cnt > kCanonCellMax) return;
  const uint32_t st = cellStart[c];
  if (st > n || cnt > n - st) {
    atomicOr(err, kErrBinRange);
    return;
  }
  uint32_t v[kCanonCellMax];
#pragma unroll
  for (uint32_t k = 0; k < kCanonCellMax; ++k) v[k] = k < cnt ? sortedTmp[st + k] : 0xffffffffu;  // padding never ranks below
#pragma unroll
  for (uint32_t k = 0; k < kCanonCellMax; ++k) {
    if (k < cnt) {
      uint32_t r = 0;
#pragma unroll
      for (uint32_t j = 0; j < kCanonCellMax; ++j) r += v[j] < v[k] ? 1u : 0u;
      sorted[st + r] = v[k];
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_bin_canon_particles(uint32_t n, const uint32_t* __restrict__ key,
                                                                  const uint32_t* __restrict__ cellStart, const uint32_t* __restrict__ cellCount,
                                                                  const uint32_t* __restrict__ sortedTmp, uint32_t* sorted, uint32_t* err) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = key[i];
  if (c == kKeyExcluded) return;
  const uint32_t st = cellStart[c], cnt = cellCount[c];
  if (cnt <= kCanonCellMax) return;  // ranked by k_bin_canon_cells
  if (st > n || cnt > n - st) {
    atomicOr(err, kErrBinRange);
    return;
  }
  uint32_t r = 0;
  for (uint32_t j = st; j < st + cnt; ++j) r += sortedTmp[j] < i ? 1u : 0u;
  sorted[st + r] = i;
}

// P2G: one thread per sorted slot, contributions added to the dense grid.
__global__ void __launch_bounds__(kThreads) k_p2g_dense(SubstepParams P, StatePtrs st, const uint32_t* __restrict__ sorted, uint32_t n,
                                                        float4* gridMom, float* gridMass) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t p = sorted[t];
  if (p >= n) return;  // a caller-supplied order with an out-of-range index
  PState s;
  s.P = st.f[0][p]; s.v = st.f[1][p];
  s.F0 = st.f[2][p]; s.F1 = st.f[3][p]; s.F2 = st.f[4][p];
  s.B0 = st.f[5][p]; s.B1 = st.f[6][p]; s.B2 = st.f[7][p];
  p2gParticle(P, s, P.dt, [&](int nx, int ny, int nz, float mx, float my, float mz, float m) {
    uint32_t nid = mortonEncode(nx, ny, nz);
    redAddV4(gridMom + nid, mx, my, mz, 0.f);
    atomicAdd(gridMass + nid, m);
  });
}

// mpm_grid_update.comp + mpm_nanovdb_bc.comp, one thread per node.
__global__ void __launch_bounds__(kThreads) k_grid_dense(SubstepParams P, float4* gridMom, const float* __restrict__ gridMass) {
  uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= P.hashCells) return;
  float mass = gridMass[gid];
  if (mass < 1e-10f) return;
  float4 mom = gridMom[gid];
  int ix, iy, iz;
  mortonDecode(gid, ix, iy, iz);
  float3 v, vo;
  gridNode(P, ix, iy, iz, mass, mom.x, mom.y, mom.z, v, vo);
  gridMom[P.hashCells + gid] = make_float4(vo.x, vo.y, vo.z, 0.f);
  gridMom[gid] = make_float4(v.x, v.y, v.z, 0.f);
}

struct DenseGrid {
  const float4* mom;
  const float* mass;
  uint32_t nc;
  __device__ __forceinline__ bool node(int x, int y, int z, float& m, float3& v, float3& vo) const {
    uint32_t nid = mortonEncode(x, y, z);
    m = __ldg(mass + nid);
    if (m < 1e-10f) return false;
    float4 a = __ldg(mom + nid);
    float4 b = __ldg(mom + nc + nid);
    v = make_float3(a.x, a.y, a.z);
    vo = make_float3(b.x, b.y, b.z);
    return true;
  }
};

__global__ void __launch_bounds__(kThreads) k_g2p_dense(SubstepParams P, StatePtrs st, uint32_t n, const float4* __restrict__ gridMom,
                                                        const float* __restrict__ gridMass, uint32_t* err) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  PState s;
  s.P = st.f[0][p]; s.v = st.f[1][p];
  s.F0 = st.f[2][p]; s.F1 = st.f[3][p]; s.F2 = st.f[4][p];
  s.B0 = st.f[5][p]; s.B1 = st.f[6][p]; s.B2 = st.f[7][p];
  DenseGrid g{gridMom, gridMass, P.hashCells};
  g2pParticle(P, s, g, P.dt);
  if (err && !(isfinite(s.P.x) && isfinite(s.P.y) && isfinite(s.P.z))) atomicOr(err, kErrNonFinite);
  st.f[0][p] = s.P; st.f[1][p] = s.v;
  st.f[2][p] = s.F0; st.f[3][p] = s.F1; st.f[4][p] = s.F2;
  st.f[5][p] = s.B0; st.f[6][p] = s.B1; st.f[7][p] = s.B2;
}

}  // namespace

size_t scanWorkspaceBytes(uint64_t n) { return (size_t(scanTiles(n)) + 2) * sizeof(unsigned long long); }

cudaError_t launchBin(const SubstepParams& P, const float4* pos, uint32_t n, const BinBuffers& b, cudaStream_t s, uint64_t* launches) {
  const uint64_t nc = P.hashCells;
  cudaError_t e = cudaMemsetAsync(b.cellCount, 0, nc * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    k_bin_count<<<blocksFor(n), kThreads, 0, s>>>(P, pos, b.typeFlag, n, b.cellCount, b.key, b.rank);
    ++*launches;
  }
  const uint32_t tiles = scanTiles(nc);
  e = cudaMemsetAsync(b.tileState, 0, (size_t(tiles) + 1) * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  k_scan_exclusive<<<tiles, kScanThreads, 0, s>>>(b.cellCount, b.cellStart, b.cellEnd, nc, b.tileState, b.tileCounter, b.err, nullptr);
  ++*launches;
  if (n > 0) {
    k_bin_scatter<<<blocksFor(n), kThreads, 0, s>>>(n, b.key, b.rank, b.cellStart, b.sortedTmp, b.err);
    k_bin_canon_cells<<<blocksFor(nc), kThreads, 0, s>>>(uint32_t(nc), n, b.cellStart, b.cellCount, b.sortedTmp, b.sorted, b.err);
    k_bin_canon_particles<<<blocksFor(n), kThreads, 0, s>>>(n, b.key, b.cellStart, b.cellCount, b.sortedTmp, b.sorted, b.err);
    *launches += 3;
  }
  return cudaGetLastError();
}

cudaError_t launchBinScanExpiryProbe(const SubstepParams& P, const BinBuffers& b, cudaStream_t s, uint64_t* launches) {
  const uint64_t nc = P.hashCells;
  const uint32_t tiles = scanTiles(nc);
  if (tiles < 2) return cudaErrorInvalidValue;
  // every status word unpublished and the tile ticket at 1: the single CTA
  // below becomes tile 1 and waits on a tile 0 that never runs
  cudaError_t e = cudaMemsetAsync(b.tileState, 0, (size_t(tiles) + 1) * sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.err, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.tileCounter, 1, 1, s);  // little-endian u32 = 1
  if (e != cudaSuccess) return e;
  k_scan_exclusive<<<1, kScanThreads, 0, s>>>(b.cellCount, b.cellStart, nullptr, nc, b.tileState, b.tileCounter, b.err, nullptr);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchP2GDense(const SubstepParams& P, StatePtrs st, const uint32_t* sorted, uint32_t n, float4* gridMom, float* gridMass,
                           cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_p2g_dense<<<blocksFor(n), kThreads, 0, s>>>(P, st, sorted, n, gridMom, gridMass);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchGridDense(const SubstepParams& P, float4* gridMom, const float* gridMass, cudaStream_t s, uint64_t* launches) {
  k_grid_dense<<<blocksFor(P.hashCells), kThreads, 0, s>>>(P, gridMom, gridMass);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launchG2PDense(const SubstepParams& P, StatePtrs st, uint32_t n, const float4* gridMom, const float* gridMass, uint32_t* err,
                           cudaStream_t s, uint64_t* launches) {
  if (n == 0) return cudaSuccess;
  k_g2p_dense<<<blocksFor(n), kThreads, 0, s>>>(P, st, n, gridMom, gridMass, err);
  ++*launches;
  return cudaGetLastError();
}

}  // namespace nebula
