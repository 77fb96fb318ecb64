// mpm_bin_noalloc.cu -- a binning entry point that allocates no device memory.
//
// nebula_mpm_bin needs a caller-provided workspace for the counting sort
// (per-cell range starts, per-particle keys and ranks, the unsorted slot list)
// and for the look-back scan's per-tile status words.  Some callers cannot
// hand one over: a thin foreign-function binding that only holds the three
// output arrays, or a host loop that must not call cudaMalloc between frames
// because cudaMalloc may synchronise the whole device.  This variant keeps the
// scratch in one file-scope __device__ array instead, sized for a fixed
// maximum problem, and runs exactly the same kernels as nebula_mpm_bin.
//
// The first call on a device (with that device current) looks up the array's
// address with cudaGetSymbolAddress; that lookup can load this file's module,
// so make the first call before beginning any stream capture.  Later calls
// reuse the cached address.  The counts, the scan status words and the error
// word are cleared on the stream by every call, so nothing has to start at
// zero.  The scratch is shared by every call on the same device: calls that
// may overlap in time (two streams, or two host threads) race on it and must
// be ordered by the caller.
#include <cstring>
#include <mutex>

#include "mpm_engine.h"
#include "mpm_internal.h"
#include "mpm_scan.cuh"

namespace nebula {
namespace {

constexpr uint32_t kNoAllocMaxCells = 1u << 21;      // 128^3 cells
constexpr uint32_t kNoAllocMaxParticles = 1u << 18;  // 262,144 particles
constexpr int kNoAllocMaxDevices = 64;

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCellStart = 0;
constexpr size_t kOffKey = al256(kOffCellStart + size_t(kNoAllocMaxCells) * 4);
constexpr size_t kOffRank = al256(kOffKey + size_t(kNoAllocMaxParticles) * 4);
constexpr size_t kOffSortedTmp = al256(kOffRank + size_t(kNoAllocMaxParticles) * 4);
constexpr size_t kOffTiles = al256(kOffSortedTmp + size_t(kNoAllocMaxParticles) * 4);
// one u64 status word per scan tile plus the u32 tile ticket (stored as a u64)
constexpr size_t kOffErr = al256(kOffTiles + (size_t((kNoAllocMaxCells + kScanTile - 1) / kScanTile) + 1) * 8);
constexpr size_t kNoAllocBytes = al256(kOffErr + 4);

__device__ __align__(256) unsigned char g_binScratch[kNoAllocBytes];

std::mutex g_scratchMutex;
void* g_scratchPtr[kNoAllocMaxDevices] = {};

// Address of g_binScratch on the current device; looked up once per device.
unsigned char* scratchForCurrentDevice() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) throw Error(NEBULA_MPM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratchMutex);
  if (!g_scratchPtr[dev]) {
    void* p = nullptr;
    check(cudaGetSymbolAddress(&p, g_binScratch), "cudaGetSymbolAddress(bin scratch)");
    if (!p) throw Error(NEBULA_MPM_ERR_CUDA, "bin scratch has no device address");
    g_scratchPtr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratchPtr[dev]);
}

}  // namespace
}  // namespace nebula

using namespace nebula;

extern "C" {

size_t nebula_mpm_bin_noalloc_max_cells(void) { return kNoAllocMaxCells; }
size_t nebula_mpm_bin_noalloc_max_particles(void) { return kNoAllocMaxParticles; }

int nebula_mpm_bin_noalloc(const nebula_mpm_pass* pass, const float* dPos4, uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSorted,
                           void* stream) {
  try {
    if (!pass) throw Error(NEBULA_MPM_ERR_INVALID, "null pass parameters");
    if (!(pass->cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
    const uint32_t cube = domainCubeRes(pass->gridRes);
    if (cube > 1024u) throw Error(NEBULA_MPM_ERR_INVALID, "grid resolution above 1024 per axis");
    if (pass->hashCells != cube * cube * cube) throw Error(NEBULA_MPM_ERR_INVALID, "hashCells must equal cubeRes^3 of gridRes");
    if (pass->hashCells > kNoAllocMaxCells)
      throw Error(NEBULA_MPM_ERR_INVALID, "nebula_mpm_bin_noalloc: hashCells " + std::to_string(pass->hashCells) + " exceeds the fixed maximum " +
                                              std::to_string(kNoAllocMaxCells) + " (128^3); use nebula_mpm_bin with a workspace");
    const uint32_t n = pass->particleCount;
    if (n > kNoAllocMaxParticles)
      throw Error(NEBULA_MPM_ERR_INVALID, "nebula_mpm_bin_noalloc: particleCount " + std::to_string(n) + " exceeds the fixed maximum " +
                                              std::to_string(kNoAllocMaxParticles) + "; use nebula_mpm_bin with a workspace");
    if (!dCellCount || !dCellOffset || (n && (!dPos4 || !dSorted))) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");

    unsigned char* ws = scratchForCurrentDevice();
    BinBuffers b;
    b.cellCount = dCellCount;
    b.cellStart = reinterpret_cast<uint32_t*>(ws + kOffCellStart);
    b.cellEnd = dCellOffset;
    b.key = reinterpret_cast<uint32_t*>(ws + kOffKey);
    b.rank = reinterpret_cast<uint32_t*>(ws + kOffRank);
    b.sortedTmp = reinterpret_cast<uint32_t*>(ws + kOffSortedTmp);
    b.sorted = dSorted;
    b.tileState = reinterpret_cast<unsigned long long*>(ws + kOffTiles);
    b.tileCounter = reinterpret_cast<uint32_t*>(b.tileState + scanTiles(pass->hashCells));
    b.err = reinterpret_cast<uint32_t*>(ws + kOffErr);

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemsetAsync(b.err, 0, 4, s), "memset");
    SubstepParams P{};
    P.cellSize = pass->cellSize;
    for (int a = 0; a < 3; ++a) {
      P.gridRes[a] = int(pass->gridRes[a]);
      P.worldMin[a] = pass->worldMin[a];
      P.worldMax[a] = pass->worldMax[a];
    }
    P.cubeRes = cube;
    P.hashCells = pass->hashCells;
    uint64_t launches = 0;
    check(launchBin(P, reinterpret_cast<const float4*>(dPos4), n, b, s, &launches), "bin");
    return NEBULA_MPM_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return NEBULA_MPM_ERR_INVALID;
  }
}

}  // extern "C"
