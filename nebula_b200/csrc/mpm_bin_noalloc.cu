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
// The first call in a CUDA context (the device's primary context, or a
// context the caller made current) looks up the array's address with
// cudaGetSymbolAddress; that lookup can load this file's module, so make the
// first call before beginning any stream capture.  Later calls in the same
// context reuse the cached address; the cache is keyed by the context's
// unique id, so a context destroyed by cudaDeviceReset and created again gets
// its address looked up afresh instead of reusing a stale one.  The counts,
// the scan status words and the error word are cleared on the stream by every
// call, so nothing has to start at zero.  The scratch is shared by every call
// on the same device: calls that may overlap in time (two streams, or two
// host threads) race on it and must be ordered by the caller.  The error word
// of the last call (an expired scan wait, an index out of range) stays in the
// scratch until the next call and is read by nebula_mpm_bin_noalloc_status.
#include <cuda.h>  // CUcontext / CUresult types only: the two driver calls are resolved at run time

#include <cstdio>
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
struct ScratchSlot {
  unsigned long long ctxId;  // cuCtxGetId of the context the address belongs to (0: none)
  void* ptr;
};
ScratchSlot g_scratch[kNoAllocMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctxGetCurrent = nullptr;
CtxGetIdFn g_ctxGetId = nullptr;

// Unique id of the calling thread's current context (0 when none is current
// yet).  cuCtxGetCurrent / cuCtxGetId come from the runtime's driver entry
// point table, so the library keeps no link-time dependency on libcuda.
unsigned long long currentContextId() {
  if (!g_ctxGetCurrent || !g_ctxGetId) {
    void* f = nullptr;
    void* g = nullptr;
    cudaDriverEntryPointQueryResult q1{}, q2{};
    check(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q1), "driver entry point cuCtxGetCurrent");
    check(cudaGetDriverEntryPointByVersion("cuCtxGetId", &g, 12000, cudaEnableDefault, &q2), "driver entry point cuCtxGetId");
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f || !g)
      throw Error(NEBULA_MPM_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
    g_ctxGetCurrent = reinterpret_cast<CtxGetCurrentFn>(f);
    g_ctxGetId = reinterpret_cast<CtxGetIdFn>(g);
  }
  CUcontext c = nullptr;
  if (g_ctxGetCurrent(&c) != CUDA_SUCCESS || !c) return 0;
  unsigned long long id = 0;
  if (g_ctxGetId(c, &id) != CUDA_SUCCESS) throw Error(NEBULA_MPM_ERR_CUDA, "cuCtxGetId failed");
  return id;
}

// Address of g_binScratch in the current context; looked up once per context.
unsigned char* scratchForCurrentContext() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) throw Error(NEBULA_MPM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratchMutex);
  unsigned long long id = currentContextId();
  ScratchSlot& slot = g_scratch[dev];
  if (id == 0 || slot.ctxId != id || !slot.ptr) {
    void* p = nullptr;
    // also creates the runtime's context when none is current yet
    check(cudaGetSymbolAddress(&p, g_binScratch), "cudaGetSymbolAddress(bin scratch)");
    if (!p) throw Error(NEBULA_MPM_ERR_CUDA, "bin scratch has no device address");
    if (id == 0) id = currentContextId();
    slot.ctxId = id;
    slot.ptr = p;
  }
  return static_cast<unsigned char*>(slot.ptr);
}

// The counting sort's buffers inside the scratch for `hashCells` cells.
BinBuffers scratchBins(unsigned char* ws, uint32_t hashCells) {
  BinBuffers b{};
  b.cellStart = reinterpret_cast<uint32_t*>(ws + kOffCellStart);
  b.key = reinterpret_cast<uint32_t*>(ws + kOffKey);
  b.rank = reinterpret_cast<uint32_t*>(ws + kOffRank);
  b.sortedTmp = reinterpret_cast<uint32_t*>(ws + kOffSortedTmp);
  b.tileState = reinterpret_cast<unsigned long long*>(ws + kOffTiles);
  b.tileCounter = reinterpret_cast<uint32_t*>(b.tileState + scanTiles(hashCells));
  b.err = reinterpret_cast<uint32_t*>(ws + kOffErr);
  return b;
}

// The checks every entry point of this file makes on the pass parameters.
uint32_t checkNoAllocPass(const nebula_mpm_pass* pass) {
  if (!pass) throw Error(NEBULA_MPM_ERR_INVALID, "null pass parameters");
  if (!(pass->cellSize > 0.f)) throw Error(NEBULA_MPM_ERR_INVALID, "cellSize must be > 0");
  const uint32_t cube = domainCubeRes(pass->gridRes);
  if (cube > 1024u) throw Error(NEBULA_MPM_ERR_INVALID, "grid resolution above 1024 per axis");
  if (pass->hashCells != cube * cube * cube) throw Error(NEBULA_MPM_ERR_INVALID, "hashCells must equal cubeRes^3 of gridRes");
  if (pass->hashCells > kNoAllocMaxCells)
    throw Error(NEBULA_MPM_ERR_INVALID, "nebula_mpm_bin_noalloc: hashCells " + std::to_string(pass->hashCells) + " exceeds the fixed maximum " +
                                            std::to_string(kNoAllocMaxCells) + " (128^3); use nebula_mpm_bin with a workspace");
  if (pass->particleCount > kNoAllocMaxParticles)
    throw Error(NEBULA_MPM_ERR_INVALID, "nebula_mpm_bin_noalloc: particleCount " + std::to_string(pass->particleCount) +
                                            " exceeds the fixed maximum " + std::to_string(kNoAllocMaxParticles) +
                                            "; use nebula_mpm_bin with a workspace");
  return cube;
}

SubstepParams binParams(const nebula_mpm_pass* pass, uint32_t cube) {
  SubstepParams P{};
  P.cellSize = pass->cellSize;
  for (int a = 0; a < 3; ++a) {
    P.gridRes[a] = int(pass->gridRes[a]);
    P.worldMin[a] = pass->worldMin[a];
    P.worldMax[a] = pass->worldMax[a];
  }
  P.cubeRes = cube;
  P.hashCells = pass->hashCells;
  return P;
}

template <class F> int guardedNoAlloc(F&& f) {
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

size_t nebula_mpm_bin_noalloc_max_cells(void) { return kNoAllocMaxCells; }
size_t nebula_mpm_bin_noalloc_max_particles(void) { return kNoAllocMaxParticles; }

int nebula_mpm_bin_noalloc(const nebula_mpm_pass* pass, const float* dPos4, uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSorted,
                           void* stream) {
  return guardedNoAlloc([&] {
    const uint32_t cube = checkNoAllocPass(pass);
    const uint32_t n = pass->particleCount;
    if (!dCellCount || !dCellOffset || (n && (!dPos4 || !dSorted))) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");
    BinBuffers b = scratchBins(scratchForCurrentContext(), pass->hashCells);
    b.cellCount = dCellCount;
    b.cellEnd = dCellOffset;
    b.sorted = dSorted;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemsetAsync(b.err, 0, 4, s), "memset");
    uint64_t launches = 0;
    check(launchBin(binParams(pass, cube), reinterpret_cast<const float4*>(dPos4), n, b, s, &launches), "bin");
  });
}

int nebula_mpm_bin_noalloc_status(uint32_t* errorBits, void* stream) {
  return guardedNoAlloc([&] {
    if (!errorBits) throw Error(NEBULA_MPM_ERR_INVALID, "null output");
    *errorBits = 0;
    const unsigned char* ws = scratchForCurrentContext();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t bits = 0;
    check(cudaMemcpyAsync(&bits, ws + kOffErr, sizeof(bits), cudaMemcpyDeviceToHost, s), "read error word");
    check(cudaStreamSynchronize(s), "stream synchronize");
    *errorBits = bits;
    throwBinErrors(bits);
  });
}

int nebula_mpm_bin_noalloc_probe_wait_expiry(const nebula_mpm_pass* pass, const uint32_t* dCellCount, void* stream) {
  return guardedNoAlloc([&] {
    const uint32_t cube = checkNoAllocPass(pass);
    if (pass->hashCells < 2u * uint32_t(kScanTile)) throw Error(NEBULA_MPM_ERR_INVALID, "the probe needs hashCells >= 4096");
    if (!dCellCount) throw Error(NEBULA_MPM_ERR_INVALID, "null buffer");
    BinBuffers b = scratchBins(scratchForCurrentContext(), pass->hashCells);
    b.cellCount = const_cast<uint32_t*>(dCellCount);
    uint64_t launches = 0;
    check(launchBinScanExpiryProbe(binParams(pass, cube), b, static_cast<cudaStream_t>(stream), &launches), "bin scan probe");
  });
}

}  // extern "C"
