// hash_bin_oracle.cpp -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
// PBF engine's spatial hash, the checker of nebula_hash_bin.
//
// zero_cells, then hash_count.comp:7-20 (cell of predP, particles flagged 6 =
// TYPE_FLAG_UNUSED skipped), hash_scan_local/global.comp + hash_add_base.comp
// (exclusive prefix of the counts; the intended scan over any number of
// cells), hash_sort.comp:9-22 (each particle takes the next slot of its cell,
// which leaves cellOffset at the END of every range).  Visiting particles in
// ascending index gives the canonical in-cell order.  The cell is
// common.glsl:100-105: clamp((p - worldMin) / cellSize, 0, gridRes - 1),
// truncated, Morton-interleaved; fmax/fmin put a NaN coordinate in cell 0 of
// its axis, as the device's fmaxf/fminf do.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

uint32_t expand10(uint32_t v) {  // bit i of v -> bit 3i
  uint32_t r = 0;
  for (int b = 0; b < 10; ++b) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

}  // namespace

extern "C" void orc_hash_bin(const float* predP4, const uint32_t* typeFlag, uint32_t n, const float* worldMin, float cellSize,
                             const uint32_t* gridRes, uint32_t hashCells, uint32_t* cellCount, uint32_t* cellOffset, uint32_t* sortedIdx) {
  std::vector<uint32_t> key(n, 0xffffffffu);
  for (uint32_t c = 0; c < hashCells; ++c) cellCount[c] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (typeFlag && typeFlag[i] == 6u) continue;
    uint32_t g[3];
    for (int a = 0; a < 3; ++a) {
      float l = (predP4[4 * size_t(i) + a] - worldMin[a]) / cellSize;
      l = std::fmin(std::fmax(l, 0.0f), float(gridRes[a]) - 1.0f);
      g[a] = uint32_t(l);
    }
    key[i] = expand10(g[0]) | (expand10(g[1]) << 1u) | (expand10(g[2]) << 2u);
    ++cellCount[key[i]];
  }
  uint32_t acc = 0;
  for (uint32_t c = 0; c < hashCells; ++c) {
    cellOffset[c] = acc;
    acc += cellCount[c];
  }
  for (uint32_t i = 0; i < n; ++i)
    if (key[i] != 0xffffffffu) sortedIdx[cellOffset[key[i]]++] = i;
}
