// A caller written against the reference's MPMEngine surface, through the
// header-only facade include/nebula_mpm.hpp: the reference's default config
// (a 32^3 lattice in a 10 m domain, h = 10/64), gravity as a force, APIC, two
// frames of 10 substeps.
// Prints one JSON line: {"ok": true, "live": n, "mean": [x, y, z]} or
// {"ok": false, "error": "..."} when no engine can be created.
#include <cmath>
#include <cstdio>

#include "nebula_mpm.hpp"

int main() {
  nebula_b200::MPMConfig cfg;  // MPMConfig defaults
  try {
    nebula_b200::MPMEngine engine(cfg);
    nebula_mpm_force g{};
    g.type = 0;  // GRAVITY: direction (0, -1, 0), strength 9.8
    g.data[1] = -1.0f;
    g.data[3] = 9.8f;
    engine.addForce(g);
    engine.flip_ratio = -1.0f;  // APIC
    engine.numSubsteps = 10;
    for (int frame = 0; frame < 2; ++frame) engine.step(nullptr, 1e-3f);
    engine.sync();
    const std::vector<float> p = engine.download(nebula_b200::Field::P);
    const uint32_t n = engine.liveParticleCount();
    double m[3] = {0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) m[a] += p[4 * size_t(i) + a];
    for (double& v : m) v /= std::max<uint32_t>(n, 1);
    std::printf("{\"ok\": true, \"live\": %u, \"mean\": [%.9g, %.9g, %.9g]}\n", n, m[0], m[1], m[2]);
  } catch (const std::exception& e) {
    std::printf("{\"ok\": false, \"error\": \"%s\"}\n", e.what());
  }
  return 0;
}
