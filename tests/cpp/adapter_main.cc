// Drives bhg_host::step_particles (the drop-in for bh::step_particles) with
// the reference's leapfrog schedule (main.cc:199-246) on particles read from
// a raw file of 64-byte records, and writes the result back.  Built against
// either the reference's own types (BHG_WITH_REFERENCE_TYPES, with the
// reference headers on the include path) or local types of the same layout.
#include "bhg_step_particles.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

#ifdef BHG_WITH_REFERENCE_TYPES
#include "integrate_ttg.h"  // bh::Particle, bh::ForceParams, bh::StepTiming
using P = bh::Particle;
using F = bh::ForceParams;
using T = bh::StepTiming;
#else
struct P {
  std::uint32_t id;
  double mass;
  double pos[3], vel[3];
};
struct F {
  double theta = 0.5, eps2 = 0.0, G = 1.0;
  bool use_quadrupole = true;
};
struct T {
  double tree_build_ms = 0, traversal_ms = 0, exchange_ms = 0;
};
#endif

int main(int argc, char** argv) {
  if (argc < 8) {
    std::fprintf(stderr, "usage: %s in.bin out.bin theta eps dt steps precision\n", argv[0]);
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::fseek(f, 0, SEEK_END);
  long bytes = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<P> particles(static_cast<std::size_t>(bytes) / sizeof(P));
  if (std::fread(particles.data(), sizeof(P), particles.size(), f) != particles.size()) return 2;
  std::fclose(f);
  F fp;
  fp.theta = std::atof(argv[3]);
  double eps = std::atof(argv[4]);
  fp.eps2 = eps * eps;
  fp.G = 1.0;
  fp.use_quadrupole = true;
  const double dt = std::atof(argv[5]);
  const int steps = std::atoi(argv[6]);
  bhg_host::default_precision() = std::atoi(argv[7]);
  try {
    bhg_host::Workspace ws;
    T timing;
    particles = bhg_host::step_particles(std::move(particles), fp, 16, 256, 16, dt / 2.0, dt, &timing, &ws);
    for (int s = 1; s < steps; ++s)
      particles = bhg_host::step_particles(std::move(particles), fp, 16, 256, 16, dt, dt, &timing, &ws);
    particles = bhg_host::step_particles(std::move(particles), fp, 16, 256, 16, dt / 2.0, 0.0, &timing, &ws);
    std::printf("last evaluation: tree %.3f ms traversal %.3f ms\n", timing.tree_build_ms, timing.traversal_ms);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  f = std::fopen(argv[2], "wb");
  if (!f) return 2;
  std::fwrite(particles.data(), sizeof(P), particles.size(), f);
  std::fclose(f);
  return 0;
}
