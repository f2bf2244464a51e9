// TEST INFRASTRUCTURE ONLY - times the reference solver on the host cores.
//
// Compiled by oracle/Makefile against the UNMODIFIED reference sources and
// the thread-pool stand-in for TTG (oracle/ttg_shim), into
// oracle/_ref/ref_bench.  It reads a raw file of 64-byte bh::Particle
// records and runs the reference's own leapfrog schedule (src/main.cc:199-246)
// through its public entry point bh::step_particles
// (src/integrate_ttg.h:66-148): a (dt/2, dt) evaluation, steps-1 (dt, dt)
// evaluations and a closing (dt/2, 0) one - or, with --evals E, only the
// first E evaluations of that schedule (a bounded sample).  Prints one JSON
// line with the wall time of every evaluation and the thread count.
#include "integrate_ttg.h"

#include <ttg.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

int main(int argc, char** argv) {
  std::string path;
  int steps = 1, evals = -1;
  unsigned max_leaf = 16;
  std::uint32_t group_size = 256, target_size = 16;
  bh::ForceParams fp;
  fp.theta = 0.5;
  fp.eps2 = 0.0;
  fp.G = 1.0;
  fp.use_quadrupole = true;
  double dt = 1.0 / 128;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() { return std::string(i + 1 < argc ? argv[++i] : ""); };
    if (a == "--particles") path = next();
    else if (a == "--steps") steps = std::atoi(next().c_str());
    else if (a == "--evals") evals = std::atoi(next().c_str());
    else if (a == "--dt") dt = std::atof(next().c_str());
    else if (a == "--theta") fp.theta = std::atof(next().c_str());
    else if (a == "--eps") { double e = std::atof(next().c_str()); fp.eps2 = e * e; }
    else if (a == "--max-leaf") max_leaf = static_cast<unsigned>(std::atoi(next().c_str()));
    else if (a == "--group-size") group_size = static_cast<std::uint32_t>(std::atoi(next().c_str()));
    else if (a == "--target-size") target_size = static_cast<std::uint32_t>(std::atoi(next().c_str()));
    else if (a == "--no-quadrupole") fp.use_quadrupole = false;
    else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); return 2; }
  }
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); return 2; }
  std::fseek(f, 0, SEEK_END);
  long bytes = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<bh::Particle> particles(static_cast<std::size_t>(bytes) / sizeof(bh::Particle));
  if (std::fread(particles.data(), sizeof(bh::Particle), particles.size(), f) != particles.size()) return 2;
  std::fclose(f);

  ttg::initialize(argc, argv, -1);
  ttg::execute();
  int total = steps + 1;
  if (evals > 0 && evals < total) total = evals;
  bh::GroupedWorkspace ws;
  std::vector<double> ms;
  for (int e = 0; e < total; ++e) {
    double kick = (e == 0 || e == steps) ? dt / 2.0 : dt;
    double drift = (e == steps) ? 0.0 : dt;
    auto t0 = std::chrono::steady_clock::now();
    particles = bh::step_particles(std::move(particles), fp, max_leaf, group_size, target_size, kick, drift, nullptr, &ws);
    ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
  ttg::fence();
  std::printf("{\"n\": %zu, \"threads\": %d, \"eval_ms\": [", particles.size(), ttg::shim::Pool::get().size());
  for (std::size_t i = 0; i < ms.size(); ++i) std::printf("%s%.3f", i ? ", " : "", ms[i]);
  std::printf("]}\n");
  ttg::finalize();
  return 0;
}
