// TEST INFRASTRUCTURE ONLY - times the reference solver on the host cores.
//
// Compiled by oracle/Makefile against the UNMODIFIED reference sources and
// the thread-pool stand-in for TTG (oracle/ttg_shim), into
// oracle/_ref/ref_bench.  It runs the reference's own leapfrog schedule
// (src/main.cc:199-246) through its public entry point bh::step_particles
// (src/integrate_ttg.h:66-148): a (dt/2, dt) evaluation, steps-1 (dt, dt)
// evaluations and a closing (dt/2, 0) one, schedule after schedule.
//
// Input: a raw file of 64-byte bh::Particle records (--particles), or
// Plummer spheres generated here from a seed (--seed S --sphere
// n,a,mass,cx,cy,cz,bx,by,bz, repeatable: each further sphere continues the
// first one's random stream, ids consecutive) by the same generator the GPU
// library uses (amt-bh-benchmark_b200/csrc/bhg_plummer.h), so the timing
// process loads nothing of the GPU library.
//
// Timing: --warmup-evals W untimed evaluations, then --timed-evals K timed
// ones (defaults 0 and one whole schedule); --evals E is the older form (the
// first E evaluations, all timed).  Prints one JSON line with the wall time
// of every timed evaluation, the thread count and the generation time.
#include "integrate_ttg.h"

#include <ttg.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bhg_plummer.h"

namespace {

// The 64-byte record the generator writes; bh::Particle has the same layout.
struct Rec {
  std::uint32_t id, pad;
  double mass, pos[3], vel[3];
};
static_assert(sizeof(Rec) == 64 && sizeof(bh::Particle) == 64, "64-byte particle records");

struct Sphere {
  std::size_t n = 0;
  double a = 1.0, mass = 1.0, c[3] = {0, 0, 0}, b[3] = {0, 0, 0};
};

bool parse_sphere(const std::string& s, Sphere* out) {
  double v[9];
  int k = std::sscanf(s.c_str(), "%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5],
                      &v[6], &v[7], &v[8]);
  if (k != 9 || !(v[0] >= 1)) return false;
  out->n = static_cast<std::size_t>(v[0]);
  out->a = v[1], out->mass = v[2];
  for (int i = 0; i < 3; ++i) out->c[i] = v[3 + i], out->b[i] = v[6 + i];
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  std::string path;
  int steps = 1, evals = -1, warmup_evals = 0, timed_evals = -1;
  unsigned max_leaf = 16;
  std::uint32_t group_size = 256, target_size = 16;
  std::uint64_t seed = 1;
  std::vector<Sphere> spheres;
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
    else if (a == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
    else if (a == "--sphere") {
      Sphere sp;
      if (!parse_sphere(next(), &sp)) { std::fprintf(stderr, "bad --sphere\n"); return 2; }
      spheres.push_back(sp);
    }
    else if (a == "--steps") steps = std::atoi(next().c_str());
    else if (a == "--evals") evals = std::atoi(next().c_str());
    else if (a == "--warmup-evals") warmup_evals = std::atoi(next().c_str());
    else if (a == "--timed-evals") timed_evals = std::atoi(next().c_str());
    else if (a == "--dt") dt = std::atof(next().c_str());
    else if (a == "--theta") fp.theta = std::atof(next().c_str());
    else if (a == "--eps") { double e = std::atof(next().c_str()); fp.eps2 = e * e; }
    else if (a == "--max-leaf") max_leaf = static_cast<unsigned>(std::atoi(next().c_str()));
    else if (a == "--group-size") group_size = static_cast<std::uint32_t>(std::atoi(next().c_str()));
    else if (a == "--target-size") target_size = static_cast<std::uint32_t>(std::atoi(next().c_str()));
    else if (a == "--no-quadrupole") fp.use_quadrupole = false;
    else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); return 2; }
  }
  std::vector<bh::Particle> particles;
  auto g0 = std::chrono::steady_clock::now();
  if (!spheres.empty()) {
    std::size_t total = 0;
    for (const Sphere& sp : spheres) total += sp.n;
    std::vector<Rec> recs(total);
    std::size_t at = 0;
    std::uint64_t s = seed;
    for (const Sphere& sp : spheres) {
      s = bhg_ic::plummer(recs.data() + at, sp.n, sp.a, sp.mass, sp.c, sp.b, static_cast<std::uint32_t>(at), s);
      at += sp.n;
    }
    for (Rec& r : recs) r.pad = 0;
    particles.resize(total);
    std::memcpy(static_cast<void*>(particles.data()), recs.data(), total * sizeof(Rec));
  } else {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); return 2; }
    std::fseek(f, 0, SEEK_END);
    long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    particles.resize(static_cast<std::size_t>(bytes) / sizeof(bh::Particle));
    if (std::fread(particles.data(), sizeof(bh::Particle), particles.size(), f) != particles.size()) return 2;
    std::fclose(f);
  }
  const double gen_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - g0).count();

  ttg::initialize(argc, argv, -1);
  ttg::execute();
  const int per = steps + 1;  // evaluations of one schedule
  int warm = warmup_evals, timed = timed_evals < 0 ? per : timed_evals;
  if (evals > 0) warm = 0, timed = evals < per ? evals : per;
  bh::GroupedWorkspace ws;
  std::vector<double> ms;
  for (int e = 0; e < warm + timed; ++e) {
    const int k = e % per;  // position in the schedule; schedules run back to back
    double kick = (k == 0 || k == steps) ? dt / 2.0 : dt;
    double drift = (k == steps) ? 0.0 : dt;
    auto t0 = std::chrono::steady_clock::now();
    particles = bh::step_particles(std::move(particles), fp, max_leaf, group_size, target_size, kick, drift, nullptr, &ws);
    if (e >= warm) ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
  ttg::fence();
  std::printf("{\"n\": %zu, \"threads\": %d, \"gen_ms\": %.3f, \"warmup_evals\": %d, \"eval_ms\": [",
              particles.size(), ttg::shim::Pool::get().size(), gen_ms, warm);
  for (std::size_t i = 0; i < ms.size(); ++i) std::printf("%s%.3f", i ? ", " : "", ms[i]);
  std::printf("]}\n");
  ttg::finalize();
  return 0;
}
