// TEST INFRASTRUCTURE ONLY - a C entry layer over the reference solver.
//
// Compiled by oracle/Makefile against the UNMODIFIED reference headers
// (devreal/AMT-BH-benchmark ttg-parsec/src, included from where they lie)
// and the stand-in TTG runtime in oracle/ttg_shim, into oracle/_ref/
// libbhref.so.  It exposes the reference's own build_flat_tree,
// run_grouped_pass, step_particles, brute_force_accel and energy functions
// to the Python tests, which use them to pin the oracle restatement
// (oracle/bh_oracle.c) and to make the golden fixtures under tests/golden/.
// Nothing here re-implements the algorithm: every number comes from the
// reference's code.
#include "brute_force.h"
#include "flat_build_ttg.h"
#include "grouped_ttg.h"
#include "integrate.h"
#include "integrate_ttg.h"
#include "io.h"

#include <ttg.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <vector>

static_assert(sizeof(bh::Particle) == 64, "bh::Particle is the 64-byte record the C side passes");
static_assert(offsetof(bh::Particle, mass) == 8 && offsetof(bh::Particle, pos) == 16 && offsetof(bh::Particle, vel) == 40,
              "bh::Particle layout");

namespace {

struct RefTree {
  bh::FlatTree f;
  bh::BuildScratch ws;
};

void ensure_runtime() {
  static bool started = false;
  if (!started) {
    ttg::initialize(0, nullptr, -1);
    ttg::execute();
    started = true;
  }
}

std::vector<bh::Particle> to_vec(const void* p, std::size_t n) {
  std::vector<bh::Particle> v(n);
  if (n) std::memcpy(v.data(), p, n * sizeof(bh::Particle));
  return v;
}

}  // namespace

extern "C" {

// build_flat_tree (flat_build_ttg.h:276-281) into a new handle.
void* bhref_build(const void* particles, std::size_t n, unsigned max_leaf, std::uint32_t group_size) {
  ensure_runtime();
  auto* t = new RefTree;
  bh::build_flat_tree(t->f, t->ws, to_vec(particles, n), max_leaf, group_size);
  return t;
}

void bhref_free(void* h) { delete static_cast<RefTree*>(h); }

std::size_t bhref_num_nodes(void* h) { return static_cast<RefTree*>(h)->f.nodes.size(); }
std::size_t bhref_num_groups(void* h) { return static_cast<RefTree*>(h)->f.groups.size(); }

// The tree's arrays: Morton-ordered particles and keys, then per node
// begin, count, first_child, num_children, leaf, depth, center[3],
// half_width, mass, com[3], iab[6].
void bhref_export(void* h, void* particles, std::uint64_t* keys, std::uint32_t* u32_6xM, double* f64_14xM,
                  double* domain4, std::uint32_t* groups) {
  auto& t = *static_cast<RefTree*>(h);
  const std::size_t n = t.f.particles.size(), M = t.f.nodes.size();
  if (particles) std::memcpy(particles, t.f.particles.data(), n * sizeof(bh::Particle));
  if (keys) std::memcpy(keys, t.ws.keys.data(), n * sizeof(std::uint64_t));
  for (std::size_t i = 0; i < M; ++i) {
    const auto& w = t.f.nodes[i];
    if (u32_6xM) {
      u32_6xM[0 * M + i] = w.particle_begin;
      u32_6xM[1 * M + i] = w.particle_count;
      u32_6xM[2 * M + i] = w.first_child;
      u32_6xM[3 * M + i] = w.num_children;
      u32_6xM[4 * M + i] = w.leaf;
      u32_6xM[5 * M + i] = w.depth;
    }
    if (f64_14xM) {
      f64_14xM[3 * i + 0] = t.f.center[i].x;
      f64_14xM[3 * i + 1] = t.f.center[i].y;
      f64_14xM[3 * i + 2] = t.f.center[i].z;
      f64_14xM[3 * M + i] = w.half_width;
      f64_14xM[4 * M + i] = w.mass;
      f64_14xM[5 * M + 3 * i + 0] = w.com.x;
      f64_14xM[5 * M + 3 * i + 1] = w.com.y;
      f64_14xM[5 * M + 3 * i + 2] = w.com.z;
      for (int k = 0; k < 6; ++k) f64_14xM[8 * M + 6 * i + k] = t.f.iab[i][k];
    }
  }
  if (domain4) {
    domain4[0] = t.f.domain.center.x;
    domain4[1] = t.f.domain.center.y;
    domain4[2] = t.f.domain.center.z;
    domain4[3] = t.f.domain.half_width;
  }
  if (groups) std::memcpy(groups, t.f.groups.data(), t.f.groups.size() * sizeof(std::uint32_t));
}

// run_grouped_pass (grouped_ttg.h:297-323) on the handle's tree; acc[3*i]
// receives G*a of the i-th particle in Morton order.  Returns `missing`.
std::uint64_t bhref_walk(void* h, double theta, double eps2, double G, int use_quadrupole, std::uint32_t target_size,
                         double* acc) {
  ensure_runtime();
  auto& t = *static_cast<RefTree*>(h);
  bh::ForceParams fp;
  fp.theta = theta;
  fp.eps2 = eps2;
  fp.G = G;
  fp.use_quadrupole = use_quadrupole != 0;
  bh::Particle* base = t.f.particles.data();
  return bh::run_grouped_pass(t.f, fp, target_size, [acc, base](bh::Particle& p, const bh::Vec3& a) {
    std::size_t i = static_cast<std::size_t>(&p - base);
    acc[3 * i + 0] = a.x;
    acc[3 * i + 1] = a.y;
    acc[3 * i + 2] = a.z;
  });
}

// One step_particles call (integrate_ttg.h:66-148) on `particles` in place
// (Morton order on return).  group_size > 0: the grouped pass.  Returns 0,
// or 1 if the reference threw.
int bhref_step(void* particles, std::size_t n, double theta, double eps2, double G, int use_quadrupole,
               unsigned max_leaf, std::uint32_t group_size, std::uint32_t target_size, double kick_dt,
               double drift_dt, double* timing3) {
  ensure_runtime();
  bh::ForceParams fp;
  fp.theta = theta;
  fp.eps2 = eps2;
  fp.G = G;
  fp.use_quadrupole = use_quadrupole != 0;
  try {
    bh::StepTiming tm;
    auto out = bh::step_particles(to_vec(particles, n), fp, max_leaf, group_size, target_size, kick_dt, drift_dt, &tm);
    std::memcpy(particles, out.data(), n * sizeof(bh::Particle));
    if (timing3) {
      timing3[0] = tm.tree_build_ms;
      timing3[1] = tm.traversal_ms;
      timing3[2] = tm.exchange_ms;
    }
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// brute_force_accel (brute_force.h:15-28): G*a for every particle.
void bhref_brute(const void* particles, std::size_t n, double eps2, double G, double* acc) {
  auto a = bh::brute_force_accel(to_vec(particles, n), eps2, G);
  for (std::size_t i = 0; i < n; ++i) {
    acc[3 * i + 0] = a[i].x;
    acc[3 * i + 1] = a[i].y;
    acc[3 * i + 2] = a[i].z;
  }
}

// accel_from_source (multipole.h:171-200) for one (target, source) pair.
void bhref_accel_from_source(const double* target, double mass, const double* com, const double* iab6, double eps2,
                             int use_quadrupole, double G, double* out3) {
  bh::Sym3 s;
  for (int k = 0; k < 6; ++k) s[k] = iab6[k];
  auto a = bh::accel_from_source(bh::Vec3{target[0], target[1], target[2]}, mass, bh::Vec3{com[0], com[1], com[2]}, s,
                                 eps2, use_quadrupole != 0, G);
  out3[0] = a.x;
  out3[1] = a.y;
  out3[2] = a.z;
}

double bhref_kinetic(const void* particles, std::size_t n) { return bh::kinetic_energy(to_vec(particles, n)); }

// read_csv (io.cc): 0 and the particles (up to cap) with their count, or 1
// and the exception's message in err.
int bhref_read_csv(const char* path, void* out, std::size_t cap, std::size_t* n, char* err, std::size_t errcap) {
  try {
    const std::vector<bh::Particle> v = bh::read_csv(path);
    *n = v.size();
    std::memcpy(out, v.data(), std::min(cap, v.size()) * sizeof(bh::Particle));
    return 0;
  } catch (const std::exception& e) {
    if (errcap) {
      std::strncpy(err, e.what(), errcap - 1);
      err[errcap - 1] = 0;
    }
    return 1;
  }
}

// write_vtk (io.cc) of n particles to path.
int bhref_write_vtk(const char* path, const void* particles, std::size_t n) {
  try {
    bh::write_vtk(path, to_vec(particles, n));
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}
double bhref_potential(const void* particles, std::size_t n, double G) {
  return bh::potential_energy(to_vec(particles, n), G);
}

}  // extern "C"
