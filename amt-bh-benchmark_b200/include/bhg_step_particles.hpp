// bhg_step_particles.hpp - drop-in GPU replacement of the reference's
// bh::step_particles, grouped branch (integrate_ttg.h:66-148).
//
// The reference's step driver builds the flat tree (build_flat_tree,
// flat_build_ttg.h:276), runs the grouped pass with the kick/drift callback
// (run_grouped_pass, grouped_ttg.h:297; integrate_ttg.h:74-77) and hands the
// Morton-ordered particles back (integrate_ttg.h:107).  This header does the
// same through the C ABI of bhg.h: same signature (templated on the
// caller's Particle / ForceParams / StepTiming types so it compiles against
// the reference's own headers or any type with their layout), same meaning
// of every argument, result in Morton order, errors as C++ exceptions
// (std::runtime_error where the reference throws std::logic_error for a
// missing node, which a single-GPU tree cannot have).
#pragma once

#include "bhg.h"

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace bhg_host {

// GPU storage kept across steps (GroupedWorkspace, integrate_ttg.h:61-64).
class Workspace {
 public:
  explicit Workspace(int device = 0, std::uint64_t hbm_budget = 0) {
    bhg_config cfg{device, hbm_budget, 0};
    if (bhg_create(&ctx_, &cfg) != BHG_OK) throw std::runtime_error("bhg_create failed (no CUDA device?)");
  }
  ~Workspace() { bhg_destroy(ctx_); }
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;
  bhg_context* get() const { return ctx_; }

  void check(int rc) const {
    if (rc != BHG_OK) throw std::runtime_error(std::string("bhg: ") + bhg_last_error(ctx_));
  }

 private:
  bhg_context* ctx_ = nullptr;
};

// Walk arithmetic used by step_particles below (BHG_PRECISION_SPLIT:
// FP32 interactions with FP64 sums; BHG_PRECISION_FP64: all FP64).
inline int& default_precision() {
  static int p = BHG_PRECISION_SPLIT;
  return p;
}

template <class Particle, class ForceParams, class StepTiming>
std::vector<Particle> step_particles(std::vector<Particle> particles, const ForceParams& fp, unsigned max_leaf,
                                     std::uint32_t group_size, std::uint32_t target_size, double kick_dt,
                                     double drift_dt, StepTiming* timing = nullptr, Workspace* workspace = nullptr) {
  static_assert(sizeof(Particle) == sizeof(bh_particle64), "Particle must be the 64-byte bh::Particle record");
  static_assert(std::is_trivially_copyable_v<Particle>, "Particle must be trivially copyable");
  if (group_size == 0)
    throw std::invalid_argument("group_size 0 selects the reference's per-node pass; the GPU path is the grouped one");
  if (particles.empty()) {
    // the reference builds an empty tree (flat_build_ttg.h:215) and walks
    // nothing: the same empty vector comes back
    if (timing) timing->tree_build_ms = timing->traversal_ms = timing->exchange_ms = 0.0;
    return particles;
  }
  Workspace* ws = workspace;
  std::unique_ptr<Workspace> own;
  if (!ws) {
    own.reset(new Workspace());
    ws = own.get();
  }
  bhg_context* c = ws->get();
  bhg_force_params p{fp.theta, fp.eps2, fp.G, fp.use_quadrupole ? 1 : 0, default_precision()};
  ws->check(bhg_upload(c, reinterpret_cast<const bh_particle64*>(particles.data()), particles.size()));
  bhg_stats before{};
  if (timing) ws->check(bhg_get_stats(c, &before, 1));
  ws->check(bhg_step(c, &p, max_leaf, group_size, target_size, kick_dt, drift_dt));
  ws->check(bhg_download(c, reinterpret_cast<bh_particle64*>(particles.data())));
  if (timing) {
    bhg_stats st{};
    ws->check(bhg_get_stats(c, &st, 1));
    timing->tree_build_ms = st.pre_ms + st.sort_ms + st.tree_ms + st.multipole_ms + st.targets_ms;
    timing->traversal_ms = st.walk_ms;
    timing->exchange_ms = 0.0;
  }
  return particles;
}

}  // namespace bhg_host
