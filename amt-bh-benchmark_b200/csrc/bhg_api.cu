// The C ABI of include/bhg.h: contexts, device memory, the per-phase calls
// and the captured whole-step graph.
#include "bhg.h"
#include "bhg_kernels.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace bhg;

namespace {

// Phases of one evaluation, each timed with CUDA events and, in bhg_step,
// replayed from its own captured graph.
enum Phase { kPre, kSort, kTree, kMoments, kTargets, kWalk, kPhases };

}  // namespace

struct bhg_context {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint64_t budget = 0, allocated = 0;
  std::string err;

  // current problem: systems back to back, each with a handle
  size_t n = 0;
  int nsys = 0;
  std::vector<uint64_t> counts, ids;
  uint64_t next_id = 1;
  std::vector<SysDev> sys_host;
  std::vector<SysParam> prm_host;
  std::vector<Tile> tiles_host;   // bounds/keys tiles (kTile particles)
  std::vector<Tile> stiles_host;  // radix-sort tiles (sort_tile keys)
  uint32_t sort_tile = kSortTileLarge;
  std::vector<std::pair<void*, size_t>> allocs;

  // capacities (cap_n covers the scratch, cap_part the state; a capacity is
  // 0 after a growth that failed part-way)
  size_t cap_n = 0, cap_part = 0, cap_nodes = 0, cap_sys = 0, cap_tiles = 0, cap_stiles = 0;
  // the walk's per-warp lists of sources only some targets of a group take
  // (list_warps warps' worth), and the particle cap of a walk group
  void* list_buf = nullptr;
  size_t list_warps = 0;
  uint32_t walk_pack = kGroupMax;

  // device buffers
  Particle *part = nullptr, *staged = nullptr;
  double4* pm = nullptr;
  uint64_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t *hist = nullptr, *offs = nullptr, *sort_lb = nullptr;
  double* partial = nullptr;
  Tile *tiles = nullptr, *stiles = nullptr;
  SysDev* sys = nullptr;
  SysParam* prm = nullptr;
  Nodes nd{};
  uint32_t *level_lb = nullptr, *mark = nullptr, *targets = nullptr, *scan_lb = nullptr;
  uint32_t *groups = nullptr, *chunks = nullptr;
  double* accel = nullptr;
  std::vector<std::pair<void*, size_t>> text_scratch;  // cached buffers of the text calls
  DevState* st = nullptr;
  DevState* st_host = nullptr;  // pinned

  // phase state
  bool built = false, moments = false, walked = false;
  unsigned max_leaf = 16;
  uint32_t group_size = 256;
  int quad = 1, precision = 0;
  bool mask = false;

  // timing: CUDA events around every phase, summed on request
  struct Pending {
    int phase;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> ev_free, ev_all;
  std::vector<Pending> pending;
  cudaEvent_t open_ev = nullptr;  // boundary event after the last phase
  double tot_ms[kPhases] = {};
  double last_walk_ms = 0.0;
  uint32_t walks_timed = 0;

  // evaluations enqueued by bhg_step_systems_async since the last bhg_sync,
  // and the count of finished evaluations before them
  int async_pending = 0;
  uint32_t async_base = 0;

  // one evaluation (every phase) captured as one graph; its phase-boundary
  // events are event-record nodes, pointed at fresh events before each
  // launch (cap_ev: the placeholders recorded during capture)
  cudaGraph_t step_graph = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  std::string step_key;
  cudaGraphNode_t step_ev_node[kPhases + 1] = {};
  cudaEvent_t cap_ev[kPhases + 1] = {};
};

namespace {

int fail(bhg_context* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(c, BHG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int dev_alloc(bhg_context* c, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (c->budget && c->allocated + bytes > c->budget)
    return fail(c, BHG_ENOMEM, "HBM budget exceeded: need " + std::to_string(c->allocated + bytes) + " bytes of " +
                                   std::to_string(c->budget));
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(c, BHG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  c->allocated += bytes;
  c->allocs.push_back({*p, bytes});
  return BHG_OK;
}

void dev_free(bhg_context* c, void* p) {
  if (!p) return;
  for (size_t i = 0; i < c->allocs.size(); ++i) {
    if (c->allocs[i].first == p) {
      c->allocated -= c->allocs[i].second;
      c->allocs.erase(c->allocs.begin() + (long)i);
      break;
    }
  }
  cudaFree(p);
}

template <typename T>
int grow(bhg_context* c, T** p, size_t count) {
  dev_free(c, *p);
  *p = nullptr;
  return dev_alloc(c, reinterpret_cast<void**>(p), count * sizeof(T));
}

void drop_graph(bhg_context* c) {
  if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
  if (c->step_graph) cudaGraphDestroy(c->step_graph);
  c->step_exec = nullptr;
  c->step_graph = nullptr;
  c->step_key.clear();
}

// Device bytes of one node slot (the SoA arrays, the walk record, the cut
// lists) and of the slots one particle brings at max_leaf 16 (0.45 each).
constexpr size_t kNodeBytes = 16 + 32 + 32 + 48 + 64 + 8 + 48 + 8 + 12 + 4;
constexpr size_t kNodeBytesPerParticle = kNodeBytes * 45 / 100;
// Device bytes of the particle-sized buffers, per particle: the state and
// its staging copy, sources, sort keys and values, marks, accelerations.
constexpr size_t kParticleBytes = 2 * sizeof(Particle) + sizeof(double4) + 24 + 4 + 24;

// Node slots for n particles: about 0.25 per particle at max_leaf 16 on
// Plummer spheres, up to ~1.5 at max_leaf 1; grown on overflow.
size_t node_estimate(size_t n, int nsys, unsigned max_leaf) {
  double per = max_leaf <= 1 ? 2.2 : max_leaf <= 4 ? 1.2 : max_leaf <= 8 ? 0.7 : 0.45;
  return std::max<size_t>(1024, (size_t)(per * (double)n) + 64 * (size_t)nsys + 64);
}

int ensure_nodes(bhg_context* c, size_t need) {
  if (need <= c->cap_nodes) return BHG_OK;
  size_t cap = need;
  if (c->cap_nodes > 0) {  // systems come and go: grow with slack, within the budget
    const size_t want = std::max(need, c->cap_nodes + c->cap_nodes / 2);
    if (!c->budget || c->allocated + (want - c->cap_nodes) * kNodeBytes <= c->budget) cap = want;
  }
  drop_graph(c);
  c->cap_nodes = 0;  // until every array below exists again
  c->nd.cap = 0;
  int r;
  if ((r = grow(c, &c->nd.begin, cap)) || (r = grow(c, &c->nd.count, cap)) || (r = grow(c, &c->nd.first, cap)) ||
      (r = grow(c, &c->nd.info, cap)) || (r = grow(c, &c->nd.box, cap)) || (r = grow(c, &c->nd.mom, cap)) ||
      (r = grow(c, &c->nd.iab, cap * 6)) || (r = grow(c, &c->nd.w, cap)) || (r = grow(c, &c->nd.q45, cap)) ||
      (r = grow(c, &c->nd.q64, cap * 6)) || (r = grow(c, &c->nd.parent, cap)) || (r = grow(c, &c->nd.upcnt, cap)) ||
      (r = grow(c, &c->targets, cap)) || (r = grow(c, &c->groups, cap)) || (r = grow(c, &c->chunks, cap)) ||
      (r = grow(c, &c->level_lb, cap / 32 + kLevels + 8)))
    return r;
  c->nd.cap = (uint32_t)cap;
  c->cap_nodes = cap;
  return BHG_OK;
}

// Look-back words of the three compactions of the walk targets, groups and
// packing chunks (one word per 4096-item tile each, and some slack).
size_t scan_words(size_t n) { return 3 * (n / 4096) + 48; }

// Particle-sized buffers and the per-system tables for n particles.  The
// state (c->part) keeps its first c->n particles across a growth, so
// systems can be added to a resident set.  A growth that fails part-way
// leaves the state intact and the failed capacity at 0: the next call
// allocates that group of buffers again.
int ensure_particles(bhg_context* c, size_t n, int nsys, size_t ntiles, size_t nstiles) {
  int r;
  if (n > c->cap_n && c->cap_n > 0) {
    // systems are added one at a time: grow with slack, within the budget
    // (counting the node slots the extra particles bring too)
    const size_t want = std::max(n, c->cap_n + c->cap_n / 2);
    if (!c->budget || c->allocated + (want - c->cap_n) * (kParticleBytes + kNodeBytesPerParticle) <= c->budget)
      n = want;
  }
  if (n > c->cap_n) {
    // the scratch goes first, so that the state's old and new copies are
    // the only large buffers alive at once
    drop_graph(c);
    c->cap_n = 0;
    dev_free(c, c->accel), dev_free(c, c->staged), dev_free(c, c->pm), dev_free(c, c->mark), dev_free(c, c->scan_lb);
    c->accel = nullptr, c->staged = nullptr, c->pm = nullptr, c->mark = nullptr, c->scan_lb = nullptr;
    for (int k = 0; k < 2; ++k) {
      dev_free(c, c->keys[k]), dev_free(c, c->vals[k]);
      c->keys[k] = nullptr, c->vals[k] = nullptr;
    }
    if (n > c->cap_part) {
      Particle* np = nullptr;
      if ((r = dev_alloc(c, reinterpret_cast<void**>(&np), n * sizeof(Particle)))) return r;
      if (c->part && c->n) CK(cudaMemcpyAsync(np, c->part, c->n * sizeof(Particle), cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      dev_free(c, c->part);
      c->part = np;
      c->cap_part = n;
    }
    // the staging buffer trades places with the state (bhg_remove_systems):
    // both have the state's capacity
    if ((r = grow(c, &c->staged, c->cap_part)) || (r = grow(c, &c->pm, n)) ||
        (r = grow(c, &c->keys[0], n)) || (r = grow(c, &c->keys[1], n)) || (r = grow(c, &c->vals[0], n)) ||
        (r = grow(c, &c->vals[1], n)) || (r = grow(c, &c->mark, n)) || (r = grow(c, &c->scan_lb, scan_words(n))))
      return r;
    CK(cudaMemsetAsync(c->mark, 0xff, n * sizeof(uint32_t), c->stream));
    c->cap_n = n;
  }
  if ((size_t)nsys > c->cap_sys) {
    nsys = (int)std::max<size_t>((size_t)nsys, c->cap_sys + c->cap_sys / 2);
    drop_graph(c);
    c->cap_sys = 0;
    if ((r = grow(c, &c->sys, nsys)) || (r = grow(c, &c->prm, nsys)) ||
        (r = grow(c, &c->hist, (size_t)nsys * kSortPasses * 256)) || (r = grow(c, &c->offs, (size_t)nsys * kSortPasses * 256)))
      return r;
    c->cap_sys = nsys;
  }
  if (ntiles > c->cap_tiles) {
    ntiles = std::max(ntiles, c->cap_tiles + c->cap_tiles / 2);
    drop_graph(c);
    c->cap_tiles = 0;
    if ((r = grow(c, &c->tiles, ntiles)) || (r = grow(c, &c->partial, ntiles * 6))) return r;
    c->cap_tiles = ntiles;
  }
  if (nstiles > c->cap_stiles) {
    nstiles = std::max(nstiles, c->cap_stiles + c->cap_stiles / 2);
    drop_graph(c);
    c->cap_stiles = 0;
    if ((r = grow(c, &c->stiles, nstiles)) || (r = grow(c, &c->sort_lb, nstiles * kSortPasses * 256))) return r;
    c->cap_stiles = nstiles;
  }
  return BHG_OK;
}

// Keys per radix-sort tile: kSortTileSmall up to kSmallSortMax particles in
// the context (four times the blocks per pass where there are few tiles),
// kSortTileLarge above.  Measured per evaluation (4096- / 1024-key tiles): 1.034 /
// 1.037 ms at 65k, 1.633 / 1.559 at 131k, 2.755 / 2.792 at 262k.
constexpr size_t kSmallSortMax = 196608;

uint32_t sort_tile_keys(size_t n) { return n <= kSmallSortMax ? kSortTileSmall : kSortTileLarge; }

// Tiles of `tile` particles over systems of the given sizes.
size_t count_tiles(const std::vector<uint64_t>& counts, uint32_t tile) {
  size_t t = 0;
  for (uint64_t k : counts) t += (k + tile - 1) / tile;
  return t;
}

// Appends the tiles of one system of n particles starting at `begin`.
void push_tiles(std::vector<Tile>& out, uint32_t sys, uint32_t begin, uint32_t n, uint32_t tile) {
  const uint32_t first = (uint32_t)out.size();
  for (uint32_t o = 0; o < n; o += tile) out.push_back(Tile{sys, begin + o, std::min<uint32_t>(tile, n - o), first});
}

int walk_grid(bhg_context* c) {
  int per = walk_blocks_per_sm(c->precision, c->quad != 0, c->mask);
  return c->sms * per;
}

// The walk's list slots (walk_slot_bytes(), ~34 KB each): two per warp of
// the walk grid (161 MB on a 148-SM B200) - one list per warp in the one-pass
// schedule, one per group in the two-pass schedule, which therefore serves
// up to two groups per warp.  Allocated before the walk is captured
// (walk_grid has also set the kernels' shared-memory limit by then).  Under
// a tight HBM budget there are fewer slots and the walk runs on as many
// blocks as have a slot per warp (at least one block): a group's result does
// not depend on the warp that walks it nor on the schedule, so the bits are
// the same, only fewer groups at a time.
constexpr size_t kSlotsPerWarp = 2;

int ensure_walk_scratch(bhg_context* c, int grid) {
  const size_t per_slot = walk_slot_bytes();
  const size_t wpb = walk_threads() / 32;
  size_t slots = (size_t)grid * wpb * kSlotsPerWarp;
  if (c->list_warps >= slots) return BHG_OK;
  if (c->budget) {
    const size_t held = c->list_warps * per_slot;  // freed below, so it counts as room
    const size_t room = c->budget > c->allocated - held ? c->budget - (c->allocated - held) : 0;
    slots = std::min(slots, std::max(wpb, room / per_slot / wpb * wpb));
    if (c->list_warps >= slots) return BHG_OK;
  }
  drop_graph(c);
  dev_free(c, c->list_buf);
  c->list_buf = nullptr;
  c->list_warps = 0;
  int r = dev_alloc(c, &c->list_buf, slots * per_slot);
  if (r) return r;
  c->list_warps = slots;
  return BHG_OK;
}

// Blocks of the walk launch: the occupancy grid, or fewer when the HBM
// budget limited the slots (one per warp at least).
int walk_launch_grid(bhg_context* c) {
  return (int)std::min<size_t>((size_t)walk_grid(c), c->list_warps / (walk_threads() / 32));
}

// Lays out the systems c->counts back to back with their sort tiles, sizes
// the buffers for them (the state's first c->n particles survive a growth)
// and resets the per-step device state.  Per-system parameters stay with
// their systems; new systems get the defaults.
int finish_async(bhg_context* c);
int read_state(bhg_context* c);

int relayout(bhg_context* c) {
  if (c->async_pending) {  // the systems change: report the enqueued evaluations first
    int r = read_state(c);
    if (r || (r = finish_async(c))) return r;
  }
  const size_t nsys = c->counts.size();
  size_t n = 0;
  for (size_t s = 0; s < nsys; ++s) {
    if (c->counts[s] == 0) return fail(c, BHG_EINVAL, "system " + std::to_string(s) + " has no particles");
    n += c->counts[s];
  }
  if (n >= (1ull << 30)) return fail(c, BHG_EINVAL, "more than 2^30 - 1 particles");
  if (nsys > 65535) return fail(c, BHG_EINVAL, "more than 65535 systems");
  const uint32_t stile = sort_tile_keys(n);
  int r = ensure_particles(c, n, (int)std::max<size_t>(nsys, 1), std::max<size_t>(count_tiles(c->counts, kTile), 1),
                           std::max<size_t>(count_tiles(c->counts, stile), 1));
  if (r) return r;
  c->sys_host.assign(nsys, SysDev{});
  c->tiles_host.clear();
  c->stiles_host.clear();
  c->sort_tile = stile;
  uint32_t begin = 0;
  for (size_t s = 0; s < nsys; ++s) {
    SysDev& d = c->sys_host[s];
    d.begin = begin;
    d.n = (uint32_t)c->counts[s];
    d.root = (uint32_t)s;
    d.tile_begin = (uint32_t)c->tiles_host.size();
    push_tiles(c->tiles_host, (uint32_t)s, begin, d.n, kTile);
    d.tile_count = (uint32_t)c->tiles_host.size() - d.tile_begin;
    push_tiles(c->stiles_host, (uint32_t)s, begin, d.n, stile);
    begin += d.n;
  }
  if (c->n != n || c->nsys != (int)nsys) drop_graph(c);
  c->n = n;
  c->nsys = (int)nsys;
  c->prm_host.resize(nsys, SysParam{0.25, 0.0, 1.0, 0.0, 0.0, {0, 0, 0}});
  if (nsys) {
    CK(cudaMemcpyAsync(c->sys, c->sys_host.data(), nsys * sizeof(SysDev), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tiles, c->tiles_host.data(), c->tiles_host.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(c->stiles, c->stiles_host.data(), c->stiles_host.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                       c->stream));
  }
  // a new layout starts with clear error bits and per-build/per-walk fields;
  // the interaction totals and the evaluation count run on until reset
  CK(cudaMemsetAsync(&c->st->status, 0, sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(reinterpret_cast<char*>(c->st) + kBuildResetOffset, 0, sizeof(DevState) - kBuildResetOffset,
                     c->stream));
  c->built = c->moments = c->walked = false;
  return BHG_OK;
}

// A fresh set of systems (bhg_upload*): new handles, default parameters,
// nothing of the old state carried over.
int set_problem(bhg_context* c, const uint64_t* counts, size_t nsys) {
  if (nsys == 0) return fail(c, BHG_EINVAL, "no systems");
  c->counts.assign(counts, counts + nsys);
  c->ids.resize(nsys);
  for (size_t s = 0; s < nsys; ++s) c->ids[s] = c->next_id++;
  c->prm_host.clear();
  c->n = 0;
  return relayout(c);
}

// After a growth that failed part-way some scratch may be missing (its
// capacity is then 0): allocates it again before anything is launched.
int ensure_layout(bhg_context* c) {
  if (c->cap_n >= c->n && c->cap_sys >= c->counts.size() && c->cap_tiles >= c->tiles_host.size() &&
      c->cap_stiles >= c->stiles_host.size())
    return BHG_OK;
  return relayout(c);
}

// ---- enqueue the phases (no host synchronisation) ---------------------------

void enq_pre(bhg_context* c) {
  cudaStream_t s = c->stream;
  const int nt = (int)c->tiles_host.size();
  cudaMemsetAsync(reinterpret_cast<char*>(c->st) + kBuildResetOffset, 0, sizeof(DevState) - kBuildResetOffset, s);
  cudaMemsetAsync(c->hist, 0, (size_t)c->nsys * kSortPasses * 256 * sizeof(uint32_t), s);
  cudaMemsetAsync(c->sort_lb, 0, c->stiles_host.size() * kSortPasses * 256 * sizeof(uint32_t), s);
  cudaMemsetAsync(c->level_lb, 0, (c->cap_nodes / 32 + kLevels + 8) * sizeof(uint32_t), s);
  launch_bounds_domain(c->part, c->tiles, nt, c->sys, c->nsys, c->partial, c->st, s);
  launch_keys(c->part, c->tiles, nt, c->sys, c->nsys, c->keys[0], c->hist, c->offs, s);
}

void enq_sort(bhg_context* c) {
  const int nt = (int)c->stiles_host.size();
  for (int p = 0; p < kSortPasses; ++p)
    launch_sort_pass(c->keys[p & 1], c->vals[p & 1], c->keys[(p + 1) & 1], c->vals[(p + 1) & 1], p, c->stiles, nt,
                     (int)c->sort_tile, c->offs, c->sort_lb + (size_t)p * nt * 256, c->st, c->stream);
}

void enq_tree(bhg_context* c) {
  // kSortPasses is even: sorted keys and the permutation are back in [0]
  launch_gather(c->part, c->vals[0], (uint32_t)c->n, c->staged, c->pm, c->sms, c->stream);
  launch_topology(c->sys, c->nsys, c->nd, c->keys[0], c->max_leaf, (uint32_t)c->n, c->level_lb, c->st, c->sms,
                  c->stream);
}

// Multipoles in one launch up to this many particles (the per-level launches
// cost more than the work there), level by level above.  Measured on Plummer
// spheres (one launch / per level): 0.061 / 0.104 ms at 131k, 0.064 / 0.106
// at 262k, 0.116 / 0.114 at 524k, 0.200 / 0.144 at 1M, 0.81 / 0.33 at 4M.
constexpr size_t kMomentsOneLaunchMax = 393216;

void enq_moments(bhg_context* c) {
  launch_moments(c->nd, c->pm, c->st, c->sms, c->n <= kMomentsOneLaunchMax, c->stream);
}

void enq_targets(bhg_context* c, uint32_t target_size) {
  cudaStream_t s = c->stream;
  cudaMemsetAsync(reinterpret_cast<char*>(c->st) + kWalkResetOffset, 0, sizeof(DevState) - kWalkResetOffset, s);
  cudaMemsetAsync(c->scan_lb, 0, scan_words(c->n) * sizeof(uint32_t), s);
  const uint32_t lim = std::min(target_size, c->group_size);
  launch_targets(c->nd, lim, c->walk_pack, (uint32_t)c->n, c->mark, c->targets, c->chunks, c->groups, c->scan_lb, c->st,
                 c->sms, s);
}

void enq_walk(bhg_context* c, bool want_accel) {
  WalkArgs a;
  a.w = c->nd.w;
  a.q45 = c->nd.q45;
  a.q64 = c->nd.q64;
  a.mom = c->nd.mom;
  a.nbegin = c->nd.begin;
  a.ncount = c->nd.count;
  a.pm = c->pm;
  a.targets = c->targets;
  a.groups = c->groups;
  a.sys = c->sys;
  a.prm = c->prm;
  a.nsys = c->nsys;
  a.staged = c->staged;
  a.out = c->part;
  a.accel = want_accel ? c->accel : nullptr;
  a.st = c->st;
  // slots: the lists, then the groups' sums, then the list lengths
  a.nslots = (uint32_t)c->list_warps;
  a.wlist = static_cast<uint2*>(c->list_buf);
  a.gsum = reinterpret_cast<double*>(reinterpret_cast<char*>(c->list_buf) +
                                     c->list_warps * (walk_slot_bytes() - kGroupMax * 3 * sizeof(double) - sizeof(uint32_t)));
  a.gnl = reinterpret_cast<uint32_t*>(a.gsum + c->list_warps * kGroupMax * 3);
  // list lengths "pending" (bytes 0xfe): the two-pass schedule's target jobs
  // wait for their group's length
  cudaMemsetAsync(a.gnl, 0xfe, c->list_warps * sizeof(uint32_t), c->stream);
  launch_walk(a, c->precision, c->quad != 0, c->mask, walk_launch_grid(c), c->stream);
  launch_eval_done(c->st, c->stream);
}

// ---- phase timing -------------------------------------------------------------

cudaEvent_t take_event(bhg_context* c) {
  if (c->ev_free.empty()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    c->ev_all.push_back(e);
    return e;
  }
  cudaEvent_t e = c->ev_free.back();
  c->ev_free.pop_back();
  return e;
}

// Folds every recorded phase time into the sums (blocks) and recycles events.
void fold_times(bhg_context* c) {
  cudaStreamSynchronize(c->stream);
  for (const auto& p : c->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      c->tot_ms[p.phase] += ms;
      if (p.phase == kWalk) {
        c->last_walk_ms = ms;
        ++c->walks_timed;
      }
    } else {
      cudaGetLastError();
    }
  }
  c->pending.clear();
  c->ev_free = c->ev_all;
  c->open_ev = nullptr;
}

// Runs `enq` as phase `phase`, with a CUDA event before and after it on the
// stream (the per-phase calls; a whole evaluation runs as one graph, enq_step).
// NVTX range names of the phases (host-side enqueue ranges; a profiler shows
// the kernels under them)
const char* const kPhaseName[kPhases] = {"bhg pre", "bhg sort", "bhg tree", "bhg moments", "bhg targets", "bhg walk"};

struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

template <typename F>
int run_phase(bhg_context* c, int phase, F enq) {
  const NvtxRange range(kPhaseName[phase]);
  if (c->pending.size() > 16384) fold_times(c);
  if (!c->open_ev) {
    c->open_ev = take_event(c);
    CK(cudaEventRecord(c->open_ev, c->stream));
  }
  cudaEvent_t a = c->open_ev;
  enq();
  CK(cudaGetLastError());
  cudaEvent_t b = take_event(c);
  CK(cudaEventRecord(b, c->stream));
  c->pending.push_back({phase, a, b});
  c->open_ev = b;
  return BHG_OK;
}

std::string graph_key(const bhg_context* c, uint32_t target_size) {
  char key[192];
  snprintf(key, sizeof key, "%zu/%d/%zu/%zu/%u/%u/%u/%u/%d/%d/%d", c->n, c->nsys, c->cap_nodes, c->list_warps,
           c->walk_pack, c->max_leaf, c->group_size, target_size, c->precision, c->quad, (int)c->mask);
  return key;
}

// The three build phases (bhg_build_tree).
int run_build(bhg_context* c) {
  int r;
  if ((r = run_phase(c, kPre, [&] { enq_pre(c); })) || (r = run_phase(c, kSort, [&] { enq_sort(c); })) ||
      (r = run_phase(c, kTree, [&] { enq_tree(c); })))
    return r;
  return BHG_OK;
}

int push_params(bhg_context* c) {
  CK(cudaMemcpyAsync(c->prm, c->prm_host.data(), c->prm_host.size() * sizeof(SysParam), cudaMemcpyHostToDevice,
                     c->stream));
  c->open_ev = nullptr;  // the copy is not part of any phase
  return BHG_OK;
}

int read_state(bhg_context* c) {
  CK(cudaMemcpyAsync(c->st_host, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

std::string status_text(uint32_t s) {
  std::string t;
  if (s & kStNonFinite) t += " non-finite particle coordinate;";
  if (s & kStNodeOverflow) t += " octree larger than its node slots;";
  if (s & kStSpinLimit) t += " a bounded wait in a sort/scan kernel gave up;";
  if (s & kStTooLarge) t += " a count exceeded 30 bits;";
  if (s & kStWalkLimit) t += " a walk visited more nodes than the tree holds;";
  return t;
}

// After a synchronising read of the state: map sticky device errors to codes.
int check_status(bhg_context* c) {
  const uint32_t s = c->st_host->status;
  if (s == 0) return BHG_OK;
  if (s & kStNonFinite) return fail(c, BHG_ENONFINITE, "particle coordinates are not finite:" + status_text(s));
  return fail(c, BHG_EDEVICE, "device reported:" + status_text(s));
}

int clear_status(bhg_context* c) {
  CK(cudaMemsetAsync(c->st, 0, sizeof(uint32_t), c->stream));
  return BHG_OK;
}

int set_force_params(bhg_context* c, const bhg_force_params* fp, double kick, double drift, bool keep_per_system) {
  if (!fp) return fail(c, BHG_EINVAL, "null force params");
  if (!(fp->theta >= 0.0) || !(fp->eps2 >= 0.0) || !std::isfinite(fp->G))
    return fail(c, BHG_EINVAL, "theta and eps2 must be >= 0, G finite");
  if (fp->precision != BHG_PRECISION_SPLIT && fp->precision != BHG_PRECISION_FP64)
    return fail(c, BHG_EINVAL, "unknown precision");
  c->quad = fp->use_quadrupole ? 1 : 0;
  c->precision = fp->precision;
  for (auto& p : c->prm_host) {
    if (!keep_per_system) {
      p.theta2 = fp->theta * fp->theta;
      p.eps2 = fp->eps2;
      p.kick_dt = kick;
      p.drift_dt = drift;
    }
    p.G = fp->G;
  }
  // The r^2 = 0 self term is masked (accumulate_list, grouped_ttg.h:117-123)
  // when a walked system has no softening.  With per-system parameters the
  // systems' own eps2 decide, not fp->eps2: one unsoftened system among
  // softened ones needs the masked kernel (its self terms would be
  // rsqrt(0) = inf times 0 otherwise).
  bool mask = !(fp->eps2 > 0.0);
  if (keep_per_system) {
    mask = false;
    for (const auto& p : c->prm_host) mask = mask || !(p.eps2 > 0.0);
  }
  c->mask = mask;
  return BHG_OK;
}

}  // namespace

// ============================================================================

extern "C" {

int bhg_create(bhg_context** out, const bhg_config* cfg) {
  if (!out) return BHG_EINVAL;
  *out = nullptr;
  auto* c = new (std::nothrow) bhg_context;
  if (!c) return BHG_ENOMEM;
  c->device = cfg ? cfg->device : 0;
  c->budget = cfg ? cfg->hbm_budget : 0;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) {
    delete c;
    cudaGetLastError();
    return BHG_ECUDA;
  }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return BHG_ECUDA;
  }
  c->own_stream = true;
  set_build_attributes();
  if (dev_alloc(c, reinterpret_cast<void**>(&c->st), sizeof(DevState)) ||
      cudaMallocHost(&c->st_host, sizeof(DevState)) != cudaSuccess) {
    bhg_destroy(c);
    return BHG_ENOMEM;
  }
  cudaMemsetAsync(c->st, 0, sizeof(DevState), c->stream);
  std::memset(c->st_host, 0, sizeof(DevState));  // the host's copy of the (zero) device state
  *out = c;
  return BHG_OK;
}

int bhg_destroy(bhg_context* c) {
  if (!c) return BHG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graph(c);
  for (auto& a : c->allocs) cudaFree(a.first);
  c->allocs.clear();
  if (c->st_host) cudaFreeHost(c->st_host);
  for (auto& ev : c->ev_all)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->cap_ev)
    if (ev) cudaEventDestroy(ev);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BHG_OK;
}

const char* bhg_last_error(const bhg_context* c) { return c ? c->err.c_str() : "null context"; }

int bhg_set_stream(bhg_context* c, void* s) {
  if (!c) return BHG_EINVAL;
  cudaSetDevice(c->device);
  fold_times(c);
  drop_graph(c);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  if (s) {
    c->stream = static_cast<cudaStream_t>(s);
    c->own_stream = false;
  } else {
    cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    c->own_stream = true;
  }
  return BHG_OK;
}

static int upload_impl(bhg_context* c, const void* src, const uint64_t* counts, size_t nsys, cudaMemcpyKind kind) {
  if (!c || (!src && counts && counts[0])) return fail(c, BHG_EINVAL, "null argument");
  cudaSetDevice(c->device);
  int r = set_problem(c, counts, nsys);
  if (r) return r;
  CK(cudaMemcpyAsync(c->part, src, c->n * sizeof(Particle), kind, c->stream));
  return BHG_OK;
}

int bhg_upload(bhg_context* c, const bh_particle64* p, size_t n) {
  uint64_t cnt = n;
  return upload_impl(c, p, &cnt, 1, cudaMemcpyHostToDevice);
}

int bhg_upload_device(bhg_context* c, const void* p, size_t n) {
  uint64_t cnt = n;
  return upload_impl(c, p, &cnt, 1, cudaMemcpyDeviceToDevice);
}

int bhg_upload_systems(bhg_context* c, const bh_particle64* p, const uint64_t* counts, size_t nsys) {
  if (!counts) return fail(c, BHG_EINVAL, "null counts");
  return upload_impl(c, p, counts, nsys, cudaMemcpyHostToDevice);
}

int bhg_download(bhg_context* c, bh_particle64* out) {
  if (!c || !out) return fail(c, BHG_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CK(cudaMemcpyAsync(out, c->part, c->n * sizeof(Particle), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

int bhg_download_device(bhg_context* c, void* out) {
  if (!c || !out) return fail(c, BHG_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CK(cudaMemcpyAsync(out, c->part, c->n * sizeof(Particle), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

size_t bhg_num_particles(const bhg_context* c) { return c ? c->n : 0; }

}  // extern "C"

// Appends one system of n particles, written into the state by fill(dst);
// on failure the resident systems are untouched.
template <typename F>
static int add_system_impl(bhg_context* c, size_t n, uint64_t* id, F fill) {
  if (!c) return BHG_EINVAL;
  if (n == 0) return fail(c, BHG_EINVAL, "empty system");
  cudaSetDevice(c->device);
  const size_t old = c->n;
  c->counts.push_back(n);
  c->ids.push_back(c->next_id);
  const uint64_t handle = c->next_id;
  auto roll_back = [&](int code) {
    const std::string why = c->err;
    c->counts.pop_back();
    c->ids.pop_back();
    c->n = old;
    relayout(c);  // a failure here leaves capacities at 0, which the next call repairs
    return fail(c, code, why);
  };
  int r = relayout(c);
  if (r) return roll_back(r);
  // the handle is spent before the fill: a failed fill can never leave two
  // resident systems with one handle
  ++c->next_id;
  if ((r = fill(c->part + old))) return roll_back(r);
  if (id) *id = handle;
  return BHG_OK;
}

extern "C" {

int bhg_reserve(bhg_context* c, size_t particles, size_t systems) {
  if (!c) return BHG_EINVAL;
  if (particles >= (1ull << 30)) return fail(c, BHG_EINVAL, "more than 2^30 - 1 particles");
  if (systems == 0 || systems > 65535) return fail(c, BHG_EINVAL, "systems must be in 1 .. 65535");
  cudaSetDevice(c->device);
  const size_t n = std::max(particles, c->n);
  const size_t nsys = std::max(systems, c->counts.size());
  int r;
  const size_t nst = std::max(n / kSortTileLarge, std::min(n, kSmallSortMax) / kSortTileSmall) + nsys;
  if ((r = ensure_particles(c, n, (int)nsys, n / kTile + nsys, nst)) || (r = ensure_nodes(c, node_estimate(n, (int)nsys, 16))))
    return r;
  return BHG_OK;
}

int bhg_add_system(bhg_context* c, const bh_particle64* p, size_t n, uint64_t* id) {
  if (!c) return BHG_EINVAL;
  if (!p) return fail(c, BHG_EINVAL, "null particles");
  return add_system_impl(c, n, id, [&](Particle* dst) -> int {
    CK(cudaMemcpyAsync(dst, p, n * sizeof(Particle), cudaMemcpyHostToDevice, c->stream));
    return BHG_OK;
  });
}

int bhg_add_generated(bhg_context* c, const bhg_sphere* spheres, int nspheres, uint64_t seed, uint32_t id0,
                      uint64_t* id) {
  if (!c) return BHG_EINVAL;
  if (!spheres || nspheres < 1 || nspheres > 2) return fail(c, BHG_EINVAL, "one or two spheres");
  size_t n = 0;
  for (int k = 0; k < nspheres; ++k) {
    if (spheres[k].n == 0 || !(spheres[k].a > 0.0) || !(spheres[k].mass > 0.0))
      return fail(c, BHG_EINVAL, "a sphere needs n > 0, a > 0 and mass > 0");
    n += spheres[k].n;
  }
  return add_system_impl(c, n, id, [&](Particle* dst) -> int {
    size_t at = 0;
    for (int k = 0; k < nspheres; ++k) {
      const bhg_sphere& sp = spheres[k];
      // the second sphere draws from its own stream of the same seed
      launch_plummer(dst + at, (uint32_t)sp.n, sp.a, sp.mass, sp.centre, sp.bulk, id0 + (uint32_t)at,
                     seed + 0x9E3779B97F4A7C15ull * (uint64_t)k, c->sms, c->stream);
      at += sp.n;
    }
    CK(cudaGetLastError());
    return BHG_OK;
  });
}

int bhg_remove_systems(bhg_context* c, const uint64_t* handles, size_t k, bh_particle64* out) {
  if (!c) return BHG_EINVAL;
  if (!handles && k) return fail(c, BHG_EINVAL, "null handles");
  cudaSetDevice(c->device);
  std::vector<size_t> pos(k);
  std::vector<uint64_t> start(c->counts.size() + 1, 0);
  for (size_t s = 0; s < c->counts.size(); ++s) start[s + 1] = start[s] + c->counts[s];
  std::vector<char> gone(c->counts.size(), 0);
  for (size_t i = 0; i < k; ++i) {
    auto it = std::find(c->ids.begin(), c->ids.end(), handles[i]);
    if (it == c->ids.end()) return fail(c, BHG_EINVAL, "no system with handle " + std::to_string(handles[i]));
    pos[i] = (size_t)(it - c->ids.begin());
    if (gone[pos[i]]) return fail(c, BHG_EINVAL, "handle given twice");
    gone[pos[i]] = 1;
  }
  // the packing goes through the staging buffer, which a growth that failed
  // part-way may have left unallocated
  if (!c->staged && c->cap_part) {
    int r = dev_alloc(c, reinterpret_cast<void**>(&c->staged), c->cap_part * sizeof(Particle));
    if (r) return r;
  }
  if (out) {  // the removed systems' particles, back to back in the given order
    size_t at = 0;
    for (size_t i = 0; i < k; ++i) {
      const size_t s = pos[i];
      CK(cudaMemcpyAsync(out + at, c->part + start[s], c->counts[s] * sizeof(Particle), cudaMemcpyDeviceToHost,
                         c->stream));
      at += c->counts[s];
    }
  }
  // the kept systems, packed into the staging buffer, which becomes the state
  size_t at = 0;
  std::vector<uint64_t> counts, ids;
  std::vector<SysParam> prm;
  for (size_t s = 0; s < c->counts.size(); ++s) {
    if (gone[s]) continue;
    CK(cudaMemcpyAsync(c->staged + at, c->part + start[s], c->counts[s] * sizeof(Particle), cudaMemcpyDeviceToDevice,
                       c->stream));
    at += c->counts[s];
    counts.push_back(c->counts[s]);
    ids.push_back(c->ids[s]);
    prm.push_back(c->prm_host[s]);
  }
  std::swap(c->part, c->staged);
  c->counts = counts;
  c->ids = ids;
  c->prm_host = prm;
  c->n = at;
  drop_graph(c);  // the state moved to the other buffer
  int r = relayout(c);
  if (r) return r;
  if (out) CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

size_t bhg_num_systems(const bhg_context* c) { return c ? c->counts.size() : 0; }

}  // extern "C"

namespace {

// Device scratch of one text operation, freed on every way out.
// Device scratch of one text operation: the k-th buffer a call asks for is
// the context's k-th cached buffer, grown when too small and kept for the
// next call (repeated ingests allocate nothing).
struct Scratch {
  bhg_context* c;
  size_t k = 0;
  explicit Scratch(bhg_context* c_) : c(c_) {}
  template <typename T>
  int get(T** p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (k == c->text_scratch.size()) c->text_scratch.push_back({nullptr, 0});
    auto& slot = c->text_scratch[k++];
    if (slot.second < bytes) {
      dev_free(c, slot.first);
      slot = {nullptr, 0};
      int r = dev_alloc(c, &slot.first, bytes);
      if (r) return r;
      slot.second = bytes;
    }
    *p = static_cast<T*>(slot.first);
    return BHG_OK;
  }
};

// read_csv's header rule (io.cc:136-141): the first line is a header when its
// first field (after blanks) does not parse as an id.
bool csv_has_header(const char* text, size_t n) {
  const char* end = text + n;
  const char* eol = static_cast<const char*>(std::memchr(text, '\n', n));
  const char* lim = eol ? eol : end;
  const char* p = text;
  while (p < lim && (*p == ' ' || *p == '\t')) ++p;
  uint64_t v = 0;
  const char* q = p;
  while (q < lim && *q >= '0' && *q <= '9') {
    v = v * 10 + (uint64_t)(*q - '0');
    if (v > 0xffffffffull) return true;
    ++q;
  }
  return q == p;
}

// Parses CSV text (host memory, or device memory when on_device) on the
// device: *n_kept particle lines; *tmp/*keep/*m stay allocated in `sc` for
// the compaction.
int csv_parse(bhg_context* c, Scratch& sc, const char* text, size_t nbytes, bool on_device, Particle** tmp,
              uint32_t** keep, uint64_t* m, uint64_t* n_kept) {
  cudaStream_t s = c->stream;
  char* dtext = nullptr;
  uint32_t* tiles = nullptr;
  uint64_t* totals = nullptr;
  uint64_t* line_start = nullptr;
  unsigned long long* bad = nullptr;
  int r;
  if ((!on_device && (r = sc.get(&dtext, nbytes))) || (r = sc.get(&tiles, csv_tiles(nbytes))) ||
      (r = sc.get(&totals, 2)) || (r = sc.get(&bad, 1)))
    return r;
  // the header rule needs the first line only
  std::string head;
  if (on_device) {
    dtext = const_cast<char*>(text);
    head.resize(std::min<size_t>(nbytes, 65536));
    if (!head.empty()) CK(cudaMemcpyAsync(&head[0], text, head.size(), cudaMemcpyDeviceToHost, s));
  } else if (nbytes) {
    CK(cudaMemcpyAsync(dtext, text, nbytes, cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemsetAsync(totals, 0, 2 * sizeof(uint64_t), s));
  CK(cudaMemsetAsync(bad, 0xff, sizeof(unsigned long long), s));
  launch_csv_count(dtext, nbytes, tiles, totals, s);
  CK(cudaGetLastError());
  uint64_t h[2] = {0, 0};
  CK(cudaMemcpyAsync(h, totals, sizeof h, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint64_t nlines = h[0] + 1;
  if ((r = sc.get(&line_start, nlines))) return r;
  CK(cudaMemsetAsync(line_start, 0, sizeof(uint64_t), s));
  launch_csv_emit(dtext, nbytes, tiles, line_start, s);
  const uint64_t first =
      nbytes && (on_device ? csv_has_header(head.data(), head.size()) : csv_has_header(text, nbytes)) ? 1 : 0;
  *m = nlines > first ? nlines - first : 0;
  uint32_t* block_count = nullptr;
  if ((r = sc.get(tmp, *m)) || (r = sc.get(keep, *m)) || (r = sc.get(&block_count, csv_keep_blocks(*m)))) return r;
  launch_csv_parse(dtext, nbytes, line_start, first, nlines, *tmp, *keep, bad, c->sms, s);
  launch_csv_compact(*tmp, *keep, *m, block_count, totals + 1, nullptr, s);
  CK(cudaGetLastError());
  unsigned long long hb = 0;
  CK(cudaMemcpyAsync(&hb, bad, sizeof hb, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h, totals, sizeof h, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hb != ~0ull) {  // the first malformed line, as read_csv reports it
    uint64_t ls[2] = {0, nbytes + 1};
    CK(cudaMemcpy(ls, line_start + hb, (hb + 1 < nlines ? 2 : 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    const size_t b = (size_t)ls[0], e = std::min<size_t>((size_t)ls[1] - 1, nbytes);
    std::string line(e > b ? std::min<size_t>(e - b, 4096) : 0, '\0');
    if (!line.empty()) CK(cudaMemcpy(&line[0], dtext + b, line.size(), cudaMemcpyDeviceToHost));
    return fail(c, BHG_EINVAL, "malformed line " + std::to_string(hb + 1) + ": '" + line + "'");
  }
  *n_kept = h[1];
  return BHG_OK;
}

}  // namespace

extern "C" {

static int upload_csv_impl(bhg_context* c, const char* text, size_t nbytes, bool on_device) {
  if (!c) return BHG_EINVAL;
  if (!text && nbytes) return fail(c, BHG_EINVAL, "null text");
  cudaSetDevice(c->device);
  Scratch sc(c);
  Particle* tmp = nullptr;
  uint32_t* keep = nullptr;
  uint64_t m = 0, n = 0;
  int r = csv_parse(c, sc, text, nbytes, on_device, &tmp, &keep, &m, &n);
  if (r) return r;
  if (n == 0) return fail(c, BHG_EINVAL, "no particles in the text");
  const uint64_t cnt = n;
  if ((r = set_problem(c, &cnt, 1))) return r;
  uint32_t* block_count = nullptr;
  uint64_t* total = nullptr;
  if ((r = sc.get(&block_count, csv_keep_blocks(m))) || (r = sc.get(&total, 1))) return r;
  launch_csv_compact(tmp, keep, m, block_count, total, c->part, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

int bhg_upload_csv(bhg_context* c, const char* text, size_t nbytes) { return upload_csv_impl(c, text, nbytes, false); }

int bhg_upload_csv_device(bhg_context* c, const void* text, size_t nbytes) {
  return upload_csv_impl(c, static_cast<const char*>(text), nbytes, true);
}

int bhg_add_csv(bhg_context* c, const char* text, size_t nbytes, uint64_t* id) {
  if (!c) return BHG_EINVAL;
  if (!text && nbytes) return fail(c, BHG_EINVAL, "null text");
  cudaSetDevice(c->device);
  Scratch sc(c);
  Particle* tmp = nullptr;
  uint32_t* keep = nullptr;
  uint64_t m = 0, n = 0;
  int r = csv_parse(c, sc, text, nbytes, false, &tmp, &keep, &m, &n);
  if (r) return r;
  if (n == 0) return fail(c, BHG_EINVAL, "no particles in the text");
  uint32_t* block_count = nullptr;
  uint64_t* total = nullptr;
  if ((r = sc.get(&block_count, csv_keep_blocks(m))) || (r = sc.get(&total, 1))) return r;
  r = add_system_impl(c, n, id, [&](Particle* dst) -> int {
    launch_csv_compact(tmp, keep, m, block_count, total, dst, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return BHG_OK;
  });
  return r;
}

int bhg_snapshot_vtk(bhg_context* c, uint64_t handle, char* out, size_t cap, size_t* len) {
  if (!c || !len) return BHG_EINVAL;
  cudaSetDevice(c->device);
  auto it = std::find(c->ids.begin(), c->ids.end(), handle);
  if (it == c->ids.end()) return fail(c, BHG_EINVAL, "no system with handle " + std::to_string(handle));
  const size_t sidx = (size_t)(it - c->ids.begin());
  size_t start = 0;
  for (size_t k = 0; k < sidx; ++k) start += c->counts[k];
  const uint32_t n = (uint32_t)c->counts[sidx];
  Scratch sc(c);
  char* slots = nullptr;
  uint32_t* lens = nullptr;
  uint32_t* bsum = nullptr;
  uint64_t* boff = nullptr;
  uint64_t* totals = nullptr;
  int r;
  if ((r = sc.get(&slots, vtk_slot_bytes(n))) || (r = sc.get(&lens, 3 * (size_t)n)) ||
      (r = sc.get(&bsum, 3 * vtk_blocks(n))) || (r = sc.get(&boff, 3 * vtk_blocks(n))) || (r = sc.get(&totals, 3)))
    return r;
  launch_vtk_format(c->part + start, n, slots, lens, bsum, boff, totals, c->sms, c->stream);
  CK(cudaGetLastError());
  uint64_t t[3];
  CK(cudaMemcpyAsync(t, totals, sizeof t, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // write_vtk's layout (io.cc:180-195)
  const std::string h0 = "# vtk DataFile Version 3.0\npepc-ttg particle snapshot\nASCII\nDATASET POLYDATA\nPOINTS " +
                         std::to_string(n) + " double\n";
  const std::string h1 = "POINT_DATA " + std::to_string(n) + "\nSCALARS mass double 1\nLOOKUP_TABLE default\n";
  const std::string h2 = "VECTORS velocity double\n";
  const size_t total = h0.size() + t[0] + h1.size() + t[1] + h2.size() + t[2];
  *len = total;
  if (!out) return BHG_OK;
  if (cap < total) return fail(c, BHG_EINVAL, "buffer too small: the snapshot needs " + std::to_string(total) + " bytes");
  char* dev = nullptr;
  if ((r = sc.get(&dev, t[0] + t[1] + t[2]))) return r;
  char* sect[3] = {dev, dev + t[0], dev + t[0] + t[1]};
  launch_vtk_gather(slots, n, lens, boff, sect, c->stream);
  CK(cudaGetLastError());
  const std::string* head[3] = {&h0, &h1, &h2};
  size_t at = 0;
  for (int k = 0; k < 3; ++k) {
    std::memcpy(out + at, head[k]->data(), head[k]->size());
    at += head[k]->size();
    if (t[k]) CK(cudaMemcpyAsync(out + at, sect[k], t[k], cudaMemcpyDeviceToHost, c->stream));
    at += t[k];
  }
  CK(cudaStreamSynchronize(c->stream));
  return BHG_OK;
}

int bhg_system_ids(const bhg_context* c, uint64_t* out) {
  if (!c || !out) return BHG_EINVAL;
  std::copy(c->ids.begin(), c->ids.end(), out);
  return BHG_OK;
}

int bhg_build_tree(bhg_context* c, unsigned max_leaf, uint32_t group_size) {
  if (!c) return BHG_EINVAL;
  if (c->n == 0) return fail(c, BHG_ESTATE, "no particles uploaded");
  if (max_leaf == 0) return fail(c, BHG_EINVAL, "max_leaf must be >= 1");
  cudaSetDevice(c->device);
  int r = ensure_layout(c);
  if (r) return r;
  c->max_leaf = max_leaf;
  c->group_size = group_size;
  if ((r = ensure_nodes(c, node_estimate(c->n, c->nsys, max_leaf)))) return r;
  for (int attempt = 0; attempt < 8; ++attempt) {
    if ((r = run_build(c))) return r;
    if ((r = read_state(c))) return r;
    if (c->st_host->status & kStNodeOverflow) {
      size_t need = std::max<size_t>(2 * c->cap_nodes, (size_t)c->st_host->n_nodes + c->st_host->n_nodes / 4 + 64);
      if ((r = clear_status(c)) || (r = ensure_nodes(c, need))) return r;
      continue;
    }
    if ((r = check_status(c))) {
      clear_status(c);
      return r;
    }
    c->built = true;
    c->moments = c->walked = false;
    return BHG_OK;
  }
  return fail(c, BHG_EDEVICE, "octree kept outgrowing its node slots");
}

int bhg_compute_multipoles(bhg_context* c) {
  if (!c) return BHG_EINVAL;
  if (!c->built) return fail(c, BHG_ESTATE, "build the tree first");
  cudaSetDevice(c->device);
  int r = run_phase(c, kMoments, [&] { enq_moments(c); });
  if (r) return r;
  c->moments = true;
  return BHG_OK;
}

int bhg_walk_forces(bhg_context* c, const bhg_force_params* fp, uint32_t target_size, double kick_dt,
                    double drift_dt, double* accel_out, uint64_t* missing) {
  if (!c) return BHG_EINVAL;
  if (!c->moments) return fail(c, BHG_ESTATE, "compute the multipoles first");
  cudaSetDevice(c->device);
  int r = set_force_params(c, fp, kick_dt, drift_dt, false);
  if (r) return r;
  if (!c->accel && (r = grow(c, &c->accel, c->cap_n * 3))) return r;
  if ((r = ensure_walk_scratch(c, walk_grid(c))) || (r = push_params(c))) return r;
  if ((r = run_phase(c, kTargets, [&] { enq_targets(c, target_size); })) ||
      (r = run_phase(c, kWalk, [&] { enq_walk(c, true); })))
    return r;
  c->walked = true;
  c->moments = false;  // the state moved: the next walk needs a new build
  c->built = false;
  if (missing) *missing = 0;
  if ((r = read_state(c))) return r;
  if ((r = check_status(c))) {
    clear_status(c);
    return r;
  }
  if (accel_out) {
    CK(cudaMemcpyAsync(accel_out, c->accel, c->n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return BHG_OK;
}

int bhg_integrate(bhg_context* c, double kick_dt, double drift_dt) {
  if (!c) return BHG_EINVAL;
  if (!c->walked || !c->accel) return fail(c, BHG_ESTATE, "walk forces first");
  cudaSetDevice(c->device);
  for (auto& p : c->prm_host) {
    p.kick_dt = kick_dt;
    p.drift_dt = drift_dt;
  }
  int r = push_params(c);
  if (r) return r;
  launch_integrate(c->part, c->accel, (uint32_t)c->n, c->sys, c->prm, c->nsys, c->sms, c->stream);
  CK(cudaGetLastError());
  return BHG_OK;
}

int bhg_set_system_params(bhg_context* c, const double* theta, const double* eps2, const double* kick_dt,
                          const double* drift_dt) {
  if (!c) return BHG_EINVAL;
  for (int s = 0; s < c->nsys; ++s) {
    SysParam& p = c->prm_host[s];
    if (theta) p.theta2 = theta[s] * theta[s];
    if (eps2) p.eps2 = eps2[s];
    if (kick_dt) p.kick_dt = kick_dt[s];
    if (drift_dt) p.drift_dt = drift_dt[s];
  }
  return BHG_OK;
}

}  // extern "C"

namespace {

// One whole evaluation (build + multipoles + targets + walk) as ONE graph
// launch: captured once per problem shape, replayed after.  An event-record
// node sits at every phase boundary; before each launch they are pointed at
// fresh events (cudaGraphExecEventRecordNodeSetEvent, which leaves launches
// already in flight alone), so the phase times of every evaluation are still
// CUDA-event times on the context's stream.
int enq_step(bhg_context* c, uint32_t target_size) {
  const NvtxRange range("bhg step");
  const std::string key = graph_key(c, target_size);
  if (c->pending.size() > 16384) fold_times(c);
  if (!c->step_exec || c->step_key != key) {
    drop_graph(c);
    for (int i = 0; i <= kPhases; ++i)
      if (!c->cap_ev[i]) CK(cudaEventCreate(&c->cap_ev[i]));
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaEventRecordWithFlags(c->cap_ev[kPre], c->stream, cudaEventRecordExternal);
    enq_pre(c);
    cudaEventRecordWithFlags(c->cap_ev[kSort], c->stream, cudaEventRecordExternal);
    enq_sort(c);
    cudaEventRecordWithFlags(c->cap_ev[kTree], c->stream, cudaEventRecordExternal);
    enq_tree(c);
    cudaEventRecordWithFlags(c->cap_ev[kMoments], c->stream, cudaEventRecordExternal);
    enq_moments(c);
    cudaEventRecordWithFlags(c->cap_ev[kTargets], c->stream, cudaEventRecordExternal);
    enq_targets(c, target_size);
    cudaEventRecordWithFlags(c->cap_ev[kWalk], c->stream, cudaEventRecordExternal);
    enq_walk(c, false);
    cudaEventRecordWithFlags(c->cap_ev[kPhases], c->stream, cudaEventRecordExternal);
    CK(cudaStreamEndCapture(c->stream, &g));
    // the event-record nodes (recorded as external events, so that capture
    // turns them into nodes), known by the placeholder event each records
    size_t nn = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(g, nodes.data(), &nn));
    for (int i = 0; i <= kPhases; ++i) c->step_ev_node[i] = nullptr;
    for (cudaGraphNode_t node : nodes) {
      cudaGraphNodeType t;
      CK(cudaGraphNodeGetType(node, &t));
      if (t != cudaGraphNodeTypeEventRecord) continue;
      cudaEvent_t e = nullptr;
      CK(cudaGraphEventRecordNodeGetEvent(node, &e));
      for (int i = 0; i <= kPhases; ++i)
        if (e == c->cap_ev[i]) c->step_ev_node[i] = node;
    }
    for (int i = 0; i <= kPhases; ++i)
      if (!c->step_ev_node[i]) {
        cudaGraphDestroy(g);
        return fail(c, BHG_ECUDA, "captured evaluation graph lacks a phase event");
      }
    cudaError_t e = cudaGraphInstantiate(&c->step_exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      c->step_exec = nullptr;
      return fail(c, BHG_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    c->step_graph = g;
    c->step_key = key;
  }
  cudaEvent_t ev[kPhases + 1];
  for (int i = 0; i <= kPhases; ++i) {
    ev[i] = take_event(c);
    CK(cudaGraphExecEventRecordNodeSetEvent(c->step_exec, c->step_ev_node[i], ev[i]));
  }
  CK(cudaGraphLaunch(c->step_exec, c->stream));
  for (int p = 0; p < kPhases; ++p) c->pending.push_back({p, ev[p], ev[p + 1]});
  c->open_ev = ev[kPhases];
  return BHG_OK;
}

int prepare_step(bhg_context* c, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                 double kick, double drift, bool keep) {
  if (c->n == 0) return fail(c, BHG_ESTATE, "no particles uploaded");
  if (max_leaf == 0) return fail(c, BHG_EINVAL, "max_leaf must be >= 1");
  cudaSetDevice(c->device);
  int r = set_force_params(c, fp, kick, drift, keep);
  if (r || (r = ensure_layout(c))) return r;
  if (c->max_leaf != max_leaf || c->group_size != group_size) drop_graph(c);
  c->max_leaf = max_leaf;
  c->group_size = group_size;
  if ((r = ensure_nodes(c, node_estimate(c->n, c->nsys, max_leaf))) || (r = ensure_walk_scratch(c, walk_grid(c))))
    return r;
  return BHG_OK;
}

// The node slots an overflowed build asked for, with room to spare.
size_t regrown_nodes(const bhg_context* c) {
  return std::max<size_t>(2 * c->cap_nodes, (size_t)c->st_host->n_nodes + c->st_host->n_nodes / 4 + 64);
}

// Reports the evaluations enqueued by bhg_step_systems_async (the device
// state has just been read).
int finish_async(bhg_context* c) {
  const int pending = c->async_pending;
  c->async_pending = 0;
  if (pending == 0) return BHG_OK;
  const uint32_t ran = c->st_host->evals_ok - c->async_base;
  const uint32_t st = c->st_host->status;
  if (st == 0) {
    c->walked = true;
    c->built = c->moments = false;
    return BHG_OK;
  }
  int r;
  if (st & kStNodeOverflow) {
    if ((r = clear_status(c)) || (r = ensure_nodes(c, regrown_nodes(c))) || (r = ensure_walk_scratch(c, walk_grid(c))))
      return r;
    return fail(c, BHG_EAGAIN, std::to_string(ran) + " of " + std::to_string(pending) +
                                   " evaluations ran: the octree outgrew its node slots (now grown)");
  }
  r = check_status(c);
  clear_status(c);
  return r;
}

// Runs evaluations i0 .. i1-1 of a schedule given by kick/drift per
// evaluation; on a node overflow grows the slots and resumes from the
// evaluation that failed (its walk was skipped, so the state is intact).
int run_evals(bhg_context* c, uint32_t target_size, const std::vector<std::pair<double, double>>& kd, bool keep) {
  size_t next = 0;
  for (int attempt = 0; attempt < 8; ++attempt) {
    int r;
    // the host's copy of the device state is current unless asynchronous
    // evaluations are still out (every other path that runs a walk ends by
    // reading it): no blocking read before the evaluations are enqueued
    if (c->async_pending && ((r = read_state(c)) || (r = finish_async(c)))) return r;
    const uint32_t base = c->st_host->evals_ok;
    for (size_t i = next; i < kd.size(); ++i) {
      if (!keep) {
        for (auto& p : c->prm_host) {
          p.kick_dt = kd[i].first;
          p.drift_dt = kd[i].second;
        }
      }
      if ((r = push_params(c)) || (r = enq_step(c, target_size))) return r;
    }
    if ((r = read_state(c))) return r;
    const uint32_t done = c->st_host->evals_ok - base;
    if (c->st_host->status == 0) {
      c->walked = true;
      c->built = c->moments = false;
      return BHG_OK;
    }
    if (c->st_host->status & kStNodeOverflow) {
      next += done;
      if ((r = clear_status(c)) || (r = ensure_nodes(c, regrown_nodes(c))) || (r = ensure_walk_scratch(c, walk_grid(c))))
        return r;
      continue;
    }
    r = check_status(c);
    clear_status(c);
    return r;
  }
  return fail(c, BHG_EDEVICE, "octree kept outgrowing its node slots");
}

}  // namespace

extern "C" {

int bhg_step(bhg_context* c, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
             uint32_t target_size, double kick_dt, double drift_dt) {
  if (!c) return BHG_EINVAL;
  int r = prepare_step(c, fp, max_leaf, group_size, kick_dt, drift_dt, false);
  if (r) return r;
  return run_evals(c, target_size, {{kick_dt, drift_dt}}, false);
}

int bhg_step_systems(bhg_context* c, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                     uint32_t target_size) {
  if (!c) return BHG_EINVAL;
  int r = prepare_step(c, fp, max_leaf, group_size, 0.0, 0.0, true);
  if (r) return r;
  return run_evals(c, target_size, {{0.0, 0.0}}, true);
}

int bhg_step_systems_async(bhg_context* c, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                           uint32_t target_size) {
  if (!c) return BHG_EINVAL;
  int r = prepare_step(c, fp, max_leaf, group_size, 0.0, 0.0, true);
  if (r) return r;
  if (c->async_pending == 0) c->async_base = c->st_host->evals_ok;  // current: read at the last sync
  if ((r = push_params(c)) || (r = enq_step(c, target_size))) return r;
  ++c->async_pending;
  return BHG_OK;
}

int bhg_download_async(bhg_context* c, bh_particle64* out) {
  if (!c || !out) return fail(c, BHG_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CK(cudaMemcpyAsync(out, c->part, c->n * sizeof(Particle), cudaMemcpyDeviceToHost, c->stream));
  return BHG_OK;
}

int bhg_sync(bhg_context* c) {
  if (!c) return BHG_EINVAL;
  cudaSetDevice(c->device);
  int r = read_state(c);
  if (r) return r;
  return finish_async(c);
}

int bhg_run_schedule(bhg_context* c, const bhg_force_params* fp, unsigned max_leaf, uint32_t group_size,
                     uint32_t target_size, double dt, int steps) {
  if (!c) return BHG_EINVAL;
  if (steps < 1) return fail(c, BHG_EINVAL, "steps must be >= 1");
  int r = prepare_step(c, fp, max_leaf, group_size, dt / 2.0, dt, false);
  if (r) return r;
  std::vector<std::pair<double, double>> kd;
  kd.push_back({dt / 2.0, dt});                                 // main.cc:206-208
  for (int s = 1; s < steps; ++s) kd.push_back({dt, dt});       // main.cc:219-222
  kd.push_back({dt / 2.0, 0.0});                                // main.cc:240-242
  return run_evals(c, target_size, kd, false);
}

int bhg_get_stats(bhg_context* c, bhg_stats* out, int reset) {
  if (!c || !out) return BHG_EINVAL;
  cudaSetDevice(c->device);
  fold_times(c);
  int r = read_state(c);
  if (r) return r;
  std::memset(out, 0, sizeof *out);
  out->pre_ms = c->tot_ms[kPre];
  out->sort_ms = c->tot_ms[kSort];
  out->tree_ms = c->tot_ms[kTree];
  out->multipole_ms = c->tot_ms[kMoments];
  out->targets_ms = c->tot_ms[kTargets];
  out->walk_ms = c->tot_ms[kWalk];
  out->last_walk_ms = c->last_walk_ms;
  out->evals = c->walks_timed;
  out->pp = c->st_host->pp_total;
  out->pc = c->st_host->pc_total;
  out->nodes = c->st_host->n_nodes;
  out->targets = c->st_host->n_targets;
  out->depth = c->st_host->max_depth;
  out->sort_passes = kSortPasses;
  // bounds + domain + keys + digit offsets; the sort passes; gather + roots +
  // one per level; the multipoles (one kernel, or one per level); mark +
  // compact of the targets, of the packing chunks, packing + compact of the
  // walk groups; the walk and its completion count
  out->kernels_per_eval = 4 + kSortPasses + (2 + kMortonDepth) + (c->n <= kMomentsOneLaunchMax ? 1 : kMortonDepth + 1) + 6 +
                          2;
  if (reset) {
    for (double& t : c->tot_ms) t = 0.0;
    c->walks_timed = 0;
    CK(cudaMemsetAsync(&c->st->pp_total, 0, 2 * sizeof(unsigned long long), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return BHG_OK;
}

int bhg_device_status(bhg_context* c, uint32_t* status) {
  if (!c || !status) return BHG_EINVAL;
  cudaSetDevice(c->device);
  int r = read_state(c);
  if (r) return r;
  *status = c->st_host->status;
  return BHG_OK;
}

int bhg_debug_export(bhg_context* c, int what, void* out, size_t bytes, size_t* written) {
  if (!c) return BHG_EINVAL;
  cudaSetDevice(c->device);
  int r = read_state(c);
  if (r) return r;
  const size_t nn = std::min<size_t>(c->st_host->n_nodes, c->cap_nodes);
  std::vector<char> buf;
  auto get = [&](const void* src, size_t b, size_t at) -> int {
    CK(cudaMemcpy(buf.data() + at, src, b, cudaMemcpyDeviceToHost));
    return BHG_OK;
  };
  switch (what) {
    case BHG_EXPORT_KEYS:
      buf.resize(c->n * 8);
      if ((r = get(c->keys[0], buf.size(), 0))) return r;
      break;
    case BHG_EXPORT_PERM:
      buf.resize(c->n * 4);
      if ((r = get(c->vals[0], buf.size(), 0))) return r;
      break;
    case BHG_EXPORT_NODES_U32: {
      buf.resize(nn * 24);
      if ((r = get(c->nd.begin, nn * 4, 0)) || (r = get(c->nd.count, nn * 4, nn * 4)) ||
          (r = get(c->nd.first, nn * 4, nn * 8)))
        return r;
      std::vector<uint32_t> info(nn);
      CK(cudaMemcpy(info.data(), c->nd.info, nn * 4, cudaMemcpyDeviceToHost));
      uint32_t* u = reinterpret_cast<uint32_t*>(buf.data());
      for (size_t i = 0; i < nn; ++i) {
        u[3 * nn + i] = info_nchild(info[i]);
        u[4 * nn + i] = info_leaf(info[i]) ? 1u : 0u;
        u[5 * nn + i] = info_depth(info[i]);
        if (u[4 * nn + i]) u[2 * nn + i] = 0;  // first_child of a leaf
      }
      break;
    }
    case BHG_EXPORT_NODES_F64: {
      buf.resize(nn * 14 * 8);
      std::vector<double4> box(nn), mom(nn);
      std::vector<double> iab(nn * 6);
      CK(cudaMemcpy(box.data(), c->nd.box, nn * sizeof(double4), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(mom.data(), c->nd.mom, nn * sizeof(double4), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(iab.data(), c->nd.iab, nn * 48, cudaMemcpyDeviceToHost));
      double* d = reinterpret_cast<double*>(buf.data());
      for (size_t i = 0; i < nn; ++i) {
        double* o = d + 14 * i;
        o[0] = box[i].x, o[1] = box[i].y, o[2] = box[i].z, o[3] = box[i].w;
        o[4] = mom[i].w, o[5] = mom[i].x, o[6] = mom[i].y, o[7] = mom[i].z;
        for (int k = 0; k < 6; ++k) o[8 + k] = iab[6 * i + k];
      }
      break;
    }
    case BHG_EXPORT_DOMAINS: {
      std::vector<SysDev> sd(c->nsys);
      CK(cudaMemcpy(sd.data(), c->sys, c->nsys * sizeof(SysDev), cudaMemcpyDeviceToHost));
      buf.resize((size_t)c->nsys * 32);
      double* d = reinterpret_cast<double*>(buf.data());
      for (int s = 0; s < c->nsys; ++s) d[4 * s] = sd[s].cx, d[4 * s + 1] = sd[s].cy, d[4 * s + 2] = sd[s].cz, d[4 * s + 3] = sd[s].hw;
      break;
    }
    case BHG_EXPORT_TARGETS:
      buf.resize((size_t)c->st_host->n_targets * 4);
      if ((r = get(c->targets, buf.size(), 0))) return r;
      break;
    case BHG_EXPORT_GROUPS:
      buf.resize((size_t)c->st_host->n_groups * 4);
      if ((r = get(c->groups, buf.size(), 0))) return r;
      break;
    case BHG_EXPORT_ACCEL:
      if (!c->accel) return fail(c, BHG_ESTATE, "no accelerations stored (bhg_walk_forces stores them)");
      buf.resize(c->n * 24);
      if ((r = get(c->accel, buf.size(), 0))) return r;
      break;
    default:
      return fail(c, BHG_EINVAL, "unknown export");
  }
  if (written) *written = buf.size();
  if (out) {
    if (bytes < buf.size()) return fail(c, BHG_EINVAL, "export buffer too small");
    std::memcpy(out, buf.data(), buf.size());
  }
  return BHG_OK;
}

int bhg_direct_sum(bhg_context* c, int sys, const uint32_t* idx, size_t ns, double eps2, double G, double* out) {
  if (!c || !idx || !out) return fail(c, BHG_EINVAL, "null argument");
  if (sys < 0 || sys >= c->nsys) return fail(c, BHG_EINVAL, "no such system");
  cudaSetDevice(c->device);
  const SysDev& d = c->sys_host[sys];
  for (size_t k = 0; k < ns; ++k)
    if (idx[k] >= d.n) return fail(c, BHG_EINVAL, "sample index out of range");
  // positions of the current state (output order) into pm
  int r;
  uint32_t* didx = nullptr;
  double* dout = nullptr;
  double4* dpm = nullptr;
  if ((r = dev_alloc(c, (void**)&didx, ns * 4)) || (r = dev_alloc(c, (void**)&dout, ns * 24)) ||
      (r = dev_alloc(c, (void**)&dpm, (size_t)d.n * sizeof(double4)))) {
    dev_free(c, didx), dev_free(c, dout), dev_free(c, dpm);
    return r;
  }
  std::vector<Particle> hp(d.n);
  cudaMemcpyAsync(hp.data(), c->part + d.begin, (size_t)d.n * sizeof(Particle), cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  std::vector<double4> h4(d.n);
  for (uint32_t i = 0; i < d.n; ++i) h4[i] = make_double4(hp[i].pos[0], hp[i].pos[1], hp[i].pos[2], hp[i].mass);
  cudaMemcpyAsync(dpm, h4.data(), (size_t)d.n * sizeof(double4), cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(didx, idx, ns * 4, cudaMemcpyHostToDevice, c->stream);
  launch_direct(dpm, 0, d.n, didx, (uint32_t)ns, eps2, G, dout, c->stream);
  cudaError_t e = cudaMemcpyAsync(out, dout, ns * 24, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dev_free(c, didx), dev_free(c, dout), dev_free(c, dpm);
  if (e != cudaSuccess) return fail(c, BHG_ECUDA, cudaGetErrorString(e));
  return BHG_OK;
}

int bhg_energy(bhg_context* c, int sys, double G, double* kinetic, double* potential) {
  if (!c) return BHG_EINVAL;
  if (sys < 0 || sys >= c->nsys) return fail(c, BHG_EINVAL, "no such system");
  cudaSetDevice(c->device);
  const SysDev& d = c->sys_host[sys];
  const uint32_t blocks = (d.n + 255) / 256;
  double* dout = nullptr;
  int r = dev_alloc(c, (void**)&dout, (size_t)blocks * 16);
  if (r) return r;
  launch_energy(c->part, d.begin, d.n, G, dout, c->sms, c->stream);
  std::vector<double> h((size_t)blocks * 2);
  cudaError_t e = cudaMemcpyAsync(h.data(), dout, h.size() * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dev_free(c, dout);
  if (e != cudaSuccess) return fail(c, BHG_ECUDA, cudaGetErrorString(e));
  double ek = 0, ep = 0;
  for (uint32_t b = 0; b < blocks; ++b) ek += h[2 * b], ep += h[2 * b + 1];
  if (kinetic) *kinetic = ek;
  if (potential) *potential = ep;
  return BHG_OK;
}

int bhg_set_walk_group(bhg_context* c, uint32_t particles) {
  if (!c) return BHG_EINVAL;
  if (particles > (uint32_t)kGroupMax)
    return fail(c, BHG_EINVAL, "a walk group holds at most " + std::to_string(kGroupMax) + " particles");
  const uint32_t p = particles ? particles : (uint32_t)kGroupMax;
  if (p != c->walk_pack) drop_graph(c);
  c->walk_pack = p;
  return BHG_OK;
}

int bhg_selftest_wait(bhg_context* c, int publish_first, uint32_t spin_limit, uint32_t* prefix) {
  if (!c) return BHG_EINVAL;
  if (spin_limit == 0 || spin_limit > (1u << 20))
    return fail(c, BHG_EINVAL, "spin_limit must be in 1 .. 2^20 (a short wait)");
  cudaSetDevice(c->device);
  int r = read_state(c);  // finish what is queued; its own errors come first
  if (r || (r = finish_async(c))) return r;
  constexpr uint32_t kTiles = 8;
  uint32_t* words = nullptr;
  if ((r = dev_alloc(c, reinterpret_cast<void**>(&words), (kTiles + 1) * sizeof(uint32_t)))) return r;
  // tiles 1..7 have published an aggregate of 1 each; tile 0 publishes an
  // inclusive prefix of 1, or nothing at all
  uint32_t h[kTiles + 1] = {};
  for (uint32_t t = 1; t < kTiles; ++t) h[t] = kFlagAgg | 1u;
  h[0] = publish_first ? (kFlagPre | 1u) : 0u;
  cudaError_t e = cudaMemcpyAsync(words, h, sizeof h, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    launch_wait_probe(words, kTiles, (int)spin_limit, c->st, words + kTiles, c->stream);
    e = cudaGetLastError();
  }
  uint32_t got = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&got, words + kTiles, sizeof got, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dev_free(c, words);
  if (e != cudaSuccess) return fail(c, BHG_ECUDA, std::string("selftest_wait: ") + cudaGetErrorString(e));
  if (prefix) *prefix = got;
  if ((r = read_state(c))) return r;
  r = check_status(c);  // a wait that gave up: BHG_EDEVICE, as from a real sort or scan
  clear_status(c);
  return r;
}

int bhg_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return BHG_EINVAL;
  *tflops = measure_fp32_peak(device);
  return *tflops > 0 ? BHG_OK : BHG_ECUDA;
}

}  // extern "C"
