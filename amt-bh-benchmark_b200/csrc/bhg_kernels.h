// Host-side launchers of the build and walk kernels (bhg_build.cu,
// bhg_walk.cu), used by the context code in bhg_api.cu.
#pragma once

#include "bhg_internal.cuh"

namespace bhg {

void set_build_attributes();
// The sort/scan kernels' bounded look-back wait on a prepared array of tile
// words (a self-test of the give-up path): exclusive prefix of `tile` to out[0].
void launch_wait_probe(const uint32_t* words, uint32_t tile, int limit, DevState* st, uint32_t* out, cudaStream_t s);
void launch_bounds_domain(const Particle* p, const Tile* tiles, int ntiles, SysDev* sys, int nsys, double* partial,
                          DevState* st, cudaStream_t s);
void launch_keys(const Particle* p, const Tile* tiles, int ntiles, const SysDev* sys, int nsys, uint64_t* keys,
                 uint32_t* hist, uint32_t* offs, cudaStream_t s);
// tiles: the sort's own tile table, tile_keys keys per tile (1024 or 4096)
void launch_sort_pass(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, int pass,
                      const Tile* tiles, int ntiles, int tile_keys, const uint32_t* offs, uint32_t* lookback,
                      DevState* st, cudaStream_t s);
void launch_gather(const Particle* p, const uint32_t* perm, uint32_t n, Particle* staged, double4* pm, int sms,
                   cudaStream_t s);
void launch_topology(const SysDev* sys, int nsys, const Nodes& nd, const uint64_t* keys, unsigned max_leaf, uint32_t n,
                     uint32_t* lookback, DevState* st, int sms, cudaStream_t s);
// Walk targets: the topmost nodes that are leaves or hold at most `lim`
// particles.  The reference visits each group root - the topmost nodes with
// at most group_size particles, or leaves (is_group_root,
// flat_tree.h:190-192) - and descends to the first node that is a leaf or
// holds at most target_size particles (grouped_ttg.h:253); on every
// root-to-leaf path that is the deeper of the two cuts, i.e. the first node
// with count <= min(target_size, group_size).  group_size 0 (the per-node
// pass) and target_size 0 both give the leaves.  The walk groups are runs of
// consecutive targets of one system, at most `pack` particles and
// kMaxTargets targets each (a larger target alone), packed inside chunks of
// the tree (chunks: node-sized scratch): groups[g] is the index of group g's
// first target, st->n_groups their number.  lookback: 3 regions of
// n / 4096 + 9 words.
void launch_targets(const Nodes& nd, uint32_t lim, uint32_t pack, uint32_t n, uint32_t* mark, uint32_t* targets,
                    uint32_t* chunks, uint32_t* groups, uint32_t* lookback, DevState* st, int sms, cudaStream_t s);
// one_launch: k_moments_up (one kernel, children-first by counters) instead of
// one kernel per level; the same bits either way
void launch_moments(const Nodes& nd, const double4* pm, const DevState* st, int sms, bool one_launch, cudaStream_t s);

struct WalkArgs {
  const WNode* w;
  const float2* q45;
  const double* q64;
  const double4* mom;  // FP64 centre of mass + mass (the FP64 walk)
  const uint32_t* nbegin;
  const uint32_t* ncount;
  const double4* pm;
  const uint32_t* targets;
  const uint32_t* groups;  // first target of each walk group
  const SysDev* sys;
  const SysParam* prm;
  int nsys;
  const Particle* staged;  // Morton-ordered input of this step
  Particle* out;           // kicked/drifted particles (the state)
  double* accel;           // optional: G*a, 3 per particle
  DevState* st;
  // list slots (nslots, at least one per warp of the grid): the sources only
  // some targets of a group take, per warp (one pass) or per group (two
  // passes, when there are at most nslots groups); per slot also the group's
  // FP64 sums (kGroupMax x 3) and list length
  uint2* wlist;
  double* gsum;
  uint32_t* gnl;
  uint32_t nslots;
};

// Walks every target and kicks/drifts its particles.  precision:
// 0 = split (FP32 offsets and FP32 interactions, FP64 sums), 1 = FP64.
void launch_walk(const WalkArgs& a, int precision, bool quad, bool mask, int grid, cudaStream_t s);
int walk_blocks_per_sm(int precision, bool quad, bool mask);
int walk_threads();
// device bytes of one list slot
size_t walk_slot_bytes();

void launch_integrate(Particle* p, const double* accel, uint32_t n, const SysDev* sys, const SysParam* prm, int nsys,
                      int sms, cudaStream_t s);
// Counts a finished evaluation when no error bit is set.
void launch_eval_done(DevState* st, cudaStream_t s);
void launch_direct(const double4* pm, uint32_t begin, uint32_t n, const uint32_t* idx, uint32_t ns, double eps2,
                   double G, double* out, cudaStream_t s);
cudaError_t launch_energy(const Particle* p, uint32_t begin, uint32_t n, double G, double* out2, int sms,
                          cudaStream_t s);
double measure_fp32_peak(int device);
// Particle text (bhg_csv.cu).  Ingest: newline count per 16 KB tile and the
// scan of the tile counts (total newlines to *total), then the line starts
// (newlines + 1 of them), then one parse per line of [first, nlines), then
// the compaction of the particle lines (kept count to *total; dst may be
// null to count only).  Snapshot: formats the three text lines of every
// particle into slots (lengths, exclusive offsets and the three section
// totals), then gathers each section back to back.
size_t csv_tiles(size_t nbytes);
void launch_csv_count(const char* text, size_t n, uint32_t* tile_count, uint64_t* total, cudaStream_t s);
void launch_csv_emit(const char* text, size_t n, const uint32_t* tile_off, uint64_t* line_start, cudaStream_t s);
void launch_csv_parse(const char* text, size_t n, const uint64_t* line_start, uint64_t first, uint64_t nlines,
                      Particle* tmp, uint32_t* keep, unsigned long long* bad, int sms, cudaStream_t s);
size_t csv_keep_blocks(uint64_t m);
void launch_csv_compact(const Particle* tmp, const uint32_t* keep, uint64_t m, uint32_t* block_count,
                        uint64_t* total, Particle* dst, cudaStream_t s);
size_t vtk_slot_bytes(uint32_t n);
size_t vtk_blocks(uint32_t n);
void launch_vtk_format(const Particle* p, uint32_t n, char* slots, uint32_t* len, uint32_t* block_sum,
                       uint64_t* block_off, uint64_t* totals, int sms, cudaStream_t s);
void launch_vtk_gather(const char* slots, uint32_t n, const uint32_t* len, const uint64_t* block_off,
                       char* const out[3], cudaStream_t s);

// n particles of one Plummer sphere (scale a, total mass `mass`, centre c[3],
// bulk velocity b[3], ids id0..), drawn from a counter-based generator keyed
// by `seed`.
void launch_plummer(Particle* out, uint32_t n, double a, double mass, const double* c, const double* b, uint32_t id0,
                    uint64_t seed, int sms, cudaStream_t s);

}  // namespace bhg
