// Device-side data layout and shared helpers of the B200 Barnes-Hut path.
//
// HBM layout of one context (n particles, M node slots, S systems):
//   particles   Particle[n]   64 B  caller's records, state between steps
//   staged      Particle[n]   64 B  Morton-ordered copy made by the gather
//   pm          double4[n]    32 B  x, y, z, m in Morton order (walk sources)
//   keys/vals   2 x (u64+u32)[n]    radix-sort ping-pong buffers
//   nodes       per node: begin/count/first/info (16 B), box double4 (32 B),
//               multipole double4 com+mass (32 B) + iab double[6] (48 B),
//               walk record WNode (64 B) + the last two quadrupole terms
//               (8 B), FP64 traceless quadrupole (48 B)
//   systems     SysDev[S]     one per independent system (domain, params)
// Every size that changes from step to step (node counts per level, target
// count, sort tiles taken) lives in DevState in device memory, so a captured
// CUDA graph replays unchanged.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bhg {

constexpr int kMortonDepth = 21;  // flat_tree.h:102
constexpr int kLevels = kMortonDepth + 1;

// Status bits (DevState::status).
enum : uint32_t {
  kStNonFinite = 1u << 0,     // a coordinate is NaN / inf
  kStNodeOverflow = 1u << 1,  // more nodes than node slots: grow and redo
  kStSpinLimit = 1u << 2,     // a bounded wait gave up
  kStTooLarge = 1u << 3,      // a count exceeded a 30-bit field
  kStWalkLimit = 1u << 4,     // a walk visited more nodes than the tree holds
};

struct alignas(64) Particle {  // bh::Particle, particle.h:7-24
  uint32_t id;
  uint32_t pad;
  double mass;
  double pos[3];
  double vel[3];
};
static_assert(sizeof(Particle) == 64, "bh::Particle is 64 bytes");

// One independent system (a segment of the particle array).
struct SysDev {
  uint32_t begin, n;      // particle range
  uint32_t root;          // its root node (level 0 slot = system index)
  uint32_t pad;
  uint32_t tile_begin, tile_count;  // its radix-sort tiles
  double cx, cy, cz, hw;  // Domain (domain.h:16-19), computed on the device
  double lox, loy, loz, scale;  // morton_key's lo and scale (flat_tree.h:115-123)
};
static_assert(sizeof(SysDev) % 8 == 0, "SysDev packs doubles");

// Per-system walk parameters, written by the host before each walk.
struct SysParam {
  double theta2;  // theta * theta, as mac_accept_bbox forms it (multipole.h:152)
  double eps2, G, kick_dt, drift_dt;
  double pad[3];
};

// One radix-sort tile: a piece of one system's particle range.
struct Tile {
  uint32_t sys, start, count, first_tile;  // first_tile: first tile of the system
};

// Walk record of a node: what every visit reads, in one 64-byte line.
struct alignas(64) WNode {
  double cx, cy, cz;  // centre of mass
  double edge2;       // (2 * half_width)^2, as mac_accept_bbox forms it
  uint32_t first;     // first child (interior) or first particle (leaf)
  uint32_t count;     // particles
  uint32_t info;      // nchild | leaf << 4 | depth << 8
  float mass;         // FP32 mass (split walk)
  float q[4];         // FP32 traceless quadrupole xx, yy, zz, xy
};
static_assert(sizeof(WNode) == 64, "WNode is one 64-byte line");

__host__ __device__ inline uint32_t info_nchild(uint32_t i) { return i & 15u; }
__host__ __device__ inline bool info_leaf(uint32_t i) { return (i >> 4) & 1u; }
__host__ __device__ inline uint32_t info_depth(uint32_t i) { return (i >> 8) & 255u; }

struct DevState {
  // sticky: cleared by the host only
  uint32_t status;    // error bits; while set, walks skip and the state stays put
  uint32_t evals_ok;  // evaluations that finished with status 0
  unsigned long long pp_total, pc_total;  // interactions of those evaluations
  // per build (zeroed by every build)
  uint32_t n_nodes;  // total nodes (may exceed the slots on overflow)
  uint32_t max_depth;
  uint32_t level_begin[kLevels + 1];
  uint32_t level_count[kLevels + 1];
  uint32_t level_tiles[kLevels + 1];  // tiles taken by each level kernel
  uint32_t sort_tiles[16];            // tiles taken by each sort pass
  // per walk (zeroed by every walk)
  uint32_t n_targets;
  uint32_t n_groups;         // walk groups (nodes whose targets share a walk)
  uint32_t walk_next;        // next group of the walk
  uint32_t scan_tiles;       // tiles taken by the target compaction
  uint32_t group_tiles;      // tiles taken by the group compaction
  uint32_t n_chunks;         // packing chunks of the walk groups
  uint32_t chunk_tiles;      // tiles taken by the chunk compaction
  uint32_t walk_next2;       // next target of the walk's second pass
  unsigned long long pp, pc;  // interaction counts of the walk
};
constexpr size_t kBuildResetOffset = offsetof(DevState, n_nodes);
constexpr size_t kWalkResetOffset = offsetof(DevState, n_targets);

// Decoupled look-back words: 2 flag bits above a 30-bit count.
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPre = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ inline uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ inline void st_volatile(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }

__device__ inline uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

}  // namespace bhg

namespace bhg {

// Node arrays (structure of arrays over node slots, level order).
struct Nodes {
  uint32_t* begin;  // first particle (Morton order)
  uint32_t* count;  // particles
  uint32_t* first;  // first child (interior) / first particle (leaf)
  uint32_t* info;   // nchild | leaf << 4 | depth << 8
  double4* box;     // cell centre xyz, half width
  double4* mom;     // centre of mass xyz, mass
  double* iab;      // 6 per node: second moment about the centre of mass
  WNode* w;         // walk records
  float2* q45;      // FP32 traceless quadrupole xz, yz
  double* q64;      // 6 per node: FP64 traceless quadrupole (the FP64 walk)
  uint32_t* parent; // parent slot (kNoParent for a root)
  uint32_t* upcnt;  // children whose multipoles are done (the upward pass)
  uint32_t cap;     // node slots
};
constexpr uint32_t kNoParent = 0xffffffffu;

// Kernel-launch helpers shared by the .cu files (defined in bhg_build.cu).
constexpr int kTile = 4096;  // particles per bounds / keys tile
// keys per radix-sort tile: small problems, the rest
constexpr int kSortTileSmall = 1024, kSortTileLarge = 4096;
constexpr int kSortPasses = 8;
constexpr int kGroupMax = 64;    // particles of a walk group (targets sharing one traversal)
constexpr int kMaxTargets = 24;  // targets of a walk group (the bits of a traversal mask)

}  // namespace bhg
