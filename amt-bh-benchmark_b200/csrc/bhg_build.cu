// Tree build of the B200 Barnes-Hut path: bounds and domain, Morton keys,
// a 64-bit LSD radix sort of (key, index), the gather into Morton order, the
// level-by-level octree topology, the walk targets and the level-by-level
// multipole upward pass.  Everything is exact: keys, order and topology are
// bit-identical to the reference's build_flat_tree (flat_build_ttg.h:276-281),
// and the multipoles repeat its floating-point operations in the same order
// (explicit round-to-nearest intrinsics, no contraction).
#include "bhg_kernels.h"

#include <algorithm>
#include <cstdio>

namespace bhg {

// ---------------------------------------------------------------------------
// small block helpers

template <typename T>
__device__ inline T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Exclusive scan of one value per thread over a block of NT threads; total
// returned through *total.  `sh` needs NT/32 + 1 words.
template <int NT>
__device__ inline uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = warp_incl_scan(v);
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < NT / 32 ? sh[lane] : 0u;
    uint32_t wi = warp_incl_scan(w);
    if (lane < NT / 32) sh[lane] = wi - w;
    if (lane == NT / 32 - 1) sh[NT / 32] = wi;
  }
  __syncthreads();
  uint32_t r = sh[warp] + inc - v;
  *total = sh[NT / 32];
  __syncthreads();
  return r;
}

// Waits (bounded) for the look-back word of tile t and sums predecessors
// until an inclusive prefix is found.  first: the chain's first tile.  A
// predecessor that has not published after `limit` polls ends the wait: the
// status bit kStSpinLimit is set and the (partial) sum returned, so the
// kernel finishes and the host reports BHG_EDEVICE instead of hanging.
__device__ inline uint32_t look_back(const uint32_t* words, uint32_t t, uint32_t first, uint32_t stride,
                                     DevState* st, int limit = kSpinLimit) {
  uint32_t excl = 0;
  while (t > first) {
    --t;
    uint32_t w;
    int spins = 0;
    do {
      w = ld_volatile(&words[(size_t)t * stride]);
      if ((w >> 30) != 0u) break;
      __nanosleep(32);  // frees issue slots for the warps doing work
    } while (++spins < limit);
    if ((w >> 30) == 0u) {
      atomicOr(&st->status, kStSpinLimit);
      return excl;
    }
    excl += w & kCountMask;
    if ((w & kFlagPre) == kFlagPre) return excl;
  }
  return excl;
}

// The wait above on a caller-prepared word array (bhg_selftest_wait): one
// thread looks back from tile `tile` to tile 0 with the given poll limit and
// writes the exclusive prefix it found.
__global__ void k_wait_probe(const uint32_t* words, uint32_t tile, int limit, DevState* st, uint32_t* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = look_back(words, tile, 0, 1, st, limit);
}

void launch_wait_probe(const uint32_t* words, uint32_t tile, int limit, DevState* st, uint32_t* out, cudaStream_t s) {
  k_wait_probe<<<1, 32, 0, s>>>(words, tile, limit, st, out);
}

// ---------------------------------------------------------------------------
// a1: bounds per tile, then the domain per system
// particle_bounds (flat_build_ttg.h:93-113) + domain_from_bounds (domain.h:23-30)

constexpr int kBoundsThreads = 256;

__global__ void __launch_bounds__(kBoundsThreads) k_bounds(const Particle* __restrict__ p, const Tile* __restrict__ tiles,
                                                           double* __restrict__ partial, DevState* st) {
  const Tile t = tiles[blockIdx.x];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool bad = false;
  for (uint32_t i = threadIdx.x; i < t.count; i += kBoundsThreads) {
    const double* q = p[t.start + i].pos;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double v = q[a];
      bad |= !isfinite(v);
      lo[a] = fmin(lo[a], v);
      hi[a] = fmax(hi[a], v);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  __shared__ double s[kBoundsThreads / 32][6];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    for (int a = 0; a < 3; ++a) {
      s[warp][a] = lo[a];
      s[warp][3 + a] = hi[a];
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&st->status, kStNonFinite);
  if (threadIdx.x < 6) {
    double v = s[0][threadIdx.x];
    for (int w = 1; w < kBoundsThreads / 32; ++w)
      v = threadIdx.x < 3 ? fmin(v, s[w][threadIdx.x]) : fmax(v, s[w][threadIdx.x]);
    partial[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
  }
}

// One warp per system.
__global__ void k_domain(SysDev* sys, int nsys, const double* __restrict__ partial) {
  const int s = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= nsys) return;
  SysDev& d = sys[s];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t t = lane; t < d.tile_count; t += 32) {
    const double* q = partial + (size_t)(d.tile_begin + t) * 6;
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], q[a]);
      hi[a] = fmax(hi[a], q[3 + a]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  if (lane != 0) return;
  // domain_from_bounds: centre = 0.5 (lo + hi); half width = 0.5 max extent,
  // 1 when degenerate, times (1 + 1e-9).
  double c[3], w = -INFINITY;
  for (int a = 0; a < 3; ++a) {
    c[a] = __dmul_rn(0.5, __dadd_rn(lo[a], hi[a]));
    double e = __dsub_rn(hi[a], lo[a]);
    if (w < e) w = e;
  }
  double hw = __dmul_rn(0.5, w);
  if (!(hw > 0.0)) hw = 1.0;
  hw = __dmul_rn(hw, 1.0 + 1e-9);
  d.cx = c[0];
  d.cy = c[1];
  d.cz = c[2];
  d.hw = hw;
  // morton_key's lower corner and scale (flat_tree.h:115-123)
  d.lox = __dsub_rn(c[0], hw);
  d.loy = __dsub_rn(c[1], hw);
  d.loz = __dsub_rn(c[2], hw);
  d.scale = __ddiv_rn((double)(1u << kMortonDepth), __dmul_rn(2.0, hw));
}

// ---------------------------------------------------------------------------
// a2: Morton keys (flat_tree.h:104-125) + the digit histograms of the sort

// Interleaves the low 21 bits of v with two zero bits after each one
// (bit i -> bit 3i) by five shift-and-mask rounds of halving group sizes.
__device__ __forceinline__ uint64_t dilate3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x001f00000000ffffull;  // 5 | 16
  x = (x | (x << 16)) & 0x001f0000ff0000ffull;  // 5 | 8 | 8
  x = (x | (x << 8)) & 0x100f00f00f00f00full;   // groups of 4
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;   // groups of 2
  x = (x | (x << 2)) & 0x1249249249249249ull;   // single bits
  return x;
}

__device__ __forceinline__ uint32_t quantise(double v, double lo, double scale) {
  double q = floor(__dmul_rn(__dsub_rn(v, lo), scale));
  q = fmin(fmax(q, 0.0), (double)((1u << kMortonDepth) - 1));
  return (uint32_t)q;
}

constexpr int kKeyThreads = 256;

__global__ void __launch_bounds__(kKeyThreads) k_keys(const Particle* __restrict__ p, const Tile* __restrict__ tiles,
                                                      const SysDev* __restrict__ sys, uint64_t* __restrict__ keys,
                                                      uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[kSortPasses * 256];
  for (int i = threadIdx.x; i < kSortPasses * 256; i += kKeyThreads) h[i] = 0;
  __syncthreads();
  const Tile t = tiles[blockIdx.x];
  const SysDev& d = sys[t.sys];
  const double lox = d.lox, loy = d.loy, loz = d.loz, sc = d.scale;
  for (uint32_t i = threadIdx.x; i < t.count; i += kKeyThreads) {
    const double* q = p[t.start + i].pos;
    uint64_t k = dilate3(quantise(q[0], lox, sc)) | (dilate3(quantise(q[1], loy, sc)) << 1) |
                 (dilate3(quantise(q[2], loz, sc)) << 2);
    keys[t.start + i] = k;
#pragma unroll
    for (int ps = 0; ps < kSortPasses; ++ps) atomicAdd(&h[ps * 256 + ((k >> (8 * ps)) & 255u)], 1u);
  }
  __syncthreads();
  uint32_t* g = hist + (size_t)t.sys * kSortPasses * 256;
  for (int i = threadIdx.x; i < kSortPasses * 256; i += kKeyThreads)
    if (h[i]) atomicAdd(&g[i], h[i]);
}

// offs[sys][pass][digit] = first output position of the digit in the system.
__global__ void __launch_bounds__(256) k_digit_offsets(const SysDev* __restrict__ sys, const uint32_t* __restrict__ hist,
                                                       uint32_t* __restrict__ offs) {
  __shared__ uint32_t sh[256 / 32 + 1];
  const uint32_t s = blockIdx.x;
  for (int ps = 0; ps < kSortPasses; ++ps) {
    size_t at = ((size_t)s * kSortPasses + ps) * 256 + threadIdx.x;
    uint32_t total;
    uint32_t e = block_excl_scan<256>(hist[at], sh, &total);
    offs[at] = sys[s].begin + e;
  }
}

// ---------------------------------------------------------------------------
// a3: one LSD radix pass (8-bit digit), one tile of keys per block.
// Each warp first counts its keys per digit (shared-memory atomics, any
// order); the counts give every warp's first position per digit in the tile
// and the tile's per-digit totals, which are published at once for the
// decoupled look-back of later tiles of the same system.  Then the first 256
// threads look back for the tile's prefix while the other warps rank: within
// a warp, equal digits (found with one ballot per digit bit) take consecutive
// places in item order, and every key goes straight to its place in the
// tile's digit order in shared memory.  The tile is written out with
// consecutive threads on consecutive addresses.  Stable, so the final order
// is (key, input index) as KeyIndex orders it (flat_build_ttg.h:62-66).
// Measured per sort of 4,194,304 keys: 0.55 ms with __match_any_sync ranks
// after the look-back (256 threads x 16 keys, 2 blocks per SM), 0.42 with
// ballots, 0.36 with the counts first and the look-back beside the ranking,
// 0.33 with 3 blocks of 512 x 8 per SM and a back-off in the look-back's poll.

constexpr int kDigits = 256;

// Shared memory of a pass with NT threads and ITEMS keys per thread: the
// tile's keys and values in digit order, per-warp digit counts, the digits'
// global bases, and the ticket plus the block scan's words.
template <int NT, int ITEMS>
constexpr size_t sort_smem() {
  return (size_t)NT * ITEMS * 12 + (size_t)(NT / 32) * kDigits * 4 + kDigits * 4 + 4 * (NT / 32 + 2);
}

// The lanes of the warp whose 8-bit digit equals this lane's: one ballot per
// digit bit, which the SM issues faster than a match instruction.
__device__ __forceinline__ uint32_t match_digit_all(uint32_t dg) {
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool bit = (dg >> b) & 1u;
    const uint32_t on = __ballot_sync(0xffffffffu, bit);
    m &= bit ? on : ~on;
  }
  return m;
}

// The same among the lanes with ok set (the result of a lane without ok is
// not used).
__device__ __forceinline__ uint32_t match_digit(uint32_t dg, bool ok) {
  return __ballot_sync(0xffffffffu, ok) & match_digit_all(dg);
}

// A pass's tile: keys (and, after the first pass, values) into registers,
// and the warp's digit counts (order does not matter here).  FULL: the tile
// holds ITEMS keys for every thread, so no lane needs a bounds check.
template <int ITEMS, bool FULL>
__device__ __forceinline__ void sort_load(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                          const Tile& t, int pass, int shift, int warp, int lane, uint64_t (&k)[ITEMS],
                                          uint32_t (&v)[ITEMS], uint32_t* my_hist) {
  const uint32_t i0 = warp * (32 * ITEMS) + lane;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const uint32_t i = i0 + j * 32;
    const bool ok = FULL || i < t.count;
    k[j] = ok ? kin[t.start + i] : 0ull;
    v[j] = ok ? (pass == 0 ? t.start + i : vin[t.start + i]) : 0u;
  }
#pragma unroll
  for (int j = 0; j < ITEMS; ++j)
    if (FULL || i0 + j * 32 < t.count) atomicAdd(&my_hist[(k[j] >> shift) & 255u], 1u);
}

// Stable ranks within the warp, in input order: each key and value goes to
// its place in the tile's digit order (my_hist: the warp's next position per
// digit).
template <int ITEMS, bool FULL>
__device__ __forceinline__ void sort_rank(const Tile& t, int shift, int warp, int lane, const uint64_t (&k)[ITEMS],
                                          const uint32_t (&v)[ITEMS], uint32_t* my_hist, uint64_t* s_keys,
                                          uint32_t* s_vals) {
  const uint32_t i0 = warp * (32 * ITEMS) + lane;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const bool ok = FULL || i0 + j * 32 < t.count;
    const uint32_t d = (uint32_t)((k[j] >> shift) & 255u);
    const uint32_t peers = FULL ? match_digit_all(d) : match_digit(d, ok);
    const uint32_t base = ok ? my_hist[d] : 0u;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) my_hist[d] = base + __popc(peers);
    __syncwarp();
    if (ok) {
      const uint32_t pos = base + __popc(peers & lt);
      s_keys[pos] = k[j];
      s_vals[pos] = v[j];
    }
  }
}

template <int NT, int ITEMS, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_sort_pass(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                        uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                        int pass, const Tile* __restrict__ tiles,
                                                        const uint32_t* __restrict__ offs, uint32_t* lookback,
                                                        DevState* st) {
  static_assert(NT >= kDigits && NT % 32 == 0, "one thread per digit");
  constexpr int kWarps = NT / 32;
  constexpr int kSortTile = NT * ITEMS;
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem);
  uint32_t* s_vals = reinterpret_cast<uint32_t*>(smem + (size_t)kSortTile * 8);
  uint32_t* s_whist = reinterpret_cast<uint32_t*>(smem + (size_t)kSortTile * 12);  // [warp][digit]
  uint32_t* s_gbase = s_whist + kWarps * kDigits;
  uint32_t* s_misc = s_gbase + kDigits;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int shift = 8 * pass;
  if (tid == 0) s_misc[0] = atomicAdd(&st->sort_tiles[pass], 1u);
  for (int i = tid; i < kWarps * kDigits; i += NT) s_whist[i] = 0;
  __syncthreads();
  const uint32_t tile = s_misc[0];
  const Tile t = tiles[tile];
  uint32_t* my_hist = s_whist + warp * kDigits;

  // the warp's keys: input positions warp * 32 * ITEMS + j * 32 + lane
  uint64_t k[ITEMS];
  uint32_t v[ITEMS];
  if (t.count == (uint32_t)kSortTile)
    sort_load<ITEMS, true>(kin, vin, t, pass, shift, warp, lane, k, v, my_hist);
  else
    sort_load<ITEMS, false>(kin, vin, t, pass, shift, warp, lane, k, v, my_hist);
  __syncthreads();

  // per digit (the first 256 threads): exclusive prefix over the warps and
  // the tile's count, published for the look-back of later tiles
  const int dg = tid;
  uint32_t run = 0;
  if (dg < kDigits) {
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = s_whist[w * kDigits + dg];
      s_whist[w * kDigits + dg] = run;
      run += c;
    }
    st_volatile(&lookback[(size_t)tile * kDigits + dg], (tile == t.first_tile ? kFlagPre : kFlagAgg) | run);
  }
  // the digit's first position in the tile, added to every warp's prefix
  uint32_t total;
  const uint32_t lb_start = block_excl_scan<NT>(dg < kDigits ? run : 0u, s_misc + 1, &total);
  if (dg < kDigits)
    for (int w = 0; w < kWarps; ++w) s_whist[w * kDigits + dg] += lb_start;
  __syncthreads();

  // the look-back for the tile's prefix in the system (digit threads; the
  // other warps go on ranking meanwhile)
  if (dg < kDigits) {
    uint32_t excl = 0;
    if (tile != t.first_tile) {
      excl = look_back(lookback + dg, tile, t.first_tile, kDigits, st);
      st_volatile(&lookback[(size_t)tile * kDigits + dg], kFlagPre | (excl + run));
    }
    s_gbase[dg] = offs[((size_t)t.sys * kSortPasses + pass) * kDigits + dg] + excl - lb_start;
  }
  // stable ranks within the warp, in input order; keys and values go to
  // their place in the tile's digit order
  if (t.count == (uint32_t)kSortTile)
    sort_rank<ITEMS, true>(t, shift, warp, lane, k, v, my_hist, s_keys, s_vals);
  else
    sort_rank<ITEMS, false>(t, shift, warp, lane, k, v, my_hist, s_keys, s_vals);
  __syncthreads();
  for (uint32_t i = tid; i < t.count; i += NT) {
    uint64_t key = s_keys[i];
    uint32_t o = s_gbase[(key >> shift) & 255u] + i;
    kout[o] = key;
    vout[o] = s_vals[i];
  }
}

// Block shapes (threads, keys per thread, blocks per SM the registers are
// held to): 1024-key tiles for small problems (four times the blocks per
// pass), 4096-key tiles above (3 blocks of 512 threads per SM: 0.331 ms per
// sort at 4M against 0.346 with 2 blocks, 0.46 with one block of 1,024 and
// 0.42 with 2,048-key tiles of 256 threads, 6 blocks per SM).
template <int NT_, int ITEMS_, int MINB_>
struct SortShape {
  static constexpr int NT = NT_, ITEMS = ITEMS_, MINB = MINB_, TILE = NT_ * ITEMS_;
  static constexpr size_t smem = sort_smem<NT_, ITEMS_>();
  static auto kernel() { return k_sort_pass<NT_, ITEMS_, MINB_>; }
};
using SortSmall = SortShape<256, 4, 1>;
using SortLarge = SortShape<512, 8, 3>;
static_assert(SortSmall::TILE == kSortTileSmall && SortLarge::TILE == kSortTileLarge, "the host's tile tables");

// ---------------------------------------------------------------------------
// gather into Morton order: staged[i] = particles[perm[i]], pm[i] = (x,y,z,m)
// (sort_particles' final loop, flat_build_ttg.h:180-188)

__global__ void k_gather(const Particle* __restrict__ p, const uint32_t* __restrict__ perm, uint32_t n,
                         Particle* __restrict__ staged, double4* __restrict__ pm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4* src = reinterpret_cast<const uint4*>(p + perm[i]);
    uint4* dst = reinterpret_cast<uint4*>(staged + i);
    uint4 a = src[0], b = src[1], c = src[2], e = src[3];
    dst[0] = a;
    dst[1] = b;
    dst[2] = c;
    dst[3] = e;
    // mass at bytes 8..15, pos at 16..39
    double mass = __hiloint2double(a.w, a.z);
    double x = __hiloint2double(b.y, b.x), y = __hiloint2double(b.w, b.z), z = __hiloint2double(c.y, c.x);
    pm[i] = make_double4(x, y, z, mass);
  }
}

// ---------------------------------------------------------------------------
// a4: octree topology, one level per launch.
// The root of system s is node s (level 0).  For a non-leaf parent at depth
// d-1 holding sorted keys [b, e), its children are the non-empty octants of
// the depth-d digit, in octant order (split_octants, flat_tree.h:167-180);
// a node stops splitting at count <= max_leaf or depth 21 (LeafRule,
// flat_tree.h:144-156); child centres are parent centre +- half of the
// parent's half width (child_center, flat_tree.h:182-185).  Level d's nodes
// are numbered in parent order (a block scan plus a look-back across tiles),
// so the layout is breadth first and deterministic.

__global__ void k_roots(const SysDev* __restrict__ sys, int nsys, Nodes nd, unsigned max_leaf, DevState* st) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    st->level_begin[0] = 0;
    st->level_count[0] = (uint32_t)nsys;
    st->level_begin[1] = (uint32_t)nsys;
    st->max_depth = 1;
    st->n_nodes = (uint32_t)nsys;
  }
  if (s >= nsys) return;
  const SysDev& d = sys[s];
  bool leaf = d.n <= max_leaf;  // depth 0 < 21
  nd.begin[s] = d.begin;
  nd.count[s] = d.n;
  nd.first[s] = leaf ? d.begin : 0u;
  nd.info[s] = (leaf ? 16u : 0u);
  nd.box[s] = make_double4(d.cx, d.cy, d.cz, d.hw);
  nd.parent[s] = kNoParent;
  nd.upcnt[s] = 0u;
}

constexpr int kLevelThreads = 256;  // 8 threads (one per octant) per parent
constexpr int kLevelParents = kLevelThreads / 8;
// blocks per SM of a level launch (tiles are taken dynamically): the tree
// phase at 4M takes 0.97 ms with 4, 0.74 with 8, 0.75 with 16
constexpr int kLevelBlocksPerSm = 8;

// The first index in [lo, hi) whose key is >= thr (hi if none; keys sorted),
// by an 8-way search: each round loads 7 evenly spaced keys at once and keeps
// the stretch between the last one below thr and the first one at or above,
// so a parent of 65,536 particles takes 6 dependent rounds instead of 16.
__device__ __forceinline__ uint32_t first_at_least(const uint64_t* __restrict__ keys, uint32_t lo, uint32_t hi,
                                                   uint64_t thr) {
  while (hi - lo > 8u) {
    const uint32_t step = (hi - lo) >> 3;
    uint32_t m = 0;  // probes lo + j * step (j = 1..7) below thr: a prefix, the keys being sorted
#pragma unroll
    for (uint32_t j = 1; j <= 7; ++j) m += keys[lo + j * step] < thr ? 1u : 0u;
    const uint32_t nlo = m ? lo + m * step + 1u : lo;
    hi = m < 7u ? lo + (m + 1u) * step : hi;
    lo = nlo;
  }
  uint32_t m = 0;
#pragma unroll
  for (uint32_t j = 0; j < 8u; ++j) m += (lo + j < hi && keys[lo + j] < thr) ? 1u : 0u;
  return lo + m;
}

__global__ void __launch_bounds__(kLevelThreads) k_level(int depth, Nodes nd, const uint64_t* __restrict__ keys,
                                                         unsigned max_leaf, uint32_t* __restrict__ lookback_all,
                                                         DevState* st) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_scan[kLevelThreads / 32 + 2];
  __shared__ uint32_t s_base;
  const uint32_t pb = st->level_begin[depth - 1], pc = st->level_count[depth - 1];
  const uint32_t cb = pb + pc;  // level_begin[depth]
  if (cb > nd.cap) {  // an earlier level overflowed the slots: nothing to read here
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&st->status, kStNodeOverflow);
    return;
  }
  const uint32_t ntiles = (pc + kLevelParents - 1) / kLevelParents;
  uint32_t* lookback = lookback_all + pb / kLevelParents + depth;
  const int tid = threadIdx.x, lane = tid & 31, oct = tid & 7;
  const int csh = 63 - 3 * depth;  // digit shift at this depth
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(&st->level_tiles[depth], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) break;
    const uint32_t parent = pb + tile * kLevelParents + (tid >> 3);
    const bool valid = parent < cb;
    uint32_t b = 0, c = 0, info = 16u;
    if (valid) {
      b = nd.begin[parent];
      c = nd.count[parent];
      info = nd.info[parent];
    }
    const bool split = valid && !info_leaf(info);
    // octant o starts at the first key in [b, b+c) whose depth digit is >= o
    uint32_t start = b;
    if (split && oct > 0) {
      const uint64_t cell = 1ull << (csh + 3);  // parent's cell size in keys
      const uint64_t thr = (keys[b] & ~(cell - 1)) | ((uint64_t)oct << csh);
      start = first_at_least(keys, b, b + c, thr);
    }
    uint32_t next = __shfl_down_sync(0xffffffffu, start, 1);
    if (oct == 7) next = b + c;
    const bool child = split && next > start;
    const uint32_t grp = (__ballot_sync(0xffffffffu, child) >> (lane & ~7)) & 0xffu;
    const uint32_t nch = __popc(grp);
    const uint32_t rank = __popc(grp & ((1u << oct) - 1u));
    // exclusive scan of nch over the tile's parents (counted once, at oct 0)
    uint32_t total;
    uint32_t pex = block_excl_scan<kLevelThreads>(oct == 0 ? nch : 0u, s_scan, &total);
    pex = __shfl_sync(0xffffffffu, pex, lane & ~7);
    if (tid == 0) {
      const bool first = tile == 0;
      st_volatile(&lookback[tile], (first ? kFlagPre : kFlagAgg) | total);
      uint32_t excl = 0;
      if (!first) {
        excl = look_back(lookback, tile, 0, 1, st);
        st_volatile(&lookback[tile], kFlagPre | (excl + total));
      }
      s_base = cb + excl;
      if (tile == ntiles - 1) {
        const uint32_t end = cb + excl + total;
        st->level_count[depth] = excl + total;
        st->level_begin[depth + 1] = end;
        st->n_nodes = end;
        if (excl + total > 0) st->max_depth = depth + 1;
        if (end > nd.cap) atomicOr(&st->status, kStNodeOverflow);
      }
    }
    __syncthreads();
    const uint32_t firstc = s_base + pex;
    if (child) {
      const uint32_t ci = firstc + rank;
      if (ci < nd.cap) {
        const uint32_t cnt = next - start;
        const bool leaf = cnt <= max_leaf || depth >= kMortonDepth;
        const double4 pbx = nd.box[parent];
        const double q = __dmul_rn(0.5, pbx.w);
        nd.begin[ci] = start;
        nd.count[ci] = cnt;
        nd.first[ci] = leaf ? start : 0u;
        nd.info[ci] = (leaf ? 16u : 0u) | ((uint32_t)depth << 8);
        nd.parent[ci] = parent;
        nd.upcnt[ci] = 0u;
        nd.box[ci] = make_double4((oct & 1) ? __dadd_rn(pbx.x, q) : __dsub_rn(pbx.x, q),
                                  (oct & 2) ? __dadd_rn(pbx.y, q) : __dsub_rn(pbx.y, q),
                                  (oct & 4) ? __dadd_rn(pbx.z, q) : __dsub_rn(pbx.z, q), q);
      }
    }
    if (split && oct == 0 && parent < nd.cap) {
      nd.first[parent] = firstc;
      nd.info[parent] = info | nch;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Cuts of the tree: the topmost nodes that are leaves or hold at most `lim`
// particles, marked at their first particle and compacted in Morton order.
// Used for the walk targets (lim = min(target_size, group_size)); the same
// compaction then lists the walk groups (k_pack_groups).

__global__ void k_mark_cut(Nodes nd, uint32_t lim, const DevState* __restrict__ st, uint32_t* __restrict__ mark) {
  if (st->status & kStNodeOverflow) return;  // children may lie beyond the slots
  const uint32_t nn = min(st->n_nodes, nd.cap), nroots = st->level_count[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    const uint32_t info = nd.info[i], cnt = nd.count[i];
    const bool cut = info_leaf(info) || cnt <= lim;
    if (i < nroots && cut) mark[nd.begin[i]] = i;
    if (!cut) {
      const uint32_t f = nd.first[i], k = info_nchild(info);
      for (uint32_t j = 0; j < k; ++j) {
        const uint32_t ch = f + j;
        if (ch >= nd.cap) break;
        if (info_leaf(nd.info[ch]) || nd.count[ch] <= lim) mark[nd.begin[ch]] = ch;
      }
    }
  }
}

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;

// Compacts the marked entries of mark[0..n) into out (Morton order), resets
// the marks, and writes the count.  Tiles chain through a decoupled look-back.
__global__ void __launch_bounds__(kScanThreads) k_compact(uint32_t* __restrict__ mark, uint32_t n,
                                                          uint32_t* __restrict__ out, uint32_t* __restrict__ lookback,
                                                          uint32_t* tile_counter, uint32_t* count_out,
                                                          DevState* st) {
  __shared__ uint32_t s_tile, s_base;
  __shared__ uint32_t s_scan[kScanThreads / 32 + 2];
  const uint32_t ntiles = (n + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) break;
    const uint32_t base = tile * kScanThreads * kScanItems + threadIdx.x * kScanItems;
    uint32_t v[kScanItems], cnt = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      v[j] = base + j < n ? mark[base + j] : 0xffffffffu;
      cnt += v[j] != 0xffffffffu;
    }
    uint32_t total;
    uint32_t ex = block_excl_scan<kScanThreads>(cnt, s_scan, &total);
    if (threadIdx.x == 0) {
      st_volatile(&lookback[tile], (tile == 0 ? kFlagPre : kFlagAgg) | total);
      uint32_t excl = 0;
      if (tile > 0) {
        excl = look_back(lookback, tile, 0, 1, st);
        st_volatile(&lookback[tile], kFlagPre | (excl + total));
      }
      s_base = excl;
      if (tile == ntiles - 1) *count_out = excl + total;
    }
    __syncthreads();
    uint32_t o = s_base + ex;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      if (v[j] != 0xffffffffu) out[o++] = v[j];
      if (base + j < n) mark[base + j] = 0xffffffffu;  // ready for the next use
    }
    __syncthreads();
  }
}

// Walk groups: runs of consecutive targets (Morton order) that share one
// traversal.  Any set of targets may share one: a node accepted for the
// bounding box of all their particles is accepted for each target's box
// inside it, and a node rejected for every point of that box is opened by
// each target (mac_accept_bbox / mac_reject_all, multipole.h:158-160), so
// every target still gets exactly its own interaction list.  A group holds at
// most `pack` (<= kGroupMax) particles and kMaxTargets targets, and a target
// larger than `pack` is a group of its own.  The targets are packed greedily
// inside packing chunks - the topmost tree nodes of at most kPackChunk
// particles (or leaves) - one warp per chunk: a chunk lies inside one system
// and its targets depend on that system alone, so a system's groups, and
// with them its results bit for bit, do not depend on the other systems of
// the context.  Group starts are marked at their first target's index for
// the compaction.
constexpr uint32_t kPackChunk = 2048;
constexpr int kPackWindows = 4;  // windows of 32 targets whose counts are loaded together

// Index of the first target whose particles start at or after particle p
// (the targets lie in particle order), by one warp: each round probes 32
// evenly spaced targets and keeps the stretch between the last probe before
// p and the first one at or after it.
__device__ __forceinline__ uint32_t first_target_at(const uint32_t* __restrict__ targets,
                                                    const uint32_t* __restrict__ nbegin, uint32_t nt, uint32_t p,
                                                    int lane) {
  uint32_t lo = 0, hi = nt;  // the answer lies in [lo, hi]
  while (hi - lo > 32u) {
    const uint32_t step = (hi - lo + 31u) / 32u;
    const uint32_t q = lo + (uint32_t)lane * step;
    const bool before = q < hi && nbegin[targets[q]] < p;
    const uint32_t m = (uint32_t)__popc(__ballot_sync(0xffffffffu, before));  // probes 0 .. m-1 lie before p
    const uint32_t nlo = m ? lo + (m - 1u) * step + 1u : lo;
    hi = min(hi, lo + m * step);
    lo = nlo;
  }
  const uint32_t q = lo + (uint32_t)lane;
  const bool before = q < hi && nbegin[targets[q]] < p;
  return lo + (uint32_t)__popc(__ballot_sync(0xffffffffu, before));
}

__global__ void k_pack_groups(const uint32_t* __restrict__ chunks, const uint32_t* __restrict__ targets,
                              const uint32_t* __restrict__ nbegin, const uint32_t* __restrict__ ncount,
                              uint32_t pack, const DevState* __restrict__ st, uint32_t* __restrict__ mark) {
  if (st->status & kStNodeOverflow) return;
  const uint32_t nchunks = st->n_chunks, nt = st->n_targets;
  const int lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  for (uint32_t c = blockIdx.x * wpb + (threadIdx.x >> 5); c < nchunks; c += gridDim.x * wpb) {
    const uint32_t cn = chunks[c];
    const uint32_t cb = nbegin[cn], ce = cb + ncount[cn];
    uint32_t cnt = 0, k = 0;
    bool first = true, end = false;
    for (uint32_t t0 = first_target_at(targets, nbegin, nt, cb, lane); !end; t0 += 32u * kPackWindows) {
      // the particle counts of the next windows' targets (past the chunk: ~0)
      uint32_t n[kPackWindows];
#pragma unroll
      for (int w = 0; w < kPackWindows; ++w) {
        const uint32_t t = t0 + 32u * w + (uint32_t)lane;
        n[w] = 0xffffffffu;
        if (t < nt) {
          const uint32_t tn = targets[t];
          if (nbegin[tn] < ce) n[w] = ncount[tn];
        }
      }
#pragma unroll
      for (int w = 0; w < kPackWindows; ++w) {
        if (end) break;
        // the greedy packing, run alike by every lane over the window's 32 counts
        uint32_t starts = 0;
        for (int i = 0; i < 32; ++i) {
          const uint32_t ni = __shfl_sync(0xffffffffu, n[w], i);
          if (ni == 0xffffffffu) {
            end = true;
            break;
          }
          if (first || cnt + ni > pack || k >= (uint32_t)kMaxTargets) {
            starts |= 1u << i;
            cnt = 0;
            k = 0;
            first = false;
          }
          cnt += ni;
          ++k;
        }
        if ((starts >> lane) & 1u) mark[t0 + 32u * w + (uint32_t)lane] = t0 + 32u * w + (uint32_t)lane;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// a5: multipoles, every node after its children (k_moments_up).  finalize_node
// (flat_tree.h:257-274): raw moments about the cell centre, of the particles
// (raw_moment_of_particle, multipole.h:52-59) or of the children shifted by
// the parallel-axis theorem (raw_moment_from_multipole, :92-102), then the
// mass, centre of mass and second moment about it (finalize_raw_moment,
// :76-87).  Also writes the walk records.

struct Raw {
  double m, m1[3], m2[6];
};

__device__ __forceinline__ void outer_sym_rn(const double d[3], double s, double o[6]) {
  // (s * d_a) * d_b, as outer_sym (multipole.h:15-18) evaluates it
  o[0] = __dmul_rn(__dmul_rn(s, d[0]), d[0]);
  o[1] = __dmul_rn(__dmul_rn(s, d[1]), d[1]);
  o[2] = __dmul_rn(__dmul_rn(s, d[2]), d[2]);
  o[3] = __dmul_rn(__dmul_rn(s, d[0]), d[1]);
  o[4] = __dmul_rn(__dmul_rn(s, d[0]), d[2]);
  o[5] = __dmul_rn(__dmul_rn(s, d[1]), d[2]);
}

__device__ __forceinline__ void raw_add(Raw& r, double m, const double d[3], const double o[6]) {
  r.m = __dadd_rn(r.m, m);
#pragma unroll
  for (int k = 0; k < 3; ++k) r.m1[k] = __dadd_rn(r.m1[k], __dmul_rn(m, d[k]));
#pragma unroll
  for (int k = 0; k < 6; ++k) r.m2[k] = __dadd_rn(r.m2[k], o[k]);
}

// The multipoles and walk record of node i, from its particles (a leaf) or
// from its children's finished multipoles (read through L2 when other
// threads of the same launch wrote them: FROM_L2).
template <bool FROM_L2>
__device__ void finalize_node(const Nodes& nd, const double4* __restrict__ pm, uint32_t i) {
  {
    const double4 bx = nd.box[i];
    const double ref[3] = {bx.x, bx.y, bx.z};
    const uint32_t info = nd.info[i];
    Raw r = {0.0, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}};
    if (info_leaf(info)) {
      const uint32_t b = nd.begin[i], e = b + nd.count[i];
      for (uint32_t p = b; p < e; ++p) {
        const double4 q = pm[p];
        const double d[3] = {__dsub_rn(q.x, ref[0]), __dsub_rn(q.y, ref[1]), __dsub_rn(q.z, ref[2])};
        double o[6];
        outer_sym_rn(d, q.w, o);
        raw_add(r, q.w, d, o);
      }
    } else {
      const uint32_t f = nd.first[i], nc = info_nchild(info);
      for (uint32_t j = 0; j < nc; ++j) {
        // children written by other threads of this launch are read from L2
        // (an L1 line may be older than their fence)
        const double2* cp = reinterpret_cast<const double2*>(nd.mom + f + j);
        const double2* ip = reinterpret_cast<const double2*>(nd.iab + (size_t)(f + j) * 6);
        const double2 c01 = FROM_L2 ? __ldcg(cp) : cp[0], c23 = FROM_L2 ? __ldcg(cp + 1) : cp[1];
        const double2 i01 = FROM_L2 ? __ldcg(ip) : ip[0], i23 = FROM_L2 ? __ldcg(ip + 1) : ip[1];
        const double2 i45 = FROM_L2 ? __ldcg(ip + 2) : ip[2];
        const double ci[6] = {i01.x, i01.y, i23.x, i23.y, i45.x, i45.y};
        const double cmw = c23.y;
        const double d[3] = {__dsub_rn(c01.x, ref[0]), __dsub_rn(c01.y, ref[1]), __dsub_rn(c23.x, ref[2])};
        double o[6];
        outer_sym_rn(d, cmw, o);
#pragma unroll
        for (int t = 0; t < 6; ++t) o[t] = __dadd_rn(ci[t], o[t]);
        raw_add(r, cmw, d, o);
      }
    }
    // finalize_raw_moment
    const double inv = __ddiv_rn(1.0, r.m);
    const double dl[3] = {__dmul_rn(inv, r.m1[0]), __dmul_rn(inv, r.m1[1]), __dmul_rn(inv, r.m1[2])};
    double sh[6], iab[6];
    outer_sym_rn(dl, r.m, sh);
#pragma unroll
    for (int t = 0; t < 6; ++t) iab[t] = __dsub_rn(r.m2[t], sh[t]);
    const double com[3] = {__dadd_rn(ref[0], dl[0]), __dadd_rn(ref[1], dl[1]), __dadd_rn(ref[2], dl[2])};
    nd.mom[i] = make_double4(com[0], com[1], com[2], r.m);
    double* out = nd.iab + (size_t)i * 6;
#pragma unroll
    for (int t = 0; t < 6; ++t) out[t] = iab[t];
    // traceless Q = 3 I - tr(I) delta (accel_from_source, multipole.h:185-188)
    const double tr = __dadd_rn(__dadd_rn(iab[0], iab[1]), iab[2]);
    double q[6];
#pragma unroll
    for (int t = 0; t < 3; ++t) q[t] = __dsub_rn(__dmul_rn(3.0, iab[t]), tr);
#pragma unroll
    for (int t = 3; t < 6; ++t) q[t] = __dmul_rn(3.0, iab[t]);
    double* qo = nd.q64 + (size_t)i * 6;
#pragma unroll
    for (int t = 0; t < 6; ++t) qo[t] = q[t];
    WNode w;
    w.cx = com[0];
    w.cy = com[1];
    w.cz = com[2];
    const double edge = __dmul_rn(2.0, bx.w);
    w.edge2 = __dmul_rn(edge, edge);
    w.first = nd.first[i];
    w.count = nd.count[i];
    w.info = info;
    w.mass = (float)r.m;
    w.q[0] = (float)q[0];
    w.q[1] = (float)q[1];
    w.q[2] = (float)q[2];
    w.q[3] = (float)q[3];
    nd.w[i] = w;
    nd.q45[i] = make_float2((float)q[4], (float)q[5]);
  }
}

// a5 level by level, deepest level first: one launch per level.
__global__ void k_moments(int depth, Nodes nd, const double4* __restrict__ pm, const DevState* __restrict__ st) {
  if (st->status & kStNodeOverflow) return;  // children may lie beyond the slots
  const uint32_t lb = st->level_begin[depth];
  const uint32_t lc = depth < (int)st->max_depth ? st->level_count[depth] : 0u;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < lc; k += gridDim.x * blockDim.x) {
    const uint32_t i = lb + k;
    if (i >= nd.cap) return;
    finalize_node<false>(nd, pm, i);
  }
}

// a5 in one launch: every leaf is finalized by one thread, which then climbs
// while it is the last of its parent's children to finish (a counter per
// node), so every node is finalized once, after all its children, and sums
// its children in order as finalize_node does level by level.  No thread
// waits for another.
__global__ void k_moments_up(Nodes nd, const double4* __restrict__ pm, const DevState* __restrict__ st) {
  if (st->status & kStNodeOverflow) return;  // children may lie beyond the slots
  const uint32_t nn = min(st->n_nodes, nd.cap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    if (!info_leaf(nd.info[i])) continue;
    uint32_t node = i;
    finalize_node<true>(nd, pm, node);
    for (;;) {
      const uint32_t par = nd.parent[node];
      if (par == kNoParent) break;
      __threadfence();  // this node's multipoles before the count
      const uint32_t done = atomicAdd(&nd.upcnt[par], 1u) + 1u;
      if (done < info_nchild(nd.info[par])) break;  // a sibling finishes the parent
      __threadfence();
      finalize_node<true>(nd, pm, par);
      node = par;
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers

void set_build_attributes() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(SortSmall::kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SortSmall::smem);
  cudaFuncSetAttribute(SortLarge::kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SortLarge::smem);
  done = true;
}

void launch_bounds_domain(const Particle* p, const Tile* tiles, int ntiles, SysDev* sys, int nsys, double* partial,
                          DevState* st, cudaStream_t s) {
  k_bounds<<<ntiles, kBoundsThreads, 0, s>>>(p, tiles, partial, st);
  k_domain<<<(nsys + 3) / 4, 128, 0, s>>>(sys, nsys, partial);
}

void launch_keys(const Particle* p, const Tile* tiles, int ntiles, const SysDev* sys, int nsys, uint64_t* keys,
                 uint32_t* hist, uint32_t* offs, cudaStream_t s) {
  k_keys<<<ntiles, kKeyThreads, 0, s>>>(p, tiles, sys, keys, hist);
  k_digit_offsets<<<nsys, 256, 0, s>>>(sys, hist, offs);
}

void launch_sort_pass(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, int pass,
                      const Tile* tiles, int ntiles, int tile_keys, const uint32_t* offs, uint32_t* lookback,
                      DevState* st, cudaStream_t s) {
  if (tile_keys == SortSmall::TILE)
    SortSmall::kernel()<<<ntiles, SortSmall::NT, SortSmall::smem, s>>>(kin, vin, kout, vout, pass, tiles, offs,
                                                                      lookback, st);
  else
    SortLarge::kernel()<<<ntiles, SortLarge::NT, SortLarge::smem, s>>>(kin, vin, kout, vout, pass, tiles, offs,
                                                                      lookback, st);
}

void launch_gather(const Particle* p, const uint32_t* perm, uint32_t n, Particle* staged, double4* pm, int sms,
                   cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > sms * 8) blocks = sms * 8;
  if (blocks < 1) blocks = 1;
  k_gather<<<blocks, 256, 0, s>>>(p, perm, n, staged, pm);
}

// Blocks for a grid that takes `units` work items `per_block` at a time, at
// most `cap` blocks (the rest of a larger grid would find no work).
static int grid_for(uint64_t units, uint64_t per_block, int cap) {
  const uint64_t b = (units + per_block - 1) / per_block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)cap));
}

// The nodes of level d-1 (the parents k_level reads) are at most 8^(d-1)
// per root, at most n, and at most 8 per interior node of the level above
// (an interior node holds more than max_leaf particles: at most
// n / (max_leaf + 1) of them per level), so the upper levels launch only the
// blocks that can find a tile.
void launch_topology(const SysDev* sys, int nsys, const Nodes& nd, const uint64_t* keys, unsigned max_leaf, uint32_t n,
                     uint32_t* lookback, DevState* st, int sms, cudaStream_t s) {
  k_roots<<<(nsys + 127) / 128, 128, 0, s>>>(sys, nsys, nd, max_leaf, st);
  const uint64_t below = std::min<uint64_t>(n, 8 * ((uint64_t)n / ((uint64_t)max_leaf + 1) + (uint64_t)nsys));
  uint64_t width = (uint64_t)nsys;  // 8^(d-1) per root
  for (int d = 1; d <= kMortonDepth; ++d) {
    const uint64_t parents = std::min(width, below);
    k_level<<<grid_for(parents, kLevelParents, sms * kLevelBlocksPerSm), kLevelThreads, 0, s>>>(d, nd, keys, max_leaf,
                                                                                               lookback, st);
    width = std::min<uint64_t>(width * 8, 1ull << 40);
  }
}

// Grids of the cut kernels (tiles and nodes taken by grid stride or by a
// counter): measured at 4M, the targets phase takes 0.179 ms with 4/2/2
// blocks per SM and 0.140 with 16/8/8.
void launch_targets(const Nodes& nd, uint32_t lim, uint32_t pack, uint32_t n, uint32_t* mark, uint32_t* targets,
                    uint32_t* chunks, uint32_t* groups, uint32_t* lookback, DevState* st, int sms, cudaStream_t s) {
  const uint32_t ntiles = (n + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
  const int gmark = grid_for(nd.cap, 256, sms * 16), gscan = grid_for(ntiles, 1, sms * 8);
  k_mark_cut<<<gmark, 256, 0, s>>>(nd, lim, st, mark);
  k_compact<<<gscan, kScanThreads, 0, s>>>(mark, n, targets, lookback, &st->scan_tiles, &st->n_targets, st);
  k_mark_cut<<<gmark, 256, 0, s>>>(nd, kPackChunk, st, mark);
  k_compact<<<gscan, kScanThreads, 0, s>>>(mark, n, chunks, lookback + (ntiles + 8), &st->chunk_tiles, &st->n_chunks,
                                           st);
  k_pack_groups<<<sms * 4, 256, 0, s>>>(chunks, targets, nd.begin, nd.count, pack, st, mark);
  k_compact<<<gscan, kScanThreads, 0, s>>>(mark, n, groups, lookback + 2 * (ntiles + 8), &st->group_tiles,
                                           &st->n_groups, st);
}

// Per-level multipoles at 16 blocks of 128 per SM: 0.233 ms at 4M, 0.270
// with 4.
void launch_moments(const Nodes& nd, const double4* pm, const DevState* st, int sms, bool one_launch, cudaStream_t s) {
  if (one_launch) {
    k_moments_up<<<grid_for(nd.cap, 128, sms * 4), 128, 0, s>>>(nd, pm, st);
  } else {
    for (int d = kMortonDepth; d >= 0; --d) k_moments<<<sms * 16, 128, 0, s>>>(d, nd, pm, st);
  }
}

}  // namespace bhg
