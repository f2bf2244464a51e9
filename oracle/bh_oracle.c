/* TEST INFRASTRUCTURE ONLY - the CPU oracle of the Barnes-Hut hot path.
 *
 * A plain-C restatement of the reference solver's grouped pipeline
 * (devreal/AMT-BH-benchmark, ttg-parsec/src): bounding cube -> 63-bit Morton
 * keys -> (key, index) sort -> octree -> multipoles -> bounding-box MAC walk
 * -> softened monopole+quadrupole forces -> kick/drift.  Every function cites
 * the reference file:line it restates.  Only tests/, the smoke check and the
 * benchmark's CPU-baseline leg load this library, and only to check or time
 * against; the product path never calls it.
 *
 * Parity pin: tests/test_oracle_pin.py checks this restatement against the
 * reference's own code compiled here (oracle/_ref, built by oracle/Makefile
 * from the unmodified reference sources) and against tests/golden/.
 *
 * Layout conventions (shared with the GPU build so arrays compare 1:1):
 *   - particles: 64-byte records {u32 id; u32 pad; f64 mass; f64 pos[3];
 *     f64 vel[3]} (bh::Particle, particle.h:7-24);
 *   - nodes: level order (breadth first from the root(s)); the children of a
 *     node are consecutive and in octant order.  The reference numbers its
 *     nodes differently (backbone BFS + per-subtree BFS,
 *     flat_build_ttg.h:200-263); node SETS are compared, not indices.
 *
 * Compile with -ffp-contract=off: the reference is built as ISO C++20
 * (CMakeLists.txt:4-6, CMAKE_CXX_EXTENSIONS OFF), under which GCC does not
 * contract a*b+c, so plain IEEE operations reproduce its rounding.
 */
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint32_t id;
  uint32_t pad;
  double mass;
  double pos[3];
  double vel[3];
} bho_particle;

#define BHO_DEPTH 21 /* kMortonDepth, flat_tree.h:102 */

/* ---- a1: bounds + domain --------------------------------------------- */

/* particle_bounds (flat_build_ttg.h:93-113) followed by domain_from_bounds
 * (domain.h:23-30).  out = {cx, cy, cz, half_width}.  Returns 1 if a
 * coordinate is not finite (the GPU path rejects such input). */
int bho_domain(const bho_particle* p, size_t n, double out[4]) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  int bad = 0;
  for (size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      double v = p[i].pos[a];
      if (!isfinite(v)) bad = 1;
      if (v < lo[a]) lo[a] = v; /* std::min(lo, v) keeps lo unless v < lo */
      if (hi[a] < v) hi[a] = v; /* std::max(hi, v) keeps hi unless hi < v */
    }
  }
  for (int a = 0; a < 3; ++a) out[a] = 0.5 * (lo[a] + hi[a]);
  double w = hi[0] - lo[0];
  if (w < hi[1] - lo[1]) w = hi[1] - lo[1]; /* std::max({..}) */
  if (w < hi[2] - lo[2]) w = hi[2] - lo[2];
  double hw = 0.5 * w;
  if (!(hw > 0.0)) hw = 1.0;
  hw *= 1.0 + 1e-9;
  out[3] = hw;
  return bad;
}

/* ---- a2: Morton keys ------------------------------------------------- */

/* spread_bits3, flat_tree.h:104-112 */
static uint64_t spread_bits3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

/* morton_key, flat_tree.h:114-125 */
static uint64_t morton_key(const double dom[4], const double* pos) {
  const double cells = (double)(1u << BHO_DEPTH);
  double scale = cells / (2.0 * dom[3]);
  uint32_t q[3];
  for (int a = 0; a < 3; ++a) {
    double lo = dom[a] - dom[3];
    double v = floor((pos[a] - lo) * scale);
    if (v < 0.0) v = 0.0; /* std::clamp(v, 0, cells - 1) */
    if (cells - 1.0 < v) v = cells - 1.0;
    q[a] = (uint32_t)v;
  }
  return spread_bits3(q[0]) | (spread_bits3(q[1]) << 1) | (spread_bits3(q[2]) << 2);
}

void bho_keys(const bho_particle* p, size_t n, const double dom[4], uint64_t* keys) {
  for (size_t i = 0; i < n; ++i) keys[i] = morton_key(dom, p[i].pos);
}

/* ---- a3: sort by (key, index) ---------------------------------------- */

typedef struct {
  uint64_t key;
  uint32_t index;
} key_index;

/* KeyIndex::operator<, flat_build_ttg.h:62-66 */
static int cmp_key_index(const void* a, const void* b) {
  const key_index* x = (const key_index*)a;
  const key_index* y = (const key_index*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return (x->index > y->index) - (x->index < y->index);
}

/* The order sort_particles (flat_build_ttg.h:117-190) produces: perm[i] is
 * the input index of the i-th particle in Morton order. */
void bho_sort(const uint64_t* keys, size_t n, uint32_t* perm, uint64_t* sorted_keys) {
  key_index* ki = (key_index*)malloc(sizeof(key_index) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) {
    ki[i].key = keys[i];
    ki[i].index = (uint32_t)i;
  }
  qsort(ki, n, sizeof(key_index), cmp_key_index);
  for (size_t i = 0; i < n; ++i) {
    perm[i] = ki[i].index;
    sorted_keys[i] = ki[i].key;
  }
  free(ki);
}

/* ---- a4: octree topology ---------------------------------------------- */

typedef struct {
  uint32_t *begin, *count, *first_child, *nchild, *leaf, *depth;
  double *center, *hw; /* center: 3 per node */
  double *mass, *com, *iab; /* com: 3 per node; iab: 6 per node (xx,yy,zz,xy,xz,yz) */
} bho_tree;

static unsigned octant_digit(uint64_t key, int depth) { /* flat_tree.h:127-129 */
  return (unsigned)((key >> (63 - 3 * depth)) & 7u);
}

/* LeafRule::stops with the whole key range owned (flat_tree.h:144-156) */
static int stops(uint32_t count, int depth, unsigned max_leaf) {
  return count <= max_leaf || depth >= BHO_DEPTH;
}

/* split_octants, flat_tree.h:167-180 (linear scan; the ranges are the same) */
static int split_octants(const uint64_t* keys, uint32_t lo, uint32_t hi, int cdepth, uint32_t rlo[8],
                         uint32_t rhi[8], unsigned roct[8]) {
  int k = 0;
  uint32_t j = lo;
  while (j < hi) {
    unsigned oct = octant_digit(keys[j], cdepth);
    uint32_t e = j + 1;
    while (e < hi && octant_digit(keys[e], cdepth) == oct) ++e;
    rlo[k] = j;
    rhi[k] = e;
    roct[k] = oct;
    ++k;
    j = e;
  }
  return k;
}

/* Number of nodes the build below creates for the segments
 * (seg_begin[s], seg_n[s]) of the sorted keys. */
size_t bho_count_nodes(const uint64_t* keys, const uint32_t* seg_begin, const uint32_t* seg_n, size_t nseg,
                       unsigned max_leaf) {
  /* explicit stack of (lo, hi, depth), as count_subtree (flat_tree.h:236-251) */
  size_t cap = 1024, top = 0, total = 0;
  uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * 3 * cap);
  for (size_t s = 0; s < nseg; ++s) {
    if (seg_n[s] == 0) continue;
    st[0] = seg_begin[s];
    st[1] = seg_begin[s] + seg_n[s];
    st[2] = 0;
    top = 1;
    while (top > 0) {
      --top;
      uint32_t lo = st[3 * top], hi = st[3 * top + 1];
      int d = (int)st[3 * top + 2];
      ++total;
      if (stops(hi - lo, d, max_leaf)) continue;
      uint32_t rlo[8], rhi[8];
      unsigned ro[8];
      int k = split_octants(keys, lo, hi, d + 1, rlo, rhi, ro);
      if (top + (size_t)k > cap) {
        cap *= 2;
        st = (uint32_t*)realloc(st, sizeof(uint32_t) * 3 * cap);
      }
      for (int c = 0; c < k; ++c, ++top) {
        st[3 * top] = rlo[c];
        st[3 * top + 1] = rhi[c];
        st[3 * top + 2] = (uint32_t)(d + 1);
      }
    }
  }
  free(st);
  return total;
}

/* The octree of each segment, breadth first over all segments' roots:
 * init_node / split_node / child_center (flat_tree.h:182-225) with the leaf
 * rule of flat_tree.h:144-156.  dom holds 4 doubles (cx, cy, cz, hw) per
 * segment.  The tree must have room for bho_count_nodes() nodes.  Returns the
 * node count. */
size_t bho_build(const uint64_t* keys, const uint32_t* seg_begin, const uint32_t* seg_n, size_t nseg,
                 const double* dom, unsigned max_leaf, bho_tree* t) {
  size_t nn = 0;
  for (size_t s = 0; s < nseg; ++s) {
    if (seg_n[s] == 0) continue;
    size_t i = nn++;
    t->begin[i] = seg_begin[s];
    t->count[i] = seg_n[s];
    t->depth[i] = 0;
    t->leaf[i] = (uint32_t)stops(seg_n[s], 0, max_leaf);
    for (int a = 0; a < 3; ++a) t->center[3 * i + a] = dom[4 * s + a];
    t->hw[i] = dom[4 * s + 3];
    t->first_child[i] = 0;
    t->nchild[i] = 0;
  }
  for (size_t i = 0; i < nn; ++i) { /* nn grows: breadth first */
    if (t->leaf[i]) continue;
    uint32_t rlo[8], rhi[8];
    unsigned ro[8];
    int d = (int)t->depth[i];
    int k = split_octants(keys, t->begin[i], t->begin[i] + t->count[i], d + 1, rlo, rhi, ro);
    t->first_child[i] = (uint32_t)nn;
    t->nchild[i] = (uint32_t)k;
    double q = 0.5 * t->hw[i]; /* child_center, flat_tree.h:182-185 */
    for (int c = 0; c < k; ++c) {
      size_t j = nn++;
      t->begin[j] = rlo[c];
      t->count[j] = rhi[c] - rlo[c];
      t->depth[j] = (uint32_t)(d + 1);
      t->leaf[j] = (uint32_t)stops(t->count[j], d + 1, max_leaf);
      t->center[3 * j + 0] = t->center[3 * i + 0] + ((ro[c] & 1u) ? q : -q);
      t->center[3 * j + 1] = t->center[3 * i + 1] + ((ro[c] & 2u) ? q : -q);
      t->center[3 * j + 2] = t->center[3 * i + 2] + ((ro[c] & 4u) ? q : -q);
      t->hw[j] = 0.5 * t->hw[i];
      t->first_child[j] = 0;
      t->nchild[j] = 0;
    }
  }
  return nn;
}

/* ---- a5: multipoles --------------------------------------------------- */

typedef struct {
  double mass, m1[3], m2[6];
} raw_moment;

/* outer_sym, multipole.h:15-18: (scale*d_a)*d_b in xx,yy,zz,xy,xz,yz order */
static void outer_sym(const double d[3], double s, double o[6]) {
  o[0] = s * d[0] * d[0];
  o[1] = s * d[1] * d[1];
  o[2] = s * d[2] * d[2];
  o[3] = s * d[0] * d[1];
  o[4] = s * d[0] * d[2];
  o[5] = s * d[1] * d[2];
}

/* RawMoment::operator+= (multipole.h:39-44) */
static void rm_add(raw_moment* a, const raw_moment* b) {
  a->mass += b->mass;
  for (int k = 0; k < 3; ++k) a->m1[k] += b->m1[k];
  for (int k = 0; k < 6; ++k) a->m2[k] += b->m2[k];
}

/* Multipoles of every node, deepest first: finalize_node (flat_tree.h:257-274)
 * with raw_moment_of_particle (multipole.h:52-59), raw_moment_from_multipole
 * (:92-102) and finalize_raw_moment (:76-87).  x,y,z,m: Morton-order SoA. */
void bho_multipoles(bho_tree* t, size_t nn, const double* x, const double* y, const double* z, const double* m) {
  for (size_t ii = nn; ii-- > 0;) {
    const double* ref = &t->center[3 * ii];
    raw_moment rm;
    memset(&rm, 0, sizeof rm);
    if (t->leaf[ii]) {
      for (uint32_t p = t->begin[ii]; p < t->begin[ii] + t->count[ii]; ++p) {
        raw_moment o;
        double d[3] = {x[p] - ref[0], y[p] - ref[1], z[p] - ref[2]};
        o.mass = m[p];
        for (int k = 0; k < 3; ++k) o.m1[k] = m[p] * d[k];
        outer_sym(d, m[p], o.m2);
        rm_add(&rm, &o);
      }
    } else {
      for (uint32_t c = 0; c < t->nchild[ii]; ++c) {
        size_t ch = t->first_child[ii] + c;
        raw_moment o;
        double d[3], sh[6];
        for (int k = 0; k < 3; ++k) d[k] = t->com[3 * ch + k] - ref[k];
        o.mass = t->mass[ch];
        for (int k = 0; k < 3; ++k) o.m1[k] = t->mass[ch] * d[k];
        outer_sym(d, t->mass[ch], sh);
        for (int k = 0; k < 6; ++k) o.m2[k] = t->iab[6 * ch + k] + sh[k];
        rm_add(&rm, &o);
      }
    }
    double inv = 1.0 / rm.mass, delta[3], sh[6];
    for (int k = 0; k < 3; ++k) delta[k] = inv * rm.m1[k];
    t->mass[ii] = rm.mass;
    for (int k = 0; k < 3; ++k) t->com[3 * ii + k] = ref[k] + delta[k];
    outer_sym(delta, rm.mass, sh);
    for (int k = 0; k < 6; ++k) t->iab[6 * ii + k] = rm.m2[k] - sh[k];
  }
}

/* ---- a6-a8: the walk --------------------------------------------------- */

/* accel_from_source (multipole.h:171-200), without the factor G */
static void accel_cell(const double tp[3], double mass, const double com[3], const double iab[6], double eps2,
                       int quad, double a[3]) {
  double d[3] = {com[0] - tp[0], com[1] - tp[1], com[2] - tp[2]};
  double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double ds2 = d2 + eps2;
  double ds = sqrt(ds2);
  double inv3 = 1.0 / (ds2 * ds);
  double s = mass * inv3;
  double r[3] = {s * d[0], s * d[1], s * d[2]};
  if (quad) {
    double tr = iab[0] + iab[1] + iab[2];
    double q[6];
    for (int k = 0; k < 3; ++k) q[k] = 3.0 * iab[k] - tr;
    for (int k = 3; k < 6; ++k) q[k] = 3.0 * iab[k];
    double qd[3] = {q[0] * d[0] + q[3] * d[1] + q[4] * d[2], q[3] * d[0] + q[1] * d[1] + q[5] * d[2],
                    q[4] * d[0] + q[5] * d[1] + q[2] * d[2]};
    double dqd = d[0] * qd[0] + d[1] * qd[1] + d[2] * qd[2];
    double inv5 = inv3 / ds2, inv7 = inv5 / ds2;
    for (int k = 0; k < 3; ++k) r[k] += (-1.0) * inv5 * qd[k];
    double c = 2.5 * dqd * inv7;
    for (int k = 0; k < 3; ++k) r[k] += c * d[k];
  }
  a[0] += r[0];
  a[1] += r[1];
  a[2] += r[2];
}

/* One particle-particle term of accumulate_list (grouped_ttg.h:124-163): the
 * r2 == 0 entries are masked when eps2 == 0 (Mask) and contribute 0 otherwise. */
static void accel_pp(const double tp[3], double sx, double sy, double sz, double sm, double eps2, double a[3]) {
  double dx = sx - tp[0], dy = sy - tp[1], dz = sz - tp[2];
  double r2 = dx * dx + dy * dy + dz * dz + eps2;
  if (!(r2 > 0.0)) return;
  double inv = 1.0 / sqrt(r2);
  double s = sm * inv * inv * inv;
  a[0] += s * dx;
  a[1] += s * dy;
  a[2] += s * dz;
}

typedef struct {
  double theta, eps2, G;
  int use_quadrupole;
} bho_params; /* ForceParams, traversal_ttg.h:136-141 */

/* Targets of the walk: the topmost nodes that are leaves or hold at most
 * min(target_size, group_size) particles.  The reference visits each group
 * root (the topmost nodes with count <= group_size, or leaves,
 * flat_tree.h:190-192) and descends to its targets (leaf or count <=
 * target_size, grouped_ttg.h:253), so a target is the deeper of the two
 * cut points on every root-to-leaf path.  group_size 0 (the per-node pass)
 * and target_size 0 both give the leaves.  Writes the target node indices
 * in Morton order (ascending particle_begin) and returns their number. */
size_t bho_targets(const bho_tree* t, size_t nn, uint32_t target_size, uint32_t group_size, uint32_t* out) {
  uint32_t lim = target_size < group_size ? target_size : group_size;
  /* walk depth first in child order from each root: Morton order */
  size_t cnt = 0, top = 0, cap = 1024;
  uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * cap);
  size_t nroots = 0;
  while (nroots < nn && t->depth[nroots] == 0) ++nroots;
  for (size_t r = 0; r < nroots; ++r) {
    st[0] = (uint32_t)r;
    top = 1;
    while (top > 0) {
      uint32_t i = st[--top];
      if (t->leaf[i] || t->count[i] <= lim) {
        out[cnt++] = i;
        continue;
      }
      if (top + 8 > cap) {
        cap *= 2;
        st = (uint32_t*)realloc(st, sizeof(uint32_t) * cap);
      }
      for (uint32_t c = t->nchild[i]; c-- > 0;) st[top++] = t->first_child[i] + c;
    }
  }
  free(st);
  return cnt;
}

/* BBox::near2 (multipole.h:132-136) and mac_accept_bbox (:151-153) */
static int mac_accept(const double lo[3], const double hi[3], const double com[3], double hw, double theta) {
  double d2 = 0.0;
  double dd[3];
  for (int a = 0; a < 3; ++a) {
    double u = lo[a] - com[a], v = com[a] - hi[a];
    double w = u > v ? u : v;
    dd[a] = w > 0.0 ? w : 0.0;
  }
  d2 = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
  double edge = 2.0 * hw;
  return theta * theta * d2 > edge * edge;
}

/* Accelerations (times G) on every particle, Morton order, by a walk from
 * the target's root per target node.  The list a target gets is the one the
 * reference's shared GroupWalker builds (grouped_ttg.h:42-51, :251-288):
 * MAC on the bounding box of the target's particles, leaves MAC-tested too,
 * everything not accepted opened, opened leaves direct-summed (the target's
 * own particles included).  Accepted cells are quadrupoles (use_quadrupole)
 * or monopoles.  roots[] gives the root node of every target's segment
 * (NULL: node 0).  counts[0] += particle-particle interactions, counts[1] +=
 * particle-cell interactions (per target particle x list entry). */
void bho_walk(const bho_tree* t, size_t nn, const uint32_t* targets, size_t ntargets, const uint32_t* roots,
              const double* x, const double* y, const double* z, const double* m, const bho_params* fp_per_target,
              double* acc, uint64_t* counts) {
  (void)nn;
  size_t cap = 4096;
  uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * cap);
  size_t lcap = 4096, ccap = 4096;
  uint32_t* cells = (uint32_t*)malloc(sizeof(uint32_t) * ccap);
  uint32_t* leaves = (uint32_t*)malloc(sizeof(uint32_t) * lcap);
  for (size_t ti = 0; ti < ntargets; ++ti) {
    const bho_params* fp = &fp_per_target[ti];
    uint32_t tn = targets[ti];
    uint32_t tb = t->begin[tn], tc = t->count[tn];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t p = tb; p < tb + tc; ++p) { /* BBox::add, multipole.h:121-128 */
      double v[3] = {x[p], y[p], z[p]};
      for (int a = 0; a < 3; ++a) {
        if (v[a] < lo[a]) lo[a] = v[a];
        if (hi[a] < v[a]) hi[a] = v[a];
      }
    }
    size_t ncell = 0, nleaf = 0, top = 0;
    st[top++] = roots ? roots[ti] : 0;
    while (top > 0) {
      uint32_t s = st[--top];
      if (mac_accept(lo, hi, &t->com[3 * s], t->hw[s], fp->theta)) {
        if (ncell == ccap) {
          ccap *= 2;
          cells = (uint32_t*)realloc(cells, sizeof(uint32_t) * ccap);
        }
        cells[ncell++] = s;
      } else if (t->leaf[s]) {
        if (nleaf == lcap) {
          lcap *= 2;
          leaves = (uint32_t*)realloc(leaves, sizeof(uint32_t) * lcap);
        }
        leaves[nleaf++] = s;
      } else {
        if (top + 8 > cap) {
          cap *= 2;
          st = (uint32_t*)realloc(st, sizeof(uint32_t) * cap);
        }
        for (uint32_t c = t->nchild[s]; c-- > 0;) st[top++] = t->first_child[s] + c;
      }
    }
    uint64_t npart = 0;
    for (size_t l = 0; l < nleaf; ++l) npart += t->count[leaves[l]];
    counts[0] += (uint64_t)tc * (npart + (fp->use_quadrupole ? 0 : ncell));
    counts[1] += (uint64_t)tc * (fp->use_quadrupole ? ncell : 0);
    for (uint32_t p = tb; p < tb + tc; ++p) {
      double tp[3] = {x[p], y[p], z[p]};
      double a[3] = {0.0, 0.0, 0.0};
      for (size_t l = 0; l < nleaf; ++l) {
        uint32_t s = leaves[l];
        for (uint32_t q = t->begin[s]; q < t->begin[s] + t->count[s]; ++q) accel_pp(tp, x[q], y[q], z[q], m[q], fp->eps2, a);
      }
      for (size_t c = 0; c < ncell; ++c) {
        uint32_t s = cells[c];
        if (fp->use_quadrupole) {
          accel_cell(tp, t->mass[s], &t->com[3 * s], &t->iab[6 * s], fp->eps2, 1, a);
        } else {
          accel_pp(tp, t->com[3 * s], t->com[3 * s + 1], t->com[3 * s + 2], t->mass[s], fp->eps2, a);
        }
      }
      /* on_result(particle, G * acc), grouped_ttg.h:281-283 */
      acc[3 * (size_t)p + 0] = fp->G * a[0];
      acc[3 * (size_t)p + 1] = fp->G * a[1];
      acc[3 * (size_t)p + 2] = fp->G * a[2];
    }
  }
  free(st);
  free(cells);
  free(leaves);
}

/* ---- oracles beside the path ------------------------------------------- */

/* brute_force_accel (brute_force.h:15-28) for the sample rows idx[0..ns):
 * softened direct sum over every other particle, times G. */
void bho_direct(const double* x, const double* y, const double* z, const double* m, size_t n, const uint32_t* idx,
                size_t ns, double eps2, double G, double* out) {
  for (long k = 0; k < (long)ns; ++k) {
    uint32_t i = idx[k];
    double tp[3] = {x[i], y[i], z[i]};
    double a[3] = {0.0, 0.0, 0.0};
    double zero[6] = {0, 0, 0, 0, 0, 0};
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double com[3] = {x[j], y[j], z[j]};
      accel_cell(tp, m[j], com, zero, eps2, 0, a);
    }
    out[3 * k + 0] = G * a[0];
    out[3 * k + 1] = G * a[1];
    out[3 * k + 2] = G * a[2];
  }
}

/* kick_one / drift_one (integrate.h:15-16) as the integrate callback of
 * step_particles applies them (integrate_ttg.h:74-77). acc already holds G*a. */
void bho_integrate(bho_particle* p, size_t n, const double* acc, double kick_dt, double drift_dt) {
  for (size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) p[i].vel[a] += kick_dt * acc[3 * i + a];
    if (drift_dt != 0.0) {
      for (int a = 0; a < 3; ++a) p[i].pos[a] += drift_dt * p[i].vel[a];
    }
  }
}

/* kinetic_energy (integrate.h:27-31) */
double bho_kinetic(const bho_particle* p, size_t n) {
  double e = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double* v = p[i].vel;
    e += 0.5 * p[i].mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  return e;
}

/* potential_energy (integrate.h:35-43): unsoftened, O(N^2) */
double bho_potential(const bho_particle* p, size_t n, double G) {
  double e = 0.0;
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = i + 1; j < n; ++j) {
      double d[3] = {p[i].pos[0] - p[j].pos[0], p[i].pos[1] - p[j].pos[1], p[i].pos[2] - p[j].pos[2]};
      e -= G * p[i].mass * p[j].mass / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
  }
  return e;
}

/* ---- a10: one whole step of one or more independent systems ------------- */

/* step_particles' grouped branch (integrate_ttg.h:88-107) for nseg systems
 * stored back to back (seg_begin/seg_n): build, walk, kick/drift, with the
 * particles of each segment returned in Morton order (the buffer swap at
 * integrate_ttg.h:107).  fp/kick/drift per segment.  acc_out (optional):
 * G*a per particle in the output order.  Returns 0, or 1 on non-finite
 * input. */
int bho_step(bho_particle* p, const uint32_t* seg_begin, const uint32_t* seg_n, size_t nseg, const bho_params* fp,
             const double* kick_dt, const double* drift_dt, unsigned max_leaf, uint32_t group_size,
             uint32_t target_size, double* acc_out, uint64_t* counts) {
  size_t n = 0;
  for (size_t s = 0; s < nseg; ++s) n += seg_n[s];
  double* dom = (double*)malloc(sizeof(double) * 4 * (nseg ? nseg : 1));
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t* skeys = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint32_t* perm = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  bho_particle* tmp = (bho_particle*)malloc(sizeof(bho_particle) * (n ? n : 1));
  int bad = 0;
  for (size_t s = 0; s < nseg; ++s) {
    const bho_particle* ps = p + seg_begin[s];
    if (seg_n[s] == 0) continue;
    bad |= bho_domain(ps, seg_n[s], &dom[4 * s]);
    bho_keys(ps, seg_n[s], &dom[4 * s], keys + seg_begin[s]);
    bho_sort(keys + seg_begin[s], seg_n[s], perm + seg_begin[s], skeys + seg_begin[s]);
    for (uint32_t i = 0; i < seg_n[s]; ++i) tmp[seg_begin[s] + i] = ps[perm[seg_begin[s] + i]];
  }
  if (bad) {
    free(dom), free(keys), free(skeys), free(perm), free(tmp);
    return 1;
  }
  memcpy(p, tmp, sizeof(bho_particle) * n);
  double* x = (double*)malloc(sizeof(double) * 4 * (n ? n : 1));
  double *y = x + n, *z = y + n, *m = z + n;
  for (size_t i = 0; i < n; ++i) {
    x[i] = p[i].pos[0];
    y[i] = p[i].pos[1];
    z[i] = p[i].pos[2];
    m[i] = p[i].mass;
  }
  size_t cap = bho_count_nodes(skeys, seg_begin, seg_n, nseg, max_leaf);
  bho_tree t;
  uint32_t* u = (uint32_t*)malloc(sizeof(uint32_t) * 6 * (cap ? cap : 1));
  t.begin = u, t.count = u + cap, t.first_child = u + 2 * cap, t.nchild = u + 3 * cap, t.leaf = u + 4 * cap,
  t.depth = u + 5 * cap;
  double* dd = (double*)malloc(sizeof(double) * 14 * (cap ? cap : 1));
  t.center = dd, t.hw = dd + 3 * cap, t.mass = dd + 4 * cap, t.com = dd + 5 * cap, t.iab = dd + 8 * cap;
  size_t nn = bho_build(skeys, seg_begin, seg_n, nseg, dom, max_leaf, &t);
  bho_multipoles(&t, nn, x, y, z, m);
  uint32_t* targets = (uint32_t*)malloc(sizeof(uint32_t) * (nn ? nn : 1));
  size_t nt = bho_targets(&t, nn, target_size, group_size, targets);
  uint32_t* roots = (uint32_t*)malloc(sizeof(uint32_t) * (nt ? nt : 1));
  bho_params* tfp = (bho_params*)malloc(sizeof(bho_params) * (nt ? nt : 1));
  double* acc = (double*)malloc(sizeof(double) * 3 * (n ? n : 1));
  /* root r of segment order: roots are nodes 0..(nonempty segments - 1) */
  {
    size_t r = 0, seg = 0;
    uint32_t* root_of_seg = (uint32_t*)malloc(sizeof(uint32_t) * (nseg ? nseg : 1));
    for (size_t s = 0; s < nseg; ++s) root_of_seg[s] = seg_n[s] ? (uint32_t)r++ : UINT32_MAX;
    for (size_t k = 0; k < nt; ++k) {
      uint32_t b = t.begin[targets[k]];
      while (!(seg_n[seg] && b >= seg_begin[seg] && b < seg_begin[seg] + seg_n[seg])) ++seg;
      roots[k] = root_of_seg[seg];
      tfp[k] = fp[seg];
    }
    free(root_of_seg);
  }
  bho_walk(&t, nn, targets, nt, roots, x, y, z, m, tfp, acc, counts);
  for (size_t s = 0; s < nseg; ++s) {
    bho_integrate(p + seg_begin[s], seg_n[s], acc + 3 * (size_t)seg_begin[s], kick_dt[s], drift_dt[s]);
  }
  if (acc_out) memcpy(acc_out, acc, sizeof(double) * 3 * n);
  free(dom), free(keys), free(skeys), free(perm), free(tmp), free(x), free(u), free(dd), free(targets), free(roots),
      free(tfp), free(acc);
  return 0;
}

/* ---- particle text: read_csv (io.cc:70-178) and write_vtk (io.cc:180-195) ----
 *
 * The numbers follow std::from_chars(double, general): the grammar is checked
 * here and the value comes from the C library's strtod on exactly the
 * accepted characters (glibc's strtod is correctly rounded, as from_chars is);
 * a nonzero value that rounds to zero or to infinity is out of range. */

static const char* bho_skip_blanks(const char* p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\t')) ++p;
  return p;
}

static int bho_lower(int c) { return c | 0x20; }

/* end of the from_chars number at p (p itself when there is none) */
static const char* bho_number_end(const char* p, const char* end, int* nonzero, int* special) {
  const char* s = p;
  *nonzero = 0;
  *special = 0;
  if (s < end && *s == '-') ++s;
  if (s + 3 <= end && bho_lower(s[0]) == 'i' && bho_lower(s[1]) == 'n' && bho_lower(s[2]) == 'f') {
    s += 3;
    if (s + 5 <= end && bho_lower(s[0]) == 'i' && bho_lower(s[1]) == 'n' && bho_lower(s[2]) == 'i' &&
        bho_lower(s[3]) == 't' && bho_lower(s[4]) == 'y')
      s += 5;
    *special = 1;
    return s;
  }
  if (s + 3 <= end && bho_lower(s[0]) == 'n' && bho_lower(s[1]) == 'a' && bho_lower(s[2]) == 'n') {
    s += 3;
    if (s < end && *s == '(') {
      const char* t = s + 1;
      while (t < end && ((*t >= '0' && *t <= '9') || (bho_lower(*t) >= 'a' && bho_lower(*t) <= 'z') || *t == '_')) ++t;
      if (t < end && *t == ')') s = t + 1;
    }
    *special = 1;
    return s;
  }
  int digits = 0;
  while (s < end && *s >= '0' && *s <= '9') digits++, *nonzero |= *s != '0', ++s;
  if (s < end && *s == '.') {
    ++s;
    while (s < end && *s >= '0' && *s <= '9') digits++, *nonzero |= *s != '0', ++s;
  }
  if (!digits) return p;
  if (s < end && bho_lower(*s) == 'e') {
    const char* t = s + 1;
    if (t < end && (*t == '+' || *t == '-')) ++t;
    if (t < end && *t >= '0' && *t <= '9') {
      while (t < end && *t >= '0' && *t <= '9') ++t;
      s = t;
    }
  }
  return s;
}

/* parse_field (io.cc:76-91) for a double; 0 on success */
static int bho_field_f64(const char** pp, const char* end, double* out, int last) {
  const char* p = bho_skip_blanks(*pp, end);
  int nonzero, special;
  const char* q = bho_number_end(p, end, &nonzero, &special);
  if (q == p) return 1;
  char buf[1100];
  char* heap = NULL;
  char* tmp = buf;
  const size_t len = (size_t)(q - p);
  if (len + 1 > sizeof buf) tmp = heap = (char*)malloc(len + 1);
  memcpy(tmp, p, len);
  tmp[len] = 0;
  const double v = strtod(tmp, NULL);
  free(heap);
  if (!special && (isinf(v) || (v == 0.0 && nonzero))) return 1; /* result_out_of_range */
  *out = v;
  q = bho_skip_blanks(q, end);
  if (last) {
    if (q < end && *q == '\r') ++q;
    if (q != end) return 1;
  } else {
    if (q >= end || *q != ',') return 1;
    ++q;
  }
  *pp = q;
  return 0;
}

/* the id field: from_chars into uint32 */
static int bho_field_id(const char** pp, const char* end, uint32_t* out) {
  const char* p = bho_skip_blanks(*pp, end);
  const char* q = p;
  uint64_t v = 0;
  while (q < end && *q >= '0' && *q <= '9') {
    v = v * 10 + (uint64_t)(*q - '0');
    if (v > 0xffffffffull) return 1;
    ++q;
  }
  if (q == p) return 1;
  *out = (uint32_t)v;
  q = bho_skip_blanks(q, end);
  if (q >= end || *q != ',') return 1;
  *pp = q + 1;
  return 0;
}

/* read_csv of a text in memory.  Returns 0 with *n particles (those beyond
 * cap are counted, not stored), or 1 with *bad_line the 0-based number of the
 * first malformed line. */
int bho_read_csv(const char* text, size_t nbytes, bho_particle* out, size_t cap, size_t* n, size_t* bad_line) {
  const char* begin = text;
  const char* end = text + nbytes;
  size_t line_no = 0;
  *n = 0;
  if (begin == end) return 0;
  { /* header: the first field of the first line is not an id (io.cc:136-141) */
    const char* eol = (const char*)memchr(begin, '\n', nbytes);
    const char* lim = eol ? eol : end;
    const char* p = bho_skip_blanks(begin, lim);
    const char* q = p;
    uint64_t v = 0;
    int over = 0;
    while (q < lim && *q >= '0' && *q <= '9') {
      v = v * 10 + (uint64_t)(*q - '0');
      if (v > 0xffffffffull) over = 1;
      ++q;
    }
    if (q == p || over) begin = eol ? eol + 1 : end, line_no = 1;
  }
  for (const char* line = begin; line < end; ++line_no) { /* parse_lines, io.cc:95-113 */
    const char* eol = (const char*)memchr(line, '\n', (size_t)(end - line));
    if (!eol) eol = end;
    const char* p = bho_skip_blanks(line, eol);
    if (p != eol && *p != '\r') {
      bho_particle q;
      memset(&q, 0, sizeof q);
      if (bho_field_id(&p, eol, &q.id) || bho_field_f64(&p, eol, &q.mass, 0) || bho_field_f64(&p, eol, &q.pos[0], 0) ||
          bho_field_f64(&p, eol, &q.pos[1], 0) || bho_field_f64(&p, eol, &q.pos[2], 0) ||
          bho_field_f64(&p, eol, &q.vel[0], 0) || bho_field_f64(&p, eol, &q.vel[1], 0) ||
          bho_field_f64(&p, eol, &q.vel[2], 1)) {
        *bad_line = line_no;
        return 1;
      }
      if (*n < cap) out[*n] = q;
      ++*n;
    }
    line = eol + 1;
  }
  return 0;
}

/* write_vtk's text (numbers as printf "%g"); returns its length and writes
 * min(length, cap) bytes to out */
size_t bho_write_vtk(const bho_particle* p, size_t n, char* out, size_t cap) {
  size_t len = 0;
  char buf[160];
#define BHO_PUT(s, k)                                         \
  do {                                                        \
    const size_t k_ = (size_t)(k);                            \
    if (len < cap) memcpy(out + len, s, len + k_ <= cap ? k_ : cap - len); \
    len += k_;                                                \
  } while (0)
  int k = snprintf(buf, sizeof buf,
                   "# vtk DataFile Version 3.0\npepc-ttg particle snapshot\nASCII\nDATASET POLYDATA\nPOINTS %zu double\n", n);
  BHO_PUT(buf, k);
  for (size_t i = 0; i < n; ++i) {
    k = snprintf(buf, sizeof buf, "%g %g %g\n", p[i].pos[0], p[i].pos[1], p[i].pos[2]);
    BHO_PUT(buf, k);
  }
  k = snprintf(buf, sizeof buf, "POINT_DATA %zu\nSCALARS mass double 1\nLOOKUP_TABLE default\n", n);
  BHO_PUT(buf, k);
  for (size_t i = 0; i < n; ++i) {
    k = snprintf(buf, sizeof buf, "%g\n", p[i].mass);
    BHO_PUT(buf, k);
  }
  BHO_PUT("VECTORS velocity double\n", 24);
  for (size_t i = 0; i < n; ++i) {
    k = snprintf(buf, sizeof buf, "%g %g %g\n", p[i].vel[0], p[i].vel[1], p[i].vel[2]);
    BHO_PUT(buf, k);
  }
#undef BHO_PUT
  return len;
}
