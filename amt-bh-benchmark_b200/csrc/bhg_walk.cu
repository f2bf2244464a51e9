// Force walk of the B200 Barnes-Hut path.
//
// What a target receives is exactly the reference's interaction list
// (GroupWalker, grouped_ttg.h:204-289): the bounding box of the target's
// particles (BBox, multipole.h:115-142) is tested against the visited nodes
// with mac_accept_bbox (multipole.h:151-153, strict theta^2 near^2 > edge^2,
// in FP64); leaves are tested too; accepted nodes are cell interactions
// (quadrupole, accel_from_source multipole.h:171-200, or monopoles in
// no-quad mode); everything else is opened - interior nodes push their
// children, leaves contribute their particles directly, the target's own
// leaf included (its self term is 0 with softening and masked at r^2 = 0
// without, accumulate_list grouped_ttg.h:117-163).
//
// One warp per walk GROUP (a run of consecutive targets of one system, at
// most kGroupMax particles and kMaxTargets targets, k_pack_groups), sharing
// the walk among the group's targets as GroupWalker::visit does, taken to
// every level: one traversal from the root whose stack entries carry the
// mask of targets that still need the node.  A node accepted for the
// group's bounding box is accepted by every target in the mask; one rejected
// for every point of it (mac_reject_all, multipole.h:158-160) is opened by
// all of them; otherwise each target in the mask tests its own box, one
// (node, target) pair per lane.  Sources every target of the group takes are
// evaluated once against all the group's particles; sources only some take
// go to the warp's list as (node or leaf run, target mask), and each target
// then passes over the list taking its own entries.  Each target's list is
// the same as a separate walk of its box from the root would build.
//
// A walk step pops up to 32 entries (one per lane) from a shared-memory
// stack; accepted cells and opened leaves' particles go to two
// shared-memory queues, and a full queue is evaluated as one batch (64 cells
// or 192 particles in split precision; one source per lane against up to 2
// targets per lane in FP64).
//
// Split precision: sources and targets become FP32 offsets from the walk's
// bounding-box centre (the subtraction in FP64), staged once per batch in
// shared memory; interactions are FP32 FMA + rsqrt.approx.ftz, lanes laid out as
// (target, source subset) (SplitEval below); FP32 partials go into FP64
// sums every 32 or more terms.  The kick/drift of integrate_ttg.h:74-77 is
// applied in FP64 in the epilogue.
#include "bhg_kernels.h"

#include <type_traits>

namespace bhg {

constexpr int kWalkWarps = 4;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kCellQ = 128;   // ring of accepted cells (a batch of up to 64 + one step's 32)
constexpr int kPartQ = 256;   // ring of direct particles (a batch of up to 192 + 32 enqueued)
constexpr int kStackCap = 704;   // per-warp stack: node + target mask per entry
constexpr int kStageF4 = 3 * 64 + 3;  // staged source records (float4): 64 cells + the zero cell
constexpr float kFarAway = 1.0e10f;  // padding source: contributes exactly 0
constexpr uint32_t kFull = 0xffffffffu;
// A list entry is (node, target mask) for a cell, or (first particle |
// kLeafBit, target mask | count << kCountShift) for a run of at most
// kMaxRun particles of a leaf (a larger leaf takes several entries), so that
// the targets' passes need no second load for it.
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr int kCountShift = 24;
constexpr uint32_t kMaxRun = 255;
static_assert(kMaxTargets <= kCountShift, "target masks and run lengths share a word");
constexpr uint32_t kListCap = 4096;         // entries of one partial-source list (32 KB)
constexpr uint32_t kNotShared = 0xffffffffu;  // a group whose list overflowed: its targets walk alone
// a group's list length before its shared walk has finished (two-pass schedule;
// the host fills the lengths with this byte pattern before every walk)
constexpr uint32_t kListPending = 0xfefefefeu;
// a walk that pops one node at a time holds at most 7 entries per level
// below the one it pops from, plus the root
static_assert(kStackCap >= 7 * kLevels + 1 + 8, "a one-at-a-time walk must fit the stack");
static_assert(kStageF4 * 16 >= 32 * 6 * 8, "the end-of-walk reduction reuses the staging records");

struct WarpSmem {
  uint32_t snode[kStackCap];  // traversal stack: node
  uint32_t smask[kStackCap];  //                  targets that still need it
  uint32_t cell[kCellQ];
  uint32_t part[kPartQ];
  float4 stage[kStageF4];
  double acc[kGroupMax][3];   // FP64 sum per particle of the group
  double tlo[kMaxTargets][3], thi[kMaxTargets][3];  // the targets' particle boxes
  double glo[3], ghi[3];                              // the group's particle box
  uint32_t tbeg[kMaxTargets], tcnt[kMaxTargets];      // the targets' particles
  uint32_t accbits[32];  // per popped entry: targets that accept it (per-target tests)
};
constexpr size_t kWalkSmem = sizeof(WarpSmem) * kWalkWarps;

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Squared distance from (x, y, z) to the nearest point of the box, as
// BBox::near2 (multipole.h:132-136) rounds it.
__device__ __forceinline__ double near2(const double lo[3], const double hi[3], double x, double y, double z) {
  double dx = fmax(fmax(__dsub_rn(lo[0], x), __dsub_rn(x, hi[0])), 0.0);
  double dy = fmax(fmax(__dsub_rn(lo[1], y), __dsub_rn(y, hi[1])), 0.0);
  double dz = fmax(fmax(__dsub_rn(lo[2], z), __dsub_rn(z, hi[2])), 0.0);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Squared distance to the farthest point of the box (BBox::far2, multipole.h:137-141).
__device__ __forceinline__ double far2(const double lo[3], const double hi[3], double x, double y, double z) {
  double dx = fmax(__dsub_rn(x, lo[0]), __dsub_rn(hi[0], x));
  double dy = fmax(__dsub_rn(y, lo[1]), __dsub_rn(hi[1], y));
  double dz = fmax(__dsub_rn(z, lo[2]), __dsub_rn(hi[2], z));
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// ---------------------------------------------------------------------------
// Evaluators: what a lane does with one chunk of sources - two per lane
// (sources j and j + L of the chunk for lane j of a group of L lanes), whose
// interactions with each target are independent chains.  Target slot k of
// lane group g is target g + k * gp; lane k mod L of the group adds that
// target's partial sums into its FP64 sum.

// Split precision.  Sources are staged once per batch in shared memory as
// FP32 records relative to the walk box's centre (the subtraction in FP64),
// and the warp is laid out as a grid of lanes: each lane owns kt (1 or 2)
// targets and one of ng lane groups, which split the batch's sources
// between them (group g takes sources g, g + ng, ...).  Every lane reads
// the records it needs from shared memory (all lanes of a group read the
// same record: a broadcast), so a source costs one global gather per warp,
// not one per lane group, and the lanes never exchange partial sums inside
// a batch.  Each loop iteration evaluates two independent (source, target)
// pairs: two sources for one target (kt = 1) or one source for two targets
// (kt = 2).  FP32 partials are added into per-lane FP64 sums once they hold
// 32 or more terms (at most one batch's worth) and at the end of the walk;
// then the lane groups' FP64 sums are added in group order (deterministic)
// into the targets' FP64 sums.
// rsqrt.approx.ftz.f32 (PTX ISA): the approximate reciprocal square root,
// subnormal inputs and results flushed to zero.  The split evaluator's r^2 is
// in units scaled to the system's size (at least eps^2 there, or masked when
// eps = 0), so the flush only drops contributions below FP32's normal range.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <bool QUAD, bool MASK>
struct SplitEval {
  // particle batches fill the staging records cells use (192 + the zero
  // record <= kStageF4): 0.35% faster at 4M than batches of 128
  static constexpr int kCellBatch = 64, kPartBatch = 192;
  // FP32 partials go into the FP64 sums once a lane has added kFlushTerms
  // or more terms to them (so they never hold more than one 64-cell
  // batch's worth), and at the end of the walk
  static constexpr int kFlushTerms = 32;
  static constexpr int kCellDummy = kCellBatch;  // record index of the zero cell (written once)
  static constexpr int kPartDummy = kPartBatch;  // record index of the zero particle (written per batch)
  static_assert(kPartBatch + 1 <= kStageF4 && kPartBatch + 32 <= kPartQ, "particle batch too large");
  const WalkArgs& a;
  float4* stage;  // records: cells 3 float4 each, particles 1 float4 each
  double* red;    // per-lane FP64 sums at the end of a walk (aliases stage)
  double cx, cy, cz;  // reference point: the walk box's centre
  float eps2;         // softening in scaled units
  // the FP32 arithmetic runs on offsets times a power of two near the
  // system's size (1 / 2^ilogb(domain half width)), so that r^-7 of the
  // smallest and largest systems stays inside FP32's range; the powers of two
  // make the scaling exact (rsqrt of an even power of two too), and the FP64
  // sums are scaled back
  double scale = 1.0, unscale2 = 1.0;  // see set_system
  float scale2f = 1.f;
  int lane, tb, kt, lpg, ng, first, stride, offb;
  float t0x, t0y, t0z, t1x, t1y, t1z;  // target positions (t1 = t0 when kt = 1)
  float a0x, a0y, a0z, a1x, a1y, a1z;  // FP32 partials of the current batch
  double s0x, s0y, s0z, s1x, s1y, s1z;  // FP64 sums of this lane
  double (*acc)[3];  // the targets' FP64 sums (shared memory)
  int pend;  // terms in this lane's FP32 partials since the last flush (an upper bound, warp-uniform)

  __device__ SplitEval(const WalkArgs& args, float4* stage_, int lane_) : a(args), stage(stage_), lane(lane_) {
    red = reinterpret_cast<double*>(stage_);
    if (lane == 0) {
      stage[3 * kCellDummy + 0] = make_float4(kFarAway, 0.f, 0.f, 0.f);
      stage[3 * kCellDummy + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
      stage[3 * kCellDummy + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncwarp();
  }

  __device__ int cell_chunk() const { return kCellBatch; }
  __device__ int part_chunk() const { return kPartBatch; }

  // softening eps2_ and the system's domain half width hw
  __device__ void set_system(double eps2_, double hw) {
    int k = hw > 0.0 ? ilogb(hw) : 0;
    k = k < -100 ? -100 : (k > 100 ? 100 : k);
    scale = ldexp(1.0, -k);            // offsets d' = d * scale
    unscale2 = ldexp(1.0, -2 * k);     // a = a' * scale^2 (a' = m d' / r'^3 = a / scale^2)
    scale2f = (float)ldexp(1.0, -2 * k);  // Q' = Q * scale^2, eps2' = eps2 * scale^2
    eps2 = (float)(eps2_ * (scale * scale));
  }

  // targets: particles p0 .. p0 + n - 1 (n <= 64); their FP64 sums are
  // added to sums[0 .. n)
  __device__ void setup(int, uint32_t p0, int n, double (*sums)[3]) {
    acc = sums;
    tb = n;
    // one target per lane with 32 / tb lane groups, or two targets per lane
    // with 32 / ceil(tb / 2) groups: whichever leaves fewer slots idle
    const int n1 = tb <= 32 ? 32 / tb : 0;
    const int l2 = (tb + 1) >> 1, n2 = 32 / l2;
    kt = (n1 == 0 || n2 >= 2 * n1) ? 2 : 1;
    lpg = kt == 1 ? tb : l2;
    ng = kt == 1 ? n1 : n2;
    const bool active = lane < lpg * ng;
    const int slot = lane % lpg;
    first = active ? lane / lpg : 1 << 30;  // inactive lanes take no sources
    stride = kt == 1 ? 2 * ng : ng;
    offb = kt == 1 ? ng : 0;
    const int t0 = slot, t1 = (kt == 2 && slot + lpg < tb) ? slot + lpg : slot;
    const double4 q0 = a.pm[p0 + t0], q1 = a.pm[p0 + t1];
    t0x = (float)(__dsub_rn(q0.x, cx) * scale), t0y = (float)(__dsub_rn(q0.y, cy) * scale);
    t0z = (float)(__dsub_rn(q0.z, cz) * scale);
    t1x = (float)(__dsub_rn(q1.x, cx) * scale), t1y = (float)(__dsub_rn(q1.y, cy) * scale);
    t1z = (float)(__dsub_rn(q1.z, cz) * scale);
    a0x = a0y = a0z = a1x = a1y = a1z = 0.f;
    s0x = s0y = s0z = s1x = s1y = s1z = 0.0;
    pend = 0;
  }

  __device__ __forceinline__ void flush() {
    s0x += (double)a0x * unscale2, s0y += (double)a0y * unscale2, s0z += (double)a0z * unscale2;
    if (kt == 1) {
      s0x += (double)a1x * unscale2, s0y += (double)a1y * unscale2, s0z += (double)a1z * unscale2;
    } else {
      s1x += (double)a1x * unscale2, s1y += (double)a1y * unscale2, s1z += (double)a1z * unscale2;
    }
    a0x = a0y = a0z = a1x = a1y = a1z = 0.f;
  }

  // one cell record's contribution to the target at (tx, ty, tz)
  __device__ __forceinline__ void cell_body(const float4* r, float tx, float ty, float tz, float& ax, float& ay,
                                            float& az) const {
    const float4 r0 = r[0];
    const float dx = r0.x - tx, dy = r0.y - ty, dz = r0.z - tz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    float ri = rsqrt_ftz(r2);
    if (!QUAD && MASK) ri = r2 > 0.f ? ri : 0.f;
    const float ri2 = ri * ri;
    const float ri3 = ri * ri2;
    if (QUAD) {
      const float4 r1 = r[1];
      const float2 r3 = *reinterpret_cast<const float2*>(&r[2]);
      // Q = [[q0 q3 q4] [q3 q1 q5] [q4 q5 q2]]
      const float qx = fmaf(r1.x, dx, fmaf(r1.w, dy, r3.x * dz));
      const float qy = fmaf(r1.w, dx, fmaf(r1.y, dy, r3.y * dz));
      const float qz = fmaf(r3.x, dx, fmaf(r3.y, dy, r1.z * dz));
      const float dqd = fmaf(dx, qx, fmaf(dy, qy, dz * qz));
      const float ri5 = ri3 * ri2;
      // m d / r^3 - Q d / r^5 + 2.5 (d Q d) d / r^7
      const float c = fmaf(2.5f * dqd, ri5 * ri2, r0.w * ri3);
      ax = fmaf(-ri5, qx, fmaf(c, dx, ax));
      ay = fmaf(-ri5, qy, fmaf(c, dy, ay));
      az = fmaf(-ri5, qz, fmaf(c, dz, az));
    } else {
      const float c = r0.w * ri3;
      ax = fmaf(c, dx, ax), ay = fmaf(c, dy, ay), az = fmaf(c, dz, az);
    }
  }

  __device__ __forceinline__ void part_body(const float4 r, float tx, float ty, float tz, float& ax, float& ay,
                                            float& az) const {
    const float dx = r.x - tx, dy = r.y - ty, dz = r.z - tz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    float ri = rsqrt_ftz(r2);
    if (MASK) ri = r2 > 0.f ? ri : 0.f;
    const float c = r.w * (ri * ri) * ri;
    ax = fmaf(c, dx, ax), ay = fmaf(c, dy, ay), az = fmaf(c, dz, az);
  }

  // accepted cells: node ids ring[(head + i) % kCellQ], i < cnt <= kCellBatch
  __device__ void cells(const uint32_t* ring, uint32_t head, int cnt) {
    for (int i = lane; i < cnt; i += 32) {
      const uint32_t n = ring[(head + (uint32_t)i) & (kCellQ - 1)];
      const WNode* w = a.w + n;
      const double2 cxy = *reinterpret_cast<const double2*>(&w->cx);
      const double czz = w->cz;
      const float4 r0 = make_float4((float)(__dsub_rn(cxy.x, cx) * scale), (float)(__dsub_rn(cxy.y, cy) * scale),
                                    (float)(__dsub_rn(czz, cz) * scale), w->mass);
      stage[3 * i] = r0;
      if (QUAD) {
        const float4 qa = *reinterpret_cast<const float4*>(w->q);
        const float2 qb = a.q45[n];
        // record layout: (q0 q1 q2 q3) (q4 q5 - -), in scaled units
        stage[3 * i + 1] = make_float4(qa.x * scale2f, qa.y * scale2f, qa.z * scale2f, qa.w * scale2f);
        stage[3 * i + 2] = make_float4(qb.x * scale2f, qb.y * scale2f, 0.f, 0.f);
      }
    }
    __syncwarp();
    for (int s = first; s < cnt; s += stride) {
      const int sb = s + offb < cnt ? s + offb : kCellDummy;
      cell_body(stage + 3 * s, t0x, t0y, t0z, a0x, a0y, a0z);
      cell_body(stage + 3 * sb, t1x, t1y, t1z, a1x, a1y, a1z);
    }
    pend += (cnt + stride - 1) / stride;
    if (pend >= kFlushTerms) flush(), pend = 0;
    __syncwarp();
  }

  // direct particles: particle indices ring[(head + i) % kPartQ], i < cnt <= kPartBatch
  __device__ void parts(const uint32_t* ring, uint32_t head, int cnt) {
    for (int i = lane; i < cnt; i += 32) {
      const double4 p = a.pm[ring[(head + (uint32_t)i) & (kPartQ - 1)]];
      stage[i] = make_float4((float)(__dsub_rn(p.x, cx) * scale), (float)(__dsub_rn(p.y, cy) * scale),
                             (float)(__dsub_rn(p.z, cz) * scale), (float)p.w);
    }
    if (lane == 0) stage[kPartDummy] = make_float4(kFarAway, 0.f, 0.f, 0.f);
    __syncwarp();
    for (int s = first; s < cnt; s += stride) {
      const int sb = s + offb < cnt ? s + offb : kPartDummy;
      part_body(stage[s], t0x, t0y, t0z, a0x, a0y, a0z);
      part_body(stage[sb], t1x, t1y, t1z, a1x, a1y, a1z);
    }
    pend += (cnt + stride - 1) / stride;
    if (pend >= kFlushTerms) flush(), pend = 0;
    __syncwarp();
  }

  // After a walk: the lane groups' sums, added in group order into every
  // target's FP64 sum.
  __device__ void finish() {
    if (pend) flush(), pend = 0;
    if (first < (1 << 30)) {
      double* r = red + 6 * lane;
      r[0] = s0x, r[1] = s0y, r[2] = s0z, r[3] = s1x, r[4] = s1y, r[5] = s1z;
    }
    __syncwarp();
    for (int t = lane; t < tb; t += 32) {
      const int k = t / lpg, sl = t - k * lpg;
      double x = 0.0, y = 0.0, z = 0.0;
      for (int g = 0; g < ng; ++g) {
        const double* r = red + 6 * (g * lpg + sl) + 3 * k;
        x += r[0], y += r[1], z += r[2];
      }
      acc[t][0] += x, acc[t][1] += y, acc[t][2] += z;
    }
    __syncwarp();
  }
};

// Plain FP64, up to 2 targets per lane, up to 64 per warp.  Absolute FP64
// positions; the formula of accel_from_source with multiplications by 1/r^2
// in place of its divisions.
template <bool QUAD, bool MASK>
struct F64Eval {
  static constexpr int TB = 2;
  const WalkArgs& a;
  double cx, cy, cz;  // unused: absolute positions
  double eps2;
  int L, gp, g, j, kmax;
  double tx[TB], ty[TB], tz[TB];
  double ax[TB], ay[TB], az[TB];
  double (*acc)[3];
  int ntb;

  __device__ F64Eval(const WalkArgs& args, float4*, int) : a(args) {}

  __device__ int cell_chunk() const { return 2 * L; }
  __device__ int part_chunk() const { return 2 * L; }
  __device__ void set_system(double eps2_, double) { eps2 = eps2_; }

  static __device__ int groups_for(int tb) {
    return tb <= 2 ? 1 : tb <= 4 ? 2 : tb <= 8 ? 4 : tb <= 16 ? 8 : tb <= 32 ? 16 : 32;
  }

  __device__ void setup(int lane, uint32_t p0, int tb, double (*sums)[3]) {
    acc = sums;
    ntb = tb;
    gp = groups_for(tb);
    L = 32 / gp;
    g = lane / L;
    j = lane & (L - 1);
    kmax = (tb + gp - 1) / gp;
    double p0x = 0, p0y = 0, p0z = 0, p1x = 0, p1y = 0, p1z = 0;
    if (lane < tb) {
      const double4 q = a.pm[p0 + lane];
      p0x = q.x, p0y = q.y, p0z = q.z;
    }
    if (lane + 32 < tb) {
      const double4 q = a.pm[p0 + 32 + lane];
      p1x = q.x, p1y = q.y, p1z = q.z;
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int t = g + k * gp;
      const double x0 = __shfl_sync(kFull, p0x, t & 31), x1 = __shfl_sync(kFull, p1x, t & 31);
      const double y0 = __shfl_sync(kFull, p0y, t & 31), y1 = __shfl_sync(kFull, p1y, t & 31);
      const double z0 = __shfl_sync(kFull, p0z, t & 31), z1 = __shfl_sync(kFull, p1z, t & 31);
      tx[k] = t < 32 ? x0 : x1;
      ty[k] = t < 32 ? y0 : y1;
      tz[k] = t < 32 ? z0 : z1;
      ax[k] = ay[k] = az[k] = 0.0;
    }
  }

  __device__ __forceinline__ void cell_one(int k, double sx, double sy, double sz, double m, const double q[6],
                                           double& rx, double& ry, double& rz) {
    const double dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
    const double r2 = dx * dx + dy * dy + dz * dz + eps2;
    double ri = rsqrt(r2);
    if (!QUAD && MASK) ri = r2 > 0.0 ? ri : 0.0;
    const double ri2 = ri * ri;
    const double ri3 = ri * ri2;
    if (QUAD) {
      const double qx = q[0] * dx + q[3] * dy + q[4] * dz;
      const double qy = q[3] * dx + q[1] * dy + q[5] * dz;
      const double qz = q[4] * dx + q[5] * dy + q[2] * dz;
      const double dqd = dx * qx + dy * qy + dz * qz;
      const double ri5 = ri3 * ri2;
      const double c = m * ri3 + 2.5 * dqd * (ri5 * ri2);
      rx = c * dx - ri5 * qx;
      ry = c * dy - ri5 * qy;
      rz = c * dz - ri5 * qz;
    } else {
      const double c = m * ri3;
      rx = c * dx, ry = c * dy, rz = c * dz;
    }
  }

  __device__ __forceinline__ void load_cell(const uint32_t* ring, uint32_t at, bool live, double& sx, double& sy,
                                            double& sz, double& m, double q[6]) {
    sx = 1.0e30, sy = sz = m = 0.0;
    q[0] = q[1] = q[2] = q[3] = q[4] = q[5] = 0.0;
    if (live) {
      const uint32_t n = ring[at & (kCellQ - 1)];
      const double4 cm = a.mom[n];
      sx = cm.x, sy = cm.y, sz = cm.z, m = cm.w;
      if (QUAD) {
        const double* qq = a.q64 + (size_t)n * 6;
#pragma unroll
        for (int t = 0; t < 6; ++t) q[t] = qq[t];
      }
    }
  }

  __device__ void cells(const uint32_t* ring, uint32_t head, int cnt) {
    double s0x, s0y, s0z, m0, q0[6], s1x, s1y, s1z, m1, q1[6];
    load_cell(ring, head + j, j < cnt, s0x, s0y, s0z, m0, q0);
    load_cell(ring, head + L + j, L + j < cnt, s1x, s1y, s1z, m1, q1);
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        double ax0, ay0, az0, ax1, ay1, az1;
        cell_one(k, s0x, s0y, s0z, m0, q0, ax0, ay0, az0);
        cell_one(k, s1x, s1y, s1z, m1, q1, ax1, ay1, az1);
        ax[k] += ax0 + ax1;
        ay[k] += ay0 + ay1;
        az[k] += az0 + az1;
      }
    }
  }

  __device__ __forceinline__ void part_one(int k, double sx, double sy, double sz, double m, double& rx, double& ry,
                                           double& rz) {
    const double dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
    const double r2 = dx * dx + dy * dy + dz * dz + eps2;
    double ri = rsqrt(r2);
    if (MASK) ri = r2 > 0.0 ? ri : 0.0;
    const double c = m * (ri * ri) * ri;
    rx = c * dx, ry = c * dy, rz = c * dz;
  }

  __device__ void parts(const uint32_t* ring, uint32_t head, int cnt) {
    double s0x = 1.0e30, s0y = 0, s0z = 0, m0 = 0, s1x = 1.0e30, s1y = 0, s1z = 0, m1 = 0;
    if (j < cnt) {
      const double4 p = a.pm[ring[(head + j) & (kPartQ - 1)]];
      s0x = p.x, s0y = p.y, s0z = p.z, m0 = p.w;
    }
    if (L + j < cnt) {
      const double4 p = a.pm[ring[(head + L + j) & (kPartQ - 1)]];
      s1x = p.x, s1y = p.y, s1z = p.z, m1 = p.w;
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        double ax0, ay0, az0, ax1, ay1, az1;
        part_one(k, s0x, s0y, s0z, m0, ax0, ay0, az0);
        part_one(k, s1x, s1y, s1z, m1, ax1, ay1, az1);
        ax[k] += ax0 + ax1;
        ay[k] += ay0 + ay1;
        az[k] += az0 + az1;
      }
    }
  }

  __device__ void finish() {
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        double vx = ax[k], vy = ay[k], vz = az[k];
        for (int o = L >> 1; o > 0; o >>= 1) {
          vx += __shfl_xor_sync(kFull, vx, o);
          vy += __shfl_xor_sync(kFull, vy, o);
          vz += __shfl_xor_sync(kFull, vz, o);
        }
        const int t = g + k * gp;
        if (j == (k & (L - 1)) && t < ntb) {
          acc[t][0] += vx;
          acc[t][1] += vy;
          acc[t][2] += vz;
        }
      }
    }
    __syncwarp();
  }
};

// ---------------------------------------------------------------------------
// Source queues shared by every traversal below.  Accepted cells go to a ring
// of node ids and opened leaves' particles to a ring of particle indices; a
// full ring (or the end of the walk) is evaluated as one batch.  A loop
// iteration does exactly one thing: evaluate a cell batch, evaluate a
// particle batch, enqueue up to 32 particles of the leaves opened last, or
// let the producer (a traversal step, a list scan) add sources.  The
// evaluators are reached from this one place each (their bodies would
// otherwise be inlined many times over).

struct Queues {
  uint32_t chead = 0, phead = 0;
  int ncell = 0, npart = 0;
  // particles of the leaves opened by the last producer step, still to enqueue
  uint32_t ptot = 0, pbase = 0, pinc = 0, pc = 0, pfirst = 0;
  unsigned long long ncells = 0, nparts = 0;  // sources evaluated
};

// Appends the lanes' accepted cells (one per lane where `take`).
__device__ __forceinline__ void push_cells(WarpSmem& S, Queues& q, bool take, uint32_t node, uint32_t lt) {
  const uint32_t am = __ballot_sync(kFull, take);
  if (take) S.cell[(q.chead + q.ncell + __popc(am & lt)) & (kCellQ - 1)] = node;
  q.ncell += __popc(am);
}

// Records the lanes' opened leaves (cnt particles from `first`; cnt 0 = none):
// their particles are enqueued by the next loop iterations.
__device__ __forceinline__ void open_leaves(Queues& q, uint32_t cnt, uint32_t first, int lane) {
  q.pc = cnt;
  q.pinc = warp_incl_scan_u32(cnt, lane);
  q.ptot = __shfl_sync(kFull, q.pinc, 31);
  q.pbase = 0;
  q.pfirst = first;
}

// One iteration's queue work; returns false when the producer should run
// (queues below a batch and no particles left to enqueue), true otherwise.
// `more`: the producer has more to add.
template <class E>
__device__ __forceinline__ bool drain_step(E& ev, WarpSmem& S, Queues& q, bool more, int lane) {
  const bool done = !more && q.pbase >= q.ptot;
  const int C = ev.cell_chunk(), CP = ev.part_chunk();
  if (q.ncell >= C || (done && q.ncell > 0)) {
    const int c = min(q.ncell, C);
    ev.cells(S.cell, q.chead, c);
    q.chead += c;
    q.ncell -= c;
    q.ncells += c;
    return true;
  }
  if (q.npart >= CP || (done && q.npart > 0)) {
    const int c = min(q.npart, CP);
    ev.parts(S.part, q.phead, c);
    q.phead += c;
    q.npart -= c;
    q.nparts += c;
    return true;
  }
  if (q.pbase < q.ptot) {  // enqueue up to 32 particles of the opened leaves
    const uint32_t idx = q.pbase + lane;
    uint32_t src = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const uint32_t v = __shfl_sync(kFull, q.pinc, (src + step - 1) & 31);
      if (v <= idx) src += step;
    }
    src = min(src, 31u);
    const uint32_t sf = __shfl_sync(kFull, q.pfirst, src);
    const uint32_t sinc = __shfl_sync(kFull, q.pinc, src);
    const uint32_t spc = __shfl_sync(kFull, q.pc, src);
    const uint32_t take = min(32u, q.ptot - q.pbase);
    if ((uint32_t)lane < take) S.part[(q.phead + q.npart + lane) & (kPartQ - 1)] = sf + (idx - (sinc - spc));
    q.npart += take;
    q.pbase += take;
    __syncwarp();
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Walk of one target's particle box from the root (the reference's
// per-target list): accepted -> cells, otherwise opened (leaves contribute
// their particles, interior nodes push their children).  Used for targets of
// more than kGroupMax particles (in batches of kGroupMax targets) and for the
// targets of a group whose shared walk outgrew its list.  Returns 1 if the
// stack would overflow (redo popping one node at a time, which bounds it).

template <class E>
__device__ __forceinline__ int target_walk(E& ev, const WalkArgs& a, WarpSmem& S, uint32_t root, const double lo[3],
                                           const double hi[3], double theta2, bool dfs, int lane, Queues& q) {
  const uint32_t lt = lanemask_lt();
  if (lane == 0) S.snode[0] = root;
  uint32_t top = 1;
  __syncwarp();
  q = Queues();
  // a walk pops each node at most once: more steps than nodes means a corrupt tree
  uint32_t steps = 0;
  const uint32_t max_steps = a.st->n_nodes + 2;
  for (;;) {
    if (drain_step(ev, S, q, top > 0, lane)) continue;
    if (top == 0) break;
    if (++steps > max_steps) {
      if (lane == 0) atomicOr(&a.st->status, kStWalkLimit);
      top = 0;
      continue;
    }
    const uint32_t n = dfs ? 1u : min(top, 32u);
    top -= n;
    const bool valid = (uint32_t)lane < n;
    const uint32_t node = valid ? S.snode[top + lane] : 0u;
    __syncwarp();
    bool accept = false, leaf = false;
    uint32_t first = 0, cnt = 0, info = 0;
    if (valid) {
      const WNode* w = a.w + node;
      const double4 c4 = *reinterpret_cast<const double4*>(&w->cx);  // com xyz, edge^2
      const uint4 u4 = *reinterpret_cast<const uint4*>(&w->first);   // first, count, info, mass
      first = u4.x, cnt = u4.y, info = u4.z;
      leaf = info_leaf(info);
      // mac_accept_bbox: theta^2 * near^2 > edge^2 (multipole.h:151-153)
      accept = __dmul_rn(theta2, near2(lo, hi, c4.x, c4.y, c4.z)) > c4.w;
    }
    push_cells(S, q, accept, node, lt);
    const uint32_t nch = (valid && !accept && !leaf) ? info_nchild(info) : 0u;
    const uint32_t cinc = warp_incl_scan_u32(nch, lane);
    const uint32_t ctot = __shfl_sync(kFull, cinc, 31);
    if (top + ctot > (uint32_t)kStackCap) return 1;
    for (uint32_t k = 0; k < nch; ++k) S.snode[top + cinc - nch + k] = first + k;
    top += ctot;
    open_leaves(q, (valid && !accept && leaf) ? cnt : 0u, first, lane);
    __syncwarp();
  }
  __syncwarp();
  return 0;
}

// ---------------------------------------------------------------------------
// The shared walk of a group of k <= kMaxTargets targets (particles p0 ..
// p0 + np - 1, np <= kGroupMax), in the spirit of GroupWalker::visit
// (grouped_ttg.h:204-289) taken to every level: one traversal from the root
// whose stack entries carry the mask of targets that still need the node.
// Each popped node is first tested against the group's particle box:
// accepted there (mac_accept_bbox) -> accepted by every target in the mask;
// rejected for every point of it (mac_reject_all, multipole.h:158-160) ->
// opened by every target in the mask; otherwise each target in the mask
// tests its own box, one (node, target) pair per lane.  A node taken by every
// target of the group goes to the group queues and is evaluated once against
// all np particles; one taken by some targets only goes to the warp's list as
// (node, mask) for the targets' own passes (target_pass).  Opened interior
// nodes push their children with the mask of the targets that opened them.
// Every target's list is exactly what a walk of its own box from the root
// gives (multipole.h's tests are monotone in the box).
// Returns 0, 1 (stack overflow: redo popping one node at a time) or 2 (list
// overflow: the targets walk on their own).

template <class E>
__device__ __forceinline__ int group_walk(E& ev, const WalkArgs& a, WarpSmem& S, uint32_t root, uint32_t k,
                                          double theta2, bool dfs, int lane, uint2* list, uint32_t& nlist, Queues& q) {
  const uint32_t lt = lanemask_lt();
  const uint32_t full = (1u << k) - 1u;  // k <= kMaxTargets < 32
  if (lane == 0) S.snode[0] = root, S.smask[0] = full;
  uint32_t top = 1;
  __syncwarp();
  q = Queues();
  nlist = 0;
  uint32_t steps = 0;
  const uint32_t max_steps = a.st->n_nodes + 2;
  for (;;) {
    if (drain_step(ev, S, q, top > 0, lane)) continue;
    if (top == 0) break;
    if (++steps > max_steps) {
      if (lane == 0) atomicOr(&a.st->status, kStWalkLimit);
      top = 0;
      continue;
    }
    // pop up to 32 entries, fewer when the stack is nearly full (each popped
    // node pushes at most 8)
    uint32_t n = dfs ? 1u : min(top, 32u);
    if (!dfs) n = min(n, max((kStackCap - top) / 7u, 1u));
    top -= n;
    const bool valid = (uint32_t)lane < n;
    uint32_t node = 0, mask = 0;
    if (valid) node = S.snode[top + lane], mask = S.smask[top + lane];
    __syncwarp();
    double4 c4 = make_double4(0.0, 0.0, 0.0, 0.0);
    uint4 u4 = make_uint4(0u, 0u, 0u, 0u);
    bool acc = false, rej = false;
    if (valid) {
      const WNode* w = a.w + node;
      c4 = *reinterpret_cast<const double4*>(&w->cx);
      u4 = *reinterpret_cast<const uint4*>(&w->first);
      acc = __dmul_rn(theta2, near2(S.glo, S.ghi, c4.x, c4.y, c4.z)) > c4.w;
      // one target: its box is the group's, so not accepted means opened
      if (!acc) rej = k == 1 || __dmul_rn(theta2, far2(S.glo, S.ghi, c4.x, c4.y, c4.z)) <= c4.w;
    }
    uint32_t A = acc ? mask : 0u, O = rej ? mask : 0u;
    // undecided nodes: every target in the mask tests its own box
    const bool und = valid && !acc && !rej;
    const uint32_t pcnt = und ? (uint32_t)__popc(mask) : 0u;
    const uint32_t pincl = warp_incl_scan_u32(pcnt, lane);
    const uint32_t ptotal = __shfl_sync(kFull, pincl, 31);
    if (ptotal) {
      S.accbits[lane] = 0u;
      __syncwarp();
      for (uint32_t base = 0; base < ptotal; base += 32) {
        const uint32_t j = base + (uint32_t)lane;
        // the entry holding pair j: the first lane whose inclusive count exceeds j
        uint32_t e = 0;
#pragma unroll
        for (int st = 16; st >= 1; st >>= 1) {
          const uint32_t v = __shfl_sync(kFull, pincl, (e + st - 1) & 31);
          if (v <= j) e += st;
        }
        e = min(e, 31u);
        const uint32_t einc = __shfl_sync(kFull, pincl, e), ecnt = __shfl_sync(kFull, pcnt, e);
        uint32_t em = __shfl_sync(kFull, mask, e);
        const double ex = __shfl_sync(kFull, c4.x, e), ey = __shfl_sync(kFull, c4.y, e);
        const double ez = __shfl_sync(kFull, c4.z, e), ee = __shfl_sync(kFull, c4.w, e);
        if (j < ptotal) {
          // target t: the r-th set bit of the entry's mask
          uint32_t r = j - (einc - ecnt), t = 0;
#pragma unroll
          for (int wdt = 16; wdt >= 1; wdt >>= 1) {
            const uint32_t low = (uint32_t)__popc(em & ((1u << wdt) - 1u));
            if (r >= low) r -= low, em >>= wdt, t += wdt;
          }
          if (__dmul_rn(theta2, near2(S.tlo[t], S.thi[t], ex, ey, ez)) > ee) atomicOr(&S.accbits[e], 1u << t);
        }
      }
      __syncwarp();
      if (und) A = S.accbits[lane], O = mask & ~A;
      __syncwarp();
    }
    const bool leaf = valid && info_leaf(u4.z);
    // sources every target takes: the group queues
    push_cells(S, q, A != 0u && A == full, node, lt);
    // sources some targets take: the list
    const bool cpart = A != 0u && A != full, lpart = leaf && O != 0u && O != full;
    const uint32_t runs = lpart ? (u4.y + kMaxRun - 1) / kMaxRun : 0u;
    const uint32_t nl = (cpart ? 1u : 0u) + runs;
    const uint32_t linc = warp_incl_scan_u32(nl, lane);
    const uint32_t ltot = __shfl_sync(kFull, linc, 31);
    if (nlist + ltot > kListCap) return 2;
    uint32_t at = nlist + linc - nl;
    if (cpart) list[at++] = make_uint2(node, A);
    for (uint32_t r = 0; r < runs; ++r) {
      const uint32_t c = min(kMaxRun, u4.y - r * kMaxRun);
      list[at++] = make_uint2((u4.x + r * kMaxRun) | kLeafBit, O | (c << kCountShift));
    }
    nlist += ltot;
    // opened interior nodes: children, with the targets that opened them
    const uint32_t nch = (O != 0u && !leaf) ? info_nchild(u4.z) : 0u;
    const uint32_t cinc = warp_incl_scan_u32(nch, lane);
    const uint32_t ctot = __shfl_sync(kFull, cinc, 31);
    if (top + ctot > (uint32_t)kStackCap) return 1;
    for (uint32_t c = 0; c < nch; ++c) S.snode[top + cinc - nch + c] = u4.x + c, S.smask[top + cinc - nch + c] = O;
    top += ctot;
    // leaves every target opens: their particles, for the group queues
    open_leaves(q, (leaf && O == full) ? u4.y : 0u, u4.x, lane);
    __syncwarp();
  }
  __syncwarp();
  return 0;
}

// Target `bit` of the group takes, from the list, the entries whose mask
// holds it: cells into its cell queue, leaves' particles into its particle
// queue; evaluated with the evaluator set up for its particles.  The scan
// moves a window of 32 entries at a time and skips windows without an entry
// for the target.
template <class E>
__device__ __forceinline__ void target_pass(E& ev, const WalkArgs& a, WarpSmem& S, const uint2* list, uint32_t nlist,
                                            uint32_t bit, int lane, Queues& q) {
  const uint32_t lt = lanemask_lt();
  q = Queues();
  uint32_t at = 0;
  // the window after `at` is loaded one window ahead, so that its load
  // overlaps the work on the current one
  uint2 next = (uint32_t)lane < nlist ? list[lane] : make_uint2(0u, 0u);
  for (;;) {
    if (drain_step(ev, S, q, at < nlist, lane)) continue;
    if (at >= nlist) break;
    uint2 e;
    bool hit;
    do {
      e = next;
      hit = (e.y >> bit) & 1u;
      at += 32;
      const uint32_t j = at + (uint32_t)lane;
      next = j < nlist ? list[j] : make_uint2(0u, 0u);
    } while (!__any_sync(kFull, hit) && at < nlist);
    const bool isleaf = (e.x & kLeafBit) != 0u;
    const bool chit = hit && !isleaf, lhit = hit && isleaf;
    if (__any_sync(kFull, chit)) push_cells(S, q, chit, e.x, lt);
    if (__any_sync(kFull, lhit)) open_leaves(q, lhit ? e.y >> kCountShift : 0u, e.x & ~kLeafBit, lane);
  }
  __syncwarp();
}

// Bounding box of particles [b, b + T) (BBox::add, multipole.h:121-128).
__device__ __forceinline__ void particle_box(const double4* pm, uint32_t b, uint32_t T, int lane, double lo[3],
                                             double hi[3]) {
  lo[0] = lo[1] = lo[2] = INFINITY;
  hi[0] = hi[1] = hi[2] = -INFINITY;
  for (uint32_t i = lane; i < T; i += 32) {
    const double4 q = pm[b + i];
    lo[0] = fmin(lo[0], q.x), hi[0] = fmax(hi[0], q.x);
    lo[1] = fmin(lo[1], q.y), hi[1] = fmax(hi[1], q.y);
    lo[2] = fmin(lo[2], q.z), hi[2] = fmax(hi[2], q.z);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(kFull, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(kFull, hi[d], o));
    }
  }
}

// The interaction counts of one evaluated list: quad -> cells are
// particle-cell interactions, else monopoles counted as particle-particle.
__device__ __forceinline__ void add_counts(const Queues& q, uint32_t targets, bool quad, unsigned long long& n_pp,
                                      unsigned long long& n_pc) {
  if (quad) {
    n_pc += q.ncells * (unsigned long long)targets;
    n_pp += q.nparts * (unsigned long long)targets;
  } else {
    n_pp += (q.ncells + q.nparts) * (unsigned long long)targets;
  }
}

// on_result(particle, G * acc) (grouped_ttg.h:281-283), then kick_one /
// drift_one (integrate.h:15-16), for particles p0 .. p0 + n - 1 whose FP64
// sums are in sums[0 .. n).
__device__ __forceinline__ void kick_drift(const WalkArgs& a, const SysParam& sp, const double (*sums)[3], uint32_t p0,
                                           uint32_t n, int lane) {
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t p = p0 + i;
    const double gx = __dmul_rn(sp.G, sums[i][0]), gy = __dmul_rn(sp.G, sums[i][1]), gz = __dmul_rn(sp.G, sums[i][2]);
    if (a.accel) {
      a.accel[3 * (size_t)p + 0] = gx;
      a.accel[3 * (size_t)p + 1] = gy;
      a.accel[3 * (size_t)p + 2] = gz;
    }
    Particle P = a.staged[p];
    P.vel[0] = __dadd_rn(P.vel[0], __dmul_rn(sp.kick_dt, gx));
    P.vel[1] = __dadd_rn(P.vel[1], __dmul_rn(sp.kick_dt, gy));
    P.vel[2] = __dadd_rn(P.vel[2], __dmul_rn(sp.kick_dt, gz));
    if (sp.drift_dt != 0.0) {
      P.pos[0] = __dadd_rn(P.pos[0], __dmul_rn(sp.drift_dt, P.vel[0]));
      P.pos[1] = __dadd_rn(P.pos[1], __dmul_rn(sp.drift_dt, P.vel[1]));
      P.pos[2] = __dadd_rn(P.pos[2], __dmul_rn(sp.drift_dt, P.vel[2]));
    }
    a.out[p] = P;
  }
  __syncwarp();
}

// The system holding particle p (systems lie back to back).
__device__ __forceinline__ uint32_t system_of(const WalkArgs& a, uint32_t p) {
  uint32_t lo = 0, hi = (uint32_t)a.nsys;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.sys[mid].begin <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Every target of the group [t0, t1) (particles p0 .. p0 + np) walks on its
// own from the root into S.acc (the group walk outgrew its list).
template <class E, bool QUAD>
__device__ void targets_alone(E& ev, const WalkArgs& a, WarpSmem& S, uint32_t root, double theta2, uint32_t k,
                              uint32_t p0, int lane, unsigned long long& n_pp, unsigned long long& n_pc) {
  Queues q;
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t tb = S.tbeg[i], tn = S.tcnt[i];
    ev.cx = 0.5 * (S.tlo[i][0] + S.thi[i][0]), ev.cy = 0.5 * (S.tlo[i][1] + S.thi[i][1]);
    ev.cz = 0.5 * (S.tlo[i][2] + S.thi[i][2]);
    int r = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      ev.setup(lane, tb, (int)tn, S.acc + (tb - p0));
      r = target_walk(ev, a, S, root, S.tlo[i], S.thi[i], theta2, attempt == 1, lane, q);
      if (r == 0) break;
    }
    ev.finish();
    add_counts(q, tn, QUAD, n_pp, n_pc);
  }
}

// The group of walk group gi: its targets [t0, t1), first particle, system.
struct GroupInfo {
  uint32_t t0, t1, k, p0, s;
};

__device__ __forceinline__ GroupInfo group_info(const WalkArgs& a, uint32_t gi, uint32_t ngroups, uint32_t ntargets) {
  GroupInfo g;
  g.t0 = a.groups[gi];
  g.t1 = gi + 1 < ngroups ? a.groups[gi + 1] : ntargets;
  g.k = g.t1 - g.t0;
  g.p0 = a.nbegin[a.targets[g.t0]];
  g.s = a.nsys > 1 ? system_of(a, g.p0) : 0u;
  return g;
}

// The second pass of the two-pass schedule (see k_walk): one warp per target
// of a group of more than one target, once its group's shared walk has
// finished (its list length is no longer kListPending): the group's FP64 sums
// for its particles, then its pass over the group's list (or, if the list
// overflowed, its own walk from the root), then the kick/drift.  A job waits
// only for a group whose walk a running warp has taken, so every wait ends;
// a wait is still bounded (kStSpinLimit, the job skipped).
template <class E, bool QUAD>
__device__ __forceinline__ void target_jobs(E& ev, const WalkArgs& a, WarpSmem& S, uint32_t ngroups, uint32_t ntargets,
                                            int lane, Queues& q, unsigned long long& n_pp, unsigned long long& n_pc) {
  for (;;) {
    uint32_t ti = 0;
    if (lane == 0) ti = atomicAdd(&a.st->walk_next2, 1u);
    ti = __shfl_sync(kFull, ti, 0);
    if (ti >= ntargets) break;
    // its group: the last whose first target is at or before ti
    uint32_t gi = 0, hi = ngroups;
    while (hi - gi > 1) {
      const uint32_t mid = (gi + hi) >> 1;
      if (a.groups[mid] <= ti) gi = mid;
      else hi = mid;
    }
    const GroupInfo g = group_info(a, gi, ngroups, ntargets);
    if (g.k == 1) continue;  // done whole in the first pass
    uint32_t nlist = ld_volatile(a.gnl + gi);
    for (int spins = 0; nlist == kListPending && spins < kSpinLimit; ++spins) {
      __nanosleep(128);
      nlist = ld_volatile(a.gnl + gi);
    }
    nlist = __shfl_sync(kFull, nlist, 0);  // one value for the warp
    if (nlist == kListPending) {
      if (lane == 0) atomicOr(&a.st->status, kStSpinLimit);
      continue;
    }
    __threadfence();  // the group's sums and list after its length
    const uint32_t tnode = a.targets[ti];
    const uint32_t tb = a.nbegin[tnode], tn = a.ncount[tnode];  // tn <= kGroupMax: inside a group
    const uint32_t root = a.sys[g.s].root;
    const SysParam& sp = a.prm[g.s];
    ev.set_system(sp.eps2, a.sys[g.s].hw);
    double lo[3], hi3[3];
    particle_box(a.pm, tb, tn, lane, lo, hi3);
    ev.cx = 0.5 * (lo[0] + hi3[0]), ev.cy = 0.5 * (lo[1] + hi3[1]), ev.cz = 0.5 * (lo[2] + hi3[2]);
    if (nlist == kNotShared) {
      for (uint32_t i = lane; i < tn; i += 32) S.acc[i][0] = S.acc[i][1] = S.acc[i][2] = 0.0;
      __syncwarp();
      int r = 0;
      for (int attempt = 0; attempt < 2; ++attempt) {
        ev.setup(lane, tb, (int)tn, S.acc);
        r = target_walk(ev, a, S, root, lo, hi3, sp.theta2, attempt == 1, lane, q);
        if (r == 0) break;
      }
      ev.finish();
      add_counts(q, tn, QUAD, n_pp, n_pc);
    } else {
      const double* gs = a.gsum + (size_t)gi * (kGroupMax * 3) + 3 * (size_t)(tb - g.p0);
      for (uint32_t i = lane; i < tn; i += 32) S.acc[i][0] = gs[3 * i], S.acc[i][1] = gs[3 * i + 1], S.acc[i][2] = gs[3 * i + 2];
      __syncwarp();
      if (nlist) {
        ev.setup(lane, tb, (int)tn, S.acc);
        target_pass(ev, a, S, a.wlist + (size_t)gi * kListCap, nlist, ti - g.t0, lane, q);
        ev.finish();
        add_counts(q, tn, QUAD, n_pp, n_pc);
      }
    }
    kick_drift(a, sp, S.acc, tb, tn, lane);
  }
}

// One warp per walk group (a run of targets, k_pack_groups).  A group of one
// target larger than kGroupMax particles walks in batches of kGroupMax
// targets.  Otherwise: the group's shared walk with every source all its
// targets take evaluated against all its particles, then each target's pass
// over the list of the sources only some take, each adding its part onto the
// group's FP64 sums in target order; then the kick/drift.
//
// With few groups (n_groups <= a.nslots: about as many as warps, so the
// largest group's targets would set the kernel's time) the work is cut in
// two passes instead: the warps first take the shared walks (and the groups
// of one target whole), each leaving its group's FP64 sums and list in the
// group's slot, then take every target's pass as a job of its own, each
// starting as soon as its group's walk is done (target_jobs).  Both
// schedules run the same passes and add each target's part onto the group's
// sums the same way, so the results are the same bits.
template <class E, bool QUAD>
__global__ void __launch_bounds__(kWalkThreads, 4) k_walk(WalkArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  WarpSmem& S = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  if (a.st->status & (kStNonFinite | kStNodeOverflow | kStSpinLimit)) return;  // the build failed: touch nothing
  const uint32_t ngroups = a.st->n_groups, ntargets = a.st->n_targets;
  const bool two_pass = ngroups <= a.nslots;
  const size_t wid = (size_t)blockIdx.x * kWalkWarps + warp;
  unsigned long long n_pp = 0, n_pc = 0;
  E ev(a, S.stage, lane);
  Queues q;
  for (;;) {
    uint32_t gi = 0;
    if (lane == 0) gi = atomicAdd(&a.st->walk_next, 1u);
    gi = __shfl_sync(kFull, gi, 0);
    if (gi >= ngroups) break;
    const GroupInfo g = group_info(a, gi, ngroups, ntargets);
    const uint32_t k = g.k, p0 = g.p0;
    const uint32_t root = a.sys[g.s].root;
    const SysParam& sp = a.prm[g.s];
    const double theta2 = sp.theta2;
    ev.set_system(sp.eps2, a.sys[g.s].hw);
    const uint32_t n0 = a.ncount[a.targets[g.t0]];
    if (k == 1 && n0 > (uint32_t)kGroupMax) {
      // a large target: batches of kGroupMax particles, each walking the
      // whole target's box from the root
      double lo[3], hi[3];
      particle_box(a.pm, p0, n0, lane, lo, hi);
      ev.cx = 0.5 * (lo[0] + hi[0]), ev.cy = 0.5 * (lo[1] + hi[1]), ev.cz = 0.5 * (lo[2] + hi[2]);
      for (uint32_t b0 = 0; b0 < n0; b0 += kGroupMax) {
        const uint32_t nb = min((uint32_t)kGroupMax, n0 - b0);
        for (uint32_t i = lane; i < nb; i += 32) S.acc[i][0] = S.acc[i][1] = S.acc[i][2] = 0.0;
        __syncwarp();
        int r = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
          ev.setup(lane, p0 + b0, (int)nb, S.acc);
          r = target_walk(ev, a, S, root, lo, hi, theta2, attempt == 1, lane, q);
          if (r == 0) break;
        }
        ev.finish();
        add_counts(q, nb, QUAD, n_pp, n_pc);
        kick_drift(a, sp, S.acc, p0 + b0, nb, lane);
      }
      continue;
    }
    // the targets: particle ranges and boxes (lane i: target i), the group box
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if ((uint32_t)lane < k) {
      const uint32_t tn = a.targets[g.t0 + lane];
      const uint32_t tb = a.nbegin[tn], tc = a.ncount[tn];
      for (uint32_t i = 0; i < tc; ++i) {
        const double4 p = a.pm[tb + i];
        lo[0] = fmin(lo[0], p.x), hi[0] = fmax(hi[0], p.x);
        lo[1] = fmin(lo[1], p.y), hi[1] = fmax(hi[1], p.y);
        lo[2] = fmin(lo[2], p.z), hi[2] = fmax(hi[2], p.z);
      }
      S.tbeg[lane] = tb, S.tcnt[lane] = tc;
#pragma unroll
      for (int d = 0; d < 3; ++d) S.tlo[lane][d] = lo[d], S.thi[lane][d] = hi[d];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(kFull, lo[d], o));
        hi[d] = fmax(hi[d], __shfl_xor_sync(kFull, hi[d], o));
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) S.glo[d] = lo[d], S.ghi[d] = hi[d];
    }
    __syncwarp();
    const uint32_t np = S.tbeg[k - 1] + S.tcnt[k - 1] - p0;
    for (uint32_t i = lane; i < np; i += 32) S.acc[i][0] = S.acc[i][1] = S.acc[i][2] = 0.0;
    __syncwarp();
    // the list: the warp's slot, or in the two-pass schedule the group's
    const bool split = two_pass && k > 1;
    uint2* list = a.wlist + (split ? (size_t)gi : wid) * kListCap;
    // the shared walk (redone one node at a time if the stack would overflow)
    ev.cx = 0.5 * (lo[0] + hi[0]), ev.cy = 0.5 * (lo[1] + hi[1]), ev.cz = 0.5 * (lo[2] + hi[2]);
    uint32_t nlist = 0;
    int r = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      ev.setup(lane, p0, (int)np, S.acc);
      r = group_walk(ev, a, S, root, k, theta2, attempt == 1, lane, list, nlist, q);
      if (r != 1) break;
    }
    if (r == 0) {
      ev.finish();
      add_counts(q, np, QUAD, n_pp, n_pc);
    }
    if (split) {  // the targets' passes run as jobs of their own (target_jobs)
      if (r == 0) {
        double* gs = a.gsum + (size_t)gi * (kGroupMax * 3);
        for (uint32_t i = lane; i < np; i += 32) gs[3 * i] = S.acc[i][0], gs[3 * i + 1] = S.acc[i][1], gs[3 * i + 2] = S.acc[i][2];
      }
      __threadfence();  // the sums and the list before the length
      __syncwarp();
      if (lane == 0) st_volatile(a.gnl + gi, r == 0 ? nlist : kNotShared);
      continue;
    }
    if (r == 0) {
      // each target's part from the list, in target order
      if (nlist) {
        for (uint32_t i = 0; i < k; ++i) {
          const uint32_t tb = S.tbeg[i], tn = S.tcnt[i];
          ev.cx = 0.5 * (S.tlo[i][0] + S.thi[i][0]), ev.cy = 0.5 * (S.tlo[i][1] + S.thi[i][1]);
          ev.cz = 0.5 * (S.tlo[i][2] + S.thi[i][2]);
          ev.setup(lane, tb, (int)tn, S.acc + (tb - p0));
          target_pass(ev, a, S, list, nlist, i, lane, q);
          ev.finish();
          add_counts(q, tn, QUAD, n_pp, n_pc);
        }
      }
    } else {
      // the list overflowed: nothing of the shared walk is kept (its partial
      // sums were never added); every target walks on its own
      targets_alone<E, QUAD>(ev, a, S, root, theta2, k, p0, lane, n_pp, n_pc);
    }
    kick_drift(a, sp, S.acc, p0, np, lane);
  }
  if (two_pass) target_jobs<E, QUAD>(ev, a, S, ngroups, ntargets, lane, q, n_pp, n_pc);
  if (lane == 0) {
    atomicAdd(&a.st->pp, n_pp);
    atomicAdd(&a.st->pc, n_pc);
  }
}

template <class E, bool QUAD>
static void launch_one(const WalkArgs& a, int grid, cudaStream_t s) {
  k_walk<E, QUAD><<<grid, kWalkThreads, kWalkSmem, s>>>(a);
}

void launch_walk(const WalkArgs& a, int precision, bool quad, bool mask, int grid, cudaStream_t s) {
  if (precision == 0) {
    if (quad) mask ? launch_one<SplitEval<true, true>, true>(a, grid, s) : launch_one<SplitEval<true, false>, true>(a, grid, s);
    else mask ? launch_one<SplitEval<false, true>, false>(a, grid, s) : launch_one<SplitEval<false, false>, false>(a, grid, s);
  } else {
    if (quad) mask ? launch_one<F64Eval<true, true>, true>(a, grid, s) : launch_one<F64Eval<true, false>, true>(a, grid, s);
    else mask ? launch_one<F64Eval<false, true>, false>(a, grid, s) : launch_one<F64Eval<false, false>, false>(a, grid, s);
  }
}

template <class E, bool QUAD>
static int occ() {
  cudaFuncSetAttribute(k_walk<E, QUAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWalkSmem);
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<E, QUAD>, kWalkThreads, kWalkSmem);
  return b > 0 ? b : 1;
}

static int walk_blocks_per_sm_query(int precision, bool quad, bool mask) {
  if (precision == 0) {
    if (quad) return mask ? occ<SplitEval<true, true>, true>() : occ<SplitEval<true, false>, true>();
    return mask ? occ<SplitEval<false, true>, false>() : occ<SplitEval<false, false>, false>();
  }
  if (quad) return mask ? occ<F64Eval<true, true>, true>() : occ<F64Eval<true, false>, true>();
  return mask ? occ<F64Eval<false, true>, false>() : occ<F64Eval<false, false>, false>();
}

// Cached: queried (and the kernels' shared-memory limit raised) once per
// variant, before any stream capture uses it.
int walk_blocks_per_sm(int precision, bool quad, bool mask) {
  static int cache[2][2][2] = {};
  int& v = cache[precision != 0][quad][mask];
  if (v == 0) v = walk_blocks_per_sm_query(precision, quad, mask);
  return v;
}

int walk_threads() { return kWalkThreads; }

// Device bytes of one list slot: the list, and the group's FP64 sums and
// list length for the two-pass schedule.
size_t walk_slot_bytes() { return kListCap * sizeof(uint2) + kGroupMax * 3 * sizeof(double) + sizeof(uint32_t); }

// ---------------------------------------------------------------------------
// Unfused integrate phase: kick_one / drift_one (integrate.h:15-16) with
// stored accelerations (G*a).

__global__ void k_integrate(Particle* __restrict__ p, const double* __restrict__ acc, uint32_t n, const SysDev* sys,
                            const SysParam* prm, int nsys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = (uint32_t)nsys;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (sys[mid].begin <= i) lo = mid;
      else hi = mid;
    }
    const double kd = prm[lo].kick_dt, dd = prm[lo].drift_dt;
    Particle P = p[i];
    for (int d = 0; d < 3; ++d) P.vel[d] = __dadd_rn(P.vel[d], __dmul_rn(kd, acc[3 * (size_t)i + d]));
    if (dd != 0.0)
      for (int d = 0; d < 3; ++d) P.pos[d] = __dadd_rn(P.pos[d], __dmul_rn(dd, P.vel[d]));
    p[i] = P;
  }
}

void launch_integrate(Particle* p, const double* accel, uint32_t n, const SysDev* sys, const SysParam* prm, int nsys,
                      int sms, cudaStream_t s) {
  k_integrate<<<sms * 4, 256, 0, s>>>(p, accel, n, sys, prm, nsys);
}

__global__ void k_eval_done(DevState* st) {
  if (st->status == 0u) {
    st->evals_ok += 1u;
    st->pp_total += st->pp;
    st->pc_total += st->pc;
  }
}

void launch_eval_done(DevState* st, cudaStream_t s) { k_eval_done<<<1, 1, 0, s>>>(st); }

// ---------------------------------------------------------------------------
// FP64 direct sum on sample rows (brute_force.h:15-28): every other particle
// of the system, accel_from_source with zero second moment, times G.  32
// rows per block, 8 threads per row, sources staged through shared memory.

constexpr int kDirRows = 32;
constexpr int kDirThreads = 256;

__global__ void __launch_bounds__(kDirThreads) k_direct(const double4* __restrict__ pm, uint32_t begin, uint32_t n,
                                                        const uint32_t* __restrict__ idx, uint32_t ns, double eps2,
                                                        double G, double* __restrict__ out) {
  __shared__ double4 src[kDirThreads];
  const uint32_t r = blockIdx.x * kDirRows + (threadIdx.x >> 3);
  const int sub = threadIdx.x & 7;
  const bool live = r < ns;
  const uint32_t me = live ? idx[r] : 0xffffffffu;  // index within the system
  double4 t = live ? pm[begin + me] : make_double4(0, 0, 0, 0);
  double ax = 0, ay = 0, az = 0;
  for (uint32_t base = 0; base < n; base += kDirThreads) {
    __syncthreads();
    if (base + threadIdx.x < n) src[threadIdx.x] = pm[begin + base + threadIdx.x];
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kDirThreads, n - base);
    for (uint32_t k = sub; k < cnt; k += 8) {
      if (base + k == me) continue;
      const double4 s = src[k];
      const double dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double ds2 = d2 + eps2;
      const double inv3 = 1.0 / (ds2 * sqrt(ds2));
      const double c = s.w * inv3;
      ax += c * dx;
      ay += c * dy;
      az += c * dz;
    }
  }
  for (int o = 4; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(kFull, ax, o);
    ay += __shfl_xor_sync(kFull, ay, o);
    az += __shfl_xor_sync(kFull, az, o);
  }
  if (live && sub == 0) {
    out[3 * (size_t)r + 0] = G * ax;
    out[3 * (size_t)r + 1] = G * ay;
    out[3 * (size_t)r + 2] = G * az;
  }
}

void launch_direct(const double4* pm, uint32_t begin, uint32_t n, const uint32_t* idx, uint32_t ns, double eps2,
                   double G, double* out, cudaStream_t s) {
  k_direct<<<(ns + kDirRows - 1) / kDirRows, kDirThreads, 0, s>>>(pm, begin, n, idx, ns, eps2, G, out);
}

// ---------------------------------------------------------------------------
// Energies (integrate.h:27-43): kinetic, and the unsoftened pairwise
// potential over i < j.  Per-block partial sums in out2[2 * block + {0,1}].

constexpr int kEnThreads = 256;

__global__ void __launch_bounds__(kEnThreads) k_energy(const Particle* __restrict__ p, uint32_t begin, uint32_t n,
                                                       double G, double* __restrict__ out2) {
  __shared__ double4 src[kEnThreads];
  __shared__ double red[2][kEnThreads / 32];
  double ek = 0.0, ep = 0.0;
  const uint32_t i = blockIdx.x * kEnThreads + threadIdx.x;
  double4 t = make_double4(0, 0, 0, 0);
  if (i < n) {
    const Particle& P = p[begin + i];
    t = make_double4(P.pos[0], P.pos[1], P.pos[2], P.mass);
    ek = 0.5 * P.mass * (P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]);
  }
  for (uint32_t base = blockIdx.x * kEnThreads; base < n; base += kEnThreads) {
    __syncthreads();
    if (base + threadIdx.x < n) {
      const Particle& Q = p[begin + base + threadIdx.x];
      src[threadIdx.x] = make_double4(Q.pos[0], Q.pos[1], Q.pos[2], Q.mass);
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kEnThreads, n - base);
    if (i < n) {
      for (uint32_t k = 0; k < cnt; ++k) {
        if (base + k <= i) continue;
        const double4 s = src[k];
        const double dx = t.x - s.x, dy = t.y - s.y, dz = t.z - s.z;
        ep -= G * t.w * s.w / sqrt(dx * dx + dy * dy + dz * dz);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    ek += __shfl_xor_sync(kFull, ek, o);
    ep += __shfl_xor_sync(kFull, ep, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ek;
    red[1][threadIdx.x >> 5] = ep;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < kEnThreads / 32; ++w) a += red[0][w], b += red[1][w];
    out2[2 * blockIdx.x] = a;
    out2[2 * blockIdx.x + 1] = b;
  }
}

// Returns this launch's own error (cudaLaunchKernel reports it directly, so
// an unrelated earlier error left on the thread is neither returned nor cleared).
cudaError_t launch_energy(const Particle* p, uint32_t begin, uint32_t n, double G, double* out2, int, cudaStream_t s) {
  void* args[] = {(void*)&p, (void*)&begin, (void*)&n, (void*)&G, (void*)&out2};
  return cudaLaunchKernel((const void*)k_energy, dim3((n + kEnThreads - 1) / kEnThreads), dim3(kEnThreads), args, 0, s);
}

// ---------------------------------------------------------------------------
// FP32 FMA throughput calibration: 8 independent FMA chains per thread.

__global__ void k_fma_peak(float* out, int iters, float seed) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = seed + threadIdx.x * 1e-7f + k;
  const float m = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 1234.5678f) out[blockIdx.x] = s;  // never true; keeps the chains live
}

double measure_fp32_peak(int device) {
  cudaSetDevice(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* out = nullptr;
  cudaMalloc(&out, sizeof(float) * sms * 64);
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_peak<<<blocks, threads>>>(out, 256, 1.0f);
  cudaEventRecord(e0);
  for (int r = 0; r < 5; ++r) k_fma_peak<<<blocks, threads>>>(out, iters, 1.0f + r);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 5.0 * blocks * threads * 8.0 * iters * 2.0;
  return ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
}

}  // namespace bhg
