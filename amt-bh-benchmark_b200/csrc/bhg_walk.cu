// Force walk of the B200 Barnes-Hut path: one warp per target node.
//
// What a target receives is the reference's interaction list
// (GroupWalker, grouped_ttg.h:204-289, which produces exactly the list of a
// separate walk from the root per target, :42-51): the bounding box of the
// target's particles (BBox, multipole.h:115-142) is tested against every
// visited node with mac_accept_bbox (multipole.h:151-153), strict
// theta^2 near^2 > edge^2 in FP64; leaves are tested too; accepted nodes are
// cell interactions (quadrupole, accel_from_source multipole.h:171-200, or
// monopoles in no-quad mode); everything else is opened - interior nodes
// push their children, leaves contribute their particles directly, the
// target's own leaf included (its self term is 0 with softening and masked
// at r^2 = 0 without, accumulate_list grouped_ttg.h:117-163).
//
// The traversal is warp-cooperative: each step pops up to 32 nodes (one per
// lane) from a per-warp stack, accepted cells and opened leaves' particles
// are appended to two small shared-memory queues, and every time a queue
// holds a full chunk the chunk is evaluated with one SOURCE PER LANE against
// all of the target's particles held in registers (lanes = sources, loop =
// targets), so all 32 lanes stay busy for any target size.  Up to 8 targets
// per lane (FP32) or 4 (FP64); larger targets split the warp into 2-8 lane
// groups that share each source chunk, and targets above 32 particles walk
// once per 32.
//
// Split precision: source and target positions become FP32 offsets from the
// target's bounding-box centre (the subtraction in FP64), interactions are
// FP32 FMA + rsqrtf, and every kFlushChunks chunks the per-lane FP32 partial
// sums are reduced across the lane group and added to an FP64 accumulator
// owned by one lane per target (compensated summation across list chunks).
// The kick/drift of integrate_ttg.h:74-77 is applied in FP64 in the epilogue.
#include "bhg_kernels.h"

namespace bhg {

constexpr int kWalkWarps = 4;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kQueue = 64;
constexpr int kFlushChunks = 16;
constexpr float kFarAway = 1.0e10f;  // padding source: contributes exactly 0
constexpr uint32_t kFull = 0xffffffffu;

struct WarpQueues {
  uint32_t cell[kQueue];
  uint32_t part[kQueue];
};

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Squared distance from (x, y, z) to the nearest point of the box, exactly as
// BBox::near2 (multipole.h:132-136) rounds it.
__device__ __forceinline__ double near2(const double lo[3], const double hi[3], double x, double y, double z) {
  double dx = fmax(fmax(__dsub_rn(lo[0], x), __dsub_rn(x, hi[0])), 0.0);
  double dy = fmax(fmax(__dsub_rn(lo[1], y), __dsub_rn(y, hi[1])), 0.0);
  double dz = fmax(fmax(__dsub_rn(lo[2], z), __dsub_rn(z, hi[2])), 0.0);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// ---------------------------------------------------------------------------
// Evaluators: what a lane does with one chunk of sources.

// Split precision, up to 8 targets per lane.
template <bool QUAD, bool MASK>
struct SplitEval {
  static constexpr int TB = 8;
  const WalkArgs& a;
  double cx, cy, cz;  // reference point (target bbox centre)
  float eps2;
  int L, g, j, kmax;  // lanes per group, my group, my index in it, live target slots
  float tx[TB], ty[TB], tz[TB];
  float ax[TB], ay[TB], az[TB];
  double ox64 = 0.0, oy64 = 0.0, oz64 = 0.0;  // FP64 sum of the target this lane owns
  int chunks = 0;

  __device__ SplitEval(const WalkArgs& args) : a(args) {}

  static __device__ int groups_for(int tb) { return tb <= 8 ? 1 : tb <= 16 ? 2 : 4; }

  __device__ void setup(int lane, uint32_t p0, int tb) {
    const int gp = groups_for(tb);
    L = 32 / gp;
    g = lane / L;
    j = lane & (L - 1);
    kmax = (tb + gp - 1) / gp;
    float px = 0.f, py = 0.f, pz = 0.f;
    if (lane < tb) {
      const double4 q = a.pm[p0 + lane];
      px = (float)__dsub_rn(q.x, cx);
      py = (float)__dsub_rn(q.y, cy);
      pz = (float)__dsub_rn(q.z, cz);
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int src = (g + k * gp) & 31;
      tx[k] = __shfl_sync(kFull, px, src);
      ty[k] = __shfl_sync(kFull, py, src);
      tz[k] = __shfl_sync(kFull, pz, src);
      ax[k] = ay[k] = az[k] = 0.f;
    }
    ox64 = oy64 = oz64 = 0.0;
    chunks = 0;
  }

  __device__ void flush() {
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        float vx = ax[k], vy = ay[k], vz = az[k];
        for (int o = L >> 1; o > 0; o >>= 1) {
          vx += __shfl_xor_sync(kFull, vx, o);
          vy += __shfl_xor_sync(kFull, vy, o);
          vz += __shfl_xor_sync(kFull, vz, o);
        }
        if (j == k) {
          ox64 += (double)vx;
          oy64 += (double)vy;
          oz64 += (double)vz;
        }
        ax[k] = ay[k] = az[k] = 0.f;
      }
    }
    chunks = 0;
  }

  __device__ void tick() {
    if (++chunks == kFlushChunks) flush();
  }

  // accepted cells: node ids ring[(head + i) % kQueue], i < cnt
  __device__ void cells(const uint32_t* ring, uint32_t head, int cnt) {
    float sx = kFarAway, sy = 0.f, sz = 0.f, m = 0.f;
    float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f, q4 = 0.f, q5 = 0.f;
    if (j < cnt) {
      const uint32_t n = ring[(head + j) & (kQueue - 1)];
      const WNode* w = a.w + n;
      const double2 cxy = *reinterpret_cast<const double2*>(&w->cx);
      const double czz = w->cz;
      sx = (float)__dsub_rn(cxy.x, cx);
      sy = (float)__dsub_rn(cxy.y, cy);
      sz = (float)__dsub_rn(czz, cz);
      m = w->mass;
      if (QUAD) {
        const float4 qa = *reinterpret_cast<const float4*>(w->q);
        const float2 qb = a.q45[n];
        q0 = qa.x, q1 = qa.y, q2 = qa.z, q3 = qa.w, q4 = qb.x, q5 = qb.y;
      }
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        const float dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float ri = rsqrtf(r2);
        if (!QUAD && MASK) ri = r2 > 0.f ? ri : 0.f;
        const float ri2 = ri * ri;
        const float ri3 = ri * ri2;
        if (QUAD) {
          const float qx = fmaf(q0, dx, fmaf(q3, dy, q4 * dz));
          const float qy = fmaf(q3, dx, fmaf(q1, dy, q5 * dz));
          const float qz = fmaf(q4, dx, fmaf(q5, dy, q2 * dz));
          const float dqd = fmaf(dx, qx, fmaf(dy, qy, dz * qz));
          const float ri5 = ri3 * ri2;
          // m d / r^3 - Q d / r^5 + 2.5 (d Q d) d / r^7
          const float c = fmaf(2.5f * dqd, ri5 * ri2, m * ri3);
          ax[k] = fmaf(c, dx, fmaf(-ri5, qx, ax[k]));
          ay[k] = fmaf(c, dy, fmaf(-ri5, qy, ay[k]));
          az[k] = fmaf(c, dz, fmaf(-ri5, qz, az[k]));
        } else {
          const float c = m * ri3;
          ax[k] = fmaf(c, dx, ax[k]);
          ay[k] = fmaf(c, dy, ay[k]);
          az[k] = fmaf(c, dz, az[k]);
        }
      }
    }
    tick();
  }

  // direct particles: particle indices ring[(head + i) % kQueue], i < cnt
  __device__ void parts(const uint32_t* ring, uint32_t head, int cnt) {
    float sx = kFarAway, sy = 0.f, sz = 0.f, m = 0.f;
    if (j < cnt) {
      const double4 p = a.pm[ring[(head + j) & (kQueue - 1)]];
      sx = (float)__dsub_rn(p.x, cx);
      sy = (float)__dsub_rn(p.y, cy);
      sz = (float)__dsub_rn(p.z, cz);
      m = (float)p.w;
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        const float dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float ri = rsqrtf(r2);
        if (MASK) ri = r2 > 0.f ? ri : 0.f;
        const float c = m * (ri * ri) * ri;
        ax[k] = fmaf(c, dx, ax[k]);
        ay[k] = fmaf(c, dy, ay[k]);
        az[k] = fmaf(c, dz, az[k]);
      }
    }
    tick();
  }

  // After the walk: the owner lane of target slot j gets its FP64 sum.
  __device__ void finish(double& rx, double& ry, double& rz) {
    flush();
    rx = ox64;
    ry = oy64;
    rz = oz64;
  }
};

// Plain FP64, up to 4 targets per lane.  Absolute FP64 positions, the same
// formula as accel_from_source with multiplications by 1/r^2 for its
// divisions.
template <bool QUAD, bool MASK>
struct F64Eval {
  static constexpr int TB = 4;
  const WalkArgs& a;
  double cx, cy, cz;  // unused (absolute positions)
  double eps2;
  int L, g, j, kmax;
  double tx[TB], ty[TB], tz[TB];
  double ax[TB], ay[TB], az[TB];

  __device__ F64Eval(const WalkArgs& args) : a(args) {}

  static __device__ int groups_for(int tb) { return tb <= 4 ? 1 : tb <= 8 ? 2 : tb <= 16 ? 4 : 8; }

  __device__ void setup(int lane, uint32_t p0, int tb) {
    const int gp = groups_for(tb);
    L = 32 / gp;
    g = lane / L;
    j = lane & (L - 1);
    kmax = (tb + gp - 1) / gp;
    double px = 0.0, py = 0.0, pz = 0.0;
    if (lane < tb) {
      const double4 q = a.pm[p0 + lane];
      px = q.x, py = q.y, pz = q.z;
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int src = (g + k * gp) & 31;
      tx[k] = __shfl_sync(kFull, px, src);
      ty[k] = __shfl_sync(kFull, py, src);
      tz[k] = __shfl_sync(kFull, pz, src);
      ax[k] = ay[k] = az[k] = 0.0;
    }
  }

  __device__ void cells(const uint32_t* ring, uint32_t head, int cnt) {
    double sx = 1.0e30, sy = 0.0, sz = 0.0, m = 0.0;
    double q0 = 0, q1 = 0, q2 = 0, q3 = 0, q4 = 0, q5 = 0;
    if (j < cnt) {
      const uint32_t n = ring[(head + j) & (kQueue - 1)];
      const double4 cm = a.mom[n];
      sx = cm.x, sy = cm.y, sz = cm.z, m = cm.w;
      if (QUAD) {
        const double* qq = a.q64 + (size_t)n * 6;
        q0 = qq[0], q1 = qq[1], q2 = qq[2], q3 = qq[3], q4 = qq[4], q5 = qq[5];
      }
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        const double dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
        const double r2 = dx * dx + dy * dy + dz * dz + eps2;
        double ri = rsqrt(r2);
        if (!QUAD && MASK) ri = r2 > 0.0 ? ri : 0.0;
        const double ri2 = ri * ri;
        const double ri3 = ri * ri2;
        if (QUAD) {
          const double qx = q0 * dx + q3 * dy + q4 * dz;
          const double qy = q3 * dx + q1 * dy + q5 * dz;
          const double qz = q4 * dx + q5 * dy + q2 * dz;
          const double dqd = dx * qx + dy * qy + dz * qz;
          const double ri5 = ri3 * ri2;
          const double c = m * ri3 + 2.5 * dqd * (ri5 * ri2);
          ax[k] += c * dx - ri5 * qx;
          ay[k] += c * dy - ri5 * qy;
          az[k] += c * dz - ri5 * qz;
        } else {
          const double c = m * ri3;
          ax[k] += c * dx;
          ay[k] += c * dy;
          az[k] += c * dz;
        }
      }
    }
  }

  __device__ void parts(const uint32_t* ring, uint32_t head, int cnt) {
    double sx = 1.0e30, sy = 0.0, sz = 0.0, m = 0.0;
    if (j < cnt) {
      const double4 p = a.pm[ring[(head + j) & (kQueue - 1)]];
      sx = p.x, sy = p.y, sz = p.z, m = p.w;
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        const double dx = sx - tx[k], dy = sy - ty[k], dz = sz - tz[k];
        const double r2 = dx * dx + dy * dy + dz * dz + eps2;
        double ri = rsqrt(r2);
        if (MASK) ri = r2 > 0.0 ? ri : 0.0;
        const double c = m * (ri * ri) * ri;
        ax[k] += c * dx;
        ay[k] += c * dy;
        az[k] += c * dz;
      }
    }
  }

  __device__ void finish(double& rx, double& ry, double& rz) {
    rx = ry = rz = 0.0;
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      if (k < kmax) {
        double vx = ax[k], vy = ay[k], vz = az[k];
        for (int o = L >> 1; o > 0; o >>= 1) {
          vx += __shfl_xor_sync(kFull, vx, o);
          vy += __shfl_xor_sync(kFull, vy, o);
          vz += __shfl_xor_sync(kFull, vz, o);
        }
        if (j == k) rx = vx, ry = vy, rz = vz;
      }
    }
  }
};


// ---------------------------------------------------------------------------
// The traversal of one target (one batch of at most 32 of its particles).
// Returns true if the stack would overflow (the caller redoes the batch
// popping one node at a time, which bounds the stack by 7 * depth + 1).

template <class E>
__device__ __forceinline__ bool walk_target(E& ev, const WalkArgs& a, WarpQueues& Q, uint32_t* stack, uint32_t root,
                                            const double lo[3], const double hi[3], double theta2, bool dfs, int lane,
                                            unsigned long long& ncells, unsigned long long& nparts) {
  const int L = ev.L;
  const uint32_t lt = lanemask_lt();
  uint32_t top = 1;
  if (lane == 0) stack[0] = root;
  __syncwarp();
  uint32_t chead = 0, phead = 0;
  int ncell = 0, npart = 0;
  ncells = nparts = 0;
  while (top > 0) {
    const uint32_t n = dfs ? 1u : min(top, 32u);
    top -= n;
    const bool valid = (uint32_t)lane < n;
    const uint32_t node = valid ? stack[top + lane] : 0u;
    __syncwarp();
    bool accept = false, leaf = false;
    uint32_t first = 0, cnt = 0, info = 0;
    if (valid) {
      const WNode* w = a.w + node;
      const double4 c4 = *reinterpret_cast<const double4*>(&w->cx);  // com xyz, edge^2
      const uint4 u4 = *reinterpret_cast<const uint4*>(&w->first);   // first, count, info, mass
      first = u4.x;
      cnt = u4.y;
      info = u4.z;
      // mac_accept_bbox: theta^2 * near^2 > edge^2 (multipole.h:151-153)
      accept = __dmul_rn(theta2, near2(lo, hi, c4.x, c4.y, c4.z)) > c4.w;
      leaf = info_leaf(info);
    }
    // accepted: cell queue
    const uint32_t am = __ballot_sync(kFull, accept);
    if (accept) Q.cell[(chead + ncell + __popc(am & lt)) & (kQueue - 1)] = node;
    ncell += __popc(am);
    // opened interior nodes: push the children
    const uint32_t nch = (valid && !accept && !leaf) ? info_nchild(info) : 0u;
    const uint32_t cinc = warp_incl_scan_u32(nch, lane);
    const uint32_t ctot = __shfl_sync(kFull, cinc, 31);
    if (top + ctot > a.stack_cap) return true;
    for (uint32_t k = 0; k < nch; ++k) stack[top + cinc - nch + k] = first + k;
    top += ctot;
    // opened leaves: their particles
    const uint32_t pc = (valid && !accept && leaf) ? cnt : 0u;
    const uint32_t pinc = warp_incl_scan_u32(pc, lane);
    const uint32_t ptot = __shfl_sync(kFull, pinc, 31);
    __syncwarp();
    while (ncell >= L) {
      ev.cells(Q.cell, chead, L);
      chead += L;
      ncell -= L;
      ncells += L;
    }
    for (uint32_t base = 0; base < ptot; base += 32) {
      const uint32_t idx = base + lane;
      uint32_t src = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t v = __shfl_sync(kFull, pinc, (src + step - 1) & 31);
        if (v <= idx) src += step;
      }
      src = min(src, 31u);
      const uint32_t sf = __shfl_sync(kFull, first, src);
      const uint32_t sinc = __shfl_sync(kFull, pinc, src);
      const uint32_t spc = __shfl_sync(kFull, pc, src);
      const uint32_t take = min(32u, ptot - base);
      if ((uint32_t)lane < take) Q.part[(phead + npart + lane) & (kQueue - 1)] = sf + (idx - (sinc - spc));
      npart += take;
      __syncwarp();
      while (npart >= L) {
        ev.parts(Q.part, phead, L);
        phead += L;
        npart -= L;
        nparts += L;
      }
    }
    __syncwarp();
  }
  if (ncell > 0) {
    ev.cells(Q.cell, chead, ncell);
    ncells += ncell;
  }
  if (npart > 0) {
    ev.parts(Q.part, phead, npart);
    nparts += npart;
  }
  __syncwarp();
  return false;
}

template <class E, bool QUAD>
__global__ void __launch_bounds__(kWalkThreads, 4) k_walk(WalkArgs a) {
  __shared__ WarpQueues sq[kWalkWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  WarpQueues& Q = sq[warp];
  uint32_t* stack = a.stack + (size_t)(blockIdx.x * kWalkWarps + warp) * a.stack_cap;
  if (a.st->status & (kStNonFinite | kStNodeOverflow | kStSpinLimit)) return;  // the build failed: touch nothing
  const uint32_t ntg = a.st->n_targets;
  unsigned long long n_pp = 0, n_pc = 0;
  E ev(a);
  for (;;) {
    uint32_t ti = 0;
    if (lane == 0) ti = atomicAdd(&a.st->walk_next, 1u);
    ti = __shfl_sync(kFull, ti, 0);
    if (ti >= ntg) break;
    const uint32_t tnode = a.targets[ti];
    const uint32_t tb = a.nbegin[tnode], T = a.ncount[tnode];
    uint32_t s = 0;
    if (a.nsys > 1) {  // the system holding particle tb
      uint32_t lo = 0, hi = (uint32_t)a.nsys;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.sys[mid].begin <= tb) lo = mid;
        else hi = mid;
      }
      s = lo;
    }
    const SysDev& sd = a.sys[s];
    const SysParam& sp = a.prm[s];
    // BBox of the target's particles (multipole.h:115-129)
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = lane; i < T; i += 32) {
      const double4 q = a.pm[tb + i];
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
    ev.cx = 0.5 * (lo[0] + hi[0]);
    ev.cy = 0.5 * (lo[1] + hi[1]);
    ev.cz = 0.5 * (lo[2] + hi[2]);
    ev.eps2 = sp.eps2;
    const double theta2 = sp.theta2, G = sp.G, kick = sp.kick_dt, drift = sp.drift_dt;
    for (uint32_t b0 = 0; b0 < T; b0 += 32) {
      const int tbn = (int)min(32u, T - b0);
      unsigned long long nc = 0, np = 0;
      for (int attempt = 0; attempt < 2; ++attempt) {
        ev.setup(lane, tb + b0, tbn);
        if (!walk_target(ev, a, Q, stack, sd.root, lo, hi, theta2, attempt == 1, lane, nc, np)) break;
      }
      double rx, ry, rz;
      ev.finish(rx, ry, rz);
      if (QUAD) {
        n_pc += nc * (unsigned long long)tbn;
        n_pp += np * (unsigned long long)tbn;
      } else {
        n_pp += (nc + np) * (unsigned long long)tbn;
      }
      const int gp = 32 / ev.L;
      const int tl = ev.g + ev.j * gp;
      if (ev.j < ev.kmax && tl < tbn) {
        const uint32_t p = tb + b0 + (uint32_t)tl;
        // on_result(particle, G * acc) (grouped_ttg.h:281-283), then
        // kick_one / drift_one (integrate.h:15-16)
        const double gx = __dmul_rn(G, rx), gy = __dmul_rn(G, ry), gz = __dmul_rn(G, rz);
        if (a.accel) {
          a.accel[3 * (size_t)p + 0] = gx;
          a.accel[3 * (size_t)p + 1] = gy;
          a.accel[3 * (size_t)p + 2] = gz;
        }
        Particle P = a.staged[p];
        P.vel[0] = __dadd_rn(P.vel[0], __dmul_rn(kick, gx));
        P.vel[1] = __dadd_rn(P.vel[1], __dmul_rn(kick, gy));
        P.vel[2] = __dadd_rn(P.vel[2], __dmul_rn(kick, gz));
        if (drift != 0.0) {
          P.pos[0] = __dadd_rn(P.pos[0], __dmul_rn(drift, P.vel[0]));
          P.pos[1] = __dadd_rn(P.pos[1], __dmul_rn(drift, P.vel[1]));
          P.pos[2] = __dadd_rn(P.pos[2], __dmul_rn(drift, P.vel[2]));
        }
        a.out[p] = P;
      }
    }
  }
  if (lane == 0) {
    atomicAdd(&a.st->pp, n_pp);
    atomicAdd(&a.st->pc, n_pc);
  }
}

template <class E, bool QUAD>
static void launch_one(const WalkArgs& a, int grid, cudaStream_t s) {
  k_walk<E, QUAD><<<grid, kWalkThreads, 0, s>>>(a);
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
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<E, QUAD>, kWalkThreads, 0);
  return b > 0 ? b : 1;
}

int walk_blocks_per_sm(int precision, bool quad, bool mask) {
  if (precision == 0) {
    if (quad) return mask ? occ<SplitEval<true, true>, true>() : occ<SplitEval<true, false>, true>();
    return mask ? occ<SplitEval<false, true>, false>() : occ<SplitEval<false, false>, false>();
  }
  if (quad) return mask ? occ<F64Eval<true, true>, true>() : occ<F64Eval<true, false>, true>();
  return mask ? occ<F64Eval<false, true>, false>() : occ<F64Eval<false, false>, false>();
}

int walk_threads() { return kWalkThreads; }

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
  if (st->status == 0u) st->evals_ok += 1u;
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

void launch_energy(const Particle* p, uint32_t begin, uint32_t n, double G, double* out2, int, cudaStream_t s) {
  k_energy<<<(n + kEnThreads - 1) / kEnThreads, kEnThreads, 0, s>>>(p, begin, n, G, out2);
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
