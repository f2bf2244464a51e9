// Particle text on the device: CSV ingest (read_csv, io.cc:122-178) and the
// VTK snapshot (write_vtk, io.cc:180-195).
//
// Ingest: the text is copied to the device once; line starts come from a
// newline count per 16 KB tile, a scan of the tile counts and an ordered
// emit of the newline positions; then one thread per line parses it as
// io.cc's parse_lines/parse_field do (blanks around fields, ',' between the
// eight fields id,mass,x,y,z,vx,vy,vz, an optional '\r' at the end; a line
// of blanks is skipped; anything else is a malformed line), with the exact
// number conversion of bhg_decimal.cuh; valid lines are compacted in order.
// The header rule of read_csv (skip the first line if its first field is
// not an id) is applied by the host, which sees the first line anyway.
//
// Snapshot: one thread per particle formats its three lines ("x y z",
// "mass", "vx vy vz", numbers as an ostream writes them) into fixed-size
// slots; a scan of the slot lengths places them in the output.
#include "bhg_kernels.h"
#include "bhg_decimal.cuh"

namespace bhg {

namespace {

constexpr int kTileBytes = 16384;
constexpr int kCsvThreads = 256;  // per block; each thread scans 64 bytes of a tile
static_assert(kTileBytes == kCsvThreads * 64, "tile = threads x 64 bytes");

__device__ __forceinline__ uint32_t count_byte(uint32_t w, uint32_t c4) {
  // bytes of w equal to the byte replicated in c4 (exact, no false positives)
  const uint32_t x = w ^ c4;
  const uint32_t t = ((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x;
  return __popc(~t & 0x80808080u);
}

// newlines in [i0, i1) of the text (byte loop at the ends, words inside)
__device__ uint32_t count_nl(const char* text, size_t i0, size_t i1) {
  uint32_t c = 0;
  size_t i = i0;
  for (; i < i1 && (i & 3); ++i) c += text[i] == '\n';
  for (; i + 4 <= i1; i += 4) c += count_byte(*reinterpret_cast<const uint32_t*>(text + i), 0x0a0a0a0au);
  for (; i < i1; ++i) c += text[i] == '\n';
  return c;
}

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t s = lane < nw ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += u;
    }
    if (lane < nw) sh[lane] = s;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  const uint32_t base = warp ? sh[warp - 1] : 0u;
  __syncthreads();
  return base + incl - v;
}

}  // namespace

__global__ void __launch_bounds__(kCsvThreads) k_nl_count(const char* __restrict__ text, size_t n,
                                                          uint32_t* __restrict__ tile_count) {
  __shared__ uint32_t sh[32];
  const size_t t0 = (size_t)blockIdx.x * kTileBytes + (size_t)threadIdx.x * 64;
  const uint32_t c = t0 < n ? count_nl(text, t0, t0 + 64 < n ? t0 + 64 : n) : 0u;
  uint32_t total;
  block_excl_scan(c, sh, total);
  if (threadIdx.x == 0) tile_count[blockIdx.x] = total;
}

// Exclusive scan of counts[0 .. m) in place (one block); total to *total.
__global__ void __launch_bounds__(1024) k_scan_counts(uint32_t* __restrict__ counts, uint32_t m,
                                                      uint64_t* __restrict__ total) {
  __shared__ uint32_t sh[32];
  uint64_t carry = 0;
  for (uint32_t base = 0; base < m; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < m ? counts[i] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, sh, tot);
    if (i < m) counts[i] = (uint32_t)(carry + ex);
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

// line_start[0] = 0; line_start[k + 1] = 1 + position of newline k.
__global__ void __launch_bounds__(kCsvThreads) k_nl_emit(const char* __restrict__ text, size_t n,
                                                         const uint32_t* __restrict__ tile_off,
                                                         uint64_t* __restrict__ line_start) {
  __shared__ uint32_t sh[32];
  const size_t t0 = (size_t)blockIdx.x * kTileBytes + (size_t)threadIdx.x * 64;
  const size_t t1 = t0 + 64 < n ? t0 + 64 : n;
  const uint32_t c = t0 < n ? count_nl(text, t0, t1) : 0u;
  uint32_t total;
  uint64_t k = (uint64_t)tile_off[blockIdx.x] + block_excl_scan(c, sh, total);
  if (blockIdx.x == 0 && threadIdx.x == 0) line_start[0] = 0;
  for (size_t i = t0; i < t1 && c; ++i)
    if (text[i] == '\n') line_start[1 + k++] = i + 1;
}

namespace {

__device__ __forceinline__ const char* skip_blanks(const char* p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\t')) ++p;
  return p;
}

// parse_field (io.cc:76-91) for the id: std::from_chars into uint32
__device__ bool field_id(const char*& p, const char* end, uint32_t& out) {
  p = skip_blanks(p, end);
  const char* q = p;
  uint64_t v = 0;
  while (q < end && *q >= '0' && *q <= '9') {
    v = v * 10 + (uint64_t)(*q - '0');
    if (v > 0xffffffffull) return false;  // result_out_of_range
    ++q;
  }
  if (q == p) return false;
  out = (uint32_t)v;
  q = skip_blanks(q, end);
  if (q >= end || *q != ',') return false;
  p = q + 1;
  return true;
}

// parse_field for a double (one out-of-line copy: the conversion is large,
// and seven inlined copies would not stay in the instruction cache)
__device__ __noinline__ bool field_f64(const char*& p, const char* end, double& out, bool last, dec::Big& w, dec::Big& b) {
  p = skip_blanks(p, end);
  const char* q;
  if (dec::parse_double(p, end, &out, &q, w, b) != dec::kOk) return false;
  q = skip_blanks(q, end);
  if (last) {
    if (q < end && *q == '\r') ++q;
    if (q != end) return false;
  } else {
    if (q >= end || *q != ',') return false;
    ++q;
  }
  p = q;
  return true;
}

}  // namespace

// One thread per line: lines [first, nlines).  keep[i - first] = 1 for a
// particle line, 0 for a blank one; *bad = the smallest malformed line.
__global__ void __launch_bounds__(128) k_csv_parse(const char* __restrict__ text, size_t n,
                                                   const uint64_t* __restrict__ line_start, uint64_t first,
                                                   uint64_t nlines, Particle* __restrict__ out,
                                                   uint32_t* __restrict__ keep, unsigned long long* __restrict__ bad) {
  dec::Big w, b;
  for (uint64_t i = first + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlines;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const char* line = text + line_start[i];
    const char* eol = i + 1 < nlines ? text + line_start[i + 1] - 1 : text + n;
    const char* p = skip_blanks(line, eol);
    uint32_t k = 0;
    if (p != eol && *p != '\r') {
      Particle q;
      q.pad = 0;
      if (field_id(p, eol, q.id) && field_f64(p, eol, q.mass, false, w, b) && field_f64(p, eol, q.pos[0], false, w, b) &&
          field_f64(p, eol, q.pos[1], false, w, b) && field_f64(p, eol, q.pos[2], false, w, b) &&
          field_f64(p, eol, q.vel[0], false, w, b) && field_f64(p, eol, q.vel[1], false, w, b) &&
          field_f64(p, eol, q.vel[2], true, w, b)) {
        out[i - first] = q;
        k = 1;
      } else {
        atomicMin(bad, (unsigned long long)i);
      }
    }
    keep[i - first] = k;
  }
}

// Per-block sums of keep[] (blocks of kCsvThreads entries).
__global__ void __launch_bounds__(kCsvThreads) k_keep_count(const uint32_t* __restrict__ keep, uint64_t m,
                                                            uint32_t* __restrict__ block_count) {
  const uint64_t i = (uint64_t)blockIdx.x * kCsvThreads + threadIdx.x;
  const int c = __syncthreads_count(i < m && keep[i]);
  if (threadIdx.x == 0) block_count[blockIdx.x] = (uint32_t)c;
}

// Kept particles, in order, to dst.
__global__ void __launch_bounds__(kCsvThreads) k_keep_scatter(const Particle* __restrict__ src,
                                                              const uint32_t* __restrict__ keep, uint64_t m,
                                                              const uint32_t* __restrict__ block_off,
                                                              Particle* __restrict__ dst) {
  __shared__ uint32_t sh[32];
  const uint64_t i = (uint64_t)blockIdx.x * kCsvThreads + threadIdx.x;
  const uint32_t k = i < m ? keep[i] : 0u;
  uint32_t total;
  const uint32_t ex = block_excl_scan(k, sh, total);
  if (k) dst[(uint64_t)block_off[blockIdx.x] + ex] = src[i];
}

// ---- snapshot ------------------------------------------------------------------

namespace {
constexpr int kPosSlot = 48, kMassSlot = 16;  // "x y z\n" <= 3 * 13 + 3, "m\n" <= 14
}

// Slots: particle i's position line at pos_text + i * kPosSlot, mass line at
// mass_text + i * kMassSlot, velocity line at vel_text + i * kPosSlot; the
// three lengths into len[i], len[n + i], len[2n + i].
__global__ void __launch_bounds__(128) k_vtk_format(const Particle* __restrict__ p, uint32_t n,
                                                    char* __restrict__ pos_text, char* __restrict__ mass_text,
                                                    char* __restrict__ vel_text, uint32_t* __restrict__ len) {
  dec::Big a, b;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Particle q = p[i];
    char* o = pos_text + (size_t)i * kPosSlot;
    int l = 0;
    for (int d = 0; d < 3; ++d) {
      l += dec::format_g6(q.pos[d], o + l, a, b);
      o[l++] = d < 2 ? ' ' : '\n';
    }
    len[i] = (uint32_t)l;
    o = mass_text + (size_t)i * kMassSlot;
    l = dec::format_g6(q.mass, o, a, b);
    o[l++] = '\n';
    len[n + i] = (uint32_t)l;
    o = vel_text + (size_t)i * kPosSlot;
    l = 0;
    for (int d = 0; d < 3; ++d) {
      l += dec::format_g6(q.vel[d], o + l, a, b);
      o[l++] = d < 2 ? ' ' : '\n';
    }
    len[2 * (size_t)n + i] = (uint32_t)l;
  }
}

// Per-block sums of 32-bit lengths (blocks of kCsvThreads entries).
__global__ void __launch_bounds__(kCsvThreads) k_len_sums(const uint32_t* __restrict__ len, uint64_t m,
                                                          uint32_t* __restrict__ block_sum) {
  __shared__ uint32_t sh[32];
  const uint64_t i = (uint64_t)blockIdx.x * kCsvThreads + threadIdx.x;
  uint32_t total;
  block_excl_scan(i < m ? len[i] : 0u, sh, total);
  if (threadIdx.x == 0) block_sum[blockIdx.x] = total;
}

// Exclusive scan of block sums into 64-bit block offsets (one block); total
// to *total.
__global__ void __launch_bounds__(1024) k_scan_sums64(const uint32_t* __restrict__ sums, uint32_t m,
                                                      uint64_t* __restrict__ off, uint64_t* __restrict__ total) {
  __shared__ uint32_t sh[32];
  uint64_t carry = 0;
  for (uint32_t base = 0; base < m; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < m ? sums[i] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, sh, tot);
    if (i < m) off[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

// Copies slot i (slot size `slot`, length len[i]) to out at its place: the
// block's offset plus the lengths before it in the block.
__global__ void __launch_bounds__(kCsvThreads) k_vtk_gather(const char* __restrict__ slots, int slot,
                                                            const uint32_t* __restrict__ len,
                                                            const uint64_t* __restrict__ block_off, uint64_t m,
                                                            char* __restrict__ out) {
  __shared__ uint32_t sh[32];
  const uint64_t i = (uint64_t)blockIdx.x * kCsvThreads + threadIdx.x;
  const uint32_t l = i < m ? len[i] : 0u;
  uint32_t total;
  const uint64_t at = block_off[blockIdx.x] + block_excl_scan(l, sh, total);
  const char* src = slots + i * slot;
  for (uint32_t c = 0; c < l; ++c) out[at + c] = src[c];
}

// ---- launchers -----------------------------------------------------------------

size_t csv_tiles(size_t nbytes) { return (nbytes + kTileBytes - 1) / kTileBytes; }

void launch_csv_count(const char* text, size_t n, uint32_t* tile_count, uint64_t* total, cudaStream_t s) {
  const size_t tiles = csv_tiles(n);
  if (tiles == 0) return;
  k_nl_count<<<(unsigned)tiles, kCsvThreads, 0, s>>>(text, n, tile_count);
  k_scan_counts<<<1, 1024, 0, s>>>(tile_count, (uint32_t)tiles, total);
}

void launch_csv_emit(const char* text, size_t n, const uint32_t* tile_off, uint64_t* line_start, cudaStream_t s) {
  const size_t tiles = csv_tiles(n);
  if (tiles == 0) return;
  k_nl_emit<<<(unsigned)tiles, kCsvThreads, 0, s>>>(text, n, tile_off, line_start);
}

void launch_csv_parse(const char* text, size_t n, const uint64_t* line_start, uint64_t first, uint64_t nlines,
                      Particle* tmp, uint32_t* keep, unsigned long long* bad, int sms, cudaStream_t s) {
  const uint64_t m = nlines > first ? nlines - first : 0;
  if (m == 0) return;
  uint64_t blocks = (m + 127) / 128;
  if (blocks > (uint64_t)sms * 16) blocks = (uint64_t)sms * 16;
  k_csv_parse<<<(unsigned)blocks, 128, 0, s>>>(text, n, line_start, first, nlines, tmp, keep, bad);
}

size_t csv_keep_blocks(uint64_t m) { return (size_t)((m + kCsvThreads - 1) / kCsvThreads); }

void launch_csv_compact(const Particle* tmp, const uint32_t* keep, uint64_t m, uint32_t* block_count,
                        uint64_t* total, Particle* dst, cudaStream_t s) {
  const size_t blocks = csv_keep_blocks(m);
  if (blocks == 0) return;
  k_keep_count<<<(unsigned)blocks, kCsvThreads, 0, s>>>(keep, m, block_count);
  k_scan_counts<<<1, 1024, 0, s>>>(block_count, (uint32_t)blocks, total);
  if (dst) k_keep_scatter<<<(unsigned)blocks, kCsvThreads, 0, s>>>(tmp, keep, m, block_count, dst);
}

size_t vtk_slot_bytes(uint32_t n) { return (size_t)n * (2 * kPosSlot + kMassSlot); }
size_t vtk_blocks(uint32_t n) { return ((size_t)n + kCsvThreads - 1) / kCsvThreads; }

void launch_vtk_format(const Particle* p, uint32_t n, char* slots, uint32_t* len, uint32_t* block_sum,
                       uint64_t* block_off, uint64_t* totals, int sms, cudaStream_t s) {
  if (n == 0) return;
  unsigned blocks = (n + 127) / 128;
  if (blocks > (unsigned)sms * 16) blocks = sms * 16;
  char* pos = slots;
  char* mass = slots + (size_t)n * kPosSlot;
  char* vel = mass + (size_t)n * kMassSlot;
  k_vtk_format<<<blocks, 128, 0, s>>>(p, n, pos, mass, vel, len);
  const size_t nb = vtk_blocks(n);
  for (int k = 0; k < 3; ++k) {
    k_len_sums<<<(unsigned)nb, kCsvThreads, 0, s>>>(len + (size_t)k * n, n, block_sum + k * nb);
    k_scan_sums64<<<1, 1024, 0, s>>>(block_sum + k * nb, (uint32_t)nb, block_off + k * nb, totals + k);
  }
}

void launch_vtk_gather(const char* slots, uint32_t n, const uint32_t* len, const uint64_t* block_off,
                       char* const out[3], cudaStream_t s) {
  if (n == 0) return;
  const char* base[3] = {slots, slots + (size_t)n * kPosSlot, slots + (size_t)n * (kPosSlot + kMassSlot)};
  const int size[3] = {kPosSlot, kMassSlot, kPosSlot};
  const size_t nb = vtk_blocks(n);
  for (int k = 0; k < 3; ++k)
    k_vtk_gather<<<(unsigned)nb, kCsvThreads, 0, s>>>(base[k], size[k], len + (size_t)k * n, block_off + k * nb, n,
                                                      out[k]);
}

}  // namespace bhg
