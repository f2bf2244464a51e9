// bhg_energy_noalloc: the energy diagnostic for callers that cannot
// allocate GPU memory.
//
// Some host programs cannot let a library call cudaMalloc: a driver that has
// already handed all of the GPU's memory to its own pool (cudaMalloc would
// fail, or take memory the pool counts on), or a time-stepping loop that
// must not stall, since cudaFree synchronises the whole device.  bhg_energy
// allocates a small buffer of per-block partial sums on every call; this
// variant keeps those partial sums in a fixed array in the library's own
// device memory instead, so it allocates nothing.
#include "bhg.h"
#include "bhg_kernels.h"

#include <mutex>

namespace {

// Per-block partial sums (kinetic, potential) of k_energy: 256 particles per
// block, so at most kNoAllocMaxBlocks * 256 particles per call.  16 KB, held
// by every GPU that loads the library until the process exits.
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 1024;
constexpr size_t kNoAllocMaxParticles = (size_t)kNoAllocMaxBlocks * kNoAllocThreads;  // 262,144

static __device__ __align__(256) double g_energy_partials[2 * kNoAllocMaxBlocks];

// Host code may not hand the symbol itself to a kernel (on the host it names
// a stand-in, not device memory); this is its device address per device,
// looked up once with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_ptr[kMaxDevices] = {};

int partials_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BHG_ECUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess) {
      cudaGetLastError();
      return BHG_ECUDA;
    }
    g_partials_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_ptr[dev];
  return BHG_OK;
}

// Sums the per-block partials in block order - the order bhg_energy sums
// them on the host - into result[0] (kinetic) and result[1] (potential).
__global__ void k_energy_total(const double* __restrict__ partials, int nblocks, double* __restrict__ result) {
  double ek = 0.0, ep = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    ek += partials[2 * b];
    ep += partials[2 * b + 1];
  }
  result[0] = ek;
  result[1] = ep;
}

}  // namespace

extern "C" int bhg_energy_noalloc(const bh_particle64* particles, size_t n, double G, double* result,
                                  void* stream) {
  if (!particles || !result || n == 0) return BHG_EINVAL;
  if (n > kNoAllocMaxParticles) return BHG_EINVAL;  // more than the fixed partial-sum array can hold
  double* partials = nullptr;
  int r = partials_for_current_device(&partials);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nblocks = (int)((n + kNoAllocThreads - 1) / kNoAllocThreads);
  // every partial this call reads is written by this call's k_energy first,
  // so the array needs no clearing between calls
  bhg::launch_energy(reinterpret_cast<const bhg::Particle*>(particles), 0u, (uint32_t)n, G, partials, 0, s);
  k_energy_total<<<1, 1, 0, s>>>(partials, nblocks, result);
  return cudaGetLastError() == cudaSuccess ? BHG_OK : BHG_ECUDA;
}
