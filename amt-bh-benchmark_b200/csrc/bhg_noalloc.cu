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

#include <cuda.h>

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
// a stand-in, not device memory); this is its device address, looked up with
// the device current.  The address belongs to the CUDA context the library's
// module was loaded into: after cudaDeviceReset the device gets a new primary
// context where the array may sit elsewhere.  So the lookups are cached per
// context (the driver's cuCtxGetCurrent, reached through the runtime's entry
// point table: no link against libcuda), and a new context looks it up again.
constexpr int kCacheSlots = 64;
std::mutex g_setup_mutex;
struct Slot {
  CUcontext ctx;
  double* ptr;
};
Slot g_slots[kCacheSlots] = {};
int g_next_slot = 0;
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn g_ctx_get_current = nullptr;

int partials_for_current_context(double** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return BHG_ECUDA;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return BHG_ECUDA;
  for (const Slot& s : g_slots)
    if (ctx && s.ctx == ctx && s.ptr) {
      *out = s.ptr;
      return BHG_OK;
    }
  // the lookup also makes the current device's primary context current on
  // this thread when none was
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess) return BHG_ECUDA;
  if (!ctx && (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)) return BHG_ECUDA;
  g_slots[g_next_slot] = Slot{ctx, static_cast<double*>(p)};
  g_next_slot = (g_next_slot + 1) % kCacheSlots;
  *out = static_cast<double*>(p);
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
  int r = partials_for_current_context(&partials);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int nblocks = (int)((n + kNoAllocThreads - 1) / kNoAllocThreads);
  // every partial this call reads is written by this call's k_energy first,
  // so the array needs no clearing between calls.  Each launch reports its
  // own error: an unrelated error left on the thread by an earlier call is
  // neither returned as this call's nor cleared.
  if (bhg::launch_energy(reinterpret_cast<const bhg::Particle*>(particles), 0u, (uint32_t)n, G, partials, 0, s) !=
      cudaSuccess)
    return BHG_ECUDA;
  void* args[] = {(void*)&partials, (void*)&nblocks, (void*)&result};
  if (cudaLaunchKernel((const void*)k_energy_total, dim3(1), dim3(1), args, 0, s) != cudaSuccess) return BHG_ECUDA;
  return BHG_OK;
}
