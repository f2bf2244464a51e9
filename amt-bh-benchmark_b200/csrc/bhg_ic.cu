// Plummer spheres generated on the device, for requests whose initial
// conditions are described by a seed rather than shipped as particles.
//
// Same distribution as the host generator (bhg_host.cc, Aarseth-Henon-Wielen
// sampling with G = 1): r = a / sqrt(X^(-2/3) - 1) redrawn while r >= 10a,
// isotropic position, speed q v_e with v_e = sqrt(2M) (r^2 + a^2)^(-1/4) and
// q by von Neumann rejection on q^2 (1 - q^2)^(7/2) under y ~ U(0, 0.1),
// isotropic velocity.  The random numbers come from a counter-based
// generator, Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011), keyed by the request seed and
// counted by (particle, purpose, attempt), so every particle is drawn
// independently and the result does not depend on the launch shape.
#include "bhg_kernels.h"

namespace bhg {

namespace {

struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;  // the published round multipliers
  const uint32_t lo0 = m0 * c.x, hi0 = __umulhi(m0, c.x);
  const uint32_t lo1 = m1 * c.z, hi1 = __umulhi(m1, c.z);
  return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ __forceinline__ U4 philox(U4 c, uint64_t key) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;  // the published key schedule (golden ratio, sqrt(3) - 1)
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Two uniforms in [0, 1) with 53 random bits each.
__device__ __forceinline__ void uniform2(uint64_t key, uint32_t i, uint32_t purpose, uint32_t attempt, double& u0,
                                         double& u1) {
  const U4 r = philox(U4{i, purpose, attempt, 0x5eedu}, key);
  const uint64_t a = ((uint64_t)r.x << 32 | r.y) >> 11, b = ((uint64_t)r.z << 32 | r.w) >> 11;
  u0 = (double)a * 0x1.0p-53;
  u1 = (double)b * 0x1.0p-53;
}

// A point on the unit sphere from two uniforms (uniform z, uniform azimuth).
__device__ __forceinline__ void unit_vector(double u0, double u1, double out[3]) {
  const double z = 2.0 * u0 - 1.0, phi = 2.0 * 3.14159265358979323846 * u1;
  const double s = sqrt(fmax(0.0, 1.0 - z * z));
  double sn, cs;
  sincos(phi, &sn, &cs);
  out[0] = s * cs, out[1] = s * sn, out[2] = z;
}

constexpr uint32_t kMaxAttempts = 4096;  // rejection loops stop (keeping a fallback value) after this

}  // namespace

__global__ void k_plummer(Particle* __restrict__ out, uint32_t n, double a, double mass, double cx, double cy,
                          double cz, double bx, double by, double bz, uint32_t id0, uint64_t seed) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double r = 9.99 * a, u0, u1;
    for (uint32_t t = 0; t < kMaxAttempts; ++t) {  // radius
      uniform2(seed, i, 1u, t, u0, u1);
      if (u0 > 0.0) {
        const double rr = a / sqrt(pow(u0, -2.0 / 3.0) - 1.0);
        if (rr < 10.0 * a) {
          r = rr;
          break;
        }
      }
    }
    double dir[3], vdir[3];
    uniform2(seed, i, 2u, 0u, u0, u1);
    unit_vector(u0, u1, dir);
    double q = 0.0;
    for (uint32_t t = 0; t < kMaxAttempts; ++t) {  // speed as a fraction of the escape speed
      uniform2(seed, i, 3u, t, u0, u1);
      const double y = 0.1 * u1;
      if (!(y > u0 * u0 * pow(1.0 - u0 * u0, 3.5))) {
        q = u0;
        break;
      }
    }
    uniform2(seed, i, 4u, 0u, u0, u1);
    unit_vector(u0, u1, vdir);
    const double ve = sqrt(2.0 * mass) * pow(r * r + a * a, -0.25);
    Particle p;
    p.id = id0 + i;
    p.pad = 0;
    p.mass = mass / (double)n;
    p.pos[0] = cx + r * dir[0], p.pos[1] = cy + r * dir[1], p.pos[2] = cz + r * dir[2];
    p.vel[0] = bx + q * ve * vdir[0], p.vel[1] = by + q * ve * vdir[1], p.vel[2] = bz + q * ve * vdir[2];
    out[i] = p;
  }
}

void launch_plummer(Particle* out, uint32_t n, double a, double mass, const double* c, const double* b, uint32_t id0,
                    uint64_t seed, int sms, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > sms * 8) blocks = sms * 8;
  if (blocks < 1) blocks = 1;
  k_plummer<<<blocks, 256, 0, s>>>(out, n, a, mass, c[0], c[1], c[2], b[0], b[1], b[2], id0, seed);
}

}  // namespace bhg
