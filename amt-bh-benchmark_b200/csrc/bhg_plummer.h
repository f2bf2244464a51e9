// Host generator of the synthetic initial conditions: Plummer spheres by
// Aarseth-Henon-Wielen (1974) sampling, G = 1.  Header-only so that the
// library (bhg_ic_plummer) and the timing harness of the reference solver
// draw exactly the same particles from the same seed.
//
//   radius   r = a / sqrt(X^(-2/3) - 1), X ~ U(0,1), drawn again while r >= 10a;
//   position r times an isotropic unit vector;
//   speed    q v_e with v_e = sqrt(2 M) (r^2 + a^2)^(-1/4), q by von Neumann
//            rejection of (q, y) ~ U(0,1) x U(0,0.1) against q^2 (1-q^2)^(7/2);
//   velocity that speed times an isotropic unit vector.
// Draw order per particle: X (repeated), 2 for the direction, (q, y)
// (repeated), 2 for the velocity direction.  Uniforms take the top 53 bits
// of std::mt19937_64 (platform independent, unlike
// std::uniform_real_distribution).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <random>

namespace bhg_ic {

struct Uniform {
  std::mt19937_64 g;
  explicit Uniform(uint64_t seed) : g(seed) {}
  double operator()() { return (double)(g() >> 11) * 0x1.0p-53; }
};

inline void unit_vector(Uniform& u, double out[3]) {
  const double z = 2.0 * u() - 1.0;
  const double phi = 2.0 * M_PI * u();
  const double s = std::sqrt(1.0 - z * z);
  out[0] = s * std::cos(phi);
  out[1] = s * std::sin(phi);
  out[2] = z;
}

// Writes n particles into out (any 64-byte bh::Particle-layout record type
// with id, pad, mass, pos[3], vel[3]); returns the generator's next output,
// the seed a second sphere uses to continue the stream.
template <class P>
uint64_t plummer(P* out, size_t n, double a, double total_mass, const double* centre, const double* bulk,
                 uint32_t id0, uint64_t seed) {
  Uniform u(seed);
  const double c[3] = {centre ? centre[0] : 0.0, centre ? centre[1] : 0.0, centre ? centre[2] : 0.0};
  const double b[3] = {bulk ? bulk[0] : 0.0, bulk ? bulk[1] : 0.0, bulk ? bulk[2] : 0.0};
  const double m = n ? total_mass / (double)n : 0.0;
  for (size_t i = 0; i < n; ++i) {
    double r;
    do {
      double x = u();
      r = x > 0.0 ? a / std::sqrt(std::pow(x, -2.0 / 3.0) - 1.0) : INFINITY;
    } while (!(r < 10.0 * a));
    double dir[3], vdir[3];
    unit_vector(u, dir);
    double q, y;
    do {
      q = u();
      y = 0.1 * u();
    } while (y > q * q * std::pow(1.0 - q * q, 3.5));
    const double ve = std::sqrt(2.0 * total_mass) * std::pow(r * r + a * a, -0.25);
    unit_vector(u, vdir);
    P& p = out[i];
    p.id = id0 + (uint32_t)i;
    p.mass = m;
    for (int k = 0; k < 3; ++k) {
      p.pos[k] = c[k] + r * dir[k];
      p.vel[k] = b[k] + q * ve * vdir[k];
    }
  }
  return u.g();
}

}  // namespace bhg_ic
