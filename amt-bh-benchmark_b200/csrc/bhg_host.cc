// Host-side helpers of the C ABI: synthetic initial conditions and the
// reference's CSV input format.
#include "bhg.h"
#include "bhg_plummer.h"

#include <cstdio>

extern "C" {

// Plummer sphere (bhg_plummer.h: Aarseth-Henon-Wielen sampling, G = 1).
uint64_t bhg_ic_plummer(bh_particle64* out, size_t n, double a, double total_mass, const double* centre,
                        const double* bulk, uint32_t id0, uint64_t seed) {
  for (size_t i = 0; i < n; ++i) out[i].pad = 0;
  return bhg_ic::plummer(out, n, a, total_mass, centre, bulk, id0, seed);
}

// id,mass,pos_x,pos_y,pos_z,vel_x,vel_y,vel_z per line (io.h:11-17), with
// round-trip precision.
int bhg_write_csv(const char* path, const bh_particle64* p, size_t n) {
  FILE* f = std::fopen(path, "w");
  if (!f) return BHG_EINVAL;
  for (size_t i = 0; i < n; ++i) {
    std::fprintf(f, "%u,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n", p[i].id, p[i].mass, p[i].pos[0], p[i].pos[1],
                 p[i].pos[2], p[i].vel[0], p[i].vel[1], p[i].vel[2]);
  }
  return std::fclose(f) == 0 ? BHG_OK : BHG_EINVAL;
}

}  // extern "C"
