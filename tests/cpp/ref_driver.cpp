// ref_driver.cpp -- the reference's kick_pme_test (src/test.cpp:182-234),
// written against the reference's own C++ signatures (include/tpm_reference.hpp)
// and linked to libtigerpm_b200.so.  Prints one "RESULT key=value ..." line.
//
// usage: ref_driver --parts_dim=N [library option flags...]
#include <cstdio>
#include <cstdlib>
#include <random>

#include "tpm_reference.hpp"

int main(int argc, char* argv[]) {
  if (!process_options(argc, argv)) return 2;
  const auto& o = get_options();
  const size_t n = (size_t)o.parts_dim * o.parts_dim * o.parts_dim;
  // particles_random_init (src/particles.cpp:100-132): uniform positions,
  // zero velocities and rungs (seeded, GSL's stream is not reproduced)
  particles_resize(n);
  std::mt19937_64 rng(1234);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  for (size_t i = 0; i < n; i++) {
    for (int d = 0; d < NDIM; d++) {
      particles_X[d][i] = fixed32(u(rng));
      particles_U[d][i] = 0.0f;
    }
    particles_R[i] = 0;
  }
  try {
    gravity_long_compute(GRAVITY_LONG_PME);
    chainmesh_create();
    chainmesh_exchange_begin();
    chainmesh_exchange_end();
    kick_pme_begin(0, 1.0, 1.0, true);
    kick_pme_end();
    // chain-mesh checks: cells tile [0, n) in (z, y, x) order and hold their particles
    const int C = o.chain_dim;
    long expect = 0, bad_cells = 0, misplaced = 0;
    for (int z = 0; z < C; z++)
      for (int y = 0; y < C; y++)
        for (int x = 0; x < C; x++) {
          array<int, NDIM> ijk;
          ijk[0] = x;
          ijk[1] = y;
          ijk[2] = z;
          const chaincell c = chainmesh_get(ijk);
          if (c.pbegin != expect || c.pend < c.pbegin) bad_cells++;
          expect = c.pend;
          for (int i = c.pbegin; i < c.pend; i++) {
            const int cx = (int)(particles_X[0][i].to_double() * C);
            const int cy = (int)(particles_X[1][i].to_double() * C);
            const int cz = (int)(particles_X[2][i].to_double() * C);
            if (cx != x || cy != y || cz != z) misplaced++;
          }
        }
    int rung_max = 0;
    for (size_t i = 0; i < n; i++) rung_max = particles_R[i] > rung_max ? particles_R[i] : rung_max;
    const auto box = gravity_long_get_phi_box();
    const auto phi = gravity_long_get_phi(box);
    gravity_short_ewald_compare(256);
    const auto e = tpmref::last_ewald_errors();
    printf("RESULT n=%zu cells_bad=%ld misplaced=%ld total=%ld phi_box=%d rung_max=%d force_rms=%.6e "
           "force_rms_vector=%.6e\n",
           n, bad_cells, misplaced, expect, (int)phi.size(), rung_max, e.force_rms, e.force_rms_vector);
    tpmref::reset();
  } catch (const std::exception& ex) {
    printf("FAILED %s\n", ex.what());
    return 1;
  }
  return 0;
}
