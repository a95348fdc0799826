// Host-side parts of the reference's C++ interface, exercised without a GPU:
// process_options with a config file (src/options.cpp:44-115), the derived
// option values (:88-95), the cosmology functions (src/cosmology.cpp) and the
// raw SoA particle files.  Prints one JSON object; tests/test_host_cxx.py
// builds, runs and checks it.
//
//   host_check <config file> <particle file> [--key value ...]
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "ct2_cosmictiger.hpp"

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  std::vector<char *> args = {argv[0]};
  std::string cf = std::string("--config_file=") + argv[1];
  args.push_back(const_cast<char *>(cf.c_str()));
  for (int i = 3; i < argc; i++) args.push_back(argv[i]);
  const bool ok = process_options((int)args.size(), args.data());
  const options &o = get_options();
  std::printf("{\"ok\": %s, \"hsoft\": %.9g, \"bwidth\": %.9g, \"eta\": %.9g, \"omega_m\": %.9g, "
              "\"hubble\": %.9g, \"Ngrid\": %zu, \"ppcell\": %d, \"mesh\": %d, \"order\": %d, "
              "\"GM\": %.9g, \"nparts\": %zu, \"code_to_cm\": %.9g, \"code_to_s\": %.9g, "
              "\"omega_r\": %.9g, \"omega_lam\": %.9g, \"config_file\": \"%s\"",
              ok ? "true" : "false", o.hsoft, o.bwidth, o.eta, o.omega_m, o.hubble, o.Ngrid,
              o.ppcell, o.mesh, o.order, o.GM, o.nparts, o.code_to_cm, o.code_to_s, o.omega_r,
              o.omega_lam, o.config_file.c_str());
  // cosmology
  const double as[] = {0.02, 0.1, 0.5, 1.0};
  std::printf(", \"dadt\": [");
  for (int i = 0; i < 4; i++) std::printf("%s%.17g", i ? ", " : "", cosmos_dadt(as[i]));
  std::printf("], \"time\": %.17g, \"conformal_time\": %.17g", cosmos_time(0.1, 0.5),
              cosmos_conformal_time(0.1, 0.5));
  double a = 0.1, adot = cosmos_dadt(0.1), adotdot = 0.0;
  const double dt = 0.02 / adot;
  cosmos_update(adotdot, adot, a, dt);
  std::printf(", \"update\": {\"dt\": %.17g, \"a\": %.17g, \"adot\": %.17g, \"adotdot\": %.17g}",
              dt, a, adot, adotdot);
  // particle file round trip
  particle_allocate(1000);
  for (int i = 0; i < 1000; i++) {
    particle_x(i) = 2654435761u * (uint32_t)i;
    particle_y(i) = 40503u * (uint32_t)i + 7u;
    particle_z(i) = ~(uint32_t)i;
    particle_vx(i) = 0.5f * i;
    particle_vy(i) = -0.25f * i;
    particle_vz(i) = 1.0f / (1 + i);
    particle_rung(i) = (char)(i % 5);
  }
  particles_save(argv[2]);
  particle_allocate(0);
  particles_load(argv[2]);
  bool same = particle_count() == 1000;
  for (int i = 0; same && i < 1000; i++)
    same = particle_x(i) == 2654435761u * (uint32_t)i && particle_vz(i) == 1.0f / (1 + i) &&
           particle_rung(i) == (char)(i % 5);
  std::printf(", \"soa_round_trip\": %s}\n", same ? "true" : "false");
  return 0;
}
