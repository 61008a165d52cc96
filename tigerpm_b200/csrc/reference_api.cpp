// reference_api.cpp -- TigerPM's C++ PME-kick functions on top of the C ABI.
//
// Each function keeps the reference's signature and meaning (see
// include/tpm_reference.hpp for the file:line of every declaration) and
// works on the host SoA globals particles_X/U/R/P/G like the reference:
// arrays go to one process-wide device context, the kernels run there, and
// results come back into the same globals.  Device memory persists between
// calls (the reference allocates and frees per kick, src/kick_pme.cu:435,616).
//
// Call protocol, as in the reference's kick_pme_test (src/test.cpp:182-234):
//   gravity_long_compute  uploads the particles, sorts them on the device and
//                         solves for phi (the host order is unchanged);
//   chainmesh_create      brings the chain-mesh order back to the host
//                         globals (re-using that device sort, so phi stays
//                         valid) or uploads and sorts when none is pending;
//   kick_pme              kicks on the device and writes v, rung, g, phi back.
// The host arrays must not change between these calls.
#include "../../include/tpm_reference.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <set>
#include <stdexcept>
#include <string>

static_assert(sizeof(fixed32) == sizeof(uint32_t), "fixed32 must be a bare uint32");

#ifndef TPM_REFERENCE_GLOBALS_EXTERNAL
array<std::vector<fixed32>, NDIM> particles_X;
array<std::vector<float>, NDIM> particles_U;
std::vector<char> particles_R;
std::vector<float> particles_P;
array<std::vector<float>, NDIM> particles_G;

int particles_size() { return (int)particles_X[0].size(); }

void particles_resize(size_t n) {
  for (int d = 0; d < NDIM; d++) {
    particles_X[d].resize(n);
    particles_U[d].resize(n);
    particles_G[d].resize(n);
  }
  particles_R.resize(n);
  particles_P.resize(n);
}

namespace {
options g_opts;
bool g_opts_set = false;

void fill_options(const tpm_options& o) {
  g_opts.four_dim = o.four_dim;
  g_opts.chain_dim = o.chain_dim;
  g_opts.parts_dim = o.parts_dim;
  g_opts.parts_o_four = o.parts_o_four;
  g_opts.parts_o_chain = o.parts_o_chain;
  g_opts.four_o_chain = o.four_o_chain;
  g_opts.eta = o.eta;
  g_opts.sigma8 = o.sigma8;
  g_opts.code_to_cm = o.code_to_cm;
  g_opts.hubble = o.hubble;
  g_opts.GM = o.GM;
  g_opts.hsoft = o.hsoft;
  g_opts.box_size = o.box_size;
  g_opts.rs = o.rs;
  g_opts.omega_m = o.omega_m;
  g_opts.z0 = o.z0;
  g_opts.ext = o;
  g_opts_set = true;
}
}  // namespace

// process_options (src/options.cpp:37-118): the reference's flags plus the
// library's extensions; prints the option summary as the reference does.
bool process_options(int argc, char* argv[]) {
  tpm_options o;
  std::vector<const char*> args;
  std::string test, config;
  for (int i = 1; i < argc; i++) {
    args.push_back(argv[i]);
    if (!strncmp(argv[i], "--test=", 7)) test = argv[i] + 7;
    if (!strncmp(argv[i], "--config_file=", 14)) config = argv[i] + 14;
  }
  const int rc = tpm_options_parse(&o, (int)args.size(), args.data());
  if (rc != TPM_OK) {
    printf("%s\n", tpm_last_error_message());
    return false;
  }
  fill_options(o);
  g_opts.test = test;
  g_opts.config_file = config;
  printf("Simulation Options\n");
  printf("box_size = %e\nparts_o_four = %e\nparts_o_chain = %e\nfour_o_chain = %e\n", g_opts.box_size,
         (double)g_opts.parts_o_four, (double)g_opts.parts_o_chain, (double)g_opts.four_o_chain);
  printf("chain_dim = %e\nfour_dim = %e\nparts_dim = %e\n", (double)g_opts.chain_dim, (double)g_opts.four_dim,
         (double)g_opts.parts_dim);
  return true;
}

const options& get_options() {
  if (!g_opts_set) {
    // process_options was never called: the derived values for 60^3
    // particles on a 20^3 mesh with a 4^3 chain mesh (parts_o_four = 3,
    // four_o_chain = 5, the reference's ratios).
    tpm_options o;
    tpm_options_init(&o, 60, 3, 5);
    fill_options(o);
  }
  return g_opts;
}
#endif  // TPM_REFERENCE_GLOBALS_EXTERNAL

namespace {

enum class Dev { Empty, Unsorted, SortedDeviceOnly, Synced };

tpm_ctx* g_ctx = nullptr;
int64_t g_cap = 0;
Dev g_dev = Dev::Empty;
tpmref::EwaldErrors g_err{0, 0, 0, 0, 0};

void check(int rc, const char* where) {
  if (rc != TPM_OK) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s (%s)", where, tpm_error_string(rc), tpm_last_error_message());
    fprintf(stderr, "%s\n", buf);
    throw std::runtime_error(buf);
  }
}

tpm_options library_options() {
#ifdef TPM_REFERENCE_GLOBALS_EXTERNAL
  const auto& r = get_options();
  tpm_options o;
  tpm_options_init(&o, r.parts_dim, 1, 1);
  o.four_dim = r.four_dim;
  o.chain_dim = r.chain_dim;
  o.parts_o_four = r.parts_o_four;
  o.parts_o_chain = r.parts_o_chain;
  o.four_o_chain = r.four_o_chain;
  o.eta = r.eta;
  o.GM = r.GM;
  o.hsoft = r.hsoft;
  o.rs = r.rs;
  o.box_size = r.box_size;
  return o;
#else
  return get_options().ext;
#endif
}

uint32_t* raw(int d) { return reinterpret_cast<uint32_t*>(particles_X[d].data()); }

void ensure_context(int64_t n) {
  if (g_ctx && g_cap >= n) return;
  if (g_ctx) tpm_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  const tpm_options o = library_options();
  const int64_t cap = std::max<int64_t>(n, 1);
  check(tpm_ctx_create(&o, cap, &g_ctx), "tpm_ctx_create");
  g_cap = cap;
  g_dev = Dev::Empty;
}

void upload() {
  const int64_t n = particles_size();
  ensure_context(n);
  particles_resize((size_t)n);  // makes the FORCE_TEST arrays as long as X
  check(tpm_set_particles(g_ctx, n, raw(0), raw(1), raw(2), particles_U[0].data(), particles_U[1].data(),
                          particles_U[2].data(), reinterpret_cast<const int8_t*>(particles_R.data())),
        "tpm_set_particles");
  g_dev = Dev::Unsorted;
}

void download_all() {
  check(tpm_get_particles(g_ctx, raw(0), raw(1), raw(2), particles_U[0].data(), particles_U[1].data(),
                          particles_U[2].data(), reinterpret_cast<int8_t*>(particles_R.data())),
        "tpm_get_particles");
}

void require_synced(const char* where) {
  if (g_dev == Dev::SortedDeviceOnly) {
    download_all();
    g_dev = Dev::Synced;
  }
  if (g_dev != Dev::Synced) {
    std::string m = std::string(where) + ": call chainmesh_create first";
    fprintf(stderr, "%s\n", m.c_str());
    throw std::runtime_error(m);
  }
}

}  // namespace

namespace tpmref {
tpm_ctx* context() {
  ensure_context(std::max<int64_t>(particles_size(), 1));
  return g_ctx;
}
void reset() {
  if (g_ctx) tpm_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  g_cap = 0;
  g_dev = Dev::Empty;
}
EwaldErrors last_ewald_errors() { return g_err; }
}  // namespace tpmref

// chainmesh_create (src/chainmesh.cpp:139-161): the particle globals end up
// in chain-mesh order (the reference's partition order, bit for bit).
void chainmesh_create() {
  if (g_dev != Dev::SortedDeviceOnly) {
    upload();
    check(tpm_chainmesh_create(g_ctx), "tpm_chainmesh_create");
  }
  download_all();
  g_dev = Dev::Synced;
}

// One box with periodic cell indices: there are no ghost cells to exchange
// (src/chainmesh.cpp:58-137 copies boundary cells between ranks).
void chainmesh_exchange_begin() {}
void chainmesh_exchange_end() {}

range<int> chainmesh_interior_box() {
  range<int> r;
  const int C = library_options().chain_dim;
  for (int d = 0; d < NDIM; d++) {
    r.begin[d] = 0;
    r.end[d] = C;
  }
  return r;
}

chaincell chainmesh_get(const array<int, NDIM>& i) {
  require_synced("chainmesh_get");
  int ijk[3] = {i[0], i[1], i[2]};
  int32_t b = 0, e = 0;
  check(tpm_chainmesh_get(g_ctx, ijk, &b, &e), "tpm_chainmesh_get");
  chaincell c;
  c.pbegin = b;
  c.pend = e;
  return c;
}

void gravity_long_compute(gravity_long_type type) {
  upload();
  check(tpm_chainmesh_create(g_ctx), "tpm_chainmesh_create");
  check(tpm_gravity_long_compute(g_ctx, (int)type), "tpm_gravity_long_compute");
  g_dev = Dev::SortedDeviceOnly;
}

vector<float> gravity_long_get_phi(const range<int>& box) {
  vector<float> out((size_t)std::max(0, box.volume()));
  int b[6] = {box.begin[0], box.begin[1], box.begin[2], box.end[0], box.end[1], box.end[2]};
  if (!out.empty()) check(tpm_gravity_long_get_phi(g_ctx, b, out.data()), "tpm_gravity_long_get_phi");
  return out;
}

range<int> gravity_long_get_phi_box() {
  range<int> r;
  int b[6];
  check(tpm_gravity_long_get_phi_box(tpmref::context(), b), "tpm_gravity_long_get_phi_box");
  for (int d = 0; d < NDIM; d++) {
    r.begin[d] = b[d];
    r.end[d] = b[3 + d];
  }
  return r;
}

std::pair<float, array<float, NDIM>> gravity_long_force_at(const array<double, NDIM>& pos) {
  double p[3] = {pos[0], pos[1], pos[2]};
  float phi = 0.f, g[3] = {0.f, 0.f, 0.f};
  check(tpm_gravity_long_force_at(g_ctx, 1, p, &phi, g), "tpm_gravity_long_force_at");
  array<float, NDIM> ga;
  for (int d = 0; d < NDIM; d++) ga[d] = g[d];
  return std::make_pair(phi, ga);
}

// kick_pme (src/kick_pme.cu:390-621): kicks the sinks of the chain cells in
// box; velocities, rungs and the FORCE_TEST g / phi come back into the
// globals (src/kick_pme.cu:572-614).
void kick_pme(range<int> box, int min_rung, double scale, double t0, bool first_call) {
  require_synced("kick_pme");
  int b[6] = {box.begin[0], box.begin[1], box.begin[2], box.end[0], box.end[1], box.end[2]};
  const int rc = tpm_kick_pme(g_ctx, b, min_rung, scale, t0, first_call ? 1 : 0);
  if (rc == TPM_ERR_RUNG) {
    printf("Rung out of range (clamped)\n");  // the reference prints, then asserts
  } else {
    check(rc, "tpm_kick_pme");
  }
  check(tpm_get_particles(g_ctx, nullptr, nullptr, nullptr, particles_U[0].data(), particles_U[1].data(),
                          particles_U[2].data(), reinterpret_cast<int8_t*>(particles_R.data())),
        "tpm_get_particles");
  check(tpm_get_forces(g_ctx, particles_G[0].data(), particles_G[1].data(), particles_G[2].data(),
                       particles_P.data()),
        "tpm_get_forces");
}

// kick_pme_begin / kick_pme_end (src/kick_pme.cpp:9-29): the interior box;
// with no ghosts appended there is nothing to drop at the end.
void kick_pme_begin(int min_rung, double scale, double t0, bool first_call) {
  kick_pme(chainmesh_interior_box(), min_rung, scale, t0, first_call);
}
void kick_pme_end() {
  if (g_ctx) check(tpm_synchronize(g_ctx), "tpm_synchronize");
}

// gravity_short_ewald_call_kernel (src/gravity_short.cu:10-91): FP64 Ewald
// potential and force at the sink positions from every particle.
std::pair<vector<double>, array<vector<double>, NDIM>> gravity_short_ewald_call_kernel(const vector<fixed32>& sinkx,
                                                                                    const vector<fixed32>& sinky,
                                                                                    const vector<fixed32>& sinkz) {
  if (g_dev == Dev::Empty) upload();
  const int64_t ns = (int64_t)sinkx.size();
  std::pair<vector<double>, array<vector<double>, NDIM>> rc;
  rc.first.resize(ns);
  for (int d = 0; d < NDIM; d++) rc.second[d].resize(ns);
  if (ns == 0) return rc;
  check(tpm_gravity_short_ewald(g_ctx, ns, reinterpret_cast<const uint32_t*>(sinkx.data()),
                                reinterpret_cast<const uint32_t*>(sinky.data()),
                                reinterpret_cast<const uint32_t*>(sinkz.data()), 1, rc.first.data(),
                                rc.second[0].data(), rc.second[1].data(), rc.second[2].data()),
        "tpm_gravity_short_ewald");
  return rc;
}

// gravity_short_ewald_compare (src/gravity_short.cpp:35-82): errors of the
// last kick's FORCE_TEST g and phi on Nsamples distinct particles, printed in
// the reference's format.  Samples come from a seeded generator (the
// reference uses rand()).
void gravity_short_ewald_compare(int Nsamples) {
  const int n = particles_size();
  std::mt19937_64 rng(4321);
  std::set<int> chosen;
  vector<int> idx;
  while ((int)idx.size() < std::min(Nsamples, n)) {
    const int i = (int)(rng() % (uint64_t)n);
    if (chosen.insert(i).second) idx.push_back(i);
  }
  vector<fixed32> sx(idx.size()), sy(idx.size()), sz(idx.size());
  for (size_t k = 0; k < idx.size(); k++) {
    sx[k] = particles_X[0][idx[k]];
    sy[k] = particles_X[1][idx[k]];
    sz[k] = particles_X[2][idx[k]];
  }
  const auto res = gravity_short_ewald_call_kernel(sx, sy, sz);
  double l2sum_phi = 0, l2norm_phi = 0, l2sum_force = 0, l2norm_force = 0, lmax_phi = 0, lmax_force = 0, vec = 0;
  for (size_t k = 0; k < idx.size(); k++) {
    const int i = idx[k];
    double g1 = 0, g2 = 0, dv = 0;
    for (int d = 0; d < NDIM; d++) {
      g1 += (double)particles_G[d][i] * particles_G[d][i];
      g2 += res.second[d][k] * res.second[d][k];
      dv += (particles_G[d][i] - res.second[d][k]) * (particles_G[d][i] - res.second[d][k]);
    }
    g1 = std::sqrt(g1);
    g2 = std::sqrt(g2);
    const double f1 = particles_P[i], f2 = res.first[k];
    l2sum_phi += (f1 - f2) * (f1 - f2);
    lmax_phi += std::abs(f1 - f2);
    l2norm_phi += f2 * f2;
    l2sum_force += (g1 - g2) * (g1 - g2);
    lmax_force += std::abs(g1 - g2);
    l2norm_force += g2 * g2;
    vec += dv;
  }
  g_err.force_rms = std::sqrt(l2sum_force / l2norm_force);
  g_err.force_max = lmax_force / std::sqrt(l2norm_force);
  g_err.phi_rms = std::sqrt(l2sum_phi / l2norm_phi);
  g_err.phi_max = lmax_phi / std::sqrt(l2norm_phi);
  g_err.force_rms_vector = std::sqrt(vec / l2norm_force);
  printf("Force RMS Error     = %e\n", g_err.force_rms);
  printf("Force Max Error     = %e\n", g_err.force_max);
  printf("Potential RMS Error = %e\n", g_err.phi_rms);
  printf("Potential Max Error = %e\n", g_err.phi_max);
}
