// tpm_reference.hpp -- the reference's C++ PME-kick interface, implemented on
// the C ABI of tpm.h (tigerpm_b200/csrc/reference_api.cpp).
//
// The declarations keep TigerPM's names, argument types and meaning:
//   kick_pme / kick_pme_begin / kick_pme_end            tigerpm/kick_pme.hpp:15-17
//   chainmesh_create / _exchange_begin / _exchange_end /
//   chainmesh_interior_box / chainmesh_get              tigerpm/chainmesh.hpp:13-17
//   gravity_long_compute / _get_phi / _get_phi_box /
//   gravity_long_force_at                               tigerpm/gravity_long.hpp:21-24
//   gravity_short_ewald_call_kernel / _compare          tigerpm/gravity_short.hpp:25-28
//   process_options / get_options                       tigerpm/options.hpp:50-51
// over the same host SoA globals particles_X/U/R/P/G (src/particles.cpp:6-12).
//
// Standalone (the default) this header defines minimal look-alikes of the
// reference's helper types (array, range, fixed32, chaincell, options) and
// the library defines the particle globals.  Built into the reference tree
// with TPM_REFERENCE_GLOBALS_EXTERNAL, it includes the reference's own
// headers instead and binds to the reference's globals.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "tpm.h"

#ifdef TPM_REFERENCE_GLOBALS_EXTERNAL
#include <tigerpm/chainmesh.hpp>
#include <tigerpm/fixed.hpp>
#include <tigerpm/gravity_long.hpp>
#include <tigerpm/gravity_short.hpp>
#include <tigerpm/kick_pme.hpp>
#include <tigerpm/options.hpp>
#include <tigerpm/particles.hpp>
#include <tigerpm/range.hpp>
#else

#define NDIM 3
#define XDIM 0
#define YDIM 1
#define ZDIM 2
#ifndef GRAVITY_LONG_PM
#define GRAVITY_LONG_PM TPM_GRAVITY_LONG_PM
#define GRAVITY_LONG_PME TPM_GRAVITY_LONG_PME
#endif

template <class T, int N>
struct array {
  T A[N];
  T& operator[](int i) { return A[i]; }
  const T& operator[](int i) const { return A[i]; }
  T* data() { return A; }
  const T* data() const { return A; }
  int size() const { return N; }
};

template <class T>
using vector = std::vector<T>;

// range<int>: half-open box, index() with z fastest (tigerpm/range.hpp:149-165).
template <class T>
struct range {
  array<T, NDIM> begin;
  array<T, NDIM> end;
  range() = default;
  explicit range(T n) {
    for (int d = 0; d < NDIM; d++) {
      begin[d] = 0;
      end[d] = n;
    }
  }
  T volume() const {
    T v = 1;
    for (int d = 0; d < NDIM; d++) {
      if (end[d] < begin[d]) return 0;
      v *= end[d] - begin[d];
    }
    return v;
  }
  range pad(T dx = 1) const {
    range r;
    for (int d = 0; d < NDIM; d++) {
      r.begin[d] = begin[d] - dx;
      r.end[d] = end[d] + dx;
    }
    return r;
  }
  int index(const array<T, NDIM>& i) const {
    return (end[2] - begin[2]) * ((end[1] - begin[1]) * (i[0] - begin[0]) + (i[1] - begin[1])) + (i[2] - begin[2]);
  }
};

// fixed<uint32_t> positions (tigerpm/fixed.hpp): raw = (uint32)(2^32 * x).
class fixed32 {
  uint32_t i_ = 0;

 public:
  fixed32() = default;
  fixed32(double x) : i_((uint32_t)(4294967296.0 * x)) {}
  static fixed32 from_raw(uint32_t r) {
    fixed32 f;
    f.i_ = r;
    return f;
  }
  uint32_t raw() const { return i_; }
  float to_float() const { return (float)i_ * (1.0f / 4294967296.0f); }
  double to_double() const { return (double)i_ * (1.0 / 4294967296.0); }
};

struct chaincell {
  int pbegin;
  int pend;
};

using gravity_long_type = int;

// struct options (tigerpm/options.hpp:6-27) plus this library's extensions.
struct options {
  int four_dim;
  int chain_dim;
  int parts_dim;
  int parts_o_four;
  int parts_o_chain;
  int four_o_chain;
  double eta;
  double sigma8;
  double code_to_cm;
  double hubble;
  double GM;
  double hsoft;
  double box_size;
  double rs;
  double omega_m;
  double z0;
  std::string config_file;
  std::string test;
  tpm_options ext;  // the full option set handed to the library
};

bool process_options(int argc, char* argv[]);
const options& get_options();

extern array<std::vector<fixed32>, NDIM> particles_X;
extern array<std::vector<float>, NDIM> particles_U;
extern std::vector<char> particles_R;
extern std::vector<float> particles_P;
extern array<std::vector<float>, NDIM> particles_G;
int particles_size();
void particles_resize(size_t n);

void kick_pme(range<int> box, int min_rung, double scale, double t0, bool first_call);
void kick_pme_begin(int min_rung, double scale, double t0, bool first_call);
void kick_pme_end();
void chainmesh_create();
void chainmesh_exchange_begin();
void chainmesh_exchange_end();
range<int> chainmesh_interior_box();
chaincell chainmesh_get(const array<int, NDIM>&);
void gravity_long_compute(gravity_long_type type = GRAVITY_LONG_PM);
vector<float> gravity_long_get_phi(const range<int>&);
range<int> gravity_long_get_phi_box();
std::pair<float, array<float, NDIM>> gravity_long_force_at(const array<double, NDIM>& pos);
std::pair<vector<double>, array<vector<double>, NDIM>> gravity_short_ewald_call_kernel(const vector<fixed32>& sinkx,
                                                                                    const vector<fixed32>& sinky,
                                                                                    const vector<fixed32>& sinkz);
void gravity_short_ewald_compare(int Nsamples);
#endif  // TPM_REFERENCE_GLOBALS_EXTERNAL

namespace tpmref {
// The process-wide context behind the functions above (created on first
// use from get_options() and the particle count; recreated when it grows).
tpm_ctx* context();
// Frees the context (device memory).
void reset();
// Errors of the last gravity_short_ewald_compare, in the reference's
// metric: force RMS / "max" of |g|, potential RMS / "max", plus the vector
// force RMS.
struct EwaldErrors {
  double force_rms, force_max, phi_rms, phi_max, force_rms_vector;
};
EwaldErrors last_ewald_errors();
}  // namespace tpmref
