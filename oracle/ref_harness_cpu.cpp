// ref_harness_cpu.cpp -- TEST INFRASTRUCTURE: runs pieces of the reference's
// own CPU code, compiled from the reference tree by oracle/build_ref.sh.
//
// build_ref.sh extracts these reference functions verbatim from their files
// (into a temporary directory, never into this repository) and #includes
// them below:
//   particles_sort                 src/particles.cpp:414-444
//   sort (chain-mesh recursion)    src/chainmesh.cpp:168-213
//   cloud4                         src/gravity_long.cpp:127-138
//   apply_laplacian                src/gravity_long.cpp:201-245
// This file supplies what they refer to: the particle globals, the options
// singleton, the chain-cell map, the complex FFT buffer, and a minimal
// stand-in for the few HPX calls they make (async runs deferred; with one
// rank there are no children to fan out to).  The reference headers come
// from -I<reference>; compiled by nvcc, tigerpm.hpp skips its HPX include.
//
// usage:
//   ref_cpu sort <C> <in> <out>       in: n, x,y,z (u32), vx,vy,vz (f32), rung (i8)
//                                     out: the permuted arrays, then pbegin/pend per
//                                     cell keyed (z*C + y)*C + x (i32)
//   ref_cpu cloud4 <in> <out>         in: m, x[m] (f64)      out: cloud4(x) (f64)
//   ref_cpu laplacian <N> <rs> <type> <in> <out>
//                                     in/out: N*N*(N/2+1) complex<float> (re, im)
//   ref_cpu fixed <in> <out>          in: m, x[m] (f64), a[m], b[m] (u32)
//                                     out: fixed32(x).raw (u32), to_float(a) (f32),
//                                     to_double(a) (f64), distance(a, b) (f32)
//                                     (tigerpm/fixed.hpp, tigerpm/gravity_short.hpp:20-22)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <future>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace hpx {
using id_type = int;
template <class T>
using future = std::future<T>;
namespace thread {
inline unsigned hardware_concurrency() { return 4; }
}  // namespace thread
template <class F, class... Args>
auto async(F&& f, Args&&... args) {
  return std::async(std::launch::deferred, std::forward<F>(f), std::forward<Args>(args)...);
}
// remote actions: only reached through hpx_children(), which is empty here
template <class Action, class... Args>
std::future<void> async(id_type, Args&&...) {
  std::promise<void> p;
  p.set_value();
  return p.get_future();
}
template <class It>
void wait_all(It b, It e) {
  for (; b != e; ++b) b->get();
}
}  // namespace hpx

#include <tigerpm/tigerpm.hpp>
#include <tigerpm/complex.hpp>
#include <tigerpm/fixed.hpp>
#include <tigerpm/range.hpp>
#include <tigerpm/options.hpp>
#include <tigerpm/particles.hpp>
#include <tigerpm/chainmesh.hpp>
#include <tigerpm/gravity_long.hpp>
#include <tigerpm/hpx.hpp>
#include <tigerpm/util.hpp>
#include <tigerpm/gravity_short.hpp>

using mutex_type = std::mutex;
using spinlock_type = std::mutex;

// ---- globals the extracted code refers to
array<vector<fixed32>, NDIM> particles_X;
array<vector<float>, NDIM> particles_U;
vector<char> particles_R;
vector<float> particles_P;
array<vector<float>, NDIM> particles_G;
static auto& X = particles_X;
static auto& U = particles_U;
static auto& R = particles_R;

static options g_opts;
const options& get_options() { return g_opts; }
int particles_size() { return (int)X[0].size(); }
const vector<hpx::id_type>& hpx_children() {
  static vector<hpx::id_type> none;
  return none;
}

struct key_hash {
  size_t operator()(const array<int, NDIM>& k) const {
    return (size_t)k[0] * 73856093u ^ (size_t)k[1] * 19349663u ^ (size_t)k[2] * 83492791u;
  }
};
struct key_eq {
  bool operator()(const array<int, NDIM>& a, const array<int, NDIM>& b) const {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
  }
};
static std::unordered_map<array<int, NDIM>, chaincell, key_hash, key_eq> cells;
static mutex_type mutex;

static range<int> g_crange;
static vector<cmplx> g_Y;
range<int> fft3d_complex_range() { return g_crange; }
vector<cmplx>& fft3d_complex_vector() { return g_Y; }
struct apply_laplacian_action {};

#include "particles_sort.inc"
#include "chainmesh_sort.inc"
#include "cloud4.inc"
#include "apply_laplacian.inc"

// initial conditions (src/initialize.cpp): the reader opens "power.init" in
// the working directory
#include <cmath>
#include <limits>
#include "power_spectrum.inc"
#include "growth_factor.inc"
#include "read_power_spectrum.inc"

static std::vector<char> slurp(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) {
    perror(path);
    exit(2);
  }
  std::vector<char> buf;
  char tmp[1 << 16];
  size_t k;
  while ((k = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
  fclose(f);
  return buf;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string mode = argv[1];
  if (mode == "sort" && argc == 5) {
    const int C = atoi(argv[2]);
    const auto in = slurp(argv[3]);
    int64_t n;
    memcpy(&n, in.data(), 8);
    const char* p = in.data() + 8;
    for (int d = 0; d < NDIM; d++) {
      X[d].resize(n);
      memcpy((void*)X[d].data(), p, 4 * n);
      p += 4 * n;
    }
    for (int d = 0; d < NDIM; d++) {
      U[d].resize(n);
      memcpy(U[d].data(), p, 4 * n);
      p += 4 * n;
    }
    R.resize(n);
    memcpy(R.data(), p, n);
    g_opts.chain_dim = C;
    range<int> box;
    for (int d = 0; d < NDIM; d++) {
      box.begin[d] = 0;
      box.end[d] = C;
    }
    sort(box, 0, (int)n);
    FILE* f = fopen(argv[4], "wb");
    for (int d = 0; d < NDIM; d++) fwrite(X[d].data(), 4, n, f);
    for (int d = 0; d < NDIM; d++) fwrite(U[d].data(), 4, n, f);
    fwrite(R.data(), 1, n, f);
    for (int z = 0; z < C; z++)
      for (int y = 0; y < C; y++)
        for (int x = 0; x < C; x++) {
          array<int, NDIM> k;
          k[0] = x;
          k[1] = y;
          k[2] = z;
          const auto it = cells.find(k);
          int32_t be[2] = {-1, -1};
          if (it != cells.end()) {
            be[0] = it->second.pbegin;
            be[1] = it->second.pend;
          }
          fwrite(be, 4, 2, f);
        }
    fclose(f);
    return 0;
  }
  if (mode == "cloud4" && argc == 4) {
    const auto in = slurp(argv[2]);
    int64_t m;
    memcpy(&m, in.data(), 8);
    std::vector<double> x(m), y(m);
    memcpy(x.data(), in.data() + 8, 8 * m);
    for (int64_t i = 0; i < m; i++) y[i] = cloud4(x[i]);
    FILE* f = fopen(argv[3], "wb");
    fwrite(y.data(), 8, m, f);
    fclose(f);
    return 0;
  }
  if (mode == "laplacian" && argc == 7) {
    const int N = atoi(argv[2]);
    const double rs_cells = atof(argv[3]);
    const int type = atoi(argv[4]);
    g_opts.four_dim = N;
    g_opts.rs = rs_cells / N;
    for (int d = 0; d < NDIM; d++) {
      g_crange.begin[d] = 0;
      g_crange.end[d] = N;
    }
    g_crange.end[ZDIM] = N / 2 + 1;
    const auto in = slurp(argv[5]);
    const size_t cnt = (size_t)N * N * (N / 2 + 1);
    g_Y.resize(cnt);
    memcpy((void*)g_Y.data(), in.data(), 8 * cnt);
    apply_laplacian(type);
    FILE* f = fopen(argv[6], "wb");
    fwrite(g_Y.data(), 8, cnt, f);
    fclose(f);
    return 0;
  }
  if (mode == "power" && argc == 6) {
    // power <hubble> <sigma8> <in> <out>; power.init in the working directory
    // in: m, k[m] (f64, 1/Mpc), then q, (omega_m, a)[q] (f64)
    // out: P(k)[m] (f32 as f64), growth_factor[q] (f64)
    g_opts.hubble = atof(argv[2]);
    g_opts.sigma8 = atof(argv[3]);
    const auto in = slurp(argv[4]);
    const int64_t m = *(const int64_t*)in.data();
    const double* k = (const double*)(in.data() + 8);
    const int64_t q = *(const int64_t*)(in.data() + 8 + 8 * m);
    const double* oa = (const double*)(in.data() + 16 + 8 * m);
    const power_spectrum_function func = read_power_spectrum();
    std::vector<double> out(m + q);
    for (int64_t i = 0; i < m; i++) out[i] = func((float)k[i]);
    for (int64_t i = 0; i < q; i++) out[m + i] = growth_factor(oa[2 * i], (float)oa[2 * i + 1]);
    FILE* f = fopen(argv[5], "wb");
    fwrite(out.data(), 8, m + q, f);
    fclose(f);
    return 0;
  }
  if (mode == "fixed" && argc == 4) {
    const auto in = slurp(argv[2]);
    int64_t m;
    memcpy(&m, in.data(), 8);
    std::vector<double> x(m);
    std::vector<uint32_t> a(m), b(m);
    memcpy(x.data(), in.data() + 8, 8 * m);
    memcpy(a.data(), in.data() + 8 + 8 * m, 4 * m);
    memcpy(b.data(), in.data() + 8 + 12 * m, 4 * m);
    std::vector<uint32_t> raw(m);
    std::vector<float> tf(m), dist(m);
    std::vector<double> td(m);
    for (int64_t i = 0; i < m; i++) {
      fixed32 f(x[i]);
      raw[i] = f.raw();
      fixed32 fa, fb;
      memcpy((void*)&fa, &a[i], 4);
      memcpy((void*)&fb, &b[i], 4);
      tf[i] = fa.to_float();
      td[i] = fa.to_double();
      dist[i] = distance(fa, fb);
    }
    FILE* f = fopen(argv[3], "wb");
    fwrite(raw.data(), 4, m, f);
    fwrite(tf.data(), 4, m, f);
    fwrite(td.data(), 8, m, f);
    fwrite(dist.data(), 4, m, f);
    fclose(f);
    return 0;
  }
  fprintf(stderr, "bad arguments\n");
  return 2;
}
