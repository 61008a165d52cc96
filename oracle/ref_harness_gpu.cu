// ref_harness_gpu.cu -- TEST INFRASTRUCTURE: runs the reference's own GPU
// code -- kick_pme (src/kick_pme.cu, whole file: host staging + kernel) and
// gravity_short_ewald_call_kernel (src/gravity_short.cu, whole file) --
// compiled from the reference tree by oracle/build_ref.sh and linked with
// this file.
//
// This file supplies the symbols those two files use from the rest of the
// reference, restated for one rank with the inputs read from a file:
//   rung_dt (src/fmmpm.cu:18)               2^-r, set before each kick
//   chainmesh_get (src/chainmesh.cpp:48)     the given cell table; ghost
//                                            coordinates wrap periodically
//                                            (the ghost cells of
//                                            chainmesh_exchange hold copies
//                                            of the same particles)
//   gravity_long_get_phi (gravity_long.cpp:23) the given periodic potential
//   get_options, particle globals, cuda_*     plain values
// cuda_free_mem reports at most 4 GiB: the reference's Ewald host code
// converts 85% of free memory / 12 to int (src/gravity_short.cu:41), which
// overflows on a 180 GB device.
//
// usage:  ref_gpu kick <in> <out>     ref_gpu ewald <in> <out>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <tigerpm/tigerpm.hpp>
#include <tigerpm/chainmesh.hpp>
#include <tigerpm/fixed.hpp>
#include <tigerpm/gravity_long.hpp>
#include <tigerpm/gravity_short.hpp>
#include <tigerpm/kick_pme.hpp>
#include <tigerpm/options.hpp>
#include <tigerpm/particles.hpp>
#include <tigerpm/range.hpp>

__constant__ float rung_dt[MAX_RUNG];

array<vector<fixed32>, NDIM> particles_X;
array<vector<float>, NDIM> particles_U;
vector<char> particles_R;
vector<float> particles_P;
array<vector<float>, NDIM> particles_G;

static options g_opts;
static int g_C = 0, g_N = 0;
static std::vector<int32_t> g_cells;  // pbegin, pend per cell
static std::vector<float> g_phi;

const options& get_options() { return g_opts; }
int particles_size() { return (int)particles_X[0].size(); }
void cuda_set_device() { cudaSetDevice(0); }
size_t cuda_free_mem() {
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  const size_t cap = (size_t)4 << 30;
  return fr < cap ? fr : cap;
}
int cuda_smp_count() {
  int c = 0;
  cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, 0);
  return c;
}

static int wrap(int i, int n) {
  const int r = i % n;
  return r < 0 ? r + n : r;
}

chaincell chainmesh_get(const array<int, NDIM>& i) {
  const int C = g_C;
  const int64_t key = ((int64_t)wrap(i[2], C) * C + wrap(i[1], C)) * C + wrap(i[0], C);
  chaincell c;
  c.pbegin = g_cells[2 * key];
  c.pend = g_cells[2 * key + 1];
  return c;
}

vector<float> gravity_long_get_phi(const range<int>& b) {
  vector<float> out(b.volume());
  array<int, NDIM> i;
  const int N = g_N;
  for (i[0] = b.begin[0]; i[0] != b.end[0]; i[0]++)
    for (i[1] = b.begin[1]; i[1] != b.end[1]; i[1]++)
      for (i[2] = b.begin[2]; i[2] != b.end[2]; i[2]++)
        out[b.index(i)] = g_phi[((size_t)wrap(i[0], N) * N + wrap(i[1], N)) * N + wrap(i[2], N)];
  return out;
}

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

template <class T>
static T take(const char*& p) {
  T v;
  memcpy(&v, p, sizeof(T));
  p += sizeof(T);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  const std::string mode = argv[1];
  const auto in = slurp(argv[2]);
  const char* p = in.data();
  if (mode == "kick") {
    const int64_t n = take<int64_t>(p);
    g_C = take<int32_t>(p);
    g_N = take<int32_t>(p);
    g_opts.four_o_chain = take<int32_t>(p);
    g_opts.rs = take<double>(p);
    g_opts.GM = take<double>(p);
    g_opts.eta = take<double>(p);
    g_opts.hsoft = take<double>(p);
    const int min_rung = take<int32_t>(p);
    const double scale = take<double>(p);
    const double t0 = take<double>(p);
    const int first_call = take<int32_t>(p);
    g_opts.four_dim = g_N;
    g_opts.chain_dim = g_C;
    for (int d = 0; d < NDIM; d++) {
      particles_X[d].resize(n);
      memcpy((void*)particles_X[d].data(), p, 4 * n);
      p += 4 * n;
    }
    for (int d = 0; d < NDIM; d++) {
      particles_U[d].resize(n);
      memcpy(particles_U[d].data(), p, 4 * n);
      p += 4 * n;
      particles_G[d].assign(n, 0.f);
    }
    particles_R.resize(n);
    memcpy(particles_R.data(), p, n);
    p += n;
    particles_P.assign(n, 0.f);
    const int64_t ncell = (int64_t)g_C * g_C * g_C;
    g_cells.resize(2 * ncell);
    memcpy(g_cells.data(), p, 8 * ncell);
    p += 8 * ncell;
    g_phi.resize((size_t)g_N * g_N * g_N);
    memcpy(g_phi.data(), p, 4 * g_phi.size());
    float rdt[MAX_RUNG];
    for (int r = 0; r < MAX_RUNG; r++) rdt[r] = (float)(1.0 / (double)(1ull << r));
    cudaMemcpyToSymbol(rung_dt, rdt, sizeof(rdt));
    range<int> box;
    for (int d = 0; d < NDIM; d++) {
      box.begin[d] = 0;
      box.end[d] = g_C;
    }
    kick_pme(box, min_rung, scale, t0, first_call != 0);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      fprintf(stderr, "CUDA: %s\n", cudaGetErrorString(e));
      return 3;
    }
    FILE* f = fopen(argv[3], "wb");
    for (int d = 0; d < NDIM; d++) fwrite(particles_U[d].data(), 4, n, f);
    fwrite(particles_R.data(), 1, n, f);
    for (int d = 0; d < NDIM; d++) fwrite(particles_G[d].data(), 4, n, f);
    fwrite(particles_P.data(), 4, n, f);
    fclose(f);
    return 0;
  }
  if (mode == "ewald") {
    const int64_t n = take<int64_t>(p);
    const int64_t ns = take<int64_t>(p);
    g_opts.hsoft = take<double>(p);
    for (int d = 0; d < NDIM; d++) {
      particles_X[d].resize(n);
      memcpy((void*)particles_X[d].data(), p, 4 * n);
      p += 4 * n;
    }
    vector<fixed32> s[NDIM];
    for (int d = 0; d < NDIM; d++) {
      s[d].resize(ns);
      memcpy((void*)s[d].data(), p, 4 * ns);
      p += 4 * ns;
    }
    const auto rc = gravity_short_ewald_call_kernel(s[0], s[1], s[2]);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      fprintf(stderr, "CUDA: %s\n", cudaGetErrorString(e));
      return 3;
    }
    FILE* f = fopen(argv[3], "wb");
    fwrite(rc.first.data(), 8, ns, f);
    for (int d = 0; d < NDIM; d++) fwrite(rc.second[d].data(), 8, ns, f);
    fclose(f);
    return 0;
  }
  return 2;
}
