// tpm_oracle.cpp -- CPU restatement of TigerPM's PME kick path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA product is
// checked against, and the CPU baseline that bench.py times beside it.  Nothing
// in the product (tigerpm_b200/) links, loads or calls it; only tests/,
// __graft_entry__.smoke() and bench.py's CPU legs do.
//
// Every function restates one piece of the reference algorithm and cites the
// reference file:line it follows (paths relative to the dmarce1/tigerpm tree).
// Arithmetic follows the reference where the reference is exact (integer and
// fixed-point work: bit-exact), and follows its formulas in the stated
// precision where it is floating point.
//
// Build: oracle/Makefile  (g++ -O2 -fopenmp -ffp-contract=off -shared).
// -ffp-contract=off keeps every a*b+c as two roundings, so the explicit fmaf()
// calls below are the only fused operations, as in the reference source.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

constexpr double kTwo32 = 4294967296.0;
constexpr float kFixed2Float = 1.0f / 4294967296.0f;  // tigerpm/fixed.hpp:26,32
constexpr int kMaxRung = 32;                            // tigerpm/tigerpm.hpp:34
constexpr int kNInterp = 6;                             // tigerpm/tigerpm.hpp:35
constexpr float kSelfPhi = float(-35.0 / 16.0);         // tigerpm/tigerpm.hpp:23

// fixed<uint32_t>::operator=(double) / fixed(double): i = c0 * number, c0 the
// float 2^32 promoted to double, truncated to uint32 (tigerpm/fixed.hpp:63-75).
inline uint32_t fixed_from_double(double x) { return (uint32_t)(kTwo32 * x); }

// fixed::to_float(): float(i) * 2^-32 (tigerpm/fixed.hpp:115-118).
inline float fixed_to_float(uint32_t i) { return (float)i * kFixed2Float; }

// fixed::to_double(): i * 2^-32, exact (tigerpm/fixed.hpp:126-129).
inline double fixed_to_double(uint32_t i) { return (double)i * (1.0 / kTwo32); }

// distance(a, b) = (fixed<int32>(a) - fixed<int32>(b)).to_float(): the int32
// wrap-around difference is the periodic minimum image
// (tigerpm/gravity_short.hpp:20-22).
inline float distance32(uint32_t a, uint32_t b) {
  const int32_t d = (int32_t)(a - b);
  return (float)d * kFixed2Float;
}
inline double distance64(uint32_t a, uint32_t b) {
  const int32_t d = (int32_t)(a - b);
  return (double)d * (1.0 / kTwo32);
}

// sqr(a, b, c) = fmaf(a, a, fmaf(b, b, c*c)) (tigerpm/util.hpp:27-30).
inline float sqr3(float a, float b, float c) { return fmaf(a, a, fmaf(b, b, c * c)); }

// erfcexp: Abramowitz & Stegun 7.1.26 erfc with exp(-x^2) returned as well
// (tigerpm/util.hpp:36-59).
inline float erfcexp(float x, float* e) {
  const float p(0.3275911f);
  const float a1(0.254829592f);
  const float a2(-0.284496736f);
  const float a3(1.421413741f);
  const float a4(-1.453152027f);
  const float a5(1.061405429f);
  const float t1 = 1.f / fmaf(p, x, 1.f);
  const float t2 = t1 * t1;
  const float t3 = t2 * t1;
  const float t4 = t2 * t2;
  const float t5 = t2 * t3;
  *e = expf(-x * x);
  return fmaf(a1, t1, fmaf(a2, t2, fmaf(a3, t3, fmaf(a4, t4, a5 * t5)))) * *e;
}

// rung_dt[r] = 2^-r as float (src/fmmpm.cu:18).
inline float rung_dt(int r) { return (float)(1.0 / (double)(1ull << r)); }

inline int wrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// ---------------------------------------------------------------- chain mesh

struct PartArrays {
  uint32_t* X[3];
  float* U[3];
  int8_t* R;
};

// particles_sort: in-place two-pointer partition by x[xdim] >= fixed32(xm),
// swapping X[3], U[3] and R only (src/particles.cpp:414-444).
int partition(PartArrays& p, int begin, int end, double xm, int xdim) {
  int lo = begin;
  int hi = end;
  const uint32_t xmid = fixed_from_double(xm);
  uint32_t* xd = p.X[xdim];
  while (lo < hi) {
    if (xd[lo] >= xmid) {
      while (lo != hi) {
        hi--;
        if (xd[hi] < xmid) {
          for (int d = 0; d < 3; d++) {
            std::swap(p.X[d][hi], p.X[d][lo]);
            std::swap(p.U[d][hi], p.U[d][lo]);
          }
          std::swap(p.R[hi], p.R[lo]);
          break;
        }
      }
    }
    lo++;
  }
  return hi;
}

struct Box {
  int b[3];
  int e[3];
};

// chainmesh sort(): recursive bisection of the chain box.  The split dim is
// the LAST dim whose span exceeds 1, mid = begin + span/2, threshold
// mid * (1.0/N) (src/chainmesh.cpp:168-213).  Leaves record {pbegin, pend}
// for the cell box.begin; cells are keyed here as (z*C + y)*C + x.
void cm_sort(PartArrays& p, int C, double Cinv, Box box, int pbegin, int pend, int32_t* cbeg,
             int32_t* cend, int task_parts) {
  int vol = 1;
  for (int d = 0; d < 3; d++) vol *= box.e[d] - box.b[d];
  if (vol == 1) {
    const int64_t key = ((int64_t)box.b[2] * C + box.b[1]) * C + box.b[0];
    cbeg[key] = pbegin;
    cend[key] = pend;
    return;
  }
  int long_dim = 0;
  int long_span = -1;
  for (int d = 0; d < 3; d++) {
    const int span = box.e[d] - box.b[d];
    if (span > 1) {
      long_span = span;
      long_dim = d;
    }
  }
  const int mid_box = box.b[long_dim] + long_span / 2;
  const double mid_x = mid_box * Cinv;
  Box left = box, right = box;
  left.e[long_dim] = right.b[long_dim] = mid_box;
  const int pmid = partition(p, pbegin, pend, mid_x, long_dim);
  if (pend - pbegin > task_parts) {
#pragma omp task default(shared) firstprivate(left, pbegin, pmid)
    cm_sort(p, C, Cinv, left, pbegin, pmid, cbeg, cend, task_parts);
    cm_sort(p, C, Cinv, right, pmid, pend, cbeg, cend, task_parts);
#pragma omp taskwait
  } else {
    cm_sort(p, C, Cinv, left, pbegin, pmid, cbeg, cend, task_parts);
    cm_sort(p, C, Cinv, right, pmid, pend, cbeg, cend, task_parts);
  }
}

// ---------------------------------------------------------------- deposit

// cloud4: cubic B-spline with the reference's 0.16666667 constant
// (src/gravity_long.cpp:127-138).
inline double cloud4(double x) {
  const double q1 = std::abs(x);
  const double q2 = q1 * q1;
  const double q3 = q2 * q1;
  if (q1 < 1.0) {
    return 0.16666667 * (4.0 - 6.0 * q2 + 3.0 * q3);
  } else if (q1 < 2.0) {
    return 0.16666667 * (8.0 - 12.0 * q1 + 6.0 * q2 - q3);
  } else {
    return 0.0;
  }
}

// Per-dimension assignment weights on a vertex-centred grid.  Returns the
// first (unwrapped) grid index; fills W weights.
//   assign 0 = cloud4, the reference scheme: I = int(X*N + PHI_BW - 1) - PHI_BW,
//              w[i] = cloud4(X*N - I - i), i = 0..3 (src/gravity_long.cpp:176-181)
//   assign 1 = CIC (extension): I = floor(XN), {1-f, f}
//   assign 2 = TSC (extension): I0 = floor(XN + 1/2), d = XN - I0,
//              {(1/2 - d)^2 / 2, 3/4 - d^2, (1/2 + d)^2 / 2} at I0-1, I0, I0+1
inline int assign_weights(int assign, double XN, double* w) {
  if (assign == 0) {
    const int I = int(XN + 3 - 1) - 3;
    for (int i = 0; i < 4; i++) w[i] = cloud4(XN - I - i);
    return I;
  } else if (assign == 1) {
    const int I = (int)XN;
    const double f = XN - I;
    w[0] = 1.0 - f;
    w[1] = f;
    return I;
  } else {
    const int I0 = (int)(XN + 0.5);
    const double d = XN - I0;
    w[0] = 0.5 * (0.5 - d) * (0.5 - d);
    w[1] = 0.75 - d * d;
    w[2] = 0.5 * (0.5 + d) * (0.5 + d);
    return I0 - 1;
  }
}

inline int assign_width(int assign) { return assign == 0 ? 4 : (assign == 1 ? 2 : 3); }

// ---------------------------------------------------------------- FFT (own)

using cd = std::complex<double>;

struct Fft1D {
  int n = 0;
  bool pow2 = true;
  std::vector<cd> tw;  // radix-2 twiddles e^{-2 pi i k / n}, k < n/2
  // Bluestein
  int m = 0;
  std::vector<cd> chirp;   // e^{-pi i k^2 / n}
  std::vector<cd> bfft;    // FFT_m of conj(chirp) arranged circularly
  std::vector<cd> tw_m;    // radix-2 twiddles for size m

  static void make_tw(int n, std::vector<cd>& tw) {
    tw.resize(n / 2 > 0 ? n / 2 : 1);
    for (int k = 0; k < n / 2; k++) {
      const double a = -2.0 * M_PI * k / n;
      tw[k] = cd(std::cos(a), std::sin(a));
    }
  }

  // In-place iterative radix-2; sign -1 forward, +1 backward; unnormalised.
  static void radix2(cd* a, int n, const std::vector<cd>& tw, int sign) {
    for (int i = 1, j = 0; i < n; i++) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1;
      const int step = n / len;
      for (int i = 0; i < n; i += len) {
        for (int k = 0; k < half; k++) {
          cd w = tw[k * step];
          if (sign > 0) w = std::conj(w);
          const cd u = a[i + k];
          const cd v = a[i + k + half] * w;
          a[i + k] = u + v;
          a[i + k + half] = u - v;
        }
      }
    }
  }

  // n = p * 2^k with p in {3, 5}: one radix-p stage over p power-of-two
  // transforms (direct, no Bluestein).
  int radix = 1;
  int sub = 0;
  std::vector<cd> tw_sub, tw_n;

  void init(int n_) {
    n = n_;
    pow2 = (n & (n - 1)) == 0;
    if (pow2) {
      make_tw(n, tw);
      return;
    }
    for (int p : {3, 5}) {
      if (n % p == 0) {
        const int q = n / p;
        if ((q & (q - 1)) == 0) {
          radix = p;
          sub = q;
          make_tw(q, tw_sub);
          tw_n.resize(n);
          for (int k = 0; k < n; k++) {
            const double a = -2.0 * M_PI * k / n;
            tw_n[k] = cd(std::cos(a), std::sin(a));
          }
          return;
        }
      }
    }
    m = 1;
    while (m < 2 * n - 1) m <<= 1;
    make_tw(m, tw_m);
    chirp.resize(n);
    for (int k = 0; k < n; k++) {
      const long long k2 = ((long long)k * k) % (2LL * n);
      const double a = -M_PI * (double)k2 / n;
      chirp[k] = cd(std::cos(a), std::sin(a));
    }
    bfft.assign(m, cd(0, 0));
    bfft[0] = std::conj(chirp[0]);
    for (int k = 1; k < n; k++) {
      bfft[k] = std::conj(chirp[k]);
      bfft[m - k] = std::conj(chirp[k]);
    }
    radix2(bfft.data(), m, tw_m, -1);
  }

  // scratch must hold m entries for Bluestein.
  void exec(cd* a, int sign, std::vector<cd>& scratch) const {
    if (pow2) {
      radix2(a, n, tw, sign);
      return;
    }
    if (radix > 1) {
      // X[k] = sum_r W_n^{r k} F_r[k mod q], F_r = FFT_q of a[p j + r]
      const int p = radix, q = sub;
      scratch.resize(n);
      for (int r = 0; r < p; r++) {
        cd* f = scratch.data() + r * q;
        for (int j = 0; j < q; j++) f[j] = a[p * j + r];
        radix2(f, q, tw_sub, sign);
      }
      for (int k = 0; k < n; k++) {
        cd acc = scratch[k % q];
        for (int r = 1; r < p; r++) {
          cd w = tw_n[(int)(((long long)r * k) % n)];
          if (sign > 0) w = std::conj(w);
          acc += w * scratch[r * q + k % q];
        }
        a[k] = acc;
      }
      return;
    }
    // Backward transform = conj(forward(conj(a))).
    scratch.assign(m, cd(0, 0));
    for (int k = 0; k < n; k++) {
      const cd x = sign > 0 ? std::conj(a[k]) : a[k];
      scratch[k] = x * chirp[k];
    }
    radix2(scratch.data(), m, tw_m, -1);
    for (int k = 0; k < m; k++) scratch[k] *= bfft[k];
    radix2(scratch.data(), m, tw_m, +1);
    const double inv = 1.0 / m;
    for (int k = 0; k < n; k++) {
      cd y = scratch[k] * inv * chirp[k];
      a[k] = sign > 0 ? std::conj(y) : y;
    }
  }
};

// Unnormalised forward r2c of a real N^3 array (x-major, z fastest) into the
// N x N x (N/2+1) half spectrum -- the layout fft3d_execute leaves behind
// (src/fft.cpp:51-67, 423-458; complex box end[z] = N/2+1, src/fft.cpp:391).
void fft3d_r2c(int N, const double* in, cd* out) {
  const int Nh = N / 2 + 1;
  Fft1D plan;
  plan.init(N);
#pragma omp parallel
  {
    std::vector<cd> line(N), scratch;
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * N; l++) {
      for (int z = 0; z < N; z++) line[z] = cd(in[l * N + z], 0.0);
      plan.exec(line.data(), -1, scratch);
      for (int z = 0; z < Nh; z++) out[l * Nh + z] = line[z];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * Nh; l++) {
      const int64_t x = l / Nh, kz = l % Nh;
      for (int y = 0; y < N; y++) line[y] = out[(x * N + y) * Nh + kz];
      plan.exec(line.data(), -1, scratch);
      for (int y = 0; y < N; y++) out[(x * N + y) * Nh + kz] = line[y];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * Nh; l++) {
      const int64_t y = l / Nh, kz = l % Nh;
      for (int x = 0; x < N; x++) line[x] = out[((int64_t)x * N + y) * Nh + kz];
      plan.exec(line.data(), -1, scratch);
      for (int x = 0; x < N; x++) out[((int64_t)x * N + y) * Nh + kz] = line[x];
    }
  }
}

// Inverse c2r with the reference's 1/N per pass, 1/N^3 overall
// (src/fft.cpp:69-84, 468, 512).  Destroys `in`.
void fft3d_c2r(int N, cd* in, double* out) {
  const int Nh = N / 2 + 1;
  Fft1D plan;
  plan.init(N);
  const double inv = 1.0 / ((double)N * N * N);
#pragma omp parallel
  {
    std::vector<cd> line(N), scratch;
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * Nh; l++) {
      const int64_t y = l / Nh, kz = l % Nh;
      for (int x = 0; x < N; x++) line[x] = in[((int64_t)x * N + y) * Nh + kz];
      plan.exec(line.data(), +1, scratch);
      for (int x = 0; x < N; x++) in[((int64_t)x * N + y) * Nh + kz] = line[x];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * Nh; l++) {
      const int64_t x = l / Nh, kz = l % Nh;
      for (int y = 0; y < N; y++) line[y] = in[(x * N + y) * Nh + kz];
      plan.exec(line.data(), +1, scratch);
      for (int y = 0; y < N; y++) in[(x * N + y) * Nh + kz] = line[y];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)N * N; l++) {
      for (int z = 0; z < Nh; z++) line[z] = in[l * Nh + z];
      for (int z = Nh; z < N; z++) line[z] = std::conj(in[l * Nh + (N - z)]);
      plan.exec(line.data(), +1, scratch);
      for (int z = 0; z < N; z++) out[l * N + z] = line[z].real() * inv;
    }
  }
}

inline double sinc(double x) { return x != 0.0 ? std::sin(x) / x : 1.0; }  // tigerpm/util.hpp:91-97

// apply_laplacian: Y *= (-1/k^2) * exp(-k^2 rs^2) [PME] * sinc(k/2)^-p,
// k = 2 pi i / N in grid units, i >= N/2 folded negative, k = 0 -> 0
// (src/gravity_long.cpp:201-245; the reference has p = 4).
void green_apply(int N, double rs_cells, int pme, int p, cd* Y) {
  const int Nh = N / 2 + 1;
  const double c0 = 2.0 * M_PI / N;
  const double rs2 = rs_cells * rs_cells;
  const double Nd = N;
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < (int64_t)N * N; l++) {
    const int i0 = (int)(l / N), i1 = (int)(l % N);
    const double kx = (i0 < Nd / 2 ? i0 : i0 - N) * c0;
    const double ky = (i1 < Nd / 2 ? i1 : i1 - N) * c0;
    for (int i2 = 0; i2 < Nh; i2++) {
      const double kz = (i2 < Nd / 2 ? i2 : i2 - N) * c0;
      const double nk2 = -(kx * kx + ky * ky + kz * kz);
      double f = nk2 < 0.0 ? 1.0 / nk2 : 0.0;
      if (pme) f *= std::exp(nk2 * rs2);
      const double s = sinc(0.5 * kx) * sinc(0.5 * ky) * sinc(0.5 * kz);
      f *= std::pow(s, -p);
      Y[l * Nh + i2] *= f;
    }
  }
}

// 6-point quintic interpolation weights and their derivatives
// (src/kick_pme.cu:208-231).
template <class T>
inline void q6_weights(T x1, T* w, T* dw) {
  T x2 = x1 * x1;
  T x3 = x1 * x2;
  T x4 = x2 * x2;
  T x5 = x3 * x2;
  const T c1_12 = T(1) / T(12), c1_24 = T(1) / T(24), c3_8 = T(3) / T(8), c13_24 = T(13) / T(24),
          c5_24 = T(5) / T(24), c2_3 = T(2) / T(3), c13_8 = T(13) / T(8), c8_3 = T(8) / T(3),
          c25_24 = T(25) / T(24), c5_4 = T(5) / T(4), c35_12 = T(35) / T(12), c21_4 = T(21) / T(4),
          c25_12 = T(25) / T(12), c11_4 = T(11) / T(4), c31_6 = T(31) / T(6), c11_8 = T(11) / T(8),
          c61_24 = T(61) / T(24), c7_24 = T(7) / T(24), c1_2 = T(0.5);
  w[0] = c1_12 * x1 - c1_24 * x2 - c3_8 * x3 + c13_24 * x4 - c5_24 * x5;
  w[1] = -c2_3 * x1 + c2_3 * x2 + c13_8 * x3 - c8_3 * x4 + c25_24 * x5;
  w[2] = T(1) - c5_4 * x2 - c35_12 * x3 + c21_4 * x4 - c25_12 * x5;
  w[3] = c2_3 * x1 + c2_3 * x2 + c11_4 * x3 - c31_6 * x4 + c25_12 * x5;
  w[4] = -c1_12 * x1 - c1_24 * x2 - c11_8 * x3 + c61_24 * x4 - c25_24 * x5;
  w[5] = c7_24 * x3 - c1_2 * x4 + c5_24 * x5;
  x5 = T(5) * x4;
  x4 = T(4) * x3;
  x3 = T(3) * x2;
  x2 = T(2) * x1;
  x1 = T(1);
  dw[0] = c1_12 * x1 - c1_24 * x2 - c3_8 * x3 + c13_24 * x4 - c5_24 * x5;
  dw[1] = -c2_3 * x1 + c2_3 * x2 + c13_8 * x3 - c8_3 * x4 + c25_24 * x5;
  dw[2] = -c5_4 * x2 - c35_12 * x3 + c21_4 * x4 - c25_12 * x5;
  dw[3] = c2_3 * x1 + c2_3 * x2 + c11_4 * x3 - c31_6 * x4 + c25_12 * x5;
  dw[4] = -c1_12 * x1 - c1_24 * x2 - c11_8 * x3 + c61_24 * x4 - c25_24 * x5;
  dw[5] = c7_24 * x3 - c1_2 * x4 + c5_24 * x5;
}

}  // namespace

extern "C" {

// --------------------------------------------------------------- fixed32

uint32_t orc_fixed32_from_double(double x) { return fixed_from_double(x); }
float orc_fixed32_to_float(uint32_t i) { return fixed_to_float(i); }
double orc_fixed32_to_double(uint32_t i) { return fixed_to_double(i); }
float orc_distance(uint32_t a, uint32_t b) { return distance32(a, b); }
float orc_erfcexp(float x, float* e) { return erfcexp(x, e); }

void orc_fixed32_from_double_array(int64_t n, const double* x, uint32_t* out) {
  for (int64_t i = 0; i < n; i++) out[i] = fixed_from_double(x[i]);
}

// Array forms of the conversions and of distance(), for the golden-vector checks.
void orc_fixed32_convert_array(int64_t n, const uint32_t* a, const uint32_t* b, float* to_float,
                               double* to_double, float* dist) {
  for (int64_t i = 0; i < n; i++) {
    to_float[i] = fixed_to_float(a[i]);
    to_double[i] = fixed_to_double(a[i]);
    dist[i] = distance32(a[i], b[i]);
  }
}

// cloud4 (src/gravity_long.cpp:127-138), one value per x.
void orc_cloud4_array(int64_t n, const double* x, double* w) {
  for (int64_t i = 0; i < n; i++) w[i] = cloud4(x[i]);
}

// particles_mesh_loc: i = int(to_double(x) * C) (tigerpm/particles.hpp:60-67).
void orc_mesh_loc(int C, int64_t n, const uint32_t* x, int32_t* loc) {
  const double Cd = C;
  for (int64_t i = 0; i < n; i++) loc[i] = (int32_t)(fixed_to_double(x[i]) * Cd);
}

// chainmesh_create on one rank (src/chainmesh.cpp:139-161): the whole
// [0,C)^3 chain box, partition-sorted in place.  pbegin/pend have C^3
// entries keyed (z*C + y)*C + x.
int orc_chainmesh_sort(int C, int64_t n, uint32_t* x, uint32_t* y, uint32_t* z, float* vx,
                       float* vy, float* vz, int8_t* rung, int32_t* pbegin, int32_t* pend,
                       int nthreads) {
  if (C < 1 || n < 0 || n > 0x7fffffff) return -1;
  PartArrays p{{x, y, z}, {vx, vy, vz}, rung};
  // `static double Ninv = 1.0 / N` (src/chainmesh.cpp:171).
  const double Cinv = 1.0 / C;
  Box box{{0, 0, 0}, {C, C, C}};
  const int64_t ncell = (int64_t)C * C * C;
  for (int64_t k = 0; k < ncell; k++) pbegin[k] = pend[k] = -1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const int task_parts = std::max<int64_t>(1 << 14, n / (8 * nthreads));
#pragma omp parallel num_threads(nthreads)
#pragma omp single
  cm_sort(p, C, Cinv, box, 0, (int)n, pbegin, pend, task_parts);
  return 0;
}

// compute_source (src/gravity_long.cpp:142-199) for one rank: every particle
// deposits W^3 weights * 4 pi N onto the periodic grid (the padded box plus
// fft3d_accumulate_real's periodic fold, src/fft.cpp:260-315, is the same as
// a periodic index).  Accumulates in double, deterministically: each thread
// owns whole x-planes.
int orc_deposit(int N, int assign, int64_t n, const uint32_t* x, const uint32_t* y,
                const uint32_t* z, double* rho, int nthreads) {
  if (N < 4 || assign < 0 || assign > 2) return -1;
  const int W = assign_width(assign);
  const double Nd = N;
  const double c0 = 4.0 * M_PI * Nd;
  const int64_t N3 = (int64_t)N * N * N;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  std::vector<int32_t> p0(n);
  std::vector<int64_t> start(N + 1, 0);
  for (int64_t i = 0; i < n; i++) {
    double w[4];
    const int I = assign_weights(assign, fixed_to_double(x[i]) * Nd, w);
    p0[i] = wrap(I, N);
    start[p0[i] + 1]++;
  }
  for (int p = 0; p < N; p++) start[p + 1] += start[p];
  std::vector<int64_t> order(n);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t i = 0; i < n; i++) order[fill[p0[i]]++] = i;
  }
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int P = 0; P < N; P++) {
    double* plane = rho + (int64_t)P * N * N;
    for (int64_t k = 0; k < (int64_t)N * N; k++) plane[k] = 0.0;
    for (int q = 0; q < W; q++) {
      const int b = wrap(P - q, N);
      for (int64_t o = start[b]; o < start[b + 1]; o++) {
        const int64_t i = order[o];
        double wx[4], wy[4], wz[4];
        assign_weights(assign, fixed_to_double(x[i]) * Nd, wx);
        const int Iy = assign_weights(assign, fixed_to_double(y[i]) * Nd, wy);
        const int Iz = assign_weights(assign, fixed_to_double(z[i]) * Nd, wz);
        for (int jy = 0; jy < W; jy++) {
          const int64_t row = (int64_t)wrap(Iy + jy, N) * N;
          const double wxy = c0 * wx[q] * wy[jy];
          for (int jz = 0; jz < W; jz++) plane[row + wrap(Iz + jz, N)] += wxy * wz[jz];
        }
      }
    }
  }
  (void)N3;
  return 0;
}

// Forward r2c / inverse c2r with the reference's normalisation; `cplx` holds
// interleaved (re, im) doubles, N*N*(N/2+1) of them.
void orc_fft3d_r2c(int N, const double* in, double* cplx) {
  fft3d_r2c(N, in, reinterpret_cast<cd*>(cplx));
}
void orc_fft3d_c2r(int N, double* cplx, double* out) {
  fft3d_c2r(N, reinterpret_cast<cd*>(cplx), out);
}
void orc_green_apply(int N, double rs_cells, int pme, int deconv_order, double* cplx) {
  green_apply(N, rs_cells, pme, deconv_order, reinterpret_cast<cd*>(cplx));
}

// gravity_long_compute (src/gravity_long.cpp:36-48): deposit, forward FFT,
// Green's function, inverse FFT.  phi is the periodic N^3 potential.
int orc_gravity_long(int N, double rs_cells, int pme, int assign, int deconv_order, int64_t n,
                     const uint32_t* x, const uint32_t* y, const uint32_t* z, double* phi,
                     int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int rc = orc_deposit(N, assign, n, x, y, z, phi, nthreads);
  if (rc) return rc;
  std::vector<cd> Y((size_t)N * N * (N / 2 + 1));
  fft3d_r2c(N, phi, Y.data());
  green_apply(N, rs_cells, pme, deconv_order, Y.data());
  fft3d_c2r(N, Y.data(), phi);
  return 0;
}

// ------------------------------------------------------------------- kick

struct orc_kick_params {
  int N;           // four_dim: PM grid points per side
  int C;           // chain_dim
  double rs;       // split scale, box units
  double GM;
  double eta;
  double hsoft;
  double rcut;     // <= 0: no cutoff, all 27 neighbour cells (the reference)
  int min_rung;
  double scale;
  double t0;
  int first_call;
  int precision;   // 0: the reference's FP32 arithmetic; 1: FP64 plain
};

}  // extern "C"

namespace {

template <class T>
struct KickOut {
  T g[3];
  T phi;
};

// Long-range part of kick_pme_kernel (src/kick_pme.cu:188-263): 6x6x6
// quintic interpolation of phi and of its analytic gradient.  Grid index is
// periodic; the reference reads a PHI_BW-padded copy of the same values.
void interp_ref(const orc_kick_params& P, const float* phi_f, const double* phi_d, uint32_t sx,
                uint32_t sy, uint32_t sz, KickOut<float>& o) {
  const int N = P.N;
  int I[3];
  float X[3] = {fixed_to_float(sx), fixed_to_float(sy), fixed_to_float(sz)};
  float w[3][kNInterp], dw[3][kNInterp];
  for (int d = 0; d < 3; d++) {
    X[d] *= N;
    I[d] = std::min(int(X[d]), N);  // phi_box.end - PHI_BW
    X[d] -= float(I[d]);
    I[d] -= 2;
  }
  for (int d = 0; d < 3; d++) q6_weights<float>(X[d], w[d], dw[d]);
  auto phi_at = [&](int a, int b, int c) -> float {
    const int64_t l = ((int64_t)wrap(a, N) * N + wrap(b, N)) * N + wrap(c, N);
    return phi_f ? phi_f[l] : (float)phi_d[l];
  };
  for (int d1 = 0; d1 < 3; d1++) {
    for (int j0 = 0; j0 < kNInterp; j0++)
      for (int j1 = 0; j1 < kNInterp; j1++)
        for (int j2 = 0; j2 < kNInterp; j2++) {
          const int j[3] = {j0, j1, j2};
          double w0 = 1.0;
          for (int d2 = 0; d2 < 3; d2++) w0 *= (d1 == d2) ? dw[d2][j[d2]] : w[d2][j[d2]];
          o.g[d1] -= w0 * phi_at(I[0] + j0, I[1] + j1, I[2] + j2) * N;
        }
  }
  for (int j0 = 0; j0 < kNInterp; j0++)
    for (int j1 = 0; j1 < kNInterp; j1++)
      for (int j2 = 0; j2 < kNInterp; j2++) {
        double w0 = (double)w[0][j0] * w[1][j1] * w[2][j2];
        o.phi += w0 * phi_at(I[0] + j0, I[1] + j1, I[2] + j2);
      }
}

void interp_fp64(const orc_kick_params& P, const float* phi_f, const double* phi_d, uint32_t sx,
                 uint32_t sy, uint32_t sz, KickOut<double>& o) {
  const int N = P.N;
  const uint32_t s[3] = {sx, sy, sz};
  int I[3];
  double w[3][kNInterp], dw[3][kNInterp];
  for (int d = 0; d < 3; d++) {
    const uint64_t t = (uint64_t)s[d] * (uint64_t)N;  // exact cell and fraction
    I[d] = (int)(t >> 32);
    const double f = (double)(uint32_t)t * (1.0 / kTwo32);
    q6_weights<double>(f, w[d], dw[d]);
    I[d] -= 2;
  }
  auto phi_at = [&](int a, int b, int c) -> double {
    const int64_t l = ((int64_t)wrap(a, N) * N + wrap(b, N)) * N + wrap(c, N);
    return phi_d ? phi_d[l] : (double)phi_f[l];
  };
  for (int j0 = 0; j0 < kNInterp; j0++)
    for (int j1 = 0; j1 < kNInterp; j1++)
      for (int j2 = 0; j2 < kNInterp; j2++) {
        const double p = phi_at(I[0] + j0, I[1] + j1, I[2] + j2);
        o.g[0] -= dw[0][j0] * w[1][j1] * w[2][j2] * p * N;
        o.g[1] -= w[0][j0] * dw[1][j1] * w[2][j2] * p * N;
        o.g[2] -= w[0][j0] * w[1][j1] * dw[2][j2] * p * N;
        o.phi += w[0][j0] * w[1][j1] * w[2][j2] * p;
      }
}

// The rung / velocity kick of kick_pme_kernel (src/kick_pme.cu:319-354).
// Returns 1 when the new rung fell outside [0, MAX_RUNG) (the reference
// prints and asserts there); the rung is clamped in that case.
int kick_update(const orc_kick_params& P, float g0, float g1, float g2, float* vx, float* vy,
                float* vz, int8_t* rung) {
  const float t0 = (float)P.t0;
  const float eta = (float)P.eta, scale = (float)P.scale, hsoft = (float)P.hsoft;
  int r = *rung;
  int bad = 0;
  if (r < 0 || r >= kMaxRung) {
    bad = 1;
    r = std::min(std::max(r, 0), kMaxRung - 1);
  }
  float dt = 0.5f * rung_dt(r) * t0;
  if (!P.first_call) {
    *vx = fmaf(g0, dt, *vx);
    *vy = fmaf(g1, dt, *vy);
    *vz = fmaf(g2, dt, *vz);
  }
  const float gg = sqr3(g0, g1, g2);
  const float factor = eta * sqrtf(scale * hsoft);
  dt = fminf(factor * (1.0f / sqrtf(sqrtf(gg))), t0);
  float rn = fmaxf(ceilf(log2f(t0) - log2f(dt)), (float)(r - 1));
  int ri = (int)rn;
  if (ri < 0 || ri >= kMaxRung) {
    bad = 1;
    ri = std::min(std::max(ri, 0), kMaxRung - 1);
  }
  *rung = (int8_t)ri;
  dt = 0.5f * rung_dt(ri) * t0;
  *vx = fmaf(g0, dt, *vx);
  *vy = fmaf(g1, dt, *vy);
  *vz = fmaf(g2, dt, *vz);
  return bad;
}

}  // namespace

extern "C" {

// kick_pme over a chain mesh (src/kick_pme.cu:128-357 with the host staging of
// :390-621 replaced by periodic cell indices).  Sinks are the active
// particles (rung >= min_rung) of the listed sink cells (all cells when
// nsink_cells < 0); sources are every particle of the 27 neighbour cells, in
// the reference's order (x-offset outermost, z innermost; within a cell, the
// chain-mesh order).  Outputs g, pot for kicked sinks; updates v, rung.
// pair_counts[0] = candidate pairs, [1] = pairs inside the cutoff.
int orc_kick_pme(const orc_kick_params* Pp, int64_t n, const uint32_t* x, const uint32_t* y,
                 const uint32_t* z, float* vx, float* vy, float* vz, int8_t* rung,
                 const int32_t* pbegin, const int32_t* pend, const float* phi_f,
                 const double* phi_d, float* gx, float* gy, float* gz, float* pot,
                 const int32_t* sink_cells, int64_t nsink_cells, int64_t* pair_counts,
                 int nthreads) {
  const orc_kick_params P = *Pp;
  const int C = P.C;
  const int64_t ncell = (int64_t)C * C * C;
  if (C < 1 || P.N < 4 || (!phi_f && !phi_d)) return -1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const int64_t ns = nsink_cells < 0 ? ncell : nsink_cells;
  // kernel_params derived constants (src/kick_pme.cu:440-453).
  const float rs_f = (float)P.rs;
  const float inv2rs = 1.0f / rs_f / 2.0f;
  const float twooversqrtpi = 2.0f / sqrtf((float)M_PI);
  const float hs = (float)P.hsoft;
  const float h2 = hs * hs;
  const float hinv = 1.f / hs;
  const float h3inv = hinv * (hinv * hinv);
  const float GM = (float)P.GM;
  const float rcut2f = P.rcut > 0 ? (float)(P.rcut * P.rcut) : INFINITY;
  const double rcut2d = P.rcut > 0 ? P.rcut * P.rcut : INFINITY;
  const double inv2rs_d = 0.5 / P.rs;
  const double h2d = P.hsoft * P.hsoft, hinvd = 1.0 / P.hsoft, h3invd = hinvd * hinvd * hinvd;
  int64_t cand = 0, inside = 0;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(+ : cand, inside, bad)
  for (int64_t si = 0; si < ns; si++) {
    const int64_t key = sink_cells ? sink_cells[si] : si;
    const int cx = (int)(key % C), cy = (int)((key / C) % C), cz = (int)(key / ((int64_t)C * C));
    int32_t nb_b[27], nb_e[27];
    int q = 0;
    for (int a = -1; a <= 1; a++)
      for (int b = -1; b <= 1; b++)
        for (int c = -1; c <= 1; c++) {
          const int64_t k2 = ((int64_t)wrap(cz + c, C) * C + wrap(cy + b, C)) * C + wrap(cx + a, C);
          nb_b[q] = pbegin[k2];
          nb_e[q] = pend[k2];
          q++;
        }
    int64_t nsrc = 0;
    for (int q2 = 0; q2 < 27; q2++) nsrc += nb_e[q2] - nb_b[q2];
    for (int32_t i = pbegin[key]; i < pend[key]; i++) {
      if (rung[i] < P.min_rung) continue;
      cand += nsrc;
      if (P.precision == 0) {
        KickOut<float> o{{0.f, 0.f, 0.f}, 0.f};
        interp_ref(P, phi_f, phi_d, x[i], y[i], z[i], o);
        for (int q2 = 0; q2 < 27; q2++) {
          for (int32_t j = nb_b[q2]; j < nb_e[q2]; j++) {
            const float dx = distance32(x[i], x[j]);
            const float dy = distance32(y[i], y[j]);
            const float dz = distance32(z[i], z[j]);
            const float r2 = sqr3(dx, dy, dz);
            if (r2 >= rcut2f) continue;
            inside++;
            float rinv, rinv3;
            if (r2 > h2) {
              const float r = sqrtf(r2);
              rinv = 1.0f / sqrtf(r2);
              const float r0 = r * inv2rs;
              float exp0;
              const float erfc0 = erfcexp(r0, &exp0);
              rinv3 = (erfc0 + twooversqrtpi * r0 * exp0) * rinv * rinv * rinv;
              rinv *= erfc0;
            } else {
              const float qq = sqrtf(r2) * hinv;
              const float q2s = qq * qq;
              rinv3 = +15.0f / 8.0f;
              rinv3 = fmaf(rinv3, q2s, -21.0f / 4.0f);
              rinv3 = fmaf(rinv3, q2s, +35.0f / 8.0f);
              rinv3 *= h3inv;
              rinv = -5.0f / 16.0f;
              rinv = fmaf(rinv, q2s, 21.0f / 16.0f);
              rinv = fmaf(rinv, q2s, -35.0f / 16.0f);
              rinv = fmaf(rinv, q2s, 35.0f / 16.0f);
              rinv *= hinv;
            }
            o.g[0] -= dx * rinv3;
            o.g[1] -= dy * rinv3;
            o.g[2] -= dz * rinv3;
            o.phi -= rinv;
          }
        }
        for (int d = 0; d < 3; d++) o.g[d] *= GM;
        o.phi *= GM;
        gx[i] = o.g[0];
        gy[i] = o.g[1];
        gz[i] = o.g[2];
        pot[i] = o.phi;
        bad += kick_update(P, o.g[0], o.g[1], o.g[2], &vx[i], &vy[i], &vz[i], &rung[i]);
      } else {
        KickOut<double> o{{0, 0, 0}, 0};
        interp_fp64(P, phi_f, phi_d, x[i], y[i], z[i], o);
        for (int q2 = 0; q2 < 27; q2++) {
          for (int32_t j = nb_b[q2]; j < nb_e[q2]; j++) {
            const double dx = distance64(x[i], x[j]);
            const double dy = distance64(y[i], y[j]);
            const double dz = distance64(z[i], z[j]);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= rcut2d) continue;
            inside++;
            double rinv, rinv3;
            if (r2 > h2d) {
              const double r = std::sqrt(r2);
              rinv = 1.0 / r;
              const double r0 = r * inv2rs_d;
              const double e0 = std::exp(-r0 * r0);
              const double ec = std::erfc(r0);
              rinv3 = (ec + (2.0 / std::sqrt(M_PI)) * r0 * e0) * rinv * rinv * rinv;
              rinv *= ec;
            } else {
              const double q2s = r2 * hinvd * hinvd;
              rinv3 = ((15.0 / 8.0 * q2s - 21.0 / 4.0) * q2s + 35.0 / 8.0) * h3invd;
              rinv = (((-5.0 / 16.0 * q2s + 21.0 / 16.0) * q2s - 35.0 / 16.0) * q2s + 35.0 / 16.0) * hinvd;
            }
            o.g[0] -= dx * rinv3;
            o.g[1] -= dy * rinv3;
            o.g[2] -= dz * rinv3;
            o.phi -= rinv;
          }
        }
        for (int d = 0; d < 3; d++) o.g[d] *= P.GM;
        o.phi *= P.GM;
        gx[i] = (float)o.g[0];
        gy[i] = (float)o.g[1];
        gz[i] = (float)o.g[2];
        pot[i] = (float)o.phi;
        bad += kick_update(P, gx[i], gy[i], gz[i], &vx[i], &vy[i], &vz[i], &rung[i]);
      }
    }
  }
  if (pair_counts) {
    pair_counts[0] = cand;
    pair_counts[1] = inside;
  }
  (void)n;
  return bad;
}

// ------------------------------------------------------------------ Ewald

// gravity_ewald_kernel restated in FP64 throughout (src/gravity_short.cu:93-201):
// alpha = 2 box^-1; real-space images |n_i| <= 4 with r < 2.6; +pi/4 per
// source; reciprocal |h|^2 <= 8; pairs with minimum-image r <= h take the
// softened Newtonian kernel instead; phi starts at -SELF_PHI/h (:31), which
// cancels the sink's own softened term.  Sums over all n sources.
void orc_ewald_ref(int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z,
                   int64_t nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz,
                   double hsoft, double* phi, double* gx, double* gy, double* gz, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const double h2 = hsoft * hsoft, hinv = 1.0 / hsoft, h3inv = hinv * hinv * hinv;
  // reciprocal vectors and coefficients
  struct KV {
    int h[3];
    double c0;
  };
  std::vector<KV> kv;
  for (int a = -2; a <= 2; a++)
    for (int b = -2; b <= 2; b++)
      for (int c = -2; c <= 2; c++) {
        const int hh = a * a + b * b + c * c;
        if (hh > 0 && hh <= 8) {
          KV k{{a, b, c}, -1.0 / hh * std::exp(-M_PI * M_PI * 0.25 * hh) * (1.0 / M_PI)};
          kv.push_back(k);
        }
      }
  for (int64_t s = 0; s < nsink; s++) {
    double P = -(double)kSelfPhi / hsoft, G0 = 0, G1 = 0, G2 = 0;
#pragma omp parallel for num_threads(nthreads) reduction(+ : P, G0, G1, G2) schedule(static)
    for (int64_t j = 0; j < n; j++) {
      const double X = distance64(sx[s], x[j]);
      const double Y = distance64(sy[s], y[j]);
      const double Z = distance64(sz[s], z[j]);
      const double R2 = X * X + Y * Y + Z * Z;
      if (R2 > h2) {
        for (int xi = -4; xi <= 4; xi++)
          for (int yi = -4; yi <= 4; yi++)
            for (int zi = -4; zi <= 4; zi++) {
              const double dx = X - xi, dy = Y - yi, dz = Z - zi;
              const double r2 = dx * dx + dy * dy + dz * dz;
              if (r2 < 2.6 * 2.6) {
                const double r = std::sqrt(r2);
                const double rinv = 1.0 / r;
                const double r3inv = rinv * rinv * rinv;
                const double exp0 = std::exp(-4.0 * r2);
                const double erfc0 = std::erfc(2.0 * r);
                const double expfactor = 4.0 / std::sqrt(M_PI) * r * exp0;
                const double d1 = (expfactor + erfc0) * r3inv;
                P += -erfc0 * rinv;
                G0 -= dx * d1;
                G1 -= dy * d1;
                G2 -= dz * d1;
              }
            }
        P += M_PI / 4.0;
        // e^{2 pi i h.X} from per-axis phases
        std::complex<double> ex[5], ey[5], ez[5];
        for (int t = -2; t <= 2; t++) {
          ex[t + 2] = std::polar(1.0, 2.0 * M_PI * X * t);
          ey[t + 2] = std::polar(1.0, 2.0 * M_PI * Y * t);
          ez[t + 2] = std::polar(1.0, 2.0 * M_PI * Z * t);
        }
        for (const KV& k : kv) {
          const std::complex<double> e = ex[k.h[0] + 2] * ey[k.h[1] + 2] * ez[k.h[2] + 2];
          const double c1 = -e.imag() * 2.0 * M_PI * k.c0;
          P += k.c0 * e.real();
          G0 -= c1 * k.h[0];
          G1 -= c1 * k.h[1];
          G2 -= c1 * k.h[2];
        }
      } else {
        const double q2 = R2 * hinv * hinv;
        const double rinv3 = ((15.0 / 8.0 * q2 - 21.0 / 4.0) * q2 + 35.0 / 8.0) * h3inv;
        const double rinv = (((-5.0 / 16.0 * q2 + 21.0 / 16.0) * q2 - 35.0 / 16.0) * q2 + 35.0 / 16.0) * hinv;
        G0 -= X * rinv3;
        G1 -= Y * rinv3;
        G2 -= Z * rinv3;
        P -= rinv;
      }
    }
    phi[s] = P;
    gx[s] = G0;
    gy[s] = G1;
    gz[s] = G2;
  }
}

// ------------------------------------------------------------------ drift

// Fixed-point drift (no reference counterpart): x += int64(trunc(v*dt*2^32))
// modulo 2^32, uint32 wrap-around being the periodic boundary.  The product
// is formed in double as (double(v) * dt) * 2^32 and truncated toward zero,
// the conversion rule of fixed(double) (tigerpm/fixed.hpp:63-75) taken
// through a signed type.  Returns -1 if any |v*dt| >= 2^31 box lengths.
int orc_drift(int64_t n, uint32_t* x, uint32_t* y, uint32_t* z, const float* vx,
              const float* vy, const float* vz, double dt) {
  uint32_t* X[3] = {x, y, z};
  const float* V[3] = {vx, vy, vz};
  for (int d = 0; d < 3; d++) {
    for (int64_t i = 0; i < n; i++) {
      const double t = (double)V[d][i] * dt;
      if (!(std::fabs(t) < 2147483648.0)) return -1;
      const int64_t di = (int64_t)(t * kTwo32);
      X[d][i] = (uint32_t)((uint64_t)X[d][i] + (uint64_t)di);
    }
  }
  return 0;
}

int orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"

// ------------------------------------------------------ initial conditions

namespace {

// Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds; each multiplies counter words 0 and 2
// by the round multipliers, swaps and xors the high halves with the other
// words and the key, and bumps the key by the Weyl constants.
void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    const uint64_t a = (uint64_t)0xD2511F53u * c[0];
    const uint64_t b = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(b >> 32) ^ c[1] ^ k0;
    const uint32_t n1 = (uint32_t)b;
    const uint32_t n2 = (uint32_t)(a >> 32) ^ c[3] ^ k1;
    const uint32_t n3 = (uint32_t)a;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// power_spectrum_function (src/initialize.cpp:10-66) in double, with the
// table transformation of read_power_spectrum (:182-211).
struct Spectrum {
  std::vector<double> P;
  double lo = 0, hi = 0, step = 1;
  double eval(double k) const {
    const double t = (std::log(k) - lo) / step;
    int i0 = std::min(std::max((int)t - 1, 0), (int)P.size() - 4);
    const double x = t - (i0 + 1);
    double y[4];
    for (int q = 0; q < 4; q++) y[q] = std::log(P[i0 + q]);
    const double s1 = 0.5 * (y[2] - y[0]), s2 = 0.5 * (y[3] - y[1]);
    // cubic Hermite between y1 and y2 with central-difference slopes
    const double c2 = -2 * s1 - s2 - 3 * y[1] + 3 * y[2];
    const double c3 = s1 + s2 + 2 * y[1] - 2 * y[2];
    return std::exp(y[1] + x * (s1 + x * (c2 + x * c3)));
  }
  double w8(double lnk, double h) const {  // sigma8 integrand over ln k
    const double R = 8.0 / h, k = std::exp(lnk);
    const double u = std::sin(k * R) - k * R * std::cos(k * R);
    return 9.0 / (2.0 * M_PI * M_PI) / std::pow(R, 6) * eval(k) * u * u / (k * k * k);
  }
  int build(const double* tk, const double* tp, int n, double h, double sigma8) {
    if (n < 4) return -1;
    P.resize(n);
    double kmin = 1e300, kmax = 0;
    for (int i = 0; i < n; i++) {
      P[i] = tp[i] / (h * h * h);
      kmin = std::min(kmin, tk[i] * h);
      kmax = std::max(kmax, tk[i] * h);
    }
    lo = std::log(kmin);
    hi = std::log(kmax);
    step = (hi - lo) / (n - 1);
    const int m = 8192;  // Simpson's rule
    const double d = (hi - lo) / m;
    double s = (w8(lo, h) + w8(hi, h)) * d / 3.0;
    for (int i = 1; i < m; i++) s += (i % 2 ? 4.0 : 2.0) / 3.0 * w8(lo + i * d, h) * d;
    for (double& p : P) p *= sigma8 * sigma8 / s;
    return 0;
  }
};

// growth_factor (src/initialize.cpp:76-83), a taken in single precision and
// the literals 4/7 and 1/70 as the reference's float constants.
double growth(double om, double a_in) {
  const double a = (double)(float)a_in;
  const double ol = 1.0 - om, a3 = a * a * a;
  const double Om = om / (om + a3 * ol), Ol = a3 * ol / (om + a3 * ol);
  return 2.5 * a * Om / (std::pow(Om, (double)(4.f / 7.f)) - Ol + (1 + Om / 2) * (1 + (double)0.014285714f * Ol));
}

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  philox(c, key[0], key[1]);
  for (int i = 0; i < 4; i++) out[i] = c[i];
}

int orc_ic_power(const double* tk, const double* tp, int n, double h, double sigma8, int64_t nk, const double* k,
                 double* out) {
  Spectrum s;
  if (s.build(tk, tp, n, h, sigma8)) return -1;
  for (int64_t i = 0; i < nk; i++) out[i] = s.eval(k[i]);
  return 0;
}

double orc_growth_factor(double om, double a) { return growth(om, a); }

// zeldovich_begin / fft3d_force_real / zeldovich_end (src/initialize.cpp:91-180,
// src/fft.cpp:86-123) in FP64 with the library's deviates: Philox-4x32-10 keyed
// by seed, counter = (i, j, kz, 0) of the half-spectrum element; x = (u0 + 1)
// 2^-32, y = u1 2^-32, deviate exp(2 pi i y) sqrt(-ln x).  npower > 0: table
// spectrum (k in h/Mpc) with the physical amplitude L^-1.5 N^3 and -D1/L
// (L = code_to_cm / 3.086e24 Mpc); npower = 0: k^index exp(-k / (kcut k_Nyq))
// in mode units.  rms_disp > 0 rescales the displacement to that rms in
// particle spacings.  Positions in lattice order (x-major), fixed32.
int orc_ic_zeldovich(int N, uint64_t seed, int npower, const double* tk, const double* tp, double index,
                     double kcut, double rms_disp, double h, double sigma8, double code_to_cm, double omega_m,
                     double z0, uint32_t* x, uint32_t* y, uint32_t* z, double* dxmax) {
  const int Nh = N / 2 + 1;
  const int64_t m_end = (int64_t)N * N / 4;
  std::vector<double> amp(std::max<int64_t>(m_end, 1), 0.0);
  double kunit = 1.0, L = 1.0, scale = -1.0;
  if (npower > 0) {
    Spectrum s;
    if (s.build(tk, tp, npower, h, sigma8)) return -1;
    L = code_to_cm / 3.086e24;
    kunit = 2.0 * M_PI / L;
    const double f = std::pow(L, -1.5) * (double)N * N * N;
    for (int64_t m = 1; m < m_end; m++) {
      const double k = kunit * std::sqrt((double)m);
      amp[m] = std::sqrt(s.eval(k)) * f / (k * k);
    }
    scale = -(growth(omega_m, 1.0 / (z0 + 1.0)) / growth(omega_m, 1.0)) / L;
  } else {
    if (!(kcut > 0) || !(rms_disp > 0)) return -1;
    for (int64_t m = 1; m < m_end; m++) {
      const double k = std::sqrt((double)m);
      amp[m] = std::sqrt(std::pow(k, index) * std::exp(-k / (kcut * 0.5 * N))) / (k * k);
    }
  }
  auto smode = [N](int i) { return i < N / 2 ? i : i - N; };
  auto value = [&](int i, int j, int kz, int d) -> cd {
    const int a = smode(i), b = smode(j), c = smode(kz);
    const int64_t i2 = (int64_t)a * a + (int64_t)b * b + (int64_t)c * c;
    if (i2 <= 0 || i2 >= m_end) return cd(0, 0);
    uint32_t ctr[4] = {(uint32_t)i, (uint32_t)j, (uint32_t)kz, 0u};
    philox(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u = ((double)ctr[0] + 1.0) / kTwo32, v = (double)ctr[1] / kTwo32;
    const double r = std::sqrt(-std::log(u));
    const int K[3] = {a, b, c};
    const double A = amp[i2] * kunit * K[d];
    return cd(r * std::cos(2 * M_PI * v) * A, r * std::sin(2 * M_PI * v) * A);
  };
  const int64_t n = (int64_t)N * N * N;
  std::vector<std::vector<double>> disp(3, std::vector<double>(n));
  std::vector<cd> Y((size_t)N * N * Nh);
  for (int d = 0; d < 3; d++) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)N * N * Nh; e++) {
      const int kz = (int)(e % Nh), j = (int)((e / Nh) % N), i = (int)(e / ((int64_t)N * Nh));
      cd v = value(i, j, kz, d);
      if (kz == 0) v = 0.5 * (v + std::conj(value((N - i) % N, (N - j) % N, 0, d)));
      Y[e] = v;
    }
    fft3d_c2r(N, Y.data(), disp[d].data());  // carries 1/N^3 as the reference's inverse
  }
  if (rms_disp > 0) {
    double ss = 0;
    for (int d = 0; d < 3; d++)
      for (int64_t p = 0; p < n; p++) ss += disp[d][p] * disp[d][p];
    scale = -(rms_disp / N) / std::sqrt(ss / (double)n);
  }
  uint32_t* X[3] = {x, y, z};
  double mx = 0;
  for (int64_t p = 0; p < n; p++) {
    const int I[3] = {(int)(p / ((int64_t)N * N)), (int)((p / N) % N), (int)(p % N)};
    for (int d = 0; d < 3; d++) {
      const double dx = scale * disp[d][p];
      mx = std::max(mx, std::fabs(dx * N));
      double q = (I[d] + 0.5) / N + dx;
      q -= std::floor(q);
      X[d][p] = (uint32_t)std::min(q * kTwo32, 4294967295.0);
    }
  }
  if (dxmax) *dxmax = mx;
  return 0;
}

}  // extern "C"
