// fft3d.cu -- the periodic Poisson solve of gravity_long_compute as five
// passes over HBM, with the Green's function fused into the middle one.
//
// Reference: gravity_long_compute (src/gravity_long.cpp:36-48) runs an FFTW
// r2c transform, apply_laplacian (:201-245) and a c2r transform.  The
// library's cuFFT path does the same in three library calls plus a Green
// kernel; this file replaces them for four_dim = N a multiple of 16 of the
// form 2^a 3^b 5^c, N <= 1024:
//
//   P1  z: two real rows (x, 2p), (x, 2p+1) form one complex line; complex
//       FFT; the two half-spectra are separated (2-for-1 real transform)
//   P2  y: forward FFT of every (x, kz) column
//   P3  x: forward FFT of every (y, kz) column, times the Green's function
//       -exp(-k^2 rs^2) sinc^-p / k^2 / N^3, inverse FFT, in one pass
//   P4  y: inverse
//   P5  z: the two half-spectra of rows (x, 2p), (x, 2p+1) recombined into
//       one complex line, inverse FFT, real and imaginary parts stored as the
//       two rows of phi
//
// The spectrum lives in a [N][N][Sz] complex array, Sz = N/2+1 rounded up to
// 8 so that a block's kz columns start on a 64-byte boundary (the padding
// columns are zero and never reach phi).  Two engines run the passes:
//
//  * line engine (the meshes with a compiled plan, TPM_LINE_SIZES): one line
//    per TL lanes of a warp, E = N / TL values per lane in registers, a
//    compile-time Stockham plan of radices 16/12/10/8/6/5/4/3/2 that divide E
//    (three stages for most sizes: 12.8.8 at 768, 12.8.4 at 384), the line's
//    row of shared memory between stages with warp-level synchronisation only,
//    and per-stage twiddle tables; the x pass runs its inverse with the
//    reversed plan straight from the forward transform's registers;
//  * block engine (every other supported N): each block holds 4 lines in
//    shared memory and transforms them with a radix-16/8/4/3/5/2 Stockham FFT
//    over two shared buffers.
//
// Twiddles are computed in FP64 on the host.  Forward transforms use
// exp(-i...), inverse exp(+i...), both unnormalised (cuFFT's convention);
// 1/N^3 is folded into the Green's function.
#include "tpm_internal.cuh"

#include <cmath>
#include <vector>

namespace tpm {
namespace {

#ifndef TPM_FFT_LINES
#define TPM_FFT_LINES 4
#endif
constexpr int kFftLines = TPM_FFT_LINES;   // lines per block (4 or 8)
constexpr int kFftThreads = 64 * kFftLines;
constexpr int kFftMaxN = 1024;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// s * i * a for s = +1 / -1
template <int S>
__device__ __forceinline__ float2 imul(float2 a) {
  return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// R-point DFTs X_k = sum_n v_n exp(S 2 pi i n k / R), in place.
template <int R, int S>
struct Dft;

template <int S>
struct Dft<2, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int S>
struct Dft<3, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float h = 0.86602540378443864676f;  // sin(2 pi / 3)
    const float2 s = cadd(v[1], v[2]);
    const float2 d = csub(v[1], v[2]);
    const float2 m = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
    const float2 t = imul<S>(make_float2(h * d.x, h * d.y));
    v[0] = cadd(v[0], s);
    v[1] = cadd(m, t);
    v[2] = csub(m, t);
  }
};

template <int S>
struct Dft<4, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const float2 c = cadd(v[1], v[3]), d = imul<S>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  }
};

template <int S>
struct Dft<5, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;  // cos(2pi/5), cos(4pi/5)
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;   // sin(2pi/5), sin(4pi/5)
    const float2 a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    const float2 b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    const float2 x0 = v[0];
    const float2 p1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    const float2 p2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    const float2 q1 = imul<S>(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    const float2 q2 = imul<S>(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
  }
};

// Power-of-two DFTs of 8 and 16 points in registers: a radix-2 split
// a_n = v_n + v_{n+R/2}, b_n = (v_n - v_{n+R/2}) w_R^n, then X_{2m} = DFT(a)_m,
// X_{2m+1} = DFT(b)_m.  w16[k] = (cos, sin)(2 pi k / 16), k < 8.
__device__ __forceinline__ float2 w16(int k, int S) {
  constexpr float c[8] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                          0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f};
  constexpr float sn[8] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
                           1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f};
  return make_float2(c[k], S > 0 ? sn[k] : -sn[k]);
}

template <int R, int S>
struct DftSplit {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr int H = R / 2;
    float2 a[H], b[H];
#pragma unroll
    for (int n = 0; n < H; n++) {
      a[n] = cadd(v[n], v[n + H]);
      const float2 d = csub(v[n], v[n + H]);
      b[n] = n == 0 ? d : cmul(d, w16(n * (16 / R), S));
    }
    Dft<H, S>::run(a);
    Dft<H, S>::run(b);
#pragma unroll
    for (int m = 0; m < H; m++) {
      v[2 * m] = a[m];
      v[2 * m + 1] = b[m];
    }
  }
};

template <int S>
struct Dft<8, S> : DftSplit<8, S> {};
template <int S>
struct Dft<16, S> : DftSplit<16, S> {};

// exp(S 2 pi i m / R) for R = 6, 10, 12 (m < R), as literals.
template <int R>
__device__ __forceinline__ float2 wtab(int m, int S) {
  static_assert(R == 6 || R == 10 || R == 12, "composite radices 6, 10, 12");
  constexpr float c6[6] = {1.0f, 0.5f, -0.5f, -1.0f, -0.5f, 0.5f};
  constexpr float s6[6] = {0.0f, 0.86602540378443865f, 0.86602540378443865f, 0.0f, -0.86602540378443865f,
                           -0.86602540378443865f};
  constexpr float c10[10] = {1.0f, 0.80901699437494742f, 0.30901699437494742f, -0.30901699437494742f,
                             -0.80901699437494742f, -1.0f, -0.80901699437494742f, -0.30901699437494742f,
                             0.30901699437494742f, 0.80901699437494742f};
  constexpr float s10[10] = {0.0f, 0.58778525229247313f, 0.95105651629515357f, 0.95105651629515357f,
                             0.58778525229247313f, 0.0f, -0.58778525229247313f, -0.95105651629515357f,
                             -0.95105651629515357f, -0.58778525229247313f};
  constexpr float c12[12] = {1.0f, 0.86602540378443865f, 0.5f, 0.0f, -0.5f, -0.86602540378443865f,
                             -1.0f, -0.86602540378443865f, -0.5f, 0.0f, 0.5f, 0.86602540378443865f};
  constexpr float s12[12] = {0.0f, 0.5f, 0.86602540378443865f, 1.0f, 0.86602540378443865f, 0.5f,
                             0.0f, -0.5f, -0.86602540378443865f, -1.0f, -0.86602540378443865f, -0.5f};
  const float c = R == 6 ? c6[m] : (R == 10 ? c10[m] : c12[m]);
  const float s = R == 6 ? s6[m] : (R == 10 ? s10[m] : s12[m]);
  return make_float2(c, S > 0 ? s : -s);
}

// a * exp(S 2 pi i m / R), with the quarter turns as swaps and negations.
template <int R, int S>
__device__ __forceinline__ float2 twc(float2 a, int m) {
  if (m == 0) return a;
  if (4 * m == R) return imul<S>(a);
  if (2 * m == R) return make_float2(-a.x, -a.y);
  if (4 * m == 3 * R) return imul<-S>(a);
  return cmul(a, wtab<R>(m, S));
}

// Composite R = A B point DFT (Cooley-Tukey in registers): with input index
// m = a B + b and output index k = k1 + A k2,
//   X[k1 + A k2] = sum_b w_B^(b k2) w_R^(b k1) sum_a v[a B + b] w_A^(a k1).
template <int A, int B, int S>
struct DftComp {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr int R = A * B;
    float2 t[R];
#pragma unroll
    for (int b = 0; b < B; b++) {
      float2 u[A];
#pragma unroll
      for (int a = 0; a < A; a++) u[a] = v[a * B + b];
      Dft<A, S>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < A; k1++) t[b * A + k1] = twc<R, S>(u[k1], b * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      float2 u[B];
#pragma unroll
      for (int b = 0; b < B; b++) u[b] = t[b * A + k1];
      Dft<B, S>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = u[k2];
    }
  }
};

template <int S>
struct Dft<6, S> : DftComp<2, 3, S> {};
template <int S>
struct Dft<10, S> : DftComp<2, 5, S> {};
template <int S>
struct Dft<12, S> : DftComp<4, 3, S> {};

// One Stockham stage of radix R over the block's lines of length N (line
// stride LS), from shared buffer x to shared buffer y: butterfly j of a line
// reads x[j + r N/R], applies the twiddles exp(S 2 pi i (j mod Ns) r / (Ns R)),
// and writes y[(j / Ns) Ns R + (j mod Ns) + r Ns].  Thread t takes line
// t mod L and butterflies j = t / L + 64 i; j / Ns is a multiply-high by
// ceil(2^32 / Ns), exact while j Ns < 2^32.
template <int R, int S>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ x, float2* __restrict__ y,
                                          const float2* __restrict__ tw, int N, int LS, int Ns, unsigned ns_inv) {
  const int nb = N / R;
  const int stride = N / (Ns * R);
  const int line = threadIdx.x & (kFftLines - 1);
  const float2* xl = x + line * LS;
  float2* yl = y + line * LS;
  for (int j = threadIdx.x / kFftLines; j < nb; j += kFftThreads / kFftLines) {
    const int q = Ns == 1 ? j : (int)__umulhi((unsigned)j, ns_inv);
    const int k = j - q * Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      float2 a = xl[j + r * nb];
      if (r > 0) {
        float2 w = tw[k * r * stride];
        if (S > 0) w.y = -w.y;
        a = cmul(a, w);
      }
      v[r] = a;
    }
    Dft<R, S>::run(v);
    float2* dst = yl + q * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[r * Ns] = v[r];
  }
  __syncthreads();
}

struct FftPlan {
  int N;
  int Sz;
  int nrad;
  int rad[12];
  unsigned ns_inv[12];  // ceil(2^32 / Ns) of each stage
};

// Full transform of the block's lines (S = -1 forward, +1 inverse) that start in
// a; b is the second buffer.  Returns the buffer holding the result.
template <int S>
__device__ __forceinline__ float2* block_fft(float2* a, float2* b, const float2* __restrict__ tw, const FftPlan& p,
                                             int LS) {
  int Ns = 1;
  for (int s = 0; s < p.nrad; s++) {
    switch (p.rad[s]) {
      case 16: fft_stage<16, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
      case 8: fft_stage<8, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
      case 4: fft_stage<4, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
      case 3: fft_stage<3, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
      case 5: fft_stage<5, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
      default: fft_stage<2, S>(a, b, tw, p.N, LS, Ns, p.ns_inv[s]); break;
    }
    Ns *= p.rad[s];
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

// Line stride in shared memory: N + 16/L complex values.  With the lines of
// a warp running fastest (L lines x 16/L positions per half-warp), the
// half-warp's 16 accesses then fall in 16 distinct bank pairs.
__device__ __forceinline__ int line_stride(int N) { return N + 16 / kFftLines; }

__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* __restrict__ tw, int N) {
  for (int i = threadIdx.x; i < N; i += blockDim.x) s_tw[i] = __ldg(tw + i);
}

// P1: forward z transform of real rows (x, 2p) and (x, 2p+1) as one complex
// line, then A_k = (Z_k + conj Z_{N-k}) / 2, B_k = (Z_k - conj Z_{N-k}) / 2i.
__global__ void __launch_bounds__(kFftThreads) k_fft_z_r2c(const float* __restrict__ rho, float2* __restrict__ Y,
                                                           FftPlan p, const float2* __restrict__ tw, int x0) {
  extern __shared__ float2 fsm[];
  const int N = p.N, LS = line_stride(N), Nh = N / 2 + 1;
  float2* buf = fsm;
  float2* alt = fsm + kFftLines * LS;
  float2* s_tw = fsm + 2 * kFftLines * LS;
  const int per_x = N / (2 * kFftLines);
  const int xb = blockIdx.x / per_x;
  const int x = x0 + xb;
  const int p0 = (blockIdx.x - xb * per_x) * kFftLines;
#pragma unroll 1
  for (int l = 0; l < kFftLines; l++) {
    const int64_t row = (int64_t)x * N + 2 * (p0 + l);
    for (int n = threadIdx.x; n < N; n += kFftThreads)
      buf[l * LS + n] = make_float2(__ldg(rho + row * N + n), __ldg(rho + (row + 1) * N + n));
  }
  load_twiddles(s_tw, tw, N);
  __syncthreads();
  buf = block_fft<-1>(buf, alt, s_tw, p, LS);
#pragma unroll 1
  for (int l = 0; l < kFftLines; l++) {
    const int64_t row = (int64_t)x * N + 2 * (p0 + l);
    for (int kz = threadIdx.x; kz < Nh; kz += kFftThreads) {
      const float2 zk = buf[l * LS + kz];
      const float2 zm = buf[l * LS + (kz == 0 ? 0 : N - kz)];
      Y[row * p.Sz + kz] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      Y[(row + 1) * p.Sz + kz] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    // padding columns: zero, so a borrowed (uninitialised) spectrum buffer
    // carries no stale values through the column passes
    for (int kz = Nh + threadIdx.x; kz < p.Sz; kz += kFftThreads) {
      Y[row * p.Sz + kz] = make_float2(0.f, 0.f);
      Y[(row + 1) * p.Sz + kz] = make_float2(0.f, 0.f);
    }
  }
}

// P2 / P4: transform along y of the L kz columns [c0, c0 + L) of plane x.
template <int S>
__global__ void __launch_bounds__(kFftThreads) k_fft_y(float2* __restrict__ Y, FftPlan p,
                                                       const float2* __restrict__ tw, int x0) {
  extern __shared__ float2 fsm[];
  const int N = p.N, LS = line_stride(N);
  float2* buf = fsm;
  float2* alt = fsm + kFftLines * LS;
  float2* s_tw = fsm + 2 * kFftLines * LS;
  const int per_x = p.Sz / kFftLines;
  const int xb = blockIdx.x / per_x;
  const int x = x0 + xb;
  const int c0 = (blockIdx.x - xb * per_x) * kFftLines;
  float2* plane = Y + (int64_t)x * N * p.Sz + c0;
  for (int e = threadIdx.x; e < kFftLines * N; e += kFftThreads) {
    const int y = e / kFftLines, c = e - y * kFftLines;
    buf[c * LS + y] = plane[(int64_t)y * p.Sz + c];
  }
  load_twiddles(s_tw, tw, N);
  __syncthreads();
  buf = block_fft<S>(buf, alt, s_tw, p, LS);
  for (int e = threadIdx.x; e < kFftLines * N; e += kFftThreads) {
    const int y = e / kFftLines, c = e - y * kFftLines;
    plane[(int64_t)y * p.Sz + c] = buf[c * LS + y];
  }
}

// P3: forward transform along x of the L kz columns [c0, c0 + L) of row y,
// the Green's function (apply_laplacian, src/gravity_long.cpp:214-239; the
// same separable tables and FP32 expression as the cuFFT path's k_green),
// and the inverse transform along x.
__global__ void __launch_bounds__(kFftThreads) k_fft_x_green(float2* __restrict__ Y, FftPlan p,
                                                             const float2* __restrict__ tw,
                                                             const float* __restrict__ gt,
                                                             const float* __restrict__ k2tab, float norm) {
  extern __shared__ float2 fsm[];
  const int N = p.N, LS = line_stride(N), Nh = N / 2 + 1;
  float2* buf = fsm;
  float2* alt = fsm + kFftLines * LS;
  float2* s_tw = fsm + 2 * kFftLines * LS;
  const int per_y = p.Sz / kFftLines;
  const int y = blockIdx.x / per_y;
  const int c0 = (blockIdx.x - y * per_y) * kFftLines;
  float2* col = Y + (int64_t)y * p.Sz + c0;
  const int64_t xs = (int64_t)N * p.Sz;
  for (int e = threadIdx.x; e < kFftLines * N; e += kFftThreads) {
    const int x = e / kFftLines, c = e - x * kFftLines;
    buf[c * LS + x] = col[x * xs + c];
  }
  load_twiddles(s_tw, tw, N);
  __syncthreads();
  buf = block_fft<-1>(buf, alt, s_tw, p, LS);
  alt = buf == fsm ? fsm + kFftLines * LS : fsm;
  const float k2y = __ldg(k2tab + y), gy = __ldg(gt + y);
  const int c = threadIdx.x & (kFftLines - 1);
  for (int n = threadIdx.x / kFftLines; n < N; n += kFftThreads / kFftLines) {
    const int kz = c0 + c;
    float g = 0.0f;
    if (kz < Nh) {
      const float k2 = __ldg(k2tab + n) + k2y + __ldg(k2tab + kz);
      g = k2 > 0.0f ? -(__ldg(gt + n) * gy * __ldg(gt + kz)) / k2 * norm : 0.0f;
    }
    float2& v = buf[c * LS + n];
    v.x *= g;
    v.y *= g;
  }
  __syncthreads();
  buf = block_fft<1>(buf, alt, s_tw, p, LS);
  for (int e = threadIdx.x; e < kFftLines * N; e += kFftThreads) {
    const int x = e / kFftLines, c = e - x * kFftLines;
    col[x * xs + c] = buf[c * LS + x];
  }
}

// P5: rows (x, 2p) and (x, 2p+1) back to real space: Z_k = A_k + i B_k with
// A_{N-k} = conj A_k (imaginary parts of k = 0 and N/2 dropped, as a real
// transform has none), inverse FFT, real part -> row 2p, imaginary -> 2p+1.
__global__ void __launch_bounds__(kFftThreads) k_fft_z_c2r(const float2* __restrict__ Y, float* __restrict__ phi,
                                                           FftPlan p, const float2* __restrict__ tw, int x0) {
  extern __shared__ float2 fsm[];
  const int N = p.N, LS = line_stride(N), Nh2 = N / 2;
  float2* buf = fsm;
  float2* alt = fsm + kFftLines * LS;
  float2* s_tw = fsm + 2 * kFftLines * LS;
  const int per_x = N / (2 * kFftLines);
  const int xb = blockIdx.x / per_x;
  const int x = x0 + xb;
  const int p0 = (blockIdx.x - xb * per_x) * kFftLines;
#pragma unroll 1
  for (int l = 0; l < kFftLines; l++) {
    const int64_t row = (int64_t)x * N + 2 * (p0 + l);
    for (int k = threadIdx.x; k < N; k += kFftThreads) {
      float2 a, b;
      if (k <= Nh2) {
        a = __ldg(Y + row * p.Sz + k);
        b = __ldg(Y + (row + 1) * p.Sz + k);
        if (k == 0 || k == Nh2) {
          a.y = 0.0f;
          b.y = 0.0f;
        }
      } else {
        a = __ldg(Y + row * p.Sz + (N - k));
        b = __ldg(Y + (row + 1) * p.Sz + (N - k));
        a.y = -a.y;
        b.y = -b.y;
      }
      buf[l * LS + k] = make_float2(a.x - b.y, a.y + b.x);
    }
  }
  load_twiddles(s_tw, tw, N);
  __syncthreads();
  buf = block_fft<1>(buf, alt, s_tw, p, LS);
#pragma unroll 1
  for (int l = 0; l < kFftLines; l++) {
    const int64_t row = (int64_t)x * N + 2 * (p0 + l);
    for (int n = threadIdx.x; n < N; n += kFftThreads) {
      const float2 v = buf[l * LS + n];
      phi[row * N + n] = v.x;
      phi[(row + 1) * N + n] = v.y;
    }
  }
}

// ------------------------------------------------------------ line engine
//
// The same five passes for the mesh sizes that have a compile-time plan:
// one line of length N is held by TL lanes of a warp (TL = 4 .. 32), E = N / TL
// values per lane in registers.  A Stockham stage of radix R (R divides E)
// gives every lane E / R butterflies j = lane + TL b; between stages the
// line goes through its own row of shared memory with only warp-level
// synchronisation, and the first stage reads its inputs (global rows, or the
// block's transposed columns) and the last stage writes its outputs in
// natural order straight from registers.  Radices, strides and divisions are
// compile-time constants.  Column passes stage kLineCols = 8 neighbouring
// columns per block (64-byte row segments) through shared memory.
constexpr int kLineCols = 8;

struct LinePlan {
  int TL, E, ns;
  int rad[6];
};

constexpr LinePlan line_plan_tl(int N, int TL) {
  LinePlan p{TL, N / TL, 0, {1, 1, 1, 1, 1, 1}};
  if (N % TL != 0) {
    p.ns = 99;
    return p;
  }
  constexpr int cand[9] = {16, 12, 10, 8, 6, 5, 4, 3, 2};
  int M = N;
  while (M > 1) {
    int pick = 0;
    for (int i = 0; i < 9; i++)
      if (pick == 0 && p.E % cand[i] == 0 && M % cand[i] == 0) pick = cand[i];
    if (pick == 0 || p.ns == 6) {
      p.ns = 99;
      return p;
    }
    p.rad[p.ns++] = pick;
    M /= pick;
  }
  return p;
}

// Fewest stages with at most 36 values per lane; ties go to more lanes per line.
constexpr LinePlan line_plan(int N) {
  LinePlan best{0, 0, 99, {1, 1, 1, 1, 1, 1}};
  constexpr int tls[4] = {32, 16, 8, 4};
  for (int i = 0; i < 4; i++) {
    const LinePlan p = line_plan_tl(N, tls[i]);
    if (p.ns < 99 && p.E <= 36 && p.ns < best.ns) best = p;
  }
  return best;
}

constexpr int ns_before(const LinePlan& p, int st) {
  int r = 1;
  for (int i = 0; i < st; i++) r *= p.rad[i];
  return r;
}

// The same radices in the opposite order.  A transform with the reversed plan
// takes its first-stage inputs in exactly the registers where the forward
// plan's last stage leaves its outputs (lane + TL b + r N / R_last).
constexpr LinePlan reverse_plan(const LinePlan& p) {
  LinePlan q = p;
  for (int i = 0; i < p.ns; i++) q.rad[i] = p.rad[p.ns - 1 - i];
  return q;
}

template <int N>
struct LineCfg {
  static constexpr LinePlan P = line_plan(N);
  static constexpr int TL = P.TL, E = P.E;
  static constexpr int kThreads = kLineCols * TL;
  // line stride = N + 4 (N % 16 == 0): the transposed column loads of 8
  // columns x 4 rows per warp then fall in distinct bank pairs
  static constexpr int LS = N + 4;
  // resident threads per SM the register budget targets: 768 (85 registers),
  // 512 (128 registers) from 28 values per lane up
  static constexpr int kMinBlocks = (E >= 28 ? 2 : 3) * 256 / kThreads;
  // the x pass (two transforms and the Green's function) from 24 values per
  // lane: 2 blocks (128 registers, no spills) beat 3 that spill
  // (768^3: 2.14 -> 2.06 ms; the y passes are slower that way at 768^3)
  static constexpr int kMinBlocksX = (E >= 24 ? 2 : 3) * 256 / kThreads;
  static constexpr size_t kSmem = sizeof(float2) * ((size_t)N + (size_t)kLineCols * LS);
  // the x pass holds the stage tables of both radix orders and the x axis's
  // Green's-function and k^2 tables (read from shared memory, not L1)
  static constexpr size_t kSmemX = kSmem + sizeof(float2) * (size_t)N + sizeof(float) * 2 * (size_t)N;
  static_assert(P.ns >= 1 && P.ns <= 6, "no line plan for this N");
};

// One line transform of sign S with the plan of N (REV: its radices reversed).
template <int N, int S, bool REV = false>
struct LineFft {
  using L = LineCfg<N>;
  static constexpr LinePlan P = REV ? reverse_plan(L::P) : L::P;
  static constexpr int TL = L::TL, E = L::E;

  // Stage ST: v holds its inputs, v[b R + r] = x[j + r N / R] for the lane's
  // butterflies j = lane + TL b; twiddles exp(S 2 pi i (j mod Ns) r / (Ns R))
  // from the stage table (line_twiddle_table): entry Ns - 1 + k (R - 1) + r - 1
  // holds exp(-2 pi i k r / (Ns R)), so the R - 1 twiddles of one butterfly
  // are contiguous and the lanes' reads stride by R - 1 values.
  template <int ST, class Out>
  __device__ __forceinline__ static void stage(float2* __restrict__ line, float2 (&v)[E],
                                               const float2* __restrict__ tw, int lane, Out& out) {
    constexpr int R = P.rad[ST];
    constexpr int NS = ns_before(P, ST);
    constexpr int NB = E / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
      if (NS > 1) {
        const int j = lane + TL * b;
        const float2* tws = tw + (NS - 1) + (j % NS) * (R - 1);
#pragma unroll
        for (int r = 1; r < R; r++) {
          float2 w = tws[r - 1];
          if (S > 0) w.y = -w.y;
          v[b * R + r] = cmul(v[b * R + r], w);
        }
      }
      Dft<R, S>::run(v + b * R);
    }
    if constexpr (ST == P.ns - 1) {
      // Ns R = N: butterfly j's outputs are x[j + r Ns], natural order
#pragma unroll
      for (int b = 0; b < NB; b++)
#pragma unroll
        for (int r = 0; r < R; r++) out(lane + TL * b + r * NS, v[b * R + r]);
    } else {
      if (NS == 1 && R % 2 == 0) {
        // first stage: butterfly j's R outputs are contiguous (x[j R + r]);
        // 16-byte stores of two values each (a lane stride of R values would
        // put 8 or 16 lanes of a scalar store on one bank pair)
#pragma unroll
        for (int b = 0; b < NB; b++) {
          float4* dst = reinterpret_cast<float4*>(line + (lane + TL * b) * R);
#pragma unroll
          for (int r = 0; r < R; r += 2)
            dst[r / 2] = make_float4(v[b * R + r].x, v[b * R + r].y, v[b * R + r + 1].x, v[b * R + r + 1].y);
        }
      } else {
#pragma unroll
        for (int b = 0; b < NB; b++) {
          const int j = lane + TL * b;
          const int q = j / NS, k = j - q * NS;
#pragma unroll
          for (int r = 0; r < R; r++) line[q * NS * R + k + r * NS] = v[b * R + r];
        }
      }
      __syncwarp();
      constexpr int R2 = P.rad[ST + 1];
#pragma unroll
      for (int b = 0; b < E / R2; b++)
#pragma unroll
        for (int r = 0; r < R2; r++) v[b * R2 + r] = line[lane + TL * b + r * (N / R2)];
      __syncwarp();
      stage<ST + 1>(line, v, tw, lane, out);
    }
  }

  // First-stage inputs into v: v[b R + r] = in(lane + TL b + r N / R).
  template <class In>
  __device__ __forceinline__ static void load(float2 (&v)[E], int lane, In in) {
    constexpr int R = P.rad[0];
#pragma unroll
    for (int b = 0; b < E / R; b++)
#pragma unroll
      for (int r = 0; r < R; r++) v[b * R + r] = in(lane + TL * b + r * (N / R));
  }

  // The transform from inputs already in v (as load leaves them); out(n, value)
  // takes output n, and v keeps the outputs, v[b R + r] = X[lane + TL b + r N / R]
  // with R the last stage's radix.
  template <class Out>
  __device__ __forceinline__ static void from_regs(float2* __restrict__ line, float2 (&v)[E],
                                                   const float2* __restrict__ tw, int lane, Out out) {
    stage<0>(line, v, tw, lane, out);
  }

  // Transform of one line: in(n) gives input n, out(n, value) takes output n.
  // line is the line's shared-memory row (TL lanes); in may read it.
  template <class In, class Out>
  __device__ __forceinline__ static void run(float2* __restrict__ line, const float2* __restrict__ tw, int lane,
                                             In in, Out out) {
    float2 v[E];
    load(v, lane, in);
    __syncwarp();
    stage<0>(line, v, tw, lane, out);
  }
};

template <int N>
__device__ __forceinline__ void line_twiddles(float2* s_tw, const float2* __restrict__ tw) {
  for (int i = threadIdx.x; i < N; i += LineCfg<N>::kThreads) s_tw[i] = __ldg(tw + i);
}

// Load / store the block's kLineCols columns (rows y < N at stride rs) into /
// from the transposed shared-memory lines, two columns per 16-byte access.
// Every load is issued before the first shared store (E / 2 loads in flight
// per thread).
template <int N>
__device__ __forceinline__ void cols_load(float2* __restrict__ lines, const float2* __restrict__ g, int64_t rs) {
  using L = LineCfg<N>;
  constexpr int IT = (kLineCols / 2) * N / L::kThreads;
  static_assert(IT * L::kThreads == (kLineCols / 2) * N, "column tile per thread");
  float4 u[IT];
#pragma unroll
  for (int i = 0; i < IT; i++) {
    const int e = threadIdx.x + i * L::kThreads;
    const int y = e / (kLineCols / 2), c = 2 * (e - y * (kLineCols / 2));
    u[i] = __ldg(reinterpret_cast<const float4*>(g + y * rs + c));
  }
#pragma unroll
  for (int i = 0; i < IT; i++) {
    const int e = threadIdx.x + i * L::kThreads;
    const int y = e / (kLineCols / 2), c = 2 * (e - y * (kLineCols / 2));
    lines[c * L::LS + y] = make_float2(u[i].x, u[i].y);
    lines[(c + 1) * L::LS + y] = make_float2(u[i].z, u[i].w);
  }
}
template <int N>
__device__ __forceinline__ void cols_store(const float2* __restrict__ lines, float2* __restrict__ g, int64_t rs) {
  using L = LineCfg<N>;
  constexpr int IT = (kLineCols / 2) * N / L::kThreads;
  // thread index through an opaque move: the load's address arithmetic is
  // then recomputed here instead of being kept live across the transform
  int t;
  asm volatile("mov.b32 %0, %1;" : "=r"(t) : "r"((int)threadIdx.x));
#pragma unroll
  for (int i = 0; i < IT; i++) {
    const int e = t + i * L::kThreads;
    const int y = e / (kLineCols / 2), c = 2 * (e - y * (kLineCols / 2));
    const float2 a = lines[c * L::LS + y], b = lines[(c + 1) * L::LS + y];
    *reinterpret_cast<float4*>(g + y * rs + c) = make_float4(a.x, a.y, b.x, b.y);
  }
}

// P1 (line engine): rows (x, 2p), (x, 2p+1) as one complex line, forward z
// transform, the two half-spectra separated into spectrum rows 2p, 2p+1.
template <int N>
__global__ void __launch_bounds__(LineCfg<N>::kThreads, LineCfg<N>::kMinBlocks)
    k_line_z_r2c(const float* __restrict__ rho, float2* __restrict__ Y, int Sz, const float2* __restrict__ tw,
                 int x0) {
  using L = LineCfg<N>;
  extern __shared__ __align__(16) float2 lsm[];
  float2* s_tw = lsm;
  line_twiddles<N>(s_tw, tw);
  const int li = threadIdx.x / L::TL, lane = threadIdx.x - li * L::TL;
  float2* line = lsm + N + li * L::LS;
  constexpr int per_x = N / (2 * kLineCols);
  const int xb = blockIdx.x / per_x;
  const int p = (blockIdx.x - xb * per_x) * kLineCols + li;
  const int64_t row = (int64_t)(x0 + xb) * N + 2 * p;
  const float* r0 = rho + row * N;
  const float* r1 = r0 + N;
  __syncthreads();
  LineFft<N, -1>::run(
      line, s_tw, lane, [&](int n) { return make_float2(__ldg(r0 + n), __ldg(r1 + n)); },
      [&](int n, float2 v) { line[n] = v; });
  __syncwarp();
  float2* y0 = Y + row * Sz;
  float2* y1 = y0 + Sz;
  constexpr int Nh = N / 2 + 1;
  for (int kz = lane; kz < Sz; kz += L::TL) {
    float2 a = make_float2(0.f, 0.f), b = a;  // padding columns stay zero
    if (kz < Nh) {
      const float2 zk = line[kz];
      const float2 zm = line[kz == 0 ? 0 : N - kz];
      a = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      b = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    y0[kz] = a;
    y1[kz] = b;
  }
}

// P2 / P4 (line engine): the 8 columns [c0, c0 + 8) of plane x along y.
template <int N, int S>
__global__ void __launch_bounds__(LineCfg<N>::kThreads, LineCfg<N>::kMinBlocks)
    k_line_y(float2* __restrict__ Y, int Sz, const float2* __restrict__ tw, int x0) {
  using L = LineCfg<N>;
  extern __shared__ __align__(16) float2 lsm[];
  float2* s_tw = lsm;
  float2* lines = lsm + N;
  line_twiddles<N>(s_tw, tw);
  const int li = threadIdx.x / L::TL, lane = threadIdx.x - li * L::TL;
  float2* line = lines + li * L::LS;
  const int per_x = Sz / kLineCols;
  const int xb = blockIdx.x / per_x;
  const int c0 = (blockIdx.x - xb * per_x) * kLineCols;
  float2* plane = Y + (int64_t)(x0 + xb) * N * Sz + c0;
  cols_load<N>(lines, plane, Sz);
  __syncthreads();
  LineFft<N, S>::run(
      line, s_tw, lane, [&](int n) { return line[n]; }, [&](int n, float2 v) { line[n] = v; });
  __syncthreads();
  cols_store<N>(lines, plane, Sz);
}

// P3 (line engine): the 8 columns [c0, c0 + 8) of row y along x: forward
// transform, Green's function (as k_fft_x_green), inverse transform.  The
// inverse runs the reversed radix plan, so it starts from the registers the
// forward transform ends in, with the Green's function applied there: the
// spectrum of the line does not go through shared memory between the two.
// tw: the forward plan's stage tables, then the reversed plan's (N each).
template <int N>
__global__ void __launch_bounds__(LineCfg<N>::kThreads, LineCfg<N>::kMinBlocksX)
    k_line_x_green(float2* __restrict__ Y, int Sz, const float2* __restrict__ tw, const float* __restrict__ gt,
                   const float* __restrict__ k2tab, float norm) {
  using L = LineCfg<N>;
  using Fwd = LineFft<N, -1, false>;
  using Inv = LineFft<N, 1, true>;
  extern __shared__ __align__(16) float2 lsm[];
  float2* s_tw = lsm;
  float2* s_twr = lsm + N;
  float2* lines = lsm + 2 * N;
  for (int i = threadIdx.x; i < 2 * N; i += L::kThreads) s_tw[i] = __ldg(tw + i);
  float* s_gt = reinterpret_cast<float*>(lines + kLineCols * L::LS);
  float* s_k2 = s_gt + N;
  for (int i = threadIdx.x; i < N; i += L::kThreads) {
    s_gt[i] = __ldg(gt + i);
    s_k2[i] = __ldg(k2tab + i);
  }
  const int li = threadIdx.x / L::TL, lane = threadIdx.x - li * L::TL;
  float2* line = lines + li * L::LS;
  const int per_y = Sz / kLineCols;
  const int y = blockIdx.x / per_y;
  const int c0 = (blockIdx.x - y * per_y) * kLineCols;
  float2* col = Y + (int64_t)y * Sz + c0;
  const int64_t xs = (int64_t)N * Sz;
  cols_load<N>(lines, col, xs);
  __syncthreads();
  const int kz = c0 + li;
  const bool live = kz < N / 2 + 1;
  const float k2yz = __ldg(k2tab + y) + (live ? __ldg(k2tab + kz) : 0.f);
  const float gyz = __ldg(gt + y) * (live ? __ldg(gt + kz) : 0.f);
  float2 v[L::E];
  Fwd::load(v, lane, [&](int n) { return line[n]; });
  __syncwarp();
  Fwd::from_regs(line, v, s_tw, lane, [](int, float2) {});
  // v[b RL + r] = X[lane + TL b + r N / RL]: the Green's function in registers
  constexpr int RL = Fwd::P.rad[Fwd::P.ns - 1];
#pragma unroll
  for (int b = 0; b < L::E / RL; b++)
#pragma unroll
    for (int r = 0; r < RL; r++) {
      const int n = lane + L::TL * b + r * (N / RL);
      const float k2 = s_k2[n] + k2yz;
      const float g = k2 > 0.0f ? -(s_gt[n] * gyz) * __frcp_rn(k2) * norm : 0.0f;
      v[b * RL + r] = make_float2(v[b * RL + r].x * g, v[b * RL + r].y * g);
    }
  // The inverse recomputes its addresses: with the lane index passed through
  // an opaque move, the forward transform's index arithmetic is not kept
  // live across the inverse (it would spill).
  int lane2;
  asm volatile("mov.b32 %0, %1;" : "=r"(lane2) : "r"(lane));
  Inv::from_regs(line, v, s_twr, lane2, [&](int n, float2 u) { line[n] = u; });
  __syncthreads();
  cols_store<N>(lines, col, xs);
}

// P5 (line engine): spectrum rows 2p, 2p+1 recombined (Z = A + i B, the
// Hermitian halves mirrored), inverse z transform, real -> row 2p, imag -> 2p+1.
template <int N>
__global__ void __launch_bounds__(LineCfg<N>::kThreads, LineCfg<N>::kMinBlocks)
    k_line_z_c2r(const float2* __restrict__ Y, float* __restrict__ phi, int Sz, const float2* __restrict__ tw,
                 int x0) {
  using L = LineCfg<N>;
  extern __shared__ __align__(16) float2 lsm[];
  float2* s_tw = lsm;
  line_twiddles<N>(s_tw, tw);
  const int li = threadIdx.x / L::TL, lane = threadIdx.x - li * L::TL;
  float2* line = lsm + N + li * L::LS;
  constexpr int per_x = N / (2 * kLineCols);
  const int xb = blockIdx.x / per_x;
  const int p = (blockIdx.x - xb * per_x) * kLineCols + li;
  const int64_t row = (int64_t)(x0 + xb) * N + 2 * p;
  const float2* y0 = Y + row * Sz;
  const float2* y1 = y0 + Sz;
  float* f0 = phi + row * N;
  float* f1 = f0 + N;
  __syncthreads();
  LineFft<N, 1>::run(
      line, s_tw, lane,
      [&](int n) {
        float2 a, b;
        if (n <= N / 2) {
          a = __ldg(y0 + n);
          b = __ldg(y1 + n);
          if (n == 0 || n == N / 2) {
            a.y = 0.0f;
            b.y = 0.0f;
          }
        } else {
          a = __ldg(y0 + (N - n));
          b = __ldg(y1 + (N - n));
          a.y = -a.y;
          b.y = -b.y;
        }
        return make_float2(a.x - b.y, a.y + b.x);
      },
      [&](int n, float2 v) {
        f0[n] = v.x;
        f1[n] = v.y;
      });
}

template <int N>
int line_set_smem() {
  using L = LineCfg<N>;
  const int s = (int)L::kSmem;
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_line_z_r2c<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_line_y<N, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_line_y<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  TPM_CUDA_TRY(
      cudaFuncSetAttribute(k_line_x_green<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::kSmemX));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_line_z_c2r<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, s));
  return TPM_OK;
}

template <int N>
int line_poisson(tpm_ctx* c, float2* Y, int Sz, const float* gt, float norm) {
  using L = LineCfg<N>;
  // the kernels' shared-memory size depends on N alone: set once per N
  static const int attr = line_set_smem<N>();
  if (attr) return attr;
  cudaStream_t s = c->stream;
  const unsigned zblocks = (unsigned)(N * (N / (2 * kLineCols)));
  const unsigned cblocks = (unsigned)(N * (Sz / kLineCols));
  const float2* tw = c->fft_tw + N;  // the stage tables of the line plan, then of its reversal
  stage_begin(c, kStFftF);
  k_line_z_r2c<N><<<zblocks, L::kThreads, L::kSmem, s>>>(c->rho, Y, Sz, tw, 0);
  k_line_y<N, -1><<<cblocks, L::kThreads, L::kSmem, s>>>(Y, Sz, tw, 0);
  stage_end(c, kStFftF);
  stage_begin(c, kStGreen);
  k_line_x_green<N><<<cblocks, L::kThreads, L::kSmemX, s>>>(Y, Sz, tw, gt, c->k2tab, norm);
  stage_end(c, kStGreen);
  stage_begin(c, kStFftI);
  k_line_y<N, 1><<<cblocks, L::kThreads, L::kSmem, s>>>(Y, Sz, tw, 0);
  k_line_z_c2r<N><<<zblocks, L::kThreads, L::kSmem, s>>>(Y, c->phi, Sz, tw, 0);
  stage_end(c, kStFftI);
  c->launches += 5;
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

// Mesh sizes with a compiled line plan (the benchmark meshes, the batched
// and served box meshes, and the powers of two up to 1024).
#define TPM_LINE_SIZES(X) \
  X(64) X(96) X(128) X(144) X(160) X(192) X(240) X(256) X(288) X(320) X(384) X(512) X(576) X(640) X(768) X(1024)

bool line_supported(int N) {
  switch (N) {
#define TPM_LINE_CASE(n) case n:
    TPM_LINE_SIZES(TPM_LINE_CASE)
#undef TPM_LINE_CASE
    return true;
    default:
      return false;
  }
}

int line_dispatch(tpm_ctx* c, float2* Y, int Sz, const float* gt, float norm) {
  switch (c->N) {
#define TPM_LINE_CASE(n) \
  case n:                \
    return line_poisson<n>(c, Y, Sz, gt, norm);
    TPM_LINE_SIZES(TPM_LINE_CASE)
#undef TPM_LINE_CASE
    default:
      return fail(TPM_ERR_INVALID, "fft3d: no line plan for this mesh");
  }
}

bool plan_radices(int N, FftPlan& p) {
  p.N = N;
  p.nrad = 0;
  int n = N;
  for (int r : {16, 8, 4, 3, 5, 2}) {
    while (n % r == 0) {
      if (p.nrad >= 12) return false;
      p.rad[p.nrad++] = r;
      n /= r;
    }
  }
  uint64_t Ns = 1;
  for (int s = 0; s < p.nrad; s++) {
    // the first stage (Ns = 1) needs no division; 2^32 does not fit
    p.ns_inv[s] = Ns == 1 ? 0u : (unsigned)(((1ull << 32) + Ns - 1) / Ns);
    Ns *= p.rad[s];
  }
  return n == 1;
}

size_t fft_smem(int N) { return sizeof(float2) * (2 * (size_t)kFftLines * (N + 16 / kFftLines) + N); }

// The dynamic shared-memory limit of the transform kernels is one setting
// per kernel for the whole process, so it is set before every solve: a
// context with a smaller mesh must not lower it for another one.
int set_fft_smem(size_t smem) {
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_fft_z_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_fft_y<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_fft_y<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_fft_x_green, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TPM_CUDA_TRY(cudaFuncSetAttribute(k_fft_z_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return TPM_OK;
}

// x-planes per launch of the z / y passes: the fft_group option, else all
// of them.  Groups whose spectrum stays in L2 between the two passes were
// measured slower at 768^3 (13 planes: z + y forward 4.22 ms against 3.21 ms
// as whole passes): the short launches leave partial waves and gaps.
int plane_group(const tpm_ctx* c, int N) {
  if (c->opt.fft_group > 0) return std::min(c->opt.fft_group, N);
  return N;
}

}  // namespace

int fft3d_padded_columns(int N) { return ((N / 2 + 1) + kLineCols - 1) / kLineCols * kLineCols; }

bool fft3d_supported(int N) {
  FftPlan p;
  return N >= 16 && N <= kFftMaxN && N % 16 == 0 && plan_radices(N, p);
}

int fft3d_init(tpm_ctx* c) {
  const int N = c->N;
  // [0, N): exp(-2 pi i m / N) for the block engine; [N, 2N) and [2N, 3N):
  // the line engine's stage tables of its plan and of the reversed plan,
  // entry Ns - 1 + k (R - 1) + r - 1 of a stage of radix R after Ns points =
  // exp(-2 pi i k r / (Ns R)), k < Ns, 0 < r < R (the stages' Ns (R - 1)
  // entries add up to N - 1).  All in FP64.
  std::vector<float2> tw(3 * (size_t)N, make_float2(0.f, 0.f));
  for (int m = 0; m < N; m++) {
    const double a = -2.0 * M_PI * (double)m / (double)N;
    tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  if (line_supported(N)) {
    const LinePlan plans[2] = {line_plan(N), reverse_plan(line_plan(N))};
    for (int pi = 0; pi < 2; pi++) {
      const LinePlan& P = plans[pi];
      float2* t = tw.data() + (size_t)(pi + 1) * N;
      int ns = 1;
      for (int s = 0; s < P.ns; s++) {
        const int R = P.rad[s];
        for (int k = 0; k < ns; k++)
          for (int r = 1; r < R; r++) {
            const double a = -2.0 * M_PI * (double)k * r / ((double)ns * R);
            t[ns - 1 + k * (R - 1) + r - 1] = make_float2((float)std::cos(a), (float)std::sin(a));
          }
        ns *= R;
      }
    }
  }
  TPM_CUDA_TRY(cudaMemcpy(c->fft_tw, tw.data(), sizeof(float2) * 3 * N, cudaMemcpyHostToDevice));
  // padding columns stay zero: the transforms keep them zero and never store them into phi
  if (c->rhok) TPM_CUDA_TRY(cudaMemset(c->rhok, 0, sizeof(float2) * (size_t)N * N * fft3d_padded_columns(N)));
  const int smem = (int)fft_smem(N);
  return set_fft_smem(smem);
}

int fft3d_poisson(tpm_ctx* c, const float* gt) {
  const int N = c->N;
  FftPlan p;
  plan_radices(N, p);
  p.Sz = fft3d_padded_columns(N);
  float2* Y = reinterpret_cast<float2*>(c->rhok);
  const float norm = (float)(1.0 / ((double)N * N * N));
  if (c->opt.fft != TPM_FFT_BLOCK && line_supported(N)) return line_dispatch(c, Y, p.Sz, gt, norm);
  const size_t smem = fft_smem(N);
  const int rca = set_fft_smem(smem);
  if (rca) return rca;
  cudaStream_t s = c->stream;
  const unsigned zblocks = (unsigned)(N * (N / (2 * kFftLines)));
  const unsigned cblocks = (unsigned)(N * (p.Sz / kFftLines));
  stage_begin(c, kStFftF);
  // The z and y passes work plane by plane in x: launched a group of planes
  // at a time, the spectrum one z pass writes is still in L2 when the y pass
  // reads it (and the inverse y pass output when the z pass reads it), so
  // those intermediates make no round trip through HBM.
  const int G = plane_group(c, N);
  const unsigned zper = (unsigned)(N / (2 * kFftLines)), cper = (unsigned)(p.Sz / kFftLines);
  for (int x0 = 0; x0 < N; x0 += G) {
    const int g = std::min(G, N - x0);
    k_fft_z_r2c<<<zper * g, kFftThreads, smem, s>>>(c->rho, Y, p, c->fft_tw, x0);
    k_fft_y<-1><<<cper * g, kFftThreads, smem, s>>>(Y, p, c->fft_tw, x0);
    c->launches += 2;
  }
  (void)zblocks;
  stage_end(c, kStFftF);
  stage_begin(c, kStGreen);
  k_fft_x_green<<<cblocks, kFftThreads, smem, s>>>(Y, p, c->fft_tw, gt, c->k2tab, norm);
  stage_end(c, kStGreen);
  stage_begin(c, kStFftI);
  for (int x0 = 0; x0 < N; x0 += G) {
    const int g = std::min(G, N - x0);
    k_fft_y<1><<<cper * g, kFftThreads, smem, s>>>(Y, p, c->fft_tw, x0);
    k_fft_z_c2r<<<zper * g, kFftThreads, smem, s>>>(Y, c->phi, p, c->fft_tw, x0);
    c->launches += 2;
  }
  stage_end(c, kStFftI);
  c->launches += 1;
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

}  // namespace tpm
