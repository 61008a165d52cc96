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
// the lines per block (4) so that a block's kz columns start on a 32-byte
// boundary (the padding columns are zero and never reach phi).  Each block
// holds 4 lines of length N in shared memory and transforms them with a
// self-sorting (Stockham)
// radix-16/8/4/3/5/2 FFT, each stage from one shared buffer into the other.  Twiddles
// exp(-2 pi i m / N) are computed in FP64 on the host and staged in shared
// memory.  Forward transforms use exp(-i...), inverse exp(+i...), both
// unnormalised (cuFFT's convention); 1/N^3 is folded into the Green's
// function.
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

int fft3d_padded_columns(int N) { return ((N / 2 + 1) + kFftLines - 1) / kFftLines * kFftLines; }

bool fft3d_supported(int N) {
  FftPlan p;
  return N >= 16 && N <= kFftMaxN && N % 16 == 0 && plan_radices(N, p);
}

int fft3d_init(tpm_ctx* c) {
  const int N = c->N;
  std::vector<float2> tw(N);
  for (int m = 0; m < N; m++) {
    const double a = -2.0 * M_PI * (double)m / (double)N;
    tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  TPM_CUDA_TRY(cudaMemcpy(c->fft_tw, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
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
  const size_t smem = fft_smem(N);
  const int rca = set_fft_smem(smem);
  if (rca) return rca;
  cudaStream_t s = c->stream;
  const unsigned zblocks = (unsigned)(N * (N / (2 * kFftLines)));
  const unsigned cblocks = (unsigned)(N * (p.Sz / kFftLines));
  const float norm = (float)(1.0 / ((double)N * N * N));
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
