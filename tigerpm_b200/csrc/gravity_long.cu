// gravity_long.cu -- long-range PM solve on the device.
//
// Reference: gravity_long_compute (src/gravity_long.cpp:36-48) =
//   compute_source (cloud4 deposit x 4 pi N, :142-199)
//   -> fft3d_execute (unnormalised r2c, src/fft.cpp:51-67)
//   -> apply_laplacian (-1/k^2 * exp(-k^2 rs^2) * sinc(k/2)^-4, :201-245)
//   -> fft3d_inv_execute (1/N^3 overall, src/fft.cpp:69-84,468,512)
//   -> get_phi (:247-256).
//
// Device design:
//  * deposit: "owner computes" mesh tiles.  One block owns a T^3 tile of the
//    grid, reads the particles of the chain cells whose assignment stencils
//    can reach it (particles are already in chain-cell order), compacts the
//    ones that reach it into a shared list and accumulates their weights in
//    shared memory; each grid point is written once, with no global atomics
//    and no zeroing pass.  Accumulation is FP32 shared atomics by default;
//    deterministic_deposit selects exact 40-bit fixed point in int64, or
//    26-bit fixed point with native 32-bit shared integer adds (a tile that
//    could overflow is deposited again with FP32 atomics); integer sums are
//    bit-for-bit reproducible whatever the thread order.
//  * FFT: the library's own five-pass transforms (fft3d.cu) for meshes of
//    the form 2^a 3^b 5^c that are multiples of 16, else (or with fft =
//    cufft) cuFFT r2c / c2r around k_green; each timed as its own stages.
//  * Green's function: exp(-k^2 rs^2) * sinc(k/2)^-p factorises per axis, so
//    a per-index table (built in FP64 on the host) and k^2 = kx^2+ky^2+kz^2
//    give G on the fly: one read + one write of the complex grid.
#include "tpm_internal.cuh"

#include <cmath>
#include <type_traits>

namespace tpm {
namespace {

// Per-axis assignment weights from the exact fixed-point split of X*N into
// cell index I and fraction f (raw * N = I * 2^32 + frac).  Returns the first
// stencil index (unwrapped).
//  cloud4 (the reference): points I-1..I+2, cubic B-spline of the distance
//    (src/gravity_long.cpp:127-138,176-181: I_ref = int(XN + 2) - 3 = I - 1);
//  CIC: points I, I+1; TSC: points I0-1..I0+1 with I0 = round(XN).
template <int ASSIGN>
__device__ __forceinline__ int stencil(uint32_t raw, int N, float* w) {
  const uint64_t t = (uint64_t)raw * (uint64_t)N;
  const int I = (int)(t >> 32);
  const float f = (float)(uint32_t)t * 2.3283064365386963e-10f;
  if (ASSIGN == TPM_ASSIGN_CLOUD4) {
    const float g = 1.0f - f;
    const float s6 = 1.0f / 6.0f;
    w[0] = s6 * g * g * g;
    w[1] = s6 * (4.0f - 6.0f * f * f + 3.0f * f * f * f);
    w[2] = s6 * (4.0f - 6.0f * g * g + 3.0f * g * g * g);
    w[3] = s6 * f * f * f;
    return I - 1;
  } else if (ASSIGN == TPM_ASSIGN_CIC) {
    w[0] = 1.0f - f;
    w[1] = f;
    return I;
  } else {
    const int up = f >= 0.5f ? 1 : 0;
    const float d = f - (float)up;
    w[0] = 0.5f * (0.5f - d) * (0.5f - d);
    w[1] = 0.75f - d * d;
    w[2] = 0.5f * (0.5f + d) * (0.5f + d);
    return I + up - 1;
  }
}

// Offset of the first stencil point from floor(X N) before the TSC
// rounding: cloud4 starts at I - 1, CIC at I, TSC at I - 1 or I (taken as
// I - 1 with one extra point of reach in touches()).
template <int ASSIGN>
constexpr int kStencilOff = ASSIGN == TPM_ASSIGN_CIC ? 0 : -1;

// Does a run of W (+1 for TSC's rounding) points starting at d (relative to
// the tile origin, any integer) meet [0, ext) on a periodic axis of N?
template <int W>
__device__ __forceinline__ bool touches(int d, int N, int ext) {
  if (d < 0) d += N;  // d = stencil start (-1 .. N+1) minus a tile origin in [0, N)
  if (d >= N) d -= N;
  return d < ext || d + W + 1 > N;
}

template <int ASSIGN>
struct Width {
  static constexpr int W = ASSIGN == TPM_ASSIGN_CLOUD4 ? 4 : (ASSIGN == TPM_ASSIGN_CIC ? 2 : 3);
};

struct DepositArgs {
  const int4* __restrict__ pos4;
  const int32_t* __restrict__ begin;
  int C;
  int N;
  int ntile;     // tiles per side
  double scale;  // 4 pi N (times the accumulator's fixed-point unit)
  float* __restrict__ rho;
};

// Accumulator of one tile point.
//  kDepF32 (default): FP32 shared atomics (compare-and-swap loops; the
//    rounding depends on the order in which threads reach a point).
//  kDepI32 (TPM_DEPOSIT_FIXED32): 26-bit fixed point in uint32 with the
//    native shared integer add; sums are order independent.  Weights
//    are at most 1, so an add never carries a point past 2^32 without some
//    earlier value at or above 2^30: every add returns the old value, and a
//    tile where any old value reached 2^30 (16 weight units at one point) is
//    deposited again with kDepF32.
//  kDepI64 (TPM_DEPOSIT_EXACT64): exact 40-bit fixed point in int64.
constexpr int kDepF32 = 0, kDepI64 = 1, kDepI32 = 2;
constexpr int kDep32FracBits = 26;
template <int M>
struct DepAcc;
template <>
struct DepAcc<kDepI64> {
  using T = unsigned long long;
  static __device__ __forceinline__ void add(T* p, float w, unsigned&) {
    atomicAdd(p, (unsigned long long)__float2ll_rn(w * 1099511627776.0f));
  }
  static __device__ __forceinline__ double value(T v, double scale) {
    return (double)(long long)v * scale * 9.094947017729282e-13;  // 2^-40
  }
};
template <>
struct DepAcc<kDepF32> {
  using T = float;
  static __device__ __forceinline__ void add(T* p, float w, unsigned&) { atomicAdd(p, w); }
  static __device__ __forceinline__ double value(T v, double scale) { return (double)v * scale; }
};
template <>
struct DepAcc<kDepI32> {
  using T = unsigned;
  static __device__ __forceinline__ void add(T* p, float w, unsigned& hi) {
    hi |= atomicAdd(p, __float2uint_rn(w * 67108864.0f));  // 2^26
  }
  static __device__ __forceinline__ double value(T v, double scale) {
    return (double)v * scale * 1.4901161193847656e-08;  // 2^-26
  }
};
static_assert(kDep32FracBits == 26 && kDepositFracBits == 40, "fixed-point scales above");

// The candidates of a tile (the particles of the chain cells that can reach
// it: 9 to 16 rows of 3 to 4 x cells, up to twice 8x the tile's own) are one
// flat index space over at most kDepRuns contiguous runs; each thread loads
// kDepBatch candidates at a time (independent loads in flight), and the
// reaching ones are compacted into a shared list of up to kDepList particle
// indices before they are deposited, so that every thread of the block
// deposits an equal share.
constexpr int kDepThreads = 256;
constexpr int kDepBatch = 4;
constexpr int kDepList = 2048;
constexpr int kDepRuns = 64;

// Weights of one particle added to the tile (stencil origin o, extent ext);
// hi collects the old values of kDepI32 adds.
template <int T, int ASSIGN, int M>
__device__ __forceinline__ void deposit_particle(typename DepAcc<M>::T* acc, int4 q, int N, const int (&o)[3],
                                                 const int (&ext)[3], unsigned& hi) {
  constexpr int W = Width<ASSIGN>::W;
  using A = DepAcc<M>;
  float wx[4], wy[4], wz[4];
  int r[3];
  r[0] = stencil<ASSIGN>((uint32_t)q.x, N, wx) - o[0];
  r[1] = stencil<ASSIGN>((uint32_t)q.y, N, wy) - o[1];
  r[2] = stencil<ASSIGN>((uint32_t)q.z, N, wz) - o[2];
  int li[3][4];
#pragma unroll
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int k = 0; k < W; k++) {
      int l = r[d] + k;
      if (l < 0) l += N;
      else if (l >= N) l -= N;
      li[d][k] = l < ext[d] ? l : -1;
    }
  }
#pragma unroll
  for (int i = 0; i < W; i++) {
    if (li[0][i] < 0) continue;
#pragma unroll
    for (int j = 0; j < W; j++) {
      if (li[1][j] < 0) continue;
      const float wxy = wx[i] * wy[j];
      typename A::T* row_acc = acc + (li[0][i] * T + li[1][j]) * T;
#pragma unroll
      for (int k = 0; k < W; k++) {
        if (li[2][k] < 0) continue;
        A::add(row_acc + li[2][k], wxy * wz[k], hi);
      }
    }
  }
}

template <int T, int ASSIGN, int M>
__global__ void __launch_bounds__(kDepThreads, 3) k_deposit(DepositArgs a) {
  constexpr int W = Width<ASSIGN>::W;
  extern __shared__ __align__(16) unsigned char dep_smem[];
  // the list follows the tile (a kDepF32 redo of a kDepI32 tile uses the
  // same 4-byte points)
  int32_t* s_list = reinterpret_cast<int32_t*>(dep_smem + sizeof(typename DepAcc<M>::T) * T * T * T);
  __shared__ int s_n;
  // run start particle, run length, candidate offset of each run
  __shared__ int32_t s_rb[kDepRuns], s_len[kDepRuns], s_rp[kDepRuns + 1];
  static_assert(kDepRuns == 64, "two runs per lane of one warp");
  const int lane = threadIdx.x & 31;
  const int N = a.N, C = a.C;
  int tb = blockIdx.x;
  const int tz = tb % a.ntile;
  tb /= a.ntile;
  const int ty = tb % a.ntile;
  const int tx = tb / a.ntile;
  const int o[3] = {tx * T, ty * T, tz * T};
  int ext[3];
  for (int d = 0; d < 3; d++) ext[d] = min(T, N - o[d]);
  // chain cells whose particles can reach the tile: XN in [o-2, o+T+1)
  int clo[3], cnt[3];
  for (int d = 0; d < 3; d++) {
    const int lo = (int)floor(((double)o[d] - 2.001) * C / N);
    const int hi = (int)floor(((double)o[d] + T + 1.001) * C / N);
    clo[d] = lo;
    cnt[d] = min(hi - lo + 1, C);
    if (cnt[d] == C) clo[d] = 0;
  }
  // The whole tile with accumulator mode MODE (its zeroing, the candidate
  // scan and the deposits); returns, for kDepI32, whether a point may have
  // overflowed.
  auto deposit_tile = [&](auto mode) -> bool {
  constexpr int MODE = decltype(mode)::value;
  using A = DepAcc<MODE>;
  typename A::T* acc = reinterpret_cast<typename A::T*>(dep_smem);
  for (int i = threadIdx.x; i < T * T * T; i += blockDim.x) acc[i] = 0;
  if (threadIdx.x == 0) s_n = 0;
  unsigned hi = 0;
  __syncthreads();
  // Deposit the listed particles, all threads sharing the list; called by
  // every thread with the list complete (after a barrier).  The list holds
  // particles in their sorted (spatially compact) order.  Consecutive
  // entries go to consecutive lanes for the integer adds; the FP32 shared
  // atomics are compare-and-swap loops that retry while lanes of a warp hit
  // the same point, so there the 32 lanes of a warp take entries
  // S = ceil(n / 32) apart (slot u = lane + 32 c takes entry lane S + c, a
  // bijection onto [0, n) over u < 32 S).
  auto flush = [&]() {
    const int n = s_n;
    const int S = MODE == kDepF32 ? (n + 31) >> 5 : 0;
    const int slots = MODE == kDepF32 ? 32 * S : n;
    for (int u = threadIdx.x; u < slots; u += kDepThreads) {
      const int e = MODE == kDepF32 ? (u & 31) * S + (u >> 5) : u;
      if (e < n) deposit_particle<T, ASSIGN, MODE>(acc, __ldg(a.pos4 + s_list[e]), N, o, ext, hi);
    }
    __syncthreads();
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
  };
  // x cells clo..clo+cnt-1 (mod C) of a (z, y) row: one or two contiguous runs
  const int x0 = wrapi(clo[0], C);
  const int xend = x0 + cnt[0];
  const int nparts = xend > C ? 2 : 1;
  const int nrows = cnt[2] * cnt[1];
  constexpr int kRowsPerBatch = kDepRuns / 2;
  for (int row0 = 0; row0 < nrows; row0 += kRowsPerBatch) {
    // run table of rows [row0, row0 + kRowsPerBatch): run t = row t / 2,
    // part t % 2 (empty where the row or the part does not exist), lengths
    // turned into candidate offsets by a warp scan
    if (threadIdx.x < kDepRuns) {
      const int t = threadIdx.x, rw = row0 + (t >> 1), part = t & 1;
      int32_t pb = 0, len = 0;
      if (rw < nrows && part < nparts) {
        const int cz = wrapi(clo[2] + rw / cnt[1], C), cy = wrapi(clo[1] + rw % cnt[1], C);
        const int64_t row = ((int64_t)cz * C + cy) * C;
        const int ca = part == 0 ? x0 : 0, cb = part == 0 ? min(xend, C) : xend - C;
        pb = __ldg(a.begin + row + ca);
        len = __ldg(a.begin + row + cb) - pb;
      }
      s_rb[t] = pb;
      s_len[t] = len;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int l = threadIdx.x;
      const int32_t a0 = s_len[2 * l], a1 = s_len[2 * l + 1];
      int32_t incl = a0 + a1;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int32_t v = __shfl_up_sync(0xffffffffu, incl, off);
        if (l >= off) incl += v;
      }
      s_rp[2 * l] = incl - a0 - a1;
      s_rp[2 * l + 1] = incl - a1;
      if (l == 31) s_rp[kDepRuns] = incl;
    }
    __syncthreads();
    const int total = s_rp[kDepRuns];
    int r = 0;  // this thread's run: candidates only increase
    for (int base = 0; base < total; base += kDepThreads * kDepBatch) {
      int32_t idx[kDepBatch];
      int4 q[kDepBatch];
#pragma unroll
      for (int b = 0; b < kDepBatch; b++) {
        const int cnd = base + b * kDepThreads + (int)threadIdx.x;
        idx[b] = -1;
        if (cnd < total) {
          while (s_rp[r + 1] <= cnd) r++;
          idx[b] = s_rb[r] + (cnd - s_rp[r]);
          q[b] = __ldg(a.pos4 + idx[b]);
        }
      }
      int end = 0;
#pragma unroll
      for (int b = 0; b < kDepBatch; b++) {
        bool reach = false;
        if (idx[b] >= 0) {
          // first stencil point per dim relative to the tile, wrapped into
          // [-N/2, N/2): the particle reaches the tile only if every dim's
          // W points meet [0, ext)
          const int s0 = (int)(((uint64_t)(uint32_t)q[b].x * (uint64_t)N) >> 32) + kStencilOff<ASSIGN>;
          const int s1 = (int)(((uint64_t)(uint32_t)q[b].y * (uint64_t)N) >> 32) + kStencilOff<ASSIGN>;
          const int s2 = (int)(((uint64_t)(uint32_t)q[b].z * (uint64_t)N) >> 32) + kStencilOff<ASSIGN>;
          reach = touches<W>(s0 - o[0], N, ext[0]) && touches<W>(s1 - o[1], N, ext[1]) &&
                  touches<W>(s2 - o[2], N, ext[2]);
        }
        // append to the list: one counter update per warp
        const unsigned m = __ballot_sync(0xffffffffu, reach);
        if (m) {
          int b0 = 0;
          if (lane == 0) b0 = atomicAdd(&s_n, __popc(m));
          b0 = __shfl_sync(0xffffffffu, b0, 0);
          if (reach) s_list[b0 + __popc(m & ((1u << lane) - 1u))] = idx[b];
          end = max(end, b0 + __popc(m));
        }
      }
      // the list holds at most kDepList - kDepThreads kDepBatch entries
      // before a batch: deposit it once the next batch could overflow it
      // (the warp that appended last knows the list's length)
      if (__syncthreads_or(end > kDepList - kDepThreads * kDepBatch)) flush();
    }
    __syncthreads();  // the run table is rebuilt for the next rows
  }
  if (s_n > 0) flush();
  if constexpr (MODE == kDepI32) return __syncthreads_or(hi >= (1u << 30)) != 0;
  __syncthreads();
  return false;
  };
  auto store_tile = [&](auto mode) {
    constexpr int MODE = decltype(mode)::value;
    using A = DepAcc<MODE>;
    const typename A::T* acc = reinterpret_cast<const typename A::T*>(dep_smem);
    for (int i = threadIdx.x; i < T * T * T; i += blockDim.x) {
      const int lz = i % T, ly = (i / T) % T, lx = i / (T * T);
      if (lx < ext[0] && ly < ext[1] && lz < ext[2])
        a.rho[((int64_t)(o[0] + lx) * N + (o[1] + ly)) * N + (o[2] + lz)] = (float)A::value(acc[i], a.scale);
    }
  };
  if (deposit_tile(std::integral_constant<int, M>{})) {
    deposit_tile(std::integral_constant<int, kDepF32>{});
    store_tile(std::integral_constant<int, kDepF32>{});
  } else {
    store_tile(std::integral_constant<int, M>{});
  }
}

__global__ void k_green(cufftComplex* __restrict__ Y, const float* __restrict__ gtab,
                        const float* __restrict__ k2tab, int N, int Nh, float norm) {
  const int64_t total = (int64_t)N * N * Nh;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int i2 = (int)(i % Nh);
    const int64_t r = i / Nh;
    const int i1 = (int)(r % N);
    const int i0 = (int)(r / N);
    const float k2 = __ldg(k2tab + i0) + __ldg(k2tab + i1) + __ldg(k2tab + i2);
    const float g = k2 > 0.0f ? -(__ldg(gtab + i0) * __ldg(gtab + i1) * __ldg(gtab + i2)) / k2 * norm : 0.0f;
    cufftComplex y = Y[i];
    y.x *= g;
    y.y *= g;
    Y[i] = y;
  }
}

__global__ void k_get_phi(const float* __restrict__ phi, int N, int b0, int b1, int b2, int s0, int s1,
                          int s2, float* __restrict__ out) {
  const int64_t total = (int64_t)s0 * s1 * s2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int i2 = (int)(i % s2);
    const int64_t r = i / s2;
    const int i1 = (int)(r % s1);
    const int i0 = (int)(r / s1);
    const int g0 = wrapi(b0 + i0, N), g1 = wrapi(b1 + i1, N), g2 = wrapi(b2 + i2, N);
    out[i] = phi[((int64_t)g0 * N + g1) * N + g2];
  }
}

// gravity_long_force_at (src/gravity_long.cpp:52-125): 4-point cubic
// interpolation weights and derivatives in double, periodic grid.
__global__ void k_force_at(const float* __restrict__ phi, int N, int64_t n, const double* __restrict__ pos,
                           float* __restrict__ phi_out, float* __restrict__ g_out) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double X[3], w[3][4], dw[3][4];
  int I[3];
  for (int d = 0; d < 3; d++) {
    X[d] = pos[3 * p + d] * N;
    I[d] = (int)X[d];
    X[d] -= (double)I[d];
    I[d] -= 1;
    const double x1 = X[d], x2 = x1 * x1, x3 = x1 * x2;
    w[d][0] = -0.5 * x1 + x2 - 0.5 * x3;
    w[d][1] = 1.0 - 2.5 * x2 + 1.5 * x3;
    w[d][2] = 0.5 * x1 + 2.0 * x2 - 1.5 * x3;
    w[d][3] = -0.5 * x2 + 0.5 * x3;
    dw[d][0] = -0.5 + 2.0 * x1 - 1.5 * x2;
    dw[d][1] = -5.0 * x1 + 4.5 * x2;
    dw[d][2] = 0.5 + 4.0 * x1 - 4.5 * x2;
    dw[d][3] = -x1 + 1.5 * x2;
  }
  double g[3] = {0, 0, 0}, ph = 0;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++)
      for (int c = 0; c < 4; c++) {
        const double v =
            phi[((int64_t)wrapi(I[0] + a, N) * N + wrapi(I[1] + b, N)) * N + wrapi(I[2] + c, N)];
        g[0] += dw[0][a] * w[1][b] * w[2][c] * v * N;
        g[1] += w[0][a] * dw[1][b] * w[2][c] * v * N;
        g[2] += w[0][a] * w[1][b] * dw[2][c] * v * N;
        ph += w[0][a] * w[1][b] * w[2][c] * v;
      }
  phi_out[p] = (float)ph;
  for (int d = 0; d < 3; d++) g_out[3 * p + d] = (float)(-g[d]);
}

template <int T, int M>
int launch_deposit_T(tpm_ctx* c, DepositArgs a) {
  a.ntile = ceil_div(c->N, T);
  const int blocks = a.ntile * a.ntile * a.ntile;
  const size_t smem = sizeof(typename DepAcc<M>::T) * T * T * T + sizeof(int32_t) * kDepList;
  a.scale = 4.0 * M_PI * c->N;
  switch (c->opt.assign) {
    case TPM_ASSIGN_CIC:
      TPM_CUDA_TRY(cudaFuncSetAttribute(k_deposit<T, TPM_ASSIGN_CIC, M>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_deposit<T, TPM_ASSIGN_CIC, M><<<blocks, 256, smem, c->stream>>>(a);
      break;
    case TPM_ASSIGN_TSC:
      TPM_CUDA_TRY(cudaFuncSetAttribute(k_deposit<T, TPM_ASSIGN_TSC, M>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_deposit<T, TPM_ASSIGN_TSC, M><<<blocks, 256, smem, c->stream>>>(a);
      break;
    default:
      TPM_CUDA_TRY(cudaFuncSetAttribute(k_deposit<T, TPM_ASSIGN_CLOUD4, M>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_deposit<T, TPM_ASSIGN_CLOUD4, M><<<blocks, 256, smem, c->stream>>>(a);
      break;
  }
  c->launches++;
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

}  // namespace

int mesh_init(tpm_ctx* c) {
  const int N = c->N;
  const int Nh = N / 2 + 1;
  // Per-index factor exp(-k^2 rs^2) * sinc(k/2)^-p and k^2, k = 2 pi i / N
  // with i >= N/2 folded negative (src/gravity_long.cpp:214-239), built in FP64.
  std::vector<float> g(N), g_pm(N), k2(N);
  const double rs_cells = c->rs_box * N;
  int p = c->opt.deconv_order;
  if (p <= 0) p = c->opt.assign == TPM_ASSIGN_CIC ? 2 : (c->opt.assign == TPM_ASSIGN_TSC ? 3 : 4);
  for (int i = 0; i < N; i++) {
    const double k = (i < N / 2.0 ? i : i - N) * 2.0 * M_PI / N;
    const double x = 0.5 * k;
    const double s = x != 0.0 ? std::sin(x) / x : 1.0;
    const double dec = std::pow(s, -p);
    g[i] = (float)(std::exp(-k * k * rs_cells * rs_cells) * dec);
    g_pm[i] = (float)dec;
    k2[i] = (float)(k * k);
  }
  TPM_CUDA_TRY(cudaMemcpy(c->gtab, g.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  TPM_CUDA_TRY(cudaMemcpy(c->gtab + N, g_pm.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  TPM_CUDA_TRY(cudaMemcpy(c->k2tab, k2.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  c->use_fft3d = c->opt.fft != TPM_FFT_CUFFT && fft3d_supported(N);
  if (c->use_fft3d) return fft3d_init(c);
  TPM_CUFFT_TRY(cufftPlan3d(&c->plan_r2c, N, N, N, CUFFT_R2C));
  TPM_CUFFT_TRY(cufftPlan3d(&c->plan_c2r, N, N, N, CUFFT_C2R));
  TPM_CUFFT_TRY(cufftSetStream(c->plan_r2c, c->stream));
  TPM_CUFFT_TRY(cufftSetStream(c->plan_c2r, c->stream));
  c->plans = true;
  (void)Nh;
  return TPM_OK;
}

int gravity_long(tpm_ctx* c, int type) {
  if (!c->sorted) return fail(TPM_ERR_STATE, "gravity_long_compute needs chainmesh_create first");
  const int N = c->N;
  const int Nh = N / 2 + 1;
  cudaStream_t s = c->stream;
  stage_begin(c, kStDeposit);
  DepositArgs a;
  a.pos4 = c->pos4;
  a.begin = c->cell_begin;
  a.C = c->C;
  a.N = N;
  a.ntile = 0;
  a.scale = 0;
  a.rho = c->rho;
  int rc;
  // tile edge: 24 points on large meshes (fewer redundant particle visits),
  // 16 / 8 on smaller ones; exact (int64) tiles of 24^3 would need 110 KB.
  if (c->opt.deterministic_deposit == TPM_DEPOSIT_EXACT64) {
    rc = N >= 128 ? launch_deposit_T<16, kDepI64>(c, a) : launch_deposit_T<8, kDepI64>(c, a);
  } else if (c->opt.deterministic_deposit == TPM_DEPOSIT_FIXED32) {
    rc = N >= 192 ? launch_deposit_T<24, kDepI32>(c, a)
                  : (N >= 64 ? launch_deposit_T<16, kDepI32>(c, a) : launch_deposit_T<8, kDepI32>(c, a));
  } else {
    rc = N >= 192 ? launch_deposit_T<24, kDepF32>(c, a)
                  : (N >= 64 ? launch_deposit_T<16, kDepF32>(c, a) : launch_deposit_T<8, kDepF32>(c, a));
  }
  if (rc) return rc;
  stage_end(c, kStDeposit);
  if (c->use_fft3d) {
    rc = fft3d_poisson(c, type == TPM_GRAVITY_LONG_PME ? c->gtab : c->gtab + N);
    if (rc) return rc;
    c->have_phi = true;
    return TPM_OK;
  }
  stage_begin(c, kStFftF);
  TPM_CUFFT_TRY(cufftExecR2C(c->plan_r2c, c->rho, c->rhok));
  stage_end(c, kStFftF);
  stage_begin(c, kStGreen);
  const int64_t total = (int64_t)N * N * Nh;
  const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), 148 * 32);
  const float* gt = type == TPM_GRAVITY_LONG_PME ? c->gtab : c->gtab + N;
  k_green<<<blocks, 256, 0, s>>>(c->rhok, gt, c->k2tab, N, Nh, (float)(1.0 / ((double)N * N * N)));
  c->launches++;
  TPM_CUDA_TRY(cudaGetLastError());
  stage_end(c, kStGreen);
  stage_begin(c, kStFftI);
  TPM_CUFFT_TRY(cufftExecC2R(c->plan_c2r, c->rhok, c->phi));
  stage_end(c, kStFftI);
  c->have_phi = true;
  return TPM_OK;
}

int gravity_long_get_phi(tpm_ctx* c, const int box[6], float* out) {
  if (!c->have_phi) return fail(TPM_ERR_STATE, "gravity_long_get_phi needs gravity_long_compute first");
  const int s0 = box[3] - box[0], s1 = box[4] - box[1], s2 = box[5] - box[2];
  if (s0 < 0 || s1 < 0 || s2 < 0) return fail(TPM_ERR_INVALID, "negative box extent");
  const int64_t total = (int64_t)s0 * s1 * s2;
  if (total == 0) return TPM_OK;
  float* d = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(float) * total, c->stream));
  k_get_phi<<<(int)std::min<int64_t>(ceil_div(total, 256), 148 * 16), 256, 0, c->stream>>>(
      c->phi, c->N, box[0], box[1], box[2], s0, s1, s2, d);
  c->launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(float) * total, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("get_phi: ") + cudaGetErrorString(e));
  return TPM_OK;
}

int gravity_long_set_phi(tpm_ctx* c, const float* phi) {
  const size_t bytes = sizeof(float) * (size_t)c->N * c->N * c->N;
  cudaError_t e = cudaMemcpyAsync(c->phi, phi, bytes, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("set_phi: ") + cudaGetErrorString(e));
  c->have_phi = true;
  return TPM_OK;
}

int gravity_long_force_at(tpm_ctx* c, int64_t n, const double* pos, float* phi_out, float* g_out) {
  if (!c->have_phi) return fail(TPM_ERR_STATE, "gravity_long_force_at needs gravity_long_compute first");
  if (n <= 0) return TPM_OK;
  double* dpos = nullptr;
  float* dout = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&dpos, sizeof(double) * 3 * n, c->stream));
  TPM_CUDA_TRY(cudaMallocAsync((void**)&dout, sizeof(float) * 4 * n, c->stream));
  cudaError_t e = cudaMemcpyAsync(dpos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    k_force_at<<<ceil_div(n, 128), 128, 0, c->stream>>>(c->phi, c->N, n, dpos, dout, dout + n);
    c->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(phi_out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g_out, dout + n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(dpos, c->stream);
  cudaFreeAsync(dout, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("force_at: ") + cudaGetErrorString(e));
  return TPM_OK;
}

}  // namespace tpm
