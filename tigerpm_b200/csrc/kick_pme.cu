// kick_pme.cu -- long-range interpolation, short-range PP and the rung kick.
//
// Reference: kick_pme_kernel (src/kick_pme.cu:128-357) behind the host
// staging of kick_pme (src/kick_pme.cu:390-621).  Per sink: the 6-point
// quintic interpolation of phi and its analytic gradient (:188-263), the
// erfc-split pair sum over every particle of the 27 neighbour chain cells
// (:265-317, erfcexp = A&S 7.1.26, tigerpm/util.hpp:36-59, softened
// polynomial for r <= h), then GM scaling, the FORCE_TEST stores and the
// half-kick / new rung / half-kick update (:319-354).
//
// Device design:
//  * No host staging: particles are already in chain-cell order on the device
//    and the 27 neighbours of a cell are 9 contiguous (z, y) rows of three x
//    cells (two runs where x wraps), read straight from cell offsets.
//  * The interpolation is its own kernel (one block per chain cell), run just
//    before the pair kernel; its results stay in L2 for the kick.
//  * Pair kernel, one block per sink cell.  Sources are staged in shared
//    memory as float offsets from the sink cell centre: the int32
//    wrap-around difference (the reference's periodic minimum image) is taken
//    once per source per block, so the pair loop is pure FP32.
//  * Culling: the cell's sinks (up to 256 per pass) are ordered by a 9-bit
//    Morton key of their position inside the cell (a deterministic bitonic
//    sort) and cut into groups of 8; a warp keeps the sources within the
//    cutoff of a group's bounding box (ballot + popc) in a float4 buffer, and
//    lanes (8 sinks x 4 source phases) evaluate it 32 sources at a time,
//    every lane together: the flush is a warp-uniform branch, pairs go two at
//    a time with one warp vote for the softened kernel.
//  * Pair terms: rsqrt / rcp / ex2 approximations (MUFU) for 1/r, the A&S
//    rational and exp(-x^2), with lengths in units of 2 r_s / sqrt(log2 e)
//    so that exp(-x0^2) = 2^-r2; an optional cutoff zeroes pairs beyond it.
//  * Precision: FP32 pair terms, per-lane FP32 partial sums folded in a fixed
//    order, added per target with Kahan compensation across staged chunks
//    (kahan option).
#include "tpm_internal.cuh"

#include <algorithm>
#include <cmath>

namespace tpm {
namespace {

constexpr int kKickThreads = 256;
// Occupancy settings, measured on B200 at 64 particles per chain cell
// (256^3 particles, 64^3 cells): 64 registers (4 resident 256-thread blocks
// per SM), a staged chunk of half the mean 27-cell neighbourhood and a sink
// pass of the power of two >= the mean cell give 8 resident 128-thread
// blocks and the shortest kick (at the time 18.8 ms against 26.9 ms at 80
// registers and 4 blocks, 20.9 ms at 48 or 40 registers, where the pair
// loop loses ILP).
#ifndef TPM_KICK_MINB
#define TPM_KICK_MINB 4  // resident 256-thread blocks per SM the register budget targets
#endif
#ifndef TPM_KICK_STAGE_X100
#define TPM_KICK_STAGE_X100 50  // staged sources per chunk, in hundredths of the mean 27-cell neighbourhood
#endif
#ifndef TPM_KICK_PASS_X
#define TPM_KICK_PASS_X 1  // 0: 256 sinks per pass; k: the power of two >= k x the mean cell, 64..256
#endif
constexpr int kMaxStage = 4096;  // sources staged per chunk (64 KB)

struct KickArgs {
  const int4* __restrict__ pos4;
  float* __restrict__ vx;
  float* __restrict__ vy;
  float* __restrict__ vz;
  int8_t* __restrict__ rung;
  float* __restrict__ gx;
  float* __restrict__ gy;
  float* __restrict__ gz;
  float* __restrict__ pot;
  const int32_t* __restrict__ begin;
  const uint32_t* __restrict__ thr;  // chain-cell split thresholds (C + 1)
  const float* __restrict__ phi;
  int* __restrict__ err;
  int C, N;
  int b0, b1, b2, s1, s2;
  int min_rung;
  int first_call;
  int kahan;
  float GM, eta, t0, scale, hsoft;
  // pair-loop lengths are in units of u = 2 r_s / sqrt(log2 e) (see pair())
  float inv2rs;  // 1 / (2 r_s), box units
  float lscale;  // 2^-32 / u: fixed32 offset -> scaled length
  float h2;      // (hsoft / u)^2
  float rcut2;   // (r_cut / u)^2, or infinity without a cutoff
  float wlen;    // the box length / u (minimum-image fold, chain_dim = 3)
};

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  const float y = v - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// 6-point quintic weights and derivatives (src/kick_pme.cu:208-231).
__device__ __forceinline__ void q6(float x1, float* w, float* dw) {
  const float x2 = x1 * x1, x3 = x1 * x2, x4 = x2 * x2, x5 = x3 * x2;
  w[0] = (1.f / 12.f) * x1 - (1.f / 24.f) * x2 - (3.f / 8.f) * x3 + (13.f / 24.f) * x4 - (5.f / 24.f) * x5;
  w[1] = -(2.f / 3.f) * x1 + (2.f / 3.f) * x2 + (13.f / 8.f) * x3 - (8.f / 3.f) * x4 + (25.f / 24.f) * x5;
  w[2] = 1.0f - (5.f / 4.f) * x2 - (35.f / 12.f) * x3 + (21.f / 4.f) * x4 - (25.f / 12.f) * x5;
  w[3] = (2.f / 3.f) * x1 + (2.f / 3.f) * x2 + (11.f / 4.f) * x3 - (31.f / 6.f) * x4 + (25.f / 12.f) * x5;
  w[4] = -(1.f / 12.f) * x1 - (1.f / 24.f) * x2 - (11.f / 8.f) * x3 + (61.f / 24.f) * x4 - (25.f / 24.f) * x5;
  w[5] = (7.f / 24.f) * x3 - (0.5f) * x4 + (5.f / 24.f) * x5;
  const float y5 = 5.0f * x4, y4 = 4.0f * x3, y3 = 3.0f * x2, y2 = 2.0f * x1;
  dw[0] = (1.f / 12.f) - (1.f / 24.f) * y2 - (3.f / 8.f) * y3 + (13.f / 24.f) * y4 - (5.f / 24.f) * y5;
  dw[1] = -(2.f / 3.f) + (2.f / 3.f) * y2 + (13.f / 8.f) * y3 - (8.f / 3.f) * y4 + (25.f / 24.f) * y5;
  dw[2] = -(5.f / 4.f) * y2 - (35.f / 12.f) * y3 + (21.f / 4.f) * y4 - (25.f / 12.f) * y5;
  dw[3] = (2.f / 3.f) + (2.f / 3.f) * y2 + (11.f / 4.f) * y3 - (31.f / 6.f) * y4 + (25.f / 12.f) * y5;
  dw[4] = -(1.f / 12.f) - (1.f / 24.f) * y2 - (11.f / 8.f) * y3 + (61.f / 24.f) * y4 - (25.f / 24.f) * y5;
  dw[5] = (7.f / 24.f) * y3 - (0.5f) * y4 + (5.f / 24.f) * y5;
}

// Long-range force and potential at a sink: g = -sum dw.w.w phi N,
// phi = sum w.w.w phi over the 6^3 points I-2..I+3 (periodic).  The cell
// index and fraction come from the exact fixed-point product raw * N.
__device__ __forceinline__ void interp_long(const KickArgs& a, int4 q, float& lx, float& ly, float& lz,
                                            float& lp) {
  const int N = a.N;
  float w[3][kNInterp], dw[3][kNInterp];
  int base[3];
  const uint32_t r[3] = {(uint32_t)q.x, (uint32_t)q.y, (uint32_t)q.z};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const uint64_t t = (uint64_t)r[d] * (uint64_t)N;
    base[d] = (int)(t >> 32) - 2;
    q6((float)(uint32_t)t * 2.3283064365386963e-10f, w[d], dw[d]);
  }
  int iy[kNInterp], iz[kNInterp];
#pragma unroll
  for (int k = 0; k < kNInterp; k++) {
    iy[k] = wrapi(base[1] + k, N) * N;
    iz[k] = wrapi(base[2] + k, N);
  }
  // The sums run over phi minus its value at the stencil's centre point:
  // the derivative weights sum to zero, so the gradient is a difference of
  // nearly equal terms, and removing the common value keeps FP32 from
  // cancelling it away (the weights sum to one, so phi adds it back).
  const float pc = __ldg(a.phi + (int64_t)wrapi(base[0] + 2, N) * N * N + iy[2] + iz[2]);
  float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
  const int z0 = iz[0];
  const int a4 = z0 & ~3;
  if ((N & 3) == 0 && a4 + 12 <= N) {
    // Each z-run of 6 points is read as two aligned float4 (8 points from
    // a4 = z0 rounded down to 4) and, when the run starts at a4 + 3, one
    // more float; the z weights are shifted by s = z0 - a4 once per sink,
    // zero outside the run.
    const int s = z0 - a4;
    float ws[9], dws[9];
#pragma unroll
    for (int m = 0; m < 9; m++) {
      float u = 0.f, du = 0.f;
#pragma unroll
      for (int k = 0; k < kNInterp; k++) {
        const bool hit = m - k == s;
        u = hit ? w[2][k] : u;
        du = hit ? dw[2][k] : du;
      }
      ws[m] = u;
      dws[m] = du;
    }
#pragma unroll 1
    for (int i = 0; i < kNInterp; i++) {
      const int64_t plane = (int64_t)wrapi(base[0] + i, N) * N * N;
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kNInterp; j++) {
        const float4* row = reinterpret_cast<const float4*>(a.phi + plane + iy[j] + a4);
        const float4 f0 = __ldg(row), f1 = __ldg(row + 1);
        const float f8 = s == 3 ? __ldg(reinterpret_cast<const float*>(row + 2)) : pc;
        const float v[9] = {f0.x - pc, f0.y - pc, f0.z - pc, f0.w - pc, f1.x - pc,
                            f1.y - pc, f1.z - pc, f1.w - pc, f8 - pc};
        float rz = 0.f, rdz = 0.f;
#pragma unroll
        for (int m = 0; m < 9; m++) {
          rz = fmaf(ws[m], v[m], rz);
          rdz = fmaf(dws[m], v[m], rdz);
        }
        px = fmaf(w[1][j], rz, px);
        py = fmaf(dw[1][j], rz, py);
        pz = fmaf(w[1][j], rdz, pz);
      }
      sx = fmaf(dw[0][i], px, sx);
      sy = fmaf(w[0][i], py, sy);
      sz = fmaf(w[0][i], pz, sz);
      sp = fmaf(w[0][i], px, sp);
    }
    lx = -sx * (float)N;
    ly = -sy * (float)N;
    lz = -sz * (float)N;
    lp = sp + pc;
    return;
  }
  for (int i = 0; i < kNInterp; i++) {
    const int64_t plane = (int64_t)wrapi(base[0] + i, N) * N * N;
    float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
    for (int j = 0; j < kNInterp; j++) {
      float rz = 0.f, rdz = 0.f;
#pragma unroll
      for (int k = 0; k < kNInterp; k++) {
        const float v = __ldg(a.phi + plane + iy[j] + iz[k]) - pc;
        rz = fmaf(w[2][k], v, rz);
        rdz = fmaf(dw[2][k], v, rdz);
      }
      px = fmaf(w[1][j], rz, px);
      py = fmaf(dw[1][j], rz, py);
      pz = fmaf(w[1][j], rdz, pz);
    }
    sx = fmaf(dw[0][i], px, sx);
    sy = fmaf(w[0][i], py, sy);
    sz = fmaf(w[0][i], pz, sz);
    sp = fmaf(w[0][i], px, sp);
  }
  lx = -sx * (float)N;
  ly = -sy * (float)N;
  lz = -sz * (float)N;
  lp = sp + pc;
}

// Long-range part at every active sink of the kick box, stored in gx/gy/gz/pot
// (unscaled); k_kick_pme adds the pair sums and applies GM.  Two kernels
// compute it, one block per sink cell, chosen by the mesh points per sink.
//
// Direct form: one thread per sink, the 216 points read through L1.
__device__ __forceinline__ void interp_cell_direct(const KickArgs& a, int64_t key, int min_rung) {
  const int32_t pb = __ldg(a.begin + key), pe = __ldg(a.begin + key + 1);
  for (int32_t i = pb + (int32_t)threadIdx.x; i < pe; i += blockDim.x) {
    if (a.rung[i] < min_rung) continue;
    float lx, ly, lz, lp;
    interp_long(a, __ldg(a.pos4 + i), lx, ly, lz, lp);
    a.gx[i] = lx;
    a.gy[i] = ly;
    a.gz[i] = lz;
    a.pot[i] = lp;
  }
}

// 12 resident 64-thread blocks per SM (at most 85 registers): 2.55 ms against
// 2.78 ms with the compiler's own choice at 256^3 on a 768^3 mesh
#ifndef TPM_INTERP_MINB
#define TPM_INTERP_MINB 12
#endif
__global__ void __launch_bounds__(64, TPM_INTERP_MINB) k_interp_direct(KickArgs a) {
  int bid = blockIdx.x;
  const int i2 = bid % a.s2;
  bid /= a.s2;
  const int i1 = bid % a.s1;
  const int i0 = bid / a.s1;
  const int C = a.C;
  interp_cell_direct(a, ((int64_t)(a.b2 + i2) * C + (a.b1 + i1)) * C + (a.b0 + i0), a.min_rung);
}

// The same interpolation from a shared-memory copy of the potential: one
// block per sink cell stages the mesh points every sink of the cell can
// reach (the cell's mesh span plus the stencil's 2 + 3 points per dim),
// then each sink reads its 6^3 points from the tile.  Blocks whose span
// exceeds the tile take the direct path.
__device__ __forceinline__ void interp_tile(const float* __restrict__ tile, int W0, int W1, int W2, int bx, int by,
                                            int bz, int4 q, int N, float& lx, float& ly, float& lz, float& lp) {
  float w[3][kNInterp], dw[3][kNInterp];
  const uint32_t r[3] = {(uint32_t)q.x, (uint32_t)q.y, (uint32_t)q.z};
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const uint64_t t = (uint64_t)r[d] * (uint64_t)N;
    base[d] = (int)(t >> 32) - 2;
    q6((float)(uint32_t)t * 2.3283064365386963e-10f, w[d], dw[d]);
  }
  // sinks of the cell lie inside the tile by construction; the clamp keeps a
  // stale (moved, unsorted) particle inside it as well
  const int ox = min(max(base[0] - bx, 0), W0 - kNInterp);
  const int oy = min(max(base[1] - by, 0), W1 - kNInterp);
  const int oz = min(max(base[2] - bz, 0), W2 - kNInterp);
  // sums over phi minus the stencil's centre value, as in interp_long
  const float pc = tile[(ox + 2) * W1 * W2 + (oy + 2) * W2 + oz + 2];
  float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
  for (int i = 0; i < kNInterp; i++) {
    const float* plane = tile + (ox + i) * W1 * W2 + oy * W2 + oz;
    float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
    for (int j = 0; j < kNInterp; j++) {
      float rz = 0.f, rdz = 0.f;
#pragma unroll
      for (int k = 0; k < kNInterp; k++) {
        const float v = plane[j * W2 + k] - pc;
        rz = fmaf(w[2][k], v, rz);
        rdz = fmaf(dw[2][k], v, rdz);
      }
      px = fmaf(w[1][j], rz, px);
      py = fmaf(dw[1][j], rz, py);
      pz = fmaf(w[1][j], rdz, pz);
    }
    sx = fmaf(dw[0][i], px, sx);
    sy = fmaf(w[0][i], py, sy);
    sz = fmaf(w[0][i], pz, sz);
    sp = fmaf(w[0][i], px, sp);
  }
  lx = -sx * (float)N;
  ly = -sy * (float)N;
  lz = -sz * (float)N;
  lp = sp + pc;
}

__global__ void __launch_bounds__(128) k_interp_tile(KickArgs a, int maxw) {
  extern __shared__ float tile[];
  int bid = blockIdx.x;
  const int i2 = bid % a.s2;
  bid /= a.s2;
  const int i1 = bid % a.s1;
  const int i0 = bid / a.s1;
  const int C = a.C, N = a.N;
  const int cc[3] = {a.b0 + i0, a.b1 + i1, a.b2 + i2};
  const int64_t key = ((int64_t)cc[2] * C + cc[1]) * C + cc[0];
  const int32_t pb = __ldg(a.begin + key), pe = __ldg(a.begin + key + 1);
  if (pb == pe) return;
  int o[3], W[3];
  bool fits = true;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const uint32_t lo_r = __ldg(a.thr + cc[d]);
    const uint32_t hi_r = cc[d] + 1 < C ? __ldg(a.thr + cc[d] + 1) - 1u : 0xffffffffu;
    const int lo = (int)(((uint64_t)lo_r * (uint64_t)N) >> 32);
    const int hi = (int)(((uint64_t)hi_r * (uint64_t)N) >> 32);
    o[d] = lo - 2;
    W[d] = hi - lo + 6;
    fits = fits && W[d] <= maxw;
  }
  if (!fits) {  // uniform per block
    for (int32_t i = pb + (int32_t)threadIdx.x; i < pe; i += blockDim.x) {
      if (a.rung[i] < a.min_rung) continue;
      float lx, ly, lz, lp;
      interp_long(a, __ldg(a.pos4 + i), lx, ly, lz, lp);
      a.gx[i] = lx;
      a.gy[i] = ly;
      a.gz[i] = lz;
      a.pot[i] = lp;
    }
    return;
  }
  const int plane = W[1] * W[2];
  const int vol = W[0] * plane;
  for (int t = threadIdx.x; t < vol; t += blockDim.x) {
    const int u = t / plane, r = t - u * plane;
    const int v = r / W[2], w = r - v * W[2];
    const int64_t g = ((int64_t)wrapi(o[0] + u, N) * N + wrapi(o[1] + v, N)) * N + wrapi(o[2] + w, N);
    tile[t] = __ldg(a.phi + g);
  }
  __syncthreads();
  for (int32_t i = pb + (int32_t)threadIdx.x; i < pe; i += blockDim.x) {
    if (a.rung[i] < a.min_rung) continue;
    float lx, ly, lz, lp;
    interp_tile(tile, W[0], W[1], W[2], o[0], o[1], o[2], __ldg(a.pos4 + i), N, lx, ly, lz, lp);
    a.gx[i] = lx;
    a.gy[i] = ly;
    a.gz[i] = lz;
    a.pot[i] = lp;
  }
}

// Pair constants that stay in registers through the pair loop, in the pair
// loop's length unit u (below): rcut2 and h2 are (r_cut / u)^2 and (h / u)^2;
// wrap_len is the box length in u (minimum-image fold, chain_dim = 3 only).
constexpr float kLog2e = 1.4426950408889634f, kSqrtLog2e = 1.2011224087864498f;
struct PairK {
  float rcut2, h2, wrap_len;
};

// One source against one sink (src/kick_pme.cu:285-314), in three parts:
// the separation and the erfc-split terms, the softened kernel, and the
// sums.  WRAP folds the offset to the minimum image, as the reference's
// int32 difference does; it is needed only when chain_dim = 3, where the 27
// cells span the whole box and an offset from the cell centre can exceed
// half the box.
//
// Lengths are in units of u = 2 r_s / s with s = sqrt(log2 e) (the caller
// scales offsets by 1 / u): r2 = log2(e) x0^2 for x0 = r / (2 r_s), so
// exp(-x0^2) = 2^-r2 takes no multiply.  With x0 = r / s the A&S and
// 2/sqrt(pi) constants are divided by s, and the sums come out as force x
// u^2 and potential x u; the caller multiplies them back.  The softened
// terms are homogeneous in r and h, so their formulas are unchanged.
template <bool WRAP>
__device__ __forceinline__ void pair_terms(const PairK& k, float& dx, float& dy, float& dz, float& r2, float& rinv3,
                                           float& q) {
  if (WRAP) {
    const float inv = 1.0f / k.wrap_len;
    dx -= rintf(dx * inv) * k.wrap_len;
    dy -= rintf(dy * inv) * k.wrap_len;
    dz -= rintf(dz * inv) * k.wrap_len;
  }
  r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  // Pairs beyond the cutoff take r^2 = 1e30: 1/r, erfc and exp(-x^2) then
  // vanish and the pair adds exactly 0, without a mask on the results.
  // Pairs at r <= h (the sink itself included, r = 0) take the softened
  // kernel, which replaces every term formed here.
  const float r2c = r2 < k.rcut2 ? r2 : 1e30f;
  const float rinv = rsqrt_approx(r2c);
  const float r = r2c * rinv;
  // A&S 7.1.26 erfc(x0), t = 1 / (1 + 0.3275911 x0) with x0 = r / s
  const float t = rcp_approx(fmaf(0.2727374808792225f, r, 1.0f));
  const float e = ex2_approx(-r2c);
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
  // potential term erfc / r, and the force term
  // (erfc + (2/sqrt(pi)) x0 e) / r^3 = (erfc / r + (2/sqrt(pi)) e / s) / r^2
  q = poly * e * rinv;
  rinv3 = fmaf(0.9394372786996513f, e, q) * (rinv * rinv);
}

// The softened Newtonian kernel where r <= h (rare), selected per lane.
__device__ __forceinline__ void soften(const PairK& k, float r2, float& rinv3, float& q) {
  const bool soft = r2 <= k.h2;
  const float hinv = rsqrtf(k.h2);
  const float q2 = r2 * hinv * hinv;
  const float s3 = fmaf(fmaf(15.0f / 8.0f, q2, -21.0f / 4.0f), q2, 35.0f / 8.0f) * (hinv * hinv * hinv);
  const float s1 = fmaf(fmaf(fmaf(-5.0f / 16.0f, q2, 21.0f / 16.0f), q2, -35.0f / 16.0f), q2, 35.0f / 16.0f) * hinv;
  rinv3 = soft ? s3 : rinv3;
  q = soft ? s1 : q;
}

__device__ __forceinline__ void add_pair(float dx, float dy, float dz, float rinv3, float q, float& gx, float& gy,
                                         float& gz, float& ph) {
  gx = fmaf(-dx, rinv3, gx);
  gy = fmaf(-dy, rinv3, gy);
  gz = fmaf(-dz, rinv3, gz);
  ph -= q;
}

// One pair, the softened kernel behind a per-lane branch (any caller).
template <bool WRAP>
__device__ __forceinline__ void pair(const PairK& k, float dx, float dy, float dz, float& gx, float& gy, float& gz,
                                     float& ph) {
  float r2, rinv3, q;
  pair_terms<WRAP>(k, dx, dy, dz, r2, rinv3, q);
  if (r2 <= k.h2) soften(k, r2, rinv3, q);
  add_pair(dx, dy, dz, rinv3, q, gx, gy, gz, ph);
}

// Two pairs of one sink, evaluated by every lane of the warp together: the
// softened kernel is entered on one warp vote for both (a uniform branch),
// and the sums take the first pair, then the second.
template <bool WRAP>
__device__ __forceinline__ void pair2(const PairK& k, const float4& sp, const float4 u0, const float4 u1, float& gx,
                                      float& gy, float& gz, float& ph) {
  float dx0 = sp.x - u0.x, dy0 = sp.y - u0.y, dz0 = sp.z - u0.z;
  float dx1 = sp.x - u1.x, dy1 = sp.y - u1.y, dz1 = sp.z - u1.z;
  float r20, rinv30, q0, r21, rinv31, q1;
  pair_terms<WRAP>(k, dx0, dy0, dz0, r20, rinv30, q0);
  pair_terms<WRAP>(k, dx1, dy1, dz1, r21, rinv31, q1);
  if (__any_sync(0xffffffffu, r20 <= k.h2 || r21 <= k.h2)) {
    soften(k, r20, rinv30, q0);
    soften(k, r21, rinv31, q1);
  }
  add_pair(dx0, dy0, dz0, rinv30, q0, gx, gy, gz, ph);
  add_pair(dx1, dy1, dz1, rinv31, q1, gx, gy, gz, ph);
}

// Offset a - b of two fixed32 coordinates (the reference's int32 wrap-around
// difference) times a length scale.
__device__ __forceinline__ float offset_scaled(uint32_t a, uint32_t b, float sc) {
  return (float)(int32_t)(a - b) * sc;
}

// 3-bit-per-axis sub-cell index of an offset (in box units) from the cell
// centre, interleaved into a 9-bit Morton key.
__device__ __forceinline__ unsigned morton9(float sx, float sy, float sz, float C) {
  unsigned q[3];
  const float s[3] = {sx, sy, sz};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int v = (int)((s[d] * C + 0.5f) * 8.0f);
    q[d] = (unsigned)min(max(v, 0), 7);
  }
  unsigned k = 0;
#pragma unroll
  for (int b = 2; b >= 0; b--) k = (k << 3) | (((q[2] >> b) & 1u) << 2) | (((q[1] >> b) & 1u) << 1) | ((q[0] >> b) & 1u);
  return k;
}

// Work decomposition.  A block owns one sink cell.  Its active sinks (up to
// kPass per pass) are sorted by a 9-bit Morton key of their position in the
// cell, then cut into groups of kGroup = 8 consecutive sinks (compact in
// space).  Warps take groups round-robin.  For each group a warp streams the
// staged neighbourhood, keeps the sources within rcut of the group's bounding
// box (ballot + popc) and copies them contiguously into its float4 buffer;
// lanes are (sink t = lane % 8) x (phase = lane / 8), so one step evaluates 8
// sinks against 4 consecutive buffered sources (conflict-free broadcast-free
// reads) and a fixed two-step shuffle reduction folds the 4 phases.  Per-sink
// sums live in shared memory with Kahan compensation across chunks.
//
// Shared memory (dynamic): src[stage] float4 | buf[W][kBuf] float4 |
// spos[kPass] float4 | acc[kPass][8] float | skey[kPass] | runb/runp.
constexpr int kPass = 256;
constexpr int kGroup = 8;
constexpr int kBuf = 64;
constexpr int kMaxRuns = 18;

// The kick of sink passes [pass_lo, pass_hi) of one sink cell (cx, cy, cz)
// by the calling block (a pass = the cell's sinks taken np at a time, np =
// the power of two >= the cell's count, at most npass); every thread of the
// block calls it with the same arguments.  A pass streams the whole 27-cell
// neighbourhood, so the passes of one cell are independent work items.
template <bool WRAP>
__device__ __forceinline__ void kick_cell(const KickArgs& a, int cx, int cy, int cz, float4* smem4, int stage,
                                          int npass, int pass_lo = 0, int pass_hi = 0x7fffffff) {
  const int T = blockDim.x, W = T >> 5;
  float4* src = smem4;
  float4* bufs = src + stage;
  float4* spos = bufs + W * kBuf;
  float* acc = reinterpret_cast<float*>(spos + npass);
  unsigned* skey = reinterpret_cast<unsigned*>(acc + npass * 8);
  int* runb = reinterpret_cast<int*>(skey + npass);
  int* runp = runb + kMaxRuns;
  const int C = a.C;
  const int64_t key = ((int64_t)cz * C + cy) * C + cx;
  const int32_t pb = __ldg(a.begin + key), pe = __ldg(a.begin + key + 1);
  if (pb == pe) return;
  const uint32_t ox = (uint32_t)((((uint64_t)(2 * cx + 1)) << 31) / (uint64_t)C);
  const uint32_t oy = (uint32_t)((((uint64_t)(2 * cy + 1)) << 31) / (uint64_t)C);
  const uint32_t oz = (uint32_t)((((uint64_t)(2 * cz + 1)) << 31) / (uint64_t)C);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t8 = lane & 7, ph = lane >> 3;
  const float Cf = (float)C;
  unsigned lt;  // lanes below this one
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  // offsets, cutoff and softening length in units of 2 r_s / sqrt(log2 e)
  // (see pair())
  const float sc = a.lscale;
  const PairK pk{a.rcut2, a.h2, a.wlen};
  // culling works on unwrapped offsets; without it every source is kept
  const float keep2 = !WRAP && a.rcut2 < INFINITY ? a.rcut2 : INFINITY;
  if (tid == 0) {
    int nr = 0, tot = 0;
    for (int dz = -1; dz <= 1; dz++) {
      const int rz = wrapi(cz + dz, C);
      for (int dy = -1; dy <= 1; dy++) {
        const int ry = wrapi(cy + dy, C);
        const int64_t row = ((int64_t)rz * C + ry) * C;
        int xa[2], xb[2], np;
        if (cx >= 1 && cx + 1 < C) {
          xa[0] = cx - 1; xb[0] = cx + 2; np = 1;
        } else if (cx == 0) {
          xa[0] = C - 1; xb[0] = C; xa[1] = 0; xb[1] = 2; np = 2;
        } else {
          xa[0] = C - 2; xb[0] = C; xa[1] = 0; xb[1] = 1; np = 2;
        }
        for (int p = 0; p < np; p++) {
          const int32_t b = __ldg(a.begin + row + xa[p]), e = __ldg(a.begin + row + xb[p]);
          runb[nr] = b;
          runp[nr] = tot;
          tot += e - b;
          nr++;
        }
      }
    }
    for (int r = nr; r <= kMaxRuns; r++) runp[r] = tot;
  }
  __syncthreads();
  const int total = runp[kMaxRuns];
  float4* buf = bufs + warp * kBuf;
  int np = 8;  // sinks per pass: the power of two >= the cell's count, at most npass
  while (np < npass && np < pe - pb) np <<= 1;
  const int32_t s_end = (int32_t)min((int64_t)pe, (int64_t)pb + (int64_t)pass_hi * np);
  for (int32_t sbase = pb + pass_lo * np; sbase < s_end; sbase += np) {
    // 1. order this pass's active sinks by sub-cell (deterministic bitonic sort)
    if (tid == 0) runp[kMaxRuns + 1] = np;  // active count when every slot is active
    for (int e = tid; e < np; e += T) {
      const int32_t i = sbase + e;
      unsigned k = 512u;  // inactive / absent sinks sort last
      if (i < pe && a.rung[i] >= a.min_rung) {
        const int4 q = __ldg(a.pos4 + i);
        k = morton9(distance32((uint32_t)q.x, ox), distance32((uint32_t)q.y, oy), distance32((uint32_t)q.z, oz), Cf);
      }
      skey[e] = (k << 8) | (unsigned)e;
    }
    __syncthreads();
    for (int kk = 2; kk <= np; kk <<= 1) {
      for (int j = kk >> 1; j > 0; j >>= 1) {
        for (int e = tid; e < np; e += T) {
          const int ixj = e ^ j;
          if (ixj > e) {
            const unsigned u = skey[e], v = skey[ixj];
            const bool up = (e & kk) == 0;
            if ((u > v) == up) {
              skey[e] = v;
              skey[ixj] = u;
            }
          }
        }
        __syncthreads();
      }
    }
    for (int e = tid; e < np; e += T) {
      const unsigned m = skey[e];
      const bool act = (m >> 8) < 512u;
      float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
      if (act) {
        const int4 q = __ldg(a.pos4 + sbase + (int32_t)(m & 0xffu));
        p = make_float4(offset_scaled((uint32_t)q.x, ox, sc), offset_scaled((uint32_t)q.y, oy, sc),
                        offset_scaled((uint32_t)q.z, oz, sc), 0.f);
      }
      spos[e] = p;
#pragma unroll
      for (int c = 0; c < 8; c++) acc[e * 8 + c] = 0.f;
      // active sinks sort first: the first inactive slot is their count
      if (!act && (e == 0 || (skey[e - 1] >> 8) < 512u)) runp[kMaxRuns + 1] = e;
    }
    __syncthreads();
    const int nact = runp[kMaxRuns + 1];
    const int ngroups = (nact + kGroup - 1) / kGroup;
    int r = 0;  // this thread's neighbourhood run: its staged indices only increase
    for (int c0 = 0; c0 < total; c0 += stage) {
      const int len = min(stage, total - c0);
      __syncthreads();
      for (int j = tid; j < len; j += T) {
        const int e = c0 + j;
        while (runp[r + 1] <= e) r++;
        const int4 u = __ldg(a.pos4 + runb[r] + (e - runp[r]));
        src[j] = make_float4(offset_scaled((uint32_t)u.x, ox, sc), offset_scaled((uint32_t)u.y, oy, sc),
                             offset_scaled((uint32_t)u.z, oz, sc), 0.f);
      }
      __syncthreads();
      for (int g = warp; g < ngroups; g += W) {
        const int gs = g * kGroup;
        const int gn = min(kGroup, nact - gs);
        const bool mysink = t8 < gn;
        const float4 sp = spos[gs + (mysink ? t8 : 0)];
        // group bounding box (lanes 0..gn-1 hold the sinks)
        float bxl = mysink ? sp.x : INFINITY, bxh = mysink ? sp.x : -INFINITY;
        float byl = mysink ? sp.y : INFINITY, byh = mysink ? sp.y : -INFINITY;
        float bzl = mysink ? sp.z : INFINITY, bzh = mysink ? sp.z : -INFINITY;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
          bxl = fminf(bxl, __shfl_xor_sync(0xffffffffu, bxl, o));
          bxh = fmaxf(bxh, __shfl_xor_sync(0xffffffffu, bxh, o));
          byl = fminf(byl, __shfl_xor_sync(0xffffffffu, byl, o));
          byh = fmaxf(byh, __shfl_xor_sync(0xffffffffu, byh, o));
          bzl = fminf(bzl, __shfl_xor_sync(0xffffffffu, bzl, o));
          bzh = fmaxf(bzh, __shfl_xor_sync(0xffffffffu, bzh, o));
        }
        // box as centre and half-extent: the distance along an axis is then
        // |s - c| - h (3 instructions instead of 4).  The half-extent is
        // widened by 1e-5 of the unit (2 r_s; offsets here are a few units,
        // whose float spacing is < 1e-6) to cover the rounding of c, h and
        // s - c, so the cull never drops a source the exact pair test keeps.
        const float cbx = 0.5f * (bxl + bxh), hbx = fmaf(0.5f, bxh - bxl, 1e-5f);
        const float cby = 0.5f * (byl + byh), hby = fmaf(0.5f, byh - byl, 1e-5f);
        const float cbz = 0.5f * (bzl + bzh), hbz = fmaf(0.5f, bzh - bzl, 1e-5f);
        float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
        int cnt = 0;
        // Every lane loads a staged source (the last one again past the end)
        // and tests it; kept sources are appended to the warp's buffer.  The
        // buffer is read only after a __syncwarp (flush or tail), so appends
        // need no barrier of their own.
        for (int j0 = 0; j0 < len; j0 += 32) {
          const int j = j0 + lane;
          const float4 s = src[min(j, len - 1)];
          const float ex = fmaxf(fabsf(s.x - cbx) - hbx, 0.f);
          const float ey = fmaxf(fabsf(s.y - cby) - hby, 0.f);
          const float ez = fmaxf(fabsf(s.z - cbz) - hbz, 0.f);
          const bool keep = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < keep2 && j < len;
          const unsigned b = __ballot_sync(0xffffffffu, keep);
          if (keep) buf[cnt + __popc(b & lt)] = s;
          cnt += __popc(b);
          // the count is the same in every lane; a vote makes the branch
          // warp-uniform for the compiler (no reconvergence region)
          if (__all_sync(0xffffffffu, cnt >= 32)) {
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 32; k += 8) {
              // lanes without a sink (a partial group) hold a copy of the
              // group's first sink; their sums are never committed
              pair2<WRAP>(pk, sp, buf[k + ph], buf[k + 4 + ph], px, py, pz, pp);
            }
            __syncwarp();
            if (lane < cnt - 32) buf[lane] = buf[32 + lane];
            cnt -= 32;
            __syncwarp();
          }
        }
        __syncwarp();
        if (WRAP) {
          for (int k = 0; k < cnt; k += 4) {
            if (k + ph < cnt && mysink) {
              const float4 u = buf[k + ph];
              pair<WRAP>(pk, sp.x - u.x, sp.y - u.y, sp.z - u.z, px, py, pz, pp);
            }
          }
        } else {
          // past the count a lane takes a source 1e18 units away: beyond any
          // cutoff, its terms are exactly 0 (no minimum-image fold here)
          const float4 far = make_float4(1e18f, 1e18f, 1e18f, 0.f);
          for (int k = 0; k < cnt; k += 8) {
            const float4 u0 = k + ph < cnt ? buf[k + ph] : far;
            const float4 u1 = k + 4 + ph < cnt ? buf[k + 4 + ph] : far;
            pair2<WRAP>(pk, sp, u0, u1, px, py, pz, pp);
          }
        }
        __syncwarp();
        // fold the four source phases (fixed order), lanes 0..7 hold the group's sums
#pragma unroll
        for (int o = 8; o <= 16; o <<= 1) {
          px += __shfl_xor_sync(0xffffffffu, px, o);
          py += __shfl_xor_sync(0xffffffffu, py, o);
          pz += __shfl_xor_sync(0xffffffffu, pz, o);
          pp += __shfl_xor_sync(0xffffffffu, pp, o);
        }
        if (ph == 0 && mysink) {
          float* A = acc + (gs + t8) * 8;
          if (a.kahan) {
            kahan_add(A[0], A[4], px);
            kahan_add(A[1], A[5], py);
            kahan_add(A[2], A[6], pz);
            kahan_add(A[3], A[7], pp);
          } else {
            A[0] += px;
            A[1] += py;
            A[2] += pz;
            A[3] += pp;
          }
        }
      }
    }
    __syncthreads();
    // 2. long-range interpolation and the kick, one thread per sorted sink
    for (int e = tid; e < nact; e += T) {
      const int32_t i = sbase + (int32_t)(skey[e] & 0xffu);
      const float lx = a.gx[i], ly = a.gy[i], lz = a.gz[i], lp = a.pot[i];  // from k_interp_long
      const float* A = acc + e * 8;
      // pair sums back from units of 2 r_s: force x (1/2r_s)^2, potential x 1/2r_s
      const float fs = a.inv2rs * a.inv2rs * kLog2e;
      const float g0 = fmaf(A[0] - A[4], fs, lx) * a.GM;
      const float g1 = fmaf(A[1] - A[5], fs, ly) * a.GM;
      const float g2 = fmaf(A[2] - A[6], fs, lz) * a.GM;
      const float phi = fmaf(A[3] - A[7], a.inv2rs * kSqrtLog2e, lp) * a.GM;
      a.gx[i] = g0;
      a.gy[i] = g1;
      a.gz[i] = g2;
      a.pot[i] = phi;
      // rung / velocity kick (src/kick_pme.cu:330-352); rung_dt[r] = 2^-r.
      int r = a.rung[i];
      if (r < 0 || r >= kMaxRung) {
        atomicOr(a.err, kErrRung);
        r = min(max(r, 0), kMaxRung - 1);
      }
      float vx = a.vx[i], vy = a.vy[i], vz = a.vz[i];
      float dt = 0.5f * ldexpf(1.0f, -r) * a.t0;
      if (!a.first_call) {
        vx = fmaf(g0, dt, vx);
        vy = fmaf(g1, dt, vy);
        vz = fmaf(g2, dt, vz);
      }
      const float gg = fmaf(g0, g0, fmaf(g1, g1, g2 * g2));
      const float factor = a.eta * sqrtf(a.scale * a.hsoft);
      dt = fminf(factor * rsqrtf(sqrtf(gg)), a.t0);
      int rn = (int)fmaxf(ceilf(log2f(a.t0) - log2f(dt)), (float)(r - 1));
      if (rn < 0 || rn >= kMaxRung) {
        atomicOr(a.err, kErrRung);
        rn = min(max(rn, 0), kMaxRung - 1);
      }
      a.rung[i] = (int8_t)rn;
      dt = 0.5f * ldexpf(1.0f, -rn) * a.t0;
      a.vx[i] = fmaf(g0, dt, vx);
      a.vy[i] = fmaf(g1, dt, vy);
      a.vz[i] = fmaf(g2, dt, vz);
    }
    __syncthreads();  // sort keys / staging reused by the next pass
  }
}

// One block per sink cell.  split (optional): the queue's per-cell class
// words; cells split into pass items (more than kSplitPasses passes) are left
// to the persistent launch over those items.
template <bool WRAP>
__global__ void __launch_bounds__(kKickThreads, TPM_KICK_MINB)
    k_kick_pme(KickArgs a, int stage, int npass, const int* __restrict__ split) {
  extern __shared__ float4 smem4[];
  int bid = blockIdx.x;
  const int i2 = bid % a.s2;
  bid /= a.s2;
  const int i1 = bid % a.s1;
  const int i0 = bid / a.s1;
  const int cx = a.b0 + i0, cy = a.b1 + i1, cz = a.b2 + i2;
  if (split && (__ldg(split + ((int64_t)cz * a.C + cy) * a.C + cx) >> 6) > 1) return;
  kick_cell<WRAP>(a, cx, cy, cz, smem4, stage, npass);
}

// ------------------------------------------------------------ batched kick
//
// Many independent boxes kicked by one persistent launch.  A work item is
// one (box, chain cell); items are ordered by estimated cost (sinks x
// neighbourhood sources, heaviest first) and taken from a global counter,
// so the blocks that finish light cells pick up the remaining ones and no
// box-sized tail is left on a few SMs.  The per-box kernel arguments live in
// a device array; the step's scalars come as kernel parameters.
struct StepScalars {
  int min_rung, first_call;
  float t0, scale;
};

__device__ __forceinline__ KickArgs box_args(const KickArgs* __restrict__ boxes, int b, const StepScalars& st) {
  KickArgs a = boxes[b];
  a.min_rung = st.min_rung;
  a.first_call = st.first_call;
  a.t0 = st.t0;
  a.scale = st.scale;
  return a;
}

// SINGLE: one box whose arguments come as the kernel parameter `one` (the
// constant bank, like the per-cell launch); else per-box arguments from
// `boxes`, kept in shared memory.
template <bool WRAP, bool SINGLE>
__global__ void __launch_bounds__(kKickThreads, TPM_KICK_MINB)
    k_kick_batch(const KickArgs* __restrict__ boxes, KickArgs one, const int4* __restrict__ items,
                 const int* __restrict__ nitems, int* __restrict__ counter, StepScalars st, int stage, int npass) {
  extern __shared__ float4 smem4[];
  __shared__ int s_item[2];
  // The box's arguments are read from shared memory where they are used:
  // held in registers, its ten array addresses would spill the pair loop.
  __shared__ KickArgs s_args;
  const int n = *nitems;
  if (threadIdx.x == 0) s_item[0] = atomicAdd(counter, 1);
  __syncthreads();
  int cur_box = -1;
  for (int k = 0;; k ^= 1) {
    const int it = s_item[k];
    if (it >= n) return;
    // the next item is fetched while this one runs; the barrier at the end of
    // the iteration orders the write against the reads of s_item[k ^ 1]
    if (threadIdx.x == 0) s_item[k ^ 1] = atomicAdd(counter, 1);
    const int4 w = __ldg(items + it);  // (box, cell key, first pass, end pass); box -1: empty slot
    if (w.x >= 0) {  // uniform: every thread read the same item
      if (SINGLE) {
        const int C = one.C;
        kick_cell<WRAP>(one, w.y % C, (w.y / C) % C, w.y / (C * C), smem4, stage, npass, w.z, w.w);
      } else {
        if (w.x != cur_box) {
          if (threadIdx.x == 0) s_args = box_args(boxes, w.x, st);
          cur_box = w.x;
          __syncthreads();
        }
        const int C = s_args.C;
        kick_cell<WRAP>(s_args, w.y % C, (w.y / C) % C, w.y / (C * C), smem4, stage, npass, w.z, w.w);
      }
    }
    __syncthreads();
  }
}

// Work items: every non-empty (box, cell) of the kick boxes, bucketed by the
// binary order of magnitude of its cost and laid out heaviest bucket first.
// A cell with more sinks than one pass is split into one item per pass (a
// halo cell a thousand times the mean then spreads over many SMs).
struct BoxCells {
  const int32_t* begin;
  int C;
  int base;    // first global cell index of the box
  int b[3];    // kick box [b, e) in chain cells
  int e[3];
};

__device__ __forceinline__ int find_box(const BoxCells* __restrict__ bc, int nbox, int g) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&bc[mid].base) <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

constexpr int kCostClasses = 64;
// A cell needing more sink passes than this becomes one item per pass.
constexpr int kSplitPasses = 4;

// Items of one cell: none outside the kick box or when empty; one item per
// sink pass (np = the power of two >= the cell's count, at most npass) when
// the cell needs more than one pass, else one item for the whole cell.  All
// of a cell's items share one cost class: sinks of a pass x neighbourhood
// sources.  Returns class | items << 6, or -1.
__device__ __forceinline__ int cell_items(const BoxCells& b, int key, int npass) {
  const int C = b.C;
  const int cx = key % C, cy = (key / C) % C, cz = key / (C * C);
  if (cx < b.b[0] || cx >= b.e[0] || cy < b.b[1] || cy >= b.e[1] || cz < b.b[2] || cz >= b.e[2]) return -1;
  const int32_t n = __ldg(b.begin + key + 1) - __ldg(b.begin + key);
  if (n == 0) return -1;
  int64_t nb = 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++) {
      const int64_t row = ((int64_t)wrapi(cz + dz, C) * C + wrapi(cy + dy, C)) * C;
      for (int dx = -1; dx <= 1; dx++) {
        const int64_t k2 = row + wrapi(cx + dx, C);
        nb += __ldg(b.begin + k2 + 1) - __ldg(b.begin + k2);
      }
    }
  int np = 8;
  while (np < npass && np < n) np <<= 1;
  const int passes = (n + np - 1) / np;
  const int items = passes > kSplitPasses ? passes : 1;
  const uint64_t cost = (uint64_t)(items > 1 ? np : n) * (uint64_t)nb;
  return (63 - __clzll((long long)(cost | 1ull))) | (items << 6);
}

__global__ void k_item_classes(const BoxCells* __restrict__ bc, int nbox, int total, int npass, int* __restrict__ cls,
                               int* __restrict__ hist) {
  __shared__ int sh[kCostClasses];
  for (int i = threadIdx.x; i < kCostClasses; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < total) {
    const int b = find_box(bc, nbox, g);
    const BoxCells box = bc[b];
    const int c = cell_items(box, g - box.base, npass);
    cls[g] = c;
    if (c >= 0 && (c >> 6) > 1) atomicAdd(&sh[c & 63], c >> 6);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kCostClasses; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

// hist[0..63] -> start offsets, heaviest class first; nitems = total items.
// One warp.
__global__ void k_item_offsets(int* __restrict__ hist, int* __restrict__ start, int* __restrict__ nitems, int total) {
  const int lane = threadIdx.x;
  // lane l owns classes 63 - 2l and 62 - 2l (descending order)
  const int a = hist[63 - 2 * lane], b = hist[62 - 2 * lane];
  int incl = a + b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int excl = incl - a - b;
  start[63 - 2 * lane] = excl;
  start[62 - 2 * lane] = excl + a;
  if (lane == 31) {
    nitems[0] = incl + total;  // split items, then one slot per cell
    nitems[1] = incl;
  }
  hist[63 - 2 * lane] = 0;  // reused as fill counters by the scatter
  hist[62 - 2 * lane] = 0;
}

// Split cells' pass items first, heaviest class first; then slot nsplit + g
// for every cell g in natural (z, y, x) order -- the whole cell as one item,
// or an empty marker (box -1) for empty, split or out-of-box cells -- so the
// ordinary cells keep the spatial order of a per-cell launch.
__global__ void k_item_scatter(const BoxCells* __restrict__ bc, int nbox, int total, const int* __restrict__ cls,
                               const int* __restrict__ start, int* __restrict__ fill,
                               const int* __restrict__ nitems, int4* __restrict__ items) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int c = cls[g];
  const int nsplit = nitems[1];
  if (c < 0) {
    items[nsplit + g] = make_int4(-1, 0, 0, 0);
    return;
  }
  const int b = find_box(bc, nbox, g);
  const int key = g - __ldg(&bc[b].base);
  const int k = c >> 6, cl = c & 63;
  if (k == 1) {
    items[nsplit + g] = make_int4(b, key, 0, 0x7fffffff);
    return;
  }
  items[nsplit + g] = make_int4(-1, 0, 0, 0);
  const int at = start[cl] + atomicAdd(fill + cl, k);
  for (int p = 0; p < k; p++) items[at + p] = make_int4(b, key, p, p + 1);
}

// Long-range interpolation of the batch: one block per global cell slot,
// every box's cells in natural order, so that neighbouring cells' stencil
// reads share the L1 and L2 as in the single-box k_interp_direct (in the
// queue's cost order, items of different boxes interleave).
__global__ void __launch_bounds__(64, TPM_INTERP_MINB)
    k_interp_slots(const KickArgs* __restrict__ boxes, const BoxCells* __restrict__ bc, int nbox, int min_rung) {
  const int g = blockIdx.x;
  const int b = find_box(bc, nbox, g);
  const KickArgs a = boxes[b];  // the fields used, in registers
  const int key = g - __ldg(&bc[b].base);
  const int32_t pb = __ldg(a.begin + key), pe = __ldg(a.begin + key + 1);
  for (int32_t i = pb + (int32_t)threadIdx.x; i < pe; i += blockDim.x) {
    if (a.rung[i] < min_rung) continue;
    float lx, ly, lz, lp;
    interp_long(a, __ldg(a.pos4 + i), lx, ly, lz, lp);
    a.gx[i] = lx;
    a.gy[i] = ly;
    a.gz[i] = lz;
    a.pot[i] = lp;
  }
}

// The batch's ordinary cells: one block per global cell slot (every box's
// cells in natural order); empty and split cells return at once.
template <bool WRAP>
__global__ void __launch_bounds__(kKickThreads, TPM_KICK_MINB)
    k_kick_slots(const KickArgs* __restrict__ boxes, const BoxCells* __restrict__ bc, int nbox,
                 const int* __restrict__ cls, StepScalars st, int stage, int npass) {
  extern __shared__ float4 smem4[];
  __shared__ KickArgs s_args;  // shared, not registers: see k_kick_batch
  const int g = blockIdx.x;
  const int c = __ldg(cls + g);
  if (c < 0 || (c >> 6) > 1) return;
  const int b = find_box(bc, nbox, g);
  if (threadIdx.x == 0) s_args = box_args(boxes, b, st);
  __syncthreads();
  const int key = g - __ldg(&bc[b].base);
  const int C = s_args.C;
  kick_cell<WRAP>(s_args, key % C, (key / C) % C, key / (C * C), smem4, stage, npass);
}

}  // namespace

namespace {

// Kernel arguments of one box (the reference's kernel_params,
// src/kick_pme.cu:439-453, all FP32) for sink cells [b, e).
KickArgs make_args(tpm_ctx* c, const int b[3], const int e[3], int min_rung, double scale, double t0,
                   int first_call) {
  KickArgs a;
  a.pos4 = c->pos4;
  a.vx = c->vx;
  a.vy = c->vy;
  a.vz = c->vz;
  a.rung = c->rung;
  a.gx = c->gx;
  a.gy = c->gy;
  a.gz = c->gz;
  a.pot = c->pot;
  a.begin = c->cell_begin;
  a.thr = c->thr;
  a.phi = c->phi;
  a.err = c->d_err;
  a.C = c->C;
  a.N = c->N;
  a.b0 = b[0];
  a.b1 = b[1];
  a.b2 = b[2];
  a.s1 = e[1] - b[1];
  a.s2 = e[2] - b[2];
  a.min_rung = min_rung;
  a.first_call = first_call ? 1 : 0;
  a.kahan = c->opt.kahan ? 1 : 0;
  a.GM = (float)c->opt.GM;
  a.eta = (float)c->opt.eta;
  a.t0 = (float)t0;
  a.scale = (float)scale;
  a.hsoft = (float)c->opt.hsoft;
  const double inv2rs = 0.5 / c->rs_box;
  a.inv2rs = (float)inv2rs;
  // lengths in u = 2 r_s / sqrt(log2 e), formed in FP64
  const double su = inv2rs * std::sqrt(1.4426950408889634);
  a.lscale = (float)(su * 2.3283064365386963e-10);
  a.h2 = (float)((c->opt.hsoft * su) * (c->opt.hsoft * su));
  a.rcut2 = c->rcut_box > 0 ? (float)((c->rcut_box * su) * (c->rcut_box * su)) : INFINITY;
  a.wlen = (float)su;
  return a;
}

size_t kick_smem(const KickShape& k) {
  return sizeof(float4) * ((size_t)k.stage + (size_t)k.warps * kBuf + k.npass) + sizeof(float) * k.npass * 8 +
         sizeof(unsigned) * k.npass + sizeof(int) * (2 * kMaxRuns + 2);
}

}  // namespace

// Block size follows the mean cell occupancy (about two groups of 8 sinks
// per warp, 2..8 warps); the stage holds a fraction of the mean 27-cell
// neighbourhood (at most kMaxStage sources; larger ones are chunked).
KickShape kick_default_shape(double mean_cell) {
  KickShape k;
  k.warps = (int)std::min(8.0, std::max(2.0, std::ceil(mean_cell / (2.0 * kGroup))));
  int stage = (int)std::min<double>(kMaxStage, std::max<double>(512.0, TPM_KICK_STAGE_X100 * 0.01 * 27.0 * mean_cell));
  k.stage = (stage + 127) / 128 * 128;
  k.npass = kPass;
  if (TPM_KICK_PASS_X > 0) {
    k.npass = 64;
    while (k.npass < kPass && k.npass < TPM_KICK_PASS_X * mean_cell) k.npass *= 2;
  }
  return k;
}

bool kick_shape_valid(const KickShape& k) {
  const bool pow2 = k.npass >= 8 && (k.npass & (k.npass - 1)) == 0;
  return k.warps >= 1 && 32 * k.warps <= kKickThreads && k.stage >= 128 && k.stage <= kMaxStage &&
         k.stage % 128 == 0 && pow2 && k.npass <= kPass && kick_smem(k) <= 200 * 1024;
}

int kick_queue_single(tpm_ctx* c, const KickArgs& a, const KickShape& k, int min_rung, double scale, double t0,
                      int first_call, const int b[3], const int e[3]);

int kick_pme(tpm_ctx* c, const int box[6], int min_rung, double scale, double t0, int first_call) {
  if (!c->sorted) return fail(TPM_ERR_STATE, "kick_pme needs chainmesh_create first");
  if (!c->have_phi) return fail(TPM_ERR_STATE, "kick_pme needs gravity_long_compute first");
  const int C = c->C;
  int b[3], e[3];
  for (int d = 0; d < 3; d++) {
    b[d] = box ? box[d] : 0;
    e[d] = box ? box[3 + d] : C;
    if (b[d] < 0 || e[d] > C || e[d] < b[d]) return fail(TPM_ERR_INVALID, "kick box outside the chain mesh");
  }
  const int64_t ncell = (int64_t)(e[0] - b[0]) * (e[1] - b[1]) * (e[2] - b[2]);
  const KickArgs a = make_args(c, b, e, min_rung, scale, t0, first_call);
  const double mean_cell = (double)c->n / ((double)C * C * C);
  const KickShape k = kick_default_shape(mean_cell);
  const size_t smem = kick_smem(k);
  const bool wrap = C == 3;
  auto kern = wrap ? k_kick_pme<true> : k_kick_pme<false>;
  TPM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // Long-range interpolation.  A shared-memory tile of phi pays when a chain
  // cell's reach (its mesh span + 5 points per dim) is small against its
  // sinks (c2: 11.7^3 points for 184 sinks, 3.0 -> 2.1 ms); at 27 mesh cells
  // per particle (18^3 points for 64 sinks) staging costs more than the direct
  // reads, which run at the L1 sector limit (3.4 ms at 256^3 on a 768^3 mesh).
  const int maxw = (c->N + C - 1) / C + 8;
  const size_t tile_bytes = sizeof(float) * (size_t)maxw * maxw * maxw;
  const double span = (double)c->N / C + 6.0;
  stage_begin(c, kStInterp);
  if (ncell > 0) {
    if (tile_bytes <= 48 * 1024 && span * span * span <= 16.0 * mean_cell) {
      k_interp_tile<<<(unsigned)ncell, 128, tile_bytes, c->stream>>>(a, maxw);
    } else {
      k_interp_direct<<<(unsigned)ncell, 64, 0, c->stream>>>(a);
    }
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
  }
  stage_end(c, kStInterp);
  stage_begin(c, kStKick);
  if (ncell > 0 && c->opt.kick_grid) {
    kern<<<(unsigned)ncell, 32 * k.warps, smem, c->stream>>>(a, k.stage, k.npass, nullptr);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
  } else if (ncell > 0) {
    // heavy cells' pass items through the persistent queue, every other cell
    // through the per-cell launch (faster for ordinary cells: 17.6 against
    // 18.6 ms at the 256^3 headline)
    const int rc = kick_queue_single(c, a, k, min_rung, scale, t0, first_call, b, e);
    if (rc) return rc;
    kern<<<(unsigned)ncell, 32 * k.warps, smem, c->stream>>>(a, k.stage, k.npass, c->kq.d_class);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
  }
  stage_end(c, kStKick);
  c->pot_valid = min_rung <= 0 && ncell == (int64_t)C * C * C;
  return TPM_OK;
}

// ------------------------------------------------------------ batched kick

size_t kick_batch_args_bytes() { return sizeof(KickArgs); }
size_t kick_batch_cells_bytes() { return sizeof(BoxCells); }

int kick_batch_write_tables(tpm_ctx* const* boxes, int nbox, void* h_args, void* h_cells, int64_t* total_cells,
                            int64_t* max_items) {
  KickArgs* A = static_cast<KickArgs*>(h_args);
  BoxCells* B = static_cast<BoxCells*>(h_cells);
  int64_t base = 0, parts = 0;
  for (int i = 0; i < nbox; i++) {
    tpm_ctx* c = boxes[i];
    const int b[3] = {0, 0, 0};
    const int e[3] = {c->C, c->C, c->C};
    A[i] = make_args(c, b, e, 0, 1.0, 1.0, 1);
    B[i].begin = c->cell_begin;
    B[i].C = c->C;
    B[i].base = (int)base;
    for (int d = 0; d < 3; d++) {
      B[i].b[d] = 0;
      B[i].e[d] = c->C;
    }
    base += (int64_t)c->C * c->C * c->C;
    parts += c->cap;
    if (base > 0x7fffffffLL) return fail(TPM_ERR_INVALID, "batch has more than 2^31 chain cells");
  }
  *total_cells = base;
  // one slot per cell, plus the pass items of split cells: a split cell of
  // n sinks gives ceil(n / np) items with np >= 8, at most one per 8 particles
  *max_items = 2 * base + parts / 8 + nbox;
  if (*max_items > 0x7fffffffLL) return fail(TPM_ERR_INVALID, "batch has more than 2^31 work items");
  return TPM_OK;
}

int kick_batch_queue(const BatchQueue& q, int npass, cudaStream_t s) {
  if (q.total_cells <= 0) return TPM_OK;
  const int total = (int)q.total_cells;
  TPM_CUDA_TRY(cudaMemsetAsync(q.d_hist, 0, sizeof(int) * 2 * kCostClasses, s));
  const unsigned blocks = (unsigned)ceil_div(total, 256);
  k_item_classes<<<blocks, 256, 0, s>>>(static_cast<const BoxCells*>(q.d_cells), q.nbox, total, npass, q.d_class,
                                        q.d_hist);
  k_item_offsets<<<1, 32, 0, s>>>(q.d_hist, q.d_hist + kCostClasses, q.d_nitems, total);
  k_item_scatter<<<blocks, 256, 0, s>>>(static_cast<const BoxCells*>(q.d_cells), q.nbox, total, q.d_class,
                                        q.d_hist + kCostClasses, q.d_hist, q.d_nitems, q.d_items);
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

int kick_batch_interp(const BatchQueue& q, int min_rung, int npass, cudaStream_t s) {
  (void)npass;
  if (q.total_cells <= 0) return TPM_OK;
  k_interp_slots<<<(unsigned)q.total_cells, 64, 0, s>>>(static_cast<const KickArgs*>(q.d_args),
                                                         static_cast<const BoxCells*>(q.d_cells), q.nbox, min_rung);
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

int kick_batch_launch(const BatchQueue& q, const KickShape& k, bool wrap, int min_rung, double scale, double t0,
                      int first_call, cudaStream_t s, int* blocks_out, const KickArgs* single, bool split_only) {
  if (!kick_shape_valid(k)) return fail(TPM_ERR_INVALID, "invalid kick shape");
  if (q.total_cells <= 0) return TPM_OK;
  const size_t smem = kick_smem(k);
  auto kern = single ? (wrap ? k_kick_batch<true, true> : k_kick_batch<false, true>)
                     : (wrap ? k_kick_batch<true, false> : k_kick_batch<false, false>);
  TPM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, dev = 0, sms = 0;
  TPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * k.warps, smem));
  TPM_CUDA_TRY(cudaGetDevice(&dev));
  TPM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return fail(TPM_ERR_INVALID, "kick shape does not fit on an SM");
  const int64_t blocks = std::min<int64_t>((int64_t)per_sm * sms, q.max_items);
  StepScalars st{min_rung, first_call ? 1 : 0, (float)t0, (float)scale};
  TPM_CUDA_TRY(cudaMemsetAsync(q.d_counter, 0, sizeof(int), s));
  // split_only: the first nitems[1] items (the split cells' passes)
  kern<<<(unsigned)blocks, 32 * k.warps, smem, s>>>(static_cast<const KickArgs*>(q.d_args), single ? *single : KickArgs{},
                                                    q.d_items, q.d_nitems + (split_only ? 1 : 0), q.d_counter, st,
                                                    k.stage, k.npass);
  TPM_CUDA_TRY(cudaGetLastError());
  if (blocks_out) *blocks_out = (int)blocks;
  return TPM_OK;
}

// The batch's kick: the split cells' pass items through the persistent
// queue, then every ordinary cell in one block-per-cell launch.
int kick_batch_kick(const BatchQueue& q, const KickShape& k, bool wrap, int min_rung, double scale, double t0,
                    int first_call, cudaStream_t s, int* blocks_out) {
  int rc = kick_batch_launch(q, k, wrap, min_rung, scale, t0, first_call, s, blocks_out, nullptr, true);
  if (rc || q.total_cells <= 0) return rc;
  const size_t smem = kick_smem(k);
  auto kern = wrap ? k_kick_slots<true> : k_kick_slots<false>;
  TPM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  StepScalars st{min_rung, first_call ? 1 : 0, (float)t0, (float)scale};
  kern<<<(unsigned)q.total_cells, 32 * k.warps, smem, s>>>(static_cast<const KickArgs*>(q.d_args),
                                                           static_cast<const BoxCells*>(q.d_cells), q.nbox,
                                                           q.d_class, st, k.stage, k.npass);
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

// The single-box kick through the same persistent queue: heavy cells split
// into pass items, so a strongly clustered box is spread over every SM.
int kick_queue_single(tpm_ctx* c, const KickArgs& a, const KickShape& k, int min_rung, double scale, double t0,
                      int first_call, const int b[3], const int e[3]) {
  BatchQueue& q = c->kq;
  const int64_t ncell = (int64_t)c->C * c->C * c->C;
  if (!q.d_args) {
    q.nbox = 1;
    q.total_cells = ncell;
    q.max_items = 2 * ncell + c->cap / 8 + 1;
    if (q.max_items > 0x7fffffffLL) return fail(TPM_ERR_INVALID, "more than 2^31 work items");
    cudaError_t err = cudaMalloc(&q.d_args, sizeof(KickArgs));
    if (err == cudaSuccess) err = cudaMalloc(&q.d_cells, sizeof(BoxCells));
    if (err == cudaSuccess) err = cudaMalloc((void**)&q.d_class, sizeof(int) * ncell);
    if (err == cudaSuccess) err = cudaMalloc((void**)&q.d_hist, sizeof(int) * 2 * kCostClasses);
    if (err == cudaSuccess) err = cudaMalloc((void**)&q.d_items, sizeof(int4) * q.max_items);
    if (err == cudaSuccess) err = cudaMalloc((void**)&q.d_nitems, sizeof(int) * 2);
    if (err == cudaSuccess) err = cudaMalloc((void**)&q.d_counter, sizeof(int) * 2);
    if (err != cudaSuccess) {
      cudaGetLastError();
      return fail(TPM_ERR_NOMEM, std::string("kick queue: ") + cudaGetErrorString(err));
    }
    c->device_bytes += sizeof(KickArgs) + sizeof(BoxCells) + 4 * ncell + 8 * kCostClasses + 16 * q.max_items + 16;
  }
  // per-call arguments: array addresses move with the sort's buffer swaps
  KickArgs* ha = reinterpret_cast<KickArgs*>(c->kq_host_args);
  BoxCells* hb = reinterpret_cast<BoxCells*>(c->kq_host_cells);
  static_assert(sizeof(KickArgs) <= sizeof(c->kq_host_args), "host argument buffer too small");
  static_assert(sizeof(BoxCells) <= sizeof(c->kq_host_cells), "host cell-table buffer too small");
  *ha = a;
  hb->begin = c->cell_begin;
  hb->C = c->C;
  hb->base = 0;
  for (int d = 0; d < 3; d++) {
    hb->b[d] = b[d];
    hb->e[d] = e[d];
  }
  TPM_CUDA_TRY(cudaMemcpyAsync(q.d_args, ha, sizeof(KickArgs), cudaMemcpyHostToDevice, c->stream));
  TPM_CUDA_TRY(cudaMemcpyAsync(q.d_cells, hb, sizeof(BoxCells), cudaMemcpyHostToDevice, c->stream));
  int rc = kick_batch_queue(q, k.npass, c->stream);
  if (rc == TPM_OK) rc = kick_batch_launch(q, k, c->C == 3, min_rung, scale, t0, first_call, c->stream, nullptr, &a, true);
  c->launches += 4;
  return rc;
}

}  // namespace tpm
