// kick_pme.cu -- fused long-range interpolation + short-range PP + rung kick.
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
//  * One block per sink cell.  Source tiles are staged in shared memory as
//    float offsets from the sink cell centre: the int32 wrap-around
//    difference (the reference's periodic minimum image) is taken once per
//    source per block, so the pair loop is pure FP32 (FADD for dx).
//  * Pair kernel: rsqrt / rcp / ex2 approximations (MUFU) for 1/r, the A&S
//    rational and exp(-x^2); an optional cutoff masks pairs beyond rcut.
//  * Precision: FP32 pair terms summed in chunks of 64 sources, chunk sums
//    added with Kahan compensation per target (kahan option).
#include "tpm_internal.cuh"

#include <cmath>

namespace tpm {
namespace {

constexpr int kKickThreads = 256;
constexpr int kTile = 1024;
constexpr int kChunk = 64;

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
  const float* __restrict__ phi;
  int* __restrict__ err;
  int C, N;
  int b0, b1, b2, s1, s2;
  int min_rung;
  int first_call;
  int kahan;
  float GM, eta, t0, scale, hsoft;
  float inv2rs, twooversqrtpi, h2, hinv, h3inv, rcut2;
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
  float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
  for (int i = 0; i < kNInterp; i++) {
    const int64_t plane = (int64_t)wrapi(base[0] + i, N) * N * N;
    float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
#pragma unroll
    for (int j = 0; j < kNInterp; j++) {
      float rz = 0.f, rdz = 0.f;
#pragma unroll
      for (int k = 0; k < kNInterp; k++) {
        const float v = __ldg(a.phi + plane + iy[j] + iz[k]);
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
    (void)pp;
  }
  lx = -sx * (float)N;
  ly = -sy * (float)N;
  lz = -sz * (float)N;
  lp = sp;
}

// One source against one sink (src/kick_pme.cu:285-314).
__device__ __forceinline__ void pair(const KickArgs& a, float dx, float dy, float dz, float& gx, float& gy,
                                     float& gz, float& ph) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float r2c = fmaxf(r2, a.h2);
  const float rinv = rsqrt_approx(r2c);
  const float x0 = r2c * rinv * a.inv2rs;
  const float t = rcp_approx(fmaf(0.3275911f, x0, 1.0f));
  const float e = ex2_approx(-1.4426950408889634f * x0 * x0);
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
  const float erfc0 = poly * e;
  const float rinv2 = rinv * rinv;
  float rinv3 = fmaf(a.twooversqrtpi * x0, e, erfc0) * rinv2 * rinv;
  float rinv1 = erfc0 * rinv;
  if (r2 <= a.h2) {  // softened Newtonian kernel inside hsoft (rare)
    const float q2 = r2 * a.hinv * a.hinv;
    rinv3 = fmaf(fmaf(15.0f / 8.0f, q2, -21.0f / 4.0f), q2, 35.0f / 8.0f) * a.h3inv;
    rinv1 = fmaf(fmaf(fmaf(-5.0f / 16.0f, q2, 21.0f / 16.0f), q2, -35.0f / 16.0f), q2, 35.0f / 16.0f) * a.hinv;
  }
  const bool in = r2 < a.rcut2;
  rinv3 = in ? rinv3 : 0.0f;
  rinv1 = in ? rinv1 : 0.0f;
  gx = fmaf(-dx, rinv3, gx);
  gy = fmaf(-dy, rinv3, gy);
  gz = fmaf(-dz, rinv3, gz);
  ph -= rinv1;
}

__global__ void __launch_bounds__(kKickThreads) k_kick_pme(KickArgs a) {
  __shared__ float4 src[kTile];
  const int C = a.C;
  int bid = blockIdx.x;
  const int i2 = bid % a.s2;
  bid /= a.s2;
  const int i1 = bid % a.s1;
  const int i0 = bid / a.s1;
  const int cx = a.b0 + i0, cy = a.b1 + i1, cz = a.b2 + i2;
  const int64_t key = ((int64_t)cz * C + cy) * C + cx;
  const int32_t pb = __ldg(a.begin + key), pe = __ldg(a.begin + key + 1);
  if (pb == pe) return;
  // sink cell centre in fixed point (offsets are taken from here)
  const uint32_t ox = (uint32_t)((((uint64_t)(2 * cx + 1)) << 31) / (uint64_t)C);
  const uint32_t oy = (uint32_t)((((uint64_t)(2 * cy + 1)) << 31) / (uint64_t)C);
  const uint32_t oz = (uint32_t)((((uint64_t)(2 * cz + 1)) << 31) / (uint64_t)C);
  const int tid = threadIdx.x;
  for (int32_t sbase = pb; sbase < pe; sbase += kKickThreads) {
    const int32_t i = sbase + tid;
    const bool active = i < pe && a.rung[i] >= a.min_rung;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    float lx = 0.f, ly = 0.f, lz = 0.f, lp = 0.f;
    if (active) {
      const int4 q = __ldg(a.pos4 + i);
      sx = distance32((uint32_t)q.x, ox);
      sy = distance32((uint32_t)q.y, oy);
      sz = distance32((uint32_t)q.z, oz);
      interp_long(a, q, lx, ly, lz, lp);
    }
    float Sx = 0.f, Sy = 0.f, Sz = 0.f, Sp = 0.f;
    float Cx = 0.f, Cy = 0.f, Cz = 0.f, Cp = 0.f;
    for (int dz = -1; dz <= 1; dz++) {
      const int rz = wrapi(cz + dz, C);
      for (int dy = -1; dy <= 1; dy++) {
        const int ry = wrapi(cy + dy, C);
        const int64_t row = ((int64_t)rz * C + ry) * C;
        int32_t rb[2], re[2];
        int nrun;
        if (cx >= 1 && cx + 1 < C) {
          rb[0] = __ldg(a.begin + row + cx - 1);
          re[0] = __ldg(a.begin + row + cx + 2);
          nrun = 1;
        } else if (cx == 0) {
          rb[0] = __ldg(a.begin + row + C - 1);
          re[0] = __ldg(a.begin + row + C);
          rb[1] = __ldg(a.begin + row);
          re[1] = __ldg(a.begin + row + 2);
          nrun = 2;
        } else {
          rb[0] = __ldg(a.begin + row + C - 2);
          re[0] = __ldg(a.begin + row + C);
          rb[1] = __ldg(a.begin + row);
          re[1] = __ldg(a.begin + row + 1);
          nrun = 2;
        }
        for (int run = 0; run < nrun; run++) {
          for (int32_t t0 = rb[run]; t0 < re[run]; t0 += kTile) {
            const int len = min(kTile, re[run] - t0);
            __syncthreads();
            for (int j = tid; j < len; j += kKickThreads) {
              const int4 q = __ldg(a.pos4 + t0 + j);
              src[j] = make_float4(distance32((uint32_t)q.x, ox), distance32((uint32_t)q.y, oy),
                                   distance32((uint32_t)q.z, oz), 0.f);
            }
            __syncthreads();
            if (active) {
              for (int jc = 0; jc < len; jc += kChunk) {
                const int je = min(len, jc + kChunk);
                float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
#pragma unroll 4
                for (int j = jc; j < je; j++) {
                  const float4 s = src[j];
                  pair(a, sx - s.x, sy - s.y, sz - s.z, px, py, pz, pp);
                }
                if (a.kahan) {
                  kahan_add(Sx, Cx, px);
                  kahan_add(Sy, Cy, py);
                  kahan_add(Sz, Cz, pz);
                  kahan_add(Sp, Cp, pp);
                } else {
                  Sx += px;
                  Sy += py;
                  Sz += pz;
                  Sp += pp;
                }
              }
            }
          }
        }
      }
    }
    if (active) {
      const float g0 = ((Sx - Cx) + lx) * a.GM;
      const float g1 = ((Sy - Cy) + ly) * a.GM;
      const float g2 = ((Sz - Cz) + lz) * a.GM;
      const float ph = ((Sp - Cp) + lp) * a.GM;
      a.gx[i] = g0;
      a.gy[i] = g1;
      a.gz[i] = g2;
      a.pot[i] = ph;
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
  }
}

}  // namespace

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
  a.phi = c->phi;
  a.err = c->d_err;
  a.C = C;
  a.N = c->N;
  a.b0 = b[0];
  a.b1 = b[1];
  a.b2 = b[2];
  a.s1 = e[1] - b[1];
  a.s2 = e[2] - b[2];
  a.min_rung = min_rung;
  a.first_call = first_call ? 1 : 0;
  a.kahan = c->opt.kahan ? 1 : 0;
  // kernel_params (src/kick_pme.cu:439-453), all FP32.
  a.GM = (float)c->opt.GM;
  a.eta = (float)c->opt.eta;
  a.t0 = (float)t0;
  a.scale = (float)scale;
  a.hsoft = (float)c->opt.hsoft;
  const float rs = (float)c->rs_box;
  a.inv2rs = 1.0f / rs / 2.0f;
  a.twooversqrtpi = 2.0f / sqrtf((float)M_PI);
  a.h2 = a.hsoft * a.hsoft;
  a.hinv = 1.f / a.hsoft;
  a.h3inv = a.hinv * (a.hinv * a.hinv);
  a.rcut2 = c->rcut_box > 0 ? (float)(c->rcut_box * c->rcut_box) : INFINITY;
  stage_begin(c, kStKick);
  if (ncell > 0) {
    k_kick_pme<<<(unsigned)ncell, kKickThreads, 0, c->stream>>>(a);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
  }
  stage_end(c, kStKick);
  return TPM_OK;
}

}  // namespace tpm
