// ewald.cu -- FP64 periodic Ewald potential and force at sampled sinks.
//
// Reference: gravity_short_ewald_call_kernel / gravity_ewald_kernel
// (src/gravity_short.cu:10-201), the oracle that gravity_short_ewald_compare
// (src/gravity_short.cpp:35-82) grades kicks with.  The reference evaluates
// FP32 terms and sums them in FP64; here every term is FP64.
//
// Conventions kept from the reference: phi = -psi with psi the zero-mean
// periodic 1/r potential (real-space erfc images, reciprocal Gaussian terms
// and the +pi/alpha^2 background per source); a source whose minimum-image
// distance is <= hsoft takes the softened Newtonian kernel only (no images,
// no reciprocal or background term); phi starts at -SELF_PHI/h = 35/(16h),
// which cancels the sink's own softened term.
//
// method 0: the reference's sum, alpha = 2: real images |n_i| <= 4 with
//           r < 2.6, reciprocal |h|^2 <= 8 (src/gravity_short.cu:117-164).
// method 1: alpha = 6, real images with r < 0.8 (erfc(4.8) = 6e-12) and
//           |h|^2 <= 120 (exp(-pi^2 120/36) = 5e-15) through precomputed
//           structure factors S(h) = sum_j exp(2 pi i h.x_j); near pairs
//           have their reciprocal terms subtracted explicitly.  Same limit,
//           O(ns * n) real-space work with ~2 images per pair.
#include "tpm_internal.cuh"

#include <cmath>

namespace tpm {
namespace {

constexpr int kEwThreads = 256;
constexpr double kPi = 3.141592653589793;

struct HVec {
  int h[3];
  int pad;
  double c0;  // -(1/(pi h^2)) exp(-pi^2 h^2 / alpha^2)
};

__device__ __forceinline__ double dist64(uint32_t a, uint32_t b) {
  return (double)(int32_t)(a - b) * 2.3283064365386963e-10;
}

__device__ __forceinline__ void block_reduce4(double v[4], double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 4; c++) sm[warp * 4 + c] = v[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++)
#pragma unroll
      for (int c = 0; c < 4; c++) v[c] += sm[w * 4 + c];
  }
}

__device__ __forceinline__ void softened(double X, double Y, double Z, double R2, double hinv, double h3inv,
                                         double* acc) {
  const double q2 = R2 * hinv * hinv;
  const double rinv3 = ((15.0 / 8.0 * q2 - 21.0 / 4.0) * q2 + 35.0 / 8.0) * h3inv;
  const double rinv = (((-5.0 / 16.0 * q2 + 21.0 / 16.0) * q2 - 35.0 / 16.0) * q2 + 35.0 / 16.0) * hinv;
  acc[0] -= rinv;
  acc[1] -= X * rinv3;
  acc[2] -= Y * rinv3;
  acc[3] -= Z * rinv3;
}

// Reciprocal-space terms of one pair, summed over the listed half-space
// vectors (x2 for the mirror vectors).
__device__ void kspace_pair(double X, double Y, double Z, const HVec* __restrict__ hv, int nh, double sign,
                            double* acc) {
  for (int k = 0; k < nh; k++) {
    const HVec v = hv[k];
    double s, c;
    sincospi(2.0 * (X * v.h[0] + Y * v.h[1] + Z * v.h[2]), &s, &c);
    const double c0 = 2.0 * v.c0 * sign;
    acc[0] += c0 * c;
    const double c1 = 2.0 * kPi * c0 * s;
    acc[1] += c1 * v.h[0];
    acc[2] += c1 * v.h[1];
    acc[3] += c1 * v.h[2];
  }
}

struct EwArgs {
  const uint32_t* __restrict__ x;
  const uint32_t* __restrict__ y;
  const uint32_t* __restrict__ z;
  int64_t n;
  const uint32_t* __restrict__ sx;
  const uint32_t* __restrict__ sy;
  const uint32_t* __restrict__ sz;
  int nchunk;
  double h2, hinv, h3inv;
  const HVec* __restrict__ hv;
  int nh;
  double* __restrict__ part;  // [ns][nchunk][4]
  int* __restrict__ near;     // [ns][nchunk]
};

// method 0: the reference's per-pair sum, FP64.
__global__ void __launch_bounds__(kEwThreads) k_ewald_ref(EwArgs a) {
  __shared__ double sm[4 * (kEwThreads / 32)];
  const int s = blockIdx.y, ch = blockIdx.x;
  const int64_t lo = a.n * ch / a.nchunk, hi = a.n * (ch + 1) / a.nchunk;
  const uint32_t px = a.sx[s], py = a.sy[s], pz = a.sz[s];
  double acc[4] = {0, 0, 0, 0};
  const double a2 = 4.0;  // alpha^2, alpha = 2
  for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    const double X = dist64(px, a.x[j]), Y = dist64(py, a.y[j]), Z = dist64(pz, a.z[j]);
    const double R2 = X * X + Y * Y + Z * Z;
    if (R2 > a.h2) {
      for (int xi = -4; xi <= 4; xi++) {
        const double dx = X - xi;
        if (dx * dx >= 2.6 * 2.6) continue;
        for (int yi = -4; yi <= 4; yi++) {
          const double dy = Y - yi;
          if (dx * dx + dy * dy >= 2.6 * 2.6) continue;
          for (int zi = -4; zi <= 4; zi++) {
            const double dz = Z - zi;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < 2.6 * 2.6) {
              const double r = sqrt(r2);
              const double rinv = 1.0 / r;
              const double erfc0 = erfc(2.0 * r);
              const double expfactor = 4.0 / sqrt(kPi) * r * exp(-a2 * r2);
              const double d1 = (expfactor + erfc0) * rinv * rinv * rinv;
              acc[0] -= erfc0 * rinv;
              acc[1] -= dx * d1;
              acc[2] -= dy * d1;
              acc[3] -= dz * d1;
            }
          }
        }
      }
      acc[0] += kPi / a2;
      kspace_pair(X, Y, Z, a.hv, a.nh, 1.0, acc);
    } else {
      softened(X, Y, Z, R2, a.hinv, a.h3inv, acc);
    }
  }
  block_reduce4(acc, sm);
  if (threadIdx.x == 0) {
    double* o = a.part + ((int64_t)s * a.nchunk + ch) * 4;
    for (int c = 0; c < 4; c++) o[c] = acc[c];
  }
}

// method 1, real space + near-pair corrections.
__global__ void __launch_bounds__(kEwThreads) k_ewald_real(EwArgs a, double alpha, double rc2) {
  __shared__ double sm[4 * (kEwThreads / 32)];
  __shared__ int snear;
  if (threadIdx.x == 0) snear = 0;
  __syncthreads();
  const int s = blockIdx.y, ch = blockIdx.x;
  const int64_t lo = a.n * ch / a.nchunk, hi = a.n * (ch + 1) / a.nchunk;
  const uint32_t px = a.sx[s], py = a.sy[s], pz = a.sz[s];
  double acc[4] = {0, 0, 0, 0};
  const double a2 = alpha * alpha;
  const double c2a = 2.0 * alpha / sqrt(kPi);
  int mynear = 0;
  for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    const double X = dist64(px, a.x[j]), Y = dist64(py, a.y[j]), Z = dist64(pz, a.z[j]);
    const double R2 = X * X + Y * Y + Z * Z;
    if (R2 > a.h2) {
      for (int xi = -1; xi <= 1; xi++) {
        const double dx = X - xi;
        if (dx * dx >= rc2) continue;
        for (int yi = -1; yi <= 1; yi++) {
          const double dy = Y - yi;
          if (dx * dx + dy * dy >= rc2) continue;
          for (int zi = -1; zi <= 1; zi++) {
            const double dz = Z - zi;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < rc2) {
              const double r = sqrt(r2);
              const double rinv = 1.0 / r;
              const double erfc0 = erfc(alpha * r);
              const double d1 = (c2a * r * exp(-a2 * r2) + erfc0) * rinv * rinv * rinv;
              acc[0] -= erfc0 * rinv;
              acc[1] -= dx * d1;
              acc[2] -= dy * d1;
              acc[3] -= dz * d1;
            }
          }
        }
      }
    } else {
      mynear++;
      softened(X, Y, Z, R2, a.hinv, a.h3inv, acc);
      kspace_pair(X, Y, Z, a.hv, a.nh, -1.0, acc);  // undo its reciprocal terms
    }
  }
  if (mynear) atomicAdd(&snear, mynear);
  block_reduce4(acc, sm);
  if (threadIdx.x == 0) {
    double* o = a.part + ((int64_t)s * a.nchunk + ch) * 4;
    for (int c = 0; c < 4; c++) o[c] = acc[c];
    a.near[(int64_t)s * a.nchunk + ch] = snear;
  }
}

// Structure factors: one block per group of 8 reciprocal vectors.
constexpr int kHPerBlock = 8;
__global__ void __launch_bounds__(kEwThreads) k_structure(const uint32_t* __restrict__ x,
                                                          const uint32_t* __restrict__ y,
                                                          const uint32_t* __restrict__ z, int64_t n,
                                                          const HVec* __restrict__ hv, int nh,
                                                          double* __restrict__ S /* [nh][2] */) {
  __shared__ double sm[2 * kHPerBlock * (kEwThreads / 32)];
  const int h0 = blockIdx.x * kHPerBlock;
  double cs[kHPerBlock], sn[kHPerBlock];
  int hh[kHPerBlock][3];
#pragma unroll
  for (int k = 0; k < kHPerBlock; k++) {
    cs[k] = sn[k] = 0;
    const int id = min(h0 + k, nh - 1);
    hh[k][0] = hv[id].h[0];
    hh[k][1] = hv[id].h[1];
    hh[k][2] = hv[id].h[2];
  }
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    const double X = (double)x[j] * 2.3283064365386963e-10;
    const double Y = (double)y[j] * 2.3283064365386963e-10;
    const double Z = (double)z[j] * 2.3283064365386963e-10;
#pragma unroll
    for (int k = 0; k < kHPerBlock; k++) {
      double s, c;
      const double ph = X * hh[k][0] + Y * hh[k][1] + Z * hh[k][2];
      sincospi(2.0 * (ph - rint(ph)), &s, &c);
      cs[k] += c;
      sn[k] += s;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kHPerBlock; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      cs[k] += __shfl_down_sync(0xffffffffu, cs[k], o);
      sn[k] += __shfl_down_sync(0xffffffffu, sn[k], o);
    }
    if (lane == 0) {
      sm[(warp * kHPerBlock + k) * 2] = cs[k];
      sm[(warp * kHPerBlock + k) * 2 + 1] = sn[k];
    }
  }
  __syncthreads();
  if (threadIdx.x < kHPerBlock && h0 + (int)threadIdx.x < nh) {
    double c = 0, s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      c += sm[(w * kHPerBlock + threadIdx.x) * 2];
      s += sm[(w * kHPerBlock + threadIdx.x) * 2 + 1];
    }
    S[(h0 + threadIdx.x) * 2] = c;
    S[(h0 + threadIdx.x) * 2 + 1] = s;
  }
}

// Reciprocal sum at each sink from the structure factors, then the final
// combination: phi = 35/(16h) + real + recip + (n - near) pi/alpha^2.
__global__ void __launch_bounds__(kEwThreads) k_ewald_finish(EwArgs a, const double* __restrict__ S, double alpha,
                                                             int method, double* __restrict__ out) {
  __shared__ double sm[4 * (kEwThreads / 32)];
  const int s = blockIdx.x;
  double acc[4] = {0, 0, 0, 0};
  if (method == 1) {
    const double X = (double)a.sx[s] * 2.3283064365386963e-10;
    const double Y = (double)a.sy[s] * 2.3283064365386963e-10;
    const double Z = (double)a.sz[s] * 2.3283064365386963e-10;
    for (int k = threadIdx.x; k < a.nh; k += blockDim.x) {
      const HVec v = a.hv[k];
      const double ph = X * v.h[0] + Y * v.h[1] + Z * v.h[2];
      double sn, cs;
      sincospi(2.0 * (ph - rint(ph)), &sn, &cs);
      const double Sc = S[2 * k], Ss = S[2 * k + 1];
      const double c0 = 2.0 * v.c0;
      acc[0] += c0 * (cs * Sc + sn * Ss);
      const double f = 2.0 * kPi * c0 * (sn * Sc - cs * Ss);
      acc[1] += f * v.h[0];
      acc[2] += f * v.h[1];
      acc[3] += f * v.h[2];
    }
  }
  block_reduce4(acc, sm);
  if (threadIdx.x == 0) {
    int64_t nnear = 0;
    for (int ch = 0; ch < a.nchunk; ch++) {
      const double* p = a.part + ((int64_t)s * a.nchunk + ch) * 4;
      for (int c = 0; c < 4; c++) acc[c] += p[c];
      if (method == 1) nnear += a.near[(int64_t)s * a.nchunk + ch];
    }
    acc[0] += 35.0 / 16.0 * a.hinv;  // -SELF_PHI / h (src/gravity_short.cu:31)
    if (method == 1) acc[0] += (double)(a.n - nnear) * kPi / (alpha * alpha);
    for (int c = 0; c < 4; c++) out[(int64_t)c * gridDim.x + s] = acc[c];
  }
}

void make_hvecs(double alpha, int hmax2, std::vector<HVec>& out, bool half) {
  const int hm = (int)std::floor(std::sqrt((double)hmax2));
  for (int a = -hm; a <= hm; a++)
    for (int b = -hm; b <= hm; b++)
      for (int c = -hm; c <= hm; c++) {
        const int hh = a * a + b * b + c * c;
        if (hh == 0 || hh > hmax2) continue;
        if (half) {  // one of each +-h pair
          if (a < 0 || (a == 0 && b < 0) || (a == 0 && b == 0 && c < 0)) continue;
        }
        HVec v;
        v.h[0] = a;
        v.h[1] = b;
        v.h[2] = c;
        v.pad = 0;
        v.c0 = -1.0 / hh * std::exp(-kPi * kPi * hh / (alpha * alpha)) / kPi;
        out.push_back(v);
      }
}

}  // namespace

// dsx/dsy/dsz: device sink positions.  Outputs are host arrays.
int ewald(tpm_ctx* c, int64_t ns, const uint32_t* dsx, const uint32_t* dsy, const uint32_t* dsz, int method,
          double* phi, double* gx, double* gy, double* gz) {
  if (method != 0 && method != 1) return fail(TPM_ERR_INVALID, "ewald method must be 0 or 1");
  if (ns <= 0) return TPM_OK;
  if (ns > 65535) return fail(TPM_ERR_INVALID, "at most 65535 Ewald sinks per call");
  const double alpha = method == 0 ? 2.0 : 6.0;
  std::vector<HVec> hv;
  // method 0 keeps the reference's full set (|h|^2 <= 8, both signs) with the
  // factor 2 folded out; method 1 uses one of each +-h pair.
  make_hvecs(alpha, method == 0 ? 8 : 120, hv, true);
  const int nh = (int)hv.size();
  int nchunk = (int)std::max<int64_t>(1, std::min<int64_t>(1024, (148 * 8 + ns - 1) / ns));
  nchunk = (int)std::min<int64_t>(nchunk, std::max<int64_t>(1, c->n / 1024));
  const int64_t need = (int64_t)ns * nchunk * 4 + 4 * ns + 2 * (int64_t)nh + ns * nchunk + 64;
  stage_begin(c, kStEwald);
  double* buf = nullptr;
  HVec* dhv = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&buf, sizeof(double) * need, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&dhv, sizeof(HVec) * nh, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dhv, hv.data(), sizeof(HVec) * nh, cudaMemcpyHostToDevice, c->stream);
  EwArgs a;
  a.x = c->x;
  a.y = c->y;
  a.z = c->z;
  a.n = c->n;
  a.sx = dsx;
  a.sy = dsy;
  a.sz = dsz;
  a.nchunk = nchunk;
  const double h = c->opt.hsoft;
  a.h2 = h * h;
  a.hinv = 1.0 / h;
  a.h3inv = a.hinv * a.hinv * a.hinv;
  a.hv = dhv;
  a.nh = nh;
  a.part = buf;
  double* out = buf + (int64_t)ns * nchunk * 4;
  double* S = out + 4 * ns;
  a.near = (int*)(S + 2 * nh);
  if (e == cudaSuccess) {
    dim3 grid(nchunk, (unsigned)ns);
    if (method == 0) {
      k_ewald_ref<<<grid, kEwThreads, 0, c->stream>>>(a);
      c->launches++;
    } else {
      k_structure<<<ceil_div(nh, kHPerBlock), kEwThreads, 0, c->stream>>>(c->x, c->y, c->z, c->n, dhv, nh, S);
      k_ewald_real<<<grid, kEwThreads, 0, c->stream>>>(a, alpha, 0.8 * 0.8);
      c->launches += 2;
    }
    k_ewald_finish<<<(unsigned)ns, kEwThreads, 0, c->stream>>>(a, S, alpha, method, out);
    c->launches++;
    e = cudaGetLastError();
  }
  std::vector<double> host((size_t)4 * ns);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), out, sizeof(double) * 4 * ns, cudaMemcpyDeviceToHost, c->stream);
  if (buf) cudaFreeAsync(buf, c->stream);
  if (dhv) cudaFreeAsync(dhv, c->stream);
  stage_end(c, kStEwald);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("ewald: ") + cudaGetErrorString(e));
  for (int64_t s = 0; s < ns; s++) {
    if (phi) phi[s] = host[s];
    if (gx) gx[s] = host[ns + s];
    if (gy) gy[s] = host[2 * ns + s];
    if (gz) gz[s] = host[3 * ns + s];
  }
  return TPM_OK;
}

}  // namespace tpm
