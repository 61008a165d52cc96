// ewald_noalloc.cu -- the FP64 Ewald sum at sampled sinks for callers that
// cannot allocate device memory.
//
// Some callers must not call cudaMalloc: a host that owns every byte of
// device memory through its own pool and forbids other allocators, or code
// that runs where an allocation would synchronise the device or fail (an
// allocation-free measurement hook inside a running simulation step).  For
// them, tpm_ewald_fp64_noalloc computes what tpm_gravity_short_ewald does with
// method 1 (alpha = 6, real-space images with r < 0.8, reciprocal vectors with
// |h|^2 <= 120 through structure factors), but every scratch byte lives in
// one fixed buffer compiled into the library, g_scratch below.  The caller
// passes the sources, the sinks and the four outputs, all in device memory.
//
// The buffer is a file-scope __device__ array: every GPU that loads the
// library holds its kScratchBytes until the process exits.  In host code the
// name g_scratch is only a stand-in for that array, never a device address;
// the address is obtained once per device with cudaGetSymbolAddress (see
// setup()), with that device current, on the first call made on it.  That
// first call also copies the reciprocal-vector table into the buffer with a
// synchronous cudaMemcpy, so it should come before any stream capture.
//
// All calls share the one buffer: calls that overlap on the GPU (different
// streams, or different host threads) race on it and must be serialised by
// the caller.  Each call rewrites every scratch entry it later reads
// (partials, near-pair counts, structure factors), so nothing has to be
// cleared between calls.
#include "tpm_internal.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace tpm {
namespace noalloc {

constexpr int kThreads = 256;
constexpr int kMaxParts = 8192;  // sinks x chunks (at most 4096 + 1184 here)
constexpr int kMaxH = 4096;      // reciprocal vectors (half space, |h|^2 <= 120)
constexpr double kPi = 3.141592653589793;
constexpr double kAlpha = 6.0;
constexpr double kRc2 = 0.8 * 0.8;
constexpr int kHmax2 = 120;

struct HVec {
  int h[3];
  int pad;
  double c0;  // -(1/(pi h^2)) exp(-pi^2 h^2 / alpha^2)
};

constexpr size_t kOffParts = 0;
constexpr size_t kOffNear = kOffParts + sizeof(double) * 4 * kMaxParts;
constexpr size_t kOffS = kOffNear + sizeof(int) * kMaxParts;
constexpr size_t kOffH = kOffS + sizeof(double) * 2 * kMaxH;
constexpr size_t kScratchBytes = kOffH + sizeof(HVec) * kMaxH;  // 448 KiB

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__device__ __forceinline__ double dist64(uint32_t a, uint32_t b) {
  return (double)(int32_t)(a - b) * 2.3283064365386963e-10;
}

__device__ __forceinline__ void reduce4(double v[4], double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < 4; c++) sm[warp * 4 + c] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < (int)(blockDim.x >> 5); w++)
#pragma unroll
      for (int c = 0; c < 4; c++) v[c] += sm[w * 4 + c];
}

struct Args {
  const uint32_t* x;
  const uint32_t* y;
  const uint32_t* z;
  int64_t n;
  const uint32_t* sx;
  const uint32_t* sy;
  const uint32_t* sz;
  int nchunk;
  int nh;
  double h2, hinv, h3inv;
  unsigned char* scratch;
};

__device__ __forceinline__ void softened(double X, double Y, double Z, double R2, const Args& a, double* acc) {
  const double q2 = R2 * a.hinv * a.hinv;
  const double rinv3 = ((15.0 / 8.0 * q2 - 21.0 / 4.0) * q2 + 35.0 / 8.0) * a.h3inv;
  const double rinv = (((-5.0 / 16.0 * q2 + 21.0 / 16.0) * q2 - 35.0 / 16.0) * q2 + 35.0 / 16.0) * a.hinv;
  acc[0] -= rinv;
  acc[1] -= X * rinv3;
  acc[2] -= Y * rinv3;
  acc[3] -= Z * rinv3;
}

// Structure factors S(h) = sum_j (cos, sin)(2 pi h.x_j), 8 vectors per block.
__global__ void __launch_bounds__(kThreads) k_structure(Args a) {
  constexpr int K = 8;
  __shared__ double sm[2 * K * (kThreads / 32)];
  const HVec* hv = reinterpret_cast<const HVec*>(a.scratch + kOffH);
  double* S = reinterpret_cast<double*>(a.scratch + kOffS);
  const int h0 = blockIdx.x * K;
  double cs[K], sn[K];
  int hh[K][3];
#pragma unroll
  for (int k = 0; k < K; k++) {
    cs[k] = sn[k] = 0;
    const int id = min(h0 + k, a.nh - 1);
    hh[k][0] = hv[id].h[0];
    hh[k][1] = hv[id].h[1];
    hh[k][2] = hv[id].h[2];
  }
  for (int64_t j = threadIdx.x; j < a.n; j += blockDim.x) {
    const double X = (double)a.x[j] * 2.3283064365386963e-10;
    const double Y = (double)a.y[j] * 2.3283064365386963e-10;
    const double Z = (double)a.z[j] * 2.3283064365386963e-10;
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s, c;
      const double ph = X * hh[k][0] + Y * hh[k][1] + Z * hh[k][2];
      sincospi(2.0 * (ph - rint(ph)), &s, &c);
      cs[k] += c;
      sn[k] += s;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      cs[k] += __shfl_down_sync(0xffffffffu, cs[k], o);
      sn[k] += __shfl_down_sync(0xffffffffu, sn[k], o);
    }
    if (lane == 0) {
      sm[(warp * K + k) * 2] = cs[k];
      sm[(warp * K + k) * 2 + 1] = sn[k];
    }
  }
  __syncthreads();
  if (threadIdx.x < K && h0 + (int)threadIdx.x < a.nh) {
    double c = 0, s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      c += sm[(w * K + threadIdx.x) * 2];
      s += sm[(w * K + threadIdx.x) * 2 + 1];
    }
    S[(h0 + threadIdx.x) * 2] = c;
    S[(h0 + threadIdx.x) * 2 + 1] = s;
  }
}

// Real-space images of every pair; a near pair (minimum image <= hsoft)
// takes the softened kernel and has its reciprocal terms taken back out.
__global__ void __launch_bounds__(kThreads) k_real(Args a) {
  __shared__ double sm[4 * (kThreads / 32)];
  __shared__ int snear;
  if (threadIdx.x == 0) snear = 0;
  __syncthreads();
  const HVec* hv = reinterpret_cast<const HVec*>(a.scratch + kOffH);
  const int s = blockIdx.y, ch = blockIdx.x;
  const int64_t lo = a.n * ch / a.nchunk, hi = a.n * (ch + 1) / a.nchunk;
  const uint32_t px = a.sx[s], py = a.sy[s], pz = a.sz[s];
  double acc[4] = {0, 0, 0, 0};
  const double a2 = kAlpha * kAlpha, c2a = 2.0 * kAlpha / sqrt(kPi);
  int mynear = 0;
  for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    const double X = dist64(px, a.x[j]), Y = dist64(py, a.y[j]), Z = dist64(pz, a.z[j]);
    const double R2 = X * X + Y * Y + Z * Z;
    if (R2 > a.h2) {
      for (int xi = -1; xi <= 1; xi++) {
        const double dx = X - xi;
        if (dx * dx >= kRc2) continue;
        for (int yi = -1; yi <= 1; yi++) {
          const double dy = Y - yi;
          if (dx * dx + dy * dy >= kRc2) continue;
          for (int zi = -1; zi <= 1; zi++) {
            const double dz = Z - zi;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < kRc2) {
              const double r = sqrt(r2);
              const double rinv = 1.0 / r;
              const double erfc0 = erfc(kAlpha * r);
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
      softened(X, Y, Z, R2, a, acc);
      for (int k = 0; k < a.nh; k++) {
        const HVec v = hv[k];
        double sn, cs;
        sincospi(2.0 * (X * v.h[0] + Y * v.h[1] + Z * v.h[2]), &sn, &cs);
        const double c0 = -2.0 * v.c0;
        acc[0] += c0 * cs;
        const double c1 = 2.0 * kPi * c0 * sn;
        acc[1] += c1 * v.h[0];
        acc[2] += c1 * v.h[1];
        acc[3] += c1 * v.h[2];
      }
    }
  }
  if (mynear) atomicAdd(&snear, mynear);
  reduce4(acc, sm);
  if (threadIdx.x == 0) {
    double* o = reinterpret_cast<double*>(a.scratch + kOffParts) + ((int64_t)s * a.nchunk + ch) * 4;
    for (int c = 0; c < 4; c++) o[c] = acc[c];
    reinterpret_cast<int*>(a.scratch + kOffNear)[(int64_t)s * a.nchunk + ch] = snear;
  }
}

// Reciprocal sum from the structure factors, then phi = 35/(16h) + real +
// recip + (n - near) pi / alpha^2, written to the caller's arrays.
__global__ void __launch_bounds__(kThreads) k_finish(Args a, double* __restrict__ phi, double* __restrict__ gx,
                                                     double* __restrict__ gy, double* __restrict__ gz) {
  __shared__ double sm[4 * (kThreads / 32)];
  const HVec* hv = reinterpret_cast<const HVec*>(a.scratch + kOffH);
  const double* S = reinterpret_cast<const double*>(a.scratch + kOffS);
  const int s = blockIdx.x;
  double acc[4] = {0, 0, 0, 0};
  const double X = (double)a.sx[s] * 2.3283064365386963e-10;
  const double Y = (double)a.sy[s] * 2.3283064365386963e-10;
  const double Z = (double)a.sz[s] * 2.3283064365386963e-10;
  for (int k = threadIdx.x; k < a.nh; k += blockDim.x) {
    const HVec v = hv[k];
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
  reduce4(acc, sm);
  if (threadIdx.x == 0) {
    const double* parts = reinterpret_cast<const double*>(a.scratch + kOffParts);
    const int* nearc = reinterpret_cast<const int*>(a.scratch + kOffNear);
    int64_t nnear = 0;
    for (int ch = 0; ch < a.nchunk; ch++) {
      const double* p = parts + ((int64_t)s * a.nchunk + ch) * 4;
      for (int c = 0; c < 4; c++) acc[c] += p[c];
      nnear += nearc[(int64_t)s * a.nchunk + ch];
    }
    acc[0] += 35.0 / 16.0 * a.hinv;  // -SELF_PHI / h cancels the sink's own softened term
    acc[0] += (double)(a.n - nnear) * kPi / (kAlpha * kAlpha);
    phi[s] = acc[0];
    gx[s] = acc[1];
    gy[s] = acc[2];
    gz[s] = acc[3];
  }
}

struct DeviceState {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_scratch on this device
  int nh = 0;
};
constexpr int kMaxDevices = 64;
DeviceState g_state[kMaxDevices];
std::mutex g_mutex;

// Once per device, with it current: the device address of g_scratch and the
// reciprocal-vector table copied into it.
int setup(int dev, DeviceState** out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceState& st = g_state[dev];
  if (!st.ready) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess)
      return fail(TPM_ERR_CUDA, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
    std::vector<HVec> hv;
    const int hm = (int)std::floor(std::sqrt((double)kHmax2));
    for (int i = -hm; i <= hm; i++)
      for (int j = -hm; j <= hm; j++)
        for (int k = -hm; k <= hm; k++) {
          const int hh = i * i + j * j + k * k;
          if (hh == 0 || hh > kHmax2) continue;
          if (i < 0 || (i == 0 && j < 0) || (i == 0 && j == 0 && k < 0)) continue;  // one of each +-h
          HVec v;
          v.h[0] = i;
          v.h[1] = j;
          v.h[2] = k;
          v.pad = 0;
          v.c0 = -1.0 / hh * std::exp(-kPi * kPi * hh / (kAlpha * kAlpha)) / kPi;
          hv.push_back(v);
        }
    if ((int)hv.size() > kMaxH) return fail(TPM_ERR_INVALID, "reciprocal-vector table exceeds its buffer");
    const cudaError_t e2 =
        cudaMemcpy((unsigned char*)ptr + kOffH, hv.data(), sizeof(HVec) * hv.size(), cudaMemcpyHostToDevice);
    if (e2 != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("reciprocal table: ") + cudaGetErrorString(e2));
    // A pageable cudaMemcpy may return once the data is staged, before it
    // lands; kernels on a non-blocking caller stream (or another thread that
    // sees `ready`) must not read the table early, so wait for the device.
    const cudaError_t e3 = cudaDeviceSynchronize();
    if (e3 != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("reciprocal table sync: ") + cudaGetErrorString(e3));
    st.scratch = (unsigned char*)ptr;
    st.nh = (int)hv.size();
    st.ready = true;
  }
  *out = &st;
  return TPM_OK;
}

}  // namespace noalloc
}  // namespace tpm

extern "C" int tpm_ewald_fp64_noalloc(const uint32_t* x, const uint32_t* y, const uint32_t* z, int64_t n,
                                      const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, int64_t ns,
                                      double hsoft, double* phi, double* gx, double* gy, double* gz,
                                      void* stream) {
  using namespace tpm;
  using namespace tpm::noalloc;
  if (ns < 0 || n < 0) return fail(TPM_ERR_INVALID, "negative count");
  if (ns > TPM_EWALD_NOALLOC_MAX_SINKS)
    return fail(TPM_ERR_INVALID, "tpm_ewald_fp64_noalloc: " + std::to_string(ns) + " sinks exceed its maximum of " +
                                     std::to_string(TPM_EWALD_NOALLOC_MAX_SINKS));
  if (n > 0x7fffffffLL) return fail(TPM_ERR_INVALID, "tpm_ewald_fp64_noalloc: more than 2^31 - 1 sources");
  if (!(hsoft > 0)) return fail(TPM_ERR_INVALID, "hsoft must be positive");
  if (ns == 0) return TPM_OK;
  if ((n > 0 && (!x || !y || !z)) || !sx || !sy || !sz || !phi || !gx || !gy || !gz)
    return fail(TPM_ERR_INVALID, "null pointer");
  int dev = 0;
  TPM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(TPM_ERR_INVALID, "device index above the supported range");
  DeviceState* st = nullptr;
  int rc = setup(dev, &st);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the same chunking as tpm_gravity_short_ewald, so the sums agree term by term
  int nchunk = (int)std::max<int64_t>(1, std::min<int64_t>(1024, (148 * 8 + ns - 1) / ns));
  nchunk = (int)std::min<int64_t>(nchunk, std::max<int64_t>(1, n / 1024));
  if ((int64_t)ns * nchunk > kMaxParts) return fail(TPM_ERR_INVALID, "partial-sum buffer too small");
  Args a;
  a.x = x;
  a.y = y;
  a.z = z;
  a.n = n;
  a.sx = sx;
  a.sy = sy;
  a.sz = sz;
  a.nchunk = nchunk;
  a.nh = st->nh;
  a.h2 = hsoft * hsoft;
  a.hinv = 1.0 / hsoft;
  a.h3inv = a.hinv * a.hinv * a.hinv;
  a.scratch = st->scratch;
  k_structure<<<ceil_div(a.nh, 8), kThreads, 0, s>>>(a);
  k_real<<<dim3(nchunk, (unsigned)ns), kThreads, 0, s>>>(a);
  k_finish<<<(unsigned)ns, kThreads, 0, s>>>(a, phi, gx, gy, gz);
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}
