// misc.cu -- whole-step entry point, pair counting and the FP32 peak probe.
#include "tpm_internal.cuh"

#include <cmath>

namespace tpm {
namespace {

// Candidate pairs (every sink of a cell x every source of its 27
// neighbours) and pairs inside the cutoff, for the roofline's algorithmic
// flop count.  One block per sink cell, same traversal as the kick.
__global__ void __launch_bounds__(256) k_count_pairs(const int4* __restrict__ pos4, const int8_t* __restrict__ rung,
                                                     const int32_t* __restrict__ begin, int C, int min_rung,
                                                     float rcut2, unsigned long long* __restrict__ out) {
  __shared__ float4 src[1024];
  __shared__ unsigned long long s_cand, s_in;
  const int cx = blockIdx.x % C, cy = (blockIdx.x / C) % C, cz = blockIdx.x / (C * C);
  const int64_t key = ((int64_t)cz * C + cy) * C + cx;
  const int32_t pb = begin[key], pe = begin[key + 1];
  if (pb == pe) return;
  if (threadIdx.x == 0) s_cand = s_in = 0;
  const uint32_t ox = (uint32_t)((((uint64_t)(2 * cx + 1)) << 31) / (uint64_t)C);
  const uint32_t oy = (uint32_t)((((uint64_t)(2 * cy + 1)) << 31) / (uint64_t)C);
  const uint32_t oz = (uint32_t)((((uint64_t)(2 * cz + 1)) << 31) / (uint64_t)C);
  unsigned long long cand = 0, in = 0;
  for (int32_t sbase = pb; sbase < pe; sbase += blockDim.x) {
    const int32_t i = sbase + threadIdx.x;
    const bool active = i < pe && rung[i] >= min_rung;
    float sx = 0, sy = 0, sz = 0;
    if (active) {
      const int4 q = pos4[i];
      sx = distance32((uint32_t)q.x, ox);
      sy = distance32((uint32_t)q.y, oy);
      sz = distance32((uint32_t)q.z, oz);
    }
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int64_t k2 = ((int64_t)wrapi(cz + dz, C) * C + wrapi(cy + dy, C)) * C + wrapi(cx + dx, C);
          const int32_t b = begin[k2], e = begin[k2 + 1];
          for (int32_t t0 = b; t0 < e; t0 += 1024) {
            const int len = min(1024, e - t0);
            __syncthreads();
            for (int j = threadIdx.x; j < len; j += blockDim.x) {
              const int4 q = pos4[t0 + j];
              src[j] = make_float4(distance32((uint32_t)q.x, ox), distance32((uint32_t)q.y, oy),
                                   distance32((uint32_t)q.z, oz), 0.f);
            }
            __syncthreads();
            if (active) {
              cand += len;
              for (int j = 0; j < len; j++) {
                const float4 s = src[j];
                float ddx = sx - s.x, ddy = sy - s.y, ddz = sz - s.z;
                if (C == 3) {  // minimum image, as in the kick
                  ddx -= rintf(ddx);
                  ddy -= rintf(ddy);
                  ddz -= rintf(ddz);
                }
                in += fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz)) < rcut2 ? 1 : 0;
              }
            }
          }
        }
  }
  atomicAdd(&s_cand, cand);
  atomicAdd(&s_in, in);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(out, s_cand);
    atomicAdd(out + 1, s_in);
  }
}

// Dense independent FMA chains: 8 accumulators per thread.
__global__ void __launch_bounds__(256) k_fma_probe(int iters, float a, float b, float* __restrict__ sink) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = (float)(threadIdx.x + k) * 1e-7f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = fmaf(r[k], a, b);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += r[k];
  if (s == 12345.678f) sink[0] = s;  // keeps the chains live
}

}  // namespace
}  // namespace tpm

using namespace tpm;

extern "C" {

int tpm_ctx_stream(tpm_ctx* c, void** stream) {
  if (!c || !stream) return fail(TPM_ERR_INVALID, "null argument");
  *stream = (void*)c->stream;
  return TPM_OK;
}

int tpm_pme_step(tpm_ctx* c, int min_rung, double scale, double t0, int first_call) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  int rc = chainmesh_sort(c);
  if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
  if (rc == TPM_OK) rc = kick_pme(c, nullptr, min_rung, scale, t0, first_call);
  return rc;
}

int tpm_check_errors(tpm_ctx* c) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  int err = 0;
  TPM_CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (err) {
    TPM_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (err & kErrTimeout) return fail(TPM_ERR_TIMEOUT, "a bounded device wait (scan look-back) gave up");
    if (err & kErrRung) return fail(TPM_ERR_RUNG, "a new rung fell outside [0, 32) and was clamped");
    return fail(TPM_ERR_INVALID, "a drift step exceeded 2^31 box lengths");
  }
  return TPM_OK;
}

int tpm_count_pairs(tpm_ctx* c, int min_rung, int64_t* candidates, int64_t* inside) {
  if (!c || !candidates || !inside) return fail(TPM_ERR_INVALID, "null argument");
  if (!c->sorted) return fail(TPM_ERR_STATE, "count_pairs needs chainmesh_create first");
  unsigned long long* d = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&d, 16, c->stream));
  cudaError_t e = cudaMemsetAsync(d, 0, 16, c->stream);
  const float rcut2 = c->rcut_box > 0 ? (float)(c->rcut_box * c->rcut_box) : INFINITY;
  const int64_t ncell = (int64_t)c->C * c->C * c->C;
  if (e == cudaSuccess && ncell > 0) {
    k_count_pairs<<<(unsigned)ncell, 256, 0, c->stream>>>(c->pos4, c->rung, c->cell_begin, c->C, min_rung,
                                                          rcut2, d);
    c->launches++;
    e = cudaGetLastError();
  }
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("count_pairs: ") + cudaGetErrorString(e));
  *candidates = (int64_t)h[0];
  *inside = (int64_t)h[1];
  return TPM_OK;
}

int tpm_fp32_peak_probe(double* tflops) {
  if (!tflops) return fail(TPM_ERR_INVALID, "null argument");
  int dev = 0, sms = 0;
  TPM_CUDA_TRY(cudaGetDevice(&dev));
  TPM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  float* sink = nullptr;
  TPM_CUDA_TRY(cudaMalloc((void**)&sink, sizeof(float)));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = sms * 8, threads = 256, iters = 1 << 16;
  k_fma_probe<<<blocks, threads>>>(1024, 0.999f, 1e-3f, sink);  // warm-up
  cudaEventRecord(a);
  k_fma_probe<<<blocks, threads>>>(iters, 0.999f, 1e-3f, sink);
  cudaEventRecord(b);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, cudaGetErrorString(e));
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return TPM_OK;
}

}  // extern "C"
