// integrate.cu -- rung-based kick-drift-kick integration over one big step,
// and FP64 energy / momentum diagnostics.
//
// The reference supplies the kick of a block time-step scheme but no driver
// and no drift: kick_pme(box, min_rung, scale, t0, first_call) kicks the
// particles with rung >= min_rung -- a closing half-kick with the old
// rung's 0.5 * 2^-rung * t0 (skipped on the first call), a new rung from
// dt = min(eta sqrt(scale h) |g|^-1/2, t0) limited to one rung down, and an
// opening half-kick with the new rung's dt (src/kick_pme.cu:319-354,
// rung_dt src/fmmpm.cu:18).  The driver here schedules those kicks over one
// big step t0 on integer ticks (2^31 per t0):
//
//   begin      (first_call) kick all particles: opening half-kicks, rungs set
//   substep    R = the largest rung present; step = 2^(31-R) ticks; drift all
//              particles to the next multiple of the step; kick with
//              min_rung = 31 - ctz(tick) (rung r is due when 2^(31-r) divides
//              the tick); at tick 2^31 every particle is due
//
// so a particle on rung r is kicked every t0 / 2^r, each kick closing one
// half-step and opening the next, and positions move between kicks with the
// velocity of the opened half-step.  Every kick is a whole PME force
// evaluation (chain-mesh sort + long-range solve + kick of the due sinks).
#include "tpm_internal.cuh"

#include <string>

namespace tpm {
namespace {

constexpr int kTickRung = 31;
constexpr int64_t kTicks = (int64_t)1 << kTickRung;

__global__ void k_max_rung(int64_t n, const int8_t* __restrict__ rung, int* __restrict__ out) {
  int m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (int)rung[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// FP64 sums: 0.5 v^2, 0.5 phi, v (per particle; the host divides by n).
__global__ void k_diagnostics(int64_t n, const float* __restrict__ vx, const float* __restrict__ vy,
                              const float* __restrict__ vz, const float* __restrict__ pot, double* __restrict__ out) {
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = vx[i], b = vy[i], c = vz[i];
    s[0] += 0.5 * (a * a + b * b + c * c);
    s[1] += pot ? 0.5 * (double)pot[i] : 0.0;
    s[2] += a;
    s[3] += b;
    s[4] += c;
  }
  __shared__ double sh[5][32];
#pragma unroll
  for (int k = 0; k < 5; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = s[k];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[threadIdx.x][w];
    atomicAdd(out + threadIdx.x, t);
  }
}

int max_rung(tpm_ctx* c, int* out) {
  int* d = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(int), c->stream));
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(int), c->stream);
  if (e == cudaSuccess && c->n > 0) {
    k_max_rung<<<(int)std::min<int64_t>(ceil_div(c->n, 256), 148 * 8), 256, 0, c->stream>>>(c->n, c->rung, d);
    c->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("max rung: ") + cudaGetErrorString(e));
  return TPM_OK;
}

int whole_kick(tpm_ctx* c, int min_rung, double scale, double t0, int first_call) {
  int rc = chainmesh_sort(c);
  if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
  if (rc == TPM_OK) rc = kick_pme(c, nullptr, min_rung, scale, t0, first_call);
  return rc;
}

int check_err(tpm_ctx* c) {
  int err = 0;
  TPM_CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (err) {
    TPM_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    if (err & kErrRung) return fail(TPM_ERR_RUNG, "a new rung fell outside [0, 32) and was clamped");
    return fail(TPM_ERR_INVALID, "|v * dt| >= 2^31 box lengths for some particle (left unmoved)");
  }
  return TPM_OK;
}

}  // namespace
}  // namespace tpm

using namespace tpm;

extern "C" {

int tpm_integrate_begin(tpm_ctx* c, double t0, double scale, int first_call) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (!(t0 > 0) || !(scale > 0)) return fail(TPM_ERR_INVALID, "t0 and scale must be positive");
  c->int_t0 = t0;
  c->int_scale = scale;
  c->int_tick = 0;
  c->int_active = true;
  if (first_call) {
    int rc = whole_kick(c, 0, scale, t0, 1);
    if (rc == TPM_OK) rc = check_err(c);
    if (rc) {
      c->int_active = false;
      return rc;
    }
  }
  return TPM_OK;
}

int tpm_integrate_substep(tpm_ctx* c, tpm_substep* info) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (!c->int_active) return fail(TPM_ERR_STATE, "tpm_integrate_begin first (or the big step is complete)");
  int R = 0;
  int rc = max_rung(c, &R);
  if (rc) return rc;
  R = std::min(std::max(R, 0), kTickRung);
  const int64_t step = (int64_t)1 << (kTickRung - R);
  const int64_t t_prev = c->int_tick;
  const int64_t t_next = (t_prev / step + 1) * step;
  const double dt = (double)(t_next - t_prev) * (c->int_t0 / (double)kTicks);
  rc = drift(c, dt);
  if (rc == TPM_OK) rc = check_err(c);
  if (rc) return rc;
  c->int_tick = t_next;
  int tz = 0;
  while (tz < kTickRung && !((t_next >> tz) & 1)) tz++;
  const int min_rung = t_next >= kTicks ? 0 : kTickRung - tz;
  rc = whole_kick(c, min_rung, c->int_scale, c->int_t0, 0);
  if (rc == TPM_OK) rc = check_err(c);
  if (info) {
    info->tick = t_next;
    info->ticks_per_step = kTicks;
    info->max_rung = R;
    info->min_rung = min_rung;
    info->drift_dt = dt;
    info->done = t_next >= kTicks ? 1 : 0;
  }
  if (t_next >= kTicks) c->int_active = false;
  return rc;
}

int tpm_integrate(tpm_ctx* c, double t0, double scale, int first_call, int max_substeps, tpm_substep* log,
                  int log_cap, int* nsub) {
  if (!c || max_substeps < 1) return fail(TPM_ERR_INVALID, "bad arguments");
  int rc = tpm_integrate_begin(c, t0, scale, first_call);
  if (rc) return rc;
  int k = 0;
  while (c->int_active) {
    if (k >= max_substeps) {
      c->int_active = false;
      if (nsub) *nsub = k;
      return fail(TPM_ERR_INVALID, "more than max_substeps substeps in one big step");
    }
    tpm_substep s;
    rc = tpm_integrate_substep(c, &s);
    if (log && k < log_cap) log[k] = s;
    k++;
    if (rc) break;
  }
  if (nsub) *nsub = k;
  return rc;
}

int tpm_diagnostics(tpm_ctx* c, tpm_diag* out) {
  if (!c || !out) return fail(TPM_ERR_INVALID, "null argument");
  double* d = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(double) * 5, c->stream));
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(double) * 5, c->stream);
  if (e == cudaSuccess && c->n > 0) {
    k_diagnostics<<<(int)std::min<int64_t>(ceil_div(c->n, 256), 148 * 8), 256, 0, c->stream>>>(
        c->n, c->vx, c->vy, c->vz, c->pot_valid ? c->pot : nullptr, d);
    c->launches++;
    e = cudaGetLastError();
  }
  double h[5] = {0, 0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("diagnostics: ") + cudaGetErrorString(e));
  const double inv = c->n > 0 ? 1.0 / (double)c->n : 0.0;
  out->kinetic = h[0] * inv;
  out->potential = c->pot_valid ? h[1] * inv : NAN;
  out->momentum[0] = h[2] * inv;
  out->momentum[1] = h[3] * inv;
  out->momentum[2] = h[4] * inv;
  out->n = c->n;
  return TPM_OK;
}

}  // extern "C"
