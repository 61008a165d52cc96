// drift.cu -- fixed-point drift.
//
// The reference has no drift routine.  This one follows the semantics of its
// fixed<uint32_t> positions (tigerpm/fixed.hpp:63-75,184-195): a displacement
// v*dt (box units) becomes trunc(v*dt*2^32) counts, added modulo 2^32, so the
// periodic wrap is exact integer arithmetic.  The product is formed in double
// as (double(v) * dt) * 2^32 with explicit round-to-nearest multiplies (no
// contraction), which makes the result bit-identical to the same arithmetic
// on the host.
#include "tpm_internal.cuh"

namespace tpm {
namespace {

__global__ void k_drift(int64_t n, uint32_t* __restrict__ x, uint32_t* __restrict__ y, uint32_t* __restrict__ z,
                        const float* __restrict__ vx, const float* __restrict__ vy,
                        const float* __restrict__ vz, double dt, int* __restrict__ err) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t* X[3] = {x, y, z};
  const float* V[3] = {vx, vy, vz};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double t = __dmul_rn((double)V[d][i], dt);
    if (!(fabs(t) < 2147483648.0)) {
      atomicOr(err, kErrBounds);
      continue;
    }
    const long long di = __double2ll_rz(__dmul_rn(t, 4294967296.0));
    X[d][i] = (uint32_t)((unsigned long long)X[d][i] + (unsigned long long)di);
  }
}

}  // namespace

int drift(tpm_ctx* c, double dt) {
  stage_begin(c, kStDrift);
  if (c->n > 0) {
    k_drift<<<ceil_div(c->n, 256), 256, 0, c->stream>>>(c->n, c->x, c->y, c->z, c->vx, c->vy, c->vz, dt,
                                                        c->d_err);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
  }
  stage_end(c, kStDrift);
  // positions moved: the chain mesh, packed positions and potential are stale
  c->sorted = false;
  c->have_phi = false;
  c->pot_valid = false;
  c->host_cells_valid = false;
  return TPM_OK;
}

}  // namespace tpm
