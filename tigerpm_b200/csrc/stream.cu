// stream.cu -- a served stream of whole PME steps with the host transfers
// overlapped: step s+1's particles upload and step s-1's kicked particles
// download while step s's kernels run.
//
// The reference's kick_pme_test (src/test.cpp:182-234) and every kick_pme
// call (src/kick_pme.cu:390-621) move the particles host -> device, run the
// kernel, and move them back, one after the other.  Here a caller hands
// nsteps independent boxes at once; three device particle sets rotate:
//   step s reads set in(s) (uploaded), sorts into set out(s), kicks there,
//   and out(s) downloads once the kick is done;
//   in(s+1) = the third set (the one step s-1 sorted into, free once its
//   download completed); out(s+1) = in(s) (free once step s's sort gathered).
// Uploads and downloads run on their own streams, ordered against the
// compute stream with events, so PCIe carries both directions while the
// GPU computes.
#include "tpm_internal.cuh"

#include <string>

namespace tpm {
namespace {

struct DevSet {
  uint32_t *x, *y, *z;
  float *vx, *vy, *vz;
  int8_t* rung;
};

DevSet cur_set(tpm_ctx* c) { return DevSet{c->x, c->y, c->z, c->vx, c->vy, c->vz, c->rung}; }
DevSet scratch_set(tpm_ctx* c) { return DevSet{c->x2, c->y2, c->z2, c->vx2, c->vy2, c->vz2, c->rung2}; }

void bind(tpm_ctx* c, const DevSet& in, const DevSet& out) {
  c->x = in.x;
  c->y = in.y;
  c->z = in.z;
  c->vx = in.vx;
  c->vy = in.vy;
  c->vz = in.vz;
  c->rung = in.rung;
  c->x2 = out.x;
  c->y2 = out.y;
  c->z2 = out.z;
  c->vx2 = out.vx;
  c->vy2 = out.vy;
  c->vz2 = out.vz;
  c->rung2 = out.rung;
}

// Third particle set, two copy streams and the event rings, made on first use.
int stream_init(tpm_ctx* c) {
  if (c->pipe_ready) return TPM_OK;
  const int64_t cap = std::max<int64_t>(c->cap, 1);
  void** ptrs[] = {(void**)&c->x3, (void**)&c->y3, (void**)&c->z3, (void**)&c->vx3, (void**)&c->vy3, (void**)&c->vz3};
  for (void** p : ptrs) {
    cudaError_t e = cudaMalloc(p, 4 * cap);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(TPM_ERR_NOMEM, std::string("third particle set: ") + cudaGetErrorString(e));
    }
  }
  cudaError_t e = cudaMalloc((void**)&c->rung3, cap);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking);
  for (int k = 0; k < 3 && e == cudaSuccess; k++) {
    e = cudaEventCreateWithFlags(&c->ev_up[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_down[k], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(TPM_ERR_CUDA, std::string("stream set-up: ") + cudaGetErrorString(e));
  }
  c->pipe_ready = true;
  return TPM_OK;
}

int upload(const DevSet& d, const tpm_host_particles& h, int64_t n, cudaStream_t s) {
  TPM_CUDA_TRY(cudaMemcpyAsync(d.x, h.x, 4 * n, cudaMemcpyHostToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(d.y, h.y, 4 * n, cudaMemcpyHostToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(d.z, h.z, 4 * n, cudaMemcpyHostToDevice, s));
  if (h.vx) TPM_CUDA_TRY(cudaMemcpyAsync(d.vx, h.vx, 4 * n, cudaMemcpyHostToDevice, s));
  else TPM_CUDA_TRY(cudaMemsetAsync(d.vx, 0, 4 * n, s));
  if (h.vy) TPM_CUDA_TRY(cudaMemcpyAsync(d.vy, h.vy, 4 * n, cudaMemcpyHostToDevice, s));
  else TPM_CUDA_TRY(cudaMemsetAsync(d.vy, 0, 4 * n, s));
  if (h.vz) TPM_CUDA_TRY(cudaMemcpyAsync(d.vz, h.vz, 4 * n, cudaMemcpyHostToDevice, s));
  else TPM_CUDA_TRY(cudaMemsetAsync(d.vz, 0, 4 * n, s));
  if (h.rung) TPM_CUDA_TRY(cudaMemcpyAsync(d.rung, h.rung, n, cudaMemcpyHostToDevice, s));
  else TPM_CUDA_TRY(cudaMemsetAsync(d.rung, 0, n, s));
  return TPM_OK;
}

int download(const tpm_host_particles& h, const DevSet& d, int64_t n, cudaStream_t s) {
  if (h.x) TPM_CUDA_TRY(cudaMemcpyAsync(h.x, d.x, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.y) TPM_CUDA_TRY(cudaMemcpyAsync(h.y, d.y, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.z) TPM_CUDA_TRY(cudaMemcpyAsync(h.z, d.z, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.vx) TPM_CUDA_TRY(cudaMemcpyAsync(h.vx, d.vx, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.vy) TPM_CUDA_TRY(cudaMemcpyAsync(h.vy, d.vy, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.vz) TPM_CUDA_TRY(cudaMemcpyAsync(h.vz, d.vz, 4 * n, cudaMemcpyDeviceToHost, s));
  if (h.rung) TPM_CUDA_TRY(cudaMemcpyAsync(h.rung, d.rung, n, cudaMemcpyDeviceToHost, s));
  return TPM_OK;
}

}  // namespace

void stream_destroy(tpm_ctx* c) {
  void* ptrs[] = {c->x3, c->y3, c->z3, c->vx3, c->vy3, c->vz3, c->rung3};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  if (c->down_stream) cudaStreamDestroy(c->down_stream);
  for (int k = 0; k < 3; k++) {
    if (c->ev_up[k]) cudaEventDestroy(c->ev_up[k]);
    if (c->ev_done[k]) cudaEventDestroy(c->ev_done[k]);
    if (c->ev_down[k]) cudaEventDestroy(c->ev_down[k]);
  }
}

}  // namespace tpm

// A CUDA error inside the step loop still restores the context's set bookkeeping.
#define STEP_TRY(call)                                                               \
  do {                                                                               \
    const cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) return finish(tpm::fail(TPM_ERR_CUDA, cudaGetErrorString(e_))); \
  } while (0)

extern "C" int tpm_pme_steps_host(tpm_ctx* c, int64_t nsteps, int64_t n, const tpm_host_particles* in,
                                  const tpm_host_particles* out, int min_rung, double scale, double t0,
                                  int first_call) {
  using namespace tpm;
  if (!c || (nsteps > 0 && (!in || !out))) return fail(TPM_ERR_INVALID, "null argument");
  if (nsteps < 0 || n < 0) return fail(TPM_ERR_INVALID, "negative step or particle count");
  if (n > c->cap) return fail(TPM_ERR_CAPACITY, "n = " + std::to_string(n) + " above capacity " + std::to_string(c->cap));
  for (int64_t s = 0; s < nsteps; s++)
    if (n > 0 && (!in[s].x || !in[s].y || !in[s].z)) return fail(TPM_ERR_INVALID, "positions are required");
  if (nsteps == 0) return TPM_OK;
  int rc = stream_init(c);
  if (rc) return rc;
  DevSet set[3] = {cur_set(c), scratch_set(c), DevSet{c->x3, c->y3, c->z3, c->vx3, c->vy3, c->vz3, c->rung3}};
  int in_i = 0, out_i = 1;
  auto finish = [&](int status) {
    cudaStreamSynchronize(c->up_stream);
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->down_stream);
    // the context keeps the last step's particles current; the set neither
    // current nor scratch becomes the third set again
    const DevSet cur = cur_set(c), scr = scratch_set(c);
    for (int k = 0; k < 3; k++) {
      if (set[k].x != cur.x && set[k].x != scr.x) {
        c->x3 = set[k].x;
        c->y3 = set[k].y;
        c->z3 = set[k].z;
        c->vx3 = set[k].vx;
        c->vy3 = set[k].vy;
        c->vz3 = set[k].vz;
        c->rung3 = set[k].rung;
      }
    }
    return status;
  };
  rc = n > 0 ? upload(set[in_i], in[0], n, c->up_stream) : TPM_OK;
  if (rc) return finish(rc);
  STEP_TRY(cudaEventRecord(c->ev_up[0], c->up_stream));
  for (int64_t s = 0; s < nsteps; s++) {
    const int slot = (int)(s % 3);
    STEP_TRY(cudaStreamWaitEvent(c->stream, c->ev_up[slot], 0));
    bind(c, set[in_i], set[out_i]);
    c->n = n;
    c->sorted = false;
    c->have_phi = false;
    c->host_cells_valid = false;
    if (n > 0) {
      float* g[4] = {c->gx, c->gy, c->gz, c->pot};
      for (float* p : g) STEP_TRY(cudaMemsetAsync(p, 0, 4 * n, c->stream));
    }
    rc = chainmesh_sort(c);  // gathers set in_i into set out_i and makes it current
    if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
    if (rc == TPM_OK) rc = kick_pme(c, nullptr, min_rung, scale, t0, first_call);
    if (rc) return finish(rc);
    STEP_TRY(cudaEventRecord(c->ev_done[slot], c->stream));
    STEP_TRY(cudaStreamWaitEvent(c->down_stream, c->ev_done[slot], 0));
    rc = n > 0 ? download(out[s], set[out_i], n, c->down_stream) : TPM_OK;
    if (rc) return finish(rc);
    STEP_TRY(cudaEventRecord(c->ev_down[slot], c->down_stream));
    if (s + 1 < nsteps) {
      const int nxt = 3 - in_i - out_i;
      // set nxt is where step s-1 sorted to: wait until it has been downloaded
      if (s >= 1) STEP_TRY(cudaStreamWaitEvent(c->up_stream, c->ev_down[(s - 1) % 3], 0));
      rc = n > 0 ? upload(set[nxt], in[s + 1], n, c->up_stream) : TPM_OK;
      if (rc) return finish(rc);
      STEP_TRY(cudaEventRecord(c->ev_up[(s + 1) % 3], c->up_stream));
      out_i = in_i;
      in_i = nxt;
    }
  }
  return finish(TPM_OK);
}
