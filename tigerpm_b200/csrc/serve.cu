// serve.cu -- a request loop serving kick + drift steps of many resident
// boxes, admitted by an HBM budget, with concurrent steps overlapping on the
// device.
//
// The reference allocates, stages, kicks and frees per kick_pme call
// (src/kick_pme.cu:390-621), one box at a time, and splits a box when free
// memory is short (:418-430).  A server keeps every admitted box resident
// (particles, chain-mesh tables, FFT twiddles and Green's-function tables:
// about 25 bytes per particle) and lends each running step its working set
// (forces, packed positions, sort scratch, PM meshes) from a stream-ordered
// memory pool.  The device budget covers both:
//
//   resident(all boxes) + working sets of the steps in flight <= budget
//
// A box is admitted only while resident bytes plus the largest working set
// of any box fit (so every box can always run), else TPM_ERR_BUDGET.  A
// request (one kick + drift step of one box) waits in FIFO order until a
// slot (stream) is free and its working set fits in what the steps in
// flight leave; requests of a box already running wait for it, others may
// pass them.  A dispatcher thread admits requests as slots and memory free
// up; each step runs on its slot's stream, so steps of different boxes
// overlap on the GPU.  A host callback marks completion.
#include "tpm_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace tpm {
namespace {

using Clock = std::chrono::steady_clock;

double now_s(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

struct ServeBox {
  tpm_ctx* c = nullptr;
  cudaStream_t own = nullptr;
  int64_t resident = 0;
  int64_t scratch = 0;
  bool busy = false;
};

struct ServeSlot {
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int* err_host = nullptr;  // pinned: the box's error word after the step
  int req = -1;
  void* mem = nullptr;
};

struct ServeReq {
  int box = 0;
  double dt = 0, scale = 1, t0 = 1;
  int min_rung = 0, first_call = 1;
  int status = TPM_OK;
  std::string msg;  // the failing call's message (set on the dispatcher thread)
  double t_submit = 0, t_start = 0, t_done = 0;
  float device_ms = 0;
  bool done = false;
  int slot = -1;
};

}  // namespace
}  // namespace tpm

struct tpm_server {
  int device = 0;
  int64_t budget = 0;
  int64_t resident = 0;
  int64_t inflight = 0;
  int64_t inflight_peak = 0;
  int64_t max_scratch = 0;
  int max_inflight_steps = 0;
  cudaMemPool_t pool = nullptr;
  // deques: growing them (new boxes, new requests) keeps references to
  // existing entries valid while the dispatcher issues a step unlocked
  std::deque<tpm::ServeBox> boxes;
  std::vector<tpm::ServeSlot> slots;
  std::deque<tpm::ServeReq> reqs;
  std::deque<int> pending;
  std::deque<int> completed;  // slots whose step finished (host callbacks)
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  tpm::Clock::time_point t0 = tpm::Clock::now();
  std::atomic<int64_t> launches{0};  // counted by the dispatcher, read by stats
  int64_t steps_done = 0;
  int64_t particles_done = 0;
  int running = 0;
  uint64_t epoch = 0;  // bumped by every submission and completion
};

using namespace tpm;

namespace {

struct CallbackArg {
  tpm_server* srv;
  int slot;
};

void CUDART_CB on_step_done(void* p) {
  CallbackArg* a = static_cast<CallbackArg*>(p);
  tpm_server* s = a->srv;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    const int r = s->slots[a->slot].req;
    if (r >= 0) s->reqs[r].t_done = now_s(s->t0);
    s->completed.push_back(a->slot);
    s->epoch++;
  }
  s->cv.notify_all();
}

// One kick + drift step of box b on slot k (no lock held).  The step is the
// served form of the reference's kick_pme_test sequence (src/test.cpp:182-234)
// followed by the fixed-point drift.
int issue(tpm_server* s, int k, const ServeReq& rq, std::vector<CallbackArg>& cb) {
  ServeSlot& sl = s->slots[k];
  ServeBox& bx = s->boxes[rq.box];
  tpm_ctx* c = bx.c;
  int rc = TPM_OK;
  cudaGetLastError();  // a step reports only its own errors
  cudaError_t e = cudaMallocFromPoolAsync(&sl.mem, (size_t)bx.scratch, s->pool, sl.s);
  if (e != cudaSuccess) {
    sl.mem = nullptr;
    rc = fail(TPM_ERR_NOMEM, std::string("working set: ") + cudaGetErrorString(e));
  } else {
    ctx_bind_scratch(c, sl.mem, sl.s);
    const int64_t l0 = c->launches;
    rc = cudaEventRecord(sl.e0, sl.s) == cudaSuccess ? TPM_OK : fail(TPM_ERR_CUDA, "event record");
    if (rc == TPM_OK) rc = chainmesh_sort(c);
    if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
    if (rc == TPM_OK) rc = kick_pme(c, nullptr, rq.min_rung, rq.scale, rq.t0, rq.first_call);
    if (rc == TPM_OK) rc = drift(c, rq.dt);
    if (rc == TPM_OK) e = cudaMemcpyAsync(sl.err_host, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, sl.s);
    if (e == cudaSuccess && rc == TPM_OK) e = cudaMemsetAsync(c->d_err, 0, sizeof(int), sl.s);
    if (e == cudaSuccess && rc == TPM_OK) e = cudaEventRecord(sl.e1, sl.s);
    if (rc == TPM_OK && e != cudaSuccess) rc = fail(TPM_ERR_CUDA, cudaGetErrorString(e));
    // the working set returns to the pool once the step's kernels are done
    const cudaError_t ef = cudaFreeAsync(sl.mem, sl.s);
    if (rc == TPM_OK && ef != cudaSuccess) rc = fail(TPM_ERR_CUDA, cudaGetErrorString(ef));
    sl.mem = nullptr;
    ctx_unbind_scratch(c, bx.own);
    s->launches += c->launches - l0;
  }
  cb[k] = CallbackArg{s, k};
  // completion is signalled after a failed issue too, so the slot returns
  const cudaError_t eh = cudaLaunchHostFunc(sl.s, on_step_done, &cb[k]);
  if (eh != cudaSuccess) {
    if (rc == TPM_OK) rc = fail(TPM_ERR_CUDA, cudaGetErrorString(eh));
    on_step_done(&cb[k]);
  }
  return rc;
}

void dispatcher(tpm_server* s) {
  std::vector<CallbackArg> cb(s->slots.size());
  std::unique_lock<std::mutex> lock(s->mu);
  while (true) {
    const uint64_t seen = s->epoch;
    // completions
    while (!s->completed.empty()) {
      const int k = s->completed.front();
      s->completed.pop_front();
      ServeSlot& sl = s->slots[k];
      const int r = sl.req;
      if (r < 0) continue;
      ServeReq& rq = s->reqs[r];
      float ms = 0;
      if (rq.status == TPM_OK && cudaEventElapsedTime(&ms, sl.e0, sl.e1) == cudaSuccess) rq.device_ms = ms;
      if (rq.status == TPM_OK && *sl.err_host) {
        rq.status = (*sl.err_host & kErrRung) ? TPM_ERR_RUNG : TPM_ERR_INVALID;
        *sl.err_host = 0;
      }
      ServeBox& bx = s->boxes[rq.box];
      bx.busy = false;
      s->inflight -= bx.scratch;
      s->running--;
      s->steps_done++;
      s->particles_done += bx.c->n;
      rq.done = true;
      sl.req = -1;
    }
    s->cv.notify_all();
    if (s->stop && s->running == 0) break;
    // admissions: FIFO; a request of a busy box is passed over, the first
    // request that does not fit in memory holds the rest back
    std::vector<std::pair<ServeReq, int>> start;  // (request copy, slot)
    std::vector<int> start_ids;
    if (!s->stop) {
      for (auto it = s->pending.begin(); it != s->pending.end();) {
        ServeReq& rq = s->reqs[*it];
        ServeBox& bx = s->boxes[rq.box];
        if (bx.busy) {
          ++it;
          continue;
        }
        int k = -1;
        for (size_t j = 0; j < s->slots.size(); j++)
          if (s->slots[j].req < 0) {
            k = (int)j;
            break;
          }
        if (k < 0) break;
        if (s->inflight + bx.scratch > s->budget - s->resident) break;
        bx.busy = true;
        s->inflight += bx.scratch;
        s->inflight_peak = std::max(s->inflight_peak, s->inflight);
        s->slots[k].req = *it;
        rq.slot = k;
        rq.t_start = now_s(s->t0);
        s->running++;
        s->max_inflight_steps = std::max(s->max_inflight_steps, s->running);
        start.emplace_back(rq, k);
        start_ids.push_back(*it);
        it = s->pending.erase(it);
      }
    }
    if (!start.empty()) {
      lock.unlock();
      for (size_t j = 0; j < start.size(); j++) {
        const int rc = issue(s, start[j].second, start[j].first, cb);
        if (rc != TPM_OK) {
          std::lock_guard<std::mutex> g(s->mu);
          s->reqs[start_ids[j]].status = rc;
          s->reqs[start_ids[j]].msg = tpm_last_error_message();
        }
      }
      lock.lock();
      continue;
    }
    // sleep until a submission, a completion or a stop changes the picture
    s->cv.wait(lock, [s, seen] { return s->epoch != seen || !s->completed.empty() || s->stop; });
  }
}

// Admits a box whose particles `init` writes into its new context.
template <class Init>
int add_box(tpm_server* s, const tpm_options* opts, int64_t n, Init init, int* box_id);

}  // namespace

extern "C" {

int tpm_serve_create(int64_t budget_bytes, int max_slots, tpm_server** out) {
  if (!out) return fail(TPM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (max_slots < 1 || max_slots > 64) return fail(TPM_ERR_INVALID, "max_slots must be in [1, 64]");
  tpm_server* s = new tpm_server();
  auto bail = [&](int rc) {
    tpm_serve_destroy(s);
    return rc;
  };
  TPM_CUDA_TRY(cudaGetDevice(&s->device));
  size_t free_b = 0, total_b = 0;
  TPM_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  s->budget = budget_bytes > 0 ? budget_bytes : (int64_t)(0.8 * (double)free_b);
  if (s->budget > (int64_t)free_b) return bail(fail(TPM_ERR_BUDGET, "budget above the device's free memory"));
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->device;
  cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = (uint64_t)s->budget;  // freed working sets stay reserved for the next steps
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e != cudaSuccess) return bail(fail(TPM_ERR_CUDA, std::string("memory pool: ") + cudaGetErrorString(e)));
  s->slots.resize(max_slots);
  for (ServeSlot& sl : s->slots) {
    e = cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.e0);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.e1);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&sl.err_host, sizeof(int));
    if (e != cudaSuccess) return bail(fail(TPM_ERR_CUDA, std::string("slots: ") + cudaGetErrorString(e)));
    *sl.err_host = 0;
  }
  s->worker = std::thread([s] {
    cudaSetDevice(s->device);
    dispatcher(s);
  });
  *out = s;
  return TPM_OK;
}

int tpm_serve_destroy(tpm_server* s) {
  if (!s) return TPM_OK;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->stop = true;
    }
    s->cv.notify_all();
    s->worker.join();
  }
  for (ServeSlot& sl : s->slots) {
    if (sl.s) cudaStreamSynchronize(sl.s);
    if (sl.e0) cudaEventDestroy(sl.e0);
    if (sl.e1) cudaEventDestroy(sl.e1);
    if (sl.err_host) cudaFreeHost(sl.err_host);
    if (sl.s) cudaStreamDestroy(sl.s);
  }
  for (ServeBox& b : s->boxes)
    if (b.c) tpm_ctx_destroy(b.c);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
  return TPM_OK;
}

// Admits a box: its particles become resident (25 bytes per particle plus
// its tables); returns TPM_ERR_BUDGET when the resident set plus the largest
// working set of any box would exceed the budget.
int tpm_serve_add_box(tpm_server* s, const tpm_options* opts, int64_t n, const uint32_t* x, const uint32_t* y,
                      const uint32_t* z, const float* vx, const float* vy, const float* vz, const int8_t* rung,
                      int* box_id) {
  if (!s || !opts || !box_id) return fail(TPM_ERR_INVALID, "null argument");
  return add_box(s, opts, n, [&](tpm_ctx* c) { return tpm_set_particles(c, n, x, y, z, vx, vy, vz, rung); },
                 box_id);
}

// The same with the box's particles generated on the device
// (tpm_ic_zeldovich) instead of copied from the host.
int tpm_serve_add_box_ic(tpm_server* s, const tpm_options* opts, const tpm_ic_params* ic, int* box_id) {
  if (!s || !opts || !ic || !box_id) return fail(TPM_ERR_INVALID, "null argument");
  const int64_t n = (int64_t)ic->n_side * ic->n_side * ic->n_side;
  return add_box(s, opts, n, [&](tpm_ctx* c) { return tpm_ic_zeldovich(c, ic, nullptr); }, box_id);
}

}  // extern "C"

namespace {

template <class Init>
int add_box(tpm_server* s, const tpm_options* opts, int64_t n, Init init, int* box_id) {
  tpm_ctx* c = nullptr;
  // plan first: resident and working-set bytes without allocating
  {
    tpm_ctx probe;
    probe.opt = *opts;
    probe.cap = n;
    probe.N = opts->four_dim;
    probe.C = opts->chain_dim;
    if (probe.N < 4 || probe.C < 3 || probe.N > 4096 || probe.C > 2048)
      return fail(TPM_ERR_INVALID, "bad mesh sizes");
    int64_t full = 0;
    int rc = tpm_plan_device_bytes(opts, n, &full);
    if (rc) return rc;
    const int64_t scratch = ctx_scratch_bytes(&probe);
    const int64_t resident = std::max<int64_t>(full - scratch, 0);
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->resident + resident + std::max(s->max_scratch, scratch) > s->budget)
      return fail(TPM_ERR_BUDGET, "box of " + std::to_string(n) + " particles does not fit the HBM budget");
  }
  int rc = ctx_create(opts, n, false, &c);
  if (rc) return rc;
  c->stable_buffers = true;
  c->stage_timing = false;
  rc = init(c);
  if (rc == TPM_OK) rc = cudaStreamSynchronize(c->stream) == cudaSuccess ? TPM_OK : fail(TPM_ERR_CUDA, "sync");
  if (rc) {
    tpm_ctx_destroy(c);
    return rc;
  }
  ServeBox b;
  b.c = c;
  b.own = c->stream;
  b.resident = c->device_bytes;
  b.scratch = ctx_scratch_bytes(c);
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->resident + b.resident + std::max(s->max_scratch, b.scratch) > s->budget) {
    tpm_ctx_destroy(c);
    return fail(TPM_ERR_BUDGET, "box of " + std::to_string(n) + " particles does not fit the HBM budget");
  }
  s->resident += b.resident;
  s->max_scratch = std::max(s->max_scratch, b.scratch);
  s->boxes.push_back(b);
  *box_id = (int)s->boxes.size() - 1;
  return TPM_OK;
}

}  // namespace

extern "C" {

// Queues one kick + drift step of a box; returns at once with its id.
int tpm_serve_submit(tpm_server* s, int box, double dt, int min_rung, double scale, double t0, int first_call,
                     int* req_id) {
  if (!s || !req_id) return fail(TPM_ERR_INVALID, "null argument");
  if (!(t0 > 0) || !(scale > 0) || !std::isfinite(dt)) return fail(TPM_ERR_INVALID, "bad step arguments");
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (box < 0 || box >= (int)s->boxes.size()) return fail(TPM_ERR_INVALID, "no such box");
    if (s->boxes[box].scratch > s->budget - s->resident)
      return fail(TPM_ERR_BUDGET, "the box's working set can never fit the budget");
    ServeReq r;
    r.box = box;
    r.dt = dt;
    r.min_rung = min_rung;
    r.scale = scale;
    r.t0 = t0;
    r.first_call = first_call ? 1 : 0;
    r.t_submit = now_s(s->t0);
    s->reqs.push_back(r);
    *req_id = (int)s->reqs.size() - 1;
    s->pending.push_back(*req_id);
    s->epoch++;
  }
  s->cv.notify_all();
  return TPM_OK;
}

int tpm_serve_wait(tpm_server* s, int req, tpm_serve_result* out) {
  if (!s) return fail(TPM_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  if (req < 0 || req >= (int)s->reqs.size()) return fail(TPM_ERR_INVALID, "no such request");
  s->cv.wait(lock, [&] { return s->reqs[req].done; });
  const ServeReq& r = s->reqs[req];
  if (out) {
    out->status = r.status;
    out->box = r.box;
    out->latency_ms = (r.t_done - r.t_submit) * 1e3;
    out->queue_ms = (r.t_start - r.t_submit) * 1e3;
    out->device_ms = r.device_ms;
    out->particles = s->boxes[r.box].c->n;
  }
  return r.status == TPM_OK ? TPM_OK
                            : fail(r.status, "served step " + std::to_string(req) + " failed: " + r.msg);
}

int tpm_serve_drain(tpm_server* s) {
  if (!s) return fail(TPM_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  s->cv.wait(lock, [&] { return s->pending.empty() && s->running == 0; });
  return TPM_OK;
}

// Submits request i at arrival_s[i] seconds after the call starts (host
// clock), then waits for all of them; results[i] per request.
int tpm_serve_replay(tpm_server* s, int nreq, const int* box, const double* arrival_s, double dt, int min_rung,
                     double scale, double t0, int first_call, tpm_serve_result* results) {
  if (!s || (nreq > 0 && (!box || !arrival_s || !results))) return fail(TPM_ERR_INVALID, "null argument");
  std::vector<int> ids(nreq);
  const Clock::time_point start = Clock::now();
  for (int i = 0; i < nreq; i++) {
    std::this_thread::sleep_until(start + std::chrono::duration_cast<Clock::duration>(
                                              std::chrono::duration<double>(std::max(0.0, arrival_s[i]))));
    const int rc = tpm_serve_submit(s, box[i], dt, min_rung, scale, t0, first_call, &ids[i]);
    if (rc) {
      tpm_serve_drain(s);
      return rc;
    }
  }
  int first_bad = TPM_OK;
  for (int i = 0; i < nreq; i++) {
    const int rc = tpm_serve_wait(s, ids[i], &results[i]);
    if (rc && first_bad == TPM_OK) first_bad = rc;
  }
  return first_bad;
}

int tpm_serve_box(tpm_server* s, int box, tpm_ctx** ctx) {
  if (!s || !ctx) return fail(TPM_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  if (box < 0 || box >= (int)s->boxes.size()) return fail(TPM_ERR_INVALID, "no such box");
  if (s->boxes[box].busy) return fail(TPM_ERR_STATE, "the box has a step in flight");
  *ctx = s->boxes[box].c;
  return TPM_OK;
}

int tpm_serve_stats(tpm_server* s, tpm_serve_stats_t* out) {
  if (!s || !out) return fail(TPM_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  out->budget_bytes = s->budget;
  out->resident_bytes = s->resident;
  out->inflight_peak_bytes = s->inflight_peak;
  out->max_working_set_bytes = s->max_scratch;
  out->boxes = (int)s->boxes.size();
  out->max_concurrent_steps = s->max_inflight_steps;
  out->steps_done = s->steps_done;
  out->particles_done = s->particles_done;
  out->launches = s->launches;
  return TPM_OK;
}

}  // extern "C"
