// batch.cu -- an ensemble of independent periodic boxes kicked together.
//
// The reference kicks one box per call: kick_pme stages the box's cells,
// splits the launch by a static contiguous cell partition per block
// (src/kick_pme.cu:139-141) and sizes or splits the box against free memory
// (:418-430).  A batch holds many boxes resident at once (each its own
// tpm_ctx: particles, chain mesh, PM mesh and FFT tables, all with fixed
// device addresses) and runs one step of all of them as:
//
//   fork    every box on its own stream: (restore its input particles),
//           chain-mesh sort, deposit and the FFT Poisson solve; the boxes'
//           kernels overlap on the device
//   join    the main stream waits for all boxes
//   queue   every non-empty (box, chain cell) becomes a work item, bucketed
//           by the binary order of magnitude of its cost (sinks x
//           neighbourhood sources), heaviest bucket first
//   interp  long-range interpolation of every item, one launch
//   kick    ONE persistent launch: resident blocks take items from a global
//           counter until the queue is empty (PP sum + rung kick)
//
// With TPM_BATCH_GRAPH the whole step is captured once as a CUDA graph (the
// fork becomes parallel branches) and replayed; a new capture is made when
// the step's scalars change.  The kick's launch shape (warps per block,
// staged sources, sinks per pass) is picked by tpm_batch_autotune, which
// times candidate shapes on the batch itself and remembers the winner for
// the batch's mean chain-cell occupancy.
#include "tpm_internal.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace tpm {
namespace {

struct InputSet {
  uint32_t *x = nullptr, *y = nullptr, *z = nullptr;
  float *vx = nullptr, *vy = nullptr, *vz = nullptr;
  int8_t* rung = nullptr;
  int64_t n = 0;
};

// Autotuned shapes, per (mean occupancy rounded, wrap).
std::mutex g_shape_mutex;
std::map<std::pair<int, int>, KickShape> g_shapes;

std::pair<int, int> shape_key(double mean_cell, bool wrap) {
  return {(int)std::lround(mean_cell), wrap ? 1 : 0};
}

}  // namespace
}  // namespace tpm

struct tpm_batch {
  int nbox = 0;
  std::vector<tpm_ctx*> box;
  std::vector<tpm::InputSet> input;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  cudaEvent_t ev_t[5] = {};  // begin, long range joined, queue built, interp done, kick done
  tpm::BatchQueue q;
  tpm::KickShape shape{};
  bool wrap = false;
  bool tuned = false;
  double mean_cell = 0;
  int64_t particles = 0;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool graph_ready = false;
  int g_flags = -1, g_min_rung = 0, g_first = 0;
  double g_scale = 0, g_t0 = 0;
  tpm::KickShape g_shape{};
  int64_t graph_kernels = 0;
  int64_t launches = 0;
  bool timed = false;
};

using namespace tpm;

namespace {

void free_input(InputSet& s) {
  void* p[] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.rung};
  for (void* q : p)
    if (q) cudaFree(q);
  s = InputSet{};
}

void drop_graph(tpm_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_ready = false;
}

int restore(tpm_batch* b, int i) {
  tpm_ctx* c = b->box[i];
  const InputSet& in = b->input[i];
  const int64_t n = in.n;
  cudaStream_t s = c->stream;
  c->n = n;
  c->sorted = false;
  c->have_phi = false;
  c->host_cells_valid = false;
  if (n == 0) return TPM_OK;
  TPM_CUDA_TRY(cudaMemcpyAsync(c->x, in.x, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->y, in.y, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->z, in.z, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->vx, in.vx, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->vy, in.vy, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->vz, in.vz, 4 * n, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA_TRY(cudaMemcpyAsync(c->rung, in.rung, n, cudaMemcpyDeviceToDevice, s));
  return TPM_OK;
}

// Phase timing events: under stream capture they must be external records
// (graph nodes that record on every replay); outside it, plain records.
void record(tpm_batch* b, int k) {
  if (!b->timed) return;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(b->stream, &st);
  if (st == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(b->ev_t[k], b->stream, cudaEventRecordExternal);
  else cudaEventRecord(b->ev_t[k], b->stream);
}

// One whole batch step on b->stream (also used under stream capture).
int issue_step(tpm_batch* b, int flags, int min_rung, double scale, double t0, int first_call) {
  record(b, 0);
  TPM_CUDA_TRY(cudaEventRecord(b->ev_fork, b->stream));
  for (int i = 0; i < b->nbox; i++) {
    tpm_ctx* c = b->box[i];
    TPM_CUDA_TRY(cudaStreamWaitEvent(c->stream, b->ev_fork, 0));
    int rc = TPM_OK;
    if (flags & TPM_BATCH_RESTORE) rc = restore(b, i);
    if (rc == TPM_OK) rc = chainmesh_sort(c);
    if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
    if (rc) return rc;
    TPM_CUDA_TRY(cudaEventRecord(b->ev_join[i], c->stream));
    TPM_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ev_join[i], 0));
  }
  record(b, 1);
  int rc = kick_batch_queue(b->q, b->shape.npass, b->stream);
  if (rc) return rc;
  record(b, 2);
  rc = kick_batch_interp(b->q, min_rung, b->shape.npass, b->stream);
  if (rc) return rc;
  record(b, 3);
  rc = kick_batch_kick(b->q, b->shape, b->wrap, min_rung, scale, t0, first_call, b->stream, nullptr);
  if (rc) return rc;
  record(b, 4);
  return TPM_OK;
}

int64_t count_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return -1;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return -1;
  int64_t k = 0;
  for (size_t i = 0; i < n; i++) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
  }
  return k;
}

int64_t box_launches(const tpm_batch* b) {
  int64_t s = 0;
  for (tpm_ctx* c : b->box) s += c->launches;
  return s;
}

bool same_shape(const KickShape& a, const KickShape& b) {
  return a.warps == b.warps && a.stage == b.stage && a.npass == b.npass;
}

}  // namespace

extern "C" {

int tpm_batch_create(int nbox, const tpm_options* opts, const int64_t* capacity, tpm_batch** out) {
  if (!out) return fail(TPM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (nbox <= 0 || !opts || !capacity) return fail(TPM_ERR_INVALID, "a batch needs nbox > 0, options and capacities");
  tpm_batch* b = new tpm_batch();
  b->nbox = nbox;
  b->box.assign(nbox, nullptr);
  b->input.assign(nbox, InputSet{});
  b->ev_join.assign(nbox, nullptr);
  auto bail = [&](int rc) {
    tpm_batch_destroy(b);
    return rc;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  for (int k = 0; k < 5 && e == cudaSuccess; k++) e = cudaEventCreate(&b->ev_t[k]);
  for (int i = 0; i < nbox && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming);
  if (e != cudaSuccess) return bail(fail(TPM_ERR_CUDA, std::string("batch streams: ") + cudaGetErrorString(e)));
  bool wrap = false;
  double cells = 0, parts = 0;
  for (int i = 0; i < nbox; i++) {
    int rc = tpm_ctx_create(&opts[i], capacity[i], &b->box[i]);
    if (rc) return bail(rc);
    tpm_ctx* c = b->box[i];
    c->stable_buffers = true;
    c->stage_timing = false;
    wrap = wrap || c->C == 3;
    cells += (double)c->C * c->C * c->C;
    parts += (double)capacity[i];
    InputSet& in = b->input[i];
    const int64_t cap = std::max<int64_t>(capacity[i], 1);
    void** p[] = {(void**)&in.x, (void**)&in.y, (void**)&in.z, (void**)&in.vx, (void**)&in.vy, (void**)&in.vz};
    for (void** q : p) {
      e = cudaMalloc(q, 4 * cap);
      if (e != cudaSuccess) break;
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&in.rung, cap);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(TPM_ERR_NOMEM, std::string("batch inputs: ") + cudaGetErrorString(e)));
    }
  }
  b->wrap = wrap;
  b->mean_cell = cells > 0 ? parts / cells : 0;
  // per-box kernel arguments and cell tables (device addresses are fixed)
  std::vector<unsigned char> h_args(kick_batch_args_bytes() * nbox), h_cells(kick_batch_cells_bytes() * nbox);
  int rc = kick_batch_write_tables(b->box.data(), nbox, h_args.data(), h_cells.data(), &b->q.total_cells,
                                   &b->q.max_items);
  if (rc) return bail(rc);
  b->q.nbox = nbox;
  const int64_t T = std::max<int64_t>(b->q.total_cells, 1);
  e = cudaMalloc(&b->q.d_args, h_args.size());
  if (e == cudaSuccess) e = cudaMalloc(&b->q.d_cells, h_cells.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->q.d_class, sizeof(int) * T);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->q.d_hist, sizeof(int) * 128);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->q.d_items, sizeof(int4) * std::max<int64_t>(b->q.max_items, 1));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->q.d_nitems, sizeof(int) * 2);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->q.d_counter, sizeof(int) * 2);
  if (e == cudaSuccess) e = cudaMemcpy(b->q.d_args, h_args.data(), h_args.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->q.d_cells, h_cells.data(), h_cells.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->q.d_nitems, 0, sizeof(int) * 2);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(TPM_ERR_NOMEM, std::string("batch queue: ") + cudaGetErrorString(e)));
  }
  {
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    auto it = g_shapes.find(shape_key(b->mean_cell, wrap));
    b->shape = it != g_shapes.end() ? it->second : kick_default_shape(b->mean_cell);
    b->tuned = it != g_shapes.end();
  }
  *out = b;
  return TPM_OK;
}

int tpm_batch_destroy(tpm_batch* b) {
  if (!b) return TPM_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (tpm_ctx* c : b->box)
    if (c) tpm_ctx_destroy(c);
  for (InputSet& s : b->input) free_input(s);
  void* p[] = {b->q.d_args, b->q.d_cells, b->q.d_class, b->q.d_hist, b->q.d_items, b->q.d_nitems, b->q.d_counter};
  for (void* q : p)
    if (q) cudaFree(q);
  for (cudaEvent_t e : b->ev_join)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_t)
    if (e) cudaEventDestroy(e);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return TPM_OK;
}

int tpm_batch_size(const tpm_batch* b, int* nbox, int64_t* particles) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  if (nbox) *nbox = b->nbox;
  if (particles) {
    int64_t s = 0;
    for (const InputSet& in : b->input) s += in.n;
    *particles = s;
  }
  return TPM_OK;
}

int tpm_batch_box(tpm_batch* b, int i, tpm_ctx** ctx) {
  if (!b || !ctx) return fail(TPM_ERR_INVALID, "null argument");
  if (i < 0 || i >= b->nbox) return fail(TPM_ERR_INVALID, "box index out of range");
  *ctx = b->box[i];
  return TPM_OK;
}

int tpm_batch_set_input(tpm_batch* b, int i, int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z,
                        const float* vx, const float* vy, const float* vz, const int8_t* rung) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  if (i < 0 || i >= b->nbox) return fail(TPM_ERR_INVALID, "box index out of range");
  tpm_ctx* c = b->box[i];
  int rc = tpm_set_particles(c, n, x, y, z, vx, vy, vz, rung);
  if (rc) return rc;
  InputSet& in = b->input[i];
  in.n = n;
  if (n > 0) {
    cudaStream_t s = c->stream;
    TPM_CUDA_TRY(cudaMemcpyAsync(in.x, c->x, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.y, c->y, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.z, c->z, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.vx, c->vx, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.vy, c->vy, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.vz, c->vz, 4 * n, cudaMemcpyDeviceToDevice, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(in.rung, c->rung, n, cudaMemcpyDeviceToDevice, s));
  }
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return TPM_OK;
}

int tpm_batch_step(tpm_batch* b, int flags, int min_rung, double scale, double t0, int first_call) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  if (!(t0 > 0) || !(scale > 0)) return fail(TPM_ERR_INVALID, "t0 and scale must be positive");
  if (flags & ~(TPM_BATCH_RESTORE | TPM_BATCH_GRAPH)) return fail(TPM_ERR_INVALID, "unknown batch step flags");
  b->timed = true;
  if (!(flags & TPM_BATCH_GRAPH)) {
    const int64_t l0 = box_launches(b);
    const int rc = issue_step(b, flags, min_rung, scale, t0, first_call);
    b->launches += box_launches(b) - l0 + 5;  // + queue (3), interp, kick
    return rc;
  }
  const bool same = b->graph_ready && b->g_flags == flags && b->g_min_rung == min_rung && b->g_scale == scale &&
                    b->g_t0 == t0 && b->g_first == first_call && same_shape(b->g_shape, b->shape);
  if (!same) {
    drop_graph(b);
    TPM_CUDA_TRY(cudaStreamSynchronize(b->stream));
    TPM_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    const int rc = issue_step(b, flags, min_rung, scale, t0, first_call);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(TPM_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    b->graph = g;
    TPM_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_kernels = count_kernel_nodes(b->graph);
    b->graph_ready = true;
    b->g_flags = flags;
    b->g_min_rung = min_rung;
    b->g_scale = scale;
    b->g_t0 = t0;
    b->g_first = first_call;
    b->g_shape = b->shape;
  }
  TPM_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
  b->launches += b->graph_kernels;
  for (tpm_ctx* c : b->box) {
    c->sorted = true;
    c->have_phi = true;
    c->host_cells_valid = false;
  }
  return TPM_OK;
}

// The same boxes, each through the plain single-box path (restore, sort,
// long-range solve, per-cell kick launch), one box after another on the
// device: the baseline a batch replaces.
int tpm_batch_steps_sequential(tpm_batch* b, int restore_inputs, int min_rung, double scale, double t0,
                               int first_call) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  b->timed = false;
  TPM_CUDA_TRY(cudaEventRecord(b->ev_fork, b->stream));
  cudaEvent_t prev = b->ev_fork;
  for (int i = 0; i < b->nbox; i++) {
    tpm_ctx* c = b->box[i];
    TPM_CUDA_TRY(cudaStreamWaitEvent(c->stream, prev, 0));
    int rc = restore_inputs ? restore(b, i) : TPM_OK;
    if (rc == TPM_OK) rc = chainmesh_sort(c);
    if (rc == TPM_OK) rc = gravity_long(c, TPM_GRAVITY_LONG_PME);
    if (rc == TPM_OK) rc = kick_pme(c, nullptr, min_rung, scale, t0, first_call);
    if (rc) return rc;
    TPM_CUDA_TRY(cudaEventRecord(b->ev_join[i], c->stream));
    prev = b->ev_join[i];
  }
  TPM_CUDA_TRY(cudaStreamWaitEvent(b->stream, prev, 0));
  return TPM_OK;
}

int tpm_batch_synchronize(tpm_batch* b) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  TPM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (tpm_ctx* c : b->box) TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return TPM_OK;
}

int tpm_batch_stream(tpm_batch* b, void** stream) {
  if (!b || !stream) return fail(TPM_ERR_INVALID, "null argument");
  *stream = b->stream;
  return TPM_OK;
}

int tpm_batch_launch_count(const tpm_batch* b, int64_t* count) {
  if (!b || !count) return fail(TPM_ERR_INVALID, "null argument");
  *count = b->launches;
  return TPM_OK;
}

int tpm_batch_phase_times(tpm_batch* b, tpm_batch_times* out) {
  if (!b || !out) return fail(TPM_ERR_INVALID, "null argument");
  TPM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  float ms[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; k++) TPM_CUDA_TRY(cudaEventElapsedTime(&ms[k], b->ev_t[k], b->ev_t[k + 1]));
  out->long_range_ms = ms[0];
  out->queue_ms = ms[1];
  out->interp_ms = ms[2];
  out->kick_ms = ms[3];
  return TPM_OK;
}

int tpm_batch_get_shape(const tpm_batch* b, tpm_kick_shape* s) {
  if (!b || !s) return fail(TPM_ERR_INVALID, "null argument");
  s->warps = b->shape.warps;
  s->stage = b->shape.stage;
  s->npass = b->shape.npass;
  s->tuned = b->tuned ? 1 : 0;
  return TPM_OK;
}

int tpm_batch_set_shape(tpm_batch* b, const tpm_kick_shape* s) {
  if (!b || !s) return fail(TPM_ERR_INVALID, "null argument");
  const KickShape k{s->warps, s->stage, s->npass};
  if (!kick_shape_valid(k)) return fail(TPM_ERR_INVALID, "invalid kick shape");
  b->shape = k;
  return TPM_OK;
}

// Times every candidate kick shape on the batch's current state (after a
// step: particles sorted, potential solved) and keeps the fastest.  Each
// trial restores the velocities and rungs, reruns the interpolation and
// times the kick; on return velocities and rungs are as before the call.
int tpm_batch_autotune(tpm_batch* b, int min_rung, int repeats, tpm_kick_shape* best_out) {
  if (!b) return fail(TPM_ERR_INVALID, "null batch");
  for (tpm_ctx* c : b->box)
    if (!c->sorted || !c->have_phi) return fail(TPM_ERR_STATE, "autotune needs a completed batch step first");
  repeats = std::max(1, repeats);
  TPM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  cudaStream_t s = b->stream;
  // the sort's scratch set holds a copy of the sorted particles after a
  // stable-buffer sort; velocities and rungs are saved there
  auto save = [&](bool back) -> int {
    for (tpm_ctx* c : b->box) {
      const int64_t n = c->n;
      if (n == 0) continue;
      float* v[3] = {c->vx, c->vy, c->vz};
      float* v2[3] = {c->vx2, c->vy2, c->vz2};
      for (int d = 0; d < 3; d++)
        TPM_CUDA_TRY(cudaMemcpyAsync(back ? v[d] : v2[d], back ? v2[d] : v[d], 4 * n, cudaMemcpyDeviceToDevice, s));
      TPM_CUDA_TRY(cudaMemcpyAsync(back ? c->rung : c->rung2, back ? c->rung2 : c->rung, n,
                                   cudaMemcpyDeviceToDevice, s));
    }
    return TPM_OK;
  };
  int rc = save(false);
  if (rc) return rc;
  rc = TPM_OK;  // the queue depends on the pass size: built per candidate
  if (rc) return rc;
  std::vector<KickShape> cand;
  const double m = std::max(b->mean_cell, 1.0);
  int p2 = 8;
  while (p2 < 256 && p2 < m) p2 *= 2;
  for (int w : {2, 4, 8})
    for (double f : {0.5, 1.0})
      for (int np : {p2, std::min(256, 2 * p2)}) {
        int st = (int)std::min(4096.0, std::max(512.0, f * 27.0 * m));
        st = (st + 127) / 128 * 128;
        const KickShape k{w, st, np};
        bool dup = false;
        for (const KickShape& c2 : cand) dup = dup || same_shape(c2, k);
        if (!dup && kick_shape_valid(k)) cand.push_back(k);
      }
  cudaEvent_t e0, e1;
  TPM_CUDA_TRY(cudaEventCreate(&e0));
  TPM_CUDA_TRY(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  KickShape best = b->shape;
  for (const KickShape& k : cand) {
    float tot = 0;
    for (int r = 0; r < repeats && rc == TPM_OK; r++) {
      rc = save(true);
      if (rc == TPM_OK) rc = kick_batch_queue(b->q, k.npass, s);
      if (rc == TPM_OK) rc = kick_batch_interp(b->q, min_rung, k.npass, s);
      if (rc == TPM_OK && cudaEventRecord(e0, s) != cudaSuccess) rc = fail(TPM_ERR_CUDA, "event");
      if (rc == TPM_OK) rc = kick_batch_kick(b->q, k, b->wrap, min_rung, 1.0, 1.0, 1, s, nullptr);
      if (rc == TPM_OK && cudaEventRecord(e1, s) != cudaSuccess) rc = fail(TPM_ERR_CUDA, "event");
      float ms = 0;
      if (rc == TPM_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = fail(TPM_ERR_CUDA, "autotune timing");
      tot += ms;
    }
    if (rc) break;
    if (tot / repeats < best_ms) {
      best_ms = tot / repeats;
      best = k;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int rc2 = save(true);
  if (rc) return rc;
  if (rc2) return rc2;
  TPM_CUDA_TRY(cudaStreamSynchronize(s));
  b->shape = best;
  b->tuned = true;
  {
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    g_shapes[shape_key(b->mean_cell, b->wrap)] = best;
  }
  if (best_out) {
    best_out->warps = best.warps;
    best_out->stage = best.stage;
    best_out->npass = best.npass;
    best_out->tuned = 1;
    best_out->ms = best_ms;
  }
  return TPM_OK;
}

}  // extern "C"
