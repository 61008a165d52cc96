// tpm_api.cu -- the C ABI (include/tpm.h): options, contexts, particle I/O
// and the entry points that stand in for the reference's kick_pme,
// chainmesh_*, gravity_long_* and gravity_short_* functions.
#include "tpm_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace tpm {

static thread_local std::string g_last_error = "no error";

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

void stage_begin(tpm_ctx* c, Stage s) {
  if (!c->stage_timing) return;
  cudaEventRecord(c->ev.beg[s][c->ev.count[s] % kStageSlots], c->stream);
}
void stage_end(tpm_ctx* c, Stage s) {
  if (!c->stage_timing) return;
  cudaEventRecord(c->ev.end[s][c->ev.count[s] % kStageSlots], c->stream);
  c->ev.count[s]++;
}

}  // namespace tpm

using namespace tpm;

namespace {

struct Alloc {
  tpm_ctx* c;
  int status = TPM_OK;
  template <class T>
  void get(T*& p, int64_t count) {
    if (status != TPM_OK) return;
    const size_t bytes = sizeof(T) * (size_t)std::max<int64_t>(count, 1);
    cudaError_t e = cudaMalloc((void**)&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      status = fail(TPM_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
      cudaGetLastError();
      return;
    }
    c->device_bytes += (int64_t)bytes;
  }
};

int64_t plan_bytes(const tpm_options& o, int64_t cap) {
  const int64_t N = o.four_dim, C = o.chain_dim;
  const int64_t ncell = C * C * C;
  int64_t b = 0;
  b += cap * (3 * 4 + 3 * 4 + 1 + 4 * 4);      // particles + forces
  b += cap * (3 * 4 + 3 * 4 + 1);              // permutation targets
  b += cap * 16;                               // pos4
  b += cap * 4 * 5 + 8;                        // key, idx, cellof, prefix, slot
  const int64_t T = kScanTileElems;
  b += 4 * (2 * ((cap + T - 1) / T + (ncell + T - 1) / T) + 64);  // blocksums
  b += 8 * ((std::max(cap, ncell) + T - 1) / T + 1);  // look-back status words
  b += 8 * (ncell + 2);                        // counts + offsets
  b += N * N * N * 4 * 2 + N * N * (int64_t)fft3d_padded_columns((int)N) * 8 + 3 * N * 8;  // rho, phi, rhok, twiddles
  return b;
}

int derive(tpm_ctx* c) {
  const tpm_options& o = c->opt;
  if (o.four_dim < 4 || o.chain_dim < 3)
    return fail(TPM_ERR_INVALID, "need four_dim >= 4 and chain_dim >= 3 (27 distinct neighbour cells)");
  if (o.four_dim > 4096 || o.chain_dim > 2048) return fail(TPM_ERR_INVALID, "mesh too large");
  if (!(o.rs > 0) || !(o.hsoft > 0)) return fail(TPM_ERR_INVALID, "rs and hsoft must be positive");
  if (o.assign < 0 || o.assign > 2) return fail(TPM_ERR_INVALID, "assign must be cloud4, cic or tsc");
  if (o.sort_mode < 0 || o.sort_mode > 1) return fail(TPM_ERR_INVALID, "sort_mode must be parity or fast");
  if (o.fft < 0 || o.fft > 2) return fail(TPM_ERR_INVALID, "fft must be auto, cufft or block");
  if (o.deterministic_deposit < TPM_DEPOSIT_FP32 || o.deterministic_deposit > TPM_DEPOSIT_FIXED32)
    return fail(TPM_ERR_INVALID, "deterministic_deposit must be 0 (fp32), 1 (exact64) or 2 (fixed32)");
  c->N = o.four_dim;
  c->C = o.chain_dim;
  c->rs_box = o.rs;
  c->rcut_box = o.rcut_over_rs > 0 ? o.rcut_over_rs * o.rs : 0.0;
  if (c->rcut_box > 0 && c->rcut_box > 1.0 / c->C * (1.0 + 1e-12))
    return fail(TPM_ERR_INVALID, "cutoff wider than a chain cell: the 27-cell neighbourhood would miss pairs");
  return TPM_OK;
}

bool parse_int(const char* s, int* out) {
  char* end = nullptr;
  long v = strtol(s, &end, 10);
  if (!s[0] || *end) return false;
  *out = (int)v;
  return true;
}
bool parse_double(const char* s, double* out) {
  char* end = nullptr;
  double v = strtod(s, &end);
  if (!s[0] || *end) return false;
  *out = v;
  return true;
}

}  // namespace

extern "C" {

const char* tpm_error_string(int status) {
  switch (status) {
    case TPM_OK: return "ok";
    case TPM_ERR_INVALID: return "invalid argument";
    case TPM_ERR_NOMEM: return "out of memory";
    case TPM_ERR_CUDA: return "CUDA error";
    case TPM_ERR_CUFFT: return "cuFFT error";
    case TPM_ERR_STATE: return "call out of order";
    case TPM_ERR_RUNG: return "rung out of range (clamped)";
    case TPM_ERR_CAPACITY: return "particle count above capacity";
    case TPM_ERR_BUDGET: return "HBM budget exceeded";
    case TPM_ERR_TIMEOUT: return "device wait timed out";
    case TPM_ERR_NOEXT: return "library part not built";
    default: return "unknown status";
  }
}

const char* tpm_last_error_message(void) { return g_last_error.c_str(); }

int tpm_options_init(tpm_options* o, int parts_dim, int parts_o_four, int four_o_chain) {
  if (!o) return fail(TPM_ERR_INVALID, "null options");
  memset(o, 0, sizeof(*o));
  if (parts_dim <= 0 || parts_o_four <= 0 || four_o_chain <= 0)
    return fail(TPM_ERR_INVALID, "sizes must be positive");
  // src/options.cpp:81-96
  o->parts_dim = parts_dim;
  o->parts_o_four = parts_o_four;
  o->four_o_chain = four_o_chain;
  o->parts_o_chain = parts_o_four * four_o_chain;
  if (parts_dim % o->parts_o_chain != 0)
    return fail(TPM_ERR_INVALID, "Parts dim must be a multiple of " + std::to_string(o->parts_o_chain));
  o->four_dim = parts_dim / parts_o_four;
  o->chain_dim = parts_dim / o->parts_o_chain;
  o->rs = 1.0 / o->four_dim;
  o->GM = 1.0;
  o->hsoft = 2.0 / 25.0 / parts_dim;
  o->eta = 0.2 / sqrt(2.0);
  o->hubble = 0.7;
  o->sigma8 = 0.84;
  o->code_to_cm = 7.108e26 * parts_dim / 1024.0 / o->hubble;
  o->omega_m = 0.3;
  o->z0 = 2.0;
  o->box_size = 1.0;
  o->rcut_over_rs = 0.0;
  o->assign = TPM_ASSIGN_CLOUD4;
  o->deconv_order = 0;
  o->sort_mode = TPM_SORT_PARITY;
  o->kahan = 1;
  o->deterministic_deposit = 0;
  o->seed = 1;
  return TPM_OK;
}

int tpm_options_parse(tpm_options* o, int argc, const char* const* argv) {
  if (!o) return fail(TPM_ERR_INVALID, "null options");
  int parts_dim = 130, parts_o_four = 3, four_o_chain = 5;  // src/options.cpp:50-52 defaults
  int four_dim = 0, chain_dim = 0, kahan = 1, sort_mode = 0, assign = 0, det_dep = 0, fft = TPM_FFT_AUTO;
  double rs_cells = 0, rcut = 0, hsoft = 0, box_size = 1;
  unsigned long long seed = 1;
  for (int i = 0; i < argc; i++) {
    const char* a = argv[i];
    if (strncmp(a, "--", 2) != 0) return fail(TPM_ERR_INVALID, std::string("unexpected argument ") + a);
    const char* eq = strchr(a, '=');
    std::string key = eq ? std::string(a + 2, eq - a - 2) : std::string(a + 2);
    std::string val;
    if (eq) val = eq + 1;
    else if (i + 1 < argc) val = argv[++i];
    else return fail(TPM_ERR_INVALID, "missing value for --" + key);
    bool ok = true;
    if (key == "parts_dim") ok = parse_int(val.c_str(), &parts_dim);
    else if (key == "parts_o_four") ok = parse_int(val.c_str(), &parts_o_four);
    else if (key == "four_o_chain") ok = parse_int(val.c_str(), &four_o_chain);
    else if (key == "box_size") ok = parse_double(val.c_str(), &box_size);
    else if (key == "test" || key == "config_file") ok = true;  // accepted, unused by the library
    else if (key == "four_dim") ok = parse_int(val.c_str(), &four_dim);
    else if (key == "chain_dim") ok = parse_int(val.c_str(), &chain_dim);
    else if (key == "rs_cells") ok = parse_double(val.c_str(), &rs_cells);
    else if (key == "rcut_over_rs") ok = parse_double(val.c_str(), &rcut);
    else if (key == "hsoft") ok = parse_double(val.c_str(), &hsoft);
    else if (key == "kahan") ok = parse_int(val.c_str(), &kahan);
    else if (key == "deterministic_deposit") ok = parse_int(val.c_str(), &det_dep);
    else if (key == "seed") seed = strtoull(val.c_str(), nullptr, 10);
    else if (key == "assign") {
      if (val == "cloud4") assign = 0;
      else if (val == "cic") assign = 1;
      else if (val == "tsc") assign = 2;
      else ok = false;
    } else if (key == "sort") {
      if (val == "parity") sort_mode = 0;
      else if (val == "fast") sort_mode = 1;
      else ok = false;
    } else if (key == "fft") {
      if (val == "auto") fft = TPM_FFT_AUTO;
      else if (val == "cufft") fft = TPM_FFT_CUFFT;
      else if (val == "block") fft = TPM_FFT_BLOCK;
      else ok = false;
    } else return fail(TPM_ERR_INVALID, "unknown option --" + key);
    if (!ok) return fail(TPM_ERR_INVALID, "bad value for --" + key + ": " + val);
  }
  // The reference requires parts_dim % (parts_o_four * four_o_chain) == 0;
  // explicit --four_dim / --chain_dim lift that for the benchmark shapes.
  int rc;
  if (four_dim > 0 || chain_dim > 0) {
    rc = tpm_options_init(o, parts_dim, 1, 1);
    if (rc) return rc;
    o->four_dim = four_dim > 0 ? four_dim : parts_dim / parts_o_four;
    o->parts_o_four = parts_o_four;
    o->chain_dim = chain_dim > 0 ? chain_dim : std::max(1, o->four_dim / four_o_chain);
    o->four_o_chain = four_o_chain;
    o->parts_o_chain = parts_o_four * four_o_chain;
    o->rs = 1.0 / o->four_dim;
  } else {
    rc = tpm_options_init(o, parts_dim, parts_o_four, four_o_chain);
    if (rc) return rc;
  }
  if (rs_cells > 0) o->rs = rs_cells / o->four_dim;
  if (hsoft > 0) o->hsoft = hsoft;
  o->box_size = box_size;
  o->rcut_over_rs = rcut;
  o->assign = assign;
  o->sort_mode = sort_mode;
  o->fft = fft;
  o->kahan = kahan;
  o->deterministic_deposit = det_dep;
  o->seed = seed;
  return TPM_OK;
}

int tpm_plan_device_bytes(const tpm_options* opts, int64_t capacity, int64_t* bytes) {
  if (!opts || !bytes || capacity < 0) return fail(TPM_ERR_INVALID, "bad arguments");
  *bytes = plan_bytes(*opts, capacity);
  return TPM_OK;
}

}  // extern "C"

namespace tpm {

// The per-step working set of a context: everything a step writes and no
// later call reads back (forces, packed positions, sort scratch, meshes).
// A served box keeps only its resident set and borrows these for a step.
namespace {
struct ScratchField {
  void** ptr;
  size_t elem;
  int64_t count;
};

std::vector<ScratchField> scratch_fields(tpm_ctx* c) {
  const int64_t cap = std::max<int64_t>(c->cap, 1);
  const int64_t N = c->N, C = c->C, ncell = C * C * C;
  const int64_t nb = (std::max(cap, ncell) + kScanTileElems - 1) / kScanTileElems;
  return {
      {(void**)&c->gx, 4, cap},      {(void**)&c->gy, 4, cap},       {(void**)&c->gz, 4, cap},
      {(void**)&c->pot, 4, cap},     {(void**)&c->pos4, 16, cap},    {(void**)&c->x2, 4, cap},
      {(void**)&c->y2, 4, cap},      {(void**)&c->z2, 4, cap},       {(void**)&c->vx2, 4, cap},
      {(void**)&c->vy2, 4, cap},     {(void**)&c->vz2, 4, cap},      {(void**)&c->rung2, 1, cap},
      {(void**)&c->key, 4, cap},     {(void**)&c->idx, 4, cap},      {(void**)&c->cellof, 4, cap},
      {(void**)&c->prefix, 4, cap + 1}, {(void**)&c->slot, 4, cap},  {(void**)&c->blocksum, 4, 2 * nb + 64},
      {(void**)&c->rho, 4, N * N * N}, {(void**)&c->rhok, 8, N * N * fft3d_padded_columns((int)N)},
      {(void**)&c->phi, 4, N * N * N},
  };
}
constexpr size_t kScratchAlign = 256;
}  // namespace

int64_t ctx_scratch_bytes(tpm_ctx* c) {
  int64_t b = 0;
  for (const ScratchField& f : scratch_fields(c))
    b += (int64_t)((f.elem * f.count + kScratchAlign - 1) / kScratchAlign * kScratchAlign);
  return b;
}

void ctx_bind_scratch(tpm_ctx* c, void* base, cudaStream_t s) {
  unsigned char* p = static_cast<unsigned char*>(base);
  for (const ScratchField& f : scratch_fields(c)) {
    *f.ptr = p;
    p += (f.elem * f.count + kScratchAlign - 1) / kScratchAlign * kScratchAlign;
  }
  c->stream = s;
  if (c->plans) {
    cufftSetStream(c->plan_r2c, s);
    cufftSetStream(c->plan_c2r, s);
  }
}

void ctx_unbind_scratch(tpm_ctx* c, cudaStream_t own) {
  for (const ScratchField& f : scratch_fields(c)) *f.ptr = nullptr;
  c->stream = own;
  if (c->plans) {
    cufftSetStream(c->plan_r2c, own);
    cufftSetStream(c->plan_c2r, own);
  }
}

}  // namespace tpm

extern "C" {

int tpm_ctx_create(const tpm_options* opts, int64_t capacity, tpm_ctx** out) {
  return tpm::ctx_create(opts, capacity, true, out);
}

}  // extern "C"

int tpm::ctx_create(const tpm_options* opts, int64_t capacity, bool with_scratch, tpm_ctx** out) {
  if (!opts || !out) return fail(TPM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (capacity < 0 || capacity > 0x7fffffffLL - 1) return fail(TPM_ERR_INVALID, "capacity out of range");
  tpm_ctx* c = new tpm_ctx();
  c->opt = *opts;
  c->has_scratch = with_scratch;
  int rc = derive(c);
  if (rc) {
    delete c;
    return rc;
  }
  cudaError_t e = cudaGetDevice(&c->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(TPM_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
  }
  for (int s = 0; s < kNumStages; s++) {
    for (int k = 0; k < kStageSlots; k++) {
      cudaEventCreate(&c->ev.beg[s][k]);
      cudaEventCreate(&c->ev.end[s][k]);
    }
    c->ev.count[s] = 0;
  }
  c->cap = capacity;
  const int64_t N = c->N, C = c->C, ncell = C * C * C;
  const int64_t nb = (std::max(capacity, ncell) + kScanTileElems - 1) / kScanTileElems;
  Alloc A{c};
  // resident set: particles, chain-mesh tables, FFT and Green tables
  A.get(c->x, capacity);
  A.get(c->y, capacity);
  A.get(c->z, capacity);
  A.get(c->vx, capacity);
  A.get(c->vy, capacity);
  A.get(c->vz, capacity);
  A.get(c->rung, capacity);
  A.get(c->scan_status, nb + 1);
  A.get(c->cell_count, ncell + 1);
  A.get(c->cell_begin, ncell + 1);
  A.get(c->thr, C + 1);
  A.get(c->tree, C * kMaxTreeDepth);
  A.get(c->depth1d, C);
  A.get(c->fft_tw, 3 * N);
  A.get(c->gtab, 2 * N);
  A.get(c->k2tab, N);
  A.get(c->d_err, 1);
  // per-step working set
  if (with_scratch) {
    for (const auto& f : scratch_fields(c)) {
      if (A.status != TPM_OK) break;
      cudaError_t ea = cudaMalloc(f.ptr, f.elem * (size_t)std::max<int64_t>(f.count, 1));
      if (ea != cudaSuccess) {
        *f.ptr = nullptr;
        cudaGetLastError();
        A.status = fail(TPM_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(ea));
      } else {
        c->device_bytes += (int64_t)(f.elem * (size_t)std::max<int64_t>(f.count, 1));
      }
    }
  }
  if (A.status != TPM_OK) {
    tpm_ctx_destroy(c);
    return A.status;
  }
  e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->scan_status, 0, sizeof(unsigned long long) * (nb + 1));
  if (e == cudaSuccess) e = cudaMemset(c->cell_begin, 0, sizeof(int32_t) * (ncell + 1));
  if (e != cudaSuccess) {
    tpm_ctx_destroy(c);
    return fail(TPM_ERR_CUDA, cudaGetErrorString(e));
  }
  rc = sort_init(c);
  if (rc == TPM_OK) rc = mesh_init(c);
  if (rc != TPM_OK) {
    tpm_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return TPM_OK;
}

extern "C" {

int tpm_ctx_destroy(tpm_ctx* c) {
  if (!c) return TPM_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->x, c->y, c->z, c->vx, c->vy, c->vz, c->rung, c->scan_status, c->cell_count, c->cell_begin,
                  c->thr, c->tree, c->depth1d, c->fft_tw, c->gtab, c->k2tab, c->d_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  void* kq[] = {c->kq.d_args, c->kq.d_cells, c->kq.d_class, c->kq.d_hist, c->kq.d_items, c->kq.d_nitems,
                c->kq.d_counter};
  for (void* p : kq)
    if (p) cudaFree(p);
  // a borrowed working set (served boxes) belongs to its lender
  if (c->has_scratch)
    for (const auto& f : scratch_fields(c))
      if (*f.ptr) cudaFree(*f.ptr);
  if (c->plans) {
    cufftDestroy(c->plan_r2c);
    cufftDestroy(c->plan_c2r);
  }
  for (int s = 0; s < kNumStages; s++) {
    for (int k = 0; k < kStageSlots; k++) {
      if (c->ev.beg[s][k]) cudaEventDestroy(c->ev.beg[s][k]);
      if (c->ev.end[s][k]) cudaEventDestroy(c->ev.end[s][k]);
    }
  }
  stream_destroy(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return TPM_OK;
}

int tpm_ctx_options(const tpm_ctx* c, tpm_options* out) {
  if (!c || !out) return fail(TPM_ERR_INVALID, "null argument");
  *out = c->opt;
  return TPM_OK;
}

int tpm_ctx_device_bytes(const tpm_ctx* c, int64_t* bytes) {
  if (!c || !bytes) return fail(TPM_ERR_INVALID, "null argument");
  *bytes = c->device_bytes;
  return TPM_OK;
}

static int set_common(tpm_ctx* c, int64_t n, cudaMemcpyKind kind, const uint32_t* x, const uint32_t* y,
                      const uint32_t* z, const float* vx, const float* vy, const float* vz, const int8_t* rung) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (n < 0) return fail(TPM_ERR_INVALID, "negative particle count");
  if (n > c->cap) return fail(TPM_ERR_CAPACITY, "n = " + std::to_string(n) + " above capacity " + std::to_string(c->cap));
  if (n > 0 && (!x || !y || !z)) return fail(TPM_ERR_INVALID, "positions are required");
  cudaStream_t s = c->stream;
  c->n = n;
  if (n > 0) {
    TPM_CUDA_TRY(cudaMemcpyAsync(c->x, x, 4 * n, kind, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(c->y, y, 4 * n, kind, s));
    TPM_CUDA_TRY(cudaMemcpyAsync(c->z, z, 4 * n, kind, s));
    if (vx) TPM_CUDA_TRY(cudaMemcpyAsync(c->vx, vx, 4 * n, kind, s));
    else TPM_CUDA_TRY(cudaMemsetAsync(c->vx, 0, 4 * n, s));
    if (vy) TPM_CUDA_TRY(cudaMemcpyAsync(c->vy, vy, 4 * n, kind, s));
    else TPM_CUDA_TRY(cudaMemsetAsync(c->vy, 0, 4 * n, s));
    if (vz) TPM_CUDA_TRY(cudaMemcpyAsync(c->vz, vz, 4 * n, kind, s));
    else TPM_CUDA_TRY(cudaMemsetAsync(c->vz, 0, 4 * n, s));
    if (rung) TPM_CUDA_TRY(cudaMemcpyAsync(c->rung, rung, n, kind, s));
    else TPM_CUDA_TRY(cudaMemsetAsync(c->rung, 0, n, s));
    if (c->gx) {  // a served box has no force arrays between steps
      TPM_CUDA_TRY(cudaMemsetAsync(c->gx, 0, 4 * n, s));
      TPM_CUDA_TRY(cudaMemsetAsync(c->gy, 0, 4 * n, s));
      TPM_CUDA_TRY(cudaMemsetAsync(c->gz, 0, 4 * n, s));
      TPM_CUDA_TRY(cudaMemsetAsync(c->pot, 0, 4 * n, s));
    }
  }
  c->sorted = false;
  c->have_phi = false;
  c->host_cells_valid = false;
  return TPM_OK;
}

int tpm_set_particles(tpm_ctx* c, int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z,
                      const float* vx, const float* vy, const float* vz, const int8_t* rung) {
  return set_common(c, n, cudaMemcpyHostToDevice, x, y, z, vx, vy, vz, rung);
}

int tpm_set_particles_device(tpm_ctx* c, int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z,
                             const float* vx, const float* vy, const float* vz, const int8_t* rung) {
  return set_common(c, n, cudaMemcpyDeviceToDevice, x, y, z, vx, vy, vz, rung);
}

int tpm_get_particles(tpm_ctx* c, uint32_t* x, uint32_t* y, uint32_t* z, float* vx, float* vy, float* vz,
                      int8_t* rung) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  const int64_t n = c->n;
  cudaStream_t s = c->stream;
  if (n > 0) {
    if (x) TPM_CUDA_TRY(cudaMemcpyAsync(x, c->x, 4 * n, cudaMemcpyDeviceToHost, s));
    if (y) TPM_CUDA_TRY(cudaMemcpyAsync(y, c->y, 4 * n, cudaMemcpyDeviceToHost, s));
    if (z) TPM_CUDA_TRY(cudaMemcpyAsync(z, c->z, 4 * n, cudaMemcpyDeviceToHost, s));
    if (vx) TPM_CUDA_TRY(cudaMemcpyAsync(vx, c->vx, 4 * n, cudaMemcpyDeviceToHost, s));
    if (vy) TPM_CUDA_TRY(cudaMemcpyAsync(vy, c->vy, 4 * n, cudaMemcpyDeviceToHost, s));
    if (vz) TPM_CUDA_TRY(cudaMemcpyAsync(vz, c->vz, 4 * n, cudaMemcpyDeviceToHost, s));
    if (rung) TPM_CUDA_TRY(cudaMemcpyAsync(rung, c->rung, n, cudaMemcpyDeviceToHost, s));
  }
  TPM_CUDA_TRY(cudaStreamSynchronize(s));
  return TPM_OK;
}

int tpm_get_forces(tpm_ctx* c, float* gx, float* gy, float* gz, float* pot) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (!c->gx) return fail(TPM_ERR_STATE, "no forces: a served box keeps no working set between steps");
  const int64_t n = c->n;
  cudaStream_t s = c->stream;
  if (n > 0) {
    if (gx) TPM_CUDA_TRY(cudaMemcpyAsync(gx, c->gx, 4 * n, cudaMemcpyDeviceToHost, s));
    if (gy) TPM_CUDA_TRY(cudaMemcpyAsync(gy, c->gy, 4 * n, cudaMemcpyDeviceToHost, s));
    if (gz) TPM_CUDA_TRY(cudaMemcpyAsync(gz, c->gz, 4 * n, cudaMemcpyDeviceToHost, s));
    if (pot) TPM_CUDA_TRY(cudaMemcpyAsync(pot, c->pot, 4 * n, cudaMemcpyDeviceToHost, s));
  }
  TPM_CUDA_TRY(cudaStreamSynchronize(s));
  return TPM_OK;
}

int tpm_get_device_arrays(tpm_ctx* c, tpm_device_arrays* o) {
  if (!c || !o) return fail(TPM_ERR_INVALID, "null argument");
  o->x = c->x;
  o->y = c->y;
  o->z = c->z;
  o->vx = c->vx;
  o->vy = c->vy;
  o->vz = c->vz;
  o->rung = c->rung;
  o->gx = c->gx;
  o->gy = c->gy;
  o->gz = c->gz;
  o->pot = c->pot;
  o->cell_begin = c->cell_begin;
  o->phi = c->phi;
  o->n = c->n;
  return TPM_OK;
}

int tpm_num_particles(const tpm_ctx* c, int64_t* n) {
  if (!c || !n) return fail(TPM_ERR_INVALID, "null argument");
  *n = c->n;
  return TPM_OK;
}

int tpm_chainmesh_create(tpm_ctx* c) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  return chainmesh_sort(c);
}

static int host_cells(tpm_ctx* c) {
  if (!c->sorted) return fail(TPM_ERR_STATE, "chainmesh_get needs chainmesh_create first");
  if (!c->host_cells_valid) {
    const int64_t nc = (int64_t)c->C * c->C * c->C + 1;
    c->host_cells.resize(nc);
    TPM_CUDA_TRY(cudaMemcpyAsync(c->host_cells.data(), c->cell_begin, 4 * nc, cudaMemcpyDeviceToHost, c->stream));
    TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->host_cells_valid = true;
  }
  return TPM_OK;
}

int tpm_chainmesh_get(tpm_ctx* c, const int ijk[3], int32_t* pbegin, int32_t* pend) {
  if (!c || !ijk || !pbegin || !pend) return fail(TPM_ERR_INVALID, "null argument");
  int rc = host_cells(c);
  if (rc) return rc;
  const int C = c->C;
  auto w = [C](int i) { int r = i % C; return r < 0 ? r + C : r; };
  const int64_t key = ((int64_t)w(ijk[2]) * C + w(ijk[1])) * C + w(ijk[0]);
  *pbegin = c->host_cells[key];
  *pend = c->host_cells[key + 1];
  return TPM_OK;
}

int tpm_chainmesh_offsets(tpm_ctx* c, int32_t* offsets) {
  if (!c || !offsets) return fail(TPM_ERR_INVALID, "null argument");
  int rc = host_cells(c);
  if (rc) return rc;
  memcpy(offsets, c->host_cells.data(), 4 * c->host_cells.size());
  return TPM_OK;
}

int tpm_chainmesh_interior_box(const tpm_ctx* c, int box[6]) {
  if (!c || !box) return fail(TPM_ERR_INVALID, "null argument");
  for (int d = 0; d < 3; d++) {
    box[d] = 0;
    box[3 + d] = c->C;
  }
  return TPM_OK;
}

int tpm_gravity_long_compute(tpm_ctx* c, int type) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (type != TPM_GRAVITY_LONG_PM && type != TPM_GRAVITY_LONG_PME) return fail(TPM_ERR_INVALID, "bad gravity_long type");
  return gravity_long(c, type);
}

int tpm_gravity_long_get_phi(tpm_ctx* c, const int box[6], float* out) {
  if (!c || !box || !out) return fail(TPM_ERR_INVALID, "null argument");
  return gravity_long_get_phi(c, box, out);
}

int tpm_gravity_long_set_phi(tpm_ctx* c, const float* phi) {
  if (!c || !phi) return fail(TPM_ERR_INVALID, "null argument");
  return gravity_long_set_phi(c, phi);
}

int tpm_gravity_long_get_phi_box(const tpm_ctx* c, int box[6]) {
  if (!c || !box) return fail(TPM_ERR_INVALID, "null argument");
  // source_box = chain box * four_o_chain padded by PHI_BW (src/gravity_long.cpp:150-156);
  // on one rank the chain box is the whole mesh.
  for (int d = 0; d < 3; d++) {
    box[d] = -kPhiBW;
    box[3 + d] = c->N + kPhiBW;
  }
  return TPM_OK;
}

int tpm_gravity_long_force_at(tpm_ctx* c, int64_t n, const double* pos, float* phi, float* g) {
  if (!c || (n > 0 && (!pos || !phi || !g))) return fail(TPM_ERR_INVALID, "null argument");
  return gravity_long_force_at(c, n, pos, phi, g);
}

int tpm_kick_pme(tpm_ctx* c, const int* box, int min_rung, double scale, double t0, int first_call) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (!(t0 > 0) || !(scale > 0)) return fail(TPM_ERR_INVALID, "t0 and scale must be positive");
  int rc = kick_pme(c, box, min_rung, scale, t0, first_call);
  if (rc) return rc;
  int err = 0;
  TPM_CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (err) {
    TPM_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    if (err & kErrRung) return fail(TPM_ERR_RUNG, "a new rung fell outside [0, 32) and was clamped");
  }
  return TPM_OK;
}

int tpm_drift(tpm_ctx* c, double dt) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  if (!std::isfinite(dt)) return fail(TPM_ERR_INVALID, "dt must be finite");
  int rc = drift(c, dt);
  if (rc) return rc;
  int err = 0;
  TPM_CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (err) {
    TPM_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return fail(TPM_ERR_INVALID, "|v * dt| >= 2^31 box lengths for some particle (left unmoved)");
  }
  return TPM_OK;
}

int tpm_gravity_short_ewald(tpm_ctx* c, int64_t ns, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz,
                            int method, double* phi, double* gx, double* gy, double* gz) {
  if (!c || (ns > 0 && (!sx || !sy || !sz))) return fail(TPM_ERR_INVALID, "null argument");
  if (ns <= 0) return TPM_OK;
  uint32_t* d = nullptr;
  TPM_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(uint32_t) * 3 * ns, c->stream));
  cudaError_t e = cudaMemcpyAsync(d, sx, 4 * ns, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + ns, sy, 4 * ns, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + 2 * ns, sz, 4 * ns, cudaMemcpyHostToDevice, c->stream);
  int rc = e == cudaSuccess ? ewald(c, ns, d, d + ns, d + 2 * ns, method, phi, gx, gy, gz)
                            : fail(TPM_ERR_CUDA, cudaGetErrorString(e));
  cudaFreeAsync(d, c->stream);
  cudaStreamSynchronize(c->stream);
  return rc;
}

int tpm_ewald_fp64(tpm_ctx* c, int64_t ns, const int64_t* sample_idx, int method, double* phi, double* gx,
                   double* gy, double* gz) {
  if (!c || (ns > 0 && !sample_idx)) return fail(TPM_ERR_INVALID, "null argument");
  if (ns <= 0) return TPM_OK;
  std::vector<uint32_t> hx(ns), hy(ns), hz(ns);
  std::vector<uint32_t> all;
  for (int64_t i = 0; i < ns; i++)
    if (sample_idx[i] < 0 || sample_idx[i] >= c->n) return fail(TPM_ERR_INVALID, "sample index out of range");
  // gather on the host from single-element copies (ns is small)
  for (int64_t i = 0; i < ns; i++) {
    TPM_CUDA_TRY(cudaMemcpyAsync(&hx[i], c->x + sample_idx[i], 4, cudaMemcpyDeviceToHost, c->stream));
    TPM_CUDA_TRY(cudaMemcpyAsync(&hy[i], c->y + sample_idx[i], 4, cudaMemcpyDeviceToHost, c->stream));
    TPM_CUDA_TRY(cudaMemcpyAsync(&hz[i], c->z + sample_idx[i], 4, cudaMemcpyDeviceToHost, c->stream));
  }
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return tpm_gravity_short_ewald(c, ns, hx.data(), hy.data(), hz.data(), method, phi, gx, gy, gz);
}

int tpm_get_stage_times(tpm_ctx* c, tpm_stage_times* out) {
  if (!c || !out) return fail(TPM_ERR_INVALID, "null argument");
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  float t[kNumStages] = {0};
  for (int s = 0; s < kNumStages; s++) {
    const int64_t n = std::min<int64_t>(c->ev.count[s], kStageSlots);
    double sum = 0;
    for (int64_t k = 0; k < n; k++) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, c->ev.beg[s][k], c->ev.end[s][k]) != cudaSuccess) {
        sum = -1;
        break;
      }
      sum += ms;
    }
    t[s] = n > 0 && sum >= 0 ? (float)(sum / n) : (n > 0 ? -1.f : 0.f);
  }
  out->sort_ms = t[kStSort];
  out->deposit_ms = t[kStDeposit];
  out->fft_forward_ms = t[kStFftF];
  out->green_ms = t[kStGreen];
  out->fft_inverse_ms = t[kStFftI];
  out->kick_ms = t[kStKick];
  out->drift_ms = t[kStDrift];
  out->ewald_ms = t[kStEwald];
  out->interp_ms = t[kStInterp];
  return TPM_OK;
}

int tpm_reset_stage_times(tpm_ctx* c) {
  if (!c) return fail(TPM_ERR_INVALID, "null argument");
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < kNumStages; s++) c->ev.count[s] = 0;
  return TPM_OK;
}

int tpm_get_launch_count(const tpm_ctx* c, int64_t* count) {
  if (!c || !count) return fail(TPM_ERR_INVALID, "null argument");
  *count = c->launches;
  return TPM_OK;
}

int tpm_synchronize(tpm_ctx* c) {
  if (!c) return fail(TPM_ERR_INVALID, "null context");
  TPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return TPM_OK;
}

}  // extern "C"
