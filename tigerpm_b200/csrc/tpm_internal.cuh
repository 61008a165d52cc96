// tpm_internal.cuh -- context layout and shared device helpers.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tpm.h"

namespace tpm {

constexpr int kMaxRung = 32;      // MAX_RUNG, tigerpm/tigerpm.hpp:34
constexpr int kNInterp = 6;       // NINTERP, tigerpm/tigerpm.hpp:35
constexpr int kPhiBW = 3;         // PHI_BW, tigerpm/tigerpm.hpp:41
// Elements per tile of the sort's scans: sizes the per-tile block sums and
// look-back status words allocated with the context (chainmesh.cu checks
// that its scan kernels use the same tile).
constexpr int kScanTileElems = 4096;
constexpr int kMaxTreeDepth = 24; // 1-D bisection depth bound (C < 2^23)
constexpr int kDepositFracBits = 40;

// Error bits a kernel may raise in ctx->d_err (never a trap).
constexpr int kErrRung = 1;
constexpr int kErrBounds = 2;
constexpr int kErrTimeout = 4;

// Records a failure message for tpm_last_error_message and returns status.
int fail(int status, const std::string& msg);
#define TPM_CUDA_TRY(call)                                                       \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return ::tpm::fail(TPM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define TPM_CUFFT_TRY(call)                                                      \
  do {                                                                           \
    cufftResult r_ = (call);                                                     \
    if (r_ != CUFFT_SUCCESS)                                                     \
      return ::tpm::fail(TPM_ERR_CUFFT, std::string(#call) + " failed: " + std::to_string((int)r_)); \
  } while (0)

// One node of the 1-D bisection tree over [0, C) that the reference's chain
// sort applies per dimension (split at lo + span/2, src/chainmesh.cpp:198).
struct TreeNode {
  int lo, mid, hi, pad;
};

// Per-stage CUDA event pairs, a ring of kStageSlots launches per stage, so
// that the average over many steps can be read after they ran.
constexpr int kStageSlots = 64;
enum Stage { kStSort = 0, kStDeposit, kStFftF, kStGreen, kStFftI, kStKick, kStDrift, kStEwald, kStInterp,
             kNumStages };
struct StageEvents {
  cudaEvent_t beg[kNumStages][kStageSlots];
  cudaEvent_t end[kNumStages][kStageSlots];
  int64_t count[kNumStages];  // records since the last reset
};

// Work queue of a persistent kick over one or many boxes (device arrays).
struct BatchQueue {
  int nbox = 0;
  int64_t total_cells = 0;   // sum of the boxes' chain cells
  int64_t max_items = 0;     // capacity of d_items
  void* d_args = nullptr;    // per-box kernel arguments (kick_batch_args_bytes each)
  void* d_cells = nullptr;   // per-box cell tables (kick_batch_cells_bytes each)
  int* d_class = nullptr;    // cost class | items << 6 of every (box, cell), total_cells
  int* d_hist = nullptr;     // 2 x 64 ints
  int4* d_items = nullptr;   // (box, cell key, first pass, end pass), heaviest first
  int* d_nitems = nullptr;   // items in use
  int* d_counter = nullptr;  // persistent-kernel work counter
};

}  // namespace tpm

struct tpm_ctx {
  tpm_options opt;
  int N = 0;  // four_dim
  int C = 0;  // chain_dim
  double rs_box = 0;
  double rcut_box = 0;  // 0: none
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t cap = 0;
  int64_t n = 0;
  bool sorted = false;
  bool have_phi = false;
  bool host_cells_valid = false;

  // particles, current order
  uint32_t *x = nullptr, *y = nullptr, *z = nullptr;
  float *vx = nullptr, *vy = nullptr, *vz = nullptr;
  int8_t* rung = nullptr;
  float *gx = nullptr, *gy = nullptr, *gz = nullptr, *pot = nullptr;
  int4* pos4 = nullptr;  // packed (x, y, z, 0) in chain order for PP staging

  // sort scratch
  uint32_t *x2 = nullptr, *y2 = nullptr, *z2 = nullptr;
  float *vx2 = nullptr, *vy2 = nullptr, *vz2 = nullptr;
  int8_t* rung2 = nullptr;
  uint32_t* key = nullptr;    // cell key of the particle at each position
  int32_t* idx = nullptr;     // original index of the particle at each position
  int32_t* cellof = nullptr;  // final cell whose range holds each position
  int32_t* prefix = nullptr;  // exclusive scan of the per-level flags (n + 1)
  int32_t* slot = nullptr;    // partner positions of right-misplaced elements
  int32_t* blocksum = nullptr;
  unsigned long long* scan_status = nullptr;  // look-back words, one per scan tile
  int32_t* cell_count = nullptr;
  int32_t* cell_begin = nullptr;  // C^3 + 1
  uint32_t* thr = nullptr;        // per-dim split thresholds, C + 1
  tpm::TreeNode* tree = nullptr;  // [C * kMaxTreeDepth]
  int* depth1d = nullptr;         // [C]
  int max_depth1d = 0;
  uint64_t scan_stamp = 0;  // distinguishes look-back status words of successive scans

  // mesh
  float* rho = nullptr;  // N^3 real grid (deposit out, r2c in)
  cufftComplex* rhok = nullptr;  // N x N x Sz spectrum (Sz = N/2+1 rounded up to 8)
  float2* fft_tw = nullptr;       // 3N twiddles of the library's own transforms (fft3d_init)
  bool use_fft3d = false;         // library transforms instead of cuFFT
  float* phi = nullptr;  // N^3
  float* gtab = nullptr;   // exp(-k^2 rs^2) sinc(k/2)^-p per index, N
  float* k2tab = nullptr;  // k^2 per index, N
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  bool plans = false;

  // ewald scratch
  double* ew_buf = nullptr;
  int64_t ew_cap = 0;

  // served stream (stream.cu): a third particle set, copy streams and event rings
  uint32_t *x3 = nullptr, *y3 = nullptr, *z3 = nullptr;
  float *vx3 = nullptr, *vy3 = nullptr, *vz3 = nullptr;
  int8_t* rung3 = nullptr;
  cudaStream_t up_stream = nullptr, down_stream = nullptr;
  cudaEvent_t ev_up[3] = {}, ev_done[3] = {}, ev_down[3] = {};
  bool pipe_ready = false;

  // Batch members: the sort copies its result back into x..rung instead of
  // swapping buffers, so device addresses stay fixed across steps (captured
  // CUDA graphs and per-box kernel-argument tables keep them); stage events
  // are skipped (a batch times its own phases).
  bool stable_buffers = false;
  bool stage_timing = true;
  // false: the per-step working set (forces, pos4, sort scratch, meshes) is
  // not owned; a server binds one for each step (ctx_bind_scratch)
  bool has_scratch = true;
  // pot holds every particle's potential in the current order (a kick of
  // the whole box with min_rung 0 since the last sort)
  bool pot_valid = false;
  // the single-box kick's work queue (allocated on the first kick) and the
  // host copies of its one-box argument and cell tables
  tpm::BatchQueue kq;
  alignas(16) unsigned char kq_host_args[256];
  alignas(16) unsigned char kq_host_cells[64];
  // big-step integrator state (integrate.cu): ticks of t0 / 2^31
  double int_t0 = 0, int_scale = 1;
  int64_t int_tick = 0;
  bool int_active = false;

  int* d_err = nullptr;
  int64_t launches = 0;
  int64_t device_bytes = 0;
  tpm::StageEvents ev{};
  std::vector<int32_t> host_cells;
};

namespace tpm {

// Stage timing helpers.
void stage_begin(tpm_ctx* c, Stage s);
void stage_end(tpm_ctx* c, Stage s);

// Launch shape of the kick kernel: warps per block, sources staged per
// chunk, sinks per pass.
struct KickShape {
  int warps, stage, npass;
};
KickShape kick_default_shape(double mean_cell);
bool kick_shape_valid(const KickShape& k);

// Work queue of a batched kick over many boxes (device arrays).
size_t kick_batch_args_bytes();
size_t kick_batch_cells_bytes();
int kick_batch_write_tables(tpm_ctx* const* boxes, int nbox, void* h_args, void* h_cells, int64_t* total_cells,
                            int64_t* max_items);
int kick_batch_queue(const BatchQueue& q, int npass, cudaStream_t s);
int kick_batch_interp(const BatchQueue& q, int min_rung, int npass, cudaStream_t s);
int kick_batch_kick(const BatchQueue& q, const KickShape& k, bool wrap, int min_rung, double scale, double t0,
                    int first_call, cudaStream_t s, int* blocks_out);

// Contexts with or without their per-step working set; the set's size and
// binding (the lender keeps the memory; own = the stream to return to).
int ctx_create(const tpm_options* opts, int64_t capacity, bool with_scratch, tpm_ctx** out);
int64_t ctx_scratch_bytes(tpm_ctx* c);
void ctx_bind_scratch(tpm_ctx* c, void* base, cudaStream_t s);
void ctx_unbind_scratch(tpm_ctx* c, cudaStream_t own);

// Kernel families (each returns TPM_OK or an error).
int chainmesh_sort(tpm_ctx* c);
int gravity_long(tpm_ctx* c, int type);
int gravity_long_get_phi(tpm_ctx* c, const int box[6], float* out);
int gravity_long_set_phi(tpm_ctx* c, const float* phi);
int gravity_long_force_at(tpm_ctx* c, int64_t n, const double* pos, float* phi, float* g);
int kick_pme(tpm_ctx* c, const int box[6], int min_rung, double scale, double t0, int first_call);
int drift(tpm_ctx* c, double dt);
int ewald(tpm_ctx* c, int64_t ns, const uint32_t* dsx, const uint32_t* dsy, const uint32_t* dsz,
          int method, double* phi, double* gx, double* gy, double* gz);
int mesh_init(tpm_ctx* c);
int fft3d_padded_columns(int N);
bool fft3d_supported(int N);
int fft3d_init(tpm_ctx* c);
int fft3d_poisson(tpm_ctx* c, const float* gt);
void stream_destroy(tpm_ctx* c);
int sort_init(tpm_ctx* c);

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// -------------------------------------------------------------- device math

// distance(a, b): int32 wrap-around difference * 2^-32
// (tigerpm/gravity_short.hpp:20-22).
__device__ __forceinline__ float distance32(uint32_t a, uint32_t b) {
  return (float)(int32_t)(a - b) * 2.3283064365386963e-10f;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ int wrapi(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

}  // namespace tpm
