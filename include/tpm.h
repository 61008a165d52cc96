/*
 * tpm.h -- C ABI of tigerpm_b200, a B200-native (sm_100a) PME kick.
 *
 * The library replaces the reference's PME kick path: the chain-mesh cell
 * sort, the long-range PM solve and the fused interpolation / short-range PP /
 * rung-kick kernel, plus the FP64 Ewald comparison.  Every entry point names
 * the reference interface it stands in for (paths relative to the
 * dmarce1/tigerpm tree).  The reference has no C ABI: its interfaces are C++
 * free functions over global state, kept as C++ wrappers in
 * include/tpm_reference.hpp on top of these calls.
 *
 * Conventions
 *  - Every call returns int: TPM_OK (0) or a negative TPM_ERR_* code.  Nothing
 *    aborts or traps; tpm_error_string() and tpm_last_error_message() explain.
 *  - A tpm_ctx holds ONE periodic box: its particles, chain mesh, PM grid,
 *    cuFFT plans and scratch live in device memory owned by the context and
 *    persist across calls.  Host pointers passed in are owned by the caller
 *    and only read/written during the call.
 *  - Positions are the reference's fixed32: raw uint32 = floor(x * 2^32),
 *    uint32 wrap-around being the periodic boundary (tigerpm/fixed.hpp).
 *  - Particle arrays are in the context's current order; tpm_chainmesh_create
 *    permutes them into chain-mesh order, exactly as the reference's
 *    chainmesh_create permutes particles_X/U/R.
 *  - One host thread per context at a time.  All work is issued on the
 *    context's CUDA stream; calls that return host data synchronise it.
 */
#ifndef TPM_H_
#define TPM_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define TPM_OK 0
#define TPM_ERR_INVALID (-1)       /* bad argument or option combination */
#define TPM_ERR_NOMEM (-2)         /* device or host allocation failed */
#define TPM_ERR_CUDA (-3)          /* a CUDA runtime call failed */
#define TPM_ERR_CUFFT (-4)         /* a cuFFT call failed */
#define TPM_ERR_STATE (-5)         /* call out of order (e.g. kick before sort) */
#define TPM_ERR_RUNG (-6)          /* a new rung fell outside [0, 32) (clamped) */
#define TPM_ERR_CAPACITY (-7)      /* particle count above the context capacity */
#define TPM_ERR_BUDGET (-8)        /* request exceeds the admitted HBM budget */
#define TPM_ERR_TIMEOUT (-9)       /* a bounded device wait gave up */
#define TPM_ERR_NOEXT (-10)        /* library built without a required part */

/* gravity_long_type (tigerpm/gravity_long.hpp:17-19) */
#define TPM_GRAVITY_LONG_PM 0
#define TPM_GRAVITY_LONG_PME 1

/* mass assignment: cloud4 = the reference's cubic B-spline deposit
 * (src/gravity_long.cpp:127-199); CIC and TSC are extensions. */
#define TPM_ASSIGN_CLOUD4 0
#define TPM_ASSIGN_CIC 1
#define TPM_ASSIGN_TSC 2

/* chain-mesh order: PARITY replays the reference's recursive partition and
 * reproduces its within-cell order bit for bit (src/chainmesh.cpp:168-213,
 * src/particles.cpp:414-444); FAST is a stable counting sort with the same
 * cell offsets and input order inside each cell. */
#define TPM_SORT_PARITY 0
#define TPM_SORT_FAST 1

/* tpm_options.deterministic_deposit */
#define TPM_DEPOSIT_FP32 0
#define TPM_DEPOSIT_EXACT64 1
#define TPM_DEPOSIT_FIXED32 2

/*
 * Options.  The first block mirrors struct options (tigerpm/options.hpp:6-27)
 * field for field; tpm_options_init derives it as process_options does
 * (src/options.cpp:81-96).  The second block holds this library's extensions;
 * zero / negative values select the reference behaviour.
 */
/* FFT of gravity_long_compute: the library's fused transforms (forward z
 * and y, forward x + Green's function + inverse x in one pass, inverse y and
 * z) when four_dim is a multiple of 16 of the form 2^a 3^b 5^c up to 1024,
 * else cuFFT; or cuFFT always. */
#define TPM_FFT_AUTO 0
#define TPM_FFT_CUFFT 1
/* the library's transforms with the generic block engine for every mesh
 * (AUTO takes the line engine where the mesh has a compiled line plan) */
#define TPM_FFT_BLOCK 2

typedef struct tpm_options {
  int four_dim;     /* PM grid points per side */
  int chain_dim;    /* chain-mesh cells per side */
  int parts_dim;    /* particles^(1/3) */
  int parts_o_four;
  int parts_o_chain;
  int four_o_chain;
  double eta;
  double sigma8;
  double code_to_cm;
  double hubble;
  double GM;
  double hsoft;     /* softening length, box units */
  double box_size;
  double rs;        /* PME split scale, box units (reference: 1 / four_dim) */
  double omega_m;
  double z0;
  /* extensions */
  double rcut_over_rs; /* <= 0: no cutoff, all 27 neighbour cells (reference) */
  int assign;          /* TPM_ASSIGN_*; default cloud4 */
  int deconv_order;    /* sinc^-p deconvolution; 0: assignment order (4/2/3) */
  int sort_mode;       /* TPM_SORT_*; default PARITY */
  int kahan;           /* 1: compensated per-target PP sums (default 1) */
  int deterministic_deposit; /* TPM_DEPOSIT_*: 0 (default) FP32 shared-memory
                              * atomics; 1 exact int64 fixed point, bit-reproducible;
                              * 2 26-bit fixed point in uint32 with integer adds
                              * (fastest), bit-reproducible unless a mesh tile holds
                              * 16 or more weight units at one point, which is then
                              * deposited again with FP32 atomics */
  int fft;             /* TPM_FFT_*: 3-D transforms of gravity_long_compute */
  uint64_t seed;       /* synthetic-input seed carried for drivers */
  int fft_group;       /* x-planes per launch of the library FFT's z / y passes
                        * (0: all; smaller groups keep the spectrum in L2 between
                        * the two passes) */
  int kick_grid;       /* 0: the PP + kick as one persistent launch over a cost-sorted
                        * queue of (cell, sink pass) items (default; balances clustered
                        * boxes); 1: one block per sink cell */
} tpm_options;

typedef struct tpm_ctx tpm_ctx;

/* Per-stage device times of the last calls, milliseconds (CUDA events). */
typedef struct tpm_stage_times {
  float sort_ms;
  float deposit_ms;
  float fft_forward_ms;
  float green_ms;
  float fft_inverse_ms;
  float kick_ms;
  float drift_ms;
  float ewald_ms;
  float interp_ms; /* long-range interpolation at the sinks (part of the kick) */
} tpm_stage_times;

/* Device addresses of the context's particle arrays (current order). */
typedef struct tpm_device_arrays {
  uint32_t* x;
  uint32_t* y;
  uint32_t* z;
  float* vx;
  float* vy;
  float* vz;
  int8_t* rung;
  float* gx;
  float* gy;
  float* gz;
  float* pot;
  int32_t* cell_begin; /* chain_dim^3 + 1 offsets, cells keyed (z*C + y)*C + x */
  float* phi;          /* four_dim^3 potential, x-major, z fastest */
  int64_t n;
} tpm_device_arrays;

const char* tpm_error_string(int status);
/* Message of the last failing call in this thread (never NULL). */
const char* tpm_last_error_message(void);

/* process_options (src/options.cpp:37-118) for the given sizes: derives
 * four_dim = parts_dim / parts_o_four, chain_dim = parts_dim / parts_o_chain,
 * rs = 1 / four_dim, GM = 1, hsoft = 2 / 25 / parts_dim, eta = 0.2 / sqrt 2
 * and the cosmology constants.  Returns TPM_ERR_INVALID where the reference
 * aborts (parts_dim not a multiple of parts_o_four * four_o_chain). */
int tpm_options_init(tpm_options* opts, int parts_dim, int parts_o_four, int four_o_chain);

/* Parses the reference's command line (--parts_dim, --parts_o_four,
 * --four_o_chain, --box_size, --test, --config_file; src/options.cpp:47-55)
 * plus this library's extensions (--four_dim, --chain_dim, --rs_cells,
 * --rcut_over_rs, --assign=cloud4|cic|tsc, --sort=parity|fast, --kahan,
 * --hsoft, --seed, --fft=auto|cufft) into opts.  Unknown flags are TPM_ERR_INVALID. */
int tpm_options_parse(tpm_options* opts, int argc, const char* const* argv);

/* Creates a context for up to `capacity` particles on the current CUDA
 * device.  Allocates all device memory up front (the reference allocates and
 * frees per kick call, src/kick_pme.cu:67-107,616). */
int tpm_ctx_create(const tpm_options* opts, int64_t capacity, tpm_ctx** out);
int tpm_ctx_destroy(tpm_ctx* ctx);
int tpm_ctx_options(const tpm_ctx* ctx, tpm_options* out);
/* Device bytes held by the context. */
int tpm_ctx_device_bytes(const tpm_ctx* ctx, int64_t* bytes);
/* Bytes a context for (opts, capacity) would hold, without allocating. */
int tpm_plan_device_bytes(const tpm_options* opts, int64_t capacity, int64_t* bytes);

/* Host SoA in/out (src/particles.cpp:6-12; particles_pos/vel/rung,
 * tigerpm/particles.hpp:69-80).  Any of vx..rung may be NULL on set (zeros). */
int tpm_set_particles(tpm_ctx* ctx, int64_t n, const uint32_t* x, const uint32_t* y,
                      const uint32_t* z, const float* vx, const float* vy, const float* vz,
                      const int8_t* rung);
/* Same from device memory (pointers on the context's device). */
int tpm_set_particles_device(tpm_ctx* ctx, int64_t n, const uint32_t* x, const uint32_t* y,
                             const uint32_t* z, const float* vx, const float* vy,
                             const float* vz, const int8_t* rung);
/* Any output may be NULL. */
int tpm_get_particles(tpm_ctx* ctx, uint32_t* x, uint32_t* y, uint32_t* z, float* vx,
                      float* vy, float* vz, int8_t* rung);
/* FORCE_TEST outputs particles_G / particles_P (src/particles.cpp:9-12). */
int tpm_get_forces(tpm_ctx* ctx, float* gx, float* gy, float* gz, float* pot);
int tpm_get_device_arrays(tpm_ctx* ctx, tpm_device_arrays* out);
int tpm_num_particles(const tpm_ctx* ctx, int64_t* n);

/* chainmesh_create (src/chainmesh.cpp:139-161; tigerpm/chainmesh.hpp:13):
 * sorts the particles into chain cells on the device, permuting positions,
 * velocities and rungs. */
int tpm_chainmesh_create(tpm_ctx* ctx);
/* chainmesh_get (src/chainmesh.cpp:48-51; tigerpm/chainmesh.hpp:17):
 * {pbegin, pend} of cell ijk = (x, y, z); indices outside [0, C) wrap
 * periodically (the reference's ghost cells hold the same particles). */
int tpm_chainmesh_get(tpm_ctx* ctx, const int ijk[3], int32_t* pbegin, int32_t* pend);
/* All C^3 + 1 cell offsets, keyed (z*C + y)*C + x. */
int tpm_chainmesh_offsets(tpm_ctx* ctx, int32_t* offsets);
/* chainmesh_interior_box (src/chainmesh.cpp:163-166): {b0,b1,b2,e0,e1,e2}. */
int tpm_chainmesh_interior_box(const tpm_ctx* ctx, int box[6]);

/* gravity_long_compute (src/gravity_long.cpp:36-48): deposit, r2c FFT,
 * Green's function, c2r FFT; the potential stays on the device. */
int tpm_gravity_long_compute(tpm_ctx* ctx, int type);
/* gravity_long_get_phi (src/gravity_long.cpp:23-34): the potential over box
 * {b0,b1,b2,e0,e1,e2} (any integer box; indices wrap periodically), written
 * x-major / z fastest as range<int>::index orders it (tigerpm/range.hpp:149-165). */
int tpm_gravity_long_get_phi(tpm_ctx* ctx, const int box[6], float* out);
/* Loads an externally computed periodic potential: four_dim^3 host floats,
 * x-major / z fastest, in the units gravity_long_compute produces.  The
 * reference's kick_pme takes its potential through gravity_long_get_phi
 * (src/kick_pme.cu:446); a caller that keeps its own long-range solver hands
 * that potential to tpm_kick_pme this way.  Valid until the next drift or
 * set_particles. */
int tpm_gravity_long_set_phi(tpm_ctx* ctx, const float* phi);
/* gravity_long_get_phi_box (src/gravity_long.cpp:19-21): the PHI_BW-padded
 * source box of this rank. */
int tpm_gravity_long_get_phi_box(const tpm_ctx* ctx, int box[6]);
/* gravity_long_force_at (src/gravity_long.cpp:52-125): the 4-point cubic
 * interpolation of phi and its gradient at n positions (double, box units),
 * evaluated on the device. */
int tpm_gravity_long_force_at(tpm_ctx* ctx, int64_t n, const double* pos_xyz, float* phi,
                              float* g_xyz);

/* kick_pme (src/kick_pme.cu:390-621; tigerpm/kick_pme.hpp:15): for the
 * sink cells in box {b0,b1,b2,e0,e1,e2} (NULL: the interior box), kicks every
 * particle with rung >= min_rung: quintic interpolation of the long-range
 * force, erfc-split PP sum over the 27 neighbour cells, half-kicks and new
 * rung.  Needs tpm_chainmesh_create and tpm_gravity_long_compute first.
 * Returns TPM_ERR_RUNG if some new rung fell outside [0, 32) (clamped, the
 * reference asserts there). */
int tpm_kick_pme(tpm_ctx* ctx, const int* box, int min_rung, double scale, double t0,
                 int first_call);

/* Fixed-point drift (no reference counterpart): x += trunc(v * dt * 2^32)
 * modulo 2^32 per coordinate. */
int tpm_drift(tpm_ctx* ctx, double dt);

/* gravity_short_ewald_call_kernel (src/gravity_short.cu:10-91;
 * tigerpm/gravity_short.hpp:25-26): FP64 periodic Ewald potential and force
 * at ns sink positions from all particles of the context.  method 0 follows
 * the reference's sum (alpha = 2, images |n| <= 4 with r < 2.6, |h|^2 <= 8);
 * method 1 uses alpha = 6 with precomputed structure factors (same limit to
 * ~1e-10 relative, much faster at large n).  Near pairs (r <= hsoft) take
 * the softened kernel as in the reference. */
int tpm_gravity_short_ewald(tpm_ctx* ctx, int64_t ns, const uint32_t* sx, const uint32_t* sy,
                            const uint32_t* sz, int method, double* phi, double* gx,
                            double* gy, double* gz);
/* Same with sinks given as particle indices in the context's current order. */
int tpm_ewald_fp64(tpm_ctx* ctx, int64_t ns, const int64_t* sample_idx, int method,
                   double* phi, double* gx, double* gy, double* gz);

/* The same FP64 Ewald sum (method 1) for callers that cannot allocate device
 * memory, e.g. a host that hands out every byte of device memory from its own
 * pool, or an allocation-free hook inside a running simulation step.  No
 * counterpart in the reference.  Sources (x, y, z: n particles), sinks
 * (sx, sy, sz: ns points) and outputs (phi, gx, gy, gz: ns each) are device
 * arrays; no context is needed.  All scratch lives in one fixed 448 KiB buffer
 * inside the library that every GPU loading it keeps until exit; no call
 * allocates or frees device memory.  ns above TPM_EWALD_NOALLOC_MAX_SINKS is
 * rejected with TPM_ERR_INVALID.  The first call on a device looks up that
 * buffer's address and copies a small table into it synchronously, so make
 * it before any stream capture.  Calls share the buffer: calls that may
 * overlap on the GPU (other streams or host threads) race and must be
 * serialised by the caller.  Work is queued on `stream` (NULL: the legacy
 * default stream); results are ready when that stream is. */
#define TPM_EWALD_NOALLOC_MAX_SINKS 4096
int tpm_ewald_fp64_noalloc(const uint32_t* x, const uint32_t* y, const uint32_t* z, int64_t n,
                           const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, int64_t ns,
                           double hsoft, double* phi, double* gx, double* gy, double* gz,
                           void* stream);

/* Average device time per call of each stage over the calls since the last
 * tpm_reset_stage_times (up to the last 64 calls per stage). */
int tpm_get_stage_times(tpm_ctx* ctx, tpm_stage_times* out);
int tpm_reset_stage_times(tpm_ctx* ctx);
/* Number of this library's kernel launches issued on the context so far. */
int tpm_get_launch_count(const tpm_ctx* ctx, int64_t* count);
/* Blocks until all work queued on the context is done. */
int tpm_synchronize(tpm_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for event timing by callers. */
int tpm_ctx_stream(tpm_ctx* ctx, void** stream);

/* One whole PME kick without host synchronisation: chainmesh_create,
 * gravity_long_compute(PME) and kick_pme over the interior box -- the
 * sequence of the reference's kick_pme_test (src/test.cpp:182-234).  Kernel
 * error flags are collected on the device; read them with tpm_check_errors. */
int tpm_pme_step(tpm_ctx* ctx, int min_rung, double scale, double t0, int first_call);

/* Host arrays of one particle set (particles_X/U/R layout, n entries each).
 * As an input, vx/vy/vz/rung may be NULL (zero); as an output, any NULL
 * array is skipped. */
typedef struct tpm_host_particles {
  uint32_t* x;
  uint32_t* y;
  uint32_t* z;
  float* vx;
  float* vy;
  float* vz;
  int8_t* rung;
} tpm_host_particles;

/* A served stream of whole PME steps from and to host memory: for each s <
 * nsteps, in[s] (n particles) is uploaded, chain-mesh sorted, given the PME
 * long-range solve and kick_pme over the whole box, and the kicked particles
 * (chain-mesh order, as tpm_get_particles returns them) are written to
 * out[s].  Steps are independent boxes.  The upload of step s+1 and the
 * download of step s-1 overlap step s's kernels (own copy streams; a third
 * device particle set is allocated on the first call).  Host arrays should be
 * page-locked for the overlap; pageable arrays work but serialise.  out[s]
 * may repeat the same arrays (later steps overwrite earlier ones, in order).
 * Returns when every output is written.  Replaces, per step, the reference's
 * host staging and copy-back around kick_pme (src/kick_pme.cu:390-621). */
int tpm_pme_steps_host(tpm_ctx* ctx, int64_t nsteps, int64_t n, const tpm_host_particles* in,
                       const tpm_host_particles* out, int min_rung, double scale, double t0,
                       int first_call);
/* Synchronises and reports (then clears) device error flags raised since the
 * last check: TPM_ERR_RUNG for a clamped rung, TPM_ERR_INVALID for a drift
 * step beyond 2^31 box lengths. */
int tpm_check_errors(tpm_ctx* ctx);

/* ------------------------------------------------------- integration
 *
 * Rung-based kick-drift-kick over one big step t0.  The reference supplies
 * the kick of a block time-step scheme (kick_pme with min_rung and
 * first_call, src/kick_pme.cu:319-354) but no driver and no drift.  Time runs
 * on integer ticks, 2^31 per t0; a particle on rung r is kicked every
 * t0 / 2^r.  tpm_integrate_begin (first_call = 1) kicks every particle
 * (opening half-kicks, rungs assigned).  Each substep finds the largest rung
 * R, drifts every particle to the next multiple of 2^(31-R) ticks and kicks
 * the particles due there, min_rung = 31 - ctz(tick) (every particle at the
 * end of the big step).  Each kick is chainmesh_create +
 * gravity_long_compute(PME) + kick_pme. */
typedef struct tpm_substep {
  int64_t tick;           /* ticks of t0 / ticks_per_step reached by the substep */
  int64_t ticks_per_step; /* 2^31 */
  int max_rung;           /* largest rung before the substep */
  int min_rung;           /* particles kicked: rung >= min_rung */
  double drift_dt;        /* time the substep drifted */
  int done;               /* 1 at the end of the big step */
} tpm_substep;

int tpm_integrate_begin(tpm_ctx* ctx, double t0, double scale, int first_call);
int tpm_integrate_substep(tpm_ctx* ctx, tpm_substep* info);
/* The whole big step; log (optional) receives up to log_cap substeps. */
int tpm_integrate(tpm_ctx* ctx, double t0, double scale, int first_call, int max_substeps, tpm_substep* log,
                  int log_cap, int* nsub);

/* FP64 reductions over the particles, per particle (equal masses): kinetic
 * energy <v^2 / 2>, potential energy <phi / 2> (NaN unless the last kick
 * covered every particle since the last sort or drift) and momentum <v>. */
typedef struct tpm_diag {
  double kinetic;
  double potential;
  double momentum[3];
  int64_t n;
} tpm_diag;
int tpm_diagnostics(tpm_ctx* ctx, tpm_diag* out);

/* -------------------------------------------------- initial conditions
 *
 * Zel'dovich initial conditions generated on the device (initialize and
 * zeldovich_begin / zeldovich_end, src/initialize.cpp:91-221): one complex
 * normal deviate per mode times sqrt(P(k)) K / k^2, the kz = 0 plane made
 * Hermitian (fft3d_force_real, src/fft.cpp:86-123), an inverse FFT, and
 * x = (I + 1/2) / N + displacement, wrapped, as fixed32.  Deviates come from
 * Philox-4x32-10 keyed by `seed` with the mode's array indices as counter
 * (the reference draws GSL taus sequentially).
 *   npower > 0: P(k) is the reference's table form (power.init columns k in
 *     h/Mpc and P in (Mpc/h)^3; cubic interpolation in ln k, normalised to
 *     the context's sigma8; amplitude from its code_to_cm box size and the
 *     growth factor at z0), unless rms_disp > 0 rescales it;
 *   npower = 0: P(k) = k^index exp(-k / (kcut_over_nyq k_Nyq)) in mode
 *     units, scaled to an rms displacement of rms_disp particle spacings.
 * Writes n_side^3 particles (x-major lattice order, zero velocities and
 * rungs) into the context; dxmax = the largest |displacement| in spacings. */
typedef struct tpm_ic_params {
  int n_side;
  uint64_t seed;
  int npower;
  const double* power_k;
  const double* power_p;
  double index;
  double kcut_over_nyq;
  double rms_disp;
} tpm_ic_params;
int tpm_ic_zeldovich(tpm_ctx* ctx, const tpm_ic_params* params, double* dxmax);
/* The power_spectrum_function of a table (src/initialize.cpp:10-66,182-211)
 * evaluated at nk wavenumbers (1/Mpc), normalised to sigma8. */
int tpm_ic_power(const double* table_k, const double* table_p, int npower, double hubble, double sigma8, int nk,
                 const double* k, double* p_out);
/* growth_factor (src/initialize.cpp:76-83). */
int tpm_growth_factor(double omega_m, double a, double* out);

/* ------------------------------------------------------------ batches
 *
 * An ensemble of independent periodic boxes (each with its own particle
 * count, PM mesh and chain mesh) kicked together.  The reference kicks one
 * box per kick_pme call, with a static contiguous split of the box's cells
 * over the launch (src/kick_pme.cu:139-141) and box splitting when device
 * memory is short (src/kick_pme.cu:418-430).  A batch step runs every box's
 * chain-mesh sort and long-range solve concurrently (one stream per box),
 * then the interpolation of all boxes in one launch and the PP sum + rung
 * kick of all boxes in ONE persistent launch over a work queue of
 * (box, chain cell) items ordered heaviest first.  Each box is a tpm_ctx
 * reachable through tpm_batch_box (results, forces, particles). */
typedef struct tpm_batch tpm_batch;

/* Launch shape of the kick kernel: warps per block, sources staged in
 * shared memory per chunk, sinks per pass (a power of two); tuned = 1 when
 * it came from tpm_batch_autotune; ms = its measured kick time. */
typedef struct tpm_kick_shape {
  int warps;
  int stage;
  int npass;
  int tuned;
  float ms;
} tpm_kick_shape;

/* Device times of the phases of the last tpm_batch_step, milliseconds. */
typedef struct tpm_batch_times {
  float long_range_ms; /* fork: every box's sort + deposit + FFT solve */
  float queue_ms;      /* work-queue build */
  float interp_ms;     /* long-range interpolation, all boxes */
  float kick_ms;       /* persistent PP + rung kick, all boxes */
} tpm_batch_times;

#define TPM_BATCH_RESTORE 1 /* restore every box's particles from its input first */
#define TPM_BATCH_GRAPH 2   /* capture the step as a CUDA graph once, replay it */

/* nbox boxes; box i gets options opts[i] and room for capacity[i] particles. */
int tpm_batch_create(int nbox, const tpm_options* opts, const int64_t* capacity, tpm_batch** out);
int tpm_batch_destroy(tpm_batch* b);
int tpm_batch_size(const tpm_batch* b, int* nbox, int64_t* particles);
/* The context of box i (owned by the batch). */
int tpm_batch_box(tpm_batch* b, int i, tpm_ctx** ctx);
/* Host particles of box i: they become its current particles and its
 * input, which TPM_BATCH_RESTORE copies back before a step. */
int tpm_batch_set_input(tpm_batch* b, int i, int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z,
                        const float* vx, const float* vy, const float* vz, const int8_t* rung);
/* One PME kick of every box: chainmesh_create + gravity_long_compute(PME) +
 * kick_pme over the interior box, per box, with the arguments of
 * tpm_pme_step.  No host synchronisation. */
int tpm_batch_step(tpm_batch* b, int flags, int min_rung, double scale, double t0, int first_call);
/* The same step through the plain single-box path, box after box. */
int tpm_batch_steps_sequential(tpm_batch* b, int restore_inputs, int min_rung, double scale, double t0,
                               int first_call);
int tpm_batch_synchronize(tpm_batch* b);
/* The batch's main stream (a cudaStream_t): a step ends there. */
int tpm_batch_stream(tpm_batch* b, void** stream);
/* This library's kernel launches issued by the batch's steps so far
 * (a graph replay counts its kernel nodes). */
int tpm_batch_launch_count(const tpm_batch* b, int64_t* count);
int tpm_batch_phase_times(tpm_batch* b, tpm_batch_times* out);
int tpm_batch_get_shape(const tpm_batch* b, tpm_kick_shape* s);
int tpm_batch_set_shape(tpm_batch* b, const tpm_kick_shape* s);
/* Times the candidate kick shapes on the batch (after a step) and keeps the
 * fastest; later batches with the same mean chain-cell occupancy start from
 * it.  Velocities and rungs are restored; forces are those of a trial. */
int tpm_batch_autotune(tpm_batch* b, int min_rung, int repeats, tpm_kick_shape* best);

/* ------------------------------------------------------------ serving
 *
 * A request loop for kick + drift steps of many resident boxes.  The
 * reference allocates, stages, kicks and frees per kick_pme call
 * (src/kick_pme.cu:390-621) and splits a box when free memory is short
 * (:418-430).  A server keeps each admitted box resident on the device
 * (particles, chain-mesh tables, FFT twiddles and Green's-function tables,
 * about 25 bytes per particle) and lends every running step its working set
 * (forces, packed positions, sort scratch, PM meshes) from a stream-ordered
 * pool, within one device budget:
 *     resident bytes of all boxes + working sets of steps in flight <= budget.
 * Requests queue in FIFO order and start as slots (streams) and memory free
 * up, so steps of different boxes overlap on the GPU; a dispatcher thread
 * admits them.  One step = chainmesh_create + gravity_long_compute(PME) +
 * kick_pme over the whole box + tpm_drift(dt). */
typedef struct tpm_server tpm_server;

typedef struct tpm_serve_result {
  int status;        /* TPM_OK or the step's error */
  int box;
  double latency_ms; /* submission to completion, host clock */
  double queue_ms;   /* submission to start (admission wait) */
  float device_ms;   /* the step's kernels, device clock */
  int64_t particles; /* particles kicked */
} tpm_serve_result;

typedef struct tpm_serve_stats_t {
  int64_t budget_bytes;
  int64_t resident_bytes;        /* held by admitted boxes */
  int64_t inflight_peak_bytes;   /* largest sum of working sets in flight */
  int64_t max_working_set_bytes; /* largest working set of any box */
  int boxes;
  int max_concurrent_steps;
  int64_t steps_done;
  int64_t particles_done;
  int64_t launches; /* this library's kernel launches of the served steps */
} tpm_serve_stats_t;

/* budget_bytes <= 0: 80 % of the device's free memory.  max_slots: steps
 * in flight at most (1..64). */
int tpm_serve_create(int64_t budget_bytes, int max_slots, tpm_server** out);
int tpm_serve_destroy(tpm_server* s);
/* Admits a box of n particles (host arrays, as tpm_set_particles) with its
 * options; TPM_ERR_BUDGET when its resident set, with the largest working
 * set of any box, would not fit the budget. */
int tpm_serve_add_box(tpm_server* s, const tpm_options* opts, int64_t n, const uint32_t* x, const uint32_t* y,
                      const uint32_t* z, const float* vx, const float* vy, const float* vz, const int8_t* rung,
                      int* box_id);
/* The same with the box's particles generated on the device by
 * tpm_ic_zeldovich (n = n_side^3). */
int tpm_serve_add_box_ic(tpm_server* s, const tpm_options* opts, const tpm_ic_params* ic, int* box_id);
/* Queues one step of a box (tpm_pme_step arguments + drift dt); returns at once. */
int tpm_serve_submit(tpm_server* s, int box, double dt, int min_rung, double scale, double t0, int first_call,
                     int* req_id);
/* Blocks until the request is done; returns its status. */
int tpm_serve_wait(tpm_server* s, int req, tpm_serve_result* out);
/* Blocks until every queued request is done. */
int tpm_serve_drain(tpm_server* s);
/* Submits request i for box[i] at arrival_s[i] seconds after the call
 * starts (host clock), then waits for all; results[i] per request. */
int tpm_serve_replay(tpm_server* s, int nreq, const int* box, const double* arrival_s, double dt, int min_rung,
                     double scale, double t0, int first_call, tpm_serve_result* results);
/* The context of an idle box (its particles, chain mesh offsets); TPM_ERR_STATE
 * while a step of it is in flight.  Its working set is not kept between steps. */
int tpm_serve_box(tpm_server* s, int box, tpm_ctx** ctx);
int tpm_serve_stats(tpm_server* s, tpm_serve_stats_t* out);

/* Candidate sink-source pairs of the 27-cell neighbourhoods (active sinks,
 * rung >= min_rung) and the pairs inside the cutoff, counted on the device. */
int tpm_count_pairs(tpm_ctx* ctx, int min_rung, int64_t* candidates, int64_t* inside);

/* Measured FP32 FMA throughput of the current device (TFLOP/s), from a
 * dense FMA-chain kernel: the denominator for the PP kernel's roofline. */
int tpm_fp32_peak_probe(double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* TPM_H_ */
