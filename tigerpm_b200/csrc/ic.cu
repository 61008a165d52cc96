// ic.cu -- Zel'dovich initial conditions generated on the device.
//
// Reference: initialize() (src/initialize.cpp:213-221) ->
//   zeldovich_begin (:91-136): for every mode (i, j, k) of the half spectrum
//     with 0 < i^2 + j^2 + k^2 < N^2/4 (integer mode numbers, negative above
//     N/2), a complex normal deviate exp(2 pi i y) sqrt(-ln x) times
//     sqrt(P(|k|)) * L^-1.5 * N^3 * K_dim / |K|^2, K = 2 pi / L * mode;
//   fft3d_force_real (src/fft.cpp:86-123): the kz = 0 plane made Hermitian,
//     Y(k) <- (Y(k) + conj Y(-k)) / 2;
//   fft3d_inv_execute: inverse transform with 1/N^3 (src/fft.cpp:69-84);
//   zeldovich_end (:138-180): x = (I + 1/2) / N - D1 * Y / L, wrapped into
//     [0, 1); it returns max |dx| N.
// The power spectrum is the reference's power_spectrum_function
// (:10-66): a (k, P) table read as power.init with k *= h, P /= h^3
// (:182-211), interpolated as a cubic in ln k through ln P and normalised to
// sigma8 by Simpson's rule over ln k; D1 = growth_factor(omega_m, a0) /
// growth_factor(omega_m, 1) (:76-83).
//
// Differences, by design: the deviates come from Philox-4x32-10 (Salmon,
// Moraes, Dror & Shaw, SC'11) keyed by the seed with the mode's (i, j, kz)
// as the counter, instead of GSL's sequential taus stream, so every mode is
// generated independently on the device (the same deviate serves all three
// dimensions, as the reference's re-seeded stream does); the mode arithmetic
// is FP64, the inverse FFT cuFFT C2R in FP32.  A second spectrum form,
// P ~ k^n exp(-k / (kcut k_Nyq)) in mode units, and a normalisation to a
// target rms displacement (in particle spacings) serve the synthetic
// benchmark boxes.
#include "tpm_internal.cuh"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace tpm {
namespace {

constexpr double kTwoPi = 6.283185307179586;
constexpr double kMpcToCm = 3.086e+24;  // constants::mpc_to_cm, tigerpm/tigerpm.hpp:76

// Philox-4x32-10 (Salmon et al. 2011): ten rounds of two 32x32 -> 64-bit
// multiplies with a Weyl-sequence key schedule.
__host__ __device__ inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t c1 = ctr[1], c3 = ctr[3];
    ctr[0] = hi1 ^ c1 ^ k0;
    ctr[1] = lo1;
    ctr[2] = hi0 ^ c3 ^ k1;
    ctr[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// The complex deviate of mode (i, j, kz) (array indices, kz < N/2 + 1).
__device__ inline double2 mode_deviate(int i, int j, int kz, uint64_t seed) {
  uint32_t c[4] = {(uint32_t)i, (uint32_t)j, (uint32_t)kz, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double x = ((double)c[0] + 1.0) * 2.3283064365386963e-10;  // (0, 1]
  const double y = (double)c[1] * 2.3283064365386963e-10;          // [0, 1)
  const double m = sqrt(-log(x));
  double s, co;
  sincospi(2.0 * y, &s, &co);
  return make_double2(co * m, s * m);
}

__device__ inline int signed_mode(int i, int N) { return i < N / 2 ? i : i - N; }

// Y_d(i, j, kz) for d = 0, 1, 2 before the Hermitian fix-up.
__device__ inline void mode_value(int i, int j, int kz, int N, uint64_t seed, const double* __restrict__ amp,
                                  double kunit, double2 y[3]) {
  const int a = signed_mode(i, N), b = signed_mode(j, N), c = signed_mode(kz, N);
  const int64_t i2 = (int64_t)a * a + (int64_t)b * b + (int64_t)c * c;
  if (i2 > 0 && i2 < (int64_t)N * N / 4) {
    const double2 rn = mode_deviate(i, j, kz, seed);
    const double A = amp[i2];
    const double K[3] = {kunit * a, kunit * b, kunit * c};
#pragma unroll
    for (int d = 0; d < 3; d++) y[d] = make_double2(rn.x * A * K[d], rn.y * A * K[d]);
  } else {
#pragma unroll
    for (int d = 0; d < 3; d++) y[d] = make_double2(0.0, 0.0);
  }
}

// One thread per half-spectrum element; the three dimensions' spectra are
// stored in place-transform layout (complex N x N x (N/2+1)).
__global__ void k_ic_modes(int N, uint64_t seed, const double* __restrict__ amp, double kunit,
                           float2* __restrict__ Y0, float2* __restrict__ Y1, float2* __restrict__ Y2) {
  const int Nh = N / 2 + 1;
  const int64_t total = (int64_t)N * N * Nh;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int kz = (int)(e % Nh);
    const int64_t r = e / Nh;
    const int j = (int)(r % N), i = (int)(r / N);
    double2 y[3];
    mode_value(i, j, kz, N, seed, amp, kunit, y);
    if (kz == 0) {  // fft3d_force_real: (Y(k) + conj Y(-k)) / 2 on the kz = 0 plane
      double2 m[3];
      mode_value((N - i) % N, (N - j) % N, 0, N, seed, amp, kunit, m);
#pragma unroll
      for (int d = 0; d < 3; d++) y[d] = make_double2(0.5 * (y[d].x + m[d].x), 0.5 * (y[d].y - m[d].y));
    }
    Y0[e] = make_float2((float)y[0].x, (float)y[0].y);
    Y1[e] = make_float2((float)y[1].x, (float)y[1].y);
    Y2[e] = make_float2((float)y[2].x, (float)y[2].y);
  }
}

// Sum of squares of the three displacement fields (padded real layout).
__global__ void k_ic_sumsq(int N, const float* __restrict__ R0, const float* __restrict__ R1,
                           const float* __restrict__ R2, double* __restrict__ out) {
  const int P = 2 * (N / 2 + 1);
  const int64_t total = (int64_t)N * N * N;
  double s = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = p / N;
    const int64_t o = row * P + (p - row * N);
    const double a = R0[o], b = R1[o], c = R2[o];
    s += a * a + b * b + c * c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    atomicAdd(out, t);
  }
}

// Particle p = (I0 N + I1) N + I2 at (I + 1/2) / N + scale * Y(I), wrapped,
// as fixed32; zero velocity and rung.  |dx| N of the largest displacement
// (bit pattern of a non-negative float, so an integer max orders it).
__global__ void k_ic_positions(int N, const float* __restrict__ R0, const float* __restrict__ R1,
                               const float* __restrict__ R2, double scale, uint32_t* __restrict__ x,
                               uint32_t* __restrict__ y, uint32_t* __restrict__ z, float* __restrict__ vx,
                               float* __restrict__ vy, float* __restrict__ vz, int8_t* __restrict__ rung,
                               unsigned* __restrict__ dxmax_bits) {
  const int P = 2 * (N / 2 + 1);
  const int64_t total = (int64_t)N * N * N;
  float mx = 0.f;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = p / N;
    const int I2 = (int)(p - row * N);
    const int I1 = (int)(row % N), I0 = (int)(row / N);
    const int64_t o = row * P + I2;
    const float* R[3] = {R0, R1, R2};
    const int I[3] = {I0, I1, I2};
    uint32_t* X[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double dx = scale * (double)R[d][o];
      mx = fmaxf(mx, (float)fabs(dx * N));
      double q = ((double)I[d] + 0.5) / N + dx;
      q -= floor(q);  // periodic wrap into [0, 1)
      double t = q * 4294967296.0;
      if (t >= 4294967295.0) t = 4294967295.0;
      X[d][p] = (uint32_t)t;
    }
    vx[p] = 0.f;
    vy[p] = 0.f;
    vz[p] = 0.f;
    rung[p] = 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dxmax_bits, __float_as_uint(mx));
}

}  // namespace

// ---------------------------------------------------------------- spectrum
//
// power_spectrum_function (src/initialize.cpp:10-66) restated in double:
// P(k) = exp(cubic in ln k through ln P of the four table entries around k),
// the first of them clamped to [0, size - 4]; normalise() scales P so that
// sigma8^2 = int P(k) W(kR)^2 k^3 / (2 pi^2) dlnk, R = 8 / h Mpc, by
// Simpson's rule with 8192 intervals between the table's ln k limits.
struct PowerTable {
  std::vector<double> P;
  double logkmin = 0, logkmax = 0, dlogk = 1;

  double operator()(double k) const {
    const double logk = std::log(k);
    const double k0 = (logk - logkmin) / dlogk;
    int i0 = (int)k0 - 1;
    i0 = std::max(0, i0);
    i0 = std::min((int)P.size() - 4, i0);
    const double x = k0 - (i0 + 1);
    const double y0 = std::log(P[i0]), y1 = std::log(P[i0 + 1]), y2 = std::log(P[i0 + 2]),
                 y3 = std::log(P[i0 + 3]);
    const double k1 = (y2 - y0) * 0.5, k2 = (y3 - y1) * 0.5;
    const double a = y1, b = k1, c = -2 * k1 - k2 - 3 * y1 + 3 * y2, d = k1 + k2 + 2 * y1 - 2 * y2;
    return std::exp(a + b * x + c * x * x + d * x * x * x);
  }
  double sigma8_integrand(double lnk, double hubble) const {
    const double R = 8.0 / hubble;
    const double c0 = 9.0 / (2.0 * M_PI * M_PI) / std::pow(R, 6);
    const double k = std::exp(lnk);
    const double t = std::sin(k * R) - k * R * std::cos(k * R);
    return c0 * (*this)(k) * t * t * std::pow(k, -3);
  }
  void normalise(double sigma8, double hubble) {
    const int n = 8 * 1024;
    const double h = (logkmax - logkmin) / n;
    double sum = (1.0 / 3.0) * (sigma8_integrand(logkmax, hubble) + sigma8_integrand(logkmin, hubble)) * h;
    for (int i = 1; i < n; i += 2) sum += (4.0 / 3.0) * sigma8_integrand(logkmin + i * h, hubble) * h;
    for (int i = 2; i < n; i += 2) sum += (2.0 / 3.0) * sigma8_integrand(logkmin + i * h, hubble) * h;
    const double f = sigma8 * sigma8 / sum;
    for (double& p : P) p *= f;
  }
};

// read_power_spectrum (src/initialize.cpp:182-211) from arrays.
int make_table(const double* k, const double* p, int n, double hubble, double sigma8, PowerTable& t) {
  if (n < 4) return fail(TPM_ERR_INVALID, "a power table needs at least 4 entries");
  double kmin = INFINITY, kmax = 0;
  t.P.resize(n);
  for (int i = 0; i < n; i++) {
    if (!(k[i] > 0) || !(p[i] > 0)) return fail(TPM_ERR_INVALID, "power table entries must be positive");
    const double kk = k[i] * hubble;
    t.P[i] = p[i] / (hubble * hubble * hubble);
    kmin = std::min(kmin, kk);
    kmax = std::max(kmax, kk);
  }
  t.logkmin = std::log(kmin);
  t.logkmax = std::log(kmax);
  t.dlogk = (t.logkmax - t.logkmin) / (n - 1);
  t.normalise(sigma8, hubble);
  return TPM_OK;
}

// growth_factor (src/initialize.cpp:76-83): the linear growth factor of a
// flat LCDM universe (Carroll, Press & Turner 1992 fit), with the
// reference's single-precision a and literals (4/7, 1/70).
double growth_factor(double omega_m, double a_in) {
  const double a = (double)(float)a_in;
  const double omega_l = 1.0 - omega_m;
  const double a3 = a * (a * a);
  const double deninv = 1.0 / (omega_m + a3 * omega_l);
  const double Om = omega_m * deninv;
  const double Ol = a3 * omega_l * deninv;
  return a * 2.5 * Om /
         (std::pow(Om, (double)(4.f / 7.f)) - Ol + (1.0 + 0.5 * Om) * (1.0 + (double)0.014285714f * Ol));
}

}  // namespace tpm

using namespace tpm;

extern "C" {

int tpm_ic_power(const double* table_k, const double* table_p, int npower, double hubble, double sigma8, int nk,
                 const double* k, double* p_out) {
  if (!table_k || !table_p || (nk > 0 && (!k || !p_out))) return fail(TPM_ERR_INVALID, "null argument");
  PowerTable t;
  int rc = make_table(table_k, table_p, npower, hubble, sigma8, t);
  if (rc) return rc;
  for (int i = 0; i < nk; i++) p_out[i] = t(k[i]);
  return TPM_OK;
}

int tpm_growth_factor(double omega_m, double a, double* out) {
  if (!out) return fail(TPM_ERR_INVALID, "null argument");
  *out = growth_factor(omega_m, a);
  return TPM_OK;
}

int tpm_ic_zeldovich(tpm_ctx* c, const tpm_ic_params* ip, double* dxmax_out) {
  if (!c || !ip) return fail(TPM_ERR_INVALID, "null argument");
  const int N = ip->n_side;
  if (N < 2 || N > 2048) return fail(TPM_ERR_INVALID, "n_side must be in [2, 2048]");
  const int64_t n = (int64_t)N * N * N;
  if (n > c->cap) return fail(TPM_ERR_CAPACITY, "n_side^3 above the context capacity");
  const tpm_options& o = c->opt;
  // amplitude per integer |mode|^2 < N^2 / 4, in FP64
  const int64_t m_end = (int64_t)N * N / 4;
  std::vector<double> amp(std::max<int64_t>(m_end, 1), 0.0);
  double kunit, scale;
  double L = 1.0;
  if (ip->npower > 0) {
    PowerTable t;
    int rc = make_table(ip->power_k, ip->power_p, ip->npower, o.hubble, o.sigma8, t);
    if (rc) return rc;
    L = o.code_to_cm / kMpcToCm;  // box size in Mpc (src/initialize.cpp:93)
    kunit = kTwoPi / L;
    const double factor = std::pow(L, -1.5) * (double)N * N * N;
    for (int64_t m = 1; m < m_end; m++) {
      const double k = kunit * std::sqrt((double)m);
      amp[m] = std::sqrt(t(k)) * factor / (k * k);
    }
    const double a0 = 1.0 / (o.z0 + 1.0);
    scale = -(growth_factor(o.omega_m, a0) / growth_factor(o.omega_m, 1.0)) / L;
  } else {
    if (!(ip->kcut_over_nyq > 0)) return fail(TPM_ERR_INVALID, "kcut_over_nyq must be positive");
    kunit = 1.0;  // mode units; the rms normalisation fixes the amplitude
    const double knyq = 0.5 * N;
    for (int64_t m = 1; m < m_end; m++) {
      const double k = std::sqrt((double)m);
      const double P = std::pow(k, ip->index) * std::exp(-k / (ip->kcut_over_nyq * knyq));
      amp[m] = std::sqrt(P) / (k * k);
    }
    scale = -1.0;
  }
  if (ip->npower <= 0 && !(ip->rms_disp > 0)) return fail(TPM_ERR_INVALID, "a power-law spectrum needs rms_disp > 0");
  cudaStream_t s = c->stream;
  const int Nh = N / 2 + 1;
  const size_t cplx = (size_t)N * N * Nh;  // complex elements per dimension (in-place: 2 Nh reals per row)
  double* d_amp = nullptr;
  float2* Y = nullptr;
  double* d_sum = nullptr;
  unsigned* d_max = nullptr;
  cufftHandle plan = 0;
  bool have_plan = false;
  int rc = TPM_OK;
  cudaError_t e = cudaMallocAsync((void**)&d_amp, sizeof(double) * amp.size(), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&Y, sizeof(float2) * cplx * 3, s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_sum, sizeof(double) + sizeof(unsigned) * 2, s);
  if (e == cudaSuccess) {
    d_max = reinterpret_cast<unsigned*>(d_sum + 1);
    e = cudaMemcpyAsync(d_amp, amp.data(), sizeof(double) * amp.size(), cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(d_sum, 0, sizeof(double) + sizeof(unsigned) * 2, s);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<int64_t>(ceil_div((int64_t)cplx, 256), 148 * 16);
    k_ic_modes<<<blocks, 256, 0, s>>>(N, ip->seed, d_amp, kunit, Y, Y + cplx, Y + 2 * cplx);
    c->launches++;
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) rc = fail(TPM_ERR_CUDA, std::string("ic modes: ") + cudaGetErrorString(e));
  if (rc == TPM_OK) {
    // inverse transforms in place (cuFFT's padded real layout), unnormalised
    if (cufftPlan3d(&plan, N, N, N, CUFFT_C2R) != CUFFT_SUCCESS || cufftSetStream(plan, s) != CUFFT_SUCCESS) {
      rc = fail(TPM_ERR_CUFFT, "ic: cufftPlan3d C2R");
    } else {
      have_plan = true;
      for (int d = 0; d < 3 && rc == TPM_OK; d++) {
        cufftComplex* in = reinterpret_cast<cufftComplex*>(Y + d * cplx);
        if (cufftExecC2R(plan, in, reinterpret_cast<cufftReal*>(in)) != CUFFT_SUCCESS)
          rc = fail(TPM_ERR_CUFFT, "ic: cufftExecC2R");
      }
    }
  }
  const float* R0 = reinterpret_cast<const float*>(Y);
  const float* R1 = reinterpret_cast<const float*>(Y + cplx);
  const float* R2 = reinterpret_cast<const float*>(Y + 2 * cplx);
  const int pblocks = (int)std::min<int64_t>(ceil_div(n, 256), 148 * 16);
  if (rc == TPM_OK && ip->rms_disp > 0) {
    k_ic_sumsq<<<pblocks, 256, 0, s>>>(N, R0, R1, R2, d_sum);
    c->launches++;
    double sum = 0;
    e = cudaMemcpyAsync(&sum, d_sum, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(TPM_ERR_CUDA, std::string("ic rms: ") + cudaGetErrorString(e));
    const double rms = std::sqrt(sum / (double)n);  // of the unnormalised transform
    if (rc == TPM_OK && !(rms > 0)) rc = fail(TPM_ERR_INVALID, "ic: the displacement field is zero");
    if (rc == TPM_OK) scale = -(ip->rms_disp / N) / rms;
  } else if (rc == TPM_OK) {
    scale /= (double)n;  // the reference's inverse transform carries 1/N^3
  }
  if (rc == TPM_OK) {
    k_ic_positions<<<pblocks, 256, 0, s>>>(N, R0, R1, R2, scale, c->x, c->y, c->z, c->vx, c->vy, c->vz, c->rung,
                                           d_max);
    c->launches++;
    e = cudaGetLastError();
    unsigned mb = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&mb, d_max, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(TPM_ERR_CUDA, std::string("ic positions: ") + cudaGetErrorString(e));
    float mx;
    memcpy(&mx, &mb, sizeof(float));
    if (dxmax_out) *dxmax_out = mx;
  }
  if (have_plan) cufftDestroy(plan);
  if (d_amp) cudaFreeAsync(d_amp, s);
  if (Y) cudaFreeAsync(Y, s);
  if (d_sum) cudaFreeAsync(d_sum, s);
  cudaStreamSynchronize(s);
  if (rc == TPM_OK) {
    c->n = n;
    c->sorted = false;
    c->have_phi = false;
    c->host_cells_valid = false;
  }
  return rc;
}

}  // extern "C"
