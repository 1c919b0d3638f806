// Adaptive Fourier mass of the boson momenta: the per-step arithmetic around
// the FFTs (hmc_sampler_batch.py:1133-1277, restated from its mathematics).
//
// The sampler estimates, per chain and bond direction, the power spectrum of
// the field's fluctuations on the real-FFT grid [Lx][Ly][Ltau/2 + 1]:
//   mean_n = (n mean_{n-1} + x) / (n + 1),
//   S_n    = (n S_{n-1} + |F(x - mean_n)|^2) / (n + 1)      (F orthonormal),
// and every so many steps turns S into the mass spectrum sigma per row
// (chain, direction): clamp to [0, c] (c = the mean over rows of each row's
// 0.99 quantile), Box-Cox with exponent lambda, rescale the row into
// [s_min, s_max], shift its mean to 1, shrink towards 1 by lmd, and invert
// for mass mode -1.  Momenta are drawn as F^-1((a + i b) / sqrt(sigma m_k))
// with a, b standard normal and m_k the multiplicity of the tau frequency
// (1 for the first and last, 2 otherwise); M^-1 p = F^-1(sigma F p).
#include <algorithm>
#include <cmath>

#include "qedf_internal.h"

namespace qedf {

// mean <- (cnt mean + x) / (cnt + 1); d = x - mean (after the update)
template <typename R>
__global__ void k_fm_accumulate(R* mean, const R* x, R* d, int64_t n, double cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const R m = (mean[i] * (R)cnt + x[i]) / (R)(cnt + 1.0);
    mean[i] = m;
    d[i] = x[i] - m;
  }
}

// S <- (cnt S + |X|^2) / (cnt + 1); X complex (re, im interleaved)
template <typename R>
__global__ void k_fm_spectrum(R* S, const R* X, int64_t n, double cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const R re = X[2 * i], im = X[2 * i + 1];
    S[i] = (S[i] * (R)cnt + (re * re + im * im)) / (R)(cnt + 1.0);
  }
}

template <typename R>
__device__ R block_reduce(R v, R* sh, int op) {  // op 0: sum, 1: min, 2: max
  for (int o = 16; o > 0; o >>= 1) {
    const R w = __shfl_xor_sync(0xffffffffu, v, o);
    v = op == 0 ? v + w : (op == 1 ? fmin(v, w) : fmax(v, w));
  }
  const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (ln == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = ln < nw ? sh[ln] : (op == 0 ? R(0) : sh[0]);
    for (int o = 16; o > 0; o >>= 1) {
      const R w = __shfl_xor_sync(0xffffffffu, v, o);
      v = op == 0 ? v + w : (op == 1 ? fmin(v, w) : fmax(v, w));
    }
    if (ln == 0) sh[32] = v;
  }
  __syncthreads();
  return sh[32];
}

// One block per row of len values: the spectrum S (read) becomes the mass
// spectrum sigma (written; may alias S).  clamp_hi: device scalar c.
template <typename R>
__global__ void k_fm_mass(const R* S, R* sigma, int64_t len, const R* clamp_hi, double lambda, double smin,
                          double smax, double lmd, int invert) {
  __shared__ R sh[33];
  const R* s = S + blockIdx.x * len;
  R* o = sigma + blockIdx.x * len;
  const R c = *clamp_hi, lam = (R)lambda;
  auto bc = [&](R v) {  // clamp to [0, c], then Box-Cox
    v = fmin(fmax(v, R(0)), c);
    return (pow(v, lam) - R(1)) / lam;
  };
  R lo = INFINITY, hi = -INFINITY;
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
    const R v = bc(s[i]);
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  lo = block_reduce(lo, sh, 1);
  hi = block_reduce(hi, sh, 2);
  const R scale = (R)(smax - smin) / fmax(hi - lo, R(1e-8));
  R sum = 0;
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) sum += (bc(s[i]) - lo) * scale + (R)smin;
  sum = block_reduce(sum, sh, 0);
  const R shift = R(1) - sum / (R)len;
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
    R v = (bc(s[i]) - lo) * scale + (R)smin + shift;
    v = (R)(1.0 - lmd) * v + (R)lmd;
    o[i] = invert ? R(1) / v : v;
  }
}

// z = (a + i b) / sqrt(sigma m_k); nk = Ltau/2 + 1 frequencies on the last axis
template <typename R>
__global__ void k_fm_noise(const R* a, const R* b, const R* sigma, R* z, int64_t n, int nk) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % nk);
    const R m = (k == 0 || k == nk - 1) ? R(1) : R(2);
    const R f = R(1) / sqrt(sigma[i] * m);
    z[2 * i] = a[i] * f;
    z[2 * i + 1] = b[i] * f;
  }
}

// P <- P sigma (complex times real)
template <typename R>
__global__ void k_fm_scale(R* P, const R* sigma, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    P[2 * i] *= sigma[i];
    P[2 * i + 1] *= sigma[i];
  }
}

static dim3 ew_grid(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return dim3((unsigned)std::min<int64_t>(b, (int64_t)num_sms() * 8));
}

template <typename R>
int fm_accumulate(R* mean, const R* x, R* d, int64_t n, double cnt, cudaStream_t st) {
  k_fm_accumulate<R><<<ew_grid(n), 256, 0, st>>>(mean, x, d, n, cnt);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template <typename R>
int fm_spectrum(R* S, const R* X, int64_t n, double cnt, cudaStream_t st) {
  k_fm_spectrum<R><<<ew_grid(n), 256, 0, st>>>(S, X, n, cnt);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template <typename R>
int fm_mass(const R* S, R* sigma, int rows, int64_t len, const R* c, double lambda, double smin, double smax,
            double lmd, int invert, cudaStream_t st) {
  k_fm_mass<R><<<rows, 256, 0, st>>>(S, sigma, len, c, lambda, smin, smax, lmd, invert);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template <typename R>
int fm_noise(const R* a, const R* b, const R* sigma, R* z, int64_t n, int nk, cudaStream_t st) {
  k_fm_noise<R><<<ew_grid(n), 256, 0, st>>>(a, b, sigma, z, n, nk);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template <typename R>
int fm_scale(R* P, const R* sigma, int64_t n, cudaStream_t st) {
  k_fm_scale<R><<<ew_grid(n), 256, 0, st>>>(P, sigma, n);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

}  // namespace qedf

using namespace qedf;

namespace {
inline bool ok_ptrs(const void* a, const void* b) { return a && b; }
}  // namespace

extern "C" {

int qedf_fm_accumulate_f32(float* mean, const float* x, float* d, int64_t n, double cnt, qedf_stream_t s) {
  if (!ok_ptrs(mean, x) || !d || n < 1 || !(cnt >= 0)) return QEDF_ERR_ARG;
  return fm_accumulate<float>(mean, x, d, n, cnt, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_accumulate_f64(double* mean, const double* x, double* d, int64_t n, double cnt, qedf_stream_t s) {
  if (!ok_ptrs(mean, x) || !d || n < 1 || !(cnt >= 0)) return QEDF_ERR_ARG;
  return fm_accumulate<double>(mean, x, d, n, cnt, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_spectrum_f32(float* S, const float* X, int64_t n, double cnt, qedf_stream_t s) {
  if (!ok_ptrs(S, X) || n < 1 || !(cnt >= 0)) return QEDF_ERR_ARG;
  return fm_spectrum<float>(S, X, n, cnt, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_spectrum_f64(double* S, const double* X, int64_t n, double cnt, qedf_stream_t s) {
  if (!ok_ptrs(S, X) || n < 1 || !(cnt >= 0)) return QEDF_ERR_ARG;
  return fm_spectrum<double>(S, X, n, cnt, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_mass_f32(const float* S, float* sigma, int rows, int64_t len, const float* clamp_hi, double lambda,
                     double smin, double smax, double lmd, int invert, qedf_stream_t s) {
  if (!ok_ptrs(S, sigma) || !clamp_hi || rows < 1 || rows > 65535 || len < 1 || !(lambda > 0)) return QEDF_ERR_ARG;
  return fm_mass<float>(S, sigma, rows, len, clamp_hi, lambda, smin, smax, lmd, invert, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_mass_f64(const double* S, double* sigma, int rows, int64_t len, const double* clamp_hi, double lambda,
                     double smin, double smax, double lmd, int invert, qedf_stream_t s) {
  if (!ok_ptrs(S, sigma) || !clamp_hi || rows < 1 || rows > 65535 || len < 1 || !(lambda > 0)) return QEDF_ERR_ARG;
  return fm_mass<double>(S, sigma, rows, len, clamp_hi, lambda, smin, smax, lmd, invert,
                         reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_noise_f32(const float* a, const float* b, const float* sigma, float* z, int64_t n, int nk,
                      qedf_stream_t s) {
  if (!ok_ptrs(a, b) || !sigma || !z || n < 1 || nk < 1) return QEDF_ERR_ARG;
  return fm_noise<float>(a, b, sigma, z, n, nk, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_noise_f64(const double* a, const double* b, const double* sigma, double* z, int64_t n, int nk,
                      qedf_stream_t s) {
  if (!ok_ptrs(a, b) || !sigma || !z || n < 1 || nk < 1) return QEDF_ERR_ARG;
  return fm_noise<double>(a, b, sigma, z, n, nk, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_scale_f32(float* P, const float* sigma, int64_t n, qedf_stream_t s) {
  if (!ok_ptrs(P, sigma) || n < 1) return QEDF_ERR_ARG;
  return fm_scale<float>(P, sigma, n, reinterpret_cast<cudaStream_t>(s));
}
int qedf_fm_scale_f64(double* P, const double* sigma, int64_t n, qedf_stream_t s) {
  if (!ok_ptrs(P, sigma) || n < 1) return QEDF_ERR_ARG;
  return fm_scale<double>(P, sigma, n, reinterpret_cast<cudaStream_t>(s));
}

}  // extern "C"
