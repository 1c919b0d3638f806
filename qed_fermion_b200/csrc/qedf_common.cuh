// Common device helpers for the qed_fermion B200 kernels.
//
// Complex numbers are stored interleaved (re, im), the layout of torch
// complex64 / complex128, so vectors are passed as plain float / double
// pointers of twice the length.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/qedf.h"

namespace qedf {

// 8-byte (complex64) / 16-byte (complex128) alignment, so that one complex
// moves with one vector access
template <typename R>
struct alignas(2 * sizeof(R)) Cx {
  R re, im;
};

template <typename R>
__host__ __device__ __forceinline__ Cx<R> mk(R a, R b) {
  Cx<R> z;
  z.re = a;
  z.im = b;
  return z;
}
template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) { return mk<R>(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) { return mk<R>(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) { return mk<R>(s * a.re, s * a.im); }
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return mk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ Cx<R> cjmul(Cx<R> a, Cx<R> b) {
  return mk<R>(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
}
// a + m * b
template <typename R>
__device__ __forceinline__ Cx<R> cfma(Cx<R> m, Cx<R> b, Cx<R> a) {
  Cx<R> z;
  z.re = fma(m.re, b.re, fma(-m.im, b.im, a.re));
  z.im = fma(m.re, b.im, fma(m.im, b.re, a.im));
  return z;
}
// a + conj(m) * b
template <typename R>
__device__ __forceinline__ Cx<R> cjfma(Cx<R> m, Cx<R> b, Cx<R> a) {
  Cx<R> z;
  z.re = fma(m.re, b.re, fma(m.im, b.im, a.re));
  z.im = fma(m.re, b.im, fma(-m.im, b.re, a.im));
  return z;
}
template <typename R>
__device__ __forceinline__ Cx<R> cneg(Cx<R> a) { return mk<R>(-a.re, -a.im); }

// e^{i x} scaled by t.  Single precision: the argument is first reduced to
// [-pi, pi] (two-constant Cody-Waite reduction with 2*pi split into its
// float value and the remainder), then the hardware approximations
// __sinf/__cosf are used, whose maximum absolute error on [-pi, pi] is
// documented as 2^-21.41 (sin) and 2^-21.19 (cos).  The phase always enters
// multiplied by tanh(dtau/2) <= tanh(dtau), so its contribution to an
// operator application is below 1e-7 relative for dtau <= 0.1.
__device__ __forceinline__ Cx<float> tphase(float x, float t) {
  const float k = rintf(x * 0.15915494309189535f);
  float r = fmaf(-k, 6.28318548202514648f, x);
  r = fmaf(-k, -1.7484556000744487e-07f, r);
  float s, c;
  __sincosf(r, &s, &c);
  return mk<float>(t * c, t * s);
}
// Double precision: CUDA's sincos().
__device__ __forceinline__ Cx<double> tphase(double x, double t) {
  double s, c;
  sincos(x, &s, &c);
  return mk<double>(t * c, t * s);
}

// Vector loads/stores of two consecutive complex numbers (16 B for complex64,
// 32 B for complex128).  Addresses are 16-byte aligned by construction: the
// first site of each pair has an even x and L is even.
__device__ __forceinline__ void ld2(const float* p, Cx<float>& a, Cx<float>& b) {
  float4 q = __ldg(reinterpret_cast<const float4*>(p));
  a = mk<float>(q.x, q.y);
  b = mk<float>(q.z, q.w);
}
__device__ __forceinline__ void ld2(const double* p, Cx<double>& a, Cx<double>& b) {
  double2 q0 = __ldg(reinterpret_cast<const double2*>(p));
  double2 q1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
  a = mk<double>(q0.x, q0.y);
  b = mk<double>(q1.x, q1.y);
}
// plain (coherent) loads for buffers written earlier in the same kernel
__device__ __forceinline__ void ld2c(const float* p, Cx<float>& a, Cx<float>& b) {
  float4 q = *reinterpret_cast<const float4*>(p);
  a = mk<float>(q.x, q.y);
  b = mk<float>(q.z, q.w);
}
__device__ __forceinline__ void ld2c(const double* p, Cx<double>& a, Cx<double>& b) {
  double2 q0 = *reinterpret_cast<const double2*>(p);
  double2 q1 = *(reinterpret_cast<const double2*>(p) + 1);
  a = mk<double>(q0.x, q0.y);
  b = mk<double>(q1.x, q1.y);
}
__device__ __forceinline__ void st2(float* p, Cx<float> a, Cx<float> b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.re, a.im, b.re, b.im);
}
__device__ __forceinline__ void st2(double* p, Cx<double> a, Cx<double> b) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a.re, a.im);
  reinterpret_cast<double2*>(p)[1] = make_double2(b.re, b.im);
}
// Storage of single-precision iteration vectors: float (complex64) or bf16
// pairs (4 bytes per complex number, the PCG's BF16 storage option for its
// search direction and preconditioned residual).
// ld2s / st2s move two consecutive complex numbers (16 B as float, 8 B as
// bf16); arithmetic stays in float.  round_st returns the value the storage
// keeps (round to nearest even for bf16), so that values kept in registers
// equal the stored ones.
using bf16 = __nv_bfloat16;
__device__ __forceinline__ void ld2s(const float* p, Cx<float>& a, Cx<float>& b) { ld2c(p, a, b); }
__device__ __forceinline__ void ld2s(const bf16* p, Cx<float>& a, Cx<float>& b) {
  const uint2 q = *reinterpret_cast<const uint2*>(p);
  const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.x));
  const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.y));
  a = mk<float>(lo.x, lo.y);
  b = mk<float>(hi.x, hi.y);
}
__device__ __forceinline__ void ld2s(const double* p, Cx<double>& a, Cx<double>& b) { ld2c(p, a, b); }
__device__ __forceinline__ void st2s(float* p, Cx<float> a, Cx<float> b) { st2(p, a, b); }
__device__ __forceinline__ void st2s(double* p, Cx<double> a, Cx<double> b) { st2(p, a, b); }
__device__ __forceinline__ void st2s(bf16* p, Cx<float> a, Cx<float> b) {
  const __nv_bfloat162 lo = __floats2bfloat162_rn(a.re, a.im);
  const __nv_bfloat162 hi = __floats2bfloat162_rn(b.re, b.im);
  uint2 q;
  q.x = *reinterpret_cast<const unsigned*>(&lo);
  q.y = *reinterpret_cast<const unsigned*>(&hi);
  *reinterpret_cast<uint2*>(p) = q;
}
template <typename S, typename R>
__device__ __forceinline__ Cx<R> round_st(Cx<R> v) {
  if constexpr (std::is_same<S, bf16>::value) {
    const float2 f = __bfloat1622float2(__floats2bfloat162_rn(v.re, v.im));
    return mk<R>(f.x, f.y);
  } else {
    return v;
  }
}

// Scaled fp16 storage (the PCG's F16 option): a vector is kept as fp16 pairs
// of v / sc, with sc a power of two chosen per vector from its norm, so the
// stored values sit in fp16's range whatever the residual's size and keep its
// 11-bit significand.  Scaling by a power of two is exact, so sc * (stored)
// is exactly the value the registers hold after round_st.  The overloads for
// the other storage types ignore the scale.
__device__ __forceinline__ void ld2s(const __half* p, Cx<float>& a, Cx<float>& b, float sc) {
  const uint2 q = *reinterpret_cast<const uint2*>(p);
  const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  a = mk<float>(lo.x * sc, lo.y * sc);
  b = mk<float>(hi.x * sc, hi.y * sc);
}
__device__ __forceinline__ void st2s(__half* p, Cx<float> a, Cx<float> b, float inv) {
  const __half2 lo = __floats2half2_rn(a.re * inv, a.im * inv);
  const __half2 hi = __floats2half2_rn(b.re * inv, b.im * inv);
  uint2 q;
  q.x = *reinterpret_cast<const unsigned*>(&lo);
  q.y = *reinterpret_cast<const unsigned*>(&hi);
  *reinterpret_cast<uint2*>(p) = q;
}
template <typename S, typename R>
__device__ __forceinline__ void ld2s(const S* p, Cx<R>& a, Cx<R>& b, R) { ld2s(p, a, b); }
template <typename S, typename R>
__device__ __forceinline__ void st2s(S* p, Cx<R> a, Cx<R> b, R) { st2s(p, a, b); }
template <typename S, typename R>
__device__ __forceinline__ Cx<R> round_st(Cx<R> v, R sc, R inv) {
  if constexpr (std::is_same<S, __half>::value) {
    const float2 f = __half22float2(__floats2half2_rn(v.re * inv, v.im * inv));
    return mk<R>(f.x * sc, f.y * sc);
  } else {
    return round_st<S>(v);
  }
}
// the power-of-two scale of a vector with squared norm nn: about its norm
// / 1024, so entries of vectors of 10^3-10^7 sites stay well inside fp16's
// normal range; 1 for a zero or non-finite norm
__device__ __forceinline__ float st_scale(double nn) {
  if (!(nn > 0.0) || !isfinite(nn)) return 1.0f;
  int e;
  frexp(nn, &e);                         // nn in [2^(e-1), 2^e)
  int es = ((e - 1) >> 1) - 10;          // floor(log2 |v|) - 10
  es = es < -120 ? -120 : (es > 120 ? 120 : es);
  return ldexpf(1.0f, es);
}

// four reals (angles or forces of two sites, both components)
__device__ __forceinline__ void ld4(const float* p, float (&a)[4]) {
  float4 q = __ldg(reinterpret_cast<const float4*>(p));
  a[0] = q.x; a[1] = q.y; a[2] = q.z; a[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&a)[4]) {
  double2 q0 = __ldg(reinterpret_cast<const double2*>(p));
  double2 q1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
  a[0] = q0.x; a[1] = q0.y; a[2] = q1.x; a[3] = q1.y;
}
__device__ __forceinline__ void st4(float* p, const float (&a)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&a)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a[0], a[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(a[2], a[3]);
}

// Asynchronous 16-byte copies global -> shared, cached in L2 only (data that
// other SMs wrote before a grid barrier is seen).  Both addresses are 16-byte
// aligned.  cp_async_wait<N>: at most the N most recent groups still pending.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bulk copies global -> shared by the copy engine (cp.async.bulk, no tensor
// map, no multicast), completed on an mbarrier through its transaction count.
// Source and destination are 16-byte aligned and the size is a multiple of 16.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// one arrival that also announces `bytes` of copies to come
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// orders this thread's view of global memory (generic proxy, e.g. data other
// blocks wrote before a grid barrier) before its following bulk copies
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
__device__ __forceinline__ bool mbar_test_parity(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// wait for phase `parity` of the mbarrier to complete; false when `budget` SM
// cycles passed first (the wait is always bounded)
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long budget) {
  if (mbar_test_parity(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test_parity(bar, parity))
    if (clock64() - t0 > budget) return false;
  return true;
}

// Two shared-memory buffers of NARR whole slices each, filled by bulk copies
// that one thread issues; stage j of a sequence goes to buffer j % 2.  The
// caller guarantees that every thread finished reading stage j - 2 (a block
// barrier lies between) before stage j is issued.  `uses` counts the
// completed phases of each buffer's mbarrier, identically in every thread.
template <int NARR>
struct SliceStages {
  unsigned long long* bar;  // [2], static shared memory, initialised once per kernel
  unsigned char* buf;       // [2][NARR][bytes]
  unsigned bytes;           // slot stride: bytes of the widest slice array
  unsigned sizes[NARR];     // bytes copied into slot k (at most `bytes`)
  unsigned uses[2];

  __device__ void setup(unsigned long long* bars, unsigned char* buffers, unsigned slice_bytes) {
    bar = bars;
    buf = buffers;
    bytes = slice_bytes;
    for (int k = 0; k < NARR; ++k) sizes[k] = slice_bytes;
    uses[0] = uses[1] = 0;
  }
  // once per kernel, by every thread (contains a block barrier)
  __device__ static void init_barriers(unsigned long long* bars) {
    if (threadIdx.x == 0) {
      mbar_init(bars, 1);
      mbar_init(bars + 1, 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  __device__ __forceinline__ unsigned char* slot(int j, int k) const {
    return buf + ((size_t)(j & 1) * NARR + k) * bytes;
  }
  // thread 0 only: copy the arrays src[k] with bit k of `mask` into stage j
  __device__ void issue(int j, const void* const (&src)[NARR], unsigned mask) {
    unsigned n = 0;
#pragma unroll
    for (int k = 0; k < NARR; ++k)
      if ((mask >> k) & 1u) n += sizes[k];
    fence_proxy_async_global();
    mbar_arrive_expect_tx(bar + (j & 1), n);
#pragma unroll
    for (int k = 0; k < NARR; ++k)
      if ((mask >> k) & 1u) bulk_copy_g2s(slot(j, k), src[k], sizes[k], bar + (j & 1));
  }
  // every thread: wait for stage j; false if the bounded wait gave up
  __device__ bool wait(int j, long long budget) {
    const int b = j & 1;
    const bool ok = mbar_wait_bounded(bar + b, uses[b] & 1u, budget);
    ++uses[b];
    return ok;
  }
};

// Coefficients of the checkerboard factors F_g = c_g (I + t_g K_g):
// g1 uses cosh/tanh(dtau), g2..g4 cosh/tanh(dtau/2); Cb = c1 c2^2 c3^2 c4^2
// is the scalar that B = F4 F3 F2 F1 F2 F3 F4 carries in front of the
// product of the unscaled factors.
struct FactorCoeffs {
  double c1, ch, t1, th, Cb;
};

inline FactorCoeffs factor_coeffs(double dtau) {
  FactorCoeffs f;
  f.c1 = cosh(dtau);
  f.ch = cosh(dtau / 2);
  f.t1 = tanh(dtau);
  f.th = tanh(dtau / 2);
  f.Cb = f.c1 * f.ch * f.ch * f.ch * f.ch * f.ch * f.ch;
  return f;
}

}  // namespace qedf
