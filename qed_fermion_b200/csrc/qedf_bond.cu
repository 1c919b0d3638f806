// Bond-bond correlators of the stochastic estimator: the two passes around
// the 2-D FFTs of the pair-averaged correlation functions T1, T21, T2 and T4
// (stochastic_estimator.py: T1 :1393, T21 :1447, T2 :1504, T4 :1561).
//
// For every noise pair s < t and slice tau the reference forms two fields on
// the spatial slice, a_st(r) and b_st(r) (products of conj(eta), G_eta and
// e^{+-i phi_x}, some at r + x), and sums
//     ifft2(a_st) * fft2(b_st)
// over pairs and slices before one inverse transform gives the correlation
// in real space.  Here
//   qedf_bb_pair_fields  writes a_st and b_st of a chunk of pairs in one pass
//                        (the torch formulation needs a gather, a roll and a
//                        product per factor, each a pass over the chunk);
//   qedf_bb_kspace_acc   accumulates sum_rows A(k) B(k) in double precision
//                        from the two transforms (cuFFT, called by the host).
// Both are HBM-bound: 2 complex writes per pair-site and 2 complex reads per
// pair-site respectively; the inputs eta, G_eta of one slice are reread from
// L2 by every pair.
#include <algorithm>

#include "qedf_common.cuh"
#include "qedf_internal.h"

namespace qedf {

namespace {

struct BondArgs {
  int kind;  // 1: T1, 21: T21, 2: T2, 4: T4
  const void* eta;
  const void* g;
  const void* ep;  // e^{i phi_x} per site, [Ltau][Vs]
  const int* ps;
  const int* pt;
  int npairs, nrv, L, Nt;
  void* fa;
  void* fb;
};

template <typename R>
__device__ __forceinline__ Cx<R> ldcx(const R* base, int64_t i) {
  return *reinterpret_cast<const Cx<R>*>(base + 2 * i);
}
template <typename R>
__device__ __forceinline__ Cx<R> conjc(Cx<R> a) {
  return mk<R>(a.re, -a.im);
}

// grid (groups of BB_GROUP consecutive pairs, slices), the group index the
// fast grid dimension: the blocks in flight cover all pairs of a few slices,
// so each noise vector's values there come from DRAM once.  Within a block
// the pairs are the inner loop of each site: e^{i phi} is read once per
// site, and the first vector's values once per run of pairs that share it
// (in torch.combinations order most consecutive pairs do), which halves the
// L2 reads of T21 and T2.  Sites are walked without integer division.
constexpr int BB_GROUP = 4;

template <typename R>
__global__ void __launch_bounds__(256) k_bb_pair_fields(BondArgs a) {
  const int L = a.L, Vs = L * L;
  const int p0 = blockIdx.x * BB_GROUP, tau = blockIdx.y;
  const int np = min(BB_GROUP, a.npairs - p0);
  const int64_t nsite = (int64_t)a.Nt * Vs;
  const int64_t sl = (int64_t)tau * Vs;
  const R* eta = reinterpret_cast<const R*>(a.eta);
  const R* g = reinterpret_cast<const R*>(a.g);
  const R* epv = reinterpret_cast<const R*>(a.ep) + 2 * sl;
  const int dx = blockDim.x % L, dy = blockDim.x / L;
  int x = threadIdx.x % L, y = threadIdx.x / L;
  for (int q = threadIdx.x; q < Vs; q += blockDim.x) {
    const int r = q, r1 = y * L + (x + 1 == L ? 0 : x + 1);
    const Cx<R> ep = ldcx(epv, r);
    const Cx<R> em = conjc(ep);
    int s_prev = -1;
    Cx<R> ecs = mk<R>(0, 0), ecs1 = ecs, gs = ecs, gs1 = ecs;
    for (int k = 0; k < np; ++k) {
      const int p = p0 + k;
      const int s = a.ps[p], t = a.pt[p];
      Cx<R>* fa = reinterpret_cast<Cx<R>*>(a.fa) + (int64_t)p * nsite + sl;
      Cx<R>* fb = reinterpret_cast<Cx<R>*>(a.fb) + (int64_t)p * nsite + sl;
      if ((unsigned)s >= (unsigned)a.nrv || (unsigned)t >= (unsigned)a.nrv) {  // not a noise vector: zero
        fa[q] = mk<R>(0, 0);
        fb[q] = mk<R>(0, 0);
        continue;
      }
      const int64_t os = (int64_t)s * nsite + sl, ot = (int64_t)t * nsite + sl;
      if (s != s_prev) {  // the first vector's values at r and r + x
        ecs = conjc(ldcx(eta, os + r));
        ecs1 = conjc(ldcx(eta, os + r1));
        gs = ldcx(g, os + r);
        gs1 = ldcx(g, os + r1);
        s_prev = s;
      }
      Cx<R> A, B;
      if (a.kind == 1) {
        // a = ec_s g_t(r+x) e,  b = g_s(r+x) ec_t e
        A = cmul(cmul(ecs, ldcx(g, ot + r1)), ep);
        B = cmul(cmul(gs1, conjc(ldcx(eta, ot + r))), ep);
      } else if (a.kind == 4) {
        // a = ec_s(r+x) g_t e*,  b = g_s ec_t(r+x) e*
        A = cmul(cmul(ecs1, ldcx(g, ot + r)), em);
        B = cmul(cmul(gs, conjc(ldcx(eta, ot + r1))), em);
      } else {
        const Cx<R> ect = conjc(ldcx(eta, ot + r)), ect1 = conjc(ldcx(eta, ot + r1));
        const Cx<R> gt = ldcx(g, ot + r), gt1 = ldcx(g, ot + r1);
        const R h = (R)0.5;
        if (a.kind == 21) {
          // a = (ec_s(r+x) g_t + ec_t(r+x) g_s) e* / 2,  b = (g_s(r+x) ec_t + g_t(r+x) ec_s) e / 2
          A = h * cmul(cmul(ecs1, gt) + cmul(ect1, gs), em);
          B = h * cmul(cmul(gs1, ect) + cmul(gt1, ecs), ep);
        } else {
          // T2: a = (ec_s g_t(r+x) + ec_t g_s(r+x)) e / 2,  b = (g_s ec_t(r+x) + g_t ec_s(r+x)) e* / 2
          A = h * cmul(cmul(ecs, gt1) + cmul(ect, gs1), ep);
          B = h * cmul(cmul(gs, ect1) + cmul(gt, ecs1), em);
        }
      }
      fa[q] = A;
      fb[q] = B;
    }
    x += dx;
    y += dy;
    if (x >= L) {
      x -= L;
      ++y;
    }
  }
}

// S[k] += sum_i A[i][k] B[i][k] over n rows of Vs columns, in double.
// Block (32 columns) x (8 row lanes); the row lanes are summed in shared
// memory and each block adds its column sums with two atomics per column.
template <typename R>
__global__ void __launch_bounds__(256) k_bb_kspace_acc(const R* A, const R* B, int64_t n, int Vs, double* S) {
  __shared__ double red[2][8][33];
  const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
  const int k = blockIdx.x * 32 + cx;
  double sr = 0, si = 0;
  if (k < Vs) {
    for (int64_t i = (int64_t)blockIdx.y * 8 + ry; i < n; i += (int64_t)gridDim.y * 8) {
      const Cx<R> u = ldcx(A, i * Vs + k), v = ldcx(B, i * Vs + k);
      const double ur = u.re, ui = u.im, vr = v.re, vi = v.im;
      sr = fma(ur, vr, fma(-ui, vi, sr));
      si = fma(ur, vi, fma(ui, vr, si));
    }
  }
  red[0][ry][cx] = sr;
  red[1][ry][cx] = si;
  __syncthreads();
  if (ry == 0 && k < Vs) {
    double tr = 0, ti = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      tr += red[0][q][cx];
      ti += red[1][q][cx];
    }
    atomicAdd(S + 2 * k, tr);
    atomicAdd(S + 2 * k + 1, ti);
  }
}

// Tvv's current field of each noise vector s (stochastic_estimator.py:1612-1652),
//   v_s(r) = g_s(r+x) conj(eta_s(r)) e^{i phi_x(r)} + g_s(r) conj(eta_s(r+x)) e^{-i phi_x(r)},
// written for every slice, and its sum over vectors and slices per site,
// added to Tv[Vs] (complex, double).  Grid (site blocks, vectors, slice
// ranges): a thread walks its site through one range of slices, so the sum
// needs one atomic per site, vector and range; the ranges give the grid
// enough blocks to fill the SMs when Vs x Nrv alone does not.
template <typename R>
__global__ void __launch_bounds__(256) k_bb_vfield(const R* eta, const R* g, const R* ep, int L, int Nt, int tlen,
                                                   R* v, double* Tv) {
  const int Vs = L * L;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  const int t0 = blockIdx.z * tlen, t1 = min(t0 + tlen, Nt);
  if (r >= Vs) return;
  const int x = r % L, y = r / L;
  const int r1 = y * L + (x + 1 == L ? 0 : x + 1);
  const int64_t base = (int64_t)s * Nt * Vs;
  double sr = 0, si = 0;
  for (int t = t0; t < t1; ++t) {
    const int64_t o = base + (int64_t)t * Vs;
    const Cx<R> e = ldcx(ep, (int64_t)t * Vs + r);
    const Cx<R> val = cmul(cmul(ldcx(g, o + r1), conjc(ldcx(eta, o + r))), e) +
                      cmul(cmul(ldcx(g, o + r), conjc(ldcx(eta, o + r1))), conjc(e));
    *reinterpret_cast<Cx<R>*>(v + 2 * (o + r)) = val;
    sr += (double)val.re;
    si += (double)val.im;
  }
  if (t1 > t0) {
    atomicAdd(Tv + 2 * r, sr);
    atomicAdd(Tv + 2 * r + 1, si);
  }
}

// The short-distance terms the correlators add to their pair sums, summed
// over vectors, slices and sites into D[3] (complex, double):
//   D[0] = sum g_s(r+x) conj(eta_s(r-x)) e^{i phi_x(r)} e^{i phi_x(r-x)}     (T1, at d = -x)
//   D[1] = sum g_s(r) conj(eta_s(r))                                         (T21 and T2, at d = 0)
//   D[2] = sum g_s(r) conj(eta_s(r+2x)) e^{-i phi_x(r)} e^{-i phi_x(r+x)}   (T4, at d = +x)
// Blocks take (vector, slice) rows in turn (grid y), one thread per site of a
// row (grid x), so no thread divides a 64-bit index.
template <typename R>
__global__ void __launch_bounds__(256) k_bb_diag(const R* eta, const R* g, const R* ep, int Nrv, int L, int Nt,
                                                 double* D) {
  __shared__ double red[6][8];
  const int Vs = L * L;
  const int rows = Nrv * Nt;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  // one site per thread (the grid's x extent covers a row); rows in turn,
  // four in flight
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < Vs) {
    const int x = r % L, y = r / L;
    const int xm = x == 0 ? L - 1 : x - 1, xp = x + 1 == L ? 0 : x + 1, xpp = xp + 1 == L ? 0 : xp + 1;
    const int rm = y * L + xm, rp = y * L + xp, rpp = y * L + xpp;
#pragma unroll 4
    for (int q = blockIdx.y; q < rows; q += gridDim.y) {
      const int64_t st = (int64_t)q * Vs;               // (vector, slice) offset
      const int64_t et = (int64_t)(q % Nt) * Vs;
      const Cx<R> e = ldcx(ep, et + r), em1 = ldcx(ep, et + rm), ep1 = ldcx(ep, et + rp);
      const Cx<R> gr = ldcx(g, st + r);
      const Cx<R> d0 = cmul(cmul(ldcx(g, st + rp), conjc(ldcx(eta, st + rm))), cmul(e, em1));
      const Cx<R> d1 = cmul(gr, conjc(ldcx(eta, st + r)));
      const Cx<R> d2 = cmul(cmul(gr, conjc(ldcx(eta, st + rpp))), conjc(cmul(e, ep1)));
      acc[0] += d0.re;
      acc[1] += d0.im;
      acc[2] += d1.re;
      acc[3] += d1.im;
      acc[4] += d2.re;
      acc[5] += d2.im;
    }
  }
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (ln == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += red[threadIdx.x][q];
    atomicAdd(D + threadIdx.x, v);
  }
}

template <typename R>
int vfield_entry(const R* eta, const R* g, const R* ep, int Nrv, int Lx, int Ltau, R* v, double* Tv,
                 cudaStream_t st) {
  if (!eta || !g || !ep || !v || !Tv || Nrv < 1 || Nrv > 65535 || Lx < 2 || Ltau < 1) return QEDF_ERR_ARG;
  const int Vs = Lx * Lx;
  // split the slices so that the grid holds about four blocks per SM
  const int64_t base_blocks = (int64_t)((Vs + 255) / 256) * Nrv;
  const int64_t want = (int64_t)num_sms() * 4;
  const int64_t split = std::max<int64_t>(1, (want + base_blocks - 1) / base_blocks);
  const int nsplit = (int)std::min<int64_t>(std::min<int64_t>(Ltau, 65535), split);
  const int tlen = (Ltau + nsplit - 1) / nsplit;
  const int nz = (Ltau + tlen - 1) / tlen;
  k_bb_vfield<R><<<dim3((Vs + 255) / 256, Nrv, nz), 256, 0, st>>>(eta, g, ep, Lx, Ltau, tlen, v, Tv);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

template <typename R>
int diag_entry(const R* eta, const R* g, const R* ep, int Nrv, int Lx, int Ltau, double* D, cudaStream_t st) {
  if (!eta || !g || !ep || !D || Nrv < 1 || Lx < 3 || Ltau < 1) return QEDF_ERR_ARG;
  const int Vs = Lx * Lx;
  if ((Vs + 255) / 256 > 65535) return QEDF_ERR_SIZE;
  const int gx = (Vs + 255) / 256;  // one thread per site of a row
  const int64_t rows = (int64_t)Nrv * Ltau;
  if (rows > INT32_MAX) return QEDF_ERR_SIZE;
  const int gy = (int)std::min<int64_t>(rows, std::max(1, num_sms() * 4 / gx));
  k_bb_diag<R><<<dim3(gx, std::min(gy, 65535)), 256, 0, st>>>(eta, g, ep, Nrv, Lx, Ltau, D);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

// ----------------------------------------------------------------------------
// One pass for a whole correlator: per (pair, slice) the two fields, their 2-D
// transforms and the product, all in shared memory (the fields never reach
// HBM).  A(k) = sum_r a(r) e^{+2 pi i k.r / L} and B(k) = sum_r b(r)
// e^{-2 pi i k.r / L} (the unnormalised transforms the two-pass path takes
// from cuFFT) are formed in place, rows then columns, each line of length
// L = p q by the two-factor Cooley-Tukey split
//   X[q k1 + k2] = sum_{n1<p} w_p^{n1 k1} w_L^{n1 k2} sum_{n2<q} x[n1 + p n2] w_q^{n2 k2}
// (w_m = e^{-+2 pi i / m}); every thread takes whole sub-transforms, with its
// q (or p) inputs in registers.  Each block adds A(k) B(k) of its items in
// double precision in shared memory and, at its end, into S.
// ----------------------------------------------------------------------------
constexpr int BB_QMAX = 8;  // largest factor of L the kernel is compiled for

// both fields of correlator `kind` for pair (s, t) at site r of slice tau
template <typename R>
__device__ __forceinline__ void pair_ab(int kind, const R* eta, const R* g, Cx<R> ep, int64_t os, int64_t ot, int r,
                                        int r1, Cx<R>& A, Cx<R>& B) {
  const Cx<R> em = conjc(ep);
  const Cx<R> ecs = conjc(ldcx(eta, os + r)), ecs1 = conjc(ldcx(eta, os + r1));
  const Cx<R> gs = ldcx(g, os + r), gs1 = ldcx(g, os + r1);
  if (kind == 1) {
    A = cmul(cmul(ecs, ldcx(g, ot + r1)), ep);
    B = cmul(cmul(gs1, conjc(ldcx(eta, ot + r))), ep);
  } else if (kind == 4) {
    A = cmul(cmul(ecs1, ldcx(g, ot + r)), em);
    B = cmul(cmul(gs, conjc(ldcx(eta, ot + r1))), em);
  } else {
    const Cx<R> ect = conjc(ldcx(eta, ot + r)), ect1 = conjc(ldcx(eta, ot + r1));
    const Cx<R> gt = ldcx(g, ot + r), gt1 = ldcx(g, ot + r1);
    const R h = (R)0.5;
    if (kind == 21) {
      A = h * cmul(cmul(ecs1, gt) + cmul(ect1, gs), em);
      B = h * cmul(cmul(gs1, ect) + cmul(gt1, ecs), ep);
    } else {
      A = h * cmul(cmul(ecs, gt1) + cmul(ect, gs1), ep);
      B = h * cmul(cmul(gs, ect1) + cmul(gt, ecs1), em);
    }
  }
}

// smem twiddle tables (forward sign e^{-2 pi i ...}); sign +1 uses conjugates
template <typename R>
__device__ __forceinline__ Cx<R> tw(const Cx<R>* t, int i, int sgn) {
  const Cx<R> w = t[i];
  return sgn > 0 ? conjc(w) : w;
}

// stage 1 of the transform of `nl` lines of field f (line l, element at
// base(l) + stride * position): T[line][n1 q + k2] = sum_{n2} x[n1 + p n2] wq^{n2 k2}
template <typename R>
__device__ __forceinline__ void dft_stage1(const Cx<R>* X, Cx<R>* T, int L, int p, int q, int line_stride,
                                           int pos_stride, int item_line, int n1, const Cx<R>* wq, int sgn) {
  Cx<R> xin[BB_QMAX];
#pragma unroll
  for (int n2 = 0; n2 < BB_QMAX; ++n2)
    if (n2 < q) xin[n2] = X[item_line * line_stride + (n1 + p * n2) * pos_stride];
  for (int k2 = 0; k2 < q; ++k2) {
    Cx<R> acc = mk<R>(0, 0);
#pragma unroll
    for (int n2 = 0; n2 < BB_QMAX; ++n2)
      if (n2 < q) acc = cfma(tw(wq, n2 * q + k2, sgn), xin[n2], acc);
    T[item_line * line_stride + (n1 * q + k2) * pos_stride] = acc;
  }
}

// stage 2: X[q k1 + k2] = sum_{n1} wp^{n1 k1} (wL^{n1 k2} T[n1 q + k2])
template <typename R>
__device__ __forceinline__ void dft_stage2(Cx<R>* X, const Cx<R>* T, int L, int p, int q, int line_stride,
                                           int pos_stride, int item_line, int k2, const Cx<R>* wp,
                                           const Cx<R>* wl, int sgn) {
  Cx<R> tin[BB_QMAX];
#pragma unroll
  for (int n1 = 0; n1 < BB_QMAX; ++n1)
    if (n1 < p) tin[n1] = cmul(tw(wl, n1 * q + k2, sgn), T[item_line * line_stride + (n1 * q + k2) * pos_stride]);
  for (int k1 = 0; k1 < p; ++k1) {
    Cx<R> acc = mk<R>(0, 0);
#pragma unroll
    for (int n1 = 0; n1 < BB_QMAX; ++n1)
      if (n1 < p) acc = cfma(tw(wp, n1 * p + k1, sgn), tin[n1], acc);
    X[item_line * line_stride + (q * k1 + k2) * pos_stride] = acc;
  }
}

template <typename R>
size_t corr_smem_bytes(int L, int p, int q) {
  const size_t Vs = (size_t)L * L;
  return 4 * Vs * sizeof(Cx<R>) + 2 * Vs * sizeof(double) + (size_t)(q * q + p * p + p * q) * sizeof(Cx<R>);
}

template <typename R>
__global__ void __launch_bounds__(256) k_bb_corr(BondArgs a, int p, int q, double* S) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int L = a.L, Vs = L * L, tid = threadIdx.x, nt = blockDim.x;
  Cx<R>* F = reinterpret_cast<Cx<R>*>(smraw);  // [2][Vs]: a, b
  Cx<R>* T = F + 2 * Vs;                        // [2][Vs]: stage temporaries
  double* P = reinterpret_cast<double*>(T + 2 * Vs);  // [Vs] complex sum
  Cx<R>* wq = reinterpret_cast<Cx<R>*>(P + 2 * Vs);
  Cx<R>* wp = wq + q * q;
  Cx<R>* wl = wp + p * p;
  for (int i = tid; i < q * q; i += nt) {
    double sn, cs;
    sincospi(-2.0 * ((i / q) * (i % q) % q) / q, &sn, &cs);
    wq[i] = mk<R>((R)cs, (R)sn);
  }
  for (int i = tid; i < p * p; i += nt) {
    double sn, cs;
    sincospi(-2.0 * ((i / p) * (i % p) % p) / p, &sn, &cs);
    wp[i] = mk<R>((R)cs, (R)sn);
  }
  for (int i = tid; i < p * q; i += nt) {
    double sn, cs;
    sincospi(-2.0 * ((i / q) * (i % q) % L) / L, &sn, &cs);
    wl[i] = mk<R>((R)cs, (R)sn);
  }
  for (int i = tid; i < 2 * Vs; i += nt) P[i] = 0.0;
  __syncthreads();
  const R* eta = reinterpret_cast<const R*>(a.eta);
  const R* g = reinterpret_cast<const R*>(a.g);
  const R* epv = reinterpret_cast<const R*>(a.ep);
  const int64_t nsite = (int64_t)a.Nt * Vs;
  const int64_t items = (int64_t)a.npairs * a.Nt;
  for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
    // slice-major order: blocks in flight share their slice's vectors in L2
    const int tau = (int)(w / a.npairs), pr = (int)(w % a.npairs);
    const int s = a.ps[pr], t = a.pt[pr];
    const bool valid = (unsigned)s < (unsigned)a.nrv && (unsigned)t < (unsigned)a.nrv;
    const int64_t sl = (int64_t)tau * Vs, os = (int64_t)s * nsite + sl, ot = (int64_t)t * nsite + sl;
    for (int r = tid; r < Vs; r += nt) {
      const int x = r % L, y = r - x;
      const int r1 = y + (x + 1 == L ? 0 : x + 1);
      Cx<R> A = mk<R>(0, 0), B = mk<R>(0, 0);
      if (valid) pair_ab<R>(a.kind, eta, g, ldcx(epv, sl + r), os, ot, r, r1, A, B);
      F[r] = A;
      F[Vs + r] = B;
    }
    __syncthreads();
    // rows (lines y, positions x): A with sign +1, B with sign -1
    for (int i = tid; i < 2 * L * p; i += nt) {
      const int f = i / (L * p), rem = i % (L * p);
      dft_stage1<R>(F + f * Vs, T + f * Vs, L, p, q, L, 1, rem / p, rem % p, wq, f == 0 ? 1 : -1);
    }
    __syncthreads();
    for (int i = tid; i < 2 * L * q; i += nt) {
      const int f = i / (L * q), rem = i % (L * q);
      dft_stage2<R>(F + f * Vs, T + f * Vs, L, p, q, L, 1, rem / q, rem % q, wp, wl, f == 0 ? 1 : -1);
    }
    __syncthreads();
    // columns (lines x, positions y); x fastest over the threads
    for (int i = tid; i < 2 * L * p; i += nt) {
      const int f = i / (L * p), rem = i % (L * p);
      dft_stage1<R>(F + f * Vs, T + f * Vs, L, p, q, 1, L, rem % L, rem / L, wq, f == 0 ? 1 : -1);
    }
    __syncthreads();
    for (int i = tid; i < 2 * L * q; i += nt) {
      const int f = i / (L * q), rem = i % (L * q);
      dft_stage2<R>(F + f * Vs, T + f * Vs, L, p, q, 1, L, rem % L, rem / L, wp, wl, f == 0 ? 1 : -1);
    }
    __syncthreads();
    for (int k = tid; k < Vs; k += nt) {
      const Cx<R> u = F[k], v = F[Vs + k];
      const double ur = u.re, ui = u.im, vr = v.re, vi = v.im;
      P[2 * k] = fma(ur, vr, fma(-ui, vi, P[2 * k]));
      P[2 * k + 1] = fma(ur, vi, fma(ui, vr, P[2 * k + 1]));
    }
    __syncthreads();
  }
  for (int k = tid; k < Vs; k += nt) {
    atomicAdd(S + 2 * k, P[2 * k]);
    atomicAdd(S + 2 * k + 1, P[2 * k + 1]);
  }
}

// the factor split L = p q with q <= BB_QMAX and p as large as possible (p <= q)
inline bool corr_factors(int L, int& p, int& q) {
  p = 0;
  for (int d = 1; d * d <= L; ++d)
    if (L % d == 0 && L / d <= BB_QMAX) p = d;
  if (!p) return false;
  q = L / p;
  return true;
}

template <typename R>
int corr_entry(int kind, const R* eta, const R* g, const R* ep, const int* ps, const int* pt, int npairs, int Nrv,
               int Lx, int Ltau, double* S, cudaStream_t st) {
  if (kind != 1 && kind != 21 && kind != 2 && kind != 4) return QEDF_ERR_ARG;
  if (!eta || !g || !ep || !ps || !pt || !S) return QEDF_ERR_ARG;
  if (npairs < 0 || Lx < 2 || Ltau < 1 || Nrv < 2) return QEDF_ERR_ARG;
  int p, q;
  if (!corr_factors(Lx, p, q)) return QEDF_ERR_SIZE;
  const size_t smem = corr_smem_bytes<R>(Lx, p, q);
  if (smem > 227 * 1024) return QEDF_ERR_SIZE;
  if (npairs == 0) return QEDF_OK;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_bb_corr<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return QEDF_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bb_corr<R>, 256, smem) != cudaSuccess || per_sm < 1)
    return QEDF_ERR_SIZE;
  BondArgs a;
  a.kind = kind;
  a.eta = eta;
  a.g = g;
  a.ep = ep;
  a.ps = ps;
  a.pt = pt;
  a.npairs = npairs;
  a.nrv = Nrv;
  a.L = Lx;
  a.Nt = Ltau;
  a.fa = nullptr;
  a.fb = nullptr;
  const int64_t items = (int64_t)npairs * Ltau;
  const int blocks = (int)std::min<int64_t>(items, (int64_t)num_sms() * per_sm);
  k_bb_corr<R><<<blocks, 256, smem, st>>>(a, p, q, S);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

template <typename R>
int pair_fields_entry(int kind, const R* eta, const R* g, const R* ep, const int* ps, const int* pt, int npairs,
                      int Nrv, int Lx, int Ltau, R* fa, R* fb, cudaStream_t st) {
  if (kind != 1 && kind != 21 && kind != 2 && kind != 4) return QEDF_ERR_ARG;
  if (!eta || !g || !ep || !ps || !pt || !fa || !fb) return QEDF_ERR_ARG;
  if (npairs < 0 || npairs > 65535 || Lx < 1 || Ltau < 1 || Ltau > 65535 || Nrv < 2) return QEDF_ERR_ARG;
  if (npairs == 0) return QEDF_OK;
  BondArgs a;
  a.kind = kind;
  a.eta = eta;
  a.g = g;
  a.ep = ep;
  a.ps = ps;
  a.pt = pt;
  a.npairs = npairs;
  a.nrv = Nrv;
  a.L = Lx;
  a.Nt = Ltau;
  a.fa = fa;
  a.fb = fb;
  dim3 grid((npairs + BB_GROUP - 1) / BB_GROUP, Ltau);
  k_bb_pair_fields<R><<<grid, 256, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

template <typename R>
int kspace_acc_entry(const R* A, const R* B, int64_t rows, int Vs, double* S, cudaStream_t st) {
  if (!A || !B || !S || rows < 0 || Vs < 1) return QEDF_ERR_ARG;
  if (rows == 0) return QEDF_OK;
  const int bx = (Vs + 31) / 32;
  const int64_t want = std::max<int64_t>(1, (int64_t)num_sms() * 8 / bx);
  const int by = (int)std::min<int64_t>(std::min<int64_t>(want, (rows + 7) / 8), 65535);
  k_bb_kspace_acc<R><<<dim3(bx, by), 256, 0, st>>>(A, B, rows, Vs, S);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

}  // namespace
}  // namespace qedf

using namespace qedf;

extern "C" {

int qedf_bb_pair_fields_c64(int kind, const float* eta, const float* g_eta, const float* ephase, const int* ps,
                            const int* pt, int npairs, int Nrv, int Lx, int Ltau, float* fa, float* fb,
                            qedf_stream_t s) {
  return pair_fields_entry<float>(kind, eta, g_eta, ephase, ps, pt, npairs, Nrv, Lx, Ltau, fa, fb,
                                  reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_pair_fields_c128(int kind, const double* eta, const double* g_eta, const double* ephase,
                             const int* ps, const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* fa,
                             double* fb, qedf_stream_t s) {
  return pair_fields_entry<double>(kind, eta, g_eta, ephase, ps, pt, npairs, Nrv, Lx, Ltau, fa, fb,
                                   reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_kspace_acc_c64(const float* A, const float* B, int64_t rows, int Vs, double* S, qedf_stream_t s) {
  return kspace_acc_entry<float>(A, B, rows, Vs, S, reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_kspace_acc_c128(const double* A, const double* B, int64_t rows, int Vs, double* S,
                            qedf_stream_t s) {
  return kspace_acc_entry<double>(A, B, rows, Vs, S, reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_corr_c64(int kind, const float* eta, const float* g_eta, const float* ephase, const int* ps,
                     const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* S, qedf_stream_t s) {
  return corr_entry<float>(kind, eta, g_eta, ephase, ps, pt, npairs, Nrv, Lx, Ltau, S,
                           reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_corr_c128(int kind, const double* eta, const double* g_eta, const double* ephase, const int* ps,
                      const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* S, qedf_stream_t s) {
  return corr_entry<double>(kind, eta, g_eta, ephase, ps, pt, npairs, Nrv, Lx, Ltau, S,
                            reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_vfield_c64(const float* eta, const float* g_eta, const float* ephase, int Nrv, int Lx, int Ltau,
                       float* v, double* Tv, qedf_stream_t s) {
  return vfield_entry<float>(eta, g_eta, ephase, Nrv, Lx, Ltau, v, Tv, reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_vfield_c128(const double* eta, const double* g_eta, const double* ephase, int Nrv, int Lx, int Ltau,
                        double* v, double* Tv, qedf_stream_t s) {
  return vfield_entry<double>(eta, g_eta, ephase, Nrv, Lx, Ltau, v, Tv, reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_diag_c64(const float* eta, const float* g_eta, const float* ephase, int Nrv, int Lx, int Ltau,
                     double* D, qedf_stream_t s) {
  return diag_entry<float>(eta, g_eta, ephase, Nrv, Lx, Ltau, D, reinterpret_cast<cudaStream_t>(s));
}
int qedf_bb_diag_c128(const double* eta, const double* g_eta, const double* ephase, int Nrv, int Lx, int Ltau,
                      double* D, qedf_stream_t s) {
  return diag_entry<double>(eta, g_eta, ephase, Nrv, Lx, Ltau, D, reinterpret_cast<cudaStream_t>(s));
}

}  // extern "C"
