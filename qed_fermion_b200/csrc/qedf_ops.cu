// Operator, preconditioner, force, boson and reduction kernels of the
// qed_fermion B200 library, plus their host launchers.
//
// Layouts (all contiguous):
//   vectors  [nvec][Nt][L][L]    complex (re, im interleaved)
//   angles   [nphi][Nt][L][L][2] real, component 0 = x-bond, 1 = y-bond
//   forces   same as angles
#include <algorithm>
#include <cstdio>

#include "qedf_internal.h"
#include "qedf_slice.cuh"

namespace qedf {

// ============================================================================
// M, M^dagger, M^dagger M over tau-slabs
// ============================================================================
//
// One thread block handles one right-hand side and one slab [a, b) of output
// slices.  With x_t the slices of the input and sigma_t = +1 (t < Nt-1) or -1
// (t = Nt-1):
//   (M x)_t      = x_t - sigma_{t-1} B_{t-1} x_{t-1}
//   (M^dag y)_t  = y_t - sigma_t B_t y_{t+1}
//   (M^dag M x)_t: y = M x is produced slice by slice in registers and M^dag
//                  applied to it, so x is read once and one extra slice of y
//                  (the slab's lower halo) is recomputed.
template <typename R, typename A, int BY, int OP, int EC>
__global__ void __launch_bounds__(MaxT<BY, EC>::value, MaxT<BY, EC>::min_blocks) k_operator(OpArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr bool PHS = (EC & EC_PHS) != 0;
  constexpr bool STASH = (EC & EC_NOSTASH) == 0;
  constexpr bool XS = (EC & EC_XS) != 0;
  constexpr int LT = ec_fixed_l(EC);
  Slice<R, BY, PHS, XS, LT> S;
  const int L = lattice_l<EC>(p.L);
  S.init(L, smem, 2, (R)p.c1, (R)p.ch, threadIdx.x);
  const int Vs = L * L;
  const size_t sv = 2 * (size_t)Vs;  // reals per slice (vector and angles)
  const int rb = blockIdx.y;
  const int a = blockIdx.x * p.T;
  const int b = min(a + p.T, p.Nt);
  const A* phi = reinterpret_cast<const A*>(p.phi) + (size_t)(rb / p.rhs_per_phi) * p.Nt * sv;
  const R* x = reinterpret_cast<const R*>(p.x) + (size_t)rb * p.Nt * sv;
  R* z = reinterpret_cast<R*>(p.z) + (size_t)rb * p.Nt * sv;
  const R t1 = (R)p.t1, th = (R)p.th, Cb = (R)p.Cb;
  const int Nt = p.Nt;
  // Three blocks live in registers; y_t waits in the thread-private stash
  // (or in a fourth register block when there is no stash).
  Cx<R> X0[BY][2], X1[BY][2], Y[BY][2];
  Cx<R> Yp[STASH ? 1 : BY][2];

  if (OP == OP_M) {
    int tp = (a - 1 + Nt) % Nt;
    if (S.on) S.load(X0, x + tp * sv);
    for (int t = a; t < b; ++t) {
      if (S.on) S.load(X1, x + t * sv);
      S.phases(phi + tp * sv, t1, th);
      S.template applyB<FAC_TILDE>(X0);
      if (S.on) {
        axpy_blk<R, BY>(Y, X1, sigma_of<R>(tp, Nt) * Cb, X0);
        S.store(z + t * sv, Y);
      }
      copy_blk<R, BY>(X0, X1);
      tp = t;
    }
  } else if (OP == OP_MH) {
    if (S.on) S.load(X0, x + a * sv);
    for (int t = a; t < b; ++t) {
      const int tn = (t + 1) % Nt;
      if (S.on) S.load(X1, x + tn * sv);
      S.phases(phi + t * sv, t1, th);
      copy_blk<R, BY>(Y, X1);
      S.template applyB<FAC_TILDE>(Y);
      if (S.on) {
        axpy_blk<R, BY>(Y, X0, sigma_of<R>(t, Nt) * Cb, Y);
        S.store(z + t * sv, Y);
      }
      copy_blk<R, BY>(X0, X1);
    }
  } else {  // OP_MHM
    // prologue: y_a = x_a - sigma_{a-1} B_{a-1} x_{a-1}
    const int tp = (a - 1 + Nt) % Nt;
    if (S.on) {
      S.load(X0, x + tp * sv);
      S.load(X1, x + a * sv);
    }
    A ang[BY][4];
    if constexpr (!PHS) S.load_angles(ang, phi + a * sv);
    S.phases(phi + tp * sv, t1, th);
    S.template applyB<FAC_TILDE>(X0);
    axpy_blk<R, BY>(Y, X1, sigma_of<R>(tp, Nt) * Cb, X0);
    if constexpr (STASH) S.park(Y); else copy_blk<R, BY>(Yp, Y);
    copy_blk<R, BY>(X0, X1);
    for (int t = a; t < b; ++t) {
      const int tn = (t + 1) % Nt;
      if (S.on) S.load(X1, x + tn * sv);
      if constexpr (!PHS) {
        // phases of slice t from angles fetched one slice ahead
        S.phases_from(ang, t1, th);
        if (t + 1 < b) S.load_angles(ang, phi + (t + 1) * sv);
      } else {
        S.phases(phi + t * sv, t1, th);
      }
      const R sg = sigma_of<R>(t, Nt) * Cb;
      S.template applyB<FAC_TILDE>(X0);          // B_t x_t
      axpy_blk<R, BY>(Y, X1, sg, X0);             // y_{t+1}
      if constexpr (STASH) {
        S.unpark(X0);                             // y_t
        S.park(Y);
      } else {
        copy_blk<R, BY>(X0, Yp);
        copy_blk<R, BY>(Yp, Y);
      }
      S.template applyB<FAC_TILDE, 1>(Y);         // B_t y_{t+1}
      if (S.on) {
        axpy_blk<R, BY>(Y, X0, sg, Y);            // z_t = y_t - sigma_t B_t y_{t+1}
        S.store(z + t * sv, Y);
      }
      copy_blk<R, BY>(X0, X1);
    }
  }
}

// ============================================================================
// b_vec_per_tau: B_t v or its six partial products, one slice
// ============================================================================
template <typename R, typename A, int BY, bool PHS>
__global__ void __launch_bounds__(MaxThreads<BY>::value, 1) k_bvec(BvecArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  Slice<R, BY, PHS> S;
  S.init(p.L, smem, 2, (R)p.c1, (R)p.ch, threadIdx.x);
  const size_t sv = 2 * (size_t)p.L * p.L;
  const A* phi = reinterpret_cast<const A*>(p.phi);
  const R* v = reinterpret_cast<const R*>(p.v) + blockIdx.x * sv;
  R* out = reinterpret_cast<R*>(p.out) + blockIdx.x * sv * (p.interm ? 6 : 1);
  Cx<R> W[BY][2];
  if (S.on) S.load(W, v);
  S.phases(phi, (R)p.t1, (R)p.th);
  S.template factor<3, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 0 * sv, W);
  S.template factor<2, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 1 * sv, W);
  S.template factor<1, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 2 * sv, W);
  S.template factor<0, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 3 * sv, W);
  S.template factor<1, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 4 * sv, W);
  S.template factor<2, FAC_TRUE>(W);
  if (p.interm && S.on) S.store(out + 5 * sv, W);
  S.template factor<3, FAC_TRUE>(W);
  if (!p.interm && S.on) S.store(out, W);
}

// ============================================================================
// preconditioner z = (P_tau (x) I) r, P_tau given as a tau-space CSR matrix
// ============================================================================
template <typename R>
__global__ void k_precon(PreconArgs p) {
  const int Vs = p.L * p.L;
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) * 2;  // two sites per thread
  if (s >= Vs) return;
  const int rb = blockIdx.z;
  const size_t sv = 2 * (size_t)Vs;
  const R* r = reinterpret_cast<const R*>(p.r) + (size_t)rb * p.Nt * sv;
  R* z = reinterpret_cast<R*>(p.z) + (size_t)rb * p.Nt * sv;
  const int t0 = blockIdx.y * p.TC;
  const int t1 = min(t0 + p.TC, p.Nt);
  for (int t = t0; t < t1; ++t) {
    Cx<R> acc0 = mk<R>(0, 0), acc1 = mk<R>(0, 0);
    for (int k = p.row_ptr[t]; k < p.row_ptr[t + 1]; ++k) {
      const R w = (R)p.val[k];
      if ((unsigned)p.col[k] >= (unsigned)p.Nt) continue;  // outside the matrix
      Cx<R> a, b;
      ld2(r + p.col[k] * sv + 2 * s, a, b);
      acc0 = mk<R>(fma(w, a.re, acc0.re), fma(w, a.im, acc0.im));
      acc1 = mk<R>(fma(w, b.re, acc1.re), fma(w, b.im, acc1.im));
    }
    st2(z + t * sv + 2 * s, acc0, acc1);
  }
}

// The same product, one block per (128-byte column of sites, right-hand side):
// 16 complex64 or 8 complex128 sites, 8 threads of 16 bytes per row.  The
// column's r rows are read once, coalesced, into shared memory.  Each thread
// then forms C consecutive output rows of its 16 bytes.  Where every one of
// those rows is the middle CSR row (t = Ltau/2) shifted along tau - taps
// t-H .. t+H with the same values, as in the bulk of a banded P_tau - a
// window of 2H+1 rows slides through registers with the taps as constants,
// one shared-memory row read per output row; other rows run over their CSR
// row.  Both orders of summation are the CSR order, so the two forms agree
// bit for bit.
template <typename R>
struct Vec16;
template <>
struct Vec16<float> {
  using T = float4;
  __device__ static T zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  __device__ static T fma(float c, T q, T a) {
    return make_float4(fmaf(c, q.x, a.x), fmaf(c, q.y, a.y), fmaf(c, q.z, a.z), fmaf(c, q.w, a.w));
  }
};
template <>
struct Vec16<double> {
  using T = double2;
  __device__ static T zero() { return make_double2(0., 0.); }
  __device__ static T fma(double c, T q, T a) { return make_double2(::fma(c, q.x, a.x), ::fma(c, q.y, a.y)); }
};

constexpr int PRE_H = 6;  // half-width of the banded form (13 taps, the builtin P_tau)
constexpr int PRE_ROW_THREADS = 8;

inline size_t precon_band_smem(int Nt) { return (size_t)Nt * (16 * PRE_ROW_THREADS + 1); }

template <typename R, int H, int C>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 2) k_precon_band(PreconArgs p) {
  using VT = Vec16<R>;
  using V = typename VT::T;
  constexpr int PER = 16 / sizeof(Cx<R>);  // complex numbers per thread
  constexpr int W = PRE_ROW_THREADS * PER;  // sites per column
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Vs = p.L * p.L, Nt = p.Nt;
  V* colv = reinterpret_cast<V*>(smem_raw);                                    // [Nt][8]
  unsigned char* regular = smem_raw + sizeof(V) * PRE_ROW_THREADS * (size_t)Nt;  // [Nt]
  const int c0 = blockIdx.x * W;
  const size_t sv = 2 * (size_t)Vs;
  const R* r = reinterpret_cast<const R*>(p.r) + (size_t)blockIdx.y * Nt * sv + 2 * (size_t)c0;
  R* z = reinterpret_cast<R*>(p.z) + (size_t)blockIdx.y * Nt * sv + 2 * (size_t)c0;
  const int j = threadIdx.x % PRE_ROW_THREADS, grp = threadIdx.x / PRE_ROW_THREADS;
  const int ngrp = blockDim.x / PRE_ROW_THREADS;  // at most 32 chunks
  const bool jon = j * PER < Vs - c0;
  __shared__ unsigned irregular_chunks;
  if (threadIdx.x == 0) irregular_chunks = 0;
  // the column's rows stream into shared memory while the rows' form is found
  if (jon)
    for (int t = grp; t < Nt; t += ngrp)
      cp_async16(colv + t * PRE_ROW_THREADS + j, reinterpret_cast<const V*>(r + t * sv) + j);
  cp_async_commit();
  // which rows are the middle row shifted (independent loads, no early exit)
  const int tm = Nt / 2, km = p.row_ptr[tm];
  bool band = Nt > 2 * H && p.row_ptr[tm + 1] - km == 2 * H + 1;
  double vm[2 * H + 1];
  if (band) {
#pragma unroll
    for (int i = 0; i <= 2 * H; ++i) {
      vm[i] = p.val[km + i];
      band &= p.col[km + i] == tm - H + i;
    }
  }
  for (int t = threadIdx.x; t < Nt; t += blockDim.x) {
    const int k0 = p.row_ptr[t];
    bool ok = band && t >= H && t < Nt - H && p.row_ptr[t + 1] - k0 == 2 * H + 1;
    if (ok) {
#pragma unroll
      for (int i = 0; i <= 2 * H; ++i) ok &= (p.col[k0 + i] == t - H + i) & (p.val[k0 + i] == vm[i]);
    }
    regular[t] = ok;
  }
  cp_async_wait<0>();
  __syncthreads();
  // chunk grp (rows t0 .. t0+C-1) is regular when all its rows are
  const int t0 = grp * C;
  bool reg = t0 + C <= Nt;
  for (int i = 0; reg && i < C; ++i) reg = regular[t0 + i];
  if (!reg && j == 0) atomicOr(&irregular_chunks, 1u << grp);
  __syncthreads();
  if (!jon) return;
  if (reg) {
    R c[2 * H + 1];
#pragma unroll
    for (int k = 0; k <= 2 * H; ++k) c[k] = (R)vm[k];
    V w[2 * H + 1];
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) w[k + 1] = colv[(t0 - H + k) * PRE_ROW_THREADS + j];
#pragma unroll
    for (int i = 0; i < C; ++i) {
#pragma unroll
      for (int k = 0; k < 2 * H; ++k) w[k] = w[k + 1];
      w[2 * H] = colv[(t0 + i + H) * PRE_ROW_THREADS + j];
      V acc = VT::zero();
#pragma unroll
      for (int k = 0; k <= 2 * H; ++k) acc = VT::fma(c[k], w[k], acc);
      __stcg(reinterpret_cast<V*>(z + (t0 + i) * sv) + j, acc);
    }
  }
  // the rows of irregular chunks, spread over all row groups
  const unsigned mask = irregular_chunks;
  const int G = __popc(mask) * C;
  for (int g = grp; g < G; g += ngrp) {
    unsigned m = mask;
    for (int q = 0; q < g / C; ++q) m &= m - 1;  // drop the chunks before the (g / C)-th
    const int t = (__ffs(m) - 1) * C + g % C;
    if (t >= Nt) continue;
    V acc = VT::zero();
    const int k1 = p.row_ptr[t + 1];
#pragma unroll 4
    for (int k = p.row_ptr[t]; k < k1; ++k) {
      const int cc = p.col[k];
      if ((unsigned)cc < (unsigned)Nt) acc = VT::fma((R)p.val[k], colv[cc * PRE_ROW_THREADS + j], acc);
    }
    __stcg(reinterpret_cast<V*>(z + t * sv) + j, acc);
  }
}

// ============================================================================
// fermion force  F = -dS_f/dphi,  S_f = psi^dag (M^dag M)^{-1} psi,  given xi
// ============================================================================
//
// Per slice t (right vector R = xi_t, left vector u = B_t xi_t - sigma_t
// xi_{t+1} = -sigma_t (M xi)_{t+1}):
//   F(bond of group g) = 2 Re sum_{k: F_g at position k of B}
//                          l_{k-1}^dag dF_g/dphi R_{7-k}
// where R_m is xi_t after the m rightmost factors and l_k is u after the k
// leftmost factors (F_g Hermitian).  R_7 = B xi_t is produced forward; the
// R_m needed afterwards are recovered backwards with F_g^{-1} = c (I - tK)
// while l is advanced forwards, so no partial product is stored.  This is the
// sum that the reference evaluates with explicit partial products
// (force_f_fast, hmc_sampler_batch.py:2150-2227; force_f_sparse :2230-2330).
template <typename R, typename A, int BY, bool PHS, int LT = 0>
struct ForceSlice {
  using Eng = Slice<R, BY, PHS, false, LT>;
  Eng& S;
  __device__ ForceSlice(Eng& s) : S(s) {}

  // term for one bond: c * [conj(l_i) (i a) R_j + conj(l_j) conj(i a) R_i]
  __device__ static __forceinline__ R term(Cx<R> li, Cx<R> lj, Cx<R> Ri, Cx<R> Rj, Cx<R> a, R c) {
    const Cx<R> ia = mk<R>(-a.im, a.re);
    const Cx<R> u = cjmul(li, cmul(ia, Rj));
    const Cx<R> w = cjmul(lj, cjmul(ia, Ri));
    return (R)2 * c * (u.re + w.re);
  }

  // one factor position: R <- F_g^{-1} R, accumulate force, l <- F_g l.
  // Uses exchange buffers 2*par, 2*par+1 (par alternates per call).
  template <int G>
  __device__ __forceinline__ void step(Cx<R> (&Rv)[BY][2], Cx<R> (&l)[BY][2], R (&Fx)[BY][2],
                                       R (&Fy)[BY][2], int par) {
    const R c = (G == 0) ? S.c1 : S.ch;
    Cx<R>* bR = S.xb[2 * par];
    Cx<R>* bl = S.xb[2 * par + 1];
    if (G == 0 || G == 2) {
      // cross row r uses slots r & ~1 (left column) and (r & ~1) + 1 (right column)
      if (S.on) {
#pragma unroll
        for (int r = 0; r < BY; ++r)
          if (Eng::xcross(G, r)) {
            S.slot(bR, r & ~1)[S.id] = Rv[r][0];
            S.slot(bR, (r & ~1) + 1)[S.id] = Rv[r][1];
            S.slot(bl, r & ~1)[S.id] = l[r][0];
            S.slot(bl, (r & ~1) + 1)[S.id] = l[r][1];
          }
      }
      __syncthreads();
      if (!S.on) return;
#pragma unroll
      for (int r = 0; r < BY; ++r) {
        if (!Eng::xcross(G, r)) {
          const Cx<R> a = S.TPX(r, 0);
          const Cx<R> Ri = Rv[r][0], Rj = Rv[r][1];
          const Cx<R> nRi = c * cfma(cneg(a), Rj, Ri);
          const Cx<R> nRj = c * cjfma(cneg(a), Ri, Rj);
          Fx[r][0] += term(l[r][0], l[r][1], nRi, nRj, a, c);
          const Cx<R> li = l[r][0], lj = l[r][1];
          l[r][0] = c * cfma(a, lj, li);
          l[r][1] = c * cjfma(a, li, lj);
          Rv[r][0] = nRi;
          Rv[r][1] = nRj;
        } else {
          const Cx<R> Rright = S.slot(bR, r & ~1)[S.idr], lright = S.slot(bl, r & ~1)[S.idr];
          const Cx<R> Rleft = S.slot(bR, (r & ~1) + 1)[S.idl], lleft = S.slot(bl, (r & ~1) + 1)[S.idl];
          // pair (i = own x0+1, j = right neighbour's x0), phase own
          const Cx<R> a = S.TPX(r, 1);
          const Cx<R> nRi = c * cfma(cneg(a), Rright, Rv[r][1]);
          const Cx<R> nRj = c * cjfma(cneg(a), Rv[r][1], Rright);
          Fx[r][1] += term(l[r][1], lright, nRi, nRj, a, c);
          // pair (i = left neighbour's x0+1, j = own x0), phase from the left
          const Cx<R> al = S.TPL(r);
          const Cx<R> nR0 = c * cjfma(cneg(al), Rleft, Rv[r][0]);
          const Cx<R> nl0 = c * cjfma(al, lleft, l[r][0]);
          const Cx<R> nl1 = c * cfma(a, lright, l[r][1]);
          Rv[r][1] = nRi;
          Rv[r][0] = nR0;
          l[r][1] = nl1;
          l[r][0] = nl0;
        }
      }
    } else {
      constexpr int CL = (G == 1) ? 0 : 1;
      constexpr int CC = 1 - CL;
      if (S.on) {
        S.slot(bR, 0)[S.id] = Rv[0][CC];
        S.slot(bR, 1)[S.id] = Rv[BY - 1][CC];
        S.slot(bl, 0)[S.id] = l[0][CC];
        S.slot(bl, 1)[S.id] = l[BY - 1][CC];
      }
      __syncthreads();
      if (!S.on) return;
      // pairs fully inside the block
#pragma unroll
      for (int r = 0; r < BY; r += 2) {
        const Cx<R> a = S.TPY(r, CL);
        const Cx<R> Ri = Rv[r][CL], Rj = Rv[r + 1][CL];
        const Cx<R> nRi = c * cfma(cneg(a), Rj, Ri);
        const Cx<R> nRj = c * cjfma(cneg(a), Ri, Rj);
        Fy[r][CL] += term(l[r][CL], l[r + 1][CL], nRi, nRj, a, c);
        const Cx<R> li = l[r][CL], lj = l[r + 1][CL];
        l[r][CL] = c * cfma(a, lj, li);
        l[r + 1][CL] = c * cjfma(a, li, lj);
        Rv[r][CL] = nRi;
        Rv[r + 1][CL] = nRj;
      }
#pragma unroll
      for (int r = 1; r + 1 < BY; r += 2) {
        const Cx<R> a = S.TPY(r, CC);
        const Cx<R> Ri = Rv[r][CC], Rj = Rv[r + 1][CC];
        const Cx<R> nRi = c * cfma(cneg(a), Rj, Ri);
        const Cx<R> nRj = c * cjfma(cneg(a), Ri, Rj);
        Fy[r][CC] += term(l[r][CC], l[r + 1][CC], nRi, nRj, a, c);
        const Cx<R> li = l[r][CC], lj = l[r + 1][CC];
        l[r][CC] = c * cfma(a, lj, li);
        l[r + 1][CC] = c * cjfma(a, li, lj);
        Rv[r][CC] = nRi;
        Rv[r + 1][CC] = nRj;
      }
      // bottom pair: i = own last row, j = lower neighbour's first row
      const Cx<R> Rbelow = S.slot(bR, 0)[S.idd], lbelow = S.slot(bl, 0)[S.idd];
      const Cx<R> Rabove = S.slot(bR, 1)[S.idu], labove = S.slot(bl, 1)[S.idu];
      const Cx<R> ab = S.TPY(BY - 1, CC);
      const Cx<R> at = S.TPT(CC);
      const Cx<R> Rb = Rv[BY - 1][CC], lb = l[BY - 1][CC];
      const Cx<R> Rt = Rv[0][CC], lt = l[0][CC];
      const Cx<R> nRi = c * cfma(cneg(ab), Rbelow, Rb);
      const Cx<R> nRj = c * cjfma(cneg(ab), Rb, Rbelow);
      Fy[BY - 1][CC] += term(lb, lbelow, nRi, nRj, ab, c);
      // top site is the j end of the upper neighbour's bond
      Rv[0][CC] = c * cjfma(cneg(at), Rabove, Rt);
      l[0][CC] = c * cjfma(at, labove, lt);
      Rv[BY - 1][CC] = nRi;
      l[BY - 1][CC] = c * cfma(ab, lbelow, lb);
    }
  }
};

template <typename R, typename A, int BY, bool PHS, int LT = 0>
__global__ void __launch_bounds__(MaxThreads<BY>::value, 1) k_force(ForceArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  Slice<R, BY, PHS, false, LT> S;
  const int L = LT ? LT : p.L;
  S.init(L, smem, 4, (R)p.c1, (R)p.ch, threadIdx.x);
  ForceSlice<R, A, BY, PHS, LT> FS(S);
  const int Vs = L * L;
  const size_t sv = 2 * (size_t)Vs;
  const int rb = blockIdx.y;
  const int a = blockIdx.x * p.T;
  const int b = min(a + p.T, p.Nt);
  const int Nt = p.Nt;
  const A* phi = reinterpret_cast<const A*>(p.phi) + (size_t)(rb / p.rhs_per_phi) * Nt * sv;
  const R* xi = reinterpret_cast<const R*>(p.xi) + (size_t)rb * Nt * sv;
  A* F = reinterpret_cast<A*>(p.F) + (size_t)rb * Nt * sv;
  Cx<R> Rv[BY][2], l[BY][2], Xn[BY][2];
  if (S.on) S.load(Rv, xi + a * sv);
  for (int t = a; t < b; ++t) {
    const int tn = (t + 1) % Nt;
    if (S.on) S.load(Xn, xi + tn * sv);
    S.phases(phi + t * sv, (R)p.t1, (R)p.th);
    S.template applyB<FAC_TRUE>(Rv);  // R_7 = B_t xi_t
    axpy_blk<R, BY>(l, Rv, sigma_of<R>(t, Nt), Xn);
    R Fx[BY][2], Fy[BY][2];
#pragma unroll
    for (int r = 0; r < BY; ++r) Fx[r][0] = Fx[r][1] = Fy[r][0] = Fy[r][1] = 0;
    // positions k = 1..7 of B = F4 F3 F2 F1 F2 F3 F4
    // (exchange buffers 2/3 first: buffers 0/1 may still be read by the
    //  last factor of applyB in slower threads)
    FS.template step<3>(Rv, l, Fx, Fy, 1);
    FS.template step<2>(Rv, l, Fx, Fy, 0);
    FS.template step<1>(Rv, l, Fx, Fy, 1);
    FS.template step<0>(Rv, l, Fx, Fy, 0);
    FS.template step<1>(Rv, l, Fx, Fy, 1);
    FS.template step<2>(Rv, l, Fx, Fy, 0);
    FS.template step<3>(Rv, l, Fx, Fy, 1);
    if (S.on) {
#pragma unroll
      for (int r = 0; r < BY; ++r) {
        A o[4] = {(A)Fx[r][0], (A)Fy[r][0], (A)Fx[r][1], (A)Fy[r][1]};
        st4(F + t * sv + 2 * ((S.y0 + r) * L + S.x0), o);
      }
    }
    copy_blk<R, BY>(Rv, Xn);
    __syncthreads();  // the next slice reuses exchange buffers 0/1
  }
}

// ============================================================================
// boson action / force (layout [bs][Nt][L][L][2])
// ============================================================================
template <typename A>
__device__ __forceinline__ A curl_at(const A* ph, int L, int x, int y) {
  const int xp = (x + 1) % L, yp = (y + 1) % L;
  return ph[2 * (x + L * y)] + ph[2 * (xp + L * y) + 1] - ph[2 * (x + L * yp)] - ph[2 * (x + L * y) + 1];
}

// F_b = -d(S_plaq + S_tau)/dphi at every bond
template <typename A>
__device__ __forceinline__ void boson_force_site(const A* phi, int L, int Nt, int t, int x, int y, A K,
                                                 A ctau, int compact, A& fx, A& fy) {
  const size_t sv = 2 * (size_t)L * L;
  const A* ph = phi + t * sv;
  const A sc = sin(curl_at(ph, L, x, y));
  const A sdy = sin(curl_at(ph, L, x, (y + L - 1) % L));
  const A sdx = sin(curl_at(ph, L, (x + L - 1) % L, y));
  fx = K * (sc - sdy);
  fy = K * (-sc + sdx);
  const A* pn = phi + ((t + 1) % Nt) * sv;
  const A* pp = phi + ((t + Nt - 1) % Nt) * sv;
  const int s2 = 2 * (x + L * y);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const A v = ph[s2 + c], vn = pn[s2 + c], vp = pp[s2 + c];
    A f;
    if (compact)
      f = -(-sin(vn - v) + sin(v - vp));
    else
      f = -(-(vn - v) + (v - vp));
    if (c == 0)
      fx += ctau * f;
    else
      fy += ctau * f;
  }
}

template <typename A>
// grid (site blocks, slice, chain): one site per thread, both bond directions
__global__ void k_boson_force(BosonArgs p) {
  const int Vs = p.L * p.L;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= Vs) return;
  const int t = blockIdx.y, b = blockIdx.z;
  const A* phi = reinterpret_cast<const A*>(p.x) + (size_t)b * p.Nt * 2 * Vs;
  A fx, fy;
  boson_force_site<A>(phi, p.L, p.Nt, t, s % p.L, s / p.L, (A)p.K, (A)p.ctau, p.compact, fx, fy);
  A* F = reinterpret_cast<A*>(p.F) + 2 * (((size_t)b * p.Nt + t) * Vs + s);
  F[0] = fx;
  F[1] = fy;
}

// The same force with one block per (slice, chain): the slice's angles are
// staged in shared memory with 16-byte loads, sin(curl) is formed once per
// plaquette (instead of three times per site), and each bond's force is the
// difference of its two plaquettes' sines plus the tau term.  The arithmetic
// of every term is that of boson_force_site, so the results are identical.
// (x, y) of the sites s = threadIdx.x + k blockDim.x of an L x L slice,
// advanced without integer division
struct SiteWalk {
  int s, x, y, dx, dy;
  __device__ explicit SiteWalk(int L)
      : s(threadIdx.x), x(threadIdx.x % L), y(threadIdx.x / L), dx(blockDim.x % L), dy(blockDim.x / L) {}
  __device__ void next(int L) {
    s += blockDim.x;
    x += dx;
    y += dy;
    if (x >= L) {
      x -= L;
      ++y;
    }
  }
};

template <typename A>
inline size_t boson_slice_smem(int L, int curls) {
  return sizeof(A) * (size_t)L * L * (2 + curls);
}

template <typename A>
__global__ void __launch_bounds__(256) k_boson_force_slice(BosonArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = p.L, Vs = L * L, Nt = p.Nt, t = blockIdx.x, b = blockIdx.y;
  A* ph = reinterpret_cast<A*>(smem_raw);  // [Vs][2] angles of slice t
  A* sc = ph + 2 * Vs;                     // [Vs] sin(curl)
  const size_t sv = 2 * (size_t)Vs;
  const A* phi = reinterpret_cast<const A*>(p.x) + (size_t)b * Nt * sv;
  const float4* src = reinterpret_cast<const float4*>(phi + t * sv);
  const int nvec = (int)(sv * sizeof(A) / 16);  // L even: whole 16-byte vectors
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) reinterpret_cast<float4*>(ph)[i] = __ldg(src + i);
  __syncthreads();
  for (SiteWalk w(L); w.s < Vs; w.next(L)) {
    const int s = w.s, x = w.x, y = w.y;
    const int xp = x + 1 == L ? 0 : x + 1, yp = y + 1 == L ? 0 : y + 1;
    sc[s] = sin(ph[2 * (x + L * y)] + ph[2 * (xp + L * y) + 1] - ph[2 * (x + L * yp)] - ph[2 * (x + L * y) + 1]);
  }
  __syncthreads();
  const Cx<A>* pn = reinterpret_cast<const Cx<A>*>(phi + ((t + 1) % Nt) * sv);
  const Cx<A>* pp = reinterpret_cast<const Cx<A>*>(phi + ((t + Nt - 1) % Nt) * sv);
  Cx<A>* F = reinterpret_cast<Cx<A>*>(p.F) + ((size_t)b * Nt + t) * Vs;
  const A K = (A)p.K, ctau = (A)p.ctau;
  for (SiteWalk w(L); w.s < Vs; w.next(L)) {
    const int s = w.s, x = w.x, y = w.y;
    const int xm = x == 0 ? L - 1 : x - 1, ym = y == 0 ? L - 1 : y - 1;
    const A c = sc[s];
    A fx = K * (c - sc[x + L * ym]);
    A fy = K * (-c + sc[xm + L * y]);
    const Cx<A> vn = pn[s], vp = pp[s];
    const A v0 = ph[2 * s], v1 = ph[2 * s + 1];
    if (p.compact) {
      fx += ctau * -(-sin(vn.re - v0) + sin(v0 - vp.re));
      fy += ctau * -(-sin(vn.im - v1) + sin(v1 - vp.im));
    } else {
      fx += ctau * -(-(vn.re - v0) + (v0 - vp.re));
      fy += ctau * -(-(vn.im - v1) + (v1 - vp.im));
    }
    F[s] = mk<A>(fx, fy);
  }
}

// p += ca[b] * F * mask[t];  then (if cb != 0) x += cb[b] * p * mask[t]
template <typename A>
__global__ void k_kick_drift(KickArgs p) {
  const int Vs = p.L * p.L;
  const size_t n = (size_t)p.bs * p.Nt * Vs * 2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t site = i / 2;
    const int t = (site / Vs) % p.Nt;
    const int b = site / ((size_t)Vs * p.Nt);
    const A m = p.mask ? (A)p.mask[t] : (A)1;
    A* P = reinterpret_cast<A*>(p.p);
    const A* F = reinterpret_cast<const A*>(p.F);
    A pv = P[i];
    if (F) pv += (A)(p.kick_scale * p.dt[b]) * F[i] * m;
    P[i] = pv;
    if (p.drift_scale != 0.0) {
      A* X = reinterpret_cast<A*>(p.x);
      X[i] += (A)(p.drift_scale * p.dt[b]) * pv * m;
    }
  }
}

// ============================================================================
// reductions (double accumulation)
// ============================================================================
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-wide sum; every thread of the block must call it
__device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (ln == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < (blockDim.x + 31) / 32) t = sh[threadIdx.x];
  if (w == 0) t = warp_sum(t);
  return t;
}

// out[b] (+)= Re sum conj(u) v over n complex entries per row (double accum)
template <typename R>
__global__ void k_cdot(const R* u, const R* v, int64_t n, double* out) {
  __shared__ double sh[32];
  const int b = blockIdx.y;
  const R* ub = u + (size_t)b * 2 * n;
  const R* vb = v + (size_t)b * 2 * n;
  double acc = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if ((n & 1) == 0 && ((reinterpret_cast<uintptr_t>(ub) | reinterpret_cast<uintptr_t>(vb)) & 15) == 0) {
    // two complex numbers per access
    for (int64_t k = i0; 2 * k < n; k += stride) {
      Cx<R> a0, a1, b0, b1;
      ld2(ub + 4 * k, a0, a1);
      ld2(vb + 4 * k, b0, b1);
      acc += (double)a0.re * (double)b0.re + (double)a0.im * (double)b0.im + (double)a1.re * (double)b1.re +
             (double)a1.im * (double)b1.im;
    }
  } else {
    for (int64_t i = i0; i < n; i += stride)
      acc += (double)ub[2 * i] * (double)vb[2 * i] + (double)ub[2 * i + 1] * (double)vb[2 * i + 1];
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) atomicAdd(out + b, acc);
}

// out[b] (+)= sum of the boson action per chain and (kin != 0) sum p^2 / (2m)
template <typename A>
__global__ void k_boson_action(BosonArgs p, double* out) {
  __shared__ double sh[32];
  const int Vs = p.L * p.L;
  const int b = blockIdx.y;
  const int n = p.Nt * Vs;  // sites of one chain (below 2^31)
  const A* phi = reinterpret_cast<const A*>(p.x) + (size_t)b * n * 2;
  const A* mom = p.F ? reinterpret_cast<const A*>(p.F) + (size_t)b * n * 2 : nullptr;
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = i % Vs;
    const int t = i / Vs;
    const A* ph = phi + t * 2 * (size_t)Vs;
    acc += p.K * (double)cos(curl_at(ph, p.L, s % p.L, s / p.L));
    const A* pn = phi + ((t + 1) % p.Nt) * 2 * (size_t)Vs;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double d = (double)pn[2 * s + c] - (double)ph[2 * s + c];
      acc += p.compact ? p.ctau * (1.0 - cos(d)) : p.ctau * 0.5 * d * d;
      if (mom) {
        const double q = mom[2 * i + c];
        acc += q * q / (2.0 * p.mass);
      }
    }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) atomicAdd(out + b, acc);
}

// The same sums with one block per (slice, chain), the slice staged in shared
// memory with 16-byte loads.
template <typename A>
__global__ void __launch_bounds__(256) k_boson_action_slice(BosonArgs p, double* out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[32];
  const int L = p.L, Vs = L * L, Nt = p.Nt, t = blockIdx.x, b = blockIdx.y;
  A* ph = reinterpret_cast<A*>(smem_raw);  // [Vs][2] angles of slice t
  const size_t sv = 2 * (size_t)Vs;
  const A* phi = reinterpret_cast<const A*>(p.x) + (size_t)b * Nt * sv;
  const float4* src = reinterpret_cast<const float4*>(phi + t * sv);
  const int nvec = (int)(sv * sizeof(A) / 16);
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) reinterpret_cast<float4*>(ph)[i] = __ldg(src + i);
  __syncthreads();
  const Cx<A>* pn = reinterpret_cast<const Cx<A>*>(phi + ((t + 1) % Nt) * sv);
  const Cx<A>* mom = p.F ? reinterpret_cast<const Cx<A>*>(p.F) + ((size_t)b * Nt + t) * Vs : nullptr;
  double acc = 0;
  for (SiteWalk w(L); w.s < Vs; w.next(L)) {
    const int s = w.s, x = w.x, y = w.y;
    const int xp = x + 1 == L ? 0 : x + 1, yp = y + 1 == L ? 0 : y + 1;
    acc += p.K * (double)cos(ph[2 * (x + L * y)] + ph[2 * (xp + L * y) + 1] - ph[2 * (x + L * yp)] -
                             ph[2 * (x + L * y) + 1]);
    const Cx<A> vn = pn[s];
    const double d0 = (double)vn.re - (double)ph[2 * s], d1 = (double)vn.im - (double)ph[2 * s + 1];
    acc += p.compact ? p.ctau * (1.0 - cos(d0)) : p.ctau * 0.5 * d0 * d0;
    acc += p.compact ? p.ctau * (1.0 - cos(d1)) : p.ctau * 0.5 * d1 * d1;
    if (mom) {
      const Cx<A> q = mom[s];
      acc += (double)q.re * (double)q.re / (2.0 * p.mass);
      acc += (double)q.im * (double)q.im / (2.0 * p.mass);
    }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) atomicAdd(out + b, acc);
}

// ============================================================================
// host launchers
// ============================================================================
static int g_num_sms = 0;
int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <typename K>
static int prepare_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return QEDF_ERR_CUDA;
  }
  return QEDF_OK;
}

static int max_threads_by(int by) {
  return by == 2 ? MaxThreads<2>::value : (by == 4 ? MaxThreads<4>::value : MaxThreads<6>::value);
}

bool by_valid(int L, int by) {
  return (by == 2 || by == 4 || by == 6) && L % by == 0 && (L / 2) * (L / by) <= max_threads_by(by);
}

int pick_by(int L, int requested, int real_bytes) {
  if (requested > 0) return by_valid(L, requested) ? requested : -1;
  // single precision: the smallest tile that fits; double precision keeps
  // 2 x 2 tiles only for small slices (register budget of 576-thread blocks)
  if (real_bytes == 4) {
    const int cands[3] = {2, 4, 6};
    for (int c : cands)
      if (by_valid(L, c)) return c;
  } else {
    if (by_valid(L, 2) && (L / 2) * (L / 2) <= 256) return 2;
    const int cands[3] = {4, 6, 2};
    for (int c : cands)
      if (by_valid(L, c)) return c;
  }
  return -1;
}

static size_t smem_limit() { return 227 * 1024; }

template <typename R, typename A, int BY, int EC>
static int launch_operator_t(int op, const OpArgs& a, cudaStream_t st) {
  const int threads = slice_threads(a.L, BY, (EC & EC_XS) != 0);
  const size_t smem = slice_smem_bytes<R, EC>(a.L, BY, 2);
  if (smem > smem_limit() || threads > MaxT<BY, EC>::value) return QEDF_ERR_SIZE;
  dim3 grid((a.Nt + a.T - 1) / a.T, a.bs);
  if (op == OP_M) {
    if (prepare_smem(k_operator<R, A, BY, OP_M, EC>, smem)) return QEDF_ERR_CUDA;
    k_operator<R, A, BY, OP_M, EC><<<grid, threads, smem, st>>>(a);
  } else if (op == OP_MH) {
    if (prepare_smem(k_operator<R, A, BY, OP_MH, EC>, smem)) return QEDF_ERR_CUDA;
    k_operator<R, A, BY, OP_MH, EC><<<grid, threads, smem, st>>>(a);
  } else {
    if (prepare_smem(k_operator<R, A, BY, OP_MHM, EC>, smem)) return QEDF_ERR_CUDA;
    k_operator<R, A, BY, OP_MHM, EC><<<grid, threads, smem, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

// Lattice sides with engines compiled for a fixed L (the benchmark lattice,
// L = 48); every other L runs the run-time-L engine.
template <typename R, typename A, int BY, int EC>
static int launch_operator_fl(int op, const OpArgs& a, cudaStream_t st) {
  if constexpr (EC == 0 || EC == EC_PHS)
    return with_fixed_l<BY>(a.L, [&](auto lt) {
      return launch_operator_t<R, A, BY, EC | EC_L(decltype(lt)::value)>(op, a, st);
    });
  return launch_operator_t<R, A, BY, EC>(op, a, st);
}

// double precision keeps the phases in shared memory when they fit; without
// room for the stash, y stays in registers
template <typename R, typename A, int BY>
static int launch_operator_by(int op, const OpArgs& a, int xs, cudaStream_t st) {
  if (sizeof(R) == 8 && slice_smem_bytes<R, EC_PHS>(a.L, BY, 2) <= smem_limit())
    return launch_operator_fl<R, A, BY, EC_PHS>(op, a, st);
  if (sizeof(R) == 4 && xs && xs_possible(a.L) && ((a.L / 2) & (a.L / 2 - 1)) == 0 &&
      slice_threads(a.L, BY, true) <= MaxT<BY, EC_XS>::value)
    return launch_operator_t<R, A, BY, EC_XS>(op, a, st);
  if (slice_smem_bytes<R, 0>(a.L, BY, 2) <= smem_limit()) return launch_operator_fl<R, A, BY, 0>(op, a, st);
  return launch_operator_t<R, A, BY, EC_NOSTASH>(op, a, st);
}

template <typename R, typename A>
int launch_operator(int op, OpArgs a, int by, cudaStream_t st) {
  by = pick_by(a.L, by, sizeof(R));
  if (by < 0) return QEDF_ERR_ARG;
  if (a.T <= 0) {
    // spread the slabs over about two waves of the SMs
    const long want = 2L * num_sms();
    long slabs = std::max(1L, want / std::max(1, a.bs));
    a.T = (int)std::max(1L, (a.Nt + slabs - 1) / slabs);
  }
  const int xs = a.xs;
  switch (by) {
    case 2: return launch_operator_by<R, A, 2>(op, a, xs, st);
    case 4: return launch_operator_by<R, A, 4>(op, a, xs, st);
    case 6: return launch_operator_by<R, A, 6>(op, a, xs, st);
  }
  return QEDF_ERR_ARG;
}
template int launch_operator<float, float>(int, OpArgs, int, cudaStream_t);
template int launch_operator<double, double>(int, OpArgs, int, cudaStream_t);

template <typename R, typename A, int BY>
static int launch_bvec_by(const BvecArgs& a, int nvec, cudaStream_t st) {
  const int threads = ((a.L / 2) * (a.L / BY) + 31) / 32 * 32;
  const size_t smem = slice_smem_bytes<R, 0>(a.L, BY, 2);
  if (smem > smem_limit()) return QEDF_ERR_SIZE;
  if (prepare_smem(k_bvec<R, A, BY, false>, smem)) return QEDF_ERR_CUDA;
  k_bvec<R, A, BY, false><<<nvec, threads, smem, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

template <typename R, typename A>
int launch_bvec(BvecArgs a, int nvec, cudaStream_t st) {
  const int by = pick_by(a.L, 0, sizeof(R));
  switch (by) {
    case 2: return launch_bvec_by<R, A, 2>(a, nvec, st);
    case 4: return launch_bvec_by<R, A, 4>(a, nvec, st);
    case 6: return launch_bvec_by<R, A, 6>(a, nvec, st);
  }
  return QEDF_ERR_ARG;
}
template int launch_bvec<float, float>(BvecArgs, int, cudaStream_t);
template int launch_bvec<double, double>(BvecArgs, int, cudaStream_t);

template <typename R>
int launch_precon(const PreconArgs& a, cudaStream_t st) {
  const int Vs = a.L * a.L;
  const size_t band_smem = precon_band_smem(a.Nt);
  if (band_smem <= smem_limit()) {
    // a tau column per block, staged in shared memory; 16, 32 or 64 rows a
    // thread, so that a block has at most 256 threads
    constexpr int W = PRE_ROW_THREADS * 16 / (int)sizeof(Cx<R>);
    dim3 grid((Vs + W - 1) / W, a.bs);
    if (a.Nt <= 512) {
      if (prepare_smem(k_precon_band<R, PRE_H, 16>, band_smem)) return QEDF_ERR_CUDA;
      k_precon_band<R, PRE_H, 16><<<grid, PRE_ROW_THREADS * ((a.Nt + 15) / 16), band_smem, st>>>(a);
    } else if (a.Nt <= 1024) {
      if (prepare_smem(k_precon_band<R, PRE_H, 32>, band_smem)) return QEDF_ERR_CUDA;
      k_precon_band<R, PRE_H, 32><<<grid, PRE_ROW_THREADS * ((a.Nt + 31) / 32), band_smem, st>>>(a);
    } else {
      if (prepare_smem(k_precon_band<R, PRE_H, 64>, band_smem)) return QEDF_ERR_CUDA;
      k_precon_band<R, PRE_H, 64><<<grid, PRE_ROW_THREADS * ((a.Nt + 63) / 64), band_smem, st>>>(a);
    }
  } else {
    const int threads = 128;
    dim3 grid((Vs / 2 + threads - 1) / threads, (a.Nt + a.TC - 1) / a.TC, a.bs);
    k_precon<R><<<grid, threads, 0, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template int launch_precon<float>(const PreconArgs&, cudaStream_t);
template int launch_precon<double>(const PreconArgs&, cudaStream_t);

template <typename R, typename A, int BY, bool PHS, int LT = 0>
static int launch_force_t(const ForceArgs& a, cudaStream_t st) {
  const int threads = ((a.L / 2) * (a.L / BY) + 31) / 32 * 32;
  // four exchange buffers; the force keeps no stash
  const size_t smem = slice_smem_bytes<R, (PHS ? EC_PHS : 0) | EC_NOSTASH>(a.L, BY, 4);
  if (smem > smem_limit()) return QEDF_ERR_SIZE;
  if (prepare_smem(k_force<R, A, BY, PHS, LT>, smem)) return QEDF_ERR_CUDA;
  dim3 grid((a.Nt + a.T - 1) / a.T, a.bs);
  k_force<R, A, BY, PHS, LT><<<grid, threads, smem, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

template <typename R, typename A, int BY>
static int launch_force_by(const ForceArgs& a, cudaStream_t st) {
  // the benchmark lattices run engines compiled for their size
  if (sizeof(R) == 8 && slice_smem_bytes<R, EC_PHS | EC_NOSTASH>(a.L, BY, 4) <= smem_limit())
    return with_fixed_l<BY>(a.L, [&](auto lt) { return launch_force_t<R, A, BY, true, decltype(lt)::value>(a, st); });
  return with_fixed_l<BY>(a.L, [&](auto lt) { return launch_force_t<R, A, BY, false, decltype(lt)::value>(a, st); });
}

template <typename R, typename A>
int launch_force(ForceArgs a, int by, cudaStream_t st) {
  by = pick_by(a.L, by, sizeof(R));
  if (by < 0) return QEDF_ERR_ARG;
  if (a.T <= 0) {
    const long want = 2L * num_sms();
    long slabs = std::max(1L, want / std::max(1, a.bs));
    a.T = (int)std::max(1L, (a.Nt + slabs - 1) / slabs);
  }
  switch (by) {
    case 2: return launch_force_by<R, A, 2>(a, st);
    case 4: return launch_force_by<R, A, 4>(a, st);
    case 6: return launch_force_by<R, A, 6>(a, st);
  }
  return QEDF_ERR_ARG;
}
template int launch_force<float, float>(ForceArgs, int, cudaStream_t);
template int launch_force<double, double>(ForceArgs, int, cudaStream_t);

template <typename A>
int launch_boson_force(const BosonArgs& a, cudaStream_t st) {
  const int threads = 256;
  const size_t smem = boson_slice_smem<A>(a.L, 1);
  if (smem <= smem_limit()) {
    if (prepare_smem(k_boson_force_slice<A>, smem)) return QEDF_ERR_CUDA;
    k_boson_force_slice<A><<<dim3(a.Nt, a.bs), threads, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
  }
  dim3 grid((a.L * a.L + threads - 1) / threads, a.Nt, a.bs);
  k_boson_force<A><<<grid, threads, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template int launch_boson_force<float>(const BosonArgs&, cudaStream_t);
template int launch_boson_force<double>(const BosonArgs&, cudaStream_t);

template <typename A>
int launch_kick_drift(const KickArgs& a, cudaStream_t st) {
  const size_t n = (size_t)a.bs * a.Nt * a.L * a.L * 2;
  const int threads = 256;
  const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, (size_t)num_sms() * 8);
  k_kick_drift<A><<<blocks, threads, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template int launch_kick_drift<float>(const KickArgs&, cudaStream_t);
template int launch_kick_drift<double>(const KickArgs&, cudaStream_t);

template <typename A>
int launch_boson_action(const BosonArgs& a, double* out, cudaStream_t st) {
  const size_t n = (size_t)a.Nt * a.L * a.L;
  const int threads = 256;
  const size_t smem = boson_slice_smem<A>(a.L, 0);
  if (smem + 32 * sizeof(double) <= smem_limit()) {
    if (prepare_smem(k_boson_action_slice<A>, smem)) return QEDF_ERR_CUDA;
    k_boson_action_slice<A><<<dim3(a.Nt, a.bs), threads, smem, st>>>(a, out);
    return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
  }
  const int bx = (int)std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads,
                                                           (size_t)num_sms() * 16 / std::max(1, a.bs) + 1));
  k_boson_action<A><<<dim3(bx, a.bs), threads, 0, st>>>(a, out);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template int launch_boson_action<float>(const BosonArgs&, double*, cudaStream_t);
template int launch_boson_action<double>(const BosonArgs&, double*, cudaStream_t);

template <typename R>
int launch_cdot(const R* u, const R* v, int64_t n, int rows, double* out, cudaStream_t st) {
  const int threads = 256;
  const int bx = (int)std::max<int64_t>(1, std::min<int64_t>((n / 2 + threads - 1) / threads,
                                                             (int64_t)num_sms() * 8 / std::max(1, rows) + 1));
  k_cdot<R><<<dim3(bx, rows), threads, 0, st>>>(u, v, n, out);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}
template int launch_cdot<float>(const float*, const float*, int64_t, int, double*, cudaStream_t);
template int launch_cdot<double>(const double*, const double*, int64_t, int, double*, cudaStream_t);

}  // namespace qedf
