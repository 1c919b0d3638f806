// Persistent batched preconditioned CG on M^dag M x = b.
//
// One cooperative launch runs the whole solve.  Each iteration is two
// grid-wide phases separated by grid barriers:
//
//   A  (operator units: one right-hand side x one tau-slab)
//        x    += alpha_old p_old          (the previous iteration's update,
//                                          on the slab's own slices)
//        p_new = z + beta p_old          (halo slices recomputed, not exchanged)
//        Op    = M^dag M p_new            (slice engine, registers + smem)
//        pAp  += Re p_new^dag Op          (double)
//   BC (elementwise units: one right-hand side x a chunk of sites, all tau)
//        r -= alpha Op
//        z  = (P_tau (x) I) r             (the chunk's r column stays in smem)
//        rr += |r|^2,  rz += Re r^dag z   (double)
//
// The last iteration's x update is applied by a reliable update's fold or at
// the end of the solve.
//
// which is the arithmetic of preconditioned_cg_fast_test
// (hmc_sampler_batch.py:751-846) with the reference's per-iteration torch
// kernels (einsum dots, axpys, _C.mhm_vec, _C.precon_vec) fused.  Every
// right-hand side has its own mask: once ||r||/||b|| <= rtol it stops
// updating (the reference's active_bs, :826).
//
// Mixed mode iterates in float and keeps x and b in double: x_lo (float)
// accumulates the update, and a reliable update folds it into x (double),
// recomputes the true residual r = b - A x with the double-precision engine
// and restarts r from it.  It runs every ru_interval iterations, when the
// iterated residual fell by ru_delta since the last one, and whenever the
// iterated residual claims convergence, so convergence is always decided on
// the true residual.
//
// Per-right-hand-side scalars (alpha, beta, masks) are recomputed by every
// thread block from the same double accumulators in the same order, so all
// blocks take identical decisions without another barrier.  Grid barriers
// spin with a clock budget; when it runs out the block raises an error flag
// that ends every block's loop, and the solve reports QEDF_ERR_TIMEOUT.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "qedf_internal.h"
#include "qedf_precon_table.h"
#include "qedf_slice.cuh"

namespace qedf {

// rows in flight per thread in the single-precision elementwise update
constexpr int PCG_EW_STAGES = 4;

__constant__ PreTable c_pre = {QEDF_PRE_LAYOUT, QEDF_PRE_EDGE_VALUES, QEDF_PRE_TAIL_VALUES,
                               QEDF_PRE_MIDDLE_VALUES, QEDF_PRE_CORNER_VALUES};
static const PreTable h_pre = {QEDF_PRE_LAYOUT, QEDF_PRE_EDGE_VALUES, QEDF_PRE_TAIL_VALUES,
                               QEDF_PRE_MIDDLE_VALUES, QEDF_PRE_CORNER_VALUES};

// ---------------------------------------------------------------------------
// bounded grid barrier
// ---------------------------------------------------------------------------
// bar[0] counts arrivals over the whole solve (zeroed per solve); barrier n
// of a block is passed once the count reaches n * nblocks.  Arrival is a
// release reduction without a reply, and waiting an acquire load of the
// count, so the last block's arrival ends the barrier directly.  bar[2] is
// the error word.  `target` is the calling block's count to wait for, kept
// by its thread 0 across calls.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, long long budget,
                                             unsigned int& target) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* err = bar + 2;
    target += nblocks;
    __threadfence();
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(bar), "r"(1u) : "memory");
    const long long t0 = clock64();
    while (true) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(bar) : "memory");
      if ((int)(v - target) >= 0) break;
      if (*err) break;
      if (clock64() - t0 > budget) {
        atomicExch(bar + 2, (unsigned int)QEDF_ERR_TIMEOUT);
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
  return *((volatile unsigned int*)(bar + 2)) == 0;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum over the block, result valid in thread 0
__device__ double block_sum_d(double v, double* sh) {
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (ln == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x + 31) / 32 ? sh[threadIdx.x] : 0.0;
    t = warp_sum_d(t);
  }
  return t;
}

// three sums over the block at once, results valid in thread 0 (sh: 96 doubles)
__device__ void block_sum3_d(double& a, double& b, double& c, double* sh) {
  a = warp_sum_d(a);
  b = warp_sum_d(b);
  c = warp_sum_d(c);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (ln == 0) {
    sh[w] = a;
    sh[32 + w] = b;
    sh[64 + w] = c;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool in = threadIdx.x < (blockDim.x + 31) / 32;
    a = warp_sum_d(in ? sh[threadIdx.x] : 0.0);
    b = warp_sum_d(in ? sh[32 + threadIdx.x] : 0.0);
    c = warp_sum_d(in ? sh[64 + threadIdx.x] : 0.0);
  }
}

// ---------------------------------------------------------------------------
// accumulator layout (doubles)
// ---------------------------------------------------------------------------
struct Acc {
  double* bb;       // [NV]
  double* pAp;      // [2][NV]
  double* rr;       // [2][NV]
  double* rz;       // [2][NV]
  double* ru_rr;    // [NV]
  double* ru_rz;    // [NV]
  double* pp;       // [2][NV] |p|^2 of the operator phase (scaled fp16 storage)
  __device__ Acc(double* a, int NV) {
    bb = a;
    pAp = a + NV;
    rr = a + 3 * NV;
    rz = a + 5 * NV;
    ru_rr = a + 7 * NV;
    ru_rz = a + 8 * NV;
    pp = a + 9 * NV;
  }
};
constexpr int ACC_PER_RHS = 11;

// unit -> system
__device__ __forceinline__ int find_sys_A(const PcgParams& p, int u) {
  int s = 0;
  while (s + 1 < p.nsys && u >= p.sys[s + 1].unitA0) ++s;
  return s;
}
__device__ __forceinline__ int find_sys_E(const PcgParams& p, int u) {
  int s = 0;
  while (s + 1 < p.nsys && u >= p.sys[s + 1].unitE0) ++s;
  return s;
}

template <typename R>
__device__ __forceinline__ Cx<R> ldc(const R* base, int64_t i) {
  return mk<R>(base[2 * i], base[2 * i + 1]);
}
template <typename R>
__device__ __forceinline__ void stc(R* base, int64_t i, Cx<R> v) {
  base[2 * i] = v.re;
  base[2 * i + 1] = v.im;
}

// Per-block copy of the per-right-hand-side state (identical in all blocks).
struct RhsState {
  double alpha[PCG_MAX_RHS], beta[PCG_MAX_RHS], rz[PCG_MAX_RHS], rzold[PCG_MAX_RHS];
  double rr[PCG_MAX_RHS], res[PCG_MAX_RHS], resmax[PCG_MAX_RHS];
  int iters[PCG_MAX_RHS], lastru[PCG_MAX_RHS], status[PCG_MAX_RHS];
  unsigned char active[PCG_MAX_RHS], ru[PCG_MAX_RHS];
  unsigned char pending[PCG_MAX_RHS];  // x += alpha p of the last iteration not yet applied
  int any_active, any_ru;
  double red[96];
};

// Per-block copy of the storage scales of z and of the two p buffers (scaled
// fp16 storage only), identical in all blocks: each is set from the squared
// residual norm, which every block holds, before the pass that writes the
// vector, and is read by the passes that load it.
struct StScales {
  float z[PCG_MAX_RHS], p[2][PCG_MAX_RHS];
};
struct StNoScales {};

// Optional phase timing (block 0, thread 0): prof[k] accumulates clock64 cycles of
//   0 init, 1 operator phase work, 2 wait after it, 3 elementwise phase work,
//   4 wait after it, 5 reliable updates (work + waits), 6 iterations, 7 total
struct PhaseClock {
  long long* prof;
  long long t;
  __device__ PhaseClock(long long* p) : prof((p && blockIdx.x == 0 && threadIdx.x == 0) ? p : nullptr), t(0) {
    if (prof) t = clock64();
  }
  __device__ __forceinline__ void lap(int k) {
    if (prof) {
      const long long n = clock64();
      prof[k] += n - t;
      t = n;
    }
  }
  __device__ __forceinline__ void add(int k, long long v) {
    if (prof) prof[k] += v;
  }
};

// ---------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------
template <typename RS, typename RH, typename A, int BY, int ECS, int ECH>
__global__ void __launch_bounds__(MaxT<BY, ECS>::value, MaxT<BY, ECS>::min_blocks)
    k_pcg(const __grid_constant__ PcgParams p) {
  constexpr bool PHS_S = (ECS & EC_PHS) != 0, STASH_S = (ECS & EC_NOSTASH) == 0;
  constexpr bool XS_S = (ECS & EC_XS) != 0;
  constexpr bool PHS_H = (ECH & EC_PHS) != 0, STASH_H = (ECH & EC_NOSTASH) == 0;
  constexpr bool STG_S = (ECS & EC_STAGE) != 0;
  static_assert(!STG_S || (STASH_S && !XS_S), "the staged engine keeps y_t in the stash");
  // storage of the search direction p and the preconditioned residual z: the
  // iteration precision, bf16 pairs (EC_BF16) or scaled fp16 pairs (EC_F16),
  // both mixed-mode options.  r, M^dag M p and x_lo always keep the iteration
  // precision, so that the residual recurrence r -= alpha M^dag M p stays that
  // of x += alpha p.
  constexpr bool BF = (ECS & EC_BF16) != 0;
  constexpr bool H16 = (ECS & EC_F16) != 0;
  constexpr bool LOWP = BF || H16;
  using SP = typename std::conditional<BF, bf16, typename std::conditional<H16, __half, RS>::type>::type;
  static_assert(!LOWP || (sizeof(RS) == 4 && !std::is_same<RS, RH>::value && !XS_S && !(BF && H16)),
                "bf16 and fp16 storage are mixed-precision modes");
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ RhsState st;
  __shared__ typename std::conditional<H16, StScales, StNoScales>::type scl;
  // scales of z and of p buffer `par` (1 for every other storage type)
  auto sc_z = [&](int v) -> RS {
    if constexpr (H16) return (RS)scl.z[v];
    else return (RS)1;
  };
  auto sc_p = [&](int par, int v) -> RS {
    if constexpr (H16) return (RS)scl.p[par][v];
    else return (RS)1;
  };
  __shared__ unsigned long long stg_bar[2];
  constexpr bool MIXED = !std::is_same<RS, RH>::value;
  // lattice side: compiled in (every system has it) or per system
  constexpr int LT = ec_fixed_l(ECS);
  auto SL = [](const PcgSys& S) { return LT ? LT : S.L; };
  const int NV = p.nrhs;
  Acc acc(p.acc, NV);
  const unsigned int nblk = gridDim.x;
  const int tid = threadIdx.x;
  const SP* zbuf = reinterpret_cast<const SP*>(p.z);
  RS* r = reinterpret_cast<RS*>(p.r);
  SP* z = reinterpret_cast<SP*>(p.z);
  RS* Op = reinterpret_cast<RS*>(p.Op);
  RS* xs = MIXED ? reinterpret_cast<RS*>(p.xlo) : reinterpret_cast<RS*>(p.x);
  RH* xh = reinterpret_cast<RH*>(p.x);
  const RH* bvec = reinterpret_cast<const RH*>(p.b);
  const A* phi_all = reinterpret_cast<const A*>(p.phi);
  const int CH = p.CH;   // sites per elementwise unit (16 or 32)
  const int CHC = CH;
  const int PPR = CHC / 2;  // site pairs per row of a unit

  // slice stages of the operator passes (EC_STAGE): two buffers of z, p_old
  // and x_lo slices behind the slice engine's tables
  SliceStages<3> stg;
  const long long budget_stage = p.timeout_cycles;
  if constexpr (STG_S) {
    SliceStages<3>::init_barriers(stg_bar);
    stg.setup(stg_bar, dsm + p.stage_off, 0);
  }
  for (int v = tid; v < NV; v += blockDim.x) {
    st.active[v] = 1;
    st.iters[v] = 0;
    st.lastru[v] = 0;
    st.status[v] = QEDF_OK;
    st.resmax[v] = 1.0;
    st.ru[v] = 0;
    st.pending[v] = 0;
  }
  __syncthreads();

  // elementwise unit decode
  auto unitE = [&](int u, int& s, int& v, int& c0, int& c1) {
    s = find_sys_E(p, u);
    const PcgSys& S = p.sys[s];
    const int lu = u - S.unitE0;
    v = S.rhs0 + lu / S.nchunk;
    const int Vs = SL(S) * SL(S);
    c0 = (lu % S.nchunk) * CH;
    c1 = min(c0 + CH, Vs);
  };
  // plain modes with an initial guess: the first pass forms r = b - A x (below)
  bool guess_pass = false;
  auto vec_base = [&](int s, int v) -> int64_t {
    const PcgSys& S = p.sys[s];
    return S.vec0 + (int64_t)(v - S.rhs0) * S.Nt * SL(S) * SL(S);
  };

  // ---- BC-type elementwise pass over one unit --------------------------------
  // kind 0: init (x = 0 unless it holds an initial guess, r = b, bb); 1:
  // iteration update; 2: preconditioner only (after a reliable update or the
  // initial guess's residual); 3: preconditioner only, r^dag z into the rz
  // slot (scaled fp16 init).  A unit is CHC sites of one right-hand side over
  // all tau; a thread handles two neighbouring sites (one 16-byte access per
  // vector in single precision) in every (blockDim/PPR)-th row.  r of the unit
  // stays in shared memory for the tau-stencil of the preconditioner, whose
  // periodic 13-band table P_tab[t][k] (offset k - 6; the corners of the
  // reference's matrix are the band's wrap-around) was prepared per system.
  auto elementwise = [&](int kind, int u, int slot) {
    int s, v, c0, c1;
    unitE(u, s, v, c0, c1);
    const PcgSys& S = p.sys[s];
    const int Vs = SL(S) * SL(S), Nt = S.Nt, w = c1 - c0;
    const int64_t base = vec_base(s, v);
    Cx<RS>* rsm = reinterpret_cast<Cx<RS>*>(dsm);
    const RS al = (RS)st.alpha[v];
    const RS* opv = Op;
    const int j = tid % PPR;
    const int rstep = blockDim.x / PPR;
    const bool jon = 2 * j < w;
    double acc_a = 0, acc_b = 0, acc_c = 0;
    if (sizeof(RS) == 4 && kind == 1) {
      // The iteration update, single precision: the two input rows (Op, r)
      // of this thread's next PCG_EW_STAGES rows are in flight while one row
      // is updated, as 16-byte cp.async copies into a staging area behind the
      // unit's r column (stage k % PCG_EW_STAGES, [vector][thread] units).  A
      // stage is refilled only after its values were used; every issue slot
      // commits a group, empty past the last row, so that the wait count is
      // a constant.
      uint4* stg = reinterpret_cast<uint4*>(dsm + ((size_t)Nt * CHC * sizeof(Cx<RS>) + 15) / 16 * 16);
      const int nthr = blockDim.x, t0 = tid / PPR;
      const int K = (jon && t0 < Nt) ? (Nt - 1 - t0) / rstep + 1 : 0;
      RS cpart = 0;  // this thread's |r|^2 in the iteration precision
      auto issue = [&](int k) {
        if (k < K) {
          const int64_t i2 = 2 * (base + (int64_t)(t0 + k * rstep) * Vs + c0 + 2 * j);
          uint4* d = stg + (size_t)(k % PCG_EW_STAGES) * 2 * nthr + tid;
          cp_async16(d, opv + i2);
          cp_async16(d + nthr, r + i2);
        }
        cp_async_commit();
      };
#pragma unroll
      for (int k = 0; k < PCG_EW_STAGES; ++k) issue(k);
      for (int k = 0; k < K; ++k) {
        cp_async_wait<PCG_EW_STAGES - 1>();
        const uint4* d = stg + (size_t)(k % PCG_EW_STAGES) * 2 * nthr + tid;
        Cx<RS> o0, o1, r0, r1;
        ld2c(reinterpret_cast<const RS*>(d), o0, o1);
        ld2c(reinterpret_cast<const RS*>(d + nthr), r0, r1);
        r0 = mk<RS>(fma(-al, o0.re, r0.re), fma(-al, o0.im, r0.im));
        r1 = mk<RS>(fma(-al, o1.re, r1.re), fma(-al, o1.im, r1.im));
        const int t = t0 + k * rstep;
        const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
        st2s(r + i2, r0, r1);
        cpart = fma(r0.re, r0.re, fma(r0.im, r0.im, fma(r1.re, r1.re, fma(r1.im, r1.im, cpart))));
        st2(reinterpret_cast<RS*>(rsm + t * CHC + 2 * j), r0, r1);
        issue(k + PCG_EW_STAGES);
      }
      cp_async_wait<0>();
      acc_c += (double)cpart;
    } else
#pragma unroll 2
    for (int t = tid / PPR; t < Nt; t += rstep) {
      if (!jon) continue;
      const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);  // reals
      Cx<RS> r0, r1;
      if (kind == 0) {
        Cx<RH> b0, b1;
        ld2c(bvec + i2, b0, b1);
        acc_a += (double)b0.re * b0.re + (double)b0.im * b0.im + (double)b1.re * b1.re + (double)b1.im * b1.im;
        r0 = mk<RS>((RS)b0.re, (RS)b0.im);
        r1 = mk<RS>((RS)b1.re, (RS)b1.im);
        // x_lo (mixed) always starts at 0; x itself unless it is the guess
        if (MIXED || !p.x_init) st2s(xs + i2, mk<RS>(0, 0), mk<RS>(0, 0));
        if (MIXED && !p.x_init) st2(xh + i2, mk<RH>(0, 0), mk<RH>(0, 0));
        st2s(r + i2, r0, r1);
      } else if (kind == 1) {
        Cx<RS> o0, o1;
        ld2s(opv + i2, o0, o1);
        ld2s(r + i2, r0, r1);
        r0 = mk<RS>(fma(-al, o0.re, r0.re), fma(-al, o0.im, r0.im));
        r1 = mk<RS>(fma(-al, o1.re, r1.re), fma(-al, o1.im, r1.im));
        st2s(r + i2, r0, r1);
      } else {
        ld2s(r + i2, r0, r1);
      }
      acc_c += (double)r0.re * r0.re + (double)r0.im * r0.im + (double)r1.re * r1.re + (double)r1.im * r1.im;
      st2(reinterpret_cast<RS*>(rsm + t * CHC + 2 * j), r0, r1);
    }
    __syncthreads();
    const float* tab = p.ptab + S.ptab0;
    RS cmid[7];  // the bulk band, by tau distance
#pragma unroll
    for (int d = 0; d < 7; ++d) cmid[d] = (RS)c_pre.middle[d];
    RS bpart = 0;  // this thread's r^dag z in the iteration precision
    // scaled fp16: the scale of z follows from |r|, known only after the init
    // pass, so that pass leaves z to a kind-3 pass
    const bool zpass = !(H16 && kind == 0);
    const RS szv = sc_z(v), izv = (RS)1 / szv;  // powers of two: exact
#pragma unroll 2
    for (int t = tid / PPR; t < Nt; t += rstep) {
      if (!jon || !zpass) continue;
      Cx<RS> r0, r1;
      ld2c(reinterpret_cast<const RS*>(rsm + t * CHC + 2 * j), r0, r1);
      Cx<RS> z0 = r0, z1 = r1;
      if (S.precon) {
        z0 = mk<RS>(0, 0);
        z1 = mk<RS>(0, 0);
        if (t >= S.pmid_lo && t < S.pmid_hi) {
          // bulk row: coefficients in registers, no wrap (t - 6 >= 0, t + 6 < Nt)
#pragma unroll
          for (int k = 0; k < 13; ++k) {
            const RS c = cmid[k < 6 ? 6 - k : k - 6];
            Cx<RS> q0, q1;
            ld2c(reinterpret_cast<const RS*>(rsm + (t - 6 + k) * CHC + 2 * j), q0, q1);
            z0 = mk<RS>(fma(c, q0.re, z0.re), fma(c, q0.im, z0.im));
            z1 = mk<RS>(fma(c, q1.re, z1.re), fma(c, q1.im, z1.im));
          }
        } else {
          int tt = t - 6 < 0 ? t - 6 + Nt : t - 6;
#pragma unroll
          for (int k = 0; k < 13; ++k) {
            const RS c = (RS)__ldg(tab + t * 13 + k);
            Cx<RS> q0, q1;
            ld2c(reinterpret_cast<const RS*>(rsm + tt * CHC + 2 * j), q0, q1);
            z0 = mk<RS>(fma(c, q0.re, z0.re), fma(c, q0.im, z0.im));
            z1 = mk<RS>(fma(c, q1.re, z1.re), fma(c, q1.im, z1.im));
            tt = tt + 1 == Nt ? 0 : tt + 1;
          }
        }
        const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
        z0 = round_st<SP>(z0, szv, izv);
        z1 = round_st<SP>(z1, szv, izv);
        st2s(z + i2, z0, z1, izv);
      } else if (LOWP) {
        // the narrow-storage engines read z even without a preconditioner:
        // z = r, rounded
        const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
        z0 = round_st<SP>(z0, szv, izv);
        z1 = round_st<SP>(z1, szv, izv);
        st2s(z + i2, z0, z1, izv);
      }
      bpart = fma(r0.re, z0.re, fma(r0.im, z0.im, fma(r1.re, z1.re, fma(r1.im, z1.im, bpart))));
    }
    acc_b += (double)bpart;
    double sa = acc_a, sb = acc_b, sc = acc_c;
    block_sum3_d(sa, sb, sc, st.red);
    if (tid == 0) {
      if (kind == 0) {
        atomicAdd(acc.bb + v, sa);
        atomicAdd(acc.rr + slot * NV + v, sc);
        atomicAdd(acc.rz + slot * NV + v, sb);
      } else if (kind == 1) {
        atomicAdd(acc.rr + slot * NV + v, sc);
        atomicAdd(acc.rz + slot * NV + v, sb);
      } else if (kind == 3) {
        atomicAdd(acc.rz + slot * NV + v, sb);
      } else {
        atomicAdd(acc.ru_rz + v, sb);
      }
    }
    __syncthreads();
  };

  // ---- operator pass over one unit -------------------------------------------
  // p_new = z + beta p_old on the slab and its halo slices, Op = M^dag M p_new,
  // and pAp = p_new^dag M^dag M p_new = sum_t |(M p_new)_t|^2 over the slab.
  auto operator_unit_sloppy = [&](int u, int slot) {
    if constexpr (!STG_S) {
    const int s = find_sys_A(p, u);
    const PcgSys& S = p.sys[s];
    const int lu = u - S.unitA0;
    const int v = S.rhs0 + lu / S.nslab;
    const int a = (lu % S.nslab) * S.T;
    const int bnd = min(a + S.T, S.Nt);
    const int Nt = S.Nt, Vs = SL(S) * SL(S);
    const size_t sv = 2 * (size_t)Vs;
    Slice<RS, BY, PHS_S, XS_S, LT> E;
    E.init(SL(S), dsm, 2, (RS)p.c1, (RS)p.ch, tid);
    const int64_t vb = 2 * vec_base(s, v);  // reals
    const A* phi = phi_all + S.phi0 + (S.shared ? 0 : (int64_t)(v - S.rhs0) * Nt * sv);
    const RS beta = (RS)st.beta[v];
    const bool has_old = st.iters[v] > 0;
    // the previous iteration's x += alpha p, applied here on the slab's own
    // slices while p_old is in registers anyway
    const bool pend = st.pending[v];
    const RS al_old = (RS)st.alpha[v];
    RS* xl = xs + vb;
    const SP* pold = reinterpret_cast<const SP*>((st.iters[v] & 1) ? p.p0 : p.p1) + vb;
    SP* pnew = reinterpret_cast<SP*>((st.iters[v] & 1) ? p.p1 : p.p0) + vb;
    // storage scales (1 unless scaled fp16): z, p_old, and p_new's, set to
    // z's at the start of the phase
    const RS s_z = sc_z(v), s_po = sc_p((st.iters[v] & 1) ^ 1, v);
    const RS s_pn = sc_p(st.iters[v] & 1, v), i_pn = (RS)1 / s_pn;
    const SP* zz = (guess_pass ? reinterpret_cast<const SP*>(xs)
                               : (S.precon || LOWP) ? zbuf : reinterpret_cast<const SP*>(r)) + vb;
    RS* O = Op + vb;
    const RS t1 = (RS)p.t1, th = (RS)p.th, Cb = (RS)p.Cb;
    Cx<RS> X0[BY][2], X1[BY][2], Y[BY][2];
    Cx<RS> Yp[STASH_S ? 1 : BY][2];
    double pap = 0;
    auto getp = [&](Cx<RS> (&X)[BY][2], int t, bool own) {
      if (!E.on) return;
      E.load_st(X, zz + t * sv, s_z);
      if (has_old) {
        Cx<RS> T0[BY][2];
        E.load_st(T0, pold + t * sv, s_po);
        if (own && pend) {
          Cx<RS> XL[BY][2];
          E.load_coherent(XL, xl + t * sv);
#pragma unroll
          for (int q = 0; q < BY; ++q)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              XL[q][c].re = fma(al_old, T0[q][c].re, XL[q][c].re);
              XL[q][c].im = fma(al_old, T0[q][c].im, XL[q][c].im);
            }
          E.store(xl + t * sv, XL);
        }
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            X[q][c].re = fma(beta, T0[q][c].re, X[q][c].re);
            X[q][c].im = fma(beta, T0[q][c].im, X[q][c].im);
            X[q][c] = round_st<SP>(X[q][c], s_pn, i_pn);
          }
      } else if constexpr (H16) {
        // p = z, stored at p's own scale (exact unless entries turn subnormal)
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) X[q][c] = round_st<SP>(X[q][c], s_pn, i_pn);
      }
    };
    const int tp = (a - 1 + Nt) % Nt;
    getp(X0, tp, false);
    getp(X1, a, true);
    if (E.on) E.store_st(pnew + a * sv, X1, i_pn);
    double ppp = 0;  // |p_new|^2 over the own slices (scaled fp16 storage)
    if constexpr (H16) ppp += sq_blk<RS, BY>(X1, E.on);
    A ang[BY][4];
    if constexpr (!PHS_S) E.load_angles(ang, phi + a * sv);
    E.phases(phi + tp * sv, t1, th);
    E.template applyB<FAC_TILDE>(X0);
    axpy_blk<RS, BY>(Y, X1, sigma_of<RS>(tp, Nt) * Cb, X0);  // y_a
    if constexpr (STASH_S) E.park(Y); else copy_blk<RS, BY>(Yp, Y);
    copy_blk<RS, BY>(X0, X1);
    for (int t = a; t < bnd; ++t) {
      const int tn = (t + 1) % Nt;
      getp(X1, tn, t + 1 < bnd);
      if (E.on && t + 1 < bnd) E.store_st(pnew + tn * sv, X1, i_pn);
      if constexpr (H16) ppp += sq_blk<RS, BY>(X1, E.on && t + 1 < bnd);
      if constexpr (!PHS_S) {
        E.phases_from(ang, t1, th);
        if (t + 1 < bnd) E.load_angles(ang, phi + (t + 1) * sv);
      } else {
        E.phases(phi + t * sv, t1, th);
      }
      const RS sg = sigma_of<RS>(t, Nt) * Cb;
      E.template applyB<FAC_TILDE>(X0);       // B_t p_t
      axpy_blk<RS, BY>(Y, X1, sg, X0);         // y_{t+1}
      if constexpr (STASH_S) {
        E.unpark(X0);                          // y_t
        E.park(Y);
      } else {
        copy_blk<RS, BY>(X0, Yp);
        copy_blk<RS, BY>(Yp, Y);
      }
      if (E.on) {
        RS sq = 0;  // the tile's |y_t|^2 in the iteration precision, then double
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) sq = fma(X0[q][c].re, X0[q][c].re, fma(X0[q][c].im, X0[q][c].im, sq));
        pap += (double)sq;
      }
      E.template applyB<FAC_TILDE, 1>(Y);     // B_t y_{t+1}
      if (E.on) {
        axpy_blk<RS, BY>(Y, X0, sg, Y);        // (M^dag M p)_t
        E.store(O + t * sv, Y);
      }
      copy_blk<RS, BY>(X0, X1);
    }
    if constexpr (H16) {
      double sa = pap, sb = ppp, sc = 0;
      block_sum3_d(sa, sb, sc, st.red);
      if (tid == 0) {
        atomicAdd(acc.pAp + slot * NV + v, sa);
        atomicAdd(acc.pp + slot * NV + v, sb);
      }
    } else {
      const double sum = block_sum_d(pap, st.red);
      if (tid == 0) atomicAdd(acc.pAp + slot * NV + v, sum);
    }
    __syncthreads();
    }
  };

  // The same pass with the slices of z, p_old and x_lo staged whole in shared
  // memory (EC_STAGE): stage j holds slice tp + j of the sequence tp, a, ...,
  // bnd (bulk copies issued by thread 0 one slice ahead), so the slice loop
  // reads its inputs from shared memory and never waits on a global load.
  auto operator_unit_staged = [&](int u, int slot) {
    if constexpr (STG_S) {
    const int s = find_sys_A(p, u);
    const PcgSys& S = p.sys[s];
    const int lu = u - S.unitA0;
    const int v = S.rhs0 + lu / S.nslab;
    const int a = (lu % S.nslab) * S.T;
    const int bnd = min(a + S.T, S.Nt);
    const int Nt = S.Nt, Vs = SL(S) * SL(S);
    const size_t sv = 2 * (size_t)Vs;
    Slice<RS, BY, PHS_S, XS_S, LT> E;
    E.init(SL(S), dsm, 2, (RS)p.c1, (RS)p.ch, tid);
    const int64_t vb = 2 * vec_base(s, v);
    const A* phi = phi_all + S.phi0 + (S.shared ? 0 : (int64_t)(v - S.rhs0) * Nt * sv);
    const RS beta = (RS)st.beta[v];
    const bool has_old = st.iters[v] > 0;
    const bool pend = st.pending[v];
    const RS al_old = (RS)st.alpha[v];
    RS* xl = xs + vb;
    const SP* pold = reinterpret_cast<const SP*>((st.iters[v] & 1) ? p.p0 : p.p1) + vb;
    SP* pnew = reinterpret_cast<SP*>((st.iters[v] & 1) ? p.p1 : p.p0) + vb;
    // storage scales (1 unless scaled fp16): z, p_old, and p_new's, set to
    // z's at the start of the phase
    const RS s_z = sc_z(v), s_po = sc_p((st.iters[v] & 1) ^ 1, v);
    const RS s_pn = sc_p(st.iters[v] & 1, v), i_pn = (RS)1 / s_pn;
    const SP* zz = (guess_pass ? reinterpret_cast<const SP*>(xs)
                               : (S.precon || LOWP) ? zbuf : reinterpret_cast<const SP*>(r)) + vb;
    RS* O = Op + vb;
    const RS t1 = (RS)p.t1, th = (RS)p.th, Cb = (RS)p.Cb;
    // slots of the iteration precision; z and p_old may be narrower
    stg.bytes = (unsigned)(Vs * 2 * sizeof(RS));
    stg.sizes[0] = stg.sizes[1] = (unsigned)(Vs * 2 * sizeof(SP));
    stg.sizes[2] = stg.bytes;
    const int nT = bnd - a;  // own slices
    const int tp = (a - 1 + Nt) % Nt;
    auto slice_of = [&](int j) { const int t = tp + j; return t >= Nt ? t - Nt : t; };
    auto issue = [&](int j) {
      if (tid != 0 || j > nT + 1) return;
      const int t = slice_of(j);
      const void* src[3] = {zz + t * sv, pold + t * sv, xl + t * sv};
      const bool own = j >= 1 && j <= nT;
      stg.issue(j, src, 1u | (has_old ? 2u : 0u) | ((own && pend && has_old) ? 4u : 0u));
    };
    auto wait = [&](int j) {
      if (!stg.wait(j, budget_stage)) atomicExch(p.bar + 2, (unsigned int)QEDF_ERR_TIMEOUT);
    };
    // p = z + beta p_old of stage j, rounded to the storage; on own slices
    // also x_lo += alpha_old p_old
    auto getp = [&](Cx<RS> (&X)[BY][2], int j, bool own) {
      if (!E.on) return;
      E.load_st(X, reinterpret_cast<const SP*>(stg.slot(j, 0)), s_z);
      if (has_old) {
        Cx<RS> T0[BY][2];
        E.load_st(T0, reinterpret_cast<const SP*>(stg.slot(j, 1)), s_po);
        if (own && pend) {
          Cx<RS> XL[BY][2];
          E.load_coherent(XL, reinterpret_cast<const RS*>(stg.slot(j, 2)));
#pragma unroll
          for (int q = 0; q < BY; ++q)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              XL[q][c].re = fma(al_old, T0[q][c].re, XL[q][c].re);
              XL[q][c].im = fma(al_old, T0[q][c].im, XL[q][c].im);
            }
          E.store(xl + slice_of(j) * sv, XL);
        }
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            X[q][c].re = fma(beta, T0[q][c].re, X[q][c].re);
            X[q][c].im = fma(beta, T0[q][c].im, X[q][c].im);
            X[q][c] = round_st<SP>(X[q][c], s_pn, i_pn);
          }
      } else if constexpr (H16) {
        // p = z, stored at p's own scale (exact unless entries turn subnormal)
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) X[q][c] = round_st<SP>(X[q][c], s_pn, i_pn);
      }
    };
    Cx<RS> X0[BY][2], X1[BY][2], Y[BY][2];
    double pap = 0;
    issue(0);
    issue(1);
    wait(0);
    getp(X0, 0, false);
    wait(1);
    getp(X1, 1, true);
    if (E.on) E.store_st(pnew + a * sv, X1, i_pn);
    double ppp = 0;  // |p_new|^2 over the own slices (scaled fp16 storage)
    if constexpr (H16) ppp += sq_blk<RS, BY>(X1, E.on);
    A ang[BY][4];
    if constexpr (!PHS_S) E.load_angles(ang, phi + a * sv);
    E.phases(phi + tp * sv, t1, th);  // block barrier: stage 0 is read
    issue(2);
    E.template applyB<FAC_TILDE>(X0);
    axpy_blk<RS, BY>(Y, X1, sigma_of<RS>(tp, Nt) * Cb, X0);  // y_a
    E.park(Y);
    copy_blk<RS, BY>(X0, X1);
    for (int i = 0; i < nT; ++i) {
      const int t = a + i, tn = (t + 1) % Nt;
      issue(i + 3);  // into the buffer of stage i + 1, read before the last barriers
      wait(i + 2);
      getp(X1, i + 2, t + 1 < bnd);
      if (E.on && t + 1 < bnd) E.store_st(pnew + tn * sv, X1, i_pn);
      if constexpr (H16) ppp += sq_blk<RS, BY>(X1, E.on && t + 1 < bnd);
      if constexpr (!PHS_S) {
        E.phases_from(ang, t1, th);
        if (t + 1 < bnd) E.load_angles(ang, phi + (t + 1) * sv);
      } else {
        E.phases(phi + t * sv, t1, th);
      }
      const RS sg = sigma_of<RS>(t, Nt) * Cb;
      E.template applyB<FAC_TILDE>(X0);       // B_t p_t
      axpy_blk<RS, BY>(Y, X1, sg, X0);         // y_{t+1}
      E.unpark(X0);                            // y_t
      E.park(Y);
      if (E.on) {
        RS sq = 0;
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) sq = fma(X0[q][c].re, X0[q][c].re, fma(X0[q][c].im, X0[q][c].im, sq));
        pap += (double)sq;
      }
      E.template applyB<FAC_TILDE, 1>(Y);     // B_t y_{t+1}
      if (E.on) {
        axpy_blk<RS, BY>(Y, X0, sg, Y);        // (M^dag M p)_t
        E.store(O + t * sv, Y);
      }
      copy_blk<RS, BY>(X0, X1);
    }
    if constexpr (H16) {
      double sa = pap, sb = ppp, sc = 0;
      block_sum3_d(sa, sb, sc, st.red);
      if (tid == 0) {
        atomicAdd(acc.pAp + slot * NV + v, sa);
        atomicAdd(acc.pp + slot * NV + v, sb);
      }
    } else {
      const double sum = block_sum_d(pap, st.red);
      if (tid == 0) atomicAdd(acc.pAp + slot * NV + v, sum);
    }
    __syncthreads();
    }
  };

  // r = b - M^dag M x in the high precision (mixed mode), rr_true
  auto operator_unit_true_residual = [&](int u) {
    const int s = find_sys_A(p, u);
    const PcgSys& S = p.sys[s];
    const int lu = u - S.unitA0;
    const int v = S.rhs0 + lu / S.nslab;
    const int a = (lu % S.nslab) * S.T;
    const int bnd = min(a + S.T, S.Nt);
    const int Nt = S.Nt, Vs = SL(S) * SL(S);
    const size_t sv = 2 * (size_t)Vs;
    Slice<RH, BY, PHS_H, false, LT> E;
    E.init(SL(S), dsm, 2, (RH)p.c1, (RH)p.ch, tid);
    const int64_t vb = 2 * vec_base(s, v);
    const A* phi = phi_all + S.phi0 + (S.shared ? 0 : (int64_t)(v - S.rhs0) * Nt * sv);
    const RH* xx = xh + vb;
    const RH* bb = bvec + vb;
    RS* rout = r + vb;
    const RH t1 = (RH)p.t1, th = (RH)p.th, Cb = (RH)p.Cb;
    Cx<RH> X0[BY][2], X1[BY][2], Y[BY][2];
    Cx<RH> Yp[STASH_H ? 1 : BY][2];
    double rr_acc = 0;
    const int tp = (a - 1 + Nt) % Nt;
    if (E.on) {
      E.load_coherent(X0, xx + tp * sv);
      E.load_coherent(X1, xx + a * sv);
    }
    E.phases(phi + tp * sv, t1, th);
    E.template applyB<FAC_TILDE>(X0);
    axpy_blk<RH, BY>(Y, X1, sigma_of<RH>(tp, Nt) * Cb, X0);
    if constexpr (STASH_H) E.park(Y); else copy_blk<RH, BY>(Yp, Y);
    copy_blk<RH, BY>(X0, X1);
    for (int t = a; t < bnd; ++t) {
      const int tn = (t + 1) % Nt;
      if (E.on) E.load_coherent(X1, xx + tn * sv);
      E.phases(phi + t * sv, t1, th);
      const RH sg = sigma_of<RH>(t, Nt) * Cb;
      E.template applyB<FAC_TILDE>(X0);
      axpy_blk<RH, BY>(Y, X1, sg, X0);
      if constexpr (STASH_H) {
        E.unpark(X0);
        E.park(Y);
      } else {
        copy_blk<RH, BY>(X0, Yp);
        copy_blk<RH, BY>(Yp, Y);
      }
      E.template applyB<FAC_TILDE, 1>(Y);
      if (E.on) {
        axpy_blk<RH, BY>(Y, X0, sg, Y);  // (A x)_t
        E.load_coherent(X0, bb + t * sv);
#pragma unroll
        for (int q = 0; q < BY; ++q)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const RH dr = X0[q][c].re - Y[q][c].re, di = X0[q][c].im - Y[q][c].im;
            rr_acc += (double)dr * dr + (double)di * di;
            const int64_t site = (int64_t)t * Vs + (E.y0 + q) * SL(S) + E.x0 + c;
            rout[2 * site] = (RS)dr;
            rout[2 * site + 1] = (RS)di;
          }
      }
      copy_blk<RH, BY>(X0, X1);
    }
    const double sum = block_sum_d(rr_acc, st.red);
    if (tid == 0) atomicAdd(acc.ru_rr + v, sum);
    __syncthreads();
  };

  // the pending x += alpha p_last of right-hand side v at one site pair
  auto apply_pending = [&](int v, int64_t i2, Cx<RS>& l0, Cx<RS>& l1) {
    if (!st.pending[v]) return;
    const SP* pl = reinterpret_cast<const SP*>((st.iters[v] & 1) ? p.p0 : p.p1);  // p of the last iteration
    const RS al = (RS)st.alpha[v];
    Cx<RS> p0v, p1v;
    ld2s(pl + i2, p0v, p1v, sc_p((st.iters[v] & 1) ^ 1, v));
    l0 = mk<RS>(fma(al, p0v.re, l0.re), fma(al, p0v.im, l0.im));
    l1 = mk<RS>(fma(al, p1v.re, l1.re), fma(al, p1v.im, l1.im));
  };

  // x (double) += x_lo (+ the pending update); x_lo = 0   for the flagged
  // right-hand sides (all_active: every one still active or with a pending
  // update, at the end of the solve)
  auto fold_unit = [&](int u, bool all_active) {
    int s, v, c0, c1;
    unitE(u, s, v, c0, c1);
    if (!(all_active ? (st.active[v] || st.pending[v]) : st.ru[v])) return;
    const PcgSys& S = p.sys[s];
    const int Vs = SL(S) * SL(S), w = c1 - c0;
    const int64_t base = vec_base(s, v);
    const int j = tid % PPR;
    if (2 * j >= w) return;
    for (int t = tid / PPR; t < S.Nt; t += blockDim.x / PPR) {
      const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
      Cx<RS> l0, l1;
      Cx<RH> h0, h1;
      ld2s(xs + i2, l0, l1);
      apply_pending(v, i2, l0, l1);
      ld2c(xh + i2, h0, h1);
      h0.re += (RH)l0.re;
      h0.im += (RH)l0.im;
      h1.re += (RH)l1.re;
      h1.im += (RH)l1.im;
      st2(xh + i2, h0, h1);
      st2s(xs + i2, mk<RS>(0, 0), mk<RS>(0, 0));
    }
  };

  // x = 0 for a right-hand side with b = 0 (its guess is replaced by the
  // exact solution)
  auto zero_x_unit = [&](int u) {
    int s, v, c0, c1;
    unitE(u, s, v, c0, c1);
    if (acc.bb[v] != 0.0) return;
    const PcgSys& S = p.sys[s];
    const int Vs = SL(S) * SL(S), w = c1 - c0;
    const int64_t base = vec_base(s, v);
    const int j = tid % PPR;
    if (2 * j >= w) return;
    for (int t = tid / PPR; t < S.Nt; t += blockDim.x / PPR) {
      const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
      st2(xh + i2, mk<RH>(0, 0), mk<RH>(0, 0));
    }
  };

  // plain modes, end of the solve: x += alpha p_last where still pending
  auto flush_unit = [&](int u) {
    int s, v, c0, c1;
    unitE(u, s, v, c0, c1);
    if (!st.pending[v]) return;
    const PcgSys& S = p.sys[s];
    const int Vs = SL(S) * SL(S), w = c1 - c0;
    const int64_t base = vec_base(s, v);
    const int j = tid % PPR;
    if (2 * j >= w) return;
    for (int t = tid / PPR; t < S.Nt; t += blockDim.x / PPR) {
      const int64_t i2 = 2 * (base + (int64_t)t * Vs + c0 + 2 * j);
      Cx<RS> l0, l1;
      ld2s(xs + i2, l0, l1);
      apply_pending(v, i2, l0, l1);
      st2s(xs + i2, l0, l1);
    }
  };

  // ---------------------------------------------------------------------------
  const long long budget = p.timeout_cycles;
  unsigned int bar_target = 0;  // grid barrier count to wait for (thread 0)
  bool ok = true;
  PhaseClock pc(p.prof);
  const long long t_begin = pc.prof ? clock64() : 0;

  // init: x = 0, r = b, z = P r
  for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) elementwise(0, u, 0);
  ok = grid_barrier(p.bar, nblk, budget, bar_target);
  int slot = 0;  // accumulator slot holding the current rr / rz
  if (ok) {
    for (int v = tid; v < NV; v += blockDim.x) {
      st.rz[v] = acc.rz[v];
      st.rzold[v] = 1.0;
      st.rr[v] = acc.rr[v];
      const double bbv = acc.bb[v];
      if (bbv == 0.0) {  // b = 0: x = 0 is exact
        st.active[v] = 0;
        st.res[v] = 0.0;
      }
    }
    __syncthreads();
  }
  if constexpr (H16) {
    // z = P r now that |r| = |b| fixes z's scale; r^dag z into the rz slot,
    // which the init pass left at zero
    if (ok) {
      for (int v = tid; v < NV; v += blockDim.x) scl.z[v] = st_scale(st.rr[v]);
      __syncthreads();
      for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) elementwise(3, u, 0);
      ok = grid_barrier(p.bar, nblk, budget, bar_target);
    }
    if (ok) {
      for (int v = tid; v < NV; v += blockDim.x) st.rz[v] = acc.rz[v];
      __syncthreads();
    }
  }
  // initial guess: a right-hand side with b = 0 gets x = 0.  Mixed modes start
  // the others with a reliable update (r = b - A x in double, z = P r); plain
  // modes with one pass of the iteration's own two phases on p = x (guess
  // pass: Op = A x, then r = b - 1 * Op and z = P r), which counts no
  // iteration and updates no x
  if (ok && p.x_init) {
    for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) zero_x_unit(u);
    guess_pass = !MIXED;
  }
  pc.lap(0);

  int it = 0;
  while (ok) {
    // ---- convergence / reliable-update decisions (identical in every block)
    if (tid == 0) {
      st.any_ru = 0;
      st.any_active = 0;
    }
    __syncthreads();
    for (int v = tid; v < NV; v += blockDim.x) {
      st.ru[v] = 0;
      if (!st.active[v]) continue;
      const double bbv = acc.bb[v];
      const double res = sqrt(st.rr[v] / bbv);
      st.res[v] = res;
      if (!isfinite(res)) {
        st.active[v] = 0;
        st.status[v] = QEDF_ERR_NAN;
        continue;
      }
      if (MIXED) {
        // (the initial guess's residual is a reliable update's)
        if (res <= p.rtol || it - st.lastru[v] >= p.ru_interval || res < p.ru_delta * st.resmax[v] ||
            (it == 0 && p.x_init)) {
          st.ru[v] = 1;
          st.any_ru = 1;
        }
      } else if (res <= p.rtol) {
        st.active[v] = 0;
      }
    }
    __syncthreads();
    if (MIXED && st.any_ru) {
      pc.lap(6);
      if (blockIdx.x == 0)
        for (int v = tid; v < NV; v += blockDim.x) {
          acc.ru_rr[v] = 0;
          acc.ru_rz[v] = 0;
        }
      for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) fold_unit(u, false);
      if (!(ok = grid_barrier(p.bar, nblk, budget, bar_target))) break;
      for (int u = blockIdx.x; u < p.unitsA; u += gridDim.x) {
        const int s = find_sys_A(p, u);
        const int v = p.sys[s].rhs0 + (u - p.sys[s].unitA0) / p.sys[s].nslab;
        if (st.ru[v]) operator_unit_true_residual(u);
      }
      if (!(ok = grid_barrier(p.bar, nblk, budget, bar_target))) break;
      if constexpr (H16) {
        for (int v = tid; v < NV; v += blockDim.x)
          if (st.ru[v]) scl.z[v] = st_scale(acc.ru_rr[v]);
        __syncthreads();
      }
      for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) {
        int s, v, c0, c1;
        unitE(u, s, v, c0, c1);
        if (st.ru[v]) elementwise(2, u, 0);
      }
      if (!(ok = grid_barrier(p.bar, nblk, budget, bar_target))) break;
      for (int v = tid; v < NV; v += blockDim.x) {
        if (!st.ru[v]) continue;
        st.pending[v] = 0;  // folded into x above
        st.rr[v] = acc.ru_rr[v];
        st.rz[v] = acc.ru_rz[v];
        const double res = sqrt(st.rr[v] / acc.bb[v]);
        st.res[v] = res;
        st.resmax[v] = res;
        st.lastru[v] = it;
        if (!isfinite(res)) {
          st.active[v] = 0;
          st.status[v] = QEDF_ERR_NAN;
        } else if (res <= p.rtol) {
          st.active[v] = 0;
        }
      }
      __syncthreads();
      pc.lap(5);
    }
    for (int v = tid; v < NV; v += blockDim.x)
      if (st.active[v]) st.any_active = 1;
    __syncthreads();
    if (!st.any_active || it >= p.max_iter) break;

    // ---- phase A
    for (int v = tid; v < NV; v += blockDim.x) {
      st.beta[v] = st.iters[v] > 0 ? st.rz[v] / st.rzold[v] : 0.0;
      if constexpr (H16)
        if (st.active[v]) {
          // the scale of the buffer p_new goes to, from a bound of its norm:
          // |z + beta p_old| <= |P| |r| + beta |p_old| (|p_old| measured in the
          // last operator phase); p grows far above r in ill-conditioned solves
          double est = p.pnorm * sqrt(st.rr[v]);
          if (st.iters[v] > 0) est += fabs(st.beta[v]) * sqrt(acc.pp[((it & 1) ^ 1) * NV + v]);
          scl.p[st.iters[v] & 1][v] = st_scale(est * est);
        }
    }
    __syncthreads();
    // (the guess pass uses the pAp slot of odd iterations, so that its BC
    // phase clears the slot of iteration 0)
    const int aslot = guess_pass ? 1 : it & 1;
    for (int u = blockIdx.x; u < p.unitsA; u += gridDim.x) {
      const int s = find_sys_A(p, u);
      const int v = p.sys[s].rhs0 + (u - p.sys[s].unitA0) / p.sys[s].nslab;
      if (st.active[v]) {
        if constexpr (STG_S) operator_unit_staged(u, aslot);
        else operator_unit_sloppy(u, aslot);
      }
    }
    // the rr/rz slot that BC will fill was last read before the previous barrier
    if (blockIdx.x == 0)
      for (int v = tid; v < NV; v += blockDim.x) {
        acc.rr[(slot ^ 1) * NV + v] = 0;
        acc.rz[(slot ^ 1) * NV + v] = 0;
      }
    pc.lap(1);
    if (!(ok = grid_barrier(p.bar, nblk, budget, bar_target))) break;
    pc.lap(2);

    // ---- phase BC
    // alpha of inactive systems stays that of their last iteration: a pending
    // x update still uses it
    for (int v = tid; v < NV; v += blockDim.x)
      if (st.active[v]) {
        st.alpha[v] = guess_pass ? 1.0 : st.rz[v] / acc.pAp[aslot * NV + v];
        if constexpr (H16) scl.z[v] = st_scale(st.rr[v]);  // |r| before this update
      }
    __syncthreads();
    for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) {
      int s, v, c0, c1;
      unitE(u, s, v, c0, c1);
      if (st.active[v]) elementwise(1, u, slot ^ 1);
    }
    if (blockIdx.x == 0)  // pAp (and |p|^2) slot of the next iteration
      for (int v = tid; v < NV; v += blockDim.x) {
        acc.pAp[(aslot ^ 1) * NV + v] = 0;
        if constexpr (H16) acc.pp[(aslot ^ 1) * NV + v] = 0;
      }
    pc.lap(3);
    if (!(ok = grid_barrier(p.bar, nblk, budget, bar_target))) break;
    pc.lap(4);
    slot ^= 1;
    for (int v = tid; v < NV; v += blockDim.x) {
      if (!st.active[v]) continue;
      st.rzold[v] = st.rz[v];
      st.rz[v] = acc.rz[slot * NV + v];
      st.rr[v] = acc.rr[slot * NV + v];
      if (guess_pass) continue;
      st.iters[v] += 1;
      st.pending[v] = 1;
    }
    __syncthreads();
    if (guess_pass) guess_pass = false;
    else ++it;
    pc.lap(6);
  }
  if (pc.prof) {
    pc.prof[7] += clock64() - t_begin;
  }

  // mixed: fold the remaining float updates of unconverged systems into x;
  // plain: apply the last iteration's x update
  if (MIXED && ok) {
    for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) fold_unit(u, true);
  } else if (ok) {
    for (int u = blockIdx.x; u < p.unitsE; u += gridDim.x) flush_unit(u);
  }
  if (blockIdx.x == 0) {
    const unsigned int err = *((volatile unsigned int*)(p.bar + 2));
    for (int v = tid; v < NV; v += blockDim.x) {
      int stt = st.status[v];
      if (err) stt = (int)err;
      else if (stt == QEDF_OK && st.active[v]) stt = QEDF_ERR_MAXITER;
      p.status[v] = stt;
      p.iters[v] = st.iters[v];
      p.relres[v] = st.res[v];
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
// shared memory of the operator passes' slice stages: 2 buffers x 3 slices of
// the iteration precision RS
template <typename RS>
static size_t pcg_stage_bytes(int L) { return 2 * 3 * (size_t)L * L * 2 * sizeof(RS); }

// (MIXED_BF16 and MIXED_F16 keep r, M^dag M p and x_lo in float; their p and z buffers use
// half of their float-sized room)
int pcg_storage_bytes(int mode) { return mode == QEDF_PCG_PLAIN_F64 ? 8 : 4; }

// Slab length of the operator units: units are dealt to the blocks in turn,
// so the busiest block runs ceil(units / nblk) units of T slices plus one
// halo slice each.  The T that minimises that count wins (the longer T on
// ties: fewer units, fewer per-unit reductions).
static int auto_slab(const qedf_system* sys, int nsys, int nblk) {
  int ntmax = 1;
  for (int k = 0; k < nsys; ++k) ntmax = std::max(ntmax, sys[k].Ltau);
  int best = ntmax;
  long long best_cost = -1;
  for (int T = ntmax; T >= 1; --T) {
    long long units = 0;
    for (int k = 0; k < nsys; ++k) units += (long long)sys[k].nrhs * ((sys[k].Ltau + T - 1) / T);
    const long long cost = (units + nblk - 1) / nblk * (T + 1);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = T;
    }
  }
  return best;
}

int pcg_plan(PcgParams& p, const qedf_system* sys, int nsys, const qedf_pcg_opts* o) {
  std::memset(&p, 0, sizeof(p));
  if (!sys || !o || nsys <= 0 || nsys > PCG_MAX_SYS) return QEDF_ERR_ARG;
  if (o->mode != QEDF_PCG_PLAIN_F32 && o->mode != QEDF_PCG_PLAIN_F64 && o->mode != QEDF_PCG_MIXED &&
      o->mode != QEDF_PCG_MIXED_BF16 && o->mode != QEDF_PCG_MIXED_F16)
    return QEDF_ERR_ARG;
  p.mode = o->mode;
  p.nsys = nsys;
  p.xs = 1;
  p.stage = o->stage > 0 ? 1 : 0;
  p.x_init = o->x_init > 0 ? 1 : 0;
  p.l2 = o->l2_persist < 0 ? -1 : 0;
  if (o->chunk != 0 && o->chunk != 16 && o->chunk != 32) return QEDF_ERR_ARG;
  // 32-site elementwise units (one longer tau column per block) fit where
  // their r column and the single-precision staging fit in shared memory next
  // to the per-block state
  int ntmax_all = 0;
  for (int s = 0; s < nsys; ++s) ntmax_all = std::max(ntmax_all, sys[s].Ltau);
  const bool wide_fits = o->mode != QEDF_PCG_PLAIN_F64 && ntmax_all <= 500;
  if (o->chunk == 32 && !wide_fits) return QEDF_ERR_SIZE;
  // 16 by default: the wider units' shared memory takes L1 from the operator
  // phase (measured at L = 48: elementwise phase -11 %, operator phase +11 %)
  p.CH = o->chunk ? o->chunk : PCG_CHUNK;
  const int nblk = num_sms();
  int rhs = 0, ua = 0, ue = 0, pt = 0;
  int64_t vec = 0, phi = 0;
  for (int s = 0; s < nsys; ++s) {
    const qedf_system& q = sys[s];
    if (q.Lx < 2 || q.Lx % 2 || q.Ltau < 2 || q.nrhs < 1) return QEDF_ERR_ARG;
    PcgSys& S = p.sys[s];
    S.L = q.Lx;
    S.Nt = q.Ltau;
    S.nrhs = q.nrhs;
    S.shared = q.shared_boson ? 1 : 0;
    S.precon = (o->use_precon && q.Ltau >= PRE_MIN_LTAU) ? 1 : 0;
    S.T = o->slab > 0 ? o->slab : auto_slab(sys, nsys, nblk);
    // the preconditioner rows that are the bulk band (middle values at every
    // distance, nothing else): one contiguous range away from both tau ends
    S.pmid_lo = S.pmid_hi = 0;
    if (S.precon) {
      int lo = -1, hi = -1;
      for (int t = 0; t < q.Ltau; ++t) {
        bool mid = t >= 6 && t + 6 < q.Ltau;
        int cnt = 0;
        pre_row(h_pre, q.Ltau, t, [&](int c, float val) {
          const int d = c > t ? c - t : t - c;
          mid = mid && d <= 6 && val == h_pre.middle[d];
          ++cnt;
        });
        mid = mid && cnt == 13;
        if (mid && lo < 0) lo = t;
        if (mid) hi = t + 1;
      }
      if (lo >= 0) {
        S.pmid_lo = lo;
        S.pmid_hi = hi;
      }
    }
    S.nslab = (q.Ltau + S.T - 1) / S.T;
    S.nchunk = (q.Lx * q.Lx + p.CH - 1) / p.CH;
    S.rhs0 = rhs;
    S.unitA0 = ua;
    S.unitE0 = ue;
    S.vec0 = vec;
    S.phi0 = phi;
    S.ptab0 = pt;
    pt += 13 * q.Ltau;
    rhs += q.nrhs;
    ua += q.nrhs * S.nslab;
    ue += q.nrhs * S.nchunk;
    vec += (int64_t)q.nrhs * q.Ltau * q.Lx * q.Lx;
    phi += (int64_t)(S.shared ? 1 : q.nrhs) * q.Ltau * q.Lx * q.Lx * 2;
  }
  if (rhs > PCG_MAX_RHS) return QEDF_ERR_SIZE;
  p.nrhs = rhs;
  p.unitsA = ua;
  p.unitsE = ue;
  p.nvec_total = vec;
  p.ptab_len = pt;
  p.max_iter = o->max_iter;
  p.rtol = o->rtol;
  // defaults measured on the benchmark solve: every 100 iterations or a
  // hundredfold residual drop take the iteration count of 50 / tenfold with
  // half the reliable-update time
  p.ru_interval = o->ru_interval > 0 ? o->ru_interval : 100;
  p.ru_delta = o->ru_delta > 0 ? o->ru_delta : 0.01;
  const FactorCoeffs f = factor_coeffs(o->dtau);
  p.c1 = f.c1;
  p.ch = f.ch;
  p.t1 = f.t1;
  p.th = f.th;
  p.Cb = f.Cb;
  // largest absolute row sum of the systems' preconditioners (a bound of its
  // 2-norm, P being symmetric); 1 for the identity
  p.pnorm = 1.0;
  for (int s = 0; s < nsys; ++s) {
    if (!p.sys[s].precon) continue;
    for (int t = 0; t < p.sys[s].Nt; ++t) {
      double row = 0;
      pre_row(h_pre, p.sys[s].Nt, t, [&](int, float val) { row += std::fabs((double)val); });
      p.pnorm = std::max(p.pnorm, row);
    }
  }
  return QEDF_OK;
}

// The workspace layout, in one place: r, p0, p1, z, Op (and x_lo in mixed
// mode) in the sloppy precision, the double accumulators (ACC_PER_RHS per
// right-hand side), 256 bytes of grid-barrier words and the preconditioner
// tables, each 256-byte aligned.  Returns the bytes the layout needs; with a
// workspace it also points p's buffers into it, and *zero_bytes receives the
// length of the block that starts at zero every solve (accumulators and
// barrier words, contiguous from p.acc).
size_t pcg_carve(PcgParams& p, int sloppy_bytes, void* workspace, size_t* zero_bytes) {
  const size_t vecb = align_up((size_t)p.nvec_total * 2 * sloppy_bytes, 256);
  const bool mixed = p.mode == QEDF_PCG_MIXED || p.mode == QEDF_PCG_MIXED_BF16 || p.mode == QEDF_PCG_MIXED_F16;
  const int nv = mixed ? 6 : 5;
  const size_t accb = align_up(sizeof(double) * ACC_PER_RHS * p.nrhs, 256);
  const size_t barb = 256;
  const size_t tabb = align_up(sizeof(float) * (size_t)p.ptab_len, 256);
  if (zero_bytes) *zero_bytes = accb + barb;
  if (workspace) {
    unsigned char* w = static_cast<unsigned char*>(workspace);
    p.r = w;
    p.p0 = w + vecb;
    p.p1 = w + 2 * vecb;
    p.z = w + 3 * vecb;
    p.Op = w + 4 * vecb;
    p.xlo = mixed ? w + 5 * vecb : nullptr;
    p.acc = reinterpret_cast<double*>(w + nv * vecb);
    p.bar = reinterpret_cast<unsigned int*>(w + nv * vecb + accb);
    p.ptab = reinterpret_cast<float*>(w + nv * vecb + accb + barb);
  }
  return nv * vecb + accb + barb + tabb;
}

size_t pcg_workspace_bytes(const PcgParams& p, int sloppy_bytes) {
  PcgParams q = p;
  return pcg_carve(q, sloppy_bytes, nullptr, nullptr);
}

// Per solve: zero the accumulators and barrier words, and write each system's
// periodic 13-band preconditioner table (entry k of row t multiplies r at
// tau = t + k - 6 mod Nt).
__global__ void k_pcg_prep(const __grid_constant__ PcgParams p, int zero_words) {
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int* z = reinterpret_cast<unsigned int*>(p.acc);
  for (int i = i0; i < zero_words; i += gridDim.x * blockDim.x) z[i] = 0u;
  for (int s = 0; s < p.nsys; ++s) {
    const int Nt = p.sys[s].Nt;
    float* tab = p.ptab + p.sys[s].ptab0;
    for (int e = i0; e < 13 * Nt; e += gridDim.x * blockDim.x) tab[e] = 0.f;
  }
  __syncthreads();
  // rows are independent; each thread fills whole rows (duplicate-free)
  for (int s = 0; s < p.nsys; ++s) {
    const int Nt = p.sys[s].Nt;
    if (!p.sys[s].precon) continue;
    float* tab = p.ptab + p.sys[s].ptab0;
    for (int t = i0; t < Nt; t += gridDim.x * blockDim.x)
      pre_row(c_pre, Nt, t, [&](int col, float val) {
        int k = col - t + 6;
        if (k < 0) k += Nt;
        if (k >= Nt) k -= Nt;
        tab[t * 13 + k] += val;
      });
  }
}

// L2 persistence for the iteration vectors.  p_old / p_new (p0, p1), z and
// M^dag M p (Op) are contiguous in the workspace; each is written in one phase
// and read in the next.  The launch carries an access-policy window over the
// four (z and Op alone when four exceed the largest window) whose hit ratio
// fits them to the context's persisting set-aside as it is: the limit is
// never changed, since a larger set-aside takes L2 from every other kernel of
// the process (measured: a solve without the window went from 30.8 to 41 ms
// after the limit was raised to 75 MB).  With the B200 default set-aside
// (about 25 MB) the bench solve takes about 4 % less time.  Errors of these
// queries only turn the window off.
// After the solve the window's lines would stay persisting and crowd every
// later kernel (another solver's workspace included) out of the set-aside.
// This kernel reads each 128-byte line of the window once under a window with
// the normal hit property, which returns the lines to normal status.
__global__ void k_l2_release(const uint4* base, size_t n16) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i * 8 < n16; i += (size_t)gridDim.x * blockDim.x) {
    unsigned int a, b, c, d;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
                 : "l"(base + i * 8));
  }
}

static bool pcg_l2_window(const PcgParams& p, cudaLaunchAttribute& at) {
  if (p.l2 < 0) return false;
  int dev = 0, maxw = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const size_t vecb = (size_t)(static_cast<const char*>(p.p1) - static_cast<const char*>(p.p0));
  const size_t maxwin = (size_t)std::max(maxw, 0);
  void* base = p.p0;
  size_t bytes = 4 * vecb;  // p0, p1, z, Op
  if (bytes > maxwin) {
    base = p.z;
    bytes = 2 * vecb;  // z, Op
  }
  if (bytes == 0 || bytes > maxwin) return false;
  size_t cur = 0;  // the context's persisting set-aside, used as it is
  if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (cur == 0) return false;
  at.id = cudaLaunchAttributeAccessPolicyWindow;
  at.val.accessPolicyWindow.base_ptr = base;
  at.val.accessPolicyWindow.num_bytes = bytes;
  at.val.accessPolicyWindow.hitRatio = std::min(1.0f, (float)((double)cur / (double)bytes));
  at.val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  at.val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  return true;
}

template <typename RS, typename RH, typename A, int BY, int ECS, int ECH>
static int launch_pcg_t(PcgParams& p, cudaStream_t st) {
  int Lmax = 0, Ntmax = 0;
  for (int s = 0; s < p.nsys; ++s) {
    Lmax = std::max(Lmax, p.sys[s].L);
    Ntmax = std::max(Ntmax, p.sys[s].Nt);
    if (p.sys[s].L % BY) return QEDF_ERR_ARG;
  }
  int eng_threads = slice_threads(Lmax, BY, (ECS & EC_XS) != 0);
  eng_threads = std::max(eng_threads, slice_threads(Lmax, BY, false));
  if (eng_threads > MaxT<BY, ECS>::value) return QEDF_ERR_SIZE;
  const int threads = std::min(MaxT<BY, ECS>::value, std::max(128, eng_threads));
  size_t smem = slice_smem_bytes<RS, ECS>(Lmax, BY, 2);
  if (ECS & EC_STAGE) {
    p.stage_off = (int)align_up(smem, 128);
    smem = p.stage_off + pcg_stage_bytes<RS>(Lmax);
  }
  smem = std::max(smem, slice_smem_bytes<RH, ECH>(Lmax, BY, 2));
  // elementwise units: the r column, and in single precision the staging
  // area of the update pass
  smem = std::max(smem, ((sizeof(Cx<RS>) * (size_t)Ntmax * p.CH + 15) / 16 * 16) +
                            (sizeof(RS) == 4 ? PCG_EW_STAGES * 2 * 16 * (size_t)threads : 0));
  if (smem + sizeof(RhsState) > 227 * 1024) return QEDF_ERR_SIZE;
  auto kern = k_pcg<RS, RH, A, BY, ECS, ECH>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return QEDF_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
    return QEDF_ERR_SIZE;
  const int nblk = num_sms() * per_sm;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblk);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const bool window = pcg_l2_window(p, attr[1]);
  if (window) cfg.numAttrs = 2;
  if (cudaLaunchKernelEx(&cfg, kern, p) != cudaSuccess) return QEDF_ERR_CUDA;
  if (p.l2 >= 0) {
    // one launch whenever the option is on (an empty one without a window)
    cudaLaunchConfig_t rc = {};
    rc.gridDim = dim3(window ? num_sms() * 4 : 1);
    rc.blockDim = dim3(256);
    rc.stream = st;
    cudaLaunchAttribute ra[1];
    size_t n16 = 0;
    const uint4* base = nullptr;
    if (window) {
      ra[0] = attr[1];
      ra[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyNormal;
      ra[0].val.accessPolicyWindow.missProp = cudaAccessPropertyNormal;
      rc.attrs = ra;
      rc.numAttrs = 1;
      base = static_cast<const uint4*>(attr[1].val.accessPolicyWindow.base_ptr);
      n16 = attr[1].val.accessPolicyWindow.num_bytes / 16;
    }
    if (cudaLaunchKernelEx(&rc, k_l2_release, base, n16) != cudaSuccess) return QEDF_ERR_CUDA;
  }
  return QEDF_OK;
}

int launch_pcg_prep(const PcgParams& p, int zero_words, cudaStream_t st) {
  k_pcg_prep<<<1, 256, 0, st>>>(p, zero_words);
  return cudaGetLastError() == cudaSuccess ? QEDF_OK : QEDF_ERR_CUDA;
}

static bool fits(size_t engine_bytes) { return engine_bytes + sizeof(RhsState) <= 227 * 1024; }
// the staged engine: its tables plus two stages of three slices
template <typename RS, int ECS>
static bool fits_staged(int L, int BY) {
  return align_up(slice_smem_bytes<RS, ECS>(L, BY, 2), 128) + pcg_stage_bytes<RS>(L) + sizeof(RhsState) <=
         227 * 1024;
}

// Engines compiled for a fixed lattice side (with_fixed_l) when every system
// has that side; otherwise the run-time-L engine.
template <typename RS, typename RH, typename A, int BY, int ECS, int ECH>
static int launch_pcg_fl(PcgParams& p, cudaStream_t st) {
  bool same = true;
  for (int s = 1; s < p.nsys; ++s) same = same && p.sys[s].L == p.sys[0].L;
  if (!same) return launch_pcg_t<RS, RH, A, BY, ECS, ECH>(p, st);
  return with_fixed_l<BY>(p.sys[0].L, [&](auto lt) {
    constexpr int LT = decltype(lt)::value;
    return launch_pcg_t<RS, RH, A, BY, ECS | EC_L(LT), ECH | EC_L(LT)>(p, st);
  });
}

template <int BY>
static int launch_pcg_by(PcgParams& p, cudaStream_t st) {
  int Lmax = 0;
  for (int s = 0; s < p.nsys; ++s) Lmax = std::max(Lmax, p.sys[s].L);
  // the shuffle engine only pays when a row of tiles fills its warp segment
  bool pow2 = true;
  for (int s = 0; s < p.nsys; ++s) pow2 = pow2 && (((p.sys[s].L / 2) & (p.sys[s].L / 2 - 1)) == 0);
  const bool xs = p.xs && pow2 && xs_possible(Lmax) && slice_threads(Lmax, BY, true) <= MaxT<BY, EC_XS>::value;
  switch (p.mode) {
    case QEDF_PCG_PLAIN_F32:
      if (p.stage && fits_staged<float, 0>(Lmax, BY))
        return launch_pcg_fl<float, float, float, BY, EC_STAGE, EC_STAGE>(p, st);
      if (xs && fits(slice_smem_bytes<float, 0>(Lmax, BY, 2)))
        return launch_pcg_t<float, float, float, BY, EC_XS, EC_XS>(p, st);
      if (fits(slice_smem_bytes<float, 0>(Lmax, BY, 2)))
        return launch_pcg_fl<float, float, float, BY, 0, 0>(p, st);
      return launch_pcg_t<float, float, float, BY, EC_NOSTASH, EC_NOSTASH>(p, st);
    case QEDF_PCG_PLAIN_F64:
      if (fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<double, double, double, BY, EC_PHS, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, 0>(Lmax, BY, 2)))
        return launch_pcg_fl<double, double, double, BY, 0, 0>(p, st);
      return launch_pcg_t<double, double, double, BY, EC_NOSTASH, EC_NOSTASH>(p, st);
    case QEDF_PCG_MIXED:
      if (p.stage && fits_staged<float, 0>(Lmax, BY) && fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_STAGE, EC_PHS>(p, st);
      if (xs && fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_t<float, double, float, BY, EC_XS, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, 0, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, 0>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, 0, 0>(p, st);
      return launch_pcg_t<float, double, float, BY, 0, EC_NOSTASH>(p, st);
    case QEDF_PCG_MIXED_BF16:
      if (p.stage && fits_staged<float, 0>(Lmax, BY) && fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_STAGE | EC_BF16, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_BF16, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, 0>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_BF16, 0>(p, st);
      return launch_pcg_t<float, double, float, BY, EC_BF16, EC_NOSTASH>(p, st);
    case QEDF_PCG_MIXED_F16:
      if (p.stage && fits_staged<float, 0>(Lmax, BY) && fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_STAGE | EC_F16, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, EC_PHS>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_F16, EC_PHS>(p, st);
      if (fits(slice_smem_bytes<double, 0>(Lmax, BY, 2)))
        return launch_pcg_fl<float, double, float, BY, EC_F16, 0>(p, st);
      return launch_pcg_t<float, double, float, BY, EC_F16, EC_NOSTASH>(p, st);
  }
  return QEDF_ERR_ARG;
}

int launch_pcg(PcgParams& p, int by, cudaStream_t st) {
  if (by <= 0) {
    // the tile must divide every system's L; prefer the smallest that fits
    int Lmax = 0;
    for (int s = 0; s < p.nsys; ++s) Lmax = std::max(Lmax, p.sys[s].L);
    const int order[3] = {2, 4, 6};
    by = -1;
    for (int c : order) {
      bool ok = (Lmax / 2) * (Lmax / c) <= (c == 2 ? MaxThreads<2>::value : c == 4 ? MaxThreads<4>::value
                                                                                 : MaxThreads<6>::value);
      for (int s = 0; s < p.nsys; ++s) ok = ok && p.sys[s].L % c == 0;
      if (ok) {
        by = c;
        break;
      }
    }
    if (by < 0) return QEDF_ERR_SIZE;
  }
  switch (by) {
    case 2: return launch_pcg_by<2>(p, st);
    case 4: return launch_pcg_by<4>(p, st);
    case 6: return launch_pcg_by<6>(p, st);
  }
  return QEDF_ERR_ARG;
}

}  // namespace qedf

extern "C" int qedf_precon_tau_csr(int Ltau, int* row_ptr, int* col, double* val, int* nnz) {
  using namespace qedf;
  if (Ltau < PRE_MIN_LTAU || !row_ptr || !nnz) return QEDF_ERR_ARG;
  int k = 0;
  for (int t = 0; t < Ltau; ++t) {
    row_ptr[t] = k;
    // collect and sort the row by column
    int cols[32];
    double vals[32];
    int n = 0;
    pre_row(h_pre, Ltau, t, [&](int c, float v) {
      cols[n] = c;
      vals[n] = (double)v;
      ++n;
    });
    for (int i = 1; i < n; ++i)
      for (int j = i; j > 0 && cols[j - 1] > cols[j]; --j) {
        std::swap(cols[j - 1], cols[j]);
        std::swap(vals[j - 1], vals[j]);
      }
    for (int i = 0; i < n; ++i, ++k)
      if (col && val) {
        col[k] = cols[i];
        val[k] = vals[i];
      }
  }
  row_ptr[Ltau] = k;
  *nnz = k;
  return QEDF_OK;
}
