// Slice engine: applies the checkerboard bond factors of one imaginary-time
// slice to a vector held in registers by one thread block.
//
// Thread mapping.  The L x L slice is tiled by 2 x BY site blocks ("tiles");
// tile (bx, by) owns x in {2bx, 2bx+1} and y in [BY*by, BY*by + BY) and has
// the id by * nbx + bx (its thread index, except in the shuffle variant).
// Because x0 and y0 are even, every bond factor pairs sites either inside the
// tile ("local") or across its edge with the neighbouring tile ("cross"):
//
//   g1 (x-bond A -> A+x):  local in even rows, cross in odd rows
//   g3 (x-bond A-x -> A):  local in odd rows,  cross in even rows
//   g2 (y-bond A -> A+y):  local in column x0, cross at the ends of x0+1
//   g4 (y-bond A-y -> A):  local in column x0+1, cross at the ends of x0
//
// (A = sites with x = y mod 2, the ordering of the reference's
// initialize_geometry, hmc_sampler_batch.py:937-969).  A factor application
// exports the values that neighbours need into a shared-memory buffer,
// synchronises once, and updates every owned site from its old value and its
// partner's old value.  Two exchange buffers alternate, so one barrier per
// factor is enough.  The bond phases t_g e^{i phi} of a slice are computed
// once by the owner of the bond's origin site and kept in registers; the
// phases a thread needs from its left and upper neighbours go through shared
// memory once per slice.
//
// Shared-memory layout.  Every table is indexed [slot][tile id], so the lanes
// of a warp touch consecutive words (no bank conflicts apart from the wrap at
// the ends of a tile row), and a neighbour's value sits at the neighbour's id.
#pragma once

#include <type_traits>

#include "qedf_common.cuh"

namespace qedf {

enum FacMode { FAC_TILDE = 0, FAC_TRUE = 1, FAC_INV = 2 };

// Largest thread block each tile height is compiled for (it fixes the
// register budget: 65536 / MAXT registers per thread).
template <int BY>
struct MaxThreads {
  static constexpr int value = BY == 2 ? 576 : (BY == 4 ? 512 : 384);
};

// Engine configuration bits (template parameter EC of the kernels):
//   EC_PHS     phases of all bonds in shared memory (else own ones in registers)
//   EC_NOSTASH no shared-memory stash: the previous y block stays in registers
//              (used only where the shared memory of the default layout does
//              not fit)
//   EC_XS      exchanges of the x-bond factors by warp shuffles: a warp holds
//              whole rows of tiles (L/2 <= 32 tiles per row, padded to a power
//              of two), so only the y-bond factors need a block barrier
//   EC_STAGE   the vector slices an operator pass reads are staged whole in
//              shared memory by bulk copies one slice ahead (SliceStages), so
//              no thread waits on a global load in the slice loop
//   EC_BF16    (PCG, mixed mode) the search direction p and the preconditioned
//              residual z are stored as bf16 pairs; the arithmetic stays in
//              single precision
//   EC_F16     (PCG, mixed mode) p and z stored as fp16 pairs scaled by a power
//              of two per vector (st_scale); the arithmetic stays in single
//              precision
//   EC_L(l)    (bits 8 and up) the lattice side fixed at compile time, so the
//              engine's index arithmetic folds into constants; 0 = run-time L
enum { EC_PHS = 1, EC_NOSTASH = 2, EC_XS = 4, EC_STAGE = 8, EC_BF16 = 16, EC_F16 = 32 };
__host__ __device__ constexpr int EC_L(int l) { return l << 8; }
__host__ __device__ constexpr int ec_fixed_l(int ec) { return ec >> 8; }
// Lattice sides with engines compiled for their size: the benchmark
// configurations' lattices with 2 x 2 tiles (L = 24, 36, 48; measured 2 to 16 %
// faster per PCG iteration than the run-time-L engine; at L = 66 the 2 x 6 tile
// engine gained nothing).  Calls f(std::integral_constant<int, LT>) with the
// side when it is one of them, else with 0 (the run-time-L engine).
template <int BY, typename F>
inline int with_fixed_l(int L, F&& f) {
  if constexpr (BY == 2) {
    if (L == 48) return f(std::integral_constant<int, 48>{});
    if (L == 36) return f(std::integral_constant<int, 36>{});
    if (L == 24) return f(std::integral_constant<int, 24>{});
  }
  return f(std::integral_constant<int, 0>{});
}

// the lattice side of a kernel compiled for engine configuration EC
template <int EC>
__host__ __device__ __forceinline__ int lattice_l(int runtime_l) {
  return ec_fixed_l(EC) ? ec_fixed_l(EC) : runtime_l;
}

// Largest thread block of a kernel compiled for tile height BY and engine
// configuration EC (it fixes the register budget: 65536 / value per thread).
template <int BY, int EC>
struct MaxT {
  static constexpr int value = (EC & EC_XS) ? (BY == 2 ? 768 : (BY == 4 ? 512 : 384))
                                            : (BY == 2 ? 576 : (BY == 4 ? 512 : 384));
  static constexpr int min_blocks = 1;
};

// threads of one slice engine (a multiple of 32)
__host__ __device__ inline int slice_threads(int L, int BY, bool xs) {
  const int nbx = L / 2, nby = L / BY;
  if (!xs) return (nbx * nby + 31) / 32 * 32;
  int W = 1;
  while (W < nbx) W <<= 1;
  const int G = 32 / W;
  return (nby + G - 1) / G * 32;
}
__host__ __device__ inline bool xs_possible(int L) { return L / 2 <= 32; }

// Shared-memory size (bytes) of one slice engine with NT = L^2 / (2 BY) tiles:
//   nbuf exchange buffers of BY * NT complex (x-bond factors: a left and a
//        right slot per cross row; y-bond factors: a top and a bottom slot),
//   phase tables: PHS [4][BY][NT] (all bonds), else [BY + 2][NT] (the
//        x-bond phases of column x0+1 and the y-bond phases of the last row),
//   the thread-private stash of one vector block, [2 BY][NT] complex.
template <typename R, int EC = 0>
__host__ __device__ inline size_t slice_smem_bytes(int L, int BY, int nbuf) {
  const size_t NT = (size_t)(L / 2) * (L / BY);
  const size_t ph = (EC & EC_PHS) ? 4 * BY * NT : (BY + 2) * NT;
  return sizeof(Cx<R>) * (nbuf * BY * NT + ph + ((EC & EC_NOSTASH) ? 0 : 2 * BY * NT));
}

template <typename R, int BY, bool PHS = false, bool XS = false, int LT = 0>
struct Slice {
  static_assert(BY % 2 == 0, "BY must be even");
  int L, nbx, nby, NT, bx, by, x0, y0, bxl, bxr, byu, byd;
  int id, idl, idr, idu, idd;  // tile ids of this tile and of its four neighbours
  int lane_l, lane_r;          // XS: lanes holding the left / right neighbour tiles
  bool on;
  Cx<R>* xb[4];  // exchange buffers (BY * NT complex each)
  Cx<R>* ph;     // phase tables (see slice_smem_bytes)
  Cx<R>* stash;  // [2 BY][NT] each thread parks its own block of one vector here
  int cur;
  R c1, ch;      // cosh(dtau), cosh(dtau/2)
  Cx<R> tpx_[PHS ? 1 : BY][2], tpy_[PHS ? 1 : BY][2], tpl_[PHS ? 1 : BY], tpt_[2];

  // phase of the x-bond / y-bond starting at own site (x0+c, y0+r), of the
  // x-bond arriving from the left in row r, of the y-bond arriving from above
  // (PHS table slots: 0 x-bond c=0, 1 y-bond c=0, 2 x-bond c=1, 3 y-bond c=1)
  __device__ __forceinline__ Cx<R> TPX(int r, int c) const {
    return PHS ? ph[(size_t)(2 * c * BY + r) * NT + id] : tpx_[PHS ? 0 : r][c];
  }
  __device__ __forceinline__ Cx<R> TPY(int r, int c) const {
    return PHS ? ph[(size_t)((2 * c + 1) * BY + r) * NT + id] : tpy_[PHS ? 0 : r][c];
  }
  __device__ __forceinline__ Cx<R> TPL(int r) const {
    return PHS ? ph[(size_t)(2 * BY + r) * NT + idl] : tpl_[PHS ? 0 : r];
  }
  __device__ __forceinline__ Cx<R> TPT(int c) const {
    return PHS ? ph[(size_t)((2 * c + 1) * BY + BY - 1) * NT + idu] : tpt_[c];
  }
  // exchange slots of a buffer: x factors use slot r & ~1 (left column) and
  // (r & ~1) + 1 (right column) of cross row r; y factors slot 0 (top row)
  // and slot 1 (bottom row)
  __device__ __forceinline__ Cx<R>* slot(Cx<R>* buf, int s) const { return buf + (size_t)s * NT; }

  // smem must hold slice_smem_bytes<R, EC>(L, BY, nbuf) for the kernel's EC
  __device__ void init(int L_, unsigned char* smem, int nbuf, R c1_, R ch_, int tid) {
    L = LT ? LT : L_;
    nbx = L / 2;
    nby = L / BY;
    NT = nbx * nby;
    if (XS) {
      int W = 1;
      while (W < nbx) W <<= 1;
      const int lane = tid & 31, seg = lane / W;
      const int tbx = lane % W, tby = (tid >> 5) * (32 / W) + seg;
      on = tbx < nbx && tby < nby;
      bx = on ? tbx : 0;
      by = on ? tby : 0;
      lane_l = on ? seg * W + (tbx == 0 ? nbx - 1 : tbx - 1) : lane;
      lane_r = on ? seg * W + (tbx + 1 == nbx ? 0 : tbx + 1) : lane;
    } else {
      // a fixed L whose tiles fill whole warps is launched with one thread per
      // tile exactly, so every thread owns a tile
      constexpr bool ALL_ON = LT > 0 && ((LT / 2) * (LT / BY)) % 32 == 0;
      on = ALL_ON || tid < NT;
      bx = on ? tid % nbx : 0;
      by = on ? tid / nbx : 0;
      lane_l = lane_r = 0;
    }
    x0 = 2 * bx;
    y0 = BY * by;
    bxl = (bx + nbx - 1) % nbx;
    bxr = (bx + 1) % nbx;
    byu = (by + nby - 1) % nby;
    byd = (by + 1) % nby;
    id = by * nbx + bx;
    idl = by * nbx + bxl;
    idr = by * nbx + bxr;
    idu = byu * nbx + bx;
    idd = byd * nbx + bx;
    Cx<R>* base = reinterpret_cast<Cx<R>*>(smem);
    for (int i = 0; i < 4; ++i) xb[i] = base + (size_t)(i < nbuf ? i : 0) * BY * NT;
    ph = base + (size_t)nbuf * BY * NT;
    stash = ph + (size_t)(PHS ? 4 * BY : BY + 2) * NT;
    cur = 0;
    c1 = c1_;
    ch = ch_;
  }

  // ---- global memory ------------------------------------------------------
  // slice: complex vector of the slice (2*Vs reals)
  __device__ __forceinline__ void load(Cx<R> (&v)[BY][2], const R* slice) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) ld2(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1]);
  }
  __device__ __forceinline__ void load_coherent(Cx<R> (&v)[BY][2], const R* slice) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) ld2c(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1]);
  }
  __device__ __forceinline__ void store(R* slice, const Cx<R> (&v)[BY][2]) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) st2(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1]);
  }
  // the same through a storage type S (float, double or bf16 pairs; see ld2s)
  template <typename S>
  __device__ __forceinline__ void load_st(Cx<R> (&v)[BY][2], const S* slice) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) ld2s(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1]);
  }
  template <typename S>
  __device__ __forceinline__ void store_st(S* slice, const Cx<R> (&v)[BY][2]) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) st2s(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1]);
  }
  // scaled storage (fp16: stored value times sc; other types ignore the scale)
  template <typename S>
  __device__ __forceinline__ void load_st(Cx<R> (&v)[BY][2], const S* slice, R sc) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) ld2s(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1], sc);
  }
  template <typename S>
  __device__ __forceinline__ void store_st(S* slice, const Cx<R> (&v)[BY][2], R inv) const {
#pragma unroll
    for (int r = 0; r < BY; ++r) st2s(slice + 2 * ((y0 + r) * L + x0), v[r][0], v[r][1], inv);
  }

  // thread-private parking of one block (no synchronisation needed)
  __device__ __forceinline__ void park(const Cx<R> (&v)[BY][2]) const {
    if (!on) return;
#pragma unroll
    for (int r = 0; r < BY; ++r) {
      slot(stash, 2 * r)[id] = v[r][0];
      slot(stash, 2 * r + 1)[id] = v[r][1];
    }
  }
  __device__ __forceinline__ void unpark(Cx<R> (&v)[BY][2]) const {
    if (!on) return;
#pragma unroll
    for (int r = 0; r < BY; ++r) {
      v[r][0] = slot(stash, 2 * r)[id];
      v[r][1] = slot(stash, 2 * r + 1)[id];
    }
  }

  // ---- bond phases of one slice --------------------------------------------
  // ang: the slice's 2*Vs angles (A = float or double); t1 = tanh(dtau),
  // th = tanh(dtau/2).
  // angles of the owned sites of one slice (issued early to hide latency)
  template <typename A>
  __device__ __forceinline__ void load_angles(A (&a)[BY][4], const A* ang) const {
    if (!on) return;
#pragma unroll
    for (int r = 0; r < BY; ++r) ld4(ang + 2 * ((y0 + r) * L + x0), a[r]);
  }

  // register mode: own phases into registers, the neighbours' through the
  // tables; contains one __syncthreads()
  template <typename A>
  __device__ void phases_from(const A (&a)[BY][4], R t1, R th) {
    static_assert(!PHS, "phases_from is for the register-phase engine");
    Cx<R>* phx = ph;                    // [BY][NT] x-bond phase of column x0+1
    Cx<R>* phy = ph + (size_t)BY * NT;  // [2][NT]  y-bond phases of row y0+BY-1
    if (on) {
#pragma unroll
      for (int r = 0; r < BY; ++r) {
        // x-bond of (x0+c, y0+r) is in g1 when the site is an A site, else g3
        tpx_[PHS ? 0 : r][0] = tphase((R)a[r][0], (r & 1) == 0 ? t1 : th);
        tpy_[PHS ? 0 : r][0] = tphase((R)a[r][1], th);
        tpx_[PHS ? 0 : r][1] = tphase((R)a[r][2], (r & 1) == 1 ? t1 : th);
        tpy_[PHS ? 0 : r][1] = tphase((R)a[r][3], th);
      }
      if (!XS) {
#pragma unroll
        for (int r = 0; r < BY; ++r) phx[(size_t)r * NT + id] = tpx_[PHS ? 0 : r][1];
      }
      phy[id] = tpy_[PHS ? 0 : BY - 1][0];
      phy[NT + id] = tpy_[PHS ? 0 : BY - 1][1];
    }
    if (XS) {
#pragma unroll
      for (int r = 0; r < BY; ++r) tpl_[PHS ? 0 : r] = shfl_c(tpx_[PHS ? 0 : r][1], lane_l);
    }
    __syncthreads();
    if (on) {
      if (!XS) {
#pragma unroll
        for (int r = 0; r < BY; ++r) tpl_[PHS ? 0 : r] = phx[(size_t)r * NT + idl];
      }
      tpt_[0] = phy[idu];
      tpt_[1] = phy[NT + idu];
    }
  }

  // phases of one slice straight from the angles; contains one __syncthreads()
  template <typename A>
  __device__ void phases(const A* ang, R t1, R th) {
    if constexpr (PHS) {
      if (on) {
#pragma unroll
        for (int r = 0; r < BY; ++r) {
          A a[4];
          ld4(ang + 2 * ((y0 + r) * L + x0), a);
          // x-bond of (x0+c, y0+r) is in g1 when the site is an A site, else g3
          ph[(size_t)(0 * BY + r) * NT + id] = tphase((R)a[0], (r & 1) == 0 ? t1 : th);
          ph[(size_t)(1 * BY + r) * NT + id] = tphase((R)a[1], th);
          ph[(size_t)(2 * BY + r) * NT + id] = tphase((R)a[2], (r & 1) == 1 ? t1 : th);
          ph[(size_t)(3 * BY + r) * NT + id] = tphase((R)a[3], th);
        }
      }
      __syncthreads();
    } else {
      A a[BY][4];
      load_angles(a, ang);
      phases_from(a, t1, th);
    }
  }

  __device__ static __forceinline__ Cx<R> shfl_c(Cx<R> v, int src) {
    return mk<R>(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
  }

  // ---- one factor ----------------------------------------------------------
  // G: 0..3 for g1..g4.  MODE: FAC_TILDE applies (I + tK), FAC_TRUE
  // c(I + tK) = F_g, FAC_INV c(I - tK) = F_g^{-1} (c^2 - s^2 = 1).
  __device__ static __forceinline__ bool xcross(int G, int r) { return G == 0 ? (r & 1) : !(r & 1); }

  template <int MODE>
  __device__ __forceinline__ void pair_update(Cx<R>& vi, Cx<R>& vj, Cx<R> a, R c) const {
    const Cx<R> oi = vi, oj = vj;
    if (MODE == FAC_INV) a = cneg(a);
    vi = cfma(a, oj, oi);
    vj = cjfma(a, oi, oj);
    if (MODE != FAC_TILDE) {
      vi = c * vi;
      vj = c * vj;
    }
  }

  // BUF: exchange buffer 0 or 1 fixed at compile time, or -1 for the
  // alternating run-time choice
  template <int G, int MODE, int BUF = -1>
  __device__ __forceinline__ void factor(Cx<R> (&v)[BY][2]) {
    const R c = (G == 0) ? c1 : ch;
    Cx<R>* buf = BUF >= 0 ? xb[BUF] : (cur ? xb[1] : xb[0]);
    if (XS && (G == 0 || G == 2)) {
      // neighbours' old values by shuffle; every lane takes part
#pragma unroll
      for (int r = 0; r < BY; ++r) {
        if (!xcross(G, r)) {
          if (on) pair_update<MODE>(v[r][0], v[r][1], TPX(r, 0), c);
        } else {
          const Cx<R> right = shfl_c(v[r][0], lane_r);
          const Cx<R> left = shfl_c(v[r][1], lane_l);
          if (on) {
            Cx<R> ao = TPX(r, 1), al = TPL(r);
            if (MODE == FAC_INV) {
              ao = cneg(ao);
              al = cneg(al);
            }
            v[r][1] = cfma(ao, right, v[r][1]);
            v[r][0] = cjfma(al, left, v[r][0]);
            if (MODE != FAC_TILDE) {
              v[r][1] = c * v[r][1];
              v[r][0] = c * v[r][0];
            }
          }
        }
      }
      return;  // no shared-memory buffer used
    }
    if (G == 0 || G == 2) {
      if (on) {
#pragma unroll
        for (int r = 0; r < BY; ++r)
          if (xcross(G, r)) {
            slot(buf, r & ~1)[id] = v[r][0];
            slot(buf, (r & ~1) + 1)[id] = v[r][1];
          }
      }
      __syncthreads();
      if (on) {
#pragma unroll
        for (int r = 0; r < BY; ++r) {
          if (!xcross(G, r)) {
            pair_update<MODE>(v[r][0], v[r][1], TPX(r, 0), c);
          } else {
            const Cx<R> right = slot(buf, r & ~1)[idr];
            const Cx<R> left = slot(buf, (r & ~1) + 1)[idl];
            Cx<R> ao = TPX(r, 1), al = TPL(r);
            if (MODE == FAC_INV) {
              ao = cneg(ao);
              al = cneg(al);
            }
            v[r][1] = cfma(ao, right, v[r][1]);
            v[r][0] = cjfma(al, left, v[r][0]);
            if (MODE != FAC_TILDE) {
              v[r][1] = c * v[r][1];
              v[r][0] = c * v[r][0];
            }
          }
        }
      }
    } else {
      constexpr int CL = (G == 1) ? 0 : 1;  // column with only local pairs
      constexpr int CC = 1 - CL;            // column with cross pairs at its ends
      if (on) {
        slot(buf, 0)[id] = v[0][CC];
        slot(buf, 1)[id] = v[BY - 1][CC];
      }
      __syncthreads();
      if (on) {
#pragma unroll
        for (int r = 0; r < BY; r += 2) pair_update<MODE>(v[r][CL], v[r + 1][CL], TPY(r, CL), c);
#pragma unroll
        for (int r = 1; r + 1 < BY; r += 2) pair_update<MODE>(v[r][CC], v[r + 1][CC], TPY(r, CC), c);
        const Cx<R> below = slot(buf, 0)[idd];
        const Cx<R> above = slot(buf, 1)[idu];
        Cx<R> ab = TPY(BY - 1, CC), at = TPT(CC);
        if (MODE == FAC_INV) {
          ab = cneg(ab);
          at = cneg(at);
        }
        Cx<R> nb = cfma(ab, below, v[BY - 1][CC]);
        Cx<R> nt = cjfma(at, above, v[0][CC]);
        if (MODE != FAC_TILDE) {
          nb = c * nb;
          nt = c * nt;
        }
        v[BY - 1][CC] = nb;
        v[0][CC] = nt;
      }
    }
    if (BUF < 0) cur ^= 1;
  }

  // B = F4 F3 F2 F1 F2 F3 F4 without the scalar Cb (FAC_TILDE) or exact.
  // The seven factors use exchange buffers P, 1-P, ..., P; two applications in
  // a row must alternate P (or be separated by a barrier).
  template <int MODE, int P = 0>
  __device__ __forceinline__ void applyB(Cx<R> (&v)[BY][2]) {
    factor<3, MODE, P>(v);
    factor<2, MODE, 1 - P>(v);
    factor<1, MODE, P>(v);
    factor<0, MODE, 1 - P>(v);
    factor<1, MODE, P>(v);
    factor<2, MODE, 1 - P>(v);
    factor<3, MODE, P>(v);
  }
};

// y = a - s * b  (s real)
template <typename R, int BY>
__device__ __forceinline__ void axpy_blk(Cx<R> (&y)[BY][2], const Cx<R> (&a)[BY][2], R s,
                                         const Cx<R> (&b)[BY][2]) {
#pragma unroll
  for (int r = 0; r < BY; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      y[r][c].re = fma(-s, b[r][c].re, a[r][c].re);
      y[r][c].im = fma(-s, b[r][c].im, a[r][c].im);
    }
}

// sum of |a|^2 over a block, in double (0 when !on)
template <typename R, int BY>
__device__ __forceinline__ double sq_blk(const Cx<R> (&a)[BY][2], bool on) {
  R s = 0;
#pragma unroll
  for (int r = 0; r < BY; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c) s = fma(a[r][c].re, a[r][c].re, fma(a[r][c].im, a[r][c].im, s));
  return on ? (double)s : 0.0;
}

template <typename R, int BY>
__device__ __forceinline__ void copy_blk(Cx<R> (&y)[BY][2], const Cx<R> (&a)[BY][2]) {
#pragma unroll
  for (int r = 0; r < BY; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c) y[r][c] = a[r][c];
}

// sigma_t: +1 for t < Nt-1 and -1 for the antiperiodic wrap t = Nt-1
template <typename R>
__device__ __forceinline__ R sigma_of(int t, int Nt) { return t == Nt - 1 ? R(-1) : R(1); }

}  // namespace qedf
