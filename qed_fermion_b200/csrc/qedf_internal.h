// Internal (C++) interface between the C-ABI layer and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/qedf.h"

namespace qedf {

enum { OP_M = 0, OP_MH = 1, OP_MHM = 2 };

struct OpArgs {
  const void* phi;  // angles [nphi][Nt][Vs][2]
  const void* x;    // input vectors [bs][Nt][Vs] complex
  void* z;          // output vectors
  int L, Nt, bs;
  int rhs_per_phi;  // consecutive vectors sharing one angle array
  int T;            // slab length (0 = auto)
  int xs;           // allow the warp-shuffle engine (single precision, L <= 64)
  double c1, ch, t1, th, Cb;
};

struct BvecArgs {
  const void* phi;  // one slice of angles [Vs][2]
  const void* v;    // [nvec][Vs] complex
  void* out;        // [nvec][6 or 1][Vs] complex
  int L, interm;
  double c1, ch, t1, th;
};

struct PreconArgs {
  const void* r;
  void* z;
  int L, Nt, bs, TC;
  const int* row_ptr;  // tau-space CSR of P_tau (device)
  const int* col;
  const double* val;
};

struct ForceArgs {
  const void* phi;
  const void* xi;
  void* F;
  int L, Nt, bs, rhs_per_phi, T;
  double c1, ch, t1, th;
};

struct BosonArgs {
  const void* x;  // angles [bs][Nt][Vs][2]
  void* F;        // force out (boson_force) or momenta in (boson_action)
  int L, Nt, bs, compact;
  double K, ctau, mass;
};

struct KickArgs {
  void* p;
  const void* F;
  void* x;
  const double* dt;    // [bs]
  const float* mask;   // [Nt] or null
  double kick_scale, drift_scale;
  int L, Nt, bs;
};

int num_sms();

// tile height (rows of the 2 x by site block per thread) for an L x L slice;
// requested = 0 picks automatically; -1 if no valid tile exists
int pick_by(int L, int requested, int real_bytes);
bool by_valid(int L, int by);

template <typename R, typename A>
int launch_operator(int op, OpArgs a, int by, cudaStream_t st);
template <typename R, typename A>
int launch_bvec(BvecArgs a, int nvec, cudaStream_t st);
template <typename R>
int launch_precon(const PreconArgs& a, cudaStream_t st);
template <typename R, typename A>
int launch_force(ForceArgs a, int by, cudaStream_t st);
template <typename A>
int launch_boson_force(const BosonArgs& a, cudaStream_t st);
template <typename A>
int launch_kick_drift(const KickArgs& a, cudaStream_t st);
template <typename A>
int launch_boson_action(const BosonArgs& a, double* out, cudaStream_t st);
template <typename R>
int launch_cdot(const R* u, const R* v, int64_t n, int rows, double* out, cudaStream_t st);

// ---- persistent PCG -------------------------------------------------------
constexpr int PCG_MAX_SYS = 32;
constexpr int PCG_MAX_RHS = 256;
constexpr int PCG_CHUNK = 16;  // sites per elementwise unit where 32 does not fit (a multiple of 2)

struct PcgSys {
  int L, Nt, nrhs, shared;
  int T, nslab;          // operator slabs per rhs
  int nchunk;            // site chunks per rhs (elementwise phases)
  int rhs0;              // first global rhs index
  int unitA0, unitE0;    // first operator / elementwise unit
  int64_t vec0;          // first complex element of the system in the packed vectors
  int64_t phi0;          // first real of the system in the packed angles
  int precon;
  int ptab0;             // first entry of the system's preconditioner band table
  int pmid_lo, pmid_hi;  // rows [lo, hi) of the preconditioner that are the bulk band
};

struct PcgParams {
  int nsys, nrhs, unitsA, unitsE, CH;
  PcgSys sys[PCG_MAX_SYS];
  int mode;  // QEDF_PCG_PLAIN_F32, QEDF_PCG_PLAIN_F64, QEDF_PCG_MIXED, QEDF_PCG_MIXED_BF16, QEDF_PCG_MIXED_F16
  int xs;    // allow the warp-shuffle engine for the single-precision iterations
  int stage; // 1: allow the staged operator engine (EC_STAGE) where its shared memory fits
  int stage_off;  // bytes: start of the operator passes' slice stages in dynamic shared memory
  int x_init;     // 1: x holds an initial guess on entry (the solve starts from b - A x)
  int l2;    // 0: L2 persisting window over the iteration vectors when they fit; -1: off
  int max_iter, ru_interval;
  double rtol, ru_delta;
  double c1, ch, t1, th, Cb;
  double pnorm;  // bound of the preconditioner's 2-norm: its largest absolute row sum (1 without)
  long long timeout_cycles;
  // data
  const void* phi;   // angles (float for F32/MIXED, double for F64)
  const void* b;     // rhs (sloppy type for plain, double for mixed)
  void* x;           // solution (same type as b)
  // workspace (sloppy precision vectors, each nvec_total complex)
  void* r;
  void* p0;
  void* p1;
  void* z;
  void* Op;
  void* xlo;         // mixed only
  double* acc;       // accumulators
  float* ptab;       // periodic 13-band tau tables of the preconditioner, per system
  unsigned int* bar; // [0] count, [1] generation, [2] error
  int* iters;
  double* relres;
  int* status;
  int64_t nvec_total;  // complex elements per vector buffer
  int ptab_len;        // floats of all preconditioner tables
  long long* prof;     // optional [8] cycle counters of block 0 (see k_pcg), or null
};

size_t pcg_workspace_bytes(const PcgParams& p, int sloppy_bytes);
size_t pcg_carve(PcgParams& p, int sloppy_bytes, void* workspace, size_t* zero_bytes);
// bytes of one real of the iteration vectors' storage for a QEDF_PCG_* mode
int pcg_storage_bytes(int mode);
int pcg_plan(PcgParams& p, const qedf_system* sys, int nsys, const qedf_pcg_opts* o);
int launch_pcg(PcgParams& p, int by, cudaStream_t st);
int launch_pcg_prep(const PcgParams& p, int zero_words, cudaStream_t st);
int pcg_solve_ws(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x, int* iters,
                 double* relres, int* status, void* workspace, int64_t ws_bytes, const qedf_pcg_opts* opts,
                 qedf_stream_t stream);

}  // namespace qedf
