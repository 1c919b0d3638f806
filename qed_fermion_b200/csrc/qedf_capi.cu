// extern "C" entry points declared in include/qedf.h: argument validation on
// the host, then the kernel launchers of qedf_ops.cu / qedf_pcg.cu.
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "qedf_common.cuh"
#include "qedf_internal.h"

using namespace qedf;

namespace {

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

inline int check_lattice(int Lx, int Ltau) {
  if (Lx < 2 || (Lx & 1) || Ltau < 2) return QEDF_ERR_ARG;
  if (pick_by(Lx, 0, 4) < 0) return QEDF_ERR_SIZE;
  return QEDF_OK;
}

template <typename R, typename A>
int op_entry(int op, const A* boson, const R* x, R* out, int bs, int Lx, int Ltau, double dtau,
             int rhs_per_boson, int by, int slab, qedf_stream_t stream) {
  if (!boson || !x || !out || bs < 1) return QEDF_ERR_ARG;
  if (int e = check_lattice(Lx, Ltau)) return e;
  if (rhs_per_boson < 1 || bs % rhs_per_boson) return QEDF_ERR_ARG;
  if (!aligned16(boson) || !aligned16(x) || !aligned16(out) || x == out) return QEDF_ERR_ARG;
  if (by != 0 && !by_valid(Lx, by)) return QEDF_ERR_ARG;
  if (slab < 0 || bs > 65535) return QEDF_ERR_ARG;
  const FactorCoeffs f = factor_coeffs(dtau);
  OpArgs a;
  a.phi = boson;
  a.x = x;
  a.z = out;
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  a.rhs_per_phi = rhs_per_boson;
  a.T = slab;
  a.xs = 1;
  a.c1 = f.c1;
  a.ch = f.ch;
  a.t1 = f.t1;
  a.th = f.th;
  a.Cb = f.Cb;
  return launch_operator<R, A>(op, a, by, reinterpret_cast<cudaStream_t>(stream));
}

template <typename R>
int bvec_entry(const R* boson_tau, const R* v, R* out, int nvec, int Lx, double dtau, int interm,
               qedf_stream_t stream) {
  if (!boson_tau || !v || !out || nvec < 1 || nvec > 65535) return QEDF_ERR_ARG;
  if (int e = check_lattice(Lx, 2)) return e;
  if (!aligned16(boson_tau) || !aligned16(v) || !aligned16(out) || v == out) return QEDF_ERR_ARG;
  const FactorCoeffs f = factor_coeffs(dtau);
  BvecArgs a;
  a.phi = boson_tau;
  a.v = v;
  a.out = out;
  a.L = Lx;
  a.interm = interm ? 1 : 0;
  a.c1 = f.c1;
  a.ch = f.ch;
  a.t1 = f.t1;
  a.th = f.th;
  return launch_bvec<R, R>(a, nvec, reinterpret_cast<cudaStream_t>(stream));
}

template <typename R>
int precon_entry(const R* r, R* out, int bs, int Lx, int Ltau, const int* row_ptr, const int* col,
                 const double* val, qedf_stream_t stream) {
  if (!r || !out || !row_ptr || !col || !val || bs < 1 || bs > 65535) return QEDF_ERR_ARG;
  if (Lx < 2 || (Lx & 1) || Ltau < 1) return QEDF_ERR_ARG;
  if (!aligned16(r) || !aligned16(out) || r == out) return QEDF_ERR_ARG;
  PreconArgs a;
  a.r = r;
  a.z = out;
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  a.TC = 16;
  a.row_ptr = row_ptr;
  a.col = col;
  a.val = val;
  return launch_precon<R>(a, reinterpret_cast<cudaStream_t>(stream));
}

template <typename R>
int force_entry(const R* boson, const R* xi, R* F, int bs, int Lx, int Ltau, double dtau, int rhs_per_boson,
                int by, int slab, qedf_stream_t stream) {
  if (!boson || !xi || !F || bs < 1 || bs > 65535) return QEDF_ERR_ARG;
  if (int e = check_lattice(Lx, Ltau)) return e;
  if (rhs_per_boson < 1 || bs % rhs_per_boson) return QEDF_ERR_ARG;
  if (!aligned16(boson) || !aligned16(xi) || !aligned16(F)) return QEDF_ERR_ARG;
  if (by != 0 && !by_valid(Lx, by)) return QEDF_ERR_ARG;
  if (slab < 0) return QEDF_ERR_ARG;
  const FactorCoeffs f = factor_coeffs(dtau);
  ForceArgs a;
  a.phi = boson;
  a.xi = xi;
  a.F = F;
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  a.rhs_per_phi = rhs_per_boson;
  a.T = slab;
  a.c1 = f.c1;
  a.ch = f.ch;
  a.t1 = f.t1;
  a.th = f.th;
  return launch_force<R, R>(a, by, reinterpret_cast<cudaStream_t>(stream));
}

template <typename A>
int boson_force_entry(const A* boson, A* F, int bs, int Lx, int Ltau, double K, double ctau, int compact,
                      qedf_stream_t stream) {
  if (!boson || !F || bs < 1 || Lx < 2 || Ltau < 2 || boson == F) return QEDF_ERR_ARG;
  BosonArgs a;
  a.x = boson;
  a.F = F;
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  a.compact = compact ? 1 : 0;
  a.K = K;
  a.ctau = ctau;
  a.mass = 1.0;
  return launch_boson_force<A>(a, reinterpret_cast<cudaStream_t>(stream));
}

template <typename A>
int boson_action_entry(const A* boson, const A* mom, double* out, int bs, int Lx, int Ltau, double K,
                       double ctau, int compact, double mass, qedf_stream_t stream) {
  if (!boson || !out || bs < 1 || bs > 65535 || Lx < 2 || Ltau < 2 || !(mass > 0)) return QEDF_ERR_ARG;
  BosonArgs a;
  a.x = boson;
  a.F = const_cast<A*>(mom);
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  a.compact = compact ? 1 : 0;
  a.K = K;
  a.ctau = ctau;
  a.mass = mass;
  return launch_boson_action<A>(a, out, reinterpret_cast<cudaStream_t>(stream));
}

template <typename A>
int kick_entry(A* p, const A* F, A* x, const double* dt, const float* mask, double kick, double drift, int bs,
               int Lx, int Ltau, qedf_stream_t stream) {
  if (!p || !dt || bs < 1 || Lx < 2 || Ltau < 1) return QEDF_ERR_ARG;
  if (drift != 0.0 && !x) return QEDF_ERR_ARG;
  KickArgs a;
  a.p = p;
  a.F = F;
  a.x = x;
  a.dt = dt;
  a.mask = mask;
  a.kick_scale = F ? kick : 0.0;
  a.drift_scale = drift;
  a.L = Lx;
  a.Nt = Ltau;
  a.bs = bs;
  return launch_kick_drift<A>(a, reinterpret_cast<cudaStream_t>(stream));
}

}  // namespace

namespace qedf {

// Solve with a caller-provided workspace (shared by qedf_pcg_solve and the
// static-scratch entry point).
int pcg_solve_ws(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x, int* iters,
                 double* relres, int* status, void* workspace, int64_t ws_bytes, const qedf_pcg_opts* opts,
                 qedf_stream_t stream) {
  PcgParams p;
  int e = pcg_plan(p, sys, nsys, opts);
  if (e) return e;
  if (!boson || !b || !x || !iters || !relres || !status || !workspace) return QEDF_ERR_ARG;
  if (!aligned16(boson) || !aligned16(b) || !aligned16(x) || !aligned16(workspace)) return QEDF_ERR_ARG;
  if (opts->max_iter < 0 || !(opts->rtol >= 0)) return QEDF_ERR_ARG;
  const int sb = pcg_storage_bytes(opts->mode);
  if (ws_bytes < (int64_t)pcg_workspace_bytes(p, sb)) return QEDF_ERR_ARG;
  size_t zero_bytes = 0;
  pcg_carve(p, sb, workspace, &zero_bytes);
  p.phi = boson;
  p.b = b;
  p.x = x;
  p.iters = iters;
  p.relres = relres;
  p.status = status;
  p.prof = opts->profile;
  const double tmo = opts->timeout_ms > 0 ? opts->timeout_ms : 2000.0;
  int dev = 0, clk_khz = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, dev);
  if (clk_khz <= 0) clk_khz = 2000000;
  p.timeout_cycles = (long long)(tmo * (double)clk_khz);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // accumulators and barrier state start at zero; preconditioner tables
  if (int e2 = launch_pcg_prep(p, (int)(zero_bytes / 4), st)) return e2;
  return launch_pcg(p, opts->by, st);
}

}  // namespace qedf

extern "C" {

const char* qedf_version(void) { return "qedf 0.1.0 (sm_100a)"; }

const char* qedf_status_string(int s) {
  switch (s) {
    case QEDF_OK: return "ok";
    case QEDF_ERR_ARG: return "invalid argument";
    case QEDF_ERR_CUDA: return "CUDA error";
    case QEDF_ERR_SIZE: return "problem exceeds a kernel limit";
    case QEDF_ERR_MAXITER: return "not converged within max_iter";
    case QEDF_ERR_TIMEOUT: return "device-side wait timed out";
    case QEDF_ERR_NAN: return "non-finite value in solver";
  }
  return "unknown status";
}

int qedf_mhm_vec_c64(const float* boson, const float* x, float* out, int bs, int Lx, int Ltau, double dtau,
                     int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<float, float>(OP_MHM, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_mhm_vec_c128(const double* boson, const double* x, double* out, int bs, int Lx, int Ltau, double dtau,
                      int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<double, double>(OP_MHM, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_mh_vec_c64(const float* boson, const float* x, float* out, int bs, int Lx, int Ltau, double dtau,
                    int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<float, float>(OP_MH, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_mh_vec_c128(const double* boson, const double* x, double* out, int bs, int Lx, int Ltau, double dtau,
                     int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<double, double>(OP_MH, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_m_vec_c64(const float* boson, const float* x, float* out, int bs, int Lx, int Ltau, double dtau,
                   int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<float, float>(OP_M, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_m_vec_c128(const double* boson, const double* x, double* out, int bs, int Lx, int Ltau, double dtau,
                    int rpb, int by, int slab, qedf_stream_t s) {
  return op_entry<double, double>(OP_M, boson, x, out, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}

int qedf_b_vec_per_tau_c64(const float* boson_tau, const float* v, float* out, int nvec, int Lx, double dtau,
                           int interm, qedf_stream_t s) {
  return bvec_entry<float>(boson_tau, v, out, nvec, Lx, dtau, interm, s);
}
int qedf_b_vec_per_tau_c128(const double* boson_tau, const double* v, double* out, int nvec, int Lx,
                            double dtau, int interm, qedf_stream_t s) {
  return bvec_entry<double>(boson_tau, v, out, nvec, Lx, dtau, interm, s);
}

int qedf_precon_vec_c64(const float* r, float* out, int bs, int Lx, int Ltau, const int* row_ptr,
                        const int* col, const double* val, qedf_stream_t s) {
  return precon_entry<float>(r, out, bs, Lx, Ltau, row_ptr, col, val, s);
}
int qedf_precon_vec_c128(const double* r, double* out, int bs, int Lx, int Ltau, const int* row_ptr,
                         const int* col, const double* val, qedf_stream_t s) {
  return precon_entry<double>(r, out, bs, Lx, Ltau, row_ptr, col, val, s);
}

int qedf_force_f_c64(const float* boson, const float* xi, float* F, int bs, int Lx, int Ltau, double dtau,
                     int rpb, int by, int slab, qedf_stream_t s) {
  return force_entry<float>(boson, xi, F, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}
int qedf_force_f_c128(const double* boson, const double* xi, double* F, int bs, int Lx, int Ltau, double dtau,
                      int rpb, int by, int slab, qedf_stream_t s) {
  return force_entry<double>(boson, xi, F, bs, Lx, Ltau, dtau, rpb, by, slab, s);
}

int qedf_boson_force_f32(const float* boson, float* F, int bs, int Lx, int Ltau, double K, double ctau,
                         int compact, qedf_stream_t s) {
  return boson_force_entry<float>(boson, F, bs, Lx, Ltau, K, ctau, compact, s);
}
int qedf_boson_force_f64(const double* boson, double* F, int bs, int Lx, int Ltau, double K, double ctau,
                         int compact, qedf_stream_t s) {
  return boson_force_entry<double>(boson, F, bs, Lx, Ltau, K, ctau, compact, s);
}
int qedf_boson_action_f32(const float* boson, const float* mom, double* out, int bs, int Lx, int Ltau, double K,
                          double ctau, int compact, double mass, qedf_stream_t s) {
  return boson_action_entry<float>(boson, mom, out, bs, Lx, Ltau, K, ctau, compact, mass, s);
}
int qedf_boson_action_f64(const double* boson, const double* mom, double* out, int bs, int Lx, int Ltau,
                          double K, double ctau, int compact, double mass, qedf_stream_t s) {
  return boson_action_entry<double>(boson, mom, out, bs, Lx, Ltau, K, ctau, compact, mass, s);
}
int qedf_kick_drift_f32(float* p, const float* F, float* x, const double* dt, const float* mask, double kick,
                        double drift, int bs, int Lx, int Ltau, qedf_stream_t s) {
  return kick_entry<float>(p, F, x, dt, mask, kick, drift, bs, Lx, Ltau, s);
}
int qedf_kick_drift_f64(double* p, const double* F, double* x, const double* dt, const float* mask, double kick,
                        double drift, int bs, int Lx, int Ltau, qedf_stream_t s) {
  return kick_entry<double>(p, F, x, dt, mask, kick, drift, bs, Lx, Ltau, s);
}

int qedf_cdot_c64(const float* u, const float* v, int64_t n, int rows, double* out, qedf_stream_t s) {
  if (!u || !v || !out || n < 1 || rows < 1 || rows > 65535) return QEDF_ERR_ARG;
  return launch_cdot<float>(u, v, n, rows, out, reinterpret_cast<cudaStream_t>(s));
}
int qedf_cdot_c128(const double* u, const double* v, int64_t n, int rows, double* out, qedf_stream_t s) {
  if (!u || !v || !out || n < 1 || rows < 1 || rows > 65535) return QEDF_ERR_ARG;
  return launch_cdot<double>(u, v, n, rows, out, reinterpret_cast<cudaStream_t>(s));
}

int64_t qedf_pcg_workspace_bytes(const qedf_system* sys, int nsys, const qedf_pcg_opts* opts) {
  PcgParams p;
  if (pcg_plan(p, sys, nsys, opts) != QEDF_OK) return -1;
  const int sb = pcg_storage_bytes(opts->mode);
  return (int64_t)pcg_workspace_bytes(p, sb);
}

int qedf_pcg_solve(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x, int* iters,
                   double* relres, int* status, void* workspace, int64_t ws_bytes, const qedf_pcg_opts* opts,
                   qedf_stream_t stream) {
  return qedf::pcg_solve_ws(sys, nsys, boson, b, x, iters, relres, status, workspace, ws_bytes, opts, stream);
}

}  // extern "C"
