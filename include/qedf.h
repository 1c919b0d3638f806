/*
 * qedf.h -- C ABI of the B200 (sm_100a) fermion hot path of qed_fermion.
 *
 * Every entry point takes device pointers, plain sizes and a CUDA stream
 * (passed as void*), launches on that stream, never synchronises the host and
 * never allocates device memory, so all of them can be captured in a CUDA
 * graph.  They return QEDF_OK or one of the status codes below; argument
 * errors are detected on the host before anything is launched.
 *
 * Data layouts are those of the reference's native extension qed_fermion._C
 * (hmc_sampler_batch.py:98-99, 772, 799, 838, 2174-2189, 2406):
 *   complex vectors  [bs][Ltau][Ly][Lx]      interleaved (re, im)
 *   angles ("boson") [bs][Ltau][Ly][Lx][2]   component 0 = x-bond, 1 = y-bond
 *                    (boson.permute([0, 4, 3, 2, 1]) of [bs, 2, Lx, Ly, Ltau])
 *   forces           same layout as the angles
 * with Ly == Lx (even), hopping t = 1.
 */
#ifndef QEDF_H
#define QEDF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QEDF_OK 0
#define QEDF_ERR_ARG 1      /* invalid argument (size, parity, alignment, null) */
#define QEDF_ERR_CUDA 2     /* a CUDA call failed */
#define QEDF_ERR_SIZE 3     /* the problem exceeds a kernel limit */
#define QEDF_ERR_MAXITER 4  /* solver stopped at max_iter without converging */
#define QEDF_ERR_TIMEOUT 5  /* a device-side wait ran out (grid barrier) */
#define QEDF_ERR_NAN 6      /* non-finite value in a solver reduction */

typedef void* qedf_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* Library version string and the text of a status code. */
const char* qedf_version(void);
const char* qedf_status_string(int status);

/* ---------------------------------------------------------------------------
 * Fermion operator M = I - sum_{t<Nt-1} E_{t+1,t} (x) B_t + E_{0,Nt-1} (x) B_{Nt-1},
 * B_t = F4 F3 F2 F1 F2 F3 F4 (checkerboard bond exponentials, get_M_sparse
 * hmc_sampler_batch.py:1741-1906).
 *
 * bs vectors are processed; vector k uses angle array k / rhs_per_boson
 * (rhs_per_boson = 1: one gauge field per vector, as _C.*; rhs_per_boson = bs:
 * one shared gauge field, the estimator's batched noise vectors).
 * by (2, 4 or 6, or 0 = automatic) is the number of rows of the 2 x by site
 * block each thread owns; slab (0 = automatic) the tau-slices per thread block.
 * ------------------------------------------------------------------------- */

/* out = M^dag M x.  Replaces _C.mhm_vec(boson, x, Lx, dtau, 4, 8)
 * (hmc_sampler_batch.py:772, 799). */
int qedf_mhm_vec_c64(const float* boson, const float* x, float* out, int bs, int Lx, int Ltau,
                     double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);
int qedf_mhm_vec_c128(const double* boson, const double* x, double* out, int bs, int Lx, int Ltau,
                      double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);

/* out = M^dag v.  Replaces _C.mh_vec(boson, v, Lx, dtau, 4, 8)
 * (hmc_sampler_batch.py:2406; stochastic_estimator.py:430). */
int qedf_mh_vec_c64(const float* boson, const float* v, float* out, int bs, int Lx, int Ltau,
                    double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);
int qedf_mh_vec_c128(const double* boson, const double* v, double* out, int bs, int Lx, int Ltau,
                     double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);

/* out = M v.  The reference has no _C entry for M alone; it is the sparse M
 * of get_M_sparse (hmc_sampler_batch.py:1884-1903) applied matrix-free. */
int qedf_m_vec_c64(const float* boson, const float* v, float* out, int bs, int Lx, int Ltau,
                   double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);
int qedf_m_vec_c128(const double* boson, const double* v, double* out, int bs, int Lx, int Ltau,
                    double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);

/* One slice: out = B_t v ([nvec][Vs]) or, with interm != 0, the six partial
 * products [nvec][6][Vs] = F4 v, F3F4 v, F2F3F4 v, F1F2F3F4 v, F2F1F2F3F4 v,
 * F3F2F1F2F3F4 v.  boson_tau is one slice of angles [Vs][2].  The raw values
 * of v are used.  Replaces _C.b_vec_per_tau(boson_tau, v, Lx, dtau, interm,
 * 4, 8) (hmc_sampler_batch.py:2174-2189). */
int qedf_b_vec_per_tau_c64(const float* boson_tau, const float* v, float* out, int nvec, int Lx,
                           double dtau, int interm, qedf_stream_t stream);
int qedf_b_vec_per_tau_c128(const double* boson_tau, const double* v, double* out, int nvec, int Lx,
                            double dtau, int interm, qedf_stream_t stream);

/* z = (P_tau (x) I_Vs) r for bs vectors; P_tau is an Ltau x Ltau matrix in
 * CSR form (device arrays row_ptr[Ltau+1], col[nnz], val[nnz]).  Replaces
 * _C.precon_vec(r, precon_csr, Lx) (hmc_sampler_batch.py:773, 838) once the
 * caller has reduced the N x N CSR to its tau part. */
int qedf_precon_vec_c64(const float* r, float* out, int bs, int Lx, int Ltau, const int* row_ptr,
                        const int* col, const double* val, qedf_stream_t stream);
int qedf_precon_vec_c128(const double* r, double* out, int bs, int Lx, int Ltau, const int* row_ptr,
                         const int* col, const double* val, qedf_stream_t stream);

/* Builtin preconditioner table: fills host arrays row_ptr[Ltau+1], col[*nnz],
 * val[*nnz] with the tau part of the hand-built banded preconditioner
 * (preconditioners_orig/precon_manual.py:15-186; values rounded to float as
 * the reference stores them).  Pass col = val = NULL to query *nnz.
 * Returns QEDF_ERR_ARG for Ltau < 26, where the table is undefined. */
int qedf_precon_tau_csr(int Ltau, int* row_ptr, int* col, double* val, int* nnz);

/* Fermion force F = -dS_f/dphi for S_f = psi^dag (M^dag M)^{-1} psi, given
 * xi = (M^dag M)^{-1} psi, in the angle layout.  Fused replacement of the
 * per-slice loop of force_f_fast (hmc_sampler_batch.py:2150-2227: four
 * _C.b_vec_per_tau calls and fourteen df_dot_bs1 per slice). */
int qedf_force_f_c64(const float* boson, const float* xi, float* F, int bs, int Lx, int Ltau,
                     double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);
int qedf_force_f_c128(const double* boson, const double* xi, double* F, int bs, int Lx, int Ltau,
                      double dtau, int rhs_per_boson, int by, int slab, qedf_stream_t stream);

/* ---------------------------------------------------------------------------
 * Boson part (angle layout).  K_int, J_int as HmcSampler scales them
 * (hmc_sampler_batch.py:166-175): ctau = 1 / (J_int dtau^2).
 * ------------------------------------------------------------------------- */

/* F = -d(S_plaq + S_tau)/dphi: force_b_plaq_matfree + force_b_tau_noncmp or
 * force_b_tau_cmp (hmc_sampler_batch.py:1338-1360, 1438-1459). */
int qedf_boson_force_f32(const float* boson, float* F, int bs, int Lx, int Ltau, double K_int,
                         double ctau, int compact, qedf_stream_t stream);
int qedf_boson_force_f64(const double* boson, double* F, int bs, int Lx, int Ltau, double K_int,
                         double ctau, int compact, qedf_stream_t stream);

/* out[b] += S_tau + S_plaq of chain b (+ sum p^2 / (2 mass) if momenta is not
 * NULL): action_boson_tau + action_boson_plaq_matfree
 * (hmc_sampler_batch.py:1363-1372, 1428-1436, 2417-2424).  Double accumulation. */
int qedf_boson_action_f32(const float* boson, const float* momenta, double* out, int bs, int Lx,
                          int Ltau, double K_int, double ctau, int compact, double mass,
                          qedf_stream_t stream);
int qedf_boson_action_f64(const double* boson, const double* momenta, double* out, int bs, int Lx,
                          int Ltau, double K_int, double ctau, int compact, double mass,
                          qedf_stream_t stream);

/* p += kick * dt[b] * F * mask[t]; then, if drift != 0, x += drift * dt[b] * p * mask[t]
 * (the updates of leapfrog_cmp / leapfrog_proposer5, hmc_sampler_batch.py:2332-2347,
 * 2505, 2530).  F may be NULL (no kick); mask may be NULL (all ones). */
int qedf_kick_drift_f32(float* p, const float* F, float* x, const double* dt, const float* mask,
                        double kick, double drift, int bs, int Lx, int Ltau, qedf_stream_t stream);
int qedf_kick_drift_f64(double* p, const double* F, double* x, const double* dt, const float* mask,
                        double kick, double drift, int bs, int Lx, int Ltau, qedf_stream_t stream);

/* out[k] += Re sum_i conj(u[k,i]) v[k,i] for rows k < rows of n complex
 * entries (double accumulation); e.g. S_f = Re psi^dag xi
 * (hmc_sampler_batch.py:2415-2418). */
int qedf_cdot_c64(const float* u, const float* v, int64_t n, int rows, double* out, qedf_stream_t stream);
int qedf_cdot_c128(const double* u, const double* v, int64_t n, int rows, double* out,
                   qedf_stream_t stream);

/* ---------------------------------------------------------------------------
 * Bond-bond correlators of the stochastic estimator (T1 :1393, T21 :1447,
 * T2 :1504, T4 :1561 of stochastic_estimator.py): the passes before and after
 * the 2-D FFTs of the pair sums.
 *
 * qedf_bb_pair_fields: for pairs p < npairs, (s, t) = (ps[p], pt[p]), writes
 * fa[p][tau][y][x] and fb[p][tau][y][x], the two fields whose transforms the
 * reference multiplies (kind 1: T1, 21: T21, 2: T2, 4: T4), from eta and G_eta
 * [Nrv][Ltau][Lx*Lx] (complex; conj(eta) is taken here) and ephase = e^{i phi_x}
 * [Ltau][Lx*Lx].  npairs <= 65535 per call.
 * qedf_bb_kspace_acc: S[k] += sum_i A[i][k] B[i][k] for rows i < rows of Vs
 * complex entries; S is complex128 [Vs], accumulated in double precision.
 * ------------------------------------------------------------------------- */
int qedf_bb_pair_fields_c64(int kind, const float* eta, const float* g_eta, const float* ephase, const int* ps,
                            const int* pt, int npairs, int Nrv, int Lx, int Ltau, float* fa, float* fb,
                            qedf_stream_t stream);
int qedf_bb_pair_fields_c128(int kind, const double* eta, const double* g_eta, const double* ephase,
                             const int* ps, const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* fa,
                             double* fb, qedf_stream_t stream);
int qedf_bb_kspace_acc_c64(const float* A, const float* B, int64_t rows, int Vs, double* S,
                           qedf_stream_t stream);
int qedf_bb_kspace_acc_c128(const double* A, const double* B, int64_t rows, int Vs, double* S,
                            qedf_stream_t stream);

/* The pair sum of correlator `kind` in one pass: S[k] += sum over the pairs
 * (ps[p], pt[p]) and all slices of A(k) B(k), A and B the unnormalised 2-D
 * transforms (e^{+2 pi i k.r / L} and e^{-2 pi i k.r / L}) of the pair's two
 * fields, which qedf_bb_pair_fields would write; the fields and transforms
 * stay in shared memory.  Lx must split as p q with q <= 8 and the shared
 * memory must fit (complex128 up to L = 48, complex64 up to L = 72), else
 * QEDF_ERR_SIZE: the caller then takes the two-pass path. */
int qedf_bb_corr_c64(int kind, const float* eta, const float* g_eta, const float* ephase, const int* ps,
                     const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* S, qedf_stream_t stream);
int qedf_bb_corr_c128(int kind, const double* eta, const double* g_eta, const double* ephase, const int* ps,
                      const int* pt, int npairs, int Nrv, int Lx, int Ltau, double* S, qedf_stream_t stream);

/* Tvv (stochastic_estimator.py:1612-1652): writes each noise vector's current
 * field v_s(r) = g_s(r+x) conj(eta_s(r)) e^{i phi_x} + g_s(r) conj(eta_s(r+x))
 * e^{-i phi_x} for all slices ([Nrv][Ltau][Lx*Lx] complex) and adds its sum
 * over vectors and slices to Tv[Lx*Lx] (complex128, double accumulation). */
int qedf_bb_vfield_c64(const float* eta, const float* g_eta, const float* ephase, int Nrv, int Lx, int Ltau,
                       float* v, double* Tv, qedf_stream_t stream);
int qedf_bb_vfield_c128(const double* eta, const double* g_eta, const double* ephase, int Nrv, int Lx, int Ltau,
                        double* v, double* Tv, qedf_stream_t stream);
/* The short-distance terms T1, T21/T2 and T4 add to their pair sums (T1 :1440,
 * T21 :1497, T4 :1605), summed over vectors, slices and sites into D[3]
 * (complex128, double accumulation): D[0] = sum g(r+x) conj(eta(r-x))
 * e^{i phi_x(r)} e^{i phi_x(r-x)}, D[1] = sum g(r) conj(eta(r)), D[2] = sum
 * g(r) conj(eta(r+2x)) e^{-i phi_x(r)} e^{-i phi_x(r+x)}. */
int qedf_bb_diag_c64(const float* eta, const float* g_eta, const float* ephase, int Nrv, int Lx, int Ltau,
                     double* D, qedf_stream_t stream);
int qedf_bb_diag_c128(const double* eta, const double* g_eta, const double* ephase, int Nrv, int Lx, int Ltau,
                      double* D, qedf_stream_t stream);

/* ---------------------------------------------------------------------------
 * Adaptive Fourier mass of the boson momenta (hmc_sampler_batch.py:1133-1277):
 * the arithmetic around the real FFTs over [Lx][Ly][Ltau] (the FFTs
 * themselves are the caller's).  Arrays are per (chain, direction) rows.
 *
 * qedf_fm_accumulate: mean = (cnt mean + x) / (cnt + 1), d = x - mean
 *   (update_sigma_hat_cpu :1202-1207, its running mean; n reals).
 * qedf_fm_spectrum: S = (cnt S + |X|^2) / (cnt + 1) for the orthonormal
 *   transform X of d (:1208-1210; n complex X, n real S).
 * qedf_fm_mass: per row of len values, sigma = the mass spectrum of S:
 *   clamp to [0, *clamp_hi], Box-Cox (exponent lambda), rescale into
 *   [smin, smax], shift the row mean to 1, shrink towards 1 by lmd, invert if
 *   invert != 0 (apply_sigma_hat_cpu :1133-1200; *clamp_hi is the mean over
 *   rows of the rows' 0.99 quantiles, a device scalar).  sigma may alias S.
 * qedf_fm_noise: z = (a + i b) / sqrt(sigma m_k), m_k = 1 for the first and
 *   last of the nk tau frequencies, else 2 (draw_momentum_fft :1254-1265).
 * qedf_fm_scale: P = P sigma, complex P times real sigma (apply_m_inv
 *   :1267-1277).
 * ------------------------------------------------------------------------- */
int qedf_fm_accumulate_f32(float* mean, const float* x, float* d, int64_t n, double cnt, qedf_stream_t stream);
int qedf_fm_accumulate_f64(double* mean, const double* x, double* d, int64_t n, double cnt, qedf_stream_t stream);
int qedf_fm_spectrum_f32(float* S, const float* X, int64_t n, double cnt, qedf_stream_t stream);
int qedf_fm_spectrum_f64(double* S, const double* X, int64_t n, double cnt, qedf_stream_t stream);
int qedf_fm_mass_f32(const float* S, float* sigma, int rows, int64_t len, const float* clamp_hi, double lambda,
                     double smin, double smax, double lmd, int invert, qedf_stream_t stream);
int qedf_fm_mass_f64(const double* S, double* sigma, int rows, int64_t len, const double* clamp_hi, double lambda,
                     double smin, double smax, double lmd, int invert, qedf_stream_t stream);
int qedf_fm_noise_f32(const float* a, const float* b, const float* sigma, float* z, int64_t n, int nk,
                      qedf_stream_t stream);
int qedf_fm_noise_f64(const double* a, const double* b, const double* sigma, double* z, int64_t n, int nk,
                      qedf_stream_t stream);
int qedf_fm_scale_f32(float* P, const float* sigma, int64_t n, qedf_stream_t stream);
int qedf_fm_scale_f64(double* P, const double* sigma, int64_t n, qedf_stream_t stream);

/* ---------------------------------------------------------------------------
 * Batched preconditioned CG on M^dag M x = b (persistent kernel).
 *
 * Replaces preconditioned_cg_fast_test (hmc_sampler_batch.py:751-846) and the
 * estimator solve of set_eta_G_eta_inner (stochastic_estimator.py:427-433).
 * Several systems (lattices of different L and Ltau) with several right-hand
 * sides each are solved in one launch; every right-hand side has its own
 * convergence mask, iteration count and status.  The whole iteration
 * (operator, preconditioner, axpys, double-precision dot products) runs in
 * one cooperative kernel whose grid barriers give up after timeout_ms and
 * report QEDF_ERR_TIMEOUT.
 *
 * Packing: system s owns nrhs_s consecutive vectors of Ltau_s * Lx_s^2 complex
 * entries in b and x, in system order; its angles are one array
 * (shared_boson = 1) or nrhs_s arrays, also in system order.
 * ------------------------------------------------------------------------- */
typedef struct {
  int Lx;           /* even, Ly = Lx */
  int Ltau;
  int nrhs;         /* right-hand sides of this system */
  int shared_boson; /* 1: one angle array for all its right-hand sides */
} qedf_system;

#define QEDF_PCG_PLAIN_F32 0 /* complex64 vectors, float angles, float arithmetic */
#define QEDF_PCG_PLAIN_F64 1 /* complex128 vectors, double angles, double arithmetic */
#define QEDF_PCG_MIXED 2     /* complex128 b/x, float angles; float iterations with
                                double reliable updates of x and the true residual */
#define QEDF_PCG_MIXED_BF16 3 /* as QEDF_PCG_MIXED, with the search direction p and the
                                 preconditioned residual z stored as bf16 pairs (4 bytes
                                 per complex number); r, M^dag M p and the float part of x
                                 stay float, as does the arithmetic */
#define QEDF_PCG_MIXED_F16 4  /* as QEDF_PCG_MIXED_BF16 with fp16 pairs, each vector scaled
                                 by a power of two taken from the residual's norm, so that
                                 its entries keep fp16's 11-bit significand */

typedef struct {
  int mode;           /* QEDF_PCG_* */
  int max_iter;
  double rtol;        /* stop when ||b - A x|| / ||b|| <= rtol */
  double dtau;
  int use_precon;     /* builtin tau-banded preconditioner (systems with Ltau >= 26) */
  int ru_interval;    /* mixed: reliable update at least every ru_interval iterations
                         (0 = 100) */
  double ru_delta;    /* mixed: and whenever the residual fell by this factor (0 = 0.01) */
  int by, slab, chunk;/* tile height (2, 4, 6), tau-slab length of the operator units, sites
                         per elementwise unit (16 or 32); 0 = automatic */
  double timeout_ms;  /* per grid-barrier wait, 0 = 2000 ms */
  long long* profile; /* optional device array of 8 counters (zeroed by the caller) that
                         accumulate SM clock cycles of block 0: 0 init, 1 operator phases,
                         2 waits after them, 3 elementwise phases, 4 waits after them,
                         5 reliable updates, 6 per-iteration bookkeeping, 7 whole solve */
  int l2_persist;     /* 0 (default): an L2 access-policy window over the iteration vectors
                         p, z and M^dag M p, fitted to the context's persisting set-aside as
                         it is (cudaLimitPersistingL2CacheSize is never changed), released
                         to normal status after the solve by one small kernel;
                         -1: no window and no extra kernel */
  int stage;          /* 1: the operator passes stage their input slices in shared memory by
                         bulk copies where the stages fit (single-precision iterations);
                         0 (default) or -1: the engine that loads them directly */
  int x_init;         /* 1: x holds an initial guess on entry; the solve starts from the
                         residual b - A x, computed in the high precision (double for
                         MIXED / MIXED_BF16 / MIXED_F16 / PLAIN_F64).  A right-hand side with b = 0
                         gets x = 0.  0 (default): x starts at 0, as in the reference */
} qedf_pcg_opts;

/* Bytes of device workspace qedf_pcg_solve needs for these systems. */
int64_t qedf_pcg_workspace_bytes(const qedf_system* sys, int nsys, const qedf_pcg_opts* opts);

/* Solve.  boson: packed angles (float for PLAIN_F32 / MIXED / MIXED_BF16 / MIXED_F16,
 * double for PLAIN_F64); b, x: packed vectors (complex64 for PLAIN_F32,
 * complex128 otherwise); iters, relres, status: device arrays with one entry per
 * right-hand side (total over systems).  relres is the last measured relative
 * residual (the recomputed true one in MIXED mode).  Returns QEDF_OK when the
 * kernel was launched; per-rhs outcomes are in status. */
int qedf_pcg_solve(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x,
                   int* iters, double* relres, int* status, void* workspace, int64_t workspace_bytes,
                   const qedf_pcg_opts* opts, qedf_stream_t stream);

/* ---------------------------------------------------------------------------
 * Allocation-free solve.  No counterpart in the reference: it exists for hosts
 * that cannot allocate device memory where they solve (a driver capturing a
 * CUDA graph, or running under an allocator or a fixed memory budget it does
 * not control).  Same inputs, outputs and status as qedf_pcg_solve, but the
 * workspace is a device array inside this library of
 * QEDF_PCG_STATIC_SCRATCH_BYTES bytes per GPU, held by every GPU that loads the
 * library until exit.  Problems whose qedf_pcg_workspace_bytes exceeds it get
 * QEDF_ERR_SIZE.  Calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller.  The first call on a device looks up the
 * array's device address (once per device, that device current); make it
 * before any stream capture begins.  That address is kept for the life of the
 * process: a process that resets the device (cudaDeviceReset) or otherwise
 * tears down its primary context must not call this entry point afterwards.
 * It calls no cudaMalloc or other allocator.
 * ------------------------------------------------------------------------- */
#define QEDF_PCG_STATIC_SCRATCH_BYTES (64ll << 20)

int qedf_pcg_solve_static(const qedf_system* sys, int nsys, const void* boson, const void* b, void* x,
                          int* iters, double* relres, int* status, const qedf_pcg_opts* opts,
                          qedf_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* QEDF_H */
