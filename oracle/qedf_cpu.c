/* CPU restatement of the fermion path in C with OpenMP, for timing the CPU
 * baseline on all host cores.  Test infrastructure, like the numpy oracle in
 * qedf_oracle.py, which it restates function by function and against which
 * tests/test_cpu_port.py checks it; nothing in the library uses it.
 *
 *   geometry          initialize_geometry   (hmc_sampler_batch.py:937-969)
 *   factor / B        get_M_sparse factors  (:1508-1550, 1770-1866), B = F4 F3 F2 F1 F2 F3 F4
 *   qedf_cpu_mhm      M^dag M               (:1884-1905)
 *   qedf_cpu_precon   P_tau (x) I           (preconditioners_orig/precon_manual.py)
 *   qedf_cpu_pcg_iter one PCG iteration     (preconditioned_cg_fast_test :751-846)
 *   qedf_cpu_force    force from xi         (force_f_sparse :2230-2330)
 *
 * Layouts: angles [Nt][Vs][2] (x-bond, y-bond), complex vectors [Nt][Vs]
 * interleaved (re, im).  Slices are distributed over OpenMP threads.
 */
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

static const int B_SEQ[7] = {3, 2, 1, 0, 1, 2, 3};

/* bond groups g = 0..3 (g1..g4): i, j sites and angle index 2 i + comp, Vs/2 each */
typedef struct {
  int L;
  int* i[4];
  int* j[4];
  int* b[4];
} Geometry;

static Geometry g_geom = {0};

static const Geometry* geometry(int L) {
  if (g_geom.L == L) return &g_geom;
  for (int g = 0; g < 4; ++g) {
    free(g_geom.i[g]);
    free(g_geom.j[g]);
    free(g_geom.b[g]);
    g_geom.i[g] = malloc(sizeof(int) * L * L / 2);
    g_geom.j[g] = malloc(sizeof(int) * L * L / 2);
    g_geom.b[g] = malloc(sizeof(int) * L * L / 2);
  }
  int n = 0;
  for (int parity = 0; parity < 2; ++parity)
    for (int y = parity; y < L; y += 2)
      for (int x = parity; x < L; x += 2, ++n) {
        const int a = x + y * L;
        g_geom.i[0][n] = a;
        g_geom.j[0][n] = (x + 1) % L + y * L;
        g_geom.i[1][n] = a;
        g_geom.j[1][n] = x + ((y + 1) % L) * L;
        g_geom.i[2][n] = (x - 1 + L) % L + y * L;
        g_geom.j[2][n] = a;
        g_geom.i[3][n] = x + ((y - 1 + L) % L) * L;
        g_geom.j[3][n] = a;
      }
  for (int g = 0; g < 4; ++g)
    for (int k = 0; k < n; ++k) g_geom.b[g][k] = 2 * g_geom.i[g][k] + (g & 1);
  g_geom.L = L;
  return &g_geom;
}

static void coeffs(double dtau, double* c, double* s) {
  c[0] = cosh(dtau);
  s[0] = sinh(dtau);
  for (int g = 1; g < 4; ++g) {
    c[g] = cosh(dtau / 2);
    s[g] = sinh(dtau / 2);
  }
}

/* F_g w in place on one slice: w_i' = c w_i + s e^{i phi} w_j, w_j' = s e^{-i phi} w_i + c w_j */
static void factor(cplx* w, const double* ph, const Geometry* G, int g, double c, double s, int half) {
  for (int k = 0; k < half; ++k) {
    const int i = G->i[g][k], j = G->j[g][k];
    const cplx e = cexp(I * ph[G->b[g][k]]);
    const cplx wi = w[i], wj = w[j];
    w[i] = c * wi + s * e * wj;
    w[j] = s * conj(e) * wi + c * wj;
  }
}

static void apply_B(cplx* w, const double* ph, const Geometry* G, const double* c, const double* s, int half) {
  for (int k = 0; k < 7; ++k) factor(w, ph, G, B_SEQ[k], c[B_SEQ[k]], s[B_SEQ[k]], half);
}

static cplx* g_buf = NULL;
static size_t g_buf_n = 0;

static cplx* scratch(size_t n) {
  if (n > g_buf_n) {
    free(g_buf);
    g_buf = malloc(sizeof(cplx) * n);
    g_buf_n = n;
  }
  return g_buf;
}

int qedf_cpu_threads(void) { return omp_get_max_threads(); }

/* out = M^dag M x */
void qedf_cpu_mhm(const double* phi, const double* xr, double* outr, int L, int Nt, double dtau) {
  const Geometry* G = geometry(L);
  const int Vs = L * L, half = Vs / 2;
  double c[4], s[4];
  coeffs(dtau, c, s);
  const cplx* x = (const cplx*)xr;
  cplx* out = (cplx*)outr;
  cplx* W = scratch((size_t)2 * Nt * Vs);
  cplx* y = W + (size_t)Nt * Vs;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < Nt; ++t) {  /* W_t = B_t x_t */
    memcpy(W + (size_t)t * Vs, x + (size_t)t * Vs, sizeof(cplx) * Vs);
    apply_B(W + (size_t)t * Vs, phi + (size_t)t * 2 * Vs, G, c, s, half);
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < Nt; ++t) {  /* y = M x */
    const cplx* wp = W + (size_t)((t + Nt - 1) % Nt) * Vs;
    const double sg = t == 0 ? 1.0 : -1.0;
    for (int k = 0; k < Vs; ++k) y[(size_t)t * Vs + k] = x[(size_t)t * Vs + k] + sg * wp[k];
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < Nt; ++t) {  /* W_t = B_t y_{t+1} */
    memcpy(W + (size_t)t * Vs, y + (size_t)((t + 1) % Nt) * Vs, sizeof(cplx) * Vs);
    apply_B(W + (size_t)t * Vs, phi + (size_t)t * 2 * Vs, G, c, s, half);
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < Nt; ++t) {  /* out = M^dag y */
    const double sg = t == Nt - 1 ? 1.0 : -1.0;
    for (int k = 0; k < Vs; ++k) out[(size_t)t * Vs + k] = y[(size_t)t * Vs + k] + sg * W[(size_t)t * Vs + k];
  }
}

/* z = (P_tau (x) I) r, P_tau as CSR over tau */
void qedf_cpu_precon(const double* rr, double* zr, int Nt, int Vs, const int* row_ptr, const int* col,
                     const double* val) {
  const cplx* r = (const cplx*)rr;
  cplx* z = (cplx*)zr;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < Nt; ++t) {
    cplx* zt = z + (size_t)t * Vs;
    for (int k = 0; k < Vs; ++k) zt[k] = 0;
    for (int e = row_ptr[t]; e < row_ptr[t + 1]; ++e) {
      const cplx* rc = r + (size_t)col[e] * Vs;
      const double v = val[e];
      for (int k = 0; k < Vs; ++k) zt[k] += v * rc[k];
    }
  }
}

static double re_dot(const cplx* a, const cplx* b, size_t n) {
  double acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
  for (size_t k = 0; k < n; ++k) acc += creal(conj(a[k]) * b[k]);
  return acc;
}

/* One PCG iteration in place: Op = A p, alpha = rz / p^dag Op, x += alpha p,
 * r -= alpha Op, z = P r (or r), beta = rz_new / rz, p = z + beta p.
 * Returns rz_new; |r|^2 in *rr_out. */
double qedf_cpu_pcg_iter(const double* phi, double* xr, double* rr, double* pr, double* zr, double* opr, int L,
                         int Nt, double dtau, double rz, const int* row_ptr, const int* col, const double* val,
                         double* rr_out) {
  const int Vs = L * L;
  const size_t n = (size_t)Nt * Vs;
  cplx *x = (cplx*)xr, *r = (cplx*)rr, *p = (cplx*)pr, *z = (cplx*)zr, *Op = (cplx*)opr;
  qedf_cpu_mhm(phi, pr, opr, L, Nt, dtau);
  const double alpha = rz / re_dot(p, Op, n);
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n; ++k) {
    x[k] += alpha * p[k];
    r[k] -= alpha * Op[k];
  }
  if (row_ptr)
    qedf_cpu_precon(rr, zr, Nt, Vs, row_ptr, col, val);
  else
    memcpy(z, r, sizeof(cplx) * n);
  const double rz_new = re_dot(r, z, n);
  *rr_out = re_dot(r, r, n);
  const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
  return rz_new;
}

/* force F = -dS_f/dphi from xi (kernel layout [Nt][Vs][2]) */
void qedf_cpu_force(const double* phi, const double* xir, double* F, int L, int Nt, double dtau) {
  const Geometry* G = geometry(L);
  const int Vs = L * L, half = Vs / 2;
  double c[4], s[4];
  coeffs(dtau, c, s);
  const cplx* xi = (const cplx*)xir;
  /* occurrences of F_g in B: (left rows index, right partial product index) */
  static const int occ_n[4] = {1, 2, 2, 2};
  static const int occ[4][2][2] = {{{3, 3}, {0, 0}}, {{2, 4}, {4, 2}}, {{1, 5}, {5, 1}}, {{0, 6}, {6, 0}}};
#pragma omp parallel
  {
    cplx* R = malloc(sizeof(cplx) * 8 * Vs);   /* right partial products R_0..R_7 */
    cplx* ln = malloc(sizeof(cplx) * 7 * Vs);  /* left rows of xi_{t+1} */
    cplx* lb = malloc(sizeof(cplx) * 7 * Vs);  /* left rows of B xi_t */
#pragma omp for schedule(static)
    for (int t = 0; t < Nt; ++t) {
      const double* ph = phi + (size_t)t * 2 * Vs;
      memcpy(R, xi + (size_t)t * Vs, sizeof(cplx) * Vs);
      for (int k = 0; k < 7; ++k) {
        memcpy(R + (size_t)(k + 1) * Vs, R + (size_t)k * Vs, sizeof(cplx) * Vs);
        factor(R + (size_t)(k + 1) * Vs, ph, G, B_SEQ[k], c[B_SEQ[k]], s[B_SEQ[k]], half);
      }
      /* left rows: conj of u after 0..6 factors */
      for (int which = 0; which < 2; ++which) {
        cplx* rows = which ? lb : ln;
        const cplx* u = which ? R + (size_t)7 * Vs : xi + (size_t)((t + 1) % Nt) * Vs;
        memcpy(rows, u, sizeof(cplx) * Vs);
        for (int k = 0; k < 6; ++k) {
          memcpy(rows + (size_t)(k + 1) * Vs, rows + (size_t)k * Vs, sizeof(cplx) * Vs);
          factor(rows + (size_t)(k + 1) * Vs, ph, G, B_SEQ[k], c[B_SEQ[k]], s[B_SEQ[k]], half);
        }
        for (size_t k = 0; k < (size_t)7 * Vs; ++k) rows[k] = conj(rows[k]);
      }
      const double sign_B = t == Nt - 1 ? 1.0 : -1.0;
      double* Ft = F + (size_t)t * 2 * Vs;
      for (int g = 0; g < 4; ++g)
        for (int k = 0; k < half; ++k) {
          const int i = G->i[g][k], j = G->j[g][k], b = G->b[g][k];
          const cplx v = s[g] * cexp(I * (ph[b] + 0.5 * acos(-1.0)));  /* s e^{i (phi + pi/2)} */
          cplx acc = 0;
          for (int o = 0; o < occ_n[g]; ++o) {
            const cplx* Lr = ln + (size_t)occ[g][o][0] * Vs;
            const cplx* Lb = lb + (size_t)occ[g][o][0] * Vs;
            const cplx* Rr = R + (size_t)occ[g][o][1] * Vs;
            acc += sign_B * (Lr[i] * Rr[j] * v + Lr[j] * Rr[i] * conj(v));
            acc += Lb[i] * Rr[j] * v + Lb[j] * Rr[i] * conj(v);
          }
          Ft[b] = 2.0 * creal(acc);
        }
    }
    free(R);
    free(ln);
    free(lb);
  }
}
