/*
 * vbd_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * FP64 CPU restatement of the Vertex Block Descent time step of the reference
 * solver (mmichelis/WarpVBD, src/vbd_solver.py, warp-lang 1.10.0).  It is the
 * checker for the CUDA solver in warpvbd_b200/ and the timed CPU baseline of
 * bench.py.  Only tests/, __graft_entry__.smoke() and bench.py may load it.
 *
 * The restatement is deliberately literal: it keeps the reference's matrix
 * formulation (dF/dx through the constant dDs/dx table and masks, traces of
 * matrix products, an explicit F^-1, a per-(vertex, tet) assemble followed by
 * a sum and a 3x3 Cholesky solve), so that the product's closed-form kernel is
 * checked against an independent formulation of the same mathematics.
 *
 * Reference functions restated (file:line in mmichelis/WarpVBD):
 *   inertial_gradient_hessian            src/vbd_solver.py:15-47
 *   elastic_gradient_hessian (SNH)       src/vbd_solver.py:50-124
 *   elastic_gradient_hessian (StVK)      src/vbd_solver.py:127-144 (commented
 *                                        out in the reference; restated as the
 *                                        alternative material)
 *   accumulate_grad_hess (+ damping)     src/vbd_solver.py:149-232
 *   solve_grad_hess                      src/vbd_solver.py:236-274
 *   position_initialization              src/vbd_solver.py:277-292
 *   compute_element_invDm_masses_volume  src/vbd_solver.py:295-343
 *   convert_youngs_poisson_to_lame       src/vbd_solver.py:345-362
 *   VBDSolver.__init__ tables            src/vbd_solver.py:449-498
 *   VBDSolver.reset / step               src/vbd_solver.py:501-612
 *   compute_adjacency_dict, graph_coloring  src/coloring.py:24-72
 *
 * Third-party arithmetic: warp-lang 1.10.0 (not vendored) supplies
 * wp.inverse, wp.determinant, wp.trace, mat33 products, tile_sum and
 * tile_cholesky / tile_cholesky_solve (MathDx).  They are restated here as
 * textbook 3x3 algebra (adjugate / determinant inverse, sequential row sum,
 * Cholesky-Banachiewicz).  The solve is parity-unpinned against Warp itself
 * (Warp cannot be imported where this was written); the mesher and colouring
 * are pinned bit-exact by tests/golden.
 *
 * Build: make -C oracle   (gcc -O2 -fopenmp -shared -fPIC)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 1e-12 /* vbd_solver.py:11 */
#define ORC_MAX_ELEMENTS_PER_VERTEX 32 /* vbd_solver.py:12 */

enum { ORC_SNH = 0, ORC_STVK = 1 };

/* ------------------------------------------------------------------------- */
/* 3x3 helpers, row-major m[r*3+c]                                            */
/* ------------------------------------------------------------------------- */
static void mm33(const double* a, const double* b, double* o) {
  double t[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      t[r * 3 + c] = a[r * 3 + 0] * b[0 * 3 + c] + a[r * 3 + 1] * b[1 * 3 + c] +
                     a[r * 3 + 2] * b[2 * 3 + c];
  memcpy(o, t, sizeof t);
}
static void tr33(const double* a, double* o) {
  double t[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) t[r * 3 + c] = a[c * 3 + r];
  memcpy(o, t, sizeof t);
}
static double trace33(const double* a) { return a[0] + a[4] + a[8]; }
static double det33(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}
/* adjugate / determinant; a singular matrix gives the zero matrix */
static void inv33(const double* m, double* o) {
  double d = det33(m);
  double t[9];
  if (d == 0.0) {
    memset(o, 0, 9 * sizeof(double));
    return;
  }
  double s = 1.0 / d;
  t[0] = (m[4] * m[8] - m[5] * m[7]) * s;
  t[1] = (m[2] * m[7] - m[1] * m[8]) * s;
  t[2] = (m[1] * m[5] - m[2] * m[4]) * s;
  t[3] = (m[5] * m[6] - m[3] * m[8]) * s;
  t[4] = (m[0] * m[8] - m[2] * m[6]) * s;
  t[5] = (m[2] * m[3] - m[0] * m[5]) * s;
  t[6] = (m[3] * m[7] - m[4] * m[6]) * s;
  t[7] = (m[1] * m[6] - m[0] * m[7]) * s;
  t[8] = (m[0] * m[4] - m[1] * m[3]) * s;
  memcpy(o, t, sizeof t);
}
/* trace(A^T B) = sum_ij A_ij B_ij */
static double ddot33(const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < 9; ++i) s += a[i] * b[i];
  return s;
}

/* dDs_dx table, vbd_solver.py:449-467: entry [a][k] is the derivative of
 * Ds = [x0-x3, x1-x3, x2-x3] with respect to component k of local vertex a:
 * e_k e_a^T for a < 3 and -e_k 1^T for a = 3. */
static void dds_dx(int a, int k, double* o) {
  memset(o, 0, 9 * sizeof(double));
  if (a < 3) {
    o[k * 3 + a] = 1.0;
  } else {
    o[k * 3 + 0] = -1.0;
    o[k * 3 + 1] = -1.0;
    o[k * 3 + 2] = -1.0;
  }
}

/* ------------------------------------------------------------------------- */
/* Per-(vertex, tet) elastic gradient / Hessian, vbd_solver.py:50-146         */
/* x: 4 vertex positions (12 doubles) in the tet's local order;               */
/* a: local index of the differentiated vertex (the mask loop :88-94 picks    */
/* exactly one).                                                              */
/* ------------------------------------------------------------------------- */
void orc_tet_grad_hess(int material, const double* x, const double* invD, double lame_mu,
                       double lame_lambda, double volume, int a, double* grad, double* hess) {
  double Ds[9], F[9], dF[3][9];
  for (int r = 0; r < 3; ++r) /* matrix_from_cols(x0-x3, x1-x3, x2-x3) :77-81 */
    for (int c = 0; c < 3; ++c) Ds[r * 3 + c] = x[c * 3 + r] - x[9 + r];
  mm33(Ds, invD, F); /* :82 */
  for (int k = 0; k < 3; ++k) { /* :86-94 */
    double D[9];
    dds_dx(a, k, D);
    mm33(D, invD, dF[k]);
  }
  double J = det33(F), Ft[9], FtF[9], Finv[9], FinvT[9];
  tr33(F, Ft);
  mm33(Ft, F, FtF);
  double Ic = trace33(FtF);
  inv33(F, Finv);
  tr33(Finv, FinvT);
  for (int i = 0; i < 3; ++i) grad[i] = 0.0;
  for (int i = 0; i < 9; ++i) hess[i] = 0.0;

  if (material == ORC_SNH) {
    /* Stable Neo-Hookean, :107-124 */
    double mu = 4.0 * lame_mu / 3.0;
    double lmbda = lame_lambda + 5.0 * lame_mu / 6.0;
    double alpha = 1.0 + 0.75 * mu / lmbda;
    double P[9];
    for (int q = 0; q < 9; ++q)
      P[q] = mu * F[q] * (1.0 - 1.0 / (Ic + 1.0)) + lmbda * (J - alpha) * J * FinvT[q];
    for (int i = 0; i < 3; ++i) {
      grad[i] = volume * ddot33(P, dF[i]); /* trace(P^T dF_i) */
      for (int j = 0; j < 3; ++j) {
        double t1[9], t2[9], t3[9], t4[9], t5[9];
        mm33(Ft, dF[i], t1);
        mm33(Ft, dF[j], t2);
        mm33(Finv, dF[i], t3);
        mm33(Finv, dF[j], t4);
        mm33(t4, t3, t5); /* Finv dF_j Finv dF_i */
        hess[i * 3 + j] =
            volume * (2.0 * mu / ((Ic + 1.0) * (Ic + 1.0)) * trace33(t1) * trace33(t2) +
                      mu * (1.0 - 1.0 / (Ic + 1.0)) * ddot33(dF[i], dF[j]) +
                      lmbda * J * (2.0 * J - alpha) * trace33(t3) * trace33(t4) -
                      lmbda * J * (J - alpha) * trace33(t5));
      }
    }
  } else {
    /* St. Venant-Kirchhoff, :127-144 (unadjusted Lame parameters) */
    double E[9];
    for (int q = 0; q < 9; ++q) E[q] = 0.5 * (FtF[q] - ((q % 4 == 0) ? 1.0 : 0.0));
    double dE[3][9];
    for (int i = 0; i < 3; ++i) {
      double t1[9], dFt[9], t2[9];
      mm33(Ft, dF[i], t1);
      tr33(dF[i], dFt);
      mm33(dFt, F, t2);
      for (int q = 0; q < 9; ++q) dE[i][q] = 0.5 * (t1[q] + t2[q]);
    }
    for (int i = 0; i < 3; ++i) {
      grad[i] = volume * (lame_lambda * trace33(E) * trace33(dE[i]) +
                          2.0 * lame_mu * ddot33(dE[i], E));
      for (int j = 0; j < 3; ++j) {
        double dFit[9], dFjt[9], t1[9], t2[9], d2E[9];
        tr33(dF[i], dFit);
        tr33(dF[j], dFjt);
        mm33(dFit, dF[j], t1);
        mm33(dFjt, dF[i], t2);
        for (int q = 0; q < 9; ++q) d2E[q] = 0.5 * (t1[q] + t2[q]);
        hess[i * 3 + j] +=
            volume * (lame_lambda * (trace33(dE[i]) * trace33(dE[j]) + trace33(E) * trace33(d2E)) +
                      2.0 * lame_mu * (ddot33(dE[i], dE[j]) + ddot33(d2E, E)));
      }
    }
  }
}

/* Strain energy of one tet (new: the reference never evaluates it).  Its
 * F-gradient is the P used above: SNH  Psi = mu'/2 (Ic-3) - mu'/2 ln(Ic+1)
 * + lambda'/2 (J-alpha)^2;  StVK  Psi = mu E:E + lambda/2 tr(E)^2. */
double orc_tet_energy(int material, const double* x, const double* invD, double lame_mu,
                      double lame_lambda, double volume) {
  double Ds[9], F[9], Ft[9], FtF[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) Ds[r * 3 + c] = x[c * 3 + r] - x[9 + r];
  mm33(Ds, invD, F);
  tr33(F, Ft);
  mm33(Ft, F, FtF);
  double Ic = trace33(FtF);
  if (material == ORC_SNH) {
    double mu = 4.0 * lame_mu / 3.0;
    double lmbda = lame_lambda + 5.0 * lame_mu / 6.0;
    double alpha = 1.0 + 0.75 * mu / lmbda;
    double J = det33(F);
    return volume * (0.5 * mu * (Ic - 3.0) - 0.5 * mu * log(Ic + 1.0) +
                     0.5 * lmbda * (J - alpha) * (J - alpha));
  }
  double E[9];
  for (int q = 0; q < 9; ++q) E[q] = 0.5 * (FtF[q] - ((q % 4 == 0) ? 1.0 : 0.0));
  double trE = trace33(E);
  return volume * (lame_mu * ddot33(E, E) + 0.5 * lame_lambda * trE * trE);
}

/* 3x3 Cholesky factor + solve of H x = b (tile_cholesky / tile_cholesky_solve,
 * vbd_solver.py:267-268).  Returns 0 when every pivot is positive and finite.
 * With a non-positive pivot the arithmetic still runs (sqrt of a negative
 * gives NaN) -- that is what the reference does. */
static int chol_solve3(const double* H, const double* b, double* out) {
  double L00 = sqrt(H[0]);
  double L10 = H[3] / L00, L20 = H[6] / L00;
  double d1 = H[4] - L10 * L10;
  double L11 = sqrt(d1);
  double L21 = (H[7] - L20 * L10) / L11;
  double d2 = H[8] - L20 * L20 - L21 * L21;
  double L22 = sqrt(d2);
  double y0 = b[0] / L00;
  double y1 = (b[1] - L10 * y0) / L11;
  double y2 = (b[2] - L20 * y0 - L21 * y1) / L22;
  out[2] = y2 / L22;
  out[1] = (y1 - L21 * out[2]) / L11;
  out[0] = (y0 - L10 * out[1] - L20 * out[2]) / L00;
  int ok = (H[0] > 0.0) && (d1 > 0.0) && (d2 > 0.0) && isfinite(L00) && isfinite(L11) &&
           isfinite(L22);
  return ok ? 0 : 1;
}

/* ------------------------------------------------------------------------- */
/* Setup kernels                                                              */
/* ------------------------------------------------------------------------- */
/* convert_youngs_poisson_to_lame, vbd_solver.py:345-362 */
void orc_lame(int T, const double* E, const double* nu, double* mu, double* lam) {
  for (int i = 0; i < T; ++i) {
    mu[i] = E[i] / (2.0 * (1.0 + nu[i]));
    lam[i] = (E[i] * nu[i]) / ((1.0 + nu[i]) * (1.0 - 2.0 * nu[i]));
  }
}

/* compute_element_invDm_masses_volume, vbd_solver.py:295-343.  Returns the
 * number of tets whose Dm * Dm^-1 misses the identity by more than EPS (the
 * debug-mode asserts at :336-343). */
int orc_invdm_mass_volume(const double* X, int T, const int32_t* tets, const double* rho,
                          double* invDm, double* mass, double* vol) {
  int bad = 0;
  for (int i = 0; i < T; ++i) {
    const int32_t* e = tets + 4 * i;
    double Dm[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) Dm[r * 3 + c] = X[3 * e[c] + r] - X[3 * e[3] + r];
    inv33(Dm, invDm + 9 * i);
    vol[i] = fabs(det33(Dm)) / 6.0;
    mass[i] = rho[i] * vol[i];
    double res[9];
    mm33(Dm, invDm + 9 * i, res);
    for (int q = 0; q < 9; ++q) {
      double want = (q % 4 == 0) ? 1.0 : 0.0;
      if (!(fabs(res[q] - want) < ORC_EPS)) {
        ++bad;
        break;
      }
    }
  }
  return bad;
}

/* compute_adjacency_dict + graph_coloring, coloring.py:24-72: greedy, vertex
 * index order, smallest colour not used by an already-coloured neighbour in
 * the tet 1-ring.  The vertex count is max(tets)+1 (coloring.py:28).
 * coloring_out must hold max(tets)+1 entries.  Returns the number of colours,
 * or -1 when a vertex would need more than 256 (coloring.py:50). */
int orc_graph_coloring(int T, const int32_t* tets, int32_t* coloring_out, int* n_vertices_out) {
  int nv = 0;
  for (int i = 0; i < 4 * T; ++i)
    if (tets[i] + 1 > nv) nv = tets[i] + 1;
  *n_vertices_out = nv;
  /* vertex -> incident tets (CSR), neighbours are read through the tets */
  int* cnt = calloc((size_t)nv + 1, sizeof(int));
  for (int i = 0; i < 4 * T; ++i) cnt[tets[i] + 1]++;
  for (int v = 0; v < nv; ++v) cnt[v + 1] += cnt[v];
  int* fill = malloc(sizeof(int) * (size_t)nv);
  int* inc = malloc(sizeof(int) * (size_t)4 * (size_t)(T > 0 ? T : 1));
  memcpy(fill, cnt, sizeof(int) * (size_t)nv);
  for (int t = 0; t < T; ++t)
    for (int q = 0; q < 4; ++q) inc[fill[tets[4 * t + q]]++] = t;
  int ncol = 0;
  for (int v = 0; v < nv; ++v) coloring_out[v] = -1;
  for (int v = 0; v < nv; ++v) {
    unsigned char used[257];
    memset(used, 0, sizeof used);
    for (int s = cnt[v]; s < cnt[v + 1]; ++s) {
      const int32_t* e = tets + 4 * inc[s];
      for (int q = 0; q < 4; ++q) {
        int n = e[q];
        if (n != v && coloring_out[n] != -1) used[coloring_out[n]] = 1;
      }
    }
    int c = 0;
    while (c < 256 && used[c]) ++c;
    if (c == 256) {
      ncol = -1;
      break;
    }
    coloring_out[v] = c;
    if (c + 1 > ncol) ncol = c + 1;
  }
  free(cnt);
  free(fill);
  free(inc);
  return ncol;
}

/* ------------------------------------------------------------------------- */
/* Solver                                                                     */
/* ------------------------------------------------------------------------- */
typedef struct {
  int V, T, K, n_colors, max_group, material, guarded;
  double kd, g[3];
  double *X0, *xprev, *vel, *xnew, *dxs;
  int32_t* tets;
  uint8_t* active;
  double *mu, *lam, *invDm, *mass, *vol;
  int32_t* colors; /* [n_colors * max_group], -1 padded (:477-483) */
  int32_t* adj;    /* [V * K], -1 padded, ascending tet id (:485-498) */
  int bad_dm;
  long long guard_hits;
} orc_solver;

void orc_destroy(orc_solver* s) {
  if (!s) return;
  free(s->X0); free(s->xprev); free(s->vel); free(s->xnew); free(s->dxs);
  free(s->tets); free(s->active); free(s->mu); free(s->lam); free(s->invDm);
  free(s->mass); free(s->vol); free(s->colors); free(s->adj);
  free(s);
}

/* VBDSolver.__init__, vbd_solver.py:367-498.  coloring may be NULL (then the
 * greedy colouring above is run) or an int32[max(tets)+1] colour per vertex. */
orc_solver* orc_create(int V, const double* X, int T, const int32_t* tets, const double* rho,
                       const double* E, const double* nu, const uint8_t* active, double kd,
                       const double* gravity, int material, int guarded,
                       const int32_t* coloring) {
  orc_solver* s = calloc(1, sizeof(orc_solver));
  s->V = V; s->T = T; s->material = material; s->guarded = guarded; s->kd = kd;
  for (int i = 0; i < 3; ++i) s->g[i] = gravity[i];
  size_t v3 = (size_t)V * 3;
  s->X0 = malloc(sizeof(double) * v3); memcpy(s->X0, X, sizeof(double) * v3);
  s->xprev = malloc(sizeof(double) * v3); memcpy(s->xprev, X, sizeof(double) * v3);
  s->vel = calloc(v3, sizeof(double));
  s->xnew = calloc(v3, sizeof(double));
  s->dxs = calloc(v3, sizeof(double));
  s->tets = malloc(sizeof(int32_t) * 4 * (size_t)T); memcpy(s->tets, tets, sizeof(int32_t) * 4 * (size_t)T);
  s->active = malloc((size_t)V);
  for (int i = 0; i < V; ++i) s->active[i] = active ? (active[i] != 0) : 1;
  s->mu = malloc(sizeof(double) * (size_t)T); s->lam = malloc(sizeof(double) * (size_t)T);
  orc_lame(T, E, nu, s->mu, s->lam);
  s->invDm = malloc(sizeof(double) * 9 * (size_t)T);
  s->mass = malloc(sizeof(double) * (size_t)T); s->vol = malloc(sizeof(double) * (size_t)T);
  s->bad_dm = orc_invdm_mass_volume(X, T, tets, rho, s->invDm, s->mass, s->vol);

  /* colouring -> padded group table, groups in ascending vertex order */
  int nv = 0;
  int32_t* col;
  for (int i = 0; i < 4 * T; ++i) if (tets[i] + 1 > nv) nv = tets[i] + 1;
  col = malloc(sizeof(int32_t) * (size_t)(nv > 0 ? nv : 1));
  if (coloring) memcpy(col, coloring, sizeof(int32_t) * (size_t)nv);
  else { int dummy; orc_graph_coloring(T, tets, col, &dummy); }
  int ncol = 0;
  for (int v = 0; v < nv; ++v) if (col[v] + 1 > ncol) ncol = col[v] + 1;
  int* gsz = calloc((size_t)ncol + 1, sizeof(int));
  for (int v = 0; v < nv; ++v) gsz[col[v]]++;
  int mg = 0;
  for (int c = 0; c < ncol; ++c) if (gsz[c] > mg) mg = gsz[c];
  s->n_colors = ncol; s->max_group = mg;
  s->colors = malloc(sizeof(int32_t) * (size_t)(ncol * mg > 0 ? ncol * mg : 1));
  for (int q = 0; q < ncol * mg; ++q) s->colors[q] = -1;
  memset(gsz, 0, sizeof(int) * (size_t)(ncol + 1));
  for (int v = 0; v < nv; ++v) { int c = col[v]; s->colors[c * mg + gsz[c]++] = v; }
  free(gsz); free(col);

  /* adj_v2e: vertex -> incident tets, ascending tet index, -1 padded */
  int* deg = calloc((size_t)V, sizeof(int));
  int K = 0;
  for (int t = 0; t < T; ++t)
    for (int q = 0; q < 4; ++q) { int v = tets[4 * t + q]; if (++deg[v] > K) K = deg[v]; }
  s->K = K;
  s->adj = malloc(sizeof(int32_t) * (size_t)V * (size_t)(K > 0 ? K : 1));
  for (size_t q = 0; q < (size_t)V * (size_t)K; ++q) s->adj[q] = -1;
  memset(deg, 0, sizeof(int) * (size_t)V);
  for (int t = 0; t < T; ++t)
    for (int q = 0; q < 4; ++q) { int v = tets[4 * t + q]; s->adj[(size_t)v * K + deg[v]++] = t; }
  free(deg);
  return s;
}

int orc_num_colors(const orc_solver* s) { return s->n_colors; }
int orc_max_group(const orc_solver* s) { return s->max_group; }
int orc_max_incident(const orc_solver* s) { return s->K; }
int orc_bad_dm(const orc_solver* s) { return s->bad_dm; }
long long orc_guard_hits(const orc_solver* s) { return s->guard_hits; }
void orc_color_table(const orc_solver* s, int32_t* out) {
  memcpy(out, s->colors, sizeof(int32_t) * (size_t)s->n_colors * (size_t)s->max_group);
}
void orc_adjacency(const orc_solver* s, int32_t* out) {
  memcpy(out, s->adj, sizeof(int32_t) * (size_t)s->V * (size_t)s->K);
}
void orc_element_data(const orc_solver* s, double* invDm, double* mass, double* vol, double* mu,
                      double* lam) {
  size_t T = (size_t)s->T;
  if (invDm) memcpy(invDm, s->invDm, sizeof(double) * 9 * T);
  if (mass) memcpy(mass, s->mass, sizeof(double) * T);
  if (vol) memcpy(vol, s->vol, sizeof(double) * T);
  if (mu) memcpy(mu, s->mu, sizeof(double) * T);
  if (lam) memcpy(lam, s->lam, sizeof(double) * T);
}

/* Sum over the vertex's incident tets of inertia + elastic + damping
 * gradient / Hessian (accumulate_grad_hess :149-232 followed by the row sum of
 * solve_grad_hess :260-264).  x: current iterate; xprev / vel: state at the
 * start of the step. */
static void vertex_grad_hess(const orc_solver* s, int v, const double* x, const double* xprev,
                             const double* vel, double dt, double* G, double* H) {
  for (int q = 0; q < 3; ++q) G[q] = 0.0;
  for (int q = 0; q < 9; ++q) H[q] = 0.0;
  for (int j = 0; j < s->K; ++j) {
    int e = s->adj[(size_t)v * s->K + j];
    if (e == -1) continue; /* :214-216 */
    /* inertial_gradient_hessian :29-47 */
    double m = s->mass[e] / 4.0, gi[3], hi[9] = {0};
    for (int q = 0; q < 3; ++q) {
      double y = xprev[3 * v + q] + dt * vel[3 * v + q];
      gi[q] = m / (dt * dt) * (x[3 * v + q] - y);
      gi[q] += -m * s->g[q];
    }
    hi[0] = hi[4] = hi[8] = m / (dt * dt);
    /* elastic_gradient_hessian */
    const int32_t* el = s->tets + 4 * e;
    double xl[12];
    int a = 0;
    for (int q = 0; q < 4; ++q) {
      for (int c = 0; c < 3; ++c) xl[3 * q + c] = x[3 * el[q] + c];
      if (el[q] == v) a = q;
    }
    double ge[3], he[9];
    orc_tet_grad_hess(s->material, xl, s->invDm + 9 * e, s->mu[e], s->lam[e], s->vol[e], a, ge, he);
    /* damping :222-223 */
    double gd[3], hd[9];
    for (int r = 0; r < 3; ++r) {
      gd[r] = 0.0;
      for (int c = 0; c < 3; ++c)
        gd[r] += s->kd * he[r * 3 + c] * (x[3 * v + c] - xprev[3 * v + c]);
      gd[r] /= dt;
    }
    for (int q = 0; q < 9; ++q) hd[q] = s->kd * he[q] / dt;
    for (int q = 0; q < 3; ++q) G[q] += gi[q] + ge[q] + gd[q];
    for (int q = 0; q < 9; ++q) H[q] += hi[q] + he[q] + hd[q];
  }
}

void orc_vertex_grad_hess(const orc_solver* s, int v, const double* x, double dt, double* G,
                          double* H) {
  vertex_grad_hess(s, v, x, s->xprev, s->vel, dt, G, H);
}

/* Lumped vertex mass sum_e m_e / 4 over the incident tets. */
static double vertex_mass(const orc_solver* s, int v) {
  double m = 0.0;
  for (int j = 0; j < s->K; ++j) {
    int e = s->adj[(size_t)v * s->K + j];
    if (e != -1) m += s->mass[e] / 4.0;
  }
  return m;
}

/* Newton step of one vertex; returns 1 when the guard fired. */
static int vertex_update(orc_solver* s, int v, double dt) {
  double G[3], H[9], nb[3], out[3];
  vertex_grad_hess(s, v, s->xnew, s->xprev, s->vel, dt, G, H);
  for (int q = 0; q < 3; ++q) nb[q] = -G[q];
  int bad = chol_solve3(H, nb, out);
  if (bad && s->guarded) {
    /* Guarded step (product behaviour, not in the reference): fall back to
     * the inertia-only Hessian (m_v/dt^2) I; a vertex without mass stays. */
    double m = vertex_mass(s, v);
    for (int q = 0; q < 3; ++q) out[q] = (m > 0.0) ? nb[q] * dt * dt / m : 0.0;
  }
  for (int q = 0; q < 3; ++q) {
    s->dxs[3 * v + q] = out[q];          /* :271 */
    s->xnew[3 * v + q] += out[q];        /* :274 */
  }
  return bad;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* VBDSolver.step, vbd_solver.py:509-612.  positions: the caller's "positions"
 * argument (NULL means the solver's own old_positions, which is what every
 * caller in the reference passes).  Writes the new positions to out (may be
 * NULL) and the number of sweeps run to *iters.  Returns 1 when the loop index
 * reached max_iter-1 (the reference's warning condition :581), else 0. */
int orc_step(orc_solver* s, const double* positions, double dt, double tol, int max_iter,
             double* out, int* iters) {
  size_t v3 = (size_t)s->V * 3;
  if (positions) memcpy(s->xprev, positions, sizeof(double) * v3); /* :535 */
  memcpy(s->xnew, s->xprev, sizeof(double) * v3);                  /* :536 */
  for (int v = 0; v < s->V; ++v) {                                 /* :277-292 */
    if (!s->active[v]) continue;
    for (int q = 0; q < 3; ++q)
      s->xnew[3 * v + q] = s->xprev[3 * v + q] + s->vel[3 * v + q] * dt + s->g[q] * dt * dt;
  }
  memset(s->dxs, 0, sizeof(double) * v3); /* :545 */
  int i = 0;
  long long guards = 0;
  for (i = 0; i < max_iter; ++i) {
    for (int c = 0; c < s->n_colors; ++c) {
      const int32_t* grp = s->colors + (size_t)c * s->max_group;
      long long gh = 0;
#pragma omp parallel for schedule(static) reduction(+ : gh)
      for (int k = 0; k < s->max_group; ++k) {
        int v = grp[k];
        if (v == -1 || !s->active[v]) continue; /* :206-212, :252-258 */
        gh += vertex_update(s, v, dt);
      }
      guards += gh;
    }
    double mx = 0.0; /* abs(dxs.sum(1)).max() :578 (NaN propagates) */
    int nan = 0;
    for (int v = 0; v < s->V; ++v) {
      double d = fabs(s->dxs[3 * v] + s->dxs[3 * v + 1] + s->dxs[3 * v + 2]);
      if (d != d) nan = 1;
      if (d > mx) mx = d;
    }
    if (!nan && mx < tol) break;
  }
  if (i == max_iter) i = max_iter - 1; /* Python's loop variable stops at max_iter-1 */
  s->guard_hits += guards;
  int warn = (i == max_iter - 1);
  if (iters) *iters = i + 1;
  for (size_t q = 0; q < v3; ++q) {       /* :609-610 */
    s->vel[q] = (s->xnew[q] - s->xprev[q]) / dt;
    s->xprev[q] = s->xnew[q];
  }
  if (out) memcpy(out, s->xnew, sizeof(double) * v3);
  return warn;
}

/* VBDSolver.reset, vbd_solver.py:501-506 */
void orc_reset(orc_solver* s) {
  memcpy(s->xprev, s->X0, sizeof(double) * (size_t)s->V * 3);
  memset(s->vel, 0, sizeof(double) * (size_t)s->V * 3);
}

void orc_get_state(const orc_solver* s, double* x, double* v) {
  if (x) memcpy(x, s->xprev, sizeof(double) * (size_t)s->V * 3);
  if (v) memcpy(v, s->vel, sizeof(double) * (size_t)s->V * 3);
}
void orc_set_state(orc_solver* s, const double* x, const double* v) {
  if (x) memcpy(s->xprev, x, sizeof(double) * (size_t)s->V * 3);
  if (v) memcpy(s->vel, v, sizeof(double) * (size_t)s->V * 3);
}

/* Incremental potential of a candidate iterate x for the step that starts
 * from the solver's current (xprev, vel):
 *   G(x) = sum_active m_v/(2 dt^2) |x_v - xprev_v - dt vel_v|^2 - m_v g.x_v
 *          + sum_e V_e Psi(F_e)
 * whose gradient in x_v is the accumulated gradient above (with kd = 0). */
double orc_incremental_potential(const orc_solver* s, const double* x, double dt) {
  double acc = 0.0;
  for (int v = 0; v < s->V; ++v) {
    if (!s->active[v]) continue;
    double m = vertex_mass(s, v), q2 = 0.0, gx = 0.0;
    for (int q = 0; q < 3; ++q) {
      double d = x[3 * v + q] - s->xprev[3 * v + q] - dt * s->vel[3 * v + q];
      q2 += d * d;
      gx += s->g[q] * x[3 * v + q];
    }
    acc += m / (2.0 * dt * dt) * q2 - m * gx;
  }
  for (int e = 0; e < s->T; ++e) {
    const int32_t* el = s->tets + 4 * e;
    double xl[12];
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < 3; ++c) xl[3 * q + c] = x[3 * el[q] + c];
    acc += orc_tet_energy(s->material, xl, s->invDm + 9 * e, s->mu[e], s->lam[e], s->vol[e]);
  }
  return acc;
}
