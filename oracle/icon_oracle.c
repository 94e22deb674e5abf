/*
 * CPU oracle (test infrastructure, never shipped): the ICON triangle shallow-water model of
 * dmplex.jl in plain C with OpenMP over entities, for the timed CPU baseline and the long
 * published-figure tests. It restates the same kernels as oracle/icon_oracle.py (which cites
 * every reference line: ICONShallowWater.jl:149-218, TRiSKShallowWater.jl:298-312,
 * RungeKutta.jl:18-29) with the same summation and association order and -ffp-contract=off,
 * so the two agree bit for bit (tests/test_icon.py checks that). Tables as the Python oracle
 * holds them: 1-based Int64, (entity, k) row-major.
 */
#include "icon_oracle.h"

#include <stdlib.h>
#include <string.h>

static int g_icon_threads = 1;

void icon_oracle_set_threads(int threads) { g_icon_threads = threads < 1 ? 1 : threads; }
int icon_oracle_tables_size(void) { return (int)sizeof(icon_oracle_tables); }

#define T2(A, w, i, j) ((A)[(int64_t)(i) * (w) + (j)])

/* -sum_k divergence[i,k] F[cell_edges[i,k]] (continuity_kernel!) */
static void continuity(const icon_oracle_tables* t, const double* F, double* out) {
  const int threads = g_icon_threads;
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t i = 0; i < t->nc; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s = s + T2(t->divergence, 3, i, k) * F[T2(t->cell_edges, 3, i, k) - 1];
    out[i] = -s;
  }
}

/* scale (D_r - D_l) / d_e (edge_gradient_kernel!) */
static void gradient(const icon_oracle_tables* t, const double* D, double scale, double* out) {
  const int threads = g_icon_threads;
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t e = 0; e < t->ne; ++e)
    out[e] = scale * (D[T2(t->edge_cells, 2, e, 1) - 1] - D[T2(t->edge_cells, 2, e, 0) - 1]) * t->inverse_dual[e];
}

void icon_oracle_tendency(const icon_oracle_tables* t, const double* y, double* dy) {
  const int64_t ne = t->ne, nc = t->nc, nv = t->nv;
  const int vw = t->vw;
  const int threads = g_icon_threads;
  const double *u = y, *h = y + ne;
  double* v = malloc(sizeof(double) * ne);
  double* Ke = malloc(sizeof(double) * ne);
  double* F = malloc(sizeof(double) * ne);
  double* K = malloc(sizeof(double) * nc);
  double* zv = malloc(sizeof(double) * nv);
  /* edges: v by RBF, K_e, F */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t e = 0; e < ne; ++e) {
    double s = 0.0;
    for (int k = 0; k < 4; ++k) s = s + T2(t->rbf, 4, e, k) * u[T2(t->rbf_edges, 4, e, k) - 1];
    v[e] = s;
    Ke[e] = (u[e] * u[e] + s * s) / 2;
    F[e] = (T2(t->edge_height, 2, e, 0) * h[T2(t->edge_cells, 2, e, 0) - 1] +
            T2(t->edge_height, 2, e, 1) * h[T2(t->edge_cells, 2, e, 1) - 1]) * u[e];
  }
  /* cells: K by the bilinear weights; vertices: zeta */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t i = 0; i < nc; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s = s + T2(t->bilinear, 3, i, k) * Ke[T2(t->cell_edges, 3, i, k) - 1];
    K[i] = s;
  }
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t x = 0; x < nv; ++x) {
    double s = 0.0;
    for (int k = 0; k < vw; ++k) s = s + T2(t->curl, vw, x, k) * u[T2(t->vertex_edges, vw, x, k) - 1];
    zv[x] = s;
  }
  /* edges: the momentum tendency */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t l = T2(t->edge_cells, 2, e, 0) - 1, r = T2(t->edge_cells, 2, e, 1) - 1;
    const double zeta = (zv[T2(t->edge_vertices, 2, e, 0) - 1] + zv[T2(t->edge_vertices, 2, e, 1) - 1]) / 2;
    const double g0 = T2(t->gradient, 2, e, 0), g1 = T2(t->gradient, 2, e, 1);
    const double gradK = Ke[e] * (g0 - g1) + g1 * K[r] - g0 * K[l];
    dy[e] = (t->edge_coriolis[e] + zeta) * v[e] - gradK - t->gravity * (h[r] - h[l]) * t->inverse_dual[e];
  }
  continuity(t, F, dy + ne);
  if (t->divergence_damping) {
    double* D = malloc(sizeof(double) * nc);
    double* G = malloc(sizeof(double) * ne);
    continuity(t, u, D);
    gradient(t, D, 1.0, G);
    continuity(t, G, D);
    gradient(t, D, -1.0, G);
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
    for (int64_t e = 0; e < ne; ++e) dy[e] = dy[e] + t->divergence_damping[e] * G[e];
    free(D);
    free(G);
  }
  free(v);
  free(Ke);
  free(F);
  free(K);
  free(zv);
}

void icon_oracle_rk4_step(const icon_oracle_tables* t, double* y, double dt, int64_t nsteps) {
  const int64_t n = t->ne + t->nc;
  const int threads = g_icon_threads;
  const double half = dt / 2, sixth = dt / 6;
  double* k1 = malloc(sizeof(double) * n);
  double* k2 = malloc(sizeof(double) * n);
  double* k3 = malloc(sizeof(double) * n);
  double* k4 = malloc(sizeof(double) * n);
  double* st = malloc(sizeof(double) * n);
  for (int64_t s = 0; s < nsteps; ++s) {
    icon_oracle_tendency(t, y, k1);
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
    for (int64_t i = 0; i < n; ++i) st[i] = y[i] + half * k1[i];
    icon_oracle_tendency(t, st, k2);
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
    for (int64_t i = 0; i < n; ++i) st[i] = y[i] + half * k2[i];
    icon_oracle_tendency(t, st, k3);
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
    for (int64_t i = 0; i < n; ++i) st[i] = y[i] + dt * k3[i];
    icon_oracle_tendency(t, st, k4);
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
    for (int64_t i = 0; i < n; ++i) y[i] = y[i] + sixth * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]);
  }
  free(k1);
  free(k2);
  free(k3);
  free(k4);
  free(st);
}
