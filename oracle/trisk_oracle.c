/*
 * CPU oracle (test infrastructure, never shipped): restatement of the TRiSK shallow-water
 * kernels of dmplex.jl in plain C. Each function cites the reference lines it follows;
 * loop order, summation order and operator association are the reference's, and
 * -ffp-contract=off keeps every multiply and add separately rounded as Julia does.
 * See trisk_oracle.h for the layout and for how parity is pinned.
 */
#include "trisk_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

void oracle_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }
int oracle_threads(void) { return g_threads; }
int oracle_model_size(void) { return (int)sizeof(oracle_model); }

/* column-major [k, j] with 1-based Julia index contents */
#define AT(A, w, k, j) ((A)[(int64_t)(k) + (int64_t)(w) * (int64_t)(j)])
#define IX(A, w, k, j) (AT(A, w, k, j) - 1)

oracle_work* oracle_work_create(const oracle_model* m) {
  oracle_work* w = (oracle_work*)calloc(1, sizeof(oracle_work));
  w->K = (double*)calloc((size_t)m->nc, sizeof(double));
  w->B = (double*)calloc((size_t)m->nc, sizeof(double));
  w->F = (double*)calloc((size_t)m->ne, sizeof(double));
  w->zv = (double*)calloc((size_t)m->nv, sizeof(double));
  w->hv = (double*)calloc((size_t)m->nv, sizeof(double));
  w->qv = (double*)calloc((size_t)m->nv, sizeof(double));
  w->qe = (double*)calloc((size_t)m->ne, sizeof(double));
  w->Kv = (double*)calloc((size_t)(m->alpha != 1.0 ? m->nv : 1), sizeof(double));
  return w;
}

void oracle_work_destroy(oracle_work* w) {
  if (!w) return;
  free(w->K);
  free(w->B);
  free(w->F);
  free(w->zv);
  free(w->hv);
  free(w->qv);
  free(w->qe);
  free(w->Kv);
  free(w);
}

/* kinetic_energy_kernel!, TRiSKShallowWater.jl:202-210 */
static void k_kinetic_energy(const oracle_model* m, double* K, double* B, const double* u, const double* h) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < m->nc; ++i) {
    double s = 0.0;
    for (int k = 0; k < m->cw; ++k) {
      double ue = u[IX(m->cell_edges, m->cw, k, i)];
      s += AT(m->kinetic, m->cw, k, i) * (ue * ue);
    }
    K[i] = s;
    B[i] = s + m->gravity * h[i];
  }
}

/* vertex_kinetic_energy_kernel!, :212-219 */
static void k_vertex_kinetic_energy(const oracle_model* m, double* Kv, const double* u) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t v = 0; v < m->nv; ++v) {
    double s = 0.0;
    for (int k = 0; k < m->vw; ++k) {
      double ue = u[IX(m->vertex_edges, m->vw, k, v)];
      s += AT(m->vk_weights, m->vw, k, v) * (ue * ue);
    }
    Kv[v] = s;
  }
}

/* cell_from_vertex_kernel!, :222-230 */
static void k_cell_from_vertex(const oracle_model* m, double* K, double* B, const double* Kv) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < m->nc; ++i) {
    double s = 0.0;
    for (int k = 0; k < m->cw; ++k) s += AT(m->vk_kites, m->cw, k, i) * Kv[IX(m->vk_cell_vertices, m->cw, k, i)];
    K[i] += s;
    B[i] += s;
  }
}

/* mass_flux_kernel!, :232-235 */
static void k_mass_flux(const oracle_model* m, double* F, const double* u, const double* h) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e)
    F[e] = (AT(m->edge_height, 2, 0, e) * h[IX(m->edge_cells, 2, 0, e)] +
            AT(m->edge_height, 2, 1, e) * h[IX(m->edge_cells, 2, 1, e)]) *
           u[e];
}

/* mixed_mass_flux_kernel!, :238-244 */
static void k_mixed_mass_flux(const oracle_model* m, double* F, const double* u, const double* h, const double* hv) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e)
    F[e] = (AT(m->edge_height, 2, 0, e) * h[IX(m->edge_cells, 2, 0, e)] +
            AT(m->edge_height, 2, 1, e) * h[IX(m->edge_cells, 2, 1, e)] +
            AT(m->vk_height, 2, 0, e) * hv[IX(m->edge_vertices, 2, 0, e)] +
            AT(m->vk_height, 2, 1, e) * hv[IX(m->edge_vertices, 2, 1, e)]) *
           u[e];
}

/* vertex_pv_kernel!, :246-259 */
static void k_vertex_pv(const oracle_model* m, double* qv, double* zv, double* hv, const double* u, const double* h) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t v = 0; v < m->nv; ++v) {
    double z = 0.0, eta = 0.0;
    for (int k = 0; k < m->vw; ++k) z += AT(m->curl, m->vw, k, v) * u[IX(m->vertex_edges, m->vw, k, v)];
    for (int k = 0; k < m->vw; ++k) eta += AT(m->vertex_height, m->vw, k, v) * h[IX(m->vertex_cells, m->vw, k, v)];
    zv[v] = z;
    hv[v] = eta;
    qv[v] = (z + m->coriolis[v]) / eta;
  }
}

/* edge_pv_kernel!, :261-264 */
static void k_edge_pv(const oracle_model* m, double* qe, const double* qv) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e)
    qe[e] = (qv[IX(m->edge_vertices, 2, 0, e)] + qv[IX(m->edge_vertices, 2, 1, e)]) / 2;
}

/* rhombus_pv_kernel!, :266-273 */
static void k_rhombus_pv(const oracle_model* m, double* qe, const double* zv, const double* hv) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e) {
    int64_t v1 = IX(m->edge_vertices, 2, 0, e), v2 = IX(m->edge_vertices, 2, 1, e);
    double z = AT(m->rhombus, 2, 0, e) * zv[v1] + AT(m->rhombus, 2, 1, e) * zv[v2];
    double eta = AT(m->rhombus, 2, 0, e) * hv[v1] + AT(m->rhombus, 2, 1, e) * hv[v2];
    qe[e] = (z + m->g_coriolis[e]) / eta;
  }
}

/* momentum_kernel!, :275-284 (serial: every edge is owned) */
static void k_momentum(const oracle_model* m, double* du, const double* F, const double* qe, const double* B) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e) {
    double s = 0.0;
    for (int k = 0; k < m->tw; ++k) {
      int64_t ep = IX(m->trisk_edges, m->tw, k, e);
      s += AT(m->trisk, m->tw, k, e) * F[ep] * (qe[e] + qe[ep]);
    }
    du[e] = s / 2 - (B[IX(m->edge_cells, 2, 1, e)] - B[IX(m->edge_cells, 2, 0, e)]) * m->inverse_dual[e];
  }
}

/* gassmann_momentum_kernel!, :286-296 */
static void k_gassmann_momentum(const oracle_model* m, double* du, const double* F, const double* qe, const double* B,
                                int mean) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t e = 0; e < m->ne; ++e) {
    double s = 0.0;
    for (int k = 0; k < 12; ++k) {
      int64_t ep = IX(m->g_edges, 12, k, e);
      double q = mean ? (qe[e] + qe[ep]) / 2 : qe[IX(m->g_pv_edges, 12, k, e)];
      s += AT(m->g_weights, 12, k, e) * F[ep] * q;
    }
    du[e] = s - (B[IX(m->edge_cells, 2, 1, e)] - B[IX(m->edge_cells, 2, 0, e)]) * m->inverse_dual[e];
  }
}

/* continuity_kernel!, :298-305 */
static void k_continuity(const oracle_model* m, double* dh, const double* F) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < m->nc; ++i) {
    double s = 0.0;
    for (int k = 0; k < m->cw; ++k) s += AT(m->divergence, m->cw, k, i) * F[IX(m->cell_edges, m->cw, k, i)];
    dh[i] = -s;
  }
}

/* kinetic_energy!, :332-340 */
void oracle_kinetic_energy(const oracle_model* m, oracle_work* w, const double* u, const double* h) {
  k_kinetic_energy(m, w->K, w->B, u, h);
  if (m->alpha != 1.0) {
    k_vertex_kinetic_energy(m, w->Kv, u);
    k_cell_from_vertex(m, w->K, w->B, w->Kv);
  }
}

/* mass_flux!, :343-352 */
void oracle_mass_flux(const oracle_model* m, oracle_work* w, const double* u, const double* h) {
  if (m->alpha == 1.0)
    k_mass_flux(m, w->F, u, h);
  else
    k_mixed_mass_flux(m, w->F, u, h, w->hv);
}

/* vertex_pv!, :355-360 */
void oracle_vertex_pv(const oracle_model* m, oracle_work* w, const double* u, const double* h) {
  k_vertex_pv(m, w->qv, w->zv, w->hv, u, h);
}

/* tendency!, :379-394 (serial: no halo exchange, no ghost zeroing) */
void oracle_tendency(const oracle_model* m, oracle_work* w, const double* y, double* dy) {
  const double* u = y;
  const double* h = y + m->ne;
  double* du = dy;
  double* dh = dy + m->ne;
  oracle_kinetic_energy(m, w, u, h);
  oracle_vertex_pv(m, w, u, h);
  oracle_mass_flux(m, w, u, h);
  if (m->pv_flux == 0) { /* pv_flux!(du, m, ::Nothing), :363-369 */
    k_edge_pv(m, w->qe, w->qv);
    k_momentum(m, du, w->F, w->qe, w->B);
  } else { /* pv_flux!(du, m, ::NamedTuple), :371-377 */
    k_rhombus_pv(m, w->qe, w->zv, w->hv);
    k_gassmann_momentum(m, du, w->F, w->qe, w->B, m->pv_flux == 2);
  }
  k_continuity(m, dh, w->F);
}

/* rk4_step!, RungeKutta.jl:18-29: broadcasts written out element by element */
void oracle_rk4_step(const oracle_model* m, oracle_work* w, double* y, double dt, double* cache) {
  const int64_t n = m->ne + m->nc;
  double* k1 = cache;
  double* k2 = cache + n;
  double* k3 = cache + 2 * n;
  double* k4 = cache + 3 * n;
  double* st = cache + 4 * n;
  const double half = dt / 2, sixth = dt / 6;
  oracle_tendency(m, w, y, k1);
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < n; ++i) st[i] = y[i] + half * k1[i];
  oracle_tendency(m, w, st, k2);
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < n; ++i) st[i] = y[i] + half * k2[i];
  oracle_tendency(m, w, st, k3);
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < n; ++i) st[i] = y[i] + dt * k3[i];
  oracle_tendency(m, w, st, k4);
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < n; ++i) y[i] += sixth * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]);
}

/* total_mass, :397-399 */
double oracle_total_mass(const oracle_model* m, const double* y) {
  const double* h = y + m->ne;
  double s = 0.0;
  for (int64_t i = 0; i < m->nc; ++i) s += m->cell_areas[i] * h[i];
  return s;
}

/* total_energy, :406-411 */
double oracle_total_energy(const oracle_model* m, oracle_work* w, const double* y) {
  const double* h = y + m->ne;
  oracle_kinetic_energy(m, w, y, h);
  double s = 0.0;
  for (int64_t i = 0; i < m->nc; ++i) s += m->cell_areas[i] * h[i] * (w->K[i] + m->gravity * h[i] / 2);
  return s;
}

/* potential_enstrophy, :414-419 */
double oracle_potential_enstrophy(const oracle_model* m, oracle_work* w, const double* y) {
  oracle_vertex_pv(m, w, y, y + m->ne);
  double s = 0.0;
  for (int64_t v = 0; v < m->nv; ++v) s += m->vertex_areas[v] * w->hv[v] * (w->qv[v] * w->qv[v]);
  return s / 2;
}

/* edge_sum_kernel!, :307-314, as relative_vorticity (:421-426) */
void oracle_relative_vorticity(const oracle_model* m, const double* y, double* zeta) {
  for (int64_t v = 0; v < m->nv; ++v) {
    double s = 0.0;
    for (int k = 0; k < m->vw; ++k) s += AT(m->curl, m->vw, k, v) * y[IX(m->vertex_edges, m->vw, k, v)];
    zeta[v] = s;
  }
}

/* edge_sum_kernel!, as tangential_velocity (:428-433) */
void oracle_tangential_velocity(const oracle_model* m, const double* u, double* vt) {
  for (int64_t e = 0; e < m->ne; ++e) {
    double s = 0.0;
    for (int k = 0; k < m->tw; ++k) s += AT(m->trisk, m->tw, k, e) * u[IX(m->trisk_edges, m->tw, k, e)];
    vt[e] = s;
  }
}
