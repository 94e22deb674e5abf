/*
 * CPU oracle (test infrastructure, never shipped): the MPAS-Gassmann horizontal operators of
 * dmplex.jl (slow_tendencies! for flat ground, src/Nonhydrostatic/MPAS/Gassmann/
 * Stepping.jl:22-56) in plain C with OpenMP over entities, for the timed CPU baseline of the
 * operators. It restates the same kernels as oracle/mpas_oracle.py (which cites every
 * reference line) with the same loop, summation and association order, and
 * -ffp-contract=off, so the two agree bit for bit (tests/test_mpas.py checks that):
 *
 *   vertex_pv_kernel!, vertex_kinetic_kernel!   Operators.jl:88-102, 18-25
 *   diagnose_kernel!, cell_from_vertex_kernel!,
 *   w_kinetic_kernel!                           Operators.jl:6-15, 28-35, 38-41
 *   edge_pv_kernel!, edge_density_kernel!,
 *   eta_kernel!                                 Operators.jl:104-115, 55-63, 44-52
 *   w_tendency_vi_kernel!, w_tendency_kernel!   Operators.jl:69-86, 118-133
 *   edge_w, vn_tendency_kernel! (oro = 0)       Gassmann/Tendencies.jl:4-12, 38-75
 *
 * Tables as the Python oracle holds them: 1-based Int64 (entity, k) row-major, trisk
 * (ne, nt) and trisk_index (ne, nt, 3) row-major; fields (nlev [+ 1], n) row-major.
 */
#include "mpas_oracle.h"

#include <math.h>

static int g_mpas_threads = 1;

void mpas_oracle_set_threads(int threads) { g_mpas_threads = threads < 1 ? 1 : threads; }
int mpas_oracle_tables_size(void) { return (int)sizeof(mpas_oracle_tables); }
int mpas_oracle_fields_size(void) { return (int)sizeof(mpas_oracle_fields); }

#define RD 287.0
#define CPD 1004.0
#define CVD (CPD - RD)
#define P0 1.0e5

#define T2(A, w, i, j) ((A)[(int64_t)(i) * (w) + (j)])
#define F2(A, n, k, i) ((A)[(int64_t)(k) * (n) + (i)])

static double edge_w(const mpas_oracle_tables* t, const mpas_oracle_fields* f, int64_t e, int64_t l, int64_t r,
                     int64_t j, int mw) {
  const int64_t nc = t->nc;
  const double w0 = T2(t->edge_weight, 2, e, 0), w1 = T2(t->edge_weight, 2, e, 1);
  double hl = 1.0, hr = 1.0;
  if (mw) {
    hl = F2(t->wlow, nc, j, l) * F2(f->rho, nc, j - 1, l) + (1 - F2(t->wlow, nc, j, l)) * F2(f->rho, nc, j, l);
    hr = F2(t->wlow, nc, j, r) * F2(f->rho, nc, j - 1, r) + (1 - F2(t->wlow, nc, j, r)) * F2(f->rho, nc, j, r);
  }
  const double M = w0 * hl * F2(f->w, nc, j, l) + w1 * hr * F2(f->w, nc, j, r);
  return M / (w0 * hl + w1 * hr);
}

void mpas_oracle_slow_tendencies(const mpas_oracle_tables* t, mpas_oracle_fields* f, double pressure) {
  const int64_t nc = t->nc, ne = t->ne, nv = t->nv, nl = t->nlev;
  const int cw = t->cw, vw = t->vw, nt = t->nt;
  const int threads = g_mpas_threads;
  const int mw = t->vertical == 2;

  /* vertices: zeta, rho_v, q_v (+ K_v) */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t v = 0; v < nv; ++v)
    for (int64_t k = 0; k < nl; ++k) {
      double z = 0.0, h = 0.0;
      for (int j = 0; j < vw; ++j) z += T2(t->curl, vw, v, j) * F2(f->vn, ne, k, T2(t->vertex_edges, vw, v, j) - 1);
      for (int j = 0; j < vw; ++j)
        h += T2(t->vertex_weight, vw, v, j) * F2(f->rho, nc, k, T2(t->vertex_cells, vw, v, j) - 1);
      F2(f->zv, nv, k, v) = z;
      F2(f->rv, nv, k, v) = h;
      F2(f->qv, nv, k, v) = (z + t->coriolis[v]) / h;
      if (t->vk) {
        double s = 0.0;
        for (int j = 0; j < vw; ++j) {
          const double x = F2(f->vn, ne, k, T2(t->vertex_edges, vw, v, j) - 1);
          s += T2(t->vk_weights, vw, v, j) * (x * x);
        }
        F2(f->Kv, nv, k, v) = s;
      }
    }

  /* cells: theta, pi, K (K_h kept for the five-band w tendency) */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t i = 0; i < nc; ++i)
    for (int64_t k = 0; k < nl; ++k) {
      double s = 0.0;
      for (int j = 0; j < cw; ++j) {
        const double x = F2(f->vn, ne, k, T2(t->cell_edges, cw, i, j) - 1);
        s += T2(t->kinetic, cw, i, j) * (x * x);
      }
      double K = s;
      const double rt = F2(f->rt, nc, k, i);
      F2(f->theta, nc, k, i) = rt / F2(f->rho, nc, k, i);
      F2(f->exner, nc, k, i) = pow(RD * rt / P0, RD / CVD);
      if (t->vk) {
        double sv = 0.0;
        for (int j = 0; j < cw; ++j)
          sv += T2(t->vk_kites, cw, i, j) * F2(f->Kv, nv, k, T2(t->vk_cell_vertices, cw, i, j) - 1);
        K = K + sv;
      }
      F2(f->Kh, nc, k, i) = K;
      if (t->vertical > 0) {
        const double wl = F2(f->w, nc, k, i), wu = F2(f->w, nc, k + 1, i);
        K = K + (F2(t->dzh_cells, nc, k, i) * (wl * wl) + F2(t->dzh_cells, nc, k + 1, i) * (wu * wu)) /
                    (4 * F2(t->dz_cells, nc, k, i));
      }
      F2(f->K, nc, k, i) = K;
    }

  /* edges: q_e, rho_e, F_s at the layers; eta at the interfaces */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t l = T2(t->edge_cells, 2, e, 0) - 1, r = T2(t->edge_cells, 2, e, 1) - 1;
    const int64_t v1 = T2(t->edge_vertices, 2, e, 0) - 1, v2 = T2(t->edge_vertices, 2, e, 1) - 1;
    const double w0 = T2(t->edge_weight, 2, e, 0), w1 = T2(t->edge_weight, 2, e, 1);
    for (int64_t k = 0; k < nl; ++k) {
      const double re = w0 * F2(f->rho, nc, k, l) + w1 * F2(f->rho, nc, k, r);
      F2(f->rhoe, ne, k, e) = re;
      F2(f->Fs, ne, k, e) = re * F2(f->vn, ne, k, e);
      if (t->iap_pv) {
        const double r0 = T2(t->rhombus, 2, e, 0), r1 = T2(t->rhombus, 2, e, 1);
        const double z = r0 * F2(f->zv, nv, k, v1) + r1 * F2(f->zv, nv, k, v2);
        const double h = r0 * F2(f->rv, nv, k, v1) + r1 * F2(f->rv, nv, k, v2);
        F2(f->qe, ne, k, e) = (z + t->edge_coriolis[e]) / h;
      } else {
        F2(f->qe, ne, k, e) = (F2(f->qv, nv, k, v1) + F2(f->qv, nv, k, v2)) / 2;
      }
    }
    if (t->vertical > 0)
      for (int64_t k = 0; k <= nl; ++k) {
        double x = 0.0;
        if (k >= 1 && k <= nl - 1)
          x = (F2(f->vn, ne, k, e) - F2(f->vn, ne, k - 1, e)) / F2(t->dzh_edges, ne, k, e) -
              (F2(f->w, nc, k, r) - F2(f->w, nc, k, l)) * t->inverse_dual[e];
        F2(f->eta, ne, k, e) = x;
      }
  }

  /* cells x interfaces: the w tendency */
  const double* Kw = t->five_band ? f->Kh : f->K;
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t i = 0; i < nc; ++i)
    for (int64_t k = 0; k <= nl; ++k) {
      if (k == 0 || k == nl) {
        F2(f->tw, nc, k, i) = 0.0;
        continue;
      }
      double s = 0.0;
      if (t->vertical > 0) {
        const double wl = F2(t->wlow, nc, k, i);
        for (int n = 0; n < cw; ++n) {
          const int64_t e = T2(t->cell_edges, cw, i, n) - 1;
          const double rl = mw ? F2(f->rhoe, ne, k - 1, e) : 1.0, ru = mw ? F2(f->rhoe, ne, k, e) : 1.0;
          s += T2(t->inner, cw, i, n) * F2(f->eta, ne, k, e) *
               (rl * F2(f->vn, ne, k - 1, e) + ru * F2(f->vn, ne, k, e)) / (2 * (wl * rl + (1 - wl) * ru));
        }
        F2(f->tw, nc, k, i) = s - (F2(Kw, nc, k, i) - F2(Kw, nc, k - 1, i)) / F2(t->dzh_cells, nc, k, i);
      } else {
        for (int n = 0; n < cw; ++n) {
          const int64_t e = T2(t->cell_edges, cw, i, n) - 1;
          const int64_t el = T2(t->edge_cells, 2, e, 0) - 1, er = T2(t->edge_cells, 2, e, 1) - 1;
          const double v = (F2(f->vn, ne, k - 1, e) + F2(f->vn, ne, k, e)) / 2;
          s += 2 * T2(t->kinetic, cw, i, n) * v * (F2(f->w, nc, k, er) - F2(f->w, nc, k, el)) * t->inverse_dual[e];
        }
        F2(f->tw, nc, k, i) = -s - F2(f->w, nc, k, i) * (F2(f->w, nc, k + 1, i) - F2(f->w, nc, k - 1, i)) /
                                       (F2(t->dz_cells, nc, k - 1, i) + F2(t->dz_cells, nc, k, i));
      }
    }

  /* edges x layers: the vn tendency */
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads)
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t l = T2(t->edge_cells, 2, e, 0) - 1, r = T2(t->edge_cells, 2, e, 1) - 1;
    const double w0 = T2(t->edge_weight, 2, e, 0), w1 = T2(t->edge_weight, 2, e, 1);
    const double invd = t->inverse_dual[e];
    for (int64_t k = 0; k < nl; ++k) {
      double s = 0.0;
      for (int j = 0; j < nt; ++j) {
        const int32_t* ti = t->trisk_index + ((int64_t)e * nt + j) * 3;
        s += T2(t->trisk, nt, e, j) * F2(f->Fs, ne, k, ti[0] - 1) *
             (F2(f->qe, ne, k, ti[1] - 1) + F2(f->qe, ne, k, ti[2] - 1));
      }
      const double te = w0 * F2(f->theta, nc, k, l) + w1 * F2(f->theta, nc, k, r);
      double out = s - invd * (F2(f->K, nc, k, r) - F2(f->K, nc, k, l));
      if (pressure > 0) {
        const double dpi = (F2(f->exner, nc, k, r) - F2(f->exner, nc, k, l)) * invd;
        out = out - pressure * (CPD * te * dpi);
      }
      if (t->vertical > 0) {
        const double Wl = k > 0 ? edge_w(t, f, e, l, r, k, mw) : 0.0;
        const double Wu = k < nl - 1 ? edge_w(t, f, e, l, r, k + 1, mw) : 0.0;
        F2(f->tvn, ne, k, e) = out - (F2(t->dzh_edges, ne, k, e) * F2(f->eta, ne, k, e) * Wl +
                                      F2(t->dzh_edges, ne, k + 1, e) * F2(f->eta, ne, k + 1, e) * Wu) /
                                         (2 * F2(t->dz_edges, ne, k, e));
      } else {
        const double we = (F2(f->w, nc, k, l) + F2(f->w, nc, k, r) + F2(f->w, nc, k + 1, l) + F2(f->w, nc, k + 1, r)) / 4;
        const double vc = F2(f->vn, ne, k, e);
        const double vlow = k > 0 ? (F2(f->vn, ne, k - 1, e) + vc) / 2 : vc;
        const double vup = k < nl - 1 ? (vc + F2(f->vn, ne, k + 1, e)) / 2 : vc;
        F2(f->tvn, ne, k, e) = out - we * (vup - vlow) / F2(t->dz_edges, ne, k, e);
      }
    }
  }
}
