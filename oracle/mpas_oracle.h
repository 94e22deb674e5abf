/*
 * CPU oracle (test infrastructure, never shipped) of the MPAS-Gassmann horizontal operators;
 * see mpas_oracle.c for the reference lines it restates.
 */
#ifndef MPAS_ORACLE_H
#define MPAS_ORACLE_H

#include <stdint.h>

typedef struct {
  int64_t nc, ne, nv, nlev;
  int32_t cw, vw, nt, vk, iap_pv, vertical, five_band, reserved;
  const int64_t *cell_edges, *edge_cells, *edge_vertices, *vertex_edges, *vertex_cells, *vk_cell_vertices;
  const double *kinetic, *inner, *vk_kites, *edge_weight, *rhombus, *inverse_dual, *edge_coriolis, *curl,
      *vertex_weight, *vk_weights, *coriolis, *trisk, *dz_cells, *dzh_cells, *wlow, *dz_edges, *dzh_edges;
  const int32_t* trisk_index;
} mpas_oracle_tables;

typedef struct {
  const double *vn, *w, *rho, *rt;
  double *theta, *exner, *K, *Kv, *qv, *zv, *rv, *qe, *rhoe, *Fs, *eta, *tvn, *tw, *Kh;
} mpas_oracle_fields;

void mpas_oracle_set_threads(int threads);
int mpas_oracle_tables_size(void);
int mpas_oracle_fields_size(void);
void mpas_oracle_slow_tendencies(const mpas_oracle_tables* t, mpas_oracle_fields* f, double pressure);

#endif
