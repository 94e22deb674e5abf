/*
 * CPU oracle (test infrastructure, never shipped) of the ICON triangle shallow-water model;
 * see icon_oracle.c for the reference lines it restates.
 */
#ifndef ICON_ORACLE_H
#define ICON_ORACLE_H

#include <stdint.h>

typedef struct {
  int64_t nc, ne, nv;
  int32_t vw, reserved;
  double gravity;
  const int64_t *cell_edges, *edge_cells, *edge_vertices, *rbf_edges, *vertex_edges;
  const double *divergence, *bilinear, *edge_height, *gradient, *inverse_dual, *rbf, *edge_coriolis, *curl,
      *cell_areas;
  const double* divergence_damping; /* ne, or NULL */
} icon_oracle_tables;

void icon_oracle_set_threads(int threads);
int icon_oracle_tables_size(void);
void icon_oracle_tendency(const icon_oracle_tables* t, const double* y, double* dy);
void icon_oracle_rk4_step(const icon_oracle_tables* t, double* y, double dt, int64_t nsteps);

#endif
