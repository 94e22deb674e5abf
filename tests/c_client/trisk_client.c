/*
 * A plain-C client of libtrisk_b200.so that uses nothing but include/trisk_b200.h, the way a
 * Julia ccall (or any other FFI) binds the library (test infrastructure). It builds a hexagon
 * mesh and its TRiSK grid through the ABI, checks the struct layouts and the error reporting,
 * builds the model tables on the host and the CPU oracle over them (oracle/trisk_oracle.h).
 *   trisk_client        without a GPU: model creation must fail with TRISK_ERR_CUDA
 *   trisk_client gpu    the tendency and three RK4 steps of the library equal the oracle's
 *                       bit for bit, and the diagnostics agree
 * It prints "cpu ok" or "gpu ok" and exits 0, or names the first failure and exits 1.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "trisk_b200.h"
#include "trisk_oracle.h"

static int failed(const char* what, int status) {
  char msg[512];
  trisk_last_error(msg, sizeof msg);
  fprintf(stderr, "FAIL %s (status %d: %s)\n", what, status, msg);
  return 1;
}

#define REQUIRE(cond, what)                     \
  do {                                          \
    if (!(cond)) {                              \
      fprintf(stderr, "FAIL %s\n", what);       \
      return 1;                                 \
    }                                           \
  } while (0)

int main(int argc, char** argv) {
  const int gpu = argc > 1 && strcmp(argv[1], "gpu") == 0;
  REQUIRE(trisk_abi_version() == 1, "ABI version");
  REQUIRE(trisk_struct_size(0) == (int32_t)sizeof(TriskGrid), "sizeof TriskGrid");
  REQUIRE(trisk_struct_size(1) == (int32_t)sizeof(TriskCoefficients), "sizeof TriskCoefficients");
  REQUIRE(trisk_struct_size(2) == (int32_t)sizeof(TriskConfig), "sizeof TriskConfig");
  REQUIRE(trisk_struct_size(3) == (int32_t)sizeof(TriskPlex), "sizeof TriskPlex");
  REQUIRE(trisk_struct_size(5) == (int32_t)sizeof(TriskMpasTables), "sizeof TriskMpasTables");
  REQUIRE(trisk_struct_size(6) == (int32_t)sizeof(TriskMpasFields), "sizeof TriskMpasFields");
  REQUIRE(trisk_struct_size(99) == -1, "unknown struct");

  /* errors: a status and a message, no exception */
  TriskMesh* bad = NULL;
  int rc = trisk_mesh_create_hexagon(-1, 0, 0.0, &bad);
  char msg[256];
  REQUIRE(rc == TRISK_ERR_ARGUMENT && bad == NULL, "bad subdivisions rejected");
  REQUIRE(trisk_last_error(msg, sizeof msg) > 0 && strlen(msg) > 0, "error message");

  /* create_hexagon_mesh(3) and its TRiSK grid */
  TriskMesh* mesh = NULL;
  if ((rc = trisk_mesh_create_hexagon(3, 0, 0.0, &mesh)) != TRISK_OK) return failed("mesh", rc);
  TriskGrid g;
  if ((rc = trisk_mesh_grid(mesh, &g)) != TRISK_OK) return failed("grid", rc);
  REQUIRE(g.nc == 642 && g.ne == 1920 && g.nv == 1280, "hexagon 3 sizes");
  const int64_t ne = g.ne, nc = g.nc, n = ne + nc;

  /* the Gassmann PV flux with the vertex kinetic energy on the unit sphere */
  TriskConfig cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.pv_flux = TRISK_PV_GASSMANN;
  cfg.reorder = 1;
  cfg.alpha = 0.0;
  cfg.gravity = 1.0;
  cfg.omega = 1.0;
  cfg.use_graph = 1;
  cfg.use_pdl = 1;
  TriskTables* tables = NULL;
  if ((rc = trisk_tables_create(&g, &cfg, &tables)) != TRISK_OK) return failed("host tables", rc);
  TriskCoefficients c;
  if ((rc = trisk_tables_view(tables, &c)) != TRISK_OK) return failed("table view", rc);
  oracle_model om = {c.nc, c.ne, c.nv, c.cw, c.vw, c.tw, c.pv_flux, c.alpha, c.gravity,
                     c.cell_edges, c.divergence, c.kinetic, c.edge_cells, c.edge_height, c.edge_vertices,
                     c.inverse_dual, c.vertex_edges, c.curl, c.vertex_cells, c.vertex_height, c.coriolis,
                     c.trisk_edges, c.trisk, c.cell_areas, c.vertex_areas, c.g_edges, c.g_pv_edges, c.g_weights,
                     c.rhombus, c.g_coriolis, c.vk_cell_vertices, c.vk_kites, c.vk_weights, c.vk_height};
  oracle_work* w = oracle_work_create(&om);

  /* Williamson case 2: u = u0 (-y, x, 0) . n at the edge points, h = 1 - (u0 + u0^2/2) z^2 */
  const double u0 = 0.2;
  double* y = malloc(sizeof(double) * n);
  double* ref = malloc(sizeof(double) * n);
  double* dy = malloc(sizeof(double) * n);
  double* y1 = malloc(sizeof(double) * n);
  double* y2 = malloc(sizeof(double) * n);
  double* cache = malloc(sizeof(double) * 5 * n);
  for (int64_t e = 0; e < ne; ++e) {
    const double* x = g.edge_points + 3 * e;
    const double* nn = g.edge_normals + 3 * e;
    y[e] = u0 * (-x[1] * nn[0] + x[0] * nn[1]);
  }
  for (int64_t i = 0; i < nc; ++i) {
    const double z = g.centers[3 * i + 2];
    y[ne + i] = 1 - (u0 + u0 * u0 / 2) * z * z;
  }
  oracle_tendency(&om, w, y, ref);
  const double dt = 0.2 * sqrt(4 * M_PI / (double)nc);

  if (!gpu) {
    TriskModel* m = NULL;
    rc = trisk_model_create(&g, &cfg, &m);
    REQUIRE(rc == TRISK_ERR_CUDA && m == NULL, "model creation fails loudly without a GPU");
    printf("cpu ok\n");
  } else {
    TriskModel* m = NULL;
    if ((rc = trisk_model_create(&g, &cfg, &m)) != TRISK_OK) return failed("model", rc);
    if ((rc = trisk_tendency(m, y, dy)) != TRISK_OK) return failed("tendency", rc);
    REQUIRE(memcmp(dy, ref, sizeof(double) * n) == 0, "tendency equals the oracle bit for bit");
    memcpy(y1, y, sizeof(double) * n);
    memcpy(y2, y, sizeof(double) * n);
    if ((rc = trisk_rk4_step(m, y1, dt, 3)) != TRISK_OK) return failed("rk4", rc);
    for (int s = 0; s < 3; ++s) oracle_rk4_step(&om, w, y2, dt, cache);
    REQUIRE(memcmp(y1, y2, sizeof(double) * n) == 0, "three RK4 steps equal the oracle bit for bit");
    double mass = 0, energy = 0, enstrophy = 0;
    if ((rc = trisk_diagnostics(m, y1, &mass, &energy, &enstrophy)) != TRISK_OK) return failed("diagnostics", rc);
    const double om_mass = oracle_total_mass(&om, y2);
    REQUIRE(fabs(mass - om_mass) <= 1e-12 * fabs(om_mass), "mass agrees with the oracle");
    trisk_model_destroy(m);
    printf("gpu ok\n");
  }
  oracle_work_destroy(w);
  trisk_tables_destroy(tables);
  trisk_mesh_destroy(mesh);
  free(y);
  free(ref);
  free(dy);
  free(y1);
  free(y2);
  free(cache);
  return 0;
}
