// C ABI of the host-side mesh generator and TRiSK grid builder (see include/trisk_b200.h).
#include <cstring>
#include <memory>

#include "common.hpp"

namespace trisk {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace trisk

struct TriskMesh {
  trisk::HexMesh hex;
  // 1-based copies of the Plex arrays, as Julia holds them
  std::vector<int64_t> cone_offsets, cones, orientations, support_offsets, supports;
  bool grid_built = false;
  trisk::Grid grid;
  std::vector<int64_t> edge_cells, edge_vertices, cell_edges, cell_vertices, vertex_edges, vertex_cells,
      trisk_edges;
};

static std::vector<int64_t> plus_one(const std::vector<int64_t>& v) {
  std::vector<int64_t> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i] + 1;
  return out;
}

static const double* flat(const std::vector<trisk::V3>& v) { return reinterpret_cast<const double*>(v.data()); }

static void copy_plex(TriskMesh* m) {
  const trisk::Plex& p = m->hex.plex;
  m->cone_offsets = plus_one(p.cone_offsets);
  m->cones = plus_one(p.cones);
  m->orientations.assign(p.orientations.begin(), p.orientations.end());
  m->support_offsets = plus_one(p.support_offsets);
  m->supports = plus_one(p.supports);
}

static void ensure_grid(TriskMesh* m) {
  if (m->grid_built) return;
  m->grid = trisk::build_grid(m->hex.plex, m->hex.generators);
  const trisk::Grid& g = m->grid;
  m->edge_cells = plus_one(g.edge_cells);
  m->edge_vertices = plus_one(g.edge_vertices);
  m->cell_edges = plus_one(g.cell_edges);
  m->cell_vertices = plus_one(g.cell_vertices);
  m->vertex_edges = plus_one(g.vertex_edges);
  m->vertex_cells = plus_one(g.vertex_cells);
  m->trisk_edges = plus_one(g.trisk_edges);
  m->grid_built = true;
}

extern "C" {

size_t trisk_last_error(char* buf, size_t len) {
  const std::string& s = trisk::g_last_error;
  if (buf && len) {
    size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

int32_t trisk_abi_version(void) { return 1; }

int32_t trisk_struct_size(int32_t which) {
  switch (which) {
    case 0: return (int32_t)sizeof(TriskGrid);
    case 1: return (int32_t)sizeof(TriskCoefficients);
    case 2: return (int32_t)sizeof(TriskConfig);
    case 3: return (int32_t)sizeof(TriskPlex);
    case 4: return (int32_t)sizeof(TriskIconTables);
    case 5: return (int32_t)sizeof(TriskMpasTables);
    case 6: return (int32_t)sizeof(TriskMpasFields);
    case 7: return (int32_t)sizeof(TriskHalo);
    default: return -1;
  }
}

int trisk_mesh_create_hexagon(int32_t subdivisions, int32_t centroidal, double spring_beta, TriskMesh** out) {
  TRISK_API_BEGIN
  if (!out) throw trisk::Error(TRISK_ERR_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (subdivisions < 0 || subdivisions > 10)
    throw trisk::Error(TRISK_ERR_ARGUMENT, "subdivisions must be in 0..10");
  if (!(spring_beta >= 0)) throw trisk::Error(TRISK_ERR_ARGUMENT, "spring_beta must be >= 0");
  auto m = std::make_unique<TriskMesh>();
  m->hex = trisk::create_hexagon_mesh(subdivisions, centroidal != 0, spring_beta);
  copy_plex(m.get());
  *out = m.release();
  TRISK_API_END
}

int trisk_mesh_create_triangles(int32_t subdivisions, int32_t centroidal, double spring_beta, TriskMesh** out) {
  TRISK_API_BEGIN
  if (!out) throw trisk::Error(TRISK_ERR_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (subdivisions < 0 || subdivisions > 10)
    throw trisk::Error(TRISK_ERR_ARGUMENT, "subdivisions must be in 0..10");
  if (!(spring_beta >= 0)) throw trisk::Error(TRISK_ERR_ARGUMENT, "spring_beta must be >= 0");
  auto m = std::make_unique<TriskMesh>();
  m->hex = trisk::create_triangle_mesh(subdivisions, centroidal != 0, spring_beta);
  copy_plex(m.get());
  *out = m.release();
  TRISK_API_END
}

int trisk_mesh_from_polygons(const int64_t* offsets, const int64_t* vertices, int64_t npolygons,
                             const double* coordinates, int64_t nv, const double* centers, TriskMesh** out) {
  // plex_from_polygons(polygons, coordinates) (Plex.jl:49-97), as the grid readers call it
  // (FileGrids.jl:59,67,91,94)
  TRISK_API_BEGIN
  if (!out) throw trisk::Error(TRISK_ERR_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (!offsets || !vertices || !coordinates) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  if (npolygons <= 0 || nv < 3) throw trisk::Error(TRISK_ERR_ARGUMENT, "need at least one polygon and three vertices");
  if (offsets[0] != 1) throw trisk::Error(TRISK_ERR_ARGUMENT, "offsets[0] must be 1");
  std::vector<std::vector<int64_t>> polys(npolygons);
  for (int64_t c = 0; c < npolygons; ++c) {
    const int64_t a = offsets[c], b = offsets[c + 1];
    if (b - a < 3) throw trisk::Error(TRISK_ERR_ARGUMENT, "polygon " + std::to_string(c + 1) + " has fewer than three vertices");
    polys[c].reserve(b - a);
    for (int64_t i = a; i < b; ++i) {
      const int64_t v = vertices[i - 1];
      if (v < 1 || v > nv)
        throw trisk::Error(TRISK_ERR_ARGUMENT, "polygon " + std::to_string(c + 1) + " names vertex " + std::to_string(v) +
                                                   " outside 1.." + std::to_string(nv));
      polys[c].push_back(v - 1);
    }
  }
  std::vector<trisk::V3> x(nv);
  std::memcpy(x.data(), coordinates, nv * sizeof(trisk::V3));
  auto m = std::make_unique<TriskMesh>();
  m->hex.plex = trisk::plex_from_polygons(polys, x);
  m->hex.generators.resize(npolygons);
  if (centers) {
    std::memcpy(m->hex.generators.data(), centers, npolygons * sizeof(trisk::V3));
  } else {  // the normalized vertex means (CellCenters.jl:35-36); plain means on a plane
    for (int64_t c = 0; c < npolygons; ++c) {
      trisk::V3 s{0, 0, 0};
      for (int64_t v : polys[c]) s = s + x[v];
      m->hex.generators[c] = m->hex.plex.sphere ? trisk::normalize(s) : s / (double)polys[c].size();
    }
  }
  copy_plex(m.get());
  *out = m.release();
  TRISK_API_END
}

int trisk_mesh_set_centers(TriskMesh* m, const double* centers) {
  TRISK_API_BEGIN
  if (!m || !centers) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  std::memcpy(m->hex.generators.data(), centers, m->hex.generators.size() * sizeof(trisk::V3));
  m->grid_built = false;  // the next trisk_mesh_grid rebuilds the tables for these centers
  TRISK_API_END
}

void trisk_mesh_destroy(TriskMesh* mesh) { delete mesh; }

int trisk_icosahedral_mesh(int32_t subdivisions, int32_t centroidal, double spring_beta, double* x,
                           int64_t* triangles) {
  TRISK_API_BEGIN
  if (!x || !triangles) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  if (subdivisions < 0 || subdivisions > 10)
    throw trisk::Error(TRISK_ERR_ARGUMENT, "subdivisions must be in 0..10");
  trisk::TriangleMesh tm = trisk::icosahedral_triangles(subdivisions, centroidal != 0, spring_beta);
  std::memcpy(x, tm.x.data(), tm.x.size() * sizeof(trisk::V3));
  for (size_t t = 0; t < tm.triangles.size(); ++t)
    for (int k = 0; k < 3; ++k) triangles[3 * t + k] = tm.triangles[t][k] + 1;
  TRISK_API_END
}

int trisk_lloyd(double* x, int64_t n, const int64_t* triangles, int64_t nt, int32_t n_fixed, int32_t history,
                int32_t* iterations) {
  TRISK_API_BEGIN
  if (!x || !triangles || !iterations || n <= 0 || nt <= 0) throw trisk::Error(TRISK_ERR_ARGUMENT, "bad argument");
  std::vector<trisk::V3> pts(n);
  std::memcpy(pts.data(), x, n * sizeof(trisk::V3));
  std::vector<std::array<int64_t, 3>> tris(nt);
  for (int64_t t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) {
      int64_t v = triangles[3 * t + k];
      if (v < 1 || v > n) throw trisk::Error(TRISK_ERR_ARGUMENT, "triangle index out of range");
      tris[t][k] = v - 1;
    }
  *iterations = trisk::lloyd(pts, tris, n_fixed, 1e-8, history, 10000);
  std::memcpy(x, pts.data(), n * sizeof(trisk::V3));
  TRISK_API_END
}

int trisk_mesh_plex(TriskMesh* m, TriskPlex* out) {
  TRISK_API_BEGIN
  if (!m || !out) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  const trisk::Plex& p = m->hex.plex;
  out->nc = p.nc;
  out->ne = p.ne;
  out->nv = p.nv;
  out->ncones = (int64_t)p.cones.size();
  out->cone_offsets = m->cone_offsets.data();
  out->cones = m->cones.data();
  out->cone_orientations = m->orientations.data();
  out->support_offsets = m->support_offsets.data();
  out->supports = m->supports.data();
  out->coordinates = flat(p.coordinates);
  TRISK_API_END
}

int trisk_mesh_generators(TriskMesh* m, const double** out) {
  TRISK_API_BEGIN
  if (!m || !out) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = flat(m->hex.generators);
  TRISK_API_END
}

int trisk_mesh_grid(TriskMesh* m, TriskGrid* out) {
  TRISK_API_BEGIN
  if (!m || !out) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  ensure_grid(m);
  const trisk::Grid& g = m->grid;
  std::memset(out, 0, sizeof(*out));
  out->nc = g.nc;
  out->ne = g.ne;
  out->nv = g.nv;
  out->cw = g.cw;
  out->vw = g.vw;
  out->tw = g.tw;
  out->centers = flat(g.centers);
  out->vertices = flat(g.vertices);
  out->edge_points = flat(g.edge_points);
  out->edge_normals = flat(g.edge_normals);
  out->primal_lengths = g.primal_lengths.data();
  out->dual_lengths = g.dual_lengths.data();
  out->edge_cells = m->edge_cells.data();
  out->edge_vertices = m->edge_vertices.data();
  out->cell_distances = g.cell_distances.data();
  out->cell_areas = g.cell_areas.data();
  out->vertex_areas = g.vertex_areas.data();
  out->cell_edges = m->cell_edges.data();
  out->cell_signs = g.cell_signs.data();
  out->cell_vertices = m->cell_vertices.data();
  out->cell_kites = g.cell_kites.data();
  out->vertex_edges = m->vertex_edges.data();
  out->vertex_signs = g.vertex_signs.data();
  out->vertex_cells = m->vertex_cells.data();
  out->vertex_kites = g.vertex_kites.data();
  out->trisk_edges = m->trisk_edges.data();
  out->trisk_weights = g.trisk_weights.data();
  TRISK_API_END
}

int trisk_mesh_hilbert_permutation(TriskMesh* m, int64_t* perm) {
  TRISK_API_BEGIN
  if (!m || !perm) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  auto p = trisk::hilbert_permutation(m->hex.plex, 16);
  for (size_t i = 0; i < p.size(); ++i) perm[i] = p[i] + 1;
  TRISK_API_END
}

int trisk_mesh_orthogonality_defect(TriskMesh* m, double* out) {
  TRISK_API_BEGIN
  if (!m || !out) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = trisk::orthogonality_defect(m->hex.plex, m->hex.generators);
  TRISK_API_END
}

int trisk_mesh_vertex_edge_areas(TriskMesh* m, double* by_vertex, double* by_edge) {
  TRISK_API_BEGIN
  if (!m || !by_vertex || !by_edge) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  ensure_grid(m);
  std::vector<double> bv, be;
  trisk::vertex_edge_areas(m->grid, bv, be);
  std::memcpy(by_vertex, bv.data(), bv.size() * sizeof(double));
  std::memcpy(by_edge, be.data(), be.size() * sizeof(double));
  TRISK_API_END
}

int trisk_mesh_gassmann(TriskMesh* m, int64_t* edges, int64_t* pv_edges, double* weights) {
  TRISK_API_BEGIN
  if (!m || !edges || !pv_edges || !weights) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  ensure_grid(m);
  std::vector<int64_t> E, P;
  std::vector<double> W;
  trisk::gassmann_coefficients(m->grid, E, P, W);
  for (size_t i = 0; i < E.size(); ++i) {
    edges[i] = E[i] + 1;
    pv_edges[i] = P[i] + 1;
  }
  std::memcpy(weights, W.data(), W.size() * sizeof(double));
  TRISK_API_END
}

}  // extern "C"
