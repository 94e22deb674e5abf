// Host-side mesh and table construction for the TRiSK C-grid shallow-water path.
//
// Everything here is set-up work that runs once per mesh on the CPU. It restates, in
// C++, the mesh generator and the neighbour-table builder of dmplex.jl:
//   - icosahedral bisection + Lloyd/Anderson SCVT  (src/Grids/Icosahedral.jl:22-61,126-216)
//   - Voronoi dual of the icosahedral mesh         (src/Grids/Hexagonal.jl:11-17,
//                                                  src/Grids/CellCenters.jl:37-42,
//                                                  src/Grids/FileGrids.jl:28-42)
//   - the CSR mesh DAG                             (src/Topology/Plex.jl:49-160,201-262)
//   - the Hilbert renumbering of cells             (src/Topology/Ordering.jl:10-92)
//   - TRiSK geometry and padded tables             (src/FiniteVolumes/TRiSKGrid.jl:76-162)
//   - vertex-edge areas and Gassmann coefficients  (src/FiniteVolumes/TRiSKGrid.jl:179-251)
//   - the premultiplied model coefficients         (src/FiniteVolumes/TRiSKShallowWater.jl:94-168)
//
// Indices are 0-based in memory. Tables use the reference's column-major `[k, entity]`
// layout (k fastest), padded with index 0 (the reference's 1) and weight 0.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace trisk {

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return a / norm(a); }
// Julia's sign(): 0.0 for 0.0
inline double jsign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
// great-circle distance, TRiSKGrid.jl:2
inline double arc_length(V3 a, V3 b) { return std::atan2(norm(cross(a, b)), dot(a, b)); }
// signed spherical triangle area, TRiSKGrid.jl:5
inline double signed_triangle_area(V3 a, V3 b, V3 c) {
  return 2 * std::atan2(dot(a, cross(b, c)), 1 + dot(a, b) + dot(b, c) + dot(c, a));
}

struct MeshError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Interpolated surface mesh DAG (Plex.jl:23-34). Points: cells [0,nc), edges [nc,nc+ne),
// vertices [nc+ne, nc+ne+nv). Orientation 0: the cell walks the edge low->high, -1 otherwise.
struct Plex {
  int64_t nc = 0, ne = 0, nv = 0;
  std::vector<int64_t> cone_offsets;  // npoints + 1
  std::vector<int64_t> cones;
  std::vector<int8_t> orientations;
  std::vector<int64_t> support_offsets;  // npoints + 1
  std::vector<int64_t> supports;
  std::vector<V3> coordinates;  // per vertex
  bool sphere = true;

  int64_t npoints() const { return nc + ne + nv; }
  int64_t cone_size(int64_t p) const { return cone_offsets[p + 1] - cone_offsets[p]; }
  const int64_t* cone(int64_t p) const { return cones.data() + cone_offsets[p]; }
  const int8_t* cone_orientation(int64_t p) const { return orientations.data() + cone_offsets[p]; }
  int64_t support_size(int64_t p) const { return support_offsets[p + 1] - support_offsets[p]; }
  const int64_t* support(int64_t p) const { return supports.data() + support_offsets[p]; }
  // stratum-local indices (Plex.jl:183-185)
  int64_t edge_index(int64_t p) const { return p - nc; }
  int64_t vertex_index(int64_t p) const { return p - nc - ne; }
  // (left, right) cells of edge point p, -1 if missing (Plex.jl:210-218)
  std::array<int64_t, 2> edge_cells(int64_t p) const;
  // vertex points of cell c, corner k starts cone edge k (Plex.jl:226-230)
  std::vector<int64_t> cell_vertices(int64_t c) const;
  // BFS transitive support (Plex.jl:251-262)
  std::vector<int64_t> star(int64_t p) const;
};

Plex plex_from_polygons(const std::vector<std::vector<int64_t>>& polygons,
                        const std::vector<V3>& coordinates);

// Triangulated sphere before it is turned into a Plex (Icosahedral.jl:22-61).
struct TriangleMesh {
  std::vector<V3> x;
  std::vector<std::array<int64_t, 3>> triangles;
};
// spring_beta > 0: spring dynamics after every level (Tomita et al. 2002); 0: none.
TriangleMesh icosahedral_triangles(int subdivisions, bool centroidal, double spring_beta = 0.0);
// Spring dynamics on the unit sphere (Icosahedral.jl:78-109). Returns iterations used.
int spring_dynamics(std::vector<V3>& x, const std::vector<std::array<int64_t, 2>>& edges, double beta,
                    double mean_length, int n_fixed, double tolerance = 1e-10, int max_iterations = 100000);
// Lloyd SCVT with Anderson mixing (Icosahedral.jl:126-183). Returns iterations used.
int lloyd(std::vector<V3>& x, const std::vector<std::array<int64_t, 3>>& triangles, int n_fixed,
          double tolerance = 1e-8, int history = 16, int max_iterations = 10000);
Plex create_spherical_mesh(int subdivisions, bool centroidal, double spring_beta = 0.0);

// Voronoi dual: hex cell i = primal vertex i; returns the plex and the generators
// (the primal vertices, passed as `centers` by the reference's examples).
struct HexMesh {
  Plex plex;
  std::vector<V3> generators;
};
HexMesh create_hexagon_mesh(int subdivisions, bool centroidal, double spring_beta = 0.0);
// The triangles of create_spherical_mesh as cells (the ICON C grid), with their circumcenters
// as `generators` (the cell centers).
HexMesh create_triangle_mesh(int subdivisions, bool centroidal, double spring_beta = 0.0);

// 3-D Hilbert key (Ordering.jl:10-41) and the cell permutation (Ordering.jl:85-92).
uint64_t hilbert_key(uint64_t x0, uint64_t x1, uint64_t x2, int bits);
std::vector<int64_t> hilbert_permutation(const Plex& dm, int bits = 16);
// sortperm of the Hilbert keys of given points (the body of hilbert_permutation).
std::vector<int64_t> hilbert_sort(const std::vector<V3>& centroids, int bits = 16);

// Geometry and padded tables (TRiSKGrid.jl:37-162). Layout [k + width*entity].
struct Grid {
  int64_t nc = 0, ne = 0, nv = 0;
  int cw = 0, vw = 0, tw = 0;  // widths of the cell, vertex and TRiSK tables
  std::vector<V3> centers, vertices, edge_points, edge_normals;
  std::vector<double> primal_lengths, dual_lengths;
  std::vector<int64_t> edge_cells, edge_vertices;  // 2 x ne
  std::vector<double> cell_distances;              // 2 x ne
  std::vector<double> cell_areas, vertex_areas;
  std::vector<int64_t> cell_edges, cell_vertices;  // cw x nc
  std::vector<double> cell_signs, cell_kites;
  std::vector<int64_t> vertex_edges, vertex_cells;  // vw x nv
  std::vector<double> vertex_signs, vertex_kites;
  std::vector<int64_t> trisk_edges;  // tw x ne
  std::vector<double> trisk_weights;
};
Grid build_grid(const Plex& dm, const std::vector<V3>& centers);
double orthogonality_defect(const Plex& dm, const std::vector<V3>& centers);
// TRiSKGrid.jl:179-191: by_vertex (vw x nv), by_edge (2 x ne)
void vertex_edge_areas(const Grid& g, std::vector<double>& by_vertex, std::vector<double>& by_edge);
// TRiSKGrid.jl:214-251: 12 x ne each
void gassmann_coefficients(const Grid& g, std::vector<int64_t>& edges, std::vector<int64_t>& pv_edges,
                           std::vector<double>& weights);

enum PvFlux { PV_TRISK = 0, PV_GASSMANN = 1, PV_GASSMANN_MEAN = 2 };

// The premultiplied tables a TRiSKShallowWater model holds (TRiSKShallowWater.jl:67-92),
// serial distribution (identity numbering). Layout [k + width*entity], 0-based indices.
struct Coefficients {
  int64_t nc = 0, ne = 0, nv = 0;
  int cw = 0, vw = 0, tw = 0;
  int pv_flux = PV_TRISK;
  double alpha = 1.0, gravity = 1.0;
  std::vector<int64_t> cell_edges;  // cw x nc
  std::vector<double> divergence, kinetic;
  std::vector<int64_t> edge_cells, edge_vertices;  // 2 x ne
  std::vector<double> edge_height;                 // 2 x ne
  std::vector<double> inverse_dual;                // ne
  std::vector<int64_t> vertex_edges, vertex_cells;  // vw x nv
  std::vector<double> curl, vertex_height;
  std::vector<double> coriolis;  // nv
  std::vector<int64_t> trisk_edges;  // tw x ne
  std::vector<double> trisk;
  std::vector<double> cell_areas, vertex_areas;
  // Gassmann (pv_flux != trisk)
  std::vector<int64_t> g_edges, g_pv_edges;  // 12 x ne
  std::vector<double> g_weights;
  std::vector<double> rhombus;     // 2 x ne
  std::vector<double> g_coriolis;  // ne
  // vertex kinetic energy (alpha != 1)
  std::vector<int64_t> vk_cell_vertices;  // cw x nc
  std::vector<double> vk_kites;           // cw x nc
  std::vector<double> vk_weights;         // vw x nv
  std::vector<double> vk_height;          // 2 x ne
  bool has_gassmann() const { return pv_flux != PV_TRISK; }
  bool has_vertex_ke() const { return alpha != 1.0; }
};
// coriolis(x) = 2 omega x[3] at the vertices and edge points unless explicit values are given.
Coefficients build_coefficients(const Grid& g, int pv_flux, double alpha, double gravity, double omega,
                                const double* coriolis_vertices = nullptr,
                                const double* coriolis_edges = nullptr);

}  // namespace trisk
