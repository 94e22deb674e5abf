// Host-side mesh generation and TRiSK table construction (set-up, runs once per mesh).
// Each function names the reference lines whose algorithm it follows; the loop and
// numbering orders are kept so that cells, edges and vertices get the reference's indices.
#include "mesh.hpp"

#include <algorithm>
#include <numeric>
#include <unordered_map>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace trisk {

// ---------------------------------------------------------------------------------------
// Plex (src/Topology/Plex.jl)

static void invert_cones(Plex& dm) {  // Plex.jl:142-160
  const int64_t np = dm.npoints();
  std::vector<int64_t> counts(np, 0);
  for (int64_t q : dm.cones) counts[q]++;
  dm.support_offsets.assign(np + 1, 0);
  for (int64_t p = 0; p < np; ++p) dm.support_offsets[p + 1] = dm.support_offsets[p] + counts[p];
  dm.supports.assign(dm.cones.size(), 0);
  std::vector<int64_t> fill(dm.support_offsets.begin(), dm.support_offsets.end() - 1);
  for (int64_t p = 0; p < np; ++p)
    for (int64_t k = dm.cone_offsets[p]; k < dm.cone_offsets[p + 1]; ++k) dm.supports[fill[dm.cones[k]]++] = p;
}

Plex plex_from_polygons(const std::vector<std::vector<int64_t>>& polygons, const std::vector<V3>& coordinates) {
  // Plex.jl:49-97 (sphere only: no periodic unwrap on this path)
  Plex dm;
  dm.coordinates = coordinates;
  bool plane = true;
  for (const V3& x : coordinates) plane = plane && x.z == 0.0;
  dm.sphere = !plane;
  const int64_t nc = (int64_t)polygons.size(), nv = (int64_t)coordinates.size();
  std::vector<std::vector<int64_t>> polys(nc);
  for (int64_t c = 0; c < nc; ++c) {  // orient_ccw, Plex.jl:99-103
    const auto& poly = polygons[c];
    const size_t n = poly.size();
    V3 normal{0, 0, 0}, centre{0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
      normal = normal + cross(coordinates[poly[i]], coordinates[poly[(i + 1) % n]]);
      centre = centre + coordinates[poly[i]];
    }
    V3 ref = dm.sphere ? normalize(centre) : V3{0, 0, 1};
    polys[c] = poly;
    if (!(dot(normal, ref) >= 0)) std::reverse(polys[c].begin(), polys[c].end());
  }
  // edges numbered by first appearance as minmax pairs (Plex.jl:58-67)
  std::unordered_map<uint64_t, int64_t> edge_ids;
  edge_ids.reserve(polys.size() * 4);
  std::vector<std::array<int64_t, 2>> edge_vertices;
  edge_vertices.reserve(polys.size() * 3);
  for (const auto& poly : polys) {
    const size_t n = poly.size();
    for (size_t i = 0; i < n; ++i) {
      int64_t a = std::min(poly[i], poly[(i + 1) % n]), b = std::max(poly[i], poly[(i + 1) % n]);
      if (a == b) throw MeshError("degenerate edge at vertex " + std::to_string(a + 1));
      uint64_t key = (uint64_t)a * (uint64_t)nv + (uint64_t)b;
      if (edge_ids.emplace(key, (int64_t)edge_vertices.size()).second) edge_vertices.push_back({a, b});
    }
  }
  const int64_t ne = (int64_t)edge_vertices.size();
  dm.nc = nc;
  dm.ne = ne;
  dm.nv = nv;
  const int64_t np = nc + ne + nv;
  dm.cone_offsets.assign(np + 1, 0);
  for (int64_t c = 0; c < nc; ++c) {
    const auto& poly = polys[c];
    const size_t n = poly.size();
    for (size_t i = 0; i < n; ++i) {
      int64_t a = poly[i], b = poly[(i + 1) % n];
      uint64_t key = (uint64_t)std::min(a, b) * (uint64_t)nv + (uint64_t)std::max(a, b);
      dm.cones.push_back(nc + edge_ids[key]);
      dm.orientations.push_back(a < b ? 0 : -1);
    }
    dm.cone_offsets[c + 1] = (int64_t)dm.cones.size();
  }
  for (int64_t k = 0; k < ne; ++k) {
    dm.cones.push_back(nc + ne + edge_vertices[k][0]);
    dm.cones.push_back(nc + ne + edge_vertices[k][1]);
    dm.orientations.push_back(0);
    dm.orientations.push_back(0);
    dm.cone_offsets[nc + k + 1] = (int64_t)dm.cones.size();
  }
  for (int64_t p = nc + ne + 1; p <= np; ++p) dm.cone_offsets[p] = (int64_t)dm.cones.size();
  invert_cones(dm);
  return dm;
}

std::array<int64_t, 2> Plex::edge_cells(int64_t p) const {  // Plex.jl:210-218
  std::array<int64_t, 2> lr{-1, -1};
  for (int64_t s = 0; s < support_size(p); ++s) {
    int64_t c = support(p)[s];
    for (int64_t k = cone_offsets[c]; k < cone_offsets[c + 1]; ++k)
      if (cones[k] == p) {
        (orientations[k] == 0 ? lr[0] : lr[1]) = c;
        break;
      }
  }
  return lr;
}

std::vector<int64_t> Plex::cell_vertices(int64_t c) const {  // Plex.jl:226-230
  std::vector<int64_t> v(cone_size(c));
  for (int64_t i = 0; i < cone_size(c); ++i) v[i] = cone(cone(c)[i])[cone_orientation(c)[i] == 0 ? 0 : 1];
  return v;
}

std::vector<int64_t> Plex::star(int64_t p) const {  // Plex.jl:251-262
  std::vector<int64_t> st{p}, frontier{p};
  while (!frontier.empty()) {
    std::vector<int64_t> next;
    for (int64_t q : frontier)
      for (int64_t s = 0; s < support_size(q); ++s) {
        int64_t r = support(q)[s];
        if (std::find(st.begin(), st.end(), r) == st.end()) {
          st.push_back(r);
          next.push_back(r);
        }
      }
    frontier.swap(next);
  }
  return st;
}

// ---------------------------------------------------------------------------------------
// Icosahedral mesh and Lloyd's algorithm (src/Grids/Icosahedral.jl)

// Deterministic parallel dot product: fixed chunking, partial sums added in order, so the
// result does not depend on the number of threads.
static double det_dot(const double* a, const double* b, int64_t n) {
  const int64_t chunk = 8192;
  const int64_t nchunks = (n + chunk - 1) / chunk;
  std::vector<double> part(nchunks, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nchunks; ++c) {
    double s = 0.0;
    const int64_t lo = c * chunk, hi = std::min(n, lo + chunk);
    for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
    part[c] = s;
  }
  double s = 0.0;
  for (double p : part) s += p;
  return s;
}

static double lloyd_step(std::vector<V3>& f, std::vector<V3>& centers, const std::vector<V3>& x,
                         const std::vector<std::array<int64_t, 3>>& tris, const std::vector<int64_t>& star_off,
                         const std::vector<int64_t>& star, const std::vector<char>& is_free) {
  // Icosahedral.jl:186-207
  const int64_t nt = (int64_t)tris.size(), n = (int64_t)x.size();
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < nt; ++t) {
    const auto& tr = tris[t];
    centers[t] = normalize(cross(x[tr[1]] - x[tr[0]], x[tr[2]] - x[tr[0]]));
  }
  double residual = 0.0;
#pragma omp parallel for schedule(static) reduction(max : residual)
  for (int64_t v = 0; v < n; ++v) {
    if (!is_free[v]) {
      f[v] = {0, 0, 0};
      continue;
    }
    const int64_t lo = star_off[v], len = star_off[v + 1] - lo;
    V3 m{0, 0, 0};
    for (int64_t k = 0; k < len; ++k) {
      V3 p = centers[star[lo + k]], q = centers[star[lo + (k + 1) % len]];
      V3 nn = cross(p, q);
      double nrm = norm(nn);
      m = m + (std::atan2(nrm, dot(p, q)) / nrm) * nn;
    }
    f[v] = normalize(m) - x[v];
    residual = std::max(residual, norm(f[v]));
  }
  return residual;
}

// Dense solve with partial pivoting (the reference's `\` on a dense matrix is an LU solve).
static void lu_solve(std::vector<double>& A, std::vector<double>& b, int m) {
  std::vector<int> piv(m);
  for (int k = 0; k < m; ++k) {
    int p = k;
    for (int i = k + 1; i < m; ++i)
      if (std::fabs(A[i * m + k]) > std::fabs(A[p * m + k])) p = i;
    if (p != k) {
      for (int j = 0; j < m; ++j) std::swap(A[k * m + j], A[p * m + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < m; ++i) {
      double l = A[i * m + k] / A[k * m + k];
      for (int j = k; j < m; ++j) A[i * m + j] -= l * A[k * m + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = m - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < m; ++j) s -= A[i * m + j] * b[j];
    b[i] = s / A[i * m + i];
  }
}

int lloyd(std::vector<V3>& x, const std::vector<std::array<int64_t, 3>>& tris, int n_fixed, double tolerance,
          int history, int max_iterations) {
  // Icosahedral.jl:126-183
  const int64_t n = (int64_t)x.size(), nt = (int64_t)tris.size();
  std::vector<char> is_free(n, 1);
  for (int i = 0; i < n_fixed && i < n; ++i) is_free[i] = 0;
  std::unordered_map<uint64_t, int64_t> after;  // directed edge (v, b) -> triangle
  after.reserve(nt * 4);
  auto key = [n](int64_t a, int64_t b) { return (uint64_t)a * (uint64_t)n + (uint64_t)b; };
  for (int64_t t = 0; t < nt; ++t) {
    const auto& tr = tris[t];
    after[key(tr[0], tr[1])] = t;
    after[key(tr[1], tr[2])] = t;
    after[key(tr[2], tr[0])] = t;
  }
  std::vector<std::vector<int64_t>> stars(n);
  for (int64_t t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) {
      int64_t v = tris[t][k], w = tris[t][(k + 2) % 3];
      if (!stars[v].empty()) continue;
      stars[v].push_back(t);
      for (;;) {
        int64_t next = after.at(key(v, w));
        if (next == t) break;
        stars[v].push_back(next);
        const auto& tn = tris[next];
        int j = tn[0] == v ? 0 : (tn[1] == v ? 1 : 2);
        w = tn[(j + 2) % 3];
      }
    }
  std::vector<int64_t> star_off(n + 1, 0), star;
  for (int64_t v = 0; v < n; ++v) star_off[v + 1] = star_off[v] + (int64_t)stars[v].size();
  star.reserve(star_off[n]);
  for (auto& s : stars) star.insert(star.end(), s.begin(), s.end());
  stars.clear();
  stars.shrink_to_fit();

  double h = 0.0;
  for (const auto& tr : tris) h += norm(x[tr[1]] - x[tr[0]]);
  h /= (double)nt;

  std::vector<V3> centers(nt), f(n), fold(n, V3{0, 0, 0}), xold(n, V3{0, 0, 0});
  const int64_t N3 = 3 * n;
  std::vector<double> dX(history > 0 ? (size_t)N3 * history : 0), dF(history > 0 ? (size_t)N3 * history : 0);
  std::vector<double> gram((size_t)std::max(history, 1) * std::max(history, 1), 0.0);
  int m = 0;
  auto flat = [](std::vector<V3>& v) { return reinterpret_cast<double*>(v.data()); };
  for (int it = 1; it <= max_iterations; ++it) {
    double residual = lloyd_step(f, centers, x, tris, star_off, star, is_free);
    if (residual < tolerance * h) {
      // Delaunay check, Icosahedral.jl:210-216
      bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok)
      for (int64_t t = 0; t < nt; ++t) {
        const auto& tr = tris[t];
        V3 c = normalize(cross(x[tr[1]] - x[tr[0]], x[tr[2]] - x[tr[0]]));
        const int64_t pairs[3][2] = {{tr[0], tr[1]}, {tr[1], tr[2]}, {tr[2], tr[0]}};
        for (auto& pq : pairs) {
          const auto& opp = tris[after.at(key(pq[1], pq[0]))];
          int64_t o = -1;
          for (int j = 0; j < 3; ++j)
            if (opp[j] != pq[0] && opp[j] != pq[1]) o = opp[j];
          if (!(dot(x[o], c) <= dot(x[tr[0]], c) + 1e-14)) ok = false;
        }
      }
      if (!ok) throw MeshError("Lloyd's algorithm left the triangulation non-Delaunay");
      return it;
    }
    double* xf = flat(x);
    double* ff = flat(f);
    if (history > 0 && it > 1) {
      const int k = (it - 2) % history;  // ring buffer slot, Icosahedral.jl:164
      const double* xo = flat(xold);
      const double* fo = flat(fold);
      double* dx = dX.data() + (size_t)k * N3;
      double* df = dF.data() + (size_t)k * N3;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < N3; ++i) {
        dx[i] = xf[i] - xo[i];
        df[i] = ff[i] - fo[i];
      }
      m = std::min(m + 1, history);
      for (int j = 0; j < m; ++j) {  // only column k changed: refresh its Gram row
        double s = det_dot(df, dF.data() + (size_t)j * N3, N3);
        gram[k * history + j] = s;
        gram[j * history + k] = s;
      }
    }
    xold = x;
    fold = f;
    if (m > 0) {
      // gamma = (A'A + 1e-12 max(diag) I) \ (A'f), Icosahedral.jl:172-175
      std::vector<double> N((size_t)m * m), g(m);
      double dmax = 0.0;
      for (int i = 0; i < m; ++i) dmax = std::max(dmax, gram[i * history + i]);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) N[i * m + j] = gram[i * history + j] + (i == j ? 1e-12 * dmax : 0.0);
      for (int j = 0; j < m; ++j) g[j] = det_dot(dF.data() + (size_t)j * N3, ff, N3);
      lu_solve(N, g, m);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < N3; ++i) {
        double bg = 0.0, ag = 0.0;
        for (int j = 0; j < m; ++j) {
          bg += dX[(size_t)j * N3 + i] * g[j];
          ag += dF[(size_t)j * N3 + i] * g[j];
        }
        xf[i] += ff[i] - (bg + ag);
      }
    } else {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < N3; ++i) xf[i] += ff[i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; ++v) x[v] = normalize(x[v]);
  }
  return max_iterations;
}

int spring_dynamics(std::vector<V3>& x, const std::vector<std::array<int64_t, 2>>& edges, double beta,
                    double mean_length, int n_fixed, double tolerance, int max_iterations) {
  // Icosahedral.jl:78-109 (uniform natural length beta * mean_length)
  const int64_t n = (int64_t)x.size();
  std::vector<char> is_free(n, 1);
  for (int i = 0; i < n_fixed && i < n; ++i) is_free[i] = 0;
  const double d0 = beta * mean_length;
  std::vector<V3> force(n), velocity(n, V3{0, 0, 0});
  const double dt = 0.3, damping = 0.05;
  for (int it = 1; it <= max_iterations; ++it) {
    std::fill(force.begin(), force.end(), V3{0, 0, 0});
    for (const auto& ij : edges) {
      V3 r = x[ij[1]] - x[ij[0]];
      double nr = norm(r);
      V3 f = ((nr - d0) / nr) * r;
      force[ij[0]] = force[ij[0]] + f;
      force[ij[1]] = force[ij[1]] - f;
    }
    double residual = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      if (!is_free[i]) continue;
      V3 f = force[i] - dot(force[i], x[i]) * x[i];
      residual = std::max(residual, norm(f));
      velocity[i] = (1 - damping) * velocity[i] + dt * f;
      velocity[i] = velocity[i] - dot(velocity[i], x[i]) * x[i];
      x[i] = normalize(x[i] + dt * velocity[i]);
    }
    if (residual < tolerance * beta * mean_length) return it;
  }
  return max_iterations;
}

TriangleMesh icosahedral_triangles(int subdivisions, bool centroidal, double spring_beta) {
  // Icosahedral.jl:22-58
  if (subdivisions < 0) throw MeshError("subdivisions must be non-negative");
  const double PHI = (1.0 + std::sqrt(5.0)) / 2.0;
  const V3 raw[12] = {{-1.0, PHI, 0.0}, {1.0, PHI, 0.0},  {-1.0, -PHI, 0.0}, {1.0, -PHI, 0.0},
                      {0.0, -1.0, PHI}, {0.0, 1.0, PHI},  {0.0, -1.0, -PHI}, {0.0, 1.0, -PHI},
                      {PHI, 0.0, -1.0}, {PHI, 0.0, 1.0},  {-PHI, 0.0, -1.0}, {-PHI, 0.0, 1.0}};
  const int base[20][3] = {{1, 12, 6}, {1, 6, 2},  {1, 2, 8},  {1, 8, 11}, {1, 11, 12}, {2, 6, 10}, {6, 12, 5},
                           {12, 11, 3}, {11, 8, 7}, {8, 2, 9},  {4, 10, 5}, {4, 5, 3},   {4, 3, 7},  {4, 7, 9},
                           {4, 9, 10}, {5, 10, 6}, {3, 5, 12}, {7, 3, 11}, {9, 7, 8},   {10, 9, 2}};
  TriangleMesh tm;
  for (const V3& v : raw) tm.x.push_back(normalize(v));
  for (const auto& t : base) tm.triangles.push_back({t[0] - 1, t[1] - 1, t[2] - 1});
  for (int level = 1; level <= subdivisions; ++level) {
    std::unordered_map<uint64_t, int64_t> midpoints;
    midpoints.reserve(tm.triangles.size() * 2);
    auto midpoint = [&](int64_t a, int64_t b) {
      uint64_t key = ((uint64_t)std::min(a, b) << 32) | (uint64_t)std::max(a, b);
      auto it = midpoints.find(key);
      if (it != midpoints.end()) return it->second;
      tm.x.push_back(normalize(tm.x[a] + tm.x[b]));
      int64_t id = (int64_t)tm.x.size() - 1;
      midpoints.emplace(key, id);
      return id;
    };
    std::vector<std::array<int64_t, 3>> refined;
    refined.reserve(tm.triangles.size() * 4);
    for (const auto& t : tm.triangles) {
      int64_t a = t[0], b = t[1], c = t[2];
      int64_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      refined.push_back({a, ab, ca});
      refined.push_back({b, bc, ab});
      refined.push_back({c, ca, bc});
      refined.push_back({ab, bc, ca});
    }
    tm.triangles.swap(refined);
    if (spring_beta > 0) {  // Icosahedral.jl:49-56
      std::vector<std::array<int64_t, 2>> edges;
      std::unordered_map<uint64_t, char> seen;
      seen.reserve(tm.triangles.size() * 2);
      for (const auto& t : tm.triangles)
        for (int k = 0; k < 3; ++k) {
          int64_t a = std::min(t[k], t[(k + 1) % 3]), b = std::max(t[k], t[(k + 1) % 3]);
          if (seen.emplace(((uint64_t)a << 32) | (uint64_t)b, 1).second) edges.push_back({a, b});
        }
      const double pi = 3.14159265358979323846;
      const double mean_length = std::sqrt(4 * pi / (5 * std::sqrt(3.0))) / std::ldexp(1.0, level);
      spring_dynamics(tm.x, edges, spring_beta, mean_length, 12);
      for (const auto& t : tm.triangles)
        if (!(dot(cross(tm.x[t[1]] - tm.x[t[0]], tm.x[t[2]] - tm.x[t[0]]), tm.x[t[0]]) > 0))
          throw MeshError("spring_beta folds the mesh over; take a smaller one");
    }
    if (centroidal) lloyd(tm.x, tm.triangles, 12);
  }
  return tm;
}

static std::vector<std::vector<int64_t>> as_polygons(const std::vector<std::array<int64_t, 3>>& tris) {
  std::vector<std::vector<int64_t>> polys(tris.size());
  for (size_t t = 0; t < tris.size(); ++t) polys[t] = {tris[t][0], tris[t][1], tris[t][2]};
  return polys;
}

Plex create_spherical_mesh(int subdivisions, bool centroidal, double spring_beta) {
  TriangleMesh tm = icosahedral_triangles(subdivisions, centroidal, spring_beta);
  return plex_from_polygons(as_polygons(tm.triangles), tm.x);
}

// FileGrids.jl:28-32
static std::vector<int64_t> sort_ring(const std::vector<int64_t>& ids, const std::vector<V3>& coords, V3 axis) {
  V3 e1 = coords[ids[0]] - axis;
  std::vector<double> angle(ids.size());
  for (size_t k = 0; k < ids.size(); ++k) {
    V3 v = coords[ids[k]] - axis;
    angle[k] = std::atan2(dot(cross(e1, v), axis), dot(e1, v));
  }
  std::vector<size_t> order(ids.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return angle[a] < angle[b]; });
  std::vector<int64_t> out(ids.size());
  for (size_t k = 0; k < ids.size(); ++k) out[k] = ids[order[k]];
  return out;
}

HexMesh create_hexagon_mesh(int subdivisions, bool centroidal, double spring_beta) {
  // Hexagonal.jl:11-17
  TriangleMesh tm = icosahedral_triangles(subdivisions, centroidal, spring_beta);
  Plex primal = plex_from_polygons(as_polygons(tm.triangles), tm.x);
  std::vector<V3> centers(primal.nc);  // circumcenters, CellCenters.jl:37-42
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < primal.nc; ++c) {
    auto v = primal.cell_vertices(c);
    V3 a = primal.coordinates[primal.vertex_index(v[0])], b = primal.coordinates[primal.vertex_index(v[1])],
       d = primal.coordinates[primal.vertex_index(v[2])];
    centers[c] = normalize(cross(b - a, d - a));
  }
  std::vector<std::vector<int64_t>> polys(primal.nv);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t v = 0; v < primal.nv; ++v) {
    std::vector<int64_t> ring;
    for (int64_t p : primal.star(primal.nc + primal.ne + v))
      if (p < primal.nc) ring.push_back(p);
    polys[v] = sort_ring(ring, centers, normalize(primal.coordinates[v]));  // dual_polygons, FileGrids.jl:40-42
  }
  HexMesh hm;
  hm.plex = plex_from_polygons(polys, centers);
  hm.generators = primal.coordinates;
  return hm;
}

HexMesh create_triangle_mesh(int subdivisions, bool centroidal, double spring_beta) {
  // create_spherical_mesh (Icosahedral.jl:22-61) as the cells, their circumcenters as the
  // cell centers (the default of a triangle mesh, CellCenters.jl:37-42)
  TriangleMesh tm = icosahedral_triangles(subdivisions, centroidal, spring_beta);
  HexMesh m;
  m.plex = plex_from_polygons(as_polygons(tm.triangles), tm.x);
  m.generators.resize(m.plex.nc);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < m.plex.nc; ++c) {
    auto v = m.plex.cell_vertices(c);
    V3 a = m.plex.coordinates[m.plex.vertex_index(v[0])], b = m.plex.coordinates[m.plex.vertex_index(v[1])],
       d = m.plex.coordinates[m.plex.vertex_index(v[2])];
    m.generators[c] = normalize(cross(b - a, d - a));
  }
  return m;
}

// ---------------------------------------------------------------------------------------
// Hilbert ordering (src/Topology/Ordering.jl)

uint64_t hilbert_key(uint64_t x0, uint64_t x1, uint64_t x2, int bits) {  // Ordering.jl:10-41
  uint64_t X[3] = {x0, x1, x2};
  const uint64_t M = (uint64_t)1 << (bits - 1);
  for (uint64_t Q = M; Q > 1; Q >>= 1) {
    const uint64_t P = Q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        uint64_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; ++i) X[i] ^= X[i - 1];
  uint64_t t = 0;
  for (uint64_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  uint64_t key = 0;
  for (int b = bits - 1; b >= 0; --b)
    for (int i = 0; i < 3; ++i) key = (key << 1) | ((X[i] >> b) & 1);
  return key;
}

std::vector<int64_t> hilbert_permutation(const Plex& dm, int bits) {  // Ordering.jl:85-92
  std::vector<V3> centroids(dm.nc);
  for (int64_t c = 0; c < dm.nc; ++c) {
    V3 s{0, 0, 0};
    auto vs = dm.cell_vertices(c);
    for (int64_t v : vs) s = s + dm.coordinates[dm.vertex_index(v)];
    centroids[c] = s / (double)vs.size();
  }
  return hilbert_sort(centroids, bits);
}

std::vector<int64_t> hilbert_sort(const std::vector<V3>& centroids, int bits) {
  if (centroids.empty()) return {};
  V3 lo = centroids[0], hi = centroids[0];
  for (const V3& c : centroids) {
    lo = {std::min(lo.x, c.x), std::min(lo.y, c.y), std::min(lo.z, c.z)};
    hi = {std::max(hi.x, c.x), std::max(hi.y, c.y), std::max(hi.z, c.z)};
  }
  const double eps = 2.220446049250313e-16, top = std::ldexp(1.0, bits) - 1;
  V3 scale{top / std::max(hi.x - lo.x, eps), top / std::max(hi.y - lo.y, eps), top / std::max(hi.z - lo.z, eps)};
  const int64_t nc = (int64_t)centroids.size();
  std::vector<uint64_t> keys(nc);
  for (int64_t c = 0; c < nc; ++c) {
    const V3& x = centroids[c];
    keys[c] = hilbert_key((uint64_t)std::nearbyint((x.x - lo.x) * scale.x),
                          (uint64_t)std::nearbyint((x.y - lo.y) * scale.y),
                          (uint64_t)std::nearbyint((x.z - lo.z) * scale.z), bits);
  }
  std::vector<int64_t> perm(nc);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
  return perm;
}

// ---------------------------------------------------------------------------------------
// TRiSK grid (src/FiniteVolumes/TRiSKGrid.jl)

template <class T>
static std::vector<T> padded(const std::vector<std::vector<T>>& columns, T fill, int& width) {
  size_t w = 0;  // TRiSKGrid.jl:67-74
  for (const auto& c : columns) w = std::max(w, c.size());
  width = (int)w;
  std::vector<T> A(w * columns.size(), fill);
  for (size_t j = 0; j < columns.size(); ++j)
    for (size_t k = 0; k < columns[j].size(); ++k) A[j * w + k] = columns[j][k];
  return A;
}

double orthogonality_defect(const Plex& dm, const std::vector<V3>& centers) {  // CellCenters.jl:90-101
  double defect = 0.0;
  for (int64_t e = dm.nc; e < dm.nc + dm.ne; ++e) {
    auto lr = dm.edge_cells(e);
    if (lr[0] < 0 || lr[1] < 0) continue;
    V3 a = dm.coordinates[dm.vertex_index(dm.cone(e)[0])], b = dm.coordinates[dm.vertex_index(dm.cone(e)[1])];
    V3 dual = cross(centers[lr[0]], centers[lr[1]]);
    defect = std::max(defect, std::fabs(dot(normalize(dual), normalize(cross(a, b)))));
  }
  return defect;
}

Grid build_grid(const Plex& dm, const std::vector<V3>& g) {
  // TRiSKGrid.jl:76-162
  if (!dm.sphere) throw MeshError("TRiSKGrid needs a spherical mesh");
  Grid G;
  const int64_t nc = dm.nc, ne = dm.ne, nv = dm.nv;
  if ((int64_t)g.size() != nc) throw MeshError("centers must have one entry per cell");
  G.nc = nc;
  G.ne = ne;
  G.nv = nv;
  G.centers = g;
  G.vertices = dm.coordinates;
  const std::vector<V3>& x = G.vertices;
  G.edge_cells.assign(2 * ne, 0);
  G.edge_vertices.assign(2 * ne, 0);
  G.edge_points.resize(ne);
  G.edge_normals.resize(ne);
  G.primal_lengths.assign(ne, 0.0);
  G.dual_lengths.assign(ne, 0.0);
  G.cell_distances.assign(2 * ne, 0.0);
  bool open_mesh = false;
#pragma omp parallel for schedule(static) reduction(|| : open_mesh)
  for (int64_t j = 0; j < ne; ++j) {
    const int64_t e = nc + j;
    auto lr = dm.edge_cells(e);
    if (lr[0] < 0 || lr[1] < 0) {
      open_mesh = true;
      continue;
    }
    const int64_t cl = lr[0], cr = lr[1];
    const int64_t a = dm.vertex_index(dm.cone(e)[0]), b = dm.vertex_index(dm.cone(e)[1]);
    G.edge_cells[2 * j] = cl;
    G.edge_cells[2 * j + 1] = cr;
    G.edge_vertices[2 * j] = a;
    G.edge_vertices[2 * j + 1] = b;
    V3 m = cross(cross(x[a], x[b]), cross(g[cl], g[cr]));
    m = norm(m) > 1e-14 ? normalize(m) : normalize(x[a] + x[b]);
    if (dot(m, x[a] + x[b]) < 0) m = -m;
    G.edge_points[j] = m;
    V3 n = normalize(cross(x[b], x[a]));
    G.edge_normals[j] = n;
    G.primal_lengths[j] = arc_length(x[a], x[b]);
    G.dual_lengths[j] = arc_length(g[cl], g[cr]);
    G.cell_distances[2 * j] = -jsign(dot(g[cl], n)) * arc_length(g[cl], m);
    G.cell_distances[2 * j + 1] = jsign(dot(g[cr], n)) * arc_length(g[cr], m);
  }
  if (open_mesh) throw MeshError("TRiSKGrid needs a closed mesh");

  std::vector<std::vector<int64_t>> cell_edges(nc), cell_vertices(nc), vertex_cells(nv);
  std::vector<std::vector<double>> cell_signs(nc), cell_kites(nc), vertex_kites(nv);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nc; ++i) {
    const int64_t n = dm.cone_size(i);
    std::vector<int64_t> edges(n), corners = dm.cell_vertices(i);
    for (int64_t k = 0; k < n; ++k) {
      edges[k] = dm.edge_index(dm.cone(i)[k]);
      corners[k] = dm.vertex_index(corners[k]);
    }
    cell_signs[i].resize(n);
    cell_kites[i].resize(n);
    for (int64_t k = 0; k < n; ++k) {
      cell_signs[i][k] = dm.cone_orientation(i)[k] == 0 ? 1.0 : -1.0;  // edge_sign, Plex.jl:201-202
      const int64_t v = corners[k];
      cell_kites[i][k] = signed_triangle_area(g[i], G.edge_points[edges[(k + n - 1) % n]], x[v]) +
                         signed_triangle_area(g[i], x[v], G.edge_points[edges[k]]);
    }
    cell_edges[i] = std::move(edges);
    cell_vertices[i] = std::move(corners);
  }
  for (int64_t i = 0; i < nc; ++i)
    for (size_t k = 0; k < cell_vertices[i].size(); ++k) {
      vertex_cells[cell_vertices[i][k]].push_back(i);
      vertex_kites[cell_vertices[i][k]].push_back(cell_kites[i][k]);
    }
  G.cell_areas.assign(nc, 0.0);
  G.vertex_areas.assign(nv, 0.0);
  for (int64_t i = 0; i < nc; ++i) {
    double s = 0.0;
    for (double kk : cell_kites[i]) s += kk;
    G.cell_areas[i] = s;
  }
  for (int64_t v = 0; v < nv; ++v) {
    double s = 0.0;
    for (double kk : vertex_kites[v]) s += kk;
    G.vertex_areas[v] = s;
  }
  std::vector<std::vector<int64_t>> vertex_edges(nv);
  std::vector<std::vector<double>> vertex_signs(nv);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nv; ++v) {
    const int64_t p = nc + ne + v;
    for (int64_t s = 0; s < dm.support_size(p); ++s) {
      int64_t e = dm.edge_index(dm.support(p)[s]);
      vertex_edges[v].push_back(e);
      vertex_signs[v].push_back(jsign(dot(G.edge_normals[e], cross(x[v], G.edge_points[e]))));
    }
  }
  // TRiSK weights: walk counter-clockwise around both cells of e (TRiSKGrid.jl:141-155)
  std::vector<std::vector<int64_t>> trisk_edges(ne);
  std::vector<std::vector<double>> trisk_weights(ne);
  for (int64_t i = 0; i < nc; ++i) {
    const auto& edges = cell_edges[i];
    const auto& signs = cell_signs[i];
    const int64_t n = (int64_t)edges.size();
    std::vector<double> R(n);
    for (int64_t k = 0; k < n; ++k) R[k] = cell_kites[i][k] / G.cell_areas[i];
    for (int64_t k = 0; k < n; ++k) {
      const int64_t e = edges[k];
      double S = 0.0;
      for (int64_t s = 1; s <= n - 1; ++s) {
        const int64_t kp = (k + s) % n;
        S += R[kp];
        trisk_edges[e].push_back(edges[kp]);
        trisk_weights[e].push_back(signs[k] * signs[kp] * (0.5 - S));
      }
    }
  }
  G.cell_edges = padded(cell_edges, (int64_t)0, G.cw);
  G.cell_signs = padded(cell_signs, 0.0, G.cw);
  G.cell_vertices = padded(cell_vertices, (int64_t)0, G.cw);
  G.cell_kites = padded(cell_kites, 0.0, G.cw);
  G.vertex_edges = padded(vertex_edges, (int64_t)0, G.vw);
  G.vertex_signs = padded(vertex_signs, 0.0, G.vw);
  int vw2 = 0;
  G.vertex_cells = padded(vertex_cells, (int64_t)0, vw2);
  G.vertex_kites = padded(vertex_kites, 0.0, vw2);
  if (vw2 != G.vw) throw MeshError("vertex tables of different widths: not a Voronoi mesh");
  G.trisk_edges = padded(trisk_edges, (int64_t)0, G.tw);
  G.trisk_weights = padded(trisk_weights, 0.0, G.tw);
  return G;
}

void vertex_edge_areas(const Grid& g, std::vector<double>& by_vertex, std::vector<double>& by_edge) {
  // TRiSKGrid.jl:179-191
  auto area = [&](int64_t e, int64_t v) {
    const int64_t left = g.edge_cells[2 * e];
    int n = 0;
    for (int k = 0; k < g.cw; ++k) n += g.cell_signs[left * g.cw + k] != 0.0;
    int j = -1;
    for (int k = 0; k < n; ++k)
      if (g.cell_edges[left * g.cw + k] == e) {
        j = k;
        break;
      }
    if (j < 0) throw MeshError("edge not in its left cell");
    const double orientation = g.cell_vertices[left * g.cw + (j + 1) % n] == v ? 1.0 : -1.0;
    return orientation * signed_triangle_area(g.centers[left], g.centers[g.edge_cells[2 * e + 1]], g.vertices[v]);
  };
  by_vertex.assign((size_t)g.vw * g.nv, 0.0);
  by_edge.assign((size_t)2 * g.ne, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < g.nv; ++v)
    for (int k = 0; k < g.vw; ++k)
      by_vertex[v * g.vw + k] = g.vertex_signs[v * g.vw + k] == 0.0 ? 0.0 : area(g.vertex_edges[v * g.vw + k], v);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < g.ne; ++e)
    for (int s = 0; s < 2; ++s) by_edge[2 * e + s] = area(e, g.edge_vertices[2 * e + s]);
}

void gassmann_coefficients(const Grid& g, std::vector<int64_t>& edges, std::vector<int64_t>& pv_edges,
                           std::vector<double>& weights) {
  // TRiSKGrid.jl:214-251
  const int64_t ne = g.ne;
  const auto& l = g.primal_lengths;
  const auto& d = g.dual_lengths;
  const auto& n = g.edge_normals;
  const auto& A = g.vertex_areas;
  edges.assign((size_t)12 * ne, 0);
  pv_edges.assign((size_t)12 * ne, 0);
  weights.assign((size_t)12 * ne, 0.0);
  auto to_vertex = [&](int64_t e, int64_t v) { return arc_length(g.edge_points[e], g.vertices[v]); };
  auto rhombus = [&](int64_t e) { return A[g.edge_vertices[2 * e]] + A[g.edge_vertices[2 * e + 1]]; };
  auto other = [&](int64_t e, int64_t v) {
    return g.edge_vertices[2 * e] == v ? g.edge_vertices[2 * e + 1] : g.edge_vertices[2 * e];
  };
  auto edges_of = [&](int64_t v) {
    std::vector<int64_t> out;
    for (int k = 0; k < g.vw; ++k)
      if (g.vertex_signs[v * g.vw + k] != 0.0) out.push_back(g.vertex_edges[v * g.vw + k]);
    return out;
  };
  bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
  for (int64_t e = 0; e < ne; ++e) {
    auto metric = [&](int64_t f) { return dot(n[f], cross(normalize(g.edge_points[e] + g.edge_points[f]), n[e])); };
    const double area = l[e] * d[e];
    int k = 0;
    for (int s = 0; s < 2; ++s) {
      const int64_t v = g.edge_vertices[2 * e + s];
      std::vector<int64_t> inner;
      for (int64_t f : edges_of(v))
        if (f != e) inner.push_back(f);
      if (inner.size() != 2) {
        bad = true;
        break;
      }
      const double a = to_vertex(e, v) * d[e] / area;
      for (int j = 0; j < 2; ++j) {
        const int64_t f = inner[j], third = inner[1 - j];
        const double b = to_vertex(f, v) * d[f];
        edges[12 * e + k] = f;
        pv_edges[12 * e + k] = third;
        weights[12 * e + k] =
            metric(f) * (-a * b / A[v] + 2.0 / 3.0 * (a * l[f] * d[f] / rhombus(f) + b / rhombus(e) +
                                                     a * b / rhombus(third)));
        ++k;
        const int64_t w = other(f, v);
        for (int64_t o : edges_of(w)) {
          if (o == f) continue;
          if (k >= 12) {
            bad = true;
            break;
          }
          edges[12 * e + k] = o;
          pv_edges[12 * e + k] = f;
          weights[12 * e + k] = 2.0 / 3.0 * metric(o) * a * to_vertex(o, w) * d[o] / rhombus(f);
          ++k;
        }
      }
    }
  }
  if (bad) throw MeshError("Gassmann's reconstruction needs three edges per vertex");
}

Coefficients build_coefficients(const Grid& g, int pv_flux, double alpha, double gravity, double omega,
                                const double* coriolis_vertices, const double* coriolis_edges) {
  // TRiSKShallowWater.jl:94-168 with the serial distribution (identity local numbering)
  if (pv_flux < PV_TRISK || pv_flux > PV_GASSMANN_MEAN)
    throw MeshError("pv_flux must be :trisk, :gassmann or :gassmann_mean");
  Coefficients C;
  const int64_t nc = g.nc, ne = g.ne, nv = g.nv;
  C.nc = nc;
  C.ne = ne;
  C.nv = nv;
  C.cw = g.cw;
  C.vw = g.vw;
  C.tw = g.tw;
  C.pv_flux = pv_flux;
  C.alpha = alpha;
  C.gravity = gravity;
  const auto& l = g.primal_lengths;
  const auto& d = g.dual_lengths;
  C.cell_edges = g.cell_edges;
  C.divergence.assign((size_t)g.cw * nc, 0.0);
  C.kinetic.assign((size_t)g.cw * nc, 0.0);
  for (int64_t i = 0; i < nc; ++i)
    for (int k = 0; k < g.cw; ++k) {
      const int64_t e = g.cell_edges[i * g.cw + k];
      const double s = g.cell_signs[i * g.cw + k];
      if (s == 0.0) continue;
      const int side = g.edge_cells[2 * e] == i ? 0 : 1;
      C.divergence[i * g.cw + k] = s * l[e] / g.cell_areas[i];
      C.kinetic[i * g.cw + k] = alpha * l[e] * g.cell_distances[2 * e + side] / (2 * g.cell_areas[i]);
    }
  C.vertex_edges = g.vertex_edges;
  C.vertex_cells = g.vertex_cells;
  C.curl.resize((size_t)g.vw * nv);
  C.vertex_height.resize((size_t)g.vw * nv);
  for (int64_t v = 0; v < nv; ++v)
    for (int k = 0; k < g.vw; ++k) {
      C.curl[v * g.vw + k] = g.vertex_signs[v * g.vw + k] * d[g.vertex_edges[v * g.vw + k]] / g.vertex_areas[v];
      C.vertex_height[v * g.vw + k] = g.vertex_kites[v * g.vw + k] / g.vertex_areas[v];
    }
  C.trisk_edges = g.trisk_edges;
  C.trisk.resize((size_t)g.tw * ne);
  for (int64_t e = 0; e < ne; ++e)
    for (int k = 0; k < g.tw; ++k)
      C.trisk[e * g.tw + k] = g.trisk_weights[e * g.tw + k] * l[g.trisk_edges[e * g.tw + k]] / d[e];
  C.edge_cells = g.edge_cells;
  C.edge_vertices = g.edge_vertices;
  C.edge_height.resize((size_t)2 * ne);
  C.rhombus.resize((size_t)2 * ne);
  C.inverse_dual.resize(ne);
  for (int64_t e = 0; e < ne; ++e) {
    for (int s = 0; s < 2; ++s) C.edge_height[2 * e + s] = alpha * g.cell_distances[2 * e + s] / d[e];
    const double a1 = g.vertex_areas[g.edge_vertices[2 * e]], a2 = g.vertex_areas[g.edge_vertices[2 * e + 1]];
    const double sum = a1 + a2;
    C.rhombus[2 * e] = a1 / sum;
    C.rhombus[2 * e + 1] = a2 / sum;
    C.inverse_dual[e] = 1 / d[e];
  }
  C.coriolis.resize(nv);
  for (int64_t v = 0; v < nv; ++v)
    C.coriolis[v] = coriolis_vertices ? coriolis_vertices[v] : 2 * omega * g.vertices[v].z;
  C.cell_areas = g.cell_areas;
  C.vertex_areas = g.vertex_areas;
  if (pv_flux != PV_TRISK) {
    gassmann_coefficients(g, C.g_edges, C.g_pv_edges, C.g_weights);
    C.g_coriolis.resize(ne);
    for (int64_t e = 0; e < ne; ++e)
      C.g_coriolis[e] = coriolis_edges ? coriolis_edges[e] : 2 * omega * g.edge_points[e].z;
  } else {
    C.rhombus.clear();
  }
  if (alpha != 1.0) {
    std::vector<double> by_vertex, by_edge;
    vertex_edge_areas(g, by_vertex, by_edge);
    C.vk_cell_vertices = g.cell_vertices;
    C.vk_kites.resize((size_t)g.cw * nc);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < g.cw; ++k)
        C.vk_kites[i * g.cw + k] = (1 - alpha) * g.cell_kites[i * g.cw + k] / g.cell_areas[i];
    C.vk_weights.resize((size_t)g.vw * nv);
    for (int64_t v = 0; v < nv; ++v)
      for (int k = 0; k < g.vw; ++k) C.vk_weights[v * g.vw + k] = by_vertex[v * g.vw + k] / g.vertex_areas[v];
    C.vk_height.resize((size_t)2 * ne);
    for (int64_t e = 0; e < ne; ++e)
      for (int s = 0; s < 2; ++s) C.vk_height[2 * e + s] = (1 - alpha) * 2 * by_edge[2 * e + s] / (l[e] * d[e]);
  }
  return C;
}

}  // namespace trisk
