/*
 * trisk_b200.h - C ABI of libtrisk_b200.so, the B200 (sm_100a) implementation of the
 * TRiSK C-grid shallow-water hot path of dmplex.jl.
 *
 * In dmplex.jl the path sits behind Julia generic functions, not an FFI:
 *   tendency!(dy, y, m::TRiSKShallowWater)          src/FiniteVolumes/TRiSKShallowWater.jl:379
 *   rk4_step!(y, dt, tendency!, cache, model)       src/TimeSteppers/RungeKutta.jl:18
 * The entry points below are what a Julia `ccall` shim binds in their place: a model type
 * whose tendency! and rk4_step! methods call trisk_tendency and trisk_rk4_step. Conventions
 * shared by every entry point:
 *   - State y = [u_1..u_ne; h_1..h_nc] in file (Plex) numbering, FP64, exactly the
 *     reference's layout (TRiSKShallowWater.jl:172-174).
 *   - Tables are passed as Julia holds them: column-major [k, entity] (k fastest),
 *     Int64 indices 1-based, padded entries index 1 / weight 0.
 *   - Pointers to state may be host or device memory; the library tells them apart.
 *   - Every function returns a status (TRISK_OK = 0); trisk_last_error() gives the
 *     message of the last failure on the calling thread. No C++ exception crosses the ABI.
 *   - A model is not re-entrant (like the reference model, whose work vectors the tendency
 *     mutates): calls on one model must be serialized. Each model owns one CUDA stream.
 */
#ifndef TRISK_B200_H
#define TRISK_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------- */
enum {
  TRISK_OK = 0,
  TRISK_ERR_ARGUMENT = 1,    /* bad argument (the reference raises ArgumentError) */
  TRISK_ERR_TABLE = 2,       /* a neighbour table fails the upload bounds check */
  TRISK_ERR_CUDA = 3,        /* a CUDA call failed, or no GPU */
  TRISK_ERR_NONFINITE = 4,   /* the state became non-finite during the call */
  TRISK_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  TRISK_ERR_UNSUPPORTED = 6, /* valid input the library does not handle */
  TRISK_ERR_MESH = 7         /* mesh generation or grid construction failed */
};
enum { TRISK_PV_TRISK = 0, TRISK_PV_GASSMANN = 1, TRISK_PV_GASSMANN_MEAN = 2 };

/* Copies the last error message of this thread into buf (always NUL-terminated);
 * returns its full length. */
size_t trisk_last_error(char* buf, size_t len);
int32_t trisk_abi_version(void);
/* sizeof of the structs below, so a binding can check its layout */
int32_t trisk_struct_size(int32_t which); /* 0 TriskGrid, 1 TriskCoefficients, 2 TriskConfig, 3 TriskPlex,
                                          4 TriskIconTables, 5 TriskMpasTables, 6 TriskMpasFields,
                                          7 TriskHalo */

/* ---- mesh generation (set-up, host) ------------------------------------------------
 * Replaces create_hexagon_mesh(n; centroidal)   src/Grids/Hexagonal.jl:11-17
 * (with create_spherical_mesh + lloyd!           src/Grids/Icosahedral.jl:22-61,126-183)
 * and TRiSKGrid(dm; centers)                     src/FiniteVolumes/TRiSKGrid.jl:76-162,
 * with centers = the icosahedral generators as the reference's examples pass them
 * (examples/trisk_shallow_water.jl:50-52). */
typedef struct TriskMesh TriskMesh;

typedef struct { /* Plex (src/Topology/Plex.jl:23-34), 1-based point numbers */
  int64_t nc, ne, nv, ncones;
  const int64_t* cone_offsets;      /* nc+ne+nv+1, 1-based offsets into cones */
  const int64_t* cones;             /* ncones */
  const int64_t* cone_orientations; /* ncones: 0 or -1 */
  const int64_t* support_offsets;   /* nc+ne+nv+1 */
  const int64_t* supports;          /* ncones */
  const double* coordinates;        /* 3 x nv */
} TriskPlex;

typedef struct { /* TRiSKGrid (src/FiniteVolumes/TRiSKGrid.jl:37-60) */
  int64_t nc, ne, nv;
  int32_t cw, vw, tw, pad_;
  const double* centers;      /* 3 x nc */
  const double* vertices;     /* 3 x nv */
  const double* edge_points;  /* 3 x ne */
  const double* edge_normals; /* 3 x ne */
  const double* primal_lengths, *dual_lengths; /* ne */
  const int64_t* edge_cells;     /* 2 x ne */
  const int64_t* edge_vertices;  /* 2 x ne */
  const double* cell_distances;  /* 2 x ne */
  const double* cell_areas;      /* nc */
  const double* vertex_areas;    /* nv */
  const int64_t* cell_edges;     /* cw x nc */
  const double* cell_signs;
  const int64_t* cell_vertices;
  const double* cell_kites;
  const int64_t* vertex_edges;   /* vw x nv */
  const double* vertex_signs;
  const int64_t* vertex_cells;
  const double* vertex_kites;
  const int64_t* trisk_edges;    /* tw x ne */
  const double* trisk_weights;
} TriskGrid;

/* spring_beta > 0 relaxes every bisection level by spring dynamics (Icosahedral.jl:49-56,
 * 78-109), 0 leaves it off; centroidal != 0 runs Lloyd's algorithm after every level. */
int trisk_mesh_create_hexagon(int32_t subdivisions, int32_t centroidal, double spring_beta, TriskMesh** out);
/* create_spherical_mesh(subdivisions; centroidal) (Icosahedral.jl:22-61) as a mesh whose
 * cells are the triangles, centers their circumcenters (CellCenters.jl:37-42): the grid of
 * ICONShallowWater (ICONShallowWater.jl:1-48). The other trisk_mesh_* calls apply. */
int trisk_mesh_create_triangles(int32_t subdivisions, int32_t centroidal, double spring_beta, TriskMesh** out);
/* plex_from_polygons(polygons, coordinates) (src/Topology/Plex.jl:49-97), the constructor the
 * grid-file readers use (src/Grids/FileGrids.jl:52-107). Polygon c (c = 1..npolygons) lists
 * the 1-based vertices vertices[offsets[c-1]-1 .. offsets[c]-2] (offsets[0] = 1, CSR like the
 * Plex cones); polygons are turned counter-clockwise and edges numbered by first appearance
 * as in the reference. coordinates: nv points (3 x nv). centers: nc cell centers for the TRiSK
 * grid (3 x nc), or NULL for the normalized vertex means; trisk_mesh_set_centers replaces
 * them. Errors: TRISK_ERR_ARGUMENT for an index outside 1..nv or a polygon of fewer than
 * three vertices, TRISK_ERR_MESH for a degenerate edge. */
int trisk_mesh_from_polygons(const int64_t* offsets, const int64_t* vertices, int64_t npolygons,
                             const double* coordinates, int64_t nv, const double* centers, TriskMesh** out);
/* Replace the cell centers (3 x nc) that trisk_mesh_grid builds the TRiSK tables from
 * (TRiSKGrid(dm; centers), TRiSKGrid.jl:76-78); the tables are rebuilt on the next call. */
int trisk_mesh_set_centers(TriskMesh* mesh, const double* centers);
void trisk_mesh_destroy(TriskMesh* mesh);
/* The hexagon Plex (views into mesh-owned memory, valid until trisk_mesh_destroy). */
int trisk_mesh_plex(TriskMesh* mesh, TriskPlex* out);
/* The icosahedral generators (3 x nc), the `centers` of the reference's examples. */
int trisk_mesh_generators(TriskMesh* mesh, const double** out);
/* TRiSKGrid(dm; centers=generators) (views into mesh-owned memory). */
int trisk_mesh_grid(TriskMesh* mesh, TriskGrid* out);
/* create_spherical_mesh(n; spring_beta, centroidal) before plex_from_polygons
 * (Icosahedral.jl:22-58): x gets 3 x (10*4^n+2) coordinates, triangles 3 x 20*4^n 1-based
 * vertex indices. */
int trisk_icosahedral_mesh(int32_t subdivisions, int32_t centroidal, double spring_beta, double* x,
                           int64_t* triangles);
/* lloyd!(x, triangles; fixed=1:n_fixed, history) (Icosahedral.jl:126-183), in place on
 * 3 x n coordinates; iterations gets the count. */
int trisk_lloyd(double* x, int64_t n, const int64_t* triangles, int64_t nt, int32_t n_fixed, int32_t history,
                int32_t* iterations);
/* hilbert_permutation(dm) (src/Topology/Ordering.jl:85-92), 1-based, nc entries. */
int trisk_mesh_hilbert_permutation(TriskMesh* mesh, int64_t* perm);
/* orthogonality_defect(dm, centers) (src/Grids/CellCenters.jl:90-101). */
int trisk_mesh_orthogonality_defect(TriskMesh* mesh, double* out);
/* vertex_edge_areas(g) (TRiSKGrid.jl:179-191): by_vertex vw x nv, by_edge 2 x ne. */
int trisk_mesh_vertex_edge_areas(TriskMesh* mesh, double* by_vertex, double* by_edge);
/* gassmann_coefficients(g) (TRiSKGrid.jl:214-251): 12 x ne each, 1-based indices. */
int trisk_mesh_gassmann(TriskMesh* mesh, int64_t* edges, int64_t* pv_edges, double* weights);

/* ---- model ---------------------------------------------------------------------------
 * Replaces TRiSKShallowWater(grid; gravity, coriolis, pv_flux, kinetic_energy, backend)
 * src/FiniteVolumes/TRiSKShallowWater.jl:94-170 (serial distribution). */
typedef struct {
  int32_t pv_flux;  /* TRISK_PV_*; :trisk, :gassmann, :gassmann_mean */
  int32_t reorder;  /* 1: renumber cells along the Hilbert curve, edges and vertices by
                       first appearance, inside the library (results stay in file numbering) */
  double alpha;     /* kinetic_energy: 1 :cell, 0 :vertex, 3/8 :mixed, any real */
  double gravity;   /* the reference's `gravity` (1 on the unit sphere) */
  double omega;     /* coriolis(x) = 2 omega x[3] when the arrays below are NULL */
  const double* coriolis_vertices; /* nv values of coriolis(x_v), or NULL */
  const double* coriolis_edges;    /* ne values of coriolis(edge point), or NULL */
  const double* cell_positions;    /* 3 x nc points for the Hilbert order (from-coefficient
                                      creation only; NULL: keep the cell numbering) */
  int32_t device;   /* CUDA device ordinal */
  int32_t use_graph;/* 1: capture the RK4 step as a CUDA graph (default) */
  int32_t use_pdl;  /* 1: programmatic dependent launch between the phases (default) */
  int32_t block;    /* threads per block of the phase kernels (0: 256) */
} TriskConfig;

/* The premultiplied tables a TRiSKShallowWater model holds (TRiSKShallowWater.jl:67-92),
 * 1-based Int64, column-major. Gassmann members NULL for :trisk; vk_* NULL for alpha == 1. */
typedef struct {
  int64_t nc, ne, nv;
  int32_t cw, vw, tw;
  int32_t pv_flux;
  double alpha;
  double gravity;
  const int64_t* cell_edges;   const double* divergence;   const double* kinetic;
  const int64_t* edge_cells;   const double* edge_height;
  const int64_t* edge_vertices; const double* inverse_dual;
  const int64_t* vertex_edges; const double* curl;
  const int64_t* vertex_cells; const double* vertex_height; const double* coriolis;
  const int64_t* trisk_edges;  const double* trisk;
  const double* cell_areas;    const double* vertex_areas;
  const int64_t* g_edges;      const int64_t* g_pv_edges;   const double* g_weights;
  const double* rhombus;       const double* g_coriolis;
  const int64_t* vk_cell_vertices; const double* vk_kites;
  const double* vk_weights;    const double* vk_height;
} TriskCoefficients;

typedef struct TriskModel TriskModel;
typedef struct TriskTables TriskTables;
typedef struct TriskClosure TriskClosure; /* the closure network, declared below */

/* Host-only restatement of the constructor's table arithmetic (TRiSKShallowWater.jl:103-158
 * with gassmann_coefficients and vertex_edge_areas): the premultiplied tables of a model,
 * built on the CPU without a device. The view stays valid until trisk_tables_destroy. */
int trisk_tables_create(const TriskGrid* grid, const TriskConfig* config, TriskTables** out);
int trisk_tables_view(TriskTables* tables, TriskCoefficients* out);
void trisk_tables_destroy(TriskTables* tables);

/* Builds the coefficients from TRiSKGrid arrays (as the reference's constructor does) and
 * uploads them once as int32/FP64 device tables. */
int trisk_model_create(const TriskGrid* grid, const TriskConfig* config, TriskModel** out);
/* Uploads the coefficient arrays of an existing TRiSKShallowWater model unchanged. */
int trisk_model_create_from_coefficients(const TriskCoefficients* coefficients, const TriskConfig* config,
                                         TriskModel** out);
void trisk_model_destroy(TriskModel* model);
/* The model's coefficient tables in the reference layout (host views, file numbering). */
int trisk_model_coefficients(TriskModel* model, TriskCoefficients* out);
/* nc, ne, nv; state length = ne + nc */
int trisk_model_sizes(TriskModel* model, int64_t sizes[3]);

/* tendency!(dy, y, m)   TRiSKShallowWater.jl:379-394. Synchronous. */
int trisk_tendency(TriskModel* model, const double* y, double* dy);
/* nsteps x rk4_step!(y, dt, tendency!, cache, m)   RungeKutta.jl:18-29, in place.
 * Synchronous; returns TRISK_ERR_NONFINITE if y became non-finite. */
int trisk_rk4_step(TriskModel* model, double* y, double dt, int64_t nsteps);
/* Same, asynchronous on the model's stream; y must be device memory. */
int trisk_rk4_step_async(TriskModel* model, double* y, double dt, int64_t nsteps);
/* Waits for the model's stream; reports a non-finite state seen since the last check. */
int trisk_synchronize(TriskModel* model);
/* total_mass, total_energy, potential_enstrophy   TRiSKShallowWater.jl:397-419. */
int trisk_diagnostics(TriskModel* model, const double* y, double* mass, double* energy, double* enstrophy);
/* relative_vorticity(m, y)   TRiSKShallowWater.jl:422-426 (nv values, file numbering). */
int trisk_relative_vorticity(TriskModel* model, const double* y, double* zeta);
/* The model's CUDA stream (cudaStream_t), for event timing by the caller. */
int trisk_model_stream(TriskModel* model, void** stream);
/* Kernel launches issued by this model so far (graph replays count their kernels). */
int64_t trisk_launch_count(TriskModel* model);
/* Algorithmic bytes per launch of the three phase kernels (vertex, flux, tend) and per
 * RK4 step (4 (T + 2N) + 15N with the model's tables T and state size N). */
int trisk_model_bytes(TriskModel* model, double out[4]);
/* The kernels' PV mode (3 = Gassmann with PV edges derived from the flux edges, verified
 * at upload), the threads per block of the three phases, and the bytes per k_tend launch
 * the derived PV edges save. No reference counterpart (implementation detail). */
int trisk_model_info(TriskModel* model, int32_t* pv_mode, int32_t block[3], double* derived_saving);
/* Autotuner (no reference counterpart): times `steps` RK4 steps of the device state y (left
 * unchanged) for every combination of the phase block sizes {64, 128, 256}, then L2-resident
 * table prefixes of 8..64 MB (trisk_model_set_l2_residency, no window) with the best blocks,
 * then the blocks again with the best prefix, then (for meshes whose tables and vectors fit
 * half the L2) the one-launch step of trisk_model_set_persistent, and keeps the fastest in
 * the model; best_ms gets its time per step. */
int trisk_autotune(TriskModel* model, double* y_device, double dt, int32_t steps, double* best_ms);
/* Sets the threads per block of the three phases (vertex, flux, tend), each a multiple of 32
 * in [64, 256], as an autotuner result found earlier (no reference counterpart). */
int trisk_model_set_block(TriskModel* model, const int32_t block[3]);
/* The one-launch RK4 step (no reference counterpart): on != 0 runs the RK4 steps of
 * trisk_rk4_step(_async) as one cooperative launch whose blocks do the twelve phases of every
 * step in turn, separated by a grid-wide barrier, instead of twelve launches per step (the
 * same numbers bit for bit); for meshes that stay in L2, where launch latency dominates. A
 * barrier wait that gives up (after a second) ends the launch; the next synchronizing call
 * returns TRISK_ERR_TIMEOUT. TRISK_ERR_UNSUPPORTED without cooperative launch. */
int trisk_model_set_persistent(TriskModel* model, int32_t on);
int trisk_model_get_persistent(TriskModel* model, int32_t* on);
/* L2 residency of the tables (no reference counterpart). The first `bytes` of the model's
 * packed table block (the tendency phase's tables first, then the flux phase's, then the
 * vertex phase's) are loaded with an L2 evict-last policy, so they stay in L2 from one
 * phase launch and one RK4 stage to the next instead of streaming from HBM; with window = 1
 * also as a persisting access-policy window of that size on every launch (this sets the
 * context's persisting-L2 limit, at most cudaDevAttrMaxPersistingL2CacheSize). bytes = 0:
 * all tables stream (the default). Results are unchanged. */
int trisk_model_set_l2_residency(TriskModel* model, int64_t bytes, int32_t window);
int trisk_model_get_l2_residency(TriskModel* model, int64_t* bytes, int32_t* window);
/* L2 size, largest persisting-L2 set-aside, largest access-policy window and the current
 * persisting-L2 limit of a device, in bytes. */
int trisk_l2_info(int32_t device, int64_t info[4]);
/* Runs nsteps RK4 steps on the device-resident state with a CUDA event pair around every
 * kernel launch and returns the mean duration in ms of each phase kernel in ms[3]. */
int trisk_profile_phases(TriskModel* model, double* y_device, double dt, int64_t nsteps, double ms[3]);

/* ---- ICON triangle shallow water (ICONShallowWater.jl) -----------------------------
 * Replaces ICONShallowWater(grid; gravity, coriolis, rbf_scale, divergence_damping,
 * kinetic_gradient) (src/FiniteVolumes/ICONShallowWater.jl:96-147): the premultiplied
 * coefficients of that constructor, 1-based Int64 and (entity, k) ordered as Julia holds
 * them, for a grid of triangles (3 edges per cell, at most 6 edges per vertex, 4-edge RBF
 * stencils). divergence_damping: nu_4 per edge, or NULL for none. */
typedef struct {
  int64_t nc, ne, nv;
  int32_t vw;
  double gravity;
  const int64_t* cell_edges;       /* nc x 3 */
  const double* divergence;        /* nc x 3: n_{e,i} l_e / A_i */
  const double* bilinear;          /* nc x 3: e_bln_c_s */
  const int64_t* edge_cells;       /* ne x 2 */
  const int64_t* edge_vertices;    /* ne x 2 */
  const double* edge_height;       /* ne x 2: c_lin_e */
  const double* gradient;          /* ne x 2: coeff_gradekin */
  const double* inverse_dual;      /* ne */
  const int64_t* rbf_edges;        /* ne x 4 */
  const double* rbf;               /* ne x 4 */
  const double* edge_coriolis;     /* ne */
  const int64_t* vertex_edges;     /* nv x vw */
  const double* curl;              /* nv x vw */
  const double* cell_areas;        /* nc (diagnostics on the caller's side) */
  const double* divergence_damping;/* ne or NULL */
} TriskIconTables;
typedef struct TriskIconModel TriskIconModel;
int trisk_icon_create(const TriskIconTables* tables, int32_t device, TriskIconModel** out);
void trisk_icon_destroy(TriskIconModel* model);
/* tendency!(dy, y, m) (ICONShallowWater.jl:191-208): host or device pointers. */
int trisk_icon_tendency(TriskIconModel* model, const double* y, double* dy);
/* rk4_step!(y, dt, tendency!, cache, m) (RungeKutta.jl:18-29), nsteps times, in place. */
int trisk_icon_rk4_step(TriskIconModel* model, double* y, double dt, int64_t nsteps);
int64_t trisk_icon_launch_count(TriskIconModel* model);

/* ---- 3-D MPAS-Gassmann horizontal operators -----------------------------------------
 * Replaces slow_tendencies!(m, ys, pressure) of MPASGassmannNonhydrostatic for flat ground
 * (src/Nonhydrostatic/MPAS/Gassmann/Stepping.jl:22-56): the kernels diagnose,
 * vertex_kinetic, cell_from_vertex, w_kinetic, eta, edge_density, w_tendency_vi or
 * w_tendency, vertex_pv, edge_pv (src/Nonhydrostatic/MPAS/Operators.jl:6-133) and
 * vn_tendency (Gassmann/Tendencies.jl:38-75, oro = 0). The tables are the model's arrays
 * (MPASGassmannNonhydrostatic.jl:131-150, built at :152-307): 1-based Int64, (entity, k)
 * ordered as Julia holds them, except the TRiSK tables, which the reference keeps
 * edge-first: trisk[e + ne*j], trisk_index[e + ne*(j + nt*c)] (Int32, c = 0..2: the edge
 * e' and the two edges of its PV). Vertical metrics per column: dz_cells[k*nc + i] (Julia's
 * m.dz), dzh_cells and wlow (nlev + 1 interfaces), dz_edges and dzh_edges (m.metric.dz,
 * .dzh). vertex_kinetic = 0 leaves the vk_* tables unread (m.vertex_kinetic === nothing). */
typedef struct {
  int64_t nc, ne, nv, nlev;
  int32_t cw, vw, nt;          /* widths: cell tables, vertex tables, TRiSK neighbours */
  int32_t vertex_kinetic;      /* 1: vk_* tables given */
  int32_t iap_pv;              /* edge PV: 1 the rhombus PV (m.iap_pv), 0 the vertex mean */
  int32_t vertical;            /* 0 advective, 1 vector invariant, 2 ICON-IAP mass fluxes */
  int32_t five_band;           /* 1: the five-band solver (K_w left out of the w tendency) */
  int32_t reserved;
  const int64_t* cell_edges;       /* nc x cw */
  const int64_t* edge_cells;       /* ne x 2 */
  const int64_t* edge_vertices;    /* ne x 2 */
  const int64_t* vertex_edges;     /* nv x vw */
  const int64_t* vertex_cells;     /* nv x vw */
  const int64_t* vk_cell_vertices; /* nc x cw */
  const double* kinetic;           /* nc x cw: alpha l_e d_{e,i} / 2A_i */
  const double* inner;             /* nc x cw: l_e d_{e,i} / A_i */
  const double* vk_kites;          /* nc x cw */
  const double* edge_weight;       /* ne x 2: d_{e,i} / d_e */
  const double* rhombus;           /* ne x 2 */
  const double* inverse_dual;      /* ne: 1 / (a d_e) */
  const double* edge_coriolis;     /* ne */
  const double* curl;              /* nv x vw: t_{e,v} d_e / (a A_v) */
  const double* vertex_weight;     /* nv x vw: K_{i,v} / A_v */
  const double* vk_weights;        /* nv x vw */
  const double* coriolis;          /* nv */
  const double* trisk;             /* edge-first ne x nt */
  const double* dz_cells;          /* nlev x nc (level slabs) */
  const double* dzh_cells;         /* (nlev + 1) x nc */
  const double* wlow;              /* (nlev + 1) x nc */
  const double* dz_edges;          /* nlev x ne */
  const double* dzh_edges;         /* (nlev + 1) x ne */
  const int32_t* trisk_index;      /* edge-first ne x nt x 3 */
} TriskMpasTables;
/* The stage state ys and the work arrays slow_tendencies! fills, all DEVICE pointers in the
 * reference's layout (level slabs, horizontal index fastest): vn nlev x ne, w (nlev + 1) x nc,
 * rho and rhotheta nlev x nc; theta, exner, K nlev x nc; Kv (may be NULL without the vertex
 * kinetic energy), qv, zetav, rhov nlev x nv; qe, rhoe, Fs nlev x ne; eta (nlev + 1) x ne
 * (left untouched by the advective form, as there); tvn nlev x ne; tw (nlev + 1) x nc. */
typedef struct {
  const double *vn, *w, *rho, *rhotheta;
  double *theta, *exner, *K, *Kv, *qv, *zetav, *rhov, *qe, *rhoe, *Fs, *eta, *tvn, *tw;
} TriskMpasFields;
typedef struct TriskMpas TriskMpas;
/* Uploads the tables once. levels_per_thread: levels each thread walks with its neighbour
 * tables in registers (0 = 8; 1, 2, 4, 8 or 16). Tables wider than 10 edges per cell, 4 per
 * vertex or 18 TRiSK neighbours return TRISK_ERR_UNSUPPORTED. */
int trisk_mpas_create(const TriskMpasTables* tables, int32_t device, int32_t levels_per_thread, TriskMpas** out);
void trisk_mpas_destroy(TriskMpas* ops);
/* slow_tendencies!(m, ys, pressure) for flat ground; returns when the results are complete.
 * Ordered after the work already queued on the legacy default stream. */
int trisk_mpas_slow_tendencies(TriskMpas* ops, const TriskMpasFields* fields, double pressure);
/* The same without waiting (trisk_mpas_stream gives the stream it runs on). */
int trisk_mpas_slow_tendencies_async(TriskMpas* ops, const TriskMpasFields* fields, double pressure);
int trisk_mpas_stream(TriskMpas* ops, void** stream);
int trisk_mpas_synchronize(TriskMpas* ops);
int64_t trisk_mpas_launch_count(TriskMpas* ops);

/* ---- one rank's part of a distributed model -------------------------------------------
 * Replaces TRiSKShallowWater(grid; comm, part)     src/FiniteVolumes/TRiSKShallowWater.jl:121-168
 * with its TRiSKDistribution                      src/FiniteVolumes/TRiSKDistribution.jl:70-106
 * and tendency! with exchange_state!              TRiSKShallowWater.jl:201,379-394
 * (exchange!, src/Parallel/Halo.jl:80-99) and rk4_step! (RungeKutta.jl:18-29) on it.
 * The model holds the rank's owned entities and its ghosts in local numbering, owned first:
 * its tables are the global ones restricted to the local entities (TriskCoefficients in
 * local numbering: local_table, TRiSKDistribution.jl:108-119). Before every tendency the ghost
 * values of the stage state are exchanged once (one packed buffer of all neighbours); the
 * ghosts' tendencies are zero, so owned values follow the undivided model bit for bit. */
typedef struct {
  int64_t ne_owned, nc_owned; /* local edges 1..ne_owned and cells 1..nc_owned are owned */
  int32_t nneighbors, pad_;
  /* neighbour k sends/receives the local state entries index[offsets[k] .. offsets[k+1]-1]
   * (offsets 0-based, nneighbors + 1 of them; indices 1-based into the local [u; h]:
   * edges 1..ne, cells ne+1..ne+nc). Sent entries are owned, received entries are ghosts. */
  const int64_t* send_offsets;
  const int64_t* send_index;
  const int64_t* recv_offsets;
  const int64_t* recv_index;
} TriskHalo;
/* The caller's exchange (the reference's MPI exchange!): fill recv (nrecv values, neighbour
 * after neighbour in the halo's order) from the neighbours, sending them `send` (nsend values,
 * in the same order). Returns 0, or a status the library passes on. */
typedef int (*TriskExchangeFn)(void* user, const double* send, int64_t nsend, double* recv, int64_t nrecv,
                               void* stream);
enum {
  TRISK_EXCHANGE_HOST = 0,   /* send/recv are host buffers; the device work before is finished */
  TRISK_EXCHANGE_DEVICE = 1, /* device buffers; the callback orders its transfers on `stream`
                                (a cudaStream_t), e.g. NCCL send/recv on that stream */
  TRISK_EXCHANGE_DEVICE_GRAPH = 2 /* as DEVICE, and each RK4 step is captured once per dt as a
                                     CUDA graph with the callback's stream work in it, so the
                                     callback must enqueue only capturable work */
};
typedef struct TriskDist TriskDist;
/* cfg: as trisk_model_create_from_coefficients (cell_positions, if given, are the local cells'
 * centers for the internal numbering, which keeps owned entities first). */
int trisk_dist_create(const TriskCoefficients* local, const TriskConfig* cfg, const TriskHalo* halo,
                      TriskDist** out);
void trisk_dist_destroy(TriskDist* dist);
int trisk_dist_set_exchange(TriskDist* dist, TriskExchangeFn fn, void* user, int32_t mode);
/* tendency! of the local state y (host or device; the ghost values used are the exchanged
 * ones, y itself is not changed); dy's ghost entries are 0. */
int trisk_dist_tendency(TriskDist* dist, const double* y, double* dy);
/* rk4_step! nsteps times in place on the local state (host or device), the stage updates
 * fused into the tendency phase as in trisk_rk4_step. */
int trisk_dist_rk4_step(TriskDist* dist, double* y, double dt, int64_t nsteps);
int trisk_dist_stream(TriskDist* dist, void** stream);
int64_t trisk_dist_launch_count(TriskDist* dist);

/* ---- batched ensembles ------------------------------------------------------------
 * No counterpart in the reference, which runs one model per process (examples/
 * trisk_shallow_water.jl:71-111); each member's arithmetic is that of rk4_step!
 * (RungeKutta.jl:18-29) on its group's model, bit for bit. A group = `members[g]` states
 * that share models[g]'s device tables (same mesh and scheme; all groups one scheme and
 * device), with its own dt[g] and step count nsteps[g]. Up to 8 groups. A group's members
 * are split into slices of consecutive members stored together; the three phases of a set of
 * slices run back to back, set after set, so a slice's work vectors stay in L2. One RK4 step
 * of all unfinished groups is one CUDA graph of persistent kernels; the models must outlive
 * the ensemble. */
typedef struct TriskEnsemble TriskEnsemble;
int trisk_ensemble_create(TriskModel* const* models, const int32_t* members, const double* dt,
                          const int64_t* nsteps, int32_t ngroups, TriskEnsemble** out);
/* As trisk_ensemble_create with the members' state, RK4 stage vectors and work vectors
 * stored in state_bits = 64 (FP64, bit for bit rk4_step!) or 32 (FP32 storage: every value
 * is rounded to float when stored, the arithmetic stays FP64, the tables stay FP64, and the
 * energy sums are FP64). set/get_member still exchange FP64 states. */
int trisk_ensemble_create_precision(TriskModel* const* models, const int32_t* members, const double* dt,
                                    const int64_t* nsteps, int32_t ngroups, int32_t state_bits,
                                    TriskEnsemble** out);
void trisk_ensemble_destroy(TriskEnsemble* ensemble);
/* Member state y = [u; h] in file numbering, host or device memory. */
int trisk_ensemble_set_member(TriskEnsemble* ensemble, int32_t group, int32_t member, const double* y);
int trisk_ensemble_get_member(TriskEnsemble* ensemble, int32_t group, int32_t member, double* y);
/* Advances every group by `steps` RK4 steps, or until it has taken nsteps[g]: one graph
 * replay per step, each replay of the groups still running. */
int trisk_ensemble_run_async(TriskEnsemble* ensemble, int64_t steps);
int trisk_ensemble_synchronize(TriskEnsemble* ensemble);
int trisk_ensemble_steps(TriskEnsemble* ensemble, int64_t* steps_taken); /* per group */
int trisk_ensemble_reset(TriskEnsemble* ensemble);                        /* step counters to 0 */
int trisk_ensemble_stream(TriskEnsemble* ensemble, void** stream);
int64_t trisk_ensemble_launch_count(TriskEnsemble* ensemble);
/* Threads per block of the ensemble's vertex, flux and tendency phases (multiples of 32 in
 * [64, 256]; default 128 each). */
int trisk_ensemble_set_block(TriskEnsemble* ensemble, const int32_t block[3]);
int trisk_ensemble_get_block(TriskEnsemble* ensemble, int32_t block[3]);
/* Members per slice of every group (ngroups values; the last slice of a group may have
 * fewer). The default is the whole group: on a B200 every slicing of the configuration-3
 * groups measured slower (tables streamed once per slice cost more than the L2 residency of
 * a slice's work vectors saves). Setting them keeps the members' states; results are the same
 * bit for bit for every slicing. */
int trisk_ensemble_set_slices(TriskEnsemble* ensemble, const int32_t* members_per_slice);
int trisk_ensemble_get_slices(TriskEnsemble* ensemble, int32_t* members_per_slice);
/* Members per thread of the three phases: 2 (two members per thread for a slice with an even
 * member count whose buffers start at an even element, else one) or 4 (four, as one 16-byte FP32 or two 16-byte FP64 vectors per
 * gathered value, so each table entry a thread loads serves four members; every slice's
 * member count must be a multiple of four, else TRISK_ERR_UNSUPPORTED, and a later slicing
 * that breaks this returns to 2). The default is 4 for an FP32-state ensemble whose groups
 * allow it, else 2. Results are the same bit for bit. */
int trisk_ensemble_set_members_per_thread(TriskEnsemble* ensemble, int32_t members);
int trisk_ensemble_get_members_per_thread(TriskEnsemble* ensemble, int32_t* members);
/* Autotuner of the batched path (no reference counterpart): times `steps` RK4 steps of all
 * groups for every combination of the phase block sizes {64, 128, 256}, then four members per
 * thread at each tendency block size (where the slices allow it), then for each group a few
 * members-per-slice values around the current one, keeps the fastest and restores the
 * members' states, step counters and step counts, so results are unchanged; best_ms gets the
 * time per step. Each call keeps one copy of the states until the ensemble is destroyed. */
int trisk_ensemble_autotune(TriskEnsemble* ensemble, int32_t steps, double* best_ms);
/* Algorithmic bytes of one RK4 step of all groups: sum 4 (T + 2 M N) + 15 M N. */
int trisk_ensemble_bytes(TriskEnsemble* ensemble, double* step_bytes);
/* Per-member total energy sum_i A_i h_i (K_i + g h_i / 2) of a group (M values, host),
 * as total_energy (TRiSKShallowWater.jl:406-411) of every member. */
int trisk_ensemble_energy(TriskEnsemble* ensemble, int32_t group, double* energies);

/* ---- learned closure inside an ensemble (no reference counterpart) ---------------------
 * With a closure, the network runs on all (edge, member) rows of the group's members (at
 * stage 1 of each RK4 step, its output reused by the other stages, or at every stage), and
 * every tendency adds, for members whose mask entry is 1, dF_e = sF y0 to the mass flux of
 * the continuity equation only (dh_i/dt = -sum_k div[i,k] (F + dF); flux form, so mass is
 * conserved; the PV flux keeps the resolved F) and du_e += sQ y1 to the momentum tendency.
 * Features per row, formed in FP64: u_e; u at the 10 TRiSK stencil edges minus u_e; mean and
 * difference (second minus first) of h at the two cells, of q at the two vertices and of K
 * at the two cells; 7 geometry values (`geometry`, ne x 7 in file edge order); normalized
 * as (x - mean) * scale with norm = [24 means, 24 scales, sF, sQ], then rounded to BF16.
 * TRiSK PV flux only.
 * flags: bit 0 (1) runs the network at every RK4 stage instead of once per step; bit 1 (2)
 * makes the momentum correction work-free per member: its component along the energy
 * gradient dE/du_e = u_e l_e (h_c0 d_c0 + h_c1 d_c1) (cell kinetic energy; l, d and the two
 * cell distances are geometry columns 0..3) is removed, so it does no work on the flow to
 * first order; bit 2 (4) runs the features, the network and the corrections as three launches
 * with the features and outputs in device memory, instead of one kernel that builds each tile's
 * features in shared memory and applies its outputs there (the same numbers bit for bit);
 * bits 8-15: the network interval n (0 or 1: every step): the network runs on the steps whose
 * group step count is a multiple of n and its corrections are kept and applied on the steps
 * between (needs the one-kernel form at stage 1 only, else TRISK_ERR_UNSUPPORTED). Turning
 * a member off (trisk_ensemble_closure_mask) clears its kept corrections at once, and the
 * network runs on the next step after the closure is set and after every call that changes
 * the members' states or layout (set_member, reset, set_slices, autotune), whatever the
 * interval.
 * net = NULL removes the group's closure. */
int trisk_ensemble_set_closure(TriskEnsemble* ensemble, int32_t group, TriskClosure* net, const float* geometry,
                               const double* norm, int32_t flags);
int trisk_ensemble_closure_mask(TriskEnsemble* ensemble, int32_t group, const float* member_on);
/* The features of the group's current member states into X (device, 16-byte aligned, rows
 * e * M + m in file edge order, 24 BF16 each), for training data. */
int trisk_ensemble_features(TriskEnsemble* ensemble, int32_t group, void* X, const double* norm,
                            const float* geometry);
/* TRISK_ERR_TIMEOUT if a bounded tensor-core wait of a closure network gave up. */
int trisk_ensemble_closure_check(TriskEnsemble* ensemble);

/* ---- learned flux closure: the network ------------------------------------------------
 * No counterpart in the reference. An edge-local MLP 24 -> 64 -> 64 -> 2 (GELU) whose two
 * hidden layers run as tcgen05 BF16 MMAs with FP32 accumulators in tensor memory, for
 * inference and training (FP32 master weights, Adam). Parameters are 5890 floats: W1 (64 x
 * 24), b1, W2 (64 x 64), b2, W3 (2 x 64), b3, row-major. Device arrays: X (n x 24, BF16),
 * targets and outputs (n x 2, FP32). A bounded wait on the tensor core that gives up
 * returns TRISK_ERR_TIMEOUT. */
int trisk_closure_create(int32_t device, const float* params, TriskClosure** out); /* params: host, or NULL */
void trisk_closure_destroy(TriskClosure* closure);
int32_t trisk_closure_param_count(void);
int trisk_closure_get_params(TriskClosure* closure, float* params);
int trisk_closure_set_params(TriskClosure* closure, const float* params);
int trisk_closure_forward(TriskClosure* closure, const void* X, int64_t n, float* Y);
/* Gradient of (1/n) sum_rows sum_k (Y_k - target_k)^2 into grads (host, or NULL to keep it on
 * the device for trisk_closure_adam) and the mean loss into *loss. */
int trisk_closure_gradients(TriskClosure* closure, const void* X, const float* target, int64_t n, float* grads,
                            float* loss);
int trisk_closure_adam(TriskClosure* closure, float lr, float beta1, float beta2, float eps);
int trisk_closure_synchronize(TriskClosure* closure);
int trisk_closure_stream(TriskClosure* closure, void** stream);
/* Launch shape of inference: the persistent grid's CTAs per SM (seven on a B200) and the SMs. */
int trisk_closure_info(TriskClosure* closure, int32_t* forward_ctas_per_sm, int32_t* sms);
/* Test of the bounded tensor-core wait (no reference counterpart): the next inference call of
 * this closure leaves the first tensor-core operation of tile `tile` (rows 128 tile ..) un-issued,
 * so that tile's wait runs out after half a second and the call returns TRISK_ERR_TIMEOUT; the
 * closure stays usable and later calls are unaffected. */
int trisk_closure_expire_wait_once(TriskClosure* closure, int64_t tile);

/* ---- allocation-free entry point ---------------------------------------------------
 * No counterpart in the reference: it exists for callers that must not have the library
 * allocate device memory (a host whose device memory all comes from its own pool, such as
 * CUDA.jl's, or code running while a stream is being captured into a CUDA graph).
 *
 * *out = sum_i a[i] * b[i] over caller-owned device vectors (with a = the cell areas and
 * b = the heights this is the total mass, dot(areas, h)). a, b and out must be
 * device pointers on one device; the work is enqueued on `stream` (a cudaStream_t, NULL for
 * the default stream) and not waited for. The call makes no cudaMalloc, cudaFree or other
 * allocating call: its scratch is a static 64 KiB device array that every GPU loading the
 * library holds until exit, which limits n to 16777216 (larger n is rejected with
 * TRISK_ERR_ARGUMENT). The first call on a device looks that array's address up
 * (cudaGetSymbolAddress), so make it before any stream capture. All calls share the array:
 * calls whose work overlaps on the GPU race and give wrong sums; serialize them. */
int trisk_weighted_sum_noalloc(const double* a, const double* b, int64_t n, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
