/*
 * CPU oracle for the TRiSK shallow-water tendency and the classical RK4 step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA path is compared with; it is
 * never linked into, loaded by, or called from the product library. Only tests/, the smoke
 * check and bench.py's CPU-baseline leg use it.
 *
 * It restates, in plain C with FP64 arithmetic and the same loop and summation order, the
 * KernelAbstractions kernels of dmplex.jl:
 *   src/FiniteVolumes/TRiSKShallowWater.jl:202-314  (kernels)
 *   src/FiniteVolumes/TRiSKShallowWater.jl:322-394  (run!, kinetic_energy!, mass_flux!,
 *                                                   vertex_pv!, pv_flux!, tendency!)
 *   src/FiniteVolumes/TRiSKShallowWater.jl:397-433  (total_mass, total_energy,
 *                                                   potential_enstrophy, relative_vorticity,
 *                                                   tangential_velocity)
 *   src/TimeSteppers/RungeKutta.jl:1-29             (RK4Cache, rk4_step!)
 *
 * The tables are the arrays a serial TRiSKShallowWater model holds, in the reference's own
 * layout: column-major [k, entity] (k fastest), Int64 indices that are 1-BASED as in Julia,
 * padded entries with index 1 and weight 0.
 *
 * Parity pinning: the reference ships no golden vectors or fixtures for this path and
 * cannot run here (no Julia). The oracle is pinned by the reference's own test-suite
 * properties (test/finite_volumes.jl: operator identities, semi-discrete energy
 * conservation, mass conservation to round-off, TC2 error and convergence bounds), which
 * tests/test_oracle.py re-runs against it, and by the accuracy figures the reference publishes
 * for this path (docs/STATUS.md: kinetic-energy, tangential and TC2 errors on plain, spring
 * and centroidal meshes; the Galewsky outcome of each PV flux), which tests/test_published.py
 * and tests/test_galewsky_pin.py reproduce to the digits printed. Bitwise agreement with
 * Julia is unverifiable.
 */
#ifndef TRISK_ORACLE_H
#define TRISK_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t nc, ne, nv;
  int32_t cw, vw, tw; /* padded widths: cell (6), vertex (3), TRiSK (10) tables */
  int32_t pv_flux;    /* 0 :trisk, 1 :gassmann, 2 :gassmann_mean */
  double alpha;       /* kinetic-energy weight: 1 :cell, 0 :vertex, 3/8 :mixed */
  double gravity;
  const int64_t* cell_edges; /* cw x nc */
  const double* divergence;
  const double* kinetic;
  const int64_t* edge_cells; /* 2 x ne */
  const double* edge_height;
  const int64_t* edge_vertices;
  const double* inverse_dual; /* ne */
  const int64_t* vertex_edges; /* vw x nv */
  const double* curl;
  const int64_t* vertex_cells;
  const double* vertex_height;
  const double* coriolis;     /* nv */
  const int64_t* trisk_edges; /* tw x ne */
  const double* trisk;
  const double* cell_areas;   /* nc */
  const double* vertex_areas; /* nv */
  /* Gassmann (pv_flux != 0), else NULL */
  const int64_t* g_edges; /* 12 x ne */
  const int64_t* g_pv_edges;
  const double* g_weights;
  const double* rhombus;    /* 2 x ne */
  const double* g_coriolis; /* ne */
  /* vertex kinetic energy (alpha != 1), else NULL */
  const int64_t* vk_cell_vertices; /* cw x nc */
  const double* vk_kites;
  const double* vk_weights; /* vw x nv */
  const double* vk_height;  /* 2 x ne */
} oracle_model;

/* Work vectors of the model (TRiSKShallowWater.jl:160-161). */
typedef struct {
  double *K, *B, *F, *zv, *hv, *qv, *qe, *Kv;
} oracle_work;

int oracle_model_size(void); /* sizeof(oracle_model), for binding checks */
oracle_work* oracle_work_create(const oracle_model* m);
void oracle_work_destroy(oracle_work* w);

/* threads <= 1: serial loops; otherwise OpenMP with a barrier after each kernel, as run!
 * does on the CPU backend (TRiSKShallowWater.jl:322-327). */
void oracle_set_threads(int threads);
int oracle_threads(void);

/* tendency!(dy, y, m), TRiSKShallowWater.jl:379-394. y = [u(ne); h(nc)]. */
void oracle_tendency(const oracle_model* m, oracle_work* w, const double* y, double* dy);
/* rk4_step!(y, dt, tendency!, cache, m), RungeKutta.jl:18-29; cache = 5 vectors of ne+nc. */
void oracle_rk4_step(const oracle_model* m, oracle_work* w, double* y, double dt, double* cache);
/* The stage tendencies of the kernels, exposed for per-kernel parity tests. */
void oracle_kinetic_energy(const oracle_model* m, oracle_work* w, const double* u, const double* h);
void oracle_vertex_pv(const oracle_model* m, oracle_work* w, const double* u, const double* h);
void oracle_mass_flux(const oracle_model* m, oracle_work* w, const double* u, const double* h);
/* Diagnostics, TRiSKShallowWater.jl:397-419. */
double oracle_total_mass(const oracle_model* m, const double* y);
double oracle_total_energy(const oracle_model* m, oracle_work* w, const double* y);
double oracle_potential_enstrophy(const oracle_model* m, oracle_work* w, const double* y);
/* edge_sum_kernel!: relative_vorticity (nv) and tangential_velocity (ne), :421-433. */
void oracle_relative_vorticity(const oracle_model* m, const double* y, double* zeta);
void oracle_tangential_velocity(const oracle_model* m, const double* u, double* vt);

#ifdef __cplusplus
}
#endif
#endif
