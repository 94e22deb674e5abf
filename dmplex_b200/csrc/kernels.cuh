// sm_100a kernels of the TRiSK shallow-water tendency and the RK4 stage updates.
//
// The reference runs 6-8 one-entity-per-thread KernelAbstractions gathers per tendency
// (src/FiniteVolumes/TRiSKShallowWater.jl:202-305) plus 4 broadcast passes per RK4 step
// (src/TimeSteppers/RungeKutta.jl:18-29). Here a tendency is three launches, one per
// grid-wide dependency level:
//
//   k_vertex : zeta_v, h_v, q_v (TRiSK only), K_v (alpha != 1)        (:212-219, :246-259)
//   k_flux   : edges -> F_e = h_e u_e and q_e;  cells -> B_i = K_i + g h_i
//                                                          (:202-210, :222-244, :261-273)
//   k_tend   : edges -> du_e (TRiSK or Gassmann PV flux - grad B);  cells -> dh_i = -div F
//              followed by the fused RK4 stage update of that state element
//                                                          (:275-305, RungeKutta.jl:21-27)
//
// Every per-entity sum keeps the reference's table-row order and association, and the
// library is compiled with --fmad=false, so results are bitwise those of the same
// arithmetic done serially (the CPU oracle), whatever the entity numbering.
//
// Memory layout in HBM: neighbour tables are int32 / FP64 "structure of arrays"
// [k][entity] with the entity dimension padded to a multiple of 32, so a warp reads each
// table row with one 128 B (int32) or 256 B (FP64) coalesced transaction. Tables are read
// with evict-first (streaming) loads: they are touched once per tendency and should not
// push the small state and work vectors (a few MB, reused across the three phases) out of
// L2. The state and work vectors are [entity][member] so that in an ensemble one gathered
// index serves the contiguous member values of that entity.
//
// Programmatic dependent launch: every kernel loads its (read-only) tables first, then
// executes griddepcontrol.wait, and only then touches data written by the previous phase.
// Launched with the programmatic-serialization attribute, the next phase's table stream
// overlaps the previous phase's tail.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace trisk {

constexpr int CW = 6;   // cell table width (hexagons; pentagons padded)
constexpr int VW = 3;   // vertex table width (Voronoi vertices have three edges)
constexpr int TWD = 10; // TRiSK table width (5 + 5 edges of the two hexagons)
constexpr int GW = 12;  // Gassmann stencil width

// PVM_GASSMANN_DERIVED: Gassmann's PV edges are not read from a table but derived from the
// flux edges. gassmann_coefficients (TRiSKGrid.jl:227-246) fills each vertex block of six
// entries as [f1, o, o, f2, o', o'] with PV edges [f2, f1, f1, f1, f2, f2]: entry k takes
// the PV of flux edge 3 or 0 of its block. The upload verifies this for every edge.
enum PvMode { PVM_TRISK = 0, PVM_GASSMANN = 1, PVM_GASSMANN_MEAN = 2, PVM_GASSMANN_DERIVED = 3 };
__host__ __device__ constexpr int derived_pv_source(int k) {
  return (k / 6) * 6 + ((k % 6 == 0 || k % 6 == 4 || k % 6 == 5) ? 3 : 0);
}
enum KeMode { KE_CELL = 0, KE_VERTEX = 1, KE_MIXED = 2 };
enum Epilogue { EPI_TENDENCY = 0, EPI_STAGE1 = 1, EPI_STAGE2 = 2, EPI_STAGE3 = 3, EPI_STAGE4 = 4 };

struct DevTables {
  int32_t nc, ne, nv;
  int32_t ldc, lde, ldv;  // padded entity counts of the [k][entity] tables
  // Owned entities: internal edges < ne_own and cells < nc_own (all of them, except on one
  // rank's part of a distributed model, whose ghosts follow and get zero tendencies).
  int32_t ne_own, nc_own;
  double gravity;
  // Table entries below keep_end (a prefix of the one packed table block) are loaded with
  // an L2 evict-last policy, so they stay in L2 from one launch to the next; nullptr: none.
  const char* keep_end;
  const int32_t* cell_edges;     // CW x ldc
  const double* divergence;      // CW x ldc
  const double* kinetic;         // CW x ldc (alpha != 0)
  const int32_t* cell_vertices;  // CW x ldc (alpha != 1)
  const double* vk_kites;        // CW x ldc (alpha != 1)
  const int32_t* edge_cells;     // 2 x lde
  const double* edge_height;     // 2 x lde (alpha != 0)
  const int32_t* edge_vertices;  // 2 x lde
  const double* inverse_dual;    // lde
  const double* vk_height;       // 2 x lde (alpha != 1)
  const double* rhombus;         // 2 x lde (Gassmann)
  const double* g_coriolis;      // lde (Gassmann)
  const int32_t* trisk_edges;    // TWD x lde (TRiSK)
  const double* trisk;           // TWD x lde (TRiSK)
  const int32_t* g_edges;        // GW x lde (Gassmann)
  const int32_t* g_pv_edges;     // GW x lde (Gassmann, not for the mean variant)
  const double* g_weights;       // GW x lde (Gassmann)
  const int32_t* vertex_edges;   // VW x ldv
  const double* curl;            // VW x ldv
  const int32_t* vertex_cells;   // VW x ldv
  const double* vertex_height;   // VW x ldv
  const double* coriolis;        // ldv
  const double* vk_weights;      // VW x ldv (alpha != 1)
};

// Work vectors of one member group, [entity][member], stored as R (double; float for an
// FP32-state ensemble, whose arithmetic stays FP64). dq, dF: the closure's momentum-
// tendency and mass-flux corrections per edge (only read by the closure variant of the
// tendency phase).
template <class R>
struct DevWorkT {
  R *K, *B, *F, *qe, *zv, *hv, *qv, *Kv;
  R* dq = nullptr;
  R* dF = nullptr;
};
using DevWork = DevWorkT<double>;

// State pointers of one stage. y = [u (ne x M); h (nc x M)].
template <class R>
struct DevStageT {
  const R* u;   // stage state read by the phases
  const R* h;
  R* y;         // base state (RK4) / unused for a plain tendency
  R* acc;       // k1 + 2 k2 + 2 k3 accumulator
  R* st;        // next stage state
  R* dy;        // plain tendency output
  double c;     // dt/2 (stages 1, 2) or dt (stage 3)
  double sixth; // dt/6
  int* flag;    // set to 1 when a non-finite state appears
};
using DevStage = DevStageT<double>;

// The same buffers seen with storage type R (the ensemble keeps its pointers as double*).
template <class R>
__host__ __device__ __forceinline__ DevWorkT<R> work_as(const DevWork& W) {
  DevWorkT<R> o;
  o.K = reinterpret_cast<R*>(W.K);
  o.B = reinterpret_cast<R*>(W.B);
  o.F = reinterpret_cast<R*>(W.F);
  o.qe = reinterpret_cast<R*>(W.qe);
  o.zv = reinterpret_cast<R*>(W.zv);
  o.hv = reinterpret_cast<R*>(W.hv);
  o.qv = reinterpret_cast<R*>(W.qv);
  o.Kv = reinterpret_cast<R*>(W.Kv);
  o.dq = reinterpret_cast<R*>(W.dq);
  o.dF = reinterpret_cast<R*>(W.dF);
  return o;
}

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ T ldt_stream(const T* p) {  // streaming (evict-first) table load
  return __ldcs(p);
}

__device__ __forceinline__ uint64_t l2_policy(bool keep) {
  uint64_t pol;
  if (keep)
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  else
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double ld_hint(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_hint(const int32_t* p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

// Table entry base[i]. KEEP = false: streaming load (evict-first). KEEP = true: tables that
// start below T.keep_end (the L2-resident prefix of the packed block) load with an L2
// evict-last policy, the others with evict-first; the choice is per table, uniform.
template <bool KEEP, class V>
__device__ __forceinline__ V ldt(const DevTables& T, const V* base, int i) {
  if constexpr (KEEP) {
    return ld_hint(base + i, l2_policy(reinterpret_cast<const char*>(base) < T.keep_end));
  } else {
    return ldt_stream(base + i);
  }
}

template <bool ENS>
__device__ __forceinline__ void split(int t, int M, int& ent, int& mem) {
  if (ENS) {
    if ((M & (M - 1)) == 0) {  // power-of-two member counts (uniform): a shift, no division
      ent = t >> (__ffs(M) - 1);
      mem = t & (M - 1);
    } else {
      ent = t / M;
      mem = t - ent * M;
    }
  } else {
    ent = t;
    mem = 0;
  }
}

// P members per thread (P = 1, 2 or 4, M a multiple of P): the thread's members are mm ..
// mm + P - 1, read and written as one P-wide vector (two 16-byte halves for four FP64
// members); the arithmetic per member is that of P = 1, so results are the same bit for bit.
template <bool ENS, int P>
__device__ __forceinline__ void split_p(int t, int M, int& ent, int& mm) {
  if (P == 1) {
    split<ENS>(t, M, ent, mm);
  } else {
    int g;
    split<ENS>(t, M / P, ent, g);
    mm = g * P;
  }
}

template <class R, int P>
__device__ __forceinline__ void ld_members(const R* p, double (&x)[P]) {
  if constexpr (P == 1) {
    x[0] = p[0];
  } else if constexpr (P == 4 && sizeof(R) == 8) {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    x[0] = a.x;
    x[1] = a.y;
    x[2] = b.x;
    x[3] = b.y;
  } else if constexpr (P == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    x[0] = v.x;
    x[1] = v.y;
    x[2] = v.z;
    x[3] = v.w;
  } else if constexpr (sizeof(R) == 8) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    x[0] = v.x;
    x[1] = v.y;
  } else {
    const float2 v = *reinterpret_cast<const float2*>(p);
    x[0] = v.x;
    x[1] = v.y;
  }
}

template <class R, int P>
__device__ __forceinline__ void st_members(R* p, const double (&x)[P]) {
  if constexpr (P == 1) {
    p[0] = (R)x[0];
  } else if constexpr (P == 4 && sizeof(R) == 8) {
    *reinterpret_cast<double2*>(p) = make_double2(x[0], x[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(x[2], x[3]);
  } else if constexpr (P == 4) {
    *reinterpret_cast<float4*>(p) = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
  } else if constexpr (sizeof(R) == 8) {
    *reinterpret_cast<double2*>(p) = make_double2(x[0], x[1]);
  } else {
    *reinterpret_cast<float2*>(p) = make_float2((float)x[0], (float)x[1]);
  }
}

// ------------------------------------------------------------------------------------
// phase 1: vertices
// Each phase is a __device__ body over one block's worth of entities (block index vb),
// called by the one-model kernels with vb = blockIdx.x and by the persistent ensemble
// kernels (ensemble.cu) for every block of work they take.
template <int PV, int KE, bool ENS, class R = double, bool KEEP = false, int P = 1>
__device__ __forceinline__ void vertex_body(const DevTables& T, const DevWorkT<R>& W, const R* u, const R* h,
                                            int M, int want_qv, int vb) {
  int v, mm;
  split_p<ENS, P>(vb * blockDim.x + threadIdx.x, M, v, mm);
  if (v >= T.nv) return;
  int ve[VW], vc[VW];
  double cu[VW], vh[VW], vkw[VW];
  double cor = 0.0;
#pragma unroll
  for (int k = 0; k < VW; ++k) {
    ve[k] = ldt<KEEP>(T, T.vertex_edges, k * T.ldv + v);
    cu[k] = ldt<KEEP>(T, T.curl, k * T.ldv + v);
    vc[k] = ldt<KEEP>(T, T.vertex_cells, k * T.ldv + v);
    vh[k] = ldt<KEEP>(T, T.vertex_height, k * T.ldv + v);
    if (KE != KE_CELL) vkw[k] = ldt<KEEP>(T, T.vk_weights, k * T.ldv + v);
  }
  const bool qv = PV == PVM_TRISK || want_qv;
  if (qv) cor = ldt<KEEP>(T, T.coriolis, v);
  pdl_wait();
  double uu[VW][P], hh[VW][P];
#pragma unroll
  for (int k = 0; k < VW; ++k) {
    ld_members<R, P>(u + (size_t)ve[k] * M + mm, uu[k]);
    ld_members<R, P>(h + (size_t)vc[k] * M + mm, hh[k]);
  }
  double z[P], eta[P], q[P], kv[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    z[p] = 0.0;
    eta[p] = 0.0;
#pragma unroll
    for (int k = 0; k < VW; ++k) z[p] += cu[k] * uu[k][p];
#pragma unroll
    for (int k = 0; k < VW; ++k) eta[p] += vh[k] * hh[k][p];
    if (qv) q[p] = (z[p] + cor) / eta[p];
    kv[p] = 0.0;
    if (KE != KE_CELL) {
#pragma unroll
      for (int k = 0; k < VW; ++k) kv[p] += vkw[k] * (uu[k][p] * uu[k][p]);
    }
  }
  const size_t o = (size_t)v * M + mm;
  // only what a later phase reads: zeta_v for the Gassmann rhombus PV, h_v for it and for
  // the vertex part of the mass flux, q_v for the TRiSK edge PV; all three for a diagnostic
  // call (want_qv)
  if (want_qv || PV != PVM_TRISK) st_members<R, P>(W.zv + o, z);
  if (want_qv || PV != PVM_TRISK || KE != KE_CELL) st_members<R, P>(W.hv + o, eta);
  if (qv) st_members<R, P>(W.qv + o, q);
  if (KE != KE_CELL) st_members<R, P>(W.Kv + o, kv);
}

template <int PV, int KE, bool ENS, class R = double, bool KEEP = false>
__global__ void __launch_bounds__(256) k_vertex(DevTables T, DevWorkT<R> W, const R* u, const R* h, int M,
                                                int want_qv) {
  pdl_trigger();
  vertex_body<PV, KE, ENS, R, KEEP>(T, W, u, h, M, want_qv, blockIdx.x);
}

// ------------------------------------------------------------------------------------
// phase 2: edges (mass flux, edge PV) and cells (Bernoulli function); blocks [0, nbE)
// take edges, the rest cells
template <int PV, int KE, bool ENS, class R = double, bool KEEP = false, int P = 1>
__device__ __forceinline__ void flux_body(const DevTables& T, const DevWorkT<R>& W, const R* u, const R* h,
                                          int M, int nbE, int want_K, int vb) {
  if (vb < nbE) {
    int e, mm;
    split_p<ENS, P>(vb * blockDim.x + threadIdx.x, M, e, mm);
    if (e >= T.ne) return;
    const int ev0 = ldt<KEEP>(T, T.edge_vertices, e), ev1 = ldt<KEEP>(T, T.edge_vertices, T.lde + e);
    int ec0 = 0, ec1 = 0;
    double eh0 = 0, eh1 = 0, vk0 = 0, vk1 = 0, r0 = 0, r1 = 0, gc = 0;
    if (KE != KE_VERTEX) {
      ec0 = ldt<KEEP>(T, T.edge_cells, e);
      ec1 = ldt<KEEP>(T, T.edge_cells, T.lde + e);
      eh0 = ldt<KEEP>(T, T.edge_height, e);
      eh1 = ldt<KEEP>(T, T.edge_height, T.lde + e);
    }
    if (KE != KE_CELL) {
      vk0 = ldt<KEEP>(T, T.vk_height, e);
      vk1 = ldt<KEEP>(T, T.vk_height, T.lde + e);
    }
    if (PV != PVM_TRISK) {
      r0 = ldt<KEEP>(T, T.rhombus, e);
      r1 = ldt<KEEP>(T, T.rhombus, T.lde + e);
      gc = ldt<KEEP>(T, T.g_coriolis, e);
    }
    pdl_wait();
    const size_t o = (size_t)e * M + mm;
    const size_t o0 = (size_t)ev0 * M + mm, o1 = (size_t)ev1 * M + mm;
    double ue[P], hv0[P], hv1[P], hc0[P], hc1[P], a0[P], a1[P];
    ld_members<R, P>(u + o, ue);
    if (KE != KE_CELL || PV != PVM_TRISK) {
      ld_members<R, P>(W.hv + o0, hv0);
      ld_members<R, P>(W.hv + o1, hv1);
    }
    if (KE != KE_VERTEX) {
      ld_members<R, P>(h + (size_t)ec0 * M + mm, hc0);
      ld_members<R, P>(h + (size_t)ec1 * M + mm, hc1);
    }
    if (PV == PVM_TRISK) {
      ld_members<R, P>(W.qv + o0, a0);
      ld_members<R, P>(W.qv + o1, a1);
    } else {
      ld_members<R, P>(W.zv + o0, a0);
      ld_members<R, P>(W.zv + o1, a1);
    }
    double Fo[P], qo[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      double he;
      if (KE == KE_CELL) {
        he = eh0 * hc0[p] + eh1 * hc1[p];
      } else if (KE == KE_VERTEX) {
        he = vk0 * hv0[p] + vk1 * hv1[p];  // the reference's zero cell part adds exactly 0
      } else {
        he = eh0 * hc0[p] + eh1 * hc1[p] + vk0 * hv0[p] + vk1 * hv1[p];
      }
      Fo[p] = he * ue[p];
      if (PV == PVM_TRISK) {
        qo[p] = (a0[p] + a1[p]) / 2;
      } else {
        const double z = r0 * a0[p] + r1 * a1[p];
        const double eta = r0 * hv0[p] + r1 * hv1[p];
        qo[p] = (z + gc) / eta;
      }
    }
    st_members<R, P>(W.F + o, Fo);
    st_members<R, P>(W.qe + o, qo);
  } else {
    int i, mm;
    split_p<ENS, P>((vb - nbE) * blockDim.x + threadIdx.x, M, i, mm);
    if (i >= T.nc) return;
    int ce[CW], cv[CW];
    double kin[CW], kk[CW];
#pragma unroll
    for (int k = 0; k < CW; ++k) {
      if (KE != KE_VERTEX) {
        ce[k] = ldt<KEEP>(T, T.cell_edges, k * T.ldc + i);
        kin[k] = ldt<KEEP>(T, T.kinetic, k * T.ldc + i);
      }
      if (KE != KE_CELL) {
        cv[k] = ldt<KEEP>(T, T.cell_vertices, k * T.ldc + i);
        kk[k] = ldt<KEEP>(T, T.vk_kites, k * T.ldc + i);
      }
    }
    pdl_wait();
    const size_t o = (size_t)i * M + mm;
    double hi[P], Kc[P], Bc[P];
    ld_members<R, P>(h + o, hi);
    double uk[CW][P], kv[CW][P];
    if (KE != KE_VERTEX) {
#pragma unroll
      for (int k = 0; k < CW; ++k) ld_members<R, P>(u + (size_t)ce[k] * M + mm, uk[k]);
    }
    if (KE != KE_CELL) {
#pragma unroll
      for (int k = 0; k < CW; ++k) ld_members<R, P>(W.Kv + (size_t)cv[k] * M + mm, kv[k]);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      double K = 0.0, B;
      if (KE != KE_VERTEX) {
#pragma unroll
        for (int k = 0; k < CW; ++k) K += kin[k] * (uk[k][p] * uk[k][p]);
        B = K + T.gravity * hi[p];
      } else {
        B = T.gravity * hi[p];  // the reference's zero cell part adds exactly 0
      }
      if (KE != KE_CELL) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < CW; ++k) s += kk[k] * kv[k][p];
        K += s;
        B += s;
      }
      Kc[p] = K;
      Bc[p] = B;
    }
    st_members<R, P>(W.B + o, Bc);
    if (want_K) st_members<R, P>(W.K + o, Kc);
  }
}

template <int PV, int KE, bool ENS, class R = double, bool KEEP = false>
__global__ void __launch_bounds__(256) k_flux(DevTables T, DevWorkT<R> W, const R* u, const R* h, int M,
                                              int nbE, int want_K) {
  pdl_trigger();
  flux_body<PV, KE, ENS, R, KEEP>(T, W, u, h, M, nbE, want_K, blockIdx.x);
}

// ------------------------------------------------------------------------------------
// phase 3: tendencies and the RK4 stage update
template <int EPI, class R = double>
__device__ __forceinline__ void epilogue(const DevStageT<R>& S, size_t j, double kv) {
  if (EPI == EPI_TENDENCY) {
    S.dy[j] = (R)kv;
  } else if (EPI == EPI_STAGE1) {
    const double y = S.y[j];
    S.acc[j] = (R)kv;
    S.st[j] = (R)(y + S.c * kv);
  } else if (EPI == EPI_STAGE2 || EPI == EPI_STAGE3) {
    const double y = S.y[j], a = S.acc[j];
    S.acc[j] = (R)(a + 2 * kv);
    S.st[j] = (R)(y + S.c * kv);
  } else {
    const double y = S.y[j], a = S.acc[j];
    const R yn = (R)(y + S.sixth * (a + kv));
    S.y[j] = yn;
    if (!isfinite(yn)) atomicOr(S.flag, 1);
  }
}

template <int PV, int EPI, bool ENS, bool CL = false, class R = double, bool KEEP = false>
__device__ __forceinline__ void tend_body(const DevTables& T, const DevWorkT<R>& W, const DevStageT<R>& S, int M,
                                          int nbE, int vb) {
  if (vb < nbE) {
    int e, mm;
    split<ENS>(vb * blockDim.x + threadIdx.x, M, e, mm);
    if (e >= T.ne) return;
    const int ec0 = ldt<KEEP>(T, T.edge_cells, e), ec1 = ldt<KEEP>(T, T.edge_cells, T.lde + e);
    const double invd = ldt<KEEP>(T, T.inverse_dual, e);
    const size_t o = (size_t)e * M + mm;
    double du;
    if (PV == PVM_TRISK) {
      int te[TWD];
      double tr[TWD];
#pragma unroll
      for (int k = 0; k < TWD; ++k) {
        te[k] = ldt<KEEP>(T, T.trisk_edges, k * T.lde + e);
        tr[k] = ldt<KEEP>(T, T.trisk, k * T.lde + e);
      }
      pdl_wait();
      const double qself = W.qe[o];
      double f[TWD], q[TWD];
#pragma unroll
      for (int k = 0; k < TWD; ++k) {
        f[k] = W.F[(size_t)te[k] * M + mm];
        q[k] = W.qe[(size_t)te[k] * M + mm];
      }
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < TWD; ++k) s += tr[k] * f[k] * (qself + q[k]);
      du = s / 2 - ((double)W.B[(size_t)ec1 * M + mm] - (double)W.B[(size_t)ec0 * M + mm]) * invd;
    } else {
      int ge[GW], gp[GW];
      double gw[GW];
#pragma unroll
      for (int k = 0; k < GW; ++k) {
        ge[k] = ldt<KEEP>(T, T.g_edges, k * T.lde + e);
        if (PV == PVM_GASSMANN) gp[k] = ldt<KEEP>(T, T.g_pv_edges, k * T.lde + e);
        gw[k] = ldt<KEEP>(T, T.g_weights, k * T.lde + e);
      }
      pdl_wait();
      double f[GW], q[GW];
      const double qself = PV == PVM_GASSMANN_MEAN ? W.qe[o] : 0.0;
      if (PV == PVM_GASSMANN_DERIVED) {  // four distinct PV gathers per edge
        const double q0 = W.qe[(size_t)ge[0] * M + mm], q3 = W.qe[(size_t)ge[3] * M + mm];
        const double q6 = W.qe[(size_t)ge[6] * M + mm], q9 = W.qe[(size_t)ge[9] * M + mm];
#pragma unroll
        for (int k = 0; k < GW; ++k) {
          const int src = derived_pv_source(k);
          q[k] = src == 0 ? q0 : (src == 3 ? q3 : (src == 6 ? q6 : q9));
        }
      }
#pragma unroll
      for (int k = 0; k < GW; ++k) {
        f[k] = W.F[(size_t)ge[k] * M + mm];
        if (PV == PVM_GASSMANN)
          q[k] = W.qe[(size_t)gp[k] * M + mm];
        else if (PV == PVM_GASSMANN_MEAN)
          q[k] = (qself + W.qe[(size_t)ge[k] * M + mm]) / 2;
      }
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < GW; ++k) s += gw[k] * f[k] * q[k];
      du = s - ((double)W.B[(size_t)ec1 * M + mm] - (double)W.B[(size_t)ec0 * M + mm]) * invd;
    }
    if (CL) du += (double)W.dq[o];  // learned momentum correction
    if (e >= T.ne_own) du = 0.0;     // a ghost edge (TRiSKShallowWater.jl:389-393)
    epilogue<EPI, R>(S, o, du);
  } else {
    int i, mm;
    split<ENS>((vb - nbE) * blockDim.x + threadIdx.x, M, i, mm);
    if (i >= T.nc) return;
    int ce[CW];
    double dv[CW];
#pragma unroll
    for (int k = 0; k < CW; ++k) {
      ce[k] = ldt<KEEP>(T, T.cell_edges, k * T.ldc + i);
      dv[k] = ldt<KEEP>(T, T.divergence, k * T.ldc + i);
    }
    pdl_wait();
    double f[CW];
#pragma unroll
    for (int k = 0; k < CW; ++k) {
      f[k] = W.F[(size_t)ce[k] * M + mm];
      if (CL) f[k] += (double)W.dF[(size_t)ce[k] * M + mm];  // learned mass-flux correction
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < CW; ++k) s += dv[k] * f[k];
    const size_t o = (size_t)i * M + mm;
    epilogue<EPI, R>(S, (size_t)T.ne * M + o, i >= T.nc_own ? 0.0 : -s);  // ghost cells: 0
  }
}

// The RK4 epilogue for P consecutive members at j (vector loads and stores of the stage
// vectors; per member the arithmetic of epilogue<EPI>).
template <int EPI, class R, int P>
__device__ __forceinline__ void epilogue_p(const DevStageT<R>& S, size_t j, const double (&kv)[P]) {
  if constexpr (P == 1) {
    epilogue<EPI, R>(S, j, kv[0]);
  } else {
    double y[P], a[P], st[P], acc[P];
    if (EPI == EPI_TENDENCY) {
      st_members<R, P>(S.dy + j, kv);
      return;
    }
    ld_members<R, P>(S.y + j, y);
    if (EPI == EPI_STAGE2 || EPI == EPI_STAGE3 || EPI == EPI_STAGE4) ld_members<R, P>(S.acc + j, a);
#pragma unroll
    for (int p = 0; p < P; ++p) {
      if (EPI == EPI_STAGE1) {
        acc[p] = kv[p];
        st[p] = y[p] + S.c * kv[p];
      } else if (EPI == EPI_STAGE2 || EPI == EPI_STAGE3) {
        acc[p] = a[p] + 2 * kv[p];
        st[p] = y[p] + S.c * kv[p];
      } else {
        st[p] = y[p] + S.sixth * (a[p] + kv[p]);
      }
    }
    if (EPI == EPI_STAGE4) {
      R out[P];
      bool bad = false;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        out[p] = (R)st[p];
        bad |= !isfinite(out[p]);
      }
      st_members<R, P>(S.y + j, st);
      if (bad) atomicOr(S.flag, 1);
    } else {
      st_members<R, P>(S.acc + j, acc);
      st_members<R, P>(S.st + j, st);
    }
  }
}

// The tendency phase of an ensemble group with P members per thread: as tend_body, with the
// stencil sums accumulated while the stencil streams (same order per member), so that two
// members fit the register budget.
template <int PV, int EPI, bool CL, class R, int P>
__device__ __forceinline__ void tend_body_p(const DevTables& T, const DevWorkT<R>& W, const DevStageT<R>& S,
                                            int M, int nbE, int vb) {
  if (vb < nbE) {
    int e, mm;
    split_p<true, P>(vb * blockDim.x + threadIdx.x, M, e, mm);
    if (e >= T.ne) return;
    const int ec0 = ldt<false>(T, T.edge_cells, e), ec1 = ldt<false>(T, T.edge_cells, T.lde + e);
    const double invd = ldt<false>(T, T.inverse_dual, e);
    const size_t o = (size_t)e * M + mm;
    double s[P], du[P];
    if (PV == PVM_TRISK) {
      pdl_wait();
      double qself[P];
      ld_members<R, P>(W.qe + o, qself);
#pragma unroll
      for (int p = 0; p < P; ++p) s[p] = 0.0;
#pragma unroll
      for (int k = 0; k < TWD; ++k) {
        const int te = ldt<false>(T, T.trisk_edges, k * T.lde + e);
        const double tr = ldt<false>(T, T.trisk, k * T.lde + e);
        double f[P], q[P];
        ld_members<R, P>(W.F + (size_t)te * M + mm, f);
        ld_members<R, P>(W.qe + (size_t)te * M + mm, q);
#pragma unroll
        for (int p = 0; p < P; ++p) s[p] += tr * f[p] * (qself[p] + q[p]);
      }
      double b0[P], b1[P];
      ld_members<R, P>(W.B + (size_t)ec0 * M + mm, b0);
      ld_members<R, P>(W.B + (size_t)ec1 * M + mm, b1);
#pragma unroll
      for (int p = 0; p < P; ++p) du[p] = s[p] / 2 - (b1[p] - b0[p]) * invd;
    } else {
      pdl_wait();
      double qself[P], q0[P], q3[P], q6[P], q9[P];
      if (PV == PVM_GASSMANN_MEAN) ld_members<R, P>(W.qe + o, qself);
      if (PV == PVM_GASSMANN_DERIVED) {
        const int g0 = ldt<false>(T, T.g_edges, e), g3 = ldt<false>(T, T.g_edges, 3 * T.lde + e);
        const int g6 = ldt<false>(T, T.g_edges, 6 * T.lde + e), g9 = ldt<false>(T, T.g_edges, 9 * T.lde + e);
        ld_members<R, P>(W.qe + (size_t)g0 * M + mm, q0);
        ld_members<R, P>(W.qe + (size_t)g3 * M + mm, q3);
        ld_members<R, P>(W.qe + (size_t)g6 * M + mm, q6);
        ld_members<R, P>(W.qe + (size_t)g9 * M + mm, q9);
      }
#pragma unroll
      for (int p = 0; p < P; ++p) s[p] = 0.0;
#pragma unroll
      for (int k = 0; k < GW; ++k) {
        const int ge = ldt<false>(T, T.g_edges, k * T.lde + e);
        const double gw = ldt<false>(T, T.g_weights, k * T.lde + e);
        double f[P], q[P];
        ld_members<R, P>(W.F + (size_t)ge * M + mm, f);
        if (PV == PVM_GASSMANN_DERIVED) {
          const int src = derived_pv_source(k);
#pragma unroll
          for (int p = 0; p < P; ++p) q[p] = src == 0 ? q0[p] : (src == 3 ? q3[p] : (src == 6 ? q6[p] : q9[p]));
        } else if (PV == PVM_GASSMANN) {
          const int gp = ldt<false>(T, T.g_pv_edges, k * T.lde + e);
          ld_members<R, P>(W.qe + (size_t)gp * M + mm, q);
        } else {
          double qk[P];
          ld_members<R, P>(W.qe + (size_t)ge * M + mm, qk);
#pragma unroll
          for (int p = 0; p < P; ++p) q[p] = (qself[p] + qk[p]) / 2;
        }
#pragma unroll
        for (int p = 0; p < P; ++p) s[p] += gw * f[p] * q[p];
      }
      double b0[P], b1[P];
      ld_members<R, P>(W.B + (size_t)ec0 * M + mm, b0);
      ld_members<R, P>(W.B + (size_t)ec1 * M + mm, b1);
#pragma unroll
      for (int p = 0; p < P; ++p) du[p] = s[p] - (b1[p] - b0[p]) * invd;
    }
    if (CL) {  // learned momentum correction
      double dqo[P];
      ld_members<R, P>(W.dq + o, dqo);
#pragma unroll
      for (int p = 0; p < P; ++p) du[p] += dqo[p];
    }
    epilogue_p<EPI, R, P>(S, o, du);
  } else {
    int i, mm;
    split_p<true, P>((vb - nbE) * blockDim.x + threadIdx.x, M, i, mm);
    if (i >= T.nc) return;
    pdl_wait();
    double s[P];
#pragma unroll
    for (int p = 0; p < P; ++p) s[p] = 0.0;
#pragma unroll
    for (int k = 0; k < CW; ++k) {
      const int ce = ldt<false>(T, T.cell_edges, k * T.ldc + i);
      const double dv = ldt<false>(T, T.divergence, k * T.ldc + i);
      double f[P];
      ld_members<R, P>(W.F + (size_t)ce * M + mm, f);
      if (CL) {
        double df[P];
        ld_members<R, P>(W.dF + (size_t)ce * M + mm, df);
#pragma unroll
        for (int p = 0; p < P; ++p) f[p] += df[p];
      }
#pragma unroll
      for (int p = 0; p < P; ++p) s[p] += dv * f[p];
    }
    double dh[P];
#pragma unroll
    for (int p = 0; p < P; ++p) dh[p] = -s[p];
    epilogue_p<EPI, R, P>(S, (size_t)T.ne * M + (size_t)i * M + mm, dh);
  }
}

template <int PV, int EPI, bool ENS, bool KEEP = false>
__global__ void __launch_bounds__(256) k_tend(DevTables T, DevWork W, DevStage S, int M, int nbE) {
  pdl_trigger();
  tend_body<PV, EPI, ENS, false, double, KEEP>(T, W, S, M, nbE, blockIdx.x);
}

// ------------------------------------------------------------------------------------
// RK4 steps in one cooperative launch, for meshes whose tables and vectors stay in L2: the
// twelve phases of a step follow one another inside the kernel, separated by a grid-wide
// barrier, instead of as twelve launches (whose start-up latency dominates when each phase
// moves a few MB). Every block loops over the phases' blocks of work (the bodies above), so
// results are those of the launches bit for bit.

// The grid barrier: arrivals counted in *count, released by incrementing *gen. A block's wait
// gives up after a second (or 2^31 polls, a backstop that the clock always beats), sets *err
// and leaves; a block that sees *err after a barrier returns, so every wait ends.
struct GridBarrier {
  unsigned* count;
  unsigned* gen;
  int* err;
};

__device__ __forceinline__ long long barrier_ns() {
  long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool grid_sync(const GridBarrier& B) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = B.gen;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(B.count, 1u) == gridDim.x - 1) {
      atomicExch(B.count, 0u);
      __threadfence();
      atomicAdd(B.gen, 1u);
    } else {
      const long long start = barrier_ns();
      for (unsigned i = 1; *gen == g; ++i)
        if (((i & 1023u) == 0 && barrier_ns() - start > 1000000000LL) || i == (1u << 31)) {
          atomicExch(B.err, 1);
          break;
        }
    }
    __threadfence();
  }
  __syncthreads();
  return *reinterpret_cast<volatile int*>(B.err) == 0;
}

template <int PV, int EPI>
__device__ __forceinline__ void tend_phase(const DevTables& T, const DevWork& W, const DevStage& S, int nbE, int nbT) {
  for (int vb = blockIdx.x; vb < nbT; vb += gridDim.x) tend_body<PV, EPI, false, false, double, false>(T, W, S, 1, nbE, vb);
}

template <int PV, int KE>
__global__ void __launch_bounds__(256) k_rk4_persistent(DevTables T, DevWork W, DevStage S, double dt, int nsteps,
                                                        GridBarrier B) {
  const int nbV = (T.nv + (int)blockDim.x - 1) / (int)blockDim.x;
  const int nbE = (T.ne + (int)blockDim.x - 1) / (int)blockDim.x;
  const int nbC = (T.nc + (int)blockDim.x - 1) / (int)blockDim.x;
  for (int step = 0; step < nsteps; ++step) {
#pragma unroll 1
    for (int stage = 1; stage <= 4; ++stage) {
      const double* u = stage == 1 ? S.y : S.st;
      for (int vb = blockIdx.x; vb < nbV; vb += gridDim.x)
        vertex_body<PV, KE, false, double, false, 1>(T, W, u, u + T.ne, 1, 0, vb);
      if (!grid_sync(B)) return;
      for (int vb = blockIdx.x; vb < nbE + nbC; vb += gridDim.x)
        flux_body<PV, KE, false, double, false, 1>(T, W, u, u + T.ne, 1, nbE, 0, vb);
      if (!grid_sync(B)) return;
      DevStage St = S;
      St.u = u;
      St.h = u + T.ne;
      St.c = stage == 3 ? dt : dt / 2;
      switch (stage) {
        case 1: tend_phase<PV, EPI_STAGE1>(T, W, St, nbE, nbE + nbC); break;
        case 2: tend_phase<PV, EPI_STAGE2>(T, W, St, nbE, nbE + nbC); break;
        case 3: tend_phase<PV, EPI_STAGE3>(T, W, St, nbE, nbE + nbC); break;
        default: tend_phase<PV, EPI_STAGE4>(T, W, St, nbE, nbE + nbC); break;
      }
      if (!grid_sync(B)) return;
    }
  }
}

}  // namespace trisk
