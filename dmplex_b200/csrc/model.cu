// TRiSK shallow-water model on one B200: table upload, the internal (Hilbert) numbering,
// the phase launches, the CUDA-graph RK4 step and the diagnostics, behind the C ABI of
// include/trisk_b200.h.
#include <algorithm>
#include <cstring>
#include <memory>
#include <type_traits>

#include "model.hpp"

using trisk::Error;

namespace trisk {

// ---------------------------------------------------------------------------------------
// small kernels: state permutation, reductions, vorticity

__global__ void k_gather(double* __restrict__ dst, const double* __restrict__ src, const int32_t* __restrict__ idx,
                         int64_t n) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) dst[j] = src[idx[j]];
}

// dst[idx[j]] = src[j], j < n
__global__ void k_scatter(double* __restrict__ dst, const double* __restrict__ src, const int32_t* __restrict__ idx,
                          int64_t n) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) dst[idx[j]] = src[j];
}

constexpr int RED_BLOCK = 256, RED_PER_THREAD = 8;

// MODE 0: a b   MODE 1: (a b)(c + g b / 2)   MODE 2: (a b)(c c)
template <int MODE>
__global__ void k_reduce_partial(const double* a, const double* b, const double* c, double g, int64_t n,
                                 double* partials) {
  __shared__ double sm[RED_BLOCK];
  const int64_t base = (int64_t)blockIdx.x * RED_BLOCK * RED_PER_THREAD;
  double s = 0.0;
  for (int r = 0; r < RED_PER_THREAD; ++r) {
    const int64_t i = base + (int64_t)r * RED_BLOCK + threadIdx.x;
    if (i < n) {
      double t;
      if (MODE == 0)
        t = a[i] * b[i];
      else if (MODE == 1)
        t = a[i] * b[i] * (c[i] + g * b[i] / 2);
      else
        t = a[i] * b[i] * (c[i] * c[i]);
      s += t;
    }
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = RED_BLOCK / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
}

__global__ void k_reduce_final(const double* partials, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += partials[i];
    *out = s;
  }
}

__global__ void k_vertex_curl(DevTables T, const double* u, double* zeta) {  // edge_sum_kernel! as curl
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= T.nv) return;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < VW; ++k) s += T.curl[k * T.ldv + v] * u[T.vertex_edges[k * T.ldv + v]];
  zeta[v] = s;
}

void order_after_caller(cudaStream_t stream, cudaEvent_t ev) {
  CUDA_CHECK(cudaEventRecord(ev, cudaStreamLegacy));
  CUDA_CHECK(cudaStreamWaitEvent(stream, ev, 0));
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void launch_gather(cudaStream_t stream, double* dst, const double* src, const int32_t* idx, int64_t n) {
  k_gather<<<(unsigned)cdiv(n, 256), 256, 0, stream>>>(dst, src, idx, n);
  CUDA_CHECK(cudaGetLastError());
}

// Host staging of all tables in one allocation (256-byte aligned pieces).
struct Packer {
  std::vector<char> host;
  size_t add(size_t bytes) {
    size_t off = (size_t)round_up((int64_t)host.size(), 256);
    host.resize(off + bytes, 0);
    return off;
  }
  template <class T>
  T* at(size_t off) {
    return reinterpret_cast<T*>(host.data() + off);
  }
};

}  // namespace trisk

using namespace trisk;

namespace {

// ---------------------------------------------------------------------------------------
// launch helpers

template <typename... KArgs, typename... Args>
void launch(TriskModel& m, void (*kernel)(KArgs...), int64_t grid, int block, cudaEvent_t ev0, cudaEvent_t ev1,
            Args&&... args) {
  if (grid <= 0) return;
  if (ev0) CUDA_CHECK(cudaEventRecord(ev0, m.stream));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = m.stream;
  cudaLaunchAttribute attr[2];
  unsigned na = 0;
  if (m.use_pdl && !ev0) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (m.l2_window) {  // the resident table prefix as a persisting L2 window
    attr[na].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[na].val.accessPolicyWindow.base_ptr = m.table_base;
    attr[na].val.accessPolicyWindow.num_bytes = m.l2_keep_bytes;
    attr[na].val.accessPolicyWindow.hitRatio = 1.0f;
    attr[na].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[na].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    ++na;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  if (ev1) CUDA_CHECK(cudaEventRecord(ev1, m.stream));
  m.launches++;
}

template <class F>
void with_modes(int pv, int ke, F&& f) {
  using std::integral_constant;
  switch (pv * 3 + ke) {
    case 0: f(integral_constant<int, 0>{}, integral_constant<int, 0>{}); break;
    case 1: f(integral_constant<int, 0>{}, integral_constant<int, 1>{}); break;
    case 2: f(integral_constant<int, 0>{}, integral_constant<int, 2>{}); break;
    case 3: f(integral_constant<int, 1>{}, integral_constant<int, 0>{}); break;
    case 4: f(integral_constant<int, 1>{}, integral_constant<int, 1>{}); break;
    case 5: f(integral_constant<int, 1>{}, integral_constant<int, 2>{}); break;
    case 6: f(integral_constant<int, 2>{}, integral_constant<int, 0>{}); break;
    case 7: f(integral_constant<int, 2>{}, integral_constant<int, 1>{}); break;
    case 8: f(integral_constant<int, 2>{}, integral_constant<int, 2>{}); break;
    case 9: f(integral_constant<int, 3>{}, integral_constant<int, 0>{}); break;
    case 10: f(integral_constant<int, 3>{}, integral_constant<int, 1>{}); break;
    case 11: f(integral_constant<int, 3>{}, integral_constant<int, 2>{}); break;
    default: throw Error(TRISK_ERR_ARGUMENT, "bad scheme");
  }
}

// One tendency: three phase launches. ev: optional 6 events (pairs around each launch).
// With an L2-resident table prefix the kernels' KEEP variants run (per-table L2 policies).
void enqueue_tendency(TriskModel& m, const DevStage& S, int epi, cudaEvent_t* ev = nullptr) {
  const int bV = m.block[0], bF = m.block[1], bT = m.block[2];
  const int64_t nbV = cdiv(m.nv, bV);
  const int64_t nbEF = cdiv(m.ne, bF), nbCF = cdiv(m.nc, bF);
  const int64_t nbET = cdiv(m.ne, bT), nbCT = cdiv(m.nc, bT);
  auto body = [&](auto pvc, auto kec, auto keepc) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    constexpr bool K = decltype(keepc)::value;
    launch(m, k_vertex<PV, KE, false, double, K>, nbV, bV, ev ? ev[0] : nullptr, ev ? ev[1] : nullptr, m.T, m.W, S.u,
           S.h, 1, 0);
    launch(m, k_flux<PV, KE, false, double, K>, nbEF + nbCF, bF, ev ? ev[2] : nullptr, ev ? ev[3] : nullptr, m.T,
           m.W, S.u, S.h, 1, (int)nbEF, 0);
    cudaEvent_t e0 = ev ? ev[4] : nullptr, e1 = ev ? ev[5] : nullptr;
    const int64_t g = nbET + nbCT;
    const int nbE = (int)nbET;
    switch (epi) {
      case EPI_TENDENCY: launch(m, k_tend<PV, EPI_TENDENCY, false, K>, g, bT, e0, e1, m.T, m.W, S, 1, nbE); break;
      case EPI_STAGE1: launch(m, k_tend<PV, EPI_STAGE1, false, K>, g, bT, e0, e1, m.T, m.W, S, 1, nbE); break;
      case EPI_STAGE2: launch(m, k_tend<PV, EPI_STAGE2, false, K>, g, bT, e0, e1, m.T, m.W, S, 1, nbE); break;
      case EPI_STAGE3: launch(m, k_tend<PV, EPI_STAGE3, false, K>, g, bT, e0, e1, m.T, m.W, S, 1, nbE); break;
      default: launch(m, k_tend<PV, EPI_STAGE4, false, K>, g, bT, e0, e1, m.T, m.W, S, 1, nbE); break;
    }
  };
  with_modes(m.pv, m.ke, [&](auto pvc, auto kec) {
    if (m.l2_keep_bytes > 0)
      body(pvc, kec, std::true_type{});
    else
      body(pvc, kec, std::false_type{});
  });
}

// One RK4 step on the internal state m.y (RungeKutta.jl:18-29). ev: optional 24 events.
void enqueue_step(TriskModel& m, double dt, cudaEvent_t* ev = nullptr) {
  DevStage S{};
  S.y = m.y;
  S.acc = m.acc;
  S.st = m.st;
  S.flag = m.flag;
  S.sixth = dt / 6;
  S.u = m.y;
  S.h = m.y + m.ne;
  S.c = dt / 2;
  enqueue_tendency(m, S, EPI_STAGE1, ev);
  S.u = m.st;
  S.h = m.st + m.ne;
  enqueue_tendency(m, S, EPI_STAGE2, ev ? ev + 6 : nullptr);
  S.c = dt;
  enqueue_tendency(m, S, EPI_STAGE3, ev ? ev + 12 : nullptr);
  enqueue_tendency(m, S, EPI_STAGE4, ev ? ev + 18 : nullptr);
}

void ensure_graph(TriskModel& m, double dt) {
  if (m.graph && m.graph_dt == dt) return;
  if (m.graph) {
    cudaGraphExecDestroy(m.graph);
    m.graph = nullptr;
  }
  const int64_t before = m.launches;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(m.stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_step(m, dt);
  } catch (...) {
    cudaStreamEndCapture(m.stream, &g);
    if (g) cudaGraphDestroy(g);
    m.launches = before;
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(m.stream, &g));
  m.launches = before;  // captured launches are counted when the graph is replayed
  cudaError_t e = cudaGraphInstantiate(&m.graph, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(e);
  m.graph_dt = dt;
}

constexpr int PERSISTENT_BLOCK = 256;

// All nsteps RK4 steps as one cooperative launch of k_rk4_persistent.
void run_persistent(TriskModel& m, double dt, int64_t nsteps) {
  DevStage S{};
  S.y = m.y;
  S.acc = m.acc;
  S.st = m.st;
  S.flag = m.flag;
  S.sixth = dt / 6;
  GridBarrier B{m.barrier, m.barrier + 1, m.barrier_err};
  for (int64_t done = 0; done < nsteps;) {
    const int n = (int)std::min<int64_t>(nsteps - done, 1 << 20);
    with_modes(m.pv, m.ke, [&](auto pvc, auto kec) {
      constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
      void* args[] = {&m.T, &m.W, &S, &dt, const_cast<int*>(&n), &B};
      CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_rk4_persistent<PV, KE>),
                                             dim3((unsigned)m.persistent_grid), dim3(PERSISTENT_BLOCK), args, 0,
                                             m.stream));
    });
    m.launches++;
    done += n;
  }
}

void run_steps(TriskModel& m, double dt, int64_t nsteps) {
  if (m.persistent) {
    run_persistent(m, dt, nsteps);
  } else if (m.use_graph) {
    ensure_graph(m, dt);
    for (int64_t s = 0; s < nsteps; ++s) {
      CUDA_CHECK(cudaGraphLaunch(m.graph, m.stream));
      m.launches += 12;
    }
  } else {
    for (int64_t s = 0; s < nsteps; ++s) enqueue_step(m, dt);
  }
}

void gather(TriskModel& m, double* dst, const double* src, const int32_t* idx, int64_t n) {
  launch_gather(m.stream, dst, src, idx, n);
  m.launches++;
}

// file-numbered user state -> internal m.y
void state_in(TriskModel& m, const double* y_user, double* dst) {
  const size_t bytes = (size_t)m.N * sizeof(double);
  if (is_device_pointer(y_user)) {
    order_after_caller(m.stream, m.caller_ev);
    if (m.identity)
      CUDA_CHECK(cudaMemcpyAsync(dst, y_user, bytes, cudaMemcpyDeviceToDevice, m.stream));
    else
      gather(m, dst, y_user, m.state_n2o, m.N);
  } else {
    if (m.identity) {
      CUDA_CHECK(cudaMemcpyAsync(dst, y_user, bytes, cudaMemcpyHostToDevice, m.stream));
    } else {
      CUDA_CHECK(cudaMemcpyAsync(m.stage, y_user, bytes, cudaMemcpyHostToDevice, m.stream));
      gather(m, dst, m.stage, m.state_n2o, m.N);
    }
  }
}

// internal src -> file-numbered user state
void state_out(TriskModel& m, double* y_user, const double* src) {
  const size_t bytes = (size_t)m.N * sizeof(double);
  if (is_device_pointer(y_user)) {
    order_after_caller(m.stream, m.caller_ev);
    if (m.identity)
      CUDA_CHECK(cudaMemcpyAsync(y_user, src, bytes, cudaMemcpyDeviceToDevice, m.stream));
    else
      gather(m, y_user, src, m.state_o2n, m.N);
  } else {
    if (m.identity) {
      CUDA_CHECK(cudaMemcpyAsync(y_user, src, bytes, cudaMemcpyDeviceToHost, m.stream));
    } else {
      gather(m, m.stage, src, m.state_o2n, m.N);
      CUDA_CHECK(cudaMemcpyAsync(y_user, m.stage, bytes, cudaMemcpyDeviceToHost, m.stream));
    }
  }
}

void check_flag(TriskModel& m) {
  int flag = 0, err = 0;
  CUDA_CHECK(cudaMemcpyAsync(&flag, m.flag, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  if (m.barrier_err) CUDA_CHECK(cudaMemcpyAsync(&err, m.barrier_err, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  if (err) {
    CUDA_CHECK(cudaMemsetAsync(m.barrier, 0, 2 * sizeof(unsigned), m.stream));
    CUDA_CHECK(cudaMemsetAsync(m.barrier_err, 0, sizeof(int), m.stream));
    CUDA_CHECK(cudaStreamSynchronize(m.stream));
    throw Error(TRISK_ERR_TIMEOUT, "a grid-barrier wait of the one-launch RK4 step gave up");
  }
  if (flag) {
    CUDA_CHECK(cudaMemsetAsync(m.flag, 0, sizeof(int), m.stream));
    throw Error(TRISK_ERR_NONFINITE, "the state became non-finite");
  }
}

// ---------------------------------------------------------------------------------------
// model construction

Coefficients coefficients_from_abi(const TriskCoefficients* c) {
  if (!c) throw Error(TRISK_ERR_ARGUMENT, "coefficients is NULL");
  Coefficients C;
  C.nc = c->nc;
  C.ne = c->ne;
  C.nv = c->nv;
  C.cw = c->cw;
  C.vw = c->vw;
  C.tw = c->tw;
  C.pv_flux = c->pv_flux;
  C.alpha = c->alpha;
  C.gravity = c->gravity;
  if (C.nc <= 0 || C.ne <= 0 || C.nv <= 0) throw Error(TRISK_ERR_ARGUMENT, "empty mesh");
  if (C.pv_flux < 0 || C.pv_flux > 2) throw Error(TRISK_ERR_ARGUMENT, "pv_flux must be :trisk, :gassmann or :gassmann_mean");
  auto idx = [](const int64_t* p, size_t n, int64_t bound, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    std::vector<int64_t> out(n);
    for (size_t i = 0; i < n; ++i) {
      if (p[i] < 1 || p[i] > bound)
        throw Error(TRISK_ERR_TABLE, std::string(name) + "[" + std::to_string(i) + "] = " + std::to_string(p[i]) +
                                         " is outside 1.." + std::to_string(bound));
      out[i] = p[i] - 1;
    }
    return out;
  };
  auto val = [](const double* p, size_t n, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    return std::vector<double>(p, p + n);
  };
  const size_t nc = C.nc, ne = C.ne, nv = C.nv;
  C.cell_edges = idx(c->cell_edges, C.cw * nc, C.ne, "cell_edges");
  C.divergence = val(c->divergence, C.cw * nc, "divergence");
  C.kinetic = val(c->kinetic, C.cw * nc, "kinetic");
  C.edge_cells = idx(c->edge_cells, 2 * ne, C.nc, "edge_cells");
  C.edge_height = val(c->edge_height, 2 * ne, "edge_height");
  C.edge_vertices = idx(c->edge_vertices, 2 * ne, C.nv, "edge_vertices");
  C.inverse_dual = val(c->inverse_dual, ne, "inverse_dual");
  C.vertex_edges = idx(c->vertex_edges, C.vw * nv, C.ne, "vertex_edges");
  C.curl = val(c->curl, C.vw * nv, "curl");
  C.vertex_cells = idx(c->vertex_cells, C.vw * nv, C.nc, "vertex_cells");
  C.vertex_height = val(c->vertex_height, C.vw * nv, "vertex_height");
  C.coriolis = val(c->coriolis, nv, "coriolis");
  if (C.pv_flux == PV_TRISK) {
    C.trisk_edges = idx(c->trisk_edges, C.tw * ne, C.ne, "trisk_edges");
    C.trisk = val(c->trisk, C.tw * ne, "trisk");
  }
  C.cell_areas = val(c->cell_areas, nc, "cell_areas");
  C.vertex_areas = val(c->vertex_areas, nv, "vertex_areas");
  if (C.pv_flux != PV_TRISK) {
    C.g_edges = idx(c->g_edges, 12 * ne, C.ne, "g_edges");
    C.g_pv_edges = idx(c->g_pv_edges, 12 * ne, C.ne, "g_pv_edges");
    C.g_weights = val(c->g_weights, 12 * ne, "g_weights");
    C.rhombus = val(c->rhombus, 2 * ne, "rhombus");
    C.g_coriolis = val(c->g_coriolis, ne, "g_coriolis");
  }
  if (C.alpha != 1.0) {
    C.vk_cell_vertices = idx(c->vk_cell_vertices, C.cw * nc, C.nv, "vk_cell_vertices");
    C.vk_kites = val(c->vk_kites, C.cw * nc, "vk_kites");
    C.vk_weights = val(c->vk_weights, C.vw * nv, "vk_weights");
    C.vk_height = val(c->vk_height, 2 * ne, "vk_height");
  }
  return C;
}

Grid grid_from_abi(const TriskGrid* g) {
  if (!g) throw Error(TRISK_ERR_ARGUMENT, "grid is NULL");
  Grid G;
  G.nc = g->nc;
  G.ne = g->ne;
  G.nv = g->nv;
  G.cw = g->cw;
  G.vw = g->vw;
  G.tw = g->tw;
  if (G.nc <= 0 || G.ne <= 0 || G.nv <= 0 || G.cw <= 0 || G.vw <= 0 || G.tw <= 0)
    throw Error(TRISK_ERR_ARGUMENT, "empty grid");
  auto v3 = [](const double* p, int64_t n, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    std::vector<V3> out(n);
    std::memcpy(out.data(), p, n * sizeof(V3));
    return out;
  };
  auto val = [](const double* p, size_t n, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    return std::vector<double>(p, p + n);
  };
  auto idx = [](const int64_t* p, size_t n, int64_t bound, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    std::vector<int64_t> out(n);
    for (size_t i = 0; i < n; ++i) {
      if (p[i] < 1 || p[i] > bound)
        throw Error(TRISK_ERR_TABLE, std::string(name) + "[" + std::to_string(i) + "] is outside 1.." +
                                         std::to_string(bound));
      out[i] = p[i] - 1;
    }
    return out;
  };
  const size_t nc = G.nc, ne = G.ne, nv = G.nv;
  G.centers = v3(g->centers, G.nc, "centers");
  G.vertices = v3(g->vertices, G.nv, "vertices");
  G.edge_points = v3(g->edge_points, G.ne, "edge_points");
  G.edge_normals = v3(g->edge_normals, G.ne, "edge_normals");
  G.primal_lengths = val(g->primal_lengths, ne, "primal_lengths");
  G.dual_lengths = val(g->dual_lengths, ne, "dual_lengths");
  G.edge_cells = idx(g->edge_cells, 2 * ne, G.nc, "edge_cells");
  G.edge_vertices = idx(g->edge_vertices, 2 * ne, G.nv, "edge_vertices");
  G.cell_distances = val(g->cell_distances, 2 * ne, "cell_distances");
  G.cell_areas = val(g->cell_areas, nc, "cell_areas");
  G.vertex_areas = val(g->vertex_areas, nv, "vertex_areas");
  G.cell_edges = idx(g->cell_edges, G.cw * nc, G.ne, "cell_edges");
  G.cell_signs = val(g->cell_signs, G.cw * nc, "cell_signs");
  G.cell_vertices = idx(g->cell_vertices, G.cw * nc, G.nv, "cell_vertices");
  G.cell_kites = val(g->cell_kites, G.cw * nc, "cell_kites");
  G.vertex_edges = idx(g->vertex_edges, G.vw * nv, G.ne, "vertex_edges");
  G.vertex_signs = val(g->vertex_signs, G.vw * nv, "vertex_signs");
  G.vertex_cells = idx(g->vertex_cells, G.vw * nv, G.nc, "vertex_cells");
  G.vertex_kites = val(g->vertex_kites, G.vw * nv, "vertex_kites");
  G.trisk_edges = idx(g->trisk_edges, G.tw * ne, G.ne, "trisk_edges");
  G.trisk_weights = val(g->trisk_weights, G.tw * ne, "trisk_weights");
  return G;
}

// Internal numbering: cells along the Hilbert curve, edges by first appearance in the
// cells' edge lists, vertices by first appearance in the edges' vertex pairs (the same
// rule as hilbert_order, src/Topology/Ordering.jl:54-82). The permutation is integer and
// exact; every table row keeps its order, so per-entity sums are unchanged bit for bit.
// Internal numbering: cells along the Hilbert curve of their centroids (the owned cells of a
// distributed model's part first, then its ghosts), edges by first appearance in the cells'
// edge lists (owned edges first), vertices by first appearance in the edges.
void build_numbering(TriskModel& m, const Coefficients& C, const std::vector<V3>* centroids) {
  const int64_t nc = C.nc, ne = C.ne, nv = C.nv;
  const int64_t nc_own = m.nc_own, ne_own = m.ne_own;
  std::vector<int64_t> cperm(nc);
  for (int64_t i = 0; i < nc; ++i) cperm[i] = i;
  if (centroids && nc_own == nc) {
    cperm = hilbert_sort(*centroids, 16);
  } else if (centroids) {  // owned cells, then ghost cells, each along the curve
    for (int part = 0; part < 2; ++part) {
      const int64_t lo = part ? nc_own : 0, hi = part ? nc : nc_own;
      std::vector<V3> c(centroids->begin() + lo, centroids->begin() + hi);
      const std::vector<int64_t> p = hilbert_sort(c, 16);
      for (int64_t j = 0; j < hi - lo; ++j) cperm[lo + j] = lo + p[j];
    }
  }
  m.cell_n2o.assign(nc, 0);
  m.cell_o2n.assign(nc, -1);
  for (int64_t j = 0; j < nc; ++j) {
    m.cell_n2o[j] = (int32_t)cperm[j];
    m.cell_o2n[cperm[j]] = (int32_t)j;
  }
  m.edge_o2n.assign(ne, -1);
  int32_t next = 0;
  if (centroids) {
    for (int64_t j = 0; j < nc; ++j) {
      const int64_t i = cperm[j];
      for (int k = 0; k < C.cw; ++k) {
        if (C.divergence[i * C.cw + k] == 0.0) continue;
        const int64_t e = C.cell_edges[i * C.cw + k];
        if (m.edge_o2n[e] < 0) m.edge_o2n[e] = next++;
      }
    }
  }
  for (int64_t e = 0; e < ne; ++e)
    if (m.edge_o2n[e] < 0) m.edge_o2n[e] = next++;
  if (ne_own < ne) {  // owned edges first, each kind in the order above
    std::vector<int64_t> order(ne);
    for (int64_t e = 0; e < ne; ++e) order[m.edge_o2n[e]] = e;
    int32_t owned = 0, ghost = (int32_t)ne_own;
    for (int64_t j = 0; j < ne; ++j) {
      const int64_t e = order[j];
      m.edge_o2n[e] = e < ne_own ? owned++ : ghost++;
    }
  }
  m.edge_n2o.assign(ne, 0);
  for (int64_t e = 0; e < ne; ++e) m.edge_n2o[m.edge_o2n[e]] = (int32_t)e;
  m.vert_o2n.assign(nv, -1);
  next = 0;
  if (centroids) {
    for (int64_t j = 0; j < ne; ++j) {
      const int64_t e = m.edge_n2o[j];
      for (int s = 0; s < 2; ++s) {
        const int64_t v = C.edge_vertices[2 * e + s];
        if (m.vert_o2n[v] < 0) m.vert_o2n[v] = next++;
      }
    }
  }
  for (int64_t v = 0; v < nv; ++v)
    if (m.vert_o2n[v] < 0) m.vert_o2n[v] = next++;
  m.vert_n2o.assign(nv, 0);
  for (int64_t v = 0; v < nv; ++v) m.vert_n2o[m.vert_o2n[v]] = (int32_t)v;
  m.identity = true;
  for (int64_t i = 0; i < nc && m.identity; ++i) m.identity = m.cell_n2o[i] == i;
  for (int64_t e = 0; e < ne && m.identity; ++e) m.identity = m.edge_n2o[e] == e;
}

// [k][ld] int32 table in internal numbering from a [k + w*entity] file-numbered table.
size_t pack_index(Packer& P, const std::vector<int64_t>& tab, int w, int wpad, int64_t n, int64_t ld,
                  const std::vector<int32_t>& n2o, const std::vector<int32_t>& target_o2n) {
  if (w > wpad) throw Error(TRISK_ERR_UNSUPPORTED, "neighbour table wider than the kernels support");
  const size_t off = P.add((size_t)wpad * ld * sizeof(int32_t));
  int32_t* out = P.at<int32_t>(off);
  for (int64_t j = 0; j < n; ++j) {
    const int64_t old = n2o[j];
    for (int k = 0; k < w; ++k) out[k * ld + j] = target_o2n[tab[old * w + k]];
  }
  return off;
}

size_t pack_weight(Packer& P, const std::vector<double>& tab, int w, int wpad, int64_t n, int64_t ld,
                   const std::vector<int32_t>& n2o) {
  if (w > wpad) throw Error(TRISK_ERR_UNSUPPORTED, "neighbour table wider than the kernels support");
  const size_t off = P.add((size_t)wpad * ld * sizeof(double));
  double* out = P.at<double>(off);
  for (int64_t j = 0; j < n; ++j) {
    const int64_t old = n2o[j];
    for (int k = 0; k < w; ++k) out[k * ld + j] = tab[old * w + k];
  }
  return off;
}

void upload(TriskModel& m, const Coefficients& C) {
  const int64_t nc = C.nc, ne = C.ne, nv = C.nv;
  const int64_t ldc = round_up(nc, 32), lde = round_up(ne, 32), ldv = round_up(nv, 32);
  if (C.vw > VW) throw Error(TRISK_ERR_UNSUPPORTED, "vertices with more than three edges are not supported");
  const bool cellK = C.alpha != 0.0, vertK = C.alpha != 1.0;
  Packer P;
  struct Off {
    size_t ce, dv, kin, cv, vkk, ec, eh, ev, invd, vkh, rh, gc, te, tr, ge, gp, gw, ve, cu, vc, vh, cor, vkw, ac, av;
  } o{};
  auto& cn = m.cell_n2o;
  auto& en = m.edge_n2o;
  auto& vn = m.vert_n2o;
  // Gassmann PV edges follow from the flux edges whenever every edge has the block
  // structure gassmann_coefficients produces; then the kernel derives them (exact).
  bool derived = false;
  if (C.pv_flux == PV_GASSMANN) {
    derived = true;
    for (int64_t e = 0; e < ne && derived; ++e)
      for (int k = 0; k < 12; ++k)
        if (C.g_pv_edges[12 * e + k] != C.g_edges[12 * e + derived_pv_source(k)]) {
          derived = false;
          break;
        }
    if (derived) m.pv = PVM_GASSMANN_DERIVED;
  }
  // Pack order: the tendency phase's tables first (edge_cells, read by two phases, leads),
  // then the flux phase's, then the vertex phase's, then the areas (diagnostics only). An
  // L2-resident prefix of the block (trisk_model_set_l2_residency) covers them in this order.
  o.ec = pack_index(P, C.edge_cells, 2, 2, ne, lde, en, m.cell_o2n);
  if (C.pv_flux != PV_TRISK) {
    o.ge = pack_index(P, C.g_edges, 12, GW, ne, lde, en, m.edge_o2n);
    if (C.pv_flux == PV_GASSMANN && !derived)
      o.gp = pack_index(P, C.g_pv_edges, 12, GW, ne, lde, en, m.edge_o2n);
    o.gw = pack_weight(P, C.g_weights, 12, GW, ne, lde, en);
  } else {
    o.te = pack_index(P, C.trisk_edges, C.tw, TWD, ne, lde, en, m.edge_o2n);
    o.tr = pack_weight(P, C.trisk, C.tw, TWD, ne, lde, en);
  }
  o.invd = pack_weight(P, C.inverse_dual, 1, 1, ne, lde, en);
  o.ce = pack_index(P, C.cell_edges, C.cw, CW, nc, ldc, cn, m.edge_o2n);
  o.dv = pack_weight(P, C.divergence, C.cw, CW, nc, ldc, cn);
  o.ev = pack_index(P, C.edge_vertices, 2, 2, ne, lde, en, m.vert_o2n);
  if (cellK) o.eh = pack_weight(P, C.edge_height, 2, 2, ne, lde, en);
  if (vertK) o.vkh = pack_weight(P, C.vk_height, 2, 2, ne, lde, en);
  if (C.pv_flux != PV_TRISK) {
    o.rh = pack_weight(P, C.rhombus, 2, 2, ne, lde, en);
    o.gc = pack_weight(P, C.g_coriolis, 1, 1, ne, lde, en);
  }
  if (cellK) o.kin = pack_weight(P, C.kinetic, C.cw, CW, nc, ldc, cn);
  if (vertK) {
    o.cv = pack_index(P, C.vk_cell_vertices, C.cw, CW, nc, ldc, cn, m.vert_o2n);
    o.vkk = pack_weight(P, C.vk_kites, C.cw, CW, nc, ldc, cn);
  }
  o.ve = pack_index(P, C.vertex_edges, C.vw, VW, nv, ldv, vn, m.edge_o2n);
  o.cu = pack_weight(P, C.curl, C.vw, VW, nv, ldv, vn);
  o.vc = pack_index(P, C.vertex_cells, C.vw, VW, nv, ldv, vn, m.cell_o2n);
  o.vh = pack_weight(P, C.vertex_height, C.vw, VW, nv, ldv, vn);
  o.cor = pack_weight(P, C.coriolis, 1, 1, nv, ldv, vn);
  if (vertK) o.vkw = pack_weight(P, C.vk_weights, C.vw, VW, nv, ldv, vn);
  o.ac = pack_weight(P, C.cell_areas, 1, 1, nc, ldc, cn);
  o.av = pack_weight(P, C.vertex_areas, 1, 1, nv, ldv, vn);
  const size_t used_bytes = o.ac;  // the kernels' tables end where the areas begin

  char* base = m.alloc<char>(P.host.size());
  CUDA_CHECK(cudaMemcpy(base, P.host.data(), P.host.size(), cudaMemcpyHostToDevice));
  m.table_base = base;
  m.table_block_bytes = used_bytes;
  auto I = [&](size_t off, bool used) { return used ? reinterpret_cast<const int32_t*>(base + off) : nullptr; };
  auto D = [&](size_t off, bool used) { return used ? reinterpret_cast<const double*>(base + off) : nullptr; };
  const bool g = C.pv_flux != PV_TRISK;
  DevTables& T = m.T;
  T.nc = (int32_t)nc;
  T.ne = (int32_t)ne;
  T.nv = (int32_t)nv;
  T.nc_own = (int32_t)m.nc_own;
  T.ne_own = (int32_t)m.ne_own;
  T.ldc = (int32_t)ldc;
  T.lde = (int32_t)lde;
  T.ldv = (int32_t)ldv;
  T.gravity = C.gravity;
  T.keep_end = nullptr;
  T.cell_edges = I(o.ce, true);
  T.divergence = D(o.dv, true);
  T.kinetic = D(o.kin, cellK);
  T.cell_vertices = I(o.cv, vertK);
  T.vk_kites = D(o.vkk, vertK);
  T.edge_cells = I(o.ec, true);
  T.edge_height = D(o.eh, cellK);
  T.edge_vertices = I(o.ev, true);
  T.inverse_dual = D(o.invd, true);
  T.vk_height = D(o.vkh, vertK);
  T.rhombus = D(o.rh, g);
  T.g_coriolis = D(o.gc, g);
  T.trisk_edges = I(o.te, !g);
  T.trisk = D(o.tr, !g);
  T.g_edges = I(o.ge, g);
  T.g_pv_edges = I(o.gp, C.pv_flux == PV_GASSMANN && !derived);
  T.g_weights = D(o.gw, g);
  T.vertex_edges = I(o.ve, true);
  T.curl = D(o.cu, true);
  T.vertex_cells = I(o.vc, true);
  T.vertex_height = D(o.vh, true);
  T.coriolis = D(o.cor, true);
  T.vk_weights = D(o.vkw, vertK);
  m.area_c = const_cast<double*>(D(o.ac, true));
  m.area_v = const_cast<double*>(D(o.av, true));

  // Algorithmic bytes in the canonical form: every table the scheme needs once (int32
  // index, FP64 weight), the Gassmann PV-edge table included even when it is derived.
  const double I4 = 4, F8 = 8;
  const bool tr = C.pv_flux == PV_TRISK, gm = C.pv_flux == PV_GASSMANN;
  m.pv_table_bytes_saved = derived ? (double)ne * GW * I4 : 0.0;
  double cellB = CW * (I4 + F8) + (cellK ? CW * F8 : 0) + (vertK ? CW * (I4 + F8) : 0);
  double edgeB = 2 * I4 + 2 * I4 + F8 + (cellK ? 2 * F8 : 0) + (vertK ? 2 * F8 : 0) +
                 (tr ? TWD * (I4 + F8) : GW * (I4 + F8) + (gm ? GW * I4 : 0) + 2 * F8 + F8);
  double vertB = VW * (I4 + F8) * 2 + (tr ? F8 : 0) + (vertK ? VW * F8 : 0);
  m.table_bytes_unique = nc * cellB + ne * edgeB + nv * vertB;
  // Per launch: the tables the kernel streams plus each state or work vector it reads or
  // writes, counted once.
  const double vV = vertB * nv + F8 * (ne + nc) + F8 * nv * (2 + (tr ? 1 : 0) + (vertK ? 1 : 0));
  const double eFlux = ne * (2 * I4 + (cellK ? 2 * I4 + 2 * F8 : 0) + (vertK ? 2 * F8 : 0) + (tr ? 0 : 3 * F8)) +
                       nc * ((cellK ? CW * (I4 + F8) : 0) + (vertK ? CW * (I4 + F8) : 0)) +
                       F8 * (ne + nc) /* u, h */ + F8 * nv * ((vertK || !tr ? 1 : 0) + 1 + (vertK ? 1 : 0)) +
                       F8 * (2 * ne + nc) /* F, qe, B */;
  const double eTend = ne * (2 * I4 + F8 + (tr ? TWD * (I4 + F8) : GW * (I4 + F8) + (gm ? GW * I4 : 0))) +
                       nc * CW * (I4 + F8) + F8 * (2 * ne + nc) /* F, qe, B */ + 28.0 * (ne + nc) /* RK4 update */;
  m.phase_bytes[0] = vV;
  m.phase_bytes[1] = eFlux;
  m.phase_bytes[2] = eTend;
}

void finish_create(TriskModel& m, const Coefficients& C, const std::vector<V3>* centroids, const TriskConfig* cfg) {
  m.nc = C.nc;
  m.ne = C.ne;
  m.nv = C.nv;
  if (m.nc_own < 0) m.nc_own = m.nc;
  if (m.ne_own < 0) m.ne_own = m.ne;
  m.N = C.ne + C.nc;
  m.pv = C.pv_flux;
  m.alpha = C.alpha;
  m.gravity = C.gravity;
  m.ke = C.alpha == 1.0 ? KE_CELL : (C.alpha == 0.0 ? KE_VERTEX : KE_MIXED);
  if (cfg) {
    m.use_graph = cfg->use_graph != 0;
    m.use_pdl = cfg->use_pdl != 0;
    if (cfg->block) {
      if (cfg->block % 32 != 0 || cfg->block < 64 || cfg->block > 256)
        throw Error(TRISK_ERR_ARGUMENT, "block must be a multiple of 32 in 64..256");
      m.block[0] = m.block[1] = m.block[2] = cfg->block;
    }
  }
  if (m.nc >= (1LL << 30) || m.ne >= (1LL << 30)) throw Error(TRISK_ERR_UNSUPPORTED, "mesh too large for int32 tables");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw Error(TRISK_ERR_CUDA, "no CUDA device is available");
  }
  if (m.device < 0 || m.device >= ndev) throw Error(TRISK_ERR_ARGUMENT, "device ordinal out of range");
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreateWithFlags(&m.caller_ev, cudaEventDisableTiming));
  build_numbering(m, C, centroids);
  upload(m, C);
  m.W.K = m.alloc<double>(m.nc);
  m.W.B = m.alloc<double>(m.nc);
  m.W.F = m.alloc<double>(m.ne);
  m.W.qe = m.alloc<double>(m.ne);
  m.W.zv = m.alloc<double>(m.nv);
  m.W.hv = m.alloc<double>(m.nv);
  m.W.qv = m.alloc<double>(m.nv);
  m.W.Kv = m.alloc<double>(m.nv);
  m.y = m.alloc<double>(m.N);
  m.acc = m.alloc<double>(m.N);
  m.st = m.alloc<double>(m.N);
  m.stage = m.alloc<double>(m.N);
  m.dy = m.alloc<double>(m.N);
  m.flag = m.alloc<int>(1);
  m.scalars = m.alloc<double>(4);
  m.partials = m.alloc<double>(cdiv(std::max(m.nc, m.nv), RED_BLOCK * RED_PER_THREAD) + 1);
  CUDA_CHECK(cudaMemset(m.flag, 0, sizeof(int)));
  CUDA_CHECK(cudaMemset(m.W.K, 0, m.nc * sizeof(double)));
  // state permutation: internal state index -> file index and back
  std::vector<int32_t> n2o(m.N), o2n(m.N);
  for (int64_t j = 0; j < m.ne; ++j) n2o[j] = m.edge_n2o[j];
  for (int64_t j = 0; j < m.nc; ++j) n2o[m.ne + j] = (int32_t)(m.ne + m.cell_n2o[j]);
  for (int64_t j = 0; j < m.N; ++j) o2n[n2o[j]] = (int32_t)j;
  m.state_n2o = m.alloc<int32_t>(m.N);
  m.state_o2n = m.alloc<int32_t>(m.N);
  m.vertex_o2n = m.alloc<int32_t>(m.nv);
  CUDA_CHECK(cudaMemcpy(m.state_n2o, n2o.data(), m.N * sizeof(int32_t), cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(m.state_o2n, o2n.data(), m.N * sizeof(int32_t), cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(m.vertex_o2n, m.vert_o2n.data(), m.nv * sizeof(int32_t), cudaMemcpyHostToDevice));
  m.C = C;
  CUDA_CHECK(cudaDeviceSynchronize());
}

// Switches the one-launch RK4 step on or off: the barrier words, and the grid of as many
// blocks as are co-resident (the cooperative launch refuses more).
void set_persistent(TriskModel& m, bool on) {
  if (!on) {
    m.persistent = false;
    return;
  }
  int coop = 0, sms = 0, occ = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, m.device));
  if (!coop) throw Error(TRISK_ERR_UNSUPPORTED, "the device has no cooperative launch");
  CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device));
  with_modes(m.pv, m.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rk4_persistent<PV, KE>, PERSISTENT_BLOCK, 0));
  });
  if (occ < 1) throw Error(TRISK_ERR_UNSUPPORTED, "the one-launch step does not fit an SM");
  const int64_t work = cdiv(m.ne + m.nc, PERSISTENT_BLOCK);  // the widest phase
  m.persistent_grid = (int)std::min<int64_t>((int64_t)sms * occ, work);
  if (!m.barrier) {
    m.barrier = m.alloc<unsigned>(2);
    m.barrier_err = m.alloc<int>(1);
  }
  CUDA_CHECK(cudaMemset(m.barrier, 0, 2 * sizeof(unsigned)));
  CUDA_CHECK(cudaMemset(m.barrier_err, 0, sizeof(int)));
  m.persistent = true;
}

TriskModel* checked(TriskModel* m) {
  if (!m) throw Error(TRISK_ERR_ARGUMENT, "model is NULL");
  return m;
}

template <int MODE>
double reduce(TriskModel& m, const double* a, const double* b, const double* c, double g, int64_t n) {
  const int nb = (int)cdiv(n, RED_BLOCK * RED_PER_THREAD);
  k_reduce_partial<MODE><<<nb, RED_BLOCK, 0, m.stream>>>(a, b, c, g, n, m.partials);
  k_reduce_final<<<1, 32, 0, m.stream>>>(m.partials, nb, m.scalars);
  CUDA_CHECK(cudaGetLastError());
  m.launches += 2;
  double out = 0;
  CUDA_CHECK(cudaMemcpyAsync(&out, m.scalars, sizeof(double), cudaMemcpyDeviceToHost, m.stream));
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  return out;
}

void export_coefficients(const Coefficients& C, CoefficientExport& keep, TriskCoefficients* out) {
  auto p1 = [](const std::vector<int64_t>& v, std::vector<int64_t>& k) -> const int64_t* {
    if (v.empty()) return nullptr;
    k.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) k[i] = v[i] + 1;
    return k.data();
  };
  auto d = [](const std::vector<double>& v) -> const double* { return v.empty() ? nullptr : v.data(); };
  std::memset(out, 0, sizeof(*out));
  out->nc = C.nc;
  out->ne = C.ne;
  out->nv = C.nv;
  out->cw = C.cw;
  out->vw = C.vw;
  out->tw = C.tw;
  out->pv_flux = C.pv_flux;
  out->alpha = C.alpha;
  out->gravity = C.gravity;
  out->cell_edges = p1(C.cell_edges, keep.t[0]);
  out->divergence = d(C.divergence);
  out->kinetic = d(C.kinetic);
  out->edge_cells = p1(C.edge_cells, keep.t[1]);
  out->edge_height = d(C.edge_height);
  out->edge_vertices = p1(C.edge_vertices, keep.t[2]);
  out->inverse_dual = d(C.inverse_dual);
  out->vertex_edges = p1(C.vertex_edges, keep.t[3]);
  out->curl = d(C.curl);
  out->vertex_cells = p1(C.vertex_cells, keep.t[4]);
  out->vertex_height = d(C.vertex_height);
  out->coriolis = d(C.coriolis);
  out->trisk_edges = p1(C.trisk_edges, keep.t[5]);
  out->trisk = d(C.trisk);
  out->cell_areas = d(C.cell_areas);
  out->vertex_areas = d(C.vertex_areas);
  out->g_edges = p1(C.g_edges, keep.t[6]);
  out->g_pv_edges = p1(C.g_pv_edges, keep.t[7]);
  out->g_weights = d(C.g_weights);
  out->rhombus = d(C.rhombus);
  out->g_coriolis = d(C.g_coriolis);
  out->vk_cell_vertices = p1(C.vk_cell_vertices, keep.t[8]);
  out->vk_kites = d(C.vk_kites);
  out->vk_weights = d(C.vk_weights);
  out->vk_height = d(C.vk_height);
}

}  // namespace

extern "C" {

int trisk_model_create(const TriskGrid* grid, const TriskConfig* cfg, TriskModel** out) {
  TRISK_API_BEGIN
  if (!out || !cfg) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  Grid G = grid_from_abi(grid);
  if (!(cfg->alpha == cfg->alpha)) throw Error(TRISK_ERR_ARGUMENT, "kinetic_energy weight is NaN");
  Coefficients C = build_coefficients(G, cfg->pv_flux, cfg->alpha, cfg->gravity, cfg->omega,
                                      cfg->coriolis_vertices, cfg->coriolis_edges);
  auto m = std::make_unique<TriskModel>();
  m->device = cfg->device;
  std::vector<V3> centroids;
  if (cfg->reorder) {  // centroid of the cell's vertices, as hilbert_permutation takes it
    centroids.resize(G.nc);
    for (int64_t i = 0; i < G.nc; ++i) {
      V3 s{0, 0, 0};
      int n = 0;
      for (int k = 0; k < G.cw; ++k)
        if (G.cell_signs[i * G.cw + k] != 0.0) {
          s = s + G.vertices[G.cell_vertices[i * G.cw + k]];
          ++n;
        }
      centroids[i] = s / (double)n;
    }
  }
  finish_create(*m, C, cfg->reorder ? &centroids : nullptr, cfg);
  *out = m.release();
  TRISK_API_END
}

int trisk_model_create_from_coefficients(const TriskCoefficients* coefficients, const TriskConfig* cfg,
                                         TriskModel** out) {
  TRISK_API_BEGIN
  if (!out || !cfg) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  Coefficients C = coefficients_from_abi(coefficients);
  auto m = std::make_unique<TriskModel>();
  m->device = cfg->device;
  std::vector<V3> centroids;
  const bool reorder = cfg->reorder && cfg->cell_positions;
  if (reorder) {
    centroids.resize(C.nc);
    std::memcpy(centroids.data(), cfg->cell_positions, C.nc * sizeof(V3));
  }
  finish_create(*m, C, reorder ? &centroids : nullptr, cfg);
  *out = m.release();
  TRISK_API_END
}

void trisk_model_destroy(TriskModel* model) { delete model; }

int trisk_model_coefficients(TriskModel* model, TriskCoefficients* out) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!out) throw Error(TRISK_ERR_ARGUMENT, "out is NULL");
  export_coefficients(m.C, m.exported, out);
  TRISK_API_END
}

int trisk_tables_create(const TriskGrid* grid, const TriskConfig* cfg, TriskTables** out) {
  TRISK_API_BEGIN
  if (!out || !cfg) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  Grid G = grid_from_abi(grid);
  if (!(cfg->alpha == cfg->alpha)) throw Error(TRISK_ERR_ARGUMENT, "kinetic_energy weight is NaN");
  auto t = std::make_unique<TriskTables>();
  t->C = build_coefficients(G, cfg->pv_flux, cfg->alpha, cfg->gravity, cfg->omega, cfg->coriolis_vertices,
                            cfg->coriolis_edges);
  *out = t.release();
  TRISK_API_END
}

int trisk_tables_view(TriskTables* tables, TriskCoefficients* out) {
  TRISK_API_BEGIN
  if (!tables || !out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  export_coefficients(tables->C, tables->exported, out);
  TRISK_API_END
}

void trisk_tables_destroy(TriskTables* tables) { delete tables; }

int trisk_model_sizes(TriskModel* model, int64_t sizes[3]) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  sizes[0] = m.nc;
  sizes[1] = m.ne;
  sizes[2] = m.nv;
  TRISK_API_END
}

int trisk_tendency(TriskModel* model, const double* y, double* dy) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y || !dy) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  DeviceGuard guard(m.device);
  state_in(m, y, m.y);
  DevStage S{};
  S.u = m.y;
  S.h = m.y + m.ne;
  S.dy = m.dy;
  S.flag = m.flag;
  enqueue_tendency(m, S, EPI_TENDENCY);
  state_out(m, dy, m.dy);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int trisk_rk4_step_async(TriskModel* model, double* y, double dt, int64_t nsteps) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  if (nsteps < 0) throw Error(TRISK_ERR_ARGUMENT, "nsteps must be non-negative");
  if (!std::isfinite(dt)) throw Error(TRISK_ERR_ARGUMENT, "dt must be finite");
  DeviceGuard guard(m.device);
  if (!is_device_pointer(y)) throw Error(TRISK_ERR_ARGUMENT, "trisk_rk4_step_async needs a device state");
  if (nsteps == 0) return TRISK_OK;
  state_in(m, y, m.y);
  run_steps(m, dt, nsteps);
  state_out(m, y, m.y);
  TRISK_API_END
}

int trisk_rk4_step(TriskModel* model, double* y, double dt, int64_t nsteps) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  if (nsteps < 0) throw Error(TRISK_ERR_ARGUMENT, "nsteps must be non-negative");
  if (!std::isfinite(dt)) throw Error(TRISK_ERR_ARGUMENT, "dt must be finite");
  DeviceGuard guard(m.device);
  if (nsteps == 0) return TRISK_OK;
  state_in(m, y, m.y);
  run_steps(m, dt, nsteps);
  state_out(m, y, m.y);
  check_flag(m);
  TRISK_API_END
}

int trisk_synchronize(TriskModel* model) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  DeviceGuard guard(m.device);
  check_flag(m);
  TRISK_API_END
}

int trisk_diagnostics(TriskModel* model, const double* y, double* mass, double* energy, double* enstrophy) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  DeviceGuard guard(m.device);
  state_in(m, y, m.y);
  const double* u = m.y;
  const double* h = m.y + m.ne;
  if (mass) *mass = reduce<0>(m, m.area_c, h, nullptr, 0.0, m.nc);
  const int B = 128;
  const bool saved = m.use_pdl;
  m.use_pdl = false;
  try {
    if (energy) {  // kinetic_energy! then sum A h (K + g h / 2)   (TRiSKShallowWater.jl:406-411)
      with_modes(m.pv, m.ke, [&](auto pvc, auto kec) {
        constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
        launch(m, k_vertex<PV, KE, false>, cdiv(m.nv, B), B, nullptr, nullptr, m.T, m.W, u, h, 1, 0);
        launch(m, k_flux<PV, KE, false>, cdiv(m.nc, B), B, nullptr, nullptr, m.T, m.W, u, h, 1, 0, 1);
      });
      *energy = reduce<1>(m, m.area_c, h, m.W.K, m.gravity, m.nc);
    }
    if (enstrophy) {  // vertex_pv! then sum A_v h_v q_v^2 / 2   (:414-419)
      with_modes(m.pv, m.ke, [&](auto pvc, auto kec) {
        constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
        launch(m, k_vertex<PV, KE, false>, cdiv(m.nv, B), B, nullptr, nullptr, m.T, m.W, u, h, 1, 1);
      });
      *enstrophy = reduce<2>(m, m.area_v, m.W.hv, m.W.qv, 0.0, m.nv) / 2;
    }
  } catch (...) {
    m.use_pdl = saved;
    throw;
  }
  m.use_pdl = saved;
  TRISK_API_END
}

int trisk_relative_vorticity(TriskModel* model, const double* y, double* zeta) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y || !zeta) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  DeviceGuard guard(m.device);
  state_in(m, y, m.y);
  k_vertex_curl<<<(unsigned)cdiv(m.nv, 256), 256, 0, m.stream>>>(m.T, m.y, m.W.zv);
  CUDA_CHECK(cudaGetLastError());
  m.launches++;
  // zeta_file[v] = zeta_int[o2n[v]]
  gather(m, m.st, m.W.zv, m.vertex_o2n, m.nv);
  if (is_device_pointer(zeta)) {
    order_after_caller(m.stream, m.caller_ev);
    CUDA_CHECK(cudaMemcpyAsync(zeta, m.st, m.nv * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
  } else
    CUDA_CHECK(cudaMemcpyAsync(zeta, m.st, m.nv * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int trisk_model_stream(TriskModel* model, void** stream) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!stream) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *stream = (void*)m.stream;
  TRISK_API_END
}

int64_t trisk_launch_count(TriskModel* model) { return model ? model->launches : -1; }

int trisk_model_bytes(TriskModel* model, double out[4]) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  out[0] = m.phase_bytes[0];
  out[1] = m.phase_bytes[1];
  out[2] = m.phase_bytes[2];
  const double N = 8.0 * (double)m.N;
  out[3] = 4 * (m.table_bytes_unique + 2 * N) + 15 * N;
  TRISK_API_END
}

int trisk_model_info(TriskModel* model, int32_t* pv_mode, int32_t block[3], double* derived_saving) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (pv_mode) *pv_mode = m.pv;
  if (block)
    for (int p = 0; p < 3; ++p) block[p] = m.block[p];
  if (derived_saving) *derived_saving = m.pv_table_bytes_saved;
  TRISK_API_END
}

int trisk_autotune(TriskModel* model, double* y, double dt, int32_t steps, double* best_ms) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y || steps <= 0) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  DeviceGuard guard(m.device);
  if (!is_device_pointer(y)) throw Error(TRISK_ERR_ARGUMENT, "trisk_autotune needs a device state");
  // Times `steps` RK4 steps (graph + PDL as configured) for every combination of the three
  // phase block sizes, then for L2-resident table prefixes of several sizes with the best
  // blocks, then the blocks again with the best prefix, and for meshes that fit half the L2
  // the one-launch step, and keeps the fastest. Every candidate computes the same numbers;
  // the state is restored from the caller's copy before each trial. A persisting window, if
  // one was set, is left off.
  m.persistent = false;
  static const int choices[] = {64, 128, 256};
  static const int keep_mb[] = {0, 8, 16, 24, 32, 40, 48, 64};
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  int l2 = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, m.device));
  int best[3] = {m.block[0], m.block[1], m.block[2]};
  size_t best_keep = 0;
  double best_t = INFINITY;
  auto trial = [&](int a, int b, int c, size_t keep) {
    m.block[0] = a;
    m.block[1] = b;
    m.block[2] = c;
    m.l2_keep_bytes = keep;
    m.l2_window = false;
    m.T.keep_end = keep ? m.table_base + keep : nullptr;
    if (m.graph) {
      cudaGraphExecDestroy(m.graph);
      m.graph = nullptr;
    }
    state_in(m, y, m.y);
    run_steps(m, dt, 2);  // warm-up (and graph capture)
    CUDA_CHECK(cudaEventRecord(e0, m.stream));
    run_steps(m, dt, steps);
    CUDA_CHECK(cudaEventRecord(e1, m.stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_t) {
      best_t = ms;
      best[0] = a;
      best[1] = b;
      best[2] = c;
      best_keep = keep;
    }
  };
  auto blocks_pass = [&](size_t keep) {
    for (int a : choices)
      for (int b : choices)
        for (int c : choices) trial(a, b, c, keep);
  };
  try {
    blocks_pass(0);
    const int b0 = best[0], b1 = best[1], b2 = best[2];
    for (int mb : keep_mb) {
      const size_t keep = (size_t)mb << 20;
      if (mb == 0 || keep >= m.table_block_bytes || keep > (size_t)l2 / 2) continue;
      trial(b0, b1, b2, keep);
    }
    if (best_keep) blocks_pass(best_keep);
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    m.persistent = false;
    throw;
  }
  // the one-launch step, for meshes whose tables and state vectors fit half the L2
  bool use_persistent = false;
  const double footprint = (double)m.table_block_bytes + 8.0 * sizeof(double) * (m.N + m.nv);
  if (footprint <= l2 / 2) {
    try {
      const bool was = m.persistent;
      set_persistent(m, true);
      const double before = best_t;
      trial(best[0], best[1], best[2], best_keep);  // the blocks do not apply to it; best_t moves if faster
      use_persistent = best_t < before;
      m.persistent = was;
    } catch (const Error&) {
      m.persistent = false;  // no cooperative launch: keep the launches
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  m.persistent = use_persistent;
  for (int p = 0; p < 3; ++p) m.block[p] = best[p];
  m.l2_keep_bytes = best_keep;
  m.l2_window = false;
  m.T.keep_end = best_keep ? m.table_base + best_keep : nullptr;
  if (m.graph) {
    cudaGraphExecDestroy(m.graph);
    m.graph = nullptr;
  }
  CUDA_CHECK(cudaMemsetAsync(m.flag, 0, sizeof(int), m.stream));
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  if (best_ms) *best_ms = best_t / steps;
  TRISK_API_END
}

int trisk_model_get_l2_residency(TriskModel* model, int64_t* bytes, int32_t* window) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!bytes || !window) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *bytes = (int64_t)m.l2_keep_bytes;
  *window = m.l2_window ? 1 : 0;
  TRISK_API_END
}

int trisk_model_set_block(TriskModel* model, const int32_t block[3]) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!block) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int p = 0; p < 3; ++p)
    if (block[p] < 64 || block[p] > 256 || block[p] % 32)
      throw Error(TRISK_ERR_ARGUMENT, "block sizes must be multiples of 32 in [64, 256]");
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  for (int p = 0; p < 3; ++p) m.block[p] = block[p];
  if (m.graph) {  // recaptured with the new launch shapes at the next step
    cudaGraphExecDestroy(m.graph);
    m.graph = nullptr;
  }
  TRISK_API_END
}

int trisk_l2_info(int32_t device, int64_t info[4]) {
  TRISK_API_BEGIN
  if (!info) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    throw Error(TRISK_ERR_ARGUMENT, "no such CUDA device");
  }
  int l2 = 0, persist = 0, window = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
  CUDA_CHECK(cudaDeviceGetAttribute(&persist, cudaDevAttrMaxPersistingL2CacheSize, device));
  CUDA_CHECK(cudaDeviceGetAttribute(&window, cudaDevAttrMaxAccessPolicyWindowSize, device));
  size_t limit = 0;
  DeviceGuard guard(device);
  CUDA_CHECK(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
  info[0] = l2;
  info[1] = persist;
  info[2] = window;
  info[3] = (int64_t)limit;
  TRISK_API_END
}

int trisk_model_set_l2_residency(TriskModel* model, int64_t bytes, int32_t window) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (bytes < 0) throw Error(TRISK_ERR_ARGUMENT, "negative size");
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  size_t keep = std::min((size_t)bytes, m.table_block_bytes);
  bool win = window != 0 && keep > 0;
  if (win) {  // the persisting set-aside of this process's context (released with it)
    int persist = 0, wmax = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&persist, cudaDevAttrMaxPersistingL2CacheSize, m.device));
    CUDA_CHECK(cudaDeviceGetAttribute(&wmax, cudaDevAttrMaxAccessPolicyWindowSize, m.device));
    keep = std::min(keep, (size_t)std::min(persist, wmax));
    size_t limit = 0;
    CUDA_CHECK(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
    if (limit < keep) CUDA_CHECK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, keep));
  }
  m.l2_keep_bytes = keep;
  m.l2_window = win && keep > 0;
  m.T.keep_end = keep ? m.table_base + keep : nullptr;
  if (m.graph) {  // recaptured with the new table pointers and launch attributes
    cudaGraphExecDestroy(m.graph);
    m.graph = nullptr;
  }
  TRISK_API_END
}

int trisk_profile_phases(TriskModel* model, double* y, double dt, int64_t nsteps, double ms[3]) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!y || !ms || nsteps <= 0) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  DeviceGuard guard(m.device);
  if (!is_device_pointer(y)) throw Error(TRISK_ERR_ARGUMENT, "trisk_profile_phases needs a device state");
  cudaEvent_t ev[24];
  for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
  double acc[3] = {0, 0, 0};
  try {
    state_in(m, y, m.y);
    for (int64_t s = 0; s < nsteps; ++s) {
      enqueue_step(m, dt, ev);
      CUDA_CHECK(cudaStreamSynchronize(m.stream));
      for (int t = 0; t < 4; ++t)
        for (int p = 0; p < 3; ++p) {
          float f = 0;
          CUDA_CHECK(cudaEventElapsedTime(&f, ev[6 * t + 2 * p], ev[6 * t + 2 * p + 1]));
          acc[p] += f;
        }
    }
    state_out(m, y, m.y);
    CUDA_CHECK(cudaStreamSynchronize(m.stream));
  } catch (...) {
    for (auto& e : ev) cudaEventDestroy(e);
    throw;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int p = 0; p < 3; ++p) ms[p] = acc[p] / (4.0 * nsteps);
  TRISK_API_END
}

// ---- one rank's part of a distributed model ------------------------------------------
}  // extern "C"

struct TriskDist {
  std::unique_ptr<TriskModel> m;
  int64_t nsend = 0, nrecv = 0;
  int32_t* send_idx = nullptr;  // internal state indices of the sent owned entries (device)
  int32_t* recv_idx = nullptr;  // ... of the received ghost entries
  double* send_dev = nullptr;
  double* recv_dev = nullptr;
  double* send_host = nullptr;  // pinned, for TRISK_EXCHANGE_HOST
  double* recv_host = nullptr;
  TriskExchangeFn fn = nullptr;
  void* user = nullptr;
  int mode = TRISK_EXCHANGE_HOST;
  cudaGraphExec_t graph = nullptr;  // one RK4 step (TRISK_EXCHANGE_DEVICE_GRAPH)
  double graph_dt = NAN;
  int64_t graph_launches = 0;
  ~TriskDist() {
    if (!m) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(m->device);
    cudaStreamSynchronize(m->stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (send_host) cudaFreeHost(send_host);
    if (recv_host) cudaFreeHost(recv_host);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

namespace {

TriskDist* checked_dist(TriskDist* d) {
  if (!d || !d->m) throw Error(TRISK_ERR_ARGUMENT, "distributed model is NULL");
  return d;
}

// Ghost values of the state vector `base` (internal numbering) from their owners: pack the
// sent entries, the caller's exchange, unpack the received ones (exchange!, Halo.jl:80-99).
void dist_exchange(TriskDist& d, double* base) {
  TriskModel& m = *d.m;
  if (d.nsend == 0 && d.nrecv == 0) return;
  if (!d.fn) throw Error(TRISK_ERR_ARGUMENT, "the part has neighbours but no exchange function");
  if (d.nsend > 0) {
    k_gather<<<(unsigned)cdiv(d.nsend, 256), 256, 0, m.stream>>>(d.send_dev, base, d.send_idx, d.nsend);
    CUDA_CHECK(cudaGetLastError());
    m.launches++;
  }
  int status;
  if (d.mode == TRISK_EXCHANGE_HOST) {
    if (d.nsend > 0)
      CUDA_CHECK(cudaMemcpyAsync(d.send_host, d.send_dev, d.nsend * sizeof(double), cudaMemcpyDeviceToHost,
                                 m.stream));
    CUDA_CHECK(cudaStreamSynchronize(m.stream));
    status = d.fn(d.user, d.send_host, d.nsend, d.recv_host, d.nrecv, nullptr);
    if (status == TRISK_OK && d.nrecv > 0)
      CUDA_CHECK(cudaMemcpyAsync(d.recv_dev, d.recv_host, d.nrecv * sizeof(double), cudaMemcpyHostToDevice,
                                 m.stream));
  } else {
    status = d.fn(d.user, d.send_dev, d.nsend, d.recv_dev, d.nrecv, (void*)m.stream);
  }
  if (status != TRISK_OK) throw Error(status, "the exchange function failed");
  if (d.nrecv > 0) {
    k_scatter<<<(unsigned)cdiv(d.nrecv, 256), 256, 0, m.stream>>>(base, d.recv_dev, d.recv_idx, d.nrecv);
    CUDA_CHECK(cudaGetLastError());
    m.launches++;
  }
}

// One RK4 step of the part (RungeKutta.jl:18-29): every tendency exchanges its stage state
// first; the ghosts' tendencies are zero (k_tend), so their stage values stay the exchanged ones.
void dist_enqueue_step(TriskDist& d, double dt) {
  TriskModel& m = *d.m;
  DevStage S{};
  S.y = m.y;
  S.acc = m.acc;
  S.st = m.st;
  S.flag = m.flag;
  S.sixth = dt / 6;
  S.u = m.y;
  S.h = m.y + m.ne;
  S.c = dt / 2;
  dist_exchange(d, m.y);
  enqueue_tendency(m, S, EPI_STAGE1);
  S.u = m.st;
  S.h = m.st + m.ne;
  dist_exchange(d, m.st);
  enqueue_tendency(m, S, EPI_STAGE2);
  S.c = dt;
  dist_exchange(d, m.st);
  enqueue_tendency(m, S, EPI_STAGE3);
  dist_exchange(d, m.st);
  enqueue_tendency(m, S, EPI_STAGE4);
}

void dist_ensure_graph(TriskDist& d, double dt) {
  TriskModel& m = *d.m;
  if (d.graph && d.graph_dt == dt) return;
  if (d.graph) {
    cudaGraphExecDestroy(d.graph);
    d.graph = nullptr;
  }
  const int64_t before = m.launches;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(m.stream, cudaStreamCaptureModeThreadLocal));
  try {
    dist_enqueue_step(d, dt);
  } catch (...) {
    cudaStreamEndCapture(m.stream, &g);
    if (g) cudaGraphDestroy(g);
    m.launches = before;
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(m.stream, &g));
  d.graph_launches = m.launches - before;
  m.launches = before;
  cudaError_t e = cudaGraphInstantiate(&d.graph, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(e);
  d.graph_dt = dt;
}

// 1-based local state indices of one side of the halo -> internal indices (device)
int32_t* halo_indices(TriskModel& m, const int64_t* offsets, const int64_t* index, int32_t nnb, bool owned_side,
                      int64_t& count) {
  if (nnb > 0 && (!offsets || !index)) throw Error(TRISK_ERR_ARGUMENT, "halo lists are NULL");
  count = nnb > 0 ? offsets[nnb] : 0;
  if (nnb > 0 && offsets[0] != 0) throw Error(TRISK_ERR_ARGUMENT, "halo offsets must start at 0");
  for (int32_t k = 0; k < nnb; ++k)
    if (offsets[k + 1] < offsets[k]) throw Error(TRISK_ERR_ARGUMENT, "halo offsets must not decrease");
  std::vector<int32_t> out((size_t)std::max<int64_t>(count, 1));
  for (int64_t j = 0; j < count; ++j) {
    const int64_t x = index[j] - 1;
    if (x < 0 || x >= m.N) throw Error(TRISK_ERR_TABLE, "halo index out of range");
    const bool edge = x < m.ne;
    const int64_t local = edge ? x : x - m.ne;
    const bool is_owned = edge ? local < m.ne_own : local < m.nc_own;
    if (is_owned != owned_side)
      throw Error(TRISK_ERR_TABLE, owned_side ? "a sent halo entry is not owned" : "a received halo entry is owned");
    out[j] = edge ? m.edge_o2n[local] : (int32_t)(m.ne + m.cell_o2n[local]);
  }
  int32_t* dev = m.alloc<int32_t>(out.size());
  CUDA_CHECK(cudaMemcpy(dev, out.data(), out.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  return dev;
}

}  // namespace

extern "C" {

int trisk_dist_create(const TriskCoefficients* local, const TriskConfig* cfg, const TriskHalo* halo,
                      TriskDist** out) {
  TRISK_API_BEGIN
  if (!out || !cfg || !halo || !local) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  Coefficients C = coefficients_from_abi(local);
  if (halo->ne_owned < 0 || halo->ne_owned > C.ne || halo->nc_owned < 0 || halo->nc_owned > C.nc)
    throw Error(TRISK_ERR_ARGUMENT, "owned counts out of range");
  if (halo->nneighbors < 0) throw Error(TRISK_ERR_ARGUMENT, "negative neighbour count");
  auto d = std::make_unique<TriskDist>();
  d->m = std::make_unique<TriskModel>();
  TriskModel& m = *d->m;
  m.device = cfg->device;
  m.ne_own = halo->ne_owned;
  m.nc_own = halo->nc_owned;
  std::vector<V3> centroids;
  const bool reorder = cfg->reorder && cfg->cell_positions;
  if (reorder) {
    centroids.resize(C.nc);
    std::memcpy(centroids.data(), cfg->cell_positions, C.nc * sizeof(V3));
  }
  finish_create(m, C, reorder ? &centroids : nullptr, cfg);
  DeviceGuard guard(m.device);
  d->send_idx = halo_indices(m, halo->send_offsets, halo->send_index, halo->nneighbors, true, d->nsend);
  d->recv_idx = halo_indices(m, halo->recv_offsets, halo->recv_index, halo->nneighbors, false, d->nrecv);
  d->send_dev = m.alloc<double>(std::max<int64_t>(d->nsend, 1));
  d->recv_dev = m.alloc<double>(std::max<int64_t>(d->nrecv, 1));
  CUDA_CHECK(cudaMallocHost((void**)&d->send_host, std::max<int64_t>(d->nsend, 1) * sizeof(double)));
  CUDA_CHECK(cudaMallocHost((void**)&d->recv_host, std::max<int64_t>(d->nrecv, 1) * sizeof(double)));
  *out = d.release();
  TRISK_API_END
}

void trisk_dist_destroy(TriskDist* dist) { delete dist; }

int trisk_dist_set_exchange(TriskDist* dist, TriskExchangeFn fn, void* user, int32_t mode) {
  TRISK_API_BEGIN
  TriskDist& d = *checked_dist(dist);
  if (mode < TRISK_EXCHANGE_HOST || mode > TRISK_EXCHANGE_DEVICE_GRAPH)
    throw Error(TRISK_ERR_ARGUMENT, "unknown exchange mode");
  d.fn = fn;
  d.user = user;
  d.mode = mode;
  if (d.graph) {
    cudaGraphExecDestroy(d.graph);
    d.graph = nullptr;
  }
  TRISK_API_END
}

int trisk_dist_tendency(TriskDist* dist, const double* y, double* dy) {
  TRISK_API_BEGIN
  TriskDist& d = *checked_dist(dist);
  TriskModel& m = *d.m;
  if (!y || !dy) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  DeviceGuard guard(m.device);
  state_in(m, y, m.y);
  dist_exchange(d, m.y);
  DevStage S{};
  S.u = m.y;
  S.h = m.y + m.ne;
  S.dy = m.dy;
  S.flag = m.flag;
  enqueue_tendency(m, S, EPI_TENDENCY);
  state_out(m, dy, m.dy);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int trisk_dist_rk4_step(TriskDist* dist, double* y, double dt, int64_t nsteps) {
  TRISK_API_BEGIN
  TriskDist& d = *checked_dist(dist);
  TriskModel& m = *d.m;
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  if (nsteps < 0 || !std::isfinite(dt)) throw Error(TRISK_ERR_ARGUMENT, "bad dt or step count");
  DeviceGuard guard(m.device);
  if (nsteps == 0) return TRISK_OK;
  state_in(m, y, m.y);
  if (d.mode == TRISK_EXCHANGE_DEVICE_GRAPH) {
    dist_ensure_graph(d, dt);
    for (int64_t s = 0; s < nsteps; ++s) {
      CUDA_CHECK(cudaGraphLaunch(d.graph, m.stream));
      m.launches += d.graph_launches;
    }
  } else {
    for (int64_t s = 0; s < nsteps; ++s) dist_enqueue_step(d, dt);
  }
  state_out(m, y, m.y);
  check_flag(m);
  TRISK_API_END
}

int trisk_dist_stream(TriskDist* dist, void** stream) {
  TRISK_API_BEGIN
  TriskDist& d = *checked_dist(dist);
  if (!stream) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *stream = (void*)d.m->stream;
  TRISK_API_END
}

int64_t trisk_dist_launch_count(TriskDist* dist) { return dist && dist->m ? dist->m->launches : -1; }

int trisk_model_set_persistent(TriskModel* model, int32_t on) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  set_persistent(m, on != 0);
  TRISK_API_END
}

int trisk_model_get_persistent(TriskModel* model, int32_t* on) {
  TRISK_API_BEGIN
  TriskModel& m = *checked(model);
  if (!on) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *on = m.persistent ? 1 : 0;
  TRISK_API_END
}

}  // extern "C"
