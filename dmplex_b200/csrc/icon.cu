// ICON triangle shallow water (dmplex.jl's ICONShallowWater, src/FiniteVolumes/
// ICONShallowWater.jl): normal velocities at the edges, heights at the triangles'
// circumcenters, vorticity at the vertices. Tables arrive 1-based and (entity, k) ordered, as
// Julia holds them, and are uploaded once as 0-based int32 / FP64 structure-of-arrays
// [k][entity] padded to multiples of 32 (file numbering is kept). One tendency is three
// phase launches (four more with divergence damping); the RK4 stage update is fused into
// the last, as for TRiSK, and the sums keep the reference's order, so results match the
// CPU restatement bit for bit.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "model.hpp"

using namespace trisk;

namespace {

constexpr int ICW = 3;   // edges per triangle
constexpr int IRW = 4;   // RBF stencil
constexpr int IVW = 6;   // edges per vertex (5 at the pentagon points, padded)

struct IconTables {
  int32_t nc, ne, nv, ldc, lde, ldv;
  double gravity;
  const int32_t* cell_edges;     // ICW x ldc
  const double* divergence;      // ICW x ldc
  const double* bilinear;        // ICW x ldc
  const int32_t* edge_cells;     // 2 x lde
  const int32_t* edge_vertices;  // 2 x lde
  const double* edge_height;     // 2 x lde
  const double* gradient;        // 2 x lde
  const double* inverse_dual;    // lde
  const int32_t* rbf_edges;      // IRW x lde
  const double* rbf;             // IRW x lde
  const double* edge_coriolis;   // lde
  const double* damping;         // lde (nullptr: no divergence damping)
  const int32_t* vertex_edges;   // IVW x ldv
  const double* curl;            // IVW x ldv
};

// gh: g (h_r - h_l) / d_e of the stage state, computed in phase 1 so that the fused
// tendency phase, whose cell threads overwrite the stage state with the next one, never
// reads heights.
struct IconWork {
  double *v, *Ke, *F, *K, *zv, *D, *G, *gh;
};

// phase 1, edges (icon_edge_kernel!, ICONShallowWater.jl:149-159): RBF tangential velocity,
// edge kinetic energy, mass flux
__global__ void __launch_bounds__(256) k_icon_edge(IconTables T, IconWork W, const double* u, const double* h) {
  pdl_trigger();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T.ne) return;
  int re[IRW];
  double rw[IRW];
#pragma unroll
  for (int k = 0; k < IRW; ++k) {
    re[k] = __ldcs(T.rbf_edges + k * T.lde + e);
    rw[k] = __ldcs(T.rbf + k * T.lde + e);
  }
  const int c0 = __ldcs(T.edge_cells + e), c1 = __ldcs(T.edge_cells + T.lde + e);
  const double eh0 = __ldcs(T.edge_height + e), eh1 = __ldcs(T.edge_height + T.lde + e);
  const double invd = __ldcs(T.inverse_dual + e);
  pdl_wait();
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < IRW; ++k) s += rw[k] * u[re[k]];
  const double ue = u[e];
  const double hl = h[c0], hr = h[c1];
  W.v[e] = s;
  W.Ke[e] = (ue * ue + s * s) / 2;
  W.F[e] = (eh0 * hl + eh1 * hr) * ue;
  W.gh[e] = T.gravity * (hr - hl) * invd;
}

// phase 2: cells K = sum bilinear Ke (edge_sum_kernel!, :305-312; kinetic_energy!, :184-189)
// and, with damping, D = -sum div u (continuity_kernel!); vertices zeta = sum curl u.
// Blocks [0, nbC) take cells, the rest vertices.
__global__ void __launch_bounds__(256) k_icon_cellvert(IconTables T, IconWork W, const double* u, int nbC) {
  pdl_trigger();
  if ((int)blockIdx.x < nbC) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.nc) return;
    int ce[ICW];
    double bl[ICW], dv[ICW];
#pragma unroll
    for (int k = 0; k < ICW; ++k) {
      ce[k] = __ldcs(T.cell_edges + k * T.ldc + i);
      bl[k] = __ldcs(T.bilinear + k * T.ldc + i);
      if (T.damping) dv[k] = __ldcs(T.divergence + k * T.ldc + i);
    }
    pdl_wait();
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < ICW; ++k) s += bl[k] * W.Ke[ce[k]];
    W.K[i] = s;
    if (T.damping) {
      double d = 0.0;
#pragma unroll
      for (int k = 0; k < ICW; ++k) d += dv[k] * u[ce[k]];
      W.D[i] = -d;
    }
  } else {
    const int v = (blockIdx.x - nbC) * blockDim.x + threadIdx.x;
    if (v >= T.nv) return;
    int ve[IVW];
    double cu[IVW];
#pragma unroll
    for (int k = 0; k < IVW; ++k) {
      ve[k] = __ldcs(T.vertex_edges + k * T.ldv + v);
      cu[k] = __ldcs(T.curl + k * T.ldv + v);
    }
    pdl_wait();
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < IVW; ++k) s += cu[k] * u[ve[k]];
    W.zv[v] = s;
  }
}

// divergence damping (divergence_damping!, :210-218): G = scale (D_r - D_l) / d at the edges
// (edge_gradient_kernel!, :173-176) ...
__global__ void __launch_bounds__(256) k_icon_gradient(IconTables T, const double* D, double* G, double scale) {
  pdl_trigger();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T.ne) return;
  const int c0 = __ldcs(T.edge_cells + e), c1 = __ldcs(T.edge_cells + T.lde + e);
  const double invd = __ldcs(T.inverse_dual + e);
  pdl_wait();
  G[e] = scale * (D[c1] - D[c0]) * invd;
}

// ... and D = -sum div G at the cells (continuity_kernel!)
__global__ void __launch_bounds__(256) k_icon_divergence(IconTables T, const double* G, double* D) {
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.nc) return;
  int ce[ICW];
  double dv[ICW];
#pragma unroll
  for (int k = 0; k < ICW; ++k) {
    ce[k] = __ldcs(T.cell_edges + k * T.ldc + i);
    dv[k] = __ldcs(T.divergence + k * T.ldc + i);
  }
  pdl_wait();
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < ICW; ++k) s += dv[k] * G[ce[k]];
  D[i] = -s;
}

// phase 3: edges du (icon_momentum_kernel!, :161-171, plus nu (-(D2_r - D2_l) / d) with
// damping), cells dh = -sum div F (continuity_kernel!); then the RK4 stage update
template <int EPI>
__global__ void __launch_bounds__(256) k_icon_tend(IconTables T, IconWork W, DevStage S, int nbE) {
  pdl_trigger();
  if ((int)blockIdx.x < nbE) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T.ne) return;
    const int l = __ldcs(T.edge_cells + e), r = __ldcs(T.edge_cells + T.lde + e);
    const int v0 = __ldcs(T.edge_vertices + e), v1 = __ldcs(T.edge_vertices + T.lde + e);
    const double g0 = __ldcs(T.gradient + e), g1 = __ldcs(T.gradient + T.lde + e);
    const double invd = __ldcs(T.inverse_dual + e), f = __ldcs(T.edge_coriolis + e);
    const double nu = T.damping ? __ldcs(T.damping + e) : 0.0;
    pdl_wait();
    const double zeta = (W.zv[v0] + W.zv[v1]) / 2;
    const double Ke = W.Ke[e];
    const double gradK = Ke * (g0 - g1) + g1 * W.K[r] - g0 * W.K[l];
    double du = (f + zeta) * W.v[e] - gradK - W.gh[e];
    if (T.damping) du = du + nu * (-(W.D[r] - W.D[l]) * invd);
    epilogue<EPI>(S, (size_t)e, du);
  } else {
    const int i = (blockIdx.x - nbE) * blockDim.x + threadIdx.x;
    if (i >= T.nc) return;
    int ce[ICW];
    double dv[ICW];
#pragma unroll
    for (int k = 0; k < ICW; ++k) {
      ce[k] = __ldcs(T.cell_edges + k * T.ldc + i);
      dv[k] = __ldcs(T.divergence + k * T.ldc + i);
    }
    pdl_wait();
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < ICW; ++k) s += dv[k] * W.F[ce[k]];
    epilogue<EPI>(S, (size_t)T.ne + i, -s);
  }
}

}  // namespace

struct TriskIconModel {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t caller_ev = nullptr;
  int64_t nc = 0, ne = 0, nv = 0, N = 0;
  IconTables T{};
  IconWork W{};
  double *y = nullptr, *acc = nullptr, *st = nullptr, *dy = nullptr;
  int* flag = nullptr;
  std::vector<void*> allocations;
  int64_t launches = 0;
  cudaGraphExec_t graph = nullptr;  // one RK4 step at graph_dt
  double graph_dt = 0.0;
  int64_t graph_launches = 0;       // kernels in the graph

  ~TriskIconModel() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    if (caller_ev) cudaEventDestroy(caller_ev);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (void* p : allocations) cudaFree(p);
    if (prev >= 0) cudaSetDevice(prev);
  }
  template <class X>
  X* alloc(size_t count) {
    void* p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(X)));
    allocations.push_back(p);
    return static_cast<X*>(p);
  }
};

namespace {

constexpr int IB = 128;

template <typename... KArgs, typename... Args>
void ilaunch(TriskIconModel& m, void (*kernel)(KArgs...), int64_t grid, bool pdl, Args&&... args) {
  if (grid <= 0) return;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(IB);
  cfg.stream = m.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  m.launches++;
}

void icon_tendency(TriskIconModel& m, const DevStage& S, int epi) {
  const int64_t nbE = cdiv(m.ne, IB), nbC = cdiv(m.nc, IB), nbV = cdiv(m.nv, IB);
  ilaunch(m, k_icon_edge, nbE, false, m.T, m.W, S.u, S.h);
  ilaunch(m, k_icon_cellvert, nbC + nbV, true, m.T, m.W, S.u, (int)nbC);
  if (m.T.damping) {
    ilaunch(m, k_icon_gradient, nbE, true, m.T, (const double*)m.W.D, m.W.G, 1.0);
    ilaunch(m, k_icon_divergence, nbC, true, m.T, (const double*)m.W.G, m.W.D);
  }
  const int64_t g = nbE + nbC;
  switch (epi) {
    case EPI_TENDENCY: ilaunch(m, k_icon_tend<EPI_TENDENCY>, g, true, m.T, m.W, S, (int)nbE); break;
    case EPI_STAGE1: ilaunch(m, k_icon_tend<EPI_STAGE1>, g, true, m.T, m.W, S, (int)nbE); break;
    case EPI_STAGE2: ilaunch(m, k_icon_tend<EPI_STAGE2>, g, true, m.T, m.W, S, (int)nbE); break;
    case EPI_STAGE3: ilaunch(m, k_icon_tend<EPI_STAGE3>, g, true, m.T, m.W, S, (int)nbE); break;
    default: ilaunch(m, k_icon_tend<EPI_STAGE4>, g, true, m.T, m.W, S, (int)nbE); break;
  }
}

// One RK4 step on the internal state m.y (RungeKutta.jl:18-29), the stage updates fused into
// the last phase of every tendency.
void icon_enqueue_step(TriskIconModel& m, double dt) {
  DevStage S{};
  S.y = m.y;
  S.acc = m.acc;
  S.st = m.st;
  S.flag = m.flag;
  S.sixth = dt / 6;
  S.u = m.y;
  S.h = m.y + m.ne;
  S.c = dt / 2;
  icon_tendency(m, S, EPI_STAGE1);
  S.u = m.st;
  S.h = m.st + m.ne;
  icon_tendency(m, S, EPI_STAGE2);
  S.c = dt;
  icon_tendency(m, S, EPI_STAGE3);
  icon_tendency(m, S, EPI_STAGE4);
}

// The step's 12 launches (20 with divergence damping) as one CUDA graph, captured again when
// dt changes; replayed once per step.
void icon_ensure_graph(TriskIconModel& m, double dt) {
  if (m.graph && m.graph_dt == dt) return;
  if (m.graph) {
    cudaGraphExecDestroy(m.graph);
    m.graph = nullptr;
  }
  const int64_t before = m.launches;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(m.stream, cudaStreamCaptureModeThreadLocal));
  try {
    icon_enqueue_step(m, dt);
  } catch (...) {
    cudaStreamEndCapture(m.stream, &g);
    if (g) cudaGraphDestroy(g);
    m.launches = before;
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(m.stream, &g));
  m.graph_launches = m.launches - before;
  m.launches = before;  // captured launches are counted when the graph is replayed
  cudaError_t e = cudaGraphInstantiate(&m.graph, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(e);
  m.graph_dt = dt;
}

TriskIconModel* checked_icon(TriskIconModel* m) {
  if (!m) throw Error(TRISK_ERR_ARGUMENT, "model is NULL");
  return m;
}

// 1-based (entity, k) int64 table -> 0-based int32 [k][entity], indices checked
void put_index(std::vector<int32_t>& out, const int64_t* tab, int w, int wpad, int64_t n, int64_t ld,
               int64_t range, const char* name) {
  if (!tab) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
  out.assign((size_t)wpad * ld, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int k = 0; k < w; ++k) {
      const int64_t x = tab[j * w + k];
      if (x < 1 || x > range) throw Error(TRISK_ERR_TABLE, std::string(name) + ": index out of range");
      out[k * ld + j] = (int32_t)(x - 1);
    }
}

void put_weight(std::vector<double>& out, const double* tab, int w, int wpad, int64_t n, int64_t ld,
                const char* name) {
  if (!tab) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
  out.assign((size_t)wpad * ld, 0.0);
  for (int64_t j = 0; j < n; ++j)
    for (int k = 0; k < w; ++k) out[k * ld + j] = tab[j * w + k];
}

template <class X>
const X* upload(TriskIconModel& m, const std::vector<X>& v) {
  X* d = m.alloc<X>(v.size());
  CUDA_CHECK(cudaMemcpy(d, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
  return d;
}

void icon_state_in(TriskIconModel& m, const double* y_user, double* dst) {
  const size_t bytes = (size_t)m.N * sizeof(double);
  if (is_device_pointer(y_user)) {
    order_after_caller(m.stream, m.caller_ev);
    CUDA_CHECK(cudaMemcpyAsync(dst, y_user, bytes, cudaMemcpyDeviceToDevice, m.stream));
  } else {
    CUDA_CHECK(cudaMemcpyAsync(dst, y_user, bytes, cudaMemcpyHostToDevice, m.stream));
  }
}

void icon_state_out(TriskIconModel& m, double* y_user, const double* src) {
  const size_t bytes = (size_t)m.N * sizeof(double);
  if (is_device_pointer(y_user)) {
    order_after_caller(m.stream, m.caller_ev);
    CUDA_CHECK(cudaMemcpyAsync(y_user, src, bytes, cudaMemcpyDeviceToDevice, m.stream));
  } else {
    CUDA_CHECK(cudaMemcpyAsync(y_user, src, bytes, cudaMemcpyDeviceToHost, m.stream));
  }
}

void icon_check_flag(TriskIconModel& m) {
  int flag = 0;
  CUDA_CHECK(cudaMemcpyAsync(&flag, m.flag, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  if (flag) {
    CUDA_CHECK(cudaMemset(m.flag, 0, sizeof(int)));
    throw Error(TRISK_ERR_NONFINITE, "the state became non-finite");
  }
}

}  // namespace

extern "C" {

int trisk_icon_create(const TriskIconTables* t, int32_t device, TriskIconModel** out) {
  TRISK_API_BEGIN
  if (!t || !out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (t->nc < 1 || t->ne < 1 || t->nv < 1 || t->vw < 1 || t->vw > IVW)
    throw Error(TRISK_ERR_ARGUMENT, "bad sizes (vertices have at most 6 edges)");
  if (t->nc >= (1LL << 30) || t->ne >= (1LL << 30)) throw Error(TRISK_ERR_UNSUPPORTED, "mesh too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw Error(TRISK_ERR_CUDA, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) throw Error(TRISK_ERR_ARGUMENT, "no such CUDA device");
  auto m = std::make_unique<TriskIconModel>();
  m->device = device;
  DeviceGuard guard(device);
  m->nc = t->nc;
  m->ne = t->ne;
  m->nv = t->nv;
  m->N = t->nc + t->ne;
  const int64_t ldc = round_up(t->nc, 32), lde = round_up(t->ne, 32), ldv = round_up(t->nv, 32);
  std::vector<int32_t> iv;
  std::vector<double> wv;
  IconTables& T = m->T;
  T.nc = (int32_t)t->nc;
  T.ne = (int32_t)t->ne;
  T.nv = (int32_t)t->nv;
  T.ldc = (int32_t)ldc;
  T.lde = (int32_t)lde;
  T.ldv = (int32_t)ldv;
  T.gravity = t->gravity;
  put_index(iv, t->cell_edges, ICW, ICW, t->nc, ldc, t->ne, "cell_edges");
  T.cell_edges = upload(*m, iv);
  put_weight(wv, t->divergence, ICW, ICW, t->nc, ldc, "divergence");
  T.divergence = upload(*m, wv);
  put_weight(wv, t->bilinear, ICW, ICW, t->nc, ldc, "bilinear");
  T.bilinear = upload(*m, wv);
  put_index(iv, t->edge_cells, 2, 2, t->ne, lde, t->nc, "edge_cells");
  T.edge_cells = upload(*m, iv);
  put_index(iv, t->edge_vertices, 2, 2, t->ne, lde, t->nv, "edge_vertices");
  T.edge_vertices = upload(*m, iv);
  put_weight(wv, t->edge_height, 2, 2, t->ne, lde, "edge_height");
  T.edge_height = upload(*m, wv);
  put_weight(wv, t->gradient, 2, 2, t->ne, lde, "gradient");
  T.gradient = upload(*m, wv);
  put_weight(wv, t->inverse_dual, 1, 1, t->ne, lde, "inverse_dual");
  T.inverse_dual = upload(*m, wv);
  put_index(iv, t->rbf_edges, IRW, IRW, t->ne, lde, t->ne, "rbf_edges");
  T.rbf_edges = upload(*m, iv);
  put_weight(wv, t->rbf, IRW, IRW, t->ne, lde, "rbf");
  T.rbf = upload(*m, wv);
  put_weight(wv, t->edge_coriolis, 1, 1, t->ne, lde, "edge_coriolis");
  T.edge_coriolis = upload(*m, wv);
  T.damping = nullptr;
  if (t->divergence_damping) {
    put_weight(wv, t->divergence_damping, 1, 1, t->ne, lde, "divergence_damping");
    T.damping = upload(*m, wv);
  }
  put_index(iv, t->vertex_edges, t->vw, IVW, t->nv, ldv, t->ne, "vertex_edges");
  T.vertex_edges = upload(*m, iv);
  put_weight(wv, t->curl, t->vw, IVW, t->nv, ldv, "curl");
  T.curl = upload(*m, wv);
  IconWork& W = m->W;
  W.v = m->alloc<double>(t->ne);
  W.Ke = m->alloc<double>(t->ne);
  W.F = m->alloc<double>(t->ne);
  W.G = m->alloc<double>(t->ne);
  W.gh = m->alloc<double>(t->ne);
  W.K = m->alloc<double>(t->nc);
  W.D = m->alloc<double>(t->nc);
  W.zv = m->alloc<double>(t->nv);
  m->y = m->alloc<double>(m->N);
  m->acc = m->alloc<double>(m->N);
  m->st = m->alloc<double>(m->N);
  m->dy = m->alloc<double>(m->N);
  m->flag = m->alloc<int>(1);
  CUDA_CHECK(cudaMemset(m->flag, 0, sizeof(int)));
  CUDA_CHECK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreateWithFlags(&m->caller_ev, cudaEventDisableTiming));
  CUDA_CHECK(cudaDeviceSynchronize());
  *out = m.release();
  TRISK_API_END
}

void trisk_icon_destroy(TriskIconModel* m) { delete m; }

int trisk_icon_tendency(TriskIconModel* model, const double* y, double* dy) {
  TRISK_API_BEGIN
  TriskIconModel& m = *checked_icon(model);
  if (!y || !dy) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  DeviceGuard guard(m.device);
  icon_state_in(m, y, m.y);
  DevStage S{};
  S.u = m.y;
  S.h = m.y + m.ne;
  S.dy = m.dy;
  S.flag = m.flag;
  icon_tendency(m, S, EPI_TENDENCY);
  icon_state_out(m, dy, m.dy);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int trisk_icon_rk4_step(TriskIconModel* model, double* y, double dt, int64_t nsteps) {
  TRISK_API_BEGIN
  TriskIconModel& m = *checked_icon(model);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  if (nsteps < 0 || !std::isfinite(dt)) throw Error(TRISK_ERR_ARGUMENT, "bad dt or step count");
  DeviceGuard guard(m.device);
  icon_state_in(m, y, m.y);
  if (nsteps > 0) icon_ensure_graph(m, dt);
  for (int64_t s = 0; s < nsteps; ++s) {
    CUDA_CHECK(cudaGraphLaunch(m.graph, m.stream));
    m.launches += m.graph_launches;
  }
  icon_state_out(m, y, m.y);
  icon_check_flag(m);
  TRISK_API_END
}

int64_t trisk_icon_launch_count(TriskIconModel* model) { return model ? model->launches : -1; }

}  // extern "C"
