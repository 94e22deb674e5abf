// Batched ensembles: many members, on meshes of several levels, advanced by one persistent
// launch per phase. A group is a set of members that share one model's tables (same mesh,
// same scheme); its state and work vectors are [entity][member], so the table entries a
// warp reads serve all the members it holds, and one gathered index reads the members'
// values as one contiguous run. The RK4 step of all groups (12 phase launches and a
// counter update) is one CUDA graph; each group has its own dt and step count, and a group
// that has taken its steps is skipped by later replays.
#include <algorithm>
#include <cstring>
#include <memory>

#include "model.hpp"

using namespace trisk;

namespace trisk {

constexpr int MAX_GROUPS = 8;

struct GroupDesc {
  DevTables T;
  DevWork W;
  double *y, *acc, *st;
  double dt;
  int M;       // members
  int nsteps;  // RK4 steps this group takes in a run
  int startV, nV;
  int startF, nEF, nCF;
  int startT, nET, nCT;
};

struct GroupSet {
  GroupDesc g[MAX_GROUPS];
  int n;
  int totalV, totalF, totalT;
  const int* counters;  // steps taken per group (device)
  int* flag;            // non-finite state seen
};

__device__ __forceinline__ int group_of(const GroupSet& G, int vb, int phase) {
  int gi = 0;
  for (int k = 1; k < G.n; ++k) {
    const int start = phase == 0 ? G.g[k].startV : (phase == 1 ? G.g[k].startF : G.g[k].startT);
    if (vb >= start) gi = k;
  }
  return gi;
}

template <int PV, int KE>
__global__ void __launch_bounds__(256) kg_vertex(const GroupSet G, int first_stage) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalV; vb += gridDim.x) {
    const int gi = group_of(G, vb, 0);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    const double* u = first_stage ? D.y : D.st;
    vertex_body<PV, KE, true>(D.T, D.W, u, u + (size_t)D.T.ne * D.M, D.M, 0, vb - D.startV);
  }
}

template <int PV, int KE>
__global__ void __launch_bounds__(256) kg_flux(const GroupSet G, int first_stage) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalF; vb += gridDim.x) {
    const int gi = group_of(G, vb, 1);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    const double* u = first_stage ? D.y : D.st;
    flux_body<PV, KE, true>(D.T, D.W, u, u + (size_t)D.T.ne * D.M, D.M, D.nEF, 0, vb - D.startF);
  }
}

template <int PV, int EPI>
__global__ void __launch_bounds__(256) kg_tend(const GroupSet G) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalT; vb += gridDim.x) {
    const int gi = group_of(G, vb, 2);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    DevStage S{};
    S.y = D.y;
    S.acc = D.acc;
    S.st = D.st;
    S.flag = G.flag;
    S.c = EPI == EPI_STAGE3 ? D.dt : D.dt / 2;
    S.sixth = D.dt / 6;
    tend_body<PV, EPI, true>(D.T, D.W, S, D.M, D.nET, vb - D.startT);
  }
}

__global__ void kg_advance(int* counters, int n) {
  if (threadIdx.x < n) counters[threadIdx.x] += 1;
}

// y_group[j M + m] = y_file[n2o[j]]  and back
__global__ void kg_scatter_member(double* dst, const double* src, const int32_t* n2o, int64_t N, int M, int m) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < N) dst[j * M + m] = src[n2o[j]];
}
__global__ void kg_gather_member(double* dst, const double* src, const int32_t* o2n, int64_t N, int M, int m) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < N) dst[j] = src[(int64_t)o2n[j] * M + m];
}

}  // namespace trisk

struct TriskEnsemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  int pv = 0, ke = 0;
  int block = 128;
  int grid[3] = {0, 0, 0};
  GroupSet G{};
  std::vector<TriskModel*> models;
  std::vector<void*> allocations;
  int* counters = nullptr;
  int* flag = nullptr;
  double* staging = nullptr;
  int64_t max_state = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t launches = 0;
  double step_bytes = 0;

  ~TriskEnsemble() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (void* p : allocations) cudaFree(p);
    if (prev >= 0) cudaSetDevice(prev);
  }
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocations.push_back(p);
    return static_cast<T*>(p);
  }
};

namespace {

template <class F>
void with_modes_e(int pv, int ke, F&& f) {
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

template <typename... KArgs, typename... Args>
void elaunch(TriskEnsemble& e, void (*kernel)(KArgs...), int grid, bool pdl, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)e.block);
  cfg.stream = e.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  e.launches++;
}

// One RK4 step of every unfinished group. The first phase of a step and the counter update
// wait for the full completion of the launch before them (no PDL): both depend on, or
// change, the step counters the others read.
void enqueue_ensemble_step(TriskEnsemble& e) {
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    for (int stage = 1; stage <= 4; ++stage) {
      elaunch(e, kg_vertex<PV, KE>, e.grid[0], stage != 1, e.G, stage == 1 ? 1 : 0);
      elaunch(e, kg_flux<PV, KE>, e.grid[1], true, e.G, stage == 1 ? 1 : 0);
      switch (stage) {
        case 1: elaunch(e, kg_tend<PV, EPI_STAGE1>, e.grid[2], true, e.G); break;
        case 2: elaunch(e, kg_tend<PV, EPI_STAGE2>, e.grid[2], true, e.G); break;
        case 3: elaunch(e, kg_tend<PV, EPI_STAGE3>, e.grid[2], true, e.G); break;
        default: elaunch(e, kg_tend<PV, EPI_STAGE4>, e.grid[2], true, e.G); break;
      }
    }
  });
  kg_advance<<<1, 32, 0, e.stream>>>(e.counters, e.G.n);
  CUDA_CHECK(cudaGetLastError());
  e.launches++;
}

void ensure_ensemble_graph(TriskEnsemble& e) {
  if (e.graph) return;
  const int64_t before = e.launches;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_ensemble_step(e);
  } catch (...) {
    cudaStreamEndCapture(e.stream, &g);
    if (g) cudaGraphDestroy(g);
    e.launches = before;
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(e.stream, &g));
  e.launches = before;
  cudaError_t err = cudaGraphInstantiate(&e.graph, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(err);
}

TriskEnsemble* checked_e(TriskEnsemble* e) {
  if (!e) throw Error(TRISK_ERR_ARGUMENT, "ensemble is NULL");
  return e;
}

const GroupDesc& group_at(TriskEnsemble& e, int g, int member) {
  if (g < 0 || g >= e.G.n) throw Error(TRISK_ERR_ARGUMENT, "group out of range");
  if (member < 0 || member >= e.G.g[g].M) throw Error(TRISK_ERR_ARGUMENT, "member out of range");
  return e.G.g[g];
}

}  // namespace

extern "C" {

int trisk_ensemble_create(TriskModel* const* models, const int32_t* members, const double* dt,
                          const int64_t* nsteps, int32_t ngroups, TriskEnsemble** out) {
  TRISK_API_BEGIN
  if (!models || !members || !dt || !nsteps || !out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (ngroups < 1 || ngroups > MAX_GROUPS)
    throw Error(TRISK_ERR_ARGUMENT, "an ensemble has 1.." + std::to_string(MAX_GROUPS) + " groups");
  auto e = std::make_unique<TriskEnsemble>();
  const TriskModel* m0 = models[0];
  if (!m0) throw Error(TRISK_ERR_ARGUMENT, "model is NULL");
  e->device = m0->device;
  e->pv = m0->pv;
  e->ke = m0->ke;
  DeviceGuard guard(e->device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  int sV = 0, sF = 0, sT = 0;
  const int B = e->block;
  for (int g = 0; g < ngroups; ++g) {
    TriskModel* m = models[g];
    if (!m) throw Error(TRISK_ERR_ARGUMENT, "model is NULL");
    if (m->device != e->device || m->pv != e->pv || m->ke != e->ke)
      throw Error(TRISK_ERR_ARGUMENT, "all groups need the same device and scheme");
    if (members[g] < 1) throw Error(TRISK_ERR_ARGUMENT, "a group needs at least one member");
    if (!(dt[g] > 0) || !std::isfinite(dt[g]) || nsteps[g] < 0 || nsteps[g] > (1LL << 30))
      throw Error(TRISK_ERR_ARGUMENT, "bad dt or step count");
    const int64_t M = members[g];
    if ((m->ne + m->nc) * M >= (1LL << 31)) throw Error(TRISK_ERR_UNSUPPORTED, "group too large");
    GroupDesc& D = e->G.g[g];
    D.T = m->T;
    D.M = (int)M;
    D.dt = dt[g];
    D.nsteps = (int)nsteps[g];
    D.W.K = e->alloc<double>(m->nc * M);
    D.W.B = e->alloc<double>(m->nc * M);
    D.W.F = e->alloc<double>(m->ne * M);
    D.W.qe = e->alloc<double>(m->ne * M);
    D.W.zv = e->alloc<double>(m->nv * M);
    D.W.hv = e->alloc<double>(m->nv * M);
    D.W.qv = e->alloc<double>(m->nv * M);
    D.W.Kv = e->alloc<double>(m->nv * M);
    D.y = e->alloc<double>(m->N * M);
    D.acc = e->alloc<double>(m->N * M);
    D.st = e->alloc<double>(m->N * M);
    CUDA_CHECK(cudaMemset(D.y, 0, m->N * M * sizeof(double)));
    D.nV = (int)cdiv(m->nv * M, B);
    D.nEF = D.nET = (int)cdiv(m->ne * M, B);
    D.nCF = D.nCT = (int)cdiv(m->nc * M, B);
    D.startV = sV;
    D.startF = sF;
    D.startT = sT;
    sV += D.nV;
    sF += D.nEF + D.nCF;
    sT += D.nET + D.nCT;
    e->models.push_back(m);
    e->max_state = std::max(e->max_state, m->N);
    const double Nb = 8.0 * (double)m->N * M;
    e->step_bytes += 4 * (m->table_bytes_unique + 2 * Nb) + 15 * Nb;
  }
  e->G.n = ngroups;
  e->G.totalV = sV;
  e->G.totalF = sF;
  e->G.totalT = sT;
  e->counters = e->alloc<int>(MAX_GROUPS);
  e->flag = e->alloc<int>(1);
  e->staging = e->alloc<double>(e->max_state);
  CUDA_CHECK(cudaMemset(e->counters, 0, MAX_GROUPS * sizeof(int)));
  CUDA_CHECK(cudaMemset(e->flag, 0, sizeof(int)));
  e->G.counters = e->counters;
  e->G.flag = e->flag;
  // persistent grids: as many blocks as stay resident, never more than the work
  int dev_sms = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, e->device));
  int occ[3] = {1, 1, 1};
  with_modes_e(e->pv, e->ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], kg_vertex<PV, KE>, B, 0));
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], kg_flux<PV, KE>, B, 0));
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], kg_tend<PV, EPI_STAGE2>, B, 0));
  });
  const int total[3] = {sV, sF, sT};
  for (int p = 0; p < 3; ++p) e->grid[p] = std::max(1, std::min(total[p], dev_sms * std::max(occ[p], 1)));
  CUDA_CHECK(cudaDeviceSynchronize());
  *out = e.release();
  TRISK_API_END
}

void trisk_ensemble_destroy(TriskEnsemble* e) { delete e; }

int trisk_ensemble_set_member(TriskEnsemble* ens, int32_t group, int32_t member, const double* y) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  const GroupDesc& D = group_at(e, group, member);
  TriskModel& m = *e.models[group];
  DeviceGuard guard(e.device);
  const double* src = y;
  if (!is_device_pointer(y)) {
    CUDA_CHECK(cudaMemcpyAsync(e.staging, y, m.N * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    src = e.staging;
  }
  kg_scatter_member<<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(D.y, src, m.state_n2o, m.N, D.M, member);
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

int trisk_ensemble_get_member(TriskEnsemble* ens, int32_t group, int32_t member, double* y) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  const GroupDesc& D = group_at(e, group, member);
  TriskModel& m = *e.models[group];
  DeviceGuard guard(e.device);
  const bool dev = is_device_pointer(y);
  double* dst = dev ? y : e.staging;
  kg_gather_member<<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(dst, D.y, m.state_o2n, m.N, D.M, member);
  CUDA_CHECK(cudaGetLastError());
  if (!dev) CUDA_CHECK(cudaMemcpyAsync(y, e.staging, m.N * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

int trisk_ensemble_run_async(TriskEnsemble* ens, int64_t steps) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (steps < 0) throw Error(TRISK_ERR_ARGUMENT, "steps must be non-negative");
  DeviceGuard guard(e.device);
  ensure_ensemble_graph(e);
  for (int64_t s = 0; s < steps; ++s) {
    CUDA_CHECK(cudaGraphLaunch(e.graph, e.stream));
    e.launches += 13;
  }
  TRISK_API_END
}

int trisk_ensemble_synchronize(TriskEnsemble* ens) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  DeviceGuard guard(e.device);
  int flag = 0;
  CUDA_CHECK(cudaMemcpyAsync(&flag, e.flag, sizeof(int), cudaMemcpyDeviceToHost, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  if (flag) {
    CUDA_CHECK(cudaMemset(e.flag, 0, sizeof(int)));
    throw Error(TRISK_ERR_NONFINITE, "a member's state became non-finite");
  }
  TRISK_API_END
}

int trisk_ensemble_steps(TriskEnsemble* ens, int64_t* steps_taken) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!steps_taken) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  DeviceGuard guard(e.device);
  int c[MAX_GROUPS] = {0};
  CUDA_CHECK(cudaMemcpyAsync(c, e.counters, sizeof(c), cudaMemcpyDeviceToHost, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  for (int g = 0; g < e.G.n; ++g) steps_taken[g] = std::min<int64_t>(c[g], e.G.g[g].nsteps);
  TRISK_API_END
}

int trisk_ensemble_reset(TriskEnsemble* ens) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaMemsetAsync(e.counters, 0, MAX_GROUPS * sizeof(int), e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

int trisk_ensemble_stream(TriskEnsemble* ens, void** stream) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!stream) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *stream = (void*)e.stream;
  TRISK_API_END
}

int64_t trisk_ensemble_launch_count(TriskEnsemble* ens) { return ens ? ens->launches : -1; }

int trisk_ensemble_bytes(TriskEnsemble* ens, double* step_bytes) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!step_bytes) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *step_bytes = e.step_bytes;
  TRISK_API_END
}

}  // extern "C"
