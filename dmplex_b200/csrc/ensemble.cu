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

#include <cuda_bf16.h>

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
  int P;  // members per thread in the three phases (2 when M is even, else 1)
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

// The group descriptors keep every buffer as double*; an FP32-state ensemble (R = float)
// reinterprets them, its buffers having been allocated with 4-byte elements.
template <class R>
__device__ __forceinline__ const R* as_r(const double* p) {
  return reinterpret_cast<const R*>(p);
}
template <class R>
__device__ __forceinline__ R* as_r(double* p) {
  return reinterpret_cast<R*>(p);
}

template <int PV, int KE, class R>
__global__ void __launch_bounds__(256) kg_vertex(const GroupSet G, int first_stage) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalV; vb += gridDim.x) {
    const int gi = group_of(G, vb, 0);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    const R* u = as_r<R>(first_stage ? D.y : D.st);
    if (D.P == 2)
      vertex_body<PV, KE, true, R, false, 2>(D.T, work_as<R>(D.W), u, u + (size_t)D.T.ne * D.M, D.M, 0,
                                             vb - D.startV);
    else
      vertex_body<PV, KE, true, R>(D.T, work_as<R>(D.W), u, u + (size_t)D.T.ne * D.M, D.M, 0, vb - D.startV);
  }
}

template <int PV, int KE, class R>
__global__ void __launch_bounds__(256) kg_flux(const GroupSet G, int first_stage, int want_K) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalF; vb += gridDim.x) {
    const int gi = group_of(G, vb, 1);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    const R* u = as_r<R>(first_stage ? D.y : D.st);
    if (D.P == 2)
      flux_body<PV, KE, true, R, false, 2>(D.T, work_as<R>(D.W), u, u + (size_t)D.T.ne * D.M, D.M, D.nEF, want_K,
                                           vb - D.startF);
    else
      flux_body<PV, KE, true, R>(D.T, work_as<R>(D.W), u, u + (size_t)D.T.ne * D.M, D.M, D.nEF, want_K,
                                 vb - D.startF);
  }
}

template <int PV, int EPI, class R>
__global__ void __launch_bounds__(256, 4) kg_tend(const GroupSet G) {  // <= 64 registers: 8 blocks of 128
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalT; vb += gridDim.x) {
    const int gi = group_of(G, vb, 2);
    const GroupDesc& D = G.g[gi];
    if (G.counters[gi] >= D.nsteps) continue;
    DevStageT<R> S{};
    S.y = as_r<R>(D.y);
    S.acc = as_r<R>(D.acc);
    S.st = as_r<R>(D.st);
    S.flag = G.flag;
    S.c = EPI == EPI_STAGE3 ? D.dt : D.dt / 2;
    S.sixth = D.dt / 6;
    if (D.P == 2) {
      if (D.W.dq)
        tend_body_p<PV, EPI, true, R, 2>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
      else
        tend_body_p<PV, EPI, false, R, 2>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
    } else if (D.W.dq) {
      tend_body<PV, EPI, true, true, R>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
    } else {
      tend_body<PV, EPI, true, false, R>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
    }
  }
}

// ---- learned closure: features, corrections, energy -------------------------------------

constexpr int NFEAT = 24, NGEOM = 7;

// Feature normalization (x - mean) * scale and the output scales of the two corrections.
struct FeatureNorm {
  double mean[NFEAT];
  double scale[NFEAT];
  double out_scale[2];
};

// The network's 24 inputs of (edge, member) rows e * M + m, formed in FP64 as the stencil's
// mean and differences so that their BF16 rounding keeps the local gradients: u_e; u at the
// 10 TRiSK stencil edges minus u_e (0 for padded entries); the mean and the difference
// (second cell minus first) of h at the two cells, of q at the two vertices and of K = B - g h
// at the two cells; and 7 geometry values of the edge. Output row: row_map ? row_map[e] * M
// + m (file edge numbering) : the internal row.
template <class R>
__global__ void kg_features(DevTables T, DevWorkT<R> W, const R* y, int M, const float* geom,
                            const FeatureNorm N, __nv_bfloat16* X, const int32_t* row_map, int64_t rows) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int e, m;  // rows < 2^31 (checked when the ensemble is made)
  split<true>((int)r, M, e, m);
  const R* u = y;
  const R* h = y + (size_t)T.ne * M;
  double f[NFEAT];
  const double ue = u[(size_t)e * M + m];
  f[0] = ue;
#pragma unroll
  for (int k = 0; k < TWD; ++k) {
    const int ep = T.trisk_edges[k * T.lde + e];
    f[1 + k] = T.trisk[k * T.lde + e] != 0.0 ? (double)u[(size_t)ep * M + m] - ue : 0.0;
  }
  const int c0 = T.edge_cells[e], c1 = T.edge_cells[T.lde + e];
  const int v0 = T.edge_vertices[e], v1 = T.edge_vertices[T.lde + e];
  const double h0 = h[(size_t)c0 * M + m], h1 = h[(size_t)c1 * M + m];
  const double q0 = W.qv[(size_t)v0 * M + m], q1 = W.qv[(size_t)v1 * M + m];
  const double K0 = (double)W.B[(size_t)c0 * M + m] - T.gravity * h0;
  const double K1 = (double)W.B[(size_t)c1 * M + m] - T.gravity * h1;
  f[11] = (h0 + h1) / 2;
  f[12] = h1 - h0;
  f[13] = (q0 + q1) / 2;
  f[14] = q1 - q0;
  f[15] = (K0 + K1) / 2;
  f[16] = K1 - K0;
#pragma unroll
  for (int k = 0; k < NGEOM; ++k) f[17 + k] = geom[(size_t)e * NGEOM + k];
  const int64_t out = row_map ? (int64_t)row_map[e] * M + m : r;
  // the row's 48 bytes as three 16-byte stores (rows are 16-byte aligned)
  __align__(16) __nv_bfloat16 b[NFEAT];
#pragma unroll
  for (int k = 0; k < NFEAT; ++k) b[k] = __float2bfloat16_rn((float)((f[k] - N.mean[k]) * N.scale[k]));
  uint4* dst = reinterpret_cast<uint4*>(X + out * NFEAT);
  const uint4* src = reinterpret_cast<const uint4*>(b);
#pragma unroll
  for (int c = 0; c < NFEAT / 8; ++c) dst[c] = src[c];
}

// dF = on[m] sF y0 (mass flux: added to F in the flux-form continuity equation only, so
// mass stays conserved and the PV flux keeps the resolved F); dq = on[m] sQ y1 (momentum
// tendency).
template <class R>
__global__ void kg_closure_apply(R* dF, R* dq, const float* Y, const float* member_on, int64_t rows, int M,
                                 double sF, double sQ) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int e, m;
  split<true>((int)r, M, e, m);
  const double on = member_on[m];
  dF[r] = (R)(on * sF * (double)Y[2 * r]);
  dq[r] = (R)(on * sQ * (double)Y[2 * r + 1]);
}

// Work-free momentum correction. With the cell kinetic energy K_i = sum_k kinetic[i,k] u_k^2,
// kinetic[i,k] = l_e d_(e,i) / (2 A_i) (the TRiSK coefficient, alpha = 1), the energy's
// gradient is g_e = dE/du_e = u_e l_e (h_c0 d_(e,c0) + h_c1 d_(e,c1)). Removing from each
// member's correction dq its component along g (dq -= (<g, dq> / <g, g>) g) leaves a
// correction that does no work on that member's flow to first order. geom: l_e, d_e and the
// two cell distances in columns 0..3 of the closure geometry (internal edge order).
__device__ __forceinline__ double energy_gradient(const DevTables& T, double ue, double h0, double h1,
                                                  const float* geom, int e) {
  const float* gm = geom + (size_t)e * NGEOM;
  return ue * (double)gm[0] * (h0 * (double)gm[2] + h1 * (double)gm[3]);
}

// Per-block partial sums of <g, dq> and <g, g> for member m: partials[(2m) gridDim.x + block]
// and partials[(2m + 1) gridDim.x + block]; block (32, 8): x members, y edges. kg_sum_rows
// then adds each row's partials in a fixed order, so the sums do not depend on the order in
// which blocks finish.
template <class R>
__global__ void kg_work_sums(DevTables T, const R* y, const R* dq, const float* geom, int M, double* partials) {
  __shared__ double s1[8][32], s2[8][32];
  const int m = blockIdx.y * 32 + threadIdx.x;
  double a = 0.0, b = 0.0;
  if (m < M) {
    const R* h = y + (size_t)T.ne * M;
    for (int e = blockIdx.x * 8 + threadIdx.y; e < T.ne; e += gridDim.x * 8) {
      const int c0 = T.edge_cells[e], c1 = T.edge_cells[T.lde + e];
      const double g = energy_gradient(T, (double)y[(size_t)e * M + m], (double)h[(size_t)c0 * M + m],
                                       (double)h[(size_t)c1 * M + m], geom, e);
      a += g * (double)dq[(size_t)e * M + m];
      b += g * g;
    }
  }
  s1[threadIdx.y][threadIdx.x] = a;
  s2[threadIdx.y][threadIdx.x] = b;
  __syncthreads();
  if (threadIdx.y == 0 && m < M) {
    for (int k = 1; k < 8; ++k) {
      a += s1[k][threadIdx.x];
      b += s2[k][threadIdx.x];
    }
    partials[(size_t)(2 * m) * gridDim.x + blockIdx.x] = a;
    partials[(size_t)(2 * m + 1) * gridDim.x + blockIdx.x] = b;
  }
}

// out[row] = the sum of partials[row * ncols + 0 .. ncols - 1] in a fixed order (each thread
// a fixed strided run, then a fixed tree): one block of 256 threads per row.
__global__ void kg_sum_rows(const double* partials, int ncols, double* out) {
  __shared__ double sm[256];
  const double* p = partials + (size_t)blockIdx.x * ncols;
  double s = 0.0;
  for (int c = threadIdx.x; c < ncols; c += 256) s += p[c];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sm[0];
}

template <class R>
__global__ void kg_work_project(DevTables T, const R* y, R* dq, const float* geom, int M, int64_t rows,
                                const double* sums) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int e, m;
  split<true>((int)r, M, e, m);
  const double gg = sums[2 * m + 1];
  if (!(gg > 0.0)) return;
  const R* h = y + (size_t)T.ne * M;
  const int c0 = T.edge_cells[e], c1 = T.edge_cells[T.lde + e];
  const double g = energy_gradient(T, (double)y[r], (double)h[(size_t)c0 * M + m], (double)h[(size_t)c1 * M + m],
                                   geom, e);
  dq[r] = (R)((double)dq[r] - sums[2 * m] / gg * g);
}

// partials[m gridDim.x + block] = sum_i A_i h_i (K_i + g h_i / 2) over this block's cells
// (TRiSKShallowWater.jl:406-411); kg_sum_rows adds them per member in a fixed order.
template <class R>
__global__ void kg_energy(const R* y, const R* K, const double* area, int nc, int ne, int M, double g,
                          double* partials) {
  __shared__ double sm[256];
  const int m = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < nc) {
    const double hi = y[(size_t)ne * M + (size_t)i * M + m];
    const double Ki = K[(size_t)i * M + m];
    s = area[i] * hi * (Ki + g * hi / 2);
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[(size_t)m * gridDim.x + blockIdx.x] = sm[0];
}

__global__ void kg_advance(int* counters, int n) {
  if (threadIdx.x < n) counters[threadIdx.x] += 1;
}

// y_group[j M + m] = y_file[n2o[j]]  and back
template <class R>
__global__ void kg_scatter_member(R* dst, const double* src, const int32_t* n2o, int64_t N, int M, int m) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < N) dst[j * M + m] = (R)src[n2o[j]];
}
template <class R>
__global__ void kg_gather_member(double* dst, const R* src, const int32_t* o2n, int64_t N, int M, int m) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < N) dst[j] = (double)src[(int64_t)o2n[j] * M + m];
}

}  // namespace trisk

// A group's learned closure: network, buffers of its (edge, member) rows and settings.
struct ClosureSlot {
  TriskClosure* net = nullptr;
  __nv_bfloat16* X = nullptr;  // rows x 24 features
  float* Y = nullptr;          // rows x 2 corrections
  float* geom = nullptr;       // ne x 7, internal edge order
  float* member_on = nullptr;  // M flags (1: closure on, 0: plain step)
  double* dF = nullptr;        // rows: mass-flux correction (continuity equation only), storage type
  double* dq = nullptr;        // rows: momentum-tendency correction, storage type
  trisk::FeatureNorm norm{};
  bool every_stage = false;    // false: the network runs at stage 1 and its output is reused
  bool work_free = false;      // project the momentum correction to do no work (per member)
  double* sums = nullptr;      // 2 M: <g, dq>, <g, g> per member
  double* partials = nullptr;  // 2 M x WORK_SUM_BLOCKS per-block partial sums of them
};

// blocks of kg_work_sums along the edges (the row length of its partial sums)
constexpr int WORK_SUM_BLOCKS = 1024;

struct TriskEnsemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t caller_ev = nullptr;  // for order_after_caller
  bool fp32 = false;                // state and work vectors stored as float (arithmetic FP64)
  int pv = 0, ke = 0;
  int block[3] = {128, 128, 128};  // threads per block of the vertex, flux and tendency phases
  int grid[3] = {0, 0, 0};
  GroupSet G{};
  ClosureSlot cl[trisk::MAX_GROUPS];
  double* energy = nullptr;           // per-member energies of the diagnostic
  double* energy_partials = nullptr;  // members x blocks partial sums of them
  size_t energy_partials_size = 0;
  std::vector<TriskModel*> models;
  std::vector<void*> allocations;
  int* counters = nullptr;
  int* flag = nullptr;
  double* staging = nullptr;
  int64_t max_state = 0;
  int max_members = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t launches = 0;
  int64_t graph_kernels = 0;
  double step_bytes = 0;

  ~TriskEnsemble() {
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
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocations.push_back(p);
    return static_cast<T*>(p);
  }
  size_t esize() const { return fp32 ? sizeof(float) : sizeof(double); }
  // a state or work vector of `count` elements of the storage type, kept as double*
  double* alloc_state(size_t count) { return reinterpret_cast<double*>(alloc<char>(count * esize())); }
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

// f(R{}) with R the ensemble's storage type.
template <class F>
void with_real(const TriskEnsemble& e, F&& f) {
  if (e.fp32)
    f(float{});
  else
    f(double{});
}

template <typename... KArgs, typename... Args>
void elaunch(TriskEnsemble& e, void (*kernel)(KArgs...), int phase, bool pdl, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)e.grid[phase]);
  cfg.blockDim = dim3((unsigned)e.block[phase]);
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
// The closure of every group that has one, after the flux phase of `stage`: features and
// the network (at stage 1, or at every stage), then the corrections of F and du.
void enqueue_closure(TriskEnsemble& e, int stage) {
  for (int g = 0; g < e.G.n; ++g) {
    ClosureSlot& c = e.cl[g];
    if (!c.net) continue;
    const GroupDesc& D = e.G.g[g];
    const int64_t rows = (int64_t)D.T.ne * D.M;
    const unsigned nb = (unsigned)cdiv(rows, 256);
    if (stage != 1 && !c.every_stage) continue;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      kg_features<R><<<nb, 256, 0, e.stream>>>(D.T, work_as<R>(D.W),
                                               reinterpret_cast<const R*>(stage == 1 ? D.y : D.st), D.M, c.geom,
                                               c.norm, c.X, nullptr, rows);
      CUDA_CHECK(cudaGetLastError());
      closure_forward_on(c.net, c.X, rows, c.Y, e.stream);
      kg_closure_apply<R><<<nb, 256, 0, e.stream>>>(reinterpret_cast<R*>(c.dF), reinterpret_cast<R*>(c.dq), c.Y,
                                                    c.member_on, rows, D.M, c.norm.out_scale[0],
                                                    c.norm.out_scale[1]);
      CUDA_CHECK(cudaGetLastError());
      if (c.work_free) {
        const R* ys = reinterpret_cast<const R*>(stage == 1 ? D.y : D.st);
        const int nx = (int)std::min<int64_t>(cdiv(D.T.ne, 8), WORK_SUM_BLOCKS);
        const dim3 grid((unsigned)nx, (unsigned)cdiv(D.M, 32));
        kg_work_sums<R><<<grid, dim3(32, 8), 0, e.stream>>>(D.T, ys, reinterpret_cast<const R*>(c.dq), c.geom, D.M,
                                                             c.partials);
        kg_sum_rows<<<(unsigned)(2 * D.M), 256, 0, e.stream>>>(c.partials, nx, c.sums);
        kg_work_project<R><<<nb, 256, 0, e.stream>>>(D.T, ys, reinterpret_cast<R*>(c.dq), c.geom, D.M, rows, c.sums);
        CUDA_CHECK(cudaGetLastError());
        e.launches += 3;
      }
    });
    e.launches += 3;
  }
}

bool any_closure(const TriskEnsemble& e) {
  for (int g = 0; g < e.G.n; ++g)
    if (e.cl[g].net) return true;
  return false;
}

void enqueue_ensemble_step(TriskEnsemble& e) {
  const bool closure = any_closure(e);
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    for (int stage = 1; stage <= 4; ++stage) {
      with_real(e, [&](auto r) {
        using R = decltype(r);
        elaunch(e, kg_vertex<PV, KE, R>, 0, stage != 1, e.G, stage == 1 ? 1 : 0);
        elaunch(e, kg_flux<PV, KE, R>, 1, true, e.G, stage == 1 ? 1 : 0, 0);
        if (closure) enqueue_closure(e, stage);
        switch (stage) {
          case 1: elaunch(e, kg_tend<PV, EPI_STAGE1, R>, 2, true, e.G); break;
          case 2: elaunch(e, kg_tend<PV, EPI_STAGE2, R>, 2, true, e.G); break;
          case 3: elaunch(e, kg_tend<PV, EPI_STAGE3, R>, 2, true, e.G); break;
          default: elaunch(e, kg_tend<PV, EPI_STAGE4, R>, 2, true, e.G); break;
        }
      });
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
  e.graph_kernels = e.launches - before;  // counted again at every replay
  e.launches = before;
  cudaError_t err = cudaGraphInstantiate(&e.graph, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(err);
}

void drop_graph(TriskEnsemble& e) {
  if (e.graph) {
    cudaGraphExecDestroy(e.graph);
    e.graph = nullptr;
  }
}

// Virtual blocks of every group per phase for the current block sizes, and the persistent
// grids (as many blocks as stay resident, never more than the work).
void layout(TriskEnsemble& e) {
  int sV = 0, sF = 0, sT = 0;
  for (int g = 0; g < e.G.n; ++g) {
    GroupDesc& D = e.G.g[g];
    const TriskModel& m = *e.models[g];
    const int64_t M = D.M;
    D.nV = (int)cdiv(m.nv * M / D.P, e.block[0]);
    D.nEF = (int)cdiv(m.ne * M / D.P, e.block[1]);
    D.nCF = (int)cdiv(m.nc * M / D.P, e.block[1]);
    D.nET = (int)cdiv(m.ne * M / D.P, e.block[2]);
    D.nCT = (int)cdiv(m.nc * M / D.P, e.block[2]);
    D.startV = sV;
    D.startF = sF;
    D.startT = sT;
    sV += D.nV;
    sF += D.nEF + D.nCF;
    sT += D.nET + D.nCT;
  }
  e.G.totalV = sV;
  e.G.totalF = sF;
  e.G.totalT = sT;
  int dev_sms = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, e.device));
  int occ[3] = {1, 1, 1};
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], kg_vertex<PV, KE, R>, e.block[0], 0));
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], kg_flux<PV, KE, R>, e.block[1], 0));
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], kg_tend<PV, EPI_STAGE2, R>, e.block[2], 0));
    });
  });
  const int total[3] = {sV, sF, sT};
  for (int p = 0; p < 3; ++p) e.grid[p] = std::max(1, std::min(total[p], dev_sms * std::max(occ[p], 1)));
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
  return trisk_ensemble_create_precision(models, members, dt, nsteps, ngroups, 64, out);
}

int trisk_ensemble_create_precision(TriskModel* const* models, const int32_t* members, const double* dt,
                                    const int64_t* nsteps, int32_t ngroups, int32_t state_bits,
                                    TriskEnsemble** out) {
  TRISK_API_BEGIN
  if (!models || !members || !dt || !nsteps || !out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (ngroups < 1 || ngroups > MAX_GROUPS)
    throw Error(TRISK_ERR_ARGUMENT, "an ensemble has 1.." + std::to_string(MAX_GROUPS) + " groups");
  if (state_bits != 64 && state_bits != 32) throw Error(TRISK_ERR_ARGUMENT, "state_bits must be 64 or 32");
  auto e = std::make_unique<TriskEnsemble>();
  e->fp32 = state_bits == 32;
  const TriskModel* m0 = models[0];
  if (!m0) throw Error(TRISK_ERR_ARGUMENT, "model is NULL");
  e->device = m0->device;
  e->pv = m0->pv;
  e->ke = m0->ke;
  DeviceGuard guard(e->device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreateWithFlags(&e->caller_ev, cudaEventDisableTiming));
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
    D.W.K = e->alloc_state(m->nc * M);
    D.W.B = e->alloc_state(m->nc * M);
    D.W.F = e->alloc_state(m->ne * M);
    D.W.qe = e->alloc_state(m->ne * M);
    D.W.zv = e->alloc_state(m->nv * M);
    D.W.hv = e->alloc_state(m->nv * M);
    D.W.qv = e->alloc_state(m->nv * M);
    D.W.Kv = e->alloc_state(m->nv * M);
    D.y = e->alloc_state(m->N * M);
    D.acc = e->alloc_state(m->N * M);
    D.st = e->alloc_state(m->N * M);
    CUDA_CHECK(cudaMemset(D.y, 0, m->N * M * e->esize()));
    D.P = M % 2 == 0 ? 2 : 1;
    e->models.push_back(m);
    e->max_state = std::max(e->max_state, m->N);
    e->max_members = std::max(e->max_members, (int)M);
    const double Nb = (double)e->esize() * (double)m->N * M;
    e->step_bytes += 4 * (m->table_bytes_unique + 2 * Nb) + 15 * Nb;
  }
  e->G.n = ngroups;
  e->counters = e->alloc<int>(MAX_GROUPS);
  e->flag = e->alloc<int>(1);
  e->staging = e->alloc<double>(e->max_state);
  CUDA_CHECK(cudaMemset(e->counters, 0, MAX_GROUPS * sizeof(int)));
  CUDA_CHECK(cudaMemset(e->flag, 0, sizeof(int)));
  e->G.counters = e->counters;
  e->G.flag = e->flag;
  layout(*e);
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
  } else {
    order_after_caller(e.stream, e.caller_ev);
  }
  with_real(e, [&](auto r) {
    using R = decltype(r);
    kg_scatter_member<R><<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(reinterpret_cast<R*>(D.y), src,
                                                                         m.state_n2o, m.N, D.M, member);
  });
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
  if (dev) order_after_caller(e.stream, e.caller_ev);
  with_real(e, [&](auto r) {
    using R = decltype(r);
    kg_gather_member<R><<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(dst, reinterpret_cast<const R*>(D.y),
                                                                        m.state_o2n, m.N, D.M, member);
  });
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
    e.launches += e.graph_kernels;
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

int trisk_ensemble_set_block(TriskEnsemble* ens, const int32_t block[3]) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!block) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int p = 0; p < 3; ++p)
    if (block[p] < 64 || block[p] > 256 || block[p] % 32)
      throw Error(TRISK_ERR_ARGUMENT, "block sizes must be multiples of 32 in [64, 256]");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  for (int p = 0; p < 3; ++p) e.block[p] = block[p];
  layout(e);
  drop_graph(e);
  TRISK_API_END
}

int trisk_ensemble_get_block(TriskEnsemble* ens, int32_t block[3]) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!block) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int p = 0; p < 3; ++p) block[p] = e.block[p];
  TRISK_API_END
}

int trisk_ensemble_autotune(TriskEnsemble* ens, int32_t steps, double* best_ms) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (steps <= 0) throw Error(TRISK_ERR_ARGUMENT, "steps must be positive");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  // Times `steps` RK4 steps of all groups for every combination of the three phases' block
  // sizes and keeps the fastest. The members' states, the step counters and each group's
  // step count are saved first and restored after every trial and at the end, so the
  // ensemble continues as if nothing had run (every candidate computes the same numbers).
  static const int choices[] = {64, 128, 256};
  std::vector<double*> saved(e.G.n);
  std::vector<int> nsteps(e.G.n);
  std::vector<int> counters(MAX_GROUPS);
  CUDA_CHECK(cudaMemcpy(counters.data(), e.counters, MAX_GROUPS * sizeof(int), cudaMemcpyDeviceToHost));
  for (int g = 0; g < e.G.n; ++g) {
    const size_t bytes = (size_t)e.models[g]->N * e.G.g[g].M * e.esize();
    saved[g] = reinterpret_cast<double*>(e.alloc<char>(bytes));  // freed with the ensemble
    CUDA_CHECK(cudaMemcpyAsync(saved[g], e.G.g[g].y, bytes, cudaMemcpyDeviceToDevice, e.stream));
    nsteps[g] = e.G.g[g].nsteps;
    e.G.g[g].nsteps = steps + 2;  // every group takes part in every timed step
  }
  auto restore = [&]() {
    for (int g = 0; g < e.G.n; ++g) {
      const size_t bytes = (size_t)e.models[g]->N * e.G.g[g].M * e.esize();
      CUDA_CHECK(cudaMemcpyAsync(e.G.g[g].y, saved[g], bytes, cudaMemcpyDeviceToDevice, e.stream));
    }
    CUDA_CHECK(cudaMemsetAsync(e.counters, 0, MAX_GROUPS * sizeof(int), e.stream));
  };
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  int best[3] = {e.block[0], e.block[1], e.block[2]};
  double best_t = INFINITY;
  try {
    for (int a : choices)
      for (int b : choices)
        for (int c : choices) {
          e.block[0] = a;
          e.block[1] = b;
          e.block[2] = c;
          layout(e);
          drop_graph(e);
          restore();
          ensure_ensemble_graph(e);
          for (int s2 = 0; s2 < 2; ++s2) CUDA_CHECK(cudaGraphLaunch(e.graph, e.stream));  // warm-up
          CUDA_CHECK(cudaEventRecord(e0, e.stream));
          for (int s2 = 0; s2 < steps; ++s2) CUDA_CHECK(cudaGraphLaunch(e.graph, e.stream));
          CUDA_CHECK(cudaEventRecord(e1, e.stream));
          CUDA_CHECK(cudaEventSynchronize(e1));
          float ms = 0;
          CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
          if (ms < best_t) {
            best_t = ms;
            best[0] = a;
            best[1] = b;
            best[2] = c;
          }
        }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int p = 0; p < 3; ++p) e.block[p] = best[p];
  for (int g = 0; g < e.G.n; ++g) e.G.g[g].nsteps = nsteps[g];
  layout(e);
  drop_graph(e);
  restore();
  CUDA_CHECK(cudaMemcpyAsync(e.counters, counters.data(), MAX_GROUPS * sizeof(int), cudaMemcpyHostToDevice,
                             e.stream));
  CUDA_CHECK(cudaMemsetAsync(e.flag, 0, sizeof(int), e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  if (best_ms) *best_ms = best_t / steps;
  TRISK_API_END
}

int trisk_ensemble_bytes(TriskEnsemble* ens, double* step_bytes) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!step_bytes) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *step_bytes = e.step_bytes;
  TRISK_API_END
}

int trisk_ensemble_set_closure(TriskEnsemble* ens, int32_t group, TriskClosure* net, const float* geometry,
                               const double* norm, int32_t flags) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (group < 0 || group >= e.G.n) throw Error(TRISK_ERR_ARGUMENT, "group out of range");
  DeviceGuard guard(e.device);
  GroupDesc& D = e.G.g[group];
  ClosureSlot& c = e.cl[group];
  drop_graph(e);
  if (!net) {  // back to the plain step
    c.net = nullptr;
    D.W.dq = D.W.dF = nullptr;
    return TRISK_OK;
  }
  TriskModel& m = *e.models[group];
  if (m.pv != PVM_TRISK) throw Error(TRISK_ERR_UNSUPPORTED, "the closure's features need the TRiSK PV flux");
  if (closure_device(net) != e.device) throw Error(TRISK_ERR_ARGUMENT, "closure on another device");
  if (!geometry || !norm) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  const int64_t rows = m.ne * (int64_t)D.M;
  if (!c.X) {
    c.X = e.alloc<__nv_bfloat16>(rows * NFEAT);
    c.Y = e.alloc<float>(rows * 2);
    c.geom = e.alloc<float>(m.ne * NGEOM);
    c.member_on = e.alloc<float>(D.M);
    c.dF = e.alloc_state(rows);
    c.dq = e.alloc_state(rows);
    std::vector<float> on(D.M, 1.0f);
    CUDA_CHECK(cudaMemcpy(c.member_on, on.data(), D.M * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(c.Y, 0, rows * 2 * sizeof(float)));
    CUDA_CHECK(cudaMemset(c.dF, 0, rows * e.esize()));
    CUDA_CHECK(cudaMemset(c.dq, 0, rows * e.esize()));
  }
  D.W.dq = c.dq;
  D.W.dF = c.dF;
  std::vector<float> g((size_t)m.ne * NGEOM);
  for (int64_t j = 0; j < m.ne; ++j)  // internal edge j = file edge edge_n2o[j]
    for (int k = 0; k < NGEOM; ++k) g[j * NGEOM + k] = geometry[(size_t)m.edge_n2o[j] * NGEOM + k];
  CUDA_CHECK(cudaMemcpy(c.geom, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice));
  for (int k = 0; k < NFEAT; ++k) {
    c.norm.mean[k] = norm[k];
    c.norm.scale[k] = norm[NFEAT + k];
  }
  c.norm.out_scale[0] = norm[2 * NFEAT];
  c.norm.out_scale[1] = norm[2 * NFEAT + 1];
  c.every_stage = (flags & 1) != 0;
  c.work_free = (flags & 2) != 0;
  if (c.work_free && !c.sums) {
    c.sums = e.alloc<double>(2 * (size_t)D.M);
    c.partials = e.alloc<double>(2 * (size_t)D.M * WORK_SUM_BLOCKS);
  }
  c.net = net;
  TRISK_API_END
}

int trisk_ensemble_closure_mask(TriskEnsemble* ens, int32_t group, const float* member_on) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (group < 0 || group >= e.G.n || !member_on) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  ClosureSlot& c = e.cl[group];
  if (!c.net) throw Error(TRISK_ERR_ARGUMENT, "the group has no closure");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaMemcpyAsync(c.member_on, member_on, e.G.g[group].M * sizeof(float), cudaMemcpyHostToDevice,
                             e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

// The closure features of the group's current member states (file edge order, rows
// e * M + m) into the device array X (rows x 24 BF16), normalized with `norm`.
int trisk_ensemble_features(TriskEnsemble* ens, int32_t group, void* X, const double* norm,
                            const float* geometry) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (group < 0 || group >= e.G.n || !X || !norm || !geometry) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  if (reinterpret_cast<uintptr_t>(X) % 16) throw Error(TRISK_ERR_ARGUMENT, "X must be 16-byte aligned");
  TriskModel& m = *e.models[group];
  if (m.pv != PVM_TRISK) throw Error(TRISK_ERR_UNSUPPORTED, "the closure's features need the TRiSK PV flux");
  DeviceGuard guard(e.device);
  const GroupDesc& D = e.G.g[group];
  const int M = D.M;
  FeatureNorm N{};
  for (int k = 0; k < NFEAT; ++k) {
    N.mean[k] = norm[k];
    N.scale[k] = norm[NFEAT + k];
  }
  std::vector<float> g((size_t)m.ne * NGEOM);
  for (int64_t j = 0; j < m.ne; ++j)
    for (int k = 0; k < NGEOM; ++k) g[j * NGEOM + k] = geometry[(size_t)m.edge_n2o[j] * NGEOM + k];
  float* geom = nullptr;
  int32_t* map = nullptr;
  CUDA_CHECK(cudaMallocAsync((void**)&geom, g.size() * sizeof(float), e.stream));
  CUDA_CHECK(cudaMallocAsync((void**)&map, m.ne * sizeof(int32_t), e.stream));
  CUDA_CHECK(cudaMemcpyAsync(geom, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice, e.stream));
  CUDA_CHECK(cudaMemcpyAsync(map, m.edge_n2o.data(), m.ne * sizeof(int32_t), cudaMemcpyHostToDevice, e.stream));
  const int B = 128;
  const int64_t rows = m.ne * (int64_t)M;
  order_after_caller(e.stream, e.caller_ev);  // X may still be read by the caller
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      const R* u = reinterpret_cast<const R*>(D.y);
      const R* h = u + (size_t)m.ne * M;
      const DevWorkT<R> W = work_as<R>(D.W);
      k_vertex<PV, KE, true, R><<<(unsigned)cdiv(m.nv * M, B), B, 0, e.stream>>>(D.T, W, u, h, M, 0);
      const int nbE = (int)cdiv(m.ne * M, B);
      k_flux<PV, KE, true, R><<<(unsigned)(nbE + cdiv(m.nc * M, B)), B, 0, e.stream>>>(D.T, W, u, h, M, nbE, 1);
      kg_features<R><<<(unsigned)cdiv(rows, 256), 256, 0, e.stream>>>(D.T, W, u, M, geom, N,
                                                                       static_cast<__nv_bfloat16*>(X), map, rows);
    });
  });
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaFreeAsync(geom, e.stream));
  CUDA_CHECK(cudaFreeAsync(map, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  e.launches += 3;
  TRISK_API_END
}

// Total energy sum_i A_i h_i (K_i + g h_i / 2) of every member of the group (host, M values).
int trisk_ensemble_energy(TriskEnsemble* ens, int32_t group, double* energies) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (group < 0 || group >= e.G.n || !energies) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  TriskModel& m = *e.models[group];
  DeviceGuard guard(e.device);
  const GroupDesc& D = e.G.g[group];
  const int M = D.M;
  if (!e.energy) e.energy = e.alloc<double>(e.max_members);
  const int nblocks = (int)cdiv(m.nc, 256);
  if (e.energy_partials_size < (size_t)nblocks * M) {  // grown on demand, kept for later calls
    e.energy_partials_size = (size_t)nblocks * M;
    e.energy_partials = e.alloc<double>(e.energy_partials_size);
  }
  const int B = 128;
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      const R* u = reinterpret_cast<const R*>(D.y);
      const R* h = u + (size_t)m.ne * M;
      const DevWorkT<R> W = work_as<R>(D.W);
      k_vertex<PV, KE, true, R><<<(unsigned)cdiv(m.nv * M, B), B, 0, e.stream>>>(D.T, W, u, h, M, 0);
      const int nbE = (int)cdiv(m.ne * M, B);
      k_flux<PV, KE, true, R><<<(unsigned)(nbE + cdiv(m.nc * M, B)), B, 0, e.stream>>>(D.T, W, u, h, M, nbE, 1);
      kg_energy<R><<<dim3((unsigned)nblocks, (unsigned)M), 256, 0, e.stream>>>(
          u, W.K, m.area_c, (int)m.nc, (int)m.ne, M, m.gravity, e.energy_partials);
      kg_sum_rows<<<(unsigned)M, 256, 0, e.stream>>>(e.energy_partials, nblocks, e.energy);
    });
  });
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaMemcpyAsync(energies, e.energy, M * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  e.launches += 4;
  TRISK_API_END
}

int trisk_ensemble_closure_check(TriskEnsemble* ens) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  DeviceGuard guard(e.device);
  for (int g = 0; g < e.G.n; ++g)
    if (e.cl[g].net) closure_check(e.cl[g].net);
  TRISK_API_END
}

}  // extern "C"
