// Batched ensembles: many members, on meshes of several levels, advanced by persistent
// launches per phase. A group is a set of members that share one model's tables (same mesh,
// same scheme). Its members are split into slices of consecutive members, each stored on its
// own ([entity][slice member] state and work vectors, one slice after the other), so the table
// entries a warp reads serve all the members it holds, one gathered index reads the members'
// values as one contiguous run, and a slice's work vectors are small enough to stay in L2
// from one phase to the next. The phases of a set of slices (a launch set) run back to back,
// set after set; the RK4 step of all unfinished groups is one CUDA graph; each group has its
// own dt and step count.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <type_traits>

#include <cuda_bf16.h>

#include "closure_mlp.cuh"
#include "model.hpp"

using namespace trisk;

namespace trisk {

constexpr int MAX_GROUPS = 8;  // groups of an ensemble
constexpr int MAX_SET = 8;     // slices of one launch set

// One slice: members [m0, m0 + M) of a group.
struct GroupDesc {
  DevTables T;
  DevWork W;
  double *y, *acc, *st;
  double dt;
  const int* counter;  // the group's steps taken (device)
  int M;       // members of the slice
  int nsteps;  // RK4 steps the group takes in a run
  int startV, nV;
  int startF, nEF, nCF;
  int startT, nET, nCT;
  int P;  // members per thread in the three phases (2 when M is even, else 1)
};

struct GroupSet {
  GroupDesc g[MAX_SET];
  int n;
  int totalV, totalF, totalT;
  int* flag;  // non-finite state seen
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

// PW: 4 for an ensemble whose every slice takes four members per thread (one instantiation
// with room for the wider registers), 0 for one or two members per thread as each slice has.
template <int PV, int KE, class R, int PW>
__global__ void __launch_bounds__(256) kg_vertex(const GroupSet G, int first_stage) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalV; vb += gridDim.x) {
    const int gi = group_of(G, vb, 0);
    const GroupDesc& D = G.g[gi];
    if (*D.counter >= D.nsteps) continue;
    const R* u = as_r<R>(first_stage ? D.y : D.st);
    const R* h = u + (size_t)D.T.ne * D.M;
    if constexpr (PW == 4)
      vertex_body<PV, KE, true, R, false, 4>(D.T, work_as<R>(D.W), u, h, D.M, 0, vb - D.startV);
    else if (D.P == 2)
      vertex_body<PV, KE, true, R, false, 2>(D.T, work_as<R>(D.W), u, h, D.M, 0, vb - D.startV);
    else
      vertex_body<PV, KE, true, R>(D.T, work_as<R>(D.W), u, h, D.M, 0, vb - D.startV);
  }
}

template <int PV, int KE, class R, int PW>
__global__ void __launch_bounds__(256) kg_flux(const GroupSet G, int first_stage, int want_K) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalF; vb += gridDim.x) {
    const int gi = group_of(G, vb, 1);
    const GroupDesc& D = G.g[gi];
    if (*D.counter >= D.nsteps) continue;
    const R* u = as_r<R>(first_stage ? D.y : D.st);
    const R* h = u + (size_t)D.T.ne * D.M;
    if constexpr (PW == 4)
      flux_body<PV, KE, true, R, false, 4>(D.T, work_as<R>(D.W), u, h, D.M, D.nEF, want_K, vb - D.startF);
    else if (D.P == 2)
      flux_body<PV, KE, true, R, false, 2>(D.T, work_as<R>(D.W), u, h, D.M, D.nEF, want_K, vb - D.startF);
    else
      flux_body<PV, KE, true, R>(D.T, work_as<R>(D.W), u, h, D.M, D.nEF, want_K, vb - D.startF);
  }
}

// <= 64 registers (8 blocks of 128) for one or two members per thread, and for four with a
// Gassmann PV flux (measured 5-6 % faster than 85 on the FP32 hexagon-6 and -7 groups); <= 85
// for four with the TRiSK PV flux (three blocks of 256: 2-5 % faster than 128 registers at two
// blocks, and 12 % faster than 64 on 128 hexagon-6 members)
template <int PV, int EPI, class R, int PW>
__global__ void __launch_bounds__(256, PW == 4 && PV == PVM_TRISK ? 3 : 4) kg_tend(const GroupSet G) {
  pdl_trigger();
  for (int vb = blockIdx.x; vb < G.totalT; vb += gridDim.x) {
    const int gi = group_of(G, vb, 2);
    const GroupDesc& D = G.g[gi];
    if (*D.counter >= D.nsteps) continue;
    DevStageT<R> S{};
    S.y = as_r<R>(D.y);
    S.acc = as_r<R>(D.acc);
    S.st = as_r<R>(D.st);
    S.flag = G.flag;
    S.c = EPI == EPI_STAGE3 ? D.dt : D.dt / 2;
    S.sixth = D.dt / 6;
    if constexpr (PW == 4) {
      if (D.W.dq)
        tend_body_p<PV, EPI, true, R, 4>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
      else
        tend_body_p<PV, EPI, false, R, 4>(D.T, work_as<R>(D.W), S, D.M, D.nET, vb - D.startT);
    } else if (D.P == 2) {
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

// The network's 24 inputs of (edge, member) row r = e * M + m of a slice, formed in FP64 as the
// stencil's mean and differences so that their BF16 rounding keeps the local gradients: u_e;
// u at the 10 TRiSK stencil edges minus u_e (0 for padded entries); the mean and the
// difference (second cell minus first) of h at the two cells, of q at the two vertices and of
// K = B - g h at the two cells; and 7 geometry values of the edge; normalized (x - mean) scale
// and rounded to BF16, as the row's 48 bytes.
template <class R>
__device__ __forceinline__ void feature_row(const DevTables& T, const DevWorkT<R>& W, const R* y, int M,
                                            const float* geom, const FeatureNorm& N, int64_t r, uint4 (&q)[3]) {
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
  __align__(16) __nv_bfloat16 b[NFEAT];
#pragma unroll
  for (int k = 0; k < NFEAT; ++k) b[k] = __float2bfloat16_rn((float)((f[k] - N.mean[k]) * N.scale[k]));
  const uint4* src = reinterpret_cast<const uint4*>(b);
  q[0] = src[0];
  q[1] = src[1];
  q[2] = src[2];
}

// The features of a slice's rows into X. Output row: row_map ? row_map[e] * Mg + m0 + m (file
// edge numbering, the group's Mg members, the slice starting at member m0) : the slice's row.
template <class R>
__global__ void kg_features(DevTables T, DevWorkT<R> W, const R* y, int M, const float* geom,
                            const FeatureNorm N, __nv_bfloat16* X, const int32_t* row_map, int64_t rows, int Mg,
                            int m0) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  uint4 q[3];
  feature_row<R>(T, W, y, M, geom, N, r, q);
  int e, m;
  split<true>((int)r, M, e, m);
  const int64_t out = row_map ? (int64_t)row_map[e] * Mg + m0 + m : r;
  uint4* dst = reinterpret_cast<uint4*>(X + out * NFEAT);  // rows are 16-byte aligned
#pragma unroll
  for (int c = 0; c < NFEAT / 8; ++c) dst[c] = q[c];
}

// dF = on[m] sF y0 (mass flux: added to F in the flux-form continuity equation only, so
// mass stays conserved and the PV flux keeps the resolved F); dq = on[m] sQ y1 (momentum
// tendency).
template <class R>
__device__ __forceinline__ void apply_row(R* dF, R* dq, int64_t r, int M, const float* member_on, double sF,
                                          double sQ, float y0, float y1) {
  int e, m;
  split<true>((int)r, M, e, m);
  const double on = member_on[m];
  dF[r] = (R)(on * sF * (double)y0);
  dq[r] = (R)(on * sQ * (double)y1);
}

template <class R>
__global__ void kg_closure_apply(R* dF, R* dq, const float* Y, const float* member_on, int64_t rows, int M,
                                 double sF, double sQ) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  apply_row<R>(dF, dq, r, M, member_on, sF, sQ, Y[2 * r], Y[2 * r + 1]);
}

// The corrections of the members whose closure is off set to zero (kept corrections of a member
// that falls back must not outlive the fallback).
template <class R>
__global__ void kg_zero_off_members(R* dF, R* dq, const float* member_on, int64_t rows, int M) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int e, m;
  split<true>((int)r, M, e, m);
  if (member_on[m] == 0.0f) {
    dF[r] = (R)0.0;
    dq[r] = (R)0.0;
  }
}

// The closure of a slice's rows in one kernel, bit for bit kg_features, the network's inference
// and kg_closure_apply in turn: per tile of 128 (edge, member) rows every thread builds its
// row's features straight into the tile's shared-memory operand, the tile runs through the
// network on the tensor cores, and every thread writes its row's two corrections. Features
// and network outputs never go to HBM (48 + 8 bytes per row each way in the three-launch form).
// A persistent grid; the bounded tensor-core waits report through the network's status word.
template <class R>
__global__ void __launch_bounds__(closure::TILE) kg_closure_fused(
    DevTables T, DevWorkT<R> W, const R* y, int M, const float* geom, const FeatureNorm N,
    const closure::ParamsBF16* wbf, const closure::Params* p, const float* member_on, double sF, double sQ, R* dF,
    R* dq, int64_t rows, closure::Status* status, const int* counter, int every, int phase) {
  using namespace closure;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(16) InferStatic st;
  const int t = threadIdx.x;
  const int64_t ntiles = (rows + TILE - 1) / TILE;
  if ((int64_t)blockIdx.x >= ntiles) return;
  if (every > 1 && (*counter - phase) % every != 0) return;  // not a network step: the corrections are kept
  const InferSmem S(smem);
  const uint32_t tmem = infer_setup(S, st, wbf, p);
  MmaWaits waits(smem_u32(S.mbar), &st.abort);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t r = tile * TILE + t;
    uint4 q[3] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    if (r < rows) feature_row<R>(T, W, y, M, geom, N, r, q);
    infer_put_row(S, q);
    float y0, y1;
    if (!infer_tile(S, st, tmem, waits, true, y0, y1)) break;
    if (r < rows) apply_row<R>(dF, dq, r, M, member_on, sF, sQ, y0, y1);
  }
  infer_finish(waits, tmem, status);
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

// the step counters of the groups in `mask`
__global__ void kg_advance(int* counters, unsigned mask) {
  if (threadIdx.x < MAX_GROUPS && ((mask >> threadIdx.x) & 1u)) counters[threadIdx.x] += 1;
}

// A group's state from slices of S_from members to slices of S_to members: member m of a
// group of M members sits in slice m / S (members m0 = S (m / S) onwards, Ss = min(S, M - m0)
// of them) at N m0 + j Ss + (m - m0) for state element j < N.
template <class R>
__global__ void kg_relayout(R* dst, const R* src, int64_t N, int M, int S_from, int S_to) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= N * M) return;
  const int64_t j = t / M;
  const int m = (int)(t - j * M);
  const int a0 = (m / S_from) * S_from, b0 = (m / S_to) * S_to;
  const int sa = min(S_from, M - a0), sb = min(S_to, M - b0);
  dst[N * b0 + j * sb + (m - b0)] = src[N * a0 + j * sa + (m - a0)];
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

// A group's learned closure: network, buffers of its (edge, member) rows and settings. The
// rows of slice [m0, m0 + Ms) are rows ne m0 .. ne (m0 + Ms) - 1 of the buffers (e Ms + m
// within the slice).
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
  bool fused = true;           // features, network and corrections in one kernel (else three)
  int every = 1;               // the network runs every `every` steps; its corrections are kept between
  int phase = 0;               // on the steps whose count is phase modulo every
  int fused_per_sm = 1;        // resident CTAs per SM of the fused kernel
  double* sums = nullptr;      // 2 M: <g, dq>, <g, g> per member
  double* partials = nullptr;  // 2 M x WORK_SUM_BLOCKS per-block partial sums of them
};

// blocks of kg_work_sums along the edges (the row length of its partial sums)
constexpr int WORK_SUM_BLOCKS = 1024;
// A launch set takes slices while their gathered stage state and work vectors stay within
// this L2 budget. The L2 is 126 MB, but each of the two dies' halves caches what its own SMs
// read, so data every SM reads sees about half of it (the single-model path thrashes beyond
// a working set of ~60 MB).
constexpr double SLICE_L2_BUDGET = 48.0 * (1 << 20);

// A user group: its members' buffers (every slice's, one after the other) and its slicing.
struct EnsembleGroup {
  TriskModel* m = nullptr;
  int M = 0;                 // members
  int S = 0;                 // members per slice (the last slice may have fewer)
  double dt = 0;
  int nsteps = 0;
  int64_t taken = 0;         // steps taken, as the host counts them
  double *y = nullptr, *acc = nullptr, *st = nullptr;
  DevWork W{};
  ClosureSlot cl;
  double member_bytes = 0;   // gathered stage state and work vectors of one member
};

struct Slice {
  int group, m0;
  GroupDesc D;
};

struct EnsembleGraph {
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;
};

struct TriskEnsemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t caller_ev = nullptr;  // for order_after_caller
  bool fp32 = false;                // state and work vectors stored as float (arithmetic FP64)
  int pv = 0, ke = 0;
  int block[3] = {128, 128, 128};  // threads per block of the vertex, flux and tendency phases
  int occ[3] = {1, 1, 1};          // resident blocks per SM of the three phases
  // members per thread: 2 (two for an even slice, else one) or 4 (every slice's member count
  // a multiple of four; set with trisk_ensemble_set_members_per_thread)
  int mpt = 2;
  int sms = 1;
  std::vector<EnsembleGroup> groups;
  std::vector<Slice> slices;                 // every group's slices, group after group
  std::map<unsigned, EnsembleGraph> graphs;  // one RK4 step of the groups in the mask
  double* energy = nullptr;                  // per-member energies of the diagnostic
  double* energy_partials = nullptr;         // members x blocks partial sums of them
  size_t energy_partials_size = 0;
  std::vector<TriskModel*> models;
  std::vector<void*> allocations;
  int* counters = nullptr;
  int* flag = nullptr;
  double* staging = nullptr;
  int64_t max_state = 0;
  int max_members = 0;
  int64_t launches = 0;
  double step_bytes = 0;

  ~TriskEnsemble() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (auto& kv : graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
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
  // element `count` of a storage-type buffer kept as double*
  double* at(double* p, int64_t count) const {
    return p ? reinterpret_cast<double*>(reinterpret_cast<char*>(p) + count * (int64_t)esize()) : nullptr;
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

// f(R{}) with R the ensemble's storage type.
template <class F>
void with_real(const TriskEnsemble& e, F&& f) {
  if (e.fp32)
    f(float{});
  else
    f(double{});
}

// The slices of every group for its current S: descriptors pointing into the group's buffers.
void build_slices(TriskEnsemble& e) {
  e.slices.clear();
  for (int g = 0; g < (int)e.groups.size(); ++g) {
    EnsembleGroup& G = e.groups[g];
    const TriskModel& m = *G.m;
    for (int m0 = 0; m0 < G.M; m0 += G.S) {
      Slice sl{};
      sl.group = g;
      sl.m0 = m0;
      GroupDesc& D = sl.D;
      const int Ms = std::min(G.S, G.M - m0);
      D.T = m.T;
      D.M = Ms;
      D.dt = G.dt;
      D.nsteps = G.nsteps;
      D.counter = e.counters + g;
      D.y = e.at(G.y, m.N * m0);
      D.acc = e.at(G.acc, m.N * m0);
      D.st = e.at(G.st, m.N * m0);
      D.W.K = e.at(G.W.K, m.nc * m0);
      D.W.B = e.at(G.W.B, m.nc * m0);
      D.W.F = e.at(G.W.F, m.ne * m0);
      D.W.qe = e.at(G.W.qe, m.ne * m0);
      D.W.zv = e.at(G.W.zv, m.nv * m0);
      D.W.hv = e.at(G.W.hv, m.nv * m0);
      D.W.qv = e.at(G.W.qv, m.nv * m0);
      D.W.Kv = e.at(G.W.Kv, m.nv * m0);
      if (G.cl.net) {
        D.W.dq = e.at(G.cl.dq, m.ne * m0);
        D.W.dF = e.at(G.cl.dF, m.ne * m0);
      }
      // Two members per thread load and store them as one 8- or 16-byte vector, which needs
      // the slice's buffers to start at an even element: every n * m0 even (n = the entity
      // counts; always so on the generated meshes, whose counts are even). Four members per
      // thread need every m0 to be a multiple of four, which four_per_thread_fits checks.
      const bool even_base = m0 % 2 == 0 || (m.ne % 2 == 0 && m.nc % 2 == 0 && m.nv % 2 == 0);
      D.P = e.mpt == 4 ? 4 : (Ms % 2 == 0 && even_base ? 2 : 1);
      e.slices.push_back(sl);
    }
  }
}

// every slice's member count a multiple of four (the slices of a group: S members each, the
// last one the rest of M)
bool four_per_thread_fits(const TriskEnsemble& e) {
  for (const EnsembleGroup& G : e.groups)
    if (G.M % 4 || G.S % 4) return false;
  return true;
}

void drop_graphs(TriskEnsemble& e);

// The next step of group G runs its closure's network, whatever its interval (its kept
// corrections belong to states or a layout that the host has just changed).
void restart_network(TriskEnsemble& e, EnsembleGroup& G) {
  ClosureSlot& c = G.cl;
  if (!c.net || c.every <= 1) return;
  const int phase = (int)(G.taken % c.every);
  if (phase != c.phase) {
    c.phase = phase;
    drop_graphs(e);  // the phase is an argument of the captured launches
  }
}

void drop_graphs(TriskEnsemble& e) {
  for (auto& kv : e.graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  e.graphs.clear();
}

// Launch sets of the slices of the groups in `mask`: slices in order, a set taking slices
// while their state and work vectors stay within the L2 budget (and at most MAX_SET of them);
// each slice's virtual blocks per phase for the current block sizes.
std::vector<GroupSet> launch_sets(TriskEnsemble& e, unsigned mask, std::vector<std::vector<int>>* members) {
  std::vector<GroupSet> sets;
  GroupSet cur{};
  double bytes = 0;
  auto close = [&]() {
    if (cur.n) sets.push_back(cur);
    cur = GroupSet{};
    cur.flag = e.flag;
    bytes = 0;
  };
  close();
  if (members) members->clear();
  std::vector<int> cur_members;
  for (int k = 0; k < (int)e.slices.size(); ++k) {
    const Slice& sl = e.slices[k];
    if (!((mask >> sl.group) & 1u)) continue;
    const EnsembleGroup& G = e.groups[sl.group];
    const double b = G.member_bytes * sl.D.M;
    if (cur.n == MAX_SET || (cur.n > 0 && bytes + b > SLICE_L2_BUDGET)) {
      close();
      if (members) members->push_back(cur_members);
      cur_members.clear();
    }
    GroupDesc D = sl.D;
    const TriskModel& m = *G.m;
    const int64_t M = D.M;
    D.nV = (int)cdiv(m.nv * M / D.P, e.block[0]);
    D.nEF = (int)cdiv(m.ne * M / D.P, e.block[1]);
    D.nCF = (int)cdiv(m.nc * M / D.P, e.block[1]);
    D.nET = (int)cdiv(m.ne * M / D.P, e.block[2]);
    D.nCT = (int)cdiv(m.nc * M / D.P, e.block[2]);
    D.startV = cur.totalV;
    D.startF = cur.totalF;
    D.startT = cur.totalT;
    cur.totalV += D.nV;
    cur.totalF += D.nEF + D.nCF;
    cur.totalT += D.nET + D.nCT;
    cur.g[cur.n++] = D;
    cur_members.push_back(k);
    bytes += b;
  }
  if (cur.n) {
    sets.push_back(cur);
    if (members) members->push_back(cur_members);
  }
  return sets;
}

// Resident blocks per SM of the three phases for the current block sizes.
void layout(TriskEnsemble& e) {
  CUDA_CHECK(cudaDeviceGetAttribute(&e.sms, cudaDevAttrMultiProcessorCount, e.device));
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      auto occ = [&](auto pwc) {
        constexpr int PW = decltype(pwc)::value;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e.occ[0], kg_vertex<PV, KE, R, PW>, e.block[0], 0));
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e.occ[1], kg_flux<PV, KE, R, PW>, e.block[1], 0));
        CUDA_CHECK(
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e.occ[2], kg_tend<PV, EPI_STAGE2, R, PW>, e.block[2], 0));
      };
      if (e.mpt == 4)
        occ(std::integral_constant<int, 4>{});
      else
        occ(std::integral_constant<int, 0>{});
    });
  });
  drop_graphs(e);
}

template <typename... KArgs, typename... Args>
void elaunch(TriskEnsemble& e, void (*kernel)(KArgs...), int phase, int total, bool pdl, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)std::max(1, std::min(total, e.sms * std::max(e.occ[phase], 1))));
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

// The closure of every slice of the set whose group has one, after the flux phase of `stage`:
// features and the network (at stage 1, or at every stage), then the corrections of F and du.
void enqueue_closure(TriskEnsemble& e, const std::vector<int>& set_slices, int stage) {
  for (int k : set_slices) {
    const Slice& sl = e.slices[k];
    EnsembleGroup& G = e.groups[sl.group];
    ClosureSlot& c = G.cl;
    if (!c.net) continue;
    if (stage != 1 && !c.every_stage) continue;
    const GroupDesc& D = sl.D;
    const int64_t ne = D.T.ne;
    const int64_t rows = ne * D.M;
    const int64_t r0 = ne * sl.m0;  // the slice's first row
    const unsigned nb = (unsigned)cdiv(rows, 256);
    __nv_bfloat16* X = c.X + r0 * NFEAT;
    float* Y = c.Y + 2 * r0;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      R* dF = reinterpret_cast<R*>(e.at(c.dF, r0));
      R* dq = reinterpret_cast<R*>(e.at(c.dq, r0));
      const R* ys = reinterpret_cast<const R*>(stage == 1 ? D.y : D.st);
      if (c.fused) {
        const closure::ParamsBF16* wbf;
        const closure::Params* p;
        closure::Status* status;
        closure::closure_device_params(c.net, &wbf, &p, &status);
        const int64_t tiles = cdiv(rows, closure::TILE);
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)e.sms * c.fused_per_sm));
        kg_closure_fused<R><<<grid, closure::TILE, closure::FWD_SMEM_BYTES, e.stream>>>(
            D.T, work_as<R>(D.W), ys, D.M, c.geom, c.norm, wbf, p, c.member_on + sl.m0, c.norm.out_scale[0],
            c.norm.out_scale[1], dF, dq, rows, status, D.counter, c.every, c.phase);
        CUDA_CHECK(cudaGetLastError());
        e.launches -= 2;  // one launch instead of three
      } else {
        kg_features<R><<<nb, 256, 0, e.stream>>>(D.T, work_as<R>(D.W), ys, D.M, c.geom, c.norm, X, nullptr, rows,
                                                 G.M, sl.m0);
        CUDA_CHECK(cudaGetLastError());
        closure_forward_on(c.net, X, rows, Y, e.stream);
        kg_closure_apply<R><<<nb, 256, 0, e.stream>>>(dF, dq, Y, c.member_on + sl.m0, rows, D.M,
                                                      c.norm.out_scale[0], c.norm.out_scale[1]);
        CUDA_CHECK(cudaGetLastError());
      }
      if (c.work_free) {
        double* sums = c.sums + 2 * sl.m0;
        double* partials = c.partials + 2 * (int64_t)sl.m0 * WORK_SUM_BLOCKS;
        const int nx = (int)std::min<int64_t>(cdiv(ne, 8), WORK_SUM_BLOCKS);
        const dim3 grid((unsigned)nx, (unsigned)cdiv(D.M, 32));
        kg_work_sums<R><<<grid, dim3(32, 8), 0, e.stream>>>(D.T, ys, dq, c.geom, D.M, partials);
        kg_sum_rows<<<(unsigned)(2 * D.M), 256, 0, e.stream>>>(partials, nx, sums);
        kg_work_project<R><<<nb, 256, 0, e.stream>>>(D.T, ys, dq, c.geom, D.M, rows, sums);
        CUDA_CHECK(cudaGetLastError());
        e.launches += 3;
      }
    });
    e.launches += 3;
  }
}

// One RK4 step of the groups in `mask`: per stage, the three phases of every launch set in
// turn. The first launch of a step waits for the full completion of the launch before it
// (no PDL): the step counters it reads were just advanced.
void enqueue_ensemble_step(TriskEnsemble& e, unsigned mask) {
  std::vector<std::vector<int>> members;
  const std::vector<GroupSet> sets = launch_sets(e, mask, &members);
  with_modes_e(e.pv, e.ke, [&](auto pvc, auto kec) {
    constexpr int PV = decltype(pvc)::value, KE = decltype(kec)::value;
    for (int stage = 1; stage <= 4; ++stage) {
      for (size_t k = 0; k < sets.size(); ++k) {
        const GroupSet& G = sets[k];
        with_real(e, [&](auto r) {
          using R = decltype(r);
          auto phases = [&](auto pwc) {
            constexpr int PW = decltype(pwc)::value;
            elaunch(e, kg_vertex<PV, KE, R, PW>, 0, G.totalV, !(stage == 1 && k == 0), G, stage == 1 ? 1 : 0);
            elaunch(e, kg_flux<PV, KE, R, PW>, 1, G.totalF, true, G, stage == 1 ? 1 : 0, 0);
            enqueue_closure(e, members[k], stage);
            switch (stage) {
              case 1: elaunch(e, kg_tend<PV, EPI_STAGE1, R, PW>, 2, G.totalT, true, G); break;
              case 2: elaunch(e, kg_tend<PV, EPI_STAGE2, R, PW>, 2, G.totalT, true, G); break;
              case 3: elaunch(e, kg_tend<PV, EPI_STAGE3, R, PW>, 2, G.totalT, true, G); break;
              default: elaunch(e, kg_tend<PV, EPI_STAGE4, R, PW>, 2, G.totalT, true, G); break;
            }
          };
          if (e.mpt == 4)
            phases(std::integral_constant<int, 4>{});
          else
            phases(std::integral_constant<int, 0>{});
        });
      }
    }
  });
  kg_advance<<<1, 32, 0, e.stream>>>(e.counters, mask);
  CUDA_CHECK(cudaGetLastError());
  e.launches++;
}

EnsembleGraph& ensure_graph(TriskEnsemble& e, unsigned mask) {
  auto it = e.graphs.find(mask);
  if (it != e.graphs.end()) return it->second;
  const int64_t before = e.launches;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_ensemble_step(e, mask);
  } catch (...) {
    cudaStreamEndCapture(e.stream, &g);
    if (g) cudaGraphDestroy(g);
    e.launches = before;
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(e.stream, &g));
  EnsembleGraph eg;
  eg.kernels = e.launches - before;  // counted again at every replay
  e.launches = before;
  cudaError_t err = cudaGraphInstantiate(&eg.exec, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(err);
  return e.graphs[mask] = eg;
}

// `steps` RK4 steps: each replay advances every unfinished group by one step, so the host
// knows which groups a replay advances and replays the graph of exactly those groups.
void run_steps(TriskEnsemble& e, int64_t steps) {
  while (steps > 0) {
    unsigned mask = 0;
    int64_t k = steps;
    for (int g = 0; g < (int)e.groups.size(); ++g) {
      const EnsembleGroup& G = e.groups[g];
      if (G.taken < G.nsteps) {
        mask |= 1u << g;
        k = std::min<int64_t>(k, G.nsteps - G.taken);
      }
    }
    if (!mask) break;  // every group has taken its steps
    EnsembleGraph& eg = ensure_graph(e, mask);
    for (int64_t s = 0; s < k; ++s) {
      CUDA_CHECK(cudaGraphLaunch(eg.exec, e.stream));
      e.launches += eg.kernels;
    }
    for (int g = 0; g < (int)e.groups.size(); ++g)
      if ((mask >> g) & 1u) e.groups[g].taken += k;
    steps -= k;
  }
}

TriskEnsemble* checked_e(TriskEnsemble* e) {
  if (!e) throw Error(TRISK_ERR_ARGUMENT, "ensemble is NULL");
  return e;
}

// the slice holding member `member` of group g
const Slice& slice_of(TriskEnsemble& e, int g, int member) {
  if (g < 0 || g >= (int)e.groups.size()) throw Error(TRISK_ERR_ARGUMENT, "group out of range");
  if (member < 0 || member >= e.groups[g].M) throw Error(TRISK_ERR_ARGUMENT, "member out of range");
  for (const Slice& sl : e.slices)
    if (sl.group == g && member >= sl.m0 && member < sl.m0 + sl.D.M) return sl;
  throw Error(TRISK_ERR_ARGUMENT, "member out of range");
}

EnsembleGroup& group_ref(TriskEnsemble& e, int g) {
  if (g < 0 || g >= (int)e.groups.size()) throw Error(TRISK_ERR_ARGUMENT, "group out of range");
  return e.groups[g];
}

// A group's state from slices of S_from members to S_to (through a temporary copy).
void relayout_group(TriskEnsemble& e, EnsembleGroup& G, const double* from, int S_from, int S_to) {
  const int64_t n = G.m->N * (int64_t)G.M;
  with_real(e, [&](auto r) {
    using R = decltype(r);
    kg_relayout<R><<<(unsigned)cdiv(n, 256), 256, 0, e.stream>>>(reinterpret_cast<R*>(G.y),
                                                                 reinterpret_cast<const R*>(from), G.m->N, G.M,
                                                                 S_from, S_to);
  });
  CUDA_CHECK(cudaGetLastError());
}

// Changes group g to slices of S members, keeping every member's state.
void reslice(TriskEnsemble& e, int g, int S) {
  EnsembleGroup& G = e.groups[g];
  if (S == G.S) return;
  const int64_t n = G.m->N * (int64_t)G.M;
  double* tmp = nullptr;
  CUDA_CHECK(cudaMallocAsync((void**)&tmp, n * e.esize(), e.stream));
  CUDA_CHECK(cudaMemcpyAsync(tmp, G.y, n * e.esize(), cudaMemcpyDeviceToDevice, e.stream));
  relayout_group(e, G, tmp, G.S, S);
  CUDA_CHECK(cudaFreeAsync(tmp, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  G.S = S;
  build_slices(e);
  drop_graphs(e);
  restart_network(e, G);
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
  e->counters = e->alloc<int>(MAX_GROUPS);
  e->flag = e->alloc<int>(1);
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
    EnsembleGroup G;
    G.m = m;
    G.M = (int)M;
    G.dt = dt[g];
    G.nsteps = (int)nsteps[g];
    G.W.K = e->alloc_state(m->nc * M);
    G.W.B = e->alloc_state(m->nc * M);
    G.W.F = e->alloc_state(m->ne * M);
    G.W.qe = e->alloc_state(m->ne * M);
    G.W.zv = e->alloc_state(m->nv * M);
    G.W.hv = e->alloc_state(m->nv * M);
    G.W.qv = e->alloc_state(m->nv * M);
    G.W.Kv = e->alloc_state(m->nv * M);
    G.y = e->alloc_state(m->N * M);
    G.acc = e->alloc_state(m->N * M);
    G.st = e->alloc_state(m->N * M);
    CUDA_CHECK(cudaMemset(G.y, 0, m->N * M * e->esize()));
    G.member_bytes = (double)e->esize() * (1.0 * m->N + 2.0 * m->nc + 2.0 * m->ne + 4.0 * m->nv);
    G.S = G.M;  // whole groups: measured faster than any slicing (the autotuner tries others)
    e->groups.push_back(G);
    e->models.push_back(m);
    e->max_state = std::max(e->max_state, m->N);
    e->max_members = std::max(e->max_members, (int)M);
    const double Nb = (double)e->esize() * (double)m->N * M;
    e->step_bytes += 4 * (m->table_bytes_unique + 2 * Nb) + 15 * Nb;
  }
  e->staging = e->alloc<double>(e->max_state);
  CUDA_CHECK(cudaMemset(e->counters, 0, MAX_GROUPS * sizeof(int)));
  CUDA_CHECK(cudaMemset(e->flag, 0, sizeof(int)));
  // FP32 state: four members per thread where every group allows it (one 16-byte load per
  // gathered value, as two FP64 members take; measured faster on every FP32 group, slower on
  // every FP64 one)
  e->mpt = e->fp32 && four_per_thread_fits(*e) ? 4 : 2;
  build_slices(*e);
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
  const Slice& sl = slice_of(e, group, member);
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
    kg_scatter_member<R><<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(reinterpret_cast<R*>(sl.D.y), src,
                                                                         m.state_n2o, m.N, sl.D.M, member - sl.m0);
  });
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  restart_network(e, e.groups[group]);  // a new state: its corrections are formed afresh
  TRISK_API_END
}

int trisk_ensemble_get_member(TriskEnsemble* ens, int32_t group, int32_t member, double* y) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!y) throw Error(TRISK_ERR_ARGUMENT, "NULL state");
  const Slice& sl = slice_of(e, group, member);
  TriskModel& m = *e.models[group];
  DeviceGuard guard(e.device);
  const bool dev = is_device_pointer(y);
  double* dst = dev ? y : e.staging;
  if (dev) order_after_caller(e.stream, e.caller_ev);
  with_real(e, [&](auto r) {
    using R = decltype(r);
    kg_gather_member<R><<<(unsigned)cdiv(m.N, 256), 256, 0, e.stream>>>(
        dst, reinterpret_cast<const R*>(sl.D.y), m.state_o2n, m.N, sl.D.M, member - sl.m0);
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
  run_steps(e, steps);
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
  for (int g = 0; g < (int)e.groups.size(); ++g) steps_taken[g] = std::min<int64_t>(c[g], e.groups[g].nsteps);
  TRISK_API_END
}

int trisk_ensemble_reset(TriskEnsemble* ens) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaMemsetAsync(e.counters, 0, MAX_GROUPS * sizeof(int), e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  for (EnsembleGroup& G : e.groups) {
    G.taken = 0;
    restart_network(e, G);
  }
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
  TRISK_API_END
}

int trisk_ensemble_get_block(TriskEnsemble* ens, int32_t block[3]) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!block) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int p = 0; p < 3; ++p) block[p] = e.block[p];
  TRISK_API_END
}

int trisk_ensemble_set_slices(TriskEnsemble* ens, const int32_t* members_per_slice) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!members_per_slice) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int g = 0; g < (int)e.groups.size(); ++g)
    if (members_per_slice[g] < 1 || members_per_slice[g] > e.groups[g].M)
      throw Error(TRISK_ERR_ARGUMENT, "members per slice must be in 1..members of the group");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  for (int g = 0; g < (int)e.groups.size(); ++g) reslice(e, g, members_per_slice[g]);
  if (e.mpt == 4 && !four_per_thread_fits(e)) {  // back to two members per thread
    e.mpt = 2;
    build_slices(e);
    layout(e);
  }
  TRISK_API_END
}

int trisk_ensemble_set_members_per_thread(TriskEnsemble* ens, int32_t members) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (members != 2 && members != 4) throw Error(TRISK_ERR_ARGUMENT, "members per thread must be 2 or 4");
  if (members == 4 && !four_per_thread_fits(e))
    throw Error(TRISK_ERR_UNSUPPORTED, "four members per thread need every slice's member count a multiple of four");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  e.mpt = members;
  build_slices(e);
  layout(e);
  TRISK_API_END
}

int trisk_ensemble_get_members_per_thread(TriskEnsemble* ens, int32_t* members) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!members) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *members = e.mpt;
  TRISK_API_END
}

int trisk_ensemble_get_slices(TriskEnsemble* ens, int32_t* members_per_slice) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!members_per_slice) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  for (int g = 0; g < (int)e.groups.size(); ++g) members_per_slice[g] = e.groups[g].S;
  TRISK_API_END
}

int trisk_ensemble_autotune(TriskEnsemble* ens, int32_t steps, double* best_ms) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (steps <= 0) throw Error(TRISK_ERR_ARGUMENT, "steps must be positive");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  // Times `steps` RK4 steps of all groups for every combination of the three phases' block
  // sizes, then four members per thread (where every slice allows it) at each tendency block
  // size, then for the members per slice of each group in turn (S, S/2, S/4 ... and 2 S ..
  // up to the group), and keeps the fastest. The members' states (in the slicing they had),
  // the step counters and each group's step count are saved first and restored after every
  // trial and at the end, so the ensemble continues as if nothing had run (every candidate
  // computes the same numbers).
  static const int choices[] = {64, 128, 256};
  const int ng = (int)e.groups.size();
  std::vector<double*> saved(ng);
  std::vector<int> nsteps(ng), S0(ng);
  std::vector<int64_t> taken(ng);
  std::vector<int> counters(MAX_GROUPS);
  CUDA_CHECK(cudaMemcpy(counters.data(), e.counters, MAX_GROUPS * sizeof(int), cudaMemcpyDeviceToHost));
  for (int g = 0; g < ng; ++g) {
    EnsembleGroup& G = e.groups[g];
    const size_t bytes = (size_t)G.m->N * G.M * e.esize();
    saved[g] = reinterpret_cast<double*>(e.alloc<char>(bytes));  // freed with the ensemble
    CUDA_CHECK(cudaMemcpyAsync(saved[g], G.y, bytes, cudaMemcpyDeviceToDevice, e.stream));
    nsteps[g] = G.nsteps;
    taken[g] = G.taken;
    S0[g] = G.S;
    G.nsteps = steps + 2;  // every group takes part in every timed step
  }
  auto restore = [&]() {  // the saved states in the current slicing, counters at zero
    for (int g = 0; g < ng; ++g) relayout_group(e, e.groups[g], saved[g], S0[g], e.groups[g].S);
    CUDA_CHECK(cudaMemsetAsync(e.counters, 0, MAX_GROUPS * sizeof(int), e.stream));
    for (EnsembleGroup& G : e.groups) G.taken = 0;
  };
  auto set_slicing = [&](int g, int S) {  // no state to keep: restore() rewrites it
    e.groups[g].S = S;
    build_slices(e);
    drop_graphs(e);
  };
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  auto trial = [&]() {
    restore();
    build_slices(e);  // the step counts changed
    drop_graphs(e);
    run_steps(e, 2);  // warm-up (and the graph's capture)
    CUDA_CHECK(cudaEventRecord(e0, e.stream));
    run_steps(e, steps);
    CUDA_CHECK(cudaEventRecord(e1, e.stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    return (double)ms;
  };
  int best[3] = {e.block[0], e.block[1], e.block[2]};
  double best_t = INFINITY;
  e.mpt = 2;  // the blocks first with one or two members per thread
  build_slices(e);
  try {
    for (int a : choices)
      for (int b : choices)
        for (int c : choices) {
          e.block[0] = a;
          e.block[1] = b;
          e.block[2] = c;
          layout(e);
          const double ms = trial();
          if (ms < best_t) {
            best_t = ms;
            best[0] = a;
            best[1] = b;
            best[2] = c;
          }
        }
    for (int p = 0; p < 3; ++p) e.block[p] = best[p];
    layout(e);
    // four members per thread, at each tendency block size, where every slice allows it
    int best_mpt = 2;
    if (four_per_thread_fits(e)) {
      const int b2 = best[2];
      e.mpt = 4;
      build_slices(e);
      for (int c : choices) {
        e.block[2] = c;
        layout(e);
        const double ms = trial();
        if (ms < best_t) {
          best_t = ms;
          best[2] = c;
          best_mpt = 4;
        }
      }
      if (best_mpt != 4) best[2] = b2;
      e.mpt = best_mpt;
      build_slices(e);
      for (int p = 0; p < 3; ++p) e.block[p] = best[p];
      layout(e);
    }
    for (int g = 0; g < ng; ++g) {
      const int M = e.groups[g].M, start = e.groups[g].S;
      int best_S = start;
      std::vector<int> candidates;
      for (int S = start / 2; S >= 1 && candidates.size() < 3; S /= 2) candidates.push_back(S);
      for (int S = start * 2; candidates.size() < 6; S *= 2) {
        candidates.push_back(std::min(S, M));
        if (S >= M) break;
      }
      for (int S : candidates) {
        if (S == start || (e.mpt == 4 && S % 4)) continue;
        set_slicing(g, S);
        const double ms = trial();
        if (ms < best_t) {
          best_t = ms;
          best_S = S;
        }
      }
      set_slicing(g, best_S);
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int g = 0; g < ng; ++g) e.groups[g].nsteps = nsteps[g];
  build_slices(e);
  drop_graphs(e);
  restore();
  for (int g = 0; g < ng; ++g) e.groups[g].taken = taken[g];
  CUDA_CHECK(cudaMemcpyAsync(e.counters, counters.data(), MAX_GROUPS * sizeof(int), cudaMemcpyHostToDevice,
                             e.stream));
  for (EnsembleGroup& G : e.groups) {  // the trials overwrote the kept corrections
    G.cl.phase = -1;
    restart_network(e, G);
  }
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
  EnsembleGroup& G = group_ref(e, group);
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  ClosureSlot& c = G.cl;
  if (!net) {  // back to the plain step
    c.net = nullptr;
    build_slices(e);
    drop_graphs(e);
    return TRISK_OK;
  }
  TriskModel& m = *G.m;
  if (m.pv != PVM_TRISK) throw Error(TRISK_ERR_UNSUPPORTED, "the closure's features need the TRiSK PV flux");
  if (closure_device(net) != e.device) throw Error(TRISK_ERR_ARGUMENT, "closure on another device");
  if (!geometry || !norm) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  const int64_t rows = m.ne * (int64_t)G.M;
  if (!c.X) {
    c.X = e.alloc<__nv_bfloat16>(rows * NFEAT);
    c.Y = e.alloc<float>(rows * 2);
    c.geom = e.alloc<float>(m.ne * NGEOM);
    c.member_on = e.alloc<float>(G.M);
    c.dF = e.alloc_state(rows);
    c.dq = e.alloc_state(rows);
    std::vector<float> on(G.M, 1.0f);
    CUDA_CHECK(cudaMemcpy(c.member_on, on.data(), G.M * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(c.Y, 0, rows * 2 * sizeof(float)));
    CUDA_CHECK(cudaMemset(c.dF, 0, rows * e.esize()));
    CUDA_CHECK(cudaMemset(c.dq, 0, rows * e.esize()));
  }
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
  c.fused = (flags & 4) == 0;
  c.every = std::max(1, (flags >> 8) & 0xFF);
  if (c.every > 1 && (c.every_stage || !c.fused))
    throw Error(TRISK_ERR_UNSUPPORTED, "a network interval of several steps needs the fused kernel, at stage 1 only");
  if (c.fused)
    with_real(e, [&](auto r) {
      using R = decltype(r);
      c.fused_per_sm = closure::infer_ctas_per_sm(reinterpret_cast<const void*>(kg_closure_fused<R>), e.device);
    });
  if (c.work_free && !c.sums) {
    c.sums = e.alloc<double>(2 * (size_t)G.M);
    c.partials = e.alloc<double>(2 * (size_t)G.M * WORK_SUM_BLOCKS);
  }
  c.net = net;
  c.phase = (int)(G.taken % c.every);  // the network runs at the next step
  build_slices(e);
  drop_graphs(e);
  TRISK_API_END
}

int trisk_ensemble_closure_mask(TriskEnsemble* ens, int32_t group, const float* member_on) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!member_on) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  EnsembleGroup& G = group_ref(e, group);
  ClosureSlot& c = G.cl;
  if (!c.net) throw Error(TRISK_ERR_ARGUMENT, "the group has no closure");
  DeviceGuard guard(e.device);
  CUDA_CHECK(cudaMemcpyAsync(c.member_on, member_on, G.M * sizeof(float), cudaMemcpyHostToDevice, e.stream));
  for (const Slice& sl : e.slices) {  // kept corrections of the members turned off
    if (&e.groups[sl.group] != &G) continue;
    const int64_t ne = sl.D.T.ne, rows = ne * sl.D.M, r0 = ne * sl.m0;
    with_real(e, [&](auto r) {
      using R = decltype(r);
      kg_zero_off_members<R><<<(unsigned)cdiv(rows, 256), 256, 0, e.stream>>>(
          reinterpret_cast<R*>(e.at(c.dF, r0)), reinterpret_cast<R*>(e.at(c.dq, r0)), c.member_on + sl.m0, rows,
          sl.D.M);
    });
    CUDA_CHECK(cudaGetLastError());
    e.launches++;
  }
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

// The closure features of the group's current member states (file edge order, rows
// e * M + m) into the device array X (rows x 24 BF16), normalized with `norm`.
int trisk_ensemble_features(TriskEnsemble* ens, int32_t group, void* X, const double* norm,
                            const float* geometry) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!X || !norm || !geometry) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  EnsembleGroup& G = group_ref(e, group);
  if (reinterpret_cast<uintptr_t>(X) % 16) throw Error(TRISK_ERR_ARGUMENT, "X must be 16-byte aligned");
  TriskModel& m = *G.m;
  if (m.pv != PVM_TRISK) throw Error(TRISK_ERR_UNSUPPORTED, "the closure's features need the TRiSK PV flux");
  DeviceGuard guard(e.device);
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
  order_after_caller(e.stream, e.caller_ev);  // X may still be read by the caller
  for (const Slice& sl : e.slices) {
    if (sl.group != group) continue;
    const GroupDesc& D = sl.D;
    const int M = D.M;
    const int64_t rows = m.ne * (int64_t)M;
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
        kg_features<R><<<(unsigned)cdiv(rows, 256), 256, 0, e.stream>>>(
            D.T, W, u, M, geom, N, static_cast<__nv_bfloat16*>(X), map, rows, G.M, sl.m0);
      });
    });
    CUDA_CHECK(cudaGetLastError());
    e.launches += 3;
  }
  CUDA_CHECK(cudaFreeAsync(geom, e.stream));
  CUDA_CHECK(cudaFreeAsync(map, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

// Total energy sum_i A_i h_i (K_i + g h_i / 2) of every member of the group (host, M values).
int trisk_ensemble_energy(TriskEnsemble* ens, int32_t group, double* energies) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  if (!energies) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  EnsembleGroup& G = group_ref(e, group);
  TriskModel& m = *G.m;
  DeviceGuard guard(e.device);
  if (!e.energy) e.energy = e.alloc<double>(e.max_members);
  const int nblocks = (int)cdiv(m.nc, 256);
  if (e.energy_partials_size < (size_t)nblocks * G.M) {  // grown on demand, kept for later calls
    e.energy_partials_size = (size_t)nblocks * G.M;
    e.energy_partials = e.alloc<double>(e.energy_partials_size);
  }
  const int B = 128;
  for (const Slice& sl : e.slices) {
    if (sl.group != group) continue;
    const GroupDesc& D = sl.D;
    const int M = D.M;
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
        kg_sum_rows<<<(unsigned)M, 256, 0, e.stream>>>(e.energy_partials, nblocks, e.energy + sl.m0);
      });
    });
    CUDA_CHECK(cudaGetLastError());
    e.launches += 4;
  }
  CUDA_CHECK(cudaMemcpyAsync(energies, e.energy, G.M * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
  CUDA_CHECK(cudaStreamSynchronize(e.stream));
  TRISK_API_END
}

int trisk_ensemble_closure_check(TriskEnsemble* ens) {
  TRISK_API_BEGIN
  TriskEnsemble& e = *checked_e(ens);
  DeviceGuard guard(e.device);
  for (EnsembleGroup& G : e.groups)
    if (G.cl.net) closure_check(G.cl.net);
  TRISK_API_END
}

}  // extern "C"
