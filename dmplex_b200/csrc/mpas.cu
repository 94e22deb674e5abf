// The horizontal operators of dmplex.jl's 3-D MPAS-Gassmann dycore: slow_tendencies! for flat
// ground (src/Nonhydrostatic/MPAS/Gassmann/Stepping.jl:22-56) — the kernels of
// src/Nonhydrostatic/MPAS/Operators.jl and vn_tendency_kernel! (Tendencies.jl:38-75) — in five
// fused launches over (entity, level), the last two side by side on two streams:
//
//   1 vertices  vertex_pv_kernel! + vertex_kinetic_kernel!         (zeta_v, rho_v, q_v, K_v)
//   2 cells     diagnose_kernel! + cell_from_vertex_kernel! + w_kinetic_kernel!  (theta, pi, K)
//   3 edges     edge_pv_kernel! + edge_density_kernel! + eta_kernel!  (q_e, rho_e, F_s, eta)
//   4 cells     w_tendency_vi_kernel! or w_tendency_kernel!        (t_w)
//   5 edges     vn_tendency_kernel!                                 (t_vn)
//
// Fields stay in the reference's layout, a Julia (n, nlev) array = level slabs with the
// horizontal index fastest, so a warp of consecutive entities reads and writes whole lines of
// one level. Each thread takes one entity and a run of levels: its neighbour indices and
// weights are loaded once (registers) and reused for every level, the role of the reference's
// blocks of 32 points x 8 levels. Tables arrive 1-based, (entity, k) ordered (the TRiSK
// tables edge-first, as the reference holds them) and are uploaded as 0-based int32 / FP64
// [k][entity] structure-of-arrays. Every sum keeps the reference's order and association and
// the build does not contract to FMA, so results equal the CPU restatement bit for bit (the
// Exner pressure uses CUDA's pow).
#include <algorithm>
#include <utility>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "model.hpp"

using namespace trisk;

namespace {

constexpr int MCW = 10;  // edges per cell
constexpr int MVW = 4;   // edges (cells) per vertex
constexpr int MNT = 18;  // TRiSK neighbours per edge
constexpr int MB = 128;  // threads (entities) per block

// src/Nonhydrostatic/Common/Constants.jl:12-15
constexpr double RD = 287.0;
constexpr double CPD = 1004.0;
constexpr double CVD = CPD - RD;
constexpr double P0 = 1.0e5;

struct MpasTables {
  int32_t nc, ne, nv, nlev, ldc, lde, ldv, cw, vw, nt;
  int32_t vk, iap_pv, vertical, five_band;
  const int32_t* cell_edges;  // cw x ldc
  const int32_t* kcv;         // cw x ldc: cells' vertices of the vertex kinetic energy
  const double* kinetic;      // cw x ldc
  const double* inner;        // cw x ldc
  const double* kites;        // cw x ldc
  const int32_t* edge_cells;  // 2 x lde
  const int32_t* edge_vertices;
  const double* edge_weight;  // 2 x lde
  const double* rhombus;      // 2 x lde
  const double* inverse_dual;  // lde
  const double* edge_coriolis;
  const int32_t* vertex_edges;  // vw x ldv
  const int32_t* vertex_cells;
  const double* curl;  // vw x ldv
  const double* vertex_weight;
  const double* vk_weights;
  const double* coriolis;  // ldv
  const int32_t* ti;       // 3 x nt x lde
  const double* trisk;     // nt x lde
  const double* dz_c;      // nlev x nc
  const double* dzh_c;     // (nlev + 1) x nc
  const double* wlow;      // (nlev + 1) x nc
  const double* dz_e;      // nlev x ne
  const double* dzh_e;     // (nlev + 1) x ne
  double* Kh;              // nlev x nc: K without K_w (five-band solver only)
};

struct MpasFieldsDev {
  const double *vn, *w, *rho, *rt;
  double *theta, *exner, *K, *Kv, *qv, *zv, *rv, *qe, *rhoe, *Fs, *eta, *tvn, *tw;
};

__device__ __forceinline__ size_t at(int k, int n, int i) { return (size_t)k * n + i; }

// 1: vertex_pv_kernel! (Operators.jl:88-102) and vertex_kinetic_kernel! (:18-25)
template <bool VK>
__global__ void __launch_bounds__(MB) k_mpas_vertex(MpasTables T, MpasFieldsDev F, int lpt) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= T.nv) return;
  const int k0 = blockIdx.y * lpt, k1 = min(k0 + lpt, T.nlev);
  int ve[MVW], vc[MVW];
  double cu[MVW], wt[MVW], kw[VK ? MVW : 1];
#pragma unroll
  for (int j = 0; j < MVW; ++j)
    if (j < T.vw) {
      ve[j] = T.vertex_edges[j * T.ldv + v];
      vc[j] = T.vertex_cells[j * T.ldv + v];
      cu[j] = T.curl[j * T.ldv + v];
      wt[j] = T.vertex_weight[j * T.ldv + v];
      if constexpr (VK) kw[j] = T.vk_weights[j * T.ldv + v];
    }
  const double f = T.coriolis[v];
  for (int k = k0; k < k1; ++k) {
    const double* vn = F.vn + (size_t)k * T.ne;
    const double* rho = F.rho + (size_t)k * T.nc;
    double z = 0.0, h = 0.0;
#pragma unroll
    for (int j = 0; j < MVW; ++j)
      if (j < T.vw) z += cu[j] * vn[ve[j]];
#pragma unroll
    for (int j = 0; j < MVW; ++j)
      if (j < T.vw) h += wt[j] * rho[vc[j]];
    F.zv[at(k, T.nv, v)] = z;
    F.rv[at(k, T.nv, v)] = h;
    F.qv[at(k, T.nv, v)] = (z + f) / h;
    if constexpr (VK) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < MVW; ++j)
        if (j < T.vw) {
          const double x = vn[ve[j]];
          s += kw[j] * (x * x);
        }
      F.Kv[at(k, T.nv, v)] = s;
    }
  }
}

// 2: diagnose_kernel! (:6-15), cell_from_vertex_kernel! (:28-35), w_kinetic_kernel! (:38-41)
template <bool VK>
__global__ void __launch_bounds__(MB) k_mpas_cell(MpasTables T, MpasFieldsDev F, int lpt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.nc) return;
  const int k0 = blockIdx.y * lpt, k1 = min(k0 + lpt, T.nlev);
  int ce[MCW], cv[VK ? MCW : 1];
  double kin[MCW], kt[VK ? MCW : 1];
#pragma unroll
  for (int j = 0; j < MCW; ++j)
    if (j < T.cw) {
      ce[j] = T.cell_edges[j * T.ldc + i];
      kin[j] = T.kinetic[j * T.ldc + i];
      if constexpr (VK) {
        cv[j] = T.kcv[j * T.ldc + i];
        kt[j] = T.kites[j * T.ldc + i];
      }
    }
  for (int k = k0; k < k1; ++k) {
    const double* vn = F.vn + (size_t)k * T.ne;
    const size_t o = at(k, T.nc, i);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < MCW; ++j)
      if (j < T.cw) {
        const double x = vn[ce[j]];
        s += kin[j] * (x * x);
      }
    double K = s;
    const double r = F.rho[o], rt = F.rt[o];
    F.theta[o] = rt / r;
    F.exner[o] = pow(RD * rt / P0, RD / CVD);
    if constexpr (VK) {
      const double* Kv = F.Kv + (size_t)k * T.nv;
      double sv = 0.0;
#pragma unroll
      for (int j = 0; j < MCW; ++j)
        if (j < T.cw) sv += kt[j] * Kv[cv[j]];
      K = K + sv;
    }
    if (T.vertical > 0) {
      const double wl = F.w[at(k, T.nc, i)], wu = F.w[at(k + 1, T.nc, i)];
      const double kwv =
          (T.dzh_c[at(k, T.nc, i)] * (wl * wl) + T.dzh_c[at(k + 1, T.nc, i)] * (wu * wu)) / (4 * T.dz_c[o]);
      if (T.five_band) T.Kh[o] = K;
      K = K + kwv;
    }
    F.K[o] = K;
  }
}

// 3: edge_pv_kernel! (:104-115), edge_density_kernel! (:55-63), eta_kernel! (:44-52); rows
// 0..nlev: layers below nlev, interfaces at every row
__global__ void __launch_bounds__(MB) k_mpas_edge(MpasTables T, MpasFieldsDev F, int lpt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T.ne) return;
  const int k0 = blockIdx.y * lpt, k1 = min(k0 + lpt, T.nlev + 1);
  const int l = T.edge_cells[e], r = T.edge_cells[T.lde + e];
  const int v1 = T.edge_vertices[e], v2 = T.edge_vertices[T.lde + e];
  const double w0 = T.edge_weight[e], w1 = T.edge_weight[T.lde + e];
  const double r0 = T.rhombus[e], r1 = T.rhombus[T.lde + e];
  const double fe = T.edge_coriolis[e], invd = T.inverse_dual[e];
  for (int k = k0; k < k1; ++k) {
    if (k < T.nlev) {
      const size_t o = at(k, T.ne, e);
      const double* rho = F.rho + (size_t)k * T.nc;
      const double re = w0 * rho[l] + w1 * rho[r];
      F.rhoe[o] = re;
      F.Fs[o] = re * F.vn[o];
      if (T.iap_pv) {
        const double* zv = F.zv + (size_t)k * T.nv;
        const double* rv = F.rv + (size_t)k * T.nv;
        const double z = r0 * zv[v1] + r1 * zv[v2];
        const double h = r0 * rv[v1] + r1 * rv[v2];
        F.qe[o] = (z + fe) / h;
      } else {
        const double* qv = F.qv + (size_t)k * T.nv;
        F.qe[o] = (qv[v1] + qv[v2]) / 2;
      }
    }
    if (T.vertical > 0) {
      double x = 0.0;
      if (k >= 1 && k <= T.nlev - 1) {
        const double* w = F.w + (size_t)k * T.nc;
        x = (F.vn[at(k, T.ne, e)] - F.vn[at(k - 1, T.ne, e)]) / T.dzh_e[at(k, T.ne, e)] - (w[r] - w[l]) * invd;
      }
      F.eta[at(k, T.ne, e)] = x;
    }
  }
}

// 4: w_tendency_vi_kernel! (:69-86) with the vector-invariant vertical advection, else
// w_tendency_kernel! (:118-133); rows 0..nlev (interfaces), zero at ground and top
template <bool VI>
__device__ __forceinline__ void wtend_rows(const MpasTables& T, const MpasFieldsDev& F, int i, int k0, int k1) {
  int ce[MCW];
  double cwt[MCW];
  int el[VI ? 1 : MCW], er[VI ? 1 : MCW];
  double ei[VI ? 1 : MCW];
#pragma unroll
  for (int j = 0; j < MCW; ++j)
    if (j < T.cw) {
      ce[j] = T.cell_edges[j * T.ldc + i];
      cwt[j] = VI ? T.inner[j * T.ldc + i] : T.kinetic[j * T.ldc + i];
      if constexpr (!VI) {
        el[j] = T.edge_cells[ce[j]];
        er[j] = T.edge_cells[T.lde + ce[j]];
        ei[j] = T.inverse_dual[ce[j]];
      }
    }
  const bool mw = T.vertical == 2;
  const double* Kc = T.five_band ? T.Kh : F.K;
  for (int k = k0; k < k1; ++k) {
    const size_t o = at(k, T.nc, i);
    if (k == 0 || k == T.nlev) {
      F.tw[o] = 0.0;
      continue;
    }
    const double* vl = F.vn + (size_t)(k - 1) * T.ne;
    const double* vu = F.vn + (size_t)k * T.ne;
    double s = 0.0;
    if constexpr (VI) {
      const double wl = T.wlow[o];
      const double* eta = F.eta + (size_t)k * T.ne;
      const double* pl = F.rhoe + (size_t)(k - 1) * T.ne;
      const double* pu = F.rhoe + (size_t)k * T.ne;
#pragma unroll
      for (int j = 0; j < MCW; ++j)
        if (j < T.cw) {
          const int e = ce[j];
          const double rl = mw ? pl[e] : 1.0, ru = mw ? pu[e] : 1.0;
          s += cwt[j] * eta[e] * (rl * vl[e] + ru * vu[e]) / (2 * (wl * rl + (1 - wl) * ru));
        }
      F.tw[o] = s - (Kc[o] - Kc[at(k - 1, T.nc, i)]) / T.dzh_c[o];
    } else {
      const double* w = F.w + (size_t)k * T.nc;
#pragma unroll
      for (int j = 0; j < MCW; ++j)
        if (j < T.cw) {
          const int e = ce[j];
          const double v = (vl[e] + vu[e]) / 2;
          s += 2 * cwt[j] * v * (w[er[j]] - w[el[j]]) * ei[j];
        }
      F.tw[o] = -s - w[i] * (F.w[at(k + 1, T.nc, i)] - F.w[at(k - 1, T.nc, i)]) /
                         (T.dz_c[at(k - 1, T.nc, i)] + T.dz_c[o]);
    }
  }
}

// w~ = M_e / rho_e at interface j (edge_w, Tendencies.jl:4-12)
__device__ __forceinline__ double edge_w(const MpasTables& T, const MpasFieldsDev& F, int l, int r, double w0,
                                         double w1, int j, bool mw) {
  double hl = 1.0, hr = 1.0;
  if (mw) {
    const double al = T.wlow[at(j, T.nc, l)], ar = T.wlow[at(j, T.nc, r)];
    hl = al * F.rho[at(j - 1, T.nc, l)] + (1 - al) * F.rho[at(j, T.nc, l)];
    hr = ar * F.rho[at(j - 1, T.nc, r)] + (1 - ar) * F.rho[at(j, T.nc, r)];
  }
  const double M = w0 * hl * F.w[at(j, T.nc, l)] + w1 * hr * F.w[at(j, T.nc, r)];
  return M / (w0 * hl + w1 * hr);
}

// 5: vn_tendency_kernel! (Tendencies.jl:38-75), flat ground (oro = 0). The TRiSK sums of
// LPT levels are accumulated neighbour by neighbour so that each table entry is read once.
template <int LPT, bool VI>
__device__ __forceinline__ void vn_rows(const MpasTables& T, const MpasFieldsDev& F, int e, int k0, double pressure) {
  const int k1 = min(k0 + LPT, T.nlev);
  double s[LPT];
#pragma unroll
  for (int q = 0; q < LPT; ++q) s[q] = 0.0;
  for (int j = 0; j < T.nt; ++j) {
    const double wt = T.trisk[(size_t)j * T.lde + e];
    const int a = T.ti[((size_t)0 * T.nt + j) * T.lde + e];
    const int b = T.ti[((size_t)1 * T.nt + j) * T.lde + e];
    const int c = T.ti[((size_t)2 * T.nt + j) * T.lde + e];
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int k = k0 + q;
      if (k < k1) {
        const size_t base = (size_t)k * T.ne;
        const double qb = F.qe[base + b];
        const double qc = c == b ? qb : F.qe[base + c];  // the rhombus PV of one edge, twice
        s[q] += wt * F.Fs[base + a] * (qb + qc);
      }
    }
  }
  const int l = T.edge_cells[e], r = T.edge_cells[T.lde + e];
  const double w0 = T.edge_weight[e], w1 = T.edge_weight[T.lde + e], invd = T.inverse_dual[e];
  const bool mw = T.vertical == 2;
  double Wl = 0.0;
  if (VI && k0 > 0) Wl = edge_w(T, F, l, r, w0, w1, k0, mw);
#pragma unroll
  for (int q = 0; q < LPT; ++q) {
    const int k = k0 + q;
    if (k >= k1) break;
    const double* th = F.theta + (size_t)k * T.nc;
    const double* K = F.K + (size_t)k * T.nc;
    const double te = w0 * th[l] + w1 * th[r];
    double t = s[q] - invd * (K[r] - K[l]);
    if (pressure > 0) {
      const double* pe = F.exner + (size_t)k * T.nc;
      const double dpi = (pe[r] - pe[l]) * invd;
      t -= pressure * (CPD * te * dpi);
    }
    const size_t o = at(k, T.ne, e);
    if constexpr (VI) {
      const double Wu = k < T.nlev - 1 ? edge_w(T, F, l, r, w0, w1, k + 1, mw) : 0.0;
      F.tvn[o] = t - (T.dzh_e[o] * F.eta[o] * Wl + T.dzh_e[at(k + 1, T.ne, e)] * F.eta[at(k + 1, T.ne, e)] * Wu) /
                         (2 * T.dz_e[o]);
      Wl = Wu;
    } else {
      const double* wlo = F.w + (size_t)k * T.nc;
      const double* wup = F.w + (size_t)(k + 1) * T.nc;
      const double we = (wlo[l] + wlo[r] + wup[l] + wup[r]) / 4;
      const double vc = F.vn[o];
      const double vlow = k > 0 ? (F.vn[at(k - 1, T.ne, e)] + vc) / 2 : vc;
      const double vup = k < T.nlev - 1 ? (vc + F.vn[at(k + 1, T.ne, e)]) / 2 : vc;
      F.tvn[o] = t - we * (vup - vlow) / T.dz_e[o];
    }
  }
}

template <bool VI>
__global__ void __launch_bounds__(MB) k_mpas_wtend(MpasTables T, MpasFieldsDev F, int lpt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = blockIdx.y * lpt;
  if (i < T.nc) wtend_rows<VI>(T, F, i, k0, min(k0 + lpt, T.nlev + 1));
}

template <int LPT, bool VI>
__global__ void __launch_bounds__(MB) k_mpas_vn(MpasTables T, MpasFieldsDev F, double pressure) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < T.ne) vn_rows<LPT, VI>(T, F, e, blockIdx.y * LPT, pressure);
}

}  // namespace

struct TriskMpas {
  int device = 0;
  int lpt = 8;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // the w tendency beside the vn tendency
  cudaEvent_t caller_ev = nullptr, fork_ev = nullptr, join_ev = nullptr;
  MpasTables T{};
  std::vector<void*> allocations;
  int64_t launches = 0;

  ~TriskMpas() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (cudaStream_t s : {stream, side})
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    for (cudaEvent_t e : {caller_ev, fork_ev, join_ev})
      if (e) cudaEventDestroy(e);
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
  template <class X>
  const X* upload(const std::vector<X>& v) {
    X* d = alloc<X>(v.size());
    CUDA_CHECK(cudaMemcpy(d, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
    return d;
  }
  template <class X>
  const X* upload(const X* p, size_t count, const char* name) {
    if (!p) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
    X* d = alloc<X>(count);
    CUDA_CHECK(cudaMemcpy(d, p, count * sizeof(X), cudaMemcpyHostToDevice));
    return d;
  }
};

namespace {

// 1-based (entity, k) int64 table -> 0-based int32 [k][entity] (ld-padded), indices checked
std::vector<int32_t> index_table(const int64_t* tab, int w, int64_t n, int64_t ld, int64_t range, const char* name) {
  if (!tab) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
  std::vector<int32_t> out((size_t)w * ld, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int k = 0; k < w; ++k) {
      const int64_t x = tab[j * w + k];
      if (x < 1 || x > range) throw Error(TRISK_ERR_TABLE, std::string(name) + ": index out of range");
      out[k * ld + j] = (int32_t)(x - 1);
    }
  return out;
}

std::vector<double> weight_table(const double* tab, int w, int64_t n, int64_t ld, const char* name) {
  if (!tab) throw Error(TRISK_ERR_ARGUMENT, std::string(name) + " is NULL");
  std::vector<double> out((size_t)w * ld, 0.0);
  for (int64_t j = 0; j < n; ++j)
    for (int k = 0; k < w; ++k) out[k * ld + j] = tab[j * w + k];
  return out;
}

TriskMpas* checked_mpas(TriskMpas* m) {
  if (!m) throw Error(TRISK_ERR_ARGUMENT, "operators handle is NULL");
  return m;
}

template <typename... KArgs, typename... Args>
void mlaunch(TriskMpas& m, cudaStream_t st, void (*kernel)(KArgs...), int64_t n, int64_t rows, int lpt,
             Args&&... args) {
  if (n <= 0 || rows <= 0) return;
  dim3 grid((unsigned)cdiv(n, MB), (unsigned)cdiv(rows, lpt));
  kernel<<<grid, MB, 0, st>>>(std::forward<Args>(args)...);
  CUDA_CHECK(cudaGetLastError());
  m.launches++;
}

template <int LPT>
void launch_vn(TriskMpas& m, const MpasFieldsDev& F, double pressure) {
  if (m.T.vertical > 0)
    mlaunch(m, m.stream, k_mpas_vn<LPT, true>, m.T.ne, m.T.nlev, LPT, m.T, F, pressure);
  else
    mlaunch(m, m.stream, k_mpas_vn<LPT, false>, m.T.ne, m.T.nlev, LPT, m.T, F, pressure);
}

void slow_tendencies(TriskMpas& m, const MpasFieldsDev& F, double pressure) {
  const MpasTables& T = m.T;
  const int lpt = m.lpt;
  if (T.vk) {
    mlaunch(m, m.stream, k_mpas_vertex<true>, T.nv, T.nlev, lpt, T, F, lpt);
    mlaunch(m, m.stream, k_mpas_cell<true>, T.nc, T.nlev, lpt, T, F, lpt);
  } else {
    mlaunch(m, m.stream, k_mpas_vertex<false>, T.nv, T.nlev, lpt, T, F, lpt);
    mlaunch(m, m.stream, k_mpas_cell<false>, T.nc, T.nlev, lpt, T, F, lpt);
  }
  mlaunch(m, m.stream, k_mpas_edge, T.ne, T.nlev + 1, lpt, T, F, lpt);
  // phases 4 and 5 read only what 1-3 wrote: the w tendency runs on a second stream beside
  // the vn tendency, joined before the call ends
  CUDA_CHECK(cudaEventRecord(m.fork_ev, m.stream));
  CUDA_CHECK(cudaStreamWaitEvent(m.side, m.fork_ev, 0));
  if (T.vertical > 0)
    mlaunch(m, m.side, k_mpas_wtend<true>, T.nc, T.nlev + 1, lpt, T, F, lpt);
  else
    mlaunch(m, m.side, k_mpas_wtend<false>, T.nc, T.nlev + 1, lpt, T, F, lpt);
  CUDA_CHECK(cudaEventRecord(m.join_ev, m.side));
  switch (lpt) {
    case 1: launch_vn<1>(m, F, pressure); break;
    case 2: launch_vn<2>(m, F, pressure); break;
    case 4: launch_vn<4>(m, F, pressure); break;
    case 16: launch_vn<16>(m, F, pressure); break;
    default: launch_vn<8>(m, F, pressure); break;
  }
  CUDA_CHECK(cudaStreamWaitEvent(m.stream, m.join_ev, 0));
}

MpasFieldsDev device_fields(const TriskMpas& m, const TriskMpasFields* f) {
  if (!f) throw Error(TRISK_ERR_ARGUMENT, "fields are NULL");
  const void* need[] = {f->vn, f->w, f->rho, f->rhotheta, f->theta, f->exner, f->K, f->qv, f->zetav,
                        f->rhov, f->qe, f->rhoe, f->Fs, f->eta, f->tvn, f->tw};
  for (const void* p : need)
    if (!p || !is_device_pointer(p)) throw Error(TRISK_ERR_ARGUMENT, "every field must be a device pointer");
  if (m.T.vk && (!f->Kv || !is_device_pointer(f->Kv)))
    throw Error(TRISK_ERR_ARGUMENT, "Kv must be a device pointer (vertex kinetic energy)");
  MpasFieldsDev F{};
  F.vn = f->vn;
  F.w = f->w;
  F.rho = f->rho;
  F.rt = f->rhotheta;
  F.theta = f->theta;
  F.exner = f->exner;
  F.K = f->K;
  F.Kv = f->Kv;
  F.qv = f->qv;
  F.zv = f->zetav;
  F.rv = f->rhov;
  F.qe = f->qe;
  F.rhoe = f->rhoe;
  F.Fs = f->Fs;
  F.eta = f->eta;
  F.tvn = f->tvn;
  F.tw = f->tw;
  return F;
}

}  // namespace

extern "C" {

int trisk_mpas_create(const TriskMpasTables* t, int32_t device, int32_t levels_per_thread, TriskMpas** out) {
  TRISK_API_BEGIN
  if (!t || !out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (t->nc < 1 || t->ne < 1 || t->nv < 1 || t->nlev < 2)
    throw Error(TRISK_ERR_ARGUMENT, "need cells, edges, vertices and at least two layers");
  if (t->cw < 3 || t->cw > MCW || t->vw < 1 || t->vw > MVW || t->nt < 1 || t->nt > MNT)
    throw Error(TRISK_ERR_UNSUPPORTED, "tables wider than the kernels handle (10 edges per cell, 4 per vertex, "
                                       "18 TRiSK neighbours)");
  if (t->vertical < 0 || t->vertical > 2) throw Error(TRISK_ERR_ARGUMENT, "vertical must be 0, 1 or 2");
  if (t->five_band && t->vertical == 0)
    throw Error(TRISK_ERR_ARGUMENT, "the five-band solver needs the vector-invariant vertical advection");
  const int lpt = levels_per_thread == 0 ? 8 : levels_per_thread;
  if (lpt != 1 && lpt != 2 && lpt != 4 && lpt != 8 && lpt != 16)
    throw Error(TRISK_ERR_ARGUMENT, "levels_per_thread must be 0 (default), 1, 2, 4, 8 or 16");
  const int64_t cells_levels = t->nc * (t->nlev + 1), edges_levels = t->ne * (t->nlev + 1);
  if (t->ne >= (1LL << 30) || edges_levels >= (1LL << 40) || cells_levels >= (1LL << 40))
    throw Error(TRISK_ERR_UNSUPPORTED, "mesh too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw Error(TRISK_ERR_CUDA, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) throw Error(TRISK_ERR_ARGUMENT, "no such CUDA device");
  auto m = std::make_unique<TriskMpas>();
  m->device = device;
  m->lpt = lpt;
  DeviceGuard guard(device);
  const int64_t nc = t->nc, ne = t->ne, nv = t->nv, nl = t->nlev;
  const int64_t ldc = round_up(nc, 32), lde = round_up(ne, 32), ldv = round_up(nv, 32);
  MpasTables& T = m->T;
  T.nc = (int32_t)nc;
  T.ne = (int32_t)ne;
  T.nv = (int32_t)nv;
  T.nlev = (int32_t)nl;
  T.ldc = (int32_t)ldc;
  T.lde = (int32_t)lde;
  T.ldv = (int32_t)ldv;
  T.cw = t->cw;
  T.vw = t->vw;
  T.nt = t->nt;
  T.vk = t->vertex_kinetic != 0;
  T.iap_pv = t->iap_pv != 0;
  T.vertical = t->vertical;
  T.five_band = t->five_band != 0;
  T.cell_edges = m->upload(index_table(t->cell_edges, t->cw, nc, ldc, ne, "cell_edges"));
  T.kinetic = m->upload(weight_table(t->kinetic, t->cw, nc, ldc, "kinetic"));
  T.inner = m->upload(weight_table(t->inner, t->cw, nc, ldc, "inner"));
  if (T.vk) {
    T.kcv = m->upload(index_table(t->vk_cell_vertices, t->cw, nc, ldc, nv, "vk_cell_vertices"));
    T.kites = m->upload(weight_table(t->vk_kites, t->cw, nc, ldc, "vk_kites"));
    T.vk_weights = m->upload(weight_table(t->vk_weights, t->vw, nv, ldv, "vk_weights"));
  }
  T.edge_cells = m->upload(index_table(t->edge_cells, 2, ne, lde, nc, "edge_cells"));
  T.edge_vertices = m->upload(index_table(t->edge_vertices, 2, ne, lde, nv, "edge_vertices"));
  T.edge_weight = m->upload(weight_table(t->edge_weight, 2, ne, lde, "edge_weight"));
  T.rhombus = m->upload(weight_table(t->rhombus, 2, ne, lde, "rhombus"));
  T.inverse_dual = m->upload(weight_table(t->inverse_dual, 1, ne, lde, "inverse_dual"));
  T.edge_coriolis = m->upload(weight_table(t->edge_coriolis, 1, ne, lde, "edge_coriolis"));
  T.vertex_edges = m->upload(index_table(t->vertex_edges, t->vw, nv, ldv, ne, "vertex_edges"));
  T.vertex_cells = m->upload(index_table(t->vertex_cells, t->vw, nv, ldv, nc, "vertex_cells"));
  T.curl = m->upload(weight_table(t->curl, t->vw, nv, ldv, "curl"));
  T.vertex_weight = m->upload(weight_table(t->vertex_weight, t->vw, nv, ldv, "vertex_weight"));
  T.coriolis = m->upload(weight_table(t->coriolis, 1, nv, ldv, "coriolis"));
  // TRiSK tables, edge-first in the reference: trisk[e + ne j], trisk_index[e + ne (j + nt c)]
  if (!t->trisk || !t->trisk_index) throw Error(TRISK_ERR_ARGUMENT, "trisk tables are NULL");
  {
    std::vector<double> tw((size_t)t->nt * lde, 0.0);
    std::vector<int32_t> ti((size_t)3 * t->nt * lde, 0);
    for (int j = 0; j < t->nt; ++j)
      for (int64_t e = 0; e < ne; ++e) {
        tw[(size_t)j * lde + e] = t->trisk[(size_t)j * ne + e];
        for (int c = 0; c < 3; ++c) {
          const int32_t x = t->trisk_index[((size_t)c * t->nt + j) * ne + e];
          if (x < 1 || x > ne) throw Error(TRISK_ERR_TABLE, "trisk_index: index out of range");
          ti[((size_t)c * t->nt + j) * lde + e] = x - 1;
        }
      }
    T.trisk = m->upload(tw);
    T.ti = m->upload(ti);
  }
  T.dz_c = m->upload(t->dz_cells, (size_t)nl * nc, "dz_cells");
  T.dzh_c = m->upload(t->dzh_cells, (size_t)(nl + 1) * nc, "dzh_cells");
  T.wlow = m->upload(t->wlow, (size_t)(nl + 1) * nc, "wlow");
  T.dz_e = m->upload(t->dz_edges, (size_t)nl * ne, "dz_edges");
  T.dzh_e = m->upload(t->dzh_edges, (size_t)(nl + 1) * ne, "dzh_edges");
  T.Kh = T.five_band ? m->alloc<double>((size_t)nl * nc) : nullptr;
  CUDA_CHECK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreateWithFlags(&m->caller_ev, cudaEventDisableTiming));
  CUDA_CHECK(cudaEventCreateWithFlags(&m->fork_ev, cudaEventDisableTiming));
  CUDA_CHECK(cudaEventCreateWithFlags(&m->join_ev, cudaEventDisableTiming));
  CUDA_CHECK(cudaDeviceSynchronize());
  *out = m.release();
  TRISK_API_END
}

void trisk_mpas_destroy(TriskMpas* ops) { delete ops; }

int trisk_mpas_slow_tendencies_async(TriskMpas* ops, const TriskMpasFields* fields, double pressure) {
  TRISK_API_BEGIN
  TriskMpas& m = *checked_mpas(ops);
  if (!std::isfinite(pressure)) throw Error(TRISK_ERR_ARGUMENT, "pressure must be finite");
  DeviceGuard guard(m.device);
  const MpasFieldsDev F = device_fields(m, fields);
  order_after_caller(m.stream, m.caller_ev);
  slow_tendencies(m, F, pressure);
  TRISK_API_END
}

int trisk_mpas_slow_tendencies(TriskMpas* ops, const TriskMpasFields* fields, double pressure) {
  TRISK_API_BEGIN
  TriskMpas& m = *checked_mpas(ops);
  const int status = trisk_mpas_slow_tendencies_async(ops, fields, pressure);
  if (status != TRISK_OK) return status;
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int trisk_mpas_stream(TriskMpas* ops, void** stream) {
  TRISK_API_BEGIN
  TriskMpas& m = *checked_mpas(ops);
  if (!stream) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *stream = (void*)m.stream;
  TRISK_API_END
}

int trisk_mpas_synchronize(TriskMpas* ops) {
  TRISK_API_BEGIN
  TriskMpas& m = *checked_mpas(ops);
  DeviceGuard guard(m.device);
  CUDA_CHECK(cudaStreamSynchronize(m.stream));
  TRISK_API_END
}

int64_t trisk_mpas_launch_count(TriskMpas* ops) { return ops ? ops->launches : -1; }

}  // extern "C"
