// The model object behind the C ABI and the helpers the model and ensemble translation
// units share.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"

#define CUDA_CHECK(x)                                                                          \
  do {                                                                                         \
    cudaError_t err__ = (x);                                                                   \
    if (err__ != cudaSuccess)                                                                  \
      throw trisk::Error(TRISK_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(err__)); \
  } while (0)

namespace trisk {

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return cdiv(a, b) * b; }

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) CUDA_CHECK(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// true for device or managed memory, false for host memory (pageable or pinned)
bool is_device_pointer(const void* p);
// Orders `stream` after all work queued so far on the legacy default stream (and, by its
// semantics, on every blocking stream), so a caller's device buffer filled or still read on
// those streams (PyTorch's default stream among them) is safe to use from `stream`.
void order_after_caller(cudaStream_t stream, cudaEvent_t ev);

// dst[j] = src[idx[j]], j < n, on `stream`
void launch_gather(cudaStream_t stream, double* dst, const double* src, const int32_t* idx, int64_t n);

}  // namespace trisk

struct TriskClosure;
namespace trisk {
// The closure network's forward pass Y = MLP(X) enqueued on `stream` (no wait).
void closure_forward_on(TriskClosure* c, const void* X, int64_t n, float* Y, cudaStream_t stream);
// Throws TRISK_ERR_TIMEOUT if a bounded tensor-core wait of the network gave up.
void closure_check(TriskClosure* c);
int closure_device(const TriskClosure* c);
}  // namespace trisk

// 1-based copies of the index tables handed out through TriskCoefficients views.
struct CoefficientExport {
  std::vector<int64_t> t[9];
};

// Host-side premultiplied tables (the reference constructor's output), no device.
struct TriskTables {
  trisk::Coefficients C;
  CoefficientExport exported;
};

struct TriskModel {
  int device = 0;
  cudaStream_t stream = nullptr;
  int pv = 0, ke = 0;  // pv: the kernels' PvMode (PVM_GASSMANN_DERIVED when the table allows it)
  double alpha = 1.0, gravity = 1.0;
  int64_t nc = 0, ne = 0, nv = 0, N = 0;
  int64_t nc_own = -1, ne_own = -1;  // owned cells and edges come first (-1: all are owned)
  int block[3] = {128, 128, 128};  // threads per block of k_vertex, k_flux, k_tend
  bool use_graph = true, use_pdl = true, identity = true;
  // RK4 steps in one cooperative launch (k_rk4_persistent): for meshes that stay in L2
  bool persistent = false;
  int persistent_grid = 0;               // co-resident blocks of 256 threads
  unsigned* barrier = nullptr;           // arrivals, generation
  int* barrier_err = nullptr;            // a grid-barrier wait gave up
  trisk::Coefficients C;  // file numbering, 0-based (kept for export)
  CoefficientExport exported;
  std::vector<int32_t> cell_n2o, edge_n2o, vert_n2o, cell_o2n, edge_o2n, vert_o2n;
  std::vector<void*> allocations;
  trisk::DevTables T{};
  trisk::DevWork W{};
  double *y = nullptr, *acc = nullptr, *st = nullptr, *stage = nullptr, *dy = nullptr;
  int32_t *state_n2o = nullptr, *state_o2n = nullptr, *vertex_o2n = nullptr;
  double *area_c = nullptr, *area_v = nullptr, *partials = nullptr, *scalars = nullptr;
  int* flag = nullptr;
  cudaGraphExec_t graph = nullptr;
  double graph_dt = NAN;
  int64_t launches = 0;
  double table_bytes_unique = 0;
  double phase_bytes[3] = {0, 0, 0};
  double pv_table_bytes_saved = 0;  // k_tend bytes per launch the derived PV edges do not read
  cudaEvent_t caller_ev = nullptr;  // for order_after_caller
  char* table_base = nullptr;       // the packed table block (tendency phase's tables first)
  size_t table_block_bytes = 0;     // its part the kernels read
  size_t l2_keep_bytes = 0;         // prefix loaded with the L2 evict-last policy
  bool l2_window = false;           // plus a persisting access-policy window on every launch

  ~TriskModel() {
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
};
