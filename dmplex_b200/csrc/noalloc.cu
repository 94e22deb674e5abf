// An entry point for callers that must not have the library allocate device memory.
//
// Who needs it: a host that owns every device byte through its own allocator or memory
// pool (the Julia side of a drop-in, whose arrays live in CUDA.jl's pool, or an
// application with a fixed memory budget), or that calls from a region where cudaMalloc
// is not allowed (while it is capturing a stream into a CUDA graph). Such a caller can
// pass its own device arrays in and out, but cannot give the library scratch space.
//
// trisk_weighted_sum_noalloc computes sum_i a_i b_i (total_mass = dot(A, h) of the model)
// from caller-owned device vectors. Its partial sums, the only scratch the reduction
// needs, live in a file-scope static device array instead of a cudaMalloc'd buffer, so
// the call allocates nothing: no cudaMalloc, no cudaFree, no allocating library routine.
#include <cuda_runtime.h>

#include <mutex>

#include "common.hpp"

namespace {

constexpr int NOALLOC_BLOCK = 256, NOALLOC_PER_THREAD = 8;
constexpr int NOALLOC_MAX_PARTIALS = 8192;  // 64 KiB of device memory per GPU
constexpr int64_t NOALLOC_MAX_N = (int64_t)NOALLOC_MAX_PARTIALS * NOALLOC_BLOCK * NOALLOC_PER_THREAD;

// The scratch: every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_PARTIALS];

// Per-device address of g_noalloc_partials. In host code the symbol's name is only a
// host-side stand-in, not a device address, so it is looked up once per device.
std::mutex g_mutex;
double* g_scratch[256] = {nullptr};

double* scratch_on(int device) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (device < 0 || device >= 256) throw trisk::Error(TRISK_ERR_ARGUMENT, "device ordinal out of range");
  if (!g_scratch[device]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_partials);
    if (e != cudaSuccess || !p)
      throw trisk::Error(TRISK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch[device] = p;
  }
  return g_scratch[device];
}

__global__ void k_noalloc_partial(const double* a, const double* b, int64_t n, double* partials) {
  __shared__ double sm[NOALLOC_BLOCK];
  const int64_t base = (int64_t)blockIdx.x * NOALLOC_BLOCK * NOALLOC_PER_THREAD;
  double s = 0.0;
  for (int r = 0; r < NOALLOC_PER_THREAD; ++r) {
    const int64_t i = base + (int64_t)r * NOALLOC_BLOCK + threadIdx.x;
    if (i < n) s += a[i] * b[i];
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = NOALLOC_BLOCK / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
}

__global__ void k_noalloc_final(const double* partials, int nb, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += partials[i];
    *out = s;
  }
}

int device_of(const void* p, const char* name) {
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw trisk::Error(TRISK_ERR_ARGUMENT, std::string(name) + " is not a device pointer");
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
    throw trisk::Error(TRISK_ERR_ARGUMENT, std::string(name) + " is not a device pointer");
  return attr.device;
}

}  // namespace

extern "C" int trisk_weighted_sum_noalloc(const double* a, const double* b, int64_t n, double* out,
                                          void* stream) {
  TRISK_API_BEGIN
  if (!a || !b || !out) throw trisk::Error(TRISK_ERR_ARGUMENT, "NULL argument");
  if (n < 0) throw trisk::Error(TRISK_ERR_ARGUMENT, "n must be non-negative");
  if (n > NOALLOC_MAX_N)
    throw trisk::Error(TRISK_ERR_ARGUMENT, "n = " + std::to_string(n) + " exceeds the maximum " +
                                               std::to_string(NOALLOC_MAX_N) +
                                               " of trisk_weighted_sum_noalloc (its static scratch holds " +
                                               std::to_string(NOALLOC_MAX_PARTIALS) + " partial sums)");
  const int dev = device_of(a, "a");
  if (device_of(b, "b") != dev || device_of(out, "out") != dev)
    throw trisk::Error(TRISK_ERR_ARGUMENT, "a, b and out must be on the same device");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) throw trisk::Error(TRISK_ERR_CUDA, "cudaGetDevice failed");
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess) throw trisk::Error(TRISK_ERR_CUDA, "cudaSetDevice failed");
  try {
    double* partials = scratch_on(dev);
    const int nb = (int)((n + NOALLOC_BLOCK * NOALLOC_PER_THREAD - 1) / (NOALLOC_BLOCK * NOALLOC_PER_THREAD));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Every partial the final sum reads is written by this call first, so the scratch
    // left by an earlier call needs no clearing.
    if (nb > 0) k_noalloc_partial<<<nb, NOALLOC_BLOCK, 0, s>>>(a, b, n, partials);
    k_noalloc_final<<<1, 32, 0, s>>>(partials, nb, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw trisk::Error(TRISK_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  } catch (...) {
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    throw;
  }
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  TRISK_API_END
}
