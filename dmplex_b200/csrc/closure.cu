// Learned flux closure: an edge-local MLP 24 -> 64 -> 64 -> 2 (GELU) whose two hidden
// layers run on the 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared
// memory, FP32 accumulators in tensor memory), for inference and for training.
//
// There is no closure in the reference; the closure is this library's addition. The MLP reads
// 24 normalized features of an edge and returns two corrections (to the edge mass flux and
// to the edge momentum tendency).
//
// A CTA = 4 warps = 128 threads; a tile = 128 edges, thread t owns row t (TMEM lane t).
// Shared-memory operands use the no-swizzle "core matrix" layout (8 rows x 16 bytes, rows
// 16 bytes apart). A buffer tiled as
//     offset(r, c) = (c / 8) * CHUNK + (r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2
// is a K-major operand with rows r along M/N and columns c along K (SBO = 128, LBO =
// CHUNK), and the same bytes are an MN-major operand with c along M/N and r along K
// (SBO = CHUNK, LBO = 128). Forward GEMMs use the first view, backward GEMMs the second,
// so no operand is ever transposed in memory.
//
// Inference (k_mlp_forward): a persistent grid, several CTAs per SM, 64 TMEM columns each.
//   Z1 = X W1^T   M=128 N=64 K=32  (A = XH[:, 0:32], X padded with zeros; B = W1 K-major)
//   H1 = gelu(Z1 + b1) -> bf16 -> XH[:, 0:64]  (over X: MMA 1 has finished reading it)
//   Z2 = H1 W2^T  M=128 N=64 K=64  (same TMEM columns: Z1 has been read)
//   Y  = bf16(gelu(Z2 + b2)) W3^T + b3 on the CUDA cores (N = 2)
// Training (k_mlp_train): forward, backward and weight gradients of one tile per step:
//   forward    Z1 = X W1^T       M=128 N=64 K=32   (A = HX[:, 64:96] K-major, B = W1 K-major)
//              H1 = gelu(Z1 + b1) -> bf16 -> HX[:, 0:64]
//              Z2 = H1 W2^T      M=128 N=64 K=64   (A = HX[:, 0:64], B = W2 K-major)
//              H2 = gelu(Z2 + b2);  Y = H2 W3^T + b3 on the CUDA cores (N = 2)
//   backward   dH2 = (dY W3) * gelu'(Z2)                       CUDA cores -> DD[:, 0:64]
//              G = dH2 W2        M=128 N=64 K=64   (A = DD[:, 0:64] K-major, B = W2 MN-major)
//              dH1 = G * gelu'(Z1)                             -> DD[:, 64:128]
//              DW += DD^T [H1 | X]   M=128 N=96 K=128 (A = DD MN-major, B = HX MN-major):
//                   rows 0..63 x cols 0..63 = dW2, rows 64..127 x cols 64..87 = dW1
//   Tensor memory: Z1 at 0, Z2 (then G) at 64, DW at 128..224 (256 columns, two CTAs per SM).
//
// GELU is the tanh form of Hendrycks and Gimpel (2016), gelu(x) = x/2 (1 + tanh(sqrt(2/pi)
// (x + 0.044715 x^3))), with tanh on the special-function unit (tanh.approx.f32); it is the
// network's activation in training and inference alike, and the oracle's.
//
// Every tensor-core wait is bounded in time. A wait that gives up marks the CTA; at the next
// CTA-wide barrier every thread sees the mark and the CTA leaves its tile loop, waits (again
// bounded) for a tensor-core operation it committed and has not seen finish, frees its tensor
// memory and reports TRISK_ERR_TIMEOUT through a status word the host reads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "closure_mlp.cuh"
#include "model.hpp"

namespace trisk {
namespace closure {

// Inference: Y (n x 2) = MLP(X) over a persistent grid. expire_tile >= 0 names a tile whose
// first tensor-core operation is not issued, so its bounded wait runs out (the test of the
// give-up path); -1 in normal use.
__global__ void __launch_bounds__(TILE) k_mlp_forward(const __nv_bfloat16* __restrict__ X, int64_t n,
                                                      const ParamsBF16* __restrict__ wbf,
                                                      const Params* __restrict__ p, float* __restrict__ Y,
                                                      Status* status, int64_t expire_tile) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(16) InferStatic st;
  const int t = threadIdx.x;
  const int64_t ntiles = (n + TILE - 1) / TILE;
  if ((int64_t)blockIdx.x >= ntiles) return;
  const InferSmem S(smem);
  const uint32_t tmem = infer_setup(S, st, wbf, p);
  MmaWaits waits(smem_u32(S.mbar), &st.abort);
  // row t of tile `tile` (24 features as three 16-byte loads; zeros past the last row)
  auto load_row = [&](int64_t tile, uint4 (&q)[3]) {
    q[0] = q[1] = q[2] = make_uint4(0, 0, 0, 0);
    const int64_t row = tile * TILE + t;
    if (tile < ntiles && row < n) {
      const uint4* src = reinterpret_cast<const uint4*>(X + row * NIN);
      q[0] = __ldcs(src);
      q[1] = __ldcs(src + 1);
      q[2] = __ldcs(src + 2);
    }
  };
  uint4 xq[3];
  load_row(blockIdx.x, xq);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t row = tile * TILE + t;
    infer_put_row(S, xq);
    load_row(tile + gridDim.x, xq);  // the next tile's row, in flight during this tile
    float y0, y1;
    if (!infer_tile(S, st, tmem, waits, tile != expire_tile, y0, y1)) break;
    if (row < n) __stcs(reinterpret_cast<float2*>(Y + row * NOUT), make_float2(y0, y1));
  }
  infer_finish(waits, tmem, status);
}

// Training accumulates the gradients of the mean squared error (1/n) sum_rows sum_k
// (y_k - t_k)^2 into grad (FP32, zeroed by the caller) and the squared-error sum into *loss.
// Column 88 of HX (the first padding column of the input chunk) holds 1 for valid rows, so
// the weight-gradient MMA also returns the bias gradients: DW[j][88] = sum_rows dH2[:, j] =
// db2[j], DW[64 + i][88] = db1[i]. W1's padded input columns are 0, so the forward product
// ignores it.
constexpr int ONES_COL = 64 + NIN;

__global__ void __launch_bounds__(TILE, 2) k_mlp_train(const __nv_bfloat16* __restrict__ X, int64_t n,
                                                       const ParamsBF16* __restrict__ wbf,
                                                       const Params* __restrict__ p,
                                                       const float* __restrict__ target, Params* __restrict__ grad,
                                                       float* loss, float inv_n, Status* status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* HX = smem;
  unsigned char* DD = smem + HX_BYTES;
  unsigned char* W1s = DD + DD_BYTES;
  unsigned char* W2s = W1s + W1_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(W2s + W2_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(W2s + W2_BYTES + 16);
  __nv_bfloat16* sH2 = reinterpret_cast<__nv_bfloat16*>(W2s + W2_BYTES + 64);  // 128 x 64
  float* sDY = reinterpret_cast<float*>(W2s + W2_BYTES + 64 + TILE * NH * 2);   // 128 x 2
  __shared__ float sb1[NH], sb2[NH], sw3[NOUT * NH], sb3[NOUT];
  __shared__ int s_abort;

  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int64_t ntiles = (n + TILE - 1) / TILE;
  if ((int64_t)blockIdx.x >= ntiles) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TRAIN_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  load_weights(W1s, W2s, sb1, sb2, sw3, sb3, wbf, p, t);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t hx = smem_u32(HX), dd = smem_u32(DD), w1 = smem_u32(W1s), w2 = smem_u32(W2s);
  const uint32_t ID_FWD = idesc_bf16(128, 64, 0, 0), ID_BWD = idesc_bf16(128, 64, 0, 1),
                 ID_WGRAD = idesc_bf16(128, 96, 1, 1);
  MmaWaits waits(smem_u32(mbar), &s_abort);
  bool first_wgrad = true;
  float loss_local = 0.0f, gw3 = 0.0f, gb3 = 0.0f;  // thread t: dW3[t / 64][t % 64]; t < 2: db3[t]
  auto sync_for_mma = [&]() {  // shared-memory writes -> visible to the tensor core
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
  };

  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t row = tile * TILE + t;
    const bool valid = row < n;
    // X -> HX[:, 64:96]: 24 features as three 16-byte chunks, then [1 (valid rows), 0 x 7]
    {
      uint4 q[3] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
      if (valid) {
        const uint4* src = reinterpret_cast<const uint4*>(X + row * NIN);
        q[0] = src[0];
        q[1] = src[1];
        q[2] = src[2];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) *reinterpret_cast<uint4*>(HX + tile_off(t, 64 + 8 * c, HX_CHUNK)) = q[c];
      float ones[8] = {valid ? 1.0f : 0.0f, 0, 0, 0, 0, 0, 0, 0};
      store8(HX, t, ONES_COL, HX_CHUNK, ones);
    }
    sync_for_mma();
    if (waits.aborted()) break;
    if (t == 0) {  // Z1 = X W1^T
#pragma unroll
      for (int kk = 0; kk < 2; ++kk)
        mma_bf16(tmem + 0, sdesc(hx + (8 + 2 * kk) * HX_CHUNK, HX_CHUNK, 128),
                 sdesc(w1 + 2 * kk * W_CHUNK, W_CHUNK, 128), ID_FWD, kk);
      mma_commit(waits.mb);
    }
    waits.wait(true);
#pragma unroll
    for (int c = 0; c < 4; ++c) {  // H1 = gelu(Z1 + b1) -> HX[:, 0:64]
      float v[16];
      tmem_ld16(lane_base + 16 * c, v);
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = gelu(v[k] + sb1[16 * c + k]);
      store8(HX, t, 16 * c, HX_CHUNK, v);
      store8(HX, t, 16 * c + 8, HX_CHUNK, v + 8);
    }
    sync_for_mma();
    if (waits.aborted()) break;
    if (t == 0) {  // Z2 = H1 W2^T
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(tmem + 64, sdesc(hx + 2 * kk * HX_CHUNK, HX_CHUNK, 128), sdesc(w2 + 2 * kk * W_CHUNK, W_CHUNK, 128),
                 ID_FWD, kk);
      mma_commit(waits.mb);
    }
    waits.wait(true);
    float y[NOUT] = {sb3[0], sb3[1]};
#pragma unroll
    for (int c = 0; c < 4; ++c) {  // Y = bf16(gelu(Z2 + b2)) W3^T + b3, FP32 accumulation
      float v[16];
      tmem_ld16(lane_base + 64 + 16 * c, v);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int j = 16 * c + k;
        const float h2 = bf(gelu(v[k] + sb2[j]));
        y[0] += h2 * sw3[j];
        y[1] += h2 * sw3[NH + j];
        sH2[t * NH + j] = __float2bfloat16_rn(h2);
      }
    }
    // ---- backward ----
    float dy[NOUT];
#pragma unroll
    for (int k = 0; k < NOUT; ++k) {
      const float diff = valid ? y[k] - target[row * NOUT + k] : 0.0f;
      loss_local += diff * diff;
      dy[k] = 2.0f * diff * inv_n;
      sDY[t * NOUT + k] = dy[k];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {  // dH2 = (dY W3) * gelu'(Z2 + b2) -> DD[:, 0:64]
      float v[16];
      tmem_ld16(lane_base + 64 + 16 * c, v);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int j = 16 * c + k;
        v[k] = (dy[0] * sw3[j] + dy[1] * sw3[NH + j]) * gelu_grad(v[k] + sb2[j]);
      }
      store8(DD, t, 16 * c, HX_CHUNK, v);
      store8(DD, t, 16 * c + 8, HX_CHUNK, v + 8);
    }
    sync_for_mma();  // also publishes sH2 and sDY
    if (waits.aborted()) break;
    if (t == 0) {    // G = dH2 W2 (overwrites Z2)
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(tmem + 64, sdesc(dd + 2 * kk * HX_CHUNK, HX_CHUNK, 128), sdesc(w2 + 2 * kk * 128, 128, W_CHUNK),
                 ID_BWD, kk);
      mma_commit(waits.mb);
    }
    {  // meanwhile: dW3[o][j] += sum_rows dY[:, o] H2[:, j], db3 += sum_rows dY
      const int o = t / NH, j = t % NH;
      float s = 0.0f;
      for (int r = 0; r < TILE; ++r) s += sDY[r * NOUT + o] * __bfloat162float(sH2[r * NH + j]);
      gw3 += s;
      if (t < NOUT) {
        float b = 0.0f;
        for (int r = 0; r < TILE; ++r) b += sDY[r * NOUT + t];
        gb3 += b;
      }
    }
    waits.wait(true);
#pragma unroll
    for (int c = 0; c < 4; ++c) {  // dH1 = G * gelu'(Z1 + b1) -> DD[:, 64:128]
      float g[16], z[16];
      tmem_ld16(lane_base + 64 + 16 * c, g);
      tmem_ld16(lane_base + 16 * c, z);
#pragma unroll
      for (int k = 0; k < 16; ++k) g[k] *= gelu_grad(z[k] + sb1[16 * c + k]);
      store8(DD, t, 64 + 16 * c, HX_CHUNK, g);
      store8(DD, t, 64 + 16 * c + 8, HX_CHUNK, g + 8);
    }
    sync_for_mma();
    if (waits.aborted()) break;
    if (t == 0) {  // DW += DD^T [H1 | X | 1]
#pragma unroll
      for (int kk = 0; kk < 8; ++kk)
        mma_bf16(tmem + 128, sdesc(dd + 2 * kk * 128, 128, HX_CHUNK), sdesc(hx + 2 * kk * 128, 128, HX_CHUNK),
                 ID_WGRAD, (first_wgrad && kk == 0) ? 0 : 1);
      mma_commit(waits.mb);
    }
    first_wgrad = false;
    waits.wait(true);
    fence_before();
    __syncthreads();  // the next tile rewrites HX, DD, sH2 and sDY
    fence_after();
    if (waits.aborted()) break;
  }

  waits.drain();
  if (!waits.aborted() && !first_wgrad) {  // row t of DW: dW2 and db2 (t < 64) or dW1 and db1
    float v[16];
    if (t < NH) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        tmem_ld16(lane_base + 128 + 16 * c, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) atomicAdd(&grad->W2[t * NH + 16 * c + k], v[k]);
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        tmem_ld16(lane_base + 128 + 64 + 16 * c, v);
        if (c == 1) atomicAdd(&grad->b2[t], v[ONES_COL - 64 - 16]);
      }
    } else {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        tmem_ld16(lane_base + 128 + 64 + 16 * c, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int in = 16 * c + k;
          if (in < NIN) atomicAdd(&grad->W1[(t - NH) * NIN + in], v[k]);
          if (in == NIN) atomicAdd(&grad->b1[t - NH], v[k]);
        }
      }
    }
    atomicAdd(&grad->W3[t], gw3);
    if (t < NOUT) atomicAdd(&grad->b3[t], gb3);
  }
  float l = loss_local;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) l += __shfl_xor_sync(0xffffffffu, l, s);
  if (lane == 0) atomicAdd(loss, l);
  if (waits.aborted() && t == 0) atomicExch(&status->error, 1);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TRAIN_TMEM_COLS)
                 : "memory");
}

// Adam on the FP32 master parameters; refreshes the BF16 copies.
__global__ void k_adam(Params* p, const Params* g, Params* m, Params* v, ParamsBF16* wbf, float lr, float beta1,
                       float beta2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  float* P = reinterpret_cast<float*>(p);
  const float* G = reinterpret_cast<const float*>(g);
  float* Mm = reinterpret_cast<float*>(m);
  float* Vv = reinterpret_cast<float*>(v);
  const float gi = G[i];
  const float mi = beta1 * Mm[i] + (1 - beta1) * gi;
  const float vi = beta2 * Vv[i] + (1 - beta2) * gi * gi;
  Mm[i] = mi;
  Vv[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_refresh_bf16(const Params* p, ParamsBF16* wbf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NH * KIN) {
    const int r = i / KIN, c = i % KIN;
    wbf->W1[i] = __float2bfloat16_rn(c < NIN ? p->W1[r * NIN + c] : 0.0f);
  }
  if (i < NH * NH) wbf->W2[i] = __float2bfloat16_rn(p->W2[i]);
  if (i < NOUT * NH) wbf->W3[i] = __float2bfloat16_rn(p->W3[i]);
}

}  // namespace closure
}  // namespace trisk

using namespace trisk;
using namespace trisk::closure;

// The closure works on the legacy default stream, so it is ordered with the caller's
// default-stream work on the feature and target arrays it reads.
struct TriskClosure {
  int device = 0;
  cudaStream_t stream = cudaStreamLegacy;
  Params* p = nullptr;
  Params *g = nullptr, *m = nullptr, *v = nullptr;
  ParamsBF16* wbf = nullptr;
  float* loss = nullptr;
  Status* status = nullptr;
  int64_t adam_step = 0;
  int64_t launches = 0;
  int sms = 0;              // the device's SM count (persistent grids)
  int forward_per_sm = 1;   // resident inference CTAs per SM (the grid's multiple of the SMs)
  int64_t expire_tile = -1;  // test of the bounded wait: see trisk_closure_expire_wait_once
  ~TriskClosure() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    for (void* q : {(void*)p, (void*)g, (void*)m, (void*)v, (void*)wbf, (void*)loss, (void*)status})
      if (q) cudaFree(q);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

namespace {

TriskClosure* checked_c(TriskClosure* c) {
  if (!c) throw Error(TRISK_ERR_ARGUMENT, "closure is NULL");
  return c;
}

void check_status(TriskClosure& c) {
  Status s{};
  CUDA_CHECK(cudaMemcpyAsync(&s, c.status, sizeof(s), cudaMemcpyDeviceToHost, c.stream));
  CUDA_CHECK(cudaStreamSynchronize(c.stream));
  if (s.error) {
    CUDA_CHECK(cudaMemset(c.status, 0, sizeof(Status)));
    throw Error(TRISK_ERR_TIMEOUT, "a bounded tensor-core wait in the closure MLP gave up");
  }
}

// persistent grids: every resident CTA of the device, or one per tile when there are fewer
int mlp_grid(const TriskClosure& c, int64_t n, int per_sm) {
  const int64_t tiles = (n + TILE - 1) / TILE;
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)c.sms * per_sm));
}

void launch_forward(TriskClosure& c, const __nv_bfloat16* X, int64_t n, float* Y, cudaStream_t stream) {
  if (n == 0) return;
  const int64_t expire = c.expire_tile;
  c.expire_tile = -1;
  k_mlp_forward<<<mlp_grid(c, n, c.forward_per_sm), TILE, FWD_SMEM_BYTES, stream>>>(X, n, c.wbf, c.p, Y, c.status,
                                                                                     expire);
  CUDA_CHECK(cudaGetLastError());
  c.launches++;
}

void launch_train(TriskClosure& c, const __nv_bfloat16* X, int64_t n, const float* target, float inv_n) {
  if (n == 0) return;
  k_mlp_train<<<mlp_grid(c, n, 2), TILE, SMEM_BYTES, c.stream>>>(X, n, c.wbf, c.p, target, c.g, c.loss, inv_n,
                                                                 c.status);
  CUDA_CHECK(cudaGetLastError());
  c.launches++;
}

}  // namespace

namespace trisk {

namespace closure {

void closure_device_params(TriskClosure* c, const ParamsBF16** wbf, const Params** p, Status** status) {
  *wbf = c->wbf;
  *p = c->p;
  *status = c->status;
}

int infer_ctas_per_sm(const void* kernel, int device) {
  // all of the unified L1/shared storage as shared memory, so that several CTAs fit an SM
  CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM_BYTES));
  CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
  // From the kernel's resources: shared memory (dynamic, static and the per-CTA reservation),
  // registers (allocated per warp in units of 256), threads, and tensor memory (512 columns).
  // The runtime's occupancy query reports one CTA for these kernels, which would leave most of
  // each SM idle, so it is not used.
  cudaFuncAttributes fa{};
  CUDA_CHECK(cudaFuncGetAttributes(&fa, kernel));
  int smem_sm = 0, reserved = 0, regs_sm = 0, threads_sm = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
  CUDA_CHECK(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device));
  CUDA_CHECK(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device));
  CUDA_CHECK(cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device));
  const int by_smem = smem_sm / (FWD_SMEM_BYTES + (int)fa.sharedSizeBytes + reserved);
  const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
  const int by_regs = regs_sm / std::max(1, warp_regs * (TILE / 32));
  const int by_threads = threads_sm / TILE;
  const int per_sm = std::min(std::min(by_smem, by_regs), std::min(by_threads, 512 / (int)FWD_TMEM_COLS));
  return std::max(1, per_sm);
}

}  // namespace closure

void closure_forward_on(TriskClosure* c, const void* X, int64_t n, float* Y, cudaStream_t stream) {
  launch_forward(*c, static_cast<const __nv_bfloat16*>(X), n, Y, stream);
}

void closure_check(TriskClosure* c) { check_status(*c); }

int closure_device(const TriskClosure* c) { return c->device; }

}  // namespace trisk

extern "C" {

int trisk_closure_create(int32_t device, const float* params, TriskClosure** out) {
  TRISK_API_BEGIN
  if (!out) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  auto c = std::make_unique<TriskClosure>();
  c->device = device;
  DeviceGuard guard(device);
  CUDA_CHECK(cudaMalloc(&c->p, sizeof(Params)));
  CUDA_CHECK(cudaMalloc(&c->g, sizeof(Params)));
  CUDA_CHECK(cudaMalloc(&c->m, sizeof(Params)));
  CUDA_CHECK(cudaMalloc(&c->v, sizeof(Params)));
  CUDA_CHECK(cudaMalloc(&c->wbf, sizeof(ParamsBF16)));
  CUDA_CHECK(cudaMalloc(&c->loss, sizeof(float)));
  CUDA_CHECK(cudaMalloc(&c->status, sizeof(Status)));
  CUDA_CHECK(cudaMemset(c->m, 0, sizeof(Params)));
  CUDA_CHECK(cudaMemset(c->v, 0, sizeof(Params)));
  CUDA_CHECK(cudaMemset(c->status, 0, sizeof(Status)));
  if (params) CUDA_CHECK(cudaMemcpy(c->p, params, sizeof(Params), cudaMemcpyHostToDevice));
  else CUDA_CHECK(cudaMemset(c->p, 0, sizeof(Params)));
  k_refresh_bf16<<<(NH * NH + 255) / 256, 256, 0, c->stream>>>(c->p, c->wbf);
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  CUDA_CHECK(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
  int sms = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  c->sms = sms;
  c->forward_per_sm = infer_ctas_per_sm(reinterpret_cast<const void*>(k_mlp_forward), device);
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  *out = c.release();
  TRISK_API_END
}

void trisk_closure_destroy(TriskClosure* c) { delete c; }

int32_t trisk_closure_param_count(void) { return NPARAM; }

int trisk_closure_get_params(TriskClosure* closure, float* params) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (!params) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  DeviceGuard guard(c.device);
  CUDA_CHECK(cudaMemcpyAsync(params, c.p, sizeof(Params), cudaMemcpyDeviceToHost, c.stream));
  CUDA_CHECK(cudaStreamSynchronize(c.stream));
  TRISK_API_END
}

int trisk_closure_set_params(TriskClosure* closure, const float* params) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (!params) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  DeviceGuard guard(c.device);
  CUDA_CHECK(cudaMemcpyAsync(c.p, params, sizeof(Params), cudaMemcpyHostToDevice, c.stream));
  k_refresh_bf16<<<(NH * NH + 255) / 256, 256, 0, c.stream>>>(c.p, c.wbf);
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaStreamSynchronize(c.stream));
  TRISK_API_END
}

// Y (n x 2, FP32) = MLP(X) for X (n x 24, BF16), all device pointers.
int trisk_closure_forward(TriskClosure* closure, const void* X, int64_t n, float* Y) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (!X || !Y || n < 0) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  DeviceGuard guard(c.device);
  launch_forward(c, static_cast<const __nv_bfloat16*>(X), n, Y, c.stream);
  check_status(c);
  TRISK_API_END
}

// Gradients (FP32, same layout as the parameters) of the mean squared error over the batch
// and the loss; grads may be NULL (then kept on the device for trisk_closure_adam).
int trisk_closure_gradients(TriskClosure* closure, const void* X, const float* target, int64_t n, float* grads,
                            float* loss) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (!X || !target || n <= 0) throw Error(TRISK_ERR_ARGUMENT, "bad argument");
  DeviceGuard guard(c.device);
  CUDA_CHECK(cudaMemsetAsync(c.g, 0, sizeof(Params), c.stream));
  CUDA_CHECK(cudaMemsetAsync(c.loss, 0, sizeof(float), c.stream));
  launch_train(c, static_cast<const __nv_bfloat16*>(X), n, target, 1.0f / (float)n);
  if (grads) CUDA_CHECK(cudaMemcpyAsync(grads, c.g, sizeof(Params), cudaMemcpyDeviceToHost, c.stream));
  float l = 0;
  CUDA_CHECK(cudaMemcpyAsync(&l, c.loss, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  check_status(c);
  if (loss) *loss = l / (float)n;
  TRISK_API_END
}

// One Adam step with the gradients left by the last trisk_closure_gradients call.
int trisk_closure_adam(TriskClosure* closure, float lr, float beta1, float beta2, float eps) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  DeviceGuard guard(c.device);
  c.adam_step++;
  const float c1 = 1.0f - powf(beta1, (float)c.adam_step), c2 = 1.0f - powf(beta2, (float)c.adam_step);
  k_adam<<<(NPARAM + 255) / 256, 256, 0, c.stream>>>(c.p, c.g, c.m, c.v, c.wbf, lr, beta1, beta2, eps, c1, c2);
  k_refresh_bf16<<<(NH * NH + 255) / 256, 256, 0, c.stream>>>(c.p, c.wbf);
  CUDA_CHECK(cudaGetLastError());
  c.launches += 2;
  TRISK_API_END
}

int trisk_closure_synchronize(TriskClosure* closure) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  DeviceGuard guard(c.device);
  check_status(c);
  TRISK_API_END
}

// Launch shape of the inference kernel: CTAs per SM of its persistent grid, and SMs.
int trisk_closure_info(TriskClosure* closure, int32_t* forward_ctas_per_sm, int32_t* sms) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (forward_ctas_per_sm) *forward_ctas_per_sm = c.forward_per_sm;
  if (sms) *sms = c.sms;
  TRISK_API_END
}

// Test of the bounded tensor-core wait: the next inference launch of this closure leaves the
// first tensor-core operation of `tile` un-issued, so that tile's wait runs out (after half a
// second) and the call reports TRISK_ERR_TIMEOUT; later calls are unaffected.
int trisk_closure_expire_wait_once(TriskClosure* closure, int64_t tile) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (tile < 0) throw Error(TRISK_ERR_ARGUMENT, "tile must be >= 0");
  c.expire_tile = tile;
  TRISK_API_END
}

int trisk_closure_stream(TriskClosure* closure, void** stream) {
  TRISK_API_BEGIN
  TriskClosure& c = *checked_c(closure);
  if (!stream) throw Error(TRISK_ERR_ARGUMENT, "NULL argument");
  *stream = (void*)c.stream;
  TRISK_API_END
}

}  // extern "C"
