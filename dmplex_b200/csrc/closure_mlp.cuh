// Device side of the closure network shared by its own kernels (closure.cu) and the fused
// feature + network + correction kernel of the ensembles (ensemble.cu): the tcgen05 helpers,
// the no-swizzle operand layout, the bounded waits, GELU, and the inference of one 128-row
// tile whose inputs are in shared memory. The layout, the tensor-memory use and the waits
// are described at the top of closure.cu.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "model.hpp"

struct TriskClosure;

namespace trisk {
namespace closure {

constexpr int NIN = 24, KIN = 32, NH = 64, NOUT = 2, TILE = 128;
constexpr int HX_CHUNK = TILE * 16;  // 2048 B: one 8-column chunk of a 128-row tile
constexpr int W_CHUNK = NH * 16;     // 1024 B: one 8-column chunk of a 64-row weight
constexpr int HX_BYTES = 12 * HX_CHUNK;  // 96 columns: H1 (0..63) | X (64..95)
constexpr int DD_BYTES = 16 * HX_CHUNK;  // 128 columns: dH2 (0..63) | dH1 (64..127)
constexpr int W1_BYTES = 4 * W_CHUNK;    // 64 x 32
constexpr int W2_BYTES = 8 * W_CHUNK;    // 64 x 64
// + 64 B (mbarrier, TMEM address) + H2 (128 x 64 BF16) and dY (128 x 2 FP32) for training
constexpr int SMEM_BYTES = HX_BYTES + DD_BYTES + W1_BYTES + W2_BYTES + 64 + TILE * NH * 2 + TILE * NOUT * 4;
constexpr uint32_t TRAIN_TMEM_COLS = 256;  // two CTAs per SM share its 512 columns
// Inference: XH (X, then H1: 8 chunks), W1, W2 and the barrier, 64 TMEM columns; at most
// seven CTAs fit an SM's shared memory, and seven (even eight) x 64 columns fit its TMEM, so
// no CTA ever waits in tcgen05.alloc.
constexpr int XH_BYTES = 8 * HX_CHUNK;
constexpr int FWD_SMEM_BYTES = XH_BYTES + W1_BYTES + W2_BYTES + 64;
constexpr uint32_t FWD_TMEM_COLS = 64;
static_assert(FWD_SMEM_BYTES * 7 <= 220 * 1024, "seven inference CTAs per SM");
// A bounded tensor-core wait gives up after this long (the operations take microseconds).
constexpr long long MBAR_WAIT_NS = 500000000LL;

// FP32 master parameters and their BF16 tensor-core copies (one contiguous block each).
struct Params {
  float W1[NH * NIN], b1[NH], W2[NH * NH], b2[NH], W3[NOUT * NH], b3[NOUT];
};
constexpr int NPARAM = sizeof(Params) / sizeof(float);
struct ParamsBF16 {
  __nv_bfloat16 W1[NH * KIN];  // padded to 32 inputs
  __nv_bfloat16 W2[NH * NH];
  __nv_bfloat16 W3[NOUT * NH];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// no-swizzle shared-memory matrix descriptor (sm100 layout: version 1 at bit 46)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16 with BF16 operands and an FP32 accumulator
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Waits for the completion of the mbarrier phase of parity `phase`, for at most MBAR_WAIT_NS
// and at most MBAR_WAIT_TRIES polls (a backstop that the clock always beats: a poll takes more
// than a nanosecond); false if it gave up.
constexpr uint32_t MBAR_WAIT_TRIES = 1u << 31;
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  long long start = 0;
  for (uint32_t i = 0; i < MBAR_WAIT_TRIES; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
    if ((i & 255) == 0) {
      const long long now = global_ns();
      if (i == 0) start = now;
      else if (now - start > MBAR_WAIT_NS) return false;
    }
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// gelu(x) = x/2 (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715 x^3) (Hendrycks and Gimpel 2016)
constexpr float GELU_C0 = 0.7978845608028654f;   // sqrt(2/pi)
constexpr float GELU_C1 = 0.035677408136300125f;  // 0.044715 sqrt(2/pi)
__device__ __forceinline__ float gelu(float x) {
  const float u = x * fmaf(GELU_C1, x * x, GELU_C0);
  const float h = 0.5f * x;
  return fmaf(h, tanh_approx(u), h);
}
// d gelu / dx = (1 + t)/2 + x/2 (1 - t^2) du/dx,  du/dx = sqrt(2/pi) (1 + 3 * 0.044715 x^2)
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float t = tanh_approx(x * fmaf(GELU_C1, x2, GELU_C0));
  const float du = fmaf(3.0f * GELU_C1, x2, GELU_C0);
  return fmaf(0.5f * x * fmaf(-t, t, 1.0f), du, fmaf(0.5f, t, 0.5f));
}
__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t tile_off(int r, int c, int chunk) {
  return (uint32_t)((c >> 3) * chunk + (r >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// 8 consecutive columns (c0 multiple of 8) of row r as one 16-byte store
__device__ __forceinline__ void store8(unsigned char* base, int r, int c0, int chunk, const float* v) {
  uint4 q;
  __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]),
                 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
  q.x = *reinterpret_cast<uint32_t*>(&p0);
  q.y = *reinterpret_cast<uint32_t*>(&p1);
  q.z = *reinterpret_cast<uint32_t*>(&p2);
  q.w = *reinterpret_cast<uint32_t*>(&p3);
  *reinterpret_cast<uint4*>(base + tile_off(r, c0, chunk)) = q;
}

struct Status {
  int error;  // 1: a bounded tensor-core wait gave up
};

// W1 (64 x 32, inputs padded with 0) and W2 (64 x 64) as K-major B operands; biases and W3
__device__ __forceinline__ void load_weights(unsigned char* W1s, unsigned char* W2s, float* sb1, float* sb2,
                                             float* sw3, float* sb3, const ParamsBF16* __restrict__ wbf,
                                             const Params* __restrict__ p, int t) {
  for (int idx = t; idx < NH * 4; idx += TILE) {
    const int r = idx >> 2, c0 = (idx & 3) * 8;
    *reinterpret_cast<uint4*>(W1s + tile_off(r, c0, W_CHUNK)) =
        *reinterpret_cast<const uint4*>(wbf->W1 + r * KIN + c0);
  }
  for (int idx = t; idx < NH * 8; idx += TILE) {
    const int r = idx >> 3, c0 = (idx & 7) * 8;
    *reinterpret_cast<uint4*>(W2s + tile_off(r, c0, W_CHUNK)) =
        *reinterpret_cast<const uint4*>(wbf->W2 + r * NH + c0);
  }
  for (int idx = t; idx < NH; idx += TILE) {
    sb1[idx] = p->b1[idx];
    sb2[idx] = p->b2[idx];
  }
  for (int idx = t; idx < NOUT * NH; idx += TILE) sw3[idx] = __bfloat162float(wbf->W3[idx]);
  if (t < NOUT) sb3[t] = p->b3[t];
}

// The bounded tensor-core waits of a CTA. wait() records a give-up in the CTA's shared abort
// word; every thread reads that word only right after a CTA-wide barrier, so all threads
// leave the tile loop together. `last` and `issued` (the parity of the last wait and whether
// an operation was committed to it) are the same in every thread.
struct MmaWaits {
  uint32_t mb;
  volatile int* abort;
  uint32_t phase = 0, last = 0;
  bool issued = false;
  __device__ MmaWaits(uint32_t mbar, int* abort_word) : mb(mbar), abort(abort_word) {}
  __device__ __forceinline__ void wait(bool committed) {
    last = phase;
    if (!mbar_wait(mb, phase)) *abort = 1;
    phase ^= 1;
    issued = committed;
    fence_after();
  }
  __device__ __forceinline__ bool aborted() const { return *abort != 0; }
  // after an abort: wait (bounded) for the committed operation whose completion was not seen,
  // so that the tensor memory it writes is no longer in use when it is freed
  __device__ __forceinline__ void drain() {
    if (*abort && issued) mbar_wait(mb, last);
  }
};

// ---- inference of one tile ------------------------------------------------------------
// A CTA of TILE threads with XH (XH_BYTES), W1s, W2s, the mbarrier and the TMEM address slot in
// dynamic shared memory (FWD_SMEM_BYTES), FWD_TMEM_COLS tensor-memory columns, and the biases
// and output weights in static shared memory.
struct InferSmem {
  unsigned char* XH;
  unsigned char* W1s;
  unsigned char* W2s;
  uint64_t* mbar;
  uint32_t* tmem_slot;
  __device__ explicit InferSmem(unsigned char* smem)
      : XH(smem), W1s(smem + XH_BYTES), W2s(smem + XH_BYTES + W1_BYTES),
        mbar(reinterpret_cast<uint64_t*>(smem + XH_BYTES + W1_BYTES + W2_BYTES)),
        tmem_slot(reinterpret_cast<uint32_t*>(smem + XH_BYTES + W1_BYTES + W2_BYTES + 16)) {}
};
struct InferStatic {
  float b1[NH], b2[NH], w3[NOUT * NH], b3[NOUT];
  int abort;
};

// Tensor memory, the mbarrier and the weights; returns the CTA's TMEM base address.
__device__ __forceinline__ uint32_t infer_setup(const InferSmem& S, InferStatic& st, const ParamsBF16* wbf,
                                                const Params* p) {
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(S.tmem_slot)),
                 "r"(FWD_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(S.mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    st.abort = 0;
  }
  load_weights(S.W1s, S.W2s, st.b1, st.b2, st.w3, st.b3, wbf, p, t);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  return *S.tmem_slot;
}

// Row t of the tile's features (24 BF16 values as three 16-byte chunks) into XH chunks 0..2,
// and zeros into chunk 3 (W1's padding columns are 0 as well).
__device__ __forceinline__ void infer_put_row(const InferSmem& S, const uint4 (&q)[3]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int c = 0; c < 3; ++c) *reinterpret_cast<uint4*>(S.XH + tile_off(t, 8 * c, HX_CHUNK)) = q[c];
  *reinterpret_cast<uint4*>(S.XH + tile_off(t, 24, HX_CHUNK)) = make_uint4(0, 0, 0, 0);
}

// The network on the tile in XH (all threads call it after writing their rows): this thread's
// two outputs; false if the CTA has given up a wait (then every thread returns false). With
// issue = false the first tensor-core operation is left out (the bounded wait's test).
__device__ __forceinline__ bool infer_tile(const InferSmem& S, const InferStatic& st, uint32_t tmem, MmaWaits& waits,
                                           bool issue, float& y0, float& y1) {
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t xh = smem_u32(S.XH), w1 = smem_u32(S.W1s), w2 = smem_u32(S.W2s);
  const uint32_t ID = idesc_bf16(128, 64, 0, 0);
  auto sync_for_mma = [&]() {  // shared-memory writes -> visible to the tensor core
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
  };
  const float4* b1v = reinterpret_cast<const float4*>(st.b1);
  const float4* b2v = reinterpret_cast<const float4*>(st.b2);
  const float4* w3a = reinterpret_cast<const float4*>(st.w3);
  const float4* w3b = reinterpret_cast<const float4*>(st.w3 + NH);
  sync_for_mma();
  if (waits.aborted()) return false;
  if (t == 0 && issue) {  // Z1 = X W1^T
#pragma unroll
    for (int kk = 0; kk < 2; ++kk)
      mma_bf16(tmem, sdesc(xh + 2 * kk * HX_CHUNK, HX_CHUNK, 128), sdesc(w1 + 2 * kk * W_CHUNK, W_CHUNK, 128), ID, kk);
    mma_commit(waits.mb);
  }
  waits.wait(issue);
#pragma unroll
  for (int c = 0; c < 4; ++c) {  // H1 = gelu(Z1 + b1) -> XH chunks 0..7 (MMA 1 has read X)
    float v[16];
    tmem_ld16(lane_base + 16 * c, v);
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4) {
      const float4 b = b1v[4 * c + k4];
      v[4 * k4 + 0] = gelu(v[4 * k4 + 0] + b.x);
      v[4 * k4 + 1] = gelu(v[4 * k4 + 1] + b.y);
      v[4 * k4 + 2] = gelu(v[4 * k4 + 2] + b.z);
      v[4 * k4 + 3] = gelu(v[4 * k4 + 3] + b.w);
    }
    store8(S.XH, t, 16 * c, HX_CHUNK, v);
    store8(S.XH, t, 16 * c + 8, HX_CHUNK, v + 8);
  }
  sync_for_mma();  // also: every thread has read Z1, which Z2 overwrites
  if (waits.aborted()) return false;
  if (t == 0) {  // Z2 = H1 W2^T
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma_bf16(tmem, sdesc(xh + 2 * kk * HX_CHUNK, HX_CHUNK, 128), sdesc(w2 + 2 * kk * W_CHUNK, W_CHUNK, 128), ID, kk);
    mma_commit(waits.mb);
  }
  waits.wait(true);
  y0 = st.b3[0];
  y1 = st.b3[1];
#pragma unroll
  for (int c = 0; c < 4; ++c) {  // Y = bf16(gelu(Z2 + b2)) W3^T + b3, FP32 accumulation
    float v[16];
    tmem_ld16(lane_base + 16 * c, v);
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4) {
      const float4 b = b2v[4 * c + k4], wa = w3a[4 * c + k4], wb = w3b[4 * c + k4];
      const __nv_bfloat162 h01 = __floats2bfloat162_rn(gelu(v[4 * k4 + 0] + b.x), gelu(v[4 * k4 + 1] + b.y));
      const __nv_bfloat162 h23 = __floats2bfloat162_rn(gelu(v[4 * k4 + 2] + b.z), gelu(v[4 * k4 + 3] + b.w));
      const float h0 = __low2float(h01), h1 = __high2float(h01), h2 = __low2float(h23), h3 = __high2float(h23);
      y0 += h0 * wa.x;
      y1 += h0 * wb.x;
      y0 += h1 * wa.y;
      y1 += h1 * wb.y;
      y0 += h2 * wa.z;
      y1 += h2 * wb.z;
      y0 += h3 * wa.w;
      y1 += h3 * wb.w;
    }
  }
  fence_before();
  __syncthreads();  // the next tile rewrites XH, and its MMA 1 overwrites Z2
  fence_after();
  return !waits.aborted();
}

// After the tile loop: the drain of a given-up wait, the status, the TMEM free.
__device__ __forceinline__ void infer_finish(MmaWaits& waits, uint32_t tmem, Status* status) {
  waits.drain();
  if (waits.aborted() && threadIdx.x == 0) atomicExch(&status->error, 1);
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(FWD_TMEM_COLS)
                 : "memory");
}

// Host side, defined in closure.cu. The network's device parameters and status word, for
// kernels that run it inline.
void closure_device_params(TriskClosure* c, const ParamsBF16** wbf, const Params** p, Status** status);
// Resident CTAs per SM of an inference-shaped kernel (TILE threads, FWD_SMEM_BYTES of dynamic
// shared memory, FWD_TMEM_COLS tensor-memory columns), from its shared memory, registers and
// threads; sets the kernel's shared-memory attributes on the current device first.
int infer_ctas_per_sm(const void* kernel, int device);

}  // namespace closure
}  // namespace trisk
