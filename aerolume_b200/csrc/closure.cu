// The learned subgrid closure of the 3D step: training pairs from a box-filtered periodic run, a
// per-cell MLP (10 -> 128 -> 128 -> 128 -> 6, SiLU) on the fifth-generation tensor cores, its
// training (forward, backward, Adam), and the eddy viscosity of the learned stress with the
// per-cell WALE fallback inside the step's eddy-viscosity pass.
//
// The reference has no learned closure; what it replaces is the WALE eddy viscosity of
// ns3d/core.py:448-482 (eddy_viscosity3d) / ns3d/fused.py:102-132 (ns3d_nut_wale), which keeps
// its role as the fallback.
//
// Tensor-core usage (sm_100a, no library): every layer is D = A * B^T on tiles of 128 rows
// (cells or samples) issued by one thread as tcgen05.mma.cta_group::1.kind::f16 with BF16
// operands in shared memory (K-major, no swizzle: 8-row x 16-byte core matrices, the K / 8 core
// matrices of an 8-row group contiguous) and the FP32 accumulator in tensor memory; its
// completion arrives on an mbarrier (tcgen05.commit) that every thread waits on with a bounded
// wait; the epilogue reads the accumulator back with tcgen05.ld (warp w owns lanes 32 w ..
// 32 w + 31, one row per thread), adds the bias, applies SiLU and writes the next layer's BF16
// operand.  A wait that runs out sets bit 2 of the status word, the CTA stops, waits (bounded)
// for its last MMA and frees its tensor memory.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tma.cuh"

namespace aero {
namespace closure {

constexpr int NIN = 10, KIN = 16, NH = 128, NOUT = 6, KOUT = 16, ROWS = 128;
constexpr int NTHREADS = 128;
constexpr int STATUS_TIMEOUT = 4;

// ------------------------------------------------------------------------------------------
// tcgen05 / TMEM primitives
// ------------------------------------------------------------------------------------------

// byte offset of element (r, k) of a K-major BF16 operand with K columns (K % 16 == 0)
__device__ __forceinline__ uint32_t kmaj(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor of that layout: leading byte offset 128 (the next 8 columns),
// stride byte offset 16 K (the next 8 rows), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t kmaj_desc(uint32_t saddr, int K) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)(((uint32_t)K * 16u) >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  tmem_wait_ld();
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  tmem_wait_ld();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// lane base of warp w's quarter of the tensor memory
__device__ __forceinline__ uint32_t lane_base(uint32_t tbase) { return tbase + ((uint32_t)((threadIdx.x >> 5) * 32) << 16); }

// D = A * B^T over K (multiple of 16): A (128 x K) and B (N x K) K-major in shared memory.
// Issued by the calling thread only; accumulate == false starts from zero.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, const void *A, const void *B, int K, int N, bool accumulate) {
  const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
  const uint32_t id = idesc_bf16(128, N);
  for (int s = 0; s < K / 16; ++s)
    mma_bf16(tmem_d, kmaj_desc(a0 + 256u * s, K), kmaj_desc(b0 + 256u * s, K), id, (accumulate || s > 0) ? 1u : 0u);
}

// Block-wide bounded wait on the MMA barrier; false (everywhere) when any thread gave up.
__device__ __forceinline__ bool mma_wait(uint64_t *bar, uint32_t &phase, int *status) {
  const bool ok = mbar_wait_bounded(bar, phase, nullptr, 1 << 22);
  phase ^= 1u;
  const bool bad = __syncthreads_or(!ok) != 0;
  if (bad && threadIdx.x == 0 && status) atomicOr(status, STATUS_TIMEOUT);
  tc_fence_after();
  return !bad;
}

// make this thread's generic shared-memory writes visible to the tensor cores, then sync
__device__ __forceinline__ void operands_ready() {
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// SiLU on the FP32 accumulator plus bias: x sigmoid(x), sigmoid(x) = (1 + tanh(x / 2)) / 2
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu(float x) { return x * fmaf(0.5f, tanh_fast(0.5f * x), 0.5f); }
// the same on a pair of BF16 pre-activations, in BF16 arithmetic (tanh.approx.bf16x2): the
// hidden activations the network runs on, forward and (recomputed) backward
__device__ __forceinline__ __nv_bfloat162 silu2(__nv_bfloat162 z) {
  const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
  const __nv_bfloat162 a = __hmul2(z, half);
  __nv_bfloat162 t;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(*reinterpret_cast<uint32_t *>(&t)) : "r"(*reinterpret_cast<const uint32_t *>(&a)));
  return __hmul2(z, __hfma2(t, half, half));
}
// d silu / dx = s + x s (1 - s)
__device__ __forceinline__ float silu_grad(float x) {
  const float s = fmaf(0.5f, tanh_fast(0.5f * x), 0.5f);
  return fmaf(x * s, 1.0f - s, s);
}

// store 8 consecutive columns c0 .. c0 + 7 (c0 % 8 == 0) of row r of a K-major operand
__device__ __forceinline__ void store8(unsigned char *base, int r, int c0, int K, const float *v) {
  __align__(16) __nv_bfloat162 p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4 *>(base + kmaj(r, c0, K)) = *reinterpret_cast<const uint4 *>(p);
}

__device__ __forceinline__ void put_bf16(unsigned char *base, int r, int k, int K, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(base + kmaj(r, k, K)) = __float2bfloat16_rn(v);
}

// ------------------------------------------------------------------------------------------
// features of a velocity gradient
// ------------------------------------------------------------------------------------------

// From the eight components of a traceless gradient g (g11, g12, g13, g21, g22, g23, g31, g32;
// g33 = -(g11 + g22), as core.py:437-445 makes it): the MLP inputs -- g / |g| (eight values) and
// two invariants, (|W|^2 - |S|^2) / |g|^2 and sqrt(6) tr(S^3) / |S|^3 -- and the scales the
// output and the dissipation need.  Returns false when |g| or |S| is too small to normalise.
struct Grad {
  float g[3][3];
  float S[3][3];
  float g2, s2;
};

__device__ __forceinline__ bool features(const float *g8, float *f, Grad &G) {
  G.g[0][0] = g8[0];
  G.g[0][1] = g8[1];
  G.g[0][2] = g8[2];
  G.g[1][0] = g8[3];
  G.g[1][1] = g8[4];
  G.g[1][2] = g8[5];
  G.g[2][0] = g8[6];
  G.g[2][1] = g8[7];
  G.g[2][2] = -(g8[0] + g8[4]);
  float g2 = 0.f, s2 = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      G.S[a][b] = 0.5f * (G.g[a][b] + G.g[b][a]);
      g2 = fmaf(G.g[a][b], G.g[a][b], g2);
      s2 = fmaf(G.S[a][b], G.S[a][b], s2);
    }
  G.g2 = g2;
  G.s2 = s2;
  const bool ok = g2 > 1e-20f && s2 > 1e-6f * g2 && isfinite(g2);
  const float ig = ok ? rsqrtf(g2) : 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) f[q] = g8[q] * ig;
  f[8] = ok ? (g2 - 2.f * s2) / g2 : 0.f;  // |W|^2 - |S|^2 with |W|^2 = |g|^2 - |S|^2
  float t3 = 0.f;                           // tr(S^3)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) t3 = fmaf(G.S[a][b] * G.S[b][c], G.S[c][a], t3);
  f[9] = ok ? 2.449489742783178f * t3 / (s2 * sqrtf(s2)) : 0.f;
  return ok;
}

// ------------------------------------------------------------------------------------------
// the MLP's parameters and a tile of forward pass
// ------------------------------------------------------------------------------------------

struct MlpWeights {
  const __nv_bfloat16 *w1, *w2, *w3, *w4;  // row-major [out][in]: (128, 10), (128, 128), (128, 128), (6, 128)
  const float *b1, *b2, *b3, *b4;          // (128), (128), (128), (6)
};

// shared memory of the forward kernels
struct FwdSmem {
  alignas(1024) unsigned char w1[NH * KIN * 2];
  alignas(1024) unsigned char w2[NH * NH * 2];
  alignas(1024) unsigned char w3[NH * NH * 2];
  alignas(1024) unsigned char w4[KOUT * NH * 2];
  alignas(1024) unsigned char a0[ROWS * KIN * 2];
  alignas(1024) unsigned char a[ROWS * NH * 2];
  float b1[NH], b2[NH], b3[NH], b4[KOUT];
  uint64_t bar;
  uint32_t tmem;
};

// weights of one layer into its K-major operand, zero-padded to (rows, K)
__device__ __forceinline__ void load_w(unsigned char *dst, const __nv_bfloat16 *src, int out, int in, int rows, int K) {
  for (int e = threadIdx.x; e < rows * K; e += blockDim.x) {
    const int r = e / K, k = e - r * K;
    const __nv_bfloat16 v = (r < out && k < in) ? src[(size_t)r * in + k] : __float2bfloat16_rn(0.f);
    *reinterpret_cast<__nv_bfloat16 *>(dst + kmaj(r, k, K)) = v;
  }
}

__device__ __forceinline__ void fwd_setup(FwdSmem &S, const MlpWeights &W) {
  load_w(S.w1, W.w1, NH, NIN, NH, KIN);
  load_w(S.w2, W.w2, NH, NH, NH, NH);
  load_w(S.w3, W.w3, NH, NH, NH, NH);
  load_w(S.w4, W.w4, NOUT, NH, KOUT, NH);
  for (int e = threadIdx.x; e < NH; e += blockDim.x) {
    S.b1[e] = W.b1[e];
    S.b2[e] = W.b2[e];
    S.b3[e] = W.b3[e];
  }
  for (int e = threadIdx.x; e < KOUT; e += blockDim.x) S.b4[e] = e < NOUT ? W.b4[e] : 0.f;
  if (threadIdx.x < 32) tmem_alloc(&S.tmem, 128);
  if (threadIdx.x == 0) {
    mbar_init(&S.bar, 1);
    mbar_fence_init();
  }
  operands_ready();
}

__device__ __forceinline__ void fwd_teardown(FwdSmem &S, uint32_t phase, bool ok) {
  if (!ok) mbar_wait_bounded(&S.bar, phase, nullptr, 1 << 22);  // a late MMA still owns the accumulator
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_free(S.tmem, 128);
}

// Hidden-layer epilogue: this thread's row of the accumulator plus bias, SiLU, into row r of
// the next operand; zpre (optional, row-major global [128 cols]) receives the pre-activation.
__device__ __forceinline__ void hidden_epilogue(FwdSmem &S, const float *bias, __nv_bfloat16 *zpre) {
  const uint32_t tl = lane_base(S.tmem);
  const int r = threadIdx.x;
#pragma unroll 1
  for (int c0 = 0; c0 < NH; c0 += 32) {
    float v[32];
    tmem_ld32(tl + c0, v);
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] += bias[c0 + i];
#pragma unroll
    for (int i = 0; i < 32; i += 8) {
      __align__(16) __nv_bfloat162 z[4], h[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        z[q] = __floats2bfloat162_rn(v[i + 2 * q], v[i + 2 * q + 1]);
        h[q] = silu2(z[q]);
      }
      if (zpre) *reinterpret_cast<uint4 *>(zpre + c0 + i) = *reinterpret_cast<const uint4 *>(z);
      *reinterpret_cast<uint4 *>(S.a + kmaj(r, c0 + i, NH)) = *reinterpret_cast<const uint4 *>(h);
    }
  }
}

// The four layers of one tile whose inputs are already in S.a0; y receives this thread's
// outputs (KOUT values, the first NOUT used).  z (optional): pre-activations of the three
// hidden layers, row-major (3, 128) per row.  False when an MMA wait ran out.
__device__ __forceinline__ bool fwd_tile(FwdSmem &S, uint32_t &phase, int *status, float *y, __nv_bfloat16 *z1,
                                         __nv_bfloat16 *z2, __nv_bfloat16 *z3) {
  operands_ready();
  if (threadIdx.x == 0) {
    gemm_issue(S.tmem, S.a0, S.w1, KIN, NH, false);
    mma_commit(&S.bar);
  }
  if (!mma_wait(&S.bar, phase, status)) return false;
  hidden_epilogue(S, S.b1, z1);
  operands_ready();
  if (threadIdx.x == 0) {
    gemm_issue(S.tmem, S.a, S.w2, NH, NH, false);
    mma_commit(&S.bar);
  }
  if (!mma_wait(&S.bar, phase, status)) return false;
  hidden_epilogue(S, S.b2, z2);
  operands_ready();
  if (threadIdx.x == 0) {
    gemm_issue(S.tmem, S.a, S.w3, NH, NH, false);
    mma_commit(&S.bar);
  }
  if (!mma_wait(&S.bar, phase, status)) return false;
  hidden_epilogue(S, S.b3, z3);
  operands_ready();
  if (threadIdx.x == 0) {
    gemm_issue(S.tmem, S.a, S.w4, NH, KOUT, false);
    mma_commit(&S.bar);
  }
  if (!mma_wait(&S.bar, phase, status)) return false;
  tmem_ld16(lane_base(S.tmem), y);
#pragma unroll
  for (int i = 0; i < KOUT; ++i) y[i] += S.b4[i];
  tc_fence_before();
  return true;
}

// ------------------------------------------------------------------------------------------
// batched inference on given inputs (n rows of KIN BF16 inputs, already normalised)
// ------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(NTHREADS, 2) mlp_forward_kernel(MlpWeights W, const __nv_bfloat16 *x, int64_t n,
                                                                  float *y, int *status) {
  pdl_wait();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  fwd_setup(S, W);
  uint32_t phase = 0;
  bool ok = true;
  const int64_t ntiles = (n + ROWS - 1) / ROWS;
  for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int64_t row = t * ROWS + threadIdx.x;
    const bool valid = row < n;
    uint4 in0 = make_uint4(0, 0, 0, 0), in1 = make_uint4(0, 0, 0, 0);
    if (valid) {
      in0 = reinterpret_cast<const uint4 *>(x + row * KIN)[0];
      in1 = reinterpret_cast<const uint4 *>(x + row * KIN)[1];
    }
    *reinterpret_cast<uint4 *>(S.a0 + kmaj(threadIdx.x, 0, KIN)) = in0;
    *reinterpret_cast<uint4 *>(S.a0 + kmaj(threadIdx.x, 8, KIN)) = in1;
    float out[KOUT];
    ok = fwd_tile(S, phase, status, out, nullptr, nullptr, nullptr);
    if (ok && valid)
      for (int i = 0; i < NOUT; ++i) y[row * NOUT + i] = out[i];
  }
  fwd_teardown(S, phase, ok);
}

// ------------------------------------------------------------------------------------------
// training: forward with the pre-activations kept, the loss and its gradient
// ------------------------------------------------------------------------------------------

struct TrainFwdParams {
  MlpWeights W;
  const __nv_bfloat16 *x;   // (N, KIN) normalised inputs
  const float *t;           // (N, NOUT) normalised targets
  const int32_t *idx;       // (B) sample rows of this batch
  int32_t batch;
  __nv_bfloat16 *z;         // (3, B, 128) pre-activations
  __nv_bfloat16 *dy;        // (B, KOUT) d loss / d output (zero-padded)
  double *loss;             // sum of squared errors (accumulated)
  int *status;
};

__global__ void __launch_bounds__(NTHREADS, 2) mlp_train_forward_kernel(const __grid_constant__ TrainFwdParams P) {
  pdl_wait();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  fwd_setup(S, P.W);
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (P.batch + ROWS - 1) / ROWS;
  const float gscale = 2.0f / ((float)P.batch * (float)NOUT);
  double sse = 0.0;
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int b = t * ROWS + threadIdx.x;
    const bool valid = b < P.batch;
    const int64_t src = valid ? (int64_t)P.idx[b] : 0;
    uint4 in0 = make_uint4(0, 0, 0, 0), in1 = make_uint4(0, 0, 0, 0);
    if (valid) {
      in0 = reinterpret_cast<const uint4 *>(P.x + src * KIN)[0];
      in1 = reinterpret_cast<const uint4 *>(P.x + src * KIN)[1];
    }
    *reinterpret_cast<uint4 *>(S.a0 + kmaj(threadIdx.x, 0, KIN)) = in0;
    *reinterpret_cast<uint4 *>(S.a0 + kmaj(threadIdx.x, 8, KIN)) = in1;
    const size_t zs = (size_t)P.batch * NH;
    const size_t zr = (size_t)(valid ? b : 0) * NH;
    float out[KOUT];
    // invalid rows of the last tile write their pre-activations over row 0's and restore
    // nothing: they are computed from zero inputs, so the batch must be a multiple of 128
    ok = fwd_tile(S, phase, P.status, out, P.z + zr, P.z + zs + zr, P.z + 2 * zs + zr);
    if (ok && valid) {
      __align__(16) __nv_bfloat16 d[KOUT];
#pragma unroll
      for (int i = 0; i < KOUT; ++i) {
        float g = 0.f;
        if (i < NOUT) {
          const float e = out[i] - P.t[src * NOUT + i];
          sse += (double)e * (double)e;
          g = gscale * e;
        }
        d[i] = __float2bfloat16_rn(g);
      }
      reinterpret_cast<uint4 *>(P.dy + (size_t)b * KOUT)[0] = reinterpret_cast<const uint4 *>(d)[0];
      reinterpret_cast<uint4 *>(P.dy + (size_t)b * KOUT)[1] = reinterpret_cast<const uint4 *>(d)[1];
    }
  }
  // block sum of the squared errors, one atomic per block
  for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(0xffffffffu, sse, o);
  __shared__ double red[NTHREADS / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sse;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < NTHREADS / 32; ++w) s += red[w];
    atomicAdd(P.loss, s);
  }
  fwd_teardown(S, phase, ok);
}

// ------------------------------------------------------------------------------------------
// training: backward through one layer
// ------------------------------------------------------------------------------------------
//
// Layer l (1-based) maps h_{l-1} (K_in wide) to z_l (N_out wide): z_l = h_{l-1} W_l^T + b_l,
// h_l = silu(z_l) (no activation after layer 4).  Given dz_l (B x N_out), one launch forms
//   dW_l += dz_l^T h_{l-1}   (tensor cores, FP32 accumulator over this CTA's tiles),
//   db_l += column sums of dz_l,
//   dz_{l-1} = (dz_l W_l) * silu'(z_{l-1})   (layers 2..4; tensor cores),
// and adds its CTA's dW_l, db_l to the FP32 gradients with one atomic per entry.

struct TrainBwdParams {
  int layer;                  // 4, 3, 2 or 1
  int32_t batch;
  const __nv_bfloat16 *w;     // W_l, row-major [n_out][k_in]
  int n_out, k_in;            // true widths (6 / 128 / 128 / 128 and 128 / 128 / 128 / 10)
  const __nv_bfloat16 *dz;    // (B, DZW) gradient of z_l (DZW = 16 for layer 4, else 128)
  const __nv_bfloat16 *zin;   // (B, 128) pre-activation of layer l-1 (layers 2..4)
  const __nv_bfloat16 *x;     // (N, KIN) inputs (layer 1)
  const int32_t *idx;         // (B) batch rows (layer 1)
  __nv_bfloat16 *dz_prev;     // (B, 128) gradient of z_{l-1} (layers 2..4)
  float *gw, *gb;             // FP32 gradients of W_l (row-major [n_out][k_in]) and b_l
  int *status;
};

// operand widths of the backward pass of a layer: DZW = padded n_out, HW = padded k_in
struct BwdSmem {
  alignas(1024) unsigned char wt[NH * NH * 2];     // W_l^T as B of dh = dz W: (k_in rows) x (n_out cols)
  alignas(1024) unsigned char dz[ROWS * NH * 2];   // dz as A of dh: (128 rows) x (n_out cols)
  alignas(1024) unsigned char dzt[NH * ROWS * 2];  // dz^T as A of dW: (n_out rows) x (128 cols)
  alignas(1024) unsigned char ht[(NH + 16) * ROWS * 2];  // h^T (+ a ones row block) as B of dW
  float gb[NH];
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(NTHREADS, 1) mlp_train_backward_kernel(const __grid_constant__ TrainBwdParams P) {
  pdl_wait();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  BwdSmem &S = *reinterpret_cast<BwdSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int L = P.layer;
  const int DZW = L == 4 ? KOUT : NH;   // padded width of dz_l
  const int HW = L == 1 ? KIN : NH;     // padded width of h_{l-1}
  const bool prev = L > 1;
  const int tid = threadIdx.x;
  // W_l^T: element (r = input j, c = output i) = W[i][j], K = DZW columns
  if (prev)
    for (int e = tid; e < NH * DZW; e += NTHREADS) {
      const int r = e / DZW, c = e - r * DZW;
      const __nv_bfloat16 v = (c < P.n_out && r < P.k_in) ? P.w[(size_t)c * P.k_in + r] : __float2bfloat16_rn(0.f);
      *reinterpret_cast<__nv_bfloat16 *>(S.wt + kmaj(r, c, DZW)) = v;
    }
  // the ones block of h^T: rows HW .. HW + 15 of the dW operand all ones, so that columns
  // HW .. HW + 15 of the dW accumulator are the column sums of dz (the bias gradient); only
  // for DZW = 128 (the M = 128 side of dW); layer 4 sums its 6 columns with shuffles
  const bool ones = DZW == NH;
  if (ones)
    for (int e = tid; e < 16 * ROWS; e += NTHREADS) {
      const int r = HW + e / ROWS, c = e % ROWS;
      *reinterpret_cast<__nv_bfloat16 *>(S.ht + kmaj(r, c, ROWS)) = __float2bfloat16_rn(1.f);
    }
  if (tid < NH) S.gb[tid] = 0.f;
  // tensor memory: dW accumulator (columns 0 .. 255) and dh accumulator (256 .. 383)
  if (tid < 32) tmem_alloc(&S.tmem, 512);
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    mbar_fence_init();
  }
  operands_ready();
  const uint32_t t_dw = S.tmem, t_dh = S.tmem + 256;
  // dW: layer 4 computes dW^T = h^T dz (M = 128 inputs, N = 16 outputs); the others
  // dW = dz^T h (M = 128 outputs, N = HW inputs + 16 ones)
  const int dw_n = L == 4 ? KOUT : HW + 16;
  uint32_t phase = 0;
  bool ok = true, first = true;
  const int ntiles = (P.batch + ROWS - 1) / ROWS;
  float gb4[KOUT];
#pragma unroll
  for (int i = 0; i < KOUT; ++i) gb4[i] = 0.f;
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int b = t * ROWS + tid;
    const bool valid = b < P.batch;
    // dz row b -> dz (row tid) and dz^T (column tid)
    for (int c0 = 0; c0 < DZW; c0 += 8) {
      uint4 raw = make_uint4(0, 0, 0, 0);
      if (valid) raw = *reinterpret_cast<const uint4 *>(P.dz + (size_t)b * DZW + c0);
      *reinterpret_cast<uint4 *>(S.dz + kmaj(tid, c0, DZW)) = raw;
      const __nv_bfloat16 *v = reinterpret_cast<const __nv_bfloat16 *>(&raw);
      for (int i = 0; i < 8; ++i) {
        if (L == 4) {
          *reinterpret_cast<__nv_bfloat16 *>(S.dzt + kmaj(c0 + i, tid, ROWS)) = v[i];   // dz^T as B (N = 16)
          gb4[c0 + i] += __bfloat162float(v[i]);
        } else {
          *reinterpret_cast<__nv_bfloat16 *>(S.dzt + kmaj(c0 + i, tid, ROWS)) = v[i];   // dz^T as A (M = 128)
        }
      }
    }
    // h_{l-1} row b -> h^T (column tid): silu of the stored pre-activation, or the inputs
    for (int c0 = 0; c0 < HW; c0 += 8) {
      uint4 raw = make_uint4(0, 0, 0, 0);
      if (valid) {
        raw = L == 1 ? *reinterpret_cast<const uint4 *>(P.x + (size_t)P.idx[b] * KIN + c0)
                     : *reinterpret_cast<const uint4 *>(P.zin + (size_t)b * NH + c0);
      }
      if (L != 1) {   // h = silu(z) exactly as the forward pass formed it
        __nv_bfloat162 *pr = reinterpret_cast<__nv_bfloat162 *>(&raw);
        for (int q = 0; q < 4; ++q) pr[q] = silu2(pr[q]);
      }
      const __nv_bfloat16 *v = reinterpret_cast<const __nv_bfloat16 *>(&raw);
      for (int i = 0; i < 8; ++i)
        *reinterpret_cast<__nv_bfloat16 *>(S.ht + kmaj(c0 + i, tid, ROWS)) = valid ? v[i] : __float2bfloat16_rn(0.f);
    }
    operands_ready();
    if (tid == 0) {
      if (L == 4)
        gemm_issue(t_dw, S.ht, S.dzt, ROWS, KOUT, !first);       // dW^T (128 x 16) += h^T dz
      else
        gemm_issue(t_dw, S.dzt, S.ht, ROWS, dw_n, !first);       // dW (128 x HW+16) += dz^T [h | 1]
      if (prev) gemm_issue(t_dh, S.dz, S.wt, DZW, NH, false);    // dh (128 x 128) = dz W
      mma_commit(&S.bar);
    }
    first = false;
    ok = mma_wait(&S.bar, phase, P.status);
    if (ok && prev) {  // dz_{l-1} = dh * silu'(z_{l-1}) for this thread's row
      const uint32_t tl = lane_base(t_dh);
      for (int c0 = 0; c0 < NH; c0 += 32) {
        float v[32];
        tmem_ld32(tl + c0, v);
        if (valid) {
          for (int i = 0; i < 32; i += 8) {
            const uint4 zr = *reinterpret_cast<const uint4 *>(P.zin + (size_t)b * NH + c0 + i);
            const __nv_bfloat16 *z = reinterpret_cast<const __nv_bfloat16 *>(&zr);
            __align__(16) __nv_bfloat16 d[8];
            for (int q = 0; q < 8; ++q) d[q] = __float2bfloat16_rn(v[i + q] * silu_grad(__bfloat162float(z[q])));
            *reinterpret_cast<uint4 *>(P.dz_prev + (size_t)b * NH + c0 + i) = *reinterpret_cast<const uint4 *>(d);
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();   // the operands of this tile are free for the next one
  }
  if (ok) {
    // this CTA's dW and db to the global FP32 gradients (thread = accumulator lane)
    const uint32_t tl = lane_base(t_dw);
    const int r = tid;
    if (L == 4) {  // lane r = input r; columns = outputs
      float v[16];
      tmem_ld16(tl, v);
      if (r < P.k_in)
        for (int i = 0; i < P.n_out; ++i) atomicAdd(P.gw + (size_t)i * P.k_in + r, v[i]);
      for (int i = 0; i < KOUT; ++i) {
        float s = gb4[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0 && i < P.n_out) atomicAdd(&S.gb[i], s);
      }
    } else {       // lane r = output r; columns = inputs, then the 16 ones columns
      for (int c0 = 0; c0 < dw_n; c0 += 16) {
        float v[16];
        tmem_ld16(tl + c0, v);
        for (int i = 0; i < 16; ++i) {
          const int c = c0 + i;
          if (r < P.n_out && c < P.k_in) atomicAdd(P.gw + (size_t)r * P.k_in + c, v[i]);
          if (c == HW && r < P.n_out) S.gb[r] = v[i];
        }
      }
    }
    __syncthreads();
    if (tid < P.n_out) atomicAdd(P.gb + tid, S.gb[tid]);
  }
  if (!ok) mbar_wait_bounded(&S.bar, phase, nullptr, 1 << 22);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid < 32) tmem_free(S.tmem, 512);
}

// ------------------------------------------------------------------------------------------
// Adam on the FP32 master parameters, with the BF16 copies the kernels read
// ------------------------------------------------------------------------------------------

__global__ void adam_kernel(float *p, float *m, float *v, float *g, __nv_bfloat16 *pb, int64_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  pdl_wait();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
    g[i] = 0.f;
  }
}

// ------------------------------------------------------------------------------------------
// training pairs: F x F x F box filter of a periodic fine run
// ------------------------------------------------------------------------------------------
//
// Fine grid n^3 (periodic, u (n, n, n + 1) with the duplicate face), coarse m = n / F.
// filt_kernel: per coarse cell the filtered cell-centred velocities' products, tau_ab =
// mean(u_a u_b) - mean(u_a) mean(u_b) over the F^3 fine cells (xx, yy, zz, xy, xz, yz), and
// the coarse face velocities (the F x F fine faces on each coarse face averaged: the
// restriction that keeps the discrete divergence zero).  grad_kernel: the coarse gradient by
// the step's own stencil (core.py:400-445: face differences on the diagonal, averages of four
// edge differences off it, g33 = -(g11 + g22)) with periodic neighbours, spacing F h.

__global__ void filt_kernel(const float *u, const float *v, const float *w, int n, int F, float *U, float *V, float *Wc,
                            float *tau) {
  pdl_wait();
  const int m = n / F;
  const int64_t cells = (int64_t)m * m * m;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int I = (int)(c % m), J = (int)((c / m) % m), K = (int)(c / ((int64_t)m * m));
    double s[3] = {0, 0, 0}, p[6] = {0, 0, 0, 0, 0, 0};
    double fu = 0, fv = 0, fw = 0;
    for (int dk = 0; dk < F; ++dk)
      for (int dj = 0; dj < F; ++dj)
        for (int di = 0; di < F; ++di) {
          const int k = K * F + dk, j = J * F + dj, i = I * F + di;
          const float uc = 0.5f * (u[((size_t)k * n + j) * (n + 1) + i] + u[((size_t)k * n + j) * (n + 1) + i + 1]);
          const float vc = 0.5f * (v[((size_t)k * (n + 1) + j) * n + i] + v[((size_t)k * (n + 1) + j + 1) * n + i]);
          const float wc = 0.5f * (w[((size_t)k * n + j) * n + i] + w[((size_t)(k + 1) * n + j) * n + i]);
          s[0] += uc;
          s[1] += vc;
          s[2] += wc;
          p[0] += (double)uc * uc;
          p[1] += (double)vc * vc;
          p[2] += (double)wc * wc;
          p[3] += (double)uc * vc;
          p[4] += (double)uc * wc;
          p[5] += (double)vc * wc;
          if (di == 0) fu += u[((size_t)k * n + j) * (n + 1) + i];
          if (dj == 0) fv += v[((size_t)k * (n + 1) + j) * n + i];
          if (dk == 0) fw += w[((size_t)k * n + j) * n + i];
        }
    const double inv = 1.0 / ((double)F * F * F), inv2 = 1.0 / ((double)F * F);
    const double a[3] = {s[0] * inv, s[1] * inv, s[2] * inv};
    tau[0 * cells + c] = (float)(p[0] * inv - a[0] * a[0]);
    tau[1 * cells + c] = (float)(p[1] * inv - a[1] * a[1]);
    tau[2 * cells + c] = (float)(p[2] * inv - a[2] * a[2]);
    tau[3 * cells + c] = (float)(p[3] * inv - a[0] * a[1]);
    tau[4 * cells + c] = (float)(p[4] * inv - a[0] * a[2]);
    tau[5 * cells + c] = (float)(p[5] * inv - a[1] * a[2]);
    U[c] = (float)(fu * inv2);
    V[c] = (float)(fv * inv2);
    Wc[c] = (float)(fw * inv2);
  }
}

__global__ void grad_kernel(const float *U, const float *V, const float *Wc, int m, float inv_d, float *g8) {
  pdl_wait();
  const int64_t cells = (int64_t)m * m * m;
  auto at = [m](const float *a, int k, int j, int i) {
    k = (k + m) % m;
    j = (j + m) % m;
    i = (i + m) % m;
    return a[((size_t)k * m + j) * m + i];
  };
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % m), j = (int)((c / m) % m), k = (int)(c / ((int64_t)m * m));
    const float q = 0.25f, h = inv_d;
    // u faces i, i + 1 of cell (k, j); v faces j, j + 1; w faces k, k + 1 (core.py:400-434)
    const float g11 = (at(U, k, j, i + 1) - at(U, k, j, i)) * h;
    const float g22 = (at(V, k, j + 1, i) - at(V, k, j, i)) * h;
    const float g12 = ((((at(U, k, j, i) - at(U, k, j - 1, i)) * h + (at(U, k, j + 1, i) - at(U, k, j, i)) * h) +
                        (at(U, k, j, i + 1) - at(U, k, j - 1, i + 1)) * h) +
                       (at(U, k, j + 1, i + 1) - at(U, k, j, i + 1)) * h) * q;
    const float g13 = ((((at(U, k, j, i) - at(U, k - 1, j, i)) * h + (at(U, k + 1, j, i) - at(U, k, j, i)) * h) +
                        (at(U, k, j, i + 1) - at(U, k - 1, j, i + 1)) * h) +
                       (at(U, k + 1, j, i + 1) - at(U, k, j, i + 1)) * h) * q;
    const float g21 = ((((at(V, k, j, i) - at(V, k, j, i - 1)) * h + (at(V, k, j + 1, i) - at(V, k, j + 1, i - 1)) * h) +
                        (at(V, k, j, i + 1) - at(V, k, j, i)) * h) +
                       (at(V, k, j + 1, i + 1) - at(V, k, j + 1, i)) * h) * q;
    const float g23 = ((((at(V, k, j, i) - at(V, k - 1, j, i)) * h + (at(V, k + 1, j, i) - at(V, k, j, i)) * h) +
                        (at(V, k, j + 1, i) - at(V, k - 1, j + 1, i)) * h) +
                       (at(V, k + 1, j + 1, i) - at(V, k, j + 1, i)) * h) * q;
    const float g31 = ((((at(Wc, k, j, i) - at(Wc, k, j, i - 1)) * h + (at(Wc, k + 1, j, i) - at(Wc, k + 1, j, i - 1)) * h) +
                        (at(Wc, k, j, i + 1) - at(Wc, k, j, i)) * h) +
                       (at(Wc, k + 1, j, i + 1) - at(Wc, k + 1, j, i)) * h) * q;
    const float g32 = ((((at(Wc, k, j, i) - at(Wc, k, j - 1, i)) * h + (at(Wc, k + 1, j, i) - at(Wc, k + 1, j - 1, i)) * h) +
                        (at(Wc, k, j + 1, i) - at(Wc, k, j, i)) * h) +
                       (at(Wc, k + 1, j + 1, i) - at(Wc, k + 1, j, i)) * h) * q;
    const float gg[8] = {g11, g12, g13, g21, g22, g23, g31, g32};
    for (int q8 = 0; q8 < 8; ++q8) g8[q8 * cells + c] = gg[q8];
  }
}

// ------------------------------------------------------------------------------------------
// features, targets and the normalised training inputs
// ------------------------------------------------------------------------------------------

struct NormParams {
  float in_mean[NIN], in_std[NIN], in_lo[NIN], in_hi[NIN];
  float out_mean[NOUT], out_std[NOUT];
};

// raw features (n, NIN) and the output scale Delta^2 |g|^2 of n gradients (SoA, 8 x n), with
// validity; with tau (SoA 6 x n) also the scaled targets tau / (Delta^2 |g|^2) (n, NOUT)
__global__ void features_kernel(const float *g8, int64_t n, float delta, float *feat, float *scale, uint8_t *valid,
                                const float *tau, float *target) {
  pdl_wait();
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    float g[8], f[NIN];
    for (int q = 0; q < 8; ++q) g[q] = g8[q * n + c];
    Grad G;
    const bool ok = features(g, f, G);
    for (int q = 0; q < NIN; ++q) feat[c * NIN + q] = f[q];
    const float sc = delta * delta * G.g2;
    scale[c] = sc;
    valid[c] = ok ? 1 : 0;
    if (tau)
      for (int q = 0; q < NOUT; ++q) target[c * NOUT + q] = ok ? tau[q * n + c] / sc : 0.f;
  }
}

// normalised BF16 inputs (n, KIN; zero-padded) and FP32 targets (n, NOUT) of raw rows
__global__ void normalise_kernel(const float *feat, const float *target, int64_t n, NormParams N, __nv_bfloat16 *x,
                                 float *t) {
  pdl_wait();
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 r[KIN];
    for (int q = 0; q < KIN; ++q)
      r[q] = __float2bfloat16_rn(q < NIN ? (feat[c * NIN + q] - N.in_mean[q]) / N.in_std[q] : 0.f);
    reinterpret_cast<uint4 *>(x + c * KIN)[0] = reinterpret_cast<const uint4 *>(r)[0];
    reinterpret_cast<uint4 *>(x + c * KIN)[1] = reinterpret_cast<const uint4 *>(r)[1];
    if (target)
      for (int q = 0; q < NOUT; ++q) t[c * NOUT + q] = (target[c * NOUT + q] - N.out_mean[q]) / N.out_std[q];
  }
}

// ------------------------------------------------------------------------------------------
// the closure in the step: eddy viscosity of the learned stress, WALE where it does not apply
// ------------------------------------------------------------------------------------------
//
// Input: the eight gradient components and the window factor (1 - chi_c) of every cell of the
// padded (nz + 2, ny + 2, nx + 2) nu array (SoA, stride `plane` between components), written by
// the eddy-viscosity pass together with its WALE nu_t.  Per cell: features, the MLP's stress
// tau = Delta^2 |g|^2 (y * out_std + out_mean), its dissipation eps = -tau : S, and
//   nu_t = fac * eps / (2 S : S)   where eps > 0 and every input lies in the training range,
// else the WALE value stays.  The maximum of the final nu_t (for the time step) is returned as
// an ordered FP32 bit pattern, like the other maxima of the step.

struct ClosureStepParams {
  MlpWeights W;
  NormParams N;
  const float *grad;          // (9, plane): g11 g12 g13 g21 g22 g23 g31 g32, window factor
  int64_t plane;              // elements per component (padded array incl. row pitch)
  int nxp, nyp, nzp, pitch;   // padded extents (nx + 2, ny + 2, nz + 2) and the row pitch
  float delta;                // filter width (the cell size)
  float *nu;                  // (nzp, nyp, pitch) nu_t: WALE in, closure out
  unsigned long long *nut_max;
  unsigned long long *counts; // [0] cells evaluated, [1] cells that kept WALE
  int *status;
};

__device__ __forceinline__ void max_atomic_f32(unsigned long long *dst, float v) {
  // the step keeps maxima as ordered bit patterns of doubles (non-negative values)
  const double d = (double)v;
  atomicMax(dst, (unsigned long long)__double_as_longlong(d));
}

// The deployed pass keeps four 128-row pipelines in flight per SM inside one CTA of 512
// threads: the four warpgroups share one copy of the weights (72 KB) and each owns its input
// and activation operands (36 KB), its 128 tensor-memory columns (all 512 of the SM) and its
// mbarrier, and synchronises only its own 128 threads (named barriers 1..4).  While one
// warpgroup runs an epilogue the tensor cores run another's layer, so the latency of the
// MMA -> epilogue -> MMA chain of a tile is hidden by the other three.  (Two CTAs of one
// pipeline each held two weight copies and ran two pipelines per SM.)
constexpr int NPIPE = 4;

struct PipeSmem {
  alignas(1024) unsigned char a0[ROWS * KIN * 2];
  alignas(1024) unsigned char a[ROWS * NH * 2];
};

struct Fwd4Smem {
  alignas(1024) unsigned char w1[NH * KIN * 2];
  alignas(1024) unsigned char w2[NH * NH * 2];
  alignas(1024) unsigned char w3[NH * NH * 2];
  alignas(1024) unsigned char w4[KOUT * NH * 2];
  PipeSmem pipe[NPIPE];
  alignas(16) float b1[NH], b2[NH], b3[NH], b4[KOUT];
  uint64_t bar[NPIPE];
  uint32_t tmem;
};

// barrier of the 128 threads of warpgroup `wg` (named barrier 1 + wg; 0 is __syncthreads)
__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(wg + 1) : "memory"); }
// the same, true in every thread when `pred` holds in any of them
__device__ __forceinline__ bool wg_sync_or(int wg, bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, %2, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)pred), "r"(wg + 1)
      : "memory");
  return out != 0;
}

struct Pipe {
  unsigned char *a0, *a;
  uint64_t *bar;
  uint32_t tmem;   // tensor-memory address of this pipeline's first column
  int wg, r;       // warpgroup and the row (lane) of this thread
};

__device__ __forceinline__ void pipe_ready(const Pipe &q) {
  fence_proxy_async();
  tc_fence_before();
  wg_sync(q.wg);
  tc_fence_after();
}

// the pipeline's leader polls the MMA barrier (bounded); the other 127 threads sleep at the
// named barrier instead of spending issue slots on polls of their own
__device__ __forceinline__ bool pipe_wait(const Pipe &q, uint32_t &phase, int *status) {
  const bool ok = q.r != 0 || mbar_wait_bounded(q.bar, phase, nullptr, 1 << 22);
  phase ^= 1u;
  const bool bad = wg_sync_or(q.wg, !ok);
  if (bad && q.r == 0 && status) atomicOr(status, STATUS_TIMEOUT);
  tc_fence_after();
  return !bad;
}

__device__ __forceinline__ void pipe_epilogue(const Pipe &q, const float *bias) {
  const uint32_t tl = q.tmem + ((uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16);
#pragma unroll 1
  for (int c0 = 0; c0 < NH; c0 += 32) {
    float v[32];
    tmem_ld32(tl + c0, v);
#pragma unroll
    for (int i = 0; i < 32; i += 4) {   // the bias in 16-byte loads
      const float4 b = *reinterpret_cast<const float4 *>(bias + c0 + i);
      v[i] += b.x;
      v[i + 1] += b.y;
      v[i + 2] += b.z;
      v[i + 3] += b.w;
    }
#pragma unroll
    for (int i = 0; i < 32; i += 8) {
      __align__(16) __nv_bfloat162 h[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) h[k] = silu2(__floats2bfloat162_rn(v[i + 2 * k], v[i + 2 * k + 1]));
      *reinterpret_cast<uint4 *>(q.a + kmaj(q.r, c0 + i, NH)) = *reinterpret_cast<const uint4 *>(h);
    }
  }
}

// the four layers of one tile of this pipeline (inputs in q.a0); false when a wait ran out
__device__ __forceinline__ bool pipe_tile(const Pipe &q, const Fwd4Smem &S, uint32_t &phase, int *status, float *y) {
  const bool lead = q.r == 0;
  pipe_ready(q);
  if (lead) {
    gemm_issue(q.tmem, q.a0, S.w1, KIN, NH, false);
    mma_commit(q.bar);
  }
  if (!pipe_wait(q, phase, status)) return false;
  pipe_epilogue(q, S.b1);
  pipe_ready(q);
  if (lead) {
    gemm_issue(q.tmem, q.a, S.w2, NH, NH, false);
    mma_commit(q.bar);
  }
  if (!pipe_wait(q, phase, status)) return false;
  pipe_epilogue(q, S.b2);
  pipe_ready(q);
  if (lead) {
    gemm_issue(q.tmem, q.a, S.w3, NH, NH, false);
    mma_commit(q.bar);
  }
  if (!pipe_wait(q, phase, status)) return false;
  pipe_epilogue(q, S.b3);
  pipe_ready(q);
  if (lead) {
    gemm_issue(q.tmem, q.a, S.w4, NH, KOUT, false);
    mma_commit(q.bar);
  }
  if (!pipe_wait(q, phase, status)) return false;
  tmem_ld16(q.tmem + ((uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16), y);
#pragma unroll
  for (int i = 0; i < KOUT; ++i) y[i] += S.b4[i];
  tc_fence_before();
  return true;
}

__global__ void __launch_bounds__(NPIPE * ROWS, 1) closure_nu_kernel(const __grid_constant__ ClosureStepParams P) {
  pdl_wait();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Fwd4Smem &S = *reinterpret_cast<Fwd4Smem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // weights, biases, barriers and all 512 tensor-memory columns, for the whole CTA
  load_w(S.w1, P.W.w1, NH, NIN, NH, KIN);
  load_w(S.w2, P.W.w2, NH, NH, NH, NH);
  load_w(S.w3, P.W.w3, NH, NH, NH, NH);
  load_w(S.w4, P.W.w4, NOUT, NH, KOUT, NH);
  for (int e = threadIdx.x; e < NH; e += blockDim.x) {
    S.b1[e] = P.W.b1[e];
    S.b2[e] = P.W.b2[e];
    S.b3[e] = P.W.b3[e];
  }
  for (int e = threadIdx.x; e < KOUT; e += blockDim.x) S.b4[e] = e < NOUT ? P.W.b4[e] : 0.f;
  if (threadIdx.x < 32) tmem_alloc(&S.tmem, NPIPE * NH);
  if (threadIdx.x == 0) {
    for (int w = 0; w < NPIPE; ++w) mbar_init(&S.bar[w], 1);
    mbar_fence_init();
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const int wg = threadIdx.x / ROWS;
  const Pipe q{S.pipe[wg].a0, S.pipe[wg].a, &S.bar[wg], S.tmem + (uint32_t)(wg * NH), wg, (int)(threadIdx.x % ROWS)};
  uint32_t phase = 0;
  bool ok = true;
  const int64_t total = P.plane;
  const int64_t ntiles = (total + ROWS - 1) / ROWS;
  float mx = 0.f;
  unsigned long long n_eval = 0, n_wale = 0;
  for (int64_t t = (int64_t)blockIdx.x * NPIPE + wg; t < ntiles && ok; t += (int64_t)gridDim.x * NPIPE) {
    const int64_t e = t * ROWS + q.r;
    const int i = (int)(e % P.pitch);
    const bool cell = e < total && i < P.nxp;
    float g[8], f[NIN], fac = 0.f;
    Grad G;
    bool use = false;
    if (cell) {
      for (int c = 0; c < 8; ++c) g[c] = P.grad[c * P.plane + e];
      fac = P.grad[8 * P.plane + e];
      use = features(g, f, G);
      for (int c = 0; c < NIN; ++c) use = use && f[c] >= P.N.in_lo[c] && f[c] <= P.N.in_hi[c];
    }
    float xin[KIN];
    for (int c = 0; c < KIN; ++c) xin[c] = (use && c < NIN) ? (f[c] - P.N.in_mean[c]) / P.N.in_std[c] : 0.f;
    store8(q.a0, q.r, 0, KIN, xin);
    store8(q.a0, q.r, 8, KIN, xin + 8);
    float y[KOUT];
    ok = pipe_tile(q, S, phase, P.status, y);
    if (!ok || !cell) continue;
    ++n_eval;
    float nut = P.nu[e];
    if (use) {
      const float sc = P.delta * P.delta * G.g2;
      float tau[NOUT];
      for (int c = 0; c < NOUT; ++c) tau[c] = sc * fmaf(y[c], P.N.out_std[c], P.N.out_mean[c]);
      const float eps = -((tau[0] * G.S[0][0] + tau[1] * G.S[1][1] + tau[2] * G.S[2][2]) +
                          2.f * ((tau[3] * G.S[0][1] + tau[4] * G.S[0][2]) + tau[5] * G.S[1][2]));
      if (eps > 0.f && isfinite(eps)) {
        nut = fac * (eps / (2.f * G.s2));
        P.nu[e] = nut;
      } else {
        use = false;
      }
    }
    if (!use) ++n_wale;
    mx = (nut > mx || nut != nut) ? nut : mx;
  }
  // a pipeline that gave up waits (bounded) for its last MMA before the memory is freed
  if (!ok) mbar_wait_bounded(q.bar, phase, nullptr, 1 << 22);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_free(S.tmem, NPIPE * NH);
  // block maximum and counts
  for (int o = 16; o > 0; o >>= 1) {
    const float other = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = (other > mx || other != other) ? other : mx;
    n_eval += __shfl_xor_sync(0xffffffffu, n_eval, o);
    n_wale += __shfl_xor_sync(0xffffffffu, n_wale, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (P.nut_max) max_atomic_f32(P.nut_max, mx);   // NaN wins, as in the other maxima
    if (P.counts) {
      atomicAdd(P.counts, n_eval);
      atomicAdd(P.counts + 1, n_wale);
    }
  }
}

}  // namespace closure
}  // namespace aero

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------

#include <mutex>
#include <string>

#include "host_common.cuh"

namespace {

using namespace aero::closure;

// offsets of the flat parameter array (include/aero_b200.h AERO_CLOSURE_NPARAM)
constexpr int64_t OFF_W1 = 0, OFF_B1 = 1280, OFF_W2 = 1408, OFF_B2 = 17792, OFF_W3 = 17920, OFF_B3 = 34304,
                  OFF_W4 = 34432, OFF_B4 = 35200, NPARAM = 35206;
static_assert(NPARAM == AERO_CLOSURE_NPARAM, "parameter layout");

constexpr size_t FWD_SMEM = sizeof(FwdSmem) + 1024, BWD_SMEM = sizeof(BwdSmem) + 1024;
constexpr size_t FWD4_SMEM = sizeof(Fwd4Smem) + 1024;

MlpWeights weights_of(const float *p, const void *pb) {
  const auto *b = static_cast<const __nv_bfloat16 *>(pb);
  return MlpWeights{b + OFF_W1, b + OFF_W2, b + OFF_W3, b + OFF_W4, p + OFF_B1, p + OFF_B2, p + OFF_B3, p + OFF_B4};
}

NormParams norm_of(const AeroClosureModel *m) {
  NormParams N{};
  for (int q = 0; q < NIN; ++q) {
    N.in_mean[q] = m->in_mean[q];
    N.in_std[q] = m->in_std[q];
    N.in_lo[q] = m->in_lo[q];
    N.in_hi[q] = m->in_hi[q];
  }
  for (int q = 0; q < NOUT; ++q) {
    N.out_mean[q] = m->out_mean[q];
    N.out_std[q] = m->out_std[q];
  }
  return N;
}

// the opt-in shared-memory sizes of the tensor-core kernels and the SM count, once per device
int prepare(int *nsm) {
  static std::mutex mu;
  static int done_dev = -1, sms = 0;
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  AERO_CUDA_TRY(cudaGetDevice(&dev));
  if (done_dev != dev) {
    AERO_CUDA_TRY(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    AERO_CUDA_TRY(
        cudaFuncSetAttribute(mlp_train_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    AERO_CUDA_TRY(cudaFuncSetAttribute(closure_nu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD4_SMEM));
    AERO_CUDA_TRY(
        cudaFuncSetAttribute(mlp_train_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BWD_SMEM));
    AERO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    done_dev = dev;
  }
  *nsm = sms;
  return AERO_OK;
}

bool finite_positive(const float *a, int n) {
  for (int q = 0; q < n; ++q)
    if (!(a[q] > 0.f) || !(a[q] < 3.0e38f)) return false;
  return true;
}

int grid_for(int64_t items, int per_block = 256) {
  const int64_t b = (items + per_block - 1) / per_block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

}  // namespace

// the closure's pass in the step (declared in host_common.cuh)
int aero_host::closure_nu(const AeroClosureModel *m, const float *grad, int64_t plane, int nxp, int nyp, int nzp,
                          int pitch, double delta, float *nu, unsigned long long *nut_max, unsigned long long *counts,
                          int *status, cudaStream_t s) {
  int nsm = 0;
  const int rc = prepare(&nsm);
  if (rc) return rc;
  ClosureStepParams P{};
  P.W = weights_of(m->params, m->params_bf16);
  P.N = norm_of(m);
  P.grad = grad;
  P.plane = plane;
  P.nxp = nxp;
  P.nyp = nyp;
  P.nzp = nzp;
  P.pitch = pitch;
  P.delta = (float)delta;
  P.nu = nu;
  P.nut_max = nut_max;
  P.counts = counts;
  P.status = status;
  const int64_t tiles = (plane + ROWS - 1) / ROWS;
  // two CTAs per SM (shared memory and tensor memory allow it): one CTA's epilogue runs
  // while the other's MMAs do
  const int grid = (int)std::min<int64_t>((tiles + NPIPE - 1) / NPIPE, (int64_t)nsm);   // one CTA per SM
  AERO_CUDA_TRY(aero::launch_k(closure_nu_kernel, grid, NPIPE * ROWS, FWD4_SMEM, s, P));
  return AERO_OK;
}

extern "C" {

int aero_closure_pairs(int32_t n, int32_t factor, const float *u, const float *v, const float *w, double h, float *g8,
                       float *tau, float *work, void *stream) {
  if (!u || !v || !w || !g8 || !tau || !work) return aero_host::set_error(AERO_EINVAL, "null argument");
  if (factor < 1 || n < factor || n % factor) return aero_host::set_error(AERO_EINVAL, "n must be a multiple of factor");
  const int m = n / factor;
  const int64_t cells = (int64_t)m * m * m;
  auto s = static_cast<cudaStream_t>(stream);
  float *U = work, *V = work + cells, *W = work + 2 * cells;
  AERO_CUDA_TRY(aero::launch_k(filt_kernel, grid_for(cells), 256, 0, s, u, v, w, (int)n, (int)factor, U, V, W, tau));
  AERO_CUDA_TRY(aero::launch_k(grad_kernel, grid_for(cells), 256, 0, s, (const float *)U, (const float *)V,
                               (const float *)W, m, (float)(1.0 / (h * factor)), g8));
  return AERO_OK;
}

int aero_closure_features(int64_t n, const float *g8, double delta, const float *tau, float *feat, float *scale,
                          uint8_t *valid, float *target, void *stream) {
  if (!g8 || !feat || !scale || !valid || (tau && !target)) return aero_host::set_error(AERO_EINVAL, "null argument");
  if (n <= 0) return AERO_OK;
  AERO_CUDA_TRY(aero::launch_k(features_kernel, grid_for(n), 256, 0, static_cast<cudaStream_t>(stream), g8, n,
                               (float)delta, feat, scale, valid, tau, target));
  return AERO_OK;
}

int aero_closure_normalise(int64_t n, const float *feat, const float *target, const AeroClosureModel *m, void *x,
                           float *t, void *stream) {
  if (!feat || !m || !x || (target && !t)) return aero_host::set_error(AERO_EINVAL, "null argument");
  if (!finite_positive(m->in_std, NIN) || !finite_positive(m->out_std, NOUT))
    return aero_host::set_error(AERO_EINVAL, "standard deviations must be positive and finite");
  if (reinterpret_cast<uintptr_t>(x) % 16) return aero_host::set_error(AERO_EINVAL, "x must be 16-byte aligned");
  if (n <= 0) return AERO_OK;
  AERO_CUDA_TRY(aero::launch_k(normalise_kernel, grid_for(n), 256, 0, static_cast<cudaStream_t>(stream), feat, target,
                               n, norm_of(m), static_cast<__nv_bfloat16 *>(x), t));
  return AERO_OK;
}

int aero_mlp_forward(const AeroClosureModel *m, const void *x, int64_t n, float *y, int32_t *status, void *stream) {
  if (!m || !m->params || !m->params_bf16 || !x || !y || !status)
    return aero_host::set_error(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(x) % 16) return aero_host::set_error(AERO_EINVAL, "x must be 16-byte aligned");
  if (n <= 0) return AERO_OK;
  int nsm = 0;
  const int rc = prepare(&nsm);
  if (rc) return rc;
  const int64_t tiles = (n + ROWS - 1) / ROWS;
  AERO_CUDA_TRY(aero::launch_k(mlp_forward_kernel, (int)std::min<int64_t>(tiles, 2 * (int64_t)nsm), NTHREADS, FWD_SMEM,
                               static_cast<cudaStream_t>(stream), weights_of(m->params, m->params_bf16),
                               static_cast<const __nv_bfloat16 *>(x), n, y, reinterpret_cast<int *>(status)));
  return AERO_OK;
}

size_t aero_mlp_train_workspace_bytes(int32_t batch) {
  if (batch <= 0) return 0;
  const size_t b = (size_t)batch;
  return aero_host::align_up(3 * b * NH * 2) + aero_host::align_up(b * KOUT * 2) + 2 * aero_host::align_up(b * NH * 2);
}

int aero_mlp_gradients(const float *params, const void *params_bf16, float *grad, const void *x, const float *t,
                       const int32_t *idx, int32_t batch, double *loss, void *workspace, int32_t *status, void *stream) {
  if (!params || !params_bf16 || !grad || !x || !t || !idx || !loss || !workspace || !status)
    return aero_host::set_error(AERO_EINVAL, "null argument");
  if (batch <= 0 || batch % ROWS) return aero_host::set_error(AERO_EINVAL, "batch must be a positive multiple of 128");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN || reinterpret_cast<uintptr_t>(x) % 16)
    return aero_host::set_error(AERO_EINVAL, "workspace must be 256-byte and x 16-byte aligned");
  int nsm = 0;
  const int rc = prepare(&nsm);
  if (rc) return rc;
  auto s = static_cast<cudaStream_t>(stream);
  auto *ws = static_cast<unsigned char *>(workspace);
  const size_t b = (size_t)batch;
  auto *z = reinterpret_cast<__nv_bfloat16 *>(ws);
  auto *dy = reinterpret_cast<__nv_bfloat16 *>(ws + aero_host::align_up(3 * b * NH * 2));
  auto *dza = reinterpret_cast<__nv_bfloat16 *>(ws + aero_host::align_up(3 * b * NH * 2) + aero_host::align_up(b * KOUT * 2));
  auto *dzb = dza + aero_host::align_up(b * NH * 2) / 2;
  const auto *pb = static_cast<const __nv_bfloat16 *>(params_bf16);
  const int tiles = batch / ROWS, grid = std::min(tiles, nsm);   // the backward kernels hold 512 TMEM columns
  TrainFwdParams F{};
  F.W = weights_of(params, params_bf16);
  F.x = static_cast<const __nv_bfloat16 *>(x);
  F.t = t;
  F.idx = idx;
  F.batch = batch;
  F.z = z;
  F.dy = dy;
  F.loss = loss;
  F.status = reinterpret_cast<int *>(status);
  AERO_CUDA_TRY(aero::launch_k(mlp_train_forward_kernel, std::min(tiles, 2 * nsm), NTHREADS, FWD_SMEM, s, F));
  const size_t zs = b * NH;
  struct L {
    int layer;
    int64_t w_off, b_off;
    int n_out, k_in;
    const __nv_bfloat16 *dz, *zin;
    __nv_bfloat16 *dz_prev;
  } layers[4] = {{4, OFF_W4, OFF_B4, NOUT, NH, dy, z + 2 * zs, dza},
                 {3, OFF_W3, OFF_B3, NH, NH, dza, z + zs, dzb},
                 {2, OFF_W2, OFF_B2, NH, NH, dzb, z, dza},
                 {1, OFF_W1, OFF_B1, NH, NIN, dza, nullptr, nullptr}};
  for (const L &l : layers) {
    TrainBwdParams B{};
    B.layer = l.layer;
    B.batch = batch;
    B.w = pb + l.w_off;
    B.n_out = l.n_out;
    B.k_in = l.k_in;
    B.dz = l.dz;
    B.zin = l.zin;
    B.x = static_cast<const __nv_bfloat16 *>(x);
    B.idx = idx;
    B.dz_prev = l.dz_prev;
    B.gw = grad + l.w_off;
    B.gb = grad + l.b_off;
    B.status = reinterpret_cast<int *>(status);
    AERO_CUDA_TRY(aero::launch_k(mlp_train_backward_kernel, grid, NTHREADS, BWD_SMEM, s, B));
  }
  return AERO_OK;
}

int aero_mlp_train_step(float *params, void *params_bf16, float *adam_m, float *adam_v, float *grad, const void *x,
                        const float *t, const int32_t *idx, int32_t batch, int32_t step, float lr, double *loss,
                        void *workspace, int32_t *status, void *stream) {
  if (!adam_m || !adam_v) return aero_host::set_error(AERO_EINVAL, "null argument");
  if (step < 1 || !(lr > 0.f)) return aero_host::set_error(AERO_EINVAL, "step must be >= 1 and lr positive");
  const int rc = aero_mlp_gradients(params, params_bf16, grad, x, t, idx, batch, loss, workspace, status, stream);
  if (rc) return rc;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  AERO_CUDA_TRY(aero::launch_k(adam_kernel, grid_for(NPARAM), 256, 0, static_cast<cudaStream_t>(stream), params,
                               adam_m, adam_v, grad, static_cast<__nv_bfloat16 *>(params_bf16), (int64_t)NPARAM, lr, b1,
                               b2, 1e-8f, c1, c2));
  return AERO_OK;
}

int aero_closure_eddy_viscosity(const AeroClosureModel *m, const float *grad9, int64_t n, double delta, float *nu,
                                unsigned long long *nut_max, uint64_t *counts, int32_t *status, void *stream) {
  if (!m || !m->params || !m->params_bf16 || !grad9 || !nu || !status)
    return aero_host::set_error(AERO_EINVAL, "null argument");
  if (n <= 0) return AERO_OK;
  if (n > INT32_MAX) return aero_host::set_error(AERO_EINVAL, "too many cells for one call");
  return aero_host::closure_nu(m, grad9, n, (int)n, 1, 1, (int)n, delta, nu, nut_max,
                               reinterpret_cast<unsigned long long *>(counts),
                               reinterpret_cast<int *>(status), static_cast<cudaStream_t>(stream));
}

}  // extern "C"
