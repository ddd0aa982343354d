// Kernels of the learned noise-PSD model: a BF16 GEMM on the tensor cores
// (tcgen05, FP32 accumulation in TMEM) and the element-wise steps of the
// 3-layer MLP's forward pass, backward pass and Adam update.
//
// GEMM: C[m][n] = sum_k A(m,k) B(n,k) (+ C when accumulate), A and B BF16,
// C FP32 row-major, FP32 accumulation in tensor memory. Operands contiguous
// along K take the pipelined kernel (k_gemm_pipe); any other strides take a
// simple one (k_gemm_bf16: one 128 x 64 tile per CTA, K steps staged
// synchronously into the canonical K-major shared-memory layout). Sizes must
// be multiples of the tile (M % 128, N % 64, K % 64): callers pad.
#include <cstdint>
#include <cmath>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fft3d_mlp.h"
#include "fft3d_attr.h"

namespace {

constexpr int GM = 128, GN = 64, GK = 64, GT = 128;
constexpr uint32_t kCols = 64;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t kmaj(int r, int k, int R) { return (uint32_t)(((k >> 3) * R + r) * 16 + (k & 7) * 2); }
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done = 0;
  for (int it = 0; it < (1 << 22) && !done; it++) {
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  }
  return done != 0;
}

// stage a rows x 64 tile of op(r, k) = P[r * sr + k * sk] into K-major smem
__device__ __forceinline__ void stage_tile(uint8_t* dst, int R, const __nv_bfloat16* P, long long sr, long long sk,
                                           int r0, int k0, int tid) {
  if (sk == 1) {  // K contiguous: 16-byte loads of 8 K values
    for (int i = tid; i < R * (GK / 8); i += GT) {
      const int r = i / (GK / 8), kc = i - r * (GK / 8);
      const uint4 v = *reinterpret_cast<const uint4*>(P + (long long)(r0 + r) * sr + (k0 + kc * 8));
      *reinterpret_cast<uint4*>(dst + kmaj(r, kc * 8, R)) = v;
    }
  } else {  // rows contiguous (transposed operand): coalesced along r
    for (int i = tid; i < R * GK; i += GT) {
      const int k = i / R, r = i - k * R;
      const __nv_bfloat16 v = P[(long long)(r0 + r) * sr + (long long)(k0 + k) * sk];
      *reinterpret_cast<__nv_bfloat16*>(dst + kmaj(r, k, R)) = v;
    }
  }
}

__global__ void __launch_bounds__(GT) k_gemm_bf16(const __nv_bfloat16* A, long long sam, long long sak,
                                                  const __nv_bfloat16* B, long long sbn, long long sbk, float* C,
                                                  long long ldc, int K, int accumulate, int* err) {
  __shared__ __align__(1024) uint8_t sA[GM * GK * 2];
  __shared__ __align__(1024) uint8_t sB[GN * GK * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tslot;
  uint32_t phase = 0;
  bool ok = true;
  for (int k0 = 0; k0 < K && ok; k0 += GK) {
    stage_tile(sA, GM, A, sam, sak, m0, k0, tid);
    stage_tile(sB, GN, B, sbn, sbk, n0, k0, tid);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t idesc = idesc_bf16(GM, GN);
      for (int ks = 0; ks < GK / 16; ks++) {
        const uint64_t da = sdesc(smem_u32(sA) + ks * 2 * GM * 16, GM * 16, 128);
        const uint64_t db = sdesc(smem_u32(sB) + ks * 2 * GN * 16, GN * 16, 128);
        const uint32_t acc = (k0 > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar))
                   : "memory");
    }
    // smem is reused by the next step only after the MMAs have read it; the
    // verdict of the bounded wait is made uniform so that no thread is left
    // behind at a barrier
    if (__syncthreads_or(mbar_wait(&bar, phase) ? 0 : 1)) {
      ok = false;
      if (tid == 0) atomicOr(err, 1);
    }
    phase ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (ok) {
    const int m = m0 + warp * 32 + lane;
    float* crow = C + (long long)m * ldc + n0;
    for (int half = 0; half < GN / 32; half++) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + half * 32;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; j += 4) {
        float4 v = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                               __uint_as_float(r[j + 3]));
        float4* dst = reinterpret_cast<float4*>(crow + half * 32 + j);
        if (accumulate) {
          const float4 o = *dst;
          v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
        }
        *dst = v;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// ---------------------------------------------------------------- pipelined GEMM (K-major operands)
// C[m][n] (=|+=) sum_k A[m*lda + k] B[n*ldb + k], both operands contiguous
// along K. 128 x BN tile per CTA (BN = 128, or 64 when N is not a multiple of
// 128), K steps of 64 in a 3-stage shared-memory ring filled with 16-byte
// cp.async copies: the MMAs of step k run while steps k+1 and k+2 load. The
// K-major no-swizzle layout is padded by 16 bytes per 8-element K chunk, so
// that the 8 threads filling one 128-byte row segment hit 8 different banks.
// Each stage's MMAs commit to that stage's mbarrier; a slot is refilled only
// after its barrier completes (bounded waits; timeout -> err bit 0).

constexpr int PM = 128, PK = 64, PS = 3;

template <int BN>
struct PipeCfg {
  static constexpr uint32_t LBO_A = (PM / 8) * 128 + 16;
  static constexpr uint32_t LBO_B = (BN / 8) * 128 + 16;
  static constexpr uint32_t SZ_A = 8 * LBO_A, SZ_B = 8 * LBO_B;
  static constexpr uint32_t STAGE = SZ_A + SZ_B;
  static constexpr uint32_t SMEM = PS * STAGE + 64;  // + mbarriers and the TMEM address slot
};

__device__ __forceinline__ void cp16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_pipe(const __nv_bfloat16* __restrict__ A, long long lda,
                                                   const __nv_bfloat16* __restrict__ B, long long ldb, float* C,
                                                   long long ldc, int K, int accumulate, int* err) {
  using Cf = PipeCfg<BN>;
  extern __shared__ __align__(1024) uint8_t sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + PS * Cf::STAGE);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + PS);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * PM, n0 = blockIdx.x * BN;
  const uint32_t sbase = smem_u32(sm);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < PS; st++) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + st)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const int nk = K / PK;
  auto load = [&](int slot, int kt) {
    const uint32_t a = sbase + slot * Cf::STAGE, b = a + Cf::SZ_A;
    const int k0 = kt * PK;
#pragma unroll
    for (int j = 0; j < PM * 8 / 128; j++) {
      const int idx = tid + 128 * j, r = idx >> 3, c = idx & 7;
      cp16(a + c * Cf::LBO_A + (r >> 3) * 128 + (r & 7) * 16, A + (long long)(m0 + r) * lda + k0 + c * 8);
    }
#pragma unroll
    for (int j = 0; j < BN * 8 / 128; j++) {
      const int idx = tid + 128 * j, r = idx >> 3, c = idx & 7;
      cp16(b + c * Cf::LBO_B + (r >> 3) * 128 + (r & 7) * 16, B + (long long)(n0 + r) * ldb + k0 + c * 8);
    }
  };
  bool ok = true;
  for (int st = 0; st < PS - 1; st++) {
    if (st < nk) load(st, st);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int kt = 0; kt < nk; kt++) {
    const int slot = kt % PS;
    asm volatile("cp.async.wait_group %0;" ::"n"(PS - 2) : "memory");  // step kt has landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a = sbase + slot * Cf::STAGE, b = a + Cf::SZ_A;
      const uint32_t idesc = idesc_bf16(PM, BN);
#pragma unroll
      for (int ks = 0; ks < PK / 16; ks++) {
        const uint64_t da = sdesc(a + ks * 2 * Cf::LBO_A, Cf::LBO_A, 128);
        const uint64_t db = sdesc(b + ks * 2 * Cf::LBO_B, Cf::LBO_B, 128);
        const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(bars + slot))
                   : "memory");
    }
    const int nxt = kt + PS - 1;
    if (nxt < nk) {
      // slot nxt % PS held step kt - 1: refill it once that step's MMAs are done
      if (kt >= 1 && !mbar_wait(bars + (kt - 1) % PS, (uint32_t)(((kt - 1) / PS) & 1))) ok = false;
      if (ok) load(nxt % PS, nxt);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  if (nk > 0 && !mbar_wait(bars + (nk - 1) % PS, (uint32_t)(((nk - 1) / PS) & 1))) ok = false;
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  const bool failed = __syncthreads_or(ok ? 0 : 1);
  if (failed && tid == 0) atomicOr(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed) {
    float* crow = C + (long long)(m0 + warp * 32 + lane) * ldc + n0;
    for (int half = 0; half < BN / 32; half++) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + half * 32;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; j += 4) {
        float4 v = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                               __uint_as_float(r[j + 3]));
        float4* dst = reinterpret_cast<float4*>(crow + half * 32 + j);
        if (accumulate) {
          const float4 o = *dst;
          v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
        }
        *dst = v;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
}

// dst[c][r] = src[r][c] (BF16), 32 x 32 tiles through shared memory
__global__ void __launch_bounds__(256) k_transpose_bf16(const __nv_bfloat16* __restrict__ src, __nv_bfloat16* dst,
                                                        int rows, int cols) {
  __shared__ __nv_bfloat16 t[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[i][threadIdx.x] = src[(long long)r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) dst[(long long)c * rows + r] = t[threadIdx.x][i];
  }
}

// ---------------------------------------------------------------- element-wise

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// Z = C + bias; store Z (pre-activation, FP32) and act(Z) as BF16
__global__ void k_bias_act(const float* C, const float* bias, float* Z, __nv_bfloat16* H, long long rows, int cols,
                           int act) {
  const long long n = rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float z = C[i] + bias[i % cols];
    if (Z) Z[i] = z;
    if (H) H[i] = __float2bfloat16_rn(act ? gelu(z) : z);
  }
}

// dZ = dH * gelu'(Z) (BF16 copy for the next GEMMs, FP32 for the bias gradient)
__global__ void k_gelu_back(const float* dH, const float* Z, float* dZ, __nv_bfloat16* dZb, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = dH[i] * gelu_grad(Z[i]);
    dZ[i] = d;
    dZb[i] = __float2bfloat16_rn(d);
  }
}

// mean squared error over the first `valid` columns; dY = 2 (Y - T) / count
__global__ void k_mse_grad(const float* Y, int ldy, const float* T, int ldt, float* dY, __nv_bfloat16* dYb,
                           long long rows, int valid, float* loss) {
  const long long n = rows * ldy;
  const float scale = 2.f / (float)(rows * valid);
  float acc = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / ldy;
    const int c = (int)(i - r * ldy);
    const float d = c < valid ? Y[i] - T[r * ldt + c] : 0.f;
    acc += d * d;
    dY[i] = scale * d;
    dYb[i] = __float2bfloat16_rn(scale * d);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc / (float)(rows * valid));
}

// column sums in two fixed-order stages: partial[chunk][c] over 64 rows, then over the chunks
constexpr int kSumRows = 64;
__global__ void k_colsum_partial(const float* X, float* partial, long long rows, int cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const long long r0 = (long long)blockIdx.y * kSumRows;
  const long long r1 = r0 + kSumRows < rows ? r0 + kSumRows : rows;
  float s = 0.f;
  for (long long r = r0; r < r1; r++) s += X[r * cols + c];
  partial[(long long)blockIdx.y * cols + c] = s;
}
__global__ void k_colsum_final(const float* partial, float* out, int chunks, int cols, float scale) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int k = 0; k < chunks; k++) s += partial[(long long)k * cols + c];
  out[c] = s * scale;
}

__global__ void k_to_bf16(const float* x, __nv_bfloat16* y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// Adam on FP32 master weights, refreshing the BF16 copy
__global__ void k_adam(float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

int grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 148 * 16 ? g : 148 * 16);
}

}  // namespace

namespace fft3d {
namespace mlp {

template <int BN>
cudaError_t launch_pipe(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* B, long long ldb, float* C,
                        long long ldc, int M, int N, int K, bool accumulate, int* err, cudaStream_t s) {
  constexpr int smem = PipeCfg<BN>::SMEM;
  cudaError_t e = fft3d::smem_attr(k_gemm_pipe<BN>, smem, true);
  if (e != cudaSuccess) return e;
  k_gemm_pipe<BN><<<dim3(N / BN, M / PM), 128, smem, s>>>(A, lda, B, ldb, C, ldc, K, accumulate ? 1 : 0, err);
  return cudaGetLastError();
}

cudaError_t gemm_bf16(const void* A, long long sam, long long sak, const void* B, long long sbn, long long sbk,
                      float* C, long long ldc, int M, int N, int K, bool accumulate, int* err, cudaStream_t s) {
  if (!gemm_shape_ok(M, N, K)) return cudaErrorInvalidValue;
  const bool kmajor = sak == 1 && sbk == 1 && sam % 8 == 0 && sbn % 8 == 0 &&
                      (((uintptr_t)A | (uintptr_t)B) & 15) == 0;
  if (kmajor) {
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    return N % 128 == 0 ? launch_pipe<128>(a, sam, b, sbn, C, ldc, M, N, K, accumulate, err, s)
                        : launch_pipe<64>(a, sam, b, sbn, C, ldc, M, N, K, accumulate, err, s);
  }
  dim3 grid(N / GN, M / GM);
  k_gemm_bf16<<<grid, GT, 0, s>>>(static_cast<const __nv_bfloat16*>(A), sam, sak,
                                  static_cast<const __nv_bfloat16*>(B), sbn, sbk, C, ldc, K, accumulate ? 1 : 0, err);
  return cudaGetLastError();
}

cudaError_t bias_act(const float* C, const float* bias, float* Z, void* H, long long rows, int cols, bool gelu_on,
                     cudaStream_t s) {
  k_bias_act<<<grid_for(rows * cols), 256, 0, s>>>(C, bias, Z, static_cast<__nv_bfloat16*>(H), rows, cols,
                                                   gelu_on ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t gelu_back(const float* dH, const float* Z, float* dZ, void* dZb, long long n, cudaStream_t s) {
  k_gelu_back<<<grid_for(n), 256, 0, s>>>(dH, Z, dZ, static_cast<__nv_bfloat16*>(dZb), n);
  return cudaGetLastError();
}

cudaError_t mse_grad(const float* Y, int ldy, const float* T, int ldt, float* dY, void* dYb, long long rows, int valid,
                     float* loss, cudaStream_t s) {
  k_mse_grad<<<grid_for(rows * ldy), 256, 0, s>>>(Y, ldy, T, ldt, dY, static_cast<__nv_bfloat16*>(dYb), rows, valid,
                                                  loss);
  return cudaGetLastError();
}

long long colsum_partial_floats(long long rows, int cols) { return (rows + kSumRows - 1) / kSumRows * cols; }

cudaError_t colsum(const float* X, float* partial, float* out, long long rows, int cols, float scale, cudaStream_t s) {
  const int chunks = (int)((rows + kSumRows - 1) / kSumRows);
  k_colsum_partial<<<dim3((cols + 127) / 128, chunks), 128, 0, s>>>(X, partial, rows, cols);
  k_colsum_final<<<(cols + 127) / 128, 128, 0, s>>>(partial, out, chunks, cols, scale);
  return cudaGetLastError();
}

cudaError_t adam(float* w, const float* g, float* m, float* v, void* wb, long long n, float lr, float b1, float b2,
                 float eps, int step, cudaStream_t s) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, s>>>(w, g, m, v, static_cast<__nv_bfloat16*>(wb), n, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t transpose_bf16(const void* src, void* dst, int rows, int cols, cudaStream_t s) {
  k_transpose_bf16<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, s>>>(
      static_cast<const __nv_bfloat16*>(src), static_cast<__nv_bfloat16*>(dst), rows, cols);
  return cudaGetLastError();
}

cudaError_t to_bf16(const float* x, void* y, long long n, cudaStream_t s) {
  k_to_bf16<<<grid_for(n), 256, 0, s>>>(x, static_cast<__nv_bfloat16*>(y), n);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace fft3d
