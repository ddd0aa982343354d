// Tensor-core (tcgen05) forward block transform: the r2c 2D DFT of the
// windowed 32x32 blocks as two dense GEMMs with split-precision BF16 operands
// and FP32 accumulation in TMEM (the "K2'" DFT-GEMM of the design).
//
// For a tile of 8 blocks (one persistent CTA of 4 warps at a time):
//  stage 1 (rows):    Z[b,y][n] = sum_x V[b,y][x] G[n][x]
//                     V = raw sample - plane base (exact in BF16 for 8-bit),
//                     G = r2c DFT along x with the analysis window folded in
//                     (rows n: Re of bins 0..16, Im of bins 1..15), G = Gh + Gl:
//                     two MMAs per K step (three when V is not exact);
//  stage 2 (columns): Y[b,c][h] = sum_y F[h][y] Zc[y], F = DFT along y with the
//                     y window folded in, as a real 64x64 matrix on interleaved
//                     (re, im); Zc = column c of Z, with the real DC and Nyquist
//                     columns packed into one complex column (c = 0), so 8
//                     blocks x 16 columns fill M = 128; three MMAs per K step
//                     (Zh Fh + Zh Fl + Zl Fh).
// Operands live in shared memory in the canonical K-major layout without
// swizzle (8-row x 16-byte core matrices); the DFT tables are copied once per
// CTA from a global image in that same layout. Waits on the MMA completion
// barrier are bounded: on timeout the kernel records an error and skips the
// tile, and TMEM is always freed before the CTA exits.
#include <cmath>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fft3d_kernels.cuh"
#include "fft3d_attr.h"

namespace fft3d {

namespace {

constexpr int TB = 32;          // block size (bw = bh = 32)
constexpr int TILE = 8;         // blocks per tile
constexpr int ROWS = TILE * TB; // 256 rows of stage 1 (two M=128 sub-tiles)
constexpr int NH = TB / 2 + 1;  // 17 complex bins per row
constexpr int THREADS = 128;
constexpr uint32_t kTmemCols = 128;  // stage 1: 2 x 32 columns, stage 2: 64 columns

// byte offset of element (r, k) in an R x K K-major operand (core matrices of
// 8 rows x 8 bf16, chunk k/8 stored as R rows of 16 bytes)
__device__ __forceinline__ uint32_t kmaj(int r, int k, int R) { return (uint32_t)(((k >> 3) * R + r) * 16 + (k & 7) * 2); }

// Stage-2 operand layout: K chunks of the same 8-row group 144 bytes apart
// (LBO, one 16-byte pad per chunk) and 8-row groups 8 x 144 bytes apart (SBO),
// so that the 32 lanes storing one row's 64 K values hit 32 different banks.
constexpr int A2_LBO = 144, A2_SBO = 8 * 144;
__device__ __forceinline__ uint32_t kmaj2(int r, int k) {
  return (uint32_t)((k >> 3) * A2_LBO + (r >> 3) * A2_SBO + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// idesc of kind::f16 with BF16 A/B, FP32 D, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// bounded wait on mbarrier phase `parity`; false on timeout
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

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
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
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// x = hi + lo in BF16 (hi = round-to-nearest of x, lo = round of the rest)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

__device__ __forceinline__ int reflect101_tc(int s, int n) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (s < 0) s = -s;
    if (s >= n) s = 2 * (n - 1) - s;
  }
  return s;
}

template <typename T>
__device__ __forceinline__ float ld_sample(const T* p) { return (float)__ldg(p); }
template <>
__device__ __forceinline__ float ld_sample<uint8_t>(const uint8_t* p) { return (float)(int)__ldg(p); }
template <>
__device__ __forceinline__ float ld_sample<uint16_t>(const uint16_t* p) { return (float)(int)__ldg(p); }

// shared memory plan (bytes)
constexpr uint32_t SZ_B1 = 32 * 32 * 2;     // G hi / lo: N=32 x K=32
constexpr uint32_t SZ_B2 = 64 * 64 * 2;     // F hi / lo: N=64 x K=64
constexpr uint32_t SZ_A1 = 128 * 32 * 2;    // one M=128 sub-tile of V (hi or lo)
constexpr uint32_t SZ_A2 = 16 * A2_SBO;     // Z columns (hi or lo): 16 groups of 8 rows
constexpr uint32_t OFF_B1H = 0, OFF_B1L = OFF_B1H + SZ_B1, OFF_B2H = OFF_B1L + SZ_B1, OFF_B2L = OFF_B2H + SZ_B2;
constexpr uint32_t OFF_A2H = OFF_B2L + SZ_B2, OFF_A2L = OFF_A2H + SZ_A2;
constexpr uint32_t OFF_BAR = OFF_A2L + SZ_A2;
constexpr uint32_t OFF_A1H = OFF_BAR + 64;                 // 2 sub-tiles
constexpr uint32_t OFF_A1L = OFF_A1H + 2 * SZ_A1;          // 2 sub-tiles, only when V is split
constexpr uint32_t SMEM_TC = OFF_A1H + 2 * SZ_A1;          // V exact (8-bit samples)
constexpr uint32_t SMEM_TC_SPLIT = OFF_A1L + 2 * SZ_A1;    // V split (9..16-bit, float)
constexpr uint32_t TABLE_BYTES = 2 * SZ_B1 + 2 * SZ_B2;    // global image of B1h, B1l, B2h, B2l

template <typename T, bool VSPLIT>
__global__ void __launch_bounds__(THREADS) k_forward_tc(ForwardArgs a, FwdFrameSet fs, const uint8_t* __restrict__ tables,
                                                        int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + OFF_BAR + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Geom& g = a.g;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // DFT tables (already in operand layout)
  {
    const uint4* src = reinterpret_cast<const uint4*>(tables);
    uint4* dst = reinterpret_cast<uint4*>(sm + OFF_B1H);
    for (int i = tid; i < (int)(TABLE_BYTES / 16); i += THREADS) dst[i] = __ldg(src + i);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t d1 = tmem;       // stage 1: sub-tile s at columns 32 s
  const uint32_t d2 = tmem + 64;  // stage 2: 64 columns
  const uint32_t sbase = smem_u32(sm);
  // work item t: tile t % ntiles of frame t / ntiles (fs: the frames' samples
  // and ring slots)
  const int ntiles = (g.nblocks + TILE - 1) / TILE;
  const int total = ntiles * fs.count;
  auto frame_of = [&](int t, const void** src, long long* stride, float2** spec) {
    const int j = t / ntiles;
#pragma unroll
    for (int q = 0; q < kMaxFwdFrames; q++)
      if (q == j) {
        *src = fs.src[q];
        *stride = fs.stride[q];
        *spec = fs.spec[q];
      }
  };
  // Rows of a tile: thread tid holds rows tid and tid + 128 of the tile's 256
  // (8 blocks x 32 rows). Interior aligned rows of 8- and 16-bit samples are
  // fetched as raw 16-byte vectors one tile ahead, so their load latency
  // overlaps the previous tile's MMAs.
  constexpr int RPT = ROWS / THREADS;
  constexpr int NV = sizeof(T) <= 2 ? TB * (int)sizeof(T) / 16 : 0;
  uint4 raw[RPT][NV > 0 ? NV : 1];
  bool have[RPT];
  auto row_src = [&](const void* src, long long stride, int blk, int y, int* x0) {
    const int by = blk / g.nox, bx = blk - by * g.nox;
    const int kr = reflect101_tc(by * g.sy + y - g.sy, g.H);
    const int row = g.interlaced ? (kr < (g.H >> 1) ? 2 * kr : g.H - 1 - 2 * (kr - (g.H >> 1))) : kr;
    *x0 = bx * g.sx - g.sx;
    return reinterpret_cast<const T*>(static_cast<const char*>(src) + (long long)row * stride);
  };
  auto prefetch = [&](int t) {
#pragma unroll
    for (int i = 0; i < RPT; i++) have[i] = false;
    if constexpr (NV > 0) {
      if (t >= total) return;
      const void* src;
      long long stride;
      float2* spec;
      frame_of(t, &src, &stride, &spec);
      const int blk0 = (t % ntiles) * TILE;
#pragma unroll
      for (int i = 0; i < RPT; i++) {
        const int r = tid + THREADS * i, b = r / TB, y = r - b * TB, blk = blk0 + b;
        if (blk < g.nblocks) {
          int x0;
          const T* p = row_src(src, stride, blk, y, &x0) + x0;
          if (x0 >= 0 && x0 + TB <= g.W && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
            for (int v = 0; v < NV; v++) raw[i][v] = __ldg(reinterpret_cast<const uint4*>(p) + v);
            have[i] = true;
          }
        }
      }
    }
  };
  uint32_t phase = 0;
  bool ok = true;
  prefetch(blockIdx.x);
  for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
    const void* fsrc;
    long long fstride;
    float2* fspec;
    frame_of(t, &fsrc, &fstride, &fspec);
    const int blk0 = (t % ntiles) * TILE;
    // ---- stage 1 operand: rows of V (two rows per thread)
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = tid + THREADS * i;
      const int b = r / TB, y = r - b * TB, blk = blk0 + b;
      const int sub = r >> 7, m = r & 127;
      uint8_t* ah = sm + OFF_A1H + sub * SZ_A1;
      uint8_t* al = sm + OFF_A1L + sub * SZ_A1;
      float v[TB];
      if (blk < g.nblocks) {
        int x0;
        const T* srow = row_src(fsrc, fstride, blk, y, &x0);
        if (NV > 0 && have[i]) {
          constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
          for (int c = 0; c < (NV > 0 ? NV : 1); c++) {
            const uint32_t w[4] = {raw[i][c].x, raw[i][c].y, raw[i][c].z, raw[i][c].w};
#pragma unroll
            for (int j = 0; j < PER; j++) {
              float f;
              if constexpr (sizeof(T) == 1) f = (float)((w[j >> 2] >> (8 * (j & 3))) & 0xffu);
              else f = (float)((w[j >> 1] >> (16 * (j & 1))) & 0xffffu);
              v[c * PER + j] = f - a.base;
            }
          }
        } else if (x0 >= 0 && x0 + TB <= g.W) {
#pragma unroll
          for (int x = 0; x < TB; x++) v[x] = ld_sample<T>(srow + x0 + x) - a.base;
        } else {
#pragma unroll
          for (int x = 0; x < TB; x++) v[x] = ld_sample<T>(srow + reflect101_tc(x0 + x, g.W)) - a.base;
        }
      } else {
#pragma unroll
        for (int x = 0; x < TB; x++) v[x] = 0.f;
      }
#pragma unroll
      for (int x = 0; x < TB; x += 2) {
        __nv_bfloat16 h0, l0, h1, l1;
        split_bf16(v[x], h0, l0);
        split_bf16(v[x + 1], h1, l1);
        *reinterpret_cast<__nv_bfloat162*>(ah + kmaj(m, x, 128)) = __halves2bfloat162(h0, h1);
        if (VSPLIT) *reinterpret_cast<__nv_bfloat162*>(al + kmaj(m, x, 128)) = __halves2bfloat162(l0, l1);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      constexpr uint32_t id1 = idesc_bf16(128, 32);
      for (int sub = 0; sub < 2; sub++) {
        const uint32_t ah = sbase + OFF_A1H + sub * SZ_A1, al = sbase + OFF_A1L + sub * SZ_A1;
        for (int ks = 0; ks < 2; ks++) {  // K = 32: two steps of 16
          const uint64_t dah = sdesc(ah + ks * 2 * 128 * 16, 128 * 16, 128);
          const uint64_t dal = sdesc(al + ks * 2 * 128 * 16, 128 * 16, 128);
          const uint64_t dbh = sdesc(sbase + OFF_B1H + ks * 2 * 32 * 16, 32 * 16, 128);
          const uint64_t dbl = sdesc(sbase + OFF_B1L + ks * 2 * 32 * 16, 32 * 16, 128);
          const uint32_t dd = d1 + sub * 32;
          mma_bf16(dd, dah, dbh, id1, ks > 0 ? 1u : 0u);
          mma_bf16(dd, dah, dbl, id1, 1u);
          if (VSPLIT) mma_bf16(dd, dal, dbh, id1, 1u);
        }
      }
      mma_commit(bar);
    }
    prefetch(t + gridDim.x);  // the next tile's rows load while this tile's MMAs run
    if (__syncthreads_or(mbar_wait(bar, phase) ? 0 : 1)) {  // uniform verdict: no thread left at a barrier
      ok = false;
      if (tid == 0) atomicOr(err, 1);
      break;
    }
    phase ^= 1;
    tc_fence_after();
    // ---- stage 2 operand: columns of Z, split hi / lo
    for (int sub = 0; sub < 2; sub++) {
      float z[32];
      tmem_ld32(d1 + ((uint32_t)(warp * 32) << 16) + sub * 32, z);  // row r = sub*128 + 32 warp + lane
      const int r = sub * 128 + warp * 32 + lane;
      const int b = r / TB, y = r - b * TB;
      // z[0..16] = Re bins 0..16, z[17..31] = Im bins 1..15
#pragma unroll
      for (int c = 0; c < 16; c++) {
        const float re = c == 0 ? z[0] : z[c];
        const float im = c == 0 ? z[16] : z[16 + c];
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16(re, rh, rl);
        split_bf16(im, ih, il);
        const int m2 = b * 16 + c;
        *reinterpret_cast<__nv_bfloat162*>(sm + OFF_A2H + kmaj2(m2, 2 * y)) = __halves2bfloat162(rh, ih);
        *reinterpret_cast<__nv_bfloat162*>(sm + OFF_A2L + kmaj2(m2, 2 * y)) = __halves2bfloat162(rl, il);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      constexpr uint32_t id2 = idesc_bf16(128, 64);
      for (int ks = 0; ks < 4; ks++) {  // K = 64
        const uint64_t dah = sdesc(sbase + OFF_A2H + ks * 2 * A2_LBO, A2_LBO, A2_SBO);
        const uint64_t dal = sdesc(sbase + OFF_A2L + ks * 2 * A2_LBO, A2_LBO, A2_SBO);
        const uint64_t dbh = sdesc(sbase + OFF_B2H + ks * 2 * 64 * 16, 64 * 16, 128);
        const uint64_t dbl = sdesc(sbase + OFF_B2L + ks * 2 * 64 * 16, 64 * 16, 128);
        mma_bf16(d2, dah, dbh, id2, ks > 0 ? 1u : 0u);
        mma_bf16(d2, dah, dbl, id2, 1u);
        mma_bf16(d2, dal, dbh, id2, 1u);
      }
      mma_commit(bar);
    }
    if (__syncthreads_or(mbar_wait(bar, phase) ? 0 : 1)) {  // uniform verdict: no thread left at a barrier
      ok = false;
      if (tid == 0) atomicOr(err, 1);
      break;
    }
    phase ^= 1;
    tc_fence_after();
    // ---- outputs: row m2 = (block, column) holds Y[h] (re, im) interleaved;
    // staged in shared memory (the stage-2 operands are free now) as the
    // tile's contiguous spectra, then written with 16-byte stores
    float2* stage = reinterpret_cast<float2*>(sm + OFF_A2H);
    {
      float y0[32], y1[32];
      tmem_ld32(d2 + ((uint32_t)(warp * 32) << 16), y0);       // h = 0..15
      tmem_ld32(d2 + ((uint32_t)(warp * 32) << 16) + 32, y1);  // h = 16..31
      const int m2 = warp * 32 + lane, b = m2 >> 4, c = m2 & 15;
      float2* out = stage + b * TB * NH;
      auto Y = [&](int h) { return h < 16 ? make_float2(y0[2 * h], y0[2 * h + 1]) : make_float2(y1[2 * h - 32], y1[2 * h - 31]); };
      if (c == 0) {
        // unpack the DC (col 0) and Nyquist (col 16) transforms:
        // A[h] = (Y[h] + conj Y[-h]) / 2, B[h] = (Y[h] - conj Y[-h]) / (2i)
#pragma unroll
        for (int h = 0; h < TB; h++) {
          const float2 yh = Y(h), ym = Y((TB - h) & (TB - 1));
          out[h * NH] = make_float2(0.5f * (yh.x + ym.x), 0.5f * (yh.y - ym.y));
          out[h * NH + 16] = make_float2(0.5f * (yh.y + ym.y), -0.5f * (yh.x - ym.x));
        }
      } else {
#pragma unroll
        for (int h = 0; h < TB; h++) out[h * NH + c] = Y(h);
      }
    }
    __syncthreads();
    {
      const int nvalid = min(TILE, g.nblocks - blk0);
      const uint4* src = reinterpret_cast<const uint4*>(stage);
      uint4* dst = reinterpret_cast<uint4*>(fspec + (size_t)blk0 * TB * NH);
      for (int i = tid; i < nvalid * TB * NH / 2; i += THREADS) dst[i] = src[i];
    }
    tc_fence_before();
    __syncthreads();  // TMEM and smem operands are reused by the next tile
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

uint32_t forward_tc_table_bytes() { return TABLE_BYTES; }
uint32_t forward_tc_smem_bytes() { return SMEM_TC_SPLIT; }

// DFT tables of the tensor-core forward transform for a 32x32 block with
// analysis windows wx, wy, in the global image layout the kernel copies to
// shared memory: G hi, G lo (32 x 32), F hi, F lo (64 x 64), each K-major.
void forward_tc_tables(const float* wx, const float* wy, uint8_t* out) {
  const double PI = 3.14159265358979323846;
  auto put = [](uint8_t* base, int r, int k, int R, double v, bool hi) {
    __nv_bfloat16 h = __float2bfloat16_rn((float)v);
    __nv_bfloat16 val = hi ? h : __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
    *reinterpret_cast<__nv_bfloat16*>(base + ((k >> 3) * R + r) * 16 + (k & 7) * 2) = val;
  };
  uint8_t* g_hi = out;
  uint8_t* g_lo = out + SZ_B1;
  uint8_t* f_hi = out + 2 * SZ_B1;
  uint8_t* f_lo = f_hi + SZ_B2;
  for (int n = 0; n < 32; n++)
    for (int x = 0; x < 32; x++) {
      // rows 0..16: Re of bin n; rows 17..31: Im of bin n-16 (forward sign)
      const int k = n <= 16 ? n : n - 16;
      const double ang = 2.0 * PI * (double)((k * x) % 32) / 32.0;
      const double v = n <= 16 ? wx[x] * std::cos(ang) : -wx[x] * std::sin(ang);
      put(g_hi, n, x, 32, v, true);
      put(g_lo, n, x, 32, v, false);
    }
  for (int h = 0; h < 32; h++)
    for (int y = 0; y < 32; y++) {
      const double ang = 2.0 * PI * (double)((h * y) % 32) / 32.0;
      const double fr = wy[y] * std::cos(ang), fi = -wy[y] * std::sin(ang);
      // rows n = 2h + s (s: re / im of Y[h]); columns k = 2y + t (t: re / im of Z[y])
      const double m[2][2] = {{fr, -fi}, {fi, fr}};
      for (int s = 0; s < 2; s++)
        for (int t = 0; t < 2; t++) {
          put(f_hi, 2 * h + s, 2 * y + t, 64, m[s][t], true);
          put(f_lo, 2 * h + s, 2 * y + t, 64, m[s][t], false);
        }
    }
}

cudaError_t launch_forward_tc(const ForwardArgs& a, const void* tables, int* err, int bytes, cudaStream_t s) {
  FwdFrameSet fs{};
  fs.count = 1;
  fs.src[0] = a.src;
  fs.stride[0] = a.src_stride;
  fs.spec[0] = a.spec;
  return launch_forward_tc_frames(a, fs, tables, err, bytes, s);
}

cudaError_t launch_forward_tc_frames(const ForwardArgs& a, const FwdFrameSet& fs, const void* tables, int* err,
                                     int bytes, cudaStream_t s) {
  if (a.g.bw != TB || a.g.bh != TB || fs.count < 1 || fs.count > kMaxFwdFrames) return cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (a.g.nblocks + TILE - 1) / TILE * fs.count;
  const int per_sm = bytes == 1 ? 3 : 2;  // shared memory limits co-resident CTAs
  const int grid = ntiles < sms * per_sm ? ntiles : sms * per_sm;
  const uint8_t* t = static_cast<const uint8_t*>(tables);
  cudaError_t e = cudaSuccess;
  if (bytes == 1) {
    e = fft3d::smem_attr(k_forward_tc<uint8_t, false>, SMEM_TC, true);
    if (e == cudaSuccess) k_forward_tc<uint8_t, false><<<grid, THREADS, SMEM_TC, s>>>(a, fs, t, err);
  } else if (bytes == 2) {
    e = fft3d::smem_attr(k_forward_tc<uint16_t, true>, SMEM_TC_SPLIT, true);
    if (e == cudaSuccess) k_forward_tc<uint16_t, true><<<grid, THREADS, SMEM_TC_SPLIT, s>>>(a, fs, t, err);
  } else {
    e = fft3d::smem_attr(k_forward_tc<float, true>, SMEM_TC_SPLIT, true);
    if (e == cudaSuccess) k_forward_tc<float, true><<<grid, THREADS, SMEM_TC_SPLIT, s>>>(a, fs, t, err);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace fft3d
