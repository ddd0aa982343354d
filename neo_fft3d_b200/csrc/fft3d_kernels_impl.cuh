// Kernel templates of the FFT3D filtering core (FP32 CUDA-core path).
// Included by the per-size translation units kern_*.cu, which instantiate the
// block sizes they own and register them in the size table (kern_registry.h).
#pragma once
#include <algorithm>
#include <cmath>

#include "fft3d_kernels.cuh"
#include "kern_registry.h"
#include "regfft.cuh"
#include "fft3d_attr.h"

namespace fft3d {
namespace {

constexpr int kWarps = 4;       // warps per CTA in k_forward / k_filter_inverse

// CTAs per SM that the frame-group forward and filter/inverse kernels are
// compiled for, where their shared memory lets that many reside (register
// budget 65536 / (128 x CTAs): 80 registers at 6). Measured at 1080p bt=5
// bw=32: 6 for both is 2.5 % faster than 5 (the filter/inverse spills 88
// bytes but gains a sixth CTA).
#ifndef FFT3D_FWD_CTAS
#define FFT3D_FWD_CTAS 6
#endif
#ifndef FFT3D_GROUP_CTAS
#define FFT3D_GROUP_CTAS 6
#endif
// forward rows of a lane walked by a loop (one copy of the row code) instead
// of unrolled: fewer instruction-cache misses, the forward's largest stall
// (measured at 1080p bw=32: 22.0 vs 23.5 us per frame over all planes)
#ifndef FFT3D_FWD_ROW_LOOP
#define FFT3D_FWD_ROW_LOOP 1
#endif
// shared memory per SM, and what the runtime reserves per resident CTA
constexpr int kSmemPerSm = 228 * 1024, kSmemPerCtaReserved = 1024;
__host__ __device__ constexpr int ctas_for(int want, int smem_per_cta) {
  const int fit = kSmemPerSm / (smem_per_cta + kSmemPerCtaReserved);
  return fit < 1 ? 1 : (fit < want ? fit : want);
}

// reflect-101 of index s into [0, n): the cover's mirror margins
// (src/buffer.cpp:19-26, 65-79); repeated for planes narrower than a margin.
__device__ __forceinline__ int reflect101(int s, int n) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (s < 0) s = -s;
    if (s >= n) s = 2 * (n - 1) - s;
  }
  return s;
}

// processed-plane row k -> source row: progressive, or interlaced with field 1
// (even rows) first and field 2 bottom-up (src/buffer.cpp:31-63, 99-115)
__device__ __forceinline__ int field_row(int k, int H, int interlaced) {
  if (!interlaced) return k;
  int half = H >> 1;
  return k < half ? 2 * k : H - 1 - 2 * (k - half);
}

// The hardware's approximate reciprocal and reciprocal square root (PTX
// rcp.approx / rsqrt.approx, the instructions __fdividef and rsqrtf stand on).
// Every caller's argument is a normal float (a power spectrum plus 1e-15,
// a noise power of at least 1e-15, a ratio clamped to >= 1e-30), where the
// .ftz forms give the same result without the handling of denormal
// arguments that the plain forms carry.
__device__ __forceinline__ float rcp_nrm(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_nrm(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// n / d for 0 <= n < 2^24, d > 0 and a quotient below 2^20 (pixel and block
// coordinates over a block step or a row length), exact: the estimate
// n * (1/d) is within (n / d) * 2^-21 < 0.5 of n / d (reciprocal <= 2 ulp,
// one rounding), so truncating it and correcting by one step either way gives
// the integer quotient, in a few instructions instead of an integer division
// by a runtime value.
__device__ __forceinline__ int div_small(int n, int d) {
  int q = __float2int_rz(__int2float_rn(n) * rcp_nrm(__int2float_rn(d)));
  const int r = n - q * d;
  q += (r >= d) - (r < 0);
  return q;
}

template <typename T>
__device__ __forceinline__ float load_sample(const T* p) { return (float)p[0]; }
template <>
__device__ __forceinline__ float load_sample<uint8_t>(const uint8_t* p) { return (float)(int)__ldg(p); }
template <>
__device__ __forceinline__ float load_sample<uint16_t>(const uint16_t* p) { return (float)(int)__ldg(p); }
template <>
__device__ __forceinline__ float load_sample<float>(const float* p) { return __ldg(p); }

// Blocks per warp of the FFT kernels: enough that the bw/2 column transforms
// of all of them (DC and Nyquist columns share one complex transform) fill
// the 32 lanes (2 for bw = 32, 4 for bw = 16, 1 for bw = 48).
template <int BW>
__host__ __device__ constexpr int blocks_per_warp() {
  return (32 / (BW / 2)) < 1 ? 1 : ((32 / (BW / 2)) > 4 ? 4 : 32 / (BW / 2));
}

template <int BW, int BH>
__host__ __device__ constexpr int fft_smem_bytes() {
  return blocks_per_warp<BW>() * BH * (BW / 2 + 1) * 8;
}

// Row of BW samples starting at p, as floats; 16-byte vector loads when the
// row is aligned (the common interior case), scalar loads otherwise.
template <typename T, int BW>
__device__ __forceinline__ void load_row(const T* p, float (&r)[BW]) {
  constexpr int BYTES = BW * (int)sizeof(T);
  if constexpr (BYTES % 16 == 0) {
    if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
      const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
      for (int v = 0; v < BYTES / 16; v++) {
        const uint4 u = __ldg(q + v);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
        constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
        for (int j = 0; j < PER; j++) {
          float f;  // 8/16-bit: exact through the 2^23 mantissa trick (decode_row)
          if constexpr (sizeof(T) == 1)
            f = __uint_as_float(__byte_perm(w[j >> 2], 0x4B000000u, 0x7540u | (uint32_t)(j & 3))) - 8388608.0f;
          else if constexpr (sizeof(T) == 2)
            f = __uint_as_float(__byte_perm(w[j >> 1], 0x4B000000u, (j & 1) ? 0x7432u : 0x7410u)) - 8388608.0f;
          else f = __uint_as_float(w[j]);
          r[v * PER + j] = f;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int x = 0; x < BW; x++) r[x] = load_sample<T>(p + x);
}

// ---------------------------------------------------------------- block FFT phases
// Sb points at one block's bh x (bw/2+1) complex tile in shared memory.

// Where a forward CTA reads its frame and writes its spectra: the launch
// arguments (one frame per launch), or pointers picked for one frame of a
// frame group (k_forward_frames).
struct ArgsFwd {
  const ForwardArgs& a;
  __device__ __forceinline__ const void* src() const { return a.src; }
  __device__ __forceinline__ long long stride() const { return a.src_stride; }
  __device__ __forceinline__ float2* spec() const { return a.spec; }
};
struct FrameFwd {
  const void* s;
  long long st;
  float2* sp;
  __device__ __forceinline__ const void* src() const { return s; }
  __device__ __forceinline__ long long stride() const { return st; }
  __device__ __forceinline__ float2* spec() const { return sp; }
};

// Source row of row y of block `blk` and the source column of its column 0;
// *row: the source row index (checked against the plane in the checked build).
template <typename T, class Win>
__device__ __forceinline__ const T* fwd_row_src(const ForwardArgs& a, const Win& win, int blk, int y, int* x0,
                                                int* row = nullptr) {
  const Geom& g = a.g;
  const int by = div_small(blk, g.nox), bx = blk - by * g.nox;
  const int k = reflect101(by * g.sy + y - g.sy, g.H);
  *x0 = bx * g.sx - g.sx;
  const int r = field_row(k, g.H, g.interlaced);
  if (row) *row = r;
  return reinterpret_cast<const T*>(static_cast<const char*>(win.src()) + (long long)r * win.stride());
}

// Rows whose BW samples are whole 16-byte vectors (8- and 16-bit samples) can
// be fetched raw ahead of their transform (forward_cta's prefetch).
template <int BW, typename T>
__host__ __device__ constexpr int raw_vectors() {
  return (sizeof(T) <= 2 && (BW * (int)sizeof(T)) % 16 == 0) ? BW * (int)sizeof(T) / 16 : 0;
}

// Samples minus `base` as floats, decoded from raw 16-byte vectors. Each
// 8/16-bit sample is placed by one byte permute into the low mantissa bits of
// 2^23 (0x4B000000 + v is exactly the float 2^23 + v for v < 2^23), and one
// FADD of -(2^23 + base) leaves v - base exactly: an ALU permute and an FMA-pipe
// add per sample instead of shift/mask and an int-to-float conversion on the
// narrower conversion pipe.
template <int BW, typename T>
__device__ __forceinline__ void decode_row(const uint4* raw, float base, float (&r)[BW]) {
  constexpr int PER = 16 / (int)sizeof(T);
  const float off = 8388608.0f + base;  // exact: base <= 2^15
#pragma unroll
  for (int v = 0; v < raw_vectors<BW, T>(); v++) {
    const uint32_t w[4] = {raw[v].x, raw[v].y, raw[v].z, raw[v].w};
#pragma unroll
    for (int j = 0; j < PER; j++) {
      uint32_t m;
      if constexpr (sizeof(T) == 1) m = __byte_perm(w[j >> 2], 0x4B000000u, 0x7540u | (uint32_t)(j & 3));
      else m = __byte_perm(w[j >> 1], 0x4B000000u, (j & 1) ? 0x7432u : 0x7410u);
      r[v * PER + j] = __uint_as_float(m) - off;
    }
  }
}

// Row y of block `blk`: gather (mirrored at the plane edges), analysis window,
// r2c along x into row y of Sb. `raw`: the row's samples already fetched
// (interior aligned rows), or null.
template <int BW, int BH, typename T, bool ARGS_WX, class Win>
__device__ __forceinline__ void fwd_row(const ForwardArgs& a, const Win& win, int blk, int y, float2* Sb,
                                        const uint4* raw) {
  constexpr int NH = BW / 2 + 1;
  const Geom& g = a.g;
  int x0, srcrow;
  const T* srow = fwd_row_src<T>(a, win, blk, y, &x0, &srcrow);
  float r[BW];
  if constexpr (raw_vectors<BW, T>() > 0) {
    if (raw) decode_row<BW, T>(raw, a.base, r);  // already minus base
  }
  if (raw_vectors<BW, T>() > 0 && raw) {
  } else {
    const bool row_ok = FFT3D_IN(srcrow >= 0 && srcrow < g.H, a.err);
    if (x0 >= 0 && x0 + BW <= g.W) {
      if (row_ok) load_row<T, BW>(srow + x0, r);
    } else {
#pragma unroll
      for (int x = 0; x < BW; x++) {
        const int xi = reflect101(x0 + x, g.W);
        r[x] = (row_ok && FFT3D_IN(xi >= 0 && xi < g.W, a.err)) ? load_sample<T>(srow + xi) : 0.f;
      }
    }
#pragma unroll
    for (int x = 0; x < BW; x++) r[x] = r[x] - a.base;
  }
  const float wy = __ldg(a.wan_y + y);
  // the x window from the launch parameters (ARGS_WX) or from the table
#pragma unroll
  for (int x = 0; x < BW; x++) r[x] = r[x] * (ARGS_WX ? a.wx[x] : __ldg(a.wan_x + x)) * wy;
  float2 c[NH];
  rfft<BW>(r, c);
  float2* row = Sb + y * NH;
#pragma unroll
  for (int kk = 0; kk < NH; kk++) row[kk] = c[kk];
}

// Column c (0 < c < bw/2) forward DFT along y in place; c == 0 transforms the
// real columns 0 and bw/2 together as one complex sequence col0 + i colN.
// The lanes of a warp differ only in what they load and store: the FFT itself
// is one code path for all of them (no divergent second pass).
template <int BW, int BH>
__device__ __forceinline__ void fwd_col(float2* Sb, int c) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2;
  float2 col[BH];
  const bool dc = c == 0;
#pragma unroll
  for (int y = 0; y < BH; y++) {
    const float2 v = Sb[y * NH + c];
    col[y] = dc ? make_float2(v.x, Sb[y * NH + HC].x) : v;
  }
  cfft<BH, -1>(col);
  if (dc) {
#pragma unroll
    for (int h = 0; h < BH; h++) {
      const float2 zh = col[h], zm = cconj(col[(BH - h) % BH]);
      Sb[h * NH] = make_float2(0.5f * (zh.x + zm.x), 0.5f * (zh.y + zm.y));
      const float2 d = csub(zh, zm);
      Sb[h * NH + HC] = make_float2(0.5f * d.y, -0.5f * d.x);
    }
  } else {
#pragma unroll
    for (int h = 0; h < BH; h++) Sb[h * NH + c] = col[h];
  }
}

// Column c inverse DFT along y in place; c == 0 handles columns 0 and bw/2
// together (both Hermitian, so both inverses are real).
template <int BW, int BH>
__device__ __forceinline__ void inv_col(float2* Sb, int c) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2;
  float2 col[BH];
  const bool dc = c == 0;
#pragma unroll
  for (int h = 0; h < BH; h++) {
    const float2 x0 = Sb[h * NH + c];
    if (dc) {
      const float2 xn = Sb[h * NH + HC];
      col[h] = make_float2(x0.x - xn.y, x0.y + xn.x);  // x0 + i xn
    } else {
      col[h] = x0;
    }
  }
  cfft<BH, +1>(col);
  if (dc) {
#pragma unroll
    for (int y = 0; y < BH; y++) {
      Sb[y * NH] = make_float2(col[y].x, 0.f);
      Sb[y * NH + HC] = make_float2(col[y].y, 0.f);
    }
  } else {
#pragma unroll
    for (int y = 0; y < BH; y++) Sb[y * NH + c] = col[y];
  }
}

// Row y: c2r along x; the BW real samples overwrite the row's own storage in
// Sb (BW floats fit in the row's BW/2+1 complex), for a coalesced copy-out.
template <int BW, int BH>
__device__ __forceinline__ void inv_row_inplace(float2* Sb, int y) {
  constexpr int NH = BW / 2 + 1;
  float2* row = Sb + y * NH;
  float2 c[NH];
#pragma unroll
  for (int k = 0; k < NH; k++) c[k] = row[k];
  float r[BW];
  irfft<BW>(c, r);
#pragma unroll
  for (int x = 0; x < BW / 2; x++) row[x] = make_float2(r[2 * x], r[2 * x + 1]);
}

// Coalesced store of one block's time-domain rows (left in Sb by
// inv_row_inplace, row pitch NH complex) to out[BH][BW].
template <int BW, int BH>
__device__ __forceinline__ void store_tdom(const float2* Sb, float* out, int lane) {
  constexpr int NH = BW / 2 + 1, HALF = BW / 2;
  float2* o = reinterpret_cast<float2*>(out);
  for (int i = lane; i < BH * HALF; i += 32) {
    const int y = i / HALF, x = i - y * HALF;
    o[i] = Sb[y * NH + x];
  }
}


// ---------------------------------------------------------------- forward

// One warp transforms blocks_per_warp<BW>() consecutive blocks (rows, then
// columns, then a coalesced 16-byte copy-out of the contiguous spectra).
// PREFETCH: fetch every row of the lane before the first transform, and take
// the x window from the launch parameters (more registers and a parameter-
// space ForwardArgs; off where the register budget is tight or the arguments
// are a copy in registers).
template <int BW, int BH, typename T, bool PREFETCH, class Win>
__device__ __forceinline__ void forward_cta_w(const ForwardArgs& a, int cta, const Win& win) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2, NBW = blocks_per_warp<BW>(), BINS = BH * NH;
  extern __shared__ float2 smem2[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* S = smem2 + warp * NBW * BINS;
  const Geom& g = a.g;
  const int blk0 = (cta * kWarps + warp) * NBW;
  if (blk0 >= g.nblocks) return;
  constexpr int RPL = (NBW * BH + 31) / 32;  // rows per lane
  constexpr int NV = PREFETCH ? raw_vectors<BW, T>() : 0;
  if constexpr (NV > 0) {
    // every row of the lane fetched before the first transform: one load
    // latency per warp instead of one per row
    uint4 raw[RPL][NV];
    bool have[RPL];
#pragma unroll
    for (int i = 0; i < RPL; i++) {
      const int t = lane + 32 * i, b = t / BH, y = t - b * BH;
      have[i] = false;
      if (t < NBW * BH && blk0 + b < g.nblocks) {
        int x0, row;
        const T* srow = fwd_row_src<T>(a, win, blk0 + b, y, &x0, &row);
        const T* p = srow + x0;
        if (x0 >= 0 && x0 + BW <= g.W && (reinterpret_cast<uintptr_t>(p) & 15) == 0 &&
            FFT3D_IN(row >= 0 && row < g.H, a.err)) {
#pragma unroll
          for (int v = 0; v < NV; v++) raw[i][v] = __ldg(reinterpret_cast<const uint4*>(p) + v);
          have[i] = true;
        }
      }
    }
#if FFT3D_FWD_ROW_LOOP
    // one copy of the row transform in the code: the lane's rows walked by a
    // loop, each row's prefetched vectors picked by selects (no local memory)
#pragma unroll 1
    for (int i = 0; i < RPL; i++) {
      const int t = lane + 32 * i, b = t / BH, y = t - b * BH;
      uint4 rr[NV];
      bool hv = false;
#pragma unroll
      for (int q = 0; q < RPL; q++) {
        if (q == i) hv = have[q];
#pragma unroll
        for (int v = 0; v < NV; v++) rr[v] = q == i ? raw[q][v] : (q == 0 ? raw[0][v] : rr[v]);
      }
      if (t < NBW * BH && blk0 + b < g.nblocks)
        fwd_row<BW, BH, T, PREFETCH>(a, win, blk0 + b, y, S + b * BINS, hv ? rr : nullptr);
    }
#else
#pragma unroll
    for (int i = 0; i < RPL; i++) {
      const int t = lane + 32 * i, b = t / BH, y = t - b * BH;
      if (t < NBW * BH && blk0 + b < g.nblocks)
        fwd_row<BW, BH, T, PREFETCH>(a, win, blk0 + b, y, S + b * BINS, have[i] ? raw[i] : nullptr);
    }
#endif
  } else {
    for (int t = lane; t < NBW * BH; t += 32) {
      const int b = t / BH, y = t - b * BH;
      if (blk0 + b < g.nblocks) fwd_row<BW, BH, T, PREFETCH>(a, win, blk0 + b, y, S + b * BINS, nullptr);
    }
  }
  __syncwarp();
  for (int t = lane; t < NBW * HC; t += 32) {
    const int b = t / HC, c = t - b * HC;
    if (blk0 + b < g.nblocks) fwd_col<BW, BH>(S + b * BINS, c);
  }
  __syncwarp();
  const int nvalid = min(NBW, g.nblocks - blk0);
  float4* dst = reinterpret_cast<float4*>(win.spec() + (size_t)blk0 * BINS);
  const float4* src = reinterpret_cast<const float4*>(S);
  for (int i = lane; i < nvalid * BINS / 2; i += 32)
    if (FFT3D_IN((size_t)blk0 * BINS / 2 + i < (size_t)g.nblocks * BINS / 2 && win.spec() != nullptr, a.err))
      dst[i] = src[i];
  __syncwarp();  // S is reused by the warp's next work item
}

template <int BW, int BH, typename T, bool PREFETCH = true>
__device__ __forceinline__ void forward_cta(const ForwardArgs& a, int cta) {
  forward_cta_w<BW, BH, T, PREFETCH, ArgsFwd>(a, cta, ArgsFwd{a});
}

template <int BW, int BH, typename T>
__global__ void __launch_bounds__(kWarps * 32, 5) k_forward(ForwardArgs a) {
  forward_cta<BW, BH, T>(a, blockIdx.x);
}

// The new frames of a frame group in one launch: CTA x transforms CTA
// x % fs.ctas of frame x / fs.ctas (one launch instead of one per frame, so
// the grid has no per-frame wave tail).
template <int BW, int BH, typename T>
__global__ void __launch_bounds__(kWarps * 32, ctas_for(FFT3D_FWD_CTAS, kWarps * fft_smem_bytes<BW, BH>()))
    k_forward_frames(ForwardArgs a, FwdFrameSet fs) {
  const int j = blockIdx.x / fs.ctas, c = blockIdx.x - j * fs.ctas;
  FrameFwd w{nullptr, 0, nullptr};
#pragma unroll
  for (int q = 0; q < kMaxFwdFrames; q++)
    if (q == j) {
      w.s = fs.src[q];
      w.st = fs.stride[q];
      w.sp = fs.spec[q];
    }
  forward_cta_w<BW, BH, T, true, FrameFwd>(a, c, w);
}

// Batched forward: work item i = (plane, CTA of that plane); the grid walks
// the items (persistent when the grid is smaller than the item count).
template <int BW, int BH, typename T>
__global__ void __launch_bounds__(kWarps * 32,
                                  ctas_for(FFT3D_FWD_CTAS, kWarps * fft_smem_bytes<BW, BH>() + (int)sizeof(ForwardArgs)))
    k_forward_batch(const ForwardArgs* __restrict__ args,
                                                                 const int2* __restrict__ items, int nitems) {
  // the item's arguments staged in shared memory: the body's stores cannot
  // alias them, they cost no registers, and the body can take the per-plane
  // kernel's row prefetch (x window read from the staged arguments)
  __shared__ __align__(16) ForwardArgs sa;
  static_assert(sizeof(ForwardArgs) % 4 == 0, "word copy");
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    __syncthreads();  // every warp is done with the previous item's arguments
    const int* src = reinterpret_cast<const int*>(args + it.x);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int w = threadIdx.x; w < (int)(sizeof(ForwardArgs) / 4); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    forward_cta<BW, BH, T, true>(sa, it.y);
  }
}

// ---------------------------------------------------------------- filters

// The per-bin table values one bin's filter reads (the same for every
// block). Loaded before the filter arithmetic, so that their latency is
// hidden behind it instead of stalling the first use.
struct BinTab {
  float2 grid;  // gridsample, when degrid != 0
  float wsh;    // sharpen weight, when sharpen != 0
  float wdh;    // dehalo weight, when dehalo != 0
};
// Only the values that MODE's filter and the sharpen pass read are loaded
// (Kalman and sharpen-only read the grid only in a sharpen pass; the weights
// are read by a sharpen pass or by Wiener 2D's fused factor).
template <int MODE>
__device__ __forceinline__ BinTab bin_tab(const InverseArgs& a, int bin) {
  BinTab t{make_float2(0.f, 0.f), 0.f, 0.f};
  const bool sh = a.c.do_sharpen || (MODE == MODE_WIENER2D && a.c.fuse_sharpen);
  if (a.c.degrid != 0.f && (MODE >= 1 || a.c.do_sharpen)) t.grid = __ldg(a.t.grid + bin);
  if (sh && a.c.use_sharpen) t.wsh = __ldg(a.t.wsharpen + bin);
  if (sh && a.c.use_dehalo) t.wdh = __ldg(a.t.wdehalo + bin);
  return t;
}

// |c|^2 + 1e-15 of a bin (the reference's psd, src/code_impl/Apply.cpp:27-31)
__device__ __forceinline__ float bin_psd(float re, float im) { return fmaf(re, re, fmaf(im, im, 1.0e-15f)); }

__device__ __forceinline__ float sharpen_fact(const InverseArgs& a, float psd, float wsh) {
  // src/code_impl/Apply.cpp:129-131: 1 + sharpen * wsh * sqrt(r) with
  // r = psd * smax2n / ((psd + smin2n)(psd + smax2n)) in [0, 1), the ratio
  // first as in the reference (the product of its terms overflows float for
  // high bit depths), its square root as r * rsqrt(r) (the clamp keeps r = 0,
  // i.e. smax = 0, finite)
  const float r = psd * a.c.smax2n * rcp_nrm((psd + a.c.smin2n) * (psd + a.c.smax2n));
  return fmaf(a.c.sharpen * wsh, r * rsqrt_nrm(fmaxf(r, 1e-30f)), 1.f);
}
__device__ __forceinline__ float dehalo_fact(const InverseArgs& a, float psd, float wdh) {
  // src/code_impl/Apply.cpp:132
  return (psd + a.c.ht2n) * rcp_nrm((psd + a.c.ht2n) + a.c.dehalo * wdh * psd);
}

// limited Wiener factor applied to one temporal component, code_impl_C.h:34-40:
// max((psd - noise) / psd, lowlimit) as max(1 - noise / psd, lowlimit) with
// the fast reciprocal (<= 2 ulp, far inside the +-1 LSB output bar)
// (both parts scaled by one packed multiply)
__device__ __forceinline__ void wiener(float2& v, float noise, float lowlimit) {
  const float q = fmaf(-noise, rcp_nrm(bin_psd(v.x, v.y)), 1.f);
  const float f = fmaxf(q, lowlimit);
  v = __fmul2_rn(v, make_float2(f, f));
}

// Learned noise power of bin `bin` of the block at spectrum offset `off`.
__device__ __forceinline__ float learned_noise(const InverseArgs& a, size_t off, int bin) {
  return a.psd_scale * __ldg(a.psd + (a.psd_per_block ? off : 0) + bin);
}

// One Kalman step of one bin, src/code_impl/Kalman.cpp:27-64: the motion test
// per component (OR), then either a reset to the current value or the gain
// update; last/cv/cp are the bin's state (filtered value, covariance, process
// covariance), updated in place. `sigma` is the bin's noise power.
__device__ __forceinline__ void kalman_step(const InverseArgs& a, float2 cur, float sigma, float2& last, float& cv,
                                            float& cp) {
  const float dr = cur.x - last.x, di = cur.y - last.y;
  if (dr * dr > sigma * a.c.kratio2 || di * di > sigma * a.c.kratio2) {
    cv = sigma;
    cp = sigma;
    last = cur;
  } else {
    const float sum = cv + cp;
    const float gain = sum * rcp_nrm(sum + sigma);
    cp = gain * gain * sigma;
    cv = (1.f - gain) * sum;
    last.x = gain * cur.x + (1.f - gain) * last.x;
    last.y = gain * cur.y + (1.f - gain) * last.y;
  }
}

// Filtered value of one bin from its values w[0..4] in frames n-2..n+2 (only
// the window's entries are read). MODE: 1 = Wiener 2D, 2..5 = Wiener 3D,
// 0 = Kalman (updates the state when `commit`), -1 = sharpen only (identity).
template <int MODE>
__device__ __forceinline__ float2 filter_vals(const InverseArgs& a, const float2 (&w)[5], size_t off, int bin, float gf,
                                              const BinTab& tb, bool commit) {
  const float2 cur = w[2];
  if constexpr (MODE == MODE_SHARPEN_ONLY) {
    return cur;
  } else if constexpr (MODE == MODE_KALMAN) {
    // src/code_impl/Kalman.cpp:27-64; the state is read once and written
    // back by this thread: coherent loads that do not allocate in L1
    float2 last;
    float cv, cp;
    asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(last.x), "=f"(last.y) : "l"(a.kal_last + off + bin));
    asm("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(cv) : "l"(a.kal_covar + off + bin));
    asm("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(cp) : "l"(a.kal_covarp + off + bin));
    float sigma = a.c.sigma2n_2d;
    if (a.psd) {
      sigma = learned_noise(a, off, bin);
      if (sigma < 1e-15f) sigma = 1e-15f;
    } else if (a.c.pattern) {
      sigma = __ldg(a.t.pattern2d + bin);
      if (sigma < 1e-15f) sigma = 1e-15f;
    }
    kalman_step(a, cur, sigma, last, cv, cp);
    if (commit) {
      a.kal_last[off + bin] = last;
      a.kal_covar[off + bin] = cv;
      a.kal_covarp[off + bin] = cp;
    }
    return last;
  } else if constexpr (MODE == MODE_WIENER2D) {
    // src/code_impl/Apply.cpp:13-65
    float2 gc = make_float2(0.f, 0.f);
    if (a.c.degrid != 0.f) gc = make_float2(gf * tb.grid.x, gf * tb.grid.y);
    const float cr = cur.x - gc.x, ci = cur.y - gc.y;
    const float psd = bin_psd(cr, ci);
    const float noise = a.psd ? learned_noise(a, off, bin) : a.c.pattern ? __ldg(a.t.pattern2d + bin) : a.c.sigma2n;
    float f = fmaxf(fmaf(-noise, rcp_nrm(psd), 1.f), a.c.lowlimit);
    if (a.c.fuse_sharpen) {
      if (a.c.use_sharpen && a.c.use_dehalo) f *= sharpen_fact(a, psd, tb.wsh) * dehalo_fact(a, psd, tb.wdh);
      else if (a.c.use_sharpen) f *= sharpen_fact(a, psd, tb.wsh);
      else if (a.c.use_dehalo) f *= dehalo_fact(a, psd, tb.wdh);
    }
    return make_float2(cr * f + gc.x, ci * f + gc.y);
  } else {
    // Wiener 3D over MODE frames, src/code_impl/Apply.cpp:67-235. The short
    // temporal DFT works on (re, im) pairs with packed f32x2 adds and
    // multiplies (one instruction per complex sum or real-scaled term); the
    // terms and their signs are the reference's, the association of a few
    // sums differs (rounding only). gc * bt (src/code_impl/Apply.cpp:78-93)
    // uses gf * MODE, the same for every bin of the block.
    const float gk = gf * (float)MODE;
    float2 g = make_float2(0.f, 0.f);
    if (a.c.degrid != 0.f) g = __fmul2_rn(tb.grid, make_float2(gk, gk));
    const float noise = a.psd ? learned_noise(a, off, bin) : a.c.pattern ? __ldg(a.t.pattern3d + bin) : a.c.sigma2n;
    const float ll = a.c.lowlimit;
    auto wf = [&](float2& v) { wiener(v, noise, ll); };
    auto add = [](float2 x, float2 y) { return __fadd2_rn(x, y); };
    auto sub = [](float2 x, float2 y) { return __fadd2_rn(x, make_float2(-y.x, -y.y)); };
    auto rot = [](float2 v) { return make_float2(v.y, -v.x); };  // -i v
    if constexpr (MODE == 2) {
      const float2 pv = w[1];
      float2 f0 = sub(add(cur, pv), g), f1 = sub(cur, pv);
      wf(f0);
      wf(f1);
      return __fmul2_rn(add(add(f0, f1), g), make_float2(0.5f, 0.5f));
    } else if constexpr (MODE == 3) {
      const float sin120 = 0.86602540378443864676372317075294f;
      const float2 pv = w[1], nx = w[3];
      const float2 pn = add(pv, nx);
      float2 fc = sub(add(cur, pn), g);
      const float2 h = __ffma2_rn(pn, make_float2(-0.5f, -0.5f), cur);      // cur - pn / 2
      const float2 m = rot(__fmul2_rn(sub(pv, nx), make_float2(sin120, sin120)));  // (di, dr)
      float2 fp = add(h, m), fn = sub(h, m);
      wf(fc);
      wf(fp);
      wf(fn);
      const float third = 1.0f / 3.0f;
      return __fmul2_rn(add(add(add(fc, fp), fn), g), make_float2(third, third));
    } else if constexpr (MODE == 4) {
      const float2 p2 = w[0], pv = w[1], nx = w[3];
      const float2 cp = add(cur, p2), cm = sub(cur, p2), pn = add(pv, nx);
      const float2 d = rot(sub(pv, nx));  // (pv.y - nx.y, nx.x - pv.x)
      float2 fp2 = sub(cp, pn), fc = sub(add(cp, pn), g);
      float2 fp = add(cm, d), fn = sub(cm, d);
      wf(fp2);
      wf(fp);
      wf(fc);
      wf(fn);
      return __fmul2_rn(add(add(add(fp2, fp), add(fc, fn)), g), make_float2(0.25f, 0.25f));
    } else {
      const float sin72 = 0.95105651629515357211643933337938f, cos72 = 0.30901699437494742410229341718282f;
      const float sin144 = 0.58778525229247312916870595463907f, cos144 = -0.80901699437494742410229341718282f;
      const float2 p2 = w[0], pv = w[1], nx = w[3], n2 = w[4];
      const float2 a2 = add(p2, n2), a1 = add(pv, nx);  // outer and inner pair sums
      const float2 e2 = sub(n2, p2), e1 = sub(pv, nx);  // their differences
      const float2 s1 = add(__ffma2_rn(a2, make_float2(cos72, cos72), __fmul2_rn(a1, make_float2(cos144, cos144))), cur);
      const float2 s2 = add(__ffma2_rn(a2, make_float2(cos144, cos144), __fmul2_rn(a1, make_float2(cos72, cos72))), cur);
      // -i (e2 sin72 + e1 sin144) and -i (e1 sin72 - e2 sin144)
      const float2 t1 = rot(__ffma2_rn(e2, make_float2(sin72, sin72), __fmul2_rn(e1, make_float2(sin144, sin144))));
      const float2 t2 = rot(__ffma2_rn(e2, make_float2(-sin144, -sin144), __fmul2_rn(e1, make_float2(sin72, sin72))));
      float2 fp2 = add(s1, t1), fn2 = sub(s1, t1);
      float2 fp = add(s2, t2), fn = sub(s2, t2);
      float2 fc = sub(add(add(a2, a1), cur), g);
      wf(fp2);
      wf(fp);
      wf(fc);
      wf(fn);
      wf(fn2);
      return __fmul2_rn(add(add(add(add(fp2, fp), add(fc, fn)), fn2), g), make_float2(0.2f, 0.2f));
    }
  }
}

// Window slots 2 - MODE/2 .. 2 + (MODE-1)/2 of a MODE-frame Wiener 3D (the
// reference's apply_in[] table, src/fft3d_engine.h:634-644); one slot otherwise.
template <int MODE>
__host__ __device__ constexpr int win_lo() { return MODE >= 2 ? 2 - MODE / 2 : 2; }
template <int MODE>
__host__ __device__ constexpr int win_hi() { return MODE >= 2 ? 2 + (MODE - 1) / 2 : 2; }

template <int MODE>
__device__ __forceinline__ float2 filter_bin(const InverseArgs& a, size_t off, int bin, float gf, bool commit) {
  float2 w[5];
#pragma unroll
  for (int k = 0; k < 5; k++)
    w[k] = (k >= win_lo<MODE>() && k <= win_hi<MODE>()) ? __ldg(a.in[k] + off + bin) : make_float2(0.f, 0.f);
  return filter_vals<MODE>(a, w, off, bin, gf, bin_tab<MODE>(a, bin), commit);
}

// separate sharpen/dehalo pass on a filtered bin, src/code_impl/Sharpen.cpp:13-63
// (the grid term removed and restored with packed f32x2 operations)
__device__ __forceinline__ float2 sharpen_bin(const InverseArgs& a, float2 v, const BinTab& tb, float gf) {
  float2 gc = make_float2(0.f, 0.f);
  if (a.c.degrid != 0.f) gc = __fmul2_rn(tb.grid, make_float2(gf, gf));
  const float2 c = __fadd2_rn(v, make_float2(-gc.x, -gc.y));
  const float psd = bin_psd(c.x, c.y);
  float f;
  if (a.c.use_sharpen && a.c.use_dehalo) f = sharpen_fact(a, psd, tb.wsh) * dehalo_fact(a, psd, tb.wdh);
  else if (a.c.use_sharpen) f = sharpen_fact(a, psd, tb.wsh);
  else f = dehalo_fact(a, psd, tb.wdh);
  return __ffma2_rn(c, make_float2(f, f), gc);
}

// ---------------------------------------------------------------- filter (streaming)

// Two neighbouring bins of a window spectrum, read once per thread: not kept
// in L1 (the per-bin tables stay there).
__device__ __forceinline__ float4 ld_stream4(const float2* p) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}

// Filter of every bin of every block as a flat stream: each thread takes two
// neighbouring bins (one 16-byte load per window frame, one 16-byte store of
// the filtered pair to F). No shared memory and few registers, so the SMs
// hold enough warps to keep the spectrum reads at HBM speed. The separate
// sharpen/dehalo pass, which needs each block's filtered DC, runs afterwards
// in k_filter_inverse<MODE_SHARPEN_ONLY> on F.
template <int MODE>
__global__ void __launch_bounds__(256) k_filter_bins(InverseArgs a, float2* F, int bins_per_block) {
  constexpr int LO = win_lo<MODE>(), NW = win_hi<MODE>() - win_lo<MODE>() + 1;
  const size_t pairs = (size_t)a.g.nblocks * bins_per_block / 2;
  const float gs0 = __ldg(&a.t.grid[0].x);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < pairs; q += (size_t)gridDim.x * blockDim.x) {
    const size_t e = 2 * q;
    const int bin = (int)(e % bins_per_block);
    const size_t off = e - bin;
    float4 wv[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) wv[k] = __ldg(reinterpret_cast<const float4*>(a.in[LO + k] + e));
    const float gf = (MODE >= 1) ? a.c.degrid * __ldg(&a.in[2][off].x) / gs0 : 0.f;
    float2 w0[5], w1[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const bool in = k >= LO && k < LO + NW;
      w0[k] = in ? make_float2(wv[k - LO].x, wv[k - LO].y) : make_float2(0.f, 0.f);
      w1[k] = in ? make_float2(wv[k - LO].z, wv[k - LO].w) : make_float2(0.f, 0.f);
    }
    const float2 v0 = filter_vals<MODE>(a, w0, off, bin, gf, bin_tab<MODE>(a, bin), true);
    const float2 v1 = filter_vals<MODE>(a, w1, off, bin + 1, gf, bin_tab<MODE>(a, bin + 1), true);
    reinterpret_cast<float4*>(F)[q] = make_float4(v0.x, v0.y, v1.x, v1.y);
  }
}

// Filter of a run of consecutive output frames of one plane (a frame group)
// in one launch: each thread takes two neighbouring bins of one block and
// walks the run's frames in order with the bins' temporal window in
// registers, so that every window spectrum is loaded once per run (not once
// per output frame), and a Kalman state once per run. fs.spec[s] is frame
// n0 - 2 + s; frame n0 + j's window is fs.spec[j + LO .. j + HI] and its
// filtered bins go to fs.out[j]. The sharpen/dehalo pass and the inverse
// transform follow per frame (k_filter_inverse_frames<MODE_SHARPEN_ONLY> on
// fs.out[j]). Few registers and no shared memory: the SMs hold enough warps
// to cover the load latency by themselves.
template <int MODE>
__global__ void __launch_bounds__(256) k_filter_frames(InverseArgs a, const __grid_constant__ FilterFrameSet fs,
                                                     int bins_per_block) {
  constexpr int LO = win_lo<MODE>(), HI = win_hi<MODE>(), NW = HI - LO + 1;
  const size_t pairs = (size_t)a.g.nblocks * bins_per_block / 2;
  const float gs0 = __ldg(&a.t.grid[0].x);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < pairs; q += (size_t)gridDim.x * blockDim.x) {
    const size_t e = 2 * q;
    const int bin = (int)(e % bins_per_block);
    const size_t off = e - bin;
    const BinTab tb0 = bin_tab<MODE>(a, bin), tb1 = bin_tab<MODE>(a, bin + 1);
    if constexpr (MODE == MODE_KALMAN) {
      // the state of both bins stays in registers across the run's frames
      float4 lv;
      float2 cv, cp;
      asm("ld.global.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
          : "=f"(lv.x), "=f"(lv.y), "=f"(lv.z), "=f"(lv.w) : "l"(a.kal_last + e));
      asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(cv.x), "=f"(cv.y) : "l"(a.kal_covar + e));
      asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(cp.x), "=f"(cp.y) : "l"(a.kal_covarp + e));
      float2 l0 = make_float2(lv.x, lv.y), l1 = make_float2(lv.z, lv.w);
      float s0 = a.c.sigma2n_2d, s1 = a.c.sigma2n_2d;
      if (a.c.pattern) {
        s0 = fmaxf(__ldg(a.t.pattern2d + bin), 1e-15f);
        s1 = fmaxf(__ldg(a.t.pattern2d + bin + 1), 1e-15f);
      }
      for (int j = 0; j < fs.count; j++) {
        const float4 c = ld_stream4(fs.spec[j + 2] + e);
        kalman_step(a, make_float2(c.x, c.y), s0, l0, cv.x, cp.x);
        kalman_step(a, make_float2(c.z, c.w), s1, l1, cv.y, cp.y);
        reinterpret_cast<float4*>(fs.out[j])[q] = make_float4(l0.x, l0.y, l1.x, l1.y);
      }
      reinterpret_cast<float4*>(a.kal_last)[q] = make_float4(l0.x, l0.y, l1.x, l1.y);
      reinterpret_cast<float2*>(a.kal_covar)[q] = cv;
      reinterpret_cast<float2*>(a.kal_covarp)[q] = cp;
    } else {
      float4 wv[NW];
#pragma unroll
      for (int k = 0; k < NW - 1; k++) wv[k] = ld_stream4(fs.spec[LO + k] + e);
      for (int j = 0; j < fs.count; j++) {
        wv[NW - 1] = ld_stream4(fs.spec[j + HI] + e);
        const float gf = (MODE >= 1) ? a.c.degrid * __ldg(&fs.spec[j + 2][off].x) / gs0 : 0.f;
        float2 w0[5], w1[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
          const bool in = k >= LO && k <= HI;
          w0[k] = in ? make_float2(wv[k - LO].x, wv[k - LO].y) : make_float2(0.f, 0.f);
          w1[k] = in ? make_float2(wv[k - LO].z, wv[k - LO].w) : make_float2(0.f, 0.f);
        }
        const float2 v0 = filter_vals<MODE>(a, w0, off, bin, gf, tb0, false);
        const float2 v1 = filter_vals<MODE>(a, w1, off, bin + 1, gf, tb1, false);
        reinterpret_cast<float4*>(fs.out[j])[q] = make_float4(v0.x, v0.y, v1.x, v1.y);
#pragma unroll
        for (int k = 0; k < NW - 1; k++) wv[k] = wv[k + 1];
      }
    }
  }
}

// ---------------------------------------------------------------- inverse

// One warp filters and inverse-transforms blocks_per_warp<BW>() blocks:
//  A. every bin of a block, consecutive bins on consecutive lanes (coalesced
//     loads of the bt spectra), through the filter and the separate
//     sharpen/dehalo pass (whose grid fraction is the filtered DC, lane 0's
//     first bin); results to shared memory;
//  B. one column per lane: inverse complex DFT along y (DC and Nyquist columns
//     together: both are Hermitian, so their inverses are real);
//  C. one row per lane: c2r along x, 16-byte stores of the time-domain rows.
template <int BW, int BH>
__host__ __device__ constexpr int fft_ctas(int nblocks) {
  return (nblocks + kWarps * blocks_per_warp<BW>() - 1) / (kWarps * blocks_per_warp<BW>());
}

// A window-spectrum value, read once per CTA: not kept in L1, where the
// per-bin tables (grid, wsharpen) that every chunk reads should stay.
__device__ __forceinline__ float2 ld_stream(const float2* p) {
  float2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}

// Where a CTA finds its window spectra and writes its time-domain blocks:
// the launch arguments (one output frame per launch), or pointers picked for
// one frame of a frame group (k_filter_inverse_frames).
// kHoistTab: a chunk's per-bin table values are loaded before its filter
// arithmetic (measured faster one frame per launch); the frame-group kernel
// loads each next to its first use (faster there: fewer live registers).
struct ArgsWin {
  static constexpr bool kHoistTab = true;
  const InverseArgs& a;
  __device__ __forceinline__ const float2* in(int k) const { return a.in[k]; }
  __device__ __forceinline__ float* tdom() const { return a.tdom; }
};
struct FrameWin {
  static constexpr bool kHoistTab = false;
  const float2* p[5];
  float* t;
  __device__ __forceinline__ const float2* in(int k) const { return p[k]; }
  __device__ __forceinline__ float* tdom() const { return t; }
};

// NEWEST_IN_S: the window's newest frame (slot win_hi) is not read from
// the window but from S, where the fused kernel's forward transform left it.
template <int BW, int BH, int MODE, bool NEWEST_IN_S, class Win>
__device__ __forceinline__ void filter_inverse_cta_w(const InverseArgs& a, int vcta, const Win& win) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2, NBW = blocks_per_warp<BW>(), BINS = BH * NH;
  constexpr int PER = (BINS + 31) / 32;
  extern __shared__ float2 smem2[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* S = smem2 + warp * NBW * BINS;
  const Geom& g = a.g;
  const int cta = a.reverse ? fft_ctas<BW, BH>(g.nblocks) - 1 - vcta : vcta;
  const int blk0 = (cta * kWarps + warp) * NBW;
  if (blk0 >= g.nblocks) return;
  const float gs0 = __ldg(&a.t.grid[0].x);
  constexpr int LO = win_lo<MODE>(), HI = win_hi<MODE>(), NW = HI - LO + 1;
  constexpr int NG = NEWEST_IN_S ? NW - 1 : NW;  // window slots read from global memory
  constexpr int NGB = NG > 0 ? NG : 1;
  // load-pipeline depth (chunks of 32 bins in flight): all chunks for a
  // one-frame window, fewer as the window (and the registers per chunk) grows
  constexpr int DW = NG <= 1 ? PER : (NG == 2 ? 10 : (NG == 3 ? 7 : (NG == 4 ? 5 : 4)));
  constexpr int D = PER < DW ? PER : DW;
#pragma unroll 1
  for (int b = 0; b < NBW; b++) {
    const int blk = blk0 + b;
    if (blk >= g.nblocks) break;
    const size_t off = (size_t)blk * BINS;
    float gf = 0.f;
    if constexpr (MODE >= 1) {
      if (NEWEST_IN_S && HI == 2) {
        gf = a.c.degrid * S[b * BINS].x / gs0;
        __syncwarp();  // every lane has the DC before lane 0 overwrites it
      } else {
        gf = a.c.degrid * __ldg(&win.in(2)[off].x) / gs0;
      }
    }
    // software pipeline: the window's values of chunk j + D are loaded while
    // chunk j is filtered, so D x NG loads per lane are always in flight
    float2 buf[D][NGB];
    auto load = [&](int j, float2(&dst)[NGB]) {
      const int i = lane + 32 * j;
#pragma unroll
      for (int k = 0; k < NG; k++)
        dst[k] = (i < BINS && FFT3D_IN(win.in(LO + k) != nullptr && off + i < (size_t)g.nblocks * BINS, a.err))
                     ? ld_stream(win.in(LO + k) + off + i)
                     : make_float2(0.f, 0.f);
    };
    if constexpr (NG > 0) {
#pragma unroll
      for (int j = 0; j < D; j++) load(j, buf[j]);
    }
    float gsh = 0.f;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int i = lane + 32 * j;
      float2 w[5];
#pragma unroll
      for (int k = 0; k < 5; k++) w[k] = (k >= LO && k < LO + NG) ? buf[j % D][k - LO] : make_float2(0.f, 0.f);
      if (NEWEST_IN_S && i < BINS) w[HI] = S[b * BINS + i];
      BinTab tb{make_float2(0.f, 0.f), 0.f, 0.f};
      if constexpr (Win::kHoistTab) {
        // the chunk's table values first: the filter arithmetic hides their latency
        if (i < BINS) tb = bin_tab<MODE>(a, i);
      } else if (MODE == MODE_WIENER2D && a.c.fuse_sharpen) {
        if (i < BINS) tb = bin_tab<MODE>(a, i);  // the Wiener factor takes the sharpen/dehalo weights
      } else {
        if (i < BINS && a.c.degrid != 0.f) tb.grid = __ldg(a.t.grid + i);
      }
      if (NG > 0 && j + D < PER) load(j + D, buf[j % D]);
      float2 v = make_float2(0.f, 0.f);
      if (i < BINS) v = filter_vals<MODE>(a, w, off, i, gf, tb, true);
      if (a.c.do_sharpen) {
        // grid fraction of the sharpen pass: the filtered DC (lane 0, chunk 0)
        if (j == 0) gsh = a.c.degrid * __shfl_sync(0xffffffffu, v.x, 0) / gs0;
        if constexpr (!Win::kHoistTab) {
          if (i < BINS && a.c.use_sharpen) tb.wsh = __ldg(a.t.wsharpen + i);
          if (i < BINS && a.c.use_dehalo) tb.wdh = __ldg(a.t.wdehalo + i);
        }
        if (i < BINS) v = sharpen_bin(a, v, tb, gsh);
      }
      if (i < BINS) S[b * BINS + i] = v;
    }
  }
  __syncwarp();
  for (int t = lane; t < NBW * HC; t += 32) {
    const int b = t / HC, c = t - b * HC;
    if (blk0 + b < g.nblocks) inv_col<BW, BH>(S + b * BINS, c);
  }
  __syncwarp();
  for (int t = lane; t < NBW * BH; t += 32) {
    const int b = t / BH, y = t - b * BH;
    if (blk0 + b < g.nblocks) inv_row_inplace<BW, BH>(S + b * BINS, y);
  }
  __syncwarp();
  for (int b = 0; b < NBW && blk0 + b < g.nblocks; b++)
    if (FFT3D_IN(win.tdom() != nullptr, a.err)) store_tdom<BW, BH>(S + b * BINS, win.tdom() + (size_t)(blk0 + b) * BH * BW, lane);
  __syncwarp();  // S is reused by the warp's next work item
}

template <int BW, int BH, int MODE, bool NEWEST_IN_S = false>
__device__ __forceinline__ void filter_inverse_cta(const InverseArgs& a, int vcta) {
  filter_inverse_cta_w<BW, BH, MODE, NEWEST_IN_S, ArgsWin>(a, vcta, ArgsWin{a});
}

// Several consecutive output frames of one plane in one launch (a frame
// group). CTA x works on frame x % count, CTA-of-frame x / count: the
// resident CTAs of all the group's frames cover the same blocks at the same
// time, so a window spectrum shared by up to bt frames is read from HBM once
// and then hit in L2. The frames differ only in their window spectra and
// time-domain buffers (fs); everything else is in a.
template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32) k_filter_inverse_frames(InverseArgs a, FrameSet fs) {
  const int j = blockIdx.x % fs.count, c = blockIdx.x / fs.count;
  // the frame's pointers, selected with constant indices (a dynamic index
  // into the parameter space would copy it to local memory)
  FrameWin w;
#pragma unroll
  for (int k = 0; k < 5; k++) w.p[k] = nullptr;
  w.t = nullptr;
#pragma unroll
  for (int q = 0; q < kMaxGroupFrames; q++)
    if (q == j) {
#pragma unroll
      for (int k = 0; k < 5; k++) w.p[k] = fs.in[q][k];
      w.t = fs.tdom[q];
    }
  filter_inverse_cta_w<BW, BH, MODE, false, FrameWin>(a, c, w);
}

template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32) k_filter_inverse(InverseArgs a) {
  filter_inverse_cta<BW, BH, MODE>(a, blockIdx.x);
}

// The work item's arguments are staged in shared memory: the body's global
// stores cannot alias them (a reference into global memory would be reloaded
// after every store), and unlike a by-value copy they cost no registers.
template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32) k_filter_inverse_batch(const InverseArgs* __restrict__ args,
                                                                     const int2* __restrict__ items, int nitems) {
  __shared__ __align__(16) InverseArgs sa;
  static_assert(sizeof(InverseArgs) % 4 == 0, "word copy");
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    __syncthreads();  // every warp is done with the previous item's arguments
    const int* src = reinterpret_cast<const int*>(args + it.x);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int w = threadIdx.x; w < (int)(sizeof(InverseArgs) / 4); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    filter_inverse_cta<BW, BH, MODE>(sa, it.y);
  }
}

// ---------------------------------------------------------------- overlap-add pixels

// Time-domain block reads of the overlap-add. Blocks written by an earlier
// launch go through the read-only path without L1 allocation (each value is
// read once; the synthesis windows stay in L1). Blocks written by other CTAs
// of the same launch (L2 = true, the fused overlap-add of a frame group) are
// read at L2, the point where those CTAs' stores are visible.
template <bool L2>
__device__ __forceinline__ float ld_tdom(const float* p) {
  if constexpr (L2) return __ldcg(p);
  else return __ldg(p);
}
template <bool L2>
__device__ __forceinline__ float4 ld_tdom4(const float* p) {
  if constexpr (L2) {
    return __ldcg(reinterpret_cast<const float4*>(p));
  } else {
    float4 q;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(q.x), "=f"(q.y), "=f"(q.z), "=f"(q.w)
        : "l"(p));
    return q;
  }
}

template <typename T>
__device__ __forceinline__ void store_sample(T* p, float v, int maxval);
template <>
__device__ __forceinline__ void store_sample<uint8_t>(uint8_t* p, float v, int maxval) {
  int i = __float2int_rz(v);  // C cast: truncation toward zero (src/buffer.cpp:406)
  i = i < 0 ? 0 : (i > maxval ? maxval : i);
  *p = (uint8_t)i;
}
template <>
__device__ __forceinline__ void store_sample<uint16_t>(uint16_t* p, float v, int maxval) {
  int i = __float2int_rz(v);
  i = i < 0 ? 0 : (i > maxval ? maxval : i);
  *p = (uint16_t)i;
}
template <>
__device__ __forceinline__ void store_sample<float>(float* p, float v, int) {
  float c = v < 0.f ? 0.f : v;  // float samples clamp to [0, 1] (src/buffer.cpp:397)
  *p = c > 1.f ? 1.f : c;
}

// One thread per output pixel of the processed region: the (at most four)
// blocks covering it, weighted with the synthesis windows and the FFT
// normalisation in the association order of src/buffer.cpp:399-559.
template <typename T, bool L2 = false>
__device__ __forceinline__ void overlap_add_px(const OlaArgs& a, int x0, int k) {
  const Geom& g = a.g;
  if (x0 >= g.W || k >= g.H) return;
  const int Y = g.sy + k, X = g.sx + x0;
  const int by = div_small(Y, g.sy), y = Y - by * g.sy;
  const int bx = div_small(X, g.sx), x = X - bx * g.sx;
  const bool yov = y < g.oh, xov = x < g.ow;
  const int bw = g.bw, bh = g.bh;
  auto at = [&](int bxx, int byy, int yy, int xx) {
    if (!FFT3D_IN(bxx >= 0 && bxx < g.nox && byy >= 0 && byy < g.noy && yy >= 0 && yy < bh && xx >= 0 && xx < bw,
                  a.err))
      return 0.f;
    return ld_tdom<L2>(a.tdom + ((size_t)(byy * g.nox + bxx) * bh + yy) * bw + xx);
  };
  const float norm = a.norm;
  float v;
  if (!yov) {
    const float d = at(bx, by, y, x);
    if (!xov) v = d * norm + a.rounder + a.base;
    else {
      const float c = at(bx - 1, by, y, x + g.sx);
      v = (c * __ldg(a.t.wsyn_xr + x) + d * __ldg(a.t.wsyn_xl + x)) * norm + a.rounder + a.base;
    }
  } else {
    const float wr = __ldg(a.t.wsyn_yr + y) * norm, wl = __ldg(a.t.wsyn_yl + y) * norm;
    const float b = at(bx, by - 1, y + g.sy, x), d = at(bx, by, y, x);
    if (!xov) v = (b * wr + d * wl) + a.rounder + a.base;
    else {
      const float aa = at(bx - 1, by - 1, y + g.sy, x + g.sx), c = at(bx - 1, by, y, x + g.sx);
      const float sxr = __ldg(a.t.wsyn_xr + x), sxl = __ldg(a.t.wsyn_xl + x);
      v = ((aa * sxr + b * sxl) * wr + (c * sxr + d * sxl) * wl) + a.rounder + a.base;
    }
  }
  const int fr = field_row(k, g.H, g.interlaced);
  if (!FFT3D_IN(fr >= 0 && fr < g.H, a.err)) return;
  T* row = reinterpret_cast<T*>(static_cast<char*>(a.dst) + (long long)fr * a.dst_stride);
  store_sample<T>(row + x0, v, a.maxval);
}

// Four adjacent output pixels per thread (x0 a multiple of 4), for planes
// whose block step, overlap, width and block width are multiples of 4 and
// whose destination rows are aligned for a 4-sample store: the four pixels
// share their blocks and overlap case, so the tdom reads are float4 loads,
// the block indices are computed once and the samples go out in one store.
// Each pixel's arithmetic is overlap_add_px's, term for term.
template <typename T>
struct Pack4;
template <>
struct Pack4<uint8_t> {
  using V = uchar4;
};
template <>
struct Pack4<uint16_t> {
  using V = ushort4;
};
template <>
struct Pack4<float> {
  using V = float4;
};

template <typename T>
__device__ __forceinline__ T clamp_sample(float v, int maxval) {
  if constexpr (sizeof(T) == 4) {
    float c = v < 0.f ? 0.f : v;
    return c > 1.f ? 1.f : c;
  } else {
    int i = __float2int_rz(v);
    i = i < 0 ? 0 : (i > maxval ? maxval : i);
    return (T)i;
  }
}

// The 4-pixel overlap-add in two steps, so that a thread can issue the block
// reads of several pixel quads before it computes any of them: ola4_fetch
// reads the (at most four) time-domain float4s of quad (x0, k) from `tdom`,
// ola4_finish weights, sums, rounds and stores them.
struct Ola4Px {
  float4 aa, b, c, d;  // blocks (bx-1, by-1), (bx, by-1), (bx-1, by), (bx, by); zero where not read
  int x, y;            // position inside the block step
  bool xov, yov, ok;
};

template <bool L2>
__device__ __forceinline__ Ola4Px ola4_fetch(const OlaArgs& a, const float* tdom, int x0, int k) {
  const Geom& g = a.g;
  Ola4Px p;
  p.aa = p.b = p.c = p.d = make_float4(0.f, 0.f, 0.f, 0.f);
  p.ok = x0 < g.W && k < g.H;
  if (!p.ok) return p;
  const int Y = g.sy + k, X = g.sx + x0;
  const int by = div_small(Y, g.sy), bx = div_small(X, g.sx);
  p.y = Y - by * g.sy;
  p.x = X - bx * g.sx;
  p.yov = p.y < g.oh;
  p.xov = p.x < g.ow;
  const int bw = g.bw, bh = g.bh;
  auto at4 = [&](int bxx, int byy, int yy, int xx) {
    if (!FFT3D_IN(bxx >= 0 && bxx < g.nox && byy >= 0 && byy < g.noy && yy >= 0 && yy < bh && xx >= 0 &&
                      xx + 3 < bw,
                  a.err))
      return make_float4(0.f, 0.f, 0.f, 0.f);
    return ld_tdom4<L2>(tdom + ((size_t)(byy * g.nox + bxx) * bh + yy) * bw + xx);
  };
  p.d = at4(bx, by, p.y, p.x);
  if (p.xov) p.c = at4(bx - 1, by, p.y, p.x + g.sx);
  if (p.yov) {
    p.b = at4(bx, by - 1, p.y + g.sy, p.x);
    if (p.xov) p.aa = at4(bx - 1, by - 1, p.y + g.sy, p.x + g.sx);
  }
  return p;
}

template <typename T>
__device__ __forceinline__ void ola4_finish(const OlaArgs& a, void* dst, long long dst_stride, int x0, int k,
                                            const Ola4Px& p) {
  if (!p.ok) return;
  const Geom& g = a.g;
  const int x = p.x, y = p.y;
  auto comp = [](const float4& q, int i) { return i == 0 ? q.x : (i == 1 ? q.y : (i == 2 ? q.z : q.w)); };
  const float norm = a.norm;
  float v[4];
  if (!p.yov) {
    if (!p.xov) {
#pragma unroll
      for (int i = 0; i < 4; i++) v[i] = comp(p.d, i) * norm + a.rounder + a.base;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++)
        v[i] = (comp(p.c, i) * __ldg(a.t.wsyn_xr + x + i) + comp(p.d, i) * __ldg(a.t.wsyn_xl + x + i)) * norm +
               a.rounder + a.base;
    }
  } else {
    const float wr = __ldg(a.t.wsyn_yr + y) * norm, wl = __ldg(a.t.wsyn_yl + y) * norm;
    if (!p.xov) {
#pragma unroll
      for (int i = 0; i < 4; i++) v[i] = (comp(p.b, i) * wr + comp(p.d, i) * wl) + a.rounder + a.base;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float sxr = __ldg(a.t.wsyn_xr + x + i), sxl = __ldg(a.t.wsyn_xl + x + i);
        v[i] = ((comp(p.aa, i) * sxr + comp(p.b, i) * sxl) * wr + (comp(p.c, i) * sxr + comp(p.d, i) * sxl) * wl) +
               a.rounder + a.base;
      }
    }
  }
  const int fr = field_row(k, g.H, g.interlaced);
  if (!FFT3D_IN(fr >= 0 && fr < g.H && x0 + 3 < g.W, a.err)) return;
  T* row = reinterpret_cast<T*>(static_cast<char*>(dst) + (long long)fr * dst_stride);
  typename Pack4<T>::V o;
  o.x = clamp_sample<T>(v[0], a.maxval);
  o.y = clamp_sample<T>(v[1], a.maxval);
  o.z = clamp_sample<T>(v[2], a.maxval);
  o.w = clamp_sample<T>(v[3], a.maxval);
  *reinterpret_cast<typename Pack4<T>::V*>(row + x0) = o;
}

template <typename T, bool L2 = false>
__device__ __forceinline__ void overlap_add_px4(const OlaArgs& a, int x0, int k) {
  const Ola4Px p = ola4_fetch<L2>(a, a.tdom, x0, k);
  ola4_finish<T>(a, a.dst, a.dst_stride, x0, k, p);
}

// ---------------------------------------------------------------- frame groups, one CTA per block

// Dynamic shared memory of k_filter_inverse_group: two grid fractions per
// frame (64 bytes), then `count` spectrum tiles.
template <int BW, int BH>
__host__ __device__ constexpr int group_smem_bytes(int count) {
  return 2 * kGroupTile * 4 + count * BH * (BW / 2 + 1) * 8;
}

// A run of count <= kGroupTile consecutive output frames of one plane with
// one mode; CTA = one block. Each stage is spread over the whole CTA, with a
// barrier between stages:
//  0. the grid fraction of each frame's block (its DC);
//  1. filter: each thread takes two neighbouring bins and walks the run's
//     frames in order, its window of MODE frames in registers (a circular
//     buffer; the next frame's bins loaded one frame ahead), so that each of
//     the block's count + MODE - 1 window spectra is read once for the run
//     (and a Kalman state once); the filtered bins of frame j go to tile j in
//     shared memory, and the thread holding the DC publishes each tile's
//     filtered DC;
//     (pairs beyond the last whole round of the CTA's threads are spread
//     over all threads as single (pair, frame) items, so that no warp walks
//     a third round alone);
//  2. the separate sharpen/dehalo pass (src/code_impl/Sharpen.cpp:13-63), its
//     grid fraction from each tile's filtered DC, the pair's tables loaded
//     once for all frames;
//  3. the inverse column DFTs of every tile (DC and Nyquist columns as one
//     complex transform), 4. the c2r rows, 5. coalesced stores of the
//     time-domain blocks.
// Every bin and every transform uses the arithmetic of k_filter_inverse
// (filter_vals, kalman_step, sharpen_bin, inv_col, inv_row_inplace), so the
// output equals one frame per launch.
// A run's window spectrum s, bins bin and bin + 1 of the block at `off`
// (checked build: the spectrum exists and the pair lies in the plane).
__device__ __forceinline__ float4 group_load(const InverseArgs& a, const TemporalSet& ts, int s, size_t off, int bin) {
  if (!FFT3D_IN(s >= 0 && s < kGroupTile + 4 && ts.spec[s] != nullptr &&
                    off + bin + 1 < (size_t)a.g.nblocks * a.g.bh * a.g.nh,
                a.err))
    return make_float4(0.f, 0.f, 0.f, 0.f);
  return ld_stream4(ts.spec[s] + off + bin);
}

template <int MODE>
__device__ __forceinline__ void group_filter_pair(const InverseArgs& a, const TemporalSet& ts, size_t off, int bin,
                                                  int count, const float* gfs, float* gsh, float gs0, float2* tile,
                                                  int tile_stride) {
  constexpr int LO = win_lo<MODE>(), HI = win_hi<MODE>(), NW = HI - LO + 1;
  auto out = [&](int j, float2 v0, float2 v1) {
    *reinterpret_cast<float4*>(tile + j * tile_stride) = make_float4(v0.x, v0.y, v1.x, v1.y);
    if (bin == 0) gsh[j] = a.c.degrid * v0.x / gs0;  // the sharpen pass's grid fraction: the filtered DC
  };
  if constexpr (MODE == MODE_KALMAN) {
    float4 lv;
    float2 cv, cp;
    asm("ld.global.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(lv.x), "=f"(lv.y), "=f"(lv.z), "=f"(lv.w) : "l"(a.kal_last + off + bin));
    asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(cv.x), "=f"(cv.y) : "l"(a.kal_covar + off + bin));
    asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(cp.x), "=f"(cp.y) : "l"(a.kal_covarp + off + bin));
    float2 l0 = make_float2(lv.x, lv.y), l1 = make_float2(lv.z, lv.w);
    float s0 = a.c.sigma2n_2d, s1 = a.c.sigma2n_2d;
    if (a.c.pattern) {
      s0 = fmaxf(__ldg(a.t.pattern2d + bin), 1e-15f);
      s1 = fmaxf(__ldg(a.t.pattern2d + bin + 1), 1e-15f);
    }
    float4 nxt = group_load(a, ts, 2, off, bin);
    for (int j = 0; j < count; j++) {
      const float4 c = nxt;
      if (j + 1 < count) nxt = group_load(a, ts, j + 3, off, bin);
      kalman_step(a, make_float2(c.x, c.y), s0, l0, cv.x, cp.x);
      kalman_step(a, make_float2(c.z, c.w), s1, l1, cv.y, cp.y);
      out(j, l0, l1);
    }
    *reinterpret_cast<float4*>(a.kal_last + off + bin) = make_float4(l0.x, l0.y, l1.x, l1.y);
    *reinterpret_cast<float2*>(a.kal_covar + off + bin) = cv;
    *reinterpret_cast<float2*>(a.kal_covarp + off + bin) = cp;
  } else if constexpr (MODE == MODE_SHARPEN_ONLY) {
    for (int j = 0; j < count; j++) {
      const float4 c = group_load(a, ts, j + 2, off, bin);
      out(j, make_float2(c.x, c.y), make_float2(c.z, c.w));
    }
  } else {
    const BinTab tb0 = bin_tab<MODE>(a, bin), tb1 = bin_tab<MODE>(a, bin + 1);
    // spectrum s (frame n0 - 2 + s) lives in r[s % NW]; frame j reads
    // s = j + LO .. j + HI; with j = j0 + u and j0 a multiple of NW every
    // index below is a compile-time constant
    float4 r[NW];
#pragma unroll
    for (int k = 0; k < NW - 1; k++) r[(LO + k) % NW] = group_load(a, ts, LO + k, off, bin);
    float4 nxt = group_load(a, ts, HI, off, bin);
    for (int j0 = 0; j0 < count; j0 += NW) {
#pragma unroll
      for (int u = 0; u < NW; u++) {
        const int j = j0 + u;
        if (j < count) {
          r[(u + HI) % NW] = nxt;
          if (j + 1 < count) nxt = group_load(a, ts, j + 1 + HI, off, bin);
          float2 w0[5], w1[5];
#pragma unroll
          for (int k = 0; k < 5; k++) {
            const bool in = k >= LO && k <= HI;
            const float4 v = r[(u + (in ? k : LO)) % NW];
            w0[k] = in ? make_float2(v.x, v.y) : make_float2(0.f, 0.f);
            w1[k] = in ? make_float2(v.z, v.w) : make_float2(0.f, 0.f);
          }
          const float gf = gfs[j];
          out(j, filter_vals<MODE>(a, w0, off, bin, gf, tb0, false), filter_vals<MODE>(a, w1, off, bin + 1, gf, tb1, false));
        }
      }
    }
  }
}

// One frame of one bin pair (the tail of the filter stage, spread over all
// threads): the pair's window for frame j loaded directly. Wiener modes.
template <int MODE>
__device__ __forceinline__ void group_filter_one(const InverseArgs& a, const TemporalSet& ts, size_t off, int bin, int j,
                                                 const float* gfs, float* gsh, float gs0, float2* tile) {
  constexpr int LO = win_lo<MODE>(), HI = win_hi<MODE>();
  float4 r[5];
#pragma unroll
  for (int k = LO; k <= HI; k++) r[k] = group_load(a, ts, j + k, off, bin);
  float2 w0[5], w1[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const bool in = k >= LO && k <= HI;
    w0[k] = in ? make_float2(r[k].x, r[k].y) : make_float2(0.f, 0.f);
    w1[k] = in ? make_float2(r[k].z, r[k].w) : make_float2(0.f, 0.f);
  }
  float2 v0, v1;
  if constexpr (MODE == MODE_SHARPEN_ONLY) {
    v0 = w0[2];
    v1 = w1[2];
  } else {
    v0 = filter_vals<MODE>(a, w0, off, bin, gfs[j], bin_tab<MODE>(a, bin), false);
    v1 = filter_vals<MODE>(a, w1, off, bin + 1, gfs[j], bin_tab<MODE>(a, bin + 1), false);
  }
  *reinterpret_cast<float4*>(tile) = make_float4(v0.x, v0.y, v1.x, v1.y);
  if (bin == 0) gsh[j] = a.c.degrid * v0.x / gs0;
}

// The overlap-add of output tile (tx, ty) (OlaFuse) for the run's frames:
// overlap_add_px4 / overlap_add_px per pixel, the blocks read from L2.
template <typename T>
__device__ __noinline__ void group_ola_tile(const OlaFuse& of, const TemporalSet& ts, int count, int tx, int ty) {
  const Geom& g = of.o.g;
  const int x_lo = (tx - 1) * g.sx, y_lo = (ty - 1) * g.sy;
  const int wd = min(g.sx, g.W - x_lo), ht = min(g.sy, g.H - y_lo);
  if (of.px4) {
    // quads (frame j, row yy, quad xx); each thread fetches K of them before
    // it finishes any, so that their L2 reads overlap
    constexpr int K = 2;
    const int q = (wd + 3) / 4, per = q * ht, total = count * per;
    for (int i0 = threadIdx.x; i0 < total; i0 += K * blockDim.x) {
      Ola4Px p[K];
      int jj[K], xs[K], ks[K];
#pragma unroll
      for (int u = 0; u < K; u++) {
        const int i = i0 + u * blockDim.x;
        const int j = i < total ? i / per : 0, r = i - j * per, yy = r / q, xx = r - yy * q;
        jj[u] = j;
        xs[u] = i < total ? x_lo + 4 * xx : g.W;  // out of range: fetch and finish skip it
        ks[u] = y_lo + yy;
        p[u] = ola4_fetch<true>(of.o, ts.tdom[j], xs[u], ks[u]);
      }
#pragma unroll
      for (int u = 0; u < K; u++) ola4_finish<T>(of.o, of.dst[jj[u]], of.dst_stride[jj[u]], xs[u], ks[u], p[u]);
    }
    return;
  }
  const int per = wd * ht;
  for (int i = threadIdx.x; i < count * per; i += blockDim.x) {
    const int j = i / per, r = i - j * per, yy = r / wd, xx = r - yy * wd;
    OlaArgs b = of.o;
    b.tdom = ts.tdom[j];
    b.dst = of.dst[j];
    b.dst_stride = of.dst_stride[j];
    overlap_add_px<T, true>(b, x_lo + xx, y_lo + yy);
  }
}

template <int BW, int BH, int MODE>
__device__ __forceinline__ void filter_inverse_group_cta(const InverseArgs& a, const TemporalSet& ts, int blk,
                                                         const OlaFuse* of = nullptr) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2, BINS = BH * NH, PAIRS = BINS / 2, NT = kWarps * 32;
  static_assert(BINS % 2 == 0, "bin pairs");
  extern __shared__ float2 smem2[];
  float* gfs = reinterpret_cast<float*>(smem2);  // grid fraction of each frame's block
  float* gsh = gfs + kGroupTile;                 // ... and of its filtered block (sharpen pass)
  float2* S = smem2 + kGroupTile;                // [count][BINS] tiles, 16-byte aligned
  const int count = ts.count;
  const size_t off = (size_t)blk * BINS;
  const float gs0 = __ldg(&a.t.grid[0].x);
  const int t = threadIdx.x;
  // 0. grid fraction of each frame's block (its DC)
  if (MODE >= 1 && t < count)
    gfs[t] = FFT3D_IN(ts.spec[t + 2] != nullptr && blk < a.g.nblocks, a.err)
                 ? a.c.degrid * __ldg(&ts.spec[t + 2][off].x) / gs0 : 0.f;
  __syncthreads();
  // 1. filter: whole rounds of bin pairs over all frames; the remaining pairs
  //    (a partial round) as (pair, frame) items spread over every thread,
  //    except for Kalman, whose frames follow one another
  constexpr int FULL = (PAIRS / NT) * NT;
  for (int p = t; p < FULL; p += NT)
    group_filter_pair<MODE>(a, ts, off, 2 * p, count, gfs, gsh, gs0, S + 2 * p, BINS);
  if constexpr (MODE == MODE_KALMAN) {
    for (int p = FULL + t; p < PAIRS; p += NT)
      group_filter_pair<MODE>(a, ts, off, 2 * p, count, gfs, gsh, gs0, S + 2 * p, BINS);
  } else {
    for (int i = t; i < (PAIRS - FULL) * count; i += NT) {
      const int q = div_small(i, count), j = i - q * count, p = FULL + q;
      group_filter_one<MODE>(a, ts, off, 2 * p, j, gfs, gsh, gs0, S + j * BINS + 2 * p);
    }
  }
  __syncthreads();
  // 2. the separate sharpen/dehalo pass (src/code_impl/Sharpen.cpp:13-63),
  //    its grid fraction from each tile's filtered DC (published by the
  //    filter stage); whole rounds of bin pairs with the pair's tables loaded
  //    once for all frames, then the remaining pairs as (pair, frame) items
  //    spread over every thread (as the filter stage does)
  if (a.c.do_sharpen) {
    auto tabs = [&](int bin, BinTab& tb0, BinTab& tb1) {
      tb0 = BinTab{make_float2(0.f, 0.f), 0.f, 0.f};
      tb1 = tb0;
      if (a.c.degrid != 0.f) {
        const float4 g = __ldg(reinterpret_cast<const float4*>(a.t.grid + bin));
        tb0.grid = make_float2(g.x, g.y);
        tb1.grid = make_float2(g.z, g.w);
      }
      if (a.c.use_sharpen) {
        tb0.wsh = __ldg(a.t.wsharpen + bin);
        tb1.wsh = __ldg(a.t.wsharpen + bin + 1);
      }
      if (a.c.use_dehalo) {
        tb0.wdh = __ldg(a.t.wdehalo + bin);
        tb1.wdh = __ldg(a.t.wdehalo + bin + 1);
      }
    };
    auto one = [&](int bin, int j, const BinTab& tb0, const BinTab& tb1) {
      float4* q = reinterpret_cast<float4*>(S + j * BINS + bin);
      const float4 v = *q;
      const float2 v0 = sharpen_bin(a, make_float2(v.x, v.y), tb0, gsh[j]);
      const float2 v1 = sharpen_bin(a, make_float2(v.z, v.w), tb1, gsh[j]);
      *q = make_float4(v0.x, v0.y, v1.x, v1.y);
    };
    for (int p = t; p < FULL; p += NT) {
      BinTab tb0, tb1;
      tabs(2 * p, tb0, tb1);
      for (int j = 0; j < count; j++) one(2 * p, j, tb0, tb1);
    }
    for (int i = t; i < (PAIRS - FULL) * count; i += NT) {
      const int q = div_small(i, count), j = i - q * count;
      BinTab tb0, tb1;
      tabs(2 * (FULL + q), tb0, tb1);
      one(2 * (FULL + q), j, tb0, tb1);
    }
    __syncthreads();
  }
  // 3. inverse column DFTs
  for (int i = t; i < count * HC; i += NT) {
    const int j = i / HC;
    inv_col<BW, BH>(S + j * BINS, i - j * HC);
  }
  __syncthreads();
  // 4. c2r rows, in place
  for (int i = t; i < count * BH; i += NT) {
    const int j = i / BH;
    inv_row_inplace<BW, BH>(S + j * BINS, i - j * BH);
  }
  __syncthreads();
  // 5. time-domain blocks (rows of BW floats, left in the tiles with a pitch of NH complex)
  constexpr int HALF = BW / 2;
  for (int i = t; i < count * BH * HALF; i += NT) {
    const int j = i / (BH * HALF), r = i - j * (BH * HALF);
    const int y = r / HALF, x = r - y * HALF;
    if (FFT3D_IN(ts.tdom[j] != nullptr && blk < a.g.nblocks, a.err))
      reinterpret_cast<float2*>(ts.tdom[j] + (size_t)blk * BH * BW)[r] = S[j * BINS + y * NH + x];
  }
  // 6. the overlap-adds of the output tiles whose last block this is (OlaFuse):
  //    release (a barrier after the stores, then a fence before each tile
  //    arrival), acquire (a fence after the arrival that completes a tile,
  //    then a barrier); no waiting
  if (of) {
    __shared__ int done[4];
    __syncthreads();  // the CTA's stores precede the arrivals below (the fence there is cumulative)
    const int bx = blk % a.g.nox, by = blk / a.g.nox;
    if (t < 4) {
      const int dx = t & 1, dy = t >> 1, tx = bx + dx, ty = by + dy;
      const unsigned need = (a.g.ow > 0 ? 2u : 1u) * (a.g.oh > 0 ? 2u : 1u);
      int last = 0;
      if ((dx == 0 || a.g.ow > 0) && (dy == 0 || a.g.oh > 0) && tx >= 1 && tx <= of->tiles_x && ty >= 1 &&
          ty <= of->tiles_y && FFT3D_IN(tx < a.g.nox && ty < a.g.noy, a.err)) {
        __threadfence();
        last = atomicAdd(of->cnt + ty * a.g.nox + tx, 1u) + 1u == need * of->epoch;
        if (last) __threadfence();
      }
      done[t] = last;
    }
    __syncthreads();
    for (int q = 0; q < 4; q++) {
      if (!done[q]) continue;
      const int tx = bx + (q & 1), ty = by + (q >> 1);
      if (of->bytes == 1) group_ola_tile<uint8_t>(*of, ts, count, tx, ty);
      else if (of->bytes == 2) group_ola_tile<uint16_t>(*of, ts, count, tx, ty);
      else group_ola_tile<float>(*of, ts, count, tx, ty);
    }
  }
}

template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32,
                                  ctas_for(FFT3D_GROUP_CTAS, group_smem_bytes<BW, BH>(group_run_frames(BW, BH))))
    k_filter_inverse_group(InverseArgs a,
                                                                     const __grid_constant__ TemporalSet ts,
                                                                     const __grid_constant__ OlaFuse of) {
  filter_inverse_group_cta<BW, BH, MODE>(a, ts, blockIdx.x, of.cnt ? &of : nullptr);
}

// Batched runs of many planes: work item (run, block of that run's plane). The
// run's arguments are staged in shared memory behind the tiles, so the body's
// stores cannot alias them (a reference into global memory would be reloaded
// after every store) and they cost no registers.
template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32,
                                  ctas_for(FFT3D_GROUP_CTAS,
                                           group_smem_bytes<BW, BH>(group_run_frames(BW, BH)) + (int)sizeof(GroupRun)))
    k_filter_inverse_group_batch(const GroupRun* __restrict__ runs,
                                                                           const int2* __restrict__ items,
                                                                           int nitems) {
  extern __shared__ float2 smem2[];
  GroupRun* sr = reinterpret_cast<GroupRun*>(smem2 + kGroupTile + group_run_frames(BW, BH) * BH * (BW / 2 + 1));
  static_assert(sizeof(GroupRun) % 4 == 0, "word copy");
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    __syncthreads();  // every thread is done with the previous item's arguments and tiles
    const int* src = reinterpret_cast<const int*>(runs + it.x);
    int* dst = reinterpret_cast<int*>(sr);
    for (int w = threadIdx.x; w < (int)(sizeof(GroupRun) / 4); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    filter_inverse_group_cta<BW, BH, MODE>(sr->a, sr->ts, it.y);
  }
}

// ---------------------------------------------------------------- inverse (bulk-staged)

constexpr int kBulkWarps = 4;
constexpr int kBulkSpin = 1 << 22;  // bounded mbarrier wait (then error flag 2)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool bulk_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done = 0;
  for (int it = 0; it < kBulkSpin && !done; it++)
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
  return done != 0;
}

template <int BW, int BH, int MODE>
__host__ __device__ constexpr int bulk_warp_bytes() {
  return (win_hi<MODE>() - win_lo<MODE>() + 2) * BH * (BW / 2 + 1) * 8;
}

// Filter + inverse with the window's spectra fetched by bulk copies: each
// warp walks its blocks (block = warp index + k * all warps, or mirrored for
// the reverse order) with a stage holding the block's window spectra (one
// contiguous BH x NH run per frame, one cp.async.bulk each, completing on
// the warp's mbarrier). The filter reads the stage and writes the block's
// filtered spectrum to S; lane 0 then refills the stage with the next
// block's spectra, which land while the warp runs the inverse transform of S
// and stores the time-domain block. Wiener and sharpen-only modes.
template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kBulkWarps * 32) k_filter_inverse_bulk(InverseArgs a) {
  constexpr int NH = BW / 2 + 1, HC = BW / 2, BINS = BH * NH, PER = (BINS + 31) / 32;
  constexpr int LO = win_lo<MODE>(), NW = win_hi<MODE>() - win_lo<MODE>() + 1;
  constexpr uint32_t SPEC_BYTES = BINS * 8;
  static_assert(SPEC_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* stage = reinterpret_cast<float2*>(smem_raw + 128 + (size_t)warp * bulk_warp_bytes<BW, BH, MODE>());
  float2* S = stage + NW * BINS;
  uint64_t* bar = bars + warp;
  const Geom& g = a.g;
  const int nwarps = gridDim.x * kBulkWarps;
  const int first = blockIdx.x * kBulkWarps + warp;
  if (first >= g.nblocks) return;
  auto block_of = [&](int idx) { return a.reverse ? g.nblocks - 1 - idx : idx; };
  auto fetch = [&](int blk) {  // lane 0
    const size_t off = (size_t)blk * BINS;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(NW * SPEC_BYTES)
                 : "memory");
#pragma unroll
    for (int k = 0; k < NW; k++)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(stage + k * BINS)),
          "l"(a.in[LO + k] + off), "r"(SPEC_BYTES), "r"(smem_addr(bar))
          : "memory");
  };
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fetch(block_of(first));
  }
  __syncwarp();
  const float gs0 = __ldg(&a.t.grid[0].x);
  uint32_t phase = 0;
  for (int idx = first; idx < g.nblocks; idx += nwarps) {
    const int blk = block_of(idx);
    if (!__all_sync(0xffffffffu, bulk_wait(bar, phase))) {
      // the copies never completed: flag it, give them one more bounded wait
      // (they target this warp's shared memory), and stop
      if (lane == 0) atomicOr(a.err, 2);
      bulk_wait(bar, phase);
      return;
    }
    phase ^= 1;
    const size_t off = (size_t)blk * BINS;
    const float gf = (MODE >= 1) ? a.c.degrid * stage[(2 - LO) * BINS].x / gs0 : 0.f;
    float gsh = 0.f;
#pragma unroll 1
    for (int j = 0; j < PER; j++) {
      const int i = lane + 32 * j;
      float2 v = make_float2(0.f, 0.f);
      BinTab tb{make_float2(0.f, 0.f), 0.f, 0.f};
      if (i < BINS) {
        tb = bin_tab<MODE>(a, i);
        float2 w[5];
#pragma unroll
        for (int k = 0; k < 5; k++)
          w[k] = (k >= LO && k < LO + NW) ? stage[(k - LO) * BINS + i] : make_float2(0.f, 0.f);
        v = filter_vals<MODE>(a, w, off, i, gf, tb, true);
      }
      if (a.c.do_sharpen) {
        if (j == 0) gsh = a.c.degrid * __shfl_sync(0xffffffffu, v.x, 0) / gs0;
        if (i < BINS) v = sharpen_bin(a, v, tb, gsh);
      }
      if (i < BINS) S[i] = v;
    }
    __syncwarp();
    if (lane == 0 && idx + nwarps < g.nblocks) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      fetch(block_of(idx + nwarps));
    }
    for (int c = lane; c < HC; c += 32) inv_col<BW, BH>(S, c);
    __syncwarp();
    for (int y = lane; y < BH; y += 32) inv_row_inplace<BW, BH>(S, y);
    __syncwarp();
    store_tdom<BW, BH>(S, a.tdom + (size_t)blk * BH * BW, lane);
    __syncwarp();
  }
}

// ---------------------------------------------------------------- fused

// Steady-state hot path of one output frame in one launch: each warp
// transforms the window's newest frame for its blocks (forward_cta: the
// spectra go to the ring for the next output frames and stay in the warp's
// shared memory), then filters and inverse-transforms them
// (filter_inverse_cta) with the older frames' spectra streamed from the ring
// through the same register load pipeline as k_filter_inverse.
template <int BW, int BH, typename T, int MODE>
__global__ void __launch_bounds__(kWarps * 32, 6) k_fused(FusedArgs A) {
  const int n = fft_ctas<BW, BH>(A.v.g.nblocks);
  forward_cta<BW, BH, T, false>(A.f, A.v.reverse ? n - 1 - (int)blockIdx.x : (int)blockIdx.x);
  filter_inverse_cta<BW, BH, MODE, true>(A.v, blockIdx.x);
}

// ---------------------------------------------------------------- launchers

template <int BW, int BH>
int fft_grid(int nblocks) {
  return fft_ctas<BW, BH>(nblocks);
}

// Batched launches of one kernel variant over many planes (see k_forward_batch).
template <int BW, int BH>
cudaError_t fwd_batch(const BatchLaunch& l, int bytes, cudaStream_t s) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  const auto* args = static_cast<const ForwardArgs*>(l.args);
  cudaError_t e = cudaSuccess;
  if (bytes == 1) {
    e = fft3d::smem_attr(k_forward_batch<BW, BH, uint8_t>, smem);
    if (e == cudaSuccess) k_forward_batch<BW, BH, uint8_t><<<l.grid, kWarps * 32, smem, s>>>(args, l.items, l.nitems);
  } else if (bytes == 2) {
    e = fft3d::smem_attr(k_forward_batch<BW, BH, uint16_t>, smem);
    if (e == cudaSuccess) k_forward_batch<BW, BH, uint16_t><<<l.grid, kWarps * 32, smem, s>>>(args, l.items, l.nitems);
  } else {
    e = fft3d::smem_attr(k_forward_batch<BW, BH, float>, smem);
    if (e == cudaSuccess) k_forward_batch<BW, BH, float><<<l.grid, kWarps * 32, smem, s>>>(args, l.items, l.nitems);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BW, int BH, int MODE>
cudaError_t inv_batch_mode(const BatchLaunch& l, cudaStream_t s) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  cudaError_t e = fft3d::smem_attr(k_filter_inverse_batch<BW, BH, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse_batch<BW, BH, MODE><<<l.grid, kWarps * 32, smem, s>>>(static_cast<const InverseArgs*>(l.args),
                                                                         l.items, l.nitems);
  return cudaGetLastError();
}

template <int BW, int BH>
cudaError_t inv_batch(const BatchLaunch& l, int mode, cudaStream_t s) {
  switch (mode) {
    case MODE_SHARPEN_ONLY: return inv_batch_mode<BW, BH, MODE_SHARPEN_ONLY>(l, s);
    case MODE_KALMAN: return inv_batch_mode<BW, BH, MODE_KALMAN>(l, s);
    case 1: return inv_batch_mode<BW, BH, 1>(l, s);
    case 2: return inv_batch_mode<BW, BH, 2>(l, s);
    case 3: return inv_batch_mode<BW, BH, 3>(l, s);
    case 4: return inv_batch_mode<BW, BH, 4>(l, s);
    case 5: return inv_batch_mode<BW, BH, 5>(l, s);
  }
  return cudaErrorInvalidValue;
}

// CTAs of one plane's unbatched launch (the work items per plane of a batch)
template <int BW, int BH>
int ctas_per_plane(int nblocks) {
  return fft_ctas<BW, BH>(nblocks);
}

// Occupancy (resident CTAs per SM) of the batched kernels.
template <int BW, int BH>
int occupancy_of(int which, int mode_or_bytes) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  int n = 0;
  if (which == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_forward_batch<BW, BH, uint8_t>, kWarps * 32, smem);
  } else if (which == 3) {
    const int gsmem = group_smem_bytes<BW, BH>(group_run_frames(BW, BH)) + (int)sizeof(GroupRun);
    fft3d::smem_attr(k_filter_inverse_group_batch<BW, BH, 5>, gsmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_filter_inverse_group_batch<BW, BH, 5>, kWarps * 32, gsmem);
  } else {
    switch (mode_or_bytes) {
      case MODE_KALMAN:
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_filter_inverse_batch<BW, BH, MODE_KALMAN>, kWarps * 32, smem);
        break;
      case 5:
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_filter_inverse_batch<BW, BH, 5>, kWarps * 32, smem);
        break;
      default:
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_filter_inverse_batch<BW, BH, 3>, kWarps * 32, smem);
    }
  }
  return n > 0 ? n : 1;
}

template <int BW, int BH>
cudaError_t fwd_sized(const ForwardArgs& a, int bytes, cudaStream_t s) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  const int grid = fft_grid<BW, BH>(a.g.nblocks);
  cudaError_t e = cudaSuccess;
  if (bytes == 1) {
    e = fft3d::smem_attr(k_forward<BW, BH, uint8_t>, smem);
    if (e == cudaSuccess) k_forward<BW, BH, uint8_t><<<grid, kWarps * 32, smem, s>>>(a);
  } else if (bytes == 2) {
    e = fft3d::smem_attr(k_forward<BW, BH, uint16_t>, smem);
    if (e == cudaSuccess) k_forward<BW, BH, uint16_t><<<grid, kWarps * 32, smem, s>>>(a);
  } else {
    e = fft3d::smem_attr(k_forward<BW, BH, float>, smem);
    if (e == cudaSuccess) k_forward<BW, BH, float><<<grid, kWarps * 32, smem, s>>>(a);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BW, int BH, int MODE>
cudaError_t inv_mode(const InverseArgs& a, cudaStream_t s) {
  constexpr int bulk_smem = 128 + kBulkWarps * bulk_warp_bytes<BW, BH, MODE>();
  if (MODE != MODE_KALMAN && a.bulk && a.err && bulk_smem <= 160 * 1024) {
    cudaError_t e = fft3d::smem_attr(k_filter_inverse_bulk<BW, BH, MODE>, bulk_smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_filter_inverse_bulk<BW, BH, MODE>, kBulkWarps * 32,
                                                  bulk_smem);
    const int need = (a.g.nblocks + kBulkWarps - 1) / kBulkWarps;
    const int grid = std::min(need, std::max(1, per_sm) * sms);
    k_filter_inverse_bulk<BW, BH, MODE><<<grid, kBulkWarps * 32, bulk_smem, s>>>(a);
    return cudaGetLastError();
  }
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  const int grid = fft_grid<BW, BH>(a.g.nblocks);
  cudaError_t e =
      fft3d::smem_attr(k_filter_inverse<BW, BH, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse<BW, BH, MODE><<<grid, kWarps * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <int BW, int BH, typename T, int MODE>
cudaError_t fused_mode(const FusedArgs& a, cudaStream_t s) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  const int grid = fft_ctas<BW, BH>(a.v.g.nblocks);
  cudaError_t e =
      fft3d::smem_attr(k_fused<BW, BH, T, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_fused<BW, BH, T, MODE><<<grid, kWarps * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <int BW, int BH, typename T>
cudaError_t fused_typed(const FusedArgs& a, int mode, cudaStream_t s) {
  switch (mode) {
    case MODE_SHARPEN_ONLY: return fused_mode<BW, BH, T, MODE_SHARPEN_ONLY>(a, s);
    case MODE_KALMAN: return fused_mode<BW, BH, T, MODE_KALMAN>(a, s);
    case 1: return fused_mode<BW, BH, T, 1>(a, s);
    case 2: return fused_mode<BW, BH, T, 2>(a, s);
    case 3: return fused_mode<BW, BH, T, 3>(a, s);
    case 4: return fused_mode<BW, BH, T, 4>(a, s);
    case 5: return fused_mode<BW, BH, T, 5>(a, s);
  }
  return cudaErrorInvalidValue;
}

template <int BW, int BH>
cudaError_t fused_sized(const FusedArgs& a, int mode, int bytes, cudaStream_t s) {
  if (bytes == 1) return fused_typed<BW, BH, uint8_t>(a, mode, s);
  if (bytes == 2) return fused_typed<BW, BH, uint16_t>(a, mode, s);
  return cudaErrorNotSupported;  // float samples use the unfused path
}

template <int BW, int BH>
cudaError_t fwd_frames(const ForwardArgs& a, const FwdFrameSet& fs, int bytes, cudaStream_t s) {
  if (fs.count < 1 || fs.count > kMaxFwdFrames) return cudaErrorInvalidValue;
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  FwdFrameSet f = fs;
  f.ctas = fft_grid<BW, BH>(a.g.nblocks);
  const int grid = f.ctas * f.count;
  cudaError_t e = cudaSuccess;
  if (bytes == 1) {
    e = fft3d::smem_attr(k_forward_frames<BW, BH, uint8_t>, smem);
    if (e == cudaSuccess) k_forward_frames<BW, BH, uint8_t><<<grid, kWarps * 32, smem, s>>>(a, f);
  } else if (bytes == 2) {
    e = fft3d::smem_attr(k_forward_frames<BW, BH, uint16_t>, smem);
    if (e == cudaSuccess) k_forward_frames<BW, BH, uint16_t><<<grid, kWarps * 32, smem, s>>>(a, f);
  } else {
    e = fft3d::smem_attr(k_forward_frames<BW, BH, float>, smem);
    if (e == cudaSuccess) k_forward_frames<BW, BH, float><<<grid, kWarps * 32, smem, s>>>(a, f);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BW, int BH, int MODE>
cudaError_t inv_frames_mode(const InverseArgs& a, const FrameSet& fs, cudaStream_t s) {
  const int smem = kWarps * fft_smem_bytes<BW, BH>();
  const int grid = fft_grid<BW, BH>(a.g.nblocks) * fs.count;
  cudaError_t e = fft3d::smem_attr(k_filter_inverse_frames<BW, BH, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse_frames<BW, BH, MODE><<<grid, kWarps * 32, smem, s>>>(a, fs);
  return cudaGetLastError();
}

// frame groups: Wiener 3D windows (the modes whose frames share spectra)
template <int BW, int BH>
cudaError_t inv_frames(const InverseArgs& a, const FrameSet& fs, int mode, cudaStream_t s) {
  if (fs.count < 1 || fs.count > kMaxGroupFrames) return cudaErrorInvalidValue;
  switch (mode) {
    case MODE_SHARPEN_ONLY: return inv_frames_mode<BW, BH, MODE_SHARPEN_ONLY>(a, fs, s);
    case 2: return inv_frames_mode<BW, BH, 2>(a, fs, s);
    case 3: return inv_frames_mode<BW, BH, 3>(a, fs, s);
    case 4: return inv_frames_mode<BW, BH, 4>(a, fs, s);
    case 5: return inv_frames_mode<BW, BH, 5>(a, fs, s);
  }
  return cudaErrorInvalidValue;
}

template <int BW, int BH, int MODE>
cudaError_t inv_group_mode(const InverseArgs& a, const TemporalSet& ts, const OlaFuse& of, cudaStream_t s) {
  const int smem = group_smem_bytes<BW, BH>(kGroupTile);
  cudaError_t e = fft3d::smem_attr(k_filter_inverse_group<BW, BH, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse_group<BW, BH, MODE>
      <<<a.g.nblocks, kWarps * 32, group_smem_bytes<BW, BH>(ts.count), s>>>(a, ts, of);
  return cudaGetLastError();
}

template <int BW, int BH>
cudaError_t inv_group(const InverseArgs& a, const TemporalSet& ts, int mode, cudaStream_t s, const OlaFuse* ofp) {
  if (ts.count < 1 || ts.count > group_run_frames(BW, BH)) return cudaErrorInvalidValue;
  OlaFuse of{};
  if (ofp) {
    of = *ofp;
    if (!of.cnt || of.epoch == 0 || of.tiles_x < 1 || of.tiles_y < 1 || of.tiles_x >= a.g.nox ||
        of.tiles_y >= a.g.noy || (of.bytes != 1 && of.bytes != 2 && of.bytes != 4))
      return cudaErrorInvalidValue;
  }
  switch (mode) {
    case MODE_SHARPEN_ONLY: return inv_group_mode<BW, BH, MODE_SHARPEN_ONLY>(a, ts, of, s);
    case MODE_KALMAN: return inv_group_mode<BW, BH, MODE_KALMAN>(a, ts, of, s);
    case 1: return inv_group_mode<BW, BH, 1>(a, ts, of, s);
    case 2: return inv_group_mode<BW, BH, 2>(a, ts, of, s);
    case 3: return inv_group_mode<BW, BH, 3>(a, ts, of, s);
    case 4: return inv_group_mode<BW, BH, 4>(a, ts, of, s);
    case 5: return inv_group_mode<BW, BH, 5>(a, ts, of, s);
  }
  return cudaErrorInvalidValue;
}

template <int BW, int BH, int MODE>
cudaError_t inv_group_batch_mode(const BatchLaunch& l, cudaStream_t s) {
  const int smem = group_smem_bytes<BW, BH>(group_run_frames(BW, BH)) + (int)sizeof(GroupRun);
  cudaError_t e = fft3d::smem_attr(k_filter_inverse_group_batch<BW, BH, MODE>, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse_group_batch<BW, BH, MODE><<<l.grid, kWarps * 32, smem, s>>>(static_cast<const GroupRun*>(l.args),
                                                                             l.items, l.nitems);
  return cudaGetLastError();
}

template <int BW, int BH>
cudaError_t inv_group_batch(const BatchLaunch& l, int mode, cudaStream_t s) {
  switch (mode) {
    case MODE_SHARPEN_ONLY: return inv_group_batch_mode<BW, BH, MODE_SHARPEN_ONLY>(l, s);
    case MODE_KALMAN: return inv_group_batch_mode<BW, BH, MODE_KALMAN>(l, s);
    case 1: return inv_group_batch_mode<BW, BH, 1>(l, s);
    case 2: return inv_group_batch_mode<BW, BH, 2>(l, s);
    case 3: return inv_group_batch_mode<BW, BH, 3>(l, s);
    case 4: return inv_group_batch_mode<BW, BH, 4>(l, s);
    case 5: return inv_group_batch_mode<BW, BH, 5>(l, s);
  }
  return cudaErrorInvalidValue;
}

template <int BW, int BH>
cudaError_t inv_sized(const InverseArgs& a, int mode, cudaStream_t s) {
  switch (mode) {
    case MODE_SHARPEN_ONLY: return inv_mode<BW, BH, MODE_SHARPEN_ONLY>(a, s);
    case MODE_KALMAN: return inv_mode<BW, BH, MODE_KALMAN>(a, s);
    case 1: return inv_mode<BW, BH, 1>(a, s);
    case 2: return inv_mode<BW, BH, 2>(a, s);
    case 3: return inv_mode<BW, BH, 3>(a, s);
    case 4: return inv_mode<BW, BH, 4>(a, s);
    case 5: return inv_mode<BW, BH, 5>(a, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

// Registers block size BW x BH of this translation unit in the size table.
#define FFT3D_REGISTER_SIZE(BW, BH)                                                                     \
  static const bool fft3d_reg_##BW##x##BH = register_size(                                             \
      SizeEntry{BW, BH, &fwd_sized<BW, BH>, &inv_sized<BW, BH>, &fused_sized<BW, BH>, &upload_twiddle_table, \
                &fwd_batch<BW, BH>, &inv_batch<BW, BH>, &ctas_per_plane<BW, BH>, &occupancy_of<BW, BH>,      \
                &inv_frames<BW, BH>, &fwd_frames<BW, BH>, &inv_group<BW, BH>, &inv_group_batch<BW, BH>});

}  // namespace fft3d
