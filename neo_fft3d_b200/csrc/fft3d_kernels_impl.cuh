// Kernel templates of the FFT3D filtering core (FP32 CUDA-core path).
// Included by the per-size translation units kern_*.cu, which instantiate the
// block sizes they own and register them in the size table (kern_registry.h).
#pragma once
#include <cmath>

#include "fft3d_kernels.cuh"
#include "kern_registry.h"
#include "regfft.cuh"

namespace fft3d {
namespace {

constexpr int kWarps = 4;  // warps (= blocks in flight) per CTA in the FFT kernels

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

template <typename T>
__device__ __forceinline__ float load_sample(const T* p) { return (float)p[0]; }
template <>
__device__ __forceinline__ float load_sample<uint8_t>(const uint8_t* p) { return (float)(int)__ldg(p); }
template <>
__device__ __forceinline__ float load_sample<uint16_t>(const uint16_t* p) { return (float)(int)__ldg(p); }
template <>
__device__ __forceinline__ float load_sample<float>(const float* p) { return __ldg(p); }

template <int BW, int BH>
__host__ __device__ constexpr int fft_smem_floats() {
  return BH * (BW + 1) + BH * (BW / 2 + 1) * 2;
}

// ---------------------------------------------------------------- forward

template <int BW, int BH, typename T>
__global__ void __launch_bounds__(kWarps * 32) k_forward(ForwardArgs a) {
  constexpr int NH = BW / 2 + 1, TP = BW + 1;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tile = smem + warp * fft_smem_floats<BW, BH>();
  float2* S = reinterpret_cast<float2*>(tile + BH * TP);
  const Geom& g = a.g;
  const int blk = blockIdx.x * kWarps + warp;
  if (blk >= g.nblocks) return;
  const int by = blk / g.nox, bx = blk - by * g.nox;
  // 1. windowed block tile (coalesced along x)
  for (int y = 0; y < BH; y++) {
    const int k = reflect101(by * g.sy + y - g.sy, g.H);
    const T* srow = reinterpret_cast<const T*>(static_cast<const char*>(a.src) +
                                               (long long)field_row(k, g.H, g.interlaced) * a.src_stride);
    const float wy = __ldg(a.wan_y + y);
    for (int x = lane; x < BW; x += 32) {
      const int c = reflect101(bx * g.sx + x - g.sx, g.W);
      const float v = load_sample<T>(srow + c) - a.base;
      tile[y * TP + x] = v * __ldg(a.wan_x + x) * wy;
    }
  }
  __syncwarp();
  // 2. r2c along x, one row per lane
  for (int y = lane; y < BH; y += 32) {
    float r[BW];
#pragma unroll
    for (int x = 0; x < BW; x++) r[x] = tile[y * TP + x];
    float2 c[NH];
    rfft<BW>(r, c);
#pragma unroll
    for (int k = 0; k < NH; k++) S[y * NH + k] = c[k];
  }
  __syncwarp();
  // 3. complex DFT along y, one column per lane; rows of the output are
  //    written by consecutive lanes (coalesced)
  float2* out = a.spec + (size_t)blk * BH * NH;
  for (int k = lane; k < NH; k += 32) {
    float2 col[BH];
#pragma unroll
    for (int y = 0; y < BH; y++) col[y] = S[y * NH + k];
    cfft<BH, -1>(col);
#pragma unroll
    for (int h = 0; h < BH; h++) out[h * NH + k] = col[h];
  }
}

// ---------------------------------------------------------------- filters

__device__ __forceinline__ float sharpen_fact(const InverseArgs& a, float psd, int bin) {
  // src/code_impl/Apply.cpp:129-131
  return 1.f + a.c.sharpen * __ldg(a.t.wsharpen + bin) *
                   sqrtf(psd * a.c.smax2n / ((psd + a.c.smin2n) * (psd + a.c.smax2n)));
}
__device__ __forceinline__ float dehalo_fact(const InverseArgs& a, float psd, int bin) {
  // src/code_impl/Apply.cpp:132
  return (psd + a.c.ht2n) / ((psd + a.c.ht2n) + a.c.dehalo * __ldg(a.t.wdehalo + bin) * psd);
}

// limited Wiener factor applied to one temporal component, code_impl_C.h:34-40
__device__ __forceinline__ void wiener(float& re, float& im, float noise, float lowlimit) {
  const float psd = re * re + im * im + 1.0e-15f;
  const float q = (psd - noise) / psd;
  const float f = q > lowlimit ? q : lowlimit;
  re *= f;
  im *= f;
}

// Filtered value of one bin. MODE: 1 = Wiener 2D, 2..5 = Wiener 3D,
// 0 = Kalman (updates the state when `commit`), -1 = sharpen only (identity).
template <int MODE>
__device__ __forceinline__ float2 filter_bin(const InverseArgs& a, size_t off, int bin, float gf, bool commit) {
  const float2 cur = a.in[2][off + bin];
  if constexpr (MODE == MODE_SHARPEN_ONLY) {
    return cur;
  } else if constexpr (MODE == MODE_KALMAN) {
    // src/code_impl/Kalman.cpp:27-64
    float2 last = a.kal_last[off + bin];
    float cv = a.kal_covar[off + bin], cp = a.kal_covarp[off + bin];
    float sigma = a.c.sigma2n_2d;
    if (a.c.pattern) {
      sigma = __ldg(a.t.pattern2d + bin);
      if (sigma < 1e-15f) sigma = 1e-15f;
    }
    const float dr = cur.x - last.x, di = cur.y - last.y;
    if (dr * dr > sigma * a.c.kratio2 || di * di > sigma * a.c.kratio2) {
      cv = sigma;
      cp = sigma;
      last = cur;
    } else {
      const float sum = cv + cp;
      const float gain = sum / (sum + sigma);
      cp = gain * gain * sigma;
      cv = (1.f - gain) * sum;
      last.x = gain * cur.x + (1.f - gain) * last.x;
      last.y = gain * cur.y + (1.f - gain) * last.y;
    }
    if (commit) {
      a.kal_last[off + bin] = last;
      a.kal_covar[off + bin] = cv;
      a.kal_covarp[off + bin] = cp;
    }
    return last;
  } else if constexpr (MODE == MODE_WIENER2D) {
    // src/code_impl/Apply.cpp:13-65
    float2 gc = make_float2(0.f, 0.f);
    if (a.c.degrid != 0.f) {
      const float2 gs = __ldg(a.t.grid + bin);
      gc = make_float2(gf * gs.x, gf * gs.y);
    }
    const float cr = cur.x - gc.x, ci = cur.y - gc.y;
    const float psd = cr * cr + ci * ci + 1e-15f;
    const float noise = a.c.pattern ? __ldg(a.t.pattern2d + bin) : a.c.sigma2n;
    const float q = (psd - noise) / psd;
    float f = q > a.c.lowlimit ? q : a.c.lowlimit;
    if (a.c.fuse_sharpen) {
      if (a.c.use_sharpen && a.c.use_dehalo) f *= sharpen_fact(a, psd, bin) * dehalo_fact(a, psd, bin);
      else if (a.c.use_sharpen) f *= sharpen_fact(a, psd, bin);
      else if (a.c.use_dehalo) f *= dehalo_fact(a, psd, bin);
    }
    return make_float2(cr * f + gc.x, ci * f + gc.y);
  } else {
    // Wiener 3D over MODE frames, src/code_impl/Apply.cpp:67-235
    constexpr float kb = (float)MODE;
    float g0 = 0.f, g1 = 0.f;
    if (a.c.degrid != 0.f) {
      const float2 gs = __ldg(a.t.grid + bin);
      g0 = gf * gs.x * kb;
      g1 = gf * gs.y * kb;
    }
    const float noise = a.c.pattern ? __ldg(a.t.pattern3d + bin) : a.c.sigma2n;
    const float ll = a.c.lowlimit;
    const float cr = cur.x, ci = cur.y;
    if constexpr (MODE == 2) {
      const float2 pv = a.in[1][off + bin];
      float f0r = cr + pv.x - g0, f0i = ci + pv.y - g1;
      float f1r = cr - pv.x, f1i = ci - pv.y;
      wiener(f0r, f0i, noise, ll);
      wiener(f1r, f1i, noise, ll);
      return make_float2((f0r + f1r + g0) * 0.5f, (f0i + f1i + g1) * 0.5f);
    } else if constexpr (MODE == 3) {
      const float sin120 = 0.86602540378443864676372317075294f;
      const float2 pv = a.in[1][off + bin], nx = a.in[3][off + bin];
      const float pnr = pv.x + nx.x, pni = pv.y + nx.y;
      float fcr = cr + pnr - g0, fci = ci + pni - g1;
      const float di = sin120 * (pv.y - nx.y), dr = sin120 * (nx.x - pv.x);
      float fpr = cr - 0.5f * pnr + di, fnr = cr - 0.5f * pnr - di;
      float fpi = ci - 0.5f * pni + dr, fni = ci - 0.5f * pni - dr;
      wiener(fcr, fci, noise, ll);
      wiener(fpr, fpi, noise, ll);
      wiener(fnr, fni, noise, ll);
      const float third = 1.0f / 3.0f;
      return make_float2((fcr + fpr + fnr + g0) * third, (fci + fpi + fni + g1) * third);
    } else if constexpr (MODE == 4) {
      const float2 p2 = a.in[0][off + bin], pv = a.in[1][off + bin], nx = a.in[3][off + bin];
      float fp2r = (cr + p2.x) - (pv.x + nx.x), fp2i = (ci + p2.y) - (pv.y + nx.y);
      float fpr = (cr - p2.x) + (pv.y - nx.y), fpi = (ci - p2.y) - (pv.x - nx.x);
      float fcr = (cr + p2.x) + (pv.x + nx.x) - g0, fci = (ci + p2.y) + (pv.y + nx.y) - g1;
      float fnr = (cr - p2.x) - (pv.y - nx.y), fni = (ci - p2.y) + (pv.x - nx.x);
      wiener(fp2r, fp2i, noise, ll);
      wiener(fpr, fpi, noise, ll);
      wiener(fcr, fci, noise, ll);
      wiener(fnr, fni, noise, ll);
      return make_float2(((fp2r + fpr) + (fcr + fnr) + g0) * 0.25f, ((fp2i + fpi) + (fci + fni) + g1) * 0.25f);
    } else {
      const float sin72 = 0.95105651629515357211643933337938f, cos72 = 0.30901699437494742410229341718282f;
      const float sin144 = 0.58778525229247312916870595463907f, cos144 = -0.80901699437494742410229341718282f;
      const float2 p2 = a.in[0][off + bin], pv = a.in[1][off + bin];
      const float2 nx = a.in[3][off + bin], n2 = a.in[4][off + bin];
      float sum = (p2.x + n2.x) * cos72 + (pv.x + nx.x) * cos144 + cr;
      float dif = (-p2.y + n2.y) * sin72 + (pv.y - nx.y) * sin144;
      float fp2r = sum + dif, fn2r = sum - dif;
      sum = (p2.y + n2.y) * cos72 + (pv.y + nx.y) * cos144 + ci;
      dif = (p2.x - n2.x) * sin72 + (-pv.x + nx.x) * sin144;
      float fp2i = sum + dif, fn2i = sum - dif;
      sum = (p2.x + n2.x) * cos144 + (pv.x + nx.x) * cos72 + cr;
      dif = (p2.y - n2.y) * sin144 + (pv.y - nx.y) * sin72;
      float fpr = sum + dif, fnr = sum - dif;
      sum = (p2.y + n2.y) * cos144 + (pv.y + nx.y) * cos72 + ci;
      dif = (-p2.x + n2.x) * sin144 + (-pv.x + nx.x) * sin72;
      float fpi = sum + dif, fni = sum - dif;
      float fcr = (p2.x + pv.x) + cr + (nx.x + n2.x) - g0;
      float fci = (p2.y + pv.y) + ci + (nx.y + n2.y) - g1;
      wiener(fp2r, fp2i, noise, ll);
      wiener(fpr, fpi, noise, ll);
      wiener(fcr, fci, noise, ll);
      wiener(fnr, fni, noise, ll);
      wiener(fn2r, fn2i, noise, ll);
      return make_float2(((fp2r + fpr) + (fcr + fnr) + fn2r + g0) * 0.2f,
                         ((fp2i + fpi) + (fci + fni) + fn2i + g1) * 0.2f);
    }
  }
}

// separate sharpen/dehalo pass on a filtered bin, src/code_impl/Sharpen.cpp:13-63
__device__ __forceinline__ float2 sharpen_bin(const InverseArgs& a, float2 v, int bin, float gf) {
  float2 gc = make_float2(0.f, 0.f);
  if (a.c.degrid != 0.f) {
    const float2 gs = __ldg(a.t.grid + bin);
    gc = make_float2(gf * gs.x, gf * gs.y);
  }
  const float cr = v.x - gc.x, ci = v.y - gc.y;
  const float psd = cr * cr + ci * ci + 1.0e-15f;
  float f;
  if (a.c.use_sharpen && a.c.use_dehalo) f = sharpen_fact(a, psd, bin) * dehalo_fact(a, psd, bin);
  else if (a.c.use_sharpen) f = sharpen_fact(a, psd, bin);
  else f = dehalo_fact(a, psd, bin);
  return make_float2(cr * f + gc.x, ci * f + gc.y);
}

// ---------------------------------------------------------------- inverse

template <int BW, int BH, int MODE>
__global__ void __launch_bounds__(kWarps * 32) k_filter_inverse(InverseArgs a) {
  constexpr int NH = BW / 2 + 1, TP = BW + 1;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tile = smem + warp * fft_smem_floats<BW, BH>();
  float2* S = reinterpret_cast<float2*>(tile + BH * TP);
  const Geom& g = a.g;
  const int blk = blockIdx.x * kWarps + warp;
  if (blk >= g.nblocks) return;
  const size_t off = (size_t)blk * BH * NH;
  const float gs0 = __ldg(&a.t.grid[0].x);
  const float gf = (MODE >= 1) ? a.c.degrid * a.in[2][off].x / gs0 : 0.f;
  // grid fraction of the separate sharpen pass: the DC of the FILTERED block
  // (Sharpen.cpp reads its input spectrum), recomputed by every lane
  float gf_sh = 0.f;
  if (a.c.do_sharpen) gf_sh = a.c.degrid * filter_bin<MODE>(a, off, 0, gf, false).x / gs0;
  // 1. filter every bin, then the inverse DFT along y (one column per lane)
  for (int k = lane; k < NH; k += 32) {
    float2 col[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) {
      const int bin = h * NH + k;
      float2 v = filter_bin<MODE>(a, off, bin, gf, true);
      if (a.c.do_sharpen) v = sharpen_bin(a, v, bin, gf_sh);
      col[h] = v;
    }
    cfft<BH, +1>(col);
#pragma unroll
    for (int h = 0; h < BH; h++) S[h * NH + k] = col[h];
  }
  __syncwarp();
  // 2. c2r along x, one row per lane
  for (int y = lane; y < BH; y += 32) {
    float2 c[NH];
#pragma unroll
    for (int k = 0; k < NH; k++) c[k] = S[y * NH + k];
    float r[BW];
    irfft<BW>(c, r);
#pragma unroll
    for (int x = 0; x < BW; x++) tile[y * TP + x] = r[x];
  }
  __syncwarp();
  // 3. coalesced store of the time-domain block
  float* out = a.tdom + (size_t)blk * BH * BW;
  for (int y = 0; y < BH; y++)
    for (int x = lane; x < BW; x += 32) out[y * BW + x] = tile[y * TP + x];
}

// ---------------------------------------------------------------- launchers

template <int BW, int BH>
cudaError_t fwd_sized(const ForwardArgs& a, int bytes, cudaStream_t s) {
  const int smem = kWarps * fft_smem_floats<BW, BH>() * 4;
  const int grid = (a.g.nblocks + kWarps - 1) / kWarps;
  cudaError_t e = cudaSuccess;
  if (bytes == 1) {
    e = cudaFuncSetAttribute(k_forward<BW, BH, uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) k_forward<BW, BH, uint8_t><<<grid, kWarps * 32, smem, s>>>(a);
  } else if (bytes == 2) {
    e = cudaFuncSetAttribute(k_forward<BW, BH, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) k_forward<BW, BH, uint16_t><<<grid, kWarps * 32, smem, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(k_forward<BW, BH, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) k_forward<BW, BH, float><<<grid, kWarps * 32, smem, s>>>(a);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BW, int BH, int MODE>
cudaError_t inv_mode(const InverseArgs& a, cudaStream_t s) {
  const int smem = kWarps * fft_smem_floats<BW, BH>() * 4;
  const int grid = (a.g.nblocks + kWarps - 1) / kWarps;
  cudaError_t e =
      cudaFuncSetAttribute(k_filter_inverse<BW, BH, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_filter_inverse<BW, BH, MODE><<<grid, kWarps * 32, smem, s>>>(a);
  return cudaGetLastError();
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
#define FFT3D_REGISTER_SIZE(BW, BH)                                                                  \
  static const bool fft3d_reg_##BW##x##BH = register_size(                                          \
      SizeEntry{BW, BH, &fwd_sized<BW, BH>, &inv_sized<BW, BH>, &upload_twiddle_table});

}  // namespace fft3d
