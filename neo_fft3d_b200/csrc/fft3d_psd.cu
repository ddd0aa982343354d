// Learned noise PSD: a 3-layer MLP (544 -> 512 -> 512 -> 544, GELU) that maps
// the log power spectrum of one 32x32 windowed block to that block's
// per-frequency noise power, with its training data generated on the device.
//
// The prediction takes the place of the reference's noise pattern
// (pattern2d / pattern3d = bt x pattern2d, src/helper.cpp:171-178,
// src/fft3d_engine.h:625-630) in the Wiener and Kalman gains.
//
// Training data (k_field, k_gen_blocks). Clean frames are seeded sums of 64
// sinusoids (periods 8-200 px, random orientation and phase, amplitude
// 0.5-1) scaled to 16..235 per frame. Each training block draws its own noise
// process: white Gaussian noise shaped by a 16x16 FIR whose frequency response
// samples a radially symmetric transfer function H(r) -- a monotone cubic
// (Fritsch-Carlson) spline through 4 knots at normalised radius 0, 1/3, 2/3, 1
// (r = |f| / 0.5 cycles per pixel, clamped to 1), knot amplitudes
// log-uniform in [span, 1] with the span log-uniform in [knot_min, 1] (white
// to steep spectra), sorted falling or rising -- scaled so that the
// noise's standard deviation is a uniform draw in [sigma_min, sigma_max]. The
// noisy block is rounded and clamped to 8 bits, windowed with the plane's
// analysis window and transformed like the filter's forward kernel.
//   input : x_k = (log(|X_k|^2 + 1) - 8) * 0.4 for the 543 non-DC bins (DC and
//           padding columns 0), as BF16
//   target: log(E|N_k|^2 + q) - 7, where E|N_k|^2 is the exact noise power of
//           the windowed block at bin k, sum_d R(d) A(d) cos(k.d), with R the
//           shaped noise's autocorrelation and A the window's, and
//           q = sum(window^2) / 12 the 8-bit rounding noise.
// Training: mean squared error of the 544 outputs, Adam on FP32 master weights,
// BF16 weights and activations into the tensor-core GEMM (mlp_kernels.cu).
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fft3d_b200.h"
#include "fft3d_kernels.cuh"
#include "fft3d_mlp.h"
#include "fft3d_psd.h"

namespace {

constexpr int BS = 32;                 // block side
constexpr int NH = BS / 2 + 1;         // 17 half-spectrum columns
constexpr int BINS = BS * NH;          // 544
constexpr int IN = FFT3D_PSD_FEATURES, HID = FFT3D_PSD_HIDDEN, OUT = FFT3D_PSD_OUTPUTS;
constexpr int FIR = 16;                // noise-shaping FIR taps per axis
constexpr int PATCH = BS + FIR - 1;    // 47: white-noise patch side
constexpr int LAGS = 2 * FIR - 1;      // 31: autocorrelation lags per axis
constexpr int NSINES = 64;
constexpr float kFeatMean = 8.f, kFeatScale = 0.4f, kLogOffset = 7.f;
constexpr int kInfo = FFT3D_PSD_INFO;
constexpr int kValBlocks = 32768;

constexpr long long O_W1 = 0, O_B1 = O_W1 + (long long)HID * IN, O_W2 = O_B1 + HID,
                    O_B2 = O_W2 + (long long)HID * HID, O_W3 = O_B2 + HID, O_B3 = O_W3 + (long long)OUT * HID,
                    NPARAM = O_B3 + OUT;

static_assert(BINS <= IN && BINS <= OUT, "padding");

// ---------------------------------------------------------------- random numbers
// Counter-based: the SplitMix64 finaliser over (seed, stream, index).
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t index) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ index);
}
// uniform in [0, 1) with 24 bits
__host__ __device__ inline float unif(uint64_t z) { return (float)(z >> 40) * (1.f / 16777216.f); }
// uniform integer in [0, n)
__host__ __device__ inline int unif_int(uint64_t z, int n) { return (int)(((z >> 40) * (uint64_t)n) >> 24); }
// standard normal from one draw (Box-Muller on two 24-bit uniforms)
__device__ inline float gauss(uint64_t z) {
  const float u1 = (float)((z >> 40) + 1) * (1.f / 16777216.f);
  const float u2 = (float)((z >> 16) & 0xFFFFFF) * (1.f / 16777216.f);
  return sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
}
enum : uint64_t { RNG_BLOCK = 1, RNG_WHITE = 2, RNG_FIELD = 3, RNG_INIT = 4 };

__device__ inline int ord_enc(float v) {
  const int i = __float_as_int(v);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float ord_dec(int e) {
  const int i = e >= 0 ? e : e ^ 0x7FFFFFFF;
  float f;
  memcpy(&f, &i, 4);
  return f;
}

// ---------------------------------------------------------------- clean frames

// field[f][y][x] = sum_k amp_k sin(2 pi (fx_k x + fy_k y + ph_k)); per-frame
// min / max into minmax[2f], minmax[2f+1] (order-preserving int encoding)
__global__ void __launch_bounds__(256) k_field(const float4* __restrict__ params, float* field, int W, int H,
                                               int* minmax) {
  const int f = blockIdx.y;
  __shared__ float4 p[NSINES];
  __shared__ int smn[8], smx[8];
  if (threadIdx.x < NSINES) p[threadIdx.x] = params[f * NSINES + threadIdx.x];
  __syncthreads();
  float mn = INFINITY, mx = -INFINITY;
  const long long npx = (long long)W * H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npx; i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i - (long long)y * W);
    float v = 0.f;
#pragma unroll 8
    for (int k = 0; k < NSINES; k++) {
      float t = fmaf(p[k].x, (float)x, fmaf(p[k].y, (float)y, p[k].z));
      t -= floorf(t);
      v = fmaf(p[k].w, sinpif(2.f * t), v);
    }
    field[f * npx + i] = v;
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    smn[warp] = ord_enc(mn);
    smx[warp] = ord_enc(mx);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = smn[0], b = smx[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      a = min(a, smn[w]);
      b = max(b, smx[w]);
    }
    atomicMin(minmax + 2 * f, a);
    atomicMax(minmax + 2 * f + 1, b);
  }
}

// ---------------------------------------------------------------- training blocks

struct GenArgs {
  const float* field;
  const int* minmax;
  int frames, W, H;
  unsigned long long seed;
  long long first, count;
  float sigma_min, sigma_max, knot_min;
  const float* win;         // analysis window: wx[32], wy[32]
  __nv_bfloat16* X;         // count x IN (may be null)
  float* T;                 // count x BINS (may be null)
  float* feat;              // count x IN floats (optional)
  float* info;              // count x kInfo (optional)
  float* clean;             // count x 1024 (optional)
  uint8_t* noisy;           // count x 1024 (optional)
};

// monotone cubic Hermite through (i/3, v[i]) with tangents m[i]
__device__ inline float spline_eval(const float* v, const float* m, float r) {
  const float d = 1.f / 3.f;
  const int i = min(2, (int)(r * 3.f));
  const float t = (r - (float)i * d) * 3.f;
  const float t2 = t * t, t3 = t2 * t;
  return (2.f * t3 - 3.f * t2 + 1.f) * v[i] + (t3 - 2.f * t2 + t) * d * m[i] + (-2.f * t3 + 3.f * t2) * v[i + 1] +
         (t3 - t2) * d * m[i + 1];
}

__global__ void __launch_bounds__(256) k_gen_blocks(GenArgs a) {
  const int tid = threadIdx.x;
  __shared__ float s_wx[BS], s_wy[BS], s_ax[LAGS], s_ay[LAGS];
  __shared__ float2 s_tw[BS];  // (cos, sin)(2 pi m / 32)
  __shared__ float s_c16[FIR];
  __shared__ float s_par[16];  // sigma, v0..v3, m0..m3, dir, frame, x0, y0, gain, sumh2
  __shared__ float s_H[FIR][FIR], s_C[FIR][FIR], s_h[FIR][FIR];
  __shared__ float s_w[PATCH * PATCH];
  __shared__ float s_pix[BS][BS + 1];
  __shared__ float2 s_row[BS][NH];
  __shared__ float2 s_spec[BINS];
  __shared__ float s_R[LAGS * LAGS];
  __shared__ float2 s_QS[LAGS][NH];
  __shared__ float s_red[8];
  if (tid < BS) {
    s_wx[tid] = a.win[tid];
    s_wy[tid] = a.win[BS + tid];
    float sn, cs;
    sincospif(2.f * (float)tid / BS, &sn, &cs);
    s_tw[tid] = make_float2(cs, sn);
  }
  if (tid < FIR) s_c16[tid] = cospif(2.f * (float)tid / FIR);
  __syncthreads();
  if (tid < 2 * LAGS) {  // window autocorrelations at lags -15..15
    const float* w = tid < LAGS ? s_wx : s_wy;
    const int d = (tid % LAGS) - (FIR - 1);
    float s = 0.f;
    for (int x = 0; x < BS; x++)
      if (x + d >= 0 && x + d < BS) s += w[x] * w[x + d];
    (tid < LAGS ? s_ax : s_ay)[tid % LAGS] = s;
  }
  float qnoise;  // rounding noise: sum(window^2) / 12
  {
    float sx = 0.f, sy = 0.f;
    for (int x = 0; x < BS; x++) {
      sx += a.win[x] * a.win[x];
      sy += a.win[BS + x] * a.win[BS + x];
    }
    qnoise = sx * sy * (1.f / 12.f);
  }
  __syncthreads();
  for (long long i = blockIdx.x; i < a.count; i += gridDim.x) {
    const unsigned long long gb = (unsigned long long)(a.first + i);
    // 1. the block's noise process and position
    if (tid == 0) {
      const uint64_t base = gb * 16;
      const float sigma = a.sigma_min + (a.sigma_max - a.sigma_min) * unif(rnd(a.seed, RNG_BLOCK, base));
      // knot amplitudes log-uniform in [span, 1], the span itself log-uniform
      // in [knot_min, 1]: from white (span near 1) to steep spectra
      float v[4];
      const float lk = logf(a.knot_min) * unif(rnd(a.seed, RNG_BLOCK, base + 9));
      for (int k = 0; k < 4; k++) v[k] = expf(lk * unif(rnd(a.seed, RNG_BLOCK, base + 1 + k)));
      const int rising = unif(rnd(a.seed, RNG_BLOCK, base + 5)) >= 0.5f ? 1 : 0;
      for (int p = 0; p < 3; p++)  // sort: falling (low-pass) or rising (high-pass)
        for (int q = 0; q < 3 - p; q++)
          if (rising ? v[q] > v[q + 1] : v[q] < v[q + 1]) {
            const float t = v[q];
            v[q] = v[q + 1];
            v[q + 1] = t;
          }
      // Fritsch-Carlson tangents
      float dl[3], m[4];
      for (int k = 0; k < 3; k++) dl[k] = (v[k + 1] - v[k]) * 3.f;
      m[0] = dl[0];
      m[3] = dl[2];
      for (int k = 1; k < 3; k++) m[k] = dl[k - 1] * dl[k] <= 0.f ? 0.f : 0.5f * (dl[k - 1] + dl[k]);
      for (int k = 0; k < 3; k++) {
        if (dl[k] == 0.f) {
          m[k] = m[k + 1] = 0.f;
        } else {
          const float al = m[k] / dl[k], be = m[k + 1] / dl[k], s2 = al * al + be * be;
          if (s2 > 9.f) {
            const float tau = 3.f / sqrtf(s2);
            m[k] = tau * al * dl[k];
            m[k + 1] = tau * be * dl[k];
          }
        }
      }
      s_par[0] = sigma;
      for (int k = 0; k < 4; k++) {
        s_par[1 + k] = v[k];
        s_par[5 + k] = m[k];
      }
      s_par[9] = (float)rising;
      s_par[10] = (float)unif_int(rnd(a.seed, RNG_BLOCK, base + 6), a.frames);
      s_par[11] = (float)unif_int(rnd(a.seed, RNG_BLOCK, base + 7), a.W - BS + 1);
      s_par[12] = (float)unif_int(rnd(a.seed, RNG_BLOCK, base + 8), a.H - BS + 1);
    }
    __syncthreads();
    // 2. transfer function samples at f = (i, j) / 16 (wrapped to [-1/2, 1/2))
    {
      const int r = tid >> 4, c = tid & 15;
      const float fi = (float)(r <= FIR / 2 ? r : r - FIR) / FIR, fj = (float)(c <= FIR / 2 ? c : c - FIR) / FIR;
      const float rad = fminf(1.f, 2.f * sqrtf(fi * fi + fj * fj));
      s_H[r][c] = spline_eval(s_par + 1, s_par + 5, rad);
    }
    __syncthreads();
    // 3. FIR = inverse DFT of the (real, even) samples, centred: s_h[a][b] is lag (a-8, b-8)
    {
      const int r = tid >> 4, c = tid & 15;
      float s = 0.f;
      for (int j = 0; j < FIR; j++) s += s_H[r][j] * s_c16[(j * c) & (FIR - 1)];
      s_C[r][c] = s;
    }
    __syncthreads();
    float hv;
    {
      const int u = tid >> 4, c = tid & 15;
      float s = 0.f;
      for (int r = 0; r < FIR; r++) s += s_c16[(r * u) & (FIR - 1)] * s_C[r][c];
      hv = s * (1.f / (FIR * FIR));
      s_h[(u + FIR / 2) & (FIR - 1)][(c + FIR / 2) & (FIR - 1)] = hv;
    }
    // 4. gain so that the shaped noise has standard deviation sigma
    {
      float s = hv * hv;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if ((tid & 31) == 0) s_red[tid >> 5] = s;
    }
    // 5. white noise over the FIR's support
    for (int p = tid; p < PATCH * PATCH; p += blockDim.x) s_w[p] = gauss(rnd(a.seed, RNG_WHITE, gb * 4096 + p));
    __syncthreads();
    if (tid == 0) {
      float s = 0.f;
      for (int w = 0; w < 8; w++) s += s_red[w];
      s_par[14] = s;
      s_par[13] = s_par[0] / sqrtf(s);
    }
    __syncthreads();
    // 6. noisy pixels: clean + gain * (FIR (x) white), rounded, clamped, windowed
    {
      const int f = (int)s_par[10], x0 = (int)s_par[11], y0 = (int)s_par[12];
      const float mn = ord_dec(a.minmax[2 * f]), mx = ord_dec(a.minmax[2 * f + 1]);
      const float sc = 219.f / (mx - mn), gain = s_par[13];
      const float* fr = a.field + (size_t)f * a.W * a.H;
      for (int q = tid; q < BS * BS; q += blockDim.x) {
        const int y = q >> 5, x = q & 31;
        float n = 0.f;
        for (int u = 0; u < FIR; u++) {
          const float* wr = s_w + (y + u) * PATCH + x;
#pragma unroll
          for (int v = 0; v < FIR; v++) n = fmaf(s_h[u][v], wr[v], n);
        }
        const float cv = 16.f + (fr[(size_t)(y0 + y) * a.W + x0 + x] - mn) * sc;
        const float nz = fminf(fmaxf(rintf(cv + gain * n), 0.f), 255.f);
        s_pix[y][x] = nz * s_wy[y] * s_wx[x];
        if (a.clean) a.clean[i * BS * BS + q] = cv;
        if (a.noisy) a.noisy[i * BS * BS + q] = (uint8_t)nz;
      }
    }
    __syncthreads();
    // 7. 2D DFT (rows, then columns) of the windowed block; exact autocorrelation
    //    of the shaped noise at lags -15..15 (gain^2 sum_ab h[a][b] h[a+dy][b+dx])
    for (int q = tid; q < BS * NH; q += blockDim.x) {
      const int y = q / NH, k = q - y * NH;
      float re = 0.f, im = 0.f;
      for (int x = 0; x < BS; x++) {
        const float2 t = s_tw[(k * x) & (BS - 1)];
        re = fmaf(s_pix[y][x], t.x, re);
        im = fmaf(-s_pix[y][x], t.y, im);
      }
      s_row[y][k] = make_float2(re, im);
    }
    for (int q = tid; q < LAGS * LAGS; q += blockDim.x) {
      const int dy = q / LAGS - (FIR - 1), dx = q % LAGS - (FIR - 1);
      const int a0 = max(0, -dy), a1 = min(FIR, FIR - dy), b0 = max(0, -dx), b1 = min(FIR, FIR - dx);
      float s = 0.f;
      for (int u = a0; u < a1; u++)
        for (int v = b0; v < b1; v++) s = fmaf(s_h[u][v], s_h[u + dy][v + dx], s);
      s_R[q] = s * s_par[13] * s_par[13];
    }
    __syncthreads();
    for (int q = tid; q < BINS; q += blockDim.x) {
      const int ky = q / NH, kx = q - ky * NH;
      float re = 0.f, im = 0.f;
      for (int y = 0; y < BS; y++) {
        const float2 t = s_tw[(ky * y) & (BS - 1)], v = s_row[y][kx];
        re += v.x * t.x + v.y * t.y;
        im += v.y * t.x - v.x * t.y;
      }
      s_spec[q] = make_float2(re, im);
    }
    for (int q = tid; q < LAGS * NH; q += blockDim.x) {
      const int dyi = q / NH, kx = q - dyi * NH;
      float qc = 0.f, qs = 0.f;
      for (int dxi = 0; dxi < LAGS; dxi++) {
        const float ra = s_R[dyi * LAGS + dxi] * s_ax[dxi];
        const float2 t = s_tw[(kx * (dxi - (FIR - 1))) & (BS - 1)];
        qc = fmaf(ra, t.x, qc);
        qs = fmaf(ra, t.y, qs);
      }
      s_QS[dyi][kx] = make_float2(qc, qs);
    }
    __syncthreads();
    // 8. model input and target
    for (int c = tid; c < IN; c += blockDim.x) {
      float x = 0.f;
      if (c > 0 && c < BINS) {
        const float2 s = s_spec[c];
        x = (logf(s.x * s.x + s.y * s.y + 1.f) - kFeatMean) * kFeatScale;
      }
      const __nv_bfloat16 xb = __float2bfloat16_rn(x);
      if (a.X) a.X[i * IN + c] = xb;
      if (a.feat) a.feat[i * IN + c] = __bfloat162float(xb);
    }
    for (int q = tid; q < BINS; q += blockDim.x) {
      const int ky = q / NH, kx = q - ky * NH;
      float p = 0.f;
      for (int dyi = 0; dyi < LAGS; dyi++) {
        const float2 t = s_tw[(ky * (dyi - (FIR - 1))) & (BS - 1)], v = s_QS[dyi][kx];
        p = fmaf(s_ay[dyi], v.x * t.x - v.y * t.y, p);
      }
      if (a.T) a.T[i * BINS + q] = logf(fmaxf(p, 0.f) + qnoise) - kLogOffset;
    }
    if (a.info && tid < kInfo) {
      float v = 0.f;
      if (tid == 0) v = s_par[0];
      else if (tid <= 4) v = s_par[tid];
      else if (tid == 5) v = s_par[9];
      else if (tid == 6) v = s_par[13];
      else if (tid <= 9) v = s_par[tid + 3];
      else if (tid == 10) v = s_par[14];
      a.info[i * kInfo + tid] = v;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- inference helpers

// model input from a plane's block spectra (blocks x 544 complex); power
// divided by pow_scale (the square of the sample scale relative to 8 bits)
__global__ void k_features(const float2* __restrict__ spec, __nv_bfloat16* X, long long blocks, float inv_pow) {
  const long long n = blocks * IN;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / IN;
    const int c = (int)(i - b * IN);
    float x = 0.f;
    if (c > 0 && c < BINS) {
      const float2 s = spec[b * BINS + c];
      x = (logf((s.x * s.x + s.y * s.y) * inv_pow + 1.f) - kFeatMean) * kFeatScale;
    }
    X[i] = __float2bfloat16_rn(x);
  }
}

__global__ void k_psd_blocks(const float* __restrict__ Y, float* out, long long blocks, float pow_scale) {
  const long long n = blocks * BINS;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / BINS;
    const int c = (int)(i - b * BINS);
    out[i] = expf(Y[b * OUT + c] + kLogOffset) * pow_scale;
  }
}

__global__ void k_psd_pooled(const float* __restrict__ mean, float* out, float pow_scale) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < BINS) out[c] = expf(mean[c] + kLogOffset) * pow_scale;
}

int grid_for(long long n) {
  const long long g = (n + 255) / 256;
  return (int)std::min<long long>(g, 148 * 16);
}

int fail(int code, const std::string& msg) {
  fft3d::set_last_error(msg);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(FFT3D_E_CUDA, std::string("neo_fft3d: CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define CK(call, what)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, what);   \
  } while (0)
#define CKE(call)                            \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return e_;        \
  } while (0)

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// Activations of up to `rows` rows (a multiple of 128); the backward buffers
// only when `train`.
struct fft3d::psd::Work {
  long long rows = 0;
  void* mem = nullptr;
  __nv_bfloat16* X = nullptr;  // inference features
  float *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr;
  __nv_bfloat16 *H1 = nullptr, *H2 = nullptr;
  float *dY = nullptr, *dH = nullptr;
  __nv_bfloat16 *dYb = nullptr, *dZb = nullptr;
  // transposed copies for the backward's K-major GEMMs: activations [features][rows], weights [in][out]
  __nv_bfloat16 *dYbT = nullptr, *dZbT = nullptr, *H1T = nullptr, *H2T = nullptr, *XT = nullptr;
  __nv_bfloat16 *W2T = nullptr, *W3T = nullptr;
  float* partial = nullptr;
  float* mean = nullptr;
};

struct fft3d_psd {
  std::mutex mu;
  int device = 0;
  int ow = 16, oh = 16, wintype = 0;
  cudaStream_t stream = nullptr;
  void* mem = nullptr;
  float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16* wb = nullptr;
  float* win = nullptr;   // analysis window wx[32], wy[32]
  int* err = nullptr;
  float* loss = nullptr;  // device scalar
  int step = 0;           // Adam steps taken
  double stats[4] = {};   // last training run: generation ms, training ms, steps, GEMM flops per step
};

namespace {

using fft3d::psd::Work;

void work_free(Work* w) {
  if (!w) return;
  if (w->mem) cudaFree(w->mem);
  delete w;
}

Work* work_alloc(long long rows, bool train) {
  Work* w = new Work;
  w->rows = rows;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align256(bytes);
    return o;
  };
  const size_t oX = take(rows * IN * 2), oZ1 = take(rows * HID * 4), oZ2 = take(rows * HID * 4),
               oY = take(rows * OUT * 4), oH1 = take(rows * HID * 2), oH2 = take(rows * HID * 2),
               oP = take(fft3d::mlp::colsum_partial_floats(rows, OUT) * 4), oM = take(OUT * 4);
  size_t odY = 0, odH = 0, odYb = 0, odZb = 0, odYbT = 0, odZbT = 0, oH1T = 0, oH2T = 0, oXT = 0, oW2T = 0, oW3T = 0;
  if (train) {
    odY = take(rows * OUT * 4);
    odH = take(rows * HID * 4);
    odYb = take(rows * OUT * 2);
    odZb = take(rows * HID * 2);
    odYbT = take(rows * OUT * 2);
    odZbT = take(rows * HID * 2);
    oH1T = take(rows * HID * 2);
    oH2T = take(rows * HID * 2);
    oXT = take(rows * IN * 2);
    oW2T = take((size_t)HID * HID * 2);
    oW3T = take((size_t)HID * OUT * 2);
  }
  if (cudaMalloc(&w->mem, off) != cudaSuccess) {
    cudaGetLastError();
    delete w;
    return nullptr;
  }
  cudaMemset(w->mem, 0, off);
  char* b = static_cast<char*>(w->mem);
  w->X = reinterpret_cast<__nv_bfloat16*>(b + oX);
  w->Z1 = reinterpret_cast<float*>(b + oZ1);
  w->Z2 = reinterpret_cast<float*>(b + oZ2);
  w->Y = reinterpret_cast<float*>(b + oY);
  w->H1 = reinterpret_cast<__nv_bfloat16*>(b + oH1);
  w->H2 = reinterpret_cast<__nv_bfloat16*>(b + oH2);
  w->partial = reinterpret_cast<float*>(b + oP);
  w->mean = reinterpret_cast<float*>(b + oM);
  if (train) {
    w->dY = reinterpret_cast<float*>(b + odY);
    w->dH = reinterpret_cast<float*>(b + odH);
    w->dYb = reinterpret_cast<__nv_bfloat16*>(b + odYb);
    w->dZb = reinterpret_cast<__nv_bfloat16*>(b + odZb);
    w->dYbT = reinterpret_cast<__nv_bfloat16*>(b + odYbT);
    w->dZbT = reinterpret_cast<__nv_bfloat16*>(b + odZbT);
    w->H1T = reinterpret_cast<__nv_bfloat16*>(b + oH1T);
    w->H2T = reinterpret_cast<__nv_bfloat16*>(b + oH2T);
    w->XT = reinterpret_cast<__nv_bfloat16*>(b + oXT);
    w->W2T = reinterpret_cast<__nv_bfloat16*>(b + oW2T);
    w->W3T = reinterpret_cast<__nv_bfloat16*>(b + oW3T);
  }
  return w;
}

// Y = MLP(X) for `rows` rows (X: rows x IN BF16)
cudaError_t forward(fft3d_psd* m, Work* w, const __nv_bfloat16* X, long long rows, cudaStream_t s) {
  using namespace fft3d::mlp;
  const int R = (int)rows;
  CKE(gemm_bf16(X, IN, 1, m->wb + O_W1, IN, 1, w->Z1, HID, R, HID, IN, false, m->err, s));
  CKE(bias_act(w->Z1, m->w + O_B1, w->Z1, w->H1, rows, HID, true, s));
  CKE(gemm_bf16(w->H1, HID, 1, m->wb + O_W2, HID, 1, w->Z2, HID, R, HID, HID, false, m->err, s));
  CKE(bias_act(w->Z2, m->w + O_B2, w->Z2, w->H2, rows, HID, true, s));
  CKE(gemm_bf16(w->H2, HID, 1, m->wb + O_W3, HID, 1, w->Y, OUT, R, OUT, HID, false, m->err, s));
  CKE(bias_act(w->Y, m->w + O_B3, w->Y, nullptr, rows, OUT, false, s));
  return cudaSuccess;
}

// gradients of the mean squared error into m->g (after forward on the same X)
cudaError_t backward(fft3d_psd* m, Work* w, const __nv_bfloat16* X, const float* T, long long rows, float* loss,
                     cudaStream_t s) {
  using namespace fft3d::mlp;
  const int R = (int)rows;
  // every GEMM below reads both operands along K (the pipelined kernel); the
  // operands that are not stored that way are transposed first
  CKE(mse_grad(w->Y, OUT, T, BINS, w->dY, w->dYb, rows, BINS, loss, s));
  // layer 3: dW3 = dY^T H2, db3 = colsum dY, dH2 = dY W3
  CKE(transpose_bf16(w->dYb, w->dYbT, R, OUT, s));
  CKE(transpose_bf16(w->H2, w->H2T, R, HID, s));
  CKE(gemm_bf16(w->dYbT, R, 1, w->H2T, R, 1, m->g + O_W3, HID, OUT, HID, R, false, m->err, s));
  CKE(colsum(w->dY, w->partial, m->g + O_B3, rows, OUT, 1.f, s));
  CKE(transpose_bf16(m->wb + O_W3, w->W3T, OUT, HID, s));
  CKE(gemm_bf16(w->dYb, OUT, 1, w->W3T, OUT, 1, w->dH, HID, R, HID, OUT, false, m->err, s));
  CKE(gelu_back(w->dH, w->Z2, w->dH, w->dZb, rows * HID, s));
  // layer 2
  CKE(transpose_bf16(w->dZb, w->dZbT, R, HID, s));
  CKE(transpose_bf16(w->H1, w->H1T, R, HID, s));
  CKE(gemm_bf16(w->dZbT, R, 1, w->H1T, R, 1, m->g + O_W2, HID, HID, HID, R, false, m->err, s));
  CKE(colsum(w->dH, w->partial, m->g + O_B2, rows, HID, 1.f, s));
  CKE(transpose_bf16(m->wb + O_W2, w->W2T, HID, HID, s));
  CKE(gemm_bf16(w->dZb, HID, 1, w->W2T, HID, 1, w->dH, HID, R, HID, HID, false, m->err, s));
  CKE(gelu_back(w->dH, w->Z1, w->dH, w->dZb, rows * HID, s));
  // layer 1
  CKE(transpose_bf16(w->dZb, w->dZbT, R, HID, s));
  CKE(transpose_bf16(X, w->XT, R, IN, s));
  CKE(gemm_bf16(w->dZbT, R, 1, w->XT, R, 1, m->g + O_W1, IN, HID, IN, R, false, m->err, s));
  CKE(colsum(w->dH, w->partial, m->g + O_B1, rows, HID, 1.f, s));
  return cudaSuccess;
}

std::vector<float> analysis_window(int wintype, int b, int o) {
  // src/fft3d_engine.h:204-283 (analysis half): wintype 0 half-cosine,
  // 1 its square root, 2 flat
  std::vector<float> w(b, 1.f);
  const float pi = 3.1415926535897932384626433832795f;
  for (int i = 0; i < o; i++) {
    const float cl = cosf(pi * (i - o + 0.5f) / (o * 2)), cr = cosf(pi * (i + 0.5f) / (o * 2));
    float l = 1.f, r = 1.f;
    if (wintype == 0) {
      l = cl;
      r = cr;
    } else if (wintype == 1) {
      l = (float)std::sqrt((double)cl);
      r = (float)std::sqrt((double)cr);
    }
    w[i] = l;
    w[b - o + i] = r;
  }
  return w;
}

double host_normal(uint64_t seed, uint64_t idx) {
  const uint64_t z = rnd(seed, RNG_INIT, idx);
  const double u1 = ((double)(z >> 40) + 1.0) / 16777216.0, u2 = (double)((z >> 16) & 0xFFFFFF) / 16777216.0;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

int check_cfg(const fft3d_psd_train_cfg* c) {
  if (!c) return fail(FFT3D_E_PARAM, "neo_fft3d: missing training configuration");
  if (c->width < BS || c->height < BS || c->clean_frames < 1)
    return fail(FFT3D_E_PARAM, "neo_fft3d: clean frames must be at least 32x32");
  if (!(c->sigma_min >= 0.f) || !(c->sigma_max >= c->sigma_min) || !(c->knot_min > 0.f) || !(c->knot_min <= 1.f))
    return fail(FFT3D_E_PARAM, "neo_fft3d: invalid noise ranges");
  return FFT3D_OK;
}

// clean frames of the configuration on the device: field + per-frame min/max
int make_field(fft3d_psd* m, const fft3d_psd_train_cfg* c, float** field, int** minmax) {
  const int F = c->clean_frames;
  std::vector<float> par((size_t)F * NSINES * 4);
  for (int f = 0; f < F; f++)
    for (int k = 0; k < NSINES; k++) {
      const uint64_t base = ((uint64_t)f * NSINES + k) * 4;
      const double period = 8.0 + 192.0 * unif(rnd(c->seed, RNG_FIELD, base));
      const double theta = M_PI * unif(rnd(c->seed, RNG_FIELD, base + 1));
      const double phase = unif(rnd(c->seed, RNG_FIELD, base + 2));  // cycles
      const double amp = 0.5 + 0.5 * unif(rnd(c->seed, RNG_FIELD, base + 3));
      float* p = &par[((size_t)f * NSINES + k) * 4];
      p[0] = (float)(std::cos(theta) / period);
      p[1] = (float)(std::sin(theta) / period);
      p[2] = (float)phase;
      p[3] = (float)amp;
    }
  float4* dpar = nullptr;
  CK(cudaMalloc(&dpar, par.size() * 4), "psd field parameters");
  const size_t npx = (size_t)c->width * c->height;
  if (cudaMalloc(field, npx * F * 4) != cudaSuccess || cudaMalloc(minmax, F * 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dpar);
    if (*field) cudaFree(*field);
    *field = nullptr;
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for the clean frames");
  }
  std::vector<int> mm(F * 2);
  for (int f = 0; f < F; f++) {
    mm[2 * f] = INT_MAX;
    mm[2 * f + 1] = INT_MIN;
  }
  CK(cudaMemcpyAsync(dpar, par.data(), par.size() * 4, cudaMemcpyHostToDevice, m->stream), "psd upload");
  CK(cudaMemcpyAsync(*minmax, mm.data(), mm.size() * sizeof(int), cudaMemcpyHostToDevice, m->stream), "psd upload");
  const int gx = (int)std::min<size_t>((npx + 255) / 256, 148 * 2);
  k_field<<<dim3(gx, F), 256, 0, m->stream>>>(dpar, *field, c->width, c->height, *minmax);
  CK(cudaGetLastError(), "field kernel");
  CK(cudaStreamSynchronize(m->stream), "field kernel");
  cudaFree(dpar);
  return FFT3D_OK;
}

GenArgs gen_args(fft3d_psd* m, const fft3d_psd_train_cfg* c, const float* field, const int* minmax, long long first,
                 long long count) {
  GenArgs g{};
  g.field = field;
  g.minmax = minmax;
  g.frames = c->clean_frames;
  g.W = c->width;
  g.H = c->height;
  g.seed = c->seed;
  g.first = first;
  g.count = count;
  g.sigma_min = c->sigma_min;
  g.sigma_max = c->sigma_max;
  g.knot_min = c->knot_min;
  g.win = m->win;
  return g;
}

cudaError_t launch_gen(const GenArgs& g, cudaStream_t s) {
  const int grid = (int)std::min<long long>(g.count, 148 * 6);
  k_gen_blocks<<<grid, 256, 0, s>>>(g);
  return cudaGetLastError();
}

int check_err(fft3d_psd* m) {
  int flag = 0;
  CK(cudaMemcpy(&flag, m->err, sizeof(int), cudaMemcpyDeviceToHost), "psd error flag");
  if (flag) {
    cudaMemset(m->err, 0, sizeof(int));
    return fail(FFT3D_E_CUDA, "neo_fft3d: tensor-core MMA completion wait timed out");
  }
  return FFT3D_OK;
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

namespace fft3d {
namespace psd {

std::string check_plane(const fft3d_psd* m, int device, int bw, int bh, int ow, int oh, int wintype) {
  if (bw != BS || bh != BS) return "the learned noise PSD needs bw = bh = 32";
  if (ow != m->ow || oh != m->oh || wintype != m->wintype)
    return "the plane's ow/oh/wintype differ from the learned noise PSD model's";
  if (device != m->device) return "the learned noise PSD model lives on another device";
  return "";
}

Work* work_create(fft3d_psd*, int nblocks) { return work_alloc((nblocks + 127) / 128 * 128, false); }
void work_destroy(Work* w) { work_free(w); }
int* err_flag(fft3d_psd* m) { return m->err; }

cudaError_t infer(fft3d_psd* m, Work* w, const float2* spec, int nblocks, bool pooled, float pow_scale, float* out,
                  cudaStream_t s) {
  const long long rows = (nblocks + 127) / 128 * 128;
  if (rows > w->rows) return cudaErrorInvalidValue;
  k_features<<<grid_for((long long)nblocks * IN), 256, 0, s>>>(spec, w->X, nblocks, 1.f / pow_scale);
  CKE(cudaGetLastError());
  CKE(forward(m, w, w->X, rows, s));
  if (pooled) {
    CKE(fft3d::mlp::colsum(w->Y, w->partial, w->mean, nblocks, OUT, 1.f / (float)nblocks, s));
    k_psd_pooled<<<(BINS + 255) / 256, 256, 0, s>>>(w->mean, out, pow_scale);
  } else {
    k_psd_blocks<<<grid_for((long long)nblocks * BINS), 256, 0, s>>>(w->Y, out, nblocks, pow_scale);
  }
  return cudaGetLastError();
}

}  // namespace psd
}  // namespace fft3d

extern "C" {

void fft3d_psd_train_default(fft3d_psd_train_cfg* c) {
  if (!c) return;
  c->blocks = 1ll << 21;
  c->batch = 4096;
  c->epochs = 3;
  c->lr = 1e-3f;
  c->lr_final = 5e-5f;
  c->seed = 4;
  c->clean_frames = 16;
  c->width = 1920;
  c->height = 1080;
  c->sigma_min = 2.f;
  c->sigma_max = 10.f;
  c->knot_min = 0.1f;
}

long long fft3d_psd_param_count(void) { return NPARAM; }

int fft3d_psd_create(int device, unsigned long long seed, int ow, int oh, int wintype, fft3d_psd** out) {
  if (!out) return fail(FFT3D_E_PARAM, "neo_fft3d: null output handle");
  *out = nullptr;
  if (ow < 0 || oh < 0 || ow > BS / 2 || oh > BS / 2 || wintype < 0 || wintype > 2)
    return fail(FFT3D_E_PARAM, "neo_fft3d: the learned noise PSD needs 0 <= ow, oh <= 16 and wintype 0..2");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(FFT3D_E_NOLIB, "neo_fft3d: no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(FFT3D_E_PARAM, "neo_fft3d: invalid device");
  DevGuard dg(device);
  fft3d_psd* m = new fft3d_psd;
  m->device = device;
  m->ow = ow;
  m->oh = oh;
  m->wintype = wintype;
  const size_t sz = align256(NPARAM * 4) * 4 + align256(NPARAM * 2) + align256(2 * BS * 4) + 256 + 256;
  if (cudaMalloc(&m->mem, sz) != cudaSuccess) {
    cudaGetLastError();
    delete m;
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for the learned noise PSD model");
  }
  char* b = static_cast<char*>(m->mem);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = b + off;
    off += align256(bytes);
    return p;
  };
  m->w = reinterpret_cast<float*>(take(NPARAM * 4));
  m->g = reinterpret_cast<float*>(take(NPARAM * 4));
  m->m1 = reinterpret_cast<float*>(take(NPARAM * 4));
  m->m2 = reinterpret_cast<float*>(take(NPARAM * 4));
  m->wb = reinterpret_cast<__nv_bfloat16*>(take(NPARAM * 2));
  m->win = reinterpret_cast<float*>(take(2 * BS * 4));
  m->err = reinterpret_cast<int*>(take(sizeof(int)));
  m->loss = reinterpret_cast<float*>(take(sizeof(float)));
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(m->mem);
    delete m;
    return fail(FFT3D_E_CUDA, "neo_fft3d: stream creation failed");
  }
  std::vector<float> w(NPARAM, 0.f);
  auto init = [&](long long o, int rows, int cols, int valid_cols) {
    const double sd = 1.0 / std::sqrt((double)valid_cols);
    for (int r = 0; r < rows; r++)
      for (int c = 0; c < cols; c++)
        w[o + (long long)r * cols + c] = c < valid_cols ? (float)(sd * host_normal(seed, o + (long long)r * cols + c)) : 0.f;
  };
  init(O_W1, HID, IN, BINS);
  init(O_W2, HID, HID, HID);
  init(O_W3, OUT, HID, HID);
  std::vector<float> win(2 * BS);
  const std::vector<float> wx = analysis_window(wintype, BS, ow), wy = analysis_window(wintype, BS, oh);
  std::copy(wx.begin(), wx.end(), win.begin());
  std::copy(wy.begin(), wy.end(), win.begin() + BS);
  int rc = fft3d_psd_set_params(m, w.data(), NPARAM);
  if (rc == FFT3D_OK) {
    if (cudaMemcpy(m->win, win.data(), win.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->err, 0, sizeof(int)) != cudaSuccess)
      rc = cuda_fail(cudaGetLastError(), "psd model upload");
  }
  if (rc != FFT3D_OK) {
    fft3d_psd_destroy(m);
    return rc;
  }
  *out = m;
  return FFT3D_OK;
}

void fft3d_psd_destroy(fft3d_psd* m) {
  if (!m) return;
  DevGuard dg(m->device);
  if (m->stream) {
    cudaStreamSynchronize(m->stream);
    cudaStreamDestroy(m->stream);
  }
  if (m->mem) cudaFree(m->mem);
  delete m;
}

int fft3d_psd_get_params(fft3d_psd* m, float* host, long long n) {
  if (!m || !host || n < NPARAM) return fail(FFT3D_E_PARAM, "neo_fft3d: parameter buffer too small");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  CK(cudaMemcpyAsync(host, m->w, NPARAM * 4, cudaMemcpyDeviceToHost, m->stream), "psd parameters");
  CK(cudaStreamSynchronize(m->stream), "psd parameters");
  return FFT3D_OK;
}

int fft3d_psd_set_params(fft3d_psd* m, const float* host, long long n) {
  if (!m || !host || n < NPARAM) return fail(FFT3D_E_PARAM, "neo_fft3d: parameter buffer too small");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  CK(cudaMemcpyAsync(m->w, host, NPARAM * 4, cudaMemcpyHostToDevice, m->stream), "psd parameters");
  CK(fft3d::mlp::to_bf16(m->w, m->wb, NPARAM, m->stream), "psd parameters");
  CK(cudaMemsetAsync(m->m1, 0, NPARAM * 4, m->stream), "psd parameters");
  CK(cudaMemsetAsync(m->m2, 0, NPARAM * 4, m->stream), "psd parameters");
  CK(cudaStreamSynchronize(m->stream), "psd parameters");
  m->step = 0;
  return FFT3D_OK;
}

int fft3d_psd_generate(fft3d_psd* m, const fft3d_psd_train_cfg* c, long long first, long long count, float* features,
                       float* target, float* info, float* clean, unsigned char* noisy) {
  if (!m) return fail(FFT3D_E_PARAM, "neo_fft3d: null model");
  int rc = check_cfg(c);
  if (rc) return rc;
  if (first < 0 || count <= 0 || count > (1 << 20))
    return fail(FFT3D_E_PARAM, "neo_fft3d: generate 1 .. 2^20 blocks per call");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  float* field = nullptr;
  int* minmax = nullptr;
  rc = make_field(m, c, &field, &minmax);
  if (rc) return rc;
  void* buf = nullptr;
  const size_t nf = count * IN * 4, nt = count * BINS * 4, ni = count * kInfo * 4, nc = count * BS * BS * 4,
               nn = count * BS * BS;
  if (cudaMalloc(&buf, nf + nt + ni + nc + nn) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(field);
    cudaFree(minmax);
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for generated blocks");
  }
  char* b = static_cast<char*>(buf);
  GenArgs g = gen_args(m, c, field, minmax, first, count);
  g.feat = reinterpret_cast<float*>(b);
  g.T = reinterpret_cast<float*>(b + nf);
  g.info = reinterpret_cast<float*>(b + nf + nt);
  g.clean = reinterpret_cast<float*>(b + nf + nt + ni);
  g.noisy = reinterpret_cast<uint8_t*>(b + nf + nt + ni + nc);
  cudaError_t e = launch_gen(g, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e == cudaSuccess && features) e = cudaMemcpy(features, g.feat, nf, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && target) e = cudaMemcpy(target, g.T, nt, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && info) e = cudaMemcpy(info, g.info, ni, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && clean) e = cudaMemcpy(clean, g.clean, nc, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && noisy) e = cudaMemcpy(noisy, g.noisy, nn, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  cudaFree(field);
  cudaFree(minmax);
  if (e != cudaSuccess) return cuda_fail(e, "block generator");
  return FFT3D_OK;
}

int fft3d_psd_train(fft3d_psd* m, const fft3d_psd_train_cfg* c, float* loss_curve, int curve_len, float* val_loss) {
  if (!m) return fail(FFT3D_E_PARAM, "neo_fft3d: null model");
  int rc = check_cfg(c);
  if (rc) return rc;
  if (c->batch <= 0 || c->batch % 128 || c->blocks < c->batch || c->epochs < 1 || !(c->lr > 0.f))
    return fail(FFT3D_E_PARAM, "neo_fft3d: batch must be a multiple of 128, blocks >= batch, epochs >= 1, lr > 0");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  float* field = nullptr;
  int* minmax = nullptr;
  rc = make_field(m, c, &field, &minmax);
  if (rc) return rc;
  const long long nb = c->blocks / c->batch, N = nb * c->batch, steps = nb * c->epochs;
  __nv_bfloat16* X = nullptr;
  float* T = nullptr;
  float* losses = nullptr;
  Work* w = work_alloc(c->batch, true);
  const long long total = N + kValBlocks;
  if (!w || cudaMalloc(&X, total * IN * 2) != cudaSuccess || cudaMalloc(&T, total * BINS * 4) != cudaSuccess ||
      cudaMalloc(&losses, (steps + 1) * 4) != cudaSuccess) {
    cudaGetLastError();
    work_free(w);
    cudaFree(X);
    cudaFree(T);
    cudaFree(field);
    cudaFree(minmax);
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for the training blocks");
  }
  cudaEvent_t ev[3] = {};
  for (auto& x : ev) cudaEventCreate(&x);
  cudaError_t e = cudaMemsetAsync(losses, 0, (steps + 1) * 4, m->stream);
  cudaEventRecord(ev[0], m->stream);
  // the training blocks, then the held-out blocks (indices after them)
  for (long long s0 = 0; s0 < total && e == cudaSuccess; s0 += 1 << 20) {
    GenArgs g = gen_args(m, c, field, minmax, s0, std::min<long long>(1 << 20, total - s0));
    g.X = X + s0 * IN;
    g.T = T + s0 * BINS;
    e = launch_gen(g, m->stream);
  }
  cudaEventRecord(ev[1], m->stream);
  for (long long s = 0; s < steps && e == cudaSuccess; s++) {
    const long long b = s % nb;
    const __nv_bfloat16* xb = X + b * c->batch * IN;
    const float* tb = T + b * c->batch * BINS;
    const float frac = steps > 1 ? (float)s / (float)(steps - 1) : 0.f;
    const float lr = c->lr + (c->lr_final - c->lr) * frac;
    e = forward(m, w, xb, c->batch, m->stream);
    if (e == cudaSuccess) e = backward(m, w, xb, tb, c->batch, losses + s, m->stream);
    if (e == cudaSuccess)
      e = fft3d::mlp::adam(m->w, m->g, m->m1, m->m2, m->wb, NPARAM, lr, 0.9f, 0.999f, 1e-8f, ++m->step, m->stream);
  }
  cudaEventRecord(ev[2], m->stream);
  // held-out loss
  const long long vchunks = kValBlocks / c->batch;
  for (long long k = 0; k < vchunks && e == cudaSuccess; k++) {
    const __nv_bfloat16* xb = X + (N + k * c->batch) * IN;
    const float* tb = T + (N + k * c->batch) * BINS;
    e = forward(m, w, xb, c->batch, m->stream);
    if (e == cudaSuccess)
      e = fft3d::mlp::mse_grad(w->Y, OUT, tb, BINS, w->dY, w->dYb, c->batch, BINS, losses + steps, m->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  std::vector<float> hl(steps + 1, 0.f);
  if (e == cudaSuccess) e = cudaMemcpy(hl.data(), losses, (steps + 1) * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) {
    float g_ms = 0.f, t_ms = 0.f;
    cudaEventElapsedTime(&g_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&t_ms, ev[1], ev[2]);
    // forward 1x, backward 2x the forward's GEMM flops
    const double fwd = 2.0 * c->batch * ((double)IN * HID + (double)HID * HID + (double)HID * OUT);
    m->stats[0] = g_ms;
    m->stats[1] = t_ms;
    m->stats[2] = (double)steps;
    m->stats[3] = 3.0 * fwd;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  work_free(w);
  cudaFree(X);
  cudaFree(T);
  cudaFree(losses);
  cudaFree(field);
  cudaFree(minmax);
  if (e != cudaSuccess) return cuda_fail(e, "psd training");
  rc = check_err(m);
  if (rc) return rc;
  if (loss_curve && curve_len > 0) {
    for (int k = 0; k < curve_len; k++) {
      const long long a0 = steps * k / curve_len, a1 = std::max(a0 + 1, steps * (k + 1) / curve_len);
      double s = 0;
      for (long long j = a0; j < a1 && j < steps; j++) s += hl[j];
      loss_curve[k] = (float)(s / (double)(a1 - a0));
    }
  }
  if (val_loss) *val_loss = vchunks > 0 ? hl[steps] / (float)vchunks : 0.f;
  return FFT3D_OK;
}

int fft3d_psd_train_stats(fft3d_psd* m, double out[4]) {
  if (!m || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(m->mu);
  std::copy(m->stats, m->stats + 4, out);
  return FFT3D_OK;
}

int fft3d_psd_gradients(fft3d_psd* m, const float* features, const float* target, int rows, float* grads,
                        float* loss) {
  if (!m || !features || !target || rows <= 0 || rows % 128)
    return fail(FFT3D_E_PARAM, "neo_fft3d: rows must be a positive multiple of 128");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  Work* w = work_alloc(rows, true);
  float *xf = nullptr, *tf = nullptr;
  if (!w || cudaMalloc(&xf, (size_t)rows * IN * 4) != cudaSuccess ||
      cudaMalloc(&tf, (size_t)rows * BINS * 4) != cudaSuccess) {
    cudaGetLastError();
    work_free(w);
    cudaFree(xf);
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory");
  }
  cudaStream_t s = m->stream;
  cudaError_t e = cudaMemcpyAsync(xf, features, (size_t)rows * IN * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tf, target, (size_t)rows * BINS * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = fft3d::mlp::to_bf16(xf, w->X, (long long)rows * IN, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->loss, 0, sizeof(float), s);
  if (e == cudaSuccess) e = forward(m, w, w->X, rows, s);
  if (e == cudaSuccess) e = backward(m, w, w->X, tf, rows, m->loss, s);
  if (e == cudaSuccess && grads) e = cudaMemcpyAsync(grads, m->g, NPARAM * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  work_free(w);
  cudaFree(xf);
  cudaFree(tf);
  if (e != cudaSuccess) return cuda_fail(e, "psd gradients");
  return check_err(m);
}

int fft3d_psd_forward(fft3d_psd* m, const float* features, int rows, float* out) {
  if (!m || !features || !out || rows <= 0) return fail(FFT3D_E_PARAM, "neo_fft3d: invalid rows");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  const long long R = (rows + 127) / 128 * 128;
  Work* w = work_alloc(R, false);
  float* xf = nullptr;
  if (!w || cudaMalloc(&xf, (size_t)R * IN * 4) != cudaSuccess) {
    cudaGetLastError();
    work_free(w);
    return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory");
  }
  cudaStream_t s = m->stream;
  cudaError_t e = cudaMemsetAsync(xf, 0, (size_t)R * IN * 4, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xf, features, (size_t)rows * IN * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = fft3d::mlp::to_bf16(xf, w->X, R * IN, s);
  if (e == cudaSuccess) e = forward(m, w, w->X, R, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(out, BINS * 4, w->Y, OUT * 4, BINS * 4, rows, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  work_free(w);
  cudaFree(xf);
  if (e != cudaSuccess) return cuda_fail(e, "psd forward");
  return check_err(m);
}

}  // extern "C"
