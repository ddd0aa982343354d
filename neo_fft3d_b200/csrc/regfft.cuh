// Register-resident mixed-radix FFTs for one thread (sm_100a).
//
// Every transform length is a compile-time constant, every loop is fully
// unrolled, so the data array lives in registers and every twiddle index is a
// constant: the twiddles are read from a __constant__ table whose operands the
// FFMA instructions take directly (constant-bank operands), with no loads.
//
// Algorithm: Stockham self-sorting passes (natural order in and out) with
// radix 4, 2 and 3 butterflies:
//   Y[j + L q + L P k] = sum_u W_P^{q u} (W_{L P}^{j u} X[j + L (k + R u)])
// for pass radix P, L = product of the earlier radices, R = N / (L P).
// Lengths: any N = 2^a 3^b dividing kTwN (384), so 2..128, 6, 12, 24, 48, 96.
#pragma once
#include <cuda_runtime.h>

namespace fft3d {

constexpr int kTwN = 384;  // W_384^k = exp(-2 pi i k / 384), k < 384
// One copy per translation unit (whole-program compilation keeps __constant__
// memory per module); each TU that includes this header uploads it with
// upload_twiddle_table() once per device.
static __constant__ float2 c_tw[kTwN];

static inline cudaError_t upload_twiddle_table() {
  float2 h[kTwN];
  for (int k = 0; k < kTwN; k++) {
    double a = -2.0 * 3.14159265358979323846 * (double)k / (double)kTwN;
    h[k] = make_float2((float)__builtin_cos(a), (float)__builtin_sin(a));
  }
  return cudaMemcpyToSymbol(c_tw, h, sizeof(h));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Complex adds as packed f32x2 operations (one instruction for both parts,
// each part rounded exactly as a scalar add).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// W_N^m for SIGN = -1 (forward) or its conjugate for SIGN = +1.
template <int N, int SIGN>
__device__ __forceinline__ float2 tw(int m) {
  static_assert(kTwN % N == 0, "transform length must divide 384");
  float2 w = c_tw[(m % N) * (kTwN / N)];
  return SIGN < 0 ? w : cconj(w);
}

// small DFTs in place, sign SIGN
template <int P, int SIGN>
__device__ __forceinline__ void small_dft(float2 (&t)[P]) {
  if constexpr (P == 2) {
    float2 a = t[0], b = t[1];
    t[0] = cadd(a, b);
    t[1] = csub(a, b);
  } else if constexpr (P == 4) {
    float2 s02 = cadd(t[0], t[2]), d02 = csub(t[0], t[2]);
    float2 s13 = cadd(t[1], t[3]), d13 = csub(t[1], t[3]);
    // d13 * (SIGN * i)
    float2 j = SIGN < 0 ? make_float2(d13.y, -d13.x) : make_float2(-d13.y, d13.x);
    t[0] = cadd(s02, s13);
    t[1] = cadd(d02, j);
    t[2] = csub(s02, s13);
    t[3] = csub(d02, j);
  } else if constexpr (P == 3) {
    const float c = -0.5f;
    const float s = SIGN < 0 ? -0.86602540378443864676f : 0.86602540378443864676f;
    float2 a = t[0], b = t[1], d = t[2];
    float2 sum = cadd(b, d), dif = csub(b, d);
    float2 m = make_float2(a.x + c * sum.x, a.y + c * sum.y);
    // i * s * dif
    float2 r = make_float2(-s * dif.y, s * dif.x);
    t[0] = cadd(a, sum);
    t[1] = cadd(m, r);
    t[2] = csub(m, r);
  }
}

template <int N>
struct Radices {
  // first radix used for length N in the recursion below (4 while N%4==0 and N>=16 or N==4)
  static constexpr int first = (N % 4 == 0) ? 4 : ((N % 2 == 0) ? 2 : 3);
};

template <int N, int SIGN, int L>
__device__ __forceinline__ void stockham(float2 (&x)[N]) {
  if constexpr (L < N) {
    constexpr int rem = N / L;
    constexpr int P = Radices<rem>::first;
    constexpr int R = N / (L * P);
    float2 y[N];
#pragma unroll
    for (int k = 0; k < R; k++) {
#pragma unroll
      for (int j = 0; j < L; j++) {
        float2 t[P];
#pragma unroll
        for (int u = 0; u < P; u++) {
          float2 a = x[j + L * (k + R * u)];
          if (j * u != 0) a = cmul(a, tw<N, SIGN>(j * u * R));  // W_{LP}^{ju} = W_N^{ju R}
          t[u] = a;
        }
        small_dft<P, SIGN>(t);
#pragma unroll
        for (int q = 0; q < P; q++) y[j + L * q + L * P * k] = t[q];
      }
    }
#pragma unroll
    for (int i = 0; i < N; i++) x[i] = y[i];
    stockham<N, SIGN, L * P>(x);
  }
}

// Unnormalised complex DFT of length N in place (SIGN -1 forward, +1 inverse).
template <int N, int SIGN>
__device__ __forceinline__ void cfft(float2 (&x)[N]) {
  if constexpr (N > 1) stockham<N, SIGN, 1>(x);
}

// Real-to-complex DFT of length N (even): out[k], k = 0..N/2, through one
// complex DFT of length N/2 on z[m] = x[2m] + i x[2m+1].
template <int N>
__device__ __forceinline__ void rfft(const float (&x)[N], float2 (&out)[N / 2 + 1]) {
  constexpr int H = N / 2;
  float2 z[H];
#pragma unroll
  for (int m = 0; m < H; m++) z[m] = make_float2(x[2 * m], x[2 * m + 1]);
  cfft<H, -1>(z);
#pragma unroll
  for (int k = 0; k <= H; k++) {
    float2 zk = z[k % H], zc = cconj(z[(H - k) % H]);
    float2 e = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
    // o = (zk - zc) / (2 i)
    float2 d = csub(zk, zc);
    float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
    out[k] = (k == 0 || k == H) ? make_float2(e.x + (k == 0 ? o.x : -o.x), e.y + (k == 0 ? o.y : -o.y))
                                : cadd(e, cmul(o, tw<N, -1>(k)));
  }
}

// Complex-to-real inverse DFT of length N (unnormalised, like FFTW's c2r): the
// imaginary parts of in[0] and in[N/2] are ignored.
template <int N>
__device__ __forceinline__ void irfft(const float2 (&in)[N / 2 + 1], float (&x)[N]) {
  constexpr int H = N / 2;
  float2 z[H];
#pragma unroll
  for (int k = 0; k < H; k++) {
    float2 a = in[k], b = in[H - k];
    if (k == 0) { a.y = 0.f; b.y = 0.f; }
    float2 bc = cconj(b);
    float2 e = cadd(a, bc);
    float2 o = csub(a, bc);
    if (k != 0) o = cmul(o, tw<N, +1>(k));
    // z = e + i o
    z[k] = make_float2(e.x - o.y, e.y + o.x);
  }
  cfft<H, +1>(z);
#pragma unroll
  for (int m = 0; m < H; m++) {
    x[2 * m] = z[m].x;
    x[2 * m + 1] = z[m].y;
  }
}

}  // namespace fft3d
