// Launchers of the learned noise-PSD model's kernels (mlp_kernels.cu).
#pragma once
#include <cuda_runtime.h>

namespace fft3d {
namespace mlp {

// Tile of the BF16 tensor-core GEMM: M % 128 == 0, N % 64 == 0, K % 64 == 0.
constexpr int kTileM = 128, kTileN = 64, kTileK = 64;
inline bool gemm_shape_ok(long long M, long long N, long long K) {
  return M > 0 && N > 0 && K > 0 && M % kTileM == 0 && N % kTileN == 0 && K % kTileK == 0;
}

// C[m*ldc + n] (=|+=) sum_k A[m*sam + k*sak] * B[n*sbn + k*sbk]; A, B BF16,
// C FP32; FP32 accumulation in tensor memory. `err` (device int) gets bit 0
// when a bounded wait on the MMA completion barrier runs out.
cudaError_t gemm_bf16(const void* A, long long sam, long long sak, const void* B, long long sbn, long long sbk,
                      float* C, long long ldc, int M, int N, int K, bool accumulate, int* err, cudaStream_t s);

// Z = C + bias (per column); H = bf16(gelu(Z) or Z). Z and H may be null; Z may alias C.
cudaError_t bias_act(const float* C, const float* bias, float* Z, void* H, long long rows, int cols, bool gelu,
                     cudaStream_t s);
// dZ = dH * gelu'(Z); dZb = bf16(dZ). dZ may alias dH.
cudaError_t gelu_back(const float* dH, const float* Z, float* dZ, void* dZb, long long n, cudaStream_t s);
// Mean squared error of Y[:, :valid] (row stride ldy) against T (row stride
// ldt); dY = 2 (Y - T) / (rows * valid), zero in the padding columns.
// `loss` (device float) is incremented by the mean.
cudaError_t mse_grad(const float* Y, int ldy, const float* T, int ldt, float* dY, void* dYb, long long rows, int valid,
                     float* loss, cudaStream_t s);
// out[c] = sum_r X[r*cols + c] in a fixed order; `partial` holds
// colsum_partial_floats(rows, cols) floats.
long long colsum_partial_floats(long long rows, int cols);
cudaError_t colsum(const float* X, float* partial, float* out, long long rows, int cols, float scale, cudaStream_t s);
// Adam step (bias-corrected) on FP32 master weights; wb (BF16 copy) may be null.
cudaError_t adam(float* w, const float* g, float* m, float* v, void* wb, long long n, float lr, float b1, float b2,
                 float eps, int step, cudaStream_t s);
cudaError_t to_bf16(const float* x, void* y, long long n, cudaStream_t s);
// dst [cols][rows] = transpose of src [rows][cols] (BF16)
cudaError_t transpose_bf16(const void* src, void* dst, int rows, int cols, cudaStream_t s);

}  // namespace mlp
}  // namespace fft3d
