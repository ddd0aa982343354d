// One-time kernel attribute setting.
#pragma once
#include <cuda_runtime.h>

namespace fft3d {

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device,
// size): launchers call this before every launch, and the runtime call itself
// costs host time that per-frame launch sequences cannot afford.
// prefer_shared: also ask for the largest shared-memory carveout (kernels
// whose resident CTAs are capped by their shared-memory tiles; the FP32 FFT
// kernels keep the default, whose larger L1 holds their loads in flight).
cudaError_t set_smem_attr(const void* func, int bytes, bool prefer_shared);

template <typename K>
inline cudaError_t smem_attr(K* kernel, int bytes, bool prefer_shared = false) {
  return set_smem_attr(reinterpret_cast<const void*>(kernel), bytes, prefer_shared);
}

}  // namespace fft3d
