// One-time kernel attribute setting.
#pragma once
#include <cuda_runtime.h>

namespace fft3d {

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device,
// size): launchers call this before every launch, and the runtime call itself
// costs host time that per-frame launch sequences cannot afford.
cudaError_t set_smem_attr(const void* func, int bytes);

template <typename K>
inline cudaError_t smem_attr(K* kernel, int bytes) {
  return set_smem_attr(reinterpret_cast<const void*>(kernel), bytes);
}

}  // namespace fft3d
