// Kernel instantiations for block sizes (bw x bh): 24 32, 32 24.
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(24, 32)
FFT3D_REGISTER_SIZE(32, 24)
}  // namespace fft3d
