// Kernel instantiations for block sizes: 16 32;32 16;16 24;24 16 (bw bh).
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(16, 32)
FFT3D_REGISTER_SIZE(32, 16)
FFT3D_REGISTER_SIZE(16, 24)
FFT3D_REGISTER_SIZE(24, 16)
}  // namespace fft3d
