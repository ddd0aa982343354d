// Kernel instantiations for block sizes: 32 48;48 32;24 32;32 24;16 48;48 16 (bw bh).
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(32, 48)
FFT3D_REGISTER_SIZE(48, 32)
FFT3D_REGISTER_SIZE(24, 32)
FFT3D_REGISTER_SIZE(32, 24)
FFT3D_REGISTER_SIZE(16, 48)
FFT3D_REGISTER_SIZE(48, 16)
}  // namespace fft3d
