// Kernel instantiations for block sizes: 16 16;8 8;12 12;24 24 (bw bh).
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(16, 16)
FFT3D_REGISTER_SIZE(8, 8)
FFT3D_REGISTER_SIZE(12, 12)
FFT3D_REGISTER_SIZE(24, 24)
}  // namespace fft3d
