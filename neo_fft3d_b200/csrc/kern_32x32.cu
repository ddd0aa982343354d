// Kernel instantiations for block sizes: 32 32 (bw bh).
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(32, 32)
}  // namespace fft3d
