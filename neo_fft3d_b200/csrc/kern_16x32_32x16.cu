// Kernel instantiations for block sizes (bw x bh): 16 32, 32 16.
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(16, 32)
FFT3D_REGISTER_SIZE(32, 16)
}  // namespace fft3d
