// Kernel instantiations for block sizes (bw x bh): 16 48, 48 16.
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(16, 48)
FFT3D_REGISTER_SIZE(48, 16)
}  // namespace fft3d
