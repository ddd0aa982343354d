// Kernel instantiations for block sizes (bw x bh): 32 48, 48 32.
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(32, 48)
FFT3D_REGISTER_SIZE(48, 32)
}  // namespace fft3d
