// Kernel instantiations for block sizes (bw x bh): 8 8, 12 12.
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(8, 8)
FFT3D_REGISTER_SIZE(12, 12)
}  // namespace fft3d
