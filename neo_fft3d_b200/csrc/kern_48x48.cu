// Kernel instantiations for block sizes: 48 48 (bw bh).
#include "fft3d_kernels_impl.cuh"

namespace fft3d {
FFT3D_REGISTER_SIZE(48, 48)
}  // namespace fft3d
