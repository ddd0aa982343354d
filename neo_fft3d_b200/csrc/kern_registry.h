// Table of the block sizes compiled into the library. Each kern_*.cu
// translation unit instantiates the kernels of a few sizes and registers them
// here at load time (FFT3D_REGISTER_SIZE in fft3d_kernels_impl.cuh).
#pragma once
#include <cuda_runtime.h>

#include "fft3d_kernels.cuh"

namespace fft3d {

struct SizeEntry {
  int bw, bh;
  cudaError_t (*fwd)(const ForwardArgs&, int bytes_per_sample, cudaStream_t);
  cudaError_t (*inv)(const InverseArgs&, int mode, cudaStream_t);
  cudaError_t (*fused)(const FusedArgs&, int mode, int bytes_per_sample, cudaStream_t);
  cudaError_t (*upload)();  // the translation unit's twiddle table, once per device
  // batched launches over many planes (fft3d_batch.cu)
  cudaError_t (*fwd_batch)(const BatchLaunch&, int bytes_per_sample, cudaStream_t);
  cudaError_t (*inv_batch)(const BatchLaunch&, int mode, cudaStream_t);
  int (*ctas)(int nblocks);                       // work items (CTAs) per plane
  int (*occupancy)(int which, int mode_or_bytes);  // resident CTAs per SM: 0 forward, 1 filter/inverse
  // frame groups (Wiener 3D modes 2..5): several output frames in one launch
  cudaError_t (*inv_frames)(const InverseArgs&, const FrameSet&, int mode, cudaStream_t);
  // and their new frames' forward transforms in one launch
  cudaError_t (*fwd_frames)(const ForwardArgs&, const FwdFrameSet&, int bytes_per_sample, cudaStream_t);
  // a run of frames filtered and inverse-transformed with one CTA per block
  cudaError_t (*inv_group)(const InverseArgs&, const TemporalSet&, int mode, cudaStream_t, const OlaFuse*);
  // and its batched form over the runs of many planes
  cudaError_t (*inv_group_batch)(const BatchLaunch&, int mode, cudaStream_t);
};

bool register_size(const SizeEntry& e);
const SizeEntry* find_size(int bw, int bh);
int registered_sizes(SizeEntry* out, int max);

}  // namespace fft3d
