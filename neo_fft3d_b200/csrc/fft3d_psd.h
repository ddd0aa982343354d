// Engine-side interface of the learned noise-PSD model (fft3d_psd.cu).
#pragma once
#include <string>

#include <cuda_runtime.h>

#include "fft3d_b200.h"

namespace fft3d {
namespace psd {

// Per-plane inference scratch (features, activations, pooled sums).
struct Work;

// Empty when a plane of this geometry can use the model, else the reason.
std::string check_plane(const fft3d_psd* m, int device, int bw, int bh, int ow, int oh, int wintype);
Work* work_create(fft3d_psd* m, int nblocks);  // null when device memory runs out
void work_destroy(Work* w);
// Noise power of every bin of every block from the blocks' spectra
// (nblocks x 544 complex): out[b * 544 + k], or out[k] for all blocks when
// pooled (exp of the mean log prediction). pow_scale: the square of the
// plane's sample scale relative to 8-bit samples (4^(bits-8) for integer
// formats); the model sees power / pow_scale and its output is scaled back.
cudaError_t infer(fft3d_psd* m, Work* w, const float2* spec, int nblocks, bool pooled, float pow_scale, float* out,
                  cudaStream_t s);
// Device flag set by the model's tensor-core kernels when a bounded wait runs out.
int* err_flag(fft3d_psd* m);

}  // namespace psd
}  // namespace fft3d
