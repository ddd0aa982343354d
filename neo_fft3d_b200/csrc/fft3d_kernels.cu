// Size table, overlap-add kernel and launch dispatch of the FFT3D filtering
// core; the FFT kernels themselves are instantiated in kern_*.cu.
#include <algorithm>
#include <mutex>
#include <vector>

#include "fft3d_kernels.cuh"
#include "fft3d_kernels_impl.cuh"
#include "kern_registry.h"

namespace fft3d {

namespace {

std::vector<SizeEntry>& table() {
  static std::vector<SizeEntry> t;
  return t;
}

template <typename T>
__device__ __forceinline__ void store_sample(T* p, float v, int maxval);
template <>
__device__ __forceinline__ void store_sample<uint8_t>(uint8_t* p, float v, int maxval) {
  int i = __float2int_rz(v);  // C cast: truncation toward zero (src/buffer.cpp:406)
  i = i < 0 ? 0 : (i > maxval ? maxval : i);
  *p = (uint8_t)i;
}
template <>
__device__ __forceinline__ void store_sample<uint16_t>(uint16_t* p, float v, int maxval) {
  int i = __float2int_rz(v);
  i = i < 0 ? 0 : (i > maxval ? maxval : i);
  *p = (uint16_t)i;
}
template <>
__device__ __forceinline__ void store_sample<float>(float* p, float v, int) {
  float c = v < 0.f ? 0.f : v;  // float samples clamp to [0, 1] (src/buffer.cpp:397)
  *p = c > 1.f ? 1.f : c;
}

// One thread per output pixel of the processed region: the (at most four)
// blocks covering it, weighted with the synthesis windows and the FFT
// normalisation in the association order of src/buffer.cpp:399-559.
template <typename T>
__global__ void k_overlap_add(OlaArgs a) {
  const Geom& g = a.g;
  const int x0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y * blockDim.y + threadIdx.y;
  if (x0 >= g.W || k >= g.H) return;
  const int Y = g.sy + k, X = g.sx + x0;
  const int by = Y / g.sy, y = Y - by * g.sy;
  const int bx = X / g.sx, x = X - bx * g.sx;
  const bool yov = y < g.oh, xov = x < g.ow;
  const int bw = g.bw, bh = g.bh;
  auto at = [&](int bxx, int byy, int yy, int xx) {
    return __ldg(a.tdom + ((size_t)(byy * g.nox + bxx) * bh + yy) * bw + xx);
  };
  const float norm = a.norm;
  float v;
  if (!yov) {
    const float d = at(bx, by, y, x);
    if (!xov) v = d * norm + a.rounder + a.base;
    else {
      const float c = at(bx - 1, by, y, x + g.sx);
      v = (c * __ldg(a.t.wsyn_xr + x) + d * __ldg(a.t.wsyn_xl + x)) * norm + a.rounder + a.base;
    }
  } else {
    const float wr = __ldg(a.t.wsyn_yr + y) * norm, wl = __ldg(a.t.wsyn_yl + y) * norm;
    const float b = at(bx, by - 1, y + g.sy, x), d = at(bx, by, y, x);
    if (!xov) v = (b * wr + d * wl) + a.rounder + a.base;
    else {
      const float aa = at(bx - 1, by - 1, y + g.sy, x + g.sx), c = at(bx - 1, by, y, x + g.sx);
      const float sxr = __ldg(a.t.wsyn_xr + x), sxl = __ldg(a.t.wsyn_xl + x);
      v = ((aa * sxr + b * sxl) * wr + (c * sxr + d * sxl) * wl) + a.rounder + a.base;
    }
  }
  T* row = reinterpret_cast<T*>(static_cast<char*>(a.dst) + (long long)field_row(k, g.H, g.interlaced) * a.dst_stride);
  store_sample<T>(row + x0, v, a.maxval);
}

}  // namespace

bool register_size(const SizeEntry& e) {
  table().push_back(e);
  return true;
}

const SizeEntry* find_size(int bw, int bh) {
  for (const auto& e : table())
    if (e.bw == bw && e.bh == bh) return &e;
  return nullptr;
}

int registered_sizes(SizeEntry* out, int max) {
  int n = 0;
  for (const auto& e : table())
    if (n < max) out[n++] = e;
  return (int)table().size();
}

bool block_size_supported(int bw, int bh) { return find_size(bw, bh) != nullptr; }

cudaError_t upload_twiddles() {
  for (const auto& e : table()) {
    cudaError_t err = e.upload();
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

cudaError_t launch_forward(const ForwardArgs& a, int bytes, cudaStream_t s) {
  const SizeEntry* e = find_size(a.g.bw, a.g.bh);
  return e ? e->fwd(a, bytes, s) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_inverse(const InverseArgs& a, int mode, cudaStream_t s) {
  const SizeEntry* e = find_size(a.g.bw, a.g.bh);
  return e ? e->inv(a, mode, s) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_bins(const InverseArgs& a, float2* F, int mode, cudaStream_t s) {
  const int bins = a.g.bh * a.g.nh;
  const size_t pairs = (size_t)a.g.nblocks * bins / 2;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<size_t>((pairs + 255) / 256, (size_t)sms * 8);
  switch (mode) {
    case MODE_KALMAN: k_filter_bins<MODE_KALMAN><<<grid, 256, 0, s>>>(a, F, bins); break;
    case 1: k_filter_bins<1><<<grid, 256, 0, s>>>(a, F, bins); break;
    case 2: k_filter_bins<2><<<grid, 256, 0, s>>>(a, F, bins); break;
    case 3: k_filter_bins<3><<<grid, 256, 0, s>>>(a, F, bins); break;
    case 4: k_filter_bins<4><<<grid, 256, 0, s>>>(a, F, bins); break;
    case 5: k_filter_bins<5><<<grid, 256, 0, s>>>(a, F, bins); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_fused(const FusedArgs& a, int mode, int bytes, cudaStream_t s) {
  const SizeEntry* e = find_size(a.v.g.bw, a.v.g.bh);
  return e ? e->fused(a, mode, bytes, s) : cudaErrorInvalidValue;
}

cudaError_t launch_overlap_add(const OlaArgs& a, int bytes, cudaStream_t s) {
  dim3 block(32, 8);
  dim3 grid((a.g.W + 31) / 32, (a.g.H + 7) / 8);
  if (bytes == 1) k_overlap_add<uint8_t><<<grid, block, 0, s>>>(a);
  else if (bytes == 2) k_overlap_add<uint16_t><<<grid, block, 0, s>>>(a);
  else k_overlap_add<float><<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace fft3d
