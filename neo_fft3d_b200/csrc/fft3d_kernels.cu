// Size table, overlap-add kernel and launch dispatch of the FFT3D filtering
// core; the FFT kernels themselves are instantiated in kern_*.cu.
#include <algorithm>
#include <mutex>
#include <vector>

#include "fft3d_kernels.cuh"
#include "fft3d_kernels_impl.cuh"
#include "kern_registry.h"

#include <set>
#include <tuple>

namespace fft3d {

cudaError_t set_smem_attr(const void* func, int bytes, bool prefer_shared) {
  static std::mutex mu;
  static std::set<std::tuple<const void*, int, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(func, dev, bytes);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(key)) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && prefer_shared)
    e = cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) done.insert(key);
  return e;
}

namespace {

std::vector<SizeEntry>& table() {
  static std::vector<SizeEntry> t;
  return t;
}

constexpr int kOlaTx = 32, kOlaTy = 8;
constexpr int kOla4BatchRows = 4 * kOlaTy;  // rows of one batched 4-pixel overlap-add item

template <typename T>
__global__ void __launch_bounds__(kOlaTx * kOlaTy) k_overlap_add4(OlaArgs a) {
  overlap_add_px4<T>(a, 4 * (blockIdx.x * blockDim.x + threadIdx.x), blockIdx.y * blockDim.y + threadIdx.y);
}

// Frame blockIdx.z of a frame group (fs): its blocks and destination.
template <typename T>
__global__ void __launch_bounds__(kOlaTx * kOlaTy) k_overlap_add4_frames(OlaArgs a, OlaFrameSet fs) {
  const int j = blockIdx.z;
  OlaArgs b = a;
#pragma unroll
  for (int q = 0; q < kMaxGroupFrames; q++)
    if (q == j) {
      b.tdom = fs.tdom[q];
      b.dst = fs.dst[q];
      b.dst_stride = fs.dst_stride[q];
    }
  overlap_add_px4<T>(b, 4 * (blockIdx.x * blockDim.x + threadIdx.x), blockIdx.y * blockDim.y + threadIdx.y);
}

template <typename T>
__global__ void __launch_bounds__(kOlaTx * kOlaTy) k_overlap_add(OlaArgs a) {
  overlap_add_px<T>(a, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

// Batched overlap-add: work item = (plane, 32x8 tile in row-major tile order).
template <typename T>
__global__ void __launch_bounds__(kOlaTx * kOlaTy) k_overlap_add_batch(const OlaArgs* __restrict__ args,
                                                                      const int2* __restrict__ items, int nitems) {
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    const OlaArgs a = args[it.x];  // private copy: fields stay in registers
    const int tx = (a.g.W + kOlaTx - 1) / kOlaTx;
    const int ty = it.y / tx, t = it.y - ty * tx;
    overlap_add_px<T>(a, t * kOlaTx + threadIdx.x, ty * kOlaTy + threadIdx.y);
  }
}

// Batched 4-pixel overlap-add: work item = (plane, 128x8-pixel tile); every
// plane of the launch meets the 4-pixel kernel's geometry and alignment rules
// (batch_overlap_add4_ok).
template <typename T>
__global__ void __launch_bounds__(kOlaTx * kOlaTy) k_overlap_add4_batch(const OlaArgs* __restrict__ args,
                                                                       const int2* __restrict__ items, int nitems) {
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    const OlaArgs a = args[it.x];  // private copy: fields stay in registers
    const int tx = (a.g.W + 4 * kOlaTx - 1) / (4 * kOlaTx);
    const int ty = it.y / tx, t = it.y - ty * tx;
    // kOla4BatchRows rows per item, so that the argument loads are shared by
    // several pixel quads per thread
#pragma unroll
    for (int r = 0; r < kOla4BatchRows; r += kOlaTy)
      overlap_add_px4<T>(a, 4 * (t * kOlaTx + threadIdx.x), ty * kOla4BatchRows + r + threadIdx.y);
  }
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

cudaError_t launch_forward_frames(const ForwardArgs& a, const FwdFrameSet& fs, int bytes, cudaStream_t s) {
  const SizeEntry* e = find_size(a.g.bw, a.g.bh);
  return e ? e->fwd_frames(a, fs, bytes, s) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_inverse_frames(const InverseArgs& a, const FrameSet& fs, int mode, cudaStream_t s) {
  const SizeEntry* e = find_size(a.g.bw, a.g.bh);
  return e ? e->inv_frames(a, fs, mode, s) : cudaErrorInvalidValue;
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

cudaError_t launch_filter_inverse_group(const InverseArgs& a, const TemporalSet& ts, int mode, cudaStream_t s,
                                        const OlaFuse* of) {
  const SizeEntry* e = find_size(a.g.bw, a.g.bh);
  return e ? e->inv_group(a, ts, mode, s, of) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_frames(const InverseArgs& a, const FilterFrameSet& fs, int mode, cudaStream_t s) {
  if (fs.count < 1 || fs.count > kMaxGroupFrames) return cudaErrorInvalidValue;
  const int bins = a.g.bh * a.g.nh;
  const size_t pairs = (size_t)a.g.nblocks * bins / 2;
  const int grid = (int)((pairs + 255) / 256);
  switch (mode) {
    case MODE_KALMAN: k_filter_frames<MODE_KALMAN><<<grid, 256, 0, s>>>(a, fs, bins); break;
    case 1: k_filter_frames<1><<<grid, 256, 0, s>>>(a, fs, bins); break;
    case 2: k_filter_frames<2><<<grid, 256, 0, s>>>(a, fs, bins); break;
    case 3: k_filter_frames<3><<<grid, 256, 0, s>>>(a, fs, bins); break;
    case 4: k_filter_frames<4><<<grid, 256, 0, s>>>(a, fs, bins); break;
    case 5: k_filter_frames<5><<<grid, 256, 0, s>>>(a, fs, bins); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_fused(const FusedArgs& a, int mode, int bytes, cudaStream_t s) {
  const SizeEntry* e = find_size(a.v.g.bw, a.v.g.bh);
  return e ? e->fused(a, mode, bytes, s) : cudaErrorInvalidValue;
}

cudaError_t launch_forward_batch(int bw, int bh, const BatchLaunch& l, int bytes, cudaStream_t s) {
  const SizeEntry* e = find_size(bw, bh);
  return e ? e->fwd_batch(l, bytes, s) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_inverse_batch(int bw, int bh, const BatchLaunch& l, int mode, cudaStream_t s) {
  const SizeEntry* e = find_size(bw, bh);
  return e ? e->inv_batch(l, mode, s) : cudaErrorInvalidValue;
}

cudaError_t launch_filter_inverse_group_batch(int bw, int bh, const BatchLaunch& l, int mode, cudaStream_t s) {
  const SizeEntry* e = find_size(bw, bh);
  return e ? e->inv_group_batch(l, mode, s) : cudaErrorInvalidValue;
}

cudaError_t launch_overlap_add_batch(const BatchLaunch& l, int bytes, cudaStream_t s) {
  dim3 block(kOlaTx, kOlaTy);
  const auto* args = static_cast<const OlaArgs*>(l.args);
  if (bytes >= kOla4Var) {  // the 4-pixel form
    bytes -= kOla4Var;
    if (bytes == 1) k_overlap_add4_batch<uint8_t><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
    else if (bytes == 2) k_overlap_add4_batch<uint16_t><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
    else k_overlap_add4_batch<float><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
    return cudaGetLastError();
  }
  if (bytes == 1) k_overlap_add_batch<uint8_t><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
  else if (bytes == 2) k_overlap_add_batch<uint16_t><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
  else k_overlap_add_batch<float><<<l.grid, block, 0, s>>>(args, l.items, l.nitems);
  return cudaGetLastError();
}

// Batched plane copies: work item = (copy, row); 16-byte moves when both
// rows are 16-byte aligned, bytes otherwise.
__global__ void __launch_bounds__(256) k_copy_batch(const CopyArgs* __restrict__ args, const int2* __restrict__ items,
                                                    int nitems) {
  for (int i = blockIdx.x; i < nitems; i += gridDim.x) {
    const int2 it = items[i];
    const CopyArgs c = args[it.x];
    const char* s = static_cast<const char*>(c.src) + (long long)it.y * c.spitch;
    char* d = static_cast<char*>(c.dst) + (long long)it.y * c.dpitch;
    if ((((uintptr_t)s | (uintptr_t)d) & 15) == 0) {
      const long long n16 = c.width / 16;
      for (long long x = threadIdx.x; x < n16; x += blockDim.x)
        reinterpret_cast<uint4*>(d)[x] = reinterpret_cast<const uint4*>(s)[x];
      for (long long x = n16 * 16 + threadIdx.x; x < c.width; x += blockDim.x) d[x] = s[x];
    } else {
      for (long long x = threadIdx.x; x < c.width; x += blockDim.x) d[x] = s[x];
    }
  }
}

cudaError_t launch_copy_batch(const BatchLaunch& l, cudaStream_t s) {
  k_copy_batch<<<l.grid, 256, 0, s>>>(static_cast<const CopyArgs*>(l.args), l.items, l.nitems);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(128) k_pattern_scores(const float2* __restrict__ spec,
                                                        const float2* __restrict__ grid,
                                                        const float* __restrict__ pwin, int nox, int noy,
                                                        int bins, float degrid, float* scores) {
  const int wx = nox - 4, wy = noy - 4;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= wx * wy) return;
  const int by = 2 + i / wx, bx = 2 + i % wx;
  const float2* s = spec + ((size_t)by * nox + bx) * bins;
  const float gcur = __fdiv_rn(__fmul_rn(degrid, s[0].x), grid[0].x);
  float acc = 0.f;
  for (int k = 0; k < bins; k++) {
    const float2 v = s[k], gs = grid[k];
    const float c0 = __fsub_rn(v.x, __fmul_rn(gcur, gs.x)), c1 = __fsub_rn(v.y, __fmul_rn(gcur, gs.y));
    acc = __fadd_rn(acc, __fmul_rn(__fadd_rn(__fmul_rn(c0, c0), __fmul_rn(c1, c1)), pwin[k]));
  }
  scores[i] = acc;
}

cudaError_t launch_pattern_scores(const float2* spec, const float2* grid, const float* pwin, int nox, int noy,
                                  int bins, float degrid, float* scores, cudaStream_t s) {
  const int n = (nox - 4) * (noy - 4);
  if (n <= 0) return cudaSuccess;
  k_pattern_scores<<<(n + 127) / 128, 128, 0, s>>>(spec, grid, pwin, nox, noy, bins, degrid, scores);
  return cudaGetLastError();
}

int batch_items_forward(const Geom& g) {
  const SizeEntry* e = find_size(g.bw, g.bh);
  return e ? e->ctas(g.nblocks) : 0;
}

int batch_items_overlap_add(const Geom& g) {
  return ((g.W + kOlaTx - 1) / kOlaTx) * ((g.H + kOlaTy - 1) / kOlaTy);
}

int batch_items_overlap_add4(const Geom& g) {
  return ((g.W + 4 * kOlaTx - 1) / (4 * kOlaTx)) * ((g.H + kOla4BatchRows - 1) / kOla4BatchRows);
}

bool batch_overlap_add4_ok(const OlaArgs& a, int bytes) {
  return a.g.sx % 4 == 0 && a.g.ow % 4 == 0 && a.g.W % 4 == 0 && a.g.bw % 4 == 0 &&
         reinterpret_cast<uintptr_t>(a.tdom) % 16 == 0 && reinterpret_cast<uintptr_t>(a.dst) % (4 * bytes) == 0 &&
         a.dst_stride % (4 * bytes) == 0;
}

int batch_occupancy(int bw, int bh, int which, int mode_or_bytes) {
  if (which == 4) return 8;  // plane copies
  if (which == 2) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_overlap_add_batch<uint8_t>, kOlaTx * kOlaTy, 0);
    return n > 0 ? n : 1;
  }
  const SizeEntry* e = find_size(bw, bh);
  return e ? e->occupancy(which, mode_or_bytes) : 1;
}

bool overlap_add_frames_supported(const OlaArgs& a, const OlaFrameSet& fs, int bytes) {
  if (fs.count < 1 || fs.count > kMaxGroupFrames) return false;
  bool four = a.g.sx % 4 == 0 && a.g.ow % 4 == 0 && a.g.W % 4 == 0 && a.g.bw % 4 == 0;
  for (int j = 0; j < fs.count && four; j++)
    four = reinterpret_cast<uintptr_t>(fs.tdom[j]) % 16 == 0 &&
           reinterpret_cast<uintptr_t>(fs.dst[j]) % (4 * bytes) == 0 && fs.dst_stride[j] % (4 * bytes) == 0;
  return four;
}

__global__ void k_fill(float* p, float v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

cudaError_t launch_fill(float* p, float v, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
  k_fill<<<grid, 256, 0, s>>>(p, v, n);
  return cudaGetLastError();
}

cudaError_t launch_overlap_add_frames(const OlaArgs& a, const OlaFrameSet& fs, int bytes, cudaStream_t s) {
  if (!overlap_add_frames_supported(a, fs, bytes)) return cudaErrorNotSupported;
  dim3 block(kOlaTx, kOlaTy);
  dim3 grid((a.g.W / 4 + kOlaTx - 1) / kOlaTx, (a.g.H + kOlaTy - 1) / kOlaTy, fs.count);
  if (bytes == 1) k_overlap_add4_frames<uint8_t><<<grid, block, 0, s>>>(a, fs);
  else if (bytes == 2) k_overlap_add4_frames<uint16_t><<<grid, block, 0, s>>>(a, fs);
  else k_overlap_add4_frames<float><<<grid, block, 0, s>>>(a, fs);
  return cudaGetLastError();
}

cudaError_t launch_overlap_add(const OlaArgs& a, int bytes, cudaStream_t s) {
  dim3 block(kOlaTx, kOlaTy);
  const bool four = a.g.sx % 4 == 0 && a.g.ow % 4 == 0 && a.g.W % 4 == 0 && a.g.bw % 4 == 0 &&
                    reinterpret_cast<uintptr_t>(a.tdom) % 16 == 0 &&
                    reinterpret_cast<uintptr_t>(a.dst) % (4 * bytes) == 0 && a.dst_stride % (4 * bytes) == 0;
  if (four) {
    dim3 grid((a.g.W / 4 + kOlaTx - 1) / kOlaTx, (a.g.H + kOlaTy - 1) / kOlaTy);
    if (bytes == 1) k_overlap_add4<uint8_t><<<grid, block, 0, s>>>(a);
    else if (bytes == 2) k_overlap_add4<uint16_t><<<grid, block, 0, s>>>(a);
    else k_overlap_add4<float><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
  }
  dim3 grid((a.g.W + kOlaTx - 1) / kOlaTx, (a.g.H + kOlaTy - 1) / kOlaTy);
  if (bytes == 1) k_overlap_add<uint8_t><<<grid, block, 0, s>>>(a);
  else if (bytes == 2) k_overlap_add<uint16_t><<<grid, block, 0, s>>>(a);
  else k_overlap_add<float><<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace fft3d
