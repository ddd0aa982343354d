// Device kernels of the FFT3D filtering core (sm_100a, FP32 CUDA-core path).
//
// Per plane and output frame the hot path is three kernels:
//   k_forward         frame -> mirrored cover -> windowed overlapped blocks ->
//                     2D r2c FFT -> one slot of the device spectrum ring
//                     (replaces FrameToCover + CoverToOverlap + FFTW r2c,
//                     src/buffer.cpp:6-379, src/fft3d_engine.h:616-618,661-664)
//   k_filter_inverse  Wiener 2D / 3D2..3D5, Kalman or sharpen-only filter of
//                     every bin, sharpen/dehalo, 2D c2r -> time-domain blocks
//                     (replaces Apply*/Kalman/Sharpen C kernels and FFTW c2r,
//                     src/code_impl/*.cpp, src/fft3d_engine.h:669-674)
//   k_overlap_add     synthesis window, overlap-add, rounding and clamped
//                     8/16-bit (or float) write-back of the plane interior
//                     (replaces OverlapToCover + CoverToFrame, src/buffer.cpp:382-600)
//
// One warp owns one block in the two FFT kernels; its tiles are staged in
// shared memory so that every global access is coalesced.
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace fft3d {

// Geometry of one plane (after crop), see src/fft3d_engine.h:115-136.
struct Geom {
  int W, H;          // processed (cropped) plane size in pixels
  int nox, noy;      // blocks per row / column (incl. the one-block mirror margin)
  int nblocks;
  int bw, bh, ow, oh;
  int sx, sy;        // block step bw-ow, bh-oh (= mirror margins mirw, mirh)
  int nh;            // bw/2 + 1
  int interlaced;
};

// Per-plane constant tables on the device.
struct Tables {
  const float* wan_x;   // [bw] analysis window along x (wanxl | 1 | wanxr)
  const float* wan_y;   // [bh]
  const float* wsyn_xl; // [ow] synthesis windows, src/fft3d_engine.h:223-233
  const float* wsyn_xr;
  const float* wsyn_yl; // [oh]
  const float* wsyn_yr;
  const float2* grid;   // [bh*nh] gridsample, src/fft3d_engine.h:380-404
  const float* wsharpen;  // [bh*nh]
  const float* wdehalo;   // [bh*nh]
  const float* pattern2d; // [bh*nh]
  const float* pattern3d; // [bh*nh]
};

// Scalar filter constants, src/fft3d_engine.h:584-607.
struct FilterConsts {
  float sigma2n;      // btcur * sigma^2 / norm
  float sigma2n_2d;   // sigma^2 / norm (Kalman)
  float lowlimit;     // (beta - 1) / beta
  float degrid;
  float sharpen, dehalo;
  float smin2n, smax2n, ht2n;
  float kratio2;
  int pattern;        // use pattern2d / pattern3d instead of sigma
  int do_sharpen;     // run the separate sharpen/dehalo pass
  int fuse_sharpen;   // 2D only: sharpen/dehalo factors inside the Wiener factor
  int use_sharpen, use_dehalo;
};

// Bounds-checked build (the kernels compiled with -DFFT3D_CHECKED=1, into
// lib/libfft3d_b200_checked.so): FFT3D_IN(cond, err) is `cond`, and when it is
// false the access it guards is skipped and bit 2 of the device error flag is
// set, which the host-buffer calls and fft3d_plane_synchronize report. In the
// regular build it is `true` (the condition is not even evaluated).
#ifndef FFT3D_CHECKED
#define FFT3D_CHECKED 0
#endif
__device__ __forceinline__ bool checked_in(bool ok, int* err) {
  if (!ok && err) atomicOr(err, 4);
  return ok;
}
#if FFT3D_CHECKED
#define FFT3D_IN(cond, err) ::fft3d::checked_in((cond), (err))
#else
#define FFT3D_IN(cond, err) true
#endif

constexpr int kMaxBw = 64;  // largest block width the kernels are built for (48) rounded up
struct ForwardArgs {
  Geom g;
  const void* src;        // frame plane at the crop origin
  long long src_stride;   // bytes
  float base;             // 2^(bits-1) for integer chroma, else 0
  const float* wan_x;
  const float* wan_y;
  float2* spec;           // blocks x bh x nh
  int* err;               // device error flag (bounds-checked build), or null
  float wx[kMaxBw];       // wan_x by value: read through the launch parameters
                          // (constant-bank operands) by the per-plane kernels
};

struct InverseArgs {
  Geom g;
  Tables t;
  FilterConsts c;
  const float2* in[5];    // spectra of frames n-2..n+2 (null when unused)
  float2* kal_last;       // Kalman state: filtered spectrum of the previous frame
  float* kal_covar;       // covariance (identical for re and im, src/code_impl/Kalman.cpp:41-64)
  float* kal_covarp;      // process covariance
  float* tdom;            // blocks x bh x bw time-domain output
  const float* psd;       // learned noise power (null: sigma / pattern): per block
                          // [blocks][bh*nh] when psd_per_block, else [bh*nh]
  float psd_scale;        // btcur for Wiener 3D (pattern3d = bt x pattern2d), else 1
  int psd_per_block;
  int* err;               // device error flag (bit 0: a bounded tensor-core wait ran out, bit 1: a
                          // bounded bulk-copy wait, bit 2: a bounds check of the checked build)
  int bulk;               // use the bulk-staged filter/inverse kernel where it applies
  int reverse;            // walk the blocks from the end (alternated per frame so
                          // that the blocks read last stay in L2 for the next frame)
};

// The per-frame part of a frame group's filter/inverse launch: frame j's
// window spectra (slots n-2..n+2 of its InverseArgs::in) and time-domain
// buffer.
constexpr int kMaxGroupFrames = 16;
struct FrameSet {
  const float2* in[kMaxGroupFrames][5];
  float* tdom[kMaxGroupFrames];
  int count;
};

// The filter of a run of consecutive output frames n0 .. n0 + count - 1 of one
// plane with one mode in one launch (k_filter_frames): spec[s] is the
// spectrum of frame n0 - 2 + s (s < count + 4; null where no window of the
// run reaches), out[j] receives frame n0 + j's filtered spectrum (blocks x
// bh x nh complex, unpadded like the ring).
struct FilterFrameSet {
  const float2* spec[kMaxGroupFrames + 4];
  float2* out[kMaxGroupFrames];
  int count;
};

// A run of consecutive output frames n0 .. n0 + count - 1 (count <=
// kGroupTile) of one plane with one mode, filtered and inverse-transformed
// by one launch with one CTA per block (k_filter_inverse_group): spec[s] is
// the spectrum of frame n0 - 2 + s (null where no window of the run reaches),
// tdom[j] receives frame n0 + j's time-domain blocks.
constexpr int kGroupTile = 8;
// Frames of one run for bw x bh blocks: up to kGroupTile, fewer where the
// run's spectrum tiles (bh x (bw/2+1) complex per frame) would keep fewer
// than 4 CTAs resident per SM (48 x 48 blocks: 5 frames, 4 CTAs instead of
// 2 with 8 frames).
__host__ __device__ constexpr int group_run_frames(int bw, int bh) {
  return ((228 * 1024 / 4 - 1024 - 2 * kGroupTile * 4) / (bh * (bw / 2 + 1) * 8)) < kGroupTile
             ? ((228 * 1024 / 4 - 1024 - 2 * kGroupTile * 4) / (bh * (bw / 2 + 1) * 8))
             : kGroupTile;
}
struct TemporalSet {
  const float2* spec[kGroupTile + 4];
  float* tdom[kGroupTile];
  int count;
};

// One run of a batched step's frame groups (work items: its plane's blocks).
struct GroupRun {
  InverseArgs a;
  TemporalSet ts;
};

// The new frames of a frame group, transformed by one launch: frame j's
// samples (src/stride as in ForwardArgs) and ring slot. ctas: CTAs per frame
// (set by the launcher).
constexpr int kMaxFwdFrames = kMaxGroupFrames + 4;
struct FwdFrameSet {
  const void* src[kMaxFwdFrames];
  long long stride[kMaxFwdFrames];
  float2* spec[kMaxFwdFrames];
  int count;
  int ctas;
};

// The overlap-adds of a frame group in one launch: frame j's time-domain
// blocks and destination plane (at the crop origin).
struct OlaFrameSet {
  const float* tdom[kMaxGroupFrames];
  void* dst[kMaxGroupFrames];
  long long dst_stride[kMaxGroupFrames];
  int count;
};

// Forward transform of the window's newest frame fused with the filter and
// the inverse transform (k_fused). f.src/f.spec: the newest frame and its ring
// slot; v.in[]: the window's spectra (the newest frame's entry is f.spec).
struct FusedArgs {
  ForwardArgs f;
  InverseArgs v;
};

struct OlaArgs {
  Geom g;
  Tables t;
  const float* tdom;
  void* dst;              // plane at the crop origin
  long long dst_stride;   // bytes
  float norm;
  float rounder;          // 0.5 for integer formats, 0 for float
  float base;
  int maxval;             // (1 << bits) - 1
  int* err;               // device error flag (bounds-checked build), or null
};

// Overlap-add fused into a run's filter/inverse launch (k_filter_inverse_group).
// Output tile (tx, ty), 1 <= tx <= tiles_x, 1 <= ty <= tiles_y, is the pixels
// x0 in [(tx-1)*sx, tx*sx), k in [(ty-1)*sy, ty*sy) of the processed region,
// whose blocks are (tx, ty), (tx-1, ty) when ow > 0, (tx, ty-1) when oh > 0
// and (tx-1, ty-1) when both. Each CTA adds one arrival to the counter of
// every tile its block feeds once its time-domain blocks are stored; the CTA
// that brings a counter to the tile's block count times the launch's epoch
// (so the counters need no reset between launches) does that tile's
// overlap-add for all the run's frames, from L2.
struct OlaFuse {
  OlaArgs o;                      // shared arguments (o.tdom, o.dst unused)
  void* dst[kGroupTile];          // frame j's destination plane at the crop origin
  long long dst_stride[kGroupTile];
  unsigned* cnt;                  // arrival counters, indexed ty * nox + tx
  unsigned epoch;                 // this launch's epoch (> 0)
  int tiles_x, tiles_y;
  int bytes;                      // sample size: 1, 2 or 4
  int px4;                        // 4-pixel form (the plane meets its rules)
};

// One batched launch: `nitems` work items (plane index into `args`, CTA of
// that plane) walked by a grid of `grid` CTAs; args/items in device memory.
struct BatchLaunch {
  const void* args;
  const int2* items;
  int nitems;
  int grid;
};

// One device-to-device plane copy of a batch (crop borders, Kalman frame 0).
struct CopyArgs {
  void* dst;
  long long dpitch;
  const void* src;
  long long spitch;
  long long width;  // bytes per row
  int height;
};

// Host-side launchers (fft3d_kernels.cu). They return cudaGetLastError().
cudaError_t launch_forward(const ForwardArgs& a, int bytes_per_sample, cudaStream_t s);
cudaError_t launch_filter_inverse(const InverseArgs& a, int mode, cudaStream_t s);
// Frame group: fs.count consecutive output frames of one plane (Wiener 3D,
// mode 2..5) in one launch; a holds everything they share.
cudaError_t launch_filter_inverse_frames(const InverseArgs& a, const FrameSet& fs, int mode, cudaStream_t s);
// A run of frames of one plane in one launch, each block's spectra read once
// for the whole run (modes -1..5; Kalman runs in frame order).
// With `of`, the run's overlap-adds are done by the same launch (OlaFuse).
cudaError_t launch_filter_inverse_group(const InverseArgs& a, const TemporalSet& ts, int mode, cudaStream_t s,
                                        const OlaFuse* of = nullptr);
// Forward transforms of fs.count frames of one plane in one launch; a holds
// what they share (geometry, windows, sample offset).
cudaError_t launch_forward_frames(const ForwardArgs& a, const FwdFrameSet& fs, int bytes_per_sample, cudaStream_t s);
cudaError_t launch_overlap_add(const OlaArgs& a, int bytes_per_sample, cudaStream_t s);
// p[0 .. n) = v (stream-ordered state resets)
cudaError_t launch_fill(float* p, float v, size_t n, cudaStream_t s);
// fs.count overlap-adds of one plane in one launch (a holds what they share);
// cudaErrorNotSupported when a frame's geometry or alignment rules out the
// 4-pixel kernel (then launch them one by one).
cudaError_t launch_overlap_add_frames(const OlaArgs& a, const OlaFrameSet& fs, int bytes_per_sample, cudaStream_t s);
bool overlap_add_frames_supported(const OlaArgs& a, const OlaFrameSet& fs, int bytes_per_sample);
// Batched forms (work items as in BatchLaunch); OLA items are 32x8-pixel tiles.
cudaError_t launch_forward_batch(int bw, int bh, const BatchLaunch& l, int bytes_per_sample, cudaStream_t s);
cudaError_t launch_filter_inverse_batch(int bw, int bh, const BatchLaunch& l, int mode, cudaStream_t s);
cudaError_t launch_overlap_add_batch(const BatchLaunch& l, int bytes_per_sample, cudaStream_t s);
// Runs of frame groups of many planes (args: GroupRun[]; items: (run, block)).
cudaError_t launch_filter_inverse_group_batch(int bw, int bh, const BatchLaunch& l, int mode, cudaStream_t s);
cudaError_t launch_copy_batch(const BatchLaunch& l, cudaStream_t s);  // items: (copy, row)
int batch_items_forward(const Geom& g);     // forward / filter-inverse work items of a plane
int batch_items_overlap_add(const Geom& g);  // overlap-add work items (tiles) of a plane
// The 4-pixel batched overlap-add (launch_overlap_add_batch with bytes +
// kOla4Var): its work items per plane, and whether a plane meets its rules.
constexpr int kOla4Var = 10;
int batch_items_overlap_add4(const Geom& g);
bool batch_overlap_add4_ok(const OlaArgs& a, int bytes_per_sample);
// which: 0 forward, 1 filter/inverse, 2 overlap-add, 3 group runs, 4 plane copies
int batch_occupancy(int bw, int bh, int which, int mode_or_bytes);
// Streaming filter of all bins (Wiener 2D/3D, Kalman) into F; the sharpen pass
// and the inverse follow with launch_filter_inverse(MODE_SHARPEN_ONLY) on F.
cudaError_t launch_filter_bins(const InverseArgs& a, float2* F, int mode, cudaStream_t s);
// Filter of a run of frames of one plane (Wiener 2D/3D or Kalman; the
// sharpen pass and the inverse follow with launch_filter_inverse_frames in
// MODE_SHARPEN_ONLY on fs.out). Kalman runs walk the frames in order, with
// the state in registers from the run's first frame to its last.
cudaError_t launch_filter_frames(const InverseArgs& a, const FilterFrameSet& fs, int mode, cudaStream_t s);
// cudaErrorNotSupported when no fused kernel exists for the sample type (float)
cudaError_t launch_fused(const FusedArgs& a, int mode, int bytes_per_sample, cudaStream_t s);
bool block_size_supported(int bw, int bh);
// FindPatternBlock scores (src/helper.cpp:46-90): scores[(by-2)*(nox-4) + bx-2] =
// sum over bins of |X - gridfraction * grid|^2 * pwin for the interior blocks
// 2 <= bx < nox-2, 2 <= by < noy-2, accumulated bin by bin with every product
// and sum rounded separately, as the reference's C loop.
cudaError_t launch_pattern_scores(const float2* spec, const float2* grid, const float* pwin, int nox, int noy,
                                  int bins, float degrid, float* scores, cudaStream_t s);
cudaError_t upload_twiddles();  // every registered size, on the current device

// Tensor-core forward transform of 32x32 blocks (fft3d_tc.cu): DFT tables for
// the plane's analysis windows (forward_tc_table_bytes() bytes, built on the
// host, copied to the device once), and the launcher. `err` receives 1 when a
// bounded wait on the MMA completion barrier times out.
uint32_t forward_tc_table_bytes();
uint32_t forward_tc_smem_bytes();
void forward_tc_tables(const float* wx, const float* wy, uint8_t* out);
cudaError_t launch_forward_tc(const ForwardArgs& a, const void* tables, int* err, int bytes_per_sample, cudaStream_t s);
// The tensor-core forward transforms of fs.count frames of one plane in one
// persistent launch (work items: the frames' tiles).
cudaError_t launch_forward_tc_frames(const ForwardArgs& a, const FwdFrameSet& fs, const void* tables, int* err,
                                     int bytes_per_sample, cudaStream_t s);

// Sets the message returned by fft3d_last_error() on this thread.
void set_last_error(const std::string& msg);

// filter modes of launch_filter_inverse
enum { MODE_SHARPEN_ONLY = -1, MODE_KALMAN = 0, MODE_WIENER2D = 1 /* 2..5: Wiener 3D with that many frames */ };

}  // namespace fft3d
