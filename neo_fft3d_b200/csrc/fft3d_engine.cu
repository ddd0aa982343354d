// Per-plane engine and C ABI (include/fft3d_b200.h) of the FFT3D filtering
// core. One fft3d_plane is the B200 counterpart of one FFT3DEngine
// (reference src/fft3d_engine.h:22-741): it owns the plane's tables, a device
// ring of per-frame spectra (the reference's LRU cache, src/cache.hpp:18-78),
// the Kalman state and one CUDA stream.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fft3d_b200.h"
#include "fft3d_batch.h"
#include "fft3d_kernels.cuh"
#include "fft3d_psd.h"

using fft3d::Geom;

namespace {

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};
// When set, launches and device copies of run_filter are recorded here
// instead of issued (the batched scheduler, fft3d_batch.cu).
thread_local fft3d::Deferred* g_defer = nullptr;
std::mutex g_dev_lock;
std::vector<int> g_tw_ready;  // devices whose twiddle tables are uploaded

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(FFT3D_E_CUDA, std::string("neo_fft3d: CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                            \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

struct Slot {
  float2* spec = nullptr;
  int frame = -1;
  uint64_t stamp = 0;
};

// Optional per-kernel timing: CUDA events recorded on the launching stream
// around every launch, resolved when the counters are read.
enum { K_FORWARD = 0, K_INVERSE = 1, K_OLA = 2, K_FUSED = 3, K_FILTER = 4, K_COUNT = 5 };
struct Timed {
  int kind;
  double bytes;
  cudaEvent_t a, b;
};

}  // namespace

struct fft3d_plane {
  std::mutex mu;
  int device = 0;
  cudaStream_t stream = nullptr;
  fft3d_params ep{};
  fft3d_plane_desc d{};
  int bytes = 1;
  Geom g{};
  int l = 0, t = 0;  // crop origin (plane units)
  float norm = 0, sigma2n_2d = 0, smin2n = 0, smax2n = 0, ht2n = 0;
  bool pattern = false, pattern_set = false, pattern3d_init = false;
  std::vector<float> h_pattern2d, h_pwin, h_grid;  // h_grid: bh*nh complex
  // device tables (one allocation)
  void* d_tables = nullptr;
  fft3d::Tables tab{};
  const float* d_wan_x = nullptr;
  const float* d_wan_y = nullptr;
  std::vector<float> h_wan_x;  // host copy of the analysis window along x
  float* d_pattern2d = nullptr;
  float* d_pattern3d = nullptr;
  std::vector<Slot> slots;
  uint64_t clock = 0;
  float* d_tdom = nullptr;
  // Frame groups (several consecutive output frames of this plane in one
  // batch step): occurrence k > 0 of the group writes its time-domain blocks
  // to tdom_extra[k - 1]; frames in [keep_lo, keep_hi] stay in the ring while
  // the group is planned; all frames of a group use one CTA order.
  std::vector<float*> tdom_extra;
  // filtered spectra of a frame group's frames (the two-pass group filter:
  // k_filter_frames, then the sharpen/inverse pass on these), grown on first use
  std::vector<float2*> filt_frames;
  // how frame groups filter (NEO_FFT3D_GROUP_FILTER): 2 (default, =block):
  // one launch per run of frames of one mode with one CTA per block, each
  // window spectrum read once for the run; 1 (=split): a streaming filter
  // launch for the run, then a sharpen/inverse launch; 0 (=fused): one
  // filter/inverse launch per Wiener 3D run, frames interleaved by CTA
  int group_split = 2;
  // NEO_FFT3D_FUSED_OLA=1: a run's overlap-adds are done by its
  // filter/inverse launch instead of a separate overlap-add launch (measured
  // slower: the tile overlap-adds at the CTAs' tails are latency-bound);
  // per-tile arrival counters (nox x noy, zeroed once) and the launch epoch
  // their targets count in
  unsigned* d_ola_cnt = nullptr;
  unsigned ola_epoch = 0;
  bool fuse_ola = false;
  int occ = 0;
  int keep_lo = 1, keep_hi = 0;
  int fixed_reverse = -1;
  uint64_t groups_done = 0;  // frame groups filtered (their CTA order alternates)
  // completion of the last work queued for this plane on a caller's stream
  // (device-buffer calls, batch steps): fft3d_plane_reset waits for it
  // before it clears the ring and the Kalman state
  cudaEvent_t last_work = nullptr;
  // pshow: spectrum scratch, constant-1 windows, and whether the windows have
  // become constant (after the first pshow frame)
  float2* d_pshow = nullptr;
  float* d_pshow_win = nullptr;
  bool pshow_flat = false;
  // a reset queued on `stream` that the next call must wait for (on its own
  // stream) before it reads the ring or the Kalman state
  cudaEvent_t reset_done = nullptr;
  bool reset_pending = false;
  float2* d_last = nullptr;
  float* d_cov = nullptr;
  float* d_covp = nullptr;
  // Host path (fft3d_plane_filter, fft3d_plane_set_pattern_frame): staging
  // sets owned by one call each until it returns (taken round robin; a call
  // waits while all are owned), uploads on s_up and downloads on s_down,
  // ordered against the kernels on `stream` by events, so that the copies of
  // one call overlap the kernels of another when the plane is called from
  // several threads. The plane's lock is held while a call is queued; the
  // caller then waits on its own completion event.
  struct Stage {
    void* in = nullptr;
    size_t in_pitch = 0;
    void* out = nullptr;
    size_t out_pitch = 0;
    cudaEvent_t in_free = nullptr;   // the kernels reading `in` are done
    cudaEvent_t out_free = nullptr;  // the download of `out` is done
    int* h_flags = nullptr;          // pinned copies of the device error flags
    // Pageable callers: the call's new frame, copied into pinned memory by
    // the calling thread before the call is queued, and its result, read
    // back through pinned memory and copied out after the call's wait
    // (unpadded rows; allocated on first pageable use).
    uint8_t* h_in = nullptr;
    uint8_t* h_out = nullptr;
    cudaEvent_t h_in_done = nullptr;   // the upload from h_in is done
    const void* staged_src = nullptr;  // the caller's frame that h_in holds
    bool pageable_out = false;         // this call downloads into h_out
    bool busy = false;                 // owned by a call (stage_cv)
  };
  static constexpr int kStages = 6;
  Stage stages[kStages];
  std::condition_variable stage_cv;  // with pool_mu: a stage became free
  // Host frame groups (fft3d_plane_filter_frames): per call, the group's
  // uploaded frames and its outputs in device planes (grown to the largest
  // group), exclusive to one call until it returns, like the one-frame stages.
  struct GroupStage {
    // planes of `row` bytes per line, no padding, one after another: frames
    // that are contiguous in host memory move in one copy
    char* in = nullptr;
    char* out = nullptr;
    int nin = 0, nout = 0;
    cudaEvent_t in_free = nullptr;   // the kernels reading `in` are done
    cudaEvent_t out_free = nullptr;  // the downloads of `out` are done
    int* h_flags = nullptr;          // pinned copy of the device error flag
    bool busy = false;               // owned by a call (gstage_cv)
  };
  static constexpr int kGroupStages = 4;
  GroupStage gstages[kGroupStages];
  int next_gstage = 0;
  std::condition_variable gstage_cv;  // with pool_mu: a group stage became free
  int next_stage = 0;
  Stage* cur = nullptr;            // the stage of the call being queued
  cudaEvent_t call_done = nullptr;  // completion event of the call being queued
  cudaStream_t s_up = nullptr, s_down = nullptr;
  std::mutex pool_mu;
  std::vector<cudaEvent_t> sync_pool;
  uint64_t frames_done = 0;
  // kernel sequence of one output frame (NEO_FFT3D_PATH = unfused (default) | split | fused):
  //   split:   k_forward (new frame), k_filter_bins (streaming filter of all
  //            bins into d_filt), k_filter_inverse<sharpen only> on d_filt
  //   unfused: k_forward, k_filter_inverse (filter + sharpen + inverse)
  //   fused:   k_fused (new frame's forward + filter + inverse in one launch)
  //   tc:      as unfused, with the forward transform on the tensor cores
  //            (k_forward_tc, 32x32 blocks; other sizes fall back to k_forward)
  int path = 1;  // 0 split, 1 unfused, 2 fused, 3 tc
  uint8_t* d_tc = nullptr;  // tensor-core DFT tables (path 3)
  int* d_err = nullptr;     // device error flag (tensor-core waits: bit 0, bulk-copy waits: bit 1)
  int bulk = 0;             // bulk-staged filter/inverse kernel (NEO_FFT3D_INV = regs | bulk)
  float2* d_filt = nullptr;
  // learned noise PSD (fft3d_plane_set_psd): model, per-block noise power, scratch
  fft3d_psd* psd_model = nullptr;
  int psd_pooled = 0;
  float psd_pow = 1.f;
  float psd_strength = 1.f;
  float* d_psd = nullptr;
  fft3d::psd::Work* psd_work = nullptr;
  // device bytes this plane holds, and the optional cap on them
  // (NEO_FFT3D_DEVICE_ALLOC_CAP at creation: a host-side fault injection
  // that makes the out-of-memory paths testable; 0 = no cap)
  size_t alloc_used = 0, alloc_cap = 0;
  bool timing = false;
  std::vector<Timed> pending;
  std::vector<cudaEvent_t> event_pool;
  double t_launches[K_COUNT] = {}, t_ms[K_COUNT] = {}, t_bytes[K_COUNT] = {};
  size_t spec_elems() const { return (size_t)g.nblocks * g.bh * g.nh; }
};

namespace {

cudaEvent_t take_event(fft3d_plane* P) {
  if (!P->event_pool.empty()) {
    cudaEvent_t e = P->event_pool.back();
    P->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Device allocations of a plane go through these: they count the plane's
// bytes (fft3d_plane_device_bytes) and honour its allocation cap, failing
// like an exhausted device would (cudaErrorMemoryAllocation).
template <typename T>
cudaError_t dmalloc(fft3d_plane* P, T** p, size_t bytes) {
  if (P->alloc_cap && P->alloc_used + bytes > P->alloc_cap) return cudaErrorMemoryAllocation;
  void* v = nullptr;
  const cudaError_t e = cudaMalloc(&v, bytes);
  if (e == cudaSuccess) {
    *p = static_cast<T*>(v);
    P->alloc_used += bytes;
  }
  return e;
}
cudaError_t dmalloc_pitch(fft3d_plane* P, void** p, size_t* pitch, size_t width, size_t height) {
  const size_t est = ((width + 511) & ~(size_t)511) * height;  // the cap is checked on a 512-byte pitch
  if (P->alloc_cap && P->alloc_used + est > P->alloc_cap) return cudaErrorMemoryAllocation;
  const cudaError_t e = cudaMallocPitch(p, pitch, width, height);
  if (e == cudaSuccess) P->alloc_used += *pitch * height;
  return e;
}
void dfree(fft3d_plane* P, void* p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  P->alloc_used -= std::min(bytes, P->alloc_used);
}

// Brackets one launch with events when timing is on; `bytes` is the launch's
// algorithmic traffic (what its interface must read and write once).
struct TimeScope {
  fft3d_plane* P;
  int kind;
  double bytes;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  TimeScope(fft3d_plane* p, int k, double b, cudaStream_t s) : P(p), kind(k), bytes(b), st(s) {
    if (P->timing && !g_defer) {
      a = take_event(P);
      cudaEventRecord(a, st);
    }
  }
  ~TimeScope() {
    if (!a) return;
    cudaEvent_t b = take_event(P);
    cudaEventRecord(b, st);
    P->pending.push_back(Timed{kind, bytes, a, b});
  }
};

// ---------------------------------------------------------------- tables
// Same formulas as the reference's constructor (src/fft3d_engine.h:204-375),
// computed in float with the double exp/sqrt the reference's C++ calls.

void windows(const fft3d_params& ep, int o, std::vector<float>& anl, std::vector<float>& anr,
             std::vector<float>& snl, std::vector<float>& snr) {
  const float pi = 3.1415926535897932384626433832795f;
  anl.assign(o, 1.f); anr.assign(o, 1.f); snl.assign(o, 1.f); snr.assign(o, 1.f);
  for (int i = 0; i < o; i++) {
    float cl = cosf(pi * (i - o + 0.5f) / (o * 2)), cr = cosf(pi * (i + 0.5f) / (o * 2));
    if (ep.wintype == 0) {
      anl[i] = cl; anr[i] = cr; snl[i] = cl; snr[i] = cr;
    } else if (ep.wintype == 1) {
      anl[i] = (float)std::sqrt((double)cl); anr[i] = (float)std::sqrt((double)cr);
      snl[i] = anl[i] * anl[i] * anl[i]; snr[i] = anr[i] * anr[i] * anr[i];
    } else {
      snl[i] = cl * cl; snr[i] = cr * cr;
    }
  }
}

std::vector<float> full_window(int b, int o, const std::vector<float>& l, const std::vector<float>& r) {
  std::vector<float> w(b, 1.f);
  for (int i = 0; i < o; i++) {
    w[i] = l[i];
    w[b - o + i] = r[i];
  }
  return w;
}

// gridsample: the spectrum of one windowed block of maximum-value samples
// (src/fft3d_engine.h:380-404). The block is separable, so its 2D DFT is the
// outer product of two 1D DFTs; evaluated in double, rounded to float.
void gridsample(const std::vector<float>& wx, const std::vector<float>& wy, double maxv, int bw, int bh,
                std::vector<float>& out) {
  int nh = bw / 2 + 1;
  std::vector<double> xr(nh), xi(nh), yr(bh), yi(bh);
  for (int k = 0; k < nh; k++) {
    double sr = 0, si = 0;
    for (int x = 0; x < bw; x++) {
      double a = -2.0 * M_PI * (double)((long)k * x % bw) / bw;
      sr += wx[x] * std::cos(a);
      si += wx[x] * std::sin(a);
    }
    xr[k] = sr; xi[k] = si;
  }
  for (int h = 0; h < bh; h++) {
    double sr = 0, si = 0;
    for (int y = 0; y < bh; y++) {
      double a = -2.0 * M_PI * (double)((long)h * y % bh) / bh;
      sr += wy[y] * std::cos(a);
      si += wy[y] * std::sin(a);
    }
    yr[h] = sr; yi[h] = si;
  }
  out.assign((size_t)bh * nh * 2, 0.f);
  for (int h = 0; h < bh; h++)
    for (int k = 0; k < nh; k++) {
      out[2 * (h * nh + k)] = (float)(maxv * (yr[h] * xr[k] - yi[h] * xi[k]));
      out[2 * (h * nh + k) + 1] = (float)(maxv * (yr[h] * xi[k] + yi[h] * xr[k]));
    }
}

// SetPattern (src/helper.cpp:92-132) from a host copy of the pattern block's
// spectrum: pattern2d = |X - gridfraction * gridsample|^2 * pwin.
void set_pattern_from_block(fft3d_plane* P, const float2* s) {
  const int nb = P->g.bh * P->g.nh;
  const float* gs = P->h_grid.data();
  const float gcur = P->ep.degrid * s[0].x / gs[0];
  for (int i = 0; i < nb; i++) {
    const float c0 = s[i].x - gcur * gs[2 * i], c1 = s[i].y - gcur * gs[2 * i + 1];
    P->h_pattern2d[i] = (c0 * c0 + c1 * c1) * P->h_pwin[i];
  }
}

int ensure_twiddles(int dev) {
  std::lock_guard<std::mutex> lk(g_dev_lock);
  if (std::find(g_tw_ready.begin(), g_tw_ready.end(), dev) != g_tw_ready.end()) return FFT3D_OK;
  CK(fft3d::upload_twiddles(), "twiddle upload");
  g_tw_ready.push_back(dev);
  return FFT3D_OK;
}

void free_plane(fft3d_plane* P) {
  if (!P) return;
  cudaSetDevice(P->device);
  if (P->stream) cudaStreamSynchronize(P->stream);
  for (auto& t : P->pending) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
  for (auto e : P->event_pool) cudaEventDestroy(e);
  for (auto& s : P->slots) cudaFree(s.spec);
  cudaFree(P->d_tables);
  cudaFree(P->d_tdom);
  cudaFree(P->d_pshow);
  cudaFree(P->d_pshow_win);
  for (auto* t : P->tdom_extra) cudaFree(t);
  for (auto* f : P->filt_frames) cudaFree(f);
  cudaFree(P->d_ola_cnt);
  cudaFree(P->d_filt);
  cudaFree(P->d_tc);
  cudaFree(P->d_err);
  cudaFree(P->d_last);
  cudaFree(P->d_cov);
  cudaFree(P->d_covp);
  cudaFree(P->d_psd);
  fft3d::psd::work_destroy(P->psd_work);
  for (auto* st : {P->s_up, P->s_down})
    if (st) cudaStreamSynchronize(st);
  for (auto& sg : P->stages) {
    cudaFree(sg.in);
    cudaFree(sg.out);
    if (sg.h_in) cudaFreeHost(sg.h_in);
    if (sg.h_out) cudaFreeHost(sg.h_out);
    if (sg.h_in_done) cudaEventDestroy(sg.h_in_done);
    if (sg.in_free) cudaEventDestroy(sg.in_free);
    if (sg.out_free) cudaEventDestroy(sg.out_free);
    if (sg.h_flags) cudaFreeHost(sg.h_flags);
  }
  for (auto& gs : P->gstages) {
    cudaFree(gs.in);
    cudaFree(gs.out);
    if (gs.in_free) cudaEventDestroy(gs.in_free);
    if (gs.out_free) cudaEventDestroy(gs.out_free);
    if (gs.h_flags) cudaFreeHost(gs.h_flags);
  }
  for (auto e : P->sync_pool) cudaEventDestroy(e);
  if (P->last_work) {
    cudaEventSynchronize(P->last_work);
    cudaEventDestroy(P->last_work);
  }
  if (P->reset_done) cudaEventDestroy(P->reset_done);
  if (P->s_up) cudaStreamDestroy(P->s_up);
  if (P->s_down) cudaStreamDestroy(P->s_down);
  if (P->stream) cudaStreamDestroy(P->stream);
  delete P;
}

int upload_pattern(fft3d_plane* P, float* dptr, const std::vector<float>& v, cudaStream_t st) {
  CK(cudaMemcpyAsync(dptr, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice, st), "pattern upload");
  // the source is a temporary host vector: the copy must have read it
  CK(cudaStreamSynchronize(st), "pattern upload");
  return FFT3D_OK;
}

Slot* find_slot(fft3d_plane* P, int frame) {
  for (auto& s : P->slots)
    if (s.frame == frame) return &s;
  return nullptr;
}

// least recently used slot whose frame is not in [lo, hi] (nor in the
// frame group's kept range); free slots (frame -1) are always candidates
Slot* evict_slot(fft3d_plane* P, int lo, int hi) {
  Slot* best = nullptr;
  for (auto& s : P->slots) {
    const bool free_slot = s.frame < 0;  // frames are >= 0
    if (!free_slot && s.frame >= lo && s.frame <= hi) continue;
    if (!free_slot && s.frame >= P->keep_lo && s.frame <= P->keep_hi) continue;
    if (!best || s.stamp < best->stamp) best = &s;
  }
  return best;
}

fft3d::ForwardArgs forward_args(fft3d_plane* P, const void* plane, long long stride, float2* spec) {
  fft3d::ForwardArgs a;
  a.g = P->g;
  a.src = static_cast<const char*>(plane) + (long long)P->t * stride + (long long)P->l * P->bytes;
  a.src_stride = stride;
  a.base = (P->bytes != 4 && P->d.is_chroma) ? (float)(1 << (P->d.bits - 1)) : 0.f;
  a.wan_x = P->d_wan_x;
  a.wan_y = P->d_wan_y;
  for (int x = 0; x < fft3d::kMaxBw; x++) a.wx[x] = x < (int)P->h_wan_x.size() ? P->h_wan_x[x] : 0.f;
  a.spec = spec;
  a.err = P->d_err;
  return a;
}

int launch_forward(fft3d_plane* P, const void* plane, long long stride, float2* spec, cudaStream_t st) {
  fft3d::ForwardArgs a = forward_args(P, plane, stride, spec);
  if (g_defer) {
    g_defer->fwd.push_back({a, P->bytes, g_defer->plane});
    return FFT3D_OK;
  }
  TimeScope ts(P, K_FORWARD, (double)P->g.W * P->g.H * P->bytes + (double)P->spec_elems() * sizeof(float2), st);
  if (P->d_tc) {
    CK(fft3d::launch_forward_tc(a, P->d_tc, P->d_err, P->bytes, st), "tensor-core forward kernel");
  } else {
    CK(fft3d::launch_forward(a, P->bytes, st), "forward kernel");
  }
  g_launches++;
  return FFT3D_OK;
}

cudaEvent_t take_sync_event(fft3d_plane* P) {
  std::lock_guard<std::mutex> lk(P->pool_mu);
  if (!P->sync_pool.empty()) {
    cudaEvent_t e = P->sync_pool.back();
    P->sync_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  return e;
}

void give_sync_event(fft3d_plane* P, cudaEvent_t e) {
  std::lock_guard<std::mutex> lk(P->pool_mu);
  P->sync_pool.push_back(e);
}

// `wait` waits for the work queued so far on `done_on` (a stream-ordered
// dependency; the event is free for reuse once the wait is queued).
int stream_after(fft3d_plane* P, cudaStream_t wait, cudaStream_t done_on) {
  cudaEvent_t e = take_sync_event(P);
  CK(cudaEventRecord(e, done_on), "event");
  CK(cudaStreamWaitEvent(wait, e, 0), "event");
  give_sync_event(P, e);
  return FFT3D_OK;
}

// Host path: the call's host frame into its staging plane, on the upload
// stream, once the kernels that read the stage's previous frame are done;
// the kernels of stream `st` then wait for the copy.
int upload_frame(fft3d_plane* P, const void* plane, int stride, cudaStream_t st) {
  fft3d_plane::Stage* sg = P->cur;
  const size_t row = (size_t)P->d.width * P->bytes;
  CK(cudaStreamWaitEvent(P->s_up, sg->in_free, 0), "event");
  if (sg->staged_src && plane == sg->staged_src) {
    // the frame the caller's thread already copied into pinned memory
    CK(cudaMemcpy2DAsync(sg->in, sg->in_pitch, sg->h_in, row, row, P->d.height, cudaMemcpyHostToDevice, P->s_up),
       "frame upload");
    CK(cudaEventRecord(sg->h_in_done, P->s_up), "event");
    sg->staged_src = nullptr;
  } else {
    CK(cudaMemcpy2DAsync(sg->in, sg->in_pitch, plane, stride, row, P->d.height, cudaMemcpyHostToDevice, P->s_up),
       "frame upload");
  }
  return stream_after(P, st, P->s_up);
}

// Whether host memory p is pinned (page-locked or registered).
bool host_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// The spectrum of frame m in a ring slot, computing it from `plane` if needed.
int spectrum_slot(fft3d_plane* P, int m, int lo, int hi, const void* plane, int stride, bool host, cudaStream_t st,
                  Slot** out) {
  Slot* s = find_slot(P, m);
  if (!s) {
    if (!plane) return fail(FFT3D_E_FRAME, "neo_fft3d: frame " + std::to_string(m) + " is needed but was not supplied");
    s = evict_slot(P, lo, hi);
    if (!s) return fail(FFT3D_E_PARAM, "neo_fft3d: spectrum ring too small");
    s->frame = -1;
    const void* src = plane;
    long long sstride = stride;
    if (host) {
      int rc = upload_frame(P, plane, stride, st);
      if (rc) return rc;
      src = P->cur->in;
      sstride = (long long)P->cur->in_pitch;
    }
    int rc = launch_forward(P, src, sstride, s->spec, st);
    if (rc) return rc;
    if (host) CK(cudaEventRecord(P->cur->in_free, st), "event");
    s->frame = m;
  }
  s->stamp = ++P->clock;
  *out = s;
  return FFT3D_OK;
}

int copy_plane(fft3d_plane* P, void* dst, int dstride, const void* src, int sstride, cudaMemcpyKind kind,
               cudaStream_t st) {
  if (g_defer && kind == cudaMemcpyDeviceToDevice) {
    g_defer->copies.push_back({dst, (size_t)dstride, src, (size_t)sstride, (size_t)P->d.width * P->bytes,
                               (size_t)P->d.height, g_defer->plane});
    return FFT3D_OK;
  }
  CK(cudaMemcpy2DAsync(dst, dstride, src, sstride, (size_t)P->d.width * P->bytes, P->d.height, kind, st),
     "plane copy");
  return FFT3D_OK;
}

// The output of one frame from its time-domain blocks: the crop borders from
// the source frame (src/fft3d.hpp:292-352), the overlap-add with the tables'
// synthesis windows and sample offset `base`, and on the host path the
// download of the result on its own stream.
int output_frame(fft3d_plane* P, float* tdom, const fft3d::Tables& tab, float base, void* dst, int dst_stride,
                 const void* cur, int cur_stride, bool host, bool learned, cudaStream_t st) {
  const fft3d_params& ep = P->ep;
  const bool crop = ep.l > 0 || ep.t > 0 || ep.r > 0 || ep.b > 0;
  void* odst = dst;
  long long ostride = dst_stride;
  if (host) {
    odst = P->cur->out;
    ostride = (long long)P->cur->out_pitch;
    // the stage's previous result must have been downloaded
    CK(cudaStreamWaitEvent(st, P->cur->out_free, 0), "event");
    if (crop) {
      if (!cur) return fail(FFT3D_E_FRAME, "neo_fft3d: the current frame is needed for the crop borders");
      for (int y = 0; y < P->d.height; y++)
        std::memcpy(static_cast<char*>(dst) + (size_t)y * dst_stride, static_cast<const char*>(cur) + (size_t)y * cur_stride,
                    (size_t)P->d.width * P->bytes);
    }
  } else if (crop) {
    if (!cur) return fail(FFT3D_E_FRAME, "neo_fft3d: the current frame is needed for the crop borders");
    int rc = copy_plane(P, dst, dst_stride, cur, cur_stride, cudaMemcpyDeviceToDevice, st);
    if (rc) return rc;
  }
  fft3d::OlaArgs oa;
  oa.g = P->g;
  oa.t = tab;
  oa.tdom = tdom;
  oa.dst = static_cast<char*>(odst) + (long long)P->t * ostride + (long long)P->l * P->bytes;
  oa.dst_stride = ostride;
  oa.norm = P->norm;
  const bool ints = P->bytes != 4;
  oa.rounder = ints ? 0.5f : 0.f;
  oa.base = base;
  // float samples clamp to [0, 1] and have no integer maximum (no shift by 32)
  oa.maxval = P->bytes == 1 ? 255 : (P->bytes == 2 ? (1 << P->d.bits) - 1 : 0);
  oa.err = P->d_err;
  if (g_defer) {
    g_defer->ola.push_back({oa, P->bytes, g_defer->plane});
  } else {
    TimeScope ts(P, K_OLA, (double)P->g.nblocks * P->g.bh * P->g.bw * 4 + (double)P->g.W * P->g.H * P->bytes, st);
    CK(fft3d::launch_overlap_add(oa, P->bytes, st), "overlap-add kernel");
    g_launches++;
  }
  if (host) {
    // download on its own stream once the kernels are done; then the error
    // flags; the caller waits on the call's completion event
    fft3d_plane::Stage* sg = P->cur;
    int rc = stream_after(P, P->s_down, st);
    if (rc) return rc;
    char* hdst = static_cast<char*>(dst) + (size_t)P->t * dst_stride + (size_t)P->l * P->bytes;
    const char* ddst = static_cast<const char*>(sg->out) + P->t * sg->out_pitch + (size_t)P->l * P->bytes;
    const size_t orow = (size_t)P->g.W * P->bytes;
    if (sg->pageable_out)  // into pinned memory; the caller's thread copies it out after its wait
      CK(cudaMemcpy2DAsync(sg->h_out, orow, ddst, sg->out_pitch, orow, P->g.H, cudaMemcpyDeviceToHost, P->s_down),
         "result download");
    else
      CK(cudaMemcpy2DAsync(hdst, dst_stride, ddst, sg->out_pitch, orow, P->g.H, cudaMemcpyDeviceToHost, P->s_down),
         "result download");
    CK(cudaEventRecord(sg->out_free, P->s_down), "event");
    sg->h_flags[0] = sg->h_flags[1] = 0;
    CK(cudaMemcpyAsync(&sg->h_flags[0], P->d_err, sizeof(int), cudaMemcpyDeviceToHost, P->s_down), "error flag");
    if (learned)
      CK(cudaMemcpyAsync(&sg->h_flags[1], fft3d::psd::err_flag(P->psd_model), sizeof(int), cudaMemcpyDeviceToHost,
                         P->s_down), "error flag");
    P->call_done = take_sync_event(P);
    CK(cudaEventRecord(P->call_done, P->s_down), "event");
  }
  return FFT3D_OK;
}

// FindPatternBlock (src/helper.cpp:46-90) on the spectra `spec`: the interior
// block with the least windowed power, scored on the device in the
// reference's summation order; the first minimum in raster order wins, as in
// the reference's loop. *px, *py are left unchanged when the plane has no
// interior block. Synchronises stream st.
int find_pattern_block(fft3d_plane* P, const float2* spec, cudaStream_t st, int* px, int* py) {
  const int nb = P->g.bh * P->g.nh;
  const int wx = P->g.nox - 4, wy = P->g.noy - 4;
  if (wx <= 0 || wy <= 0) return FFT3D_OK;
  float* d_buf = nullptr;
  CK(cudaMalloc(&d_buf, ((size_t)wx * wy + nb) * sizeof(float)), "pattern scores");
  std::vector<float> scores((size_t)wx * wy);
  cudaError_t e = cudaMemcpyAsync(d_buf + (size_t)wx * wy, P->h_pwin.data(), nb * sizeof(float),
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = fft3d::launch_pattern_scores(spec, P->tab.grid, d_buf + (size_t)wx * wy, P->g.nox, P->g.noy, nb, P->ep.degrid,
                                     d_buf, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(scores.data(), d_buf, scores.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_buf);
  if (e != cudaSuccess) return cuda_fail(e, "pattern scores");
  float best = 1e15f;
  for (size_t k = 0; k < scores.size(); k++)
    if (scores[k] < best) {
      best = scores[k];
      *px = 2 + (int)(k % wx);
      *py = 2 + (int)(k / wx);
    }
  return FFT3D_OK;
}

// pshow (src/fft3d_engine.h:505-565): instead of the filtered frame, the noise
// pattern's block alone. The block is found on frame n itself (or is px, py);
// from then on the analysis and synthesis windows are constant 1, as the
// reference overwrites them; frame n is transformed again with those windows
// and a sample offset of 2^(bits-1) for every plane of a non-RGB clip (the
// reference's CoverToOverlap flag there is "not RGB"), every other block's
// spectrum is zeroed (PutPatternOnly, src/helper.cpp:134-170), and the
// inverse and overlap-add give the block's pixels on a flat background. The
// reference's caption is a TODO there and is not drawn.
int pshow_frame(fft3d_plane* P, int n, const void* const src[5], const int stride[5], void* dst, int dst_stride,
                bool host, cudaStream_t st) {
  (void)n;
  const void* cur = src ? src[2] : nullptr;
  if (!cur) return fail(FFT3D_E_FRAME, "neo_fft3d: frame " + std::to_string(n) + " is needed but was not supplied");
  const size_t spec_bytes = P->spec_elems() * sizeof(float2);
  if (!P->d_pshow) {
    const int nt = P->g.bw + P->g.bh + 2 * P->g.ow + 2 * P->g.oh;
    float* t = nullptr;
    if (dmalloc(P, &P->d_pshow, spec_bytes) != cudaSuccess || dmalloc(P, &t, nt * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (pshow)");
    }
    P->d_pshow_win = t;
    std::vector<float> ones(nt, 1.f);
    CK(cudaMemcpy(t, ones.data(), nt * sizeof(float), cudaMemcpyHostToDevice), "pshow tables");
  }
  const void* plane = cur;
  long long pstride = stride[2];
  if (host) {
    int rc = upload_frame(P, cur, stride[2], st);
    if (rc) return rc;
    plane = P->cur->in;
    pstride = (long long)P->cur->in_pitch;
  }
  const float* ones = P->d_pshow_win;
  auto forward = [&](bool constant, float base) {
    fft3d::ForwardArgs a = forward_args(P, plane, pstride, P->d_pshow);
    if (constant) {
      a.wan_x = ones;
      a.wan_y = ones;
      for (float& w : a.wx) w = 1.f;
    }
    a.base = base;
    g_launches++;
    return fft3d::launch_forward(a, P->bytes, st);
  };
  const bool ints = P->bytes != 4;
  const float half = ints ? (float)(1 << (P->d.bits - 1)) : 0.f;
  // the block: on frame n with the current windows and the plane's own offset
  int pxf = P->ep.px, pyf = P->ep.py;
  CK(forward(P->pshow_flat, P->d.is_chroma ? half : 0.f), "forward kernel (pshow)");
  if (P->ep.px == 0 && P->ep.py == 0) {
    int rc = find_pattern_block(P, P->d_pshow, st, &pxf, &pyf);
    if (rc) return rc;
  }
  P->pshow_flat = true;
  // the frame with constant windows; every block but the pattern's zeroed
  const float base = P->d.rgb ? 0.f : half;
  CK(forward(true, base), "forward kernel (pshow)");
  const size_t nb = (size_t)P->g.bh * P->g.nh, blk = (size_t)pyf * P->g.nox + pxf;
  if (blk > 0) CK(cudaMemsetAsync(P->d_pshow, 0, blk * nb * sizeof(float2), st), "pshow");
  if (blk + 1 < (size_t)P->g.nblocks)
    CK(cudaMemsetAsync(P->d_pshow + (blk + 1) * nb, 0, ((size_t)P->g.nblocks - blk - 1) * nb * sizeof(float2), st),
       "pshow");
  if (host) CK(cudaEventRecord(P->cur->in_free, st), "event");
  fft3d::Tables tab = P->tab;
  tab.wan_x = ones;
  tab.wan_y = ones;
  tab.wsyn_xl = tab.wsyn_xr = ones;
  tab.wsyn_yl = tab.wsyn_yr = ones;
  fft3d::InverseArgs ia{};
  ia.g = P->g;
  ia.t = tab;
  ia.in[2] = P->d_pshow;
  ia.tdom = P->d_tdom;
  ia.err = P->d_err;
  CK(fft3d::launch_filter_inverse(ia, fft3d::MODE_SHARPEN_ONLY, st), "inverse kernel (pshow)");
  g_launches++;
  return output_frame(P, P->d_tdom, tab, base, dst, dst_stride, cur, stride[2], host, false, st);
}

int run_filter(fft3d_plane* P, int n, const void* const src[5], const int stride[5], void* dst, int dst_stride,
               bool host, cudaStream_t st) {
  if (P->reset_pending) {  // fft3d_plane_reset queued on the plane's stream
    CK(cudaStreamWaitEvent(st, P->reset_done, 0), "reset");
    P->reset_pending = false;
  }
  const fft3d_params& ep = P->ep;
  // pshow shows the pattern block before any filtering (src/fft3d_engine.h:505)
  if (ep.pshow && ep.pfactor != 0) return pshow_frame(P, n, src, stride, dst, dst_stride, host, st);
  const int bt = ep.bt;
  int btcur = bt;  // src/fft3d_engine.h:579-582
  if ((bt / 2 > n) || (bt - 1) / 2 > (P->d.num_frames - 1 - n)) btcur = 1;
  const void* cur = src ? src[2] : nullptr;
  if (bt == 0 && n == 0) {  // Kalman: frame 0 is returned unprocessed (:681-687)
    if (!cur) return fail(FFT3D_E_FRAME, "neo_fft3d: frame 0 was not supplied");
    if (host) {
      for (int y = 0; y < P->d.height; y++)
        std::memcpy(static_cast<char*>(dst) + (size_t)y * dst_stride, static_cast<const char*>(cur) + (size_t)y * stride[2],
                    (size_t)P->d.width * P->bytes);
      return FFT3D_OK;
    }
    return copy_plane(P, dst, dst_stride, cur, stride[2], cudaMemcpyDeviceToDevice, st);
  }
  if (P->pattern && !P->pattern_set)
    return fail(FFT3D_E_PARAM, "neo_fft3d: noise pattern not estimated yet (fft3d_plane_set_pattern_frame)");
  const int from = bt > 0 && btcur > 1 ? -btcur / 2 : 0;
  const int to = bt > 0 && btcur > 1 ? (btcur - 1) / 2 : 0;
  if (bt > 0 && btcur > 1 && P->pattern && !P->pattern3d_init) {  // :625-630
    std::vector<float> p3(P->h_pattern2d.size());
    for (size_t i = 0; i < p3.size(); i++) p3[i] = P->h_pattern2d[i] * (float)btcur;
    int rc = upload_pattern(P, P->d_pattern3d, p3, st);
    if (rc) return rc;
    P->pattern3d_init = true;
  }
  const int mode = bt > 0 ? btcur : bt;
  const bool learned = P->psd_model && mode != fft3d::MODE_SHARPEN_ONLY;
  fft3d::InverseArgs ia{};
  // The steady state computes one new spectrum per output frame, the newest
  // of the window, in the fused kernel; older frames missing from the ring
  // (clip start, seeks) are transformed first by the forward kernel.
  const int newest = n + to;
  const bool fused = P->path == 2 && P->bytes != 4 && !learned && !find_slot(P, newest);
  for (int d = from; d <= (fused ? to - 1 : to); d++) {
    Slot* s = nullptr;
    int rc = spectrum_slot(P, n + d, n + from, n + to, src ? src[2 + d] : nullptr, stride ? stride[2 + d] : 0, host,
                           st, &s);
    if (rc) return rc;
    ia.in[2 + d] = s->spec;
  }
  Slot* news = nullptr;
  const void* new_src = nullptr;
  long long new_stride = 0;
  if (fused) {
    const void* plane = src ? src[2 + to] : nullptr;
    if (!plane) return fail(FFT3D_E_FRAME, "neo_fft3d: frame " + std::to_string(newest) + " is needed but was not supplied");
    news = evict_slot(P, n + from, n + to);
    if (!news) return fail(FFT3D_E_PARAM, "neo_fft3d: spectrum ring too small");
    news->frame = -1;
    new_src = plane;
    new_stride = stride[2 + to];
    if (host) {
      int rc = upload_frame(P, plane, stride[2 + to], st);
      if (rc) return rc;
      new_src = P->cur->in;
      new_stride = (long long)P->cur->in_pitch;
    }
    ia.in[2 + to] = news->spec;
  }
  ia.g = P->g;
  ia.t = P->tab;
  fft3d::FilterConsts& c = ia.c;
  c.sigma2n = btcur * ep.sigma * ep.sigma / P->norm;  // :589
  c.sigma2n_2d = P->sigma2n_2d;
  c.lowlimit = (ep.beta - 1) / ep.beta;
  c.degrid = ep.degrid;
  c.sharpen = ep.sharpen;
  c.dehalo = ep.dehalo;
  c.smin2n = P->smin2n;
  c.smax2n = P->smax2n;
  c.ht2n = P->ht2n;
  c.kratio2 = ep.kratio * ep.kratio;
  c.pattern = P->pattern ? 1 : 0;
  c.use_sharpen = ep.sharpen != 0;
  c.use_dehalo = ep.dehalo != 0;
  // a learned noise power takes the pattern's place, sharpen included (:620-621)
  c.fuse_sharpen = (mode == 1 && !P->pattern && !learned) ? 1 : 0;
  c.do_sharpen = ((ep.sharpen != 0 || ep.dehalo != 0) && (mode != 1 || P->pattern || learned)) ? 1 : 0;
  if (learned) {
    // the model reads the current frame's block spectra
    CK(fft3d::psd::infer(P->psd_model, P->psd_work, ia.in[2], P->g.nblocks, P->psd_pooled != 0, P->psd_pow, P->d_psd,
                         st),
       "learned noise PSD");
    g_launches += P->psd_pooled ? 10 : 8;  // features, 3 x (GEMM, bias/GELU), output
    ia.psd = P->d_psd;
    ia.psd_scale = P->psd_strength * (mode >= 2 ? (float)btcur : 1.f);
    ia.psd_per_block = P->psd_pooled ? 0 : 1;
  }
  ia.kal_last = P->d_last;
  ia.kal_covar = P->d_cov;
  ia.kal_covarp = P->d_covp;
  float* tdom = P->occ > 0 ? P->tdom_extra[P->occ - 1] : P->d_tdom;
  ia.tdom = tdom;
  ia.err = P->d_err;
  ia.bulk = (P->path == 1 || P->path == 3) ? P->bulk : 0;
  ia.reverse = (int)(P->frames_done++ & 1);
  if (P->fixed_reverse >= 0) ia.reverse = P->fixed_reverse;
  {
    const double S = (double)P->spec_elems() * sizeof(float2);
    const double state = bt == 0 ? 2.0 * (double)P->spec_elems() * 16 : 0.0;
    const double T = (double)P->g.nblocks * P->g.bh * P->g.bw * 4;
    if (fused) {
      // reads: the newest frame's pixels and the older spectra (+ Kalman state);
      // writes: the newest spectrum and the time-domain blocks
      fft3d::FusedArgs fa;
      fa.f = forward_args(P, new_src, new_stride, news->spec);
      fa.v = ia;
      {
        TimeScope ts(P, K_FUSED, (double)P->g.W * P->g.H * P->bytes + (to - from) * S + S + state + T, st);
        CK(fft3d::launch_fused(fa, mode, P->bytes, st), "fused kernel");
      }
      if (host) CK(cudaEventRecord(P->cur->in_free, st), "event");
    } else if (P->path == 0 && mode != fft3d::MODE_SHARPEN_ONLY) {
      {
        // reads: the spectra of the window (+ Kalman state); writes: the filtered spectrum
        TimeScope ts(P, K_FILTER, (to - from + 1) * S + state + S, st);
        CK(fft3d::launch_filter_bins(ia, P->d_filt, mode, st), "filter kernel");
      }
      g_launches++;
      fft3d::InverseArgs sa = ia;
      for (auto& p : sa.in) p = nullptr;
      sa.in[2] = P->d_filt;
      // reads: the filtered spectrum; writes: the time-domain blocks
      TimeScope ts(P, K_INVERSE, S + T, st);
      CK(fft3d::launch_filter_inverse(sa, fft3d::MODE_SHARPEN_ONLY, st), "sharpen/inverse kernel");
    } else if (g_defer) {
      g_defer->inv.push_back({ia, mode, g_defer->plane});
    } else {
      // reads: the spectra of the window (+ Kalman state); writes: the time-domain blocks
      TimeScope ts(P, K_INVERSE, (to - from + 1) * S + state + T, st);
      CK(fft3d::launch_filter_inverse(ia, mode, st), "filter/inverse kernel");
    }
  }
  if (fused) {
    news->frame = newest;
    news->stamp = ++P->clock;
  }
  if (!g_defer) g_launches++;
  const bool ints = P->bytes != 4;
  return output_frame(P, tdom, P->tab, (ints && P->d.is_chroma) ? (float)(1 << (P->d.bits - 1)) : 0.f, dst,
                      dst_stride, cur, stride ? stride[2] : 0, host, learned, st);
}

// A stage for one host-path call, exclusive until the call returns (the
// stages are used round robin; a call waits while all are owned).
fft3d_plane::Stage* acquire_stage(fft3d_plane* P) {
  std::unique_lock<std::mutex> lk(P->pool_mu);
  for (;;) {
    for (int k = 0; k < fft3d_plane::kStages; k++) {
      const int i = (P->next_stage + k) % fft3d_plane::kStages;
      if (!P->stages[i].busy) {
        P->stages[i].busy = true;
        P->next_stage = (i + 1) % fft3d_plane::kStages;
        return &P->stages[i];
      }
    }
    P->stage_cv.wait(lk);
  }
}

void release_stage(fft3d_plane* P, fft3d_plane::Stage* sg) {
  {
    std::lock_guard<std::mutex> lk(P->pool_mu);
    sg->busy = false;
  }
  P->stage_cv.notify_one();
}

// Pageable host buffers of a one-frame call: the window's newest frame, if
// the plane will need it and it is pageable, is copied into the stage's
// pinned input by the calling thread (outside the plane's lock), and a
// pageable destination gets its result through the stage's pinned output.
int stage_pageable(fft3d_plane* P, fft3d_plane::Stage* sg, int n, const void* const src[5], const int stride[5],
                   void* dst) {
  sg->staged_src = nullptr;
  sg->pageable_out = !host_pinned(dst);
  const size_t row = (size_t)P->d.width * P->bytes, plane = row * P->d.height;
  const size_t orow = (size_t)P->g.W * P->bytes, oplane = orow * P->g.H;
  if (sg->pageable_out && !sg->h_out && cudaMallocHost(&sg->h_out, oplane) != cudaSuccess) {
    cudaGetLastError();
    sg->h_out = nullptr;
    sg->pageable_out = false;  // the driver copies instead
  }
  if (!src) return FFT3D_OK;
  const int bt = P->ep.bt;
  int to = 0;
  if (bt > 1 && !((bt / 2 > n) || (bt - 1) / 2 > (P->d.num_frames - 1 - n))) to = (bt - 1) / 2;
  const void* fsrc = src[2 + to];
  if (!fsrc || (bt == 0 && n == 0)) return FFT3D_OK;
  {
    std::lock_guard<std::mutex> lk(P->mu);
    if (find_slot(P, n + to)) return FFT3D_OK;  // cached: nothing to upload
  }
  if (host_pinned(fsrc)) return FFT3D_OK;
  if (!sg->h_in) {
    if (cudaMallocHost(&sg->h_in, plane) != cudaSuccess ||
        cudaEventCreateWithFlags(&sg->h_in_done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return FFT3D_OK;  // the driver copies instead
    }
  } else {
    CK(cudaEventSynchronize(sg->h_in_done), "staging");  // its last upload is done
  }
  for (int y = 0; y < P->d.height; y++)
    std::memcpy(sg->h_in + (size_t)y * row, static_cast<const char*>(fsrc) + (size_t)y * stride[2 + to], row);
  sg->staged_src = fsrc;
  return FFT3D_OK;
}

// Waits for a queued host-path call and reports a device error flag it saw.
// Frames whose spectra a frame group n0 .. n0 + count - 1 needs at once.
void group_range(const fft3d_plane* P, int n0, int count, int* lo, int* hi) {
  const int bt = std::max(P->ep.bt, 1);
  *lo = n0 - bt / 2;
  *hi = n0 + count - 1 + (bt - 1) / 2;
}

// A frame group keeps the spectra of frames lo..hi in the ring at once and
// writes one time-domain buffer per frame: both grow on first use.
int group_resources(fft3d_plane* P, int lo, int hi, int count) {
  while ((int)P->slots.size() < hi - lo + 2) {
    Slot s;
    if (dmalloc(P, &s.spec, P->spec_elems() * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (spectrum ring of a frame group)");
    }
    P->slots.push_back(s);
  }
  while ((int)P->tdom_extra.size() < count - 1) {
    float* t = nullptr;
    if (dmalloc(P, &t, (size_t)P->g.nblocks * P->g.bh * P->g.bw * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (time-domain blocks of a frame group)");
    }
    P->tdom_extra.push_back(t);
  }
  while (P->group_split == 1 && (int)P->filt_frames.size() < count) {
    float2* f = nullptr;
    if (dmalloc(P, &f, P->spec_elems() * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (filtered spectra of a frame group)");
    }
    P->filt_frames.push_back(f);
  }
  return FFT3D_OK;
}

// Recorded forward transforms that will not run (planning failed): their
// slots hold no spectrum.
void discard_recorded(fft3d_plane* P, const fft3d::Deferred& d) {
  for (const auto& f : d.fwd)
    for (auto& s : P->slots)
      if (s.spec == f.a.spec) s.frame = -1;
}

// Fuses the overlap-adds of the run d.inv[i, e) into its filter/inverse
// launch (fills *of, marks the records in ola_done) when the plane asks for
// it (NEO_FFT3D_FUSED_OLA=1) and allows it:
// every frame of the run has its overlap-add record, and the plane's output
// tiles are inside its block grid. Otherwise (or when the arrival counters
// cannot be allocated) the overlap-adds stay separate launches.
bool fuse_run_ola(fft3d_plane* P, const fft3d::Deferred& d, const fft3d::TemporalSet& ts, size_t i, size_t e,
                  std::vector<char>& ola_done, fft3d::OlaFuse* of, cudaStream_t st) {
  if (!P->fuse_ola || e - i > (size_t)fft3d::kGroupTile) return false;
  const fft3d::Geom& g = P->g;
  const int tiles_x = (g.sx + g.W - 1) / g.sx, tiles_y = (g.sy + g.H - 1) / g.sy;
  if (tiles_x < 1 || tiles_y < 1 || tiles_x >= g.nox || tiles_y >= g.noy) return false;
  size_t idx[fft3d::kGroupTile];
  for (size_t k = i; k < e; k++) {
    size_t m = 0;
    while (m < d.ola.size() && (ola_done[m] || d.ola[m].a.tdom != d.inv[k].a.tdom)) m++;
    if (m == d.ola.size() || (k > i && d.ola[m].bytes != d.ola[idx[0]].bytes)) return false;
    idx[k - i] = m;
  }
  const size_t cnt_bytes = (size_t)g.nblocks * sizeof(unsigned);
  if (!P->d_ola_cnt) {
    if (dmalloc(P, &P->d_ola_cnt, cnt_bytes) != cudaSuccess) {
      cudaGetLastError();
      P->d_ola_cnt = nullptr;
      return false;
    }
    if (cudaMemsetAsync(P->d_ola_cnt, 0, cnt_bytes, st) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(P->d_ola_cnt);
      P->d_ola_cnt = nullptr;
      return false;
    }
    P->ola_epoch = 0;
  }
  if (P->ola_epoch >= (1u << 29)) {  // targets stay below 2^32: start the counts over
    if (cudaMemsetAsync(P->d_ola_cnt, 0, cnt_bytes, st) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    P->ola_epoch = 0;
  }
  P->ola_epoch++;
  *of = fft3d::OlaFuse{};
  of->o = d.ola[idx[0]].a;
  of->o.tdom = nullptr;
  of->o.dst = nullptr;
  fft3d::OlaFrameSet fs{};
  fs.count = (int)(e - i);
  for (size_t k = 0; k < e - i; k++) {
    of->dst[k] = d.ola[idx[k]].a.dst;
    of->dst_stride[k] = d.ola[idx[k]].a.dst_stride;
    fs.tdom[k] = ts.tdom[k];
    fs.dst[k] = of->dst[k];
    fs.dst_stride[k] = of->dst_stride[k];
    ola_done[idx[k]] = 1;
  }
  of->cnt = P->d_ola_cnt;
  of->epoch = P->ola_epoch;
  of->tiles_x = tiles_x;
  of->tiles_y = tiles_y;
  of->bytes = d.ola[idx[0]].bytes;
  of->px4 = fft3d::overlap_add_frames_supported(of->o, fs, of->bytes) ? 1 : 0;
  return true;
}

// Issues the launches of a frame group recorded for plane P, phase by phase:
// the new spectra, the plane copies (crop borders), then the filter/inverse
// of runs of consecutive frames of one mode (with their overlap-adds when
// fused), then the remaining overlap-adds.
int run_group(fft3d_plane* P, const fft3d::Deferred& d, cudaStream_t st) {
  const double S = (double)P->spec_elems() * sizeof(float2);
  const double T = (double)P->g.nblocks * P->g.bh * P->g.bw * 4;
  const double pix = (double)P->g.W * P->g.H * P->bytes;
  // the new frames' forward transforms: one launch for all of them
  for (size_t i = 0; i < d.fwd.size();) {
    const size_t e = std::min(d.fwd.size(), i + (size_t)fft3d::kMaxFwdFrames);
    TimeScope ts(P, K_FORWARD, (double)(e - i) * (pix + S), st);
    fft3d::FwdFrameSet fs{};
    fs.count = (int)(e - i);
    for (size_t k = i; k < e; k++) {
      fs.src[k - i] = d.fwd[k].a.src;
      fs.stride[k - i] = d.fwd[k].a.src_stride;
      fs.spec[k - i] = d.fwd[k].a.spec;
    }
    if (P->d_tc) {
      CK(fft3d::launch_forward_tc_frames(d.fwd[i].a, fs, P->d_tc, P->d_err, d.fwd[i].bytes, st),
         "tensor-core forward kernel (frame group)");
    } else if (e - i == 1) {
      CK(fft3d::launch_forward(d.fwd[i].a, d.fwd[i].bytes, st), "forward kernel");
    } else {
      CK(fft3d::launch_forward_frames(d.fwd[i].a, fs, d.fwd[i].bytes, st), "forward kernel (frame group)");
    }
    g_launches++;
    i = e;
  }
  // the plane copies (a cropped frame's source plane, whose interior the
  // overlap-add then overwrites; Kalman frame 0): before any overlap-add,
  // which a run's filter/inverse launch may do itself
  for (const auto& c : d.copies)
    CK(cudaMemcpy2DAsync(c.dst, c.dpitch, c.src, c.spitch, c.width, c.height, cudaMemcpyDeviceToDevice, st),
       "plane copy");
  std::vector<char> ola_done(d.ola.size(), 0);  // overlap-adds done by a run's launch
  for (size_t i = 0; P->group_split == 2 && i < d.inv.size();) {
    // One launch per run of up to group_run_frames consecutive frames of one mode,
    // one CTA per block: each window spectrum (and a Kalman state) is read
    // once for the run and every filtered tile stays in shared memory.
    const int mode = d.inv[i].mode;
    size_t e = i + 1;
    while (e < d.inv.size() && d.inv[e].mode == mode &&
           (int)(e - i) < fft3d::group_run_frames(P->g.bw, P->g.bh))
      e++;
    const int n = (int)(e - i);
    fft3d::TemporalSet ts{};
    ts.count = n;
    std::vector<const float2*> seen;
    for (size_t k = i; k < e; k++) {
      for (int w = 0; w < 5; w++) {
        const float2* sp = d.inv[k].a.in[w];
        if (!sp) continue;
        ts.spec[(k - i) + w] = sp;
        if (std::find(seen.begin(), seen.end(), sp) == seen.end()) seen.push_back(sp);
      }
      ts.tdom[k - i] = d.inv[k].a.tdom;
    }
    const double state = mode == fft3d::MODE_KALMAN ? 2.0 * (double)P->spec_elems() * 16 : 0.0;
    fft3d::OlaFuse of{};
    const bool fused = fuse_run_ola(P, d, ts, i, e, ola_done, &of, st);
    // reads: each window spectrum of the run once (+ Kalman state); writes: the
    // time-domain blocks, or with the overlap-adds fused the output pixels
    TimeScope tsc(P, K_INVERSE, (double)seen.size() * S + state + n * (fused ? pix : T), st);
    fft3d::InverseArgs ga = d.inv[i].a;
    for (auto& p : ga.in) p = nullptr;
    const cudaError_t le = fft3d::launch_filter_inverse_group(ga, ts, mode, st, fused ? &of : nullptr);
    if (le != cudaSuccess && fused) P->ola_epoch--;  // no arrivals were counted for this epoch
    CK(le, "filter/inverse kernel (frame group)");
    g_launches++;
    i = e;
  }
  for (size_t i = 0; P->group_split == 1 && i < d.inv.size();) {
    // Two passes per run of consecutive frames of one mode: the filter of all
    // the run's frames (each window spectrum and the Kalman state read once),
    // then the sharpen/dehalo pass and the inverse transform of each frame.
    const int mode = d.inv[i].mode;
    size_t e = i + 1;
    while (e < d.inv.size() && d.inv[e].mode == mode && (int)(e - i) < fft3d::kMaxGroupFrames &&
           (int)(e - i) < (int)P->filt_frames.size())
      e++;
    const int n = (int)(e - i);
    fft3d::FrameSet fs{};
    fs.count = n;
    if (mode != fft3d::MODE_SHARPEN_ONLY) {
      fft3d::FilterFrameSet ff{};
      ff.count = n;
      std::vector<const float2*> seen;
      for (size_t k = i; k < e; k++) {
        for (int w = 0; w < 5; w++) {
          const float2* sp = d.inv[k].a.in[w];
          if (!sp) continue;
          ff.spec[(k - i) + w] = sp;
          if (std::find(seen.begin(), seen.end(), sp) == seen.end()) seen.push_back(sp);
        }
        ff.out[k - i] = P->filt_frames[k - i];
      }
      const double state = mode == fft3d::MODE_KALMAN ? 2.0 * (double)P->spec_elems() * 16 : 0.0;
      // reads: each window spectrum of the run once (+ Kalman state); writes: the filtered spectra
      TimeScope ts(P, K_FILTER, (double)seen.size() * S + state + n * S, st);
      CK(fft3d::launch_filter_frames(d.inv[i].a, ff, mode, st), "filter kernel (frame group)");
      g_launches++;
    }
    for (size_t k = i; k < e; k++) {
      fs.in[k - i][2] = mode == fft3d::MODE_SHARPEN_ONLY ? d.inv[k].a.in[2] : P->filt_frames[k - i];
      fs.tdom[k - i] = d.inv[k].a.tdom;
    }
    {
      // reads: the filtered spectra; writes: the time-domain blocks
      TimeScope ts(P, K_INVERSE, n * (S + T), st);
      fft3d::InverseArgs sa = d.inv[i].a;
      for (auto& p : sa.in) p = nullptr;
      CK(fft3d::launch_filter_inverse_frames(sa, fs, fft3d::MODE_SHARPEN_ONLY, st),
         "sharpen/inverse kernel (frame group)");
      g_launches++;
    }
    i = e;
  }
  for (size_t i = 0; !P->group_split && i < d.inv.size();) {
    const int mode = d.inv[i].mode;
    size_t e = i + 1;
    if (mode >= 2)
      while (e < d.inv.size() && d.inv[e].mode == mode && (int)(e - i) < fft3d::kMaxGroupFrames) e++;
    std::vector<const float2*> seen;
    for (size_t k = i; k < e; k++)
      for (const float2* p : d.inv[k].a.in)
        if (p && std::find(seen.begin(), seen.end(), p) == seen.end()) seen.push_back(p);
    // reads: each window spectrum of the run once; writes: the time-domain blocks
    TimeScope ts(P, K_INVERSE, (double)seen.size() * S + (double)(e - i) * T, st);
    if (e - i == 1) {
      CK(fft3d::launch_filter_inverse(d.inv[i].a, mode, st), "filter/inverse kernel");
    } else {
      fft3d::FrameSet fs{};
      fs.count = (int)(e - i);
      for (size_t k = i; k < e; k++) {
        for (int w = 0; w < 5; w++) fs.in[k - i][w] = d.inv[k].a.in[w];
        fs.tdom[k - i] = d.inv[k].a.tdom;
      }
      CK(fft3d::launch_filter_inverse_frames(d.inv[i].a, fs, mode, st), "filter/inverse kernel (frame group)");
    }
    g_launches++;
    i = e;
  }
  // the other overlap-adds: one launch for all frames where the 4-pixel kernel applies
  std::vector<const fft3d::Deferred::Ola*> rest;
  for (size_t k = 0; k < d.ola.size(); k++)
    if (!ola_done[k]) rest.push_back(&d.ola[k]);
  bool merged = false;
  if (rest.size() > 1 && rest.size() <= (size_t)fft3d::kMaxGroupFrames) {
    fft3d::OlaFrameSet fs{};
    fs.count = (int)rest.size();
    for (size_t k = 0; k < rest.size(); k++) {
      fs.tdom[k] = rest[k]->a.tdom;
      fs.dst[k] = rest[k]->a.dst;
      fs.dst_stride[k] = rest[k]->a.dst_stride;
    }
    if (fft3d::overlap_add_frames_supported(rest[0]->a, fs, rest[0]->bytes)) {
      TimeScope ts(P, K_OLA, (double)rest.size() * (T + pix), st);
      CK(fft3d::launch_overlap_add_frames(rest[0]->a, fs, rest[0]->bytes, st), "overlap-add kernel (frame group)");
      merged = true;
      g_launches++;
    }
  }
  if (!merged)
    for (const auto* o : rest) {
      TimeScope ts(P, K_OLA, T + pix, st);
      CK(fft3d::launch_overlap_add(o->a, o->bytes, st), "overlap-add kernel");
      g_launches++;
    }
  return FFT3D_OK;
}

int finish_call(fft3d_plane* P, cudaEvent_t done, fft3d_plane::Stage* sg, bool learned) {
  const cudaError_t e = cudaEventSynchronize(done);
  give_sync_event(P, done);
  if (e != cudaSuccess) return cuda_fail(e, "synchronize");
  const int flags[2] = {sg->h_flags[0], sg->h_flags[1]};
  for (int k = 0; k < 2; k++) {
    const int flag = flags[k];
    if (!flag) continue;
    int* dflag = k == 0 ? P->d_err : (learned ? fft3d::psd::err_flag(P->psd_model) : nullptr);
    if (dflag) cudaMemset(dflag, 0, sizeof(int));
    return fail(FFT3D_E_CUDA, (flag & 4) ? "neo_fft3d: a bounds check of the checked build failed"
                              : (flag & 2) ? "neo_fft3d: bulk copy completion wait timed out"
                                           : "neo_fft3d: tensor-core MMA completion wait timed out");
  }
  return FFT3D_OK;
}

}  // namespace

namespace fft3d {
void set_last_error(const std::string& msg) { g_err = msg; }

int plane_plan(fft3d_plane* P, int n, const void* const src[5], const int stride[5], void* dst, int dst_stride,
               cudaStream_t st, Deferred* d, const FrameGroup* grp) {
  cudaSetDevice(P->device);
  if (grp) {
    int lo, hi;
    group_range(P, grp->n0, grp->count, &lo, &hi);
    int rc = group_resources(P, lo, hi, grp->count);
    if (rc) return rc;
    P->occ = n - grp->n0;
    P->keep_lo = lo;
    P->keep_hi = hi;
    P->fixed_reverse = grp->reverse;
  }
  g_defer = d;
  const int rc = run_filter(P, n, src, stride, dst, dst_stride, false, st);
  g_defer = nullptr;
  P->occ = 0;
  P->keep_lo = 1;
  P->keep_hi = 0;
  P->fixed_reverse = -1;
  return rc;
}

int plane_bt(const fft3d_plane* P) { return P->ep.bt; }
void plane_discard(fft3d_plane* P, const Deferred& d) { discard_recorded(P, d); }
void plane_mark_work(fft3d_plane* P, cudaStream_t st);

std::mutex& plane_mutex(fft3d_plane* P) { return P->mu; }
int plane_device(const fft3d_plane* P) { return P->device; }

std::string plane_batchable(const fft3d_plane* P) {
  if (P->path != 1) return "the batched scheduler runs the default (unfused) path";
  if (P->d_tc) return "tensor-core planes are not batched";
  if (P->psd_model) return "planes with a learned noise PSD are not batched";
  if (P->bulk) return "the bulk-staged inverse is not batched";
  if (P->ep.pshow && P->ep.pfactor != 0) return "pshow planes are not batched";
  return "";
}

void count_launches(uint64_t n) { g_launches += n; }
int engine_fail(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace fft3d

namespace {

// Records the completion of the work just queued for P on stream st.
void mark_work(fft3d_plane* P, cudaStream_t st) {
  if (!P->last_work && cudaEventCreateWithFlags(&P->last_work, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    P->last_work = nullptr;
    return;
  }
  cudaEventRecord(P->last_work, st);
}

int check_group_args(const fft3d_plane* P, int count, const void* const* src, const int* src_stride,
                     void* const* dst, const int* dst_stride) {
  if (!P || !src || !src_stride || !dst || !dst_stride || count < 1 || count > FFT3D_MAX_FRAME_GROUP)
    return fail(FFT3D_E_PARAM, "neo_fft3d: invalid frame group arguments");
  for (int j = 0; j < count; j++)
    if (!dst[j]) return fail(FFT3D_E_PARAM, "neo_fft3d: null output frame in a frame group");
  return FFT3D_OK;
}

// Whether a call of `count` frames runs as a frame group: planes on the
// default or the tensor-core path. Their new frames' forward transforms and
// their overlap-adds run as one launch each; the filter/inverse runs as one
// launch per run of
// Wiener 3D frames and one launch per frame otherwise (Kalman, whose state
// runs from frame to frame, in frame order).
bool group_path(const fft3d_plane* P, int count) {
  return count > 1 && (P->path == 1 || P->path == 3) && !P->psd_model && !P->bulk &&
         !(P->ep.pshow && P->ep.pfactor != 0);
}

// Frames n0 .. n0 + count - 1 from device frames (the window of frame n0 + j
// is src[j .. j + 4]), queued on st; the caller holds P->mu.
int filter_group(fft3d_plane* P, int n0, int count, const void* const* src, const int* src_stride,
                 void* const* dst, const int* dst_stride, cudaStream_t st) {
  if (!group_path(P, count)) {
    for (int j = 0; j < count; j++) {
      int rc = run_filter(P, n0 + j, src + j, src_stride + j, dst[j], dst_stride[j], false, st);
      if (rc) return rc;
    }
    return FFT3D_OK;
  }
  int lo, hi;
  group_range(P, n0, count, &lo, &hi);
  int rc = group_resources(P, lo, hi, count);
  if (rc) return rc;
  fft3d::Deferred d;
  P->keep_lo = lo;
  P->keep_hi = hi;
  P->fixed_reverse = (int)(P->groups_done++ & 1);
  for (int j = 0; j < count && rc == FFT3D_OK; j++) {
    P->occ = j;
    d.plane = j;
    g_defer = &d;
    rc = run_filter(P, n0 + j, src + j, src_stride + j, dst[j], dst_stride[j], false, st);
    g_defer = nullptr;
  }
  P->occ = 0;
  P->keep_lo = 1;
  P->keep_hi = 0;
  P->fixed_reverse = -1;
  if (rc) {
    discard_recorded(P, d);
    return rc;
  }
  return run_group(P, d, st);
}

// Device planes of a host frame group's stage: `nin` input and `nout`
// output planes (grown, never shrunk; growing waits for the stage's previous
// use), its events and its pinned flag.
int group_stage_size(fft3d_plane* P, fft3d_plane::GroupStage* gs, int nin, int nout) {
  const size_t plane = (size_t)P->d.width * P->bytes * P->d.height;
  if (gs->nin < nin || gs->nout < nout) {
    if (gs->in_free) {
      cudaEventSynchronize(gs->in_free);
      cudaEventSynchronize(gs->out_free);
    }
    dfree(P, gs->in, plane * gs->nin);
    dfree(P, gs->out, plane * gs->nout);
    gs->in = gs->out = nullptr;
    gs->nin = gs->nout = 0;
    if (dmalloc(P, &gs->in, plane * nin) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (frame group staging)");
    }
    gs->nin = nin;
    if (dmalloc(P, &gs->out, plane * nout) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (frame group staging)");
    }
    gs->nout = nout;
  }
  if (!gs->in_free) {
    if (cudaEventCreateWithFlags(&gs->in_free, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&gs->out_free, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&gs->h_flags, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FFT3D_E_CUDA, "neo_fft3d: frame group staging setup failed");
    }
    gs->h_flags[0] = 0;
  }
  return FFT3D_OK;
}

// A group stage for one host frame-group call, exclusive until the call
// returns: its pinned error flag is read after the call's wait, so no other
// call may reset it meanwhile (a call waits while all stages are owned).
struct GroupStageLease {
  fft3d_plane* P;
  fft3d_plane::GroupStage* gs = nullptr;
  explicit GroupStageLease(fft3d_plane* p) : P(p) {
    std::unique_lock<std::mutex> lk(P->pool_mu);
    for (;;) {
      for (int k = 0; k < fft3d_plane::kGroupStages; k++) {
        const int i = (P->next_gstage + k) % fft3d_plane::kGroupStages;
        if (!P->gstages[i].busy) {
          gs = &P->gstages[i];
          gs->busy = true;
          P->next_gstage = (i + 1) % fft3d_plane::kGroupStages;
          return;
        }
      }
      P->gstage_cv.wait(lk);
    }
  }
  ~GroupStageLease() {
    {
      std::lock_guard<std::mutex> lk(P->pool_mu);
      gs->busy = false;
    }
    P->gstage_cv.notify_one();
  }
  GroupStageLease(const GroupStageLease&) = delete;
  GroupStageLease& operator=(const GroupStageLease&) = delete;
};

// Host frame group: the frames the group needs and the ring lacks go up on
// the upload stream into the stage's planes, the group runs on the plane's
// stream, and its outputs come down on the download stream; the plane's
// lock is held only while the call is queued (as in fft3d_plane_filter).
int filter_group_host(fft3d_plane* P, int n0, int count, const void* const* src, const int* src_stride,
                      void* const* dst, const int* dst_stride) {
  cudaEvent_t done = nullptr;
  GroupStageLease lease(P);
  fft3d_plane::GroupStage* gs = lease.gs;
  {
    std::lock_guard<std::mutex> lk(P->mu);
    CK(cudaSetDevice(P->device), "cudaSetDevice");
    cudaStream_t st = P->stream;
    int rc = group_stage_size(P, gs, count + 4, count);
    if (rc) return rc;
    const size_t row = (size_t)P->d.width * P->bytes;
    const size_t plane = row * P->d.height;
    int lo, hi;
    group_range(P, n0, count, &lo, &hi);
    lo = std::max(lo, 0);
    hi = std::min(hi, P->d.num_frames - 1);
    const void* dsrc[FFT3D_MAX_FRAME_GROUP + 4] = {};
    int dsstride[FFT3D_MAX_FRAME_GROUP + 4] = {};
    bool need[FFT3D_MAX_FRAME_GROUP + 4] = {};
    bool uploads = false;
    for (int m = lo; m <= hi; m++) {
      if (find_slot(P, m)) continue;
      const int k = m - (n0 - 2);
      if (!src[k])
        return fail(FFT3D_E_FRAME, "neo_fft3d: frame " + std::to_string(m) + " is needed but was not supplied");
      need[k] = true;
      dsrc[k] = gs->in + k * plane;
      dsstride[k] = (int)row;
      uploads = true;
    }
    if (uploads) {
      // the kernels that read the stage's previous frames are done
      CK(cudaStreamWaitEvent(P->s_up, gs->in_free, 0), "event");
      for (int k = 0; k < count + 4;) {
        if (!need[k]) {
          k++;
          continue;
        }
        // a run of frames that are contiguous unpadded planes in host memory
        // moves in one copy
        int e = k + 1;
        if ((size_t)src_stride[k] == row)
          while (e < count + 4 && need[e] && (size_t)src_stride[e] == row &&
                 static_cast<const char*>(src[e]) == static_cast<const char*>(src[e - 1]) + plane)
            e++;
        if (e - k > 1)
          CK(cudaMemcpyAsync(gs->in + k * plane, src[k], plane * (e - k), cudaMemcpyHostToDevice, P->s_up),
             "frame upload");
        else
          CK(cudaMemcpy2DAsync(gs->in + k * plane, row, src[k], src_stride[k], row, P->d.height,
                               cudaMemcpyHostToDevice, P->s_up),
             "frame upload");
        k = e;
      }
    }
    if (uploads) {
      rc = stream_after(P, st, P->s_up);
      if (rc) return rc;
    }
    // the stage's previous outputs must have been downloaded
    CK(cudaStreamWaitEvent(st, gs->out_free, 0), "event");
    void* ddst[FFT3D_MAX_FRAME_GROUP];
    int ddstride[FFT3D_MAX_FRAME_GROUP];
    for (int j = 0; j < count; j++) {
      ddst[j] = gs->out + j * plane;
      ddstride[j] = (int)row;
    }
    rc = filter_group(P, n0, count, dsrc, dsstride, ddst, ddstride, st);
    if (rc) return rc;
    CK(cudaEventRecord(gs->in_free, st), "event");
    rc = stream_after(P, P->s_down, st);
    if (rc) return rc;
    for (int j = 0; j < count;) {
      int e = j + 1;
      if ((size_t)dst_stride[j] == row)
        while (e < count && (size_t)dst_stride[e] == row &&
               static_cast<char*>(dst[e]) == static_cast<char*>(dst[e - 1]) + plane)
          e++;
      if (e - j > 1)
        CK(cudaMemcpyAsync(dst[j], gs->out + j * plane, plane * (e - j), cudaMemcpyDeviceToHost, P->s_down),
           "result download");
      else
        CK(cudaMemcpy2DAsync(dst[j], dst_stride[j], gs->out + j * plane, row, row, P->d.height,
                             cudaMemcpyDeviceToHost, P->s_down),
           "result download");
      j = e;
    }
    CK(cudaEventRecord(gs->out_free, P->s_down), "event");
    gs->h_flags[0] = 0;
    CK(cudaMemcpyAsync(gs->h_flags, P->d_err, sizeof(int), cudaMemcpyDeviceToHost, P->s_down), "error flag");
    done = take_sync_event(P);
    CK(cudaEventRecord(done, P->s_down), "event");
  }
  cudaSetDevice(P->device);
  const cudaError_t e = cudaEventSynchronize(done);
  give_sync_event(P, done);
  if (e != cudaSuccess) return cuda_fail(e, "synchronize");
  if (gs->h_flags[0]) {
    const int flag = gs->h_flags[0];
    cudaMemset(P->d_err, 0, sizeof(int));
    return fail(FFT3D_E_CUDA, (flag & 4) ? "neo_fft3d: a bounds check of the checked build failed"
                                         : "neo_fft3d: a bounded completion wait timed out");
  }
  return FFT3D_OK;
}

}  // namespace

namespace fft3d {
void plane_mark_work(fft3d_plane* P, cudaStream_t st) { mark_work(P, st); }
}  // namespace fft3d

extern "C" {

void fft3d_params_default(fft3d_params* p) {
  // src/fft3d.hpp:77-106
  std::memset(p, 0, sizeof(*p));
  p->sigma = 2.0f; p->beta = 1.0f;
  p->bw = 32; p->bh = 32; p->bt = 3; p->ow = -1; p->oh = -1;
  p->kratio = 2.0f; p->sharpen = 0.0f; p->scutoff = 0.3f; p->svr = 1.0f; p->smin = 4.0f; p->smax = 20.0f;
  p->measure = 1; p->interlaced = 0; p->wintype = 0;
  p->pframe = 0; p->px = 0; p->py = 0; p->pshow = 0;
  p->pcutoff = 0.1f; p->pfactor = 0.0f;
  p->sigma2 = p->sigma3 = p->sigma4 = 2.0f;
  p->degrid = 1.0f; p->dehalo = 0.0f; p->hr = 2.0f; p->ht = 50.0f;
  p->opt = 0; p->ncpu = 2; p->mt = 0;
}

const char* fft3d_last_error(void) { return g_err.c_str(); }

uint64_t fft3d_kernel_launches(void) { return g_launches.load(); }

int fft3d_plane_create(const fft3d_params* p, const fft3d_plane_desc* d, int device, fft3d_plane** out) {
  if (!p || !d || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  *out = nullptr;
  auto* P = new fft3d_plane();
  P->ep = *p;
  P->d = *d;
  P->device = device;
  {
    const char* f = std::getenv("NEO_FFT3D_PATH");
    std::string v = f ? f : "unfused";
    P->path = v == "fused" ? 2 : (v == "split" ? 0 : (v == "tc" ? 3 : 1));
    // filter/inverse kernel of the unfused and tc paths: register-pipelined (default) or bulk-staged
    const char* iv = std::getenv("NEO_FFT3D_INV");
    P->bulk = iv && std::string(iv) == "bulk";
    const char* gf = std::getenv("NEO_FFT3D_GROUP_FILTER");
    const std::string gv = gf ? gf : "block";
    P->group_split = gv == "fused" ? 0 : (gv == "split" ? 1 : 2);
    const char* fo = std::getenv("NEO_FFT3D_FUSED_OLA");
    P->fuse_ola = fo && std::string(fo) == "1";
  }
  fft3d_params& ep = P->ep;
  if (d->bits < 8 || (d->bits > 16 && d->bits != 32)) { delete P; return fail(FFT3D_E_PARAM, "neo_fft3d: unsupported bit depth"); }
  P->bytes = d->bits <= 8 ? 1 : (d->bits <= 16 ? 2 : 4);
  // bit-depth scaling, src/fft3d_engine.h:91-103
  float factor = P->bytes == 1 ? 1.0f : (P->bytes == 2 ? float(1 << (d->bits - 8)) : 1 / 255.0f);
  ep.sigma *= factor; ep.sigma2 *= factor; ep.sigma3 *= factor; ep.sigma4 *= factor;
  ep.smin *= factor; ep.smax *= factor;
  // reference checks and defaults, src/fft3d_engine.h:105-126
  if (ep.ow * 2 > ep.bw) { delete P; return fail(FFT3D_E_PARAM, "ow must be less than bw / 2"); }
  if (ep.oh * 2 > ep.bh) { delete P; return fail(FFT3D_E_PARAM, "oh must be less than bh / 2"); }
  if (ep.ow < 0) ep.ow = ep.bw / 3;
  if (ep.oh < 0) ep.oh = ep.bh / 3;
  if (ep.bt < -1 || ep.bt > 5) { delete P; return fail(FFT3D_E_PARAM, "bt must be -1 (Sharpen), 0 (Kalman), 1..5 (Wiener)"); }
  if (ep.beta < 1) { delete P; return fail(FFT3D_E_PARAM, "beta must be not less 1.0"); }
  if (!fft3d::block_size_supported(ep.bw, ep.bh)) {
    delete P;
    return fail(FFT3D_E_UNSUPPORTED, "neo_fft3d: block size " + std::to_string(ep.bw) + "x" + std::to_string(ep.bh) +
                                         " is not built into this library (bw, bh in 8,12,16,24,32,48)");
  }

  // crop in plane units, src/buffer.cpp:564-570
  P->l = d->is_chroma ? (ep.l >> d->ssw) : ep.l;
  int r = d->is_chroma ? (ep.r >> d->ssw) : ep.r;
  P->t = d->is_chroma ? (ep.t >> d->ssh) : ep.t;
  int b = d->is_chroma ? (ep.b >> d->ssh) : ep.b;
  Geom& g = P->g;
  g.W = d->width - P->l - r;
  g.H = d->height - P->t - b;
  if (g.W <= 0) { delete P; return fail(FFT3D_E_PARAM, "Width cannot be cropped to zero or below"); }
  if (g.H <= 0) { delete P; return fail(FFT3D_E_PARAM, "Height cannot be cropped to zero or below"); }
  if (ep.interlaced && (g.H & 1)) { delete P; return fail(FFT3D_E_UNSUPPORTED, "neo_fft3d: interlaced planes need an even height"); }
  g.bw = ep.bw; g.bh = ep.bh; g.ow = ep.ow; g.oh = ep.oh;
  g.sx = ep.bw - ep.ow; g.sy = ep.bh - ep.oh;
  g.nox = (g.W - ep.ow + (ep.bw - ep.ow - 1)) / (ep.bw - ep.ow) + 2;  // :115-121
  g.noy = (g.H - ep.oh + (ep.bh - ep.oh - 1)) / (ep.bh - ep.oh) + 2;
  g.nblocks = g.nox * g.noy;
  g.nh = ep.bw / 2 + 1;
  g.interlaced = ep.interlaced ? 1 : 0;
  // tables
  std::vector<float> axl, axr, sxl, sxr, ayl, ayr, syl, syr;
  windows(ep, ep.ow, axl, axr, sxl, sxr);
  windows(ep, ep.oh, ayl, ayr, syl, syr);
  std::vector<float> wx = full_window(ep.bw, ep.ow, axl, axr), wy = full_window(ep.bh, ep.oh, ayl, ayr);
  P->h_wan_x = wx;
  const int bh = ep.bh, bw = ep.bw, nh = g.nh, nb = bh * nh;
  std::vector<float> wsharpen(nb), wdehalo(nb);
  float wmax = 0;
  for (int j = 0; j < bh; j++) {  // :285-327
    int dj = j >= bh / 2 ? bh - j : j;
    float d2v = float(dj * dj) * (ep.svr * ep.svr) / ((bh / 2) * (bh / 2));
    for (int i = 0; i < nh; i++) {
      float d2 = d2v + float(i * i) / ((bw / 2) * (bw / 2));
      wsharpen[j * nh + i] = (float)(1 - std::exp((double)(-d2 / (2 * ep.scutoff * ep.scutoff))));
      float dh = (float)(std::exp((double)(-0.7f * d2 * ep.hr * ep.hr)) - std::exp((double)(-d2 * ep.hr * ep.hr)));
      wdehalo[j * nh + i] = dh;
      if (dh > wmax) wmax = dh;
    }
  }
  for (auto& v : wdehalo) v /= wmax;
  P->norm = 1.0f / (ep.bw * ep.bh);  // :329-336
  P->sigma2n_2d = ep.sigma * ep.sigma / P->norm;
  P->smin2n = ep.smin * ep.smin / P->norm;
  P->smax2n = ep.smax * ep.smax / P->norm;
  P->ht2n = ep.ht * ep.ht / P->norm;
  P->h_pwin.assign(nb, 0.f);  // :346-361
  for (int j = 0; j < bh; j++) {
    int dj = std::min(j, bh - j);
    float fh = dj * 2.0f / bh, fh2 = fh * fh;
    for (int i = 0; i < nh; i++) {
      float fw2 = (i * 2.0f / bw) * (i * 2.0f / bw);
      P->h_pwin[j * nh + i] = (fh2 + fw2) / (fh2 + fw2 + ep.pcutoff * ep.pcutoff);
    }
  }
  P->h_pattern2d.assign(nb, 0.f);
  if ((ep.sigma2 != ep.sigma || ep.sigma3 != ep.sigma || ep.sigma4 != ep.sigma) && ep.pfactor == 0) {
    // SigmasToPattern, src/helper.cpp:14-43; src/fft3d_engine.h:366-371
    float ft2 = (float)(std::sqrt((double)0.5f) / 2), ft3 = (float)(std::sqrt((double)0.5f) / 4);
    for (int h = 0; h < bh; h++)
      for (int w = 0; w < nh; w++) {
        float fy = (bh - 2.0f * std::abs(h - bh / 2)) / bh;
        float fx = (w * 1.0f) / nh;
        float f = (float)std::sqrt((double)((fx * fx + fy * fy) * 0.5f));
        float s;
        if (f < ft3) s = ep.sigma4 + (ep.sigma3 - ep.sigma4) * f / ft3;
        else if (f < ft2) s = ep.sigma3 + (ep.sigma2 - ep.sigma3) * (f - ft3) / (ft2 - ft3);
        else s = ep.sigma + (ep.sigma2 - ep.sigma) * (1 - f) / (1 - ft2);
        P->h_pattern2d[h * nh + w] = s * s / P->norm;
      }
    P->pattern_set = true;
    ep.pfactor = 1;
  }
  P->pattern = ep.pfactor != 0;
  double maxv = P->bytes == 1 ? 255.0 : (P->bytes == 2 ? (double)((1 << d->bits) - 1) : 1.0);
  gridsample(wx, wy, maxv, bw, bh, P->h_grid);

  if (const char* cap = std::getenv("NEO_FFT3D_DEVICE_ALLOC_CAP")) P->alloc_cap = std::strtoull(cap, nullptr, 10);
  // device resources
  int rc = FFT3D_OK;
  auto bail = [&](int code) { free_plane(P); return code; };
  {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaSetDevice"); return bail(rc == FFT3D_E_CUDA ? FFT3D_E_NOLIB : rc); }
  }
  if ((rc = ensure_twiddles(device))) return bail(rc);
  {
    cudaError_t e = cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->s_up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->s_down, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(e, "stream create"));
  }
  // one table allocation: wan_x, wan_y, wsyn_xl/xr, wsyn_yl/yr, grid, wsharpen, wdehalo, pattern2d, pattern3d
  std::vector<float> blob;
  auto put = [&](const std::vector<float>& v) {
    size_t off = blob.size();
    blob.insert(blob.end(), v.begin(), v.end());
    while (blob.size() % 4) blob.push_back(0.f);
    return off;
  };
  auto one = [](std::vector<float> v) { if (v.empty()) v.push_back(1.f); return v; };
  size_t o_wx = put(wx), o_wy = put(wy), o_sxl = put(one(sxl)), o_sxr = put(one(sxr)), o_syl = put(one(syl)),
         o_syr = put(one(syr)), o_grid = put(P->h_grid), o_wsh = put(wsharpen), o_wdh = put(wdehalo),
         o_p2 = put(P->h_pattern2d), o_p3 = put(std::vector<float>(nb, 0.f));
  {
    cudaError_t e = dmalloc(P, &P->d_tables, blob.size() * sizeof(float));
    if (e != cudaSuccess) return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (tables)"));
    e = cudaMemcpy(P->d_tables, blob.data(), blob.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(cuda_fail(e, "table upload"));
  }
  float* T = static_cast<float*>(P->d_tables);
  P->d_wan_x = T + o_wx;
  P->d_wan_y = T + o_wy;
  P->tab.wan_x = T + o_wx;
  P->tab.wan_y = T + o_wy;
  P->tab.wsyn_xl = T + o_sxl;
  P->tab.wsyn_xr = T + o_sxr;
  P->tab.wsyn_yl = T + o_syl;
  P->tab.wsyn_yr = T + o_syr;
  P->tab.grid = reinterpret_cast<const float2*>(T + o_grid);
  P->tab.wsharpen = T + o_wsh;
  P->tab.wdehalo = T + o_wdh;
  P->d_pattern2d = T + o_p2;
  P->d_pattern3d = T + o_p3;
  P->tab.pattern2d = P->d_pattern2d;
  P->tab.pattern3d = P->d_pattern3d;
  // spectrum ring: bt frames for the window plus slack for look-ahead
  int nslots = (ep.bt > 1 ? ep.bt : 1) + 2;
  P->slots.resize(nslots);
  for (auto& s : P->slots) {
    if (dmalloc(P, &s.spec, P->spec_elems() * sizeof(float2)) != cudaSuccess)
      return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (spectrum ring)"));
  }
  if (P->path == 3 && ep.bw == 32 && ep.bh == 32) {
    std::vector<uint8_t> tc(fft3d::forward_tc_table_bytes());
    fft3d::forward_tc_tables(wx.data(), wy.data(), tc.data());
    if (dmalloc(P, &P->d_tc, tc.size()) != cudaSuccess)
      return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (tensor-core tables)"));
    if (cudaMemcpy(P->d_tc, tc.data(), tc.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(FFT3D_E_CUDA, "neo_fft3d: tensor-core table upload failed"));
  }
  if (dmalloc(P, &P->d_err, sizeof(int)) != cudaSuccess || cudaMemset(P->d_err, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (error flag)"));
  if (P->path == 0 && dmalloc(P, &P->d_filt, P->spec_elems() * sizeof(float2)) != cudaSuccess)
    return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (filtered spectrum)"));
  if (dmalloc(P, &P->d_tdom, (size_t)g.nblocks * bh * bw * sizeof(float)) != cudaSuccess)
    return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (time-domain blocks)"));
  if (ep.bt == 0) {  // Kalman state, :339-344
    if (dmalloc(P, &P->d_last, P->spec_elems() * sizeof(float2)) != cudaSuccess ||
        dmalloc(P, &P->d_cov, P->spec_elems() * sizeof(float)) != cudaSuccess ||
        dmalloc(P, &P->d_covp, P->spec_elems() * sizeof(float)) != cudaSuccess)
      return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (Kalman state)"));
  }
  for (auto& sg : P->stages) {
    if (dmalloc_pitch(P, &sg.in, &sg.in_pitch, (size_t)d->width * P->bytes, d->height) != cudaSuccess ||
        dmalloc_pitch(P, &sg.out, &sg.out_pitch, (size_t)d->width * P->bytes, d->height) != cudaSuccess ||
        cudaMallocHost(&sg.h_flags, 2 * sizeof(int)) != cudaSuccess)
      return bail(fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory (staging)"));
    if (cudaEventCreateWithFlags(&sg.in_free, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sg.out_free, cudaEventDisableTiming) != cudaSuccess)
      return bail(fail(FFT3D_E_CUDA, "neo_fft3d: event creation failed"));
  }
  *out = P;
  if ((rc = fft3d_plane_reset(P))) { *out = nullptr; return bail(rc); }
  return FFT3D_OK;
}

int fft3d_plane_reset(fft3d_plane* P) {
  if (!P) return fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  // Stream-ordered: the reset runs on the plane's stream after the work
  // already queued for the plane (on whatever stream), and the next call
  // waits for it on its own stream; the host does not wait.
  if (P->last_work) CK(cudaStreamWaitEvent(P->stream, P->last_work, 0), "reset");
  for (auto& s : P->slots) { s.frame = -1; s.stamp = 0; }
  if (P->ep.bt == 0) {
    const size_t n = P->spec_elems();
    CK(cudaMemsetAsync(P->d_last, 0, n * sizeof(float2), P->stream), "Kalman reset");
    CK(fft3d::launch_fill(P->d_cov, P->sigma2n_2d, n, P->stream), "Kalman reset");
    CK(fft3d::launch_fill(P->d_covp, P->sigma2n_2d, n, P->stream), "Kalman reset");
  }
  if (!P->reset_done) CK(cudaEventCreateWithFlags(&P->reset_done, cudaEventDisableTiming), "reset");
  CK(cudaEventRecord(P->reset_done, P->stream), "reset");
  P->reset_pending = true;
  return FFT3D_OK;
}

void fft3d_plane_destroy(fft3d_plane* P) { free_plane(P); }

int fft3d_plane_filter(fft3d_plane* P, int n, const void* const src[5], const int src_stride[5], void* dst,
                       int dst_stride) {
  if (!P || !dst) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  cudaEvent_t done = nullptr;
  bool learned = false;
  // the call owns a stage until its result is in dst
  fft3d_plane::Stage* sg = acquire_stage(P);
  struct Release {
    fft3d_plane* P;
    fft3d_plane::Stage* sg;
    ~Release() { release_stage(P, sg); }
  } release{P, sg};
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  // Pageable frames (e.g. a frame server's buffers) would be copied by the
  // driver while the plane is locked: the new frame is copied here into
  // pinned memory first, and the result comes back through pinned memory.
  int rc = stage_pageable(P, sg, n, src, src_stride, dst);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(P->mu);
    P->cur = sg;
    P->call_done = nullptr;
    rc = run_filter(P, n, src, src_stride, dst, dst_stride, true, P->stream);
    done = P->call_done;
    P->call_done = nullptr;
    P->cur = nullptr;
    sg->staged_src = nullptr;
    learned = P->psd_model != nullptr;
    if (rc) {
      if (done) {
        cudaEventSynchronize(done);
        give_sync_event(P, done);
      }
      return rc;
    }
  }
  if (!done) return FFT3D_OK;  // answered on the host (Kalman frame 0)
  cudaSetDevice(P->device);
  rc = finish_call(P, done, sg, learned);
  if (rc == FFT3D_OK && sg->pageable_out) {
    const size_t orow = (size_t)P->g.W * P->bytes;
    char* hdst = static_cast<char*>(dst) + (size_t)P->t * dst_stride + (size_t)P->l * P->bytes;
    for (int y = 0; y < P->g.H; y++) std::memcpy(hdst + (size_t)y * dst_stride, sg->h_out + (size_t)y * orow, orow);
  }
  return rc;
}

int fft3d_plane_filter_device(fft3d_plane* P, int n, const void* const src[5], const int src_stride[5], void* dst,
                              int dst_stride, void* stream) {
  if (!P || !dst) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : P->stream;
  const int rc = run_filter(P, n, src, src_stride, dst, dst_stride, false, st);
  mark_work(P, st);
  return rc;
}

int fft3d_plane_filter_frames_device(fft3d_plane* P, int n0, int count, const void* const* src, const int* src_stride,
                                     void* const* dst, const int* dst_stride, void* stream) {
  int rc = check_group_args(P, count, src, src_stride, dst, dst_stride);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  cudaStream_t st = stream ? (cudaStream_t)stream : P->stream;
  rc = filter_group(P, n0, count, src, src_stride, dst, dst_stride, st);
  mark_work(P, st);
  return rc;
}

int fft3d_plane_filter_frames(fft3d_plane* P, int n0, int count, const void* const* src, const int* src_stride,
                              void* const* dst, const int* dst_stride) {
  int rc = check_group_args(P, count, src, src_stride, dst, dst_stride);
  if (rc) return rc;
  bool grouped;
  {
    std::lock_guard<std::mutex> lk(P->mu);
    // crop borders are copied from the host frames by the one-frame host path
    grouped = group_path(P, count) && P->ep.l == 0 && P->ep.t == 0 && P->ep.r == 0 && P->ep.b == 0;
  }
  if (grouped) return filter_group_host(P, n0, count, src, src_stride, dst, dst_stride);
  for (int j = 0; j < count; j++) {
    rc = fft3d_plane_filter(P, n0 + j, src + j, src_stride + j, dst[j], dst_stride[j]);
    if (rc) return rc;
  }
  return FFT3D_OK;
}

int fft3d_plane_cached(fft3d_plane* P, int n) {
  if (!P) return 0;
  std::lock_guard<std::mutex> lk(P->mu);
  return find_slot(P, n) ? 1 : 0;
}

int fft3d_plane_spectrum(fft3d_plane* P, int n, float* out) {
  if (!P || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(P->mu);
  Slot* s = find_slot(P, n);
  if (!s) return fail(FFT3D_E_FRAME, "neo_fft3d: frame " + std::to_string(n) + " is not cached");
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(P->stream), "synchronize");
  CK(cudaMemcpy(out, s->spec, P->spec_elems() * sizeof(float2), cudaMemcpyDeviceToHost), "spectrum download");
  return FFT3D_OK;
}

int fft3d_plane_geometry(fft3d_plane* P, int out[8]) {
  if (!P || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  out[0] = P->g.nox; out[1] = P->g.noy;
  out[2] = P->g.nox * P->g.sx + P->g.ow; out[3] = P->g.noy * P->g.sy + P->g.oh;
  out[4] = P->g.nh; out[5] = P->g.nblocks; out[6] = P->g.ow; out[7] = P->g.oh;
  return FFT3D_OK;
}

// Estimate the noise pattern from one frame (host memory), as the reference
// does from frame pframe on its first GetFrame (src/fft3d_engine.h:485-504).
int fft3d_plane_set_pattern_frame(fft3d_plane* P, const void* src, int stride) {
  if (!P || !src) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  // the upload goes through a staging set of its own (taken before the
  // plane's lock, as the host-path calls do)
  fft3d_plane::Stage* sg = acquire_stage(P);
  struct Release {
    fft3d_plane* P;
    fft3d_plane::Stage* sg;
    ~Release() { release_stage(P, sg); }
  } release{P, sg};
  std::lock_guard<std::mutex> lk(P->mu);
  // pshow finds the pattern block on every frame itself (src/fft3d_engine.h:505-527)
  if (!P->pattern || P->ep.pshow) return FFT3D_OK;
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  // work already queued for the plane still reads the ring
  for (auto* st : {P->s_up, P->stream, P->s_down}) CK(cudaStreamSynchronize(st), "synchronize");
  if (P->last_work) CK(cudaEventSynchronize(P->last_work), "synchronize");
  Slot* s = evict_slot(P, 1, 0);
  s->frame = -1;
  CK(cudaMemcpy2DAsync(sg->in, sg->in_pitch, src, stride, (size_t)P->d.width * P->bytes, P->d.height,
                       cudaMemcpyHostToDevice, P->stream), "frame upload");
  int rc = launch_forward(P, sg->in, (long long)sg->in_pitch, s->spec, P->stream);
  if (rc) return rc;
  const int nb = P->g.bh * P->g.nh;
  if (P->ep.px == 0 && P->ep.py == 0) {
    rc = find_pattern_block(P, s->spec, P->stream, &P->ep.px, &P->ep.py);
    if (rc) return rc;
  }
  std::vector<float2> blk(nb);
  CK(cudaMemcpyAsync(blk.data(), s->spec + ((size_t)P->ep.py * P->g.nox + P->ep.px) * nb, nb * sizeof(float2),
                     cudaMemcpyDeviceToHost, P->stream),
     "pattern block download");
  CK(cudaStreamSynchronize(P->stream), "synchronize");
  set_pattern_from_block(P, blk.data());
  rc = upload_pattern(P, P->d_pattern2d, P->h_pattern2d, P->stream);
  if (rc) return rc;
  CK(cudaStreamSynchronize(P->stream), "synchronize");
  P->pattern_set = true;
  P->pattern3d_init = false;
  return FFT3D_OK;
}

int fft3d_plane_set_psd(fft3d_plane* P, fft3d_psd* m, int pooled, float strength) {
  if (!P) return fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  if (m && !(strength > 0.f)) return fail(FFT3D_E_PARAM, "neo_fft3d: the learned noise strength must be positive");
  std::lock_guard<std::mutex> lk(P->mu);
  cudaSetDevice(P->device);
  CK(cudaStreamSynchronize(P->stream), "synchronize");
  if (!m) {
    P->psd_model = nullptr;
    return FFT3D_OK;
  }
  const std::string why =
      fft3d::psd::check_plane(m, P->device, P->g.bw, P->g.bh, P->g.ow, P->g.oh, P->ep.wintype);
  if (!why.empty()) return fail(FFT3D_E_UNSUPPORTED, "neo_fft3d: " + why);
  if (!P->d_psd) {
    if (dmalloc(P, &P->d_psd, P->spec_elems() * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      P->d_psd = nullptr;
      return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for the learned noise power");
    }
  }
  if (!P->psd_work) {
    P->psd_work = fft3d::psd::work_create(m, P->g.nblocks);
    if (!P->psd_work) return fail(FFT3D_E_NOMEM, "neo_fft3d: out of device memory for the learned noise PSD");
  }
  // sample scale relative to 8-bit codes: 2^(bits-8) for integer samples, 1/255 for float
  const double scale = P->bytes == 4 ? 1.0 / 255.0 : std::ldexp(1.0, P->d.bits - 8);
  P->psd_pow = (float)(scale * scale);
  P->psd_model = m;
  P->psd_pooled = pooled ? 1 : 0;
  P->psd_strength = strength;
  return FFT3D_OK;
}

int fft3d_plane_device_bytes(fft3d_plane* P, uint64_t* out) {
  if (!P || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(P->mu);
  *out = P->alloc_used;
  return FFT3D_OK;
}

int fft3d_plane_synchronize(fft3d_plane* P) {
  if (!P) return fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  if (P->last_work) CK(cudaEventSynchronize(P->last_work), "synchronize");
  for (auto* st : {P->s_up, P->stream, P->s_down}) CK(cudaStreamSynchronize(st), "synchronize");
  int flags[2] = {0, 0};
  CK(cudaMemcpy(&flags[0], P->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
  if (P->psd_model) CK(cudaMemcpy(&flags[1], fft3d::psd::err_flag(P->psd_model), sizeof(int), cudaMemcpyDeviceToHost),
                       "error flag");
  for (int k = 0; k < 2; k++) {
    if (!flags[k]) continue;
    CK(cudaMemset(k == 0 ? P->d_err : fft3d::psd::err_flag(P->psd_model), 0, sizeof(int)), "error flag");
    return fail(FFT3D_E_CUDA, (flags[k] & 4) ? "neo_fft3d: a bounds check of the checked build failed"
                              : (flags[k] & 2) ? "neo_fft3d: bulk copy completion wait timed out"
                                               : "neo_fft3d: tensor-core MMA completion wait timed out");
  }
  return FFT3D_OK;
}

int fft3d_plane_debug_set_error_flag(fft3d_plane* P, int bits) {
  if (!P) return fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  // after the work already queued for the plane, like a kernel of the next call
  if (P->last_work) CK(cudaEventSynchronize(P->last_work), "synchronize");
  CK(cudaStreamSynchronize(P->stream), "synchronize");
  CK(cudaMemcpy(P->d_err, &bits, sizeof(int), cudaMemcpyHostToDevice), "error flag");
  return FFT3D_OK;
}

int fft3d_plane_set_timing(fft3d_plane* P, int enable) {
  if (!P) return fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(P->mu);
  P->timing = enable != 0;
  return FFT3D_OK;
}

int fft3d_plane_timing(fft3d_plane* P, double out[15]) {
  if (!P || !out) return fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(P->mu);
  CK(cudaSetDevice(P->device), "cudaSetDevice");
  for (auto& t : P->pending) {
    CK(cudaEventSynchronize(t.b), "event synchronize");
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, t.a, t.b), "event elapsed time");
    P->t_launches[t.kind] += 1;
    P->t_ms[t.kind] += ms;
    P->t_bytes[t.kind] += t.bytes;
    P->event_pool.push_back(t.a);
    P->event_pool.push_back(t.b);
  }
  P->pending.clear();
  for (int k = 0; k < K_COUNT; k++) {
    out[3 * k] = P->t_launches[k];
    out[3 * k + 1] = P->t_ms[k];
    out[3 * k + 2] = P->t_bytes[k];
    P->t_launches[k] = P->t_ms[k] = P->t_bytes[k] = 0;
  }
  return FFT3D_OK;
}

}  // extern "C"
