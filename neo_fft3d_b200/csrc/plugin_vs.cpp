// VapourSynth plugin shell of the B200 FFT3D core: a drop-in for the
// reference plugin's VapourSynth entry (namespace neo_fft3d, function FFT3D,
// src/neo_fft3d.hpp:13-22, include/dualsynth/vs_wrapper.hpp:206-303) with the
// same argument list and defaults (src/fft3d.hpp:29-106), the same plane
// selection, crop handling and filter modes. Each processed plane is one
// fft3d_plane of libfft3d_b200 (include/fft3d_b200.h); frames are uploaded
// to the GPU, filtered there and downloaded into the output frame.
#include <VapourSynth.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "fft3d_b200.h"

namespace {

// The outputs of one frame group (frames n0 .. n0 + k - 1), computed once by
// whichever request gets there first and then served to the others.
struct GroupOut {
  std::mutex mu;
  bool done = false;
  std::string err;
  std::vector<const VSFrameRef*> out;
};

struct FFT3DFilter {
  VSNodeRef* node = nullptr;
  VSVideoInfo vi{};
  fft3d_params p{};
  bool process[4] = {false, false, false, false};
  fft3d_plane* plane[4] = {nullptr, nullptr, nullptr, nullptr};
  bool crop = false;
  std::mutex pattern_lock;
  bool pattern_done = false;
  // Frame groups (Wiener 3D, opt-in): a request for frame n filters its whole
  // aligned group of `group` frames in one fft3d_plane_filter_frames call per
  // plane and keeps the outputs for the group's other requests (`cache`, the
  // most recent kCachedGroups groups). group <= 1: one frame per call.
  int group = 1;
  std::mutex cache_lock;
  std::map<int, std::shared_ptr<GroupOut>> cache;
  std::deque<int> cache_order;
};

constexpr int kCachedGroups = 6;

// Reads an optional argument with the reference's VS semantics: absent keys
// keep the default (include/dualsynth/vs_wrapper.hpp:114-137).
template <typename T>
void read_int(const VSMap* in, const VSAPI* api, const char* k, T& v) {
  int err = 0;
  int64_t x = api->propGetInt(in, k, 0, &err);
  if (!err) v = (T)x;
}
void read_float(const VSMap* in, const VSAPI* api, const char* k, float& v) {
  int err = 0;
  double x = api->propGetFloat(in, k, 0, &err);
  if (!err) v = (float)x;
}

void VS_CC fft3d_init(VSMap*, VSMap*, void** instance, VSNode* node, VSCore*, const VSAPI* api) {
  auto* d = static_cast<FFT3DFilter*>(*instance);
  api->setVideoInfo(&d->vi, 1, node);
}

void VS_CC fft3d_free(void* instance, VSCore*, const VSAPI* api) {
  auto* d = static_cast<FFT3DFilter*>(instance);
  for (auto& kv : d->cache)
    for (auto* f : kv.second->out)
      if (f) api->freeFrame(f);
  for (auto* h : d->plane)
    if (h) fft3d_plane_destroy(h);
  if (d->node) api->freeNode(d->node);
  delete d;
}

int plane_w(const VSVideoInfo& vi, int p) { return p ? vi.width >> vi.format->subSamplingW : vi.width; }
int plane_h(const VSVideoInfo& vi, int p) { return p ? vi.height >> vi.format->subSamplingH : vi.height; }

// Noise pattern from frame pframe, once, before the first filtered frame.
std::string ensure_pattern(FFT3DFilter* d, VSFrameContext* ctx, const VSAPI* api) {
  std::string err;
  std::lock_guard<std::mutex> lk(d->pattern_lock);
  if (d->pattern_done) return err;
  const int last = d->vi.numFrames - 1;
  const VSFrameRef* pf = api->getFrameFilter(std::min(std::max(d->p.pframe, 0), last), d->node, ctx);
  for (int p = 0; p < d->vi.format->numPlanes && err.empty(); p++)
    if (d->plane[p] && fft3d_plane_set_pattern_frame(d->plane[p], api->getReadPtr(pf, p), api->getStride(pf, p)))
      err = fft3d_last_error();
  api->freeFrame(pf);
  d->pattern_done = true;
  return err;
}

// The group's outputs: the window's frames (n0 - bt/2 .. n0 + k - 1 +
// (bt-1)/2, as requested), one fft3d_plane_filter_frames call per processed
// plane, the other planes copied.
void compute_group(FFT3DFilter* d, GroupOut* e, int n0, int k, VSFrameContext* ctx, VSCore* core, const VSAPI* api) {
  const VSFormat* fi = d->vi.format;
  const int last = d->vi.numFrames - 1;
  const int lo = std::max(n0 - d->p.bt / 2, 0), hi = std::min(n0 + k - 1 + (d->p.bt - 1) / 2, last);
  std::vector<const VSFrameRef*> src(k + 4, nullptr);  // frame n0 - 2 + j
  for (int m = lo; m <= hi; m++) src[m - (n0 - 2)] = api->getFrameFilter(m, d->node, ctx);
  e->out.assign(k, nullptr);
  for (int j = 0; j < k; j++) e->out[j] = api->newVideoFrame(fi, d->vi.width, d->vi.height, src[j + 2], core);
  for (int p = 0; p < fi->numPlanes && e->err.empty(); p++) {
    if (!d->plane[p]) {  // planes not processed are copied (process = 2)
      const int rb = plane_w(d->vi, p) * fi->bytesPerSample;
      for (int j = 0; j < k; j++) {
        const uint8_t* sp = api->getReadPtr(src[j + 2], p);
        uint8_t* dp = api->getWritePtr(const_cast<VSFrameRef*>(e->out[j]), p);
        const int ss = api->getStride(src[j + 2], p), ds = api->getStride(e->out[j], p);
        for (int y = 0; y < plane_h(d->vi, p); y++) std::memcpy(dp + (size_t)y * ds, sp + (size_t)y * ss, rb);
      }
      continue;
    }
    std::vector<const void*> ptrs(k + 4, nullptr);
    std::vector<int> strides(k + 4, 0);
    for (int j = 0; j < k + 4; j++)
      if (src[j]) {
        ptrs[j] = api->getReadPtr(src[j], p);
        strides[j] = api->getStride(src[j], p);
      }
    std::vector<void*> dst(k);
    std::vector<int> dstride(k);
    for (int j = 0; j < k; j++) {
      dst[j] = api->getWritePtr(const_cast<VSFrameRef*>(e->out[j]), p);
      dstride[j] = api->getStride(e->out[j], p);
    }
    if (fft3d_plane_filter_frames(d->plane[p], n0, k, ptrs.data(), strides.data(), dst.data(), dstride.data()))
      e->err = fft3d_last_error();
  }
  for (auto* f : src)
    if (f) api->freeFrame(f);
}

const VSFrameRef* group_get_frame(FFT3DFilter* d, int n, int reason, VSFrameContext* ctx, VSCore* core,
                                  const VSAPI* api) {
  const int G = d->group, last = d->vi.numFrames - 1;
  const int g = n / G, n0 = g * G, k = std::min(G, last + 1 - n0);
  if (reason == arInitial) {
    {
      std::lock_guard<std::mutex> lk(d->cache_lock);
      auto it = d->cache.find(g);
      if (it != d->cache.end()) {
        std::lock_guard<std::mutex> gl(it->second->mu);
        if (it->second->done && it->second->err.empty()) return api->cloneFrameRef(it->second->out[n - n0]);
      }
    }
    const int lo = std::max(n0 - d->p.bt / 2, 0), hi = std::min(n0 + k - 1 + (d->p.bt - 1) / 2, last);
    for (int m = lo; m <= hi; m++) api->requestFrameFilter(m, d->node, ctx);
    if (d->p.pfactor != 0 && !d->pattern_done)
      api->requestFrameFilter(std::min(std::max(d->p.pframe, 0), last), d->node, ctx);
    return nullptr;
  }
  if (reason != arAllFramesReady) return nullptr;
  if (d->p.pfactor != 0) {
    const std::string perr = ensure_pattern(d, ctx, api);
    if (!perr.empty()) {
      api->setFilterError(("FFT3D: " + perr).c_str(), ctx);
      return nullptr;
    }
  }
  std::shared_ptr<GroupOut> e;
  {
    std::lock_guard<std::mutex> lk(d->cache_lock);
    auto& slot = d->cache[g];
    if (!slot) {
      slot = std::make_shared<GroupOut>();
      d->cache_order.push_back(g);
      while ((int)d->cache_order.size() > kCachedGroups) {
        const int old = d->cache_order.front();
        d->cache_order.pop_front();
        auto it = d->cache.find(old);
        if (it == d->cache.end()) continue;
        // not while it is being computed; a request still holding it
        // recomputes it (its window frames are requested)
        std::lock_guard<std::mutex> gl(it->second->mu);
        for (auto* f : it->second->out)
          if (f) api->freeFrame(f);
        it->second->out.clear();
        it->second->done = false;
        d->cache.erase(it);
      }
    }
    e = slot;
  }
  std::string err;
  const VSFrameRef* out = nullptr;
  {
    std::lock_guard<std::mutex> gl(e->mu);
    if (!e->done) {
      e->err.clear();
      compute_group(d, e.get(), n0, k, ctx, core, api);
      e->done = true;
    }
    if (e->err.empty()) {
      out = api->cloneFrameRef(e->out[n - n0]);
    } else {
      err = e->err;
      for (auto* f : e->out)
        if (f) api->freeFrame(f);
      e->out.clear();
      e->done = false;
    }
  }
  if (!err.empty()) {
    {
      // a failed group is not kept (lock order: cache, then group)
      std::lock_guard<std::mutex> lk(d->cache_lock);
      auto it = d->cache.find(g);
      if (it != d->cache.end() && it->second == e) d->cache.erase(it);
    }
    api->setFilterError(("FFT3D: " + err).c_str(), ctx);
    return nullptr;
  }
  return out;
}

const VSFrameRef* VS_CC fft3d_get_frame(int n, int reason, void** instance, void**, VSFrameContext* ctx, VSCore* core,
                                        const VSAPI* api) {
  auto* d = static_cast<FFT3DFilter*>(*instance);
  if (d->group > 1) return group_get_frame(d, n, reason, ctx, core, api);
  const int bt = d->p.bt;
  const int last = d->vi.numFrames - 1;
  // frames of the temporal window, src/fft3d.hpp:201-219
  const int from = bt > 1 ? std::max(n - bt / 2, 0) : n;
  const int to = bt > 1 ? std::min(n + (bt - 1) / 2, last) : n;
  const bool need_pattern = d->p.pfactor != 0 && !d->pattern_done;
  if (reason == arInitial) {
    for (int i = from; i <= to; i++) api->requestFrameFilter(i, d->node, ctx);
    if (need_pattern) api->requestFrameFilter(std::min(std::max(d->p.pframe, 0), last), d->node, ctx);
    return nullptr;
  }
  if (reason != arAllFramesReady) return nullptr;
  const VSFrameRef* win[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  for (int i = from; i <= to; i++) win[2 + i - n] = api->getFrameFilter(i, d->node, ctx);
  const VSFrameRef* src = win[2];
  const VSFormat* fi = d->vi.format;
  VSFrameRef* dst = api->newVideoFrame(fi, d->vi.width, d->vi.height, src, core);
  std::string err;
  if (need_pattern) {
    std::lock_guard<std::mutex> lk(d->pattern_lock);
    if (!d->pattern_done) {
      const VSFrameRef* pf = api->getFrameFilter(std::min(std::max(d->p.pframe, 0), last), d->node, ctx);
      for (int p = 0; p < fi->numPlanes && err.empty(); p++)
        if (d->plane[p] && fft3d_plane_set_pattern_frame(d->plane[p], api->getReadPtr(pf, p), api->getStride(pf, p)))
          err = fft3d_last_error();
      api->freeFrame(pf);
      d->pattern_done = true;
    }
  }
  for (int p = 0; p < fi->numPlanes && err.empty(); p++) {
    uint8_t* dp = api->getWritePtr(dst, p);
    const int ds = api->getStride(dst, p);
    if (!d->plane[p]) {  // planes not processed are copied (process = 2)
      const uint8_t* sp = api->getReadPtr(src, p);
      const int ss = api->getStride(src, p);
      const int rb = plane_w(d->vi, p) * fi->bytesPerSample;
      for (int y = 0; y < plane_h(d->vi, p); y++) std::memcpy(dp + (size_t)y * ds, sp + (size_t)y * ss, rb);
      continue;
    }
    // the whole window is passed; frames whose spectra the plane still holds
    // are not uploaded again
    const void* ptrs[5];
    int strides[5];
    for (int k = 0; k < 5; k++) {
      ptrs[k] = win[k] ? api->getReadPtr(win[k], p) : nullptr;
      strides[k] = win[k] ? api->getStride(win[k], p) : 0;
    }
    if (fft3d_plane_filter(d->plane[p], n, ptrs, strides, dp, ds)) err = fft3d_last_error();
  }
  for (auto* f : win)
    if (f) api->freeFrame(f);
  if (!err.empty()) {
    api->freeFrame(dst);
    api->setFilterError(("FFT3D: " + err).c_str(), ctx);
    return nullptr;
  }
  return dst;
}

void VS_CC fft3d_create(const VSMap* in, VSMap* out, void*, VSCore* core, const VSAPI* api) {
  auto* d = new FFT3DFilter();
  auto fail = [&](const std::string& msg) {
    api->setError(out, ("FFT3D: " + msg).c_str());  // reference format, vs_wrapper.hpp:277-280
    for (auto*& h : d->plane)
      if (h) { fft3d_plane_destroy(h); h = nullptr; }
    if (d->node) api->freeNode(d->node);
    delete d;
  };
  d->node = api->propGetNode(in, "clip", 0, nullptr);
  d->vi = *api->getVideoInfo(d->node);
  const VSFormat* fi = d->vi.format;
  if (!fi || d->vi.width == 0 || d->vi.height == 0) return fail("only constant format input supported");
  // parameters and defaults, src/fft3d.hpp:77-139
  fft3d_params& p = d->p;
  fft3d_params_default(&p);
  read_float(in, api, "sigma", p.sigma);
  p.sigma2 = p.sigma3 = p.sigma4 = p.sigma;
  read_float(in, api, "beta", p.beta);
  read_int(in, api, "bw", p.bw);
  read_int(in, api, "bh", p.bh);
  read_int(in, api, "bt", p.bt);
  read_int(in, api, "ow", p.ow);
  read_int(in, api, "oh", p.oh);
  read_float(in, api, "kratio", p.kratio);
  read_float(in, api, "sharpen", p.sharpen);
  read_float(in, api, "scutoff", p.scutoff);
  read_float(in, api, "svr", p.svr);
  read_float(in, api, "smin", p.smin);
  read_float(in, api, "smax", p.smax);
  read_int(in, api, "measure", p.measure);
  read_int(in, api, "interlaced", p.interlaced);
  read_int(in, api, "wintype", p.wintype);
  read_int(in, api, "pframe", p.pframe);
  read_int(in, api, "px", p.px);
  read_int(in, api, "py", p.py);
  read_int(in, api, "pshow", p.pshow);
  read_float(in, api, "pcutoff", p.pcutoff);
  read_float(in, api, "pfactor", p.pfactor);
  read_float(in, api, "sigma2", p.sigma2);
  read_float(in, api, "sigma3", p.sigma3);
  read_float(in, api, "sigma4", p.sigma4);
  read_float(in, api, "degrid", p.degrid);
  read_float(in, api, "dehalo", p.dehalo);
  read_float(in, api, "hr", p.hr);
  read_float(in, api, "ht", p.ht);
  read_int(in, api, "l", p.l); p.l = std::max(p.l, 0);
  read_int(in, api, "t", p.t); p.t = std::max(p.t, 0);
  read_int(in, api, "r", p.r); p.r = std::max(p.r, 0);
  read_int(in, api, "b", p.b); p.b = std::max(p.b, 0);
  read_int(in, api, "opt", p.opt);
  read_int(in, api, "ncpu", p.ncpu);
  read_int(in, api, "mt", p.mt);
  d->crop = p.l > 0 || p.r > 0 || p.t > 0 || p.b > 0;
  if (p.l + p.r >= d->vi.width) return fail("Width cannot be cropped to zero or below");
  if (p.t + p.b >= d->vi.height) return fail("Height cannot be cropped to zero or below");
  // planes (default 0, 1, 2), src/fft3d.hpp:149-161
  const int np = api->propNumElements(in, "planes");
  if (np < 0) {
    for (int i = 0; i < 3 && i < fi->numPlanes; i++) d->process[i] = true;
  } else {
    for (int i = 0; i < np; i++) {
      int err = 0;
      int pl = (int)api->propGetInt(in, "planes", i, &err);
      if (!err && pl >= 0 && pl < fi->numPlanes) d->process[pl] = true;
    }
  }
  const bool yuv = fi->colorFamily == cmYUV || fi->colorFamily == cmGray;
  for (int i = 0; i < fi->numPlanes; i++) {
    if (!d->process[i]) continue;
    fft3d_plane_desc pd;
    pd.width = plane_w(d->vi, i);
    pd.height = plane_h(d->vi, i);
    pd.bits = fi->sampleType == stFloat ? 32 : fi->bitsPerSample;
    pd.is_chroma = yuv && i != 0 ? 1 : 0;
    pd.ssw = fi->subSamplingW;
    pd.ssh = fi->subSamplingH;
    pd.num_frames = d->vi.numFrames;
    pd.rgb = fi->colorFamily == cmRGB ? 1 : 0;
    if (fft3d_plane_create(&p, &pd, 0, &d->plane[i])) return fail(fft3d_last_error());
  }
  // Wiener 3D: frame groups of NEO_FFT3D_FRAME_GROUP frames when set (off by
  // default: with the core's pageable frame buffers the host copies bound the
  // plugin, and a group serialises the copies of its frames' requests)
  if (p.bt >= 2) {
    const char* env = std::getenv("NEO_FFT3D_FRAME_GROUP");
    d->group = env ? std::max(1, std::min(std::atoi(env), FFT3D_MAX_FRAME_GROUP)) : 1;
  }
  // Kalman is history-dependent: frames in order (src/fft3d.hpp:27-28)
  api->createFilter(in, out, "FFT3D", fft3d_init, fft3d_get_frame, fft3d_free, p.bt == 0 ? fmSerial : fmParallel, 0,
                    d, core);
}

// The reference's VapourSynth argument string (src/fft3d.hpp:29-73 through
// include/dualsynth/ds_filter.hpp:19-42; y/u/v are AviSynth-only).
const char* kArgs =
    "clip:clip;sigma:float:opt;beta:float:opt;planes:int[]:opt;bw:int:opt;bh:int:opt;bt:int:opt;ow:int:opt;"
    "oh:int:opt;kratio:float:opt;sharpen:float:opt;scutoff:float:opt;svr:float:opt;smin:float:opt;smax:float:opt;"
    "measure:int:opt;interlaced:int:opt;wintype:int:opt;pframe:int:opt;px:int:opt;py:int:opt;pshow:int:opt;"
    "pcutoff:float:opt;pfactor:float:opt;sigma2:float:opt;sigma3:float:opt;sigma4:float:opt;degrid:float:opt;"
    "dehalo:float:opt;hr:float:opt;ht:float:opt;l:int:opt;t:int:opt;r:int:opt;b:int:opt;opt:int:opt;ncpu:int:opt;"
    "mt:int:opt;";

}  // namespace

VS_EXTERNAL_API(void) VapourSynthPluginInit(VSConfigPlugin config, VSRegisterFunction reg, VSPlugin* plugin) {
  config("in.7086.neo_fft3d", "neo_fft3d", "Neo FFT3D Filter (B200 sm_100a)", VAPOURSYNTH_API_VERSION, 1, plugin);
  reg("FFT3D", kArgs, fft3d_create, nullptr, plugin);
}
