// AviSynth+ plugin shell of the B200 FFT3D core: a drop-in for the reference
// plugin's AviSynth+ entry (function neo_fft3d, src/fft3d.hpp:26-72 through
// include/dualsynth/avs_wrapper.hpp:205-227 and ds_filter.hpp:44-70) with the
// same parameter string, defaults, per-plane modes (y/u/v: 3 filter, 2 copy,
// other values leave the plane unwritten; src/fft3d.hpp:149-168), crop
// handling, MT mode (src/fft3d.hpp:266-269) and error messages
// ("neo_fft3d: <message>", avs_wrapper.hpp:213-221). Each filtered plane is one
// fft3d_plane of libfft3d_b200 (include/fft3d_b200.h): frames are uploaded to
// the GPU, filtered there and downloaded into the output frame.
#include <avisynth.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "fft3d_b200.h"

const AVS_Linkage* AVS_linkage = nullptr;

namespace {

struct Fail {
  std::string msg;
};

class NeoFFT3D : public GenericVideoFilter {
 public:
  NeoFFT3D(PClip child, const fft3d_params& p, const int process[4], IScriptEnvironment* env)
      : GenericVideoFilter(child), p_(p) {
    for (int i = 0; i < 4; i++) process_[i] = process[i];
    yuv_ = vi.IsYUV() || vi.IsYUVA();
    nplanes_ = vi.NumComponents();
    const int ids_yuv[4] = {PLANAR_Y, PLANAR_U, PLANAR_V, PLANAR_A};
    const int ids_rgb[4] = {PLANAR_R, PLANAR_G, PLANAR_B, PLANAR_A};
    for (int i = 0; i < 4; i++) ids_[i] = yuv_ ? ids_yuv[i] : ids_rgb[i];
    try {
      env->CheckVersion(8);
      has_v8_ = true;
    } catch (const AvisynthError&) {
      has_v8_ = false;
    }
    // the reference sizes a plane by its subsampling when the clip is YUV and
    // the plane is not the first (src/fft3d.hpp:188-191)
    for (int i = 0; i < nplanes_; i++) {
      if (process_[i] != 3) continue;
      fft3d_plane_desc d;
      const bool chroma = yuv_ && i != 0;
      const int ssw = vi.IsY() ? 0 : vi.GetPlaneWidthSubsampling(PLANAR_U);
      const int ssh = vi.IsY() ? 0 : vi.GetPlaneHeightSubsampling(PLANAR_U);
      d.width = chroma ? vi.width >> ssw : vi.width;
      d.height = chroma ? vi.height >> ssh : vi.height;
      d.bits = vi.BitsPerComponent();
      d.is_chroma = chroma ? 1 : 0;
      d.ssw = ssw;
      d.ssh = ssh;
      d.num_frames = vi.num_frames;
      d.rgb = yuv_ ? 0 : 1;
      if (fft3d_plane_create(&p_, &d, 0, &plane_[i])) {
        Fail f{fft3d_last_error()};
        release();
        throw f;
      }
      ++engines_;
    }
  }

  ~NeoFFT3D() override { release(); }

  PVideoFrame __stdcall GetFrame(int n, IScriptEnvironment* env) override {
    const int last = vi.num_frames - 1;
    n = std::min(std::max(n, 0), last);
    // the reference requests the bt window only for Wiener 3D with at least
    // one filtered plane (src/fft3d.hpp:201-219)
    const bool window = p_.bt > 1 && engines_ > 0;
    const int from = window ? std::max(n - p_.bt / 2, 0) : n;
    const int to = window ? std::min(n + (p_.bt - 1) / 2, last) : n;
    PVideoFrame win[5];
    for (int i = from; i <= to; i++) win[2 + i - n] = child->GetFrame(i, env);
    PVideoFrame src = win[2];
    if (engines_ == 0) return src;
    if (p_.pfactor != 0) set_pattern(env);
    PVideoFrame dst = has_v8_ ? env->NewVideoFrameP(vi, &src) : env->NewVideoFrame(vi);
    for (int i = 0; i < nplanes_; i++) {
      const int id = ids_[i];
      if (process_[i] == 3) {
        const void* ptrs[5];
        int strides[5];
        for (int k = 0; k < 5; k++) {
          ptrs[k] = win[k] ? win[k]->GetReadPtr(id) : nullptr;
          strides[k] = win[k] ? win[k]->GetPitch(id) : 0;
        }
        if (fft3d_plane_filter(plane_[i], n, ptrs, strides, dst->GetWritePtr(id), dst->GetPitch(id)))
          env->ThrowError("neo_fft3d: %s", fft3d_last_error());
      } else if (process_[i] == 2) {
        env->BitBlt(dst->GetWritePtr(id), dst->GetPitch(id), src->GetReadPtr(id), src->GetPitch(id),
                    src->GetRowSize(id), src->GetHeight(id));
      }
    }
    return dst;
  }

  // Kalman (bt = 0) carries state from frame to frame: serialized; the other
  // modes are pure functions of their window
  int __stdcall SetCacheHints(int hints, int) override {
    return hints == CACHE_GET_MTMODE ? (p_.bt == 0 ? MT_SERIALIZED : MT_NICE_FILTER) : 0;
  }

 private:
  // noise pattern from frame pframe, once (src/fft3d_engine.h:485-500)
  void set_pattern(IScriptEnvironment* env) {
    std::lock_guard<std::mutex> lk(pattern_lock_);
    if (pattern_done_) return;
    PVideoFrame pf = child->GetFrame(std::min(std::max(p_.pframe, 0), vi.num_frames - 1), env);
    for (int i = 0; i < nplanes_; i++)
      if (plane_[i] && fft3d_plane_set_pattern_frame(plane_[i], pf->GetReadPtr(ids_[i]), pf->GetPitch(ids_[i])))
        env->ThrowError("neo_fft3d: %s", fft3d_last_error());
    pattern_done_ = true;
  }

  void release() {
    for (auto*& h : plane_)
      if (h) {
        fft3d_plane_destroy(h);
        h = nullptr;
      }
  }

  fft3d_params p_;
  int process_[4] = {2, 2, 2, 2};
  int ids_[4] = {0, 0, 0, 0};
  fft3d_plane* plane_[4] = {nullptr, nullptr, nullptr, nullptr};
  bool yuv_ = false, has_v8_ = false;
  int nplanes_ = 0, engines_ = 0;
  std::mutex pattern_lock_;
  bool pattern_done_ = false;
};

// Argument slots of kParams, in order (clip is slot 0).
enum {
  A_CLIP, A_SIGMA, A_BETA, A_BW, A_BH, A_BT, A_OW, A_OH, A_KRATIO, A_SHARPEN, A_SCUTOFF, A_SVR, A_SMIN, A_SMAX,
  A_MEASURE, A_INTERLACED, A_WINTYPE, A_PFRAME, A_PX, A_PY, A_PSHOW, A_PCUTOFF, A_PFACTOR, A_SIGMA2, A_SIGMA3,
  A_SIGMA4, A_DEGRID, A_DEHALO, A_HR, A_HT, A_Y, A_U, A_V, A_L, A_T, A_R, A_B, A_OPT, A_NCPU, A_MT
};

// The reference's AviSynth+ parameter string: its parameter list
// (src/fft3d.hpp:29-72) less the VapourSynth-only `planes`, optional
// parameters as [name]type (include/dualsynth/ds_filter.hpp:44-70).
const char* kParams =
    "c[sigma]f[beta]f[bw]i[bh]i[bt]i[ow]i[oh]i[kratio]f[sharpen]f[scutoff]f[svr]f[smin]f[smax]f[measure]b"
    "[interlaced]b[wintype]i[pframe]i[px]i[py]i[pshow]b[pcutoff]f[pfactor]f[sigma2]f[sigma3]f[sigma4]f[degrid]f"
    "[dehalo]f[hr]f[ht]f[y]i[u]i[v]i[l]i[t]i[r]i[b]i[opt]i[ncpu]i[mt]b";

AVSValue __cdecl create(AVSValue args, void*, IScriptEnvironment* env) {
  auto geti = [&](int k, int& v) { v = args[k].AsInt(v); };
  auto getf = [&](int k, float& v) { v = (float)args[k].AsFloat(v); };
  auto getb = [&](int k, int& v) { v = args[k].AsBool(v != 0) ? 1 : 0; };
  PClip clip = args[A_CLIP].AsClip();
  const VideoInfo& vi = clip->GetVideoInfo();
  // packed formats (YUY2, RGB24/32/48/64) have no planes to address; the
  // reference rejects them first, with this message
  // (include/dualsynth/ds_format.hpp:44-47)
  if (!vi.IsPlanar()) env->ThrowError("neo_fft3d: neo-dfttest only supports planar formats.");
  // parameters and defaults, src/fft3d.hpp:77-139
  fft3d_params p;
  fft3d_params_default(&p);
  getf(A_SIGMA, p.sigma);
  p.sigma2 = p.sigma3 = p.sigma4 = p.sigma;
  getf(A_BETA, p.beta);
  geti(A_BW, p.bw);
  geti(A_BH, p.bh);
  geti(A_BT, p.bt);
  geti(A_OW, p.ow);
  geti(A_OH, p.oh);
  getf(A_KRATIO, p.kratio);
  getf(A_SHARPEN, p.sharpen);
  getf(A_SCUTOFF, p.scutoff);
  getf(A_SVR, p.svr);
  getf(A_SMIN, p.smin);
  getf(A_SMAX, p.smax);
  getb(A_MEASURE, p.measure);
  getb(A_INTERLACED, p.interlaced);
  geti(A_WINTYPE, p.wintype);
  geti(A_PFRAME, p.pframe);
  geti(A_PX, p.px);
  geti(A_PY, p.py);
  getb(A_PSHOW, p.pshow);
  getf(A_PCUTOFF, p.pcutoff);
  getf(A_PFACTOR, p.pfactor);
  getf(A_SIGMA2, p.sigma2);
  getf(A_SIGMA3, p.sigma3);
  getf(A_SIGMA4, p.sigma4);
  getf(A_DEGRID, p.degrid);
  getf(A_DEHALO, p.dehalo);
  getf(A_HR, p.hr);
  getf(A_HT, p.ht);
  geti(A_L, p.l);
  geti(A_T, p.t);
  geti(A_R, p.r);
  geti(A_B, p.b);
  p.l = std::max(p.l, 0);
  p.t = std::max(p.t, 0);
  p.r = std::max(p.r, 0);
  p.b = std::max(p.b, 0);
  geti(A_OPT, p.opt);
  geti(A_NCPU, p.ncpu);
  getb(A_MT, p.mt);
  if (p.l + p.r >= vi.width) env->ThrowError("neo_fft3d: Width cannot be cropped to zero or below");
  if (p.t + p.b >= vi.height) env->ThrowError("neo_fft3d: Height cannot be cropped to zero or below");
  // y/u/v default 3 (filter); the alpha plane is copied (src/fft3d.hpp:149-168)
  int process[4] = {3, 3, 3, 2};
  geti(A_Y, process[0]);
  geti(A_U, process[1]);
  geti(A_V, process[2]);
  try {
    return new NeoFFT3D(clip, p, process, env);
  } catch (const Fail& f) {
    env->ThrowError("neo_fft3d: %s", f.msg.c_str());
  }
  return AVSValue();
}

}  // namespace

extern "C" __attribute__((visibility("default"))) const char* __stdcall AvisynthPluginInit3(
    IScriptEnvironment* env, const AVS_Linkage* const vectors) {
  AVS_linkage = vectors;
  env->AddFunction("neo_fft3d", kParams, create, nullptr);
  return "Neo FFT3D Filter (B200 sm_100a)";
}
