// Headless AviSynth+ host: a minimal core that loads AviSynth+ plugins
// (AvisynthPluginInit3), invokes their functions and serves frames from host
// memory, so that the neo_fft3d AviSynth+ plugin can be driven and compared
// with the reference's without an AviSynth+ installation. It implements the
// core side of the AviSynth+ C++ interface (compiled with BUILDING_AVSCORE):
// VideoInfo queries, frame buffers and frames, the PClip / PVideoFrame
// smart pointers, AVSValue, the linkage table plugins call through, and the
// IScriptEnvironment calls filters make (AddFunction, ThrowError, frame
// allocation); the other environment calls throw "not implemented".
// Single-threaded: one GetFrame at a time. Test support, C API below.
#include <dlfcn.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "avisynth.h"

// ---------------------------------------------------------------- VideoInfo

namespace {
int sample_bits(int pixel_type) {
  switch ((pixel_type & VideoInfo::CS_Sample_Bits_Mask) >> VideoInfo::CS_Shift_Sample_Bits) {
    case 0: return 8;
    case 1: return 16;
    case 2: return 32;
    case 5: return 10;
    case 6: return 12;
    case 7: return 14;
  }
  return 8;
}
}  // namespace

bool VideoInfo::HasVideo() const { return width != 0; }
bool VideoInfo::HasAudio() const { return false; }
bool VideoInfo::IsPlanar() const { return (pixel_type & CS_PLANAR) != 0; }
bool VideoInfo::IsYUV() const { return (pixel_type & CS_YUV) != 0; }
bool VideoInfo::IsYUVA() const { return (pixel_type & CS_YUVA) != 0; }
bool VideoInfo::IsRGB() const { return (pixel_type & CS_BGR) != 0; }
bool VideoInfo::IsY() const { return IsPlanar() && (pixel_type & CS_INTERLEAVED) && IsYUV(); }
bool VideoInfo::IsY8() const { return IsY() && sample_bits(pixel_type) == 8; }
bool VideoInfo::IsYUY2() const { return (pixel_type & CS_YUY2) == CS_YUY2; }
bool VideoInfo::IsRGB24() const { return (pixel_type & CS_BGR24) == CS_BGR24 && !IsPlanar(); }
bool VideoInfo::IsRGB32() const { return (pixel_type & CS_BGR32) == CS_BGR32 && !IsPlanar(); }
bool VideoInfo::IsPlanarRGB() const { return IsPlanar() && IsRGB() && (pixel_type & CS_RGB_TYPE); }
bool VideoInfo::IsPlanarRGBA() const { return IsPlanar() && IsRGB() && (pixel_type & CS_RGBA_TYPE); }
bool VideoInfo::IsFieldBased() const { return (image_type & IT_FIELDBASED) != 0; }
bool VideoInfo::IsColorSpace(int c) const {
  return IsPlanar() ? ((pixel_type & CS_PLANAR_MASK) == (c & CS_PLANAR_FILTER)) : ((pixel_type & c) == c);
}
int VideoInfo::BitsPerComponent() const { return sample_bits(pixel_type); }
int VideoInfo::ComponentSize() const {
  const int b = sample_bits(pixel_type);
  return b == 8 ? 1 : (b == 32 ? 4 : 2);
}
int VideoInfo::NumComponents() const {
  if (IsY()) return 1;
  if (IsYUVA() || IsPlanarRGBA()) return 4;
  return 3;
}
// subsampled planes: U and V of planar YUV(A) with chroma
int VideoInfo::GetPlaneWidthSubsampling(int plane) const {
  if (!(plane & (PLANAR_U | PLANAR_V)) || !(IsYUV() || IsYUVA()) || IsY()) return 0;
  return ((pixel_type >> CS_Shift_Sub_Width) + 1) & 3;
}
int VideoInfo::GetPlaneHeightSubsampling(int plane) const {
  if (!(plane & (PLANAR_U | PLANAR_V)) || !(IsYUV() || IsYUVA()) || IsY()) return 0;
  return ((pixel_type >> CS_Shift_Sub_Height) + 1) & 3;
}
namespace {
bool has_chroma(const VideoInfo& vi) { return (vi.IsYUV() || vi.IsYUVA()) && !vi.IsY() && vi.IsPlanar(); }
}  // namespace
bool VideoInfo::Is444() const { return has_chroma(*this) && GetPlaneWidthSubsampling(PLANAR_U) == 0 && GetPlaneHeightSubsampling(PLANAR_U) == 0; }
bool VideoInfo::Is422() const { return has_chroma(*this) && GetPlaneWidthSubsampling(PLANAR_U) == 1 && GetPlaneHeightSubsampling(PLANAR_U) == 0; }
bool VideoInfo::Is420() const { return has_chroma(*this) && GetPlaneWidthSubsampling(PLANAR_U) == 1 && GetPlaneHeightSubsampling(PLANAR_U) == 1; }
int VideoInfo::RowSize(int plane) const {
  const int w = (plane & (PLANAR_U | PLANAR_V)) ? (width >> GetPlaneWidthSubsampling(plane)) : width;
  return w * ComponentSize();
}
int VideoInfo::BytesFromPixels(int pixels) const { return pixels * ComponentSize() * (IsPlanar() ? 1 : NumComponents()); }

// ---------------------------------------------------------------- frames

VideoFrameBuffer::VideoFrameBuffer(int size, int margin, Device*)
    : data(nullptr), data_size(size), sequence_number(0), refcount(0), device(nullptr) {
  (void)margin;
  data = static_cast<BYTE*>(std::aligned_alloc(64, ((size_t)size + 63) / 64 * 64));
}
VideoFrameBuffer::VideoFrameBuffer() : data(nullptr), data_size(0), sequence_number(0), refcount(0), device(nullptr) {}
void VideoFrameBuffer::DESTRUCTOR() { std::free(data); }
const BYTE* VideoFrameBuffer::GetReadPtr() const { return data; }
BYTE* VideoFrameBuffer::GetWritePtr() {
  ++sequence_number;
  return data;
}
int VideoFrameBuffer::GetDataSize() const { return data_size; }
int VideoFrameBuffer::GetSequenceNumber() const { return (int)sequence_number; }
int VideoFrameBuffer::GetRefcount() const { return (int)refcount; }

void* VideoFrame::operator new(size_t size) { return ::operator new(size); }

VideoFrame::VideoFrame(VideoFrameBuffer* _vfb, AVSMap* avsmap, int _offset, int _pitch, int _row_size, int _height,
                       int _offsetU, int _offsetV, int _pitchUV, int _row_sizeUV, int _heightUV, int _offsetA,
                       int _pixel_type)
    : refcount(0), vfb(_vfb), offset(_offset), pitch(_pitch), row_size(_row_size), height(_height),
      offsetU(_offsetU), offsetV(_offsetV), pitchUV(_pitchUV), row_sizeUV(_row_sizeUV), heightUV(_heightUV),
      offsetA(_offsetA), pitchA(_offsetA ? _pitch : 0), row_sizeA(_offsetA ? _row_size : 0), properties(avsmap),
      pixel_type(_pixel_type) {
  ++vfb->refcount;
}

void VideoFrame::AddRef() { ++refcount; }
void VideoFrame::Release() {
  if (--refcount == 0) {
    DESTRUCTOR();
    ::operator delete(this);
  }
}
void VideoFrame::DESTRUCTOR() {
  if (vfb && --vfb->refcount == 0) {
    vfb->DESTRUCTOR();
    ::operator delete(vfb);
  }
  vfb = nullptr;
}

namespace {
// plane -> 0 (first: Y / G), 1 (second: U / B), 2 (third: V / R), 3 (alpha)
int plane_slot(int plane) {
  if (plane & (PLANAR_U | PLANAR_B)) return 1;
  if (plane & (PLANAR_V | PLANAR_R)) return 2;
  if (plane & PLANAR_A) return 3;
  return 0;
}
// the planes of a clip in the order its filters number them: Y U V A, or
// R G B A (src/fft3d.hpp:182-184 of the reference plugin)
int plane_ids(const VideoInfo& vi, int ids[4]) {
  const bool rgb = vi.IsRGB() || vi.IsPlanarRGBA();
  const int yuv_ids[4] = {PLANAR_Y, PLANAR_U, PLANAR_V, PLANAR_A};
  const int rgb_ids[4] = {PLANAR_R, PLANAR_G, PLANAR_B, PLANAR_A};
  for (int i = 0; i < 4; i++) ids[i] = rgb ? rgb_ids[i] : yuv_ids[i];
  return vi.NumComponents();
}
}  // namespace

int VideoFrame::GetPitch(int plane) const {
  const int s = plane_slot(plane);
  return s == 0 ? pitch : (s == 3 ? pitchA : pitchUV);
}
int VideoFrame::GetRowSize(int plane) const {
  const int s = plane_slot(plane);
  return s == 0 ? row_size : (s == 3 ? row_sizeA : row_sizeUV);
}
int VideoFrame::GetHeight(int plane) const {
  const int s = plane_slot(plane);
  return (s == 1 || s == 2) ? heightUV : height;
}
int VideoFrame::GetOffset(int plane) const {
  const int s = plane_slot(plane);
  return s == 0 ? offset : (s == 1 ? offsetU : (s == 2 ? offsetV : offsetA));
}
VideoFrameBuffer* VideoFrame::GetFrameBuffer() const { return vfb; }
const BYTE* VideoFrame::GetReadPtr(int plane) const { return vfb->GetReadPtr() + GetOffset(plane); }
bool VideoFrame::IsWritable() const { return refcount == 1 && vfb->refcount == 1; }
BYTE* VideoFrame::GetWritePtr(int plane) const { return vfb->GetWritePtr() + GetOffset(plane); }
int VideoFrame::GetPixelType() const { return pixel_type; }

void PVideoFrame::Init(VideoFrame* x) {
  p = x;
  if (p) p->AddRef();
}
void PVideoFrame::Set(VideoFrame* x) {
  if (x) x->AddRef();
  if (p) p->Release();
  p = x;
}
void PVideoFrame::CONSTRUCTOR0() { p = nullptr; }
void PVideoFrame::CONSTRUCTOR1(const PVideoFrame& x) { Init(x.p); }
void PVideoFrame::CONSTRUCTOR2(VideoFrame* x) { Init(x); }
void PVideoFrame::OPERATOR_ASSIGN0(VideoFrame* x) { Set(x); }
void PVideoFrame::OPERATOR_ASSIGN1(const PVideoFrame& x) { Set(x.p); }
void PVideoFrame::DESTRUCTOR() {
  if (p) p->Release();
  p = nullptr;
}
PVideoFrame::PVideoFrame() { CONSTRUCTOR0(); }
PVideoFrame::PVideoFrame(const PVideoFrame& x) { CONSTRUCTOR1(x); }
PVideoFrame::PVideoFrame(VideoFrame* x) { CONSTRUCTOR2(x); }
void PVideoFrame::operator=(VideoFrame* x) { OPERATOR_ASSIGN0(x); }
void PVideoFrame::operator=(const PVideoFrame& x) { OPERATOR_ASSIGN1(x); }
PVideoFrame::~PVideoFrame() { DESTRUCTOR(); }

// ---------------------------------------------------------------- clips and values

void IClip::AddRef() { ++refcnt; }
void IClip::Release() {
  if (--refcnt == 0) delete this;
}

void PClip::Init(IClip* x) {
  p = x;
  if (p) p->AddRef();
}
void PClip::Set(IClip* x) {
  if (x) x->AddRef();
  if (p) p->Release();
  p = x;
}
IClip* PClip::GetPointerWithAddRef() const {
  if (p) p->AddRef();
  return p;
}
void PClip::CONSTRUCTOR0() { p = nullptr; }
void PClip::CONSTRUCTOR1(const PClip& x) { Init(x.p); }
void PClip::CONSTRUCTOR2(IClip* x) { Init(x); }
void PClip::OPERATOR_ASSIGN0(IClip* x) { Set(x); }
void PClip::OPERATOR_ASSIGN1(const PClip& x) { Set(x.p); }
void PClip::DESTRUCTOR() {
  if (p) p->Release();
  p = nullptr;
}
PClip::PClip() { CONSTRUCTOR0(); }
PClip::PClip(const PClip& x) { CONSTRUCTOR1(x); }
PClip::PClip(IClip* x) { CONSTRUCTOR2(x); }
void PClip::operator=(IClip* x) { OPERATOR_ASSIGN0(x); }
void PClip::operator=(const PClip& x) { OPERATOR_ASSIGN1(x); }
PClip::~PClip() { DESTRUCTOR(); }

// Arrays are not owned by the values that point at them (the host keeps the
// argument arrays it passes to filters alive for the call).
void AVSValue::Assign(const AVSValue* src, bool init) {
  if (src->type == 'c' && src->clip) src->clip->AddRef();
  if (!init && type == 'c' && clip) clip->Release();
  type = src->type;
  array_size = src->array_size;
  longlong = src->longlong;
}
void AVSValue::CONSTRUCTOR0() {
  type = 'v';
  array_size = 0;
  longlong = 0;
}
void AVSValue::CONSTRUCTOR1(IClip* c) {
  type = 'c';
  array_size = 0;
  longlong = 0;
  clip = c;
  if (c) c->AddRef();
}
void AVSValue::CONSTRUCTOR2(const PClip& c) { CONSTRUCTOR1(c.p); }
void AVSValue::CONSTRUCTOR3(bool b) {
  CONSTRUCTOR0();
  type = 'b';
  boolean = b;
}
void AVSValue::CONSTRUCTOR4(int i) {
  CONSTRUCTOR0();
  type = 'i';
  integer = i;
}
void AVSValue::CONSTRUCTOR5(float f) {
  CONSTRUCTOR0();
  type = 'f';
  floating_pt = f;
}
void AVSValue::CONSTRUCTOR6(double f) {
  CONSTRUCTOR0();
  type = 'f';
  floating_pt = (float)f;
}
void AVSValue::CONSTRUCTOR7(const char* s) {
  CONSTRUCTOR0();
  type = 's';
  string = s;
}
void AVSValue::CONSTRUCTOR8(const AVSValue* a, int size) {
  CONSTRUCTOR0();
  type = 'a';
  array = a;
  array_size = (short)size;
}
void AVSValue::CONSTRUCTOR9(const AVSValue& v) { Assign(&v, true); }
void AVSValue::CONSTRUCTOR12(int64_t l) {
  CONSTRUCTOR0();
  type = 'l';
  longlong = l;
}
AVSValue::AVSValue() { CONSTRUCTOR0(); }
AVSValue::AVSValue(IClip* c) { CONSTRUCTOR1(c); }
AVSValue::AVSValue(const PClip& c) { CONSTRUCTOR2(c); }
AVSValue::AVSValue(bool b) { CONSTRUCTOR3(b); }
AVSValue::AVSValue(int i) { CONSTRUCTOR4(i); }
AVSValue::AVSValue(float f) { CONSTRUCTOR5(f); }
AVSValue::AVSValue(double f) { CONSTRUCTOR6(f); }
AVSValue::AVSValue(const char* s) { CONSTRUCTOR7(s); }
AVSValue::AVSValue(const AVSValue* a, int size) { CONSTRUCTOR8(a, size); }
AVSValue::AVSValue(const AVSValue& a, int size) { CONSTRUCTOR8(&a, size); }
AVSValue::AVSValue(const AVSValue& v) { CONSTRUCTOR9(v); }
AVSValue::AVSValue(int64_t l) { CONSTRUCTOR12(l); }
AVSValue::~AVSValue() { DESTRUCTOR(); }
AVSValue& AVSValue::operator=(const AVSValue& v) { return OPERATOR_ASSIGN(v); }
const AVSValue& AVSValue::operator[](int index) const { return OPERATOR_INDEX(index); }
void AVSValue::DESTRUCTOR() {
  if (type == 'c' && clip) clip->Release();
  type = 'v';
}
AVSValue& AVSValue::OPERATOR_ASSIGN(const AVSValue& v) {
  if (&v != this) Assign(&v, false);
  return *this;
}
const AVSValue& AVSValue::OPERATOR_INDEX(int index) const {
  return (type == 'a' && index >= 0 && index < array_size) ? array[index] : *this;
}
bool AVSValue::Defined() const { return type != 'v'; }
bool AVSValue::IsClip() const { return type == 'c'; }
bool AVSValue::IsBool() const { return type == 'b'; }
bool AVSValue::IsInt() const { return type == 'i' || type == 'l'; }
bool AVSValue::IsLongStrict() const { return type == 'l'; }
bool AVSValue::IsFloat() const { return type == 'f' || type == 'd' || type == 'i' || type == 'l'; }
bool AVSValue::IsFloatfStrict() const { return type == 'f'; }
bool AVSValue::IsString() const { return type == 's'; }
bool AVSValue::IsArray() const { return type == 'a'; }
PClip AVSValue::AsClip() const { return IsClip() ? PClip(clip) : PClip(); }
bool AVSValue::AsBool1() const { return boolean; }
int AVSValue::AsInt1() const { return type == 'l' ? (int)longlong : integer; }
int64_t AVSValue::AsLong1() const { return type == 'l' ? longlong : integer; }
const char* AVSValue::AsString1() const { return IsString() ? string : nullptr; }
double AVSValue::AsFloat1() const {
  return type == 'i' ? (double)integer : (type == 'l' ? (double)longlong : (double)floating_pt);
}
bool AVSValue::AsBool2(bool def) const { return IsBool() ? boolean : def; }
int AVSValue::AsInt2(int def) const { return IsInt() ? AsInt1() : def; }
int64_t AVSValue::AsLong2(int64_t def) const { return IsInt() ? AsLong1() : def; }
double AVSValue::AsDblDef(double def) const { return IsFloat() ? AsFloat1() : def; }
double AVSValue::AsFloat2(float def) const { return IsFloat() ? AsFloat1() : (double)def; }
const char* AVSValue::AsString2(const char* def) const { return IsString() ? string : def; }
int AVSValue::ArraySize() const { return IsArray() ? array_size : 1; }

// ---------------------------------------------------------------- linkage

namespace {
AVS_Linkage make_linkage() {
  AVS_Linkage L;
  std::memset(&L, 0, sizeof(L));
  L.Size = sizeof(L);
  L.HasVideo = &VideoInfo::HasVideo;
  L.HasAudio = &VideoInfo::HasAudio;
  L.IsRGB = &VideoInfo::IsRGB;
  L.IsRGB24 = &VideoInfo::IsRGB24;
  L.IsRGB32 = &VideoInfo::IsRGB32;
  L.IsYUV = &VideoInfo::IsYUV;
  L.IsYUY2 = &VideoInfo::IsYUY2;
  L.IsY8 = &VideoInfo::IsY8;
  L.IsColorSpace = &VideoInfo::IsColorSpace;
  L.IsPlanar = &VideoInfo::IsPlanar;
  L.IsFieldBased = &VideoInfo::IsFieldBased;
  L.BytesFromPixels = &VideoInfo::BytesFromPixels;
  L.RowSize = &VideoInfo::RowSize;
  L.GetPlaneWidthSubsampling = &VideoInfo::GetPlaneWidthSubsampling;
  L.GetPlaneHeightSubsampling = &VideoInfo::GetPlaneHeightSubsampling;
  L.NumComponents = &VideoInfo::NumComponents;
  L.ComponentSize = &VideoInfo::ComponentSize;
  L.BitsPerComponent = &VideoInfo::BitsPerComponent;
  L.Is444 = &VideoInfo::Is444;
  L.Is422 = &VideoInfo::Is422;
  L.Is420 = &VideoInfo::Is420;
  L.IsY = &VideoInfo::IsY;
  L.IsYUVA = &VideoInfo::IsYUVA;
  L.IsPlanarRGB = &VideoInfo::IsPlanarRGB;
  L.IsPlanarRGBA = &VideoInfo::IsPlanarRGBA;
  L.VFBGetReadPtr = &VideoFrameBuffer::GetReadPtr;
  L.VFBGetWritePtr = &VideoFrameBuffer::GetWritePtr;
  L.GetDataSize = &VideoFrameBuffer::GetDataSize;
  L.GetSequenceNumber = &VideoFrameBuffer::GetSequenceNumber;
  L.GetRefcount = &VideoFrameBuffer::GetRefcount;
  L.GetPitch = &VideoFrame::GetPitch;
  L.GetRowSize = &VideoFrame::GetRowSize;
  L.GetHeight = &VideoFrame::GetHeight;
  L.GetFrameBuffer = &VideoFrame::GetFrameBuffer;
  L.GetOffset = &VideoFrame::GetOffset;
  L.VFGetReadPtr = &VideoFrame::GetReadPtr;
  L.IsWritable = &VideoFrame::IsWritable;
  L.VFGetWritePtr = &VideoFrame::GetWritePtr;
  L.VideoFrame_DESTRUCTOR = &VideoFrame::DESTRUCTOR;
  L.VideoFrame_GetPixelType = &VideoFrame::GetPixelType;
  L.VideoFrameBuffer_DESTRUCTOR = &VideoFrameBuffer::DESTRUCTOR;
  L.PClip_CONSTRUCTOR0 = &PClip::CONSTRUCTOR0;
  L.PClip_CONSTRUCTOR1 = &PClip::CONSTRUCTOR1;
  L.PClip_CONSTRUCTOR2 = &PClip::CONSTRUCTOR2;
  L.PClip_OPERATOR_ASSIGN0 = &PClip::OPERATOR_ASSIGN0;
  L.PClip_OPERATOR_ASSIGN1 = &PClip::OPERATOR_ASSIGN1;
  L.PClip_DESTRUCTOR = &PClip::DESTRUCTOR;
  L.PVideoFrame_CONSTRUCTOR0 = &PVideoFrame::CONSTRUCTOR0;
  L.PVideoFrame_CONSTRUCTOR1 = &PVideoFrame::CONSTRUCTOR1;
  L.PVideoFrame_CONSTRUCTOR2 = &PVideoFrame::CONSTRUCTOR2;
  L.PVideoFrame_OPERATOR_ASSIGN0 = &PVideoFrame::OPERATOR_ASSIGN0;
  L.PVideoFrame_OPERATOR_ASSIGN1 = &PVideoFrame::OPERATOR_ASSIGN1;
  L.PVideoFrame_DESTRUCTOR = &PVideoFrame::DESTRUCTOR;
  L.AVSValue_CONSTRUCTOR0 = &AVSValue::CONSTRUCTOR0;
  L.AVSValue_CONSTRUCTOR1 = &AVSValue::CONSTRUCTOR1;
  L.AVSValue_CONSTRUCTOR2 = &AVSValue::CONSTRUCTOR2;
  L.AVSValue_CONSTRUCTOR3 = &AVSValue::CONSTRUCTOR3;
  L.AVSValue_CONSTRUCTOR4 = &AVSValue::CONSTRUCTOR4;
  L.AVSValue_CONSTRUCTOR5 = &AVSValue::CONSTRUCTOR5;
  L.AVSValue_CONSTRUCTOR6 = &AVSValue::CONSTRUCTOR6;
  L.AVSValue_CONSTRUCTOR7 = &AVSValue::CONSTRUCTOR7;
  L.AVSValue_CONSTRUCTOR8 = &AVSValue::CONSTRUCTOR8;
  L.AVSValue_CONSTRUCTOR9 = &AVSValue::CONSTRUCTOR9;
  L.AVSValue_CONSTRUCTOR12 = &AVSValue::CONSTRUCTOR12;
  L.AVSValue_DESTRUCTOR = &AVSValue::DESTRUCTOR;
  L.AVSValue_OPERATOR_ASSIGN = &AVSValue::OPERATOR_ASSIGN;
  L.AVSValue_OPERATOR_INDEX = &AVSValue::OPERATOR_INDEX;
  L.Defined = &AVSValue::Defined;
  L.IsClip = &AVSValue::IsClip;
  L.IsBool = &AVSValue::IsBool;
  L.IsInt = &AVSValue::IsInt;
  L.IsFloat = &AVSValue::IsFloat;
  L.IsString = &AVSValue::IsString;
  L.IsArray = &AVSValue::IsArray;
  L.AsClip = &AVSValue::AsClip;
  L.AsBool1 = &AVSValue::AsBool1;
  L.AsInt1 = &AVSValue::AsInt1;
  L.AsString1 = &AVSValue::AsString1;
  L.AsFloat1 = &AVSValue::AsFloat1;
  L.AsBool2 = &AVSValue::AsBool2;
  L.AsInt2 = &AVSValue::AsInt2;
  L.AsDblDef = &AVSValue::AsDblDef;
  L.AsFloat2 = &AVSValue::AsFloat2;
  L.AsString2 = &AVSValue::AsString2;
  L.ArraySize = &AVSValue::ArraySize;
  L.IsLongStrict = &AVSValue::IsLongStrict;
  L.IsFloatfStrict = &AVSValue::IsFloatfStrict;
  L.AsLong1 = &AVSValue::AsLong1;
  L.AsLong2 = &AVSValue::AsLong2;
  return L;
}
const AVS_Linkage g_linkage = make_linkage();

// AvisynthError keeps the pointer it is given: the message lives in a
// per-thread buffer until the next error.
thread_local std::string g_throw;
[[noreturn]] void unimplemented(const char* what) {
  g_throw = std::string("avshost: ") + what + " is not implemented by this host";
  throw AvisynthError(g_throw.c_str());
}

// ---------------------------------------------------------------- environment

struct Function {
  std::string name, params;
  IScriptEnvironment::ApplyFunc apply;
  void* user_data;
};

}  // namespace

class ScriptEnvironment : public IScriptEnvironment {
 public:
  std::vector<Function> functions;
  std::vector<std::string*> strings;
  std::string last_error;

  ~ScriptEnvironment() override {
    for (auto* s : strings) delete s;
  }
  int __stdcall GetCPUFlags() override { return 0; }
  int64_t __stdcall GetCPUFlagsEx() override { return 0; }
  char* __stdcall SaveString(const char* s, int length) override {
    auto* str = new std::string(s, length < 0 ? std::strlen(s) : (size_t)length);
    strings.push_back(str);
    return &(*str)[0];
  }
  char* __stdcall VSprintf(const char* fmt, va_list val) override {
    char buf[4096];
    std::vsnprintf(buf, sizeof(buf), fmt, val);
    return SaveString(buf, -1);
  }
  char* Sprintf(const char* fmt, ...) override {
    va_list ap;
    va_start(ap, fmt);
    char* r = VSprintf(fmt, ap);
    va_end(ap);
    return r;
  }
  void ThrowError(const char* fmt, ...) override {
    va_list ap;
    va_start(ap, fmt);
    char* r = VSprintf(fmt, ap);
    va_end(ap);
    throw AvisynthError(r);
  }
  void __stdcall AddFunction(const char* name, const char* params, ApplyFunc apply, void* user_data) override {
    functions.push_back(Function{name, params, apply, user_data});
  }
  bool __stdcall FunctionExists(const char*) override { return false; }
  void __stdcall CheckVersion(int version) override {
    if (version > AVISYNTH_INTERFACE_VERSION) ThrowError("avshost: interface version %d is not available", version);
  }
  PVideoFrame __stdcall NewVideoFrame(const VideoInfo& vi, int align) override { return NewFrame(vi); }
  PVideoFrame __stdcall NewVideoFrameP(const VideoInfo& vi, const PVideoFrame*, int align) override { return NewFrame(vi); }
  void __stdcall copyFrameProps(const PVideoFrame&, PVideoFrame&) override {}
  bool __stdcall MakeWritable(PVideoFrame* pvf) override {
    if ((*pvf)->IsWritable()) return false;
    unimplemented("MakeWritable of a shared frame");
  }
  void __stdcall BitBlt(BYTE* dstp, int dst_pitch, const BYTE* srcp, int src_pitch, int row_size, int height) override {
    for (int y = 0; y < height; y++) std::memcpy(dstp + (size_t)y * dst_pitch, srcp + (size_t)y * src_pitch, row_size);
  }
  void* __stdcall ManageCache(int, void*) override { return nullptr; }
  int __stdcall SetMemoryMax(int) override { return 0; }
  void __stdcall AtExit(ShutdownFunc, void*) override {}
  void __stdcall DeleteScriptEnvironment() override {}
  const AVS_Linkage* __stdcall GetAVSLinkage() override { return &g_linkage; }
  size_t __stdcall GetEnvProperty(AvsEnvProperty) override { return 0; }
  bool __stdcall AcquireGlobalLock(const char*) override { return true; }
  void __stdcall ReleaseGlobalLock(const char*) override {}
  AVSValue __stdcall GetVarDef(const char*, const AVSValue& def) override { return def; }
  bool __stdcall GetVarTry(const char*, AVSValue*) const override { return false; }
  bool __stdcall GetVarBool(const char*, bool def) const override { return def; }
  int __stdcall GetVarInt(const char*, int def) const override { return def; }
  double __stdcall GetVarDouble(const char*, double def) const override { return def; }
  const char* __stdcall GetVarString(const char*, const char* def) const override { return def; }
  int64_t __stdcall GetVarLong(const char*, int64_t def) const override { return def; }
  AVSValue __stdcall GetVar(const char* name) override { unimplemented("GetVar"); }
  bool __stdcall SetVar(const char* name, const AVSValue& val) override { unimplemented("SetVar"); }
  bool __stdcall SetGlobalVar(const char* name, const AVSValue& val) override { unimplemented("SetGlobalVar"); }
  void __stdcall PopContext() override { unimplemented("PopContext"); }
  PVideoFrame __stdcall Subframe(PVideoFrame src, int rel_offset, int new_pitch, int new_row_size, int new_height) override { unimplemented("Subframe"); }
  int __stdcall SetWorkingDir(const char * newdir) override { unimplemented("SetWorkingDir"); }
  bool __stdcall PlanarChromaAlignment(PlanarChromaAlignmentMode key) override { unimplemented("PlanarChromaAlignment"); }
  PVideoFrame __stdcall SubframePlanar(PVideoFrame src, int rel_offset, int new_pitch, int new_row_size, int new_height, int rel_offsetU, int rel_offsetV, int new_pitchUV) override { unimplemented("SubframePlanar"); }
  void __stdcall ApplyMessage(PVideoFrame* frame, const VideoInfo& vi, const char* message, int size, int textcolor, int halocolor, int bgcolor) override { unimplemented("ApplyMessage"); }
  PVideoFrame __stdcall SubframePlanarA(PVideoFrame src, int rel_offset, int new_pitch, int new_row_size, int new_height, int rel_offsetU, int rel_offsetV, int new_pitchUV, int rel_offsetA) override { unimplemented("SubframePlanarA"); }
  const AVSMap* __stdcall getFramePropsRO(const PVideoFrame& frame) override { unimplemented("getFramePropsRO"); }
  AVSMap* __stdcall getFramePropsRW(PVideoFrame& frame) override { unimplemented("getFramePropsRW"); }
  int __stdcall propNumKeys(const AVSMap* map) override { unimplemented("propNumKeys"); }
  const char* __stdcall propGetKey(const AVSMap* map, int index) override { unimplemented("propGetKey"); }
  int __stdcall propNumElements(const AVSMap* map, const char* key) override { unimplemented("propNumElements"); }
  char __stdcall propGetType(const AVSMap* map, const char* key) override { unimplemented("propGetType"); }
  int64_t __stdcall propGetInt(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetInt"); }
  double __stdcall propGetFloat(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetFloat"); }
  const char* __stdcall propGetData(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetData"); }
  int __stdcall propGetDataSize(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetDataSize"); }
  PClip __stdcall propGetClip(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetClip"); }
  const PVideoFrame __stdcall propGetFrame(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetFrame"); }
  int __stdcall propDeleteKey(AVSMap* map, const char* key) override { unimplemented("propDeleteKey"); }
  int __stdcall propSetInt(AVSMap* map, const char* key, int64_t i, int append) override { unimplemented("propSetInt"); }
  int __stdcall propSetFloat(AVSMap* map, const char* key, double d, int append) override { unimplemented("propSetFloat"); }
  int __stdcall propSetData(AVSMap* map, const char* key, const char* d, int length, int append) override { unimplemented("propSetData"); }
  int __stdcall propSetClip(AVSMap* map, const char* key, PClip& clip, int append) override { unimplemented("propSetClip"); }
  int __stdcall propSetFrame(AVSMap* map, const char* key, const PVideoFrame& frame, int append) override { unimplemented("propSetFrame"); }
  const int64_t* __stdcall propGetIntArray(const AVSMap* map, const char* key, int* error) override { unimplemented("propGetIntArray"); }
  const double* __stdcall propGetFloatArray(const AVSMap* map, const char* key, int* error) override { unimplemented("propGetFloatArray"); }
  int __stdcall propSetIntArray(AVSMap* map, const char* key, const int64_t* i, int size) override { unimplemented("propSetIntArray"); }
  int __stdcall propSetFloatArray(AVSMap* map, const char* key, const double* d, int size) override { unimplemented("propSetFloatArray"); }
  AVSMap* __stdcall createMap() override { unimplemented("createMap"); }
  void __stdcall freeMap(AVSMap* map) override { unimplemented("freeMap"); }
  void __stdcall clearMap(AVSMap* map) override { unimplemented("clearMap"); }
  void* __stdcall Allocate(size_t nBytes, size_t alignment, AvsAllocType type) override { unimplemented("Allocate"); }
  void __stdcall Free(void* ptr) override { unimplemented("Free"); }
  bool __stdcall MakePropertyWritable(PVideoFrame* pvf) override { unimplemented("MakePropertyWritable"); }
  int __stdcall propGetIntSaturated(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetIntSaturated"); }
  float __stdcall propGetFloatSaturated(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetFloatSaturated"); }
  int __stdcall propGetDataTypeHint(const AVSMap* map, const char* key, int index, int* error) override { unimplemented("propGetDataTypeHint"); }
  int __stdcall propSetDataH(AVSMap* map, const char* key, const char* d, int length, int type, int append) override { unimplemented("propSetDataH"); }
  void __stdcall ApplyMessageEx(PVideoFrame* frame, const VideoInfo& vi, const char* message, int size, int textcolor, int halocolor, int bgcolor, bool utf8) override { unimplemented("ApplyMessageEx"); }
  AVSValue __stdcall Invoke(const char* name, const AVSValue args, const char* const* arg_names) override { unimplemented("Invoke"); }
  void __stdcall PushContext(int level) override { unimplemented("PushContext"); }
  bool __stdcall InvokeTry(AVSValue* result, const char* name, const AVSValue& args, const char* const* arg_names) override { unimplemented("InvokeTry"); }
  AVSValue __stdcall Invoke2(const AVSValue& implicit_last, const char* name, const AVSValue args, const char* const* arg_names) override { unimplemented("Invoke2"); }
  bool __stdcall Invoke2Try(AVSValue* result, const AVSValue& implicit_last, const char* name, const AVSValue args, const char* const* arg_names) override { unimplemented("Invoke2Try"); }
  AVSValue __stdcall Invoke3(const AVSValue& implicit_last, const PFunction& func, const AVSValue args, const char* const* arg_names) override { unimplemented("Invoke3"); }
  bool __stdcall Invoke3Try(AVSValue* result, const AVSValue& implicit_last, const PFunction& func, const AVSValue args, const char* const* arg_names) override { unimplemented("Invoke3Try"); }
  // planar frames only: planes one after another, 64-byte aligned pitches
  PVideoFrame NewFrame(const VideoInfo& vi) {
    const int cs = vi.ComponentSize();
    const bool planar = vi.IsPlanar();
    const int np = planar ? vi.NumComponents() : 1;
    const int row = planar ? vi.width * cs : vi.BytesFromPixels(vi.width);
    const int pitch = (row + 63) / 64 * 64;
    const int sw = planar && np > 1 ? vi.GetPlaneWidthSubsampling(PLANAR_U) : 0;
    const int sh = planar && np > 1 ? vi.GetPlaneHeightSubsampling(PLANAR_U) : 0;
    const int rowUV = (vi.width >> sw) * cs, pitchUV = np > 1 ? (rowUV + 63) / 64 * 64 : 0;
    const int hUV = np > 1 ? vi.height >> sh : 0;
    const int offU = pitch * vi.height, offV = offU + pitchUV * hUV;
    const int offA = np == 4 ? offV + pitchUV * hUV : 0;
    const int size = (np == 4 ? offA + pitch * vi.height : offV + pitchUV * hUV);
    auto* vfb = new VideoFrameBuffer(size, 0, nullptr);
    auto* f = new VideoFrame(vfb, nullptr, 0, pitch, row, vi.height, np > 1 ? offU : 0, np > 1 ? offV : 0, pitchUV,
                             np > 1 ? rowUV : 0, hUV, offA, vi.pixel_type);
    return PVideoFrame(f);
  }
};

namespace {

// A source clip of planar frames copied from the host's buffers.
class SourceClip : public IClip {
 public:
  VideoInfo vi;
  std::vector<std::vector<uint8_t>> frames;  // per frame: planes one after another, packed rows
  PVideoFrame __stdcall GetFrame(int n, IScriptEnvironment* env) override {
    n = n < 0 ? 0 : (n >= vi.num_frames ? vi.num_frames - 1 : n);
    PVideoFrame f = static_cast<ScriptEnvironment*>(env)->NewFrame(vi);
    const uint8_t* src = frames[n].data();
    int planes[4];
    const int np = plane_ids(vi, planes);
    for (int p = 0; p < np; p++) {
      const int row = f->GetRowSize(planes[p]), h = f->GetHeight(planes[p]);
      BYTE* d = f->GetWritePtr(planes[p]);
      for (int y = 0; y < h; y++) std::memcpy(d + (size_t)y * f->GetPitch(planes[p]), src + (size_t)y * row, row);
      src += (size_t)row * h;
    }
    return f;
  }
  bool __stdcall GetParity(int) override { return false; }
  void __stdcall GetAudio(void*, int64_t, int64_t, IScriptEnvironment*) override {}
  int __stdcall SetCacheHints(int, int) override { return 0; }
  const VideoInfo& __stdcall GetVideoInfo() override { return vi; }
};

struct Host {
  ScriptEnvironment env;
  std::vector<void*> libs;
};

struct Clip {
  PClip clip;
  int mt_mode = 0;
};

thread_local std::string g_error;

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

// Every function below returns 0 on success or -1 with avsh_error() set.
const char* avsh_error() { return g_error.c_str(); }

void* avsh_create() { return new Host; }

// pixel_type of a planar format: family 0 Y only, 1 YUV, 2 RGB, 3 YUVA;
// bits 8, 10, 12, 14, 16 or 32 (float); ssw/ssh chroma shifts (0..2). -1 if
// the combination has no AviSynth+ format.
int avsh_pixel_type(int family, int bits, int ssw, int ssh) {
  int sb;
  switch (bits) {
    case 8: sb = VideoInfo::CS_Sample_Bits_8; break;
    case 10: sb = VideoInfo::CS_Sample_Bits_10; break;
    case 12: sb = VideoInfo::CS_Sample_Bits_12; break;
    case 14: sb = VideoInfo::CS_Sample_Bits_14; break;
    case 16: sb = VideoInfo::CS_Sample_Bits_16; break;
    case 32: sb = VideoInfo::CS_Sample_Bits_32; break;
    default: return -1;
  }
  if (ssw < 0 || ssw > 2 || ssh < 0 || ssh > 2) return -1;
  // subsampling codes: shift s is stored as (s - 1) & 3
  const int sub = (((ssw - 1) & 3) << VideoInfo::CS_Shift_Sub_Width) | (((ssh - 1) & 3) << VideoInfo::CS_Shift_Sub_Height);
  switch (family) {
    case 0: return VideoInfo::CS_GENERIC_Y | sb;
    case 1: return VideoInfo::CS_PLANAR | VideoInfo::CS_YUV | VideoInfo::CS_VPlaneFirst | sub | sb;
    case 2: return VideoInfo::CS_GENERIC_RGBP | sb;
    case 3: return VideoInfo::CS_PLANAR | VideoInfo::CS_YUVA | VideoInfo::CS_VPlaneFirst | sub | sb;
  }
  return -1;
}

void avsh_destroy(void* h) { delete static_cast<Host*>(h); }

int avsh_load_plugin(void* h, const char* path) {
  auto* host = static_cast<Host*>(h);
  void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!lib) {
    g_error = dlerror();
    return -1;
  }
  using Init = const char* (*)(IScriptEnvironment*, const AVS_Linkage* const);
  auto init = reinterpret_cast<Init>(dlsym(lib, "AvisynthPluginInit3"));
  if (!init) {
    g_error = "AvisynthPluginInit3 not exported";
    return -1;
  }
  try {
    init(&host->env, &g_linkage);
  } catch (const AvisynthError& e) {
    g_error = e.msg;
    return -1;
  } catch (...) {
    g_error = "uncaught exception in AvisynthPluginInit3";
    return -1;
  }
  host->libs.push_back(lib);
  return 0;
}

// Registered function k of the host (name and parameter string), or -1.
int avsh_function(void* h, int k, const char** name, const char** params) {
  auto* host = static_cast<Host*>(h);
  if (k < 0 || k >= (int)host->env.functions.size()) return -1;
  *name = host->env.functions[k].name.c_str();
  *params = host->env.functions[k].params.c_str();
  return 0;
}

// A planar source clip: `frames` frames of `data` (per frame, the planes one
// after another with packed rows).
void* avsh_clip(void* h, int width, int height, int pixel_type, int num_frames, const uint8_t* data,
                long long frame_bytes) {
  auto* c = new SourceClip;
  std::memset(&c->vi, 0, sizeof(c->vi));
  c->vi.width = width;
  c->vi.height = height;
  c->vi.pixel_type = pixel_type;
  c->vi.num_frames = num_frames;
  c->vi.fps_numerator = 25;
  c->vi.fps_denominator = 1;
  c->frames.resize(num_frames);
  for (int n = 0; n < num_frames; n++)
    c->frames[n].assign(data + (size_t)n * frame_bytes, data + (size_t)(n + 1) * frame_bytes);
  auto* out = new Clip;
  out->clip = PClip(c);
  return out;
}

void avsh_clip_free(void* c) { delete static_cast<Clip*>(c); }

int avsh_clip_info(void* c, int out[4]) {
  const VideoInfo& vi = static_cast<Clip*>(c)->clip->GetVideoInfo();
  out[0] = vi.width;
  out[1] = vi.height;
  out[2] = vi.pixel_type;
  out[3] = vi.num_frames;
  return 0;
}

// Calls function `name` on `clip` with named arguments: kinds[i] is 'i'
// (ints[i]), 'f' (floats[i]) or 'b' (ints[i] != 0). Positional slots follow
// the function's parameter string ("c[sigma]f[beta]f..."). On success *out is
// the resulting clip; its MT mode (the plugin's SetCacheHints answer) in mt.
int avsh_invoke(void* h, const char* name, void* clip, int nargs, const char* const* names, const char* kinds,
                const int* ints, const double* floats, void** out, int* mt) {
  auto* host = static_cast<Host*>(h);
  const Function* fn = nullptr;
  for (auto& f : host->env.functions)
    if (f.name == name) fn = &f;
  if (!fn) {
    g_error = std::string("no function ") + name;
    return -1;
  }
  // slots of the parameter string
  std::vector<std::string> slots;
  const std::string& p = fn->params;
  for (size_t i = 0; i < p.size();) {
    if (p[i] == '[') {
      const size_t j = p.find(']', i);
      slots.push_back(p.substr(i + 1, j - i - 1));
      i = j + 2;  // skip the type letter
    } else {
      slots.push_back("");
      i += 1;
    }
  }
  std::vector<AVSValue> args(slots.size());
  args[0] = AVSValue(static_cast<Clip*>(clip)->clip);
  for (int a = 0; a < nargs; a++) {
    size_t k = 0;
    while (k < slots.size() && slots[k] != names[a]) k++;
    if (k == slots.size()) {
      g_error = std::string(name) + " does not have a named argument \"" + names[a] + "\"";
      return -1;
    }
    if (kinds[a] == 'i') args[k] = AVSValue(ints[a]);
    else if (kinds[a] == 'b') args[k] = AVSValue(ints[a] != 0);
    else args[k] = AVSValue(floats[a]);
  }
  try {
    AVSValue r = fn->apply(AVSValue(args.data(), (int)args.size()), fn->user_data, &host->env);
    if (!r.IsClip()) {
      g_error = "the function did not return a clip";
      return -1;
    }
    auto* c = new Clip;
    c->clip = r.AsClip();
    // the core reads a new filter's VideoInfo before serving frames from it
    // (AviSynth+ wraps it in a cache at this point)
    c->clip->GetVideoInfo();
    c->mt_mode = c->clip->SetCacheHints(CACHE_GET_MTMODE, 0);
    if (mt) *mt = c->mt_mode;
    *out = c;
    return 0;
  } catch (const AvisynthError& e) {
    g_error = e.msg;
    return -1;
  } catch (const char* e) {
    g_error = std::string("uncaught exception: ") + e;
    return -1;
  } catch (...) {
    g_error = "uncaught exception";
    return -1;
  }
}

// Frame n of `clip`, its planes copied to dst[p] (rows of `stride[p]` bytes).
int avsh_get_frame(void* h, void* clip, int n, void* const* dst, const int* stride) {
  auto* host = static_cast<Host*>(h);
  auto* c = static_cast<Clip*>(clip);
  try {
    PVideoFrame f = c->clip->GetFrame(n, &host->env);
    const VideoInfo& vi = c->clip->GetVideoInfo();
    int planes[4];
    const int np = plane_ids(vi, planes);
    for (int p = 0; p < np; p++) {
      const int row = f->GetRowSize(planes[p]), hh = f->GetHeight(planes[p]);
      for (int y = 0; y < hh; y++)
        std::memcpy(static_cast<char*>(dst[p]) + (size_t)y * stride[p], f->GetReadPtr(planes[p]) + (size_t)y * f->GetPitch(planes[p]),
                    row);
    }
    return 0;
  } catch (const AvisynthError& e) {
    g_error = e.msg;
    return -1;
  } catch (const char* e) {
    g_error = std::string("uncaught exception: ") + e;
    return -1;
  } catch (...) {
    g_error = "uncaught exception";
    return -1;
  }
}

#pragma GCC visibility pop
}  // extern "C"
