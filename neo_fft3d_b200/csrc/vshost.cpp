// Headless VapourSynth API v3.6 host.
//
// Loads a VapourSynth plugin (.so), registers its functions, feeds it clips that
// live in caller memory and renders frames — without a VapourSynth install.
// It implements the VSAPI members that a DualSynth-style plugin uses
// (the reference's include/dualsynth/vs_wrapper.hpp:107-303, ds_frame.hpp:35-153,
// ds_format.hpp:18-42, ds_videoinfo.hpp:146-165) and nothing else; every
// other member is a null pointer.
//
// Frame requests follow VapourSynth's two-phase protocol: getFrame(n,
// arInitial) records requestFrameFilter() calls, the host renders those input
// frames, then getFrame(n, arAllFramesReady) returns the output. Filters whose
// mode is fmParallel may be called from several host threads at once; other
// modes are serialised per node (fmSerial filters are called in frame order).
//
// Exported C interface: see the vsh_* functions at the end of this file.
#include <VapourSynth.h>

#include <dlfcn.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

const VSAPI* api();

struct Prop {
  char type = ptUnset;
  std::vector<int64_t> i;
  std::vector<double> f;
  std::vector<std::string> s;
  std::vector<VSNodeRef*> c;
  std::vector<const VSFrameRef*> v;
  int size() const {
    switch (type) {
      case ptInt: return (int)i.size();
      case ptFloat: return (int)f.size();
      case ptData: return (int)s.size();
      case ptNode: return (int)c.size();
      case ptFrame: return (int)v.size();
      default: return 0;
    }
  }
};

}  // namespace

struct VSMap {
  std::map<std::string, Prop> props;
  std::string error;
};

struct VSFrameRef {
  const VSFormat* format = nullptr;
  int width = 0, height = 0;
  int stride[3] = {0, 0, 0};
  uint8_t* data[3] = {nullptr, nullptr, nullptr};
  bool owns = true;
  std::atomic<int> refs{1};
  VSMap props;
  ~VSFrameRef() {
    if (owns)
      for (auto* d : data) std::free(d);
  }
};

struct VSCore;

struct Node {
  // a source node (frames in caller memory) or a filter node (plugin callbacks)
  bool is_source = true;
  VSVideoInfo vi{};
  // source
  std::vector<VSFrameRef*> frames;
  // filter
  VSFilterGetFrame getframe = nullptr;
  VSFilterFree freefn = nullptr;
  void* instance = nullptr;
  int mode = fmParallel;
  VSCore* core = nullptr;
  std::mutex serial;
  std::atomic<int> refs{1};
  ~Node() {
    if (freefn) freefn(instance, core, api());
    for (auto* f : frames) api()->freeFrame(f);
  }
};

struct VSNodeRef {
  std::shared_ptr<Node> node;
};

struct VSNode {
  std::shared_ptr<Node> node;
};

struct VSFrameContext {
  std::vector<std::pair<std::shared_ptr<Node>, int>> requests;
  std::map<std::pair<Node*, int>, const VSFrameRef*> ready;
  std::string error;
};

struct VSPlugin {
  std::string id, ns, name;
  struct Func {
    std::string args;
    VSPublicFunction fn;
    void* data;
  };
  std::map<std::string, Func> funcs;
  void* handle = nullptr;
};

struct VSCore {
  std::mutex fmt_lock;
  std::vector<std::unique_ptr<VSFormat>> formats;
  std::vector<std::unique_ptr<VSPlugin>> plugins;
};

namespace {

thread_local std::string g_last_error;

const VSFormat* register_format(int cf, int st, int bits, int ssw, int ssh, VSCore* core) {
  if (!core) return nullptr;
  std::lock_guard<std::mutex> g(core->fmt_lock);
  for (auto& f : core->formats)
    if (f->colorFamily == cf && f->sampleType == st && f->bitsPerSample == bits && f->subSamplingW == ssw &&
        f->subSamplingH == ssh)
      return f.get();
  auto f = std::make_unique<VSFormat>();
  std::memset(f.get(), 0, sizeof(VSFormat));
  std::snprintf(f->name, sizeof(f->name), "fmt%d_%d_%d_%d_%d", cf, st, bits, ssw, ssh);
  f->id = (int)core->formats.size() + 1;
  f->colorFamily = cf;
  f->sampleType = st;
  f->bitsPerSample = bits;
  f->bytesPerSample = bits <= 8 ? 1 : (bits <= 16 ? 2 : 4);
  f->subSamplingW = ssw;
  f->subSamplingH = ssh;
  f->numPlanes = (cf == cmGray) ? 1 : 3;
  core->formats.push_back(std::move(f));
  return core->formats.back().get();
}

int plane_w(const VSFormat* f, int w, int p) { return p ? (w >> f->subSamplingW) : w; }
int plane_h(const VSFormat* f, int h, int p) { return p ? (h >> f->subSamplingH) : h; }

VSFrameRef* alloc_frame(const VSFormat* f, int w, int h) {
  auto* fr = new VSFrameRef();
  fr->format = f;
  fr->width = w;
  fr->height = h;
  for (int p = 0; p < f->numPlanes; p++) {
    int rb = plane_w(f, w, p) * f->bytesPerSample;
    int stride = (rb + 63) / 64 * 64;
    fr->stride[p] = stride;
    void* d = nullptr;
    if (posix_memalign(&d, 64, (size_t)stride * plane_h(f, h, p) + 64) != 0) d = nullptr;
    fr->data[p] = (uint8_t*)d;
  }
  return fr;
}

// ---- VSAPI members -------------------------------------------------------

const VSFrameRef* VS_CC cloneFrameRef(const VSFrameRef* f) noexcept {
  if (f) const_cast<VSFrameRef*>(f)->refs++;
  return f;
}
VSNodeRef* VS_CC cloneNodeRef(VSNodeRef* n) noexcept { return n ? new VSNodeRef{n->node} : nullptr; }
void VS_CC freeFrame(const VSFrameRef* f) noexcept {
  if (f && --const_cast<VSFrameRef*>(f)->refs == 0) delete f;
}
void VS_CC freeNode(VSNodeRef* n) noexcept { delete n; }
VSFrameRef* VS_CC newVideoFrame(const VSFormat* f, int w, int h, const VSFrameRef*, VSCore*) noexcept {
  return alloc_frame(f, w, h);
}
VSFrameRef* VS_CC newVideoFrame2(const VSFormat* f, int w, int h, const VSFrameRef** src, const int* planes,
                                 const VSFrameRef*, VSCore*) noexcept {
  VSFrameRef* fr = alloc_frame(f, w, h);
  for (int p = 0; p < f->numPlanes; p++) {
    if (!src || !src[p]) continue;
    const VSFrameRef* s = src[p];
    int sp = planes[p];
    int rb = plane_w(f, w, p) * f->bytesPerSample;
    for (int y = 0; y < plane_h(f, h, p); y++)
      std::memcpy(fr->data[p] + (size_t)y * fr->stride[p], s->data[sp] + (size_t)y * s->stride[sp], rb);
  }
  return fr;
}
void VS_CC setError(VSMap* m, const char* msg) noexcept { if (m) m->error = msg ? msg : "error"; }
const char* VS_CC getError(const VSMap* m) noexcept { return (m && !m->error.empty()) ? m->error.c_str() : nullptr; }
void VS_CC setFilterError(const char* msg, VSFrameContext* ctx) noexcept { if (ctx) ctx->error = msg ? msg : "error"; }
const VSFormat* VS_CC registerFormat(int cf, int st, int bits, int ssw, int ssh, VSCore* core) noexcept {
  return register_format(cf, st, bits, ssw, ssh, core);
}
int VS_CC getStride(const VSFrameRef* f, int p) noexcept { return f->stride[p]; }
const uint8_t* VS_CC getReadPtr(const VSFrameRef* f, int p) noexcept { return f->data[p]; }
uint8_t* VS_CC getWritePtr(VSFrameRef* f, int p) noexcept { return f->data[p]; }
const VSVideoInfo* VS_CC getVideoInfo(VSNodeRef* n) noexcept { return &n->node->vi; }
void VS_CC setVideoInfo(const VSVideoInfo* vi, int, VSNode* node) noexcept { node->node->vi = *vi; }
const VSFormat* VS_CC getFrameFormat(const VSFrameRef* f) noexcept { return f->format; }
int VS_CC getFrameWidth(const VSFrameRef* f, int p) noexcept { return plane_w(f->format, f->width, p); }
int VS_CC getFrameHeight(const VSFrameRef* f, int p) noexcept { return plane_h(f->format, f->height, p); }
const VSMap* VS_CC getFramePropsRO(const VSFrameRef* f) noexcept { return &f->props; }
VSMap* VS_CC getFramePropsRW(VSFrameRef* f) noexcept { return &f->props; }

VSMap* VS_CC createMap() noexcept { return new VSMap(); }
void VS_CC freeMap(VSMap* m) noexcept {
  if (!m) return;
  for (auto& kv : m->props) {
    for (auto* n : kv.second.c) freeNode(n);
    for (auto* f : kv.second.v) freeFrame(f);
  }
  delete m;
}
int VS_CC propNumElements(const VSMap* m, const char* key) noexcept {
  auto it = m->props.find(key);
  return it == m->props.end() ? -1 : it->second.size();
}
char VS_CC propGetType(const VSMap* m, const char* key) noexcept {
  auto it = m->props.find(key);
  return it == m->props.end() ? ptUnset : it->second.type;
}
const Prop* lookup(const VSMap* m, const char* key, char type, int index, int* err) {
  auto it = m->props.find(key);
  int e = 0;
  const Prop* p = nullptr;
  if (it == m->props.end()) e = peUnset;
  else if (it->second.type != type) e = peType;
  else if (index < 0 || index >= it->second.size()) e = peIndex;
  else p = &it->second;
  if (err) *err = e;
  return p;
}
int64_t VS_CC propGetInt(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptInt, index, err);
  return p ? p->i[index] : 0;
}
double VS_CC propGetFloat(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptFloat, index, err);
  if (!p) {  // VapourSynth promotes int arguments to float parameters at call time
    auto* q = lookup(m, key, ptInt, index, nullptr);
    if (q) { if (err) *err = 0; return (double)q->i[index]; }
  }
  return p ? p->f[index] : 0.0;
}
const char* VS_CC propGetData(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptData, index, err);
  return p ? p->s[index].c_str() : nullptr;
}
int VS_CC propGetDataSize(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptData, index, err);
  return p ? (int)p->s[index].size() : 0;
}
VSNodeRef* VS_CC propGetNode(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptNode, index, err);
  return p ? cloneNodeRef(p->c[index]) : nullptr;
}
const VSFrameRef* VS_CC propGetFrame(const VSMap* m, const char* key, int index, int* err) noexcept {
  auto* p = lookup(m, key, ptFrame, index, err);
  return p ? cloneFrameRef(p->v[index]) : nullptr;
}
Prop& slot(VSMap* m, const char* key, char type, int append) {
  Prop& p = m->props[key];
  if (append == paReplace || p.type != type) {
    for (auto* n : p.c) freeNode(n);
    for (auto* f : p.v) freeFrame(f);
    p = Prop();
    p.type = type;
  }
  return p;
}
int VS_CC propSetInt(VSMap* m, const char* key, int64_t i, int append) noexcept {
  slot(m, key, ptInt, append).i.push_back(i);
  return 0;
}
int VS_CC propSetFloat(VSMap* m, const char* key, double d, int append) noexcept {
  slot(m, key, ptFloat, append).f.push_back(d);
  return 0;
}
int VS_CC propSetData(VSMap* m, const char* key, const char* d, int size, int append) noexcept {
  slot(m, key, ptData, append).s.push_back(size < 0 ? std::string(d) : std::string(d, size));
  return 0;
}
int VS_CC propSetNode(VSMap* m, const char* key, VSNodeRef* n, int append) noexcept {
  slot(m, key, ptNode, append).c.push_back(cloneNodeRef(n));
  return 0;
}
int VS_CC propDeleteKey(VSMap* m, const char* key) noexcept {
  auto it = m->props.find(key);
  if (it == m->props.end()) return 0;
  for (auto* n : it->second.c) freeNode(n);
  for (auto* f : it->second.v) freeFrame(f);
  m->props.erase(it);
  return 1;
}

void VS_CC createFilter(const VSMap* in, VSMap* out, const char* name, VSFilterInit init, VSFilterGetFrame getframe,
                        VSFilterFree freefn, int mode, int flags, void* instance, VSCore* core) noexcept {
  (void)name; (void)flags;
  auto node = std::make_shared<Node>();
  node->is_source = false;
  node->getframe = getframe;
  node->freefn = freefn;
  node->instance = instance;
  node->mode = mode;
  node->core = core;
  VSNode wrapper{node};
  init(const_cast<VSMap*>(in), out, &node->instance, &wrapper, core, api());
  if (getError(out)) return;
  VSNodeRef ref{node};
  propSetNode(out, "clip", &ref, paAppend);
}

const VSFrameRef* render(const std::shared_ptr<Node>& node, int n, std::string& err);

const VSFrameRef* VS_CC getFrameFilter(int n, VSNodeRef* node, VSFrameContext* ctx) noexcept {
  auto it = ctx->ready.find({node->node.get(), n});
  if (it != ctx->ready.end()) return cloneFrameRef(it->second);
  // a frame the filter did not request: rendered on demand (VapourSynth
  // itself would return NULL here)
  std::string err;
  return render(node->node, n, err);
}
void VS_CC requestFrameFilter(int n, VSNodeRef* node, VSFrameContext* ctx) noexcept {
  ctx->requests.emplace_back(node->node, n);
}
const VSFrameRef* VS_CC getFrame(int n, VSNodeRef* node, char* errmsg, int bufsize) noexcept {
  std::string err;
  const VSFrameRef* f = render(node->node, n, err);
  if (!f && errmsg && bufsize > 0) std::snprintf(errmsg, bufsize, "%s", err.c_str());
  return f;
}
void VS_CC logMessage(int, const char* msg) noexcept { std::fprintf(stderr, "vshost: %s\n", msg); }

const VSFrameRef* render(const std::shared_ptr<Node>& node, int n, std::string& err) {
  if (n < 0) n = 0;
  if (node->vi.numFrames > 0 && n >= node->vi.numFrames) n = node->vi.numFrames - 1;
  if (node->is_source) return cloneFrameRef(node->frames[n]);
  std::unique_lock<std::mutex> lk(node->serial, std::defer_lock);
  if (node->mode != fmParallel) lk.lock();
  VSFrameContext ctx;
  void* frame_data = nullptr;
  const VSFrameRef* out = node->getframe(n, arInitial, &node->instance, &frame_data, &ctx, node->core, api());
  if (!out && ctx.error.empty()) {
    for (auto& rq : ctx.requests) {
      auto key = std::make_pair(rq.first.get(), rq.second);
      if (ctx.ready.count(key)) continue;
      const VSFrameRef* f = render(rq.first, rq.second, err);
      if (!f) return nullptr;
      ctx.ready[key] = f;
    }
    out = node->getframe(n, arAllFramesReady, &node->instance, &frame_data, &ctx, node->core, api());
  }
  for (auto& kv : ctx.ready) freeFrame(kv.second);
  if (!ctx.error.empty()) {
    err = ctx.error;
    if (out) freeFrame(out);
    return nullptr;
  }
  if (!out) err = "filter returned no frame";
  return out;
}

// ---- plugin registration -------------------------------------------------

thread_local VSPlugin* g_loading = nullptr;

void VS_CC configPlugin(const char* id, const char* ns, const char* name, int, int, VSPlugin* p) {
  p->id = id;
  p->ns = ns;
  p->name = name;
}
void VS_CC registerFunction(const char* name, const char* args, VSPublicFunction fn, void* data, VSPlugin* p) {
  p->funcs[name] = VSPlugin::Func{args, fn, data};
}

VSAPI make_api() {
  VSAPI a;
  std::memset(&a, 0, sizeof(a));
  a.cloneFrameRef = cloneFrameRef;
  a.cloneNodeRef = cloneNodeRef;
  a.freeFrame = freeFrame;
  a.freeNode = freeNode;
  a.newVideoFrame = newVideoFrame;
  a.newVideoFrame2 = newVideoFrame2;
  a.createFilter = createFilter;
  a.setError = setError;
  a.getError = getError;
  a.setFilterError = setFilterError;
  a.registerFormat = registerFormat;
  a.getFrame = getFrame;
  a.getFrameFilter = getFrameFilter;
  a.requestFrameFilter = requestFrameFilter;
  a.getStride = getStride;
  a.getReadPtr = getReadPtr;
  a.getWritePtr = getWritePtr;
  a.createMap = createMap;
  a.freeMap = freeMap;
  a.getVideoInfo = getVideoInfo;
  a.setVideoInfo = setVideoInfo;
  a.getFrameFormat = getFrameFormat;
  a.getFrameWidth = getFrameWidth;
  a.getFrameHeight = getFrameHeight;
  a.getFramePropsRO = getFramePropsRO;
  a.getFramePropsRW = getFramePropsRW;
  a.propNumElements = propNumElements;
  a.propGetType = propGetType;
  a.propGetInt = propGetInt;
  a.propGetFloat = propGetFloat;
  a.propGetData = propGetData;
  a.propGetDataSize = propGetDataSize;
  a.propGetNode = propGetNode;
  a.propGetFrame = propGetFrame;
  a.propDeleteKey = propDeleteKey;
  a.propSetInt = propSetInt;
  a.propSetFloat = propSetFloat;
  a.propSetData = propSetData;
  a.propSetNode = propSetNode;
  a.logMessage = logMessage;
  return a;
}

const VSAPI* api() {
  static const VSAPI a = make_api();
  return &a;
}

size_t frame_bytes(const VSFormat* f, int w, int h) {
  size_t s = 0;
  for (int p = 0; p < f->numPlanes; p++) s += (size_t)plane_w(f, w, p) * plane_h(f, h, p) * f->bytesPerSample;
  return s;
}

}  // namespace

// ---- exported C interface ---------------------------------------------------
//
// Packed frame layout used by vsh_clip_new / vsh_render: for each frame, its
// planes one after another, each plane_w*plane_h*bytesPerSample bytes, rows
// without padding.

extern "C" {

const VSAPI* vsh_api(void) { return api(); }
const char* vsh_last_error(void) { return g_last_error.c_str(); }

VSCore* vsh_core_new(void) { return new VSCore(); }
void vsh_core_free(VSCore* c) {
  if (!c) return;
  // plugin handles are left loaded: plugin globals may outlive filter nodes
  delete c;
}

// Load a plugin and return its handle, or NULL (see vsh_last_error()).
VSPlugin* vsh_load_plugin(VSCore* core, const char* path) {
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) { g_last_error = dlerror(); return nullptr; }
  auto init = (VSInitPlugin)dlsym(h, "VapourSynthPluginInit");
  if (!init) { g_last_error = "VapourSynthPluginInit not exported"; return nullptr; }
  auto p = std::make_unique<VSPlugin>();
  p->handle = h;
  init(configPlugin, registerFunction, p.get());
  core->plugins.push_back(std::move(p));
  return core->plugins.back().get();
}

const char* vsh_plugin_namespace(VSPlugin* p) { return p->ns.c_str(); }
const char* vsh_plugin_id(VSPlugin* p) { return p->id.c_str(); }
// Argument string of a registered function, or NULL.
const char* vsh_function_args(VSPlugin* p, const char* name) {
  auto it = p->funcs.find(name);
  return it == p->funcs.end() ? nullptr : it->second.args.c_str();
}

VSMap* vsh_map_new(void) { return createMap(); }
void vsh_map_free(VSMap* m) { freeMap(m); }
void vsh_map_set_int(VSMap* m, const char* k, int64_t v, int append) { propSetInt(m, k, v, append); }
void vsh_map_set_float(VSMap* m, const char* k, double v, int append) { propSetFloat(m, k, v, append); }
void vsh_map_set_node(VSMap* m, const char* k, VSNodeRef* n) { propSetNode(m, k, n, paReplace); }
const char* vsh_map_error(VSMap* m) { return getError(m); }
VSNodeRef* vsh_map_get_node(VSMap* m, const char* k) {
  int e = 0;
  VSNodeRef* n = propGetNode(m, k, 0, &e);
  return e ? nullptr : n;
}

// Call a registered function; returns the output map (check vsh_map_error).
VSMap* vsh_invoke(VSCore* core, VSPlugin* p, const char* name, VSMap* args) {
  VSMap* out = createMap();
  auto it = p->funcs.find(name);
  if (it == p->funcs.end()) { setError(out, "no such function"); return out; }
  it->second.fn(args, out, it->second.data, core, api());
  return out;
}

// A source clip over caller memory (zero copy): `data` holds num_frames packed
// frames and must outlive the clip. color_family is a VSColorFamily.
VSNodeRef* vsh_clip_new(VSCore* core, int color_family, int sample_type, int bits, int ssw, int ssh, int width,
                        int height, int num_frames, const void* data) {
  const VSFormat* f = register_format(color_family, sample_type, bits, ssw, ssh, core);
  auto node = std::make_shared<Node>();
  node->is_source = true;
  node->vi.format = f;
  node->vi.fpsNum = 24;
  node->vi.fpsDen = 1;
  node->vi.width = width;
  node->vi.height = height;
  node->vi.numFrames = num_frames;
  size_t fb = frame_bytes(f, width, height);
  const uint8_t* base = (const uint8_t*)data;
  for (int n = 0; n < num_frames; n++) {
    auto* fr = new VSFrameRef();
    fr->format = f;
    fr->width = width;
    fr->height = height;
    fr->owns = false;
    const uint8_t* q = base + fb * n;
    for (int p = 0; p < f->numPlanes; p++) {
      fr->stride[p] = plane_w(f, width, p) * f->bytesPerSample;
      fr->data[p] = const_cast<uint8_t*>(q);
      q += (size_t)fr->stride[p] * plane_h(f, height, p);
    }
    node->frames.push_back(fr);
  }
  return new VSNodeRef{node};
}

void vsh_node_free(VSNodeRef* n) { freeNode(n); }

// Video info of a node: {width, height, num_frames, color_family, bits, ssw, ssh, planes}
void vsh_node_info(VSNodeRef* n, int* out8) {
  const VSVideoInfo& vi = n->node->vi;
  out8[0] = vi.width; out8[1] = vi.height; out8[2] = vi.numFrames;
  out8[3] = vi.format ? vi.format->colorFamily : 0;
  out8[4] = vi.format ? vi.format->bitsPerSample : 0;
  out8[5] = vi.format ? vi.format->subSamplingW : 0;
  out8[6] = vi.format ? vi.format->subSamplingH : 0;
  out8[7] = vi.format ? vi.format->numPlanes : 0;
}

// Render frames [first, first+count) into `dst` (count packed frames).
// Frames are handed out to `threads` host threads in increasing order; nodes
// that are not fmParallel are serialised. Returns 0, or -1 on a filter error.
int vsh_render(VSNodeRef* n, int first, int count, int threads, void* dst) {
  const VSVideoInfo& vi = n->node->vi;
  const VSFormat* f = vi.format;
  size_t fb = frame_bytes(f, vi.width, vi.height);
  std::atomic<int> next{0};
  std::atomic<int> failed{0};
  std::mutex err_lock;
  std::string err_all;
  auto worker = [&] {
    for (;;) {
      int i = next++;
      if (i >= count || failed) return;
      std::string err;
      const VSFrameRef* fr = render(n->node, first + i, err);
      if (!fr) {
        failed = 1;
        std::lock_guard<std::mutex> g(err_lock);
        err_all = err;
        return;
      }
      uint8_t* q = (uint8_t*)dst + fb * i;
      for (int p = 0; p < f->numPlanes; p++) {
        int rb = plane_w(f, vi.width, p) * f->bytesPerSample;
        for (int y = 0; y < plane_h(f, vi.height, p); y++) {
          std::memcpy(q, fr->data[p] + (size_t)y * fr->stride[p], rb);
          q += rb;
        }
      }
      freeFrame(fr);
    }
  };
  if (n->node->mode != fmParallel && !n->node->is_source) threads = 1;  // keep frame order
  if (threads <= 1) worker();
  else {
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++) th.emplace_back(worker);
    for (auto& t : th) t.join();
  }
  if (failed) { g_last_error = err_all; return -1; }
  return 0;
}

}  // extern "C"
