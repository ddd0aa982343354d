// Batched multi-plane scheduler: one time step of many planes (luma and
// chroma of many clips, mixed sizes, block sizes and bt) as one batched
// persistent launch per kernel variant and phase, captured into a CUDA graph.
//
// A step plans every plane with the engine's own per-frame control (spectrum
// ring, btcur edges, Kalman passthrough, crop) while the launches are
// recorded instead of issued (fft3d::plane_plan). The records are grouped by
// kernel variant -- forward by (bw, bh, sample type), filter/inverse by
// (bw, bh, mode), plane copies, overlap-add by sample type -- and each group
// becomes ONE launch whose CTAs walk a list of (plane, CTA-of-that-plane)
// work items, so a step of 48 clips x 3 planes is tens of launches instead of
// ~430.
//
// Waves. Launching each phase over ALL planes streams the new spectra and
// time-domain blocks of every plane through HBM between the phases, while a
// plane filtered on its own finds them in L2. So a step can be cut into waves
// of consecutive planes whose new spectra + time-domain blocks fit a byte
// budget, the phases running wave by wave.
//
// Autotuner. The step's shape (variants and per-plane work items) is its
// signature. The first steps of a new signature time the whole step under
// each candidate wave budget (24..192 MiB, or one wave), then time every
// launch under each candidate schedule -- persistent grid of 1, 2, 4 or all
// resident CTAs per SM, or one CTA per work item; work items plane-major or
// interleaved across planes -- and keep the fastest budget and the fastest
// schedule per launch. The tuned step is then captured once into a CUDA graph
// (argument upload from pinned staging + the launches); later steps of that
// signature only rewrite the pinned arguments and launch the graph. Two
// graph instances alternate over two staging buffers so that the host can
// prepare a step while the previous one runs.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fft3d_b200.h"
#include "fft3d_batch.h"
#include "fft3d_kernels.cuh"

namespace {

using fft3d::Deferred;

int cuda_fail(cudaError_t e, const char* what) {
  return fft3d::engine_fail(FFT3D_E_CUDA,
                            std::string("neo_fft3d: CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define CK(call, what)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// candidate schedules: resident CTAs per SM of the persistent grid (0 = one
// CTA per work item) x work-item order
struct Sched {
  int per_sm;
  int interleave;
};
const Sched kCandidates[] = {{0, 0}, {1, 0}, {2, 0}, {4, 0}, {64, 0}, {0, 1}, {1, 1}, {2, 1}, {4, 1}, {64, 1}};
constexpr int kNumCand = sizeof(kCandidates) / sizeof(kCandidates[0]);

// phases in launch order; plane copies (crop borders, Kalman frame 0) go
// before the overlap-add, which writes the interior over them
enum Phase { PH_FWD = 0, PH_INV = 1, PH_COPY = 2, PH_OLA = 3 };

// Wave budgets tried by the tuner: the new spectra and time-domain blocks of
// the planes of one wave (forward -> filter/inverse -> overlap-add) should
// stay in the 126 MB L2 between the phases; 0 = all planes in one wave.
const size_t kBudgets[] = {size_t(24) << 20, size_t(48) << 20, size_t(96) << 20, size_t(192) << 20, 0};
constexpr int kNumBudgets = sizeof(kBudgets) / sizeof(kBudgets[0]);
constexpr size_t kDefaultBudget = 0;

struct Group {
  int wave, phase, bw, bh, var;  // var: bytes per sample (forward, overlap-add) or filter mode
  std::vector<int> recs;    // indices into the Deferred vector of the phase
  std::vector<int> per;     // work items per record
  int nitems = 0;
  int occupancy = 1;        // resident CTAs per SM
  size_t args_off = 0, items_off = 0, arg_size = 0;
  Sched sched{64, 0};
  int grid = 1;
};

struct Plan {
  std::vector<Group> groups;
  std::string sig;
  size_t args_bytes = 0, items_bytes = 0;
};

struct Tune {
  int stage = 0;                       // 0: wave budget, 1: per-launch schedule, 2: done
  int next = 0;                        // next candidate of the stage
  std::vector<float> budget_ms;        // whole-step time per budget
  size_t budget = kDefaultBudget;
  std::vector<std::vector<float>> ms;  // [group][schedule candidate]
  std::vector<Sched> best;
};

struct Captured {
  void* d_buf = nullptr;      // device: args then items
  void* h_stage[2] = {};      // pinned: args of a step
  cudaGraphExec_t exec[2] = {};
  cudaEvent_t done[2] = {};
  bool used[2] = {};
  int parity = 0;
  ~Captured() {
    for (int p = 0; p < 2; p++) {
      if (exec[p]) cudaGraphExecDestroy(exec[p]);
      if (done[p]) cudaEventDestroy(done[p]);
      if (h_stage[p]) cudaFreeHost(h_stage[p]);
    }
    if (d_buf) cudaFree(d_buf);
  }
};

// filter/inverse groups whose var is kRunVar + mode launch runs of frame groups
constexpr int kRunVar = 100;

size_t arg_size(int phase, int var) {
  switch (phase) {
    case PH_FWD: return sizeof(fft3d::ForwardArgs);
    case PH_INV: return var >= kRunVar ? sizeof(fft3d::GroupRun) : sizeof(fft3d::InverseArgs);
    case PH_COPY: return sizeof(fft3d::CopyArgs);
    default: return sizeof(fft3d::OlaArgs);
  }
}

const fft3d::Geom& rec_geom(const Deferred& d, int phase, int var, int r) {
  if (phase == PH_INV && var >= kRunVar) return d.runs[r].r.a.g;
  return phase == PH_FWD ? d.fwd[r].a.g : (phase == PH_INV ? d.inv[r].a.g : d.ola[r].a.g);
}

fft3d::CopyArgs copy_args(const Deferred::Copy& c) {
  fft3d::CopyArgs a;
  a.dst = c.dst;
  a.dpitch = (long long)c.dpitch;
  a.src = c.src;
  a.spitch = (long long)c.spitch;
  a.width = (long long)c.width;
  a.height = (int)c.height;
  return a;
}

}  // namespace

struct fft3d_batch {
  std::mutex mu;
  int device = 0;
  int sms = 148;
  int tuning = 1;
  cudaStream_t cap = nullptr;  // capture stream
  std::map<std::string, Tune> tunes;
  std::map<std::string, std::unique_ptr<Captured>> graphs;
  void* d_direct = nullptr;
  size_t d_direct_cap = 0;
  void* h_direct = nullptr;
  size_t h_direct_cap = 0;
  cudaEvent_t direct_done = nullptr;
  // steps, graph launches, tuning steps, host ms planning the planes (sum),
  // kernels of the last step, step shapes, wave budget (MiB) of the last
  // tuned step, host ms of the steps (sum)
  double stats[8] = {};
  // optional per-phase timing: tuned steps run without the graph, with
  // events around each launch, resolved when the counters are read
  struct Pending {
    int phase;
    double bytes;
    cudaEvent_t a, b;
  };
  bool timing = false;
  std::vector<Pending> pending;
  double t_phase[4][3] = {};  // launches, ms, algorithmic bytes
};

namespace {

int rec_plane(const Deferred& d, int phase, int var, int r) {
  switch (phase) {
    case PH_FWD: return d.fwd[r].plane;
    case PH_INV: return var >= kRunVar ? d.runs[r].plane : d.inv[r].plane;
    case PH_COPY: return d.copies[r].plane;
    default: return d.ola[r].plane;
  }
}

// Groups the records by (wave, phase, kernel variant); budget 0 = one wave.
void build_groups(const Deferred& d, int nplanes, size_t budget, Plan& plan) {
  std::vector<double> weight(nplanes, 0.0);
  for (const auto& r : d.inv) {
    const fft3d::Geom& g = r.a.g;
    weight[r.plane] += (double)g.nblocks * g.bh * (g.bw / 2 + 1) * 8 + (double)g.nblocks * g.bh * g.bw * 4;
  }
  // a run's frames count against the wave of its first plane item
  for (const auto& r : d.runs)
    for (int k = 1; k < r.r.ts.count; k++) weight[r.plane] += weight[r.plane + k], weight[r.plane + k] = 0.0;
  std::vector<int> wave(nplanes, 0);
  int w = 0;
  double acc = 0.0;
  for (int p = 0; p < nplanes; p++) {
    // an item whose work is merged into an earlier item's run (weight 0)
    // stays in that item's wave: the run reads the spectra it transforms
    if (budget && weight[p] > 0.0 && acc > 0.0 && acc + weight[p] > (double)budget) {
      w++;
      acc = 0.0;
    }
    wave[p] = w;
    acc += weight[p];
  }
  std::map<std::tuple<int, int, int, int, int>, int> index;
  auto add = [&](int phase, int r, int bw, int bh, int var) {
    const int wv = wave[rec_plane(d, phase, var, r)];
    auto key = std::make_tuple(wv, phase, bw, bh, var);
    auto it = index.find(key);
    int gi;
    if (it == index.end()) {
      gi = (int)plan.groups.size();
      index[key] = gi;
      Group g;
      g.wave = wv;
      g.phase = phase;
      g.bw = bw;
      g.bh = bh;
      g.var = var;
      plan.groups.push_back(g);
    } else {
      gi = it->second;
    }
    Group& g = plan.groups[gi];
    int items;
    if (phase == PH_COPY) items = (int)d.copies[r].height;
    else if (phase == PH_OLA)
      items = var >= fft3d::kOla4Var ? fft3d::batch_items_overlap_add4(rec_geom(d, phase, var, r))
                                     : fft3d::batch_items_overlap_add(rec_geom(d, phase, var, r));
    else if (phase == PH_INV && var >= kRunVar) items = d.runs[r].r.a.g.nblocks;  // one CTA per block
    else items = fft3d::batch_items_forward(rec_geom(d, phase, var, r));
    g.recs.push_back(r);
    g.per.push_back(items);
    g.nitems += items;
  };
  for (int r = 0; r < (int)d.fwd.size(); r++) add(PH_FWD, r, d.fwd[r].a.g.bw, d.fwd[r].a.g.bh, d.fwd[r].bytes);
  for (int r = 0; r < (int)d.inv.size(); r++)
    if (d.inv_in_run.empty() || !d.inv_in_run[r]) add(PH_INV, r, d.inv[r].a.g.bw, d.inv[r].a.g.bh, d.inv[r].mode);
  for (int r = 0; r < (int)d.runs.size(); r++)
    add(PH_INV, r, d.runs[r].r.a.g.bw, d.runs[r].r.a.g.bh, kRunVar + d.runs[r].mode);
  for (int r = 0; r < (int)d.copies.size(); r++) add(PH_COPY, r, 0, 0, 0);
  // overlap-adds: the 4-pixel form for planes that meet its rules
  for (int r = 0; r < (int)d.ola.size(); r++)
    add(PH_OLA, r, 0, 0,
        d.ola[r].bytes + (fft3d::batch_overlap_add4_ok(d.ola[r].a, d.ola[r].bytes) ? fft3d::kOla4Var : 0));
  // waves in order, phases in order within a wave; the larger groups first
  std::stable_sort(plan.groups.begin(), plan.groups.end(), [](const Group& a, const Group& b) {
    if (a.wave != b.wave) return a.wave < b.wave;
    return a.phase != b.phase ? a.phase < b.phase : a.nitems > b.nitems;
  });
  std::string sig;
  size_t off = 0;
  for (auto& g : plan.groups) {
    g.arg_size = arg_size(g.phase, g.var);
    g.args_off = off;
    off = align_up(off + g.arg_size * g.recs.size(), 256);
    sig += std::to_string(g.wave) + "/" + std::to_string(g.phase) + "/" + std::to_string(g.bw) + "x" +
           std::to_string(g.bh) + "/" + std::to_string(g.var) + ":";
    for (int n : g.per) sig += std::to_string(n) + ",";
    sig += ";";
  }
  plan.args_bytes = off;
  for (auto& g : plan.groups) {
    g.items_off = off;
    off = align_up(off + sizeof(int2) * g.nitems, 256);
  }
  plan.items_bytes = off - plan.args_bytes;
  plan.sig = sig;
}

void write_args(const Deferred& d, const Plan& plan, char* base) {
  for (const auto& g : plan.groups) {
    char* p = base + g.args_off;
    for (size_t i = 0; i < g.recs.size(); i++) {
      const int r = g.recs[i];
      if (g.phase == PH_COPY) {
        const fft3d::CopyArgs c = copy_args(d.copies[r]);
        std::memcpy(p + i * g.arg_size, &c, g.arg_size);
        continue;
      }
      const void* src = g.phase == PH_FWD ? (const void*)&d.fwd[r].a
                        : g.phase == PH_INV ? (g.var >= kRunVar ? (const void*)&d.runs[r].r : (const void*)&d.inv[r].a)
                                            : (const void*)&d.ola[r].a;
      std::memcpy(p + i * g.arg_size, src, g.arg_size);
    }
  }
}

void write_items(const Plan& plan, char* base) {  // base: start of the items area
  for (const auto& g : plan.groups) {
    int2* it = reinterpret_cast<int2*>(base + (g.items_off - plan.args_bytes));
    int k = 0;
    if (!g.sched.interleave) {
      for (size_t i = 0; i < g.recs.size(); i++)
        for (int c = 0; c < g.per[i]; c++) it[k++] = make_int2((int)i, c);
    } else {
      const int most = *std::max_element(g.per.begin(), g.per.end());
      for (int c = 0; c < most; c++)
        for (size_t i = 0; i < g.recs.size(); i++)
          if (c < g.per[i]) it[k++] = make_int2((int)i, c);
    }
  }
}

// Algorithmic bytes of one group's launch: what its records must read and
// write at least. Filter/inverse: each distinct window spectrum once (the
// frames of a frame group share theirs), the time-domain blocks written, and
// the Kalman state.
double group_bytes(const Deferred& d, const Group& g) {
  double bytes = 0.0;
  std::vector<const void*> seen;
  for (int r : g.recs) {
    if (g.phase == PH_FWD) {
      const fft3d::Geom& q = d.fwd[r].a.g;
      bytes += (double)q.W * q.H * d.fwd[r].bytes + (double)q.nblocks * q.bh * q.nh * 8;
    } else if (g.phase == PH_INV && g.var >= kRunVar) {
      const fft3d::GroupRun& u = d.runs[r].r;
      const double S = (double)u.a.g.nblocks * u.a.g.bh * u.a.g.nh * 8;
      for (const float2* p : u.ts.spec)
        if (p && std::find(seen.begin(), seen.end(), (const void*)p) == seen.end()) {
          seen.push_back(p);
          bytes += S;
        }
      bytes += (double)u.ts.count * u.a.g.nblocks * u.a.g.bh * u.a.g.bw * 4;
      if (d.runs[r].mode == 0) bytes += 2.0 * S * 2;
    } else if (g.phase == PH_INV) {
      const fft3d::InverseArgs& a = d.inv[r].a;
      const double S = (double)a.g.nblocks * a.g.bh * a.g.nh * 8;
      for (const float2* p : a.in)
        if (p && std::find(seen.begin(), seen.end(), (const void*)p) == seen.end()) {
          seen.push_back(p);
          bytes += S;
        }
      bytes += (double)a.g.nblocks * a.g.bh * a.g.bw * 4;
      if (d.inv[r].mode == 0) bytes += 2.0 * S * 2;
    } else if (g.phase == PH_COPY) {
      bytes += 2.0 * d.copies[r].width * d.copies[r].height;
    } else {
      const fft3d::Geom& q = d.ola[r].a.g;
      bytes += (double)q.nblocks * q.bh * q.bw * 4 + (double)q.W * q.H * d.ola[r].bytes;
    }
  }
  return bytes;
}

// Untuned steps with frame groups take their work items interleaved across
// records, so that the resident CTAs of all frames of a group work on the
// same blocks (and share their window spectra in L2).
void interleave_all(Plan& plan) {
  for (auto& g : plan.groups) g.sched.interleave = 1;
}

void set_grids(fft3d_batch* b, Plan& plan) {
  for (auto& g : plan.groups) {
    const int which = g.phase == PH_FWD ? 0 : g.phase == PH_INV ? (g.var >= kRunVar ? 3 : 1) : g.phase == PH_OLA ? 2 : 4;
    g.occupancy = fft3d::batch_occupancy(g.bw, g.bh, which, g.var);
    const int per_sm = g.sched.per_sm == 0 ? 0 : std::min(g.sched.per_sm, g.occupancy);
    g.grid = per_sm == 0 ? g.nitems : std::max(1, std::min(g.nitems, per_sm * b->sms));
  }
}

cudaError_t launch_group(const Group& g, const char* d_base, cudaStream_t s) {
  fft3d::BatchLaunch l;
  l.args = d_base + g.args_off;
  l.items = reinterpret_cast<const int2*>(d_base + g.items_off);
  l.nitems = g.nitems;
  l.grid = g.grid;
  if (g.phase == PH_FWD) return fft3d::launch_forward_batch(g.bw, g.bh, l, g.var, s);
  if (g.phase == PH_INV && g.var >= kRunVar)
    return fft3d::launch_filter_inverse_group_batch(g.bw, g.bh, l, g.var - kRunVar, s);
  if (g.phase == PH_INV) return fft3d::launch_filter_inverse_batch(g.bw, g.bh, l, g.var, s);
  if (g.phase == PH_COPY) return fft3d::launch_copy_batch(l, s);
  return fft3d::launch_overlap_add_batch(l, g.var, s);
}

cudaError_t run_groups(const Plan& plan, const char* d_base, cudaStream_t s, std::vector<cudaEvent_t>* ev) {
  for (size_t i = 0; i < plan.groups.size(); i++) {
    if (ev) cudaEventRecord((*ev)[2 * i], s);
    cudaError_t e = launch_group(plan.groups[i], d_base, s);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord((*ev)[2 * i + 1], s);
  }
  return cudaSuccess;
}

// A step without a graph: arguments and items through pinned staging.
int run_direct(fft3d_batch* b, Plan& plan, const Deferred& d, cudaStream_t s, std::vector<cudaEvent_t>* ev) {
  const size_t total = plan.args_bytes + plan.items_bytes;
  if (b->direct_done) CK(cudaEventSynchronize(b->direct_done), "batch staging");
  if (total > b->h_direct_cap) {
    if (b->h_direct) cudaFreeHost(b->h_direct);
    b->h_direct = nullptr;
    CK(cudaMallocHost(&b->h_direct, total), "batch staging");
    b->h_direct_cap = total;
  }
  if (total > b->d_direct_cap) {
    if (b->d_direct) {
      cudaStreamSynchronize(s);
      cudaFree(b->d_direct);
    }
    b->d_direct = nullptr;
    CK(cudaMalloc(&b->d_direct, total), "batch arguments");
    b->d_direct_cap = total;
  }
  char* h = static_cast<char*>(b->h_direct);
  write_args(d, plan, h);
  write_items(plan, h + plan.args_bytes);
  CK(cudaMemcpyAsync(b->d_direct, h, total, cudaMemcpyHostToDevice, s), "batch arguments");
  CK(run_groups(plan, static_cast<const char*>(b->d_direct), s, ev), "batched launch");
  if (!b->direct_done) CK(cudaEventCreateWithFlags(&b->direct_done, cudaEventDisableTiming), "batch event");
  CK(cudaEventRecord(b->direct_done, s), "batch event");
  return FFT3D_OK;
}

int capture(fft3d_batch* b, Plan& plan, Captured* c) {
  const size_t total = plan.args_bytes + plan.items_bytes;
  CK(cudaMalloc(&c->d_buf, total), "batch graph buffers");
  std::vector<char> items(plan.items_bytes);
  write_items(plan, items.data());
  CK(cudaMemcpy(static_cast<char*>(c->d_buf) + plan.args_bytes, items.data(), plan.items_bytes,
                cudaMemcpyHostToDevice),
     "batch graph items");
  for (int p = 0; p < 2; p++) {
    CK(cudaMallocHost(&c->h_stage[p], plan.args_bytes), "batch graph staging");
    CK(cudaEventCreateWithFlags(&c->done[p], cudaEventDisableTiming), "batch graph event");
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "batch graph capture");
    cudaError_t e = cudaMemcpyAsync(c->d_buf, c->h_stage[p], plan.args_bytes, cudaMemcpyHostToDevice, b->cap);
    if (e == cudaSuccess) e = run_groups(plan, static_cast<const char*>(c->d_buf), b->cap, nullptr);
    cudaError_t e2 = cudaStreamEndCapture(b->cap, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return cuda_fail(e != cudaSuccess ? e : e2, "batch graph capture");
    }
    e = cudaGraphInstantiate(&c->exec[p], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
  }
  return FFT3D_OK;
}

}  // namespace

extern "C" {

int fft3d_batch_create(int device, fft3d_batch** out) {
  if (!out) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null output handle");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fft3d::engine_fail(FFT3D_E_NOLIB, "neo_fft3d: no CUDA device");
  }
  if (device < 0 || device >= ndev) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: invalid device");
  cudaSetDevice(device);
  auto* b = new fft3d_batch;
  b->device = device;
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return fft3d::engine_fail(FFT3D_E_CUDA, "neo_fft3d: stream creation failed");
  }
  *out = b;
  return FFT3D_OK;
}

void fft3d_batch_destroy(fft3d_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  b->graphs.clear();
  for (auto& p : b->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  if (b->direct_done) cudaEventDestroy(b->direct_done);
  if (b->h_direct) cudaFreeHost(b->h_direct);
  if (b->d_direct) cudaFree(b->d_direct);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
}

int fft3d_batch_set_tuning(fft3d_batch* b, int enable) {
  if (!b) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(b->mu);
  b->tuning = enable ? 1 : 0;
  return FFT3D_OK;
}

int fft3d_batch_step(fft3d_batch* b, int count, fft3d_plane* const* planes, const int* n, const void* const* src,
                     const int* src_stride, void* const* dst, const int* dst_stride, void* stream) {
  if (!b || count <= 0 || !planes || !n || !src || !src_stride || !dst || !dst_stride)
    return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: invalid batch step arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  using Clock = std::chrono::steady_clock;
  const auto t_step = Clock::now();
  struct StepClock {
    double& acc;
    Clock::time_point t0;
    ~StepClock() { acc += std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
  } step_clock{b->stats[7], t_step};
  cudaSetDevice(b->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // A plane may appear several times with consecutive frames (a frame
  // group): n, n + 1, ... in item order. Every plane stays locked until its
  // recorded work is queued.
  std::map<fft3d_plane*, fft3d::FrameGroup> groups;
  for (int i = 0; i < count; i++) {
    auto it = groups.find(planes[i]);
    if (it == groups.end()) {
      groups[planes[i]] = fft3d::FrameGroup{n[i], 1, 0};
      continue;
    }
    fft3d::FrameGroup& g = it->second;
    if (n[i] != g.n0 + g.count)
      return fft3d::engine_fail(FFT3D_E_PARAM,
                                "neo_fft3d: a plane appears twice in one batch step with frames that are not "
                                "consecutive (n, n + 1, ...)");
    if (planes[i] && fft3d::plane_bt(planes[i]) == 0)
      return fft3d::engine_fail(FFT3D_E_PARAM,
                                "neo_fft3d: a Kalman plane (bt = 0) appears twice in one batch step");
    g.count++;
  }
  std::vector<fft3d_plane*> order;
  for (auto& kv : groups) order.push_back(kv.first);
  for (auto* P : order) {
    if (!P) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null plane in batch step");
    if (fft3d::plane_device(P) != b->device)
      return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: batch planes must live on the batch's device");
    const std::string why = fft3d::plane_batchable(P);
    if (!why.empty()) return fft3d::engine_fail(FFT3D_E_UNSUPPORTED, "neo_fft3d: " + why);
  }
  std::vector<std::unique_lock<std::mutex>> locks;
  for (auto* P : order) locks.emplace_back(fft3d::plane_mutex(P));
  bool grouped = false;
  for (auto& kv : groups) grouped = grouped || kv.second.count > 1;
  Deferred d;
  // the frames of a group share one CTA order, alternating from step to step
  const int reverse = (int)((uint64_t)b->stats[0] & 1);
  for (auto& kv : groups) kv.second.reverse = reverse;
  // whatever the step queues on s, fft3d_plane_reset of its planes waits for it
  struct MarkOnExit {
    const std::vector<fft3d_plane*>& planes;
    cudaStream_t s;
    ~MarkOnExit() {
      for (auto* P : planes) fft3d::plane_mark_work(P, s);
    }
  } mark_on_exit{order, s};
  const auto t_plan = Clock::now();
  for (int i = 0; i < count; i++) {
    d.plane = i;
    const fft3d::FrameGroup& g = groups[planes[i]];
    int rc = fft3d::plane_plan(planes[i], n[i], src + 5 * i, src_stride + 5 * i, dst[i], dst_stride[i], s, &d,
                               g.count > 1 ? &g : nullptr);
    if (rc) {
      for (auto* P : order) fft3d::plane_discard(P, d);
      return rc;
    }
  }
  b->stats[3] += std::chrono::duration<double, std::milli>(Clock::now() - t_plan).count();
  // Frame groups: the consecutive filter/inverse records of one plane and
  // mode become runs, each launched with one CTA per block for all its
  // frames (each window spectrum read once per run).
  d.inv_in_run.assign(d.inv.size(), 0);
  for (size_t i = 0; i < d.inv.size();) {
    size_t e = i + 1;
    while (e < d.inv.size() && planes[d.inv[e].plane] == planes[d.inv[i].plane] && d.inv[e].mode == d.inv[i].mode &&
           d.inv[e].plane == d.inv[e - 1].plane + 1 &&
           (int)(e - i) < fft3d::group_run_frames(d.inv[i].a.g.bw, d.inv[i].a.g.bh))
      e++;
    if (e - i >= 2) {
      Deferred::Run run{};
      run.mode = d.inv[i].mode;
      run.plane = d.inv[i].plane;
      run.r.a = d.inv[i].a;
      for (auto& p : run.r.a.in) p = nullptr;
      run.r.ts.count = (int)(e - i);
      for (size_t k = i; k < e; k++) {
        for (int w = 0; w < 5; w++)
          if (d.inv[k].a.in[w]) run.r.ts.spec[(k - i) + w] = d.inv[k].a.in[w];
        run.r.ts.tdom[k - i] = d.inv[k].a.tdom;
        d.inv_in_run[k] = 1;
      }
      d.runs.push_back(run);
    }
    i = e;
  }
  cudaSetDevice(b->device);
  Plan shape;  // the step's shape (one wave) keys its tuning
  build_groups(d, count, 0, shape);
  Tune& t = b->tunes[shape.sig];
  b->stats[0] += 1;
  if (t.budget_ms.empty()) {
    t.budget_ms.assign(kNumBudgets, 0.f);
    b->stats[5] += 1;
    if (!b->tuning) t.stage = 2;
  }
  Plan plan;
  if (t.stage == 0) {
    // tuning, stage 0: the wave budget, default schedules, whole step timed
    build_groups(d, count, kBudgets[t.next], plan);
    if (grouped) interleave_all(plan);
    set_grids(b, plan);
    cudaEvent_t ev[2];
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    cudaEventRecord(ev[0], s);
    int rc = run_direct(b, plan, d, s, nullptr);
    cudaEventRecord(ev[1], s);
    if (rc == FFT3D_OK) {
      cudaError_t e = cudaEventSynchronize(ev[1]);
      if (e != cudaSuccess) rc = cuda_fail(e, "batch tuning");
      else cudaEventElapsedTime(&t.budget_ms[t.next], ev[0], ev[1]);
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (rc) return rc;
    b->stats[2] += 1;
    b->stats[4] = (double)plan.groups.size();
    fft3d::count_launches(plan.groups.size());
    if (++t.next == kNumBudgets) {
      t.budget = kBudgets[std::min_element(t.budget_ms.begin(), t.budget_ms.end()) - t.budget_ms.begin()];
      t.stage = 1;
      t.next = 0;
    }
    return FFT3D_OK;
  }
  build_groups(d, count, t.budget, plan);
  b->stats[4] = (double)plan.groups.size();
  fft3d::count_launches(plan.groups.size());
  if (t.stage == 1) {
    // tuning, stage 1: one schedule candidate for every launch, each launch timed
    if (t.ms.empty()) t.ms.assign(plan.groups.size(), std::vector<float>(kNumCand, 0.f));
    for (auto& g : plan.groups) g.sched = kCandidates[t.next];
    set_grids(b, plan);
    std::vector<cudaEvent_t> ev(2 * plan.groups.size());
    for (auto& e : ev) cudaEventCreate(&e);
    int rc = run_direct(b, plan, d, s, &ev);
    if (rc == FFT3D_OK) {
      cudaError_t e = cudaEventSynchronize(ev.back());
      if (e != cudaSuccess) rc = cuda_fail(e, "batch tuning");
    }
    if (rc == FFT3D_OK)
      for (size_t gi = 0; gi < plan.groups.size(); gi++)
        cudaEventElapsedTime(&t.ms[gi][t.next], ev[2 * gi], ev[2 * gi + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    b->stats[2] += 1;
    if (++t.next == kNumCand) {
      t.best.resize(plan.groups.size());
      for (size_t gi = 0; gi < plan.groups.size(); gi++) {
        const auto& m = t.ms[gi];
        t.best[gi] = kCandidates[std::min_element(m.begin(), m.end()) - m.begin()];
      }
      t.stage = 2;
    }
    return FFT3D_OK;
  }
  if (t.best.size() == plan.groups.size()) {
    for (size_t gi = 0; gi < plan.groups.size(); gi++) plan.groups[gi].sched = t.best[gi];
  } else if (grouped) {
    interleave_all(plan);
  }
  set_grids(b, plan);
  b->stats[6] = (double)(t.budget >> 20);
  if (b->timing) {
    std::vector<cudaEvent_t> ev(2 * plan.groups.size());
    for (auto& e : ev) CK(cudaEventCreate(&e), "batch timing event");
    int rc = run_direct(b, plan, d, s, &ev);
    for (size_t gi = 0; gi < plan.groups.size(); gi++)
      b->pending.push_back({plan.groups[gi].phase, group_bytes(d, plan.groups[gi]), ev[2 * gi], ev[2 * gi + 1]});
    return rc;
  }
  auto& slot = b->graphs[plan.sig];
  if (!slot) {
    slot.reset(new Captured);
    int rc = capture(b, plan, slot.get());
    if (rc) {
      slot.reset();
      b->graphs.erase(plan.sig);
      return rc;
    }
  }
  Captured* c = slot.get();
  const int p = c->parity;
  if (c->used[p]) CK(cudaEventSynchronize(c->done[p]), "batch graph staging");
  write_args(d, plan, static_cast<char*>(c->h_stage[p]));
  CK(cudaGraphLaunch(c->exec[p], s), "batch graph launch");
  CK(cudaEventRecord(c->done[p], s), "batch graph event");
  c->used[p] = true;
  c->parity ^= 1;
  b->stats[1] += 1;
  return FFT3D_OK;
}

int fft3d_batch_set_timing(fft3d_batch* b, int enable) {
  if (!b) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null handle");
  std::lock_guard<std::mutex> lk(b->mu);
  b->timing = enable != 0;
  return FFT3D_OK;
}

int fft3d_batch_timing(fft3d_batch* b, double out[12]) {
  if (!b || !out) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  int rc = FFT3D_OK;
  for (auto& p : b->pending) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(p.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p.a, p.b);
    if (e != cudaSuccess && rc == FFT3D_OK) rc = cuda_fail(e, "batch timing");
    b->t_phase[p.phase][0] += 1;
    b->t_phase[p.phase][1] += ms;
    b->t_phase[p.phase][2] += p.bytes;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  b->pending.clear();
  for (int ph = 0; ph < 4; ph++)
    for (int k = 0; k < 3; k++) out[3 * ph + k] = b->t_phase[ph][k];
  return rc;
}

int fft3d_batch_stats(fft3d_batch* b, double out[8]) {
  if (!b || !out) return fft3d::engine_fail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  std::lock_guard<std::mutex> lk(b->mu);
  std::copy(b->stats, b->stats + 8, out);
  return FFT3D_OK;
}

}  // extern "C"
