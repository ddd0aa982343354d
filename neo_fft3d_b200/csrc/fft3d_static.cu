// Allocation-free entry point: fft3d_filter2d_static (include/fft3d_b200.h).
//
// Filters ONE frame of one plane with the spatial modes of the filter (bt = 1
// Wiener with sharpen/dehalo, or bt = -1 sharpen/dehalo only). Everything the
// call needs beyond the caller's input and output planes -- the plane's
// tables, the frame's spectrum and its inverse-transformed blocks -- lives in
// one file-scope device array of fixed size, so the call never allocates or
// frees device memory. It is meant for callers that cannot do that at frame
// time: applications whose device memory is entirely owned by their own pool
// allocator, and real-time pipelines that must not risk the implicit device
// synchronisation and latency of cudaMalloc/cudaFree once they are running.
//
// Limits and sharing rules:
//  * the array holds kStaticScratchBytes (32 MiB) on every GPU that loads this
//    library, until the process exits; a plane whose tables + spectrum +
//    time-domain blocks need more is rejected with FFT3D_E_UNSUPPORTED
//    (e.g. 720p luma and 1080p chroma with bw=bh=32, ow=oh=16 fit;
//    1080p luma does not: use fft3d_plane_filter_device for it);
//  * all calls on a device share the array, and it keeps whatever the last
//    call left there; nothing has to start at zero because each call writes
//    every byte it later reads. Calls whose GPU work overlaps (different
//    streams, or other host threads) race on the array: order them on one
//    stream, or wait for one before issuing the next;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) and uploads the FFT twiddle tables; make that
//    first call before any stream capture. Later calls only launch kernels on
//    the caller's stream (the plane's tables go up as kernel parameters), so
//    they never wait on the stream from the host;
//  * the address and the twiddle tables are kept per device number for the
//    life of the process: do not use the call across a cudaDeviceReset of a
//    device it has run on (they would belong to the destroyed context).
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "fft3d_b200.h"
#include "fft3d_kernels.cuh"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_lock;
std::vector<std::pair<int, void*>> g_static_base;  // device -> address of g_static_scratch

// failures are reported through fft3d_last_error(), like every other call
int sfail(int code, const std::string& msg) {
  fft3d::set_last_error(msg);
  return code;
}

// Device address of the scratch array on `dev` (the current device); the first
// call per device resolves it and uploads the twiddle tables.
int static_base(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_static_lock);
  for (auto& e : g_static_base)
    if (e.first == dev) {
      *out = e.second;
      return FFT3D_OK;
    }
  void* ptr = nullptr;
  cudaError_t err = cudaGetSymbolAddress(&ptr, g_static_scratch);
  if (err != cudaSuccess)
    return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(err));
  err = fft3d::upload_twiddles();
  if (err != cudaSuccess)
    return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: twiddle upload: ") + cudaGetErrorString(err));
  g_static_base.emplace_back(dev, ptr);
  *out = ptr;
  return FFT3D_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// The plane's tables travel to the scratch array as the launch parameters of a
// copy kernel: the launch takes them by value, so the call keeps no host
// buffer alive, never waits on the stream from the host (a cudaMemcpyAsync
// from pageable memory would), and the upload is ordered on the caller's
// stream like the kernels that read it. The largest table set (48x48 blocks)
// is 5248 floats; kernel parameters may take up to 32 KB.
constexpr int kStaticTableFloats = 7168;
struct StaticTableBlob {
  float v[kStaticTableFloats];
};

// dst[0 .. n) = blob, then dst[n .. n + zeros) = 0 (the unused pattern tables)
__global__ void k_static_tables(const __grid_constant__ StaticTableBlob b, int n, int zeros, float* dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + zeros; i += gridDim.x * blockDim.x)
    dst[i] = i < n ? b.v[i] : 0.f;
}

}  // namespace

extern "C" int fft3d_filter2d_static(const fft3d_params* p0, const fft3d_plane_desc* d, const void* src,
                                     int src_stride, void* dst, int dst_stride, void* stream) {
  if (!p0 || !d || !src || !dst) return sfail(FFT3D_E_PARAM, "neo_fft3d: null argument");
  fft3d_params ep = *p0;
  if (ep.bt != 1 && ep.bt != -1)
    return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: the allocation-free call filters single frames (bt = 1 or -1)");
  if (ep.pfactor != 0 || ep.sigma2 != ep.sigma || ep.sigma3 != ep.sigma || ep.sigma4 != ep.sigma)
    return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: noise patterns need fft3d_plane_create");
  if (ep.interlaced) return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: interlaced planes need fft3d_plane_create");
  if (d->bits < 8 || (d->bits > 16 && d->bits != 32)) return sfail(FFT3D_E_PARAM, "neo_fft3d: unsupported bit depth");
  const int bytes = d->bits <= 8 ? 1 : (d->bits <= 16 ? 2 : 4);
  const float factor = bytes == 1 ? 1.0f : (bytes == 2 ? float(1 << (d->bits - 8)) : 1 / 255.0f);
  ep.sigma *= factor;
  ep.smin *= factor;
  ep.smax *= factor;
  if (ep.ow * 2 > ep.bw) return sfail(FFT3D_E_PARAM, "ow must be less than bw / 2");
  if (ep.oh * 2 > ep.bh) return sfail(FFT3D_E_PARAM, "oh must be less than bh / 2");
  if (ep.ow < 0) ep.ow = ep.bw / 3;
  if (ep.oh < 0) ep.oh = ep.bh / 3;
  if (ep.beta < 1) return sfail(FFT3D_E_PARAM, "beta must be not less 1.0");
  if (!fft3d::block_size_supported(ep.bw, ep.bh))
    return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: block size not built into this library");
  const int l = d->is_chroma ? (ep.l >> d->ssw) : ep.l, r = d->is_chroma ? (ep.r >> d->ssw) : ep.r;
  const int t = d->is_chroma ? (ep.t >> d->ssh) : ep.t, b = d->is_chroma ? (ep.b >> d->ssh) : ep.b;
  fft3d::Geom g{};
  g.W = d->width - l - r;
  g.H = d->height - t - b;
  if (g.W <= 0) return sfail(FFT3D_E_PARAM, "Width cannot be cropped to zero or below");
  if (g.H <= 0) return sfail(FFT3D_E_PARAM, "Height cannot be cropped to zero or below");
  g.bw = ep.bw; g.bh = ep.bh; g.ow = ep.ow; g.oh = ep.oh;
  g.sx = ep.bw - ep.ow; g.sy = ep.bh - ep.oh;
  g.nox = (g.W - ep.ow + (ep.bw - ep.ow - 1)) / (ep.bw - ep.ow) + 2;
  g.noy = (g.H - ep.oh + (ep.bh - ep.oh - 1)) / (ep.bh - ep.oh) + 2;
  g.nblocks = g.nox * g.noy;
  g.nh = ep.bw / 2 + 1;
  g.interlaced = 0;
  const int bw = ep.bw, bh = ep.bh, nh = g.nh, nb = bh * nh;

  // host tables (the reference constructor's formulas, as in fft3d_plane_create)
  const float pi = 3.1415926535897932384626433832795f;
  auto win = [&](int o, std::vector<float>& an_l, std::vector<float>& an_r, std::vector<float>& sy_l,
                 std::vector<float>& sy_r) {
    an_l.assign(std::max(o, 1), 1.f); an_r.assign(std::max(o, 1), 1.f);
    sy_l.assign(std::max(o, 1), 1.f); sy_r.assign(std::max(o, 1), 1.f);
    for (int i = 0; i < o; i++) {
      float cl = cosf(pi * (i - o + 0.5f) / (o * 2)), cr = cosf(pi * (i + 0.5f) / (o * 2));
      if (ep.wintype == 0) { an_l[i] = cl; an_r[i] = cr; sy_l[i] = cl; sy_r[i] = cr; }
      else if (ep.wintype == 1) {
        an_l[i] = (float)std::sqrt((double)cl); an_r[i] = (float)std::sqrt((double)cr);
        sy_l[i] = an_l[i] * an_l[i] * an_l[i]; sy_r[i] = an_r[i] * an_r[i] * an_r[i];
      } else { sy_l[i] = cl * cl; sy_r[i] = cr * cr; }
    }
  };
  std::vector<float> axl, axr, sxl, sxr, ayl, ayr, syl, syr;
  win(ep.ow, axl, axr, sxl, sxr);
  win(ep.oh, ayl, ayr, syl, syr);
  std::vector<float> wx(bw, 1.f), wy(bh, 1.f);
  for (int i = 0; i < ep.ow; i++) { wx[i] = axl[i]; wx[bw - ep.ow + i] = axr[i]; }
  for (int i = 0; i < ep.oh; i++) { wy[i] = ayl[i]; wy[bh - ep.oh + i] = ayr[i]; }
  std::vector<float> grid((size_t)nb * 2), wsh(nb), wdh(nb);
  {
    const double maxv = bytes == 1 ? 255.0 : (bytes == 2 ? (double)((1 << d->bits) - 1) : 1.0);
    std::vector<double> xr(nh), xi(nh), yr(bh), yi(bh);
    for (int k = 0; k < nh; k++) {
      double sr = 0, si = 0;
      for (int x = 0; x < bw; x++) {
        double a = -2.0 * M_PI * (double)((long)k * x % bw) / bw;
        sr += wx[x] * std::cos(a); si += wx[x] * std::sin(a);
      }
      xr[k] = sr; xi[k] = si;
    }
    for (int h = 0; h < bh; h++) {
      double sr = 0, si = 0;
      for (int y = 0; y < bh; y++) {
        double a = -2.0 * M_PI * (double)((long)h * y % bh) / bh;
        sr += wy[y] * std::cos(a); si += wy[y] * std::sin(a);
      }
      yr[h] = sr; yi[h] = si;
    }
    for (int h = 0; h < bh; h++)
      for (int k = 0; k < nh; k++) {
        grid[2 * (h * nh + k)] = (float)(maxv * (yr[h] * xr[k] - yi[h] * xi[k]));
        grid[2 * (h * nh + k) + 1] = (float)(maxv * (yr[h] * xi[k] + yi[h] * xr[k]));
      }
    float wmax = 0;
    for (int j = 0; j < bh; j++) {
      int dj = j >= bh / 2 ? bh - j : j;
      float d2v = float(dj * dj) * (ep.svr * ep.svr) / ((bh / 2) * (bh / 2));
      for (int i = 0; i < nh; i++) {
        float d2 = d2v + float(i * i) / ((bw / 2) * (bw / 2));
        wsh[j * nh + i] = (float)(1 - std::exp((double)(-d2 / (2 * ep.scutoff * ep.scutoff))));
        float dh = (float)(std::exp((double)(-0.7f * d2 * ep.hr * ep.hr)) - std::exp((double)(-d2 * ep.hr * ep.hr)));
        wdh[j * nh + i] = dh;
        if (dh > wmax) wmax = dh;
      }
    }
    for (auto& v : wdh) v /= wmax;
  }
  // scratch layout: tables | spectrum | time-domain blocks
  std::vector<float> blob;
  auto put = [&](const std::vector<float>& v) {
    size_t off = blob.size();
    blob.insert(blob.end(), v.begin(), v.end());
    while (blob.size() % 64) blob.push_back(0.f);
    return off;
  };
  const size_t o_wx = put(wx), o_wy = put(wy), o_sxl = put(sxl), o_sxr = put(sxr), o_syl = put(syl),
               o_syr = put(syr), o_grid = put(grid), o_wsh = put(wsh), o_wdh = put(wdh);
  const size_t o_pat = blob.size();  // nb zeros, written by the table kernel
  if (blob.size() > (size_t)kStaticTableFloats)
    return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: the allocation-free call's tables exceed its launch parameters");
  const size_t tables_bytes = align256((o_pat + nb) * sizeof(float));
  const size_t spec_bytes = align256((size_t)g.nblocks * nb * sizeof(float2));
  const size_t tdom_bytes = align256((size_t)g.nblocks * bh * bw * sizeof(float));
  const size_t need = tables_bytes + spec_bytes + tdom_bytes;
  if (need > kStaticScratchBytes)
    return sfail(FFT3D_E_UNSUPPORTED, "neo_fft3d: this plane needs " + std::to_string(need) +
                                          " bytes of scratch; the allocation-free call has " +
                                          std::to_string(kStaticScratchBytes) + " (use fft3d_plane_filter_device)");
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return sfail(FFT3D_E_NOLIB, std::string("neo_fft3d: ") + cudaGetErrorString(err));
  void* base = nullptr;
  int rc = static_base(dev, &base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* B = static_cast<char*>(base);
  {
    StaticTableBlob tb;
    std::memcpy(tb.v, blob.data(), blob.size() * sizeof(float));
    k_static_tables<<<8, 256, 0, st>>>(tb, (int)blob.size(), nb, reinterpret_cast<float*>(B));
    err = cudaGetLastError();
    if (err != cudaSuccess)
      return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: table upload: ") + cudaGetErrorString(err));
  }
  const float* T = reinterpret_cast<const float*>(B);
  float2* spec = reinterpret_cast<float2*>(B + tables_bytes);
  float* tdom = reinterpret_cast<float*>(B + tables_bytes + spec_bytes);
  fft3d::Tables tab{};
  tab.wan_x = T + o_wx; tab.wan_y = T + o_wy;
  tab.wsyn_xl = T + o_sxl; tab.wsyn_xr = T + o_sxr; tab.wsyn_yl = T + o_syl; tab.wsyn_yr = T + o_syr;
  tab.grid = reinterpret_cast<const float2*>(T + o_grid);
  tab.wsharpen = T + o_wsh; tab.wdehalo = T + o_wdh; tab.pattern2d = T + o_pat; tab.pattern3d = T + o_pat;
  const bool ints = bytes != 4;
  const float base_val = (ints && d->is_chroma) ? (float)(1 << (d->bits - 1)) : 0.f;
  const float norm = 1.0f / (ep.bw * ep.bh);

  fft3d::ForwardArgs fa;
  fa.g = g;
  fa.src = static_cast<const char*>(src) + (long long)t * src_stride + (long long)l * bytes;
  fa.src_stride = src_stride;
  fa.base = base_val;
  fa.wan_x = tab.wan_x;
  fa.wan_y = tab.wan_y;
  fa.spec = spec;
  fa.err = nullptr;
  for (int x = 0; x < fft3d::kMaxBw; x++) fa.wx[x] = x < ep.bw ? blob[o_wx + x] : 0.f;
  err = fft3d::launch_forward(fa, bytes, st);
  if (err != cudaSuccess) return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: forward kernel: ") + cudaGetErrorString(err));

  fft3d::InverseArgs ia{};
  ia.g = g;
  ia.t = tab;
  ia.in[2] = spec;
  fft3d::FilterConsts& c = ia.c;
  const int mode = ep.bt;  // 1: Wiener 2D, -1: sharpen only
  c.sigma2n = 1 * ep.sigma * ep.sigma / norm;
  c.sigma2n_2d = ep.sigma * ep.sigma / norm;
  c.lowlimit = (ep.beta - 1) / ep.beta;
  c.degrid = ep.degrid;
  c.sharpen = ep.sharpen;
  c.dehalo = ep.dehalo;
  c.smin2n = ep.smin * ep.smin / norm;
  c.smax2n = ep.smax * ep.smax / norm;
  c.ht2n = ep.ht * ep.ht / norm;
  c.kratio2 = ep.kratio * ep.kratio;
  c.pattern = 0;
  c.use_sharpen = ep.sharpen != 0;
  c.use_dehalo = ep.dehalo != 0;
  c.fuse_sharpen = mode == 1 ? 1 : 0;
  c.do_sharpen = ((ep.sharpen != 0 || ep.dehalo != 0) && mode != 1) ? 1 : 0;
  ia.tdom = tdom;
  ia.reverse = 0;
  err = fft3d::launch_filter_inverse(ia, mode, st);
  if (err != cudaSuccess) return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: filter kernel: ") + cudaGetErrorString(err));

  if (ep.l > 0 || ep.t > 0 || ep.r > 0 || ep.b > 0) {  // crop borders come from the source
    err = cudaMemcpy2DAsync(dst, dst_stride, src, src_stride, (size_t)d->width * bytes, d->height,
                            cudaMemcpyDeviceToDevice, st);
    if (err != cudaSuccess) return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: border copy: ") + cudaGetErrorString(err));
  }
  fft3d::OlaArgs oa;
  oa.g = g;
  oa.t = tab;
  oa.tdom = tdom;
  oa.dst = static_cast<char*>(dst) + (long long)t * dst_stride + (long long)l * bytes;
  oa.dst_stride = dst_stride;
  oa.norm = norm;
  oa.rounder = ints ? 0.5f : 0.f;
  oa.base = base_val;
  oa.maxval = bytes == 1 ? 255 : (bytes == 2 ? (1 << d->bits) - 1 : 0);  // float: clamp to [0, 1]
  oa.err = nullptr;
  err = fft3d::launch_overlap_add(oa, bytes, st);
  if (err != cudaSuccess) return sfail(FFT3D_E_CUDA, std::string("neo_fft3d: overlap-add kernel: ") + cudaGetErrorString(err));
  return FFT3D_OK;
}
