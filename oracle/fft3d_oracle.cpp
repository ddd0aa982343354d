// CPU restatement of the neo_fft3d per-plane pipeline — THE ORACLE.
//
// TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the CPU-baseline leg of
// bench.py call it as the checker; the product (neo_fft3d_b200) never links or
// calls it.
//
// It restates, per plane, what the reference's FFT3DEngine does
// (src/fft3d_engine.h:87-734) with the kernels of the reference's C path
// (opt=1): src/buffer.cpp (FrameToCover/CoverToOverlap/OverlapToCover/
// CoverToFrame), src/code_impl/Apply.cpp, Kalman.cpp, Sharpen.cpp,
// code_impl_C.h and src/helper.cpp. Each function cites the lines it follows.
//
// Two instantiations:
//   * R = float: every float expression keeps the reference's operand order and
//     its float/double promotions (glibc exp/sqrt of a float argument are the
//     double functions there), so with the same FFT (o_fft.hpp, which is also
//     what the FFTW-API shim runs) it reproduces the reference plugin bit for
//     bit; tests pin this against the reference built from its own sources.
//   * R = double: the same pipeline in FP64 (tables, FFT, filter, overlap-add);
//     the error of every float implementation is stated against it.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fft3d_b200.h"
#include "o_fft.hpp"

namespace {

template <typename R>
struct Plane {
  fft3d_params ep;
  fft3d_plane_desc d;
  int bytes = 1;        // bytes per sample
  int bw, bh, ow, oh, bt;
  int nox, noy, coverw, coverh, mirw, mirh, outwidth, nblocks;
  int l = 0, t = 0, r = 0, b = 0, width = 0, height = 0;  // crop (plane units) and cropped size
  std::vector<R> wanxl, wanxr, wanyl, wanyr, wsynxl, wsynxr, wsynyl, wsynyr;
  std::vector<R> wsharpen, wdehalo, pattern2d, pattern3d, pwin;
  std::vector<R> gridsample;  // bh x outwidth complex (interleaved)
  bool pattern = false, pattern_set = false, pattern3d_init = false;
  R norm, sigma2n, smin2n, smax2n, ht2n, kratio2;
  std::vector<R> outLast, covar, covarProcess;  // Kalman state, complex interleaved
  std::unique_ptr<offt::Block2D<R>> fft;
  std::vector<R> cover;                            // coverh x coverw (pixel values as R)
  std::vector<R> in;                               // blocks x bh x bw
  std::vector<R> outrez;                           // blocks x bh x outwidth complex
  std::map<int, std::vector<R>> cache;             // frame -> spectrum
  std::list<int> lru;
  R sigma2n_cur = 0;                               // btcur * sigma^2 / norm of the current call
  std::vector<R> last_filtered;                    // spectrum sent to the last inverse transform

  size_t spec_size() const { return (size_t)nblocks * bh * outwidth * 2; }
};

// ---------------------------------------------------------------- set-up
// src/fft3d_engine.h:87-408

template <typename R>
R cos_window(int i, int o);
template <>
float cos_window<float>(int i, int o) {
  // src/fft3d_engine.h:207,214-215: float pi, float argument, cosf
  const float pi = 3.1415926535897932384626433832795f;
  return cosf(pi * (i - o + 0.5f) / (o * 2));
}
template <>
double cos_window<double>(int i, int o) { return std::cos(M_PI * (i - o + 0.5) / (o * 2.0)); }
template <typename R>
R cos_window_r(int i, int o);
template <>
float cos_window_r<float>(int i, int o) {
  const float pi = 3.1415926535897932384626433832795f;
  return cosf(pi * (i + 0.5f) / (o * 2));
}
template <>
double cos_window_r<double>(int i, int o) { return std::cos(M_PI * (i + 0.5) / (o * 2.0)); }

template <typename R>
void make_windows(Plane<R>& P, int o, std::vector<R>& anl, std::vector<R>& anr, std::vector<R>& snl,
                  std::vector<R>& snr) {
  // src/fft3d_engine.h:204-283 (wintype 0, 1, 2)
  anl.assign(o, 1); anr.assign(o, 1); snl.assign(o, 1); snr.assign(o, 1);
  for (int i = 0; i < o; i++) {
    R cl = cos_window<R>(i, o), cr = cos_window_r<R>(i, o);
    if (P.ep.wintype == 0) {
      anl[i] = cl; anr[i] = cr; snl[i] = cl; snr[i] = cr;
    } else if (P.ep.wintype == 1) {
      anl[i] = (R)std::sqrt((double)cl); anr[i] = (R)std::sqrt((double)cr);
      snl[i] = anl[i] * anl[i] * anl[i]; snr[i] = anr[i] * anr[i] * anr[i];
    } else {
      anl[i] = 1; anr[i] = 1;
      snl[i] = cl * cl; snr[i] = cr * cr;
    }
  }
}

// Block pixel value for block (bx, by), pixel (x, y), from the cover, with the
// analysis window. The product order of the reference depends on the region
// (src/buffer.cpp:137-378): rows and columns are "edge" (outer half of the
// first/last block row/column), "overlap" (shared with a neighbour) or
// "plain"; see the table in the body.
template <typename R>
R windowed(const Plane<R>& P, R v, int bx, int by, int x, int y) {
  const int bw = P.bw, bh = P.bh, ow = P.ow, oh = P.oh;
  // y class: 0 plain, 1 edge, 2 overlap
  int yc = 0, xc = 0;
  R wy = 1, wx = 1;
  if (y < oh) { wy = P.wanyl[y]; yc = (by == 0) ? 1 : 2; }
  else if (y >= bh - oh) { wy = P.wanyr[y - (bh - oh)]; yc = (by == P.noy - 1) ? 1 : 2; }
  if (x < ow) { wx = P.wanxl[x]; xc = (bx == 0) ? 1 : 2; }
  else if (x >= bw - ow) { wx = P.wanxr[x - (bw - ow)]; xc = (bx == P.nox - 1) ? 1 : 2; }
  if (yc == 0) return xc == 0 ? v : wx * v;                    // :183,187,196-197,204
  if (yc == 1) {
    if (xc == 1) return (wx * wy) * v;                          // :144,172,339,369
    if (xc == 2) return (wy * v) * wx;                          // :156-158,353-355
    return wy * v;                                              // :148,165,344,362
  }
  if (xc == 1) return (wx * v) * wy;                            // :235-237,271-273
  if (xc == 2) return (v * wx) * wy;                            // :252-255
  return v * wy;                                                // :241-243,262-264
}

template <typename R>
void cover_to_blocks(Plane<R>& P, const std::vector<R>& cov, bool chroma_base) {
  // src/buffer.cpp:119-379 (block (bx,by) pixel (x,y) <- cover[by*(bh-oh)+y][bx*(bw-ow)+x])
  R base = 0;
  if (P.bytes != 4 && chroma_base) base = (R)(1 << (P.d.bits - 1));
  for (int by = 0; by < P.noy; by++)
    for (int bx = 0; bx < P.nox; bx++) {
      R* blk = P.in.data() + ((size_t)by * P.nox + bx) * P.bh * P.bw;
      for (int y = 0; y < P.bh; y++)
        for (int x = 0; x < P.bw; x++) {
          R v = cov[(size_t)(by * (P.bh - P.oh) + y) * P.coverw + bx * (P.bw - P.ow) + x] - base;
          blk[y * P.bw + x] = windowed(P, v, bx, by, x, y);
        }
    }
}

template <typename R>
void make_tables(Plane<R>& P) {
  const fft3d_params& ep = P.ep;
  const int bw = P.bw, bh = P.bh, ow_ = P.outwidth;
  // wsharpen, wdehalo: src/fft3d_engine.h:285-327 (exp of a float argument is
  // the double function; the result is stored as float)
  P.wsharpen.assign((size_t)bh * ow_, 0);
  P.wdehalo.assign((size_t)bh * ow_, 0);
  R wmax = 0;
  for (int j = 0; j < bh; j++) {
    int dj = j >= bh / 2 ? bh - j : j;
    R d2v = R(dj * dj) * (ep.svr * ep.svr) / ((bh / 2) * (bh / 2));
    for (int i = 0; i < ow_; i++) {
      R d2 = d2v + R(i * i) / ((bw / 2) * (bw / 2));
      P.wsharpen[j * ow_ + i] = (R)(1 - std::exp((double)(-d2 / (2 * ep.scutoff * ep.scutoff))));
      R hr = (R)ep.hr;
      R dh = (R)(std::exp((double)((R)(-0.7f) * d2 * hr * hr)) - std::exp((double)(-d2 * hr * hr)));
      P.wdehalo[j * ow_ + i] = dh;
      if (dh > wmax) wmax = dh;
    }
  }
  for (auto& v : P.wdehalo) v /= wmax;
  // normalisation and normed constants: src/fft3d_engine.h:329-336
  P.norm = (R)1 / (R)(bw * bh);
  P.sigma2n = (R)ep.sigma * (R)ep.sigma / P.norm;
  P.smin2n = (R)ep.smin * (R)ep.smin / P.norm;
  P.smax2n = (R)ep.smax * (R)ep.smax / P.norm;
  P.ht2n = (R)ep.ht * (R)ep.ht / P.norm;
  P.kratio2 = (R)ep.kratio * (R)ep.kratio;
  // pattern window: src/fft3d_engine.h:346-361
  P.pwin.assign((size_t)bh * ow_, 0);
  for (int j = 0; j < bh; j++) {
    int dj = std::min(j, bh - j);
    R fh = dj * (R)2 / bh;
    R fh2 = fh * fh;
    for (int i = 0; i < ow_; i++) {
      R fw2 = (i * (R)2 / bw) * (i * (R)2 / bw);
      P.pwin[j * ow_ + i] = (fh2 + fw2) / (fh2 + fw2 + (R)ep.pcutoff * (R)ep.pcutoff);
    }
  }
  // sigmas -> pattern: src/fft3d_engine.h:366-375, src/helper.cpp:14-43
  P.pattern2d.assign((size_t)bh * ow_, 0);
  P.pattern3d.assign((size_t)bh * ow_, 0);
  if ((ep.sigma2 != ep.sigma || ep.sigma3 != ep.sigma || ep.sigma4 != ep.sigma) && ep.pfactor == 0) {
    R ft2 = (R)(std::sqrt((double)(R)0.5) / 2), ft3 = (R)(std::sqrt((double)(R)0.5) / 4);
    for (int h = 0; h < bh; h++)
      for (int w = 0; w < ow_; w++) {
        R fy = (bh - (R)2 * std::abs(h - bh / 2)) / bh;
        R fx = (w * (R)1) / ow_;
        R f = (R)std::sqrt((double)((fx * fx + fy * fy) * (R)0.5));
        R s;
        if (f < ft3) s = (R)ep.sigma4 + ((R)ep.sigma3 - (R)ep.sigma4) * f / ft3;
        else if (f < ft2) s = (R)ep.sigma3 + ((R)ep.sigma2 - (R)ep.sigma3) * (f - ft3) / (ft2 - ft3);
        else s = (R)ep.sigma + ((R)ep.sigma2 - (R)ep.sigma) * (1 - f) / (1 - ft2);
        P.pattern2d[h * ow_ + w] = s * s / P.norm;
      }
    P.pattern_set = true;
    P.ep.pfactor = 1;
  }
  P.pattern = P.ep.pfactor != 0;
}

template <typename R>
void make_gridsample(Plane<R>& P) {
  // src/fft3d_engine.h:380-404: r2c of block (0,0) of a cover filled with the
  // maximum sample value, gathered without the chroma offset.
  R maxv = P.bytes == 1 ? (R)255 : (P.bytes == 2 ? (R)((1 << P.d.bits) - 1) : (R)1);
  std::vector<R> blk((size_t)P.bh * P.bw);
  for (int y = 0; y < P.bh; y++)
    for (int x = 0; x < P.bw; x++) blk[y * P.bw + x] = windowed(P, maxv, 0, 0, x, y);
  P.gridsample.assign((size_t)P.bh * P.outwidth * 2, 0);
  P.fft->r2c(blk.data(), P.bw, P.gridsample.data(), P.outwidth);
}

// ---------------------------------------------------------------- frame I/O

template <typename R>
R load_px(const Plane<R>& P, const uint8_t* row, int x) {
  if (P.bytes == 1) return (R)(int)row[x];
  if (P.bytes == 2) return (R)(int)((const uint16_t*)row)[x];
  return (R)((const float*)row)[x];
}

// src/buffer.cpp:6-81: crop-reduced plane into the cover at (mirw, mirh),
// reflect-101 borders (rows mirrored after the columns).
template <typename R>
void frame_to_cover(Plane<R>& P, const uint8_t* src, int stride) {
  const uint8_t* base = src + (size_t)P.t * stride + (size_t)P.l * P.bytes;
  const int W = P.width, H = P.height, cw = P.coverw;
  // source row for cover row mirh + k; interlaced (even H): field 1 (rows
  // 0, 2, ..) then field 2 bottom-up (rows H-1, H-3, ..), src/buffer.cpp:31-63
  auto src_row = [&](int k) -> const uint8_t* {
    if (!P.ep.interlaced) return base + (size_t)k * stride;
    int half = H / 2;
    int row = k < half ? 2 * k : H - 1 - 2 * (k - half);
    return base + (size_t)row * stride;
  };
  for (int k = 0; k < H; k++) {
    R* c = P.cover.data() + (size_t)(P.mirh + k) * cw;
    const uint8_t* s = src_row(k);
    for (int x = 0; x < W; x++) c[P.mirw + x] = load_px(P, s, x);
    for (int w = 0; w < P.mirw; w++) c[w] = c[2 * P.mirw - w];
    int width2 = 2 * W + 2 * P.mirw - 2;
    for (int w = W + P.mirw; w < cw; w++) c[w] = c[width2 - w];
  }
  for (int y = H + P.mirh; y < P.coverh; y++)
    std::memcpy(&P.cover[(size_t)y * cw], &P.cover[(size_t)(2 * (H + P.mirh - 1) - y) * cw], sizeof(R) * cw);
  for (int y = 0; y < P.mirh; y++)
    std::memcpy(&P.cover[(size_t)y * cw], &P.cover[(size_t)(2 * P.mirh - y) * cw], sizeof(R) * cw);
}

// float -> integer sample as the reference does: truncation toward zero of
// v, then clamp (src/buffer.cpp:392-397,406)
template <typename R>
void store_px(const Plane<R>& P, uint8_t* row, int x, R v) {
  if (P.bytes == 4) {
    R c = v < 0 ? 0 : v;
    ((float*)row)[x] = (float)(c > 1 ? 1 : c);
    return;
  }
  long long iv = (long long)v;  // C cast truncates toward zero
  long long mx = (1LL << P.d.bits) - 1;
  if (P.bytes == 1) mx = 255;
  if (iv < 0) iv = 0;
  if (iv > mx) iv = mx;
  if (P.bytes == 1) row[x] = (uint8_t)iv;
  else ((uint16_t*)row)[x] = (uint16_t)iv;
}

// src/buffer.cpp:382-560: overlap-add of the inverse-transformed blocks with the
// synthesis window and the FFT normalisation, rounding and clamping, for the
// interior of the cover (the part CoverToFrame copies out, src/buffer.cpp:83-116).
// The association order of each region is the reference's.
template <typename R>
void blocks_to_frame(Plane<R>& P, uint8_t* dst, int stride) {
  const int bw = P.bw, bh = P.bh, ow = P.ow, oh = P.oh, sx = bw - ow, sy = bh - oh;
  const R norm = P.norm;
  const bool ints = P.bytes != 4;
  const R rounder = ints ? (R)0.5 : (R)0;
  R base = 0;
  if (ints && P.d.is_chroma) base = (R)(1 << (P.d.bits - 1));
  auto blk = [&](int bx, int by) { return P.in.data() + ((size_t)by * P.nox + bx) * bh * bw; };
  uint8_t* out = dst + (size_t)P.t * stride + (size_t)P.l * P.bytes;
  const int H = P.height;
  auto dst_row = [&](int k) -> uint8_t* {  // cover row mirh + k -> destination row
    if (!P.ep.interlaced) return out + (size_t)k * stride;
    int half = H / 2;  // the inverse of frame_to_cover's field order (src/buffer.cpp:99-115)
    int row = k < half ? 2 * k : H - 1 - 2 * (k - half);
    return out + (size_t)row * stride;
  };
  for (int k = 0; k < H; k++) {
    int Y = P.mirh + k;
    // rows: single block row (by, y) or overlap of (by-1, y+sy) and (by, y)
    int by = Y / sy, y = Y - by * sy;
    bool yov = (by >= 1 && y < oh && by < P.noy);
    if (by >= P.noy) { by = P.noy - 1; y = Y - by * sy; }  // last oh rows (padding only)
    uint8_t* row = dst_row(k);
    for (int x0 = 0; x0 < P.width; x0++) {
      int X = P.mirw + x0;
      int bx = X / sx, x = X - bx * sx;
      bool xov = (bx >= 1 && x < ow && bx < P.nox);
      if (bx >= P.nox) { bx = P.nox - 1; x = X - bx * sx; }
      R v;
      if (!yov) {
        const R* b1 = blk(bx, by) + y * bw;
        if (!xov) v = b1[x] * norm + rounder + base;  // :406,420,427,489,503,510
        else {
          const R* b0 = blk(bx - 1, by) + y * bw;
          v = (b0[x + sx] * P.wsynxr[x] + b1[x] * P.wsynxl[x]) * norm + rounder + base;  // :414,497
        }
      } else {
        R wr = P.wsynyr[y] * norm, wl = P.wsynyl[y] * norm;  // :449-450
        const R* up1 = blk(bx, by - 1) + (y + sy) * bw;
        const R* dn1 = blk(bx, by) + y * bw;
        // (:454 adds the base after the cast, but only for cover columns left of
        // mirw, which CoverToFrame never copies out)
        if (!xov) {
          v = (up1[x] * wr + dn1[x] * wl) + rounder + base;  // :469,476
        } else {
          const R* up0 = blk(bx - 1, by - 1) + (y + sy) * bw;
          const R* dn0 = blk(bx - 1, by) + y * bw;
          v = ((up0[x + sx] * P.wsynxr[x] + up1[x] * P.wsynxl[x]) * wr +
               (dn0[x + sx] * P.wsynxr[x] + dn1[x] * P.wsynxl[x]) * wl) + rounder + base;  // :462-463
        }
      }
      store_px(P, row, x0, v);
    }
  }
}

// ---------------------------------------------------------------- spectral kernels
// Spectra are blocks x bh x outwidth complex (the reference pads rows to
// outpitch; its kernels only touch w < outwidth, code_impl_C.h:66-69).

template <typename R>
R sharpen_factor(const Plane<R>& P, R psd, int bin) {
  // s_fact with the double sqrt of a float argument (Apply.cpp:129-131)
  double root = std::sqrt((double)(psd * P.smax2n / ((psd + P.smin2n) * (psd + P.smax2n))));
  return (R)(1 + (double)((R)P.ep.sharpen * P.wsharpen[bin]) * root);
}
template <typename R>
R dehalo_factor(const Plane<R>& P, R psd, int bin) {
  return (psd + P.ht2n) / ((psd + P.ht2n) + (R)P.ep.dehalo * P.wdehalo[bin] * psd);  // Apply.cpp:132
}

// Apply2D_C (src/code_impl/Apply.cpp:13-65) on one spectrum, in place.
template <typename R>
void apply2d(Plane<R>& P, R* spec) {
  const int nb = P.bh * P.outwidth;
  const bool degrid = P.ep.degrid != 0, pat = P.pattern;
  const bool sh = P.ep.sharpen != 0 || P.ep.dehalo == 0;  // Apply2D_C dispatch (:151-158)
  const bool dh = P.ep.dehalo != 0;
  const R lowlimit = ((R)P.ep.beta - 1) / (R)P.ep.beta;
  for (int blk = 0; blk < P.nblocks; blk++) {
    R* s = spec + (size_t)blk * nb * 2;
    R gf = (R)P.ep.degrid * s[0] / P.gridsample[0];  // code_impl_C.h:64
    for (int i = 0; i < nb; i++) {
      R g0 = 0, g1 = 0;
      if (degrid) { g0 = gf * P.gridsample[2 * i]; g1 = gf * P.gridsample[2 * i + 1]; }
      R cr = s[2 * i] - g0, ci = s[2 * i + 1] - g1;
      R psd = cr * cr + ci * ci + (R)1e-15f;
      R noise = pat ? P.pattern2d[i] : P.sigma2n_cur;
      R q = (psd - noise) / psd;
      R f = q > lowlimit ? q : lowlimit;  // MAX() of fft3d_common.h:51-53
      if (!pat) {
        if (sh && !dh) f *= sharpen_factor(P, psd, i);
        else if (!sh && dh) f *= dehalo_factor(P, psd, i);
        else if (sh && dh) f *= sharpen_factor(P, psd, i) * dehalo_factor(P, psd, i);
      }
      s[2 * i] = cr * f + g0;
      s[2 * i + 1] = ci * f + g1;
    }
  }
}

// limited Wiener factor of one temporal component (code_impl_C.h:34-40)
template <typename R>
inline void wiener3(const Plane<R>& P, R& re, R& im, int bin, R lowlimit) {
  R psd = re * re + im * im + (R)1.0e-15f;
  R q = (psd - (P.pattern ? P.pattern3d[bin] : P.sigma2n_cur)) / psd;
  R f = q > lowlimit ? q : lowlimit;
  re *= f;
  im *= f;
}

// Apply3D{2,3,4,5}_C (src/code_impl/Apply.cpp:67-235): length-bt DFT over the
// frames of each bin, Wiener factor per temporal frequency, inverse at the
// current frame. in[0..4] = frames n-2..n+2 (unused slots null).
template <typename R>
void apply3d(Plane<R>& P, R* const in[5], R* out, int btc) {
  const int nb = P.bh * P.outwidth;
  const bool degrid = P.ep.degrid != 0;
  const R lowlimit = ((R)P.ep.beta - 1) / (R)P.ep.beta;
  const R sin120 = (R)0.86602540378443864676372317075294, athird = (R)1 / (R)3;
  const R sin72 = (R)0.95105651629515357211643933337938, cos72 = (R)0.30901699437494742410229341718282;
  const R sin144 = (R)0.58778525229247312916870595463907, cos144 = (R)-0.80901699437494742410229341718282;
  for (int blk = 0; blk < P.nblocks; blk++) {
    size_t off = (size_t)blk * nb * 2;
    const R* cur = in[2] + off;
    R gf = (R)P.ep.degrid * cur[0] / P.gridsample[0];
    R* o = out + off;
    for (int i = 0; i < nb; i++) {
      R g0 = 0, g1 = 0;
      if (degrid) { g0 = gf * P.gridsample[2 * i] * (R)btc; g1 = gf * P.gridsample[2 * i + 1] * (R)btc; }
      const R cr = cur[2 * i], ci = cur[2 * i + 1];
      if (btc == 2) {
        const R* pv = in[1] + off;
        R pr = pv[2 * i], pi = pv[2 * i + 1];
        R f0r = cr + pr - g0, f0i = ci + pi - g1;
        R f1r = cr - pr, f1i = ci - pi;
        wiener3(P, f0r, f0i, i, lowlimit);
        wiener3(P, f1r, f1i, i, lowlimit);
        o[2 * i] = (f0r + f1r + g0) * (R)0.5;
        o[2 * i + 1] = (f0i + f1i + g1) * (R)0.5;
      } else if (btc == 3) {
        const R* pv = in[1] + off; const R* nx = in[3] + off;
        R pnr = pv[2 * i] + nx[2 * i], pni = pv[2 * i + 1] + nx[2 * i + 1];
        R fcr = cr + pnr - g0, fci = ci + pni - g1;
        R di = sin120 * (pv[2 * i + 1] - nx[2 * i + 1]);
        R dr = sin120 * (nx[2 * i] - pv[2 * i]);
        R fpr = cr - (R)0.5 * pnr + di, fnr = cr - (R)0.5 * pnr - di;
        R fpi = ci - (R)0.5 * pni + dr, fni = ci - (R)0.5 * pni - dr;
        wiener3(P, fcr, fci, i, lowlimit);
        wiener3(P, fpr, fpi, i, lowlimit);
        wiener3(P, fnr, fni, i, lowlimit);
        o[2 * i] = (fcr + fpr + fnr + g0) * athird;
        o[2 * i + 1] = (fci + fpi + fni + g1) * athird;
      } else if (btc == 4) {
        const R* p2 = in[0] + off; const R* pv = in[1] + off; const R* nx = in[3] + off;
        R fp2r = (cr + p2[2 * i]) - (pv[2 * i] + nx[2 * i]);
        R fp2i = (ci + p2[2 * i + 1]) - (pv[2 * i + 1] + nx[2 * i + 1]);
        R fpr = (cr - p2[2 * i]) + (pv[2 * i + 1] - nx[2 * i + 1]);
        R fpi = (ci - p2[2 * i + 1]) - (pv[2 * i] - nx[2 * i]);
        R fcr = (cr + p2[2 * i]) + (pv[2 * i] + nx[2 * i]) - g0;
        R fci = (ci + p2[2 * i + 1]) + (pv[2 * i + 1] + nx[2 * i + 1]) - g1;
        R fnr = (cr - p2[2 * i]) - (pv[2 * i + 1] - nx[2 * i + 1]);
        R fni = (ci - p2[2 * i + 1]) + (pv[2 * i] - nx[2 * i]);
        wiener3(P, fp2r, fp2i, i, lowlimit);
        wiener3(P, fpr, fpi, i, lowlimit);
        wiener3(P, fcr, fci, i, lowlimit);
        wiener3(P, fnr, fni, i, lowlimit);
        o[2 * i] = ((fp2r + fpr) + (fcr + fnr) + g0) * (R)0.25;
        o[2 * i + 1] = ((fp2i + fpi) + (fci + fni) + g1) * (R)0.25;
      } else {  // 5
        const R* p2 = in[0] + off; const R* pv = in[1] + off; const R* nx = in[3] + off; const R* n2 = in[4] + off;
        R p2r = p2[2 * i], p2i = p2[2 * i + 1], pr = pv[2 * i], pi = pv[2 * i + 1];
        R nr = nx[2 * i], ni = nx[2 * i + 1], n2r = n2[2 * i], n2i = n2[2 * i + 1];
        R sum = (p2r + n2r) * cos72 + (pr + nr) * cos144 + cr;
        R dif = (-p2i + n2i) * sin72 + (pi - ni) * sin144;
        R fp2r = sum + dif, fn2r = sum - dif;
        sum = (p2i + n2i) * cos72 + (pi + ni) * cos144 + ci;
        dif = (p2r - n2r) * sin72 + (-pr + nr) * sin144;
        R fp2i = sum + dif, fn2i = sum - dif;
        sum = (p2r + n2r) * cos144 + (pr + nr) * cos72 + cr;
        dif = (p2i - n2i) * sin144 + (pi - ni) * sin72;
        R fpr = sum + dif, fnr = sum - dif;
        sum = (p2i + n2i) * cos144 + (pi + ni) * cos72 + ci;
        dif = (-p2r + n2r) * sin144 + (-pr + nr) * sin72;
        R fpi = sum + dif, fni = sum - dif;
        R fcr = (p2r + pr) + cr + (nr + n2r) - g0;
        R fci = (p2i + pi) + ci + (ni + n2i) - g1;
        wiener3(P, fp2r, fp2i, i, lowlimit);
        wiener3(P, fpr, fpi, i, lowlimit);
        wiener3(P, fcr, fci, i, lowlimit);
        wiener3(P, fnr, fni, i, lowlimit);
        wiener3(P, fn2r, fn2i, i, lowlimit);
        o[2 * i] = ((fp2r + fpr) + (fcr + fnr) + fn2r + g0) * (R)0.2;
        o[2 * i + 1] = ((fp2i + fpi) + (fci + fni) + fn2i + g1) * (R)0.2;
      }
    }
  }
}

// Sharpen_C (src/code_impl/Sharpen.cpp:13-63): sharpen / dehalo of a filtered
// spectrum, grid fraction from that spectrum's own DC.
template <typename R>
void sharpen(Plane<R>& P, R* spec) {
  if (P.ep.sharpen == 0 && P.ep.dehalo == 0) return;
  const int nb = P.bh * P.outwidth;
  const bool degrid = P.ep.degrid != 0;
  const bool sh = P.ep.sharpen != 0, dh = P.ep.dehalo != 0;
  for (int blk = 0; blk < P.nblocks; blk++) {
    R* s = spec + (size_t)blk * nb * 2;
    R gf = (R)P.ep.degrid * s[0] / P.gridsample[0];
    for (int i = 0; i < nb; i++) {
      R g0 = 0, g1 = 0;
      if (degrid) { g0 = gf * P.gridsample[2 * i]; g1 = gf * P.gridsample[2 * i + 1]; }
      R cr = s[2 * i] - g0, ci = s[2 * i + 1] - g1;
      R psd = cr * cr + ci * ci + (R)1.0e-15f;
      R f;
      if (sh && !dh) f = sharpen_factor(P, psd, i);
      else if (!sh && dh) f = dehalo_factor(P, psd, i);
      else f = sharpen_factor(P, psd, i) * dehalo_factor(P, psd, i);
      s[2 * i] = cr * f + g0;
      s[2 * i + 1] = ci * f + g1;
    }
  }
}

// Kalman_C (src/code_impl/Kalman.cpp:13-67): per-bin recursive filter; state
// (outLast, covar, covarProcess) updated in place.
template <typename R>
void kalman(Plane<R>& P, const R* cur) {
  const int nb = P.bh * P.outwidth;
  for (int blk = 0; blk < P.nblocks; blk++) {
    size_t off = (size_t)blk * nb * 2;
    const R* c = cur + off;
    R* last = P.outLast.data() + off;
    R* cv = P.covar.data() + off;
    R* cp = P.covarProcess.data() + off;
    for (int i = 0; i < nb; i++) {
      R sigma;
      if (P.pattern) { sigma = P.pattern2d[i]; if (sigma < (R)1e-15f) sigma = (R)1e-15f; }
      else sigma = P.sigma2n;
      R dr = c[2 * i] - last[2 * i], di = c[2 * i + 1] - last[2 * i + 1];
      if (dr * dr > sigma * P.kratio2 || di * di > sigma * P.kratio2) {
        cv[2 * i] = sigma; cv[2 * i + 1] = sigma;
        cp[2 * i] = sigma; cp[2 * i + 1] = sigma;
        last[2 * i] = c[2 * i]; last[2 * i + 1] = c[2 * i + 1];
      } else {
        for (int k = 0; k < 2; k++) {
          R sum = cv[2 * i + k] + cp[2 * i + k];
          R gain = sum / (sum + sigma);
          cp[2 * i + k] = gain * gain * sigma;
          cv[2 * i + k] = (1 - gain) * sum;
          last[2 * i + k] = gain * c[2 * i + k] + (1 - gain) * last[2 * i + k];
        }
      }
    }
  }
}

// helper.cpp:46-90 FindPatternBlock and :92-132 SetPattern
template <typename R>
void find_and_set_pattern(Plane<R>& P, const R* spec, bool find) {
  const int ow_ = P.outwidth, nb = P.bh * ow_;
  if (find) {
    R best = (R)1e15f;
    for (int by = 2; by < P.noy - 2; by++)
      for (int bx = 2; bx < P.nox - 2; bx++) {
        const R* s = spec + ((size_t)by * P.nox + bx) * nb * 2;
        R acc = 0;
        R g = (R)P.ep.degrid * s[0] / P.gridsample[0];
        for (int i = 0; i < nb; i++) {
          R c0 = s[2 * i] - g * P.gridsample[2 * i], c1 = s[2 * i + 1] - g * P.gridsample[2 * i + 1];
          acc += (c0 * c0 + c1 * c1) * P.pwin[i];
        }
        if (acc < best) { P.ep.px = bx; P.ep.py = by; best = acc; }
      }
  }
  const R* s = spec + ((size_t)P.ep.py * P.nox + P.ep.px) * nb * 2;
  R g = (R)P.ep.degrid * s[0] / P.gridsample[0];
  for (int i = 0; i < nb; i++) {
    R c0 = s[2 * i] - g * P.gridsample[2 * i], c1 = s[2 * i + 1] - g * P.gridsample[2 * i + 1];
    P.pattern2d[i] = (c0 * c0 + c1 * c1) * P.pwin[i];
  }
}

// ---------------------------------------------------------------- engine

template <typename R>
void forward(Plane<R>& P, const uint8_t* src, int stride, R* spec) {
  frame_to_cover(P, src, stride);
  cover_to_blocks(P, P.cover, P.d.is_chroma != 0);
  for (int blk = 0; blk < P.nblocks; blk++)
    P.fft->r2c(P.in.data() + (size_t)blk * P.bh * P.bw, P.bw, spec + (size_t)blk * P.bh * P.outwidth * 2,
               P.outwidth);
}

template <typename R>
void inverse_and_store(Plane<R>& P, const R* spec, const uint8_t* src, int sstride, uint8_t* dst, int dstride) {
  for (int blk = 0; blk < P.nblocks; blk++)
    P.fft->c2r(spec + (size_t)blk * P.bh * P.outwidth * 2, P.outwidth, P.in.data() + (size_t)blk * P.bh * P.bw,
               P.bw);
  // whole plane from the source first (crop borders), then the filtered region
  int pw = P.d.width, ph = P.d.height;
  for (int y = 0; y < ph; y++) std::memcpy(dst + (size_t)y * dstride, src + (size_t)y * sstride, (size_t)pw * P.bytes);
  blocks_to_frame(P, dst, dstride);
}

template <typename R>
R* spectrum_of(Plane<R>& P, int frame, const uint8_t* src, int stride, int keep) {
  auto it = P.cache.find(frame);
  if (it != P.cache.end()) return it->second.data();
  if (!src) return nullptr;
  std::vector<R>& s = P.cache[frame];
  s.assign(P.spec_size(), 0);
  forward(P, src, stride, s.data());
  P.lru.push_back(frame);
  while ((int)P.lru.size() > keep) {
    int old = P.lru.front();
    P.lru.pop_front();
    if (old != frame) P.cache.erase(old);
  }
  return s.data();
}

template <typename R>
int filter(Plane<R>& P, int n, const void* const src[5], const int stride[5], void* dstv, int dstride) {
  uint8_t* dst = (uint8_t*)dstv;
  const uint8_t* cur = (const uint8_t*)src[2];
  if (!cur) return FFT3D_E_FRAME;
  const int bt = P.bt;
  int btcur = bt;  // src/fft3d_engine.h:579-582
  if ((bt / 2 > n) || (bt - 1) / 2 > (P.d.num_frames - 1 - n)) btcur = 1;
  P.sigma2n_cur = (R)btcur * (R)P.ep.sigma * (R)P.ep.sigma / P.norm;  // :589
  P.outrez.assign(P.spec_size(), 0);
  if (P.pattern && !P.pattern_set) return FFT3D_E_UNSUPPORTED;  // needs oracle_estimate_pattern first
  if (bt > 0) {
    if (btcur == 1) {
      forward(P, cur, stride[2], P.outrez.data());
      apply2d(P, P.outrez.data());
      if (P.pattern) sharpen(P, P.outrez.data());
    } else {
      if (!P.pattern3d_init) {  // :625-630
        for (size_t i = 0; i < P.pattern2d.size(); i++) P.pattern3d[i] = P.pattern2d[i] * (R)btcur;
        P.pattern3d_init = true;
      }
      R* ins[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
      for (int i = -btcur / 2; i <= (btcur - 1) / 2; i++) {
        ins[2 + i] = spectrum_of(P, n + i, (const uint8_t*)src[2 + i], stride[2 + i], bt + 3);
        if (!ins[2 + i]) return FFT3D_E_FRAME;
      }
      apply3d(P, ins, P.outrez.data(), btcur);
      sharpen(P, P.outrez.data());
    }
  } else if (bt == 0) {  // Kalman, src/fft3d_engine.h:679-712
    if (n == 0) {
      for (int y = 0; y < P.d.height; y++)
        std::memcpy(dst + (size_t)y * dstride, cur + (size_t)y * stride[2], (size_t)P.d.width * P.bytes);
      return FFT3D_OK;
    }
    forward(P, cur, stride[2], P.outrez.data());
    kalman(P, P.outrez.data());
    P.outrez = P.outLast;
    sharpen(P, P.outrez.data());
  } else {  // bt == -1: sharpen only, :713-724
    forward(P, cur, stride[2], P.outrez.data());
    sharpen(P, P.outrez.data());
  }
  P.last_filtered = P.outrez;
  inverse_and_store(P, P.outrez.data(), cur, stride[2], dst, dstride);
  return FFT3D_OK;
}

thread_local std::string g_err;

template <typename R>
Plane<R>* create(const fft3d_params* p, const fft3d_plane_desc* d) {
  auto P = std::make_unique<Plane<R>>();
  P->ep = *p;
  P->d = *d;
  P->bytes = d->bits <= 8 ? 1 : (d->bits <= 16 ? 2 : 4);
  fft3d_params& ep = P->ep;
  // bit-depth scaling: src/fft3d_engine.h:91-103
  float factor = P->bytes == 1 ? 1.0f : (P->bytes == 2 ? float(1 << (d->bits - 8)) : 1 / 255.0f);
  ep.sigma *= factor; ep.sigma2 *= factor; ep.sigma3 *= factor; ep.sigma4 *= factor;
  ep.smin *= factor; ep.smax *= factor;
  // checks and defaults: :105-126
  if (ep.ow * 2 > ep.bw) { g_err = "ow must be less than bw / 2"; return nullptr; }
  if (ep.oh * 2 > ep.bh) { g_err = "oh must be less than bh / 2"; return nullptr; }
  if (ep.ow < 0) ep.ow = ep.bw / 3;
  if (ep.oh < 0) ep.oh = ep.bh / 3;
  if (ep.bt < -1 || ep.bt > 5) { g_err = "bt must be -1 (Sharpen), 0 (Kalman), 1..5 (Wiener)"; return nullptr; }
  if (ep.beta < 1) { g_err = "beta must be not less 1.0"; return nullptr; }
  P->bw = ep.bw; P->bh = ep.bh; P->ow = ep.ow; P->oh = ep.oh; P->bt = ep.bt;
  // crop in plane units (src/buffer.cpp:564-570)
  P->l = d->is_chroma ? (ep.l >> d->ssw) : ep.l;
  P->r = d->is_chroma ? (ep.r >> d->ssw) : ep.r;
  P->t = d->is_chroma ? (ep.t >> d->ssh) : ep.t;
  P->b = d->is_chroma ? (ep.b >> d->ssh) : ep.b;
  P->width = d->width - P->l - P->r;
  P->height = d->height - P->t - P->b;
  // geometry: :115-136
  P->nox = (P->width - ep.ow + (ep.bw - ep.ow - 1)) / (ep.bw - ep.ow) + 2;
  P->noy = (P->height - ep.oh + (ep.bh - ep.oh - 1)) / (ep.bh - ep.oh) + 2;
  P->mirw = ep.bw - ep.ow;
  P->mirh = ep.bh - ep.oh;
  P->coverw = P->nox * (ep.bw - ep.ow) + ep.ow;
  P->coverh = P->noy * (ep.bh - ep.oh) + ep.oh;
  P->outwidth = ep.bw / 2 + 1;
  P->nblocks = P->nox * P->noy;
  P->fft.reset(new offt::Block2D<R>(ep.bh, ep.bw));
  P->cover.assign((size_t)P->coverw * P->coverh, 0);
  P->in.assign((size_t)P->nblocks * ep.bh * ep.bw, 0);
  make_windows(*P, ep.ow, P->wanxl, P->wanxr, P->wsynxl, P->wsynxr);
  make_windows(*P, ep.oh, P->wanyl, P->wanyr, P->wsynyl, P->wsynyr);
  make_tables(*P);
  if (ep.bt == 0) {  // :339-344
    P->outLast.assign(P->spec_size(), 0);
    P->covar.assign(P->spec_size(), P->sigma2n);
    P->covarProcess.assign(P->spec_size(), P->sigma2n);
  }
  make_gridsample(*P);
  return P.release();
}

struct Handle {
  int dbl;
  void* p;
};

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

void* oracle_create(int dbl, const fft3d_params* p, const fft3d_plane_desc* d) {
  void* pl = dbl ? (void*)create<double>(p, d) : (void*)create<float>(p, d);
  if (!pl) return nullptr;
  return new Handle{dbl, pl};
}

void oracle_destroy(void* h) {
  auto* H = (Handle*)h;
  if (!H) return;
  if (H->dbl) delete (Plane<double>*)H->p;
  else delete (Plane<float>*)H->p;
  delete H;
}

int oracle_filter(void* h, int n, const void* const src[5], const int stride[5], void* dst, int dstride) {
  auto* H = (Handle*)h;
  return H->dbl ? filter(*(Plane<double>*)H->p, n, src, stride, dst, dstride)
                : filter(*(Plane<float>*)H->p, n, src, stride, dst, dstride);
}

// nox, noy, cover w, cover h, outwidth, blocks, ow, oh
void oracle_geometry(void* h, int* out) {
  auto* H = (Handle*)h;
  auto fill = [&](auto& P) {
    out[0] = P.nox; out[1] = P.noy; out[2] = P.coverw; out[3] = P.coverh;
    out[4] = P.outwidth; out[5] = P.nblocks; out[6] = P.ow; out[7] = P.oh;
  };
  if (H->dbl) fill(*(Plane<double>*)H->p);
  else fill(*(Plane<float>*)H->p);
}

// Forward spectrum of one frame (blocks x bh x outwidth complex) as doubles.
int oracle_spectrum(void* h, const void* src, int stride, double* out) {
  auto* H = (Handle*)h;
  auto run = [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.norm)>::type;
    std::vector<R> s(P.spec_size());
    forward(P, (const uint8_t*)src, stride, s.data());
    for (size_t i = 0; i < s.size(); i++) out[i] = (double)s[i];
  };
  if (H->dbl) run(*(Plane<double>*)H->p);
  else run(*(Plane<float>*)H->p);
  return 0;
}

// Spectrum that the last oracle_filter call sent to the inverse transform.
int oracle_last_filtered(void* h, double* out) {
  auto* H = (Handle*)h;
  auto run = [&](auto& P) {
    for (size_t i = 0; i < P.last_filtered.size(); i++) out[i] = (double)P.last_filtered[i];
  };
  if (H->dbl) run(*(Plane<double>*)H->p);
  else run(*(Plane<float>*)H->p);
  return 0;
}

// Noise pattern from one frame (the reference takes frame pframe,
// src/fft3d_engine.h:485-504): block (px, py), or the quietest block if both are 0.
int oracle_estimate_pattern(void* h, const void* src, int stride) {
  auto* H = (Handle*)h;
  auto run = [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.norm)>::type;
    std::vector<R> s(P.spec_size());
    forward(P, (const uint8_t*)src, stride, s.data());
    find_and_set_pattern(P, s.data(), P.ep.px == 0 && P.ep.py == 0);
    P.pattern_set = true;
  };
  if (H->dbl) run(*(Plane<double>*)H->p);
  else run(*(Plane<float>*)H->p);
  return 0;
}

// gridsample (bh x outwidth complex) as doubles.
int oracle_gridsample(void* h, double* out) {
  auto* H = (Handle*)h;
  auto run = [&](auto& P) {
    for (size_t i = 0; i < P.gridsample.size(); i++) out[i] = (double)P.gridsample[i];
  };
  if (H->dbl) run(*(Plane<double>*)H->p);
  else run(*(Plane<float>*)H->p);
  return 0;
}

}  // extern "C"
