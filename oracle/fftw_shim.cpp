// FFTW-API shim — TEST INFRASTRUCTURE ONLY.
//
// The reference loads FFTW at run time with dlopen("libfftw3f_threads.so") and
// binds exactly nine symbols (src/fftwlite.h:33-43, loaded at :71-85). No FFTW
// exists on this image, so this library provides those nine entry points with
// FFTW's documented semantics on top of the oracle FFT (o_fft.hpp). It lets the
// UNMODIFIED reference plugin run here as the parity oracle.
//
// Supported plans: rank 2, istride = ostride = 1, any howmany / dist / embed,
// which is what the reference creates (src/fft3d_engine.h:161-189, :387-388).
// Threads: fftwf_plan_with_nthreads(n) makes later plans split their batch of
// blocks over n std::threads, like FFTW's threaded planner does for howmany.
// Environment: FFT3D_SHIM_F64=1 makes plans compute in double and round the
// result to float (isolates FFT rounding from the rest of the pipeline).
#include <cstdlib>
#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

#include "o_fft.hpp"

typedef float fftwf_complex[2];

namespace {

int g_nthreads = 1;

struct Plan {
  bool r2c;
  int n0, n1, howmany;
  int ipitch, idist, opitch, odist;  // element units of the respective arrays
  int nthreads;
  bool f64;
  std::vector<std::unique_ptr<offt::Block2D<float>>> ws32;
  std::vector<std::unique_ptr<offt::Block2D<double>>> ws64;

  void run_range(int t, int b0, int b1, const float* in, float* out) {
    if (!f64) {
      auto& w = *ws32[t];
      for (int b = b0; b < b1; b++) {
        if (r2c) w.r2c(in + (size_t)b * idist, ipitch, out + 2 * (size_t)b * odist, opitch);
        else     w.c2r(in + 2 * (size_t)b * idist, ipitch, out + (size_t)b * odist, opitch);
      }
      return;
    }
    auto& w = *ws64[t];
    int nh = n1 / 2 + 1;
    std::vector<double> src((size_t)n0 * (size_t)(n1 + 2) * 2), dst((size_t)n0 * (size_t)(n1 + 2) * 2);
    for (int b = b0; b < b1; b++) {
      if (r2c) {
        const float* ib = in + (size_t)b * idist;
        for (int y = 0; y < n0; y++)
          for (int x = 0; x < n1; x++) src[(size_t)y * n1 + x] = ib[(size_t)y * ipitch + x];
        w.r2c(src.data(), n1, dst.data(), nh);
        float* ob = out + 2 * (size_t)b * odist;
        for (int y = 0; y < n0; y++)
          for (int k = 0; k < nh; k++) {
            ob[2 * ((size_t)y * opitch + k)] = (float)dst[2 * ((size_t)y * nh + k)];
            ob[2 * ((size_t)y * opitch + k) + 1] = (float)dst[2 * ((size_t)y * nh + k) + 1];
          }
      } else {
        const float* ib = in + 2 * (size_t)b * idist;
        for (int y = 0; y < n0; y++)
          for (int k = 0; k < nh; k++) {
            src[2 * ((size_t)y * nh + k)] = ib[2 * ((size_t)y * ipitch + k)];
            src[2 * ((size_t)y * nh + k) + 1] = ib[2 * ((size_t)y * ipitch + k) + 1];
          }
        w.c2r(src.data(), nh, dst.data(), n1);
        float* ob = out + (size_t)b * odist;
        for (int y = 0; y < n0; y++)
          for (int x = 0; x < n1; x++) ob[(size_t)y * opitch + x] = (float)dst[(size_t)y * n1 + x];
      }
    }
  }

  void execute(const float* in, float* out) {
    if (nthreads <= 1 || howmany < 2 * nthreads) { run_range(0, 0, howmany, in, out); return; }
    std::vector<std::thread> th;
    int per = (howmany + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int b0 = t * per, b1 = std::min(howmany, b0 + per);
      if (b0 >= b1) break;
      th.emplace_back([=] { run_range(t, b0, b1, in, out); });
    }
    for (auto& x : th) x.join();
  }
};

Plan* make_plan(bool r2c, int rank, const int* n, int howmany, const int* inembed, int istride, int idist,
                const int* onembed, int ostride, int odist) {
  if (rank != 2 || istride != 1 || ostride != 1 || howmany < 1) return nullptr;
  auto* p = new Plan();
  p->r2c = r2c;
  p->n0 = n[0]; p->n1 = n[1]; p->howmany = howmany;
  int nh = n[1] / 2 + 1;
  // default (NULL) embeds are the logical sizes of the respective arrays
  int in_last = inembed ? inembed[1] : (r2c ? n[1] : nh);
  int out_last = onembed ? onembed[1] : (r2c ? nh : n[1]);
  p->ipitch = in_last; p->idist = idist; p->opitch = out_last; p->odist = odist;
  p->nthreads = g_nthreads < 1 ? 1 : g_nthreads;
  const char* e = std::getenv("FFT3D_SHIM_F64");
  p->f64 = e && e[0] == '1';
  for (int t = 0; t < p->nthreads; t++) {
    if (p->f64) p->ws64.emplace_back(new offt::Block2D<double>(n[0], n[1]));
    else        p->ws32.emplace_back(new offt::Block2D<float>(n[0], n[1]));
  }
  return p;
}

}  // namespace

extern "C" {

typedef void* fftwf_plan;  // opaque, as in FFTW

fftwf_complex* fftwf_malloc(size_t n) {
  void* p = nullptr;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
  return (fftwf_complex*)p;
}

void fftwf_free(void* p) { std::free(p); }

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(true, rank, n, howmany, inembed, istride, idist, onembed, ostride, odist);
}

fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out, const int* onembed, int ostride, int odist,
                                   unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(false, rank, n, howmany, inembed, istride, idist, onembed, ostride, odist);
}

void fftwf_destroy_plan(fftwf_plan p) { delete (Plan*)p; }

void fftwf_execute_dft_r2c(fftwf_plan p, float* in, fftwf_complex* out) { ((Plan*)p)->execute(in, (float*)out); }

void fftwf_execute_dft_c2r(fftwf_plan p, fftwf_complex* in, float* out) { ((Plan*)p)->execute((const float*)in, out); }

int fftwf_init_threads(void) { return 1; }

void fftwf_plan_with_nthreads(int n) { g_nthreads = n < 1 ? 1 : n; }

}  // extern "C"
