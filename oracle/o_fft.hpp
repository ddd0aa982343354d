// Oracle FFT — TEST INFRASTRUCTURE ONLY (used by the FFTW-API shim and by the
// CPU restatement of the neo_fft3d pipeline; never by the product path).
//
// The reference (neo_fft3d) delegates its block transforms to FFTW
// (src/fftwlite.h:33-43, plans created at src/fft3d_engine.h:161-189). FFTW is
// not vendored by the reference and not installed on this image, so this file
// restates FFTW's *documented* semantics with its own algorithm:
//   * forward sign -1, backward sign +1, no normalisation;
//   * 2D r2c over an n0 x n1 real array gives n0 x (n1/2+1) complex, the last
//     dimension halved (FFTW manual, "Multi-Dimensional DFTs of Real Data");
//   * 2D c2r is the inverse of that; like FFTW, it ignores the imaginary part of
//     the k1 = 0 and k1 = n1/2 columns after the transform along dimension 0.
//
// Algorithm: Stockham self-sorting mixed radix (2, 3, 4, 5, generic p) on split
// re/im arrays with the batch index innermost, so that every butterfly runs over
// a contiguous row of independent transforms (vectorisable). Twiddles are formed
// in double precision and rounded to the working type R.
#pragma once
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

namespace offt {

// Factor n into the radices used by the passes (4 first, then 2, 3, 5, others).
inline std::vector<int> factorize(int n) {
  std::vector<int> f;
  while (n % 4 == 0) { f.push_back(4); n /= 4; }
  while (n % 2 == 0) { f.push_back(2); n /= 2; }
  for (int p = 3; n > 1; p += 2)
    while (n % p == 0) { f.push_back(p); n /= p; }
  return f;
}

// A length-n complex transform applied to `batch` sequences at once. Element j
// of sequence b lives at re[j*ld + b], im[j*ld + b].
template <typename R>
struct BatchFFT {
  int n = 0;
  std::vector<int> radix;
  // per pass: twiddle W_{L*p}^{j*u} for j < L, u < p (sign -1) as re/im
  std::vector<std::vector<R>> twr, twi;
  std::vector<std::vector<R>> wpr, wpi;  // W_p^{k} k < p (sign -1)

  explicit BatchFFT(int n_ = 1) { init(n_); }

  void init(int n_) {
    n = n_;
    radix = factorize(n);
    twr.clear(); twi.clear(); wpr.clear(); wpi.clear();
    int L = 1;
    for (int p : radix) {
      std::vector<R> tr(L * p), ti(L * p), pr(p), pi(p);
      for (int j = 0; j < L; j++)
        for (int u = 0; u < p; u++) {
          long e = (long)j * u;
          double a = -2.0 * M_PI * (double)(e % (L * p)) / (double)(L * p);
          tr[j * p + u] = (R)std::cos(a);
          ti[j * p + u] = (R)std::sin(a);
        }
      for (int k = 0; k < p; k++) {
        double a = -2.0 * M_PI * (double)k / (double)p;
        pr[k] = (R)std::cos(a);
        pi[k] = (R)std::sin(a);
      }
      twr.push_back(tr); twi.push_back(ti); wpr.push_back(pr); wpi.push_back(pi);
      L *= p;
    }
  }

  // In-place (result in xr/xi) transform; tr/ti are scratch of the same size.
  // sign = -1 forward, +1 backward.
  void run(R* xr, R* xi, R* tr, R* ti, int batch, int ld, int sign) const {
    R* ar = xr; R* ai = xi; R* br = tr; R* bi = ti;
    int L = 1;
    for (size_t s = 0; s < radix.size(); s++) {
      int p = radix[s];
      int r = n / (L * p);
      const R* TR = twr[s].data();
      const R* TI = twi[s].data();
      for (int k = 0; k < r; k++) {
        for (int j = 0; j < L; j++) {
          // inputs X[j + L*(k + r*u)], u < p ; outputs Y[j + L*q + L*p*k]
          const R* inr[8]; const R* ini[8];
          R* outr[8]; R* outi[8];
          std::vector<const R*> vinr, vini; std::vector<R*> voutr, vouti;
          const R** pir = inr; const R** pii = ini; R** por = outr; R** poi = outi;
          if (p > 8) { vinr.resize(p); vini.resize(p); voutr.resize(p); vouti.resize(p);
                       pir = vinr.data(); pii = vini.data(); por = voutr.data(); poi = vouti.data(); }
          for (int u = 0; u < p; u++) {
            pir[u] = ar + (size_t)(j + L * (k + r * u)) * ld;
            pii[u] = ai + (size_t)(j + L * (k + r * u)) * ld;
            por[u] = br + (size_t)(j + L * u + L * p * k) * ld;
            poi[u] = bi + (size_t)(j + L * u + L * p * k) * ld;
          }
          R wr[8], wi[8];
          std::vector<R> vwr, vwi; R* pwr = wr; R* pwi = wi;
          if (p > 8) { vwr.resize(p); vwi.resize(p); pwr = vwr.data(); pwi = vwi.data(); }
          // the table holds sign -1 twiddles; the backward transform conjugates
          for (int u = 0; u < p; u++) {
            pwr[u] = TR[j * p + u];
            pwi[u] = sign > 0 ? -TI[j * p + u] : TI[j * p + u];
          }
          butterfly(p, s, pir, pii, por, poi, pwr, pwi, batch, sign);
        }
      }
      std::swap(ar, br); std::swap(ai, bi);
      L *= p;
    }
    if (ar != xr) {
      for (int j = 0; j < n; j++) {
        std::memcpy(xr + (size_t)j * ld, ar + (size_t)j * ld, sizeof(R) * batch);
        std::memcpy(xi + (size_t)j * ld, ai + (size_t)j * ld, sizeof(R) * batch);
      }
    }
  }

 private:
  void butterfly(int p, size_t s, const R** ir, const R** ii, R** orr, R** oi,
                 const R* wr, const R* wi, int batch, int sign) const {
    // twiddled inputs t_u = W^{ju} x_u, then a p-point DFT with sign
    const R sg = (R)sign;
    if (p == 2) {
      for (int b = 0; b < batch; b++) {
        R x0r = ir[0][b], x0i = ii[0][b];
        R x1r = ir[1][b] * wr[1] - ii[1][b] * wi[1];
        R x1i = ir[1][b] * wi[1] + ii[1][b] * wr[1];
        orr[0][b] = x0r + x1r; oi[0][b] = x0i + x1i;
        orr[1][b] = x0r - x1r; oi[1][b] = x0i - x1i;
      }
    } else if (p == 4) {
      for (int b = 0; b < batch; b++) {
        R x0r = ir[0][b], x0i = ii[0][b];
        R x1r = ir[1][b] * wr[1] - ii[1][b] * wi[1];
        R x1i = ir[1][b] * wi[1] + ii[1][b] * wr[1];
        R x2r = ir[2][b] * wr[2] - ii[2][b] * wi[2];
        R x2i = ir[2][b] * wi[2] + ii[2][b] * wr[2];
        R x3r = ir[3][b] * wr[3] - ii[3][b] * wi[3];
        R x3i = ir[3][b] * wi[3] + ii[3][b] * wr[3];
        R s02r = x0r + x2r, s02i = x0i + x2i, d02r = x0r - x2r, d02i = x0i - x2i;
        R s13r = x1r + x3r, s13i = x1i + x3i, d13r = x1r - x3r, d13i = x1i - x3i;
        // multiply d13 by (sign * i): forward (sign -1) -> -i
        R jr = -sg * d13i, ji = sg * d13r;
        orr[0][b] = s02r + s13r; oi[0][b] = s02i + s13i;
        orr[1][b] = d02r + jr;   oi[1][b] = d02i + ji;
        orr[2][b] = s02r - s13r; oi[2][b] = s02i - s13i;
        orr[3][b] = d02r - jr;   oi[3][b] = d02i - ji;
      }
    } else {
      // generic p-point DFT (p = 3, 5, other primes)
      const R* pr = wpr[s].data();
      const R* pi = wpi[s].data();
      std::vector<R> tr(p), ti(p);
      for (int b = 0; b < batch; b++) {
        for (int u = 0; u < p; u++) {
          tr[u] = ir[u][b] * wr[u] - ii[u][b] * wi[u];
          ti[u] = ir[u][b] * wi[u] + ii[u][b] * wr[u];
        }
        for (int q = 0; q < p; q++) {
          R accr = tr[0], acci = ti[0];
          for (int u = 1; u < p; u++) {
            int e = (q * u) % p;
            R cr = pr[e], ci = sign > 0 ? -pi[e] : pi[e];
            accr += tr[u] * cr - ti[u] * ci;
            acci += tr[u] * ci + ti[u] * cr;
          }
          orr[q][b] = accr; oi[q][b] = acci;
        }
      }
    }
  }
};

// 2D block transforms with FFTW's real-data conventions (rows = dimension 0 of
// length n0, columns = dimension 1 of length n1).
template <typename R>
struct Block2D {
  int n0, n1, nh;  // nh = n1/2 + 1
  BatchFFT<R> f1, f0;
  std::vector<R> ar, ai, br, bi;
  Block2D(int n0_, int n1_) : n0(n0_), n1(n1_), nh(n1_ / 2 + 1), f1(n1_), f0(n0_) {
    size_t m = (size_t)std::max(n0, n1) * std::max(n0, n1) + 64;
    ar.resize(m); ai.resize(m); br.resize(m); bi.resize(m);
  }
  // in: real n0 x n1 with row pitch ipitch; out: complex (interleaved re,im)
  // n0 x nh with row pitch opitch (in complex elements).
  void r2c(const R* in, int ipitch, R* out, int opitch) {
    // transforms along dimension 1 (length n1), batch = n0 rows: layout [x][y]
    for (int x = 0; x < n1; x++)
      for (int y = 0; y < n0; y++) { ar[(size_t)x * n0 + y] = in[(size_t)y * ipitch + x]; ai[(size_t)x * n0 + y] = 0; }
    f1.run(ar.data(), ai.data(), br.data(), bi.data(), n0, n0, -1);
    // transpose to [y][k] (k < nh), transform along dimension 0, batch = nh
    for (int y = 0; y < n0; y++)
      for (int k = 0; k < nh; k++) { br[(size_t)y * nh + k] = ar[(size_t)k * n0 + y]; bi[(size_t)y * nh + k] = ai[(size_t)k * n0 + y]; }
    f0.run(br.data(), bi.data(), ar.data(), ai.data(), nh, nh, -1);
    for (int y = 0; y < n0; y++)
      for (int k = 0; k < nh; k++) {
        out[2 * ((size_t)y * opitch + k)] = br[(size_t)y * nh + k];
        out[2 * ((size_t)y * opitch + k) + 1] = bi[(size_t)y * nh + k];
      }
  }
  // in: complex n0 x nh (pitch ipitch complex); out: real n0 x n1 (pitch opitch)
  void c2r(const R* in, int ipitch, R* out, int opitch) {
    for (int y = 0; y < n0; y++)
      for (int k = 0; k < nh; k++) {
        ar[(size_t)y * nh + k] = in[2 * ((size_t)y * ipitch + k)];
        ai[(size_t)y * nh + k] = in[2 * ((size_t)y * ipitch + k) + 1];
      }
    f0.run(ar.data(), ai.data(), br.data(), bi.data(), nh, nh, +1);
    // Hermitian extension along dimension 1: layout [x][y]; the imaginary parts
    // of k = 0 and (even n1) k = n1/2 are ignored.
    for (int y = 0; y < n0; y++) {
      for (int k = 0; k < nh; k++) {
        R re = ar[(size_t)y * nh + k], im = ai[(size_t)y * nh + k];
        if (k == 0 || (2 * k == n1)) im = 0;
        br[(size_t)k * n0 + y] = re; bi[(size_t)k * n0 + y] = im;
        if (k > 0 && 2 * k != n1) { br[(size_t)(n1 - k) * n0 + y] = re; bi[(size_t)(n1 - k) * n0 + y] = -im; }
      }
    }
    f1.run(br.data(), bi.data(), ar.data(), ai.data(), n0, n0, +1);
    for (int y = 0; y < n0; y++)
      for (int x = 0; x < n1; x++) out[(size_t)y * opitch + x] = br[(size_t)x * n0 + y];
  }
};

}  // namespace offt
