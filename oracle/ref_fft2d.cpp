// ref_fft2d.cpp -- TEST INFRASTRUCTURE (oracle), never shipped or measured.
//
// Implements the hvd::Fft2d interface declared in the reference's
// hvd-core/src/engine/fft2d.h:22-58 so that the reference engine compiles
// without FFTW3f (absent from this image; the reference's own fft2d.cpp
// binds FFTW, fft2d.cpp:19-79). Semantics follow fft2d.h:10-13: Forward is
// the unnormalised DFT with exp(-2 pi i jk / n), Inverse uses exp(+...) and
// divides by (height * width), i.e. numpy.fft.fft2 / ifft2.
//
// Algorithm (own code, published methods): iterative radix-2 Cooley-Tukey
// for power-of-two lengths and Bluestein's chirp-z embedding (Bluestein
// 1970) into a power-of-two length >= 2n-1 for every other length, with
// per-length bit-reversal and twiddle tables. All arithmetic is in double
// precision; results are rounded to float once, so this is at least as
// accurate as FFTW's single-precision transforms. It is slower than FFTW's
// plans for these sizes; the CPU timings that include it say so.

#include <cmath>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "engine/fft2d.h"

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

bool IsPow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Complex product written out: std::complex<double>'s operator* goes through
// the C99 Annex G NaN-recovery path (a library call per product) without
// -ffast-math; these transforms never see non-finite values.
inline cd Mul(const cd& a, const cd& b) {
  return cd(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// Tables of one power-of-two length: bit-reversal permutation and the
// twiddles exp(-2 pi i k / n), k < n / 2.
struct Pow2Table {
  int n = 0;
  std::vector<int> rev;
  std::vector<cd> tw;
};

Pow2Table MakePow2(int n) {
  Pow2Table t;
  t.n = n;
  t.rev.resize(n);
  int bits = 0;
  while ((1 << bits) < n) ++bits;
  for (int i = 0; i < n; ++i) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
    t.rev[i] = r;
  }
  t.tw.resize(n / 2 > 0 ? n / 2 : 1);
  for (int k = 0; k < n / 2; ++k) t.tw[k] = cd(std::cos(2.0 * kPi * k / n), -std::sin(2.0 * kPi * k / n));
  return t;
}

// In-place iterative radix-2 FFT; sign = -1 forward, +1 backward (no scale).
void FftPow2(const Pow2Table& t, cd* a, int sign) {
  const int n = t.n;
  for (int i = 0; i < n; ++i) {
    const int j = t.rev[i];
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1;
    const int step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < half; ++k) {
        cd w = t.tw[k * step];
        if (sign > 0) w = std::conj(w);
        const cd u = a[i + k];
        const cd v = Mul(a[i + k + half], w);
        a[i + k] = u + v;
        a[i + k + half] = u - v;
      }
    }
  }
}

// Plan for one length n (both signs): radix-2 directly for powers of two,
// Bluestein otherwise.
struct Plan1D {
  int n = 0;
  int m = 0;                 // power-of-two embedding length (0: n is a power of two)
  Pow2Table pow2;            // tables of n (power of two) or of m
  std::vector<cd> chirp;     // exp(-i pi k^2 / n), k in [0, n)
  std::vector<cd> bhat_fwd;  // FFT_m of the forward chirp filter
  std::vector<cd> bhat_bwd;  // FFT_m of the backward chirp filter
};

std::shared_ptr<Plan1D> MakePlan(int n) {
  auto p = std::make_shared<Plan1D>();
  p->n = n;
  if (IsPow2(n)) {
    p->pow2 = MakePow2(n);
    return p;
  }
  int m = 1;
  while (m < 2 * n - 1) m <<= 1;
  p->m = m;
  p->pow2 = MakePow2(m);
  p->chirp.resize(n);
  for (int k = 0; k < n; ++k) {
    // k^2 mod 2n keeps the argument small (exact integer reduction).
    const int64_t kk = (static_cast<int64_t>(k) * k) % (2LL * n);
    const double a = kPi * static_cast<double>(kk) / n;
    p->chirp[k] = cd(std::cos(a), -std::sin(a));
  }
  for (int s = 0; s < 2; ++s) {
    std::vector<cd> b(m, cd(0, 0));
    // forward: X[k] = w*[k] sum x[j] w*[j] w[k-j] with w = exp(+i pi k^2/n)
    for (int k = 0; k < n; ++k) {
      const cd w = s == 0 ? std::conj(p->chirp[k]) : p->chirp[k];
      b[k] = w;
      if (k) b[m - k] = w;
    }
    FftPow2(p->pow2, b.data(), -1);
    (s == 0 ? p->bhat_fwd : p->bhat_bwd) = std::move(b);
  }
  return p;
}

// 1-D DFT of `x` (stride 1), sign -1 / +1, no normalisation.
void Dft1D(const Plan1D& p, cd* x, int sign, std::vector<cd>& work) {
  const int n = p.n;
  if (p.m == 0) {
    FftPow2(p.pow2, x, sign);
    return;
  }
  const int m = p.m;
  work.assign(m, cd(0, 0));
  for (int k = 0; k < n; ++k) {
    const cd w = sign < 0 ? p.chirp[k] : std::conj(p.chirp[k]);
    work[k] = Mul(x[k], w);
  }
  FftPow2(p.pow2, work.data(), -1);
  const std::vector<cd>& bh = sign < 0 ? p.bhat_fwd : p.bhat_bwd;
  for (int i = 0; i < m; ++i) work[i] = Mul(work[i], bh[i]);
  FftPow2(p.pow2, work.data(), +1);
  const double inv_m = 1.0 / m;
  for (int k = 0; k < n; ++k) {
    const cd w = sign < 0 ? p.chirp[k] : std::conj(p.chirp[k]);
    x[k] = Mul(work[k] * inv_m, w);
  }
}

std::mutex& PlanMutex() {
  static std::mutex m;
  return m;
}

std::shared_ptr<Plan1D> PlanFor(int n) {
  static std::map<int, std::shared_ptr<Plan1D>> cache;
  std::lock_guard<std::mutex> lock(PlanMutex());
  auto it = cache.find(n);
  if (it != cache.end()) return it->second;
  auto p = MakePlan(n);
  cache.emplace(n, p);
  return p;
}

}  // namespace

namespace hvd {

struct Fft2d::Impl {
  int thread_count = 1;
};

Fft2d::Fft2d() : impl_(new Impl) {}
Fft2d::~Fft2d() { delete impl_; }
void Fft2d::SetThreadCount(int n) { impl_->thread_count = n < 1 ? 1 : n; }

ComplexPlane Fft2d::Run(const ComplexPlane& in, int sign, bool normalise) {
  const int h = in.height();
  const int w = in.width();
  ComplexPlane out(h, w);
  if (h == 0 || w == 0) return out;
  std::vector<cd> a(static_cast<size_t>(h) * w);
  for (size_t i = 0; i < a.size(); ++i) a[i] = cd(in[i].real(), in[i].imag());
  const auto pw = PlanFor(w);
  const auto ph = PlanFor(h);
  std::vector<cd> work;
  for (int y = 0; y < h; ++y) Dft1D(*pw, a.data() + static_cast<size_t>(y) * w, sign, work);
  // columns through a transposed copy (contiguous 1-D transforms)
  std::vector<cd> t(a.size());
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) t[static_cast<size_t>(x) * h + y] = a[static_cast<size_t>(y) * w + x];
  for (int x = 0; x < w; ++x) Dft1D(*ph, t.data() + static_cast<size_t>(x) * h, sign, work);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) a[static_cast<size_t>(y) * w + x] = t[static_cast<size_t>(x) * h + y];
  const double scale = normalise ? 1.0 / (static_cast<double>(h) * w) : 1.0;
  for (size_t i = 0; i < a.size(); ++i)
    out[i] = Complex(static_cast<float>(a[i].real() * scale),
                     static_cast<float>(a[i].imag() * scale));
  return out;
}

ComplexPlane Fft2d::Forward(const ComplexPlane& in) { return Run(in, -1, false); }
ComplexPlane Fft2d::Inverse(const ComplexPlane& in) { return Run(in, +1, true); }

}  // namespace hvd
