// Replays the FFT call patterns of apollo-fft's callers through the C ABI and
// checks every transform against the oracle (f64, relative L2 <= 1e-12).
//
// The callers hold a concrete FftPlan1D<f64> and call the slice methods on
// host buffers; `CudaPlan1D` below is that type over the C ABI, the same shape
// a Rust binding takes (constructor from the length, in-place forward and
// normalized inverse on a contiguous slice):
//   * apollo-stft  StftPlan::new / forward (stft/dimension_1d.rs:42-66, 225-239):
//     Hann-windowed frames centred at m*hop - frame_len/2, zero outside the
//     signal, one forward_complex_slice_inplace per frame.
//   * apollo-czt   czt_bluestein_forward_into_with_workspace (kernel/bluestein.rs:83-130)
//     with the plan of czt/dimension_1d.rs:60-95: chirp premultiply into a
//     zero-filled workspace of length next_pow2(n + m - 1), forward, pointwise
//     product with the FFT of the chirp kernel, normalized inverse, chirp
//     postmultiply.  With A = 1 and W = exp(-2 pi i / n), m = n, the CZT is the
//     length-n DFT, which the oracle computes directly.
//   * apollo-nufft NufftPlan1D (transform/dimension_1d.rs:110-150): one plan of
//     the oversampled length sigma * n, forward and inverse on the spread grid.
//   * apollo-dctdst dct2_dst2_fast / dct3_fast / dst3_fast
//     (infrastructure/kernel/fast.rs:144-345): one 2N-point fft_1d_complex of
//     the zero-padded signal for DCT-II and DST-II, a 2N-point normalized
//     ifft_1d_complex of the Hermitian pre-twiddled spectrum for DCT-III, a
//     2N-point forward FFT of the pre-twiddled signal for DST-III; checked
//     against the definitions summed in long double.
//   * apollo-dht   dht_fast_with_scratch (infrastructure/kernel/fast.rs:10-27):
//     H_k = Re X_k - Im X_k of one forward FFT; checked against the cas sum.
//   * apollo-hilbert analytic_signal_into (infrastructure/kernel/direct.rs:85-106):
//     forward, the analytic mask (1 at DC and Nyquist, 2 on positive bins, 0 on
//     negative), normalized inverse, real part reset to the input; checked
//     against the same steps on the oracle.
// A device-resident batch of all STFT frames (one afc_execute over `frames`
// lanes) is checked too: the fused form a caller moves to.
//
// Build and run: tests/test_gpu_replay.py (needs a CUDA device).
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "apollofft_cuda.h"

extern "C" void or_fft1d_c128(double* d, uint64_t n, uint64_t lanes, int inverse, int threads);

using C = std::complex<double>;

static void check(afc_status s, const char* what) {
  if (s != AFC_OK) throw std::runtime_error(std::string(what) + ": " + afc_last_error_message());
}

// The drop-in for FftPlan1D<f64>: cached plan, host-slice calls.
class CudaPlan1D {
 public:
  explicit CudaPlan1D(int64_t n) : n_(n) {
    check(afc_plan_get_cached(&p_, 1, &n, AFC_PREC_F64, AFC_KIND_C2C, 1, 0), "plan");
  }
  ~CudaPlan1D() { afc_plan_destroy(p_); }
  CudaPlan1D(const CudaPlan1D&) = delete;
  CudaPlan1D& operator=(const CudaPlan1D&) = delete;
  int64_t len() const { return n_; }
  void forward_complex_slice_inplace(C* s, size_t len) const {
    if ((int64_t)len != n_) throw std::runtime_error("complex forward shape mismatch");
    check(afc_execute_host(p_, s, s, AFC_FORWARD), "forward");
  }
  void inverse_complex_slice_inplace(C* s, size_t len) const {
    if ((int64_t)len != n_) throw std::runtime_error("complex inverse shape mismatch");
    check(afc_execute_host(p_, s, s, AFC_INVERSE), "inverse");
  }

 private:
  afc_plan p_ = nullptr;
  int64_t n_;
};

static std::vector<C> oracle_fft(std::vector<C> v, bool inverse) {
  or_fft1d_c128(reinterpret_cast<double*>(v.data()), v.size(), 1, inverse ? 1 : 0, 1);
  return v;
}

static double rel_l2(const std::vector<C>& a, const std::vector<C>& b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += std::norm(a[i] - b[i]);
    den += std::norm(b[i]);
  }
  return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

static int g_fail = 0;
static double g_worst = 0;
static void expect(const char* what, double err, double tol = 1e-12) {
  if (err > g_worst) g_worst = err;
  const bool ok = err <= tol;
  if (!ok) ++g_fail;
  std::printf("%-44s rel_l2 %.3e %s\n", what, err, ok ? "ok" : "FAIL");
}

static void replay_stft() {
  const int64_t frame_len = 512, hop = 128;
  const size_t nsig = 8192;
  std::mt19937_64 rng(11);
  std::normal_distribution<double> nd;
  std::vector<double> signal(nsig), window(frame_len);
  for (auto& s : signal) s = nd(rng);
  for (int64_t n = 0; n < frame_len; ++n)  // periodic Hann
    window[n] = 0.5 - 0.5 * std::cos(2.0 * M_PI * (double)n / (double)frame_len);
  const size_t frames = 1 + (nsig + hop - 1) / hop;  // StftPlan::frame_count (dimension_1d.rs:102-108)
  CudaPlan1D plan(frame_len);
  std::vector<C> all(frames * frame_len), all_ref(frames * frame_len);
  double worst = 0;
  for (size_t m = 0; m < frames; ++m) {
    std::vector<C> frame(frame_len);
    const int64_t start = (int64_t)m * hop - frame_len / 2;
    for (int64_t n = 0; n < frame_len; ++n) {
      const int64_t si = start + n;
      frame[n] = (si >= 0 && si < (int64_t)nsig) ? C(signal[si] * window[n], 0.0) : C(0.0, 0.0);
    }
    std::copy(frame.begin(), frame.end(), all.begin() + m * frame_len);
    std::vector<C> ref = oracle_fft(frame, false);
    std::copy(ref.begin(), ref.end(), all_ref.begin() + m * frame_len);
    plan.forward_complex_slice_inplace(frame.data(), frame.size());
    worst = std::max(worst, rel_l2(frame, ref));
  }
  expect("stft: per-frame host slices (65 x 512)", worst);
  // the same frames as one device batch
  afc_plan bp = nullptr;
  check(afc_plan_create(&bp, 1, &frame_len, AFC_PREC_F64, AFC_KIND_C2C, (int64_t)frames, 0), "batch plan");
  std::vector<C> out(all.size());
  check(afc_execute_host(bp, all.data(), out.data(), AFC_FORWARD), "batch forward");
  expect("stft: all frames in one batched call", rel_l2(out, all_ref));
  afc_plan_destroy(bp);
}

static void replay_czt() {
  const size_t n = 1000, m = 1000;
  size_t conv = 1;
  while (conv < n + m - 1) conv <<= 1;
  CudaPlan1D plan((int64_t)conv);
  // A = 1, W = exp(-2 pi i / n): W^(x) = exp(-2 pi i x / n); phases reduced
  // modulo 2n in integers (k^2 / 2 turns of 2 pi / n) before the sin/cos.
  auto wpow_half_sq = [&](int64_t k, double sign) {
    const int64_t r = (k * k) % (int64_t)(2 * n);  // W^(k^2/2) = exp(-i pi k^2 / n)
    const double ph = -M_PI * (double)r / (double)n * sign;
    return C(std::cos(ph), std::sin(ph));
  };
  std::vector<C> chirp_n(n), chirp_k(m), kernel(conv, C(0, 0));
  for (size_t i = 0; i < n; ++i) chirp_n[i] = wpow_half_sq((int64_t)i, 1.0);
  for (size_t k = 0; k < m; ++k) chirp_k[k] = wpow_half_sq((int64_t)k, 1.0);
  for (size_t k = 0; k < m; ++k) kernel[k] = wpow_half_sq((int64_t)k, -1.0);
  for (size_t j = 1; j < n; ++j) kernel[conv - j] = wpow_half_sq((int64_t)j, -1.0);
  std::vector<C> fk = kernel;
  plan.forward_complex_slice_inplace(fk.data(), fk.size());
  expect("czt: kernel spectrum (forward 2048)", rel_l2(fk, oracle_fft(kernel, false)));

  std::mt19937_64 rng(12);
  std::uniform_real_distribution<double> ud(-1.0, 1.0);
  std::vector<C> x(n);
  for (auto& v : x) v = C(ud(rng), ud(rng));
  std::vector<C> ws(conv, C(0, 0));
  for (size_t i = 0; i < n; ++i) ws[i] = x[i] * chirp_n[i];
  std::vector<C> ws_ref = oracle_fft(ws, false);
  plan.forward_complex_slice_inplace(ws.data(), ws.size());
  expect("czt: workspace forward", rel_l2(ws, ws_ref));
  for (size_t i = 0; i < conv; ++i) ws[i] *= fk[i];
  std::vector<C> inv_ref = oracle_fft(ws, true);
  plan.inverse_complex_slice_inplace(ws.data(), ws.size());
  expect("czt: workspace inverse (normalized)", rel_l2(ws, inv_ref));
  std::vector<C> out(m);
  for (size_t k = 0; k < m; ++k) out[k] = chirp_k[k] * ws[k];
  expect("czt: A=1, W=e^(-2pi i/n) equals the DFT", rel_l2(out, oracle_fft(x, false)), 1e-11);
}

static void replay_nufft() {
  const int64_t n = 1536, sigma = 2, mlen = sigma * n;  // 3072 = 3 * 2^10
  CudaPlan1D plan(mlen);
  std::mt19937_64 rng(13);
  std::normal_distribution<double> nd;
  for (int rep = 0; rep < 4; ++rep) {
    std::vector<C> grid(mlen);
    for (auto& g : grid) g = C(nd(rng), nd(rng));
    std::vector<C> f_ref = oracle_fft(grid, false);
    std::vector<C> i_ref = oracle_fft(grid, true);
    std::vector<C> f = grid, iv = grid;
    plan.forward_complex_slice_inplace(f.data(), f.size());
    plan.inverse_complex_slice_inplace(iv.data(), iv.size());
    if (rep == 0) {
      expect("nufft: oversampled grid forward (3072)", rel_l2(f, f_ref));
      expect("nufft: oversampled grid inverse (3072)", rel_l2(iv, i_ref));
    } else if (rel_l2(f, f_ref) > 1e-12 || rel_l2(iv, i_ref) > 1e-12) {
      expect("nufft: repeated calls on the cached plan", std::max(rel_l2(f, f_ref), rel_l2(iv, i_ref)));
    }
  }
}

// cos / sin of 2 pi m / period in long double, m reduced mod period first
static long double cos_frac(long long m, long long period) {
  return std::cos(2.0L * 3.141592653589793238462643383279502884L * (long double)(m % period) / (long double)period);
}
static long double sin_frac(long long m, long long period) {
  return std::sin(2.0L * 3.141592653589793238462643383279502884L * (long double)(m % period) / (long double)period);
}

static double rel_l2_real(const std::vector<double>& a, const std::vector<long double>& b) {
  long double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += ((long double)a[i] - b[i]) * ((long double)a[i] - b[i]);
    den += b[i] * b[i];
  }
  return (double)std::sqrt(num / den);
}

static void replay_dctdst() {
  const long long n = 1000, two_n = 2 * n;
  std::mt19937_64 rng(17);
  std::normal_distribution<double> nd;
  std::vector<double> x(n);
  for (auto& v : x) v = nd(rng);
  const double half_cycle = M_PI / (double)two_n;
  CudaPlan1D plan(two_n);
  // DCT-II and DST-II from one forward FFT of the zero-padded signal
  std::vector<C> f(two_n);
  for (long long i = 0; i < n; ++i) f[i] = C(x[i], 0.0);
  plan.forward_complex_slice_inplace(f.data(), f.size());
  std::vector<double> dct2(n), dst2(n);
  for (long long k = 0; k < n; ++k) {
    dct2[k] = (std::polar(1.0, -half_cycle * (double)k) * f[k]).real();
    dst2[k] = -(std::polar(1.0, -half_cycle * (double)(k + 1)) * f[k + 1]).imag();
  }
  std::vector<long double> dct2_ref(n, 0.0L), dst2_ref(n, 0.0L);
  for (long long k = 0; k < n; ++k)
    for (long long i = 0; i < n; ++i) {
      dct2_ref[k] += (long double)x[i] * cos_frac((2 * i + 1) * k, 2 * two_n);
      dst2_ref[k] += (long double)x[i] * sin_frac((2 * i + 1) * (k + 1), 2 * two_n);
    }
  expect("dctdst: DCT-II via 2N forward (n = 1000)", rel_l2_real(dct2, dct2_ref));
  expect("dctdst: DST-II via 2N forward (n = 1000)", rel_l2_real(dst2, dst2_ref));
  // DCT-III: Hermitian pre-twiddled spectrum, normalized 2N inverse, N Re(y)
  std::vector<C> g(two_n);
  g[0] = C(x[0], 0.0);
  for (long long k = 1; k < n; ++k) g[k] = C(x[k], 0.0) * std::polar(1.0, half_cycle * (double)k);
  for (long long k = 1; k < n; ++k) g[two_n - k] = std::conj(g[k]);
  plan.inverse_complex_slice_inplace(g.data(), g.size());
  std::vector<double> dct3(n);
  for (long long i = 0; i < n; ++i) dct3[i] = (double)n * g[i].real();
  std::vector<long double> dct3_ref(n);
  for (long long i = 0; i < n; ++i) {
    long double acc = 0.5L * x[0];
    for (long long k = 1; k < n; ++k) acc += (long double)x[k] * cos_frac((2 * i + 1) * k, 2 * two_n);
    dct3_ref[i] = acc;
  }
  expect("dctdst: DCT-III via 2N normalized inverse", rel_l2_real(dct3, dct3_ref));
  // DST-III: pre-twiddled signal with the half boundary term, 2N forward
  std::vector<C> v(two_n);
  for (long long i = 0; i < n; ++i)
    v[i] = C(i < n - 1 ? x[i] : 0.5 * x[i], 0.0) * std::polar(1.0, -half_cycle * (double)i);
  plan.forward_complex_slice_inplace(v.data(), v.size());
  std::vector<double> dst3(n);
  for (long long k = 0; k < n; ++k)
    dst3[k] = (std::polar(1.0, half_cycle * (double)(2 * k + 1)) * std::conj(v[k])).imag();
  std::vector<long double> dst3_ref(n);
  for (long long k = 0; k < n; ++k) {
    long double acc = (k % 2 ? -0.5L : 0.5L) * x[n - 1];
    for (long long i = 0; i + 1 < n; ++i) acc += (long double)x[i] * sin_frac((i + 1) * (2 * k + 1), 2 * two_n);
    dst3_ref[k] = acc;
  }
  expect("dctdst: DST-III via 2N forward", rel_l2_real(dst3, dst3_ref));
}

static void replay_dht() {
  for (long long n : {1000LL, 1009LL, 4096LL}) {
    std::mt19937_64 rng(19 + n);
    std::normal_distribution<double> nd;
    std::vector<double> x(n);
    for (auto& v : x) v = nd(rng);
    CudaPlan1D plan(n);
    std::vector<C> scratch(n);
    for (long long i = 0; i < n; ++i) scratch[i] = C(x[i], 0.0);
    plan.forward_complex_slice_inplace(scratch.data(), scratch.size());
    std::vector<double> h(n);
    for (long long k = 0; k < n; ++k) h[k] = scratch[k].real() - scratch[k].imag();
    std::vector<long double> ref(n, 0.0L);
    for (long long k = 0; k < n; ++k)
      for (long long i = 0; i < n; ++i) ref[k] += (long double)x[i] * (cos_frac(k * i, n) + sin_frac(k * i, n));
    char what[64];
    std::snprintf(what, sizeof what, "dht: Re X - Im X (n = %lld)", n);
    expect(what, rel_l2_real(h, ref));
  }
}

static void analytic_mask(std::vector<C>& s) {
  const size_t len = s.size(), positive_end = (len + 1) / 2;
  for (size_t k = 0; k < len; ++k) {
    const double scale = (k == 0 || (len % 2 == 0 && k == len / 2)) ? 1.0 : (k < positive_end ? 2.0 : 0.0);
    s[k] *= scale;
  }
}

static void replay_hilbert() {
  for (long long n : {1000LL, 1001LL}) {
    std::mt19937_64 rng(23 + n);
    std::normal_distribution<double> nd;
    std::vector<double> x(n);
    for (auto& v : x) v = nd(rng);
    CudaPlan1D plan(n);
    std::vector<C> a(n);
    for (long long i = 0; i < n; ++i) a[i] = C(x[i], 0.0);
    std::vector<C> ref = a;
    plan.forward_complex_slice_inplace(a.data(), a.size());
    analytic_mask(a);
    plan.inverse_complex_slice_inplace(a.data(), a.size());
    for (long long i = 0; i < n; ++i) a[i] = C(x[i], a[i].imag());
    ref = oracle_fft(ref, false);
    analytic_mask(ref);
    ref = oracle_fft(ref, true);
    for (long long i = 0; i < n; ++i) ref[i] = C(x[i], ref[i].imag());
    char what[64];
    std::snprintf(what, sizeof what, "hilbert: analytic signal (n = %lld)", n);
    expect(what, rel_l2(a, ref));
  }
}

int main() {
  try {
    replay_stft();
    replay_czt();
    replay_nufft();
    replay_dctdst();
    replay_dht();
    replay_hilbert();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 2;
  }
  std::printf("replay: %d failure(s), worst rel_l2 %.3e\n", g_fail, g_worst);
  return g_fail ? 1 : 0;
}
