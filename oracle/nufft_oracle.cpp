// CPU restatement of apollo-nufft's NUFFT plans, compiled into the oracle
// library.  TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline of
// the device NUFFT; the apollofft_b200 library never links or calls it.
//
// Follows, step by step (crates/apollo-nufft/src/...):
//   * domain/kernel/kaiser_bessel.rs:55-133  I0 by its power series, the
//     Kaiser-Bessel kernel and its Fourier transform (deconvolution);
//   * application/execution/transform/dimension_1d.rs:101-272  NufftPlan1D:
//     m = sigma n, spreading to round(m x / L) + p, forward FFT, bins
//     k_signed mod m times the deconvolution; type 2 through the normalized
//     inverse times m;
//   * application/execution/transform/dimension_3d.rs:48-620  NufftPlan3D:
//     per axis m = next_pow2(max(sigma n, 2w + 1)), separable weights, 3D
//     FFT, per-axis deconvolution; type 2 through the normalized inverse axis
//     passes (no rescale).
// Points are taken in input order, one thread, as the reference's plans run
// (its bucket sort only reorders the additions).  The FFTs are this oracle's
// plan restatements (or_fft1d_c128 / or_fft3d_c128, one thread).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

extern "C" void or_fft1d_c128(double* d, uint64_t n, uint64_t lanes, int inverse, int threads);
extern "C" void or_fft3d_c128(double* d, uint64_t nx, uint64_t ny, uint64_t nz, int inverse, int threads);

namespace {

using C = std::complex<double>;

double nu_i0(double z) {
  const double scaled = 0.25 * z * z;
  double sum = 1.0, term = 1.0;
  for (int k = 1; k <= 256; ++k) {
    term *= scaled / ((double)k * (double)k);
    sum += term;
    if (term <= 2.220446049250313e-16 * sum) break;
  }
  return sum;
}

double nu_kb(double x, int w, double beta, double i0b) {
  const double u = x / (double)w;
  const double u2 = u * u;
  if (u2 >= 1.0) return 0.0;
  return nu_i0(beta * std::sqrt(1.0 - u2)) / i0b;
}

double nu_kb_ft(double xi, int w, double beta, double i0b) {
  const double t = 2.0 * M_PI * (double)w * xi;
  const double z2 = beta * beta - t * t;
  const double pre = 2.0 * (double)w / i0b;
  if (std::fabs(z2) < 1e-30) return pre;
  if (z2 > 0.0) {
    const double s = std::sqrt(z2);
    return pre * std::sinh(s) / s;
  }
  const double s = std::sqrt(-z2);
  return pre * std::sin(s) / s;
}

long long signed_index(long long k, long long n) { return k <= n / 2 ? k : k - n; }

long long wrap(long long i, long long m) {
  const long long r = i % m;
  return r < 0 ? r + m : r;
}

// x mod L (Euclidean), t = m x / L, m0 = round(t) (half away from zero), d = t - m0
void centre(double x, double len, long long m, long long& m0, double& d) {
  double r = std::fmod(x, len);
  if (r < 0.0) r += len;
  const double t = (double)m * r / len;
  const double rt = std::round(t);
  m0 = (long long)rt;
  d = t - rt;
}

double beta_of(long long sigma, int w) { return M_PI * (1.0 - 1.0 / (2.0 * (double)sigma)) * (double)(2 * w); }

long long over_len_3d(long long n, long long sigma, int w) {
  long long lower = std::max<long long>(n * sigma, 2 * w + 1), m = 1;
  while (m < lower) m <<= 1;
  return m;
}

std::vector<double> deconv(long long n, long long m, int w, double beta, double i0b) {
  std::vector<double> d(n);
  for (long long k = 0; k < n; ++k) d[k] = 1.0 / nu_kb_ft((double)signed_index(k, n) / (double)m, w, beta, i0b);
  return d;
}

void weights(double x, double len, long long m, int w, double beta, double i0b, long long& m0, double* wt) {
  double d;
  centre(x, len, m, m0, d);
  for (int p = -w; p <= w; ++p) wt[p + w] = nu_kb((double)p - d, w, beta, i0b);
}

}  // namespace

extern "C" {

void or_nufft1d_type1(int64_t n, double dx, int64_t sigma, int64_t width, const double* pos, const double* val,
                      int64_t npts, double* out) {
  const int w = (int)width;
  const long long m = sigma * n;
  const double beta = beta_of(sigma, w), i0b = nu_i0(beta), len = (double)n * dx;
  std::vector<C> grid(m);
  std::vector<double> wt(2 * w + 1);
  for (int64_t j = 0; j < npts; ++j) {
    long long m0;
    weights(pos[j], len, m, w, beta, i0b, m0, wt.data());
    const C v(val[2 * j], val[2 * j + 1]);
    for (int p = -w; p <= w; ++p) grid[wrap(m0 + p, m)] += v * wt[p + w];
  }
  or_fft1d_c128(reinterpret_cast<double*>(grid.data()), (uint64_t)m, 1, 0, 1);
  const std::vector<double> dc = deconv(n, m, w, beta, i0b);
  for (int64_t k = 0; k < n; ++k) {
    const C c = grid[wrap(signed_index(k, n), m)] * dc[k];
    out[2 * k] = c.real();
    out[2 * k + 1] = c.imag();
  }
}

void or_nufft1d_type2(int64_t n, double dx, int64_t sigma, int64_t width, const double* coeffs, const double* pos,
                      int64_t npts, double* out) {
  const int w = (int)width;
  const long long m = sigma * n;
  const double beta = beta_of(sigma, w), i0b = nu_i0(beta), len = (double)n * dx;
  const std::vector<double> dc = deconv(n, m, w, beta, i0b);
  std::vector<C> grid(m);
  for (int64_t k = 0; k < n; ++k) grid[wrap(signed_index(k, n), m)] = C(coeffs[2 * k], coeffs[2 * k + 1]) * dc[k];
  or_fft1d_c128(reinterpret_cast<double*>(grid.data()), (uint64_t)m, 1, 1, 1);
  for (auto& g : grid) g *= (double)m;  // the reference rescales the normalized inverse by m
  std::vector<double> wt(2 * w + 1);
  for (int64_t j = 0; j < npts; ++j) {
    long long m0;
    weights(pos[j], len, m, w, beta, i0b, m0, wt.data());
    C acc(0.0, 0.0);
    for (int p = -w; p <= w; ++p) acc += grid[wrap(m0 + p, m)] * wt[p + w];
    out[2 * j] = acc.real();
    out[2 * j + 1] = acc.imag();
  }
}

void or_nufft3d_type1(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz, int64_t sigma,
                      int64_t width, const double* pos, const double* val, int64_t npts, double* out) {
  const int w = (int)width, T = 2 * w + 1;
  const long long mx = over_len_3d(nx, sigma, w), my = over_len_3d(ny, sigma, w), mz = over_len_3d(nz, sigma, w);
  const double beta = beta_of(sigma, w), i0b = nu_i0(beta);
  const double lx = (double)nx * dx, ly = (double)ny * dy, lz = (double)nz * dz;
  std::vector<C> grid((size_t)(mx * my * mz));
  std::vector<double> wx(T), wy(T), wz(T);
  for (int64_t j = 0; j < npts; ++j) {
    long long m0x, m0y, m0z;
    weights(pos[3 * j], lx, mx, w, beta, i0b, m0x, wx.data());
    weights(pos[3 * j + 1], ly, my, w, beta, i0b, m0y, wy.data());
    weights(pos[3 * j + 2], lz, mz, w, beta, i0b, m0z, wz.data());
    const C v(val[2 * j], val[2 * j + 1]);
    for (int px = 0; px < T; ++px) {
      const long long ix = wrap(m0x + px - w, mx);
      for (int py = 0; py < T; ++py) {
        const long long iy = wrap(m0y + py - w, my);
        C* row = grid.data() + (ix * my + iy) * mz;
        for (int pz = 0; pz < T; ++pz) row[wrap(m0z + pz - w, mz)] += v * (wx[px] * wy[py] * wz[pz]);
      }
    }
  }
  or_fft3d_c128(reinterpret_cast<double*>(grid.data()), (uint64_t)mx, (uint64_t)my, (uint64_t)mz, 0, 1);
  const std::vector<double> dcx = deconv(nx, mx, w, beta, i0b), dcy = deconv(ny, my, w, beta, i0b),
                            dcz = deconv(nz, mz, w, beta, i0b);
  for (int64_t kx = 0; kx < nx; ++kx)
    for (int64_t ky = 0; ky < ny; ++ky)
      for (int64_t kz = 0; kz < nz; ++kz) {
        const long long gi = (wrap(signed_index(kx, nx), mx) * my + wrap(signed_index(ky, ny), my)) * mz +
                             wrap(signed_index(kz, nz), mz);
        const C c = grid[gi] * (dcx[kx] * dcy[ky] * dcz[kz]);
        const int64_t o = (kx * ny + ky) * nz + kz;
        out[2 * o] = c.real();
        out[2 * o + 1] = c.imag();
      }
}

void or_nufft3d_type2(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz, int64_t sigma,
                      int64_t width, const double* modes, const double* pos, int64_t npts, double* out) {
  const int w = (int)width, T = 2 * w + 1;
  const long long mx = over_len_3d(nx, sigma, w), my = over_len_3d(ny, sigma, w), mz = over_len_3d(nz, sigma, w);
  const double beta = beta_of(sigma, w), i0b = nu_i0(beta);
  const double lx = (double)nx * dx, ly = (double)ny * dy, lz = (double)nz * dz;
  const std::vector<double> dcx = deconv(nx, mx, w, beta, i0b), dcy = deconv(ny, my, w, beta, i0b),
                            dcz = deconv(nz, mz, w, beta, i0b);
  std::vector<C> grid((size_t)(mx * my * mz));
  for (int64_t kx = 0; kx < nx; ++kx)
    for (int64_t ky = 0; ky < ny; ++ky)
      for (int64_t kz = 0; kz < nz; ++kz) {
        const long long gi = (wrap(signed_index(kx, nx), mx) * my + wrap(signed_index(ky, ny), my)) * mz +
                             wrap(signed_index(kz, nz), mz);
        const int64_t o = (kx * ny + ky) * nz + kz;
        grid[gi] = C(modes[2 * o], modes[2 * o + 1]) * (dcx[kx] * dcy[ky] * dcz[kz]);
      }
  // the reference's three normalized inverse axis passes, no rescale
  or_fft3d_c128(reinterpret_cast<double*>(grid.data()), (uint64_t)mx, (uint64_t)my, (uint64_t)mz, 1, 1);
  std::vector<double> wx(T), wy(T), wz(T);
  for (int64_t j = 0; j < npts; ++j) {
    long long m0x, m0y, m0z;
    weights(pos[3 * j], lx, mx, w, beta, i0b, m0x, wx.data());
    weights(pos[3 * j + 1], ly, my, w, beta, i0b, m0y, wy.data());
    weights(pos[3 * j + 2], lz, mz, w, beta, i0b, m0z, wz.data());
    C acc(0.0, 0.0);
    for (int px = 0; px < T; ++px) {
      const long long ix = wrap(m0x + px - w, mx);
      for (int py = 0; py < T; ++py) {
        const long long iy = wrap(m0y + py - w, my);
        const C* row = grid.data() + (ix * my + iy) * mz;
        for (int pz = 0; pz < T; ++pz) acc += row[wrap(m0z + pz - w, mz)] * (wx[px] * wy[py] * wz[pz]);
      }
    }
    out[2 * j] = acc.real();
    out[2 * j + 1] = acc.imag();
  }
}

}  // extern "C"
