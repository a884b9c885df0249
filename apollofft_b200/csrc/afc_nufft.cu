// afc_nufft.cu -- Kaiser-Bessel spreading / interpolation for the 1D NUFFT
// (apollo-nufft NufftPlan1D, transform/dimension_1d.rs:156-272).
//
// Type 1: every non-uniform point adds value * phi(p - d) to the 2w+1
// oversampled grid cells around round(m x / L) (atomic adds: points are not
// sorted), the grid goes through this library's forward FFT, and the n output
// bins are the grid bins k_signed mod m times the deconvolution factors.
// Type 2: the n coefficients times the deconvolution factors are placed at
// k_signed mod m, the grid goes through the unnormalized inverse FFT, and every
// point gathers its 2w+1 cells weighted by phi.  phi is the reference's kernel
// phi(x) = I0(beta sqrt(1 - (x/w)^2)) / I0(beta), |x| < w, with I0 by its power
// series (kaiser_bessel.rs:55-116), evaluated in FP64 per tap.
#include <cuda_runtime.h>
#include "afc_internal.h"

namespace afc {

// I0(z) = sum_k ((z/2)^2)^k / (k!)^2, summed until the term drops below
// epsilon of the sum (at most 256 terms).
__device__ __forceinline__ double nu_i0(double z) {
  const double scaled = 0.25 * z * z;
  double sum = 1.0, term = 1.0;
  for (int k = 1; k <= 256; ++k) {
    const double kf = (double)k;
    term *= scaled / (kf * kf);
    sum += term;
    if (term <= 2.220446049250313e-16 * sum) break;
  }
  return sum;
}

__device__ __forceinline__ double nu_kb(double x, double w, double beta, double i0b) {
  const double u = x / w;
  const double u2 = u * u;
  if (u2 >= 1.0) return 0.0;
  return nu_i0(beta * sqrt(1.0 - u2)) / i0b;
}

struct NuGeom {
  long long m;     // oversampled length
  int w;           // kernel half width
  double beta, i0b;
  double len;      // periodic domain length n dx
};

// Position -> (m0, d): x mod L (Euclidean), t = m x / L, m0 = round(t) (half
// away from zero), d = t - m0.
__device__ __forceinline__ void nu_place(const NuGeom& g, double x, long long& m0, double& d) {
  double r = fmod(x, g.len);
  if (r < 0.0) r += g.len;
  const double t = (double)g.m * r / g.len;
  const double rt = round(t);
  m0 = (long long)rt;
  d = t - rt;
}

__device__ __forceinline__ long long nu_wrap(long long i, long long m) {
  long long r = i % m;
  return r < 0 ? r + m : r;
}

__global__ void nu_spread(NuGeom g, const double* __restrict__ pos, const double2* __restrict__ val, long long npts,
                          double2* grid) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x) {
    long long m0;
    double d;
    nu_place(g, pos[j], m0, d);
    const double2 v = val[j];
    for (int p = -g.w; p <= g.w; ++p) {
      const double wt = nu_kb((double)p - d, (double)g.w, g.beta, g.i0b);
      if (wt != 0.0) {
        double2* c = grid + nu_wrap(m0 + p, g.m);
        atomicAdd(&c->x, v.x * wt);
        atomicAdd(&c->y, v.y * wt);
      }
    }
  }
}

__global__ void nu_interp(NuGeom g, const double2* __restrict__ grid, const double* __restrict__ pos, long long npts,
                          double2* out) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x) {
    long long m0;
    double d;
    nu_place(g, pos[j], m0, d);
    double2 acc = make_double2(0.0, 0.0);
    for (int p = -g.w; p <= g.w; ++p) {
      const double wt = nu_kb((double)p - d, (double)g.w, g.beta, g.i0b);
      if (wt != 0.0) {
        const double2 c = grid[nu_wrap(m0 + p, g.m)];
        acc.x += c.x * wt;
        acc.y += c.y * wt;
      }
    }
    out[j] = acc;
  }
}

// k -> k_signed mod m (fft_signed_index: k <= n/2 stays, else k - n).
__device__ __forceinline__ long long nu_bin(long long k, long long n, long long m) {
  const long long ks = k <= n / 2 ? k : k - n;
  return nu_wrap(ks, m);
}

__global__ void nu_deconv_out(const double2* __restrict__ grid, const double* __restrict__ deconv, long long n,
                              long long m, double2* out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double2 c = grid[nu_bin(k, n, m)];
    const double f = deconv[k];
    out[k] = make_double2(c.x * f, c.y * f);
  }
}

__global__ void nu_place_coeffs(const double2* __restrict__ coeffs, const double* __restrict__ deconv, long long n,
                                long long m, double2* grid) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double2 c = coeffs[k];
    const double f = deconv[k];
    grid[nu_bin(k, n, m)] = make_double2(c.x * f, c.y * f);
  }
}

static unsigned nu_grid(long long work) {
  long long b = (work + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)b;
}

cudaError_t nufft_spread_dev(const NuLaunch& L, const double* pos, const void* val, long long npts, void* grid,
                             cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  const NuGeom g{L.m, L.w, L.beta, L.i0b, L.len};
  nu_spread<<<nu_grid(npts), 256, 0, st>>>(g, pos, static_cast<const double2*>(val), npts, static_cast<double2*>(grid));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft_interp_dev(const NuLaunch& L, const void* grid, const double* pos, long long npts, void* out,
                             cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  const NuGeom g{L.m, L.w, L.beta, L.i0b, L.len};
  nu_interp<<<nu_grid(npts), 256, 0, st>>>(g, static_cast<const double2*>(grid), pos, npts, static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft_deconv_out_dev(const void* grid, const double* deconv, long long n, long long m, void* out,
                                 cudaStream_t st) {
  nu_deconv_out<<<nu_grid(n), 256, 0, st>>>(static_cast<const double2*>(grid), deconv, n, m, static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft_place_coeffs_dev(const void* coeffs, const double* deconv, long long n, long long m, void* grid,
                                   cudaStream_t st) {
  nu_place_coeffs<<<nu_grid(n), 256, 0, st>>>(static_cast<const double2*>(coeffs), deconv, n, m,
                                              static_cast<double2*>(grid));
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
