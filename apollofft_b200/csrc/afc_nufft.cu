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

// ─── 3D (apollo-nufft NufftPlan3D, transform/dimension_3d.rs:193-620) ───
// Separable kernel: weight = phi_x phi_y phi_z over (2w+1)^3 taps; grid C-order
// [ix][iy][iz] of size mx x my x mz.
struct NuGeom3 {
  long long mx, my, mz;
  int w;
  double beta, i0b;
  double lx, ly, lz;
};

constexpr int kNuMaxTaps = 65;  // 2 w + 1 for w <= 32

__device__ __forceinline__ void nu_weights(double t, long long m, const NuGeom3& g, long long& m0, double* wt) {
  const double rt = round(t);
  m0 = (long long)rt;
  const double d = t - rt;
  for (int p = -g.w; p <= g.w; ++p) wt[p + g.w] = nu_kb((double)p - d, (double)g.w, g.beta, g.i0b);
  (void)m;
}

__device__ __forceinline__ double nu_axis_t(double x, double len, long long m) {
  double r = fmod(x, len);
  if (r < 0.0) r += len;
  return (double)m * r / len;
}

__global__ void nu_spread3(NuGeom3 g, const double* __restrict__ pos, const double2* __restrict__ val, long long npts,
                           double2* grid) {
  double wx[kNuMaxTaps], wy[kNuMaxTaps], wz[kNuMaxTaps];
  const int taps = 2 * g.w + 1;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x) {
    long long m0x, m0y, m0z;
    nu_weights(nu_axis_t(pos[3 * j], g.lx, g.mx), g.mx, g, m0x, wx);
    nu_weights(nu_axis_t(pos[3 * j + 1], g.ly, g.my), g.my, g, m0y, wy);
    nu_weights(nu_axis_t(pos[3 * j + 2], g.lz, g.mz), g.mz, g, m0z, wz);
    const double2 v = val[j];
    for (int px = 0; px < taps; ++px) {
      if (wx[px] == 0.0) continue;
      const long long ix = nu_wrap(m0x + px - g.w, g.mx);
      for (int py = 0; py < taps; ++py) {
        if (wy[py] == 0.0) continue;
        const long long iy = nu_wrap(m0y + py - g.w, g.my);
        const double wxy = wx[px] * wy[py];
        double2* row = grid + (ix * g.my + iy) * g.mz;
        for (int pz = 0; pz < taps; ++pz) {
          if (wz[pz] == 0.0) continue;
          const double wt = wxy * wz[pz];
          double2* c = row + nu_wrap(m0z + pz - g.w, g.mz);
          atomicAdd(&c->x, v.x * wt);
          atomicAdd(&c->y, v.y * wt);
        }
      }
    }
  }
}

__global__ void nu_interp3(NuGeom3 g, const double2* __restrict__ grid, const double* __restrict__ pos, long long npts,
                           double2* out) {
  double wx[kNuMaxTaps], wy[kNuMaxTaps], wz[kNuMaxTaps];
  const int taps = 2 * g.w + 1;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x) {
    long long m0x, m0y, m0z;
    nu_weights(nu_axis_t(pos[3 * j], g.lx, g.mx), g.mx, g, m0x, wx);
    nu_weights(nu_axis_t(pos[3 * j + 1], g.ly, g.my), g.my, g, m0y, wy);
    nu_weights(nu_axis_t(pos[3 * j + 2], g.lz, g.mz), g.mz, g, m0z, wz);
    double2 acc = make_double2(0.0, 0.0);
    for (int px = 0; px < taps; ++px) {
      if (wx[px] == 0.0) continue;
      const long long ix = nu_wrap(m0x + px - g.w, g.mx);
      for (int py = 0; py < taps; ++py) {
        if (wy[py] == 0.0) continue;
        const long long iy = nu_wrap(m0y + py - g.w, g.my);
        const double wxy = wx[px] * wy[py];
        const double2* row = grid + (ix * g.my + iy) * g.mz;
        for (int pz = 0; pz < taps; ++pz) {
          if (wz[pz] == 0.0) continue;
          const double wt = wxy * wz[pz];
          const double2 c = row[nu_wrap(m0z + pz - g.w, g.mz)];
          acc.x += c.x * wt;
          acc.y += c.y * wt;
        }
      }
    }
    out[j] = acc;
  }
}

// modes[kx][ky][kz] <-> grid[kx_signed mod mx][ky_signed mod my][kz_signed mod mz], times dx dy dz deconvolution.
__global__ void nu_modes3(long long nx, long long ny, long long nz, long long mx, long long my, long long mz,
                          const double* __restrict__ dcx, const double* __restrict__ dcy, const double* __restrict__ dcz,
                          const double2* src, double2* dst, int to_grid) {
  const long long total = nx * ny * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long kz = e % nz, ky = (e / nz) % ny, kx = e / (ny * nz);
    const long long gi = (nu_bin(kx, nx, mx) * my + nu_bin(ky, ny, my)) * mz + nu_bin(kz, nz, mz);
    const double f = dcx[kx] * dcy[ky] * dcz[kz];
    if (to_grid) {
      const double2 c = src[e];
      dst[gi] = make_double2(c.x * f, c.y * f);
    } else {
      const double2 c = src[gi];
      dst[e] = make_double2(c.x * f, c.y * f);
    }
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

static NuGeom3 geom3(const NuLaunch3& L) {
  return NuGeom3{L.mx, L.my, L.mz, L.w, L.beta, L.i0b, L.lx, L.ly, L.lz};
}

cudaError_t nufft3_spread_dev(const NuLaunch3& L, const double* pos, const void* val, long long npts, void* grid,
                              cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  nu_spread3<<<nu_grid(npts), 128, 0, st>>>(geom3(L), pos, static_cast<const double2*>(val), npts,
                                            static_cast<double2*>(grid));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft3_interp_dev(const NuLaunch3& L, const void* grid, const double* pos, long long npts, void* out,
                              cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  nu_interp3<<<nu_grid(npts), 128, 0, st>>>(geom3(L), static_cast<const double2*>(grid), pos, npts,
                                            static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft3_modes_dev(const NuLaunch3& L, const double* dcx, const double* dcy, const double* dcz,
                             const void* src, void* dst, bool to_grid, cudaStream_t st) {
  nu_modes3<<<nu_grid(L.nx * L.ny * L.nz), 256, 0, st>>>(L.nx, L.ny, L.nz, L.mx, L.my, L.mz, dcx, dcy, dcz,
                                                         static_cast<const double2*>(src), static_cast<double2*>(dst),
                                                         to_grid ? 1 : 0);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
