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

// I0(z) = sum_k ((z/2)^2)^k / (k!)^2: term_k = term_{k-1} (z/2)^2 / k^2, the
// ratios from a table of 1/k^2 (so the running product is a chain of
// multiplies, not divides), summed four terms at a time until the last of them
// drops below epsilon of the sum (at most 256 terms).  The terms the reference
// would not add are below epsilon of the sum.
struct NuInvSquares {
  double v[257];
  constexpr NuInvSquares() : v() {
    for (int k = 1; k <= 256; ++k) v[k] = 1.0 / ((double)k * (double)k);
  }
};
__constant__ NuInvSquares c_nu_inv_k2 = NuInvSquares();

__device__ __forceinline__ double nu_i0(double z) {
  const double scaled = 0.25 * z * z;
  double sum = 1.0, term = 1.0;
  for (int k = 1; k <= 256; k += 4) {
    const double q0 = scaled * c_nu_inv_k2.v[k], q1 = scaled * c_nu_inv_k2.v[k + 1];
    const double q2 = scaled * c_nu_inv_k2.v[k + 2], q3 = scaled * c_nu_inv_k2.v[k + 3];
    term *= q0;
    sum += term;
    term *= q1;
    sum += term;
    term *= q2;
    sum += term;
    term *= q3;
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
// Separable kernel: weight = phi_x phi_y phi_z over T^3 taps, T = 2w + 1; grid
// C-order [ix][iy][iz] of size mx x my x mz, every m a power of two.
// One warp per point: the lanes evaluate the 3T axis weights into shared
// memory, then walk the T x T (py, pz) plane flattened over the 32 lanes for
// every px, so one warp instruction touches two or three contiguous runs of T
// cells (T = 13: 6 instructions per plane) instead of 32 scattered cells.
struct NuGeom3 {
  long long mx, my, mz;
  int w;
  double beta, i0b;
  double lx, ly, lz;
};

constexpr int kNuMaxTaps = 65;       // T for w <= 32
constexpr int kNuWarps = 8;          // warps (points in flight) per 256-thread CTA

__device__ __forceinline__ double nu_axis_t(double x, double len, long long m) {
  double r = fmod(x, len);
  if (r < 0.0) r += len;
  return (double)m * r / len;
}

// Lanes fill wt[0..T) for one axis and return m0 (the same in every lane).
__device__ __forceinline__ long long nu_axis_weights(double x, double len, long long m, const NuGeom3& g, int lane,
                                                     double* wt) {
  const double t = nu_axis_t(x, len, m);
  const double rt = round(t);
  const double d = t - rt;
  for (int p = lane; p <= 2 * g.w; p += 32) wt[p] = nu_kb((double)(p - g.w) - d, (double)g.w, g.beta, g.i0b);
  return (long long)rt;
}

struct NuPlaneWalk {  // lane's (py, pz) start and the constant stride of 32 flattened cells
  int py0, pz0, dpy, dpz, iters;
  __device__ NuPlaneWalk(int T, int lane)
      : py0(lane / T), pz0(lane % T), dpy(32 / T), dpz(32 % T), iters((T * T + 31) / 32) {}
};

__global__ void __launch_bounds__(32 * kNuWarps) nu_spread3(NuGeom3 g, const double* __restrict__ pos,
                                                              const double2* __restrict__ val, long long npts,
                                                              double2* grid) {
  __shared__ double sw[kNuWarps][3][kNuMaxTaps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int T = 2 * g.w + 1;
  const NuPlaneWalk pw(T, lane);
  const long long mxm = g.mx - 1, mym = g.my - 1, mzm = g.mz - 1;
  double* wx = sw[wid][0];
  double* wy = sw[wid][1];
  double* wz = sw[wid][2];
  const long long warps = (long long)gridDim.x * kNuWarps;
  for (long long j = (long long)blockIdx.x * kNuWarps + wid; j < npts; j += warps) {
    const long long m0x = nu_axis_weights(pos[3 * j], g.lx, g.mx, g, lane, wx);
    const long long m0y = nu_axis_weights(pos[3 * j + 1], g.ly, g.my, g, lane, wy);
    const long long m0z = nu_axis_weights(pos[3 * j + 2], g.lz, g.mz, g, lane, wz);
    const double2 v = val[j];
    __syncwarp();
    for (int px = 0; px < T; ++px) {
      const double wxv = wx[px];
      if (wxv == 0.0) continue;
      double2* plane = grid + ((m0x + px - g.w) & mxm) * g.my * g.mz;
      int py = pw.py0, pz = pw.pz0;
      for (int it = 0; it < pw.iters; ++it) {
        if (py < T) {
          const double wt = wxv * wy[py] * wz[pz];
          if (wt != 0.0) {
            double2* c = plane + ((m0y + py - g.w) & mym) * g.mz + ((m0z + pz - g.w) & mzm);
            atomicAdd(&c->x, v.x * wt);
            atomicAdd(&c->y, v.y * wt);
          }
        }
        py += pw.dpy;
        pz += pw.dpz;
        if (pz >= T) pz -= T, ++py;
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(32 * kNuWarps) nu_interp3(NuGeom3 g, const double2* __restrict__ grid,
                                                              const double* __restrict__ pos, long long npts,
                                                              double2* out) {
  __shared__ double sw[kNuWarps][3][kNuMaxTaps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int T = 2 * g.w + 1;
  const NuPlaneWalk pw(T, lane);
  const long long mxm = g.mx - 1, mym = g.my - 1, mzm = g.mz - 1;
  double* wx = sw[wid][0];
  double* wy = sw[wid][1];
  double* wz = sw[wid][2];
  const long long warps = (long long)gridDim.x * kNuWarps;
  for (long long j = (long long)blockIdx.x * kNuWarps + wid; j < npts; j += warps) {
    const long long m0x = nu_axis_weights(pos[3 * j], g.lx, g.mx, g, lane, wx);
    const long long m0y = nu_axis_weights(pos[3 * j + 1], g.ly, g.my, g, lane, wy);
    const long long m0z = nu_axis_weights(pos[3 * j + 2], g.lz, g.mz, g, lane, wz);
    __syncwarp();
    double ax = 0.0, ay = 0.0;
    for (int px = 0; px < T; ++px) {
      const double wxv = wx[px];
      if (wxv == 0.0) continue;
      const double2* plane = grid + ((m0x + px - g.w) & mxm) * g.my * g.mz;
      int py = pw.py0, pz = pw.pz0;
      for (int it = 0; it < pw.iters; ++it) {
        if (py < T) {
          const double wt = wxv * wy[py] * wz[pz];
          if (wt != 0.0) {
            const double2 c = plane[((m0y + py - g.w) & mym) * g.mz + ((m0z + pz - g.w) & mzm)];
            ax += c.x * wt;
            ay += c.y * wt;
          }
        }
        py += pw.dpy;
        pz += pw.dpz;
        if (pz >= T) pz -= T, ++py;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (lane == 0) out[j] = make_double2(ax, ay);
    __syncwarp();
  }
}

// ─── tiled 3D spreading / interpolation ───
// Points are bucketed by the B^3 tile of cells that holds their centre cell
// round(t) mod m (the reference bucket-sorts its points too, sort_points_3d,
// dimension_3d.rs:74-117); one CTA per tile keeps the tile and its w-cell halo,
// E^3 cells with E = B + 2w, in shared memory.  Spreading: warp k owns the
// x-planes lx = k mod 16 of the tile and adds every point's taps on its planes
// with plain shared-memory read-modify-writes (no two warps share a cell),
// then the CTA adds its E^3 cells to the grid with coalesced atomics (tiles'
// halos overlap); grid atomics drop from (2w+1)^3 per point to E^3 per tile.
// Interpolation: the CTA loads its E^3 cells once, stages the weights of 64
// points at a time with all its threads, and one warp per point gathers from
// shared memory.
constexpr int kNuTileThreads = 512;
constexpr int kNuTileWarps = kNuTileThreads / 32;
constexpr int kNuChunk = 64;  // points whose weights a tile CTA stages at once

struct NuTiles {
  int B, E, nty, ntz;
  const int* off;  // ntiles + 1 offsets into idx
  const int* idx;  // point indices grouped by tile
};

__device__ __forceinline__ int nu_centre(double x, double len, long long m) {
  return (int)((long long)round(nu_axis_t(x, len, m)) & (m - 1));
}

__global__ void nu3_bin(NuGeom3 g, int B, int nty, int ntz, const double* __restrict__ pos, long long npts,
                        int* __restrict__ cnt, int* __restrict__ tile, int* __restrict__ rank) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x) {
    const int cx = nu_centre(pos[3 * j], g.lx, g.mx);
    const int cy = nu_centre(pos[3 * j + 1], g.ly, g.my);
    const int cz = nu_centre(pos[3 * j + 2], g.lz, g.mz);
    const int t = ((cx / B) * nty + cy / B) * ntz + cz / B;
    tile[j] = t;
    rank[j] = atomicAdd(&cnt[t], 1);
  }
}

// Exclusive prefix sum of cnt[0..n) into off[0..n], one CTA of 1024 threads,
// each over a contiguous chunk.
__global__ void __launch_bounds__(1024) nu3_scan(const int* __restrict__ cnt, int* __restrict__ off, int n) {
  __shared__ int wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int per = (n + 1023) / 1024;
  const int lo = min(n, tid * per), hi = min(n, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += cnt[i];
  int v = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  int ex = v - s + (wid > 0 ? wsum[wid - 1] : 0);
  for (int i = lo; i < hi; ++i) {
    off[i] = ex;
    ex += cnt[i];
  }
  if (tid == 1023) off[n] = ex;
}

__global__ void nu3_scatter(const int* __restrict__ tile, const int* __restrict__ rank, const int* __restrict__ off,
                            long long npts, int* __restrict__ idx) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts; j += (long long)gridDim.x * blockDim.x)
    idx[off[tile[j]] + rank[j]] = (int)j;
}

struct NuTileCoord {
  int tx, ty, tz;
  __device__ NuTileCoord(int tile, const NuTiles& tl)
      : tx(tile / (tl.nty * tl.ntz)), ty((tile / tl.ntz) % tl.nty), tz(tile % tl.ntz) {}
};

// Axis-a weight of tap `tap` for the point at pos, and (lc non-null) the
// point's centre cell relative to the tile origin, in [0, B).
__device__ __forceinline__ double nu_tile_weight(const NuGeom3& g, const NuTiles& tl, const NuTileCoord& tc,
                                                 const double* pos, int a, int tap, int* lc) {
  const double len = a == 0 ? g.lx : a == 1 ? g.ly : g.lz;
  const long long m = a == 0 ? g.mx : a == 1 ? g.my : g.mz;
  const int t0 = a == 0 ? tc.tx : a == 1 ? tc.ty : tc.tz;
  const double t = nu_axis_t(pos[a], len, m);
  const double rt = round(t);
  if (lc) *lc = (int)((long long)rt & (m - 1)) - t0 * tl.B;
  return nu_kb((double)(tap - g.w) - (t - rt), (double)g.w, g.beta, g.i0b);
}

// The lane's cells of a T x T (py, pz) plane: at most kNuTileIters, packed
// py << 8 | pz (-1 past the plane), fixed for the whole kernel.
constexpr int kNuTileIters = 12;  // ceil(T^2 / 32) for T <= 19 (w <= 9)

struct NuLaneCells {
  int pyz[kNuTileIters];
  __device__ NuLaneCells(int T, int lane) {
#pragma unroll
    for (int it = 0; it < kNuTileIters; ++it) {
      const int f = it * 32 + lane;
      pyz[it] = f < T * T ? ((f / T) << 8) | (f % T) : -1;
    }
  }
};

__global__ void __launch_bounds__(kNuTileThreads) nu3_spread_tiles(NuGeom3 g, NuTiles tl,
                                                                    const double* __restrict__ pos,
                                                                    const double2* __restrict__ val, double2* grid) {
  extern __shared__ __align__(16) unsigned char nu_smem[];
  const int tile = blockIdx.x;
  const int start = tl.off[tile], end = tl.off[tile + 1];
  if (start == end) return;
  const int T = 2 * g.w + 1, E = tl.E, E2 = E * E, E3 = E2 * E;
  double2* acc = reinterpret_cast<double2*>(nu_smem);
  double* wts = reinterpret_cast<double*>(acc + E3);       // kNuChunk x 3 x T
  int* loc = reinterpret_cast<int*>(wts + kNuChunk * 3 * T);  // kNuChunk x 3
  for (int c = threadIdx.x; c < E3; c += kNuTileThreads) acc[c] = make_double2(0.0, 0.0);
  const NuTileCoord tc(tile, tl);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const NuLaneCells lc(T, lane);
  for (int base = start; base < end; base += kNuChunk) {
    const int cnt = min(kNuChunk, end - base);
    __syncthreads();  // zeroing done / previous chunk's weights consumed
    for (int e = threadIdx.x; e < cnt * 3 * T; e += kNuTileThreads) {
      const int p = e / (3 * T), r = e - p * 3 * T, a = r / T, tap = r - a * T;
      const long long j = tl.idx[base + p];
      wts[e] = nu_tile_weight(g, tl, tc, pos + 3 * j, a, tap, tap == 0 ? &loc[p * 3 + a] : nullptr);
    }
    __syncthreads();
    for (int p = 0; p < cnt; ++p) {
      const int lx0 = loc[p * 3], ly0 = loc[p * 3 + 1], lz0 = loc[p * 3 + 2];
      int px = (wid - lx0) % kNuTileWarps;
      if (px < 0) px += kNuTileWarps;
      if (px >= T) continue;  // warp-uniform: none of this point's planes is ours
      const double* wx = wts + p * 3 * T;
      const double* wy = wx + T;
      const double* wz = wy + T;
      const double2 v = val[tl.idx[base + p]];
      for (; px < T; px += kNuTileWarps) {
        const double wxv = wx[px];
        double2* plane = acc + (lx0 + px) * E2 + ly0 * E + lz0;
        // six of the lane's cells at a time: all loads first, then the adds and
        // stores (the lane's cells are distinct, and so are different lanes'),
        // so six shared-memory loads are in flight instead of one
#pragma unroll
        for (int h = 0; h < kNuTileIters; h += 6) {
          if (h * 32 >= T * T) break;
          double2 cv[6];
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            const int f = lc.pyz[h + i];
            if (f >= 0) cv[i] = plane[(f >> 8) * E + (f & 255)];
          }
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            const int f = lc.pyz[h + i];
            if (f >= 0) {
              const double wt = wxv * wy[f >> 8] * wz[f & 255];
              cv[i].x += v.x * wt;
              cv[i].y += v.y * wt;
              plane[(f >> 8) * E + (f & 255)] = cv[i];
            }
          }
        }
      }
      __syncwarp();  // the next point's lanes may touch the cells written here
    }
  }
  __syncthreads();
  const long long mxm = g.mx - 1, mym = g.my - 1, mzm = g.mz - 1;
  const long long gx0 = (long long)tc.tx * tl.B - g.w, gy0 = (long long)tc.ty * tl.B - g.w,
                  gz0 = (long long)tc.tz * tl.B - g.w;
  for (int c = threadIdx.x; c < E3; c += kNuTileThreads) {
    const double2 a = acc[c];
    if (a.x == 0.0 && a.y == 0.0) continue;
    const int cx = c / E2, cy = (c / E) % E, cz = c % E;
    double2* d = grid + (((gx0 + cx) & mxm) * g.my + ((gy0 + cy) & mym)) * g.mz + ((gz0 + cz) & mzm);
    atomicAdd(&d->x, a.x);
    atomicAdd(&d->y, a.y);
  }
}

__global__ void __launch_bounds__(kNuTileThreads) nu3_interp_tiles(NuGeom3 g, NuTiles tl,
                                                                    const double2* __restrict__ grid,
                                                                    const double* __restrict__ pos, double2* out) {
  extern __shared__ __align__(16) unsigned char nu_smem[];
  const int tile = blockIdx.x;
  const int start = tl.off[tile], end = tl.off[tile + 1];
  if (start == end) return;
  const int T = 2 * g.w + 1, E = tl.E, E2 = E * E, E3 = E2 * E;
  double2* cells = reinterpret_cast<double2*>(nu_smem);
  double* wts = reinterpret_cast<double*>(cells + E3);       // kNuChunk x 3 x T
  int* loc = reinterpret_cast<int*>(wts + kNuChunk * 3 * T);  // kNuChunk x 3
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const NuTileCoord tc(tile, tl);
  const long long mxm = g.mx - 1, mym = g.my - 1, mzm = g.mz - 1;
  const long long gx0 = (long long)tc.tx * tl.B - g.w, gy0 = (long long)tc.ty * tl.B - g.w,
                  gz0 = (long long)tc.tz * tl.B - g.w;
  for (int c = threadIdx.x; c < E3; c += kNuTileThreads) {
    const int cx = c / E2, cy = (c / E) % E, cz = c % E;
    cells[c] = grid[(((gx0 + cx) & mxm) * g.my + ((gy0 + cy) & mym)) * g.mz + ((gz0 + cz) & mzm)];
  }
  const NuLaneCells lc(T, lane);
  int coff[kNuTileIters];
#pragma unroll
  for (int it = 0; it < kNuTileIters; ++it) coff[it] = lc.pyz[it] >= 0 ? (lc.pyz[it] >> 8) * E + (lc.pyz[it] & 255) : 0;
  for (int base = start; base < end; base += kNuChunk) {
    const int cnt = min(kNuChunk, end - base);
    __syncthreads();  // cells loaded / previous chunk's weights consumed
    // the chunk's 3T axis weights per point over all threads of the CTA
    for (int e = threadIdx.x; e < cnt * 3 * T; e += kNuTileThreads) {
      const int p = e / (3 * T), r = e - p * 3 * T, a = r / T, tap = r - a * T;
      const long long j = tl.idx[base + p];
      wts[e] = nu_tile_weight(g, tl, tc, pos + 3 * j, a, tap, tap == 0 ? &loc[p * 3 + a] : nullptr);
    }
    __syncthreads();
    for (int p = wid; p < cnt; p += kNuTileWarps) {
      const double* wx = wts + p * 3 * T;
      const double* wy = wx + T;
      const double* wz = wy + T;
      double wyz[kNuTileIters];
#pragma unroll
      for (int it = 0; it < kNuTileIters; ++it)
        wyz[it] = lc.pyz[it] >= 0 ? wy[lc.pyz[it] >> 8] * wz[lc.pyz[it] & 255] : 0.0;
      // two accumulator pairs (even / odd cells) halve the dependent FMA chain
      double ax0 = 0.0, ay0 = 0.0, ax1 = 0.0, ay1 = 0.0;
      const double2* plane = cells + loc[p * 3] * E2 + loc[p * 3 + 1] * E + loc[p * 3 + 2];
      for (int px = 0; px < T; ++px, plane += E2) {
        const double wxv = wx[px];
#pragma unroll
        for (int it = 0; it < kNuTileIters; ++it) {
          if (lc.pyz[it] >= 0) {
            const double wt = wxv * wyz[it];
            const double2 c = plane[coff[it]];
            if (it & 1) {
              ax1 += c.x * wt;
              ay1 += c.y * wt;
            } else {
              ax0 += c.x * wt;
              ay0 += c.y * wt;
            }
          }
        }
      }
      double ax = ax0 + ax1, ay = ay0 + ay1;
      for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
      }
      if (lane == 0) out[tl.idx[base + p]] = make_double2(ax, ay);
    }
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

static unsigned nu_warp_grid(long long npts) {
  long long b = (npts + kNuWarps - 1) / kNuWarps;
  return (unsigned)(b < 148 * 8 ? b : 148 * 8);
}

cudaError_t nufft3_spread_dev(const NuLaunch3& L, const double* pos, const void* val, long long npts, void* grid,
                              cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  nu_spread3<<<nu_warp_grid(npts), 32 * kNuWarps, 0, st>>>(geom3(L), pos, static_cast<const double2*>(val), npts,
                                            static_cast<double2*>(grid));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nufft3_interp_dev(const NuLaunch3& L, const void* grid, const double* pos, long long npts, void* out,
                              cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  nu_interp3<<<nu_warp_grid(npts), 32 * kNuWarps, 0, st>>>(geom3(L), static_cast<const double2*>(grid), pos, npts,
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

int nufft3_tile_size(int w) {
  if ((2 * w + 1) * (2 * w + 1) > 32 * kNuTileIters) return 0;  // more plane cells than a lane's list holds
  for (int B : {8, 4})
    if (nufft3_tile_smem(B, w) <= 220 * 1024) return B;
  return 0;
}

size_t nufft3_tile_smem(int B, int w) {
  const size_t E = (size_t)(B + 2 * w), T = (size_t)(2 * w + 1);
  const size_t cells = E * E * E * sizeof(double2);
  // both kernels stage the axis weights and centre cells of kNuChunk points
  return cells + kNuChunk * 3 * T * sizeof(double) + kNuChunk * 3 * sizeof(int);
}

cudaError_t nufft3_tiled_dev(const NuLaunch3& L, const NuTileLaunch& TL, bool spread, const double* pos,
                             const void* src, long long npts, void* dst, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  const NuGeom3 g = geom3(L);
  const int ntiles = TL.ntx * TL.nty * TL.ntz;
  cudaError_t e = cudaMemsetAsync(TL.cnt, 0, (size_t)ntiles * sizeof(int), st);
  if (e != cudaSuccess) return e;
  nu3_bin<<<nu_grid(npts), 256, 0, st>>>(g, TL.B, TL.nty, TL.ntz, pos, npts, TL.cnt, TL.tile, TL.rank);
  nu3_scan<<<1, 1024, 0, st>>>(TL.cnt, TL.off, ntiles);
  nu3_scatter<<<nu_grid(npts), 256, 0, st>>>(TL.tile, TL.rank, TL.off, npts, TL.idx);
  const NuTiles tl{TL.B, TL.B + 2 * L.w, TL.nty, TL.ntz, TL.off, TL.idx};
  const size_t smem = nufft3_tile_smem(TL.B, L.w);
  if (spread) {
    e = kernel_smem_grant(reinterpret_cast<const void*>(nu3_spread_tiles), smem);
    if (e != cudaSuccess) return e;
    nu3_spread_tiles<<<ntiles, kNuTileThreads, smem, st>>>(g, tl, pos, static_cast<const double2*>(src),
                                                           static_cast<double2*>(dst));
  } else {
    e = kernel_smem_grant(reinterpret_cast<const void*>(nu3_interp_tiles), smem);
    if (e != cudaSuccess) return e;
    nu3_interp_tiles<<<ntiles, kNuTileThreads, smem, st>>>(g, tl, static_cast<const double2*>(src), pos,
                                                           static_cast<double2*>(dst));
  }
  count_launch(4);
  return cudaGetLastError();
}

// ───────────────────── exact direct non-uniform DFTs ─────────────────────
// apollo-nufft's exact direct sums (transform/dimension_1d.rs:428-472,
// dimension_3d.rs:677-712): every output is the full sum over the inputs with
// the phase (2 pi / L) k x, k the FFT-signed index (k <= n/2 stays, else
// k - n; kaiser_bessel.rs:152-158), evaluated in FP64 like the reference.
// One thread per output; the inputs stream through shared memory in chunks of
// the block size, so each is read from global memory once per block.

constexpr int kDirectThreads = 256;
constexpr double kTwoPi = 6.283185307179586476925286766559;  // 2 pi

__device__ __forceinline__ long long direct_signed(long long k, long long n) { return k <= n / 2 ? k : k - n; }

// out[k] = sum_j v_j exp(-i (2 pi / L) k_s x_j), k < n
__global__ void __launch_bounds__(kDirectThreads) nudft1_type1(const double* __restrict__ pos,
                                                               const double2* __restrict__ val, long long npts,
                                                               long long n, double two_pi_over_l, double2* out) {
  __shared__ double sx[kDirectThreads];
  __shared__ double2 sv[kDirectThreads];
  const long long k = (long long)blockIdx.x * kDirectThreads + threadIdx.x;
  const double ks = (double)direct_signed(k < n ? k : 0, n);
  double re = 0.0, im = 0.0;
  for (long long j0 = 0; j0 < npts; j0 += kDirectThreads) {
    const long long j = j0 + threadIdx.x;
    __syncthreads();
    if (j < npts) {
      sx[threadIdx.x] = pos[j];
      sv[threadIdx.x] = val[j];
    }
    __syncthreads();
    const int cnt = (int)(npts - j0 < kDirectThreads ? npts - j0 : kDirectThreads);
    for (int i = 0; i < cnt; ++i) {
      const double angle = -two_pi_over_l * ks * sx[i];
      double sn, cs;
      sincos(angle, &sn, &cs);
      const double2 v = sv[i];
      re += v.x * cs - v.y * sn;
      im += v.x * sn + v.y * cs;
    }
  }
  if (k < n) out[k] = make_double2(re, im);
}

// out[j] = sum_k c_k exp(+i (2 pi / L) k_s x_j), j < npts
__global__ void __launch_bounds__(kDirectThreads) nudft1_type2(const double2* __restrict__ coeffs, long long n,
                                                               const double* __restrict__ pos, long long npts,
                                                               double two_pi_over_l, double2* out) {
  __shared__ double2 sc[kDirectThreads];
  const long long j = (long long)blockIdx.x * kDirectThreads + threadIdx.x;
  const double x = j < npts ? pos[j] : 0.0;
  double re = 0.0, im = 0.0;
  for (long long k0 = 0; k0 < n; k0 += kDirectThreads) {
    __syncthreads();
    if (k0 + threadIdx.x < n) sc[threadIdx.x] = coeffs[k0 + threadIdx.x];
    __syncthreads();
    const int cnt = (int)(n - k0 < kDirectThreads ? n - k0 : kDirectThreads);
    for (int i = 0; i < cnt; ++i) {
      const double angle = two_pi_over_l * (double)direct_signed(k0 + i, n) * x;
      double sn, cs;
      sincos(angle, &sn, &cs);
      const double2 c = sc[i];
      re += c.x * cs - c.y * sn;
      im += c.x * sn + c.y * cs;
    }
  }
  if (j < npts) out[j] = make_double2(re, im);
}

// out[kx, ky, kz] = sum_j v_j exp(-i (wx kx_s x_j + wy ky_s y_j + wz kz_s z_j))
__global__ void __launch_bounds__(kDirectThreads) nudft3_type1(const double* __restrict__ pos,
                                                               const double2* __restrict__ val, long long npts,
                                                               long long nx, long long ny, long long nz, double wx,
                                                               double wy, double wz, double2* out) {
  __shared__ double sp[3 * kDirectThreads];
  __shared__ double2 sv[kDirectThreads];
  const long long total = nx * ny * nz;
  const long long m = (long long)blockIdx.x * kDirectThreads + threadIdx.x;
  const long long mm = m < total ? m : 0;
  const double kx = (double)direct_signed(mm / (ny * nz), nx);
  const double ky = (double)direct_signed((mm / nz) % ny, ny);
  const double kz = (double)direct_signed(mm % nz, nz);
  double re = 0.0, im = 0.0;
  for (long long j0 = 0; j0 < npts; j0 += kDirectThreads) {
    const long long j = j0 + threadIdx.x;
    __syncthreads();
    if (j < npts) {
      sp[3 * threadIdx.x] = pos[3 * j];
      sp[3 * threadIdx.x + 1] = pos[3 * j + 1];
      sp[3 * threadIdx.x + 2] = pos[3 * j + 2];
      sv[threadIdx.x] = val[j];
    }
    __syncthreads();
    const int cnt = (int)(npts - j0 < kDirectThreads ? npts - j0 : kDirectThreads);
    for (int i = 0; i < cnt; ++i) {
      const double angle = -(wx * kx * sp[3 * i] + wy * ky * sp[3 * i + 1] + wz * kz * sp[3 * i + 2]);
      double sn, cs;
      sincos(angle, &sn, &cs);
      const double2 v = sv[i];
      re += v.x * cs - v.y * sn;
      im += v.x * sn + v.y * cs;
    }
  }
  if (m < total) out[m] = make_double2(re, im);
}

cudaError_t nudft1_type1_dev(const double* pos, const void* val, long long npts, long long n, double len, void* out,
                             cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((n + kDirectThreads - 1) / kDirectThreads);
  nudft1_type1<<<grid, kDirectThreads, 0, st>>>(pos, static_cast<const double2*>(val), npts, n, kTwoPi / len,
                                                static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nudft1_type2_dev(const void* coeffs, long long n, const double* pos, long long npts, double len, void* out,
                             cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((npts + kDirectThreads - 1) / kDirectThreads);
  nudft1_type2<<<grid, kDirectThreads, 0, st>>>(static_cast<const double2*>(coeffs), n, pos, npts, kTwoPi / len,
                                                static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t nudft3_type1_dev(const double* pos, const void* val, long long npts, long long nx, long long ny,
                             long long nz, double lx, double ly, double lz, void* out, cudaStream_t st) {
  const long long total = nx * ny * nz;
  if (total <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((total + kDirectThreads - 1) / kDirectThreads);
  nudft3_type1<<<grid, kDirectThreads, 0, st>>>(pos, static_cast<const double2*>(val), npts, nx, ny, nz,
                                                kTwoPi / lx, kTwoPi / ly, kTwoPi / lz,
                                                static_cast<double2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
