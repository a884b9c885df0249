// afc_callers.cu -- element-wise and solver kernels of the fused caller
// operations whose transform does not fit one CTA: STFT frame gather, CZT chirp
// products around a multi-pass FFT, and the inverse CZT's Vandermonde solve.
#include <cuda_runtime.h>
#include "afc_internal.h"

namespace afc {

// ─────────────────────────── STFT frame gather ───────────────────────────
// apollo-stft's analysis frames (stft/dimension_1d.rs:96-108, 225-239): frame
// m holds signal[m hop - frame_len / 2 + i] * window[i] (zero outside the
// signal), as complex numbers, one frame per row of `out`.
template <class T>
__global__ void stft_gather(const T* __restrict__ sig, const T* __restrict__ win, long long nsig, long long flen,
                            long long hop, long long frames, typename CT<T>::type* __restrict__ out) {
  using C = typename CT<T>::type;
  const long long total = frames * flen;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long m = e / flen, i = e % flen;
    const long long s = m * hop - flen / 2 + i;
    const T v = (s >= 0 && s < nsig) ? sig[s] * win[i] : (T)0;
    out[e] = C{v, (T)0};
  }
}

cudaError_t stft_gather_dev(const void* sig, const void* win, long long nsig, long long flen, long long hop,
                            long long frames, void* out, bool dbl, cudaStream_t st) {
  const long long total = frames * flen;
  if (total <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148LL * 16);
  if (dbl)
    stft_gather<double><<<grid, 256, 0, st>>>(static_cast<const double*>(sig), static_cast<const double*>(win), nsig,
                                              flen, hop, frames, static_cast<double2*>(out));
  else
    stft_gather<float><<<grid, 256, 0, st>>>(static_cast<const float*>(sig), static_cast<const float*>(win), nsig,
                                             flen, hop, frames, static_cast<float2*>(out));
  count_launch(1);
  return cudaGetLastError();
}

// ─────────────────────────── CZT chirp products ───────────────────────────
// dst[b, i] = src[b, i] * table[i] for i < valid, 0 for valid <= i < nout
// (b < batch; row strides ss and ds).  One kernel serves apollo-czt's
// premultiply into the zero-padded convolution, the kernel-spectrum product
// and the postmultiply of the first m bins (kernel/bluestein.rs:83-130).
template <class T>
__global__ void chirp_rows(const typename CT<T>::type* src, long long ss, long long valid,
                           const typename CT<T>::type* __restrict__ table, typename CT<T>::type* dst, long long ds,
                           long long nout, long long batch) {
  using C = typename CT<T>::type;
  const long long total = batch * nout;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long b = e / nout, i = e % nout;
    C v{(T)0, (T)0};
    if (i < valid) v = cmul(src[b * ss + i], table[i]);
    dst[b * ds + i] = v;
  }
}

cudaError_t chirp_rows_dev(const void* src, long long ss, long long valid, const void* table, void* dst, long long ds,
                           long long nout, long long batch, bool dbl, cudaStream_t st) {
  const long long total = batch * nout;
  if (total <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148LL * 16);
  if (dbl)
    chirp_rows<double><<<grid, 256, 0, st>>>(static_cast<const double2*>(src), ss, valid,
                                             static_cast<const double2*>(table), static_cast<double2*>(dst), ds, nout,
                                             batch);
  else
    chirp_rows<float><<<grid, 256, 0, st>>>(static_cast<const float2*>(src), ss, valid,
                                            static_cast<const float2*>(table), static_cast<float2*>(dst), ds, nout,
                                            batch);
  count_launch(1);
  return cudaGetLastError();
}

// ─────────────────────────── inverse CZT ───────────────────────────
// apollo-czt's exact inverse of a square CZT (czt_bjork_pereyra_inverse_into,
// kernel/bluestein.rs:181-223): the Björck-Pereyra solve of the Vandermonde
// system on the nodes z_k = W^k, then x_k = y_k A^k.  One CTA per spectrum,
// in FP64 like the reference (complex64 plans convert on load and store).
// Every pass of a phase reads only the previous pass's values, so its updates
// are independent: the passes ping-pong between two shared arrays.
//   phase 1, j = 0 .. n-2, k > j:      c_k = (c_k - c_{k-1}) / (z_k - z_{k-j-1})
//   phase 2, j = n-2 .. 0, j <= k < n-1: c_k = c_k - z_j c_{k+1}
__device__ __forceinline__ double2 cdiv_ref(double2 a, double2 b) {
  // num-complex's division: (a conj(b)) / |b|^2
  const double nrm = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / nrm, (a.y * b.x - a.x * b.y) / nrm);
}

template <class C>
__device__ __forceinline__ double2 to_d2(C v) {
  return make_double2((double)v.x, (double)v.y);
}

template <class T>
__global__ void __launch_bounds__(256) czt_inverse_kernel(const typename CT<T>::type* __restrict__ spec,
                                                          typename CT<T>::type* __restrict__ out,
                                                          const double2* __restrict__ nodes,
                                                          const double2* __restrict__ apow, int n) {
  using C = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char czt_smem[];
  double2* a = reinterpret_cast<double2*>(czt_smem);
  double2* b = a + n;
  const long long lane = blockIdx.x;
  const C* y = spec + lane * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) a[k] = to_d2(y[k]);
  __syncthreads();
  double2* src = a;
  double2* dst = b;
  for (int j = 0; j + 1 < n; ++j) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      if (k > j) {
        const double2 zk = nodes[k], zl = nodes[k - j - 1];
        const double2 num = make_double2(src[k].x - src[k - 1].x, src[k].y - src[k - 1].y);
        dst[k] = cdiv_ref(num, make_double2(zk.x - zl.x, zk.y - zl.y));
      } else {
        dst[k] = src[k];
      }
    }
    __syncthreads();
    double2* t = src;
    src = dst;
    dst = t;
  }
  for (int j = n - 2; j >= 0; --j) {
    const double2 zj = nodes[j];
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      if (k >= j && k < n - 1) {
        const double2 c1 = src[k + 1];
        dst[k] = make_double2(src[k].x - (zj.x * c1.x - zj.y * c1.y), src[k].y - (zj.x * c1.y + zj.y * c1.x));
      } else {
        dst[k] = src[k];
      }
    }
    __syncthreads();
    double2* t = src;
    src = dst;
    dst = t;
  }
  C* x = out + lane * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double2 v = src[k], p = apow[k];
    x[k] = C{(T)(v.x * p.x - v.y * p.y), (T)(v.x * p.y + v.y * p.x)};
  }
}

size_t czt_inverse_smem(long long n) { return 2 * (size_t)n * sizeof(double2); }

cudaError_t czt_inverse_dev(const void* spec, void* out, const void* nodes, const void* apow, long long n,
                            long long batch, bool dbl, cudaStream_t st) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  const size_t smem = czt_inverse_smem(n);
  const void* k = dbl ? reinterpret_cast<const void*>(czt_inverse_kernel<double>)
                      : reinterpret_cast<const void*>(czt_inverse_kernel<float>);
  cudaError_t e = kernel_smem_grant(k, smem);
  if (e != cudaSuccess) return e;
  if (dbl)
    czt_inverse_kernel<double><<<(unsigned)batch, 256, smem, st>>>(
        static_cast<const double2*>(spec), static_cast<double2*>(out), static_cast<const double2*>(nodes),
        static_cast<const double2*>(apow), (int)n);
  else
    czt_inverse_kernel<float><<<(unsigned)batch, 256, smem, st>>>(
        static_cast<const float2*>(spec), static_cast<float2*>(out), static_cast<const double2*>(nodes),
        static_cast<const double2*>(apow), (int)n);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
