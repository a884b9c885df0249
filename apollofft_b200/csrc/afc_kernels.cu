// afc_kernels.cu -- sm_100a kernels of apollofft_b200 and their launchers.
//
// lanes_kernel     : L lanes per CTA through the Stockham engine; the global
//                    load/store operator is chosen per launch (complex, real
//                    widen, Hermitian expand, chirp premultiply / four-step
//                    twiddle, pointwise spectrum, real part, truncation,
//                    chirp postmultiply).
// conv_kernel      : a whole Rader or Bluestein transform per lane in shared
//                    memory: staged gather (generator order) or chirp
//                    premultiply, forward FFT, kernel-spectrum multiply,
//                    inverse FFT, staged scatter (+ x0, DC sum) or chirp
//                    postmultiply.
// table kernels    : FP64 generation of stage twiddles, two-level four-step
//                    twiddles, Bluestein chirps and Rader kernels, narrowed once.
#include <cuda_runtime.h>
#include <tuple>
#include <mutex>
#include <map>
#include <cstring>
#include "afc_engine.cuh"
#include "afc_internal.h"

namespace afc {

// ───────────────────────────── kernel arguments ─────────────────────────────

template <class T> struct KArgs {
  using C = typename CT<T>::type;
  StageList sl;
  const C* tw;
  long long lanes;
  int L, P, ld;
  int in_op, out_op;
  int stage_in, stage_out;
  LaneMap im, om;          // input / output lane maps
  const void* in;
  void* out;
  T scale;
  // element-index map of index-aware operators: j = i * jmul + col(q),
  // col(q) = (q / col_div) % col_mod.
  long long jmul, col_div, col_mod;
  long long nlen;          // valid length (chirp / truncation) or p (Rader)
  long long herm_n;        // full length behind a half spectrum
  T pair_w;                // Hermitian weight of paired bins (adjoints); 1 otherwise
  // four-step twiddle W_N^{(col * i) mod N} = hi[m / B] * lo[m % B], conj if tw_conj
  long long twN, twB;
  int tw_conj;
  const C* tw_hi;
  const C* tw_lo;
  const C* spec;           // pointwise spectrum
  long long spec_ld;       // convolution tiles: lane spectrum = spec + col * spec_ld (0: shared)
  const C* chirp;          // Bluestein chirp (forward sign; conj if chirp_conj)
  int chirp_conj;
  const int* gather;       // Rader: gather[q] = g^q mod p
  const int* scatter;      // Rader: scatter[q] = g^{-q} mod p
  int lane_minor;          // tile kernel: consecutive threads take consecutive lanes
  int in_sel, out_sel;     // batch descriptors: 0 absolute pointer, else base[sel] + offset
  const C* chirp_out;      // OUT_CHIRP: post-multiply table when it differs from chirp (CZT)
  long long nlen_out;      // OUT_CHIRP: outputs kept when > 0 (else nlen)
  const T* window;         // IN_FRAME: analysis window
  long long frame_off;     // IN_FRAME: frame q covers signal[q hop - frame_off + i]
};

template <class T>
__device__ __forceinline__ typename CT<T>::type gload(const KArgs<T>& a, long long base, long long col, int i) {
  using C = typename CT<T>::type;
  const C zero = C{(T)0, (T)0};
  switch (a.in_op) {
    case IN_C:
      return static_cast<const C*>(a.in)[base + (long long)i * a.im.es];
    case IN_R:  // real input widened (reference RealFftData, real_storage.rs:186-303)
      return C{static_cast<const T*>(a.in)[base + (long long)i * a.im.es], (T)0};
    case IN_HERM: {  // half spectrum (n/2+1 bins) expanded by Hermitian symmetry
      const C* p = static_cast<const C*>(a.in);
      const long long n = a.herm_n;
      C v;
      if (2LL * i <= n) {
        v = p[base + (long long)i * a.im.es];
      } else {
        v = p[base + (n - i) * a.im.es];
        v.y = -v.y;
      }
      if (i > 0 && 2LL * i != n) v = cscale(v, a.pair_w);
      return v;
    }
    case IN_CHIRP:
    case IN_CHIRP_R: {  // Bluestein premultiply x[j] * chirp[j], zero for j >= nlen
      const long long j = (long long)i * a.jmul + col;
      if (j >= a.nlen) return zero;
      const long long off = base + (long long)i * a.im.es;
      C x = a.in_op == IN_CHIRP ? static_cast<const C*>(a.in)[off] : C{static_cast<const T*>(a.in)[off], (T)0};
      const C c = a.chirp[j];
      return a.chirp_conj ? cmulc(x, c) : cmul(x, c);
    }
    case IN_GATHER:
    case IN_GATHER_R: {  // Rader: x[g^i] for i < p-1, zero padding beyond
      if (i >= a.nlen - 1) return zero;
      const long long off = base + (long long)a.gather[i] * a.im.es;
      return a.in_op == IN_GATHER ? static_cast<const C*>(a.in)[off] : C{static_cast<const T*>(a.in)[off], (T)0};
    }
    case IN_FRAME: {  // STFT analysis frame: signal[base - frame_off + i] * window[i], zero outside the signal
      const long long j = base - a.frame_off + i;
      if (j < 0 || j >= a.nlen) return zero;
      return C{static_cast<const T*>(a.in)[j] * a.window[i], (T)0};
    }
  }
  return zero;
}

template <class T>
__device__ __forceinline__ void gstore(const KArgs<T>& a, long long base, long long col, int i,
                                       typename CT<T>::type v, typename CT<T>::type x0) {
  using C = typename CT<T>::type;
  const long long off = base + (long long)i * a.om.es;
  switch (a.out_op) {
    case OUT_C:
      static_cast<C*>(a.out)[off] = cscale(v, a.scale);
      return;
    case OUT_RE:  // real part (reference C2R: full inverse then .re)
      static_cast<T*>(a.out)[off] = v.x * a.scale;
      return;
    case OUT_TRUNC: {  // keep j < nlen (half spectrum); paired bins weighted by pair_w
      const long long j = (long long)i * a.jmul + col;
      if (j < a.nlen) {
        const bool paired = (j > 0) && (2 * j != a.herm_n);
        static_cast<C*>(a.out)[off] = cscale(v, paired ? a.scale * a.pair_w : a.scale);
      }
      return;
    }
    case OUT_TW: {  // four-step: multiply by W_N^{col * i}; twB is a power of two
      unsigned long long m = (unsigned long long)col * (unsigned long long)i;
      if (m >= (unsigned long long)a.twN) m %= (unsigned long long)a.twN;  // col * i < N in every four-step pass
      const int sh = __ffsll(a.twB) - 1;
      const C w = cmul(a.tw_hi[m >> sh], a.tw_lo[m & (unsigned long long)(a.twB - 1)]);
      v = a.tw_conj ? cmulc(v, w) : cmul(v, w);
      static_cast<C*>(a.out)[off] = cscale(v, a.scale);
      return;
    }
    case OUT_MUL: {  // pointwise spectrum at natural index j
      const long long j = (long long)i * a.jmul + col;
      static_cast<C*>(a.out)[off] = cmul(v, a.spec[j]);
      return;
    }
    case OUT_CHIRP:
    case OUT_CHIRP_RE: {  // Bluestein / CZT post-multiply, keep j < nlen (nlen_out when set)
      const long long j = (long long)i * a.jmul + col;
      if (j < (a.nlen_out > 0 ? a.nlen_out : a.nlen)) {
        const C c = a.chirp_out ? a.chirp_out[j] : a.chirp[j];
        v = cscale(a.chirp_conj ? cmulc(v, c) : cmul(v, c), a.scale);
        if (a.out_op == OUT_CHIRP) static_cast<C*>(a.out)[off] = v;
        else static_cast<T*>(a.out)[off] = v.x;
      }
      return;
    }
    case OUT_SCATTER:
    case OUT_SCATTER_RE: {  // Rader: X[g^{-i}] = x0 + conv[i]
      if (i < a.nlen - 1) {
        const long long o2 = base + (long long)a.scatter[i] * a.om.es;
        const C y = cscale(cadd(x0, v), a.scale);
        if (a.out_op == OUT_SCATTER) static_cast<C*>(a.out)[o2] = y;
        else static_cast<T*>(a.out)[o2] = y.x;
      }
      return;
    }
  }
}

// Per-thread context the engine loads from / stores to.  Direct global access
// is plain (complex or real-widened loads, complex or real-part stores with the
// scale); every other operator goes through the staged copies below.
template <class T> struct Ctx {
  using C = typename CT<T>::type;
  const KArgs<T>& a;
  long long ib, ob;
  bool valid;
  __device__ __forceinline__ C gload(int i) const {
    if (!valid) return C{(T)0, (T)0};
    const long long off = ib + (long long)i * a.im.es;
    if (a.in_op == IN_R) return C{static_cast<const T*>(a.in)[off], (T)0};
    return static_cast<const C*>(a.in)[off];
  }
  __device__ __forceinline__ void gstore(int i, C v) const {
    if (!valid) return;
    const long long off = ob + (long long)i * a.om.es;
    if (a.out_op == OUT_RE) static_cast<T*>(a.out)[off] = v.x * a.scale;
    else static_cast<C*>(a.out)[off] = cscale(v, a.scale);
  }
};

template <class T> __device__ __forceinline__ long long col_of(const KArgs<T>& a, long long q) {
  return (q / a.col_div) % a.col_mod;
}

// ─────────────────────────────── lanes kernel ───────────────────────────────
// Shared memory: L lanes x nbuf buffers x ld elements, then 3L lane descriptors.

// One tile of L lanes starting at lane q0.  Threads beyond L x P idle through
// the barriers (the persistent batch kernel runs tiles of different shapes).
template <class T, bool INV>
__device__ __forceinline__ void lanes_tile(const KArgs<T>& a, long long q0, unsigned char* smraw) {
  using C = typename CT<T>::type;
  C* sm = reinterpret_cast<C*>(smraw);
  const int P = a.P, L = a.L, n = a.sl.n, ld = a.ld;
  const int nbuf = engine_buffers(a.sl.nst, a.stage_in, a.stage_out);
  long long* lb = reinterpret_cast<long long*>(sm + (long long)L * nbuf * ld);  // in base, out base, col
  const int tid = threadIdx.x;
  const bool active = tid < L * P;
  const int l = active ? tid / P : 0;
  const int t = active ? tid - l * P : (1 << 30);  // idle threads own no butterfly
  const int lanes_here = (int)((a.lanes - q0) < L ? (a.lanes - q0) : L);
  if (tid < L) {
    const long long qq = q0 + tid;
    const bool v = tid < lanes_here;
    lb[tid] = v ? a.im.base(qq) : 0;
    lb[L + tid] = v ? a.om.base(qq) : 0;
    lb[2 * L + tid] = v ? col_of(a, qq) : 0;
  }
  C* b0 = sm + (long long)l * nbuf * ld;
  C* b1 = b0 + (nbuf > 1 ? ld : 0);
  __syncthreads();
  if (a.stage_in && blockDim.x % lanes_here == 0) {
    // the block covers whole rows: each thread keeps one lane, four loads in flight
    const int l2 = tid % lanes_here, i0 = tid / lanes_here, di = blockDim.x / lanes_here;
    const long long ib = lb[l2], colv = lb[2 * L + l2];
    C* dstl = sm + (long long)l2 * nbuf * ld;
    int i = i0;
    for (; i + 3 * di < n; i += 4 * di) {
      C v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = gload(a, ib, colv, i + u * di);
#pragma unroll
      for (int u = 0; u < 4; ++u) dstl[spad(i + u * di)] = v[u];
    }
    for (; i < n; i += di) dstl[spad(i)] = gload(a, ib, colv, i);
    __syncthreads();
  } else if (a.stage_in) {
    // four independent loads in flight per thread before their shared stores
    const int total = lanes_here * n;
    const int stride = blockDim.x;
    int e = tid;
    for (; e + 3 * stride < total; e += 4 * stride) {
      C v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        const int l2 = ee % lanes_here, i = ee / lanes_here;
        v[u] = gload(a, lb[l2], lb[2 * L + l2], i);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        const int l2 = ee % lanes_here, i = ee / lanes_here;
        sm[(long long)l2 * nbuf * ld + spad(i)] = v[u];
      }
    }
    for (; e < total; e += stride) {
      const int l2 = e % lanes_here, i = e / lanes_here;
      sm[(long long)l2 * nbuf * ld + spad(i)] = gload(a, lb[l2], lb[2 * L + l2], i);
    }
    __syncthreads();
  }
  const Ctx<T> cx{a, lb[l], lb[L + l], active && l < lanes_here};
  C* res = run_stages<INV>(cx, a.sl, a.tw, t, P, b0, b1, a.stage_in != 0, a.stage_out != 0);
  if (a.stage_out && blockDim.x % lanes_here == 0) {
    const long long off = res ? (long long)(res - b0) : 0;
    const C z = C{(T)0, (T)0};
    const int l2 = tid % lanes_here, di = blockDim.x / lanes_here;
    const long long ob = lb[L + l2], colv = lb[2 * L + l2];
    const C* srcl = sm + (long long)l2 * nbuf * ld + off;
    for (int i = tid / lanes_here; i < n; i += di) gstore(a, ob, colv, i, srcl[spad(i)], z);
  } else if (a.stage_out) {
    // every lane ends in the same buffer slot: offset of res within its lane block
    const long long off = res ? (long long)(res - b0) : 0;
    const int total = lanes_here * n;
    const C z = C{(T)0, (T)0};
    for (int e = tid; e < total; e += blockDim.x) {
      const int l2 = e % lanes_here, i = e / lanes_here;
      gstore(a, lb[L + l2], lb[2 * L + l2], i, sm[(long long)l2 * nbuf * ld + off + spad(i)], z);
    }
  }
}

template <class T, bool INV>
__global__ void __launch_bounds__(512) lanes_kernel(const __grid_constant__ KArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  lanes_tile<T, INV>(a, (long long)blockIdx.x * a.L, smraw);
}


// ─────────────────────────────── tile kernel ───────────────────────────────
// Persistent CTAs walk tiles of L lanes.  The next tile is prefetched into
// shared memory with cp.async while the current one is transformed, so HBM
// reads overlap the butterflies and the stores.  Shared memory: two tile
// buffers and one work buffer, each L x ld (padded) elements; the input tile is
// first viewed linearly (lane-minor [i][l] for strided lanes, lane-major [l][i]
// for contiguous ones) and, once stage 0 has consumed it, reused as a padded
// work buffer.  Strided lanes run lane-minor (consecutive threads take
// consecutive lanes: conflict-free shared accesses, coalesced rows of L
// elements); contiguous lanes run lane-major.  The last stage stores straight
// to global memory.  Plain complex input, complex or real-part output.

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// element i of lane l: p[l * ls + i * is + (pad ? i >> 4 : 0)]
template <class C> struct SView {
  C* p;
  int ls, is, pad;
  __device__ __forceinline__ C& at(int l, int i) const { return p[l * ls + i * is + (pad ? (i >> 4) : 0)]; }
};

template <int R, bool INV, class T>
__device__ __forceinline__ void tstage(const KArgs<T>& a, SView<typename CT<T>::type> src, SView<typename CT<T>::type> dst,
                                       bool to_global, long long ob, bool valid, int l, int n, int Ns,
                                       const typename CT<T>::type* __restrict__ tw, int t, int P) {
  using C = typename CT<T>::type;
  const int nb = n / R;
  for (int j = t; j < nb; j += P) {
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src.at(l, j + r * nb);
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const C wr = tw[(long long)(r - 1) * Ns + k];
        v[r] = INV ? cmulc(v[r], wr) : cmul(v[r], wr);
      }
    }
    DFT<R, INV>::run(v);
    const int o = (j - k) * R + k;
    if (to_global) {
      if (valid) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const long long off = ob + (long long)(o + r * Ns) * a.om.es;
          if (a.out_op == OUT_RE) static_cast<T*>(a.out)[off] = v[r].x * a.scale;
          else static_cast<C*>(a.out)[off] = cscale(v[r], a.scale);
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) dst.at(l, o + r * Ns) = v[r];
    }
  }
}

template <class T>
__device__ __forceinline__ void tile_issue(const KArgs<T>& a, typename CT<T>::type* buf, const long long* lbi, long long q0,
                                           int L, int n, bool lm) {
  using C = typename CT<T>::type;
  const long long rem = a.lanes - q0;
  const int lanes_here = (int)(rem < L ? rem : L);
  const int total = lanes_here * n;
  const C* in = static_cast<const C*>(a.in);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    int l2, i;
    if (lm) { l2 = e % lanes_here; i = e / lanes_here; }
    else { l2 = e / n; i = e - l2 * n; }
    const C* g = in + lbi[l2] + (long long)i * a.im.es;
    C* s = lm ? buf + i * L + l2 : buf + l2 * n + i;
    if (sizeof(C) == 16) cp_async16(s, g);
    else cp_async8(s, g);
  }
}

template <class T, bool INV>
__global__ void __launch_bounds__(256) tile_kernel(const __grid_constant__ KArgs<T> a) {
  using C = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int L = a.L, P = a.P, n = a.sl.n, ld = a.ld;
  C* bufs[2];
  bufs[0] = reinterpret_cast<C*>(smraw);
  bufs[1] = bufs[0] + L * ld;
  C* work = bufs[1] + L * ld;
  long long* lbi = reinterpret_cast<long long*>(work + L * ld);  // [2][L] input lane bases
  long long* lbo = lbi + 2 * L;                                     // [2][L] output lane bases
  const bool lm = a.lane_minor != 0;
  const int tid = threadIdx.x;
  const int l = lm ? tid % L : tid / P;
  const int t = lm ? tid / L : tid % P;
  const long long ntiles = (a.lanes + L - 1) / L;
  long long tile = blockIdx.x;
  if (tile >= ntiles) return;
  if (tid < L) {
    const long long q = tile * L + tid;
    lbi[tid] = q < a.lanes ? a.im.base(q) : 0;
    lbo[tid] = q < a.lanes ? a.om.base(q) : 0;
  }
  __syncthreads();
  tile_issue(a, bufs[0], lbi, tile * L, L, n, lm);
  cp_async_commit();
  const SView<C> wv{work, ld, 1, 1};
  for (int it = 0;; ++it) {
    const int cb = it & 1;
    const long long nxt = tile + gridDim.x;
    if (nxt < ntiles && tid < L) {
      const long long q = nxt * L + tid;
      lbi[(cb ^ 1) * L + tid] = q < a.lanes ? a.im.base(q) : 0;
      lbo[(cb ^ 1) * L + tid] = q < a.lanes ? a.om.base(q) : 0;
    }
    __syncthreads();
    if (nxt < ntiles) tile_issue(a, bufs[cb ^ 1], lbi + (cb ^ 1) * L, nxt * L, L, n, lm);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const long long q = tile * L + l;
    const bool valid = q < a.lanes;
    const long long ob = lbo[cb * L + l];
    C* cur = bufs[cb];
    const SView<C> inv_lin = lm ? SView<C>{cur, 1, L, 0} : SView<C>{cur, n, 1, 0};
    const SView<C> cv{cur, ld, 1, 1};
    const int nst = a.sl.nst;
    if (nst == 0) {
      if (t == 0 && valid) {
        const C v = inv_lin.at(l, 0);
        if (a.out_op == OUT_RE) static_cast<T*>(a.out)[ob] = v.x * a.scale;
        else static_cast<C*>(a.out)[ob] = cscale(v, a.scale);
      }
    }
    for (int s = 0; s < nst; ++s) {
      const StageDesc sd = a.sl.st[s];
      const bool last = s == nst - 1;
      const SView<C> src = s == 0 ? inv_lin : ((s & 1) ? wv : cv);
      const SView<C> dst = (s & 1) ? cv : wv;
      const C* twi = a.tw + sd.twoff;
#define AFC_TS(R) tstage<R, INV, T>(a, src, dst, last, ob, valid, l, n, sd.Ns, twi, t, P)
      switch (sd.R) {
        case 2: AFC_TS(2); break;
        case 3: AFC_TS(3); break;
        case 4: AFC_TS(4); break;
        case 5: AFC_TS(5); break;
        case 6: AFC_TS(6); break;
        case 7: AFC_TS(7); break;
        case 8: AFC_TS(8); break;
        case 9: AFC_TS(9); break;
        case 10: AFC_TS(10); break;
        case 12: AFC_TS(12); break;
        case 14: AFC_TS(14); break;
        case 15: AFC_TS(15); break;
        case 11: AFC_TS(11); break;
        case 13: AFC_TS(13); break;
        case 16: AFC_TS(16); break;
        default: break;
      }
#undef AFC_TS
      if (!last) __syncthreads();
    }
    tile = nxt;
    if (tile >= ntiles) break;
  }
  cp_async_wait0();
}

// ──────────────────────── convolution kernel (Rader / Bluestein) ────────────────────────
// One lane = one transform of length p (Rader) or n (Bluestein); the cyclic
// convolution of length M = sl.n runs in shared memory (two buffers per lane):
// staged gather / chirp premultiply, forward FFT, spectrum multiply (spec
// carries 1/M), inverse FFT, staged scatter (+ x0, DC) / chirp postmultiply.

template <class T>
__device__ __forceinline__ void conv_tile(const KArgs<T>& a, long long q0, unsigned char* smraw) {
  using C = typename CT<T>::type;
  C* sm = reinterpret_cast<C*>(smraw);
  const int P = a.P, L = a.L, M = a.sl.n, ld = a.ld;
  const int tid = threadIdx.x;
  const bool active = tid < L * P;
  const int l = active ? tid / P : 0;
  const int t = active ? tid - l * P : (1 << 30);  // idle threads own no butterfly
  const bool rader = a.in_op == IN_GATHER || a.in_op == IN_GATHER_R;
  C* extra = sm + (long long)L * 2 * ld;                         // [2L]: x0, DC per lane
  long long* lb = reinterpret_cast<long long*>(extra + 2 * L);   // [3L]: in base, out base, col
  const int lanes_here = (int)((a.lanes - q0) < L ? (a.lanes - q0) : L);
  if (tid < L) {
    const long long qq = q0 + tid;
    const bool v = tid < lanes_here;
    lb[tid] = v ? a.im.base(qq) : 0;
    lb[L + tid] = v ? a.om.base(qq) : 0;
    lb[2 * L + tid] = v ? col_of(a, qq) : 0;
    C x0 = C{(T)0, (T)0};
    if (v && rader) x0 = a.in_op == IN_GATHER ? static_cast<const C*>(a.in)[lb[tid]] : C{static_cast<const T*>(a.in)[lb[tid]], (T)0};
    extra[2 * tid] = x0;
  }
  __syncthreads();
  {
    // four independent loads in flight per thread before their shared stores
    const int total = lanes_here * M, stride = blockDim.x;
    int e = tid;
    for (; e + 3 * stride < total; e += 4 * stride) {
      C v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        v[u] = gload(a, lb[ee % lanes_here], 0, ee / lanes_here);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        sm[(long long)(ee % lanes_here) * 2 * ld + spad(ee / lanes_here)] = v[u];
      }
    }
    for (; e < total; e += stride) {
      const int l2 = e % lanes_here, i = e / lanes_here;
      sm[(long long)l2 * 2 * ld + spad(i)] = gload(a, lb[l2], 0, i);
    }
  }
  __syncthreads();
  C* b0 = sm + (long long)l * 2 * ld;
  C* b1 = b0 + ld;
  const Ctx<T> cx{a, 0, 0, false};
  C* res = run_stages<false>(cx, a.sl, a.tw, t, P, b0, b1, true, true);
  const long long off = (long long)(res - b0);
  if (tid < lanes_here) extra[2 * tid + 1] = sm[(long long)tid * 2 * ld + off];  // DC = sum of the gathered values
  __syncthreads();
  {
    const int total = lanes_here * M, stride = blockDim.x;
    int e = tid;
    for (; e + 3 * stride < total; e += 4 * stride) {
      C w[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        w[u] = a.spec[lb[2 * L + ee % lanes_here] * a.spec_ld + ee / lanes_here];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * stride;
        C* p = sm + (long long)(ee % lanes_here) * 2 * ld + off + spad(ee / lanes_here);
        *p = cmul(*p, w[u]);
      }
    }
    for (; e < total; e += stride) {
      const int l2 = e % lanes_here, i = e / lanes_here;
      C* p = sm + (long long)l2 * 2 * ld + off + spad(i);
      *p = cmul(*p, a.spec[lb[2 * L + l2] * a.spec_ld + i]);
    }
  }
  __syncthreads();
  // the inverse FFT starts from the buffer holding the product
  C* res2 = off == 0 ? run_stages<true>(cx, a.sl, a.tw, t, P, b0, b1, true, true)
                     : run_stages<true>(cx, a.sl, a.tw, t, P, b1, b0, true, true);
  const long long off2 = (long long)(res2 - b0);
  for (int e = tid; e < lanes_here * M; e += blockDim.x) {
    const int l2 = e % lanes_here, i = e / lanes_here;
    gstore(a, lb[L + l2], lb[2 * L + l2], i, sm[(long long)l2 * 2 * ld + off2 + spad(i)], extra[2 * l2]);
  }
  if (rader && tid < lanes_here) {
    const C dc = cscale(cadd(extra[2 * tid], extra[2 * tid + 1]), a.scale);
    if (a.out_op == OUT_SCATTER) static_cast<C*>(a.out)[lb[L + tid]] = dc;
    else static_cast<T*>(a.out)[lb[L + tid]] = dc.x;
  }
  __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(512) conv_kernel(const __grid_constant__ KArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  conv_tile<T>(a, (long long)blockIdx.x * a.L, smraw);
}

// ───────────────────────── persistent batch kernel ─────────────────────────
// One launch runs a whole phase of an uneven batch: a list of tiles, each a
// lanes tile or a convolution tile of some transform length, described by a
// KArgs record in global memory (kind 0 forward lanes, 2 inverse lanes, 1
// convolution: a phase can mix directions).  CTAs fetch tiles from an atomic counter
// (longest tiles first), copy the record into shared memory, resolve its
// buffer selectors against this launch's bases and run the tile.

template <class T>
__global__ void __launch_bounds__(kBatchThreads, sizeof(T) == 4 ? 3 : 2) batch_kernel(const KArgs<T>* __restrict__ descs, const BatchItem* __restrict__ items,
                                                   int nitems, int* counter, const void* in_base, void* out_base,
                                                   void* ws_base) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(16) KArgs<T> ka;
  __shared__ int cur;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) cur = atomicAdd(counter, 1);
    __syncthreads();
    const int it = cur;
    if (it >= nitems) break;
    const BatchItem bi = items[it];
    const int* src = reinterpret_cast<const int*>(descs + bi.desc);
    int* dst = reinterpret_cast<int*>(&ka);
    for (int w = tid; w < (int)(sizeof(KArgs<T>) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    if (tid == 0) {
      char* bases[4] = {nullptr, (char*)in_base, (char*)out_base, (char*)ws_base};
      if (ka.in_sel) ka.in = bases[ka.in_sel] + (size_t)ka.in;
      if (ka.out_sel) ka.out = bases[ka.out_sel] + (size_t)ka.out;
    }
    __syncthreads();
    if (bi.kind == 0) lanes_tile<T, false>(ka, bi.q0, smraw);
    else if (bi.kind == 2) lanes_tile<T, true>(ka, bi.q0, smraw);
    else conv_tile<T>(ka, bi.q0, smraw);
    __syncthreads();
  }
}

// ────────────────────────────── table kernels ──────────────────────────────

// Stage twiddles: tw[off + (r-1) Ns + k] = exp(-2 pi i (r k mod NsR) / (NsR)), r-major so
// that the butterflies of consecutive threads (consecutive k) read consecutive entries.
template <class T>
__global__ void gen_stage_twiddles(typename CT<T>::type* tw, StageList sl) {
  using C = typename CT<T>::type;
  for (int s = 0; s < sl.nst; ++s) {
    const int R = sl.st[s].R, Ns = sl.st[s].Ns, off = sl.st[s].twoff;
    if (Ns <= 1) continue;
    const long long cnt = (long long)Ns * (R - 1);
    const long long Lr = (long long)Ns * R;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt; e += (long long)gridDim.x * blockDim.x) {
      const long long r = e / Ns + 1, k = e % Ns;
      const long long m = (r * k) % Lr;
      double sn, cs;
      sincospi(-2.0 * (double)m / (double)Lr, &sn, &cs);
      tw[off + e] = C{(T)cs, (T)sn};
    }
  }
}

// out[j] = exp(-2 pi i (j * mult mod N) / N) for j < cnt.
template <class T>
__global__ void gen_roots(typename CT<T>::type* out, long long cnt, long long mult, long long N) {
  using C = typename CT<T>::type;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < cnt; j += (long long)gridDim.x * blockDim.x) {
    const unsigned long long m = (unsigned long long)(((__int128)j * mult) % N);
    double sn, cs;
    sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
    out[j] = C{(T)cs, (T)sn};
  }
}

// Bluestein chirp, forward sign: c[j] = exp(-i pi (j^2 mod 2n) / n); the phase
// is reduced in exact 64-bit integer arithmetic before the FP64 sincospi.
template <class T>
__global__ void gen_chirp(typename CT<T>::type* out, long long n) {
  using C = typename CT<T>::type;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const unsigned long long m = (unsigned long long)(((__int128)j * j) % (2 * n));
    double sn, cs;
    sincospi(-(double)m / (double)n, &sn, &cs);
    out[j] = C{(T)cs, (T)sn};
  }
}

// Bluestein convolution kernel (length M): b[m] = conj(c_dir[|m|]) for |m| < n
// placed cyclically, c_dir = c (forward) or conj(c) (inverse); scaled by 1/M.
template <class T>
__global__ void gen_bluestein_b(typename CT<T>::type* b, const typename CT<T>::type* chirp, long long n, long long M,
                                int inverse) {
  using C = typename CT<T>::type;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
    long long m = -1;
    if (i < n) m = i;
    else if (i > M - n) m = M - i;
    C v = C{(T)0, (T)0};
    if (m >= 0) {
      const C c = chirp[m];
      v = inverse ? c : C{c.x, -c.y};
      v = cscale(v, (T)(1.0 / (double)M));
    }
    b[i] = v;
  }
}

// Rader kernel b[q] = exp(sign 2 pi i (g^{-q} mod p) / p), q < p-1 (scalar/rader.rs:3-19
// of the reference builds the same sequence); the length-(p-1) cyclic kernel is
// embedded in M >= 2(p-1)-1 when M != p-1.  Scaled by 1/M.
template <class T>
__global__ void gen_rader_b(typename CT<T>::type* b, const int* scatter, long long p, long long M, int inverse) {
  using C = typename CT<T>::type;
  const long long L = p - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
    long long qq = -1;
    if (M == L || i < L) qq = i;
    else if (i > M - L) qq = L - (M - i);
    C v = C{(T)0, (T)0};
    if (qq >= 0) {
      double sn, cs;
      sincospi((inverse ? 2.0 : -2.0) * (double)scatter[qq] / (double)p, &sn, &cs);
      v = C{(T)(cs / (double)M), (T)(sn / (double)M)};
    }
    b[i] = v;
  }
}

// Row-major spectrum for the fused middle pass of a large Bluestein
// convolution: dst[k1 N2 + k2] = src[k1 + N1 k2] (natural index k = k1 + N1 k2).
template <class T>
__global__ void gen_row_spectrum(typename CT<T>::type* dst, const typename CT<T>::type* src, long long N1, long long N2) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N1 * N2; e += (long long)gridDim.x * blockDim.x) {
    const long long k1 = e / N2, k2 = e % N2;
    dst[e] = src[k1 + N1 * k2];
  }
}

// Inverse STFT weighted overlap-add (apollo-stft inverse_complex64_slice_into,
// stft/dimension_1d.rs:287-345): sample i sums frame[m][i - start_m] * window and
// window^2 over the frames covering it (start_m = m hop - frame_len / 2) and
// divides; zero where no frame covers it.  One thread per sample, gathering.
template <class T>
__global__ void stft_ola(const T* __restrict__ frames, const T* __restrict__ window, long long nframes, long long flen,
                         long long hop, long long nsig, T* __restrict__ out) {
  const long long half = flen / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsig; i += (long long)gridDim.x * blockDim.x) {
    // frames with start_m <= i < start_m + flen: m hop in (i + half - flen, i + half]
    long long m_hi = (i + half) / hop;
    long long lo = i + half - flen + 1;
    long long m_lo = lo <= 0 ? 0 : (lo + hop - 1) / hop;
    if (m_hi > nframes - 1) m_hi = nframes - 1;
    T acc = (T)0, wsum = (T)0;
    for (long long m = m_lo; m <= m_hi; ++m) {
      const long long nidx = i - (m * hop - half);
      const T w = window[nidx];
      acc += frames[m * flen + nidx] * w;
      wsum += w * w;
    }
    out[i] = wsum > (T)0 ? acc / wsum : (T)0;
  }
}

// ─────────────────────────────── launchers ────────────────────────────────

template <class T> static KArgs<T> to_kargs(const LaunchDesc& d) {
  using C = typename CT<T>::type;
  KArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.sl = d.sl;
  a.tw = static_cast<const C*>(d.tw);
  a.lanes = d.lanes;
  a.L = d.L;
  a.P = d.P;
  a.ld = d.ld;
  a.in_op = d.in_op;
  a.out_op = d.out_op;
  a.stage_in = d.stage_in;
  a.stage_out = d.stage_out;
  a.im = d.im;
  a.om = d.om;
  a.in = d.in;
  a.out = d.out;
  a.scale = (T)d.scale;
  a.jmul = d.jmul ? d.jmul : 1;
  a.col_div = d.col_div ? d.col_div : 1;
  a.col_mod = d.col_mod ? d.col_mod : 1;
  a.nlen = d.nlen;
  a.herm_n = d.herm_n;
  a.pair_w = (T)d.pair_w;
  a.twN = d.twN ? d.twN : 1;
  a.twB = d.twB ? d.twB : 1;
  a.tw_conj = d.tw_conj;
  a.tw_hi = static_cast<const C*>(d.tw_hi);
  a.tw_lo = static_cast<const C*>(d.tw_lo);
  a.spec = static_cast<const C*>(d.spec);
  a.spec_ld = d.spec_ld;
  a.window = static_cast<const T*>(d.window);
  a.chirp_out = static_cast<const C*>(d.chirp_out);
  a.nlen_out = d.nlen_out;
  a.frame_off = d.frame_off;
  a.chirp = static_cast<const C*>(d.chirp);
  a.chirp_conj = d.chirp_conj;
  a.gather = d.gather;
  a.scatter = d.scatter;
  a.lane_minor = d.lane_minor;
  a.in_sel = d.in_sel;
  a.out_sel = d.out_sel;
  return a;
}

static std::mutex g_kfact_mu;
static std::map<std::pair<int, const void*>, size_t> g_kgrant;
static std::map<std::tuple<int, const void*, int, size_t>, int> g_kper;

cudaError_t kernel_smem_grant(const void* kern, size_t smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(dev, kern);
  {
    std::lock_guard<std::mutex> lk(g_kfact_mu);
    auto it = g_kgrant.find(key);
    if (it != g_kgrant.end() && it->second >= smem) return cudaSuccess;
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_kfact_mu);
  size_t& g = g_kgrant[key];
  if (g < smem) g = smem;
  return cudaSuccess;
}

int kernel_ctas_per_sm(const void* kern, int threads, size_t smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, kern, threads, smem);
  {
    std::lock_guard<std::mutex> lk(g_kfact_mu);
    auto it = g_kper.find(key);
    if (it != g_kper.end()) return it->second;
  }
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess || per < 1) {
    cudaGetLastError();  // an estimate only: a refused query must not surface at the next launch
    per = 1;
  }
  std::lock_guard<std::mutex> lk(g_kfact_mu);
  g_kper[key] = per;
  return per;
}

template <class K> static cudaError_t prep_smem(K kern, size_t smem) {
  return kernel_smem_grant(reinterpret_cast<const void*>(kern), smem);
}

template <class T, bool INV> static cudaError_t launch_lanes_t(const LaunchDesc& d, cudaStream_t st) {
  auto k = lanes_kernel<T, INV>;
  const size_t smem = lanes_smem_bytes(d, sizeof(typename CT<T>::type));
  cudaError_t e = prep_smem(k, smem);
  if (e != cudaSuccess) return e;
  const long long grid = (d.lanes + d.L - 1) / d.L;
  k<<<(unsigned)grid, d.L * d.P, smem, st>>>(to_kargs<T>(d));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t launch_lanes(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st) {
  if (d.lanes <= 0) return cudaSuccess;
  if (dbl) return inv ? launch_lanes_t<double, true>(d, st) : launch_lanes_t<double, false>(d, st);
  return inv ? launch_lanes_t<float, true>(d, st) : launch_lanes_t<float, false>(d, st);
}

static int g_sm_count = 0;

template <class T, bool INV> static cudaError_t launch_tile_t(const LaunchDesc& d, cudaStream_t st) {
  auto k = tile_kernel<T, INV>;
  const size_t smem = tile_smem_bytes(d, sizeof(typename CT<T>::type));
  cudaError_t e = prep_smem(k, smem);
  if (e != cudaSuccess) return e;
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  const int per_sm = kernel_ctas_per_sm(reinterpret_cast<const void*>(k), d.L * d.P, smem);
  const long long ntiles = (d.lanes + d.L - 1) / d.L;
  long long grid = (long long)g_sm_count * per_sm;
  if (grid > ntiles) grid = ntiles;
  KArgs<T> ka = to_kargs<T>(d);
  ka.lane_minor = d.lane_minor;
  k<<<(unsigned)grid, d.L * d.P, smem, st>>>(ka);
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t launch_tile(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st) {
  if (d.lanes <= 0) return cudaSuccess;
  if (dbl) return inv ? launch_tile_t<double, true>(d, st) : launch_tile_t<double, false>(d, st);
  return inv ? launch_tile_t<float, true>(d, st) : launch_tile_t<float, false>(d, st);
}

template <class T> static cudaError_t launch_conv_t(const LaunchDesc& d, cudaStream_t st) {
  auto k = conv_kernel<T>;
  const size_t smem = conv_smem_bytes(d, sizeof(typename CT<T>::type));
  cudaError_t e = prep_smem(k, smem);
  if (e != cudaSuccess) return e;
  const long long grid = (d.lanes + d.L - 1) / d.L;
  k<<<(unsigned)grid, d.L * d.P, smem, st>>>(to_kargs<T>(d));
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t launch_conv(const LaunchDesc& d, bool dbl, cudaStream_t st) {
  if (d.lanes <= 0) return cudaSuccess;
  return dbl ? launch_conv_t<double>(d, st) : launch_conv_t<float>(d, st);
}

size_t kargs_size(bool dbl) { return dbl ? sizeof(KArgs<double>) : sizeof(KArgs<float>); }

void kargs_pack(const LaunchDesc& d, bool dbl, void* dst) {
  if (dbl) {
    KArgs<double> a = to_kargs<double>(d);
    memcpy(dst, &a, sizeof(a));
  } else {
    KArgs<float> a = to_kargs<float>(d);
    memcpy(dst, &a, sizeof(a));
  }
}

template <class T>
static cudaError_t launch_batch_t(const void* descs, const BatchItem* items, int nitems, int* counter, size_t smem,
                                  int grid, const void* in, void* out, void* ws, cudaStream_t st) {
  auto k = batch_kernel<T>;
  cudaError_t e = prep_smem(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, kBatchThreads, smem, st>>>(static_cast<const KArgs<T>*>(descs), items, nitems, counter, in, out, ws);
  count_launch(1);
  return cudaGetLastError();
}

cudaError_t launch_batch(const void* descs, const BatchItem* items, int nitems, int* counter, size_t smem, int grid,
                         const void* in, void* out, void* ws, bool dbl, bool inv, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  (void)inv;
  if (dbl) return launch_batch_t<double>(descs, items, nitems, counter, smem, grid, in, out, ws, st);
  return launch_batch_t<float>(descs, items, nitems, counter, smem, grid, in, out, ws, st);
}

int batch_blocks_per_sm(size_t smem, bool dbl, bool inv) {
  (void)inv;
  int per = 1;
  cudaError_t e;
  if (dbl) {
    e = prep_smem(batch_kernel<double>, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel<double>, kBatchThreads, smem);
  } else {
    e = prep_smem(batch_kernel<float>, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel<float>, kBatchThreads, smem);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();  // an estimate only; the launch itself reports a real failure
    per = 1;
  }
  return per < 1 ? 1 : per;
}

static unsigned table_grid(long long n) {
  long long g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 4096) g = 4096;
  return (unsigned)g;
}

cudaError_t gen_stage_twiddles_dev(void* tw, const StageList& sl, bool dbl, cudaStream_t st) {
  if (dbl) gen_stage_twiddles<double><<<table_grid(sl.n), 256, 0, st>>>(static_cast<double2*>(tw), sl);
  else gen_stage_twiddles<float><<<table_grid(sl.n), 256, 0, st>>>(static_cast<float2*>(tw), sl);
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t gen_row_spectrum_dev(void* dst, const void* src, long long N1, long long N2, bool dbl, cudaStream_t st) {
  if (dbl)
    gen_row_spectrum<double><<<table_grid(N1 * N2), 256, 0, st>>>(static_cast<double2*>(dst),
                                                                   static_cast<const double2*>(src), N1, N2);
  else
    gen_row_spectrum<float><<<table_grid(N1 * N2), 256, 0, st>>>(static_cast<float2*>(dst),
                                                                 static_cast<const float2*>(src), N1, N2);
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t stft_ola_dev(const void* frames, const void* window, long long nframes, long long flen, long long hop,
                         long long nsig, void* out, bool dbl, cudaStream_t st) {
  if (dbl)
    stft_ola<double><<<table_grid(nsig), 256, 0, st>>>(static_cast<const double*>(frames),
                                                       static_cast<const double*>(window), nframes, flen, hop, nsig,
                                                       static_cast<double*>(out));
  else
    stft_ola<float><<<table_grid(nsig), 256, 0, st>>>(static_cast<const float*>(frames),
                                                      static_cast<const float*>(window), nframes, flen, hop, nsig,
                                                      static_cast<float*>(out));
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t gen_roots_dev(void* out, long long cnt, long long mult, long long N, bool dbl, cudaStream_t st) {
  if (dbl) gen_roots<double><<<table_grid(cnt), 256, 0, st>>>(static_cast<double2*>(out), cnt, mult, N);
  else gen_roots<float><<<table_grid(cnt), 256, 0, st>>>(static_cast<float2*>(out), cnt, mult, N);
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t gen_chirp_dev(void* out, long long n, bool dbl, cudaStream_t st) {
  if (dbl) gen_chirp<double><<<table_grid(n), 256, 0, st>>>(static_cast<double2*>(out), n);
  else gen_chirp<float><<<table_grid(n), 256, 0, st>>>(static_cast<float2*>(out), n);
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t gen_bluestein_b_dev(void* b, const void* chirp, long long n, long long M, bool inverse, bool dbl,
                                cudaStream_t st) {
  if (dbl)
    gen_bluestein_b<double><<<table_grid(M), 256, 0, st>>>(static_cast<double2*>(b), static_cast<const double2*>(chirp), n, M, inverse);
  else
    gen_bluestein_b<float><<<table_grid(M), 256, 0, st>>>(static_cast<float2*>(b), static_cast<const float2*>(chirp), n, M, inverse);
  count_launch(1);
  return cudaGetLastError();
}
cudaError_t gen_rader_b_dev(void* b, const int* scatter, long long p, long long M, bool inverse, bool dbl,
                            cudaStream_t st) {
  if (dbl) gen_rader_b<double><<<table_grid(M), 256, 0, st>>>(static_cast<double2*>(b), scatter, p, M, inverse);
  else gen_rader_b<float><<<table_grid(M), 256, 0, st>>>(static_cast<float2*>(b), scatter, p, M, inverse);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
