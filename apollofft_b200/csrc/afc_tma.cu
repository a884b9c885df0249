// afc_tma.cu -- TMA-fed axis passes (sm_100a).
//
// Persistent CTAs walk tiles of L lanes.  One thread moves whole tiles with the
// Tensor Memory Accelerator: a 3D tiled tensor map for strided lanes (the
// volume viewed as [2*es scalars, n, outer], box [2L, bn, 1]: rows of L
// adjacent lanes, one row per element of the transformed axis) or one 1D bulk
// copy for contiguous lanes.  Loads complete on an mbarrier (bounded wait; a
// timeout sets the error word and the CTA returns); the next tile is loaded
// while the current one is transformed.  The last stage writes the tile back
// into shared memory in the same layout and one thread stores it with a TMA
// store, so no thread spends instructions on global addresses.  Loads use no
// cluster multicast.
//
// Shared memory: two tile slots (L x max(ld, rows) elements) and one padded
// work buffer (L x ld), then two mbarriers.  Stage 0 reads the slot linearly,
// intermediate stages ping-pong between the work buffer and the slot viewed as
// padded, and the last stage writes the linear layout into whichever of the two
// the previous stage did not use; that buffer is the TMA store's source.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
#include "afc_async.cuh"
#include "afc_engine.cuh"
#include "afc_internal.h"

namespace afc {

template <class T> struct TmaArgs {
  using C = typename CT<T>::type;
  CUtensorMap tmi;  // strided mode: input / output tensor maps
  CUtensorMap tmo;
  StageList sl;
  const C* tw;
  const C* in;      // contiguous mode: bulk copy sources / destinations
  C* out;
  long long lanes;  // total lanes
  long long ntiles;
  long long kb;     // strided: lane blocks per outer index, ceil(es / L)
  int L, P, ld, slot_elems;
  int mode;         // 0 contiguous (1D bulk), 1 strided (tensor)
  int inplace;      // stages run in place in the slot (no work buffer)
  int real_in;      // contiguous in-place mode: input lanes are real (widened to complex in stage 0)
  int real_out;     // contiguous in-place mode: output lanes are the real parts
  int nbx, bn;      // boxes along the transformed axis, rows per box
  unsigned tw_bytes;  // > 0: one tile per CTA, the twiddle table is copied into the idle second slot
  int tw_res;         // > 0: persistent CTAs keep the first tw_res twiddles resident in shared memory
  int nslot;          // tile slots in the ring (2 or 3): nslot - 1 tile loads in flight
  long long tpp, lpp; // contiguous mode, tpp > 0: tiles never straddle planes of lpp lanes (tpp tiles per
                      // plane, the last one of a plane shorter); tpp = 0: tile q covers lanes [q L, q L + L)
  T scale;
  unsigned* err;
  C* hm_out;          // hm_cmax > 0: output base and column count of the mirrored columns
  long long hm_es;
  int hm_cmax;
  int out_cols;       // contiguous mode, > 0: only the first out_cols elements of each lane are stored
};

// First lane and lane count of contiguous-mode tile `tile`.
template <class T>
__device__ __forceinline__ void tile_lanes(const TmaArgs<T>& a, long long tile, long long& q0, int& nl) {
  long long rem;
  if (a.tpp > 0) {
    const long long pl = tile / a.tpp, k = tile % a.tpp;
    q0 = pl * a.lpp + k * a.L;
    rem = a.lpp - k * a.L;
  } else {
    q0 = tile * a.L;
    rem = a.lanes - q0;
  }
  nl = (int)(rem < a.L ? rem : a.L);
}

// Exercises the timeout path of the bounded wait: one thread waits on a
// barrier that nothing arrives on, gives up after `polls` polls and records the
// timeout in the error word, exactly as the transform kernels do.
__global__ void wait_probe_kernel(unsigned* err, int polls) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    if (!mbar_wait(&bar, 0, polls)) atomicExch(err, 1u);
  }
}
template <class C> struct TView {
  C* p;
  int ls, is, pad;
  __device__ __forceinline__ C& at(int l, int i) const { return p[l * ls + i * is + (pad ? (i >> 4) : 0)]; }
  // Elements i0 + r d (r < R) of lane l as a pointer and a fixed stride when
  // the padding term is linear in r: no padding, d a multiple of 16, or the
  // whole run inside one 16-element block.  False otherwise.
  __device__ __forceinline__ bool run(int l, int i0, int d, int R, C*& q, int& s) const {
    if (pad && (d & 15) && (i0 & 15) + (R - 1) * d >= 16) return false;
    q = p + l * ls + i0 * is + (pad ? (i0 >> 4) : 0);
    s = d * is + (pad ? (d >> 4) : 0);
    return true;
  }
};

template <int R, bool INV, class C, class S>
__device__ __forceinline__ void tma_stage(TView<C> src, TView<C> dst, int l, int n, int Ns, const C* __restrict__ tw,
                                          int t, int P, bool scale_out, S sc) {
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
#pragma unroll
    for (int r = 0; r < R; ++r) dst.at(l, o + r * Ns) = scale_out ? cscale(v[r], sc) : v[r];
  }
}

// One stage in place: every thread owns at most one butterfly of its lane
// (n / R <= P).  All reads of the stage finish before the barrier, all writes
// come after it, so source and destination may share the slot.  Every thread
// of the CTA reaches the barrier.
// One stage in place: a thread holds one butterfly of its lane, or with NB2 up
// to two of a radix <= 8 stage (the plan guarantees the count).  All
// reads of the stage finish before the barrier, all writes come after it, so
// source and destination may share the slot.  Every thread of the CTA reaches
// the barrier.  rsrc / rdst (contiguous lanes only): when set, the stage reads
// real input lanes (widened to complex) from rsrc, or writes the real parts of
// its output to rdst, both with lane stride n.
template <int R, bool INV, int NB2, class C, class S>
__device__ __forceinline__ void tma_stage_inplace(TView<C> src, TView<C> dst, int l, int n, int Ns,
                                                  const C* __restrict__ tw, int t, int P, bool scale_out, S sc,
                                                  const S* rsrc = nullptr, S* rdst = nullptr) {
  constexpr int NB = (R <= 8 && NB2) ? 2 : 1;
  const int nb = n / R;
  C v[NB][R];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * P;
    if (j < nb) {
      C* q;
      int qs;
      if (rsrc) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = C{rsrc[(long long)l * n + j + r * nb], (S)0};
      } else if (sizeof(S) == 4 && src.run(l, j, nb, R, q, qs)) {  // complex64 only: complex128 spills
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = q[r * qs];
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = src.at(l, j + r * nb);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * P;
    if (j < nb) {
      const int k = j % Ns;
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C wr = tw[(long long)(r - 1) * Ns + k];
          v[b][r] = INV ? cmulc(v[b][r], wr) : cmul(v[b][r], wr);
        }
      }
      DFT<R, INV>::run(v[b]);
      const int o = (j - k) * R + k;
      C* q;
      int qs;
      if (rdst) {
#pragma unroll
        for (int r = 0; r < R; ++r) rdst[(long long)l * n + o + r * Ns] = scale_out ? v[b][r].x * sc : v[b][r].x;
      } else if (sizeof(S) == 4 && dst.run(l, o, Ns, R, q, qs)) {
#pragma unroll
        for (int r = 0; r < R; ++r) q[r * qs] = scale_out ? cscale(v[b][r], sc) : v[b][r];
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) dst.at(l, o + r * Ns) = scale_out ? cscale(v[b][r], sc) : v[b][r];
      }
    }
  }
}

// Hermitian columns.  The rows of a full-spectrum R2C after its real-input
// pass satisfy X[m][es - c] = conj(X[m][c]), so the transform along the rows'
// axis of column es - c is the conjugate of column c's read backwards:
// Y[k][es - c] = conj(Y[(n - k) mod n][c]).  A tile of columns [c0, c0 + L)
// whose transform sits in obuf ([row][lane]) also stores columns es - c for c
// in [1, hm_cmax]; no tile of the pass reads those columns.
template <class T>
__device__ __forceinline__ void hermitian_mirror(const TmaArgs<T>& a, long long tile,
                                                 const typename CT<T>::type* obuf, int tid) {
  using C = typename CT<T>::type;
  const int L = a.L, n = a.sl.n, nt = blockDim.x;  // strided tiles: nt = L P, a multiple of L
  const int c = (int)(tile % a.kb) * L + tid % L;  // each thread keeps one lane
  if (c < 1 || c > a.hm_cmax) return;
  const long long es = a.hm_es, wrap = (long long)n * es, step = (long long)(nt / L) * es;
  C* const col = a.hm_out + (tile / a.kb) * wrap + es - c;  // column es - c of row 0
  int r = tid / L;
  long long off = (long long)(n - r) * es;  // row (n - r) mod n
  const C* src = obuf + tid;
#pragma unroll 4
  for (; r < n; r += nt / L, src += nt, off -= step) {
    const C v = *src;
    col[off == wrap ? 0 : off] = C{v.x, -v.y};
  }
}

template <class T>
// tw_dst non-null: the twiddle table (a.tw_bytes) rides on the same barrier.
__device__ __forceinline__ void tma_issue_load(const TmaArgs<T>& a, long long tile, typename CT<T>::type* slot,
                                               unsigned long long* bar, typename CT<T>::type* tw_dst = nullptr) {
  using C = typename CT<T>::type;
  const unsigned extra = tw_dst ? a.tw_bytes : 0u;
  if (a.mode == 0) {
    long long q0;
    int lanes_here;
    tile_lanes(a, tile, q0, lanes_here);
    const size_t es = a.real_in ? sizeof(T) : sizeof(C);
    const unsigned bytes = (unsigned)((long long)lanes_here * a.sl.n * es);
    mbar_expect_tx(bar, bytes + extra);
    bulk_load(slot, reinterpret_cast<const char*>(a.in) + q0 * a.sl.n * es, bytes, bar);
  } else {
    const int o = (int)(tile / a.kb), kb = (int)(tile % a.kb);
    const unsigned box_bytes = (unsigned)(2 * a.L * a.bn * sizeof(T));
    mbar_expect_tx(bar, box_bytes * a.nbx + extra);
    for (int b = 0; b < a.nbx; ++b)
      tma_load_3d(slot + (long long)b * a.bn * a.L, &a.tmi, 2 * kb * a.L, b * a.bn, o, bar);
  }
  if (extra) bulk_load(tw_dst, a.tw, extra, bar);
}

template <class T>
__device__ __forceinline__ void tma_issue_store(const TmaArgs<T>& a, long long tile, const typename CT<T>::type* buf) {
  using C = typename CT<T>::type;
  if (a.mode == 0) {
    long long q0;
    int lanes_here;
    tile_lanes(a, tile, q0, lanes_here);
    const size_t es = a.real_out ? sizeof(T) : sizeof(C);
    if (a.out_cols > 0) {  // one copy per lane: its first out_cols elements
      for (int j = 0; j < lanes_here; ++j)
        bulk_store(reinterpret_cast<char*>(a.out) + (q0 + j) * a.sl.n * es, buf + (long long)j * a.sl.n,
                   (unsigned)(a.out_cols * es));
    } else {
      bulk_store(reinterpret_cast<char*>(a.out) + q0 * a.sl.n * es, buf, (unsigned)((long long)lanes_here * a.sl.n * es));
    }
  } else {
    const int o = (int)(tile / a.kb), kb = (int)(tile % a.kb);
    for (int b = 0; b < a.nbx; ++b) {
      // the last box may run past n: rows beyond n hold no data and are clipped by the tensor bounds
      tma_store_3d(&a.tmo, 2 * kb * a.L, b * a.bn, o, buf + (long long)b * a.bn * a.L);
    }
  }
  bulk_commit();
}

// Threads per CTA and CTAs per SM each kernel build is compiled for.
struct FixNone {
  static constexpr int BUILD_THREADS = 0;
};
// FX::BUILD_THREADS > 0: a compile-time stage list built for that many threads
// at one CTA per SM (wider strided tiles)
template <class T, int V, class FX = FixNone> struct TmaBuild {
  static constexpr int threads = FX::BUILD_THREADS ? FX::BUILD_THREADS
                                 : (V == 2 || (V == 5 && sizeof(T) == 8)) ? 128
                                                                           : 256;
  // complex64 4096-point build: three CTAs per SM (80 registers; measured on
  // B200 16384 x 4096 forward 255 -> 242 us against two); the complex64
  // 256-point build gained nothing from a third CTA (256^3: 151 -> 154 us)
  static constexpr int ctas = FX::BUILD_THREADS ? 1
                              : threads == 128 || (V == 6 && sizeof(T) == 4)
                                  ? 3
                                  : (V == 3 || V == 7 || ((V == 1 || V == 4 || V == 5 || V == 8) && sizeof(T) == 4))
                                        ? 2
                                        : 1;
};

// n = 256 as two radix-16 stages in place, every shared-memory address a
// compile-time offset from one per-thread base (variant 5).  The general
// stage code computes each element's address from the runtime lane stride,
// element stride and padding, and selects between the scaled and unscaled
// output of every stage: on B200 that is more integer and select instructions
// per point than FP64 ones.  Layouts as in the general path: the slot holds
// the tile linearly (strided mode: element i of lane l at i LK + l;
// contiguous: at 256 l + i), stage 0 writes the padded layout (element i at
// 273 l + i + i / 16) and stage 1 writes the linear layout back.  The thread
// (l, t) owns butterfly t < 16 of lane l in both stages.  Strided tiles hold
// LK lanes (8 complex128 / 16 complex64).
template <class T, bool INV, bool LM, int LK>
__device__ __forceinline__ void stages256(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                          const typename CT<T>::type* __restrict__ twb, int l, int t) {
  using C = typename CT<T>::type;
  constexpr int LD = 273;                // padded lane stride of a 256-point lane
  constexpr int S = LM ? 16 * LK : 16;   // linear layout: distance of elements t and t + 16
  C* const lin = LM ? cur + l + t * LK : cur + l * 256 + t;
  C v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = lin[r * S];
  __syncthreads();
  DFT<16, INV>::run(v);
  C* const p0 = cur + l * LD + 17 * t;  // outputs 16 t + r, no twiddles (Ns = 1)
#pragma unroll
  for (int r = 0; r < 16; ++r) p0[r] = v[r];
  __syncthreads();
  C* const p1 = cur + l * LD + t;  // inputs t + 16 r at t + 17 r
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = p1[17 * r];
  __syncthreads();
  const C* const tw = twb + a.sl.st[1].twoff + t;  // Ns = 16: twiddle (r - 1) 16 + t
#pragma unroll
  for (int r = 1; r < 16; ++r) v[r] = INV ? cmulc(v[r], tw[(r - 1) * 16]) : cmul(v[r], tw[(r - 1) * 16]);
  DFT<16, INV>::run(v);
  const T sc = a.scale;
  if (sc != (T)1) {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = cscale(v[r], sc);
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) lin[r * S] = v[r];  // outputs t + 16 r
  __syncthreads();
}

// n = 4096 as three radix-16 stages in place on one contiguous lane per tile
// (variant 6), addresses fixed as in stages256: thread t < 256 owns butterfly
// t of every stage.  Stage 0 reads the linear lane (t + 256 r) and writes the
// padded layout (element i at i + i / 16) at 16 t + r; stage 1 (Ns = 16) reads
// t + 256 r and writes 16 (t - k) + k + 16 r with k = t mod 16; stage 2
// (Ns = 256) reads t + 256 r and writes the linear lane at t + 256 r.
template <class T, bool INV>
__device__ __forceinline__ void stages4096(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                           const typename CT<T>::type* __restrict__ twb, int t) {
  using C = typename CT<T>::type;
  C v[16];
  C* const lin = cur + t;
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = lin[256 * r];
  __syncthreads();
  DFT<16, INV>::run(v);
  C* const p0 = cur + 17 * t;
#pragma unroll
  for (int r = 0; r < 16; ++r) p0[r] = v[r];
  __syncthreads();
  C* const pin = cur + t + (t >> 4);  // padded t + 256 r: t + t / 16 + 272 r
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = pin[272 * r];
  __syncthreads();
  const int k = t & 15;
  const C* const tw1 = twb + a.sl.st[1].twoff + k;
#pragma unroll
  for (int r = 1; r < 16; ++r) v[r] = INV ? cmulc(v[r], tw1[(r - 1) * 16]) : cmul(v[r], tw1[(r - 1) * 16]);
  DFT<16, INV>::run(v);
  C* const p1 = cur + 272 * (t >> 4) + k;  // padded 256 (t / 16) + k + 16 r
#pragma unroll
  for (int r = 0; r < 16; ++r) p1[17 * r] = v[r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = pin[272 * r];
  __syncthreads();
  const C* const tw2 = twb + a.sl.st[2].twoff + t;
#pragma unroll
  for (int r = 1; r < 16; ++r) v[r] = INV ? cmulc(v[r], tw2[(r - 1) * 256]) : cmul(v[r], tw2[(r - 1) * 256]);
  DFT<16, INV>::run(v);
  const T sc = a.scale;
  if (sc != (T)1) {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = cscale(v[r], sc);
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) lin[256 * r] = v[r];
  __syncthreads();
}

// A stage list fixed at compile time (variant 7): length N as radices R0 R1
// [R2], P threads per lane, LK lanes per strided tile (0: contiguous lanes).
// Each stage is the general out-of-place Stockham stage with every stride a
// constant, and without the 16-element padding: the smooth odd lengths this
// build serves (343 = 7^3, 243 = 9 9 3, 250 = 10 5 5) have odd or
// non-power-of-two strides, so their shared-memory accesses do not need it.
// Intermediate stages ping-pong between the slot and the work buffer in the
// lane layout (element i of lane l at N l + i); contiguous tiles hold the
// same layout, strided tiles hold element i of lane l at LK i + l.
template <int N_, int R0_, int R1_, int R2_, int P_, int LK_> struct Fix {
  static constexpr int BUILD_THREADS = 0;
  static constexpr int N = N_, P = P_, LK = LK_;
  static constexpr int NST = R2_ ? 3 : 2;
  static constexpr int R(int s) { return s == 0 ? R0_ : s == 1 ? R1_ : R2_; }
  static constexpr int NS(int s) { return s == 0 ? 1 : s == 1 ? R0_ : R0_ * R1_; }
};

template <class T, bool INV, class FX, int S>
__device__ __forceinline__ void fixed_stage(const TmaArgs<T>& a, const typename CT<T>::type* src,
                                            typename CT<T>::type* dst, const typename CT<T>::type* __restrict__ twb,
                                            int l, int t) {
  using C = typename CT<T>::type;
  constexpr int N = FX::N, P = FX::P, R = FX::R(S), NS = FX::NS(S), NB = N / R, IT = (NB + P - 1) / P;
  constexpr bool LM = FX::LK > 0, LAST = S == FX::NST - 1;
  // intermediate lanes at an odd stride: the lanes of a strided tile sit in the
  // same wavefront (8 complex128 / 16 complex64 lanes, one element each), and an
  // odd stride puts them in distinct banks
  constexpr int LDU = N | 1;
  constexpr int SLS = S == 0 ? (LM ? 1 : N) : LDU, SIS = (S == 0 && LM) ? FX::LK : 1;
  constexpr int DLS = LAST ? (LM ? 1 : N) : LDU, DIS = (LAST && LM) ? FX::LK : 1;
  const C* const tw = twb + a.sl.st[S].twoff;
  const T sc = a.scale;
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int j = t + it * P;
    if (j < NB) {
      C v[R];
      const C* s = src + l * SLS + j * SIS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[r * NB * SIS];
      const int k = NS == 1 ? 0 : j % NS;
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C w = tw[(r - 1) * NS + k];
          v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
        }
      }
      DFT<R, INV>::run(v);
      if (LAST && sc != (T)1) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = cscale(v[r], sc);
      }
      C* d = dst + l * DLS + ((j - k) * R + k) * DIS;
#pragma unroll
      for (int r = 0; r < R; ++r) d[r * NS * DIS] = v[r];
    }
  }
}

// A power-of-two stage list fixed at compile time and run in place in the
// slot (variant 8): length N as radices R0 R1 R2 [R3], P threads per lane
// (a thread holds N / (R P) butterflies of a stage across its barrier), LK
// lanes per strided tile (0: contiguous lanes, whose stage 0 may read real
// input and whose last stage may store real parts).  The padded layout
// (element i of lane l at LD l + i + i / 16) keeps every address a
// compile-time offset from one per-butterfly base wherever the stage's
// input stride N / R and output stride Ns are multiples of 16 or the
// first stage is radix 16; elsewhere the padding term is computed per element.
// Padded lane stride of the in-place builds: the plan's (odd) stride for
// contiguous tiles; for strided tiles of LK lanes, whose lanes share a
// shared-memory wavefront (128 bytes: 16 complex64 or 8 complex128 elements,
// LK lanes x 16 / LK or 8 / LK butterflies), the first stride at least as
// large that is congruent to (elements per wavefront) / LK, so the lanes'
// elements fall in distinct banks.
__host__ __device__ constexpr int fixip_ld(int n, int lk, int csz) {
  const int ld = (n + (n - 1) / 16 + 1) | 1;
  const int per = 128 / csz;
  if (lk <= 1 || lk >= per) return ld;
  const int want = per / lk;
  int v = ld;
  while (v % per != want) ++v;
  return v;
}

template <int N_, int R0_, int R1_, int R2_, int R3_, int P_, int LK_> struct FixIP {
  static constexpr int BUILD_THREADS = LK_ * P_ > 256 ? LK_ * P_ : 0;
  static constexpr int N = N_, P = P_, LK = LK_;
  static constexpr int NST = R3_ ? 4 : R2_ ? 3 : 2;
  static constexpr int R(int s) { return s == 0 ? R0_ : s == 1 ? R1_ : s == 2 ? R2_ : R3_; }
  static constexpr int NS(int s) { return s == 0 ? 1 : R(s - 1) * NS(s - 1); }
};

template <class T, bool INV, class FX, int S>
__device__ __forceinline__ void fixed_stage_ip(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                               const typename CT<T>::type* __restrict__ twb, int l, int t) {
  using C = typename CT<T>::type;
  constexpr int N = FX::N, P = FX::P, LD = fixip_ld(FX::N, FX::LK, (int)sizeof(C)), R = FX::R(S), NS = FX::NS(S),
                NB = N / R;
  constexpr int NBT = (NB + P - 1) / P;
  constexpr bool LM = FX::LK > 0, LAST = S == FX::NST - 1;
  static_assert(NB % P == 0, "every thread holds the same number of butterflies");
  C v[NBT][R];
  // ── reads: element j + r NB ──
#pragma unroll
  for (int b = 0; b < NBT; ++b) {
    const int j = t + b * P;
    if constexpr (S == 0) {
      if (!LM && a.real_in) {
        const T* s = reinterpret_cast<const T*>(cur) + l * N + j;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = C{s[r * NB], (T)0};
      } else {
        const C* s = LM ? cur + l + j * FX::LK : cur + l * N + j;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = s[r * NB * (LM ? FX::LK : 1)];
      }
    } else {
      static_assert(NB % 16 == 0, "padded reads need a stride that is a multiple of 16");
      const C* s = cur + l * LD + j + (j >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = s[r * (NB + NB / 16)];
    }
  }
  __syncthreads();
  const T sc = a.scale;
#pragma unroll
  for (int b = 0; b < NBT; ++b) {
    const int j = t + b * P;
    const int k = j & (NS - 1);
    if constexpr (NS > 1) {
      const C* const tw = twb + a.sl.st[S].twoff + k;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const C w = tw[(r - 1) * NS];
        v[b][r] = INV ? cmulc(v[b][r], w) : cmul(v[b][r], w);
      }
    }
    DFT<R, INV>::run(v[b]);
    const int o = (j - k) * R + k;  // outputs o + r NS
    if constexpr (LAST) {
      if (sc != (T)1) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = cscale(v[b][r], sc);
      }
      if (!LM && a.real_out) {
        T* d = reinterpret_cast<T*>(cur) + l * N + o;
#pragma unroll
        for (int r = 0; r < R; ++r) d[r * NS] = v[b][r].x;
      } else {
        C* d = LM ? cur + l + o * FX::LK : cur + l * N + o;
#pragma unroll
        for (int r = 0; r < R; ++r) d[r * NS * (LM ? FX::LK : 1)] = v[b][r];
      }
    } else if constexpr (NS % 16 == 0) {
      C* d = cur + l * LD + o + (o >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) d[r * (NS + NS / 16)] = v[b][r];
    } else if constexpr (NS == 1 && R == 16) {
      C* d = cur + l * LD + 17 * j;  // o + r = 16 j + r, padded 17 j + r
#pragma unroll
      for (int r = 0; r < R; ++r) d[r] = v[b][r];
    } else {
      C* d = cur + l * LD;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int p = o + r * NS;
        d[p + (p >> 4)] = v[b][r];
      }
    }
  }
  __syncthreads();
}

template <class T, bool INV, class FX>
__device__ __forceinline__ void fixed_stages_ip(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                                const typename CT<T>::type* twb, int l, int t) {
  fixed_stage_ip<T, INV, FX, 0>(a, cur, twb, l, t);
  fixed_stage_ip<T, INV, FX, 1>(a, cur, twb, l, t);
  if constexpr (FX::NST >= 3) fixed_stage_ip<T, INV, FX, 2>(a, cur, twb, l, t);
  if constexpr (FX::NST >= 4) fixed_stage_ip<T, INV, FX, 3>(a, cur, twb, l, t);
}

// Every stage of a fixed list; returns the buffer holding the linear result.
template <class T, bool INV, class FX>
__device__ __forceinline__ typename CT<T>::type* fixed_stages(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                                              typename CT<T>::type* work,
                                                              const typename CT<T>::type* twb, int l, int t) {
  fixed_stage<T, INV, FX, 0>(a, cur, work, twb, l, t);
  __syncthreads();
  fixed_stage<T, INV, FX, 1>(a, work, cur, twb, l, t);
  __syncthreads();
  if constexpr (FX::NST == 3) {
    fixed_stage<T, INV, FX, 2>(a, cur, work, twb, l, t);
    __syncthreads();
    return work;
  } else {
    return cur;
  }
}

// Every stage of the tile in slot `cur` (`work` is the ping-pong buffer when
// the stages do not run in place).  Returns the buffer that holds the result in
// the linear layout, the TMA store's source.  Every thread of the CTA calls it
// (the stages hold CTA barriers); (l, t) is the thread's lane and position in
// the lane, with t >= P for a thread that has no butterflies in this tile.
template <class T, bool INV, int V, bool IP, class FX = FixNone>
__device__ __forceinline__ typename CT<T>::type* tma_stages(const TmaArgs<T>& a, typename CT<T>::type* cur,
                                                            typename CT<T>::type* work,
                                                            const typename CT<T>::type* twb, int l, int t) {
  constexpr bool P2 = V == 1 || V == 2 || V == 4;
  constexpr bool S7 = V == 3;
  using C = typename CT<T>::type;
  if constexpr (V == 7) return fixed_stages<T, INV, FX>(a, cur, work, twb, l, t);
  if constexpr (V == 8) {
    fixed_stages_ip<T, INV, FX>(a, cur, twb, l, t);
    return cur;
  }
  if constexpr (V == 5) {
    constexpr int LK = sizeof(T) == 8 ? 8 : 16;
    if (a.mode == 1)
      stages256<T, INV, true, LK>(a, cur, twb, l, t);
    else
      stages256<T, INV, false, LK>(a, cur, twb, l, t);
    return cur;
  }
  if constexpr (V == 6) {
    stages4096<T, INV>(a, cur, twb, t);
    return cur;
  }
  const int L = a.L, P = a.P, n = a.sl.n, ld = a.ld;
  const bool lm = a.mode == 1;
  const TView<C> wv{work, ld, 1, 1};
  const int nst = a.sl.nst;
  const TView<C> lin = lm ? TView<C>{cur, 1, L, 0} : TView<C>{cur, n, 1, 0};
  const TView<C> cpad{cur, ld, 1, 1};
  // output buffer (linear layout): the one the last stage does not read
  C* obuf = (IP || !(nst & 1)) ? cur : work;
  const TView<C> olin = lm ? TView<C>{obuf, 1, L, 0} : TView<C>{obuf, n, 1, 0};
  for (int s = 0; IP && s < nst; ++s) {
    const StageDesc sd = a.sl.st[s];
    const bool last = s == nst - 1;
    const TView<C> src = s == 0 ? lin : cpad;
    const TView<C> dst = last ? olin : cpad;
    const C* twi = twb + sd.twoff;
    const T* rsrc = (s == 0 && a.real_in) ? reinterpret_cast<const T*>(cur) : nullptr;
    T* rdst = (last && a.real_out) ? reinterpret_cast<T*>(cur) : nullptr;
#define AFC_TI(R) tma_stage_inplace<R, INV, (V == 4 ? 1 : 0)>(src, dst, l, n, sd.Ns, twi, t, P, last, a.scale, rsrc, rdst)
    if constexpr (P2) {
      switch (sd.R) {
        case 2: AFC_TI(2); break;
        case 4: AFC_TI(4); break;
        case 8: AFC_TI(8); break;
        case 16: AFC_TI(16); break;
        default: break;
      }
    } else {
      switch (sd.R) {
        case 2: AFC_TI(2); break;
        case 3: AFC_TI(3); break;
        case 4: AFC_TI(4); break;
        case 5: AFC_TI(5); break;
        case 7: AFC_TI(7); break;
        case 8: AFC_TI(8); break;
        case 11: AFC_TI(11); break;
        case 13: AFC_TI(13); break;
        case 16: AFC_TI(16); break;
        default: break;
      }
    }
#undef AFC_TI
    __syncthreads();
  }
  for (int s = 0; !IP && s < nst; ++s) {
    const StageDesc sd = a.sl.st[s];
    const bool last = s == nst - 1;
    const TView<C> src = s == 0 ? lin : ((s & 1) ? wv : cpad);
    const TView<C> dst = last ? olin : ((s & 1) ? cpad : wv);
    const C* twi = twb + sd.twoff;
#define AFC_TM(R) tma_stage<R, INV>(src, dst, l, n, sd.Ns, twi, t, P, last, a.scale)
    if constexpr (P2) {
      switch (sd.R) {
        case 2: AFC_TM(2); break;
        case 4: AFC_TM(4); break;
        case 8: AFC_TM(8); break;
        case 16: AFC_TM(16); break;
        default: break;
      }
    } else if constexpr (S7) {
      switch (sd.R) {
        case 2: AFC_TM(2); break;
        case 3: AFC_TM(3); break;
        case 4: AFC_TM(4); break;
        case 5: AFC_TM(5); break;
        case 6: AFC_TM(6); break;
        case 7: AFC_TM(7); break;
        case 8: AFC_TM(8); break;
        case 9: AFC_TM(9); break;
        case 10: AFC_TM(10); break;
        case 12: AFC_TM(12); break;
        case 14: AFC_TM(14); break;
        case 15: AFC_TM(15); break;
        case 16: AFC_TM(16); break;
        default: break;
      }
    } else {
      switch (sd.R) {
        case 2: AFC_TM(2); break;
        case 3: AFC_TM(3); break;
        case 4: AFC_TM(4); break;
        case 5: AFC_TM(5); break;
        case 6: AFC_TM(6); break;
        case 7: AFC_TM(7); break;
        case 8: AFC_TM(8); break;
        case 9: AFC_TM(9); break;
        case 10: AFC_TM(10); break;
        case 12: AFC_TM(12); break;
        case 14: AFC_TM(14); break;
        case 15: AFC_TM(15); break;
        case 11: AFC_TM(11); break;
        case 13: AFC_TM(13); break;
        case 16: AFC_TM(16); break;
        default: break;
      }
    }
#undef AFC_TM
    __syncthreads();
  }
  return obuf;
}

// V (variant): 0 any radix, 256 threads; 1 every stage radix 2/4/8/16 (no
// odd-radix butterflies, fewer registers; complex64 built for two CTAs per
// SM); 2 the same for complex128 tiles of at most 128 threads, built for three
// CTAs per SM (at most 168 registers).
// IP: stages run in place (TmaPlan::inplace); variant 2 is always in place.
// Variant 3: 7-smooth plans (radix 2/3/4/5/7/8/16, no 11 or 13), built for two
// CTAs of up to 256 threads per SM (at most 128 registers).  Variant 4:
// complex64 power-of-two in place with two butterflies per thread in the
// radix <= 8 stages (the 256-thread build of variant 1 otherwise).  Variant 5:
// n = 256 as radix 16 x 16 in place (stages256), 16 threads per lane, built
// like variant 2 for complex128 and like variant 1 for complex64.
template <class T, bool INV, int V, bool IP, class FX = FixNone>
__global__ void __launch_bounds__(TmaBuild<T, V, FX>::threads, TmaBuild<T, V, FX>::ctas)
    tma_kernel(const __grid_constant__ TmaArgs<T> a) {
  using C = typename CT<T>::type;
  extern __shared__ __align__(128) unsigned char smraw[];
  const int L = a.L, P = a.P, ld = a.ld;
  // a ring of ns tile slots: while one tile is transformed, the loads of the
  // next ns - 1 tiles are in flight
  const int ns = a.nslot;
  C* slots[3];
  for (int k = 0; k < 3; ++k) slots[k] = reinterpret_cast<C*>(smraw) + (long long)k * a.slot_elems;
  C* work = IP ? nullptr : slots[0] + (long long)ns * a.slot_elems;
  C* twsm = IP ? slots[0] + (long long)ns * a.slot_elems : work + (long long)L * ld;  // resident twiddles (a.tw_res)
  C* end = twsm + a.tw_res;
  unsigned long long* bars =
      reinterpret_cast<unsigned long long*>(reinterpret_cast<uintptr_t>(end + 1) & ~(uintptr_t)7);
  const bool lm = a.mode == 1;
  const int tid = threadIdx.x;
  const int l = lm ? tid % L : tid / P;
  const int t = lm ? tid / L : tid % P;
  long long tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  if (smem_u32(smraw) & 127) {  // the tile slots must start on 128 bytes: report, never copy
    if (tid == 0) atomicExch(a.err, 1u);
    return;
  }
  const long long G = gridDim.x;
  if (tid == 0) {
    for (int k = 0; k < ns; ++k) mbar_init(&bars[k], 1);
    fence_proxy_async();
    // a CTA with a single tile never prefetches: the twiddle table is staged
    // in the idle second slot on the tile's barrier (stage twiddles then come
    // from shared memory instead of L1 misses to L2).  The table belongs to
    // the plan, so its copy starts before the wait below.
    if (a.tw_bytes) {
      mbar_expect_tx_only(&bars[0], a.tw_bytes);
      bulk_load(slots[1], a.tw, a.tw_bytes, &bars[0]);
    }
    // launched with programmatic stream serialization, this CTA may start
    // while the previous pass is finishing: thread 0, the only thread that
    // touches the previous pass's output or this pass's output (the tile
    // copies), waits for it to complete here; the other threads read only the
    // plan's twiddle table
    griddep_wait();
    tma_issue_load(a, tile, slots[0], &bars[0]);
    for (int d = 1; d < ns - 1; ++d)
      if (tile + d * G < a.ntiles) tma_issue_load(a, tile + d * G, slots[d], &bars[d]);
  }
  // the next pass may launch onto SMs this one frees (it waits for this one
  // to complete before touching memory)
  griddep_launch_dependents();
  // a persistent CTA copies the table once into its own region
  for (int i = tid; i < a.tw_res; i += blockDim.x) twsm[i] = a.tw[i];
  __syncthreads();
  const C* twb = a.tw_res ? twsm : a.tw_bytes ? slots[1] : a.tw;
  for (int it = 0;; ++it) {
    const int cs = it % ns;
    const long long pf = tile + (long long)(ns - 1) * G;  // the tile whose load is issued now
    if (tid == 0) {
      bulk_wait_read0();  // the previous tile's store has finished reading its buffer (slot (it - 1) % ns)
      if (pf < a.ntiles) tma_issue_load(a, pf, slots[(it + ns - 1) % ns], &bars[(it + ns - 1) % ns]);
    }
    const bool ok = mbar_wait(&bars[cs], (unsigned)((it / ns) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(a.err, 1u);
        // let the loads already in flight land before the CTA leaves (bounded)
        for (int d = 1; d < ns; ++d)
          if (tile + d * G < a.ntiles) mbar_wait(&bars[(it + d) % ns], (unsigned)(((it + d) / ns) & 1));
        bulk_wait0();
      }
      return;
    }
    C* cur = slots[cs];
    C* obuf = tma_stages<T, INV, V, IP, FX>(a, cur, work, twb, l, t);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) tma_issue_store(a, tile, obuf);
    if (a.hm_cmax > 0) {
      hermitian_mirror(a, tile, obuf, tid);
      __syncthreads();  // the slot (or work buffer) is refilled next iteration
    }
    tile += G;
    if (tile >= a.ntiles) break;
  }
  if (tid == 0) bulk_wait0();
}

// ───────────────────── two axis passes, plane by plane ─────────────────────
//
// The first two axis passes of a 3D transform (forward: z then y; inverse: y
// then z) both stay inside one x-plane (the outermost index), so they can run
// plane by plane: a thread-block cluster owns a plane, its CTAs transform the
// plane's phase-0 tiles, meet at the cluster barrier, then transform its
// phase-1 tiles.  The plane between the two phases (1 MiB at 256^2
// complex128) is written and read back through L2 while few enough planes are
// in flight (the clusters in flight x the plane size stays far below the 126
// MB L2), so a 3D transform reads and writes the volume in DRAM twice instead
// of three times.  The only synchronization is one cluster barrier per plane.
//
// The cluster barrier has no timeout, so every CTA of a cluster reaches every
// barrier: a CTA whose bounded wait timed out sets the error word and skips
// the rest of its copies and transforms, but keeps arriving.

template <class T> struct TmaPairArgs {
  TmaArgs<T> ph[2];   // phase 0 and phase 1 (the CTA has the larger L * P of the two)
  long long planes;   // x-planes (outermost index, batch included)
  int n0, n1;         // tiles per plane of each phase
  int slot_elems;     // per slot: the larger of the two phases
};

// This CTA's work items: per plane q of the cluster (p = cluster + q * clusters),
// its phase-0 tiles r, r + CS, ... < n0, one barrier, its phase-1 tiles
// r, r + CS, ... < n1.  Position `pos` within a plane: < a0 phase 0, == a0 the
// barrier, > a0 phase 1.  The schedule lives in shared memory, written by
// thread 0 and read by every thread after a CTA barrier: nothing of it is live
// in registers while a tile is transformed (the stages of the complex128
// build use all 168 registers the three-CTA occupancy allows).
struct PairCtl {
  int q, pos;     // the item being processed
  int cs;         // slot of the tile being transformed
  int par[2];     // mbarrier phase of each slot
  int bad;        // a bounded wait timed out: no more copies or transforms (barriers go on)
  int prefetch;   // the next item is a tile whose load was issued with this one's transform
};

struct PairGeo {
  int r, CS, a0, a1, A;
  long long cid, ncl, nq;
};

template <class T> __device__ __forceinline__ PairGeo pair_geo(const TmaPairArgs<T>& pa) {
  PairGeo g;
  g.r = (int)cluster_rank();
  g.CS = (int)cluster_nrank();
  g.cid = cluster_id();
  g.ncl = cluster_count();
  g.nq = g.cid < pa.planes ? (pa.planes - 1 - g.cid) / g.ncl + 1 : 0;  // planes of this cluster
  g.a0 = g.r < pa.n0 ? (pa.n0 - 1 - g.r) / g.CS + 1 : 0;               // this CTA's tiles per phase
  g.a1 = g.r < pa.n1 ? (pa.n1 - 1 - g.r) / g.CS + 1 : 0;
  g.A = g.a0 + 1 + g.a1;  // items per plane, the barrier included
  return g;
}

// (phase, global tile) of the item at (q, pos), pos != a0
template <class T>
__device__ __forceinline__ long long pair_tile(const TmaPairArgs<T>& pa, const PairGeo& g, int q, int pos, int& ph) {
  const long long p = g.cid + (long long)q * g.ncl;
  if (pos < g.a0) {
    ph = 0;
    return p * pa.n0 + g.r + (long long)pos * g.CS;
  }
  ph = 1;
  return p * pa.n1 + g.r + (long long)(pos - g.a0 - 1) * g.CS;
}

__device__ __forceinline__ void pair_advance(const PairGeo& g, int& q, int& pos) {
  if (++pos == g.A) {
    pos = 0;
    ++q;
  }
}

template <class T, bool INV, int V, bool IP>
__device__ __forceinline__ typename CT<T>::type* pair_transform(const TmaArgs<T>& a, typename CT<T>::type* slot,
                                                                typename CT<T>::type* work,
                                                                const typename CT<T>::type* tw, int tid) {
  const bool lm = a.mode == 1;
  const int L = a.L, P = a.P;
  // a phase with fewer threads than the CTA leaves the rest idle (no
  // butterflies: t beyond every stage's count), still at every barrier
  const bool act = tid < L * P;
  const int l = !act ? 0 : lm ? tid % L : tid / P;
  const int t = !act ? (1 << 20) : lm ? tid / L : tid % P;
  return tma_stages<T, INV, V, IP>(a, slot, work, tw, l, t);
}

template <class T, bool INV, int V, bool IP>
__global__ void __launch_bounds__(TmaBuild<T, V>::threads, TmaBuild<T, V>::ctas)
    tma_pair_kernel(const __grid_constant__ TmaPairArgs<T> pa) {
  using C = typename CT<T>::type;
  // no static shared variables: they would move the dynamic block off the
  // 128-byte boundary the tensor copies' destinations need
  extern __shared__ __align__(128) unsigned char smraw[];
  C* const slot0 = reinterpret_cast<C*>(smraw);
  C* const slot1 = slot0 + pa.slot_elems;
  int wl = pa.ph[0].L * pa.ph[0].ld;
  if (pa.ph[1].L * pa.ph[1].ld > wl) wl = pa.ph[1].L * pa.ph[1].ld;
  C* const work = IP ? nullptr : slot1 + pa.slot_elems;
  C* const tw0 = IP ? slot1 + pa.slot_elems : work + wl;  // resident twiddles of each phase (tw_res)
  C* const tw1 = tw0 + pa.ph[0].tw_res;
  C* end = tw1 + pa.ph[1].tw_res;
  unsigned long long* const bars =
      reinterpret_cast<unsigned long long*>(reinterpret_cast<uintptr_t>(end + 1) & ~(uintptr_t)7);
  volatile PairCtl* const ctl = reinterpret_cast<volatile PairCtl*>(bars + 2);
  const int tid = threadIdx.x;
  // a misaligned block is a plan error every CTA of the launch sees alike: no
  // CTA copies, and none reaches a cluster barrier
  if (smem_u32(smraw) & 127) {
    if (tid == 0) atomicExch(pa.ph[0].err, 1u);
    return;
  }
  if (tid == 0) {
    const PairGeo g = pair_geo(pa);
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_proxy_async();
    ctl->q = g.nq > 0 ? 0 : 1 << 30;
    ctl->pos = g.a0 == 0 ? -1 : 0;  // no phase-0 tile here: the plane starts at its barrier
    ctl->cs = 0;
    ctl->par[0] = ctl->par[1] = 0;
    ctl->bad = 0;
    ctl->prefetch = 0;
    if (g.nq > 0 && g.a0 > 0) {
      int ph;
      const long long tile = pair_tile(pa, g, 0, 0, ph);
      tma_issue_load(pa.ph[ph], tile, slot0, &bars[0]);
    }
  }
  for (int i = tid; i < pa.ph[0].tw_res; i += blockDim.x) tw0[i] = pa.ph[0].tw[i];
  for (int i = tid; i < pa.ph[1].tw_res; i += blockDim.x) tw1[i] = pa.ph[1].tw[i];
  __syncthreads();
  for (;;) {
    // every thread reads the item; thread 0 wrote it before the last barrier
    const int q = ctl->q;
    if (q >= (1 << 30)) break;
    const int bad = ctl->bad;
    if (ctl->pos < 0) {
      // the barrier between a plane's phases: this CTA's phase-0 stores are
      // complete and visible before any CTA of the cluster loads phase-1 tiles
      cluster_sync_all();
      if (tid == 0) {
        const PairGeo g = pair_geo(pa);
        int nq_ = q, pos = g.a0;
        pair_advance(g, nq_, pos);
        if (nq_ < g.nq && pos != g.a0 && !bad) {
          fence_proxy_async_global();  // the tensor loads below read what the barrier published
          int ph;
          const long long tile = pair_tile(pa, g, nq_, pos, ph);
          const int cs = ctl->cs ^ 1;
          tma_issue_load(pa.ph[ph], tile, cs ? slot1 : slot0, &bars[cs]);
          ctl->cs = cs;
        } else if (nq_ < g.nq && pos != g.a0) {
          ctl->cs ^= 1;
        }
        ctl->q = nq_ < g.nq ? nq_ : 1 << 30;
        ctl->pos = pos == g.a0 ? -1 : pos;
      }
      __syncthreads();
      continue;
    }
    const int cs = ctl->cs;
    const unsigned par = (unsigned)ctl->par[cs];
    C* const cur = cs ? slot1 : slot0;
    int ph = 0;
    if (tid == 0) {
      const PairGeo g = pair_geo(pa);
      const int pos = ctl->pos;
      int nq_ = q, npos = pos;
      pair_advance(g, nq_, npos);
      const bool prefetch = nq_ < g.nq && npos != g.a0;  // no barrier between: load the next tile now
      ctl->prefetch = prefetch;
      if (!bad) {
        bulk_wait_read0();  // the previous tile's store has finished reading its buffer
        if (prefetch) {
          int nph;
          const long long ntile = pair_tile(pa, g, nq_, npos, nph);
          tma_issue_load(pa.ph[nph], ntile, cs ? slot0 : slot1, &bars[cs ^ 1]);
        }
      }
    }
    bool ok = true;
    if (!bad) ok = mbar_wait(&bars[cs], par);
    const bool timed_out = __syncthreads_or(!ok);
    if (tid == 0) {
      ctl->par[cs] = (int)(par ^ 1u);
      if (timed_out && !bad) {
        atomicExch(pa.ph[0].err, 1u);
        if (ctl->prefetch) mbar_wait(&bars[cs ^ 1], (unsigned)ctl->par[cs ^ 1]);  // let it land (bounded)
        bulk_wait0();
        ctl->bad = 1;
      }
    }
    if (!bad && !timed_out) {
      ph = ctl->pos < pair_geo(pa).a0 ? 0 : 1;
      C* obuf = pair_transform<T, INV, V, IP>(pa.ph[ph], cur, work, pa.ph[ph].tw_res ? (ph ? tw1 : tw0) : pa.ph[ph].tw,
                                              tid);
      fence_proxy_async();
      __syncthreads();
      if (tid == 0) {
        const PairGeo g = pair_geo(pa);
        int tph;
        const long long tile = pair_tile(pa, g, ctl->q, ctl->pos, tph);
        tma_issue_store(pa.ph[tph], tile, obuf);
      }
    }
    if (tid == 0) {
      const PairGeo g = pair_geo(pa);
      int nq_ = ctl->q, npos = ctl->pos;
      pair_advance(g, nq_, npos);
      if (ctl->prefetch) ctl->cs = cs ^ 1;
      if (nq_ < g.nq && npos == g.a0) {
        // the plane's barrier comes next: complete and publish this CTA's stores
        if (!ctl->bad) {
          bulk_wait0();
          fence_proxy_async_global();
        }
        npos = -1;
      }
      ctl->q = nq_ < g.nq ? nq_ : 1 << 30;
      ctl->pos = npos;
    }
    __syncthreads();
  }
  if (tid == 0 && !ctl->bad) bulk_wait0();
}

// ─────────────────────────────── host side ───────────────────────────────

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

static bool make_map(CUtensorMap* m, const void* base, bool dbl, long long es, long long n, long long outer, int L,
                     int bn) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const size_t el = dbl ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)(2 * es), (cuuint64_t)n, (cuuint64_t)outer};
  cuuint64_t strides[2] = {(cuuint64_t)(2 * es * el), (cuuint64_t)(2 * es * n * el)};
  cuuint32_t box[3] = {(cuuint32_t)(2 * L), (cuuint32_t)bn, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, dbl ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base),
                  dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tma_lane_map(CUtensorMap* m, const void* base, bool dbl, long long es, long long n, long long outer, int L,
                  int bn) {
  return make_map(m, base, dbl, es, n, outer, L, bn);
}

static int g_tma_sm = 0;

size_t tma_smem_bytes(const TmaPlan& tp, size_t csz) {
  return (size_t)tp.nslot * tp.slot_elems * csz + (tp.inplace ? 0 : (size_t)tp.L * tp.ld * csz) +
         (size_t)tp.tw_res * csz + 64;
}

// Twiddle entries the stages read (r-major, twoff + (R - 1) Ns per stage).
static long long twiddle_count(const StageList& sl) {
  long long twc = 0;
  for (int s = 0; s < sl.nst; ++s)
    if (sl.st[s].Ns > 1) twc = std::max<long long>(twc, sl.st[s].twoff + (long long)(sl.st[s].R - 1) * sl.st[s].Ns);
  return twc;
}

// CTAs per SM the register budget of a kernel build allows (its launch bounds).
static int build_ctas_per_sm(int variant, bool dbl) {
  if (variant == 2 || (variant == 5 && dbl) || (variant == 6 && !dbl)) return 3;
  if (variant == 3 || variant == 7 || ((variant == 1 || variant == 4 || variant == 5 || variant == 8) && !dbl))
    return 2;
  return 1;
}

// Threads per CTA a kernel build is compiled for (its launch bounds).
static int build_threads(int variant, bool dbl) { return (variant == 2 || (variant == 5 && dbl)) ? 128 : 256; }

// The compile-time stage lists built (variant 7): the smooth odd axis lengths
// of the 243 x 250 x 343 volume, with the thread and lane counts tma_plan
// picks for them (contiguous tiles, and strided tiles of 8 complex128 / 16
// complex64 lanes).
#define AFC_FIXED_LIST(X)                                                                                \
  X(true, 343, 7, 7, 7, 22, 0) X(true, 343, 7, 7, 7, 22, 8) X(true, 243, 9, 9, 3, 16, 0)              \
  X(true, 243, 9, 9, 3, 16, 8) X(true, 250, 10, 5, 5, 16, 0) X(true, 250, 10, 5, 5, 16, 8)            \
  X(false, 343, 7, 7, 7, 22, 0) X(false, 343, 7, 7, 7, 11, 16) X(false, 243, 9, 9, 3, 16, 0)          \
  X(false, 243, 9, 9, 3, 16, 16) X(false, 250, 10, 5, 5, 16, 0) X(false, 250, 10, 5, 5, 16, 16)
struct FixedEntry {
  bool dbl;
  int n, r0, r1, r2, r3, P, LK;
};
static const FixedEntry kFixed[] = {
#define AFC_FX_ENTRY(D, N, R0, R1, R2, P, LK) {D, N, R0, R1, R2, 0, P, LK},
    AFC_FIXED_LIST(AFC_FX_ENTRY)
#undef AFC_FX_ENTRY
};
// The in-place power-of-two stage lists built (variant 8): 2048 points in
// complex64 (the 2048 x 2048 images), contiguous (complex or real lanes) and
// strided tiles of 2 lanes.
#define AFC_FIXED_IP_LIST(X)                                                                            \
  X(false, 2048, 16, 16, 8, 0, 128, 0) X(false, 2048, 16, 16, 8, 0, 128, 4) X(false, 2048, 16, 16, 8, 0, 128, 2)
static const FixedEntry kFixedIP[] = {
#define AFC_FXI_ENTRY(D, N, R0, R1, R2, R3, P, LK) {D, N, R0, R1, R2, R3, P, LK},
    AFC_FIXED_IP_LIST(AFC_FXI_ENTRY)
#undef AFC_FXI_ENTRY
};
// Keeps the twiddle table resident in shared memory when that costs no CTA
// per SM (228 KB per SM, 1 KB reserved per CTA), for the odd-radix builds
// only: measured on B200, 243 x 250 x 343 complex128 went from 1.32 to 1.25 ms
// per forward + inverse, while the power-of-two passes, whose shared memory is
// already the busiest unit, got slower (16384 x 4096 complex64: 333 -> 355 us).
static void plan_resident_twiddles(const StageList& sl, bool dbl, TmaPlan& tp, size_t extra = 0) {
  const size_t csz = dbl ? 16 : 8;
  tp.tw_res = 0;
  if (tp.variant != 0 && tp.variant != 3 && tp.variant != 7) return;
  const long long twc = twiddle_count(sl);
  if (twc <= 0) return;
  const size_t base = tma_smem_bytes(tp, csz) + extra;
  const int ctas = build_ctas_per_sm(tp.variant, dbl);
  if ((size_t)ctas * (base + (size_t)twc * csz + 1024) <= 233472 && base + (size_t)twc * csz <= 220 * 1024)
    tp.tw_res = (int)twc;
}

// Decides whether an axis pass can run on the TMA kernel and with which tiles.
bool tma_plan(const StageList& sl, int ld, long long lanes, const LaneMap& im, const LaneMap& om, const void* in,
              void* out, bool dbl, int lanes_pref, TmaPlan& tp, bool real_in, bool real_out, bool mirror) {
  const size_t csz = dbl ? 16 : 8;
  const long long n = sl.n;
  const bool real = real_in || real_out;
  if (real && (im.es != 1 || (n * (long long)(csz / 2)) % 16)) return false;
  if (im.off || om.off) return false;
  if (im.d1 != 1 || om.d1 != 1 || im.d2 != om.d2 || im.s0 != om.s0 || im.es != om.es || im.s2 != om.s2) return false;
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) return false;
  if (n < 2) return false;
  // contiguous complex64 lanes of odd length: a lane starts on 8 bytes only,
  // so tiles hold an even number of lanes and start at even lanes
  const bool lane2 = im.es == 1 && (n * (long long)csz) % 16 != 0;
  if (im.es == 1) {  // contiguous lanes at q * n
    if (im.d2 != 1 || im.s0 != n) return false;
    if (lane2 && (real || (n * (long long)csz) % 8 || (lanes & 1))) return false;
    tp.mode = 0;
    tp.L = 1;
    tp.bn = (int)n;
    tp.nbx = 1;
    tp.kb = 1;
  } else {  // strided lanes: lane (o, k) at o * n * es + k, element stride es
    const long long es = im.es;
    if (im.d2 != es || im.s0 != n * es || im.s2 != 1) return false;
    if (!dbl && (es & 1)) return false;  // 16-byte tensor strides
    if (lanes % es) return false;
    tp.mode = 1;
    tp.L = lanes_pref > 0 ? lanes_pref : (dbl ? 8 : 16);
    tp.nbx = (int)((n + 255) / 256);
    tp.bn = (int)((n + tp.nbx - 1) / tp.nbx);
    // long axes: narrower tiles (down to 16-byte rows) until two slots and a
    // work buffer fit twice per SM
    const long long rows = (long long)tp.nbx * tp.bn;
    const int Lmin = dbl ? 1 : 2;
    while (lanes_pref <= 0 && tp.L > Lmin &&
           3 * (size_t)tp.L * (size_t)std::max<long long>(ld, rows) * csz + 64 > 110 * 1024)
      tp.L /= 2;
    tp.kb = (es + tp.L - 1) / tp.L;
  }
  tp.ld = ld;
  // threads: one radix-16 butterfly per thread and stage when possible
  int P = (int)std::max<long long>(1, std::min<long long>(256, (n + 15) / 16));
  bool p2 = true;
  long long nbmax = 1;
  for (int i = 0; i < sl.nst; ++i) {
    const int R = sl.st[i].R;
    p2 = p2 && (R == 2 || R == 4 || R == 8 || R == 16);
    nbmax = std::max<long long>(nbmax, n / R);
  }
  (void)nbmax;
  if (real && !p2) return false;  // real lanes need in-place stages
  // in place: a thread holds one butterfly per stage (complex64: two of a radix <= 8 stage)
  auto fits_inplace = [&](int Pc, bool two) {
    if (!p2) return false;
    for (int i = 0; i < sl.nst; ++i) {
      const long long nb = n / sl.st[i].R;
      if ((nb + Pc - 1) / Pc > ((two && sl.st[i].R <= 8 && !dbl) ? 2 : 1)) return false;
    }
    return true;
  };
  // complex128 power-of-two tiles of <= 128 threads whose stages run in place
  // use the three-CTA build
  const bool ip128 = P <= 128 && fits_inplace(P, false);
  static const int v2_on = [] {
    const char* e = getenv("AFC_TMA_V2");
    return e && *e ? atoi(e) : 1;
  }();
  const int tmax = (v2_on && dbl && p2 && ip128) ? 128 : 256;
  if (tp.mode == 0) {
    int L = std::max(1, tmax / P);
    if (lane2) L = std::max(2, L & ~1);
    tp.L = L;
  }
  while (tp.L * P > tmax) P = std::max(1, P / 2);
  tp.P = P;
  bool s7 = true;
  for (int i = 0; i < sl.nst; ++i) s7 = s7 && sl.st[i].R != 11 && sl.st[i].R != 13;
  static const int v3_on = [] {
    const char* e = getenv("AFC_TMA_V3");
    return e && *e ? atoi(e) : 1;
  }();
  tp.variant = p2 ? (tmax == 128 ? 2 : 1) : ((s7 && v3_on) ? 3 : 0);
  // in place only for power-of-two plans: odd-radix butterflies held across
  // the barrier cost spills
  tp.inplace = fits_inplace(P, false);
  if (!tp.inplace && !dbl && fits_inplace(P, true)) {
    tp.inplace = true;
    tp.variant = 4;
  }
  if (real && !tp.inplace) return false;
  // a 7-smooth out-of-place plan whose stage list, threads and tile are built
  // at compile time (AFC_TMA_FIXED=0 keeps the general build; read at every plan)
  {
    const char* fx_env = getenv("AFC_TMA_FIXED");
    const bool fx_on = !(fx_env && *fx_env && atoi(fx_env) == 0);
    const int nent = (int)(sizeof(kFixed) / sizeof(kFixed[0]));
    for (int i = 0; fx_on && tp.variant == 3 && !tp.inplace && !real && i < nent; ++i) {
      const FixedEntry& e = kFixed[i];
      const int nst = e.r2 ? 3 : 2;
      if (e.dbl != dbl || e.n != n || sl.nst != nst || sl.st[0].R != e.r0 || sl.st[1].R != e.r1 ||
          (nst == 3 && sl.st[2].R != e.r2) || P != e.P)
        continue;
      if (e.LK == 0 ? tp.mode != 0 : (tp.mode != 1 || tp.L != e.LK)) continue;
      tp.variant = 7;
      tp.fix = i;
      break;
    }
    const int nip = (int)(sizeof(kFixedIP) / sizeof(kFixedIP[0]));
    for (int i = 0; fx_on && (tp.variant == 1 || tp.variant == 4) && tp.inplace && i < nip; ++i) {
      const FixedEntry& e = kFixedIP[i];
      const int nst = e.r3 ? 4 : e.r2 ? 3 : 2;
      if (e.dbl != dbl || e.n != n || sl.nst != nst || sl.st[0].R != e.r0 || sl.st[1].R != e.r1 ||
          (nst >= 3 && sl.st[2].R != e.r2) || (nst >= 4 && sl.st[3].R != e.r3) || P != e.P)
        continue;
      // strided tiles of 4 lanes at 512 threads (one CTA per SM, two 70 KB
      // slots) in place of the planner's 2 lanes at two CTAs per SM: half as
      // many 16-byte TMA rows per point.  Measured on B200, 8 x 2048^2 R2C
      // forward 0.31 -> 0.285 ms, forward + backward 1.59 -> 1.47 ms.
      // AFC_TMA_L4=0 keeps 2 lanes.
      const char* l4_env = getenv("AFC_TMA_L4");
      const bool l4_on = !(l4_env && *l4_env && atoi(l4_env) == 0);
      const bool widen = e.LK == 4 && l4_on && tp.mode == 1 && tp.L == 2 && !real;
      if (!widen && (e.LK == 0 ? tp.mode != 0 : (tp.mode != 1 || tp.L != e.LK || real))) continue;
      if (ld != ((e.n + (e.n - 1) / 16 + 1) | 1) || (!widen && tp.L * P > 256)) continue;
      if (widen) {
        tp.L = 4;
        tp.kb = (im.es + tp.L - 1) / tp.L;
      }
      tp.variant = 8;
      tp.fix = i;
      break;
    }
  }
  // n = 256 as radix 16 x 16 on complex lanes: the build with fixed addresses.
  // Measured on B200 at 256^3 (forward, 20 warm repetitions): complex64 went
  // from 206 to 151 us per transform (2.6x fewer instructions: the general
  // stages' address and select arithmetic bounded the passes), while
  // complex128, whose passes are DRAM-bound at 3 CTAs per SM either way, went
  // from 285 to 298 us (twiddles resident in shared memory changed nothing),
  // so complex128 keeps the general build.  AFC_TMA_N256: 0 off, 1 complex64
  // (default), 2 both; read at every plan.
  const char* n256_env = getenv("AFC_TMA_N256");
  const int n256_on = n256_env && *n256_env ? atoi(n256_env) : 1;
  if (n256_on && (!dbl || n256_on >= 2) && n == 256 && sl.nst == 2 && sl.st[0].R == 16 && sl.st[1].R == 16 && sl.st[0].Ns == 1 &&
      sl.st[1].Ns == 16 && tp.inplace && !real && ld == 273 && P == 16 &&
      (tp.variant == 2 || (tp.variant == 1 && !dbl)) && tp.L * P == build_threads(5, dbl) &&
      (tp.mode == 0 || tp.L == (dbl ? 8 : 16)))
    tp.variant = 5;
  // n = 4096 as radix 16 x 16 x 16 on one contiguous complex lane per tile:
  // the fixed-address build.  Measured on B200: 16384 x 4096 complex64
  // forward from 350 to 255 us, 64 x 4096 complex128 forward + inverse from
  // 20.8 to 17.9 us.  AFC_TMA_N4096: 0 off, 1 complex64 only, 2 both (default).
  const char* n4096_env = getenv("AFC_TMA_N4096");
  const int n4096_on = n4096_env && *n4096_env ? atoi(n4096_env) : 2;
  if (n4096_on && (!dbl || n4096_on >= 2) && n == 4096 && sl.nst == 3 && sl.st[0].R == 16 && sl.st[1].R == 16 &&
      sl.st[2].R == 16 && sl.st[0].Ns == 1 && sl.st[1].Ns == 16 && sl.st[2].Ns == 256 && tp.inplace && !real &&
      ld == 4353 && P == 256 && tp.mode == 0 && tp.L == 1 && tp.variant == 1)
    tp.variant = 6;
  tp.real_in = real_in;
  tp.real_out = real_out;
  const int align = dbl ? 8 : 16;  // 128-byte aligned slots
  long long rows = tp.mode == 1 ? (long long)tp.nbx * tp.bn : n;
  long long se = (long long)tp.L * std::max<long long>(ld, rows);
  se = (se + align - 1) / align * align;
  tp.slot_elems = (int)se;
  // shrink the contiguous tile until it fits comfortably
  while (tp.mode == 0 && tp.L > (lane2 ? 2 : 1) && tma_smem_bytes(tp, csz) > 110 * 1024) {
    tp.L -= lane2 ? 2 : 1;
    se = (long long)tp.L * std::max<long long>(ld, n);
    se = (se + align - 1) / align * align;
    tp.slot_elems = (int)se;
  }
  if (tp.variant == 8) {  // the slot holds the tile in the build's padded layout
    const FixedEntry& e = kFixedIP[tp.fix];
    const long long need = ((long long)tp.L * fixip_ld(e.n, e.LK, (int)csz) + align - 1) / align * align;
    if (need > tp.slot_elems) tp.slot_elems = (int)need;
  }
  if (tma_smem_bytes(tp, csz) > 220 * 1024) return false;
  // a third slot (two tile loads in flight per CTA) when it costs no CTA per
  // SM: the passes whose CTAs hold few bytes in flight are bandwidth x latency
  // bound with two
  {
    TmaPlan t3 = tp;
    t3.nslot = 3;
    const size_t b3 = tma_smem_bytes(t3, csz);
    const int ctas = build_ctas_per_sm(tp.variant, dbl);
    // measured on B200: no pass got faster with the third slot (16384 x 4096
    // complex64 went from 355 to 386 us, its smem displacing the resident
    // twiddles), so two slots stay the default; AFC_TMA_SLOTS=3 opts in
    static const int slots_env = [] {
      const char* e = getenv("AFC_TMA_SLOTS");
      return e && *e ? atoi(e) : 2;
    }();
    if (slots_env >= 3 && (size_t)ctas * (b3 + 1024) <= 233472 && b3 <= 220 * 1024) tp.nslot = 3;
  }
  plan_resident_twiddles(sl, dbl, tp);
  // Hermitian input rows: tiles over columns [0, kb L) with kb L > es / 2,
  // columns [kb L, es) stored as mirrors of columns [1, es - kb L]
  if (mirror && tp.mode == 1 && !real) {
    const long long kbh = im.es / 2 / tp.L + 1;
    if (kbh < tp.kb && im.es - kbh * tp.L > 0) {
      tp.kb = kbh;
      tp.hm_cmax = (int)(im.es - kbh * tp.L);
    }
  }
  tp.ntiles = tp.mode == 0 ? (lanes + tp.L - 1) / tp.L : (lanes / im.es) * tp.kb;
  tp.outer = tp.mode == 1 ? lanes / im.es : 0;
  return true;
}

// Kernel arguments of one axis pass on the TMA kernels (tensor maps for
// strided lanes); false when a tensor map cannot be encoded.
template <class T> static bool fill_tma_args(const LaunchDesc& d, const TmaPlan& tp, unsigned* err, TmaArgs<T>& a) {
  using C = typename CT<T>::type;
  memset(&a, 0, sizeof(a));
  const bool dbl = sizeof(T) == 8;
  if (tp.mode == 1) {
    if (!make_map(&a.tmi, d.in, dbl, d.im.es, d.sl.n, tp.outer, tp.L, tp.bn)) return false;
    if (!make_map(&a.tmo, d.out, dbl, d.om.es, d.sl.n, tp.outer, tp.L, tp.bn)) return false;
  }
  a.sl = d.sl;
  a.tw = static_cast<const C*>(d.tw);
  a.in = static_cast<const C*>(d.in);
  a.out = static_cast<C*>(d.out);
  a.lanes = d.lanes;
  a.ntiles = tp.ntiles;
  a.kb = tp.kb;
  a.L = tp.L;
  a.P = tp.P;
  a.ld = tp.ld;
  a.slot_elems = tp.slot_elems;
  a.mode = tp.mode;
  a.inplace = tp.inplace ? 1 : 0;
  a.real_in = tp.real_in ? 1 : 0;
  a.real_out = tp.real_out ? 1 : 0;
  a.nbx = tp.nbx;
  a.bn = tp.bn;
  a.scale = (T)d.scale;
  a.err = err;
  a.tw_res = tp.tw_res;
  a.nslot = tp.nslot;
  a.hm_out = static_cast<C*>(d.out);
  a.hm_es = d.om.es;
  a.hm_cmax = tp.hm_cmax;
  a.out_cols = tp.store_cols;
  return true;
}

static int sm_count() {
  if (g_tma_sm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_tma_sm, cudaDevAttrMultiProcessorCount, dev);
    if (g_tma_sm <= 0) g_tma_sm = 148;
  }
  return g_tma_sm;
}

template <class T, bool INV> static auto fixed_kernel(int fix) -> decltype(&tma_kernel<T, INV, 0, false>) {
  int i = 0;
#define AFC_FX_KERNEL(D, N, R0, R1, R2, P, LK)                                  \
  if constexpr ((sizeof(T) == 8) == D) {                                        \
    if (fix == i) return &tma_kernel<T, INV, 7, false, Fix<N, R0, R1, R2, P, LK>>; \
  }                                                                             \
  ++i;
  AFC_FIXED_LIST(AFC_FX_KERNEL)
#undef AFC_FX_KERNEL
  return nullptr;
}
template <class T, bool INV> static auto fixed_ip_kernel(int fix) -> decltype(&tma_kernel<T, INV, 0, false>) {
  int i = 0;
#define AFC_FXI_KERNEL(D, N, R0, R1, R2, R3, P, LK)                                       \
  if constexpr ((sizeof(T) == 8) == D) {                                                  \
    if (fix == i) return &tma_kernel<T, INV, 8, true, FixIP<N, R0, R1, R2, R3, P, LK>>; \
  }                                                                                       \
  ++i;
  AFC_FIXED_IP_LIST(AFC_FXI_KERNEL)
#undef AFC_FXI_KERNEL
  return nullptr;
}

template <class T, bool INV>
static cudaError_t launch_tma_t(const LaunchDesc& d, const TmaPlan& tp, unsigned* err, cudaStream_t st) {
  using C = typename CT<T>::type;
  auto k = tp.variant == 8  ? fixed_ip_kernel<T, INV>(tp.fix)
           : tp.variant == 7 ? fixed_kernel<T, INV>(tp.fix)
           : tp.variant == 6 ? tma_kernel<T, INV, 6, true>
           : tp.variant == 5 ? tma_kernel<T, INV, 5, true>
           : tp.variant == 4 ? tma_kernel<T, INV, 4, true>
           : tp.variant == 2 ? tma_kernel<T, INV, 2, true>
           : tp.variant == 1 ? (tp.inplace ? tma_kernel<T, INV, 1, true> : tma_kernel<T, INV, 1, false>)
           : tp.variant == 3 ? tma_kernel<T, INV, 3, false>
                             : tma_kernel<T, INV, 0, false>;
  if (!k) return cudaErrorInvalidValue;
  const size_t smem = tma_smem_bytes(tp, sizeof(C));
  cudaError_t e = kernel_smem_grant(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  TmaArgs<T> a;
  if (!fill_tma_args<T>(d, tp, err, a)) return cudaErrorInvalidValue;
  const int per_sm = kernel_ctas_per_sm(reinterpret_cast<const void*>(k), tp.L * tp.P, smem);
  long long grid = (long long)sm_count() * per_sm;
  if (grid >= tp.ntiles) {
    // one tile per CTA: stage the twiddle table (r-major, twoff + (R - 1) Ns
    // entries per stage) in the second slot when it fits and can be bulk-copied
    const long long twc = twiddle_count(d.sl);
    const long long twb = twc * (long long)sizeof(C);
    if (twc > 0 && twb % 16 == 0 && twc <= tp.slot_elems && (reinterpret_cast<uintptr_t>(d.tw) & 15) == 0) {
      a.tw_bytes = (unsigned)twb;
      a.tw_res = 0;
    }
  }
  if (grid > tp.ntiles) grid = tp.ntiles;
  // programmatic stream serialization for passes whose CTAs each take one
  // tile (latency-bound launches): the pass's CTAs may start on SMs the
  // previous launch in the stream frees while its last CTAs finish, and set up
  // while it drains (the kernel's thread 0 waits for that launch before any
  // global copy).  Measured on B200: 64 x 4096 complex128 forward + inverse
  // 16.5 -> 14.4 us; on the persistent bandwidth-bound passes it cost time
  // (256^3 complex128 0.580 -> 0.595 ms, 8 x 2048^2 R2C 0.301 -> 0.330 ms),
  // so they launch plainly.  AFC_PDL: 0 never, 1 single-round passes
  // (default), 2 every pass.
  static const int pdl_env = [] {
    const char* e = getenv("AFC_PDL");
    return e && *e ? atoi(e) : 1;
  }();
  const bool pdl = pdl_env >= 2 || (pdl_env == 1 && tp.ntiles <= grid);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3((unsigned)(tp.L * tp.P), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  e = cudaLaunchKernelEx(&cfg, k, a);
  count_launch(1);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <class T, bool INV> static const void* pair_kernel_ptr(int variant, bool ip) {
  auto k = variant == 6   ? tma_pair_kernel<T, INV, 6, true>
           : variant == 5 ? tma_pair_kernel<T, INV, 5, true>
           : variant == 4 ? tma_pair_kernel<T, INV, 4, true>
           : variant == 2 ? tma_pair_kernel<T, INV, 2, true>
           : variant == 1 ? (ip ? tma_pair_kernel<T, INV, 1, true> : tma_pair_kernel<T, INV, 1, false>)
                          : tma_pair_kernel<T, INV, 3, false>;
  return reinterpret_cast<const void*>(k);
}
static const void* pair_kernel_ptr(bool dbl, bool inv, int variant, bool ip) {
  if (dbl) return inv ? pair_kernel_ptr<double, true>(variant, ip) : pair_kernel_ptr<double, false>(variant, ip);
  return inv ? pair_kernel_ptr<float, true>(variant, ip) : pair_kernel_ptr<float, false>(variant, ip);
}

// Two axis passes of the same x-planes in one launch (tma_pair_kernel).  Both
// phases must run on the same kernel build; the CTA gets the larger of the
// two phases' thread counts.  The cluster size is chosen by a small cost
// model: rounds of planes (planes / clusters in flight) times the tiles a CTA
// transforms per plane plus about half a tile for the barrier, with the
// planes in flight held to 56 MiB of L2.
bool tma_pair_plan(const LaunchDesc& d0, const LaunchDesc& d1, long long planes, long long plane_bytes, bool dbl,
                   bool inv, TmaPairPlan& pp) {
  // Opt-in (AFC_PAIR=1, read per plan execution): measured on B200 at
  // 256^3 complex128 the pair launch keeps the intermediate in L2 (DRAM bytes
  // halved) but takes 287 us against 2 x 95 us for the separate passes, whose
  // tile transform is already as slow as their DRAM traffic (shared-memory
  // and latency bound), so halving the traffic cannot pay yet.
  const char* env = getenv("AFC_PAIR");
  if (!(env && *env && atoi(env) != 0) || planes < 1) return false;
  for (int ph = 0; ph < 2; ++ph) {
    const LaunchDesc& d = ph ? d1 : d0;
    TmaPlan& tp = pp.ph[ph];
    // complex lanes, or real rows widened on load (first phase of a forward
    // real transform) / real parts stored (last phase of its inverse)
    const bool rin = d.in_op == IN_R && d.out_op == OUT_C && ph == 0;
    const bool rout = d.in_op == IN_C && d.out_op == OUT_RE && ph == 1;
    if (!(d.in_op == IN_C && d.out_op == OUT_C) && !rin && !rout) return false;
    if (!tma_plan(d.sl, d.ld, d.lanes, d.im, d.om, d.in, d.out, dbl, 0, tp, rin, rout)) return false;
    if (d.lanes % planes) return false;
    if (tp.mode == 0) {
      pp.lpp[ph] = d.lanes / planes;
      // odd-length complex64 lanes: every tile of a plane must start at an even lane
      if ((d.sl.n * (long long)(dbl ? 16 : 8)) % 16 && (pp.lpp[ph] & 1)) return false;
      pp.n[ph] = (int)((pp.lpp[ph] + tp.L - 1) / tp.L);
    } else {
      if (tp.outer != planes) return false;
      pp.lpp[ph] = 0;
      pp.n[ph] = (int)tp.kb;
    }
  }
  const TmaPlan &a = pp.ph[0], &b = pp.ph[1];
  if (a.variant != b.variant || a.inplace != b.inplace) return false;
  if (a.variant == 0) return false;  // radix 11 / 13 plans keep the separate passes
  const size_t csz = dbl ? 16 : 8;
  pp.slot_elems = std::max(a.slot_elems, b.slot_elems);
  pp.threads = std::max(a.L * a.P, b.L * b.P);
  if (pp.threads > build_threads(a.variant, dbl)) return false;
  // the fixed-address build gives every thread a butterfly in both phases
  if (a.variant == 5 && (a.L * a.P != pp.threads || b.L * b.P != pp.threads)) return false;
  pp.smem = 2 * (size_t)pp.slot_elems * csz +
            (a.inplace ? 0 : (size_t)std::max(a.L * a.ld, b.L * b.ld) * csz) + 64;
  if (pp.smem > 220 * 1024) return false;
  // both phases' twiddles resident when that costs no CTA per SM
  {
    const long long tw = (long long)pp.ph[0].tw_res + pp.ph[1].tw_res;
    const int ctas = build_ctas_per_sm(a.variant, dbl);
    if (tw > 0 && (size_t)ctas * (pp.smem + (size_t)tw * csz + 1024) <= 233472) {
      pp.smem += (size_t)tw * csz;
    } else {
      pp.ph[0].tw_res = pp.ph[1].tw_res = 0;
    }
  }
  pp.planes = planes;
  const void* k = pair_kernel_ptr(dbl, inv, a.variant, a.inplace);
  if (kernel_smem_grant(k, pp.smem) != cudaSuccess) return false;
  const long long budget = 56ll << 20;
  double best = 0;
  pp.cs = 0;
  for (int cs : {4, 8, 16}) {
    if (cs == 16 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(pp.threads, 1, 1);
    cfg.dynamicSmemBytes = pp.smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, k, &cfg) != cudaSuccess || ncl < 1) {
      cudaGetLastError();
      continue;
    }
    const long long want = std::min<long long>(ncl, planes);
    const long long use = std::min<long long>(want, std::max<long long>(1, budget / std::max<long long>(plane_bytes, 1)));
    // planes too large for the L2 budget would leave most SMs idle: the
    // separate passes are faster then
    if (2 * use < want) continue;
    const long long rounds = (planes + use - 1) / use;
    const double per = (double)((pp.n[0] + cs - 1) / cs + (pp.n[1] + cs - 1) / cs) + 0.6;
    const double cost = (double)rounds * per;
    if (!pp.cs || cost < best) {
      best = cost;
      pp.cs = cs;
      pp.nclusters = (int)use;
    }
  }
  return pp.cs > 0;
}

template <class T, bool INV>
static cudaError_t launch_tma_pair_t(const LaunchDesc& d0, const LaunchDesc& d1, const TmaPairPlan& pp, unsigned* err,
                                     cudaStream_t st) {
  const void* k = pair_kernel_ptr<T, INV>(pp.ph[0].variant, pp.ph[0].inplace);
  cudaError_t e = kernel_smem_grant(k, pp.smem);
  if (e != cudaSuccess) return e;
  TmaPairArgs<T> a;
  memset(&a, 0, sizeof(a));
  if (!fill_tma_args<T>(d0, pp.ph[0], err, a.ph[0]) || !fill_tma_args<T>(d1, pp.ph[1], err, a.ph[1]))
    return cudaErrorInvalidValue;
  for (int ph = 0; ph < 2; ++ph)
    if (pp.ph[ph].mode == 0) {  // tiles never straddle a plane
      a.ph[ph].tpp = pp.n[ph];
      a.ph[ph].lpp = pp.lpp[ph];
    }
  a.planes = pp.planes;
  a.n0 = pp.n[0];
  a.n1 = pp.n[1];
  a.slot_elems = pp.slot_elems;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pp.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(pp.nclusters * pp.cs), 1, 1);
  cfg.blockDim = dim3(pp.threads, 1, 1);
  cfg.dynamicSmemBytes = pp.smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {&a};
  e = cudaLaunchKernelExC(&cfg, k, args);
  count_launch(1);
  return e;
}

cudaError_t launch_tma_pair(const LaunchDesc& d0, const LaunchDesc& d1, const TmaPairPlan& pp, unsigned* err,
                            bool dbl, bool inv, cudaStream_t st) {
  if (dbl)
    return inv ? launch_tma_pair_t<double, true>(d0, d1, pp, err, st)
               : launch_tma_pair_t<double, false>(d0, d1, pp, err, st);
  return inv ? launch_tma_pair_t<float, true>(d0, d1, pp, err, st)
             : launch_tma_pair_t<float, false>(d0, d1, pp, err, st);
}

cudaError_t launch_tma(const LaunchDesc& d, const TmaPlan& tp, unsigned* err, bool dbl, bool inv, cudaStream_t st) {
  if (d.lanes <= 0) return cudaSuccess;
  if (dbl) return inv ? launch_tma_t<double, true>(d, tp, err, st) : launch_tma_t<double, false>(d, tp, err, st);
  return inv ? launch_tma_t<float, true>(d, tp, err, st) : launch_tma_t<float, false>(d, tp, err, st);
}

cudaError_t launch_wait_probe(unsigned* err, int polls, cudaStream_t st) {
  wait_probe_kernel<<<1, 32, 0, st>>>(err, polls);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
