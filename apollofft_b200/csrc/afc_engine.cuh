// afc_engine.cuh -- the shared-memory Stockham engine behind every transform.
//
// One CTA transforms L lanes (independent 1D transforms of length n).  Each
// lane is worked on by P threads (lane-major: tid = l * P + t).  A transform
// is a list of Stockham stages; stage s has radix R and Ns = product of the
// radices before it (the formulation of radix_composite/core.rs:169-183):
//
//   butterfly j in [0, n/R), k = j mod Ns
//   read    x[j + r * n/R]                     r = 0..R-1
//   twiddle x_r *= W_{Ns R}^{r k}               (forward W = exp(-2 pi i / .))
//   R-point DFT
//   write   y[(j - k) * R + k + r * Ns]
//
// Stages ping-pong between two shared buffers per lane (or read global memory
// directly in stage 0 and write it directly in the last stage).  Each thread
// walks its butterflies j = t, t + P, ... one at a time, so only one radix-R
// butterfly is live in registers and one barrier separates stages.  For
// contiguous lanes the direct stage-0 read and last-stage write are coalesced
// (consecutive threads touch consecutive elements); strided lanes and
// operators with index maps (chirps, gathers, twiddles, truncation) are staged
// through shared memory by cooperative copies in the kernels.
//
// Shared index of element i: i + (i >> 4) (one pad element every 16 breaks the
// stride-R bank conflicts of stage outputs).
#pragma once
#include <cstdint>
#include "afc_butterfly.cuh"

namespace afc {

constexpr int kMaxStages = 24;

struct StageDesc {
  int R;
  int Ns;
  int twoff;  // offset (in complex elements) of this stage's twiddles, stored r-major: [(r-1) Ns + k]
};

struct StageList {
  int n;
  int nst;
  StageDesc st[kMaxStages];
};

// Lane q -> base offset (in elements):  c = q % d2, b = (q / d2) % d1, a = q / (d1 d2),
// base = a*s0 + b*s1 + c*s2.  Element i of the lane lives at base + i*es.
// With an offset table (uneven batches): base = off[q / d2] + (q % d2) * s2.
struct LaneMap {
  long long d1, d2;
  long long s0, s1, s2;
  long long es;
  const long long* off;
  __host__ __device__ __forceinline__ long long base(long long q) const {
    if (off) return off[q / d2] + (q % d2) * s2;
    long long c = q % d2;
    long long t = q / d2;
    long long b = t % d1;
    long long a = t / d1;
    return a * s0 + b * s1 + c * s2;
  }
};

__host__ __device__ __forceinline__ int spad(int i) { return i + (i >> 4); }

// Number of shared buffers a stage list needs per lane, given whether the
// input is staged into shared memory and whether the output is staged out.
__host__ __device__ inline int engine_buffers(int nst, bool stage_in, bool stage_out) {
  if (nst == 0) return 1;
  int in_buf = stage_in ? 0 : -1, maxb = stage_in ? 0 : -1;
  for (int i = 0; i < nst; ++i) {
    const bool last = i == nst - 1;
    if (last && !stage_out) break;
    const int ob = in_buf == 0 ? 1 : 0;
    maxb = ob > maxb ? ob : maxb;
    in_buf = ob;
  }
  return maxb + 1 > 0 ? maxb + 1 : 1;
}

// One stage of one lane.  src == nullptr: read global through cx; dst ==
// nullptr: write global through cx.
template <int R, bool INV, class Ctx, class C>
__device__ __forceinline__ void stage(const Ctx& cx, const C* __restrict__ src, C* __restrict__ dst, int n, int Ns,
                                      const C* __restrict__ tw, int t, int P) {
  const int nb = n / R;
  for (int j = t; j < nb; j += P) {
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src ? src[spad(j + r * nb)] : cx.gload(j + r * nb);
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
    for (int r = 0; r < R; ++r) {
      if (dst) dst[spad(o + r * Ns)] = v[r];
      else cx.gstore(o + r * Ns, v[r]);
    }
  }
}

// Runs every stage of `sl` for this thread's lane.  buf0/buf1: the lane's
// shared buffers; stage_in: the input already sits in buf0; stage_out: leave
// the result in shared memory.  Returns the buffer holding the result when
// stage_out (nullptr otherwise).  Ends with a barrier after every stage.
template <bool INV, class Ctx, class C>
__device__ __forceinline__ C* run_stages(const Ctx& cx, const StageList& sl, const C* __restrict__ tw, int t, int P,
                                         C* buf0, C* buf1, bool stage_in, bool stage_out) {
  const int nst = sl.nst;
  C* cur = stage_in ? buf0 : nullptr;
  if (nst == 0) {  // n = 1: a (scaled / converted) copy
    if (t == 0) {
      const C v = cur ? cur[0] : cx.gload(0);
      if (stage_out) buf0[0] = v;
      else cx.gstore(0, v);
    }
    __syncthreads();
    return stage_out ? buf0 : nullptr;
  }
  for (int i = 0; i < nst; ++i) {
    const bool last = i == nst - 1;
    C* nxt = (last && !stage_out) ? nullptr : (cur == buf0 ? buf1 : buf0);
    const StageDesc s = sl.st[i];
    const C* twi = tw + s.twoff;
#define AFC_ST(R) stage<R, INV>(cx, cur, nxt, sl.n, s.Ns, twi, t, P)
    switch (s.R) {
      case 2: AFC_ST(2); break;
      case 3: AFC_ST(3); break;
      case 4: AFC_ST(4); break;
      case 5: AFC_ST(5); break;
      case 6: AFC_ST(6); break;
      case 7: AFC_ST(7); break;
      case 8: AFC_ST(8); break;
      case 9: AFC_ST(9); break;
      case 10: AFC_ST(10); break;
      case 12: AFC_ST(12); break;
      case 14: AFC_ST(14); break;
      case 15: AFC_ST(15); break;
      case 11: AFC_ST(11); break;
      case 13: AFC_ST(13); break;
      case 16: AFC_ST(16); break;
      default: break;
    }
#undef AFC_ST
    __syncthreads();
    cur = nxt;
  }
  return cur;
}

}  // namespace afc
