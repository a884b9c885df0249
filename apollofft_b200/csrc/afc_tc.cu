// afc_tc.cu -- split-precision tensor-core radix-16 stages (tcgen05, sm_100a).
//
// A radix-16 Stockham stage applied to 128 butterflies is one small matrix
// product: D[b][o] = sum_i X[b][i] F[o][i], with X the 128 x 32 real block of
// twiddled inputs (row b = butterfly b: 16 real parts then 16 imaginary parts)
// and F the 32 x 32 real form of the 16-point DFT matrix (rows: 16 real then 16
// imaginary outputs).  X and F are split into hi + lo halves of BF16 or FP16
// (v = hi + lo, lo = v - hi rounded again) and the four products
// Xh Fh + Xh Fl + Xl Fh + Xl Fl accumulate in FP32 in tensor memory: one
// tcgen05.mma (M = 128, N = 32, K = 16) per half-K step, issued by one thread;
// the accumulator row of butterfly b lives in TMEM lane b, so after
// tcgen05.ld each thread holds its butterfly's 16 outputs.  FP16 blocks are
// scaled per butterfly by a power of two so high-dynamic-range rows stay in
// range (the scale is undone exactly after the product).
//
// Operands sit in shared memory in the canonical K-major, no-swizzle layout:
// 8-row x 16-byte core matrices, LBO = 128 B between the two K halves of a
// 16-wide K step, SBO = 512 B between 8-row groups (K = 32 per row group).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include "afc_engine.cuh"
#include "afc_internal.h"

namespace afc {

__device__ __forceinline__ unsigned tc_smem(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(const void* p) {
  const uint64_t addr = (uint64_t)(tc_smem(p) >> 4) & 0x3FFF;
  const uint64_t lbo = (128 >> 4) & 0x3FFF;
  const uint64_t sbo = (512 >> 4) & 0x3FFF;
  return addr | (lbo << 16) | (sbo << 32) | ((uint64_t)1 << 46);  // version 1, base 0, SWIZZLE_NONE
}

// kind::f16 instruction descriptor: D f32, A/B bf16 (fmt 1) or f16 (fmt 0), both K-major, M = 128, N = 32.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(tc_smem(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void tc_mbar_init(unsigned long long* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc_smem(b)) : "memory");
}
__device__ __forceinline__ bool tc_mbar_wait(unsigned long long* b, unsigned parity) {
  for (int i = 0; i < (1 << 21); ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(tc_smem(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// TMEM: 32 columns per CTA, allocated by warp 0.
__device__ __forceinline__ void tmem_alloc32(unsigned* dst_smem) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;\n" ::"r"(tc_smem(dst_smem))
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc32(unsigned taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;\n" ::"r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with K = 32 (16-bit elements).
__device__ __forceinline__ int kmaj_off(int row, int k) {
  return (row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

template <bool FP16> struct Half;
template <> struct Half<false> {
  using H = __nv_bfloat16;
  using H2 = __nv_bfloat162;
  __device__ static H from(float v) { return __float2bfloat16_rn(v); }
  __device__ static float to(H h) { return __bfloat162float(h); }
  __device__ static H2 from2(float a, float b) { return __floats2bfloat162_rn(a, b); }
  __device__ static float2 to2(H2 h) { return __bfloat1622float2(h); }
};
template <> struct Half<true> {
  using H = __half;
  using H2 = __half2;
  __device__ static H from(float v) { return __float2half_rn(v); }
  __device__ static float to(H h) { return __half2float(h); }
  __device__ static H2 from2(float a, float b) { return __floats2half2_rn(a, b); }
  __device__ static float2 to2(H2 h) { return __half22float2(h); }
};

// Writes one row (32 values) as hi and lo halves into two K-major tiles
// (pairs converted together: one conversion per two values and half).
template <bool FP16>
__device__ __forceinline__ void split_row(unsigned char* hi, unsigned char* lo, int row, const float* v) {
  using HH = Half<FP16>;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    alignas(16) typename HH::H2 h4[4], l4[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float x0 = v[c * 8 + 2 * e], x1 = v[c * 8 + 2 * e + 1];
      h4[e] = HH::from2(x0, x1);
      const float2 hf = HH::to2(h4[e]);
      l4[e] = HH::from2(x0 - hf.x, x1 - hf.y);
    }
    *reinterpret_cast<uint4*>(hi + kmaj_off(row, c * 8)) = *reinterpret_cast<const uint4*>(h4);
    *reinterpret_cast<uint4*>(lo + kmaj_off(row, c * 8)) = *reinterpret_cast<const uint4*>(l4);
  }
}

// The real 32 x 32 form of the 16-point DFT (sign -1 forward, +1 inverse), hi/lo split.
template <bool FP16>
__device__ void build_dft16(unsigned char* Fh, unsigned char* Fl, bool inverse) {
  for (int o = threadIdx.x; o < 32; o += blockDim.x) {
    float row[32];
    const int k = o & 15;
    const bool im_out = o >= 16;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      double s, c;
      sincospi((inverse ? 2.0 : -2.0) * (double)((k * m) & 15) / 16.0, &s, &c);
      // out_re = sum c*re - s*im ; out_im = sum s*re + c*im   (w = c + i s)
      row[m] = im_out ? (float)s : (float)c;
      row[16 + m] = im_out ? (float)c : (float)-s;
    }
    split_row<FP16>(Fh, Fl, o, row);
  }
}

// Self test: D = A * B^T for A (128 x 32) and B (32 x 32) f32 inputs, split like the FFT.
template <bool FP16>
__global__ void __launch_bounds__(128) tc_selftest_kernel(const float* A, const float* B, float* D, unsigned* err) {
  __shared__ __align__(1024) unsigned char Ah[8192], Al[8192], Bh[2048], Bl[2048];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ unsigned tslot;
  const int t = threadIdx.x;
  if (t < 32) tmem_alloc32(&tslot);
  if (t == 0) tc_mbar_init(&bar);
  float v[32];
  for (int k = 0; k < 32; ++k) v[k] = A[t * 32 + k];
  split_row<FP16>(Ah, Al, t, v);
  if (t < 32) {
    for (int k = 0; k < 32; ++k) v[k] = B[t * 32 + k];
    split_row<FP16>(Bh, Bl, t, v);
  }
  tc_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned taddr = tslot;
  if (t == 0) {
    const uint32_t id = umma_idesc(FP16 ? 0u : 1u);
    const unsigned char* As[2] = {Ah, Al};
    const unsigned char* Bs[2] = {Bh, Bl};
    int first = 1;
    for (int ai = 0; ai < 2; ++ai)
      for (int bi = 0; bi < 2; ++bi)
        for (int ks = 0; ks < 2; ++ks) {
          tc_mma(taddr, umma_desc(As[ai] + ks * 256), umma_desc(Bs[bi] + ks * 256), id, first ? 0u : 1u);
          first = 0;
        }
    tc_commit(&bar);
  }
  const bool ok = tc_mbar_wait(&bar, 0);
  if (!ok && t == 0) atomicExch(err, 1u);
  tc_fence_after();
  float out[32];
  tmem_ld32(taddr + ((unsigned)((t >> 5) * 32) << 16), out);
  for (int c = 0; c < 32; ++c) D[t * 32 + c] = out[c];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (t < 32) tmem_dealloc32(taddr);
}

// ───────────────────────── tensor-core FFT of 16^s points ─────────────────────────
// Persistent CTAs of 256 threads over tiles of L = 4096 / n lanes, so every
// radix-16 stage has exactly 256 butterflies = two 128-row MMA tiles, one per
// thread.  Lanes arrive by 1D bulk copy (two slots: the next tile's copy flies
// while this one is transformed) and leave by bulk store.  Per stage, in place
// in the slot: each thread gathers its butterfly's 16 inputs and twiddles
// them (FP32), splits them into hi / lo rows of its A tile, one thread issues
// the 2 x 6 MMAs (Xh Fh, Xh Fl, Xl Fh over two K halves per tile; Xl Fl is
// below FP32 rounding and skipped) and commits to an mbarrier, and each thread
// reads its row of the accumulators back from TMEM (warp w: lanes 32 (w mod 4),
// columns 32 (w / 4)) and writes its 16 outputs in Stockham order.

struct TcArgs {
  const float2* in;
  float2* out;
  const float2* tw;   // stage twiddles of the radix-16 plan (r-major, same table as the SIMT plan)
  StageList sl;
  long long lanes, ntiles;
  int L, ld, slot_elems;
  float scale;
  int inverse;
  unsigned* err;
};

__device__ __forceinline__ void tcb_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc_smem(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tcb_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   tc_smem(dst)),
               "l"(src), "r"(bytes), "r"(tc_smem(bar))
               : "memory");
}
__device__ __forceinline__ void tcb_store(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(tc_smem(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void tcb_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void tcb_wait0() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc64(unsigned* dst_smem) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;\n" ::"r"(tc_smem(dst_smem))
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc64(unsigned taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;\n" ::"r"(taddr) : "memory");
}

__device__ __forceinline__ void tc_issue_load(const TcArgs& a, long long tile, float2* slot, unsigned long long* bar) {
  const long long q0 = tile * a.L;
  const long long rem = a.lanes - q0;
  const int here = (int)(rem < a.L ? rem : a.L);
  const unsigned bytes = (unsigned)((long long)here * a.sl.n * sizeof(float2));
  tcb_expect_tx(bar, bytes);
  tcb_load(slot, a.in + q0 * a.sl.n, bytes, bar);
}

// The radix-2/4/8 stage of a power-of-two length that is not 16^s, on the
// CUDA cores in FP32, in place in the slot like the tensor-core stages: the
// tile's 4096 / R butterflies are 16 / R per thread (the whole stage's reads
// finish before the barrier, its writes come after).  Same layouts as the
// tensor-core stages: the first stage reads lane l at n l + i, later stages the
// padded layout ld l + i + i / 16, the last stage writes n l + i.
template <int R>
__device__ __forceinline__ void tc_simt_stage(float2* cur, int n, int ld, int Ns, const float2* __restrict__ tws,
                                              bool first, bool last, bool inverse, float scale, int t) {
  constexpr int PER = 16 / R;
  const int nb = n / R;
  float2 v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int g = t + b * 256, l = g / nb, j = g - l * nb;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = j + r * nb;
      v[b][r] = first ? cur[l * n + i] : cur[l * ld + i + (i >> 4)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int g = t + b * 256, l = g / nb, j = g - l * nb;
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = tws[(r - 1) * Ns + k];
        const float wy = inverse ? -w.y : w.y;
        const float2 x = v[b][r];
        v[b][r] = make_float2(x.x * w.x - x.y * wy, x.x * wy + x.y * w.x);
      }
    }
    if (inverse)
      DFT<R, true>::run(v[b]);
    else
      DFT<R, false>::run(v[b]);
    const int o = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int pos = o + r * Ns;
      if (last)
        cur[l * n + pos] = make_float2(v[b][r].x * scale, v[b][r].y * scale);
      else
        cur[l * ld + pos + (pos >> 4)] = v[b][r];
    }
  }
  __syncthreads();
}

// SMALL: the plan has one radix-2/4/8 stage (lengths that are not 16^s); the
// 16^s build carries no code for it (with it, 16384 x 4096 measured 506 -> 628
// us in BF16 on B200).
// FIXN = 4096: n = 4096 as three radix-16 stages with every shared-memory
// index a compile-time offset from one per-thread base (one lane per tile,
// thread t owns butterfly t of each stage), as in the SIMT 4096-point build.
template <bool FP16, bool SMALL, int FIXN>
__global__ void __launch_bounds__(256, 2) tc_fft_kernel(const __grid_constant__ TcArgs a) {
  // Declared 16-byte aligned on purpose: with separately compiled device code
  // the dynamic block starts at any 16-byte boundary after the static
  // variables (0x410 here), whatever alignment the declaration claims, and a
  // larger claimed alignment lets the compiler fold the padding below to zero.
  // Operand tiles off a 1024-byte boundary read back wrong in the MMA.
  extern __shared__ __align__(16) unsigned char smraw[];
  // layout from the first 1024-byte boundary:
  // A0h 8K | A0l 8K | A1h 8K | A1l 8K | Fh 2K | Fl 2K | slot0 | slot1
  unsigned char* A = smraw + ((1024u - (tc_smem(smraw) & 1023u)) & 1023u);
  unsigned char* Fh = A + 4 * 8192;
  unsigned char* Fl = Fh + 2048;
  float2* slots[2];
  slots[0] = reinterpret_cast<float2*>(Fl + 2048);
  slots[1] = slots[0] + a.slot_elems;
  __shared__ __align__(8) unsigned long long bars[3];  // two slot loads, one MMA completion
  __shared__ unsigned tslot;
  const int t = threadIdx.x;
  long long tile = blockIdx.x;
  if (tile >= a.ntiles) return;  // uniform: before any TMEM allocation
  const int n = a.sl.n, nb = n / 16, ld = a.ld;
  const int l = t / nb, j = t - l * nb;  // lane in the tile, butterfly in the lane (L nb = 256)
  const int mt = t >> 7, row = t & 127;  // MMA tile and row of this butterfly
  unsigned char* Ah = A + mt * 16384;
  unsigned char* Al = Ah + 8192;
  if (t < 32) tmem_alloc64(&tslot);
  if (t == 0) {
    tc_mbar_init(&bars[0]);
    tc_mbar_init(&bars[1]);
    tc_mbar_init(&bars[2]);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  build_dft16<FP16>(Fh, Fl, a.inverse != 0);
  tc_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned taddr = tslot;
  const unsigned trow = taddr + ((unsigned)(((t >> 5) & 3) * 32) << 16) + (unsigned)(32 * mt);
  const uint32_t id = umma_idesc(FP16 ? 0u : 1u);
  if (t == 0) tc_issue_load(a, tile, slots[0], &bars[0]);
  unsigned mphase = 0;
  bool failed = false;
  for (int it = 0; !failed; ++it) {
    const int cb = it & 1;
    const long long nxt = tile + gridDim.x;
    if (t == 0) {
      tcb_wait_read0();  // the previous tile's store has finished reading its slot
      if (nxt < a.ntiles) tc_issue_load(a, nxt, slots[cb ^ 1], &bars[cb ^ 1]);
    }
    const bool okl = tc_mbar_wait(&bars[cb], (unsigned)((it >> 1) & 1));
    if (__syncthreads_or(!okl)) {
      if (t == 0) {
        atomicExch(a.err, 1u);
        if (nxt < a.ntiles) tc_mbar_wait(&bars[cb ^ 1], (unsigned)(((it + 1) >> 1) & 1));
      }
      failed = true;
      break;
    }
    float2* cur = slots[cb];
#pragma unroll
    for (int s = 0; s < (FIXN ? 3 : a.sl.nst); ++s) {
      const int Ns = FIXN ? (s == 0 ? 1 : s == 1 ? 16 : 256) : a.sl.st[s].Ns;
      const float2* tws = a.tw + a.sl.st[s].twoff;
      const bool last = FIXN ? s == 2 : s == a.sl.nst - 1;
      if constexpr (SMALL) {
        if (a.sl.st[s].R != 16) {  // the one radix-2/4/8 stage of a 2^k plan, on the CUDA cores
          const int R = a.sl.st[s].R;
          const bool inv = a.inverse != 0;
          if (R == 8)
            tc_simt_stage<8>(cur, n, ld, Ns, tws, s == 0, last, inv, a.scale, t);
          else if (R == 4)
            tc_simt_stage<4>(cur, n, ld, Ns, tws, s == 0, last, inv, a.scale, t);
          else
            tc_simt_stage<2>(cur, n, ld, Ns, tws, s == 0, last, inv, a.scale, t);
          continue;
        }
      }
      const int k = j % Ns;
      float v[32];
      float sc = 1.0f;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int i = j + r * nb;
        float2 x;
        if constexpr (FIXN == 4096)  // element t + 256 r: linear, or padded at t + t / 16 + 272 r
          x = s == 0 ? cur[t + 256 * r] : cur[t + (t >> 4) + 272 * r];
        else
          x = s == 0 ? cur[l * n + i] : cur[l * ld + i + (i >> 4)];
        if (Ns > 1 && r > 0) {
          const float2 w = tws[(long long)(r - 1) * Ns + k];
          const float wy = a.inverse ? -w.y : w.y;
          x = make_float2(x.x * w.x - x.y * wy, x.x * wy + x.y * w.x);
        }
        v[r] = x.x;
        v[16 + r] = x.y;
      }
      if (FP16) {  // power-of-two row scale: largest magnitude near 2^11
        float m = 0.f;
#pragma unroll
        for (int r = 0; r < 32; ++r) m = fmaxf(m, fabsf(v[r]));
        int e = 0;
        frexpf(m, &e);
        sc = (m > 0.f && m < 3.0e38f) ? ldexpf(1.0f, 11 - e) : 1.0f;
#pragma unroll
        for (int r = 0; r < 32; ++r) v[r] *= sc;
      }
      split_row<FP16>(Ah, Al, row, v);
      tc_proxy_fence();
      tc_fence_before();
      __syncthreads();  // every gather of this stage is done: the slot may be overwritten below
      tc_fence_after();
      if (t == 0) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const unsigned char* qh = A + q * 16384;
          const unsigned char* ql = qh + 8192;
          const uint32_t d = taddr + 32 * q;
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            tc_mma(d, umma_desc(qh + ks * 256), umma_desc(Fh + ks * 256), id, ks);
            tc_mma(d, umma_desc(qh + ks * 256), umma_desc(Fl + ks * 256), id, 1u);
            tc_mma(d, umma_desc(ql + ks * 256), umma_desc(Fh + ks * 256), id, 1u);
          }
        }
        tc_commit(&bars[2]);
      }
      const bool okm = tc_mbar_wait(&bars[2], mphase);
      mphase ^= 1u;
      if (__syncthreads_or(!okm)) {
        if (t == 0) atomicExch(a.err, 1u);
        failed = true;
        break;
      }
      tc_fence_after();
      float o[32];
      tmem_ld32(trow, o);
      const float inv_sc = 1.0f / sc;
      const int ob = (j - k) * 16 + k;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int pos = ob + r * Ns;
        float2 y = make_float2(o[r] * inv_sc, o[16 + r] * inv_sc);
        if constexpr (FIXN == 4096) {
          // outputs 16 t + r (s = 0), 256 (t / 16) + t % 16 + 16 r (s = 1),
          // t + 256 r linear (s = 2)
          if (s == 2) {
            y.x *= a.scale;
            y.y *= a.scale;
            cur[t + 256 * r] = y;
          } else if (s == 1) {
            cur[272 * (t >> 4) + (t & 15) + 17 * r] = y;
          } else {
            cur[17 * t + r] = y;
          }
        } else if (last) {
          y.x *= a.scale;
          y.y *= a.scale;
          cur[l * n + pos] = y;
        } else {
          cur[l * ld + pos + (pos >> 4)] = y;
        }
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
    if (failed) {
      if (t == 0 && nxt < a.ntiles) tc_mbar_wait(&bars[cb ^ 1], (unsigned)(((it + 1) >> 1) & 1));
      break;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      const long long q0 = tile * a.L;
      const long long rem = a.lanes - q0;
      const int here = (int)(rem < a.L ? rem : a.L);
      tcb_store(a.out + q0 * n, cur, (unsigned)((long long)here * n * sizeof(float2)));
    }
    tile = nxt;
    if (tile >= a.ntiles) break;
  }
  if (t == 0) tcb_wait0();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (t < 32) tmem_dealloc64(taddr);
}

cudaError_t launch_tc_selftest(const float* A, const float* B, float* D, unsigned* err, bool fp16, cudaStream_t st) {
  if (fp16) tc_selftest_kernel<true><<<1, 128, 0, st>>>(A, B, D, err);
  else tc_selftest_kernel<false><<<1, 128, 0, st>>>(A, B, D, err);
  count_launch(1);
  return cudaGetLastError();
}

// Tile geometry for n = 2^k, 16 <= n <= 4096: L = 4096 / n lanes (256
// radix-16 butterflies per stage), slots of L x max(ld, n) complex64
// (ld = n + n/16 + 1, odd).
static void tc_geometry(int n, int& L, int& ld, int& slot) {
  L = 4096 / n;
  ld = n + (n - 1) / 16 + 1;
  if ((ld & 1) == 0) ++ld;
  slot = L * (ld > n ? ld : n);
  slot = (slot + 15) / 16 * 16;  // 128-byte aligned second slot
}

size_t tc_fft_smem(int n) {
  int L, ld, slot;
  tc_geometry(n, L, ld, slot);
  return 1024 + 4 * 8192 + 2 * 2048 + 2 * (size_t)slot * sizeof(float2);
}

cudaError_t launch_tc_fft(const TcLaunch& d, bool fp16, cudaStream_t st) {
  if (d.lanes <= 0) return cudaSuccess;
  // bulk copies move whole tiles: both buffers must start on a 16-byte boundary
  if ((reinterpret_cast<uintptr_t>(d.in) | reinterpret_cast<uintptr_t>(d.out)) & 15) return cudaErrorInvalidValue;
  TcArgs a;
  memset(&a, 0, sizeof(a));
  a.in = static_cast<const float2*>(d.in);
  a.out = static_cast<float2*>(d.out);
  a.tw = static_cast<const float2*>(d.tw);
  a.sl = d.sl;
  a.lanes = d.lanes;
  tc_geometry(d.sl.n, a.L, a.ld, a.slot_elems);
  a.ntiles = (d.lanes + a.L - 1) / a.L;
  a.scale = (float)d.scale;
  a.inverse = d.inverse;
  a.err = d.err;
  const size_t smem = tc_fft_smem(d.sl.n);
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  cudaError_t e;
  // CTAs per SM from the kernel's registers and shared memory (the occupancy
  // query reports one CTA for this kernel although two fit)
  cudaFuncAttributes fa;
  bool small = false;
  for (int s2 = 0; s2 < d.sl.nst; ++s2) small = small || d.sl.st[s2].R != 16;
  // n = 4096 on the compile-time build (AFC_TC_FIX=0 keeps the general one)
  static const int fix_env = [] {
    const char* e = getenv("AFC_TC_FIX");
    return e && *e ? atoi(e) : 1;
  }();
  const bool fix = fix_env && !small && d.sl.n == 4096 && d.sl.nst == 3;
  void (*k)(TcArgs) = fp16 ? (fix ? tc_fft_kernel<true, false, 4096>
                                  : small ? tc_fft_kernel<true, true, 0> : tc_fft_kernel<true, false, 0>)
                           : (fix ? tc_fft_kernel<false, false, 4096>
                                  : small ? tc_fft_kernel<false, true, 0> : tc_fft_kernel<false, false, 0>);
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k);
  if (e != cudaSuccess) return e;
  static int smem_sm = 0, smem_rsv = 0;
  if (!smem_sm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (smem_sm <= 0) smem_sm = 228 * 1024;
  }
  const int by_regs = fa.numRegs > 0 ? 65536 / (fa.numRegs * 256) : 1;
  const int by_smem = (int)((size_t)smem_sm / (smem + fa.sharedSizeBytes + (size_t)smem_rsv));
  int per = std::min(by_regs, by_smem);
  if (per < 1) per = 1;
  // every resident CTA holds 64 TMEM columns; 512 columns per SM
  if (per > 8) per = 8;
  long long grid = (long long)sms * per;
  if (grid > a.ntiles) grid = a.ntiles;
  k<<<(unsigned)grid, 256, smem, st>>>(a);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace afc
