// afc_api.cu -- host side of apollofft_b200: integer layer, GPU planner, plan
// cache and the C ABI declared in include/apollofft_cuda.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/apollofft_cuda.h"
#include "afc_internal.h"

namespace afc {

// ───────────────────────────── errors / counters ─────────────────────────────

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};
void count_launch(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }

static afc_status fail(afc_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}
static afc_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return fail(AFC_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(AFC_ERR_DEVICE, "%s: %s", what, cudaGetErrorString(e));
}
#define AFC_CUDA(call, what)                    \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Test hook: fail the next N device allocations with AFC_ERR_OUT_OF_MEMORY.
static std::atomic<int> g_fail_allocs{0};
static cudaError_t dev_alloc(void** p, size_t bytes) {
  if (g_fail_allocs.load() > 0) {
    g_fail_allocs.fetch_sub(1);
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  if (bytes == 0) bytes = 16;
  return cudaMalloc(p, bytes);
}

// ───────────────────────────── integer layer ─────────────────────────────
// The library's own statement of the reference's integer maps; results are
// bit-exact with crates/apollo-fft (tests compare against the oracle and the
// reference's known-answer tests).

using u64 = uint64_t;

static u64 mulmod(u64 a, u64 b, u64 m) { return (u64)((unsigned __int128)a * b % m); }
static u64 powmod(u64 b, u64 e, u64 m) {
  u64 r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = mulmod(r, b, m);
    b = mulmod(b, b, m);
    e >>= 1;
  }
  return r;
}
static std::vector<u64> prime_factors(u64 n) {  // ascending, with multiplicity
  std::vector<u64> f;
  while (n > 0 && n % 2 == 0) { f.push_back(2); n /= 2; }
  for (u64 d = 3; d * d <= n; d += 2)
    while (n % d == 0) { f.push_back(d); n /= d; }
  if (n > 1) f.push_back(n);
  return f;
}
static bool is_prime_u(u64 n) {  // radix_shape.rs:172-190
  if (n <= 1) return false;
  if (n <= 3) return true;
  if (n % 2 == 0 || n % 3 == 0) return false;
  for (u64 i = 5; i * i <= n; i += 6)
    if (n % i == 0 || n % (i + 2) == 0) return false;
  return true;
}
// radix_shape.rs:60-170: odd primes of {3..23} innermost (largest first), 2s outermost;
// None for other primes or pure powers of two.
static bool factorize23(u64 n, std::vector<u64>& out) {
  out.clear();
  if (n <= 1) return true;
  const u64 pr[8] = {23, 17, 13, 11, 7, 5, 3, 2};
  u64 cnt[8] = {0}, m = n;
  for (int i = 7; i >= 0; --i)
    while (m % pr[i] == 0) { m /= pr[i]; cnt[i]++; }
  if (m != 1) return false;
  bool odd = false;
  for (int i = 0; i < 7; ++i) odd |= cnt[i] > 0;
  if (!odd) return false;
  for (int i = 0; i < 8; ++i)
    for (u64 k = 0; k < cnt[i]; ++k) out.push_back(pr[i]);
  return true;
}
static std::vector<u64> lower_pairs(const std::vector<u64>& r) {  // radix_shape.rs:221-234
  std::vector<u64> o;
  for (size_t i = 0; i < r.size();) {
    if (i + 1 < r.size() && r[i] == 2 && r[i + 1] == 2) { o.push_back(4); i += 2; }
    else o.push_back(r[i++]);
  }
  return o;
}
// radix_shape.rs:192-219: n1 = power of the largest prime factor, n2 = rest.
static bool coprime_split(u64 n, u64& n1, u64& n2) {
  auto f = prime_factors(n);
  if (f.empty()) return false;
  std::vector<u64> pp;
  for (size_t i = 0; i < f.size();) {
    u64 p = f[i], pw = 1;
    while (i < f.size() && f[i] == p) { pw *= p; ++i; }
    pp.push_back(pw);
  }
  if (pp.size() < 2) return false;
  n1 = pp.back();
  n2 = n / n1;
  return true;
}
static bool short_winograd(u64 n) {  // mixed_radix/traits.rs:172-176
  if (n >= 2 && n <= 56) return true;
  return n == 58 || n == 60 || n == 62 || n == 63 || n == 64 || n == 81 || n == 128;
}
// good_thomas/mod.rs:29-31 with three_by_prime.rs:1-11 and the fixed.rs:31-45
// generator rule (apollo-fft-macros/src/good_thomas.rs:244-325).
static bool static_coprime_codelet(u64 n1, u64 n2) {
  static const u64 tbp[] = {5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
  if (n2 == 3)
    for (u64 p : tbp) if (p == n1) return true;
  static const u64 ss[] = {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17,
                           18, 19, 23, 24, 25, 27, 29, 31, 32, 36, 37, 41, 43, 47, 53};
  auto in_ss = [&](u64 v) { for (u64 s : ss) if (s == v) return true; return false; };
  const u64 n = n1 * n2;
  if (!in_ss(n1) || !in_ss(n2) || n1 < 2 || n2 < 2 || n > 200 || in_ss(n)) return false;
  u64 a = n1, b = n2;
  while (b) { u64 t = a % b; a = b; b = t; }
  if (a != 1) return false;
  u64 c1, c2;
  if (!coprime_split(n, c1, c2) || c1 != n1 || c2 != n2) return false;
  const u64 lo = std::min(n1, n2), hi = std::max(n1, n2);
  static const u64 dpp[] = {5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
  if (lo == 2 || lo == 3)
    for (u64 p : dpp)
      if (p == hi) return false;
  return true;
}
// rader/generator.rs:18-94: fixed table, then the smallest generator.
static u64 primitive_root_u(u64 p) {
  static const std::pair<u64, u64> tab[] = {
      {2, 1},   {3, 2},   {5, 2},   {7, 3},    {11, 2},  {13, 2},  {17, 3},  {19, 2},
      {23, 5},  {29, 2},  {31, 3},  {37, 2},   {41, 6},  {43, 3},  {47, 5},  {53, 2},
      {59, 2},  {61, 2},  {67, 2},  {71, 7},   {73, 5},  {79, 3},  {83, 2},  {89, 3},
      {97, 5},  {101, 2}, {109, 6}, {113, 3},  {127, 3}, {131, 2}, {151, 6}, {167, 5},
      {173, 2}, {179, 2}, {181, 2}, {193, 5},  {197, 2}, {199, 3}, {10007, 5}};
  for (auto& e : tab) if (e.first == p) return e.second;
  if (p == 2) return 1;
  auto f = prime_factors(p - 1);
  f.erase(std::unique(f.begin(), f.end()), f.end());
  for (u64 g = 2; g < p; ++g) {
    bool ok = true;
    for (u64 q : f) if (powmod(g, (p - 1) / q, p) == 1) { ok = false; break; }
    if (ok) return g;
  }
  return 0;
}
static u64 inv_mod(u64 a, u64 m) {  // rader/generator.rs:96-120 (a in [1, m))
  if (m == 1) return 0;
  int64_t r0 = (int64_t)m, r1 = (int64_t)(a % m), s0 = 0, s1 = 1;
  while (r1 != 0) {
    int64_t q = r0 / r1, t = r0 - q * r1;
    r0 = r1; r1 = t;
    t = s0 - q * s1; s0 = s1; s1 = t;
  }
  if (s0 < 0) s0 += (int64_t)m;
  return (u64)s0;
}
static int strategy_of(u64 n) {  // mixed_radix/dispatch.rs:26-132
  if (n <= 1) return 0;
  if ((n & (n - 1)) == 0 && n >= 64) return (n >= 4096 && (__builtin_ctzll(n) % 2 == 0)) ? 2 : 1;
  if (short_winograd(n)) return 3;
  u64 n1 = 0, n2 = 0;
  bool cop = coprime_split(n, n1, n2);
  if (cop && static_coprime_codelet(n1, n2)) return 4;
  std::vector<u64> r;
  if (factorize23(n, r)) return 5;
  if (cop) return 6;
  if (is_prime_u(n)) return (n - 1 >= 1024) ? 8 : 7;
  return 9;
}

// ───────────────────────────── GPU planning ─────────────────────────────

enum Algo { ALGO_SMEM = 0, ALGO_FOURSTEP = 1, ALGO_RADER = 2, ALGO_BLUESTEIN = 3, ALGO_NOOP = 4 };
static const size_t kSmemMax = 220 * 1024;
static const int64_t kRaderMax = 1024;  // Rader below, Bluestein above (primes)

// Radices the engine executes for n: odd primes <= 13 (innermost, largest
// first, as the reference orders its factors) then the power of two as 16s and
// one 8/4/2.  False when n has another prime factor (Rader / Bluestein).
// GPU stage radices of n.  Pure powers of two: radix 16 stages, then one of
// 8 / 4 / 2.  Lengths with factors 3, 5, 7: the fewest stages over the radices
// 2..16 of the register butterflies (composites 6, 9, 10, 12, 14, 15 are
// nested butterflies), ties broken toward the cheaper butterflies; 11 and 13
// each take a stage.  Non-power-of-two radices come first.
static bool gpu_radices_uncached(int64_t n, std::vector<int>& rad);
static bool gpu_radices(int64_t n, std::vector<int>& rad) {
  // memo: plan building asks for the same lengths many times
  static std::mutex mu;
  static std::map<int64_t, std::pair<bool, std::vector<int>>> memo;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = memo.find(n);
    if (it != memo.end()) {
      rad = it->second.second;
      return it->second.first;
    }
  }
  const bool ok = gpu_radices_uncached(n, rad);
  std::lock_guard<std::mutex> lk(mu);
  memo[n] = std::make_pair(ok, rad);
  return ok;
}

static bool gpu_radices_uncached(int64_t n, std::vector<int>& rad) {
  rad.clear();
  if (n <= 1) return false;
  int64_t m = n;
  int e[6] = {0, 0, 0, 0, 0, 0};  // exponents of 2, 3, 5, 7, 11, 13
  static const int pr[6] = {2, 3, 5, 7, 11, 13};
  for (int i = 0; i < 6; ++i)
    while (m % pr[i] == 0) { m /= pr[i]; ++e[i]; }
  if (m != 1) return false;
  for (int i = 0; i < e[5]; ++i) rad.push_back(13);
  for (int i = 0; i < e[4]; ++i) rad.push_back(11);
  int k = e[0];
  if (e[1] + e[2] + e[3] > 0) {
    // radix -> exponents of (2, 3, 5, 7) and a tie-break penalty
    struct Opt { int r, a, b, c, d, pen; };
    static const Opt opts[] = {{16, 4, 0, 0, 0, 0}, {15, 0, 1, 1, 0, 2}, {14, 1, 0, 0, 1, 3}, {12, 2, 1, 0, 0, 2},
                               {10, 1, 0, 1, 0, 3}, {9, 0, 2, 0, 0, 2},  {8, 3, 0, 0, 0, 1},  {7, 0, 0, 0, 1, 3},
                               {6, 1, 1, 0, 0, 3},  {5, 0, 0, 1, 0, 3},  {4, 2, 0, 0, 0, 2},  {3, 0, 1, 0, 0, 4},
                               {2, 1, 0, 0, 0, 3}};
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> memo;  // state -> (cost, option)
    std::function<int(int, int, int, int)> best = [&](int a, int b, int c, int d) -> int {
      if (a == 0 && b == 0 && c == 0 && d == 0) return 0;
      const auto key = std::make_tuple(a, b, c, d);
      auto it = memo.find(key);
      if (it != memo.end()) return it->second.first;
      int bc = 1 << 30, bo = -1;
      for (int o = 0; o < (int)(sizeof(opts) / sizeof(opts[0])); ++o) {
        const Opt& q = opts[o];
        if (q.a > a || q.b > b || q.c > c || q.d > d) continue;
        const int sub = best(a - q.a, b - q.b, c - q.c, d - q.d);
        if (sub >= (1 << 30)) continue;
        const int cost = sub + 64 + q.pen;  // stages first, then the penalty
        if (cost < bc) { bc = cost; bo = o; }
      }
      memo[key] = std::make_pair(bc, bo);
      return bc;
    };
    best(k, e[1], e[2], e[3]);
    std::vector<int> p2;
    int a = k, b = e[1], c = e[2], d = e[3];
    while (a || b || c || d) {
      const Opt& q = opts[memo[std::make_tuple(a, b, c, d)].second];
      if (q.b || q.c || q.d) rad.push_back(q.r);
      else p2.push_back(q.r);
      a -= q.a; b -= q.b; c -= q.c; d -= q.d;
    }
    std::sort(p2.begin(), p2.end(), std::greater<int>());
    rad.insert(rad.end(), p2.begin(), p2.end());
    return (int)rad.size() <= kMaxStages;
  }
  while (k >= 4) { rad.push_back(16); k -= 4; }
  if (k == 3) rad.push_back(8);
  else if (k == 2) rad.push_back(4);
  else if (k == 1) rad.push_back(2);
  return (int)rad.size() <= kMaxStages;
}

struct LenPlan {
  StageList sl{};
  void* tw = nullptr;
  int P = 0, ld = 0;
  int64_t n = 0;
};

static int ld_for(int64_t n) {
  int64_t ld = n + (n - 1) / 16 + 1;
  if ((ld & 1) == 0) ld += 1;
  return (int)ld;
}

// Threads per lane: one butterfly of the largest radix per thread and stage
// (smaller radices loop), at most 512 threads.
static int choose_threads(int64_t n, const std::vector<int>& rad) {
  int rmax = 2;
  for (int r : rad) rmax = std::max(rmax, r);
  int64_t p = (n + rmax - 1) / rmax;
  return (int)std::max<int64_t>(1, std::min<int64_t>(512, p));
}

// Shared-memory budget of one single-CTA lane; batch plans lower it so that
// every tile of their persistent kernel fits several CTAs per SM.
static thread_local size_t tl_smem_cap = kSmemMax;

// Per-CTA shared memory of persistent batch tiles: three complex64 CTAs per SM
// (the float batch kernel is built for three), two complex128 CTAs.
static size_t batch_smem_cap(bool dbl) {
  static const long kb = [] {
    const char* e = getenv("AFC_BATCH_SMEM_KB");
    return e && *e ? atol(e) : 0L;
  }();
  if (kb > 0) return (size_t)kb * 1024;
  return dbl ? 100 * 1024 : 72 * 1024;
}

// A single-CTA plan needs two shared buffers of ld elements for one lane.
static bool plannable(int64_t n, size_t csz, std::vector<int>* rad_out = nullptr) {
  std::vector<int> rad;
  if (!gpu_radices(n, rad)) return false;
  if (2 * (size_t)ld_for(n) * csz + 64 > tl_smem_cap) return false;
  if (rad_out) *rad_out = rad;
  return true;
}

static afc_status build_lenplan(int64_t n, bool dbl, LenPlan& lp, cudaStream_t st) {
  const size_t csz = dbl ? 16 : 8;
  std::vector<int> rad;
  if (!plannable(n, csz, &rad)) return fail(AFC_ERR_UNSUPPORTED, "length %lld has no shared-memory plan", (long long)n);
  lp.n = n;
  lp.P = choose_threads(n, rad);
  lp.ld = ld_for(n);
  lp.sl.n = (int)n;
  lp.sl.nst = (int)rad.size();
  int Ns = 1, off = 0;
  for (size_t s = 0; s < rad.size(); ++s) {
    lp.sl.st[s].R = rad[s];
    lp.sl.st[s].Ns = Ns;
    lp.sl.st[s].twoff = off;
    if (Ns > 1) off += Ns * (rad[s] - 1);
    Ns *= rad[s];
  }
  AFC_CUDA(dev_alloc(&lp.tw, (size_t)std::max(off, 1) * csz), "twiddle table");
  if (off > 0) AFC_CUDA(gen_stage_twiddles_dev(lp.tw, lp.sl, dbl, st), "twiddle generation");
  return AFC_OK;
}

struct AxisPlan {
  int64_t n = 0;
  int algo = ALGO_NOOP;
  LenPlan lp;                        // SMEM: n; RADER / BLUESTEIN in smem: M
  LenPlan lp1, lp2;                  // FOURSTEP: N1 and N2
  int64_t N1 = 0, N2 = 0, twB = 1;
  void* tw_hi = nullptr;
  void* tw_lo = nullptr;
  int64_t M = 0;                     // convolution length
  bool conv_smem = true;
  void* chirp = nullptr;
  void* spec_f = nullptr;
  void* spec_i = nullptr;
  void* spec_rf = nullptr;           // large Bluestein: spectra in row-major [k1][k2] order
  void* spec_ri = nullptr;
  int* gather = nullptr;
  int* scatter = nullptr;
  std::unique_ptr<AxisPlan> sub;     // four-step plan of length M (large Bluestein)
  int tuned_P = 0, tuned_L = 0;      // autotuned tile shape (batch plans)
  ~AxisPlan() {
    void* ptrs[] = {lp.tw, lp1.tw, lp2.tw, tw_hi, tw_lo, chirp, spec_f, spec_i, spec_rf, spec_ri, gather, scatter};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

static afc_status build_axis(int64_t n, bool dbl, AxisPlan& ap, cudaStream_t st);

// One device word per device that bounded waits in the kernels set on timeout.
static std::mutex g_err_mu;
static std::map<int, unsigned*> g_err_words;
static unsigned* device_err_word() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_err_mu);
  auto it = g_err_words.find(dev);
  if (it != g_err_words.end()) return it->second;
  unsigned* p = nullptr;
  if (cudaMalloc(&p, sizeof(unsigned)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, sizeof(unsigned));
  g_err_words[dev] = p;
  return p;
}

static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v && *v ? atoi(v) : dflt;
}

static afc_status build_fourstep(int64_t n, bool dbl, AxisPlan& ap, cudaStream_t st) {
  const size_t csz = dbl ? 16 : 8;
  // N1 = divisor nearest sqrt(n) with both factors plannable.
  int64_t best = 0;
  double target = std::sqrt((double)n);
  for (int64_t d = 2; d * d <= n * 4 && d < n; ++d) {
    if (n % d) continue;
    if (!plannable(d, csz) || !plannable(n / d, csz)) continue;
    if (best == 0 || std::fabs(std::log((double)d / target)) < std::fabs(std::log((double)best / target))) best = d;
  }
  if (best == 0) return fail(AFC_ERR_UNSUPPORTED, "length %lld has no two-pass split", (long long)n);
  ap.algo = ALGO_FOURSTEP;
  ap.N1 = best;
  ap.N2 = n / best;
  afc_status s = build_lenplan(ap.N1, dbl, ap.lp1, st);
  if (s != AFC_OK) return s;
  s = build_lenplan(ap.N2, dbl, ap.lp2, st);
  if (s != AFC_OK) return s;
  // two-level twiddle W_n^m = W_n^{B (m / B)} W_n^{m mod B}, B a power of two >= sqrt(n)
  // so the kernels split m with a shift and a mask
  int64_t B = 1;
  while (B * B < n) B <<= 1;
  ap.twB = B;
  int64_t nhi = (n + B - 1) / B;
  AFC_CUDA(dev_alloc(&ap.tw_lo, (size_t)B * csz), "four-step twiddles");
  AFC_CUDA(dev_alloc(&ap.tw_hi, (size_t)nhi * csz), "four-step twiddles");
  AFC_CUDA(gen_roots_dev(ap.tw_lo, B, 1, n, dbl, st), "four-step twiddles");
  AFC_CUDA(gen_roots_dev(ap.tw_hi, nhi, B, n, dbl, st), "four-step twiddles");
  return AFC_OK;
}

struct AxisIO {
  const void* in = nullptr;
  void* out = nullptr;
  long long lanes = 0;
  LaneMap im{}, om{};
  int in_op = IN_C, out_op = OUT_C;
  double scale = 1.0;
  long long nlen = 0;    // OUT_TRUNC bins kept
  long long herm_n = 0;  // full length for IN_HERM / OUT_TRUNC pairing
  double pair_w = 1.0;
  // the input rows along the lanes' element stride are Hermitian (the pass
  // after a full-spectrum R2C's real-input pass): a TMA pass may transform
  // half the columns and store the rest as their conjugate mirrors
  bool mirror = false;
  // set when the previous pass stored only the columns this pass reads: the
  // mirrored TMA pass is then the only correct one
  bool need_mirror = false;
  // contiguous real-input lanes: elements stored per lane (0: all)
  long long store_cols = 0;
};

// Lanes per CTA: about 256 threads, at least 8 (f64) / 16 (f32) adjacent lanes
// when a side is staged (full 128-byte rows), shared memory per CTA kept
// moderate so several CTAs share an SM.
static int choose_L(const LenPlan& lp, long long lanes, bool stage_in, bool stage_out, size_t csz,
                    size_t extra_per_lane = 0, int nbuf_override = 0) {
  const int nbuf = nbuf_override ? nbuf_override : engine_buffers(lp.sl.nst, stage_in, stage_out);
  const size_t per_lane = (size_t)nbuf * lp.ld * csz + extra_per_lane + 3 * sizeof(long long);
  int L = std::max(1, 256 / lp.P);
  const bool staged = stage_in || stage_out;
  const int Lmin = staged ? (csz == 16 ? 8 : 16) : 1;
  L = std::max(L, Lmin);
  while (L > 1 && ((size_t)L * lp.P > 512 || (size_t)L * per_lane > kSmemMax)) --L;
  while (L > Lmin && (size_t)L * per_lane > std::min<size_t>(100 * 1024, tl_smem_cap)) --L;
  if ((long long)L > lanes) L = (int)std::max(1LL, lanes);
  return L;
}

// The engine reads/writes global memory directly only for plain complex or
// real data along contiguous lanes; everything else is staged.
static bool plain_in(int op) { return op == IN_C || op == IN_R; }
static bool plain_out(int op) { return op == OUT_C || op == OUT_RE; }

// Tile-kernel configuration: threads per lane P ~ n/16 (each thread walks its
// butterflies), lanes per CTA L (>= 8 complex128 / 16 complex64 lanes when
// strided, so each row is a full 128-byte line), at most 256 threads, three
// L x ld shared buffers kept under ~110 KB when possible (two CTAs per SM).
static bool tile_config(const LenPlan& lp, long long lanes, bool lm, size_t csz, int& L, int& P) {
  const int n = (int)lp.n;
  const size_t per_lane = 3 * (size_t)lp.ld * csz + 4 * sizeof(long long);
  const int Lmin = lm ? (csz == 16 ? 8 : 16) : 1;
  if ((size_t)Lmin * per_lane > kSmemMax) return false;
  P = std::max(1, std::min(256 / Lmin, (n + 15) / 16));
  L = std::max(Lmin, 256 / P);
  while (L > Lmin && ((size_t)L * per_lane > 110 * 1024 || L * P > 256)) L = lm ? L / 2 : L - 1;
  if ((long long)L > lanes && !lm) L = (int)std::max(1LL, lanes);
  return (size_t)L * per_lane <= kSmemMax && L * P <= 256;
}

static void fill_common(LaunchDesc& d, const LenPlan& lp) {
  d.sl = lp.sl;
  d.tw = lp.tw;
  d.P = lp.P;
  d.ld = lp.ld;
}

static cudaError_t exec_axis(const AxisPlan& ap, bool dbl, bool inv, const AxisIO& io, void* ws, cudaStream_t st);


// Launch recorder: while a batch plan is being built, the planning code below
// records its launches (descriptor + kind + direction) instead of issuing
// them; pointers passed in are tagged with a base selector in their top byte
// (1 = batch input, 2 = batch output, 3 = batch workspace) and resolved by the
// persistent kernel at run time.
struct RecLaunch {
  LaunchDesc d;
  int kind;  // 0 lanes, 1 convolution
  bool inv;
};
struct Recorder {
  std::vector<RecLaunch> launches;
  int max_threads = kBatchThreads;
};
static thread_local Recorder* tl_rec = nullptr;

static const uint64_t kTagShift = 56;
static void* tag_ptr(int sel, uint64_t off) { return reinterpret_cast<void*>(((uint64_t)sel << kTagShift) | off); }
static void untag(const void*& p, int& sel) {
  const uint64_t v = reinterpret_cast<uint64_t>(p);
  sel = (int)(v >> kTagShift);
  p = reinterpret_cast<const void*>(v & (((uint64_t)1 << kTagShift) - 1));
}

static void record(LaunchDesc d, int kind, bool inv) {
  const void* in = d.in;
  const void* out = d.out;
  untag(in, d.in_sel);
  untag(out, d.out_sel);
  d.in = in;
  d.out = const_cast<void*>(out);
  const int mt = tl_rec->max_threads;
  while (d.L > 1 && d.L * d.P > mt) d.L = d.L > 1 ? d.L / 2 : 1;
  if (d.L * d.P > mt) d.P = std::max(1, mt / d.L);
  tl_rec->launches.push_back(RecLaunch{d, kind, inv});
}

static cudaError_t do_lanes(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st) {
  if (tl_rec) {
    record(d, 0, inv);
    return cudaSuccess;
  }
  return launch_lanes(d, dbl, inv, st);
}
static cudaError_t do_conv(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st) {
  if (tl_rec) {
    record(d, 1, inv);
    return cudaSuccess;
  }
  return launch_conv(d, dbl, st);
}

// Four-step execution of one axis: pass A (N1-point columns, twiddle) into the
// workspace, pass B (N2-point rows) into the output with the transposed store.
static cudaError_t exec_fourstep(const AxisPlan& ap, bool dbl, bool inv, const AxisIO& io, void* ws,
                                 cudaStream_t st, int in_op_B = IN_C) {
  const size_t csz = dbl ? 16 : 8;
  const long long n = ap.n, N1 = ap.N1, N2 = ap.N2;
  const long long d2 = io.im.d2;
  LaunchDesc a;
  fill_common(a, ap.lp1);
  a.lanes = io.lanes * N2;
  a.im = io.im.off ? LaneMap{1, N2, 0, 0, io.im.es, N2 * io.im.es, io.im.off}
                   : LaneMap{N2, d2, io.im.s0, io.im.es, io.im.s2, N2 * io.im.es, nullptr};
  a.om = LaneMap{N2, d2, d2 * n, 1, n, N2, nullptr};
  a.in = io.in;
  a.out = ws;
  a.in_op = io.in_op;
  a.out_op = OUT_TW;
  a.jmul = N2;
  a.col_div = d2;
  a.col_mod = N2;
  a.twN = n;
  a.twB = ap.twB;
  a.tw_hi = ap.tw_hi;
  a.tw_lo = ap.tw_lo;
  a.tw_conj = inv ? 1 : 0;
  a.stage_in = a.im.es != 1 || !plain_in(a.in_op);
  a.stage_out = true;
  a.L = choose_L(ap.lp1, a.lanes, a.stage_in, a.stage_out, csz);
  cudaError_t e = do_lanes(a, dbl, inv, st);
  if (e != cudaSuccess) return e;
  LaunchDesc b;
  fill_common(b, ap.lp2);
  b.lanes = io.lanes * N1;
  b.im = LaneMap{N1, d2, d2 * n, N2, n, 1, nullptr};
  b.om = io.om.off ? LaneMap{1, N1, 0, 0, io.om.es, N1 * io.om.es, io.om.off}
                   : LaneMap{N1, io.om.d2, io.om.s0, io.om.es, io.om.s2, N1 * io.om.es, nullptr};
  b.in = ws;
  b.out = io.out;
  b.in_op = in_op_B;
  b.out_op = io.out_op;
  b.scale = io.scale;
  b.jmul = N1;
  b.col_div = d2;
  b.col_mod = N1;
  b.nlen = io.nlen;
  b.herm_n = io.herm_n;
  b.pair_w = io.pair_w;
  b.stage_in = false;
  b.stage_out = b.om.es != 1 || !plain_out(b.out_op);
  if (ap.lp2.sl.nst <= 1) b.stage_out = true;
  b.L = choose_L(ap.lp2, b.lanes, b.stage_in, b.stage_out, csz);
  return do_lanes(b, dbl, inv, st);
}

// Columns [0, H) that the Hermitian (mirrored) TMA pass of `io` transforms,
// or 0 when that pass would not take the mirrored TMA path; the same planner
// call as exec_axis makes, so the pass then takes exactly that path.
static long long mirror_cols(const AxisPlan& ap, bool dbl, const AxisIO& io) {
  static const int tma_on = env_int("AFC_TMA", 1), tma_lanes = env_int("AFC_TMA_LANES", 0);
  if (!io.mirror || ap.algo != ALGO_SMEM || tl_rec || !tma_on || io.lanes <= 0) return 0;
  if (io.in_op != IN_C || io.out_op != OUT_C) return 0;
  unsigned* err = device_err_word();
  TmaPlan tp;
  if (!err || !tma_plan(ap.lp.sl, ap.lp.ld, io.lanes, io.im, io.om, io.in, io.out, dbl, tma_lanes, tp, false, false,
                        true))
    return 0;
  return tp.hm_cmax > 0 ? tp.kb * tp.L : 0;
}

static cudaError_t exec_axis(const AxisPlan& ap, bool dbl, bool inv, const AxisIO& io, void* ws, cudaStream_t st) {
  const size_t csz = dbl ? 16 : 8;
  if (io.lanes <= 0) return cudaSuccess;
  switch (ap.algo) {
    case ALGO_SMEM: {
      LaunchDesc d;
      fill_common(d, ap.lp);
      d.lanes = io.lanes;
      d.im = io.im;
      d.om = io.om;
      d.in = io.in;
      d.out = io.out;
      d.in_op = io.in_op;
      d.out_op = io.out_op;
      d.scale = io.scale;
      d.nlen = io.nlen;
      d.herm_n = io.herm_n;
      d.pair_w = io.pair_w;
      const bool rin = io.in_op == IN_R && io.out_op == OUT_C, rout = io.in_op == IN_C && io.out_op == OUT_RE;
      static const int tma_on = env_int("AFC_TMA", 1), tma_lanes = env_int("AFC_TMA_LANES", 0);
      if (!tl_rec && ((io.in_op == IN_C && io.out_op == OUT_C) || rin || rout) && tma_on) {
        TmaPlan tp;
        unsigned* err = device_err_word();
        if (err && tma_plan(ap.lp.sl, ap.lp.ld, io.lanes, io.im, io.om, io.in, io.out, dbl, tma_lanes, tp, rin, rout,
                                io.mirror)) {
          if (io.need_mirror && tp.hm_cmax <= 0) return cudaErrorInvalidValue;
          if (io.store_cols > 0 && io.store_cols < ap.lp.sl.n && tp.mode == 0 && rin &&
              (io.store_cols * (long long)csz) % 16 == 0)
            tp.store_cols = (int)io.store_cols;
          return launch_tma(d, tp, err, dbl, inv, st);
        }
      }
      if (io.need_mirror) return cudaErrorInvalidValue;
      if (!tl_rec && io.in_op == IN_C && plain_out(io.out_op)) {
        const bool lm = io.im.es != 1;
        int L, P;
        if (tile_config(ap.lp, io.lanes, lm, csz, L, P)) {
          d.L = L;
          d.P = P;
          d.lane_minor = lm ? 1 : 0;
          return launch_tile(d, dbl, inv, st);
        }
      }
      d.stage_in = io.im.es != 1 || !plain_in(io.in_op);
      d.stage_out = io.om.es != 1 || !plain_out(io.out_op) || ap.lp.sl.nst <= 1;
      d.L = choose_L(ap.lp, io.lanes, d.stage_in, d.stage_out, csz);
      if (tl_rec && ap.tuned_P > 0) {
        d.P = ap.tuned_P;
        d.L = std::max(1, std::min(d.L, ap.tuned_L));
      }
      return do_lanes(d, dbl, inv, st);
    }
    case ALGO_FOURSTEP:
      return exec_fourstep(ap, dbl, inv, io, ws, st);
    case ALGO_RADER:
    case ALGO_BLUESTEIN: {
      const bool rader = ap.algo == ALGO_RADER;
      const bool real_in = io.in_op == IN_R;
      const bool real_out = io.out_op == OUT_RE;
      if (ap.conv_smem) {
        LaunchDesc d;
        fill_common(d, ap.lp);
        d.lanes = io.lanes;
        d.im = io.im;
        d.om = io.om;
        d.in = io.in;
        d.out = io.out;
        d.scale = io.scale;
        if (rader) {
          d.in_op = real_in ? IN_GATHER_R : IN_GATHER;
          d.out_op = real_out ? OUT_SCATTER_RE : OUT_SCATTER;
          d.nlen = ap.n;
        } else {
          d.in_op = real_in ? IN_CHIRP_R : IN_CHIRP;
          d.out_op = real_out ? OUT_CHIRP_RE : OUT_CHIRP;
          d.nlen = io.out_op == OUT_TRUNC ? io.nlen : ap.n;
        }
        d.spec = inv ? ap.spec_i : ap.spec_f;
        d.chirp = ap.chirp;
        d.chirp_conj = inv ? 1 : 0;
        d.gather = ap.gather;
        d.scatter = ap.scatter;
        d.L = choose_L(ap.lp, io.lanes, true, true, csz, 2 * csz, 2);
        return do_conv(d, dbl, inv, st);
      }
      // Bluestein with a four-step convolution of length M = N1 x N2, three
      // passes over two workspaces (input n = N2 n1 + n2, spectrum k = k1 + N1 k2):
      //   1. columns n2: chirp premultiply, DFT_N1 over n1, twiddle W_M^{n2 k1}
      //      -> w1[k1 N2 + n2];
      //   2. rows k1 (one convolution tile): DFT_N2 over n2, times the
      //      spectrum at k1 + N1 k2, inverse DFT_N2 back over n2, conjugate
      //      twiddle W_M^{-n2 k1} -> w2[k1 N2 + n2];
      //   3. columns n2: inverse DFT_N1 over k1, chirp postmultiply -> output
      //      index N2 n1 + n2 (kept for indices < n).
      // The forward DFT's output stays in the transposed order between the
      // two row transforms, so no transpose pass is needed.
      const AxisPlan& mp = *ap.sub;
      const long long M = ap.M, N1 = mp.N1, N2 = mp.N2, d2 = io.im.d2;
      char* w1 = static_cast<char*>(ws);
      char* w2 = w1 + (size_t)io.lanes * M * csz;
      LaunchDesc a;
      fill_common(a, mp.lp1);
      a.lanes = io.lanes * N2;
      a.im = io.im.off ? LaneMap{1, N2, 0, 0, io.im.es, N2 * io.im.es, io.im.off}
                       : LaneMap{N2, d2, io.im.s0, io.im.es, io.im.s2, N2 * io.im.es, nullptr};
      a.om = LaneMap{N2, d2, d2 * M, 1, M, N2, nullptr};
      a.in = io.in;
      a.out = w1;
      a.in_op = real_in ? IN_CHIRP_R : IN_CHIRP;
      a.out_op = OUT_TW;
      a.jmul = N2;
      a.col_div = d2;
      a.col_mod = N2;
      a.nlen = ap.n;
      a.chirp = ap.chirp;
      a.chirp_conj = inv ? 1 : 0;
      a.twN = M;
      a.twB = mp.twB;
      a.tw_hi = mp.tw_hi;
      a.tw_lo = mp.tw_lo;
      a.stage_in = true;
      a.stage_out = true;
      a.L = choose_L(mp.lp1, a.lanes, a.stage_in, a.stage_out, csz);
      cudaError_t e = do_lanes(a, dbl, false, st);
      if (e != cudaSuccess) return e;
      LaunchDesc b;
      fill_common(b, mp.lp2);
      b.lanes = io.lanes * N1;
      b.im = LaneMap{N1, d2, d2 * M, N2, M, 1, nullptr};
      b.om = b.im;
      b.in = w1;
      b.out = w2;
      b.in_op = IN_C;
      b.out_op = OUT_TW;
      b.tw_conj = 1;
      b.twN = M;
      b.twB = mp.twB;
      b.tw_hi = mp.tw_hi;
      b.tw_lo = mp.tw_lo;
      b.spec = inv ? ap.spec_ri : ap.spec_rf;
      b.spec_ld = N2;
      b.col_div = d2;
      b.col_mod = N1;
      b.L = choose_L(mp.lp2, b.lanes, true, true, csz, 2 * csz + 3 * sizeof(long long), 2);
      e = do_conv(b, dbl, false, st);
      if (e != cudaSuccess) return e;
      LaunchDesc c;
      fill_common(c, mp.lp1);
      c.lanes = io.lanes * N2;
      c.im = LaneMap{N2, d2, d2 * M, 1, M, N2, nullptr};
      c.om = io.om.off ? LaneMap{1, N2, 0, 0, io.om.es, N2 * io.om.es, io.om.off}
                       : LaneMap{N2, io.om.d2, io.om.s0, io.om.es, io.om.s2, N2 * io.om.es, nullptr};
      c.in = w2;
      c.out = io.out;
      c.in_op = IN_C;
      c.out_op = real_out ? OUT_CHIRP_RE : OUT_CHIRP;
      c.scale = io.scale;
      c.jmul = N2;
      c.col_div = d2;
      c.col_mod = N2;
      c.nlen = io.out_op == OUT_TRUNC ? io.nlen : ap.n;
      c.chirp = ap.chirp;
      c.chirp_conj = inv ? 1 : 0;
      c.stage_in = true;
      c.stage_out = true;
      c.L = choose_L(mp.lp1, c.lanes, c.stage_in, c.stage_out, csz);
      return do_lanes(c, dbl, true, st);
    }
    default:
      return cudaSuccess;
  }
}

static size_t axis_ws_bytes(const AxisPlan& ap, long long lanes, size_t csz) {
  if (ap.algo == ALGO_FOURSTEP) return (size_t)lanes * ap.n * csz;
  if (ap.algo == ALGO_BLUESTEIN && !ap.conv_smem) return 2 * (size_t)lanes * ap.M * csz;
  return 0;
}

// FFT of a single length-M table (plan build) through an axis plan.
static afc_status fft_table(const AxisPlan& mp, bool dbl, void* buf, cudaStream_t st) {
  const size_t csz = dbl ? 16 : 8;
  AxisIO io;
  io.in = buf;
  io.out = buf;
  io.lanes = 1;
  io.im = LaneMap{1, 1, mp.n, 0, 0, 1, nullptr};
  io.om = io.im;
  void* ws = nullptr;
  size_t wsb = axis_ws_bytes(mp, 1, csz);
  if (wsb) AFC_CUDA(dev_alloc(&ws, wsb), "table workspace");
  cudaError_t e = exec_axis(mp, dbl, false, io, ws, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (ws) cudaFree(ws);
  if (e != cudaSuccess) return cuda_fail(e, "table FFT");
  return AFC_OK;
}

static int plan_stages_uncached(int64_t m, size_t csz);

// Stages of the GPU plan of length m (one CTA, or the two passes of a
// four-step split plus a weight for its extra global-memory round trip);
// -1 when m has no GPU plan.
static int plan_stages(int64_t m, size_t csz) {
  // memo per (length, element size, shared-memory budget): batch plans ask
  // for hundreds of candidate lengths per prime
  static std::mutex mu;
  static std::map<std::tuple<int64_t, size_t, size_t>, int> memo;
  const auto key = std::make_tuple(m, csz, tl_smem_cap);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
  }
  const int r = plan_stages_uncached(m, csz);
  std::lock_guard<std::mutex> lk(mu);
  memo[key] = r;
  return r;
}

static int plan_stages_uncached(int64_t m, size_t csz) {
  std::vector<int> rad;
  if (!gpu_radices(m, rad)) return -1;
  if (plannable(m, csz)) return (int)rad.size();
  int best = -1;
  for (int64_t d = 2; d * d <= m * 4 && d < m; ++d) {
    if (m % d) continue;
    std::vector<int> r1, r2;
    if (!plannable(d, csz, &r1) || !plannable(m / d, csz, &r2)) continue;
    const int c = (int)(r1.size() + r2.size()) + 2;
    if (best < 0 || c < best) best = c;
  }
  return best;
}

// Convolution length for Rader / Bluestein: the length >= need with the least
// work (length x stages) among the next power of two and the 7-smooth lengths
// below it (Bluestein's convolution is exact for any length >= 2n - 1).
static int64_t conv_length(int64_t need, size_t csz) {
  int64_t p2 = 1;
  while (p2 < need) p2 <<= 1;
  int64_t best = p2;
  static const int mode = env_int("AFC_CONV_LEN", 0);  // 0 cost model, 1 powers of two only
  if (mode == 1) return p2;
  const int s2 = plan_stages(p2, csz);
  double best_cost = s2 > 0 ? (double)p2 * s2 : 1e300;
  for (int64_t a = 1; a < p2; a *= 2)
    for (int64_t b = a; b < p2; b *= 3)
      for (int64_t c = b; c < p2; c *= 5)
        for (int64_t d = c; d < p2; d *= 7) {
          if (d < need) continue;
          const int sd = plan_stages(d, csz);
          if (sd <= 0) continue;
          const double cost = (double)d * sd;
          if (cost < 0.97 * best_cost) {
            best_cost = cost;
            best = d;
          }
        }
  return best;
}

static afc_status build_axis(int64_t n, bool dbl, AxisPlan& ap, cudaStream_t st) {
  const size_t csz = dbl ? 16 : 8;
  ap.n = n;
  if (n <= 1) { ap.algo = ALGO_NOOP; return AFC_OK; }
  std::vector<int> rad;
  if (gpu_radices(n, rad)) {
    if (plannable(n, csz)) { ap.algo = ALGO_SMEM; return build_lenplan(n, dbl, ap.lp, st); }
    return build_fourstep(n, dbl, ap, st);
  }
  if (is_prime_u((u64)n) && n < kRaderMax) {
    // Rader: generator order of the reference (rader/mod.rs:76-122), cyclic
    // convolution of length p-1, exact or zero-padded to a power of two.
    const int64_t L = n - 1;
    int64_t M = L;
    if (!plannable(L, csz)) M = conv_length(2 * L - 1, csz);
    if (!plannable(M, csz))
      return fail(AFC_ERR_UNSUPPORTED, "no Rader plan for %lld", (long long)n);
    ap.algo = ALGO_RADER;
    ap.M = M;
    afc_status s = build_lenplan(M, dbl, ap.lp, st);
    if (s != AFC_OK) return s;
    const u64 g = primitive_root_u((u64)n);
    std::vector<int> gat(L), sca(L);
    u64 v = 1;
    for (int64_t q = 0; q < L; ++q) { gat[q] = (int)v; v = mulmod(v, g, (u64)n); }
    for (int64_t q = 0; q < L; ++q) sca[q] = q == 0 ? gat[0] : gat[L - q];
    AFC_CUDA(dev_alloc((void**)&ap.gather, L * sizeof(int)), "Rader maps");
    AFC_CUDA(dev_alloc((void**)&ap.scatter, L * sizeof(int)), "Rader maps");
    AFC_CUDA(cudaMemcpyAsync(ap.gather, gat.data(), L * sizeof(int), cudaMemcpyHostToDevice, st), "Rader maps");
    AFC_CUDA(cudaMemcpyAsync(ap.scatter, sca.data(), L * sizeof(int), cudaMemcpyHostToDevice, st), "Rader maps");
    AFC_CUDA(dev_alloc(&ap.spec_f, (size_t)M * csz), "Rader spectrum");
    AFC_CUDA(dev_alloc(&ap.spec_i, (size_t)M * csz), "Rader spectrum");
    AFC_CUDA(gen_rader_b_dev(ap.spec_f, ap.scatter, n, M, false, dbl, st), "Rader kernel");
    AFC_CUDA(gen_rader_b_dev(ap.spec_i, ap.scatter, n, M, true, dbl, st), "Rader kernel");
    AxisPlan mp;
    mp.n = M;
    mp.algo = ALGO_SMEM;
    mp.lp = ap.lp;
    s = fft_table(mp, dbl, ap.spec_f, st);
    if (s == AFC_OK) s = fft_table(mp, dbl, ap.spec_i, st);
    mp.lp.tw = nullptr;  // owned by ap
    return s;
  }
  // Bluestein chirp-z with a convolution of length M >= 2n-1.
  const int64_t M = conv_length(2 * n - 1, csz);
  ap.algo = ALGO_BLUESTEIN;
  ap.M = M;
  AFC_CUDA(dev_alloc(&ap.chirp, (size_t)n * csz), "chirp");
  AFC_CUDA(gen_chirp_dev(ap.chirp, n, dbl, st), "chirp");
  AFC_CUDA(dev_alloc(&ap.spec_f, (size_t)M * csz), "Bluestein spectrum");
  AFC_CUDA(dev_alloc(&ap.spec_i, (size_t)M * csz), "Bluestein spectrum");
  AFC_CUDA(gen_bluestein_b_dev(ap.spec_f, ap.chirp, n, M, false, dbl, st), "Bluestein kernel");
  AFC_CUDA(gen_bluestein_b_dev(ap.spec_i, ap.chirp, n, M, true, dbl, st), "Bluestein kernel");
  afc_status s;
  if (plannable(M, csz)) {
    ap.conv_smem = true;
    s = build_lenplan(M, dbl, ap.lp, st);
    if (s != AFC_OK) return s;
    AxisPlan mp;
    mp.n = M;
    mp.algo = ALGO_SMEM;
    mp.lp = ap.lp;
    s = fft_table(mp, dbl, ap.spec_f, st);
    if (s == AFC_OK) s = fft_table(mp, dbl, ap.spec_i, st);
    mp.lp.tw = nullptr;
    return s;
  }
  ap.conv_smem = false;
  ap.sub.reset(new AxisPlan());
  ap.sub->n = M;
  s = build_fourstep(M, dbl, *ap.sub, st);
  if (s != AFC_OK) return s;
  s = fft_table(*ap.sub, dbl, ap.spec_f, st);
  if (s == AFC_OK) s = fft_table(*ap.sub, dbl, ap.spec_i, st);
  if (s != AFC_OK) return s;
  // the fused middle pass reads each row k1 of the spectrum contiguously
  AFC_CUDA(dev_alloc(&ap.spec_rf, (size_t)M * csz), "Bluestein spectrum");
  AFC_CUDA(dev_alloc(&ap.spec_ri, (size_t)M * csz), "Bluestein spectrum");
  AFC_CUDA(gen_row_spectrum_dev(ap.spec_rf, ap.spec_f, ap.sub->N1, ap.sub->N2, dbl, st), "Bluestein spectrum");
  AFC_CUDA(gen_row_spectrum_dev(ap.spec_ri, ap.spec_i, ap.sub->N1, ap.sub->N2, dbl, st), "Bluestein spectrum");
  return AFC_OK;
}

// ───────────────────────────── plans ─────────────────────────────

struct PlanKey {
  int rank;
  int64_t d[3];
  int prec, kind;
  int64_t batch;
  int device;
  bool operator<(const PlanKey& o) const {
    return std::tie(rank, d[0], d[1], d[2], prec, kind, batch, device) <
           std::tie(o.rank, o.d[0], o.d[1], o.d[2], o.prec, o.kind, o.batch, o.device);
  }
};

// ─────────────────── ordering of plan-owned device buffers ───────────────────
// Plan-owned scratch (execution workspaces, NUFFT grids, batch workspaces) is
// reused by every call on the plan.  The reference's plans are shared across
// threads (Arc, Send + Sync; apollo-stft runs Rayon over one FftPlan1D,
// stft/dimension_1d.rs:225-239), so a call on one stream must not touch such a
// buffer while a call on another stream still does.  A Fence is an event
// recorded on the stream of the buffer's last use; the next user's stream waits
// for it on the GPU, so no host thread blocks.  Inside a stream capture the
// fence is skipped (an event recorded outside a capture cannot be waited on in
// it): replays of a captured graph are ordered with other calls on the plan by
// the caller.

static bool stream_capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs != cudaStreamCaptureStatusNone;
}

struct Fence {
  cudaEvent_t ev = nullptr;
  bool used = false;
  cudaError_t before(cudaStream_t st, bool cap) const {
    if (cap || !used) return cudaSuccess;
    return cudaStreamWaitEvent(st, ev, 0);
  }
  cudaError_t after(cudaStream_t st, bool cap) {
    if (cap) return cudaSuccess;
    if (!ev) {
      cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    used = true;
    return cudaEventRecord(ev, st);
  }
  Fence() = default;
  Fence(const Fence&) = delete;
  Fence& operator=(const Fence&) = delete;
  ~Fence() {
    if (ev) cudaEventDestroy(ev);
  }
};

// One execution workspace, bound to the stream that last used it.
struct WsSlot {
  cudaStream_t st = nullptr;
  void* ptr = nullptr;
  Fence fence;
  uint64_t last = 0;
  ~WsSlot() {
    if (ptr) cudaFree(ptr);
  }
};

// Device staging of one afc_execute_host call in flight: its own stream (and
// through it its own workspace) and input / output buffers.
struct HostStage {
  cudaStream_t st = nullptr;
  void* in = nullptr;
  void* out = nullptr;
  bool busy = false;
  ~HostStage() {
    if (in) cudaFree(in);
    if (out) cudaFree(out);
    if (st) cudaStreamDestroy(st);
  }
};

// Workspaces per plan: concurrent streams get their own up to this count, then
// take turns on the least recently used one (ordered by its fence).
static const size_t kWsSlots = 4;
// afc_execute_host calls of one plan in flight at once; more callers wait.
static const size_t kHostStages = 4;

}  // namespace afc

struct afc_plan_s {
  int rank = 0;
  int64_t dims[3] = {1, 1, 1};
  afc_precision prec = AFC_PREC_F64;
  afc_kind kind = AFC_KIND_C2C;
  int64_t batch = 1;
  int device = 0;
  bool dbl = true;
  int tc = 0;  // 1 BF16 split, 2 FP16 split tensor-core stages
  std::unique_ptr<afc::AxisPlan> axes[3];
  std::atomic<int> refs{1};
  bool cached = false;
  afc::PlanKey key{};
  // execution workspaces, one per stream in use (at most afc::kWsSlots)
  std::mutex ws_mu;
  std::vector<std::unique_ptr<afc::WsSlot>> ws_slots;
  uint64_t ws_tick = 0;
  size_t ws_bytes = 0;
  // staging of afc_execute_host calls in flight (at most afc::kHostStages)
  std::mutex host_mu;
  std::condition_variable host_cv;
  std::vector<std::unique_ptr<afc::HostStage>> stages;
  int64_t N() const { return dims[0] * dims[1] * dims[2]; }
};

// 1D NUFFT plan (apollo-nufft NufftPlan1D, transform/dimension_1d.rs:101-154):
// n uniform bins on a periodic domain of length n dx, oversampled grid
// m = sigma n, Kaiser-Bessel kernel of half width w, beta = pi (1 - 1/(2 sigma)) 2w.
struct afc_nufft_plan_s {
  int64_t n = 0, m = 0;
  int w = 0;
  double dx = 0, beta = 0, i0b = 1;
  int device = 0;
  afc_plan fft = nullptr;          // C2C f64 plan of length m
  double* deconv = nullptr;        // 1 / kb_ft(k_signed / m), k < n
  void* grid = nullptr;            // plan-owned oversampled grid (m complex128)
  std::mutex mu;                   // one caller enqueues on the grid at a time
  afc::Fence fence;                // the grid's last use on the GPU
  ~afc_nufft_plan_s();
};

// 3D NUFFT plan (apollo-nufft NufftPlan3D, transform/dimension_3d.rs:193-230):
// per axis m = next_pow2(max(sigma n, 2w + 1)), one C2C f64 plan of
// (mx, my, mz) over the plan-owned grid, deconvolution factors per axis.
struct afc_nufft3d_plan_s {
  int64_t n[3] = {0, 0, 0}, m[3] = {0, 0, 0};
  double d[3] = {0, 0, 0};
  int w = 0;
  double beta = 0, i0b = 1;
  int device = 0;
  afc_plan fft = nullptr;
  double* deconv = nullptr;  // nx + ny + nz factors, axis after axis
  void* grid = nullptr;      // mx my mz complex128, C order
  afc::NuTileLaunch tiles;   // B = 0: per-point kernels
  int64_t pts_cap = 0;       // points the tile / rank / index buffers hold
  std::mutex mu;             // one caller enqueues on the grid at a time
  afc::Fence fence;          // the grid's (and tile buffers') last use on the GPU
  ~afc_nufft3d_plan_s();
};

// Chirp z-transform plan (apollo-czt CztPlan, plan/czt/dimension_1d.rs:60-120):
// input length n, output length m, X_k = sum_j x_j A^-j W^(j k) by Bluestein's
// identity over a convolution of length L = next_pow2(n + m - 1).
struct afc_czt_plan_s {
  int64_t n = 0, m = 0, L = 0;
  bool dbl = true;
  int device = 0;
  afc::LenPlan lp;                 // the length-L convolution in one CTA (when it fits)
  std::unique_ptr<afc::AxisPlan> big;  // else the multi-pass plan of length L
  void* chirp_n = nullptr;         // A^-j W^(j^2/2), j < n
  void* chirp_k = nullptr;         // W^(k^2/2), k < m
  void* spec = nullptr;            // FFT of the chirp kernel, scaled by 1/L
  // square plans: the inverse's Vandermonde nodes W^k and A^k (complex128),
  // and whether the nodes are distinct enough to invert
  void* nodes = nullptr;
  void* apow = nullptr;
  bool invertible = false;
  ~afc_czt_plan_s() {
    void* ptrs[] = {lp.tw, chirp_n, chirp_k, spec, nodes, apow};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

// Analytic-signal plan (apollo-hilbert HilbertPlan, application/execution/plan/
// hilbert.rs:21-75, over analytic_signal_into, infrastructure/kernel/direct.rs:
// 85-106): forward FFT of the real signal, the analytic mask, inverse FFT, all
// in one convolution tile per lane.
struct afc_hilbert_plan_s {
  int64_t n = 0;
  bool dbl = true;
  int device = 0;
  afc::LenPlan lp;        // the length-n transform in one CTA (n >= 2)
  void* mask = nullptr;   // mask(k) / n as complex: 1 at DC (and n/2 for even n), 2 below (n+1)/2, 0 above
  ~afc_hilbert_plan_s() {
    void* ptrs[] = {lp.tw, mask};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

namespace afc {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

static int64_t last_len(const afc_plan_s& p) { return p.dims[p.rank - 1]; }
static int64_t half_len(const afc_plan_s& p) { return last_len(p) / 2 + 1; }

// Element counts of the arrays one execution touches.
static void io_elems(const afc_plan_s& p, bool inv, int64_t& in_e, int64_t& out_e) {
  const int64_t N = p.N() * p.batch;
  const int64_t Nh = N / last_len(p) * half_len(p);
  switch (p.kind) {
    case AFC_KIND_C2C: in_e = out_e = N; break;
    case AFC_KIND_R2C_FULL: in_e = out_e = N; break;
    case AFC_KIND_R2C_HALF:
      in_e = inv ? Nh : N;
      out_e = inv ? N : Nh;
      break;
  }
}

// Lane map of axis a in the (batch, d0..d_{r-1}) array whose last dim is `last`.
static LaneMap axis_map(const afc_plan_s& p, int a, int64_t last, long long& lanes) {
  int64_t shp[3] = {p.dims[0], p.dims[1], p.dims[2]};
  shp[p.rank - 1] = last;
  int64_t es = 1;
  for (int b = a + 1; b < p.rank; ++b) es *= shp[b];
  int64_t total = p.batch;
  for (int b = 0; b < p.rank; ++b) total *= shp[b];
  lanes = total / shp[a];
  if (es == 1) return LaneMap{1, 1, shp[a], 0, 0, 1, nullptr};
  return LaneMap{1, es, shp[a] * es, 0, 1, es, nullptr};
}

// x-planes of the plane-by-plane pass pair (the last two axes of a C2C or
// full-spectrum real plan of rank >= 2, each in one CTA per lane), 0 when the
// plan has no such pair.  Planes are the batch times the leading axis (rank 3)
// or the batch (rank 2).
static long long pair_planes(const afc_plan_s& p) {
  if ((p.kind != AFC_KIND_C2C && p.kind != AFC_KIND_R2C_FULL) || p.rank < 2 || p.tc) return 0;
  const AxisPlan& a = *p.axes[p.rank - 1];
  const AxisPlan& b = *p.axes[p.rank - 2];
  if (a.algo != ALGO_SMEM || b.algo != ALGO_SMEM) return 0;
  return p.batch * (p.rank == 3 ? p.dims[0] : 1);
}

static size_t axes_ws_bytes(const afc_plan_s& p) {
  const size_t csz = p.dbl ? 16 : 8;
  size_t need = 0;
  for (int a = 0; a < p.rank; ++a) {
    long long lanes;
    int64_t last = (p.kind == AFC_KIND_R2C_HALF && a != p.rank - 1) ? half_len(p) : last_len(p);
    axis_map(p, a, last, lanes);
    need = std::max(need, axis_ws_bytes(*p.axes[a], lanes, csz));
  }
  return (need + 255) / 256 * 256;
}

// Workspace layout: [complex intermediate of the C2R forms][axis passes][pair counters].
static size_t plan_ws_bytes(const afc_plan_s& p) {
  const size_t csz = p.dbl ? 16 : 8;
  // C2R forms keep their complex intermediate in the workspace.
  size_t inter = 0;
  if (p.rank > 1 && p.kind == AFC_KIND_R2C_FULL) inter = (size_t)p.N() * p.batch * csz;
  if (p.rank > 1 && p.kind == AFC_KIND_R2C_HALF) inter = (size_t)(p.N() / last_len(p) * half_len(p)) * p.batch * csz;
  inter = (inter + 255) / 256 * 256;
  return inter + axes_ws_bytes(p);
}

// The two plane-local passes (axes a0 then a1, with the buffers and
// operators run_plan chose for them) as one pair launch; false when the TMA
// kernels cannot take them (the caller then runs the passes one by one).
static bool try_pair(const afc_plan_s& p, int a0, int a1, const AxisIO& io0, const AxisIO& io1, bool inv,
                     cudaStream_t st, cudaError_t& e) {
  const long long planes = pair_planes(p);
  if (!planes || tl_rec) return false;
  LaunchDesc d[2];
  const int ax[2] = {a0, a1};
  const AxisIO* io[2] = {&io0, &io1};
  for (int k = 0; k < 2; ++k) {
    const AxisPlan& ap = *p.axes[ax[k]];
    fill_common(d[k], ap.lp);
    d[k].im = io[k]->im;
    d[k].om = io[k]->om;
    d[k].lanes = io[k]->lanes;
    d[k].in = io[k]->in;
    d[k].out = io[k]->out;
    d[k].in_op = io[k]->in_op;
    d[k].out_op = io[k]->out_op;
    d[k].scale = io[k]->scale;
  }
  // one x-plane of the intermediate (complex), for the L2 budget of the lag
  const long long plane_bytes = (long long)(p.axes[a0]->n * p.axes[a1]->n) * (p.dbl ? 16 : 8);
  TmaPairPlan pp;
  if (!tma_pair_plan(d[0], d[1], planes, plane_bytes, p.dbl, inv, pp)) return false;
  unsigned* err = device_err_word();
  if (!err) return false;
  e = launch_tma_pair(d[0], d[1], pp, err, p.dbl, inv, st);
  return true;
}

// The two plane-local passes as one launch of the cluster plane kernel when
// both axes have 256 points (radix 16 x 16) and the passes are plain complex
// lanes: rows (the last axis) then columns, whichever order run_plan chose
// (the two orders differ by rounding only).  Reads the first pass's input,
// writes the second pass's output; false when the kernel cannot take them.
static bool try_plane(const afc_plan_s& p, const AxisIO& io0, const AxisIO& io1, bool inv, cudaStream_t st,
                      cudaError_t& e) {
  if (p.kind != AFC_KIND_C2C || p.rank < 2 || p.tc || tl_rec) return false;
  const AxisPlan& az = *p.axes[p.rank - 1];
  const AxisPlan& ay = *p.axes[p.rank - 2];
  for (const AxisPlan* ap : {&az, &ay}) {
    const StageList& sl = ap->lp.sl;
    if (ap->algo != ALGO_SMEM || ap->n != 256 || sl.nst != 2 || sl.st[0].R != 16 || sl.st[1].R != 16 ||
        sl.st[0].Ns != 1 || sl.st[1].Ns != 16 || !ap->lp.tw)
      return false;
  }
  for (const AxisIO* io : {&io0, &io1})
    if (io->in_op != IN_C || io->out_op != OUT_C) return false;
  // the second pass transforms the first pass's output in place
  if (io1.in != io0.out || io1.out != io0.out) return false;
  const long long planes = p.batch * (p.rank == 3 ? p.dims[0] : 1);
  PlanePlan pp;
  if (!plane_plan(planes, p.dbl, inv, io0.in, io1.out, pp)) return false;
  unsigned* err = device_err_word();
  if (!err) return false;
  const size_t csz = p.dbl ? 16 : 8;
  const char* twz = static_cast<const char*>(az.lp.tw) + (size_t)az.lp.sl.st[1].twoff * csz;
  const char* twy = static_cast<const char*>(ay.lp.tw) + (size_t)ay.lp.sl.st[1].twoff * csz;
  e = launch_plane(pp, io0.in, io1.out, twz, twy, io0.scale * io1.scale, err, p.dbl, inv, st);
  return true;
}

// Runs one transform of the plan.  scale is applied on the last pass;
// pair_w is the Hermitian weight used by the R2C_HALF adjoints.
static cudaError_t run_plan(const afc_plan_s& p, const void* in, void* out, bool inv, double scale, double pair_w,
                            void* ws, cudaStream_t st) {
  const size_t csz = p.dbl ? 16 : 8;
  const int r = p.rank;
  const int64_t n_last = last_len(p), h = half_len(p);
  size_t inter_b = 0;
  if (r > 1 && p.kind == AFC_KIND_R2C_FULL) inter_b = (size_t)p.N() * p.batch * csz;
  if (r > 1 && p.kind == AFC_KIND_R2C_HALF) inter_b = (size_t)(p.N() / n_last * h) * p.batch * csz;
  inter_b = (inter_b + 255) / 256 * 256;
  void* inter = ws;
  void* axis_ws = static_cast<char*>(ws) + inter_b;

  // Pass order: forward last axis first (plan/fft/dimension_3d.rs:148-157,
  // dimension_2d.rs forward rows then columns); inverse first axis first.
  std::vector<int> order;
  if (!inv) for (int a = r - 1; a >= 0; --a) order.push_back(a);
  else for (int a = 0; a < r; ++a) order.push_back(a);
  const void* src = in;
  void* dst = out;
  // Each pass's buffers, lane maps and load / store operators.
  std::vector<AxisIO> ios(order.size());
  for (size_t k = 0; k < order.size(); ++k) {
    const int a = order[k];
    const bool first = k == 0;
    const bool lastpass = k + 1 == order.size();
    AxisIO& io = ios[k];
    io.scale = lastpass ? scale : 1.0;
    io.pair_w = 1.0;
    long long lanes = 0;
    if (p.kind == AFC_KIND_C2C) {
      io.im = io.om = axis_map(p, a, n_last, lanes);
      io.in = first ? src : dst;
      io.out = dst;
    } else if (p.kind == AFC_KIND_R2C_FULL) {
      io.im = io.om = axis_map(p, a, n_last, lanes);
      if (!inv) {
        io.in = first ? src : dst;
        io.out = dst;
        if (first) io.in_op = IN_R;
        // the second pass's input rows (along the last axis) are the spectra
        // of real rows; AFC_R2C_MIRROR=0 transforms every column
        if (k == 1) {
          const char* m_env = getenv("AFC_R2C_MIRROR");
          io.mirror = !(m_env && *m_env && atoi(m_env) == 0);
        }
      } else {
        void* cbuf = (r > 1) ? inter : nullptr;
        io.in = first ? src : cbuf;
        io.out = lastpass ? dst : cbuf;
        if (lastpass) io.out_op = OUT_RE;
      }
    } else {  // R2C_HALF
      if (!inv) {
        if (first) {  // a == r-1: real rows of n -> half rows of h
          long long l2;
          io.im = axis_map(p, a, n_last, lanes);
          io.om = axis_map(p, a, h, l2);
          io.in = src;
          io.out = dst;
          io.in_op = IN_R;
          io.out_op = OUT_TRUNC;
          io.nlen = h;
          io.herm_n = n_last;
          io.pair_w = pair_w;
        } else {
          io.im = io.om = axis_map(p, a, h, lanes);
          io.in = dst;
          io.out = dst;
        }
      } else {
        if (!lastpass) {  // leading axes on the half array, into the intermediate
          io.im = io.om = axis_map(p, a, h, lanes);
          io.in = first ? src : inter;
          io.out = inter;
        } else {  // a == r-1: half rows -> real rows
          long long l2;
          io.im = axis_map(p, a, h, lanes);
          io.om = axis_map(p, a, n_last, l2);
          io.in = (r > 1) ? inter : src;
          io.out = dst;
          io.in_op = IN_HERM;
          io.out_op = OUT_RE;
          io.herm_n = n_last;
          io.pair_w = pair_w;
        }
      }
    }
    io.lanes = lanes;
  }
  for (size_t k = 0; k < order.size(); ++k) {
    const int a = order[k];
    const AxisPlan& ap = *p.axes[a];
    const AxisIO& io = ios[k];
    // the last two axes run plane by plane in one launch (z then y forward,
    // y then z inverse) when both fit the TMA kernels
    if (k + 1 < order.size() && a >= r - 2 && order[k + 1] >= r - 2) {
      cudaError_t pe = cudaSuccess;
      if (try_plane(p, io, ios[k + 1], inv, st, pe) || try_pair(p, a, order[k + 1], io, ios[k + 1], inv, st, pe)) {
        if (pe != cudaSuccess) return pe;
        ++k;
        continue;
      }
    }
    // A length-1 axis is the identity, but it may still have to move or convert data.
    if (ap.algo == ALGO_NOOP) {
      AxisPlan one;
      one.n = 1;
      if (io.in == io.out && io.in_op == IN_C && io.out_op == OUT_C && io.scale == 1.0) {
        continue;
      }
      // route through a radix-free copy: a length-1 "transform" is a scaled copy
      LaunchDesc d;
      d.sl.n = 1;
      d.sl.nst = 0;
      d.P = 1;
      d.ld = 3;
      d.lanes = io.lanes;
      d.im = io.im;
      d.om = io.om;
      d.in = io.in;
      d.out = io.out;
      d.in_op = io.in_op;
      d.out_op = io.out_op;
      d.scale = io.scale;
      d.nlen = io.nlen ? io.nlen : 1;
      d.herm_n = io.herm_n ? io.herm_n : 1;
      d.pair_w = io.pair_w;
      d.stage_in = d.stage_out = true;
      d.L = (int)std::min<long long>(256, std::max(1LL, io.lanes));
      cudaError_t e = launch_lanes(d, p.dbl, inv, st);
      if (e != cudaSuccess) return e;
      continue;
    }
    // full-spectrum R2C forward: when the next pass transforms only the
    // columns [0, H) and mirrors the rest, the real-row pass stores only
    // those columns (AFC_R2C_TRUNC=0 stores whole rows)
    AxisIO io0 = io;
    if (k == 0 && order.size() > 1 && ios[1].mirror) {
      const char* t_env = getenv("AFC_R2C_TRUNC");
      const long long H = mirror_cols(*p.axes[order[1]], p.dbl, ios[1]);
      if (H > 0) {
        ios[1].need_mirror = true;
        if (!(t_env && *t_env && atoi(t_env) == 0)) io0.store_cols = H;
      }
    }
    cudaError_t e = exec_axis(ap, p.dbl, inv, io0, axis_ws, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static std::mutex g_cache_mu;
static std::map<PlanKey, afc_plan_s*> g_cache;

static afc_status create_plan(afc_plan* out, int rank, const int64_t* dims, afc_precision prec, afc_kind kind,
                              int64_t batch, int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  if (rank < 1 || rank > 3) return fail(AFC_ERR_VALIDATION, "validation failed for `rank`: `%d` violates `1..=3`", rank);
  if (!dims) return fail(AFC_ERR_VALIDATION, "validation failed for `dims`: `null` violates `must be non-null`");
  static const char* names[3][3] = {{"n", "", ""}, {"nx", "ny", ""}, {"nx", "ny", "nz"}};
  for (int a = 0; a < rank; ++a)
    if (dims[a] <= 0)
      return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%lld` violates `must be > 0`", names[rank - 1][a],
                  (long long)dims[a]);
  if (batch < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `batch`: `%lld` violates `must be > 0`", (long long)batch);
  if (prec != AFC_PREC_F32 && prec != AFC_PREC_F64 && prec != AFC_PREC_TC_BF16_SPLIT && prec != AFC_PREC_TC_FP16_SPLIT)
    return fail(AFC_ERR_VALIDATION, "validation failed for `precision`: `%d` violates `F32|F64|TC_BF16_SPLIT|TC_FP16_SPLIT`", (int)prec);
  const bool tcp = prec == AFC_PREC_TC_BF16_SPLIT || prec == AFC_PREC_TC_FP16_SPLIT;
  if (tcp) {
    const int64_t n = dims[0];
    const bool pow2 = rank == 1 && kind == AFC_KIND_C2C && n >= 16 && (n & (n - 1)) == 0;
    if (!pow2 || n > 4096)
      return fail(AFC_ERR_UNSUPPORTED,
                  "tensor-core plans are rank-1 C2C with n = 2^k, 16 <= n <= 4096 (radix-16 stages on the tensor "
                  "cores, one radix-2/4/8 stage on the CUDA cores); got rank %d, n %lld",
                  rank, (long long)n);
  }
  if (kind != AFC_KIND_C2C && kind != AFC_KIND_R2C_FULL && kind != AFC_KIND_R2C_HALF)
    return fail(AFC_ERR_VALIDATION, "validation failed for `kind`: `%d` violates `C2C|R2C_FULL|R2C_HALF`", (int)kind);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(AFC_ERR_BACKEND_UNAVAILABLE, "backend unavailable: cuda (no device)");
  if (device < 0 || device >= ndev)
    return fail(AFC_ERR_VALIDATION, "validation failed for `device`: `%d` violates `< %d`", device, ndev);
  DeviceGuard g(device);
  std::unique_ptr<afc_plan_s> p(new afc_plan_s());
  p->rank = rank;
  for (int a = 0; a < rank; ++a) p->dims[a] = dims[a];
  p->prec = prec;
  p->kind = kind;
  p->batch = batch;
  p->device = device;
  p->dbl = prec == AFC_PREC_F64;
  p->tc = prec == AFC_PREC_TC_BF16_SPLIT ? 1 : (prec == AFC_PREC_TC_FP16_SPLIT ? 2 : 0);
  cudaStream_t st;
  AFC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  afc_status s = AFC_OK;
  for (int a = 0; a < rank && s == AFC_OK; ++a) {
    p->axes[a].reset(new AxisPlan());
    s = build_axis(dims[a], p->dbl, *p->axes[a], st);
  }
  if (s == AFC_OK && kind == AFC_KIND_R2C_HALF) {
    const AxisPlan& la = *p->axes[rank - 1];
    if (la.algo != ALGO_SMEM && la.algo != ALGO_FOURSTEP && la.algo != ALGO_NOOP)
      s = fail(AFC_ERR_UNSUPPORTED, "half-spectrum plans need a smooth last dimension (got %lld)", (long long)dims[rank - 1]);
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (s != AFC_OK) return s;
  if (e != cudaSuccess) return cuda_fail(e, "plan build");
  p->ws_bytes = plan_ws_bytes(*p);
  *out = p.release();
  return AFC_OK;
}

// The workspace a call on stream st uses (caller holds p.ws_mu): the one st
// used last; else a new one while the plan has fewer than kWsSlots; else the
// least recently used one, whose fence orders st after its last use.  Inside a
// capture nothing is allocated when a workspace exists: the capture takes the
// most recently used one.
static afc_status take_ws_slot(afc_plan_s& p, cudaStream_t st, bool cap, WsSlot** out) {
  for (auto& w : p.ws_slots)
    if (w->st == st) {
      *out = w.get();
      return AFC_OK;
    }
  WsSlot* lru = nullptr;
  WsSlot* mru = nullptr;
  for (auto& w : p.ws_slots) {
    if (!lru || w->last < lru->last) lru = w.get();
    if (!mru || w->last > mru->last) mru = w.get();
  }
  if (cap && mru) {
    *out = mru;
    return AFC_OK;
  }
  if (p.ws_slots.size() < kWsSlots) {
    std::unique_ptr<WsSlot> w(new WsSlot());
    AFC_CUDA(dev_alloc(&w->ptr, p.ws_bytes), "workspace");
    w->st = st;
    p.ws_slots.push_back(std::move(w));
    *out = p.ws_slots.back().get();
    return AFC_OK;
  }
  *out = lru;
  return AFC_OK;
}

static afc_status execute(afc_plan p, const void* in, void* out, afc_direction dir, double scale, bool use_scale,
                          double pair_w, void* ws, size_t ws_bytes, bool own_ws, void* stream) {
  if (!p) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!in || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (dir != AFC_FORWARD && dir != AFC_INVERSE)
    return fail(AFC_ERR_VALIDATION, "validation failed for `direction`: `%d` violates `FORWARD|INVERSE`", (int)dir);
  const bool inv = dir == AFC_INVERSE;
  if (in == out && p->kind != AFC_KIND_C2C)
    return fail(AFC_ERR_SHAPE_MISMATCH, "shape mismatch: expected distinct real and complex buffers, got in == out");
  const double sc = use_scale ? scale : (inv ? 1.0 / (double)p->N() : 1.0);
  DeviceGuard g(p->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (p->tc) {
    const AxisPlan& ap = *p->axes[0];
    TcLaunch d;
    d.in = in;
    d.out = out;
    d.tw = ap.lp.tw;
    d.sl = ap.lp.sl;
    d.lanes = p->batch;
    d.scale = sc;
    d.inverse = inv ? 1 : 0;
    d.err = device_err_word();
    if (!d.err) return fail(AFC_ERR_OUT_OF_MEMORY, "error word allocation failed");
    cudaError_t e = launch_tc_fft(d, p->tc == 2, st);
    if (e != cudaSuccess) return cuda_fail(e, "execute (tensor cores)");
    return AFC_OK;
  }
  if (own_ws) {
    if (!p->ws_bytes) {  // single-pass plans touch no plan-owned buffer
      cudaError_t e = run_plan(*p, in, out, inv, sc, pair_w, nullptr, st);
      if (e != cudaSuccess) return cuda_fail(e, "execute");
      return AFC_OK;
    }
    std::lock_guard<std::mutex> lk(p->ws_mu);
    const bool cap = stream_capturing(st);
    WsSlot* w = nullptr;
    afc_status s = take_ws_slot(*p, st, cap, &w);
    if (s != AFC_OK) return s;
    AFC_CUDA(w->fence.before(st, cap), "workspace ordering");
    cudaError_t e = run_plan(*p, in, out, inv, sc, pair_w, w->ptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "execute");
    AFC_CUDA(w->fence.after(st, cap), "workspace ordering");
    w->st = st;
    w->last = ++p->ws_tick;
    return AFC_OK;
  }
  if (ws_bytes < p->ws_bytes)
    return fail(AFC_ERR_VALIDATION, "validation failed for `workspace_bytes`: `%zu` violates `>= %zu`", ws_bytes, p->ws_bytes);
  if (p->ws_bytes && !ws) return fail(AFC_ERR_VALIDATION, "validation failed for `workspace`: `null` violates `must be non-null`");
  cudaError_t e = run_plan(*p, in, out, inv, sc, pair_w, ws, st);
  if (e != cudaSuccess) return cuda_fail(e, "execute");
  return AFC_OK;
}

// ───────────────────────────── uneven batches ─────────────────────────────

struct BatchGroup {
  int64_t n = 0;
  long long lanes = 0;
  std::unique_ptr<AxisPlan> ap;
  long long* d_off = nullptr;  // device lane offsets (packed layout)
  size_t ws_off = 0;           // this group's workspace region (groups of a phase run concurrently)
  ~BatchGroup() {
    if (d_off) cudaFree(d_off);
  }
};

}  // namespace afc

struct afc_batch_plan_s {
  bool dbl = false;
  int device = 0;
  int64_t total = 0;
  std::vector<int64_t> lengths;
  std::vector<std::unique_ptr<afc::BatchGroup>> groups;
  size_t ws_bytes = 0;
  void* ws = nullptr;
  std::mutex mu;
  // persistent phases, per direction
  struct Phase {
    void* descs = nullptr;          // device KArgs records
    afc::BatchItem* items = nullptr;  // device tile list
    int nitems = 0;
    size_t smem = 0;
    int grid = 0;
  };
  std::vector<Phase> phases[2];
  int* counters = nullptr;  // one per phase and direction
  afc::Fence fence;         // last use of ws / counters on the GPU
  // CUDA graph of the persistent phases, keyed by (in, out, direction)
  cudaGraphExec_t gexec = nullptr;
  const void* g_in = nullptr;
  void* g_out = nullptr;
  int g_dir = -1;
  ~afc_batch_plan_s() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (ws) cudaFree(ws);
    for (auto& v : phases)
      for (auto& ph : v) {
        if (ph.descs) cudaFree(ph.descs);
        if (ph.items) cudaFree(ph.items);
      }
    if (counters) cudaFree(counters);
  }
};

namespace afc {

// Plain per-length launches (mode 1): the same kernels the single plans use.
static cudaError_t run_batch(afc_batch_plan_s& bp, const void* in, void* out, bool inv, cudaStream_t st) {
  for (auto& g : bp.groups) {
    AxisIO io;
    io.in = in;
    io.out = out;
    io.lanes = g->lanes;
    io.im = LaneMap{1, 1, 0, 0, 1, 1, g->d_off};
    io.om = io.im;
    io.scale = inv ? 1.0 / (double)g->n : 1.0;
    cudaError_t e;
    if (g->ap->algo == ALGO_NOOP) {
      if (in == out) continue;
      LaunchDesc d;
      d.sl.n = 1;
      d.sl.nst = 0;
      d.P = 1;
      d.ld = 3;
      d.lanes = io.lanes;
      d.im = io.im;
      d.om = io.om;
      d.in = in;
      d.out = out;
      d.stage_in = d.stage_out = true;
      d.L = (int)std::min<long long>(256, std::max(1LL, io.lanes));
      e = do_lanes(d, bp.dbl, inv, st);
    } else {
      e = exec_axis(*g->ap, bp.dbl, inv, io, static_cast<char*>(bp.ws) + g->ws_off, st);
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Persistent phases (mode 0): one batch_kernel launch per phase.
static cudaError_t run_batch_persistent(afc_batch_plan_s& bp, const void* in, void* out, bool inv, cudaStream_t st) {
  auto& ph = bp.phases[inv ? 1 : 0];
  const size_t np = ph.size();
  int* ctr = bp.counters + (inv ? 8 : 0);
  cudaError_t e = cudaMemsetAsync(ctr, 0, np * sizeof(int), st);
  if (e != cudaSuccess) return e;
  for (size_t k = 0; k < np; ++k) {
    e = launch_batch(ph[k].descs, ph[k].items, ph[k].nitems, ctr + k, ph[k].smem, ph[k].grid, in, out, bp.ws, bp.dbl,
                     inv, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Autotuner: for each distinct smem-resident length, time the lanes kernel on a
// scratch buffer for a few threads-per-lane / lanes-per-tile shapes (tiles run
// on the persistent kernel's kBatchThreads-thread CTAs) and keep the fastest.  Results are
// cached per (length, precision) for the process.
static std::mutex g_tune_mu;
static std::map<std::pair<int64_t, int>, std::pair<int, int>> g_tune;

static void tune_group(BatchGroup& g, bool dbl, void* scratch, cudaStream_t st) {
  AxisPlan& ap = *g.ap;
  if (ap.algo != ALGO_SMEM) return;
  const auto key = std::make_pair(g.n, dbl ? 1 : 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      ap.tuned_P = it->second.first;
      ap.tuned_L = it->second.second;
      return;
    }
  }
  const size_t csz = dbl ? 16 : 8;
  int rmax = 2;
  for (int s2 = 0; s2 < ap.lp.sl.nst; ++s2) rmax = std::max(rmax, ap.lp.sl.st[s2].R);
  std::vector<int> cands;
  for (int div : {1, 2, 4, 8}) {
    int P = (int)std::min<int64_t>(kBatchThreads,
                                   std::max<int64_t>(1, (g.n + (int64_t)rmax * div - 1) / ((int64_t)rmax * div)));
    if (std::find(cands.begin(), cands.end(), P) == cands.end()) cands.push_back(P);
  }
  const long long lanes = std::max(1LL, std::min<long long>(g.lanes * 4, 64));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bestP = cands[0], bestL = 1;
  for (int P : cands) {
    LaunchDesc d;
    d.sl = ap.lp.sl;
    d.tw = ap.lp.tw;
    d.ld = ap.lp.ld;
    d.P = P;
    d.lanes = lanes;
    d.im = LaneMap{1, 1, g.n, 0, 0, 1, nullptr};
    d.om = d.im;
    d.in = scratch;
    d.out = scratch;
    const size_t per_lane = 2 * (size_t)d.ld * csz + 3 * sizeof(long long);
    int L = std::max(1, kBatchThreads / P);
    while (L > 1 && (size_t)L * per_lane > batch_smem_cap(dbl)) --L;
    d.L = L;
    d.stage_out = ap.lp.sl.nst <= 1;
    // a shape the device refuses is skipped; its error is consumed here so it
    // is not reported by a later launch
    if (launch_lanes(d, dbl, false, st) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3; ++r) launch_lanes(d, dbl, false, st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    // cost per lane on the persistent kernel: a tile of L lanes occupies one CTA
    const float per = ms / (float)lanes;
    if (per < best) {
      best = per;
      bestP = P;
      bestL = L;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ap.tuned_P = bestP;
  ap.tuned_L = bestL;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = std::make_pair(bestP, bestL);
}

// Records every group's launches for one direction and turns them into the
// phase lists of the persistent kernel (launch k of a group runs in phase k).
static afc_status build_phases(afc_batch_plan_s& bp, bool inv, cudaStream_t st) {
  const size_t ksz = kargs_size(bp.dbl);
  const size_t csz = bp.dbl ? 16 : 8;
  struct PhaseAcc {
    std::vector<unsigned char> descs;
    std::vector<BatchItem> items;
    std::vector<double> cost;
    size_t smem = 0;
  };
  std::vector<PhaseAcc> acc;
  for (auto& g : bp.groups) {
    Recorder rec;
    tl_rec = &rec;
    AxisIO io;
    io.in = tag_ptr(1, 0);
    io.out = tag_ptr(2, 0);
    io.lanes = g->lanes;
    io.im = LaneMap{1, 1, 0, 0, 1, 1, g->d_off};
    io.om = io.im;
    io.scale = inv ? 1.0 / (double)g->n : 1.0;
    cudaError_t e = cudaSuccess;
    if (g->ap->algo == ALGO_NOOP) {
      LaunchDesc d;
      d.sl.n = 1;
      d.sl.nst = 0;
      d.P = 1;
      d.ld = 3;
      d.lanes = io.lanes;
      d.im = io.im;
      d.om = io.om;
      d.in = io.in;
      d.out = io.out;
      d.stage_in = d.stage_out = true;
      d.L = (int)std::min<long long>(64, std::max(1LL, io.lanes));
      e = do_lanes(d, bp.dbl, inv, st);
    } else {
      e = exec_axis(*g->ap, bp.dbl, inv, io, tag_ptr(3, g->ws_off), st);
    }
    tl_rec = nullptr;
    if (e != cudaSuccess) return cuda_fail(e, "batch record");
    for (size_t k = 0; k < rec.launches.size(); ++k) {
      if (acc.size() <= k) acc.resize(k + 1);
      PhaseAcc& pa = acc[k];
      const RecLaunch& rl = rec.launches[k];
      const int di = (int)(pa.descs.size() / ksz);
      pa.descs.resize(pa.descs.size() + ksz);
      kargs_pack(rl.d, bp.dbl, pa.descs.data() + (size_t)di * ksz);
      const size_t sm = rl.kind == 0 ? lanes_smem_bytes(rl.d, csz) : conv_smem_bytes(rl.d, csz);
      pa.smem = std::max(pa.smem, sm);
      const long long tiles = (rl.d.lanes + rl.d.L - 1) / rl.d.L;
      const double c = (double)rl.d.sl.n * std::max(1, rl.d.sl.nst) * (rl.kind ? 2.0 : 1.0) * rl.d.L;
      for (long long t = 0; t < tiles; ++t) {
        pa.items.push_back(BatchItem{di, rl.kind == 1 ? 1 : (rl.inv ? 2 : 0), t * rl.d.L});
        pa.cost.push_back(c);
      }
    }
  }
  if (acc.size() > 8) return fail(AFC_ERR_UNSUPPORTED, "batch plan needs %zu phases (max 8)", acc.size());
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, bp.device);
  auto& out = bp.phases[inv ? 1 : 0];
  for (auto& pa : acc) {
    // longest tiles first, so the atomic tile counter balances the tail
    std::vector<size_t> ord(pa.items.size());
    for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return pa.cost[a] > pa.cost[b]; });
    std::vector<BatchItem> items(ord.size());
    for (size_t i = 0; i < ord.size(); ++i) items[i] = pa.items[ord[i]];
    afc_batch_plan_s::Phase ph;
    ph.nitems = (int)items.size();
    ph.smem = (pa.smem + 15) / 16 * 16;
    AFC_CUDA(dev_alloc(&ph.descs, pa.descs.size()), "batch descriptors");
    AFC_CUDA(dev_alloc((void**)&ph.items, items.size() * sizeof(BatchItem)), "batch items");
    AFC_CUDA(cudaMemcpyAsync(ph.descs, pa.descs.data(), pa.descs.size(), cudaMemcpyHostToDevice, st), "batch descriptors");
    AFC_CUDA(cudaMemcpyAsync(ph.items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, st),
             "batch items");
    const int per = batch_blocks_per_sm(ph.smem, bp.dbl, inv);
    ph.grid = (int)std::min<long long>((long long)sms * per, std::max(1, ph.nitems));
    out.push_back(ph);
  }
  return AFC_OK;
}

// ───────────────────────────── allocation-free entry point ─────────────────────────────
// Scratch for afc_execute_1d_no_alloc: the intermediate between the two passes
// of the four-step kernels.  A file-scope device array, so the entry point
// never allocates; every GPU that loads the library holds it until the process
// exits.  Host code must not use the array's name as a device address: the
// address comes from cudaGetSymbolAddress, once per device, with that device
// current.
static const size_t kNoAllocScratchBytes = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_no_alloc_scratch[kNoAllocScratchBytes];

static std::mutex g_no_alloc_mu;
static std::map<int, void*> g_no_alloc_ptr;  // device -> device address of g_no_alloc_scratch

static afc_status no_alloc_scratch(int dev, void** ptr) {
  std::lock_guard<std::mutex> lk(g_no_alloc_mu);
  auto it = g_no_alloc_ptr.find(dev);
  if (it != g_no_alloc_ptr.end()) {
    *ptr = it->second;
    return AFC_OK;
  }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_no_alloc_scratch);
  if (e != cudaSuccess || !p) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "no-alloc scratch address");
  g_no_alloc_ptr[dev] = p;
  *ptr = p;
  return AFC_OK;
}

}  // namespace afc

using namespace afc;

afc_nufft_plan_s::~afc_nufft_plan_s() {
  if (fft) afc_plan_destroy(fft);
  if (deconv) cudaFree(deconv);
  if (grid) cudaFree(grid);
}

afc_nufft3d_plan_s::~afc_nufft3d_plan_s() {
  for (int* b : {tiles.cnt, tiles.off, tiles.tile, tiles.rank, tiles.idx})
    if (b) cudaFree(b);
  if (fft) afc_plan_destroy(fft);
  if (deconv) cudaFree(deconv);
  if (grid) cudaFree(grid);
}

extern "C" {

afc_status afc_plan_create(afc_plan* out, int rank, const int64_t* dims, afc_precision precision, afc_kind kind,
                           int64_t batch, int device) {
  return create_plan(out, rank, dims, precision, kind, batch, device);
}

afc_status afc_plan_get_cached(afc_plan* out, int rank, const int64_t* dims, afc_precision precision, afc_kind kind,
                               int64_t batch, int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (rank < 1 || rank > 3 || !dims) return create_plan(out, rank, dims, precision, kind, batch, device);
  PlanKey k{};
  k.rank = rank;
  for (int a = 0; a < 3; ++a) k.d[a] = a < rank ? dims[a] : 1;
  k.prec = precision;
  k.kind = kind;
  k.batch = batch;
  k.device = device;
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_cache.find(k);
  if (it != g_cache.end()) {
    it->second->refs.fetch_add(1);
    *out = it->second;
    return AFC_OK;
  }
  afc_plan p = nullptr;
  afc_status s = create_plan(&p, rank, dims, precision, kind, batch, device);
  if (s != AFC_OK) return s;
  p->cached = true;
  p->key = k;
  p->refs.store(2);  // one for the cache, one for the caller
  g_cache[k] = p;
  *out = p;
  return AFC_OK;
}

afc_status afc_plan_destroy(afc_plan plan) {
  if (!plan) return AFC_OK;
  if (plan->cached) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (plan->refs.fetch_sub(1) > 1) return AFC_OK;
    g_cache.erase(plan->key);
  } else if (plan->refs.fetch_sub(1) > 1) {
    return AFC_OK;
  }
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_execute(afc_plan plan, const void* in, void* out, afc_direction direction, void* stream) {
  return execute(plan, in, out, direction, 0.0, false, 1.0, nullptr, 0, true, stream);
}

afc_status afc_execute_scaled(afc_plan plan, const void* in, void* out, afc_direction direction, double scale,
                              void* stream) {
  return execute(plan, in, out, direction, scale, true, 1.0, nullptr, 0, true, stream);
}

afc_status afc_execute_adjoint(afc_plan plan, const void* in, void* out, afc_direction direction, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  const double N = (double)plan->N();
  // adjoint of forward = unnormalized inverse map; adjoint of inverse = forward / N
  if (direction == AFC_FORWARD) {
    double pw = plan->kind == AFC_KIND_R2C_HALF ? 0.5 : 1.0;
    return execute(plan, in, out, AFC_INVERSE, 1.0, true, pw, nullptr, 0, true, stream);
  }
  if (direction == AFC_INVERSE) {
    double pw = plan->kind == AFC_KIND_R2C_HALF ? 2.0 : 1.0;
    return execute(plan, in, out, AFC_FORWARD, 1.0 / N, true, pw, nullptr, 0, true, stream);
  }
  return fail(AFC_ERR_VALIDATION, "validation failed for `direction`: `%d` violates `FORWARD|INVERSE`", (int)direction);
}

afc_status afc_workspace_size(afc_plan plan, size_t* bytes) {
  if (!plan || !bytes) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *bytes = plan->ws_bytes;
  return AFC_OK;
}

afc_status afc_execute_ws(afc_plan plan, const void* in, void* out, afc_direction direction, double scale, int use_scale,
                          void* workspace, size_t workspace_bytes, void* stream) {
  return execute(plan, in, out, direction, scale, use_scale != 0, 1.0, workspace, workspace_bytes, false, stream);
}

// STFT analysis frames of apollo-stft (stft/dimension_1d.rs:96-108): frames
// centred at m hop, 1 + ceil(signal_len / hop) of them; none when the signal is
// shorter than a frame.
static int64_t stft_frames(int64_t frame_len, int64_t hop, int64_t signal_len) {
  if (signal_len < frame_len) return 0;
  return 1 + (signal_len + hop - 1) / hop;
}

afc_status afc_stft_frame_count(int64_t frame_len, int64_t hop, int64_t signal_len, int64_t* frames) {
  if (!frames) return fail(AFC_ERR_VALIDATION, "validation failed for `frames`: `null` violates `must be non-null`");
  if (frame_len < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `frame_len`: `%lld` violates `> 0`", (long long)frame_len);
  if (hop < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `> 0`", (long long)hop);
  *frames = stft_frames(frame_len, hop, signal_len < 0 ? 0 : signal_len);
  return AFC_OK;
}

afc_status afc_stft_forward(afc_plan plan, const void* signal, int64_t signal_len, const void* window, int64_t hop,
                            void* out, int64_t out_elems, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!signal || !window || !out)
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (plan->rank != 1 || plan->kind != AFC_KIND_C2C || plan->tc)
    return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `rank %d` violates `rank-1 C2C f32/f64 plan`", plan->rank);
  const int64_t n = plan->dims[0];
  if (hop < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `> 0`", (long long)hop);
  if (hop > n)
    return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `<= frame_len %lld`", (long long)hop,
                (long long)n);
  if (signal_len < n)
    return fail(AFC_ERR_VALIDATION, "validation failed for `signal_len`: `%lld` violates `>= frame_len %lld`",
                (long long)signal_len, (long long)n);
  const int64_t frames = stft_frames(n, hop, signal_len);
  if (out_elems != frames * n)
    return fail(AFC_ERR_SHAPE_MISMATCH, "shape mismatch: expected %lld output elements (%lld frames x %lld), got %lld",
                (long long)(frames * n), (long long)frames, (long long)n, (long long)out_elems);
  const AxisPlan& ap = *plan->axes[0];
  const size_t csz = plan->dbl ? 16 : 8;
  DeviceGuard g(plan->device);
  if (ap.algo != ALGO_SMEM) {
    // frames beyond one CTA: gather the windowed frames into the output, then
    // the multi-pass plan in place (its workspace stream-ordered)
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    AFC_CUDA(stft_gather_dev(signal, window, signal_len, n, hop, frames, out, plan->dbl, st), "stft frames");
    AxisIO io;
    io.in = out;
    io.out = out;
    io.lanes = frames;
    io.im = io.om = LaneMap{1, 1, n, 0, 0, 1, nullptr};
    const size_t ab = axis_ws_bytes(ap, frames, csz);
    void* w = nullptr;
    if (ab) AFC_CUDA(cudaMallocAsync(&w, ab, st), "stft workspace");
    cudaError_t e = exec_axis(ap, plan->dbl, false, io, w, st);
    cudaError_t ef = w ? cudaFreeAsync(w, st) : cudaSuccess;
    if (e != cudaSuccess) return cuda_fail(e, "stft forward");
    AFC_CUDA(ef, "stft workspace");
    return AFC_OK;
  }
  LaunchDesc d;
  fill_common(d, ap.lp);
  d.lanes = frames;
  d.im = LaneMap{1, 1, hop, 0, 0, 1, nullptr};  // frame m: base m hop
  d.om = LaneMap{1, 1, n, 0, 0, 1, nullptr};
  d.in = signal;
  d.out = out;
  d.in_op = IN_FRAME;
  d.out_op = OUT_C;
  d.scale = 1.0;
  d.nlen = signal_len;
  d.window = window;
  d.frame_off = n / 2;
  d.stage_in = true;
  d.stage_out = ap.lp.sl.nst <= 1;
  d.L = choose_L(ap.lp, d.lanes, d.stage_in, d.stage_out, csz);
  cudaError_t e = launch_lanes(d, plan->dbl, false, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "stft forward");
  return AFC_OK;
}

afc_status afc_stft_inverse_workspace(afc_plan plan, int64_t hop, int64_t signal_len, size_t* bytes) {
  if (!plan || !bytes) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (hop < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `> 0`", (long long)hop);
  const int64_t n = plan->dims[0];
  *bytes = (size_t)stft_frames(n, hop, signal_len) * (size_t)n * (plan->dbl ? 8 : 4);
  return AFC_OK;
}

afc_status afc_stft_inverse(afc_plan plan, const void* spectrum, int64_t spectrum_elems, const void* window, int64_t hop,
                            void* out, int64_t signal_len, void* workspace, size_t workspace_bytes, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!spectrum || !window || !out || !workspace)
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (plan->rank != 1 || plan->kind != AFC_KIND_C2C || plan->tc)
    return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `rank %d` violates `rank-1 C2C f32/f64 plan`", plan->rank);
  const int64_t n = plan->dims[0];
  if (hop < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `> 0`", (long long)hop);
  if (hop > n)
    return fail(AFC_ERR_VALIDATION, "validation failed for `hop_len`: `%lld` violates `<= frame_len %lld`", (long long)hop,
                (long long)n);
  if (signal_len < n)
    return fail(AFC_ERR_VALIDATION, "validation failed for `signal_len`: `%lld` violates `>= frame_len %lld`",
                (long long)signal_len, (long long)n);
  const int64_t frames = stft_frames(n, hop, signal_len);
  if (spectrum_elems != frames * n)
    return fail(AFC_ERR_SHAPE_MISMATCH, "shape mismatch: expected %lld spectrum elements (%lld frames x %lld), got %lld",
                (long long)(frames * n), (long long)frames, (long long)n, (long long)spectrum_elems);
  const size_t rsz = plan->dbl ? 8 : 4;
  if (workspace_bytes < (size_t)frames * (size_t)n * rsz)
    return fail(AFC_ERR_VALIDATION, "validation failed for `workspace_bytes`: `%zu` violates `>= %zu`", workspace_bytes,
                (size_t)frames * (size_t)n * rsz);
  const AxisPlan& ap = *plan->axes[0];
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // frames beyond one CTA run the multi-pass plan, its workspace stream-ordered
  const size_t ab = axis_ws_bytes(ap, frames, plan->dbl ? 16 : 8);
  void* w = nullptr;
  if (ab) AFC_CUDA(cudaMallocAsync(&w, ab, st), "stft workspace");
  // 1. every frame: normalized inverse FFT, real part, into the workspace
  AxisIO io;
  io.in = spectrum;
  io.out = workspace;
  io.lanes = frames;
  io.im = LaneMap{1, 1, n, 0, 0, 1, nullptr};
  io.om = io.im;
  io.in_op = IN_C;
  io.out_op = OUT_RE;
  io.scale = 1.0 / (double)n;
  cudaError_t e = exec_axis(ap, plan->dbl, true, io, w, st);
  cudaError_t ef = w ? cudaFreeAsync(w, st) : cudaSuccess;
  if (e != cudaSuccess) return cuda_fail(e, "stft inverse frames");
  AFC_CUDA(ef, "stft workspace");
  // 2. windowed overlap-add, normalized by the summed squared window
  e = stft_ola_dev(workspace, window, frames, n, hop, signal_len, out, plan->dbl, st);
  if (e != cudaSuccess) return cuda_fail(e, "stft overlap-add");
  return AFC_OK;
}

// num-complex's product (a.re b.re - a.im b.im, a.re b.im + a.im b.re)
static std::complex<double> cmul_ref(std::complex<double> a, std::complex<double> b) {
  return {a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real()};
}

// num-complex powf (polar form): |z|^e exp(i arg(z) e), as the reference's
// CztPlan builds its chirps (czt/dimension_1d.rs:85-98).
static std::complex<double> czt_pow(std::complex<double> z, double e) {
  return std::polar(std::pow(std::abs(z), e), std::arg(z) * e);
}

afc_status afc_czt_plan_create(afc_czt_plan* out, int64_t n, int64_t m, double a_re, double a_im, double w_re,
                               double w_im, afc_precision prec, int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  if (n < 1 || m < 1)
    return fail(AFC_ERR_VALIDATION, "validation failed for `length`: `n=%lld, m=%lld` violates `> 0`", (long long)n,
                (long long)m);
  if (!std::isfinite(a_re) || !std::isfinite(a_im) || !std::isfinite(w_re) || !std::isfinite(w_im) ||
      (a_re == 0.0 && a_im == 0.0) || (w_re == 0.0 && w_im == 0.0))
    return fail(AFC_ERR_VALIDATION, "validation failed for `a, w`: `non-finite or zero` violates `finite, non-zero`");
  if (prec != AFC_PREC_F32 && prec != AFC_PREC_F64)
    return fail(AFC_ERR_VALIDATION, "validation failed for `precision`: `%d` violates `F32|F64`", (int)prec);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(AFC_ERR_BACKEND_UNAVAILABLE, "backend unavailable: cuda (no device)");
  if (device < 0 || device >= ndev)
    return fail(AFC_ERR_VALIDATION, "validation failed for `device`: `%d` violates `< %d`", device, ndev);
  const bool dbl = prec == AFC_PREC_F64;
  const size_t csz = dbl ? 16 : 8;
  int64_t L = 1;
  while (L < n + m - 1) L <<= 1;
  DeviceGuard g(device);
  std::unique_ptr<afc_czt_plan_s> p(new afc_czt_plan_s());
  p->n = n;
  p->m = m;
  p->L = L;
  p->dbl = dbl;
  p->device = device;
  const std::complex<double> A(a_re, a_im), W(w_re, w_im);
  std::vector<std::complex<double>> cn(n), ck(m), ker(L, 0.0);
  for (int64_t j = 0; j < n; ++j) cn[j] = czt_pow(A, -(double)j) * czt_pow(W, 0.5 * (double)j * (double)j);
  for (int64_t k = 0; k < m; ++k) ck[k] = czt_pow(W, 0.5 * (double)k * (double)k);
  for (int64_t k = 0; k < m; ++k) ker[k] = czt_pow(W, -0.5 * (double)k * (double)k) / (double)L;
  for (int64_t j = 1; j < n; ++j) ker[L - j] = czt_pow(W, -0.5 * (double)j * (double)j) / (double)L;
  auto upload = [&](const std::vector<std::complex<double>>& v, void** dst) -> cudaError_t {
    cudaError_t e = dev_alloc(dst, v.size() * csz);
    if (e != cudaSuccess) return e;
    if (dbl) return cudaMemcpy(*dst, v.data(), v.size() * csz, cudaMemcpyHostToDevice);
    std::vector<float> f(2 * v.size());
    for (size_t i = 0; i < v.size(); ++i) {
      f[2 * i] = (float)v[i].real();
      f[2 * i + 1] = (float)v[i].imag();
    }
    return cudaMemcpy(*dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
  };
  AFC_CUDA(upload(cn, &p->chirp_n), "CZT chirp");
  AFC_CUDA(upload(ck, &p->chirp_k), "CZT chirp");
  AFC_CUDA(upload(ker, &p->spec), "CZT kernel");
  // square plans: the inverse's nodes z_k = W^k and A^k by the reference's
  // recurrences (czt_inverse_nodes, kernel/bluestein.rs:167-175; the A^n
  // scaling of czt_bjork_pereyra_inverse_into, :215-220), and its collision
  // test |z_k - z_(k-j-1)| < 1024 eps over every pair the solve divides by
  if (n == m && (size_t)n * 32 <= kSmemMax) {
    std::vector<std::complex<double>> z(n), ap(n);
    std::complex<double> wk(1.0, 0.0), ak(1.0, 0.0);
    for (int64_t k = 0; k < n; ++k) {
      z[k] = wk;
      ap[k] = ak;
      wk = cmul_ref(wk, W);
      ak = cmul_ref(ak, A);
    }
    bool ok = true;
    for (int64_t d = 1; d < n && ok; ++d)
      for (int64_t k = d; k < n; ++k)
        if (std::hypot(z[k].real() - z[k - d].real(), z[k].imag() - z[k - d].imag()) <
            std::numeric_limits<double>::epsilon() * 1024.0) {
          ok = false;
          break;
        }
    p->invertible = ok;
    AFC_CUDA(dev_alloc(&p->nodes, (size_t)n * 16), "CZT nodes");
    AFC_CUDA(cudaMemcpy(p->nodes, z.data(), (size_t)n * 16, cudaMemcpyHostToDevice), "CZT nodes");
    AFC_CUDA(dev_alloc(&p->apow, (size_t)n * 16), "CZT nodes");
    AFC_CUDA(cudaMemcpy(p->apow, ap.data(), (size_t)n * 16, cudaMemcpyHostToDevice), "CZT nodes");
  }
  cudaStream_t st;
  AFC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  afc_status s = AFC_OK;
  if (plannable(L, csz)) {  // one convolution tile per lane
    s = build_lenplan(L, dbl, p->lp, st);
    if (s == AFC_OK) {
      AxisPlan mp;
      mp.n = L;
      mp.algo = ALGO_SMEM;
      mp.lp = p->lp;
      s = fft_table(mp, dbl, p->spec, st);
      mp.lp.tw = nullptr;  // owned by the CZT plan
    }
  } else {  // the convolution through the library's multi-pass plan of length L
    p->big.reset(new AxisPlan());
    s = build_axis(L, dbl, *p->big, st);
    if (s == AFC_OK) s = fft_table(*p->big, dbl, p->spec, st);
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (s != AFC_OK) return s;
  *out = p.release();
  return AFC_OK;
}

afc_status afc_czt_execute(afc_czt_plan plan, const void* in, void* out, int64_t batch, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!in || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (batch < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `batch`: `%lld` violates `> 0`", (long long)batch);
  const size_t csz = plan->dbl ? 16 : 8;
  DeviceGuard g(plan->device);
  if (plan->big) {
    // premultiply into a zero-padded workspace, forward FFT of length L,
    // product with the kernel spectrum (scaled 1/L), unnormalized inverse,
    // postmultiply of the first m bins (kernel/bluestein.rs:83-130); the
    // workspace is stream-ordered, so the call allocates nothing the host waits for
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t L = plan->L;
    const size_t wb = ((size_t)batch * L * csz + 255) / 256 * 256;
    const size_t ab = axis_ws_bytes(*plan->big, batch, csz);
    void* w = nullptr;
    AFC_CUDA(cudaMallocAsync(&w, wb + ab, st), "CZT workspace");
    AxisIO io;
    io.in = w;
    io.out = w;
    io.lanes = batch;
    io.im = io.om = LaneMap{1, 1, L, 0, 0, 1, nullptr};
    io.scale = 1.0;
    void* aws = static_cast<char*>(w) + wb;
    cudaError_t e = chirp_rows_dev(in, plan->n, plan->n, plan->chirp_n, w, L, L, batch, plan->dbl, st);
    if (e == cudaSuccess) e = exec_axis(*plan->big, plan->dbl, false, io, aws, st);
    if (e == cudaSuccess) e = chirp_rows_dev(w, L, L, plan->spec, w, L, L, batch, plan->dbl, st);
    if (e == cudaSuccess) e = exec_axis(*plan->big, plan->dbl, true, io, aws, st);
    if (e == cudaSuccess) e = chirp_rows_dev(w, L, plan->m, plan->chirp_k, out, plan->m, plan->m, batch, plan->dbl, st);
    cudaError_t ef = cudaFreeAsync(w, st);
    if (e != cudaSuccess) return cuda_fail(e, "czt execute");
    AFC_CUDA(ef, "CZT workspace");
    return AFC_OK;
  }
  LaunchDesc d;
  fill_common(d, plan->lp);
  d.lanes = batch;
  d.im = LaneMap{1, 1, plan->n, 0, 0, 1, nullptr};
  d.om = LaneMap{1, 1, plan->m, 0, 0, 1, nullptr};
  d.in = in;
  d.out = out;
  d.in_op = IN_CHIRP;      // x_j A^-j W^(j^2/2) for j < n, zero up to L
  d.out_op = OUT_CHIRP;    // W^(k^2/2) times the convolution, k < m
  d.nlen = plan->n;
  d.nlen_out = plan->m;
  d.chirp = plan->chirp_n;
  d.chirp_out = plan->chirp_k;
  d.chirp_conj = 0;
  d.spec = plan->spec;
  d.scale = 1.0;
  d.L = choose_L(plan->lp, batch, true, true, csz, 2 * csz + 3 * sizeof(long long), 2);
  cudaError_t e = do_conv(d, plan->dbl, false, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "czt execute");
  return AFC_OK;
}

afc_status afc_hilbert_plan_create(afc_hilbert_plan* out, int64_t n, afc_precision prec, int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  if (n < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `len`: `%lld` violates `> 0`", (long long)n);
  if (prec != AFC_PREC_F32 && prec != AFC_PREC_F64)
    return fail(AFC_ERR_VALIDATION, "validation failed for `precision`: `%d` violates `F32|F64`", (int)prec);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(AFC_ERR_BACKEND_UNAVAILABLE, "backend unavailable: cuda (no device)");
  if (device < 0 || device >= ndev)
    return fail(AFC_ERR_VALIDATION, "validation failed for `device`: `%d` violates `< %d`", device, ndev);
  const bool dbl = prec == AFC_PREC_F64;
  const size_t csz = dbl ? 16 : 8;
  if (n >= 2 && !plannable(n, csz))
    return fail(AFC_ERR_UNSUPPORTED, "analytic signal of length %lld needs a smooth length that fits one CTA",
                (long long)n);
  DeviceGuard g(device);
  std::unique_ptr<afc_hilbert_plan_s> p(new afc_hilbert_plan_s());
  p->n = n;
  p->dbl = dbl;
  p->device = device;
  if (n == 1) {  // x + 0i: no transform
    *out = p.release();
    return AFC_OK;
  }
  // the reference's apply_analytic_mask (direct.rs:130-143), with the inverse's 1/n folded in
  std::vector<double> mk(2 * n, 0.0);
  const int64_t positive_end = (n + 1) / 2;
  for (int64_t k = 0; k < n; ++k) {
    const double sc = (k == 0 || (n % 2 == 0 && k == n / 2)) ? 1.0 : (k < positive_end ? 2.0 : 0.0);
    mk[2 * k] = sc / (double)n;
  }
  if (dbl) {
    AFC_CUDA(dev_alloc(&p->mask, (size_t)n * csz), "analytic mask");
    AFC_CUDA(cudaMemcpy(p->mask, mk.data(), (size_t)n * csz, cudaMemcpyHostToDevice), "analytic mask");
  } else {
    std::vector<float> f(mk.begin(), mk.end());
    AFC_CUDA(dev_alloc(&p->mask, (size_t)n * csz), "analytic mask");
    AFC_CUDA(cudaMemcpy(p->mask, f.data(), (size_t)n * csz, cudaMemcpyHostToDevice), "analytic mask");
  }
  cudaStream_t st;
  AFC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  afc_status s = build_lenplan(n, dbl, p->lp, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (s != AFC_OK) return s;
  *out = p.release();
  return AFC_OK;
}

afc_status afc_hilbert_analytic(afc_hilbert_plan plan, const void* signal, void* out, int64_t batch, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!signal || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (batch < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `batch`: `%lld` violates `> 0`", (long long)batch);
  const size_t rsz = plan->dbl ? 8 : 4, csz = 2 * rsz;
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (plan->n == 1) {  // (x, 0) per lane
    AFC_CUDA(cudaMemsetAsync(out, 0, (size_t)batch * csz, st), "analytic signal");
    AFC_CUDA(cudaMemcpy2DAsync(out, csz, signal, rsz, rsz, (size_t)batch, cudaMemcpyDeviceToDevice, st),
             "analytic signal");
    return AFC_OK;
  }
  LaunchDesc d;
  fill_common(d, plan->lp);
  d.lanes = batch;
  d.im = LaneMap{1, 1, plan->n, 0, 0, 1, nullptr};
  d.om = LaneMap{1, 1, plan->n, 0, 0, 1, nullptr};
  d.in = signal;
  d.out = out;
  d.in_op = IN_R;     // real signal widened
  d.out_op = OUT_C;   // analytic signal
  d.spec = plan->mask;
  d.scale = 1.0;
  d.L = choose_L(plan->lp, batch, true, true, csz, 2 * csz + 3 * sizeof(long long), 2);
  cudaError_t e = do_conv(d, plan->dbl, false, st);
  if (e != cudaSuccess) return cuda_fail(e, "analytic signal");
  return AFC_OK;
}

afc_status afc_hilbert_plan_destroy(afc_hilbert_plan plan) {
  if (!plan) return AFC_OK;
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_czt_inverse(afc_czt_plan plan, const void* spectrum, void* out, int64_t batch, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!spectrum || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (batch < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `batch`: `%lld` violates `> 0`", (long long)batch);
  // the reference's errors (plan/czt/dimension_1d.rs:250-293, kernel/bluestein.rs:193-205)
  if (plan->n != plan->m)
    return fail(AFC_ERR_VALIDATION, "not invertible: inverse is only defined for square (M == N) CZT plans");
  if (!plan->nodes)
    return fail(AFC_ERR_UNSUPPORTED, "the device inverse CZT holds the length in shared memory: n <= %zu (got %lld)",
                kSmemMax / 32, (long long)plan->n);
  if (!plan->invertible)
    return fail(AFC_ERR_VALIDATION, "not invertible: Vandermonde nodes z_k collide; W is a root of unity of order <= N");
  DeviceGuard g(plan->device);
  AFC_CUDA(czt_inverse_dev(spectrum, out, plan->nodes, plan->apow, plan->n, batch, plan->dbl,
                           static_cast<cudaStream_t>(stream)),
           "czt inverse");
  return AFC_OK;
}

afc_status afc_czt_conv_len(afc_czt_plan plan, int64_t* conv_len) {
  if (!plan || !conv_len) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *conv_len = plan->L;
  return AFC_OK;
}

// I0 by the reference's power series (kaiser_bessel.rs:55-69) and the KB
// kernel's Fourier transform (kaiser_bessel.rs:120-133), host side.
static double nu_i0_host(double z) {
  const double scaled = 0.25 * z * z;
  double sum = 1.0, term = 1.0;
  for (int k = 1; k <= 256; ++k) {
    term *= scaled / ((double)k * (double)k);
    sum += term;
    if (term <= 2.220446049250313e-16 * sum) break;
  }
  return sum;
}
static double nu_kb_ft(double xi, int w, double beta, double i0b) {
  const double twx = 2.0 * M_PI * (double)w * xi;
  const double z2 = beta * beta - twx * twx;
  const double pre = 2.0 * (double)w / i0b;
  if (std::fabs(z2) < 1e-30) return pre;
  if (z2 > 0.0) {
    const double sq = std::sqrt(z2);
    return pre * std::sinh(sq) / sq;
  }
  const double sq = std::sqrt(-z2);
  return pre * std::sin(sq) / sq;
}

afc_status afc_nufft1d_plan_create(afc_nufft_plan* out, int64_t n, double dx, int64_t sigma, int64_t kernel_width,
                                   int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  if (n < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `n`: `%lld` violates `must be > 0`", (long long)n);
  if (!std::isfinite(dx) || dx <= 0.0)
    return fail(AFC_ERR_VALIDATION, "validation failed for `dx`: `%g` violates `must be finite and > 0`", dx);
  if (sigma < 2) return fail(AFC_ERR_VALIDATION, "validation failed for `sigma`: `%lld` violates `>= 2`", (long long)sigma);
  if (kernel_width < 2 || kernel_width > 32)
    return fail(AFC_ERR_VALIDATION, "validation failed for `kernel_width`: `%lld` violates `2..32`", (long long)kernel_width);
  std::unique_ptr<afc_nufft_plan_s> p(new afc_nufft_plan_s());
  p->n = n;
  p->m = sigma * n;
  p->w = (int)kernel_width;
  p->dx = dx;
  p->beta = M_PI * (1.0 - 1.0 / (2.0 * (double)sigma)) * (double)(2 * kernel_width);
  p->i0b = nu_i0_host(p->beta);
  p->device = device;
  afc_status s = afc_plan_create(&p->fft, 1, &p->m, AFC_PREC_F64, AFC_KIND_C2C, 1, device);
  if (s != AFC_OK) return s;
  DeviceGuard g(device);
  std::vector<double> dec(n);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t ks = k <= n / 2 ? k : k - n;
    dec[k] = 1.0 / nu_kb_ft((double)ks / (double)p->m, p->w, p->beta, p->i0b);
  }
  AFC_CUDA(dev_alloc((void**)&p->deconv, (size_t)n * sizeof(double)), "NUFFT deconvolution");
  AFC_CUDA(cudaMemcpy(p->deconv, dec.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice), "NUFFT deconvolution");
  AFC_CUDA(dev_alloc(&p->grid, (size_t)p->m * 16), "NUFFT grid");
  *out = p.release();
  return AFC_OK;
}

static NuLaunch nu_launch(const afc_nufft_plan_s& p) {
  NuLaunch L;
  L.m = p.m;
  L.w = p.w;
  L.beta = p.beta;
  L.i0b = p.i0b;
  L.len = (double)p.n * p.dx;
  return L;
}

afc_status afc_nufft1d_type1(afc_nufft_plan plan, const double* positions, const void* values, int64_t npts, void* out,
                             void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!out || (npts > 0 && (!positions || !values)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(plan->mu);
  const bool cap = stream_capturing(st);
  AFC_CUDA(plan->fence.before(st, cap), "NUFFT ordering");
  AFC_CUDA(cudaMemsetAsync(plan->grid, 0, (size_t)plan->m * 16, st), "NUFFT grid");
  AFC_CUDA(nufft_spread_dev(nu_launch(*plan), positions, values, npts, plan->grid, st), "NUFFT spread");
  afc_status s = afc_execute(plan->fft, plan->grid, plan->grid, AFC_FORWARD, stream);
  if (s != AFC_OK) return s;
  AFC_CUDA(nufft_deconv_out_dev(plan->grid, plan->deconv, plan->n, plan->m, out, st), "NUFFT deconvolution");
  AFC_CUDA(plan->fence.after(st, cap), "NUFFT ordering");
  return AFC_OK;
}

afc_status afc_nufft1d_type2(afc_nufft_plan plan, const void* coeffs, const double* positions, int64_t npts, void* out,
                             void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!coeffs || (npts > 0 && (!positions || !out)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(plan->mu);
  const bool cap = stream_capturing(st);
  AFC_CUDA(plan->fence.before(st, cap), "NUFFT ordering");
  AFC_CUDA(cudaMemsetAsync(plan->grid, 0, (size_t)plan->m * 16, st), "NUFFT grid");
  AFC_CUDA(nufft_place_coeffs_dev(coeffs, plan->deconv, plan->n, plan->m, plan->grid, st), "NUFFT coefficients");
  // the reference's normalized inverse times m = the unnormalized inverse
  afc_status s = afc_execute_scaled(plan->fft, plan->grid, plan->grid, AFC_INVERSE, 1.0, stream);
  if (s != AFC_OK) return s;
  AFC_CUDA(nufft_interp_dev(nu_launch(*plan), plan->grid, positions, npts, out, st), "NUFFT interpolation");
  AFC_CUDA(plan->fence.after(st, cap), "NUFFT ordering");
  return AFC_OK;
}

// Domain checks of UniformDomain1D::new / UniformGrid3D::new
// (apollo-nufft/src/domain/metadata/grid.rs:36-48,76-101).
static afc_status check_domain(const char* nname, int64_t n, const char* dname, double d) {
  if (n <= 0) return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%lld` violates `must be > 0`", nname, (long long)n);
  if (!std::isfinite(d) || d <= 0.0)
    return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%g` violates `must be finite and > 0`", dname, d);
  return AFC_OK;
}

static afc_status direct_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(AFC_ERR_BACKEND_UNAVAILABLE, "backend unavailable: cuda (no device)");
  if (device < 0 || device >= ndev)
    return fail(AFC_ERR_VALIDATION, "validation failed for `device`: `%d` violates `< %d`", device, ndev);
  return AFC_OK;
}

afc_status afc_nudft1d_type1(const double* positions, const void* values, int64_t npts, int64_t n, double dx,
                             void* out, int device, void* stream) {
  afc_status s = check_domain("n", n, "dx", dx);
  if (s != AFC_OK) return s;
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!out || (npts > 0 && (!positions || !values)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if ((s = direct_device(device)) != AFC_OK) return s;
  DeviceGuard g(device);
  AFC_CUDA(nudft1_type1_dev(positions, values, npts, n, (double)n * dx, out, static_cast<cudaStream_t>(stream)),
           "direct type-1 NUDFT");
  return AFC_OK;
}

afc_status afc_nudft1d_type2(const void* coeffs, int64_t n, const double* positions, int64_t npts, double dx,
                             void* out, int device, void* stream) {
  afc_status s = check_domain("n", n, "dx", dx);
  if (s != AFC_OK) return s;
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!coeffs || (npts > 0 && (!positions || !out)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if ((s = direct_device(device)) != AFC_OK) return s;
  DeviceGuard g(device);
  AFC_CUDA(nudft1_type2_dev(coeffs, n, positions, npts, (double)n * dx, out, static_cast<cudaStream_t>(stream)),
           "direct type-2 NUDFT");
  return AFC_OK;
}

afc_status afc_nudft3d_type1(const double* positions, const void* values, int64_t npts, int64_t nx, int64_t ny,
                             int64_t nz, double dx, double dy, double dz, void* out, int device, void* stream) {
  afc_status s = AFC_OK;
  if ((s = check_domain("nx", nx, "dx", dx)) != AFC_OK) return s;
  if ((s = check_domain("ny", ny, "dy", dy)) != AFC_OK) return s;
  if ((s = check_domain("nz", nz, "dz", dz)) != AFC_OK) return s;
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!out || (npts > 0 && (!positions || !values)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if ((s = direct_device(device)) != AFC_OK) return s;
  DeviceGuard g(device);
  AFC_CUDA(nudft3_type1_dev(positions, values, npts, nx, ny, nz, (double)nx * dx, (double)ny * dy, (double)nz * dz, out,
                            static_cast<cudaStream_t>(stream)),
           "direct 3D type-1 NUDFT");
  return AFC_OK;
}

afc_status afc_nufft_plan_destroy(afc_nufft_plan plan) {
  if (!plan) return AFC_OK;
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_nufft3d_plan_create(afc_nufft3d_plan* out, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                   double dz, int64_t sigma, int64_t kernel_width, int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  const int64_t n[3] = {nx, ny, nz};
  const double d[3] = {dx, dy, dz};
  static const char* nname[3] = {"nx", "ny", "nz"};
  static const char* dname[3] = {"dx", "dy", "dz"};
  for (int a = 0; a < 3; ++a) {
    if (n[a] < 1)
      return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%lld` violates `must be > 0`", nname[a],
                  (long long)n[a]);
    if (!std::isfinite(d[a]) || d[a] <= 0.0)
      return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%g` violates `must be finite and > 0`", dname[a],
                  d[a]);
  }
  if (sigma < 2) return fail(AFC_ERR_VALIDATION, "validation failed for `sigma`: `%lld` violates `>= 2`", (long long)sigma);
  if (kernel_width < 2 || kernel_width > 32)
    return fail(AFC_ERR_VALIDATION, "validation failed for `kernel_width`: `%lld` violates `2..32`", (long long)kernel_width);
  std::unique_ptr<afc_nufft3d_plan_s> p(new afc_nufft3d_plan_s());
  p->w = (int)kernel_width;
  p->beta = M_PI * (1.0 - 1.0 / (2.0 * (double)sigma)) * (double)(2 * kernel_width);
  p->i0b = nu_i0_host(p->beta);
  p->device = device;
  int64_t total_n = 0;
  for (int a = 0; a < 3; ++a) {
    p->n[a] = n[a];
    p->d[a] = d[a];
    if (n[a] > (int64_t(1) << 40) / sigma)
      return fail(AFC_ERR_VALIDATION, "validation failed for `%s`: `%lld` violates `oversampled length overflow`",
                  nname[a], (long long)n[a]);
    int64_t lower = std::max<int64_t>(n[a] * sigma, 2 * kernel_width + 1), m = 1;
    while (m < lower) m <<= 1;
    p->m[a] = m;
    total_n += n[a];
  }
  afc_status s = afc_plan_create(&p->fft, 3, p->m, AFC_PREC_F64, AFC_KIND_C2C, 1, device);
  if (s != AFC_OK) return s;
  DeviceGuard g(device);
  std::vector<double> dec;
  dec.reserve((size_t)total_n);
  for (int a = 0; a < 3; ++a)
    for (int64_t k = 0; k < n[a]; ++k) {
      const int64_t ks = k <= n[a] / 2 ? k : k - n[a];
      dec.push_back(1.0 / nu_kb_ft((double)ks / (double)p->m[a], p->w, p->beta, p->i0b));
    }
  AFC_CUDA(dev_alloc((void**)&p->deconv, (size_t)total_n * sizeof(double)), "NUFFT deconvolution");
  AFC_CUDA(cudaMemcpy(p->deconv, dec.data(), (size_t)total_n * sizeof(double), cudaMemcpyHostToDevice),
           "NUFFT deconvolution");
  AFC_CUDA(dev_alloc(&p->grid, (size_t)(p->m[0] * p->m[1] * p->m[2]) * 16), "NUFFT grid");
  const int B = nufft3_tile_size(p->w);
  const int64_t ntiles = B ? (p->m[0] / B) * (p->m[1] / B) * (p->m[2] / B) : 0;
  if (B && ntiles < (int64_t(1) << 30)) {
    p->tiles.B = B;
    p->tiles.ntx = (int)(p->m[0] / B);
    p->tiles.nty = (int)(p->m[1] / B);
    p->tiles.ntz = (int)(p->m[2] / B);
    AFC_CUDA(dev_alloc((void**)&p->tiles.cnt, (size_t)ntiles * sizeof(int)), "NUFFT tiles");
    AFC_CUDA(dev_alloc((void**)&p->tiles.off, (size_t)(ntiles + 1) * sizeof(int)), "NUFFT tiles");
  }
  *out = p.release();
  return AFC_OK;
}

// Grows the per-point tile buffers (synchronous allocation) when a call brings
// more points than any call before it; false -> the per-point kernels run.
static afc_status nu3_reserve(afc_nufft3d_plan_s& p, int64_t npts, bool* tiled) {
  *tiled = p.tiles.B != 0 && npts > 0 && npts <= INT32_MAX;
  if (!*tiled || npts <= p.pts_cap) return AFC_OK;
  for (int** b : {&p.tiles.tile, &p.tiles.rank, &p.tiles.idx}) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  p.pts_cap = 0;
  for (int** b : {&p.tiles.tile, &p.tiles.rank, &p.tiles.idx})
    AFC_CUDA(dev_alloc((void**)b, (size_t)npts * sizeof(int)), "NUFFT point buckets");
  p.pts_cap = npts;
  return AFC_OK;
}

afc_status afc_nufft3d_grid_dims(afc_nufft3d_plan plan, int64_t* m) {
  if (!plan || !m) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  for (int a = 0; a < 3; ++a) m[a] = plan->m[a];
  return AFC_OK;
}

static NuLaunch3 nu_launch3(const afc_nufft3d_plan_s& p) {
  NuLaunch3 L;
  L.nx = p.n[0], L.ny = p.n[1], L.nz = p.n[2];
  L.mx = p.m[0], L.my = p.m[1], L.mz = p.m[2];
  L.w = p.w;
  L.beta = p.beta;
  L.i0b = p.i0b;
  L.lx = (double)p.n[0] * p.d[0];
  L.ly = (double)p.n[1] * p.d[1];
  L.lz = (double)p.n[2] * p.d[2];
  return L;
}

afc_status afc_nufft3d_type1(afc_nufft3d_plan plan, const double* positions, const void* values, int64_t npts,
                             void* out, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!out || (npts > 0 && (!positions || !values)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(plan->mu);
  const bool cap = stream_capturing(st);
  AFC_CUDA(plan->fence.before(st, cap), "NUFFT ordering");
  const NuLaunch3 L = nu_launch3(*plan);
  AFC_CUDA(cudaMemsetAsync(plan->grid, 0, (size_t)(L.mx * L.my * L.mz) * 16, st), "NUFFT grid");
  bool tiled = false;
  afc_status r = nu3_reserve(*plan, npts, &tiled);
  if (r != AFC_OK) return r;
  if (tiled)
    AFC_CUDA(nufft3_tiled_dev(L, plan->tiles, true, positions, values, npts, plan->grid, st), "NUFFT spread");
  else
    AFC_CUDA(nufft3_spread_dev(L, positions, values, npts, plan->grid, st), "NUFFT spread");
  afc_status s = afc_execute(plan->fft, plan->grid, plan->grid, AFC_FORWARD, stream);
  if (s != AFC_OK) return s;
  const double* dc = plan->deconv;
  AFC_CUDA(nufft3_modes_dev(L, dc, dc + L.nx, dc + L.nx + L.ny, plan->grid, out, false, st), "NUFFT deconvolution");
  AFC_CUDA(plan->fence.after(st, cap), "NUFFT ordering");
  return AFC_OK;
}

afc_status afc_nufft3d_type2(afc_nufft3d_plan plan, const void* modes, const double* positions, int64_t npts,
                             void* out, void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (npts < 0) return fail(AFC_ERR_VALIDATION, "validation failed for `npts`: `%lld` violates `>= 0`", (long long)npts);
  if (!modes || (npts > 0 && (!positions || !out)))
    return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(plan->mu);
  const bool cap = stream_capturing(st);
  AFC_CUDA(plan->fence.before(st, cap), "NUFFT ordering");
  const NuLaunch3 L = nu_launch3(*plan);
  AFC_CUDA(cudaMemsetAsync(plan->grid, 0, (size_t)(L.mx * L.my * L.mz) * 16, st), "NUFFT grid");
  const double* dc = plan->deconv;
  AFC_CUDA(nufft3_modes_dev(L, dc, dc + L.nx, dc + L.nx + L.ny, modes, plan->grid, true, st), "NUFFT modes");
  // the reference's three normalized inverse axis passes: scale 1/(mx my mz)
  afc_status s = afc_execute(plan->fft, plan->grid, plan->grid, AFC_INVERSE, stream);
  if (s != AFC_OK) return s;
  bool tiled = false;
  s = nu3_reserve(*plan, npts, &tiled);
  if (s != AFC_OK) return s;
  if (tiled)
    AFC_CUDA(nufft3_tiled_dev(L, plan->tiles, false, positions, plan->grid, npts, out, st), "NUFFT interpolation");
  else
    AFC_CUDA(nufft3_interp_dev(L, plan->grid, positions, npts, out, st), "NUFFT interpolation");
  AFC_CUDA(plan->fence.after(st, cap), "NUFFT ordering");
  return AFC_OK;
}

afc_status afc_nufft3d_plan_destroy(afc_nufft3d_plan plan) {
  if (!plan) return AFC_OK;
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_czt_plan_destroy(afc_czt_plan plan) {
  if (!plan) return AFC_OK;
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_plan_io_elems(afc_plan plan, afc_direction direction, int64_t* in_elems, int64_t* out_elems) {
  if (!plan || !in_elems || !out_elems)
    return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  int64_t a, b;
  io_elems(*plan, direction == AFC_INVERSE, a, b);
  *in_elems = a;
  *out_elems = b;
  return AFC_OK;
}

afc_status afc_execute_host(afc_plan plan, const void* host_in, void* host_out, afc_direction direction) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!host_in || !host_out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  const bool inv = direction == AFC_INVERSE;
  int64_t ie, oe;
  io_elems(*plan, inv, ie, oe);
  const size_t csz = plan->dbl ? 16 : 8, rsz = plan->dbl ? 8 : 4;
  bool real_in = plan->kind != AFC_KIND_C2C && !inv;
  bool real_out = plan->kind != AFC_KIND_C2C && inv;
  const size_t ib = (size_t)ie * (real_in ? rsz : csz), ob = (size_t)oe * (real_out ? rsz : csz);
  const size_t maxb = (size_t)std::max(ie, oe) * csz;
  DeviceGuard g(plan->device);
  // Take a free staging set (own stream, own buffers), creating one while the
  // plan has fewer than kHostStages; otherwise wait until a call returns one.
  // Concurrent host threads on one shared plan thus never share a buffer.
  HostStage* hs = nullptr;
  {
    std::unique_lock<std::mutex> lk(plan->host_mu);
    for (;;) {
      for (auto& s : plan->stages)
        if (!s->busy) {
          hs = s.get();
          break;
        }
      if (hs || plan->stages.size() < kHostStages) break;
      plan->host_cv.wait(lk);
    }
    if (!hs) {
      std::unique_ptr<HostStage> ns(new HostStage());
      AFC_CUDA(cudaStreamCreateWithFlags(&ns->st, cudaStreamNonBlocking), "stream");
      AFC_CUDA(dev_alloc(&ns->in, maxb), "staging");
      AFC_CUDA(dev_alloc(&ns->out, maxb), "staging");
      plan->stages.push_back(std::move(ns));
      hs = plan->stages.back().get();
    }
    hs->busy = true;
  }
  struct Release {
    afc_plan p;
    HostStage* s;
    ~Release() {
      std::lock_guard<std::mutex> lk(p->host_mu);
      s->busy = false;
      p->host_cv.notify_one();
    }
  } release{plan, hs};
  cudaStream_t st = hs->st;
  AFC_CUDA(cudaMemcpyAsync(hs->in, host_in, ib, cudaMemcpyHostToDevice, st), "host to device");
  afc_status s = afc_execute(plan, hs->in, hs->out, direction, st);
  if (s != AFC_OK) {
    cudaStreamSynchronize(st);  // the staging set goes back idle
    return s;
  }
  AFC_CUDA(cudaMemcpyAsync(host_out, hs->out, ob, cudaMemcpyDeviceToHost, st), "device to host");
  AFC_CUDA(cudaStreamSynchronize(st), "synchronize");
  return AFC_OK;
}

afc_status afc_capabilities(afc_capabilities_t* caps) {
  if (!caps) return fail(AFC_ERR_VALIDATION, "validation failed for `caps`: `null` violates `must be non-null`");
  memset(caps, 0, sizeof(*caps));
  caps->kind = 2;
  caps->normalization = 0;
  caps->supports_1d = caps->supports_2d = caps->supports_3d = 1;
  caps->supports_real_to_complex = 1;
  caps->supports_mixed_precision = 1;
  caps->default_precision = AFC_PREC_F64;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
  caps->device_count = n;
  if (n > 0) {
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, 0) == cudaSuccess) {
      caps->sm_count = pr.multiProcessorCount;
      caps->cc_major = pr.major;
      caps->cc_minor = pr.minor;
      caps->max_smem_per_block = pr.sharedMemPerBlockOptin;
    }
  }
  return AFC_OK;
}

afc_status afc_length_info(uint64_t n, afc_length_info_t* info) {
  if (!info) return fail(AFC_ERR_VALIDATION, "validation failed for `info`: `null` violates `must be non-null`");
  memset(info, 0, sizeof(*info));
  if (n == 0) return fail(AFC_ERR_VALIDATION, "validation failed for `n`: `0` violates `must be > 0`");
  info->strategy = strategy_of(n);
  std::vector<u64> f;
  if (factorize23(n, f)) {
    auto lo = lower_pairs(f);
    info->n_radices = (int)lo.size();
    for (size_t i = 0; i < lo.size() && i < 64; ++i) info->radices[i] = lo[i];
  } else {
    info->n_radices = -1;
  }
  u64 a, b;
  if (coprime_split(n, a, b)) { info->coprime_n1 = a; info->coprime_n2 = b; }
  if ((n & (n - 1)) == 0 && n > 1) {
    unsigned k = __builtin_ctzll(n), k1 = k / 2;
    info->four_step_n1 = 1ull << k1;
    info->four_step_n2 = 1ull << (k - k1);
  }
  info->is_prime = is_prime_u(n);
  if (info->is_prime) {
    info->primitive_root = primitive_root_u(n);
    info->primitive_root_inv = inv_mod(info->primitive_root, n);
  }
  info->is_short_winograd = short_winograd(n);
  info->has_static_coprime_codelet = coprime_split(n, a, b) ? static_coprime_codelet(a, b) : 0;
  // GPU choice (as build_axis would make it for f64)
  std::vector<int> rad;
  if (n <= 1) info->gpu_algo = ALGO_NOOP;
  else if (gpu_radices((int64_t)n, rad)) {
    if (plannable((int64_t)n, 16)) {
      info->gpu_algo = ALGO_SMEM;
      info->gpu_n_radices = (int)rad.size();
      for (size_t i = 0; i < rad.size(); ++i) info->gpu_radices[i] = rad[i];
    } else {
      info->gpu_algo = ALGO_FOURSTEP;
    }
  } else if (is_prime_u(n) && (int64_t)n < kRaderMax) {
    info->gpu_algo = ALGO_RADER;
    int64_t L = (int64_t)n - 1, M = L;
    if (!plannable(L, 16)) { M = 1; while (M < 2 * L - 1) M <<= 1; }
    info->gpu_conv_len = (u64)M;
  } else {
    info->gpu_algo = ALGO_BLUESTEIN;
    int64_t M = 1;
    while (M < 2 * (int64_t)n - 1) M <<= 1;
    info->gpu_conv_len = (u64)M;
  }
  return AFC_OK;
}

afc_status afc_rader_maps(uint64_t p, uint64_t* gather, uint64_t* scatter) {
  if (!gather || !scatter) return fail(AFC_ERR_VALIDATION, "validation failed for `maps`: `null` violates `must be non-null`");
  if (!is_prime_u(p)) return fail(AFC_ERR_VALIDATION, "validation failed for `p`: `%llu` violates `must be prime`", (unsigned long long)p);
  const u64 g = primitive_root_u(p), L = p - 1;
  u64 v = 1;
  for (u64 q = 0; q < L; ++q) { gather[q] = v; v = mulmod(v, g, p); }
  for (u64 q = 0; q < L; ++q) scatter[q] = q == 0 ? gather[0] : gather[L - q];
  return AFC_OK;
}

afc_status afc_pfa_perm(uint64_t n1, uint64_t n2, uint64_t* in_perm, uint64_t* out_perm) {
  if (!in_perm || !out_perm) return fail(AFC_ERR_VALIDATION, "validation failed for `perm`: `null` violates `must be non-null`");
  u64 a = n1, b = n2;
  while (b) { u64 t = a % b; a = b; b = t; }
  if (n1 < 1 || n2 < 1 || a != 1)
    return fail(AFC_ERR_VALIDATION, "validation failed for `n1,n2`: `%llu,%llu` violates `coprime`", (unsigned long long)n1,
                (unsigned long long)n2);
  const u64 n = n1 * n2;
  const u64 i21 = n1 > 1 ? inv_mod(n2 % n1, n1) : 0, i12 = n2 > 1 ? inv_mod(n1 % n2, n2) : 0;
  for (u64 x = 0; x < n1; ++x)
    for (u64 y = 0; y < n2; ++y) in_perm[x * n2 + y] = (x * n2 + y * n1) % n;
  for (u64 k1 = 0; k1 < n1; ++k1)
    for (u64 k2 = 0; k2 < n2; ++k2)
      out_perm[k2 * n1 + k1] = (u64)(((unsigned __int128)k1 * n2 * i21 + (unsigned __int128)k2 * n1 * i12) % n);
  return AFC_OK;
}

afc_status afc_plan_describe(afc_plan plan, int axis, afc_length_info_t* info) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (axis < 0 || axis >= plan->rank) return fail(AFC_ERR_VALIDATION, "validation failed for `axis`: `%d` violates `< rank`", axis);
  afc_status s = afc_length_info((uint64_t)plan->dims[axis], info);
  if (s != AFC_OK) return s;
  const AxisPlan& ap = *plan->axes[axis];
  info->gpu_algo = ap.algo;
  info->gpu_conv_len = (u64)ap.M;
  info->gpu_split_n1 = (u64)ap.N1;
  info->gpu_split_n2 = (u64)ap.N2;
  const LenPlan& lp = ap.algo == ALGO_FOURSTEP ? ap.lp1 : ap.lp;
  info->gpu_n_radices = ap.algo == ALGO_FOURSTEP ? 0 : lp.sl.nst;
  for (int s2 = 0; s2 < info->gpu_n_radices; ++s2) info->gpu_radices[s2] = lp.sl.st[s2].R;
  return AFC_OK;
}


afc_status afc_batch_plan_create(afc_batch_plan* out, const int64_t* lengths, int64_t count, afc_precision precision,
                                 int device) {
  if (!out) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *out = nullptr;
  if (!lengths || count < 1) return fail(AFC_ERR_VALIDATION, "validation failed for `count`: `%lld` violates `must be > 0`", (long long)count);
  if (precision != AFC_PREC_F32 && precision != AFC_PREC_F64)
    return fail(AFC_ERR_UNSUPPORTED, "batch plans support f32 and f64");
  for (int64_t i = 0; i < count; ++i)
    if (lengths[i] <= 0) return fail(AFC_ERR_VALIDATION, "validation failed for `lengths[%lld]`: `%lld` violates `must be > 0`", (long long)i, (long long)lengths[i]);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(AFC_ERR_BACKEND_UNAVAILABLE, "backend unavailable: cuda (no device)");
  if (device < 0 || device >= ndev) return fail(AFC_ERR_VALIDATION, "validation failed for `device`: `%d` violates `< %d`", device, ndev);
  DeviceGuard g(device);
  std::unique_ptr<afc_batch_plan_s> bp(new afc_batch_plan_s());
  bp->dbl = precision == AFC_PREC_F64;
  bp->device = device;
  bp->lengths.assign(lengths, lengths + count);
  std::map<int64_t, std::vector<long long>> by_len;
  long long off = 0;
  for (int64_t i = 0; i < count; ++i) {
    by_len[lengths[i]].push_back(off);
    off += lengths[i];
  }
  bp->total = off;
  cudaStream_t st;
  AFC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  const size_t csz = bp->dbl ? 16 : 8;
  afc_status s = AFC_OK;
  // single-CTA lengths of a batch keep several persistent CTAs per SM
  tl_smem_cap = batch_smem_cap(bp->dbl);
  int64_t max_smem_len = 1;
  for (auto& kv : by_len) {
    std::unique_ptr<BatchGroup> grp(new BatchGroup());
    grp->n = kv.first;
    grp->lanes = (long long)kv.second.size();
    grp->ap.reset(new AxisPlan());
    s = build_axis(kv.first, bp->dbl, *grp->ap, st);
    if (s != AFC_OK) break;
    if (grp->ap->algo == ALGO_SMEM) max_smem_len = std::max<int64_t>(max_smem_len, kv.first * (int64_t)grp->lanes);
    cudaError_t e = dev_alloc((void**)&grp->d_off, kv.second.size() * sizeof(long long));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(grp->d_off, kv.second.data(), kv.second.size() * sizeof(long long), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { s = cuda_fail(e, "batch offsets"); break; }
    grp->ws_off = bp->ws_bytes;
    bp->ws_bytes += (axis_ws_bytes(*grp->ap, grp->lanes, csz) + 255) / 256 * 256;
    bp->groups.push_back(std::move(grp));
  }
  if (s == AFC_OK) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = cuda_fail(e, "batch plan build");
  }
  // autotune the smem-resident lengths on a scratch buffer
  if (s == AFC_OK && env_int("AFC_AUTOTUNE", 1)) {
    void* scratch = nullptr;
    // four times the largest shared-memory group (the tuner runs up to 4x its
    // lanes, at most 64) plus 1 MiB
    const size_t sb = (size_t)std::max<int64_t>(max_smem_len, 1) * 4 * csz + ((size_t)1 << 20);
    if (dev_alloc(&scratch, sb) != cudaSuccess) {
      cudaGetLastError();  // no scratch: the lengths keep their default shapes
    } else {
      cudaMemsetAsync(scratch, 0, sb, st);
      for (auto& grp : bp->groups) tune_group(*grp, bp->dbl, scratch, st);
      cudaStreamSynchronize(st);
      cudaFree(scratch);
    }
  }
  if (s == AFC_OK && bp->ws_bytes) {
    cudaError_t e = dev_alloc(&bp->ws, bp->ws_bytes);
    if (e != cudaSuccess) s = cuda_fail(e, "batch workspace");
  }
  if (s == AFC_OK) {
    cudaError_t e = dev_alloc((void**)&bp->counters, 16 * sizeof(int));
    if (e != cudaSuccess) s = cuda_fail(e, "batch counters");
  }
  if (s == AFC_OK) s = build_phases(*bp, false, st);
  if (s == AFC_OK) s = build_phases(*bp, true, st);
  tl_smem_cap = kSmemMax;
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (s != AFC_OK) return s;
  if (e != cudaSuccess) return cuda_fail(e, "batch plan build");
  *out = bp.release();
  return AFC_OK;
}

afc_status afc_batch_plan_destroy(afc_batch_plan plan) {
  if (!plan) return AFC_OK;
  DeviceGuard g(plan->device);
  delete plan;
  return AFC_OK;
}

afc_status afc_batch_total_elems(afc_batch_plan plan, int64_t* elems) {
  if (!plan || !elems) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  *elems = plan->total;
  return AFC_OK;
}

afc_status afc_batch_execute(afc_batch_plan plan, const void* in, void* out, afc_direction direction, int mode,
                             void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!in || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (direction != AFC_FORWARD && direction != AFC_INVERSE)
    return fail(AFC_ERR_VALIDATION, "validation failed for `direction`: `%d` violates `FORWARD|INVERSE`", (int)direction);
  const bool inv = direction == AFC_INVERSE;
  DeviceGuard g(plan->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(plan->mu);
  // the plan-owned workspace and tile counters: ordered after their last use
  const bool cap = stream_capturing(st);
  AFC_CUDA(plan->fence.before(st, cap), "batch ordering");
  if (mode == 1) {
    cudaError_t e = run_batch(*plan, in, out, inv, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch execute");
    AFC_CUDA(plan->fence.after(st, cap), "batch ordering");
    return AFC_OK;
  }
  if (mode == 2) {  // persistent phases without the graph
    cudaError_t e = run_batch_persistent(*plan, in, out, inv, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch execute");
    AFC_CUDA(plan->fence.after(st, cap), "batch ordering");
    return AFC_OK;
  }
  // mode 0: the persistent phases as one CUDA graph, captured once per (in,
  // out, direction).  A call without a matching graph runs the phases
  // directly (so every kernel of the plan has run outside a capture before it
  // is captured, and the driver has sized its local memory), then captures the
  // graph for the next call.  A capture the driver refuses leaves the plan
  // without a graph: the next call runs the phases directly and tries again.
  // Inside a caller's own capture the phases are recorded into it directly.
  if (cap) {
    cudaError_t e = run_batch_persistent(*plan, in, out, inv, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch execute");
    AFC_CUDA(plan->fence.after(st, cap), "batch ordering");
    return AFC_OK;
  }
  if (!plan->gexec || plan->g_in != in || plan->g_out != out || plan->g_dir != (int)direction) {
    if (plan->gexec) { cudaGraphExecDestroy(plan->gexec); plan->gexec = nullptr; }
    cudaError_t e = run_batch_persistent(*plan, in, out, inv, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch execute");
    AFC_CUDA(plan->fence.after(st, cap), "batch ordering");
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess) {
      cudaGraph_t graph = nullptr;
      e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const cudaError_t e2 = run_batch_persistent(*plan, in, out, inv, cs);
        e = cudaStreamEndCapture(cs, &graph);
        if (e2 != cudaSuccess) e = e2;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&plan->gexec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      cudaStreamDestroy(cs);
      if (e == cudaSuccess) {
        plan->g_in = in;
        plan->g_out = out;
        plan->g_dir = (int)direction;
      } else {
        if (plan->gexec) cudaGraphExecDestroy(plan->gexec);
        plan->gexec = nullptr;
      }
    }
    cudaGetLastError();  // a refused capture is not an error of this call
    return AFC_OK;
  }
  AFC_CUDA(cudaGraphLaunch(plan->gexec, st), "batch graph launch");
  AFC_CUDA(plan->fence.after(st, cap), "batch ordering");
  return AFC_OK;
}

const char* afc_last_error_message(void) { return g_last_error.c_str(); }

uint64_t afc_kernel_launch_count(void) { return g_launches.load(); }

// Test hook (not part of the public header): the next `count` device
// allocations fail, so tests can check the AFC_ERR_OUT_OF_MEMORY path.

AFC_API afc_status afc_execute_1d_no_alloc(afc_plan plan, const void* in, void* out, afc_direction direction,
                                           void* stream) {
  if (!plan) return fail(AFC_ERR_VALIDATION, "validation failed for `plan`: `null` violates `must be non-null`");
  if (!in || !out) return fail(AFC_ERR_VALIDATION, "validation failed for `buffer`: `null` violates `must be non-null`");
  if (direction != AFC_FORWARD && direction != AFC_INVERSE)
    return fail(AFC_ERR_VALIDATION, "validation failed for `direction`: `%d` violates `FORWARD|INVERSE`", (int)direction);
  if (plan->rank != 1 || plan->kind != AFC_KIND_C2C || plan->axes[0]->algo != ALGO_FOURSTEP)
    return fail(AFC_ERR_UNSUPPORTED, "afc_execute_1d_no_alloc runs rank-1 C2C plans on the two-pass kernels (got rank %d, kind %d, algo %d)",
                plan->rank, (int)plan->kind, plan->axes[0]->algo);
  const size_t csz = plan->dbl ? 16 : 8;
  const size_t need = (size_t)plan->batch * (size_t)plan->dims[0] * csz;
  if (need > kNoAllocScratchBytes)
    return fail(AFC_ERR_VALIDATION,
                "validation failed for `batch * n`: needs %zu bytes of scratch, the static scratch holds %zu bytes (16 MiB)",
                need, kNoAllocScratchBytes);
  DeviceGuard g(plan->device);
  void* scratch = nullptr;
  afc_status s = no_alloc_scratch(plan->device, &scratch);
  if (s != AFC_OK) return s;
  const bool inv = direction == AFC_INVERSE;
  long long lanes = 0;
  AxisIO io;
  io.im = io.om = axis_map(*plan, 0, plan->dims[0], lanes);
  io.lanes = lanes;
  io.in = in;
  io.out = out;
  io.scale = inv ? 1.0 / (double)plan->N() : 1.0;
  cudaError_t e = exec_fourstep(*plan->axes[0], plan->dbl, inv, io, scratch, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "execute (no alloc)");
  return AFC_OK;
}

// Test hook (not part of the public header): one tensor-core tile
// D = A * B^T (A 128 x 32, B 32 x 32, f32 host arrays split into hi/lo BF16 or
// FP16 halves), used to check the operand descriptors.  Returns AFC_ERR_TIMEOUT
// if the MMA completion barrier timed out.
AFC_API afc_status afc_test_tc_tile(const float* hA, const float* hB, float* hD, int fp16) {
  float *dA = nullptr, *dB = nullptr, *dD = nullptr;
  unsigned* err = nullptr;
  AFC_CUDA(cudaMalloc(&dA, 128 * 32 * 4), "alloc");
  AFC_CUDA(cudaMalloc(&dB, 32 * 32 * 4), "alloc");
  AFC_CUDA(cudaMalloc(&dD, 128 * 32 * 4), "alloc");
  AFC_CUDA(cudaMalloc(&err, 4), "alloc");
  cudaMemcpy(dA, hA, 128 * 32 * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB, 32 * 32 * 4, cudaMemcpyHostToDevice);
  cudaMemset(err, 0, 4);
  cudaError_t e = launch_tc_selftest(dA, dB, dD, err, fp16 != 0, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned he = 0;
  if (e == cudaSuccess) e = cudaMemcpy(hD, dD, 128 * 32 * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(err);
  if (e != cudaSuccess) return cuda_fail(e, "tc tile");
  if (he) return fail(AFC_ERR_TIMEOUT, "tensor-core completion barrier timed out");
  return AFC_OK;
}

// Reads and clears the device error word bounded waits set on timeout (after
// synchronizing the device): AFC_ERR_TIMEOUT if any kernel gave up waiting.
AFC_API afc_status afc_test_take_device_error(void) {
  unsigned* w = device_err_word();
  if (!w) return fail(AFC_ERR_OUT_OF_MEMORY, "error word");
  unsigned h = 0;
  AFC_CUDA(cudaDeviceSynchronize(), "synchronize");
  AFC_CUDA(cudaMemcpy(&h, w, 4, cudaMemcpyDeviceToHost), "read error word");
  cudaMemset(w, 0, 4);
  if (h) return fail(AFC_ERR_TIMEOUT, "a kernel's bounded wait timed out");
  return AFC_OK;
}

// Runs one bounded wait that nothing completes (a barrier with no arrival), so
// the timeout path can be tested without a fault: the wait gives up after
// `polls` polls, the kernel returns, and the result is read back through the
// error word like any kernel timeout (AFC_ERR_TIMEOUT).
AFC_API afc_status afc_test_bounded_wait(int polls) {
  if (polls < 1 || polls > (1 << 21))
    return fail(AFC_ERR_VALIDATION, "validation failed for `polls`: `%d` violates `1..2^21`", polls);
  unsigned* w = device_err_word();
  if (!w) return fail(AFC_ERR_OUT_OF_MEMORY, "error word");
  cudaError_t e = launch_wait_probe(w, polls, 0);
  if (e != cudaSuccess) return cuda_fail(e, "wait probe");
  return afc_test_take_device_error();
}

AFC_API void afc_test_fail_next_allocs(int count) { g_fail_allocs.store(count); }

}  // extern "C"
