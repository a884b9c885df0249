// apollo_oracle.cpp -- CPU restatement of apollo-fft's dense FFT plan execution.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the timed
// CPU baseline for the apollofft_b200 CUDA library.  Nothing in the shipped
// library links, loads or calls it; only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg do, and only as the checker.
//
// The reference (ryancinsight/apollofft) is Rust and cannot be compiled here
// (no cargo/rustc), so this is a restatement of its algorithms in C++17.
// Every function names the reference file:line it follows (paths relative to
// crates/apollo-fft/src unless stated).  Integer maps are restated verbatim in
// behaviour (bit-exact); floating-point kernels follow the same algorithm and
// twiddle generation, with the hand-written Winograd/PFA codelets replaced by
// generic DFTs of the same size (exact DFTs; agreement ~1e-15 relative).
//
// Parity pinning: the integer layer is checked against the reference's own
// known-answer tests and the float layer against its published fixtures
// (DFT4, IDFT4, impulse->flat spectrum) plus an independent long-double
// direct DFT and scipy.fft, in tests/test_oracle_*.py.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

using usize = uint64_t;

// ───────────────────────────── integer layer ─────────────────────────────

// apollo-fft-macros/src/shared_math.rs:15-23 (gcd)
static usize gcd(usize a, usize b) {
  while (b != 0) { usize r = a % b; a = b; b = r; }
  return a;
}

// apollo-fft-macros/src/shared_math.rs:25-38 (mod_pow, square-and-multiply)
static usize mod_pow(usize base, usize exp, usize m) {
  unsigned __int128 res = 1, b = base % m;
  while (exp > 0) {
    if (exp & 1) res = (res * b) % m;
    b = (b * b) % m;
    exp >>= 1;
  }
  return (usize)res;
}

// apollo-fft-macros/src/shared_math.rs:40-62 (modular_inverse, extended Euclid)
static usize modular_inverse(usize a, usize m) {
  int64_t old_r = (int64_t)a, r = (int64_t)m, old_s = 1, s = 0;
  while (r != 0) {
    int64_t q = old_r / r;
    int64_t t = old_r - q * r; old_r = r; r = t;
    t = old_s - q * s; old_s = s; s = t;
  }
  int64_t res = old_s % (int64_t)m;
  if (res < 0) res += (int64_t)m;
  return (usize)res;
}

// apollo-fft-macros/src/shared_math.rs:64-87 (prime_factors_all, ascending)
static std::vector<usize> prime_factors_all(usize n) {
  std::vector<usize> f;
  while (n % 2 == 0 && n > 0) { f.push_back(2); n /= 2; }
  for (usize d = 3; d * d <= n; d += 2)
    while (n % d == 0) { f.push_back(d); n /= d; }
  if (n > 1) f.push_back(n);
  return f;
}

// application/execution/kernel/radix_shape.rs:60-170 (factorize_composite).
// Returns false for "None": unsupported prime factor or pure power of two.
// Order: 23s, 17s, 13s, 11s, 7s, 5s, 3s (innermost) then 2s (outermost).
static bool factorize_composite(usize n, std::vector<usize>& out) {
  out.clear();
  if (n <= 1) return true;  // Some(empty)
  static const usize primes[8] = {2, 3, 5, 7, 11, 13, 17, 23};
  usize cnt[8] = {0};
  usize rem = n;
  for (int i = 0; i < 8; ++i)
    while (rem % primes[i] == 0) { cnt[i]++; rem /= primes[i]; }
  if (rem > 1) return false;
  bool only2 = true;
  for (int i = 1; i < 8; ++i) if (cnt[i]) only2 = false;
  if (only2) return false;
  for (int i = 7; i >= 0; --i)
    for (usize k = 0; k < cnt[i]; ++k) out.push_back(primes[i]);
  return true;
}

// radix_shape.rs:172-190 (is_prime, 6k±1 trial division)
static bool is_prime(usize n) {
  if (n <= 1) return false;
  if (n <= 3) return true;
  if (n % 2 == 0 || n % 3 == 0) return false;
  for (usize i = 5; i * i <= n; i += 6)
    if (n % i == 0 || n % (i + 2) == 0) return false;
  return true;
}

// radix_shape.rs:192-219 (coprime_factors): n1 = prime power of the largest
// prime factor, n2 = n / n1.  None for prime powers.
static bool coprime_factors(usize n, usize& n1, usize& n2) {
  std::vector<usize> f = prime_factors_all(n);
  if (f.empty()) return false;
  std::vector<usize> pp;
  usize cur = f[0], pw = f[0];
  for (size_t i = 1; i < f.size(); ++i) {
    if (f[i] == cur) pw *= f[i];
    else { pp.push_back(pw); cur = f[i]; pw = f[i]; }
  }
  pp.push_back(pw);
  if (pp.size() < 2) return false;
  n1 = pp.back();
  pp.pop_back();
  n2 = 1;
  for (usize v : pp) n2 *= v;
  return true;
}

// radix_shape.rs:221-234 (lower_radix2_pairs_to_radix4, greedy left to right)
static std::vector<usize> lower_radix2_pairs_to_radix4(const std::vector<usize>& r) {
  std::vector<usize> o;
  size_t i = 0;
  while (i < r.size()) {
    if (i + 1 < r.size() && r[i] == 2 && r[i + 1] == 2) { o.push_back(4); i += 2; }
    else { o.push_back(r[i]); i += 1; }
  }
  return o;
}

// mixed_radix/caches/misc.rs:94-122 (cached_prime23_radices = lowered factorization)
static bool prime23_radices(usize n, std::vector<usize>& out) {
  std::vector<usize> f;
  if (!factorize_composite(n, f)) return false;
  out = lower_radix2_pairs_to_radix4(f);
  return true;
}

// mixed_radix/traits.rs:172-176 (SHORT_WINOGRAD_SIZES)
static const usize kShortWinograd[] = {
    2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22,
    23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43,
    44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 58, 60, 62, 63, 64, 81, 128};
static bool is_short_winograd(usize n) {
  for (usize v : kShortWinograd) if (v == n) return true;
  return false;
}

// components/good_thomas/three_by_prime.rs:1-11 and apollo-fft-macros/src/lib.rs:145-147:
// supports(n1, n2) = n2 == 3 && n1 in THREE_BY_PRIME_PRIMES.
static const usize kThreeByPrime[] = {5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
static bool three_by_prime_supports(usize n1, usize n2) {
  if (n2 != 3) return false;
  for (usize p : kThreeByPrime) if (p == n1) return true;
  return false;
}

// apollo-fft-macros/src/good_thomas.rs:300-325 (canonical_coprime_factors)
static bool canonical_coprime_factors(usize n, usize& n1, usize& n2) {
  usize rem = n;
  std::vector<usize> pp;
  usize p = 2;
  while (p * p <= rem) {
    if (rem % p == 0) {
      usize pw = 1;
      while (rem % p == 0) { pw *= p; rem /= p; }
      pp.push_back(pw);
    }
    p += (p == 2) ? 1 : 2;
  }
  if (rem > 1) pp.push_back(rem);
  if (pp.size() < 2) return false;
  n1 = pp.back();
  pp.pop_back();
  n2 = 1;
  for (usize v : pp) n2 *= v;
  return true;
}

// components/good_thomas/fixed.rs:31-45 + apollo-fft-macros/src/good_thomas.rs:244-297
// (parse_dispatch_pairs): the statically generated (n1, n2) codelet pairs.
static bool fixed_supports(usize n1, usize n2) {
  static const usize short_sizes[] = {2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12,
                                      13, 14, 15, 16, 17, 18, 19, 23, 24, 25, 27,
                                      29, 31, 32, 36, 37, 41, 43, 47, 53};
  static const usize direct_pair_primes[] = {11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                             5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43,
                                             47, 53};
  const usize max_n = 200;
  bool a_in = false, b_in = false;
  for (usize s : short_sizes) { if (s == n1) a_in = true; if (s == n2) b_in = true; }
  if (!a_in || !b_in) return false;
  usize n = n1 * n2;
  if (!(n1 > 1 && n2 > 1 && n <= max_n && gcd(n1, n2) == 1)) return false;
  for (usize s : short_sizes) if (s == n) return false;
  usize c1, c2;
  if (!canonical_coprime_factors(n, c1, c2) || c1 != n1 || c2 != n2) return false;
  usize lo = std::min(n1, n2), hi = std::max(n1, n2);
  if (lo == 2 || lo == 3)
    for (usize p : direct_pair_primes) if (p == hi) return false;
  return true;
}

// components/good_thomas/mod.rs:29-31 (has_static_coprime_codelet)
static bool has_static_coprime_codelet(usize n1, usize n2) {
  return three_by_prime_supports(n1, n2) || fixed_supports(n1, n2);
}

// components/rader/generator.rs:18-64 (primitive_root: static table then search)
// apollo-fft-macros/src/shared_primitives.rs holds the same table.
static usize primitive_root_dynamic(usize p) {
  if (p == 2) return 1;
  usize phi = p - 1;
  std::vector<usize> f = prime_factors_all(phi);
  f.erase(std::unique(f.begin(), f.end()), f.end());
  for (usize g = 2; g < p; ++g) {
    bool ok = true;
    for (usize q : f) if (mod_pow(g, phi / q, p) == 1) { ok = false; break; }
    if (ok) return g;
  }
  return 0;
}
static usize primitive_root(usize p) {
  switch (p) {
    case 2: return 1;   case 3: return 2;   case 5: return 2;   case 7: return 3;
    case 11: return 2;  case 13: return 2;  case 17: return 3;  case 19: return 2;
    case 23: return 5;  case 29: return 2;  case 31: return 3;  case 37: return 2;
    case 41: return 6;  case 43: return 3;  case 47: return 5;  case 53: return 2;
    case 59: return 2;  case 61: return 2;  case 67: return 2;  case 71: return 7;
    case 73: return 5;  case 79: return 3;  case 83: return 2;  case 89: return 3;
    case 97: return 5;  case 101: return 2; case 109: return 6; case 113: return 3;
    case 127: return 3; case 131: return 2; case 151: return 6; case 167: return 5;
    case 173: return 2; case 179: return 2; case 181: return 2; case 193: return 5;
    case 197: return 2; case 199: return 3; case 10007: return 5;
    default: return primitive_root_dynamic(p);
  }
}

// components/rader/generator.rs:96-120 (inverse_mod)
static usize inverse_mod(usize a, usize m) {
  if (m == 1) return 0;
  int64_t m0 = (int64_t)m, y = 0, x = 1, ai = (int64_t)a;
  while (ai > 1) {
    int64_t q = ai / m0;
    int64_t t = m0;
    m0 = ai % m0;
    ai = t;
    t = y;
    y = x - q * y;
    x = t;
  }
  if (x < 0) x += (int64_t)m;
  return (usize)x;
}

// components/rader/mod.rs:237-246 (build_generator_order: order[q] = g^q mod n)
static std::vector<usize> generator_order(usize n, usize g) {
  std::vector<usize> o(n - 1);
  usize v = 1;
  for (usize q = 0; q < n - 1; ++q) { o[q] = v; v = (usize)(((unsigned __int128)v * g) % n); }
  return o;
}

// components/rader/mod.rs:215-228 (inverse_generator_order_at: g^{-q})
static usize inverse_generator_order_at(const std::vector<usize>& o, usize q) {
  return q == 0 ? o[0] : o[o.size() - q];
}

// mixed_radix/caches/misc.rs:233-256 (build_pfa_perm)
static void build_pfa_perm(usize n1, usize n2, std::vector<usize>& in_perm,
                           std::vector<usize>& out_perm) {
  usize n = n1 * n2;
  usize inv_n2_n1 = modular_inverse(n2 % n1, n1);
  usize inv_n1_n2 = modular_inverse(n1 % n2, n2);
  in_perm.assign(n, 0);
  out_perm.assign(n, 0);
  for (usize i1 = 0; i1 < n1; ++i1)
    for (usize i2 = 0; i2 < n2; ++i2) in_perm[i1 * n2 + i2] = (i1 * n2 + i2 * n1) % n;
  for (usize k1 = 0; k1 < n1; ++k1)
    for (usize k2 = 0; k2 < n2; ++k2)
      out_perm[k2 * n1 + k1] =
          (usize)(((unsigned __int128)k1 * n2 * inv_n2_n1 + (unsigned __int128)k2 * n1 * inv_n1_n2) % n);
}

// Strategy codes: which kernel family mixed_radix/dispatch.rs:26-82 routes n to.
enum Strategy : int {
  kNoop = 0,          // n <= 1
  kStockham = 1,      // pow2 >= 64, not four-step (dispatch.rs:112-130)
  kFourStep = 2,      // pow2 >= 4096, even log2 (dispatch.rs:97-110, tuning.rs:13)
  kWinograd = 3,      // SHORT_WINOGRAD_SIZES (traits.rs:172)
  kPfaStatic = 4,     // coprime split with generated codelet (dispatch.rs:44-53)
  kComposite = 5,     // {2,3,5,7,11,13,17,23}-smooth (dispatch.rs:56-63)
  kPfaGeneric = 6,    // coprime split, generic PFA (dispatch.rs:65-73)
  kRaderFull = 7,     // prime, N-1 < 1024 (rader/mod.rs:67-73)
  kRaderHalf = 8,     // prime, N-1 >= 1024: half-cyclic CRT split
  kUntransformed = 9  // prime power p^k, p > 23, not short: dispatch returns unchanged
};

static int dispatch_strategy(usize n) {
  if (n <= 1) return kNoop;
  bool pow2 = (n & (n - 1)) == 0;
  if (pow2 && n >= 64) {
    if (n >= 4096 && (__builtin_ctzll(n) % 2 == 0)) return kFourStep;
    return kStockham;
  }
  if (is_short_winograd(n)) return kWinograd;
  usize n1 = 0, n2 = 0;
  bool cop = coprime_factors(n, n1, n2);
  if (cop && has_static_coprime_codelet(n1, n2)) return kPfaStatic;
  std::vector<usize> r;
  if (prime23_radices(n, r)) return kComposite;
  if (cop) return kPfaGeneric;
  if (is_prime(n)) return (n - 1 >= 1024) ? kRaderHalf : kRaderFull;
  return kUntransformed;
}

// ──────────────────────────── float kernels ─────────────────────────────

template <class F> using Cx = std::complex<F>;

// Plain complex product written out so no compiler contracts it differently from
// num-complex's `*` (re = a.re*b.re - a.im*b.im, im = a.re*b.im + a.im*b.re).
template <class F> static inline Cx<F> cmul(Cx<F> a, Cx<F> b) {
  return Cx<F>(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// twiddle_table.rs:153-195 (build_twiddle_table): n-1 entries, stage s (len=2^s)
// at offset len/2-1, W_len^j by f64 recurrence, narrowed to F.
template <class F> static std::vector<Cx<F>> build_twiddle_table(usize n, double sign) {
  std::vector<Cx<F>> t;
  if (n <= 1) return t;
  t.resize(n - 1);
  usize cursor = 0;
  for (usize len = 2; len <= n; len <<= 1) {
    usize half = len >> 1;
    double a = sign * 2.0 * M_PI / (double)len;
    double wr = std::cos(a), wi = std::sin(a), tr = 1.0, ti = 0.0;
    for (usize j = 0; j < half; ++j) {
      t[cursor + j] = Cx<F>((F)tr, (F)ti);
      double nr = tr * wr - ti * wi, ni = tr * wi + ti * wr;
      tr = nr; ti = ni;
    }
    cursor += half;
  }
  return t;
}

template <class F> struct TwCache {
  std::map<std::pair<usize, int>, std::vector<Cx<F>>> pow2;
  std::map<std::pair<usize, int>, std::vector<Cx<F>>> four;
  std::map<std::pair<std::vector<usize>, int>, std::vector<Cx<F>>> comp;
};
template <class F> static TwCache<F>& tw_cache() {
  static thread_local TwCache<F> c;
  return c;
}
template <class F> static const std::vector<Cx<F>>& pow2_table(usize n, bool inv) {
  auto& m = tw_cache<F>().pow2;
  auto key = std::make_pair(n, (int)inv);
  auto it = m.find(key);
  if (it != m.end()) return it->second;
  return m.emplace(key, build_twiddle_table<F>(n, inv ? 1.0 : -1.0)).first->second;
}

// Radix-2 Stockham autosort, pass with prev_len P: read src[b + k*n/2], write
// dst[g*2P + j + k*P] with b = g*P + j, input k=1 multiplied by W_{2P}^j taken
// from the pow2 table (offset P-1).  Semantics of stockham/butterfly/stage.rs:31-84
// and the transform driver stockham/transform.rs:16-147 (fusing 2-4 radix-2
// stages changes operation order only).
template <class F>
static void stockham_pow2(Cx<F>* data, Cx<F>* scratch, usize n, const Cx<F>* tw, F scale, bool do_scale) {
  Cx<F>* src = data;
  Cx<F>* dst = scratch;
  usize half = n / 2;
  for (usize P = 1; P < n; P <<= 1) {
    const Cx<F>* w = tw + (P - 1);
    for (usize b = 0; b < half; ++b) {
      usize j = b % P, g = b / P;
      Cx<F> x0 = src[b], x1 = cmul(src[b + half], w[j]);
      dst[g * 2 * P + j] = x0 + x1;
      dst[g * 2 * P + j + P] = x0 - x1;
    }
    std::swap(src, dst);
  }
  if (src != data) std::memcpy((void*)data, (void*)src, n * sizeof(Cx<F>));
  if (do_scale) for (usize i = 0; i < n; ++i) data[i] *= scale;
}

// Generic size-r DFT in F precision with roots from f64 trig narrowed to F.
// Stands in for the Winograd codelets (mixed_radix/traits.rs:39-244), which
// compute the same exact DFT with hand-derived constants.
// Roots of the size-r DFT, w[e] = exp(sign 2 pi i e / r) narrowed to F (w[0] = 1),
// built once per (r, direction) and thread (the reference caches its codelet
// constants statically; caching changes no value, only the host time).
template <class F> static const std::vector<Cx<F>>& dft_roots(usize r, bool inv) {
  static thread_local std::map<std::pair<usize, int>, std::vector<Cx<F>>> cache;
  auto key = std::make_pair(r, (int)inv);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  std::vector<Cx<F>> w(r);
  double sign = inv ? 1.0 : -1.0;
  for (usize e = 0; e < r; ++e) {
    double a = sign * 2.0 * M_PI * (double)e / (double)r;
    w[e] = e == 0 ? Cx<F>(1, 0) : Cx<F>((F)std::cos(a), (F)std::sin(a));
  }
  return cache.emplace(key, std::move(w)).first->second;
}

template <class F> static void small_dft(Cx<F>* x, usize r, bool inv, usize stride = 1) {
  if (r == 1) return;
  Cx<F> tmp[128];
  std::vector<Cx<F>> big;
  Cx<F>* out = tmp;
  if (r > 128) { big.resize(r); out = big.data(); }
  const Cx<F>* w = dft_roots<F>(r, inv).data();
  for (usize k = 0; k < r; ++k) {
    Cx<F> s(0, 0);
    for (usize m = 0; m < r; ++m) s += cmul(x[m * stride], w[(m * k) % r]);
    out[k] = s;
  }
  for (usize k = 0; k < r; ++k) x[k * stride] = out[k];
}

// radix_composite/cache.rs:75-140 (build_composite_twiddles): per stage with
// prev_len P and radix r, arm k (1..r-1) at offset (k-1)*P holds W_{rP}^{k j};
// arm 1 by recurrence in F precision, arm k = arm(k-1) * arm 1 elementwise.
template <class F>
static std::vector<Cx<F>> build_composite_twiddles(const std::vector<usize>& radices, bool inv,
                                                   std::vector<usize>& offsets) {
  double sign = inv ? 1.0 : -1.0;
  std::vector<Cx<F>> all;
  offsets.clear();
  usize P = 1;
  for (usize r : radices) {
    usize L = P * r;
    offsets.push_back(all.size());
    double a = sign * 2.0 * M_PI / (double)L;
    Cx<F> wb((F)std::cos(a), (F)std::sin(a));
    size_t arm1 = all.size();
    Cx<F> tw(1, 0);
    for (usize j = 0; j < P; ++j) { all.push_back(tw); tw = cmul(tw, wb); }
    for (usize k = 2; k < r; ++k) {
      size_t prev = all.size() - P;
      for (usize j = 0; j < P; ++j) all.push_back(cmul(all[prev + j], all[arm1 + j]));
    }
    P = L;
  }
  return all;
}

// radix_composite/core.rs:184-282 (flat_stockham_fused): pass s with prev_len P,
// G = n/(rP): read src[j + g*P + k*G*P], twiddle input k by W_{rP}^{kj}, r-point
// DFT, write dst[g*rP + j + k*P].  Optional pointwise multiply on the last pass.
template <class F>
static void composite_stockham(Cx<F>* data, usize n, const std::vector<usize>& radices, bool inv,
                               const Cx<F>* pointwise) {
  std::vector<usize> offs;
  auto key = std::make_pair(radices, (int)inv);
  auto& cc = tw_cache<F>().comp;
  auto it = cc.find(key);
  if (it == cc.end()) it = cc.emplace(key, build_composite_twiddles<F>(radices, inv, offs)).first;
  offs.clear();
  {
    usize P = 1, acc = 0;
    for (usize r : radices) { offs.push_back(acc); acc += P * (r - 1); P *= r; }
  }
  const std::vector<Cx<F>>& tw = it->second;
  std::vector<Cx<F>> scratch(n);
  Cx<F>* src = data;
  Cx<F>* dst = scratch.data();
  usize P = 1;
  Cx<F> v[64];
  std::vector<Cx<F>> vbig;
  for (size_t s = 0; s < radices.size(); ++s) {
    usize r = radices[s], L = P * r, G = n / L;
    Cx<F>* vv = v;
    if (r > 64) { vbig.resize(r); vv = vbig.data(); }
    const Cx<F>* t = tw.data() + offs[s];
    bool last = (s + 1 == radices.size());
    for (usize g = 0; g < G; ++g)
      for (usize j = 0; j < P; ++j) {
        for (usize k = 0; k < r; ++k) {
          Cx<F> x = src[j + g * P + k * G * P];
          if (k > 0) x = cmul(x, t[(k - 1) * P + j]);
          vv[k] = x;
        }
        small_dft<F>(vv, r, inv);
        for (usize k = 0; k < r; ++k) {
          usize o = g * L + j + k * P;
          dst[o] = (last && pointwise) ? cmul(vv[k], pointwise[o]) : vv[k];
        }
      }
    std::swap(src, dst);
    P = L;
  }
  if (src != data) std::memcpy((void*)data, (void*)src, n * sizeof(Cx<F>));
}

template <class F> static void normalize(Cx<F>* d, usize n) {
  // mixed_radix/scalar/impls.rs:148-150,277-279: multiply by (1/n) computed in F.
  F s = (F)1 / (F)n;
  for (usize i = 0; i < n; ++i) d[i] *= s;
}

template <class F> static void dispatch_inplace(Cx<F>* d, usize n, bool inv, bool norm);

// four_step/mod.rs:58-155 (four_step_fft) with four_step.rs:41-116 twiddle matrix.
template <class F> static void four_step(Cx<F>* data, usize n, bool inv) {
  unsigned k = __builtin_ctzll(n), k1 = k / 2, k2 = k - k1;
  usize n1 = 1ull << k1, n2 = 1ull << k2;
  const auto& tw1 = pow2_table<F>(n1, inv);
  const auto& tw2 = pow2_table<F>(n2, inv);
  auto& fc = tw_cache<F>().four;
  auto key = std::make_pair(n, (int)inv);
  auto it = fc.find(key);
  if (it == fc.end()) {
    // Double recurrence: row 1 = W_N^k by recurrence, row j = row(j-1) * row 1.
    std::vector<double> re(n1 * n2, 0.0), im(n1 * n2, 0.0);
    for (usize q = 0; q < n1; ++q) re[q] = 1.0;
    if (n2 > 1) {
      double a = (inv ? 1.0 : -1.0) * 2.0 * M_PI / (double)n;
      double wr = std::cos(a), wi = std::sin(a), cr = 1, ci = 0;
      for (usize q = 0; q < n1; ++q) {
        re[n1 + q] = cr; im[n1 + q] = ci;
        double nr = cr * wr - ci * wi, ni = cr * wi + ci * wr;
        cr = nr; ci = ni;
      }
      for (usize j = 2; j < n2; ++j)
        for (usize q = 0; q < n1; ++q) {
          double pr = re[(j - 1) * n1 + q], pi = im[(j - 1) * n1 + q];
          double br = re[n1 + q], bi = im[n1 + q];
          re[j * n1 + q] = pr * br - pi * bi;
          im[j * n1 + q] = pr * bi + pi * br;
        }
    }
    std::vector<Cx<F>> t(n1 * n2);
    for (usize i = 0; i < n1 * n2; ++i) t[i] = Cx<F>((F)re[i], (F)im[i]);
    it = fc.emplace(key, std::move(t)).first;
  }
  const std::vector<Cx<F>>& twm = it->second;
  std::vector<Cx<F>> scratch(n);
  // Step 1: scratch[c*n1 + r] = data[r*n2 + c]  (N1 x N2 -> N2 x N1)
  for (usize r = 0; r < n1; ++r)
    for (usize c = 0; c < n2; ++c) scratch[c * n1 + r] = data[r * n2 + c];
  // Step 2: n2 rows of length n1
  for (usize i = 0; i < n2; ++i)
    stockham_pow2<F>(scratch.data() + i * n1, data + i * n1, n1, tw1.data(), 1, false);
  // Step 3: data[c*n2 + r] = scratch[r*n1 + c] * W_N^{r c}
  for (usize r = 0; r < n2; ++r)
    for (usize c = 0; c < n1; ++c) data[c * n2 + r] = cmul(scratch[r * n1 + c], twm[r * n1 + c]);
  // Step 4: n1 rows of length n2
  for (usize i = 0; i < n1; ++i)
    stockham_pow2<F>(data + i * n2, scratch.data() + i * n2, n2, tw2.data(), 1, false);
  // Step 5: natural order (transpose n1 x n2 -> n2 x n1)
  if (n1 == n2) {
    for (usize r = 0; r < n1; ++r)
      for (usize c = r + 1; c < n1; ++c) std::swap(data[r * n1 + c], data[c * n1 + r]);
  } else {
    for (usize r = 0; r < n1; ++r)
      for (usize c = 0; c < n2; ++c) scratch[c * n1 + r] = data[r * n2 + c];
    std::memcpy((void*)data, (void*)scratch.data(), n * sizeof(Cx<F>));
  }
}

// components/good_thomas/mod.rs:37-155 (pfa_fft / pfa_fft_natural_inplace):
// CRT input gather into an n1 x n2 matrix, length-n2 row DFTs, length-n1 column
// DFTs, CRT output scatter (misc.rs:233-256 permutations).
template <class F> static void pfa(Cx<F>* data, usize n1, usize n2, bool inv) {
  usize n = n1 * n2;
  std::vector<usize> ip, op;
  build_pfa_perm(n1, n2, ip, op);
  std::vector<Cx<F>> m(n), col(n1);
  for (usize i = 0; i < n; ++i) m[i] = data[ip[i]];
  for (usize i1 = 0; i1 < n1; ++i1) dispatch_inplace<F>(m.data() + i1 * n2, n2, inv, false);
  for (usize i2 = 0; i2 < n2; ++i2) {
    for (usize i1 = 0; i1 < n1; ++i1) col[i1] = m[i1 * n2 + i2];
    dispatch_inplace<F>(col.data(), n1, inv, false);
    for (usize k1 = 0; k1 < n1; ++k1) data[op[i2 * n1 + k1]] = col[k1];
  }
}

// Forward/inverse used by the Rader convolutions: the reference routes these
// through short Winograd / composite / PFA / full dispatch (convolution.rs:98-144),
// all of which are exact DFTs; here the full dispatch is used.
// Tables of one Rader prime and direction: the generator order and the kernel
// spectra (cyclic, or the half-cyclic pair and its twist).  The reference
// caches the spectra per (p, direction, g^-1) (scalar/rader.rs, caches); here
// once per thread.  Built exactly as the uncached form did, so every value is
// unchanged.
template <class F> struct RaderTables {
  std::vector<usize> order;
  std::vector<Cx<F>> ker, kc, kn, tw;
};

template <class F> static const RaderTables<F>& rader_tables(usize n, bool inv) {
  static thread_local std::map<std::pair<usize, int>, RaderTables<F>> cache;
  auto key = std::make_pair(n, (int)inv);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  RaderTables<F> t;
  usize g = primitive_root(n);
  usize g_inv = inverse_mod(g, n);
  t.order = generator_order(n, g);
  usize L = n - 1;
  double sign = inv ? 1.0 : -1.0;
  if (L >= 1024) {
    // Half-cyclic CRT split (convolution.rs:155-280; spectra scalar/rader.rs:37-91).
    usize m = L / 2;
    t.kc.resize(m);
    t.kn.resize(m);
    t.tw.resize(m);
    double pi_m = M_PI / (double)m;
    usize cur = 1;
    for (usize j = 0; j < m; ++j) {
      double a = sign * 2.0 * M_PI * (double)cur / (double)n;
      t.kc[j] = Cx<F>((F)std::cos(a), (F)std::sin(a));
      cur = (usize)(((unsigned __int128)cur * g_inv) % n);
    }
    for (usize j = 0; j < m; ++j) {
      double a = sign * 2.0 * M_PI * (double)cur / (double)n;
      Cx<F> upper((F)std::cos(a), (F)std::sin(a));
      Cx<F> lower = t.kc[j];
      t.kc[j] = lower + upper;
      double ta = pi_m * (double)j;
      Cx<F> twist((F)std::cos(ta), (F)std::sin(ta));
      t.kn[j] = cmul(lower - upper, twist);
      t.tw[j] = twist;
      cur = (usize)(((unsigned __int128)cur * g_inv) % n);
    }
    dispatch_inplace<F>(t.kc.data(), m, false, false);
    dispatch_inplace<F>(t.kn.data(), m, false, false);
  } else {
    // Full cyclic convolution (convolution.rs:98-144; spectrum scalar/rader.rs:3-19).
    t.ker.resize(L);
    usize cur = 1;
    for (usize q = 0; q < L; ++q) {
      double a = sign * 2.0 * M_PI * (double)cur / (double)n;
      t.ker[q] = Cx<F>((F)std::cos(a), (F)std::sin(a));
      cur = (usize)(((unsigned __int128)cur * g_inv) % n);
    }
    dispatch_inplace<F>(t.ker.data(), L, false, false);
  }
  return cache.emplace(key, std::move(t)).first->second;
}

template <class F> static void rader(Cx<F>* data, usize n, bool inv) {
  const RaderTables<F>& T = rader_tables<F>(n, inv);
  const std::vector<usize>& order = T.order;
  usize L = n - 1;
  Cx<F> x0 = data[0];
  std::vector<Cx<F>> pad(L);
  // gather_sum_slice (rader/mod.rs:125-177)
  Cx<F> sum(0, 0);
  for (usize i = 0; i < L; ++i) sum += data[1 + i];
  for (usize q = 0; q < L; ++q) pad[q] = data[order[q]];
  if (L >= 1024) {
    // Half-cyclic CRT split (convolution.rs:155-280).
    usize m = L / 2;
    const std::vector<Cx<F>>& kc = T.kc;
    const std::vector<Cx<F>>& kn = T.kn;
    const std::vector<Cx<F>>& tw = T.tw;
    Cx<F>* first = pad.data();
    Cx<F>* second = pad.data() + m;
    for (usize j = 0; j < m; ++j) {
      Cx<F> a = first[j], b = second[j];
      first[j] = a + b;
      second[j] = cmul(a - b, tw[j]);
    }
    dispatch_inplace<F>(first, m, false, false);
    for (usize j = 0; j < m; ++j) first[j] = cmul(first[j], kc[j]);
    dispatch_inplace<F>(first, m, true, true);
    dispatch_inplace<F>(second, m, false, false);
    for (usize j = 0; j < m; ++j) second[j] = cmul(second[j], kn[j]);
    dispatch_inplace<F>(second, m, true, true);
    F half = (F)0.5;
    for (usize j = 0; j < m; ++j) {
      Cx<F> c = first[j];
      Cx<F> v = second[j], t = tw[j];
      Cx<F> nn(v.real() * t.real() + v.imag() * t.imag(), v.imag() * t.real() - v.real() * t.imag());
      first[j] = (c + nn) * half;
      second[j] = (c - nn) * half;
    }
  } else {
    // Full cyclic convolution (convolution.rs:98-144).
    const std::vector<Cx<F>>& ker = T.ker;
    dispatch_inplace<F>(pad.data(), L, false, false);
    for (usize q = 0; q < L; ++q) pad[q] = cmul(pad[q], ker[q]);
    dispatch_inplace<F>(pad.data(), L, true, true);
  }
  // scatter_slice (rader/mod.rs:180-212)
  data[0] = x0 + sum;
  for (usize q = 0; q < L; ++q) data[inverse_generator_order_at(order, q)] = x0 + pad[q];
}

// mixed_radix/dispatch.rs:26-132 (dispatch_inplace + try_power_of_two_fast_path)
template <class F> static void dispatch_inplace(Cx<F>* d, usize n, bool inv, bool norm) {
  int s = dispatch_strategy(n);
  switch (s) {
    case kNoop:
    case kUntransformed:
      return;
    case kFourStep:
      four_step<F>(d, n, inv);
      if (inv && norm) normalize(d, n);
      return;
    case kStockham: {
      const auto& tw = pow2_table<F>(n, inv);
      std::vector<Cx<F>> scratch(n);
      stockham_pow2<F>(d, scratch.data(), n, tw.data(), (F)1 / (F)n, inv && norm);
      return;
    }
    case kWinograd:
      small_dft<F>(d, n, inv);
      if (inv && norm) normalize(d, n);
      return;
    case kPfaStatic:
    case kPfaGeneric: {
      usize n1, n2;
      coprime_factors(n, n1, n2);
      pfa<F>(d, n1, n2, inv);
      if (inv && norm) normalize(d, n);
      return;
    }
    case kComposite: {
      std::vector<usize> r;
      prime23_radices(n, r);
      composite_stockham<F>(d, n, r, inv, nullptr);
      if (inv && norm) normalize(d, n);  // radix_composite/mod.rs:44-75 normalize_scalar
      return;
    }
    case kRaderFull:
    case kRaderHalf:
      rader<F>(d, n, inv);
      if (inv && norm) normalize(d, n);
      return;
  }
}

// Lane parallelism: the reference runs Rayon par_chunks_mut over lanes once the
// lane set exceeds 32768 elements (plan/fft/dimension_3d.rs:48,224-228).
static const usize kRayonThreshold = 32768;

template <class F>
static void lanes_contiguous(Cx<F>* d, usize n, usize lanes, bool inv, int threads) {
  bool par = n * lanes > kRayonThreshold && threads != 1;
#pragma omp parallel for schedule(dynamic, 1) if (par) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (long long l = 0; l < (long long)lanes; ++l) dispatch_inplace<F>(d + (usize)l * n, n, inv, inv);
}

// plan/fft/dimension_2d.rs:77-227: rows (axis 1, contiguous) then columns (axis 0,
// via 32x32 tiled transpose into scratch); inverse in reverse order, each axis
// normalized by 1/n_axis.
template <class F> static void plan2d(Cx<F>* d, usize nx, usize ny, bool inv, int threads) {
  auto cols = [&]() {
    std::vector<Cx<F>> s(nx * ny);
    for (usize i = 0; i < nx; ++i)
      for (usize j = 0; j < ny; ++j) s[j * nx + i] = d[i * ny + j];
    lanes_contiguous<F>(s.data(), nx, ny, inv, threads);
    for (usize i = 0; i < nx; ++i)
      for (usize j = 0; j < ny; ++j) d[i * ny + j] = s[j * nx + i];
  };
  if (!inv) {
    if (ny > 1) lanes_contiguous<F>(d, ny, nx, inv, threads);
    if (nx > 1) cols();
  } else {
    if (nx > 1) cols();
    if (ny > 1) lanes_contiguous<F>(d, ny, nx, inv, threads);
  }
}

// plan/fft/dimension_3d.rs:148-335: forward z (contiguous), y (gather [i,k,j]),
// x (gather [j,k,i]); inverse x, y, z; per-axis 1/n on the inverse.
template <class F>
static void plan3d(Cx<F>* d, usize nx, usize ny, usize nz, bool inv, int threads) {
  const usize T = 32;  // GATHER_TILE (dimension_3d.rs:54)
  auto axis2 = [&]() { if (nz > 1) lanes_contiguous<F>(d, nz, nx * ny, inv, threads); };
  auto axis1 = [&]() {
    if (ny <= 1) return;
    std::vector<Cx<F>> s(nx * ny * nz);
    for (usize i = 0; i < nx; ++i)
      for (usize jt = 0; jt < ny; jt += T)
        for (usize kt = 0; kt < nz; kt += T)
          for (usize j = jt; j < std::min(jt + T, ny); ++j)
            for (usize k = kt; k < std::min(kt + T, nz); ++k)
              s[(i * nz + k) * ny + j] = d[(i * ny + j) * nz + k];
    lanes_contiguous<F>(s.data(), ny, nx * nz, inv, threads);
    for (usize i = 0; i < nx; ++i)
      for (usize jt = 0; jt < ny; jt += T)
        for (usize kt = 0; kt < nz; kt += T)
          for (usize j = jt; j < std::min(jt + T, ny); ++j)
            for (usize k = kt; k < std::min(kt + T, nz); ++k)
              d[(i * ny + j) * nz + k] = s[(i * nz + k) * ny + j];
  };
  auto axis0 = [&]() {
    if (nx <= 1) return;
    std::vector<Cx<F>> s(nx * ny * nz);
    for (usize i = 0; i < nx; ++i)
      for (usize jt = 0; jt < ny; jt += T)
        for (usize kt = 0; kt < nz; kt += T)
          for (usize j = jt; j < std::min(jt + T, ny); ++j)
            for (usize k = kt; k < std::min(kt + T, nz); ++k)
              s[(j * nz + k) * nx + i] = d[(i * ny + j) * nz + k];
    lanes_contiguous<F>(s.data(), nx, ny * nz, inv, threads);
    for (usize i = 0; i < nx; ++i)
      for (usize jt = 0; jt < ny; jt += T)
        for (usize kt = 0; kt < nz; kt += T)
          for (usize j = jt; j < std::min(jt + T, ny); ++j)
            for (usize k = kt; k < std::min(kt + T, nz); ++k)
              d[(i * ny + j) * nz + k] = s[(j * nz + k) * nx + i];
  };
  if (!inv) { axis2(); axis1(); axis0(); }
  else { axis0(); axis1(); axis2(); }
}

// kernel/direct.rs:147-244 (dft_forward / dft_inverse) evaluated in long double
// with exact integer phase reduction (k*j mod n), used as independent truth.
static void direct_dft(const double* in, double* out, usize n, bool inv) {
  long double sign = inv ? 1.0L : -1.0L;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (usize k = 0; k < n; ++k) {
    long double sr = 0, si = 0;
    for (usize j = 0; j < n; ++j) {
      usize e = (usize)(((unsigned __int128)k * j) % n);
      long double a = sign * two_pi * (long double)e / (long double)n;
      long double c = cosl(a), s = sinl(a);
      long double xr = in[2 * j], xi = in[2 * j + 1];
      sr += xr * c - xi * s;
      si += xr * s + xi * c;
    }
    if (inv) { sr /= (long double)n; si /= (long double)n; }
    out[2 * k] = (double)sr;
    out[2 * k + 1] = (double)si;
  }
}

}  // namespace oracle

// ───────────────────────────── C ABI (ctypes) ─────────────────────────────
using namespace oracle;

extern "C" {

int or_factorize_composite(uint64_t n, uint64_t* out, int cap) {
  std::vector<usize> f;
  if (!factorize_composite(n, f)) return -1;
  if ((int)f.size() > cap) return -2;
  for (size_t i = 0; i < f.size(); ++i) out[i] = f[i];
  return (int)f.size();
}
int or_lower_radix4(const uint64_t* in, int cnt, uint64_t* out) {
  std::vector<usize> v(in, in + cnt);
  auto o = lower_radix2_pairs_to_radix4(v);
  for (size_t i = 0; i < o.size(); ++i) out[i] = o[i];
  return (int)o.size();
}
int or_prime23_radices(uint64_t n, uint64_t* out, int cap) {
  std::vector<usize> r;
  if (!prime23_radices(n, r)) return -1;
  if ((int)r.size() > cap) return -2;
  for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
  return (int)r.size();
}
int or_coprime_factors(uint64_t n, uint64_t* n1, uint64_t* n2) {
  usize a = 0, b = 0;
  if (!coprime_factors(n, a, b)) return 0;
  *n1 = a; *n2 = b;
  return 1;
}
int or_is_prime(uint64_t n) { return is_prime(n) ? 1 : 0; }
int or_prime_factors_all(uint64_t n, uint64_t* out, int cap) {
  auto f = prime_factors_all(n);
  if ((int)f.size() > cap) return -2;
  for (size_t i = 0; i < f.size(); ++i) out[i] = f[i];
  return (int)f.size();
}
uint64_t or_mod_pow(uint64_t b, uint64_t e, uint64_t m) { return mod_pow(b, e, m); }
uint64_t or_modular_inverse(uint64_t a, uint64_t m) { return modular_inverse(a, m); }
uint64_t or_primitive_root(uint64_t p) { return primitive_root(p); }
uint64_t or_primitive_root_dynamic(uint64_t p) { return primitive_root_dynamic(p); }
uint64_t or_inverse_mod(uint64_t a, uint64_t m) { return inverse_mod(a, m); }
void or_generator_order(uint64_t p, uint64_t g, uint64_t* out) {
  auto o = generator_order(p, g);
  for (size_t i = 0; i < o.size(); ++i) out[i] = o[i];
}
void or_inverse_generator_order(uint64_t p, uint64_t g, uint64_t* out) {
  auto o = generator_order(p, g);
  for (usize q = 0; q < p - 1; ++q) out[q] = inverse_generator_order_at(o, q);
}
void or_pfa_perm(uint64_t n1, uint64_t n2, uint64_t* in_perm, uint64_t* out_perm) {
  std::vector<usize> a, b;
  build_pfa_perm(n1, n2, a, b);
  for (size_t i = 0; i < a.size(); ++i) { in_perm[i] = a[i]; out_perm[i] = b[i]; }
}
int or_is_short_winograd(uint64_t n) { return is_short_winograd(n) ? 1 : 0; }
int or_has_static_coprime_codelet(uint64_t n1, uint64_t n2) {
  return has_static_coprime_codelet(n1, n2) ? 1 : 0;
}
int or_dispatch_strategy(uint64_t n) { return dispatch_strategy(n); }
void or_four_step_split(uint64_t n, uint64_t* n1, uint64_t* n2) {
  unsigned k = __builtin_ctzll(n), k1 = k / 2;
  *n1 = 1ull << k1;
  *n2 = 1ull << (k - k1);
}
void or_twiddle_table_f64(uint64_t n, double sign, double* out) {
  auto t = build_twiddle_table<double>(n, sign);
  for (size_t i = 0; i < t.size(); ++i) { out[2 * i] = t[i].real(); out[2 * i + 1] = t[i].imag(); }
}

// Float entry points.  Buffers are interleaved (re, im).  `inverse` runs the
// normalized inverse of the reference plans (FftwCompatible, 1/N).
void or_fft1d_c128(double* d, uint64_t n, uint64_t lanes, int inverse, int threads) {
  lanes_contiguous<double>((Cx<double>*)d, n, lanes, inverse != 0, threads);
}
void or_fft1d_c64(float* d, uint64_t n, uint64_t lanes, int inverse, int threads) {
  lanes_contiguous<float>((Cx<float>*)d, n, lanes, inverse != 0, threads);
}
// Unnormalized single-lane dispatch (forward_inplace / inverse_inplace_unnorm).
void or_dispatch_c128(double* d, uint64_t n, int inverse, int normalize) {
  dispatch_inplace<double>((Cx<double>*)d, n, inverse != 0, normalize != 0);
}
void or_dispatch_c64(float* d, uint64_t n, int inverse, int normalize) {
  dispatch_inplace<float>((Cx<float>*)d, n, inverse != 0, normalize != 0);
}
void or_fft2d_c128(double* d, uint64_t nx, uint64_t ny, uint64_t batch, int inverse, int threads) {
  for (usize b = 0; b < batch; ++b) plan2d<double>((Cx<double>*)d + b * nx * ny, nx, ny, inverse != 0, threads);
}
void or_fft2d_c64(float* d, uint64_t nx, uint64_t ny, uint64_t batch, int inverse, int threads) {
  for (usize b = 0; b < batch; ++b) plan2d<float>((Cx<float>*)d + b * nx * ny, nx, ny, inverse != 0, threads);
}
void or_fft3d_c128(double* d, uint64_t nx, uint64_t ny, uint64_t nz, int inverse, int threads) {
  plan3d<double>((Cx<double>*)d, nx, ny, nz, inverse != 0, threads);
}
void or_fft3d_c64(float* d, uint64_t nx, uint64_t ny, uint64_t nz, int inverse, int threads) {
  plan3d<float>((Cx<float>*)d, nx, ny, nz, inverse != 0, threads);
}
// Uneven batch: lanes of different lengths packed back to back (offsets[i],
// lengths[i]); lengths are spread over threads like the reference's callers do.
void or_fft_uneven_c64(float* d, const uint64_t* offsets, const uint64_t* lengths, uint64_t count,
                       int inverse, int threads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (long long i = 0; i < (long long)count; ++i)
    dispatch_inplace<float>((Cx<float>*)d + offsets[i], lengths[i], inverse != 0, inverse != 0);
}
void or_fft_uneven_c128(double* d, const uint64_t* offsets, const uint64_t* lengths, uint64_t count,
                        int inverse, int threads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (long long i = 0; i < (long long)count; ++i)
    dispatch_inplace<double>((Cx<double>*)d + offsets[i], lengths[i], inverse != 0, inverse != 0);
}
void or_direct_dft(const double* in, double* out, uint64_t n, int inverse) {
  direct_dft(in, out, n, inverse != 0);
}
int or_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
