// afc_butterfly.cuh -- register-resident DFT butterflies for the Stockham engine.
//
// Complex values are interleaved (re, im) pairs held in float2 / double2.
// DFT<R, INV>::run(v) overwrites v[0..R) with its R-point DFT, natural order:
//   forward  y[k] = sum_m v[m] * exp(-2*pi*i*m*k/R)
//   inverse  y[k] = sum_m v[m] * exp(+2*pi*i*m*k/R)   (unnormalized)
// Power-of-two radices (2, 4, 8, 16) use the exact +-1/+-i structure with the
// W8/W16 constants; odd prime radices use the symmetric-pair form
//   a_k = v[k] + v[R-k],  b_k = v[k] - v[R-k]
//   y[m] = v0 + sum_k a_k cos(2pi km/R) -/+ i sum_k b_k sin(2pi km/R).
#pragma once
#include <cuda_runtime.h>
#include "afc_roots.cuh"

namespace afc {

template <class T> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };

template <class C> __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <class C> __device__ __forceinline__ C cmulc(C a, C b) {
  return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <class C, class S> __device__ __forceinline__ C cscale(C a, S s) { return C{a.x * s, a.y * s}; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, class C> __device__ __forceinline__ C rot90(C a) {
  return INV ? C{-a.y, a.x} : C{a.y, -a.x};
}
template <class C> __device__ __forceinline__ C cconj(C a) { return C{a.x, -a.y}; }

template <int R, bool INV> struct DFT;

template <bool INV> struct DFT<2, INV> {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV> struct DFT<4, INV> {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    C s13 = cadd(v[1], v[3]), d13 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  }
};

// exp(sign * 2 pi i * j / 16) for the twiddles inside the 8/16-point butterflies.
template <bool INV, class C> __device__ __forceinline__ C w16mul(C a, int j) {
  using T = decltype(a.x);
  const T c1 = (T)0.9238795325112867, s1 = (T)0.3826834323650898, r2 = (T)0.7071067811865476;
  // forward uses exp(-i theta); inverse exp(+i theta)
  T cs, sn;
  switch (j & 15) {
    case 0: return a;
    case 1: cs = c1; sn = s1; break;
    case 2: cs = r2; sn = r2; break;
    case 3: cs = s1; sn = c1; break;
    case 4: return rot90<INV>(a);
    case 6: cs = -r2; sn = r2; break;
    case 9: cs = -c1; sn = -s1; break;
    default: {
      // not used by the 8/16-point butterflies below
      cs = (T)1; sn = (T)0; break;
    }
  }
  if (!INV) sn = -sn;
  return C{a.x * cs - a.y * sn, a.x * sn + a.y * cs};
}

// 8 = 2 x 4: inner DFT4 over b of v[a + 2b] (a = 0, 1), twiddle W8^{a c}, outer DFT2.
template <bool INV> struct DFT<8, INV> {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    DFT<4, INV>::run(e);
    DFT<4, INV>::run(o);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      C t = w16mul<INV>(o[c], 2 * c);
      v[c] = cadd(e[c], t);
      v[c + 4] = csub(e[c], t);
    }
  }
};

// 16 = 4 x 4: inner DFT4 over b of v[a + 4b], twiddle W16^{a c}, outer DFT4 over a,
// output index c + 4 d.
template <bool INV> struct DFT<16, INV> {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    C z[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
      for (int b = 0; b < 4; ++b) z[a][b] = v[a + 4 * b];
      DFT<4, INV>::run(z[a]);
    }
#pragma unroll
    for (int a = 1; a < 4; ++a)
#pragma unroll
      for (int c = 1; c < 4; ++c) z[a][c] = w16mul<INV>(z[a][c], a * c);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      C col[4] = {z[0][c], z[1][c], z[2][c], z[3][c]};
      DFT<4, INV>::run(col);
#pragma unroll
      for (int d = 0; d < 4; ++d) v[c + 4 * d] = col[d];
    }
  }
};

template <int R> struct OddRoots;
template <> struct OddRoots<3> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return -0.5;
      case 2: return -0.5;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.8660254037844386;
      case 2: return -0.8660254037844386;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<5> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.30901699437494745;
      case 2: return -0.8090169943749475;
      case 3: return -0.8090169943749475;
      case 4: return 0.30901699437494745;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.9510565162951535;
      case 2: return 0.5877852522924731;
      case 3: return -0.5877852522924731;
      case 4: return -0.9510565162951535;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<7> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.6234898018587335;
      case 2: return -0.2225209339563144;
      case 3: return -0.9009688679024191;
      case 4: return -0.9009688679024191;
      case 5: return -0.2225209339563144;
      case 6: return 0.6234898018587335;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.7818314824680298;
      case 2: return 0.9749279121818236;
      case 3: return 0.4338837391175581;
      case 4: return -0.4338837391175581;
      case 5: return -0.9749279121818236;
      case 6: return -0.7818314824680298;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<11> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.8412535328311812;
      case 2: return 0.41541501300188644;
      case 3: return -0.14231483827328514;
      case 4: return -0.6548607339452851;
      case 5: return -0.9594929736144974;
      case 6: return -0.9594929736144974;
      case 7: return -0.6548607339452851;
      case 8: return -0.14231483827328514;
      case 9: return 0.41541501300188644;
      case 10: return 0.8412535328311812;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.5406408174555976;
      case 2: return 0.9096319953545183;
      case 3: return 0.9898214418809327;
      case 4: return 0.7557495743542583;
      case 5: return 0.28173255684142967;
      case 6: return -0.28173255684142967;
      case 7: return -0.7557495743542583;
      case 8: return -0.9898214418809327;
      case 9: return -0.9096319953545183;
      case 10: return -0.5406408174555976;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<13> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.8854560256532099;
      case 2: return 0.5680647467311558;
      case 3: return 0.12053668025532305;
      case 4: return -0.3546048870425356;
      case 5: return -0.7485107481711011;
      case 6: return -0.970941817426052;
      case 7: return -0.970941817426052;
      case 8: return -0.7485107481711011;
      case 9: return -0.3546048870425356;
      case 10: return 0.12053668025532305;
      case 11: return 0.5680647467311558;
      case 12: return 0.8854560256532099;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.46472317204376856;
      case 2: return 0.8229838658936564;
      case 3: return 0.992708874098054;
      case 4: return 0.9350162426854148;
      case 5: return 0.6631226582407952;
      case 6: return 0.23931566428755777;
      case 7: return -0.23931566428755777;
      case 8: return -0.6631226582407952;
      case 9: return -0.9350162426854148;
      case 10: return -0.992708874098054;
      case 11: return -0.8229838658936564;
      case 12: return -0.46472317204376856;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<17> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9324722294043558;
      case 2: return 0.7390089172206591;
      case 3: return 0.44573835577653825;
      case 4: return 0.092268359463302;
      case 5: return -0.2736629900720829;
      case 6: return -0.6026346363792564;
      case 7: return -0.8502171357296141;
      case 8: return -0.9829730996839018;
      case 9: return -0.9829730996839018;
      case 10: return -0.8502171357296141;
      case 11: return -0.6026346363792564;
      case 12: return -0.2736629900720829;
      case 13: return 0.092268359463302;
      case 14: return 0.44573835577653825;
      case 15: return 0.7390089172206591;
      case 16: return 0.9324722294043558;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.3612416661871529;
      case 2: return 0.6736956436465572;
      case 3: return 0.8951632913550623;
      case 4: return 0.9957341762950345;
      case 5: return 0.961825643172819;
      case 6: return 0.7980172272802395;
      case 7: return 0.5264321628773558;
      case 8: return 0.18374951781657034;
      case 9: return -0.18374951781657034;
      case 10: return -0.5264321628773558;
      case 11: return -0.7980172272802395;
      case 12: return -0.961825643172819;
      case 13: return -0.9957341762950345;
      case 14: return -0.8951632913550623;
      case 15: return -0.6736956436465572;
      case 16: return -0.3612416661871529;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<19> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9458172417006346;
      case 2: return 0.7891405093963936;
      case 3: return 0.5469481581224269;
      case 4: return 0.24548548714079915;
      case 5: return -0.08257934547233232;
      case 6: return -0.4016954246529695;
      case 7: return -0.6772815716257411;
      case 8: return -0.8794737512064891;
      case 9: return -0.9863613034027223;
      case 10: return -0.9863613034027223;
      case 11: return -0.8794737512064891;
      case 12: return -0.6772815716257411;
      case 13: return -0.4016954246529695;
      case 14: return -0.08257934547233232;
      case 15: return 0.24548548714079915;
      case 16: return 0.5469481581224269;
      case 17: return 0.7891405093963936;
      case 18: return 0.9458172417006346;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.3246994692046835;
      case 2: return 0.6142127126896678;
      case 3: return 0.8371664782625285;
      case 4: return 0.9694002659393304;
      case 5: return 0.9965844930066698;
      case 6: return 0.9157733266550574;
      case 7: return 0.7357239106731316;
      case 8: return 0.47594739303707356;
      case 9: return 0.1645945902807339;
      case 10: return -0.1645945902807339;
      case 11: return -0.47594739303707356;
      case 12: return -0.7357239106731316;
      case 13: return -0.9157733266550574;
      case 14: return -0.9965844930066698;
      case 15: return -0.9694002659393304;
      case 16: return -0.8371664782625285;
      case 17: return -0.6142127126896678;
      case 18: return -0.3246994692046835;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<23> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9629172873477992;
      case 2: return 0.8544194045464886;
      case 3: return 0.6825531432186541;
      case 4: return 0.46006503773115215;
      case 5: return 0.20345601305263378;
      case 6: return -0.06824241336467098;
      case 7: return -0.33487961217098616;
      case 8: return -0.5766803221148672;
      case 9: return -0.7757112907044198;
      case 10: return -0.917211301505453;
      case 11: return -0.9906859460363308;
      case 12: return -0.9906859460363308;
      case 13: return -0.917211301505453;
      case 14: return -0.7757112907044198;
      case 15: return -0.5766803221148672;
      case 16: return -0.33487961217098616;
      case 17: return -0.06824241336467098;
      case 18: return 0.20345601305263378;
      case 19: return 0.46006503773115215;
      case 20: return 0.6825531432186541;
      case 21: return 0.8544194045464886;
      case 22: return 0.9629172873477992;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.2697967711570243;
      case 2: return 0.5195839500354336;
      case 3: return 0.7308359642781241;
      case 4: return 0.8878852184023752;
      case 5: return 0.9790840876823229;
      case 6: return 0.9976687691905392;
      case 7: return 0.9422609221188205;
      case 8: return 0.816969893010442;
      case 9: return 0.6310879443260528;
      case 10: return 0.39840108984624145;
      case 11: return 0.1361666490962466;
      case 12: return -0.1361666490962466;
      case 13: return -0.39840108984624145;
      case 14: return -0.6310879443260528;
      case 15: return -0.816969893010442;
      case 16: return -0.9422609221188205;
      case 17: return -0.9976687691905392;
      case 18: return -0.9790840876823229;
      case 19: return -0.8878852184023752;
      case 20: return -0.7308359642781241;
      case 21: return -0.5195839500354336;
      case 22: return -0.2697967711570243;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<29> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9766205557100867;
      case 2: return 0.907575419670957;
      case 3: return 0.7960930657056438;
      case 4: return 0.6473862847818277;
      case 5: return 0.46840844069979015;
      case 6: return 0.2675283385292208;
      case 7: return 0.054138908585417526;
      case 8: return -0.16178199655276473;
      case 9: return -0.37013815533991434;
      case 10: return -0.5611870653623824;
      case 11: return -0.7259954919231308;
      case 12: return -0.8568571761675893;
      case 13: return -0.9476531711828025;
      case 14: return -0.9941379571543596;
      case 15: return -0.9941379571543596;
      case 16: return -0.9476531711828025;
      case 17: return -0.8568571761675893;
      case 18: return -0.7259954919231308;
      case 19: return -0.5611870653623824;
      case 20: return -0.37013815533991434;
      case 21: return -0.16178199655276473;
      case 22: return 0.054138908585417526;
      case 23: return 0.2675283385292208;
      case 24: return 0.46840844069979015;
      case 25: return 0.6473862847818277;
      case 26: return 0.7960930657056438;
      case 27: return 0.907575419670957;
      case 28: return 0.9766205557100867;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.21497044021102407;
      case 2: return 0.4198891015602646;
      case 3: return 0.6051742151937651;
      case 4: return 0.7621620551276365;
      case 5: return 0.8835120444460229;
      case 6: return 0.9635499925192229;
      case 7: return 0.9985334138511238;
      case 8: return 0.9868265225415261;
      case 9: return 0.9289767198167914;
      case 10: return 0.8276889981568906;
      case 11: return 0.6876994588534233;
      case 12: return 0.5155538571770217;
      case 13: return 0.31930153013597995;
      case 14: return 0.10811901842394177;
      case 15: return -0.10811901842394177;
      case 16: return -0.31930153013597995;
      case 17: return -0.5155538571770217;
      case 18: return -0.6876994588534233;
      case 19: return -0.8276889981568906;
      case 20: return -0.9289767198167914;
      case 21: return -0.9868265225415261;
      case 22: return -0.9985334138511238;
      case 23: return -0.9635499925192229;
      case 24: return -0.8835120444460229;
      case 25: return -0.7621620551276365;
      case 26: return -0.6051742151937651;
      case 27: return -0.4198891015602646;
      case 28: return -0.21497044021102407;
      default: return 0.0;
    }
  }
};
template <> struct OddRoots<31> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9795299412524945;
      case 2: return 0.9189578116202306;
      case 3: return 0.8207634412072763;
      case 4: return 0.6889669190756865;
      case 5: return 0.5289640103269625;
      case 6: return 0.3473052528448203;
      case 7: return 0.15142777750457667;
      case 8: return -0.05064916883871271;
      case 9: return -0.25065253225872053;
      case 10: return -0.4403941515576343;
      case 11: return -0.6121059825476628;
      case 12: return -0.7587581226927909;
      case 13: return -0.8743466161445821;
      case 14: return -0.9541392564000488;
      case 15: return -0.9948693233918952;
      case 16: return -0.9948693233918952;
      case 17: return -0.9541392564000488;
      case 18: return -0.8743466161445821;
      case 19: return -0.7587581226927909;
      case 20: return -0.6121059825476628;
      case 21: return -0.4403941515576343;
      case 22: return -0.25065253225872053;
      case 23: return -0.05064916883871271;
      case 24: return 0.15142777750457667;
      case 25: return 0.3473052528448203;
      case 26: return 0.5289640103269625;
      case 27: return 0.6889669190756865;
      case 28: return 0.8207634412072763;
      case 29: return 0.9189578116202306;
      case 30: return 0.9795299412524945;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.2012985200886601;
      case 2: return 0.39435585511331855;
      case 3: return 0.5712682150947923;
      case 4: return 0.72479278722912;
      case 5: return 0.8486442574947509;
      case 6: return 0.9377521321470804;
      case 7: return 0.9884683243281114;
      case 8: return 0.9987165071710528;
      case 9: return 0.9680771188662043;
      case 10: return 0.8978045395707417;
      case 11: return 0.7907757369376985;
      case 12: return 0.6513724827222223;
      case 13: return 0.48530196253108104;
      case 14: return 0.29936312297335793;
      case 15: return 0.10116832198743218;
      case 16: return -0.10116832198743218;
      case 17: return -0.29936312297335793;
      case 18: return -0.48530196253108104;
      case 19: return -0.6513724827222223;
      case 20: return -0.7907757369376985;
      case 21: return -0.8978045395707417;
      case 22: return -0.9680771188662043;
      case 23: return -0.9987165071710528;
      case 24: return -0.9884683243281114;
      case 25: return -0.9377521321470804;
      case 26: return -0.8486442574947509;
      case 27: return -0.72479278722912;
      case 28: return -0.5712682150947923;
      case 29: return -0.39435585511331855;
      case 30: return -0.2012985200886601;
      default: return 0.0;
    }
  }
};

// Odd prime radix by symmetric pairs; roots tabulated above (cos/sin of 2 pi j / R).
template <int R, bool INV> struct DFT {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    constexpr int H = (R - 1) / 2;
    C a[H], b[H];
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      a[k - 1] = cadd(v[k], v[R - k]);
      b[k - 1] = csub(v[k], v[R - k]);
    }
    C x0 = v[0];
    C y0 = x0;
#pragma unroll
    for (int k = 0; k < H; ++k) y0 = cadd(y0, a[k]);
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      C re = x0, im = C{(T)0, (T)0};
#pragma unroll
      for (int k = 1; k <= H; ++k) {
        const int e = (k * m) % R;
        const T c = (T)OddRoots<R>::c(e);
        const T s = (T)OddRoots<R>::s(e);
        re.x += a[k - 1].x * c;
        re.y += a[k - 1].y * c;
        im.x += b[k - 1].x * s;
        im.y += b[k - 1].y * s;
      }
      // forward: y[m] = re - i*im, y[R-m] = re + i*im ; inverse swaps.
      C mi = C{im.y, -im.x};  // -i * im
      if (INV) {
        v[m] = csub(re, mi);
        v[R - m] = cadd(re, mi);
      } else {
        v[m] = cadd(re, mi);
        v[R - m] = csub(re, mi);
      }
    }
    v[0] = y0;
  }
};

// Composite radix R = R1 x R2 (6, 9, 10, 12, 14, 15) as nested butterflies:
// input m = a + R1 b, output k = c + R2 d; R1 DFTs of size R2 over b, twiddle
// W_R^{a c}, R2 DFTs of size R1 over a (the same index split as DFT<16>).
template <int R1, int R2, bool INV> struct DFTNest {
  template <class C> __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    constexpr int R = R1 * R2;
    C z[R1][R2];
#pragma unroll
    for (int a = 0; a < R1; ++a) {
#pragma unroll
      for (int b = 0; b < R2; ++b) z[a][b] = v[a + R1 * b];
      DFT<R2, INV>::run(z[a]);
    }
#pragma unroll
    for (int a = 1; a < R1; ++a)
#pragma unroll
      for (int c = 1; c < R2; ++c) {
        const T cs = (T)CompRoots<R>::c(a * c), sn = (T)CompRoots<R>::s(a * c);
        const C x = z[a][c];
        // forward multiplies by exp(-i theta) = cs - i sn, inverse by cs + i sn
        z[a][c] = INV ? C{x.x * cs - x.y * sn, x.y * cs + x.x * sn} : C{x.x * cs + x.y * sn, x.y * cs - x.x * sn};
      }
#pragma unroll
    for (int c = 0; c < R2; ++c) {
      C col[R1];
#pragma unroll
      for (int a = 0; a < R1; ++a) col[a] = z[a][c];
      DFT<R1, INV>::run(col);
#pragma unroll
      for (int d = 0; d < R1; ++d) v[c + R2 * d] = col[d];
    }
  }
};
template <bool INV> struct DFT<6, INV> : DFTNest<3, 2, INV> {};
template <bool INV> struct DFT<9, INV> : DFTNest<3, 3, INV> {};
template <bool INV> struct DFT<10, INV> : DFTNest<5, 2, INV> {};
template <bool INV> struct DFT<12, INV> : DFTNest<4, 3, INV> {};
template <bool INV> struct DFT<14, INV> : DFTNest<7, 2, INV> {};
template <bool INV> struct DFT<15, INV> : DFTNest<5, 3, INV> {};

}  // namespace afc
