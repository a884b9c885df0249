// afc_roots.cuh -- generated by gen_roots.py: cos / sin (2 pi e / R) for the
// composite radices of the nested butterflies.
#pragma once

namespace afc {

template <int R> struct CompRoots;
template <> struct CompRoots<6> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.5;
      case 2: return -0.5;
      case 3: return -1.0;
      case 4: return -0.5;
      case 5: return 0.5;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.8660254037844386;
      case 2: return 0.8660254037844386;
      case 3: return 2.155640679034182e-59;
      case 4: return -0.8660254037844386;
      case 5: return -0.8660254037844386;
      default: return 0.0;
    }
  }
};
template <> struct CompRoots<9> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.766044443118978;
      case 2: return 0.17364817766693036;
      case 3: return -0.5;
      case 4: return -0.9396926207859084;
      case 5: return -0.9396926207859084;
      case 6: return -0.5;
      case 7: return 0.17364817766693036;
      case 8: return 0.766044443118978;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.6427876096865394;
      case 2: return 0.984807753012208;
      case 3: return 0.8660254037844386;
      case 4: return 0.3420201433256687;
      case 5: return -0.3420201433256687;
      case 6: return -0.8660254037844386;
      case 7: return -0.984807753012208;
      case 8: return -0.6427876096865394;
      default: return 0.0;
    }
  }
};
template <> struct CompRoots<10> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.8090169943749475;
      case 2: return 0.30901699437494745;
      case 3: return -0.30901699437494745;
      case 4: return -0.8090169943749475;
      case 5: return -1.0;
      case 6: return -0.8090169943749475;
      case 7: return -0.30901699437494745;
      case 8: return 0.30901699437494745;
      case 9: return 0.8090169943749475;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.5877852522924731;
      case 2: return 0.9510565162951535;
      case 3: return 0.9510565162951535;
      case 4: return 0.5877852522924731;
      case 5: return 2.155640679034182e-59;
      case 6: return -0.5877852522924731;
      case 7: return -0.9510565162951535;
      case 8: return -0.9510565162951535;
      case 9: return -0.5877852522924731;
      default: return 0.0;
    }
  }
};
template <> struct CompRoots<12> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.8660254037844386;
      case 2: return 0.5;
      case 3: return 6.378690523721779e-60;
      case 4: return -0.5;
      case 5: return -0.8660254037844386;
      case 6: return -1.0;
      case 7: return -0.8660254037844386;
      case 8: return -0.5;
      case 9: return -7.151699326031473e-59;
      case 10: return 0.5;
      case 11: return 0.8660254037844386;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.5;
      case 2: return 0.8660254037844386;
      case 3: return 1.0;
      case 4: return 0.8660254037844386;
      case 5: return 0.5;
      case 6: return 2.155640679034182e-59;
      case 7: return -0.5;
      case 8: return -0.8660254037844386;
      case 9: return -1.0;
      case 10: return -0.8660254037844386;
      case 11: return -0.5;
      default: return 0.0;
    }
  }
};
template <> struct CompRoots<14> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9009688679024191;
      case 2: return 0.6234898018587335;
      case 3: return 0.2225209339563144;
      case 4: return -0.2225209339563144;
      case 5: return -0.6234898018587335;
      case 6: return -0.9009688679024191;
      case 7: return -1.0;
      case 8: return -0.9009688679024191;
      case 9: return -0.6234898018587335;
      case 10: return -0.2225209339563144;
      case 11: return 0.2225209339563144;
      case 12: return 0.6234898018587335;
      case 13: return 0.9009688679024191;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.4338837391175581;
      case 2: return 0.7818314824680298;
      case 3: return 0.9749279121818236;
      case 4: return 0.9749279121818236;
      case 5: return 0.7818314824680298;
      case 6: return 0.4338837391175581;
      case 7: return 2.155640679034182e-59;
      case 8: return -0.4338837391175581;
      case 9: return -0.7818314824680298;
      case 10: return -0.9749279121818236;
      case 11: return -0.9749279121818236;
      case 12: return -0.7818314824680298;
      case 13: return -0.4338837391175581;
      default: return 0.0;
    }
  }
};
template <> struct CompRoots<15> {
  __host__ __device__ __forceinline__ static constexpr double c(int e) {
    switch (e) {
      case 0: return 1.0;
      case 1: return 0.9135454576426009;
      case 2: return 0.6691306063588582;
      case 3: return 0.30901699437494745;
      case 4: return -0.10452846326765347;
      case 5: return -0.5;
      case 6: return -0.8090169943749475;
      case 7: return -0.9781476007338057;
      case 8: return -0.9781476007338057;
      case 9: return -0.8090169943749475;
      case 10: return -0.5;
      case 11: return -0.10452846326765347;
      case 12: return 0.30901699437494745;
      case 13: return 0.6691306063588582;
      case 14: return 0.9135454576426009;
      default: return 0.0;
    }
  }
  __host__ __device__ __forceinline__ static constexpr double s(int e) {
    switch (e) {
      case 0: return 0.0;
      case 1: return 0.4067366430758002;
      case 2: return 0.7431448254773942;
      case 3: return 0.9510565162951535;
      case 4: return 0.9945218953682733;
      case 5: return 0.8660254037844386;
      case 6: return 0.5877852522924731;
      case 7: return 0.20791169081775934;
      case 8: return -0.20791169081775934;
      case 9: return -0.5877852522924731;
      case 10: return -0.8660254037844386;
      case 11: return -0.9945218953682733;
      case 12: return -0.9510565162951535;
      case 13: return -0.7431448254773942;
      case 14: return -0.4067366430758002;
      default: return 0.0;
    }
  }
};

}  // namespace afc
