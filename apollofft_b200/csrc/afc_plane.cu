// afc_plane.cu -- the last two axes of a C2C transform whose planes are
// 256 x 256, in one pass over HBM (sm_100a thread-block clusters).
//
// A 3D transform as three axis passes reads and writes the volume in HBM three
// times.  Here a cluster of CS CTAs (one per SM) owns one plane at a time (the
// outermost index; 1 MiB in complex128): CTA `rank` copies rows
// [R rank, R rank + R) of the plane (R = 256 / CS) into its shared memory with
// one bulk copy, transforms them along the row (z), and after a cluster
// barrier reads the columns [R rank, R rank + R) of every row from the other
// CTAs' shared memory (distributed shared memory, ld.shared::cluster),
// transforms them along the column (y) and writes them back with one tensor
// store.  The plane never round-trips through L2 or HBM between its two
// axes, so with the leading axis as one more TMA pass a 3D transform reads
// and writes the volume twice.  Loads use no cluster multicast.
//
// Each 256-point transform is two radix-16 stages in registers (apollo-fft's
// Stockham radix-16 stage, crates/apollo-fft/src/application/execution/
// kernel/radix_stages.rs): stage 0 without twiddles writes element 16 t + r
// of the padded lane (element i at i + i / 16, lane stride 273), stage 1
// multiplies by the axis table's twiddles (r - 1) 16 + t and leaves element
// t + 16 r.  Thread t < 16 of a lane owns butterfly t in both stages, B = R / 16
// lanes per thread.  Per plane and CTA:
//
//   rows (linear, from HBM)  --z stage 0-->  padded rows  --z stage 1-->  padded rows
//   cluster barrier 1 (every CTA's rows are transformed)
//   remote padded rows  --y stage 0 (registers)-->
//   cluster barrier 2 (no CTA reads this plane's rows any more)
//   --> padded columns  --y stage 1-->  [y][column] linear  --tensor store-->  HBM
//
// With two plane buffers per CTA the next plane's rows load while this one is
// transformed.  Every wait on a copy is bounded; a CTA whose wait timed out
// sets the error word and stops copying, but keeps arriving at every cluster
// barrier (which has no timeout) so that no CTA of its cluster is left waiting.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "afc_async.cuh"
#include "afc_engine.cuh"
#include "afc_internal.h"

namespace afc {

constexpr int kPlaneLd = 273;  // padded 256-point lane: element i at i + i / 16
constexpr int kPlaneThreads = 256;
constexpr int kPlaneTw = 240;  // second-stage twiddles of one axis: (r - 1) 16 + k, 1 <= r < 16, k < 16

template <class T> struct PlaneArgs {
  using C = typename CT<T>::type;
  CUtensorMap tmo;  // output as [2 x 256 scalars, 256 rows, planes], box [2 R, 256, 1]
  const C* in;      // planes of 256 rows (y) x 256 columns (z), contiguous
  const C* twz;     // second-stage twiddles of the row (z) and column (y) axes
  const C* twy;
  long long planes;
  T scale;  // applied to the column stage's outputs
  unsigned* err;
};

template <class T, int CS, int NBUF> struct PlaneGeo {
  using C = typename CT<T>::type;
  static constexpr int R = 256 / CS;  // rows, then columns, per CTA
  static constexpr int B = R / 16;    // lanes per thread and stage
  static constexpr int buf_elems = R * kPlaneLd;  // >= R x 256, the store layout
  static constexpr size_t buf_bytes = (size_t)buf_elems * sizeof(C);
  static_assert(buf_bytes % 128 == 0, "plane buffers must stay on 128-byte boundaries");
  static constexpr size_t smem = NBUF * buf_bytes + 2 * kPlaneTw * sizeof(C) + 2 * sizeof(unsigned long long);
};

template <class T, bool INV, int CS, int NBUF, int MINB>
__global__ void __launch_bounds__(kPlaneThreads, MINB) plane_kernel(const __grid_constant__ PlaneArgs<T> a) {
  using C = typename CT<T>::type;
  using G = PlaneGeo<T, CS, NBUF>;
  constexpr int R = G::R, B = G::B, LD = kPlaneLd;
  extern __shared__ __align__(128) unsigned char smraw[];
  C* const buf0 = reinterpret_cast<C*>(smraw);
  C* const twz = buf0 + NBUF * G::buf_elems;
  C* const twy = twz + kPlaneTw;
  unsigned long long* const bars = reinterpret_cast<unsigned long long*>(twy + kPlaneTw);
  const int tid = threadIdx.x;
  // a misaligned block is the same for every CTA of the launch: none copies
  // and none reaches a cluster barrier
  if (smem_u32(smraw) & 127) {
    if (tid == 0) atomicExch(a.err, 1u);
    return;
  }
  const unsigned rank = cluster_rank();
  const long long cid = cluster_id(), ncl = cluster_count();
  constexpr unsigned rows_bytes = (unsigned)(R * 256 * sizeof(C));
  auto load = [&](long long p, int b) {  // thread 0: this CTA's rows of plane p into buffer b
    mbar_expect_tx(&bars[b], rows_bytes);
    bulk_load(buf0 + b * G::buf_elems, a.in + (p * 256 + (long long)R * rank) * 256, rows_bytes, &bars[b]);
  };
  if (tid == 0) {
    for (int b = 0; b < NBUF; ++b) mbar_init(&bars[b], 1);
    fence_proxy_async();
    if (cid < a.planes) load(cid, 0);
  }
  for (int i = tid; i < kPlaneTw; i += kPlaneThreads) {
    twz[i] = a.twz[i];
    twy[i] = a.twy[i];
  }
  __syncthreads();
  const T sc = a.scale;
  const int t = tid & 15;   // row stages: butterfly t of lanes (tid / 16) + 16 b
  const int tc = tid >> 4;  // column stages: butterfly tc of columns (tid % 16) + 16 b
  bool bad = false;
  int it = 0;
  for (long long p = cid; p < a.planes; p += ncl, ++it) {
    const int cb = NBUF == 2 ? (it & 1) : 0;
    C* const cur = buf0 + cb * G::buf_elems;
    const bool pf = NBUF == 2 && p + ncl < a.planes;  // the next plane's rows load during this one
    if (tid == 0 && !bad) {
      bulk_wait_read0();  // the previous plane's store has read its buffer
      if (pf)
        load(p + ncl, cb ^ 1);
      else if (NBUF == 1 && it > 0)
        load(p, 0);
    }
    const bool ok = bad || mbar_wait(&bars[cb], NBUF == 2 ? ((it >> 1) & 1) : (it & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0 && !bad) {
        atomicExch(a.err, 1u);
        if (pf) mbar_wait(&bars[cb ^ 1], ((it + 1) >> 1) & 1);  // let the prefetch land (bounded)
      }
      bad = true;
    }
    C v[B][16];
    // ── rows (z): linear -> padded -> padded, in place ──
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const C* s = cur + ((tid >> 4) + 16 * b) * 256 + t;
#pragma unroll
      for (int r = 0; r < 16; ++r) v[b][r] = s[16 * r];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      DFT<16, INV>::run(v[b]);
      C* d = cur + ((tid >> 4) + 16 * b) * LD + 17 * t;  // outputs 16 t + r (Ns = 1: no twiddles)
#pragma unroll
      for (int r = 0; r < 16; ++r) d[r] = v[b][r];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const C* s = cur + ((tid >> 4) + 16 * b) * LD + t;  // inputs t + 16 r at t + 17 r
#pragma unroll
      for (int r = 0; r < 16; ++r) v[b][r] = s[17 * r];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
#pragma unroll
      for (int r = 1; r < 16; ++r) {
        const C w = twz[(r - 1) * 16 + t];
        v[b][r] = INV ? cmulc(v[b][r], w) : cmul(v[b][r], w);
      }
      DFT<16, INV>::run(v[b]);
      C* d = cur + ((tid >> 4) + 16 * b) * LD + t;  // outputs t + 16 r, padded
#pragma unroll
      for (int r = 0; r < 16; ++r) d[17 * r] = v[b][r];
    }
    cluster_sync_all();  // 1: every CTA's rows of the plane are transformed
    // ── columns (y), stage 0 from the other CTAs' rows ──
    const unsigned base = smem_u32(cur);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int z = R * (int)rank + (tid & 15) + 16 * b;
      const int zoff = z + (z >> 4);
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        // element y = tc + 16 r sits in CTA y / R, row y % R (tc < 16 <= R)
        const unsigned owner = (unsigned)((16 * r) / R);
        const int yl = (16 * r) % R + tc;
        v[b][r] = ld_cluster<C>(cluster_map(base, owner) + (unsigned)((yl * LD + zoff) * (int)sizeof(C)));
      }
      DFT<16, INV>::run(v[b]);
    }
    cluster_sync_all();  // 2: no CTA reads this plane's rows any more
#pragma unroll
    for (int b = 0; b < B; ++b) {
      C* d = cur + ((tid & 15) + 16 * b) * LD + 17 * tc;
#pragma unroll
      for (int r = 0; r < 16; ++r) d[r] = v[b][r];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const C* s = cur + ((tid & 15) + 16 * b) * LD + tc;
#pragma unroll
      for (int r = 0; r < 16; ++r) v[b][r] = s[17 * r];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
#pragma unroll
      for (int r = 1; r < 16; ++r) {
        const C w = twy[(r - 1) * 16 + tc];
        v[b][r] = INV ? cmulc(v[b][r], w) : cmul(v[b][r], w);
      }
      DFT<16, INV>::run(v[b]);
      if (sc != (T)1) {
#pragma unroll
        for (int r = 0; r < 16; ++r) v[b][r] = cscale(v[b][r], sc);
      }
      C* d = cur + tc * R + (tid & 15) + 16 * b;  // element (y = tc + 16 r, column) of the store box
#pragma unroll
      for (int r = 0; r < 16; ++r) d[16 * r * R] = v[b][r];
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0 && !bad) {
      tma_store_3d(&a.tmo, 2 * R * (int)rank, 0, (int)p, cur);
      bulk_commit();
    }
  }
  if (tid == 0 && !bad) bulk_wait0();
}

// ─────────────────────────────── host side ───────────────────────────────

template <class T, bool INV> static const void* plane_kernel_ptr(int cfg) {
  const void* k = nullptr;
  switch (cfg) {
    case 0: k = reinterpret_cast<const void*>(plane_kernel<T, INV, 16, 2, 1>); break;
    case 1: k = reinterpret_cast<const void*>(plane_kernel<T, INV, 16, 1, 2>); break;
    default:
      // clusters of 8: two complex128 plane buffers would not fit
      if constexpr (sizeof(T) == 8)
        k = reinterpret_cast<const void*>(plane_kernel<T, INV, 8, 1, 1>);
      else
        k = reinterpret_cast<const void*>(plane_kernel<T, INV, 8, 2, 1>);
      break;
  }
  return k;
}
static const void* plane_kernel_ptr(bool dbl, bool inv, int cfg) {
  if (dbl) return inv ? plane_kernel_ptr<double, true>(cfg) : plane_kernel_ptr<double, false>(cfg);
  return inv ? plane_kernel_ptr<float, true>(cfg) : plane_kernel_ptr<float, false>(cfg);
}
// cluster size and dynamic shared memory of configuration `cfg`
static void plane_cfg(bool dbl, int cfg, int& cs, size_t& smem) {
  if (cfg == 0) {
    cs = 16;
    smem = dbl ? PlaneGeo<double, 16, 2>::smem : PlaneGeo<float, 16, 2>::smem;
  } else if (cfg == 1) {
    cs = 16;
    smem = dbl ? PlaneGeo<double, 16, 1>::smem : PlaneGeo<float, 16, 1>::smem;
  } else {
    cs = 8;
    smem = dbl ? PlaneGeo<double, 8, 1>::smem : PlaneGeo<float, 8, 2>::smem;
  }
}

// Clusters of configuration `cfg` that can be resident at once (0: none).
static int plane_clusters(bool dbl, bool inv, int cfg) {
  static std::mutex mu;
  static std::map<std::tuple<int, bool, bool, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, dbl, inv, cfg);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int cs = 0;
  size_t smem = 0;
  plane_cfg(dbl, cfg, cs, smem);
  const void* k = plane_kernel_ptr(dbl, inv, cfg);
  int ncl = 0;
  if (kernel_smem_grant(k, smem) == cudaSuccess &&
      (cs <= 8 || cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess)) {
    cudaLaunchConfig_t cfgl = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfgl.gridDim = dim3(cs, 1, 1);
    cfgl.blockDim = dim3(kPlaneThreads, 1, 1);
    cfgl.dynamicSmemBytes = smem;
    cfgl.attrs = attr;
    cfgl.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&ncl, k, &cfgl) != cudaSuccess) ncl = 0;
  }
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = ncl;
  return ncl;
}

bool plane_plan(long long planes, bool dbl, bool inv, const void* in, const void* out, PlanePlan& pp) {
  // AFC_PLANE (read at every plan): 0 off (default), 1 automatic, 2 + c
  // forces configuration c (0: clusters of 16 with two plane buffers, 1:
  // clusters of 16 with one buffer and two CTAs per SM, 2: clusters of 8).
  // Opt-in: measured on B200 at 256^3 (forward, 20 warm repetitions), the
  // plane launch plus the leading-axis pass took 388-452 us in complex128 and
  // 189-214 us in complex64, against 285 and 151 us for three axis passes.
  // Clusters of 8 and 16 CTAs of this size fit on 112-120 of the 148 SMs, and
  // the kernel is latency-bound (12 % issue, 8 warps per SM): with the
  // distributed-shared-memory reads replaced by local ones it still took 286 /
  // 150 us, and with the cluster barriers also removed 256 / 124 us, so even
  // a free exchange would gain at most 10-18 %.
  const char* env = getenv("AFC_PLANE");
  const int mode = env && *env ? atoi(env) : 0;
  if (mode == 0 || planes < 1 || planes > (1ll << 31) - 1) return false;
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) return false;
  std::vector<int> cand;
  if (mode >= 2)
    cand.push_back(mode - 2);
  else
    cand = {0, 2, 1};
  for (int cfg : cand) {
    if (cfg < 0 || cfg > 2) continue;
    const int ncl = plane_clusters(dbl, inv, cfg);
    if (ncl < 1) continue;
    pp.cfg = cfg;
    plane_cfg(dbl, cfg, pp.cs, pp.smem);
    pp.nclusters = (int)std::min<long long>(ncl, planes);
    pp.planes = planes;
    return true;
  }
  return false;
}

template <class T, bool INV>
static cudaError_t launch_plane_t(const PlanePlan& pp, const void* in, void* out, const void* twz, const void* twy,
                                  double scale, unsigned* err, cudaStream_t st) {
  using C = typename CT<T>::type;
  const void* k = plane_kernel_ptr<T, INV>(pp.cfg);
  cudaError_t e = kernel_smem_grant(k, pp.smem);
  if (e != cudaSuccess) return e;
  if (pp.cs > 8) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  PlaneArgs<T> a;
  memset(&a, 0, sizeof(a));
  if (!tma_lane_map(&a.tmo, out, sizeof(T) == 8, 256, 256, pp.planes, 256 / pp.cs, 256)) return cudaErrorInvalidValue;
  a.in = static_cast<const C*>(in);
  a.twz = static_cast<const C*>(twz);
  a.twy = static_cast<const C*>(twy);
  a.planes = pp.planes;
  a.scale = (T)scale;
  a.err = err;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pp.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(pp.nclusters * pp.cs), 1, 1);
  cfg.blockDim = dim3(kPlaneThreads, 1, 1);
  cfg.dynamicSmemBytes = pp.smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {&a};
  e = cudaLaunchKernelExC(&cfg, k, args);
  count_launch(1);
  return e;
}

cudaError_t launch_plane(const PlanePlan& pp, const void* in, void* out, const void* twz, const void* twy,
                         double scale, unsigned* err, bool dbl, bool inv, cudaStream_t st) {
  if (dbl)
    return inv ? launch_plane_t<double, true>(pp, in, out, twz, twy, scale, err, st)
               : launch_plane_t<double, false>(pp, in, out, twz, twy, scale, err, st);
  return inv ? launch_plane_t<float, true>(pp, in, out, twz, twy, scale, err, st)
             : launch_plane_t<float, false>(pp, in, out, twz, twy, scale, err, st);
}

}  // namespace afc
