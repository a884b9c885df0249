// afc_internal.h -- host <-> kernel interface inside libapollofft_cuda.so.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include "afc_engine.cuh"

namespace afc {

enum InOpKind { IN_C = 0, IN_R = 1, IN_HERM = 2, IN_CHIRP = 3, IN_CHIRP_R = 4, IN_GATHER = 5, IN_GATHER_R = 6, IN_FRAME = 7 };
enum OutOpKind {
  OUT_C = 0, OUT_RE = 1, OUT_TRUNC = 2, OUT_TW = 3, OUT_MUL = 4, OUT_CHIRP = 5, OUT_CHIRP_RE = 6,
  OUT_SCATTER = 7, OUT_SCATTER_RE = 8
};

// Everything one launch of the lanes / conv kernels needs (type-erased).
struct LaunchDesc {
  StageList sl;
  const void* tw = nullptr;
  long long lanes = 0;
  int L = 1, P = 1, ld = 1;
  LaneMap im{}, om{};
  const void* in = nullptr;
  void* out = nullptr;
  double scale = 1.0;
  int in_op = IN_C, out_op = OUT_C;
  bool stage_in = false, stage_out = false;
  long long jmul = 1, col_div = 1, col_mod = 1;
  long long nlen = 0, herm_n = 0;
  double pair_w = 1.0;
  long long twN = 1, twB = 1;
  int tw_conj = 0;
  const void* tw_hi = nullptr;
  const void* tw_lo = nullptr;
  const void* spec = nullptr;
  long long spec_ld = 0;  // convolution tiles: lane spectrum = spec + col * spec_ld (0: one spectrum for all lanes)
  const void* chirp = nullptr;
  int chirp_conj = 0;
  const int* gather = nullptr;
  const int* scatter = nullptr;
  int lane_minor = 0;
  int in_sel = 0, out_sel = 0;  // batch descriptors: pointer = base[sel] + offset
  const void* chirp_out = nullptr;  // OUT_CHIRP: post-multiply table when it differs from `chirp` (CZT)
  long long nlen_out = 0;          // OUT_CHIRP: outputs kept (j < nlen_out) when > 0, else nlen
  const void* window = nullptr;  // IN_FRAME: analysis window (real, frame length)
  long long frame_off = 0;       // IN_FRAME: frames start at lane base - frame_off
};

// A tile of the persistent batch kernel: descriptor index, kind (0 forward lanes
// tile, 1 convolution tile, 2 inverse lanes tile) and first lane.
struct BatchItem {
  int desc;
  int kind;
  long long q0;
};

// dynamic shared memory of lanes_kernel: L lanes x buffers x ld + 3 L lane descriptors
inline size_t lanes_smem_bytes(const LaunchDesc& d, size_t csz) {
  const int nbuf = engine_buffers(d.sl.nst, d.stage_in, d.stage_out);
  return (size_t)d.L * nbuf * (size_t)d.ld * csz + (size_t)d.L * 3 * sizeof(long long);
}
// conv_kernel: L lanes x 2 buffers x ld + 2 L extra complex + 2 L lane descriptors
inline size_t conv_smem_bytes(const LaunchDesc& d, size_t csz) {
  return (size_t)d.L * 2 * (size_t)d.ld * csz + (size_t)d.L * 2 * csz + (size_t)d.L * 3 * sizeof(long long);
}

// tile_kernel: 3 buffers of L x ld elements + 4 L lane bases
inline size_t tile_smem_bytes(const LaunchDesc& d, size_t csz) {
  return 3 * (size_t)d.L * (size_t)d.ld * csz + (size_t)d.L * 4 * sizeof(long long);
}

// TMA tile configuration of one axis pass (afc_tma.cu)
struct TmaPlan {
  int mode = 0;  // 0 contiguous lanes (1D bulk copies), 1 strided lanes (3D tensor maps)
  int L = 1, P = 1, ld = 1, slot_elems = 0;
  int nbx = 1, bn = 1;
  long long kb = 1, ntiles = 0, outer = 0;
  // every stage has at most P butterflies per lane: stages run in place in the
  // tile's slot (registers hold the butterfly across a barrier), no work buffer
  bool inplace = false;
  // kernel build: 0 any radix (256 threads), 1 radix 2/4/8/16 (256 threads),
  // 2 radix 2/4/8/16 complex128 at <= 128 threads, three CTAs per SM,
  // 3 7-smooth, 4 complex64 in place with two butterflies of a radix <= 8 stage,
  // 5 n = 256 as radix 16 x 16 in place with fixed shared-memory offsets,
  // 6 n = 4096 as radix 16 x 16 x 16 likewise, 7 a compile-time stage list
  // of a smooth odd length (out of place)
  int variant = 0;
  // contiguous in-place tiles only: real input lanes (widened in the first
  // stage) / real output lanes (real parts stored by the last stage)
  bool real_in = false, real_out = false;
  // twiddle entries kept resident in shared memory by persistent CTAs (0: read from global)
  int tw_res = 0;
  // tile slots of the load ring (2 or 3): slots - 1 tile loads in flight per CTA
  int nslot = 2;
  // variant 7: index of the compile-time stage list (afc_tma.cu, kFixed)
  int fix = -1;
  // strided lanes whose input rows are Hermitian (the pass after a real-input
  // pass of a full-spectrum R2C): the tiles cover columns [0, kb L) only and
  // column c in [1, hm_cmax] is also stored, conjugated and row-reversed, as
  // column es - c
  int hm_cmax = 0;
  // contiguous lanes: elements stored per lane (0: all n); the rest of each
  // output lane is written by a later pass (the Hermitian column pass's mirrors)
  int store_cols = 0;
};
bool tma_plan(const StageList& sl, int ld, long long lanes, const LaneMap& im, const LaneMap& om, const void* in,
              void* out, bool dbl, int lanes_pref, TmaPlan& tp, bool real_in = false, bool real_out = false,
              bool mirror = false);
size_t tma_smem_bytes(const TmaPlan& tp, size_t csz);
cudaError_t launch_tma(const LaunchDesc& d, const TmaPlan& tp, unsigned* err, bool dbl, bool inv, cudaStream_t st);

// Tensor map of lanes viewed as [2 es scalars, n, outer] with box [2 L, bn, 1]
// (afc_tma.cu); false when the driver cannot encode it.
bool tma_lane_map(CUtensorMap* m, const void* base, bool dbl, long long es, long long n, long long outer, int L, int bn);

// The last two axes of a C2C transform with 256 x 256 planes in one launch
// (afc_plane.cu, plane_kernel): a thread-block cluster owns a plane, its CTAs
// transform their rows, exchange columns through distributed shared memory and
// transform the columns.
struct PlanePlan {
  int cfg = 0;        // kernel build (cluster size, plane buffers, CTAs per SM)
  int cs = 0;         // CTAs per cluster
  int nclusters = 0;  // clusters launched (persistent over the planes)
  size_t smem = 0;
  long long planes = 0;
};
bool plane_plan(long long planes, bool dbl, bool inv, const void* in, const void* out, PlanePlan& pp);
cudaError_t launch_plane(const PlanePlan& pp, const void* in, void* out, const void* twz, const void* twy,
                         double scale, unsigned* err, bool dbl, bool inv, cudaStream_t st);

// Two axis passes over the same x-planes in one launch (afc_tma.cu,
// tma_pair_kernel): a thread-block cluster per plane transforms the plane's
// first-axis tiles, meets at the cluster barrier, then transforms its
// second-axis tiles, so the intermediate stays in L2.
struct TmaPairPlan {
  TmaPlan ph[2];
  int n[2] = {0, 0};            // tiles per plane of each phase
  long long lpp[2] = {0, 0};    // contiguous phases: lanes per plane
  long long planes = 0;
  int slot_elems = 0, threads = 0;
  int cs = 0, nclusters = 0;    // CTAs per cluster, clusters launched
  size_t smem = 0;
};
bool tma_pair_plan(const LaunchDesc& d0, const LaunchDesc& d1, long long planes, long long plane_bytes, bool dbl,
                   bool inv, TmaPairPlan& pp);
cudaError_t launch_tma_pair(const LaunchDesc& d0, const LaunchDesc& d1, const TmaPairPlan& pp, unsigned* err,
                            bool dbl, bool inv, cudaStream_t st);

// tensor-core radix-16 FFT (afc_tc.cu)
struct TcLaunch {
  const void* in = nullptr;
  void* out = nullptr;
  const void* tw = nullptr;
  StageList sl{};
  long long lanes = 0;
  double scale = 1.0;
  int inverse = 0;
  unsigned* err = nullptr;
};
cudaError_t launch_tc_fft(const TcLaunch& d, bool fp16, cudaStream_t st);

// 1D NUFFT spreading / interpolation (afc_nufft.cu), complex128 grids
struct NuLaunch {
  long long m = 0;   // oversampled grid length
  int w = 0;         // kernel half width
  double beta = 0, i0b = 1, len = 1;
};
cudaError_t nufft_spread_dev(const NuLaunch& L, const double* pos, const void* val, long long npts, void* grid,
                             cudaStream_t st);
cudaError_t nufft_interp_dev(const NuLaunch& L, const void* grid, const double* pos, long long npts, void* out,
                             cudaStream_t st);
cudaError_t nufft_deconv_out_dev(const void* grid, const double* deconv, long long n, long long m, void* out,
                                 cudaStream_t st);
struct NuLaunch3 {
  long long nx = 0, ny = 0, nz = 0, mx = 0, my = 0, mz = 0;
  int w = 0;
  double beta = 0, i0b = 1, lx = 1, ly = 1, lz = 1;
};
cudaError_t nufft3_spread_dev(const NuLaunch3& L, const double* pos, const void* val, long long npts, void* grid,
                              cudaStream_t st);
cudaError_t nufft3_interp_dev(const NuLaunch3& L, const void* grid, const double* pos, long long npts, void* out,
                              cudaStream_t st);
// Tiled spreading / interpolation: tile edge B (8 or 4; 0 = the kernel is too
// wide for a shared-memory tile and the per-point kernels run instead).
struct NuTileLaunch {
  int B = 0, ntx = 0, nty = 0, ntz = 0;
  int* cnt = nullptr;   // ntiles
  int* off = nullptr;   // ntiles + 1
  int* tile = nullptr;  // npts
  int* rank = nullptr;  // npts
  int* idx = nullptr;   // npts
};
int nufft3_tile_size(int w);
size_t nufft3_tile_smem(int B, int w);
cudaError_t nufft3_tiled_dev(const NuLaunch3& L, const NuTileLaunch& TL, bool spread, const double* pos,
                             const void* src, long long npts, void* dst, cudaStream_t st);
cudaError_t nufft3_modes_dev(const NuLaunch3& L, const double* dcx, const double* dcy, const double* dcz,
                             const void* src, void* dst, bool to_grid, cudaStream_t st);
cudaError_t nufft_place_coeffs_dev(const void* coeffs, const double* deconv, long long n, long long m, void* grid,
                                   cudaStream_t st);
// exact direct non-uniform DFTs (afc_nufft.cu), complex128
cudaError_t nudft1_type1_dev(const double* pos, const void* val, long long npts, long long n, double len, void* out,
                             cudaStream_t st);
cudaError_t nudft1_type2_dev(const void* coeffs, long long n, const double* pos, long long npts, double len, void* out,
                             cudaStream_t st);
cudaError_t nudft3_type1_dev(const double* pos, const void* val, long long npts, long long nx, long long ny,
                             long long nz, double lx, double ly, double lz, void* out, cudaStream_t st);
cudaError_t launch_wait_probe(unsigned* err, int polls, cudaStream_t st);
cudaError_t launch_tc_selftest(const float* A, const float* B, float* D, unsigned* err, bool fp16, cudaStream_t st);
size_t tc_fft_smem(int n);

// Launch facts cached per device and kernel (afc_kernels.cu): the dynamic
// shared memory already granted (cudaFuncSetAttribute only when a launch needs
// more) and CTAs per SM for a (threads, shared memory) shape, so repeated
// executions of a plan skip those driver calls.
cudaError_t kernel_smem_grant(const void* kern, size_t smem);
int kernel_ctas_per_sm(const void* kern, int threads, size_t smem);
cudaError_t launch_lanes(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st);
size_t kargs_size(bool dbl);
void kargs_pack(const LaunchDesc& d, bool dbl, void* dst);
// Threads of a persistent batch CTA (a tile uses at most this many).
constexpr int kBatchThreads = 256;
cudaError_t launch_batch(const void* descs, const BatchItem* items, int nitems, int* counter, size_t smem, int grid,
                         const void* in, void* out, void* ws, bool dbl, bool inv, cudaStream_t st);
int batch_blocks_per_sm(size_t smem, bool dbl, bool inv);
cudaError_t launch_tile(const LaunchDesc& d, bool dbl, bool inv, cudaStream_t st);
cudaError_t launch_conv(const LaunchDesc& d, bool dbl, cudaStream_t st);

// caller kernels of multi-pass transforms (afc_callers.cu)
cudaError_t stft_gather_dev(const void* sig, const void* win, long long nsig, long long flen, long long hop,
                            long long frames, void* out, bool dbl, cudaStream_t st);
cudaError_t chirp_rows_dev(const void* src, long long ss, long long valid, const void* table, void* dst, long long ds,
                           long long nout, long long batch, bool dbl, cudaStream_t st);
size_t czt_inverse_smem(long long n);
cudaError_t czt_inverse_dev(const void* spec, void* out, const void* nodes, const void* apow, long long n,
                            long long batch, bool dbl, cudaStream_t st);
cudaError_t stft_ola_dev(const void* frames, const void* window, long long nframes, long long flen, long long hop,
                         long long nsig, void* out, bool dbl, cudaStream_t st);
cudaError_t gen_row_spectrum_dev(void* dst, const void* src, long long N1, long long N2, bool dbl, cudaStream_t st);
cudaError_t gen_stage_twiddles_dev(void* tw, const StageList& sl, bool dbl, cudaStream_t st);
cudaError_t gen_roots_dev(void* out, long long cnt, long long mult, long long N, bool dbl, cudaStream_t st);
cudaError_t gen_chirp_dev(void* out, long long n, bool dbl, cudaStream_t st);
cudaError_t gen_bluestein_b_dev(void* b, const void* chirp, long long n, long long M, bool inverse, bool dbl,
                                cudaStream_t st);
cudaError_t gen_rader_b_dev(void* b, const int* scatter, long long p, long long M, bool inverse, bool dbl,
                            cudaStream_t st);

void count_launch(int k);

}  // namespace afc
