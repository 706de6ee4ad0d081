// tracker_launch.cuh -- launch templates shared by the per-precision translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

#include "ghc_internal.h"
#include "tracker.cuh"

namespace ghc {
namespace launch_detail {

constexpr int kBlock = 128;

// Threads per CTA: 128, or fewer (64, 32) when that many sub-warps' shared memory (per-sub-warp
// coefficient buffers grow with the problem's coefficient count: 565 complex values x 2 for the
// generalized 3-view 6-line problem) exceeds what one CTA may use.  0: does not fit at all.
inline int block_threads(size_t tables, size_t per_sub, int W, int max_block = kBlock) {
  static int optin = 0;
  if (optin == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0) v = 48 * 1024;
    optin = v;
  }
  for (int b = max_block; b >= 32; b /= 2)
    if (tables + (size_t)(b / W) * per_sub <= (size_t)optin) return b;
  return 0;
}

template <typename R, typename RL, int N, int KIND, int V, int S, int WK>
int launch_track_w(const TrackParams& p, cudaStream_t s, int n_sm) {
  constexpr int W = (N <= 4) ? 4 : (N <= 8) ? 8 : (N <= 16) ? 16 : 32;
  auto kern = dev::track_kernel<R, RL, N, W, KIND, V, S, WK>;
  const int Mc = (KIND == KIND_P2C) ? p.M + 1 : p.P + 1;
  const int slots = (dev::kFlatAlways<N> || p.flat_eval) ? p.scr_slots : 0;
  const size_t tables = dev::tables_bytes(N, p.n_hx_terms, p.n_ht_terms);
  const size_t per_sub = dev::sub_bytes(N, Mc, W, slots, 2 * (int)sizeof(RL), 2 * (int)sizeof(R));
  const int block = block_threads(tables, per_sub, W, GHC_BLOCK(N, R, RL, V));
  if (block == 0) return -24;
  const int subs = block / W;
  const size_t smem = tables + subs * per_sub;
  // Host calls in the launch path delay small launches, so per instantiation and device the
  // shared-memory attribute is only ever raised (to the largest size asked for, so a concurrent
  // launch never sees it below its own size) and the occupancy of the last size is kept.
  constexpr int kDevs = 16;
  static std::atomic<long long> attr_max[kDevs], occ_key[kDevs];
  static std::atomic<int> occ_val[kDevs];
  int dev_id = 0;
  cudaError_t e = cudaGetDevice(&dev_id);
  if (e != cudaSuccess) return -20;
  const int d = dev_id & (kDevs - 1);
  long long have = attr_max[d].load();
  while (have < (long long)smem) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return -20;
    if (attr_max[d].compare_exchange_weak(have, (long long)smem)) break;
  }
  const long long okey = (long long)smem * 256 + block + 1;
  int occ = occ_key[d].load() == okey ? occ_val[d].load() : 0;
  if (occ < 1) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
    if (e != cudaSuccess || occ < 1) return -21;
    occ_val[d].store(occ);
    occ_key[d].store(okey);
  }
  // persistent grid: fill the GPU once, but never launch more sub-warps than items; a launch
  // with fewer paths than one warp per scheduler of every SM gives each path its own warp
  TrackParams q = p;
  const int warps = block / 32;
  q.spread = (W < 32 && p.n_items <= (long long)n_sm * warps) ? 1 : 0;
  const int per_cta = q.spread ? warps : subs;
  long long grid = (long long)occ * n_sm;
  const long long need = (p.n_items + per_cta - 1) / per_cta;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  // spread: every path is placed at launch and the (unsigned) counter only ever yields items
  // >= n_items, so it needs no reset
  if (!q.spread) {
    e = cudaMemsetAsync(p.counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return -22;
  }
  kern<<<(unsigned)grid, block, smem, s>>>(q);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -23;
}

// one kernel per H_x walk (entry-wise, row-wise, balanced where built; above 16 unknowns never entry-wise)
template <typename R, typename RL, int N, int KIND, int V, int S>
int launch_track_s(const TrackParams& p, cudaStream_t s, int n_sm) {
  if constexpr (N > 16) {
    if (p.flat_eval == 2 && balanced_walk_built(N)) return launch_track_w<R, RL, N, KIND, V, S, 2>(p, s, n_sm);
    return launch_track_w<R, RL, N, KIND, V, S, 1>(p, s, n_sm);
  } else {
    // one kernel per walk here too: only the chosen walk's code is in the loop body
    if (p.flat_eval == 2 && balanced_walk_built(N)) return launch_track_w<R, RL, N, KIND, V, S, 2>(p, s, n_sm);
    if (p.flat_eval != 0) return launch_track_w<R, RL, N, KIND, V, S, 1>(p, s, n_sm);
    return launch_track_w<R, RL, N, KIND, V, S, 0>(p, s, n_sm);
  }
}

template <typename R, typename RL, int N, int KIND, int V>
int launch_track_t(const TrackParams& p, cudaStream_t s, int n_sm) {
  switch (p.shape) {
    case EVAL_1_2:
      return launch_track_s<R, RL, N, KIND, V, EVAL_1_2>(p, s, n_sm);
    case EVAL_2_3:
      return launch_track_s<R, RL, N, KIND, V, EVAL_2_3>(p, s, n_sm);
    default:
      return launch_track_s<R, RL, N, KIND, V, EVAL_GENERAL>(p, s, n_sm);
  }
}

template <int N, int KIND, int S>
int launch_polish_s(const PolishParams& p, cudaStream_t s) {
  constexpr int W = (N <= 4) ? 4 : (N <= 8) ? 8 : (N <= 16) ? 16 : 32;
  auto kern = dev::polish_kernel<N, W, KIND, S>;
  const int Mc = (KIND == KIND_P2C) ? p.M + 1 : p.P + 1;
  const int slots = (dev::kFlatAlways<N> || p.flat_eval) ? p.scr_slots : 0;
  const size_t tables = dev::tables_bytes(N, p.n_hx_terms, p.n_ht_terms);
  const size_t per_sub = dev::sub_bytes(N, Mc, W, slots, 16, 16);
  const int block = block_threads(tables, per_sub, W);
  if (block == 0) return -24;
  const int subs = block / W;
  const size_t smem = tables + subs * per_sub;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -20;
  long long grid = (p.n_items + subs - 1) / subs;
  if (grid > 65535LL * 16) grid = 65535LL * 16;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, block, smem, s>>>(p);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

template <int N, int KIND>
int launch_polish_t(const PolishParams& p, cudaStream_t s) {
  switch (p.shape) {
    case EVAL_1_2:
      return launch_polish_s<N, KIND, EVAL_1_2>(p, s);
    case EVAL_2_3:
      return launch_polish_s<N, KIND, EVAL_2_3>(p, s);
    default:
      return launch_polish_s<N, KIND, EVAL_GENERAL>(p, s);
  }
}

}  // namespace launch_detail


#ifndef GHC_P2C_SIZES
#define GHC_P2C_SIZES(X) X(3) X(4) X(5) X(6) X(8) X(10) X(11) X(12) X(16) X(18)
#endif

// dispatch of one precision mode (state R, linear algebra RL) over the compiled sizes
template <typename R, typename RL, int V>
int launch_mode(const TrackParams& p, cudaStream_t s, int n_sm) {
  using namespace launch_detail;
  if (p.kind == KIND_P2C) {
    switch (p.N) {
#define CASE(n) \
  case n:       \
    return launch_track_t<R, RL, n, KIND_P2C, V>(p, s, n_sm);
      GHC_P2C_SIZES(CASE)
#undef CASE
      default:
        return -10;
    }
  }
  if (p.kind == KIND_PH && p.N == 30) return launch_track_t<R, RL, 30, KIND_PH, V>(p, s, n_sm);
  return -10;
}

// one translation unit per (precision, variant): tracker_fp64.cu, tracker_fp64_v1.cu, tracker_fp32.cu,
// tracker_fp32_v1.cu, tracker_mixed.cu, tracker_mixed_v1.cu; launch_track_fp64 / _fp32 / _mixed
// (tracker.cu) pick by TrackParams::variant
int launch_track_fp64_v0(const TrackParams& p, cudaStream_t s, int n_sm);
int launch_track_fp64_v1(const TrackParams& p, cudaStream_t s, int n_sm);
int launch_track_fp32_v0(const TrackParams& p, cudaStream_t s, int n_sm);
int launch_track_fp32_v1(const TrackParams& p, cudaStream_t s, int n_sm);
int launch_track_mixed_v0(const TrackParams& p, cudaStream_t s, int n_sm);
int launch_track_mixed_v1(const TrackParams& p, cudaStream_t s, int n_sm);
inline int launch_track_fp64(const TrackParams& p, cudaStream_t s, int n_sm) {
  return p.variant ? launch_track_fp64_v1(p, s, n_sm) : launch_track_fp64_v0(p, s, n_sm);
}
inline int launch_track_fp32(const TrackParams& p, cudaStream_t s, int n_sm) {
  return p.variant ? launch_track_fp32_v1(p, s, n_sm) : launch_track_fp32_v0(p, s, n_sm);
}
inline int launch_track_mixed(const TrackParams& p, cudaStream_t s, int n_sm) {
  return p.variant ? launch_track_mixed_v1(p, s, n_sm) : launch_track_mixed_v0(p, s, n_sm);
}

}  // namespace ghc
