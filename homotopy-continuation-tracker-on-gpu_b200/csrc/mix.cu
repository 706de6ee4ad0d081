// mix.cu -- ghc_track_mix: batches of problems of different sizes in one persistent launch.
//
// The reference dispatches one hand-written kernel per problem
// (GPU-HC/magmaHC/GPU_HC_Solver.cpp:207-349); a mixed workload is a sequence of
// launches, each ending in the tail of its longest paths.  Here the buckets of a
// mix -- one (problem, batch) each -- share one grid: CTA ranges start on their
// own bucket (sized by its expected work), every bucket keeps its own work
// counter, and a CTA whose bucket has no items left moves on to the others and
// takes items from their counters, so the short buckets fill the SMs while the
// long one drains, and no bucket's tail idles the GPU alone.
//
// The kernel holds one tracker body per bucket slot, compiled for the size
// buckets of the uneven-mix workload: P2C N = 3 (1,2), N = 6 (2,3), N = 12 (1,2)
// and PH N = 30 (2,3) term shapes, plain FP64.  Its registers are those of the
// largest body (N = 30: three CTAs per SM).  Every path is tracked exactly as a
// ghc_track launch of its bucket tracks it (the same arithmetic; which CTA takes
// an item does not matter), so the results are bit-identical to per-bucket
// launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/ghc.h"
#include "abi_internal.h"
#include "ghc_internal.h"
#include "problem.h"
#include "tracker.cuh"

namespace ghc {
namespace {

constexpr int kMixSlots = 4;
constexpr int kMixBlock = 128;

struct MixParams {
  TrackParams b[kMixSlots];
  long long begin[kMixSlots + 1];  // CTA range of each slot's own bucket (empty for unused slots)
  int used[kMixSlots];
};

// compiled slots: (N, kind, term shape, lanes per path, H_x walk)
template <int N_, int KIND_, int S_, int WK_>
struct Slot {
  static constexpr int N = N_, KIND = KIND_, S = S_, WK = WK_, W = subwarp_width(N_);
};
using Slot0 = Slot<3, KIND_P2C, EVAL_1_2, -1>;
using Slot1 = Slot<6, KIND_P2C, EVAL_2_3, -1>;
using Slot2 = Slot<12, KIND_P2C, EVAL_1_2, -1>;
using Slot3 = Slot<30, KIND_PH, EVAL_2_3, 1>;

template <class SL>
__device__ __forceinline__ void run_slot(const MixParams& mp, int k, unsigned char* smem, bool visitor) {
  dev::track_body<double, double, SL::N, SL::W, SL::KIND, SL::S, SL::WK>(mp.b[k], smem, (long long)blockIdx.x - mp.begin[k],
                                                                      mp.begin[k + 1] - mp.begin[k], visitor);
}

__device__ __forceinline__ void run(const MixParams& mp, int k, unsigned char* smem, bool visitor) {
  switch (k) {
    case 0:
      run_slot<Slot0>(mp, 0, smem, visitor);
      break;
    case 1:
      run_slot<Slot1>(mp, 1, smem, visitor);
      break;
    case 2:
      run_slot<Slot2>(mp, 2, smem, visitor);
      break;
    default:
      run_slot<Slot3>(mp, 3, smem, visitor);
      break;
  }
}

__global__ void __launch_bounds__(kMixBlock, 3) mix_kernel(const __grid_constant__ MixParams mp) {
  extern __shared__ __align__(16) unsigned char smem[];
  int home = 0;
  while (home < kMixSlots - 1 && blockIdx.x >= mp.begin[home + 1]) ++home;
  for (int j = 0; j < kMixSlots; ++j) {
    const int k = (home + j) % kMixSlots;
    if (!mp.used[k]) continue;
    if (j > 0) __syncthreads();  // every warp is done with the previous bucket's tables in shared memory
    run(mp, k, smem, j > 0);
  }
}

template <class SL>
bool slot_fits(const Problem& pb) {
  return pb.N == SL::N && pb.kind == SL::KIND && eval_shape_of(pb.kind, pb.Px, pb.Pt) == SL::S;
}

template <class SL>
size_t slot_smem(const TrackParams& p) {
  const int Mc = (SL::KIND == KIND_P2C) ? p.M + 1 : p.P + 1;
  const int walk = SL::WK >= 0 ? SL::WK : ((dev::kFlatAlways<SL::N> && p.flat_eval == 0) ? 1 : p.flat_eval);
  const int slots = walk ? p.scr_slots : 0;
  return dev::tables_bytes(SL::N, p.n_hx_terms, p.n_ht_terms) +
         (size_t)(kMixBlock / SL::W) * dev::sub_bytes(SL::N, Mc, SL::W, slots, 16, 16);
}

}  // namespace
}  // namespace ghc

using namespace ghc;

extern "C" int ghc_track_mix(const ghc_problem* const* pbs, const ghc_track_args* args, int32_t n_buckets,
                             void* stream) {
  if (!pbs || !args || n_buckets < 1 || n_buckets > kMixSlots) {
    set_error("ghc_track_mix: 1 to 4 buckets");
    return GHC_ERR_ARG;
  }
  MixParams mp;
  std::memset(&mp, 0, sizeof(mp));
  double weight[kMixSlots] = {0, 0, 0, 0};
  size_t smem = 0;
  cudaStream_t st = (cudaStream_t)stream;
  for (int i = 0; i < n_buckets; ++i) {
    const ghc_track_args* a = &args[i];
    if (!pbs[i] || a->n_hyp < 0 || !a->d_start_sols || !a->d_endpoints || !a->d_counter) {
      set_error("ghc_track_mix: null argument");
      return GHC_ERR_ARG;
    }
    if (a->precision != GHC_PREC_FP64 || a->polish_iters > 0 || a->d_resid) {
      set_error("ghc_track_mix: plain FP64 tracking only (polish with ghc_track's own launches)");
      return GHC_ERR_ARG;
    }
    Problem& pb = const_cast<Problem&>(pbs[i]->pb);
    const int k = slot_fits<Slot0>(pb) ? 0 : slot_fits<Slot1>(pb) ? 1 : slot_fits<Slot2>(pb) ? 2
                                                                   : slot_fits<Slot3>(pb) ? 3 : -1;
    if (k < 0 || mp.used[k]) {
      set_error("ghc_track_mix: compiled for one bucket each of P2C N = 3 (1,2), 6 (2,3), 12 (1,2) and PH N = 30 "
                "(2,3) term shapes; " + pb.name + (k < 0 ? " is none of them" : " repeats a bucket"));
      return GHC_ERR_RANGE;
    }
    int rc = ensure_device(pb);
    if (rc) return rc;
    TrackParams& p = mp.b[k];
    if ((rc = track_params(pb, a, p))) return rc;
    p.spread = 0;
    mp.used[k] = a->n_hyp > 0 && p.n_items > 0;
    if (!mp.used[k]) continue;
    if (cudaMemsetAsync(p.counter, 0, sizeof(int), st) != cudaSuccess) return cuda_fail("ghc_track_mix: counter");
    const size_t b = k == 0 ? slot_smem<Slot0>(p) : k == 1 ? slot_smem<Slot1>(p) : k == 2 ? slot_smem<Slot2>(p)
                                                                                    : slot_smem<Slot3>(p);
    smem = std::max(smem, b);
    // expected work of the bucket: paths x (H_x terms + an N^3 LU) per evaluation
    weight[k] = (double)p.n_items * ((double)p.n_hx_terms + (double)pb.N * pb.N * pb.N);
  }
  int any = 0;
  for (int k = 0; k < kMixSlots; ++k) any |= mp.used[k];
  if (!any) return GHC_OK;
  if (cudaFuncSetAttribute(mix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cuda_fail("ghc_track_mix: shared memory");
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mix_kernel, kMixBlock, smem) != cudaSuccess || occ < 1)
    return cuda_fail("ghc_track_mix: occupancy");
  const long long grid = (long long)occ * sm_count();
  // CTA ranges in proportion to the expected work, at least one CTA per used bucket
  double total = 0;
  int n_used = 0;
  for (int k = 0; k < kMixSlots; ++k) {
    total += weight[k];
    n_used += mp.used[k];
  }
  long long at = 0;
  long long left = grid - n_used;
  for (int k = 0; k < kMixSlots; ++k) {
    mp.begin[k] = at;
    if (!mp.used[k]) continue;
    long long c = 1 + (long long)((double)left * weight[k] / total);
    at += c;
  }
  mp.begin[kMixSlots] = at;
  mix_kernel<<<(unsigned)at, kMixBlock, smem, st>>>(mp);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("ghc_track_mix: launch: ") + cudaGetErrorString(e));
    return GHC_ERR_CUDA;
  }
  return GHC_OK;
}
