// tracker.cu -- entry points of the path tracker and the polish pass.
//
// One kernel per (system size N, homotopy kind, precision mode); the three
// precision modes are instantiated in tracker_fp64.cu, tracker_fp32.cu and
// tracker_mixed.cu.  The sizes cover every problem of the reference (P2C with
// N in {3,4,5,6,8,10,11,12,16,18}, PH with N = 30); others are rejected.
#include <cuda_runtime.h>

#include "ghc_internal.h"
#include "tracker_launch.cuh"

namespace ghc {

int track_subwarp_width(int N) {
  if (N <= 4) return 4;
  if (N <= 8) return 8;
  if (N <= 16) return 16;
  return 32;
}

int launch_track(const TrackParams& p, int precision, void* stream, int n_sm) {
  cudaStream_t s = (cudaStream_t)stream;
  if (p.n_items <= 0) return 0;
  switch (precision) {
    case PREC_FP64:
      return launch_track_fp64(p, s, n_sm);
    case PREC_FP32:
      return launch_track_fp32(p, s, n_sm);
    case PREC_MIXED:
      return launch_track_mixed(p, s, n_sm);
    default:
      return -11;
  }
}

int launch_polish(const PolishParams& p, void* stream) {
  using namespace launch_detail;
  cudaStream_t s = (cudaStream_t)stream;
  if (p.n_items <= 0 || p.iters < 0) return 0;
  if (p.kind == KIND_P2C) {
    switch (p.N) {
#define CASE(n) \
  case n:       \
    return launch_polish_t<n, KIND_P2C>(p, s);
      GHC_P2C_SIZES(CASE)
#undef CASE
      default:
        return -10;
    }
  }
  if (p.kind == KIND_PH && p.N == 30) return launch_polish_t<30, KIND_PH>(p, s);
  return -10;
}

}  // namespace ghc
