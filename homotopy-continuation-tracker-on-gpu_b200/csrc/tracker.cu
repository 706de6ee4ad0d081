// tracker.cu -- entry points of the path tracker and the polish pass.
//
// One kernel per (system size N, homotopy kind, precision); the two
// precisions are instantiated in tracker_fp64.cu and tracker_fp32.cu.  The
// sizes cover every problem of the reference (P2C with N in
// {3,4,5,6,8,10,11,12,16,18}, PH with N = 30); others are rejected.
//
// Mixed precision is two launches on one stream.  The FP32 tracker takes every
// path from t = 0 to t_switch; a path that fails kMixedFailLimit steps in a row
// or diverges is handed over early, always at its last accepted point.  It
// writes its float track into the first half of each item's double endpoint
// slot and t, dt, step and corrector counts into t_end, dt_end, steps, corr.
// The FP64 tracker then resumes every path from there (reading the float track
// in place) to t = 1, so the end game, every retried stretch and the final
// answer are FP64.  The FP32 phase asks its corrector for no more than float
// can deliver: |dx|^2 < max(corr_tol2, kMixedF32Tol2) |x|^2.
#include <cuda_runtime.h>

#include <algorithm>

#include "ghc_internal.h"
#include "tracker_launch.cuh"

namespace ghc {

int track_subwarp_width(int N) {
  if (N <= 4) return 4;
  if (N <= 8) return 8;
  if (N <= 16) return 16;
  return 32;
}

constexpr int kMixedFailLimit = 2;
constexpr double kMixedMaxSwitch = 0.95;
constexpr double kMixedF32Tol2 = 1e-9;

int launch_track(const TrackParams& p, int precision, double t_switch, void* stream, int n_sm) {
  cudaStream_t s = (cudaStream_t)stream;
  if (p.n_items <= 0) return 0;
  switch (precision) {
    case PREC_FP64:
      return launch_track_fp64(p, s, n_sm);
    case PREC_FP32:
      return launch_track_fp32(p, s, n_sm);
    case PREC_MIXED: {
      if (!p.t_end || !p.dt_end || !p.steps || !p.corr || p.track_in || p.resume) return -12;
      if (!(t_switch > 0.0)) return launch_track_fp64(p, s, n_sm);
      TrackParams a = p;
      a.t_handover = std::min(t_switch, kMixedMaxSwitch);
      a.fail_limit = kMixedFailLimit;
      a.variant = p.variant_f32;
      a.flat_eval = p.flat_eval_f32;
      a.corr_tol2 = std::max(p.corr_tol2, kMixedF32Tol2);
      a.start_other = 1;        // double start solutions into the FP32 tracker
      a.ld_out = 2 * p.ld_out;  // float track in the first half of each double slot
      int rc = launch_track_fp32(a, s, n_sm);
      if (rc) return rc;
      TrackParams b = p;
      b.resume = 1;
      b.t_in = p.t_end;
      b.dt_in = p.dt_end;
      b.track_in = p.endpoints;
      b.ld_track = 2 * p.ld_out;
      b.track_other = 1;
      return launch_track_fp64(b, s, n_sm);
    }
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
