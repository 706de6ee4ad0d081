// tracker.cu -- entry points of the path tracker and the polish pass.
//
// One kernel per (system size N, homotopy kind, precision); the two
// precisions are instantiated in tracker_fp64.cu and tracker_fp32.cu.  The
// sizes cover every problem of the reference (P2C with N in
// {3,4,5,6,8,10,11,12,16,18}, PH with N = 30); others are rejected.
//
// Mixed precision is two launches on one stream.  The mixed tracker keeps the
// track, t, the step control, the norms and the corrector's residual H in FP64
// and evaluates H_x and H_t and factors the system in FP32 (Newton with an FP32
// solve of an FP64 residual: the endpoints converge to FP64 accuracy at a rate
// set by the FP32 solve, about cond(H_x) times FP32's rounding).  It takes every
// path to t = 1 (or to t_switch, when t_switch < 1); a path stops early after a
// step in which an FP32 solve's pivot magnitudes spanned more than cond_limit
// (the Jacobian is too ill-conditioned for FP32: Newton would stall), once its
// step falls below dt_floor (FP32 keeps failing the corrector where FP64 would
// not: a few per cent of paths near t = 1 otherwise crawl to the step cap),
// after kMixedFailLimit failed steps in a row, or on divergence (then at its
// last accepted point), with t, dt and its step and corrector counts in t_end,
// dt_end, steps and corr.  The FP64 tracker then resumes every
// path from there: a path the mixed tracker finished stops at once, a handed-over
// one continues with FP64 linear algebra (ill-conditioned Jacobians near a
// singular endpoint).
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

constexpr int kMixedFailLimit = 4;
constexpr double kMixedCondLimit = 1e5;
constexpr double kMixedDtFloor = 1e-4;

int launch_track(const TrackParams& p, int precision, double t_switch, void* stream, int n_sm) {
  cudaStream_t s = (cudaStream_t)stream;
  if (p.n_items <= 0) return 0;
  TrackParams q = p;
  q.cond_limit = 0.0;  // the plain trackers never stop on conditioning or step size
  q.dt_floor = 0.0;
  switch (precision) {
    case PREC_FP64:
      return launch_track_fp64(q, s, n_sm);
    case PREC_FP32:
      return launch_track_fp32(q, s, n_sm);
    case PREC_MIXED: {
      if (!p.t_end || !p.dt_end || !p.steps || !p.corr || p.track_in || p.resume) return -12;
      if (!(t_switch > 0.0)) return launch_track_fp64(q, s, n_sm);
      TrackParams a = p;
      a.t_handover = t_switch < 1.0 ? t_switch : 0.0;  // 0: no time boundary, the whole path
      a.fail_limit = kMixedFailLimit;
      a.cond_limit = p.cond_limit > 0.0 ? p.cond_limit : kMixedCondLimit;
      a.dt_floor = p.dt_floor > 0.0 ? p.dt_floor : kMixedDtFloor;
      a.variant = p.variant_f32;
      a.flat_eval = p.flat_eval_f32;
      int rc = launch_track_mixed(a, s, n_sm);
      if (rc) return rc;
      TrackParams b = q;
      b.resume = 1;
      b.t_in = p.t_end;
      b.dt_in = p.dt_end;
      b.track_in = p.endpoints;
      b.ld_track = p.ld_out;
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
