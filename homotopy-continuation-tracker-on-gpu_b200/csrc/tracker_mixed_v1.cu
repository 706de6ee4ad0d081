// tracker_mixed_v1.cu -- mixed tracker (FP64 state and residual, FP32 H_x, H_t and LU), register-budget variant 1 (more CTAs per SM).
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_mixed_v1(const TrackParams& p, cudaStream_t s, int n_sm) {
  return launch_mode<double, float, 1>(p, s, n_sm);
}
}  // namespace ghc
