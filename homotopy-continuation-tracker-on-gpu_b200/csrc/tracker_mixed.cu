// tracker_mixed.cu -- mixed tracker (FP64 state and residual, FP32 H_x, H_t and LU), register-budget variant 0.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_mixed_v0(const TrackParams& p, cudaStream_t s, int n_sm) {
  return launch_mode<double, float, 0>(p, s, n_sm);
}
}  // namespace ghc
