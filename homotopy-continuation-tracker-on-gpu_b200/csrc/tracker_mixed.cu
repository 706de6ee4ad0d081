// tracker_mixed.cu -- FP64 state; FP32 predictor; FP32 corrector before t_switch, FP64 after.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_mixed(const TrackParams& p, cudaStream_t s, int n_sm) {
  return launch_mode<double, float, float, double>(p, s, n_sm);
}
}  // namespace ghc
