// tracker_fp64.cu -- plain FP64: state, predictor and corrector in double.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp64(const TrackParams& p, cudaStream_t s, int n_sm) {
  return launch_mode<double>(p, s, n_sm);
}
}  // namespace ghc
