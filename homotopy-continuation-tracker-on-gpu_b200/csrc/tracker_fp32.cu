// tracker_fp32.cu -- reference precision: everything in float.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp32(const TrackParams& p, cudaStream_t s, int n_sm) {
  return launch_mode<float>(p, s, n_sm);
}
}  // namespace ghc
