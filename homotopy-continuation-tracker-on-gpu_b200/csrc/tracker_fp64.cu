// tracker_fp64.cu -- plain FP64 tracker, register-budget variant 0.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp64_v0(const TrackParams& p, cudaStream_t s, int n_sm) { return launch_mode<double, double, 0>(p, s, n_sm); }
}  // namespace ghc
