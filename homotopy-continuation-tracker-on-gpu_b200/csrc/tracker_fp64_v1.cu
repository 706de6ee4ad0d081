// tracker_fp64_v1.cu -- plain FP64 tracker, register-budget variant 1 (one more CTA per SM).
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp64_v1(const TrackParams& p, cudaStream_t s, int n_sm) { return launch_mode<double, double, 1>(p, s, n_sm); }
}  // namespace ghc
