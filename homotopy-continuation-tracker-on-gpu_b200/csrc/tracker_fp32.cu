// tracker_fp32.cu -- FP32 tracker (the reference's precision), register-budget variant 0.
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp32_v0(const TrackParams& p, cudaStream_t s, int n_sm) { return launch_mode<float, float, 0>(p, s, n_sm); }
}  // namespace ghc
