// tracker_fp32_v1.cu -- FP32 tracker, register-budget variant 1 (more CTAs per SM).
#include "tracker_launch.cuh"

namespace ghc {
int launch_track_fp32_v1(const TrackParams& p, cudaStream_t s, int n_sm) { return launch_mode<float, float, 1>(p, s, n_sm); }
}  // namespace ghc
