// abi_internal.h -- the problem handle and the launch helpers shared by the C-ABI
// translation units (abi.cu, no_alloc.cu), so that every entry point that tracks
// builds its launch the same way.
#pragma once
#include "../../include/ghc.h"
#include "ghc_internal.h"
#include "problem.h"

struct ghc_problem {
  ghc::Problem pb;
};

namespace ghc {

int sm_count();                     // SMs of the current device
int cuda_fail(const char* what);    // GHC_ERR_CUDA with the last CUDA error as the message
int track_code(int rc);             // launch_track / launch_polish codes -> GHC_* with a message
TrackParams base_params(const Problem& pb);
PolishParams polish_params(const TrackParams& t, double* endpoints, const uint8_t* conv, double* resid, int iters);
// The launch parameters of a ghc_track call: the problem's sizes, tuning and device tables
// (pb.dev), the caller's buffers and step control, a->d_counter as the work-stealing counter.
int track_params(const Problem& pb, const ghc_track_args* a, TrackParams& p);
// The tracker launch(es) of a->precision, then the FP64 polish when asked for.
int run_track(const TrackParams& p, const ghc_track_args* a, void* stream);

}  // namespace ghc
