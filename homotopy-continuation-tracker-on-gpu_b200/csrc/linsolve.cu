// linsolve.cu -- the tracker's linear solve on its own (ghc_lu_solve_device).
//
// The same partial-pivot LU and back substitution the tracker runs on every
// evaluation (tracker.cuh lu_solve, the reference's cgesv_batched_small_device,
// GPU-HC/magmaHC/dev-cgesv-batched-small.cuh:40-107), one sub-warp per system,
// lane r holding row r in registers.  It exists so that the pivot rule and the
// elimination can be checked against the oracle on chosen matrices (near ties,
// zero pivots, NaN) that a tracked path would rarely produce.
#include <cuda_runtime.h>

#include <string>

#include "../../include/ghc.h"
#include "ghc_internal.h"
#include "problem.h"
#include "tracker.cuh"

namespace ghc {
namespace {

using dev::cx;

template <typename R, int N, int W>
__global__ void __launch_bounds__(128) lu_kernel(long long n_sys, const R* __restrict__ A, const R* __restrict__ b,
                                                 R* __restrict__ z) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int l = lane % W;
  const int g = threadIdx.x / W;
  const int subs = blockDim.x / W;
  // per sub-warp: the solve scratch [lu_scratch_len(N)] (pivot rows, or the whole system), solution [N]
  cx<R>* sx = dev::view<R>(smem) + (size_t)g * (dev::lu_scratch_len(N) + N);
  cx<R>* sol = sx + dev::lu_scratch_len(N);
  for (long long s0 = (long long)blockIdx.x * subs; s0 < n_sys; s0 += (long long)gridDim.x * subs) {
    const long long s = s0 + g;
    const bool mine = s < n_sys && l < N;
    cx<R> row[N];
    dev::static_for<0, N>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      row[j] = mine ? dev::mk(A[2 * ((s * N + l) * N + j)], A[2 * ((s * N + l) * N + j) + 1]) : dev::mk(R(0), R(0));
    });
    const cx<R> rhs = mine ? dev::mk(b[2 * (s * N + l)], b[2 * (s * N + l) + 1]) : dev::mk(R(0), R(0));
    dev::lu_solve<R, N, W>(row, rhs, l, sx, sol);
    if (mine) {
      z[2 * (s * N + l)] = sol[l].re;
      z[2 * (s * N + l) + 1] = sol[l].im;
    }
    __syncwarp(dev::kFull);
  }
}

template <typename R, int N>
int launch_lu(long long n_sys, const void* A, const void* b, void* z, cudaStream_t s) {
  constexpr int W = subwarp_width(N);
  const int subs = 128 / W;
  const size_t smem = (size_t)subs * (dev::lu_scratch_len(N) + N) * sizeof(cx<R>);
  long long grid = (n_sys + subs - 1) / subs;
  if (grid > 148LL * 16) grid = 148LL * 16;
  lu_kernel<R, N, W><<<(unsigned)grid, 128, smem, s>>>(n_sys, (const R*)A, (const R*)b, (R*)z);
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return GHC_OK;
  set_error(std::string("linear-solve launch: ") + cudaGetErrorString(e));
  return GHC_ERR_CUDA;
}

template <typename R>
int launch_lu_n(int N, long long n_sys, const void* A, const void* b, void* z, cudaStream_t s) {
  switch (N) {
#define CASE(n) \
  case n:       \
    return launch_lu<R, n>(n_sys, A, b, z, s);
    CASE(3) CASE(4) CASE(5) CASE(6) CASE(8) CASE(10) CASE(11) CASE(12) CASE(16) CASE(18) CASE(30)
#undef CASE
    default:
      set_error("no compiled linear solve for this size (N in {3,4,5,6,8,10,11,12,16,18,30})");
      return GHC_ERR_RANGE;
  }
}

}  // namespace
}  // namespace ghc

extern "C" int ghc_lu_solve_device(int32_t N, int32_t precision, int64_t n_sys, const void* d_A, const void* d_b,
                                   void* d_z, void* stream) {
  if (n_sys < 0 || (n_sys > 0 && (!d_A || !d_b || !d_z))) {
    ghc::set_error("null argument or negative count");
    return GHC_ERR_ARG;
  }
  if (precision != GHC_PREC_FP64 && precision != GHC_PREC_FP32) {
    ghc::set_error("precision must be GHC_PREC_FP64 or GHC_PREC_FP32");
    return GHC_ERR_ARG;
  }
  if (n_sys == 0) return GHC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return precision == GHC_PREC_FP64 ? ghc::launch_lu_n<double>(N, n_sys, d_A, d_b, d_z, s)
                                    : ghc::launch_lu_n<float>(N, n_sys, d_A, d_b, d_z, s);
}
