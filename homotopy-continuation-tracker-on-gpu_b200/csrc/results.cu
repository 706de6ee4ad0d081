// results.cu -- result counts of every hypothesis of a batch, on the device.
//
// The reference's Evaluations (GPU-HC/magmaHC/Evaluations.cpp:88-110 and
// 127-176) restated for a batch, with the same rules as the host
// ghc_count_results:
//   converged / infinity   the tracker's flags;
//   real                   converged and every |Im x_v| <= imag_tol;
//   unique                 walk the paths bs in order; a converged bs outside the
//                          current skip set collects every later ds (whatever its
//                          flags) that agrees in every Re and Im within dup_tol;
//                          none -> bs counts as unique, otherwise the skip set is
//                          REPLACED by those ds and bs is not counted.
// The walk is sequential per hypothesis, so one warp takes one hypothesis: bs
// advances uniformly, the lanes test the later paths in aligned chunks of 32
// (a chunk's ballot is one word of the duplicate bit set), and the skip set is a
// bit set in shared memory.  A class byte per path (bit 0 converged, bit 1 real,
// bit 2 counted as unique) lets a caller compact the results without leaving the
// device.
#include <cuda_runtime.h>

#include <cstdint>

#include "ghc_internal.h"

namespace ghc {
namespace {

constexpr int kWarps = 4;  // hypotheses per CTA
constexpr unsigned kFull = 0xffffffffu;

__global__ void __launch_bounds__(32 * kWarps)
    results_kernel(int N, int paths, long long n_hyp, const double* __restrict__ z, const uint8_t* __restrict__ conv,
                   const uint8_t* __restrict__ inf, double imag_tol, double dup_tol, int* __restrict__ counts,
                   uint8_t* __restrict__ cls) {
  extern __shared__ unsigned smask[];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int words = (paths + 31) / 32;
  unsigned* skip = smask + (size_t)w * 2 * words;
  unsigned* dup = skip + words;
  for (long long h = (long long)blockIdx.x * kWarps + w; h < n_hyp; h += (long long)gridDim.x * kWarps) {
    const double* zh = z + 2 * h * paths * (long long)N;
    const uint8_t* ch = conv + h * paths;
    const uint8_t* ih = inf + h * paths;
    uint8_t* clh = cls ? cls + h * paths : nullptr;
    // converged / infinity / real (Evaluations.cpp:88-110)
    int nc = 0, ni = 0, nr = 0;
    for (int p = lane; p < paths; p += 32) {
      const bool c = ch[p] != 0;
      nc += c;
      ni += ih[p] != 0;
      bool real = c;
      for (int v = 0; v < N && real; ++v) real = fabs(zh[2 * ((size_t)p * N + v) + 1]) <= imag_tol;
      nr += real;
      if (clh) clh[p] = (uint8_t)((c ? 1 : 0) | (real ? 2 : 0));
    }
    nc = __reduce_add_sync(kFull, nc);
    ni = __reduce_add_sync(kFull, ni);
    nr = __reduce_add_sync(kFull, nr);
    // unique (Evaluations.cpp:127-176)
    for (int k = lane; k < words; k += 32) skip[k] = 0u;
    __syncwarp(kFull);
    bool have_skip = false;
    int nu = 0;
    for (int bs = 0; bs < paths; ++bs) {
      if (!ch[bs]) continue;
      if (have_skip && ((skip[bs >> 5] >> (bs & 31)) & 1u)) continue;
      bool any = false;
      for (int c0 = (bs + 1) & ~31; c0 < paths; c0 += 32) {
        const int ds = c0 + lane;
        bool same = ds > bs && ds < paths;
        for (int v = 0; v < N && __any_sync(kFull, same); ++v) {
          if (same) {
            const double* a = zh + 2 * ((size_t)bs * N + v);
            const double* b = zh + 2 * ((size_t)ds * N + v);
            same = fabs(a[0] - b[0]) < dup_tol && fabs(a[1] - b[1]) < dup_tol;
          }
        }
        const unsigned m = __ballot_sync(kFull, same);
        if (lane == 0) dup[c0 >> 5] = m;
        any = any || m != 0u;
      }
      if (any) {
        __syncwarp(kFull);
        const int first = (bs + 1) >> 5;  // words below hold no later path
        for (int k = lane; k < words; k += 32) skip[k] = k >= first ? dup[k] : 0u;
        __syncwarp(kFull);
        have_skip = true;
      } else {
        ++nu;
        if (clh && lane == 0) clh[bs] = (uint8_t)(clh[bs] | 4);
      }
    }
    if (lane == 0) {
      counts[4 * h + 0] = nc;
      counts[4 * h + 1] = nr;
      counts[4 * h + 2] = ni;
      counts[4 * h + 3] = nu;
    }
    __syncwarp(kFull);
  }
}

}  // namespace

size_t results_smem_bytes(int paths) { return (size_t)kWarps * 2 * ((paths + 31) / 32) * sizeof(unsigned); }

int launch_results(int N, int paths, long long n_hyp, const double* z, const uint8_t* conv, const uint8_t* inf,
                   double imag_tol, double dup_tol, int* counts, uint8_t* cls, void* stream) {
  if (n_hyp <= 0 || paths <= 0) return 0;
  const size_t smem = results_smem_bytes(paths);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(results_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -20;
  long long grid = (n_hyp + kWarps - 1) / kWarps;
  if (grid > 148LL * 32) grid = 148LL * 32;
  results_kernel<<<(unsigned)grid, 32 * kWarps, smem, (cudaStream_t)stream>>>(N, paths, n_hyp, z, conv, inf,
                                                                               imag_tol, dup_tol, counts, cls);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

}  // namespace ghc
