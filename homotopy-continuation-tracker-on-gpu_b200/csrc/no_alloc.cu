// no_alloc.cu -- ghc_track_noalloc: the batched tracker for callers that must
// not allocate device memory.
//
// Who needs this: a host application that owns every byte of device memory
// through its own pool or a fixed budget (for example a RANSAC stage embedded
// in a larger vision pipeline), or a latency-sensitive loop that cannot afford
// cudaMalloc, which may synchronise the device and can fail under memory
// pressure in the middle of a run.  Such callers hand over their inputs and
// outputs and expect the library to take nothing else from the device.
//
// ghc_track needs two pieces of device memory besides the caller's buffers:
// the work-stealing counter, and the compiled index tables of the problem
// (which it uploads into the problem handle on first use).  Here both live
// in one fixed array, g_noalloc_scratch, defined below with static storage:
// every GPU that loads this library holds it until the process exits.
//
//   * size: GHC_NOALLOC_SCRATCH_BYTES (64 KiB): 256 bytes for the counter,
//     the rest for the compiled tables; larger problems are rejected with
//     GHC_ERR_LIMIT and a message naming the sizes.
//   * set-up: the first call on each device, with that device current, looks
//     up the array's device address with cudaGetSymbolAddress and caches it.
//     The entry point is for eager calls; capture in a CUDA graph is neither
//     claimed nor tested (a call may copy tables from host memory).
//   * sharing: all calls on a device use the same array and it keeps the last
//     call's contents.  A call copies its problem's tables in on the caller's
//     stream unless the array already holds them (the last call on this device
//     was for the same handle), and the launch clears the counter on the
//     stream, so calls that follow each other in stream order are independent;
//     calls that overlap on the GPU (different streams, or different host
//     threads without ordering) race on the array.
//
// Everything else -- launch parameters, tuning, the precision modes and the
// polish -- is ghc_track's own code (abi_internal.h); only the table and
// counter pointers differ.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ghc.h"
#include "abi_internal.h"
#include "ghc_internal.h"
#include "problem.h"

using namespace ghc;

#define GHC_NOALLOC_SCRATCH_BYTES (64 * 1024)
#define GHC_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[GHC_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_mu;
void* g_addr[GHC_NOALLOC_MAX_DEVICES] = {};
uint64_t g_tables_of[GHC_NOALLOC_MAX_DEVICES] = {};  // uid of the handle whose tables the array holds

// device address of g_noalloc_scratch on the current device (looked up once per device)
int scratch_address(int* dev_out, void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= GHC_NOALLOC_MAX_DEVICES) {
    set_error("ghc_track_noalloc: no usable current CUDA device");
    return GHC_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("ghc_track_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return GHC_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *dev_out = dev;
  *out = g_addr[dev];
  return GHC_OK;
}

size_t up16(size_t v) { return (v + 15) & ~(size_t)15; }

}  // namespace

extern "C" int ghc_track_noalloc(const ghc_problem* h, const ghc_track_args* a, void* stream) {
  if (!h || !a || a->n_hyp < 0) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  if (a->n_hyp == 0) return GHC_OK;
  if (!a->d_start_sols || !a->d_endpoints) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  const Problem& pb = h->pb;
  // scratch layout: [counter | hx terms | hx offsets | ht terms | ht offsets]
  const size_t o_hx = 256;
  const size_t o_hxo = o_hx + up16(pb.hx_terms.size() * sizeof(uint64_t));
  const size_t o_ht = o_hxo + up16(pb.hx_off.size() * sizeof(uint16_t));
  const size_t o_hto = o_ht + up16(pb.ht_terms.size() * sizeof(uint64_t));
  const size_t need = o_hto + up16(pb.ht_off.size() * sizeof(uint16_t));
  if (need > GHC_NOALLOC_SCRATCH_BYTES) {
    set_error("ghc_track_noalloc: the compiled tables need " + std::to_string(need) +
              " bytes of scratch, more than the fixed " + std::to_string(GHC_NOALLOC_SCRATCH_BYTES) +
              "; use ghc_track for this problem");
    return GHC_ERR_LIMIT;
  }
  ghc_track_args args = *a;
  args.d_counter = nullptr;  // the array's own counter
  TrackParams p;
  int rc = track_params(pb, &args, p);
  if (rc) return rc;
  int dev = 0;
  void* base = nullptr;
  if ((rc = scratch_address(&dev, &base))) return rc;
  unsigned char* s = static_cast<unsigned char*>(base);
  cudaStream_t st = (cudaStream_t)stream;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_tables_of[dev] != pb.uid) {
      if (cudaMemcpyAsync(s + o_hx, pb.hx_terms.data(), pb.hx_terms.size() * sizeof(uint64_t),
                          cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(s + o_hxo, pb.hx_off.data(), pb.hx_off.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                          st) != cudaSuccess ||
          cudaMemcpyAsync(s + o_ht, pb.ht_terms.data(), pb.ht_terms.size() * sizeof(uint64_t),
                          cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(s + o_hto, pb.ht_off.data(), pb.ht_off.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                          st) != cudaSuccess) {
        g_tables_of[dev] = 0;
        return cuda_fail("ghc_track_noalloc: table copy");
      }
      g_tables_of[dev] = pb.uid;
    }
  }
  p.hx_terms = reinterpret_cast<const uint64_t*>(s + o_hx);
  p.hx_off = reinterpret_cast<const uint16_t*>(s + o_hxo);
  p.ht_terms = reinterpret_cast<const uint64_t*>(s + o_ht);
  p.ht_off = reinterpret_cast<const uint16_t*>(s + o_hto);
  p.counter = reinterpret_cast<int*>(s);  // cleared on `stream` by the launch
  return run_track(p, &args, stream);
}
