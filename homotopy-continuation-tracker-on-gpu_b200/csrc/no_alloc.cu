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
//     up the array's device address with cudaGetSymbolAddress and caches it;
//     make that first call before any stream capture.
//   * sharing: all calls on a device use the same array and it keeps the last
//     call's contents.  The tables are copied in and the counter is cleared
//     on the caller's stream by every call, so calls that follow each other in
//     stream order are independent; calls that overlap on the GPU (different
//     streams, or different host threads without ordering) race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ghc.h"
#include "ghc_internal.h"
#include "problem.h"

using namespace ghc;

// same layout as the handle defined in abi.cu
struct ghc_problem {
  Problem pb;
};

#define GHC_NOALLOC_SCRATCH_BYTES (64 * 1024)
#define GHC_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[GHC_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_mu;
void* g_addr[GHC_NOALLOC_MAX_DEVICES] = {};

// device address of g_noalloc_scratch on the current device (looked up once per device)
int scratch_address(void** out) {
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
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char* s = static_cast<unsigned char*>(base);
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(s + o_hx, pb.hx_terms.data(), pb.hx_terms.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      cudaMemcpyAsync(s + o_hxo, pb.hx_off.data(), pb.hx_off.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      cudaMemcpyAsync(s + o_ht, pb.ht_terms.data(), pb.ht_terms.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      cudaMemcpyAsync(s + o_hto, pb.ht_off.data(), pb.ht_off.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                      st) != cudaSuccess) {
    set_error(std::string("ghc_track_noalloc: table copy failed: ") + cudaGetErrorString(cudaGetLastError()));
    return GHC_ERR_CUDA;
  }

  TrackParams p;
  std::memset(&p, 0, sizeof(p));
  p.kind = pb.kind;
  p.N = pb.N;
  p.P = pb.P;
  p.M = pb.M;
  p.K = pb.K;
  p.max_steps = a->max_steps > 0 ? a->max_steps : pb.max_steps;
  p.max_corr = a->max_corr > 0 ? a->max_corr : pb.max_corr;
  p.incr = a->incr_steps > 0 ? a->incr_steps : pb.incr;
  p.n_hx_terms = (int)pb.hx_terms.size();
  p.n_ht_terms = (int)pb.ht_terms.size();
  p.hx_terms = reinterpret_cast<const uint64_t*>(s + o_hx);
  p.hx_off = reinterpret_cast<const uint16_t*>(s + o_hxo);
  p.ht_terms = reinterpret_cast<const uint64_t*>(s + o_ht);
  p.ht_off = reinterpret_cast<const uint16_t*>(s + o_hto);
  apply_tuning(pb, a->precision, p);
  p.scr_slots = row_nonzeros_max(pb.hx_off.data(), pb.N);
  p.shape = eval_shape_of(pb.kind, pb.Px, pb.Pt);
  p.n_items = a->n_hyp * (long long)(a->paths > 0 ? a->paths : pb.paths);
  p.paths_per_hyp = a->paths > 0 ? a->paths : pb.paths;
  p.start_sols = a->d_start_sols;
  p.ld_start = pb.N;
  p.ld_track = pb.N;
  if (pb.kind == KIND_P2C) {
    if (!a->d_coef_hx || !a->d_coef_ht) {
      set_error("P2C problem needs d_coef_hx / d_coef_ht");
      return GHC_ERR_ARG;
    }
    p.coef_hx = a->d_coef_hx;
    p.coef_ht = a->d_coef_ht;
    p.stride_hx = (long long)(pb.M + 1) * (pb.K + 1);
    p.stride_ht = (long long)(pb.M + 1) * pb.K;
  } else {
    if (!a->d_p_start || !a->d_p_target || !a->d_p_diff) {
      set_error("PH problem needs d_p_start / d_p_target / d_p_diff");
      return GHC_ERR_ARG;
    }
    p.p_start = a->d_p_start;
    p.p_tgt = a->d_p_target;
    p.p_diff = a->d_p_diff;
    p.stride_p = pb.P + 1;
  }
  p.endpoints = a->d_endpoints;
  p.ld_out = pb.N;
  p.status = a->d_status;
  p.conv = a->d_conv;
  p.infy = a->d_inf;
  p.steps = a->d_steps;
  p.corr = a->d_corr;
  p.t_end = a->d_t_end;
  p.dt_end = a->d_dt_end;
  p.counter = reinterpret_cast<int*>(s);  // cleared on `stream` by the launch
  p.corr_tol2 = a->corr_tol2 > 0 ? a->corr_tol2 : 1e-6;
  p.first_tol2 = a->first_tol2 > 0 ? a->first_tol2 : HUGE_VAL;
  p.dt_max = a->dt_max > 0 ? a->dt_max : HUGE_VAL;
  int dev = 0, n_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  rc = launch_track(p, a->precision, a->t_switch, stream, n_sm > 0 ? n_sm : 1);
  if (rc == -10) {
    set_error("system size or kind has no compiled tracker");
    return GHC_ERR_RANGE;
  }
  if (rc == -11) {
    set_error("unknown precision mode");
    return GHC_ERR_ARG;
  }
  if (rc == -12) {
    set_error("mixed precision needs d_steps, d_corr, d_t_end and d_dt_end (the FP32 -> FP64 handover state)");
    return GHC_ERR_ARG;
  }
  if (rc) {
    set_error(std::string("ghc_track_noalloc: launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    return GHC_ERR_CUDA;
  }
  const bool fp64_state = a->precision == GHC_PREC_FP64 || a->precision == GHC_PREC_MIXED;
  if ((a->polish_iters > 0 || a->d_resid) && fp64_state) {
    if (!a->d_conv) {
      set_error("polish needs d_conv");
      return GHC_ERR_ARG;
    }
    PolishParams q;
    std::memset(&q, 0, sizeof(q));
    q.kind = p.kind;
    q.N = p.N;
    q.P = p.P;
    q.M = p.M;
    q.K = p.K;
    q.n_hx_terms = p.n_hx_terms;
    q.n_ht_terms = p.n_ht_terms;
    q.flat_eval = p.flat_eval;
    q.scr_slots = p.scr_slots;
    q.shape = p.shape;
    q.hx_terms = p.hx_terms;
    q.hx_off = p.hx_off;
    q.ht_terms = p.ht_terms;
    q.ht_off = p.ht_off;
    q.n_items = p.n_items;
    q.paths_per_hyp = p.paths_per_hyp;
    q.coef_hx = p.coef_hx;
    q.stride_hx = p.stride_hx;
    q.coef_ht = p.coef_ht;
    q.stride_ht = p.stride_ht;
    q.p_start = p.p_start;
    q.p_tgt = p.p_tgt;
    q.p_diff = p.p_diff;
    q.stride_p = p.stride_p;
    q.endpoints = (double*)a->d_endpoints;
    q.ld = p.ld_out;
    q.conv = a->d_conv;
    q.resid = a->d_resid;
    q.iters = a->polish_iters;
    if (launch_polish(q, stream)) {
      set_error(std::string("ghc_track_noalloc: polish launch failed: ") + cudaGetErrorString(cudaGetLastError()));
      return GHC_ERR_CUDA;
    }
  }
  return GHC_OK;
}
