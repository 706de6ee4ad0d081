// abi.cu -- the extern "C" entry points declared in include/ghc.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "../../include/ghc.h"
#include "abi_internal.h"
#include "ghc_internal.h"
#include "problem.h"

namespace ghc {
const char* last_error();
int launch_f2d(const float* s, double* d, long long n, void* stream);
int launch_debug_f(const uint8_t* conv, const double* t, const double* dt, float* dbg, long long n, void* stream);
int launch_debug_d(const uint8_t* conv, const double* t, const double* dt, double* dbg, long long n, void* stream);
int launch_diff_d(const double* s, const double* t, double* d, long long n_hyp, int P1, void* stream);

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

int cuda_fail(const char* what) {
  const cudaError_t e = cudaGetLastError();
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return GHC_ERR_CUDA;
}

int track_code(int rc) {
  if (rc == 0) return GHC_OK;
  if (rc == -10) {
    set_error("system size or kind has no compiled tracker (P2C N in {3,4,5,6,8,10,11,12,16,18}, PH N = 30)");
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
  if (rc == -24) {
    set_error("the problem's tables and coefficient buffers exceed one CTA's shared memory even at 32 threads");
    return GHC_ERR_LIMIT;
  }
  return cuda_fail("tracker launch");
}

TrackParams base_params(const Problem& pb) {
  TrackParams p;
  std::memset(&p, 0, sizeof(p));
  p.kind = pb.kind;
  p.N = pb.N;
  p.P = pb.P;
  p.M = pb.M;
  p.K = pb.K;
  p.max_steps = pb.max_steps;
  p.max_corr = pb.max_corr;
  p.incr = pb.incr;
  p.n_hx_terms = (int)pb.hx_terms.size();
  p.n_ht_terms = (int)pb.ht_terms.size();
  p.hx_terms = pb.dev.hx_terms;
  p.hx_off = pb.dev.hx_off;
  p.ht_terms = pb.dev.ht_terms;
  p.ht_off = pb.dev.ht_off;
  p.flat_eval = flat_eval_pays(pb.hx_off.data(), pb.N);
  p.scr_slots = row_nonzeros_max(pb.hx_off.data(), pb.N);
  p.shape = eval_shape_of(pb.kind, pb.Px, pb.Pt);
  // the reference's step control (kernel_HC_Solver_P3P.cu:214): no contraction test, no step cap
  p.corr_tol2 = 1e-6;
  p.first_tol2 = HUGE_VAL;
  p.dt_max = HUGE_VAL;
  return p;
}

PolishParams polish_params(const TrackParams& t, double* endpoints, const uint8_t* conv, double* resid, int iters) {
  PolishParams q;
  std::memset(&q, 0, sizeof(q));
  q.kind = t.kind;
  q.N = t.N;
  q.P = t.P;
  q.M = t.M;
  q.K = t.K;
  q.n_hx_terms = t.n_hx_terms;
  q.n_ht_terms = t.n_ht_terms;
  q.flat_eval = t.flat_eval;
  q.scr_slots = t.scr_slots;
  q.shape = t.shape;
  q.hx_terms = t.hx_terms;
  q.hx_off = t.hx_off;
  q.ht_terms = t.ht_terms;
  q.ht_off = t.ht_off;
  q.n_items = t.n_items;
  q.paths_per_hyp = t.paths_per_hyp;
  q.coef_hx = t.coef_hx;
  q.stride_hx = t.stride_hx;
  q.coef_ht = t.coef_ht;
  q.stride_ht = t.stride_ht;
  q.p_start = t.p_start;
  q.p_tgt = t.p_tgt;
  q.p_diff = t.p_diff;
  q.stride_p = t.stride_p;
  q.endpoints = endpoints;
  q.ld = t.ld_out;
  q.conv = conv;
  q.resid = resid;
  q.iters = iters;
  return q;
}

int track_params(const Problem& pb, const ghc_track_args* a, TrackParams& p) {
  p = base_params(pb);
  apply_tuning(pb, a->precision, p);
  if (a->max_steps > 0) p.max_steps = a->max_steps;
  if (a->max_corr > 0) p.max_corr = a->max_corr;
  if (a->incr_steps > 0) p.incr = a->incr_steps;
  p.n_items = a->n_hyp * (long long)(a->paths > 0 ? a->paths : pb.paths);
  p.paths_per_hyp = a->paths > 0 ? a->paths : pb.paths;
  p.start_sols = a->d_start_sols;
  p.ld_start = pb.N;
  p.track_in = nullptr;
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
  p.counter = a->d_counter;
  if (a->corr_tol2 > 0) p.corr_tol2 = a->corr_tol2;
  if (a->first_tol2 > 0) p.first_tol2 = a->first_tol2;
  if (a->dt_max > 0) p.dt_max = a->dt_max;
  if (a->cond_limit > 0) p.cond_limit = a->cond_limit;
  if (a->dt_floor > 0) p.dt_floor = a->dt_floor;
  return GHC_OK;
}

int run_track(const TrackParams& p, const ghc_track_args* a, void* stream) {
  int rc = track_code(launch_track(p, a->precision, a->t_switch, stream, sm_count()));
  if (rc) return rc;
  const bool fp64_state = a->precision == GHC_PREC_FP64 || a->precision == GHC_PREC_MIXED;
  if ((a->polish_iters > 0 || a->d_resid) && fp64_state) {
    if (!a->d_conv) {
      set_error("polish needs d_conv");
      return GHC_ERR_ARG;
    }
    PolishParams q = polish_params(p, (double*)a->d_endpoints, a->d_conv, a->d_resid, a->polish_iters);
    rc = launch_polish(q, stream);
    if (rc) return track_code(rc);
  }
  return GHC_OK;
}

}  // namespace ghc

using namespace ghc;

namespace {

// Pointer array of the reference layout: entry p == base + p * (N+1) complex.  Read on the
// caller's stream (after the work the caller queued there), then checked on the host.
template <typename T>
int regular_base(T* const* d_ptrs, long long n, int N, T** base, cudaStream_t st) {
  std::vector<T*> h((size_t)n);
  if (cudaMemcpyAsync(h.data(), d_ptrs, n * sizeof(T*), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return cuda_fail("copy of pointer array");
  for (long long i = 0; i < n; ++i) {
    if (h[i] != h[0] + 2 * i * (N + 1)) {
      set_error("pointer array is not the reference's regular layout (base + p*(N+1))");
      return GHC_ERR_LAYOUT;
    }
  }
  *base = h[0];
  return GHC_OK;
}

// Tables passed to a drop-in wrapper, read on the caller's stream: the handle's compiled copy when
// they are identical to the files it loaded; else their compiled copy kept in the handle, compiled
// and uploaded (on the caller's stream) only when they differ from the last such tables.
int dropin_tables(Problem& pb, const int* d_hx, const int* d_ht, TrackParams& p, cudaStream_t st) {
  std::vector<int32_t> hx(pb.hx_raw.size()), ht(pb.ht_raw.size());
  if (cudaMemcpyAsync(hx.data(), d_hx, hx.size() * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(ht.data(), d_ht, ht.size() * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return cuda_fail("copy of index tables");
  if (hx == pb.hx_raw && ht == pb.ht_raw) return GHC_OK;
  CallerTables& c = pb.dev.caller;
  if (!(c.dev[0] && hx == c.hx_raw && ht == c.ht_raw)) {
    CallerTables fresh;
    int rc = compile_tables(hx, ht, pb, fresh.hx_terms, fresh.hx_off, fresh.ht_terms, fresh.ht_off);
    if (rc) return rc;
    c.release();
    c = std::move(fresh);
    c.hx_raw = hx;
    c.ht_raw = ht;
    const size_t bytes[4] = {std::max<size_t>(1, c.hx_terms.size()) * 8, c.hx_off.size() * 2,
                             std::max<size_t>(1, c.ht_terms.size()) * 8, c.ht_off.size() * 2};
    const void* src[4] = {c.hx_terms.data(), c.hx_off.data(), c.ht_terms.data(), c.ht_off.data()};
    const size_t used[4] = {c.hx_terms.size() * 8, c.hx_off.size() * 2, c.ht_terms.size() * 8, c.ht_off.size() * 2};
    for (int k = 0; k < 4; ++k) {
      if (cudaMalloc(&c.dev[k], bytes[k]) != cudaSuccess) {
        c.release();
        return cuda_fail("table upload");
      }
      if (used[k] && cudaMemcpyAsync(c.dev[k], src[k], used[k], cudaMemcpyHostToDevice, st) != cudaSuccess) {
        c.release();
        return cuda_fail("table upload");
      }
    }
  }
  p.hx_terms = (const uint64_t*)c.dev[0];
  p.hx_off = (const uint16_t*)c.dev[1];
  p.ht_terms = (const uint64_t*)c.dev[2];
  p.ht_off = (const uint16_t*)c.dev[3];
  p.n_hx_terms = (int)c.hx_terms.size();
  p.n_ht_terms = (int)c.ht_terms.size();
  p.flat_eval = flat_eval_pays(c.hx_off.data(), pb.N);  // the caller's own tables: their own walk
  p.scr_slots = row_nonzeros_max(c.hx_off.data(), pb.N);
  return GHC_OK;
}

// Shared body of the four drop-in wrappers.  Real = float or double.
template <typename Real>
double dropin(const ghc_problem* h, void* stream, int max_steps, int max_corr, int incr, Real** d_start_arr,
              Real** d_track_arr, const int* d_hx, const int* d_ht, const Real* coef_hx, const Real* coef_ht,
              const Real* p_start, const Real* p_tgt, const Real* p_diff, uint8_t* d_conv, uint8_t* d_inf,
              Real* d_debug) {
  if (!h || !d_start_arr || !d_track_arr || !d_hx || !d_ht || !d_conv || !d_inf) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  Problem& pb = const_cast<Problem&>(h->pb);
  int rc = ensure_device(pb);
  if (rc) return rc;
  const bool fp32 = std::is_same<Real, float>::value;
  const long long n = pb.paths;
  cudaStream_t st = (cudaStream_t)stream;
  Real *start_base, *track_base;
  if ((rc = regular_base(d_start_arr, n, pb.N, &start_base, st)) ||
      (rc = regular_base(d_track_arr, n, pb.N, &track_base, st)))
    return rc;
  TrackParams p = base_params(pb);
  apply_tuning(pb, fp32 ? PREC_FP32 : PREC_FP64, p);
  if ((rc = dropin_tables(pb, d_hx, d_ht, p, st))) return rc;
  p.max_steps = max_steps;
  p.max_corr = max_corr;
  p.incr = incr;
  p.n_items = n;
  p.paths_per_hyp = pb.paths;
  p.start_sols = start_base;
  p.ld_start = pb.N + 1;
  p.track_in = track_base;
  p.ld_track = pb.N + 1;
  p.endpoints = track_base;
  p.ld_out = pb.N + 1;
  // scratch: double copies of coefficient/parameter tables + t/dt
  const long long nhx = pb.kind == KIND_P2C ? 2LL * (pb.M + 1) * (pb.K + 1) : 0;
  const long long nht = pb.kind == KIND_P2C ? 2LL * (pb.M + 1) * pb.K : 0;
  const long long npar = pb.kind == KIND_PH ? 2LL * (pb.P + 1) : 0;
  const size_t bytes = sizeof(double) * (size_t)(nhx + nht + 3 * npar + 2 * n) + 256;
  double* s = (double*)scratch(pb, bytes);
  if (!s) return cuda_fail("scratch allocation");
  double* d_chx = s;
  double* d_cht = d_chx + nhx;
  double* d_ps = d_cht + nht;
  double* d_pt = d_ps + npar;
  double* d_pd = d_pt + npar;
  double* d_t = d_pd + npar;
  double* d_dt = d_t + n;
  auto to_double = [&](const Real* src, double* dst, long long cnt) -> int {
    if (cnt <= 0) return 0;
    if (fp32) return launch_f2d((const float*)src, dst, cnt, stream);
    return cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess ? 0 : -1;
  };
  if (pb.kind == KIND_P2C) {
    if (!coef_hx || !coef_ht) {
      set_error("null coefficient table");
      return GHC_ERR_ARG;
    }
    if (to_double(coef_hx, d_chx, nhx) || to_double(coef_ht, d_cht, nht)) return cuda_fail("coefficient copy");
    p.coef_hx = d_chx;
    p.coef_ht = d_cht;
  } else {
    if (!p_start || !p_tgt || !p_diff) {
      set_error("null parameter array");
      return GHC_ERR_ARG;
    }
    if (to_double(p_start, d_ps, npar) || to_double(p_tgt, d_pt, npar) || to_double(p_diff, d_pd, npar))
      return cuda_fail("parameter copy");
    p.p_start = d_ps;
    p.p_tgt = d_pt;
    p.p_diff = d_pd;
  }
  p.conv = d_conv;
  p.infy = d_inf;
  p.t_end = d_t;
  p.dt_end = d_dt;
  p.counter = pb.dev.counter;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  rc = track_code(launch_track(p, fp32 ? PREC_FP32 : PREC_FP64, 0.0, stream, sm_count()));
  cudaEventRecord(e1, st);
  if (!rc && d_debug) {
    if (fp32) rc = launch_debug_f(d_conv, d_t, d_dt, (float*)d_debug, n, stream);
    else rc = launch_debug_d(d_conv, d_t, d_dt, (double*)d_debug, n, stream);
    if (rc) rc = cuda_fail("debug output");
  }
  float ms = 0;
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = cuda_fail("tracker execution");
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  return ms * 1e-3;
}

}  // namespace

extern "C" {

const char* ghc_last_error(void) { return ghc::last_error(); }
int ghc_version(void) { return 1; }

int ghc_problem_load(const char* root, const char* name, ghc_problem** out) {
  if (!root || !name || !out) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  std::unique_ptr<ghc_problem> h(new ghc_problem());
  const int rc = load_problem(root, name, h->pb);
  if (rc) return rc;
  *out = h.release();
  return GHC_OK;
}

void ghc_problem_free(ghc_problem* pb) { delete pb; }

int ghc_problem_get_info(const ghc_problem* h, ghc_problem_info* info) {
  if (!h || !info) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  const Problem& pb = h->pb;
  std::memset(info, 0, sizeof(*info));
  std::strncpy(info->name, pb.name.c_str(), sizeof(info->name) - 1);
  info->kind = pb.kind;
  info->N = pb.N;
  info->P = pb.P;
  info->M = pb.M;
  info->K = pb.K;
  info->paths = pb.paths;
  info->Tx = pb.Tx;
  info->Px = pb.Px;
  info->Tt = pb.Tt;
  info->Pt = pb.Pt;
  info->max_steps = pb.max_steps;
  info->max_corr = pb.max_corr;
  info->incr_steps = pb.incr;
  info->n_hx_terms = (int)pb.hx_off[(size_t)pb.N * pb.N];
  info->n_ht_terms = (int)pb.ht_off.back();
  info->has_p2c_terms = pb.has_terms ? 1 : 0;
  info->subwarp = track_subwarp_width(pb.N);
  info->device = pb.dev.device;
  return GHC_OK;
}

int ghc_problem_start_sols(const ghc_problem* h, double* out) {
  if (!h || !out) return GHC_ERR_ARG;
  std::memcpy(out, h->pb.start_sols.data(), h->pb.start_sols.size() * sizeof(double));
  return GHC_OK;
}

int ghc_problem_params(const ghc_problem* h, double* start, double* target) {
  if (!h) return GHC_ERR_ARG;
  if (start) std::memcpy(start, h->pb.start_params.data(), h->pb.start_params.size() * sizeof(double));
  if (target) std::memcpy(target, h->pb.target_params.data(), h->pb.target_params.size() * sizeof(double));
  return GHC_OK;
}

int ghc_problem_raw_tables(const ghc_problem* h, int32_t* hx, int32_t* ht) {
  if (!h) return GHC_ERR_ARG;
  if (hx) std::memcpy(hx, h->pb.hx_raw.data(), h->pb.hx_raw.size() * 4);
  if (ht) std::memcpy(ht, h->pb.ht_raw.data(), h->pb.ht_raw.size() * 4);
  return GHC_OK;
}

int ghc_problem_compiled_tables(const ghc_problem* h, uint64_t* words, int32_t words_cap, uint16_t* off,
                                int32_t off_cap, int32_t* n_words, int32_t* n_off) {
  if (!h || !n_words || !n_off) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  const Problem& pb = h->pb;
  *n_words = (int32_t)pb.hx_terms.size();
  *n_off = (int32_t)pb.hx_off.size();
  if ((words && words_cap < *n_words) || (off && off_cap < *n_off)) {
    set_error("buffer smaller than the compiled tables");
    return GHC_ERR_LIMIT;
  }
  if (words) std::memcpy(words, pb.hx_terms.data(), pb.hx_terms.size() * sizeof(uint64_t));
  if (off) std::memcpy(off, pb.hx_off.data(), pb.hx_off.size() * sizeof(uint16_t));
  return GHC_OK;
}

int ghc_p2c(const ghc_problem* h, const double* start, const double* target, double* hx, double* ht, int exact_ht) {
  if (!h || !start || !target || !hx || !ht) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  return p2c_host(h->pb, start, target, hx, ht, exact_ht);
}

int ghc_p2c_device(const ghc_problem* h, int64_t n_hyp, const double* d_start, const double* d_targets, double* d_hx,
                   double* d_ht, int exact_ht, void* stream) {
  if (!h || !d_start || !d_targets || !d_hx || !d_ht || n_hyp < 0) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  Problem& pb = const_cast<Problem&>(h->pb);
  if (pb.kind != KIND_P2C || !pb.has_terms) {
    set_error("problem has no coefficient expressions (p2c_terms.txt)");
    return GHC_ERR_NOP2C;
  }
  int rc = ensure_device(pb);
  if (rc) return rc;
  P2CParams p;
  p.M = pb.M;
  p.K = pb.K;
  p.P = pb.P;
  p.n_terms = (int)pb.p2c.size();
  p.term_k = pb.dev.t_k;
  p.term_coef = pb.dev.t_coef;
  p.term_nf = pb.dev.t_nf;
  p.term_fac_off = pb.dev.t_fac_off;
  p.term_fac = pb.dev.t_fac;
  p.k_off = pb.dev.k_off;
  p.n_hyp = n_hyp;
  p.p_start = d_start;
  p.p_tgt = d_targets;
  p.coef_hx = d_hx;
  p.coef_ht = d_ht;
  p.exact_ht = exact_ht;
  rc = launch_p2c(p, stream);
  if (rc == -10) {
    set_error("Max_Order_Of_T above 8");
    return GHC_ERR_RANGE;
  }
  return rc ? cuda_fail("p2c launch") : GHC_OK;
}

int ghc_track(const ghc_problem* h, const ghc_track_args* a, void* stream) {
  if (!h || !a || a->n_hyp < 0) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  if (a->n_hyp == 0) return GHC_OK;
  if (!a->d_start_sols || !a->d_endpoints || !a->d_counter) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  Problem& pb = const_cast<Problem&>(h->pb);
  int rc = ensure_device(pb);
  if (rc) return rc;
  TrackParams p;
  if ((rc = track_params(pb, a, p))) return rc;
  return run_track(p, a, stream);
}

int ghc_count_results(int32_t N, int32_t paths, const double* z, const uint8_t* conv, const uint8_t* inf,
                      double imag_tol, double dup_tol, ghc_counts* out) {
  if (N < 1 || paths < 0 || !z || !conv || !inf || !out) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  // Evaluations::Evaluate_GPUHC_Sols (Evaluations.cpp:88-110)
  ghc_counts c = {0, 0, 0, 0};
  for (int bs = 0; bs < paths; ++bs) {
    if (conv[bs]) ++c.converged;
    if (inf[bs]) ++c.infinity;
    if (conv[bs]) {
      int nreal = 0;
      for (int v = 0; v < N; ++v)
        if (std::fabs(z[2 * ((size_t)bs * N + v) + 1]) <= imag_tol) ++nreal;
      if (nreal == N) ++c.real;
    }
  }
  // Evaluations::Find_Unique_Sols (Evaluations.cpp:127-176): the skip set is
  // replaced (not merged) by each new duplicate set; members of a duplicate
  // cluster are not counted.
  std::set<int> skip, dup;
  for (int bs = 0; bs < paths; ++bs) {
    if (!conv[bs]) continue;
    if (!skip.empty()) {
      if (skip.count(bs)) continue;
      dup.clear();
    }
    for (int ds = bs + 1; ds < paths; ++ds) {
      int same = 0;
      for (int v = 0; v < N; ++v) {
        const double* a = z + 2 * ((size_t)bs * N + v);
        const double* b = z + 2 * ((size_t)ds * N + v);
        if (std::fabs(a[0] - b[0]) < dup_tol && std::fabs(a[1] - b[1]) < dup_tol) ++same;
      }
      if (same == N) dup.insert(ds);
    }
    if (dup.empty()) ++c.unique;
    else skip = dup;
  }
  *out = c;
  return GHC_OK;
}

int ghc_set_tuning(ghc_problem* h, int32_t precision, int32_t variant, int32_t flat) {
  if (!h || (variant != 0 && variant != 1) || flat < -1 || flat > 2 ||
      (precision != GHC_PREC_FP64 && precision != GHC_PREC_FP32 && precision != GHC_PREC_MIXED)) {
    set_error("bad tuning argument");
    return GHC_ERR_ARG;
  }
  Problem& pb = h->pb;
  if (precision != GHC_PREC_FP32) {
    pb.tune_variant[0] = variant;
    pb.tune_flat[0] = flat;
  }
  if (precision != GHC_PREC_FP64) {
    pb.tune_variant[1] = variant;
    pb.tune_flat[1] = flat;
  }
  return GHC_OK;
}

int ghc_get_tuning(const ghc_problem* h, int32_t precision, int32_t* variant, int32_t* flat) {
  if (!h || !variant || !flat || (precision != GHC_PREC_FP64 && precision != GHC_PREC_FP32)) {
    set_error("bad tuning argument");
    return GHC_ERR_ARG;
  }
  const int k = precision == GHC_PREC_FP32 ? 1 : 0;
  *variant = h->pb.tune_variant[k];
  *flat = h->pb.tune_flat[k];
  return GHC_OK;
}

int ghc_autotune(ghc_problem* h, const ghc_track_args* a, void* stream, ghc_tune_choice* best) {
  if (!h || !a || !best) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  Problem& pb = h->pb;
  const int prec = a->precision;
  if (prec != GHC_PREC_FP64 && prec != GHC_PREC_FP32 && prec != GHC_PREC_MIXED) {
    set_error("unknown precision mode");
    return GHC_ERR_ARG;
  }
  struct Cand {
    int v64, v32, flat;
  };
  std::vector<Cand> cand;
  const bool mixed = prec == GHC_PREC_MIXED;
  const bool balanced = pb.hx_off[(size_t)pb.N * pb.N + 1] != kNoLanes;
  for (int f = balanced ? 2 : 1; f >= (pb.N > 16 ? 1 : 0); --f)
    for (int v = 0; v < 2; ++v)
      for (int w = 0; w < (mixed ? 2 : 1); ++w) cand.push_back({v, mixed ? w : v, f});
  const int keep_v[2] = {pb.tune_variant[0], pb.tune_variant[1]};
  const int keep_f[2] = {pb.tune_flat[0], pb.tune_flat[1]};
  auto apply = [&](const Cand& c) {
    if (prec == GHC_PREC_FP32) {
      pb.tune_variant[1] = c.v64;
      pb.tune_flat[1] = c.flat;
    } else {
      pb.tune_variant[0] = c.v64;
      pb.tune_flat[0] = c.flat;
      if (mixed) {
        pb.tune_variant[1] = c.v32;
        pb.tune_flat[1] = c.flat;
      }
    }
  };
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return cuda_fail("autotune events");
  double best_ms = HUGE_VAL;
  int rc = GHC_OK;
  Cand win = cand[0];
  for (const auto& c : cand) {
    apply(c);
    for (int rep = 0; rep < 2 && !rc; ++rep) {  // the first run warms up (kernel attributes, caches)
      cudaEventRecord(e0, st);
      rc = ghc_track(h, a, stream);
      cudaEventRecord(e1, st);
    }
    if (rc) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = cuda_fail("autotune run");
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      win = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {  // leave the handle as it was
    pb.tune_variant[0] = keep_v[0];
    pb.tune_variant[1] = keep_v[1];
    pb.tune_flat[0] = keep_f[0];
    pb.tune_flat[1] = keep_f[1];
    return rc;
  }
  apply(win);
  best->variant = win.v64;
  best->variant_f32 = mixed ? win.v32 : (prec == GHC_PREC_FP32 ? win.v64 : pb.tune_variant[1]);
  best->flat = win.flat;
  best->ms = best_ms;
  best->candidates = (int)cand.size();
  return GHC_OK;
}

int ghc_count_results_device(int32_t N, int32_t paths, int64_t n_hyp, const double* d_endpoints,
                             const uint8_t* d_conv, const uint8_t* d_inf, double imag_tol, double dup_tol,
                             ghc_counts* d_counts, uint8_t* d_class, void* stream) {
  if (N < 1 || N > kMaxN || paths < 0 || n_hyp < 0) {
    set_error("bad size");
    return GHC_ERR_ARG;
  }
  if (n_hyp == 0 || paths == 0) return GHC_OK;
  if (!d_endpoints || !d_conv || !d_inf || !d_counts) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  if (paths > 200000) {
    set_error("more than 200,000 paths per hypothesis");
    return GHC_ERR_RANGE;
  }
  if (launch_results(N, paths, n_hyp, d_endpoints, d_conv, d_inf, imag_tol, dup_tol, (int*)d_counts, d_class,
                     stream))
    return cuda_fail("result counts");
  return GHC_OK;
}

double ghc_kernel_HC_Solver_P2C(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                float** d_startSols_array, float** d_Track_array, const int* d_Hx_idx,
                                const int* d_Ht_idx, const float* d_phc_coeffs_Hx, const float* d_phc_coeffs_Ht,
                                uint8_t* d_conv, uint8_t* d_inf, float* d_debug) {
  if (pb && pb->pb.kind != KIND_P2C) {
    set_error("not a P2C problem");
    return GHC_ERR_ARG;
  }
  return dropin<float>(pb, stream, max_steps, max_corr, incr, d_startSols_array, d_Track_array, d_Hx_idx, d_Ht_idx,
                       d_phc_coeffs_Hx, d_phc_coeffs_Ht, nullptr, nullptr, nullptr, d_conv, d_inf, d_debug);
}

double ghc_kernel_HC_Solver_P2C_z(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                  double** d_startSols_array, double** d_Track_array, const int* d_Hx_idx,
                                  const int* d_Ht_idx, const double* d_phc_coeffs_Hx,
                                  const double* d_phc_coeffs_Ht, uint8_t* d_conv, uint8_t* d_inf,
                                  double* d_debug) {
  if (pb && pb->pb.kind != KIND_P2C) {
    set_error("not a P2C problem");
    return GHC_ERR_ARG;
  }
  return dropin<double>(pb, stream, max_steps, max_corr, incr, d_startSols_array, d_Track_array, d_Hx_idx, d_Ht_idx,
                        d_phc_coeffs_Hx, d_phc_coeffs_Ht, nullptr, nullptr, nullptr, d_conv, d_inf, d_debug);
}

double ghc_kernel_HC_Solver_PH(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                               float** d_startSols_array, float** d_Track_array, const float* d_startParams,
                               const float* d_targetParams, const float* d_diffParams, const int* d_Hx_idx,
                               const int* d_Ht_idx, uint8_t* d_conv, uint8_t* d_inf, float* d_debug) {
  if (pb && pb->pb.kind != KIND_PH) {
    set_error("not a PH problem");
    return GHC_ERR_ARG;
  }
  return dropin<float>(pb, stream, max_steps, max_corr, incr, d_startSols_array, d_Track_array, d_Hx_idx, d_Ht_idx,
                       nullptr, nullptr, d_startParams, d_targetParams, d_diffParams, d_conv, d_inf, d_debug);
}

double ghc_kernel_HC_Solver_PH_z(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                 double** d_startSols_array, double** d_Track_array, const double* d_startParams,
                                 const double* d_targetParams, const double* d_diffParams, const int* d_Hx_idx,
                                 const int* d_Ht_idx, uint8_t* d_conv, uint8_t* d_inf, double* d_debug) {
  if (pb && pb->pb.kind != KIND_PH) {
    set_error("not a PH problem");
    return GHC_ERR_ARG;
  }
  return dropin<double>(pb, stream, max_steps, max_corr, incr, d_startSols_array, d_Track_array, d_Hx_idx, d_Ht_idx,
                        nullptr, nullptr, d_startParams, d_targetParams, d_diffParams, d_conv, d_inf, d_debug);
}

int ghc_solve_host(const ghc_problem* h, int32_t precision, int64_t n_hyp, const double* h_targets, double t_switch,
                   int32_t polish_iters, double* h_endpoints, uint8_t* h_status, uint8_t* h_conv, uint8_t* h_inf,
                   int32_t* h_steps, double* h_ms) {
  if (!h || !h_endpoints || n_hyp < 1) {
    set_error("null argument");
    return GHC_ERR_ARG;
  }
  if (precision != GHC_PREC_FP64 && precision != GHC_PREC_FP32 && precision != GHC_PREC_MIXED) {
    set_error("unknown precision mode");
    return GHC_ERR_ARG;
  }
  Problem& pb = const_cast<Problem&>(h->pb);
  if (!h_targets) n_hyp = 1;
  int rc = ensure_device(pb);
  if (rc) return rc;
  const bool fp32 = precision == GHC_PREC_FP32;
  const long long n = n_hyp * (long long)pb.paths;
  const int N = pb.N, P1 = pb.P + 1;
  const size_t rs = fp32 ? sizeof(float) : sizeof(double);
  const long long nhx = 2LL * (pb.M + 1) * (pb.K + 1), nht = 2LL * (pb.M + 1) * pb.K;
  // all device buffers from one grow-only arena of the handle (no allocation once it is large
  // enough), work on the handle's own non-blocking stream
  const size_t sz[10] = {2 * (size_t)pb.paths * N * rs,
                         2 * (size_t)P1 * sizeof(double),
                         2 * (size_t)P1 * n_hyp * sizeof(double),
                         2 * (size_t)P1 * n_hyp * sizeof(double),
                         pb.kind == KIND_P2C ? nhx * n_hyp * sizeof(double) : 0,
                         pb.kind == KIND_P2C ? std::max(nht, 1LL) * n_hyp * sizeof(double) : 0,
                         2 * (size_t)n * N * rs,
                         3 * (size_t)n,
                         (size_t)n * 8,
                         (size_t)n * 16};
  size_t total = 0;
  for (size_t b : sz) total += (b + 255) & ~(size_t)255;
  if (total > pb.dev.solve_bytes) {
    cudaFree(pb.dev.solve_arena);
    pb.dev.solve_arena = nullptr;
    pb.dev.solve_bytes = 0;
    if (cudaMalloc(&pb.dev.solve_arena, total) != cudaSuccess) return cuda_fail("allocation");
    pb.dev.solve_bytes = total;
  }
  if (!pb.dev.solve_stream) {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return cuda_fail("stream");
    pb.dev.solve_stream = s;
  }
  void* buf[10];
  {
    char* q = (char*)pb.dev.solve_arena;
    for (int k = 0; k < 10; ++k) {
      buf[k] = sz[k] ? q : nullptr;
      q += (sz[k] + 255) & ~(size_t)255;
    }
  }
  void* d_start = buf[0];
  double* d_ps = (double*)buf[1];
  double* d_tg = (double*)buf[2];
  double* d_pd = (double*)buf[3];
  double* d_hx = (double*)buf[4];
  double* d_ht = (double*)buf[5];
  void* d_ep = buf[6];
  uint8_t* d_flags = (uint8_t*)buf[7];
  int32_t* d_steps = (int32_t*)buf[8];  // steps, corrector iterations
  double* d_tdt = (double*)buf[9];      // t_end, dt_end
  if (pb.kind == KIND_P2C && !pb.has_terms) {
    set_error("problem has no coefficient expressions (p2c_terms.txt)");
    return GHC_ERR_NOP2C;
  }
  cudaStream_t st = (cudaStream_t)pb.dev.solve_stream;
  cudaEvent_t ev[4];
  for (auto& e : ev) cudaEventCreate(&e);
  std::vector<float> sf;
  cudaEventRecord(ev[0], st);
  if (fp32) {
    sf.resize(pb.start_sols.size());
    for (size_t i = 0; i < sf.size(); ++i) sf[i] = (float)pb.start_sols[i];
    cudaMemcpyAsync(d_start, sf.data(), sf.size() * 4, cudaMemcpyHostToDevice, st);
  } else {
    cudaMemcpyAsync(d_start, pb.start_sols.data(), pb.start_sols.size() * 8, cudaMemcpyHostToDevice, st);
  }
  cudaMemcpyAsync(d_ps, pb.start_params.data(), 2 * (size_t)P1 * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_tg, h_targets ? h_targets : pb.target_params.data(), 2 * (size_t)P1 * n_hyp * 8,
                  cudaMemcpyHostToDevice, st);
  cudaEventRecord(ev[1], st);
  if (pb.kind == KIND_P2C) {
    rc = ghc_p2c_device(h, n_hyp, d_ps, d_tg, d_hx, d_ht, 0, st);
  } else {
    rc = launch_diff_d(d_ps, d_tg, d_pd, n_hyp, P1, st) ? cuda_fail("diff") : GHC_OK;
  }
  ghc_track_args a;
  std::memset(&a, 0, sizeof(a));
  a.n_hyp = n_hyp;
  a.precision = precision;
  a.t_switch = t_switch;
  a.polish_iters = polish_iters;
  a.d_start_sols = d_start;
  a.d_coef_hx = d_hx;
  a.d_coef_ht = d_ht;
  a.d_p_start = d_ps;
  a.d_p_target = d_tg;
  a.d_p_diff = d_pd;
  a.d_endpoints = d_ep;
  a.d_status = d_flags;
  a.d_conv = d_flags + n;
  a.d_inf = d_flags + 2 * n;
  a.d_steps = d_steps;
  a.d_corr = d_steps + n;
  a.d_t_end = d_tdt;
  a.d_dt_end = d_tdt + n;
  a.d_counter = pb.dev.counter;
  if (!rc) rc = ghc_track(h, &a, st);
  cudaEventRecord(ev[2], st);
  std::vector<float> ef;
  if (!rc) {
    if (fp32) {
      ef.resize(2 * (size_t)n * N);
      cudaMemcpyAsync(ef.data(), d_ep, ef.size() * 4, cudaMemcpyDeviceToHost, st);
    } else {
      cudaMemcpyAsync(h_endpoints, d_ep, 2 * (size_t)n * N * 8, cudaMemcpyDeviceToHost, st);
    }
    if (h_status) cudaMemcpyAsync(h_status, d_flags, n, cudaMemcpyDeviceToHost, st);
    if (h_conv) cudaMemcpyAsync(h_conv, d_flags + n, n, cudaMemcpyDeviceToHost, st);
    if (h_inf) cudaMemcpyAsync(h_inf, d_flags + 2 * n, n, cudaMemcpyDeviceToHost, st);
    if (h_steps) cudaMemcpyAsync(h_steps, d_steps, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
  }
  cudaEventRecord(ev[3], st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = cuda_fail("solve");
  if (!rc && fp32)
    for (size_t i = 0; i < ef.size(); ++i) h_endpoints[i] = ef[i];
  if (h_ms) {
    float m = 0;
    cudaEventElapsedTime(&m, ev[0], ev[1]);
    h_ms[0] = m;
    cudaEventElapsedTime(&m, ev[1], ev[2]);
    h_ms[1] = m;
    cudaEventElapsedTime(&m, ev[2], ev[3]);
    h_ms[2] = m;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}

}  // extern "C"
