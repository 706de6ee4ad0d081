// ghc_internal.h -- definitions shared by the host library and the CUDA tracker.
//
// Problem layout (reference, GPU-HC/magmaHC/GPU_HC_Solver.cpp:44-83):
//   N unknowns, P parameters, M unique coefficients (P2C), K = max order of t,
//   dHdx table [N][N][Tx][Px], dHdt table [N][Tt][Pt]   (P2C, row-major)
//   dHdx table [N*Tx*Px][N],   dHdt table [Tt*Pt][N]     (PH, transposed)
//
// The device never walks the raw tables.  The host compiles them once into
// "terms": one 64-bit word per non-padding monomial term, grouped by Jacobian
// entry (row, col) for H_x and by row for H / H_t, with CSR offsets; the words
// are stored row-interleaved (term k of row r at k * N + r).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GHC_HD __host__ __device__
#else
#define GHC_HD
#endif

namespace ghc {

enum Kind : int { KIND_P2C = 0, KIND_PH = 1 };
enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1, PREC_MIXED = 2 };
enum Status : int { ST_CONVERGED = 0, ST_DIVERGED = 1, ST_STEP_CAP = 2, ST_NONFINITE = 3, ST_SINGULAR = 4 };

constexpr int kMaxN = 32;
constexpr int kMaxVarsPerTerm = 7;

// term word layout
//   bits  0.. 7  integer scale (int8)
//   bits  8..10  number of variable slots nv (the same for every term of a table; slot N = the constant 1)
//   bits 11..20  P2C: coefficient index k (0..1023)
//   bits 11..16  PH : parameter index a ; bits 17..22 PH: parameter index b
//   bit  23      H_x terms: the last term of its entry (row, column)
//   bits 24..58  variable indices, 5 bits each, table order
//   bits 49..58  words of the balanced H_x walk (at most 5 variable slots): the entry's row
//                (49..53) and its slot among the row's non-zero entries (54..58)
//   bits 59..63  H_x terms: the Jacobian column of the term (its row is implied by the CSR row)
GHC_HD inline int term_scale(uint64_t w) { return (int)(int8_t)(w & 0xffu); }
GHC_HD inline int term_nv(uint64_t w) { return (int)((w >> 8) & 7u); }
GHC_HD inline int term_coef(uint64_t w) { return (int)((w >> 11) & 0x3ffu); }
GHC_HD inline int term_pa(uint64_t w) { return (int)((w >> 11) & 0x3fu); }
GHC_HD inline int term_pb(uint64_t w) { return (int)((w >> 17) & 0x3fu); }
GHC_HD inline int term_var(uint64_t w, int q) { return (int)((w >> (24 + 5 * q)) & 31u); }
GHC_HD inline int term_col(uint64_t w) { return (int)(w >> 59); }
constexpr uint64_t kTermLast = 1ull << 23;
GHC_HD inline bool term_last(uint64_t w) { return (w & kTermLast) != 0; }
GHC_HD inline int term_dst_row(uint64_t w) { return (int)((w >> 49) & 31u); }
GHC_HD inline int term_dst_slot(uint64_t w) { return (int)((w >> 54) & 31u); }
constexpr int kMaxVarsBalanced = 5;

// lanes per path (the sub-warp width) for N unknowns
GHC_HD constexpr int subwarp_width(int N) { return N <= 4 ? 4 : N <= 8 ? 8 : N <= 16 ? 16 : 32; }

// Sizes that get the balanced H_x walk (tables and kernel code): every size.  B200, tuned: 5-point
// (N = 6) +11 %, 30x30 (N = 30) +4 %.  (When the walk was chosen at run time inside one kernel, the
// balanced code cost the N = 12 problems 4-5 % on their row-wise walk; each walk is its own kernel
// now, so building it costs the other walks nothing.)
GHC_HD constexpr bool balanced_walk_built(int) { return true; }

// The compiled H_x offsets: [N*N+1] CSR offsets of the terms per (row, column), then the
// balanced walk: [1] its first word in the term array (kNoLanes: no balanced walk) and
// [W] the number of terms each lane walks.
constexpr uint16_t kNoLanes = 0xffff;
GHC_HD constexpr int hx_off_len(int N) { return N * N + 2 + subwarp_width(N); }

// The H_x walk the tracker should use by default: 0 entry by entry, 1 each lane its
// row as one term list (staging the entries in shared memory), 2 the entries dealt
// to all lanes balanced by term count.  Entry by entry, a sub-warp runs, for every
// column, as many iterations as the row with the most terms in that column;
// row-wise as many as the longest row; balanced as many as the longest lane.
// Above 16 unknowns the kernels never walk entry by entry (that code would be
// unrolled N times).  hx_off: the compiled H_x offsets (hx_off_len(N) entries).
// The most structurally non-zero entries in one row of H_x: the row-wise walk stages each
// row's non-zero entries in that many shared-memory slots.
inline int row_nonzeros_max(const uint16_t* hx_off, int N) {
  int most = 0;
  for (int r = 0; r < N; ++r) {
    int nz = 0;
    for (int i = 0; i < N; ++i) nz += hx_off[r * N + i + 1] > hx_off[r * N + i];
    if (nz > most) most = nz;
  }
  return most;
}

inline int flat_eval_pays(const uint16_t* hx_off, int N) {
  int longest = 0, per_entry = 0, walk = 1;
  for (int r = 0; r < N; ++r) {
    const int len = hx_off[r * N + N] - hx_off[r * N];
    if (len > longest) longest = len;
  }
  if (hx_off[N * N + 1] != kNoLanes) {
    // the balanced walk moves the same shared-memory traffic onto more lanes and adds a
    // sub-warp synchronisation: by default only where the rows are uneven (longest row at
    // least 1.4x the longest lane; the autotuner times it everywhere it is built)
    int lane = 0;
    for (int l = 0; l < subwarp_width(N); ++l)
      if (hx_off[N * N + 2 + l] > lane) lane = hx_off[N * N + 2 + l];
    if (10 * longest >= 14 * lane) {
      longest = lane;
      walk = 2;
    }
  }
  for (int i = 0; i < N; ++i) {
    int m = 0;
    for (int r = 0; r < N; ++r) {
      const int c = hx_off[r * N + i + 1] - hx_off[r * N + i];
      if (c > m) m = c;
    }
    per_entry += m;
  }
  return 4 * per_entry > 5 * longest ? walk : 0;
}

// Term shape of a problem: (variable slots per H_x term, per H_t term).  Every term of a
// table has parts - 1 - (coefficient slots) variable slots (compile_tables keeps slot N,
// the constant 1); the two shapes of the shipped problems get kernels with straight-line
// term evaluation, any other shape the general kernel.
enum EvalShape : int { EVAL_GENERAL = 0, EVAL_1_2 = 1, EVAL_2_3 = 2 };
inline int eval_shape_of(int kind, int Px, int Pt) {
  const int c = kind == KIND_PH ? 2 : 1, a = Px - 1 - c, b = Pt - 1 - c;
  return (a == 1 && b == 2) ? EVAL_1_2 : (a == 2 && b == 3) ? EVAL_2_3 : EVAL_GENERAL;
}
GHC_HD constexpr int shape_nvx(int S) { return S == EVAL_1_2 ? 1 : S == EVAL_2_3 ? 2 : -1; }
GHC_HD constexpr int shape_nvt(int S) { return S == EVAL_1_2 ? 2 : S == EVAL_2_3 ? 3 : -1; }

// Everything the tracker kernel needs, by value.
struct TrackParams {
  // problem
  int kind, N, P, M, K;
  int max_steps, max_corr, incr;
  int n_hx_terms, n_ht_terms;
  int flat_eval;              // H_x walk: 0 entry-wise, 1 row-wise, 2 balanced (flat_eval_pays() or the autotuner)
  int shape;                  // eval_shape_of() of the problem
  int scr_slots;              // row_nonzeros_max() of the tables
  int variant;                // compiled register-budget variant (0 or 1)
  int variant_f32, flat_eval_f32;  // the FP32 phase's choices in mixed precision
  const uint64_t* hx_terms;   // device
  const uint16_t* hx_off;     // device [N*N+1]
  const uint64_t* ht_terms;   // device
  const uint16_t* ht_off;     // device [N+1]
  // work items: item i = hypothesis i / paths_per_hyp, start path i % paths_per_hyp
  long long n_items;
  int paths_per_hyp;
  // inputs (complex arrays interleaved re,im; state precision RS for sols)
  const void* start_sols;  // [paths_per_hyp][ld_start]
  int ld_start;
  const void* track_in;    // optional initial track [n_items][ld_track] (nullptr -> start_sols)
  int ld_track;
  int start_other;         // start_sols / track_in hold the other precision than the kernel's
  int track_other;         //   (double for the FP32 tracker, float for the FP64 tracker)
  // resuming: per item start t and step (nullptr -> 0 and the initial step), and the
  // step / corrector counts already in steps / corr
  const double* t_in;
  const double* dt_in;
  int resume;
  const double* coef_hx;   // P2C [n_hyp][(M+1)(K+1)] complex double
  long long stride_hx;     // in complex entries (0 -> shared by all hypotheses)
  const double* coef_ht;   // P2C [n_hyp][(M+1)K]
  long long stride_ht;
  const double* p_start;   // PH [P+1]
  const double* p_tgt;     // PH [n_hyp][P+1]
  const double* p_diff;    // PH [n_hyp][P+1]
  long long stride_p;
  // outputs
  void* endpoints;         // [n_items][ld_out] complex RS
  int ld_out;
  uint8_t* status;
  uint8_t* conv;
  uint8_t* infy;
  int* steps;
  int* corr;
  double* t_end;
  double* dt_end;
  // scratch
  int* counter;            // one int, used as unsigned: zeroed before every launch that steals work
  int spread;              // set by the launcher: one path per warp (launches smaller than one wave)
  // handover (first phase of mixed precision): stop at t_handover (> 0) or after
  // fail_limit (> 0) consecutive failed steps or on divergence, keeping the last accepted point
  double t_handover;
  int fail_limit;
  // step control (reference: corr_tol2 = 1e-6, first_tol2 = dt_max = +inf)
  double corr_tol2;   // corrector success: |dx|^2 < corr_tol2 |x|^2
  double first_tol2;  // reject when the first Newton update has |dx|^2 > first_tol2 |x|^2
  double dt_max;      // step-size cap
  // mixed tracker: stop a path (handover) after a step in which a solve's pivot magnitudes spanned
  // more than cond_limit, or one was NaN (0: never), or once its step falls below dt_floor (0: never)
  double cond_limit;
  double dt_floor;
};

struct PolishParams {
  int kind, N, P, M, K;
  int n_hx_terms, n_ht_terms;
  int flat_eval, scr_slots, shape;
  const uint64_t* hx_terms;
  const uint16_t* hx_off;
  const uint64_t* ht_terms;
  const uint16_t* ht_off;
  long long n_items;
  int paths_per_hyp;
  const double* coef_hx;
  long long stride_hx;
  const double* coef_ht;
  long long stride_ht;
  const double* p_start;
  const double* p_tgt;
  const double* p_diff;
  long long stride_p;
  double* endpoints;  // [n_items][ld] complex double, in/out
  int ld;
  const uint8_t* conv;
  double* resid;      // [n_items] |H(x,1)| after polish, -1 when not converged
  int iters;
};

struct P2CParams {
  int M, K, P;
  int n_terms;
  const int* term_k;        // [n_terms]
  const double* term_coef;  // [n_terms]
  const int* term_nf;       // [n_terms]
  const int* term_fac_off;  // [n_terms+1]
  const int* term_fac;      // factors (param indices)
  const int* k_off;         // [M+1] term ranges per coefficient
  long long n_hyp;
  const double* p_start;    // [P+1] complex
  const double* p_tgt;      // [n_hyp][P+1] complex
  double* coef_hx;          // [n_hyp][(M+1)(K+1)]
  double* coef_ht;          // [n_hyp][(M+1)K]
  int exact_ht;
};

// launch entry points implemented in tracker.cu / p2c.cu
// precision PREC_MIXED runs two launches (FP32 to t_switch with handover, then FP64) and
// needs p.steps, p.corr, p.t_end and p.dt_end; t_switch is ignored by the other modes.
int launch_track(const TrackParams& p, int precision, double t_switch, void* stream, int n_sm);
int launch_polish(const PolishParams& p, void* stream);
int launch_p2c(const P2CParams& p, void* stream);
int track_subwarp_width(int N);
// results.cu: per-hypothesis counts (int[4] per hypothesis) and class bytes on the device
size_t results_smem_bytes(int paths);
int launch_results(int N, int paths, long long n_hyp, const double* z, const uint8_t* conv, const uint8_t* inf,
                   double imag_tol, double dup_tol, int* counts, uint8_t* cls, void* stream);

}  // namespace ghc
