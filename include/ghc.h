/*
 * ghc.h -- C ABI of the B200 homotopy-continuation path tracker.
 *
 * Plain C types only (pointers, sizes, ints).  Complex arrays are interleaved
 * (re, im) pairs.  Functions taking "d_" pointers expect device memory on the
 * current CUDA device; "h_" pointers are host memory.  Every function returns
 * GHC_OK (0) or a negative GHC_ERR_* code; ghc_last_error() returns a message.
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the C-H-Chien/Homotopy-Continuation-Tracker-on-GPU tree).
 */
#ifndef GHC_H
#define GHC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GHC_OK 0
#define GHC_ERR_ARG (-1)      /* bad argument */
#define GHC_ERR_IO (-2)       /* missing or unreadable file */
#define GHC_ERR_FORMAT (-3)   /* malformed YAML or table */
#define GHC_ERR_RANGE (-4)    /* table index out of range / size unsupported */
#define GHC_ERR_CUDA (-5)     /* CUDA runtime error */
#define GHC_ERR_LAYOUT (-6)   /* pointer arrays not a regular strided layout */
#define GHC_ERR_NOP2C (-7)    /* problem has no coefficient expressions */
#define GHC_ERR_LIMIT (-8)    /* request exceeds a fixed capacity */

#define GHC_KIND_P2C 0
#define GHC_KIND_PH 1

#define GHC_PREC_FP64 0  /* plain FP64 tracker */
#define GHC_PREC_FP32 1  /* reference precision (complex FP32) */
#define GHC_PREC_MIXED 2 /* FP64 state and residual with FP32 H_x, H_t and LU; FP64 after ill-conditioning */

#define GHC_STATUS_CONVERGED 0
#define GHC_STATUS_DIVERGED 1 /* |x|^2 > 1e14 in the corrector ("infinity") */
#define GHC_STATUS_STEP_CAP 2 /* ran out of steps before t = 1 */
#define GHC_STATUS_NONFINITE 3 /* stopped with a NaN or infinite component in its track */
#define GHC_STATUS_SINGULAR 4  /* stopped (step cap or handover) after a step in which a solve had a zero pivot */

typedef struct ghc_problem ghc_problem;

typedef struct {
  char name[96];
  int32_t kind;                        /* GHC_KIND_P2C or GHC_KIND_PH */
  int32_t N, P, M, K;                  /* unknowns, parameters, coefficients (P2C), max order of t */
  int32_t paths;                       /* start solutions */
  int32_t Tx, Px, Tt, Pt;              /* table shapes */
  int32_t max_steps, max_corr, incr_steps;
  int32_t n_hx_terms, n_ht_terms;      /* non-padding monomial terms */
  int32_t has_p2c_terms;               /* p2c_terms.txt present (host/device P2C available) */
  int32_t subwarp;                     /* lanes per path on the GPU */
  int32_t device;                      /* device holding the handle's compiled tables and work counter
                                          (uploaded by its first tracking call), -1: none */
} ghc_problem_info;

/* Result counts of one hypothesis. */
typedef struct {
  int32_t converged, real, infinity, unique;
} ghc_counts;

/* Last error message of the calling thread. */
const char* ghc_last_error(void);
int ghc_version(void);

/* ---------------------------------------------------------------------------
 * Problem data.
 * Replaces GPU_HC_Solver::GPU_HC_Solver (GPU-HC/magmaHC/GPU_HC_Solver.cpp:40-102),
 * GPU_HC_Solver::Read_Problem_Data (GPU_HC_Solver.cpp:142-181) and the readers
 * Data_Reader::Read_Start_Params / Read_Target_Params / Read_Start_Sols /
 * Read_dHdx_Indices / Read_dHdt_Indices (GPU-HC/magmaHC/Data_Reader.cpp:91-225).
 * Loads <problems_root>/<name>/gpuhc_settings.yaml and the five text files,
 * validates every table index, and compiles the tables for the device.
 * ------------------------------------------------------------------------- */
int ghc_problem_load(const char* problems_root, const char* name, ghc_problem** out);
void ghc_problem_free(ghc_problem* pb);
int ghc_problem_get_info(const ghc_problem* pb, ghc_problem_info* info);
/* h_out: [paths][N] complex */
int ghc_problem_start_sols(const ghc_problem* pb, double* h_out);
/* h_start, h_target: [P+1] complex each, slot P = 1 (Data_Reader.cpp:161-183) */
int ghc_problem_params(const ghc_problem* pb, double* h_start, double* h_target);
/* raw tables as read: h_hx [N*N*Tx*Px], h_ht [N*Tt*Pt] */
int ghc_problem_raw_tables(const ghc_problem* pb, int32_t* h_hx, int32_t* h_ht);
/* The compiled H_x tables the tracker walks (for inspection): *n_words 64-bit term words (the
 * row-interleaved block: term k of row r at k*N + r; then the balanced walk's block: term q of
 * lane l at first + q*W + l) and *n_off 16-bit offsets (N*N+1 CSR offsets per (row, column),
 * the balanced block's first word or 0xffff when the size has no balanced walk, W lane lengths).
 * Copies when h_words / h_off are non-null and hold *n_words / *n_off entries (GHC_ERR_LIMIT if
 * the capacities are smaller); null buffers only return the sizes. */
int ghc_problem_compiled_tables(const ghc_problem* pb, uint64_t* h_words, int32_t words_cap, uint16_t* h_off,
                                int32_t off_cap, int32_t* n_words, int32_t* n_off);

/* ---------------------------------------------------------------------------
 * Coefficient homotopy tables (P2C problems).
 * Replaces magmaHCWrapper::p2c_<problem> (GPU-HC/magmaHC/PHC_Coeffs/p2c-*.h)
 * called from Data_Reader::Construct_Coeffs_From_Params (Data_Reader.cpp:59-89).
 * h_hx: [(M+1)(K+1)] complex, ascending powers of t; h_ht: [(M+1)K].
 * exact_ht = 0 keeps the reference's sentinel (c'_M = 1), 1 sets it to 0.
 * ------------------------------------------------------------------------- */
int ghc_p2c(const ghc_problem* pb, const double* h_start, const double* h_target, double* h_hx, double* h_ht,
            int exact_ht);
/* Same for n_hyp hypotheses on the device: d_targets [n_hyp][P+1],
 * d_hx [n_hyp][(M+1)(K+1)], d_ht [n_hyp][(M+1)K]. */
int ghc_p2c_device(const ghc_problem* pb, int64_t n_hyp, const double* d_start, const double* d_targets,
                   double* d_hx, double* d_ht, int exact_ht, void* stream);

/* ---------------------------------------------------------------------------
 * Batched tracker (device buffers, asynchronous on `stream`).
 * Replaces the per-problem launch wrappers kernel_HC_Solver_<problem>
 * (GPU-HC/magmaHC/gpu-kernels/magmaHC-kernels.hpp; e.g.
 * kernel_HC_Solver_P3P.cu:267-377 and kernel_HC_Solver_trifocal_2op1p_30x30.cu:313-486)
 * for n_hyp hypotheses x paths in one launch.  Work item i tracks start path
 * i % paths of hypothesis i / paths.
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n_hyp;
  int32_t precision;          /* GHC_PREC_* */
  int32_t max_steps;          /* <= 0: YAML value */
  int32_t max_corr;           /* <= 0: YAML value */
  int32_t incr_steps;         /* <= 0: YAML value */
  double t_switch;            /* GHC_PREC_MIXED: the mixed tracker (FP64 track, t, step control and corrector
                                 residual H; FP32 H_x, H_t and LU) for t < t_switch (>= 1: to t = 1;
                                 <= 0: all FP64); a path goes on in FP64 after a step whose FP32 solve had
                                 pivot magnitudes spanning more than cond_limit, once its step falls below
                                 dt_floor, after 4 failed steps in a row, or on divergence (at its last
                                 accepted point); needs d_steps, d_corr, d_t_end, d_dt_end */
  int32_t polish_iters;       /* Newton iterations at t = 1 after tracking (FP64 state only) */
  /* step control; <= 0 selects the reference's value (kernel_HC_Solver_P3P.cu:214) */
  double corr_tol2;           /* corrector success |dx|^2 < corr_tol2 |x|^2 (reference 1e-6) */
  double first_tol2;          /* reject a step whose first Newton update has |dx|^2 > first_tol2 |x|^2 (off) */
  double dt_max;              /* step-size cap (off) */
  /* inputs */
  const void* d_start_sols;   /* [paths][N] complex, state precision (double; float for FP32) */
  const double* d_coef_hx;    /* P2C: [n_hyp][(M+1)(K+1)] complex */
  const double* d_coef_ht;    /* P2C: [n_hyp][(M+1)K] complex */
  const double* d_p_start;    /* PH: [P+1] complex */
  const double* d_p_target;   /* PH: [n_hyp][P+1] complex */
  const double* d_p_diff;     /* PH: [n_hyp][P+1] complex (target - start) */
  /* outputs (n_items = n_hyp * paths) */
  void* d_endpoints;          /* [n_items][N] complex, state precision */
  uint8_t* d_status;          /* [n_items] GHC_STATUS_* */
  uint8_t* d_conv;            /* [n_items] */
  uint8_t* d_inf;             /* [n_items] */
  int32_t* d_steps;           /* [n_items] attempted steps (optional) */
  int32_t* d_corr;            /* [n_items] corrector iterations (optional) */
  double* d_t_end;            /* [n_items] (optional) */
  double* d_dt_end;           /* [n_items] (optional) */
  double* d_resid;            /* [n_items] |H(x,1)| after polish, -1 if not converged (optional) */
  /* scratch */
  int32_t* d_counter;         /* one int of device memory (work-stealing counter) */
  /* start solutions per hypothesis in d_start_sols; <= 0: the problem's Num_Of_Tracks */
  int32_t paths;
  /* GHC_PREC_MIXED: the pivot-magnitude span max|U_ii| / min|U_ii| of an FP32 solve above which the
     path goes on in FP64 (<= 0: 1e5), and the step size below which it does (<= 0: 1e-4) */
  double cond_limit;
  double dt_floor;
} ghc_track_args;

int ghc_track(const ghc_problem* pb, const ghc_track_args* args, void* stream);

/* ghc_track for callers that must not allocate device memory -- no counterpart
 * in the reference.  For applications that own all device memory through their
 * own pool or budget, or loops that cannot take cudaMalloc's synchronisation or
 * its failure mid-run.  Same arguments and results as ghc_track (every precision
 * mode, polish included), except that args->d_counter is ignored: the
 * work-stealing counter and the compiled index tables live in a fixed static
 * device array of 64 KiB per device, held by every GPU that loads the library
 * until the process exits, and the problem handle itself stays without device
 * memory.  Problems whose compiled tables do not fit return GHC_ERR_LIMIT.  The
 * first call on each device looks up the array's address.  For eager calls:
 * nothing is said or tested about capturing it in a CUDA graph (a call may copy
 * tables from host memory).  All calls on a device share the array and it keeps the last
 * call's contents: a call copies its tables in on `stream` unless the array
 * already holds this handle's tables, and clears the counter on `stream`, so
 * calls ordered on one stream are independent, while calls that overlap on the
 * GPU race.  Allocates nothing: no cudaMalloc, cudaFree or allocating library
 * call. */
int ghc_track_noalloc(const ghc_problem* pb, const ghc_track_args* args, void* stream);

/* ---------------------------------------------------------------------------
 * Batches of problems of different sizes in one persistent launch (the uneven
 * mix).  Replaces the reference's one-launch-per-problem dispatch
 * (GPU-HC/magmaHC/GPU_HC_Solver.cpp:207-349) for a mixed workload: bucket i is
 * (pbs[i], args[i]) exactly as for ghc_track (its own d_counter; plain FP64, no
 * polish); CTA ranges start on their own bucket in proportion to its expected
 * work and move on to the other buckets' counters when it is done, so short
 * buckets fill the GPU while the long one drains.  Results are bit-identical
 * to ghc_track launches of the buckets one by one.  Compiled for at most one
 * bucket each of P2C N = 3, 6, 12 and PH N = 30 with the term shapes of
 * P3P_TD, 5pt_rel_pos_alg_form_quat, generalized_3views_4pts and
 * trifocal_2op1p_30x30 (others: GHC_ERR_RANGE).  Asynchronous on `stream`.
 * ------------------------------------------------------------------------- */
int ghc_track_mix(const ghc_problem* const* pbs, const ghc_track_args* args, int32_t n_buckets, void* stream);

/* ---------------------------------------------------------------------------
 * Launch tuning.  The reference fixes threads-per-path and block shape per
 * problem in its 21 hand-written wrappers (e.g. kernel_HC_Solver_P3P.cu:284-297:
 * one block of N threads per path); here the sub-warp width follows N and two
 * things are chosen per problem handle and precision:
 *   variant  the compiled register budget (0: the default table of CTAs per SM,
 *            1: one more CTA per SM with fewer registers per thread);
 *   flat     how H_x is walked (1: each lane walks its row once through a
 *            shared-memory scratch row, 2: the entries are dealt to all lanes
 *            of the sub-warp balanced by term count, each sum stored into its
 *            row's scratch slot, 0: one loop per column; -1: chosen from the
 *            table structure; above 16 unknowns 1 or 2).
 * Every choice computes bit-identical results; only the speed differs.
 *
 * ghc_autotune runs the caller's sample batch (`sample`, exactly as for
 * ghc_track, outputs overwritten) once per candidate after a warm-up, times it
 * with CUDA events on `stream`, keeps the fastest in the handle for
 * sample->precision (mixed: both phases, their variants chosen independently)
 * and returns it.  It synchronises
 * `stream`; do not run it while the handle is tracking elsewhere.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t variant, flat;
  double ms;                  /* the sample's time with this choice */
  int32_t candidates;         /* how many were timed */
  int32_t variant_f32;        /* GHC_PREC_MIXED: the FP32 phase's variant (the FP64 phase's is `variant`) */
} ghc_tune_choice;

int ghc_autotune(ghc_problem* pb, const ghc_track_args* sample, void* stream, ghc_tune_choice* best);
/* precision GHC_PREC_FP64 or GHC_PREC_FP32 (GHC_PREC_MIXED: both) */
int ghc_set_tuning(ghc_problem* pb, int32_t precision, int32_t variant, int32_t flat);
int ghc_get_tuning(const ghc_problem* pb, int32_t precision, int32_t* variant, int32_t* flat);

/* ---------------------------------------------------------------------------
 * Result counts of one hypothesis on the host.
 * Replaces Evaluations::Evaluate_GPUHC_Sols and Evaluations::Find_Unique_Sols
 * (GPU-HC/magmaHC/Evaluations.cpp:88-110, 127-176).  h_endpoints [paths][N].
 * ------------------------------------------------------------------------- */
int ghc_count_results(int32_t N, int32_t paths, const double* h_endpoints, const uint8_t* h_conv,
                      const uint8_t* h_inf, double imag_tol, double dup_tol, ghc_counts* out);

/* ---------------------------------------------------------------------------
 * Result counts of every hypothesis of a batch on the device (asynchronous on
 * `stream`), with the rules of ghc_count_results -- the batched, on-device form
 * of Evaluations::Evaluate_GPUHC_Sols / Find_Unique_Sols
 * (GPU-HC/magmaHC/Evaluations.cpp:88-110, 127-176).
 * d_endpoints [n_hyp][paths][N] complex double (the tracker's layout);
 * d_conv, d_inf [n_hyp][paths]; d_counts [n_hyp] out; d_class [n_hyp][paths] out
 * (optional): bit 0 converged, bit 1 real, bit 2 counted as unique.
 * paths up to 200,000.
 * ------------------------------------------------------------------------- */
int ghc_count_results_device(int32_t N, int32_t paths, int64_t n_hyp, const double* d_endpoints,
                             const uint8_t* d_conv, const uint8_t* d_inf, double imag_tol, double dup_tol,
                             ghc_counts* d_counts, uint8_t* d_class, void* stream);

/* ---------------------------------------------------------------------------
 * Drop-in launch wrappers with the reference kernel ABI
 * (GPU-HC/magmaHC/gpu-kernels/magmaHC-kernels.hpp, e.g. kernel_HC_Solver_P3P.cu:267-282
 * and kernel_HC_Solver_trifocal_2op1p_30x30.cu:413-427).  magma_queue_t becomes a
 * cudaStream_t (`stream`), magmaFloatComplex a float pair, magma_int_t an int.
 * Pointer arrays must describe the reference's layout (entry p = base + p*(N+1)).
 * Tracks are in/out; conv/inf are one byte per path; debug (optional) receives
 * (1,0) for converged paths and (t, dt) otherwise.  Synchronous; returns the
 * elapsed seconds of the launch, or a negative GHC_ERR_* code.
 * The _z variants are the plain FP64 twins (double pairs).
 * ------------------------------------------------------------------------- */
double ghc_kernel_HC_Solver_P2C(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                float** d_startSols_array, float** d_Track_array, const int* d_Hx_idx,
                                const int* d_Ht_idx, const float* d_phc_coeffs_Hx, const float* d_phc_coeffs_Ht,
                                uint8_t* d_conv, uint8_t* d_inf, float* d_debug);
double ghc_kernel_HC_Solver_P2C_z(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                  double** d_startSols_array, double** d_Track_array, const int* d_Hx_idx,
                                  const int* d_Ht_idx, const double* d_phc_coeffs_Hx,
                                  const double* d_phc_coeffs_Ht, uint8_t* d_conv, uint8_t* d_inf,
                                  double* d_debug);
double ghc_kernel_HC_Solver_PH(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                               float** d_startSols_array, float** d_Track_array, const float* d_startParams,
                               const float* d_targetParams, const float* d_diffParams, const int* d_Hx_idx,
                               const int* d_Ht_idx, uint8_t* d_conv, uint8_t* d_inf, float* d_debug);
double ghc_kernel_HC_Solver_PH_z(const ghc_problem* pb, void* stream, int max_steps, int max_corr, int incr,
                                 double** d_startSols_array, double** d_Track_array, const double* d_startParams,
                                 const double* d_targetParams, const double* d_diffParams, const int* d_Hx_idx,
                                 const int* d_Ht_idx, uint8_t* d_conv, uint8_t* d_inf, double* d_debug);

/* ---------------------------------------------------------------------------
 * One-call host solve (the CLI path): host buffers in and out, all copies,
 * P2C, tracking and polish inside.  Replaces GPU_HC_Solver::Allocate_Arrays,
 * Data_Transfer_From_Host_To_Device and Solve_by_GPU_HC
 * (GPU-HC/magmaHC/GPU_HC_Solver.cpp:104-140, 183-384) for n_hyp target sets.
 * h_targets: [n_hyp][P+1] complex (NULL: the problem's target_params.txt, n_hyp = 1).
 * h_endpoints: [n_hyp*paths][N] complex double.  h_status, h_steps optional.
 * h_ms (optional): [0] H2D, [1] P2C + track + polish, [2] D2H, milliseconds.
 * Device buffers come from a grow-only arena of the handle and the work runs on the
 * handle's own stream, so calls on one handle must not overlap.
 * ------------------------------------------------------------------------- */
int ghc_solve_host(const ghc_problem* pb, int32_t precision, int64_t n_hyp, const double* h_targets,
                   double t_switch, int32_t polish_iters, double* h_endpoints, uint8_t* h_status, uint8_t* h_conv,
                   uint8_t* h_inf, int32_t* h_steps, double* h_ms);

/* ---------------------------------------------------------------------------
 * Diagnostics (no counterpart in the reference): measured CUDA-core FMA
 * throughput of the current device in FLOP/s, the roofline denominator of
 * the tracker's complex FP64/FP32 arithmetic.  precision: GHC_PREC_FP64 or
 * GHC_PREC_FP32.  ms (optional): duration of the timed launch.
 * ------------------------------------------------------------------------- */
int ghc_measure_fma_peak(int precision, double* flops_per_s, double* ms);

/* ---------------------------------------------------------------------------
 * The tracker's linear solve on its own (diagnostics).  Replaces nothing callable:
 * it runs the device LU that stands in for cgesv_batched_small_device
 * (GPU-HC/magmaHC/dev-cgesv-batched-small.cuh:40-107) -- pivot = the largest |Re|+|Im|
 * among the unpivoted rows, the lowest position on ties, a NaN at the current position
 * kept and a NaN below never taken; a zero pivot skips its elimination -- on n_sys
 * systems A z = b of N unknowns, one sub-warp per system, asynchronously on `stream`.
 * d_A [n_sys][N][N] (row-major), d_b [n_sys][N], d_z [n_sys][N] complex: double pairs
 * for GHC_PREC_FP64, float pairs for GHC_PREC_FP32.  N in {3,4,5,6,8,10,11,12,16,18,30}.
 * ------------------------------------------------------------------------- */
int ghc_lu_solve_device(int32_t N, int32_t precision, int64_t n_sys, const void* d_A, const void* d_b, void* d_z,
                        void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GHC_H */
