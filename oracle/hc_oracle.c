/*
 * hc_oracle.c -- CPU oracle of the homotopy path tracker.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference tracker,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The product never links or calls it.
 *
 * The precision-generic body lives in hc_oracle_body.h and is instantiated
 * for double (suffix _d), float (suffix _f), and the mixed tracker's first phase
 * (suffix _m: double state, float linear algebra).  Build flags (oracle/build.py):
 * -O2 -ffp-contract=off -fopenmp, so no multiply-add is fused except through
 * the explicit fma()/fmaf() calls.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_NMAX 32
#define ORC_MMAX 640

enum { ORC_P2C = 0, ORC_PH = 1 };
enum { ORC_CONVERGED = 0, ORC_DIVERGED = 1, ORC_STEP_CAP = 2, ORC_NONFINITE = 3, ORC_SINGULAR = 4 };

/* Problem description: the YAML sizes plus the raw index tables in the
 * reference layout (GPU-HC/magmaHC/GPU_HC_Solver.cpp:44-83). */
typedef struct {
  int32_t kind; /* ORC_P2C or ORC_PH */
  int32_t N, P, M, K;
  int32_t Tx, Px, Tt, Pt;
  int32_t max_steps, max_corr, incr_steps;
  int32_t polish_iters;
  const int32_t* hx_idx;
  const int32_t* ht_idx;
  /* step control; the reference's values are corr_tol2 = 1e-6, first_tol2 = inf, dt_max = inf */
  double corr_tol2;  /* corrector success: |dx|^2 < corr_tol2 * |x|^2 */
  double first_tol2; /* reject the step when the first Newton update has |dx|^2 > first_tol2 * |x|^2 */
  double dt_max;     /* upper bound of the step size */
  /* two-phase mixed precision (the tracker library's GHC_PREC_MIXED, not a reference feature):
   * the first (float) phase stops a path at t_handover (> 0), after fail_limit (> 0)
   * consecutive failed steps, or on divergence at its last accepted point; the second
   * (double) phase resumes every path from endpoints / t_end / dt_end / steps / corr */
  double t_handover;
  int32_t fail_limit;
  int32_t resume;
  /* mixed tracker: hand a path over after a step in which a float solve's pivot magnitudes spanned
   * more than cond_limit (0: never) */
  double cond_limit;
  /* mixed tracker: hand a path over once its step falls below dt_floor (0: never) */
  double dt_floor;
} orc_problem;

typedef struct {
  uint8_t converged, infinity, status;
  int32_t steps, corr;
  double t_end, dt_end, resid;
} orc_path_out;

#define REAL double
#define SUFFIX _d
#define FMA fma
#define FABS fabs
#include "hc_oracle_body.h"
#undef REAL
#undef SUFFIX
#undef FMA
#undef FABS

#define REAL float
#define SUFFIX _f
#define FMA fmaf
#define FABS fabsf
#include "hc_oracle_body.h"
#undef REAL
#undef SUFFIX
#undef FMA
#undef FABS

/* the mixed tracker's first phase (the tracker library's GHC_PREC_MIXED, not a reference feature):
 * double state, step control, norms and corrector residual, with H_x, H_t and the LU in float */
#define ORC_MIXED_LA 1
#define REAL double
#define SUFFIX _m
#define FMA fma
#define FABS fabs
#include "hc_oracle_body.h"
#undef REAL
#undef SUFFIX
#undef FMA
#undef FABS
#undef ORC_MIXED_LA

int orc_abi_version(void) { return 1; }
int orc_sizeof_problem(void) { return (int)sizeof(orc_problem); }
