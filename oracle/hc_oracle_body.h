/*
 * hc_oracle_body.h -- precision-generic body of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is included twice by hc_oracle.c, once
 * with REAL=double and once with REAL=float.  Nothing in the product links it;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the resulting shared library, and only as the checker.
 *
 * It restates, path by path and in plain sequential C, the homotopy path
 * tracker of the reference:
 *   - per-path loop, end-zone step clamp, loopy RK4, Newton corrector and
 *     step control:   GPU-HC/magmaHC/gpu-kernels/kernel_HC_Solver_P3P.cu:96-260
 *     (PH variant:    GPU-HC/magmaHC/gpu-kernels/kernel_HC_Solver_trifocal_2op1p_30x30.cu:115-301)
 *   - coefficient homotopy c_k(t), H_x, H_t, H from the index tables:
 *                     GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-P3P.cuh:33-120
 *     (PH variant:    GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-trifocal_2op1p_30x30.cuh:46-168)
 *   - partial-pivot complex LU + back substitution:
 *                     GPU-HC/magmaHC/dev-cgesv-batched-small.cuh:40-107
 *
 * Arithmetic is written in one fixed operation order (explicit fma() where a
 * product is fused, nothing else fused; the library is built with
 * -ffp-contract=off).  The CUDA tracker uses the same order, so in FP64 the
 * two produce identical endpoints, step counts and flags.  Deliberate choices
 * where the reference is undefined or ambiguous:
 *   - norms are summed over the N live rows only (the reference sums 32 warp
 *     lanes, of which lanes >= N do not exist), as a pairwise tree over the
 *     next power of two >= N;
 *   - all lanes see freshly evaluated coefficients (the reference has no
 *     __syncwarp between eval_parameter_homotopy and eval_Jacobian_Hx);
 *   - PH target parameters beyond index N are read per hypothesis (the
 *     reference reads them without the hypothesis offset);
 *   - padding terms (integer scale 0) are skipped (variable slot N, the
 *     constant 1, is multiplied in like any other slot, as in the reference);
 *   - the pivot reciprocal is conj(b)/|b|^2 (one reciprocal); the back
 *     substitution multiplies by the reciprocal formed during elimination.
 * The pivot rule is the reference's own: strict argmax of |Re|+|Im| over the
 * unpivoted positions in order (lowest position on ties).
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define SFX(name) CAT(name, SUFFIX)

typedef struct { REAL re, im; } SFX(cx_);
#define CX SFX(cx_)

static inline CX SFX(c_make)(REAL a, REAL b) { CX r; r.re = a; r.im = b; return r; }
static inline CX SFX(c_add)(CX a, CX b) { return SFX(c_make)(a.re + b.re, a.im + b.im); }
static inline CX SFX(c_sub)(CX a, CX b) { return SFX(c_make)(a.re - b.re, a.im - b.im); }
static inline CX SFX(c_scale)(REAL s, CX a) { return SFX(c_make)(s * a.re, s * a.im); }
/* a*b */
static inline CX SFX(c_mul)(CX a, CX b) {
  return SFX(c_make)(FMA(a.re, b.re, -(a.im * b.im)), FMA(a.re, b.im, a.im * b.re));
}
/* c + a*b */
static inline CX SFX(c_fma)(CX a, CX b, CX c) {
  return SFX(c_make)(FMA(a.re, b.re, FMA(-a.im, b.im, c.re)), FMA(a.re, b.im, FMA(a.im, b.re, c.im)));
}
/* c - a*b */
static inline CX SFX(c_fnma)(CX a, CX b, CX c) {
  return SFX(c_make)(FMA(-a.re, b.re, FMA(a.im, b.im, c.re)), FMA(-a.re, b.im, FMA(-a.im, b.re, c.im)));
}
/* 1/b = conj(b) / |b|^2 with one correctly rounded reciprocal */
static inline CX SFX(c_rcp)(CX b) {
  const REAL s = FMA(b.re, b.re, b.im * b.im);
  const REAL inv = (REAL)1 / s;
  return SFX(c_make)(b.re * inv, -(b.im * inv));
}
/* |a|^2 */
static inline REAL SFX(c_abs2)(CX a) { return FMA(a.re, a.re, a.im * a.im); }

/* pairwise sum in the order of an xor butterfly over NP = next pow2 >= n lanes */
static REAL SFX(tree_sum)(const REAL* v, int n) {
  REAL buf[ORC_NMAX], nxt[ORC_NMAX];
  int np = 1;
  while (np < n) np <<= 1;
  for (int l = 0; l < np; ++l) buf[l] = (l < n) ? v[l] : (REAL)0;
  for (int off = np >> 1; off > 0; off >>= 1) {
    for (int l = 0; l < np; ++l) nxt[l] = buf[l] + buf[l ^ off];
    for (int l = 0; l < np; ++l) buf[l] = nxt[l];
  }
  return buf[0];
}

/* accumulate one monomial term: acc += s * first * x[v0] * x[v1] ... over every variable
 * slot of the table, slot N being the constant 1 (GPU-HC/magmaHC/gpu-idx-evals/
 * dev-eval-indxing-P3P.cuh:70-118); the last product is fused into the accumulation */
static inline CX SFX(acc_term)(CX acc, CX p, const int32_t* vars, int nvar, const CX* x) {
  if (nvar == 0) return SFX(c_add)(acc, p);
  for (int q = 0; q < nvar - 1; ++q) p = SFX(c_mul)(p, x[vars[q]]);
  return SFX(c_fma)(p, x[vars[nvar - 1]], acc);
}

typedef struct {
  /* P2C: coefficient homotopy values at t */
  CX c[ORC_MMAX];   /* c_k(t)  (from the H_x coefficient table) */
  CX cp[ORC_MMAX];  /* c'_k(t) (from the H_t coefficient table) */
  /* PH: parameter homotopy values at t and parameter differences */
  CX ph[ORC_MMAX];
  CX dp[ORC_MMAX];
#ifdef ORC_MIXED_LA
  coefs__f lo; /* the same values rounded to float, for H_x, H_t and the float LU */
#endif
} SFX(coefs_);
#define COEFS SFX(coefs_)

typedef struct {
  const orc_problem* pb;
  const CX* hx_coef; /* P2C raw table [(M+1)(K+1)] */
  const CX* ht_coef; /* P2C raw table [(M+1)K] */
  const CX* p_start; /* PH [P+1] */
  const CX* p_tgt;   /* PH [P+1] */
  const CX* p_diff;  /* PH [P+1] */
} SFX(hyp_);
#define HYP SFX(hyp_)

/* coefficient homotopy at t (reference eval_parameter_homotopy / compute_param_homotopy) */
static void SFX(eval_coefs)(const HYP* h, REAL t, COEFS* cf) {
  const orc_problem* pb = h->pb;
  if (pb->kind == ORC_P2C) {
    const int K = pb->K, M = pb->M;
    for (int k = 0; k <= M; ++k) {
      const CX* a = h->hx_coef + (size_t)k * (K + 1);
      CX v = a[K];
      for (int j = K - 1; j >= 0; --j) v = SFX(c_make)(FMA(v.re, t, a[j].re), FMA(v.im, t, a[j].im));
      cf->c[k] = v;
      if (K >= 1) {
        const CX* b = h->ht_coef + (size_t)k * K;
        CX w = b[K - 1];
        for (int j = K - 2; j >= 0; --j) w = SFX(c_make)(FMA(w.re, t, b[j].re), FMA(w.im, t, b[j].im));
        cf->cp[k] = w;
      } else {
        cf->cp[k] = SFX(c_make)(0, 0);
      }
    }
  } else {
    const int P = pb->P;
    const REAL u = (REAL)1 - t;
    for (int k = 0; k < P; ++k) {
      CX g = h->p_tgt[k], s = h->p_start[k];
      cf->ph[k] = SFX(c_make)(FMA(g.re, t, s.re * u), FMA(g.im, t, s.im * u));
      cf->dp[k] = h->p_diff[k];
    }
    cf->ph[P] = SFX(c_make)(1, 0);
    cf->dp[P] = h->p_diff[P];
  }
#ifdef ORC_MIXED_LA
  /* mixed: every coefficient computed in double, then rounded once to float */
  const int nk = (pb->kind == ORC_P2C) ? pb->M + 1 : pb->P + 1;
  for (int k = 0; k < nk; ++k) {
    if (pb->kind == ORC_P2C) {
      cf->lo.c[k] = c_make_f((float)cf->c[k].re, (float)cf->c[k].im);
      cf->lo.cp[k] = c_make_f((float)cf->cp[k].re, (float)cf->cp[k].im);
    } else {
      cf->lo.ph[k] = c_make_f((float)cf->ph[k].re, (float)cf->ph[k].im);
      cf->lo.dp[k] = c_make_f((float)cf->dp[k].re, (float)cf->dp[k].im);
    }
  }
#endif
}

/* Row r of H_x into A[0..N) */
static void SFX(eval_hx_row)(const orc_problem* pb, const COEFS* cf, const CX* x, int r, CX* A) {
  const int N = pb->N, Tx = pb->Tx, Px = pb->Px;
  for (int i = 0; i < N; ++i) {
    CX acc = SFX(c_make)(0, 0);
    for (int j = 0; j < Tx; ++j) {
      int32_t tm[8] = {0};
      if (pb->kind == ORC_P2C) {
        const int32_t* e = pb->hx_idx + (size_t)r * N * Tx * Px + (size_t)i * Tx * Px + (size_t)j * Px;
        for (int q = 0; q < Px; ++q) tm[q] = e[q];
        if (tm[0] == 0) continue;
        CX p = SFX(c_scale)((REAL)tm[0], cf->c[tm[1]]);
        acc = SFX(acc_term)(acc, p, tm + 2, Px - 2, x);
      } else {
        for (int q = 0; q < Px; ++q) tm[q] = pb->hx_idx[((size_t)i * Tx * Px + (size_t)j * Px + q) * N + r];
        if (tm[0] == 0) continue;
        CX p = SFX(c_scale)((REAL)tm[0], cf->ph[tm[1]]);
        p = SFX(c_mul)(p, cf->ph[tm[2]]);
        acc = SFX(acc_term)(acc, p, tm + 3, Px - 3, x);
      }
    }
    A[i] = acc;
  }
}

/* Row r of H (which = 0) or of H_t (which = 1) from the dH/dt table */
static CX SFX(eval_h_row)(const orc_problem* pb, const COEFS* cf, const CX* x, int r, int which) {
  const int N = pb->N, Tt = pb->Tt, Pt = pb->Pt;
  CX acc = SFX(c_make)(0, 0);
  for (int j = 0; j < Tt; ++j) {
    int32_t tm[8] = {0};
    if (pb->kind == ORC_P2C) {
      const int32_t* e = pb->ht_idx + (size_t)r * Tt * Pt + (size_t)j * Pt;
      for (int q = 0; q < Pt; ++q) tm[q] = e[q];
      if (tm[0] == 0) continue;
      CX p = SFX(c_scale)((REAL)tm[0], which ? cf->cp[tm[1]] : cf->c[tm[1]]);
      acc = SFX(acc_term)(acc, p, tm + 2, Pt - 2, x);
    } else {
      for (int q = 0; q < Pt; ++q) tm[q] = pb->ht_idx[((size_t)j * Pt + q) * N + r];
      if (tm[0] == 0) continue;
      CX p;
      if (which) {
        CX u = SFX(c_fma)(cf->dp[tm[2]], cf->ph[tm[1]], SFX(c_mul)(cf->dp[tm[1]], cf->ph[tm[2]]));
        p = SFX(c_scale)((REAL)tm[0], u);
      } else {
        p = SFX(c_scale)((REAL)tm[0], cf->ph[tm[1]]);
        p = SFX(c_mul)(p, cf->ph[tm[2]]);
      }
      acc = SFX(acc_term)(acc, p, tm + 3, Pt - 3, x);
    }
  }
  return acc;
}

/*
 * Solve A z = b with partial pivoting, one row per (virtual) lane.
 * Pivot of column i: the reference's scan (GPU-HC/magmaHC/dev-cgesv-batched-small.cuh:54-65)
 * over the positions i..N-1 in order, starting from position i and moving only to a strictly
 * larger |Re|+|Im|: the largest magnitude, the lowest position among equal ones; a NaN at
 * position i is kept, a NaN below is never taken.  A zero pivot skips the elimination for that
 * column and leaves a non-finite solution, as in the reference.  The solution is returned in
 * variable order.  trace (optional): piv[i] = the pivot position of column i, and
 * mags[i*N + j] = |Re|+|Im| of the row at position j (j >= i) when column i was searched.
 */
static void SFX(lu_solve_trace)(int N, CX A[][ORC_NMAX], CX* b, CX* z, int32_t* piv, REAL* mags, REAL* piv_range) {
  int pos[ORC_NMAX], row_at[ORC_NMAX];
  CX myrcp[ORC_NMAX];
  for (int r = 0; r < N; ++r) pos[r] = row_at[r] = r;
  for (int i = 0; i < N; ++i) {
    int best_pos = i;
    REAL best = FABS(A[row_at[i]][i].re) + FABS(A[row_at[i]][i].im);
    if (mags) mags[i * N + i] = best;
    for (int j = i + 1; j < N; ++j) {
      const REAL v = FABS(A[row_at[j]][i].re) + FABS(A[row_at[j]][i].im);
      if (mags) mags[i * N + j] = v;
      if (v > best) {
        best = v;
        best_pos = j;
      }
    }
    if (piv) piv[i] = best_pos;
    if (piv_range) { /* the pivot magnitudes' range (|U_ii| as |Re|+|Im|) and whether one was NaN */
      if (i == 0 || best < piv_range[0]) piv_range[0] = best;
      if (i == 0 || best > piv_range[1]) piv_range[1] = best;
      if (best != best) piv_range[2] = 1;
    }
    const int best_r = row_at[best_pos];
    /* zero pivot: the pivot row's own magnitude is exactly 0 */
    const int zero = (best == (REAL)0);
    /* the pivot row moves to position i, the row at position i to the pivot's position */
    const int r_i = row_at[i];
    pos[r_i] = best_pos;
    row_at[best_pos] = r_i;
    pos[best_r] = i;
    row_at[i] = best_r;
    CX sx[ORC_NMAX];
    for (int j = i; j < N; ++j) sx[j] = A[best_r][j];
    const CX sb = b[best_r];
    const CX rc = SFX(c_rcp)(zero ? SFX(c_make)(0, 0) : sx[i]);
    myrcp[best_r] = rc;
    if (zero) continue; /* zero pivot: no elimination in this column */
    for (int r = 0; r < N; ++r) {
      if (pos[r] > i) {
        A[r][i] = SFX(c_mul)(A[r][i], rc);
        for (int j = i + 1; j < N; ++j) A[r][j] = SFX(c_fnma)(A[r][i], sx[j], A[r][j]);
        b[r] = SFX(c_fnma)(A[r][i], sb, b[r]);
      }
    }
  }
  for (int i = N - 1; i >= 0; --i) {
    const int ri = row_at[i];
    const CX xi = SFX(c_mul)(b[ri], myrcp[ri]);
    for (int r = 0; r < N; ++r)
      if (pos[r] < i) b[r] = SFX(c_fnma)(A[r][i], xi, b[r]);
    b[ri] = xi;
    z[i] = xi;
  }
}

static void SFX(lu_solve)(int N, CX A[][ORC_NMAX], CX* b, CX* z) { SFX(lu_solve_trace)(N, A, b, z, NULL, NULL, NULL); }

/* one evaluation + solve: z = H_x^{-1} * rhs; rhs = -H_t (which=1) or H (which=0) */
static void SFX(eval_solve)(const orc_problem* pb, const COEFS* cf, const CX* x, int which, CX* z, int* ill,
                            int* sing) {
  const int N = pb->N;
  (void)ill;
#ifdef ORC_MIXED_LA
  /* mixed: H_x and -H_t in float from the float coefficients and the track rounded to float; the
   * corrector's residual H in double, rounded to float; the LU in float; the step back in double */
  {
    cx__f xf[ORC_NMAX + 1], A[ORC_NMAX][ORC_NMAX], b[ORC_NMAX], zf[ORC_NMAX];
    for (int r = 0; r < N; ++r) xf[r] = c_make_f((float)x[r].re, (float)x[r].im);
    xf[N] = c_make_f(1, 0);
    for (int r = 0; r < N; ++r) {
      eval_hx_row_f(pb, &cf->lo, xf, r, A[r]);
      if (which) {
        const cx__f h = eval_h_row_f(pb, &cf->lo, xf, r, 1);
        b[r] = c_make_f(-h.re, -h.im);
      } else {
        const CX h = SFX(eval_h_row)(pb, cf, x, r, 0);
        b[r] = c_make_f((float)h.re, (float)h.im);
      }
    }
    float range[3] = {0, 0, 0};
    lu_solve_trace_f(N, A, b, zf, NULL, NULL, range);
    if (sing && range[0] == 0) *sing = 1;
    for (int r = 0; r < N; ++r) z[r] = SFX(c_make)((double)zf[r].re, (double)zf[r].im);
    /* ill-conditioned for the float solve: the pivot magnitudes span more than cond_limit (or NaN) */
    if (pb->cond_limit > 0 && ill && (range[2] != 0 || !(range[1] <= (float)pb->cond_limit * range[0]))) *ill = 1;
    return;
  }
#endif
  CX A[ORC_NMAX][ORC_NMAX];
  CX b[ORC_NMAX];
  for (int r = 0; r < N; ++r) {
    SFX(eval_hx_row)(pb, cf, x, r, A[r]);
    CX h = SFX(eval_h_row)(pb, cf, x, r, which);
    b[r] = which ? SFX(c_make)(-h.re, -h.im) : h;
  }
  REAL range[3] = {0, 0, 0};
  SFX(lu_solve_trace)(N, A, b, z, NULL, NULL, range);
  if (sing && range[0] == 0) *sing = 1;
}

/*
 * Track one path from t=0 to t=1 (reference HC_solver_<p> body).
 * x_io: in = start point (N values), out = endpoint.
 * With pb->resume the path starts at out->t_end with step out->dt_end and the
 * counts out->steps / out->corr; pb->t_handover / fail_limit add the stopping
 * rules of the first phase of the two-phase mixed-precision tracker.
 */
static void SFX(track_path)(const HYP* h, CX* x_io, orc_path_out* out) {
  const orc_problem* pb = h->pb;
  const int N = pb->N;
  COEFS* cf = (COEFS*)malloc(sizeof(COEFS));
  CX x[ORC_NMAX + 1], x0[ORC_NMAX + 1], sols[ORC_NMAX + 1], k[ORC_NMAX];
  for (int r = 0; r < N; ++r) x[r] = x0[r] = sols[r] = x_io[r];
  x[N] = x0[N] = sols[N] = SFX(c_make)(1, 0);

  const int ph = (pb->kind == ORC_PH);
  REAL t0 = 0, t_step = 0, dt = ph ? (REAL)0.01 : (REAL)0.05;
  int end_zone = 0, nsucc = 0, nfail = 0;
  int success = 0, inf = 0;
  int32_t steps = 0, corr = 0;
  const int handover = pb->t_handover > 0 || pb->fail_limit > 0;
  const REAL t_hand = (REAL)pb->t_handover;
  if (pb->resume) {
    t0 = (REAL)out->t_end;
    dt = (REAL)out->dt_end;
    steps = out->steps;
    corr = out->corr;
  }
  static const REAL wgt[3] = {(REAL)(1.0 / 6.0), (REAL)(2.0 / 6.0), (REAL)(2.0 / 6.0)};
  static const REAL frac[3] = {(REAL)0.5, (REAL)0.5, (REAL)1.0};

  REAL dt_pre = dt; /* the step without the handover clamp: the next phase resumes with it */
  int ill = 0, ill_stop = 0; /* mixed: a solve of this step was ill-conditioned for float; stop after it */
  int step_sing = 0, last_sing = 0; /* a solve of this step / of the last completed step had a zero pivot */
  for (int step = steps; step <= pb->max_steps; ++step) {
    if (!(t0 < (REAL)1 && (REAL)1 - t0 > (REAL)1e-7)) break;
    if (pb->t_handover > 0 && t_hand - t0 <= (REAL)1e-6) {
      if (dt < dt_pre) dt = dt_pre;
      break;
    }
    if (pb->fail_limit > 0 && nfail >= pb->fail_limit) break;
    if (ill_stop) break;
    ++steps;
    ill = 0;
    step_sing = 0;
    /* end-zone step clamp (kernel_HC_Solver_P3P.cu:121-131; PH edge 0.95 at trifocal_2op1p_30x30.cu:163-182) */
    if (!end_zone && FABS((REAL)1 - t0) <= (REAL)0.0500001) end_zone = 1;
    if (end_zone) {
      if (dt > FABS((REAL)1 - t0)) dt = FABS((REAL)1 - t0);
    } else {
      const REAL edge = ph ? FABS((REAL)0.95 - t0) : FABS(((REAL)1 - (REAL)0.05) - t0);
      if (dt > edge) dt = edge;
    }
    dt_pre = dt;
    if (pb->t_handover > 0 && dt > t_hand - t0) dt = t_hand - t0;
    t_step = t0;
    const REAL half = (REAL)0.5 * dt;

    /* loopy RK4 predictor (kernel_HC_Solver_P3P.cu:139-183) */
    for (int rk = 0; rk < 4; ++rk) {
      SFX(eval_coefs)(h, t0, cf);
      SFX(eval_solve)(pb, cf, x, 1, k, &ill, &step_sing);
      if (rk < 3) {
        const REAL a = dt * wgt[rk];
        const REAL d = dt * frac[rk];
        for (int r = 0; r < N; ++r) {
          sols[r] = SFX(c_make)(FMA(k[r].re, a, sols[r].re), FMA(k[r].im, a, sols[r].im));
          x[r] = SFX(c_make)(FMA(k[r].re, d, x0[r].re), FMA(k[r].im, d, x0[r].im));
        }
        if (rk != 1) t0 = t0 + half;
      }
    }
    {
      const REAL a = dt * (REAL)(1.0 / 6.0);
      for (int r = 0; r < N; ++r) {
        sols[r] = SFX(c_make)(FMA(k[r].re, a, sols[r].re), FMA(k[r].im, a, sols[r].im));
        x[r] = sols[r];
      }
    }

    /* Newton corrector with the coefficients of the last RK stage (kernel_HC_Solver_P3P.cu:191-223) */
    success = 0;
    inf = 0;
    for (int it = 0; it < pb->max_corr; ++it) {
      ++corr;
      SFX(eval_solve)(pb, cf, x, 0, k, &ill, &step_sing);
      REAL ns[ORC_NMAX], nc[ORC_NMAX];
      for (int r = 0; r < N; ++r) {
        x[r] = SFX(c_sub)(x[r], k[r]);
        ns[r] = SFX(c_abs2)(k[r]);
        nc[r] = SFX(c_abs2)(x[r]);
      }
      const REAL sn = SFX(tree_sum)(ns, N), sc = SFX(tree_sum)(nc, N);
      success = ((double)sn < pb->corr_tol2 * (double)sc);
      inf = ((double)sc > 1e14);
      if (inf || success) break;
      if (it == 0 && (double)sn > pb->first_tol2 * (double)sc) break; /* predictor too far off: reject */
    }
    if (inf) {
      if (handover) { /* hand the last accepted point over */
        for (int r = 0; r < N; ++r) x[r] = x0[r];
        t0 = t_step;
      }
      break;
    }

    /* step control (kernel_HC_Solver_P3P.cu:230-249) */
    if (!success) {
      dt = dt * (REAL)0.5;
      for (int r = 0; r < N; ++r) x[r] = sols[r] = x0[r];
      nsucc = 0;
      t0 = t_step;
      ++nfail;
    } else {
      nfail = 0;
      ++nsucc;
      for (int r = 0; r < N; ++r) x0[r] = sols[r] = x[r];
      if (nsucc >= pb->incr_steps) {
        nsucc = 0;
        dt = dt * (REAL)2;
        if ((double)dt > pb->dt_max) dt = (REAL)pb->dt_max;
      }
    }
    if (ill) ill_stop = 1;
    if (pb->dt_floor > 0 && (double)dt < pb->dt_floor) ill_stop = 1; /* mixed: steps this small mean float is stuck */
    last_sing = step_sing;
  }

  const int conv = (t0 >= (REAL)1 || ((REAL)1 - t0 <= (REAL)1e-7));
  out->converged = (uint8_t)conv;
  out->infinity = (uint8_t)inf;
  int nonfinite = 0;
  for (int r = 0; r < N; ++r) nonfinite |= !(isfinite(x[r].re) && isfinite(x[r].im));
  out->status = conv ? ORC_CONVERGED
                : inf ? ORC_DIVERGED
                : nonfinite ? ORC_NONFINITE
                : last_sing ? ORC_SINGULAR
                : ORC_STEP_CAP;
  out->steps = steps;
  out->corr = corr;
  /* handed over at the boundary: resume at exactly t_handover (the tracker library does the same) */
  out->t_end = (pb->t_handover > 0 && !inf && t_hand - t0 <= (REAL)1e-6) ? pb->t_handover : (double)t0;
  out->dt_end = (double)dt;

  /* optional Newton polish at t = 1 of converged paths, then the residual |H(x,1)| */
  double resid = -1.0;
  if (conv) {
    SFX(eval_coefs)(h, (REAL)1, cf);
    for (int it = 0; it < pb->polish_iters; ++it) {
      SFX(eval_solve)(pb, cf, x, 0, k, NULL, NULL);
      for (int r = 0; r < N; ++r) x[r] = SFX(c_sub)(x[r], k[r]);
    }
    REAL hr[ORC_NMAX];
    for (int r = 0; r < N; ++r) hr[r] = SFX(c_abs2)(SFX(eval_h_row)(pb, cf, x, r, 0));
    resid = sqrt((double)SFX(tree_sum)(hr, N));
  }
  out->resid = resid;
  for (int r = 0; r < N; ++r) x_io[r] = x[r];
  free(cf);
}

/*
 * Batched driver: item i tracks start path (i % paths_per_hyp) of hypothesis
 * (i / paths_per_hyp).  Complex arrays are interleaved (re, im).
 */
int SFX(orc_track)(const orc_problem* pb, int64_t n_items, int32_t paths_per_hyp,
                   const REAL* start_sols, const REAL* coef_hx, const REAL* coef_ht,
                   int64_t stride_hx, int64_t stride_ht, const REAL* p_start, const REAL* p_tgt,
                   const REAL* p_diff, int64_t stride_p, REAL* endpoints, uint8_t* conv, uint8_t* infy,
                   uint8_t* status, int32_t* steps, int32_t* corr, double* t_end, double* dt_end,
                   double* resid, int32_t nthreads) {
  if (pb->N < 1 || pb->N > ORC_NMAX) return -1;
  if (pb->kind == ORC_P2C && (pb->M + 1 > ORC_MMAX || pb->K < 0 || pb->K > 8)) return -2;
  if (pb->kind == ORC_PH && pb->P + 1 > ORC_MMAX) return -3;
  if (pb->Px > 8 || pb->Pt > 8) return -4;
  if (paths_per_hyp <= 0) return -5;
  if (pb->resume && (!t_end || !dt_end || !steps || !corr)) return -6;
  const int N = pb->N;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t i = 0; i < n_items; ++i) {
    const int64_t hy = i / paths_per_hyp;
    const int64_t p = i % paths_per_hyp;
    HYP h;
    h.pb = pb;
    h.hx_coef = coef_hx ? (const CX*)(coef_hx + 2 * hy * stride_hx) : NULL;
    h.ht_coef = coef_ht ? (const CX*)(coef_ht + 2 * hy * stride_ht) : NULL;
    h.p_start = p_start ? (const CX*)p_start : NULL;
    h.p_tgt = p_tgt ? (const CX*)(p_tgt + 2 * hy * stride_p) : NULL;
    h.p_diff = p_diff ? (const CX*)(p_diff + 2 * hy * stride_p) : NULL;
    CX x[ORC_NMAX];
    orc_path_out o;
    if (pb->resume) {
      for (int r = 0; r < N; ++r) x[r] = SFX(c_make)(endpoints[2 * (i * N + r)], endpoints[2 * (i * N + r) + 1]);
      o.t_end = t_end[i];
      o.dt_end = dt_end[i];
      o.steps = steps[i];
      o.corr = corr[i];
    } else {
      for (int r = 0; r < N; ++r) x[r] = SFX(c_make)(start_sols[2 * (p * N + r)], start_sols[2 * (p * N + r) + 1]);
    }
    SFX(track_path)(&h, x, &o);
    for (int r = 0; r < N; ++r) {
      endpoints[2 * (i * N + r)] = x[r].re;
      endpoints[2 * (i * N + r) + 1] = x[r].im;
    }
    if (conv) conv[i] = o.converged;
    if (infy) infy[i] = o.infinity;
    if (status) status[i] = o.status;
    if (steps) steps[i] = o.steps;
    if (corr) corr[i] = o.corr;
    if (t_end) t_end[i] = o.t_end;
    if (dt_end) dt_end[i] = o.dt_end;
    if (resid) resid[i] = o.resid;
  }
  return 0;
}

/* One linear solve, exposed for the LU unit tests. */
int SFX(orc_lu_solve)(int32_t N, const REAL* A_rowmajor, const REAL* b, REAL* z) {
  if (N < 1 || N > ORC_NMAX) return -1;
  CX A[ORC_NMAX][ORC_NMAX], bb[ORC_NMAX], zz[ORC_NMAX];
  for (int r = 0; r < N; ++r) {
    for (int c = 0; c < N; ++c) A[r][c] = SFX(c_make)(A_rowmajor[2 * (r * N + c)], A_rowmajor[2 * (r * N + c) + 1]);
    bb[r] = SFX(c_make)(b[2 * r], b[2 * r + 1]);
  }
  SFX(lu_solve)(N, A, bb, zz);
  for (int r = 0; r < N; ++r) {
    z[2 * r] = zz[r].re;
    z[2 * r + 1] = zz[r].im;
  }
  return 0;
}

/* One linear solve with its pivot trace (piv [N], mags [N*N], see lu_solve_trace). */
int SFX(orc_lu_pivots)(int32_t N, const REAL* A_rowmajor, const REAL* b, REAL* z, int32_t* piv, REAL* mags) {
  if (N < 1 || N > ORC_NMAX) return -1;
  CX A[ORC_NMAX][ORC_NMAX], bb[ORC_NMAX], zz[ORC_NMAX];
  for (int r = 0; r < N; ++r) {
    for (int c = 0; c < N; ++c) A[r][c] = SFX(c_make)(A_rowmajor[2 * (r * N + c)], A_rowmajor[2 * (r * N + c) + 1]);
    bb[r] = SFX(c_make)(b[2 * r], b[2 * r + 1]);
  }
  SFX(lu_solve_trace)(N, A, bb, zz, piv, mags, NULL);
  for (int r = 0; r < N; ++r) {
    z[2 * r] = zz[r].re;
    z[2 * r + 1] = zz[r].im;
  }
  return 0;
}

/* H (which=0), -H_t (which=1) and H_x at (x, t) for one hypothesis; for evaluator tests. */
int SFX(orc_eval)(const orc_problem* pb, const REAL* coef_hx, const REAL* coef_ht, const REAL* p_start,
                  const REAL* p_tgt, const REAL* p_diff, const REAL* x_in, REAL t, REAL* H, REAL* Ht,
                  REAL* Hx) {
  const int N = pb->N;
  if (N < 1 || N > ORC_NMAX) return -1;
  HYP h;
  h.pb = pb;
  h.hx_coef = (const CX*)coef_hx;
  h.ht_coef = (const CX*)coef_ht;
  h.p_start = (const CX*)p_start;
  h.p_tgt = (const CX*)p_tgt;
  h.p_diff = (const CX*)p_diff;
  COEFS* cf = (COEFS*)malloc(sizeof(COEFS));
  SFX(eval_coefs)(&h, t, cf);
  CX x[ORC_NMAX + 1];
  for (int r = 0; r < N; ++r) x[r] = SFX(c_make)(x_in[2 * r], x_in[2 * r + 1]);
  x[N] = SFX(c_make)(1, 0);
  for (int r = 0; r < N; ++r) {
    CX hv = SFX(eval_h_row)(pb, cf, x, r, 0);
    CX tv = SFX(eval_h_row)(pb, cf, x, r, 1);
    H[2 * r] = hv.re;
    H[2 * r + 1] = hv.im;
    Ht[2 * r] = tv.re;
    Ht[2 * r + 1] = tv.im;
    CX A[ORC_NMAX];
    SFX(eval_hx_row)(pb, cf, x, r, A);
    for (int c = 0; c < N; ++c) {
      Hx[2 * (r * N + c)] = A[c].re;
      Hx[2 * (r * N + c) + 1] = A[c].im;
    }
  }
  free(cf);
  return 0;
}

#undef CX
#undef COEFS
#undef HYP
