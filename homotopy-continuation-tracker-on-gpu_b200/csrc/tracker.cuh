// tracker.cuh -- the homotopy path tracker for sm_100a.
//
// One sub-warp of W lanes (W = next power of two >= N, at least 4) tracks one
// path: lane r owns equation row r (its row of H_x lives in registers) and
// component r of the track.  The 32/W sub-warps of a warp run in lockstep
// through one warp-uniform loop (one path step per trip), so every shuffle and
// __syncwarp sees the full warp; a sub-warp whose path ends writes its
// endpoint and takes the next path from a global counter (work stealing).
//
// Per path step (reference GPU-HC/magmaHC/gpu-kernels/kernel_HC_Solver_P3P.cu:115-254,
// PH variant kernel_HC_Solver_trifocal_2op1p_30x30.cu:155-301):
//   end-zone clamp -> 4 RK stages (coefficients c_k(t) -> H_x, -H_t -> LU solve)
//   -> Newton corrector (H_x, H -> LU solve, success/infinity tests) -> step control.
//
// Arithmetic follows the oracle's operation order exactly (explicit fma,
// *_rn intrinsics so nothing else is contracted), so the FP64 tracker matches
// the oracle bit for bit.  Index tables are pre-compiled into term words
// (ghc_internal.h) and staged once per CTA in shared memory.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>
#include <type_traits>

#include "ghc_internal.h"

namespace ghc {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;

template <typename R>
struct cx {
  R re, im;
};

__device__ __forceinline__ double f_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float f_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double f_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double f_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double f_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float f_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double f_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float f_div(float a, float b) { return __fdiv_rn(a, b); }

template <typename R>
__device__ __forceinline__ cx<R>* view(unsigned char* p) {
  return reinterpret_cast<cx<R>*>(p);
}

template <typename R>
__device__ __forceinline__ cx<R> mk(R a, R b) {
  cx<R> r;
  r.re = a;
  r.im = b;
  return r;
}
template <typename R>
__device__ __forceinline__ cx<R> c_add(cx<R> a, cx<R> b) {
  return mk(f_add(a.re, b.re), f_add(a.im, b.im));
}
template <typename R>
__device__ __forceinline__ cx<R> c_sub(cx<R> a, cx<R> b) {
  return mk(f_sub(a.re, b.re), f_sub(a.im, b.im));
}
template <typename R>
__device__ __forceinline__ cx<R> c_scale(R s, cx<R> a) {
  return mk(f_mul(s, a.re), f_mul(s, a.im));
}
// a*b
template <typename R>
__device__ __forceinline__ cx<R> c_mul(cx<R> a, cx<R> b) {
  return mk(f_fma(a.re, b.re, -f_mul(a.im, b.im)), f_fma(a.re, b.im, f_mul(a.im, b.re)));
}
// c + a*b
template <typename R>
__device__ __forceinline__ cx<R> c_fma(cx<R> a, cx<R> b, cx<R> c) {
  return mk(f_fma(a.re, b.re, f_fma(-a.im, b.im, c.re)), f_fma(a.re, b.im, f_fma(a.im, b.re, c.im)));
}
// c - a*b
template <typename R>
__device__ __forceinline__ cx<R> c_fnma(cx<R> a, cx<R> b, cx<R> c) {
  return mk(f_fma(-a.re, b.re, f_fma(a.im, b.im, c.re)), f_fma(-a.re, b.im, f_fma(-a.im, b.re, c.im)));
}
// 1/b = conj(b) / |b|^2 with one correctly rounded reciprocal
__device__ __forceinline__ double f_rcp(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float f_rcp(float a) { return __frcp_rn(a); }
template <typename R>
__device__ __forceinline__ cx<R> c_rcp(cx<R> b) {
  const R s = f_fma(b.re, b.re, f_mul(b.im, b.im));
  const R inv = f_rcp(s);
  return mk(f_mul(b.re, inv), -f_mul(b.im, inv));
}
template <typename R>
__device__ __forceinline__ R c_abs2(cx<R> a) {
  return f_fma(a.re, a.re, f_mul(a.im, a.im));
}
template <typename R, typename S>
__device__ __forceinline__ cx<R> c_cast(cx<S> a) {
  return mk((R)a.re, (R)a.im);
}

__device__ __forceinline__ double shfl_xor(double v, int off, int w) { return __shfl_xor_sync(kFull, v, off, w); }
__device__ __forceinline__ float shfl_xor(float v, int off, int w) { return __shfl_xor_sync(kFull, v, off, w); }

// compiled tables staged in shared memory
struct Tables {
  const uint64_t* hx_terms;
  const uint16_t* hx_off;
  const uint64_t* ht_terms;
  const uint16_t* ht_off;
};

// acc += p * x[v0] * x[v1] ... over the term's variable slots (reference monomial term,
// dev-eval-indxing-P3P.cuh:70-118; slot N is the constant 1).  Every term of a table has
// the same number of slots: NV >= 0 fixes it at compile time (straight-line code), NV < 0
// reads it from the word.
template <typename R, int NV>
__device__ __forceinline__ cx<R> acc_term(cx<R> acc, cx<R> p, uint64_t w, const cx<R>* xs) {
  if constexpr (NV >= 0) {
    if (NV == 0) return c_add(acc, p);
#pragma unroll
    for (int q = 0; q < NV - 1; ++q) p = c_mul(p, xs[term_var(w, q)]);
    return c_fma(p, xs[term_var(w, NV - 1)], acc);
  } else {
    const int nv = term_nv(w);
    if (nv == 0) return c_add(acc, p);
#pragma unroll 1
    for (int q = 0; q < nv - 1; ++q) p = c_mul(p, xs[term_var(w, q)]);
    return c_fma(p, xs[term_var(w, nv - 1)], acc);
  }
}

// c_k(t), c'_k(t) for k = l, l+W, ... (reference eval_parameter_homotopy), computed in R and
// stored in RO; with HI the R values of c_k(t) are also kept in hi (the residual's copy)
template <typename R, typename RO, int W, bool HI>
__device__ __forceinline__ void coef_eval_p2c(const double* __restrict__ hx, const double* __restrict__ ht, int M,
                                              int K, R t, cx<RO>* c, cx<RO>* cp, cx<R>* hi, int l) {
  for (int k = l; k <= M; k += W) {
    const double* a = hx + 2 * (size_t)k * (K + 1);
    cx<R> v = mk((R)__ldg(a + 2 * K), (R)__ldg(a + 2 * K + 1));
    for (int j = K - 1; j >= 0; --j) v = mk(f_fma(v.re, t, (R)__ldg(a + 2 * j)), f_fma(v.im, t, (R)__ldg(a + 2 * j + 1)));
    c[k] = c_cast<RO>(v);
    if (HI) hi[k] = v;
    if (K >= 1) {
      const double* b = ht + 2 * (size_t)k * K;
      cx<R> u = mk((R)__ldg(b + 2 * (K - 1)), (R)__ldg(b + 2 * (K - 1) + 1));
      for (int j = K - 2; j >= 0; --j) u = mk(f_fma(u.re, t, (R)__ldg(b + 2 * j)), f_fma(u.im, t, (R)__ldg(b + 2 * j + 1)));
      cp[k] = c_cast<RO>(u);
    } else {
      cp[k] = mk(RO(0), RO(0));
    }
  }
}

// p(t) = p1 t + p0 (1-t) and the parameter differences (reference compute_param_homotopy), computed
// in R and stored in RO; with HI the R values of p(t) are also kept in hi
template <typename R, typename RO, int W, bool HI>
__device__ __forceinline__ void coef_eval_ph(const double* __restrict__ ps, const double* __restrict__ pt,
                                             const double* __restrict__ pd, int P, R t, cx<RO>* ph, cx<RO>* dp,
                                             cx<R>* hi, int l) {
  const R u = f_sub(R(1), t);
  for (int k = l; k < P; k += W) {
    const R gr = (R)__ldg(pt + 2 * k), gi = (R)__ldg(pt + 2 * k + 1);
    const R sr = (R)__ldg(ps + 2 * k), si = (R)__ldg(ps + 2 * k + 1);
    const cx<R> v = mk(f_fma(gr, t, f_mul(sr, u)), f_fma(gi, t, f_mul(si, u)));
    ph[k] = c_cast<RO>(v);
    if (HI) hi[k] = v;
    dp[k] = mk((RO)__ldg(pd + 2 * k), (RO)__ldg(pd + 2 * k + 1));
  }
  if (l == 0) {
    ph[P] = mk(RO(1), RO(0));
    if (HI) hi[P] = mk(R(1), R(0));
    dp[P] = mk((RO)__ldg(pd + 2 * P), (RO)__ldg(pd + 2 * P + 1));
  }
}

// term value p (coefficient, or product of two homotopy parameters, times the integer scale)
template <typename R, int KIND>
__device__ __forceinline__ cx<R> term_coef_value(uint64_t w, const cx<R>* ca) {
  if (KIND == KIND_P2C) return c_scale((R)term_scale(w), ca[term_coef(w)]);
  const cx<R> p = c_scale((R)term_scale(w), ca[term_pa(w)]);
  return c_mul(p, ca[term_pb(w)]);
}

// Row r of H_x into A.
//
// Flat (always above 16 unknowns, else when the problem's flat_eval is set):
// the row's terms are walked as one list (CSR row r, entry ends flagged in the term word),
// so a sub-warp spends max_r(terms of row r) iterations instead of
// sum_i max_r(terms of entry (r, i)).  The k-th non-zero entry of the row is
// staged in the sub-warp's scratch slot scr[k][r] (only as many slots as the
// fullest row has non-zero entries) and read back into registers through the
// lane's non-zero mask nz (entry i is in slot popc(nz & (2^i - 1))); every slot
// below the row's count is rewritten by every evaluation.  Balanced (walk 2): the
// entries are dealt to all W lanes at table-compile time by term count, a lane
// stores each finished sum into its row's slot, and the rows read their slots back
// after a sub-warp synchronisation (max over lanes instead of over rows: 65 -> 43
// iterations for the 5-point problem, whose rows hold 4..65 terms).  Entry-wise:
// one loop per column, straight into registers.  Every walk sums each entry in
// table order, as in the oracle.
template <int N>
constexpr bool kFlatAlways = N > 16;

// Row r of H (which = 0) or of -H_t (which = 1) from the H_t term table, in precision R
template <typename R, int N, int KIND, int NVT>
__device__ __forceinline__ cx<R> eval_rhs(const Tables& tb, const cx<R>* ca, const cx<R>* cb, const cx<R>* xs, int r,
                                          bool live, int which) {
  cx<R> h = mk(R(0), R(0));
  if (live) {
    const int len = tb.ht_off[r + 1] - tb.ht_off[r];
    for (int k = 0; k < len; ++k) {
      const uint64_t w = tb.ht_terms[k * N + r];
      cx<R> p;
      if (KIND == KIND_P2C) {
        p = c_scale((R)term_scale(w), which ? cb[term_coef(w)] : ca[term_coef(w)]);
      } else if (which) {
        const int a = term_pa(w), bb = term_pb(w);
        const cx<R> u = c_fma(cb[bb], ca[a], c_mul(cb[a], ca[bb]));
        p = c_scale((R)term_scale(w), u);
      } else {
        p = c_scale((R)term_scale(w), ca[term_pa(w)]);
        p = c_mul(p, ca[term_pb(w)]);
      }
      h = acc_term<R, NVT>(h, p, w, xs);
    }
  }
  return which ? mk(-h.re, -h.im) : h;
}

template <typename R, int N, int W, int KIND, int NVX>
__device__ __forceinline__ void eval_row(const Tables& tb, const cx<R>* ca, const cx<R>* xs, int r, bool live,
                                         cx<R> (&A)[N], int walk, unsigned char* scr, unsigned nz) {
  auto slot = [&](int k) -> cx<R>* { return view<R>(scr) + (k * W + r); };
  const int lanes = balanced_walk_built(N) ? tb.hx_off[N * N + 1] : kNoLanes;
  const bool balanced = balanced_walk_built(N) && walk == 2 && lanes != kNoLanes;
  if (!kFlatAlways<N> && walk == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      cx<R> acc = mk(R(0), R(0));
      if (live) {
        const int base = tb.hx_off[r * N], j0 = tb.hx_off[r * N + i], j1 = tb.hx_off[r * N + i + 1];
        for (int j = j0; j < j1; ++j) {
          const uint64_t w = tb.hx_terms[(j - base) * N + r];
          acc = acc_term<R, NVX>(acc, term_coef_value<R, KIND>(w, ca), w, xs);
        }
      }
      A[i] = acc;
    }
  } else if (balanced) {
    // this lane's share of the entries (every lane of the sub-warp takes part); each finished
    // sum goes into the slot of its row, read back after the sub-warp synchronises
    const int len = tb.hx_off[N * N + 2 + r];
    cx<R> acc = mk(R(0), R(0));
    for (int q = 0; q < len; ++q) {
      const uint64_t w = tb.hx_terms[lanes + q * W + r];
      acc = acc_term<R, NVX>(acc, term_coef_value<R, KIND>(w, ca), w, xs);
      if (term_last(w)) {
        view<R>(scr)[term_dst_slot(w) * W + term_dst_row(w)] = acc;
        acc = mk(R(0), R(0));
      }
    }
    __syncwarp(kFull);  // other lanes wrote this row's slots
#pragma unroll
    for (int i = 0; i < N; ++i)
      A[i] = ((nz >> i) & 1u) ? *slot(__popc(nz & ((1u << i) - 1u))) : mk(R(0), R(0));
  } else {
    if (live) {
      const int len = tb.hx_off[r * N + N] - tb.hx_off[r * N];
      int k = 0;
      cx<R> acc = mk(R(0), R(0));
      for (int q = 0; q < len; ++q) {
        const uint64_t w = tb.hx_terms[q * N + r];
        acc = acc_term<R, NVX>(acc, term_coef_value<R, KIND>(w, ca), w, xs);
        if (term_last(w)) {  // the entry's sum is complete
          *slot(k++) = acc;
          acc = mk(R(0), R(0));
        }
      }
    }
    // row-wise: this lane's own slots (each walk reads back inside its own branch: a read-back
    // shared by the walks after the branches cost hundreds of bytes of register spills)
#pragma unroll
    for (int i = 0; i < N; ++i)
      A[i] = ((nz >> i) & 1u) ? *slot(__popc(nz & ((1u << i) - 1u))) : mk(R(0), R(0));
  }
}

// Pivot key of a row for column i: magnitude |Re|+|Im| cut to its upper bits, position in the
// low 5 bits (largest key = largest cut magnitude, lowest position among equal ones).  Pivoted
// rows 0; a NaN at the current position wins, a NaN below never does.  The cut only speeds up the
// search: a near tie it gets wrong is found and redone on the full magnitudes (pivot_exact).
__device__ __forceinline__ unsigned mag_bits(double v) { return (unsigned)__double2hiint(v); }
__device__ __forceinline__ unsigned mag_bits(float v) { return __float_as_uint(v); }
template <typename R>
__device__ __forceinline__ unsigned pivot_key(R v, int pos, int i) {
  if (pos < i) return 0u;
  if (v != v) return (pos == i) ? (0xffffffe0u | (unsigned)(31 - pos)) : 0u;
  return ((mag_bits(v) >> 5) << 5) | (unsigned)(31 - pos);
}
__device__ __forceinline__ unsigned long long full_bits(double v) { return (unsigned long long)__double_as_longlong(v); }
__device__ __forceinline__ unsigned long long full_bits(float v) { return (unsigned long long)__float_as_uint(v); }

// compile-time loop: f(integral_constant<int, I>) for I in [B, E)
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// Partial-pivot LU + back substitution, one row per lane, rows in registers.
// The pivot is found by an integer max butterfly over the sub-warp.  A
// zero pivot skips that column's elimination and leaves a non-finite
// solution, as in the reference.  Solution lands in sol[0..N); sx holds two
// pivot-row buffers of N+1 entries (row + right-hand side), used by
// alternate columns so that one __syncwarp per column suffices.
//
// Two code shapes with the same operations in the same order:
//   LU_UNROLLED  every column unrolled at compile time (template recursion, so
//                the row stays in registers at any N; code grows as N^2),
//   LU_ROLLED    a rolled column loop whose row update runs over all N entries
//                predicated on j > i (N^2 instead of N^2/2 issue slots, code
//                linear in N).
// pragma unroll alone gives up above N = 16 and moves the row to local memory.
//   LU_SERIAL    (N <= 3) every lane of the sub-warp gathers the whole system
//                through shared memory and eliminates it in its registers, rows
//                swapped by selects: no pivot search across lanes and no
//                broadcast per column, so a lone small system's solve is a short
//                chain (the single-instance P3P case is latency bound).
constexpr int LU_UNROLLED = 0, LU_ROLLED = 1, LU_SERIAL = 2;
#ifndef GHC_LU_LARGE
#define GHC_LU_LARGE LU_UNROLLED
#endif
#ifndef GHC_LU_SERIAL_MAX_N
#define GHC_LU_SERIAL_MAX_N 3
#endif
template <int N>
constexpr int kLuForm = N <= GHC_LU_SERIAL_MAX_N ? LU_SERIAL : N <= 16 ? LU_UNROLLED : GHC_LU_LARGE;
// complex values of the per-sub-warp solve scratch sx: two pivot rows with their right-hand sides,
// or, for the serial form, the whole system
__host__ __device__ inline int lu_scratch_len(int N) {
  return N <= GHC_LU_SERIAL_MAX_N ? N * (N + 1) : 2 * (N + 1);
}

// Pivot position of column i by the reference's rule (dev-cgesv-batched-small.cuh:54-65): the
// largest |Re|+|Im| among the unpivoted rows, the lowest position among equal magnitudes, a NaN at
// position i kept and a NaN below never taken.  Sub-warps of 16 and 32 lanes: pivot_redux3 (below),
// exact in three warp reductions.  Narrower sub-warps, two steps:
//   pivot_fast   an integer max butterfly over pivot_key (one shuffle per level): the largest cut
//                magnitude, the lowest position among equal cut magnitudes;
//   cut_was_wrong  after the chosen row is broadcast, true on a lane whose row shares the winner's
//                cut magnitude but has a strictly larger full one -- the only way the cut choice
//                can differ from the exact one (equal full magnitudes are ordered by position in
//                both);
//   pivot_exact  the full magnitudes and the positions reduced as pairs, run (by the whole warp)
//                only when some lane saw cut_was_wrong.
template <typename R, int W>
__device__ __forceinline__ unsigned pivot_fast(unsigned key) {
  unsigned best = key;
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) best = max(best, __shfl_xor_sync(kFull, best, off, W));
  return best;
}
// (magnitudes compared as bit patterns: non-negative values order like their bits, and a NaN --
// only a NaN below the current position can share a bucket -- merely sends the column to the exact
// reduction, which never takes it)
template <typename R>
__device__ __forceinline__ bool cut_was_wrong(R m, unsigned key, unsigned best, bool cand, R pm) {
  return cand && ((key ^ best) >> 5) == 0u && full_bits(m) > full_bits(pm);
}
template <typename R, int W>
__device__ __forceinline__ int pivot_exact(R m, bool cand, int pos, int i) {
  // (magnitude bits, position): non-negative magnitudes order as their bit patterns; a NaN at
  // position i first, a NaN below and the pivoted rows last
  unsigned long long mb = 0ull;
  int mp = 64;
  if (cand) {
    if (m == m) {
      mb = full_bits(m);
      mp = pos;
    } else if (pos == i) {
      mb = ~0ull;
      mp = pos;
    }
  }
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(kFull, mb, off, W);
    const int op = __shfl_xor_sync(kFull, mp, off, W);
    if (ob > mb || (ob == mb && op < mp)) {
      mb = ob;
      mp = op;
    }
  }
  return mp;
}

// Warp reductions of the sub-warp (W = 16 or 32): max and min of a 32-bit value over the
// sub-warp's lanes; two sub-warps of 16 reduce at once, one by the operation, the other by the
// opposite operation on complemented values.
template <int W>
__device__ __forceinline__ unsigned subwarp_max(unsigned v) {
  static_assert(W == 16 || W == 32, "redux reductions need a sub-warp of 16 or 32");
  if constexpr (W == 32) {
    return __reduce_max_sync(kFull, v);
  } else {
    const bool upper = (threadIdx.x & 16u) != 0u;
    const unsigned lo = __reduce_max_sync(kFull, upper ? 0u : v);
    const unsigned hi = __reduce_min_sync(kFull, upper ? ~v : ~0u);
    return upper ? ~hi : lo;
  }
}
template <int W>
__device__ __forceinline__ unsigned subwarp_min(unsigned v) {
  static_assert(W == 16 || W == 32, "redux reductions need a sub-warp of 16 or 32");
  if constexpr (W == 32) {
    return __reduce_min_sync(kFull, v);
  } else {
    const bool upper = (threadIdx.x & 16u) != 0u;
    const unsigned lo = __reduce_min_sync(kFull, upper ? ~0u : v);
    const unsigned hi = __reduce_max_sync(kFull, upper ? ~v : 0u);
    return upper ? ~hi : lo;
  }
}
// The exact pivot position of column i in three sub-warp reductions (sub-warps of 16 or 32):
// the largest upper word of the candidates' magnitudes (shifted up by one so that a candidate
// with magnitude 0 still outranks a non-candidate; a NaN at position i above everything, a NaN
// below excluded), then the largest lower word among the candidates with that upper word, then
// the lowest position among those with both -- the reference's strict-> scan in position order.
// The candidate at position i always takes part, so some lane always wins.
template <typename R, int W>
__device__ __forceinline__ int pivot_redux3(R m, bool cand, int pos, int i) {
  const unsigned long long mb = full_bits(m);
  const unsigned hi = sizeof(R) == 8 ? (unsigned)(mb >> 32) : (unsigned)mb;
  unsigned khi = 0u;
  if (cand) khi = (m == m) ? hi + 1u : (pos == i ? 0xffffffffu : 0u);
  const unsigned top = subwarp_max<W>(khi);
  bool win = khi != 0u && khi == top;
  if constexpr (sizeof(R) == 8) {
    const unsigned lo = (unsigned)mb;
    const unsigned low = subwarp_max<W>(win ? lo : 0u);
    win = win && lo == low;
  }
  return (int)subwarp_min<W>(win ? (unsigned)pos : 63u);
}
template <int W>
constexpr bool kPivotRedux3 = W == 16 || W == 32;

// PivotRange: what one solve saw of its pivot magnitudes |U_ii| (|Re|+|Im|), in the oracle's
// comparison order.  singular(): a zero pivot, unless column 0's magnitude was NaN (the oracle's
// running minimum then stays NaN).  With SPAN (the mixed tracker's conditioning test) also the
// smallest and largest magnitudes and whether any was NaN; without it only two flags stay live
// across the LU.
template <typename R, bool SPAN>
struct PivotRange {
  R lo, hi;
  bool nan, zero, nan0;
  __device__ __forceinline__ void add(int i, R pm) {
    if (i == 0) {
      nan0 = pm != pm;
      zero = pm == R(0);
    } else {
      zero = zero || pm == R(0);
    }
    if constexpr (SPAN) {
      lo = (i == 0 || pm < lo) ? pm : lo;
      hi = (i == 0 || pm > hi) ? pm : hi;
      nan = (i != 0 && nan) || pm != pm;
    }
  }
  __device__ __forceinline__ bool singular() const { return zero && !nan0; }
};

template <typename R, int N, int W, bool SPAN>
__device__ __forceinline__ void lu_solve_unrolled(cx<R> (&A)[N], cx<R> b, int l, cx<R>* sx, cx<R>* sol,
                                                  PivotRange<R, SPAN>& rg) {
  const bool live = l < N;
  int pos = l;
  static_for<0, N>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    cx<R>* px = sx + (i & 1) * (N + 1);
    const R m = fabs(A[i].re) + fabs(A[i].im);
    const bool cand = live && pos >= i;
    int bp;
    unsigned key = 0u, best = 0u;
    if constexpr (kPivotRedux3<W>) {
      bp = pivot_redux3<R, W>(m, cand, pos, i);
    } else {
      key = live ? pivot_key(m, pos, i) : 0u;
      best = pivot_fast<R, W>(key);
      bp = 31 - (int)(best & 31u);
    }
    if (live && pos == bp) {
      static_for<i, N>([&](auto jc) { px[decltype(jc)::value] = A[decltype(jc)::value]; });
      px[N] = b;
    }
    __syncwarp(kFull);
    cx<R> p_i = px[i];
    R pm = fabs(p_i.re) + fabs(p_i.im);
    if (!kPivotRedux3<W> && __any_sync(kFull, cut_was_wrong(m, key, best, cand, pm))) {
      bp = pivot_exact<R, W>(m, cand, pos, i);
      __syncwarp(kFull);  // every lane has read the first choice
      if (live && pos == bp) {
        static_for<i, N>([&](auto jc) { px[decltype(jc)::value] = A[decltype(jc)::value]; });
        px[N] = b;
      }
      __syncwarp(kFull);
      p_i = px[i];
      pm = fabs(p_i.re) + fabs(p_i.im);
    }
    const bool is_piv = live && (pos == bp);
    if (live) {
      if (pos == bp) pos = i;
      else if (pos == i) pos = bp;
    }
    const bool zero = (pm == R(0));
    rg.add(i, pm);
    // (a zero pivot's reciprocal is NaN, as the oracle's c_rcp(0))
    const cx<R> rc = c_rcp(p_i);
    // the pivot row's reciprocal waits in the solution slot of its position until the back
    // substitution (the slot is written there only after this lane has read it)
    if (is_piv) sol[i] = rc;
    // rows below the pivot take the update, the others keep their values
    const bool upd = live && pos > i && !zero;
    if (upd) {
      A[i] = c_mul(A[i], rc);
      static_for<i + 1, N>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        A[j] = c_fnma(A[i], px[j], A[j]);
      });
      b = c_fnma(A[i], px[N], b);
    }
  });
  static_for<0, N>([&](auto ic) {
    constexpr int i = N - 1 - decltype(ic)::value;
    if (live && pos == i) sol[i] = c_mul(b, sol[i]);
    __syncwarp(kFull);
    const cx<R> xi = sol[i];
    if (live && pos < i) b = c_fnma(A[i], xi, b);
  });
  __syncwarp(kFull);
}

template <typename R, int N>
__device__ __forceinline__ cx<R> pick(const cx<R> (&A)[N], int i) {
  cx<R> a = A[0];
#pragma unroll
  for (int j = 1; j < N; ++j)
    if (j == i) a = A[j];
  return a;
}

template <typename R, int N, int W, bool SPAN>
__device__ __forceinline__ void lu_solve_rolled(cx<R> (&A)[N], cx<R> b, int l, cx<R>* sx, cx<R>* sol,
                                                PivotRange<R, SPAN>& rg) {
  const bool live = l < N;
  int pos = l;
  cx<R> myrcp = mk(R(0), R(0));
#pragma unroll 1
  for (int i = 0; i < N; ++i) {
    cx<R> ai = pick(A, i);
    const R m = fabs(ai.re) + fabs(ai.im);
    const bool cand = live && pos >= i;
    const unsigned key = live ? pivot_key(m, pos, i) : 0u;
    const unsigned best = pivot_fast<R, W>(key);
    int bp = 31 - (int)(best & 31u);
    if (live && pos == bp) {
#pragma unroll
      for (int j = 0; j < N; ++j)
        if (j >= i) sx[j] = A[j];
      sx[N] = b;
    }
    __syncwarp(kFull);
    cx<R> p_i = sx[i];
    R pm = fabs(p_i.re) + fabs(p_i.im);
    if (__any_sync(kFull, cut_was_wrong(m, key, best, cand, pm))) {
      bp = pivot_exact<R, W>(m, cand, pos, i);
      __syncwarp(kFull);  // every lane has read the first choice
      if (live && pos == bp) {
#pragma unroll
        for (int j = 0; j < N; ++j)
          if (j >= i) sx[j] = A[j];
        sx[N] = b;
      }
      __syncwarp(kFull);
      p_i = sx[i];
      pm = fabs(p_i.re) + fabs(p_i.im);
    }
    const bool is_piv = live && (pos == bp);
    if (live) {
      if (pos == bp) pos = i;
      else if (pos == i) pos = bp;
    }
    const bool zero = (pm == R(0));
    rg.add(i, pm);
    const cx<R> rc = c_rcp(zero ? mk(R(0), R(0)) : p_i);
    if (is_piv) myrcp = rc;
    if (live && pos > i && !zero) {
      ai = c_mul(ai, rc);
#pragma unroll
      for (int j = 0; j < N; ++j) {
        if (j == i) A[j] = ai;
        if (j > i) A[j] = c_fnma(ai, sx[j], A[j]);
      }
      b = c_fnma(ai, sx[N], b);
    }
    __syncwarp(kFull);
  }
#pragma unroll 1
  for (int i = N - 1; i >= 0; --i) {
    if (live && pos == i) sol[i] = c_mul(b, myrcp);
    __syncwarp(kFull);
    const cx<R> xi = sol[i];
    if (live && pos < i) b = c_fnma(pick(A, i), xi, b);
  }
  __syncwarp(kFull);
}

// The serial form: the oracle's elimination (rows at positions, strict-> scan from position i,
// zero pivot skipping its column, back substitution by the stored reciprocals) run by every lane
// on its own copy of the system; lane l leaves component l of the solution in sol[l].
template <typename R, int N, int W, bool SPAN>
__device__ __forceinline__ void lu_solve_serial(cx<R> (&A)[N], cx<R> b, int l, cx<R>* sx, cx<R>* sol,
                                                PivotRange<R, SPAN>& rg) {
  constexpr int C = N + 1;  // row length with the right-hand side
  if (l < N) {
    static_for<0, N>([&](auto jc) { sx[l * C + decltype(jc)::value] = A[decltype(jc)::value]; });
    sx[l * C + N] = b;
  }
  __syncwarp(kFull);
  cx<R> M[N][C];
  static_for<0, N>([&](auto rc_) {
    static_for<0, C>([&](auto jc) { M[decltype(rc_)::value][decltype(jc)::value] = sx[decltype(rc_)::value * C + decltype(jc)::value]; });
  });
  __syncwarp(kFull);  // every lane has its copy before the next solve rewrites sx
  cx<R> rcp[N];
  static_for<0, N>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    R best = fabs(M[i][i].re) + fabs(M[i][i].im);
    int bp = i;
    static_for<i + 1, N>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      const R v = fabs(M[j][i].re) + fabs(M[j][i].im);
      if (v > best) {
        best = v;
        bp = j;
      }
    });
    rg.add(i, best);
    // the pivot row moves to position i, the row at position i to the pivot's position
    static_for<i + 1, N>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      if (bp == j) {
        static_for<i, C>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          const cx<R> t = M[i][k];
          M[i][k] = M[j][k];
          M[j][k] = t;
        });
      }
    });
    const bool zero = best == R(0);
    rcp[i] = c_rcp(M[i][i]);
    if (!zero) {
      static_for<i + 1, N>([&](auto rc_) {
        constexpr int r = decltype(rc_)::value;
        M[r][i] = c_mul(M[r][i], rcp[i]);
        static_for<i + 1, C>([&](auto jc) {
          constexpr int j = decltype(jc)::value;
          M[r][j] = c_fnma(M[r][i], M[i][j], M[r][j]);
        });
      });
    }
  });
  cx<R> z[N];
  static_for<0, N>([&](auto ic) {
    constexpr int i = N - 1 - decltype(ic)::value;
    z[i] = c_mul(M[i][N], rcp[i]);
    static_for<0, i>([&](auto rc_) {
      constexpr int r = decltype(rc_)::value;
      M[r][N] = c_fnma(M[r][i], z[i], M[r][N]);
    });
  });
  cx<R> mine = z[0];
  static_for<1, N>([&](auto jc) {
    if (l == decltype(jc)::value) mine = z[decltype(jc)::value];
  });
  if (l < N) sol[l] = mine;
  __syncwarp(kFull);
}

template <typename R, int N, int W, bool SPAN>
__device__ __forceinline__ void lu_solve(cx<R> (&A)[N], cx<R> b, int l, cx<R>* sx, cx<R>* sol,
                                         PivotRange<R, SPAN>& rg) {
  if constexpr (kLuForm<N> == LU_SERIAL) lu_solve_serial<R, N, W>(A, b, l, sx, sol, rg);
  else if constexpr (kLuForm<N> == LU_ROLLED) lu_solve_rolled<R, N, W>(A, b, l, sx, sol, rg);
  else lu_solve_unrolled<R, N, W>(A, b, l, sx, sol, rg);
}
template <typename R, int N, int W>
__device__ __forceinline__ void lu_solve(cx<R> (&A)[N], cx<R> b, int l, cx<R>* sx, cx<R>* sol) {
  PivotRange<R, false> rg;
  lu_solve<R, N, W>(A, b, l, sx, sol, rg);
}

// xor-butterfly sum over the first NP lanes of the sub-warp (order = oracle tree_sum)
template <typename R, int N, int W>
__device__ __forceinline__ R tree_sum(R v) {
  constexpr int NP = (N <= 1) ? 1 : (N <= 2) ? 2 : (N <= 4) ? 4 : (N <= 8) ? 8 : (N <= 16) ? 16 : 32;
  static_assert(NP <= W, "sub-warp narrower than the reduction tree");
#pragma unroll
  for (int off = NP / 2; off > 0; off >>= 1) v = f_add(v, shfl_xor(v, off, W));
  return v;
}

// per-sub-warp shared-memory views
struct SubMem {
  unsigned char* coefA;  // c_k(t)   or p(t)     [Mc]
  unsigned char* coefB;  // c'_k(t)  or p1 - p0  [Mc]
  unsigned char* xs;     // track [N+1]
  unsigned char* sx;     // solve scratch [lu_scratch_len(N)]: two pivot rows + rhs, or the whole system
  unsigned char* sol;    // solution [N]
  unsigned char* state;  // per lane: RK base point x0 [W], RK accumulator [W] (state precision)
  unsigned char* scr;    // H_x row scratch [slots][W], null unless the evaluation is flat
  unsigned char* rec;    // the path's scalar state while the sub-warp evaluates and solves [kRecBytes]
  unsigned char* coefH;  // mixed: c_k(t) or p(t) in state precision, for the residual H [Mc] (else null)
  unsigned char* xsH;    // mixed: the track in state precision [N+1] (else null)
  unsigned char* xst;    // the track in state precision: xsH when mixed, else xs
  unsigned nz;           // this lane's row: bit i set when H_x entry (row, i) has terms
  int walk;              // H_x walk: 0 entry-wise, 1 row-wise, 2 balanced
};
constexpr int kRecBytes = 128;

// bit i set when row r of H_x has terms in column i (0 for lanes beyond the rows)
template <int N>
__device__ __forceinline__ unsigned row_mask(const uint16_t* hx_off, int r) {
  unsigned m = 0u;
  if (r < N)
    for (int i = 0; i < N; ++i)
      if (hx_off[r * N + i + 1] > hx_off[r * N + i]) m |= 1u << i;
  return m;
}

// Row l of H_x and the right-hand side (which = 1: -H_t, which = 0: H), term walk of table shape S
// (EvalShape), in the linear-algebra precision RL.  With a state precision R above RL (mixed), the
// corrector's H is evaluated in R from the R copies of the coefficients and the track, then rounded
// to RL for the solve: Newton then converges to the R-accurate root at a rate set by the RL solve.
template <typename R, typename RL, int N, int W, int KIND, int S>
__device__ __forceinline__ void eval_any(const Tables& tb, const SubMem& sm, int l, cx<RL> (&A)[N], cx<RL>& b,
                                         int which) {
  eval_row<RL, N, W, KIND, shape_nvx(S)>(tb, view<RL>(sm.coefA), view<RL>(sm.xs), l, l < N, A, sm.walk, sm.scr,
                                         sm.nz);
  if constexpr (std::is_same<R, RL>::value) {
    b = eval_rhs<RL, N, KIND, shape_nvt(S)>(tb, view<RL>(sm.coefA), view<RL>(sm.coefB), view<RL>(sm.xs), l, l < N,
                                            which);
  } else {
    if (which)
      b = eval_rhs<RL, N, KIND, shape_nvt(S)>(tb, view<RL>(sm.coefA), view<RL>(sm.coefB), view<RL>(sm.xs), l,
                                              l < N, 1);
    else
      b = c_cast<RL>(eval_rhs<R, N, KIND, shape_nvt(S)>(tb, view<R>(sm.coefH), view<R>(sm.coefH), view<R>(sm.xsH),
                                                        l, l < N, 0));
  }
}

// one evaluation + solve in precision RL; returns this lane's solution component in R.  ill (mixed
// tracker, cond_limit > 0): the pivot magnitudes spanned more than cond_limit or one was NaN -- the
// RL solve is too ill-conditioned to keep Newton's contraction
template <typename R, typename RL, int N, int W, int KIND, int S>
__device__ __forceinline__ cx<R> eval_solve(const Tables& tb, const SubMem& sm, int l, int which, double cond_limit,
                                            bool& ill, bool& sing) {
  cx<RL> A[N];
  cx<RL> b;
  eval_any<R, RL, N, W, KIND, S>(tb, sm, l, A, b, which);
  constexpr bool kSpan = !std::is_same<R, RL>::value;  // only the mixed tracker tests conditioning
  PivotRange<RL, kSpan> rg;
  lu_solve<RL, N, W>(A, b, l, view<RL>(sm.sx), view<RL>(sm.sol), rg);
  if constexpr (kSpan) ill = cond_limit > 0.0 && (rg.nan || !(rg.hi <= (RL)cond_limit * rg.lo));
  else ill = false;
  sing = rg.singular();
  const cx<RL> k = (l < N) ? view<RL>(sm.sol)[l] : mk(RL(0), RL(0));
  return c_cast<R>(k);
}
template <typename R, typename RL, int N, int W, int KIND, int S>
__device__ __forceinline__ cx<R> eval_solve(const Tables& tb, const SubMem& sm, int l, int which) {
  bool ill, sing;
  return eval_solve<R, RL, N, W, KIND, S>(tb, sm, l, which, 0.0, ill, sing);
}

// the track into shared memory: in RL for H_x and H_t, and (mixed) in R for the residual
template <typename R, typename RL, int N>
__device__ __forceinline__ void write_track(const SubMem& sm, int l, cx<R> x) {
  cx<RL>* xs = view<RL>(sm.xs);
  if (l < N) xs[l] = c_cast<RL>(x);
  if (l == 0) xs[N] = mk(RL(1), RL(0));
  if constexpr (!std::is_same<R, RL>::value) {
    cx<R>* xh = view<R>(sm.xsH);
    if (l < N) xh[l] = x;
    if (l == 0) xh[N] = mk(R(1), R(0));
  }
}

template <typename R, typename RL, int W, int KIND>
__device__ __forceinline__ void coef_eval(const TrackParams& p, const SubMem& sm, long long hyp, R t, int l) {
  constexpr bool HI = !std::is_same<R, RL>::value;
  if (KIND == KIND_P2C) {
    coef_eval_p2c<R, RL, W, HI>(p.coef_hx + 2 * hyp * p.stride_hx, p.coef_ht + 2 * hyp * p.stride_ht, p.M, p.K, t,
                                view<RL>(sm.coefA), view<RL>(sm.coefB), view<R>(sm.coefH), l);
  } else {
    coef_eval_ph<R, RL, W, HI>(p.p_start, p.p_tgt + 2 * hyp * p.stride_p, p.p_diff + 2 * hyp * p.stride_p, p.P, t,
                               view<RL>(sm.coefA), view<RL>(sm.coefB), view<R>(sm.coefH), l);
  }
}

// byte sizes of the shared-memory layout
__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }
__host__ __device__ inline size_t tables_bytes(int N, int n_hx, int n_ht) {
  return align16(8 * (size_t)(n_hx + n_ht) + 2 * (size_t)(hx_off_len(N) + N + 1));
}
// Per sub-warp: the path record [kRecBytes], then, in complex values of e bytes (linear-algebra
// precision): coefficient buffers [2 Mc], track [N+1], solve scratch [lu_scratch_len(N)], solution [N]; the
// lane state [2 W] in complex values of es bytes (state precision); scratch slots [slots W] (flat);
// and, when es != e (mixed), the state-precision coefficients [Mc] and track [N+1].
struct SubOffsets {
  size_t coefA, coefB, xs, sx, sol, state, scr, coefH, xsH, bytes;
};
__host__ __device__ inline SubOffsets sub_offsets(int N, int Mc, int W, int slots, int e, int es) {
  const bool mixed = es != e;
  SubOffsets o;
  size_t off = kRecBytes;
  o.coefA = off;
  off += (size_t)e * Mc;
  o.coefB = off;
  off += (size_t)e * Mc;
  o.xs = off;
  off += (size_t)e * (N + 1);
  o.sx = off;
  off += (size_t)e * lu_scratch_len(N);
  o.sol = off;
  off += (size_t)e * N;
  if (mixed) off = align16(off);
  o.state = off;
  off += (size_t)es * 2 * W;
  o.scr = off;
  off += (size_t)e * slots * W;
  o.coefH = o.xsH = 0;
  if (mixed) {
    off = align16(off);
    o.coefH = off;
    off += (size_t)es * Mc;
    o.xsH = off;
    off += (size_t)es * (N + 1);
  }
  o.bytes = kRecBytes + align16(off - kRecBytes);
  return o;
}
__host__ __device__ inline size_t sub_bytes(int N, int Mc, int W, int slots, int e, int es) {
  return sub_offsets(N, Mc, W, slots, e, es).bytes;
}
template <typename R, typename RL>
__device__ __forceinline__ SubMem sub_layout(unsigned char* base, int N, int Mc, int W, int slots, bool flat) {
  const SubOffsets o = sub_offsets(N, Mc, W, flat ? slots : 0, (int)sizeof(cx<RL>), (int)sizeof(cx<R>));
  SubMem sm;
  sm.rec = base;
  sm.coefA = base + o.coefA;
  sm.coefB = base + o.coefB;
  sm.xs = base + o.xs;
  sm.sx = base + o.sx;
  sm.sol = base + o.sol;
  sm.state = base + o.state;
  sm.scr = flat ? base + o.scr : nullptr;
  const bool mixed = !std::is_same<R, RL>::value;
  sm.coefH = mixed ? base + o.coefH : nullptr;
  sm.xsH = mixed ? base + o.xsH : nullptr;
  sm.xst = mixed ? sm.xsH : sm.xs;
  return sm;
}

// complex entry idx of an array of doubles (f64) or floats, in precision R
template <typename R>
__device__ __forceinline__ cx<R> load_cx(const void* base, bool f64, long long idx) {
  if (f64) {
    const double* d = reinterpret_cast<const double*>(base) + 2 * idx;
    return mk((R)d[0], (R)d[1]);
  }
  const float* f = reinterpret_cast<const float*>(base) + 2 * idx;
  return mk((R)f[0], (R)f[1]);
}

// CTAs per SM the tracker asks the register allocator for: the row of H_x (N
// complex values) dominates the registers, so small systems afford more.  Two
// compiled variants per size and precision; the autotuner (ghc_autotune) picks
// one per problem.  Variant 0 is the best of B200 sweeps over the shipped
// problems (512 hypotheses, autotuning off, 3..7 CTAs): FP64 N = 3 at 6 (at 8
// the 64 registers spill), N = 6 flat within noise, N = 12 at 5 (generalized
// 3-view 5360 vs 5326 hyp/s at 4, uncalibrated trifocal 1376 vs 1348; 6 and 7
// spill), N = 30 at 3 (406 vs 397 at 4); FP32 N = 12 at 7, N = 30 at 5 (577
// vs 552 at 3).  Variant 1 is the runner-up budget.  The mixed tracker (FP64 state, FP32
// linear algebra) holds the row in FP32 and asks for about the FP32 budget.
template <int N, typename R, typename RL, int V>
constexpr int track_min_blocks() {
  return !std::is_same<R, RL>::value
             ? (V == 0 ? (N <= 8 ? 6 : N <= 12 ? 6 : N <= 18 ? 4 : 4) : (N <= 8 ? 8 : N <= 12 ? 5 : N <= 18 ? 5 : 3))
         : V == 0 ? (sizeof(R) == 8 ? (N <= 4 ? 6 : N <= 8 ? 4 : N <= 12 ? 5 : 3)
                                    : (N <= 8 ? 8 : N <= 12 ? 7 : N <= 18 ? 4 : 5))
                  : (sizeof(R) == 8 ? (N <= 4 ? 8 : N <= 8 ? 6 : N <= 12 ? 4 : N <= 18 ? 4 : 2)
                                    : (N <= 8 ? 10 : N <= 12 ? 8 : N <= 18 ? 5 : 4));
}

__device__ __forceinline__ Tables stage_tables(unsigned char* smem, const uint64_t* g_hx, const uint16_t* g_hxo,
                                               const uint64_t* g_ht, const uint16_t* g_hto, int N, int n_hx,
                                               int n_ht) {
  uint64_t* s_hx = reinterpret_cast<uint64_t*>(smem);
  uint64_t* s_ht = s_hx + n_hx;
  uint16_t* s_hxo = reinterpret_cast<uint16_t*>(s_ht + n_ht);
  uint16_t* s_hto = s_hxo + hx_off_len(N);
  for (int i = threadIdx.x; i < n_hx; i += blockDim.x) s_hx[i] = __ldg(g_hx + i);
  for (int i = threadIdx.x; i < n_ht; i += blockDim.x) s_ht[i] = __ldg(g_ht + i);
  for (int i = threadIdx.x; i < hx_off_len(N); i += blockDim.x) s_hxo[i] = __ldg(g_hxo + i);
  for (int i = threadIdx.x; i < N + 1; i += blockDim.x) s_hto[i] = __ldg(g_hto + i);
  __syncthreads();
  Tables t;
  t.hx_terms = s_hx;
  t.hx_off = s_hxo;
  t.ht_terms = s_ht;
  t.ht_off = s_hto;
  return t;
}

// -------------------------------------------------------------------------------------------------
// the tracker kernel: state, step control and norms in precision R, H_x, H_t and the LU in RL
// (R = RL: the plain FP64 and FP32 trackers; R = double, RL = float: the mixed tracker, whose
// corrector evaluates its residual H in R, so its endpoints converge to FP64 accuracy)
//
// Each sub-warp runs its path as a small state machine (phase 0..3 = RK stage,
// 4 = Newton iteration).  One trip of the warp loop performs exactly one
// evaluate-and-solve for every sub-warp, whatever its phase, so the unrolled
// LU exists once in the code and sub-warps of one warp never wait on each
// other's corrector iterations.
//
// Handover (first phase of the mixed-precision mode: t_handover > 0 or
// fail_limit > 0): a path also stops when t reaches t_handover, after
// fail_limit consecutive failed steps, or when the corrector sees divergence,
// leaving its last accepted point, t and dt in endpoints / t_end / dt_end.
// A resuming launch (resume = 1) starts every item from track_in at t_in[i]
// with step dt_in[i] and the step / corrector counts already in steps / corr.
// -------------------------------------------------------------------------------------------------
#ifdef GHC_TRACK_MIN_BLOCKS
#define GHC_MINB(N, R, RL, V) GHC_TRACK_MIN_BLOCKS
#else
#define GHC_MINB(N, R, RL, V) ::ghc::dev::track_min_blocks<N, R, RL, V>()
#endif
// Threads per CTA of a tracker instantiation (the launch may still halve it when the per-sub-warp
// shared memory does not fit).  128 everywhere by default.
template <int N, typename R, typename RL, int V>
constexpr int track_block() {
  return 128;
}
#ifdef GHC_TRACK_BLOCK
#define GHC_BLOCK(N, R, RL, V) GHC_TRACK_BLOCK
#else
#define GHC_BLOCK(N, R, RL, V) ::ghc::dev::track_block<N, R, RL, V>()
#endif
// WK >= 0: the H_x walk is fixed at compile time (only that walk's code is in the kernel, which
// spares the register allocator the other walk's read-back: above 16 unknowns, where the row fills
// most of the registers); WK < 0: chosen at run time from p.flat_eval.
//
// track_body is the work of one CTA on the items of p: CTA number `cta` of the `n_cta` CTAs that
// serve p (first items static: one per sub-warp slot of the CTA; then the shared counter), or,
// as a `visitor` (a CTA of another bucket of a mixed launch whose own items are done), items
// from p's counter only.  smem: the CTA's dynamic shared memory.
template <typename R, typename RL, int N, int W, int KIND, int S, int WK>
__device__ __forceinline__ void track_body(const TrackParams& p, unsigned char* smem, long long cta, long long n_cta,
                                           bool visitor) {
  const Tables tb = stage_tables(smem, p.hx_terms, p.hx_off, p.ht_terms, p.ht_off, N, p.n_hx_terms, p.n_ht_terms);

  const int lane = threadIdx.x & 31;
  const int l = lane % W;
  const int g = threadIdx.x / W;
  const int Mc = (KIND == KIND_P2C) ? p.M + 1 : p.P + 1;
  const int walk = WK >= 0 ? WK : ((kFlatAlways<N> && p.flat_eval == 0) ? 1 : p.flat_eval);
  const bool flat = walk != 0;
  SubMem sm = sub_layout<R, RL>(smem + tables_bytes(N, p.n_hx_terms, p.n_ht_terms) +
                                    (size_t)g * sub_bytes(N, Mc, W, flat ? p.scr_slots : 0, (int)sizeof(cx<RL>),
                                                          (int)sizeof(cx<R>)),
                                N, Mc, W, p.scr_slots, flat);
  sm.nz = row_mask<N>(tb.hx_off, l);
  sm.walk = walk;
  // this lane's RK base point x0 and accumulator sols live in shared memory (register relief)
  cx<R>& x0 = view<R>(sm.state)[l];
  cx<R>& sols = view<R>(sm.state)[W + l];

  // Paths go to sub-warps in order, or, when the launch has fewer paths than one wave of warps
  // (spread), one path to each warp: a lone instance then has no two paths in one warp, whose
  // phases would serialise each other's step logic.  The other sub-warps of the warp track the
  // same path in lockstep (identical work, so no divergence and no idle lanes computing on stale
  // shared memory); only the first one (primary) writes results and takes the next path.
  const int subs_per_cta = blockDim.x / W;
  const int slots_per_cta = p.spread ? (int)(blockDim.x / 32) : subs_per_cta;
  const long long n_sw = n_cta * slots_per_cta;
  const bool primary = !p.spread || lane < W;
  const int leader = lane - l;
  const bool handover = p.t_handover > 0.0 || p.fail_limit > 0;
  const R t_hand = (R)p.t_handover;

  // per-path state (replicated across the sub-warp's lanes)
  long long item = p.spread ? cta * slots_per_cta + (threadIdx.x >> 5) : cta * subs_per_cta + g;
  if (visitor) {  // the first item from the counter too (the static ones belong to p's own CTAs)
    long long nxt = 0;
    if (l == 0 && primary) nxt = n_sw + (long long)atomicAdd(reinterpret_cast<unsigned*>(p.counter), 1u);
    item = __shfl_sync(kFull, nxt, p.spread ? 0 : leader);
  }
  bool alive = item < p.n_items;
  long long hyp = 0;
  cx<R> x = mk(R(0), R(0));
  R t0 = 0, dt = 0, t_step = 0, half = 0, dt_pre = 0;
  R coef_t = R(-1);  // the t at which this sub-warp's coefficient buffers hold c_k(t) (-1: none)
  bool end_zone = false, success = false, inf = false, finished = false;
  // mixed tracker only: a solve of this step was ill-conditioned, or the step fell below the floor: stop
  constexpr bool kMixed = !std::is_same<R, RL>::value;
  bool step_ill = false, ill_stop = false;
  bool step_sing = false, last_sing = false;  // a solve of this step / the last completed step had a zero pivot
  int nsucc = 0, step = 0, ncorr = 0, phase = 0, cit = 0, nfail = 0;
  const R dt_init = (KIND == KIND_PH) ? R(0.01) : R(0.05);

  // end-zone clamp and bookkeeping at the start of a step (kernel_HC_Solver_P3P.cu:121-134)
  auto prologue = [&]() {
    if (!end_zone && fabs(f_sub(R(1), t0)) <= R(0.0500001)) end_zone = true;
    if (end_zone) {
      const R rem = fabs(f_sub(R(1), t0));
      if (dt > rem) dt = rem;
    } else {
      const R edge = (KIND == KIND_PH) ? fabs(f_sub(R(0.95), t0)) : fabs(f_sub(f_sub(R(1), R(0.05)), t0));
      if (dt > edge) dt = edge;
    }
    dt_pre = dt;  // the step without the handover clamp: the next phase resumes with it
    if (p.t_handover > 0.0 && dt > f_sub(t_hand, t0)) dt = f_sub(t_hand, t0);
    t_step = t0;
    half = f_mul(R(0.5), dt);
    phase = 0;
    cit = 0;
    step_ill = false;
    step_sing = false;
  };
  // the path stops before its next step (kernel_HC_Solver_P3P.cu:247-249, plus the handover rules)
  auto at_end = [&]() -> bool {
    return !(t0 < R(1) && f_sub(R(1), t0) > R(1e-7)) || step > p.max_steps ||
           (p.t_handover > 0.0 && f_sub(t_hand, t0) <= R(1e-6)) || (p.fail_limit > 0 && nfail >= p.fail_limit) ||
           (kMixed && ill_stop);
  };
  auto init_path = [&](long long it) {
    hyp = it / p.paths_per_hyp;
    const long long pidx = it % p.paths_per_hyp;
    if (l < N) {
      if (p.track_in) {
        x = load_cx<R>(p.track_in, (sizeof(R) == 8) != (p.track_other != 0), it * p.ld_track + l);
      } else {
        x = load_cx<R>(p.start_sols, (sizeof(R) == 8) != (p.start_other != 0), pidx * p.ld_start + l);
      }
    } else {
      x = mk(R(0), R(0));
    }
    x0 = x;
    sols = x;
    t0 = p.t_in ? (R)p.t_in[it] : R(0);
    coef_t = R(-1);  // a new path may belong to another hypothesis
    dt = p.dt_in ? (R)p.dt_in[it] : dt_init;
    dt_pre = dt;
    step = p.resume ? p.steps[it] : 0;
    ncorr = p.resume ? p.corr[it] : 0;
    end_zone = false;
    success = false;
    inf = false;
    nsucc = 0;
    nfail = 0;
    step_ill = ill_stop = step_sing = last_sing = false;
    finished = at_end();
    if (!finished) prologue();
  };
  if (alive) init_path(item);

  // The path's scalar state (the same in every lane of the sub-warp) and this lane's track
  // component wait in shared memory while the sub-warp evaluates and solves, so that no
  // register holds them across the LU (register relief).  Volatile: stored and reloaded,
  // never forwarded.
  volatile R* rec_r = reinterpret_cast<volatile R*>(sm.rec);
  volatile long long* rec_l = reinterpret_cast<volatile long long*>(sm.rec + 6 * sizeof(R));
  volatile int* rec_i = reinterpret_cast<volatile int*>(sm.rec + 6 * sizeof(R) + 2 * sizeof(long long));
  auto stash = [&]() {
    rec_r[0] = t0;
    rec_r[1] = dt;
    rec_r[2] = t_step;
    rec_r[3] = half;
    rec_r[4] = dt_pre;
    rec_r[5] = coef_t;
    rec_l[0] = item;
    rec_l[1] = hyp;
    rec_i[0] = step;
    rec_i[1] = ncorr;
    rec_i[2] = phase;
    rec_i[3] = cit;
    rec_i[4] = nfail;
    rec_i[5] = nsucc;
    rec_i[6] = (alive ? 1 : 0) | (finished ? 2 : 0) | (end_zone ? 4 : 0) | (success ? 8 : 0) | (inf ? 16 : 0) |
               (step_ill ? 32 : 0) | (ill_stop ? 64 : 0) | (step_sing ? 128 : 0) | (last_sing ? 256 : 0);
  };
  auto unstash = [&]() {
    t0 = rec_r[0];
    dt = rec_r[1];
    t_step = rec_r[2];
    half = rec_r[3];
    dt_pre = rec_r[4];
    coef_t = rec_r[5];
    item = rec_l[0];
    hyp = rec_l[1];
    step = rec_i[0];
    ncorr = rec_i[1];
    phase = rec_i[2];
    cit = rec_i[3];
    nfail = rec_i[4];
    nsucc = rec_i[5];
    const int f = rec_i[6];
    alive = f & 1;
    finished = (f >> 1) & 1;
    end_zone = (f >> 2) & 1;
    success = (f >> 3) & 1;
    inf = (f >> 4) & 1;
    step_ill = (f >> 5) & 1;
    ill_stop = (f >> 6) & 1;
    step_sing = (f >> 7) & 1;
    last_sing = (f >> 8) & 1;
    const volatile cx<R>* xv = reinterpret_cast<const volatile cx<R>*>(sm.xst);
    x = (l < N) ? mk(xv[l].re, xv[l].im) : mk(R(0), R(0));
  };

  while (__any_sync(kFull, alive)) {
    const bool served = alive && !finished;
    const bool rk = served && phase < 4;
    const bool corr = served && phase == 4;
    // ---------------- coefficients c_k(t) of the RK stage; the corrector reuses the last stage's
    // (RK stages 2 and 3 share t + dt/2, and after an accepted step the next step starts at the t
    // of the last stage, whose coefficients are still in the buffers: evaluate only on a new t)
    if (rk && t0 != coef_t) {
      coef_eval<R, RL, W, KIND>(p, sm, hyp, t0, l);
      coef_t = t0;
    }
    // ---------------- one evaluate-and-solve per sub-warp (predictor: -H_t, corrector: H)
    write_track<R, RL, N>(sm, l, x);
    stash();
    __syncwarp(kFull);
    bool ill = false, sing = false;
    const cx<R> v = eval_solve<R, RL, N, W, KIND, S>(tb, sm, l, rk ? 1 : 0, p.cond_limit, ill, sing);
    unstash();
    if (kMixed && served && ill) step_ill = true;
    if (served && sing) step_sing = true;
    // ---------------- corrector norms (kernel_HC_Solver_P3P.cu:204-219), all lanes take part
    R ns0 = 0, nc0 = 0;
    if (__any_sync(kFull, corr)) {
      const cx<R> xn = c_sub(x, v);
      const R ns = tree_sum<R, N, W>((corr && l < N) ? c_abs2(v) : R(0));
      const R nc = tree_sum<R, N, W>((corr && l < N) ? c_abs2(xn) : R(0));
      ns0 = __shfl_sync(kFull, ns, leader);
      nc0 = __shfl_sync(kFull, nc, leader);
    }
    // ---------------- per-sub-warp state update (no synchronisation below until the fetch)
    bool end_step = false;
    if (rk) {
      if (phase < 3) {
        const R a = f_mul(dt, phase == 0 ? R(1.0 / 6.0) : R(2.0 / 6.0));
        const R d = f_mul(dt, phase == 2 ? R(1.0) : R(0.5));
        sols = mk(f_fma(v.re, a, sols.re), f_fma(v.im, a, sols.im));
        x = mk(f_fma(v.re, d, x0.re), f_fma(v.im, d, x0.im));
        if (phase != 1) t0 = f_add(t0, half);
        ++phase;
      } else {
        const R a = f_mul(dt, R(1.0 / 6.0));
        sols = mk(f_fma(v.re, a, sols.re), f_fma(v.im, a, sols.im));
        x = sols;
        phase = 4;
        cit = 0;
        success = false;
        inf = false;
        if (p.max_corr <= 0) end_step = true;
      }
    } else if (corr) {
      x = c_sub(x, v);
      ++ncorr;
      ++cit;
      success = ((double)ns0 < p.corr_tol2 * (double)nc0);
      inf = ((double)nc0 > 1e14);
      end_step = inf || success || cit >= p.max_corr || (cit == 1 && (double)ns0 > p.first_tol2 * (double)nc0);
    }
    bool done = alive && finished;
    if (end_step) {
      // step control (kernel_HC_Solver_P3P.cu:225-249)
      if (inf) {
        if (handover) {  // hand the last accepted point over
          x = x0;
          t0 = t_step;
        }
        done = true;
      } else if (!success) {
        dt = f_mul(dt, R(0.5));
        x = x0;
        sols = x0;
        nsucc = 0;
        t0 = t_step;
        ++nfail;
      } else {
        nfail = 0;
        ++nsucc;
        x0 = x;
        sols = x;
        if (nsucc >= p.incr) {
          nsucc = 0;
          dt = f_mul(dt, R(2));
          if ((double)dt > p.dt_max) dt = (R)p.dt_max;
        }
      }
      ++step;
      if (kMixed && (step_ill || (p.dt_floor > 0.0 && (double)dt < p.dt_floor))) ill_stop = true;
      last_sing = step_sing;
      if (!done) done = at_end();
      if (done && !inf && p.t_handover > 0.0 && f_sub(t_hand, t0) <= R(1e-6) && step <= p.max_steps &&
          dt < dt_pre)
        dt = dt_pre;
      if (!done) prologue();
    }

    // ---------------- finished paths: write out and take the next path
    // (a non-finite track anywhere in the sub-warp; every lane takes part in the vote)
    const unsigned bad = __ballot_sync(kFull, l < N && !(isfinite(x.re) && isfinite(x.im)));
    const bool nonfinite = ((W == 32 ? bad : bad >> leader) & (W == 32 ? kFull : ((1u << (W & 31)) - 1u))) != 0u;
    if (done && primary) {
      R* ep = reinterpret_cast<R*>(p.endpoints) + 2 * item * p.ld_out;
      if (l < N) {
        ep[2 * l] = x.re;
        ep[2 * l + 1] = x.im;
      }
      if (l == 0) {
        const bool conv = (t0 >= R(1) || f_sub(R(1), t0) <= R(1e-7));
        if (p.conv) p.conv[item] = conv ? 1 : 0;
        if (p.infy) p.infy[item] = inf ? 1 : 0;
        if (p.status)
          p.status[item] = conv        ? ST_CONVERGED
                           : inf       ? ST_DIVERGED
                           : nonfinite ? ST_NONFINITE
                           : last_sing ? ST_SINGULAR
                                       : ST_STEP_CAP;
        if (p.steps) p.steps[item] = step;
        if (p.corr) p.corr[item] = ncorr;
        // a path handed over at the boundary resumes at exactly t_handover, not at its float t
        // (a float t just short of the boundary would put the next step just short of the end
        // zone, where the edge clamp shrinks dt to the gap)
        const bool boundary = p.t_handover > 0.0 && !inf && f_sub(t_hand, t0) <= R(1e-6);
        if (p.t_end) p.t_end[item] = boundary ? p.t_handover : (double)t0;
        if (p.dt_end) p.dt_end[item] = (double)dt;
      }
    }
    long long nxt = 0;
    if (done && l == 0 && primary) nxt = n_sw + (long long)atomicAdd(reinterpret_cast<unsigned*>(p.counter), 1u);
    nxt = __shfl_sync(kFull, nxt, p.spread ? 0 : leader);
    if (done) {
      item = nxt;
      alive = item < p.n_items;
      if (alive) init_path(item);
    }
  }
}

template <typename R, typename RL, int N, int W, int KIND, int V, int S, int WK>
__global__ void __launch_bounds__(GHC_BLOCK(N, R, RL, V), GHC_MINB(N, R, RL, V)) track_kernel(const TrackParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  track_body<R, RL, N, W, KIND, S, WK>(p, smem, blockIdx.x, gridDim.x, false);
}

// -------------------------------------------------------------------------------------------------
// Newton polish at t = 1 and the residual |H(x,1)| (double); one sub-warp per item
// -------------------------------------------------------------------------------------------------
template <int N, int W, int KIND, int S>
__global__ void __launch_bounds__(128) polish_kernel(const PolishParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Tables tb = stage_tables(smem, p.hx_terms, p.hx_off, p.ht_terms, p.ht_off, N, p.n_hx_terms, p.n_ht_terms);
  const int lane = threadIdx.x & 31;
  const int l = lane % W;
  const int g = threadIdx.x / W;
  const int Mc = (KIND == KIND_P2C) ? p.M + 1 : p.P + 1;
  const int walk = (kFlatAlways<N> && p.flat_eval == 0) ? 1 : p.flat_eval;
  const bool flat = walk != 0;
  SubMem sm = sub_layout<double, double>(smem + tables_bytes(N, p.n_hx_terms, p.n_ht_terms) +
                                             (size_t)g * sub_bytes(N, Mc, W, flat ? p.scr_slots : 0, 16, 16),
                                         N, Mc, W, p.scr_slots, flat);
  sm.nz = row_mask<N>(tb.hx_off, l);
  sm.walk = walk;
  const int subs_per_cta = blockDim.x / W;
  const int leader = lane - l;
  for (long long item0 = (long long)blockIdx.x * subs_per_cta; item0 < p.n_items;
       item0 += (long long)gridDim.x * subs_per_cta) {
    const long long item = item0 + g;
    const bool valid = item < p.n_items;
    const bool conv = valid && p.conv[item];
    const long long hyp = valid ? item / p.paths_per_hyp : 0;
    double* ep = p.endpoints + 2 * (valid ? item : 0) * p.ld;
    cx<double> x = (valid && l < N) ? mk(ep[2 * l], ep[2 * l + 1]) : mk(0.0, 0.0);
    if (conv) {
      if (KIND == KIND_P2C) {
        coef_eval_p2c<double, double, W, false>(p.coef_hx + 2 * hyp * p.stride_hx, p.coef_ht + 2 * hyp * p.stride_ht,
                                                p.M, p.K, 1.0, view<double>(sm.coefA), view<double>(sm.coefB),
                                                nullptr, l);
      } else {
        coef_eval_ph<double, double, W, false>(p.p_start, p.p_tgt + 2 * hyp * p.stride_p,
                                               p.p_diff + 2 * hyp * p.stride_p, p.P, 1.0, view<double>(sm.coefA),
                                               view<double>(sm.coefB), nullptr, l);
      }
    }
    __syncwarp(kFull);
    for (int it = 0; it < p.iters; ++it) {
      write_track<double, double, N>(sm, l, x);
      __syncwarp(kFull);
      const cx<double> d = eval_solve<double, double, N, W, KIND, S>(tb, sm, l, 0);
      if (conv) x = c_sub(x, d);
    }
    // residual |H(x,1)|
    write_track<double, double, N>(sm, l, x);
    __syncwarp(kFull);
    cx<double> A[N];
    cx<double> h;
    eval_any<double, double, N, W, KIND, S>(tb, sm, l, A, h, 0);
    const double s = tree_sum<double, N, W>(l < N ? c_abs2(h) : 0.0);
    const double s0 = __shfl_sync(kFull, s, leader);
    if (valid) {
      if (conv && l < N) {
        ep[2 * l] = x.re;
        ep[2 * l + 1] = x.im;
      }
      if (l == 0 && p.resid) p.resid[item] = conv ? sqrt(s0) : -1.0;
    }
    __syncwarp(kFull);
  }
}

}  // namespace dev
}  // namespace ghc
