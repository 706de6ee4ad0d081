/*
 * Stand-in for MAGMA's magma_v2.h, just enough for the reference's generated
 * P2C coefficient builders (GPU-HC/magmaHC/PHC_Coeffs/p2c-*.h) and its
 * evaluator templates (GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-*.cuh) to
 * compile on the host.  TEST INFRASTRUCTURE ONLY (oracle/_ref).  The complex scalar type
 * is chosen with REF_REAL (double by default) so the reference's coefficient
 * expressions can be evaluated in the tracker's precision.
 */
#ifndef ORACLE_REF_SHIM_MAGMA_V2_H
#define ORACLE_REF_SHIM_MAGMA_V2_H
#include <type_traits>
#ifndef REF_REAL
#define REF_REAL double
#endif
/* one type name per precision, so the double and float builds can share a library */
#ifndef ref_cx
#define ref_cx ref_cx_double
#endif
struct ref_cx {
  REF_REAL x, y;
  ref_cx() : x(0), y(0) {}
  ref_cx(REF_REAL a, REF_REAL b) : x(a), y(b) {}
};
inline ref_cx operator+(ref_cx a, ref_cx b) { return ref_cx(a.x + b.x, a.y + b.y); }
inline ref_cx operator-(ref_cx a, ref_cx b) { return ref_cx(a.x - b.x, a.y - b.y); }
inline ref_cx operator-(ref_cx a) { return ref_cx(-a.x, -a.y); }
inline ref_cx operator*(ref_cx a, ref_cx b) { return ref_cx(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator*(S s, ref_cx a) { return ref_cx((REF_REAL)s * a.x, (REF_REAL)s * a.y); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator*(ref_cx a, S s) { return ref_cx((REF_REAL)s * a.x, (REF_REAL)s * a.y); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator+(S s, ref_cx a) { return ref_cx((REF_REAL)s + a.x, a.y); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator+(ref_cx a, S s) { return ref_cx(a.x + (REF_REAL)s, a.y); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator-(S s, ref_cx a) { return ref_cx((REF_REAL)s - a.x, -a.y); }
template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
inline ref_cx operator-(ref_cx a, S s) { return ref_cx(a.x - (REF_REAL)s, a.y); }
inline ref_cx& operator+=(ref_cx& a, ref_cx b) { a.x += b.x; a.y += b.y; return a; }
inline ref_cx& operator-=(ref_cx& a, ref_cx b) { a.x -= b.x; a.y -= b.y; return a; }
typedef ref_cx magmaFloatComplex;
#define MAGMA_C_MAKE(a, b) ref_cx((REF_REAL)(a), (REF_REAL)(b))
#define MAGMA_C_ONE ref_cx(1, 0)
#define MAGMA_C_ZERO ref_cx(0, 0)
#endif
