// p2c.cu -- per-hypothesis coefficient homotopy tables on the device, and the
// small layout kernels of the drop-in wrappers.
//
// For every hypothesis h and coefficient k (one thread each):
//   c_k(t) = sum_terms coef * prod_j (q_j + t (p_j - q_j))     expanded in t
//   Hx[h][k][e] = coefficient of t^e, Ht[h][k][e] = (e+1) Hx[h][k][e+1]
// plus the constant-1 sentinel k = M (reference createUnivPoly4Coeffs.m:227, :333),
// the same tables the reference builds on the host per problem in
// GPU-HC/magmaHC/PHC_Coeffs/p2c-<problem>.h.
#include <cuda_runtime.h>

#include "ghc_internal.h"

namespace ghc {
namespace {

constexpr int kMaxK = 8;

__global__ void p2c_kernel(const P2CParams p) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Mc = p.M + 1;
  if (gid >= p.n_hyp * Mc) return;
  const long long h = gid / Mc;
  const int k = (int)(gid % Mc);
  const int K = p.K;
  const double* q = p.p_start;
  const double* tg = p.p_tgt + 2 * h * (p.P + 1);
  double ar[kMaxK + 1], ai[kMaxK + 1];
#pragma unroll
  for (int e = 0; e <= kMaxK; ++e) ar[e] = ai[e] = 0.0;
  if (k == p.M) {
    ar[0] = 1.0;
  } else {
    for (int ti = p.k_off[k]; ti < p.k_off[k + 1]; ++ti) {
      double pr[kMaxK + 1], pi[kMaxK + 1];
#pragma unroll
      for (int e = 0; e <= kMaxK; ++e) pr[e] = pi[e] = 0.0;
      pr[0] = p.term_coef[ti];
      int deg = 0;
      for (int f = p.term_fac_off[ti]; f < p.term_fac_off[ti + 1]; ++f) {
        const int j = p.term_fac[f];
        const double qr = q[2 * j], qi = q[2 * j + 1];
        const double dr = tg[2 * j] - qr, di = tg[2 * j + 1] - qi;
        // multiply by (q + t d), highest power first so it can be done in place
        for (int e = deg + 1; e >= 0; --e) {
          double nr = 0.0, ni = 0.0;
          if (e <= deg) {
            nr += pr[e] * qr - pi[e] * qi;
            ni += pr[e] * qi + pi[e] * qr;
          }
          if (e >= 1) {
            nr += pr[e - 1] * dr - pi[e - 1] * di;
            ni += pr[e - 1] * di + pi[e - 1] * dr;
          }
          pr[e] = nr;
          pi[e] = ni;
        }
        ++deg;
      }
      for (int e = 0; e <= K; ++e) {
        ar[e] += pr[e];
        ai[e] += pi[e];
      }
    }
  }
  double* hx = p.coef_hx + 2 * (h * Mc * (K + 1) + (long long)k * (K + 1));
  for (int e = 0; e <= K; ++e) {
    hx[2 * e] = ar[e];
    hx[2 * e + 1] = ai[e];
  }
  double* ht = p.coef_ht + 2 * (h * Mc * K + (long long)k * K);
  for (int e = 0; e < K; ++e) {
    double r = (e + 1) * ar[e + 1], i = (e + 1) * ai[e + 1];
    if (k == p.M) {
      r = (e == 0 && !p.exact_ht) ? 1.0 : 0.0;
      i = 0.0;
    }
    ht[2 * e] = r;
    ht[2 * e + 1] = i;
  }
}

__global__ void f2d_kernel(const float* __restrict__ s, double* __restrict__ d, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = (double)s[i];
}

template <typename T>
__global__ void debug_kernel(const uint8_t* conv, const double* t_end, const double* dt_end, T* dbg, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dbg[2 * i] = conv[i] ? T(1) : (T)t_end[i];
  dbg[2 * i + 1] = conv[i] ? T(0) : (T)dt_end[i];
}

template <typename T>
__global__ void diff_kernel(const T* s, const T* t, double* d, long long n_hyp, int P1) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_hyp * P1) return;
  const int k = (int)(i % P1);
  d[2 * i] = (double)t[2 * i] - (double)s[2 * k];
  d[2 * i + 1] = (double)t[2 * i + 1] - (double)s[2 * k + 1];
}

}  // namespace

int launch_p2c(const P2CParams& p, void* stream) {
  if (p.K > kMaxK) return -10;
  const long long n = p.n_hyp * (p.M + 1);
  if (n <= 0) return 0;
  const int block = 128;
  const long long grid = (n + block - 1) / block;
  p2c_kernel<<<(unsigned)grid, block, 0, (cudaStream_t)stream>>>(p);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

int launch_f2d(const float* s, double* d, long long n, void* stream) {
  if (n <= 0) return 0;
  f2d_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, (cudaStream_t)stream>>>(s, d, n);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

int launch_debug_f(const uint8_t* conv, const double* t, const double* dt, float* dbg, long long n, void* stream) {
  if (n <= 0) return 0;
  debug_kernel<float><<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(conv, t, dt, dbg, n);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

int launch_debug_d(const uint8_t* conv, const double* t, const double* dt, double* dbg, long long n, void* stream) {
  if (n <= 0) return 0;
  debug_kernel<double><<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(conv, t, dt, dbg, n);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

int launch_diff_d(const double* s, const double* t, double* d, long long n_hyp, int P1, void* stream) {
  if (n_hyp * P1 <= 0) return 0;
  diff_kernel<double><<<(unsigned)((n_hyp * P1 + 127) / 128), 128, 0, (cudaStream_t)stream>>>(s, t, d, n_hyp, P1);
  return cudaGetLastError() == cudaSuccess ? 0 : -23;
}

}  // namespace ghc
