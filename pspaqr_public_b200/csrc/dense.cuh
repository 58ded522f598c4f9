// dense.cuh -- CTA-cooperative FP64 Householder building blocks for sm_100a.
//
// Every routine is called by all threads of one CTA (kThreads threads) and
// synchronises internally; matrices are column-major (element (i,j) at
// p[i + j*ld]) and may live in global or shared memory (generic pointers).
// Conventions follow LAPACK so results agree with the reference's LAPACK
// calls up to rounding:
//   * reflectors H = I - tau v v^T with v(0) = 1, beta = -sign(alpha)*||x||,
//     tau = (beta - alpha)/beta, v(1:) = x(1:)/(alpha - beta)  (dlarfg);
//   * a block of k reflectors is I - V T V^T with V unit lower trapezoidal and
//     T upper triangular (dlarft 'F','C'); the T here always spans all k
//     reflectors (one block), which is the same operator LAPACK's nb-blocked
//     T factors represent.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace spq {
namespace dev {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA-wide sum; `red` is a shared scratch of >= kWarps+1 doubles.
__device__ __forceinline__ double cta_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < kWarps ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[kWarps] = t;
  }
  __syncthreads();
  double r = red[kWarps];
  __syncthreads();
  return r;
}

// dlarfg on (alpha, x[0:len]) given sumsq = ||x||^2.  Returns tau, writes
// beta; the caller scales x by *scal (0 when tau == 0).
__device__ __forceinline__ double house(double alpha, double sumsq, double* beta, double* scal) {
  if (sumsq == 0.0) {
    *beta = alpha;
    *scal = 0.0;
    return 0.0;
  }
  double b = -copysign(hypot(alpha, sqrt(sumsq)), alpha);
  *beta = b;
  *scal = 1.0 / (alpha - b);
  return (b - alpha) / b;
}

// T factor (k x k, upper) from G(l,j) = v_l^T v_j stored in the strictly upper
// part of T on entry, and tau[0:k] (shared).  dlarft recurrence:
//   T(0:j, j) = -tau_j * T(0:j, 0:j) * G(0:j, j),  T(j,j) = tau_j.
__device__ void larft_from_gram(double* T, int ldt, int k, const double* tau, double* tmp /*smem >= k*/) {
  for (int j = 0; j < k; ++j) {
    for (int i = threadIdx.x; i < j; i += kThreads) tmp[i] = T[i + (size_t)j * ldt];
    __syncthreads();
    const double tj = tau[j];
    for (int i = threadIdx.x; i < j; i += kThreads) {
      double s = 0.0;
      for (int l = i; l < j; ++l) s += T[i + (size_t)l * ldt] * tmp[l];
      T[i + (size_t)j * ldt] = -tj * s;
    }
    if (threadIdx.x == 0) T[j + (size_t)j * ldt] = tj;
    __syncthreads();
  }
  // zero the strictly lower part
  for (int idx = threadIdx.x; idx < k * k; idx += kThreads) {
    int i = idx % k, j = idx / k;
    if (i > j) T[i + (size_t)j * ldt] = 0.0;
  }
  __syncthreads();
}

// Householder QR (m >= n assumed by callers; handles m < n too) of A (m x n).
// On exit R in the upper triangle, V below the diagonal, T (n x n) upper.
// tau: shared scratch >= n; red: shared >= kWarps+1; tmp: shared >= n.
__device__ void geqrt(double* A, int lda, int m, int n, double* T, int ldt, double* tau, double* red, double* tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kmax = m < n ? m : n;
  for (int j = 0; j < kmax; ++j) {
    double* aj = A + (size_t)j * lda;
    double s = 0.0;
    for (int i = j + 1 + threadIdx.x; i < m; i += kThreads) s += aj[i] * aj[i];
    s = cta_sum(s, red);
    const double alpha = aj[j];
    double beta, scal;
    const double tj = house(alpha, s, &beta, &scal);
    if (tj != 0.0)
      for (int i = j + 1 + threadIdx.x; i < m; i += kThreads) aj[i] *= scal;
    __syncthreads();
    if (threadIdx.x == 0) {
      aj[j] = beta;
      tau[j] = tj;
    }
    if (tj != 0.0) {
      for (int k = j + 1 + warp; k < n; k += kWarps) {
        double* ak = A + (size_t)k * lda;
        double d = lane == 0 ? ak[j] : 0.0;
        for (int i = j + 1 + lane; i < m; i += 32) d += aj[i] * ak[i];
        d = warp_sum(d) * tj;
        if (lane == 0) ak[j] -= d;
        for (int i = j + 1 + lane; i < m; i += 32) ak[i] -= aj[i] * d;
      }
    }
    __syncthreads();
  }
  for (int j = kmax; j < n; ++j)
    if (threadIdx.x == 0) tau[j] = 0.0;
  // Gram of the unit lower trapezoidal V: G(l,j) = A(j,l) + sum_{i>j} A(i,l) A(i,j)
  const int npairs = kmax * (kmax - 1) / 2;
  for (int p = warp; p < npairs; p += kWarps) {
    int j = (int)((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
    while (j * (j - 1) / 2 > p) --j;
    while ((j + 1) * j / 2 <= p) ++j;
    const int l = p - j * (j - 1) / 2;
    const double* al = A + (size_t)l * lda;
    const double* aj = A + (size_t)j * lda;
    double d = lane == 0 ? al[j] : 0.0;
    for (int i = j + 1 + lane; i < m; i += 32) d += al[i] * aj[i];
    d = warp_sum(d);
    if (lane == 0) T[l + (size_t)j * ldt] = d;
  }
  __syncthreads();
  larft_from_gram(T, ldt, kmax, tau, tmp);
  for (int idx = threadIdx.x; idx < n * n; idx += kThreads) {
    int i = idx % n, j = idx / n;
    if (i >= kmax || j >= kmax) T[i + (size_t)j * ldt] = 0.0;
  }
  __syncthreads();
}

// Triangular-pentagonal QR with l = 0 (dtpqrt): [R (n x n upper); B (m x n)].
// R's upper triangle and B are overwritten (B becomes the reflector tails);
// T (n x n) is the block factor of I - [I; B] T [I; B]^T.
__device__ void tpqrt(double* R, int ldr, double* B, int ldb, int m, int n, double* T, int ldt, double* tau,
                      double* red, double* tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < n; ++j) {
    double* bj = B + (size_t)j * ldb;
    double s = 0.0;
    for (int i = threadIdx.x; i < m; i += kThreads) s += bj[i] * bj[i];
    s = cta_sum(s, red);
    const double alpha = R[j + (size_t)j * ldr];
    double beta, scal;
    const double tj = house(alpha, s, &beta, &scal);
    if (tj != 0.0)
      for (int i = threadIdx.x; i < m; i += kThreads) bj[i] *= scal;
    __syncthreads();
    if (threadIdx.x == 0) {
      R[j + (size_t)j * ldr] = beta;
      tau[j] = tj;
    }
    if (tj != 0.0) {
      for (int k = j + 1 + warp; k < n; k += kWarps) {
        double* bk = B + (size_t)k * ldb;
        double* rjk = R + j + (size_t)k * ldr;
        double d = lane == 0 ? *rjk : 0.0;
        for (int i = lane; i < m; i += 32) d += bj[i] * bk[i];
        d = warp_sum(d) * tj;
        if (lane == 0) *rjk -= d;
        for (int i = lane; i < m; i += 32) bk[i] -= bj[i] * d;
      }
    }
    __syncthreads();
  }
  const int npairs = n * (n - 1) / 2;
  for (int p = warp; p < npairs; p += kWarps) {
    int j = (int)((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
    while (j * (j - 1) / 2 > p) --j;
    while ((j + 1) * j / 2 <= p) ++j;
    const int l = p - j * (j - 1) / 2;
    const double* bl = B + (size_t)l * ldb;
    const double* bj = B + (size_t)j * ldb;
    double d = 0.0;
    for (int i = lane; i < m; i += 32) d += bl[i] * bj[i];
    d = warp_sum(d);
    if (lane == 0) T[l + (size_t)j * ldt] = d;
  }
  __syncthreads();
  larft_from_gram(T, ldt, n, tau, tmp);
}

// C (m x nc) <- (I - V T V^T)^T C, V unit lower trapezoidal (m x k).
// W: shared scratch of 2*k*chunk doubles; chunk = columns per pass.
__device__ void apply_qt_left(const double* V, int ldv, const double* T, int ldt, int k, double* C, int ldc, int m,
                              int nc, double* W, int chunk) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (k <= 0 || nc <= 0 || m <= 0) return;
  double* W2 = W + (size_t)k * chunk;
  for (int c0 = 0; c0 < nc; c0 += chunk) {
    const int cn = (nc - c0) < chunk ? (nc - c0) : chunk;
    for (int p = warp; p < k * cn; p += kWarps) {
      const int i = p % k, c = p / k;
      const double* v = V + (size_t)i * ldv;
      const double* x = C + (size_t)(c0 + c) * ldc;
      double d = (lane == 0 && i < m) ? x[i] : 0.0;
      for (int r = i + 1 + lane; r < m; r += 32) d += v[r] * x[r];
      d = warp_sum(d);
      if (lane == 0) W[i + (size_t)c * k] = d;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k * cn; p += kThreads) {
      const int i = p % k, c = p / k;
      const double* t = T + (size_t)i * ldt;
      double s = 0.0;
      for (int l = 0; l <= i; ++l) s += t[l] * W[l + (size_t)c * k];
      W2[i + (size_t)c * k] = s;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < m * cn; p += kThreads) {
      const int r = p % m, c = p / m;
      const int lim = r < k ? r : k;
      double s = (r < k) ? W2[r + (size_t)c * k] : 0.0;
      for (int i = 0; i < lim; ++i) s += V[r + (size_t)i * ldv] * W2[i + (size_t)c * k];
      C[r + (size_t)(c0 + c) * ldc] -= s;
    }
    __syncthreads();
  }
}

// [A (k x nc); B (m x nc)] <- Q^T [A; B], Q = I - [I; V] T [I; V]^T, V full (m x k).
__device__ void apply_tpqt_left(const double* V, int ldv, const double* T, int ldt, int k, double* A, int lda,
                                double* B, int ldb, int m, int nc, double* W, int chunk) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (k <= 0 || nc <= 0) return;
  double* W2 = W + (size_t)k * chunk;
  for (int c0 = 0; c0 < nc; c0 += chunk) {
    const int cn = (nc - c0) < chunk ? (nc - c0) : chunk;
    for (int p = warp; p < k * cn; p += kWarps) {
      const int i = p % k, c = p / k;
      const double* v = V + (size_t)i * ldv;
      const double* x = B + (size_t)(c0 + c) * ldb;
      double d = lane == 0 ? A[i + (size_t)(c0 + c) * lda] : 0.0;
      for (int r = lane; r < m; r += 32) d += v[r] * x[r];
      d = warp_sum(d);
      if (lane == 0) W[i + (size_t)c * k] = d;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k * cn; p += kThreads) {
      const int i = p % k, c = p / k;
      const double* t = T + (size_t)i * ldt;
      double s = 0.0;
      for (int l = 0; l <= i; ++l) s += t[l] * W[l + (size_t)c * k];
      W2[i + (size_t)c * k] = s;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k * cn; p += kThreads) {
      const int i = p % k, c = p / k;
      A[i + (size_t)(c0 + c) * lda] -= W2[i + (size_t)c * k];
    }
    for (int p = threadIdx.x; p < m * cn; p += kThreads) {
      const int r = p % m, c = p / m;
      double s = 0.0;
      for (int i = 0; i < k; ++i) s += V[r + (size_t)i * ldv] * W2[i + (size_t)c * k];
      B[r + (size_t)(c0 + c) * ldb] -= s;
    }
    __syncthreads();
  }
}

// C (m x n) <- C (I - V T V^T), V unit lower trapezoidal (n x k).
__device__ void apply_q_right(const double* V, int ldv, const double* T, int ldt, int k, double* C, int ldc, int m,
                              int n, double* W, int chunk) {
  if (k <= 0 || m <= 0 || n <= 0) return;
  double* W2 = W + (size_t)k * chunk;
  for (int r0 = 0; r0 < m; r0 += chunk) {
    const int rn = (m - r0) < chunk ? (m - r0) : chunk;
    // W(r,i) = sum_{c>=i} C(r,c) V(c,i), V(i,i) = 1   (stored W[i + r*k])
    for (int p = threadIdx.x; p < k * rn; p += kThreads) {
      const int r = p % rn, i = p / rn;
      const double* v = V + (size_t)i * ldv;
      double s = C[(r0 + r) + (size_t)i * ldc];
      for (int c = i + 1; c < n; ++c) s += C[(r0 + r) + (size_t)c * ldc] * v[c];
      W[i + (size_t)r * k] = s;
    }
    __syncthreads();
    // W2(r,i) = sum_{l<=i} W(r,l) T(l,i)
    for (int p = threadIdx.x; p < k * rn; p += kThreads) {
      const int r = p % rn, i = p / rn;
      const double* t = T + (size_t)i * ldt;
      double s = 0.0;
      for (int l = 0; l <= i; ++l) s += W[l + (size_t)r * k] * t[l];
      W2[i + (size_t)r * k] = s;
    }
    __syncthreads();
    // C(r,c) -= sum_{i <= min(c,k-1)} W2(r,i) V(c,i)
    for (int p = threadIdx.x; p < rn * n; p += kThreads) {
      const int r = p % rn, c = p / rn;
      double s = (c < k) ? W2[c + (size_t)r * k] : 0.0;
      const int top = (c < k) ? c : k;
      for (int i = 0; i < top; ++i) s += W2[i + (size_t)r * k] * V[c + (size_t)i * ldv];
      C[(r0 + r) + (size_t)c * ldc] -= s;
    }
    __syncthreads();
  }
}

// C (m x n) <- C R^{-1}, R upper triangular (n x n).  One thread per row.
__device__ void trsm_right_upper(const double* R, int ldr, double* C, int ldc, int m, int n) {
  for (int r = threadIdx.x; r < m; r += kThreads) {
    for (int j = 0; j < n; ++j) {
      double s = C[r + (size_t)j * ldc];
      const double* rj = R + (size_t)j * ldr;
      for (int i = 0; i < j; ++i) s -= C[r + (size_t)i * ldc] * rj[i];
      C[r + (size_t)j * ldc] = s / rj[j];
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- vectors
// x (m) <- (I - V T V^T)^T x, V unit lower trapezoidal (m x k).  w: shared >= 2k.
__device__ void apply_qt_vec(const double* V, int ldv, const double* T, int ldt, int k, double* x, int m, double* w) {
  apply_qt_left(V, ldv, T, ldt, k, x, m, m, 1, w, 1);
}

// x (m) <- (I - V T V^T) x  (forward product applied without transpose).
__device__ void apply_q_vec(const double* V, int ldv, const double* T, int ldt, int k, double* x, int m, double* w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (k <= 0 || m <= 0) return;
  double* w2 = w + k;
  for (int i = warp; i < k; i += kWarps) {
    const double* v = V + (size_t)i * ldv;
    double d = (lane == 0 && i < m) ? x[i] : 0.0;
    for (int r = i + 1 + lane; r < m; r += 32) d += v[r] * x[r];
    d = warp_sum(d);
    if (lane == 0) w[i] = d;
  }
  __syncthreads();
  // w2 = T w  (T upper: w2(i) = sum_{l>=i} T(i,l) w(l))
  for (int i = threadIdx.x; i < k; i += kThreads) {
    double s = 0.0;
    for (int l = i; l < k; ++l) s += T[i + (size_t)l * ldt] * w[l];
    w2[i] = s;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < m; r += kThreads) {
    const int top = r < k ? r : k;
    double s = (r < k) ? w2[r] : 0.0;
    for (int i = 0; i < top; ++i) s += V[r + (size_t)i * ldv] * w2[i];
    x[r] -= s;
  }
  __syncthreads();
}

// Upper triangular solve x <- R^{-1} x (n x n), blocked by 32: one warp solves
// each diagonal block with shuffles, the CTA updates the rows above.
__device__ void trsv_upper(const double* R, int ldr, double* x, int n, double* xs /*shared >= 32*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int hi = n; hi > 0; hi -= 32) {
    const int lo = hi > 32 ? hi - 32 : 0;
    const int bs = hi - lo;
    if (warp == 0) {
      double xv = lane < bs ? x[lo + lane] : 0.0;
      for (int j = bs - 1; j >= 0; --j) {
        if (lane == j) xv = xv / R[(lo + j) + (size_t)(lo + j) * ldr];
        const double xj = __shfl_sync(0xffffffffu, xv, j);
        if (lane < j) xv -= R[(lo + lane) + (size_t)(lo + j) * ldr] * xj;
      }
      if (lane < bs) {
        x[lo + lane] = xv;
        xs[lane] = xv;
      }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < lo; r += kThreads) {
      double s = 0.0;
      for (int j = 0; j < bs; ++j) s += R[r + (size_t)(lo + j) * ldr] * xs[j];
      x[r] -= s;
    }
    __syncthreads();
  }
}

}  // namespace dev
}  // namespace spq
