// dense.cuh -- CTA-cooperative FP64 Householder building blocks for sm_100a.
//
// Matrices are column-major (element (i,j) at p[i + j*ld]).  Conventions
// follow LAPACK so results agree with the reference's LAPACK calls up to
// rounding:
//   * reflectors H = I - tau v v^T with v(0) = 1, beta = -sign(alpha)*||x||,
//     tau = (beta - alpha)/beta, v(1:) = x(1:)/(alpha - beta)  (dlarfg);
//   * k reflectors form I - V T V^T with V unit lower trapezoidal; T is kept
//     in LAPACK's blocked layout with panel width kNB (dgeqrt/dtpqrt with
//     nb = 32): an kNB x k array, columns [p*kNB, p*kNB+kb) holding the kb x kb
//     upper-triangular T of panel p.  Q = Q_0 Q_1 ... Q_{P-1} over panels.
// Apply routines are called by all threads of one CTA and synchronise
// internally; factorization routines in kernels.cu distribute panels over
// the CTAs of a thread-block cluster.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace spq {
namespace dev {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kNB = 32;  // panel width of the blocked reflector storage

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA-wide sum; `red` is a shared scratch of >= kWarps+1 doubles.
template <typename T>
__device__ __forceinline__ T cta_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    T t = lane < kWarps ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[kWarps] = t;
  }
  __syncthreads();
  T r = red[kWarps];
  __syncthreads();
  return r;
}

// dlarfg on (alpha, x) given sumsq = ||x||^2.  Returns tau, writes beta and
// the scale the caller applies to x (0 when tau == 0).
template <typename T>
__device__ __forceinline__ T house(T alpha, T sumsq, T* beta, T* scal) {
  if (sumsq == 0.0) {
    *beta = alpha;
    *scal = 0.0;
    return 0.0;
  }
  T b = -copysign(hypot(alpha, sqrt(sumsq)), alpha);
  *beta = b;
  *scal = 1.0 / (alpha - b);
  return (b - alpha) / b;
}

// T (kb x kb, ld ldt) from G(l,j) = v_l^T v_j in its strictly upper part on
// entry and tau[0:kb].  dlarft recurrence T(0:j,j) = -tau_j T(0:j,0:j) G(0:j,j).
template <typename T>
__device__ void larft_from_gram(T* Tm, int ldt, int kb, const T* tau, T* tmp /*>= kb*/) {
  for (int j = 0; j < kb; ++j) {
    for (int i = threadIdx.x; i < j; i += kThreads) tmp[i] = Tm[i + (size_t)j * ldt];
    __syncthreads();
    const T tj = tau[j];
    for (int i = threadIdx.x; i < j; i += kThreads) {
      T s = 0.0;
      for (int l = i; l < j; ++l) s += Tm[i + (size_t)l * ldt] * tmp[l];
      Tm[i + (size_t)j * ldt] = -tj * s;
    }
    if (threadIdx.x == 0) Tm[j + (size_t)j * ldt] = tj;
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kb * kb; idx += kThreads) {
    const int i = idx % kb, j = idx / kb;
    if (i > j) Tm[i + (size_t)j * ldt] = 0.0;
  }
  __syncthreads();
}

// Pair index p -> (l, j), l < j, p = j(j-1)/2 + l.
__device__ __forceinline__ void pair_of(int p, int* l, int* j) {
  int jj = (int)((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
  while (jj * (jj - 1) / 2 > p) --jj;
  while ((jj + 1) * jj / 2 <= p) ++jj;
  *j = jj;
  *l = p - jj * (jj - 1) / 2;
}

// Panel T of kb reflectors stored unit-lower-trapezoidal in V (m x kb, rows
// from the panel's diagonal).  unit = 1: V(i,i) = 1 implied (geqrt / RRQR);
// unit = 0: full tails of a pentagonal panel (tpqrt, identity on top).
template <typename T>
__device__ void panel_t(const T* V, int ldv, int m, int kb, int unit, const T* tau, T* Tm, int ldt,
                        T* tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int npairs = kb * (kb - 1) / 2;
  for (int p = warp; p < npairs; p += kWarps) {
    int l, j;
    pair_of(p, &l, &j);
    const T* vl = V + (size_t)l * ldv;
    const T* vj = V + (size_t)j * ldv;
    T d = 0.0;
    if (unit) {
      d = lane == 0 ? vl[j] : 0.0;
      for (int i = j + 1 + lane; i < m; i += 32) d += vl[i] * vj[i];
    } else {
      for (int i = lane; i < m; i += 32) d += vl[i] * vj[i];
    }
    d = warp_sum(d);
    if (lane == 0) Tm[l + (size_t)j * ldt] = d;
  }
  __syncthreads();
  larft_from_gram(Tm, ldt, kb, tau, tmp);
}

// panel_t for a panel in shared memory, with T built by one warp: the Gram
// V^T V of the panel's reflectors goes to sG (kNB x (kNB + 1), shared), then
// lane i holds row i of T in registers and forms column j as
//   T(i, j) = -tau_j sum_{l=i}^{j-1} T(i, l) G(l, j),  T(j, j) = tau_j,
// the sums of larft_from_gram in the same order, without its two barriers
// and global round trips per column.  Tm is written by warp 0; the caller
// synchronises before T is read.
template <typename T>
__device__ void panel_t_warp(const T* V, int ldv, int m, int kb, int unit, const T* tau, T* Tm, int ldt, T* sG) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kLG = kNB + 1;
  const int npairs = kb * (kb - 1) / 2;
  for (int p = warp; p < npairs; p += kWarps) {
    int l, j;
    pair_of(p, &l, &j);
    const T* vl = V + (size_t)l * ldv;
    const T* vj = V + (size_t)j * ldv;
    T d = 0.0;
    if (unit) {
      d = lane == 0 ? vl[j] : 0.0;
      for (int i = j + 1 + lane; i < m; i += 32) d += vl[i] * vj[i];
    } else {
      for (int i = lane; i < m; i += 32) d += vl[i] * vj[i];
    }
    d = warp_sum(d);
    if (lane == 0) sG[l * kLG + j] = d;
  }
  __syncthreads();
  if (warp == 0) {
    T t[kNB];
#pragma unroll
    for (int j = 0; j < kNB; ++j) t[j] = 0.0;
#pragma unroll
    for (int j = 0; j < kNB; ++j) {
      if (j < kb) {
        T s = 0.0;
#pragma unroll
        for (int l = 0; l < kNB; ++l)
          if (l < j && l >= lane) s += t[l] * sG[l * kLG + j];
        const T tj = tau[j];
        t[j] = lane < j ? -tj * s : (lane == j ? tj : (T)0.0);
      }
    }
    if (lane < kb)
#pragma unroll
      for (int j = 0; j < kNB; ++j)
        if (j < kb) Tm[lane + (size_t)j * ldt] = t[j];
  }
}

// ---------------------------------------------------------------- applies
// C (m x nc) <- (I - V T V^T)^T C for one block of k <= kNB reflectors,
// V unit lower trapezoidal (m x k), T (k x k, ld ldt).  W: 2*k*nc doubles.
template <typename T>
__device__ void block_qt(const T* V, int ldv, const T* Tm, int ldt, int k, T* C, int ldc, int m, int nc,
                         T* W) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* W2 = W + (size_t)k * nc;
  for (int p = warp; p < k * nc; p += kWarps) {
    const int i = p % k, c = p / k;
    const T* v = V + (size_t)i * ldv;
    const T* x = C + (size_t)c * ldc;
    T d = (lane == 0 && i < m) ? x[i] : 0.0;
    for (int r = i + 1 + lane; r < m; r += 32) d += v[r] * x[r];
    d = warp_sum(d);
    if (lane == 0) W[i + (size_t)c * k] = d;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < k * nc; p += kThreads) {
    const int i = p % k, c = p / k;
    const T* t = Tm + (size_t)i * ldt;
    T s = 0.0;
    for (int l = 0; l <= i; ++l) s += t[l] * W[l + (size_t)c * k];
    W2[i + (size_t)c * k] = s;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < m * nc; p += kThreads) {
    const int r = p % m, c = p / m;
    const int lim = r < k ? r : k;
    T s = (r < k) ? W2[r + (size_t)c * k] : 0.0;
    for (int i = 0; i < lim; ++i) s += V[r + (size_t)i * ldv] * W2[i + (size_t)c * k];
    C[r + (size_t)c * ldc] -= s;
  }
  __syncthreads();
}

// C (m x nc) <- (I - V T V^T) C for one block (no transpose).
template <typename T>
__device__ void block_q(const T* V, int ldv, const T* Tm, int ldt, int k, T* C, int ldc, int m, int nc,
                        T* W) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* W2 = W + (size_t)k * nc;
  for (int p = warp; p < k * nc; p += kWarps) {
    const int i = p % k, c = p / k;
    const T* v = V + (size_t)i * ldv;
    const T* x = C + (size_t)c * ldc;
    T d = (lane == 0 && i < m) ? x[i] : 0.0;
    for (int r = i + 1 + lane; r < m; r += 32) d += v[r] * x[r];
    d = warp_sum(d);
    if (lane == 0) W[i + (size_t)c * k] = d;
  }
  __syncthreads();
  // W2 = T W  (T upper: W2(i) = sum_{l>=i} T(i,l) W(l))
  for (int p = threadIdx.x; p < k * nc; p += kThreads) {
    const int i = p % k, c = p / k;
    T s = 0.0;
    for (int l = i; l < k; ++l) s += Tm[i + (size_t)l * ldt] * W[l + (size_t)c * k];
    W2[i + (size_t)c * k] = s;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < m * nc; p += kThreads) {
    const int r = p % m, c = p / m;
    const int lim = r < k ? r : k;
    T s = (r < k) ? W2[r + (size_t)c * k] : 0.0;
    for (int i = 0; i < lim; ++i) s += V[r + (size_t)i * ldv] * W2[i + (size_t)c * k];
    C[r + (size_t)c * ldc] -= s;
  }
  __syncthreads();
}

// [A (k x nc, rows of the panel); B (m x nc)] <- Q^T [A; B] for one pentagonal
// block, Q = I - [I; V] T [I; V]^T with V full (m x k).
template <typename T>
__device__ void block_tpqt(const T* V, int ldv, const T* Tm, int ldt, int k, T* A, int lda, T* B,
                           int ldb, int m, int nc, T* W) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* W2 = W + (size_t)k * nc;
  for (int p = warp; p < k * nc; p += kWarps) {
    const int i = p % k, c = p / k;
    const T* v = V + (size_t)i * ldv;
    const T* x = B + (size_t)c * ldb;
    T d = lane == 0 ? A[i + (size_t)c * lda] : 0.0;
    for (int r = lane; r < m; r += 32) d += v[r] * x[r];
    d = warp_sum(d);
    if (lane == 0) W[i + (size_t)c * k] = d;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < k * nc; p += kThreads) {
    const int i = p % k, c = p / k;
    const T* t = Tm + (size_t)i * ldt;
    T s = 0.0;
    for (int l = 0; l <= i; ++l) s += t[l] * W[l + (size_t)c * k];
    W2[i + (size_t)c * k] = s;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < k * nc; p += kThreads) {
    const int i = p % k, c = p / k;
    A[i + (size_t)c * lda] -= W2[i + (size_t)c * k];
  }
  for (int p = threadIdx.x; p < m * nc; p += kThreads) {
    const int r = p % m, c = p / m;
    T s = 0.0;
    for (int i = 0; i < k; ++i) s += V[r + (size_t)i * ldv] * W2[i + (size_t)c * k];
    B[r + (size_t)c * ldb] -= s;
  }
  __syncthreads();
}

// C (m x n) <- C (I - V T V^T) for one block, V unit lower trapezoidal (n x k).
// W: 2*k*m doubles.
template <typename T>
__device__ void block_q_right(const T* V, int ldv, const T* Tm, int ldt, int k, T* C, int ldc, int m,
                              int n, T* W) {
  T* W2 = W + (size_t)k * m;
  for (int p = threadIdx.x; p < k * m; p += kThreads) {
    const int r = p % m, i = p / m;
    const T* v = V + (size_t)i * ldv;
    T s = C[r + (size_t)i * ldc];
    for (int c = i + 1; c < n; ++c) s += C[r + (size_t)c * ldc] * v[c];
    W[i + (size_t)r * k] = s;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < k * m; p += kThreads) {
    const int r = p % m, i = p / m;
    const T* t = Tm + (size_t)i * ldt;
    T s = 0.0;
    for (int l = 0; l <= i; ++l) s += W[l + (size_t)r * k] * t[l];
    W2[i + (size_t)r * k] = s;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < m * n; p += kThreads) {
    const int r = p % m, c = p / m;
    T s = (c < k) ? W2[c + (size_t)r * k] : 0.0;
    const int top = (c < k) ? c : k;
    for (int i = 0; i < top; ++i) s += W2[i + (size_t)r * k] * V[c + (size_t)i * ldv];
    C[r + (size_t)c * ldc] -= s;
  }
  __syncthreads();
}

// Panel-blocked applies over k reflectors (T in kNB x k layout).
// Q^T C: panels in order; each acts on rows [j0, m).
template <typename T>
__device__ void apply_qt(const T* V, int ldv, const T* Tm, int k, T* C, int ldc, int m, int nc,
                         T* W, int wcap) {
  if (k <= 0 || nc <= 0 || m <= 0) return;
  const int cmax = (wcap / (2 * kNB)) > 0 ? (wcap / (2 * kNB)) : 1;
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int c0 = 0; c0 < nc; c0 += cmax) {
      const int cn = (nc - c0) < cmax ? (nc - c0) : cmax;
      block_qt(V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, C + j0 + (size_t)c0 * ldc, ldc, m - j0,
               cn, W);
    }
  }
}
// Q C: panels in reverse order.
template <typename T>
__device__ void apply_q(const T* V, int ldv, const T* Tm, int k, T* C, int ldc, int m, int nc, T* W,
                        int wcap) {
  if (k <= 0 || nc <= 0 || m <= 0) return;
  const int cmax = (wcap / (2 * kNB)) > 0 ? (wcap / (2 * kNB)) : 1;
  const int np = (k + kNB - 1) / kNB;
  for (int p = np - 1; p >= 0; --p) {
    const int j0 = p * kNB;
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int c0 = 0; c0 < nc; c0 += cmax) {
      const int cn = (nc - c0) < cmax ? (nc - c0) : cmax;
      block_q(V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, C + j0 + (size_t)c0 * ldc, ldc, m - j0,
              cn, W);
    }
  }
}
// [A (k x nc); B (m x nc)] <- Q^T [A; B] for a pentagonal (tpqrt) factor.
template <typename T>
__device__ void apply_tpqt(const T* V, int ldv, const T* Tm, int k, T* A, int lda, T* B, int ldb,
                           int m, int nc, T* W, int wcap) {
  if (k <= 0 || nc <= 0) return;
  const int cmax = (wcap / (2 * kNB)) > 0 ? (wcap / (2 * kNB)) : 1;
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int c0 = 0; c0 < nc; c0 += cmax) {
      const int cn = (nc - c0) < cmax ? (nc - c0) : cmax;
      block_tpqt(V + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, A + j0 + (size_t)c0 * lda, lda,
                 B + (size_t)c0 * ldb, ldb, m, cn, W);
    }
  }
}
// C (m x n) <- C Q, panels in order; each acts on columns [j0, n).
template <typename T>
__device__ void apply_q_right(const T* V, int ldv, const T* Tm, int k, T* C, int ldc, int m, int n,
                              T* W, int wcap) {
  if (k <= 0 || m <= 0 || n <= 0) return;
  const int rmax = (wcap / (2 * kNB)) > 0 ? (wcap / (2 * kNB)) : 1;
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int r0 = 0; r0 < m; r0 += rmax) {
      const int rn = (m - r0) < rmax ? (m - r0) : rmax;
      block_q_right(V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, C + r0 + (size_t)j0 * ldc, ldc, rn,
                    n - j0, W);
    }
  }
}


// ---------------------------------------------------------------- tiled matrix applies
// Register-tiled block reflector applies on matrices: rows are streamed
// through shared memory in tiles of kRT; the left apply keeps two tiles in
// flight (the next tile's global loads are issued before the current tile's
// products).  `sm` holds kTileSmem elements (2 kTileSmem for T = float).
constexpr int kNC = 64;   // columns (rows for right applies) per pass
constexpr int kRT = 32;   // rows (columns) per shared-memory tile
// Row strides of the V and C tiles of the left apply: 16-byte aligned rows
// whose starts fall on distinct 16-byte bank groups for 8 consecutive rows.
template <typename T>
__host__ __device__ constexpr int tile_lv() { return kNB + (sizeof(T) == 4 ? 4 : 2); }
template <typename T>
__host__ __device__ constexpr int tile_lc() { return kNC + (sizeof(T) == 4 ? 4 : 2); }
constexpr int kTileSmem = 2 * kRT * tile_lv<float>() + 2 * kRT * tile_lc<float>() + kNB * kNC;

// Load through L2 (kCg: data written by another CTA of the cluster) or as is.
template <bool kCg, typename T>
__device__ __forceinline__ T ld_v(const T* p) {
  if (kCg) return __ldcg(p);
  return *p;
}

// C (m x nc <= kNC) <- Q^T C with one panel: unit = 1: V unit lower trapezoidal
// (geqrt / RRQR reflectors), A unused; unit = 0: pentagonal tpqrt panel,
// [A (kb x nc); C] <- Q^T [A; C] with V full (m x kb).  Column c of A and C
// is column c + (c / kNB) * cgap of the arrays (cgap > 0: the column panels
// a CTA owns in a cluster-distributed factorization).  kCg: V and T are read
// through L2.
template <typename T, bool kCg = false>
__device__ void tile_left_qt(const T* V, int ldv, const T* Tm, int ldt, int kb, int unit, T* A, int lda,
                             T* C, int ldc, int m, int nc, T* sm, int cgap = 0) {
  static_assert(kThreads == 256 && kNB == 32 && kNC == 64 && kRT == 32, "tile shapes");
  constexpr int kLV = tile_lv<T>(), kLC = tile_lc<T>();
  // FP32 callers pass 2 kTileSmem elements (kTileSmem doubles): the partial
  // sums and W2 then go past the tile buffers
  constexpr bool kKeep = sizeof(T) == 4;
  static_assert(!kKeep || 3 * kNB * kNC + kNB * kNC <= kTileSmem, "FP32 park and W2 areas");
  constexpr int kVS = kRT * kLV, kCS = kRT * kLC;
  T* sV0 = sm;               // two [kRT][kLV] tiles of V
  T* sC0 = sV0 + 2 * kVS;    // two [kRT][kLC] tiles of C
  T* sW = sC0 + 2 * kCS;     // [kNB][kNC]: W, then the partial sums' landing area is sV0..sC0
  const int t = threadIdx.x;
  auto col = [&](int c) { return (size_t)(c + (c / kNB) * cgap); };
  // global loads of one tile: lane = row (a warp reads 32 consecutive rows of
  // one column: coalesced), warp w = columns kSV w .. (V) and kSC w .. (C), so
  // that a thread stashes one row segment with 16-byte stores
  constexpr int kSV = kRT * kNB / kThreads, kSC = kRT * kNC / kThreads;
  const int lr = t & (kRT - 1), lw = t / kRT;
  T rv[kSV], rc[kSC];
  auto vload = [&](int r0) {
    const int gr = r0 + lr;
#pragma unroll
    for (int q = 0; q < kSV; ++q) {
      const int i = lw * kSV + q;
      T v = 0.0;
      if (gr < m && i < kb)
        v = unit ? (gr == i ? (T)1.0 : (gr < i ? (T)0.0 : ld_v<kCg>(V + gr + (size_t)i * ldv)))
                 : ld_v<kCg>(V + gr + (size_t)i * ldv);
      rv[q] = v;
    }
  };
  auto vstash = [&](int b) {
    T* d = sV0 + b * kVS + lr * kLV + lw * kSV;
#pragma unroll
    for (int q = 0; q < kSV; ++q) d[q] = rv[q];
  };
  auto cload = [&](int r0) {
    const int gr = r0 + lr;
#pragma unroll
    for (int q = 0; q < kSC; ++q) {
      const int c = lw * kSC + q;
      rc[q] = (gr < m && c < nc) ? C[gr + col(c) * ldc] : (T)0.0;
    }
  };
  auto cstash = [&](int b) {
    T* d = sC0 + b * kCS + lr * kLC + lw * kSC;
#pragma unroll
    for (int q = 0; q < kSC; ++q) d[q] = rc[q];
  };
  const int ntile = (m + kRT - 1) / kRT;
  // T (and the top block A of a pentagonal panel) are read now, used after
  // the products: element idx = t + kThreads q, T(l = idx & 31, i = idx >> 5)
  // and A(i = idx & 31, c = idx >> 5)
  constexpr int kST = kNB * kNB / kThreads, kSA = kNB * kNC / kThreads;
  T rt[kST], ra[kSA];
#pragma unroll
  for (int q = 0; q < kST; ++q) {
    const int idx = t + q * kThreads, l = idx & (kNB - 1), i = idx / kNB;
    rt[q] = (l <= i && i < kb) ? ld_v<kCg>(Tm + l + (size_t)i * ldt) : (T)0.0;
  }
#pragma unroll
  for (int q = 0; q < kSA; ++q) {
    const int idx = t + q * kThreads, i = idx & (kNB - 1), c = idx / kNB;
    ra[q] = (!unit && i < kb && c < nc) ? A[i + col(c) * lda] : (T)0.0;
  }
  // ---- W = V^T C.  A thread accumulates W(i0:i0+kIW, c0:c0+4); the kSets
  // row sets of kTPO threads each take kRows consecutive rows of every tile
  {
    constexpr int kIW = sizeof(T) == 4 ? 8 : 4;           // reflectors per thread
    constexpr int kTPO = (kNB / kIW) * (kNC / 4);          // threads per set
    constexpr int kSets = kThreads / kTPO, kRows = kRT / kSets;
    const int set = t / kTPO, i0 = ((t % kTPO) / (kNC / 4)) * kIW, c0 = (t % (kNC / 4)) * 4;
    T acc[kIW][4];
#pragma unroll
    for (int a = 0; a < kIW; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    vload(0);
    cload(0);
    vstash(0);
    cstash(0);
    __syncthreads();
    for (int tt = 0; tt < ntile; ++tt) {
      const int b = tt & 1;
      const bool more = tt + 1 < ntile;
      if (more) {
        vload((tt + 1) * kRT);
        cload((tt + 1) * kRT);
      }
      const T* sV = sV0 + b * kVS + (set * kRows) * kLV + i0;
      const T* sC = sC0 + b * kCS + (set * kRows) * kLC + c0;
#pragma unroll 8
      for (int r = 0; r < kRows; ++r) {
        T v[kIW], c[4];
#pragma unroll
        for (int a = 0; a < kIW; ++a) v[a] = sV[r * kLV + a];
#pragma unroll
        for (int q = 0; q < 4; ++q) c[q] = sC[r * kLC + q];
#pragma unroll
        for (int a = 0; a < kIW; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[a][q] += v[a] * c[q];
      }
      if (more) {
        vstash(b ^ 1);
        cstash(b ^ 1);
      }
      __syncthreads();
    }
    // sets 1.. park their partial sums in the tile buffers (FP32: past them,
    // so that a single tile stays staged for the update), set 0 adds them in
    // set order
    static_assert((kSets - 1) * kNB * kNC <= 2 * kVS + 2 * kCS, "park area");
    T* park = kKeep ? sm + kTileSmem : sV0;
    if (set > 0)
#pragma unroll
      for (int a = 0; a < kIW; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) park[(set - 1) * kNB * kNC + (i0 + a) * kNC + c0 + q] = acc[a][q];
    __syncthreads();
    if (set == 0)
#pragma unroll
      for (int a = 0; a < kIW; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = i0 + a, c = c0 + q;
          T w = acc[a][q];
#pragma unroll
          for (int p = 0; p < kSets - 1; ++p) w += park[p * kNB * kNC + i * kNC + c];
          sW[i * kNC + c] = w;
        }
  }
  __syncthreads();
  // T to shared memory (the tail of the tile buffers), A into W
  T* sT = sV0 + 2 * kVS + 2 * kCS - kNB * (kNB + 1);  // sT[l * (kNB+1) + i] = T(l, i)
#pragma unroll
  for (int q = 0; q < kST; ++q) {
    const int idx = t + q * kThreads;
    sT[(idx & (kNB - 1)) * (kNB + 1) + idx / kNB] = rt[q];
  }
  if (!unit)
#pragma unroll
    for (int q = 0; q < kSA; ++q) {
      const int idx = t + q * kThreads;
      sW[(idx & (kNB - 1)) * kNC + idx / kNB] += ra[q];
    }
  __syncthreads();
  // ---- W2 = T^T W (T upper triangular: W2(i) = sum_{l <= i} T(l, i) W(l))
  T* sW2 = kKeep ? sm + kTileSmem + (kThreads / ((kNB / 8) * (kNC / 4)) - 1) * kNB * kNC : sV0;
  static_assert(kNB * kNC <= 2 * kVS + 2 * kCS - kNB * (kNB + 1), "W2 and T areas");
  for (int idx = t; idx < kNB * kNC; idx += kThreads) {
    const int i = idx / kNC, c = idx % kNC;
    T s = 0.0;
    if (i < kb)
      for (int l = 0; l <= i; ++l) s += sT[l * (kNB + 1) + i] * sW[l * kNC + c];
    sW2[i * kNC + c] = s;
  }
  __syncthreads();
  if (!unit)
    for (int idx = t; idx < kb * nc; idx += kThreads) {
      const int i = idx % kb, c = idx / kb;
      A[i + col(c) * lda] -= sW2[i * kNC + c];
    }
  // ---- C -= V W2.  A thread keeps W2(:, its kCW columns) in registers and
  // owns kRW rows of each tile (a warp shares its rows: V rows are broadcast)
  constexpr int kCW = sizeof(T) == 4 ? 2 : 1;     // columns per thread
  constexpr int kRW = kRT * kNC / kThreads / kCW;  // rows per thread
  const int cq = (t % (kNC / kCW)) * kCW, rq = (t / (kNC / kCW)) * kRW;
  T w2[kNB][kCW];
#pragma unroll
  for (int i = 0; i < kNB; ++i)
#pragma unroll
    for (int q = 0; q < kCW; ++q) w2[i][q] = sW2[i * kNC + cq + q];
  __syncthreads();
  if (!(kKeep && ntile == 1)) {  // a single FP32 tile is still staged in buffer 0
    vload(0);
    cload(0);
    vstash(0);
    cstash(0);
    __syncthreads();
  }
  for (int tt = 0; tt < ntile; ++tt) {
    const int b = tt & 1, r0 = tt * kRT;
    const bool more = tt + 1 < ntile;
    if (more) {
      vload(r0 + kRT);
      cload(r0 + kRT);
    }
    const T* sV = sV0 + b * kVS;
    T* sC = sC0 + b * kCS;
#pragma unroll
    for (int r = 0; r < kRW; ++r) {
      const T* vr = sV + (rq + r) * kLV;
      T u[kCW];
#pragma unroll
      for (int q = 0; q < kCW; ++q) u[q] = 0.0;
#pragma unroll
      for (int i = 0; i < kNB; ++i) {
        const T a = vr[i];
#pragma unroll
        for (int q = 0; q < kCW; ++q) u[q] += a * w2[i][q];
      }
#pragma unroll
      for (int q = 0; q < kCW; ++q) sC[(rq + r) * kLC + cq + q] -= u[q];
    }
    __syncthreads();
    // the updated tile back to global memory, coalesced
    if (r0 + lr < m)
#pragma unroll
      for (int q = 0; q < kSC; ++q) {
        const int c = lw * kSC + q;
        if (c < nc) C[(r0 + lr) + col(c) * ldc] = sC[lr * kLC + c];
      }
    if (more) {
      vstash(b ^ 1);
      cstash(b ^ 1);
    }
    __syncthreads();
  }
}

// C (m <= kNC rows x n) <- C (I - V T V^T) with one panel, V unit lower
// trapezoidal (n x kb).  Column tiles of kRT stream through two shared
// buffers: the next tile's global loads are issued before the current tile's
// products.
template <typename T>
__device__ void tile_right_q(const T* V, int ldv, const T* Tm, int ldt, int kb, T* C, int ldc, int m,
                             int n, T* sm) {
  constexpr int kVS = kRT * (kNB + 1), kCS = kNC * (kRT + 1);
  static_assert(2 * kVS + 2 * kCS + kNC * kNB <= kTileSmem, "right apply scratch");
  T* sV0 = sm;               // two [kRT][kNB+1] tiles: V rows c0..c0+31
  T* sC0 = sV0 + 2 * kVS;    // two [kNC][kRT+1] tiles: C(r, c0+c)
  T* sW = sC0 + 2 * kCS;     // [kNC][kNB] W(r, i)
  const int t = threadIdx.x;
  constexpr int kSV = kRT * kNB / kThreads, kSC = kNC * kRT / kThreads;
  T rv[kSV], rc[kSC];
  auto vload = [&](int c0) {
#pragma unroll
    for (int q = 0; q < kSV; ++q) {
      const int idx = t + q * kThreads, c = idx % kRT, i = idx / kRT, gc = c0 + c;
      T v = 0.0;
      if (gc < n && i < kb) v = gc == i ? (T)1.0 : (gc < i ? (T)0.0 : V[gc + (size_t)i * ldv]);
      rv[q] = v;
    }
  };
  auto vstash = [&](int b) {
#pragma unroll
    for (int q = 0; q < kSV; ++q) {
      const int idx = t + q * kThreads;
      sV0[b * kVS + (idx % kRT) * (kNB + 1) + idx / kRT] = rv[q];
    }
  };
  auto cload = [&](int c0) {
#pragma unroll
    for (int q = 0; q < kSC; ++q) {
      const int idx = t + q * kThreads, r = idx % kNC, c = idx / kNC;
      rc[q] = (r < m && c0 + c < n) ? C[r + (size_t)(c0 + c) * ldc] : (T)0.0;
    }
  };
  auto cstash = [&](int b) {
#pragma unroll
    for (int q = 0; q < kSC; ++q) {
      const int idx = t + q * kThreads;
      sC0[b * kCS + (idx % kNC) * (kRT + 1) + idx / kNC] = rc[q];
    }
  };
  const int ntile = (n + kRT - 1) / kRT;
  const int ti = t & 7, tr = t >> 3;  // i = ti*4..+3, r = tr*2..+1
  T acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
  vload(0);
  cload(0);
  vstash(0);
  cstash(0);
  __syncthreads();
  for (int tt = 0; tt < ntile; ++tt) {
    const int b = tt & 1;
    const bool more = tt + 1 < ntile;
    if (more) {
      vload((tt + 1) * kRT);
      cload((tt + 1) * kRT);
    }
    const T* sV = sV0 + b * kVS;
    const T* sC = sC0 + b * kCS;
#pragma unroll 8
    for (int c = 0; c < kRT; ++c) {
      const T a0 = sC[(tr * 2) * (kRT + 1) + c], a1 = sC[(tr * 2 + 1) * (kRT + 1) + c];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T v = sV[c * (kNB + 1) + ti * 4 + q];
        acc[0][q] += a0 * v;
        acc[1][q] += a1 * v;
      }
    }
    if (more) {
      vstash(b ^ 1);
      cstash(b ^ 1);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) sW[(tr * 2 + p) * kNB + ti * 4 + q] = acc[p][q];
  __syncthreads();
  // W2 = W T (W2(r,i) = sum_{l <= i} W(r,l) T(l,i)), T staged in shared memory
  T* sT = sC0;                 // [kNB][kNB+1]
  T* sW2 = sC0 + kNB * (kNB + 1);  // [kNC][kNB]
  for (int idx = t; idx < kNB * kNB; idx += kThreads) {
    const int l = idx % kNB, i = idx / kNB;
    sT[l * (kNB + 1) + i] = (l <= i && i < kb) ? Tm[l + (size_t)i * ldt] : (T)0.0;
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = tr * 2 + p, i = ti * 4 + q;
      T s = 0.0;
      if (i < kb)
        for (int l = 0; l <= i; ++l) s += sW[r * kNB + l] * sT[l * (kNB + 1) + i];
      sW2[r * kNB + i] = s;
    }
  __syncthreads();
  // C(r, c) -= sum_i W2(r, i) V(c, i): thread rows rr, rr+32, columns cc*4..+3
  // of each tile; the next tile's V is loaded before the current products
  const int rr = t & 31, cc = t >> 5;
  vload(0);
  vstash(0);
  __syncthreads();
  for (int tt = 0; tt < ntile; ++tt) {
    const int b = tt & 1, c0 = tt * kRT;
    const bool more = tt + 1 < ntile;
    if (more) vload(c0 + kRT);
    const T* sV = sV0 + b * kVS;
    T u[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll 8
    for (int i = 0; i < kNB; ++i) {
      const T w0 = sW2[rr * kNB + i], w1 = sW2[(rr + 32) * kNB + i];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T v = sV[(cc * 4 + q) * (kNB + 1) + i];
        u[0][q] += w0 * v;
        u[1][q] += w1 * v;
      }
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = rr + 32 * p, c = cc * 4 + q;
        if (r < m && c0 + c < n) C[r + (size_t)(c0 + c) * ldc] -= u[p][q];
      }
    if (more) vstash(b ^ 1);
    __syncthreads();
  }
}

// Panel loops of the tiled applies over k reflectors (T in kNB x k layout).
template <typename T>
__device__ void mat_apply_qt(const T* V, int ldv, const T* Tm, int k, T* C, int ldc, int m, int nc,
                             T* sm) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int c0 = 0; c0 < nc; c0 += kNC)
      tile_left_qt<T>(V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 1, nullptr, 0,
                   C + j0 + (size_t)c0 * ldc, ldc, m - j0, (nc - c0) < kNC ? (nc - c0) : kNC, sm);
  }
}
template <typename T>
__device__ void mat_apply_tpqt(const T* V, int ldv, const T* Tm, int k, T* A, int lda, T* B,
                               int ldb, int m, int nc, T* sm) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int c0 = 0; c0 < nc; c0 += kNC)
      tile_left_qt(V + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 0, A + j0 + (size_t)c0 * lda, lda,
                   B + (size_t)c0 * ldb, ldb, m, (nc - c0) < kNC ? (nc - c0) : kNC, sm);
  }
}
template <typename T>
__device__ void mat_apply_q_right(const T* V, int ldv, const T* Tm, int k, T* C, int ldc, int m, int n,
                                  T* sm) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    for (int r0 = 0; r0 < m; r0 += kNC)
      tile_right_q(V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, C + r0 + (size_t)j0 * ldc, ldc,
                   (m - r0) < kNC ? (m - r0) : kNC, n - j0, sm);
  }
}


// ---------------------------------------------------------------- single-vector applies
// Shared scratch of vec_panel (elements): partial sums and W2.
constexpr int kVecRed = (kWarps + 1) * 32;

// One panel of kb <= kNB reflectors on a vector in shared memory:
//   unit = 1: x (m) <- (I - V T V^T)^T x (trans) or (I - V T V^T) x, V unit
//             lower trapezoidal from the panel's diagonal;
//   unit = 0: [a (kb); x (m)] <- Q^T [a; x], Q = I - [I; V] T [I; V]^T, V full.
// Every thread takes rows t, t + kThreads, ... and issues the kb loads of a row
// together; the kb partial sums are reduce-scattered across each warp (lane i
// ends with reflector i's sum) and across the warps through `red`.
template <typename T>
__device__ void vec_panel(const T* V, int ldv, const T* Tm, int ldt, int kb, int unit, bool trans, T* a, T* x,
                          int m, T* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // warp 0: column `lane` (trans) or row `lane` of T, loaded now and used
  // after the rows' products, so that its latency overlaps them
  T tv[kNB];
  if (warp == 0) {
#pragma unroll
    for (int l = 0; l < kNB; ++l) {
      const bool ok = l < kb && lane < kb && (trans ? l <= lane : l >= lane);
      tv[l] = ok ? (trans ? Tm[l + (size_t)lane * ldt] : Tm[lane + (size_t)l * ldt]) : (T)0.0;
    }
  }
  T acc[kNB];
#pragma unroll
  for (int i = 0; i < kNB; ++i) acc[i] = 0.0;
  for (int r = threadIdx.x; r < m; r += kThreads) {
    const T xr = x[r];
#pragma unroll
    for (int i = 0; i < kNB; ++i) {
      T v = 0.0;
      if (i < kb) v = unit ? (r == i ? (T)1.0 : (r < i ? (T)0.0 : V[r + (size_t)i * ldv])) : V[r + (size_t)i * ldv];
      acc[i] += v * xr;
    }
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int q = 0; q < o; ++q) {
      const T send = up ? acc[q] : acc[q + o];
      const T keep = up ? acc[q + o] : acc[q];
      acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  red[warp * 32 + lane] = acc[0];
  __syncthreads();
  T* w2 = red + kWarps * 32;
  if (warp == 0) {
    T w = 0.0;
    for (int q = 0; q < kWarps; ++q) w += red[q * 32 + lane];
    if (!unit && lane < kb) w += a[lane];
    T s = 0.0;
#pragma unroll
    for (int l = 0; l < kNB; ++l) s += tv[l] * __shfl_sync(0xffffffffu, w, l);
    w2[lane] = lane < kb ? s : (T)0.0;
    if (!unit && lane < kb) a[lane] -= s;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < m; r += kThreads) {
    T s = 0.0;
#pragma unroll
    for (int i = 0; i < kNB; ++i) {
      T v = 0.0;
      if (i < kb) v = unit ? (r == i ? (T)1.0 : (r < i ? (T)0.0 : V[r + (size_t)i * ldv])) : V[r + (size_t)i * ldv];
      s += v * w2[i];
    }
    x[r] -= s;
  }
  __syncthreads();
}

// [a (k); x (m)] <- Q^T [a; x] for a pentagonal (tpqrt) factor, V full (m x k).
template <typename T>
__device__ void vec_apply_tpqt(const T* V, int ldv, const T* Tm, int k, T* a, T* x, int m, T* red) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    vec_panel<T>(V + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 0, true, a + j0, x, m, red);
  }
}

// ---------------------------------------------------------------- staged single-vector applies
// Asynchronous global -> shared copies (cp.async): 16-byte chunks where the
// source is 16-byte aligned, single elements at the unaligned head and tail.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* sdst, const T* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  if (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Elements of a 16-byte chunk, and the shift that gives a shared copy of
// g[0, len) the same 16-byte phase as g.
template <typename T>
constexpr int kE16 = 16 / (int)sizeof(T);
template <typename T>
__device__ __forceinline__ int phase_of(const T* g) {
  return (int)(((uintptr_t)g & 15u) / sizeof(T));
}

// One warp copies g[0, len) to d[0, len); d must have g's 16-byte phase.
template <typename T>
__device__ __forceinline__ void warp_copy_async(T* d, const T* g, int len, int lane) {
  int h = (kE16<T> - phase_of(g)) % kE16<T>;
  if (h > len) h = len;
  for (int e = lane; e < h; e += 32) cp_async_elem(d + e, g + e);
  const int nc = (len - h) / kE16<T>;
  for (int c = lane; c < nc; c += 32) cp_async16(d + h + c * kE16<T>, g + h + c * kE16<T>);
  for (int e = h + nc * kE16<T> + lane; e < len; e += 32) cp_async_elem(d + e, g + e);
}

// Shared memory (elements) of vec_apply_staged for m rows: two panel buffers
// of kNB columns (column stride staged_ld), two T blocks (each with room for
// a 16-byte phase shift), W and W2.
template <typename T>
__host__ __device__ constexpr int staged_ld(int m) {
  return (m + 2 * kE16<T> - 1) / kE16<T> * kE16<T>;
}
template <typename T>
__host__ __device__ constexpr int staged_tld() {
  return kNB * kNB + kE16<T>;
}
template <typename T>
__host__ __device__ constexpr size_t staged_elems(int m) {
  return 2 * (size_t)kNB * staged_ld<T>(m) + 2 * (size_t)staged_tld<T>() + 2 * kNB;
}

// x (m) <- Q^T x (trans) or Q x for k unit lower trapezoidal reflectors (T in
// kNB x k layout) with the panels streamed through shared memory: while panel
// p is applied from one buffer, panel p + 1 (its rows from its diagonal down,
// and its T block) is copied into the other with cp.async, so a whole panel
// of loads is in flight instead of a few per thread.  Per panel:
//   W = V^T x   (a warp per reflector, lanes over rows);
//   W2 = T^T W (trans) or T W, by warp 0;
//   x -= V W2   (a thread per row).
// With `a` (pentagonal, trans only): [a (k); x (m)] <- Q^T [a; x] for
// Q = I - [I; V] T [I; V]^T with V full (m x k), as in vec_apply_tpqt: every
// panel covers all m rows, W adds a, and a -= W2.
// x (and a) in shared memory; buf: staged_elems<T>(m) elements, 16-byte
// aligned.  All threads of the CTA call it; it synchronises internally.
template <typename T>
__device__ void vec_apply_staged(const T* V, int ldv, const T* Tm, int k, T* x, int m, bool trans, T* buf,
                                 T* a = nullptr) {
  if (k <= 0 || m <= 0) return;
  __shared__ int s_off[2][kNB];  // element (r, i) of the staged panel at pb[.][s_off[.][i] + r]
  __shared__ int s_toff[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lds = staged_ld<T>(m);
  T* const pb0 = buf;
  T* const tb0 = buf + 2 * (size_t)kNB * lds;
  T* const W = tb0 + 2 * staged_tld<T>();
  T* const W2 = W + kNB;
  const int np = (k + kNB - 1) / kNB;
  auto j0_of = [&](int s) { return (trans ? s : np - 1 - s) * kNB; };
  auto stage = [&](int s, int b) {
    const int j0 = j0_of(s);
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    const int rs = a ? 0 : j0;  // first staged row
    T* pb = pb0 + (size_t)b * kNB * lds;
    for (int i = warp; i < kb; i += kWarps) {
      const T* g = V + (size_t)(j0 + i) * ldv + rs;
      const int ph = phase_of(g);
      warp_copy_async(pb + (size_t)i * lds + ph, g, m - rs, lane);
      if (lane == 0) s_off[b][i] = i * lds + ph - rs;
    }
    if (warp == kWarps - 1) {
      const T* g = Tm + (size_t)j0 * kNB;
      const int ph = phase_of(g);
      warp_copy_async(tb0 + (size_t)b * staged_tld<T>() + ph, g, kNB * kb, lane);
      if (lane == 0) s_toff[b] = b * staged_tld<T>() + ph;
    }
    cp_async_commit();
  };
  stage(0, 0);
  for (int s = 0; s < np; ++s) {
    const int b = s & 1;
    const int j0 = j0_of(s);
    const int kb = (k - j0) < kNB ? (k - j0) : kNB;
    if (s + 1 < np) {
      stage(s + 1, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* pb = pb0 + (size_t)b * kNB * lds;
    const T* tp = tb0 + s_toff[b];
    // W(i) = x(j0 + i) + sum_{r > j0 + i} V(r, i) x(r), or a(j0 + i) + sum_r V(r, i) x(r)
    for (int i = warp; i < kb; i += kWarps) {
      const T* col = pb + s_off[b][i];
      T d = 0.0;
      for (int r = (a ? 0 : j0 + i + 1) + lane; r < m; r += 32) d += col[r] * x[r];
      d = warp_sum(d);
      if (lane == 0) W[i] = d + (a ? a[j0 + i] : x[j0 + i]);
    }
    __syncthreads();
    if (warp == 0) {
      T acc = 0.0;
      if (lane < kb) {
        if (trans)
          for (int l = 0; l <= lane; ++l) acc += tp[l + lane * kNB] * W[l];
        else
          for (int l = lane; l < kb; ++l) acc += tp[lane + l * kNB] * W[l];
        if (a) a[j0 + lane] -= acc;
      }
      W2[lane] = acc;
    }
    __syncthreads();
    if (a) {
      for (int r = threadIdx.x; r < m; r += kThreads) {
        T acc = 0.0;
#pragma unroll 8
        for (int i = 0; i < kb; ++i) acc += pb[s_off[b][i] + r] * W2[i];
        x[r] -= acc;
      }
    } else {
      for (int r = j0 + threadIdx.x; r < m; r += kThreads) {
        const int lim = (r - j0) < kb ? (r - j0) : kb;
        T acc = (r - j0) < kb ? W2[r - j0] : (T)0.0;
#pragma unroll 8
        for (int i = 0; i < lim; ++i) acc += pb[s_off[b][i] + r] * W2[i];
        x[r] -= acc;
      }
    }
    __syncthreads();
  }
}

// C (m <= kNC rows x n) <- C R^{-1}, R upper triangular (n x n), blocked by 32
// columns: C(:, J) -= C(:, 0:j0) R(0:j0, J) through shared-memory tiles, then
// the 32 x 32 diagonal block is solved one row per thread.
template <typename T>
__device__ void tile_trsm_right_upper(const T* R, int ldr, T* C, int ldc, int m, int n, T* sm) {
  constexpr int kRS = kRT * (kNB + 1), kCS = kNC * (kRT + 1);
  static_assert(2 * kRS + 2 * kCS <= kTileSmem, "right solve scratch");
  T* sR0 = sm;                 // two [kRT][kNB+1] tiles: R(l0+l, j0+j)
  T* sC0 = sR0 + 2 * kRS;      // two [kNC][kRT+1] tiles: C(r, l0+l)
  T* sR = sR0;                 // the diagonal block, after the products
  T* sC = sC0;                 // the block being solved
  const int t = threadIdx.x;
  const int tj = t & 7, tr = t >> 3;    // cols tj*4..+3, rows tr*2..+1
  constexpr int kSR = kRT * kNB / kThreads, kSC = kNC * kRT / kThreads;
  T rr[kSR], rc[kSC];
  // tiles of the already solved columns, the next one loaded before the
  // current one's products
  auto load = [&](int l0, int j0, int jb) {
#pragma unroll
    for (int q = 0; q < kSR; ++q) {
      const int idx = t + q * kThreads, l = idx % kRT, j = idx / kRT;
      rr[q] = (j < jb) ? R[(l0 + l) + (size_t)(j0 + j) * ldr] : (T)0.0;
    }
#pragma unroll
    for (int q = 0; q < kSC; ++q) {
      const int idx = t + q * kThreads, r = idx % kNC, l = idx / kNC;
      rc[q] = (r < m) ? C[r + (size_t)(l0 + l) * ldc] : (T)0.0;
    }
  };
  auto stash = [&](int b) {
#pragma unroll
    for (int q = 0; q < kSR; ++q) {
      const int idx = t + q * kThreads;
      sR0[b * kRS + (idx % kRT) * (kNB + 1) + idx / kRT] = rr[q];
    }
#pragma unroll
    for (int q = 0; q < kSC; ++q) {
      const int idx = t + q * kThreads;
      sC0[b * kCS + (idx % kNC) * (kRT + 1) + idx / kNC] = rc[q];
    }
  };
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int jb = (n - j0) < kNB ? (n - j0) : kNB;
    T acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    const int nl = (j0 + kRT - 1) / kRT;
    if (nl > 0) {
      load(0, j0, jb);
      stash(0);
      __syncthreads();
    }
    for (int it = 0; it < nl; ++it) {
      const int b = it & 1;
      const bool more = it + 1 < nl;
      if (more) load((it + 1) * kRT, j0, jb);
      const T* tR = sR0 + b * kRS;
      const T* tC = sC0 + b * kCS;
#pragma unroll 4
      for (int l = 0; l < kRT; ++l) {
        const T a0 = tC[(tr * 2) * (kRT + 1) + l], a1 = tC[(tr * 2 + 1) * (kRT + 1) + l];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const T rv = tR[l * (kNB + 1) + tj * 4 + q];
          acc[0][q] += a0 * rv;
          acc[1][q] += a1 * rv;
        }
      }
      if (more) stash(b ^ 1);
      __syncthreads();
    }
    // subtract into the block, stage it in shared memory with the diagonal R block
    for (int idx = t; idx < kNB * kNB; idx += kThreads) {
      const int l = idx % kNB, j = idx / kNB;
      sR[l * (kNB + 1) + j] = (l < jb && j < jb) ? R[(j0 + l) + (size_t)(j0 + j) * ldr] : 0.0;
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = tr * 2 + p, j = tj * 4 + q;
        sC[r * (kRT + 1) + j] = (r < m && j < jb) ? C[r + (size_t)(j0 + j) * ldc] - acc[p][q] : 0.0;
      }
    __syncthreads();
    for (int r = t; r < m; r += kThreads) {
      T* cr = sC + r * (kRT + 1);
      for (int j = 0; j < jb; ++j) {
        T s = cr[j];
        for (int l = 0; l < j; ++l) s -= cr[l] * sR[l * (kNB + 1) + j];
        cr[j] = s / sR[j * (kNB + 1) + j];
      }
    }
    __syncthreads();
    for (int idx = t; idx < kNC * kNB; idx += kThreads) {
      const int r = idx % kNC, j = idx / kNC;
      if (r < m && j < jb) C[r + (size_t)(j0 + j) * ldc] = sC[r * (kRT + 1) + j];
    }
    __syncthreads();
  }
}

// C (m x n) <- C R^{-1}, R upper triangular (n x n).  One thread per row.
template <typename T>
__device__ void trsm_right_upper(const T* R, int ldr, T* C, int ldc, int m, int n) {
  for (int r = threadIdx.x; r < m; r += kThreads) {
    for (int j = 0; j < n; ++j) {
      T s = C[r + (size_t)j * ldc];
      const T* rj = R + (size_t)j * ldr;
      for (int i = 0; i < j; ++i) s -= C[r + (size_t)i * ldc] * rj[i];
      C[r + (size_t)j * ldc] = s / rj[j];
    }
  }
  __syncthreads();
}

// Upper triangular solve x <- R^{-1} x (n x n), blocked by 32, bottom block
// first.  Warp 0 holds the diagonal block in registers (lane i: row i's part
// on and above the diagonal), loaded while the CTA updates the rows above the
// previous block, and solves it with shuffles; the CTA then updates the rows
// above with the solved block.
template <typename T>
__device__ void trsv_upper(const T* R, int ldr, T* x, int n, T* xs /*shared >= 32*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T rv[32];
  auto fetch = [&](int lo, int bs) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      rv[j] = (j < bs && lane <= j) ? R[(lo + lane) + (size_t)(lo + j) * ldr] : (T)0.0;
  };
  if (warp == 0 && n > 0) fetch(n > 32 ? n - 32 : 0, n > 32 ? 32 : n);
  for (int hi = n; hi > 0; hi -= 32) {
    const int lo = hi > 32 ? hi - 32 : 0;
    const int bs = hi - lo;
    if (warp == 0) {
      T xv = lane < bs ? x[lo + lane] : 0.0;
#pragma unroll
      for (int j = 31; j >= 0; --j) {
        if (j < bs) {
          if (lane == j) xv = xv / rv[j];
          const T xj = __shfl_sync(0xffffffffu, xv, j);
          if (lane < j) xv -= rv[j] * xj;
        }
      }
      if (lane < bs) {
        x[lo + lane] = xv;
        xs[lane] = xv;
      }
      if (lo > 0) fetch(lo > 32 ? lo - 32 : 0, lo > 32 ? 32 : lo);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < lo; r += kThreads) {
      T s = 0.0;
      for (int j = 0; j < bs; ++j) s += R[r + (size_t)(lo + j) * ldr] * xs[j];
      x[r] -= s;
    }
    __syncthreads();
  }
}

}  // namespace dev
}  // namespace spq
