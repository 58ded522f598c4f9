// kernels.cu -- grouped FP64 kernels of the factorization, the preconditioner
// apply and the Krylov loop for sm_100a.
//
// Factorizations whose work is sequential over reflectors (the diagonal QR +
// tsqrt chain of an interior, the scaling QR, the pivoted QR of the
// sparsification) run one task per thread-block cluster: the task's 32-column
// panels are dealt round-robin to the cluster's CTAs, the CTA owning column j
// builds reflector j, a cluster barrier publishes it, and every CTA applies it
// to its own panels.  Small tasks use clusters of one CTA.  Block applies that
// are independent across columns (or rows) are split into chunks, one CTA each.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "dense.cuh"
#include "kernels.hpp"
#include "tasks.hpp"
#include "tc_apply.cuh"

namespace cg = cooperative_groups;

namespace spq {
namespace {

using dev::kNB;
using dev::kThreads;
using dev::kWarps;

constexpr int kRed = 16;     // reduction scratch (doubles)
// dist_qr's staged panel beyond its rows x kNB: the tpqrt's R block (kNB x
// kNB) and the panel's Gram matrix (kNB x (kNB + 1))
constexpr int kPanExtra = kNB * kNB + kNB * (kNB + 1);
constexpr int kWcap = dev::kTileSmem;  // shared scratch (doubles) of the tiled block applies

__device__ __forceinline__ void csync(int cs) {
  if (cs > 1) cg::this_cluster().sync();
  else __syncthreads();
}
__device__ __forceinline__ int crank(int cs) { return cs > 1 ? (int)cg::this_cluster().block_rank() : 0; }
__device__ __forceinline__ bool owns(int col, int rank, int cs) { return ((col / kNB) % cs) == rank; }

// ------------------------------------------------------------ assembly
// Factor blocks hold T (double, or float in the mixed-precision
// factorization); descriptors carry their addresses as double*.
template <typename T>
__device__ __forceinline__ T* as(double* p) {
  return reinterpret_cast<T*>(p);
}
template <typename T>
__device__ __forceinline__ const T* as(const double* p) {
  return reinterpret_cast<const T*>(p);
}

template <typename T>
__global__ void k_scatter(int nnz, const double* __restrict__ val, double* const* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x)
    *as<T>(dst[i]) = (T)val[i];
}

// ------------------------------------------------------------ distributed Householder QR
// Blocked Householder QR over a cluster: a geqrt (unit = 1: reflector j is
// v = [1; R(j+1:m, j)]) or a tpqrt (unit = 0: v = [1 (on R(j,j)); B(:, j)]).
// The 32-column panels are dealt round-robin to the cluster's CTAs.  For each
// panel its owner builds the kb reflectors, applying each only inside the
// panel, and the panel's T factor; after one cluster barrier every CTA
// applies the block reflector to its own later panels with the tiled apply
// (two of its panels per pass).  `lt` holds the owner's tau values, `tg`
// the global copy, `vb` a reflector tail, `tile` dev::kTileSmem elements.
//
// With `pan` (ldp >= the panel's rows; ldp * kNB + kPanExtra elements, may
// alias `tile`), the owner copies the panel into shared memory, runs the kb
// reflector steps and the T factor there (one barrier per reflector, T by
// one warp) and writes the panel back once.
template <typename T>
__device__ void dist_qr(T* R, int ldr, T* B, int ldb, int m, int n, int unit, T* Tout, T* tg,
                        T* lt, T* vb, T* red, T* tmp, T* tile, int cs, int* status = nullptr, T* pan = nullptr,
                        int ldp = 0) {
  const int rank = crank(cs);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gap = (cs - 1) * kNB;  // columns between two panels of one CTA
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int kb = (n - j0) < kNB ? (n - j0) : kNB;
    const int pend = j0 + kb;
    if (owns(j0, rank, cs) && pan) {
      // panel rows: [j0, m) of R's columns (geqrt) or B's m rows (tpqrt)
      const int pm = unit ? m - j0 : m;
      T* pr = pan + (size_t)ldp * kNB;  // tpqrt: R(j0:pend, j0:pend), ld kNB
      T* sG = pr + kNB * kNB;           // the panel's Gram matrix (panel_t_warp)
      __syncthreads();                  // `pan` may alias the tiled apply's scratch
      for (int c = warp; c < kb; c += kWarps) {
        const T* src = unit ? (R + j0 + (size_t)(j0 + c) * ldr) : (B + (size_t)(j0 + c) * ldb);
        for (int i = lane; i < pm; i += 32) pan[i + (size_t)c * ldp] = __ldcg(src + i);
      }
      if (!unit)
        for (int e = threadIdx.x; e < kb * kb; e += kThreads) {
          const int r = e % kb, c = e / kb;
          if (r <= c) pr[r + c * kNB] = __ldcg(R + (j0 + r) + (size_t)(j0 + c) * ldr);
        }
      __syncthreads();
      // One barrier per reflector.  Every thread forms reflector j from its
      // alpha and the squared norm of its tail; warp w applies it to columns
      // j + 1 + w, ... with v = tail * scal formed on the fly, and the warp of
      // column j + 1 also sums that column's new tail for reflector j + 1.
      // The scaled tail and beta are stored one step later, when no warp
      // reads them.
      __shared__ T s_nrm2[2];
      T nrm2;
      {
        const int vlen = unit ? m - j0 - 1 : m;
        const T* tail = unit ? pan + 1 : pan;
        T sq = 0.0;
        for (int i = threadIdx.x; i < vlen; i += kThreads) sq += tail[i] * tail[i];
        nrm2 = dev::cta_sum(sq, red);
      }
      T* prev_tail = nullptr;
      T prev_scal = 0.0;
      int prev_vlen = 0;
      T* prev_ajj = nullptr;
      T prev_beta = 0.0;
      for (int j = j0; j < pend; ++j) {
        const int jj = j - j0;
        const int vlen = unit ? (m - j - 1) : m;
        T* tail = unit ? (pan + (jj + 1) + (size_t)jj * ldp) : (pan + (size_t)jj * ldp);
        T* ajj = unit ? (pan + jj + (size_t)jj * ldp) : (pr + jj + jj * kNB);
        const T alpha = *ajj;
        T beta, scal;
        const T tj = dev::house(alpha, nrm2, &beta, &scal);
        if (prev_tail)
          for (int i = threadIdx.x; i < prev_vlen; i += kThreads) prev_tail[i] *= prev_scal;
        if (threadIdx.x == 0) {
          if (prev_ajj) *prev_ajj = prev_beta;
          lt[j] = tj;
          tg[j] = tj;
          // R(j, j) = 0 or not finite: the triangular solves would break down
          if (status && !(isfinite(beta) && beta != (T)0)) atomicOr(status, isfinite(beta) ? 8 : 4);
        }
        for (int k = j + 1 + warp; k < pend; k += kWarps) {
          const int kk = k - j0;
          T* rjk = unit ? (pan + jj + (size_t)kk * ldp) : (pr + jj + kk * kNB);
          T* tk = unit ? (pan + (jj + 1) + (size_t)kk * ldp) : (pan + (size_t)kk * ldp);
          if (tj != 0.0) {
            T d = lane == 0 ? *rjk : 0.0;
            for (int i = lane; i < vlen; i += 32) d += (tail[i] * scal) * tk[i];
            d = dev::warp_sum(d) * tj;
            if (lane == 0) *rjk -= d;
            for (int i = lane; i < vlen; i += 32) tk[i] -= (tail[i] * scal) * d;
          }
          if (k == j + 1) {  // reflector j + 1's tail: rows below its diagonal
            T sq = 0.0;
            for (int i = lane; i < vlen; i += 32)
              if (!unit || i > 0) sq += tk[i] * tk[i];
            sq = dev::warp_sum(sq);
            if (lane == 0) s_nrm2[(j + 1) & 1] = sq;
          }
        }
        prev_tail = tj != 0.0 ? tail : nullptr;
        prev_scal = scal;
        prev_vlen = vlen;
        prev_ajj = ajj;
        prev_beta = beta;
        __syncthreads();
        nrm2 = s_nrm2[(j + 1) & 1];
      }
      if (prev_tail)
        for (int i = threadIdx.x; i < prev_vlen; i += kThreads) prev_tail[i] *= prev_scal;
      if (threadIdx.x == 0 && prev_ajj) *prev_ajj = prev_beta;
      __syncthreads();
      dev::panel_t_warp(pan, ldp, pm, kb, unit, lt + j0, Tout + (size_t)j0 * kNB, kNB, sG);
      for (int c = warp; c < kb; c += kWarps) {
        T* dst = unit ? (R + j0 + (size_t)(j0 + c) * ldr) : (B + (size_t)(j0 + c) * ldb);
        for (int i = lane; i < pm; i += 32) dst[i] = pan[i + (size_t)c * ldp];
      }
      if (!unit)
        for (int e = threadIdx.x; e < kb * kb; e += kThreads) {
          const int r = e % kb, c = e / kb;
          if (r <= c) R[(j0 + r) + (size_t)(j0 + c) * ldr] = pr[r + c * kNB];
        }
      __threadfence();
      __syncthreads();
    } else if (owns(j0, rank, cs)) {
      for (int j = j0; j < pend; ++j) {
        const int vlen = unit ? (m - j - 1) : m;
        T* tail = unit ? (R + (j + 1) + (size_t)j * ldr) : (B + (size_t)j * ldb);
        T s = 0.0;
        for (int i = threadIdx.x; i < vlen; i += kThreads) s += tail[i] * tail[i];
        s = dev::cta_sum(s, red);
        const T alpha = R[j + (size_t)j * ldr];
        T beta, scal;
        const T tj = dev::house(alpha, s, &beta, &scal);
        if (tj != 0.0)
          for (int i = threadIdx.x; i < vlen; i += kThreads) {
            const T v = tail[i] * scal;
            tail[i] = v;
            vb[i] = v;
          }
        if (threadIdx.x == 0) {
          R[j + (size_t)j * ldr] = beta;
          lt[j] = tj;
          tg[j] = tj;
          // R(j, j) = 0 or not finite: the triangular solves would break down
          if (status && !(isfinite(beta) && beta != (T)0)) atomicOr(status, isfinite(beta) ? 8 : 4);
        }
        __syncthreads();
        // H_j on the panel's later columns
        if (tj != 0.0)
          for (int k = j + 1 + warp; k < pend; k += kWarps) {
            T* rjk = R + j + (size_t)k * ldr;
            T* tk = unit ? (R + (j + 1) + (size_t)k * ldr) : (B + (size_t)k * ldb);
            T d = lane == 0 ? *rjk : 0.0;
            for (int i = lane; i < vlen; i += 32) d += vb[i] * tk[i];
            d = dev::warp_sum(d) * tj;
            if (lane == 0) *rjk -= d;
            for (int i = lane; i < vlen; i += 32) tk[i] -= vb[i] * d;
          }
        __syncthreads();
      }
      if (unit)
        dev::panel_t(R + j0 + (size_t)j0 * ldr, ldr, m - j0, kb, 1, lt + j0, Tout + (size_t)j0 * kNB, kNB, tmp);
      else
        dev::panel_t(B + (size_t)j0 * ldb, ldb, m, kb, 0, lt + j0, Tout + (size_t)j0 * kNB, kNB, tmp);
      __threadfence();
    }
    csync(cs);
    // the panel's block reflector on own later panels, two per pass
    const T* Tm = Tout + (size_t)j0 * kNB;
    int q0 = pend;  // first column of own later panels
    while (q0 < n && !owns(q0, rank, cs)) q0 += kNB;
    for (; q0 < n; q0 += 2 * cs * kNB) {
      const int second = q0 + cs * kNB;
      const int nc = (q0 + kNB < n ? kNB : n - q0) + (second < n ? ((second + kNB < n ? kNB : n - second)) : 0);
      if (unit)
        dev::tile_left_qt<T, true>(R + j0 + (size_t)j0 * ldr, ldr, Tm, kNB, kb, 1, nullptr, 0,
                                   R + j0 + (size_t)q0 * ldr, ldr, m - j0, nc, tile, gap);
      else
        dev::tile_left_qt<T, true>(B + (size_t)j0 * ldb, ldb, Tm, kNB, kb, 0, R + j0 + (size_t)q0 * ldr, ldr,
                                   B + (size_t)q0 * ldb, ldb, m, nc, tile, gap);
    }
  }
  csync(cs);
}

// kStage: panels factored in shared memory (dist_qr's `pan`, aliasing the
// tiled apply's scratch; vmax rows).
template <typename T, bool kStage>
__global__ void __launch_bounds__(kThreads, 2) k_elim(const ElimTask* __restrict__ tasks, const ElimOut* __restrict__ outs,
                                                   int cs, int vmax, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const ElimTask t = tasks[blockIdx.x / cs];
  T* red = sm;
  T* tmp = red + kRed;
  T* lt = tmp + kNB;
  T* vb = lt + t.n;
  T* tile = vb + vmax;
  T* pan = kStage ? tile : nullptr;
  dist_qr<T>(as<T>(t.S), t.n, nullptr, 0, t.n, t.n, 1, as<T>(t.T), as<T>(t.tau), lt, vb, red, tmp, tile, cs, status,
             pan, vmax);
  for (int o = t.out_begin; o < t.out_end; ++o) {
    const ElimOut e = outs[o];
    dist_qr<T>(as<T>(t.S), t.n, as<T>(e.B), e.m, e.m, t.n, 0, as<T>(e.T), as<T>(t.tau), lt, vb, red, tmp, tile,
               cs, status, pan, vmax);
  }
}

// kStage: panels factored in shared memory (nmax rows), as in k_elim.
template <typename T, bool kStage>
__global__ void __launch_bounds__(kThreads, 2) k_scale(const ScaleTask* __restrict__ tasks, int cs, int nmax,
                                                    int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const ScaleTask t = tasks[blockIdx.x / cs];
  T* red = sm;
  T* tmp = red + kRed;
  T* lt = tmp + kNB;
  T* vb = lt + nmax;
  T* tile = vb + nmax;
  dist_qr<T>(as<T>(t.S), t.n, nullptr, 0, t.n, t.n, 1, as<T>(t.T), as<T>(t.tau), lt, vb, red, tmp, tile, cs,
             status, kStage ? tile : nullptr, nmax);
}

// ------------------------------------------------------------ chunked applies
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_update(const UpdTask* __restrict__ tasks, const UpdOp* __restrict__ ops) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const UpdTask t = tasks[blockIdx.x];
  for (int o = t.op_begin; o < t.op_end; ++o) {
    const UpdOp op = ops[o];
    if (op.kind == 0)
      dev::mat_apply_qt<T>(as<T>(op.V), op.ldv, as<T>(op.T), op.k, as<T>(op.A) + (size_t)t.col0 * op.lda, op.lda, op.m,
                           t.ncols, sm);
    else
      dev::mat_apply_tpqt<T>(as<T>(op.V), op.ldv, as<T>(op.T), op.k, as<T>(op.A) + (size_t)t.col0 * op.lda, op.lda,
                             as<T>(op.B) + (size_t)t.col0 * op.ldb, op.ldb, op.m, t.ncols, sm);
  }
}

// row scaling: columns [lo, lo+cnt) of A <- Qs^T A
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_edge_left(const EdgeChunk* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  int cnt = t.cnt;
  if (t.limdev) {
    const int lim = *t.limdev;
    if (t.lo >= lim) return;
    cnt = min(cnt, lim - t.lo);
  }
  dev::mat_apply_qt<T>(as<T>(t.V), t.ldv, as<T>(t.T), k, as<T>(t.A) + (size_t)t.lo * t.lda, t.lda, t.m, cnt, sm);
}

// Row scaling / left compression of small blocks, one warp per chunk: m <= 32
// rows, at most 32 reflectors (one panel), columns in halves of 32.  Lane r
// holds row r of V in registers and updates row r of C; W = V^T C is formed
// with lane i as reflector i, reading column i of V and broadcast rows of C
// from the warp's shared memory; W2 = T^T W likewise (T read by its column);
// then C -= V W2 on the rows.  No CTA barrier: a CTA of kWarps warps runs
// kWarps chunks at once (the tiled kernel runs one chunk per CTA through
// about nine CTA barriers).
constexpr int kSmallRows = 32;
constexpr int kSmallLd = 36;  // shared row stride: 16-byte aligned rows
template <typename T>
constexpr size_t small_left_smem() {
  return (size_t)kWarps * 2 * kSmallRows * kSmallLd * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_edge_left_small(const EdgeChunk* __restrict__ tasks, int ntasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int kVec = 16 / (int)sizeof(T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ti = blockIdx.x * kWarps + warp;
  if (ti >= ntasks) return;
  const EdgeChunk t = tasks[ti];
  const int k = t.kdev ? *t.kdev : t.k;
  int cnt = t.cnt;
  if (t.limdev) {
    const int lim = *t.limdev;
    if (t.lo >= lim) return;
    cnt = min(cnt, lim - t.lo);
  }
  const int m = t.m;
  if (k <= 0 || cnt <= 0 || m <= 0) return;
  T* sV = reinterpret_cast<T*>(smraw) + (size_t)warp * 2 * kSmallRows * kSmallLd;  // sV[r * ld + i] = V(r, i)
  T* sC = sV + kSmallRows * kSmallLd;  // C, then W, then W2 (row-major, 32 columns)
  const T* V = as<T>(t.V);
  const T* Tm = as<T>(t.T);
  T vrow[kSmallRows];
#pragma unroll
  for (int i = 0; i < kSmallRows; ++i) {
    T v = 0.0;
    if (lane < m && i < k) v = lane == i ? (T)1.0 : (lane < i ? (T)0.0 : V[lane + (size_t)i * t.ldv]);
    vrow[i] = v;
    sV[lane * kSmallLd + i] = v;
  }
  for (int h = 0; h < cnt; h += 32) {
    const int hc = min(32, cnt - h);
    T* A = as<T>(t.A) + (size_t)(t.lo + h) * t.lda;
#pragma unroll
    for (int j = 0; j < 32; ++j) sC[lane * kSmallLd + j] = (lane < m && j < hc) ? A[lane + (size_t)j * t.lda] : (T)0.0;
    __syncwarp();
    // W(lane, j) = sum_r V(r, lane) C(r, j)
    T w[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) w[j] = 0.0;
    for (int r = 0; r < m; ++r) {
      const T vri = sV[r * kSmallLd + lane];
      const V4* cr = reinterpret_cast<const V4*>(sC + r * kSmallLd);
#pragma unroll
      for (int q = 0; q < 32 / kVec; ++q) {
        const V4 x = cr[q];
        const T* xs = reinterpret_cast<const T*>(&x);
#pragma unroll
        for (int u = 0; u < kVec; ++u) w[q * kVec + u] += vri * xs[u];
      }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j) sC[lane * kSmallLd + j] = w[j];
    __syncwarp();
    // W2(lane, j) = sum_{l <= lane} T(l, lane) W(l, j)
#pragma unroll
    for (int j = 0; j < 32; ++j) w[j] = 0.0;
#pragma unroll
    for (int l = 0; l < kSmallRows; ++l) {
      if (l < k) {
        const T tl = (l <= lane && lane < k) ? Tm[l + (size_t)lane * kNB] : (T)0.0;  // T(l, lane)
        const V4* wl = reinterpret_cast<const V4*>(sC + l * kSmallLd);
#pragma unroll
        for (int q = 0; q < 32 / kVec; ++q) {
          const V4 x = wl[q];
          const T* xs = reinterpret_cast<const T*>(&x);
#pragma unroll
          for (int u = 0; u < kVec; ++u) w[q * kVec + u] += tl * xs[u];
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j) sC[lane * kSmallLd + j] = w[j];
    __syncwarp();
    // C(lane, j) -= sum_i V(lane, i) W2(i, j)
#pragma unroll
    for (int j = 0; j < 32; ++j) w[j] = 0.0;
#pragma unroll
    for (int i = 0; i < kSmallRows; ++i) {
      if (i < k) {
        const T vi = vrow[i];
        const V4* wi = reinterpret_cast<const V4*>(sC + i * kSmallLd);
#pragma unroll
        for (int q = 0; q < 32 / kVec; ++q) {
          const V4 x = wi[q];
          const T* xs = reinterpret_cast<const T*>(&x);
#pragma unroll
          for (int u = 0; u < kVec; ++u) w[q * kVec + u] += vi * xs[u];
        }
      }
    }
    if (lane < m)
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < hc) A[lane + (size_t)j * t.lda] -= w[j];
    __syncwarp();
  }
}

// Trailing updates of small column chunks (FP32 factors): one team of 64
// threads per chunk, kTeams teams per 128-thread CTA, synchronised by their
// own named barrier.  Every op of the chunk's chain has at most 64
// reflectors and 64 rows.  The ops of one interior c (its geqrt apply, then
// its tsqrt steps) all update the same block A(c, m): per 32-column half, the
// team keeps that block in shared memory across the whole run of ops with
// the same A and brings in only each step's neighbour block B(n, m) and the
// reflector panels; every panel of an op is applied before B is written back.
// Per panel: thread r stages row r of the panel of V (registers and shared
// memory); thread t forms W(t mod 32, 16 columns) = V^T C (+ the top rows of
// A for a tsqrt step), then W2 = T^T W; thread r updates its row.
constexpr int kTeam = 64;
constexpr int kTeams = 2;  // teams per CTA
constexpr int kTeamThreads = kTeam * kTeams;
constexpr int kSmallOp = 64;  // rows, reflectors and columns of an op on the small path
// floats per team: A, B, V panel (64 x kSmallLd each), W (32 x kSmallLd), T (32 x 33)
constexpr size_t kTeamSmem = (size_t)(3 * kSmallOp + kNB) * kSmallLd + kNB * (kNB + 1);
constexpr size_t kUpdSmallSmem = kTeams * kTeamSmem * sizeof(float);

__device__ __forceinline__ void team_sync(int team) {
  asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(kTeam) : "memory");
}

// One panel (reflectors j0 .. j0 + kb) of an op on blocks in shared memory:
// kind 0: C = sA rows [j0, m) <- Q^T C (V unit lower, rows j0 ..);
// kind 1: [sA rows j0 .. j0 + kb; sB rows 0 .. m) <- Q^T [.] (V full, m rows).
__device__ __forceinline__ void team_panel(const UpdOp& op, int j0, int kb, float* sA, float* sB, float* sV,
                                           float* sW, float* sT, int team, int tl) {
  const int r0 = op.kind ? 0 : j0;
  const int nr = op.m - r0;
  float* sC = op.kind ? sB : sA + (size_t)j0 * kSmallLd;  // rows r0 .. of the block V acts on
  const float* V = as<float>(op.V);
  const float* Tm = as<float>(op.T) + (size_t)j0 * kNB;
  float vrow[kNB];
#pragma unroll
  for (int i = 0; i < kNB; ++i) {
    float v = 0.0f;
    if (tl < nr && i < kb) {
      const int r = r0 + tl;
      v = op.kind ? V[r + (size_t)(j0 + i) * op.ldv]
                  : (tl == i ? 1.0f : (tl < i ? 0.0f : V[r + (size_t)(j0 + i) * op.ldv]));
    }
    vrow[i] = v;
    sV[tl * kSmallLd + i] = v;
  }
  for (int e = tl; e < kNB * kNB; e += kTeam) {  // T transposed: sT[i * 33 + l] = T(l, i)
    const int l = e % kNB, i = e / kNB;
    sT[i * (kNB + 1) + l] = (l <= i && i < kb) ? Tm[l + (size_t)i * kNB] : 0.0f;
  }
  team_sync(team);
  const int wi = tl & 31, jc = (tl >> 5) * 16;
  float w[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) w[u] = (op.kind && wi < kb) ? sA[(j0 + wi) * kSmallLd + jc + u] : 0.0f;
  for (int r = 0; r < nr; ++r) {
    const float vri = sV[r * kSmallLd + wi];
    const float4* cr = reinterpret_cast<const float4*>(sC + r * kSmallLd + jc);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 x = cr[q];
      w[4 * q] += vri * x.x;
      w[4 * q + 1] += vri * x.y;
      w[4 * q + 2] += vri * x.z;
      w[4 * q + 3] += vri * x.w;
    }
  }
#pragma unroll
  for (int u = 0; u < 16; ++u) sW[wi * kSmallLd + jc + u] = w[u];
  team_sync(team);
#pragma unroll
  for (int u = 0; u < 16; ++u) w[u] = 0.0f;
  for (int l = 0; l < kb; ++l) {
    const float tlw = sT[wi * (kNB + 1) + l];  // T(l, wi); zero unless l <= wi < kb
    const float4* wl = reinterpret_cast<const float4*>(sW + l * kSmallLd + jc);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 x = wl[q];
      w[4 * q] += tlw * x.x;
      w[4 * q + 1] += tlw * x.y;
      w[4 * q + 2] += tlw * x.z;
      w[4 * q + 3] += tlw * x.w;
    }
  }
  team_sync(team);
#pragma unroll
  for (int u = 0; u < 16; ++u) sW[wi * kSmallLd + jc + u] = w[u];
  team_sync(team);
  if (op.kind)  // the top rows: A(j0 + i, .) -= W2(i, .)
    for (int e = tl; e < kb * 32; e += kTeam) {
      const int i = e >> 5, j = e & 31;
      sA[(j0 + i) * kSmallLd + j] -= sW[i * kSmallLd + j];
    }
  if (tl < nr) {  // C(r, .) -= V(r, :) W2
    float acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
#pragma unroll
    for (int i = 0; i < kNB; ++i) {
      if (i < kb) {
        const float vi = vrow[i];
        const float4* wr = reinterpret_cast<const float4*>(sW + i * kSmallLd);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 x = wr[q];
          acc[4 * q] += vi * x.x;
          acc[4 * q + 1] += vi * x.y;
          acc[4 * q + 2] += vi * x.z;
          acc[4 * q + 3] += vi * x.w;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) sC[tl * kSmallLd + j] -= acc[j];
  }
  team_sync(team);
}

__global__ void __launch_bounds__(kTeamThreads, 3) k_update_small(const UpdTask* __restrict__ tasks,
                                                              const UpdOp* __restrict__ ops, int ntasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int team = threadIdx.x / kTeam, tl = threadIdx.x % kTeam;
  const int ti = blockIdx.x * kTeams + team;
  if (ti >= ntasks) return;  // the whole team
  float* sA = reinterpret_cast<float*>(smraw) + (size_t)team * kTeamSmem;  // sA[r * ld + j] = A(r, h + j)
  float* sB = sA + kSmallOp * kSmallLd;                                    // sB[r * ld + j] = B(r, h + j)
  float* sV = sB + kSmallOp * kSmallLd;
  float* sW = sV + kSmallOp * kSmallLd;
  float* sT = sW + kNB * kSmallLd;
  const UpdTask t = tasks[ti];
  for (int h = 0; h < t.ncols; h += 32) {
    const int hc = min(32, t.ncols - h);
    int o = t.op_begin;
    while (o < t.op_end) {
      const double* Aid = ops[o].A;
      float* A = as<float>(ops[o].A) + (size_t)(t.col0 + h) * ops[o].lda;
      const int lda = ops[o].lda;
      const int arows = ops[o].kind ? ops[o].k : ops[o].m;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        sA[tl * kSmallLd + j] = (tl < arows && j < hc) ? A[tl + (size_t)j * lda] : 0.0f;
      team_sync(team);
      for (; o < t.op_end && ops[o].A == Aid; ++o) {
        const UpdOp op = ops[o];
        float* B = nullptr;
        if (op.kind) {
          B = as<float>(op.B) + (size_t)(t.col0 + h) * op.ldb;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            sB[tl * kSmallLd + j] = (tl < op.m && j < hc) ? B[tl + (size_t)j * op.ldb] : 0.0f;
          // made visible by the barrier inside team_panel
        }
        for (int j0 = 0; j0 < op.k; j0 += kNB) team_panel(op, j0, min(kNB, op.k - j0), sA, sB, sV, sW, sT, team, tl);
        if (op.kind && tl < op.m)
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j < hc) B[tl + (size_t)j * op.ldb] = sB[tl * kSmallLd + j];
        team_sync(team);  // sB is reused by the next step
      }
      if (tl < arows)
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (j < hc) A[tl + (size_t)j * lda] = sA[tl * kSmallLd + j];
      team_sync(team);  // sA is reused by the next group
    }
  }
}

// ------------------------------------------------------------ tensor-core applies (float factors)
// The panel loops of dev::mat_apply_qt / mat_apply_tpqt on the tensor cores
// (tc::left_qt, 3xTF32); chunks of at most 64 columns.
__device__ void tc_apply_qt(tc::Ctx& x, const float* V, int ldv, const float* Tm, int k, float* C, int ldc, int m,
                            int nc) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = min(k - j0, kNB);
    for (int c0 = 0; c0 < nc; c0 += 64)
      tc::left_qt(x, V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 1, nullptr, 0,
                  C + j0 + (size_t)c0 * ldc, ldc, m - j0, min(nc - c0, 64));
  }
}
__device__ void tc_apply_tpqt(tc::Ctx& x, const float* V, int ldv, const float* Tm, int k, float* A, int lda,
                              float* B, int ldb, int m, int nc) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = min(k - j0, kNB);
    for (int c0 = 0; c0 < nc; c0 += 64)
      tc::left_qt(x, V + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 0, A + j0 + (size_t)c0 * lda, lda,
                  B + (size_t)c0 * ldb, ldb, m, min(nc - c0, 64));
  }
}

// C (m x n) <- C Q, panels in order (dev::mat_apply_q_right), on the tensor
// cores: each panel is the left apply Q^T of the transposed chunk.  m <= 64.
__device__ void tc_apply_q_right(tc::Ctx& x, const float* V, int ldv, const float* Tm, int k, float* C, int ldc,
                                 int m, int n) {
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int kb = min(k - j0, kNB);
    tc::left_qt<true>(x, V + j0 + (size_t)j0 * ldv, ldv, Tm + (size_t)j0 * kNB, kNB, kb, 1, nullptr, 0,
                      C + (size_t)j0 * ldc, ldc, n - j0, m);
  }
}

// k_update on the tensor cores (float factors)
__global__ void __launch_bounds__(kThreads, 2) k_update_tc(const UpdTask* __restrict__ tasks,
                                                         const UpdOp* __restrict__ ops, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  tc::Ctx x = tc::begin(smraw, status);
  const UpdTask t = tasks[blockIdx.x];
  for (int o = t.op_begin; o < t.op_end; ++o) {
    const UpdOp op = ops[o];
    if (op.kind == 0)
      tc_apply_qt(x, as<float>(op.V), op.ldv, as<float>(op.T), op.k, as<float>(op.A) + (size_t)t.col0 * op.lda,
                  op.lda, op.m, t.ncols);
    else
      tc_apply_tpqt(x, as<float>(op.V), op.ldv, as<float>(op.T), op.k, as<float>(op.A) + (size_t)t.col0 * op.lda,
                    op.lda, as<float>(op.B) + (size_t)t.col0 * op.ldb, op.ldb, op.m, t.ncols);
  }
  tc::end(x);
}

// k_edge_left on the tensor cores (float factors)
__global__ void __launch_bounds__(kThreads, 2) k_edge_left_tc(const EdgeChunk* __restrict__ tasks, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  tc::Ctx x = tc::begin(smraw, status);
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  int cnt = t.cnt;
  if (t.limdev) cnt = min(cnt, *t.limdev - t.lo);
  if (cnt > 0) tc_apply_qt(x, as<float>(t.V), t.ldv, as<float>(t.T), k, as<float>(t.A) + (size_t)t.lo * t.lda, t.lda,
                           t.m, cnt);
  tc::end(x);
}

// the operand-layout diagnostic of tc_apply.cuh (one CTA)
__global__ void __launch_bounds__(kThreads, 1) k_tc_probe(const float* C, const float* V, const float* W2, int m,
                                                       int flags, float* out1, float* out2, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  tc::Ctx x = tc::begin(smraw, status);
  tc::probe(x, C, V, W2, m, flags, out1, out2);
  tc::end(x);
}

// k_edge_right on the tensor cores (float factors): rows [lo, lo+cnt) of A <- A Q
__global__ void __launch_bounds__(kThreads, 2) k_edge_right_tc(const EdgeChunk* __restrict__ tasks, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  tc::Ctx x = tc::begin(smraw, status);
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  if (t.cnt > 0) tc_apply_q_right(x, as<float>(t.V), t.ldv, as<float>(t.T), k, as<float>(t.A) + t.lo, t.lda, t.cnt, t.nc);
  tc::end(x);
}

// column scaling: rows [lo, lo+cnt) of A <- A R^{-1}
template <typename T>
__global__ void __launch_bounds__(kThreads) k_edge_trsm(const EdgeChunk* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const EdgeChunk t = tasks[blockIdx.x];
  dev::tile_trsm_right_upper<T>(as<T>(t.V), t.ldv, as<T>(t.A) + t.lo, t.lda, t.cnt, t.nc, sm);
}

// Column scaling of small blocks (FP32, at most 32 columns, chunks of at most
// 64 rows), one warp per chunk: lane r holds rows r and r + 32 of C, R sits
// in the warp's shared memory, and the columns are solved in order,
// c_j = (c_j - sum_{i<j} c_i R(i, j)) / R(j, j), from broadcast reads; no
// barrier beyond the warp's.
constexpr int kTrsmLd = 33;
__global__ void __launch_bounds__(kThreads, 2) k_edge_trsm_small(const EdgeChunk* __restrict__ tasks, int ntasks) {
  __shared__ float sRall[kWarps][32 * kTrsmLd];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ti = blockIdx.x * kWarps + warp;
  if (ti >= ntasks) return;
  const EdgeChunk t = tasks[ti];
  const int n = t.nc, m = t.cnt;
  float* sR = sRall[warp];  // sR[i * ld + j] = R(i, j)
  const float* R = as<float>(t.V);
#pragma unroll
  for (int j = 0; j < 32; ++j) sR[lane * kTrsmLd + j] = (lane < n && j < n && lane <= j) ? R[lane + (size_t)j * t.ldv] : 0.0f;
  float* C = as<float>(t.A) + t.lo;
  float c0[32], c1[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    c0[j] = (j < n && lane < m) ? C[lane + (size_t)j * t.lda] : 0.0f;
    c1[j] = (j < n && lane + 32 < m) ? C[lane + 32 + (size_t)j * t.lda] : 0.0f;
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < n) {
      float s0 = c0[j], s1 = c1[j];
#pragma unroll
      for (int i = 0; i < j; ++i) {
        const float rij = sR[i * kTrsmLd + j];
        s0 -= c0[i] * rij;
        s1 -= c1[i] * rij;
      }
      const float d = sR[j * kTrsmLd + j];
      c0[j] = s0 / d;
      c1[j] = s1 / d;
    }
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < n && lane < m) C[lane + (size_t)j * t.lda] = c0[j];
    if (j < n && lane + 32 < m) C[lane + 32 + (size_t)j * t.lda] = c1[j];
  }
}

// Right compression of small blocks (FP32, at most 32 columns, chunks of at
// most 64 rows), one warp per chunk: C <- C (I - V T V^T), V unit lower
// (n x k).  Every row is independent: lane r takes rows r and r + 32 in turn
// and forms W = C(r, :) V, W2 = W T, C(r, :) -= W2 V^T with V and T read as
// 16-byte broadcasts from the warp's shared memory.
constexpr int kRightLd = 36;
constexpr size_t kRightSmallSmem = (size_t)kWarps * 2 * 32 * kRightLd * sizeof(float);
__global__ void __launch_bounds__(kThreads, 2) k_edge_right_small(const EdgeChunk* __restrict__ tasks, int ntasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ti = blockIdx.x * kWarps + warp;
  if (ti >= ntasks) return;
  const EdgeChunk t = tasks[ti];
  const int n = t.nc, m = t.cnt;
  const int k = t.kdev ? *t.kdev : t.k;
  if (k <= 0 || n <= 0 || m <= 0) return;
  float* sV = reinterpret_cast<float*>(smraw) + (size_t)warp * 2 * 32 * kRightLd;  // sV[j * ld + i] = V(j, i)
  float* sT = sV + 32 * kRightLd;                                                   // sT[l * ld + i] = T(l, i)
  const float* V = as<float>(t.V);
  const float* Tm = as<float>(t.T);
  for (int i = 0; i < 32; ++i) {
    float v = 0.0f;
    if (lane < n && i < k) v = lane == i ? 1.0f : (lane < i ? 0.0f : V[lane + (size_t)i * t.ldv]);
    sV[lane * kRightLd + i] = v;
    sT[lane * kRightLd + i] = (lane <= i && i < k) ? Tm[lane + (size_t)i * kNB] : 0.0f;
  }
  __syncwarp();
  float* C = as<float>(t.A) + t.lo;
  for (int half = 0; half < 2; ++half) {
    if (32 * half >= m) break;  // uniform over the warp
    const int r = lane + 32 * half;
    const bool live = r < m;
    float w[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) w[i] = 0.0f;
    for (int j = 0; j < n; ++j) {  // W = C(r, :) V
      const float cj = live ? C[r + (size_t)j * t.lda] : 0.0f;
      const float4* vr = reinterpret_cast<const float4*>(sV + j * kRightLd);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 x = vr[q];
        w[4 * q] += cj * x.x;
        w[4 * q + 1] += cj * x.y;
        w[4 * q + 2] += cj * x.z;
        w[4 * q + 3] += cj * x.w;
      }
    }
    // W2 = W T in place, columns from the last: W2(i) uses W(l) for l <= i only
#pragma unroll
    for (int i = 31; i >= 0; --i) {
      float sacc = 0.0f;
#pragma unroll
      for (int l = 0; l <= i; ++l) sacc += w[l] * sT[l * kRightLd + i];
      w[i] = sacc;
    }
    for (int j = 0; j < n; ++j) {  // C(r, j) -= W2 V(j, :)^T
      const float4* vr = reinterpret_cast<const float4*>(sV + j * kRightLd);
      float u = 0.0f;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 x = vr[q];
        u += (w[4 * q] * x.x + w[4 * q + 1] * x.y) + (w[4 * q + 2] * x.z + w[4 * q + 3] * x.w);
      }
      if (live) C[r + (size_t)j * t.lda] -= u;
    }
  }
}

// right compression: rows [lo, lo+cnt) of A <- A Q
template <typename T>
__global__ void __launch_bounds__(kThreads) k_edge_right(const EdgeChunk* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  dev::mat_apply_q_right<T>(as<T>(t.V), t.ldv, as<T>(t.T), k, as<T>(t.A) + t.lo, t.lda, t.cnt, t.nc, sm);
}

// ------------------------------------------------------------ RRQR
// Truncated column-pivoted QR of the compression matrix C (m x w) of one
// interface: LAPACK geqp3 stopped at the first i >= 1 with
// |R(i,i)| / |R(0,0)| < tol (ptree.cpp:373-439, util.cpp:830-851).
//
// The pivot sequence follows dlaqp2 step by step: the pivot is the first
// POSITION (column order after dlaqp2's swaps) whose partial norm is within
// pivot_rtol of the largest, partial norms are downdated with row i of R and
// recomputed when the downdate loses accuracy (tol3z = sqrt(eps)).  C itself
// is never rewritten: row i of R is q_i^T C, where q_i is column i of the
// orthonormal factor, obtained by Gram-Schmidt with reorthogonalisation (CGS2)
// of the pivot column against q_0..q_{i-1}; |R(i,i)| is the norm left after
// the projection.  Each step therefore READS C once (one GEMV) instead of
// reading and rewriting the trailing matrix.  With the pivots known, the
// Householder reflectors are those of an unpivoted QR of the selected
// columns in pivot order (the first k steps of a pivoted QR act on exactly
// those columns), computed by dist_qr into V, tau and the panel factors T.
//
// A task runs on one thread-block cluster.  C is stored transposed (Ct, w x m)
// so the GEMV is coalesced with one column per thread; columns are dealt to
// the CTAs in contiguous ranges and rows of the basis in contiguous slices.
// Five cluster barriers per step publish the two pivot reductions, the two
// Gram-Schmidt projections and the new basis vector; every published value
// is reduced over the CTAs in rank order, so all CTAs take identical
// decisions.

// Gathers the compression matrix of every task, transposed: C column c0 + jj
// is row jj of an out-block A(n,p) or column jj of an in-block A(p,m).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_rrqr_assemble(const RrqrSrc* __restrict__ srcs) {
  __shared__ double tile[32][33];
  const RrqrSrc s = srcs[blockIdx.x];
  const T* SA = as<T>(s.A);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* dst = s.Ct + s.c0;
  if (s.transpose) {
    for (int r = warp; r < s.cols; r += kWarps)
      for (int jj = lane; jj < s.rows; jj += 32) dst[(size_t)r * s.w + jj] = (double)SA[jj + (size_t)r * s.lda];
    return;
  }
  for (int j0 = 0; j0 < s.cols; j0 += 32)
    for (int r0 = 0; r0 < s.rows; r0 += 32) {
      for (int q = warp; q < 32; q += kWarps) {
        const int r = r0 + lane, j = j0 + q;
        tile[q][lane] = (r < s.rows && j < s.cols) ? (double)SA[r + (size_t)j * s.lda] : 0.0;
      }
      __syncthreads();
      for (int q = warp; q < 32; q += kWarps) {
        const int r = r0 + q, j = j0 + lane;
        if (r < s.rows && j < s.cols) dst[(size_t)r * s.w + j] = tile[lane][q];
      }
      __syncthreads();
    }
}

// Column dots over the CTA's own columns [ja, ja + nloc) of C:
// fin(jl, sum_r C(r, ja + jl) * x(r)) (kSq: x = the column itself) for every
// jl with act(jl).  A lane reads two adjacent columns per 16-byte load, a warp
// 64 consecutive columns (512 bytes of a row of Ct) per load instruction and
// four such segments at once; the warps split into RG row groups (rows
// r = rg mod RG, about 16 rows each) times kWarps / RG column groups.  The
// loads of kRows rows are issued before their products, so every thread
// keeps sixteen 16-byte loads in flight (64 KB per CTA).  Partial sums meet in `gp` (8 * kThreads doubles)
// and are added in row-group order.
constexpr int kRows = 4;  // rows of loads issued together in col_dots

template <bool kSq, bool kShared, typename Act, typename Fin>
__device__ __forceinline__ void col_dots(const double* __restrict__ Ct, int ldw, int m, int ja, int nloc,
                                         const double* x, double* gp, Act act, Fin fin) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int RG = 1;
  while (RG < kWarps && RG * 16 < m) RG <<= 1;
  const int CG = kWarps / RG;
  const int rg = warp % RG, cgp = warp / RG;
  for (int base = 0; base < nloc; base += 256 * CG) {
    const int cb = base + 256 * cgp + 2 * lane;
    bool a[4][2], l[4];
    double acc[4][2];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int jl = cb + 64 * u + e;
        a[u][e] = jl < nloc && act(jl);
        acc[u][e] = 0.0;
      }
      l[u] = a[u][0] || a[u][1];
    }
    const double* col = Ct + ja + cb;
    for (int r0 = rg; r0 < m; r0 += kRows * RG) {
      double2 v[kRows][4];
#pragma unroll
      for (int k = 0; k < kRows; ++k) {
        const int r = r0 + k * RG;
        const double2* row = reinterpret_cast<const double2*>(col + (size_t)r * ldw);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[k][u] = (r < m && l[u]) ? (kShared ? row[32 * u] : __ldg(row + 32 * u)) : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int k = 0; k < kRows; ++k) {
        const int r = r0 + k * RG;
        const double xr = kSq ? 0.0 : (r < m ? x[r] : 0.0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          acc[u][0] += kSq ? v[k][u].x * v[k][u].x : v[k][u].x * xr;
          acc[u][1] += kSq ? v[k][u].y * v[k][u].y : v[k][u].y * xr;
        }
      }
    }
    if (RG > 1) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) gp[(size_t)((warp * 4 + u) * 2 + e) * 32 + lane] = acc[u][e];
      __syncthreads();
      if (rg == 0) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int e = 0; e < 2; ++e)
            for (int q = 1; q < RG; ++q) acc[u][e] += gp[(size_t)(((warp + q) * 4 + u) * 2 + e) * 32 + lane];
      }
      __syncthreads();
    }
    if (rg == 0) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (a[u][e]) fin(cb + 64 * u + e, acc[u][e]);
    }
  }
  __syncthreads();
}

// Sum over the cluster's CTAs, in rank order, of the value at shared address
// x in each CTA; the remote loads are issued together.
__device__ __forceinline__ double cluster_sum(double* x, int cs) {
  if (cs == 1) return *x;
  cg::cluster_group cl = cg::this_cluster();
  double v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = q < cs ? *cl.map_shared_rank(x, q) : 0.0;
  double sum = v[0];
#pragma unroll
  for (int q = 1; q < 16; ++q)
    if (q < cs) sum += v[q];
  return sum;
}

// (position, column) with the smallest position across the warp
__device__ __forceinline__ void warp_min_pos(int& bp, int& bc) {
  for (int o = 16; o > 0; o >>= 1) {
    const int op = __shfl_xor_sync(0xffffffffu, bp, o);
    const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
    if (op < bp || (op == bp && oc < bc)) {
      bp = op;
      bc = oc;
    }
  }
}

// Partial-sum scratch of k_rrqr; vn1, vn2 and it also hold the tiled-apply
// scratch of the final QR (dev::kTileSmem doubles).
__host__ __device__ constexpr int rrqr_gp_doubles(int nlmax) {
  return 8 * kThreads > dev::kTileSmem - 2 * nlmax ? 8 * kThreads : dev::kTileSmem - 2 * nlmax;
}

// Shared-memory carve of k_rrqr (doubles, then ints); rrqr_smem mirrors it.
struct RrqrSmem {
  double *red, *tmp, *spa, *spb, *s1, *s2, *sq, *cv, *qf, *vn1, *vn2, *gp;
  int *pos, *flg;
  __device__ RrqrSmem(double* sm, int mmax, int kmax, int nlmax, int rcmax) {
    red = sm;
    tmp = red + kRed;
    spa = tmp + kNB;
    spb = spa + kmax + 1;
    s1 = spb + kmax + 1;
    s2 = s1 + kmax + 1;
    sq = s2 + kmax + 1;
    cv = sq + rcmax;
    qf = cv + rcmax;
    vn1 = qf + mmax;
    vn2 = vn1 + nlmax;
    gp = vn2 + nlmax;
    pos = reinterpret_cast<int*>(gp + rrqr_gp_doubles(nlmax));
    flg = pos + nlmax;
  }
};

// First own active position (>= i) whose partial norm is >= thr: position,
// global column and norm in s_k[0][0], s_k[1][0], s_xv[0] (INT_MAX, -1, -1 if none).
__device__ __forceinline__ void own_first(const RrqrSmem& S, int nloc, int ja, int i, double thr, int (*s_k)[kWarps],
                                          double* s_xv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int bp = 0x7fffffff, bc = -1;
  double bvn = -1.0;
  for (int jl = threadIdx.x; jl < nloc; jl += kThreads) {
    const int p = S.pos[jl];
    if (p >= i && p < bp && S.vn1[jl] >= thr) {
      bp = p;
      bc = ja + jl;
      bvn = S.vn1[jl];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const int op = __shfl_xor_sync(0xffffffffu, bp, o);
    const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
    const double ov = __shfl_xor_sync(0xffffffffu, bvn, o);
    if (op < bp) {
      bp = op;
      bc = oc;
      bvn = ov;
    }
  }
  __syncthreads();  // s_k / s_xv free (an earlier reader may still hold them)
  if (lane == 0) {
    s_k[0][warp] = bp;
    s_k[1][warp] = bc;
    s_xv[warp] = bvn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < kWarps; ++q)
      if (s_k[0][q] < s_k[0][0]) {
        s_k[0][0] = s_k[0][q];
        s_k[1][0] = s_k[1][q];
        s_xv[0] = s_xv[q];
      }
  }
  __syncthreads();
}

template <bool kSmemC>
__global__ void __launch_bounds__(kThreads, 2) k_rrqr(const RrqrTask* __restrict__ tasks, double tol,
                                                      double pivot_rtol, int cs, int mmax, int kmax, int nlmax,
                                                      int rcmax) {
  extern __shared__ double sm[];
  __shared__ double s_x[kWarps];
  __shared__ int s_k[2][kWarps];
  __shared__ double s_xv[kWarps];
  // published by step parity: own largest partial norm M, the first own
  // position P whose norm is within pivot_rtol of M, its column and norm;
  // P2/C2 for the exact second round
  __shared__ double s_pm[2], s_pv[2];
  __shared__ int s_pp[2], s_pc[2], s_p2[2], s_c2[2];
  __shared__ int s_piv[3];
  __shared__ double s_thr;
  __shared__ int s_nflag;
  RrqrSmem S(sm, mmax, kmax, nlmax, rcmax);
  const RrqrTask t = tasks[blockIdx.x / cs];
  const int rank = crank(cs);
  const int m = t.m, w = t.w, ldq = t.ldq;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double* __restrict__ Ct = t.C;
  const int ldw = t.ldw;
  double* Qt = t.Q;

  // own columns [ja, jb) and own rows [ra, rb)
  const int wc = rrqr_cols_per_cta(w, cs, kSmemC);
  const int ja = min(w, rank * wc), jb = min(w, ja + wc), nloc = jb - ja;
  const int rc = (m + cs - 1) / cs;
  const int ra = min(m, rank * rc), rb = min(m, ra + rc);
  const int kmin = min(m, w);
  // remote shared memory of cluster rank q (the CTA's own for cs == 1)
  auto remote = [&](double* p, int q) -> double {
    if (cs == 1) return *p;
    return *cg::this_cluster().map_shared_rank(p, q);
  };
  auto remote_i = [&](int* p, int q) -> int {
    if (cs == 1) return *p;
    return *cg::this_cluster().map_shared_rank(p, q);
  };
  // initial norms, positions
  // kSmemC: the CTA's column block of C (m x nlp, nlp = nloc rounded up to
  // even, the pad column zero) is held in shared memory after S's arrays and
  // every pivot step reads it there
  const int nlp = (nloc + 1) & ~1;
  double* sC = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(S.flg + nlmax) + 15) & ~(uintptr_t)15);
  if (kSmemC) {
    for (size_t e = threadIdx.x; e < (size_t)m * nlp; e += kThreads) {
      const int r = (int)(e / nlp), jl = (int)(e % nlp);
      sC[e] = jl < nloc ? __ldg(Ct + (size_t)r * ldw + ja + jl) : 0.0;
    }
    __syncthreads();
  }
  const double* Cb = kSmemC ? sC : Ct + ja;
  const int ldb = kSmemC ? nlp : ldw;
  col_dots<true, kSmemC>(Cb, ldb, m, 0, nloc, nullptr, S.gp, [](int) { return true; }, [&](int jl, double ss) {
    const double v = sqrt(ss);
    S.vn1[jl] = v;
    S.vn2[jl] = v;
    S.pos[jl] = ja + jl;
    t.colat[ja + jl] = ja + jl;
  });
  __threadfence();
  csync(cs);
  const double tol3z = sqrt(1.1102230246251565e-16);
  double r00 = 0.0;
  int rk = kmin, nrecomp = 0;
  long long ph[4] = {0, 0, 0, 0};  // cycles: pivot choice, projections, basis vector, row of R
  long long tc = clock64();
  auto lap = [&](int k) {
    const long long now = clock64();
    ph[k] += now - tc;
    tc = now;
  };
  for (int i = 0; i < kmin; ++i) {
    const int par = i & 1;
    // (a) own largest partial norm M over active columns (position >= i)
    double bv = -1.0;
    for (int jl = threadIdx.x; jl < nloc; jl += kThreads)
      if (S.pos[jl] >= i) bv = fmax(bv, S.vn1[jl]);
    for (int o = 16; o > 0; o >>= 1) bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, o));
    if (lane == 0) s_x[warp] = bv;
    __syncthreads();
    double mloc = s_x[0];
    for (int q = 1; q < kWarps; ++q) mloc = fmax(mloc, s_x[q]);
    // (b) first own position within pivot_rtol of M, published with M
    own_first(S, nloc, ja, i, mloc * (1.0 - pivot_rtol), s_k, s_xv);
    if (threadIdx.x == 0) {
      s_pm[par] = mloc;
      s_pp[par] = s_k[0][0];
      s_pc[par] = s_k[1][0];
      s_pv[par] = s_xv[0];
    }
    csync(cs);
    // the pivot: the first position within pivot_rtol of the cluster's largest
    // norm.  A CTA's published position is exact unless its own maximum is
    // within pivot_rtol of the largest but the published column is not: then
    // a second round at the cluster's threshold decides.
    if (warp == 0) {
      double M = -1.0, V = -1.0;
      int P = 0x7fffffff, Cc = -1;
      if (lane < cs) {
        M = remote(&s_pm[par], lane);
        V = remote(&s_pv[par], lane);
        P = remote_i(&s_pp[par], lane);
        Cc = remote_i(&s_pc[par], lane);
      }
      double gm = M;
      for (int o = 16; o > 0; o >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, o));
      const double thr = gm * (1.0 - pivot_rtol);
      const bool amb = lane < cs && M >= thr && !(V >= thr);
      int bp = (lane < cs && M >= thr && V >= thr) ? P : 0x7fffffff, bc = bp != 0x7fffffff ? Cc : -1;
      warp_min_pos(bp, bc);
      const bool any_amb = __any_sync(0xffffffffu, amb);
      if (lane == 0) {
        s_piv[0] = bp;
        s_piv[1] = bc;
        s_piv[2] = any_amb ? 1 : 0;
        s_thr = thr;
      }
    }
    __syncthreads();
    int ppos = s_piv[0], pcol = s_piv[1];
    if (s_piv[2]) {
      own_first(S, nloc, ja, i, s_thr, s_k, s_xv);
      if (threadIdx.x == 0) {
        s_p2[par] = s_k[0][0];
        s_c2[par] = s_k[1][0];
      }
      csync(cs);
      if (warp == 0) {
        int bp = 0x7fffffff, bc = -1;
        if (lane < cs) {
          bp = remote_i(&s_p2[par], lane);
          bc = remote_i(&s_c2[par], lane);
        }
        warp_min_pos(bp, bc);
        if (lane == 0) {
          s_piv[0] = bp;
          s_piv[1] = bc;
        }
      }
      __syncthreads();
      ppos = s_piv[0];
      pcol = s_piv[1];
    }
    const int cur = __ldcg(t.colat + i);  // column now at position i
    if (pcol < 0) {  // no finite maximum (NaN norms): keep the column at position i
      ppos = i;
      pcol = cur;
    }
    lap(0);
    // (c) projection s = Q^T c of the pivot column on q_0..q_{i-1} and ||c||^2,
    // partial sums over own rows published together
    for (int r = ra + threadIdx.x; r < rb; r += kThreads) S.cv[r - ra] = __ldg(Ct + (size_t)r * ldw + pcol);
    __syncthreads();
    for (int l = threadIdx.x; l < i; l += kThreads) {
      double acc = 0.0;
      for (int r = ra; r < rb; ++r) acc += Qt[(size_t)r * ldq + l] * S.cv[r - ra];
      S.spa[l] = acc;
    }
    {
      double cc = 0.0;
      for (int r = ra + threadIdx.x; r < rb; r += kThreads) cc += S.cv[r - ra] * S.cv[r - ra];
      cc = dev::cta_sum(cc, S.red);
      if (threadIdx.x == 0) S.spa[kmax] = cc;
    }
    csync(cs);
    double ss = 0.0;
    for (int l = threadIdx.x; l < i; l += kThreads) {
      const double v = cluster_sum(S.spa + l, cs);
      S.s1[l] = v;
      ss += v * v;
    }
    ss = dev::cta_sum(ss, S.red);
    const double cc = cluster_sum(S.spa + kmax, cs);
    // |R(i,i)|^2 = ||c||^2 - ||s||^2 while that loses at most 1e-10 relative
    // accuracy; otherwise a second, explicit projection pass (CGS2)
    double nrm2 = cc - ss;
    const double* proj = S.s1;
    __syncthreads();
    for (int r = ra + warp; r < rb; r += kWarps) {
      const double* qr = Qt + (size_t)r * ldq;
      double d = 0.0;
      for (int l = lane; l < i; l += 32) d += qr[l] * S.s1[l];
      d = dev::warp_sum(d);
      if (lane == 0) S.cv[r - ra] -= d;
    }
    if (!(nrm2 >= 1e-6 * cc)) {
      __syncthreads();
      for (int l = threadIdx.x; l < i; l += kThreads) {
        double acc = 0.0;
        for (int r = ra; r < rb; ++r) acc += Qt[(size_t)r * ldq + l] * S.cv[r - ra];
        S.spb[l] = acc;
      }
      {
        double nn = 0.0;
        for (int r = ra + threadIdx.x; r < rb; r += kThreads) nn += S.cv[r - ra] * S.cv[r - ra];
        nn = dev::cta_sum(nn, S.red);
        if (threadIdx.x == 0) S.spb[kmax] = nn;
      }
      csync(cs);
      double s2s = 0.0;
      for (int l = threadIdx.x; l < i; l += kThreads) {
        const double v = cluster_sum(S.spb + l, cs);
        S.s2[l] = v;
        s2s += v * v;
      }
      s2s = dev::cta_sum(s2s, S.red);
      nrm2 = cluster_sum(S.spb + kmax, cs) - s2s;
      proj = S.s2;
    }
    const double nrm = sqrt(fmax(nrm2, 0.0));  // |R(i,i)|
    lap(1);
    if (i == 0) {
      r00 = nrm;
    } else if (!(nrm / r00 >= tol)) {
      rk = i;
      break;
    }
    // (d) every CTA has read colat[i]; book the swap, update own positions
    if (pcol >= ja && pcol < jb && threadIdx.x == 0) {
      t.colat[ppos] = cur;
      t.colat[i] = pcol;
      __threadfence();
    }
    for (int jl = threadIdx.x; jl < nloc; jl += kThreads) {
      const int gc = ja + jl;
      if (gc == pcol) S.pos[jl] = i;
      else if (gc == cur) S.pos[jl] = ppos;
    }
    // q_i = (c - Q s [- Q s2]) / |R(i,i)| on own rows, then gathered whole
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    const bool second = proj == S.s2;
    for (int r = ra + warp; r < rb; r += kWarps) {
      double* qr = Qt + (size_t)r * ldq;
      double d = 0.0;
      if (second)
        for (int l = lane; l < i; l += 32) d += qr[l] * S.s2[l];
      d = dev::warp_sum(d);
      if (lane == 0) {
        const double v = (S.cv[r - ra] - d) * inv;
        S.sq[r - ra] = v;
        qr[i] = v;
        t.Qc[r + (size_t)i * m] = v;
      }
    }
    __threadfence();
    csync(cs);
    for (int r = threadIdx.x; r < m; r += kThreads) {
      const int q = r / rc;
      S.qf[r] = remote(S.sq + (r - q * rc), q);
    }
    if (threadIdx.x == 0) s_nflag = 0;
    __syncthreads();
    lap(2);
    // (e) row i of R over own active columns (kept in F for recomputations);
    // dlaqp2 downdate of the partial norms
    double* Fi = t.F + (size_t)i * w + ja;
    col_dots<false, kSmemC>(Cb, ldb, m, 0, nloc, S.qf, S.gp, [&](int jl) { return S.pos[jl] > i; },
                    [&](int jl, double rij) {
                      Fi[jl] = rij;
                      const double v1 = S.vn1[jl];
                      if (v1 == 0.0) return;
                      double temp = fabs(rij) / v1;
                      temp = 1.0 - temp * temp;
                      temp = temp < 0.0 ? 0.0 : temp;
                      const double qq = v1 / S.vn2[jl];
                      if (temp * qq * qq <= tol3z) S.flg[atomicAdd(&s_nflag, 1)] = jl;
                      else S.vn1[jl] = v1 * sqrt(temp);
                    });
    // recomputed partial norms ||c_j - Q(:, 0:i) R(0:i, j)||, one warp per column
    const int nf = s_nflag;
    nrecomp += nf;
    for (int f = warp; f < nf; f += kWarps) {
      const int jl = S.flg[f], j = ja + jl;
      double res = 0.0;
      if (i + 1 < m) {
        for (int r = lane; r < m; r += 32) {
          double x[4] = {0.0, 0.0, 0.0, 0.0};
          int l = 0;
          for (; l + 8 <= i + 1; l += 8) {
            double qv[8], fv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              qv[u] = __ldcg(t.Qc + (size_t)(l + u) * m + r);
              fv[u] = t.F[(size_t)(l + u) * w + j];
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) x[u & 3] += qv[u] * fv[u];
          }
          for (; l <= i; ++l) x[0] += __ldcg(t.Qc + (size_t)l * m + r) * t.F[(size_t)l * w + j];
          const double e = __ldg(Ct + (size_t)r * ldw + j) - ((x[0] + x[1]) + (x[2] + x[3]));
          res += e * e;
        }
        res = dev::warp_sum(res);
      }
      if (lane == 0) {
        S.vn1[jl] = sqrt(res);
        S.vn2[jl] = sqrt(res);
      }
    }
    __syncthreads();
    lap(3);
  }
  csync(cs);  // no CTA reads another's shared memory past this point
  if (rank == 0 && threadIdx.x == 0 && t.stats) {
    t.stats[0] = nrecomp;
    t.stats[1] = rk;
    for (int k = 0; k < 4; ++k) t.stats[2 + k] = (int)(ph[k] >> 10);
    t.stats[7] = 0;
  }
  const long long tq = clock64();
  // Householder QR of the selected columns C(:, colat[0:rk]) into V
  for (int l = warp; l < rk; l += kWarps) {
    if (!owns(l, rank, cs)) continue;
    const int c = __ldcg(t.colat + l);
    for (int r = lane; r < m; r += 32) t.V[r + (size_t)l * m] = __ldg(Ct + (size_t)r * ldw + c);
  }
  __syncthreads();
  dist_qr<double>(t.V, m, nullptr, 0, m, rk, 1, t.T, t.tau, S.s1, S.qf, S.red, S.tmp, S.vn1, cs);
  if (rank == 0 && threadIdx.x == 0) {
    *t.rank = rk;
    if (t.stats) t.stats[6] = (int)((clock64() - tq) >> 10);
  }
}

// Householder QR of the selected columns C(:, colat[0:rank]) of a row-major C
// (the pivot order fixed beforehand) into V / T / tau, then the orthonormal
// basis Qc = C_sel R^{-1} (column-major, ld m) over the cluster's row blocks:
// tiles of rt rows, 32-column blocks of R, a blocked update from the solved
// columns and a triangular solve on the diagonal block.
// kStage: the QR's panels are factored in shared memory (dist_qr's `pan`,
// aliasing the basis tiles; mmax rows).
template <bool kStage>
__global__ void __launch_bounds__(kThreads, 2) k_selected_qr(const RrqrTask* __restrict__ tasks, int cs, int mmax,
                                                          int nmax, int rt) {
  extern __shared__ double sm[];
  const RrqrTask t = tasks[blockIdx.x / cs];
  const int rank = crank(cs);
  const int m = t.m, ldw = t.ldw;
  const int rk = __ldcg(t.rank);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* red = sm;
  double* tmp = red + kRed;
  double* lt = tmp + kNB;
  double* vb = lt + nmax;
  const int ldq = nmax + 1;
  double* Qt = vb + mmax;      // rt x ldq: rows of the basis being solved (first the QR's tile scratch)
  double* Rb = Qt + (size_t)rt * ldq;  // 32 x 33 block of R
  const double* __restrict__ C = t.C;
  for (int l = warp; l < rk; l += kWarps) {
    if (!owns(l, rank, cs)) continue;
    const int c = __ldg(t.colat + l);
    for (int r = lane; r < m; r += 32) t.V[r + (size_t)l * m] = __ldg(C + (size_t)r * ldw + c);
  }
  __syncthreads();
  dist_qr<double>(t.V, m, nullptr, 0, m, rk, 1, t.T, t.tau, lt, vb, red, tmp, Qt, cs, nullptr,
                  kStage ? Qt : nullptr, mmax);
  // R(l, j) = V[l + j m] for l <= j, written by the owners of column j
  auto R = [&](int l, int j) { return __ldcg(t.V + l + (size_t)j * m); };
  const int rc = (m + cs - 1) / cs;
  const int ra = min(m, rank * rc), rb = min(m, ra + rc);
  for (int r0 = ra; r0 < rb; r0 += rt) {
    const int nr = min(rt, rb - r0);
    for (int e = threadIdx.x; e < nr * rk; e += kThreads) {
      const int rr = e / rk, l = e % rk;
      Qt[rr * ldq + l] = __ldg(C + (size_t)(r0 + rr) * ldw + __ldg(t.colat + l));
    }
    __syncthreads();
    for (int j0 = 0; j0 < rk; j0 += 32) {
      const int jb = min(32, rk - j0);
      // Q(:, j0:j0+jb) = X - Q(:, 0:j0) R(0:j0, j0:j0+jb), outputs (o / 32, o % 32)
      double acc[(32 * 32 + kThreads - 1) / kThreads] = {};
      for (int l0 = 0; l0 < j0; l0 += 32) {
        for (int e = threadIdx.x; e < 32 * 32; e += kThreads) {
          const int jj = e >> 5, ll = e & 31;
          Rb[ll * 33 + jj] = jj < jb ? R(l0 + ll, j0 + jj) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < (32 * 32 + kThreads - 1) / kThreads; ++u) {
          const int o = threadIdx.x + u * kThreads, rr = o >> 5, jj = o & 31;
          if (rr < nr) {
            const double* q = Qt + rr * ldq + l0;
            double a = 0.0;
#pragma unroll 8
            for (int ll = 0; ll < 32; ++ll) a += q[ll] * Rb[ll * 33 + jj];
            acc[u] += a;
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int u = 0; u < (32 * 32 + kThreads - 1) / kThreads; ++u) {
        const int o = threadIdx.x + u * kThreads, rr = o >> 5, jj = o & 31;
        if (rr < nr && jj < jb) Qt[rr * ldq + j0 + jj] -= acc[u];
      }
      for (int e = threadIdx.x; e < 32 * 32; e += kThreads) {
        const int jj = e >> 5, ll = e & 31;
        Rb[ll * 33 + jj] = (jj < jb && ll <= jj) ? R(j0 + ll, j0 + jj) : 0.0;
      }
      __syncthreads();
      // triangular solve on the diagonal block, one thread per row
      for (int rr = threadIdx.x; rr < nr; rr += kThreads) {
        double* q = Qt + rr * ldq + j0;
        for (int jj = 0; jj < jb; ++jj) {
          double x = q[jj];
          for (int ll = 0; ll < jj; ++ll) x -= q[ll] * Rb[ll * 33 + jj];
          const double dgn = Rb[jj * 33 + jj];
          q[jj] = dgn != 0.0 ? x / dgn : 0.0;
        }
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < nr * rk; e += kThreads) {
      const int l = e / nr, rr = e % nr;
      t.Qc[(r0 + rr) + (size_t)l * m] = Qt[rr * ldq + l];
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ merge
template <typename T>
__global__ void k_merge(const MergeTask* __restrict__ tasks) {
  const MergeTask t = tasks[blockIdx.x];
  const int total = t.rows * t.cols;
  const T* src = as<T>(t.src);
  T* dst = as<T>(t.dst);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int i = idx % t.rows, j = t.c0 + idx / t.rows;
    const T v = t.identity ? (i == j ? (T)1 : (T)0) : src[i + (size_t)j * t.ld_src];
    dst[(t.roff + i) + (size_t)(t.coff + j) * t.ld_dst] = v;
  }
}

// ------------------------------------------------------------ solve
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Forward elimination sweep of one level.  Interiors are taken in ascending
// order through a ticket; a chain step on neighbour n waits (bounded) until
// every interior ordered before this one in n's transform order has applied
// its step, so the order matches the factorization (order_of_trans).  Waits
// only target lower tickets, which are held by running CTAs, so the sweep
// cannot deadlock; a wait that exceeds `spin_limit` cycles sets *status = 2.
// kStaged: the interior's own reflectors stream through shared memory
// (dev::vec_apply_staged), for levels with large interiors.
template <typename T, bool kStaged>
__global__ void __launch_bounds__(kThreads, 2) k_fwd_elim(const FwdElimTask* __restrict__ tasks,
                                                       const FwdOut* __restrict__ outs, int ntasks, int* ticket,
                                                       int* status, long long spin_limit, int nmax, int mmax) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  __shared__ int s_task, s_abort;
  if (threadIdx.x == 0) {
    s_task = atomicAdd(ticket, 1);
    s_abort = 0;
  }
  __syncthreads();
  const int ti = s_task;
  if (ti >= ntasks) return;
  const FwdElimTask t = tasks[ti];
  T* red = sm + (kStaged ? dev::staged_elems<T>(max(nmax, mmax)) : 0);
  T* xc = red + dev::kVecRed;
  T* xn = xc + (nmax > 0 ? nmax : 1);
  for (int i = threadIdx.x; i < t.n; i += kThreads) xc[i] = __ldcg(as<T>(t.x) + i);
  __syncthreads();
  if (kStaged) dev::vec_apply_staged<T>(as<T>(t.S), t.n, as<T>(t.T), t.n, xc, t.n, true, sm);
  else dev::apply_qt<T>(as<T>(t.S), t.n, as<T>(t.T), t.n, xc, t.n, t.n, 1, red, 2 * kNB);
  for (int o = t.out_begin; o < t.out_end; ++o) {
    const FwdOut e = outs[o];
    if (threadIdx.x == 0) {
      const long long t0 = clock64();
      for (;;) {
        const int v = ld_acquire(e.turn);
        if (v == e.my_turn) break;
        if (ld_acquire(status) != 0) {
          s_abort = 1;
          break;
        }
        if (clock64() - t0 > spin_limit) {
          atomicExch(status, 2);
          s_abort = 1;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
    }
    __syncthreads();
    if (s_abort) return;
    for (int i = threadIdx.x; i < e.m; i += kThreads) xn[i] = __ldcg(as<T>(e.xn) + i);
    __syncthreads();
    if (kStaged) dev::vec_apply_staged<T>(as<T>(e.V), e.m, as<T>(e.T), t.n, xn, e.m, true, sm, xc);
    else dev::vec_apply_tpqt<T>(as<T>(e.V), e.m, as<T>(e.T), t.n, xc, xn, e.m, red);
    for (int i = threadIdx.x; i < e.m; i += kThreads) __stcg(as<T>(e.xn) + i, xn[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(e.turn, e.my_turn + 1);
    }
  }
  for (int i = threadIdx.x; i < t.n; i += kThreads) __stcg(as<T>(t.x) + i, xc[i]);
}

// kStaged: the reflector panels stream through shared memory
// (dev::vec_apply_staged), for levels with large interfaces.
template <typename T, bool kStaged>
__global__ void __launch_bounds__(kThreads) k_fwd_spars(const FwdSparsTask* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const FwdSparsTask t = tasks[blockIdx.x];
  T* red = sm + (kStaged ? dev::staged_elems<T>(t.n) : 0);
  T* x = red + 2 * kNB;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = as<T>(t.x)[i];
  __syncthreads();
  if (kStaged) {
    dev::vec_apply_staged<T>(as<T>(t.Qs), t.n, as<T>(t.Ts), t.n, x, t.n, true, sm);
    dev::vec_apply_staged<T>(as<T>(t.V), t.n, as<T>(t.T), *t.rank, x, t.n, true, sm);
  } else {
    dev::apply_qt<T>(as<T>(t.Qs), t.n, as<T>(t.Ts), t.n, x, t.n, t.n, 1, red, 2 * kNB);
    dev::apply_qt<T>(as<T>(t.V), t.n, as<T>(t.T), *t.rank, x, t.n, t.n, 1, red, 2 * kNB);
  }
  for (int i = threadIdx.x; i < t.n; i += kThreads) as<T>(t.x)[i] = x[i];
}

template <typename T, bool kStaged>
__global__ void __launch_bounds__(kThreads) k_bwd_spars(const FwdSparsTask* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const FwdSparsTask t = tasks[blockIdx.x];
  T* red = sm + (kStaged ? dev::staged_elems<T>(t.n) : 0);
  T* xs = red + 2 * kNB;
  T* x = xs + 32;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = as<T>(t.x)[i];
  __syncthreads();
  if (kStaged) dev::vec_apply_staged<T>(as<T>(t.V), t.n, as<T>(t.T), *t.rank, x, t.n, false, sm);
  else dev::apply_q<T>(as<T>(t.V), t.n, as<T>(t.T), *t.rank, x, t.n, t.n, 1, red, 2 * kNB);
  dev::trsv_upper<T>(as<T>(t.Qs), t.n, x, t.n, xs);
  for (int i = threadIdx.x; i < t.n; i += kThreads) as<T>(t.x)[i] = x[i];
}

// Forward / backward scaling + sparsification steps of small interfaces (FP32,
// n <= 32), one warp per interface: lane r holds x(r); each reflector block
// (a single panel) and its T are staged in the warp's shared memory and the
// sums run over shuffles.  The CTA kernels spend a 256-thread CTA and three
// CTA barriers per panel on vectors of this size.
constexpr int kSpLd = 33;
constexpr size_t kSparsSmallSmem = (size_t)kWarps * 2 * 32 * kSpLd * sizeof(float);

// Returns lane r's entry of Q^T x (trans) or Q x, Q = I - V T V^T for k <= 32
// unit lower reflectors of n <= 32 rows (T in kNB x k layout).
__device__ __forceinline__ float warp_apply_unit(const float* V, int ldv, const float* Tm, int k, float xr, int n,
                                                 bool trans, float* sV, float* sT, int lane) {
  for (int i = 0; i < 32; ++i) {
    float v = 0.0f;
    if (i < k && lane < n) v = lane == i ? 1.0f : (lane < i ? 0.0f : V[lane + (size_t)i * ldv]);
    sV[lane * kSpLd + i] = v;                                                         // V(lane, i)
    sT[lane * kSpLd + i] = (lane <= i && i < k) ? Tm[lane + (size_t)i * kNB] : 0.0f;  // T(lane, i)
  }
  __syncwarp();
  float w = 0.0f;  // W(lane) = sum_r V(r, lane) x(r)
  for (int r = 0; r < 32; ++r) {
    const float xb = __shfl_sync(0xffffffffu, xr, r);
    if (r < n) w += sV[r * kSpLd + lane] * xb;
  }
  float w2 = 0.0f;  // W2 = T^T W (trans) or T W
  for (int l = 0; l < 32; ++l) {
    const float wl = __shfl_sync(0xffffffffu, w, l);
    if (trans ? l <= lane : l >= lane) w2 += (trans ? sT[l * kSpLd + lane] : sT[lane * kSpLd + l]) * wl;
  }
  if (lane >= k) w2 = 0.0f;
  float acc = 0.0f;  // (V W2)(lane)
  for (int i = 0; i < 32; ++i) {
    const float wi = __shfl_sync(0xffffffffu, w2, i);
    acc += sV[lane * kSpLd + i] * wi;
  }
  __syncwarp();  // the next block overwrites sV / sT
  return xr - acc;
}

__global__ void __launch_bounds__(kThreads) k_fwd_spars_small(const FwdSparsTask* __restrict__ tasks, int ntasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ti = blockIdx.x * kWarps + warp;
  if (ti >= ntasks) return;
  const FwdSparsTask t = tasks[ti];
  float* sV = reinterpret_cast<float*>(smraw) + (size_t)warp * 2 * 32 * kSpLd;
  float* sT = sV + 32 * kSpLd;
  float* x = as<float>(t.x);
  const int n = t.n;
  float xr = lane < n ? x[lane] : 0.0f;
  xr = warp_apply_unit(as<float>(t.Qs), n, as<float>(t.Ts), n, xr, n, true, sV, sT, lane);
  xr = warp_apply_unit(as<float>(t.V), n, as<float>(t.T), *t.rank, xr, n, true, sV, sT, lane);
  if (lane < n) x[lane] = xr;
}

__global__ void __launch_bounds__(kThreads) k_bwd_spars_small(const FwdSparsTask* __restrict__ tasks, int ntasks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ti = blockIdx.x * kWarps + warp;
  if (ti >= ntasks) return;
  const FwdSparsTask t = tasks[ti];
  float* sV = reinterpret_cast<float*>(smraw) + (size_t)warp * 2 * 32 * kSpLd;
  float* sT = sV + 32 * kSpLd;
  float* x = as<float>(t.x);
  const int n = t.n;
  float xr = lane < n ? x[lane] : 0.0f;
  xr = warp_apply_unit(as<float>(t.V), n, as<float>(t.T), *t.rank, xr, n, false, sV, sT, lane);
  // x <- R^{-1} x, R the upper triangle of Qs: the diagonal-block solve of trsv_upper
  const float* R = as<float>(t.Qs);
  for (int j = 0; j < 32; ++j) sV[lane * kSpLd + j] = (lane < n && j < n && j >= lane) ? R[lane + (size_t)j * n] : 0.0f;
  __syncwarp();
  for (int j = 31; j >= 0; --j) {
    if (j < n) {
      if (lane == j) xr = xr / sV[j * kSpLd + j];
      const float xj = __shfl_sync(0xffffffffu, xr, j);
      if (lane < j) xr -= sV[lane * kSpLd + j] * xj;
    }
  }
  if (lane < n) x[lane] = xr;
}

// kBwdRows: rows per lane of the backward GEMV (interiors of <= 32 kBwdRows
// rows); 0: one thread per row.
template <typename T, int kBwdRows>
__global__ void __launch_bounds__(kThreads) k_bwd_elim(const BwdElimTask* __restrict__ tasks,
                                                       const BwdIn* __restrict__ ins, int nmax) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const BwdElimTask t = tasks[blockIdx.x];
  T* xs = sm;
  T* x = sm + 32;
  T* part = x + nmax;  // kWarps x nmax partial sums (kBwdRows > 0)
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = as<T>(t.x)[i];
  if (kBwdRows > 0) {
    // x -= sum over in-edges of R_e x_e: warp w streams the columns j = w mod
    // kWarps (lanes over rows, coalesced), two columns' loads in flight, into
    // a partial vector held in registers; the warps' partials meet in `part`
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nrs = (t.n + 31) / 32;
    constexpr int kR = kBwdRows > 0 ? kBwdRows : 1;
    T y[kR];
#pragma unroll
    for (int u = 0; u < kR; ++u) y[u] = 0.0;
    for (int q = t.in_begin; q < t.in_end; ++q) {
      const BwdIn e = ins[q];
      const T* R = as<T>(e.R);
      const T* xm = as<T>(e.xm);
      int j = warp;
      if (kR <= 12)  // four columns' loads in flight while the registers allow it
        for (; j + 3 * kWarps < e.s; j += 4 * kWarps) {
          const T* c0 = R + (size_t)j * e.ldr;
          const T* c1 = c0 + (size_t)kWarps * e.ldr;
          const T* c2 = c1 + (size_t)kWarps * e.ldr;
          const T* c3 = c2 + (size_t)kWarps * e.ldr;
          T v0[kR], v1[kR], v2[kR], v3[kR];
#pragma unroll
          for (int u = 0; u < kR; ++u) {
            const int r = lane + 32 * u;
            const bool ok = u < nrs && r < t.n;
            v0[u] = ok ? c0[r] : (T)0.0;
            v1[u] = ok ? c1[r] : (T)0.0;
            v2[u] = ok ? c2[r] : (T)0.0;
            v3[u] = ok ? c3[r] : (T)0.0;
          }
          const T x0 = xm[j], x1 = xm[j + kWarps], x2 = xm[j + 2 * kWarps], x3 = xm[j + 3 * kWarps];
#pragma unroll
          for (int u = 0; u < kR; ++u) y[u] += (v0[u] * x0 + v1[u] * x1) + (v2[u] * x2 + v3[u] * x3);
        }
      for (; j + kWarps < e.s; j += 2 * kWarps) {
        const T* c0 = R + (size_t)j * e.ldr;
        const T* c1 = c0 + (size_t)kWarps * e.ldr;
        T v0[kR], v1[kR];
#pragma unroll
        for (int u = 0; u < kR; ++u) {
          const int r = lane + 32 * u;
          const bool ok = u < nrs && r < t.n;
          v0[u] = ok ? c0[r] : (T)0.0;
          v1[u] = ok ? c1[r] : (T)0.0;
        }
        const T x0 = xm[j], x1 = xm[j + kWarps];
#pragma unroll
        for (int u = 0; u < kR; ++u) y[u] += v0[u] * x0 + v1[u] * x1;
      }
      if (j < e.s) {
        const T* c0 = R + (size_t)j * e.ldr;
        const T x0 = xm[j];
#pragma unroll
        for (int u = 0; u < kR; ++u) {
          const int r = lane + 32 * u;
          if (u < nrs && r < t.n) y[u] += c0[r] * x0;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kR; ++u) {
      const int r = lane + 32 * u;
      if (u < nrs && r < t.n) part[warp * nmax + r] = y[u];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < t.n; i += kThreads) {
      T s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += part[w * nmax + i];
      x[i] -= s;
    }
  } else {
    __syncthreads();
    for (int q = t.in_begin; q < t.in_end; ++q) {
      const BwdIn e = ins[q];
      for (int i = threadIdx.x; i < t.n; i += kThreads) {
        T s = 0.0;
        for (int j = 0; j < e.s; ++j) s += as<T>(e.R)[i + (size_t)j * e.ldr] * as<T>(e.xm)[j];
        x[i] -= s;
      }
    }
  }
  __syncthreads();
  dev::trsv_upper<T>(as<T>(t.S), t.n, x, t.n, xs);
  for (int i = threadIdx.x; i < t.n; i += kThreads) as<T>(t.x)[i] = x[i];
}

__global__ void k_permute(int n, const int* __restrict__ perm, const double* __restrict__ src, double* dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[perm[i]] = src[i];
}

template <typename T>
__global__ void k_copy_idx(int n, const int* __restrict__ src, const int* __restrict__ dst, double* xd) {
  T* x = as<T>(xd);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[dst[i]] = x[src[i]];
}

// ------------------------------------------------------------ sparse + Krylov
__global__ void k_spmv(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) s += val[k] * x[col[k]];
    y[r] = s;
  }
}

// One modified Gram-Schmidt step, fused: q -= hprev * Qprev (when Qprev),
// then partial sums of q.Qi (or of q.q when Qi is null).  The last CTA to
// finish reduces the partials in index order and writes *out (deterministic).
__global__ void __launch_bounds__(kThreads) k_mgs_step(int n, double* __restrict__ q, const double* __restrict__ Qprev,
                                                       const double* hprev, const double* __restrict__ Qi,
                                                       double* partial, unsigned int* done, double* out,
                                                       int take_sqrt) {
  __shared__ double red[kRed];
  __shared__ bool last;
  const double h = Qprev ? *hprev : 0.0;
  double s = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    double v = q[i];
    if (Qprev) {
      v -= h * Qprev[i];
      q[i] = v;
    }
    s += Qi ? v * Qi[i] : v * v;
  }
  s = dev::cta_sum(s, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s;
    __threadfence();
    const unsigned int prev = atomicAdd(done, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double t = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += kThreads) t += __ldcg(partial + b);
    t = dev::cta_sum(t, red);
    if (threadIdx.x == 0) {
      *out = take_sqrt ? sqrt(t) : t;
      *done = 0u;
    }
  }
}

__global__ void k_scale_copy(int n, const double* __restrict__ src, const double* s, double* __restrict__ dst) {
  const double inv = 1.0 / *s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i] * inv;
}

// x = Q(:, 0:k) y  (Q column-major n x ldq)
__global__ void k_combine(int n, int k, const double* __restrict__ Q, size_t ldq, const double* __restrict__ y,
                          double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < k; ++j) s += Q[i + j * ldq] * y[j];
    x[i] = s;
  }
}

__global__ void k_sub(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c[i] = a[i] - b[i];
}


inline int grid_for(int n, int per = 256, int cap = 148 * 16) {
  int g = (n + per - 1) / per;
  return g < 1 ? 1 : (g > cap ? cap : g);
}

inline size_t smem_bytes(size_t doubles) { return doubles * sizeof(double); }

}  // namespace

// ------------------------------------------------------------ precision conversion
// dst (float) <- src (double), n elements
__global__ void k_to_f32(long long n, const double* __restrict__ src, float* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}
__global__ void k_to_f64(long long n, const float* __restrict__ src, double* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
// batched: one CTA per array
__global__ void k_to_f32_batch(const ConvTask* __restrict__ tasks) {
  const ConvTask t = tasks[blockIdx.x];
  float* dst = reinterpret_cast<float*>(t.dst);
  for (long long i = t.off + threadIdx.x; i < t.off + t.n; i += blockDim.x) dst[i] = (float)t.src[i];
}

// ---------------------------------------------------------------- launchers
namespace {
std::atomic<long long> g_launches{0};
thread_local bool g_fp32 = false;  // factor storage of the next launches
thread_local bool g_tc = false;     // float left applies on the tensor cores
thread_local int* g_status = nullptr;  // status word of the factorization kernels
inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }

constexpr size_t kSmemMax = 227 * 1024;

template <typename K>
cudaError_t prep(K kern, size_t bytes) {
  if (bytes > kSmemMax) return cudaErrorInvalidValue;
  // Above 48 KB of dynamic plus static shared memory the kernel must opt in;
  // static shared memory of these kernels stays below 8 KB.  The opt-in is
  // only ever raised: a launch captured into a CUDA graph keeps its size, and
  // a later, smaller launch of the same kernel must not lower the limit under
  // it (a graph node relaunched against the lowered limit fails).
  if (bytes <= 40 * 1024) return cudaSuccess;
  static std::mutex mu;
  static std::unordered_map<const void*, size_t> raised;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = raised[reinterpret_cast<const void*>(kern)];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_clustered(void (*kern)(KArgs...), int ntasks, int cs, size_t smem, cudaStream_t st,
                             Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ntasks * cs));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  counted();
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

inline cudaError_t last() { return cudaGetLastError(); }
thread_local const char* g_last_launch = "";
// Clears a stale error left by an earlier runtime call so that the status a
// launcher returns belongs to its own launch; a stale error is reported as is.
inline cudaError_t begin(const char* name) {
  g_last_launch = name;
  return cudaGetLastError();
}
}  // namespace

const char* last_launch_name() { return g_last_launch; }
void set_factor_fp32(bool on) { g_fp32 = on; }
void set_tensor_cores(bool on) { g_tc = on; }
void set_status_word(int* status) { g_status = status; }
bool tensor_cores_on() { return g_tc; }
bool factor_fp32() { return g_fp32; }
void set_last_launch(const char* name) { g_last_launch = name; }

long long kernel_launches() { return g_launches.load(); }
void add_kernel_launches(long long n) { g_launches.fetch_add(n); }

cudaError_t launch_scatter(int nnz, const double* val, double* const* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_scatter")) return pre;
  if (nnz <= 0) return cudaSuccess;
  counted();
  if (g_fp32) k_scatter<float><<<grid_for(nnz), 256, 0, st>>>(nnz, val, dst);
  else k_scatter<double><<<grid_for(nnz), 256, 0, st>>>(nnz, val, dst);
  return last();
}

cudaError_t launch_permute(int n, const int* perm, const double* src, double* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_permute")) return pre;
  if (n <= 0) return cudaSuccess;
  counted();
  k_permute<<<grid_for(n), 256, 0, st>>>(n, perm, src, dst);
  return last();
}

// Shared memory of a dist_qr kernel whose panels are factored in shared
// memory: `head` bytes, then one region that serves as the tiled apply's
// scratch and as the panel buffer (rows x kNB plus a kNB x kNB block); 0
// when that does not fit (the kernel then factors panels in global memory).
template <typename T>
size_t staged_panel_bytes(size_t head, int rows) {
  const size_t panel = ((size_t)rows * kNB + kPanExtra) * sizeof(T);
  const size_t region = std::max(smem_bytes(kWcap), panel);
  return head + region + 1024 <= kSmemMax ? head + region : 0;
}

cudaError_t launch_elim(const ElimTask* t, const ElimOut* o, int ntasks, int cs, int nmax, int vmax,
                        cudaStream_t st) {
  if (cudaError_t pre = begin("launch_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  vmax = std::max(vmax, 1);
  const size_t head = smem_bytes(kRed + kNB + (size_t)nmax + (size_t)vmax);
  if (g_fp32) {
    const size_t bs = staged_panel_bytes<float>(head, vmax);
    if (bs) {
      if (cudaError_t e = prep(k_elim<float, true>, bs)) return e;
      return launch_clustered(k_elim<float, true>, ntasks, cs, bs, st, t, o, cs, vmax, g_status);
    }
    if (cudaError_t e = prep(k_elim<float, false>, head + smem_bytes(kWcap))) return e;
    return launch_clustered(k_elim<float, false>, ntasks, cs, head + smem_bytes(kWcap), st, t, o, cs, vmax,
                            g_status);
  }
  const size_t bs = staged_panel_bytes<double>(head, vmax);
  if (bs) {
    if (cudaError_t e = prep(k_elim<double, true>, bs)) return e;
    return launch_clustered(k_elim<double, true>, ntasks, cs, bs, st, t, o, cs, vmax, g_status);
  }
  if (cudaError_t e = prep(k_elim<double, false>, head + smem_bytes(kWcap))) return e;
  return launch_clustered(k_elim<double, false>, ntasks, cs, head + smem_bytes(kWcap), st, t, o, cs, vmax, g_status);
}

cudaError_t launch_scale(const ScaleTask* t, int ntasks, int cs, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_scale")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  nmax = std::max(nmax, 1);
  const size_t head = smem_bytes(kRed + kNB + 2 * (size_t)nmax);
  if (g_fp32) {
    const size_t bs = staged_panel_bytes<float>(head, nmax);
    if (bs) {
      if (cudaError_t e = prep(k_scale<float, true>, bs)) return e;
      return launch_clustered(k_scale<float, true>, ntasks, cs, bs, st, t, cs, nmax, g_status);
    }
    if (cudaError_t e = prep(k_scale<float, false>, head + smem_bytes(kWcap))) return e;
    return launch_clustered(k_scale<float, false>, ntasks, cs, head + smem_bytes(kWcap), st, t, cs, nmax, g_status);
  }
  const size_t bs = staged_panel_bytes<double>(head, nmax);
  if (bs) {
    if (cudaError_t e = prep(k_scale<double, true>, bs)) return e;
    return launch_clustered(k_scale<double, true>, ntasks, cs, bs, st, t, cs, nmax, g_status);
  }
  if (cudaError_t e = prep(k_scale<double, false>, head + smem_bytes(kWcap))) return e;
  return launch_clustered(k_scale<double, false>, ntasks, cs, head + smem_bytes(kWcap), st, t, cs, nmax, g_status);
}

cudaError_t launch_update(const UpdTask* t, const UpdOp* o, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_update")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kWcap);
  counted();
  if (g_fp32 && g_tc) {
    if (cudaError_t e = prep(k_update_tc, tc::kSmemBytes)) return e;
    k_update_tc<<<ntasks, kThreads, tc::kSmemBytes, st>>>(t, o, g_status);
  } else if (g_fp32) {
    if (cudaError_t e = prep(k_update<float>, b)) return e;
    k_update<float><<<ntasks, kThreads, b, st>>>(t, o);
  } else {
    if (cudaError_t e = prep(k_update<double>, b)) return e;
    k_update<double><<<ntasks, kThreads, b, st>>>(t, o);
  }
  return last();
}

cudaError_t launch_edge(int kind, const EdgeChunk* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_edge")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kWcap);
  cudaError_t e = cudaSuccess;
  counted();
  auto go = [&](auto* left, auto* trsm, auto* right) -> cudaError_t {
    if (kind == 0) {
      if ((e = prep(left, b))) return e;
      left<<<ntasks, kThreads, b, st>>>(t);
    } else if (kind == 1) {
      if ((e = prep(trsm, b))) return e;
      trsm<<<ntasks, kThreads, b, st>>>(t);
    } else {
      if ((e = prep(right, b))) return e;
      right<<<ntasks, kThreads, b, st>>>(t);
    }
    return last();
  };
  if (g_fp32 && g_tc && kind == 0) {
    if ((e = prep(k_edge_left_tc, tc::kSmemBytes))) return e;
    k_edge_left_tc<<<ntasks, kThreads, tc::kSmemBytes, st>>>(t, g_status);
    return last();
  }
  if (g_fp32 && g_tc && kind == 2) {
    if ((e = prep(k_edge_right_tc, tc::kSmemBytes))) return e;
    k_edge_right_tc<<<ntasks, kThreads, tc::kSmemBytes, st>>>(t, g_status);
    return last();
  }
  return g_fp32 ? go(k_edge_left<float>, k_edge_trsm<float>, k_edge_right<float>)
                : go(k_edge_left<double>, k_edge_trsm<double>, k_edge_right<double>);
}

cudaError_t launch_update_small(const UpdTask* t, const UpdOp* o, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_update_small")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  if (!g_fp32) return cudaErrorInvalidValue;  // FP32 factors only
  counted();
  if (cudaError_t e = prep(k_update_small, kUpdSmallSmem)) return e;
  k_update_small<<<(ntasks + kTeams - 1) / kTeams, kTeamThreads, kUpdSmallSmem, st>>>(t, o, ntasks);
  return last();
}

bool update_op_small(int k, int m) { return k <= kSmallOp && m <= kSmallOp; }

cudaError_t launch_edge_left_small(const EdgeChunk* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_edge_left_small")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  counted();
  if (!g_fp32) return cudaErrorInvalidValue;  // FP32 factors only
  const int grid = (ntasks + kWarps - 1) / kWarps;
  if (cudaError_t e = prep(k_edge_left_small<float>, small_left_smem<float>())) return e;
  k_edge_left_small<float><<<grid, kThreads, small_left_smem<float>(), st>>>(t, ntasks);
  return last();
}

bool edge_left_small(int m) { return m <= kSmallRows; }

cudaError_t launch_edge_trsm_small(const EdgeChunk* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_edge_trsm_small")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  if (!g_fp32) return cudaErrorInvalidValue;  // FP32 factors only
  counted();
  k_edge_trsm_small<<<(ntasks + kWarps - 1) / kWarps, kThreads, 0, st>>>(t, ntasks);
  return last();
}

bool edge_trsm_small(int ncols, int rows) { return ncols <= 32 && rows <= 64; }

cudaError_t launch_edge_right_small(const EdgeChunk* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_edge_right_small")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  if (!g_fp32) return cudaErrorInvalidValue;  // FP32 factors only
  counted();
  if (cudaError_t e = prep(k_edge_right_small, kRightSmallSmem)) return e;
  k_edge_right_small<<<(ntasks + kWarps - 1) / kWarps, kThreads, kRightSmallSmem, st>>>(t, ntasks);
  return last();
}

cudaError_t launch_tc_probe(const float* C, const float* V, const float* W2, int m, int flags, float* out1,
                            float* out2, int* status, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_tc_probe")) return pre;
  if (m < 1 || m > 64) return cudaErrorInvalidValue;
  if (cudaError_t e = prep(k_tc_probe, tc::kSmemBytes)) return e;
  counted();
  k_tc_probe<<<1, kThreads, tc::kSmemBytes, st>>>(C, V, W2, m, flags, out1, out2, status);
  return last();
}

size_t rrqr_smem(int mmax, int kmax, int nlmax, int rcmax, size_t c_doubles) {
  const size_t d = kRed + kNB + 4 * ((size_t)kmax + 1) + 2 * (size_t)rcmax + (size_t)std::max(mmax, 1) +
                   2 * (size_t)nlmax + (size_t)rrqr_gp_doubles(nlmax);
  size_t b = smem_bytes(d) + sizeof(int) * 2 * (size_t)nlmax;
  if (c_doubles) b += 16 + smem_bytes(c_doubles);
  return b;
}

template <bool kSmemC>
bool rrqr_fits(int cs, size_t smem) {
  if (smem > kSmemMax) return false;
  if (cs <= 8) return true;
  if (prep(k_rrqr<kSmemC>, smem)) return false;
  if (cudaFuncSetAttribute(k_rrqr<kSmemC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cs);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_rrqr<kSmemC>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}

bool rrqr_cluster_fits(int cs, size_t smem, bool smem_c) {
  return smem_c ? rrqr_fits<true>(cs, smem) : rrqr_fits<false>(cs, smem);
}

cudaError_t launch_rrqr_assemble(const RrqrSrc* s, int nsrc, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_rrqr_assemble")) return pre;
  if (nsrc <= 0) return cudaSuccess;
  counted();
  if (g_fp32) k_rrqr_assemble<float><<<nsrc, kThreads, 0, st>>>(s);
  else k_rrqr_assemble<double><<<nsrc, kThreads, 0, st>>>(s);
  return last();
}

template <bool kSmemC>
cudaError_t launch_rrqr_t(const RrqrTask* t, int ntasks, int cs, int mmax, int kmax, int nlmax, int rcmax,
                          size_t c_doubles, double tol, double pivot_rtol, cudaStream_t st) {
  const size_t b = rrqr_smem(mmax, kmax, nlmax, rcmax, kSmemC ? c_doubles : 0);
  cudaError_t e = prep(k_rrqr<kSmemC>, b);
  if (!e && cs > 8) e = cudaFuncSetAttribute(k_rrqr<kSmemC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e) return e;
  return launch_clustered(k_rrqr<kSmemC>, ntasks, cs, b, st, t, tol, pivot_rtol, cs, mmax, kmax, nlmax, rcmax);
}

cudaError_t launch_rrqr(const RrqrTask* t, int ntasks, int cs, int mmax, int kmax, int nlmax, int rcmax,
                        size_t c_doubles, double tol, double pivot_rtol, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_rrqr")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  return c_doubles ? launch_rrqr_t<true>(t, ntasks, cs, mmax, kmax, nlmax, rcmax, c_doubles, tol, pivot_rtol, st)
                   : launch_rrqr_t<false>(t, ntasks, cs, mmax, kmax, nlmax, rcmax, 0, tol, pivot_rtol, st);
}

int selected_qr_rows(int nmax) { return std::max(1, std::min(32, 12288 / (std::max(nmax, 1) + 1))); }

// stage: with room for the QR's staged panel (0 when that does not fit)
size_t selected_qr_smem(int mmax, int nmax, bool stage) {
  const int rt = selected_qr_rows(nmax);
  mmax = std::max(mmax, 1);
  size_t region = std::max((size_t)rt * (std::max(nmax, 1) + 1) + 32 * 33, (size_t)kWcap);
  if (stage) region = std::max(region, (size_t)mmax * kNB + kPanExtra);
  const size_t b = smem_bytes(kRed + kNB + (size_t)std::max(nmax, 1) + (size_t)mmax + region);
  return !stage || b + 1024 <= kSmemMax ? b : 0;
}

cudaError_t launch_selected_qr(const RrqrTask* t, int ntasks, int cs, int mmax, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_selected_qr")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const int mm = std::max(mmax, 1), nn = std::max(nmax, 1), rt = selected_qr_rows(nmax);
  if (const size_t bs = selected_qr_smem(mmax, nmax, true)) {
    if (cudaError_t e = prep(k_selected_qr<true>, bs)) return e;
    return launch_clustered(k_selected_qr<true>, ntasks, cs, bs, st, t, cs, mm, nn, rt);
  }
  const size_t b = selected_qr_smem(mmax, nmax, false);
  if (cudaError_t e = prep(k_selected_qr<false>, b)) return e;
  return launch_clustered(k_selected_qr<false>, ntasks, cs, b, st, t, cs, mm, nn, rt);
}

cudaError_t launch_merge(const MergeTask* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_merge")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  counted();
  if (g_fp32) k_merge<float><<<ntasks, 256, 0, st>>>(t);
  else k_merge<double><<<ntasks, 256, 0, st>>>(t);
  return last();
}

// The staged sweep kernels (reflector panels streamed through shared memory)
// serve levels whose largest block has at least kStagedMin rows and whose
// buffers fit; smaller blocks keep more CTAs per SM with the direct loads.
constexpr int kStagedMin = 256;
template <typename T>
bool use_staged(int nmax, size_t other_bytes) {
  // 1 KB left for the kernels' static shared memory
  return nmax >= kStagedMin && dev::staged_elems<T>(nmax) * sizeof(T) + other_bytes + 1024 <= kSmemMax;
}

cudaError_t launch_fwd_elim(const FwdElimTask* t, const FwdOut* o, int ntasks, int nmax, int mmax, int* ticket,
                            int* status, long long spin_limit, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_fwd_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  nmax = std::max(nmax, 1);
  mmax = std::max(mmax, 1);
  const size_t b = smem_bytes(dev::kVecRed + (size_t)nmax + (size_t)mmax);
  const int srows = std::max(nmax, mmax);  // rows of a staged panel: the interior's or a neighbour's
  counted();
  auto go = [&](auto kern, size_t bytes) -> cudaError_t {
    if (cudaError_t e = prep(kern, bytes)) return e;
    kern<<<ntasks, kThreads, bytes, st>>>(t, o, ntasks, ticket, status, spin_limit, nmax, mmax);
    return cudaSuccess;
  };
  cudaError_t e;
  // staged where the interiors themselves are large (the top levels, few
  // CTAs); large neighbours of small interiors alone do not pay for it
  const bool big = nmax >= kStagedMin;
  if (g_fp32)
    e = big && use_staged<float>(srows, b)
            ? go(k_fwd_elim<float, true>, dev::staged_elems<float>(srows) * sizeof(float) + b)
            : go(k_fwd_elim<float, false>, b);
  else
    e = big && use_staged<double>(srows, b)
            ? go(k_fwd_elim<double, true>, dev::staged_elems<double>(srows) * sizeof(double) + b)
            : go(k_fwd_elim<double, false>, b);
  if (e) return e;
  return last();
}

// k_fwd_spars / k_bwd_spars over ntasks interfaces of at most nmax rows
template <bool kFwd>
cudaError_t launch_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  const size_t b = smem_bytes(2 * kNB + 32 + (size_t)std::max(nmax, 1));
  counted();
  auto go = [&](auto kern, size_t bytes) -> cudaError_t {
    if (cudaError_t e = prep(kern, bytes)) return e;
    kern<<<ntasks, kThreads, bytes, st>>>(t);
    return cudaSuccess;
  };
  cudaError_t e;
  if (g_fp32) {
    const size_t bs = dev::staged_elems<float>(nmax) * sizeof(float) + b;
    if (use_staged<float>(nmax, b)) e = kFwd ? go(k_fwd_spars<float, true>, bs) : go(k_bwd_spars<float, true>, bs);
    else e = kFwd ? go(k_fwd_spars<float, false>, b) : go(k_bwd_spars<float, false>, b);
  } else {
    const size_t bs = dev::staged_elems<double>(nmax) * sizeof(double) + b;
    if (use_staged<double>(nmax, b)) e = kFwd ? go(k_fwd_spars<double, true>, bs) : go(k_bwd_spars<double, true>, bs);
    else e = kFwd ? go(k_fwd_spars<double, false>, b) : go(k_bwd_spars<double, false>, b);
  }
  if (e) return e;
  return last();
}

// The warp-per-interface forms (FP32, n <= 32): kFwd chooses the forward step.
cudaError_t launch_spars_small(bool fwd, const FwdSparsTask* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_spars_small")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  if (!g_fp32) return cudaErrorInvalidValue;  // FP32 factors only
  counted();
  const int grid = (ntasks + kWarps - 1) / kWarps;
  if (fwd) {
    if (cudaError_t e = prep(k_fwd_spars_small, kSparsSmallSmem)) return e;
    k_fwd_spars_small<<<grid, kThreads, kSparsSmallSmem, st>>>(t, ntasks);
  } else {
    if (cudaError_t e = prep(k_bwd_spars_small, kSparsSmallSmem)) return e;
    k_bwd_spars_small<<<grid, kThreads, kSparsSmallSmem, st>>>(t, ntasks);
  }
  return last();
}

bool spars_small(int n) { return n <= 32; }

cudaError_t launch_fwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_fwd_spars")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  return launch_spars<true>(t, ntasks, nmax, st);
}

cudaError_t launch_bwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_bwd_spars")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  return launch_spars<false>(t, ntasks, nmax, st);
}

cudaError_t launch_bwd_elim(const BwdElimTask* t, const BwdIn* in, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_bwd_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  nmax = std::max(nmax, 1);
  const int rows = nmax <= 128 ? 4 : nmax <= 384 ? 12 : nmax <= 1024 ? 32 : 0;
  const size_t b = smem_bytes(32 + (size_t)nmax + (rows ? (size_t)kWarps * nmax : 0));
  counted();
  auto go = [&](auto kern) -> cudaError_t {
    if (cudaError_t e = prep(kern, b)) return e;
    kern<<<ntasks, kThreads, b, st>>>(t, in, nmax);
    return cudaSuccess;
  };
  cudaError_t e;
  if (g_fp32)
    e = rows == 4 ? go(k_bwd_elim<float, 4>) : rows == 12 ? go(k_bwd_elim<float, 12>)
        : rows == 32 ? go(k_bwd_elim<float, 32>) : go(k_bwd_elim<float, 0>);
  else
    e = rows == 4 ? go(k_bwd_elim<double, 4>) : rows == 12 ? go(k_bwd_elim<double, 12>)
        : rows == 32 ? go(k_bwd_elim<double, 32>) : go(k_bwd_elim<double, 0>);
  if (e) return e;
  return last();
}

cudaError_t launch_copy_idx(int n, const int* src, const int* dst, double* x, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_copy_idx")) return pre;
  if (n <= 0) return cudaSuccess;
  counted();
  if (g_fp32) k_copy_idx<float><<<grid_for(n), 256, 0, st>>>(n, src, dst, x);
  else k_copy_idx<double><<<grid_for(n), 256, 0, st>>>(n, src, dst, x);
  return last();
}

cudaError_t launch_to_f32(long long n, const double* src, double* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_to_f32")) return pre;
  if (n <= 0) return cudaSuccess;
  counted();
  k_to_f32<<<grid_for((int)std::min<long long>(n, 1 << 30)), 256, 0, st>>>(n, src, reinterpret_cast<float*>(dst));
  return last();
}

cudaError_t launch_to_f64(long long n, const double* src, double* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_to_f64")) return pre;
  if (n <= 0) return cudaSuccess;
  counted();
  k_to_f64<<<grid_for((int)std::min<long long>(n, 1 << 30)), 256, 0, st>>>(n, reinterpret_cast<const float*>(src),
                                                                           dst);
  return last();
}

cudaError_t launch_to_f32_batch(const ConvTask* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_to_f32_batch")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  counted();
  k_to_f32_batch<<<ntasks, 256, 0, st>>>(t);
  return last();
}

cudaError_t launch_spmv(int n, const int* rowptr, const int* col, const double* val, const double* x, double* y,
                        cudaStream_t st) {
  if (cudaError_t pre = begin("launch_spmv")) return pre;
  counted();
  k_spmv<<<grid_for(n), 256, 0, st>>>(n, rowptr, col, val, x, y);
  return last();
}

int mgs_grid(int n) { return grid_for(n, kThreads * 4, 148 * 4); }

cudaError_t launch_mgs_step(int n, double* q, const double* Qprev, const double* hprev, const double* Qi,
                            double* partial, unsigned int* done, double* out, int take_sqrt, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_mgs_step")) return pre;
  counted();
  k_mgs_step<<<mgs_grid(n), kThreads, 0, st>>>(n, q, Qprev, hprev, Qi, partial, done, out, take_sqrt);
  return last();
}

cudaError_t launch_scale_copy(int n, const double* src, const double* s, double* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_scale_copy")) return pre;
  counted();
  k_scale_copy<<<grid_for(n), 256, 0, st>>>(n, src, s, dst);
  return last();
}

cudaError_t launch_combine(int n, int k, const double* Q, size_t ldq, const double* y, double* x, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_combine")) return pre;
  counted();
  k_combine<<<grid_for(n), 256, 0, st>>>(n, k, Q, ldq, y, x);
  return last();
}

cudaError_t launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_sub")) return pre;
  counted();
  k_sub<<<grid_for(n), 256, 0, st>>>(n, a, b, c);
  return last();
}

}  // namespace spq
