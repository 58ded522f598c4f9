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

#include "dense.cuh"
#include "kernels.hpp"
#include "tasks.hpp"

namespace cg = cooperative_groups;

namespace spq {
namespace {

using dev::kNB;
using dev::kThreads;
using dev::kWarps;

constexpr int kRed = 16;     // reduction scratch (doubles)
constexpr int kWcap = 4096;  // W scratch (doubles) of the chunked block applies

__device__ __forceinline__ void csync(int cs) {
  if (cs > 1) cg::this_cluster().sync();
  else __syncthreads();
}
__device__ __forceinline__ int crank(int cs) { return cs > 1 ? (int)cg::this_cluster().block_rank() : 0; }
__device__ __forceinline__ bool owns(int col, int rank, int cs) { return ((col / kNB) % cs) == rank; }

// ------------------------------------------------------------ assembly
__global__ void k_scatter(int nnz, const double* __restrict__ val, double* const* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) *dst[i] = val[i];
}

// ------------------------------------------------------------ distributed Householder QR
// Reflector j of a geqrt (unit = 1: v = [1; S(j+1:m, j)]) or of a tpqrt step
// (unit = 0: v = [1 (on R(j,j)); B(:, j)]).  The owner of column j computes it;
// after the cluster barrier every CTA loads the tail into shared `vb` and
// applies H_j to its own columns k > j.  `lt` holds the owner's tau values for
// its panels (T factors), `tg` broadcasts tau through global memory.
__device__ void dist_qr(double* R, int ldr, double* B, int ldb, int m, int n, int unit, double* Tout, double* tg,
                        double* lt, double* vb, double* red, double* tmp, int cs) {
  const int rank = crank(cs);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // unit: reflector tails live in R itself (rows j+1..m-1 of column j), m rows
  // pentagonal: tails are the m rows of B, the diagonal lives in R
  for (int j = 0; j < n; ++j) {
    const int vlen = unit ? (m - j - 1) : m;
    double* tail = unit ? (R + (j + 1) + (size_t)j * ldr) : (B + (size_t)j * ldb);
    if (owns(j, rank, cs)) {
      double s = 0.0;
      for (int i = threadIdx.x; i < vlen; i += kThreads) s += tail[i] * tail[i];
      s = dev::cta_sum(s, red);
      const double alpha = R[j + (size_t)j * ldr];
      double beta, scal;
      const double tj = dev::house(alpha, s, &beta, &scal);
      if (tj != 0.0)
        for (int i = threadIdx.x; i < vlen; i += kThreads) tail[i] *= scal;
      __syncthreads();
      if (threadIdx.x == 0) {
        R[j + (size_t)j * ldr] = beta;
        lt[j] = tj;
        tg[j] = tj;
      }
      __threadfence();
    }
    csync(cs);
    const double tj = __ldcg(tg + j);
    if (tj != 0.0) {
      for (int i = threadIdx.x; i < vlen; i += kThreads) vb[i] = __ldcg(tail + i);
      __syncthreads();
      // apply H_j to own columns k > j
      for (int k = j + 1 + warp; k < n; k += kWarps) {
        if (!owns(k, rank, cs)) continue;
        double* rjk = R + j + (size_t)k * ldr;
        double* tk = unit ? (R + (j + 1) + (size_t)k * ldr) : (B + (size_t)k * ldb);
        double d = lane == 0 ? *rjk : 0.0;
        for (int i = lane; i < vlen; i += 32) d += vb[i] * tk[i];
        d = dev::warp_sum(d) * tj;
        if (lane == 0) *rjk -= d;
        for (int i = lane; i < vlen; i += 32) tk[i] -= vb[i] * d;
      }
    }
    __syncthreads();
  }
  // block factors of own panels
  for (int j0 = rank * kNB; j0 < n; j0 += cs * kNB) {
    const int kb = (n - j0) < kNB ? (n - j0) : kNB;
    if (unit)
      dev::panel_t(R + j0 + (size_t)j0 * ldr, ldr, m - j0, kb, 1, lt + j0, Tout + (size_t)j0 * kNB, kNB, tmp);
    else
      dev::panel_t(B + (size_t)j0 * ldb, ldb, m, kb, 0, lt + j0, Tout + (size_t)j0 * kNB, kNB, tmp);
  }
  csync(cs);
}

__global__ void __launch_bounds__(kThreads) k_elim(const ElimTask* __restrict__ tasks, const ElimOut* __restrict__ outs,
                                                   int cs, int vmax) {
  extern __shared__ double sm[];
  const ElimTask t = tasks[blockIdx.x / cs];
  double* red = sm;
  double* tmp = red + kRed;
  double* lt = tmp + kNB;
  double* vb = lt + t.n;
  (void)vmax;
  dist_qr(t.S, t.n, nullptr, 0, t.n, t.n, 1, t.T, t.tau, lt, vb, red, tmp, cs);
  for (int o = t.out_begin; o < t.out_end; ++o) {
    const ElimOut e = outs[o];
    dist_qr(t.S, t.n, e.B, e.m, e.m, t.n, 0, e.T, t.tau, lt, vb, red, tmp, cs);
  }
}

__global__ void __launch_bounds__(kThreads) k_scale(const ScaleTask* __restrict__ tasks, int cs) {
  extern __shared__ double sm[];
  const ScaleTask t = tasks[blockIdx.x / cs];
  double* red = sm;
  double* tmp = red + kRed;
  double* lt = tmp + kNB;
  double* vb = lt + t.n;
  dist_qr(t.S, t.n, nullptr, 0, t.n, t.n, 1, t.T, t.tau, lt, vb, red, tmp, cs);
}

// ------------------------------------------------------------ chunked applies
__global__ void __launch_bounds__(kThreads) k_update(const UpdTask* __restrict__ tasks, const UpdOp* __restrict__ ops) {
  extern __shared__ double sm[];
  const UpdTask t = tasks[blockIdx.x];
  for (int o = t.op_begin; o < t.op_end; ++o) {
    const UpdOp op = ops[o];
    if (op.kind == 0)
      dev::apply_qt(op.V, op.ldv, op.T, op.k, op.A + (size_t)t.col0 * op.lda, op.lda, op.m, t.ncols, sm, kWcap);
    else
      dev::apply_tpqt(op.V, op.ldv, op.T, op.k, op.A + (size_t)t.col0 * op.lda, op.lda, op.B + (size_t)t.col0 * op.ldb,
                      op.ldb, op.m, t.ncols, sm, kWcap);
  }
}

// row scaling: columns [lo, lo+cnt) of A <- Qs^T A
__global__ void __launch_bounds__(kThreads) k_edge_left(const EdgeChunk* __restrict__ tasks) {
  extern __shared__ double sm[];
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  int cnt = t.cnt;
  if (t.limdev) {
    const int lim = *t.limdev;
    if (t.lo >= lim) return;
    cnt = min(cnt, lim - t.lo);
  }
  dev::apply_qt(t.V, t.ldv, t.T, k, t.A + (size_t)t.lo * t.lda, t.lda, t.m, cnt, sm, kWcap);
}

// column scaling: rows [lo, lo+cnt) of A <- A R^{-1}
__global__ void __launch_bounds__(kThreads) k_edge_trsm(const EdgeChunk* __restrict__ tasks) {
  const EdgeChunk t = tasks[blockIdx.x];
  dev::trsm_right_upper(t.V, t.ldv, t.A + t.lo, t.lda, t.cnt, t.nc);
}

// right compression: rows [lo, lo+cnt) of A <- A Q
__global__ void __launch_bounds__(kThreads) k_edge_right(const EdgeChunk* __restrict__ tasks) {
  extern __shared__ double sm[];
  const EdgeChunk t = tasks[blockIdx.x];
  const int k = t.kdev ? *t.kdev : t.k;
  dev::apply_q_right(t.V, t.ldv, t.T, k, t.A + t.lo, t.lda, t.cnt, t.nc, sm, kWcap);
}

// ------------------------------------------------------------ RRQR
// Column-pivoted Householder QR of C (m x w) stopped at the first i >= 1 with
// |R(i,i)| / |R(0,0)| < tol (util.cpp:830-851 choose_rank on the dgeqp3
// diagonal).  Pivot and norm downdating follow LAPACK dlaqp2, with the pivot
// taken as the first POSITION (LAPACK's column order after its swaps) whose
// partial norm is within pivot_rtol of the largest.  Columns stay in place;
// pos[] (per CTA, own columns) and colat[] (global) track the swaps.
__global__ void __launch_bounds__(kThreads) k_rrqr(const RrqrTask* __restrict__ tasks, const RrqrSrc* __restrict__ srcs,
                                                   double tol, double pivot_rtol, int cs, int wloc_max) {
  extern __shared__ double sm[];
  __shared__ double s_x[2][kWarps];
  __shared__ int s_k[2][kWarps];
  __shared__ double s_cmax;   // this CTA's max partial norm (read by the cluster)
  __shared__ int s_cpos, s_ccol;
  const RrqrTask t = tasks[blockIdx.x / cs];
  const int rank = crank(cs);
  const int m = t.m, w = t.w;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* C = t.C;
  double* red = sm;
  double* tmp = red + kRed;
  double* vb = tmp + kNB;
  double* ltau = vb + (m > 0 ? m : 1);
  int* pos = reinterpret_cast<int*>(ltau + (m > 0 ? m : 1));  // own columns, by local index
  (void)wloc_max;
  double* vn1 = t.vn;
  double* vn2 = t.vn + w;
  // assemble own panels of C
  {
    int col = 0;
    for (int s = t.src_begin; s < t.src_end; ++s) {
      const RrqrSrc src = srcs[s];
      const int width = src.transpose ? src.rows : src.cols;
      for (int idx = threadIdx.x; idx < width * m; idx += kThreads) {
        const int c = idx / m, r = idx % m;
        const int gc = col + c;
        if (!owns(gc, rank, cs)) continue;
        C[r + (size_t)gc * m] = src.transpose ? src.A[c + (size_t)r * src.lda] : src.A[r + (size_t)c * src.lda];
      }
      col += width;
    }
  }
  __syncthreads();
  // own columns: local index li <-> global column gc
  const int npan = (w + kNB - 1) / kNB;
  auto gcol = [&](int li) { return ((li / kNB) * cs + rank) * kNB + (li % kNB); };
  const int own_pan = (npan - rank + cs - 1) / cs;
  int nloc = 0;
  if (own_pan > 0) {
    const int last_pan = rank + (own_pan - 1) * cs;
    nloc = (own_pan - 1) * kNB + min(kNB, w - last_pan * kNB);
  }
  for (int li = warp; li < nloc; li += kWarps) {
    const int gc = gcol(li);
    const double* cj = C + (size_t)gc * m;
    double s = 0.0;
    for (int r = lane; r < m; r += 32) s += cj[r] * cj[r];
    s = sqrt(dev::warp_sum(s));
    if (lane == 0) {
      vn1[gc] = s;
      vn2[gc] = s;
      pos[li] = gc;
      t.colat[gc] = gc;
    }
  }
  __syncthreads();
  csync(cs);
  const int kmin = m < w ? m : w;
  const double tol3z = sqrt(1.1102230246251565e-16);
  int rk = kmin;
  for (int i = 0; i < kmin; ++i) {
    // (a) largest partial norm over active columns (position >= i)
    double bv = -1.0;
    for (int li = threadIdx.x; li < nloc; li += kThreads)
      if (pos[li] >= i) bv = fmax(bv, vn1[gcol(li)]);
    for (int o = 16; o > 0; o >>= 1) bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, o));
    if (lane == 0) s_x[0][warp] = bv;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = s_x[0][0];
      for (int q = 1; q < kWarps; ++q) v = fmax(v, s_x[0][q]);
      s_cmax = v;
    }
    csync(cs);
    double gmax = -1.0;
    if (cs > 1) {
      cg::cluster_group cl = cg::this_cluster();
      for (int q = 0; q < cs; ++q) gmax = fmax(gmax, *cl.map_shared_rank(&s_cmax, q));
    } else {
      gmax = s_cmax;
    }
    // (b) first position with vn1 >= (1 - pivot_rtol) * max
    const double thr = gmax * (1.0 - pivot_rtol);
    int bp = 0x7fffffff, bc = -1;
    for (int li = threadIdx.x; li < nloc; li += kThreads) {
      const int p = pos[li];
      if (p >= i && p < bp && vn1[gcol(li)] >= thr) {
        bp = p;
        bc = gcol(li);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
      if (op < bp) {
        bp = op;
        bc = oc;
      }
    }
    if (lane == 0) {
      s_k[0][warp] = bp;
      s_k[1][warp] = bc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int p = s_k[0][0], c = s_k[1][0];
      for (int q = 1; q < kWarps; ++q)
        if (s_k[0][q] < p) {
          p = s_k[0][q];
          c = s_k[1][q];
        }
      s_cpos = p;
      s_ccol = c;
    }
    csync(cs);
    int ppos = 0x7fffffff, pcol = -1;
    if (cs > 1) {
      cg::cluster_group cl = cg::this_cluster();
      for (int q = 0; q < cs; ++q) {
        const int p = *cl.map_shared_rank(&s_cpos, q);
        const int c = *cl.map_shared_rank(&s_ccol, q);
        if (p < ppos) {
          ppos = p;
          pcol = c;
        }
      }
    } else {
      ppos = s_cpos;
      pcol = s_ccol;
    }
    if (pcol < 0) {  // no finite maximum (NaN norms): take the column at position i
      ppos = i;
      pcol = __ldcg(t.colat + i);
    }
    // (c) the owner of the pivot column builds reflector i and books the swap
    const int cur = __ldcg(t.colat + i);  // column now at position i
    if (owns(pcol, rank, cs)) {
      double* cp = C + (size_t)pcol * m;
      double s = 0.0;
      for (int r = i + 1 + threadIdx.x; r < m; r += kThreads) s += cp[r] * cp[r];
      s = dev::cta_sum(s, red);
      const double alpha = cp[i];
      double beta, scal;
      const double ti = dev::house(alpha, s, &beta, &scal);
      double* vo = t.V + (size_t)i * m;
      for (int r = threadIdx.x; r < m; r += kThreads) {
        double v = 0.0;
        if (r == i) v = 1.0;
        else if (r > i) v = ti != 0.0 ? cp[r] * scal : cp[r];
        vo[r] = v;
      }
      if (threadIdx.x == 0) {
        t.tau[i] = ti;
        double stop = 0.0;
        const double absb = fabs(beta);
        if (i == 0) t.bc[2] = absb;
        else if (!(absb / __ldcg(t.bc + 2) >= tol)) stop = 1.0;
        t.bc[i & 1] = stop;
      }
      __threadfence();
    }
    csync(cs);
    if (__ldcg(t.bc + (i & 1)) != 0.0) {
      rk = i;
      break;
    }
    // every CTA has read colat[i] above; book the swap for the next steps
    if (owns(pcol, rank, cs) && threadIdx.x == 0) {
      t.colat[ppos] = cur;
      t.colat[i] = pcol;
      __threadfence();
    }
    // (d) position bookkeeping of own columns
    for (int li = threadIdx.x; li < nloc; li += kThreads) {
      const int gc = gcol(li);
      if (gc == pcol) pos[li] = i;
      else if (gc == cur) pos[li] = ppos;
    }
    const double ti = __ldcg(t.tau + i);
    for (int r = threadIdx.x; r < m - i; r += kThreads) vb[r] = __ldcg(t.V + (size_t)i * m + i + r);
    __syncthreads();
    // (e) apply H_i to own active columns and downdate their norms
    for (int li = warp; li < nloc; li += kWarps) {
      if (pos[li] <= i) continue;
      const int gc = gcol(li);
      double* cj = C + (size_t)gc * m;
      if (ti != 0.0) {
        double d = 0.0;
        for (int r = lane; r < m - i; r += 32) d += vb[r] * cj[i + r];
        d = dev::warp_sum(d) * ti;
        __syncwarp();
        for (int r = lane; r < m - i; r += 32) cj[i + r] -= vb[r] * d;
        __syncwarp();
      }
      const double v1 = vn1[gc];
      if (v1 != 0.0) {
        double temp = fabs(cj[i]) / v1;
        temp = 1.0 - temp * temp;
        temp = temp < 0.0 ? 0.0 : temp;
        const double q = v1 / vn2[gc];
        if (temp * q * q <= tol3z) {
          double nn = 0.0;
          for (int r = i + 1 + lane; r < m; r += 32) nn += cj[r] * cj[r];
          nn = (i + 1 < m) ? sqrt(dev::warp_sum(nn)) : 0.0;
          if (lane == 0) {
            vn1[gc] = nn;
            vn2[gc] = nn;
          }
        } else if (lane == 0) {
          vn1[gc] = v1 * sqrt(temp);
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
  csync(cs);
  // block factors of the kept reflectors, panels dealt over the cluster
  for (int j0 = rank * kNB; j0 < rk; j0 += cs * kNB) {
    const int kb = (rk - j0) < kNB ? (rk - j0) : kNB;
    for (int q = threadIdx.x; q < kb; q += kThreads) ltau[q] = __ldcg(t.tau + j0 + q);
    __syncthreads();
    dev::panel_t(t.V + j0 + (size_t)j0 * m, m, m - j0, kb, 1, ltau, t.T + (size_t)j0 * kNB, kNB, tmp);
  }
  if (rank == 0 && threadIdx.x == 0) *t.rank = rk;
  csync(cs);
}

// ------------------------------------------------------------ merge
__global__ void k_merge(const MergeTask* __restrict__ tasks) {
  const MergeTask t = tasks[blockIdx.x];
  const int total = t.rows * t.cols;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int i = idx % t.rows, j = idx / t.rows;
    const double v = t.identity ? (i == j ? 1.0 : 0.0) : t.src[i + (size_t)j * t.ld_src];
    t.dst[(t.roff + i) + (size_t)(t.coff + j) * t.ld_dst] = v;
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
__global__ void __launch_bounds__(kThreads) k_fwd_elim(const FwdElimTask* __restrict__ tasks,
                                                       const FwdOut* __restrict__ outs, int ntasks, int* ticket,
                                                       int* status, long long spin_limit, int nmax) {
  extern __shared__ double sm[];
  __shared__ int s_task, s_abort;
  if (threadIdx.x == 0) {
    s_task = atomicAdd(ticket, 1);
    s_abort = 0;
  }
  __syncthreads();
  const int ti = s_task;
  if (ti >= ntasks) return;
  const FwdElimTask t = tasks[ti];
  double* w = sm;
  double* xc = w + 2 * kNB;
  double* xn = xc + (nmax > 0 ? nmax : 1);
  for (int i = threadIdx.x; i < t.n; i += kThreads) xc[i] = __ldcg(t.x + i);
  __syncthreads();
  dev::apply_qt(t.S, t.n, t.T, t.n, xc, t.n, t.n, 1, w, 2 * kNB);
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
    for (int i = threadIdx.x; i < e.m; i += kThreads) xn[i] = __ldcg(e.xn + i);
    __syncthreads();
    dev::apply_tpqt(e.V, e.m, e.T, t.n, xc, t.n, xn, e.m, e.m, 1, w, 2 * kNB);
    for (int i = threadIdx.x; i < e.m; i += kThreads) __stcg(e.xn + i, xn[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(e.turn, e.my_turn + 1);
    }
  }
  for (int i = threadIdx.x; i < t.n; i += kThreads) __stcg(t.x + i, xc[i]);
}

__global__ void __launch_bounds__(kThreads) k_fwd_spars(const FwdSparsTask* __restrict__ tasks) {
  extern __shared__ double sm[];
  const FwdSparsTask t = tasks[blockIdx.x];
  double* w = sm;
  double* x = sm + 2 * kNB;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = t.x[i];
  __syncthreads();
  dev::apply_qt(t.Qs, t.n, t.Ts, t.n, x, t.n, t.n, 1, w, 2 * kNB);
  dev::apply_qt(t.V, t.n, t.T, *t.rank, x, t.n, t.n, 1, w, 2 * kNB);
  for (int i = threadIdx.x; i < t.n; i += kThreads) t.x[i] = x[i];
}

__global__ void __launch_bounds__(kThreads) k_bwd_spars(const FwdSparsTask* __restrict__ tasks) {
  extern __shared__ double sm[];
  const FwdSparsTask t = tasks[blockIdx.x];
  double* w = sm;
  double* xs = w + 2 * kNB;
  double* x = xs + 32;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = t.x[i];
  __syncthreads();
  dev::apply_q(t.V, t.n, t.T, *t.rank, x, t.n, t.n, 1, w, 2 * kNB);
  dev::trsv_upper(t.Qs, t.n, x, t.n, xs);
  for (int i = threadIdx.x; i < t.n; i += kThreads) t.x[i] = x[i];
}

__global__ void __launch_bounds__(kThreads) k_bwd_elim(const BwdElimTask* __restrict__ tasks,
                                                       const BwdIn* __restrict__ ins) {
  extern __shared__ double sm[];
  const BwdElimTask t = tasks[blockIdx.x];
  double* xs = sm;
  double* x = sm + 32;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = t.x[i];
  __syncthreads();
  for (int q = t.in_begin; q < t.in_end; ++q) {
    const BwdIn e = ins[q];
    for (int i = threadIdx.x; i < t.n; i += kThreads) {
      double s = 0.0;
      for (int j = 0; j < e.s; ++j) s += e.R[i + (size_t)j * e.ldr] * e.xm[j];
      x[i] -= s;
    }
  }
  __syncthreads();
  dev::trsv_upper(t.S, t.n, x, t.n, xs);
  for (int i = threadIdx.x; i < t.n; i += kThreads) t.x[i] = x[i];
}

__global__ void k_copy_idx(int n, const int* __restrict__ src, const int* __restrict__ dst, double* x) {
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

// ---------------------------------------------------------------- launchers
namespace {
std::atomic<long long> g_launches{0};
inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }

constexpr size_t kSmemMax = 227 * 1024;

template <typename K>
cudaError_t prep(K kern, size_t bytes) {
  if (bytes > kSmemMax) return cudaErrorInvalidValue;
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
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

long long kernel_launches() { return g_launches.load(); }
void add_kernel_launches(long long n) { g_launches.fetch_add(n); }

cudaError_t launch_scatter(int nnz, const double* val, double* const* dst, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_scatter")) return pre;
  if (nnz <= 0) return cudaSuccess;
  counted();
  k_scatter<<<grid_for(nnz), 256, 0, st>>>(nnz, val, dst);
  return last();
}

cudaError_t launch_elim(const ElimTask* t, const ElimOut* o, int ntasks, int cs, int nmax, int vmax,
                        cudaStream_t st) {
  if (cudaError_t pre = begin("launch_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kRed + kNB + (size_t)nmax + (size_t)std::max(vmax, 1));
  cudaError_t e = prep(k_elim, b);
  if (e) return e;
  return launch_clustered(k_elim, ntasks, cs, b, st, t, o, cs, vmax);
}

cudaError_t launch_scale(const ScaleTask* t, int ntasks, int cs, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_scale")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kRed + kNB + 2 * (size_t)nmax);
  cudaError_t e = prep(k_scale, b);
  if (e) return e;
  return launch_clustered(k_scale, ntasks, cs, b, st, t, cs);
}

cudaError_t launch_update(const UpdTask* t, const UpdOp* o, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_update")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kWcap);
  cudaError_t e = prep(k_update, b);
  if (e) return e;
  counted();
  k_update<<<ntasks, kThreads, b, st>>>(t, o);
  return last();
}

cudaError_t launch_edge(int kind, const EdgeChunk* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_edge")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kWcap);
  cudaError_t e = cudaSuccess;
  counted();
  if (kind == 0) {
    if ((e = prep(k_edge_left, b))) return e;
    k_edge_left<<<ntasks, kThreads, b, st>>>(t);
  } else if (kind == 1) {
    k_edge_trsm<<<ntasks, kThreads, 0, st>>>(t);
  } else {
    if ((e = prep(k_edge_right, b))) return e;
    k_edge_right<<<ntasks, kThreads, b, st>>>(t);
  }
  return last();
}

cudaError_t launch_rrqr(const RrqrTask* t, const RrqrSrc* s, int ntasks, int cs, int mmax, int wloc_max, double tol,
                        double pivot_rtol, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_rrqr")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(kRed + kNB + 2 * (size_t)std::max(mmax, 1)) + sizeof(int) * (size_t)(wloc_max + 1);
  cudaError_t e = prep(k_rrqr, b);
  if (e) return e;
  return launch_clustered(k_rrqr, ntasks, cs, b, st, t, s, tol, pivot_rtol, cs, wloc_max);
}

cudaError_t launch_merge(const MergeTask* t, int ntasks, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_merge")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  counted();
  k_merge<<<ntasks, 256, 0, st>>>(t);
  return last();
}

cudaError_t launch_fwd_elim(const FwdElimTask* t, const FwdOut* o, int ntasks, int nmax, int mmax, int* ticket,
                            int* status, long long spin_limit, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_fwd_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(2 * kNB + (size_t)std::max(nmax, 1) + (size_t)std::max(mmax, 1));
  cudaError_t e = prep(k_fwd_elim, b);
  if (e) return e;
  counted();
  k_fwd_elim<<<ntasks, kThreads, b, st>>>(t, o, ntasks, ticket, status, spin_limit, nmax);
  return last();
}

cudaError_t launch_fwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_fwd_spars")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(2 * kNB + (size_t)nmax);
  cudaError_t e = prep(k_fwd_spars, b);
  if (e) return e;
  counted();
  k_fwd_spars<<<ntasks, kThreads, b, st>>>(t);
  return last();
}

cudaError_t launch_bwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_bwd_spars")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(2 * kNB + 32 + (size_t)nmax);
  cudaError_t e = prep(k_bwd_spars, b);
  if (e) return e;
  counted();
  k_bwd_spars<<<ntasks, kThreads, b, st>>>(t);
  return last();
}

cudaError_t launch_bwd_elim(const BwdElimTask* t, const BwdIn* in, int ntasks, int nmax, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_bwd_elim")) return pre;
  if (ntasks <= 0) return cudaSuccess;
  const size_t b = smem_bytes(32 + (size_t)nmax);
  cudaError_t e = prep(k_bwd_elim, b);
  if (e) return e;
  counted();
  k_bwd_elim<<<ntasks, kThreads, b, st>>>(t, in);
  return last();
}

cudaError_t launch_copy_idx(int n, const int* src, const int* dst, double* x, cudaStream_t st) {
  if (cudaError_t pre = begin("launch_copy_idx")) return pre;
  if (n <= 0) return cudaSuccess;
  counted();
  k_copy_idx<<<grid_for(n), 256, 0, st>>>(n, src, dst, x);
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
