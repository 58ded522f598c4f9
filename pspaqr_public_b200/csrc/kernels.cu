// kernels.cu -- grouped FP64 kernels of the factorization, the preconditioner
// apply and the Krylov loop.  One CTA per task; tasks of a launch touch
// disjoint blocks except where noted (forward elimination sweep).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "dense.cuh"
#include "kernels.hpp"
#include "tasks.hpp"

namespace spq {
namespace {

using dev::kThreads;
using dev::kWarps;

constexpr int kRed = 16;        // reduction scratch (doubles)
constexpr int kWcap = 6144;     // W scratch (doubles) of the blocked reflector applies

// W scratch of `wcap` doubles holds W and W2 (k x chunk each); the launcher
// guarantees wcap >= 2*k for every k of the launch.
__device__ __forceinline__ int chunk_for(int k, int wcap) {
  int c = (wcap / 2) / (k > 0 ? k : 1);
  return c < 1 ? 1 : c;
}

// ------------------------------------------------------------ assembly
__global__ void k_scatter(int nnz, const double* __restrict__ val, double* const* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) *dst[i] = val[i];
}

// ------------------------------------------------------------ elimination
__global__ void __launch_bounds__(kThreads) k_elim(const ElimTask* __restrict__ tasks, const ElimOut* __restrict__ outs) {
  extern __shared__ double sm[];
  const ElimTask t = tasks[blockIdx.x];
  double* red = sm;
  double* tau = sm + kRed;
  double* tmp = tau + t.n;
  dev::geqrt(t.S, t.n, t.n, t.n, t.T, t.n, tau, red, tmp);
  for (int o = t.out_begin; o < t.out_end; ++o) {
    const ElimOut e = outs[o];
    dev::tpqrt(t.S, t.n, e.B, e.m, e.m, t.n, e.T, t.n, tau, red, tmp);
  }
}

__global__ void __launch_bounds__(kThreads) k_update(const UpdTask* __restrict__ tasks, const UpdOp* __restrict__ ops,
                                                     int wcap) {
  extern __shared__ double sm[];
  const UpdTask t = tasks[blockIdx.x];
  for (int o = t.op_begin; o < t.op_end; ++o) {
    const UpdOp op = ops[o];
    if (op.kind == 0)
      dev::apply_qt_left(op.V, op.ldv, op.T, op.k, op.k, op.A, op.lda, op.m, t.ncols, sm, chunk_for(op.k, wcap));
    else
      dev::apply_tpqt_left(op.V, op.ldv, op.T, op.k, op.k, op.A, op.lda, op.B, op.ldb, op.m, t.ncols, sm,
                           chunk_for(op.k, wcap));
  }
}

// ------------------------------------------------------------ scaling
__global__ void __launch_bounds__(kThreads) k_scale(const ScaleTask* __restrict__ tasks) {
  extern __shared__ double sm[];
  const ScaleTask t = tasks[blockIdx.x];
  double* red = sm;
  double* tau = sm + kRed;
  double* tmp = tau + t.n;
  dev::geqrt(t.S, t.n, t.n, t.n, t.T, t.n, tau, red, tmp);
}

__global__ void __launch_bounds__(kThreads) k_scale_edge(const ScaleEdgeTask* __restrict__ tasks, int wcap) {
  extern __shared__ double sm[];
  const ScaleEdgeTask t = tasks[blockIdx.x];
  if (t.Qr) dev::apply_qt_left(t.Qr, t.ldqr, t.Tr, t.ldqr, t.m, t.A, t.lda, t.m, t.nc, sm, chunk_for(t.m, wcap));
  if (t.Qc) dev::trsm_right_upper(t.Qc, t.ldqc, t.A, t.lda, t.m, t.nc);
}

// ------------------------------------------------------------ RRQR
// Column-pivoted Householder QR of C (m x w), stopped at the first i >= 1 with
// |R(i,i)| / |R(0,0)| < tol (util.cpp:830-851 choose_rank on the dgeqp3
// diagonal).  Pivoting and norm downdating follow LAPACK dlaqp2.
__global__ void __launch_bounds__(kThreads) k_rrqr(const RrqrTask* __restrict__ tasks,
                                                   const RrqrSrc* __restrict__ srcs, double tol,
                                                   double pivot_rtol) {
  extern __shared__ double sm[];
  __shared__ int s_piv;
  __shared__ double s_v[kWarps];
  __shared__ int s_i[kWarps];
  const RrqrTask t = tasks[blockIdx.x];
  const int m = t.m, w = t.w;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* C = t.C;
  double* red = sm;
  double* tau = sm + kRed;
  double* tmp = tau + (m > 0 ? m : 1);
  // assemble C
  int col = 0;
  for (int s = t.src_begin; s < t.src_end; ++s) {
    const RrqrSrc src = srcs[s];
    if (src.transpose) {
      for (int idx = threadIdx.x; idx < src.rows * m; idx += kThreads) {
        const int i = idx % src.rows, j = idx / src.rows;
        C[j + (size_t)(col + i) * m] = src.A[i + (size_t)j * src.lda];
      }
      col += src.rows;
    } else {
      for (int idx = threadIdx.x; idx < m * src.cols; idx += kThreads) {
        const int i = idx % m, j = idx / m;
        C[i + (size_t)(col + j) * m] = src.A[i + (size_t)j * src.lda];
      }
      col += src.cols;
    }
  }
  __syncthreads();
  double* vn1 = t.vn;
  double* vn2 = t.vn + w;
  for (int j = warp; j < w; j += kWarps) {
    const double* cj = C + (size_t)j * m;
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += cj[i] * cj[i];
    s = sqrt(dev::warp_sum(s));
    if (lane == 0) {
      vn1[j] = s;
      vn2[j] = s;
      t.jpvt[j] = j;
    }
  }
  __syncthreads();
  const int kmin = m < w ? m : w;
  const double tol3z = sqrt(1.1102230246251565e-16);
  int rank = kmin;
  double r00 = 0.0;
  for (int i = 0; i < kmin; ++i) {
    // pivot = first column whose partial norm is within pivot_rtol of the
    // largest remaining one (pivot_rtol = 0: LAPACK idamax, first maximum)
    double bv = -1.0;
    for (int j = i + threadIdx.x; j < w; j += kThreads) bv = fmax(bv, vn1[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, o));
    if (lane == 0) s_v[warp] = bv;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = s_v[0];
      for (int q = 1; q < kWarps; ++q) v = fmax(v, s_v[q]);
      s_v[0] = v;
    }
    __syncthreads();
    const double thr = s_v[0] * (1.0 - pivot_rtol);
    int bi = w;
    for (int j = i + threadIdx.x; j < w; j += kThreads)
      if (vn1[j] >= thr) {
        bi = j;
        break;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bi = min(bi, __shfl_xor_sync(0xffffffffu, bi, o));
    __syncthreads();
    if (lane == 0) s_i[warp] = bi;
    __syncthreads();
    if (threadIdx.x == 0) {
      int id = s_i[0];
      for (int q = 1; q < kWarps; ++q) id = min(id, s_i[q]);
      s_piv = (id >= i && id < w) ? id : i;  // no finite maximum (NaN norms): keep column i
    }
    __syncthreads();
    const int pvt = s_piv;
    if (pvt != i) {
      double* ci = C + (size_t)i * m;
      double* cp = C + (size_t)pvt * m;
      for (int r = threadIdx.x; r < m; r += kThreads) {
        const double a = ci[r];
        ci[r] = cp[r];
        cp[r] = a;
      }
      if (threadIdx.x == 0) {
        vn1[pvt] = vn1[i];
        vn2[pvt] = vn2[i];
        const int ip = t.jpvt[pvt];
        t.jpvt[pvt] = t.jpvt[i];
        t.jpvt[i] = ip;
      }
      __syncthreads();
    }
    double* ci = C + (size_t)i * m;
    double s = 0.0;
    for (int r = i + 1 + threadIdx.x; r < m; r += kThreads) s += ci[r] * ci[r];
    s = dev::cta_sum(s, red);
    const double alpha = ci[i];
    double beta, scal;
    const double ti = dev::house(alpha, s, &beta, &scal);
    const double absb = fabs(beta);
    if (i == 0) r00 = absb;
    else if (!(absb / r00 >= tol)) {
      rank = i;
      break;
    }
    if (ti != 0.0)
      for (int r = i + 1 + threadIdx.x; r < m; r += kThreads) ci[r] *= scal;
    __syncthreads();
    if (threadIdx.x == 0) {
      ci[i] = beta;
      tau[i] = ti;
      t.tau[i] = ti;
    }
    for (int j = i + 1 + warp; j < w; j += kWarps) {
      double* cj = C + (size_t)j * m;
      double d = lane == 0 ? cj[i] : 0.0;
      for (int r = i + 1 + lane; r < m; r += 32) d += ci[r] * cj[r];
      d = dev::warp_sum(d) * ti;
      const double top = __shfl_sync(0xffffffffu, cj[i], 0) - d;
      __syncwarp();
      if (lane == 0) cj[i] = top;
      for (int r = i + 1 + lane; r < m; r += 32) cj[r] -= ci[r] * d;
      __syncwarp();
      const double v1 = vn1[j];
      if (v1 != 0.0) {
        double temp = fabs(top) / v1;
        temp = 1.0 - temp * temp;
        temp = temp < 0.0 ? 0.0 : temp;
        const double q = v1 / vn2[j];
        const double temp2 = temp * q * q;
        if (temp2 <= tol3z) {
          double nn = 0.0;
          for (int r = i + 1 + lane; r < m; r += 32) nn += cj[r] * cj[r];
          nn = (i + 1 < m) ? sqrt(dev::warp_sum(nn)) : 0.0;
          if (lane == 0) {
            vn1[j] = nn;
            vn2[j] = nn;
          }
        } else if (lane == 0) {
          vn1[j] = v1 * sqrt(temp);
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
  __syncthreads();
  // block factor of the kept reflectors
  const int npairs = rank * (rank - 1) / 2;
  for (int p = warp; p < npairs; p += kWarps) {
    int j = (int)((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
    while (j * (j - 1) / 2 > p) --j;
    while ((j + 1) * j / 2 <= p) ++j;
    const int l = p - j * (j - 1) / 2;
    const double* cl = C + (size_t)l * m;
    const double* cj = C + (size_t)j * m;
    double d = lane == 0 ? cl[j] : 0.0;
    for (int r = j + 1 + lane; r < m; r += 32) d += cl[r] * cj[r];
    d = dev::warp_sum(d);
    if (lane == 0) t.T[l + (size_t)j * m] = d;
  }
  __syncthreads();
  dev::larft_from_gram(t.T, m, rank, tau, tmp);
  if (threadIdx.x == 0) *t.rank = rank;
}

__global__ void __launch_bounds__(kThreads) k_spars_edge(const SparsEdgeTask* __restrict__ tasks, int wcap) {
  extern __shared__ double sm[];
  const SparsEdgeTask t = tasks[blockIdx.x];
  const int rc = t.Vc ? *t.rank_c : t.nc;
  if (t.Vc) dev::apply_q_right(t.Vc, t.ldvc, t.Tc, t.ldvc, rc, t.A, t.lda, t.m, t.nc, sm, chunk_for(rc, wcap));
  if (t.Vr) {
    const int rr = *t.rank_r;
    dev::apply_qt_left(t.Vr, t.ldvr, t.Tr, t.ldvr, rr, t.A, t.lda, t.m, rc, sm, chunk_for(rr, wcap));
  }
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
                                                       int* status, long long spin_limit) {
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
  double* xc = sm;
  double* w = xc + t.n;
  double* xn = w + 2 * (t.n > 0 ? t.n : 1);
  for (int i = threadIdx.x; i < t.n; i += kThreads) xc[i] = __ldcg(t.x + i);
  __syncthreads();
  dev::apply_qt_vec(t.S, t.n, t.T, t.n, t.n, xc, t.n, w);
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
    dev::apply_tpqt_left(e.V, e.m, e.T, t.n, t.n, xc, t.n, xn, e.m, e.m, 1, w, 1);
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
  double* x = sm;
  double* w = sm + t.n;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = t.x[i];
  __syncthreads();
  dev::apply_qt_vec(t.Qs, t.n, t.Ts, t.n, t.n, x, t.n, w);
  dev::apply_qt_vec(t.V, t.n, t.T, t.n, *t.rank, x, t.n, w);
  for (int i = threadIdx.x; i < t.n; i += kThreads) t.x[i] = x[i];
}

__global__ void __launch_bounds__(kThreads) k_bwd_spars(const FwdSparsTask* __restrict__ tasks) {
  extern __shared__ double sm[];
  const FwdSparsTask t = tasks[blockIdx.x];
  double* x = sm;
  double* w = sm + t.n;
  double* xs = w + 2 * t.n;
  for (int i = threadIdx.x; i < t.n; i += kThreads) x[i] = t.x[i];
  __syncthreads();
  dev::apply_q_vec(t.V, t.n, t.T, t.n, *t.rank, x, t.n, w);
  dev::trsv_upper(t.Qs, t.n, x, t.n, xs);
  for (int i = threadIdx.x; i < t.n; i += kThreads) t.x[i] = x[i];
}

__global__ void __launch_bounds__(kThreads) k_bwd_elim(const BwdElimTask* __restrict__ tasks,
                                                       const BwdIn* __restrict__ ins) {
  extern __shared__ double sm[];
  const BwdElimTask t = tasks[blockIdx.x];
  double* x = sm;
  double* xs = sm + t.n;
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
#define SPQ_SET_SMEM(kern, bytes)                                                              \
  do {                                                                                         \
    if ((bytes) > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(bytes)); \
  } while (0)

void launch_scatter(int nnz, const double* val, double* const* dst, cudaStream_t st) {
  if (nnz > 0) k_scatter<<<grid_for(nnz), 256, 0, st>>>(nnz, val, dst);
}
void launch_elim(const ElimTask* t, const ElimOut* o, int ntasks, int nmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(kRed + 2 * (size_t)nmax);
  SPQ_SET_SMEM(k_elim, b);
  k_elim<<<ntasks, kThreads, b, st>>>(t, o);
}
inline int wcap_for(int kmax) { return std::max(kWcap, 2 * std::max(kmax, 1)); }

void launch_update(const UpdTask* t, const UpdOp* o, int ntasks, int kmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  const int wcap = wcap_for(kmax);
  size_t b = smem_bytes(wcap);
  SPQ_SET_SMEM(k_update, b);
  k_update<<<ntasks, kThreads, b, st>>>(t, o, wcap);
}
void launch_scale(const ScaleTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(kRed + 2 * (size_t)nmax);
  SPQ_SET_SMEM(k_scale, b);
  k_scale<<<ntasks, kThreads, b, st>>>(t);
}
void launch_scale_edge(const ScaleEdgeTask* t, int ntasks, int kmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  const int wcap = wcap_for(kmax);
  size_t b = smem_bytes(wcap);
  SPQ_SET_SMEM(k_scale_edge, b);
  k_scale_edge<<<ntasks, kThreads, b, st>>>(t, wcap);
}
void launch_rrqr(const RrqrTask* t, const RrqrSrc* s, int ntasks, int mmax, double tol, double pivot_rtol,
                 cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(kRed + 2 * (size_t)(mmax > 0 ? mmax : 1));
  SPQ_SET_SMEM(k_rrqr, b);
  k_rrqr<<<ntasks, kThreads, b, st>>>(t, s, tol, pivot_rtol);
}
void launch_spars_edge(const SparsEdgeTask* t, int ntasks, int kmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  const int wcap = wcap_for(kmax);
  size_t b = smem_bytes(wcap);
  SPQ_SET_SMEM(k_spars_edge, b);
  k_spars_edge<<<ntasks, kThreads, b, st>>>(t, wcap);
}
void launch_merge(const MergeTask* t, int ntasks, cudaStream_t st) {
  if (ntasks > 0) k_merge<<<ntasks, 256, 0, st>>>(t);
}
void launch_fwd_elim(const FwdElimTask* t, const FwdOut* o, int ntasks, int nmax, int mmax, int* ticket, int* status,
                     long long spin_limit, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(3 * (size_t)(nmax > 0 ? nmax : 1) + (size_t)(mmax > 0 ? mmax : 1));
  SPQ_SET_SMEM(k_fwd_elim, b);
  k_fwd_elim<<<ntasks, kThreads, b, st>>>(t, o, ntasks, ticket, status, spin_limit);
}
void launch_fwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(3 * (size_t)nmax);
  SPQ_SET_SMEM(k_fwd_spars, b);
  k_fwd_spars<<<ntasks, kThreads, b, st>>>(t);
}
void launch_bwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes(3 * (size_t)nmax + 32);
  SPQ_SET_SMEM(k_bwd_spars, b);
  k_bwd_spars<<<ntasks, kThreads, b, st>>>(t);
}
void launch_bwd_elim(const BwdElimTask* t, const BwdIn* in, int ntasks, int nmax, cudaStream_t st) {
  if (ntasks <= 0) return;
  size_t b = smem_bytes((size_t)nmax + 32);
  SPQ_SET_SMEM(k_bwd_elim, b);
  k_bwd_elim<<<ntasks, kThreads, b, st>>>(t, in);
}
void launch_copy_idx(int n, const int* src, const int* dst, double* x, cudaStream_t st) {
  if (n > 0) k_copy_idx<<<grid_for(n), 256, 0, st>>>(n, src, dst, x);
}
void launch_spmv(int n, const int* rowptr, const int* col, const double* val, const double* x, double* y,
                 cudaStream_t st) {
  k_spmv<<<grid_for(n), 256, 0, st>>>(n, rowptr, col, val, x, y);
}
int mgs_grid(int n) { return grid_for(n, kThreads * 4, 148 * 4); }
void launch_mgs_step(int n, double* q, const double* Qprev, const double* hprev, const double* Qi, double* partial,
                     unsigned int* done, double* out, int take_sqrt, cudaStream_t st) {
  k_mgs_step<<<mgs_grid(n), kThreads, 0, st>>>(n, q, Qprev, hprev, Qi, partial, done, out, take_sqrt);
}
void launch_scale_copy(int n, const double* src, const double* s, double* dst, cudaStream_t st) {
  k_scale_copy<<<grid_for(n), 256, 0, st>>>(n, src, s, dst);
}
void launch_combine(int n, int k, const double* Q, size_t ldq, const double* y, double* x, cudaStream_t st) {
  k_combine<<<grid_for(n), 256, 0, st>>>(n, k, Q, ldq, y, x);
}
void launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st) {
  k_sub<<<grid_for(n), 256, 0, st>>>(n, a, b, c);
}

}  // namespace spq
