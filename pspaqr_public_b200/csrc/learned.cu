// learned.cu -- kernels of the learned-rank sparsification and of the rank
// MLP's training (see learned.hpp for the method).
//
// Random test matrices Omega are Rademacher (+-1) from a counter-based hash
// (splitmix64 finaliser, Steele, Lea & Flood 2014) of (seed, row, column
// block): one 64-bit hash gives the signs of 64 consecutive columns, so the
// sketch never stores Omega.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "dense.cuh"
#include "kernels.hpp"
#include "learned.hpp"

namespace spq {
namespace {

constexpr int kT = 256;  // threads of the per-task and GEMM kernels
constexpr int kTile = 64;
constexpr int kKStep = 32;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// signs of Omega(j, 64 b .. 64 b + 63), bit t set = +1
__device__ __forceinline__ unsigned long long omega_bits(unsigned long long seed, int j, int b) {
  return mix64(seed ^ mix64(((unsigned long long)j << 16) | (unsigned long long)b));
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sumd(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum / max over kT threads through `red` (kT / 32 doubles).
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sumd(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int q = 0; q < kT / 32; ++q) s += red[q];
  __syncthreads();
  return s;
}
__device__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = red[0];
  for (int q = 1; q < kT / 32; ++q) s = fmax(s, red[q]);
  __syncthreads();
  return s;
}

// ---------------------------------------------------------------- features
// Signs of the 4-column feature sketch of column j: bit c set = +1.
__device__ __forceinline__ unsigned feat_signs(unsigned long long seed, int j) {
  return (unsigned)(omega_bits(seed ^ 0x5DEECE66Dull, j, 0) & 15u);
}

// One CTA per block of kFeatCols columns (tile.c0): squared norms of its
// columns (a thread per column, eight rows in flight), then its part of the
// 4-column Rademacher sketch (a warp per row, the block's columns over the
// lanes) into y4p[(block * 4 + c) * m + r].
__global__ void __launch_bounds__(kT) k_feature_blocks(const SketchTask* __restrict__ tasks,
                                                       const GemmTile* __restrict__ blocks) {
  const GemmTile g = blocks[blockIdx.x];
  const SketchTask t = tasks[g.task];
  const int m = t.m, w = t.w;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = g.c0 + threadIdx.x;
  if (j < w) {
    const double* col = t.C + j;
    double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int r = 0;
    for (; r + 8 <= m; r += 8) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldg(col + (size_t)(r + u) * t.ldw);
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] += v[u] * v[u];
    }
    for (; r < m; ++r) {
      const double v = __ldg(col + (size_t)r * t.ldw);
      a[0] += v * v;
    }
    t.cn2[j] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
  }
  constexpr int kPer = kFeatCols / 32;
  unsigned sg[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int jj = g.c0 + lane + 32 * u;
    sg[u] = jj < w ? feat_signs(t.seed, jj) : 0u;
  }
  const int blk = g.c0 / kFeatCols;
  for (int r = warp; r < m; r += kT / 32) {
    const double* row = t.C + (size_t)r * t.ldw;
    double y[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int jj = g.c0 + lane + 32 * u;
      const double v = jj < w ? __ldg(row + jj) : 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) y[c] += ((sg[u] >> c) & 1u) ? v : -v;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) y[c] = warp_sumd(y[c]);
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < 4; ++c) t.y4p[((size_t)blk * 4 + c) * m + r] = y[c];
  }
}

// One CTA per interface: the sketch (partials summed in block order), its QR
// diagonal, the norm statistics and the 11 features.  Dynamic shared memory:
// 4 * mmax doubles.
__global__ void __launch_bounds__(kT) k_rank_features(const SketchTask* __restrict__ tasks, double tol) {
  extern __shared__ double sm[];
  __shared__ double red[kT / 32];
  const SketchTask t = tasks[blockIdx.x];
  const int m = t.m, w = t.w;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* y4 = sm;
  const int nblk = (w + kFeatCols - 1) / kFeatCols;
  for (int e = threadIdx.x; e < 4 * m; e += kT) {
    const int c = e / m, r = e % m;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += t.y4p[((size_t)b * 4 + c) * m + r];
    y4[e] = s;
  }
  double cmax = 0.0, fro = 0.0;
  for (int j = threadIdx.x; j < w; j += kT) {
    const double s = t.cn2[j];
    cmax = fmax(cmax, s);
    fro += s;
  }
  cmax = block_max(cmax, red);
  fro = block_sum(fro, red);
  // counts of columns above fractions of the largest norm
  const double thr[3] = {tol * tol * cmax, 0.01 * cmax, 0.25 * cmax};
  int cnt[3] = {0, 0, 0};
  for (int j = threadIdx.x; j < w; j += kT) {
    const double c = t.cn2[j];
#pragma unroll
    for (int q = 0; q < 3; ++q) cnt[q] += c >= thr[q] ? 1 : 0;
  }
  double cq[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) cq[q] = block_sum((double)cnt[q], red);
  __syncthreads();
  // diagonal of R in a QR of the sketch (modified Gram-Schmidt, warp 0)
  double d[4] = {0, 0, 0, 0};
  if (warp == 0) {
    for (int c = 0; c < 4; ++c) {
      double* yc = y4 + (size_t)c * m;
      for (int p = 0; p < c; ++p) {
        const double* yp = y4 + (size_t)p * m;
        double s = 0.0;
        for (int r = lane; r < m; r += 32) s += yp[r] * yc[r];
        s = warp_sumd(s);
        for (int r = lane; r < m; r += 32) yc[r] -= s * yp[r];
        __syncwarp();
      }
      double s = 0.0;
      for (int r = lane; r < m; r += 32) s += yc[r] * yc[r];
      s = sqrt(warp_sumd(s));
      d[c] = s;
      const double inv = s > 0.0 ? 1.0 / s : 0.0;
      for (int r = lane; r < m; r += 32) yc[r] *= inv;
      __syncwarp();
    }
  }
  if (threadIdx.x == 0) {
    const int kmin = m < w ? m : w;
    const double km = kmin > 0 ? (double)kmin : 1.0;
    float* f = t.feat;
    f[0] = (float)log2((double)m + 1.0);
    f[1] = (float)log2((double)w + 1.0);
    f[2] = (float)log10(tol);
    f[3] = (float)fmin(1.0, cq[0] / km);
    f[4] = (float)fmin(1.0, cq[1] / km);
    f[5] = (float)fmin(1.0, cq[2] / km);
    f[6] = (float)fmin(10.0, cmax > 0.0 ? fro / (cmax * km) : 0.0);
    for (int c = 1; c < 4; ++c) f[6 + c] = (float)(d[0] > 0.0 ? log10(fmax(d[c] / d[0], 1e-12)) : -12.0);
    f[10] = (float)t.level;
    *t.cmax2 = cmax;
  }
}

// ---------------------------------------------------------------- MLP
__device__ __forceinline__ float sigmoidf(float z) { return 1.0f / (1.0f + expf(-z)); }

constexpr int kOffB1 = kMlpHidden * kRankFeatures;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden;

// forward pass of one standardised feature vector
__device__ float mlp_forward(const float* __restrict__ P, const float* x) {
  float h1[kMlpHidden];
#pragma unroll 4
  for (int i = 0; i < kMlpHidden; ++i) {
    float s = P[kOffB1 + i];
#pragma unroll
    for (int f = 0; f < kRankFeatures; ++f) s += P[i * kRankFeatures + f] * x[f];
    h1[i] = s > 0.0f ? s : 0.0f;
  }
  float z = P[kOffB3];
  for (int i = 0; i < kMlpHidden; ++i) {
    float s = P[kOffB2 + i];
#pragma unroll 8
    for (int j = 0; j < kMlpHidden; ++j) s += P[kOffW2 + i * kMlpHidden + j] * h1[j];
    z += P[kOffW3 + i] * (s > 0.0f ? s : 0.0f);
  }
  return sigmoidf(z);
}

__global__ void k_rank_predict(const SketchTask* __restrict__ tasks, int ntasks, RankModel model) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntasks) return;
  const SketchTask t = tasks[q];
  const int kmin = t.m < t.w ? t.m : t.w;
  float x[kRankFeatures];
  for (int f = 0; f < kRankFeatures; ++f) x[f] = (t.feat[f] - model.mean[f]) / model.stdev[f];
  float p = mlp_forward(model.params, x) + model.margin;
  p = p < 1.0f ? p : 1.0f;
  int ell = (int)ceilf(p * (float)kmin) + model.oversample;
  ell = ell < 1 ? 1 : ell;
  *t.ell = kmin < ell ? kmin : ell;
}

__global__ void k_mlp_predict(const float* __restrict__ P, const float* __restrict__ X, int n, float* out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[kRankFeatures];
  for (int f = 0; f < kRankFeatures; ++f) x[f] = X[(size_t)s * kRankFeatures + f];
  out[s] = mlp_forward(P, x);
}

// Loss and gradient partials of 64 samples per block (128 threads):
// loss = sum_s (sigmoid(z_s) - y_s)^2 / n.  Activations stay in shared
// memory; every parameter's partial is a sum over the block's samples in
// sample order, written to part[block * (kMlpParams + 1) + p] (loss last).
constexpr int kMlpBatch = 64;
constexpr int kMlpThreads = 128;
constexpr size_t kMlpSmem =
    sizeof(float) * ((size_t)kMlpBatch * kRankFeatures + 3 * (size_t)kMlpBatch * kMlpHidden + kMlpBatch +
                     (size_t)kMlpHidden * kMlpHidden);

__global__ void __launch_bounds__(kMlpThreads) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ X,
                                                          const float* __restrict__ y, int n, float* part) {
  extern __shared__ float fs[];
  float* Xs = fs;                                  // 64 x F
  float* H1 = Xs + kMlpBatch * kRankFeatures;      // 64 x 64
  float* H2 = H1 + kMlpBatch * kMlpHidden;         // 64 x 64, then dL/dpre2
  float* D1 = H2 + kMlpBatch * kMlpHidden;         // 64 x 64: dL/dpre1
  float* dz = D1 + kMlpBatch * kMlpHidden;         // 64
  float* W2 = dz + kMlpBatch;                      // 64 x 64
  const int s0 = blockIdx.x * kMlpBatch;
  for (int i = threadIdx.x; i < kMlpHidden * kMlpHidden; i += kMlpThreads) W2[i] = P[kOffW2 + i];
  for (int i = threadIdx.x; i < kMlpBatch * kRankFeatures; i += kMlpThreads) {
    const int s = s0 + i / kRankFeatures;
    Xs[i] = s < n ? X[(size_t)s0 * kRankFeatures + i] : 0.0f;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kMlpBatch * kMlpHidden; idx += kMlpThreads) {
    const int s = idx / kMlpHidden, i = idx % kMlpHidden;
    float a = P[kOffB1 + i];
    for (int f = 0; f < kRankFeatures; ++f) a += P[i * kRankFeatures + f] * Xs[s * kRankFeatures + f];
    H1[idx] = a > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kMlpBatch * kMlpHidden; idx += kMlpThreads) {
    const int s = idx / kMlpHidden, i = idx % kMlpHidden;
    float a = P[kOffB2 + i];
    for (int j = 0; j < kMlpHidden; ++j) a += W2[i * kMlpHidden + j] * H1[s * kMlpHidden + j];
    H2[idx] = a > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  float* out = part + (size_t)blockIdx.x * (kMlpParams + 1);
  if (threadIdx.x < kMlpBatch) {
    const int s = threadIdx.x;
    float z = P[kOffB3];
    for (int i = 0; i < kMlpHidden; ++i) z += P[kOffW3 + i] * H2[s * kMlpHidden + i];
    const float p = sigmoidf(z);
    const bool valid = s0 + s < n;
    const float diff = valid ? p - y[s0 + s] : 0.0f;
    dz[s] = valid ? 2.0f * diff * p * (1.0f - p) / (float)n : 0.0f;
    D1[s] = diff * diff;  // per-sample loss; D1 is rewritten by the backward pass
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = 0.0f;
    for (int s = 0; s < kMlpBatch; ++s) l += D1[s];
    out[kMlpParams] = l / (float)n;
  }
  // layer 3
  for (int i = threadIdx.x; i <= kMlpHidden; i += kMlpThreads) {
    float g = 0.0f;
    for (int s = 0; s < kMlpBatch; ++s) g += dz[s] * (i < kMlpHidden ? H2[s * kMlpHidden + i] : 1.0f);
    out[i < kMlpHidden ? kOffW3 + i : kOffB3] = g;
  }
  __syncthreads();
  // dL/dpre2 in place of H2
  for (int idx = threadIdx.x; idx < kMlpBatch * kMlpHidden; idx += kMlpThreads) {
    const int s = idx / kMlpHidden, i = idx % kMlpHidden;
    H2[idx] = H2[idx] > 0.0f ? dz[s] * P[kOffW3 + i] : 0.0f;
  }
  __syncthreads();
  // dL/dpre1
  for (int idx = threadIdx.x; idx < kMlpBatch * kMlpHidden; idx += kMlpThreads) {
    const int s = idx / kMlpHidden, j = idx % kMlpHidden;
    float a = 0.0f;
    if (H1[idx] > 0.0f)
      for (int i = 0; i < kMlpHidden; ++i) a += W2[i * kMlpHidden + j] * H2[s * kMlpHidden + i];
    D1[idx] = a;
  }
  __syncthreads();
  // layer 2 and layer 1
  for (int p = threadIdx.x; p < kMlpHidden * kMlpHidden + kMlpHidden; p += kMlpThreads) {
    float g = 0.0f;
    if (p < kMlpHidden * kMlpHidden) {
      const int i = p / kMlpHidden, j = p % kMlpHidden;
      for (int s = 0; s < kMlpBatch; ++s) g += H2[s * kMlpHidden + i] * H1[s * kMlpHidden + j];
      out[kOffW2 + p] = g;
    } else {
      const int i = p - kMlpHidden * kMlpHidden;
      for (int s = 0; s < kMlpBatch; ++s) g += H2[s * kMlpHidden + i];
      out[kOffB2 + i] = g;
    }
  }
  for (int p = threadIdx.x; p < kMlpHidden * kRankFeatures + kMlpHidden; p += kMlpThreads) {
    float g = 0.0f;
    if (p < kMlpHidden * kRankFeatures) {
      const int i = p / kRankFeatures, f = p % kRankFeatures;
      for (int s = 0; s < kMlpBatch; ++s) g += D1[s * kMlpHidden + i] * Xs[s * kRankFeatures + f];
      out[p] = g;
    } else {
      const int i = p - kMlpHidden * kRankFeatures;
      for (int s = 0; s < kMlpBatch; ++s) g += D1[s * kMlpHidden + i];
      out[kOffB1 + i] = g;
    }
  }
}

// grad[p] = sum over blocks (in block order) of the partials; loss likewise
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblocks, float* grad, float* loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kMlpParams) return;
  float s = 0.0f;
  for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * (kMlpParams + 1) + p];
  if (p < kMlpParams) grad[p] = s;
  else *loss = s;
}

__global__ void k_mlp_adam(float* P, const float* __restrict__ g, float* m1, float* m2, float lr, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float b1 = 0.9f, b2 = 0.999f;
  const float a = b1 * m1[p] + (1.0f - b1) * g[p];
  const float v = b2 * m2[p] + (1.0f - b2) * g[p] * g[p];
  m1[p] = a;
  m2[p] = v;
  P[p] -= lr * (a / c1) / (sqrtf(v / c2) + 1e-8f);
}

// ---------------------------------------------------------------- sketch / projection GEMMs
// 64 x 64 output tile per CTA, k-steps of 32, each thread a 4 x 4 block of
// outputs at rows ty + 16 a (the sketch: rows 4 ty + a), columns tx + 16 b.
// In the sketch the next
// k-step's C tile is copied into the other half of a double buffer with
// cp.async while the current one is multiplied (the projection loads each
// step's tiles directly: its two tiles in a double buffer would halve the
// CTAs per SM); every output sums its k terms in ascending order.
__global__ void __launch_bounds__(kT) k_sketch(const SketchTask* __restrict__ tasks,
                                               const GemmTile* __restrict__ tiles) {
  // C(r0 + rr, j0 + jj) at As[.][jj][rr]: a thread's four consecutive rows are
  // two 16-byte loads (rows of kTile + 2 doubles keep them 16-byte aligned)
  __shared__ __align__(16) double As[2][kKStep][kTile + 2];
  __shared__ unsigned long long Ws[2][kKStep];  // signs of Omega(j0 + jj, c0 .. c0 + 63)
  const GemmTile g = tiles[blockIdx.x];
  const SketchTask t = tasks[g.task];
  const int ell = *t.ell;
  if (g.c0 >= ell) return;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int nsteps = (t.w + kKStep - 1) / kKStep;
  auto load = [&](int s, int b) {
    const int j0 = s * kKStep;
    for (int e = threadIdx.x; e < kTile * kKStep; e += kT) {
      const int rr = e / kKStep, jj = e % kKStep;
      const int r = g.r0 + rr, j = j0 + jj;
      if (r < t.m && j < t.w) dev::cp_async_elem(&As[b][jj][rr], t.C + (size_t)r * t.ldw + j);
      else As[b][jj][rr] = 0.0;
    }
    if (threadIdx.x < kKStep) Ws[b][threadIdx.x] = omega_bits(t.seed, j0 + threadIdx.x, g.c0 >> 6);
    dev::cp_async_commit();
  };
  double acc[4][4] = {};
  if (nsteps > 0) load(0, 0);
  for (int s = 0; s < nsteps; ++s) {
    const int b = s & 1;
    if (s + 1 < nsteps) {
      load(s + 1, b ^ 1);
      dev::cp_async_wait<1>();
    } else {
      dev::cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll 8
    for (int jj = 0; jj < kKStep; ++jj) {
      const unsigned long long w = Ws[b][jj];
      const double2 a01 = *reinterpret_cast<const double2*>(&As[b][jj][4 * ty]);
      const double2 a23 = *reinterpret_cast<const double2*>(&As[b][jj][4 * ty + 2]);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y};
      double bq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bq[q] = ((w >> (tx + 16 * q)) & 1ull) ? 1.0 : -1.0;
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * bq[q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int r = g.r0 + 4 * ty + p;
    if (r >= t.m) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = g.c0 + tx + 16 * q;
      if (c < ell) t.Y[(size_t)r * t.ldy + c] = acc[p][q];
    }
  }
}

// B(l, j) = sum_r Q(r, l) C(r, j); tile rows l (basis vectors), columns j
__global__ void __launch_bounds__(kT) k_project(const SketchTask* __restrict__ tasks,
                                                const GemmTile* __restrict__ tiles) {
  __shared__ double As[kKStep][kTile + 1];  // Q(r0 + rr, l0 + ll) at As[rr][ll]
  __shared__ double Bs[kKStep][kTile + 1];  // C(r0 + rr, j0 + jj) at Bs[rr][jj]
  const GemmTile g = tiles[blockIdx.x];
  const SketchTask t = tasks[g.task];
  const int ell = *t.ell;
  if (g.r0 >= ell) return;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < t.m; k0 += kKStep) {
    for (int e = threadIdx.x; e < kTile * kKStep; e += kT) {
      const int ll = e / kKStep, rr = e % kKStep;
      const int l = g.r0 + ll, r = k0 + rr;
      As[rr][ll] = (l < ell && r < t.m) ? __ldg(t.Qc + (size_t)l * t.m + r) : 0.0;
    }
    for (int e = threadIdx.x; e < kTile * kKStep; e += kT) {
      const int rr = e / kTile, jj = e % kTile;
      const int r = k0 + rr, j = g.c0 + jj;
      Bs[rr][jj] = (r < t.m && j < t.w) ? __ldg(t.C + (size_t)r * t.ldw + j) : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < kKStep; ++rr) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[rr][ty + 16 * q];
        b[q] = Bs[rr][tx + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * b[q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int l = g.r0 + ty + 16 * p;
    if (l >= ell) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = g.c0 + tx + 16 * q;
      if (j < t.w) t.B[(size_t)l * t.w + j] = acc[p][q];
    }
  }
}

// G(i, j) = sum_r Y(r, i) Y(r, j) on tiles with r0 <= c0; an off-diagonal
// tile is stored twice (G and its transpose) so that rows of G are whole.
__global__ void __launch_bounds__(kT) k_gram(const SketchTask* __restrict__ tasks, const GemmTile* __restrict__ tiles) {
  __shared__ double As[kKStep][kTile + 1];  // Y(k0 + kk, r0 + ii) at As[kk][ii]
  __shared__ double Bs[kKStep][kTile + 1];  // Y(k0 + kk, c0 + jj) at Bs[kk][jj]
  const GemmTile g = tiles[blockIdx.x];
  const SketchTask t = tasks[g.task];
  const int ell = *t.ell;
  if (g.r0 >= ell || g.c0 >= ell) return;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < t.m; k0 += kKStep) {
    for (int e = threadIdx.x; e < kTile * kKStep; e += kT) {
      const int kk = e / kTile, ii = e % kTile;
      const int r = k0 + kk;
      const double* row = t.Y + (size_t)r * t.ldy;
      As[kk][ii] = (r < t.m && g.r0 + ii < ell) ? row[g.r0 + ii] : 0.0;
      Bs[kk][ii] = (r < t.m && g.c0 + ii < ell) ? row[g.c0 + ii] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kKStep; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty + 16 * q];
        b[q] = Bs[kk][tx + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * b[q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = g.r0 + ty + 16 * p;
    if (i >= ell) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = g.c0 + tx + 16 * q;
      if (j >= ell) continue;
      t.G[(size_t)i * t.ldy + j] = acc[p][q];
      if (g.r0 != g.c0) t.G[(size_t)j * t.ldy + i] = acc[p][q];
    }
  }
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

// Left-looking pivoted Cholesky of G = Y^T Y, one CTA per task.  d holds the
// diagonal of the Schur complement (the squared partial column norms of the
// pivoted QR of Y); step i picks the pivot as the pivoted QR does (the first
// position within pivot_rtol of the largest norm, LAPACK-style position
// swaps), stops at |L(i,i)| < stol |L(0,0)|, and computes column i of L over
// the active columns from the rows of Lt kept in global memory:
//   L(c, i) = (G(c, p) - sum_{k<i} L(c, k) L(p, k)) / L(i, i).
// Threads are (k-group, column) pairs so that short columns still keep the
// CTA's loads in flight.
template <int kPT>
__global__ void __launch_bounds__(kPT) k_pchol(const SketchTask* __restrict__ tasks, const int* __restrict__ order,
                                               double stol, double pivot_rtol) {
  extern __shared__ double psm[];
  __shared__ double s_v[kPT / 32];
  __shared__ int s_p[kPT / 32], s_c[kPT / 32];
  __shared__ int s_piv[2];
  const SketchTask t = tasks[order[blockIdx.x]];
  const int n = *t.ell, ld = t.ldy;
  if (n <= 0 || t.m <= 0 || t.w <= 0 || !t.G) return;
  const int kmin = min(t.m, n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* d = psm;
  double* lp = d + n;
  double* part = lp + n;
  int* pos = reinterpret_cast<int*>(part + kPT);
  int* at = pos + n;
  const int cw = n < kPT ? (n + 31) / 32 * 32 : kPT;  // column slots
  const int ng = kPT / cw;                            // k-groups
  const int grp = threadIdx.x / cw, slot = threadIdx.x % cw;
  for (int c = threadIdx.x; c < n; c += kPT) {
    d[c] = t.G[(size_t)c * ld + c];
    pos[c] = c;
    at[c] = c;
  }
  __syncthreads();
  double r00 = 0.0;
  int rk = kmin;
  for (int i = 0; i < kmin; ++i) {
    // the largest partial norm over the active columns
    double bv = -1.0;
    for (int c = threadIdx.x; c < n; c += kPT)
      if (pos[c] >= i) bv = fmax(bv, sqrt(fmax(d[c], 0.0)));
    bv = warp_max(bv);
    if (lane == 0) s_v[warp] = bv;
    __syncthreads();
    double M = s_v[0];
    for (int q = 1; q < kPT / 32; ++q) M = fmax(M, s_v[q]);
    // the first position within pivot_rtol of it
    const double thr = M * (1.0 - pivot_rtol);
    int bp = 0x7fffffff, bc = -1;
    for (int c = threadIdx.x; c < n; c += kPT) {
      const int p = pos[c];
      if (p >= i && p < bp && sqrt(fmax(d[c], 0.0)) >= thr) {
        bp = p;
        bc = c;
      }
    }
    warp_min_pos(bp, bc);
    if (lane == 0) {
      s_p[warp] = bp;
      s_c[warp] = bc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int P = s_p[0], Cc = s_c[0];
      for (int q = 1; q < kPT / 32; ++q)
        if (s_p[q] < P) {
          P = s_p[q];
          Cc = s_c[q];
        }
      s_piv[0] = P;
      s_piv[1] = Cc;
    }
    __syncthreads();
    int ppos = s_piv[0], pcol = s_piv[1];
    const int cur = at[i];
    if (pcol < 0) {  // no finite maximum (NaN norms): keep the column at position i
      ppos = i;
      pcol = cur;
    }
    const double nrm = sqrt(fmax(d[pcol], 0.0));  // |R(i,i)|
    if (i == 0) {
      r00 = nrm;
    } else if (!(nrm / r00 >= stol)) {
      rk = i;
      break;
    }
    __syncthreads();  // every thread has read at[i] and d[pcol]
    if (threadIdx.x == 0) {
      at[ppos] = cur;
      pos[cur] = ppos;
      at[i] = pcol;
      pos[pcol] = i;
      t.Lt[(size_t)i * ld + pcol] = nrm;
    }
    for (int k = threadIdx.x; k < i; k += kPT) lp[k] = t.Lt[(size_t)k * ld + pcol];
    __syncthreads();
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    for (int c0 = 0; c0 < n; c0 += cw) {
      const int c = c0 + slot;
      const bool act = grp < ng && c < n && pos[c] > i;
      double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (act) {
        const double* col = t.Lt + c;
        int k = grp;
        // eight rows of Lt in flight per thread
        for (; k + 7 * ng < i; k += 8 * ng) {
          double v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) v[u] = col[(size_t)(k + u * ng) * ld];
#pragma unroll
          for (int u = 0; u < 8; ++u) a[u] += v[u] * lp[k + u * ng];
        }
        for (; k < i; k += ng) a[0] += col[(size_t)k * ld] * lp[k];
      }
      const double acc = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
      if (ng > 1) {
        part[threadIdx.x] = acc;
        __syncthreads();
      }
      if (grp == 0 && c < n && pos[c] > i) {
        double sum = acc;
        for (int q = 1; q < ng; ++q) sum += part[q * cw + slot];
        const double l = (t.G[(size_t)c * ld + pcol] - sum) * inv;
        t.Lt[(size_t)i * ld + c] = l;
        d[c] -= l * l;
      }
      __syncthreads();
    }
  }
  for (int k = threadIdx.x; k < n; k += kPT) t.colat[k] = at[k];
  if (threadIdx.x == 0) *t.ell = rk;
}

// Residual scan over a block of 256 columns: res_j(k) = ||c_j||^2 -
// sum_{l<k} B(l,j)^2, and M[k] = max_j res_j(k) by atomicMax on the bit
// patterns of non-negative doubles (their order equals the values' order).
__global__ void __launch_bounds__(kT) k_residual_scan(const SketchTask* __restrict__ tasks,
                                                      const GemmTile* __restrict__ blocks) {
  const GemmTile g = blocks[blockIdx.x];
  const SketchTask t = tasks[g.task];
  const int ell = *t.ell;
  const int j = g.c0 + threadIdx.x;
  const bool ok = j < t.w;
  double res = ok ? t.cn2[j] : 0.0;
  const int lane = threadIdx.x & 31;
  for (int l = 0; l < ell; ++l) {
    if (ok) {
      const double b = t.B[(size_t)l * t.w + j];
      res -= b * b;
    }
    const double mx = warp_max(ok ? fmax(res, 0.0) : 0.0);
    if (lane == 0) atomicMax(t.M + l + 1, (unsigned long long)__double_as_longlong(mx));
  }
}

__global__ void k_rank_select(const SketchTask* __restrict__ tasks, int ntasks, double tol) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntasks) return;
  const SketchTask t = tasks[q];
  const int ell = *t.ell;
  const double thr = tol * tol * *t.cmax2;
  int rank = 0;
  for (int k = 1; k <= ell; ++k)
    if (__longlong_as_double((long long)t.M[k]) < thr) {
      rank = k;
      break;
    }
  *t.fallback = rank == 0 ? 1 : 0;
  if (rank > 0) *t.rank = rank;
}

cudaError_t done_launch(const char* name) {
  set_last_launch(name);
  add_kernel_launches(1);
  return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------- launchers
size_t rank_features_smem(int mmax) { return sizeof(double) * 4 * (size_t)std::max(mmax, 1); }

cudaError_t launch_rank_features(const SketchTask* t, int ntasks, const GemmTile* blocks, int nblocks, double tol,
                                 int mmax, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntasks <= 0) return cudaSuccess;
  const size_t smem = rank_features_smem(mmax);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_rank_features, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e) return e;
  if (nblocks > 0) {
    k_feature_blocks<<<nblocks, kT, 0, st>>>(t, blocks);
    if ((e = done_launch("launch_feature_blocks"))) return e;
  }
  k_rank_features<<<ntasks, kT, smem, st>>>(t, tol);
  return done_launch("launch_rank_features");
}

cudaError_t launch_rank_predict(const SketchTask* t, int ntasks, RankModel model, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntasks <= 0) return cudaSuccess;
  k_rank_predict<<<(ntasks + 127) / 128, 128, 0, st>>>(t, ntasks, model);
  return done_launch("launch_rank_predict");
}

cudaError_t launch_sketch(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntiles <= 0) return cudaSuccess;
  k_sketch<<<ntiles, kT, 0, st>>>(t, tiles);
  return done_launch("launch_sketch");
}

cudaError_t launch_project(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntiles <= 0) return cudaSuccess;
  k_project<<<ntiles, kT, 0, st>>>(t, tiles);
  return done_launch("launch_project");
}

cudaError_t launch_gram(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntiles <= 0) return cudaSuccess;
  k_gram<<<ntiles, kT, 0, st>>>(t, tiles);
  return done_launch("launch_gram");
}

// threads of the pivoted Cholesky: 128 for sketches of at most 64 columns
static int pchol_threads(int nmax) { return nmax <= 64 ? 128 : 1024; }

size_t pchol_smem(int nmax) {
  const size_t n = (size_t)std::max(nmax, 1);
  return sizeof(double) * (2 * n + pchol_threads(nmax)) + sizeof(int) * 2 * n;
}

cudaError_t launch_pchol(const SketchTask* t, const int* order, int ntasks, int nmax, double stol, double pivot_rtol,
                         cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntasks <= 0) return cudaSuccess;
  const size_t smem = pchol_smem(nmax);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  auto go = [&](auto kern, int threads) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return e;
    kern<<<ntasks, threads, smem, st>>>(t, order, stol, pivot_rtol);
    return cudaSuccess;
  };
  const cudaError_t e = pchol_threads(nmax) == 128 ? go(k_pchol<128>, 128) : go(k_pchol<1024>, 1024);
  if (e) return e;
  return done_launch("launch_pchol");
}

cudaError_t launch_residual_scan(const SketchTask* t, const GemmTile* blocks, int nblocks, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (nblocks <= 0) return cudaSuccess;
  k_residual_scan<<<nblocks, kT, 0, st>>>(t, blocks);
  return done_launch("launch_residual_scan");
}

cudaError_t launch_rank_select(const SketchTask* t, int ntasks, double tol, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (ntasks <= 0) return cudaSuccess;
  k_rank_select<<<(ntasks + 127) / 128, 128, 0, st>>>(t, ntasks, tol);
  return done_launch("launch_rank_select");
}

size_t mlp_work_floats(int n) { return (size_t)((n + kMlpBatch - 1) / kMlpBatch) * (kMlpParams + 1); }

cudaError_t mlp_loss_grad(const float* params, const float* X, const float* y, int n, float* loss, float* grad,
                          float* work, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (n <= 0) return cudaErrorInvalidValue;
  const int nb = (n + kMlpBatch - 1) / kMlpBatch;
  cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMlpSmem);
  if (e) return e;
  k_mlp_grad<<<nb, kMlpThreads, kMlpSmem, st>>>(params, X, y, n, work);
  if ((e = done_launch("mlp_grad"))) return e;
  k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256, 0, st>>>(work, nb, grad, loss);
  return done_launch("mlp_reduce");
}

cudaError_t mlp_predict(const float* params, const float* X, int n, float* out, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  if (n <= 0) return cudaSuccess;
  k_mlp_predict<<<(n + 127) / 128, 128, 0, st>>>(params, X, n, out);
  return done_launch("mlp_predict");
}

cudaError_t mlp_adam(float* params, const float* grad, float* m1, float* m2, float lr, int step, cudaStream_t st) {
  if (cudaError_t e = cudaGetLastError()) return e;
  const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, grad, m1, m2, lr, c1, c2);
  return done_launch("mlp_adam");
}

}  // namespace spq
