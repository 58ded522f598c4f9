// tc_apply.cuh -- block reflector applies of the float factorization on the
// fifth-generation tensor cores (tcgen05, sm_100a).
//
// One panel of kb <= 32 reflectors (V, T) applied from the left to a chunk of
// nc <= 64 columns, Q^T C = C - V T^T V^T C, is two GEMMs around a tiny
// triangular product:
//
//   W^T (nc x kb)  = C^T V          tcgen05.mma M = 64 (columns), N = 32, K = rows
//   W2^T (nc x kb) = W^T T          32 x 32 upper-triangular T, on the CUDA cores
//   C (m x nc)    -= V W2           tcgen05.mma M = 128 (rows), N = 64, K = 32
//
// (a pentagonal tpqrt panel adds its top block A to W and subtracts W2 from
// it).  Operands are float; every product runs as three kind::tf32 MMAs on a
// hi/lo split (x = hi + lo, hi = x rounded to tf32, lo = x - hi exactly):
// A_hi B_hi + A_hi B_lo + A_lo B_hi, the 3xTF32 scheme, accumulated in FP32 in
// tensor memory.  The dropped A_lo B_lo term and the tf32 rounding of lo put
// the products at about 2^-21 relative error, the float rounding level.
//
// Operands are staged by the CUDA cores into shared memory in the canonical
// no-swizzle UMMA layouts (8 rows x 16 bytes per core matrix), with row-chunk
// strides padded by 16 bytes so that a warp storing 32 consecutive rows of one
// column hits 32 distinct banks.  One copy of a V tile serves both GEMMs: as
// the K-major B operand of the first and the MN-major A operand of the second.
// One thread issues the MMAs and commits them to an mbarrier; every wait on it
// is bounded (about 2 s of clock), after which the kernel records status 2 and
// stops using the tensor cores for the rest of its work.
#pragma once
#include <cstdint>

#include "dense.cuh"

namespace spq {
namespace tc {

using dev::kNB;
using dev::kThreads;

// ---------------------------------------------------------------- layouts (bytes)
// Every operand is K-major (no-swizzle canonical layout: core matrices of 8
// rows x 16 bytes, the 16 bytes holding 4 consecutive K elements).  V is kept
// twice: VR with K = rows (B operand of the first GEMM) and VI with K =
// reflectors (A operand of the second).  Tiles are 64 rows; both GEMMs use
// M = 64 (accumulator rows r at TMEM lanes (r % 16) + 32 (r / 16)).
constexpr int kRows = 64;                     // rows of a staged tile
constexpr int kVGroup = 128;                  // VR: 8 reflectors x 16 B
constexpr int kVChunk = 4 * kVGroup + 16;     // VR: one 4-row chunk of all 32 reflectors, padded
constexpr int kVBytes = (kRows / 4) * kVChunk;
constexpr int kIChunk = 128;                  // VI: 8 rows x 4 reflectors
constexpr int kIGroup = 8 * kIChunk;          // VI: 8 rows x all 32 reflectors
constexpr int kIBytes = (kRows / 8) * kIGroup;
constexpr int kCGroup = 128;                  // C: 8 columns x 16 B
constexpr int kCChunk = 8 * kCGroup + 16;     // C: one 4-row chunk of all 64 columns, padded
constexpr int kCBytes = (kRows / 4) * kCChunk;
constexpr int kWChunk = 128;                  // W2^T: 8 columns x 4 reflectors
constexpr int kWGroup = 8 * kWChunk;          // W2^T: 8 columns x all 32 reflectors
constexpr int kWBytes = 8 * kWGroup;          // 64 columns
constexpr int kOffVhi = 0;
constexpr int kOffVlo = kOffVhi + kVBytes;
constexpr int kOffIhi = kOffVlo + kVBytes;
constexpr int kOffIlo = kOffIhi + kIBytes;
constexpr int kOffChi = kOffIlo + kIBytes;
constexpr int kOffClo = kOffChi + kCBytes;
constexpr int kOffWhi = kOffClo + kCBytes;
constexpr int kOffWlo = kOffWhi + kWBytes;
constexpr int kOffT = kOffWlo + kWBytes;            // T (32 x 33 floats), then W (32 x 64 floats)
constexpr int kOffWs = kOffT + kNB * (kNB + 1) * 4;
constexpr int kOffBar = kOffWs + kNB * 64 * 4;      // mbarrier (8 B) + TMEM address (4 B)
constexpr int kSmemBytes = kOffBar + 256;
constexpr uint32_t kTmemCols = 128;                 // two 64-column accumulators
static_assert(kOffVlo % 16 == 0 && kOffIhi % 16 == 0 && kOffIlo % 16 == 0 && kOffChi % 16 == 0 &&
                  kOffClo % 16 == 0 && kOffWhi % 16 == 0 && kOffWlo % 16 == 0 && kOffT % 16 == 0 &&
                  kOffBar % 16 == 0,
              "UMMA operands start on 16-byte boundaries");
static_assert(2 * kSmemBytes + 2048 <= 228 * 1024, "two CTAs per SM");

// VR (K = rows): element (r, i); a warp storing 32 consecutive rows of one
// reflector hits 32 distinct banks (the 16-byte pad of kVChunk)
__host__ __device__ constexpr int v_off(int r, int i) {
  return (r >> 2) * kVChunk + (i >> 3) * kVGroup + (i & 7) * 16 + (r & 3) * 4;
}
// VI (K = reflectors): element (r, i); 16-byte stores of 4 consecutive
// reflectors by 8 consecutive rows fill one core matrix
__host__ __device__ constexpr int vi_off(int r, int i) {
  return (r >> 3) * kIGroup + (i >> 2) * kIChunk + (r & 7) * 16 + (i & 3) * 4;
}
__host__ __device__ constexpr int c_off(int r, int c) {
  return (r >> 2) * kCChunk + (c >> 3) * kCGroup + (c & 7) * 16 + (r & 3) * 4;
}
__host__ __device__ constexpr int w_off(int c, int i) {
  return (c >> 3) * kWGroup + (i >> 2) * kWChunk + (c & 7) * 16 + (i & 3) * 4;
}

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor of kind::tf32 with FP32 accumulation: M x N, A / B
// K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)),
               "r"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}
// 32 lanes x 32 consecutive 32-bit columns of tensor memory into v (lane l of
// the warp gets TMEM lane (taddr >> 16) + l).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 consecutive 32-bit columns of tensor memory from v.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  uint32_t r[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) r[i] = __float_as_uint(v[i]);
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
      "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
      "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------- context
// Per-CTA state: shared-memory buffers, the TMEM allocation, the mbarrier's
// phase and the error state.  Created by begin() (all threads), released by
// end() (all threads).
struct Ctx {
  unsigned char* sm;
  uint64_t* bar;
  uint32_t tmem;
  uint32_t phase;
  int* status;
  bool failed;
};

__device__ __forceinline__ Ctx begin(unsigned char* sm, int* status) {
  Ctx x;
  x.sm = sm;
  x.bar = reinterpret_cast<uint64_t*>(sm + kOffBar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kOffBar + 8);
  if (threadIdx.x == 0) mbar_init(x.bar);
  if (threadIdx.x < 32) tmem_alloc(slot);
  fence_before();
  __syncthreads();
  fence_after();
  x.tmem = *slot;
  x.phase = 0;
  x.status = status;
  x.failed = false;
  return x;
}

__device__ __forceinline__ void end(Ctx& x) {
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after();
    tmem_dealloc(x.tmem);
  }
}

// Wait for the MMAs committed last (all threads).  Bounded: after about 2e9
// cycles a thread gives up; the CTA agrees on the outcome with a barrier, so
// that every thread takes the same branches afterwards.  A failed CTA records
// status 2, issues no further MMAs and skips the rest of its applies (the
// factorization reports the error).
__device__ __forceinline__ void wait_mma(Ctx& x) {
  bool timed_out = false;
  if (!x.failed) {
    const long long t0 = clock64();
    while (!mbar_try(x.bar, x.phase)) {
      if (clock64() - t0 > 2000000000ll) {
        timed_out = true;
        break;
      }
    }
  }
  x.phase ^= 1u;
  if (__syncthreads_or(timed_out ? 1 : 0)) {
    if (!x.failed && threadIdx.x == 0 && x.status) atomicCAS(x.status, 0, 2);
    x.failed = true;
  }
  fence_after();
}

// ---------------------------------------------------------------- panel apply
// [A (kb x nc); C (m x nc)] <- Q^T [A; C] for one panel, as dev::tile_left_qt:
// unit = 1: V unit lower trapezoidal (m x kb) from the panel's diagonal, A
// unused; unit = 0: V full (m x kb), pentagonal top block A.  nc <= 64,
// kb <= 32.  kTrans: the operand is the transpose of the array at C, element
// (r, c) at C[c + r * ldc] -- the right apply D (I - V T V^T) of a chunk of
// nc rows of D, since (D Q)^T = Q^T D^T.  Called by all threads of the CTA.
template <bool kTrans = false>
__device__ void left_qt(Ctx& x, const float* V, int ldv, const float* Tm, int ldt, int kb, int unit, float* A,
                        int lda, float* C, int ldc, int m, int nc) {
  if (m <= 0 || nc <= 0 || kb <= 0 || x.failed) return;
  unsigned char* sm = x.sm;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  float* sT = reinterpret_cast<float*>(sm + kOffT);   // sT[l * 33 + i] = T(l, i)
  float* sW = reinterpret_cast<float*>(sm + kOffWs);  // sW[l * 64 + c] = W(l, c)
  const uint32_t base = saddr(sm);
  // T (upper triangular, zero beyond kb)
  for (int idx = t; idx < kNB * kNB; idx += kThreads) {
    const int l = idx & 31, i = idx >> 5;
    sT[l * (kNB + 1) + i] = (l <= i && i < kb) ? Tm[l + (size_t)i * ldt] : 0.f;
  }
  auto vval = [&](int gr, int i) -> float {
    if (gr >= m || i >= kb) return 0.f;
    if (unit) return gr == i ? 1.f : (gr < i ? 0.f : V[gr + (size_t)i * ldv]);
    return V[gr + (size_t)i * ldv];
  };
  // element (r, c) of the operand; a warp reads consecutive addresses (rows of
  // C, or columns of the transposed operand)
  auto cidx = [&](int idx, int& r, int& c) {
    if (kTrans) {
      c = idx & 63;
      r = idx >> 6;
    } else {
      r = idx & (kRows - 1);
      c = idx >> 6;
    }
  };
  auto cptr = [&](int r, int c) { return kTrans ? C + c + (size_t)r * ldc : C + r + (size_t)c * ldc; };
  const int nt = (m + kRows - 1) / kRows;
  constexpr int kLC = kRows * 64 / kThreads;
  float rc[kLC], rv[8];
  auto loadc = [&](int rt) {
    const int r0 = rt * kRows;
#pragma unroll
    for (int q = 0; q < kLC; ++q) {
      int r, c;
      cidx(t + q * kThreads, r, c);
      rc[q] = (r0 + r < m && c < nc) ? *cptr(r0 + r, c) : 0.f;
    }
  };
  auto storec = [&]() {
#pragma unroll
    for (int q = 0; q < kLC; ++q) {
      int r, c;
      cidx(t + q * kThreads, r, c);
      const float hi = tf32_hi(rc[q]);
      *reinterpret_cast<float*>(sm + kOffChi + c_off(r, c)) = hi;
      *reinterpret_cast<float*>(sm + kOffClo + c_off(r, c)) = rc[q] - hi;
    }
  };
  // V: thread (row t & 63, reflector groups 4 g .. 4 g + 3 for g = (t >> 6) and
  // (t >> 6) + 4); a warp reads 32 consecutive rows of one reflector
  auto loadv = [&](int rt) {
    const int gr = rt * kRows + (t & (kRows - 1));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int g = (t >> 6) + 4 * h;
#pragma unroll
      for (int j = 0; j < 4; ++j) rv[4 * h + j] = vval(gr, 4 * g + j);
    }
  };
  auto storev = [&](bool vr) {  // VI always, VR when vr
    const int r = t & (kRows - 1);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int g = (t >> 6) + 4 * h;
      float hi[4], lo[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        hi[j] = tf32_hi(rv[4 * h + j]);
        lo[j] = rv[4 * h + j] - hi[j];
      }
      *reinterpret_cast<float4*>(sm + kOffIhi + vi_off(r, 4 * g)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<float4*>(sm + kOffIlo + vi_off(r, 4 * g)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
      if (vr)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          *reinterpret_cast<float*>(sm + kOffVhi + v_off(r, 4 * g + j)) = hi[j];
          *reinterpret_cast<float*>(sm + kOffVlo + v_off(r, 4 * g + j)) = lo[j];
        }
    }
  };
  // ---- first GEMM over 64-row tiles: D1 (TMEM columns 0..31) = C^T V
  constexpr uint32_t kId = idesc_tf32(64, 32, 0, 0);
  loadc(0);
  loadv(0);
  for (int rt = 0; rt < nt; ++rt) {
    if (rt > 0) wait_mma(x);  // the previous tile's MMAs have read the buffers
    storec();
    storev(true);
    fence_smem_async();
    fence_before();
    __syncthreads();
    if (rt + 1 < nt) {  // next tile's loads overlap these MMAs
      loadc(rt + 1);
      loadv(rt + 1);
    }
    if (t == 0 && !x.failed) {
      fence_after();
      const int ksteps = ((m - rt * kRows < kRows ? m - rt * kRows : kRows) + 7) / 8;
      for (int ks = 0; ks < ksteps; ++ks) {
        const uint32_t a_hi = base + kOffChi + 2 * ks * kCChunk, a_lo = base + kOffClo + 2 * ks * kCChunk;
        const uint32_t b_hi = base + kOffVhi + 2 * ks * kVChunk, b_lo = base + kOffVlo + 2 * ks * kVChunk;
        const uint32_t acc0 = (rt > 0 || ks > 0) ? 1u : 0u;
        mma(x.tmem, sdesc(a_hi, kCChunk, kCGroup), sdesc(b_hi, kVChunk, kVGroup), kId, acc0);
        mma(x.tmem, sdesc(a_hi, kCChunk, kCGroup), sdesc(b_lo, kVChunk, kVGroup), kId, 1u);
        mma(x.tmem, sdesc(a_lo, kCChunk, kCGroup), sdesc(b_hi, kVChunk, kVGroup), kId, 1u);
      }
      commit(x.bar);
    }
  }
  wait_mma(x);
  if (x.failed) return;
  // ---- W = D1^T (+ A), parked in sW; rows c = 16 w + lane of warps 0..3
  if (warp < 4) {
    float d[32];
    tmem_ld32(x.tmem + ((uint32_t)(32 * warp) << 16), d);
    const int c = 16 * warp + lane;
    if (lane < 16) {
#pragma unroll
      for (int l = 0; l < 32; ++l) {
        float w = d[l];
        if (!unit && l < kb && c < nc) w += A[l + (size_t)c * lda];
        sW[l * 64 + c] = w;
      }
    }
  }
  fence_before();
  __syncthreads();
  // ---- W2^T = W^T T: thread (c = t & 63, reflectors 8 (t >> 6) ..), into the
  // second GEMM's B operand (hi / lo); the top block A loses W2
  {
    const int c = t & 63, i0 = (t >> 6) * 8;
    float w2[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) w2[a] = 0.f;
    for (int l = 0; l < i0 + 8; ++l) {
      const float wl = sW[l * 64 + c];
#pragma unroll
      for (int a = 0; a < 8; ++a) w2[a] += sT[l * (kNB + 1) + i0 + a] * wl;  // T(l, i) = 0 for l > i
    }
    if (!unit && c < nc)
#pragma unroll
      for (int a = 0; a < 8; ++a)
        if (i0 + a < kb) A[(i0 + a) + (size_t)c * lda] -= w2[a];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float4 hi, lo;
      hi.x = tf32_hi(w2[4 * h + 0]), lo.x = w2[4 * h + 0] - hi.x;
      hi.y = tf32_hi(w2[4 * h + 1]), lo.y = w2[4 * h + 1] - hi.y;
      hi.z = tf32_hi(w2[4 * h + 2]), lo.z = w2[4 * h + 2] - hi.z;
      hi.w = tf32_hi(w2[4 * h + 3]), lo.w = w2[4 * h + 3] - hi.w;
      *reinterpret_cast<float4*>(sm + kOffWhi + w_off(c, i0 + 4 * h)) = hi;
      *reinterpret_cast<float4*>(sm + kOffWlo + w_off(c, i0 + 4 * h)) = lo;
    }
    fence_smem_async();
  }
  // ---- second GEMM over 64-row tiles into alternating 64-column
  // accumulators: D2 = V W2 (A = VI, B = W2^T, M = 64, N = 64, K = 32); the
  // epilogue of tile rt - 1 overlaps the MMAs of tile rt
  const bool restage = nt > 1;  // a single tile's VI is still staged
  constexpr uint32_t kId2 = idesc_tf32(64, 64, 0, 0);
  auto epilogue = [&](int rt) {
    const int q4 = warp & 3, half = warp >> 2;
    float d[32];
    tmem_ld32(x.tmem + ((uint32_t)(32 * q4) << 16) + 64u * (uint32_t)(rt & 1) + 32u * (uint32_t)half, d);
    const int rl = 16 * q4 + lane, r = rt * kRows + rl;  // M = 64: row rl at lane (rl % 16) + 32 (rl / 16)
    if (lane < 16 && r < m) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int c = 32 * half + j;
        if (c < nc) {
          float* p = cptr(r, c);
          float old;
          if (!restage)  // the single C tile is still staged
            old = *reinterpret_cast<const float*>(sm + kOffChi + c_off(rl, c)) +
                  *reinterpret_cast<const float*>(sm + kOffClo + c_off(rl, c));
          else
            old = *p;
          *p = old - d[j];
        }
      }
    }
  };
  for (int rt = 0; rt < nt; ++rt) {
    if (restage) {
      loadv(rt);
      if (rt > 0) wait_mma(x);  // MMAs of tile rt - 1 are done with VI
      storev(false);
      fence_smem_async();
    }
    fence_before();
    __syncthreads();
    if (t == 0 && !x.failed) {
      fence_after();
      const uint32_t d = x.tmem + 64u * (uint32_t)(rt & 1);
      for (int ks = 0; ks < 4; ++ks) {
        const uint32_t a_hi = base + kOffIhi + 2 * ks * kIChunk, a_lo = base + kOffIlo + 2 * ks * kIChunk;
        const uint32_t b_hi = base + kOffWhi + 2 * ks * kWChunk, b_lo = base + kOffWlo + 2 * ks * kWChunk;
        mma(d, sdesc(a_hi, kIChunk, kIGroup), sdesc(b_hi, kWChunk, kWGroup), kId2, ks > 0 ? 1u : 0u);
        mma(d, sdesc(a_hi, kIChunk, kIGroup), sdesc(b_lo, kWChunk, kWGroup), kId2, 1u);
        mma(d, sdesc(a_lo, kIChunk, kIGroup), sdesc(b_hi, kWChunk, kWGroup), kId2, 1u);
      }
      commit(x.bar);
    }
    if (rt > 0 && !x.failed) epilogue(rt - 1);
    if (rt + 1 == nt) {
      wait_mma(x);
      if (x.failed) return;
      epilogue(rt);
    }
  }
  fence_before();
  __syncthreads();  // the buffers and accumulators are free for the next panel
}

// ---------------------------------------------------------------- layout probe
// Diagnostic of the operand layouts (one CTA): stages C (m <= 64 rows x 64
// columns, ld m) and V (m x 32, ld m) as left_qt does and W2 (32 x 64, ld 32),
// runs the first GEMM (D1 = C^T V, M = 64) into TMEM columns 0..31 and the
// second (D2 = V W2, M = 64) into columns 64..127, and dumps every TMEM lane:
// out1 (128 x 32) and out2 (128 x 64), row = lane.  TMEM is zeroed first, so
// lanes an MMA does not write read 0.  flags bit b swaps the leading and
// stride byte offsets of: 0 the first GEMM's A, 1 its B, 2 the second GEMM's
// A, 3 its B.  Every variant reads inside the staged buffers.
__device__ void probe(Ctx& x, const float* C, const float* V, const float* W2, int m, int flags, float* out1,
                      float* out2) {
  unsigned char* sm = x.sm;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t base = saddr(sm);
  if (warp < 4) {
    float z[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) z[i] = 0.f;
    for (int c0 = 0; c0 < 128; c0 += 32) tmem_st32(x.tmem + ((uint32_t)(32 * warp) << 16) + c0, z);
  }
  auto put = [&](int off, float v) {
    const float hi = tf32_hi(v);
    *reinterpret_cast<float*>(sm + off) = hi;
    return v - hi;
  };
  for (int idx = t; idx < 64 * 64; idx += kThreads) {
    const int r = idx & 63, c = idx >> 6;
    const float v = r < m ? C[r + (size_t)c * m] : 0.f;
    *reinterpret_cast<float*>(sm + kOffClo + c_off(r, c)) = put(kOffChi + c_off(r, c), v);
  }
  for (int idx = t; idx < 64 * 32; idx += kThreads) {
    const int r = idx & 63, i = idx >> 6;
    const float v = r < m ? V[r + (size_t)i * m] : 0.f;
    *reinterpret_cast<float*>(sm + kOffVlo + v_off(r, i)) = put(kOffVhi + v_off(r, i), v);
    *reinterpret_cast<float*>(sm + kOffIlo + vi_off(r, i)) = put(kOffIhi + vi_off(r, i), v);
  }
  for (int idx = t; idx < 32 * 64; idx += kThreads) {
    const int i = idx & 31, c = idx >> 5;
    *reinterpret_cast<float*>(sm + kOffWlo + w_off(c, i)) = put(kOffWhi + w_off(c, i), W2[i + (size_t)c * 32]);
  }
  fence_smem_async();
  fence_before();
  __syncthreads();
  auto d = [&](uint32_t a, int lbo, int sbo, bool swap) { return swap ? sdesc(a, sbo, lbo) : sdesc(a, lbo, sbo); };
  if (t == 0) {
    fence_after();
    constexpr uint32_t kId1 = idesc_tf32(64, 32, 0, 0), kId2 = idesc_tf32(64, 64, 0, 0);
    for (int ks = 0; ks < (m + 7) / 8; ++ks) {
      const uint32_t ah = base + kOffChi + 2 * ks * kCChunk, al = base + kOffClo + 2 * ks * kCChunk;
      const uint32_t bh = base + kOffVhi + 2 * ks * kVChunk, bl = base + kOffVlo + 2 * ks * kVChunk;
      mma(x.tmem, d(ah, kCChunk, kCGroup, flags & 1), d(bh, kVChunk, kVGroup, flags & 2), kId1, ks > 0);
      mma(x.tmem, d(ah, kCChunk, kCGroup, flags & 1), d(bl, kVChunk, kVGroup, flags & 2), kId1, 1u);
      mma(x.tmem, d(al, kCChunk, kCGroup, flags & 1), d(bh, kVChunk, kVGroup, flags & 2), kId1, 1u);
    }
    for (int ks = 0; ks < 4; ++ks) {
      const uint32_t ah = base + kOffIhi + 2 * ks * kIChunk, al = base + kOffIlo + 2 * ks * kIChunk;
      const uint32_t bh = base + kOffWhi + 2 * ks * kWChunk, bl = base + kOffWlo + 2 * ks * kWChunk;
      mma(x.tmem + 64, d(ah, kIChunk, kIGroup, flags & 4), d(bh, kWChunk, kWGroup, flags & 8), kId2, ks > 0);
      mma(x.tmem + 64, d(ah, kIChunk, kIGroup, flags & 4), d(bl, kWChunk, kWGroup, flags & 8), kId2, 1u);
      mma(x.tmem + 64, d(al, kIChunk, kIGroup, flags & 4), d(bh, kWChunk, kWGroup, flags & 8), kId2, 1u);
    }
    commit(x.bar);
  }
  wait_mma(x);
  if (warp < 4 && !x.failed) {
    const int row = 32 * warp + lane;
    float v[32];
    tmem_ld32(x.tmem + ((uint32_t)(32 * warp) << 16), v);
    for (int j = 0; j < 32; ++j) out1[(size_t)row * 32 + j] = v[j];
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(x.tmem + ((uint32_t)(32 * warp) << 16) + 64 + 32 * h, v);
      for (int j = 0; j < 32; ++j) out2[(size_t)row * 64 + 32 * h + j] = v[j];
    }
  }
}

}  // namespace tc
}  // namespace spq
