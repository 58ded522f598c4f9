// kernels.hpp -- host launchers of the grouped kernels (kernels.cu).  Every
// launcher returns the launch status (cudaGetLastError after the launch).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "tasks.hpp"

namespace spq {

// Number of kernels launched by this library (process-wide counter).
long long kernel_launches();
// Name of the launcher called last on this thread (error reports).
const char* last_launch_name();
// name reported with the next launch error (launchers outside kernels.cu)
void set_last_launch(const char* name);
// Storage of factor blocks for the launchers of this thread that follow:
// float (mixed-precision factorization and preconditioner apply) or double.
// Descriptors carry block addresses as double* either way.
void set_factor_fp32(bool on);
bool factor_fp32();
// Left block-reflector applies of float factors (trailing updates, row
// scaling, left compression) on the tensor cores (tcgen05, 3xTF32) for the
// launchers of this thread that follow.
void set_tensor_cores(bool on);
bool tensor_cores_on();
// Device status word of the factorization kernels launched by this thread:
// bit 2 (value 2) a tensor-core wait ran out, 4 a non-finite pivot, 8 a zero
// pivot in a QR factorization (elimination chains, scaling QR).
void set_status_word(int* status);
// Diagnostic of the tensor-core operand layouts (tc_apply.cuh tc::probe).
cudaError_t launch_tc_probe(const float* C, const float* V, const float* W2, int m, int flags, float* out1,
                            float* out2, int* status, cudaStream_t st);
// n doubles -> n floats stored at dst, and back (vectors, factors)
cudaError_t launch_to_f32(long long n, const double* src, double* dst, cudaStream_t st);
cudaError_t launch_to_f64(long long n, const double* src, double* dst, cudaStream_t st);
cudaError_t launch_to_f32_batch(const ConvTask* t, int ntasks, cudaStream_t st);
void add_kernel_launches(long long n);

cudaError_t launch_scatter(int nnz, const double* val, double* const* dst, cudaStream_t st);
// dst[perm[i]] = src[i], i < n
cudaError_t launch_permute(int n, const int* perm, const double* src, double* dst, cudaStream_t st);
// cs = CTAs per task (thread-block cluster size); vmax = longest reflector tail
cudaError_t launch_elim(const ElimTask* t, const ElimOut* o, int ntasks, int cs, int nmax, int vmax, cudaStream_t st);
cudaError_t launch_scale(const ScaleTask* t, int ntasks, int cs, int nmax, cudaStream_t st);
cudaError_t launch_update(const UpdTask* t, const UpdOp* o, int ntasks, cudaStream_t st);
// kind 0: left apply on column chunks, 1: right triangular solve on row chunks,
// 2: right apply on row chunks
cudaError_t launch_edge(int kind, const EdgeChunk* t, int ntasks, cudaStream_t st);
// Columns of C one CTA of a cs-CTA cluster owns in the pivoted QR: a
// contiguous range, a multiple of 32 columns when C streams from global
// memory (whole 256-byte row segments), of 2 when the CTA's block is held in
// shared memory (16-byte loads).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int rrqr_cols_per_cta(int w, int cs, bool smem_c) {
  const int a = smem_c ? 2 : 32;
  return ((w + cs - 1) / cs + a - 1) / a * a;
}
// Shared memory of one pivoted-QR CTA for tasks of at most mmax rows, kmax
// steps, nlmax own columns and rcmax own rows; c_doubles = the largest
// m x (own columns rounded to even) of a task whose block of C is held in
// shared memory (0: C streams from global memory).
size_t rrqr_smem(int mmax, int kmax, int nlmax, int rcmax, size_t c_doubles = 0);
// a cluster of cs CTAs with smem bytes each of the pivoted QR can be resident
bool rrqr_cluster_fits(int cs, size_t smem, bool smem_c = false);
// transposed gather of the compression matrices (one CTA per source block)
cudaError_t launch_rrqr_assemble(const RrqrSrc* s, int nsrc, cudaStream_t st);
cudaError_t launch_rrqr(const RrqrTask* t, int ntasks, int cs, int mmax, int kmax, int nlmax, int rcmax,
                        size_t c_doubles, double tol, double pivot_rtol, cudaStream_t st);
// Householder QR of the columns C(:, colat[0:*rank]) (pivot order given) into
// V / T / tau and the orthonormal basis Qc = C_sel R^{-1}; cs-CTA clusters,
// tasks of at most mmax rows and nmax selected columns.  Uses C, Qc, V, T,
// tau, colat, rank, m, ldw of the task.
// Shared memory of k_selected_qr; stage: with room for the QR's panels in
// shared memory (0 when that does not fit).
size_t selected_qr_smem(int mmax, int nmax, bool stage);
cudaError_t launch_selected_qr(const RrqrTask* t, int ntasks, int cs, int mmax, int nmax, cudaStream_t st);
cudaError_t launch_merge(const MergeTask* t, int ntasks, cudaStream_t st);
// Row scaling / left compression (launch_edge kind 0) of FP32 chunks whose
// blocks have at most 32 rows, one warp per chunk; edge_left_small(m) says which.
cudaError_t launch_edge_left_small(const EdgeChunk* t, int ntasks, cudaStream_t st);
bool edge_left_small(int m);
// Column scaling (launch_edge kind 1) of FP32 chunks with edge_trsm_small(nc,
// cnt) (at most 32 columns and 64 rows), one warp per chunk.
cudaError_t launch_edge_trsm_small(const EdgeChunk* t, int ntasks, cudaStream_t st);
bool edge_trsm_small(int ncols, int rows);
// Right compression (launch_edge kind 2) of FP32 chunks with
// edge_trsm_small(nc, cnt), one warp per chunk.
cudaError_t launch_edge_right_small(const EdgeChunk* t, int ntasks, cudaStream_t st);
// Trailing updates (FP32 factors) of tasks whose ops all satisfy
// update_op_small(k, m) (at most 64 reflectors and 64 rows), a 64-thread team
// per task.
cudaError_t launch_update_small(const UpdTask* t, const UpdOp* o, int ntasks, cudaStream_t st);
bool update_op_small(int k, int m);
// Forward (fwd) or backward scaling + sparsification steps of FP32 interfaces
// with spars_small(n) (at most 32 rows), one warp per interface.
cudaError_t launch_spars_small(bool fwd, const FwdSparsTask* t, int ntasks, cudaStream_t st);
bool spars_small(int n);

cudaError_t launch_fwd_elim(const FwdElimTask* t, const FwdOut* o, int ntasks, int nmax, int mmax, int* ticket,
                            int* status, long long spin_limit, cudaStream_t st);
cudaError_t launch_fwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st);
cudaError_t launch_bwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st);
cudaError_t launch_bwd_elim(const BwdElimTask* t, const BwdIn* in, int ntasks, int nmax, cudaStream_t st);
cudaError_t launch_copy_idx(int n, const int* src, const int* dst, double* x, cudaStream_t st);

cudaError_t launch_spmv(int n, const int* rowptr, const int* col, const double* val, const double* x, double* y,
                        cudaStream_t st);
int mgs_grid(int n);
cudaError_t launch_mgs_step(int n, double* q, const double* Qprev, const double* hprev, const double* Qi,
                            double* partial, unsigned int* done, double* out, int take_sqrt, cudaStream_t st);
cudaError_t launch_scale_copy(int n, const double* src, const double* s, double* dst, cudaStream_t st);
cudaError_t launch_combine(int n, int k, const double* Q, size_t ldq, const double* y, double* x, cudaStream_t st);
cudaError_t launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st);

}  // namespace spq
