// kernels.hpp -- host launchers of the grouped kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "tasks.hpp"

namespace spq {

void launch_scatter(int nnz, const double* val, double* const* dst, cudaStream_t st);
void launch_elim(const ElimTask* t, const ElimOut* o, int ntasks, int nmax, cudaStream_t st);
void launch_update(const UpdTask* t, const UpdOp* o, int ntasks, int kmax, cudaStream_t st);
void launch_scale(const ScaleTask* t, int ntasks, int nmax, cudaStream_t st);
void launch_scale_edge(const ScaleEdgeTask* t, int ntasks, int kmax, cudaStream_t st);
void launch_rrqr(const RrqrTask* t, const RrqrSrc* s, int ntasks, int mmax, double tol, double pivot_rtol,
                 cudaStream_t st);
void launch_spars_edge(const SparsEdgeTask* t, int ntasks, int kmax, cudaStream_t st);
void launch_merge(const MergeTask* t, int ntasks, cudaStream_t st);

void launch_fwd_elim(const FwdElimTask* t, const FwdOut* o, int ntasks, int nmax, int mmax, int* ticket, int* status,
                     long long spin_limit, cudaStream_t st);
void launch_fwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st);
void launch_bwd_spars(const FwdSparsTask* t, int ntasks, int nmax, cudaStream_t st);
void launch_bwd_elim(const BwdElimTask* t, const BwdIn* in, int ntasks, int nmax, cudaStream_t st);
void launch_copy_idx(int n, const int* src, const int* dst, double* x, cudaStream_t st);

void launch_spmv(int n, const int* rowptr, const int* col, const double* val, const double* x, double* y,
                 cudaStream_t st);
int mgs_grid(int n);
void launch_mgs_step(int n, double* q, const double* Qprev, const double* hprev, const double* Qi, double* partial,
                     unsigned int* done, double* out, int take_sqrt, cudaStream_t st);
void launch_scale_copy(int n, const double* src, const double* s, double* dst, cudaStream_t st);
void launch_combine(int n, int k, const double* Q, size_t ldq, const double* y, double* x, cudaStream_t st);
void launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st);

}  // namespace spq
