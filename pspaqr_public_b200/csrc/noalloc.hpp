// noalloc.hpp -- fixed device workspace of the allocation-free GMRES entry point.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace spq {

// Doubles in the fixed workspace (48 MiB).  A GMRES with n unknowns and maxit
// iterations needs n * (maxit + 3) + maxit + grid + 4 of them (grid <= 1024).
constexpr size_t kNoAllocDoubles = (size_t)6 << 20;
// Iterations the allocation-free GMRES accepts (its Hessenberg matrix and
// Givens rotations live in fixed host arrays of this order).
constexpr int kNoAllocMaxit = 100;

// Device address of the workspace on the current device (set up on the first
// call per device).
cudaError_t noalloc_workspace(double** ws);

}  // namespace spq
