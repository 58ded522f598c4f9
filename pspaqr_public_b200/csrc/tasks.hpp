// tasks.hpp -- descriptors of the grouped kernels.
//
// The host plans each level once the sizes of its clusters are known and
// uploads arrays of these plain structs; every pointer is a device address
// inside the block pool.  Blocks are column-major with an explicit leading
// dimension that never changes after allocation (truncation by the
// sparsification only shrinks the logical size).  Block reflector factors T
// use the blocked layout of dense.cuh (kNB x k, one triangle per 32 columns).
#pragma once
#include <cstdint>

namespace spq {

// Per interior c: geqrt of its diagonal block, then the tsqrt chain over its
// out-blocks in ascending neighbour order (ptree.cpp:170-214).  Run by one
// thread-block cluster; 32-column panels are distributed over its CTAs.
struct ElimTask {
  double* S;      // n x n diagonal block (ld = n)
  double* T;      // kNB x n block factors of the diagonal QR
  double* tau;    // n doubles of scratch (reflector broadcast)
  int n;
  int out_begin, out_end;  // range in ElimOut
};
struct ElimOut {
  double* B;  // m x n block A(n_j, c), ld = m; becomes the reflector tails
  double* T;  // kNB x n block factors of this tsqrt step
  int m;
};

// Trailing update of columns [col0, col0+ncols) of one column cluster
// (ptree.cpp:216-266): the ops of the cluster applied in order; kind 0 =
// larfb of an interior's diagonal reflectors on A(c, m), kind 1 = tpmqrt of
// one chain step on [A(c, m); A(n_j, m)].
struct UpdTask {
  int op_begin, op_end;
  int col0, ncols;
};
struct UpdOp {
  const double* V;
  const double* T;
  double* A;  // k-row top block (kind 1) or the m x ncols block (kind 0)
  double* B;  // m x ncols lower block (kind 1)
  int kind, k, m, ldv, lda, ldb;
};

// Distributed geqrt of one diagonal block (scaling QR, ptree.cpp:269-286).
struct ScaleTask {
  double* S;
  double* T;
  double* tau;
  int n;
};

// One chunk of a block apply between interfaces.  Row-scaling / left
// compression act on columns [lo, lo+cnt) of A; column-scaling / right
// compression act on rows [lo, lo+cnt).
struct EdgeChunk {
  double* A;
  const double* V;     // reflectors (or the upper-triangular R for column scaling)
  const double* T;     // block factors (kNB x k)
  const int* kdev;     // number of reflectors read on the device (rank), or null: use k
  const int* limdev;   // left compression: only columns < *limdev exist, or null
  int lda, m, nc, ldv, k, lo, cnt;
};

// Truncated column-pivoted QR of the compression matrix of one interface
// (ptree.cpp:373-439): C = [A(n,p)^T ... | A(p,m) ...], m = size of p.
// C is assembled transposed (w x m, element (j, r) at Ct[r * w + j]) and stays
// read-only while a thread-block cluster selects the pivots; the reflectors
// are then computed from the selected columns.
struct RrqrTask {
  const double* C;  // Ct: element (j, r) at C[r * ldw + j], ldw >= w a multiple of 4
  double* Q;        // m x ldq scratch: row r of the orthonormal basis at Q[r * ldq]
  double* Qc;       // the same basis column-major (m x ldq, ld m)
  double* F;        // ldq x w scratch: row i of R at F[i * w]
  double* V;        // m x m output: reflector j below the diagonal of column j, R above (ld m)
  double* T;        // kNB x m output block factors
  double* tau;      // m
  int* colat;       // w: column at each pivot position
  int* rank;        // output
  int* stats;       // 8 ints or null: recomputations, rank, kilocycles of pivot choice,
                    // projections, basis vector, row of R, final QR, whole selection
  int m, w, ldq, ldw;
};
struct RrqrSrc {
  const double* A;
  int lda, rows, cols;
  int transpose;  // 1: out-block A(n,p) (rows x m) enters transposed
  double* Ct;     // destination: columns [c0, c0 + width) of the task's C
  int w, c0;      // w: leading dimension of Ct
};

// Merge of one child block into its parent block (ptree.cpp:289-340).
struct MergeTask {
  const double* src;
  double* dst;
  int ld_src, ld_dst, rows, cols, roff, coff;
  int identity;  // 1: write I_rows (the diagonal block of a sparsified child)
  int c0;        // first column of this slab of the child block (large blocks are split)
};

// ----------------------------------------------------------------- solve
// Forward elimination sweep of one interior (ptree.cpp:2160-2187, 2840-2939).
struct FwdElimTask {
  const double* S;  // n x n (V below diagonal)
  const double* T;
  double* x;        // n
  int n;
  int out_begin, out_end;  // range in FwdOut
};
struct FwdOut {
  const double* V;  // m x n reflector tails
  const double* T;
  double* xn;       // neighbour's vector (m)
  int* turn;        // neighbour's turn counter
  int m;
  int my_turn;      // position of this interior in the neighbour's order
};
// Forward scaling + sparsification of one interface (ptree.cpp:2950-2981).
struct FwdSparsTask {
  const double* Qs;  // n x n
  const double* Ts;
  const double* V;   // n x rank
  const double* T;
  const int* rank;
  double* x;
  int n;
};
// Backward substitution of one interior (ptree.cpp:3060-3089, 3140-3174).
struct BwdElimTask {
  const double* S;
  double* x;
  int n;
  int in_begin, in_end;  // range in BwdIn
};
struct BwdIn {
  const double* R;  // n_c x s block A(c, m), ld = ldr
  const double* xm;
  int ldr, s;
};

// Conversion of one double array to float (mixed-precision factorization).
struct ConvTask {
  const double* src;
  double* dst;  // holds floats
  long long n;
  long long off;  // first element of this piece (large arrays are split)
};

}  // namespace spq
