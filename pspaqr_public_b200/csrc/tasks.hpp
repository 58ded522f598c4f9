// tasks.hpp -- descriptors of the grouped (one CTA per task) kernels.
//
// The host plans each level once the sizes of its clusters are known and
// uploads arrays of these plain structs; every pointer is a device address
// inside the block pool.  Blocks are column-major with an explicit leading
// dimension that never changes after allocation (truncation by the
// sparsification only shrinks the logical size).
#pragma once
#include <cstdint>

namespace spq {

// Per interior c: geqrt of its diagonal block, then the tsqrt chain over its
// out-blocks in ascending neighbour order (ptree.cpp:170-214).
struct ElimTask {
  double* S;      // n x n diagonal block (ld = n)
  double* T;      // n x n block factor of the diagonal QR
  int n;
  int out_begin, out_end;  // range in ElimOut
};
struct ElimOut {
  double* B;  // m x n block A(n_j, c), ld = m; becomes the reflector tails
  double* T;  // n x n block factor of this tsqrt step
  int m;
};

// Trailing update of one column cluster (ptree.cpp:216-266): a list of ops
// applied in order; kind 0 = larfb of an interior's diagonal reflectors on
// A(c, m), kind 1 = tpmqrt of one chain step on [A(c, m); A(n_j, m)].
struct UpdTask {
  int op_begin, op_end;
  int ncols;
};
struct UpdOp {
  const double* V;
  const double* T;
  double* A;  // k-row top block (kind 1) or the m x ncols block (kind 0)
  double* B;  // m x ncols lower block (kind 1)
  int kind, k, m, ldv, lda, ldb;
};

// Scaling of a sparsified interface (ptree.cpp:269-286): QR of its diagonal
// block in place (the block keeps Qs/Rs), block factor Ts.
struct ScaleTask {
  double* S;
  double* T;
  int n;
};
// Scaling of one block between interfaces (ptree.cpp:1613-1659):
// rows by Qs^T of the row cluster, columns by Rs^{-1} of the column cluster.
struct ScaleEdgeTask {
  double* A;
  const double* Qr;  // row cluster's Qs (null: not scaled)
  const double* Tr;
  const double* Qc;  // column cluster's Qs holding Rs (null: not scaled)
  int lda, m, nc, ldqr, ldqc;
};

// Truncated column-pivoted QR of the compression matrix of one interface
// (ptree.cpp:373-439): C = [A(n,p)^T ... | A(p,m) ...], m = cols of p.
struct RrqrTask {
  double* C;      // m x w, ld m; keeps V in its first rank columns
  double* tau;    // >= m
  double* T;      // m x m region for the rank x rank block factor
  double* vn;     // 2*w scratch (partial column norms)
  int* jpvt;      // w scratch
  int* rank;      // output
  int m, w;
  int src_begin, src_end;  // range in RrqrSrc
};
struct RrqrSrc {
  const double* A;
  int lda, rows, cols;
  int transpose;  // 1: out-block A(n,p) (rows x m) enters transposed
};

// Compression of one block between interfaces (ptree.cpp:1860-1903):
// A <- Q_r^T A Q_c restricted to rank_r x rank_c.
struct SparsEdgeTask {
  double* A;
  const double* Vr;  // row cluster's sparsification reflectors (m x rank_r), null if none
  const double* Tr;
  const int* rank_r;
  const double* Vc;  // column cluster's reflectors (nc x rank_c), null if none
  const double* Tc;
  const int* rank_c;
  int lda, m, nc, ldvr, ldvc;
};

// Merge of one child block into its parent block (ptree.cpp:289-340).
struct MergeTask {
  const double* src;
  double* dst;
  int ld_src, ld_dst, rows, cols, roff, coff;
  int identity;  // 1: write I_rows (the diagonal block of a sparsified child)
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

}  // namespace spq
