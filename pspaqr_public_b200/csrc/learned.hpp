// learned.hpp -- learned-rank sparsification: interface features, the rank
// MLP (inference and training kernels), the randomized range finder and the
// posterior rank selection.
//
// For each sparsifiable interface p with compression matrix C (m x w) the
// plain path runs a column-pivoted QR over all of C (ptree.cpp:373-439).  The
// learned path instead
//   1. computes features of C (sizes, column-norm statistics, the leading
//      diagonal of a QR of a 4-column Rademacher sketch) -- k_rank_features;
//   2. predicts the kept fraction rank / min(m, w) with a 3-layer MLP and
//      sets the sketch width ell = min(min(m,w), ceil(pred * min(m,w)) + p);
//   3. forms Y = C Omega (m x ell, Omega Rademacher) -- k_sketch;
//   4. runs the pivoted QR of Y, stopped at a tolerance ten times below tol,
//      giving Householder reflectors and an orthonormal basis q_0..q_{k_Y-1}
//      of the dominant part of range(Y).  The pivots come from a pivoted
//      Cholesky of the Gram matrix G = Y^T Y (k_gram, k_pchol): the pivot's
//      Schur-complement diagonal is |R(i,i)|^2 of the pivoted QR of Y, so the
//      pivot order and the stop rule are those of the pivoted QR; the
//      Householder QR of the chosen columns and Qc = Y_sel R^{-1} follow
//      (k_selected_qr).  Below a stop tolerance of kGramMinTol the Gram
//      matrix cannot resolve the stop rule and the plain pivoted-QR kernel
//      runs on Y instead;
//   5. forms B = Q^T C and, for every k <= k_Y, the largest residual column
//      norm max_j ||c_j - Q_k Q_k^T c_j|| -- k_project, k_residual_scan;
//   6. keeps the smallest k >= 1 whose largest residual is below
//      tol * max_j ||c_j|| (the stop rule of the pivoted QR: util.cpp:830-851
//      stops at the first |R(k,k)| < tol |R(0,0)|, and |R(k,k)| is the largest
//      residual column norm after k greedy steps) -- k_rank_select.  When no
//      k <= k_Y qualifies the interface falls back to the plain pivoted QR.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace spq {

constexpr int kRankFeatures = 11;
constexpr int kMlpHidden = 64;
// parameters: W1 (64 x F), b1, W2 (64 x 64), b2, w3 (64), b3
constexpr int kMlpParams = kMlpHidden * kRankFeatures + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpHidden + 1;

// One interface of the learned path.
struct SketchTask {
  const double* C;  // compression matrix, row-major m x w (ld ldw): C(r, j) = C[r * ldw + j]
  double* cn2;      // w: squared column norms
  float* feat;      // kRankFeatures
  double* cmax2;    // max_j ||c_j||^2
  int* ell;         // sketch width (written by the predictor, then the sketch's QR rank)
  double* Y;        // row-major m x ell sketch (ld ldy)
  const double* Qc; // m x ell orthonormal basis of range(Y), column-major (ld m)
  double* G;        // ell x ell Gram matrix Y^T Y, row-major (ld ldy)
  double* Lt;       // ell x ell: Lt[k * ldy + c] = L(c, k) of the pivoted Cholesky of G
  int* colat;       // ell: column of Y at each pivot position
  double* y4p;      // 4 x m partial sketches per block of kFeatCols columns (features)
  double* B;        // ell x w projections Q^T C, row-major (ld w)
  unsigned long long* M;  // ell + 1 largest squared residuals (bit patterns of doubles >= 0)
  int* rank;        // kept rank (output)
  int* fallback;    // 1 when no rank <= ell qualifies
  unsigned long long seed;
  int m, w, ldw, ldy, level;
};

// One 64 x 64 output tile of a batched GEMM over the tasks.
struct GemmTile {
  int task, r0, c0;
};

// Rank MLP: features are standardised with (mean, std) before the first
// layer; the output is sigmoid(z), the kept fraction rank / min(m, w).
struct RankModel {
  const float* params;  // kMlpParams
  const float* mean;    // kRankFeatures
  const float* stdev;   // kRankFeatures
  int oversample;
  float margin;  // added to the predicted kept fraction before sizing the sketch
};

// Features in two launches: per block of kFeatCols columns of an interface
// (tile.c0) the squared column norms and the partial 4-column sketch; then one
// CTA per interface (mmax bounds m) sums the partials in block order and forms
// the features.
constexpr int kFeatCols = 256;
size_t rank_features_smem(int mmax);
cudaError_t launch_rank_features(const SketchTask* t, int ntasks, const GemmTile* blocks, int nblocks, double tol,
                                 int mmax, cudaStream_t st);
cudaError_t launch_rank_predict(const SketchTask* t, int ntasks, RankModel model, cudaStream_t st);
// Y = C Omega over the given tiles (tile rows: kSketchRows rows of C; tile
// columns: kSketchCols columns of Y)
constexpr int kSketchRows = 64, kSketchCols = 64;
cudaError_t launch_sketch(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st);
// smallest stop tolerance (relative to |R(0,0)|) the Gram pivoting resolves:
// |R(i,i)|^2 / |R(0,0)|^2 >= 1e-10 stays four orders above the rounding of G
constexpr double kGramMinTol = 1e-5;
// G = Y^T Y over the given tiles (r0 <= c0; both triangles are written)
cudaError_t launch_gram(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st);
// Pivoted Cholesky of G (one CTA per task tasks[order[i]], nmax >= their ell;
// 128 threads when nmax <= 64, else 1024): the pivot order
// to colat and the rank -- the first i with |L(i,i)| < stol |L(0,0)|, else
// min(m, ell) -- over *ell.  Ties within pivot_rtol of the largest diagonal
// go to the smallest position, as in the pivoted QR.
size_t pchol_smem(int nmax);
cudaError_t launch_pchol(const SketchTask* t, const int* order, int ntasks, int nmax, double stol, double pivot_rtol,
                         cudaStream_t st);
// B = Q^T C over the given tiles (tile rows: kProjectRows basis vectors; tile
// columns: kProjectCols columns of C)
constexpr int kProjectRows = 64, kProjectCols = 64;
cudaError_t launch_project(const SketchTask* t, const GemmTile* tiles, int ntiles, cudaStream_t st);
// residual scan over column blocks of 256 (tile.c0), then the rank choice
cudaError_t launch_residual_scan(const SketchTask* t, const GemmTile* blocks, int nblocks, cudaStream_t st);
cudaError_t launch_rank_select(const SketchTask* t, int ntasks, double tol, cudaStream_t st);

// Training and evaluation of the rank MLP on row-major standardised features
// X (n x kRankFeatures) and targets y in [0, 1]: mean squared error of the
// sigmoid output.  All buffers are device pointers.
// loss and gradient (kMlpParams) of the n samples, deterministic
cudaError_t mlp_loss_grad(const float* params, const float* X, const float* y, int n, float* loss, float* grad,
                          float* work, cudaStream_t st);
size_t mlp_work_floats(int n);
cudaError_t mlp_predict(const float* params, const float* X, int n, float* out, cudaStream_t st);
cudaError_t mlp_adam(float* params, const float* grad, float* m1, float* m2, float lr, int step, cudaStream_t st);

}  // namespace spq
