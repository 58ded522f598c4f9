// engine.hpp -- the device factorization engine behind the C ABI.
//
// Tree owns one CUDA stream, a block arena in HBM and the symbolic structure.
// factorize() runs the level loop: per level the host plans task descriptors
// for the sizes it knows (level-0 sizes are static; later sizes follow from
// the ranks read back after the previous level's sparsification), uploads
// them in one copy and launches the grouped kernels.  The preconditioner apply
// is captured once into a CUDA graph after the factorization.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "structure.hpp"
#include "tasks.hpp"

namespace spq {

// Bump allocator over large cudaMalloc'd chunks.
class Arena {
 public:
  ~Arena();
  void* alloc(size_t bytes);
  double* dalloc(size_t n) { return static_cast<double*>(alloc(n * sizeof(double))); }
  // forget every allocation but keep the chunks for reuse (no cudaFree)
  void reset();
  // the allocator's state: chunk bases, fill offsets and current chunk (two
  // equal states hand out the same addresses for the same requests)
  void state(std::vector<const char*>& base, std::vector<size_t>& off, size_t& cur) const;
  // [p, p + bytes) lies inside one chunk
  bool contains(const void* p, size_t bytes) const;
  void release();
  size_t used() const { return used_; }
  size_t reserved() const { return reserved_; }

 private:
  struct Chunk {
    char* base;
    size_t size, off;
  };
  std::vector<Chunk> chunks_;
  size_t cur_ = 0;  // chunk being filled
  size_t used_ = 0, reserved_ = 0;
};

// Descriptor lists of one level kept for the next factorization of the same
// partition.  Every list is a deterministic function of the level's cluster
// sizes, the flags below and the allocators' states at the level's start
// (which fix every block, factor and scratch address the lists hold), so a
// later factorization whose key is equal reuses them instead of rebuilding;
// the merge list also depends on the level's kept ranks.  The allocations
// themselves are still made in the same order, so addresses stay identical.
struct LevelPlanKey {
  std::vector<const char*> abase, sbase;
  std::vector<size_t> aoff;
  size_t acur = 0;
  std::vector<int> sizes;
  int flags = 0;
  bool operator==(const LevelPlanKey& o) const {
    return acur == o.acur && flags == o.flags && sizes == o.sizes && aoff == o.aoff && abase == o.abase &&
           sbase == o.sbase;
  }
};
struct LevelPlan {
  bool valid = false;
  LevelPlanKey key;  // allocator chunks up to the current one, sizes, flags
  // chunk bases of both allocators once the level was planned: a later run
  // whose chunk lists start with these lands every allocation at the same place
  std::vector<const char*> abase_end, sbase_end;
  std::vector<UpdTask> ut;
  std::vector<UpdOp> uo;
  double fl_upd = 0, fl_sapp = 0;
  std::vector<EdgeChunk> rows_scale, cols_scale;
  std::vector<int> sp_w;
  std::vector<RrqrSrc> rs;
  bool compress_valid = false;
  std::vector<EdgeChunk> right, left;
  bool merge_valid = false;
  std::vector<int> merge_key;  // kept ranks of the level's sparsified interfaces
  std::vector<MergeTask> mt;
};

struct LevelTiming {
  float elim_ms = 0, scale_ms = 0, spars_ms = 0, merge_ms = 0;
  // finer split: geqrt+tsqrt chains, trailing updates, scaling QR, scaling
  // applies, RRQR, compression applies
  float e1_ms = 0, e2_ms = 0, sqr_ms = 0, sapp_ms = 0, rrqr_ms = 0, capp_ms = 0;
  // nominal flops of the same phases (chains, updates, scaling QR, scaling
  // applies, pivoted QR / learned ranks, compression applies)
  double flops[6] = {0, 0, 0, 0, 0, 0};
  int ntasks_elim = 0, ntasks_upd = 0, nspars = 0;
  // the three kinds of tuned applies: trailing updates, left applies (row
  // scaling + left compression), right compression
  float kind_ms[3] = {0, 0, 0};
  bool kind_tc[3] = {false, false, false};  // ran on the tensor cores
};

class Tree {
 public:
  Tree(int nlevels, int skip);
  ~Tree();

  // settings (ParTree setters, ptree.h:122-127 / tree.h:299-305)
  int nlevels, skip;
  double tol = 1e-1;
  int scale = 1, hsl = 0, nthreads = 1, verbose = 0, ttor_log = 0, square = 1;
  float order = 1.0f;
  // RRQR pivot: first column whose partial norm is within pivot_rtol of the
  // largest (0 = LAPACK's first maximum).  Equal norms in exact arithmetic
  // (symmetric stencils) are otherwise resolved by rounding noise.
  double pivot_rtol = 1e-6;
  // pivoted QR: elements of the compression matrix each CTA of a cluster
  // handles per pivot step (sets the cluster size, 1..16 CTAs per interface)
  double rrqr_work = 65536;
  // ... and a level's compression work is spread over about rrqr_fill CTAs per SM
  double rrqr_fill = 2;
  // factor storage and preconditioner arithmetic: 64 (plain) or 32 (mixed
  // precision: float blocks and solve, double SpMV, Krylov loop and pivoted
  // QR of the compression matrices); takes effect at the next assemble
  int precision = 64;
  // Krylov method of gmres: 0 = left-preconditioned GMRES (is.cpp:447-527),
  // 1 = flexible right-preconditioned GMRES, -1 (default) = flexible exactly
  // when the factors are float
  int krylov = -1;
  // float factors: where the block-reflector applies (trailing updates, row
  // scaling and left compression, right compression) run: 0 = CUDA cores,
  // 1 = tensor cores (3xTF32), 2 = tuned per level and kind of apply from the
  // measured times of the first two float factorizations of a partition (the
  // first on the tensor cores, the second on the CUDA cores)
  int tensor_cores = 2;
  // cycle budget of every bounded spin wait of the preconditioner apply's
  // forward sweep (takes effect at the next factorize, which captures the
  // apply); a wait that runs out fails the apply with status -12
  long long spin_limit = 2000000000LL;
  // host-side checks of the trailing-update, compression and merge
  // descriptors before each upload: every block address lies in the block
  // pool (failure: status -5, nothing launched)
  bool check_descriptors = false;
  // fault injection for the checks above (tests): the next factorize moves
  // one trailing-update descriptor's block address out of the pool before the
  // check; forces check_descriptors on
  bool corrupt_next_descriptor = false;
  // reuse a level's descriptor lists when a later factorization meets the
  // same sizes and allocator states (LevelPlan)
  bool plan_cache = true;
  long long plan_hits() const { return plan_hits_; }
  // per level: 3 kinds x (tensor-core ms, CUDA-core ms, chosen: 1 tensor, 0 CUDA,
  // -1 not tuned yet)
  void tune_table(std::vector<float>& out) const;
  // learned ranks: the sketch's pivoted QR stops at sketch_tol * tol (the
  // kept rank is then chosen on C itself)
  double sketch_tol = 0.1;
  // the sketch's pivoted QR holds each CTA's block of the sketch in shared
  // memory when it fits
  bool sketch_smem = false;
  // learned ranks: added to the predicted kept fraction before the sketch is
  // sized (an upper quantile of the predictor's error on its training pairs)
  float rank_margin = 0.0f;

  int set_coords(int dim, int n, const double* X);
  int set_coords_tensor(int n, int d);
  int partition(int nrows, int ncols, const int* colptr, const int* rowidx, const double* val);
  int assemble();
  int factorize();
  // preconditioner apply, x in permuted order (device or host pointer)
  int solve_device(double* x);
  int solve_host(double* x);
  int solve_global(const double* b, double* x);
  int spmv_device(const double* x, double* y);
  int spmv_host(const double* x, double* y);
  // Factor backward error in nprobe directions: eta[p] = ||A z - u_p|| / ||u_p||
  // with z = M^{-1} u_p, which is ||(A P - Q R) z|| / ||Q R z||.  U (n x nprobe,
  // column-major, permuted order) gives the probes; U = null draws u_p ~ N(0,1)
  // from std::mt19937_64(seed + p).
  int backward_error(int nprobe, const double* U, unsigned long long seed, double* eta);
  int gmres_host(double* b, int maxit, double tol, int* iters, double* relres, double* hist, int hist_cap);
  int gmres_device(double* b_dev, int maxit, double tol, int* iters, double* relres, double* hist, int hist_cap);
  int fgmres_device(double* b, int maxit, double gtol, int* iters, double* relres, double* hist, int hist_cap);
  // gmres_device on a caller-given device workspace of ws_doubles doubles,
  // with fixed host arrays (maxit <= kNoAllocMaxit); allocates nothing
  int gmres_device_fixed(double* b, int maxit, double gtol, int* iters, double* relres, double* ws, size_t ws_doubles);

  // preconditioner apply of nrhs vectors at once (column r at X + r * ldx):
  // one graph of nrhs concurrent sweeps, built on first use (allocates)
  int solve_block_device(double* X, int nrhs, size_t ldx);
  // flexible GMRES of nrhs right-hand sides in lockstep (block preconditioner
  // apply, one host synchronisation per iteration for all of them)
  int block_fgmres_device(double* B, int nrhs, size_t ldb, int maxit, double gtol, int* iters, double* relres);
  int block_gmres_host(double* B, int nrhs, size_t ldb, int maxit, double gtol, int* iters, double* relres);

  int set_stream(cudaStream_t s);
  cudaStream_t stream() const { return stream_; }

  // introspection
  int n() const { return st_.n; }
  const Structure& structure() const { return st_; }
  std::vector<int> cluster_sizes() const { return size_; }
  std::vector<int> cluster_sizes_org() const { return size_org_; }
  int get_block(int n1, int n2, double* out, int* rows, int* cols, int* ld) const;
  int get_factor(int order, int which, double* out, int* shape) const;
  const std::vector<LevelTiming>& level_timing() const { return lt_; }
  double t_partition = 0, t_assemble = 0, t_factorize = 0, t_solve = 0, t_gmres = 0;
  int last_gmres_iters = 0;
  std::string error;
  size_t pool_bytes() const { return arena_.used(); }
  double factor_flops() const { return flops_; }
  // bytes of the compression matrices the pivoted QR moves (the transposed
  // gather, one pass for the norms, one per pivot step over the active columns)
  double rrqr_bytes() const { return rrqr_bytes_; }

  // learned ranks: params (kMlpParams), feature mean / std (kRankFeatures
  // each); null params switch the plain pivoted QR back on
  int set_rank_model(const float* params, const float* mean, const float* stdev, int oversample);
  void set_rank_log(bool on) { rank_log_ = on; }
  void clear_rank_log() {
    log_feat_.clear();
    log_rank_.clear();
    log_kmin_.clear();
    log_level_.clear();
  }
  const std::vector<float>& log_features() const { return log_feat_; }
  const std::vector<int>& log_ranks() const { return log_rank_; }
  const std::vector<int>& log_kmin() const { return log_kmin_; }
  const std::vector<int>& log_levels() const { return log_level_; }
  void learned_counts(long long* accepted, long long* fallbacks, long long* ell) const {
    *accepted = learned_accepted_;
    *fallbacks = learned_fallbacks_;
    *ell = learned_ell_;
  }
  int device_status();
  // zero the device status word (stream-ordered): every factorize, solve and
  // GMRES entry starts from a clean status, so a wait that ran out once does
  // not fail the calls after it
  void clear_status();

 private:
  int fail(int code, const std::string& msg) {
    error = msg;
    return code;
  }
  int check_cuda(cudaError_t e, const char* where);
  // into the per-level scratch arena, staged through pinned host memory so
  // that the copy does not wait for the stream's earlier work
  void* upload(const void* host, size_t bytes);
  // pinned staging area of upload(): reused after the stream has drained
  void* stage(size_t bytes);
  void stage_reset() { pin_cur_ = 0, pin_off_ = 0; }
  int build_solve_graph();
  // one vector's apply: descriptors for workspace xw / turn counters, and its capture
  struct SolvePlan {
    FwdElimTask* fe = nullptr;
    FwdOut* fo = nullptr;
    int nfe = 0, fe_nmax = 1, fe_mmax = 1;
    FwdSparsTask* fs = nullptr;
    int nfs = 0, fs_nmax = 1;
    int nfs_small = 0;  // FP32: the first nfs_small tasks take the warp-per-interface kernels
    BwdElimTask* be = nullptr;
    BwdIn* bi = nullptr;
    int nbe = 0, be_nmax = 1;
    int* gsrc = nullptr;
    int* gdst = nullptr;
    int ng = 0;
  };
  int plan_solve(double* xw, int* turn, std::vector<SolvePlan>& ls);
  int capture_solve(const std::vector<SolvePlan>& ls, double* xw, int* turn, int* tickets, cudaGraph_t* g,
                    long long* kernels);
  int build_block_solve(int nrhs);
  void release_block_solve();
  int solve_block_cols(const std::vector<double*>& cols);
  // one zeroed region for the blocks of `edges`; sets ptr_/ld_ (rows_/cols_ must be set)
  int alloc_level_blocks(const std::vector<int>& edges);

  Structure st_;
  Csc A_;
  std::vector<double> X_;
  int dim_ = 0;
  bool partitioned_ = false, assembled_ = false, factorized_ = false;

  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  Arena arena_;        // blocks and factors (lives until destruction)
  Arena scratch_;      // descriptors of the factorization (released after it)
  std::vector<std::pair<char*, size_t>> pin_;  // pinned staging chunks
  size_t pin_cur_ = 0, pin_off_ = 0;

  // per cluster
  std::vector<int> size_, size_org_, rpos_;
  std::vector<double*> T_, Ts_, Qsp_, Tsp_;
  std::vector<int64_t> xoff_;
  int* d_rank_ = nullptr;
  // per edge
  std::vector<double*> ptr_;
  std::vector<int> ld_, rows_, cols_;
  std::vector<double*> tsqrtT_;  // per out-edge of an interior: T of the chain step

  // device copies for SpMV / GMRES
  int* d_rowptr_ = nullptr;
  int* d_col_ = nullptr;
  double* d_val_ = nullptr;
  // assembly maps built once per partition and storage precision: the block
  // element of each nonzero (CSC order), its CSR position, the CSC values
  double** d_dst_ = nullptr;
  int* d_perm_ = nullptr;
  double* d_cval_ = nullptr;
  double* h_cval_ = nullptr;  // pinned copy of the values for the upload
  std::vector<double*> asm_ptr0_;  // level-0 block addresses the maps were built for
  int asm_fp32_ = -1;
  bool asm_valid_ = false;
  double* d_xw_ = nullptr;     // solve workspace (all cluster vectors)
  int64_t xw_size_ = 0;
  int* d_turn_ = nullptr;      // per cluster turn counters
  int* d_tickets_ = nullptr;   // per level
  int* d_status_ = nullptr;
  cudaGraphExec_t solve_exec_ = nullptr;
  cudaGraph_t solve_graph_ = nullptr;
  long long solve_graph_kernels_ = 0;
  // block apply of block_nrhs_ vectors: workspaces, turn counters, tickets
  cudaGraphExec_t block_exec_ = nullptr;
  cudaGraph_t block_graph_ = nullptr;
  long long block_graph_kernels_ = 0;
  int block_nrhs_ = 0;
  double* d_xwb_ = nullptr;
  int* d_turnb_ = nullptr;
  int* d_ticketsb_ = nullptr;
  double* d_tmp_ = nullptr;    // 2 vectors for host-pointer entry points
  // Krylov workspace kept across GMRES calls
  double* d_krylov_ = nullptr;
  size_t krylov_doubles_ = 0;
  int ensure_krylov(size_t doubles);
  std::vector<LevelTiming> lt_;
  std::vector<LevelPlan> plans_;  // per level, cleared by partition
  // tuning of the float applies (tensor_cores == 2): per level and kind, the
  // measured milliseconds on the tensor cores [0] and on the CUDA cores [1]
  std::vector<std::array<float, 3>> tune_ms_[2];
  int tune_runs_ = 0;  // float factorizations of this partition measured so far
  bool use_tc(int lvl, int kind) const;
  long long plan_hits_ = 0;       // levels whose lists were reused
  double flops_ = 0;
  double rrqr_bytes_ = 0;
  bool fp32_ = false;  // factor blocks hold float (set by assemble)
  // address of element off of a factor array (element size by precision)
  double* elem(double* p, size_t off) const;
  void read_elems(const double* p, size_t off, size_t n, double* out) const;

  // learned ranks (learned.hpp): model on the device (params | mean | std),
  // logged training pairs, counters since the last set_rank_model
  float* d_model_ = nullptr;
  bool rank_model_ = false;
  int oversample_ = 10;
  bool rank_log_ = false;
  std::vector<float> log_feat_;
  std::vector<int> log_rank_, log_kmin_, log_level_;
  long long learned_accepted_ = 0, learned_fallbacks_ = 0, learned_ell_ = 0;
};

}  // namespace spq
