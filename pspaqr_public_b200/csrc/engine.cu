// engine.cu -- host orchestration of the factorization, solve and GMRES.
#include "engine.hpp"

#include <algorithm>
#include <random>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "kernels.hpp"
#include "learned.hpp"
#include "noalloc.hpp"

namespace spq {

namespace {
double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
constexpr size_t kAlign = 256;
constexpr size_t kArenaChunk = size_t(1) << 30;
// bounded wait of the forward sweep: ~1 s at 2 GHz
constexpr int kChunk = 64;        // columns (rows) per CTA of the chunked applies
constexpr int kUpdSmallMinTasks = 4096;  // small update tasks needed for the team-per-task kernel
constexpr float kTuneMargin = 0.95f;      // tensor cores chosen where at least 5 % faster

// Row scaling / left compression chunks of the FP32 factorization: those of
// blocks small enough for the warp-per-chunk kernel first (stable, so a stored
// plan stays partitioned); returns how many.  The FP64 factorization keeps
// the tiled kernel (the warp form would spill its registers in FP64).
static int partition_small_left(std::vector<EdgeChunk>& v, bool fp32) {
  if (!fp32) return 0;
  const auto mid = std::stable_partition(v.begin(), v.end(), [](const EdgeChunk& c) { return edge_left_small(c.m); });
  return (int)(mid - v.begin());
}
constexpr int kBigCluster = 8;    // CTAs per task for blocks of >= 8 panels
constexpr int kRrqrMaxCols = 1024;  // own columns of C per CTA (four per thread)
// shared memory of a CTA holding its block of C (the sketches of the learned
// path): the block itself, the CTA's whole allotment, and the growth a
// launch group's arrays may add when sized by its largest task
constexpr size_t kRrqrSmemBlock = 120 * 1024;
constexpr size_t kRrqrSmemBudget = 176 * 1024;
constexpr size_t kRrqrSmemSlack = 48 * 1024;

// SMs of the current device (queried once per process)
int num_sms() {
  static int n = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      return 148;
    }
    return v > 0 ? v : 148;
  }();
  return n;
}
inline int dev_nb() { return 32; }  // panel width of the blocked T factors (dense.cuh kNB)
}  // namespace

// ---------------------------------------------------------------- Arena
Arena::~Arena() { release(); }

void* Arena::alloc(size_t bytes) {
  bytes = (bytes + kAlign - 1) / kAlign * kAlign;
  if (bytes == 0) bytes = kAlign;
  // first chunk from the current one on that still has room
  while (cur_ < chunks_.size() && chunks_[cur_].off + bytes > chunks_[cur_].size) ++cur_;
  if (cur_ == chunks_.size()) {
    size_t sz = std::max(kArenaChunk, bytes);
    void* p = nullptr;
    if (cudaMalloc(&p, sz) != cudaSuccess) return nullptr;
    chunks_.push_back({static_cast<char*>(p), sz, 0});
    reserved_ += sz;
  }
  Chunk& c = chunks_[cur_];
  void* r = c.base + c.off;
  c.off += bytes;
  used_ += bytes;
  return r;
}

void Arena::state(std::vector<const char*>& base, std::vector<size_t>& off, size_t& cur) const {
  base.clear();
  off.clear();
  for (const Chunk& c : chunks_) {
    base.push_back(c.base);
    off.push_back(c.off);
  }
  cur = cur_;
}

bool Arena::contains(const void* p, size_t bytes) const {
  const char* q = static_cast<const char*>(p);
  for (const Chunk& c : chunks_)
    if (q >= c.base && q + bytes <= c.base + c.size) return true;
  return false;
}

void Arena::reset() {
  for (auto& c : chunks_) c.off = 0;
  cur_ = 0;
  used_ = 0;
}

void Arena::release() {
  for (auto& c : chunks_) cudaFree(c.base);
  chunks_.clear();
  cur_ = 0;
  used_ = reserved_ = 0;
}

// ---------------------------------------------------------------- Tree
Tree::Tree(int L, int s) : nlevels(L), skip(s) {
  // SPQ_TENSOR_CORES=0 / 1 / 2 in the environment sets the starting mode of
  // spq_set_tensor_cores (CUDA cores / tensor cores / tuned per level)
  if (const char* e = std::getenv("SPQ_TENSOR_CORES")) tensor_cores = std::min(std::max(std::atoi(e), 0), 2);
}

Tree::~Tree() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& c : pin_) cudaFreeHost(c.first);
  cudaFree(d_model_);
  if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
  if (solve_graph_) cudaGraphDestroy(solve_graph_);
  release_block_solve();
  cudaFree(d_rank_);
  cudaFree(d_rowptr_);
  cudaFree(d_col_);
  cudaFree(d_val_);
  cudaFree(d_xw_);
  cudaFree(d_turn_);
  cudaFree(d_tickets_);
  cudaFree(d_status_);
  cudaFree(d_tmp_);
  cudaFree(d_dst_);
  cudaFree(d_perm_);
  cudaFree(d_cval_);
  cudaFreeHost(h_cval_);
  cudaFree(d_krylov_);
  scratch_.release();
  arena_.release();
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
}

int Tree::check_cuda(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return 0;
  error = std::string(where) + ": " + cudaGetErrorString(e) + " (last launcher: " + last_launch_name() + ")";
  return -10;
}

int Tree::set_stream(cudaStream_t s) {
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
  stream_ = s;
  own_stream_ = false;
  if (solve_exec_) {
    cudaGraphExecDestroy(solve_exec_);
    cudaGraphDestroy(solve_graph_);
    solve_exec_ = nullptr;
    solve_graph_ = nullptr;
    if (factorized_) return build_solve_graph();
  }
  return 0;
}

void Tree::clear_status() {
  if (d_status_) cudaMemsetAsync(d_status_, 0, sizeof(int), stream_);
}

int Tree::device_status() {
  int s = 0;
  if (d_status_) cudaMemcpy(&s, d_status_, sizeof(int), cudaMemcpyDeviceToHost);
  return s;
}

void* Tree::stage(size_t bytes) {
  bytes = (bytes + 255) / 256 * 256;
  while (pin_cur_ < pin_.size() && pin_off_ + bytes > pin_[pin_cur_].second) {
    ++pin_cur_;
    pin_off_ = 0;
  }
  if (pin_cur_ == pin_.size()) {
    const size_t sz = std::max<size_t>(size_t(64) << 20, bytes);
    void* p = nullptr;
    if (cudaHostAlloc(&p, sz, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    pin_.push_back({static_cast<char*>(p), sz});
  }
  char* r = pin_[pin_cur_].first + pin_off_;
  pin_off_ += bytes;
  return r;
}

void* Tree::upload(const void* host, size_t bytes) {
  void* d = scratch_.alloc(std::max<size_t>(bytes, 1));
  if (!d || !bytes || !host) return d;
  if (void* p = stage(bytes)) {
    std::memcpy(p, host, bytes);
    cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, stream_);
  } else {
    cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, stream_);
  }
  return d;
}

int Tree::set_coords(int dim, int n, const double* X) {
  if (dim <= 0 || n <= 0 || !X) return fail(-1, "bad coordinates");
  dim_ = dim;
  X_.assign(X, X + (size_t)dim * n);
  return 0;
}

// util.cpp:901-930 linspace_nd: node i0*n^(d-1) + ... + i_{d-1} at (i0, ..., i_{d-1})
int Tree::set_coords_tensor(int n, int d) {
  if (n <= 0 || d <= 0 || d > 3) return fail(-1, "tensor coordinates need n > 0 and 1 <= d <= 3");
  int64_t N = 1;
  for (int i = 0; i < d; ++i) N *= n;
  dim_ = d;
  X_.assign((size_t)N * d, 0.0);
  for (int64_t id = 0; id < N; ++id) {
    int64_t r = id;
    for (int k = d - 1; k >= 0; --k) {
      X_[(size_t)id * d + k] = (double)(r % n);
      r /= n;
    }
  }
  return 0;
}

int Tree::partition(int nrows, int ncols, const int* colptr, const int* rowidx, const double* val) {
  double t0 = wall();
  if (nrows != ncols) return fail(-2, "only square matrices are supported (rectangular path not built)");
  if (!colptr || !rowidx || !val) return fail(-1, "null matrix pointer");
  if (dim_ == 0) return fail(-3, "no coordinates: call set_coords or set_coords_tensor first");
  if ((int64_t)X_.size() != (int64_t)dim_ * ncols) return fail(-3, "coordinates do not match the matrix size");
  A_.nrows = nrows;
  A_.ncols = ncols;
  A_.colptr.assign(colptr, colptr + ncols + 1);
  const int nnz = colptr[ncols];
  A_.rowidx.assign(rowidx, rowidx + nnz);
  A_.val.assign(val, val + nnz);
  for (int j = 0; j < ncols; ++j)
    if (colptr[j + 1] < colptr[j]) return fail(-1, "colptr is not monotone");
  for (int k = 0; k < nnz; ++k)
    if (rowidx[k] < 0 || rowidx[k] >= nrows) return fail(-1, "row index out of range");
  // a NaN or infinite value would reach every kernel of the factorization
  for (int j = 0; j < ncols; ++j)
    for (int k = colptr[j]; k < colptr[j + 1]; ++k)
      if (!std::isfinite(val[k]))
        return fail(-2, "matrix value (row " + std::to_string(rowidx[k]) + ", column " + std::to_string(j) +
                            ") is not finite");
  int rc = build_structure(st_, A_, nlevels, skip, tol, X_, dim_);
  if (rc != 0) return fail(rc, st_.error);
  partitioned_ = true;
  assembled_ = factorized_ = false;
  asm_valid_ = false;
  plans_.clear();
  tune_runs_ = 0;
  t_partition = wall() - t0;
  if (verbose) printf("Time to partition: %g\n", t_partition);
  return 0;
}

int Tree::assemble() {
  if (!partitioned_) return fail(-4, "assemble called before partition");
  double t0 = wall();
  if (!stream_) {
    if (check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream")) return -10;
    own_stream_ = true;
  }
  if (check_cuda(cudaStreamSynchronize(stream_), "assemble")) return -10;
  stage_reset();
  const int n = st_.n;
  const int ncl = (int)st_.clusters.size();
  const int ned = (int)st_.edges.size();
  // factor storage is fixed here: float for the mixed-precision factorization
  fp32_ = precision == 32;
  set_factor_fp32(fp32_);
  size_.assign(ncl, 0);
  size_org_.assign(ncl, 0);
  rpos_.assign(ncl, 0);
  T_.assign(ncl, nullptr);
  Ts_.assign(ncl, nullptr);
  Qsp_.assign(ncl, nullptr);
  Tsp_.assign(ncl, nullptr);
  ptr_.assign(ned, nullptr);
  ld_.assign(ned, 0);
  rows_.assign(ned, 0);
  cols_.assign(ned, 0);
  tsqrtT_.assign(ned, nullptr);
  // a re-assembly reuses the device memory of the previous factorization
  if (check_cuda(cudaStreamSynchronize(stream_), "assemble")) return -10;
  if (solve_exec_) {
    cudaGraphExecDestroy(solve_exec_);
    cudaGraphDestroy(solve_graph_);
    solve_exec_ = nullptr;
    solve_graph_ = nullptr;
  }
  arena_.reset();
  const Level& L0 = st_.levels[0];
  for (int o = L0.first; o < L0.first + L0.count; ++o) size_[o] = size_org_[o] = st_.clusters[o].size0;
  // level-0 blocks, zeroed, then the nonzeros of App scattered in
  for (int e : L0.edges) {
    const Edge& E = st_.edges[e];
    rows_[e] = size_[E.n2];
    cols_[e] = size_[E.n1];
  }
  if (int rc = alloc_level_blocks(L0.edges)) return rc;
  const Csc& P = st_.App;
  const int nnz = (int)P.rowidx.size();
  std::vector<double*> ptr0;
  for (int e : L0.edges) ptr0.push_back(ptr_[e]);
  if (!asm_valid_ || asm_fp32_ != (fp32_ ? 1 : 0) || ptr0 != asm_ptr0_) {
    // maps of this partition and block layout: the destination of every
    // nonzero and the CSR (row-major) order of the SpMV copy
    std::vector<int> leaf_of(n);
    for (int o = L0.first; o < L0.first + L0.count; ++o)
      for (int k = st_.clusters[o].cstart; k < st_.clusters[o].cstart + st_.clusters[o].size0; ++k) leaf_of[k] = o;
    std::vector<double*> dst(nnz);
    for (int j = 0; j < n; ++j) {
      const int cj = leaf_of[j];
      for (int k = P.colptr[j]; k < P.colptr[j + 1]; ++k) {
        const int i = P.rowidx[k];
        const int ri = leaf_of[i];
        const int e = st_.find_edge(cj, ri);
        dst[k] = elem(ptr_[e], (i - st_.clusters[ri].cstart) + (size_t)(j - st_.clusters[cj].cstart) * ld_[e]);
      }
    }
    std::vector<int> rowptr(n + 1, 0), col(nnz), perm(nnz);
    for (int k = 0; k < nnz; ++k) rowptr[P.rowidx[k] + 1]++;
    std::partial_sum(rowptr.begin(), rowptr.end(), rowptr.begin());
    {
      std::vector<int> pos(rowptr.begin(), rowptr.end() - 1);
      for (int j = 0; j < n; ++j)
        for (int k = P.colptr[j]; k < P.colptr[j + 1]; ++k) {
          const int q = pos[P.rowidx[k]]++;
          col[q] = j;
          perm[k] = q;
        }
    }
    cudaFree(d_rowptr_);
    cudaFree(d_col_);
    cudaFree(d_val_);
    cudaFree(d_dst_);
    cudaFree(d_perm_);
    cudaFree(d_cval_);
    cudaFree(d_rank_);
    cudaFree(d_status_);
    cudaFree(d_tmp_);
    cudaFreeHost(h_cval_);
    d_rowptr_ = nullptr, d_col_ = nullptr, d_val_ = nullptr, d_dst_ = nullptr, d_perm_ = nullptr;
    d_cval_ = nullptr, d_rank_ = nullptr, d_status_ = nullptr, d_tmp_ = nullptr, h_cval_ = nullptr;
    const size_t nz = (size_t)std::max(nnz, 1);
    if (check_cuda(cudaMalloc(&d_rowptr_, sizeof(int) * (n + 1)), "malloc") ||
        check_cuda(cudaMalloc(&d_col_, sizeof(int) * nz), "malloc") ||
        check_cuda(cudaMalloc(&d_val_, sizeof(double) * nz), "malloc") ||
        check_cuda(cudaMalloc(&d_dst_, sizeof(double*) * nz), "malloc") ||
        check_cuda(cudaMalloc(&d_perm_, sizeof(int) * nz), "malloc") ||
        check_cuda(cudaMalloc(&d_cval_, sizeof(double) * nz), "malloc") ||
        check_cuda(cudaMalloc(&d_rank_, sizeof(int) * ncl), "malloc") ||
        check_cuda(cudaMalloc(&d_status_, sizeof(int)), "malloc") ||
        check_cuda(cudaMalloc(&d_tmp_, sizeof(double) * 2 * n), "malloc") ||
        check_cuda(cudaHostAlloc(&h_cval_, sizeof(double) * nz, cudaHostAllocDefault), "host alloc"))
      return -10;
    if (check_cuda(cudaMemcpy(d_rowptr_, rowptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice), "upload") ||
        check_cuda(cudaMemcpy(d_col_, col.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice), "upload") ||
        check_cuda(cudaMemcpy(d_dst_, dst.data(), sizeof(double*) * nnz, cudaMemcpyHostToDevice), "upload") ||
        check_cuda(cudaMemcpy(d_perm_, perm.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice), "upload"))
      return -10;
    asm_ptr0_ = ptr0;
    asm_fp32_ = fp32_ ? 1 : 0;
    asm_valid_ = true;
  }
  scratch_.reset();
  cudaMemsetAsync(d_status_, 0, sizeof(int), stream_);
  // the values of App (CSC order): one copy from pinned memory, scattered into
  // the blocks and permuted into the SpMV's CSR order on the device
  std::memcpy(h_cval_, P.val.data(), sizeof(double) * nnz);
  if (check_cuda(cudaMemcpyAsync(d_cval_, h_cval_, sizeof(double) * nnz, cudaMemcpyHostToDevice, stream_), "values") ||
      check_cuda(launch_scatter(nnz, d_cval_, d_dst_, stream_), "scatter") ||
      check_cuda(launch_permute(nnz, d_perm_, d_cval_, d_val_, stream_), "value permutation"))
    return -10;
  if (check_cuda(cudaStreamSynchronize(stream_), "assemble")) return -10;
  scratch_.reset();
  assembled_ = true;
  factorized_ = false;
  t_assemble = wall() - t0;
  if (verbose) printf("Time to assemble: %g\n", t_assemble);
  return 0;
}

// Cluster size (CTAs per task) of the distributed factorizations: one CTA
// for small blocks, a thread-block cluster of kBigCluster CTAs once a block
// has enough 32-column panels to share.
static int cluster_for(int ncols) {
  const int panels = (ncols + dev_nb() - 1) / dev_nb();
  if (panels >= 8) return kBigCluster;
  if (panels >= 4) return 4;
  return 1;
}

int Tree::factorize() {
  if (!assembled_) return fail(-4, "factorize called before assemble");
  set_factor_fp32(fp32_);
  set_tensor_cores(false);
  set_status_word(d_status_);
  if (factorized_) return fail(-4, "factorize called twice; assemble again first");
  clear_status();
  double t0 = wall();
  const int L = st_.nlevels;
  const int NB = dev_nb();
  lt_.assign(L, LevelTiming());
  flops_ = 0;
  rrqr_bytes_ = 0;
  cudaEvent_t ev[5], fe[6];
  for (auto& e : ev) cudaEventCreate(&e);
  for (auto& e : fe) cudaEventCreate(&e);
  std::vector<int> host_rank(st_.clusters.size(), 0);
  auto ck = [&](cudaError_t e, const char* where) { return check_cuda(e, where); };
  for (int lvl = 0; lvl < L; ++lvl) {
    const Level& Lv = st_.levels[lvl];
    stage_reset();  // the previous level (or assemble) ended with a stream synchronisation
    const double h0 = wall();
    double hwait = 0;  // host time blocked in the level's intermediate synchronisations
    auto sync_timed = [&](const char* where) {
      const double a = wall();
      const cudaError_t e = cudaStreamSynchronize(stream_);
      hwait += wall() - a;
      return ck(e, where);
    };
    cudaEventRecord(ev[0], stream_);
    // descriptor lists of an earlier factorization with equal sizes and
    // allocator states are reused (LevelPlan)
    if ((int)plans_.size() != L) plans_.assign(L, LevelPlan());
    LevelPlan& P = plans_[lvl];
    bool hit = false;
    {
      LevelPlanKey key;
      std::vector<const char*> abase, sbase;
      std::vector<size_t> soff;
      size_t scur = 0;
      arena_.state(abase, key.aoff, key.acur);
      scratch_.state(sbase, soff, scur);
      // the chunks up to the current one (later ones are still empty)
      const size_t na = std::min(abase.size(), key.acur + 1);
      key.abase.assign(abase.begin(), abase.begin() + na);
      key.aoff.resize(na);
      // scratch is reset every level: its chunks need only start with those the
      // recorded level ended with (checked below)
      key.sizes.assign(size_.begin() + Lv.first, size_.begin() + Lv.first + Lv.count);
      key.flags = (fp32_ ? 1 : 0) | (rank_model_ ? 2 : 0) | (rank_log_ ? 4 : 0) | (verbose >= 2 ? 8 : 0);
      auto prefix = [](const std::vector<const char*>& have, const std::vector<const char*>& rec) {
        return have.size() >= rec.size() && std::equal(rec.begin(), rec.end(), have.begin());
      };
      hit = plan_cache && P.valid && P.key == key && prefix(abase, P.abase_end) && prefix(sbase, P.sbase_end);
      if (!hit) {
        P = LevelPlan();
        P.key = std::move(key);
      } else {
        ++plan_hits_;
      }
    }
    // ---------------- elimination: geqrt + tsqrt chains, grouped by cluster size
    std::vector<ElimTask> et[3];
    std::vector<ElimOut> eo;
    int nmax[3] = {1, 1, 1}, vmax[3] = {1, 1, 1};
    const int csz[3] = {1, 4, kBigCluster};
    for (size_t ii = 0; ii < Lv.interiors.size(); ++ii) {
      const int c = Lv.interiors[ii];
      const int nc = size_[c];
      const int se = Lv.self_edge_of[c - Lv.first];
      T_[c] = arena_.dalloc((size_t)NB * std::max(nc, 1));
      ElimTask t;
      t.S = ptr_[se];
      t.T = T_[c];
      t.tau = scratch_.dalloc(std::max(nc, 1));
      t.n = nc;
      t.out_begin = (int)eo.size();
      lt_[lvl].flops[0] += 2.0 * nc * nc * (nc - nc / 3.0);
      int vm = nc;
      for (int q = Lv.out_begin[ii]; q < Lv.out_end[ii]; ++q) {
        const int e = Lv.out_edges[q];
        tsqrtT_[e] = arena_.dalloc((size_t)NB * std::max(nc, 1));
        ElimOut o;
        o.B = ptr_[e];
        o.T = tsqrtT_[e];
        o.m = rows_[e];
        eo.push_back(o);
        vm = std::max(vm, o.m);
        lt_[lvl].flops[0] += 2.0 * rows_[e] * nc * nc;
      }
      t.out_end = (int)eo.size();
      if (!t.T || !t.tau) return fail(-11, "out of device memory (elimination)");
      const int cs = cluster_for(nc);
      const int g = cs == 1 ? 0 : (cs == 4 ? 1 : 2);
      et[g].push_back(t);
      nmax[g] = std::max(nmax[g], nc);
      vmax[g] = std::max(vmax[g], vm);
    }
    // the chains run while the host builds the update lists
    {
      auto* d_eo = static_cast<ElimOut*>(upload(eo.data(), sizeof(ElimOut) * eo.size()));
      for (int g = 0; g < 3; ++g) {
        if (et[g].empty()) continue;
        auto* d_et = static_cast<ElimTask*>(upload(et[g].data(), sizeof(ElimTask) * et[g].size()));
        if (!d_et || !d_eo) return fail(-11, "out of device memory (elimination descriptors)");
        if (ck(launch_elim(d_et, d_eo, (int)et[g].size(), csz[g], nmax[g], vmax[g], stream_), "elimination kernel"))
          return -10;
      }
      cudaEventRecord(fe[0], stream_);
    }
    // trailing updates: one task per (column cluster, chunk of kChunk columns)
    std::vector<UpdTask>& ut = P.ut;
    std::vector<UpdOp>& uo = P.uo;
    for (size_t ct = 0; !hit && ct < Lv.col_m.size(); ++ct) {
      const int m = Lv.col_m[ct];
      const int op_begin = (int)uo.size();
      const int ncol = size_[m];
      for (int q = Lv.col_begin[ct]; q < Lv.col_end[ct]; ++q) {
        const int c = Lv.col_c[q];
        const int ecm = Lv.col_ecm[q];
        const int nc = size_[c];
        const int se = Lv.self_edge_of[c - Lv.first];
        UpdOp a;
        a.kind = 0;
        a.V = ptr_[se];
        a.T = T_[c];
        a.A = ptr_[ecm];
        a.B = nullptr;
        a.k = nc;
        a.m = nc;
        a.ldv = ld_[se];
        a.lda = ld_[ecm];
        a.ldb = 0;
        uo.push_back(a);
        P.fl_upd += 4.0 * nc * nc * ncol;
        const int ii = (int)(std::lower_bound(Lv.interiors.begin(), Lv.interiors.end(), c) - Lv.interiors.begin());
        int j = Lv.col_emn_begin[q];
        for (int r = Lv.out_begin[ii]; r < Lv.out_end[ii]; ++r, ++j) {
          const int ecn = Lv.out_edges[r];
          const int emn = Lv.col_emn[j];
          UpdOp b;
          b.kind = 1;
          b.V = ptr_[ecn];
          b.T = tsqrtT_[ecn];
          b.A = ptr_[ecm];
          b.B = ptr_[emn];
          b.k = nc;
          b.m = rows_[ecn];
          b.ldv = ld_[ecn];
          b.lda = ld_[ecm];
          b.ldb = ld_[emn];
          uo.push_back(b);
          P.fl_upd += 4.0 * rows_[ecn] * nc * ncol;
        }
      }
      const int op_end = (int)uo.size();
      for (int c0 = 0; c0 < ncol; c0 += kChunk) ut.push_back({op_begin, op_end, c0, std::min(kChunk, ncol - c0)});
    }
    lt_[lvl].flops[1] += P.fl_upd;
    lt_[lvl].ntasks_elim = (int)Lv.interiors.size();
    lt_[lvl].ntasks_upd = (int)ut.size();
    if (verbose >= 2) {
      double n3 = 0, mn2 = 0;
      for (int g = 0; g < 3; ++g)
        for (const ElimTask& t : et[g]) {
          n3 += (double)t.n * t.n * t.n;
          for (int o = t.out_begin; o < t.out_end; ++o) mn2 += (double)eo[o].m * t.n * t.n;
        }
      printf("level %d elim groups (cs 1/4/%d): %zu/%zu/%zu tasks, nmax %d/%d/%d, outs %zu, sum n^3 %.3g, sum m n^2 %.3g\n",
             lvl, kBigCluster, et[0].size(), et[1].size(), et[2].size(), nmax[0], nmax[1], nmax[2], eo.size(), n3, mn2);
      double fsum = 0, fmax = 0;
      int omax = 0;
      for (const UpdTask& u : ut) {
        double f = 0;
        for (int o = u.op_begin; o < u.op_end; ++o)
          f += 4.0 * uo[o].k * (uo[o].kind == 0 ? uo[o].m : uo[o].m + uo[o].k) * u.ncols;
        fsum += f;
        fmax = std::max(fmax, f);
        omax = std::max(omax, u.op_end - u.op_begin);
      }
      printf("level %d updates: %zu tasks, %zu ops, %.3g flops, mean %.3g max %.3g per task, max ops %d\n", lvl,
             ut.size(), uo.size(), fsum, fsum / std::max<size_t>(ut.size(), 1), fmax, omax);
    }
    {
      std::vector<UpdOp> uo_bad;  // the fault-injection copy (the cached list stays intact)
      const std::vector<UpdOp>* uop = &uo;
      if (corrupt_next_descriptor && !uo.empty()) {
        corrupt_next_descriptor = false;
        check_descriptors = true;
        uo_bad = uo;
        uo_bad[uo.size() / 2].B = uo_bad[uo.size() / 2].A + ((size_t)1 << 40);  // far outside the pool
        uo_bad[uo.size() / 2].kind = 1;
        uop = &uo_bad;
      }
      if (check_descriptors) {
        const size_t es = fp32_ ? 4 : 8;
        for (const UpdTask& u : ut)
          for (int o = u.op_begin; o < u.op_end; ++o) {
            const UpdOp& op = (*uop)[o];
            const size_t ncol = (size_t)u.col0 + u.ncols;
            if (!arena_.contains(op.V, es * ((size_t)op.ldv * (op.k - 1) + op.m)) ||
                !arena_.contains(op.T, es * (size_t)NB * op.k) ||
                !arena_.contains(op.A, es * ((size_t)op.lda * (ncol - 1) + (op.kind ? op.k : op.m))) ||
                (op.kind == 1 && !arena_.contains(op.B, es * ((size_t)op.ldb * (ncol - 1) + op.m))))
              return fail(-5, "trailing-update descriptor " + std::to_string(o) + " of level " + std::to_string(lvl) +
                                  " addresses memory outside the block pool; nothing launched");
          }
      }
      // FP32: tasks whose ops are all small first, for the team-per-task kernel
      // (stable, so a stored plan stays partitioned)
      int nut_small = 0;
      if (fp32_) {
        const auto mid = std::stable_partition(ut.begin(), ut.end(), [&](const UpdTask& u) {
          for (int o = u.op_begin; o < u.op_end; ++o)
            if (!update_op_small(uo[o].k, uo[o].m)) return false;
          return true;
        });
        nut_small = (int)(mid - ut.begin());
        // a team runs one op chain slower than a CTA does: the team kernel pays
        // only where there are enough small tasks to fill the GPU many times
        if (nut_small < kUpdSmallMinTasks) nut_small = 0;
      }
      auto* d_ut = static_cast<UpdTask*>(upload(ut.data(), sizeof(UpdTask) * ut.size()));
      auto* d_uo = static_cast<UpdOp*>(upload(uop->data(), sizeof(UpdOp) * uop->size()));
      if (!d_ut || !d_uo) return fail(-11, "out of device memory (update descriptors)");
      set_tensor_cores(use_tc(lvl, 0));
      lt_[lvl].kind_tc[0] = tensor_cores_on();
      if (ck(launch_update_small(d_ut, d_uo, nut_small, stream_), "update kernel (small blocks)") ||
          ck(launch_update(d_ut + nut_small, d_uo, (int)ut.size() - nut_small, stream_), "update kernel"))
        return -10;
    }
    cudaEventRecord(ev[1], stream_);
    // ---------------- scaling + sparsification
    const bool spars = !Lv.spars_clusters.empty();
    if (spars) {
      std::vector<ScaleTask> sc[3];
      int smax[3] = {1, 1, 1};
      for (int p : Lv.spars_clusters) {
        const int np = size_[p];
        Ts_[p] = arena_.dalloc((size_t)NB * std::max(np, 1));
        ScaleTask t;
        t.S = ptr_[Lv.self_edge_of[p - Lv.first]];
        t.T = Ts_[p];
        t.tau = scratch_.dalloc(std::max(np, 1));
        t.n = np;
        if (!t.T || !t.tau) return fail(-11, "out of device memory (scaling)");
        const int cs = cluster_for(np);
        const int g = cs == 1 ? 0 : (cs == 4 ? 1 : 2);
        sc[g].push_back(t);
        smax[g] = std::max(smax[g], np);
        lt_[lvl].flops[2] += 2.0 * np * np * (np - np / 3.0);
      }
      if (verbose >= 2) {
        double n3 = 0;
        for (int g = 0; g < 3; ++g)
          for (const ScaleTask& t : sc[g]) n3 += (double)t.n * t.n * t.n;
        printf("level %d scale groups: %zu/%zu/%zu tasks, nmax %d/%d/%d, sum n^3 %.3g\n", lvl, sc[0].size(),
               sc[1].size(), sc[2].size(), smax[0], smax[1], smax[2], n3);
      }
      // each stage is launched as soon as its descriptors exist, so that the
      // host builds the next lists while the GPU runs it
      auto up_vec = [&](auto& v) { return upload(v.data(), sizeof(v[0]) * v.size()); };
      for (int g = 0; g < 3; ++g) {
        if (sc[g].empty()) continue;
        auto* d = static_cast<ScaleTask*>(up_vec(sc[g]));
        if (!d || ck(launch_scale(d, (int)sc[g].size(), csz[g], smax[g], stream_), "scaling kernel")) return -10;
      }
      cudaEventRecord(fe[1], stream_);
      std::vector<EdgeChunk>& rows_scale = P.rows_scale;
      std::vector<EdgeChunk>& cols_scale = P.cols_scale;
      for (size_t ei = 0; !hit && ei < Lv.spars_edges.size(); ++ei) {
        const int e = Lv.spars_edges[ei];
        const Edge& E = st_.edges[e];
        const bool r = st_.clusters[E.n2].sparsify, c = st_.clusters[E.n1].sparsify;
        EdgeChunk t{};
        t.A = ptr_[e];
        t.lda = ld_[e];
        t.m = rows_[e];
        t.nc = cols_[e];
        if (r) {
          t.V = ptr_[Lv.self_edge_of[E.n2 - Lv.first]];
          t.T = Ts_[E.n2];
          t.ldv = size_[E.n2];
          t.k = t.m;
          for (int c0 = 0; c0 < t.nc; c0 += kChunk) {
            t.lo = c0;
            t.cnt = std::min(kChunk, t.nc - c0);
            rows_scale.push_back(t);
          }
          P.fl_sapp += 4.0 * t.m * t.m * t.nc;
        }
        if (c) {
          t.V = ptr_[Lv.self_edge_of[E.n1 - Lv.first]];
          t.T = nullptr;
          t.ldv = size_[E.n1];
          for (int r0 = 0; r0 < t.m; r0 += kChunk) {
            t.lo = r0;
            t.cnt = std::min(kChunk, t.m - r0);
            cols_scale.push_back(t);
          }
          P.fl_sapp += (double)t.m * t.nc * t.nc;
        }
      }
      lt_[lvl].flops[3] += P.fl_sapp;
      {
        const int nrows_small = partition_small_left(rows_scale, fp32_);
        const int ncols_small =
            fp32_ ? (int)(std::stable_partition(cols_scale.begin(), cols_scale.end(),
                                                [](const EdgeChunk& c) { return edge_trsm_small(c.nc, c.cnt); }) -
                          cols_scale.begin())
                  : 0;
        auto* d_rows = static_cast<EdgeChunk*>(up_vec(rows_scale));
        auto* d_cols = static_cast<EdgeChunk*>(up_vec(cols_scale));
        if (!d_rows || !d_cols) return fail(-11, "out of device memory (scaling)");
        set_tensor_cores(use_tc(lvl, 1));
        lt_[lvl].kind_tc[1] = tensor_cores_on();
        if (ck(launch_edge_left_small(d_rows, nrows_small, stream_), "row scaling (small blocks)") ||
            ck(launch_edge(0, d_rows + nrows_small, (int)rows_scale.size() - nrows_small, stream_), "row scaling"))
          return -10;
        cudaEventRecord(fe[3], stream_);
        if (ck(launch_edge_trsm_small(d_cols, ncols_small, stream_), "column scaling (small blocks)") ||
            ck(launch_edge(1, d_cols + ncols_small, (int)cols_scale.size() - ncols_small, stream_), "column scaling"))
          return -10;
      }
      cudaEventRecord(ev[2], stream_);
      // compression matrices C (m x w) of the level's interfaces, gathered
      // transposed into scratch by k_rrqr_assemble
      const size_t nsp = Lv.spars_clusters.size();
      std::vector<RrqrSrc>& rs = P.rs;
      std::vector<int>& sp_w = P.sp_w;
      if (!hit) sp_w.assign(nsp, 0);
      std::vector<int> sp_ldw(nsp);
      std::vector<double*> sp_C(nsp), spV(nsp), spT(nsp);
      std::vector<int> sp_q(st_.clusters.size(), -1);  // interface -> index in this level's list
      for (size_t q = 0; q < nsp; ++q) sp_q[Lv.spars_clusters[q]] = (int)q;
      std::vector<std::pair<double, double>> rr_dims;
      std::vector<int> rr_cs(nsp, 0);
      std::vector<char> plain_qr(nsp, 1);            // interface ran the plain pivoted QR on C
      std::vector<std::array<double, 3>> sketch_qr;  // (m, ell, steps) of each sketch's pivoted QR
      int* d_stats = verbose >= 2 ? static_cast<int*>(scratch_.alloc(sizeof(int) * 8 * nsp + 8)) : nullptr;
      double level_work = 0;
      for (size_t q = 0; q < nsp; ++q) {
        const int p = Lv.spars_clusters[q];
        const int mp = size_[p];
        if (!hit) {
          int w = 0;
          for (int k = Lv.sp_out_begin[q]; k < Lv.sp_out_end[q]; ++k) w += rows_[Lv.sp_out[k]];
          for (int k = Lv.sp_in_begin[q]; k < Lv.sp_in_end[q]; ++k) w += cols_[Lv.sp_in[k]];
          sp_w[q] = w;
        }
        const int w = sp_w[q];
        sp_ldw[q] = (w + 3) / 4 * 4;
        level_work += (double)mp * w;
        double* Ct = scratch_.dalloc((size_t)std::max(mp, 1) * std::max(sp_ldw[q], 4));
        if (!Ct) return fail(-11, "out of device memory (rrqr)");
        sp_C[q] = Ct;
        int c0 = 0;
        for (int k = Lv.sp_out_begin[q]; !hit && k < Lv.sp_out_end[q]; ++k) {
          const int e = Lv.sp_out[k];
          if (rows_[e] > 0 && mp > 0) rs.push_back({ptr_[e], ld_[e], rows_[e], cols_[e], 1, Ct, sp_ldw[q], c0});
          c0 += rows_[e];
        }
        for (int k = Lv.sp_in_begin[q]; !hit && k < Lv.sp_in_end[q]; ++k) {
          const int e = Lv.sp_in[k];
          if (cols_[e] > 0 && mp > 0) rs.push_back({ptr_[e], ld_[e], rows_[e], cols_[e], 0, Ct, sp_ldw[q], c0});
          c0 += cols_[e];
        }
        Qsp_[p] = arena_.dalloc((size_t)std::max(mp, 1) * std::max(mp, 1));
        Tsp_[p] = arena_.dalloc((size_t)NB * std::max(mp, 1));
        if (!Qsp_[p] || !Tsp_[p]) return fail(-11, "out of device memory (rrqr)");
        // the pivoted QR writes double; float factors get a converted copy
        spV[q] = fp32_ ? scratch_.dalloc((size_t)std::max(mp, 1) * std::max(mp, 1)) : Qsp_[p];
        spT[q] = fp32_ ? scratch_.dalloc((size_t)NB * std::max(mp, 1)) : Tsp_[p];
        if (!spV[q] || !spT[q]) return fail(-11, "out of device memory (rrqr)");
        rr_dims.push_back({(double)mp, (double)w});
      }
      // pivoted-QR launch groups: index 2 * log2(cluster size) + (the CTAs'
      // blocks of C held in shared memory)
      struct RrqrGroups {
        std::vector<RrqrTask> t[10];
        int m[10], k[10], nl[10], rc[10];
        size_t cd[10];  // largest block of C in shared memory (doubles)
        RrqrGroups() {
          for (int g = 0; g < 10; ++g) {
            m[g] = k[g] = nl[g] = rc[g] = 1;
            cd[g] = 0;
          }
        }
      };
      // A set of compression matrices of total work W is dealt so that about
      // rrqr_fill CTAs per SM share it: each CTA holds at most
      // max(floor, W / (rrqr_fill * SMs)) elements of C.
      auto work_cap = [&](double W, double floor_elems) {
        return std::max(floor_elems, W / (rrqr_fill * num_sms()));
      };
      // a pivoted QR of the row-major m x w matrix C (ld ldw) into V / T of
      // interface p; rank to *rank; the orthonormal basis (m x min(m,w)) to Qc
      // when given.  The cluster is the smallest whose CTAs each hold at most
      // `cap` elements of C and kRrqrMaxCols columns.  With `smem` the
      // smallest cluster whose CTAs' blocks of C fit in kRrqrSmemBlock bytes
      // of shared memory keeps them there (when one exists).  Returns the
      // cluster size, 0 on failure.
      auto add_rrqr = [&](RrqrGroups& G, const double* C, int mp, int w, int ldw, int p, int* rank, double* Qc,
                          int* stats, double cap, bool smem) -> int {
        const double work = (double)mp * w;
        const int npan = (w + NB - 1) / NB;
        int lg = 0;
        bool in_smem = false;
        if (smem) {
          for (int l2 = 0; l2 <= 4 && !in_smem; ++l2) {
            const int c = 1 << l2;
            if (c > 1 && (w + 1) / 2 < c) break;
            const int nl = rrqr_cols_per_cta(w, c, true);
            const size_t cdb = (size_t)mp * ((nl + 1) & ~1);
            const size_t b = rrqr_smem(mp, std::min(mp, w), nl, (mp + c - 1) / c, cdb);
            if (sizeof(double) * cdb <= kRrqrSmemBlock && b <= kRrqrSmemBudget &&
                (c <= 8 || rrqr_cluster_fits(c, b + kRrqrSmemSlack, true))) {
              lg = l2;
              in_smem = true;
            }
          }
        }
        if (!in_smem) {
          auto lc = [&](int c) { return rrqr_cols_per_cta(w, c, false); };
          while (lg < 4 && (work > cap * (1 << lg) || lc(1 << lg) > kRrqrMaxCols) && npan >= (2 << lg)) ++lg;
          if (lg == 4 && !rrqr_cluster_fits(16, rrqr_smem(std::max(G.m[8], mp), std::max(G.k[8], std::min(mp, w)),
                                                          std::max(G.nl[8], lc(16)), std::max(G.rc[8], (mp + 15) / 16))))
            lg = 3;
        }
        const int cs = 1 << lg;
        const int nlc = rrqr_cols_per_cta(w, cs, in_smem);
        if (nlc > kRrqrMaxCols) {
          fail(-12, "interface too wide for the pivoted QR kernel");
          return 0;
        }
        const int g = 2 * lg + (in_smem ? 1 : 0);
        RrqrTask t{};
        t.m = mp;
        t.w = w;
        t.ldw = ldw;
        t.ldq = std::max(1, std::min(mp, w));
        t.C = C;
        t.Q = scratch_.dalloc((size_t)std::max(mp, 1) * t.ldq);
        t.Qc = Qc ? Qc : scratch_.dalloc((size_t)std::max(mp, 1) * t.ldq);
        t.F = scratch_.dalloc((size_t)std::max(w, 1) * t.ldq);
        t.V = spV[sp_q[p]];
        t.T = spT[sp_q[p]];
        t.tau = scratch_.dalloc(std::max(mp, 1));
        t.colat = static_cast<int*>(scratch_.alloc(sizeof(int) * std::max(w, 1)));
        t.rank = rank;
        t.stats = stats;
        if (!t.Q || !t.Qc || !t.F || !t.tau || !t.colat) {
          fail(-11, "out of device memory (rrqr)");
          return 0;
        }
        G.t[g].push_back(t);
        G.m[g] = std::max(G.m[g], mp);
        G.k[g] = std::max(G.k[g], std::min(mp, w));
        G.nl[g] = std::max(G.nl[g], nlc);
        G.rc[g] = std::max(G.rc[g], (mp + cs - 1) / cs);
        if (in_smem) G.cd[g] = std::max(G.cd[g], (size_t)mp * ((nlc + 1) & ~1));
        return cs;
      };
      auto up_any = [&](auto& v) { return upload(v.data(), sizeof(v[0]) * v.size()); };
      auto run_rrqr = [&](RrqrGroups& G, double tol) -> int {
        for (int g = 0; g < 10; ++g) {
          if (G.t[g].empty()) continue;
          auto* d = static_cast<RrqrTask*>(up_any(G.t[g]));
          if (!d) return fail(-11, "out of device memory (rrqr tasks)");
          const int cs = 1 << (g / 2);
          if (ck(launch_rrqr(d, (int)G.t[g].size(), cs, G.m[g], G.k[g], G.nl[g], G.rc[g], G.cd[g], tol, pivot_rtol,
                             stream_),
                 "rrqr kernel")) {
            error += " [cluster " + std::to_string(cs) + ((g & 1) ? " (C in shared memory)" : "") + ", tasks " +
                     std::to_string(G.t[g].size()) + ", rows " + std::to_string(G.m[g]) + ", steps " +
                     std::to_string(G.k[g]) + ", columns/CTA " + std::to_string(G.nl[g]) + ", shared " +
                     std::to_string(rrqr_smem(G.m[g], G.k[g], G.nl[g], G.rc[g], G.cd[g])) + " B]";
            return -10;
          }
        }
        return 0;
      };
      auto* d_rs = static_cast<RrqrSrc*>(up_vec(rs));
      if (!d_rs) return fail(-11, "out of device memory (sparsification)");
      if (ck(launch_rrqr_assemble(d_rs, (int)rs.size(), stream_), "rrqr assembly")) return -10;
      // chunk lists of the compression applies: built while the GPU runs the
      // scaling and the pivoted-QR or rank-prediction stages queued before them
      std::vector<EdgeChunk>& right = P.right;
      std::vector<EdgeChunk>& left = P.left;
      EdgeChunk* d_right = nullptr;
      EdgeChunk* d_left = nullptr;
      int nleft_small = 0, nright_small = 0;
      bool compress_built = false;
      auto build_compress = [&]() -> int {
        if (compress_built) return 0;
        compress_built = true;
        const bool reuse = hit && P.compress_valid;
        if (!reuse) {
          right.clear();
          left.clear();
        }
        for (size_t ei = 0; !reuse && ei < Lv.spars_edges.size(); ++ei) {
          const int e = Lv.spars_edges[ei];
          const Edge& E = st_.edges[e];
          const bool r = st_.clusters[E.n2].sparsify, c = st_.clusters[E.n1].sparsify;
          EdgeChunk t{};
          t.A = ptr_[e];
          t.lda = ld_[e];
          t.m = rows_[e];
          t.nc = cols_[e];
          if (c) {
            t.V = Qsp_[E.n1];
            t.T = Tsp_[E.n1];
            t.kdev = d_rank_ + E.n1;
            t.ldv = size_[E.n1];
            for (int r0 = 0; r0 < t.m; r0 += kChunk) {
              t.lo = r0;
              t.cnt = std::min(kChunk, t.m - r0);
              right.push_back(t);
            }
          }
          if (r) {
            t.V = Qsp_[E.n2];
            t.T = Tsp_[E.n2];
            t.kdev = d_rank_ + E.n2;
            t.ldv = size_[E.n2];
            t.limdev = c ? d_rank_ + E.n1 : nullptr;
            for (int c0 = 0; c0 < t.nc; c0 += kChunk) {
              t.lo = c0;
              t.cnt = std::min(kChunk, t.nc - c0);
              left.push_back(t);
            }
          }
        }
        P.compress_valid = true;
        if (check_descriptors) {
          const size_t es = fp32_ ? 4 : 8;
          for (const auto* lst : {&right, &left})
            for (const EdgeChunk& c : *lst)
              if (!arena_.contains(c.A, es * ((size_t)c.lda * (c.nc - 1) + c.m)) ||
                  !arena_.contains(c.V, es * (size_t)c.ldv * c.ldv))  // Q_sp: size x size
                return fail(-5, "compression descriptor of level " + std::to_string(lvl) +
                                    " addresses memory outside the block pool; nothing launched");
        }
        nleft_small = partition_small_left(left, fp32_);
        nright_small = fp32_ ? (int)(std::stable_partition(right.begin(), right.end(),
                                                           [](const EdgeChunk& c) {
                                                             return edge_trsm_small(c.nc, c.cnt);
                                                           }) -
                                     right.begin())
                             : 0;
        d_right = static_cast<EdgeChunk*>(up_vec(right));
        d_left = static_cast<EdgeChunk*>(up_vec(left));
        if (!d_right || !d_left) return fail(-11, "out of device memory (compression)");
        return 0;
      };
      // interface features: inputs of the rank model, or logged with the
      // plain ranks as its training pairs
      std::vector<SketchTask> sk;
      float* d_feat = nullptr;
      int* d_ell = nullptr;
      int* d_fb = nullptr;
      if (rank_model_ || rank_log_) {
        sk.resize(nsp);
        int mmax = 1;
        std::vector<GemmTile> fblocks;  // column blocks of the feature pass
        d_feat = static_cast<float*>(scratch_.alloc(sizeof(float) * kRankFeatures * std::max<size_t>(nsp, 1)));
        double* d_cmax2 = scratch_.dalloc(std::max<size_t>(nsp, 1));
        d_ell = static_cast<int*>(scratch_.alloc(sizeof(int) * std::max<size_t>(nsp, 1)));
        d_fb = static_cast<int*>(scratch_.alloc(sizeof(int) * std::max<size_t>(nsp, 1)));
        if (!d_feat || !d_cmax2 || !d_ell || !d_fb) return fail(-11, "out of device memory (rank features)");
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          SketchTask& t = sk[q];
          t = SketchTask{};
          t.C = sp_C[q];
          t.m = size_[p];
          t.w = sp_w[q];
          t.ldw = sp_ldw[q];
          t.cn2 = scratch_.dalloc(std::max(t.w, 1));
          const int nblk = (t.w + kFeatCols - 1) / kFeatCols;
          t.y4p = scratch_.dalloc((size_t)std::max(nblk, 1) * 4 * std::max(t.m, 1));
          for (int b = 0; b < nblk; ++b) fblocks.push_back({(int)q, 0, b * kFeatCols});
          t.feat = d_feat + q * kRankFeatures;
          t.cmax2 = d_cmax2 + q;
          t.ell = d_ell + q;
          t.rank = d_rank_ + p;
          t.fallback = d_fb + q;
          t.seed = 0x5EEDull ^ ((unsigned long long)lvl << 40) ^ ((unsigned long long)p * 0x9E3779B97F4A7C15ull);
          t.level = lvl;
          if (!t.cn2 || !t.y4p) return fail(-11, "out of device memory (rank features)");
          mmax = std::max(mmax, t.m);
        }
        auto* d_sk = static_cast<SketchTask*>(up_any(sk));
        auto* d_fb_blocks = static_cast<GemmTile*>(up_any(fblocks));
        if (!d_sk || !d_fb_blocks) return fail(-11, "out of device memory (rank features)");
        if (ck(launch_rank_features(d_sk, (int)nsp, d_fb_blocks, (int)fblocks.size(), tol, mmax, stream_),
               "rank features"))
          return -10;
        if (rank_model_) {
          RankModel model{d_model_, d_model_ + kMlpParams, d_model_ + kMlpParams + kRankFeatures, oversample_,
                          rank_margin};
          if (ck(launch_rank_predict(d_sk, (int)nsp, model, stream_), "rank prediction")) return -10;
          if (int rc = build_compress()) return rc;
        }
      }
      if (!rank_model_) {
        RrqrGroups G;
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          rr_cs[q] = add_rrqr(G, sp_C[q], size_[p], sp_w[q], sp_ldw[q], p, d_rank_ + p, nullptr,
                              d_stats ? d_stats + 8 * q : nullptr, work_cap(level_work, rrqr_work), false);
          if (!rr_cs[q]) return -12;
        }
        if (int rc = run_rrqr(G, tol)) return rc;
        if (int rc = build_compress()) return rc;
      } else {
        // learned ranks: sketch widths back on the host to plan the sketch
        // GEMMs; pivoted QR of the sketches, projections, rank choice; the
        // plain pivoted QR for the interfaces that fall back
        cudaEvent_t le[6];
        for (auto& e : le) cudaEventCreate(&e);
        cudaEventRecord(le[0], stream_);
        std::vector<int> ell(nsp);
        if (ck(cudaMemcpyAsync(ell.data(), d_ell, sizeof(int) * nsp, cudaMemcpyDeviceToHost, stream_), "sketch widths") ||
            sync_timed("rank prediction"))
          return -10;
        std::vector<GemmTile> sk_tiles, pj_tiles, scan_blocks, gram_tiles;
        RrqrGroups G;
        // the sketch's pivots from the pivoted Cholesky of its Gram matrix
        // where the stop tolerance allows, else the pivoted-QR kernel on Y
        const double stol = sketch_tol * tol;
        const bool gram = stol >= kGramMinTol;
        std::vector<RrqrTask> sel[3];
        int sel_m[3] = {1, 1, 1}, sel_n[3] = {1, 1, 1};
        std::vector<int> pc_order[2];  // pivoted Cholesky: sketches of <= 64 columns, wider ones
        int pc_max[2] = {1, 1};
        const int sel_cs[3] = {1, 4, kBigCluster};
        size_t mtot = 0;
        double sketch_work = 0;
        for (size_t q = 0; q < nsp; ++q) {
          mtot += (size_t)ell[q] + 1;
          sketch_work += (double)sk[q].m * std::max(1, ell[q]);
        }
        auto* d_M =
            static_cast<unsigned long long*>(scratch_.alloc(sizeof(unsigned long long) * std::max<size_t>(mtot, 1)));
        if (!d_M || ck(cudaMemsetAsync(d_M, 0, sizeof(unsigned long long) * mtot, stream_), "residuals"))
          return fail(-11, "out of device memory (sketch)");
        size_t moff = 0;
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          SketchTask& t = sk[q];
          const int l = std::max(1, ell[q]);
          t.ldy = (l + 3) / 4 * 4;
          t.Y = scratch_.dalloc((size_t)std::max(t.m, 1) * t.ldy);
          double* Qc = scratch_.dalloc((size_t)std::max(t.m, 1) * l);
          t.Qc = Qc;
          t.B = scratch_.dalloc((size_t)l * std::max(t.w, 1));
          t.M = d_M + moff;
          moff += (size_t)ell[q] + 1;
          if (!t.Y || !Qc || !t.B) return fail(-11, "out of device memory (sketch)");
          if (t.m <= 0 || t.w <= 0) continue;
          for (int r0 = 0; r0 < t.m; r0 += kSketchRows)
            for (int c0 = 0; c0 < ell[q]; c0 += kSketchCols) sk_tiles.push_back({(int)q, r0, c0});
          for (int l0 = 0; l0 < ell[q]; l0 += kProjectRows)
            for (int j0 = 0; j0 < t.w; j0 += kProjectCols) pj_tiles.push_back({(int)q, l0, j0});
          for (int j0 = 0; j0 < t.w; j0 += 256) scan_blocks.push_back({(int)q, 0, j0});
          // the sketch's pivoted QR stops at sketch_tol * tol and writes its
          // rank over the sketch width: later stages use only those vectors
          if (gram) {
            t.G = scratch_.dalloc((size_t)l * t.ldy);
            t.Lt = scratch_.dalloc((size_t)l * t.ldy);
            t.colat = static_cast<int*>(scratch_.alloc(sizeof(int) * l));
            RrqrTask r{};
            r.C = t.Y;
            r.ldw = t.ldy;
            r.m = t.m;
            r.w = ell[q];
            r.Qc = Qc;
            r.V = spV[q];
            r.T = spT[q];
            r.tau = scratch_.dalloc(std::max(t.m, 1));
            r.colat = t.colat;
            r.rank = d_ell + q;
            if (!t.G || !t.Lt || !t.colat || !r.tau) return fail(-11, "out of device memory (sketch)");
            for (int r0 = 0; r0 < ell[q]; r0 += 64)
              for (int c0 = r0; c0 < ell[q]; c0 += 64) gram_tiles.push_back({(int)q, r0, c0});
            const int cs = cluster_for(ell[q]);
            const int g = cs == 1 ? 0 : (cs == 4 ? 1 : 2);
            sel[g].push_back(r);
            sel_m[g] = std::max(sel_m[g], t.m);
            sel_n[g] = std::max(sel_n[g], ell[q]);
            const int pg = ell[q] <= 64 ? 0 : 1;
            pc_order[pg].push_back((int)q);
            pc_max[pg] = std::max(pc_max[pg], ell[q]);
          } else if (!add_rrqr(G, t.Y, t.m, ell[q], t.ldy, p, d_ell + q, Qc, d_stats ? d_stats + 8 * q : nullptr,
                               work_cap(sketch_work, 4096), sketch_smem)) {
            return -12;
          }
        }
        auto* d_sk = static_cast<SketchTask*>(up_any(sk));
        auto* d_skt = static_cast<GemmTile*>(up_any(sk_tiles));
        auto* d_pjt = static_cast<GemmTile*>(up_any(pj_tiles));
        auto* d_scb = static_cast<GemmTile*>(up_any(scan_blocks));
        if (!d_sk || !d_skt || !d_pjt || !d_scb) return fail(-11, "out of device memory (sketch)");
        cudaEventRecord(le[1], stream_);
        if (ck(launch_sketch(d_sk, d_skt, (int)sk_tiles.size(), stream_), "sketch")) return -10;
        cudaEventRecord(le[2], stream_);
        if (gram) {
          auto* d_gt = static_cast<GemmTile*>(up_any(gram_tiles));
          if (!d_gt) return fail(-11, "out of device memory (sketch)");
          if (ck(launch_gram(d_sk, d_gt, (int)gram_tiles.size(), stream_), "sketch Gram matrix")) return -10;
          for (int pg = 0; pg < 2; ++pg) {
            if (pc_order[pg].empty()) continue;
            auto* d_ord = static_cast<int*>(up_any(pc_order[pg]));
            if (!d_ord) return fail(-11, "out of device memory (sketch)");
            if (ck(launch_pchol(d_sk, d_ord, (int)pc_order[pg].size(), pc_max[pg], stol, pivot_rtol, stream_),
                   "sketch pivots"))
              return -10;
          }
          for (int g = 0; g < 3; ++g) {
            if (sel[g].empty()) continue;
            auto* d_sel = static_cast<RrqrTask*>(up_any(sel[g]));
            if (!d_sel) return fail(-11, "out of device memory (sketch)");
            if (ck(launch_selected_qr(d_sel, (int)sel[g].size(), sel_cs[g], sel_m[g], sel_n[g], stream_),
                   "sketch QR"))
              return -10;
          }
        } else if (int rc = run_rrqr(G, stol)) {
          return rc;
        }
        cudaEventRecord(le[3], stream_);
        if (ck(launch_project(d_sk, d_pjt, (int)pj_tiles.size(), stream_), "projection") ||
            ck(launch_residual_scan(d_sk, d_scb, (int)scan_blocks.size(), stream_), "residual scan") ||
            ck(launch_rank_select(d_sk, (int)nsp, tol, stream_), "rank selection"))
          return -10;
        cudaEventRecord(le[4], stream_);
        std::vector<int> fb(nsp);
        if (ck(cudaMemcpyAsync(fb.data(), d_fb, sizeof(int) * nsp, cudaMemcpyDeviceToHost, stream_), "fallback flags") ||
            sync_timed("rank selection"))
          return -10;
        RrqrGroups Fb;
        double fb_work = 0;
        for (size_t q = 0; q < nsp; ++q)
          if (fb[q]) fb_work += (double)sk[q].m * sk[q].w;
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          const SketchTask& t = sk[q];
          lt_[lvl].flops[4] += 4.0 * t.m * (double)t.w * ell[q];  // sketch + projection GEMMs
          learned_ell_ += ell[q];
          if (t.m <= 0 || t.w <= 0) continue;
          sketch_qr.push_back({(double)t.m, (double)ell[q], (double)ell[q]});
          plain_qr[q] = fb[q] ? 1 : 0;
          if (fb[q]) {
            ++learned_fallbacks_;
            rr_cs[q] = add_rrqr(Fb, sp_C[q], t.m, t.w, t.ldw, p, d_rank_ + p, nullptr, nullptr,
                                work_cap(fb_work, 16384), false);
            if (!rr_cs[q]) return -12;
          } else {
            ++learned_accepted_;
          }
        }
        if (int rc = run_rrqr(Fb, tol)) return rc;
        cudaEventRecord(le[5], stream_);
        if (verbose >= 2) {
          cudaEventSynchronize(le[5]);
          float ms[5];
          for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&ms[k], le[k], le[k + 1]);
          int nfb = 0;
          for (int f : fb) nfb += f;
          printf("learned level %d: plan %.2f sketch %.2f qr %.2f project %.2f fallback(%d) %.2f ms\n", lvl, ms[0], ms[1],
                 ms[2], ms[3], nfb, ms[4]);
          if (d_stats && !gram) {
            std::vector<int> st(8 * nsp);
            cudaMemcpy(st.data(), d_stats, sizeof(int) * st.size(), cudaMemcpyDeviceToHost);
            double steps = 0, recomp = 0, kc[6] = {0, 0, 0, 0, 0, 0}, ellsum = 0;
            for (size_t q = 0; q < nsp; ++q) {
              recomp += st[8 * q];
              steps += st[8 * q + 1];
              for (int k = 0; k < 5; ++k) kc[k] += st[8 * q + 2 + k];
              ellsum += ell[q];
            }
            printf("  sketch QR: tasks %zu mean ell %.0f mean steps %.0f recomputes/task %.0f  kcycles/task pivot %.0f "
                   "proj %.0f basis %.0f rowR %.0f finalQR %.0f\n",
                   nsp, ellsum / nsp, steps / nsp, recomp / nsp, kc[0] / nsp, kc[1] / nsp, kc[2] / nsp, kc[3] / nsp,
                   kc[4] / nsp);
          }
        }
        for (auto& e : le) cudaEventDestroy(e);
      }
      if (fp32_ && nsp) {
        // one CTA per piece of at most kConvPiece elements
        constexpr long long kConvPiece = 65536;
        std::vector<ConvTask> cv;
        auto conv = [&](const double* src, double* dst, long long n) {
          for (long long off = 0; off < n; off += kConvPiece) cv.push_back({src, dst, std::min(kConvPiece, n - off), off});
        };
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          const long long mp = std::max(size_[p], 1);
          conv(spV[q], Qsp_[p], mp * mp);
          conv(spT[q], Tsp_[p], (long long)NB * mp);
        }
        auto* d_cv = static_cast<ConvTask*>(up_any(cv));
        if (!d_cv || ck(launch_to_f32_batch(d_cv, (int)cv.size(), stream_), "factor conversion")) return -10;
      }
      if (int rc = build_compress()) return rc;
      cudaEventRecord(fe[2], stream_);
      set_tensor_cores(use_tc(lvl, 2));
      lt_[lvl].kind_tc[2] = tensor_cores_on();
      if (ck(launch_edge_right_small(d_right, nright_small, stream_), "right compression (small blocks)") ||
          ck(launch_edge(2, d_right + nright_small, (int)right.size() - nright_small, stream_), "right compression"))
        return -10;
      cudaEventRecord(fe[4], stream_);
      set_tensor_cores(use_tc(lvl, 1));
      if (ck(launch_edge_left_small(d_left, nleft_small, stream_), "left compression (small blocks)") ||
          ck(launch_edge(0, d_left + nleft_small, (int)left.size() - nleft_small, stream_), "left compression"))
        return -10;
      cudaEventRecord(ev[3], stream_);
      if (ck(cudaMemcpyAsync(host_rank.data(), d_rank_, sizeof(int) * host_rank.size(), cudaMemcpyDeviceToHost, stream_),
             "rank readback") ||
          sync_timed("sparsification"))
        return -10;
      // compression applies: Q^T of the interface's r reflectors on the rows
      // of its edges, Q on their columns (4 m r - 2 r^2 per vector)
      for (int e : Lv.spars_edges) {
        const Edge& E = st_.edges[e];
        if (st_.clusters[E.n1].sparsify) {
          const double n = size_[E.n1], r = host_rank[E.n1];
          lt_[lvl].flops[5] += (4.0 * n * r - 2.0 * r * r) * rows_[e];
        }
        if (st_.clusters[E.n2].sparsify) {
          const double m = size_[E.n2], r = host_rank[E.n2];
          lt_[lvl].flops[5] += (4.0 * m * r - 2.0 * r * r) * cols_[e];
        }
      }
      for (int p : Lv.spars_clusters) size_[p] = host_rank[p];
      if (rank_log_ && nsp) {
        std::vector<float> f(kRankFeatures * nsp);
        if (ck(cudaMemcpy(f.data(), d_feat, sizeof(float) * f.size(), cudaMemcpyDeviceToHost), "rank features"))
          return -10;
        log_feat_.insert(log_feat_.end(), f.begin(), f.end());
        for (size_t q = 0; q < nsp; ++q) {
          const int p = Lv.spars_clusters[q];
          log_rank_.push_back(host_rank[p]);
          log_kmin_.push_back(std::min((int)rr_dims[q].first, (int)rr_dims[q].second));
          log_level_.push_back(lvl);
        }
      }
      std::vector<int> stats;
      if (d_stats) {
        stats.resize(8 * Lv.spars_clusters.size());
        if (ck(cudaMemcpy(stats.data(), d_stats, sizeof(int) * stats.size(), cudaMemcpyDeviceToHost), "rrqr stats"))
          return -10;
      }
      // nominal flops (LAPACK Working Note 41 geqp3 count) and the bytes of C
      // the pivoted QR moves: the transposed gather (read + write), one pass
      // for the norms, one per pivot step over the active columns
      auto account = [&](double m, double w, double steps, double r) {
        lt_[lvl].flops[4] += 4.0 * m * w * r - 2.0 * r * r * (m + w) + 4.0 * r * r * r / 3.0 + m * r * r;
        rrqr_bytes_ += 8.0 * m * (3.0 * w + steps * w - steps * (steps + 1.0) / 2.0);
      };
      for (const auto& e : sketch_qr) account(e[0], e[1], e[2], e[2]);
      for (size_t q = 0; q < Lv.spars_clusters.size(); ++q) {
        const double m = rr_dims[q].first, w = rr_dims[q].second, r = size_[Lv.spars_clusters[q]];
        if (plain_qr[q]) account(m, w, std::min(r + 1.0, std::min(m, w)), r);
        if (verbose >= 2)
          printf("rrqr level %d m %d w %d rank %d cluster %d recomputed %d kcycles %d %d %d %d %d %d\n", lvl, (int)m,
                 (int)w, (int)r, rr_cs[q], stats[8 * q], stats[8 * q + 2], stats[8 * q + 3], stats[8 * q + 4],
                 stats[8 * q + 5], stats[8 * q + 6], stats[8 * q + 7]);
      }
      for (int e : Lv.spars_edges) {
        rows_[e] = size_[st_.edges[e].n2];
        cols_[e] = size_[st_.edges[e].n1];
      }
      lt_[lvl].nspars = (int)Lv.spars_clusters.size();
    } else {
      cudaEventRecord(fe[1], stream_);
      cudaEventRecord(ev[2], stream_);
      cudaEventRecord(fe[2], stream_);
      cudaEventRecord(ev[3], stream_);
    }
    // ---------------- merge into the next level
    if (lvl + 1 < L) {
      const Level& N = st_.levels[lvl + 1];
      for (int P = N.first; P < N.first + N.count; ++P) {
        const Cluster& C = st_.clusters[P];
        int off = 0;
        for (int k = C.child_begin; k < C.child_end; ++k) {
          const int ch = st_.children[k];
          rpos_[ch] = off;
          off += size_[ch];
        }
        size_[P] = size_org_[P] = off;
      }
      for (int e : N.edges) {
        const Edge& E = st_.edges[e];
        rows_[e] = size_[E.n2];
        cols_[e] = size_[E.n1];
      }
      if (int rc = alloc_level_blocks(N.edges)) return rc;
      // the merge list also depends on the kept ranks of the level's interfaces
      std::vector<int> mkey;
      mkey.reserve(Lv.spars_clusters.size());
      for (int p : Lv.spars_clusters) mkey.push_back(size_[p]);
      const bool mreuse = hit && P.merge_valid && P.merge_key == mkey;
      std::vector<MergeTask>& mt = P.mt;
      if (!mreuse) {
        mt.clear();
        P.merge_key = std::move(mkey);
      }
      for (size_t q = 0; !mreuse && q < Lv.merge_src.size(); ++q) {
        const int s = Lv.merge_src[q], d = Lv.merge_dst[q];
        const Edge& E = st_.edges[s];
        MergeTask t;
        t.src = ptr_[s];
        t.dst = ptr_[d];
        t.ld_src = ld_[s];
        t.ld_dst = ld_[d];
        t.rows = size_[E.n2];
        t.cols = size_[E.n1];
        t.roff = rpos_[E.n2];
        t.coff = rpos_[E.n1];
        t.identity = (E.n1 == E.n2 && st_.clusters[E.n1].sparsify) ? 1 : 0;
        // one CTA per slab of at most about 16K elements
        const int slab = std::max(1, 16384 / std::max(t.rows, 1));
        for (int c0 = 0; t.rows > 0 && c0 < t.cols; c0 += slab) {
          MergeTask u = t;
          u.c0 = c0;
          u.cols = std::min(slab, t.cols - c0);
          mt.push_back(u);
        }
      }
      P.merge_valid = true;
      if (check_descriptors) {
        const size_t es = fp32_ ? 4 : 8;
        for (const MergeTask& m : mt)
          if (!arena_.contains(m.src, es * ((size_t)m.ld_src * (m.c0 + m.cols - 1) + m.rows)) ||
              !arena_.contains(m.dst, es * ((size_t)m.ld_dst * (m.coff + m.c0 + m.cols - 1) + m.roff + m.rows)))
            return fail(-5, "merge descriptor of level " + std::to_string(lvl) +
                                " addresses memory outside the block pool; nothing launched");
      }
      auto* d_mt = static_cast<MergeTask*>(upload(mt.data(), sizeof(MergeTask) * mt.size()));
      if (!d_mt) return fail(-11, "out of device memory (merge)");
      if (ck(launch_merge(d_mt, (int)mt.size(), stream_), "merge kernel")) return -10;
    }
    if (!P.valid) {  // every list of the level is stored
      std::vector<size_t> off;
      size_t cur = 0;
      arena_.state(P.abase_end, off, cur);
      scratch_.state(P.sbase_end, off, cur);
      P.valid = true;
    }
    cudaEventRecord(ev[4], stream_);
    const double h1 = wall();
    // the status word comes back with the level's synchronisation (staged in
    // pinned memory), not through a second blocking copy
    int* h_status = d_status_ ? static_cast<int*>(stage(sizeof(int))) : nullptr;
    if (h_status) {
      *h_status = 0;
      cudaMemcpyAsync(h_status, d_status_, sizeof(int), cudaMemcpyDeviceToHost, stream_);
    }
    if (ck(cudaStreamSynchronize(stream_), "factorize level")) return -10;
    if (const int ds = h_status ? *h_status : device_status()) {
      clear_status();
      if (ds & 2) return fail(-12, "tensor-core MMA wait timed out on the device at level " + std::to_string(lvl));
      return fail(-13, std::string(ds & 4 ? "non-finite" : "zero") + " pivot in the QR factorizations of level " +
                           std::to_string(lvl));
    }
    if (verbose >= 2) {
      float gpu_ms = 0;
      cudaEventElapsedTime(&gpu_ms, ev[0], ev[4]);
      printf("level %d host: busy %.2f ms, waits %.2f + final %.2f ms, GPU level %.2f ms\n", lvl,
             1e3 * (h1 - h0 - hwait), 1e3 * hwait, 1e3 * (wall() - h1), gpu_ms);
    }
    cudaEventElapsedTime(&lt_[lvl].elim_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&lt_[lvl].scale_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&lt_[lvl].spars_ms, ev[2], ev[3]);
    cudaEventElapsedTime(&lt_[lvl].merge_ms, ev[3], ev[4]);
    cudaEventElapsedTime(&lt_[lvl].e1_ms, ev[0], fe[0]);
    cudaEventElapsedTime(&lt_[lvl].e2_ms, fe[0], ev[1]);
    cudaEventElapsedTime(&lt_[lvl].sqr_ms, ev[1], fe[1]);
    cudaEventElapsedTime(&lt_[lvl].sapp_ms, fe[1], ev[2]);
    cudaEventElapsedTime(&lt_[lvl].rrqr_ms, ev[2], fe[2]);
    cudaEventElapsedTime(&lt_[lvl].capp_ms, fe[2], ev[3]);
    if (spars) {
      float a = 0, b = 0, c = 0;
      cudaEventElapsedTime(&a, fe[1], fe[3]);  // row scaling
      cudaEventElapsedTime(&b, fe[2], fe[4]);  // right compression
      cudaEventElapsedTime(&c, fe[4], ev[3]);  // left compression
      lt_[lvl].kind_ms[1] = a + c;
      lt_[lvl].kind_ms[2] = b;
    }
    lt_[lvl].kind_ms[0] = lt_[lvl].e2_ms;
    scratch_.reset();
    if (verbose)
      printf("%d    elim %.3f ms  scale %.3f ms  spars %.3f ms  merge %.3f ms  (interiors %zu, interfaces %zu)\n", lvl,
             lt_[lvl].elim_ms, lt_[lvl].scale_ms, lt_[lvl].spars_ms, lt_[lvl].merge_ms, Lv.interiors.size(),
             Lv.interfaces.size());
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (auto& e : fe) cudaEventDestroy(e);
  for (const LevelTiming& t : lt_)
    for (double f : t.flops) flops_ += f;
  // tuning of the float applies: the first two factorizations measure each
  // level's applies on the tensor cores, then on the CUDA cores
  if (fp32_ && tensor_cores == 2 && tune_runs_ < 2) {
    tune_ms_[tune_runs_].assign(L, {0.f, 0.f, 0.f});
    for (int l = 0; l < L; ++l)
      for (int k = 0; k < 3; ++k) tune_ms_[tune_runs_][l][k] = lt_[l].kind_ms[k];
    ++tune_runs_;
  }
  factorized_ = true;
  int rc = build_solve_graph();
  if (rc) return rc;
  t_factorize = wall() - t0;
  if (verbose) {
    printf("Tolerance set: %e\n", tol);
    printf("Time to factorize:  %g\n", t_factorize);
  }
  return 0;
}

bool Tree::use_tc(int lvl, int kind) const {
  if (!fp32_ || tensor_cores == 0) return false;
  if (tensor_cores == 1) return true;
  if (tune_runs_ < 2) return tune_runs_ == 0;  // measuring: tensor cores first, then CUDA cores
  // the tensor cores only where they were clearly faster: near-ties (a level
  // whose two timings differ by a few microseconds) would otherwise flip from
  // run to run and with them the rounding of the factor
  return tune_ms_[0][lvl][kind] < kTuneMargin * tune_ms_[1][lvl][kind];
}

void Tree::tune_table(std::vector<float>& out) const {
  const int L = st_.nlevels;
  out.assign((size_t)L * 9, -1.f);
  for (int l = 0; l < L; ++l)
    for (int k = 0; k < 3; ++k) {
      float* o = out.data() + (size_t)l * 9 + 3 * k;
      if (tune_runs_ >= 1 && (int)tune_ms_[0].size() == L) o[0] = tune_ms_[0][l][k];
      if (tune_runs_ >= 2 && (int)tune_ms_[1].size() == L) {
        o[1] = tune_ms_[1][l][k];
        o[2] = use_tc(l, k) ? 1.f : 0.f;  // the choice the factorizations make
      }
    }
}

int Tree::alloc_level_blocks(const std::vector<int>& edges) {
  // blocks padded to 32 doubles (256 B) so every block starts aligned
  size_t total = 0;
  for (int e : edges) {
    ld_[e] = std::max(1, rows_[e]);
    total += ((size_t)ld_[e] * cols_[e] + 31) / 32 * 32;
  }
  double* base = arena_.dalloc(std::max<size_t>(total, 32));
  if (!base) return fail(-11, "out of device memory (level blocks)");
  size_t off = 0;
  for (int e : edges) {
    ptr_[e] = base + off;
    off += ((size_t)ld_[e] * cols_[e] + 31) / 32 * 32;
  }
  if (check_cuda(cudaMemsetAsync(base, 0, sizeof(double) * std::max<size_t>(total, 32), stream_), "memset")) return -10;
  return 0;
}

// Cluster vectors: level-0 clusters at their permuted columns [0, n); every
// later cluster gets its own segment of its level size.
// Descriptors of one vector's preconditioner apply: per level the forward
// elimination / sparsification tasks, the backward ones and the merge index
// maps, all addressing the cluster vectors of the workspace xw (turn counters
// in turn).  Uploaded into the block pool.
int Tree::plan_solve(double* xw, int* turn, std::vector<SolvePlan>& ls) {
  const int L = st_.nlevels;
  ls.assign(L, SolvePlan());
  auto up = [&](const void* h, size_t bytes) -> void* {
    void* d = arena_.alloc(std::max<size_t>(bytes, 1));
    if (d && bytes && h) cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream_);
    return d;
  };
  for (int lvl = 0; lvl < L; ++lvl) {
    const Level& Lv = st_.levels[lvl];
    SolvePlan& S = ls[lvl];
    // turn order per neighbour: interiors ascending
    std::vector<int> seen(Lv.count, 0);
    std::vector<FwdElimTask> fe;
    std::vector<FwdOut> fo;
    for (size_t ii = 0; ii < Lv.interiors.size(); ++ii) {
      const int c = Lv.interiors[ii];
      FwdElimTask t;
      t.S = ptr_[Lv.self_edge_of[c - Lv.first]];
      t.T = T_[c];
      t.x = elem(xw, xoff_[c]);
      t.n = size_[c];
      t.out_begin = (int)fo.size();
      for (int q = Lv.out_begin[ii]; q < Lv.out_end[ii]; ++q) {
        const int e = Lv.out_edges[q];
        const int nb = st_.edges[e].n2;
        FwdOut o;
        o.V = ptr_[e];
        o.T = tsqrtT_[e];
        o.xn = elem(xw, xoff_[nb]);
        o.turn = turn + nb;
        o.m = rows_[e];
        o.my_turn = seen[nb - Lv.first]++;
        fo.push_back(o);
        S.fe_mmax = std::max(S.fe_mmax, o.m);
      }
      t.out_end = (int)fo.size();
      fe.push_back(t);
      S.fe_nmax = std::max(S.fe_nmax, t.n);
    }
    std::vector<FwdSparsTask> fs;
    for (int p : Lv.spars_clusters) {
      FwdSparsTask t;
      t.Qs = ptr_[Lv.self_edge_of[p - Lv.first]];
      t.Ts = Ts_[p];
      t.V = Qsp_[p];
      t.T = Tsp_[p];
      t.rank = d_rank_ + p;
      t.x = elem(xw, xoff_[p]);
      t.n = size_org_[p];
      fs.push_back(t);
      S.fs_nmax = std::max(S.fs_nmax, t.n);
    }
    std::vector<BwdElimTask> be;
    std::vector<BwdIn> bi;
    for (size_t ii = 0; ii < Lv.interiors.size(); ++ii) {
      const int c = Lv.interiors[ii];
      BwdElimTask t;
      t.S = ptr_[Lv.self_edge_of[c - Lv.first]];
      t.x = elem(xw, xoff_[c]);
      t.n = size_[c];
      t.in_begin = (int)bi.size();
      for (int q = Lv.in_begin[ii]; q < Lv.in_end[ii]; ++q) {
        const int e = Lv.in_edges[q];
        BwdIn b;
        b.R = ptr_[e];
        b.ldr = ld_[e];
        b.s = cols_[e];
        b.xm = elem(xw, xoff_[st_.edges[e].n1]);
        bi.push_back(b);
      }
      t.in_end = (int)bi.size();
      be.push_back(t);
      S.be_nmax = std::max(S.be_nmax, t.n);
    }
    std::vector<int> gs, gd;
    if (lvl + 1 < L) {
      const Level& N = st_.levels[lvl + 1];
      for (int P = N.first; P < N.first + N.count; ++P) {
        const Cluster& C = st_.clusters[P];
        for (int k = C.child_begin; k < C.child_end; ++k) {
          const int ch = st_.children[k];
          for (int i = 0; i < size_[ch]; ++i) {
            gs.push_back((int)(xoff_[ch] + i));
            gd.push_back((int)(xoff_[P] + rpos_[ch] + i));
          }
        }
      }
    }
    S.nfe = (int)fe.size();
    S.nfs = (int)fs.size();
    if (fp32_)
      S.nfs_small = (int)(std::stable_partition(fs.begin(), fs.end(),
                                                [](const FwdSparsTask& t) { return spars_small(t.n); }) -
                          fs.begin());
    S.nbe = (int)be.size();
    S.ng = (int)gs.size();
    S.fe = static_cast<FwdElimTask*>(up(fe.data(), sizeof(FwdElimTask) * fe.size()));
    S.fo = static_cast<FwdOut*>(up(fo.data(), sizeof(FwdOut) * fo.size()));
    S.fs = static_cast<FwdSparsTask*>(up(fs.data(), sizeof(FwdSparsTask) * fs.size()));
    S.be = static_cast<BwdElimTask*>(up(be.data(), sizeof(BwdElimTask) * be.size()));
    S.bi = static_cast<BwdIn*>(up(bi.data(), sizeof(BwdIn) * bi.size()));
    S.gsrc = static_cast<int*>(up(gs.data(), sizeof(int) * gs.size()));
    S.gdst = static_cast<int*>(up(gd.data(), sizeof(int) * gd.size()));
    if (!S.fe || !S.fo || !S.fs || !S.be || !S.bi || !S.gsrc || !S.gdst)
      return fail(-11, "out of device memory (solve descriptors)");
  }
  return check_cuda(cudaStreamSynchronize(stream_), "solve descriptors");
}

// Captures one vector's sweep (forward levels, then backward levels) into *g.
int Tree::capture_solve(const std::vector<SolvePlan>& ls, double* xw, int* turn, int* tickets, cudaGraph_t* g,
                        long long* kernels) {
  const int L = st_.nlevels;
  const int ncl = (int)st_.clusters.size();
  if (check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture")) return -10;
  const long long launches_before = kernel_launches();
  cudaError_t cerr = cudaSuccess;
  cudaMemsetAsync(turn, 0, sizeof(int) * ncl, stream_);
  cudaMemsetAsync(tickets, 0, sizeof(int) * L, stream_);
  for (int lvl = 0; lvl < L; ++lvl) {
    const SolvePlan& S = ls[lvl];
    cerr = cerr ? cerr : launch_fwd_elim(S.fe, S.fo, S.nfe, S.fe_nmax, S.fe_mmax, tickets + lvl, d_status_, spin_limit, stream_);
    cerr = cerr ? cerr : launch_spars_small(true, S.fs, S.nfs_small, stream_);
    cerr = cerr ? cerr : launch_fwd_spars(S.fs + S.nfs_small, S.nfs - S.nfs_small, S.fs_nmax, stream_);
    cerr = cerr ? cerr : launch_copy_idx(S.ng, S.gsrc, S.gdst, xw, stream_);
  }
  for (int lvl = L - 1; lvl >= 0; --lvl) {
    const SolvePlan& S = ls[lvl];
    cerr = cerr ? cerr : launch_spars_small(false, S.fs, S.nfs_small, stream_);
    cerr = cerr ? cerr : launch_bwd_spars(S.fs + S.nfs_small, S.nfs - S.nfs_small, S.fs_nmax, stream_);
    cerr = cerr ? cerr : launch_bwd_elim(S.be, S.bi, S.nbe, S.be_nmax, stream_);
    if (lvl > 0) cerr = cerr ? cerr : launch_copy_idx(ls[lvl - 1].ng, ls[lvl - 1].gdst, ls[lvl - 1].gsrc, xw, stream_);
  }
  *kernels = kernel_launches() - launches_before;
  add_kernel_launches(-*kernels);  // captured, not executed
  cudaError_t ce = cudaStreamEndCapture(stream_, g);
  if (check_cuda(cerr, "solve kernel launch") || check_cuda(ce, "end capture")) return -10;
  return 0;
}

int Tree::build_solve_graph() {
  set_factor_fp32(fp32_);
  const int L = st_.nlevels;
  const int ncl = (int)st_.clusters.size();
  xoff_.assign(ncl, 0);
  int64_t off = st_.n;
  const Level& L0 = st_.levels[0];
  for (int o = L0.first; o < L0.first + L0.count; ++o) xoff_[o] = st_.clusters[o].cstart;
  for (int o = L0.first + L0.count; o < ncl; ++o) {
    xoff_[o] = off;
    off += size_org_[o];
  }
  xw_size_ = off;
  cudaFree(d_xw_);
  cudaFree(d_turn_);
  cudaFree(d_tickets_);
  d_xw_ = nullptr, d_turn_ = nullptr, d_tickets_ = nullptr;
  release_block_solve();
  if (check_cuda(cudaMalloc(&d_xw_, sizeof(double) * std::max<int64_t>(xw_size_, 1)), "malloc") ||
      check_cuda(cudaMalloc(&d_turn_, sizeof(int) * ncl), "malloc") ||
      check_cuda(cudaMalloc(&d_tickets_, sizeof(int) * L), "malloc"))
    return -10;
  std::vector<SolvePlan> ls;
  if (int rc = plan_solve(d_xw_, d_turn_, ls)) return rc;
  if (solve_exec_) {
    cudaGraphExecDestroy(solve_exec_);
    cudaGraphDestroy(solve_graph_);
    solve_exec_ = nullptr;
  }
  if (int rc = capture_solve(ls, d_xw_, d_turn_, d_tickets_, &solve_graph_, &solve_graph_kernels_)) return rc;
  if (check_cuda(cudaGraphInstantiate(&solve_exec_, solve_graph_, 0), "instantiate")) return -10;
  return 0;
}

void Tree::release_block_solve() {
  if (block_exec_) cudaGraphExecDestroy(block_exec_);
  if (block_graph_) cudaGraphDestroy(block_graph_);
  block_exec_ = nullptr;
  block_graph_ = nullptr;
  cudaFree(d_xwb_);
  cudaFree(d_turnb_);
  cudaFree(d_ticketsb_);
  d_xwb_ = nullptr, d_turnb_ = nullptr, d_ticketsb_ = nullptr;
  block_nrhs_ = 0;
  block_graph_kernels_ = 0;
}

// The preconditioner apply of nrhs vectors as one graph: nrhs independent
// sweeps (own workspace, turn counters and tickets each) as parallel branches,
// so that the GPU runs them concurrently.  Built on first use per factorization
// and nrhs (it allocates), reused after.
int Tree::build_block_solve(int nrhs) {
  if (block_exec_ && block_nrhs_ == nrhs) return 0;
  release_block_solve();
  const int L = st_.nlevels;
  const int ncl = (int)st_.clusters.size();
  if (check_cuda(cudaMalloc(&d_xwb_, sizeof(double) * (size_t)std::max<int64_t>(xw_size_, 1) * nrhs), "malloc") ||
      check_cuda(cudaMalloc(&d_turnb_, sizeof(int) * (size_t)ncl * nrhs), "malloc") ||
      check_cuda(cudaMalloc(&d_ticketsb_, sizeof(int) * (size_t)L * nrhs), "malloc"))
    return -11;
  if (check_cuda(cudaGraphCreate(&block_graph_, 0), "graph")) return -10;
  set_factor_fp32(fp32_);
  for (int r = 0; r < nrhs; ++r) {
    double* xw = elem(d_xwb_, (size_t)r * xw_size_);
    std::vector<SolvePlan> ls;
    if (int rc = plan_solve(xw, d_turnb_ + (size_t)r * ncl, ls)) return rc;
    cudaGraph_t g = nullptr;
    long long nk = 0;
    if (int rc = capture_solve(ls, xw, d_turnb_ + (size_t)r * ncl, d_ticketsb_ + (size_t)r * L, &g, &nk)) return rc;
    cudaGraphNode_t node;
    const cudaError_t e = cudaGraphAddChildGraphNode(&node, block_graph_, nullptr, 0, g);
    cudaGraphDestroy(g);  // the child node holds a copy
    if (check_cuda(e, "block solve graph")) return -10;
    block_graph_kernels_ += nk;
  }
  if (check_cuda(cudaGraphInstantiate(&block_exec_, block_graph_, 0), "instantiate block solve")) return -10;
  block_nrhs_ = nrhs;
  return 0;
}

// M^{-1} x in place for the device vectors cols[0..nrhs) (permuted order), as
// one block graph launch.
int Tree::solve_block_cols(const std::vector<double*>& cols) {
  if (!factorized_) return fail(-4, "solve called before factorize");
  const int nrhs = (int)cols.size();
  if (int rc = build_block_solve(nrhs)) return rc;
  const int n = st_.n;
  set_factor_fp32(fp32_);
  for (int r = 0; r < nrhs; ++r) {
    double* xw = elem(d_xwb_, (size_t)r * xw_size_);
    if (fp32_) {
      if (check_cuda(launch_to_f32(n, cols[r], xw, stream_), "block solve input")) return -10;
    } else {
      cudaMemcpyAsync(xw, cols[r], sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
    }
  }
  if (check_cuda(cudaGraphLaunch(block_exec_, stream_), "block solve graph")) return -10;
  add_kernel_launches(block_graph_kernels_);
  for (int r = 0; r < nrhs; ++r) {
    double* xw = elem(d_xwb_, (size_t)r * xw_size_);
    if (fp32_) {
      if (check_cuda(launch_to_f64(n, xw, cols[r], stream_), "block solve output")) return -10;
    } else {
      cudaMemcpyAsync(cols[r], xw, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
    }
  }
  return 0;
}

// M^{-1} X for nrhs device vectors (column r at X + r * ldx, permuted order).
int Tree::solve_block_device(double* X, int nrhs, size_t ldx) {
  if (nrhs < 1 || ldx < (size_t)st_.n) return fail(-1, "solve_block: nrhs >= 1 and ldx >= n required");
  clear_status();
  std::vector<double*> cols(nrhs);
  for (int r = 0; r < nrhs; ++r) cols[r] = X + (size_t)r * ldx;
  return solve_block_cols(cols);
}

// Flexible GMRES for nrhs right-hand sides in lockstep: every iteration applies
// the preconditioner to all of them in one block graph, runs the SpMV and the
// modified Gram-Schmidt of each, and reads all Hessenberg columns back with one
// synchronisation.  A right-hand side that has converged is frozen (its later
// columns are computed but not used).  B (device, column r at B + r * ldb) is
// overwritten by the solutions; iters[r] / relres[r] as fgmres_device.
int Tree::block_fgmres_device(double* B, int nrhs, size_t ldb, int maxit, double gtol, int* iters,
                              double* relres) {
  if (!factorized_) return fail(-4, "gmres called before factorize");
  if (maxit < 1 || nrhs < 1 || ldb < (size_t)st_.n) return fail(-1, "block gmres: maxit, nrhs >= 1, ldb >= n");
  clear_status();
  double t0 = wall();
  const int n = st_.n;
  const size_t ldq = (size_t)n;
  const int grid = mgs_grid(n);
  // per right-hand side: V (n x maxit+1) | Z (n x maxit) | q | b | H column;
  // then the shared partial sums and counter
  const size_t hcap = (size_t)maxit + 3;
  const size_t per = ldq * (2 * (size_t)maxit + 1) + 2 * ldq + hcap;
  if (int erc = ensure_krylov(per * nrhs + grid + 1)) return erc;
  auto Vr = [&](int r) { return d_krylov_ + per * r; };
  auto Zr = [&](int r) { return Vr(r) + ldq * (maxit + 1); };
  auto qr = [&](int r) { return Zr(r) + ldq * maxit; };
  auto br = [&](int r) { return qr(r) + ldq; };
  auto hr = [&](int r) { return br(r) + ldq; };
  double* partial = d_krylov_ + per * nrhs;
  unsigned int* done = reinterpret_cast<unsigned int*>(partial + grid);
  cudaError_t ge = cudaSuccess;
  auto g = [&](cudaError_t e) {
    if (!ge) ge = e;
  };
  g(cudaMemsetAsync(done, 0, sizeof(unsigned int), stream_));
  for (int r = 0; r < nrhs; ++r) {
    g(cudaMemcpyAsync(br(r), B + (size_t)r * ldb, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
    g(cudaMemcpyAsync(qr(r), br(r), sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
    g(launch_mgs_step(n, qr(r), nullptr, nullptr, nullptr, partial, done, hr(r), 1, stream_));  // ||b||
    g(launch_scale_copy(n, qr(r), hr(r), Vr(r), stream_));
  }
  std::vector<double> hk(hcap * nrhs, 0.0);
  auto readback = [&](int cnt) {
    for (int r = 0; r < nrhs; ++r)
      g(cudaMemcpyAsync(hk.data() + hcap * r, hr(r), sizeof(double) * cnt, cudaMemcpyDeviceToHost, stream_));
    return check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "block gmres");
  };
  int rc = readback(1);
  std::vector<double> rnorm(nrhs);
  for (int r = 0; r < nrhs; ++r) rnorm[r] = hk[hcap * r];
  const size_t hs = (size_t)(maxit + 1) * maxit;
  std::vector<double> H(hs * nrhs, 0.0), cs((size_t)maxit * nrhs, 0.0), sn((size_t)maxit * nrhs, 0.0),
      beta((size_t)(maxit + 1) * nrhs, 0.0);
  std::vector<int> kfin(nrhs, -1);
  for (int r = 0; r < nrhs; ++r) {
    beta[(size_t)(maxit + 1) * r] = rnorm[r];
    if (!rc && !(rnorm[r] > 0)) rc = fail(-1, "zero or invalid right-hand side " + std::to_string(r));
  }
  int k = 0, active = nrhs;
  for (; !rc && k < maxit && active > 0; ++k) {
    // Z(:, k) = M^{-1} V(:, k) for every right-hand side: the block apply works
    // on the columns Z_r(:, k) in place
    for (int r = 0; r < nrhs; ++r)
      g(cudaMemcpyAsync(Zr(r) + (size_t)k * ldq, Vr(r) + (size_t)k * ldq, sizeof(double) * n,
                        cudaMemcpyDeviceToDevice, stream_));
    if (ge) break;
    std::vector<double*> zk(nrhs);
    for (int r = 0; r < nrhs; ++r) zk[r] = Zr(r) + (size_t)k * ldq;
    if ((rc = solve_block_cols(zk))) break;
    for (int r = 0; r < nrhs; ++r) {
      double* zk = Zr(r) + (size_t)k * ldq;
      double* Q = Vr(r);
      double* q = qr(r);
      double* hcol = hr(r);
      if ((rc = spmv_device(zk, q))) break;
      for (int i = 0; i <= k; ++i)
        g(launch_mgs_step(n, q, i ? Q + (size_t)(i - 1) * ldq : nullptr, i ? hcol + (i - 1) : nullptr,
                          Q + (size_t)i * ldq, partial, done, hcol + i, 0, stream_));
      g(launch_mgs_step(n, q, Q + (size_t)k * ldq, hcol + k, nullptr, partial, done, hcol + k + 1, 1, stream_));
      g(launch_scale_copy(n, q, hcol + k + 1, Q + (size_t)(k + 1) * ldq, stream_));
    }
    if (rc || (rc = readback(k + 2))) break;
    for (int r = 0; r < nrhs; ++r) {
      if (kfin[r] >= 0) continue;
      double* Hr = H.data() + hs * r;
      double* c = cs.data() + (size_t)maxit * r;
      double* s2 = sn.data() + (size_t)maxit * r;
      double* be = beta.data() + (size_t)(maxit + 1) * r;
      auto Hc = [&](int i, int j) -> double& { return Hr[(size_t)j * (maxit + 1) + i]; };
      for (int i = 0; i <= k + 1; ++i) Hc(i, k) = hk[hcap * r + i];
      for (int i = 0; i < k; ++i) {
        const double temp = c[i] * Hc(i, k) + s2[i] * Hc(i + 1, k);
        Hc(i + 1, k) = -s2[i] * Hc(i, k) + c[i] * Hc(i + 1, k);
        Hc(i, k) = temp;
      }
      if (Hc(k, k) == 0) {
        c[k] = 0;
        s2[k] = 1;
      } else {
        const double t = std::sqrt(Hc(k, k) * Hc(k, k) + Hc(k + 1, k) * Hc(k + 1, k));
        c[k] = std::fabs(Hc(k, k)) / t;
        s2[k] = c[k] * Hc(k + 1, k) / Hc(k, k);
      }
      Hc(k, k) = c[k] * Hc(k, k) + s2[k] * Hc(k + 1, k);
      Hc(k + 1, k) = 0.0;
      be[k + 1] = -s2[k] * be[k];
      be[k] = c[k] * be[k];
      const double err = std::fabs(be[k + 1]) / rnorm[r];
      if (verbose) printf("block FGMRES: rhs %d error at step %d is %e\n", r, k, err);
      if (err <= gtol || k + 1 == maxit) {
        kfin[r] = k;
        --active;
      }
    }
  }
  if (!rc && device_status() != 0) rc = fail(-12, "forward sweep wait timed out on the device");
  if (!rc) {
    std::vector<double> nr(2 * nrhs, 1.0);
    for (int r = 0; r < nrhs; ++r) {
      const int kr = kfin[r] >= 0 ? kfin[r] : std::min(k, maxit) - 1;
      double* Hr = H.data() + hs * r;
      double* be = beta.data() + (size_t)(maxit + 1) * r;
      auto Hc = [&](int i, int j) -> double& { return Hr[(size_t)j * (maxit + 1) + i]; };
      std::vector<double> y(kr + 1, 0.0);
      for (int i = kr; i >= 0; --i) {
        y[i] = be[i];
        for (int j = i + 1; j < kr + 1; ++j) y[i] -= Hc(i, j) * y[j];
        y[i] /= Hc(i, i);
      }
      double* x = B + (size_t)r * ldb;
      double* q = qr(r);
      double* hcol = hr(r);
      g(cudaMemcpyAsync(hcol, y.data(), sizeof(double) * (kr + 1), cudaMemcpyHostToDevice, stream_));
      g(launch_combine(n, kr + 1, Zr(r), ldq, hcol, x, stream_));
      g(spmv_device(x, q) ? cudaErrorUnknown : cudaSuccess);
      g(launch_sub(n, br(r), q, q, stream_));
      g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));
      g(launch_mgs_step(n, br(r), nullptr, nullptr, nullptr, partial, done, hcol + 1, 1, stream_));
      g(cudaMemcpyAsync(nr.data() + 2 * r, hcol, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_));
      // the host copy of y must stay alive until the copy has run
      if ((rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "block gmres finish"))) break;
      iters[r] = kr;
    }
    for (int r = 0; !rc && r < nrhs; ++r) relres[r] = nr[2 * r] / nr[2 * r + 1];
  }
  t_gmres = wall() - t0;
  return rc;
}

int Tree::solve_device(double* x) {
  if (!factorized_) return fail(-4, "solve called before factorize");
  const int n = st_.n;
  set_factor_fp32(fp32_);
  if (fp32_) {
    // the preconditioner applies in the factors' precision
    if (check_cuda(launch_to_f32(n, x, d_xw_, stream_), "solve input")) return -10;
  } else {
    cudaMemcpyAsync(d_xw_, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
  }
  if (check_cuda(cudaGraphLaunch(solve_exec_, stream_), "solve graph")) return -10;
  add_kernel_launches(solve_graph_kernels_);
  if (fp32_) {
    if (check_cuda(launch_to_f64(n, d_xw_, x, stream_), "solve output")) return -10;
  } else {
    cudaMemcpyAsync(x, d_xw_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
  }
  return 0;
}

int Tree::solve_host(double* x) {
  double t0 = wall();
  const int n = st_.n;
  if (!factorized_) return fail(-4, "solve called before factorize");
  clear_status();
  cudaMemcpyAsync(d_tmp_, x, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  int rc = solve_device(d_tmp_);
  if (rc) return rc;
  cudaMemcpyAsync(x, d_tmp_, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
  if (check_cuda(cudaStreamSynchronize(stream_), "solve")) return -10;
  if (device_status() != 0) return fail(-12, "forward sweep wait timed out on the device");
  t_solve = wall() - t0;
  return 0;
}

int Tree::backward_error(int nprobe, const double* U, unsigned long long seed, double* eta) {
  if (!factorized_) return fail(-4, "backward error called before factorize");
  if (nprobe < 1 || !eta) return fail(-1, "backward error: nprobe >= 1 and an output array are required");
  const int n = st_.n;
  std::vector<double> u(n), y(n);
  for (int p = 0; p < nprobe; ++p) {
    if (U) {
      std::copy(U + (size_t)p * n, U + (size_t)(p + 1) * n, u.begin());
    } else {
      std::mt19937_64 gen(seed + (unsigned long long)p);
      std::normal_distribution<double> nd(0.0, 1.0);
      for (double& v : u) v = nd(gen);
    }
    clear_status();
    cudaMemcpyAsync(d_tmp_, u.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
    if (int rc = solve_device(d_tmp_)) return rc;
    if (int rc = spmv_device(d_tmp_, d_tmp_ + n)) return rc;
    cudaMemcpyAsync(y.data(), d_tmp_ + n, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
    if (check_cuda(cudaStreamSynchronize(stream_), "backward error")) return -10;
    if (device_status() != 0) return fail(-12, "forward sweep wait timed out on the device");
    double r2 = 0, u2 = 0;
    for (int i = 0; i < n; ++i) {
      r2 += (y[i] - u[i]) * (y[i] - u[i]);
      u2 += u[i] * u[i];
    }
    eta[p] = std::sqrt(r2) / std::sqrt(u2);
  }
  return 0;
}

int Tree::solve_global(const double* b, double* x) {
  const int n = st_.n;
  std::vector<double> t(n);
  for (int i = 0; i < n; ++i) t[i] = b[st_.rperm[i]];
  int rc = solve_host(t.data());
  if (rc) return rc;
  for (int i = 0; i < n; ++i) x[st_.cperm[i]] = t[i];
  return 0;
}

int Tree::spmv_device(const double* x, double* y) {
  if (!assembled_) return fail(-4, "spmv called before assemble");
  return check_cuda(launch_spmv(st_.n, d_rowptr_, d_col_, d_val_, x, y, stream_), "spmv");
}

int Tree::spmv_host(const double* x, double* y) {
  const int n = st_.n;
  if (!assembled_) return fail(-4, "spmv called before assemble");
  cudaMemcpyAsync(d_tmp_, x, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  spmv_device(d_tmp_, d_tmp_ + n);
  cudaMemcpyAsync(y, d_tmp_ + n, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
  return check_cuda(cudaStreamSynchronize(stream_), "spmv");
}

// is.cpp:447-527: left-preconditioned, unrestarted GMRES with MGS Arnoldi,
// x0 = 0, stopping on the preconditioned residual |beta(k+1)|/||M^-1 b||.
// On exit b holds the solution; relres is the true ||b - A x|| / ||b||.
int Tree::gmres_device(double* b, int maxit, double gtol, int* iters, double* relres, double* hist, int hist_cap) {
  if (!factorized_) return fail(-4, "gmres called before factorize");
  if (krylov == 1 || (krylov < 0 && fp32_)) return fgmres_device(b, maxit, gtol, iters, relres, hist, hist_cap);
  if (maxit < 1) return fail(-1, "maxit must be >= 1");
  clear_status();
  double t0 = wall();
  const int n = st_.n;
  const size_t ldq = (size_t)n;
  const int grid = mgs_grid(n);
  // workspace: basis (n x maxit+1) | q | b | H column | partial sums | counter
  const size_t need = ldq * (maxit + 1) + 2 * (size_t)n + (maxit + 3) + grid + 1;
  if (int erc = ensure_krylov(need)) return erc;
  double* Q = d_krylov_;
  double* q = Q + ldq * (maxit + 1);
  double* bsave = q + n;
  double* hcol = bsave + n;
  double* partial = hcol + (maxit + 3);
  unsigned int* done = reinterpret_cast<unsigned int*>(partial + grid);
  cudaMemsetAsync(done, 0, sizeof(unsigned int), stream_);
  cudaMemcpyAsync(bsave, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
  cudaMemcpyAsync(q, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_);
  if (int src = solve_device(q)) return src;
  cudaError_t ge = cudaSuccess;
  auto g = [&](cudaError_t e) {
    if (!ge) ge = e;
  };
  g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));  // ||r||
  g(launch_scale_copy(n, q, hcol, Q, stream_));
  double r_norm = 0;
  cudaMemcpyAsync(&r_norm, hcol, sizeof(double), cudaMemcpyDeviceToHost, stream_);
  int rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres start");
  std::vector<double> H((size_t)(maxit + 1) * maxit, 0.0), cs(maxit, 0.0), sn(maxit, 0.0), beta(maxit + 1, 0.0);
  auto Hc = [&](int i, int j) -> double& { return H[(size_t)j * (maxit + 1) + i]; };
  beta[0] = r_norm;
  int k = 0;
  std::vector<double> hk(maxit + 2);
  int nh = 0;
  if (!rc && (std::isnan(r_norm) || device_status() != 0)) rc = fail(-12, "preconditioner apply failed");
  for (; !rc && k < maxit; ++k) {
    if ((rc = spmv_device(Q + (size_t)k * ldq, q)) || (rc = solve_device(q))) break;
    for (int i = 0; i <= k; ++i)
      g(launch_mgs_step(n, q, i ? Q + (size_t)(i - 1) * ldq : nullptr, i ? hcol + (i - 1) : nullptr,
                        Q + (size_t)i * ldq, partial, done, hcol + i, 0, stream_));
    g(launch_mgs_step(n, q, Q + (size_t)k * ldq, hcol + k, nullptr, partial, done, hcol + k + 1, 1, stream_));
    g(launch_scale_copy(n, q, hcol + k + 1, Q + (size_t)(k + 1) * ldq, stream_));
    cudaMemcpyAsync(hk.data(), hcol, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, stream_);
    if ((rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres iteration"))) break;
    for (int i = 0; i <= k + 1; ++i) Hc(i, k) = hk[i];
    for (int i = 0; i < k; ++i) {
      const double temp = cs[i] * Hc(i, k) + sn[i] * Hc(i + 1, k);
      Hc(i + 1, k) = -sn[i] * Hc(i, k) + cs[i] * Hc(i + 1, k);
      Hc(i, k) = temp;
    }
    if (Hc(k, k) == 0) {
      cs[k] = 0;
      sn[k] = 1;
    } else {
      const double t = std::sqrt(Hc(k, k) * Hc(k, k) + Hc(k + 1, k) * Hc(k + 1, k));
      cs[k] = std::fabs(Hc(k, k)) / t;
      sn[k] = cs[k] * Hc(k + 1, k) / Hc(k, k);
    }
    Hc(k, k) = cs[k] * Hc(k, k) + sn[k] * Hc(k + 1, k);
    Hc(k + 1, k) = 0.0;
    beta[k + 1] = -sn[k] * beta[k];
    beta[k] = cs[k] * beta[k];
    const double err = std::fabs(beta[k + 1]) / r_norm;
    if (hist && nh < hist_cap) hist[nh++] = err;
    if (verbose) printf("GMRES: error at step %d is %e\n", k, err);
    if (err <= gtol) break;
  }
  if (!rc) {
    if (device_status() != 0) rc = fail(-12, "forward sweep wait timed out on the device");
  }
  if (!rc) {
    k = std::min(k, maxit - 1);
    std::vector<double> y(k + 1, 0.0);  // util.cpp:1019-1032 LUSolve
    for (int i = k; i >= 0; --i) {
      y[i] = beta[i];
      for (int j = i + 1; j < k + 1; ++j) y[i] -= Hc(i, j) * y[j];
      y[i] /= Hc(i, i);
    }
    double* dy = hcol;
    cudaMemcpyAsync(dy, y.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, stream_);
    g(launch_combine(n, k + 1, Q, ldq, dy, b, stream_));
    g(spmv_device(b, q) ? cudaErrorUnknown : cudaSuccess);
    g(launch_sub(n, bsave, q, q, stream_));
    g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));
    g(launch_mgs_step(n, bsave, nullptr, nullptr, nullptr, partial, done, hcol + 1, 1, stream_));
    double nr[2] = {0, 1};
    cudaMemcpyAsync(nr, hcol, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_);
    rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres finish");
    *iters = k;
    *relres = nr[0] / nr[1];
    last_gmres_iters = k;
  }
  t_gmres = wall() - t0;
  return rc;
}

// The GMRES loop of gmres_device on a caller-given device workspace and fixed
// host arrays: nothing is allocated on the device or the heap.  The workspace
// counter the reductions use is cleared on every call.
int Tree::gmres_device_fixed(double* b, int maxit, double gtol, int* iters, double* relres, double* ws,
                             size_t ws_doubles) {
  if (!factorized_) return fail(-4, "gmres called before factorize");
  if (maxit < 1 || maxit > kNoAllocMaxit)
    return fail(-1, "maxit must be in [1, " + std::to_string(kNoAllocMaxit) + "] for the allocation-free GMRES");
  clear_status();
  double t0 = wall();
  const int n = st_.n;
  const size_t ldq = (size_t)n;
  const int grid = mgs_grid(n);
  const size_t need = ldq * (maxit + 1) + 2 * (size_t)n + (maxit + 3) + grid + 1;
  if (need > ws_doubles)
    return fail(-14, "allocation-free GMRES needs " + std::to_string(need) + " doubles of workspace, the fixed array holds " +
                         std::to_string(ws_doubles) + "; lower maxit or use spq_gmres_device");
  double* Q = ws;
  double* q = Q + ldq * (maxit + 1);
  double* bsave = q + n;
  double* hcol = bsave + n;
  double* partial = hcol + (maxit + 3);
  unsigned int* done = reinterpret_cast<unsigned int*>(partial + grid);
  cudaError_t ge = cudaSuccess;
  auto g = [&](cudaError_t e) {
    if (!ge) ge = e;
  };
  g(cudaMemsetAsync(done, 0, sizeof(unsigned int), stream_));
  g(cudaMemcpyAsync(bsave, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
  g(cudaMemcpyAsync(q, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
  if (ge) return check_cuda(ge, "gmres start");
  if (int src = solve_device(q)) return src;
  g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));  // ||r||
  g(launch_scale_copy(n, q, hcol, Q, stream_));
  double r_norm = 0;
  g(cudaMemcpyAsync(&r_norm, hcol, sizeof(double), cudaMemcpyDeviceToHost, stream_));
  int rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres start");
  constexpr int M = kNoAllocMaxit;
  double H[(M + 1) * M], cs[M], sn[M], beta[M + 1], hk[M + 2], y[M];
  for (int i = 0; i < (M + 1) * M; ++i) H[i] = 0.0;
  for (int i = 0; i < M; ++i) cs[i] = sn[i] = beta[i] = 0.0;
  beta[M] = 0.0;
  auto Hc = [&](int i, int j) -> double& { return H[(size_t)j * (maxit + 1) + i]; };
  beta[0] = r_norm;
  int k = 0;
  if (!rc && (std::isnan(r_norm) || device_status() != 0)) rc = fail(-12, "preconditioner apply failed");
  for (; !rc && k < maxit; ++k) {
    if ((rc = spmv_device(Q + (size_t)k * ldq, q)) || (rc = solve_device(q))) break;
    for (int i = 0; i <= k; ++i)
      g(launch_mgs_step(n, q, i ? Q + (size_t)(i - 1) * ldq : nullptr, i ? hcol + (i - 1) : nullptr,
                        Q + (size_t)i * ldq, partial, done, hcol + i, 0, stream_));
    g(launch_mgs_step(n, q, Q + (size_t)k * ldq, hcol + k, nullptr, partial, done, hcol + k + 1, 1, stream_));
    g(launch_scale_copy(n, q, hcol + k + 1, Q + (size_t)(k + 1) * ldq, stream_));
    g(cudaMemcpyAsync(hk, hcol, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, stream_));
    if ((rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres iteration"))) break;
    for (int i = 0; i <= k + 1; ++i) Hc(i, k) = hk[i];
    for (int i = 0; i < k; ++i) {
      const double temp = cs[i] * Hc(i, k) + sn[i] * Hc(i + 1, k);
      Hc(i + 1, k) = -sn[i] * Hc(i, k) + cs[i] * Hc(i + 1, k);
      Hc(i, k) = temp;
    }
    if (Hc(k, k) == 0) {
      cs[k] = 0;
      sn[k] = 1;
    } else {
      const double t = std::sqrt(Hc(k, k) * Hc(k, k) + Hc(k + 1, k) * Hc(k + 1, k));
      cs[k] = std::fabs(Hc(k, k)) / t;
      sn[k] = cs[k] * Hc(k + 1, k) / Hc(k, k);
    }
    Hc(k, k) = cs[k] * Hc(k, k) + sn[k] * Hc(k + 1, k);
    Hc(k + 1, k) = 0.0;
    beta[k + 1] = -sn[k] * beta[k];
    beta[k] = cs[k] * beta[k];
    const double err = std::fabs(beta[k + 1]) / r_norm;
    if (verbose) printf("GMRES: error at step %d is %e\n", k, err);
    if (err <= gtol) break;
  }
  if (!rc && device_status() != 0) rc = fail(-12, "forward sweep wait timed out on the device");
  if (!rc) {
    k = std::min(k, maxit - 1);
    for (int i = k; i >= 0; --i) {  // util.cpp:1019-1032 LUSolve
      y[i] = beta[i];
      for (int j = i + 1; j < k + 1; ++j) y[i] -= Hc(i, j) * y[j];
      y[i] /= Hc(i, i);
    }
    double* dy = hcol;
    g(cudaMemcpyAsync(dy, y, sizeof(double) * (k + 1), cudaMemcpyHostToDevice, stream_));
    g(launch_combine(n, k + 1, Q, ldq, dy, b, stream_));
    g(spmv_device(b, q) ? cudaErrorUnknown : cudaSuccess);
    g(launch_sub(n, bsave, q, q, stream_));
    g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));
    g(launch_mgs_step(n, bsave, nullptr, nullptr, nullptr, partial, done, hcol + 1, 1, stream_));
    double nr[2] = {0, 1};
    g(cudaMemcpyAsync(nr, hcol, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_));
    rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres finish");
    *iters = k;
    *relres = nr[0] / nr[1];
    last_gmres_iters = k;
  }
  t_gmres = wall() - t0;
  return rc;
}

int Tree::set_rank_model(const float* params, const float* mean, const float* stdev, int oversample) {
  learned_accepted_ = learned_fallbacks_ = learned_ell_ = 0;
  if (!params) {
    rank_model_ = false;
    return 0;
  }
  if (!mean || !stdev || oversample < 0) return fail(-1, "rank model: mean, std and oversample >= 0 required");
  for (int f = 0; f < kRankFeatures; ++f)
    if (!(stdev[f] > 0)) return fail(-1, "rank model: feature std must be positive");
  const size_t n = (size_t)kMlpParams + 2 * kRankFeatures;
  if (!d_model_ && check_cuda(cudaMalloc(&d_model_, sizeof(float) * n), "malloc rank model")) return -11;
  std::vector<float> h(n);
  std::copy(params, params + kMlpParams, h.begin());
  std::copy(mean, mean + kRankFeatures, h.begin() + kMlpParams);
  std::copy(stdev, stdev + kRankFeatures, h.begin() + kMlpParams + kRankFeatures);
  if (check_cuda(cudaMemcpy(d_model_, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "upload rank model"))
    return -10;
  rank_model_ = true;
  oversample_ = oversample;
  return 0;
}

// Flexible (right-preconditioned) GMRES: z_k = M^-1 v_k is kept, the Arnoldi
// relation is built on A z_k and x = Z y, so the Givens residual is the true
// residual ||b - A x|| (in exact arithmetic) whatever the accuracy of the
// preconditioner.  Used with the float factorization, whose preconditioner
// apply would contaminate the left-preconditioned residual below ~1e-7.
// No reference counterpart (the reference's is.cpp:447-527 is left GMRES).
int Tree::fgmres_device(double* b, int maxit, double gtol, int* iters, double* relres, double* hist, int hist_cap) {
  if (!factorized_) return fail(-4, "gmres called before factorize");
  if (maxit < 1) return fail(-1, "maxit must be >= 1");
  clear_status();
  double t0 = wall();
  const int n = st_.n;
  const size_t ldq = (size_t)n;
  const int grid = mgs_grid(n);
  // workspace: V (n x maxit+1) | Z (n x maxit) | q | b | H column | partial sums | counter
  const size_t need = ldq * (2 * (size_t)maxit + 1) + 2 * (size_t)n + (maxit + 3) + grid + 1;
  if (int erc = ensure_krylov(need)) return erc;
  double* Q = d_krylov_;
  double* Z = Q + ldq * (maxit + 1);
  double* q = Z + ldq * maxit;
  double* bsave = q + n;
  double* hcol = bsave + n;
  double* partial = hcol + (maxit + 3);
  unsigned int* done = reinterpret_cast<unsigned int*>(partial + grid);
  cudaError_t ge = cudaSuccess;
  auto g = [&](cudaError_t e) {
    if (!ge) ge = e;
  };
  g(cudaMemsetAsync(done, 0, sizeof(unsigned int), stream_));
  g(cudaMemcpyAsync(bsave, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
  g(cudaMemcpyAsync(q, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
  g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));  // ||b||
  g(launch_scale_copy(n, q, hcol, Q, stream_));
  double r_norm = 0;
  g(cudaMemcpyAsync(&r_norm, hcol, sizeof(double), cudaMemcpyDeviceToHost, stream_));
  int rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres start");
  std::vector<double> H((size_t)(maxit + 1) * maxit, 0.0), cs(maxit, 0.0), sn(maxit, 0.0), beta(maxit + 1, 0.0);
  auto Hc = [&](int i, int j) -> double& { return H[(size_t)j * (maxit + 1) + i]; };
  beta[0] = r_norm;
  int k = 0, nh = 0;
  std::vector<double> hk(maxit + 2);
  if (!rc && !(r_norm > 0)) rc = fail(-1, "zero or invalid right-hand side");
  for (; !rc && k < maxit; ++k) {
    double* zk = Z + (size_t)k * ldq;
    g(cudaMemcpyAsync(zk, Q + (size_t)k * ldq, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream_));
    if ((rc = solve_device(zk)) || (rc = spmv_device(zk, q))) break;
    for (int i = 0; i <= k; ++i)
      g(launch_mgs_step(n, q, i ? Q + (size_t)(i - 1) * ldq : nullptr, i ? hcol + (i - 1) : nullptr,
                        Q + (size_t)i * ldq, partial, done, hcol + i, 0, stream_));
    g(launch_mgs_step(n, q, Q + (size_t)k * ldq, hcol + k, nullptr, partial, done, hcol + k + 1, 1, stream_));
    g(launch_scale_copy(n, q, hcol + k + 1, Q + (size_t)(k + 1) * ldq, stream_));
    g(cudaMemcpyAsync(hk.data(), hcol, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, stream_));
    if ((rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres iteration"))) break;
    for (int i = 0; i <= k + 1; ++i) Hc(i, k) = hk[i];
    for (int i = 0; i < k; ++i) {
      const double temp = cs[i] * Hc(i, k) + sn[i] * Hc(i + 1, k);
      Hc(i + 1, k) = -sn[i] * Hc(i, k) + cs[i] * Hc(i + 1, k);
      Hc(i, k) = temp;
    }
    if (Hc(k, k) == 0) {
      cs[k] = 0;
      sn[k] = 1;
    } else {
      const double t = std::sqrt(Hc(k, k) * Hc(k, k) + Hc(k + 1, k) * Hc(k + 1, k));
      cs[k] = std::fabs(Hc(k, k)) / t;
      sn[k] = cs[k] * Hc(k + 1, k) / Hc(k, k);
    }
    Hc(k, k) = cs[k] * Hc(k, k) + sn[k] * Hc(k + 1, k);
    Hc(k + 1, k) = 0.0;
    beta[k + 1] = -sn[k] * beta[k];
    beta[k] = cs[k] * beta[k];
    const double err = std::fabs(beta[k + 1]) / r_norm;
    if (hist && nh < hist_cap) hist[nh++] = err;
    if (verbose) printf("FGMRES: error at step %d is %e\n", k, err);
    if (err <= gtol) break;
  }
  if (!rc && device_status() != 0) rc = fail(-12, "forward sweep wait timed out on the device");
  if (!rc) {
    k = std::min(k, maxit - 1);
    std::vector<double> y(k + 1, 0.0);
    for (int i = k; i >= 0; --i) {
      y[i] = beta[i];
      for (int j = i + 1; j < k + 1; ++j) y[i] -= Hc(i, j) * y[j];
      y[i] /= Hc(i, i);
    }
    double* dy = hcol;
    g(cudaMemcpyAsync(dy, y.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, stream_));
    g(launch_combine(n, k + 1, Z, ldq, dy, b, stream_));
    g(spmv_device(b, q) ? cudaErrorUnknown : cudaSuccess);
    g(launch_sub(n, bsave, q, q, stream_));
    g(launch_mgs_step(n, q, nullptr, nullptr, nullptr, partial, done, hcol, 1, stream_));
    g(launch_mgs_step(n, bsave, nullptr, nullptr, nullptr, partial, done, hcol + 1, 1, stream_));
    double nr[2] = {0, 1};
    g(cudaMemcpyAsync(nr, hcol, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_));
    rc = check_cuda(ge ? ge : cudaStreamSynchronize(stream_), "gmres finish");
    *iters = k;
    *relres = nr[0] / nr[1];
    last_gmres_iters = k;
  }
  t_gmres = wall() - t0;
  return rc;
}

// block_fgmres_device with host right-hand sides / solutions (column r at
// B + r * ldb): uploaded into one device buffer per call.
int Tree::block_gmres_host(double* B, int nrhs, size_t ldb, int maxit, double gtol, int* iters, double* relres) {
  if (!factorized_) return fail(-4, "gmres called before factorize");
  if (nrhs < 1 || ldb < (size_t)st_.n) return fail(-1, "block gmres: nrhs >= 1, ldb >= n");
  const size_t n = st_.n;
  double* d = nullptr;
  if (check_cuda(cudaMalloc(&d, sizeof(double) * n * nrhs), "malloc block right-hand sides")) return -11;
  for (int r = 0; r < nrhs; ++r)
    cudaMemcpyAsync(d + n * r, B + ldb * r, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  int rc = block_fgmres_device(d, nrhs, n, maxit, gtol, iters, relres);
  if (!rc) {
    for (int r = 0; r < nrhs; ++r)
      cudaMemcpyAsync(B + ldb * r, d + n * r, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
    rc = check_cuda(cudaStreamSynchronize(stream_), "block gmres download");
  }
  cudaFree(d);
  return rc;
}

int Tree::ensure_krylov(size_t doubles) {
  if (doubles <= krylov_doubles_) return 0;
  cudaFree(d_krylov_);
  d_krylov_ = nullptr;
  krylov_doubles_ = 0;
  if (check_cuda(cudaMalloc(&d_krylov_, sizeof(double) * doubles), "malloc Krylov workspace")) return -11;
  krylov_doubles_ = doubles;
  return 0;
}

int Tree::gmres_host(double* b, int maxit, double gtol, int* iters, double* relres, double* hist, int hist_cap) {
  const int n = st_.n;
  if (!factorized_) return fail(-4, "gmres called before factorize");
  double* d = nullptr;
  if (check_cuda(cudaMalloc(&d, sizeof(double) * n), "malloc")) return -10;
  cudaMemcpyAsync(d, b, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  int rc = gmres_device(d, maxit, gtol, iters, relres, hist, hist_cap);
  if (!rc) {
    cudaMemcpyAsync(b, d, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
    rc = check_cuda(cudaStreamSynchronize(stream_), "gmres copy-out");
  }
  cudaFree(d);
  return rc;
}

double* Tree::elem(double* p, size_t off) const {
  return fp32_ ? reinterpret_cast<double*>(reinterpret_cast<float*>(p) + off) : p + off;
}

// n elements of a factor array at element offset off, widened to double
void Tree::read_elems(const double* p, size_t off, size_t n, double* out) const {
  if (!fp32_) {
    cudaMemcpy(out, p + off, sizeof(double) * n, cudaMemcpyDeviceToHost);
    return;
  }
  std::vector<float> f(n);
  cudaMemcpy(f.data(), reinterpret_cast<const float*>(p) + off, sizeof(float) * n, cudaMemcpyDeviceToHost);
  for (size_t i = 0; i < n; ++i) out[i] = f[i];
}

int Tree::get_block(int n1, int n2, double* out, int* rows, int* cols, int* ld) const {
  const int e = st_.find_edge(n1, n2);
  if (e < 0 || e >= (int)ptr_.size() || !ptr_[e]) return -1;
  *rows = rows_[e];
  *cols = cols_[e];
  *ld = ld_[e];
  if (out) read_elems(ptr_[e], 0, (size_t)ld_[e] * cols_[e], out);
  return 0;
}

// which: 0 = block factors of an interior's diagonal QR (32 x n), 1 = scaling
// block factors (32 x n), 2 = sparsification reflectors V (n x rank), 3 = their
// block factors (32 x rank).
int Tree::get_factor(int order, int which, double* out, int* shape) const {
  if (!factorized_ || order < 0 || order >= (int)size_.size()) return -4;
  const double* p = nullptr;
  int r = 0, c = 0, ld = 0;
  const int n = size_org_[order];
  switch (which) {
    case 0: p = T_[order]; r = ld = dev_nb(); c = n; break;
    case 1: p = Ts_[order]; r = ld = dev_nb(); c = n; break;
    case 2: p = Qsp_[order]; r = ld = n; c = size_[order]; break;
    case 3: p = Tsp_[order]; r = ld = dev_nb(); c = size_[order]; break;
    default: return -1;
  }
  if (!p) return -1;
  shape[0] = r;
  shape[1] = c;
  shape[2] = ld;
  if (out)
    for (int j = 0; j < c; ++j) read_elems(p, (size_t)j * ld, r, out + (size_t)j * r);
  return 0;
}

}  // namespace spq
