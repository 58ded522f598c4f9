// capi.cpp -- extern "C" boundary (include/spaqr_b200.h) over spq::Tree.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/spaqr_b200.h"
#include "capi_internal.hpp"
#include "engine.hpp"
#include "kernels.hpp"
#include "noalloc.hpp"
#include "shard.hpp"


namespace {
int done(spq_tree* h, int rc) {
  if (rc != 0) h->err = h->t->error;
  return rc;
}
thread_local std::string g_err;
}  // namespace

extern "C" {

int spq_create(int nlevels, int skip, spq_tree** out) {
  if (!out) return -1;
  *out = nullptr;
  if (nlevels < 2 || skip < 0) return -1;
  spq_tree* h = new spq_tree;
  h->t = new spq::Tree(nlevels, skip);
  *out = h;
  return 0;
}

int spq_destroy(spq_tree* h) {
  if (!h) return -1;
  delete h->t;
  delete h;
  return 0;
}

#define SPQ_SETTER(name, type, field) \
  int name(spq_tree* h, type v) {     \
    if (!h) return -1;                \
    h->t->field = v;                  \
    return 0;                         \
  }
SPQ_SETTER(spq_set_tol, double, tol)
SPQ_SETTER(spq_set_skip, int, skip)
SPQ_SETTER(spq_set_scale, int, scale)
SPQ_SETTER(spq_set_order, float, order)
SPQ_SETTER(spq_set_hsl, int, hsl)
SPQ_SETTER(spq_set_nthreads, int, nthreads)
SPQ_SETTER(spq_set_verbose, int, verbose)
SPQ_SETTER(spq_set_ttor_log, int, ttor_log)
#undef SPQ_SETTER

int spq_set_pivot_rtol(spq_tree* h, double r) {
  if (!h || r < 0 || r >= 1) return -1;
  h->t->pivot_rtol = r;
  return 0;
}

int spq_set_rrqr_work(spq_tree* h, double elems, double fill) {
  if (!h || !(elems >= 1024) || !(fill > 0 && fill <= 64)) return -1;
  h->t->rrqr_work = elems;
  h->t->rrqr_fill = fill;
  return 0;
}

int spq_set_precision(spq_tree* h, int bits) {
  if (!h || (bits != 32 && bits != 64)) return -1;
  h->t->precision = bits;
  return 0;
}

int spq_set_plan_cache(spq_tree* h, int on) {
  if (!h || on < 0 || on > 1) return -1;
  h->t->plan_cache = on != 0;
  return 0;
}
long long spq_plan_hits(spq_tree* h) { return h ? h->t->plan_hits() : -1; }

int spq_set_spin_limit(spq_tree* h, long long cycles) {
  if (!h || cycles < 0) return -1;
  h->t->spin_limit = cycles;
  return 0;
}

int spq_set_checks(spq_tree* h, int on) {
  if (!h || on < 0 || on > 1) return -1;
  h->t->check_descriptors = on != 0;
  return 0;
}

int spq_debug_corrupt_descriptor(spq_tree* h) {
  if (!h) return -1;
  h->t->corrupt_next_descriptor = true;
  return 0;
}

int spq_debug_tc_probe(const float* C, const float* V, const float* W2, int m, int flags, float* out1, float* out2) {
  if (!C || !V || !W2 || !out1 || !out2 || m < 1 || m > 64 || flags < 0 || flags > 15) return -1;
  float* d = nullptr;
  int* st = nullptr;
  const size_t nc = (size_t)m * 64, nv = (size_t)m * 32, nw = 32 * 64, n1 = 128 * 32, n2 = 128 * 64;
  if (cudaMalloc(&d, sizeof(float) * (nc + nv + nw + n1 + n2)) != cudaSuccess) return -11;
  if (cudaMalloc(&st, sizeof(int)) != cudaSuccess) {
    cudaFree(d);
    return -11;
  }
  float *dC = d, *dV = dC + nc, *dW = dV + nv, *d1 = dW + nw, *d2 = d1 + n1;
  cudaMemset(st, 0, sizeof(int));
  cudaMemcpy(dC, C, sizeof(float) * nc, cudaMemcpyHostToDevice);
  cudaMemcpy(dV, V, sizeof(float) * nv, cudaMemcpyHostToDevice);
  cudaMemcpy(dW, W2, sizeof(float) * nw, cudaMemcpyHostToDevice);
  cudaError_t e = spq::launch_tc_probe(dC, dV, dW, m, flags, d1, d2, st, nullptr);
  if (!e) e = cudaDeviceSynchronize();
  int status = 0;
  if (!e) e = cudaMemcpy(out1, d1, sizeof(float) * n1, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(out2, d2, sizeof(float) * n2, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(st);
  return e ? -10 : (status ? -12 : 0);
}

int spq_set_tensor_cores(spq_tree* h, int mode) {
  if (!h || mode < 0 || mode > 2) return -1;
  h->t->tensor_cores = mode;
  return 0;
}

int spq_tune_table(spq_tree* h, float* out) {
  if (!h || !out) return -1;
  std::vector<float> v;
  h->t->tune_table(v);
  std::copy(v.begin(), v.end(), out);
  return 0;
}

int spq_set_krylov(spq_tree* h, int method) {
  if (!h || method < -1 || method > 1) return -1;
  h->t->krylov = method;
  return 0;
}

int spq_set_square(spq_tree* h, int s) {
  if (!h) return -1;
  if (!s) {
    h->err = "rectangular (least-squares) systems are not supported by this build";
    return -2;
  }
  h->t->square = 1;
  return 0;
}

int spq_set_coords(spq_tree* h, int dim, int n, const double* X) {
  if (!h) return -1;
  return done(h, h->t->set_coords(dim, n, X));
}
int spq_set_coords_tensor(spq_tree* h, int n, int d) {
  if (!h) return -1;
  return done(h, h->t->set_coords_tensor(n, d));
}
int spq_partition(spq_tree* h, int nrows, int ncols, const int* colptr, const int* rowidx, const double* vals) {
  if (!h) return -1;
  if (h->t->hsl) {
    h->err = "bipartite matching (HSL MC64) is not part of this build";
    return -2;
  }
  return done(h, h->t->partition(nrows, ncols, colptr, rowidx, vals));
}
int spq_assemble(spq_tree* h) { return h ? done(h, h->t->assemble()) : -1; }
int spq_factorize(spq_tree* h) { return h ? done(h, h->t->factorize()) : -1; }
int spq_solve_inplace(spq_tree* h, double* x) { return (h && x) ? done(h, h->t->solve_host(x)) : -1; }
int spq_solve_inplace_device(spq_tree* h, double* x) {
  if (!h || !x) return -1;
  h->t->clear_status();
  return done(h, h->t->solve_device(x));
}
int spq_solve_global(spq_tree* h, const double* b, double* x) {
  return (h && b && x) ? done(h, h->t->solve_global(b, x)) : -1;
}
int spq_spmv(spq_tree* h, const double* x, double* y) { return (h && x && y) ? done(h, h->t->spmv_host(x, y)) : -1; }
int spq_factor_backward_error(spq_tree* h, int nprobe, const double* U, unsigned long long seed, double* eta) {
  return h ? done(h, h->t->backward_error(nprobe, U, seed, eta)) : -1;
}
int spq_gmres(spq_tree* h, double* b, int maxit, double tol, int* iters, double* relres, double* hist, int hist_cap) {
  if (!h || !b || !iters || !relres) return -1;
  return done(h, h->t->gmres_host(b, maxit, tol, iters, relres, hist, hist_cap));
}
int spq_gmres_device(spq_tree* h, double* b, int maxit, double tol, int* iters, double* relres, double* hist,
                     int hist_cap) {
  if (!h || !b || !iters || !relres) return -1;
  return done(h, h->t->gmres_device(b, maxit, tol, iters, relres, hist, hist_cap));
}
int spq_gmres_device_noalloc(spq_tree* h, double* b, int maxit, double tol, int* iters, double* relres) {
  if (!h || !b || !iters || !relres) return -1;
  double* ws = nullptr;
  if (cudaError_t e = spq::noalloc_workspace(&ws)) {
    h->t->error = std::string("allocation-free GMRES workspace: ") + cudaGetErrorString(e);
    return -10;
  }
  return done(h, h->t->gmres_device_fixed(b, maxit, tol, iters, relres, ws, spq::kNoAllocDoubles));
}
int spq_solve_block_device(spq_tree* h, double* X, int nrhs, long long ldx) {
  if (!h || !X || nrhs < 1 || ldx < 1) return -1;
  return done(h, h->t->solve_block_device(X, nrhs, (size_t)ldx));
}
int spq_gmres_block(spq_tree* h, double* B, int nrhs, long long ldb, int maxit, double tol, int* iters,
                    double* relres) {
  if (!h || !B || !iters || !relres || nrhs < 1 || ldb < 1) return -1;
  return done(h, h->t->block_gmres_host(B, nrhs, (size_t)ldb, maxit, tol, iters, relres));
}
int spq_gmres_block_device(spq_tree* h, double* B, int nrhs, long long ldb, int maxit, double tol, int* iters,
                           double* relres) {
  if (!h || !B || !iters || !relres || nrhs < 1 || ldb < 1) return -1;
  return done(h, h->t->block_fgmres_device(B, nrhs, (size_t)ldb, maxit, tol, iters, relres));
}
int spq_distribute_x(spq_tree* h, const double* x, double* xl) {
  if (!h || !x || !xl) return -1;
  const auto& s = h->t->structure();
  if (s.rperm.empty()) return -4;
  for (int i = 0; i < s.n; ++i) xl[i] = x[s.rperm[i]];
  return 0;
}
int spq_extract_x(spq_tree* h, const double* xl, double* x) {
  if (!h || !x || !xl) return -1;
  const auto& s = h->t->structure();
  if (s.cperm.empty()) return -4;
  for (int i = 0; i < s.n; ++i) x[s.cperm[i]] = xl[i];
  return 0;
}
int spq_n(spq_tree* h) { return h ? h->t->n() : -1; }
int spq_set_stream(spq_tree* h, void* stream) {
  return h ? done(h, h->t->set_stream(static_cast<cudaStream_t>(stream))) : -1;
}

int spq_scale_columns(int ncols, const int* colptr, double* vals) {
  if (ncols < 0 || !colptr || !vals) return -1;
  for (int j = 0; j < ncols; ++j) {
    double s = 0.0;
    for (int k = colptr[j]; k < colptr[j + 1]; ++k) s += vals[k] * vals[k];
    const double d = 1.0 / std::sqrt(s);
    for (int k = colptr[j]; k < colptr[j + 1]; ++k) vals[k] = (vals[k] * d) * 10.0;
  }
  return 0;
}

int spq_random_reference(int n, int seed, double* out) {
  if (n < 0 || !out) return -1;
  std::mt19937 rng;
  rng.seed(seed);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (int i = 0; i < n; ++i) out[i] = dist(rng);
  return 0;
}

int spq_get_perm(spq_tree* h, int* cperm) {
  if (!h || !cperm) return -1;
  const auto& s = h->t->structure();
  if (s.cperm.empty()) return -4;
  std::memcpy(cperm, s.cperm.data(), sizeof(int) * s.n);
  return 0;
}
int spq_num_clusters(spq_tree* h) { return h ? (int)h->t->structure().clusters.size() : -1; }
int spq_num_levels(spq_tree* h) { return h ? h->t->structure().nlevels : -1; }
int spq_cluster_info(spq_tree* h, int order, int* info) {
  if (!h || !info) return -1;
  const auto& s = h->t->structure();
  if (order < 0 || order >= (int)s.clusters.size()) return -1;
  const spq::Cluster& c = s.clusters[order];
  auto sz = h->t->cluster_sizes();
  auto so = h->t->cluster_sizes_org();
  const bool have = !sz.empty();
  info[0] = c.lvl;
  info[1] = c.merge_lvl;
  info[2] = have ? sz[order] : c.size0;
  info[3] = have ? sz[order] : c.size0;
  info[4] = c.parent;
  info[5] = c.cstart;
  info[6] = c.id.self.sep;
  info[7] = c.id.l.lvl;
  info[8] = c.id.l.sep;
  info[9] = c.id.r.lvl;
  info[10] = c.id.r.sep;
  info[11] = c.id.section;
  info[12] = have ? so[order] : c.size0;
  info[13] = c.sparsify ? 1 : 0;
  info[14] = c.child_end - c.child_begin;
  info[15] = c.interior ? 1 : 0;
  return 0;
}
int spq_level_range(spq_tree* h, int lvl, int* first, int* count) {
  if (!h || !first || !count) return -1;
  const auto& s = h->t->structure();
  if (lvl < 0 || lvl >= (int)s.levels.size()) return -1;
  *first = s.levels[lvl].first;
  *count = s.levels[lvl].count;
  return 0;
}
int spq_num_edges(spq_tree* h) { return h ? (int)h->t->structure().edges.size() : -1; }
int spq_find_edge(spq_tree* h, int n1, int n2) { return h ? h->t->structure().find_edge(n1, n2) : -1; }
int spq_get_block(spq_tree* h, int n1, int n2, double* out, int* shape) {
  if (!h || !shape) return -1;
  return h->t->get_block(n1, n2, out, shape, shape + 1, shape + 2);
}
int spq_get_factor(spq_tree* h, int order, int which, double* out, int* shape) {
  if (!h || !shape) return -1;
  return h->t->get_factor(order, which, out, shape);
}
int spq_times(spq_tree* h, double* times) {
  if (!h || !times) return -1;
  times[0] = h->t->t_partition;
  times[1] = h->t->t_assemble;
  times[2] = h->t->t_factorize;
  times[3] = h->t->t_solve;
  times[4] = h->t->t_gmres;
  return 0;
}
int spq_level_flops(spq_tree* h, double* flops) {
  if (!h || !flops) return -1;
  const auto& lt = h->t->level_timing();
  for (size_t l = 0; l < lt.size(); ++l)
    for (int k = 0; k < 6; ++k) flops[6 * l + k] = lt[l].flops[k];
  return 0;
}

int spq_level_times(spq_tree* h, float* ms) {
  if (!h || !ms) return -1;
  const auto& lt = h->t->level_timing();
  for (size_t l = 0; l < lt.size(); ++l) {
    float* m = ms + 8 * l;
    m[0] = lt[l].e1_ms;
    m[1] = lt[l].e2_ms;
    m[2] = lt[l].sqr_ms;
    m[3] = lt[l].sapp_ms;
    m[4] = lt[l].rrqr_ms;
    m[5] = lt[l].capp_ms;
    m[6] = lt[l].merge_ms;
    m[7] = lt[l].elim_ms + lt[l].scale_ms + lt[l].spars_ms + lt[l].merge_ms;
  }
  return 0;
}
double spq_factor_flops(spq_tree* h) { return h ? h->t->factor_flops() : -1.0; }
double spq_rrqr_bytes(spq_tree* h) { return h ? h->t->rrqr_bytes() : -1.0; }
double spq_pool_bytes(spq_tree* h) { return h ? (double)h->t->pool_bytes() : -1.0; }
long long spq_kernel_launches(void) { return spq::kernel_launches(); }
int spq_shard_plan(spq_tree* h, int nranks, int* cluster_owner, int* row_owner, int* nexchange) {
  if (!h || nranks < 1) return -1;
  const auto& s = h->t->structure();
  if (s.clusters.empty()) {
    h->err = "shard plan requested before partition";
    return -4;
  }
  spq::ShardPlan p;
  if (spq::build_shard_plan(s, nranks, p)) {
    h->err = "nranks must be a power of two no larger than the number of leaf parts";
    return -1;
  }
  if (cluster_owner) std::copy(p.cluster_owner.begin(), p.cluster_owner.end(), cluster_owner);
  if (row_owner) std::copy(p.row_owner.begin(), p.row_owner.end(), row_owner);
  if (nexchange)
    for (int l = 0; l < s.nlevels; ++l) nexchange[l] = (int)p.exchange[l].size();
  return 0;
}

int spq_shard_exchange(spq_tree* h, int nranks, int lvl, int* out) {
  if (!h || nranks < 1) return -1;
  const auto& s = h->t->structure();
  if (lvl < 0 || lvl >= s.nlevels) return -1;
  spq::ShardPlan p;
  if (spq::build_shard_plan(s, nranks, p)) return -1;
  int k = 0;
  for (const auto& x : p.exchange[lvl]) {
    out[k++] = x.kind;
    out[k++] = x.id;
    out[k++] = x.dst;
    out[k++] = x.from;
    out[k++] = x.to;
  }
  return 0;
}

int spq_get_edges(spq_tree* h, int* out) {
  if (!h || !out) return -1;
  const auto& s = h->t->structure();
  for (size_t e = 0; e < s.edges.size(); ++e) {
    out[3 * e] = s.edges[e].n1;
    out[3 * e + 1] = s.edges[e].n2;
    out[3 * e + 2] = s.edges[e].level;
  }
  return 0;
}

const char* spq_last_error(spq_tree* h) {
  if (!h) return "null handle";
  return h->err.c_str();
}
}
