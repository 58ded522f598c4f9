// capi_learned.cpp -- extern "C" entry points of the learned-rank path: the
// rank model of a tree, the logged training pairs, and the MLP's training
// and evaluation on the GPU (learned.cu kernels).  No reference counterpart.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/spaqr_b200.h"
#include "capi_internal.hpp"
#include "engine.hpp"
#include "learned.hpp"

namespace {

thread_local std::string g_mlp_err;

// device buffers released on scope exit
struct DevBuf {
  std::vector<void*> ptrs;
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~DevBuf() {
    for (void* p : ptrs) cudaFree(p);
  }
};

int cuda_fail(cudaError_t e, const char* where) {
  g_mlp_err = std::string(where) + ": " + cudaGetErrorString(e);
  return -10;
}

}  // namespace

extern "C" {

int spq_rank_model_size(int* nparams, int* nfeatures) {
  if (!nparams || !nfeatures) return -1;
  *nparams = spq::kMlpParams;
  *nfeatures = spq::kRankFeatures;
  return 0;
}

int spq_set_rank_model(spq_tree* h, const float* params, const float* mean, const float* stdev, int oversample) {
  if (!h) return -1;
  const int rc = h->t->set_rank_model(params, mean, stdev, oversample);
  if (rc) h->err = h->t->error;
  return rc;
}

int spq_set_rank_margin(spq_tree* h, float margin) {
  if (!h || !(margin >= 0.0f && margin <= 1.0f)) return -1;
  h->t->rank_margin = margin;
  return 0;
}

int spq_set_sketch_tuning(spq_tree* h, double sketch_tol, int smem) {
  if (!h || !(sketch_tol > 0 && sketch_tol <= 1)) return -1;
  h->t->sketch_tol = sketch_tol;
  h->t->sketch_smem = smem != 0;
  return 0;
}

int spq_learned_counts(spq_tree* h, long long* out) {
  if (!h || !out) return -1;
  h->t->learned_counts(out, out + 1, out + 2);
  return 0;
}

int spq_set_rank_log(spq_tree* h, int on) {
  if (!h) return -1;
  h->t->set_rank_log(on != 0);
  return 0;
}

int spq_rank_log_count(spq_tree* h) { return h ? (int)h->t->log_ranks().size() : -1; }

int spq_rank_log(spq_tree* h, float* features, int* ranks, int* kmin, int* levels) {
  if (!h || !features || !ranks || !kmin || !levels) return -1;
  const auto& f = h->t->log_features();
  std::copy(f.begin(), f.end(), features);
  std::copy(h->t->log_ranks().begin(), h->t->log_ranks().end(), ranks);
  std::copy(h->t->log_kmin().begin(), h->t->log_kmin().end(), kmin);
  std::copy(h->t->log_levels().begin(), h->t->log_levels().end(), levels);
  return 0;
}

int spq_rank_log_clear(spq_tree* h) {
  if (!h) return -1;
  h->t->clear_rank_log();
  return 0;
}

const char* spq_mlp_last_error(void) { return g_mlp_err.c_str(); }

int spq_mlp_loss_grad(const float* params, const float* X, const float* y, int n, float* loss, float* grad) {
  if (!params || !X || !y || n <= 0 || !loss || !grad) return -1;
  const int F = spq::kRankFeatures, P = spq::kMlpParams;
  DevBuf b;
  float* dP = b.get<float>(P);
  float* dX = b.get<float>((size_t)n * F);
  float* dy = b.get<float>(n);
  float* dG = b.get<float>(P);
  float* dl = b.get<float>(1);
  float* work = b.get<float>(spq::mlp_work_floats(n));
  if (!dP || !dX || !dy || !dG || !dl || !work) return cuda_fail(cudaErrorMemoryAllocation, "mlp buffers");
  cudaError_t e;
  if ((e = cudaMemcpy(dP, params, sizeof(float) * P, cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(dX, X, sizeof(float) * n * F, cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice)) ||
      (e = spq::mlp_loss_grad(dP, dX, dy, n, dl, dG, work, nullptr)) ||
      (e = cudaMemcpy(grad, dG, sizeof(float) * P, cudaMemcpyDeviceToHost)) ||
      (e = cudaMemcpy(loss, dl, sizeof(float), cudaMemcpyDeviceToHost)))
    return cuda_fail(e, "mlp loss/gradient");
  return 0;
}

int spq_mlp_predict(const float* params, const float* X, int n, float* out) {
  if (!params || !X || n < 0 || !out) return -1;
  if (n == 0) return 0;
  const int F = spq::kRankFeatures, P = spq::kMlpParams;
  DevBuf b;
  float* dP = b.get<float>(P);
  float* dX = b.get<float>((size_t)n * F);
  float* dO = b.get<float>(n);
  if (!dP || !dX || !dO) return cuda_fail(cudaErrorMemoryAllocation, "mlp buffers");
  cudaError_t e;
  if ((e = cudaMemcpy(dP, params, sizeof(float) * P, cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(dX, X, sizeof(float) * n * F, cudaMemcpyHostToDevice)) ||
      (e = spq::mlp_predict(dP, dX, n, dO, nullptr)) ||
      (e = cudaMemcpy(out, dO, sizeof(float) * n, cudaMemcpyDeviceToHost)))
    return cuda_fail(e, "mlp predict");
  return 0;
}

// Adam on mini-batches of a seeded per-epoch shuffle; loss_hist[epoch] is the
// sample-weighted mean of the batch losses of that epoch (may be null).
int spq_mlp_train(float* params, const float* X, const float* y, int n, int epochs, int batch, float lr,
                  unsigned long long seed, float* loss_hist) {
  if (!params || !X || !y || n <= 0 || epochs < 0 || batch <= 0 || !(lr > 0)) return -1;
  const int F = spq::kRankFeatures, P = spq::kMlpParams;
  batch = std::min(batch, n);
  const int nbatch = (n + batch - 1) / batch;
  DevBuf b;
  float* dP = b.get<float>(P);
  float* dG = b.get<float>(P);
  float* m1 = b.get<float>(P);
  float* m2 = b.get<float>(P);
  float* dX = b.get<float>((size_t)n * F);
  float* dy = b.get<float>(n);
  float* dl = b.get<float>(nbatch);
  float* work = b.get<float>(spq::mlp_work_floats(batch));
  if (!dP || !dG || !m1 || !m2 || !dX || !dy || !dl || !work)
    return cuda_fail(cudaErrorMemoryAllocation, "mlp buffers");
  cudaError_t e;
  if ((e = cudaMemcpy(dP, params, sizeof(float) * P, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(m1, 0, sizeof(float) * P)) || (e = cudaMemset(m2, 0, sizeof(float) * P)))
    return cuda_fail(e, "mlp setup");
  std::mt19937_64 rng(seed);
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::vector<float> Xp((size_t)n * F), yp(n), bl(nbatch);
  int step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    for (int i = 0; i < n; ++i) {
      std::copy(X + (size_t)perm[i] * F, X + (size_t)perm[i] * F + F, Xp.begin() + (size_t)i * F);
      yp[i] = y[perm[i]];
    }
    if ((e = cudaMemcpy(dX, Xp.data(), sizeof(float) * Xp.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(dy, yp.data(), sizeof(float) * n, cudaMemcpyHostToDevice)))
      return cuda_fail(e, "mlp data upload");
    for (int k = 0; k < nbatch; ++k) {
      const int s0 = k * batch, nb = std::min(batch, n - s0);
      if ((e = spq::mlp_loss_grad(dP, dX + (size_t)s0 * F, dy + s0, nb, dl + k, dG, work, nullptr)) ||
          (e = spq::mlp_adam(dP, dG, m1, m2, lr, ++step, nullptr)))
        return cuda_fail(e, "mlp step");
    }
    if (loss_hist) {
      if ((e = cudaMemcpy(bl.data(), dl, sizeof(float) * nbatch, cudaMemcpyDeviceToHost)))
        return cuda_fail(e, "mlp loss");
      double s = 0.0;
      for (int k = 0; k < nbatch; ++k) s += (double)bl[k] * std::min(batch, n - k * batch);
      loss_hist[ep] = (float)(s / n);
    }
  }
  if ((e = cudaMemcpy(params, dP, sizeof(float) * P, cudaMemcpyDeviceToHost))) return cuda_fail(e, "mlp download");
  return 0;
}

}  // extern "C"
