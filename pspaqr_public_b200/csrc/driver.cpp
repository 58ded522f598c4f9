// driver.cpp -- the spaQR command-line driver (pspaQR.cpp:16-290) over the
// GPU library: same options and report lines, one B200 instead of MPI ranks.
//
//   spaqr -m A.mtx [-l levels] [-n cn -d cd] [-t tol] [--skip s] [--order o]
//         [--scale 0|1] [-i iterations] [--res tol] [--n_threads k] [--verb v]
//         [--log 0|1] [--hsl 0|1]
//
// The matrix is read from a Matrix Market coordinate file (real, general or
// symmetric), columns are scaled to norm 10 (pspaQR.cpp:133-146), the tree is
// partitioned on the tensor grid cn^cd, factorized, applied once to the
// reference's random right-hand side (seed 2021) and used as the
// preconditioner of GMRES.  --coordinates files, --rhs, --hsl, --log and
// rectangular matrices are not supported by this build (--hsl and --log are
// accepted and ignored like the library setters).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "spaqr_b200.h"

namespace {

struct Csc {
  int rows = 0, cols = 0;
  std::vector<int> colptr, rowidx;
  std::vector<double> vals;
};

// Matrix Market coordinate real (general or symmetric) -> 0-based CSC with
// sorted rows and duplicates summed.
bool read_mm(const std::string& path, Csc& A, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::string line;
  if (!std::getline(f, line) || line.rfind("%%MatrixMarket", 0) != 0) {
    err = "not a Matrix Market file";
    return false;
  }
  std::string lower = line;
  for (auto& c : lower) c = (char)std::tolower((unsigned char)c);
  if (lower.find("coordinate") == std::string::npos || lower.find("complex") != std::string::npos) {
    err = "only real coordinate matrices are supported";
    return false;
  }
  const bool sym = lower.find("symmetric") != std::string::npos;
  const bool pattern = lower.find("pattern") != std::string::npos;
  while (std::getline(f, line))
    if (!line.empty() && line[0] != '%') break;
  long nnz = 0;
  {
    std::istringstream s(line);
    s >> A.rows >> A.cols >> nnz;
  }
  std::vector<int> r, c;
  std::vector<double> v;
  r.reserve(sym ? 2 * nnz : nnz);
  for (long k = 0; k < nnz; ++k) {
    int i, j;
    double x = 1.0;
    if (!(f >> i >> j)) {
      err = "truncated entries";
      return false;
    }
    if (!pattern) f >> x;
    r.push_back(i - 1);
    c.push_back(j - 1);
    v.push_back(x);
    if (sym && i != j) {
      r.push_back(j - 1);
      c.push_back(i - 1);
      v.push_back(x);
    }
  }
  std::vector<std::vector<std::pair<int, double>>> col(A.cols);
  for (size_t k = 0; k < r.size(); ++k) col[c[k]].push_back({r[k], v[k]});
  A.colptr.assign(A.cols + 1, 0);
  for (int j = 0; j < A.cols; ++j) {
    auto& e = col[j];
    std::sort(e.begin(), e.end());
    for (size_t k = 0; k < e.size(); ++k) {
      if (k && e[k].first == e[k - 1].first) {
        A.vals.back() += e[k].second;
        continue;
      }
      A.rowidx.push_back(e[k].first);
      A.vals.push_back(e[k].second);
    }
    A.colptr[j + 1] = (int)A.rowidx.size();
  }
  return true;
}

double norm2(const std::vector<double>& x) {
  double s = 0;
  for (double v : x) s += v * v;
  return std::sqrt(s);
}

bool arg(int& i, int argc, char** argv, const char* s, const char* l, std::string& out) {
  const char* a = argv[i];
  if ((s && std::strcmp(a, s) == 0) || (l && std::strcmp(a, l) == 0)) {
    if (i + 1 >= argc) return false;
    out = argv[++i];
    return true;
  }
  if (l) {
    const size_t n = std::strlen(l);
    if (std::strncmp(a, l, n) == 0 && a[n] == '=') {
      out = a + n + 1;
      return true;
    }
  }
  return false;
}

int check(int rc, spq_tree* t, const char* what) {
  if (rc) std::fprintf(stderr, "%s failed (status %d): %s\n", what, rc, t ? spq_last_error(t) : "");
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  std::string matrix, v;
  int nlevels = -1, cn = -1, cd = -1, skip = 0, scale = 1, iterations = 300, nthreads = 1, verb = 0, hsl = 0, tlog = 0;
  double tol = 1e-1, res = 1e-12;
  float order = 1.0f;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--help") == 0) {
      std::printf(
          "spaQR (B200): Sparsified QR for sparse matrices\n"
          "  -m, --matrix FILE        matrix in Matrix Market format (mandatory)\n"
          "  -l, --lvl N              number of levels (default ceil(log2(ncols/64)))\n"
          "  -n, --coordinates_n N    tensor grid N^d geometric partition (with -d)\n"
          "  -d, --coordinates_d D\n"
          "  -t, --tol T              sparsification tolerance (default 1e-1)\n"
          "      --skip S             levels without sparsification (default 0)\n"
          "      --order O            accepted (order 1 scheme)\n"
          "      --scale 0|1          scaling (default 1)\n"
          "  -i, --iterations N       GMRES iterations (default 300)\n"
          "      --res R              GMRES relative residual (default 1e-12)\n"
          "      --n_threads N        accepted (one GPU)\n"
          "      --verb V             verbose printing\n"
          "      --hsl, --log         accepted and ignored\n");
      return 0;
    }
    if (arg(i, argc, argv, "-m", "--matrix", v)) matrix = v;
    else if (arg(i, argc, argv, "-l", "--lvl", v)) nlevels = std::atoi(v.c_str());
    else if (arg(i, argc, argv, "-n", "--coordinates_n", v)) cn = std::atoi(v.c_str());
    else if (arg(i, argc, argv, "-d", "--coordinates_d", v)) cd = std::atoi(v.c_str());
    else if (arg(i, argc, argv, "-t", "--tol", v)) tol = std::atof(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--skip", v)) skip = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--order", v)) order = (float)std::atof(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--scale", v)) scale = std::atoi(v.c_str());
    else if (arg(i, argc, argv, "-i", "--iterations", v)) iterations = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--res", v)) res = std::atof(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--n_threads", v)) nthreads = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--verb", v)) verb = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--hsl", v)) hsl = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--log", v)) tlog = std::atoi(v.c_str());
    else if (arg(i, argc, argv, nullptr, "--coordinates", v) || arg(i, argc, argv, nullptr, "--rhs", v)) {
      std::fprintf(stderr, "%s is not supported by this build\n", argv[i - 1]);
      return 1;
    } else {
      std::fprintf(stderr, "unknown option %s (see --help)\n", argv[i]);
      return 1;
    }
  }
  if (matrix.empty()) {
    std::printf("--matrix is mandatory\n");
    return 0;
  }
  if ((cn == -1) != (cd == -1)) {
    std::printf("cn and cd should be both provided, or none should be provided\n");
    return 1;
  }
  if (cn < 0) {
    std::fprintf(stderr, "only the tensor-grid geometric partition (-n, -d) is supported by this build\n");
    return 1;
  }
  Csc A;
  std::string err;
  if (!read_mm(matrix, A, err)) {
    std::fprintf(stderr, "reading %s: %s\n", matrix.c_str(), err.c_str());
    return 1;
  }
  if (A.rows != A.cols) {
    std::fprintf(stderr, "only square matrices are supported by this build\n");
    return 1;
  }
  std::printf("Matrix %s with %d rows,  %d columns loaded\n", matrix.c_str(), A.rows, A.cols);
  if (nlevels < 0) {
    nlevels = (int)std::ceil(std::log2((double)(A.cols / 64)));
    std::printf("--Levels not provided\n Levels set to ceil(log2(ncols/64)) =  %d\n", nlevels);
  }
  // column scaling to norm 10 (pspaQR.cpp:133-146)
  std::vector<double> vals = A.vals;
  if (spq_scale_columns(A.cols, A.colptr.data(), vals.data())) return 1;
  if (tol == 0) skip = nlevels - 1;
  if (std::pow((double)cn, cd) != A.cols) {
    std::printf("Error: cn and cd where both provided, but cn^cd != N where A is NxN\n");
    return 1;
  }
  std::printf("Tensor coordinate matrix of size %d^%d built\n", cn, cd);

  spq_tree* t = nullptr;
  if (check(spq_create(nlevels, skip, &t), nullptr, "create")) return 1;
  spq_set_scale(t, scale);
  spq_set_tol(t, tol);
  spq_set_order(t, order);
  spq_set_hsl(t, hsl);
  spq_set_nthreads(t, nthreads);
  spq_set_verbose(t, verb);
  spq_set_ttor_log(t, tlog);
  spq_set_square(t, 1);
  if (check(spq_set_coords_tensor(t, cn, cd), t, "coordinates") ||
      check(spq_partition(t, A.rows, A.cols, A.colptr.data(), A.rowidx.data(), vals.data()), t, "partition") ||
      check(spq_assemble(t), t, "assemble"))
    return 1;
  const int ferr = check(spq_factorize(t), t, "factorize");
  double times[5] = {0, 0, 0, 0, 0};
  spq_times(t, times);
  std::printf("Time to partition: %g\nTime to assemble: %g\nTime to factorize:  %g\n", times[0], times[1], times[2]);
  auto spmv_host = [&](const std::vector<double>& x) {  // y = A_scaled x, original order
    std::vector<double> y(A.rows, 0.0);
    for (int j = 0; j < A.cols; ++j)
      for (int k = A.colptr[j]; k < A.colptr[j + 1]; ++k) y[A.rowidx[k]] += vals[k] * x[j];
    return y;
  };
  if (!ferr) {
    std::vector<double> b(A.rows), x(A.cols, 0.0);
    spq_random_reference(A.rows, 2021, b.data());
    if (check(spq_solve_global(t, b.data(), x.data()), t, "solve")) return 1;
    spq_times(t, times);
    std::vector<double> r = spmv_host(x);
    for (int i = 0; i < A.rows; ++i) r[i] -= b[i];
    std::printf("<<<<tsolv=%g\nOne-time solve (Random b):\n<<<<|(Ax-b)|/|b| : %e\n", times[3], norm2(r) / norm2(b));
    std::vector<double> xl(spq_n(t));
    spq_random_reference((int)xl.size(), 2021, xl.data());
    int iters = 0;
    double relres = 0;
    if (check(spq_gmres(t, xl.data(), iterations, res, &iters, &relres, nullptr, 0), t, "gmres")) return 1;
    spq_times(t, times);
    std::printf("GMRES: #iterations: %d, residual |Ax-b|/|b|: %g\n  GMRES: %g s.\n<<<<GMRES=%d\n", iters, relres,
                times[4], iters);
  }
  spq_destroy(t);
  return ferr ? 1 : 0;
}
