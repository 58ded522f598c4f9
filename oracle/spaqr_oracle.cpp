// spaqr_oracle.cpp -- CPU ORACLE for the pspaQR factorize-and-solve path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness checker and the
// timed CPU baseline; the product (pspaqr_public_b200) never links, loads or
// calls it.  It restates, in plain sequential C++ on top of LAPACK/CBLAS
// (SciPy's bundled OpenBLAS, reached through its `scipy_`-prefixed exports),
// the square-matrix path of the reference ParTree:
//
//   partition  : partition.cpp:241-350 (bissect_geo, GeometricPartitionAtA),
//                partition.cpp:514-587 (getInterfacesUsingA), tree.cpp:48-57
//                (initPermutation), cluster.cpp:23-32 (merge_if),
//                ptree.cpp:495-701 (leaf clusters, hierarchy)
//   assemble   : ptree.cpp:703-864 (dense blocks via block2dense, dist2connxs)
//   factorize  : ptree.cpp:873-2154 (fill-in, geqrt/tsqrt/larfb/ssrfb,
//                scaling, RRQR sparsification, merge)
//   solve      : ptree.cpp:2160-2262, 2788-3210 (fwd Q^T sweep, bwd R^-1 sweep)
//   spmv       : ptree.cpp:3212-3262
//   gmres      : is.cpp:447-527 (left-preconditioned, unrestarted MGS-GMRES)
//
// Parity is UNPINNED: the reference ships no golden vectors and cannot be
// built in this environment (Eigen, MPI, TaskTorrent and LAPACKE headers are
// absent), so this restatement is pinned only by the structural counts quoted
// from a replica of the reference partition and by its own self-consistency.
//
// Deterministic schedule.  Where the reference leaves the order of two
// non-commuting updates to its task runtime (several interiors updating one
// target block; the order of the tsqrt transforms recorded in order_of_trans),
// this oracle fixes it to ascending interior order.  Tasks that touch disjoint
// data run in OpenMP parallel loops; the result is bitwise independent of the
// thread count when the BLAS runs single-threaded.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
int scipy_LAPACKE_dgeqrt(int, int, int, int, double*, int, double*, int);
int scipy_LAPACKE_dtpqrt(int, int, int, int, int, double*, int, double*, int, double*, int);
int scipy_LAPACKE_dtpmqrt(int, char, char, int, int, int, int, int, const double*, int, const double*, int,
                          double*, int, double*, int);
int scipy_LAPACKE_dlarfb(int, char, char, char, char, int, int, int, const double*, int, const double*, int,
                         double*, int);
int scipy_LAPACKE_dlarft(int, char, char, int, int, const double*, int, const double*, double*, int);
int scipy_LAPACKE_dgeqp3(int, int, int, double*, int, int*, double*);
int scipy_LAPACKE_dormqr(int, char, char, int, int, int, const double*, int, const double*, double*, int);
void scipy_cblas_dtrsm(int, int, int, int, int, int, int, double, const double*, int, double*, int);
void scipy_cblas_dtrsv(int, int, int, int, int, const double*, int, double*, int);
void scipy_openblas_set_num_threads(int);
}

namespace {
constexpr int kColMajor = 102;
constexpr int kLeft = 141, kRight = 142, kUpper = 121, kNoTrans = 111, kNonUnit = 131;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ----------------------------------------------------------------- ids
// cluster.h:37-135
struct SepID {
  int lvl = -1, sep = 0;
  SepID() = default;
  SepID(int l, int s) : lvl(l), sep(s) {}
  bool operator==(const SepID& o) const { return lvl == o.lvl && sep == o.sep; }
  bool operator!=(const SepID& o) const { return !(*this == o); }
  bool operator<(const SepID& o) const { return lvl < o.lvl || (lvl == o.lvl && sep < o.sep); }
};
struct ClusterID {
  SepID self, l, r;
  int part = 2, section = 0;
  bool operator==(const ClusterID& o) const {
    return self == o.self && l == o.l && r == o.r && part == o.part && section == o.section;
  }
  bool operator!=(const ClusterID& o) const { return !(*this == o); }
  bool operator<(const ClusterID& o) const {
    if (self != o.self) return self < o.self;
    if (l != o.l) return l < o.l;
    if (r != o.r) return r < o.r;
    if (section != o.section) return section < o.section;
    return part < o.part;
  }
};
SepID merge_sep(SepID s) { return SepID(s.lvl + 1, s.sep / 2); }
// cluster.cpp:23-32
ClusterID merge_if(const ClusterID& c, int lvl) {
  ClusterID o;
  o.self = c.self;
  o.l = c.l.lvl < lvl ? merge_sep(c.l) : c.l;
  o.r = c.r.lvl < lvl ? merge_sep(c.r) : c.r;
  o.section = lvl > 0 ? c.section / 2 : c.section;
  o.part = c.self.lvl == lvl ? 2 : c.part;
  return o;
}
// partition.cpp:63-100
SepID find_highest_common(SepID a, SepID b) {
  int l1 = a.lvl, l2 = b.lvl, s1 = a.sep, s2 = b.sep;
  while (l1 < l2) { l1++; s1 /= 2; }
  while (l2 < l1) { l2++; s2 /= 2; }
  while (s1 != s2) { l1++; l2++; s1 /= 2; s2 /= 2; }
  return SepID(l1, s1);
}
SepID find_lowest_common(SepID a, SepID b) { return a.lvl < b.lvl ? a : b; }

// ----------------------------------------------------------------- CSC
struct CSC {
  int nrows = 0, ncols = 0;
  std::vector<int> colptr, rowidx;
  std::vector<double> val;
};
CSC transpose(const CSC& A) {
  CSC T;
  T.nrows = A.ncols;
  T.ncols = A.nrows;
  T.colptr.assign(A.nrows + 1, 0);
  for (int k = 0; k < (int)A.rowidx.size(); ++k) T.colptr[A.rowidx[k] + 1]++;
  for (int i = 0; i < A.nrows; ++i) T.colptr[i + 1] += T.colptr[i];
  T.rowidx.resize(A.rowidx.size());
  T.val.resize(A.rowidx.size());
  std::vector<int> pos(T.colptr.begin(), T.colptr.end() - 1);
  for (int j = 0; j < A.ncols; ++j)
    for (int k = A.colptr[j]; k < A.colptr[j + 1]; ++k) {
      int p = pos[A.rowidx[k]]++;
      T.rowidx[p] = j;
      T.val[p] = A.val[k];
    }
  return T;
}
// Structural pattern of A^T A (sorted row indices per column, diagonal included).
CSC ata_pattern(const CSC& A) {
  CSC At = transpose(A);
  CSC P;
  P.nrows = P.ncols = A.ncols;
  P.colptr.assign(A.ncols + 1, 0);
  std::vector<int> mark(A.ncols, -1), tmp;
  for (int j = 0; j < A.ncols; ++j) {
    tmp.clear();
    for (int k = A.colptr[j]; k < A.colptr[j + 1]; ++k) {
      int r = A.rowidx[k];
      for (int q = At.colptr[r]; q < At.colptr[r + 1]; ++q) {
        int c = At.rowidx[q];
        if (mark[c] != j) { mark[c] = j; tmp.push_back(c); }
      }
    }
    std::sort(tmp.begin(), tmp.end());
    P.rowidx.insert(P.rowidx.end(), tmp.begin(), tmp.end());
    P.colptr[j + 1] = (int)P.rowidx.size();
  }
  P.val.assign(P.rowidx.size(), 1.0);
  return P;
}

// ----------------------------------------------------------------- dense
struct Mat {
  int r = 0, c = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int r_, int c_) : r(r_), c(c_), a((size_t)r_ * c_, 0.0) {}
  double* p() { return a.data(); }
  const double* p() const { return a.data(); }
  double& operator()(int i, int j) { return a[(size_t)j * r + i]; }
  double operator()(int i, int j) const { return a[(size_t)j * r + i]; }
  void zero() { std::fill(a.begin(), a.end(), 0.0); }
  // Eigen conservativeResize semantics: keep the top-left overlap, new entries 0
  void resize_keep(int nr, int nc) {
    Mat m(nr, nc);
    for (int j = 0; j < std::min(c, nc); ++j)
      for (int i = 0; i < std::min(r, nr); ++i) m(i, j) = (*this)(i, j);
    *this = std::move(m);
  }
  Mat top_rows(int k) const {
    Mat m(k, c);
    for (int j = 0; j < c; ++j)
      for (int i = 0; i < k; ++i) m(i, j) = (*this)(i, j);
    return m;
  }
  void set_top_rows(const Mat& t) {
    for (int j = 0; j < c; ++j)
      for (int i = 0; i < t.r; ++i) (*this)(i, j) = t(i, j);
  }
};

// util.cpp:414-498 larfb wrappers (LAPACKE path; side/trans as given)
void larfb(const Mat& V, const Mat& T, double* C, int m, int n, char side = 'L', char trans = 'T') {
  if (m == 0 || n == 0) return;
  int k = V.c;
  int ldv = (side == 'L') ? m : n;
  int info = scipy_LAPACKE_dlarfb(kColMajor, side, trans, 'F', 'C', m, n, k, V.p(), ldv, T.p(), k, C, m);
  if (info != 0) fprintf(stderr, "oracle: dlarfb info %d\n", info);
}

// ----------------------------------------------------------------- tree
struct Edge {
  int n1, n2;  // column cluster n1, row cluster n2: block A(rows n2, cols n1)
  Mat A;
  int interior_deps = 0;
};

struct Cluster {
  int cstart = 0, csize = 0, rstart = 0, rsize = 0;
  ClusterID id;
  int order = 0, merge_lvl = 0;
  bool eliminated = false;
  int rank = 0, csize_org = 0, rsize_org = 0;
  int parent = -1;
  std::vector<int> children;  // cluster orders sorted by id
  int rpos = 0, cpos = 0;
  std::set<int> d2;           // dist2connxs (cluster orders)
  std::vector<int> out;       // out edges (this cluster's column blocks), sorted by n2 order
  std::vector<int> in;        // in edges (this cluster's row blocks)
  int self_edge = -1;
  int col_interior_deps = 0;
  // factors
  Mat T;                       // geqrt T of interiors
  std::map<int, Mat> Tmap;     // tpqrt T per out-neighbour order (nb x cols)
  bool sparsified = false;
  Mat Qs, Ts;                  // scaling QR
  Mat Qsp, Tsp;                // sparsification reflectors (cols x rank) and T
  std::vector<double> tausp;
  std::vector<int> order_of_trans;
  std::vector<double> x;
  int lvl() const { return id.self.lvl; }
  int rows() const { return rsize; }
  int cols() const { return csize; }
  void set_size(int r, int c) { rsize = r; csize = c; rank = c; x.assign(r, 0.0); }
  void reset_size(int r, int c) { rsize = r; csize = c; rank = c; }
};

// Column-pivoted Householder QR of C (m x w, col-major), restating LAPACK
// dgeqp3's unblocked path dlaqp2 (pivot on the largest partial column norm,
// LAWN 176 norm downdating with recomputation when temp2 <= sqrt(eps)), stopped
// at the first i >= 1 with |R(i,i)|/|R(0,0)| < tol (util.cpp:830-851
// choose_rank).  Pivot: the first column whose partial norm is within
// pivot_rtol of the largest (pivot_rtol = 0 is LAPACK's idamax rule).
// Returns the rank; tau[0:rank] and V (below the diagonal of the first rank
// columns) as dgeqp3 leaves them.
int geqp3_trunc(double* C, int m, int w, double tol, double pivot_rtol, std::vector<double>& tau) {
  const int kmin = std::min(m, w);
  tau.assign(std::max(kmin, 1), 0.0);
  std::vector<double> vn1(w), vn2(w);
  auto col = [&](int j) { return C + (size_t)j * m; };
  for (int j = 0; j < w; ++j) {
    double s = 0;
    for (int r = 0; r < m; ++r) s += col(j)[r] * col(j)[r];
    vn1[j] = vn2[j] = std::sqrt(s);
  }
  const double tol3z = std::sqrt(1.1102230246251565e-16);
  double r00 = 0;
  for (int i = 0; i < kmin; ++i) {
    double mx = -1.0;
    for (int j = i; j < w; ++j) mx = std::max(mx, vn1[j]);
    const double thr = mx * (1.0 - pivot_rtol);
    int pvt = i;
    for (int j = i; j < w; ++j)
      if (vn1[j] >= thr) { pvt = j; break; }
    if (pvt != i) {
      for (int r = 0; r < m; ++r) std::swap(col(i)[r], col(pvt)[r]);
      vn1[pvt] = vn1[i];
      vn2[pvt] = vn2[i];
    }
    double* ci = col(i);
    double ss = 0;
    for (int r = i + 1; r < m; ++r) ss += ci[r] * ci[r];
    const double alpha = ci[i];
    double beta = alpha, t = 0.0, scal = 0.0;
    if (ss != 0.0) {
      beta = -std::copysign(std::hypot(alpha, std::sqrt(ss)), alpha);
      t = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    const double absb = std::fabs(beta);
    if (i == 0) r00 = absb;
    else if (!(absb / r00 >= tol)) return i;
    if (t != 0.0)
      for (int r = i + 1; r < m; ++r) ci[r] *= scal;
    ci[i] = beta;
    tau[i] = t;
    for (int j = i + 1; j < w; ++j) {
      double* cj = col(j);
      if (t != 0.0) {
        double d = cj[i];
        for (int r = i + 1; r < m; ++r) d += ci[r] * cj[r];
        d *= t;
        cj[i] -= d;
        for (int r = i + 1; r < m; ++r) cj[r] -= ci[r] * d;
      }
      if (vn1[j] != 0.0) {
        double temp = std::fabs(cj[i]) / vn1[j];
        temp = std::max(1.0 - temp * temp, 0.0);
        const double q = vn1[j] / vn2[j];
        if (temp * q * q <= tol3z) {
          double nn = 0;
          for (int r = i + 1; r < m; ++r) nn += cj[r] * cj[r];
          vn1[j] = vn2[j] = (i + 1 < m) ? std::sqrt(nn) : 0.0;
        } else {
          vn1[j] *= std::sqrt(temp);
        }
      }
    }
  }
  return kmin;
}

struct Timers {
  double partition = 0, assemble = 0, factorize = 0, solve = 0, gmres = 0;
  std::vector<double> lvl_fill, lvl_elim, lvl_scale, lvl_spars, lvl_merge;
};

struct Oracle {
  int nlevels, skip;
  double tol;
  int nthreads = 1;
  int pivot_mode = 1;          // 0: LAPACK dgeqp3 as the reference calls it; 1: restated dlaqp2 with tie rule
  double pivot_rtol = 1e-6;
  int n = 0;
  CSC A;      // scaled input matrix (original order)
  CSC App;    // permuted matrix (rows rperm, cols cperm)
  std::vector<double> X;  // coordinates d x n col-major
  int dim = 0;
  std::vector<int> cperm, rperm;
  std::vector<ClusterID> cpermed;
  std::vector<Cluster> cl;
  std::vector<std::vector<int>> bottoms, interiors, interfaces;
  std::vector<Edge> edges;
  std::unordered_map<uint64_t, int> edge_of;  // (n1,n2) -> edge index
  int current_bottom = 0;
  bool partitioned = false, assembled = false, factorized = false;
  Timers tm;
  std::vector<std::vector<double>> gmres_hist;

  Oracle(int L, int s, double t) : nlevels(L), skip(s), tol(t) {}

  static uint64_t key(int a, int b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }
  int find_edge(int n1, int n2) const {
    auto it = edge_of.find(key(n1, n2));
    return it == edge_of.end() ? -1 : it->second;
  }

  // ptree.cpp:29-41
  bool want_sparsify(const Cluster& c) const {
    if (c.merge_lvl < skip || c.merge_lvl >= nlevels - 2 || tol == 0) return false;
    if (c.lvl() > c.merge_lvl)
      if (c.id.l.lvl <= c.merge_lvl && c.id.r.lvl <= c.merge_lvl) return true;
    return false;
  }

  // ptree.cpp:101-121 new_edgeOut
  int new_edge(int c1, int c2) {
    Edge e;
    e.n1 = c1;
    e.n2 = c2;
    e.A = Mat(cl[c2].rows(), cl[c1].cols());
    edges.push_back(std::move(e));
    int id = (int)edges.size() - 1;
    edge_of[key(c1, c2)] = id;
    cl[c1].out.push_back(id);
    if (c1 != c2) {
      cl[c2].in.push_back(id);
      if (cl[c1].lvl() == cl[c1].merge_lvl) cl[c2].col_interior_deps++;
    }
    return id;
  }
  bool is_spars_edge(const Edge& e) const {
    return e.n1 != e.n2 && cl[e.n1].lvl() > current_bottom && cl[e.n2].lvl() > current_bottom;
  }
  void sort_out(int c) {
    auto& o = cl[c].out;
    std::sort(o.begin(), o.end(), [&](int a, int b) { return cl[edges[a].n2].order < cl[edges[b].n2].order; });
  }

  // -------------------------------------------------- partition
  std::vector<ClusterID> geometric_partition() {
    int c = A.ncols;
    CSC AtA = ata_pattern(A);
    std::vector<int> parts(c, 0);
    for (int depth = 0; depth < nlevels - 1; ++depth) {
      int np = 1 << depth;
      std::vector<std::vector<int>> dofs(np);
      for (int i = 0; i < c; ++i) dofs[parts[i]].push_back(i);
      for (int k = 0; k < np; ++k) {  // partition.cpp:241-279
        auto& d = dofs[k];
        int N = (int)d.size();
        if (N == 0) continue;
        int best = -1;
        double maxrange = -1.0;
        for (int dd = 0; dd < dim; ++dd) {
          double mx = -1e300, mn = 1e300;
          for (int i : d) { mx = std::max(mx, X[(size_t)i * dim + dd]); mn = std::min(mn, X[(size_t)i * dim + dd]); }
          if (mx - mn > maxrange) { maxrange = mx - mn; best = dd; }
        }
        std::vector<double> coords(N);
        for (int i = 0; i < N; ++i) coords[i] = X[(size_t)d[i] * dim + best];
        std::nth_element(coords.begin(), coords.begin() + N / 2, coords.end());
        double midv = coords[N / 2];
        for (int i = 0; i < N; ++i) parts[d[i]] = (X[(size_t)d[i] * dim + best] <= midv) ? 2 * k : 2 * k + 1;
      }
    }
    std::vector<ClusterID> cmap(c);
    for (int depth = 0; depth < nlevels - 1; ++depth) {  // partition.cpp:306-333
      int l = nlevels - depth - 1;
      for (int i = 0; i < c; ++i) {
        if (cmap[i].self.lvl != -1) continue;
        int pi = parts[i] >> (l - 1);
        if (pi % 2 != 0) continue;
        bool sep = false;
        for (int k = AtA.colptr[i]; k < AtA.colptr[i + 1]; ++k) {
          int j = AtA.rowidx[k];
          if (cmap[j].self.lvl == -1 && (parts[j] >> (l - 1)) == pi + 1) { sep = true; break; }
        }
        if (sep) { cmap[i].self = SepID(l, pi / 2); cmap[i].section = parts[i]; }
      }
    }
    for (int i = 0; i < c; ++i)
      if (cmap[i].self.lvl == -1) {
        cmap[i].self = cmap[i].l = cmap[i].r = SepID(0, parts[i]);
        cmap[i].section = parts[i];
      }
    // getInterfacesUsingA (partition.cpp:514-587); square, no matching: rmap == cmap
    std::vector<ClusterID> rmap = cmap;
    CSC At = transpose(A);  // column i of At = row i of A
    for (int i = 0; i < A.nrows; ++i) {
      SepID self = rmap[i].self;
      if (self.lvl <= 0) continue;
      SepID left(-1, 0), right(-1, 0);
      for (int k = At.colptr[i]; k < At.colptr[i + 1]; ++k) {
        SepID nbr = cmap[At.rowidx[k]].self;
        if (nbr.lvl < self.lvl) {
          int pj = nbr.sep >> (self.lvl - nbr.lvl - 1);
          if (pj % 2 == 0) left = (left.lvl == -1) ? nbr : find_lowest_common(nbr, left);
          else right = (right.lvl == -1) ? nbr : find_lowest_common(nbr, right);
        }
      }
      rmap[i].l = left;
      rmap[i].r = right;
    }
    cmap = rmap;
    for (int i = 0; i < A.nrows; ++i) {
      SepID self = rmap[i].self, left = rmap[i].l, right = rmap[i].r;
      if (right == SepID()) {
        for (int k = At.colptr[i]; k < At.colptr[i + 1]; ++k) {
          int j = At.rowidx[k];
          if (self == cmap[j].self && cmap[j].r != SepID())
            right = (right == SepID()) ? cmap[j].r : find_highest_common(right, cmap[j].r);
        }
      } else if (left == SepID()) {
        for (int k = At.colptr[i]; k < At.colptr[i + 1]; ++k) {
          int j = At.rowidx[k];
          if (self == cmap[j].self && cmap[j].l != SepID())
            left = (left == SepID()) ? cmap[j].l : find_highest_common(left, cmap[j].l);
        }
      }
      rmap[i].l = left;
      rmap[i].r = right;
    }
    for (int i = 0; i < A.nrows; ++i) {
      if (rmap[i].l == SepID()) rmap[i].l = rmap[i].self;
      if (rmap[i].r == SepID()) rmap[i].r = rmap[i].self;
    }
    return rmap;
  }

  int partition() {
    double t0 = now_s();
    if (A.nrows != A.ncols) return -2;
    if (X.empty()) return -3;
    n = A.ncols;
    std::vector<ClusterID> cmap = geometric_partition();
    // tree.cpp:48-57 initPermutation
    cperm.resize(n);
    for (int i = 0; i < n; ++i) cperm[i] = i;
    std::vector<ClusterID> pm = cmap;
    auto cmp = [&](int i, int j) { return pm[i] < pm[j]; };
    std::stable_sort(cperm.begin(), cperm.end(), cmp);
    for (int lvl = 1; lvl < nlevels; ++lvl) {
      for (auto& s : pm) s = merge_if(s, lvl);
      std::stable_sort(cperm.begin(), cperm.end(), cmp);
    }
    cpermed.resize(n);
    for (int k = 0; k < n; ++k) cpermed[k] = cmap[cperm[k]];
    rperm = cperm;
    // ptree.cpp:587-635 leaf clusters
    bottoms.assign(nlevels, {});
    interiors.assign(nlevels, {});
    interfaces.assign(nlevels, {});
    cl.clear();
    for (int k = 0; k < n;) {
      int kn = k + 1;
      while (kn < n && cpermed[kn] == cpermed[k]) kn++;
      Cluster c;
      c.cstart = c.rstart = k;
      c.csize = c.rsize = c.csize_org = c.rsize_org = c.rank = kn - k;
      c.id = cpermed[k];
      c.order = (int)cl.size();
      c.merge_lvl = 0;
      c.x.assign(c.rsize, 0.0);
      cl.push_back(c);
      bottoms[0].push_back(c.order);
      (c.id.self.lvl == 0 ? interiors[0] : interfaces[0]).push_back(c.order);
      k = kn;
    }
    // ptree.cpp:638-691 hierarchy
    for (int lvl = 1; lvl < nlevels; ++lvl) {
      std::vector<int> src;
      for (int o : bottoms[lvl - 1])
        if (cl[o].lvl() >= lvl) src.push_back(o);
      std::vector<ClusterID> pid(src.size());
      for (size_t i = 0; i < src.size(); ++i) pid[i] = merge_if(cl[src[i]].id, lvl);
      for (size_t k = 0; k < src.size();) {
        size_t kn = k + 1;
        while (kn < src.size() && pid[kn] == pid[k]) kn++;
        Cluster p;
        p.id = pid[k];
        p.order = (int)cl.size();
        p.merge_lvl = lvl;
        p.cstart = cl[src[k]].cstart;
        p.rstart = cl[src[k]].rstart;
        int cs = 0, rs = 0;
        for (size_t q = k; q < kn; ++q) { cs += cl[src[q]].csize; rs += cl[src[q]].rsize; }
        p.csize = p.csize_org = p.rank = cs;
        p.rsize = p.rsize_org = rs;
        for (size_t q = k; q < kn; ++q) p.children.push_back(src[q]);
        cl.push_back(p);
        for (size_t q = k; q < kn; ++q) cl[src[q]].parent = p.order;
        auto& ch = cl.back().children;
        std::sort(ch.begin(), ch.end(), [&](int a, int b) { return cl[a].id < cl[b].id; });
        bottoms[lvl].push_back(p.order);
        (p.id.self.lvl == lvl ? interiors[lvl] : interfaces[lvl]).push_back(p.order);
        k = kn;
      }
    }
    partitioned = true;
    tm.partition = now_s() - t0;
    return 0;
  }

  // -------------------------------------------------- assemble
  int assemble() {
    if (!partitioned) return -1;
    double t0 = now_s();
    // App = A[rperm, cperm]
    std::vector<int> rinv(n);
    for (int i = 0; i < n; ++i) rinv[rperm[i]] = i;
    App.nrows = App.ncols = n;
    App.colptr.assign(n + 1, 0);
    App.rowidx.clear();
    App.val.clear();
    std::vector<std::pair<int, double>> colbuf;
    for (int j = 0; j < n; ++j) {
      int src = cperm[j];
      colbuf.clear();
      for (int k = A.colptr[src]; k < A.colptr[src + 1]; ++k) colbuf.push_back({rinv[A.rowidx[k]], A.val[k]});
      std::sort(colbuf.begin(), colbuf.end());
      for (auto& pr : colbuf) { App.rowidx.push_back(pr.first); App.val.push_back(pr.second); }
      App.colptr[j + 1] = (int)App.rowidx.size();
    }
    std::vector<int> cmapc(n), rmapc(n);
    for (int o : bottoms[0]) {
      for (int k = cl[o].cstart; k < cl[o].cstart + cl[o].csize; ++k) cmapc[k] = o;
      for (int i = cl[o].rstart; i < cl[o].rstart + cl[o].rsize; ++i) rmapc[i] = o;
    }
    edges.clear();
    edge_of.clear();
    current_bottom = 0;
    // ptree.cpp:728-775: dense blocks for every (self, nbr) pair
    for (int s : bottoms[0]) {
      std::set<int> nb;
      for (int j = cl[s].cstart; j < cl[s].cstart + cl[s].csize; ++j)
        for (int k = App.colptr[j]; k < App.colptr[j + 1]; ++k) nb.insert(rmapc[App.rowidx[k]]);
      nb.insert(s);
      for (int nbr : nb) {
        int e = new_edge(s, nbr);
        Mat& M = edges[e].A;
        for (int j = 0; j < cl[s].csize; ++j) {
          int col = cl[s].cstart + j;
          for (int k = App.colptr[col]; k < App.colptr[col + 1]; ++k) {
            int row = App.rowidx[k];
            if (row >= cl[nbr].rstart && row < cl[nbr].rstart + cl[nbr].rsize) M(row - cl[nbr].rstart, j) = App.val[k];
          }
        }
        if (nbr == s) cl[s].self_edge = e;
      }
      sort_out(s);
    }
    // ptree.cpp:832-854: original distance-2 connections
    CSC AtA = ata_pattern(App);
    std::vector<char> visited(bottoms[0].size(), 0);
    for (int s : bottoms[0]) {
      for (int col = cl[s].cstart; col < cl[s].cstart + cl[s].csize; ++col) {
        for (int k = AtA.colptr[col]; k < AtA.colptr[col + 1]; ++k) {
          int pn = cmapc[AtA.rowidx[k]];
          if (visited[pn]) continue;
          if (cl[pn].lvl() >= cl[s].lvl() && pn != s) cl[s].d2.insert(pn);
          else if (cl[pn].lvl() < cl[s].lvl()) cl[s].d2.insert(cl[pn].d2.begin(), cl[pn].d2.end());
          visited[pn] = 1;
        }
      }
      std::fill(visited.begin(), visited.end(), 0);
    }
    assembled = true;
    tm.assemble = now_s() - t0;
    return 0;
  }

  // -------------------------------------------------- kernels (ptree.cpp:170-439)
  void geqrt_cluster(int c) {  // ptree.cpp:170-195
    Mat& S = edges[cl[c].self_edge].A;
    int m = S.r, nc = S.c;
    cl[c].T = Mat(nc, nc);
    scipy_LAPACKE_dgeqrt(kColMajor, m, nc, nc, S.p(), m, cl[c].T.p(), nc);
  }
  void tsqrt_edge(int e) {  // ptree.cpp:197-214
    Cluster& c = cl[edges[e].n1];
    Mat& B = edges[e].A;
    int nb = std::min(32, c.cols());
    Mat T(nb, B.c);
    Mat top = edges[c.self_edge].A.top_rows(c.cols());
    scipy_LAPACKE_dtpqrt(kColMajor, B.r, B.c, 0, nb, top.p(), c.cols(), B.p(), B.r, T.p(), nb);
    edges[c.self_edge].A.set_top_rows(top);
    c.Tmap[cl[edges[e].n2].order] = std::move(T);
  }
  void larfb_edge(int e) {  // ptree.cpp:216-221: A_{c,m} <- Q_c^T A_{c,m}
    Cluster& c = cl[edges[e].n2];
    Mat& C = edges[e].A;
    larfb(edges[c.self_edge].A, c.T, C.p(), C.r, C.c);
  }
  void ssrfb(int e_cn, int e_cm, int e_mn) {  // ptree.cpp:223-266
    Cluster& c = cl[edges[e_cn].n1];
    int n = edges[e_cn].n2;
    Mat& B = edges[e_mn].A;
    int k = c.cols(), nb = std::min(32, k);
    Mat top = edges[e_cm].A.top_rows(k);
    const Mat& V = edges[e_cn].A;
    const Mat& T = c.Tmap.at(n);
    scipy_LAPACKE_dtpmqrt(kColMajor, 'L', 'T', B.r, B.c, k, 0, nb, V.p(), B.r, T.p(), nb, top.p(), k, B.p(), B.r);
    edges[e_cm].A.set_top_rows(top);
  }
  void scale_cluster(int p) {  // ptree.cpp:269-286
    Cluster& c = cl[p];
    Mat& S = edges[c.self_edge].A;
    Mat Q = S;
    Mat T(c.cols(), c.cols());
    scipy_LAPACKE_dgeqrt(kColMajor, Q.r, Q.c, Q.c, Q.p(), Q.r, T.p(), Q.c);
    S.zero();
    for (int i = 0; i < c.cols(); ++i) S(i, i) = 1.0;
    c.Qs = std::move(Q);
    c.Ts = std::move(T);
  }
  void scale_apply(int e) {  // ptree.cpp:1631-1659 (larfb on rows of n2, trsm on cols of n1)
    Cluster& c = cl[edges[e].n2];
    Cluster& nn = cl[edges[e].n1];
    Mat& M = edges[e].A;
    if (want_sparsify(c)) larfb(c.Qs, c.Ts, M.p(), M.r, M.c);
    if (want_sparsify(nn)) {  // trsm_edge ptree.cpp:365-370
      int k = nn.cols();
      Mat R(k, k);
      for (int j = 0; j < k; ++j)
        for (int i = 0; i <= j; ++i) R(i, j) = nn.Qs(i, j);
      if (M.r > 0 && M.c > 0)
        scipy_cblas_dtrsm(kColMajor, kRight, kUpper, kNoTrans, kNonUnit, M.r, M.c, 1.0, R.p(), k, M.p(), M.r);
    }
  }
  std::vector<int> spars_out(int p) const {
    std::vector<int> v;
    for (int e : cl[p].out)
      if (is_spars_edge(edges[e])) v.push_back(e);
    std::sort(v.begin(), v.end(), [&](int a, int b) { return edges[a].n2 < edges[b].n2; });
    return v;
  }
  std::vector<int> spars_in(int p) const {
    std::vector<int> v;
    for (int e : cl[p].in)
      if (is_spars_edge(edges[e])) v.push_back(e);
    std::sort(v.begin(), v.end(), [&](int a, int b) { return edges[a].n1 < edges[b].n1; });
    return v;
  }
  // ptree.cpp:373-439 sparsify_rrqr_only (non-MKL geqp3 branch)
  void sparsify_rrqr(int p) {
    Cluster& c = cl[p];
    auto so = spars_out(p), si = spars_in(p);
    int w = 0;
    for (int e : so) w += edges[e].A.r;
    for (int e : si) w += edges[e].A.c;
    int m = c.cols();
    Mat C(m, w);
    int ist = 0;
    for (int e : so) {
      const Mat& M = edges[e].A;  // rows n2 x cols p -> transpose
      for (int i = 0; i < M.r; ++i)
        for (int j = 0; j < M.c; ++j) C(j, ist + i) = M(i, j);
      ist += M.r;
    }
    for (int e : si) {
      const Mat& M = edges[e].A;  // rows p x cols n1 -> top cols_p rows
      for (int j = 0; j < M.c; ++j)
        for (int i = 0; i < m; ++i) C(i, ist + j) = M(i, j);
      ist += M.c;
    }
    int kmin = std::min(m, w);
    std::vector<int> jpvt(w, 0);
    std::vector<double> tau(kmin, 0.0);
    int rank;
    if (pivot_mode == 1 && tol > 0 && tol < 1.0 && kmin > 1) {
      rank = geqp3_trunc(C.p(), m, w, tol, pivot_rtol, tau);
    } else {
      if (m > 0 && w > 0) scipy_LAPACKE_dgeqp3(kColMajor, m, w, C.p(), m, jpvt.data(), tau.data());
      // util.cpp:830-851 choose_rank (relative)
      if (tol == 0) rank = kmin;
      else if (tol >= 1.0) rank = 0;
      else if (kmin <= 1) rank = kmin;
      else {
        double sref = std::fabs(C(0, 0));
        rank = 1;
        while (rank < kmin && std::fabs(C(rank, rank)) / sref >= tol) rank++;
      }
    }
    Mat V(m, rank);
    for (int j = 0; j < rank; ++j)
      for (int i = 0; i < m; ++i) V(i, j) = C(i, j);
    std::vector<double> h(tau.begin(), tau.begin() + rank);
    Mat T(rank, rank);
    if (rank > 0) scipy_LAPACKE_dlarft(kColMajor, 'F', 'C', m, rank, V.p(), m, h.data(), T.p(), rank);
    c.Qsp = std::move(V);
    c.tausp = std::move(h);
    c.Tsp = std::move(T);
    c.sparsified = true;
    Mat& S = edges[c.self_edge].A;
    S = Mat(rank, rank);
    for (int i = 0; i < rank; ++i) S(i, i) = 1.0;
    c.reset_size(rank, rank);
  }
  // ptree.cpp:1860-1903 sparsify_larfb (square)
  void sparsify_apply(int e) {
    Cluster& c = cl[edges[e].n2];
    Cluster& nn = cl[edges[e].n1];
    Mat A = edges[e].A;
    if (want_sparsify(nn)) {
      larfb(nn.Qsp, nn.Tsp, A.p(), A.r, A.c, 'R', 'N');
      edges[e].A = A;
    }
    edges[e].A.resize_keep(c.rank, nn.rank);
    if (want_sparsify(c)) {
      int qr = c.Qsp.r;
      Mat A11(qr, nn.rank);
      for (int j = 0; j < nn.rank; ++j)
        for (int i = 0; i < qr; ++i) A11(i, j) = A(i, j);
      larfb(c.Qsp, c.Tsp, A11.p(), A11.r, A11.c);
      for (int j = 0; j < nn.rank; ++j)
        for (int i = 0; i < c.rank; ++i) edges[e].A(i, j) = A11(i, j);
    }
  }

  // ptree.cpp:289-340 compute_new_edges
  void compute_new_edges(int snew) {
    std::set<int> nbrs;
    for (int so : cl[snew].children) {
      for (int e : cl[so].out) {
        int nn = edges[e].n2;
        if (!cl[nn].eliminated) nbrs.insert(cl[nn].parent);
      }
      for (int d : cl[so].d2)
        if (cl[d].lvl() >= current_bottom) cl[snew].d2.insert(cl[d].parent);
    }
    for (int nn : nbrs) {
      int e = new_edge(snew, nn);
      if (nn == snew) cl[snew].self_edge = e;
    }
    sort_out(snew);
  }
  void fill_new_edges(int snew) {
    for (int so : cl[snew].children)
      for (int e : cl[so].out) {
        int nold = edges[e].n2;
        if (cl[nold].eliminated) continue;
        int ne = find_edge(snew, cl[nold].parent);
        Mat& P = edges[ne].A;
        const Mat& S = edges[e].A;
        for (int j = 0; j < S.c; ++j)
          for (int i = 0; i < S.r; ++i) P(cl[nold].rpos + i, cl[so].cpos + j) = S(i, j);
        edges[e].A = Mat();  // free the merged child block
      }
  }

  template <class F>
  void par_for(int ntask, F f) {
    if (ntask <= 0) return;
#ifdef _OPENMP
    if (nthreads > 1 && ntask >= nthreads) {
      scipy_openblas_set_num_threads(1);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
      for (int i = 0; i < ntask; ++i) f(i);
      return;
    }
    scipy_openblas_set_num_threads(nthreads);
#endif
    for (int i = 0; i < ntask; ++i) f(i);
    scipy_openblas_set_num_threads(1);
  }

  // -------------------------------------------------- factorize
  int factorize() {
    if (!assembled) return -1;
    double t0 = now_s();
    tm.lvl_fill.assign(nlevels, 0);
    tm.lvl_elim.assign(nlevels, 0);
    tm.lvl_scale.assign(nlevels, 0);
    tm.lvl_spars.assign(nlevels, 0);
    tm.lvl_merge.assign(nlevels, 0);
    for (int ilvl = 0; ilvl < nlevels; ++ilvl) {
      current_bottom = ilvl;
      double ta = now_s();
      auto& inter = interiors[ilvl];
      // fill-in (ptree.cpp:866-871, 140-153)
      for (int c : inter)
        for (int e : cl[c].in) cl[c].d2.insert(edges[e].n1);
      for (int c : inter) {
        for (int n2 : cl[c].d2) {
          if (n2 == c) continue;
          std::vector<int> outs = cl[c].out;
          for (int e : outs) {
            int x = edges[e].n2;
            int f = find_edge(n2, x);
            if (f < 0) f = new_edge(n2, x);
            edges[f].interior_deps++;
          }
        }
      }
      for (int c : inter)
        for (int e : cl[c].in)
          if (cl[edges[e].n1].lvl() == ilvl) {
            fprintf(stderr, "oracle: interiors %d and %d of level %d are coupled\n", c, edges[e].n1, ilvl);
            return -5;
          }
      double tb = now_s();
      // E1: geqrt + tsqrt chain per interior (touches only the interior's column blocks)
      par_for((int)inter.size(), [&](int i) {
        int c = inter[i];
        geqrt_cluster(c);
        for (int e : cl[c].out)
          if (edges[e].n2 != c) tsqrt_edge(e);
      });
      // order_of_trans: ascending interior order (the schedule this oracle fixes)
      for (int c : inter)
        for (int e : cl[c].out)
          if (edges[e].n2 != c) cl[edges[e].n2].order_of_trans.push_back(c);
      // E2: larfb + ssrfb, grouped by target column cluster m; interiors ascending
      std::map<int, std::vector<int>> by_col;  // m -> interiors c with edge m->c
      for (int c : inter)
        for (int e : cl[c].in) by_col[edges[e].n1].push_back(c);
      std::vector<std::pair<int, std::vector<int>>> cols(by_col.begin(), by_col.end());
      int bad = 0;
      par_for((int)cols.size(), [&](int i) {
        int m = cols[i].first;
        for (int c : cols[i].second) {
          int e_cm = find_edge(m, c);
          larfb_edge(e_cm);
          for (int e_cn : cl[c].out) {
            int nn = edges[e_cn].n2;
            if (nn == c) continue;
            int e_mn = find_edge(m, nn);
            if (e_mn < 0) { bad = 1; continue; }
            ssrfb(e_cn, e_cm, e_mn);
          }
        }
      });
      if (bad) return -6;
      for (int c : inter) cl[c].eliminated = true;
      double tc = now_s();
      // scaling + sparsification (ptree.cpp:1533-1903)
      auto& itf = interfaces[ilvl];
      std::vector<int> sp;
      for (int p : itf)
        if (want_sparsify(cl[p])) sp.push_back(p);
      std::vector<int> sedges;
      for (int p : itf)
        for (int e : cl[p].out)
          if (is_spars_edge(edges[e])) sedges.push_back(e);
      if (!sp.empty()) {
        par_for((int)sp.size(), [&](int i) { scale_cluster(sp[i]); });
        par_for((int)sedges.size(), [&](int i) { scale_apply(sedges[i]); });
      }
      double td = now_s();
      if (!sp.empty()) {
        par_for((int)sp.size(), [&](int i) { sparsify_rrqr(sp[i]); });
        par_for((int)sedges.size(), [&](int i) { sparsify_apply(sedges[i]); });
      }
      double te = now_s();
      // merge (ptree.cpp:1940-2123)
      if (ilvl < nlevels - 1) {
        current_bottom = ilvl + 1;
        for (int snew : bottoms[ilvl + 1]) {
          int rs = 0, cs = 0;
          for (int so : cl[snew].children) {
            cl[so].rpos = rs;
            cl[so].cpos = cs;
            rs += cl[so].rows();
            cs += cl[so].cols();
          }
          cl[snew].set_size(rs, cs);
          cl[snew].rsize_org = rs;
          cl[snew].csize_org = cs;
        }
        for (int snew : bottoms[ilvl + 1]) compute_new_edges(snew);
        par_for((int)bottoms[ilvl + 1].size(), [&](int i) { fill_new_edges(bottoms[ilvl + 1][i]); });
      }
      double tf = now_s();
      tm.lvl_fill[ilvl] = tb - ta;
      tm.lvl_elim[ilvl] = tc - tb;
      tm.lvl_scale[ilvl] = td - tc;
      tm.lvl_spars[ilvl] = te - td;
      tm.lvl_merge[ilvl] = tf - te;
    }
    factorized = true;
    tm.factorize = now_s() - t0;
    return 0;
  }

  // -------------------------------------------------- solve (ptree.cpp:2788-3210)
  void solve(double* xv) {
    for (int c : bottoms[0]) {
      Cluster& C = cl[c];
      C.x.assign(xv + C.cstart, xv + C.cstart + C.csize_org);
    }
    for (int l = 0; l < nlevels; ++l) {
      for (int c : interiors[l]) {
        Cluster& C = cl[c];
        const Mat& S = edges[C.self_edge].A;
        larfb(S, C.T, C.x.data(), S.r, 1);  // fwd_geqrt
        for (int e : C.out) {                // fwd_tsqrt chain (QR_tsqrt_fwd ptree.cpp:2160-2187)
          int nn = edges[e].n2;
          if (nn == c) continue;
          const Mat& V = edges[e].A;
          int k = C.cols(), nb = std::min(32, k);
          scipy_LAPACKE_dtpmqrt(kColMajor, 'L', 'T', V.r, 1, k, 0, nb, V.p(), V.r, C.Tmap.at(nn).p(), nb, C.x.data(), k,
                                cl[nn].x.data(), V.r);
        }
      }
      for (int p : interfaces[l]) {
        Cluster& P = cl[p];
        if (!want_sparsify(P)) continue;
        larfb(P.Qs, P.Ts, P.x.data(), P.Qs.r, 1);  // scaleD_fwd
        if (P.Qsp.c > 0)                            // orthogonalD_fwd
          scipy_LAPACKE_dormqr(kColMajor, 'L', 'T', P.csize_org, 1, P.Qsp.c, P.Qsp.p(), P.Qsp.r, P.tausp.data(),
                               P.x.data(), P.csize_org);
      }
      if (l < nlevels - 1)
        for (int par : bottoms[l + 1]) {  // merge_fwd
          int k = 0;
          for (int ch : cl[par].children)
            for (int i = 0; i < cl[ch].rows(); ++i) cl[par].x[k++] = cl[ch].x[i];
        }
    }
    for (int l = nlevels - 1; l >= 0; --l) {
      for (int p : interfaces[l]) {
        Cluster& P = cl[p];
        if (!want_sparsify(P)) continue;
        if (P.Qsp.c > 0)  // orthogonalD_bwd
          scipy_LAPACKE_dormqr(kColMajor, 'L', 'N', P.csize_org, 1, P.Qsp.c, P.Qsp.p(), P.Qsp.r, P.tausp.data(),
                               P.x.data(), P.csize_org);
        int k = P.csize_org;  // scaleD_bwd
        scipy_cblas_dtrsv(kColMajor, kUpper, kNoTrans, kNonUnit, k, P.Qs.p(), P.Qs.r, P.x.data(), 1);
      }
      for (int c : interiors[l]) {
        Cluster& C = cl[c];
        std::vector<int> ins = C.in;
        std::sort(ins.begin(), ins.end(), [&](int a, int b) { return edges[a].n1 < edges[b].n1; });
        std::vector<double> t(C.cols());
        for (int e : ins) {  // bwd_spars reduce_x: x_c -= R_{c,m} x_m
          const Mat& R = edges[e].A;
          const Cluster& M = cl[edges[e].n1];
          for (int i = 0; i < C.cols(); ++i) {
            double s = 0;
            for (int j = 0; j < R.c; ++j) s += R(i, j) * M.x[j];
            t[i] = s;
          }
          for (int i = 0; i < C.cols(); ++i) C.x[i] -= t[i];
        }
        const Mat& S = edges[C.self_edge].A;  // trsv_bwd
        if (C.cols() > 0) scipy_cblas_dtrsv(kColMajor, kUpper, kNoTrans, kNonUnit, C.cols(), S.p(), S.r, C.x.data(), 1);
      }
      if (l > 0)
        for (int par : bottoms[l]) {  // merge_bwd
          int k = 0;
          for (int ch : cl[par].children)
            for (int i = 0; i < cl[ch].cols(); ++i) cl[ch].x[i] = cl[par].x[k++];
        }
    }
    for (int c : bottoms[0]) {
      const Cluster& C = cl[c];
      for (int i = 0; i < C.csize_org; ++i) xv[C.cstart + i] = C.x[i];
    }
  }

  // ptree.cpp:3212-3262: y = App x, accumulated per leaf column cluster
  void spmv(const double* xv, double* y) const {
    std::fill(y, y + n, 0.0);
    std::vector<double> t(n, 0.0);
    for (int c : bottoms[0]) {
      const Cluster& C = cl[c];
      std::vector<int> touched;
      for (int j = C.cstart; j < C.cstart + C.csize_org; ++j)
        for (int k = App.colptr[j]; k < App.colptr[j + 1]; ++k) {
          int r = App.rowidx[k];
          t[r] += App.val[k] * xv[j];
          touched.push_back(r);
        }
      for (int r : touched) { y[r] += t[r]; t[r] = 0.0; }
    }
  }

  // is.cpp:447-527 dist_gmres (single rank)
  int gmres(double* b, int iter, double gtol, int* iters_out, double* relres_out, std::vector<double>& hist) {
    double t0 = now_s();
    std::vector<double> r(b, b + n);
    solve(r.data());
    auto nrm = [&](const double* v) {
      double s = 0;
      for (int i = 0; i < n; ++i) s += v[i] * v[i];
      return std::sqrt(s);
    };
    double b_norm = nrm(b), r_norm = nrm(r.data());
    (void)b_norm;
    if (std::isnan(r_norm)) return -7;
    std::vector<double> sn(iter, 0), cs(iter, 0), beta(iter + 1, 0);
    std::vector<double> Q((size_t)n * (iter + 1), 0.0), H((size_t)(iter + 1) * iter, 0.0);
    auto Hc = [&](int i, int j) -> double& { return H[(size_t)j * (iter + 1) + i]; };
    for (int i = 0; i < n; ++i) Q[i] = r[i] / r_norm;
    beta[0] = r_norm;
    std::vector<double> q(n);
    int k = 0;
    hist.clear();
    for (; k < iter; ++k) {
      spmv(&Q[(size_t)k * n], q.data());
      solve(q.data());
      for (int i = 0; i <= k; ++i) {
        const double* Qi = &Q[(size_t)i * n];
        double d = 0;
        for (int t = 0; t < n; ++t) d += q[t] * Qi[t];
        Hc(i, k) = d;
        for (int t = 0; t < n; ++t) q[t] -= d * Qi[t];
      }
      double hn = nrm(q.data());
      Hc(k + 1, k) = hn;
      for (int t = 0; t < n; ++t) Q[(size_t)(k + 1) * n + t] = q[t] / hn;
      for (int i = 0; i < k; ++i) {
        double temp = cs[i] * Hc(i, k) + sn[i] * Hc(i + 1, k);
        Hc(i + 1, k) = -sn[i] * Hc(i, k) + cs[i] * Hc(i + 1, k);
        Hc(i, k) = temp;
      }
      if (Hc(k, k) == 0) { cs[k] = 0; sn[k] = 1; }
      else {
        double t = std::sqrt(Hc(k, k) * Hc(k, k) + Hc(k + 1, k) * Hc(k + 1, k));
        cs[k] = std::fabs(Hc(k, k)) / t;
        sn[k] = cs[k] * Hc(k + 1, k) / Hc(k, k);
      }
      Hc(k, k) = cs[k] * Hc(k, k) + sn[k] * Hc(k + 1, k);
      Hc(k + 1, k) = 0.0;
      beta[k + 1] = -sn[k] * beta[k];
      beta[k] = cs[k] * beta[k];
      double err = std::fabs(beta[k + 1]) / r_norm;
      hist.push_back(err);
      if (err <= gtol) break;
    }
    k = std::min(k, iter - 1);
    std::vector<double> y(k + 1, 0.0);  // util.cpp:1019-1032 LUSolve
    for (int i = k; i >= 0; --i) {
      y[i] = beta[i];
      for (int j = i + 1; j < k + 1; ++j) y[i] -= Hc(i, j) * y[j];
      y[i] /= Hc(i, i);
    }
    std::vector<double> bcopy(b, b + n);
    for (int t = 0; t < n; ++t) {
      double s = 0;
      for (int i = 0; i <= k; ++i) s += Q[(size_t)i * n + t] * y[i];
      b[t] = s;
    }
    std::vector<double> Ax(n);
    spmv(b, Ax.data());
    double rn = 0, bn = 0;
    for (int t = 0; t < n; ++t) { rn += (bcopy[t] - Ax[t]) * (bcopy[t] - Ax[t]); bn += bcopy[t] * bcopy[t]; }
    *iters_out = k;
    *relres_out = std::sqrt(rn) / std::sqrt(bn);
    tm.gmres = now_s() - t0;
    return 0;
  }
};

int fill_cluster_info(const Oracle& o, int order, int* info) {
  if (order < 0 || order >= (int)o.cl.size()) return -1;
  const Cluster& c = o.cl[order];
  info[0] = c.lvl();
  info[1] = c.merge_lvl;
  info[2] = c.rsize;
  info[3] = c.csize;
  info[4] = c.rank;
  info[5] = c.parent;
  info[6] = c.cstart;
  info[7] = c.id.self.sep;
  info[8] = c.id.l.lvl;
  info[9] = c.id.l.sep;
  info[10] = c.id.r.lvl;
  info[11] = c.id.r.sep;
  info[12] = c.id.section;
  info[13] = c.csize_org;
  info[14] = c.sparsified ? 1 : 0;
  info[15] = (int)c.children.size();
  return 0;
}
}  // namespace

// ----------------------------------------------------------------- C ABI (ctypes)
extern "C" {
void* orc_create(int nlevels, int skip, double tol, int nthreads) {
  if (nlevels < 2) return nullptr;
  Oracle* o = new Oracle(nlevels, tol == 0 ? nlevels - 1 : skip, tol);
  o->nthreads = std::max(1, nthreads);
  scipy_openblas_set_num_threads(1);
  return o;
}
void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }
int orc_set_pivot(void* h, int mode, double rtol) {
  Oracle* o = static_cast<Oracle*>(h);
  o->pivot_mode = mode;
  o->pivot_rtol = rtol;
  return 0;
}
int orc_set_threads(void* h, int t) {
  static_cast<Oracle*>(h)->nthreads = std::max(1, t);
  return 0;
}
// Matrix in CSC (0-based).  scale != 0 applies the driver's column scaling
// A <- A * diag(1/||A(:,j)||) * 10 (pspaQR.cpp:133-146).
int orc_set_matrix(void* h, int nrows, int ncols, const int* colptr, const int* rowidx, const double* val, int scale) {
  Oracle* o = static_cast<Oracle*>(h);
  o->A.nrows = nrows;
  o->A.ncols = ncols;
  o->A.colptr.assign(colptr, colptr + ncols + 1);
  int nnz = colptr[ncols];
  o->A.rowidx.assign(rowidx, rowidx + nnz);
  o->A.val.assign(val, val + nnz);
  if (scale) {
    for (int j = 0; j < ncols; ++j) {
      double s = 0;
      for (int k = colptr[j]; k < colptr[j + 1]; ++k) s += val[k] * val[k];
      double d = 1.0 / std::sqrt(s);
      for (int k = colptr[j]; k < colptr[j + 1]; ++k) o->A.val[k] = (val[k] * d) * 10.0;
    }
  }
  return 0;
}
int orc_get_matrix_values(void* h, double* val) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->A.val.begin(), o->A.val.end(), val);
  return 0;
}
// Tensor-grid coordinates (util.cpp:901-930 linspace_nd): node i*n^(d-1)+... .
int orc_set_coords_tensor(void* h, int n, int d) {
  Oracle* o = static_cast<Oracle*>(h);
  long N = 1;
  for (int i = 0; i < d; ++i) N *= n;
  o->dim = d;
  o->X.assign((size_t)N * d, 0.0);
  for (long id = 0; id < N; ++id) {
    long r = id;
    for (int dd = d - 1; dd >= 0; --dd) { o->X[(size_t)id * d + dd] = (double)(r % n); r /= n; }
  }
  return 0;
}
int orc_partition(void* h) { return static_cast<Oracle*>(h)->partition(); }
int orc_assemble(void* h) { return static_cast<Oracle*>(h)->assemble(); }
int orc_factorize(void* h) { return static_cast<Oracle*>(h)->factorize(); }
int orc_solve_inplace(void* h, double* x) {
  Oracle* o = static_cast<Oracle*>(h);
  if (!o->factorized) return -1;
  double t0 = now_s();
  o->solve(x);
  o->tm.solve = now_s() - t0;
  return 0;
}
// One-shot solve with a global (unpermuted) right-hand side (ptree.cpp:2268-2785, square)
int orc_solve_global(void* h, const double* b, double* x) {
  Oracle* o = static_cast<Oracle*>(h);
  if (!o->factorized) return -1;
  std::vector<double> t(o->n);
  for (int i = 0; i < o->n; ++i) t[i] = b[o->rperm[i]];
  o->solve(t.data());
  for (int i = 0; i < o->n; ++i) x[o->cperm[i]] = t[i];
  return 0;
}
int orc_spmv(void* h, const double* x, double* y) {
  Oracle* o = static_cast<Oracle*>(h);
  if (!o->assembled) return -1;
  o->spmv(x, y);
  return 0;
}
int orc_gmres(void* h, double* b, int maxit, double tol, int* iters, double* relres, double* hist, int hist_cap) {
  Oracle* o = static_cast<Oracle*>(h);
  if (!o->factorized) return -1;
  std::vector<double> hv;
  int rc = o->gmres(b, maxit, tol, iters, relres, hv);
  for (int i = 0; i < (int)hv.size() && i < hist_cap; ++i) hist[i] = hv[i];
  return rc;
}
int orc_n(void* h) { return static_cast<Oracle*>(h)->n; }
int orc_get_perm(void* h, int* cperm) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->cperm.begin(), o->cperm.end(), cperm);
  return 0;
}
int orc_num_clusters(void* h) { return (int)static_cast<Oracle*>(h)->cl.size(); }
int orc_level_count(void* h, int lvl, int which) {  // which: 0 bottoms, 1 interiors, 2 interfaces
  Oracle* o = static_cast<Oracle*>(h);
  if (lvl < 0 || lvl >= o->nlevels) return -1;
  return (int)(which == 0 ? o->bottoms[lvl] : which == 1 ? o->interiors[lvl] : o->interfaces[lvl]).size();
}
int orc_level_first(void* h, int lvl) {
  Oracle* o = static_cast<Oracle*>(h);
  if (lvl < 0 || lvl >= o->nlevels || o->bottoms[lvl].empty()) return -1;
  return o->bottoms[lvl][0];
}
int orc_cluster_info(void* h, int order, int* info) { return fill_cluster_info(*static_cast<Oracle*>(h), order, info); }
int orc_num_edges(void* h) { return (int)static_cast<Oracle*>(h)->edges.size(); }
// Final dense block of the edge n1 -> n2 (after factorization: V/R blocks of interiors).
int orc_block_shape(void* h, int n1, int n2, int* shape) {
  Oracle* o = static_cast<Oracle*>(h);
  int e = o->find_edge(n1, n2);
  if (e < 0) return -1;
  shape[0] = o->edges[e].A.r;
  shape[1] = o->edges[e].A.c;
  return 0;
}
int orc_block(void* h, int n1, int n2, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  int e = o->find_edge(n1, n2);
  if (e < 0) return -1;
  std::copy(o->edges[e].A.a.begin(), o->edges[e].A.a.end(), out);
  return 0;
}
// Edge list dump: for k in [0, num_edges): (n1, n2, rows, cols)
int orc_edges(void* h, int* out4) {
  Oracle* o = static_cast<Oracle*>(h);
  for (size_t k = 0; k < o->edges.size(); ++k) {
    out4[4 * k] = o->edges[k].n1;
    out4[4 * k + 1] = o->edges[k].n2;
    out4[4 * k + 2] = o->edges[k].A.r;
    out4[4 * k + 3] = o->edges[k].A.c;
  }
  return 0;
}
// Sparsification factors of an interface: Q_sp (rows x rank), tau (rank)
int orc_qsp_shape(void* h, int order, int* shape) {
  Oracle* o = static_cast<Oracle*>(h);
  const Cluster& c = o->cl[order];
  shape[0] = c.Qsp.r;
  shape[1] = c.Qsp.c;
  return 0;
}
int orc_qsp(void* h, int order, double* V, double* tau) {
  Oracle* o = static_cast<Oracle*>(h);
  const Cluster& c = o->cl[order];
  std::copy(c.Qsp.a.begin(), c.Qsp.a.end(), V);
  std::copy(c.tausp.begin(), c.tausp.end(), tau);
  return 0;
}
double orc_time(void* h, int which) {
  Oracle* o = static_cast<Oracle*>(h);
  switch (which) {
    case 0: return o->tm.partition;
    case 1: return o->tm.assemble;
    case 2: return o->tm.factorize;
    case 3: return o->tm.solve;
    case 4: return o->tm.gmres;
  }
  return -1;
}
// Reference RHS (util.cpp:992-1001): mt19937 seeded, U(-1,1).
int orc_random_reference(int n, int seed, double* out) {
  std::mt19937 rng;
  rng.seed(seed);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (int i = 0; i < n; ++i) out[i] = dist(rng);
  return 0;
}
}
