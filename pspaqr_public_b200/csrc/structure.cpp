// structure.cpp -- partition + symbolic factorization (see structure.hpp).
#include "structure.hpp"

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <set>

namespace spq {

bool ClusterID::operator<(const ClusterID& o) const {
  if (self != o.self) return self < o.self;
  if (l != o.l) return l < o.l;
  if (r != o.r) return r < o.r;
  if (section != o.section) return section < o.section;
  return part < o.part;
}

static SepID sep_up(SepID s) { return SepID(s.lvl + 1, s.sep / 2); }

// cluster.cpp:23-32
ClusterID merge_if(const ClusterID& c, int lvl) {
  ClusterID o = c;
  if (c.l.lvl < lvl) o.l = sep_up(c.l);
  if (c.r.lvl < lvl) o.r = sep_up(c.r);
  if (lvl > 0) o.section = c.section / 2;
  if (c.self.lvl == lvl) o.part = 2;
  return o;
}

int Structure::find_edge(int n1, int n2) const {
  auto it = edge_of.find(((uint64_t)(uint32_t)n1 << 32) | (uint32_t)n2);
  return it == edge_of.end() ? -1 : it->second;
}

namespace {

// Column j of the transpose lists the columns of row j.
Csc transpose_pattern(const Csc& A) {
  Csc T;
  T.nrows = A.ncols;
  T.ncols = A.nrows;
  T.colptr.assign(A.nrows + 1, 0);
  for (int r : A.rowidx) T.colptr[r + 1]++;
  std::partial_sum(T.colptr.begin(), T.colptr.end(), T.colptr.begin());
  T.rowidx.resize(A.rowidx.size());
  std::vector<int> pos(T.colptr.begin(), T.colptr.end() - 1);
  for (int j = 0; j < A.ncols; ++j)
    for (int k = A.colptr[j]; k < A.colptr[j + 1]; ++k) T.rowidx[pos[A.rowidx[k]]++] = j;
  return T;
}

// Pattern of A^T A: columns sharing at least one row (diagonal included).
Csc normal_pattern(const Csc& A) {
  Csc At = transpose_pattern(A);
  Csc P;
  P.nrows = P.ncols = A.ncols;
  P.colptr.assign(A.ncols + 1, 0);
  std::vector<int> stamp(A.ncols, -1), buf;
  for (int j = 0; j < A.ncols; ++j) {
    buf.clear();
    for (int k = A.colptr[j]; k < A.colptr[j + 1]; ++k) {
      int row = A.rowidx[k];
      for (int q = At.colptr[row]; q < At.colptr[row + 1]; ++q) {
        int c = At.rowidx[q];
        if (stamp[c] != j) {
          stamp[c] = j;
          buf.push_back(c);
        }
      }
    }
    std::sort(buf.begin(), buf.end());
    P.rowidx.insert(P.rowidx.end(), buf.begin(), buf.end());
    P.colptr[j + 1] = (int)P.rowidx.size();
  }
  return P;
}

SepID highest_common(SepID a, SepID b) {
  while (a.lvl < b.lvl) a = sep_up(a);
  while (b.lvl < a.lvl) b = sep_up(b);
  while (a.sep != b.sep) {
    a = sep_up(a);
    b = sep_up(b);
  }
  return a;
}

SepID lowest_common(SepID cand, SepID cur) { return cand.lvl < cur.lvl ? cand : cur; }

}  // namespace

std::vector<ClusterID> geometric_partition(const Csc& A, int nlevels, const std::vector<double>& X, int dim) {
  const int n = A.ncols;
  Csc ata = normal_pattern(A);
  std::vector<int> part(n, 0);
  // recursive coordinate bisection (partition.cpp:241-304): cut the largest
  // coordinate range at the N/2-th smallest coordinate value, "<=" goes left.
  std::vector<double> coord;
  for (int depth = 0; depth + 1 < nlevels; ++depth) {
    const int nparts = 1 << depth;
    std::vector<std::vector<int>> members(nparts);
    for (int i = 0; i < n; ++i) members[part[i]].push_back(i);
    for (int k = 0; k < nparts; ++k) {
      const auto& mem = members[k];
      if (mem.empty()) continue;
      int axis = -1;
      double widest = -1.0;
      for (int d = 0; d < dim; ++d) {
        double lo = X[(size_t)mem[0] * dim + d], hi = lo;
        for (int i : mem) {
          double v = X[(size_t)i * dim + d];
          lo = std::min(lo, v);
          hi = std::max(hi, v);
        }
        if (hi - lo > widest) {
          widest = hi - lo;
          axis = d;
        }
      }
      coord.resize(mem.size());
      for (size_t i = 0; i < mem.size(); ++i) coord[i] = X[(size_t)mem[i] * dim + axis];
      auto mid = coord.begin() + mem.size() / 2;
      std::nth_element(coord.begin(), mid, coord.end());
      const double cut = *mid;
      for (int i : mem) part[i] = (X[(size_t)i * dim + axis] <= cut) ? 2 * k : 2 * k + 1;
    }
  }
  // separators from the top level down: a left-part node AtA-adjacent to a
  // not-yet-separator node of the matching right part (partition.cpp:306-333)
  std::vector<ClusterID> cmap(n);
  for (int depth = 0; depth + 1 < nlevels; ++depth) {
    const int l = nlevels - depth - 1;
    for (int i = 0; i < n; ++i) {
      if (cmap[i].self.lvl != -1) continue;
      const int pi = part[i] >> (l - 1);
      if (pi & 1) continue;
      for (int k = ata.colptr[i]; k < ata.colptr[i + 1]; ++k) {
        int j = ata.rowidx[k];
        if (cmap[j].self.lvl == -1 && (part[j] >> (l - 1)) == pi + 1) {
          cmap[i].self = SepID(l, pi / 2);
          cmap[i].section = part[i];
          break;
        }
      }
    }
  }
  for (int i = 0; i < n; ++i)
    if (cmap[i].self.lvl == -1) {
      cmap[i].self = cmap[i].l = cmap[i].r = SepID(0, part[i]);
      cmap[i].section = part[i];
    }
  // left / right neighbourhoods of separator rows (partition.cpp:514-587)
  Csc rowsA = transpose_pattern(A);  // column i = columns present in row i
  std::vector<ClusterID> rmap = cmap;
  for (int i = 0; i < A.nrows; ++i) {
    const SepID self = rmap[i].self;
    if (self.lvl <= 0) continue;
    SepID left, right;
    for (int k = rowsA.colptr[i]; k < rowsA.colptr[i + 1]; ++k) {
      const SepID nb = cmap[rowsA.rowidx[k]].self;
      if (nb.lvl >= self.lvl) continue;
      const int side = nb.sep >> (self.lvl - nb.lvl - 1);
      SepID& tgt = (side & 1) ? right : left;
      tgt = (tgt.lvl == -1) ? nb : lowest_common(nb, tgt);
    }
    rmap[i].l = left;
    rmap[i].r = right;
  }
  cmap = rmap;
  for (int i = 0; i < A.nrows; ++i) {
    const SepID self = rmap[i].self;
    SepID left = rmap[i].l, right = rmap[i].r;
    if (right == SepID()) {
      for (int k = rowsA.colptr[i]; k < rowsA.colptr[i + 1]; ++k) {
        const ClusterID& cj = cmap[rowsA.rowidx[k]];
        if (cj.self == self && cj.r != SepID()) right = (right == SepID()) ? cj.r : highest_common(right, cj.r);
      }
    } else if (left == SepID()) {
      for (int k = rowsA.colptr[i]; k < rowsA.colptr[i + 1]; ++k) {
        const ClusterID& cj = cmap[rowsA.rowidx[k]];
        if (cj.self == self && cj.l != SepID()) left = (left == SepID()) ? cj.l : highest_common(left, cj.l);
      }
    }
    rmap[i].l = (left == SepID()) ? self : left;
    rmap[i].r = (right == SepID()) ? self : right;
  }
  return rmap;
}

namespace {

struct Builder {
  Structure& s;
  // dynamic adjacency while building
  std::vector<std::vector<int>> out, in;
  std::vector<std::set<int>> d2;

  explicit Builder(Structure& st) : s(st) {}

  int add_edge(int n1, int n2, int level) {
    Edge e;
    e.n1 = n1;
    e.n2 = n2;
    e.level = level;
    const Cluster& a = s.clusters[n1];
    const Cluster& b = s.clusters[n2];
    e.spars = (n1 != n2) && a.lvl > level && b.lvl > level;
    s.edges.push_back(e);
    int id = (int)s.edges.size() - 1;
    s.edge_of[((uint64_t)(uint32_t)n1 << 32) | (uint32_t)n2] = id;
    out[n1].push_back(id);
    if (n1 != n2) in[n2].push_back(id);
    s.levels[level].edges.push_back(id);
    return id;
  }

  void sort_out(int c) {
    auto& o = out[c];
    std::sort(o.begin(), o.end(), [&](int a, int b) { return s.edges[a].n2 < s.edges[b].n2; });
  }

  bool want_sparsify(const Cluster& c) const {
    if (c.merge_lvl < s.skip || c.merge_lvl >= s.nlevels - 2 || s.tol == 0) return false;
    return c.lvl > c.merge_lvl && c.id.l.lvl <= c.merge_lvl && c.id.r.lvl <= c.merge_lvl;
  }
};

}  // namespace

int build_structure(Structure& s, const Csc& A, int nlevels, int skip, double tol, const std::vector<double>& X,
                    int dim) {
  if (A.nrows != A.ncols) {
    s.error = "only square matrices are supported";
    return -2;
  }
  if (nlevels < 2) {
    s.error = "nlevels must be >= 2";
    return -2;
  }
  const int n = A.ncols;
  if ((int64_t)X.size() != (int64_t)n * dim || dim <= 0) {
    s.error = "coordinates do not match the matrix size";
    return -3;
  }
  if ((n >> (nlevels - 1)) < 1) {
    s.error = "too many levels for the matrix size";
    return -2;
  }
  s.n = n;
  s.nlevels = nlevels;
  s.skip = (tol == 0) ? nlevels - 1 : skip;
  s.tol = tol;

  std::vector<ClusterID> cmap = geometric_partition(A, nlevels, X, dim);

  // initPermutation (tree.cpp:48-57): stable sorts by the ids merged level by level
  s.cperm.resize(n);
  std::iota(s.cperm.begin(), s.cperm.end(), 0);
  std::vector<ClusterID> key = cmap;
  auto by_key = [&](int i, int j) { return key[i] < key[j]; };
  std::stable_sort(s.cperm.begin(), s.cperm.end(), by_key);
  for (int lvl = 1; lvl < nlevels; ++lvl) {
    for (auto& k : key) k = merge_if(k, lvl);
    std::stable_sort(s.cperm.begin(), s.cperm.end(), by_key);
  }
  s.rperm = s.cperm;
  s.cpermed.resize(n);
  for (int k = 0; k < n; ++k) s.cpermed[k] = cmap[s.cperm[k]];

  // clusters: leaves = runs of equal ids; parents = runs of equal merged ids
  s.clusters.clear();
  s.children.clear();
  s.levels.assign(nlevels, Level());
  auto finish_cluster = [&](Cluster& c, int lvl) {
    c.lvl = c.id.self.lvl;
    c.merge_lvl = lvl;
    c.interior = (c.lvl == lvl);
  };
  s.levels[0].first = 0;
  for (int k = 0; k < n;) {
    int e = k + 1;
    while (e < n && s.cpermed[e] == s.cpermed[k]) ++e;
    Cluster c;
    c.id = s.cpermed[k];
    c.cstart = k;
    c.size0 = e - k;
    finish_cluster(c, 0);
    s.clusters.push_back(c);
    k = e;
  }
  s.levels[0].count = (int)s.clusters.size();
  for (int lvl = 1; lvl < nlevels; ++lvl) {
    const Level& prev = s.levels[lvl - 1];
    std::vector<int> src;
    for (int o = prev.first; o < prev.first + prev.count; ++o)
      if (s.clusters[o].lvl >= lvl) src.push_back(o);
    s.levels[lvl].first = (int)s.clusters.size();
    for (size_t k = 0; k < src.size();) {
      ClusterID pid = merge_if(s.clusters[src[k]].id, lvl);
      size_t e = k + 1;
      while (e < src.size() && merge_if(s.clusters[src[e]].id, lvl) == pid) ++e;
      Cluster p;
      p.id = pid;
      p.cstart = s.clusters[src[k]].cstart;
      finish_cluster(p, lvl);
      std::vector<int> kids(src.begin() + k, src.begin() + e);
      std::sort(kids.begin(), kids.end(), [&](int a, int b) { return s.clusters[a].id < s.clusters[b].id; });
      p.child_begin = (int)s.children.size();
      for (int ch : kids) {
        s.children.push_back(ch);
        p.size0 += s.clusters[ch].size0;
      }
      p.child_end = (int)s.children.size();
      int me = (int)s.clusters.size();
      s.clusters.push_back(p);
      for (int ch : kids) s.clusters[ch].parent = me;
      k = e;
    }
    s.levels[lvl].count = (int)s.clusters.size() - s.levels[lvl].first;
  }
  Builder b(s);
  for (auto& c : s.clusters) c.sparsify = b.want_sparsify(c);
  for (int lvl = 0; lvl < nlevels; ++lvl) {
    Level& L = s.levels[lvl];
    for (int o = L.first; o < L.first + L.count; ++o) (s.clusters[o].interior ? L.interiors : L.interfaces).push_back(o);
  }

  // App = A[rperm, cperm]
  {
    std::vector<int> rinv(n);
    for (int i = 0; i < n; ++i) rinv[s.rperm[i]] = i;
    Csc& P = s.App;
    P.nrows = P.ncols = n;
    P.colptr.assign(n + 1, 0);
    P.rowidx.clear();
    P.val.clear();
    P.rowidx.reserve(A.rowidx.size());
    P.val.reserve(A.rowidx.size());
    std::vector<std::pair<int, double>> col;
    for (int j = 0; j < n; ++j) {
      int src = s.cperm[j];
      col.clear();
      for (int k = A.colptr[src]; k < A.colptr[src + 1]; ++k) col.push_back({rinv[A.rowidx[k]], A.val[k]});
      std::sort(col.begin(), col.end());
      for (auto& pr : col) {
        P.rowidx.push_back(pr.first);
        P.val.push_back(pr.second);
      }
      P.colptr[j + 1] = (int)P.rowidx.size();
    }
  }

  const int ncl = (int)s.clusters.size();
  b.out.assign(ncl, {});
  b.in.assign(ncl, {});
  b.d2.assign(ncl, {});
  s.edges.clear();
  s.edge_of.clear();

  // level-0 blocks: every (column cluster, row cluster) pair with a nonzero
  std::vector<int> leaf_of(n);
  const Level& L0 = s.levels[0];
  for (int o = L0.first; o < L0.first + L0.count; ++o)
    for (int k = s.clusters[o].cstart; k < s.clusters[o].cstart + s.clusters[o].size0; ++k) leaf_of[k] = o;
  for (int o = L0.first; o < L0.first + L0.count; ++o) {
    std::set<int> nb;
    const Cluster& c = s.clusters[o];
    for (int j = c.cstart; j < c.cstart + c.size0; ++j)
      for (int k = s.App.colptr[j]; k < s.App.colptr[j + 1]; ++k) nb.insert(leaf_of[s.App.rowidx[k]]);
    nb.insert(o);
    for (int t : nb) b.add_edge(o, t, 0);
    b.sort_out(o);
  }
  // original distance-2 connections (ptree.cpp:832-854)
  {
    Csc ata = normal_pattern(s.App);
    std::vector<char> seen(L0.count, 0);
    std::vector<int> touched;
    for (int o = L0.first; o < L0.first + L0.count; ++o) {
      const Cluster& c = s.clusters[o];
      touched.clear();
      for (int col = c.cstart; col < c.cstart + c.size0; ++col)
        for (int k = ata.colptr[col]; k < ata.colptr[col + 1]; ++k) {
          int q = leaf_of[ata.rowidx[k]];
          if (seen[q - L0.first]) continue;
          seen[q - L0.first] = 1;
          touched.push_back(q);
          if (s.clusters[q].lvl >= c.lvl && q != o) b.d2[o].insert(q);
          else if (s.clusters[q].lvl < c.lvl) b.d2[o].insert(b.d2[q].begin(), b.d2[q].end());
        }
      for (int q : touched) seen[q - L0.first] = 0;
    }
  }

  for (int lvl = 0; lvl < nlevels; ++lvl) {
    Level& L = s.levels[lvl];
    // fill-in (ptree.cpp:866-871 get_sparsity, 140-153 alloc_fillin)
    for (int c : L.interiors)
      for (int e : b.in[c]) b.d2[c].insert(s.edges[e].n1);
    for (int c : L.interiors) {
      std::vector<int> front = b.out[c];
      for (int nb : b.d2[c]) {
        if (nb == c) continue;
        for (int e : front) {
          int x = s.edges[e].n2;
          if (s.find_edge(nb, x) < 0) b.add_edge(nb, x, lvl);
        }
      }
    }
    for (int c : L.interiors)
      for (int e : b.in[c])
        if (s.clusters[s.edges[e].n1].interior) {
          s.error = "two interiors of level " + std::to_string(lvl) + " are coupled";
          return -5;
        }
    // elimination lists
    L.self_edge_of.assign(L.count, -1);
    for (int o = L.first; o < L.first + L.count; ++o) L.self_edge_of[o - L.first] = s.find_edge(o, o);
    for (int c : L.interiors) {
      L.out_begin.push_back((int)L.out_edges.size());
      for (int e : b.out[c])
        if (s.edges[e].n2 != c) L.out_edges.push_back(e);
      L.out_end.push_back((int)L.out_edges.size());
      std::vector<int> ins = b.in[c];
      std::sort(ins.begin(), ins.end(), [&](int x, int y) { return s.edges[x].n1 < s.edges[y].n1; });
      L.in_begin.push_back((int)L.in_edges.size());
      L.in_edges.insert(L.in_edges.end(), ins.begin(), ins.end());
      L.in_end.push_back((int)L.in_edges.size());
    }
    // trailing updates grouped by column cluster (interiors ascending inside)
    {
      std::vector<std::vector<std::pair<int, int>>> bycol(L.count);
      for (size_t ii = 0; ii < L.interiors.size(); ++ii) {
        int c = L.interiors[ii];
        for (int e = L.in_begin[ii]; e < L.in_end[ii]; ++e) {
          int ecm = L.in_edges[e];
          bycol[s.edges[ecm].n1 - L.first].push_back({(int)ii, ecm});
        }
        (void)c;
      }
      for (int m = 0; m < L.count; ++m) {
        if (bycol[m].empty()) continue;
        L.col_m.push_back(L.first + m);
        L.col_begin.push_back((int)L.col_c.size());
        for (auto& pr : bycol[m]) {
          int ii = pr.first;
          int c = L.interiors[ii];
          L.col_c.push_back(c);
          L.col_ecm.push_back(pr.second);
          L.col_emn_begin.push_back((int)L.col_emn.size());
          for (int q = L.out_begin[ii]; q < L.out_end[ii]; ++q) {
            int nn = s.edges[L.out_edges[q]].n2;
            int emn = s.find_edge(L.first + m, nn);
            if (emn < 0) {
              s.error = "missing fill block at level " + std::to_string(lvl);
              return -6;
            }
            L.col_emn.push_back(emn);
          }
        }
        L.col_end.push_back((int)L.col_c.size());
      }
    }
    // sparsification lists
    for (int p : L.interfaces) {
      for (int e : b.out[p])
        if (s.edges[e].spars) L.spars_edges.push_back(e);
      if (!s.clusters[p].sparsify) continue;
      L.spars_clusters.push_back(p);
      std::vector<int> so, si;
      for (int e : b.out[p])
        if (s.edges[e].spars) so.push_back(e);
      for (int e : b.in[p])
        if (s.edges[e].spars) si.push_back(e);
      std::sort(so.begin(), so.end(), [&](int x, int y) { return s.edges[x].n2 < s.edges[y].n2; });
      std::sort(si.begin(), si.end(), [&](int x, int y) { return s.edges[x].n1 < s.edges[y].n1; });
      L.sp_out_begin.push_back((int)L.sp_out.size());
      L.sp_out.insert(L.sp_out.end(), so.begin(), so.end());
      L.sp_out_end.push_back((int)L.sp_out.size());
      L.sp_in_begin.push_back((int)L.sp_in.size());
      L.sp_in.insert(L.sp_in.end(), si.begin(), si.end());
      L.sp_in_end.push_back((int)L.sp_in.size());
    }
    if (lvl + 1 >= nlevels) break;
    // merge: parents' blocks (ptree.cpp:289-340)
    Level& N = s.levels[lvl + 1];
    for (int snew = N.first; snew < N.first + N.count; ++snew) {
      const Cluster& P = s.clusters[snew];
      std::set<int> nbrs;
      for (int k = P.child_begin; k < P.child_end; ++k) {
        int so = s.children[k];
        for (int e : b.out[so]) {
          int t = s.edges[e].n2;
          if (!s.clusters[t].interior) nbrs.insert(s.clusters[t].parent);
        }
        for (int d : b.d2[so])
          if (s.clusters[d].lvl >= lvl + 1) b.d2[snew].insert(s.clusters[d].parent);
      }
      for (int t : nbrs) b.add_edge(snew, t, lvl + 1);
      b.sort_out(snew);
    }
    for (int p : L.interfaces)
      for (int e : b.out[p]) {
        int t = s.edges[e].n2;
        if (s.clusters[t].interior) continue;
        L.merge_src.push_back(e);
        L.merge_dst.push_back(s.find_edge(s.clusters[p].parent, s.clusters[t].parent));
      }
  }
  return 0;
}

}  // namespace spq
