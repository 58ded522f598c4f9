// structure.hpp -- host-side partition and symbolic factorization of the
// pspaQR tree (square systems, tensor-grid / coordinate nested dissection).
//
// Everything here is integer work done once on the host: the geometric
// nested-dissection ordering (partition.cpp:241-350, 514-587 of the
// reference), the cluster hierarchy (ptree.cpp:587-691), the level-0 blocks
// and their distance-2 connections (ptree.cpp:703-864), and the block
// structure of every later level: fill-in (ptree.cpp:101-153, 866-1010) and
// the merge into parent clusters (ptree.cpp:289-340, 1940-2123).  The block
// STRUCTURE of all levels is independent of the ranks chosen by the
// sparsification, so it is built before any numerics; only block SIZES depend
// on ranks and are resolved level by level on the device side.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace spq {

struct SepID {
  int lvl = -1, sep = 0;
  SepID() = default;
  SepID(int l, int s) : lvl(l), sep(s) {}
  bool operator==(const SepID& o) const { return lvl == o.lvl && sep == o.sep; }
  bool operator!=(const SepID& o) const { return !(*this == o); }
  bool operator<(const SepID& o) const { return lvl < o.lvl || (lvl == o.lvl && sep < o.sep); }
};

// Cluster identity (cluster.h:61-135).  Ordering: self, l, r, section, part.
struct ClusterID {
  SepID self, l, r;
  int part = 2, section = 0;
  bool operator==(const ClusterID& o) const {
    return self == o.self && l == o.l && r == o.r && part == o.part && section == o.section;
  }
  bool operator!=(const ClusterID& o) const { return !(*this == o); }
  bool operator<(const ClusterID& o) const;
};
ClusterID merge_if(const ClusterID& c, int lvl);

// Compressed sparse column matrix, 0-based, sorted row indices.
struct Csc {
  int nrows = 0, ncols = 0;
  std::vector<int> colptr, rowidx;
  std::vector<double> val;
};

// One node of the cluster hierarchy.  Orders are global, assigned level by
// level in creation order (Tree::get_new_order), so the clusters of one level
// have consecutive orders.
struct Cluster {
  ClusterID id;
  int lvl = 0;        // separator level (id.self.lvl)
  int merge_lvl = 0;  // hierarchy level this cluster lives on
  bool interior = false;  // eliminated at merge_lvl (lvl == merge_lvl)
  bool sparsify = false;  // want_sparsify (ptree.cpp:29-41)
  int parent = -1;
  int child_begin = 0, child_end = 0;  // range in Structure::children
  int cstart = 0;     // first permuted column (leaves: exact; parents: first child's)
  int size0 = 0;      // uncompressed size (sum of leaf sizes below)
};

// Block A(rows of n2, cols of n1) at one level.
struct Edge {
  int n1 = 0, n2 = 0;
  int level = 0;
  bool spars = false;  // both ends are interfaces of the level, n1 != n2
};

// Per-level symbolic lists.
struct Level {
  int first = 0, count = 0;         // cluster orders [first, first+count)
  std::vector<int> interiors, interfaces;
  std::vector<int> edges;            // all edges living on this level
  // elimination (per interior, ascending order)
  std::vector<int> self_edge_of;     // indexed by cluster order - first
  std::vector<int> out_begin, out_end;  // per interior: range in out_edges (sorted by n2, self excluded)
  std::vector<int> out_edges;
  // trailing update, grouped by column cluster m: list of (interior c, edge m->c)
  std::vector<int> col_m, col_begin, col_end;  // per column task
  std::vector<int> col_c, col_ecm;             // entries
  std::vector<int> col_emn;                    // per entry, aligned with c's out-edges (size = deg(c))
  std::vector<int> col_emn_begin;              // per entry: start in col_emn
  // interiors' row blocks (edges m -> c), per interior, sorted by m (backward solve)
  std::vector<int> in_begin, in_end, in_edges;
  // sparsification
  std::vector<int> spars_clusters;   // interfaces with want_sparsify
  std::vector<int> spars_edges;      // edges between interfaces (n1 != n2)
  std::vector<int> sp_out_begin, sp_out_end, sp_out;  // per spars cluster, sorted by n2
  std::vector<int> sp_in_begin, sp_in_end, sp_in;     // per spars cluster, sorted by n1
  // merge into the next level: each surviving edge maps to a parent edge
  std::vector<int> merge_src, merge_dst;   // child edge -> parent edge (next level)
};

struct Structure {
  int n = 0, nlevels = 0, skip = 0;
  double tol = 0;
  std::vector<int> cperm, rperm;   // permuted index k holds original column cperm[k]
  std::vector<ClusterID> cpermed;
  std::vector<Cluster> clusters;
  std::vector<int> children;
  std::vector<Edge> edges;
  std::vector<Level> levels;
  std::unordered_map<uint64_t, int> edge_of;
  Csc App;                          // A[rperm, cperm]
  std::string error;

  int find_edge(int n1, int n2) const;
};

// Geometric nested dissection on A^T A (partition.cpp:282-350) followed by the
// interface classification of getInterfacesUsingA (partition.cpp:514-587).
// X: coordinates, dim x n column-major.  Returns cmap (one ClusterID per column).
std::vector<ClusterID> geometric_partition(const Csc& A, int nlevels, const std::vector<double>& X, int dim);

// Build ordering, hierarchy and the symbolic structure of every level.
// Returns 0 or a negative status (message in s.error).
int build_structure(Structure& s, const Csc& A, int nlevels, int skip, double tol, const std::vector<double>& X,
                    int dim);

}  // namespace spq
