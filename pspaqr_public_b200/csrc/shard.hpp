// shard.hpp -- nested-dissection subtree sharding of the tree over ranks (one
// GPU per rank): which rank owns each cluster, each unknown and each block,
// and the blocks that cross ranks when a level is merged into the next.
//
// The mapping restates the reference's ParTree::get_rank / cluster2rank /
// edge2rank (ptree.cpp:65-91): at merge level l there are nparts / 2^l
// sections; with more sections than ranks each rank owns a contiguous run of
// sections, otherwise section s belongs to rank s.  Leaves are therefore
// block-distributed and the top log2(nranks) levels sit on fewer ranks (the
// root on rank 0).  A block A(n2, n1) lives with the owner of its column
// cluster n1 (edge2rank).  After a level's sparsification its surviving
// blocks are merged into the parent blocks of the next level
// (compute_new_edges, ptree.cpp:289-340); a block whose parent block has
// another owner is sent there (send_edge_am, ptree.cpp:2005-2038) -- the one
// data exchange per level.
#pragma once
#include <vector>

#include "structure.hpp"

namespace spq {

// get_rank(part, mergelvl) of ptree.cpp:65-79 for 2^(nlevels-1) leaf parts.
int shard_owner(int section, int merge_lvl, int nlevels, int nranks);

// One transfer between ranks at a level.
//   kind 0: merge -- child block `id` (edge) into parent block `dst` (edge of
//           level + 1) owned elsewhere (send_edge_am, ptree.cpp:2005-2038);
//   kind 1: elimination factors -- the reflectors of interior cluster `id`
//           (diagonal QR and tsqrt chain) to the owner of a column cluster its
//           trailing updates modify (ptree.cpp:1081-1098, 1419-1441);
//   kind 2: interface factors -- the scaling and sparsification reflectors of
//           interface `id` to the owner of a neighbour block they are applied
//           to (ptree.cpp:1500-1531, 1662-1693);
//   kind 3: compression gather -- block `id` (edge A(p, m)) to the owner of
//           interface p, whose compression matrix takes its rows
//           (ptree.cpp:373-439).
// Each (kind, id, to) appears once.
struct ShardExchange {
  int kind, id, dst;
  int from, to;  // ranks
};

struct ShardPlan {
  int nranks = 1;
  std::vector<int> cluster_owner;  // per cluster order
  std::vector<int> edge_owner;     // per edge (owner of its column cluster)
  std::vector<int> row_owner;      // per permuted unknown (owner of its leaf cluster)
  std::vector<std::vector<ShardExchange>> exchange;  // per level: transfers crossing ranks
};

// Returns 0, or -1 when nranks is not a power of two or exceeds the number of
// leaf parts.
int build_shard_plan(const Structure& s, int nranks, ShardPlan& plan);

}  // namespace spq
