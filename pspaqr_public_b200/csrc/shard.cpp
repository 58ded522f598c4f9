// shard.cpp -- nested-dissection subtree sharding plan (shard.hpp).
#include "shard.hpp"

#include <set>
#include <tuple>

namespace spq {

int shard_owner(int section, int merge_lvl, int nlevels, int nranks) {
  int nparts_lvl = 1 << (nlevels - 1);
  for (int l = 0; l < merge_lvl; ++l) nparts_lvl /= 2;
  if (nparts_lvl > nranks) return section / (nparts_lvl / nranks);
  return section;
}

int build_shard_plan(const Structure& s, int nranks, ShardPlan& plan) {
  const int nparts = 1 << (s.nlevels - 1);
  if (nranks < 1 || (nranks & (nranks - 1)) != 0 || nranks > nparts) return -1;
  plan = ShardPlan();
  plan.nranks = nranks;
  const int ncl = (int)s.clusters.size();
  plan.cluster_owner.resize(ncl);
  for (int c = 0; c < ncl; ++c) {
    const Cluster& C = s.clusters[c];
    plan.cluster_owner[c] = shard_owner(C.id.section, C.merge_lvl, s.nlevels, nranks);
  }
  plan.edge_owner.resize(s.edges.size());
  for (size_t e = 0; e < s.edges.size(); ++e) plan.edge_owner[e] = plan.cluster_owner[s.edges[e].n1];
  // unknowns: the level-0 clusters hold contiguous permuted columns
  plan.row_owner.assign(s.n, 0);
  const Level& L0 = s.levels[0];
  for (int o = L0.first; o < L0.first + L0.count; ++o) {
    const int begin = s.clusters[o].cstart, end = begin + s.clusters[o].size0;
    for (int k = begin; k < end; ++k) plan.row_owner[k] = plan.cluster_owner[o];
  }
  plan.exchange.assign(s.nlevels, {});
  for (int l = 0; l < s.nlevels; ++l) {
    const Level& Lv = s.levels[l];
    auto& ex = plan.exchange[l];
    std::set<std::tuple<int, int, int>> seen;  // (kind, id, to)
    auto add = [&](int kind, int id, int dst, int from, int to) {
      if (from != to && seen.insert({kind, id, to}).second) ex.push_back({kind, id, dst, from, to});
    };
    const auto& own = plan.cluster_owner;
    // trailing updates: interior c modifies the blocks of column cluster m
    for (size_t ct = 0; ct < Lv.col_m.size(); ++ct) {
      const int m = Lv.col_m[ct];
      for (int q = Lv.col_begin[ct]; q < Lv.col_end[ct]; ++q) add(1, Lv.col_c[q], -1, own[Lv.col_c[q]], own[m]);
    }
    // scaling / compression applies on blocks A(n2, n1) between interfaces
    for (int e : Lv.spars_edges) {
      const Edge& E = s.edges[e];
      if (s.clusters[E.n2].sparsify) add(2, E.n2, -1, own[E.n2], own[E.n1]);
    }
    // compression matrices: the in-blocks A(p, m) of interface p
    for (size_t q = 0; q < Lv.spars_clusters.size(); ++q) {
      const int p = Lv.spars_clusters[q];
      for (int k = Lv.sp_in_begin[q]; k < Lv.sp_in_end[q]; ++k) {
        const int e = Lv.sp_in[k];
        add(3, e, -1, plan.edge_owner[e], own[p]);
      }
    }
    // merge into the next level
    for (size_t q = 0; q < Lv.merge_src.size(); ++q) {
      const int src = Lv.merge_src[q], dst = Lv.merge_dst[q];
      add(0, src, dst, plan.edge_owner[src], plan.edge_owner[dst]);
    }
  }
  return 0;
}

}  // namespace spq
