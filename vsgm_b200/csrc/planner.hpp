// Query construction and the heuristic planner (host side).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vsgm_plan.h"

namespace vsgm {

// A pattern after vertex re-mapping, with its pairwise condition table
// (cond[i][j] == GetConditionType(i, j) of the reference query).
struct Query {
  std::vector<std::vector<int>> adj;
  std::vector<std::vector<uint8_t>> cond;
  int n_edges = 0;

  static Query from_adjacency(const std::vector<std::vector<int>>& adj, int n_edges);
  static bool preset(int p, Query* out);                     // Pattern((PresetPatternType)p, false)
  static bool clique(int k, Query* out);                     // Clique(k)
  static bool from_bits(int n, const uint8_t* bits, Query* out);  // Query(n, e, adj)
  static std::vector<Query> graphlets(int k);                // Graphlet(k)->GetQueries()
};

// Plan::Optimize; with custom_seq != nullptr the search sequence is taken from
// the caller (any order whose every later vertex has an earlier neighbour) and
// every downstream table is derived from it exactly as Optimize derives them.
bool build_plan(const Query& q, const int* custom_seq, vsgm_plan* out, std::string* err);

// |Aut(P)| of the planned pattern.
uint64_t automorphism_count(const vsgm_plan& p);

}  // namespace vsgm
