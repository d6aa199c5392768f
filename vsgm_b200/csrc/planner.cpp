// Query construction and the matching-order planner.
//
// Reproduces the reference's query semantics and its heuristic planner so that a
// plan built here drives the engine exactly as Plan::Optimize drives VSGM:
//   - preset patterns P0..P18           src/query/pattern.h:9-400
//   - k-cliques with the 0<1<..<k-1 chain src/query/clique.h:9-37
//   - generic adjacency queries          src/query/query.h:62-78
//   - connected k-graphlets              src/query/graphlet.h:15-136
//   - vertex re-mapping                  src/query/query.h:123-185
//   - symmetry-breaking partial orders   src/query/partial_order.h:96-144
//   - Plan::Optimize and its tables      src/query/plan.h:122-561
// Automorphisms are enumerated directly over all n! permutations (n <= 7) instead
// of calling bliss; the partial-order algorithm only needs the group as a set, so
// the conditions it derives are identical.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <queue>
#include <set>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "planner.hpp"

namespace vsgm {

namespace {

// ---------------------------------------------------------------------------
// preset patterns (adjacency as the reference lists them, before re-mapping)
// ---------------------------------------------------------------------------
struct PresetDef {
  int n;
  int m;
  std::vector<std::vector<int>> adj;
};

PresetDef preset(int p) {
  switch (p) {
    case 0:  // triangle
      return {3, 3, {{1, 2}, {0, 2}, {0, 1}}};
    case 1:  // square (4-cycle)
      return {4, 4, {{1, 3}, {0, 2}, {1, 3}, {0, 2}}};
    case 2:  // chordal square (diamond)
      return {4, 5, {{1, 2, 3}, {0, 2}, {0, 1, 3}, {0, 2}}};
    case 3:  // triangle with a 2-edge tail
      return {5, 5, {{1, 2}, {0, 2}, {0, 1, 3}, {2, 4}, {3}}};
    case 4:  // house
      return {5, 6, {{1, 2}, {0, 2, 3}, {0, 1, 4}, {1, 4}, {2, 3}}};
    case 5:  // chordal house
      return {5, 8, {{1, 2, 3, 4}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2, 4}, {0, 3}}};
    case 6:  // chordal roof
      return {5, 7, {{1, 2, 3}, {0, 2, 3}, {0, 1, 4}, {0, 1, 4}, {2, 3}}};
    case 7:  // three triangles sharing vertex 0
      return {5, 7, {{1, 2, 3, 4}, {0, 3, 2}, {0, 1, 4}, {0, 1}, {0, 2}}};
    case 8:  // solar square (wheel W4)
      return {5, 8, {{1, 2, 3, 4}, {0, 2, 4}, {0, 1, 3}, {0, 2, 4}, {0, 1, 3}}};
    case 9:  // near 5-clique
      return {5, 9, {{1, 2, 3, 4}, {0, 2, 3, 4}, {0, 1, 3}, {0, 1, 2, 4}, {0, 1, 3}}};
    case 10:  // four triangles (fan)
      return {6, 9, {{1, 2, 3, 4, 5}, {0, 2}, {0, 1, 3}, {0, 2, 4}, {0, 3, 5}, {0, 4}}};
    case 11:  // one triangle inside three
      return {6, 9, {{1, 2, 3, 5}, {0, 2, 3, 4}, {0, 1, 4, 5}, {0, 1}, {1, 2}, {0, 2}}};
    case 12:  // near 6-clique
      return {6, 11, {{1, 2}, {0, 2, 3, 4, 5}, {0, 1, 3, 4, 5}, {1, 2, 4}, {1, 2, 3, 5}, {1, 2, 4}}};
    case 13:  // square on top
      return {6, 8, {{1, 2}, {0, 3}, {0, 3, 4, 5}, {1, 2, 4, 5}, {2, 3}, {2, 3}}};
    case 14:  // near 7-clique
      return {7, 15, {{1, 2, 3, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 5}, {0, 1, 2, 4, 5, 6}, {0, 3, 5}, {0, 1, 2, 3, 4, 6}, {3, 5}}};
    case 15:  // 5-clique on top
      return {7, 14, {{1, 2, 3, 4}, {0, 2, 3, 4}, {0, 1, 3, 4}, {0, 1, 2, 4, 5, 6}, {0, 1, 2, 3, 5, 6}, {3, 4}, {3, 4}}};
    case 16:  // 5-cycle
      return {5, 5, {{1, 2}, {0, 3}, {0, 4}, {1, 4}, {2, 3}}};
    case 17:  // 6-cycle
      return {6, 6, {{1, 2}, {0, 3}, {0, 4}, {1, 5}, {2, 5}, {3, 4}}};
    case 18:  // hourglass / prism
      return {6, 9, {{1, 2, 4}, {0, 2, 5}, {0, 1, 3}, {2, 4, 5}, {0, 3, 5}, {1, 3, 4}}};
    default:
      return {0, 0, {}};
  }
}

using Adj = std::vector<std::vector<int>>;

// Relabel pattern vertices: BFS from the highest-degree vertex, each BFS level
// ordered by (degree desc, links into the explored region desc, id asc).
// Follows Query::ReMapVertexId (src/query/query.h:123-185), including the point at
// which "explored" is sampled: after the whole level has pushed its neighbours.
Adj remap_vertices(const Adj& adj) {
  const int n = (int)adj.size();
  int root = 0;
  size_t best = 0;
  for (int i = 0; i < n; i++)
    if (adj[i].size() > best) {
      best = adj[i].size();
      root = i;
    }
  std::vector<char> seen(n, 0);
  std::vector<int> relabel(n, 0);
  std::queue<int> frontier;
  frontier.push(root);
  seen[root] = 1;
  int next_id = 0;
  while (!frontier.empty()) {
    const size_t width = frontier.size();
    std::vector<int> level;
    for (size_t i = 0; i < width; i++) {
      int x = frontier.front();
      frontier.pop();
      level.push_back(x);
      for (int y : adj[x])
        if (!seen[y]) {
          seen[y] = 1;
          frontier.push(y);
        }
    }
    std::vector<std::tuple<size_t, size_t, int>> key;
    for (int x : level) {
      size_t links = 0;
      for (int y : adj[x]) links += seen[y] ? 1 : 0;
      key.emplace_back(adj[x].size(), links, x);
    }
    std::sort(key.begin(), key.end(), [](const auto& a, const auto& b) {
      if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) > std::get<0>(b);
      if (std::get<1>(a) != std::get<1>(b)) return std::get<1>(a) > std::get<1>(b);
      return std::get<2>(a) < std::get<2>(b);
    });
    for (auto& k : key) relabel[std::get<2>(k)] = next_id++;
  }
  Adj out(n);
  for (int i = 0; i < n; i++)
    for (int y : adj[i]) out[relabel[i]].push_back(relabel[y]);
  for (auto& row : out) std::sort(row.begin(), row.end());
  return out;
}

// All automorphisms of a small simple graph, by enumeration of permutations.
std::vector<std::vector<int>> automorphisms(const Adj& adj) {
  const int n = (int)adj.size();
  std::vector<uint32_t> bits(n, 0);
  for (int i = 0; i < n; i++)
    for (int y : adj[i]) bits[i] |= 1u << y;
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  std::vector<std::vector<int>> group;
  do {
    bool ok = true;
    for (int i = 0; i < n && ok; i++) {
      uint32_t img = 0;
      for (int y = 0; y < n; y++)
        if (bits[i] >> y & 1) img |= 1u << perm[y];
      ok = (img == bits[perm[i]]);
    }
    if (ok) group.push_back(perm);
  } while (std::next_permutation(perm.begin(), perm.end()));
  return group;
}

std::map<int, std::set<int>> orbits(const std::vector<std::vector<int>>& group, int n) {
  std::map<int, std::set<int>> out;
  for (int i = 0; i < n; i++) {
    std::set<int> orb;
    for (auto& g : group) orb.insert(g[i]);
    if (orb.empty()) continue;
    out[*orb.begin()].insert(orb.begin(), orb.end());
  }
  return out;
}

// Symmetry-breaking pairs (a, b) meaning a < b, following
// PartialOrder::GetConditions (src/query/partial_order.h:96-144): repeatedly take
// the first non-trivial orbit, pin its smallest member n0 against, for every
// group element, the orbit member it maps lowest, then restrict to the stabiliser
// of n0.
std::vector<std::pair<int, int>> symmetry_pairs(const Adj& adj) {
  const int n = (int)adj.size();
  auto group = automorphisms(adj);
  std::vector<std::pair<int, int>> pairs;
  auto nontrivial = [](const std::map<int, std::set<int>>& o) {
    for (auto it = o.begin(); it != o.end(); ++it)
      if (it->second.size() > 1) return it;
    return o.end();
  };
  auto orb = orbits(group, n);
  auto it = nontrivial(orb);
  while (it != orb.end()) {
    const std::set<int> cls = it->second;
    const int n0 = *cls.begin();
    for (auto& g : group) {
      int best = -1;
      for (auto m = std::next(cls.begin()); m != cls.end(); ++m)
        if (best < 0 || g[*m] < g[best]) best = *m;
      pairs.emplace_back(n0, best);
    }
    group.erase(std::remove_if(group.begin(), group.end(), [n0](const std::vector<int>& g) { return g[n0] != n0; }), group.end());
    orb = orbits(group, n);
    it = nontrivial(orb);
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  return pairs;
}

bool connected(const Adj& adj) {
  const int n = (int)adj.size();
  if (n == 0) return false;
  std::vector<char> seen(n, 0);
  std::vector<int> stack{0};
  seen[0] = 1;
  while (!stack.empty()) {
    int x = stack.back();
    stack.pop_back();
    for (int y : adj[x])
      if (!seen[y]) {
        seen[y] = 1;
        stack.push_back(y);
      }
  }
  for (char s : seen)
    if (!s) return false;
  return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// Query
// ---------------------------------------------------------------------------
Query Query::from_adjacency(const Adj& adj, int n_edges) {
  Query q;
  q.adj = remap_vertices(adj);
  q.n_edges = n_edges;
  const int n = (int)q.adj.size();
  q.cond.assign(n, std::vector<uint8_t>(n, VSGM_NON_EQUAL));
  for (auto& pr : symmetry_pairs(q.adj)) {
    q.cond[pr.first][pr.second] = VSGM_LESS_THAN;
    q.cond[pr.second][pr.first] = VSGM_LARGER_THAN;
  }
  return q;
}

bool Query::preset(int p, Query* out) {
  PresetDef d = vsgm::preset(p);
  if (d.n == 0) return false;
  *out = from_adjacency(d.adj, d.m);
  return true;
}

bool Query::clique(int k, Query* out) {
  if (k < 3 || k > VSGM_MAX_QV) return false;
  Query q;
  q.adj.assign(k, {});
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++)
      if (i != j) q.adj[i].push_back(j);
  q.n_edges = k * (k - 1) / 2;
  // the hard-coded chain of Clique (src/query/clique.h:31-36): only consecutive
  // vertices carry an order, every other pair defaults to NON_EQUAL
  q.cond.assign(k, std::vector<uint8_t>(k, VSGM_NON_EQUAL));
  for (int i = 0; i + 1 < k; i++) {
    q.cond[i][i + 1] = VSGM_LESS_THAN;
    q.cond[i + 1][i] = VSGM_LARGER_THAN;
  }
  *out = q;
  return true;
}

bool Query::from_bits(int n, const uint8_t* bits, Query* out) {
  if (n < 2 || n > VSGM_MAX_QV) return false;
  Adj adj(n);
  int m = 0;
  for (int i = 0; i < n; i++) {
    if (bits[i] >> i & 1) return false;
    for (int j = 0; j < n; j++)
      if (bits[i] >> j & 1) {
        if (!(bits[j] >> i & 1)) return false;
        adj[i].push_back(j);
        if (i < j) m++;
      }
  }
  if (!connected(adj)) return false;
  *out = from_adjacency(adj, m);
  return true;
}

// Connected graphlets of k vertices, in the order Graphlet::GenerateAll
// (src/query/graphlet.h:48-122) produces them: remove e = 0.. edges from the
// k-clique, combinations in lexicographic order, keep the first connected member
// of every isomorphism class.  The reference removes the combination's indices
// one after another from a shrinking list, so later indices address shifted
// positions, and an index at or past the end drops the last edge; both are
// reproduced here.
std::vector<Query> Query::graphlets(int k) {
  std::vector<Query> out;
  if (k < 3 || k > 5) return out;
  std::vector<std::pair<int, int>> all_edges;
  for (int v = 0; v < k; v++)
    for (int u = 0; u < k; u++)
      if (v < u) all_edges.emplace_back(v, u);
  const int m_full = (int)all_edges.size();
  auto build = [&](const std::vector<std::pair<int, int>>& el) {
    Adj adj(k);
    for (auto& e : el) {
      adj[e.first].push_back(e.second);
      adj[e.second].push_back(e.first);
    }
    return adj;
  };
  auto canon = [&](const Adj& adj) {
    // smallest adjacency bit-string over all relabelings
    std::vector<int> perm(k);
    for (int i = 0; i < k; i++) perm[i] = i;
    uint64_t best = ~0ull;
    do {
      uint64_t code = 0;
      for (int i = 0; i < k; i++)
        for (int y : adj[i]) code |= 1ull << (perm[i] * k + perm[y]);
      best = std::min(best, code);
    } while (std::next_permutation(perm.begin(), perm.end()));
    return best;
  };
  std::vector<std::pair<Adj, int>> kept;
  for (int e = 0; e <= m_full - (k - 1); e++) {
    if (e == 0) {
      kept.emplace_back(build(all_edges), m_full);
      continue;
    }
    std::vector<int> comb(e);
    for (int i = 0; i < e; i++) comb[i] = i;
    std::vector<uint64_t> classes;
    bool first_connected = true;
    while (true) {
      std::vector<std::pair<int, int>> el = all_edges;
      for (int idx : comb) {
        if (idx >= (int)el.size())
          el.pop_back();
        else
          el.erase(el.begin() + idx);
      }
      Adj adj = build(el);
      if (connected(adj)) {
        uint64_t c = canon(adj);
        if (first_connected) {
          kept.emplace_back(adj, (int)el.size());
          classes.push_back(c);
          first_connected = false;
        } else if (std::find(classes.begin(), classes.end(), c) == classes.end()) {
          kept.emplace_back(adj, (int)el.size());
          classes.push_back(c);
        }
      }
      // next combination
      int i = e - 1;
      while (i >= 0 && comb[i] == m_full - e + i) i--;
      if (i < 0) break;
      comb[i]++;
      for (int j = i + 1; j < e; j++) comb[j] = comb[j - 1] + 1;
    }
  }
  for (auto& kv : kept) out.push_back(from_adjacency(kv.first, kv.second));
  return out;
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
namespace {

// BFS depth from u, plus one if the deepest level has an internal edge
// (Plan::GetMinHopWithBFS, src/query/plan.h:156-183).
int min_hop(const Adj& adj, int root) {
  const int n = (int)adj.size();
  std::vector<int> level(n, -1);
  std::queue<int> q;
  q.push(root);
  level[root] = 0;
  int deepest = -1, intra = -1;
  while (!q.empty()) {
    int x = q.front();
    q.pop();
    deepest = level[x];
    for (int y : adj[x]) {
      if (level[y] < 0) {
        level[y] = level[x] + 1;
        q.push(y);
      } else if (level[y] == level[x]) {
        intra = level[y];
      }
    }
  }
  return deepest + (deepest == intra ? 1 : 0);
}

struct Op {
  uint8_t type;
  uint8_t v;
};

}  // namespace

bool build_plan(const Query& q, const int* custom_seq, vsgm_plan* out, std::string* err) {
  const int n = (int)q.adj.size();
  if (n < 2 || n > VSGM_MAX_QV) {
    if (err) *err = "pattern must have 2..7 vertices";
    return false;
  }
  std::memset(out, 0, sizeof(*out));

  // 1. root: least hop, ties to the higher degree (Plan::FindRoot, plan.h:185-208)
  int root = 0, hop = 10;
  size_t root_deg = 0;
  for (int u = 0; u < n; u++) {
    int h = min_hop(q.adj, u);
    if (h < hop || (h == hop && root_deg < q.adj[u].size())) {
      root = u;
      hop = h;
      root_deg = q.adj[u].size();
    }
  }

  // 2. search sequence: (hop asc, degree desc, id asc) from the root
  //    (Plan::GenerateSearchSequence, plan.h:210-265)
  std::vector<int> seq;
  if (custom_seq) {
    std::vector<char> used(n, 0);
    for (int i = 0; i < n; i++) {
      int u = custom_seq[i];
      if (u < 0 || u >= n || used[u]) {
        if (err) *err = "custom sequence is not a permutation";
        return false;
      }
      used[u] = 1;
      seq.push_back(u);
    }
    // every later vertex needs a neighbour earlier in the sequence
    for (int i = 1; i < n; i++) {
      bool linked = false;
      for (int y : q.adj[seq[i]])
        for (int j = 0; j < i; j++) linked |= (seq[j] == y);
      if (!linked) {
        if (err) *err = "custom sequence has a vertex without a backward neighbour";
        return false;
      }
    }
    // the view halo must cover the chosen root
    root = seq[0];
    hop = min_hop(q.adj, root);
    root_deg = q.adj[root].size();
  } else {
    std::vector<std::tuple<int, int, int>> key(n);
    std::vector<int> depth(n, -1);
    std::queue<int> bfs;
    bfs.push(root);
    depth[root] = 0;
    while (!bfs.empty()) {
      int x = bfs.front();
      bfs.pop();
      for (int y : q.adj[x])
        if (depth[y] < 0) {
          depth[y] = depth[x] + 1;
          bfs.push(y);
        }
    }
    for (int u = 0; u < n; u++) key[u] = std::make_tuple(depth[u], (int)q.adj[u].size(), u);
    std::sort(key.begin(), key.end(), [](const auto& a, const auto& b) {
      if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) < std::get<0>(b);
      if (std::get<1>(a) != std::get<1>(b)) return std::get<1>(a) > std::get<1>(b);
      return std::get<2>(a) < std::get<2>(b);
    });
    for (auto& k : key) seq.push_back(std::get<2>(k));
  }

  // 3. backward connectivity (plan.h:267-290), in adjacency order
  std::vector<std::vector<int>> back(n);
  {
    std::vector<char> before(n, 0);
    for (int u : seq) {
      for (int y : q.adj[u])
        if (before[y]) back[u].push_back(y);
      before[u] = 1;
    }
  }

  // 4. compute sequence with lazy materialisation (plan.h:292-318)
  std::vector<Op> ops;
  {
    std::vector<char> mat(n, 0);
    ops.push_back({VSGM_MATERIALIZE, (uint8_t)seq[0]});
    mat[seq[0]] = 1;
    for (int i = 1; i < n; i++) {
      int u = seq[i];
      for (int p : back[u])
        if (!mat[p]) {
          ops.push_back({VSGM_MATERIALIZE, (uint8_t)p});
          mat[p] = 1;
        }
      ops.push_back({VSGM_COMPUTE, (uint8_t)u});
    }
  }

  // 5. the counting tail (plan.h:329-430)
  auto index_of = [&](uint8_t type, int u) {
    for (size_t i = 0; i < ops.size(); i++)
      if (ops[i].type == type && ops[i].v == u) return i;
    return ops.size();
  };
  auto tail_two = [&](const std::vector<int>& um, const std::vector<bool>& nf) -> bool {
    if (nf[0] && nf[1]) {
      ops.push_back({VSGM_FILTER_COMPUTE, (uint8_t)um[0]});
      ops.push_back({VSGM_FILTER_COMPUTE, (uint8_t)um[1]});
      ops.push_back({VSGM_COUNT, (uint8_t)n});
    } else if (!nf[0] && !nf[1]) {
      size_t i0 = ops.size(), i1 = ops.size();
      for (int j = (int)ops.size() - 1; j >= 0; --j) {
        if (ops[j].v == um[0]) i0 = j;
        if (ops[j].v == um[1]) i1 = j;
      }
      size_t last = std::max(i0, i1);
      if (last != ops.size() - 1) return false;
      ops[last].type = VSGM_COMPUTE_COUNT;
    } else {
      int f = nf[0] ? um[0] : um[1];
      int c = nf[0] ? um[1] : um[0];
      size_t at = index_of(VSGM_COMPUTE, c);
      ops.erase(ops.begin() + at);
      ops.push_back({VSGM_FILTER_COMPUTE, (uint8_t)f});
      ops.push_back({VSGM_COMPUTE_COUNT, (uint8_t)c});
    }
    return true;
  };
  {
    std::vector<char> mat(n, 0);
    for (auto& o : ops)
      if (o.type == VSGM_MATERIALIZE) mat[o.v] = 1;
    std::vector<int> um;
    std::vector<bool> nf;
    for (int u = 0; u < n; u++)
      if (!mat[u]) {
        um.push_back(u);
        size_t at = index_of(VSGM_COMPUTE, u);
        bool later = false;
        for (size_t i = at + 1; i < ops.size(); i++) later |= (ops[i].type == VSGM_MATERIALIZE);
        nf.push_back(later);
      }
    bool ok = true;
    if (um.size() == 1) {
      if (nf[0]) {
        ops.push_back({VSGM_FILTER_COMPUTE, (uint8_t)um[0]});
        ops.push_back({VSGM_COUNT, (uint8_t)n});
      } else {
        ok = (ops.back().type == VSGM_COMPUTE && ops.back().v == um[0]);
        ops.back().type = VSGM_COMPUTE_COUNT;
      }
    } else if (um.size() == 2) {
      ok = tail_two(um, nf);
    } else if (um.size() > 2) {
      for (size_t i = 2; i < um.size(); i++) ops.push_back({VSGM_MATERIALIZE, (uint8_t)um[i]});
      ok = tail_two({um[0], um[1]}, {true, true});
    } else {
      ok = false;
    }
    if (!ok) {
      if (err) *err = "planner invariant violated while building the counting tail";
      return false;
    }
  }
  if (ops.size() > VSGM_MAX_OPS) {
    if (err) *err = "execution sequence too long";
    return false;
  }

  // 6. per-op vertex groups (plan.h:432-452)
  {
    std::vector<char> mat(n, 0);
    std::vector<int> mats, comps;
    for (size_t i = 0; i < ops.size(); i++) {
      vsgm_vgroup& mg = out->materialized[i];
      vsgm_vgroup& cg = out->computed_unmat[i];
      for (int u : mats) mg.v[mg.count++] = (uint8_t)u;
      for (int u : comps)
        if (!mat[u]) cg.v[cg.count++] = (uint8_t)u;
      if (ops[i].type == VSGM_COMPUTE || ops[i].type == VSGM_COMPUTE_PATH_COUNT) {
        comps.push_back(ops[i].v);
      } else if (ops[i].type == VSGM_MATERIALIZE) {
        mats.push_back(ops[i].v);
        mat[ops[i].v] = 1;
      }
    }
  }

  // condition tables (plan.h:460-528)
  {
    std::vector<int> mats;
    for (size_t i = 0; i < ops.size(); i++) {
      const uint8_t t = ops[i].type;
      const int u = ops[i].v;
      if (t == VSGM_COMPUTE || t == VSGM_COMPUTE_COUNT || t == VSGM_COMPUTE_PATH_COUNT) {
        vsgm_conds& c = out->compute_cond[u];
        c.count = 0;
        for (int p : mats) {
          c.op[c.count] = q.cond[u][p];
          c.v[c.count++] = (uint8_t)p;
        }
      } else if (t == VSGM_MATERIALIZE) {
        mats.push_back(u);
      }
      if (t == VSGM_MATERIALIZE || t == VSGM_FILTER_COMPUTE) {
        // vertices materialised after u was computed, newest first
        vsgm_conds& c = (t == VSGM_MATERIALIZE) ? out->materialize_cond[u] : out->filter_cond[u];
        c.count = 0;
        for (int j = (int)i - 1; j >= 0; --j) {
          if (ops[j].type == VSGM_COMPUTE && ops[j].v == u) break;
          if (ops[j].type == VSGM_MATERIALIZE) {
            int p = ops[j].v;
            c.op[c.count] = q.cond[u][p];
            c.v[c.count++] = (uint8_t)p;
          }
        }
      }
    }
  }

  out->n_vertices = (uint32_t)n;
  out->n_edges = (uint32_t)q.n_edges;
  out->hop = hop;
  out->root_degree = (uint32_t)root_deg;
  out->root = (uint32_t)seq[0];
  out->n_ops = (uint32_t)ops.size();
  for (int i = 0; i < n; i++) {
    out->seq[i] = (uint8_t)seq[i];
    for (int y : q.adj[i]) out->adj[i] |= (uint8_t)(1u << y);
    for (int j = 0; j < n; j++) out->order[i][j] = (i == j) ? (uint8_t)VSGM_OPERATOR_NONE : q.cond[i][j];
    vsgm_vgroup& b = out->backward[i];
    for (int p : back[i]) b.v[b.count++] = (uint8_t)p;
  }
  for (size_t i = 0; i < ops.size(); i++) {
    out->op_type[i] = ops[i].type;
    out->op_vertex[i] = ops[i].v;
  }
  return true;
}

uint64_t automorphism_count(const vsgm_plan& p) {
  Adj adj(p.n_vertices);
  for (uint32_t i = 0; i < p.n_vertices; i++)
    for (uint32_t j = 0; j < p.n_vertices; j++)
      if (p.adj[i] >> j & 1) adj[i].push_back((int)j);
  return automorphisms(adj).size();
}

}  // namespace vsgm
