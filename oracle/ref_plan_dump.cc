// Test infrastructure, not product code: a driver compiled against the
// reference's own planner headers (src/query/*.h) and bliss 0.73 sources, which
// prints the reference's plans as JSON lines so that the product planner can be
// pinned to them.  Built into oracle/_ref/ by oracle/Makefile; never linked into
// the library.
//
// usage: ref_plan_dump -p <id> | -kc <k> | -km <k> | -stdin
//   -stdin reads lines "n a00a01..a0n-1 a10..." (adjacency matrix as 0/1 digits)
//   and plans each with the generic Query(n, e, adj) constructor
//   (src/query/query.h:62-78).
#include <algorithm>  // the reference headers rely on a transitive include of this
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "query/clique.h"
#include "query/graphlet.h"
#include "query/pattern.h"
#include "query/plan.h"
#include "query/query.h"

static std::string groups(const MultiVTGroup& g) {
  std::ostringstream s;
  s << "[";
  for (size_t i = 0; i < g.size(); i++) {
    s << (i ? "," : "") << "[";
    for (size_t j = 0; j < g[i].size(); j++) s << (j ? "," : "") << g[i][j];
    s << "]";
  }
  s << "]";
  return s.str();
}

static std::string conds(const AllCondType& c, size_t n) {
  std::ostringstream s;
  s << "[";
  for (size_t i = 0; i < n; i++) {
    s << (i ? "," : "") << "[";
    if (i < c.size())
      for (size_t j = 0; j < c[i].size(); j++) s << (j ? "," : "") << "[" << (int)c[i][j].first << "," << c[i][j].second << "]";
    s << "]";
  }
  s << "]";
  return s.str();
}

static void dump(const std::string& name, Query* q) {
  Plan plan(q);
  plan.Optimize();
  size_t n = q->GetVertexCount();
  AllConnType& conn = q->GetConnectivity();
  AllCondType& order = q->GetOrder();
  std::ostringstream s;
  s << "{\"name\":\"" << name << "\",\"n\":" << n << ",\"edges\":" << q->GetEdgeCount();
  s << ",\"adj\":" << groups(conn);
  s << ",\"order\":[";
  for (size_t i = 0; i < n; i++) {
    s << (i ? "," : "") << "[";
    for (size_t j = 0; j < n; j++) s << (j ? "," : "") << (i == j ? 3 : (int)GetConditionType(i, j, order));
    s << "]";
  }
  s << "]";
  s << ",\"hop\":" << plan.GetHop() << ",\"root_degree\":" << plan.GetRootDegree();
  s << ",\"exec\":[";
  auto& ex = plan.GetExecuteOperations();
  for (size_t i = 0; i < ex.size(); i++) s << (i ? "," : "") << "[" << (int)ex[i].first << "," << ex[i].second << "]";
  s << "]";
  s << ",\"backward\":" << groups(plan.GetBackwardConnectivity());
  s << ",\"materialized\":" << groups(plan.GetMaterializedVertices());
  s << ",\"computed_unmat\":" << groups(plan.GetComputedUnmaterializedVertices());
  AllCondType cc, mc, fc;
  plan.GetComputeCondition(cc);
  plan.GetMaterializeCondition(mc);
  plan.GetFilterCondition(fc);
  s << ",\"compute_cond\":" << conds(cc, n);
  s << ",\"materialize_cond\":" << conds(mc, n);
  s << ",\"filter_cond\":" << conds(fc, n);
  s << "}";
  std::cout << s.str() << std::endl;
}

int main(int argc, char** argv) {
  // keep the reference's own progress prints off stdout
  std::streambuf* real = std::cout.rdbuf();
  std::ostringstream sink;
  if (argc < 2) return 1;
  std::string mode = argv[1];
  if (mode == "-p" && argc > 2) {
    std::cout.rdbuf(sink.rdbuf());
    Query* q = new Pattern((PresetPatternType)atoi(argv[2]), false);
    std::cout.rdbuf(real);
    dump(std::string("p") + argv[2], q);
  } else if (mode == "-kc" && argc > 2) {
    Query* q = new Clique(atoi(argv[2]));
    dump(std::string("kc") + argv[2], q);
  } else if (mode == "-km" && argc > 2) {
    std::cout.rdbuf(sink.rdbuf());
    Graphlet* g = new Graphlet(atoi(argv[2]));
    std::cout.rdbuf(real);
    auto& qs = g->GetQueries();
    for (size_t i = 0; i < qs.size(); i++) dump(std::string("km") + argv[2] + "_" + std::to_string(i), qs[i]);
  } else if (mode == "-stdin") {
    std::string line;
    int idx = 0;
    while (std::getline(std::cin, line)) {
      if (line.empty()) continue;
      std::istringstream in(line);
      int n;
      std::string bits;
      in >> n >> bits;
      std::vector<std::vector<int>> adj(n);
      size_t m = 0;
      for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
          if (bits[i * n + j] == '1') {
            adj[i].push_back(j);
            if (i < j) m++;
          }
      Query* q = new Query(n, m, adj);
      dump("rand" + std::to_string(idx++), q);
    }
  } else {
    return 1;
  }
  return 0;
}
