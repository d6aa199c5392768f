// CPU ORACLE - test infrastructure only.
//
// Nothing in the product links, imports or executes this file.  It restates the
// reference's offline view-bin tools, single-threaded and in the reference's own
// loop order, so that tests can check them without the reference's binaries:
//
//   oracle_kmeans        cosine k-means with the random initialisation
//                        (src/tools/kmeans.cc:125-141 RandomInit, :171-196
//                        UpdateAllCentroids, :198-221 UpdateAssignment(s),
//                        :386-486 Run over one level, :452-471 the -rc renumbering,
//                        :491-510 RemoveEmptyClusters; the similarity and centroid
//                        arithmetic of src/tools/kmeans_utils.h:40-160)
//   oracle_view_packing  next-fit view-bin packing with one open bin per sequence
//                        (src/tools/view_bin.h:22-138 GetKHopViewSize,
//                        FindOneAndInsert, CreateOrSwapOne; the merge of
//                        src/tools/view_packing.cc:247-280)
//
// The reference sorts with std::sort where ties are possible (the -rc order, the
// merge by bin size); this file calls std::sort on the same sequences with the same
// comparisons, so equal keys end in the reference's order.  Built with
// -ffp-contract=off: every multiply and add is rounded on its own, as in the
// reference's build on a target without fused multiply-add.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <utility>
#include <vector>

namespace {

struct Rows {
  const uint64_t* rp;
  const uint32_t* ci;
  uint64_t deg(uint32_t v) const { return rp[v + 1] - rp[v]; }
};

// UpdateAllCentroids: per cluster, the members in increasing id add
// sqrt(1 / deg) to the entries of their rows; divide by the size; squared norm
void centroids(const Rows& g, uint64_t V, int K, const std::vector<int>& assign, std::vector<std::vector<double>>& cen, std::vector<int>& size,
               std::vector<double>& sqr) {
  std::vector<std::vector<uint32_t>> members(K);
  for (uint64_t v = 0; v < V; v++) members[assign[v]].push_back((uint32_t)v);
  for (int p = 0; p < K; p++) {
    std::fill(cen[p].begin(), cen[p].end(), 0.0);
    size[p] = 0;
    for (uint32_t v : members[p]) {
      const double r = std::sqrt(1. / (double)g.deg(v));
      for (uint64_t i = g.rp[v]; i < g.rp[v + 1]; i++) cen[p][g.ci[i]] += r;
      size[p]++;
    }
    if (size[p] > 0)
      for (double& x : cen[p]) x /= size[p];
    double s = 0;
    for (double x : cen[p]) s += x * x;
    sqr[p] = s;
  }
}

// CosineSimilarity against a dense centroid; the first strictly most similar wins
int assignment_of(const Rows& g, uint32_t v, int K, const std::vector<std::vector<double>>& cen, const std::vector<double>& sqr) {
  const double r = std::sqrt(1. / (double)g.deg(v));
  int best = 0;
  double best_sim = 0;
  for (int k = 0; k < K; k++) {
    double sum = 0;
    for (uint64_t i = g.rp[v]; i < g.rp[v + 1]; i++) sum += cen[k][g.ci[i]] * r;
    const double sim = sum / std::sqrt(sqr[k]);
    if (k == 0)
      best_sim = sim;
    else if (sim > best_sim) {
      best = k;
      best_sim = sim;
    }
  }
  return best;
}

// ViewBin::GetKHopViewSize: row entries of the vertices the (hop-1)-ball of v adds
// to the bin; `visited` marks the vertices expanded with a hop above one
uint64_t khop_size(const Rows& g, uint32_t v, int hop, std::vector<bool>& added, std::vector<bool>& visited, std::vector<uint32_t>& added_list,
                   std::vector<uint32_t>& visited_list) {
  uint64_t size = 0;
  if (!added[v]) {
    added[v] = true;
    size = g.deg(v);
    added_list.push_back(v);
  }
  if (hop > 1) {
    visited[v] = true;
    visited_list.push_back(v);
    for (uint64_t i = g.rp[v]; i < g.rp[v + 1]; i++)
      if (!visited[g.ci[i]]) size += khop_size(g, g.ci[i], hop - 1, added, visited, added_list, visited_list);
  }
  return size;
}

}  // namespace

extern "C" {

// kmeans -k K -i iters -init 1 [-rc] over one level; starts[p] is the cluster the
// reference's thread p draws (n_starts = its thread count).  Writes the final
// assignment (empty clusters removed) and the number of clusters; 0 on success.
int oracle_kmeans(uint64_t V, const uint64_t* rp, const uint32_t* ci, int K, int iters, const int32_t* starts, int n_starts, int reorder,
                  int32_t* assign_out, int32_t* n_clusters) {
  if (K < 1 || n_starts < 1) return -1;
  const Rows g{rp, ci};
  std::vector<int> assign(V);
  for (int p = 0; p < n_starts; p++) {  // RandomInit: thread p's vertices p, p + T, ...
    int id = starts[p];
    for (uint64_t v = p; v < V; v += n_starts) {
      assign[v] = id;
      if (++id >= K) id = 0;
    }
  }
  std::vector<std::vector<double>> cen(K, std::vector<double>(V, 0.0));
  std::vector<int> size(K);
  std::vector<double> sqr(K);
  centroids(g, V, K, assign, cen, size, sqr);
  for (int it = 0; it < iters; it++) {
    std::vector<int> next(V);  // every vertex is assigned against the same centroids
    for (uint64_t v = 0; v < V; v++) next[v] = assignment_of(g, (uint32_t)v, K, cen, sqr);
    assign.swap(next);
    centroids(g, V, K, assign, cen, size, sqr);
  }
  std::vector<unsigned> old2new(K);
  std::iota(old2new.begin(), old2new.end(), 0u);
  if (reorder) {  // non-zero entries counted for the first min(K, threads) centroids only
    std::vector<unsigned> nonzero(K, 0), new2old(K);
    for (int c = 0; c < std::min(K, n_starts); c++)
      for (double x : cen[c]) nonzero[c] += x != 0;
    std::iota(new2old.begin(), new2old.end(), 0u);
    std::sort(new2old.begin(), new2old.end(), [&](auto a, auto b) { return nonzero[a] > nonzero[b]; });
    for (int i = 0; i < K; i++) old2new[new2old[i]] = (unsigned)i;
  }
  std::vector<int> renum_size(K, 0), dense(K, -1);
  for (int k = 0; k < K; k++) renum_size[old2new[k]] = size[k];
  int n = 0;
  for (int k = 0; k < K; k++)
    if (renum_size[k]) dense[k] = n++;
  for (uint64_t v = 0; v < V; v++) assign_out[v] = dense[old2new[assign[v]]];
  *n_clusters = n;
  return 0;
}

// view_packing -s 1 -h hop over the sequences order[offs[q] .. offs[q+1]); bins
// hold at most cap row entries.  Writes the .vbmap content and the row entries of
// each merged bin (V entries of space); -2 when a source's ball alone exceeds cap
// (the reference loses that source and stops on its vertex-count assertion).
int oracle_view_packing(uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* order, const uint64_t* offs, int n_seqs, int hop,
                        uint64_t cap, int32_t* bins_out, int32_t* n_bins, uint64_t* sizes_out) {
  const Rows g{rp, ci};
  struct Bin {
    std::vector<uint32_t> sources;
    uint64_t total = 0;
  };
  std::vector<Bin> bins;
  for (int q = 0; q < n_seqs; q++) {
    // one pool per thread with one open bin: a source that does not fit closes it
    bins.emplace_back();
    std::vector<bool> added(V, false), visited(V, false);
    for (uint64_t p = offs[q]; p < offs[q + 1]; p++) {
      const uint32_t s = order[p];
      for (int attempt = 0; attempt < 2; attempt++) {
        std::vector<uint32_t> al, vl;
        const uint64_t inc = khop_size(g, s, hop, added, visited, al, vl);
        if (bins.back().total + inc <= cap) {
          bins.back().total += inc;
          bins.back().sources.push_back(s);
          break;
        }
        if (attempt == 1) return -2;  // the new, empty bin cannot take it either
        // DoRecall on the closed bin does not matter: it is never used again
        bins.emplace_back();
        std::fill(added.begin(), added.end(), false);
        std::fill(visited.begin(), visited.end(), false);
      }
    }
  }
  std::vector<std::pair<int, size_t>> id_size;
  for (size_t i = 0; i < bins.size(); i++) id_size.push_back({(int)i, (size_t)bins[i].total});
  std::sort(id_size.begin(), id_size.end(), [](const auto& a, const auto& b) { return a.second < b.second; });
  std::vector<std::vector<int>> merged_ids(bins.size());
  int merged = 0;
  size_t old_size = 0;
  for (const auto& [id, sz] : id_size) {
    if (old_size + sz > cap) {
      merged++;
      old_size = sz;
    } else {
      old_size += sz;
    }
    merged_ids[merged].push_back(id);
  }
  merged++;
  for (int i = 0; i < merged; i++) {
    sizes_out[i] = 0;
    for (int id : merged_ids[i]) {
      sizes_out[i] += bins[id].total;
      for (uint32_t v : bins[id].sources) bins_out[v] = i;
    }
  }
  *n_bins = merged;
  return 0;
}

}  // extern "C"
