// pm_pipeline: command-line driver with the reference's flags and output lines
// (src/app/pattern_matching_pipeline.cu:27-201), over the vsgm C ABI.
//
//   pm_pipeline -f <graph.bin> [-m GB] [-p P | -kc k | -km k] [-t threads] [-qs queue]
//               [-pn producers] [-cn consumers] [-dm 0|1] [-df 0|1] [-dr 0|1] [-ds 0|1] [-dst n] [-gv 0|1|2]
//               [-rl 0|1]
//
// With -gv 2 (default) every consumer keeps the whole graph on its GPU and
// matches each view bin's sources over it directly (vsgm_graph_view, no halo
// needed); with -gv 1 it builds each bin's k-hop halo there
// (vsgm_materialize_view).  In both, producers only hand out bin ids.  With
// -gv 0 producers materialise the halos on the host into a bounded queue of
// host buffers, as the reference does, and each consumer uploads them.
// There the consumers stream the views: a view's copies (in compact form, from a
// pool of -qs pinned holders) run while the previous view is matched.  Either way
// one consumer per GPU matches every plan and accumulates exact counts.  Without a .vbmap file (the file does not exist) every vertex is a source
// of one bin; any other failure to open it is an error.  With -rl 1 (default) the
// graph is relabelled so that ids ascend with degree before any view is built
// (inside the timed region; on the device with -gv 1 / 2, on the host with the bins
// following their vertices with -gv 0): the plans' order conditions then cut every
// adjacency window short, and exact totals do not depend on the labelling.  Prints
// "total count for query i: N" and "finish total time, elapsed_time=Xms" like the
// reference.
#include <sys/stat.h>
#include <sys/time.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vsgm.h"

namespace {

struct Args {
  std::string file = "./data/com-friendster.ungraph.txt.bin";
  double mem = 10;
  int pattern = 1, kc = 0, km = 0, threads = 1, qs = 1, pn = 1, cn = 1, dm = 1, df = 1, dr = 0, ds = 0, dst = 1, gv = 2, rl = 1;
};

// CommandLine's linear scan (src/common/command_line.h:32-86)
const char* opt(int argc, char** argv, const char* name) {
  for (int i = 1; i + 1 < argc; i++)
    if (std::strcmp(argv[i], name) == 0) return argv[i + 1];
  return nullptr;
}

double now_us() {
  timeval t;
  gettimeofday(&t, nullptr);
  return t.tv_sec * 1e6 + t.tv_usec;
}

struct View {
  int id = -1;
  std::vector<uint32_t> sources;
  // -gv 0: a host-built halo in compact form, in pinned buffers of a holder that is
  // recycled between producers and consumers (the reference's ViewBinBuffer)
  std::vector<uint64_t> row_ptrs;  // full-V offsets as the materialiser writes them
  uint32_t* cols = nullptr;        // pinned, cap entries
  uint32_t* vert = nullptr;        // pinned, V entries
  uint64_t* off = nullptr;         // pinned, V + 1 entries
  uint32_t* src = nullptr;         // pinned, V entries
  uint64_t n_cols = 0, n_vert = 0;
};

// bounded hand-off between producer and consumer threads
struct Queue {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<View*> items;
  size_t cap;
  bool closed = false;
  explicit Queue(size_t c) : cap(c) {}
  void push(View* v) {
    std::unique_lock<std::mutex> l(mu);
    cv.wait(l, [&] { return items.size() < cap; });
    items.push_back(v);
    cv.notify_all();
  }
  View* pop() {
    std::unique_lock<std::mutex> l(mu);
    cv.wait(l, [&] { return !items.empty() || closed; });
    if (items.empty()) return nullptr;
    View* v = items.front();
    items.pop_front();
    cv.notify_all();
    return v;
  }
  void close() {
    std::lock_guard<std::mutex> l(mu);
    closed = true;
    cv.notify_all();
  }
};

uint64_t work_of(const std::vector<uint32_t>& src, const uint64_t* rp) {
  uint64_t s = 0;
  for (uint32_t v : src) s += rp[v + 1] - rp[v];
  return s;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 1) return -1;
  Args a;
  if (auto v = opt(argc, argv, "-f")) a.file = v;
  if (auto v = opt(argc, argv, "-m")) a.mem = std::atof(v);
  if (auto v = opt(argc, argv, "-p")) a.pattern = std::atoi(v);
  if (auto v = opt(argc, argv, "-kc")) a.kc = std::atoi(v);
  if (auto v = opt(argc, argv, "-km")) a.km = std::atoi(v);
  if (auto v = opt(argc, argv, "-t")) a.threads = std::atoi(v);
  if (auto v = opt(argc, argv, "-qs")) a.qs = std::atoi(v);
  if (auto v = opt(argc, argv, "-pn")) a.pn = std::atoi(v);
  if (auto v = opt(argc, argv, "-cn")) a.cn = std::atoi(v);
  if (auto v = opt(argc, argv, "-dm")) a.dm = std::atoi(v);
  if (auto v = opt(argc, argv, "-df")) a.df = std::atoi(v);
  if (auto v = opt(argc, argv, "-dr")) a.dr = std::atoi(v);
  if (auto v = opt(argc, argv, "-ds")) a.ds = std::atoi(v);
  if (auto v = opt(argc, argv, "-dst")) a.dst = std::atoi(v);
  if (auto v = opt(argc, argv, "-gv")) a.gv = std::atoi(v);
  if (auto v = opt(argc, argv, "-rl")) a.rl = std::atoi(v);
  if (a.qs < a.cn || a.pn < 1 || a.cn < 1) {
    std::fprintf(stderr, "error: need -qs >= -cn >= 1 and -pn >= 1\n");
    return 1;
  }
  std::printf("m: %g t: %d qs: %d pn: %d cn: %d\n", a.mem, a.threads, a.qs, a.pn, a.cn);

  // queries and plans (pattern_matching_pipeline.cu:58-87)
  std::vector<vsgm_plan> plans;
  if (a.kc) {
    plans.resize(1);
    if (vsgm_plan_clique(a.kc, &plans[0])) return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
  } else if (a.km) {
    int n = 0;
    plans.resize(64);
    if (vsgm_plan_graphlets(a.km, plans.data(), 64, &n)) return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
    plans.resize(n);
  } else {
    plans.resize(1);
    if (vsgm_plan_pattern(a.pattern, &plans[0])) return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
  }
  int hop = 0;
  uint64_t root_degree = a.df ? ~0ull : 0;
  for (auto& p : plans) {
    hop = std::max(hop, p.hop);
    if (p.root_degree < root_degree) root_degree = p.root_degree;
  }

  // graph and view bins (:89-100)
  uint64_t V = 0, E = 0;
  uint64_t* rp = nullptr;
  uint32_t* ci = nullptr;
  if (vsgm_read_csr_bin(a.file.c_str(), &V, &E, &rp, &ci)) return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
  std::printf("vertex_count=%llu,edge_count=%llu\n", (unsigned long long)V, (unsigned long long)E);
  std::string vbmap = a.file + "." + std::to_string(hop) + ".hop.vbmap";
  std::vector<int32_t> bins(V);
  int32_t n_bins = 0;
  struct stat vb_st;
  bool have_vbmap = true;
  if (::stat(vbmap.c_str(), &vb_st) != 0) {
    if (errno != ENOENT) return std::fprintf(stderr, "error: cannot stat %s: %s\n", vbmap.c_str(), std::strerror(errno)), 1;
    // no partition file: one bin holding every source (what view_packing produces
    // when the whole graph fits the budget).  A halo built from it is the whole
    // graph, so with -gv 0 / 1 it must fit the -m budget.
    if (a.gv != 2 && 4.0 * (double)E > a.mem * 1e9)
      return std::fprintf(stderr, "error: no %s, and one view of the whole graph (%.2f GB of adjacency) exceeds -m %g\n", vbmap.c_str(),
                          4.0 * (double)E / 1e9, a.mem),
             1;
    std::printf("no view bin partition file %s: one view bin of every vertex\n", vbmap.c_str());
    have_vbmap = false;
    n_bins = 1;
  } else if (!S_ISREG(vb_st.st_mode)) {
    return std::fprintf(stderr, "error: %s is not a regular file\n", vbmap.c_str()), 1;
  } else if (vsgm_read_vbmap(vbmap.c_str(), V, bins.data(), &n_bins)) {
    return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
  }
  double t0 = now_us();
  if (a.rl && a.gv == 0) {
    // views built on the host: relabel the host graph (ids ascending with degree;
    // the bins follow their vertices).  With -gv 1 / 2 every consumer relabels its
    // resident copy on the device instead, and the bins stay in the file's ids.
    std::vector<uint32_t> new_of_old(V);
    uint64_t* rp2 = (uint64_t*)std::malloc(sizeof(uint64_t) * (V + 1));
    uint32_t* ci2 = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<uint64_t>(E, 1));
    if (!rp2 || !ci2) return std::fprintf(stderr, "error: host allocation failed (relabel)\n"), 1;
    if (vsgm_degree_relabel(V, rp, ci, 1, a.threads > 1 ? a.threads : 0, new_of_old.data(), rp2, ci2))
      return std::fprintf(stderr, "error: %s\n", vsgm_last_error()), 1;
    vsgm_free(rp);
    vsgm_free(ci);
    rp = rp2;
    ci = ci2;
    std::vector<int32_t> moved(V);
    for (uint64_t v = 0; v < V; v++) moved[new_of_old[v]] = bins[v];
    bins.swap(moved);
  }
  std::vector<std::vector<uint32_t>> pool(n_bins);
  for (uint64_t v = 0; v < V; v++) pool[bins[v]].push_back((uint32_t)v);
  pool.erase(std::remove_if(pool.begin(), pool.end(), [](const std::vector<uint32_t>& s) { return s.empty(); }), pool.end());
  if (a.ds) {
    // ViewBinManager::Split (src/view/view_bin_manager.h:69-134): split the bin
    // furthest above the mean degree sum into two by alternating sources of
    // descending degree, until the bin count is a multiple of the consumers
    int target = ((int)pool.size() / a.cn + a.dst) * a.cn;
    while ((int)pool.size() < target) {
      uint64_t sum = 0;
      for (auto& s : pool) sum += work_of(s, rp);
      uint64_t avg = sum / pool.size(), best = 0;
      size_t at = 0;
      for (size_t i = 0; i < pool.size(); i++) {
        uint64_t w = work_of(pool[i], rp);
        if (w >= avg && w - avg > best) best = w - avg, at = i;
      }
      std::vector<uint32_t> s = pool[at];
      std::stable_sort(s.begin(), s.end(), [&](uint32_t x, uint32_t y) { return rp[x + 1] - rp[x] > rp[y + 1] - rp[y]; });
      std::vector<uint32_t> odd, even;
      for (size_t i = 0; i < s.size(); i++) (i % 2 ? odd : even).push_back(s[i]);
      pool.erase(pool.begin() + at);
      pool.push_back(odd);
      pool.push_back(even);
    }
  }
  if (a.dr || a.ds)
    std::stable_sort(pool.begin(), pool.end(), [&](const auto& x, const auto& y) { return work_of(x, rp) > work_of(y, rp); });
  if (have_vbmap) std::printf("loaded view bin partition file, %zu view bins\n", pool.size());

  const uint64_t cap = std::min<uint64_t>(E, (uint64_t)(a.mem * 1e9 / sizeof(uint32_t)));
  Queue q(a.qs);
  // -gv 0: qs pinned holders, handed back through `spare` once their copies are done
  Queue spare(a.qs);
  std::vector<View> holders(a.gv == 0 ? a.qs : 0);
  for (View& h : holders) {
    h.row_ptrs.resize(V + 1);
    void *c = nullptr, *vt = nullptr, *o = nullptr, *sr = nullptr;
    if (vsgm_host_alloc(sizeof(uint32_t) * std::max<uint64_t>(cap, 1), &c) || vsgm_host_alloc(sizeof(uint32_t) * std::max<uint64_t>(V, 1), &vt) ||
        vsgm_host_alloc(sizeof(uint64_t) * (V + 1), &o) || vsgm_host_alloc(sizeof(uint32_t) * std::max<uint64_t>(V, 1), &sr))
      return std::fprintf(stderr, "error: pinned view buffers: %s\n", vsgm_last_error()), 1;
    h.cols = (uint32_t*)c;
    h.vert = (uint32_t*)vt;
    h.off = (uint64_t*)o;
    h.src = (uint32_t*)sr;
    spare.push(&h);
  }
  std::atomic<size_t> next{0};
  std::atomic<int> failed{0};
  std::vector<std::vector<uint64_t>> counts(a.cn, std::vector<uint64_t>(plans.size(), 0));

  std::vector<std::thread> producers, consumers;
  for (int p = 0; p < a.pn; p++)
    producers.emplace_back([&] {
      for (size_t id; (id = next++) < pool.size();) {
        if (a.gv) {  // the consumer builds the halo on its GPU
          View* v = new View();
          v->id = (int)id;
          v->sources = pool[id];
          q.push(v);
          continue;
        }
        View* v = spare.pop();  // a free pinned holder
        if (!v) break;
        v->id = (int)id;
        v->sources = pool[id];
        std::memcpy(v->src, v->sources.data(), sizeof(uint32_t) * v->sources.size());
        if (vsgm_view_materialize(V, rp, ci, v->sources.data(), v->sources.size(), hop, root_degree, a.threads, v->row_ptrs.data(), v->cols, cap,
                                  &v->n_cols) ||
            vsgm_view_compact(V, v->row_ptrs.data(), v->vert, v->off, &v->n_vert)) {
          std::fprintf(stderr, "error: view %zu: %s\n", id, vsgm_last_error());
          failed = 1;
          spare.push(v);
          continue;
        }
        q.push(v);
      }
    });
  // a view a consumer gives up: pooled holders go back to the producers
  auto drop = [&](View* v) {
    if (a.gv == 0)
      spare.push(v);
    else
      delete v;
  };
  for (int c = 0; c < a.cn; c++)
    consumers.emplace_back([&, c] {
      vsgm_engine* e = nullptr;
      if (vsgm_create(c, V, plans.data(), (int)plans.size(), 0, 0, &e)) {
        std::fprintf(stderr, "error: consumer %d: %s\n", c, vsgm_engine_error(nullptr));
        failed = 1;
        while (View* v = q.pop()) drop(v);  // keep producers moving
        return;
      }
      if (a.gv && a.rl && vsgm_set_option(e, "relabel", 1)) {
        std::fprintf(stderr, "error: consumer %d: %s\n", c, vsgm_engine_error(e));
        failed = 1;
        while (View* v = q.pop()) drop(v);
        vsgm_destroy(e);
        return;
      }
      if (a.gv && vsgm_upload_graph(e, rp, ci, E)) {
        std::fprintf(stderr, "error: consumer %d: %s\n", c, vsgm_engine_error(e));
        failed = 1;
        while (View* v = q.pop()) drop(v);
        vsgm_destroy(e);
        return;
      }
      auto fail_here = [&] {
        std::fprintf(stderr, "error: consumer %d: %s\n", c, vsgm_engine_error(e));
        failed = 1;
      };
      if (a.gv) {
        while (View* v = q.pop()) {
          int rc = a.gv == 2 ? vsgm_graph_view(e, v->sources.data(), v->sources.size())
                             : vsgm_materialize_view(e, v->sources.data(), v->sources.size(), hop, root_degree);
          delete v;
          if (!rc && a.dm) rc = vsgm_match(e);
          if (rc) fail_here();
        }
      } else {
        // host-built views: the next view's copies run while the current one is matched
        auto prefetch = [&](View* v) {
          return vsgm_prefetch_view(e, v->vert, v->n_vert, v->off, v->cols, v->src, v->sources.size());
        };
        auto install = [&](View* v) {  // current := prefetched; the holder goes back to the producers
          int rc = vsgm_swap_view(e);
          if (!rc) rc = vsgm_view_released(e);
          spare.push(v);
          return rc;
        };
        View* v = q.pop();
        int rc = 0;
        if (v) {
          rc = prefetch(v);
          if (!rc) rc = install(v);
          else spare.push(v);
        }
        while (v) {
          View* nx = rc ? nullptr : q.pop();
          if (nx && (rc = prefetch(nx)) != 0) {
            spare.push(nx);
            nx = nullptr;
          }
          if (!rc && a.dm) rc = vsgm_match(e);
          if (!nx) break;
          if (!rc) rc = install(nx);
          else spare.push(nx);
          v = nx;
        }
        if (rc) {
          fail_here();
          while (View* w = q.pop()) spare.push(w);  // keep producers moving
        }
      }
      vsgm_get_counts(e, counts[c].data());
      vsgm_destroy(e);
    });
  for (auto& t : producers) t.join();
  q.close();
  for (auto& t : consumers) t.join();
  double t1 = now_us();
  std::printf("finish total time, elapsed_time=%fms\n", (t1 - t0) / 1000.0);
  for (size_t i = 0; i < plans.size(); i++) {
    uint64_t s = 0;
    for (int c = 0; c < a.cn; c++) s += counts[c][i];
    std::printf("total count for query %zu: %llu\n", i, (unsigned long long)s);
  }
  for (View& h : holders) {
    vsgm_host_free(h.cols);
    vsgm_host_free(h.vert);
    vsgm_host_free(h.off);
    vsgm_host_free(h.src);
  }
  vsgm_free(rp);
  vsgm_free(ci);
  return failed ? 2 : 0;
}
