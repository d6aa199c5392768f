// view_tools: the reference's offline view-bin chain on the GPU, with its flags
// and its files.
//
//   view_tools features -f G.bin -h 1                     -> G.bin.1hop.bin
//   view_tools kmeans -f G.bin.1hop.bin -k K -i I -init 1 -t T [-rc 0|1] [-o PREFIX] [-d 1]
//                                                         -> PREFIX + K (default G.bin.1hop.bin.kmeans.K)
//   view_tools view_packing -gf G.bin -pf PARTITION -h H -m GB -t T -s 1 [-o 0|1] [-d 1]
//                                                         -> G.bin.H.hop.vbmap, G.bin.H.hop.vbstat
//
// src/tools/features.cc:64-208, src/tools/kmeans.cc:636-694,
// src/tools/view_packing.cc:326-361.  Supported: features -h 1; kmeans -init 1 with
// a single level ("K" or "1xK"); view_packing -s 1 (one open bin per thread).  The
// random start of -init 1 is the reference's std::rand() % K per thread, drawn here
// in thread order in this fresh process (with -t 1 exactly the reference's draw).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "vsgm.h"

namespace {

struct Args {
  std::map<std::string, std::string> kv;
  Args(int argc, char** argv, int from) {
    for (int i = from; i + 1 < argc; i += 2) kv[argv[i]] = argv[i + 1];
  }
  std::string str(const std::string& k, const std::string& d) const {
    auto it = kv.find(k);
    return it == kv.end() ? d : it->second;
  }
  int num(const std::string& k, int d) const { return std::stoi(str(k, std::to_string(d))); }
  double real(const std::string& k, double d) const {
    auto it = kv.find(k);
    return it == kv.end() ? d : std::stod(it->second);
  }
};

int die(const std::string& what) {
  std::cerr << "view_tools: " << what << ": " << vsgm_last_error() << std::endl;
  return 1;
}

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

struct HostGraph {
  uint64_t V = 0, E = 0;
  uint64_t* rp = nullptr;
  uint32_t* ci = nullptr;
  ~HostGraph() {
    vsgm_free(rp);
    vsgm_free(ci);
  }
  bool read(const std::string& path) { return vsgm_read_csr_bin(path.c_str(), &V, &E, &rp, &ci) == VSGM_OK; }
};

int features(const Args& a, int device) {
  const std::string f = a.str("-f", "./data/com-dblp.ungraph.txt");
  if (a.num("-h", 2) != 1) {
    std::cerr << "view_tools features: only -h 1 (the self-loop feature graph) is built on the GPU" << std::endl;
    return 2;
  }
  HostGraph g;
  if (!g.read(f)) return die("reading " + f);
  std::vector<uint64_t> rp(g.V + 1);
  std::vector<uint32_t> ci(g.E + g.V);
  const auto t = std::chrono::steady_clock::now();
  if (vsgm_features_1hop(device, g.V, g.rp, g.ci, rp.data(), ci.data()) != VSGM_OK) return die("features");
  std::cout << "new edge count: " << g.E + g.V << "\n" << "features on the GPU: " << ms_since(t) << " ms" << std::endl;
  const std::string out = f + ".1hop.bin";
  if (vsgm_write_csr_bin(out.c_str(), g.V, g.E + g.V, rp.data(), ci.data()) != VSGM_OK) return die("writing " + out);
  std::cout << "wrote " << out << std::endl;
  return 0;
}

int kmeans(const Args& a, int device) {
  const std::string f = a.str("-f", "./data/com-dblp.ungraph.txt");
  std::string ks = a.str("-k", "4");
  const int iters = a.num("-i", 20), threads = a.num("-t", 16), rc = a.num("-rc", 0), dump = a.num("-d", 1);
  const std::string out = a.str("-o", f + ".kmeans.") + ks;
  if (a.num("-init", 0) != 1) {
    std::cerr << "view_tools kmeans: only -init 1 (random start) is supported; -init 0 seeds from the clock" << std::endl;
    return 2;
  }
  int K = 0;
  if (ks.find('^') != std::string::npos) {
    std::cerr << "view_tools kmeans: -k a^x is not supported" << std::endl;
    return 2;
  }
  if (ks.find('x') != std::string::npos) {  // "1xK": the first level keeps one cluster, the second splits it
    const int first = std::stoi(ks.substr(0, ks.find('x')));
    const std::string rest = ks.substr(ks.find('x') + 1);
    if (first != 1 || rest.find('x') != std::string::npos) {
      std::cerr << "view_tools kmeans: of the multi-level forms only 1xK is supported" << std::endl;
      return 2;
    }
    K = std::stoi(rest);
  } else {
    K = std::stoi(ks);
  }
  HostGraph g;
  if (!g.read(f)) return die("reading " + f);
  std::vector<int32_t> starts(std::max(1, threads));
  for (auto& s : starts) s = std::rand() % K;  // RandomInit's draw per thread (kmeans.cc:128)
  std::vector<int32_t> assign(g.V);
  std::vector<int64_t> sizes(K);
  int32_t n = 0;
  const auto t = std::chrono::steady_clock::now();
  if (vsgm_kmeans(device, g.V, g.rp, g.ci, K, iters, starts.data(), (int)starts.size(), rc, assign.data(), sizes.data(), &n) != VSGM_OK)
    return die("kmeans");
  std::cout << "Cluster sizes: [";
  for (int k = 0; k < n; k++) std::cout << sizes[k] << ", ";
  std::cout << "]\nkmeans on the GPU: " << ms_since(t) << " ms" << std::endl;
  if (dump) {
    std::string buf;
    buf.reserve(g.V * 3);
    char tmp[16];
    for (uint64_t v = 0; v < g.V; v++) {
      const int len = std::snprintf(tmp, sizeof(tmp), "%d\n", assign[v]);
      buf.append(tmp, len);
    }
    FILE* fp = std::fopen(out.c_str(), "wb");
    if (!fp || std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) {
      std::cerr << "view_tools kmeans: cannot write " << out << std::endl;
      if (fp) std::fclose(fp);
      return 1;
    }
    std::fclose(fp);
    std::cout << "wrote " << out << std::endl;
  }
  return 0;
}

int view_packing(const Args& a, int device) {
  const std::string gf = a.str("-gf", "./data/com-dblp.ungraph.txt.bin");
  const std::string pf = a.str("-pf", "./data/com-dblp.ungraph.txt.bin.kmeans.4");
  const int hop = a.num("-h", 2), threads = a.num("-t", 16), pool = a.num("-s", 1), opt = a.num("-o", 0), dump = a.num("-d", 1);
  const double mem = a.real("-m", 10);
  if (pool != 1) {
    std::cerr << "view_tools view_packing: only -s 1 (next-fit, one open bin per thread) is supported" << std::endl;
    return 2;
  }
  HostGraph g;
  if (!g.read(gf)) return die("reading " + gf);
  const size_t max_bin = (mem * 1000 * 1000 * 1000) / sizeof(uint32_t);  // view_packing.cc:352
  std::cout << "mem: " << mem << "G, max view bin size: " << max_bin << std::endl;
  // the partition file: one cluster id per line (ReadPartitionFile, view_packing.cc:114-137)
  std::vector<int> part;
  part.reserve(g.V);
  {
    std::ifstream in(pf);
    if (!in) {
      std::cerr << "view_tools view_packing: cannot read " << pf << std::endl;
      return 1;
    }
    std::string line;
    while (std::getline(in, line)) part.push_back(std::stoi(line));
  }
  if (part.size() != g.V) {
    std::cerr << "view_tools view_packing: " << pf << " has " << part.size() << " lines for " << g.V << " vertices" << std::endl;
    return 1;
  }
  // each thread's source order (view_packing.cc:150-190)
  const std::string suffix = pf.substr(pf.find_last_of('.') + 1);
  int first = 0, second = 1;
  const bool layered = suffix.find('x') != std::string::npos;
  first = std::stoi(layered ? suffix.substr(0, suffix.find('x')) : suffix);
  if (layered) second = std::stoi(suffix.substr(suffix.find('x') + 1));
  if (first != threads) {
    std::cerr << "view_tools view_packing: partition " << suffix << " needs -t " << first << std::endl;
    return 2;
  }
  std::vector<size_t> degrees(g.V);
  for (uint64_t v = 0; v < g.V; v++) degrees[v] = g.rp[v + 1] - g.rp[v];
  std::vector<std::vector<uint32_t>> chunks(threads);
  std::vector<std::vector<std::vector<uint32_t>>> cells(threads, std::vector<std::vector<uint32_t>>(second));
  for (uint64_t u = 0; u < g.V; u++) {
    const int p = part[u];
    const int c = layered ? p / second : p, j = layered ? p % second : 0;
    if (p < 0 || c >= threads) {
      std::cerr << "view_tools view_packing: cluster " << p << " of vertex " << u << " is outside the partition " << suffix << std::endl;
      return 1;
    }
    cells[c][j].push_back((uint32_t)u);
  }
  for (int i = 0; i < threads; i++)
    for (int j = 0; j < second; j++) {
      if (opt) std::sort(cells[i][j].begin(), cells[i][j].end(), [&](const auto& x, const auto& y) { return degrees[x] > degrees[y]; });
      chunks[i].insert(chunks[i].end(), cells[i][j].begin(), cells[i][j].end());
    }
  std::vector<uint32_t> order;
  std::vector<uint64_t> offsets{0};
  for (auto& c : chunks) {
    order.insert(order.end(), c.begin(), c.end());
    offsets.push_back(order.size());
  }
  std::vector<int32_t> bins(g.V);
  std::vector<uint64_t> sizes(g.V);
  int32_t nb = 0;
  const auto t = std::chrono::steady_clock::now();
  if (vsgm_view_packing(device, g.V, g.rp, g.ci, order.data(), offsets.data(), threads, hop, max_bin, bins.data(), &nb, sizes.data(), g.V) != VSGM_OK)
    return die("view_packing");
  std::cout << "total " << nb << " bins after merging\nview packing on the GPU: " << ms_since(t) << " ms" << std::endl;
  if (dump) {
    const std::string stat = gf + "." + std::to_string(hop) + ".hop.vbstat";
    std::vector<size_t> sources(nb, 0);
    for (uint64_t v = 0; v < g.V; v++) sources[bins[v]]++;
    std::ofstream s(stat);
    s << "view bin count: " << nb << "\n";
    for (int i = 0; i < nb; i++) s << "view bin id: " << i << ", sources: " << sources[i] << ", total size: " << sizes[i] << "\n";
    const std::string map = gf + "." + std::to_string(hop) + ".hop.vbmap";
    if (vsgm_write_vbmap(map.c_str(), g.V, bins.data(), nb) != VSGM_OK) return die("writing " + map);
    std::cout << "wrote " << map << " and " << stat << std::endl;
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: view_tools features|kmeans|view_packing [reference flags] [-gpu DEVICE]" << std::endl;
    return 2;
  }
  const std::string tool = argv[1];
  Args a(argc, argv, 2);
  const int device = a.num("-gpu", 0);
  if (tool == "features") return features(a, device);
  if (tool == "kmeans") return kmeans(a, device);
  if (tool == "view_packing") return view_packing(a, device);
  std::cerr << "view_tools: unknown tool " << tool << std::endl;
  return 2;
}
