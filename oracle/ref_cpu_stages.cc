// Test and baseline infrastructure (not part of the product): the reference's own
// CPU stages compiled from its sources, GraphIO::ReadCSRBinFile
// (src/graph/graph_io.h:57-100) and ViewBinManager::LoadViewBinPartition +
// ViewBin::Materialize (src/view/view_bin_manager.h:30-67, src/view/view_bin.h:49-142).
// The pinned host buffers of ViewBinHolder (src/view/view_bin_holder.h:14-24) are
// plain malloc here, so no GPU or CUDA runtime is needed.
//
//   ref_cpu_stages read  <graph.bin>
//       -> "read V E sum_cols ms"
//   ref_cpu_stages views <graph.bin> <vbmap> <hop> <root_degree> <threads> [dump_dir]
//       -> one "view id sources vertices cols ms" line per bin, then "total ms";
//          with dump_dir, bin i's view is written to dump_dir/view_i.bin as
//          u64 V, u64 n_cols, u64 row_ptrs[V+1], u32 cols[n_cols].
#include <cuda_runtime.h>  // for the types the reference's headers name

#include <cstdio>
#include <cstdlib>
#include <string>

static cudaError_t harness_host_alloc(void** p, size_t bytes) {
  *p = std::malloc(bytes ? bytes : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
#define cudaMallocHost(p, bytes) harness_host_alloc((void**)(p), (bytes))
#define cudaFreeHost(p) std::free(p)
#define CUDA_ERROR(e) (e)

#include "graph/cpu_graph.h"
#include "view/view_bin_manager.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_cpu_stages read <graph.bin> | views <graph.bin> <vbmap> <hop> <root_degree> <threads> [dump_dir]\n");
    return 2;
  }
  const std::string mode = argv[1];
  TimeMeasurer t;
  t.StartTimer();
  Graph g(argv[2], false);
  t.EndTimer();
  const size_t V = g.GetVertexCount(), E = g.GetEdgeCount();
  if (mode == "read") {
    unsigned long long sum = 0;
    for (size_t j = 0; j < E; j++) sum += g.GetCols()[j];
    std::printf("read %zu %zu %llu %.3f\n", V, E, sum, t.GetElapsedMicroSeconds() / 1000.0);
    return 0;
  }
  if (mode != "views" || argc < 7) return 2;
  const int hop = std::atoi(argv[4]);
  const size_t root_degree = std::strtoull(argv[5], nullptr, 10);
  const int threads = std::atoi(argv[6]);
  const char* dump = argc > 7 ? argv[7] : nullptr;
  ViewBinManager m(&g, hop, threads);
  m.LoadViewBinPartition(argv[3]);
  std::unique_ptr<ViewBinHolder> h(new ViewBinHolder(V, E * sizeof(uintV)));
  double total = 0;
  for (const auto& vb : m.GetViewBinPool()) {
    if (vb->GetSourcesNum() == 0) continue;  // Materialize asserts on an empty bin
    TimeMeasurer tv;
    tv.StartTimer();
    vb->Materialize(h, root_degree);
    tv.EndTimer();
    const double ms = tv.GetElapsedMicroSeconds() / 1000.0;
    total += ms;
    const uintE n = h->GetRowPtrs()[V];
    std::printf("view %zu %zu %zu %llu %.3f\n", vb->GetId(), h->GetSourcesNum(), vb->GetVerticesNum(), (unsigned long long)n, ms);
    if (dump) {
      const std::string path = std::string(dump) + "/view_" + std::to_string(vb->GetId()) + ".bin";
      FILE* f = std::fopen(path.c_str(), "wb");
      if (!f) return 3;
      const unsigned long long hdr[2] = {V, n};
      std::fwrite(hdr, sizeof(hdr), 1, f);
      std::fwrite(h->GetRowPtrs(), sizeof(uintE), V + 1, f);
      std::fwrite(h->GetCols(), sizeof(uintV), n, f);
      std::fclose(f);
    }
  }
  std::printf("total %.3f\n", total);
  return 0;
}
