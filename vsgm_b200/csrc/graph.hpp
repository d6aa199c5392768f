// Host-side graph layer: CSR container, file formats, synthetic generators and
// view (k-hop halo) materialisation.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace vsgm {

// Undirected simple graph in CSR: row_ptrs[V+1] (u64), cols[E] (u32), every row
// sorted ascending, no self-loops, no duplicates; E counts both directions.
struct Csr {
  uint64_t V = 0;
  std::vector<uint64_t> row_ptrs;
  std::vector<uint32_t> cols;
  uint64_t E() const { return cols.size(); }
};

// counter-based random numbers: value i of stream `seed`
uint64_t mix64(uint64_t seed, uint64_t i);
double unit_double(uint64_t seed, uint64_t i);

// Build a CSR from undirected edge endpoints: self-loops dropped, both
// directions added, duplicates removed (the rules of
// src/preprocess/preprocess_graph.h:12-92, without dropping isolated vertices).
void csr_from_edges(uint64_t V, std::vector<uint32_t>&& src, std::vector<uint32_t>&& dst, int threads, Csr* out);

// R-MAT: edge_factor * 2^scale draws, quadrant probabilities a, b, c, 1-a-b-c.
void gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int threads, Csr* out);

// Chung-Lu: expected degrees w_i = dmax * ((i + i0) / i0)^(-1/(gamma-1)) with i0
// chosen so that sum(w) = 2 * target_edges; target_edges endpoint pairs drawn
// independently with probability proportional to w.
void gen_chung_lu(uint64_t V, uint64_t target_edges, double gamma, uint64_t dmax, uint64_t seed, int threads, Csr* out);

// CSR .bin (src/graph/graph_io.h:57-100 reader, :313-339 writer layout):
// u64 sizeof(uintV)=4, u64 sizeof(uintE)=8, u64 V, u64 E, u64 row_ptrs[V+1], u32 cols[E]
bool read_csr_bin(const std::string& path, Csr* out, std::string* err);
// The header alone, with the file's size checked against it exactly (the reference
// asserts that the file ends right after the cols).
bool csr_bin_header(const std::string& path, uint64_t* V, uint64_t* E, std::string* err);
// row_ptrs and cols straight into caller buffers (V+1 and E entries) with parallel
// positioned reads of large chunks: no intermediate copy, no zero fill.
bool read_csr_bin_into(const std::string& path, uint64_t V, uint64_t E, uint64_t* row_ptrs, uint32_t* cols, int threads, std::string* err);
bool write_csr_bin(const std::string& path, const Csr& g, std::string* err);

// .vbmap (src/tools/view_packing.cc:309-322, read at src/view/view_bin_manager.h:30-67):
// line 1 = number of bins, then one bin id per vertex.
bool read_vbmap(const std::string& path, uint64_t V, std::vector<int32_t>* bins, int32_t* n_bins, std::string* err);
bool write_vbmap(const std::string& path, const std::vector<int32_t>& bins, int32_t n_bins, std::string* err);

// GraphIO::Validate (src/graph/graph_io.h:416-444) without the dangling check:
// returns the number of unsorted/duplicate entries and self loops (0 = valid).
uint64_t csr_defects(const Csr& g);

// ViewBin::Materialize (src/view/view_bin.h:49-142): every source whose degree
// is >= root_degree (all sources when root_degree == 0) plus everything within
// hop-1 steps of it keeps its full adjacency row; all other rows are empty.
// Writes a full-V CSR (view_row_ptrs[V+1]); returns false if cols_cap is too small.
bool materialize_view(const uint64_t* row_ptrs, const uint32_t* cols, uint64_t V, const uint32_t* sources, uint64_t n_sources, int hop,
                      uint64_t root_degree, int threads, uint64_t* view_row_ptrs, uint32_t* view_cols, uint64_t cols_cap, uint64_t* n_cols);

// Degree-ordered relabelling: new id = rank of (degree, old id), ascending or
// descending; rows are rewritten through the permutation and re-sorted.  Exact
// counts are invariant to any relabelling (the partial orders pick one
// representative of every automorphism class whatever the labels); per-view
// counts are not, so a relabelling must be applied to the whole graph and its
// .vbmap before views are built.
void degree_relabel(const Csr& g, bool ascending, int threads, std::vector<uint32_t>* new_of_old, Csr* out);

// Connected random pattern: n uniform in [n_min, n_max], each pair an edge with
// probability p, rejection-sampled until connected.  Draws come from stream
// `seed` starting at *counter, which is advanced past the draws used.
void random_pattern(int n_min, int n_max, double p, uint64_t seed, uint64_t* counter, int* n, uint8_t bits[7]);

// Message returned by vsgm_last_error on this thread (for entry points defined
// outside capi_host.cpp).
void set_host_error(const std::string& msg);

}  // namespace vsgm
