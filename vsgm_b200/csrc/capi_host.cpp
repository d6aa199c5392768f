// C ABI for the host-side layers (planning, files, generators, views).
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "graph.hpp"
#include "planner.hpp"
#include "vsgm.h"

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

template <typename T>
T* export_vec(const std::vector<T>& v) {
  T* p = (T*)std::malloc(v.size() * sizeof(T) + 1);
  if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}
}  // namespace

void vsgm::set_host_error(const std::string& msg) { g_err = msg; }

extern "C" {

const char* vsgm_last_error(void) { return g_err.c_str(); }

void vsgm_free(void* p) { std::free(p); }

int vsgm_plan_pattern(int pattern_id, vsgm_plan* out) {
  if (!out) return fail(VSGM_EINVAL, "null output plan");
  vsgm::Query q;
  if (!vsgm::Query::preset(pattern_id, &q)) return fail(VSGM_EINVAL, "pattern id must be 0..18");
  std::string err;
  if (!vsgm::build_plan(q, nullptr, out, &err)) return fail(VSGM_EINVAL, err);
  return VSGM_OK;
}

int vsgm_plan_clique(int k, vsgm_plan* out) {
  if (!out) return fail(VSGM_EINVAL, "null output plan");
  vsgm::Query q;
  if (!vsgm::Query::clique(k, &q)) return fail(VSGM_EINVAL, "clique size must be 3..7");
  std::string err;
  if (!vsgm::build_plan(q, nullptr, out, &err)) return fail(VSGM_EINVAL, err);
  return VSGM_OK;
}

int vsgm_plan_query(int n, const uint8_t* adj_bits, vsgm_plan* out) {
  if (!out || !adj_bits) return fail(VSGM_EINVAL, "null argument");
  vsgm::Query q;
  if (!vsgm::Query::from_bits(n, adj_bits, &q)) return fail(VSGM_EINVAL, "pattern must be a connected simple graph on 2..7 vertices");
  std::string err;
  if (!vsgm::build_plan(q, nullptr, out, &err)) return fail(VSGM_EINVAL, err);
  return VSGM_OK;
}

int vsgm_plan_graphlets(int k, vsgm_plan* out, int cap, int* n_out) {
  if (k < 3 || k > 5) return fail(VSGM_EINVAL, "graphlet size must be 3..5");
  auto qs = vsgm::Query::graphlets(k);
  if (n_out) *n_out = (int)qs.size();
  std::string err;
  for (int i = 0; i < (int)qs.size() && i < cap; i++)
    if (!vsgm::build_plan(qs[i], nullptr, out + i, &err)) return fail(VSGM_EINVAL, err);
  return VSGM_OK;
}

int vsgm_plan_reorder(const vsgm_plan* base, const uint8_t* seq, vsgm_plan* out) {
  if (!base || !seq || !out) return fail(VSGM_EINVAL, "null argument");
  vsgm::Query q;
  const int n = (int)base->n_vertices;
  q.adj.assign(n, {});
  q.cond.assign(n, std::vector<uint8_t>(n, VSGM_NON_EQUAL));
  int m = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      if (base->adj[i] >> j & 1) {
        q.adj[i].push_back(j);
        if (i < j) m++;
      }
      if (i != j) q.cond[i][j] = base->order[i][j];
    }
  q.n_edges = m;
  int s[VSGM_MAX_QV];
  for (int i = 0; i < n; i++) s[i] = seq[i];
  std::string err;
  if (!vsgm::build_plan(q, s, out, &err)) return fail(VSGM_EINVAL, err);
  return VSGM_OK;
}

uint64_t vsgm_plan_automorphisms(const vsgm_plan* p) { return p ? vsgm::automorphism_count(*p) : 0; }

int vsgm_read_csr_bin(const char* path, uint64_t* V, uint64_t* E, uint64_t** row_ptrs, uint32_t** cols) {
  if (!path || !V || !E || !row_ptrs || !cols) return fail(VSGM_EINVAL, "null argument");
  std::string err;
  uint64_t nv = 0, ne = 0;
  if (!vsgm::csr_bin_header(path, &nv, &ne, &err)) return fail(VSGM_EIO, err);
  uint64_t* rp = (uint64_t*)std::malloc(sizeof(uint64_t) * (nv + 1));
  uint32_t* ci = (uint32_t*)std::malloc(sizeof(uint32_t) * ne + 1);
  if (!rp || !ci) {
    std::free(rp);
    std::free(ci);
    return fail(VSGM_ENOMEM, "host allocation failed");
  }
  if (!vsgm::read_csr_bin_into(path, nv, ne, rp, ci, 0, &err)) {
    std::free(rp);
    std::free(ci);
    return fail(VSGM_EIO, err);
  }
  *V = nv;
  *E = ne;
  *row_ptrs = rp;
  *cols = ci;
  return VSGM_OK;
}

int vsgm_csr_bin_header(const char* path, uint64_t* V, uint64_t* E) {
  if (!path || !V || !E) return fail(VSGM_EINVAL, "null argument");
  std::string err;
  if (!vsgm::csr_bin_header(path, V, E, &err)) return fail(VSGM_EIO, err);
  return VSGM_OK;
}

int vsgm_read_csr_bin_into(const char* path, uint64_t V, uint64_t E, uint64_t* row_ptrs, uint32_t* cols, int threads) {
  if (!path || !row_ptrs || (E && !cols)) return fail(VSGM_EINVAL, "null argument");
  std::string err;
  if (!vsgm::read_csr_bin_into(path, V, E, row_ptrs, cols, threads, &err)) return fail(VSGM_EIO, err);
  return VSGM_OK;
}

int vsgm_write_csr_bin(const char* path, uint64_t V, uint64_t E, const uint64_t* row_ptrs, const uint32_t* cols) {
  if (!path || !row_ptrs || (!cols && E)) return fail(VSGM_EINVAL, "null argument");
  if (row_ptrs[V] != E) return fail(VSGM_EINVAL, "row_ptrs[V] != E");
  vsgm::Csr g;
  g.V = V;
  g.row_ptrs.assign(row_ptrs, row_ptrs + V + 1);
  g.cols.assign(cols, cols + E);
  std::string err;
  if (!vsgm::write_csr_bin(path, g, &err)) return fail(VSGM_EIO, err);
  return VSGM_OK;
}

int vsgm_read_vbmap(const char* path, uint64_t V, int32_t* bins, int32_t* n_bins) {
  if (!path || !bins || !n_bins) return fail(VSGM_EINVAL, "null argument");
  std::vector<int32_t> b;
  std::string err;
  if (!vsgm::read_vbmap(path, V, &b, n_bins, &err)) return fail(VSGM_EIO, err);
  std::memcpy(bins, b.data(), V * sizeof(int32_t));
  return VSGM_OK;
}

int vsgm_write_vbmap(const char* path, uint64_t V, const int32_t* bins, int32_t n_bins) {
  if (!path || !bins) return fail(VSGM_EINVAL, "null argument");
  std::string err;
  if (!vsgm::write_vbmap(path, std::vector<int32_t>(bins, bins + V), n_bins, &err)) return fail(VSGM_EIO, err);
  return VSGM_OK;
}

uint64_t vsgm_csr_defects(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols) {
  vsgm::Csr g;
  g.V = V;
  g.row_ptrs.assign(row_ptrs, row_ptrs + V + 1);
  g.cols.assign(cols, cols + row_ptrs[V]);
  return vsgm::csr_defects(g);
}

int vsgm_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int threads, uint64_t* V, uint64_t* E,
                  uint64_t** row_ptrs, uint32_t** cols) {
  if (scale < 1 || scale > 31 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1) return fail(VSGM_EINVAL, "bad R-MAT parameters");
  vsgm::Csr g;
  vsgm::gen_rmat(scale, edge_factor, a, b, c, seed, threads, &g);
  *V = g.V;
  *E = g.E();
  *row_ptrs = export_vec(g.row_ptrs);
  *cols = export_vec(g.cols);
  if (!*row_ptrs || !*cols) return fail(VSGM_ENOMEM, "host allocation failed");
  return VSGM_OK;
}

int vsgm_gen_chung_lu(uint64_t V, uint64_t target_edges, double gamma, uint64_t max_degree, uint64_t seed, int threads, uint64_t* E,
                      uint64_t** row_ptrs, uint32_t** cols) {
  if (V < 2 || V > 0xFFFFFFFFull || gamma <= 1.0 || max_degree < 1) return fail(VSGM_EINVAL, "bad Chung-Lu parameters");
  vsgm::Csr g;
  vsgm::gen_chung_lu(V, target_edges, gamma, max_degree, seed, threads, &g);
  *E = g.E();
  *row_ptrs = export_vec(g.row_ptrs);
  *cols = export_vec(g.cols);
  if (!*row_ptrs || !*cols) return fail(VSGM_ENOMEM, "host allocation failed");
  return VSGM_OK;
}

int vsgm_degree_relabel(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, int ascending, int threads, uint32_t* new_of_old,
                        uint64_t* row_ptrs_out, uint32_t* cols_out) {
  if (!row_ptrs || (row_ptrs[V] && !cols) || !new_of_old || !row_ptrs_out || (row_ptrs[V] && !cols_out)) return fail(VSGM_EINVAL, "null argument");
  vsgm::Csr g, h;
  g.V = V;
  g.row_ptrs.assign(row_ptrs, row_ptrs + V + 1);
  g.cols.assign(cols, cols + row_ptrs[V]);
  std::vector<uint32_t> perm;
  vsgm::degree_relabel(g, ascending != 0, threads, &perm, &h);
  std::memcpy(new_of_old, perm.data(), V * sizeof(uint32_t));
  std::memcpy(row_ptrs_out, h.row_ptrs.data(), (V + 1) * sizeof(uint64_t));
  if (h.cols.size()) std::memcpy(cols_out, h.cols.data(), h.cols.size() * sizeof(uint32_t));
  return VSGM_OK;
}

int vsgm_random_pattern(int n_min, int n_max, double p, uint64_t seed, uint64_t* counter, int* n, uint8_t* adj_bits) {
  if (n_min < 2 || n_max > VSGM_MAX_QV || n_min > n_max || p <= 0 || !counter || !n || !adj_bits) return fail(VSGM_EINVAL, "bad pattern parameters");
  vsgm::random_pattern(n_min, n_max, p, seed, counter, n, adj_bits);
  return VSGM_OK;
}

int vsgm_view_compact(uint64_t V, const uint64_t* row_ptrs, uint32_t* vertices, uint64_t* offsets, uint64_t* n_vertices) {
  if (!row_ptrs || !vertices || !offsets || !n_vertices) return fail(VSGM_EINVAL, "null argument");
  uint64_t n = 0;
  offsets[0] = 0;
  for (uint64_t v = 0; v < V; v++) {
    const uint64_t d = row_ptrs[v + 1] - row_ptrs[v];
    if (!d) continue;
    if (row_ptrs[v] != offsets[n]) return fail(VSGM_EINVAL, "row_ptrs[0] must be 0 and rows contiguous");
    vertices[n] = (uint32_t)v;
    offsets[n + 1] = offsets[n] + d;
    n++;
  }
  *n_vertices = n;
  return VSGM_OK;
}

int vsgm_view_materialize(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, const uint32_t* sources, uint64_t n_sources, int hop,
                          uint64_t root_degree, int threads, uint64_t* view_row_ptrs, uint32_t* view_cols, uint64_t cols_cap, uint64_t* n_cols) {
  if (!row_ptrs || !view_row_ptrs || !n_cols || (n_sources && !sources) || hop < 1) return fail(VSGM_EINVAL, "bad view arguments");
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= V) return fail(VSGM_EINVAL, "source id out of range");
  if (!vsgm::materialize_view(row_ptrs, cols, V, sources, n_sources, hop, root_degree, threads, view_row_ptrs, view_cols, cols_cap, n_cols))
    return fail(VSGM_ENOMEM, "view needs " + std::to_string(*n_cols) + " adjacency entries, capacity is " + std::to_string(cols_cap));
  return VSGM_OK;
}

}  // extern "C"
