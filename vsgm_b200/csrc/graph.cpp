// Host-side graph layer (see graph.hpp).
#include "graph.hpp"

#include <fcntl.h>
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <utility>

namespace vsgm {

uint64_t mix64(uint64_t seed, uint64_t i) {
  // splitmix64 finaliser over a seed-salted counter
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + i * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double unit_double(uint64_t seed, uint64_t i) { return (double)(mix64(seed, i) >> 11) * (1.0 / 9007199254740992.0); }

static int nthreads(int t) { return t > 0 ? t : omp_get_max_threads(); }

void csr_from_edges(uint64_t V, std::vector<uint32_t>&& src, std::vector<uint32_t>&& dst, int threads, Csr* out) {
  // Symmetrise, drop self loops and duplicates, sort every row.  Both copies of
  // every edge are first partitioned by the block of 2^16 rows their source falls
  // in (per-thread counts, no atomics), then each block is counting-sorted by row
  // with block-local counters that stay in cache, and its rows are sorted and
  // de-duplicated.  The result depends only on the edge set.
  const int T = nthreads(threads);
  const uint64_t m = src.size();
  constexpr int kShift = 16;
  const uint64_t B = (V >> kShift) + 1;
  auto slice = [&](int t, uint64_t* lo, uint64_t* hi) {
    *lo = m * (uint64_t)t / (uint64_t)T;
    *hi = m * (uint64_t)(t + 1) / (uint64_t)T;
  };
  std::vector<uint64_t> cnt((size_t)T * B, 0);
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    uint64_t lo, hi;
    slice(t, &lo, &hi);
    uint64_t* c = cnt.data() + (size_t)t * B;
    for (uint64_t i = lo; i < hi; i++) {
      const uint32_t a = src[i], b = dst[i];
      if (a == b) continue;
      c[a >> kShift]++;
      c[b >> kShift]++;
    }
  }
  std::vector<uint64_t> boff(B + 1, 0);
  {
    uint64_t run = 0;
    for (uint64_t b = 0; b < B; b++) {
      boff[b] = run;
      for (int t = 0; t < T; t++) {
        const uint64_t n = cnt[(size_t)t * B + b];
        cnt[(size_t)t * B + b] = run;  // becomes this thread's write cursor in block b
        run += n;
      }
    }
    boff[B] = run;
  }
  std::vector<uint64_t> pairs(boff[B]);  // (row << 32) | neighbour
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    uint64_t lo, hi;
    slice(t, &lo, &hi);
    uint64_t* cur = cnt.data() + (size_t)t * B;
    for (uint64_t i = lo; i < hi; i++) {
      const uint32_t a = src[i], b = dst[i];
      if (a == b) continue;
      pairs[cur[a >> kShift]++] = ((uint64_t)a << 32) | b;
      pairs[cur[b >> kShift]++] = ((uint64_t)b << 32) | a;
    }
  }
  // the edge lists are consumed: release them before the next buffer (peak host
  // memory stays at pairs + edge lists, then pairs + rows, then rows + result)
  std::vector<uint32_t>().swap(src);
  std::vector<uint32_t>().swap(dst);
  // per block: rows by counting sort, then sort + unique each row
  std::vector<uint32_t> tmp(boff[B]);
  std::vector<uint64_t> start(V + 1, 0), kept(V, 0), bkept(B + 1, 0);
#pragma omp parallel num_threads(T)
  {
    std::vector<uint64_t> pos;
#pragma omp for schedule(dynamic, 1)
    for (int64_t b = 0; b < (int64_t)B; b++) {
      const uint64_t v0 = (uint64_t)b << kShift, v1 = std::min<uint64_t>(V, v0 + (1ull << kShift));
      if (v0 >= v1) continue;
      pos.assign(v1 - v0 + 1, 0);
      for (uint64_t k = boff[b]; k < boff[b + 1]; k++) pos[(pairs[k] >> 32) - v0 + 1]++;
      pos[0] = boff[b];
      for (uint64_t r = 1; r <= v1 - v0; r++) pos[r] += pos[r - 1];
      for (uint64_t r = 0; r < v1 - v0; r++) start[v0 + r] = pos[r];
      for (uint64_t k = boff[b]; k < boff[b + 1]; k++) tmp[pos[(pairs[k] >> 32) - v0]++] = (uint32_t)pairs[k];
      uint64_t sum = 0;
      for (uint64_t v = v0; v < v1; v++) {
        uint32_t* rb = tmp.data() + start[v];
        uint32_t* re = tmp.data() + (v + 1 < v1 ? start[v + 1] : boff[b + 1]);
        std::sort(rb, re);
        kept[v] = (uint64_t)(std::unique(rb, re) - rb);
        sum += kept[v];
      }
      bkept[b + 1] = sum;
    }
  }
  std::vector<uint64_t>().swap(pairs);
  for (uint64_t b = 0; b < B; b++) bkept[b + 1] += bkept[b];
  out->V = V;
  out->row_ptrs.assign(V + 1, 0);
  out->cols.resize(bkept[B]);
#pragma omp parallel for num_threads(T) schedule(dynamic, 1)
  for (int64_t b = 0; b < (int64_t)B; b++) {
    const uint64_t v0 = (uint64_t)b << kShift, v1 = std::min<uint64_t>(V, v0 + (1ull << kShift));
    uint64_t at = bkept[b];
    for (uint64_t v = v0; v < v1; v++) {
      out->row_ptrs[v] = at;
      std::memcpy(out->cols.data() + at, tmp.data() + start[v], kept[v] * sizeof(uint32_t));
      at += kept[v];
    }
  }
  out->row_ptrs[V] = bkept[B];
}

void gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int threads, Csr* out) {
  const uint64_t V = 1ull << scale;
  const uint64_t m = (uint64_t)edge_factor << scale;
  std::vector<uint32_t> src(m), dst(m);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (int64_t i = 0; i < (int64_t)m; i++) {
    uint64_t s = 0, d = 0;
    for (int l = 0; l < scale; l++) {
      double r = unit_double(seed, (uint64_t)i * 64 + l);
      s <<= 1;
      d <<= 1;
      if (r < a) {
      } else if (r < ab) {
        d |= 1;
      } else if (r < abc) {
        s |= 1;
      } else {
        s |= 1;
        d |= 1;
      }
    }
    src[i] = (uint32_t)s;
    dst[i] = (uint32_t)d;
  }
  csr_from_edges(V, std::move(src), std::move(dst), threads, out);
}

void gen_chung_lu(uint64_t V, uint64_t target_edges, double gamma, uint64_t dmax, uint64_t seed, int threads, Csr* out) {
  const int T = nthreads(threads);
  const double beta = 1.0 / (gamma - 1.0);
  // sum of w for offset i0, by direct summation (V up to ~1e8 is fine)
  auto total = [&](double i0) {
    double s = 0;
#pragma omp parallel for num_threads(T) reduction(+ : s)
    for (int64_t i = 0; i < (int64_t)V; i++) s += (double)dmax * std::pow((i + i0) / i0, -beta);
    return s;
  };
  const double want = 2.0 * (double)target_edges;
  double lo = 1e-3, hi = (double)V * 4;
  for (int it = 0; it < 80; it++) {
    double mid = std::sqrt(lo * hi);
    if (total(mid) < want)
      lo = mid;
    else
      hi = mid;
  }
  const double i0 = std::sqrt(lo * hi);
  std::vector<double> cdf(V);
  {
    double s = 0;
    for (uint64_t i = 0; i < V; i++) {
      s += (double)dmax * std::pow((i + i0) / i0, -beta);
      cdf[i] = s;
    }
    for (uint64_t i = 0; i < V; i++) cdf[i] /= s;
    cdf[V - 1] = 1.0;
  }
  // Inverse-CDF sampling through a bucket index: bucket k covers r in [k/K, (k+1)/K)
  // and idx[k] = upper_bound(cdf, k/K), so upper_bound(cdf, r) lies in
  // [idx[k], idx[k+1]] and the short search there returns exactly what a search
  // over the whole array would (same graphs as before, without walking a
  // cache-missing binary search over all V entries per endpoint).
  const uint64_t K = std::max<uint64_t>(1, std::min<uint64_t>(V, 1ull << 26));
  auto edge_of = [K](uint64_t k) { return (double)k / (double)K; };
  std::vector<uint64_t> idx(K + 1);
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t k = 0; k <= (int64_t)K; k++) idx[k] = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), edge_of((uint64_t)k)) - cdf.begin());
  auto sample = [&](double r) -> uint32_t {
    uint64_t k = (uint64_t)(r * (double)K);
    if (k >= K) k = K - 1;
    while (k > 0 && edge_of(k) > r) k--;
    while (k + 1 < K && edge_of(k + 1) <= r) k++;
    const uint64_t pos = (uint64_t)(std::upper_bound(cdf.begin() + idx[k], cdf.begin() + idx[k + 1], r) - cdf.begin());
    return (uint32_t)(pos >= V ? V - 1 : pos);
  };
  const uint64_t m = target_edges;
  std::vector<uint32_t> src(m), dst(m);
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t i = 0; i < (int64_t)m; i++) {
    src[i] = sample(unit_double(seed, 2 * (uint64_t)i));
    dst[i] = sample(unit_double(seed, 2 * (uint64_t)i + 1));
  }
  csr_from_edges(V, std::move(src), std::move(dst), threads, out);
}

bool csr_bin_header(const std::string& path, uint64_t* V, uint64_t* E, std::string* err) {
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) {
    if (err) *err = "cannot open " + path;
    return false;
  }
  uint64_t hdr[4];
  struct stat st;
  const bool got = ::pread(fd, hdr, sizeof(hdr), 0) == (ssize_t)sizeof(hdr) && ::fstat(fd, &st) == 0;
  ::close(fd);
  if (!got) {
    if (err) *err = "truncated or inconsistent csr file " + path;
    return false;
  }
  if (hdr[0] != 4 || hdr[1] != 8) {
    if (err) *err = "unsupported id widths in " + path;
    return false;
  }
  // the sizes must describe the file exactly (and must not overflow doing so)
  const uint64_t Vn = hdr[2], En = hdr[3];
  if (Vn >= (1ull << 40) || En >= (1ull << 60) || (uint64_t)st.st_size != 32 + 8 * (Vn + 1) + 4 * En) {
    if (err) *err = "truncated or inconsistent csr file " + path;
    return false;
  }
  *V = Vn;
  *E = En;
  return true;
}

// read len bytes at off into dst in chunks spread over T threads
static bool pread_all(int fd, char* dst, uint64_t off, uint64_t len, int T) {
  const uint64_t chunk = 64ull << 20;
  const int64_t n = (int64_t)((len + chunk - 1) / chunk);
  std::atomic<bool> ok{true};
#pragma omp parallel for num_threads(T) schedule(dynamic, 1)
  for (int64_t k = 0; k < n; k++) {
    uint64_t a = (uint64_t)k * chunk, z = std::min<uint64_t>(len, a + chunk);
    while (a < z && ok.load(std::memory_order_relaxed)) {
      const ssize_t r = ::pread(fd, dst + a, z - a, (off_t)(off + a));
      if (r <= 0) {
        ok = false;
        break;
      }
      a += (uint64_t)r;
    }
  }
  return ok.load();
}

bool read_csr_bin_into(const std::string& path, uint64_t V, uint64_t E, uint64_t* row_ptrs, uint32_t* cols, int threads, std::string* err) {
  uint64_t fv = 0, fe = 0;
  if (!csr_bin_header(path, &fv, &fe, err)) return false;
  if (fv != V || fe != E) {
    if (err) *err = "csr file " + path + " does not have the expected sizes";
    return false;
  }
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) {
    if (err) *err = "cannot open " + path;
    return false;
  }
  const int T = nthreads(threads);
  bool ok = pread_all(fd, (char*)row_ptrs, 32, 8 * (V + 1), T) && pread_all(fd, (char*)cols, 32 + 8 * (V + 1), 4 * E, T);
  ::close(fd);
  ok = ok && row_ptrs[V] == E;
  if (!ok && err) *err = "truncated or inconsistent csr file " + path;
  return ok;
}

bool read_csr_bin(const std::string& path, Csr* out, std::string* err) {
  uint64_t V = 0, E = 0;
  if (!csr_bin_header(path, &V, &E, err)) return false;
  out->V = V;
  out->row_ptrs.resize(V + 1);
  out->cols.resize(E);
  return read_csr_bin_into(path, V, E, out->row_ptrs.data(), out->cols.data(), 0, err);
}

bool write_csr_bin(const std::string& path, const Csr& g, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    if (err) *err = "cannot create " + path;
    return false;
  }
  uint64_t hdr[4] = {4, 8, g.V, g.E()};
  bool ok = std::fwrite(hdr, sizeof(uint64_t), 4, f) == 4;
  ok = ok && std::fwrite(g.row_ptrs.data(), sizeof(uint64_t), g.V + 1, f) == g.V + 1;
  ok = ok && std::fwrite(g.cols.data(), sizeof(uint32_t), g.E(), f) == g.E();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok && err) *err = "write failed for " + path;
  return ok;
}

// The whole file is read at once and parsed by hand: decimal integers separated by
// whitespace, the first being the number of bins (the reference streams it with
// operator>>, src/view/view_bin_manager.h:37-41).
static bool next_int(const char*& p, const char* end, int64_t* out) {
  while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
  if (p >= end) return false;
  bool neg = false;
  if (*p == '-') {
    neg = true;
    p++;
  }
  if (p >= end || *p < '0' || *p > '9') return false;
  int64_t v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    v = v * 10 + (*p - '0');
    if (v > (1ll << 40)) return false;
    p++;
  }
  *out = neg ? -v : v;
  return true;
}

bool read_vbmap(const std::string& path, uint64_t V, std::vector<int32_t>* bins, int32_t* n_bins, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    if (err) *err = "cannot open " + path;
    return false;
  }
  std::string buf;
  {
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n : 0);
    const bool ok = n >= 0 && std::fread(&buf[0], 1, buf.size(), f) == buf.size();
    std::fclose(f);
    if (!ok) {
      if (err) *err = "cannot read " + path;
      return false;
    }
  }
  const char* p = buf.data();
  const char* end = p + buf.size();
  int64_t nb = 0;
  if (!next_int(p, end, &nb) || nb < 0 || nb > 0x7fffffff) {
    if (err) *err = "bad bin count in " + path;
    return false;
  }
  bins->resize(V);
  for (uint64_t i = 0; i < V; i++) {
    int64_t b;
    if (!next_int(p, end, &b) || b < 0 || b >= nb) {
      if (err) *err = "bad or missing bin id for vertex " + std::to_string(i) + " in " + path;
      return false;
    }
    (*bins)[i] = (int32_t)b;
  }
  *n_bins = (int32_t)nb;
  return true;
}

bool write_vbmap(const std::string& path, const std::vector<int32_t>& bins, int32_t n_bins, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    if (err) *err = "cannot create " + path;
    return false;
  }
  std::string out;
  out.reserve(12 * (bins.size() + 1));
  auto put = [&](int64_t v) {
    char tmp[24];
    int n = 0;
    bool neg = v < 0;
    uint64_t u = neg ? (uint64_t)(-v) : (uint64_t)v;
    do {
      tmp[n++] = (char)('0' + u % 10);
      u /= 10;
    } while (u);
    if (neg) out.push_back('-');
    while (n) out.push_back(tmp[--n]);
    out.push_back('\n');
  };
  put(n_bins);
  for (int32_t b : bins) put(b);
  bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok && err) *err = "write failed for " + path;
  return ok;
}

uint64_t csr_defects(const Csr& g) {
  uint64_t bad = 0;
  for (uint64_t v = 0; v < g.V; v++)
    for (uint64_t j = g.row_ptrs[v]; j < g.row_ptrs[v + 1]; j++) {
      if (g.cols[j] == v || g.cols[j] >= g.V) bad++;
      if (j > g.row_ptrs[v] && g.cols[j] <= g.cols[j - 1]) bad++;
    }
  return bad;
}

bool materialize_view(const uint64_t* row_ptrs, const uint32_t* cols, uint64_t V, const uint32_t* sources, uint64_t n_sources, int hop,
                      uint64_t root_degree, int threads, uint64_t* view_row_ptrs, uint32_t* view_cols, uint64_t cols_cap, uint64_t* n_cols) {
  const int T = nthreads(threads);
  std::vector<uint8_t> in_view(V, 0);
  std::vector<uint32_t> frontier;
  frontier.reserve(n_sources);
  for (uint64_t i = 0; i < n_sources; i++) {
    uint32_t s = sources[i];
    if (root_degree == 0 || row_ptrs[s + 1] - row_ptrs[s] >= root_degree) {
      if (!in_view[s]) frontier.push_back(s);
      in_view[s] = 1;
    }
  }
  // breadth-first layers: a vertex at distance < hop from a kept source gets its row;
  // the last layer only marks (no frontier is needed after it)
  for (int layer = 1; layer < hop; layer++) {
    const bool last = layer + 1 == hop;
    std::vector<std::vector<uint32_t>> next(T);
#pragma omp parallel num_threads(T)
    {
      auto& mine = next[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 256)
      for (int64_t i = 0; i < (int64_t)frontier.size(); i++) {
        uint32_t x = frontier[i];
        for (uint64_t j = row_ptrs[x]; j < row_ptrs[x + 1]; j++) {
          uint32_t y = cols[j];
          if (__atomic_load_n(&in_view[y], __ATOMIC_RELAXED)) continue;
          if (last)
            __atomic_store_n(&in_view[y], (uint8_t)1, __ATOMIC_RELAXED);
          else if (!__atomic_exchange_n(&in_view[y], (uint8_t)1, __ATOMIC_RELAXED))
            mine.push_back(y);
        }
      }
    }
    if (last) break;
    frontier.clear();
    for (auto& v : next) frontier.insert(frontier.end(), v.begin(), v.end());
  }
  // offsets: per-block sums, then the block prefix, then each block's own prefix
  const int64_t nb = (int64_t)((V + 65535) >> 16);
  std::vector<uint64_t> bsum(nb + 1, 0);
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t b = 0; b < nb; b++) {
    uint64_t s = 0;
    for (uint64_t v = (uint64_t)b << 16; v < std::min<uint64_t>(V, ((uint64_t)b + 1) << 16); v++)
      if (in_view[v]) s += row_ptrs[v + 1] - row_ptrs[v];
    bsum[b + 1] = s;
  }
  for (int64_t b = 0; b < nb; b++) bsum[b + 1] += bsum[b];
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t b = 0; b < nb; b++) {
    uint64_t at = bsum[b];
    for (uint64_t v = (uint64_t)b << 16; v < std::min<uint64_t>(V, ((uint64_t)b + 1) << 16); v++) {
      view_row_ptrs[v] = at;
      if (in_view[v]) at += row_ptrs[v + 1] - row_ptrs[v];
    }
  }
  const uint64_t total = bsum[nb];
  view_row_ptrs[V] = total;
  *n_cols = total;
  if (total > cols_cap) return false;
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)V; v++)
    if (in_view[v]) std::memcpy(view_cols + view_row_ptrs[v], cols + row_ptrs[v], (row_ptrs[v + 1] - row_ptrs[v]) * sizeof(uint32_t));
  return true;
}

void degree_relabel(const Csr& g, bool ascending, int threads, std::vector<uint32_t>* new_of_old, Csr* out) {
  const int T = nthreads(threads);
  const uint64_t V = g.V;
  auto deg = [&](uint32_t v) { return g.row_ptrs[v + 1] - g.row_ptrs[v]; };
  // rank by (degree, id): a counting sort over degrees, ids ascending inside each
  // degree (the order a stable sort by degree gives)
  uint64_t dmax = 0;
  for (uint64_t v = 0; v < V; v++) dmax = std::max<uint64_t>(dmax, deg((uint32_t)v));
  std::vector<uint64_t> at(dmax + 2, 0);
  for (uint64_t v = 0; v < V; v++) at[(ascending ? deg((uint32_t)v) : dmax - deg((uint32_t)v)) + 1]++;
  for (uint64_t d = 0; d <= dmax; d++) at[d + 1] += at[d];
  std::vector<uint32_t> order(V);
  for (uint64_t v = 0; v < V; v++) order[at[ascending ? deg((uint32_t)v) : dmax - deg((uint32_t)v)]++] = (uint32_t)v;
  new_of_old->assign(V, 0);
  for (uint64_t r = 0; r < V; r++) (*new_of_old)[order[r]] = (uint32_t)r;
  out->V = V;
  out->row_ptrs.assign(V + 1, 0);
  for (uint64_t r = 0; r < V; r++) out->row_ptrs[r + 1] = out->row_ptrs[r] + deg(order[r]);
  out->cols.resize(g.cols.size());
  const std::vector<uint32_t>& nmap = *new_of_old;
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int64_t r = 0; r < (int64_t)V; r++) {
    const uint32_t v = order[r];
    uint32_t* dst = out->cols.data() + out->row_ptrs[r];
    uint64_t n = 0;
    for (uint64_t j = g.row_ptrs[v]; j < g.row_ptrs[v + 1]; j++) dst[n++] = nmap[g.cols[j]];
    std::sort(dst, dst + n);
  }
}

void random_pattern(int n_min, int n_max, double p, uint64_t seed, uint64_t* counter, int* n_out, uint8_t bits[7]) {
  auto next = [&]() { return unit_double(seed, (*counter)++); };
  while (true) {
    int n = n_min + (int)(next() * (n_max - n_min + 1));
    if (n > n_max) n = n_max;
    std::memset(bits, 0, 7);
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++)
        if (next() < p) {
          bits[i] |= (uint8_t)(1u << j);
          bits[j] |= (uint8_t)(1u << i);
        }
    uint32_t seen = 1, grow = 1;
    while (grow) {
      uint32_t add = 0;
      for (int i = 0; i < n; i++)
        if (seen >> i & 1) add |= bits[i];
      grow = add & ~seen;
      seen |= add;
    }
    if (seen == (1u << n) - 1) {
      *n_out = n;
      return;
    }
  }
}

}  // namespace vsgm
