/* CPU ORACLE - test infrastructure only.
 *
 * Nothing in the product links, imports or executes this file.  It is used by
 * tests/ (to check results), by __graft_entry__.smoke() and by bench.py's CPU
 * baseline / reference arm.
 *
 * 1. oracle_count: a restatement of the reference executor for one plan, one
 *    view (CSR) and its sources.  The reference runs the execution sequence
 *    level by level over memory-bounded batches; batching never changes a
 *    count, and every op acts on each partial match independently, so this
 *    restatement walks the same sequence depth-first per root, with the same
 *    per-path semantics:
 *      MATERIALIZE at level 0  src/executor/ops/materialize.h:11-18
 *      COMPUTE                 src/executor/ops/compute.h:7-41 and the GPSM
 *                              traversal src/gpu/gpu_utils_gpsm_bin_search.h:14-130
 *                              (pivot = backward neighbour of least degree,
 *                              src/gpu/gpu_check_constraints_common.h:11-29;
 *                              membership by lower-bound search, :32-53 and
 *                              src/gpu/gpu_utils_bin_search.h:17-29)
 *      MATERIALIZE             src/executor/ops/materialize.h:20-126
 *      FILTER_COMPUTE          src/executor/ops/filter_compute.h:14-127
 *      COMPUTE_COUNT           src/executor/ops/compute_count.h:9-84 with
 *                              ThreadCountWithComputedVertex
 *                              src/gpu/gpu_check_constraints_common.h:120-139
 *      COUNT                   src/executor/ops/count.h:16-167
 *      COMPUTE_PATH_COUNT      src/executor/ops/compute_path_count.h:7-49 (sizes
 *                              only; never emitted by the reference planner)
 *      conditions              src/gpu/gpu_utils_filter.h:11-23
 *    OpenMP parallelises over roots.
 * 2. oracle_bruteforce: independent ground truth - injective edge-preserving
 *    maps P -> G divided by |Aut(P)|; small graphs only.
 * 3. oracle_op_paths: number of partial matches entering every op (summed over
 *    roots), used to check the engine's per-level statistics.
 * 4. oracle_c4_by_largest: 4-cycles whose largest vertex is one of the given
 *    sources, by pairwise neighbour intersections - the attribution the engine's
 *    wedge-aggregation operator uses (the reference's 4-cycle plan attributes a
 *    cycle to its smallest vertex; totals over all vertices agree).
 *    oracle_c4_by_largest_wedges: the same count by wedge counting, fast enough
 *    for hub roots of the full-size graphs; pinned to the pairwise form.
 * 5. oracle_cliques_by_smallest: k-cliques whose smallest vertex is a source, by
 *    definition (ordered candidate sets) - the clique plans' per-root attribution,
 *    fast on hub roots; pinned to oracle_count root by root.
 * 6. oracle_gen_rmat / oracle_degree_relabel: the benchmark's synthetic input
 *    (R-MAT graph, ids ascending with degree), so that the timed CPU baseline
 *    needs nothing from the product library.
 * 7. oracle_tools.cc (same library): the reference's offline view-bin tools
 *    restated, kmeans -init 1 and view_packing -s 1; pinned to the reference
 *    tools' own outputs (tests/golden/ref_view_tools.npz and the binaries built in
 *    oracle/_ref, tests/test_view_tools.py).
 *
 * Parity: the reference's matching path cannot be built here (its moderngpu and
 * MPMCQueue submodules are not vendored and it needs a GPU), and the reference
 * ships no golden counts.  This restatement is pinned instead by the brute-force
 * counter and by closed forms in tests/test_oracle.py; the plans it executes are
 * pinned to the reference planner's own output (tests/golden/ref_plans.jsonl).
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vsgm_plan.h"

typedef struct {
  const uint64_t* rp;
  const uint32_t* ci;
  const vsgm_plan* p;
  uint32_t M[VSGM_MAX_QV];
  const uint32_t* cand[VSGM_MAX_QV];
  uint64_t clen[VSGM_MAX_QV];
  uint32_t* buf[VSGM_MAX_OPS]; /* one candidate buffer per op */
  uint64_t total;
  uint64_t* op_paths; /* optional per-op partial-match counter */
} walk_t;

static uint64_t lower_bound_u32(const uint32_t* a, uint64_t n, uint32_t x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

static int cond_holds(uint8_t op, uint32_t a, uint32_t b) {
  switch (op) {
    case VSGM_LESS_THAN: return a < b;
    case VSGM_LARGER_THAN: return a > b;
    case VSGM_NON_EQUAL: return a != b;
    default: return 1;
  }
}

static int conds_hold(const vsgm_conds* c, const uint32_t* M, uint32_t x) {
  for (int i = 0; i < c->count; i++)
    if (!cond_holds(c->op[i], x, M[c->v[i]])) return 0;
  return 1;
}

/* candidates of u: members of N(M[pivot]) adjacent to every other backward
 * neighbour and satisfying the compute conditions, written to out in order */
static uint64_t intersect(walk_t* w, int u, uint32_t* out) {
  const vsgm_plan* p = w->p;
  const vsgm_vgroup* B = &p->backward[u];
  int pivot = B->v[0];
  uint64_t best = w->rp[w->M[pivot] + 1] - w->rp[w->M[pivot]];
  for (int i = 1; i < B->count; i++) {
    uint32_t v = w->M[B->v[i]];
    uint64_t d = w->rp[v + 1] - w->rp[v];
    if (best > d) {
      best = d;
      pivot = B->v[i];
    }
  }
  const uint32_t* list = w->ci + w->rp[w->M[pivot]];
  uint64_t n = 0;
  for (uint64_t k = 0; k < best; k++) {
    uint32_t c = list[k];
    int ok = 1;
    for (int i = 0; i < B->count && ok; i++) {
      if (B->v[i] == pivot) continue;
      uint32_t v = w->M[B->v[i]];
      const uint32_t* a = w->ci + w->rp[v];
      uint64_t len = w->rp[v + 1] - w->rp[v];
      uint64_t pos = lower_bound_u32(a, len, c);
      ok = (pos < len && a[pos] == c);
    }
    if (ok && conds_hold(&p->compute_cond[u], w->M, c)) out[n++] = c;
  }
  return n;
}

/* elements of a (sorted) that stand in relation op to x, x op a[j] */
static uint64_t count_vs_set(const uint32_t* a, uint64_t n, uint32_t x, uint8_t op) {
  if (n == 0) return 0;
  uint64_t pos = lower_bound_u32(a, n, x);
  int eq = pos < n && a[pos] == x;
  if (op == VSGM_LESS_THAN) return n - pos - (eq ? 1 : 0);
  if (op == VSGM_LARGER_THAN) return pos;
  return n - (eq ? 1 : 0);
}

static void run(walk_t* w, int i) {
  const vsgm_plan* p = w->p;
  if (i == (int)p->n_ops) return;
  if (w->op_paths) w->op_paths[i]++;
  const int u = p->op_vertex[i];
  switch (p->op_type[i]) {
    case VSGM_COMPUTE: {
      uint64_t n = intersect(w, u, w->buf[i]);
      const uint32_t* old = w->cand[u];
      uint64_t oldn = w->clen[u];
      w->cand[u] = w->buf[i];
      w->clen[u] = n;
      run(w, i + 1);
      w->cand[u] = old;
      w->clen[u] = oldn;
    } break;
    case VSGM_MATERIALIZE: {
      const uint32_t* c = w->cand[u];
      uint64_t n = w->clen[u];
      for (uint64_t k = 0; k < n; k++)
        if (conds_hold(&p->materialize_cond[u], w->M, c[k])) {
          w->M[u] = c[k];
          run(w, i + 1);
        }
    } break;
    case VSGM_FILTER_COMPUTE: {
      const uint32_t* c = w->cand[u];
      uint64_t n = w->clen[u], m = 0;
      for (uint64_t k = 0; k < n; k++)
        if (conds_hold(&p->filter_cond[u], w->M, c[k])) w->buf[i][m++] = c[k];
      w->cand[u] = w->buf[i];
      w->clen[u] = m;
      run(w, i + 1);
      w->cand[u] = c;
      w->clen[u] = n;
    } break;
    case VSGM_COMPUTE_PATH_COUNT: {
      /* src/executor/ops/compute_path_count.h: the candidate set's size per path;
       * only a COUNT may read it, which reads the size alone */
      uint64_t n = intersect(w, u, w->buf[i]);
      const uint32_t* old = w->cand[u];
      uint64_t oldn = w->clen[u];
      w->cand[u] = w->buf[i];
      w->clen[u] = n;
      run(w, i + 1);
      w->cand[u] = old;
      w->clen[u] = oldn;
    } break;
    case VSGM_COMPUTE_COUNT: {
      uint64_t n = intersect(w, u, w->buf[i]);
      const vsgm_vgroup* um = &p->computed_unmat[i];
      if (um->count == 0) {
        w->total += n;
      } else {
        int o = um->v[0];
        uint8_t op = p->order[u][o];
        for (uint64_t k = 0; k < n; k++) w->total += count_vs_set(w->cand[o], w->clen[o], w->buf[i][k], op);
      }
    } break;
    case VSGM_COUNT: {
      const vsgm_vgroup* um = &p->computed_unmat[i];
      if (um->count == 1) {
        w->total += w->clen[um->v[0]];
      } else {
        int u0 = um->v[0], u1 = um->v[1];
        uint8_t op = p->order[u0][u1];
        uint64_t n0 = w->clen[u0], n1 = w->clen[u1];
        /* walk the smaller set, search the larger (src/executor/ops/count.h:16-107) */
        if (n0 <= n1) {
          for (uint64_t k = 0; k < n0; k++) w->total += count_vs_set(w->cand[u1], n1, w->cand[u0][k], op);
        } else {
          uint8_t rev = op == VSGM_LESS_THAN ? VSGM_LARGER_THAN : (op == VSGM_LARGER_THAN ? VSGM_LESS_THAN : op);
          for (uint64_t k = 0; k < n1; k++) w->total += count_vs_set(w->cand[u0], n0, w->cand[u1][k], rev);
        }
      }
    } break;
    default:
      break;
  }
}

static uint64_t max_degree(uint64_t V, const uint64_t* rp) {
  uint64_t d = 0;
  for (uint64_t v = 0; v < V; v++)
    if (rp[v + 1] - rp[v] > d) d = rp[v + 1] - rp[v];
  return d;
}

static uint64_t walk_all(const vsgm_plan* p, uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources,
                         int threads, uint64_t* op_paths) {
  const uint64_t dmax = max_degree(V, rp) + 1;
  const int T = threads > 0 ? threads : omp_get_max_threads();
  uint64_t total = 0;
  uint64_t paths[VSGM_MAX_OPS] = {0};
#pragma omp parallel num_threads(T) reduction(+ : total)
  {
    walk_t w;
    memset(&w, 0, sizeof(w));
    w.rp = rp;
    w.ci = ci;
    w.p = p;
    uint64_t mine[VSGM_MAX_OPS] = {0};
    w.op_paths = op_paths ? mine : NULL;
    for (uint32_t i = 0; i < p->n_ops; i++) w.buf[i] = (uint32_t*)malloc(dmax * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 64)
    for (int64_t s = 0; s < (int64_t)n_sources; s++) {
      w.M[p->op_vertex[0]] = sources[s];
      if (w.op_paths) mine[0]++;
      run(&w, 1);
    }
    for (uint32_t i = 0; i < p->n_ops; i++) free(w.buf[i]);
    total += w.total;
    if (op_paths) {
#pragma omp critical
      for (uint32_t i = 0; i < p->n_ops; i++) paths[i] += mine[i];
    }
  }
  if (op_paths)
    for (uint32_t i = 0; i < p->n_ops; i++) op_paths[i] = paths[i];
  return total;
}

uint64_t oracle_count(const vsgm_plan* p, uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources, int threads) {
  return walk_all(p, V, rp, ci, sources, n_sources, threads, NULL);
}

uint64_t oracle_op_paths(const vsgm_plan* p, uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources, int threads,
                         uint64_t* op_paths) {
  return walk_all(p, V, rp, ci, sources, n_sources, threads, op_paths);
}

/* ---------------------------------------------------------------- brute force */
typedef struct {
  const uint64_t* rp;
  const uint32_t* ci;
  int n;
  uint8_t adj[VSGM_MAX_QV];
  int order[VSGM_MAX_QV]; /* connected visiting order */
  uint32_t img[VSGM_MAX_QV];
  uint64_t maps;
} brute_t;

static int adjacent(const brute_t* b, uint32_t x, uint32_t y) {
  const uint32_t* a = b->ci + b->rp[x];
  uint64_t n = b->rp[x + 1] - b->rp[x];
  uint64_t pos = lower_bound_u32(a, n, y);
  return pos < n && a[pos] == y;
}

static void brute(brute_t* b, int k) {
  if (k == b->n) {
    b->maps++;
    return;
  }
  int u = b->order[k];
  /* an earlier-mapped neighbour of u supplies the candidates */
  int anchor = -1;
  for (int j = 0; j < k; j++)
    if (b->adj[u] >> b->order[j] & 1) {
      anchor = b->order[j];
      break;
    }
  uint32_t a = b->img[anchor];
  for (uint64_t e = b->rp[a]; e < b->rp[a + 1]; e++) {
    uint32_t x = b->ci[e];
    int ok = 1;
    for (int j = 0; j < k && ok; j++) {
      int w = b->order[j];
      if (b->img[w] == x) ok = 0;
      else if ((b->adj[u] >> w & 1) && w != anchor && !adjacent(b, x, b->img[w])) ok = 0;
    }
    if (ok) {
      b->img[u] = x;
      brute(b, k + 1);
    }
  }
}

/* injective edge-preserving maps of the pattern into G, divided by |Aut(P)| */
uint64_t oracle_bruteforce(const vsgm_plan* p, uint64_t V, const uint64_t* rp, const uint32_t* ci, uint64_t n_automorphisms, int threads) {
  const int n = (int)p->n_vertices;
  int order[VSGM_MAX_QV];
  {
    uint32_t seen = 1;
    order[0] = 0;
    for (int k = 1; k < n; k++)
      for (int u = 0; u < n; u++)
        if (!(seen >> u & 1) && (p->adj[u] & seen)) {
          order[k] = u;
          seen |= 1u << u;
          break;
        }
  }
  uint64_t maps = 0;
  const int T = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(T) reduction(+ : maps)
  {
    brute_t b;
    memset(&b, 0, sizeof(b));
    b.rp = rp;
    b.ci = ci;
    b.n = n;
    memcpy(b.adj, p->adj, sizeof(b.adj));
    memcpy(b.order, order, sizeof(order));
#pragma omp for schedule(dynamic, 16)
    for (int64_t v = 0; v < (int64_t)V; v++) {
      b.img[order[0]] = (uint32_t)v;
      brute(&b, 1);
    }
    maps += b.maps;
  }
  return n_automorphisms ? maps / n_automorphisms : 0;
}

/* 4-cycles u-v-w-v' whose largest vertex u is a source: for every pair v < v' of
 * neighbours of u below u, the common neighbours w of v and v' below u (w != u by
 * construction).  The opposite vertex and the pair {v, v'} fix the cycle, so each
 * is counted once. */
uint64_t oracle_c4_by_largest(uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources, int threads) {
  (void)V;
  uint64_t total = 0;
  const int T = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(T) schedule(dynamic, 16) reduction(+ : total)
  for (int64_t s = 0; s < (int64_t)n_sources; s++) {
    const uint32_t u = sources[s];
    for (uint64_t i = rp[u]; i < rp[u + 1] && ci[i] < u; i++)
      for (uint64_t j = i + 1; j < rp[u + 1] && ci[j] < u; j++) {
        const uint32_t v = ci[i], x = ci[j];
        uint64_t a = rp[v], b = rp[x];
        while (a < rp[v + 1] && b < rp[x + 1] && ci[a] < u && ci[b] < u) {
          if (ci[a] < ci[b])
            a++;
          else if (ci[a] > ci[b])
            b++;
          else {
            total++;
            a++;
            b++;
          }
        }
      }
  }
  return total;
}

/* The same count by wedge aggregation, for roots whose neighbourhoods are too large
 * for the pairwise form: for a source u, L[w] = number of wedges u-v-w with
 * v, w < u (w != u), and the cycles closed at u are sum_w C(L[w], 2) - a pair of
 * distinct wedge centres v, v' through the same opposite vertex w.  One dense
 * counter array per thread, reset through the list of the ids it touched.
 * tests/test_oracle.py pins it to oracle_c4_by_largest on small graphs. */
uint64_t oracle_c4_by_largest_wedges(uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources, int threads) {
  uint64_t total = 0;
  const int T = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(T) reduction(+ : total)
  {
    uint32_t* L = (uint32_t*)calloc(V ? V : 1, sizeof(uint32_t));
    uint32_t* touched = (uint32_t*)malloc((V ? V : 1) * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 1)
    for (int64_t s = 0; s < (int64_t)n_sources; s++) {
      const uint32_t u = sources[s];
      uint64_t nt = 0;
      for (uint64_t i = rp[u]; i < rp[u + 1] && ci[i] < u; i++) {
        const uint32_t v = ci[i];
        for (uint64_t j = rp[v]; j < rp[v + 1] && ci[j] < u; j++)
          if (L[ci[j]]++ == 0) touched[nt++] = ci[j];
      }
      for (uint64_t k = 0; k < nt; k++) {
        const uint64_t c = L[touched[k]];
        total += c * (c - 1) / 2;
        L[touched[k]] = 0;
      }
    }
    free(L);
    free(touched);
  }
  return total;
}

/* ---------------------------------------------------------------- rooted cliques */
/* k-cliques whose smallest vertex is a source - the attribution of the reference's
 * clique plans, whose order conditions chain v0 < v1 < ... < v(k-1)
 * (src/query/clique.h with the partial order of src/query/partial_order.h).  An
 * independent count, by definition rather than by the plan: candidates at each
 * depth are the previous set's members above the vertex just chosen that are also
 * its neighbours, found by a merge that starts both lists at the first value above
 * that vertex (so hub rows are never walked in full).  tests/test_oracle.py pins it
 * to oracle_count on the clique plans, root by root. */
static uint64_t clique_rec(const uint64_t* rp, const uint32_t* ci, const uint32_t* S, uint64_t n, int left, uint32_t* bufs) {
  /* S: sorted candidates (all adjacent to every chosen vertex); left: vertices
   * still to choose from S */
  if (left == 1) return n;
  uint64_t total = 0;
  uint32_t* out = bufs;
  for (uint64_t a = 0; a + 1 < n; a++) {
    const uint32_t x = S[a];
    const uint32_t* N = ci + rp[x];
    const uint64_t dn = rp[x + 1] - rp[x];
    uint64_t j = lower_bound_u32(N, dn, x + 1), i = a + 1, m = 0;
    while (i < n && j < dn) {
      if (S[i] < N[j])
        i++;
      else if (S[i] > N[j])
        j++;
      else {
        out[m++] = S[i];
        i++;
        j++;
      }
    }
    if (m >= (uint64_t)(left - 1)) total += clique_rec(rp, ci, out, m, left - 1, bufs + m);
  }
  return total;
}

uint64_t oracle_cliques_by_smallest(int k, uint64_t V, const uint64_t* rp, const uint32_t* ci, const uint32_t* sources, uint64_t n_sources,
                                    int threads) {
  if (k < 2) return 0;
  const uint64_t dmax = max_degree(V, rp) + 1;
  uint64_t total = 0;
  const int T = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(T) reduction(+ : total)
  {
    /* one buffer of dmax per depth, handed out as a stack */
    uint32_t* bufs = (uint32_t*)malloc((size_t)k * dmax * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 1)
    for (int64_t s = 0; s < (int64_t)n_sources; s++) {
      const uint32_t v = sources[s];
      const uint32_t* N = ci + rp[v];
      const uint64_t dn = rp[v + 1] - rp[v];
      const uint64_t a = lower_bound_u32(N, dn, v + 1);
      total += clique_rec(rp, ci, N + a, dn - a, k - 1, bufs);
    }
    free(bufs);
  }
  return total;
}

/* ------------------------------------------------------- workload (reference arm) */
/* The benchmark's synthetic input, restated so that the timed CPU baseline builds
 * it without the product library: the R-MAT generator (per edge i and level l one
 * uniform double from a splitmix64 finaliser over a seed-salted counter i*64 + l;
 * quadrant by a, a+b, a+b+c), then symmetrised with self loops and duplicates
 * dropped and every row sorted - the layout the reference's preprocessing writes
 * (src/preprocess/preprocess_graph.h:12-92).  tests/test_oracle.py checks it edge
 * for edge against the library's generator. */
static uint64_t wl_mix64(uint64_t seed, uint64_t i) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + i * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double wl_unit(uint64_t seed, uint64_t i) { return (double)(wl_mix64(seed, i) >> 11) * (1.0 / 9007199254740992.0); }

static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : x > y;
}

/* rows from (src, dst) edge lists: both directions, no loops, sorted, unique.
 * *rp (V+1) and *ci are malloc'd here. */
static void wl_csr(uint64_t V, const uint32_t* src, const uint32_t* dst, uint64_t m, int T, uint64_t** rp_out, uint32_t** ci_out) {
  uint64_t* cnt = (uint64_t*)calloc(V + 1, sizeof(uint64_t));
  for (uint64_t i = 0; i < m; i++)
    if (src[i] != dst[i]) {
      cnt[src[i] + 1]++;
      cnt[dst[i] + 1]++;
    }
  for (uint64_t v = 0; v < V; v++) cnt[v + 1] += cnt[v];
  uint32_t* tmp = (uint32_t*)malloc((cnt[V] ? cnt[V] : 1) * sizeof(uint32_t));
  uint64_t* cur = (uint64_t*)malloc((V ? V : 1) * sizeof(uint64_t));
  memcpy(cur, cnt, V * sizeof(uint64_t));
  for (uint64_t i = 0; i < m; i++)
    if (src[i] != dst[i]) {
      tmp[cur[src[i]]++] = dst[i];
      tmp[cur[dst[i]]++] = src[i];
    }
  uint64_t* kept = cur; /* reused: unique entries per row */
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)V; v++) {
    uint32_t* r = tmp + cnt[v];
    const uint64_t n = cnt[v + 1] - cnt[v];
    qsort(r, n, sizeof(uint32_t), cmp_u32);
    uint64_t k = 0;
    for (uint64_t j = 0; j < n; j++)
      if (k == 0 || r[j] != r[k - 1]) r[k++] = r[j];
    kept[v] = k;
  }
  uint64_t* rp = (uint64_t*)malloc((V + 1) * sizeof(uint64_t));
  rp[0] = 0;
  for (uint64_t v = 0; v < V; v++) rp[v + 1] = rp[v] + kept[v];
  uint32_t* ci = (uint32_t*)malloc((rp[V] ? rp[V] : 1) * sizeof(uint32_t));
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)V; v++) memcpy(ci + rp[v], tmp + cnt[v], kept[v] * sizeof(uint32_t));
  free(tmp);
  free(cur);
  free(cnt);
  *rp_out = rp;
  *ci_out = ci;
}

void oracle_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int threads, uint64_t* V_out, uint64_t** rp,
                     uint32_t** ci) {
  const uint64_t V = 1ull << scale, m = (uint64_t)edge_factor << scale;
  const int T = threads > 0 ? threads : omp_get_max_threads();
  uint32_t* src = (uint32_t*)malloc(m * sizeof(uint32_t));
  uint32_t* dst = (uint32_t*)malloc(m * sizeof(uint32_t));
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t i = 0; i < (int64_t)m; i++) {
    uint64_t s = 0, d = 0;
    for (int l = 0; l < scale; l++) {
      const double r = wl_unit(seed, (uint64_t)i * 64 + l);
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
  wl_csr(V, src, dst, m, T, rp, ci);
  free(src);
  free(dst);
  *V_out = V;
}

/* new id = rank of (degree, old id), ascending: a stable counting sort by degree;
 * rows moved to their new ids, entries renamed and sorted.  Output malloc'd. */
void oracle_degree_relabel(uint64_t V, const uint64_t* rp, const uint32_t* ci, int threads, uint64_t** rp_out, uint32_t** ci_out) {
  const int T = threads > 0 ? threads : omp_get_max_threads();
  const uint64_t dmax = max_degree(V, rp);
  uint64_t* at = (uint64_t*)calloc(dmax + 2, sizeof(uint64_t));
  for (uint64_t v = 0; v < V; v++) at[rp[v + 1] - rp[v] + 1]++;
  for (uint64_t d = 0; d <= dmax; d++) at[d + 1] += at[d];
  uint32_t* order = (uint32_t*)malloc((V ? V : 1) * sizeof(uint32_t));
  uint32_t* nid = (uint32_t*)malloc((V ? V : 1) * sizeof(uint32_t));
  for (uint64_t v = 0; v < V; v++) order[at[rp[v + 1] - rp[v]]++] = (uint32_t)v;
  for (uint64_t r = 0; r < V; r++) nid[order[r]] = (uint32_t)r;
  uint64_t* nrp = (uint64_t*)malloc((V + 1) * sizeof(uint64_t));
  nrp[0] = 0;
  for (uint64_t r = 0; r < V; r++) nrp[r + 1] = nrp[r] + (rp[order[r] + 1] - rp[order[r]]);
  uint32_t* nci = (uint32_t*)malloc((nrp[V] ? nrp[V] : 1) * sizeof(uint32_t));
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int64_t r = 0; r < (int64_t)V; r++) {
    const uint32_t v = order[r];
    uint32_t* dst = nci + nrp[r];
    const uint64_t n = rp[v + 1] - rp[v];
    for (uint64_t j = 0; j < n; j++) dst[j] = nid[ci[rp[v] + j]];
    qsort(dst, n, sizeof(uint32_t), cmp_u32);
  }
  free(at);
  free(order);
  free(nid);
  *rp_out = nrp;
  *ci_out = nci;
}

void oracle_free(void* p) { free(p); }
