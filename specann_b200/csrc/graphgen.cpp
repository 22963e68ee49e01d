// Seeded synthetic Ising instances (host code, no CUDA): Barabasi-Albert and Erdos-Renyi graphs
// written straight into CSR arrays (int64 row pointers, int32 columns, float32 couplings).
//
// Barabasi-Albert follows the preferential-attachment model that NetworkX's
// barabasi_albert_graph implements (star graph on m + 1 nodes, then each new node links to m
// distinct nodes drawn from the list in which every node appears once per incident edge), which
// the reference names as the generator of its BA instances (README.md, "How the Barabasi-Albert
// and Erdos-Renyi graphs were generated"). It has exactly m * (n - m) edges. The random stream is
// this project's own (counter-based SplitMix64), so graphs are reproducible from the seed on any
// machine, but they are not NetworkX's graphs for the same seed.
//
// Erdos-Renyi G(n, p) uses geometric skipping over the pairs i < j (Batagelj and Brandes, 2005).
//
// Coupling modes: 0 -> J = -A (unit MaxCut weights); 1 -> +-1 from a fair coin per undirected
// edge; 2 -> a nonzero integer uniform in [-100, 100] per undirected edge.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform integer in [0, bound) from a 64-bit word (multiply-shift).
inline uint64_t bounded(uint64_t word, uint64_t bound) {
  return (uint64_t)(((__uint128_t)word * (__uint128_t)bound) >> 64);
}

inline float coupling(int mode, uint64_t wseed, uint64_t edge) {
  uint64_t h = splitmix64(wseed ^ (edge * 0xD1B54A32D192ED03ull));
  if (mode == 0) return -1.0f;
  if (mode == 1) return (h & 1) ? 1.0f : -1.0f;
  int v = (int)bounded(h, 200);      // 0..199 -> -100..-1, 1..100
  return (float)(v < 100 ? v - 100 : v - 99);
}

// Edge lists (u, v) with u != v, no duplicates, plus weights -> symmetric CSR with sorted rows.
void edges_to_csr(int64_t n, const std::vector<uint32_t>& eu, const std::vector<uint32_t>& ev,
                  int mode, uint64_t wseed, int64_t* rowptr, int32_t* col, float* val) {
  const int64_t m = (int64_t)eu.size();
  std::vector<int64_t> deg(n + 1, 0);
  for (int64_t e = 0; e < m; ++e) { deg[eu[e]]++; deg[ev[e]]++; }
  rowptr[0] = 0;
  for (int64_t i = 0; i < n; ++i) rowptr[i + 1] = rowptr[i] + deg[i];
  std::vector<std::atomic<int64_t>> fill(n);
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) fill[i].store(rowptr[i], std::memory_order_relaxed);
  #pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; ++e) {
    const float w = coupling(mode, wseed, (uint64_t)e);
    const uint32_t a = eu[e], b = ev[e];
    int64_t pa = fill[a].fetch_add(1, std::memory_order_relaxed);
    col[pa] = (int32_t)b; val[pa] = w;
    int64_t pb = fill[b].fetch_add(1, std::memory_order_relaxed);
    col[pb] = (int32_t)a; val[pb] = w;
  }
  // Sort each row by column (the fill order above is not deterministic under threads).
  #pragma omp parallel
  {
    std::vector<std::pair<int32_t, float>> tmp;
    #pragma omp for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t b = rowptr[i], e = rowptr[i + 1];
      tmp.resize(e - b);
      for (int64_t p = b; p < e; ++p) tmp[p - b] = {col[p], val[p]};
      std::sort(tmp.begin(), tmp.end(),
                [](const std::pair<int32_t, float>& x, const std::pair<int32_t, float>& y) {
                  return x.first < y.first;
                });
      for (int64_t p = b; p < e; ++p) { col[p] = tmp[p - b].first; val[p] = tmp[p - b].second; }
    }
  }
}

void ba_edges(int64_t n, int64_t m, uint64_t seed, std::vector<uint32_t>& eu,
              std::vector<uint32_t>& ev) {
  const int64_t n_edges = m * (n - m);
  eu.resize(n_edges);
  ev.resize(n_edges);
  // repeated: node ids, each repeated once per incident edge (NetworkX's repeated_nodes).
  std::vector<uint32_t> repeated;
  repeated.resize(2 * n_edges);
  int64_t len = 0, e = 0;
  for (int64_t t = 1; t <= m; ++t) {     // star graph: 0 - t
    eu[e] = 0; ev[e] = (uint32_t)t; ++e;
    repeated[len++] = 0;
  }
  for (int64_t t = 1; t <= m; ++t) repeated[len++] = (uint32_t)t;
  const uint64_t base = splitmix64(seed ^ 0xBA0000000000BA01ull);
  std::vector<uint32_t> targets(m);
  for (int64_t src = m + 1; src < n; ++src) {
    // Prefetch the first m draws of the next source (counter-based stream: draw t of source s
    // is splitmix64(base + s * 2^24 + t)).
    if (src + 1 < n) {
      const uint64_t nlen = (uint64_t)(len + 2 * m);
      for (int64_t t = 0; t < m; ++t) {
        uint64_t r = bounded(splitmix64(base + ((uint64_t)(src + 1) << 24) + (uint64_t)t), nlen);
        __builtin_prefetch(&repeated[r]);
      }
    }
    int64_t got = 0;
    uint64_t t = 0;
    while (got < m) {
      uint64_t r = bounded(splitmix64(base + ((uint64_t)src << 24) + t), (uint64_t)len);
      ++t;
      const uint32_t cand = repeated[r];
      bool dup = false;
      for (int64_t q = 0; q < got; ++q) dup |= (targets[q] == cand);
      if (!dup) targets[got++] = cand;
    }
    for (int64_t q = 0; q < m; ++q) {
      eu[e] = (uint32_t)src; ev[e] = targets[q]; ++e;
      repeated[len++] = targets[q];
    }
    for (int64_t q = 0; q < m; ++q) repeated[len++] = (uint32_t)src;
  }
}

void er_edges(int64_t n, double p, uint64_t seed, std::vector<uint32_t>& eu,
              std::vector<uint32_t>& ev) {
  eu.clear(); ev.clear();
  if (n < 2 || p <= 0.0) return;
  const uint64_t base = splitmix64(seed ^ 0xE200000000000E21ull);
  const double lp = std::log1p(-std::min(p, 1.0 - 1e-16));
  int64_t v = 1, w = -1;
  uint64_t draw = 0;
  while (v < n) {
    // uniform in (0, 1]: 53 random bits
    const double r = ((double)(splitmix64(base + draw++) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double skip = p >= 1.0 ? 0.0 : std::floor(std::log(r) / lp);
    w = w + 1 + (int64_t)skip;
    while (w >= v && v < n) { w -= v; ++v; }
    if (v < n) { eu.push_back((uint32_t)v); ev.push_back((uint32_t)w); }
  }
}

struct EdgeCache {
  int kind = -1;
  int64_t n = 0;
  uint64_t seed = 0;
  double p = 0.0;
  std::vector<uint32_t> eu, ev;
};
EdgeCache g_er_cache;

}  // namespace

extern "C" {

// Number of stored entries (both triangles) of BA(n, m): 2 m (n - m); -1 for invalid sizes.
int64_t sa_graph_ba_nnz(int64_t n, int64_t m) {
  if (m < 1 || n <= m || n > (int64_t)INT32_MAX) return -1;
  return 2 * m * (n - m);
}

// Fill CSR arrays of BA(n, m) (caller allocates n + 1 row pointers and sa_graph_ba_nnz entries).
int sa_graph_ba(int64_t n, int64_t m, uint64_t seed, int mode, int64_t* rowptr, int32_t* col,
                float* val) {
  if (sa_graph_ba_nnz(n, m) < 0 || !rowptr || !col || !val || mode < 0 || mode > 2) return 1;
  std::vector<uint32_t> eu, ev;
  ba_edges(n, m, seed, eu, ev);
  edges_to_csr(n, eu, ev, mode, splitmix64(seed ^ 0x3E1647500000001ull), rowptr, col, val);
  return 0;
}

// Stored entries of G(n, p) for this seed (generates and caches the edge list).
int64_t sa_graph_er_nnz(int64_t n, double p, uint64_t seed) {
  if (n < 1 || n > (int64_t)INT32_MAX || !(p >= 0.0 && p <= 1.0)) return -1;
  g_er_cache.kind = 1; g_er_cache.n = n; g_er_cache.p = p; g_er_cache.seed = seed;
  er_edges(n, p, seed, g_er_cache.eu, g_er_cache.ev);
  return 2 * (int64_t)g_er_cache.eu.size();
}

int sa_graph_er(int64_t n, double p, uint64_t seed, int mode, int64_t* rowptr, int32_t* col,
                float* val) {
  if (!rowptr || !col || !val || mode < 0 || mode > 2) return 1;
  if (!(g_er_cache.kind == 1 && g_er_cache.n == n && g_er_cache.p == p && g_er_cache.seed == seed)) {
    if (sa_graph_er_nnz(n, p, seed) < 0) return 1;
  }
  edges_to_csr(n, g_er_cache.eu, g_er_cache.ev, mode, splitmix64(seed ^ 0x3E1647500000001ull),
               rowptr, col, val);
  return 0;
}

}  // extern "C"
