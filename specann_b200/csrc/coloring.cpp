// Greedy largest-first proper colouring of a CSR graph (host code): the colour classes of the
// independent-set local search (models/local_search_guards/common.py:136-159). Nodes are taken by
// degree descending, ties by index, and each gets the smallest colour not used by an already
// coloured neighbour.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

extern "C" int sa_greedy_coloring(int64_t n, const int64_t* rowptr, const int32_t* col, int32_t* colors,
                                  int32_t* num_colors) {
  if (n < 0 || (n > 0 && (!rowptr || !colors)) || !num_colors) return 1;
  std::vector<int64_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return (rowptr[a + 1] - rowptr[a]) > (rowptr[b + 1] - rowptr[b]);
  });
  std::fill(colors, colors + n, -1);
  std::vector<int64_t> seen(std::max<int64_t>(1, n) + 1, -1);
  int32_t used = 0;
  for (int64_t stamp = 0; stamp < n; ++stamp) {
    const int64_t v = order[stamp];
    for (int64_t p = rowptr[v]; p < rowptr[v + 1]; ++p) {
      const int32_t j = col[p];
      if (j < 0 || j >= n) return 1;
      if (colors[j] >= 0) seen[colors[j]] = stamp;
    }
    int32_t c = 0;
    while (seen[c] == stamp) ++c;
    colors[v] = c;
    used = std::max(used, c + 1);
  }
  *num_colors = used;
  return 0;
}
