// Native instance loader: the two text formats of the reference's utils/data_loader.py, parsed in
// C++ straight into a CSR with the reference's semantics (utils/data_loader.py:112-204):
//   * Gset: "n m", then "i j w" lines (nodes from 1); every edge is stored in both triangles with
//     weight -w (the minimum energy is the largest cut);
//   * linear-bias (every other dataset): "n m", n lines with the field h_i, then "i j w" lines;
//     nonzero fields become couplings h_i between node i and one extra bias node (index n).
// Edge lines follow _robust_parse_line: blank lines and lines starting with '#' or '%' are skipped,
// as are lines with fewer than three fields or fields that do not parse; node numbers are read as
// int(float(x)); edges with an endpoint out of range or i == j are dropped. Duplicates are summed
// (in file order, FP64), and nodes whose couplings all sum to zero in absolute value are removed
// (the kept rows' file ids are returned), as the reference's COO -> CSR and _remove_isolated_nodes do.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct Instance {
  int64_t n_original = 0;
  int64_t n = 0;
  int64_t bias_index = -1;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<double> val;
  std::vector<int64_t> node_ids;
};

// Python float() of one token (leading/trailing blanks already removed): strtod over the whole
// token, accepting what it accepts (decimal, exponent, inf, nan).
bool parse_double(const std::string& tok, double* out) {
  if (tok.empty()) return false;
  errno = 0;
  char* end = nullptr;
  const double v = std::strtod(tok.c_str(), &end);
  if (end != tok.c_str() + tok.size()) return false;
  *out = v;
  return true;
}

// int(float(tok)): truncation toward zero; nan fails; +-inf is an error of the whole load (Python
// raises OverflowError there, which the reference does not catch).
int parse_index(const std::string& tok, int64_t* out) {
  double v;
  if (!parse_double(tok, &v) || std::isnan(v)) return 0;
  if (std::isinf(v) || std::fabs(v) > 9.0e18) return -1;
  *out = (int64_t)std::trunc(v);
  return 1;
}

std::string strip(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// One "i j w" line: 1 parsed, 0 skipped, -1 error of the whole load.
int parse_edge(const std::string& raw, int64_t* i, int64_t* j, double* w) {
  const std::string line = strip(raw);
  if (line.empty() || line[0] == '#' || line[0] == '%') return 0;
  std::istringstream ss(line);
  std::string t0, t1, t2;
  if (!(ss >> t0 >> t1 >> t2)) return 0;
  const int a = parse_index(t0, i);
  if (a <= 0) return a;
  const int b = parse_index(t1, j);
  if (b <= 0) return b;
  if (!parse_double(t2, w)) return 0;
  return 1;
}

// The edge list of an instance file in file order (fields as edges to the bias node appended last),
// before duplicates are summed: what both the host CSR (load) and the device build (sa_coo_to_csr)
// start from.
struct EdgeList {
  int64_t n_original = 0, n_vertices = 0, bias = -1;
  std::vector<int64_t> ei, ej;
  std::vector<double> ew;
};

int parse_edges(const char* path, int gset, EdgeList* el) {
  std::ifstream f(path);
  if (!f) return 2;
  std::string line;
  if (!std::getline(f, line)) return 3;
  int64_t n = 0, m = 0;
  {
    std::istringstream ss(strip(line));
    std::string a, b, extra;
    if (!(ss >> a >> b) || (ss >> extra)) return 3;
    char* e1 = nullptr;
    char* e2 = nullptr;
    n = std::strtoll(a.c_str(), &e1, 10);
    m = std::strtoll(b.c_str(), &e2, 10);
    if (*e1 || *e2 || n < 0) return 3;
  }
  (void)m;
  std::vector<double> h;
  if (!gset) {
    h.resize((size_t)n);
    for (int64_t q = 0; q < n; ++q) {
      if (!std::getline(f, line)) return 3;
      if (!parse_double(strip(line), &h[(size_t)q])) return 3;
    }
  }
  std::vector<int64_t> ei, ej;
  std::vector<double> ew;
  while (std::getline(f, line)) {
    int64_t i, j;
    double w;
    const int r = parse_edge(line, &i, &j, &w);
    if (r < 0) return 4;
    if (r == 0) continue;
    i -= 1;
    j -= 1;
    if (i >= 0 && i < n && j >= 0 && j < n && i != j) {
      ei.push_back(i);
      ej.push_back(j);
      ew.push_back(gset ? -w : w);
    }
  }
  int64_t nv = n;
  int64_t bias = -1;
  if (!gset) {
    bool any = false;
    for (double x : h) any |= (x != 0.0);
    if (any) {
      bias = n;
      nv = n + 1;
      for (int64_t q = 0; q < n; ++q)
        if (h[(size_t)q] != 0.0) { ei.push_back(bias); ej.push_back(q); ew.push_back(h[(size_t)q]); }
    }
  }
  el->n_original = n;
  el->n_vertices = nv;
  el->bias = bias;
  el->ei.swap(ei);
  el->ej.swap(ej);
  el->ew.swap(ew);
  return 0;
}

int load(const char* path, int gset, Instance* out) {
  EdgeList el;
  const int pst = parse_edges(path, gset, &el);
  if (pst != 0) return pst;
  const int64_t n = el.n_original, nv = el.n_vertices, bias = el.bias;
  const std::vector<int64_t>& ei = el.ei;
  const std::vector<int64_t>& ej = el.ej;
  const std::vector<double>& ew = el.ew;
  // both triangles, in the order the reference appends them: (i, j, w) then (j, i, w) per edge
  const size_t ne = ei.size();
  std::vector<int64_t> r(2 * ne), c(2 * ne);
  std::vector<double> v(2 * ne);
  for (size_t q = 0; q < ne; ++q) {
    r[2 * q] = ei[q]; c[2 * q] = ej[q]; v[2 * q] = ew[q];
    r[2 * q + 1] = ej[q]; c[2 * q + 1] = ei[q]; v[2 * q + 1] = ew[q];
  }
  std::vector<size_t> ord(2 * ne);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
    return r[a] != r[b] ? r[a] < r[b] : c[a] < c[b];
  });
  // duplicates summed in file order
  std::vector<int64_t> ur, uc;
  std::vector<double> uv;
  for (size_t k = 0; k < ord.size(); ++k) {
    const size_t q = ord[k];
    if (!ur.empty() && ur.back() == r[q] && uc.back() == c[q]) uv.back() += v[q];
    else { ur.push_back(r[q]); uc.push_back(c[q]); uv.push_back(v[q]); }
  }
  // isolated nodes: |J| row sums of zero
  std::vector<double> rs((size_t)nv, 0.0);
  for (size_t k = 0; k < ur.size(); ++k) rs[(size_t)ur[k]] += std::fabs(uv[k]);
  std::vector<int64_t> newid((size_t)nv, -1);
  out->node_ids.clear();
  for (int64_t q = 0; q < nv; ++q)
    if (rs[(size_t)q] != 0.0) { newid[(size_t)q] = (int64_t)out->node_ids.size(); out->node_ids.push_back(q); }
  const bool drop = (int64_t)out->node_ids.size() != nv && !ur.empty();
  if (!drop) {
    out->node_ids.resize((size_t)nv);
    std::iota(out->node_ids.begin(), out->node_ids.end(), 0);
    for (int64_t q = 0; q < nv; ++q) newid[(size_t)q] = q;
  }
  const int64_t nk = (int64_t)out->node_ids.size();
  if (nk > (int64_t)INT32_MAX) return 5;
  out->n_original = n;
  out->n = nk;
  out->bias_index = bias >= 0 ? newid[(size_t)bias] : -1;
  out->rowptr.assign((size_t)nk + 1, 0);
  out->col.clear();
  out->val.clear();
  for (size_t k = 0; k < ur.size(); ++k) {
    const int64_t a = newid[(size_t)ur[k]], b = newid[(size_t)uc[k]];
    if (a < 0 || b < 0) continue;
    out->rowptr[(size_t)a + 1] += 1;
    out->col.push_back((int32_t)b);
    out->val.push_back(uv[k]);
  }
  for (int64_t q = 0; q < nk; ++q) out->rowptr[(size_t)q + 1] += out->rowptr[(size_t)q];
  return 0;
}

}  // namespace

extern "C" {

// Parse an instance file into a host object: 0 on success, 2 unreadable file, 3 bad header or
// field lines, 4 an infinite node number, 5 more than 2^31 - 1 rows. Sizes are returned for the
// caller to allocate the arrays of sa_instance_fetch.
int sa_instance_load(const char* path, int32_t gset, void** inst, int64_t* n, int64_t* nnz, int64_t* n_original,
                     int64_t* bias_index) {
  if (!path || !inst || !n || !nnz || !n_original || !bias_index) return 1;
  Instance* x = new Instance();
  const int st = load(path, gset ? 1 : 0, x);
  if (st != 0) { delete x; *inst = nullptr; return st; }
  *inst = x;
  *n = x->n;
  *nnz = (int64_t)x->col.size();
  *n_original = x->n_original;
  *bias_index = x->bias_index;
  return 0;
}

// Parse an instance file into its edge list (file order, fields as bias edges last) for the device
// build (sa_coo_to_csr): 0 on success, or the codes of sa_instance_load.
int sa_instance_edges(const char* path, int32_t gset, void** edges, int64_t* num_edges, int64_t* num_vertices,
                      int64_t* n_original, int64_t* bias_index) {
  if (!path || !edges || !num_edges || !num_vertices || !n_original || !bias_index) return 1;
  EdgeList* x = new EdgeList();
  const int st = parse_edges(path, gset ? 1 : 0, x);
  if (st != 0) { delete x; *edges = nullptr; return st; }
  *edges = x;
  *num_edges = (int64_t)x->ei.size();
  *num_vertices = x->n_vertices;
  *n_original = x->n_original;
  *bias_index = x->bias;
  return 0;
}

// Copy the edge list into caller arrays (num_edges each), then free the object.
int sa_instance_fetch_edges(void* edges, int64_t* ei, int64_t* ej, double* ew) {
  EdgeList* x = (EdgeList*)edges;
  if (!x || ((!ei || !ej || !ew) && !x->ei.empty())) return 1;
  std::copy(x->ei.begin(), x->ei.end(), ei);
  std::copy(x->ej.begin(), x->ej.end(), ej);
  std::copy(x->ew.begin(), x->ew.end(), ew);
  delete x;
  return 0;
}

// Copy the CSR (row pointers n + 1, columns and values nnz) and the kept rows' file node ids (n)
// into caller arrays, then free the object.
int sa_instance_fetch(void* inst, int64_t* rowptr, int32_t* col, double* val, int64_t* node_ids) {
  Instance* x = (Instance*)inst;
  if (!x || !rowptr || !node_ids || ((!col || !val) && !x->col.empty())) return 1;
  std::copy(x->rowptr.begin(), x->rowptr.end(), rowptr);
  std::copy(x->col.begin(), x->col.end(), col);
  std::copy(x->val.begin(), x->val.end(), val);
  std::copy(x->node_ids.begin(), x->node_ids.end(), node_ids);
  delete x;
  return 0;
}

}  // extern "C"
