// Stand-alone writer of the seeded synthetic graphs for the CPU baseline. TEST INFRASTRUCTURE ONLY.
//
// bench.py's reference arm times the oracle (SciPy/NumPy, CPU) on the same graph as the GPU arm
// without loading any of the product's shared libraries into its process: it runs this executable,
// linked from the same generator source (specann_b200/csrc/graphgen.cpp), and reads the CSR it
// writes.
//
//   ba_graph ba <n> <m> <seed> <mode> <out>      Barabasi-Albert(n, m)
//   ba_graph er <n> <p> <seed> <mode> <out>      Erdos-Renyi G(n, p)
//
// mode: 0 unit (J = -A), 1 +-1, 2 integers in [-100, 100]. Output: int64 n, int64 nnz, then
// int64 rowptr[n + 1], int32 col[nnz], float32 val[nnz], little-endian.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {
int64_t sa_graph_ba_nnz(int64_t n, int64_t m);
int sa_graph_ba(int64_t n, int64_t m, uint64_t seed, int mode, int64_t* rowptr, int32_t* col, float* val);
int64_t sa_graph_er_nnz(int64_t n, double p, uint64_t seed);
int sa_graph_er(int64_t n, double p, uint64_t seed, int mode, int64_t* rowptr, int32_t* col, float* val);
}

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s ba|er <n> <m|p> <seed> <mode> <out>\n", argv[0]);
    return 2;
  }
  const bool ba = std::strcmp(argv[1], "ba") == 0;
  const int64_t n = std::atoll(argv[2]);
  const uint64_t seed = std::strtoull(argv[4], nullptr, 10);
  const int mode = std::atoi(argv[5]);
  const int64_t nnz = ba ? sa_graph_ba_nnz(n, std::atoll(argv[3])) : sa_graph_er_nnz(n, std::atof(argv[3]), seed);
  if (nnz < 0) {
    std::fprintf(stderr, "invalid graph size\n");
    return 1;
  }
  std::vector<int64_t> rowptr(n + 1);
  std::vector<int32_t> col(nnz);
  std::vector<float> val(nnz);
  const int st = ba ? sa_graph_ba(n, std::atoll(argv[3]), seed, mode, rowptr.data(), col.data(), val.data())
                    : sa_graph_er(n, std::atof(argv[3]), seed, mode, rowptr.data(), col.data(), val.data());
  if (st != 0) return 1;
  FILE* f = std::fopen(argv[6], "wb");
  if (!f) return 1;
  const int64_t head[2] = {n, nnz};
  bool ok = std::fwrite(head, sizeof(head), 1, f) == 1 &&
            std::fwrite(rowptr.data(), sizeof(int64_t), rowptr.size(), f) == rowptr.size() &&
            std::fwrite(col.data(), sizeof(int32_t), col.size(), f) == col.size() &&
            std::fwrite(val.data(), sizeof(float), val.size(), f) == val.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : 1;
}
