// sa_spmv_scaled_noalloc: the fused scaled operator y = rho x - N_alpha x for callers that cannot
// allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a host framework that owns all of the
// device's memory through its own pool allocator (nothing is left for a second allocator), or a
// latency-sensitive caller that must not pay for cudaMalloc's implicit device synchronisation.
// They also cannot hand the library a workspace of their own sized for the handle API. This entry
// point needs no handle and no workspace: its scratch (the scaling D^{-alpha/2} / sqrt(c), the
// scaled input, and the max-degree accumulator) lives in one file-scope device array of fixed size,
// so the caller passes only the CSR, x and y. It allocates nothing.
//
// Limits and sharing: n must be at most SA_NOALLOC_MAX_N (the array holds two float vectors of
// that length, 8 MiB, plus a few bytes; every GPU that loads the library keeps it until the process
// exits). Every call uses the same array and leaves the last call's values in it; the accumulator
// that must start at zero is cleared at the start of each call. Calls whose executions overlap on
// the GPU (for example on two streams, or from two host threads) race on the array: serialise them.
//
// Inputs it cannot reject without a synchronisation: a column outside [0, n) is skipped (its product
// counts as zero) so that no read leaves the scaled input; a matrix whose couplings are all zero
// (c = 0, where the normalisation J / c is undefined) gives the defined result N = 0, y = rho x.
#include <cmath>
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace sa {
void count_launches(int k);
}

namespace {

constexpr long long kMaxN = SA_NOALLOC_MAX_N;
constexpr int kMaxDevices = 64;

// [0, kMaxN): per-row scaling sigma; [kMaxN, 2 kMaxN): u = sigma * x; then the max-degree bits.
static __device__ __align__(256) float g_noalloc_scratch[2 * kMaxN + 64];

std::mutex g_setup_mutex;
float* g_scratch_ptr[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

// Device address of the scratch array on the current device and that device's SM count, looked up
// once per device (the host-side symbol is only a stand-in for the device array and must not be
// passed to a kernel).
int scratch_for_current_device(float** out, int* sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SA_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    int count = 0;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SA_ERR_CUDA;
    if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count < 1)
      return SA_ERR_CUDA;
    g_sm_count[dev] = count;
    g_scratch_ptr[dev] = (float*)p;
  }
  *out = g_scratch_ptr[dev];
  *sms = g_sm_count[dev];
  return SA_OK;
}

__global__ void na_degrees(const int* rp, const float* val, long long n, float* sigma_deg,
                           unsigned long long* cmax) {
  unsigned long long lmax = 0ull;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = __ldg(rp + i); p < __ldg(rp + i + 1); ++p) s += fabs((double)__ldg(val + p));
    sigma_deg[i] = (float)s;
    const unsigned long long bits = __double_as_longlong(s);
    lmax = bits > lmax ? bits : lmax;
  }
  atomicMax(cmax, lmax);
}

__global__ void na_scale(long long n, double alpha, const unsigned long long* cmax, const float* x,
                         float* sigma, float* u) {
  const double c = __longlong_as_double((long long)*cmax);
  if (!(c > 0.0)) {   // no non-zero coupling: N = 0
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      sigma[i] = u[i] = 0.0f;
    return;
  }
  const double half_log2_c = 0.5 * log2(c);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)sigma[i] / c;
    const double ld = d > 0.0 ? log2(d) : -INFINITY;
    const double logD = (alpha == 0.0) ? 0.0 : alpha * ld;
    const double logDc = fmax(logD, -39.86313713864835);   // D = max(d^alpha, 1e-12)
    const float s = (float)exp2(-0.5 * logDc - half_log2_c);
    sigma[i] = s;
    u[i] = s * x[i];
  }
}

__global__ void na_spmv(const int* rp, const int* col, const float* val, long long n, float rho,
                        const float* x, const float* sigma, const float* u, float* y) {
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    float acc = 0.0f;
    for (int p = __ldg(rp + r) + lane; p < __ldg(rp + r + 1); p += 32) {
      const int j = __ldg(col + p);
      if (j >= 0 && j < n) acc += __ldg(val + p) * __ldg(u + j);
    }
    acc = sa::warp_sum(acc);
    if (lane == 0) y[r] = rho * x[r] - sigma[r] * acc;
  }
}

}  // namespace

extern "C" int sa_spmv_scaled_noalloc(int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* col,
                                      const float* val, double alpha, double rho, const float* x, float* y,
                                      void* stream) {
  if (n < 1 || n > kMaxN || nnz < 0 || nnz > INT32_MAX || !rowptr || !x || !y || (nnz > 0 && (!col || !val)))
    return SA_ERR_INVALID_ARG;
  float* scratch = nullptr;
  int sms = 0;
  const int st = scratch_for_current_device(&scratch, &sms);
  if (st != SA_OK) return st;
  float* sigma = scratch;
  float* u = scratch + kMaxN;
  unsigned long long* cmax = (unsigned long long*)(scratch + 2 * kMaxN);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(cmax, 0, sizeof(unsigned long long), s) != cudaSuccess) return SA_ERR_CUDA;
  const int threads = 256;
  const int blocks = (int)std::min<long long>((n + threads - 1) / threads, (long long)sms * 8);
  na_degrees<<<blocks, threads, 0, s>>>(rowptr, val, n, sigma, cmax);
  na_scale<<<blocks, threads, 0, s>>>(n, alpha, cmax, x, sigma, u);
  const int sblocks = (int)std::min<long long>((n * 32 + threads - 1) / threads, (long long)sms * 16);
  na_spmv<<<sblocks, threads, 0, s>>>(rowptr, col, val, n, (float)rho, x, sigma, u, y);
  sa::count_launches(3);
  return cudaGetLastError() == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}
