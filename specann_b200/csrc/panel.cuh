// Column-panel SpMV: the gathers of the scaled input come from shared memory instead of L2.
//
// A random 4-byte gather from global memory costs one L1 tag wavefront per lane, so the work-list
// SpMV is bound by the L1TEX pipe (about 0.7 gathers per SM per clock on a Barabasi-Albert graph).
// Here each CTA owns a block of rows whose partial sums live in shared memory, and walks the
// columns in panels: panel p of the scaled input (panel_buf_bytes, `width` columns) is staged in shared
// memory by one bulk asynchronous copy (completion on an mbarrier, double-buffered so the copy of
// panel p + 1 overlaps the work on panel p), and the block's entries with a column in panel p are
// gathered from it. A random shared-memory gather of a warp costs about 3.5 wavefronts instead of
// 32. Every CTA reads the whole input once per SpMV (from L2), which pays when the average row has
// more than ~20 entries.
//
// Layout (built once per matrix, sa_panel_build): rows are cut into blocks of at most
// kPanelRowBytes / sizeof(T) rows with about equal entries; the entries of block b with a column in
// panel p form segment (b, p) (blocks major, panels minor), in row order. Each segment is cut at row
// boundaries into kWarps chunks of about equal length, so a row's entries of one panel belong to
// one warp. An entry is one 32-bit word: bits 31-16 the row in the block, bit 15 the sign of the
// coupling, bits 14-0 the column in the panel; the value is +-wmag when every coupling has one
// magnitude, else it is streamed from `val` in the same order.
//
// Summation order is fixed: a row's products in one panel are added by one warp (a segmented
// shuffle scan over runs of equal rows, in entry order), and the panels are added in panel order
// (a CTA barrier separates them). No atomics.
#pragma once
#include "common.cuh"
#include "spmv.cuh"

namespace sa {

constexpr int kPanelBufs = 2;               // panels in flight
constexpr int kPanelRowBytes = 64 * 1024;   // row sums of one block
// One staged panel of the scaled input: 64 KB in FP32, 48 KB in FP64 (the FP64 kernels hold more
// static shared memory); the dynamic shared memory of a panel kernel is the buffers + the row sums.
__host__ __device__ constexpr int panel_buf_bytes(int elem) { return elem == 4 ? 64 * 1024 : 48 * 1024; }
__host__ __device__ constexpr int panel_smem_bytes(int elem) { return kPanelBufs * panel_buf_bytes(elem) + kPanelRowBytes; }
constexpr unsigned long long kPanelSpinLimit = 1ull << 22;   // bounded wait for a panel copy

struct PanelArgs {
  const unsigned int* ent;   // packed entries, segment (b, p) order
  const void* val;           // values in entry order, or null (one magnitude: +-wmag)
  const long long* chunk;    // chunk starts: [(b * n_panels + p) * kWarps + w], one extra end entry
  const int* row0;           // first row of each block, n_blocks + 1
  int n_blocks, n_panels, width;
  int pad;
  long long n;
  double wmag;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Stage `bytes` (a multiple of 16, both addresses 16-byte aligned) from global memory into shared
// memory with completion on `bar` (one arrival carrying the byte count). One thread.
__device__ __forceinline__ void panel_fill(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Orders this thread's earlier generic-proxy accesses (the reads of a panel buffer that is about to
// be refilled, and global writes of the input made visible by a barrier) before its following
// async-proxy copies.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }

// Barrier set-up of a kernel that runs panel SpMVs (thread 0, then a CTA barrier).
__device__ __forceinline__ void panel_init(unsigned long long* bars) {
  if (threadIdx.x == 0) {
    for (int q = 0; q < kPanelBufs; ++q) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ unsigned panel_bytes(const PanelArgs& P, int p) {
  const long long c0 = (long long)p * P.width;
  const long long cols = (P.n - c0 < P.width) ? (P.n - c0) : P.width;
  return (unsigned)(((cols * (long long)sizeof(T)) + 15) & ~15ll);
}

template <typename T>
__device__ __forceinline__ void panel_issue(const PanelArgs& P, const T* u, int p, char* smem,
                                            unsigned long long* bars) {
  const int buf = p % kPanelBufs;
  panel_fill(smem + (size_t)buf * panel_buf_bytes(sizeof(T)), u + (long long)p * P.width, panel_bytes<T>(P, p),
             &bars[buf]);
}

// A batch is 256 entries of a warp's chunk: lane l takes the 8 consecutive entries
// [e + 8 l, e + 8 l + 8) (chunks are padded with kPanelPad words to multiples of 8, so a lane's
// entries are all real or all padding and its two 16-byte loads are aligned).
constexpr unsigned kPanelPad = 0xFFFF0000u;   // row 0xFFFF (never written), column 0
constexpr int kPanelLane = 8;                 // entries per lane of a batch
constexpr int kPanelBatchEntries = 32 * kPanelLane;

__device__ __forceinline__ uint4 ld_stream_v4(const unsigned* p, unsigned long long pol) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ void panel_load_batch(const unsigned int* ent, long long e, long long ce, int lane,
                                                 unsigned (&r)[kPanelLane], unsigned long long pol) {
  const long long k = e + (long long)kPanelLane * lane;
  if (k < ce) {
    const uint4 a = ld_stream_v4(ent + k, pol), b = ld_stream_v4(ent + k + 4, pol);
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
  } else {
#pragma unroll
    for (int j = 0; j < kPanelLane; ++j) r[j] = kPanelPad;
  }
}

template <typename T>
__device__ __forceinline__ void panel_load_vals(const T* val, long long e, long long ce, int lane,
                                                T (&v)[kPanelLane], unsigned long long pol) {
  const long long k = e + (long long)kPanelLane * lane;
#pragma unroll
  for (int j = 0; j < kPanelLane; ++j) v[j] = (k < ce) ? ld_stream(val + k + j, pol) : T(0);
}

// Products of one batch added into the block's row sums ys. The entries are in row order, so
// every row is a run of consecutive entries: runs inside a lane are summed in registers (left to
// right); a run that crosses lanes is summed by a segmented scan over the lanes' tail sums and
// added by the lane where it ends. Each run is added to ys once per batch, by one lane, and the
// runs of one lane have distinct rows, so all of a lane's loads of ys can precede its stores.
template <typename T>
__device__ __forceinline__ void panel_batch(const unsigned (&r)[kPanelLane], const T (&v)[kPanelLane], bool uniform,
                                            T wmag, int lane, const T* xs, T* ys) {
  unsigned key[kPanelLane];
  T s[kPanelLane];
#pragma unroll
  for (int j = 0; j < kPanelLane; ++j) {
    key[j] = r[j] >> 16;
    const T x = xs[r[j] & 0x7FFFu];
    const T a = uniform ? ((r[j] & 0x8000u) ? -wmag : wmag) : v[j];
    s[j] = a * x;
  }
#pragma unroll
  for (int j = 1; j < kPanelLane; ++j)
    if (key[j] == key[j - 1]) s[j] = s[j - 1] + s[j];
  const unsigned k0 = key[0], k7 = key[kPanelLane - 1];
  const unsigned kprev = __shfl_up_sync(0xffffffffu, k7, 1);     // last row of lane - 1
  const unsigned knext = __shfl_down_sync(0xffffffffu, k0, 1);   // first row of lane + 1
  // inclusive segmented scan of the tail sums over lanes; segments: equal last rows
  const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || kprev != k7);
  const int seg0 = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
  T inc = s[kPanelLane - 1];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const T t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane - d >= seg0) inc = t + inc;
  }
  const T cin = __shfl_up_sync(0xffffffffu, inc, 1);
  const T carry = (lane > 0 && kprev == k0) ? cin : T(0);
  const bool cont = lane < 31 && knext == k7;
  bool wr[kPanelLane];
  T add[kPanelLane], old[kPanelLane];
#pragma unroll
  for (int j = 0; j < kPanelLane; ++j) {
    const bool end = (j == kPanelLane - 1) ? !cont : (key[j + 1] != key[j]);
    wr[j] = end && key[j] != (kPanelPad >> 16);
    add[j] = (key[j] == k0) ? s[j] + carry : s[j];
  }
#pragma unroll
  for (int j = 0; j < kPanelLane; ++j) old[j] = wr[j] ? ys[key[j]] : T(0);
#pragma unroll
  for (int j = 0; j < kPanelLane; ++j)
    if (wr[j]) ys[key[j]] = old[j] + add[j];
  __syncwarp();
}

// One SpMV over the blocks of this CTA (b = blk, blk + nblk, ...): fin(row, sum) once per row with
// sum = sum_j val_ij u_j. smem: panel_smem_bytes(sizeof(T)) dynamic bytes (panel buffers, then the row sums); bars:
// kPanelBufs mbarriers set up by panel_init; par: the barriers' phase bits (one bit per buffer,
// kept by the caller across calls; every thread holds the same value). Returns false, with
// SA_ERR_BARRIER_TIMEOUT in *err, if a panel copy does not complete in time.
template <typename T, class Fin>
__device__ __forceinline__ bool panel_spmv(const PanelArgs& P, const T* u, int blk, int nblk, char* smem,
                                           unsigned long long* bars, unsigned& par, int* err, Fin&& fin) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned long long pol = l2_policy_evict_first();
  T* ys = (T*)(smem + (size_t)kPanelBufs * panel_buf_bytes(sizeof(T)));
  const bool uniform = P.val == nullptr;
  const T wmag = (T)P.wmag;
  const T* val = (const T*)P.val;
  const int np = P.n_panels;
  for (int b = blk; b < P.n_blocks; b += nblk) {
    const int r0 = __ldg(P.row0 + b), nr = __ldg(P.row0 + b + 1) - r0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) ys[i] = T(0);
    if (threadIdx.x == 0) {
      fence_proxy_async();
      for (int q = 0; q < kPanelBufs && q < np; ++q) panel_issue<T>(P, u, q, smem, bars);
    }
    __syncthreads();
    const long long* ch = P.chunk + (long long)b * np * kWarps + wid;
    long long cs = __ldg(ch), ce = __ldg(ch + 1);
    unsigned cur[kPanelLane];
    T cv[kPanelLane] = {};
    panel_load_batch(P.ent, cs, ce, lane, cur, pol);
    if (!uniform) panel_load_vals(val, cs, ce, lane, cv, pol);
    for (int p = 0; p < np; ++p) {
      // the next panel's chunk bounds, consumed at the end of this panel
      long long ns = 0, ne = 0;
      if (p + 1 < np) {
        ns = __ldg(ch + (long long)(p + 1) * kWarps);
        ne = __ldg(ch + (long long)(p + 1) * kWarps + 1);
      }
      const int buf = p % kPanelBufs;
      const unsigned par0 = par;   // the same in every thread of the CTA
      // Bounded wait for panel p. A thread that gives up skips the panel's work and the CTA decides
      // at the barrier that ends the panel (__syncthreads_or), so every thread returns together.
      bool late = false;
      for (unsigned long long spins = 0; !mbar_try_wait(&bars[buf], (par0 >> buf) & 1u);)
        if (++spins > kPanelSpinLimit) {
          late = true;
          break;
        }
      late = __any_sync(0xffffffffu, late);   // the batch loop's shuffles need whole warps
      par ^= 1u << buf;
      const T* xs = (const T*)(smem + (size_t)buf * panel_buf_bytes(sizeof(T)));
      for (long long e = cs; !late; e += kPanelBatchEntries) {
        const bool more = e + kPanelBatchEntries < ce;
        unsigned nx[kPanelLane];
        T nv[kPanelLane] = {};
        if (more) {
          panel_load_batch(P.ent, e + kPanelBatchEntries, ce, lane, nx, pol);
          if (!uniform) panel_load_vals(val, e + kPanelBatchEntries, ce, lane, nv, pol);
        } else {
          panel_load_batch(P.ent, ns, ne, lane, nx, pol);
          if (!uniform) panel_load_vals(val, ns, ne, lane, nv, pol);
        }
        if (e < ce) panel_batch<T>(cur, cv, uniform, wmag, lane, xs, ys);
#pragma unroll
        for (int q = 0; q < kPanelLane; ++q) {
          cur[q] = nx[q];
          cv[q] = nv[q];
        }
        if (!more) break;
      }
      cs = ns;
      ce = ne;
      if (__syncthreads_or(late)) {
        // Give up: record the timeout, then wait (bounded again) for the copies this CTA still has
        // in flight into its shared memory (panels p .. p + kPanelBufs - 1) before returning.
        if (threadIdx.x == 0) {
          atomicExch(err, SA_ERR_BARRIER_TIMEOUT);
          for (int q = p; q < p + kPanelBufs && q < np; ++q) {
            const int qb = q % kPanelBufs;
            for (unsigned long long spins = 0; !mbar_try_wait(&bars[qb], (par0 >> qb) & 1u);)
              if (++spins > kPanelSpinLimit) break;
          }
        }
        __syncthreads();
        return false;
      }
      if (threadIdx.x == 0 && p + kPanelBufs < np) {
        fence_proxy_async();
        panel_issue<T>(P, u, p + kPanelBufs, smem, bars);
      }
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) fin((long long)r0 + i, ys[i]);
    __syncthreads();
  }
  return true;
}

}  // namespace sa
