// sparse_abi.cu — the B200 explicit-incidence engine: coldcore's plugin
// ABI 2 (flat sparse_* symbols, include/coldcore_b200/sparse.h).
//
// The problem is a bipartite incidence (coldcore src/plugins/sparse/
// sparse.cu:1-13, src/coldcore/incidence.py:1-35): candidates cover rows of
// universe elements; cnt (int32, over the universe) counts how often each
// element is covered by the solution, and a field is, per candidate, a sum
// over its row of a role of cnt.  Every answer is integer and equals the
// reference's exactly.
//
// B200 layout and kernels:
//   * one allocation per array, rows contiguous (dense n_cand x d, or CSR);
//     cnt, map, staging and extraction buffers in HBM;
//   * a candidate row is processed by a SEGMENT of L lanes, L the power of
//     two at or above the row length (at most 32): a warp serves 32 / L
//     rows at once, its loads of consecutive rows are one contiguous span,
//     and the row sum is a width-L shuffle reduction.  A warp per row (the
//     reference's form) would leave 26 of 32 lanes idle on the 6-element
//     rows of a C(v,4,2) design;
//   * updates are one thread per incidence with int32 atomics on cnt;
//   * reductions (count, deficit, max) reduce in registers per warp, then
//     one atomic per warp.
// Candidate lists are checked on the host, so no kernel indexes outside
// its arrays; nothing waits on another kernel or rank.
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "coldcore_b200/sparse.h"

#define SK(x)                                                               \
  do {                                                                      \
    cudaError_t e_ = (x);                                                   \
    if (e_ != cudaSuccess) {                                                \
      fprintf(stderr, "coldcore_b200 sparse: CUDA error %s at %s:%d\n",     \
              cudaGetErrorString(e_), __FILE__, __LINE__);                  \
      return -(100 + (int)e_);                                              \
    }                                                                       \
  } while (0)

namespace {

constexpr int kMemDev = 0;        // HBM
constexpr int kMemManaged = 2;    // managed memory preferring the host
constexpr int kHistMax = 4096;
constexpr int kThreads = 256;

struct Cell {
  bool live = false, csr = false;
  long long ncand = 0, nuniv = 0, nnz = 0;
  int d = 0, mu = 1, inc_mode = kMemDev, lanes = 32;
  int32_t *inc = nullptr;          // dense rows, or CSR indices
  int64_t *indptr = nullptr;       // CSR row offsets (ncand + 1)
  int32_t *w = nullptr;            // CSR incidence weights
  int32_t *uw = nullptr;           // CSR universe weights (HBM)
  int32_t *cnt = nullptr, *map = nullptr;
  unsigned long long *acc = nullptr;   // reduction / extraction counters
  int32_t *hist = nullptr;
  int64_t *xidx = nullptr;
  int32_t *xval = nullptr;
  int xcap = 0;
  uint32_t *bits = nullptr;        // role bit per universe element
  long long *words = nullptr;      // staged candidate lists
  int32_t *out = nullptr;          // staged per-candidate outputs
  long long wcap = 0;
  long long dev_bytes = 0, host_bytes = 0;
  int sms = 148;
};
Cell C;
cudaStream_t g_s = nullptr;
int g_mu = 1;                      // kept across cells like the reference's

// CTAs for `threads` threads, at most CC_SPARSE_BLOCKS_PER_SM per SM
// (default 32: four waves of resident 256-thread CTAs, which ran the
// C(30,8,4) field 12% faster than one wave); every kernel strides its loop
// over the grid, so any grid covers all the work
int grid_for(long long threads) {
  long long b = (threads + kThreads - 1) / kThreads;
  const char *e = getenv("CC_SPARSE_BLOCKS_PER_SM");
  long long per = e ? atoll(e) : 32;
  if (per < 1) per = 1;
  if (per > 64) per = 64;
  const long long cap = (long long)C.sms * per;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

int lanes_for(long long len) {      // power of two >= len, in 1..32
  int L = 1;
  while (L < 32 && L < len) L <<= 1;
  return L;
}

// ------------------------------------------------------------- kernels
// coverage role of a multiplicity (incidence.py:180-187): 0 deficient,
// 1 critical, any other target the literal cnt == target
__device__ __forceinline__ int role(int c, int target, int mu) {
  if (target == 0) return c < mu;
  if (target == 1) return c >= 1 && c <= mu;
  return c == target;
}

// weighted marginals (incidence.py:374-384, sparse.cu:223-238)
__device__ __forceinline__ long long wval(int c, int w, int u, int target,
                                          int mu) {
  if (target == 0) {
    int def = mu - c;
    if (def < 0) def = 0;
    return (long long)u * (w < def ? w : def);
  }
  if (target == 1) {
    if (c < w) return 0;             // an element this candidate never covered
    int a = mu - c + w, b = mu - c;
    if (a < 0) a = 0;
    if (b < 0) b = 0;
    return (long long)u * (a - b);
  }
  return c == target;
}

// Row sums over candidates i < m (row words[i], or i itself when words is
// null) into out[i]: L lanes per row, 32 / L rows per warp.  The group loop
// is uniform across the warp, so every lane reaches the shuffles.  L is a
// compile-time stride, so a lane's loads of its row entries (and then of
// their counters) issue together instead of one dependent pair at a time.
template <int L>
__global__ void k_rows_dense(const int32_t *__restrict__ inc, int d,
                             const int32_t *__restrict__ cnt,
                             const long long *__restrict__ words, long long m,
                             int target, int mu,
                             int32_t *__restrict__ out) {
  const int lane = threadIdx.x & 31, seg = lane / L, sl = lane % L;
  const int P = 32 / L;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x)
                         >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ngroups = (m + P - 1) / P;
  for (long long g = warp; g < ngroups; g += nwarps) {
    const long long i = g * P + seg;
    int s = 0;
    if (i < m) {
      const long long r = words ? words[i] : i;
      const int32_t *row = inc + r * d;
#pragma unroll 4
      for (int j = sl; j < d; j += L) s += role(cnt[row[j]], target, mu);
    }
    for (int o = L >> 1; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o, L);
    if (sl == 0 && i < m) out[i] = s;
  }
}

// One bit per universe element: bit u of bits[u / 32] = role(cnt[u]).  The
// loop bound is uniform across a warp, so every lane reaches the ballot.
__global__ void k_role_bits(const int32_t *__restrict__ cnt, long long nuniv,
                            int target, int mu, uint32_t *__restrict__ bits) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = (long long)blockIdx.x * blockDim.x +
                          (threadIdx.x & ~31);
  const int lane = threadIdx.x & 31;
  for (long long base = start; base < nuniv; base += stride) {
    const long long u = base + lane;
    const bool p = u < nuniv && role(cnt[u], target, mu);
    const unsigned b = __ballot_sync(0xffffffffu, p);
    if (lane == 0) bits[base >> 5] = b;
  }
}

// k_rows_dense over the role bits instead of cnt: each CTA copies the
// nwords bit words into shared memory, then a row entry costs one shared
// bit test instead of a counter gather through L1/L2.
template <int L>
__global__ void k_rows_dense_bits(const int32_t *__restrict__ inc, int d,
                                  const uint32_t *__restrict__ bits,
                                  int nwords,
                                  const long long *__restrict__ words,
                                  long long m, int32_t *__restrict__ out) {
  extern __shared__ uint32_t sbits[];
  for (int t = threadIdx.x; t < nwords; t += blockDim.x) sbits[t] = bits[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, seg = lane / L, sl = lane % L;
  const int P = 32 / L;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x)
                         >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ngroups = (m + P - 1) / P;
  for (long long g = warp; g < ngroups; g += nwarps) {
    const long long i = g * P + seg;
    int s = 0;
    if (i < m) {
      const long long r = words ? words[i] : i;
      const int32_t *row = inc + r * d;
#pragma unroll 4
      for (int j = sl; j < d; j += L) {
        const int u = row[j];
        s += (sbits[u >> 5] >> (u & 31)) & 1;
      }
    }
    for (int o = L >> 1; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o, L);
    if (sl == 0 && i < m) out[i] = s;
  }
}

template <int L>
__global__ void k_rows_csr(const int64_t *__restrict__ indptr,
                           const int32_t *__restrict__ indices,
                           const int32_t *__restrict__ w,
                           const int32_t *__restrict__ uw,
                           const int32_t *__restrict__ cnt,
                           const long long *__restrict__ words, long long m,
                           int target, int mu,
                           int32_t *__restrict__ out) {
  const int lane = threadIdx.x & 31, seg = lane / L, sl = lane % L;
  const int P = 32 / L;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x)
                         >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ngroups = (m + P - 1) / P;
  for (long long g = warp; g < ngroups; g += nwarps) {
    const long long i = g * P + seg;
    long long s = 0;
    if (i < m) {
      const long long r = words ? words[i] : i;
      const long long e = indptr[r + 1];
#pragma unroll 4
      for (long long j = indptr[r] + sl; j < e; j += L) {
        const int u = indices[j];
        s += wval(cnt[u], w[j], uw[u], target, mu);
      }
    }
    for (int o = L >> 1; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o, L);
    if (sl == 0 && i < m) out[i] = (int32_t)s;
  }
}

// cnt[u] += delta for every incidence (c, u) of the listed candidates
__global__ void k_update_dense(const int32_t *__restrict__ inc, int d,
                               const long long *__restrict__ words,
                               long long m, int delta, int32_t *cnt) {
  const long long total = m * d;
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       t < total; t += gs) {
    const long long i = t / d;
    const int j = (int)(t - i * d);
    atomicAdd(&cnt[inc[words[i] * d + j]], delta);
  }
}

// cnt[u] += delta * w for every weighted incidence, L lanes per row
__global__ void k_update_csr(const int64_t *__restrict__ indptr,
                             const int32_t *__restrict__ indices,
                             const int32_t *__restrict__ w,
                             const long long *__restrict__ words, long long m,
                             int delta, int L, int32_t *cnt) {
  const int lane = threadIdx.x & 31, seg = lane / L, sl = lane % L;
  const int P = 32 / L;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x)
                         >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = warp * P + seg; i < m; i += nwarps * P) {
    const long long r = words[i], e = indptr[r + 1];
    for (long long j = indptr[r] + sl; j < e; j += L)
      atomicAdd(&cnt[indices[j]], delta * w[j]);
  }
}

__device__ __forceinline__ long long warp_sum64(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// kind 0: #{u : cnt == target}; kind 1: sum max(0, mu - cnt) (x uw)
__global__ void k_cnt_reduce(const int32_t *__restrict__ cnt,
                             const int32_t *__restrict__ uw, long long n,
                             int kind, int target, int mu,
                             unsigned long long *acc) {
  long long s = 0;
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gs) {
    const int c = cnt[i];
    if (kind == 0) s += c == target;
    else if (c < mu) s += (long long)(uw ? uw[i] : 1) * (mu - c);
  }
  s = warp_sum64(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, (unsigned long long)s);
}

__global__ void k_map_max(const int32_t *__restrict__ map, long long n,
                          int *out) {
  int v = 0;
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gs)
    v = max(v, map[i]);
  for (int o = 16; o > 0; o >>= 1)
    v = max(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0) atomicMax(out, v);
}

// positive v in bin (v - 1) * nbins / vmax, clipped to the last bin
__global__ void k_hist(const int32_t *__restrict__ map, long long n,
                       int nbins, int vmax, int32_t *hist) {
  extern __shared__ int32_t bins[];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) bins[b] = 0;
  __syncthreads();
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gs) {
    const int v = map[i];
    if (v > 0) {
      long long b = (long long)(v - 1) * nbins / vmax;
      if (b >= nbins) b = nbins - 1;
      atomicAdd(&bins[b], 1);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    if (bins[b]) atomicAdd(&hist[b], bins[b]);
}

// map >= thr: slot by an atomic counter that keeps counting past cap
__global__ void k_extract(const int32_t *__restrict__ map, long long n,
                          int thr, int cap, int64_t *oidx, int32_t *oval,
                          unsigned long long *count) {
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gs) {
    const int v = map[i];
    if (v >= thr) {
      const unsigned long long slot = atomicAdd(count, 1ULL);
      if (slot < (unsigned long long)cap) {
        oidx[slot] = i;
        oval[slot] = v;
      }
    }
  }
}

__global__ void k_read_at(const int32_t *__restrict__ map,
                          const long long *__restrict__ words, long long k,
                          int32_t *out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < k) out[i] = map[words[i]];
}

// ------------------------------------------------------------- host side
int ensure_stream() {
  if (!g_s) SK(cudaStreamCreateWithFlags(&g_s, cudaStreamNonBlocking));
  return 0;
}

// the incidence arrays: HBM, or managed memory preferring the host (the
// reference's CPU placement on a host without coherent C2C)
int alloc_inc(void **p, size_t bytes, int mode, const void *src) {
  if (bytes == 0) bytes = 4;
  if (mode == 0) {
    SK(cudaMalloc(p, bytes));
    C.dev_bytes += bytes;
    // on the engine's stream (which does not order with the legacy one),
    // complete before the call returns
    if (src) {
      SK(cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, g_s));
      SK(cudaStreamSynchronize(g_s));
    }
    return 0;
  }
  SK(cudaMallocManaged(p, bytes));
  C.host_bytes += bytes;
  int dev = 0;
  SK(cudaGetDevice(&dev));
  cudaMemAdvise(*p, bytes, cudaMemAdviseSetPreferredLocation, cudaCpuDeviceId);
  cudaMemAdvise(*p, bytes, cudaMemAdviseSetAccessedBy, dev);
  cudaGetLastError();                // advice is a hint: ignore refusals
  if (src) memcpy(*p, src, bytes);
  return 0;
}

int alloc_dev(void **p, size_t bytes) {
  if (bytes == 0) bytes = 4;
  SK(cudaMalloc(p, bytes));
  C.dev_bytes += bytes;
  return 0;
}

// cnt, map and the query buffers (every cell)
int alloc_fields(int extract_cap) {
  int rc;
  if ((rc = alloc_dev((void **)&C.cnt, (size_t)C.nuniv * 4))) return rc;
  if ((rc = alloc_dev((void **)&C.map, (size_t)C.ncand * 4))) return rc;
  if ((rc = alloc_dev((void **)&C.acc, 16))) return rc;
  if ((rc = alloc_dev((void **)&C.hist, (size_t)kHistMax * 4))) return rc;
  C.xcap = extract_cap;
  if ((rc = alloc_dev((void **)&C.xidx, (size_t)extract_cap * 8))) return rc;
  if ((rc = alloc_dev((void **)&C.xval, (size_t)extract_cap * 4))) return rc;
  SK(cudaMemsetAsync(C.cnt, 0, (size_t)C.nuniv * 4, g_s));
  SK(cudaMemsetAsync(C.map, 0, (size_t)C.ncand * 4, g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

void free_all() {
  auto F = [](void *p) { if (p) cudaFree(p); };
  F(C.inc); F(C.indptr); F(C.w); F(C.uw); F(C.cnt); F(C.map); F(C.acc);
  F(C.hist); F(C.xidx); F(C.xval); F(C.words); F(C.out); F(C.bits);
  C = Cell();
}

int begin_cell(long long ncand, long long nuniv, int inc_mode) {
  C = Cell();
  C.ncand = ncand;
  C.nuniv = nuniv;
  C.inc_mode = inc_mode == 0 ? kMemDev : kMemManaged;
  g_mu = 1;
  int rc = ensure_stream();
  if (rc) return rc;
  int dev = 0;
  SK(cudaGetDevice(&dev));
  SK(cudaDeviceGetAttribute(&C.sms, cudaDevAttrMultiProcessorCount, dev));
  if (C.sms < 1) C.sms = 1;
  C.live = true;                     // so that a failure below frees all
  return 0;
}

// a candidate list: m >= 0 entries, each in [0, n_cand)
int check_words(const long long *idx, long long m) {
  if (m < 0) return -1;
  if (m && !idx) return -2;
  for (long long i = 0; i < m; i++)
    if (idx[i] < 0 || idx[i] >= C.ncand) return -2;
  return 0;
}

int stage_words(const long long *idx, long long m) {
  if (m > C.wcap) {
    long long cap = C.wcap ? C.wcap : 4096;
    while (cap < m) cap *= 2;
    if (C.words) { cudaFree(C.words); C.dev_bytes -= C.wcap * 8; }
    if (C.out) { cudaFree(C.out); C.dev_bytes -= C.wcap * 4; }
    C.words = nullptr;
    C.out = nullptr;
    C.wcap = 0;
    int rc;
    if ((rc = alloc_dev((void **)&C.words, (size_t)cap * 8))) return rc;
    if ((rc = alloc_dev((void **)&C.out, (size_t)cap * 4))) return rc;
    C.wcap = cap;
  }
  SK(cudaMemcpyAsync(C.words, idx, (size_t)m * 8, cudaMemcpyHostToDevice,
                     g_s));
  return 0;
}

// The role-bit form of a dense field or gather, the default (CC_SPARSE_BITS
// =0 turns it off): the bits of the whole universe in at most 48 KB of
// shared memory a CTA.  On C(30,8,4) a field took 0.763 ms in this form
// against 0.848 ms with per-entry counter reads.
constexpr long long kBitsMaxWords = 48 * 1024 / 4;

bool use_bits() {
  const char *e = getenv("CC_SPARSE_BITS");
  return !(e && atoi(e) == 0) && !C.csr &&
         (C.nuniv + 31) / 32 <= kBitsMaxWords;
}

int launch_rows_bits(const long long *words, long long m, int target,
                     int32_t *out) {
  const int nwords = (int)((C.nuniv + 31) / 32);
  int rc;
  if (!C.bits && (rc = alloc_dev((void **)&C.bits, (size_t)nwords * 4)))
    return rc;
  k_role_bits<<<grid_for((long long)nwords * 32), kThreads, 0, g_s>>>(
      C.cnt, C.nuniv, target, g_mu, C.bits);
  SK(cudaGetLastError());
  const int L = C.lanes, P = 32 / L;
  const int grid = grid_for((m + P - 1) / P * 32);
  const size_t smem = (size_t)nwords * 4;
#define CC_BITS(LL)                                                         \
  case LL:                                                                  \
    k_rows_dense_bits<LL><<<grid, kThreads, smem, g_s>>>(                   \
        C.inc, C.d, C.bits, nwords, words, m, out);                         \
    break;
  switch (L) {
    CC_BITS(1) CC_BITS(2) CC_BITS(4) CC_BITS(8) CC_BITS(16) CC_BITS(32)
    default:
      return -2;
  }
#undef CC_BITS
  SK(cudaGetLastError());
  return 0;
}

// per-candidate row sums: the field (words null, into map) or a gather
int launch_rows(const long long *words, long long m, int target,
                int32_t *out) {
  if (use_bits()) return launch_rows_bits(words, m, target, out);
  const int L = C.lanes, P = 32 / L;
  const int grid = grid_for((m + P - 1) / P * 32);
#define CC_ROWS(LL)                                                         \
  case LL:                                                                  \
    if (C.csr)                                                              \
      k_rows_csr<LL><<<grid, kThreads, 0, g_s>>>(                           \
          C.indptr, C.inc, C.w, C.uw, C.cnt, words, m, target, g_mu, out);  \
    else                                                                    \
      k_rows_dense<LL><<<grid, kThreads, 0, g_s>>>(                         \
          C.inc, C.d, C.cnt, words, m, target, g_mu, out);                  \
    break;
  switch (L) {
    CC_ROWS(1) CC_ROWS(2) CC_ROWS(4) CC_ROWS(8) CC_ROWS(16) CC_ROWS(32)
    default:
      return -2;                     // lanes_for gives powers of two <= 32
  }
#undef CC_ROWS
  SK(cudaGetLastError());
  return 0;
}

int update_impl(const long long *idx, long long m, int delta) {
  int rc = check_words(idx, m);
  if (rc) return rc;
  if (m == 0) return 0;
  if ((rc = stage_words(idx, m))) return rc;
  if (C.csr) {
    const int P = 32 / C.lanes;
    k_update_csr<<<grid_for((m + P - 1) / P * 32), kThreads, 0, g_s>>>(
        C.indptr, C.inc, C.w, C.words, m, delta, C.lanes, C.cnt);
  } else {
    k_update_dense<<<grid_for(m * C.d), kThreads, 0, g_s>>>(
        C.inc, C.d, C.words, m, delta, C.cnt);
  }
  SK(cudaGetLastError());
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

long long read_acc() {
  unsigned long long v = 0;
  SK(cudaMemcpyAsync(&v, C.acc, 8, cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  return (long long)v;
}

// ------------------------------------------------- covering designs
// C(v,k,t) rows built on the device, in the reference's layout
// (coldcore src/coldcore/problems/covering_design.py:95-135): candidate c is
// the k-subset of colex rank c (s_0 < ... < s_{k-1}, c = sum C(s_j, j+1));
// its row lists, for the t-subsets of block POSITIONS in lex order (pos,
// d x t), the colex rank sum_j C(s[pos_j], j+1) of that t-subset.
constexpr int kDesignMaxV = 128, kDesignMaxK = 32;
constexpr long long kBinomSat = 1LL << 62;   // binomials saturate here

__global__ void k_design_rows(int v, int k, int t, long long ncand, int d,
                              const unsigned char *__restrict__ pos,
                              const long long *__restrict__ binom,
                              int32_t *inc) {
  extern __shared__ long long B[];            // (v + 1) x (k + 1)
  const int K1 = k + 1, nb = (v + 1) * K1;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) B[i] = binom[i];
  __syncthreads();
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       c < ncand; c += gs) {
    int s[kDesignMaxK];
    long long rem = c;
    int a = v - 1;
    for (int j = k - 1; j >= 0; j--) {
      // the largest a with C(a, j+1) <= rem; C(j, j+1) = 0 stops the walk
      // at a = j at the latest, and every later a lies below this one
      while (B[a * K1 + j + 1] > rem) a--;
      s[j] = a;
      rem -= B[a * K1 + j + 1];
      a--;
    }
    int32_t *row = inc + c * d;
    for (int col = 0; col < d; col++) {
      const unsigned char *p = pos + (long long)col * t;
      long long r = 0;
      for (int j = 0; j < t; j++) r += B[s[p[j]] * K1 + j + 1];
      row[col] = (int32_t)r;
    }
  }
}

}  // namespace

extern "C" {

int sparse_abi_version(void) { return 2; }
long long sparse_dev_bytes(void) { return C.dev_bytes; }
long long sparse_host_bytes(void) { return C.host_bytes; }
long long sparse_b200_stream(void) { return (long long)(uintptr_t)g_s; }
int sparse_b200_row_lanes(void) { return C.live ? C.lanes : -1; }

int sparse_free(void) {
  if (!C.live) return 0;
  if (g_s) cudaStreamSynchronize(g_s);
  free_all();
  g_mu = 1;
  return 0;
}

int sparse_init(long long n_cand, int d, long long n_univ, const int32_t *inc,
                int inc_mode, int extract_cap, long long *bytes_dev,
                long long *bytes_host) {
  if (C.live) return -1;
  if (n_cand < 1 || d < 1 || n_univ < 1 || n_univ > INT_MAX || !inc)
    return -2;
  if (inc_mode < 0 || inc_mode > 1 || extract_cap < 1) return -2;
  if (n_cand > LLONG_MAX / 4 / d) return -2;
  const long long total = n_cand * d;
  for (long long t = 0; t < total; t++)       // every entry in the universe
    if (inc[t] < 0 || inc[t] >= n_univ) return -2;
  int rc = begin_cell(n_cand, n_univ, inc_mode);
  if (rc) { free_all(); return rc; }
  C.d = d;
  C.lanes = lanes_for(d);
  if ((rc = alloc_inc((void **)&C.inc, (size_t)total * 4, inc_mode, inc)) ||
      (rc = alloc_fields(extract_cap))) {
    free_all();
    return rc;
  }
  if (bytes_dev) *bytes_dev = C.dev_bytes;
  if (bytes_host) *bytes_host = C.host_bytes;
  return 0;
}

int sparse_init_csr(long long n_cand, long long n_univ, long long nnz,
                    const int64_t *indptr, const int32_t *indices,
                    const int32_t *w, const int32_t *uw, int inc_mode,
                    int extract_cap, long long *bytes_dev,
                    long long *bytes_host) {
  if (C.live) return -1;
  if (n_cand < 1 || n_univ < 1 || n_univ > INT_MAX || nnz < 0) return -2;
  if (inc_mode < 0 || inc_mode > 1 || extract_cap < 1) return -2;
  if (!indptr || !uw || (nnz && (!indices || !w))) return -2;
  // a valid CSR offset array, entries in the universe, weights >= 1
  if (indptr[0] != 0 || indptr[n_cand] != nnz) return -2;
  for (long long c = 0; c < n_cand; c++)
    if (indptr[c + 1] < indptr[c]) return -2;
  for (long long j = 0; j < nnz; j++)
    if (indices[j] < 0 || indices[j] >= n_univ || w[j] < 1) return -2;
  for (long long u = 0; u < n_univ; u++)
    if (uw[u] < 1) return -2;
  int rc = begin_cell(n_cand, n_univ, inc_mode);
  if (rc) { free_all(); return rc; }
  C.csr = true;
  C.nnz = nnz;
  C.lanes = lanes_for((nnz + n_cand - 1) / n_cand);
  if ((rc = alloc_inc((void **)&C.indptr, (size_t)(n_cand + 1) * 8, inc_mode,
                      indptr)) ||
      (rc = alloc_inc((void **)&C.inc, (size_t)nnz * 4, inc_mode,
                      nnz ? indices : nullptr)) ||
      (rc = alloc_inc((void **)&C.w, (size_t)nnz * 4, inc_mode,
                      nnz ? w : nullptr)) ||
      (rc = alloc_dev((void **)&C.uw, (size_t)n_univ * 4))) {
    free_all();
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(C.uw, uw, (size_t)n_univ * 4,
                                  cudaMemcpyHostToDevice, g_s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_s);
  if (e != cudaSuccess) { free_all(); return -(100 + (int)e); }
  if ((rc = alloc_fields(extract_cap))) { free_all(); return rc; }
  if (bytes_dev) *bytes_dev = C.dev_bytes;
  if (bytes_host) *bytes_host = C.host_bytes;
  return 0;
}

int sparse_b200_init_design(int v, int k, int t, int inc_mode,
                            int extract_cap, long long *bytes_dev,
                            long long *bytes_host) {
  if (C.live) return -1;
  if (v < 1 || v > kDesignMaxV || k < 1 || k > v || k > kDesignMaxK ||
      t < 1 || t > k || inc_mode < 0 || inc_mode > 1 || extract_cap < 1)
    return -2;
  const int K1 = k + 1;
  std::vector<long long> B((size_t)(v + 1) * K1, 0);
  for (int a = 0; a <= v; a++) {
    B[(size_t)a * K1] = 1;
    for (int b = 1; b <= k && b <= a; b++) {
      const long long x = B[(size_t)(a - 1) * K1 + b - 1] +
                          B[(size_t)(a - 1) * K1 + b];
      B[(size_t)a * K1 + b] = x > kBinomSat ? kBinomSat : x;
    }
  }
  const long long ncand = B[(size_t)v * K1 + k];
  const long long dd = B[(size_t)k * K1 + t];
  const long long nuniv = B[(size_t)v * K1 + t];
  if (ncand >= kBinomSat || nuniv > INT_MAX || dd > (1 << 20)) return -2;
  if (ncand > LLONG_MAX / 4 / dd) return -2;
  const int d = (int)dd;
  // the t-subsets of block positions 0..k-1, lex order
  std::vector<unsigned char> pos((size_t)d * t);
  std::vector<int> p(t);
  for (int j = 0; j < t; j++) p[j] = j;
  for (int col = 0; col < d; col++) {
    for (int j = 0; j < t; j++) pos[(size_t)col * t + j] = (unsigned char)p[j];
    int j = t - 1;
    while (j >= 0 && p[j] == k - t + j) j--;
    if (j < 0) break;
    p[j]++;
    for (int i = j + 1; i < t; i++) p[i] = p[i - 1] + 1;
  }
  int rc = begin_cell(ncand, nuniv, inc_mode);
  if (rc) { free_all(); return rc; }
  C.d = d;
  C.lanes = lanes_for(d);
  long long *dB = nullptr;
  unsigned char *dpos = nullptr;
  cudaError_t e = cudaSuccess;
  if ((rc = alloc_inc((void **)&C.inc, (size_t)ncand * d * 4, inc_mode,
                      nullptr)))
    goto fail;
  e = cudaMalloc((void **)&dB, B.size() * 8);
  if (e == cudaSuccess) e = cudaMalloc((void **)&dpos, pos.size());
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dB, B.data(), B.size() * 8, cudaMemcpyHostToDevice,
                        g_s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dpos, pos.data(), pos.size(), cudaMemcpyHostToDevice,
                        g_s);
  if (e == cudaSuccess) {
    k_design_rows<<<grid_for(ncand), kThreads, B.size() * 8, g_s>>>(
        v, k, t, ncand, d, dpos, dB, C.inc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_s);
  if (dB) cudaFree(dB);
  if (dpos) cudaFree(dpos);
  if (e != cudaSuccess) {
    fprintf(stderr, "coldcore_b200 sparse: design build: %s\n",
            cudaGetErrorString(e));
    rc = -(100 + (int)e);
    goto fail;
  }
  if ((rc = alloc_fields(extract_cap))) goto fail;
  if (bytes_dev) *bytes_dev = C.dev_bytes;
  if (bytes_host) *bytes_host = C.host_bytes;
  return 0;
fail:
  free_all();
  return rc;
}

int sparse_b200_read_rows(long long c0, long long n, int32_t *out) {
  if (!C.live) return -1;
  if (C.csr || c0 < 0 || n < 0 || c0 + n > C.ncand) return -2;
  if (n == 0) return 0;
  if (!out) return -2;
  SK(cudaMemcpyAsync(out, C.inc + c0 * C.d, (size_t)n * C.d * 4,
                     cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

int sparse_inc_mode(void) { return C.live ? C.inc_mode : -1; }
int sparse_is_csr(void) { return C.live && C.csr; }

int sparse_set_mu(int mu) {
  if (mu < 1) return -1;
  g_mu = mu;
  return 0;
}

int sparse_get_mu(void) { return g_mu; }

int sparse_ball_update(const long long *idx, long long m, int delta) {
  if (!C.live) return -1;
  return update_impl(idx, m, delta);
}

int sparse_recount(const long long *idx, long long m) {
  if (!C.live) return -1;
  int rc = check_words(idx, m);        // reject before clearing cnt
  if (rc) return rc;
  SK(cudaMemsetAsync(C.cnt, 0, (size_t)C.nuniv * 4, g_s));
  if (m == 0) {
    SK(cudaStreamSynchronize(g_s));
    return 0;
  }
  return update_impl(idx, m, 1);
}

int sparse_field(int target) {
  if (!C.live) return -1;
  int rc = launch_rows(nullptr, C.ncand, target, C.map);
  if (rc) return rc;
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

int sparse_ball_gather(const long long *idx, long long m, int target,
                       int32_t *out) {
  if (!C.live) return -1;
  int rc = check_words(idx, m);
  if (rc) return rc;
  if (m == 0) return 0;
  if (!out) return -2;
  if ((rc = stage_words(idx, m))) return rc;
  if ((rc = launch_rows(C.words, m, target, C.out))) return rc;
  SK(cudaMemcpyAsync(out, C.out, (size_t)m * 4, cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

long long sparse_count_eq(int target) {
  if (!C.live) return -1;
  SK(cudaMemsetAsync(C.acc, 0, 8, g_s));
  k_cnt_reduce<<<grid_for(C.nuniv), kThreads, 0, g_s>>>(
      C.cnt, nullptr, C.nuniv, 0, target, g_mu, C.acc);
  SK(cudaGetLastError());
  return read_acc();
}

long long sparse_count_deficit(void) {
  if (!C.live) return -1;
  SK(cudaMemsetAsync(C.acc, 0, 8, g_s));
  k_cnt_reduce<<<grid_for(C.nuniv), kThreads, 0, g_s>>>(
      C.cnt, C.csr ? C.uw : nullptr, C.nuniv, 1, 0, g_mu, C.acc);
  SK(cudaGetLastError());
  return read_acc();
}

int sparse_map_max(int32_t *out) {
  if (!C.live) return -1;
  if (!out) return -2;
  SK(cudaMemsetAsync(C.acc, 0, 8, g_s));
  k_map_max<<<grid_for(C.ncand), kThreads, 0, g_s>>>(
      C.map, C.ncand, reinterpret_cast<int *>(C.acc));
  SK(cudaGetLastError());
  int v = 0;
  SK(cudaMemcpyAsync(&v, C.acc, 4, cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  *out = v;
  return 0;
}

int sparse_map_hist(int nbins, int32_t vmax, int32_t *out) {
  if (!C.live) return -1;
  if (nbins < 1 || nbins > kHistMax || vmax < 1 || !out) return -2;
  SK(cudaMemsetAsync(C.hist, 0, (size_t)nbins * 4, g_s));
  k_hist<<<grid_for(C.ncand), kThreads, (size_t)nbins * 4, g_s>>>(
      C.map, C.ncand, nbins, vmax, C.hist);
  SK(cudaGetLastError());
  SK(cudaMemcpyAsync(out, C.hist, (size_t)nbins * 4, cudaMemcpyDeviceToHost,
                     g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

long long sparse_map_extract(int32_t thr, int64_t *idx, int32_t *val,
                             int cap) {
  if (!C.live) return -1;
  if (cap > C.xcap) cap = C.xcap;
  if (cap < 0) return -2;
  SK(cudaMemsetAsync(C.acc, 0, 8, g_s));
  k_extract<<<grid_for(C.ncand), kThreads, 0, g_s>>>(
      C.map, C.ncand, thr, cap, C.xidx, C.xval, C.acc);
  SK(cudaGetLastError());
  const long long found = read_acc();
  if (found < 0) return found;
  const long long m = found < cap ? found : cap;
  if (m > 0) {
    if (!idx || !val) return -2;
    SK(cudaMemcpyAsync(idx, C.xidx, (size_t)m * 8, cudaMemcpyDeviceToHost,
                       g_s));
    SK(cudaMemcpyAsync(val, C.xval, (size_t)m * 4, cudaMemcpyDeviceToHost,
                       g_s));
    SK(cudaStreamSynchronize(g_s));
  }
  return found;
}

int sparse_map_read_at(const long long *idx, long long k, int32_t *out) {
  if (!C.live) return -1;
  int rc = check_words(idx, k);
  if (rc) return rc;
  if (k == 0) return 0;
  if (!out) return -2;
  if ((rc = stage_words(idx, k))) return rc;
  k_read_at<<<(unsigned)((k + kThreads - 1) / kThreads), kThreads, 0, g_s>>>(
      C.map, C.words, k, C.out);
  SK(cudaGetLastError());
  SK(cudaMemcpyAsync(out, C.out, (size_t)k * 4, cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

int sparse_read_cnt(long long off, long long len, int32_t *out) {
  if (!C.live) return -1;
  if (off < 0 || len < 0 || off + len > C.nuniv) return -2;
  if (len == 0) return 0;
  if (!out) return -2;
  SK(cudaMemcpyAsync(out, C.cnt + off, (size_t)len * 4,
                     cudaMemcpyDeviceToHost, g_s));
  SK(cudaStreamSynchronize(g_s));
  return 0;
}

}  // extern "C"
