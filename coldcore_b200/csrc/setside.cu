// setside.cu — set-side gathers: count a candidate's ball words that satisfy
// a predicate by comparing the candidate with the LIST of such words instead
// of walking its ball.
//
// Semantics follow the reference's set side (coldcore
// src/plugins/covering/dct_hc.cu:589-760, dctcore_fast.cuh k_compact_pred /
// k_gather_set): near a cover the deficient set Z = {x : cnt[x] < mu} (or
// {cnt == 0}) is small, and
//     #{x in B(c) : pred(cnt[x])} = #{z in Z : d(c, z) <= R}
// whenever the support table is exactly the metric ball (checked on the host
// at init).  The answer is the same integer the walk gives.
//
// Layout here: Z is listed once per cnt state as packed words, one 4-bit
// nibble per digit in a uint64 (cells with n <= 16 axes of size <= 16).  The
// gather kernel holds a tile of 32 candidates in shared memory; each thread
// streams Z words from HBM/L2 (coalesced 8-byte loads) and compares each
// with the 32 candidates, keeping 32 counters in registers.  Hamming
// distance is a popcount over the nonzero nibbles of the XOR; Lee, torus and
// grid loop over the digits.  Counters are reduced per warp and added to the
// output with one atomic per candidate per block.
#include "engine.h"

namespace cc {

struct SetGeom {
  int prob, n, R;
  int ax[16];
};

__device__ __forceinline__ unsigned long long pack_digits(long long x,
                                                          const SetGeom &g) {
  unsigned long long p = 0;
  for (int j = 0; j < g.n; j++) {
    const long long a = g.ax[j];
    p |= (unsigned long long)(x % a) << (4 * j);
    x /= a;
  }
  return p;
}

// words whose cnt satisfies the predicate, packed; *found counts all of
// them, only the first cap are stored
__global__ void __launch_bounds__(256)
k_list_pred(const uint16_t *cnt, long long N, int mode, int target, int mu,
            SetGeom g, unsigned long long *out, long long cap,
            unsigned long long *found) {
  const long long gs = (long long)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const long long nvec = (N + 7) >> 3;         // cnt is padded to 64
  const uint4 *v = reinterpret_cast<const uint4 *>(cnt);
  for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < nvec;
       i0 += gs) {
    const long long i = i0 + threadIdx.x;
    unsigned hits = 0;
    if (i < nvec) {
      const uint4 q = v[i];
      const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int h = 0; h < 8; h++) {
        const int c = (int)((w4[h >> 1] >> (16 * (h & 1))) & 0xFFFFu);
        if (i * 8 + h < N && cnt_pred(mode, c, target, mu)) hits |= 1u << h;
      }
    }
    const int mine = __popc(hits);
    int incl = mine;                               // warp inclusive scan
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) continue;
    unsigned long long base = 0;
    if (lane == 31) base = atomicAdd(found, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    long long slot = (long long)base + incl - mine;
    while (hits) {
      const int h = __ffs(hits) - 1;
      hits &= hits - 1;
      if (slot < cap) out[slot] = pack_digits(i * 8 + h, g);
      slot++;
    }
  }
}

// d(a, b) <= R for packed words; ax: the axis sizes (shared memory)
template <int PROB>
__device__ __forceinline__ bool within(unsigned long long a,
                                       unsigned long long b, int n, int R,
                                       const int *ax) {
  if (PROB == kHamming) {
    unsigned long long x = a ^ b;
    x = (x | (x >> 1) | (x >> 2) | (x >> 3)) & 0x1111111111111111ull;
    return __popcll(x) <= R;
  }
  int acc = 0;
  for (int j = 0; j < n; j++) {
    const int da = (int)((a >> (4 * j)) & 15u), db = (int)((b >> (4 * j)) & 15u);
    int d = da > db ? da - db : db - da;
    if (PROB != kGrid) d = min(d, ax[j] - d);     // circular
    if (PROB == kLee) acc += d;
    else acc = max(acc, d);                       // L-infinity
  }
  return acc <= R;
}

constexpr int kSetTile = 32;     // candidates per block

// out[c] += #{z in Z[chunk] : d(c, z) <= R}; out zeroed by the caller
template <int PROB>
__global__ void __launch_bounds__(256, 2)
k_gather_set(const long long *cand, int nc, const unsigned long long *Z,
             long long zn, long long zchunk, SetGeom g, int32_t *out) {
  __shared__ unsigned long long cw[kSetTile];
  __shared__ int sums[kSetTile];
  __shared__ int sax[16];
  const int c0 = blockIdx.x * kSetTile;
  const int nt = min(kSetTile, nc - c0);
  if (threadIdx.x < 16) sax[threadIdx.x] = g.ax[threadIdx.x];
  if (threadIdx.x < kSetTile) {
    sums[threadIdx.x] = 0;
    cw[threadIdx.x] = threadIdx.x < nt ? pack_digits(cand[c0 + threadIdx.x], g)
                                       : ~0ull;
  }
  __syncthreads();
  const long long z0 = (long long)blockIdx.y * zchunk;
  const long long z1 = min(zn, z0 + zchunk);
  int acc[kSetTile];
#pragma unroll
  for (int t = 0; t < kSetTile; t++) acc[t] = 0;
  for (long long i = z0 + threadIdx.x; i < z1; i += blockDim.x) {
    const unsigned long long z = Z[i];
#pragma unroll
    for (int t = 0; t < kSetTile; t++)
      acc[t] += within<PROB>(cw[t], z, g.n, g.R, sax);
  }
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int t = 0; t < kSetTile; t++) {
    const int s = __reduce_add_sync(0xffffffffu, (unsigned)acc[t]);
    if (lane == 0 && s) atomicAdd(&sums[t], s);
  }
  __syncthreads();
  if (threadIdx.x < nt && sums[threadIdx.x])
    atomicAdd(&out[c0 + threadIdx.x], sums[threadIdx.x]);
}

// exclusive scan of n (<= 65535) counts into offs[0..n], clipped at cap
// (a total above cap reads cap + 1: the caller falls back); cursor[i] =
// offs[i].  Sums are 64-bit, so k drops of large balls cannot wrap.
__global__ void __launch_bounds__(1024)
k_seg_scan(const int32_t *cnt, int n, long long cap, int32_t *offs,
           int32_t *cursor) {
  __shared__ long long part[1024];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(n, b + per);
  long long sum = 0;
  for (int i = b; i < e; i++) sum += cnt[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {     // Hillis-Steele
    const long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - sum;
  for (int i = b; i < e; i++) {
    const int32_t o = (int32_t)min(run, cap);
    offs[i] = o;
    cursor[i] = o;
    run += cnt[i];
  }
  if (threadIdx.x == blockDim.x - 1)
    offs[n] = (int32_t)min(part[threadIdx.x], cap + 1);
}

int launch_seg_scan(const int32_t *cnt, int n, long long cap, int32_t *offs,
                    int32_t *cursor, cudaStream_t s) {
  k_seg_scan<<<1, 1024, 0, s>>>(cnt, n, cap, offs, cursor);
  CC_CK(cudaGetLastError());
  return 0;
}

constexpr int kCorrChunk = 2048;  // listed words staged per block pass

// swap evaluation, correction: gain[j] += #{w in list segment of drop(j) :
// d(cand[j], w) <= R}.  One block per drop: its segment is packed into
// shared memory chunk by chunk, and each warp takes the drop's candidates
// (the contiguous range coff[i] .. coff[i+1]) one at a time.
template <int PROB>
__global__ void __launch_bounds__(256)
k_swap_corr(const long long *cand, const int32_t *coff,
            const int32_t *offs, const long long *list, long long cap,
            SetGeom g, int32_t *gain) {
  __shared__ unsigned long long seg[kCorrChunk];
  __shared__ int sax[16];
  const int i = blockIdx.x;
  if (threadIdx.x < 16) sax[threadIdx.x] = g.ax[threadIdx.x];
  const long long s0 = offs[i];
  const long long s1 = min((long long)offs[i + 1], cap);
  const int c0 = coff[i], c1 = coff[i + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  for (long long base = s0; base < s1; base += kCorrChunk) {
    const int len = (int)min((long long)kCorrChunk, s1 - base);
    __syncthreads();
    for (int t = threadIdx.x; t < len; t += blockDim.x)
      seg[t] = pack_digits(list[base + t], g);
    __syncthreads();
    for (int j = c0 + warp; j < c1; j += nwarps) {
      const unsigned long long cw = pack_digits(cand[j], g);
      unsigned hit = 0;
      for (int t = lane; t < len; t += 32)
        hit += within<PROB>(cw, seg[t], g.n, g.R, sax);
      hit = __reduce_add_sync(0xffffffffu, hit);
      if (lane == 0 && hit) atomicAdd(&gain[j], (int32_t)hit);
    }
  }
}

static SetGeom set_geom(const Geometry &g) {
  SetGeom s{};
  s.prob = g.prob;
  s.n = g.n;
  s.R = g.R;
  for (int j = 0; j < g.n && j < 16; j++) s.ax[j] = g.ax[j];
  return s;
}

int launch_list_pred(const Geometry &g, const uint16_t *cnt, int mode,
                     int target, unsigned long long *out, long long cap,
                     unsigned long long *found, cudaStream_t s) {
  CC_CK(cudaMemsetAsync(found, 0, 8, s));
  const long long nvec = (g.space + 7) >> 3;
  long long blocks = (nvec + 255) / 256;
  if (blocks > (long long)sm_count() * 8) blocks = (long long)sm_count() * 8;
  if (blocks < 1) blocks = 1;
  k_list_pred<<<(unsigned)blocks, 256, 0, s>>>(cnt, g.space, mode, target,
                                                g.mu, set_geom(g), out, cap,
                                                found);
  CC_CK(cudaGetLastError());
  return 0;
}

int launch_gather_set(const Geometry &g, const long long *dcand, int nc,
                      const unsigned long long *Z, long long zn, int32_t *out,
                      bool zeroed, cudaStream_t s) {
  if (nc <= 0) return 0;
  if (!zeroed) CC_CK(cudaMemsetAsync(out, 0, (size_t)nc * 4, s));
  if (zn <= 0) return 0;
  const long long tiles = (nc + kSetTile - 1) / kSetTile;
  // enough Z chunks to give every SM several blocks, each chunk at least
  // one pass of the block's threads
  long long want = (long long)sm_count() * 8 / tiles;
  long long chunks = (zn + 255) / 256;
  if (chunks > want) chunks = want;
  if (chunks > 65535) chunks = 65535;
  if (chunks < 1) chunks = 1;
  const long long zchunk = (zn + chunks - 1) / chunks;
  chunks = (zn + zchunk - 1) / zchunk;
  const dim3 grid((unsigned)tiles, (unsigned)chunks);
  const SetGeom sg = set_geom(g);
  switch (g.prob) {
    case kHamming:
      k_gather_set<kHamming><<<grid, 256, 0, s>>>(dcand, nc, Z, zn, zchunk, sg,
                                                  out);
      break;
    case kLee:
      k_gather_set<kLee><<<grid, 256, 0, s>>>(dcand, nc, Z, zn, zchunk, sg,
                                              out);
      break;
    case kTorus:
      k_gather_set<kTorus><<<grid, 256, 0, s>>>(dcand, nc, Z, zn, zchunk, sg,
                                                out);
      break;
    default:
      k_gather_set<kGrid><<<grid, 256, 0, s>>>(dcand, nc, Z, zn, zchunk, sg,
                                               out);
      break;
  }
  CC_CK(cudaGetLastError());
  return 0;
}

int launch_swap_corr(const Geometry &g, int k, const long long *dcand,
                     const int32_t *dcoff, const int32_t *offs,
                     const long long *list, long long cap, int32_t *gain,
                     cudaStream_t s) {
  if (k <= 0) return 0;
  const SetGeom sg = set_geom(g);
  switch (g.prob) {
    case kHamming:
      k_swap_corr<kHamming><<<k, 256, 0, s>>>(dcand, dcoff, offs, list, cap,
                                              sg, gain);
      break;
    case kLee:
      k_swap_corr<kLee><<<k, 256, 0, s>>>(dcand, dcoff, offs, list, cap, sg,
                                          gain);
      break;
    case kTorus:
      k_swap_corr<kTorus><<<k, 256, 0, s>>>(dcand, dcoff, offs, list, cap, sg,
                                            gain);
      break;
    default:
      k_swap_corr<kGrid><<<k, 256, 0, s>>>(dcand, dcoff, offs, list, cap, sg,
                                           gain);
      break;
  }
  CC_CK(cudaGetLastError());
  return 0;
}

}  // namespace cc
