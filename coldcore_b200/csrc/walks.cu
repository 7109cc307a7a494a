// walks.cu — exact incremental updates and per-candidate queries over a
// word's support set (its metric ball).
//
// Semantics of the reference's support walks
// (coldcore src/plugins/covering/dctcore_core.cuh:158-273, dctcore_grid.cuh
// :239-342, dctcore_mu.cuh:75-105, dctcore_fast.cuh:360-389): the ball of a
// centre w is the support table's patterns applied to w's digits, each
// pattern a set of (position, circular shift) pairs; the open grid rejects a
// pattern whose shift wraps past a board edge.  cnt is a uint16 plane,
// updated with packed 32-bit atomics on the aligned counter pair (the plane
// is padded, so the partner of the last counter exists and stays 0).
//
// The table is held as 32-bit (position, delta) slots instead of the v1
// nibble bytes, so axes of any width walk (the v1 format stops at 16).  A
// block owns one word (or a slice of its ball when the ball is large): the
// word's digits, axis sizes and strides sit in shared memory, and each
// thread resolves one pattern at a time with a few integer ops per slot.
#include <cstdlib>

#include "engine.h"

namespace cc {

struct WordSmem {
  int dig[kMaxAxes];
  int ax[kMaxAxes];
  long long pw[kMaxAxes];
};

__device__ __forceinline__ void word_setup(const Geometry &g, long long w,
                                           WordSmem &s) {
  for (int j = threadIdx.x; j < g.n; j += blockDim.x) {
    s.dig[j] = (int)((w / g.pw[j]) % g.ax[j]);
    s.ax[j] = g.ax[j];
    s.pw[j] = g.pw[j];
  }
  __syncthreads();
}

// word index of pattern t around w; -1 when the open grid rejects it
template <bool GRID>
__device__ __forceinline__ long long walk_word(const WalkArgs &a, long long w,
                                               long long t, const WordSmem &s) {
  long long x = w;
#pragma unroll 1
  for (int k = 0; k < a.slots; k++) {
    const int code = a.tbl[(long long)k * a.len + t];
    if (!code) break;
    const int p = code >> 24, dl = code & 0xFFFFFF;
    const int dg = s.dig[p];
    int nd = dg + dl;
    if (nd >= s.ax[p]) nd -= s.ax[p];
    const int sh = nd - dg;
    if (GRID && (sh > a.g.R || sh < -a.g.R)) return -1;
    x += (long long)sh * s.pw[p];
  }
  return x;
}

__device__ __forceinline__ long long block_sum(long long v) {
  __shared__ long long red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();                      // red may be in use by a prior call
  if (lane == 0) red[wid] = v;
  __syncthreads();
  v = threadIdx.x < (blockDim.x >> 5) ? red[lane] : 0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;                             // valid in thread 0
}

// cnt[x] += delta over each word's support set.  trans != nullptr also
// counts the deficit transitions read off the atomics' old values (an
// increment from c < mu, a decrement from c <= mu).
template <bool GRID, bool PARAM>
__global__ void __launch_bounds__(256)
k_update(const WalkArgs a, const long long *words, const WordsParam pw,
         int split, int delta, unsigned long long *trans) {
  __shared__ WordSmem s;
  const int wi = blockIdx.x / split, seg = blockIdx.x % split;
  const long long w = PARAM ? pw.w[wi] : words[wi];
  word_setup(a.g, w, s);
  long long acc = 0;
  const long long step = (long long)split * blockDim.x;
  for (long long t = (long long)seg * blockDim.x + threadIdx.x; t < a.len;
       t += step) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0) continue;
    uint32_t *cell = reinterpret_cast<uint32_t *>(a.cnt + (x & ~1LL));
    const int sh = (x & 1) ? 16 : 0;
    const uint32_t add = 1u << sh;
    const uint32_t old = delta > 0 ? atomicAdd(cell, add) : atomicSub(cell, add);
    if (trans) {
      const int c = (int)((old >> sh) & 0xFFFFu);
      acc += delta > 0 ? (c < a.g.mu) : (c <= a.g.mu);
    }
  }
  if (trans) {
    acc = block_sum(acc);
    if (threadIdx.x == 0 && acc) atomicAdd(trans, (unsigned long long)acc);
  }
}

// out[wi] = #{x in B(w_i) : pred(cnt[x])}; split blocks per word add up
template <bool GRID>
__global__ void __launch_bounds__(256)
k_gather(const WalkArgs a, const long long *words, int split, int mode,
         int target, int32_t *out) {
  __shared__ WordSmem s;
  const int wi = blockIdx.x / split, seg = blockIdx.x % split;
  const long long w = words[wi];
  word_setup(a.g, w, s);
  long long acc = 0;
  const long long step = (long long)split * blockDim.x;
  for (long long t = (long long)seg * blockDim.x + threadIdx.x; t < a.len;
       t += step) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x >= 0) acc += cnt_pred(mode, (int)a.cnt[x], target, a.g.mu);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) {
    if (split == 1) out[wi] = (int32_t)acc;
    else if (acc) atomicAdd(&out[wi], (int32_t)acc);
  }
}

// out[wi][b] = #{x in B(w_i) : bin(x) == b}.  src 0 bins the map in log2
// steps (0 for v <= 0, 1 for v == 1, 2 for 2..3, 3 for 4..7, ...), src 1
// bins cnt linearly (cnt == b); both clip to nbins - 1.
template <bool GRID>
__global__ void __launch_bounds__(256)
k_ball_hist(const WalkArgs a, const long long *words, int split,
            const int32_t *map, int src, int nbins, int32_t *out) {
  __shared__ WordSmem s;
  __shared__ int32_t hist[32];
  const int wi = blockIdx.x / split, seg = blockIdx.x % split;
  const long long w = words[wi];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) hist[b] = 0;
  word_setup(a.g, w, s);
  const long long step = (long long)split * blockDim.x;
  for (long long t = (long long)seg * blockDim.x + threadIdx.x; t < a.len;
       t += step) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0) continue;
    int b;
    if (src == 0) {
      const int32_t v = map[x];
      b = v <= 0 ? 0 : min(nbins - 1, 32 - __clz(v));
    } else {
      b = min(nbins - 1, (int)a.cnt[x]);
    }
    atomicAdd(&hist[b], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    if (hist[b]) atomicAdd(&out[(long long)wi * nbins + b], hist[b]);
}

int launch_ball_hist(const WalkArgs &w, const long long *dwords, int nb,
                     const int32_t *map, int src, int nbins, int32_t *out,
                     cudaStream_t s) {
  if (nb <= 0) return 0;
  const int split = pick_split(w.len, nb);
  CC_CK(cudaMemsetAsync(out, 0, (size_t)nb * nbins * 4, s));
  const dim3 grid((unsigned)nb * split);
  if (w.g.prob == kGrid)
    k_ball_hist<true><<<grid, 256, 0, s>>>(w, dwords, split, map, src, nbins,
                                           out);
  else
    k_ball_hist<false><<<grid, 256, 0, s>>>(w, dwords, split, map, src,
                                            nbins, out);
  CC_CK(cudaGetLastError());
  return 0;
}

// the R + 1 layer values at each of k words: out[i][d]
__global__ void k_layers_at(const int32_t *layers, long long plane, int R1,
                            const long long *idx, int k, int32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  for (int d = 0; d < R1; d++) out[(long long)i * R1 + d] =
      layers[d * plane + idx[i]];
}

int launch_layers_at(const int32_t *layers, long long plane, int R1,
                     const long long *idx, int k, int32_t *out,
                     cudaStream_t s) {
  if (k <= 0) return 0;
  k_layers_at<<<(k + 255) / 256, 256, 0, s>>>(layers, plane, R1, idx, k, out);
  CC_CK(cudaGetLastError());
  return 0;
}

// swap evaluation, first walk: per drop word, its loss (critical ball words)
// and nmu = its ball words at exactly mu, the words that become deficient
// when one copy of the drop is removed
template <bool GRID>
__global__ void __launch_bounds__(256)
k_drop_count(const WalkArgs a, const long long *drops, int split,
             int32_t *loss, int32_t *nmu) {
  __shared__ WordSmem s;
  const int wi = blockIdx.x / split, seg = blockIdx.x % split;
  const long long w = drops[wi];
  word_setup(a.g, w, s);
  long long lo = 0, at = 0;
  const long long step = (long long)split * blockDim.x;
  for (long long t = (long long)seg * blockDim.x + threadIdx.x; t < a.len;
       t += step) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0) continue;
    const int c = (int)a.cnt[x];
    lo += c >= 1 && c <= a.g.mu;
    at += c == a.g.mu;
  }
  lo = block_sum(lo);
  if (threadIdx.x == 0 && lo) atomicAdd(&loss[wi], (int32_t)lo);
  at = block_sum(at);
  if (threadIdx.x == 0 && at) atomicAdd(&nmu[wi], (int32_t)at);
}

// second walk: the words at exactly mu, into the drop's segment of `list`
// (cursor[i] starts at the segment's offset); slots past cap are dropped and
// the caller, seeing the total above cap, falls back
template <bool GRID>
__global__ void __launch_bounds__(256)
k_drop_list(const WalkArgs a, const long long *drops, int split,
            int32_t *cursor, long long cap, long long *list) {
  __shared__ WordSmem s;
  const int wi = blockIdx.x / split, seg = blockIdx.x % split;
  const long long w = drops[wi];
  word_setup(a.g, w, s);
  const long long step = (long long)split * blockDim.x;
  for (long long t = (long long)seg * blockDim.x + threadIdx.x; t < a.len;
       t += step) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0 || (int)a.cnt[x] != a.g.mu) continue;
    const int slot = atomicAdd(&cursor[wi], 1);
    if (slot < cap) list[slot] = x;
  }
}

int launch_drop_walks(const WalkArgs &w, const long long *ddrops, int k,
                      int32_t *loss, int32_t *nmu, int32_t *offs,
                      int32_t *cursor, long long cap, long long *list,
                      cudaStream_t s) {
  if (k <= 0) return 0;
  const int split = pick_split(w.len, k);
  const dim3 grid((unsigned)k * split);
  const bool gp = w.g.prob == kGrid;
  if (gp) k_drop_count<true><<<grid, 256, 0, s>>>(w, ddrops, split, loss, nmu);
  else k_drop_count<false><<<grid, 256, 0, s>>>(w, ddrops, split, loss, nmu);
  CC_CK(cudaGetLastError());
  int rc = launch_seg_scan(nmu, k, cap, offs, cursor, s);
  if (rc) return rc;
  if (gp)
    k_drop_list<true><<<grid, 256, 0, s>>>(w, ddrops, split, cursor, cap, list);
  else
    k_drop_list<false><<<grid, 256, 0, s>>>(w, ddrops, split, cursor, cap,
                                            list);
  CC_CK(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------ device greedy
// State of one device-side greedy fill (all fields in device memory).
// best: the packed argmax key of the current step, (gain ^ sign) << 32 |
// ~index, so the largest gain wins and ties go to the smallest index.
struct GreedyState {
  unsigned long long best;
  long long deficit;          // sum max(0, mu - cnt), maintained exactly
  int done;                   // 1: no positive gain or nothing uncovered
  int placed;                 // words placed so far
  int nnew;                   // words satisfied by the last placement
  int pad;
};
static_assert(sizeof(GreedyState) == kGreedyStateBytes, "state layout");

__device__ __forceinline__ unsigned long long greedy_key(int32_t v,
                                                         long long x) {
  return ((unsigned long long)((uint32_t)v ^ 0x80000000u) << 32) |
         (uint32_t)~(uint32_t)x;
}

// map[x] = exclude for every listed word (incumbents never re-enter)
__global__ void k_greedy_exclude(int32_t *map, const long long *words, int n,
                                 int32_t exclude) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) map[words[i]] = exclude;
}

// step 1: best = argmax map (largest value, then smallest index)
__global__ void __launch_bounds__(256)
k_greedy_argmax(const int32_t *map, long long N, GreedyState *st) {
  if (st->done) return;
  unsigned long long k = 0;
  const long long gs = (long long)gridDim.x * blockDim.x;
  const long long nv = N >> 2;
  const int4 *v4 = reinterpret_cast<const int4 *>(map);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       i < nv; i += gs) {
    const int4 q = __ldcg(v4 + i);
    k = max(k, greedy_key(q.x, 4 * i));
    k = max(k, greedy_key(q.y, 4 * i + 1));
    k = max(k, greedy_key(q.z, 4 * i + 2));
    k = max(k, greedy_key(q.w, 4 * i + 3));
  }
  if (blockIdx.x == 0 && threadIdx.x < (N & 3))
    k = max(k, greedy_key(map[nv * 4 + threadIdx.x], nv * 4 + threadIdx.x));
  for (int o = 16; o > 0; o >>= 1)
    k = max(k, __shfl_down_sync(0xffffffffu, k, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&st->best, k);
}

// step 2: place the argmax word (one block): cnt += 1 over its ball, the
// words it satisfies (old count mu - 1) go to `fresh`, the deficit drops by
// the words it serves (old count < mu)
template <bool GRID>
__global__ void __launch_bounds__(256)
k_greedy_place(const WalkArgs a, int32_t *map, GreedyState *st,
               long long *placed, int max_add, long long *fresh,
               int32_t exclude) {
  __shared__ WordSmem s;
  __shared__ long long w_s;
  __shared__ int stop;
  __shared__ int nfresh;
  __shared__ long long served;
  if (threadIdx.x == 0) {
    stop = st->done;
    if (!stop) {
      const unsigned long long k = st->best;
      const int32_t v = (int32_t)((uint32_t)(k >> 32) ^ 0x80000000u);
      const long long x = (long long)(uint32_t)~(uint32_t)k;
      if (v <= 0 || st->deficit <= 0 || st->placed >= max_add) {
        st->done = 1;
        stop = 1;
      } else {
        w_s = x;
        placed[st->placed] = x;
        st->placed += 1;
        map[x] = exclude;
      }
    }
    st->best = 0;                     // fresh for the next step's argmax
    st->nnew = 0;
    nfresh = 0;
    served = 0;
  }
  __syncthreads();
  if (stop) return;
  const long long w = w_s;
  word_setup(a.g, w, s);
  long long mine = 0;
  for (long long t = threadIdx.x; t < a.len; t += blockDim.x) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0) continue;
    uint32_t *cell = reinterpret_cast<uint32_t *>(a.cnt + (x & ~1LL));
    const int sh = (x & 1) ? 16 : 0;
    const uint32_t old = atomicAdd(cell, 1u << sh);
    const int c = (int)((old >> sh) & 0xFFFFu);
    if (c < a.g.mu) mine++;
    if (c == a.g.mu - 1) fresh[atomicAdd(&nfresh, 1)] = x;
  }
  mine = block_sum(mine);
  if (threadIdx.x == 0) {
    st->deficit -= mine;
    st->nnew = nfresh;
  }
}

// step 3: every word satisfied by the placement stops counting towards the
// gain of the candidates whose balls hold it: map[y] -= 1 for y in B(u)
template <bool GRID>
__global__ void __launch_bounds__(256)
k_greedy_refresh(const WalkArgs a, int32_t *map, const GreedyState *st,
                 const long long *fresh) {
  __shared__ WordSmem s;
  if (st->done) return;
  const int n = st->nnew;
  for (int u = blockIdx.x; u < n; u += gridDim.x) {
    const long long x0 = fresh[u];
    __syncthreads();                      // s is reused across words
    word_setup(a.g, x0, s);
    for (long long t = threadIdx.x; t < a.len; t += blockDim.x) {
      const long long y = walk_word<GRID>(a, x0, t, s);
      if (y >= 0) atomicSub(&map[y], 1);
    }
  }
}

// ------------------------------------------------------------ batched greedy
// The same exact greedy over many cells at once (the batched engine's
// campaign repair): one argmax, one place and one refresh launch per step
// for every cell, each cell's state and buffers in its BatchGreedyCell.
// Cells that are done return at once, so the launches of a step cost only
// the cells still placing.
constexpr int kArgmaxChunk = 8192;        // words per argmax block

__global__ void __launch_bounds__(256)
k_bgreedy_argmax(const BatchGreedyCell *cells) {
  const BatchGreedyCell &c = cells[blockIdx.y];
  GreedyState *st = reinterpret_cast<GreedyState *>(c.st);
  if (st->done) return;
  const long long N = c.w.g.space;
  const long long x0 = (long long)blockIdx.x * kArgmaxChunk;
  if (x0 >= N) return;
  const long long x1 = min(N, x0 + (long long)kArgmaxChunk);
  unsigned long long k = 0;
  for (long long x = x0 + threadIdx.x; x < x1; x += blockDim.x)
    k = max(k, greedy_key(__ldcg(c.map + x), x));
  for (int o = 16; o > 0; o >>= 1)
    k = max(k, __shfl_down_sync(0xffffffffu, k, o));
  if ((threadIdx.x & 31) == 0 && k) atomicMax(&st->best, k);
}

template <bool GRID>
__device__ __forceinline__ void bgreedy_place(const BatchGreedyCell &c,
                                              int32_t exclude) {
  __shared__ WordSmem s;
  __shared__ long long w_s;
  __shared__ int stop;
  __shared__ int nfresh;
  GreedyState *st = reinterpret_cast<GreedyState *>(c.st);
  const WalkArgs &a = c.w;
  if (threadIdx.x == 0) {
    stop = st->done;
    if (!stop) {
      const unsigned long long k = st->best;
      const int32_t v = (int32_t)((uint32_t)(k >> 32) ^ 0x80000000u);
      const long long x = (long long)(uint32_t)~(uint32_t)k;
      if (k == 0 || v <= 0 || st->deficit <= 0 || st->placed >= c.max_add) {
        st->done = 1;
        stop = 1;
      } else {
        w_s = x;
        c.placed[st->placed] = x;
        st->placed += 1;
        c.map[x] = exclude;
      }
    }
    st->best = 0;
    st->nnew = 0;
    nfresh = 0;
  }
  __syncthreads();
  if (stop) return;
  const long long w = w_s;
  word_setup(a.g, w, s);
  long long mine = 0;
  for (long long t = threadIdx.x; t < a.len; t += blockDim.x) {
    const long long x = walk_word<GRID>(a, w, t, s);
    if (x < 0) continue;
    uint32_t *cell = reinterpret_cast<uint32_t *>(a.cnt + (x & ~1LL));
    const int sh = (x & 1) ? 16 : 0;
    const uint32_t old = atomicAdd(cell, 1u << sh);
    const int cv = (int)((old >> sh) & 0xFFFFu);
    if (cv < a.g.mu) mine++;
    if (cv == a.g.mu - 1) c.fresh[atomicAdd(&nfresh, 1)] = x;
  }
  mine = block_sum(mine);
  if (threadIdx.x == 0) {
    st->deficit -= mine;
    st->nnew = nfresh;
  }
}

__global__ void __launch_bounds__(256)
k_bgreedy_place(const BatchGreedyCell *cells, int32_t exclude) {
  const BatchGreedyCell &c = cells[blockIdx.x];
  if (c.w.g.prob == kGrid) bgreedy_place<true>(c, exclude);
  else bgreedy_place<false>(c, exclude);
}

template <bool GRID>
__device__ __forceinline__ void bgreedy_refresh(const BatchGreedyCell &c) {
  __shared__ WordSmem s;
  const GreedyState *st = reinterpret_cast<const GreedyState *>(c.st);
  if (st->done) return;
  const int n = st->nnew;
  for (int u = blockIdx.x; u < n; u += gridDim.x) {
    const long long x0 = c.fresh[u];
    __syncthreads();
    word_setup(c.w.g, x0, s);
    for (long long t = threadIdx.x; t < c.w.len; t += blockDim.x) {
      const long long y = walk_word<GRID>(c.w, x0, t, s);
      if (y >= 0) atomicSub(&c.map[y], 1);
    }
  }
}

__global__ void __launch_bounds__(256)
k_bgreedy_refresh(const BatchGreedyCell *cells) {
  const BatchGreedyCell &c = cells[blockIdx.y];
  if (c.w.g.prob == kGrid) bgreedy_refresh<true>(c);
  else bgreedy_refresh<false>(c);
}

// one step for every cell of the table
int launch_batch_greedy_step(const BatchGreedyCell *dcells, int ncells,
                             long long max_space, int32_t exclude,
                             cudaStream_t s) {
  if (ncells <= 0) return 0;
  const dim3 ga((unsigned)((max_space + kArgmaxChunk - 1) / kArgmaxChunk),
                (unsigned)ncells);
  k_bgreedy_argmax<<<ga, 256, 0, s>>>(dcells);
  k_bgreedy_place<<<(unsigned)ncells, 256, 0, s>>>(dcells, exclude);
  k_bgreedy_refresh<<<dim3(16, (unsigned)ncells), 256, 0, s>>>(dcells);
  CC_CK(cudaGetLastError());
  return 0;
}

int launch_greedy_exclude(int32_t *map, const long long *dwords, int n,
                          int32_t exclude, cudaStream_t s) {
  if (n <= 0) return 0;
  k_greedy_exclude<<<(n + 255) / 256, 256, 0, s>>>(map, dwords, n, exclude);
  CC_CK(cudaGetLastError());
  return 0;
}

int launch_greedy_step(const WalkArgs &w, int32_t *map, long long N,
                       GreedyState *st, long long *placed, int max_add,
                       long long *fresh, int32_t exclude, cudaStream_t s) {
  long long blocks = ((N >> 2) + 255) / 256;
  const long long cap = (long long)sm_count() * 4;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  k_greedy_argmax<<<(unsigned)blocks, 256, 0, s>>>(map, N, st);
  const bool gp = w.g.prob == kGrid;
  if (gp)
    k_greedy_place<true><<<1, 256, 0, s>>>(w, map, st, placed, max_add, fresh,
                                           exclude);
  else
    k_greedy_place<false><<<1, 256, 0, s>>>(w, map, st, placed, max_add,
                                            fresh, exclude);
  const unsigned rb = (unsigned)(sm_count() * 4);
  if (gp) k_greedy_refresh<true><<<rb, 256, 0, s>>>(w, map, st, fresh);
  else k_greedy_refresh<false><<<rb, 256, 0, s>>>(w, map, st, fresh);
  CC_CK(cudaGetLastError());
  return 0;
}

// blocks per word so that single-word walks still fill the GPU
// ------------------------------------------------------------ tiled gather
// Many candidates over a large ball: the per-word kernel above re-reads the
// whole support table for every candidate (|B| x slots x 4 bytes, 546 KB a
// candidate at ternary n=16, R=4), so a call with 10^5 candidates streams
// tens of GB of table through L2.  Here a block takes a tile of kTilePat
// patterns and a group of kTileCand candidates:
//   * the tile is decoded once into 16-bit offset indices, four to a 64-bit
//     shared word (a missing slot points at a zero entry, so every pattern
//     takes the same adds, branch-free);
//   * each candidate's index offsets per (position, shift) sit in shared
//     memory (32-bit: cells below 2^31 words);
//   * each warp walks the whole tile for one candidate at a time, 32
//     consecutive patterns a step and eight steps in flight, so one
//     candidate's loads stay close together in time and in address (the
//     table is sorted by offset) and reuse L1 like a per-word sweep.
// The table is read once per candidate group instead of once per candidate.
constexpr int kTilePat = 512;           // patterns per block
constexpr int kTileCand = 32;           // candidates per block
constexpr int kTileMaxOff = 128;        // offset entries per candidate

// The predicate of one gather call as a bit plane: bit x of bits is
// pred(cnt[x]).  Eight counters (one 16-byte load) per thread and byte.
__global__ void __launch_bounds__(256)
k_pred_bits(const uint16_t *cnt, long long n, int mode, int target, int mu,
            uint8_t *bits) {
  const long long nbytes = (n + 7) / 8;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       i < nbytes; i += stride) {
    unsigned m = 0;
    if (8 * i + 8 <= n) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(cnt) + i);
      const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        m |= (unsigned)cnt_pred(mode, (int)(w[k] & 0xFFFFu), target, mu)
             << (2 * k);
        m |= (unsigned)cnt_pred(mode, (int)(w[k] >> 16), target, mu)
             << (2 * k + 1);
      }
    } else {
      for (long long x = 8 * i; x < n; x++)
        m |= (unsigned)cnt_pred(mode, (int)cnt[x], target, mu)
             << (int)(x - 8 * i);
    }
    bits[i] = (uint8_t)m;
  }
}

template <int MAXS, bool BITS>
__global__ void __launch_bounds__(256, 6)
k_gather_tiled(const WalkArgs a, const long long *words, int nb, int mode,
               int target, int32_t *out, int noff, const uint8_t *bits) {
  constexpr int NQ = MAXS / 4;            // 64-bit words of indices a pattern
  __shared__ int32_t off[kTileCand * kTileMaxOff];
  __shared__ unsigned long long idx[kTilePat * NQ];
  __shared__ int32_t base[kMaxAxes];
  __shared__ int32_t cand[kTileCand];
  const int c0 = blockIdx.y * kTileCand;
  const int nc = min(kTileCand, nb - c0);
  const long long t0 = (long long)blockIdx.x * kTilePat;
  const int np = (int)min((long long)kTilePat, a.len - t0);
  if (threadIdx.x == 0) {
    int b = 0;
    for (int j = 0; j < a.g.n; j++) { base[j] = b; b += a.g.ax[j] - 1; }
  }
  if (threadIdx.x < kTileCand)
    cand[threadIdx.x] = threadIdx.x < nc ? (int32_t)words[c0 + threadIdx.x]
                                         : 0;
  __syncthreads();
  // index offsets of every (position, shift) around each candidate; entry
  // noff is the zero a missing slot adds
  for (int i = threadIdx.x; i < nc * (noff + 1); i += blockDim.x) {
    const int c = i / (noff + 1), e = i % (noff + 1);
    int v = 0;
    if (e < noff) {
      int j = 0;
      while (j + 1 < a.g.n && base[j + 1] <= e) j++;
      const int q = a.g.ax[j], dl = e - base[j] + 1;
      const int pw = (int)a.g.pw[j];
      const int dg = (cand[c] / pw) % q;
      const int nd = dg + dl >= q ? dg + dl - q : dg + dl;
      v = (nd - dg) * pw;
    }
    off[c * kTileMaxOff + e] = v;
  }
  // the tile's patterns as offset indices
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
#pragma unroll
    for (int h = 0; h < NQ; h++) {
      unsigned long long wv = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int s = 4 * h + k;
        int code = 0;
        if (s < a.slots) code = a.tbl[(long long)s * a.len + t0 + p];
        const unsigned e = code ? (unsigned)(base[code >> 24] +
                                             (code & 0xFFFFFF) - 1)
                                : (unsigned)noff;
        wv |= (unsigned long long)e << (16 * k);
      }
      idx[p * NQ + h] = wv;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  for (int c = warp; c < nc; c += nwarps) {
    const int32_t *oc = off + c * kTileMaxOff;
    const int32_t w = cand[c];
    int hits = 0;
#pragma unroll 8
    for (int p = lane; p < np; p += 32) {
      int32_t x = w;
#pragma unroll
      for (int h = 0; h < NQ; h++) {
        const unsigned long long wv = idx[p * NQ + h];
        x += oc[wv & 0xFFFF] + oc[(wv >> 16) & 0xFFFF] +
             oc[(wv >> 32) & 0xFFFF] + oc[wv >> 48];
      }
      if (BITS)
        hits += (__ldg(bits + (x >> 3)) >> (x & 7)) & 1;
      else
        hits += cnt_pred(mode, (int)__ldg(a.cnt + x), target, a.g.mu);
    }
    hits = __reduce_add_sync(0xffffffffu, hits);
    if (lane == 0 && hits) atomicAdd(&out[c0 + c], hits);
  }
}

// the tiled gather applies: Hamming / Lee / torus cells below 2^31 words,
// offsets table within bounds, at most 8 slots, enough candidates to share
// a table tile (CC_GATHER_TILED=0 turns it off, =1 forces it on)
bool gather_tiled_ok(const WalkArgs &w, int nb, int *noff) {
  if (w.g.prob == kGrid || w.g.space >= (1LL << 31) || w.slots > 8 ||
      w.len >= (1LL << 31))
    return false;
  int n = 0;
  for (int j = 0; j < w.g.n; j++) n += w.g.ax[j] - 1;
  if (n >= kTileMaxOff) return false;          // entry n is the zero
  *noff = n;
  if ((long long)nb > 65535LL * kTileCand) return false;   // grid y
  const char *e = getenv("CC_GATHER_TILED");
  if (e) return atoi(e) != 0;
  return nb >= 16 && w.len >= 2048;
}

// A bit plane pays when the call reads more ball words than the plane
// costs to build (one pass over cnt): candidates x |B| >= |X|.
// CC_GATHER_BITS=0 turns it off, =1 forces it on.
bool gather_bits_pay(const WalkArgs &w, int nb) {
  int noff = 0;
  if (!gather_tiled_ok(w, nb, &noff)) return false;
  const char *e = getenv("CC_GATHER_BITS");
  if (e) return atoi(e) != 0;
  return (double)nb * (double)w.len >= (double)w.g.space;
}

int pick_split(long long len, int nb) {
  long long cover = (len + 255) / 256;
  long long split = (long long)sm_count() * 64 / (nb > 0 ? nb : 1);
  if (split < 1) split = 1;
  if (split > cover) split = cover;
  if (split > 65535) split = 65535;
  return (int)split;
}

int launch_update(const WalkArgs &w, const long long *dwords,
                  const WordsParam *pw, int nb, int delta,
                  unsigned long long *trans, cudaStream_t s) {
  if (nb <= 0) return 0;
  const int split = pick_split(w.len, nb);
  const dim3 grid((unsigned)nb * split);
  const bool grid_prob = w.g.prob == kGrid;
  static WordsParam empty;
  if (dwords) {
    if (grid_prob) k_update<true, false><<<grid, 256, 0, s>>>(w, dwords, empty, split, delta, trans);
    else k_update<false, false><<<grid, 256, 0, s>>>(w, dwords, empty, split, delta, trans);
  } else {
    if (grid_prob) k_update<true, true><<<grid, 256, 0, s>>>(w, nullptr, *pw, split, delta, trans);
    else k_update<false, true><<<grid, 256, 0, s>>>(w, nullptr, *pw, split, delta, trans);
  }
  CC_CK(cudaGetLastError());
  return 0;
}

int launch_gather(const WalkArgs &w, const long long *dwords, int nb,
                  int mode, int target, int32_t *out, bool zeroed,
                  cudaStream_t s, uint8_t *bits) {
  if (nb <= 0) return 0;
  int noff = 0;
  if (gather_tiled_ok(w, nb, &noff)) {
    if (!zeroed) CC_CK(cudaMemsetAsync(out, 0, (size_t)nb * 4, s));
    if (bits) {
      const long long nbytes = (w.g.space + 7) / 8;
      long long nbk = (nbytes + 255) / 256;
      if (nbk > (long long)sm_count() * 32) nbk = (long long)sm_count() * 32;
      k_pred_bits<<<(unsigned)nbk, 256, 0, s>>>(w.cnt, w.g.space, mode,
                                                target, w.g.mu, bits);
      CC_CK(cudaGetLastError());
    }
    const dim3 tg((unsigned)((w.len + kTilePat - 1) / kTilePat),
                  (unsigned)((nb + kTileCand - 1) / kTileCand));
#define TG(M, B) k_gather_tiled<M, B><<<tg, 256, 0, s>>>(                  \
        w, dwords, nb, mode, target, out, noff, bits)
    if (w.slots <= 4) { if (bits) TG(4, true); else TG(4, false); }
    else { if (bits) TG(8, true); else TG(8, false); }
#undef TG
    CC_CK(cudaGetLastError());
    return 0;
  }
  const int split = pick_split(w.len, nb);
  if (split > 1 && !zeroed)
    CC_CK(cudaMemsetAsync(out, 0, (size_t)nb * 4, s));
  const dim3 grid((unsigned)nb * split);
  if (w.g.prob == kGrid)
    k_gather<true><<<grid, 256, 0, s>>>(w, dwords, split, mode, target, out);
  else
    k_gather<false><<<grid, 256, 0, s>>>(w, dwords, split, mode, target, out);
  CC_CK(cudaGetLastError());
  return 0;
}

}  // namespace cc
