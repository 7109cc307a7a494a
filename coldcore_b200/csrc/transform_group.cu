// transform_group.cu — multi-axis transform kernels for the distance-layer
// families (Hamming, Lee) and small-axis window families (torus, grid).
//
// The per-axis recurrences are the reference's
// (coldcore src/plugins/covering/dctcore_hamming.cuh:4-8 for Hamming,
//  dctcore_lee.cuh:4-14 for Lee, dctcore_torus.cuh:1-12 and
//  dctcore_grid.cuh:1-30 for the window sums); the schedule is this engine's
// own.  One launch runs a GROUP of consecutive axes over a tile held in
// shared memory, so the (R+1) int32 layer planes cross HBM once per group
// instead of once per axis:
//
//   * a tile is W consecutive inner positions x the group's mid = prod a_j
//     words x Bo outer slabs (W = 32 words = one 128-byte line on strided
//     groups, W = 1 and a contiguous range on the first group);
//   * a ROUND loads, per thread, a register block of Q^rb words spanning rb
//     of the group's axes (all layers), applies the rb axis recurrences in
//     registers and stores the block back; rounds exchange through shared
//     memory, the first round reads HBM (or derives layer 0 from cnt / the
//     sorted code) and the last writes HBM (layers, the map, or cnt);
//   * thread-to-word maps keep 32 consecutive lanes on 32 consecutive words
//     wherever the round's stride allows (coalesced 128-byte requests), and
//     power-of-two tiles are skewed one word per block to keep the low-axis
//     rounds free of bank conflicts.
//
// Integer arithmetic is exactly the reference's, so every field is bit-exact.
#include <algorithm>

#include "engine.h"

namespace cc {

template <int Q, int B>
struct IPow { static constexpr int v = Q * IPow<Q, B - 1>::v; };
template <int Q>
struct IPow<Q, 0> { static constexpr int v = 1; };

enum Op { kOpHamming = 0, kOpLee = 1, kOpTorus = 2, kOpGrid = 3 };

// ---------------------------------------------------------------- axis ops
// Hamming: newA_d[a] = A_d[a] + T_{d-1} - A_{d-1}[a], T = fibre sum
template <int Q, int R1, int QB, int ST>
__device__ __forceinline__ void axis_hamming(int32_t (&v)[R1][QB]) {
#pragma unroll
  for (int e = 0; e < QB; e++) {
    if ((e / ST) % Q != 0) continue;
    int32_t T[R1];
#pragma unroll
    for (int d = 0; d + 1 < R1; d++) {
      int32_t s = 0;
#pragma unroll
      for (int a = 0; a < Q; a++) s += v[d][e + a * ST];
      T[d] = s;
    }
#pragma unroll
    for (int d = R1 - 1; d >= 1; d--)
#pragma unroll
      for (int a = 0; a < Q; a++)
        v[d][e + a * ST] += T[d - 1] - v[d - 1][e + a * ST];
  }
}

// Lee: newA_d[a] = A_d[a] + sum_{w=1..min(d,Q/2)} (A_{d-w}[a-w] + A_{d-w}[a+w]),
// the two terms counted once when they coincide (even Q, w = Q/2)
template <int Q, int R1, int QB, int ST>
__device__ __forceinline__ void axis_lee(int32_t (&v)[R1][QB]) {
  constexpr int H = Q / 2;
#pragma unroll
  for (int e = 0; e < QB; e++) {
    if ((e / ST) % Q != 0) continue;
#pragma unroll
    for (int d = R1 - 1; d >= 1; d--) {
      int32_t nv[Q];
#pragma unroll
      for (int a = 0; a < Q; a++) {
        int32_t s = v[d][e + a * ST];
#pragma unroll
        for (int w = 1; w <= (d < H ? d : H); w++) {
          const int am = (a - w + Q) % Q, ap = (a + w) % Q;
          s += v[d - w][e + am * ST];
          if (ap != am) s += v[d - w][e + ap * ST];
        }
        nv[a] = s;
      }
#pragma unroll
      for (int a = 0; a < Q; a++) v[d][e + a * ST] = nv[a];
    }
  }
}

// torus / grid: newA[a] = sum over the circular (torus) or clamped (grid)
// window of radius R
template <int Q, int R1, int QB, int ST, bool GRID>
__device__ __forceinline__ void axis_window(int32_t (&v)[R1][QB], int R) {
#pragma unroll
  for (int e = 0; e < QB; e++) {
    if ((e / ST) % Q != 0) continue;
    int32_t nv[Q];
#pragma unroll
    for (int a = 0; a < Q; a++) {
      int32_t s = 0;
#pragma unroll
      for (int b = 0; b < Q; b++) {
        int dd = a > b ? a - b : b - a;
        if (!GRID && Q - dd < dd) dd = Q - dd;
        if (dd <= R) s += v[0][e + b * ST];
      }
      nv[a] = s;
    }
#pragma unroll
    for (int a = 0; a < Q; a++) v[0][e + a * ST] = nv[a];
  }
}

template <int OP, int Q, int R1, int QB, int ST>
__device__ __forceinline__ void apply_axis(int32_t (&v)[R1][QB], int R) {
  if (OP == kOpHamming) axis_hamming<Q, R1, QB, ST>(v);
  else if (OP == kOpLee) axis_lee<Q, R1, QB, ST>(v);
  else axis_window<Q, R1, QB, ST, OP == kOpGrid>(v, R);
}

template <int OP, int Q, int R1, int BM, int T>
struct AxisLoop {
  static __device__ __forceinline__ void run(
      int32_t (&v)[R1][IPow<Q, BM>::v], int rb, int R) {
    if (T < rb) apply_axis<OP, Q, R1, IPow<Q, BM>::v, IPow<Q, T>::v>(v, R);
    AxisLoop<OP, Q, R1, BM, T + 1>::run(v, rb, R);
  }
};
template <int OP, int Q, int R1, int BM>
struct AxisLoop<OP, Q, R1, BM, BM> {
  static __device__ __forceinline__ void run(
      int32_t (&)[R1][IPow<Q, BM>::v], int, int) {}
};

__device__ __forceinline__ int skewed(int p, int skew) {
  return skew ? p + (p >> skew) : p;
}

// Fill layer 0 of the tile (shared memory) with the code multiplicities
// of the contiguous range [x0, x0 + len); other layers are implicit zeros.
__device__ __forceinline__ void stage_code(const GroupArgs &g, int32_t *sm,
                                           long long x0, int len) {
  __shared__ long long s_lo, s_hi;
  for (int p = threadIdx.x; p < len; p += blockDim.x)
    sm[skewed(p, g.skew)] = 0;
  if (threadIdx.x == 0) {
    long long lo = 0, hi = g.ncode;     // lower_bound(x0)
    while (lo < hi) {
      long long md = (lo + hi) >> 1;
      if (g.code[md] < x0) lo = md + 1; else hi = md;
    }
    long long a = lo;
    hi = g.ncode;                       // lower_bound(x0 + len)
    while (lo < hi) {
      long long md = (lo + hi) >> 1;
      if (g.code[md] < x0 + len) lo = md + 1; else hi = md;
    }
    s_lo = a;
    s_hi = lo;
  }
  __syncthreads();
  for (long long t = s_lo + threadIdx.x; t < s_hi; t += blockDim.x)
    atomicAdd(&sm[skewed((int)(g.code[t] - x0), g.skew)], 1);
  __syncthreads();
}

// ------------------------------------------------------------------ kernel
template <int OP, int Q, int R1, int BM>
__global__ void __launch_bounds__(kGroupThreads)
group_kernel(const GroupArgs g) {
  constexpr int QB = IPow<Q, BM>::v;
  extern __shared__ int32_t sm[];
  const long long imid = g.inner * (long long)g.mid;
  const int W = g.W;
  const int tile_words = g.Bo * g.mid;
  const int SD = (skewed(tile_words, g.skew) + 1) * W;   // layer stride
  for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
    const long long o0 = (tile / g.nchunk) * g.Bo;
    const long long i0 = (tile % g.nchunk) * W;
    if (g.src == kSrcCode) {
      // first group only: W == 1, inner == 1, the tile is contiguous
      long long len = (g.outer - o0) * (long long)g.mid;
      stage_code(g, sm, o0 * g.mid, (int)(len < tile_words ? len : tile_words));
    }
    for (int r = 0; r < g.nrounds; r++) {
      const int rb = g.rb[r], S = g.rs[r];
      int ne = 1;
      for (int t = 0; t < rb; t++) ne *= Q;
      const int nh = g.mid / (S * ne);
      const int nblk = W * S * nh * g.Bo;
      const bool first = r == 0, last = r == g.nrounds - 1;
      for (int blk = threadIdx.x; blk < nblk; blk += blockDim.x) {
        const int w = blk % W;
        int rest = blk / W;
        const int mlo = rest % S;
        rest /= S;
        const int mhi = rest % nh;
        const int ob = rest / nh;
        const bool valid = (o0 + ob < g.outer) && (i0 + w < g.inner);
        const long long xb = (o0 + ob) * imid + i0 + w;
        const int pb = ob * g.mid + mlo + S * ne * mhi;   // tile word of e=0
        int32_t v[R1][QB];
        // -------- load
#pragma unroll
        for (int e = 0; e < QB; e++) {
          const int m = mlo + S * e + S * ne * mhi;
          const long long x = xb + (long long)m * g.inner;
          const int sp = skewed(pb + S * e, g.skew) * W + w;
#pragma unroll
          for (int d = 0; d < R1; d++) v[d][e] = 0;
          if (e >= ne) continue;
          if (first && g.src == kSrcLayers) {
            if (valid) {
#pragma unroll
              for (int d = 0; d < R1; d++)
                if (d < g.lin) v[d][e] = g.layers[d * g.plane + x];
            }
          } else if (first && g.src == kSrcCnt) {
            if (valid)
              v[0][e] = cnt_pred(g.pmode, (int)g.cnt[x], g.ptarget, g.mu);
          } else if (first) {                       // kSrcCode: layer 0 only
            v[0][e] = sm[sp];
          } else {
#pragma unroll
            for (int d = 0; d < R1; d++) v[d][e] = sm[d * SD + sp];
          }
        }
        // -------- rb axis recurrences in registers
        AxisLoop<OP, Q, R1, BM, 0>::run(v, rb, g.R);
        // -------- store
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (e >= ne) continue;
          const int m = mlo + S * e + S * ne * mhi;
          const long long x = xb + (long long)m * g.inner;
          const int sp = skewed(pb + S * e, g.skew) * W + w;
          if (!last) {
#pragma unroll
            for (int d = 0; d < R1; d++) sm[d * SD + sp] = v[d][e];
          } else if (valid) {
            if (g.dst == kDstLayers) {
#pragma unroll
              for (int d = 0; d < R1; d++)
                if (d < g.lout) g.layers[d * g.plane + x] = v[d][e];
            } else {
              int32_t s = 0;
#pragma unroll
              for (int d = 0; d < R1; d++) s += v[d][e];
              if (g.dst == kDstMap) g.layers[x] = s;
              else g.cnt[x] = (uint16_t)(s > 65535 ? 65535 : s);
            }
          }
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ generic kernel
// Any axis size (<= 16) and layer count (<= 8), one axis per round, fibres
// processed in place in shared memory.  Used for the cells without a
// register-blocked instantiation (mixed radix, wide Hamming / Lee alphabets,
// small torus / grid axes).
__global__ void __launch_bounds__(512) group_generic(const GroupArgs g) {
  extern __shared__ int32_t sm[];
  const int R1 = g.prob == kTorus || g.prob == kGrid ? 1 : g.R + 1;
  const long long imid = g.inner * (long long)g.mid;
  const int W = g.W;
  const int tile_words = g.Bo * g.mid;
  const int SD = (skewed(tile_words, g.skew) + 1) * W;
  const int nel = tile_words * W;
  for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
    const long long o0 = (tile / g.nchunk) * g.Bo;
    const long long i0 = (tile % g.nchunk) * W;
    if (g.src == kSrcCode) {
      long long len = (g.outer - o0) * (long long)g.mid;
      stage_code(g, sm, o0 * g.mid, (int)(len < tile_words ? len : tile_words));
    }
    // -------- load the tile
    for (int t = threadIdx.x; t < nel; t += blockDim.x) {
      const int w = t % W, p = t / W, ob = p / g.mid, m = p % g.mid;
      const bool valid = (o0 + ob < g.outer) && (i0 + w < g.inner);
      const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
      const int sp = skewed(p, g.skew) * W + w;
      for (int d = 0; d < R1; d++) {
        int32_t val = 0;
        if (g.src == kSrcLayers) {
          if (valid && d < g.lin) val = g.layers[d * g.plane + x];
        } else if (g.src == kSrcCnt) {
          if (valid && d == 0)
            val = cnt_pred(g.pmode, (int)g.cnt[x], g.ptarget, g.mu);
        } else if (d == 0) {
          val = sm[sp];
        }
        sm[d * SD + sp] = val;
      }
    }
    __syncthreads();
    // -------- one axis at a time
    int S = 1;
    for (int j = 0; j < g.k; j++) {
      const int q = g.qax[j];
      const int nh = g.mid / (S * q);
      const int nfib = W * S * nh * g.Bo;
      for (int f = threadIdx.x; f < nfib; f += blockDim.x) {
        const int w = f % W;
        int rest = f / W;
        const int mlo = rest % S;
        rest /= S;
        const int mhi = rest % nh, ob = rest / nh;
        const int pb = ob * g.mid + mlo + S * q * mhi;
        int sp[16];
        for (int a = 0; a < q; a++) sp[a] = skewed(pb + S * a, g.skew) * W + w;
        if (g.prob == kHamming) {
          int32_t T[kMaxLayers];
          for (int d = 0; d + 1 < R1; d++) {
            int32_t s = 0;
            for (int a = 0; a < q; a++) s += sm[d * SD + sp[a]];
            T[d] = s;
          }
          for (int d = R1 - 1; d >= 1; d--)
            for (int a = 0; a < q; a++)
              sm[d * SD + sp[a]] += T[d - 1] - sm[(d - 1) * SD + sp[a]];
        } else if (g.prob == kLee) {
          const int H = q / 2;
          for (int d = R1 - 1; d >= 1; d--) {
            const int wm = d < H ? d : H;
            for (int a = 0; a < q; a++) {
              int32_t s = sm[d * SD + sp[a]];
              for (int w2 = 1; w2 <= wm; w2++) {
                int am = a - w2; if (am < 0) am += q;
                int ap = a + w2; if (ap >= q) ap -= q;
                s += sm[(d - w2) * SD + sp[am]];
                if (ap != am) s += sm[(d - w2) * SD + sp[ap]];
              }
              sm[d * SD + sp[a]] = s;   // reads only lower layers + itself
            }
          }
        } else {
          int32_t old[16];
          for (int a = 0; a < q; a++) old[a] = sm[sp[a]];
          for (int a = 0; a < q; a++) {
            int32_t s = 0;
            for (int b = 0; b < q; b++) {
              int dd = a > b ? a - b : b - a;
              if (g.prob == kTorus && q - dd < dd) dd = q - dd;
              if (dd <= g.R) s += old[b];
            }
            sm[sp[a]] = s;
          }
        }
      }
      S *= q;
      __syncthreads();
    }
    // -------- store the tile
    for (int t = threadIdx.x; t < nel; t += blockDim.x) {
      const int w = t % W, p = t / W, ob = p / g.mid, m = p % g.mid;
      const bool valid = (o0 + ob < g.outer) && (i0 + w < g.inner);
      if (!valid) continue;
      const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
      const int sp = skewed(p, g.skew) * W + w;
      if (g.dst == kDstLayers) {
        for (int d = 0; d < g.lout; d++)
          g.layers[d * g.plane + x] = sm[d * SD + sp];
      } else {
        int32_t s = 0;
        for (int d = 0; d < R1; d++) s += sm[d * SD + sp];
        if (g.dst == kDstMap) g.layers[x] = s;
        else g.cnt[x] = (uint16_t)(s > 65535 ? 65535 : s);
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ dispatch table
typedef void (*GroupFn)(const GroupArgs);
struct KernelEntry { int op, q, r1, bm; GroupFn fn; };

#define KE(OP, Q, R1, BM) {OP, Q, R1, BM, group_kernel<OP, Q, R1, BM>}
static const KernelEntry kTable[] = {
    // Hamming, binary: 16-word blocks up to 4 layers, 8-word above
    KE(kOpHamming, 2, 2, 4), KE(kOpHamming, 2, 3, 4), KE(kOpHamming, 2, 4, 4),
    KE(kOpHamming, 2, 5, 3), KE(kOpHamming, 2, 6, 3), KE(kOpHamming, 2, 7, 3),
    KE(kOpHamming, 2, 8, 3),
    // Hamming, ternary: 9-word blocks
    KE(kOpHamming, 3, 2, 2), KE(kOpHamming, 3, 3, 2), KE(kOpHamming, 3, 4, 2),
    KE(kOpHamming, 3, 5, 2), KE(kOpHamming, 3, 6, 2), KE(kOpHamming, 3, 7, 2),
    // Hamming, quaternary
    KE(kOpHamming, 4, 2, 2), KE(kOpHamming, 4, 3, 2), KE(kOpHamming, 4, 4, 2),
    KE(kOpHamming, 4, 5, 1),
    // Lee: one axis per round
    KE(kOpLee, 7, 3, 1), KE(kOpLee, 7, 4, 1), KE(kOpLee, 7, 5, 1),
    KE(kOpLee, 5, 2, 1), KE(kOpLee, 5, 3, 1), KE(kOpLee, 5, 4, 1),
    // small-axis window sums (torus / grid)
    KE(kOpTorus, 3, 1, 3), KE(kOpTorus, 4, 1, 2), KE(kOpTorus, 5, 1, 2),
};
#undef KE
static const int kTableLen = sizeof(kTable) / sizeof(kTable[0]);

static int op_of(int prob) {
  return prob == kHamming ? kOpHamming : prob == kLee ? kOpLee
         : prob == kTorus ? kOpTorus : kOpGrid;
}

// Kernel id for a group whose axes all have size q; -1 = generic kernel.
int pick_group_kernel(int prob, int q, int R1, int *bm) {
  const int op = op_of(prob);
  for (int i = 0; i < kTableLen; i++)
    if (kTable[i].op == op && kTable[i].q == q && kTable[i].r1 == R1) {
      *bm = kTable[i].bm;
      return i;
    }
  *bm = 1;
  return -1;
}

size_t group_smem_bytes(const GroupArgs &a, int R1) {
  const int tile_words = a.Bo * a.mid;
  const int skw = a.skew ? tile_words + (tile_words >> a.skew) : tile_words;
  return (size_t)(skw + 1) * a.W * R1 * sizeof(int32_t);
}

int launch_group(const GroupPlan &p, cudaStream_t s) {
  GroupFn fn = p.kernel >= 0 ? kTable[p.kernel].fn : group_generic;
  // opt in to the dynamic shared memory this launch needs (the per-block
  // limit counts the kernel's static shared memory too)
  static size_t attr_set[64 + 1];
  const int slot = p.kernel >= 0 ? p.kernel : 64;
  if (p.smem > 48 * 1024 && p.smem > attr_set[slot]) {
    CC_CK(cudaFuncSetAttribute((const void *)fn,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)p.smem));
    attr_set[slot] = p.smem;
  }
  fn<<<p.grid, p.threads, p.smem, s>>>(p.a);
  CC_CK(cudaGetLastError());
  return 0;
}

}  // namespace cc
