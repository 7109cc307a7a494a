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
#include <cstdlib>

#include "engine.h"

namespace cc {

template <int Q, int B>
struct IPow { static constexpr int v = Q * IPow<Q, B - 1>::v; };
template <int Q>
struct IPow<Q, 0> { static constexpr int v = 1; };

enum Op { kOpHamming = 0, kOpLee = 1, kOpTorus = 2, kOpGrid = 3 };

// ---------------------------------------------------------------- axis ops
// Hamming: newA_d[a] = A_d[a] + T_{d-1} - A_{d-1}[a], T = fibre sum.
// T_{d-1} - A_{d-1}[a] is the sum of the fibre's OTHER entries of layer
// d-1, which is how it is formed here: one add per entry for Q = 2, two for
// Q = 3, and T minus the entry above.  Descending d reads layer d-1 before
// it is rewritten, so every term is the old value, as in the recurrence.
template <int Q, int R1, int QB, int ST>
__device__ __forceinline__ void axis_hamming(int32_t (&v)[R1][QB]) {
#pragma unroll
  for (int e = 0; e < QB; e++) {
    if ((e / ST) % Q != 0) continue;
#pragma unroll
    for (int d = R1 - 1; d >= 1; d--) {
      if (Q == 2) {
        const int32_t a0 = v[d - 1][e], a1 = v[d - 1][e + ST];
        v[d][e] += a1;
        v[d][e + ST] += a0;
      } else if (Q == 3) {
        const int32_t a0 = v[d - 1][e], a1 = v[d - 1][e + ST],
                      a2 = v[d - 1][e + 2 * ST];
        v[d][e] += a1 + a2;
        v[d][e + ST] += a0 + a2;
        v[d][e + 2 * ST] += a0 + a1;
      } else {
        int32_t T = 0;
#pragma unroll
        for (int a = 0; a < Q; a++) T += v[d - 1][e + a * ST];
#pragma unroll
        for (int a = 0; a < Q; a++)
          v[d][e + a * ST] += T - v[d - 1][e + a * ST];
      }
    }
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
#pragma unroll
      for (int a = 0; a < Q; a++) {
        int32_t s = 0;
#pragma unroll
        for (int w = 1; w <= (d < H ? d : H); w++) {
          const int am = (a - w + Q) % Q, ap = (a + w) % Q;
          s += v[d - w][e + am * ST];
          if (ap != am) s += v[d - w][e + ap * ST];
        }
        v[d][e + a * ST] += s;       // only lower layers are read
      }
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

// Fill layer 0 of tile `tile` (shared memory) with the code multiplicities
// of its contiguous range [x0, x0 + len); other layers are implicit zeros.
// The tile's slice of the sorted code is code[bounds[tile], bounds[tile+1])
// (k_code_bounds, one binary search per tile boundary).
__device__ __forceinline__ void stage_code(const GroupArgs &g, int32_t *sm,
                                           long long tile, long long x0,
                                           int len) {
  for (int p = threadIdx.x; p < len; p += blockDim.x)
    sm[skewed(p, g.skew)] = 0;
  __syncthreads();
  const long long lo = g.code_bounds[tile], hi = g.code_bounds[tile + 1];
  for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x)
    atomicAdd(&sm[skewed((int)(g.code[t] - x0), g.skew)], 1);
  __syncthreads();
}

// The same for a first group whose words sit in pairs (inner == 2): word p
// of the range adds 1 to the half (p & 1) of packed lane p / 2.  Counts stay
// below 2^16 (the occurrence bound), so no add carries across halves.
__device__ __forceinline__ void stage_code_pairs(const GroupArgs &g,
                                                 int32_t *sm, long long tile,
                                                 long long x0, int len) {
  for (int P = threadIdx.x; P < (len + 1) / 2; P += blockDim.x)
    sm[skewed(P, g.skew)] = 0;
  __syncthreads();
  const long long lo = g.code_bounds[tile], hi = g.code_bounds[tile + 1];
  for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x) {
    const int p = (int)(g.code[t] - x0);
    atomicAdd(&sm[skewed(p >> 1, g.skew)], 1 << (16 * (p & 1)));
  }
  __syncthreads();
}

// bounds[t] = lower_bound(code, t * tile_words) for t = 0..ntiles
__global__ void k_code_bounds(const long long *code, long long ncode,
                              long long tile_words, long long ntiles,
                              long long *bounds) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  const long long x = t * tile_words;
  long long lo = 0, hi = ncode;
  while (lo < hi) {
    const long long md = (lo + hi) >> 1;
    if (code[md] < x) lo = md + 1; else hi = md;
  }
  bounds[t] = lo;
}

int launch_code_bounds(const long long *code, long long ncode,
                       long long tile_words, long long ntiles,
                       long long *bounds, cudaStream_t s) {
  k_code_bounds<<<(unsigned)((ntiles + 1 + 255) / 256), 256, 0, s>>>(
      code, ncode, tile_words, ntiles, bounds);
  CC_CK(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------ kernel
// Where a round's block comes from and goes to: the first round reads HBM
// (layers, the cnt predicate) or the staged code, the last writes HBM
// (layers, map, cnt); every other side is shared memory.
enum RoundIo { kIoSmem = 0, kIoLayers = 1, kIoCnt = 2, kIoCode = 3,
               kIoMap = 4, kIoCntOut = 5, kIoCntSmem = 6 };

// One round over the whole tile: every thread takes register blocks of
// ne = Q^rb words (all layers), rb of the group's axes at local stride S.
// FULL: rb == BM (no per-word bound checks).  Addresses step linearly with
// the block word e: in HBM by S*inner words, in shared memory by sstep —
// the skew (one pad word per 2^skew) keeps that linear, because a round's
// stride S is 1 or a multiple of 2^skew and S == 1 blocks start on a
// multiple of 2^skew.
//
// PACK: every register, shared-memory word and lane carries TWO inner words
// (w, w+1) as 16-bit halves of one 32-bit value, so each add and each
// shared-memory access serves both.  Exact while every value stays below
// 2^16 (the planner's 16-bit bound) and the inner stride is even, so a pair
// never straddles a row; the group's HBM sides are u16 planes (one 32-bit
// access per pair), the int32 map and the u16 cnt (unpacked at the store).
// Epilogue reductions of a launch's output (GroupArgs::red_mode): 2 the
// maximum of the map written (0 when no value is positive), 1 the deficit
// sum max(0, mu - c) of the cnt written.  Per thread, then per warp, one
// 64-bit atomic.
__device__ __forceinline__ void red_map(long long *acc, long long a,
                                        long long b) {
  const long long m = a > b ? a : b;
  if (m > *acc) *acc = m;
}
__device__ __forceinline__ void red_def(long long *acc, int mu, int c0,
                                        int c1) {
  *acc += (c0 < mu ? mu - c0 : 0) + (c1 < mu ? mu - c1 : 0);
}
__device__ __forceinline__ void red_flush(const GroupArgs &g, long long acc) {
  for (int o = 16; o > 0; o >>= 1) {
    const long long other = __shfl_down_sync(0xffffffffu, acc, o);
    acc = g.red_mode == 2 ? (other > acc ? other : acc) : acc + other;
  }
  if ((threadIdx.x & 31) == 0 && acc) {
    if (g.red_mode == 2)
      atomicMax((unsigned long long *)g.red, (unsigned long long)acc);
    else
      atomicAdd((unsigned long long *)g.red, (unsigned long long)acc);
  }
}

template <int OP, int Q, int R1, int BM, bool FULL, bool PACK = false>
__device__ __forceinline__ void run_round(const GroupArgs &g, int32_t *sm,
                                          int SD, long long o0, long long i0,
                                          int rb, int S, int src, int dst,
                                          int nl = R1,
                                          const uint16_t *cs = nullptr,
                                          long long *racc = nullptr) {
  constexpr int QB = IPow<Q, BM>::v;
  int ne = QB;
  if (!FULL) { ne = 1; for (int t = 0; t < rb; t++) ne *= Q; }
  const int W = PACK ? g.W >> 1 : g.W;         // lanes (pairs) per row
  const int nh = g.mid / (S * ne);
  const int nblk = W * S * nh * g.Bo;
  const long long imid = g.inner * (long long)g.mid;
  const long long gstep = (long long)S * g.inner;      // HBM word step of e
  const int sstep = g.skew == 0 ? S * W
                    : (S == 1 ? W : (S + (S >> g.skew)) * W);
  // predicate as a range: lo <= cnt <= hi
  const int plo = g.pmode == kPredDef ? 0 : g.pmode == kPredCrit ? 1
                  : g.ptarget;
  const int phi = g.pmode == kPredDef ? g.mu - 1 : g.pmode == kPredCrit
                  ? g.mu : g.ptarget;
  const unsigned pspan = (unsigned)(phi - plo);
  // blk = ((ob * nh + mhi) * S + mlo) * W + w, kept as mixed-radix digits
  // that advance by blockDim.x per trip (one compare per digit, no
  // division in the loop); every digit sum stays below twice its radix
  int w, mlo, mhi, ob, dw, dmlo, dmhi, dob;
  {
    int r = threadIdx.x;
    w = r % W; r /= W; mlo = r % S; r /= S; mhi = r % nh; ob = r / nh;
    r = blockDim.x;
    dw = r % W; r /= W; dmlo = r % S; r /= S; dmhi = r % nh; dob = r / nh;
  }
  for (int blk = threadIdx.x; blk < nblk; blk += blockDim.x) {
    const int wi = PACK ? 2 * w : w;                     // inner word
    const bool valid = (o0 + ob < g.outer) && (i0 + wi < g.inner);
    const int pb = ob * g.mid + mlo + S * ne * mhi;      // tile word, e = 0
    const int sp0 = skewed(pb, g.skew) * W + w;
    const long long xb = (o0 + ob) * imid + (long long)(mlo + S * ne * mhi)
                         * g.inner + i0 + wi;
    int32_t v[R1][QB];
#pragma unroll
    for (int d = 0; d < R1; d++)
#pragma unroll
      for (int e = 0; e < QB; e++) v[d][e] = 0;
    // -------- load
    if (src == kIoCntSmem) {                     // prefetched cnt window
      const uint16_t *p = cs + pb;
#pragma unroll
      for (int e = 0; e < QB; e++) {
        if (!FULL && e >= ne) break;
        v[0][e] = (unsigned)((int)p[e * S] - plo) <= pspan;
      }
    } else if (src == kIoSmem || src == kIoCode) {
      if (src == kIoCode) nl = 1;
#pragma unroll
      for (int d = 0; d < R1; d++) {
        if (d >= nl) break;
        const int32_t *p = sm + d * SD + sp0;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          v[d][e] = p[e * sstep];
        }
      }
    } else if (valid) {
      if (PACK && src == kIoLayers) {            // one u32 per word pair
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lin) break;
          const uint16_t *p = g.layers16 + d * g.plane + xb;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            v[d][e] = (int32_t)__ldcs(reinterpret_cast<const uint32_t *>(p));
            p += gstep;
          }
        }
      } else if (src == kIoLayers && g.in16) {
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lin) break;
          const uint16_t *p = g.layers16 + d * g.plane + xb;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            v[d][e] = __ldcs(p);
            p += gstep;
          }
        }
      } else if (src == kIoLayers) {
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lin) break;
          const int32_t *p = g.layers + d * g.plane + xb;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            v[d][e] = __ldcs(p);
            p += gstep;
          }
        }
      } else if (PACK) {                         // kIoCnt, a word pair
        const uint16_t *p = g.cnt + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          const uint32_t c = __ldcs(reinterpret_cast<const uint32_t *>(p));
          const uint32_t lo = (unsigned)((int)(c & 0xFFFFu) - plo) <= pspan;
          const uint32_t hi = (unsigned)((int)(c >> 16) - plo) <= pspan;
          v[0][e] = (int32_t)(lo | (hi << 16));
          p += gstep;
        }
      } else {                                   // kIoCnt
        const uint16_t *p = g.cnt + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          v[0][e] = (unsigned)((int)__ldcs(p) - plo) <= pspan;
          p += gstep;
        }
      }
    }
    // -------- axis 0 inside each pair (binary Hamming first group), once:
    // in the round that reads the code or cnt.  newA_d[a] = A_d[a] +
    // A_{d-1}[a ^ 1] is an add of the halves swapped, layers descending.
    if (PACK && OP == kOpHamming && Q == 2 && g.pair_axis &&
        (src == kIoCnt || src == kIoCode)) {
#pragma unroll
      for (int e = 0; e < QB; e++)
#pragma unroll
        for (int d = R1 - 1; d >= 1; d--)
          v[d][e] += (int32_t)__funnelshift_l((uint32_t)v[d - 1][e],
                                              (uint32_t)v[d - 1][e], 16);
    }
    // -------- rb axis recurrences in registers
    if (FULL) AxisLoop<OP, Q, R1, BM, 0>::run(v, BM, g.R);
    else AxisLoop<OP, Q, R1, BM, 0>::run(v, rb, g.R);
    // -------- store
    if (dst == kIoSmem) {
#pragma unroll
      for (int d = 0; d < R1; d++) {
        int32_t *p = sm + d * SD + sp0;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          p[e * sstep] = v[d][e];
        }
      }
    } else if (valid) {
      if (PACK && dst == kIoLayers) {            // one u32 per word pair
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lout) break;
          uint16_t *p = g.layers16 + d * g.plane + xb;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            __stcs(reinterpret_cast<uint32_t *>(p), (uint32_t)v[d][e]);
            p += gstep;
          }
        }
      } else if (PACK && dst == kIoMap) {        // both halves, widened
        int32_t *p = (g.map ? g.map : g.layers) + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          uint32_t s = 0;
#pragma unroll
          for (int d = 0; d < R1; d++) s += (uint32_t)v[d][e];
          __stcs(reinterpret_cast<int2 *>(p),
                 make_int2((int)(s & 0xFFFFu), (int)(s >> 16)));
          if (racc) red_map(racc, (long long)(s & 0xFFFFu), (long long)(s >> 16));
          p += gstep;
        }
      } else if (PACK) {                         // cnt: both halves at once
        uint16_t *p = g.cnt + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          uint32_t s = 0;
#pragma unroll
          for (int d = 0; d < R1; d++) s += (uint32_t)v[d][e];
          *reinterpret_cast<uint32_t *>(p) = s;
          if (racc) red_def(racc, g.mu, (int)(s & 0xFFFFu), (int)(s >> 16));
          p += gstep;
        }
      } else if (dst == kIoLayers && g.out16) {
        // a first group (inner 1) of a padded plan: the slab's row starts
        // at a pitch of g.pitch words
        const long long xo = g.pitch
            ? (o0 + ob) * g.pitch + (long long)(mlo + S * ne * mhi) *
                  g.inner + i0 + wi
            : xb;
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lout) break;
          uint16_t *p = g.layers16 + d * g.plane + xo;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            __stcs(p, (uint16_t)v[d][e]);
            p += gstep;
          }
        }
      } else if (dst == kIoLayers) {
#pragma unroll
        for (int d = 0; d < R1; d++) {
          if (d >= g.lout) break;
          int32_t *p = g.layers + d * g.plane + xb;
#pragma unroll
          for (int e = 0; e < QB; e++) {
            if (!FULL && e >= ne) break;
            __stcs(p, v[d][e]);
            p += gstep;
          }
        }
      } else if (dst == kIoMap) {
        int32_t *p = (g.map ? g.map : g.layers) + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          int32_t s = 0;
#pragma unroll
          for (int d = 0; d < R1; d++) s += v[d][e];
          __stcs(p, s);
          if (racc) red_map(racc, (long long)s, 0);
          p += gstep;
        }
      } else {
        uint16_t *p = g.cnt + xb;
#pragma unroll
        for (int e = 0; e < QB; e++) {
          if (!FULL && e >= ne) break;
          int32_t s = 0;
#pragma unroll
          for (int d = 0; d < R1; d++) s += v[d][e];
          *p = (uint16_t)(s > 65535 ? 65535 : s);
          if (racc) red_def(racc, g.mu, s > 65535 ? 65535 : s, g.mu);
          p += gstep;
        }
      }
    }
    // advance the digits by blockDim.x
    w += dw;
    int c = w >= W;
    if (c) w -= W;
    mlo += dmlo + c;
    c = mlo >= S;
    if (c) mlo -= S;
    mhi += dmhi + c;
    c = mhi >= nh;
    if (c) mhi -= nh;
    ob += dob + c;
  }
}

// A round of rb axes runs with a register block of exactly Q^rb words: the
// kernel's own block size BM for full rounds, a compile-time smaller block
// for the group's last, partial round (no runtime bounds in the loops).
template <int OP, int Q, int R1, int B, bool PACK = false>
struct RoundSel {
  static __device__ __forceinline__ void run(
      const GroupArgs &g, int32_t *sm, int SD, long long o0, long long i0,
      int rb, int S, int src, int dst, int nl, const uint16_t *cs,
      long long *racc = nullptr) {
    if (rb == B)
      run_round<OP, Q, R1, B, true, PACK>(g, sm, SD, o0, i0, B, S, src, dst,
                                          nl, cs, racc);
    else
      RoundSel<OP, Q, R1, B - 1, PACK>::run(g, sm, SD, o0, i0, rb, S, src,
                                            dst, nl, cs, racc);
  }
};
template <int OP, int Q, int R1, bool PACK>
struct RoundSel<OP, Q, R1, 0, PACK> {
  static __device__ __forceinline__ void run(
      const GroupArgs &, int32_t *, int, long long, long long, int, int, int,
      int, int, const uint16_t *, long long * = nullptr) {}
};

template <int OP, int Q, int R1, int BM>
__global__ void __launch_bounds__(kGroupThreads)
group_kernel(const GroupArgs g) {
  extern __shared__ int32_t sm[];
  const int W = g.W;
  const int tile_words = g.Bo * g.mid;
  const int SW = g.pack ? W >> 1 : W;                    // lanes per row
  const int SD = (skewed(tile_words, g.skew) + 1) * SW;  // layer stride
  const int first_src = g.src == kSrcLayers ? kIoLayers
                        : g.src == kSrcCnt ? kIoCnt : kIoCode;
  const int last_dst = g.dst == kDstLayers ? kIoLayers
                       : g.dst == kDstMap ? kIoMap : kIoCntOut;
  long long acc = 0;                    // epilogue reduction (red_mode)
  long long *racc = g.red_mode && g.dst != kDstLayers ? &acc : nullptr;
  for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
    const long long o0 = (tile / g.nchunk) * g.Bo;
    const long long i0 = (tile % g.nchunk) * W;
    if (g.src == kSrcCode && g.pack) {
      // first group, axis 0 in pairs: inner == 2, the tile is contiguous
      const long long imid = g.inner * (long long)g.mid;
      const long long len = (g.outer - o0) * imid;
      const long long tw = (long long)tile_words * g.inner;
      stage_code_pairs(g, sm, tile, o0 * imid, (int)(len < tw ? len : tw));
    } else if (g.src == kSrcCode) {
      // first group only: W == 1, inner == 1, the tile is contiguous
      long long len = (g.outer - o0) * (long long)g.mid;
      stage_code(g, sm, tile, o0 * g.mid,
                 (int)(len < tile_words ? len : tile_words));
    }
    for (int r = 0; r < g.nrounds; r++) {
      const int src = r == 0 ? first_src : kIoSmem;
      const int dst = r == g.nrounds - 1 ? last_dst : kIoSmem;
      if (g.pack)
        RoundSel<OP, Q, R1, BM, true>::run(g, sm, SD, o0, i0, g.rb[r],
                                           g.rs[r], src, dst, R1, nullptr,
                                           racc);
      else
        RoundSel<OP, Q, R1, BM>::run(g, sm, SD, o0, i0, g.rb[r], g.rs[r],
                                     src, dst, R1, nullptr, racc);
      __syncthreads();
    }
  }
  if (racc) red_flush(g, acc);
}

// --------------------------------------------------------- pipelined kernel
// The same rounds, with the next tile's input prefetched into a second
// shared-memory buffer by cp.async while the current tile computes, so the
// HBM reads of one tile overlap the register work and the HBM writes of the
// previous one.  Layer sources copy (lin layers) x tile words, 16 bytes at a
// time where the rows allow; a cnt source (the first group: a contiguous
// range) copies the 16-byte-aligned window of 2-byte counters around it.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s),
               "l"(src));
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s),
               "l"(src));
}
__device__ __forceinline__ void cp_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void cp_wait_prev() {
  asm volatile("cp.async.wait_group 1;\n" ::);
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::);
}

__device__ __forceinline__ void prefetch_layers(const GroupArgs &g,
                                                int32_t *buf, int SD,
                                                long long tile) {
  const long long o0 = (tile / g.nchunk) * g.Bo;
  const long long i0 = (tile % g.nchunk) * g.W;
  const long long imid = g.inner * (long long)g.mid;
  const int W = g.W, tw = g.Bo * g.mid;
  if (W % 4 == 0 && g.inner % 4 == 0) {        // 16-byte rows of 4 words
    const int W4 = W / 4, n = tw * W4;
    for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
      const int w = (idx % W4) * 4, p = idx / W4;
      const int ob = p / g.mid, m = p % g.mid;
      if (o0 + ob >= g.outer || i0 + w >= g.inner) continue;
      const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
      const int sp = skewed(p, g.skew) * W + w;
      for (int d = 0; d < g.lin; d++)
        cp_async16(buf + d * SD + sp, g.layers + d * g.plane + x);
    }
  } else {
    const int n = tw * W;
    for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
      const int w = idx % W, p = idx / W;
      const int ob = p / g.mid, m = p % g.mid;
      if (o0 + ob >= g.outer || i0 + w >= g.inner) continue;
      const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
      const int sp = skewed(p, g.skew) * W + w;
      for (int d = 0; d < g.lin; d++)
        cp_async4(buf + d * SD + sp, g.layers + d * g.plane + x);
    }
  }
}

// packed pairs from 16-bit planes: a 16-byte copy is 8 inner words, i.e.
// 4 packed lanes, and lands as is (two words per 32-bit shared word, low
// half first, the order run_round's packed lanes use).  The launcher admits
// this form only with W and the inner stride multiples of 8, so every
// source and destination is 16-byte aligned and no copy crosses a row end.
__device__ __forceinline__ void prefetch_pairs(const GroupArgs &g,
                                               int32_t *buf, int SD,
                                               long long tile) {
  const long long o0 = (tile / g.nchunk) * g.Bo;
  const long long i0 = (tile % g.nchunk) * g.W;
  const long long imid = g.inner * (long long)g.mid;
  const int W8 = g.W / 8, SW = g.W / 2, n = g.Bo * g.mid * W8;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int w = (idx % W8) * 8, p = idx / W8;
    const int ob = p / g.mid, m = p % g.mid;
    if (o0 + ob >= g.outer || i0 + w >= g.inner) continue;
    const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
    const int sp = skewed(p, g.skew) * SW + w / 2;
    for (int d = 0; d < g.lin; d++)
      cp_async16(buf + d * SD + sp, g.layers16 + d * g.plane + x);
  }
}

// first group (inner == 1): the tile is the contiguous range
// [x0, x0 + len); copy the aligned 8-counter window around it and return
// the offset of x0 inside the window
__device__ __forceinline__ int prefetch_cnt(const GroupArgs &g, uint16_t *cs,
                                            long long tile) {
  const long long x0 = (tile / g.nchunk) * g.Bo * (long long)g.mid;
  long long len = g.outer * (long long)g.mid - x0;
  if (len > (long long)g.Bo * g.mid) len = (long long)g.Bo * g.mid;
  const long long a0 = x0 & ~7LL, a1 = (x0 + len + 7) & ~7LL;
  const int nch = (int)((a1 - a0) >> 3);
  for (int c = threadIdx.x; c < nch; c += blockDim.x)
    cp_async16(cs + 8 * c, g.cnt + a0 + 8 * c);
  return (int)(x0 - a0);
}

template <int OP, int Q, int R1, int BM>
__global__ void __launch_bounds__(kGroupThreads)
group_kernel_pipe(const GroupArgs g) {
  extern __shared__ __align__(16) int32_t sm[];
  const int W = g.W;
  const int tile_words = g.Bo * g.mid;
  // packed pairs (16-bit layer source only): W / 2 lanes per row
  constexpr bool kPackable = (OP == kOpHamming && Q <= 3) || OP == kOpLee;
  const bool pk = kPackable && g.pack;
  const int SW = pk ? W >> 1 : W;
  const int SD = (skewed(tile_words, g.skew) + 1) * SW;  // layer stride
  const bool from_cnt = g.src == kSrcCnt;
  const int cbw = (tile_words + 16 + 7) & ~7;            // cnt window words
  // every buffer starts on a 16-byte boundary (cp.async 16-byte copies)
  const int lay_words = (R1 * SD + 3) & ~3;
  int32_t *const buf0 = sm;
  int32_t *const buf1 = from_cnt ? sm : sm + lay_words;
  uint16_t *const cb0 = reinterpret_cast<uint16_t *>(sm + lay_words);
  uint16_t *const cb1 = cb0 + cbw;
  const int last_dst = g.dst == kDstLayers ? kIoLayers
                       : g.dst == kDstMap ? kIoMap : kIoCntOut;
  long long acc = 0;                    // epilogue reduction (red_mode)
  long long *racc = g.red_mode && g.dst != kDstLayers ? &acc : nullptr;
  int off0 = 0, off1 = 0;
  long long tile = blockIdx.x;
  if (tile < g.ntiles) {
    if (from_cnt) off0 = prefetch_cnt(g, cb0, tile);
    else if (pk) prefetch_pairs(g, buf0, SD, tile);
    else prefetch_layers(g, buf0, SD, tile);
  }
  cp_commit();
  for (int i = 0; tile < g.ntiles; i++, tile += gridDim.x) {
    const bool odd = i & 1;
    const long long next = tile + gridDim.x;
    if (next < g.ntiles) {
      if (from_cnt) {
        const int o = prefetch_cnt(g, odd ? cb0 : cb1, next);
        if (odd) off0 = o; else off1 = o;
      } else if (pk) {
        prefetch_pairs(g, odd ? buf0 : buf1, SD, next);
      } else {
        prefetch_layers(g, odd ? buf0 : buf1, SD, next);
      }
    }
    cp_commit();
    cp_wait_prev();                 // this thread's copies of `tile` landed
    __syncthreads();                // ... and everyone else's
    const long long o0 = (tile / g.nchunk) * g.Bo;
    const long long i0 = (tile % g.nchunk) * W;
    int32_t *buf = odd ? buf1 : buf0;
    const uint16_t *cs = odd ? cb1 + off1 : cb0 + off0;
    for (int r = 0; r < g.nrounds; r++) {
      const int src = r > 0 ? kIoSmem : from_cnt ? kIoCntSmem : kIoSmem;
      const int dst = r == g.nrounds - 1 ? last_dst : kIoSmem;
      const int nl = r > 0 ? R1 : g.lin;
      if (pk)
        RoundSel<OP, Q, R1, BM, kPackable>::run(g, buf, SD, o0, i0, g.rb[r],
                                                g.rs[r], src, dst, nl, cs,
                                                racc);
      else
        RoundSel<OP, Q, R1, BM>::run(g, buf, SD, o0, i0, g.rb[r], g.rs[r],
                                     src, dst, nl, cs, racc);
      __syncthreads();
    }
  }
  cp_wait_all();
  if (racc) red_flush(g, acc);
}

// ------------------------------------------------------------ generic kernel
// Any axis size (<= 16) and layer count (<= 8), one axis per round, fibres
// processed in place in shared memory.  Used for the cells without a
// register-blocked instantiation (mixed radix, wide Hamming / Lee alphabets,
// small torus / grid axes) and, one tile per work item, by the batched
// engine (CG: global reads through L2 only, because other SMs of the same
// launch wrote them).  Optional epilogue reductions of the output (red_mode
// 1: deficit sum max(0, mu - cnt) of a written cnt; 2: maximum of a written
// map) add into *red.
template <bool CG>
__device__ __forceinline__ int32_t ld_i32(const int32_t *p) {
  return CG ? __ldcg(p) : *p;
}
template <bool CG>
__device__ __forceinline__ int ld_u16(const uint16_t *p) {
  return CG ? (int)__ldcg(p) : (int)*p;
}

template <bool CG>
__device__ void generic_tile(const GroupArgs &g, long long tile,
                             int32_t *sm) {
  const int R1 = g.prob == kTorus || g.prob == kGrid ? 1 : g.R + 1;
  const long long imid = g.inner * (long long)g.mid;
  const int W = g.W;
  const int tile_words = g.Bo * g.mid;
  const int SD = (skewed(tile_words, g.skew) + 1) * W;
  const int nel = tile_words * W;
  int32_t *map = g.map ? g.map : g.layers;
  const long long o0 = (tile / g.nchunk) * g.Bo;
  const long long i0 = (tile % g.nchunk) * W;
  if (g.src == kSrcCode) {
    long long len = (g.outer - o0) * (long long)g.mid;
    stage_code(g, sm, tile, o0 * g.mid,
               (int)(len < tile_words ? len : tile_words));
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
        if (valid && d < g.lin)
          val = g.in16 ? ld_u16<CG>(g.layers16 + d * g.plane + x)
                       : ld_i32<CG>(g.layers + d * g.plane + x);
      } else if (g.src == kSrcCnt) {
        if (valid && d == 0)
          val = cnt_pred(g.pmode, ld_u16<CG>(g.cnt + x), g.ptarget, g.mu);
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
  // -------- store the tile (+ epilogue reduction)
  long long red = 0;
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int w = t % W, p = t / W, ob = p / g.mid, m = p % g.mid;
    const bool valid = (o0 + ob < g.outer) && (i0 + w < g.inner);
    if (!valid) continue;
    const long long x = (o0 + ob) * imid + (long long)m * g.inner + i0 + w;
    const int sp = skewed(p, g.skew) * W + w;
    if (g.dst == kDstLayers) {
      for (int d = 0; d < g.lout; d++) {
        if (g.out16) g.layers16[d * g.plane + x] = (uint16_t)sm[d * SD + sp];
        else g.layers[d * g.plane + x] = sm[d * SD + sp];
      }
    } else {
      int32_t s = 0;
      for (int d = 0; d < R1; d++) s += sm[d * SD + sp];
      if (g.dst == kDstMap) {
        map[x] = s;
        if (g.red_mode == 2 && s > red) red = s;
      } else {
        const int c = s > 65535 ? 65535 : s;
        g.cnt[x] = (uint16_t)c;
        if (g.red_mode == 1 && c < g.mu) red += g.mu - c;
      }
    }
  }
  if (g.red_mode) {
    for (int o = 16; o > 0; o >>= 1) {
      const long long other = __shfl_down_sync(0xffffffffu, red, o);
      red = g.red_mode == 2 ? (other > red ? other : red) : red + other;
    }
    if ((threadIdx.x & 31) == 0 && red) {
      if (g.red_mode == 2) atomicMax((unsigned long long *)g.red,
                                     (unsigned long long)red);
      else atomicAdd((unsigned long long *)g.red, (unsigned long long)red);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(512) group_generic(const GroupArgs g) {
  extern __shared__ int32_t sm[];
  for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x)
    generic_tile<false>(g, tile, sm);
}

// ------------------------------------------------------------ batched engine
// One persistent launch over many independent cells.  Work items (pass,
// tile) are claimed in table order from one atomic counter; the table is
// ordered by pass level (every cell's pass 0, then every cell's pass 1, ...)
// and a pass depends only on the previous pass of its own cell, so an item
// only ever waits for items claimed before it — by CTAs already running —
// and the schedule cannot deadlock.  The wait is bounded: after
// kBatchSpinLimit polls the CTA records an error and stops, and the host
// reports it.  Data written by other CTAs of the launch is read through L2
// (generic_tile<true>).
constexpr long long kBatchSpinLimit = 1LL << 22;

__global__ void __launch_bounds__(256)
batch_kernel(const GroupArgs *passes, const int *pass_dep,
             const unsigned *pass_need, const int4 *items, long long nitems,
             unsigned *done, unsigned long long *next, int *err) {
  extern __shared__ int32_t sm[];
  __shared__ long long s_it;
  __shared__ int s_bad;
  __shared__ GroupArgs sg;
  for (;;) {
    if (threadIdx.x == 0) {
      s_it = (long long)atomicAdd(next, 1ULL);
      s_bad = 0;
    }
    __syncthreads();
    const long long it = s_it;
    if (it >= nitems) break;
    const int4 item = items[it];           // pass, first tile, tiles
    const int *src = reinterpret_cast<const int *>(passes + item.x);
    int *dst = reinterpret_cast<int *>(&sg);
    for (int i = threadIdx.x; i < (int)(sizeof(GroupArgs) / 4);
         i += blockDim.x)
      dst[i] = src[i];
    if (threadIdx.x == 0) {
      const int dep = pass_dep[item.x];
      if (dep >= 0) {
        const unsigned need = pass_need[dep];
        long long spins = 0;
        while (*(volatile unsigned *)(done + dep) < need) {
          if (++spins > kBatchSpinLimit) {
            atomicExch(err, 1);
            s_bad = 1;
            break;
          }
          __nanosleep(256);
        }
        __threadfence();
      }
    }
    __syncthreads();
    if (s_bad) break;
    for (int t = 0; t < item.z; t++)
      generic_tile<true>(sg, (long long)item.y + t, sm);
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + item.x, (unsigned)item.z);
    }
    __syncthreads();
  }
}

int launch_batch(const BatchLaunch &b, cudaStream_t s) {
  batch_kernel<<<b.grid, 256, b.smem, s>>>(b.passes, b.dep, b.need, b.items,
                                           b.nitems, b.done, b.next, b.err);
  CC_CK(cudaGetLastError());
  return 0;
}

// opts the kernel in to `smem` bytes of dynamic shared memory (outside any
// stream capture) and returns the persistent grid: every CTA that fits
int batch_grid(size_t smem) {
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    if (cudaFuncSetAttribute((const void *)batch_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) == cudaSuccess)
      attr = smem;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, 256,
                                                smem);
  if (per_sm < 1) per_sm = 1;
  return per_sm * sm_count();
}

// ------------------------------------------------------------ dispatch table
typedef void (*GroupFn)(const GroupArgs);
struct KernelEntry { int op, q, r1, bm; GroupFn fn, fn_pipe; };

#define KE(OP, Q, R1, BM)                                                   \
  {OP, Q, R1, BM, group_kernel<OP, Q, R1, BM>,                              \
   group_kernel_pipe<OP, Q, R1, BM>}
static const KernelEntry kTable[] = {
    // Hamming, binary: 16-word blocks up to 4 layers, 8-word above
    KE(kOpHamming, 2, 2, 4), KE(kOpHamming, 2, 3, 4), KE(kOpHamming, 2, 4, 4),
    KE(kOpHamming, 2, 4, 3),   // 8-word blocks: fewer registers per thread
    KE(kOpHamming, 2, 5, 3), KE(kOpHamming, 2, 6, 3), KE(kOpHamming, 2, 7, 3),
    KE(kOpHamming, 2, 8, 3),
    // Hamming, ternary: 9-word blocks; 3-word blocks for wider CTAs
    KE(kOpHamming, 3, 2, 2), KE(kOpHamming, 3, 3, 2), KE(kOpHamming, 3, 4, 2),
    KE(kOpHamming, 3, 5, 2), KE(kOpHamming, 3, 6, 2), KE(kOpHamming, 3, 7, 2),
    KE(kOpHamming, 3, 4, 1), KE(kOpHamming, 3, 5, 1),
    // Hamming, quaternary
    KE(kOpHamming, 4, 2, 2), KE(kOpHamming, 4, 3, 2), KE(kOpHamming, 4, 4, 2),
    KE(kOpHamming, 4, 5, 1),
    // Hamming, q = 5, 6: one axis per round (up to 5 layers)
    KE(kOpHamming, 5, 2, 1), KE(kOpHamming, 5, 3, 1), KE(kOpHamming, 5, 4, 1),
    KE(kOpHamming, 5, 5, 1),
    KE(kOpHamming, 6, 2, 1), KE(kOpHamming, 6, 3, 1), KE(kOpHamming, 6, 4, 1),
    KE(kOpHamming, 6, 5, 1),
    // Lee: one axis per round
    KE(kOpLee, 7, 3, 1), KE(kOpLee, 7, 4, 1), KE(kOpLee, 7, 5, 1),
    KE(kOpLee, 5, 2, 1), KE(kOpLee, 5, 3, 1), KE(kOpLee, 5, 4, 1),
    KE(kOpLee, 5, 5, 1),
    KE(kOpLee, 2, 2, 1), KE(kOpLee, 2, 3, 1), KE(kOpLee, 2, 4, 1),
    KE(kOpLee, 2, 5, 1),
    KE(kOpLee, 3, 2, 1), KE(kOpLee, 3, 3, 1), KE(kOpLee, 3, 4, 1),
    KE(kOpLee, 3, 5, 1),
    KE(kOpLee, 4, 2, 1), KE(kOpLee, 4, 3, 1), KE(kOpLee, 4, 4, 1),
    KE(kOpLee, 4, 5, 1),
    KE(kOpLee, 6, 2, 1), KE(kOpLee, 6, 3, 1), KE(kOpLee, 6, 4, 1),
    KE(kOpLee, 6, 5, 1),
    // small-axis window sums (torus / grid)
    KE(kOpTorus, 3, 1, 3), KE(kOpTorus, 4, 1, 2), KE(kOpTorus, 5, 1, 2),
};
#undef KE
static const int kTableLen = sizeof(kTable) / sizeof(kTable[0]);
static_assert(sizeof(kTable) / sizeof(kTable[0]) <= 64,
              "the shared-memory opt-in cache holds 64 kernels per form");

static int op_of(int prob) {
  return prob == kHamming ? kOpHamming : prob == kLee ? kOpLee
         : prob == kTorus ? kOpTorus : kOpGrid;
}

// Every register-blocked kernel for (problem, q, R1): ids and block axes,
// in table order; returns how many (at most cap).
int group_kernel_variants(int prob, int q, int R1, int *kids, int *bms,
                          int cap) {
  const int op = op_of(prob);
  int n = 0;
  for (int i = 0; i < kTableLen && n < cap; i++)
    if (kTable[i].op == op && kTable[i].q == q && kTable[i].r1 == R1) {
      kids[n] = i;
      bms[n] = kTable[i].bm;
      n++;
    }
  return n;
}

// Kernel id for a group whose axes all have size q; -1 = generic kernel.
int pick_group_kernel(int prob, int q, int R1, int *bm) {
  const int op = op_of(prob);
  // CC_BLOCK_AXES caps the axes of one register block (tuning)
  const char *cap_env = getenv("CC_BLOCK_AXES");
  const int cap = cap_env ? atoi(cap_env) : 99;
  for (int i = 0; i < kTableLen; i++)
    if (kTable[i].op == op && kTable[i].q == q && kTable[i].r1 == R1 &&
        kTable[i].bm <= cap) {
      *bm = kTable[i].bm;
      return i;
    }
  *bm = 1;
  return -1;
}

size_t group_smem_bytes(const GroupArgs &a, int R1) {
  const int tile_words = a.Bo * a.mid;
  const int skw = a.skew ? tile_words + (tile_words >> a.skew) : tile_words;
  const size_t lay = (size_t)(skw + 1) * (a.pack ? a.W / 2 : a.W) * R1;
  const size_t tile = ((lay + 3) & ~(size_t)3) * sizeof(int32_t);
  if (!a.pipe) return tile;
  if (a.src == kSrcCnt)                     // one tile + two cnt windows
    return tile + 2 * (size_t)((tile_words + 16 + 7) & ~7) * 2;
  return 2 * tile;                          // two tiles
}

static GroupFn group_fn(const GroupPlan &p) {
  return p.kernel < 0 ? group_generic
         : p.a.pipe ? kTable[p.kernel].fn_pipe : kTable[p.kernel].fn;
}

// Opt the plan's kernel in to the dynamic shared memory it needs (the
// per-block limit counts the kernel's static shared memory too).  The
// opt-in only ever grows, so one launch never lowers another's.
int ensure_group_smem(const GroupPlan &p) {
  if (p.a.tma) return tma_prepare(p);
  static size_t attr_set[2 * 64 + 1];
  const int slot = p.kernel < 0 ? 128 : p.kernel + (p.a.pipe ? 64 : 0);
  if (p.smem > 48 * 1024 && p.smem > attr_set[slot]) {
    CC_CK(cudaFuncSetAttribute((const void *)group_fn(p),
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)p.smem));
    attr_set[slot] = p.smem;
  }
  return 0;
}

// ahead of a stream capture, so that the capture only records launches
int prepare_group(const GroupPlan &p) { return ensure_group_smem(p); }

// CTAs of plan p's kernel that are resident on one SM at once (its
// registers, shared memory and threads all counted), or 0 when the runtime
// cannot say
int group_blocks_per_sm(const GroupPlan &p) {
  static int have_device = -1;                // plans are also built on hosts
  if (have_device < 0) {                      // without a GPU (plan probes)
    int n = 0;
    have_device = cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    cudaGetLastError();
  }
  if (!have_device) return 0;
  if (p.a.tma) return tma_blocks_per_sm(p);
  // a tile above the per-block limit has no occupancy (a plan built only
  // for its grouping); a refused opt-in leaves no error for later checks
  if (p.smem > 227 * 1024) return 0;
  if (ensure_group_smem(p)) {
    cudaGetLastError();
    return 0;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, (const void *)group_fn(p), p.threads, p.smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// The packed form of the prefetching kernel: 16-byte copies of 16-bit
// layers into packed lanes need W and the inner stride multiples of 8 words,
// 16-byte aligned planes, and a layer source (not the pair first group).
bool pipe_pairs_ok(const GroupArgs &a) {
  return a.pack && a.in16 && !a.pair_axis && a.src == kSrcLayers &&
         a.W % 8 == 0 && a.inner % 8 == 0 && a.plane % 8 == 0 &&
         (reinterpret_cast<uintptr_t>(a.layers16) & 15) == 0;
}

int launch_group(const GroupPlan &p, cudaStream_t s) {
  if (p.a.tma) return launch_tma_group(p, s);
  // packed pairs need 4-byte aligned pair accesses: an even inner stride
  // and row width, 16-bit planes in, a register kernel with a packed form
  // (Hamming q <= 3, Lee), and prefetching only in its 16-byte form
  const bool packs = p.kernel >= 0 &&
                     ((kTable[p.kernel].op == kOpHamming &&
                       kTable[p.kernel].q <= 3) ||
                      kTable[p.kernel].op == kOpLee);
  if (p.a.pack && (p.a.inner % 2 || p.a.W % 2 ||
                   !(p.a.in16 || p.a.pair_axis) || !packs ||
                   (p.a.pipe && !pipe_pairs_ok(p.a)))) {
    fprintf(stderr, "coldcore_b200: refused a packed group with inner %lld "
            "W %d pipe %d\n", p.a.inner, p.a.W, p.a.pipe);
    return -9;
  }
  // the unpacked prefetch copies 32-bit layers: no 16-bit source
  if (!p.a.pack && p.a.pipe && p.a.in16) {
    fprintf(stderr, "coldcore_b200: refused a prefetching group over "
            "16-bit planes\n");
    return -9;
  }
  GroupFn fn = group_fn(p);
  const int rc = ensure_group_smem(p);
  if (rc) return rc;
  fn<<<grid_knob(p.grid, p.a.ntiles), p.threads, p.smem, s>>>(p.a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    fprintf(stderr, "coldcore_b200: group launch (kernel %d pipe %d grid %d "
            "threads %d smem %zu tiles %lld) failed\n", p.kernel, p.a.pipe,
            p.grid, p.threads, p.smem, p.a.ntiles);
  CC_CK(e);
  return 0;
}

}  // namespace cc
