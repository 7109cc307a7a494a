// planner.cu — transform schedules: which axes each launch covers, its
// tile, rounds, CTA size and grid (used by the singleton cell and by the
// large cells of a batch).
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>

#include "engine.h"

namespace cc {
namespace {

int ipow(int q, int e) { int r = 1; while (e-- > 0) r *= q; return r; }

void set_rounds(GroupArgs &a, int q, int bm) {
  const int nr = (a.k + bm - 1) / bm;
  std::vector<int> rb(nr), rs(nr);
  for (int r = 0; r < nr; r++) {
    rb[r] = std::min(bm, a.k - r * bm);
    rs[r] = ipow(q, r * bm);
  }
  std::vector<int> order(nr);
  for (int r = 0; r < nr; r++) order[r] = r;
  if ((a.W == 1 || a.pair_axis) && nr >= 3) {
    // HBM-facing rounds get the widest strides (coalesced lanes): the
    // widest round stores every layer, the second widest loads the
    // 2-byte cnt, the rest exchange through shared memory in between
    order.clear();
    order.push_back(nr - 2);
    for (int r = 0; r < nr - 2; r++) order.push_back(r);
    order.push_back(nr - 1);
  }
  a.nrounds = nr;
  for (int i = 0; i < nr; i++) {
    a.rb[i] = rb[order[i]];
    a.rs[i] = rs[order[i]];
    a.rq[i] = q;
  }
}

int threads_for(const GroupArgs &a, int kid, int bm, int q) {
  int t;
  if (kid >= 0) {
    // register blocks per round: packed lanes carry two words each
    const long long words = (long long)(a.pack ? a.W / 2 : a.W) * a.mid *
                            a.Bo;
    const int ne = ipow(q, std::min(bm, a.k));
    t = (int)std::min<long long>(kGroupThreads, words / ne);
  } else {
    t = (int)std::min<long long>(256, (long long)a.W * a.mid * a.Bo);
  }
  t = (t + 31) / 32 * 32;
  const char *cap = getenv("CC_THREADS");          // tuning cap
  if (cap && atoi(cap) >= 32 && t > atoi(cap)) t = atoi(cap) / 32 * 32;
  return t < 32 ? 32 : t;
}

int occupancy_grid(const GroupPlan &p) {
  // persistent: as many CTAs as are resident at once (registers included:
  // a grid above that runs its last CTAs as a second, unbalanced wave),
  // capped by the tile count
  int per_sm = group_blocks_per_sm(p);
  if (per_sm < 1) {                   // estimate from shared memory, threads
    const size_t budget_sm = 228 * 1024;
    per_sm = (int)std::max<size_t>(1, budget_sm / (p.smem + 1024));
    const int by_threads = 2048 / p.threads;
    if (per_sm > by_threads) per_sm = by_threads;
    if (per_sm > 32) per_sm = 32;     // resident CTAs per SM, at most
    if (per_sm < 1) per_sm = 1;
  }
  long long grid = (long long)sm_count() * per_sm;
  if (grid > p.a.ntiles) grid = p.a.ntiles;
  return (int)std::max<long long>(1, grid);
}

// streamed launches sized once, at planning, not at every launch
void size_streamed(std::vector<GroupPlan> &groups) {
  for (auto &gp : groups)
    if (gp.a.tma && gp.grid < 1) gp.grid = occupancy_grid(gp);
}

// Distance layers that can be nonzero after axes 0..j-1: each Hamming axis
// adds at most 1 to the distance, each Lee axis at most floor(a/2).
int live_layers(const Geometry &g, const AxisRange &r, int j) {
  long long reach = r.reach0;
  for (int i = r.begin; i < j; i++) reach += axis_reach(g.prob, g.ax[i]);
  return (int)std::min<long long>(reach, g.R) + 1;
}

}  // namespace

// Groups of consecutive axes for one transform of cell `g`: the most axes
// per launch whose tile fits kn.budget bytes of shared memory, the
// register-blocked kernel where one exists for the axis size and layer
// count, 128- or 64-byte rows on strided groups, rounds ordered so the
// HBM-facing ones have the widest strides.
std::vector<GroupPlan> plan_groups(const Geometry &g, int R1,
                                   const PlanPtrs &ptr, int src, int dst,
                                   Knobs kn, AxisRange range) {
  std::vector<GroupPlan> out;
  const bool layered = R1 > 1;
  const size_t budget = kn.budget;
  const int end = range.end < 0 ? g.n : range.end;
  if (range.begin < 0 || range.begin >= end || end > g.n) return {};
  int j = range.begin;
  while (j < end) {
    const int q = g.ax[j];
    int bm = 1;
    const int kid = pick_group_kernel(g.prob, q, R1, &bm);
    GroupArgs base{};
    base.layers = ptr.layers;
    base.plane = ptr.plane;
    base.cnt = ptr.cnt;
    base.code = ptr.code;
    base.ncode = ptr.ncode;
    base.map = ptr.map;
    base.layers16 = ptr.layers16;
    base.in16 = kn.half && j > 0;          // every later group reads u16
    // the first group of a binary Hamming cell with 16-bit values: axis 0
    // is the word pair itself (inner = 2, applied as a swap-add inside each
    // lane) and the group's rounds run over axes 1.. on packed pairs
    const bool pair = j == 0 && kn.half && kn.pair && kid >= 0 &&
                      g.prob == kHamming && q == 2 && end >= 2 &&
                      g.ax[1] == 2 && src != kSrcLayers;
    const int j0 = j + (pair ? 1 : 0);     // first axis of the rounds
    base.pair_axis = pair ? 1 : 0;
    base.inner = pair ? 2 : g.pw[j];
    // two inner words per lane: 16-bit values, an even inner stride (so a
    // pair never straddles a row and every pair access is 4-byte aligned),
    // and recurrences made of adds only (Hamming with q <= 3, Lee), whose
    // every partial sum is a layer value
    base.pack = pair || (base.in16 && kid >= 0 && base.inner % 2 == 0 &&
                         ((g.prob == kHamming && q <= 3) || g.prob == kLee));
    base.prob = g.prob;
    base.R = g.R;
    base.mu = g.mu;
    base.src = j == range.begin ? src : kSrcLayers;
    // pipe 1 and 3 prefetch the cnt-reading first group; 3 also the last
    // group when it writes the 4-byte map (reads every layer, writes one
    // plane), decided below; 2 prefetches every group (16-bit layers only
    // in packed pairs, whose 16-byte form is checked once W is known)
    base.pipe = kid >= 0 && base.src != kSrcCode && !pair &&
                (!base.in16 || base.pack) &&
                (kn.pipe == 2 || ((kn.pipe == 1 || kn.pipe == 3) &&
                                  base.src == kSrcCnt));
    // the most axes that fit one tile of W inner words
    auto grow = [&](int W) {
      GroupArgs a = base;
      a.W = W;
      long long mid = 1;
      for (;;) {
        if (j0 + a.k >= end || a.k >= kMaxRounds) break;
        const int qn = g.ax[j0 + a.k];
        if (kid >= 0 && qn != q) break;
        if (kid < 0 && qn > 16) break;
        const long long mid2 = mid * qn;
        GroupArgs t = a;
        t.k = a.k + 1;
        t.mid = (int)std::min<long long>(mid2, INT_MAX / 64);
        const long long outer = g.space / (a.inner * mid2);
        t.Bo = W >= 16 ? 1
               : (int)std::max<long long>(1, std::min<long long>(
                     outer, 2048 / (W * mid2)));
        t.skew = 0;
        if (kid >= 0 && (W == 1 || (pair && W == 2)) &&
            (q & (q - 1)) == 0) {
          int lg = 0;
          while ((1 << lg) < ipow(q, bm)) lg++;
          t.skew = lg;
        }
        const bool fits = group_smem_bytes(t, R1) <= budget &&
                          mid2 < (1 << 24);
        if (a.k > 0 && !fits) break;
        a = t;
        mid = mid2;
      }
      return a;
    };
    GroupArgs a;
    if (base.inner >= 32) {
      // 128-byte rows, or 64-byte rows when that fits more axes
      a = grow(32);
      GroupArgs b16 = grow(16);
      if (b16.k > a.k) a = b16;
    } else {
      a = grow((int)base.inner);
    }
    if (a.k < 1 || a.mid < 1) return {};     // no axis fits: no plan
    if (a.pipe && a.in16 && !pipe_pairs_ok(a)) a.pipe = 0;
    a.outer = g.space / (a.inner * (long long)a.mid);
    a.nchunk = (a.inner + a.W - 1) / a.W;
    a.ntiles = (a.outer + a.Bo - 1) / a.Bo * a.nchunk;
    for (int t = 0; t < a.k; t++) a.qax[t] = g.ax[j0 + t];
    if (kid >= 0) set_rounds(a, q, bm);
    else a.nrounds = 0;
    const bool last = j0 + a.k == end;
    a.dst = last ? dst : kDstLayers;
    a.out16 = kn.half && !(last && range.final);
    if (kn.pipe == 3 && kid >= 0 && last && dst != kDstLayers &&
        a.src == kSrcLayers && !a.in16) {
      // read-heavy last group: prefetch its tiles too (if they still fit)
      GroupArgs t = a;
      t.pipe = 1;
      if (group_smem_bytes(t, R1) <= budget) a.pipe = 1;
    }
    a.lin = layered ? live_layers(g, range, j) : 1;
    a.lout = layered ? live_layers(g, range, j0 + a.k) : 1;
    if (last && range.final && dst == kDstLayers)
      a.lout = R1;                                // every layer, zeros too
    a.pmode = kPredEq;
    a.ptarget = 0;
    GroupPlan p;
    p.a = a;
    p.kernel = kid;
    p.smem = group_smem_bytes(a, R1);
    p.threads = threads_for(a, kid, bm, q);
    p.grid = occupancy_grid(p);
    out.push_back(p);
    j = j0 + a.k;
  }
  return out;
}

std::vector<GroupPlan> group_variants(const GroupPlan &p, int R1,
                                      size_t smem_cap) {
  std::vector<GroupPlan> out{p};
  if (p.kernel < 0 || p.a.nrounds <= 0) return out;
  const int q = p.a.rq[0];
  int kids[8], bms[8];
  const int nk = group_kernel_variants(p.a.prob, q, R1, kids, bms, 8);
  // the cp.async-prefetching form too, where its second buffer fits (over
  // 16-bit layers only in its packed 16-byte form)
  const bool can_pipe = p.a.src != kSrcCode &&
                        ((!p.a.in16 && !p.a.pack) || pipe_pairs_ok(p.a));
  // strided groups of 32-word rows also as 16-word rows: half the tile, so
  // twice the CTAs (and warps) per SM over the same axes
  std::vector<int> rows{p.a.W};
  if (p.a.W == 32 && p.a.Bo == 1 && p.a.inner >= 32 && !p.a.pair_axis)
    rows.push_back(16);
  // the streamed form (tensor loads into shared-memory stages) where the
  // group qualifies: 32 or 64-word rows, 2 or 3 stages, 256 or 512 threads
  const char *tma_env = getenv("CC_TMA");
  const bool tma_off = tma_env && atoi(tma_env) == 0;
  // a ternary first group over packed row pairs (its tiles are the pairs
  // the group already has, so a recount's code bounds stay valid)
  for (int th : {256, 512}) {
    if (tma_off || (p.a.tma == 3 && p.threads == th)) continue;
    GroupPlan v = tern_first_variant(p, th);
    if (!tern_first_ok(v.a, R1)) continue;
    v.grid = occupancy_grid(v);
    out.push_back(v);
  }
  // (three-axis rounds, tbm 3, timed 0.21 against 0.175 ms on the eight-
  // axis group of H2(26,3): they are not offered; CC_TMA_BM=3 forces them)
  for (int lanes : {16, 32})
    for (int stages : {1, 2, 3, 4})
      for (int tbm : {0}) {
        if (tma_off || (stages == 4 && !p.a.in8)) continue;
        GroupPlan t = p;
        t.a.tbm = tbm;
        if (!tma_group_ok(tma_variant(t, lanes, stages, 256).a, q, R1, lanes,
                          stages))
          continue;
        // three-axis rounds have twice the blocks: 512 threads only
        for (int th : {256, 512}) {
          if (tbm == 3 && th != 512) continue;
          GroupPlan v = tma_variant(t, lanes, stages, th);
          v.grid = occupancy_grid(v);
          out.push_back(v);
        }
      }
  // a padded plan's later groups run streamed only (the register kernels
  // address the canonical layout)
  if (p.a.pitch && p.a.tma == 1) return out;
  for (int stages : {0, 2, 3})
    if (!tma_off && tma_first_ok(p.a, R1, stages))
      for (int th : {128, 256, 512}) {
        GroupPlan v = tma_first_variant(p, stages, th);
        v.grid = occupancy_grid(v);
        out.push_back(v);
      }
  // 8-bit planes: only the streamed forms read or write them
  if (p.a.in8 || p.a.out8) return out;
  for (int W : rows)
  for (int i = 0; i < nk; i++)
  for (int pipe = 0; pipe <= (can_pipe ? 1 : 0); pipe++) {
    GroupPlan t = p;
    t.kernel = kids[i];
    t.a.tma = 0;
    t.a.stages = 0;
    t.a.pipe = pipe;
    if (W != p.a.W) {
      t.a.W = W;
      t.a.nchunk = (t.a.inner + W - 1) / W;
      t.a.ntiles = t.a.outer * t.a.nchunk;        // Bo == 1
    }
    if ((t.a.W == 1 || t.a.pair_axis) && (q & (q - 1)) == 0) {
      int lg = 0;
      while ((1 << lg) < ipow(q, bms[i])) lg++;
      t.a.skew = lg;
    }
    set_rounds(t.a, q, bms[i]);
    t.smem = group_smem_bytes(t.a, R1);
    if (t.smem > smem_cap) continue;
    const int full = threads_for(t.a, t.kernel, bms[i], q);
    std::vector<int> widths{full};
    if (full > 256) widths.push_back(256);
    if (full > 128) widths.push_back(128);
    for (int th : widths) {
      GroupPlan v = t;
      v.threads = th;
      v.grid = occupancy_grid(v);
      if (v.kernel == p.kernel && v.threads == p.threads &&
          v.a.pipe == p.a.pipe && v.a.W == p.a.W && v.a.tma == p.a.tma)
        continue;
      out.push_back(v);
    }
  }
  return out;
}

// The padded plan of a cell whose first group has an odd word count T0
// (ternary): the first group writes its 16-bit layers at a pitch of P0 =
// round_up(T0, 64) words a row, so every later group's rows start on 128-
// byte boundaries and run as streamed launches over packed pairs; the last
// writes the map or cnt back at the canonical index.  The axes after the
// first group are split evenly into groups of at most kPadMaxAxes (the
// widest streamed ternary group), and the first group takes the packed
// row-pair form where it applies.  false when the cell does not qualify or
// the padded planes do not fit the room16 u16 words of the allocation.
constexpr int kPadMaxAxes = 5;

bool pad_plan(std::vector<GroupPlan> &groups, const Geometry &g,
              const PlanPtrs &ptr, int dst, int R1, long long room16) {
  if (groups.size() < 2 || g.prob != kHamming) return false;
  GroupPlan &f = groups[0];
  const GroupArgs &a0 = f.a;
  if (f.kernel < 0 || a0.inner != 1 || a0.W != 1 || !a0.out16 || a0.pack ||
      a0.pair_axis || (a0.mid & 1) == 0)
    return false;
  const int k0 = a0.k;
  const int rem = g.n - k0;
  if (rem < 1) return false;
  for (int j = k0; j < g.n; j++)
    if (g.ax[j] != g.ax[k0]) return false;
  const long long T0 = a0.mid;
  const long long P0 = (T0 + 63) / 64 * 64;
  const long long rows = g.space / T0;
  const long long plane16 = (rows * P0 + kPlaneAlign - 1) / kPlaneAlign *
                            kPlaneAlign;
  // room16: the u16 words from the start of the 16-bit planes on
  if ((long long)R1 * plane16 > room16) return false;
  std::vector<GroupPlan> later;
  const int nch = (rem + kPadMaxAxes - 1) / kPadMaxAxes;
  // one group per range: the budget only has to admit its K axes
  const Knobs kn{(size_t)1 << 30, 0, 1, 0, 0};
  long long reach = 0;
  for (int i = 0; i < k0; i++) reach += axis_reach(g.prob, g.ax[i]);
  int j = k0;
  for (int c = 0; c < nch; c++) {
    const int K = rem / nch + (c < rem % nch ? 1 : 0);
    const bool last = c == nch - 1;
    AxisRange r;
    r.begin = j;
    r.end = j + K;
    r.reach0 = reach;
    r.final = last;
    std::vector<GroupPlan> gs = plan_groups(g, R1, ptr, kSrcLayers,
                                            last ? dst : kDstLayers, kn, r);
    if (gs.size() != 1 || gs[0].a.k != K || gs[0].kernel < 0) return false;
    GroupArgs t = gs[0].a;
    if (!t.in16 || t.inner % T0) return false;
    t.inner = t.inner / T0 * P0;
    t.pitch = P0;
    t.t0 = T0;
    t.plane = plane16;
    t.pack = 1;
    GroupPlan base = gs[0];
    base.a = t;
    bool done = false;
    for (int lanes : {32, 16})
      for (int stages : {3, 2}) {
        if (done) break;
        GroupPlan v = tma_variant(base, lanes, stages, 256);
        if (tma_group_ok(v.a, t.rq[0], R1, lanes, stages)) {
          later.push_back(v);
          done = true;
        }
      }
    if (!done) return false;
    for (int i = j; i < j + K; i++) reach += axis_reach(g.prob, g.ax[i]);
    j += K;
  }
  f.a.pitch = P0;
  f.a.t0 = T0;
  f.a.plane = plane16;
  // row pairs as the first group's tiles: the packed ternary form runs on
  // them (the register kernels take them as Bo = 2)
  GroupPlan fv = f;
  fv.a.Bo = 2;
  fv.a.ntiles = (fv.a.outer + 1) / 2;
  if (f.a.Bo == 1 && f.a.nchunk == 1 && tern_first_ok(fv.a, R1))
    f = tern_first_variant(fv, 256);
  groups.resize(1);
  groups.insert(groups.end(), later.begin(), later.end());
  size_streamed(groups);
  return true;
}

// Every group that a streamed form serves takes it: the binary first group
// staged from cnt or counted from the code (three stages, then two), a
// strided group as tensor loads (64-word rows first, three stages where
// they fit).
void stream_groups(std::vector<GroupPlan> &groups, int R1) {
  // CC_TMA_BM=3: three-axis register rounds (512 threads) where they exist
  const char *be = getenv("CC_TMA_BM");
  const int tbm = be && atoi(be) == 3 ? 3 : 0;
  for (auto &p : groups) {
    if (p.kernel < 0 || p.a.nrounds <= 0) continue;
    bool done = false;
    for (int lanes : {16, 32})
      for (int stages : {3, 2}) {
        if (done || !tbm) break;
        GroupPlan t = p;
        t.a.tbm = tbm;
        GroupPlan v = tma_variant(t, lanes, stages, 512);
        if (tma_group_ok(v.a, p.a.rq[0], R1, lanes, stages)) {
          p = v;
          done = true;
        }
      }
    for (int stages : {3, 2, 0})
      if (!done && tma_first_ok(p.a, R1, stages)) {
        p = tma_first_variant(p, stages, 256);
        done = true;
      }
    for (int lanes : {32, 16})
      for (int stages : {3, 2}) {
        if (done) break;
        GroupPlan v = tma_variant(p, lanes, stages, 256);
        if (tma_group_ok(v.a, p.a.rq[0], R1, lanes, stages)) {
          p = v;
          done = true;
        }
      }
  }
  size_streamed(groups);
}

// Algorithmic HBM bytes of one group launch: every word of the space read
// once from its source (2-byte cnt, or lin layers of 2 or 4 bytes; a
// code-sourced launch reads its 8-byte code words) and written once to its
// destination (lout layers of 2 or 4 bytes, the 4-byte map or the 2-byte
// cnt).  Pad words of a padded plan are not counted.
long long group_bytes(const GroupArgs &a) {
  const long long words = a.outer * a.mid * (a.pitch && a.t0
                          ? a.inner / a.pitch * a.t0 : a.inner);
  long long rd = 0, wr = 0;
  if (a.src == kSrcCnt) rd = 2 * words;
  else if (a.src == kSrcCode) rd = 8 * a.ncode;
  else rd = (long long)a.lin * (a.in8 ? 1 : a.in16 ? 2 : 4) * words;
  if (a.dst == kDstLayers)
    wr = (long long)a.lout * (a.out8 ? 1 : a.out16 ? 2 : 4) * words;
  else if (a.dst == kDstMap) wr = 4 * words;
  else wr = 2 * words;
  return rd + wr;
}

// 8-bit planes between the streamed binary first group (read from cnt:
// gain and loss) and the streamed launch after it.  After the first group's
// k0 axes (the pair axis included), layer d of a 0/1 predicate counts at
// most C(k0, d) words, so max over d <= R of C(k0, d) <= 255 makes every
// value fit a byte: the first group writes half the bytes and the next
// launch reads half.  The byte planes sit past the R1 16-bit planes of the
// region (room16 u16 words); the launch after the first group writes those
// 16-bit planes while it reads the byte planes.  false leaves `groups`
// unchanged.
bool u8_plan(std::vector<GroupPlan> &groups, int R1, long long room16) {
  if (groups.size() < 2) return false;
  const GroupPlan &f = groups[0], &n = groups[1];
  if (f.a.tma != 2 || f.a.src != kSrcCnt || f.a.dst != kDstLayers ||
      n.a.tma != 1 || n.a.src != kSrcLayers || !n.a.in16 || n.a.pitch)
    return false;
  const int k0 = f.a.k + f.a.pair_axis;
  long long c = 1, mx = 1;
  for (int d = 1; d <= f.a.R && d <= k0; d++) {
    c = c * (k0 - d + 1) / d;
    mx = std::max(mx, c);
  }
  if (mx > 255) return false;
  const long long off8 = 2LL * R1 * f.a.plane;
  if (off8 + (long long)R1 * f.a.plane > 2 * room16 || n.a.plane != f.a.plane)
    return false;
  GroupPlan f8 = f;
  f8.a.out8 = 1;
  f8.a.off8 = off8;
  if (!tma_first_ok(f8.a, R1, f8.a.stages)) return false;
  const int q = n.a.rq[0] ? n.a.rq[0] : n.a.qax[0];
  const int lanes = n.a.W / 2;
  GroupPlan n8 = n;
  n8.a.in8 = 1;
  n8.a.off8 = off8;
  bool done = false;
  for (int st : {n.a.stages, 3, 4, 2}) {
    if (done) break;
    GroupPlan v = tma_variant(n8, lanes, st, n.threads);
    if (tma_group_ok(v.a, q, R1, lanes, st)) {
      n8 = v;
      done = true;
    }
  }
  if (!done) return false;
  groups[0] = f8;
  groups[1] = n8;
  groups[0].grid = groups[1].grid = 0;
  size_streamed(groups);
  return true;
}

}  // namespace cc
