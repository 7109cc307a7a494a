// outofcore.cu — transforms of cells whose distance layers exceed HBM.
//
// Placement follows the reference's policy for cells over the HBM budget:
// the layer planes go to host memory while cnt stays on the device
// (coldcore src/coldcore/gpu.py:253-260).  The reference then lets its
// kernels read the host planes in place over GH200's coherent C2C link
// (src/plugins/covering/dctcore_core.cuh:86-119).  A B200 host link is not
// coherent, so here the planes are streamed through device pieces by
// explicit copies, in two phases that together apply every axis once:
//
//   phase 1, slabs:   axes 0..s-1 on contiguous slabs of h rows of
//                     P_low = a_0 ... a_{s-1} words (one copy per plane);
//   phase 2, columns: axes s..n-1 on column blocks, words [x0, x0 + w) of
//                     each of the P_high = a_s ... a_{n-1} rows (one pitched
//                     2-D copy per plane).
//
// Each live plane crosses the host link twice per transform: slabs out
// (device to host) in phase 1, columns in (host to device) in phase 2.  cnt,
// the map and the code stay in HBM: the code is scattered into each slab,
// the cnt predicate read in place, and the map or cnt of a column block is
// copied into its pitched place in HBM.  Two device pieces on two streams
// overlap one piece's copies with the other's launches.  The launches are
// the in-memory engine's group kernels, planned over each piece's own
// geometry with an axis range (AxisRange): axes [0, s) of
// a_0 x ... x a_{s-1} x h, and axes [1, n-s+1) of w x a_s x ... x a_{n-1}.
//
// A record mode runs the same schedule without a device and returns every
// copy, fill, scatter and launch as a row, so the schedule's addressing and
// its result can be checked on a host.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>
#include "../../include/coldcore_b200/plugin.h"
#include "engine.h"

namespace cc {
namespace {

constexpr int kRecFields = 20;
constexpr long long kMaxPieceAxis = 1LL << 30;   // a piece's own axis
constexpr int kDefaultMinWidth = 32;             // 128-byte rows at 4 B
constexpr long long kMaxPitch = 2147483647LL;    // bytes, 2-D copy pitch
constexpr size_t kTileBudget = 100 * 1024;       // shared bytes per tile

enum Buf {
  kBufHost = 0, kBufPiece0 = 1, kBufPiece1 = 2, kBufStage0 = 3,
  kBufStage1 = 4, kBufCode = 5, kBufCnt = 6, kBufOut = 7, kNumBufs = 8
};
enum RecOp {
  kRecCopy = 1, kRecCopy2D = 2, kRecZero = 3, kRecScatter = 4,
  kRecLaunch = 5, kRecJoin = 6
};

struct Pieces {
  int split = 0;
  long long p_low = 0, p_high = 0, slab_rows = 0, n_slabs = 0;
  long long col_width = 0, n_cols = 0;
};

// The split and the piece sizes for pieces of at most `cap` words a plane:
// the largest low block P_low whose one-row slab fits (and whose row pitch a
// 2-D copy accepts) such that a column block of min(min_width, P_low) words
// of every high row fits too; then the most rows a slab and the widest
// column (whole multiples of min_width) that fit.
bool plan_pieces(const int *ax, int n, long long cap, long long min_width,
                 long long max_pitch_words, Pieces *out) {
  long long size = 1;
  for (int i = 0; i < n; i++) size *= ax[i];
  bool found = false;
  long long p_low = 1, wcap = 0;
  for (int s = 1; s < n; s++) {
    p_low *= ax[s - 1];
    if (p_low > cap || p_low > max_pitch_words) break;
    const long long p_high = size / p_low;
    if (cap / p_high >= std::min(min_width, p_low)) {
      out->split = s;
      out->p_low = p_low;
      out->p_high = p_high;
      wcap = cap / p_high;
      found = true;
    }
  }
  if (!found) return false;
  const long long pl = out->p_low, ph = out->p_high;
  const long long h =
      std::max(1LL, std::min(std::min(ph, cap / pl), kMaxPieceAxis));
  long long w = std::min(std::min(pl, wcap), kMaxPieceAxis);
  if (w >= min_width) w -= w % min_width;
  out->slab_rows = h;
  out->n_slabs = (ph + h - 1) / h;
  out->col_width = w;
  out->n_cols = (pl + w - 1) / w;
  return true;
}

// Words within distance R of one word (for grid_linf the largest such
// count, at an interior word), saturating at 2^40.
long long ball_size(const Geometry &g) {
  const long long kCap = 1LL << 40;
  if (g.prob == kTorus || g.prob == kGrid) {
    long long b = 1;
    for (int i = 0; i < g.n; i++)
      b = std::min(kCap, b * std::min<long long>(2 * g.R + 1, g.ax[i]));
    return b;
  }
  // distance distribution of the product: per axis, the offsets at each
  // distance (Hamming: 1 at 0, a-1 at 1; Lee on Z_a: 1 at 0, 2 at each
  // 0 < d < a/2, 1 at a/2 when a is even)
  std::vector<long long> poly(g.R + 1, 0), per(g.R + 1), nxt(g.R + 1);
  poly[0] = 1;
  for (int i = 0; i < g.n; i++) {
    const int a = g.ax[i];
    std::fill(per.begin(), per.end(), 0);
    per[0] = 1;
    if (g.prob == kHamming) {
      per[1] = a - 1;
    } else {
      for (int d = 1; d <= std::min(g.R, a / 2); d++)
        per[d] = 2 * d == a ? 1 : 2;
    }
    std::fill(nxt.begin(), nxt.end(), 0);
    for (int u = 0; u <= g.R; u++)
      for (int v = 0; u + v <= g.R; v++)
        nxt[u + v] = std::min(kCap, nxt[u + v] + poly[u] * per[v]);
    poly.swap(nxt);
  }
  long long s = 0;
  for (long long v : poly) s = std::min(kCap, s + v);
  return s;
}

// the cnt predicate of a gain (1) or loss (2) source at multiplicity mu,
// as the in-memory engine sets it
void predicate(int init_mode, int mu, int *pm, int *pt) {
  *pm = kPredEq;
  *pt = 0;
  if (init_mode == 1) {
    if (mu > 1) *pm = kPredDef;
  } else if (init_mode == 2) {
    if (mu == 1) *pt = 1; else *pm = kPredCrit;
  }
}

struct Cell {
  Geometry g{};
  int R1 = 1, init_mode = 0, out_mode = 1, mu = 1;
  int half = 0;        // 16-bit planes on the host and between phases
  int hb = 4;          // host bytes per word of one plane
  int live_mid = 1;    // live planes after phase 1
  long long M = 0, ball = 0, cap = 0, P = 0;
  long long host_bytes = 0, device_bytes = 0, link_bytes = 0;
  Pieces pc;
};

// The cell, its piece plan and its memory needs; the same validation as
// the in-memory engine's init and transform entry points (dct_init3,
// dct_set_code's counter rule, dct_transform's modes).  Window-pass cells
// (torus / grid axes above 16) are not streamed (-3).
int make_cell(int problem, int n, const int *ax, int R, int init_mode,
              int out_mode, int mu, long long M, long long maxmult,
              long long budget, int min_width, Cell *c) {
  if (n < 1 || n > kMaxAxes || R < 1 || !ax || problem < 0 || problem > 3)
    return -1;
  if (init_mode < 0 || init_mode > 2 || out_mode < 1 || out_mode > 3 ||
      (out_mode == 2 && init_mode != 0))
    return -1;
  if (mu < 1 || M < 0 || maxmult < 0 || min_width < 0 || budget < 1)
    return -1;
  const bool layered = problem == kHamming || problem == kLee;
  if (layered && R + 1 > kMaxLayers) return -1;
  if (!layered && out_mode == 3) return -1;
  Geometry &g = c->g;
  g.prob = problem; g.n = n; g.R = R; g.mu = mu;
  g.pw[0] = 1;
  for (int i = 0; i < n; i++) {
    if (ax[i] < 2 || ax[i] >= (1 << 24)) return -1;
    if (layered && ax[i] > 16) return -1;
    if (problem == kTorus && (ax[i] < 3 || 2 * R + 1 > ax[i])) return -1;
    if (ax[i] > 16) return -3;
    if (g.pw[i] > (1LL << 40) / ax[i]) return -2;
    g.ax[i] = ax[i];
    g.pw[i + 1] = g.pw[i] * ax[i];
  }
  g.space = g.pw[n];
  c->R1 = layered ? R + 1 : 1;
  c->init_mode = init_mode;
  c->out_mode = out_mode;
  c->mu = mu;
  c->M = init_mode == 0 ? M : 0;
  c->ball = ball_size(g);
  if (init_mode == 0) {
    // no uint16 counter above 65535: min(total, max multiplicity x |B|)
    const long long bound =
        maxmult > 0 && c->ball > LLONG_MAX / maxmult ? LLONG_MAX
                                                     : maxmult * c->ball;
    if (std::min(M, bound) > 65535) return -1;
  }
  const char *e = getenv("CC_HALF");
  const bool half_env = !(e && atoi(e) == 0);
  c->half = half_env && c->R1 >= 2 && out_mode != 3 &&
            (init_mode == 0 || c->ball <= 65535);
  c->hb = c->half ? 2 : 4;
  const long long per = 2LL * (c->R1 * 4LL + (out_mode == 2 ? 2 : 0));
  const long long avail = budget - c->M * 8;
  c->cap = avail / per - kPlaneAlign;
  if (c->cap < 1) return -2;
  const long long mw = min_width > 0 ? min_width : kDefaultMinWidth;
  if (!plan_pieces(ax, n, c->cap, mw, kMaxPitch / 4, &c->pc)) return -2;
  const Pieces &pc = c->pc;
  const long long words = std::max(pc.slab_rows * pc.p_low,
                                   pc.col_width * pc.p_high);
  c->P = (words + kPlaneAlign - 1) / kPlaneAlign * kPlaneAlign;
  long long reach = 0;
  for (int i = 0; i < pc.split; i++) reach += axis_reach(problem, ax[i]);
  c->live_mid = layered ? (int)std::min<long long>(reach, R) + 1 : 1;
  const long long X = g.space;
  c->host_bytes = (out_mode == 3 ? c->R1 : c->live_mid) * X * c->hb;
  c->device_bytes = c->P * per + c->M * 8;
  c->link_bytes = 2 * X * c->hb * c->live_mid +
                  (out_mode == 3 ? X * 4 * c->R1 : 0);
  return 0;
}

// The group launches of one piece: phase 1 runs axes [0, s) of
// a_0..a_{s-1} x len (len = slab rows), phase 2 axes [1, n-s+1) of
// len x a_s..a_{n-1} (len = column width).  Pointers are stand-ins, set per
// piece at launch; prefetching and the pair first group stay off (both
// assume the alignment of a whole plane, not of a piece).
std::vector<GroupPlan> plan_piece(const Cell &c, int phase, long long len) {
  const Geometry &G = c.g;
  const int s = c.pc.split;
  Geometry g{};
  g.prob = G.prob; g.R = G.R; g.mu = c.mu;
  AxisRange r;
  int src, dst;
  if (phase == 1) {
    g.n = s + 1;
    for (int i = 0; i < s; i++) g.ax[i] = G.ax[i];
    g.ax[s] = (int)len;
    r.begin = 0; r.end = s; r.reach0 = 0; r.final = false;
    src = c.init_mode == 0 ? kSrcLayers : kSrcCnt;
    dst = kDstLayers;
  } else {
    g.n = G.n - s + 1;
    g.ax[0] = (int)len;
    for (int i = s; i < G.n; i++) g.ax[i - s + 1] = G.ax[i];
    long long reach = 0;
    for (int i = 0; i < s; i++) reach += axis_reach(G.prob, G.ax[i]);
    r.begin = 1; r.end = g.n; r.reach0 = reach; r.final = true;
    src = kSrcLayers;
    dst = c.out_mode == 1 ? kDstMap : c.out_mode == 2 ? kDstCnt : kDstLayers;
  }
  g.pw[0] = 1;
  for (int i = 0; i < g.n; i++) g.pw[i + 1] = g.pw[i] * g.ax[i];
  g.space = g.pw[g.n];
  int32_t *const fake = reinterpret_cast<int32_t *>(uintptr_t(1) << 12);
  PlanPtrs ptr{fake, c.P, reinterpret_cast<uint16_t *>(fake), nullptr, 0,
               nullptr};
  ptr.layers16 = reinterpret_cast<uint16_t *>(fake + c.P);
  Knobs kn{kTileBudget, 0};
  kn.half = c.half;
  kn.pair = 0;
  return plan_groups(g, c.R1, ptr, src, dst, kn, r);
}

// The planes a phase hands to the next must be the ones it reads: phase 1
// ends writing live_mid planes of the host width, phase 2 starts reading
// them, and no launch prefetches or pairs.
bool plans_agree(const Cell &c, const std::vector<GroupPlan> &p, int phase) {
  if (p.empty()) return false;
  for (const GroupPlan &q : p)
    if (q.a.pipe || q.a.pair_axis) return false;
  if (phase == 1) {
    const GroupArgs &a = p.back().a;
    return a.dst == kDstLayers && a.lout == c.live_mid &&
           a.out16 == c.half;
  }
  const GroupArgs &a = p.front().a;
  return a.src == kSrcLayers && a.lin == c.live_mid && a.in16 == c.half;
}

__global__ void k_scatter_slab(int32_t *plane0, const long long *code,
                               long long n, long long x0) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += stride)
    atomicAdd(plane0 + (code[i] - x0), 1);
}

// Issues the schedule's operations: on the device, or as rows of kRecFields
// values (record mode).
struct Exec {
  char *base[kNumBufs] = {};
  cudaStream_t st[2] = {nullptr, nullptr};
  cudaEvent_t join[2] = {nullptr, nullptr};
  cudaEvent_t mark[3] = {nullptr, nullptr, nullptr};
  bool rec = false;
  long long rows = 0, cap_rows = 0;
  long long *out_rows = nullptr;

  void put(std::initializer_list<long long> v) {
    if (out_rows && rows < cap_rows) {
      long long *r = out_rows + rows * kRecFields;
      int i = 0;
      for (long long x : v) r[i++] = x;
      for (; i < kRecFields; i++) r[i] = 0;
    }
    rows++;
  }
  static cudaMemcpyKind kind(int db, int sb) {
    if (sb == kBufHost) return db == kBufHost ? cudaMemcpyHostToHost
                                              : cudaMemcpyHostToDevice;
    return db == kBufHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  }
  int copy(int s, int db, long long doff, int sb, long long soff,
           long long bytes) {
    if (rec) { put({kRecCopy, s, db, doff, sb, soff, bytes}); return 0; }
    CC_CK(cudaMemcpyAsync(base[db] + doff, base[sb] + soff, (size_t)bytes,
                          kind(db, sb), st[s]));
    return 0;
  }
  int copy2d(int s, int db, long long doff, long long dpitch, int sb,
             long long soff, long long spitch, long long wbytes,
             long long height) {
    if (rec) {
      put({kRecCopy2D, s, db, doff, dpitch, sb, soff, spitch, wbytes,
           height});
      return 0;
    }
    CC_CK(cudaMemcpy2DAsync(base[db] + doff, (size_t)dpitch,
                            base[sb] + soff, (size_t)spitch, (size_t)wbytes,
                            (size_t)height, kind(db, sb), st[s]));
    return 0;
  }
  int zero(int s, int b, long long off, long long bytes) {
    if (rec) { put({kRecZero, s, b, off, bytes}); return 0; }
    CC_CK(cudaMemsetAsync(base[b] + off, 0, (size_t)bytes, st[s]));
    return 0;
  }
  // plane 0 of piece b counts the code words [c0, c0 + n), all inside the
  // slab [x0, x0 + slab words)
  int scatter(int s, int b, long long c0, long long n, long long x0) {
    if (rec) { put({kRecScatter, s, b, c0, n, x0}); return 0; }
    const long long blocks = std::min<long long>((n + 255) / 256,
                                                 (long long)sm_count() * 8);
    k_scatter_slab<<<(unsigned)std::max(1LL, blocks), 256, 0, st[s]>>>(
        reinterpret_cast<int32_t *>(base[b]),
        reinterpret_cast<const long long *>(base[kBufCode]) + c0, n, x0);
    CC_CK(cudaGetLastError());
    return 0;
  }
  int launch(int s, const GroupPlan &p, const Cell &c, long long aux_off,
             long long space, int phase, int axis0) {
    const GroupArgs &a = p.a;
    const int piece = kBufPiece0 + s;
    if (rec) {
      put({kRecLaunch, s, piece, c.P, c.P * 4, a.src, a.dst, a.lin, a.lout,
           a.in16, a.out16, axis0, a.k, aux_off, space, phase, a.inner,
           a.mid, a.outer, a.pack});
      return 0;
    }
    GroupPlan q = p;
    GroupArgs &b = q.a;
    int32_t *lay = reinterpret_cast<int32_t *>(base[piece]);
    b.layers = lay;
    b.plane = c.P;
    b.layers16 = reinterpret_cast<uint16_t *>(lay + c.P);
    b.cnt = nullptr;
    if (b.src == kSrcCnt)
      b.cnt = const_cast<uint16_t *>(
                  reinterpret_cast<const uint16_t *>(base[kBufCnt])) +
              aux_off;
    else if (b.dst == kDstCnt)
      b.cnt = reinterpret_cast<uint16_t *>(base[kBufStage0 + s]);
    b.map = nullptr;
    b.code = nullptr;
    b.ncode = 0;
    b.code_bounds = nullptr;
    b.red = nullptr;
    b.red_mode = 0;
    predicate(c.init_mode, c.mu, &b.pmode, &b.ptarget);
    b.mu = c.mu;
    return launch_group(q, st[s]);
  }
  // every operation issued so far on either stream precedes every later
  // one (and mark[k] records the point)
  int join_streams(int k) {
    if (rec) { put({kRecJoin, k}); return 0; }
    CC_CK(cudaEventRecord(join[k & 1], st[1]));
    CC_CK(cudaStreamWaitEvent(st[0], join[k & 1], 0));
    CC_CK(cudaEventRecord(mark[k], st[0]));
    CC_CK(cudaStreamWaitEvent(st[1], mark[k], 0));
    return 0;
  }
};

int run_schedule(const Cell &c, Exec &x, const long long *code) {
  const Pieces &pc = c.pc;
  const long long X = c.g.space, P = c.P, hb = c.hb;
  const long long h_last = pc.p_high - (pc.n_slabs - 1) * pc.slab_rows;
  const long long w_last = pc.p_low - (pc.n_cols - 1) * pc.col_width;
  const std::vector<GroupPlan> p1 = plan_piece(c, 1, pc.slab_rows);
  const std::vector<GroupPlan> p1r =
      h_last == pc.slab_rows ? p1 : plan_piece(c, 1, h_last);
  const std::vector<GroupPlan> p2 = plan_piece(c, 2, pc.col_width);
  const std::vector<GroupPlan> p2r =
      w_last == pc.col_width ? p2 : plan_piece(c, 2, w_last);
  if (!plans_agree(c, p1, 1) || !plans_agree(c, p1r, 1) ||
      !plans_agree(c, p2, 2) || !plans_agree(c, p2r, 2))
    return -5;
  // byte offset of plane d in a piece: 32-bit planes from 0, 16-bit planes
  // from 32-bit plane 1 on (clear of plane 0, the scattered code and the map)
  auto plane_off = [&](int d) {
    return c.half ? P * 4 + (long long)d * P * 2 : (long long)d * P * 4;
  };
  int rc;
  if ((rc = x.join_streams(0))) return rc;
  // ---- phase 1: slabs, axes 0..s-1
  for (long long i = 0; i < pc.n_slabs; i++) {
    const int s = (int)(i & 1);
    const int piece = kBufPiece0 + s;
    const long long rows = std::min(pc.slab_rows, pc.p_high - i * pc.slab_rows);
    const long long words = rows * pc.p_low;
    const long long x0 = i * pc.slab_rows * pc.p_low;
    if (c.init_mode == 0) {
      if ((rc = x.zero(s, piece, 0, words * 4))) return rc;
      const long long c0 = std::lower_bound(code, code + c.M, x0) - code;
      const long long c1 =
          std::lower_bound(code + c0, code + c.M, x0 + words) - code;
      if (c1 > c0 && (rc = x.scatter(s, piece, c0, c1 - c0, x0))) return rc;
    }
    int axis0 = 0;
    for (const GroupPlan &p : rows == pc.slab_rows ? p1 : p1r) {
      if ((rc = x.launch(s, p, c, x0, words, 1, axis0))) return rc;
      axis0 += p.a.k;
    }
    for (int d = 0; d < c.live_mid; d++)
      if ((rc = x.copy(s, kBufHost, (d * X + x0) * hb, piece, plane_off(d),
                       words * hb)))
        return rc;
  }
  if ((rc = x.join_streams(1))) return rc;
  // ---- phase 2: column blocks, axes s..n-1
  for (long long i = 0; i < pc.n_cols; i++) {
    const int s = (int)(i & 1);
    const int piece = kBufPiece0 + s;
    const long long x0 = i * pc.col_width;
    const long long wc = std::min(pc.col_width, pc.p_low - x0);
    const long long words = wc * pc.p_high;
    for (int d = 0; d < c.live_mid; d++)
      if ((rc = x.copy2d(s, piece, plane_off(d), wc * hb, kBufHost,
                         (d * X + x0) * hb, pc.p_low * hb, wc * hb,
                         pc.p_high)))
        return rc;
    int axis0 = 1;
    for (const GroupPlan &p : wc == pc.col_width ? p2 : p2r) {
      if ((rc = x.launch(s, p, c, 0, words, 2, axis0))) return rc;
      axis0 += p.a.k;
    }
    if (c.out_mode == 1) {
      rc = x.copy2d(s, kBufOut, x0 * 4, pc.p_low * 4, piece, 0, wc * 4,
                    wc * 4, pc.p_high);
    } else if (c.out_mode == 2) {
      rc = x.copy2d(s, kBufOut, x0 * 2, pc.p_low * 2, kBufStage0 + s, 0,
                    wc * 2, wc * 2, pc.p_high);
    } else {
      for (int d = 0; d < c.R1 && !rc; d++)
        rc = x.copy2d(s, kBufHost, (d * X + x0) * 4, pc.p_low * 4, piece,
                      (long long)d * P * 4, wc * 4, wc * 4, pc.p_high);
    }
    if (rc) return rc;
  }
  return x.join_streams(2);
}

// sorted copy of a host code, its largest multiplicity; false on a word
// outside [0, X)
bool sort_code(const long long *code, long long M, long long X,
               std::vector<long long> *out, long long *maxmult) {
  out->assign(code, code + M);
  for (long long w : *out)
    if (w < 0 || w >= X) return false;
  std::sort(out->begin(), out->end());
  *maxmult = 0;
  for (long long i = 0; i < M;) {
    long long j = i + 1;
    while (j < M && (*out)[j] == (*out)[i]) j++;
    *maxmult = std::max(*maxmult, j - i);
    i = j;
  }
  return true;
}

long long space_of(int n, const int *ax) {
  if (n < 1 || n > kMaxAxes || !ax) return -1;
  long long X = 1;
  for (int i = 0; i < n; i++) {
    if (ax[i] < 2 || X > (1LL << 40) / ax[i]) return -1;
    X *= ax[i];
  }
  return X;
}

// Frees what one streamed transform allocated, on every way out.
struct Owned {
  void *dev[5] = {};
  cudaStream_t st[2] = {};
  cudaEvent_t ev[5] = {};
  ~Owned() {
    for (cudaStream_t s : st)
      if (s) cudaStreamSynchronize(s);
    for (void *p : dev)
      if (p) cudaFree(p);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    for (cudaStream_t s : st)
      if (s) cudaStreamDestroy(s);
  }
};

}  // namespace
}  // namespace cc

using namespace cc;

extern "C" {

int dct_b200_ooc_plan(int problem, int n, const int *ax, int R,
                      int init_mode, int out_mode, long long M,
                      long long maxmult, long long device_budget,
                      int min_width, long long *info, int cap) {
  Cell c;
  const int rc = make_cell(problem, n, ax, R, init_mode, out_mode, 1, M,
                           maxmult, device_budget, min_width, &c);
  if (rc) return rc;
  const Pieces &pc = c.pc;
  const long long v[17] = {pc.split,   pc.p_low,        pc.p_high,
                           pc.slab_rows, pc.n_slabs,    pc.col_width,
                           pc.n_cols,  c.cap,           c.P,
                           c.half,     c.live_mid,      c.host_bytes,
                           c.device_bytes, c.link_bytes, c.ball,
                           c.R1,       c.hb};
  for (int i = 0; i < 17 && i < cap; i++)
    if (info) info[i] = v[i];
  return 0;
}

long long dct_b200_ooc_record(int problem, int n, const int *ax, int R,
                              int init_mode, int out_mode, int mu,
                              const long long *code, long long M,
                              long long device_budget, int min_width,
                              long long *rows, long long cap_rows) {
  const long long X = space_of(n, ax);
  if (X < 0 || M < 0 || (init_mode == 0 && M > 0 && !code)) return -1;
  std::vector<long long> sorted;
  long long mx = 0;
  if (init_mode == 0 && !sort_code(code, M, X, &sorted, &mx)) return -1;
  Cell c;
  int rc = make_cell(problem, n, ax, R, init_mode, out_mode, mu, M, mx,
                     device_budget, min_width, &c);
  if (rc) return rc;
  Exec x;
  x.rec = true;
  x.out_rows = rows;
  x.cap_rows = rows ? cap_rows : 0;
  rc = run_schedule(c, x, sorted.data());
  if (rc) return rc;
  return x.rows;
}

int dct_b200_ooc_transform(int problem, int n, const int *ax, int R,
                           int init_mode, int out_mode, int mu,
                           const long long *code, long long M,
                           const uint16_t *cnt, void *out, void *host,
                           long long host_bytes, long long device_budget,
                           int min_width, float *ms) {
  const long long X = space_of(n, ax);
  if (X < 0 || M < 0 || (init_mode == 0 && M > 0 && !code)) return -1;
  std::vector<long long> sorted;
  long long mx = 0;
  if (init_mode == 0 && !sort_code(code, M, X, &sorted, &mx)) return -1;
  Cell c;
  int rc = make_cell(problem, n, ax, R, init_mode, out_mode, mu, M, mx,
                     device_budget, min_width, &c);
  if (rc) return rc;
  if (!host || host_bytes < c.host_bytes) return -1;
  if (init_mode != 0 && !cnt) return -1;
  if (out_mode != 3 && !out) return -1;
  // the caller's cnt and out may still be written by work on other streams
  CC_CK(cudaDeviceSynchronize());
  Owned own;
  Exec x;
  const size_t piece = (size_t)c.P * c.R1 * 4;
  for (int b = 0; b < 2; b++) {
    CC_CK(cudaMalloc(&own.dev[b], piece));
    x.base[kBufPiece0 + b] = static_cast<char *>(own.dev[b]);
    if (out_mode == 2) {
      CC_CK(cudaMalloc(&own.dev[2 + b], (size_t)c.P * 2));
      x.base[kBufStage0 + b] = static_cast<char *>(own.dev[2 + b]);
    }
    CC_CK(cudaStreamCreateWithFlags(&own.st[b], cudaStreamNonBlocking));
    x.st[b] = own.st[b];
  }
  for (int k = 0; k < 5; k++) CC_CK(cudaEventCreate(&own.ev[k]));
  x.join[0] = own.ev[0];
  x.join[1] = own.ev[1];
  for (int k = 0; k < 3; k++) x.mark[k] = own.ev[2 + k];
  if (init_mode == 0 && c.M > 0) {
    CC_CK(cudaMalloc(&own.dev[4], (size_t)c.M * 8));
    CC_CK(cudaMemcpyAsync(own.dev[4], sorted.data(), (size_t)c.M * 8,
                          cudaMemcpyHostToDevice, x.st[0]));
    x.base[kBufCode] = static_cast<char *>(own.dev[4]);
  }
  x.base[kBufHost] = static_cast<char *>(host);
  x.base[kBufCnt] = reinterpret_cast<char *>(const_cast<uint16_t *>(cnt));
  x.base[kBufOut] = static_cast<char *>(out);
  rc = run_schedule(c, x, sorted.data());
  if (rc) return rc;
  CC_CK(cudaEventSynchronize(x.mark[2]));
  if (ms) {
    CC_CK(cudaEventElapsedTime(&ms[0], x.mark[0], x.mark[1]));
    CC_CK(cudaEventElapsedTime(&ms[1], x.mark[1], x.mark[2]));
  }
  return 0;
}

}  // extern "C"
