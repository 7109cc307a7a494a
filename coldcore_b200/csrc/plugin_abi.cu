// plugin_abi.cu — the extern "C" plugin ABI v1 of the B200 covering engine.
//
// Host side of every entry point declared in include/coldcore_b200/plugin.h:
// validation before any mutation, the represented multisets (uploaded /
// active, coldcore src/plugins/covering/dct_hc.cu:46-56), staging through
// pinned buffers, the transform planner, and the result copies.  Semantics
// follow the reference entry points cited per function; the device work is
// this engine's own (transform_group.cu, transform_window.cu, walks.cu,
// reduce.cu) and runs in call order on one engine-owned stream.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../include/coldcore_b200/plugin.h"
#include "engine.h"

namespace cc {

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int g_dct_blocks = 0;

}  // namespace cc

using namespace cc;

namespace {

constexpr long long kCounterMax = 65535;    // uint16 cnt
constexpr long long kStageCap = 1 << 16;    // words per staged chunk

struct Plan {
  std::vector<GroupPlan> groups;   // layered / small-axis path
  std::vector<WindowArgs> passes;  // wide window path
  bool window = false;
  int scatter_plane = -1;          // window recount: plane of the code counts
};

struct State {
  bool live = false;
  Geometry g{};
  int R1 = 1;                      // planes the transform math uses
  int nplanes = 0;                 // planes allocated
  long long plane = 0;
  int32_t *layers = nullptr;
  uint16_t *cnt = nullptr;
  long long cnt_len = 0;
  uint32_t *owner = nullptr;
  int use_owner = 0;
  int layers_mode = 0, cnt_mode = 0;
  // layers_mode 1: the R+1 layer planes in pinned host memory (plane d at
  // h_layers + d*|X|), streamed by every transform (outofcore.cu); the
  // device keeps plane 0 alone, the map
  bool streamed = false;
  int32_t *h_layers = nullptr;
  long long h_layers_bytes = 0;
  // support tables, SoA slots
  int32_t *tbl = nullptr, *tbl2 = nullptr;
  int slots = 0, slots2 = 0;
  long long len = 0;
  int fmt = 0;
  // code
  long long *d_code = nullptr;
  long long code_cap = 0, codeM = 0;
  long long *d_bounds = nullptr;   // per-tile code slices of a recount
  long long bounds_cap = 0;
  // staging
  long long *h_words = nullptr, *d_words = nullptr;
  int32_t *h_out = nullptr, *d_out = nullptr;
  long long *h_scalar = nullptr, *d_scalar = nullptr;
  // one bit per word, the predicate of a large gather call (walks.cu)
  uint8_t *d_bits = nullptr;
  int32_t *d_hist = nullptr;
  uint32_t *d_ext32 = nullptr;
  int64_t *d_ext64 = nullptr;
  int32_t *d_extv = nullptr;
  long long extract_cap = 0;
  // multisets (coldcore dct_hc.cu:46-56) + max multiplicity of `active`
  // uploaded: the staged code, sorted; active: the represented multiset.
  // A recount makes active = uploaded; the hash map is then built lazily,
  // on the first call that needs per-word counts (ensure_active).
  std::vector<long long> up_sorted;
  std::unordered_map<long long, int> active;
  bool active_pending = false;
  long long active_size = 0;
  int up_max = 0;
  std::vector<int> mult_hist;      // distinct active words per multiplicity
  int act_max = 0;
  long long stats[8] = {0};
  long long bytes_dev = 0, bytes_host = 0;
  unsigned long long dd_last = 0;
  bool layered_out = false;        // last transform left N_0..N_R
  // set side (setside.cu): the listed predicate set Z, cached per cnt state
  bool set_ok = false;             // support table proven == metric ball
  int set_policy = 1;              // DCT_SET_GATHER: 0 off, 1 auto, 2 force
  long long set_min = -1;          // DCT_SET_MIN: walk size that tries it
  long long set_ratio = 2;         // DCT_SET_RATIO: set side while |Z| <= r|B|
  unsigned long long *zbuf = nullptr, *d_found = nullptr;
  long long zcap = 0, zcap_max = 0;
  unsigned long long cnt_ver = 1;  // bumped by every cnt mutation
  int z_mode = -1, z_target = 0, z_mu = 0;
  unsigned long long z_ver = 0;
  bool z_valid = false;
  long long z_n = 0;
  // swap_eval fast path: packed host/device staging and the drop lists
  char *h_swap = nullptr, *d_swap = nullptr;
  long long *d_list = nullptr;
  long long lcap = 0;
  // device greedy: state, placed words, words satisfied per placement
  char *d_greedy = nullptr;
  long long *d_placed = nullptr, *h_placed = nullptr, *d_fresh = nullptr;
  long long placed_cap = 0;
  Plan plans[3][4];                // [init_mode][out_mode]
  bool plan_ok[3][4] = {{false}};
  bool tuned[3][4] = {{false}};
  float tune_ms[3][4] = {{0}};
};

State S;
cudaStream_t g_stream = nullptr;
int g_mu = 1;

// per-launch device timing of the last transform (DCT_TIMING=1 in the
// environment at load, or dct_b200_set_timing(1)): events around every
// launch, read after the transform's final synchronisation
constexpr int kMaxTimed = 64;
int g_timing = -1;
cudaEvent_t g_ev[kMaxTimed + 1];
float g_last_ms[kMaxTimed];
int g_last_n = 0;

bool timing_on() {
  if (g_timing < 0) g_timing = getenv("DCT_TIMING") ? 1 : 0;
  return g_timing == 1;
}

int timing_mark(int i) {
  if (!timing_on() || i > kMaxTimed) return 0;
  if (!g_ev[i]) CC_CK(cudaEventCreate(&g_ev[i]));
  CC_CK(cudaEventRecord(g_ev[i], g_stream));
  return 0;
}

long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

int dev_alloc(void **p, size_t bytes, int mode) {
  cudaError_t e;
  if (mode == 0) {
    e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) S.bytes_dev += bytes;
  } else {
    // the reference's LPDDR / managed placements (dct_hc.cu alloc_buf):
    // a B200 host has no coherent C2C memory, so both map to managed
    // memory that the driver pages in on demand
    e = cudaMallocManaged(p, bytes);
    if (e == cudaSuccess) S.bytes_host += bytes;
  }
  if (e != cudaSuccess) {
    fprintf(stderr, "coldcore_b200: allocation of %zu bytes failed: %s\n",
            bytes, cudaGetErrorString(e));
    *p = nullptr;
    return -1;
  }
  return 0;
}

bool valid_words(const long long *w, long long n) {
  if (n < 0 || (n && !w)) return false;
  for (long long i = 0; i < n; i++)
    if (w[i] < 0 || w[i] >= S.g.space) return false;
  return true;
}

// exact uint16 bound: no counter can exceed min(total, maxmult * |B|)
bool within_counter(long long total, long long maxmult) {
  long long b = maxmult * S.len;
  if (b > total) b = total;
  return b <= kCounterMax;
}

void hist_move(int from, int to) {
  if (from > 0) S.mult_hist[from]--;
  if (to > 0) S.mult_hist[to]++;
  if (to > S.act_max) S.act_max = to;
  while (S.act_max > 0 && S.mult_hist[S.act_max] == 0) S.act_max--;
}

void set_active(const std::unordered_map<long long, int> &m, long long sz) {
  S.active_pending = false;
  S.active = m;
  S.active_size = sz;
  std::fill(S.mult_hist.begin(), S.mult_hist.end(), 0);
  S.act_max = 0;
  for (const auto &e : m) {
    S.mult_hist[e.second]++;
    if (e.second > S.act_max) S.act_max = e.second;
  }
}

// the multiset of the last recount, as a hash map with its histogram
void ensure_active() {
  if (!S.active_pending) return;
  S.active_pending = false;
  S.active.clear();
  S.active.reserve(S.up_sorted.size() * 2 + 1);
  std::fill(S.mult_hist.begin(), S.mult_hist.end(), 0);
  S.act_max = 0;
  const auto &v = S.up_sorted;
  for (size_t i = 0; i < v.size();) {
    size_t j = i + 1;
    while (j < v.size() && v[j] == v[i]) j++;
    const int c = (int)(j - i);
    S.active.emplace(v[i], c);
    S.mult_hist[c]++;
    if (c > S.act_max) S.act_max = c;
    i = j;
  }
  S.active_size = (long long)v.size();
}

void apply_active(const std::unordered_map<long long, int> &batch,
                  int delta, long long nw) {
  ensure_active();
  for (const auto &e : batch) {
    int &c = S.active[e.first];
    const int before = c;
    c += delta * e.second;
    hist_move(before, c);
    if (c == 0) S.active.erase(e.first);
  }
  S.active_size += delta * nw;
}

// validate an update batch against `active`; fills `batch`
int check_update(const long long *words, int nw, int delta,
                 std::unordered_map<long long, int> &batch) {
  ensure_active();
  if (!valid_words(words, nw) || (delta != 1 && delta != -1)) return -1;
  batch.reserve((size_t)nw * 2 + 1);
  for (int i = 0; i < nw; i++) ++batch[words[i]];
  if (delta == -1) {
    for (const auto &e : batch) {
      auto it = S.active.find(e.first);
      if (it == S.active.end() || it->second < e.second) return -1;
    }
  } else {
    long long mx = S.act_max;
    for (const auto &e : batch) {
      auto it = S.active.find(e.first);
      long long m = (it == S.active.end() ? 0 : it->second) + e.second;
      if (m > mx) mx = m;
    }
    if (!within_counter(S.active_size + nw, mx)) return -1;
  }
  return 0;
}

int fetch_scalar(long long *r, int slot = 0) {
  CC_CK(cudaMemcpyAsync(S.h_scalar + slot, S.d_scalar + slot, 8,
                        cudaMemcpyDeviceToHost, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  *r = S.h_scalar[slot];
  return 0;
}

int stage_words(const long long *words, long long nb) {
  memcpy(S.h_words, words, (size_t)nb * 8);
  CC_CK(cudaMemcpyAsync(S.d_words, S.h_words, (size_t)nb * 8,
                        cudaMemcpyHostToDevice, g_stream));
  return 0;
}

WalkArgs walk_args() {
  WalkArgs w;
  w.g = S.g;
  w.g.mu = g_mu;
  const bool ox = S.fmt == 1 && S.tbl2;
  w.tbl = ox ? S.tbl2 : S.tbl;
  w.slots = ox ? S.slots2 : S.slots;
  w.len = S.len;
  w.cnt = S.cnt;
  return w;
}

void free_all() {
  if (g_stream) cudaStreamSynchronize(g_stream);
  auto F = [](void *p) { if (p) cudaFree(p); };
  auto FH = [](void *p) { if (p) cudaFreeHost(p); };
  F(S.layers); F(S.cnt); F(S.owner); F(S.tbl); F(S.tbl2); F(S.d_code);
  F(S.d_bounds);
  F(S.d_words); F(S.d_out); F(S.d_scalar); F(S.d_hist); F(S.d_ext32);
  F(S.d_ext64); F(S.d_extv); F(S.zbuf); F(S.d_found);
  F(S.d_swap); F(S.d_list); FH(S.h_swap);
  F(S.d_greedy); F(S.d_placed); F(S.d_fresh); FH(S.h_placed);
  F(S.d_bits);
  FH(S.h_layers);
  FH(S.h_words); FH(S.h_out); FH(S.h_scalar);
  S.~State();
  new (&S) State();
}

// ------------------------------------------------------------ planner
// shared-memory budget of one tile (CC_SMEM_BUDGET_KB overrides; read
// whenever a plan is built, i.e. once per cell and transform kind)
size_t smem_budget() {
  const char *e = getenv("CC_SMEM_BUDGET_KB");
  long long b = e ? atoll(e) * 1024 : 100 * 1024;
  if (b < 16 * 1024) b = 16 * 1024;
  if (b > 220 * 1024) b = 220 * 1024;
  return (size_t)b;
}

// Schedule knobs of a group plan (planner.cu): CC_SMEM_BUDGET_KB /
// CC_PIPE override the defaults; the autotuner tries several.
Knobs default_knobs() {
  const char *pe = getenv("CC_PIPE");
  return {smem_budget(), pe ? atoi(pe) : 1};
}

// 16-bit planes between the launches of one transform are exact when no
// intermediate layer value can pass 65535: a layer counts words within a
// distance, so it is at most the occurrences (<= 65535 by the rule that
// set_code enforces) for a code, and at most |B| for a predicate.  They sit
// from int32 plane 1 on, clear of the int32 map in plane 0; a transform
// that outputs every layer keeps int32 planes throughout.  CC_HALF=0 turns
// them off.
bool half_planes_ok(int src, int dst) {
  const char *e = getenv("CC_HALF");
  if (e && atoi(e) == 0) return false;
  if (S.R1 < 2 || dst == kDstLayers) return false;
  return src == kSrcCode || S.len <= 65535;
}

Plan build_group_plan(int src, int dst, Knobs kn) {
  Plan P;
  PlanPtrs ptr{S.layers, S.plane, S.cnt, S.d_code, S.codeM, nullptr};
  kn.half = half_planes_ok(src, dst) ? 1 : 0;
  ptr.layers16 = reinterpret_cast<uint16_t *>(S.layers + S.plane);
  Geometry g = transform_geometry(S.g);
  g.mu = g_mu;
  P.groups = plan_groups(g, S.R1, ptr, src, dst, kn);
  if (kn.pad) {
    // a padded plan or none (the tuner then skips this knob setting)
    if (!kn.half || !pad_plan(P.groups, g, ptr, dst, S.R1,
                              (long long)(S.nplanes - 1) * S.plane * 2))
      P.groups.clear();
    return P;
  }
  // CC_TMA=1: every group the streamed form serves takes it (64-word rows
  // first, three stages where they fit); the autotuner otherwise times it
  // beside the other forms
  const char *ue = getenv("CC_U8");
  const bool u8_off = ue && atoi(ue) == 0;
  if (kn.u8) {
    // 8-bit planes after the streamed first group, or no plan
    stream_groups(P.groups, S.R1);
    if (u8_off || !u8_plan(P.groups, S.R1,
                         (long long)(S.nplanes - 1) * S.plane * 2)) P.groups.clear();
    return P;
  }
  const char *te = getenv("CC_TMA");
  if (te && atoi(te) == 1) {
    stream_groups(P.groups, S.R1);
    if (!u8_off) u8_plan(P.groups, S.R1,
                         (long long)(S.nplanes - 1) * S.plane * 2);
  }
  return P;
}

bool any_wide_axis() {
  for (int j = 0; j < S.g.n; j++)
    if (S.g.ax[j] > 16) return true;
  return false;
}

// window path: pass j reads buf[j] and writes buf[j+1]; buffers are planes
// 0..2, kSrc from cnt (-1) or a plane, the last one the map / cnt (-2)
Plan build_window_plan(int init_mode, int out_mode) {
  Plan P;
  P.window = true;
  const Geometry &g = S.g;
  const int n = g.n;
  std::vector<int> buf(n + 1);
  buf[0] = init_mode == 0 ? 2 : -1;
  P.scatter_plane = init_mode == 0 ? 2 : -1;
  buf[n] = out_mode == 2 ? -2 : 0;
  for (int j = n - 1; j >= 1; j--) {
    const int nxt = buf[j + 1];
    int pick = 0;
    while (pick == nxt || (j == 1 && pick == buf[0])) pick++;
    buf[j] = pick;
  }
  for (int j = 0; j < n; j++) {
    WindowArgs w{};
    const int s = buf[j], d = buf[j + 1];
    if (s == -1) w.src16 = S.cnt; else w.src32 = S.layers + s * S.plane;
    if (d == -2) w.dst16 = S.cnt; else w.dst32 = S.layers + d * S.plane;
    w.pmode = kPredEq;
    w.mu = g_mu;
    w.space = g.space;
    w.stride = g.pw[j];
    w.q = g.ax[j];
    w.R = g.R;
    w.grid = g.prob == kGrid;
    P.passes.push_back(w);
  }
  return P;
}

Plan make_plan(int init_mode, int out_mode, Knobs kn) {
  const int src = init_mode == 0 ? kSrcCode : kSrcCnt;
  const int dst = out_mode == 1 ? kDstMap
                  : out_mode == 2 ? kDstCnt : kDstLayers;
  if ((S.g.prob == kTorus || S.g.prob == kGrid) && any_wide_axis())
    return build_window_plan(init_mode, out_mode);
  return build_group_plan(src, dst, kn);
}

Plan &plan_for(int init_mode, int out_mode) {
  if (!S.plan_ok[init_mode][out_mode]) {
    Plan P;
    // CC_TMA=1 also asks for the padded plan where a cell has one
    const char *te = getenv("CC_TMA");
    if (te && atoi(te) == 1) {
      Knobs kn = default_knobs();
      kn.pad = 1;
      P = make_plan(init_mode, out_mode, kn);
    }
    if (P.groups.empty() && !P.window)
      P = make_plan(init_mode, out_mode, default_knobs());
    S.plans[init_mode][out_mode] = P;
    S.plan_ok[init_mode][out_mode] = true;
  }
  return S.plans[init_mode][out_mode];
}

void set_predicate(int init_mode, int *pm, int *pt) {
  *pm = kPredEq;
  *pt = 0;
  if (init_mode == 1) {
    if (g_mu == 1) *pt = 0; else *pm = kPredDef;
  } else if (init_mode == 2) {
    if (g_mu == 1) *pt = 1; else *pm = kPredCrit;
  }
}

// Device bytes a streamed transform may allocate: CC_OOC_BUDGET_KB, else
// 80% of the free device memory less 256 MiB.
long long ooc_budget() {
  if (const char *e = getenv("CC_OOC_BUDGET_KB")) return atoll(e) << 10;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return std::max(0LL, (long long)(fr / 10 * 8) - (256LL << 20));
}

// A transform of a layers_mode-1 cell: the code (uploaded, sorted) or cnt
// in, the map (plane 0) or cnt out on the device, or every layer out into
// the host planes.
int run_streamed(int init_mode, int out_mode) {
  CC_CK(cudaStreamSynchronize(g_stream));
  void *out = out_mode == 1 ? static_cast<void *>(S.layers)
              : out_mode == 2 ? static_cast<void *>(S.cnt) : nullptr;
  float ms[2] = {0, 0};
  const long long M = init_mode == 0 ? S.codeM : 0;
  const int rc = dct_b200_ooc_transform(
      S.g.prob, S.g.n, S.g.ax, S.g.R, init_mode, out_mode, g_mu,
      M ? S.up_sorted.data() : nullptr, M, S.cnt, out, S.h_layers,
      S.h_layers_bytes, ooc_budget(), 0, ms);
  if (rc) return rc;
  g_last_n = 0;
  if (timing_on()) {
    g_last_ms[0] = ms[0];
    g_last_ms[1] = ms[1];
    g_last_n = 2;
  }
  return 0;
}

int run_transform(int init_mode, int out_mode) {
  if (tma_fault_pending()) {
    // an earlier streamed launch gave up waiting for its tile loads
    tma_fault_clear();
    fprintf(stderr, "coldcore_b200: a streamed group launch timed out "
            "waiting for its tensor loads\n");
    return -8;
  }
  if (S.streamed) return run_streamed(init_mode, out_mode);
  Plan &P = plan_for(init_mode, out_mode);
  int pm, pt;
  set_predicate(init_mode, &pm, &pt);
  int nt = 0, rc = 0;
  if (P.window) {
    if (init_mode == 0) {
      int32_t *pl = S.layers + P.scatter_plane * S.plane;
      CC_CK(cudaMemsetAsync(pl, 0, (size_t)S.g.space * 4, g_stream));
      rc = launch_scatter(pl, S.d_code, S.codeM, g_stream);
      if (rc) return rc;
    }
    if ((rc = timing_mark(nt))) return rc;
    for (auto &w : P.passes) {
      WindowArgs x = w;
      x.pmode = pm;
      x.ptarget = pt;
      x.mu = g_mu;
      if ((rc = launch_window(x, g_stream))) return rc;
      if ((rc = timing_mark(++nt))) return rc;
    }
  } else {
    if (P.groups.empty()) return -1;           // the planner found no tile
    if (init_mode == 0) {
      const GroupArgs &a0 = P.groups[0].a;
      const long long need = a0.ntiles + 1;
      if (need > S.bounds_cap) {
        if (S.d_bounds) cudaFree(S.d_bounds);
        S.d_bounds = nullptr;
        CC_CK(cudaMalloc(&S.d_bounds, (size_t)need * 8));
        S.bounds_cap = need;
      }
      rc = launch_code_bounds(S.d_code, S.codeM,
                              (long long)a0.Bo * a0.mid * a0.inner,
                              a0.ntiles,
                              S.d_bounds, g_stream);
      if (rc) return rc;
    }
    if ((rc = timing_mark(nt))) return rc;
    for (auto &gp : P.groups) {
      GroupPlan p = gp;
      p.a.pmode = pm;
      p.a.ptarget = pt;
      p.a.mu = g_mu;
      p.a.code = S.d_code;
      p.a.ncode = S.codeM;
      p.a.code_bounds = S.d_bounds;
      if ((rc = launch_group(p, g_stream))) return rc;
      if ((rc = timing_mark(++nt))) return rc;
    }
  }
  g_last_n = 0;
  if (timing_on()) {
    CC_CK(cudaStreamSynchronize(g_stream));
    const int m = nt < kMaxTimed ? nt : kMaxTimed;
    for (int i = 0; i < m; i++)
      CC_CK(cudaEventElapsedTime(&g_last_ms[i], g_ev[i], g_ev[i + 1]));
    g_last_n = m;
    if (getenv("DCT_TIMING"))
      for (int i = 0; i < m; i++)
        fprintf(stderr, "DCT_TIMING transform(%d,%d) launch %d: %.4f ms\n",
                init_mode, out_mode, i, g_last_ms[i]);
  }
  return 0;
}

// CC_TUNE_LOG=1: every timed variant of the per-launch tuning on stderr
bool tune_log() {
  static const bool on = [] {
    const char *e = getenv("CC_TUNE_LOG");
    return e && atoi(e) == 1;
  }();
  return on;
}

// Per-launch tuning of plan P with its grouping fixed: every register block
// size, row width, prefetching form and CTA width of each launch, each
// timed alone (three launches after a warm one).  A launch run again works
// in place on its own planes, which only scrambles values; the real
// transform runs from scratch afterwards.
int tune_launches(Plan &P, int init_mode, int out_mode, cudaEvent_t e0,
                  cudaEvent_t e1) {
  // one transform with P: its code bounds (a recount's first group) and
  // planes are then the ones every variant below reads; the variants keep
  // the first group's tiles, so the bounds stay valid for all of them
  S.plans[init_mode][out_mode] = P;
  S.plan_ok[init_mode][out_mode] = true;
  int rc = run_transform(init_mode, out_mode);
  if (rc) return rc;
  int pm, pt;
  set_predicate(init_mode, &pm, &pt);
  for (size_t gi = 0; gi < P.groups.size(); gi++) {
    std::vector<GroupPlan> vars = group_variants(P.groups[gi], S.R1,
                                                 220 << 10);
    if (vars.size() < 2) continue;
    float bv = 1e30f;
    size_t bi = 0;
    for (size_t vi = 0; vi < vars.size(); vi++) {
      GroupPlan p = vars[vi];
      p.a.pmode = pm;
      p.a.ptarget = pt;
      p.a.mu = g_mu;
      p.a.code = S.d_code;
      p.a.ncode = S.codeM;
      p.a.code_bounds = S.d_bounds;
      if ((rc = prepare_group(p))) return rc;
      rc = launch_group(p, g_stream);
      if (rc == -9) { rc = 0; continue; }     // a form the launcher refused
      if (rc) return rc;
      CC_CK(cudaEventRecord(e0, g_stream));
      for (int r = 0; r < 3; r++)
        if ((rc = launch_group(p, g_stream))) return rc;
      CC_CK(cudaEventRecord(e1, g_stream));
      CC_CK(cudaEventSynchronize(e1));
      float ms = 0;
      CC_CK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < bv) { bv = ms; bi = vi; }
      if (tune_log())
        fprintf(stderr, "CC_TUNE_LOG transform(%d,%d) group %zu variant %zu: "
                "kernel %d tma %d stages %d W %d threads %d grid %d smem %zu "
                "pipe %d in8 %d out8 %d: %.4f ms\n", init_mode, out_mode, gi,
                vi, p.kernel, p.a.tma, p.a.stages, p.a.W, p.threads, p.grid,
                p.smem, p.a.pipe, p.a.in8, p.a.out8, ms / 3);
    }
    P.groups[gi] = vars[bi];
  }
  return 0;
}

// the axes, rows and prefetching of each launch: two knob settings that
// give the same grouping are tuned once
std::vector<long long> grouping_key(const Plan &P) {
  std::vector<long long> k;
  for (const auto &g : P.groups)
    k.push_back(((long long)g.a.k << 32) | (g.a.W << 8) | (g.a.pipe << 1) |
                g.a.pair_axis | ((g.a.pitch ? 1LL : 0LL) << 24) |
                ((long long)(g.a.in8 | g.a.out8) << 25));
  return k;
}

// Autotuner: on the first transform of a kind on a large cell, every
// distinct grouping the knob settings give (shared-memory budget x
// prefetching mode) gets its per-launch tuning, and then the whole tuned
// transform is timed (CUDA events on the engine stream, two runs after a
// warm one); the fastest is kept.  Every schedule computes the same
// integers, so tuning runs are ordinary transforms.  CC_TUNE=0 turns it
// off; explicit CC_PIPE / CC_SMEM_BUDGET_KB settings also pin the schedule.
int autotune(int init_mode, int out_mode) {
  if (S.streamed || S.tuned[init_mode][out_mode]) return 0;
  S.tuned[init_mode][out_mode] = true;
  const char *te = getenv("CC_TUNE");
  if ((te && atoi(te) == 0) || getenv("CC_PIPE") ||
      getenv("CC_SMEM_BUDGET_KB") || S.g.space < (1LL << 22) ||
      ((S.g.prob == kTorus || S.g.prob == kGrid) && any_wide_axis()))
    return 0;
  static const Knobs cands[] = {{100 << 10, 1}, {160 << 10, 1},
                                {64 << 10, 1}, {200 << 10, 1},
                                {100 << 10, 2}, {100 << 10, 3},
                                {200 << 10, 3}, {160 << 10, 2},
                                {200 << 10, 2},
                                // padded plans (ternary cells)
                                {64 << 10, 1, 0, 1, 1},
                                {100 << 10, 1, 0, 1, 1},
                                {160 << 10, 1, 0, 1, 1},
                                {200 << 10, 1, 0, 1, 1},
                                // 8-bit planes after the first group
                                {64 << 10, 1, 0, 1, 0, 1},
                                {100 << 10, 1, 0, 1, 0, 1},
                                {160 << 10, 1, 0, 1, 0, 1}};
  EventPair ev;
  int rc = ev.create();
  if (rc) return rc;
  cudaEvent_t e0 = ev.e0, e1 = ev.e1;
  float best = 1e30f;
  Plan keep;
  std::vector<std::vector<long long>> seen;
  for (const Knobs &kn : cands) {
    Plan P = make_plan(init_mode, out_mode, kn);
    if (P.window || P.groups.empty()) continue;
    const std::vector<long long> key = grouping_key(P);
    bool dup = false;
    for (const auto &k : seen) dup = dup || k == key;
    if (dup) continue;
    seen.push_back(key);
    if ((rc = tune_launches(P, init_mode, out_mode, e0, e1))) break;
    S.plans[init_mode][out_mode] = P;
    S.plan_ok[init_mode][out_mode] = true;
    if ((rc = run_transform(init_mode, out_mode))) break;      // warm
    CC_CK(cudaEventRecord(e0, g_stream));
    for (int r = 0; r < 2 && !rc; r++) rc = run_transform(init_mode, out_mode);
    if (rc) break;
    CC_CK(cudaEventRecord(e1, g_stream));
    CC_CK(cudaEventSynchronize(e1));
    float ms = 0;
    CC_CK(cudaEventElapsedTime(&ms, e0, e1));
    if (tune_log()) {
      fprintf(stderr, "CC_TUNE_LOG transform(%d,%d) plan budget %zu KB pipe "
              "%d pad %d u8 %d axes", init_mode, out_mode, kn.budget >> 10,
              kn.pipe, kn.pad, kn.u8);
      for (const auto &gp : P.groups)
        fprintf(stderr, " %d", gp.a.k + gp.a.pair_axis);
      fprintf(stderr, ": %.4f ms\n", ms / 2);
    }
    if (ms < best) { best = ms; keep = P; }
  }
  if (rc) return rc;
  if (!keep.groups.empty()) S.plans[init_mode][out_mode] = keep;
  else S.plans[init_mode][out_mode] = make_plan(init_mode, out_mode,
                                                default_knobs());
  S.plan_ok[init_mode][out_mode] = true;
  S.tune_ms[init_mode][out_mode] = best < 1e29f ? best / 2 : 0.f;
  return 0;
}

int ensure_stream() {
  if (!g_stream)
    CC_CK(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  return 0;
}

// v1 packed table -> SoA slots; -1 on malformed entries
int unpack_v1(const uint64_t *pat, long long len, std::vector<int32_t> &out,
              int *slots) {
  int w = 1;
  for (long long t = 0; t < len; t++) {
    int k = 0;
    while (k < 8 && ((pat[t] >> (8 * k)) & 255u)) k++;
    if (k > w) w = k;
  }
  out.assign((size_t)w * len, 0);
  for (long long t = 0; t < len; t++) {
    for (int k = 0; k < 8; k++) {
      const unsigned b = (unsigned)(pat[t] >> (8 * k)) & 255u;
      if (!b) break;
      const int pos = (int)(b >> 4), dl = (int)(b & 15u);
      if (pos >= S.g.n || dl < 1 || dl >= S.g.ax[pos]) return -1;
      out[(size_t)k * len + t] = (pos << 24) | dl;
    }
  }
  *slots = w;
  return 0;
}

int init_common(int problem, int n, const int *ax, int R, long long len,
                int extract_cap, int layers_mode, int cnt_mode,
                int use_owner) {
  if (n < 1 || n > kMaxAxes || R < 1 || !ax || len < 1 || len > INT_MAX ||
      extract_cap < 1)
    return -1;
  const bool layered = problem == kHamming || problem == kLee;
  if (problem < 0 || problem > 3) return -1;
  if (layered && R + 1 > kMaxLayers) return -1;
  for (int i = 0; i < n; i++) {
    if (ax[i] < 2 || ax[i] >= (1 << 24)) return -1;
    if (layered && ax[i] > 16) return -1;        // register / tile kernels
    if (problem == kTorus && (ax[i] < 3 || 2 * R + 1 > ax[i])) return -1;
  }
  long long space = 1;
  for (int i = 0; i < n; i++) {
    if (space > (1LL << 40) / ax[i]) return -2;
    space *= ax[i];
  }
  free_all();
  int rc = ensure_stream();
  if (rc) return rc;
  // coldcore's launch-size knob: 256 CTAs at least (dct_hc.cu:274-276)
  const char *bl = getenv("DCT_BLOCKS");
  g_dct_blocks = bl ? std::max(256, atoi(bl)) : 0;
  S.g.prob = problem; S.g.n = n; S.g.R = R; S.g.mu = g_mu;
  S.g.space = space;
  S.g.pw[0] = 1;
  for (int i = 0; i < n; i++) {
    S.g.ax[i] = ax[i];
    S.g.pw[i + 1] = S.g.pw[i] * ax[i];
  }
  S.R1 = layered ? R + 1 : 1;
  S.nplanes = layered ? R + 1 : 3;
  S.plane = round_up(space, kPlaneAlign);
  S.layers_mode = layers_mode;
  S.cnt_mode = cnt_mode;
  S.use_owner = use_owner;
  S.len = len;
  // layers_mode 1, the reference's host placement of the layer planes
  // (dctcore_core.cuh:86-119): pinned host planes streamed through the
  // device (cells with a two-phase split, i.e. group-transform cells of
  // two or more axes); otherwise, and for mode 2, managed planes
  bool wide = false;
  for (int i = 0; i < n; i++) wide = wide || ax[i] > 16;
  S.streamed = layers_mode == 1 && n >= 2 && !wide;
  if (S.streamed) {
    if (dev_alloc((void **)&S.layers, (size_t)S.plane * 4, 0)) {
      free_all(); return -3;
    }
    S.h_layers_bytes = (long long)S.R1 * space * 4;
    if (cudaHostAlloc((void **)&S.h_layers, (size_t)S.h_layers_bytes,
                      cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      S.h_layers = nullptr;
      fprintf(stderr, "coldcore_b200: pinned host planes of %lld bytes "
              "failed\n", S.h_layers_bytes);
      free_all(); return -3;
    }
    S.bytes_host += S.h_layers_bytes;
  } else if (dev_alloc((void **)&S.layers, (size_t)S.plane * S.nplanes * 4,
                       layers_mode)) { free_all(); return -3; }
  S.cnt_len = round_up(space, kPlaneAlign);
  if (dev_alloc((void **)&S.cnt, (size_t)S.cnt_len * 2, cnt_mode)) {
    free_all(); return -4;
  }
  CC_CK(cudaMemsetAsync(S.cnt, 0, (size_t)S.cnt_len * 2, g_stream));
  if (use_owner) {
    if (dev_alloc((void **)&S.owner, (size_t)space * 4, cnt_mode)) {
      free_all(); return -5;
    }
  }
  CC_CK(cudaMalloc(&S.d_words, kStageCap * 8));
  CC_CK(cudaMalloc(&S.d_out, kStageCap * 4));
  CC_CK(cudaMalloc(&S.d_scalar, 64 * 8));
  CC_CK(cudaMalloc(&S.d_hist, 4096 * 4));
  CC_CK(cudaHostAlloc((void **)&S.h_words, kStageCap * 8,
                      cudaHostAllocDefault));
  CC_CK(cudaHostAlloc((void **)&S.h_out, kStageCap * 4,
                      cudaHostAllocDefault));
  CC_CK(cudaHostAlloc((void **)&S.h_scalar, 64 * 8, cudaHostAllocDefault));
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 64 * 8, g_stream));
  S.bytes_dev += kStageCap * 12 + 64 * 8 + 4096 * 4;
  S.extract_cap = extract_cap;
  CC_CK(cudaMalloc(&S.d_ext32, (size_t)extract_cap * 4));
  CC_CK(cudaMalloc(&S.d_ext64, (size_t)extract_cap * 8));
  CC_CK(cudaMalloc(&S.d_extv, (size_t)extract_cap * 4));
  S.bytes_dev += (long long)extract_cap * 16;
  S.mult_hist.assign(kCounterMax + 2, 0);
  S.live = true;
  return 0;
}

int upload_table(const std::vector<int32_t> &soa, int slots, int32_t **dst,
                 int *dslots) {
  CC_CK(cudaMalloc(dst, soa.size() * 4));
  CC_CK(cudaMemcpyAsync(*dst, soa.data(), soa.size() * 4,
                        cudaMemcpyHostToDevice, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  S.bytes_dev += (long long)soa.size() * 4;
  *dslots = slots;
  return 0;
}

int finish_init(long long *bytes) {
  CC_CK(cudaStreamSynchronize(g_stream));
  if (bytes) *bytes = S.bytes_dev + S.bytes_host;
  return 0;
}

// Is the support table exactly the metric ball?  Every pattern must move
// distinct axes by admissible deltas within radius R, the patterns must be
// distinct, and their number must equal the ball's cardinality (coldcore
// dct_hc.cu:158-204 states the same test).  Only then may a gather count
// listed words by distance instead of walking the table.
bool table_is_ball(const std::vector<int32_t> &soa, int slots, long long len) {
  const int n = S.g.n, R = S.g.R, prob = S.g.prob;
  if (n > 16) return false;
  for (int i = 0; i < n; i++)
    if (S.g.ax[i] > 16) return false;
  auto weight = [&](int pos, int d) -> int {      // -1: inadmissible
    const int a = S.g.ax[pos];
    if (d < 1 || d >= a) return -1;
    const int c = std::min(d, a - d);
    if (prob == kHamming) return 1;
    if (prob == kLee) return c <= R ? c : -1;
    return c <= R ? 0 : -1;                        // L-infinity
  };
  std::vector<unsigned long long> keys;
  keys.reserve((size_t)len);
  for (long long t = 0; t < len; t++) {
    unsigned seen = 0;
    unsigned long long key = 0;
    int w = 0;
    for (int k = 0; k < slots; k++) {
      const int32_t c = soa[(size_t)k * len + t];
      if (!c) continue;
      const int pos = c >> 24, d = c & 0xFFFFFF;
      if (pos >= n || ((seen >> pos) & 1u)) return false;
      seen |= 1u << pos;
      const int e = weight(pos, d);
      if (e < 0) return false;
      w += e;
      key |= (unsigned long long)d << (4 * pos);
    }
    if (w > R) return false;
    keys.push_back(key);
  }
  std::sort(keys.begin(), keys.end());
  if (std::adjacent_find(keys.begin(), keys.end()) != keys.end()) return false;
  // cardinality: coefficients 0..W of prod_i (1 + sum_d t^weight(i, d))
  const int W = (prob == kHamming || prob == kLee) ? R : 0;
  std::vector<long double> poly(W + 1, 0.0L);
  poly[0] = 1.0L;
  for (int i = 0; i < n; i++) {
    std::vector<long double> nx(W + 1, 0.0L);
    for (int w = 0; w <= W; w++) {
      if (poly[w] == 0) continue;
      nx[w] += poly[w];
      for (int d = 1; d < S.g.ax[i]; d++) {
        const int e = weight(i, d);
        if (e >= 0 && w + e <= W) nx[w + e] += poly[w];
      }
    }
    poly.swap(nx);
  }
  long double tot = 0;
  for (int w = 0; w <= W; w++) tot += poly[w];
  return tot == (long double)len;
}

void set_side_init(const std::vector<int32_t> &soa, int slots) {
  const char *sp = getenv("DCT_SET_GATHER");
  const char *sm = getenv("DCT_SET_MIN");
  const char *sr = getenv("DCT_SET_RATIO");
  S.set_policy = sp ? atoi(sp) : 1;
  S.set_min = sm ? atoll(sm) : -1;
  S.set_ratio = sr ? std::max(1LL, atoll(sr)) : 2;
  S.set_ok = S.set_policy != 0 && table_is_ball(soa, slots, S.len);
  S.zcap_max = std::min<long long>(S.g.space, 1LL << 27);
  S.z_mode = -1;
}

// the walk of nb candidates reads nb*|B| counters: worth trying the list?
bool want_set(int mode, int target, int nb) {
  if (!S.set_ok || !(mode == kPredDef || (mode == kPredEq && target == 0)))
    return false;
  if (S.set_policy == 2) return true;
  const long long walk = (long long)nb * S.len;
  const long long lim = S.set_min >= 0 ? S.set_min
                        : std::max<long long>(S.g.space / 8, 1LL << 21);
  return walk >= lim;
}

// List Z = {x : pred(cnt[x])} for the current cnt, unless it is listed
// already.  Returns 1 when the list is usable (|Z| <= ratio*|B|), 0 when
// the caller must walk, negative on error.
int ensure_zlist(int mode, int target) {
  if (S.z_mode == mode && S.z_target == target && S.z_mu == g_mu &&
      S.z_ver == S.cnt_ver)
    return S.z_valid ? 1 : 0;
  const long long lim = std::min(S.len * S.set_ratio, S.zcap_max);
  if (!S.d_found) CC_CK(cudaMalloc(&S.d_found, 8));
  long long want = std::min<long long>(std::max<long long>(S.len / 4, 4096),
                                       1LL << 22);
  want = std::min(want, lim);
  for (;;) {
    if (S.zcap < want) {
      if (S.zbuf) CC_CK(cudaFree(S.zbuf));
      S.zbuf = nullptr;
      S.zcap = 0;
      CC_CK(cudaMalloc(&S.zbuf, (size_t)want * 8));
      S.zcap = want;
    }
    Geometry g = S.g;
    g.mu = g_mu;
    int rc = launch_list_pred(g, S.cnt, mode, target, S.zbuf, S.zcap,
                              S.d_found, g_stream);
    if (rc) return rc;
    CC_CK(cudaMemcpyAsync(S.h_scalar + 8, S.d_found, 8,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    const long long found = S.h_scalar[8];
    S.stats[2]++;
    if (found > S.zcap && found <= lim) { want = found; continue; }
    S.z_mode = mode; S.z_target = target; S.z_mu = g_mu;
    S.z_ver = S.cnt_ver;
    S.z_n = found;
    S.z_valid = found <= lim;
    if (!S.z_valid) S.stats[3]++;
    return S.z_valid ? 1 : 0;
  }
}

// launch the gather of nb staged words into dout (set side or walk)
int gather_launch(int mode, int target, int nb, const long long *dw,
                  int32_t *dout, bool zeroed) {
  const int zs = want_set(mode, target, nb) ? ensure_zlist(mode, target) : 0;
  if (zs < 0) return zs;
  if (zs == 1) {
    S.stats[0]++;
    if (S.z_n > 32768) S.stats[7]++;
    Geometry g = S.g;
    g.mu = g_mu;
    return launch_gather_set(g, dw, nb, S.zbuf, S.z_n, dout, zeroed,
                             g_stream);
  }
  S.stats[1]++;
  const WalkArgs wa = walk_args();
  uint8_t *bits = nullptr;
  if (gather_bits_pay(wa, nb)) {
    if (!S.d_bits)
      CC_CK(cudaMalloc(&S.d_bits, (size_t)((S.g.space + 7) / 8 + 16)));
    bits = S.d_bits;
  }
  return launch_gather(wa, dw, nb, mode, target, dout, zeroed, g_stream,
                       bits);
}

int gather_impl(const long long *words, int nwords, int mode, int target,
                int32_t *out) {
  if (nwords <= 0) return 0;
  if (!out || !valid_words(words, nwords)) return -1;
  for (long long off = 0; off < nwords; off += kStageCap) {
    const int nb = (int)std::min<long long>(kStageCap, nwords - off);
    int rc = stage_words(words + off, nb);
    if (rc) return rc;
    rc = gather_launch(mode, target, nb, S.d_words, S.d_out, false);
    if (rc) return rc;
    CC_CK(cudaMemcpyAsync(S.h_out, S.d_out, (size_t)nb * 4,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(out + off, S.h_out, (size_t)nb * 4);
  }
  return 0;
}

// cnt += delta over the balls of `words`; trans: running transition counter
int update_impl(const long long *words, int nwords, int delta,
                unsigned long long *trans) {
  const WalkArgs w = walk_args();
  S.cnt_ver++;
  for (long long off = 0; off < nwords; off += kStageCap) {
    const int nb = (int)std::min<long long>(kStageCap, nwords - off);
    int rc;
    if (nb <= kParamWords) {
      WordsParam p;
      memcpy(p.w, words + off, (size_t)nb * 8);
      rc = launch_update(w, nullptr, &p, nb, delta, trans, g_stream);
      if (rc) return rc;
    } else {
      rc = stage_words(words + off, nb);
      if (rc) return rc;
      rc = launch_update(w, S.d_words, nullptr, nb, delta, trans, g_stream);
      if (rc) return rc;
      CC_CK(cudaStreamSynchronize(g_stream));   // staging buffer reused
    }
  }
  return 0;
}

int mode_role(int role, int *mode, int *target) {
  if (role == 0) { *mode = g_mu == 1 ? kPredEq : kPredDef; *target = 0; }
  else { *mode = g_mu == 1 ? kPredEq : kPredCrit; *target = 1; }
  return 0;
}

}  // namespace

extern "C" {

long long dct_host_bytes(void) { return S.bytes_host; }

int dct_set_mu(int mu) {
  if (mu < 1 || mu > 65535) return -1;
  g_mu = mu;
  S.g.mu = mu;
  return 0;
}

int dct_get_mu(void) { return g_mu; }

int dct_init3(int problem, int n, const int *ax, int R,
              const uint64_t *ballpat, long long balllen, int extract_cap,
              long long *bytes, int layers_mode, int cnt_mode,
              int use_owner) {
  // the v1 table packs position and delta in one nibble each: n <= 16,
  // axes <= 16 (wider cells use dct_init3w)
  if (!ballpat || !ax || n < 1 || n > 16) return -1;
  for (int i = 0; i < n; i++)
    if (ax[i] < 2 || ax[i] > 16) return -1;
  if (layers_mode < 0 || layers_mode > 2 || cnt_mode < 0 || cnt_mode > 2)
    return -1;
  int rc = init_common(problem, n, ax, R, balllen, extract_cap, layers_mode,
                       cnt_mode, use_owner);
  if (rc) return rc;
  std::vector<int32_t> soa;
  int slots = 0;
  if (unpack_v1(ballpat, balllen, soa, &slots)) { free_all(); return -1; }
  rc = upload_table(soa, slots, &S.tbl, &S.slots);
  if (rc) return rc;
  set_side_init(soa, slots);
  return finish_init(bytes);
}

int dct_init3w(int problem, int n, const int *ax, int R, const int32_t *tbl,
               int slots, long long len, int extract_cap, long long *bytes) {
  return dct_b200_init3wm(problem, n, ax, R, tbl, slots, len, extract_cap,
                          bytes, 0, 0);
}

int dct_b200_init3wm(int problem, int n, const int *ax, int R,
                     const int32_t *tbl, int slots, long long len,
                     int extract_cap, long long *bytes, int layers_mode,
                     int cnt_mode) {
  if (!tbl || slots < 1 || slots > kMaxSlots) return -1;
  if (layers_mode < 0 || layers_mode > 2 || cnt_mode < 0 || cnt_mode > 2)
    return -1;
  int rc = init_common(problem, n, ax, R, len, extract_cap, layers_mode,
                       cnt_mode, 0);
  if (rc) return rc;
  std::vector<int32_t> soa((size_t)slots * len, 0);
  for (long long t = 0; t < len; t++)
    for (int k = 0; k < slots; k++) {
      const int32_t c = tbl[t * slots + k];
      if (!c) continue;
      const int pos = c >> 24, dl = c & 0xFFFFFF;
      if (pos < 0 || pos >= n || dl < 1 || dl >= ax[pos]) {
        free_all();
        return -1;
      }
      soa[(size_t)k * len + t] = c;
    }
  rc = upload_table(soa, slots, &S.tbl, &S.slots);
  if (rc) return rc;
  set_side_init(soa, slots);
  return finish_init(bytes);
}

int dct_init2(int q, int n, int R, const uint64_t *ballpat, long long balllen,
              int extract_cap, long long *bytes, int layers_mode,
              int cnt_mode, int use_owner) {
  int ax[kMaxAxes];
  if (n < 1 || n > kMaxAxes) return -1;
  for (int i = 0; i < n; i++) ax[i] = q;
  return dct_init3(kHamming, n, ax, R, ballpat, balllen, extract_cap, bytes,
                   layers_mode, cnt_mode, use_owner);
}

int dct_init(int q, int n, int R, const uint64_t *ballpat, long long balllen,
             int extract_cap, long long *bytes) {
  return dct_init2(q, n, R, ballpat, balllen, extract_cap, bytes, 0, 0, 0);
}

int dct_free(void) {
  free_all();
  g_mu = 1;                       // singleton: mu never leaks into a new cell
  return 0;
}

int dct_set_tbl2(const uint16_t *mask, const uint64_t *offs, long long len) {
  if (!S.live || len != S.len || !mask || !offs) return -1;
  int w = 1;
  for (long long t = 0; t < len; t++) w = std::max(w, __builtin_popcount(mask[t]));
  std::vector<int32_t> soa((size_t)w * len, 0);
  for (long long t = 0; t < len; t++) {
    unsigned m = mask[t];
    int k = 0;
    while (m) {
      const int p = __builtin_ctz(m);
      m &= m - 1;
      const int dl = (int)((offs[t] >> (4 * p)) & 15u);
      if (p >= S.g.n || dl < 1 || dl >= S.g.ax[p]) return -1;
      soa[(size_t)k * len + t] = (p << 24) | dl;
      k++;
    }
  }
  if (S.tbl2) { cudaFree(S.tbl2); S.tbl2 = nullptr; }
  return upload_table(soa, w, &S.tbl2, &S.slots2);
}

int dct_use_fmt(int fmt) {
  if (fmt < 0 || fmt > 1) return -1;
  if (fmt == 1 && !S.tbl2) return -1;
  if (fmt == 1 && S.g.prob == kGrid) return -1;   // the ox walk is circulant
  S.fmt = fmt;
  return 0;
}

int dct_set_code(const long long *idx, int M) {
  if (!S.live || !valid_words(idx, M)) return -1;
  std::vector<long long> sorted(idx, idx + M);
  if (!std::is_sorted(sorted.begin(), sorted.end()))
    std::sort(sorted.begin(), sorted.end());
  int mx = 0;                                  // largest multiplicity
  for (int i = 0; i < M;) {
    int j = i + 1;
    while (j < M && sorted[j] == sorted[i]) j++;
    mx = std::max(mx, j - i);
    i = j;
  }
  if (!within_counter(M, mx)) return -1;
  if (M > S.code_cap) {
    if (S.d_code) cudaFree(S.d_code);
    S.d_code = nullptr;
    const long long cap = std::max<long long>(M, 1024);
    CC_CK(cudaMalloc(&S.d_code, (size_t)cap * 8));
    S.code_cap = cap;
  }
  if (M) {
    CC_CK(cudaMemcpyAsync(S.d_code, sorted.data(), (size_t)M * 8,
                          cudaMemcpyHostToDevice, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
  }
  S.codeM = M;
  S.up_sorted.swap(sorted);
  S.up_max = mx;
  return 0;
}

int dct_transform(int init_mode, int out_mode) {
  if (!S.live) return -1;
  if (init_mode < 0 || init_mode > 2 || out_mode < 1 || out_mode > 3 ||
      (out_mode == 2 && init_mode != 0))
    return -1;
  if (out_mode == 3 && S.R1 == 1) return -1;
  int rc = autotune(init_mode, out_mode);
  if (rc) return rc;
  rc = run_transform(init_mode, out_mode);
  if (rc) return rc;
  CC_CK(cudaStreamSynchronize(g_stream));
  S.layered_out = out_mode == 3;
  if (out_mode == 2) {
    // active = uploaded; its size and largest multiplicity now, the
    // per-word counts when a call needs them
    S.active_pending = true;
    S.active_size = S.codeM;
    S.act_max = S.up_max;
    S.cnt_ver++;
  }
  return 0;
}

int dct_ball_update(const long long *words, int nwords, int delta) {
  if (!S.live) return -1;
  std::unordered_map<long long, int> batch;
  if (check_update(words, nwords, delta, batch)) return -1;
  if (nwords == 0) return 0;
  int rc = update_impl(words, nwords, delta, nullptr);
  if (rc) return rc;
  apply_active(batch, delta, nwords);
  return 0;
}

int dct_ball_update_delta(const long long *words, int nwords, int delta,
                          long long *dd) {
  if (!dd) return -1;
  *dd = 0;
  if (!S.live) return -1;
  std::unordered_map<long long, int> batch;
  if (check_update(words, nwords, delta, batch)) return -1;
  if (nwords == 0) return 0;
  auto *trans = reinterpret_cast<unsigned long long *>(S.d_scalar + 2);
  int rc = update_impl(words, nwords, delta, trans);
  if (rc) return rc;
  long long now;
  rc = fetch_scalar(&now, 2);
  if (rc) return rc;
  const long long tr = (long long)((unsigned long long)now - S.dd_last);
  S.dd_last = (unsigned long long)now;
  *dd = delta > 0 ? -tr : tr;
  apply_active(batch, delta, nwords);
  return 0;
}

int dct_ball_gather(const long long *words, int nwords, int target,
                    int32_t *out) {
  if (!S.live) return -1;
  return gather_impl(words, nwords, kPredEq, target, out);
}

int dct_ball_gather_mu(const long long *words, int nwords, int role,
                       int32_t *out) {
  if (!S.live) return -1;
  if (nwords <= 0) return 0;
  if (role < 0 || role > 1) return -1;
  return gather_impl(words, nwords, role == 0 ? kPredDef : kPredCrit, 0, out);
}

// Read-only swap evaluation with one synchronisation (coldcore
// dct_hc.cu:882-963): loss[i] and the list of drop i's ball words at exactly
// mu come from two walks of its ball; gain[j] is the role-0 gather of cand j
// on the current cnt (set side or walk) plus the listed words of its drop
// within distance R, the words that removing the drop makes deficient.
// Returns 1 when the list overflowed (the caller falls back), else 0 or an
// error code.
int swap_eval_fast(const long long *drops, int k, const long long *cand,
                   const long long *off, int32_t *gain, int32_t *loss) {
  constexpr long long kMaxN = 65536;
  // staging: [cand kMaxN x 8][drops kMaxN x 8][coff (kMaxN + 1) x 4]
  // results: [gain kMaxN x 4][loss kMaxN x 4][nmu x 4][offs (+1) x 4]
  //          [cursor x 4]
  const size_t in_drop = kMaxN * 8, in_coff = 2 * kMaxN * 8;
  const size_t in_bytes = in_coff + (kMaxN + 1) * 4;
  const size_t r0 = in_bytes + 64;           // results start, 16-aligned
  const size_t r_loss = r0 + kMaxN * 4, r_nmu = r_loss + kMaxN * 4;
  const size_t r_offs = r_nmu + kMaxN * 4, r_cur = r_offs + (kMaxN + 1) * 4;
  const size_t total_bytes = r_cur + kMaxN * 4 + 64;
  if (!S.d_swap) {
    CC_CK(cudaMalloc(&S.d_swap, total_bytes));
    CC_CK(cudaHostAlloc((void **)&S.h_swap, total_bytes,
                        cudaHostAllocDefault));
    S.lcap = std::min<long long>(std::max<long long>(4 * S.len, 1 << 16),
                                 1LL << 22);
    CC_CK(cudaMalloc(&S.d_list, (size_t)S.lcap * 8));
  }
  const long long nc = off[k];
  char *h = S.h_swap, *d = S.d_swap;
  if (nc) memcpy(h, cand, (size_t)nc * 8);
  memcpy(h + in_drop, drops, (size_t)k * 8);
  int32_t *hc = reinterpret_cast<int32_t *>(h + in_coff);
  for (int i = 0; i <= k; i++) hc[i] = (int32_t)off[i];
  const long long *d_cand = reinterpret_cast<const long long *>(d);
  const long long *d_drop = reinterpret_cast<const long long *>(d + in_drop);
  const int32_t *d_coff = reinterpret_cast<const int32_t *>(d + in_coff);
  int32_t *d_gain = reinterpret_cast<int32_t *>(d + r0);
  int32_t *d_loss = reinterpret_cast<int32_t *>(d + r_loss);
  int32_t *d_nmu = reinterpret_cast<int32_t *>(d + r_nmu);
  int32_t *d_offs = reinterpret_cast<int32_t *>(d + r_offs);
  int32_t *d_cur = reinterpret_cast<int32_t *>(d + r_cur);
  CC_CK(cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, g_stream));
  CC_CK(cudaMemsetAsync(d + r0, 0, r_offs - r0, g_stream));
  WalkArgs w = walk_args();
  int rc = launch_drop_walks(w, d_drop, k, d_loss, d_nmu, d_offs, d_cur,
                             S.lcap, S.d_list, g_stream);
  if (rc) return rc;
  if (nc) {
    int gm, gt;
    mode_role(0, &gm, &gt);
    rc = gather_launch(gm, gt, (int)nc, d_cand, d_gain, true);
    if (rc) return rc;
    Geometry g = S.g;
    g.mu = g_mu;
    rc = launch_swap_corr(g, k, d_cand, d_coff, d_offs, S.d_list, S.lcap,
                          d_gain, g_stream);
    if (rc) return rc;
  }
  // gain, loss and the list total (offs[k]) in one copy
  CC_CK(cudaMemcpyAsync(h + r0, d + r0, r_offs - r0 + (size_t)(k + 1) * 4,
                        cudaMemcpyDeviceToHost, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  const int32_t listed = reinterpret_cast<int32_t *>(h + r_offs)[k];
  if (listed > S.lcap) return 1;
  memcpy(loss, h + r_loss, (size_t)k * 4);
  if (nc) memcpy(gain, h + r0, (size_t)nc * 4);
  S.stats[4]++;
  return 0;
}

// Exact greedy repair on the device (no counterpart in the reference; its
// greedy_fill is the Python lazy greedy of search.py:260-360).  From the
// gain map of the current cnt, with the active words excluded, each
// step places the word of largest exact gain (ties: smallest index),
// updates cnt over its ball and lowers the gain of every candidate whose
// ball holds a word the placement satisfied, all without leaving the GPU;
// it stops at zero deficit, at no positive gain, or after max_add words.
// The placed words are added to the active multiset.  placed (capacity
// max_add) receives them in placement order; *deficit the deficit left.
// Returns the number placed, or a negative error.  The map is clobbered.
int greedy_fill_impl(int max_add, long long *placed, long long *deficit) {
  if (!S.live || max_add < 0 || (max_add && !placed) || !deficit) return -1;
  if (S.g.space >= (1LL << 32)) return -1;    // 32-bit index in the key
  ensure_active();
  // placed words are new (multiplicity 1): the counters stay within uint16
  if (!within_counter(S.active_size + max_add, std::max(S.act_max, 1)))
    return -1;
  std::vector<long long> code;
  code.reserve(S.active.size());
  for (const auto &e : S.active) code.push_back(e.first);
  const long long M = (long long)code.size();
  if (!S.d_greedy) {
    CC_CK(cudaMalloc(&S.d_greedy, kGreedyStateBytes));
    CC_CK(cudaMalloc(&S.d_fresh, (size_t)S.len * 8));
  }
  if (max_add > S.placed_cap) {
    if (S.d_placed) CC_CK(cudaFree(S.d_placed));
    if (S.h_placed) CC_CK(cudaFreeHost(S.h_placed));
    S.d_placed = S.h_placed = nullptr;
    S.placed_cap = 0;
    const long long cap = std::max<long long>(max_add, 1024);
    CC_CK(cudaMalloc(&S.d_placed, (size_t)cap * 8));
    CC_CK(cudaHostAlloc((void **)&S.h_placed, (size_t)cap * 8,
                        cudaHostAllocDefault));
    S.placed_cap = cap;
  }
  // the deficit to start from, and the gain map of the current cnt
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 8, g_stream));
  int rc = launch_cnt_reduce(S.cnt, S.g.space, kPredDef, 0, g_mu,
                             S.d_scalar, g_stream);
  if (rc) return rc;
  long long d0;
  rc = fetch_scalar(&d0);
  if (rc) return rc;
  *deficit = d0;
  if (max_add == 0 || d0 == 0) return 0;
  rc = autotune(1, 1);
  if (rc) return rc;
  rc = run_transform(1, 1);
  if (rc) return rc;
  S.layered_out = false;
  constexpr int32_t kExcluded = INT_MIN / 2;
  for (long long off = 0; off < M; off += kStageCap) {
    const int nb = (int)std::min<long long>(kStageCap, M - off);
    rc = stage_words(code.data() + off, nb);
    if (rc) return rc;
    rc = launch_greedy_exclude(S.layers, S.d_words, nb, kExcluded, g_stream);
    if (rc) return rc;
    CC_CK(cudaStreamSynchronize(g_stream));     // staging buffer reused
  }
  struct { unsigned long long best; long long deficit; int done, placed,
           nnew, pad; } st0 = {0, d0, 0, 0, 0, 0};
  static_assert(sizeof(st0) == kGreedyStateBytes, "state layout");
  CC_CK(cudaMemcpyAsync(S.d_greedy, &st0, sizeof(st0),
                        cudaMemcpyHostToDevice, g_stream));
  const WalkArgs w = walk_args();
  GreedyState *st = reinterpret_cast<GreedyState *>(S.d_greedy);
  // every placement serves at least one deficient word: at most d0 steps.
  // Steps go out in chunks (32, 64, ... 512) with one look at the state
  // between chunks; steps after the stop are no-ops on the device.
  const long long steps = std::min<long long>(max_add, d0);
  long long issued = 0, chunk = 32;
  while (issued < steps) {
    const long long n = std::min(chunk, steps - issued);
    for (long long i = 0; i < n; i++) {
      rc = launch_greedy_step(w, S.layers, S.g.space, st, S.d_placed,
                              max_add, S.d_fresh, kExcluded, g_stream);
      if (rc) return rc;
    }
    issued += n;
    CC_CK(cudaMemcpyAsync(S.h_scalar + 16, S.d_greedy, sizeof(st0),
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(&st0, S.h_scalar + 16, sizeof(st0));
    if (st0.done) break;
    chunk = std::min<long long>(chunk * 2, 512);
  }
  const int n = st0.placed;
  if (n) {
    CC_CK(cudaMemcpyAsync(S.h_placed, S.d_placed, (size_t)n * 8,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(placed, S.h_placed, (size_t)n * 8);
    std::unordered_map<long long, int> batch;
    for (int i = 0; i < n; i++) ++batch[placed[i]];
    apply_active(batch, +1, n);
  }
  S.cnt_ver++;
  *deficit = st0.deficit;
  return n;
}

int dct_b200_greedy_fill(int max_add, long long *placed, long long *deficit) {
  return greedy_fill_impl(max_add, placed, deficit);
}

int dct_swap_eval(const long long *drops, int k, const long long *cand,
                  const long long *off, int32_t *gain, int32_t *loss) {
  if (!S.live) return -1;
  if (k <= 0) return 0;
  if (k > 65535 || !off || off[0] != 0 || !drops || !loss) return -1;
  for (int i = 0; i < k; i++)
    if (off[i + 1] < off[i]) return -1;
  const long long nc = off[k];
  if (nc > 65535 || (nc && (!cand || !gain))) return -1;
  if (!valid_words(drops, k) || !valid_words(cand, nc)) return -1;
  ensure_active();
  for (int i = 0; i < k; i++)
    if (S.active.find(drops[i]) == S.active.end()) return -1;
  if (S.set_ok) {
    const int rc = swap_eval_fast(drops, k, cand, off, gain, loss);
    if (rc <= 0) return rc;                  // done (0) or an error
  }
  // drop / gather / undo per drop word; cnt ends where it started
  S.stats[5]++;
  int lm, lt, gm, gt;
  mode_role(1, &lm, &lt);
  mode_role(0, &gm, &gt);
  for (int i = 0; i < k; i++) {
    int rc = gather_impl(drops + i, 1, lm, lt, loss + i);
    if (rc) return rc;
    const long long ni = off[i + 1] - off[i];
    if (!ni) continue;
    rc = update_impl(drops + i, 1, -1, nullptr);
    if (rc) return rc;
    rc = gather_impl(cand + off[i], (int)ni, gm, gt, gain + off[i]);
    const int rc2 = update_impl(drops + i, 1, +1, nullptr);
    if (rc) return rc;
    if (rc2) return rc2;
  }
  return 0;
}

int dct_loss_owner(const long long *words, int M, int32_t *out) {
  if (!S.live || !S.owner) return -1;
  if (!valid_words(words, M) || (M && !out)) return -2;
  std::unordered_map<long long, int> ms;
  int mx = 0;
  for (int i = 0; i < M; i++) mx = std::max(mx, ++ms[words[i]]);
  if (!within_counter(M, mx)) return -2;
  CC_CK(cudaMemsetAsync(S.cnt, 0, (size_t)S.cnt_len * 2, g_stream));
  int rc = update_impl(words, M, +1, nullptr);
  if (rc) return rc;
  set_active(ms, M);
  if (M == 0) return 0;
  int lm, lt;
  mode_role(1, &lm, &lt);
  return gather_impl(words, M, lm, lt, out);
}

int dct_stats(long long *out, int n) {
  if (n > 8) n = 8;
  for (int i = 0; i < n; i++) out[i] = S.stats[i];
  return n < 0 ? 0 : n;
}

long long dct_count_eq(int target) {
  if (!S.live) return -1;
  // the zero-word list of a set-side gather already counted them
  if (target == 0 && S.z_valid && S.z_ver == S.cnt_ver &&
      (S.z_mode == kPredEq ? S.z_target == 0
                           : (S.z_mode == kPredDef && S.z_mu == 1))) {
    S.stats[6]++;
    return S.z_n;
  }
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 8, g_stream));
  int rc = launch_cnt_reduce(S.cnt, S.g.space, kPredEq, target, g_mu,
                             S.d_scalar, g_stream);
  if (rc) return rc;
  long long r;
  rc = fetch_scalar(&r);
  return rc ? rc : r;
}

long long dct_count_deficit(void) {
  if (!S.live) return -1;
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 8, g_stream));
  int rc = launch_cnt_reduce(S.cnt, S.g.space, kPredDef, 0, g_mu, S.d_scalar,
                             g_stream);
  if (rc) return rc;
  long long r;
  rc = fetch_scalar(&r);
  return rc ? rc : r;
}

int dct_map_max(int32_t *out) {
  if (!S.live || !out) return -1;
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 8, g_stream));
  int rc = launch_max(S.layers, S.g.space, S.d_scalar, g_stream);
  if (rc) return rc;
  long long r;
  rc = fetch_scalar(&r);
  if (rc) return rc;
  *out = (int32_t)r;
  return 0;
}

int dct_map_hist(int nbins, int32_t vmax, int32_t *out) {
  if (!S.live || nbins < 1 || nbins > 4096 || vmax < 1 || !out) return -1;
  CC_CK(cudaMemsetAsync(S.d_hist, 0, (size_t)nbins * 4, g_stream));
  int rc = launch_hist(S.layers, S.g.space, nbins, vmax, S.d_hist, g_stream);
  if (rc) return rc;
  CC_CK(cudaMemcpyAsync(S.h_out, S.d_hist, (size_t)nbins * 4,
                        cudaMemcpyDeviceToHost, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  memcpy(out, S.h_out, (size_t)nbins * 4);
  return 0;
}

static long long extract_impl(int32_t thr, void *out_idx, bool wide,
                              int32_t *out_val, int cap) {
  if (!S.live) return -1;
  if (cap > S.extract_cap) cap = (int)S.extract_cap;
  if (cap < 0) cap = 0;
  CC_CK(cudaMemsetAsync(S.d_scalar, 0, 8, g_stream));
  void *didx = wide ? (void *)S.d_ext64 : (void *)S.d_ext32;
  int rc = launch_extract(S.layers, S.g.space, thr, didx, wide, S.d_extv, cap,
                          S.d_scalar, g_stream);
  if (rc) return rc;
  long long found;
  rc = fetch_scalar(&found);
  if (rc) return rc;
  const long long m = found < cap ? found : cap;
  if (m > 0) {
    CC_CK(cudaMemcpyAsync(out_idx, didx, (size_t)m * (wide ? 8 : 4),
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaMemcpyAsync(out_val, S.d_extv, (size_t)m * 4,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
  }
  return found;
}

long long dct_map_extract(int32_t thr, uint32_t *idx, int32_t *val, int cap) {
  return extract_impl(thr, idx, false, val, cap);
}

long long dct_map_extract64(int32_t thr, int64_t *idx, int32_t *val,
                            int cap) {
  return extract_impl(thr, idx, true, val, cap);
}

int dct_map_read_at(const long long *idx, int k, int32_t *out) {
  if (!S.live) return -1;
  if (k <= 0) return 0;
  if (!out || !valid_words(idx, k)) return -1;
  for (long long off = 0; off < k; off += kStageCap) {
    const int nb = (int)std::min<long long>(kStageCap, k - off);
    int rc = stage_words(idx + off, nb);
    if (rc) return rc;
    rc = launch_read_at(S.layers, S.d_words, nb, S.d_out, g_stream);
    if (rc) return rc;
    CC_CK(cudaMemcpyAsync(S.h_out, S.d_out, (size_t)nb * 4,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(out + off, S.h_out, (size_t)nb * 4);
  }
  return 0;
}

int dct_read_cnt(long long off, long long len, uint16_t *out) {
  if (!S.live || off < 0 || len < 0 || off + len > S.g.space ||
      (len && !out))
    return -1;
  if (len)
    CC_CK(cudaMemcpyAsync(out, S.cnt + off, (size_t)len * 2,
                          cudaMemcpyDefault, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));   // async updates were in flight
  return 0;
}

long long dct_b200_stream(void) {
  if (ensure_stream()) return 0;
  return (long long)(uintptr_t)g_stream;
}

int dct_b200_plan(int init_mode, int out_mode, long long *info, int cap) {
  // a streamed cell runs the out-of-core schedule (dct_b200_ooc_plan)
  if (!S.live || S.streamed || init_mode < 0 || init_mode > 2 ||
      out_mode < 1 || out_mode > 3)
    return -1;
  Plan &P = plan_for(init_mode, out_mode);
  const long long X = S.g.space;
  int n = 0;
  if (P.window) {
    for (size_t i = 0; i < P.passes.size(); i++, n++) {
      const WindowArgs &w = P.passes[i];
      const long long by = X * ((w.src16 ? 2 : 4) + (w.dst16 ? 2 : 4));
      if (info && 4 * n + 3 < cap) {
        info[4 * n] = (long long)i; info[4 * n + 1] = 1;
        info[4 * n + 2] = by; info[4 * n + 3] = -2;
      }
    }
    return n;
  }
  int j = 0;
  for (const auto &p : P.groups) {
    long long rd = 0, wr = 0;
    if (p.a.src == kSrcCnt) rd = 2;
    else if (p.a.src == kSrcLayers)
      rd = (p.a.in8 ? 1LL : p.a.in16 ? 2LL : 4LL) * p.a.lin;
    if (p.a.dst == kDstLayers)
      wr = (p.a.out8 ? 1LL : p.a.out16 ? 2LL : 4LL) * p.a.lout;
    else if (p.a.dst == kDstMap) wr = 4;
    else wr = 2;
    long long by = X * (rd + wr);
    if (p.a.src == kSrcCode) by += 8 * S.codeM;
    if (info && 4 * n + 3 < cap) {
      info[4 * n] = j; info[4 * n + 1] = p.a.k + p.a.pair_axis;
      info[4 * n + 2] = by; info[4 * n + 3] = p.kernel;
    }
    j += p.a.k + p.a.pair_axis;
    n++;
  }
  return n;
}

int dct_b200_plan_probe(int problem, int n, const int *ax, int R,
                        int init_mode, int out_mode, int budget_kb, int pipe,
                        int half, long long *rows, int cap) {
  if (n < 1 || n > kMaxAxes || R < 1 || !ax || problem < 0 || problem > 3 ||
      init_mode < 0 || init_mode > 2 || out_mode < 1 || out_mode > 3 ||
      (out_mode == 2 && init_mode != 0) || budget_kb < 16 ||
      budget_kb > 220 || pipe < 0 || pipe > 3 || cap < 0)
    return -1;
  const bool layered = problem == kHamming || problem == kLee;
  if (layered && R + 1 > kMaxLayers) return -1;
  if (!layered && out_mode == 3) return -1;
  Geometry g{};
  g.prob = problem; g.n = n; g.R = R; g.mu = 1;
  g.pw[0] = 1;
  for (int i = 0; i < n; i++) {
    if (ax[i] < 2 || ax[i] >= (1 << 24)) return -1;
    if (layered && ax[i] > 16) return -1;
    if (problem == kTorus && (ax[i] < 3 || 2 * R + 1 > ax[i])) return -1;
    if (g.pw[i] > (1LL << 40) / ax[i]) return -2;
    g.ax[i] = ax[i];
    g.pw[i + 1] = g.pw[i] * ax[i];
  }
  g.space = g.pw[n];
  g = transform_geometry(g);                  // as a cell would plan it
  bool wide = false;
  for (int i = 0; i < n; i++) wide = wide || ax[i] > 16;
  if (!layered && wide) return 0;             // window passes, not groups
  const int R1 = layered ? R + 1 : 1;
  const int src = init_mode == 0 ? kSrcCode : kSrcCnt;
  const int dst = out_mode == 1 ? kDstMap
                  : out_mode == 2 ? kDstCnt : kDstLayers;
  // never dereferenced: aligned stand-ins for the planes
  int32_t *const fake = reinterpret_cast<int32_t *>(uintptr_t(1) << 12);
  const long long plane = round_up(g.space, kPlaneAlign);
  PlanPtrs ptr{fake, plane, reinterpret_cast<uint16_t *>(fake),
               reinterpret_cast<long long *>(fake), 0, nullptr};
  ptr.layers16 = reinterpret_cast<uint16_t *>(fake + plane);
  Knobs kn{(size_t)budget_kb << 10, pipe};
  kn.half = half && R1 >= 2 && dst != kDstLayers;
  const std::vector<GroupPlan> P = plan_groups(g, R1, ptr, src, dst, kn);
  int m = 0, j = 0;
  for (const auto &p : P) {
    const GroupArgs &a = p.a;
    int rbsum = 0;
    for (int r = 0; r < a.nrounds; r++) rbsum += a.rb[r];
    const long long row[24] = {
        j, a.k + a.pair_axis, a.pair_axis, a.W, a.mid, a.Bo, a.inner,
        a.outer, a.ntiles, p.kernel, a.pipe, a.pack, a.in16, a.out16,
        (long long)p.smem, p.threads, a.lin, a.lout, a.skew, p.grid, a.src,
        a.dst, a.nrounds, rbsum};
    if (rows && 24 * (m + 1) <= cap)
      for (int t = 0; t < 24; t++) rows[24 * m + t] = row[t];
    j += a.k + a.pair_axis;
    m++;
  }
  return m;
}

int dct_b200_plan_forms(int init_mode, int out_mode, int *forms, int cap) {
  if (!S.live || S.streamed || init_mode < 0 || init_mode > 2 || out_mode < 1 ||
      out_mode > 3 || cap < 0)
    return -1;
  Plan &P = plan_for(init_mode, out_mode);
  if (P.window) return 0;
  int n = 0;
  for (const auto &p : P.groups) {
    if (forms && n < cap)
      forms[n] = (p.a.pipe ? 1 : 0) | (p.a.pack ? 2 : 0) |
                 (p.a.in16 ? 4 : 0) | (p.a.out16 ? 8 : 0) |
                 (p.a.pair_axis ? 16 : 0) | (p.a.tma ? 32 : 0) |
                 (p.a.in8 || p.a.out8 ? 64 : 0);
    n++;
  }
  return n;
}

int dct_b200_ball_hist(const long long *words, int nw, int src, int nbins,
                       int32_t *out) {
  if (!S.live || nbins < 1 || nbins > 32 || !out || (src != 0 && src != 1))
    return -1;
  if (nw <= 0) return 0;
  if (!valid_words(words, nw)) return -1;
  const WalkArgs w = walk_args();
  const long long cap = kStageCap / nbins;   // nb * nbins fits d_out
  for (long long off = 0; off < nw; off += cap) {
    const int nb = (int)std::min<long long>(cap, nw - off);
    int rc = stage_words(words + off, nb);
    if (rc) return rc;
    rc = launch_ball_hist(w, S.d_words, nb, S.layers, src, nbins, S.d_out,
                          g_stream);
    if (rc) return rc;
    CC_CK(cudaMemcpyAsync(S.h_out, S.d_out, (size_t)nb * nbins * 4,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(out + off * nbins, S.h_out, (size_t)nb * nbins * 4);
  }
  return 0;
}

int dct_b200_layers_at(const long long *idx, int k, int32_t *out) {
  if (!S.live || !S.layered_out || (k && !out)) return -1;
  if (k <= 0) return 0;
  if (!valid_words(idx, k)) return -1;
  if (S.streamed) {
    const long long X = S.g.space;
    for (int i = 0; i < k; i++)
      for (int d = 0; d < S.R1; d++)
        out[(long long)i * S.R1 + d] = S.h_layers[d * X + idx[i]];
    return 0;
  }
  const long long cap = kStageCap / S.R1;
  for (long long off = 0; off < k; off += cap) {
    const int nb = (int)std::min<long long>(cap, k - off);
    int rc = stage_words(idx + off, nb);
    if (rc) return rc;
    rc = launch_layers_at(S.layers, S.plane, S.R1, S.d_words, nb, S.d_out,
                          g_stream);
    if (rc) return rc;
    CC_CK(cudaMemcpyAsync(S.h_out, S.d_out, (size_t)nb * S.R1 * 4,
                          cudaMemcpyDeviceToHost, g_stream));
    CC_CK(cudaStreamSynchronize(g_stream));
    memcpy(out + off * S.R1, S.h_out, (size_t)nb * S.R1 * 4);
  }
  return 0;
}

int dct_b200_set_timing(int on) {
  g_timing = on ? 1 : 0;
  return 0;
}

int dct_b200_last_timings(float *ms, int cap) {
  const int n = g_last_n < cap ? g_last_n : cap;
  for (int i = 0; i < n && ms; i++) ms[i] = g_last_ms[i];
  return g_last_n;
}

int dct_b200_read_map(long long off, long long len, int32_t *out) {
  if (!S.live || off < 0 || len < 0 || off + len > S.g.space ||
      (len && !out))
    return -1;
  if (len)
    CC_CK(cudaMemcpyAsync(out, S.layers + off, (size_t)len * 4,
                          cudaMemcpyDeviceToHost, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  return 0;
}

int dct_b200_read_layer(int d, long long off, long long len, int32_t *out) {
  if (!S.live || !S.layered_out || d < 0 || d >= S.R1 || off < 0 ||
      len < 0 || off + len > S.g.space || (len && !out))
    return -1;
  if (len && S.streamed) {
    memcpy(out, S.h_layers + d * S.g.space + off, (size_t)len * 4);
    return 0;
  }
  if (len)
    CC_CK(cudaMemcpyAsync(out, S.layers + d * S.plane + off,
                          (size_t)len * 4, cudaMemcpyDeviceToHost, g_stream));
  CC_CK(cudaStreamSynchronize(g_stream));
  return 0;
}

}  // extern "C"
