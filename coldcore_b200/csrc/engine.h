// engine.h — internal state and launch interfaces of the B200 covering engine.
//
// One process-wide cell (the plugin ABI v1 singleton model, coldcore
// src/include/coldcore/plugin.h:8-10).  Every kernel takes its geometry by
// value (no __constant__ state shared between translation units), and every
// launch goes to the engine's own stream, so device work runs in call order.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include <vector>

namespace cc {

constexpr int kMaxAxes = 40;      // |X| <= 2^40 with every axis >= 2
constexpr int kMaxLayers = 8;     // R + 1 distance layers (R <= 7)
constexpr int kMaxSlots = 8;      // changed positions per support pattern
constexpr int kPlaneAlign = 64;   // plane stride rounded to 64 elements

// problem ids: coldcore src/include/coldcore/plugin.h:45-53
enum Problem { kHamming = 0, kTorus = 1, kLee = 2, kGrid = 3 };

// cnt predicates (coldcore src/plugins/covering/dctcore_mu.cuh:28-40)
enum Pred { kPredEq = 0, kPredDef = 1, kPredCrit = 2, kPredIdent = 3 };

struct Geometry {
  int prob, n, R, mu;
  long long space;
  int ax[kMaxAxes];
  long long pw[kMaxAxes + 1];
};

__host__ __device__ inline bool cnt_pred(int mode, int c, int target, int mu) {
  if (mode == kPredDef) return c < mu;
  if (mode == kPredCrit) return c >= 1 && c <= mu;
  return c == target;
}

// ------------------------------------------------------------ transform plan
// One kernel launch covers a GROUP of consecutive axes [j0, j0+k).  The
// group's words factor as x = o*(inner*mid) + m*inner + i with
// inner = pw[j0], mid = prod of the group's axes; a tile is W consecutive
// inner positions x mid x Bo consecutive outer slabs, staged in shared
// memory.  Rounds process `rb` axes each in registers (local stride rs in m).
constexpr int kMaxRounds = 24;
constexpr int kGroupThreads = 512;   // CTA size cap: 128 registers per thread

enum Src { kSrcLayers = 0, kSrcCnt = 1, kSrcCode = 2 };
enum Dst { kDstLayers = 0, kDstMap = 1, kDstCnt = 2 };

struct GroupArgs {
  int32_t *layers;        // plane 0 base; plane d at layers + d*plane
  long long plane;        // plane stride (elements)
  uint16_t *cnt;
  const long long *code;  // sorted code (kSrcCode)
  long long ncode;
  const long long *code_bounds;  // per-tile slice of the code (kSrcCode)
  long long inner, outer, ntiles, nchunk;
  int mid, W, Bo, k;
  int nrounds;
  int rb[kMaxRounds];     // axes per round
  int rs[kMaxRounds];     // local stride (in m) of the round's first axis
  int rq[kMaxRounds];     // axis size of the round (all axes of a round equal)
  int qax[kMaxRounds];    // per-axis size inside the group (generic kernel)
  int src, dst, lin, lout;
  int pmode, ptarget, mu, R;
  int skew;               // log2 of the shared-memory skew period (0 = none)
  int prob;
  int pipe;               // prefetch the next tile while computing (cp.async)
  int32_t *map;           // kDstMap target (nullptr: plane 0 of layers)
  // 16-bit intermediate planes: plane d at layers16 + d*plane (u16 words),
  // read when in16, written when out16 (values provably <= 65535)
  uint16_t *layers16;
  int in16, out16;
  // 8-bit planes between a streamed binary first group (out8) and the
  // streamed launch after it (in8), where every layer value after the
  // first group's k axes stays below 256: a 0/1 predicate source and
  // C(k, d) <= 255 for every d <= R.  Plane d at byte off8 + d*plane of
  // the 16-bit plane region, past the 16-bit planes that the launch
  // reading them writes (so no tile overwrites bytes another has yet to
  // read).
  int in8, out8;
  long long off8;
  // streamed group: axes per register round (0: RoundAxes, the default)
  int tbm;
  int pack;               // two inner words per 32-bit lane (group_kernel)
  // first group of a binary Hamming cell: axis 0 is the word pair itself
  // (inner = 2), applied once as a swap-add inside each packed lane
  int pair_axis;
  long long *red;         // epilogue reduction target (generic tiles, the
                          // register kernels and the streamed groups)
  int red_mode;           // 0 none, 1 deficit of the cnt written, 2 map max
  // streamed form (transform_tma.cu): tensor loads into `stages` shared
  // memory stages, W = 2 x lanes inner words a tile (tma 1); the first
  // group staged from cnt by bulk copies (tma 2); a ternary first group
  // over row pairs packed in 32-bit lanes (tma 3, Bo = 2)
  int tma;
  int stages;
  // padded layout of the 16-bit planes (ternary cells): every run of t0
  // words (the first group's mid) is stored at a pitch of `pitch` words
  // (a multiple of 64), so rows of the later groups start on 128-byte
  // boundaries.  The first group writes its layers padded; the later
  // groups' `inner` is then the padded one, and the last group's map or
  // cnt goes back to the canonical index.  0 = the canonical layout.
  long long pitch;
  long long t0;
};

// arguments of a streamed group launch (transform_tma.cu)
constexpr int kTmaMaxStages = 4;
struct TmaArgs {
  uint16_t *layers16;
  long long plane;
  int32_t *map;
  uint16_t *cnt;
  long long inner, nchunk, ntiles;
  int lin, lout, stages;
  int *fault;             // mapped host word, set when a wait runs out
  // first group (tma_first): the cnt source and its predicate
  const uint16_t *cnt_in;
  int pmode, ptarget, mu;
  // first group of a recount (code_first): the sorted code, per-tile slices
  const long long *code;
  const long long *code_bounds;
  // padded planes (GroupArgs::pitch): the canonical inner stride, the
  // pitch and the valid words of each padded run
  long long inner_c, pitch, t0;
  // ternary first group (tern_first): the rows of the cell
  long long rows;
  // 8-bit layer planes (tma_first OUT 5): their byte offset from layers16
  long long off8;
  // epilogue reduction of a map or cnt written (GroupArgs::red_mode)
  long long *red;
  int red_mode;
};

struct GroupPlan {
  GroupArgs a;
  int kernel;             // index into the launcher table
  int threads;
  size_t smem;
  int grid;
};

// planner.cu: schedule knobs and the group plan of one transform
// pipe: see plan_groups; half: 16-bit planes between the launches
// pair: allow the pair first group (binary Hamming, 16-bit planes)
// pad: the padded 16-bit layout for a ternary cell (streamed later groups)
// u8: 8-bit planes after a streamed binary first group (gain / loss)
struct Knobs { size_t budget; int pipe; int half = 0; int pair = 1;
               int pad = 0; int u8 = 0; };
struct PlanPtrs {
  int32_t *layers; long long plane; uint16_t *cnt;
  const long long *code; long long ncode; int32_t *map;
  uint16_t *layers16 = nullptr;   // u16 plane region (Knobs::half)
};
// An axis range of one transform: the launches cover axes [begin, end) of
// g (end < 0: through the last axis).  reach0 is the distance reach of axes
// applied by an earlier range (so the live layers at axis j are
// min(reach0 + reach of axes [begin, j), R) + 1); `final` is false when
// the range's layers feed a later range, which keeps the last launch's
// plane width (16-bit planes) and writes only its live layers.
struct AxisRange {
  int begin = 0;
  int end = -1;
  long long reach0 = 0;
  bool final = true;
};
std::vector<GroupPlan> plan_groups(const Geometry &g, int R1,
                                   const PlanPtrs &ptr, int src, int dst,
                                   Knobs kn, AxisRange range = AxisRange());
// distance reach of one axis: 1 for Hamming, floor(a/2) for Lee
inline long long axis_reach(int prob, int a) { return prob == kLee ? a / 2 : 1; }
// The transform geometry of a cell: Lee distance on axes of size 2 or 3 is
// the Hamming distance (every nonzero digit difference has weight
// min(d, q - d) = 1), so such a cell plans and runs as Hamming, with the
// Hamming kernels' streamed forms.
inline Geometry transform_geometry(Geometry g) {
  if (g.prob != kLee) return g;
  for (int j = 0; j < g.n; j++)
    if (g.ax[j] > 3) return g;
  g.prob = kHamming;
  return g;
}

// launchers (transform_*.cu)
int launch_group(const GroupPlan &p, cudaStream_t s);
int prepare_group(const GroupPlan &p);
int group_blocks_per_sm(const GroupPlan &p);
size_t group_smem_bytes(const GroupArgs &a, int R1);
// the prefetching kernel has a packed form for 16-bit layer sources
bool pipe_pairs_ok(const GroupArgs &a);
int pick_group_kernel(int prob, int q, int R1, int *bm);
int group_kernel_variants(int prob, int q, int R1, int *kids, int *bms,
                          int cap);
// the same group with every other register-blocked kernel and CTA width
// (rounds, skew and grid recomputed; tiles unchanged), the plan itself first
// the padded plan of a ternary cell (planner.cu), in place; false leaves
// `groups` unchanged
bool pad_plan(std::vector<GroupPlan> &groups, const Geometry &g,
              const PlanPtrs &ptr, int dst, int R1, long long room16);
// every group a streamed form serves takes it (planner.cu)
void stream_groups(std::vector<GroupPlan> &groups, int R1);
// 8-bit planes between the streamed first group and the launch after it
// (planner.cu), in place; false leaves `groups` unchanged
bool u8_plan(std::vector<GroupPlan> &groups, int R1, long long room16);
// algorithmic HBM bytes of one group launch (planner.cu)
long long group_bytes(const GroupArgs &a);
std::vector<GroupPlan> group_variants(const GroupPlan &p, int R1,
                                      size_t smem_cap);
// streamed form of a strided group (transform_tma.cu)
size_t tma_smem_bytes(int q, int k, int r1, int lanes, int stages,
                      int in8 = 0);
bool tma_group_ok(const GroupArgs &a, int q, int r1, int lanes, int stages);
GroupPlan tma_variant(const GroupPlan &p, int lanes, int stages, int threads);
// the first group read from cnt (axis 0 in the pair), a.tma == 2
size_t tma_first_smem_bytes(int kk, int r1, int stages);
bool tma_first_ok(const GroupArgs &a, int r1, int stages);
GroupPlan tma_first_variant(const GroupPlan &p, int stages, int threads);
// the first group of a ternary Hamming cell over row pairs, a.tma == 3
bool tern_first_ok(const GroupArgs &a, int r1);
GroupPlan tern_first_variant(const GroupPlan &p, int threads);
int launch_tma_group(const GroupPlan &p, cudaStream_t s);
int tma_prepare(const GroupPlan &p);
int tma_blocks_per_sm(const GroupPlan &p);
int tma_fault_pending();
void tma_fault_clear();
int launch_code_bounds(const long long *code, long long ncode,
                       long long tile_words, long long ntiles,
                       long long *bounds, cudaStream_t s);

// batched engine: one persistent launch over (pass, tile) work items
struct BatchLaunch {
  const GroupArgs *passes;
  const int *dep;
  const unsigned *need;
  const int4 *items;            // (pass, first tile, tiles, 0)
  long long nitems;
  unsigned *done;
  unsigned long long *next;
  int *err;
  size_t smem;
  int grid;
};
int launch_batch(const BatchLaunch &b, cudaStream_t s);
int batch_grid(size_t smem);

// window pass (torus / grid) over one axis, any width, out of place
struct WindowArgs {
  const int32_t *src32; const uint16_t *src16; int pmode, ptarget, mu;
  int32_t *dst32; uint16_t *dst16;
  long long space, stride; int q, R, grid;
};
int launch_window(const WindowArgs &w, cudaStream_t s);

// ------------------------------------------------------------ walks
// Support table in structure-of-arrays form: slot s of pattern t is
// tbl[s*len + t] = (pos << 24) | delta, delta a circular shift in
// 1..ax_pos-1; 0 = unused slot.  Entry 0 is the centre.
struct WalkArgs {
  Geometry g;
  const int32_t *tbl;
  int slots;
  long long len;
  uint16_t *cnt;
};
constexpr int kParamWords = 1024;       // words passed by value per launch
struct WordsParam { long long w[kParamWords]; };

// nb words from `dwords` (device) or, when dwords == nullptr, from `pw`
int launch_update(const WalkArgs &w, const long long *dwords,
                  const WordsParam *pw, int nb, int delta,
                  unsigned long long *trans, cudaStream_t s);
// bits: (|X|+7)/8 bytes of scratch for the predicate bit plane of a large
// call (gather_bits_pay), or nullptr
int launch_gather(const WalkArgs &w, const long long *dwords, int nb,
                  int mode, int target, int32_t *out, bool zeroed,
                  cudaStream_t s, uint8_t *bits = nullptr);
bool gather_bits_pay(const WalkArgs &w, int nb);
int pick_split(long long len, int nb);
// set side (setside.cu): list {x : pred(cnt[x])} as packed digit words, then
// count, per candidate, the listed words within distance R
int launch_list_pred(const Geometry &g, const uint16_t *cnt, int mode,
                     int target, unsigned long long *out, long long cap,
                     unsigned long long *found, cudaStream_t s);
int launch_gather_set(const Geometry &g, const long long *dcand, int nc,
                      const unsigned long long *Z, long long zn, int32_t *out,
                      bool zeroed, cudaStream_t s);
// device-side exact greedy (walks.cu): state in device memory, one step =
// argmax of the gain map, placement of that word, incremental gain update
struct GreedyState;
constexpr int kGreedyStateBytes = 32;
int launch_greedy_exclude(int32_t *map, const long long *dwords, int n,
                          int32_t exclude, cudaStream_t s);
// the batched form: one cell's walk, gain map, state and buffers
struct BatchGreedyCell {
  WalkArgs w;
  int32_t *map;
  void *st;                 // GreedyState (kGreedyStateBytes)
  long long *placed;
  long long *fresh;         // |B| words
  int max_add;
};
int launch_batch_greedy_step(const BatchGreedyCell *dcells, int ncells,
                             long long max_space, int32_t exclude,
                             cudaStream_t s);
int launch_greedy_step(const WalkArgs &w, int32_t *map, long long N,
                       GreedyState *st, long long *placed, int max_add,
                       long long *fresh, int32_t exclude, cudaStream_t s);
// swap evaluation fast path: per drop its loss and the list of its ball
// words at exactly mu (two walks and a segment scan), then per candidate
// the listed words of its drop within distance R
int launch_seg_scan(const int32_t *cnt, int n, long long cap, int32_t *offs,
                    int32_t *cursor, cudaStream_t s);
int launch_drop_walks(const WalkArgs &w, const long long *ddrops, int k,
                      int32_t *loss, int32_t *nmu, int32_t *offs,
                      int32_t *cursor, long long cap, long long *list,
                      cudaStream_t s);
int launch_swap_corr(const Geometry &g, int k, const long long *dcand,
                     const int32_t *dcoff, const int32_t *offs,
                     const long long *list, long long cap, int32_t *gain,
                     cudaStream_t s);
int launch_ball_hist(const WalkArgs &w, const long long *dwords, int nb,
                     const int32_t *map, int src, int nbins, int32_t *out,
                     cudaStream_t s);
int launch_layers_at(const int32_t *layers, long long plane, int R1,
                     const long long *idx, int k, int32_t *out,
                     cudaStream_t s);

// ------------------------------------------------------------ reductions
int launch_cnt_reduce(const uint16_t *cnt, long long N, int mode, int target,
                      int mu, long long *out, cudaStream_t s);
int launch_max(const int32_t *A, long long N, long long *out, cudaStream_t s);
int launch_hist(const int32_t *A, long long N, int nbins, int32_t vmax,
                int32_t *hist, cudaStream_t s);
int launch_extract(const int32_t *A, long long N, int32_t thr, void *oidx,
                   bool wide, int32_t *oval, long long cap, long long *ocount,
                   cudaStream_t s);
int launch_read_at(const int32_t *A, const long long *idx, int k,
                   int32_t *out, cudaStream_t s);
int launch_scatter(int32_t *A, const long long *idx, long long M,
                   cudaStream_t s);

int sm_count();
// DCT_BLOCKS, read at each cell's init as coldcore's plugin reads it: when
// set, the grid of every persistent transform launch (at least 256 CTAs, at
// most one per tile; every such kernel strides its tiles by the grid); 0
// leaves the grids to the occupancy rule.
extern int g_dct_blocks;
inline int grid_knob(int grid, long long ntiles) {
  if (g_dct_blocks <= 0) return grid;
  long long g = g_dct_blocks;
  if (g > ntiles) g = ntiles;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace cc

#define CC_CK(x)                                                            \
  do {                                                                      \
    cudaError_t e_ = (x);                                                   \
    if (e_ != cudaSuccess) {                                                \
      fprintf(stderr, "coldcore_b200: CUDA error %s at %s:%d\n",            \
              cudaGetErrorString(e_), __FILE__, __LINE__);                  \
      return -(100 + (int)e_);                                              \
    }                                                                       \
  } while (0)

namespace cc {
// Two timing events, destroyed on every way out of the scope that made
// them (error returns included).
struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int create() {
    CC_CK(cudaEventCreate(&e0));
    CC_CK(cudaEventCreate(&e1));
    return 0;
  }
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};
}  // namespace cc
