/* coldcore_b200/plugin.h — C ABI of the B200 covering engine
 * (libcoldcore_covering.so, built for sm_100a).
 *
 * Drop-in for coldcore's plugin ABI v1: the same flat `dct_*` symbols with
 * the same signatures, return codes and validation, so coldcore's ctypes
 * binding (src/coldcore/gpu.py:52-103) loads this library unchanged through
 * COLDCORE_PLUGIN_PATH.  Each declaration cites the reference declaration
 * it replaces (coldcore src/include/coldcore/plugin.h) and the reference
 * implementation whose behaviour it keeps (src/plugins/covering/dct_hc.cu).
 *
 * Conventions kept from the reference (plugin.h:7-17):
 *  - singleton context: one cell per process per loaded library;
 *  - 0 = ok, negative = engine error, -100-e = CUDA error e (message on
 *    stderr);
 *  - caller-allocated outputs; input arrays are read before the call returns;
 *  - invalid indices, update signs other than +-1, over-removals and
 *    counter overflow are rejected before any state changes.
 *
 * Differences (additive or relaxed, never narrowing):
 *  - up to 40 axes, R <= 7, Hamming / Lee axes up to 16, torus / grid axes
 *    up to 2^24 (torus: 2R+1 <= axis); the v1 table packs positions and
 *    deltas in nibbles (n <= 16, axes <= 16), so larger cells — binary
 *    Hamming n = 26, the king 2048x2048 torus — use dct_init3w;
 *  - the occurrence limit is exact instead of global: a multiset is
 *    accepted while min(total occurrences, max multiplicity x |B|) <= 65535
 *    (no uint16 counter can then exceed 65535), which admits every cell
 *    the reference's 65,535 global cap admits;
 *  - all device work runs, in call order, on one stream owned by the
 *    engine (dct_b200_stream) instead of the legacy default stream.
 */
#ifndef COLDCORE_B200_PLUGIN_H
#define COLDCORE_B200_PLUGIN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COLDCORE_PLUGIN_ABI_VERSION 1

#if defined(__GNUC__)
#define CCP_API __attribute__((visibility("default")))
#else
#define CCP_API
#endif

/* problem ids — plugin.h:45-53 */
#define CCP_PROB_HAMMING    0
#define CCP_PROB_TORUS_LINF 1
#define CCP_PROB_LEE        2
#define CCP_PROB_GRID_LINF  3

/* ---- lifecycle ---- */
/* plugin.h:62-65; dct_hc.cu:230-374.  ballpat: v1 packed table, byte k =
 * pos<<4 | delta, zero byte terminates, entry 0 the centre. */
CCP_API int  dct_init3(int problem, int n, const int *ax, int R,
               const uint64_t *ballpat, long long balllen, int extract_cap,
               long long *bytes, int layers_mode, int cnt_mode,
               int use_owner);
/* plugin.h:70-72; dct_hc.cu:377-385 (homogeneous Hamming) */
CCP_API int  dct_init2(int q, int n, int R, const uint64_t *ballpat,
               long long balllen, int extract_cap, long long *bytes,
               int layers_mode, int cnt_mode, int use_owner);
/* plugin.h:73-74; dct_hc.cu:387-391 */
CCP_API int  dct_init (int q, int n, int R, const uint64_t *ballpat,
               long long balllen, int extract_cap, long long *bytes);
/* plugin.h:66; dct_hc.cu:393-428 (also resets mu to 1) */
CCP_API int  dct_free(void);
/* plugin.h:67; dct_hc.cu:208 — bytes outside HBM (managed modes) */
CCP_API long long dct_host_bytes(void);

/* ---- solution / transforms ---- */
/* plugin.h:81; dct_hc.cu:452-459 — stages the code multiset */
CCP_API int  dct_set_code(const long long *idx, int M);
/* plugin.h:82; dct_hc.cu:465-521 — pairs (0,1) (0,2) (1,1) (2,1).
 * Additive: out_mode 3 (Hamming / Lee) leaves the exact distance layers
 * N_0..N_R of the transform in the planes instead of their sum, for
 * dct_b200_read_layer. */
CCP_API int  dct_transform(int init_mode, int out_mode);

/* ---- mu-fold multiple covering ---- */
CCP_API int  dct_set_mu(int mu);             /* plugin.h:91; dct_hc.cu:214-220 */
CCP_API int  dct_get_mu(void);               /* plugin.h:92; dct_hc.cu:222 */

/* ---- incremental / exact per-candidate ---- */
/* plugin.h:95; dct_hc.cu:567-587 (batches <= 1024 words return before the
 * device finishes; the next data-returning call waits) */
CCP_API int  dct_ball_update(const long long *words, int nwords, int delta);
/* plugin.h:96-97; dct_hc.cu:785-788 */
CCP_API int  dct_ball_gather(const long long *words, int nwords, int target,
                     int32_t *out);
/* plugin.h:100-101; dct_hc.cu:794-799 (role 0 deficient, 1 critical) */
CCP_API int  dct_ball_gather_mu(const long long *words, int nwords, int role,
                        int32_t *out);
/* plugin.h:102; dct_hc.cu:997-1022 — needs use_owner at init */
CCP_API int  dct_loss_owner(const long long *words, int M, int32_t *out);

/* ---- v0.3 optional ---- */
/* plugin.h:111-112; dct_hc.cu:826-866 */
CCP_API int  dct_ball_update_delta(const long long *words, int nwords, int delta,
                           long long *dd);
/* plugin.h:113-115; dct_hc.cu:882-977 */
CCP_API int  dct_swap_eval(const long long *drops, int k, const long long *cand,
                   const long long *off, int32_t *gain, int32_t *loss);
/* plugin.h:116; dct_hc.cu:779-783 — counters: [0] gathers served by the
 * set side, [1] by the walk, [2] predicate-set scans, [3] scans that
 * overflowed, [4] swap_eval fast path, [5] swap_eval fallback, [6]
 * count_eq(0) answered by the listing pass, [7] tiled set gathers */
CCP_API int  dct_stats(long long *out, int n);

/* ---- reductions / map queries ---- */
CCP_API long long dct_count_eq(int target);          /* plugin.h:122; dct_hc.cu:1024 */
CCP_API long long dct_count_deficit(void);           /* plugin.h:125; dct_hc.cu:981 */
CCP_API int  dct_map_max(int32_t *out);              /* plugin.h:126; dct_hc.cu:1056 */
CCP_API int  dct_map_hist(int nbins, int32_t vmax,   /* plugin.h:127; dct_hc.cu:1071 */
                  int32_t *out);
CCP_API long long dct_map_extract  (int32_t thr,     /* plugin.h:128; dct_hc.cu:1093 */
                            uint32_t *idx, int32_t *val, int cap);
CCP_API long long dct_map_extract64(int32_t thr,     /* plugin.h:130; dct_hc.cu:1114 */
                            int64_t *idx, int32_t *val, int cap);
CCP_API int  dct_map_read_at(const long long *idx,   /* plugin.h:132; dct_hc.cu:1136 */
                     int k, int32_t *out);
CCP_API int  dct_read_cnt(long long off,             /* plugin.h:133; dct_hc.cu:1153 */
                  long long len, uint16_t *out);

/* ---- alternative support-table format (ox) ---- */
/* plugin.h:136-138; dct_hc.cu:431-450 */
CCP_API int  dct_set_tbl2(const uint16_t *mask, const uint64_t *offs,
                  long long len);
CCP_API int  dct_use_fmt(int fmt);

/* ---- additive symbols of this engine (no reference counterpart) ---- */
/* dct_init3 with a wide support table: `slots` int32 per pattern, each
 * (pos << 24) | delta with delta a circular shift in 1..ax[pos]-1, 0 =
 * unused slot; row 0 the centre.  Lifts the 16-wide axis limit of the v1
 * nibble format (king 2048x2048 needs it).  Replaces the table argument of
 * plugin.h:62-65 only. */
CCP_API int  dct_init3w(int problem, int n, const int *ax, int R,
                const int32_t *tbl, int slots, long long len,
                int extract_cap, long long *bytes);
/* dct_init3w with dct_init3's placement arguments (layers_mode 1: host
 * planes streamed by each transform; 2: managed; cnt_mode 1/2: managed),
 * so that wide-table cells can take the out-of-core path too. */
CCP_API int  dct_b200_init3wm(int problem, int n, const int *ax, int R,
                              const int32_t *tbl, int slots, long long len,
                              int extract_cap, long long *bytes,
                              int layers_mode, int cnt_mode);
/* the engine's CUDA stream (cudaStream_t as an integer), for host timing */
CCP_API long long dct_b200_stream(void);
/* describe the launches of one dct_transform(init_mode, out_mode) without
 * running it: per launch 4 values (first axis, axes in the launch,
 * algorithmic HBM bytes read + written, kernel id); returns the number of
 * launches (at most cap/4 described) or a negative error (-1 for a cell
 * whose layers stream from host memory: dct_b200_ooc_plan describes it). */
CCP_API int  dct_b200_plan(int init_mode, int out_mode, long long *info, int cap);
/* schedule form of each group launch of one transform (no counterpart in
 * the reference): bit 1 prefetching (cp.async) kernel, 2 packed word pairs,
 * 4 16-bit layer source, 8 16-bit layer output, 16 axis 0 inside each pair;
 * returns the number of launches (0 for window passes) or a negative error */
CCP_API int  dct_b200_plan_forms(int init_mode, int out_mode, int *forms, int cap);
/* the group schedule the planner gives a geometry, without a cell or a GPU
 * (no counterpart in the reference): for problem / axes / R, transform
 * (init_mode, out_mode), tile budget (KB), prefetch mode 0-3 and 16-bit
 * planes on/off, 24 values per launch: first axis, axes, pair axis, W,
 * mid, Bo, inner, outer, tiles, kernel id, prefetching, packed, 16-bit
 * source, 16-bit output, shared bytes, threads, live layers in, out,
 * skew, grid, source, destination, rounds, axes over all rounds.  Returns
 * the number of launches (0 for window passes) or a negative error. */
CCP_API int  dct_b200_plan_probe(int problem, int n, const int *ax, int R,
                                 int init_mode, int out_mode, int budget_kb,
                                 int pipe, int half, long long *rows, int cap);
/* per-launch device timing of transforms (events around every launch;
 * DCT_TIMING=1 in the environment turns it on too and prints each time to
 * stderr, the reference's DCT_TIMING, dctcore_hamming.cuh:464-511) */
CCP_API int  dct_b200_set_timing(int on);
/* milliseconds of each launch of the last transform; returns the count */
CCP_API int  dct_b200_last_timings(float *ms, int cap);
/* words [off, off+len) of the map (the last transform's out_mode 1 field) */
CCP_API int  dct_b200_read_map(long long off, long long len, int32_t *out);
/* ---- batched campaign (no counterpart in the reference, which runs one
 * process per cell: src/coldcore/campaign.py:186-221).  A batch holds many
 * independent cells (any problem, axes <= 16, each code within the exact
 * uint16 bound min(occurrences, max multiplicity x |B|) <= 65,535) and
 * computes, for every cell, cnt from its code, the deficit
 * sum max(0, mu - cnt), the gain map and its maximum and the loss map and
 * its maximum in ONE persistent launch replayed from a CUDA graph.  Handles
 * are independent of the dct_* singleton cell. ---- */
CCP_API long long dct_batch_create(void);
/* returns the cell index, or a negative error */
CCP_API int  dct_batch_add(long long h, int problem, int n, const int *ax,
                           int R, int mu, const long long *code, int M);
/* allocates and schedules; tile_kb = shared memory per tile, 0 = autotune */
CCP_API int  dct_batch_build(long long h, int tile_kb);
/* mode 0: the persistent graph launch; 1: one launch per pass per cell
 * (same kernels and streams, no graph); 2: self-test of the bounded
 * dependency wait (returns -7, no hang) */
CCP_API int  dct_batch_run(long long h, int mode);
/* field 0 cnt (uint16), 1 gain map (int32), 2 loss map (int32) */
CCP_API int  dct_batch_read(long long h, int cell, int field, long long off,
                            long long len, void *out);
/* per cell: deficit, gain maximum, loss maximum; returns values written */
CCP_API int  dct_batch_scalars(long long h, long long *out, int cap);
/* cells, passes, work items, tile KB, grid, tuned step microseconds; with
 * cap >= 8 also the step's algorithmic HBM bytes and those of the cells
 * with their own launches (returns the values written, 6 or 8) */
CCP_API int  dct_batch_info(long long h, long long *out, int cap);
/* Per-cell calls between launches, so a search can run on each cell
 * (the role of a campaign job's own plugin context, campaign.py:88-179).
 * set_code replaces a cell's code (room for 4x its first size, at least
 * min(|X|, 2^18) words, else -3); the next launch recounts from it.  set_table gives
 * the cell's support table (len x slots int32, (pos << 24) | shift, as
 * dct_init3w takes it).  update adds delta (+1 / -1) over the balls of nw
 * <= 65,536 words; gather counts ball words by role (0 deficient, 1
 * critical, else cnt == role); extract lists the gain (field 1) or loss
 * (field 2) map entries >= thr, unordered, and returns how many exist. */
CCP_API int  dct_batch_set_code(long long h, int cell, const long long *code,
                                int M);
CCP_API int  dct_batch_set_table(long long h, int cell, const int32_t *tbl,
                                 int slots, long long len);
CCP_API int  dct_batch_update(long long h, int cell, const long long *words,
                              int nw, int delta);
CCP_API int  dct_batch_gather(long long h, int cell, const long long *words,
                              int nw, int role, int32_t *out);
CCP_API long long dct_batch_extract(long long h, int cell, int field,
                                   int32_t thr, long long *idx, int32_t *val,
                                   int cap);
/* Exact greedy on n listed cells at once, one argmax / place / refresh
 * launch per step for all of them: from each cell's gain map as the last
 * launch left it (no update since), code words excluded, place the word of
 * largest gain (ties: smallest index) until the deficit is 0, nothing
 * gains, or max_add[k] (<= cap) words are placed; the same rule as
 * dct_b200_greedy_fill.  placed_out: cap words per listed cell. */
CCP_API int  dct_batch_greedy(long long h, const int *cells, int n,
                              const int *max_add, long long *placed_out,
                              int cap, int *nplaced_out,
                              long long *deficit_out);
/* mode 0: #{x : cnt[x] == target}; mode 1: sum max(0, mu - cnt[x]) */
CCP_API long long dct_batch_count(long long h, int cell, int mode,
                                 int target);
/* the gain (field 1) or loss (field 2) map at k <= 65,536 words */
CCP_API int  dct_batch_read_at(long long h, int cell, int field,
                               const long long *idx, int k, int32_t *out);
CCP_API int  dct_batch_free(long long h);

/* ---- learned ruin proposal scorer (no counterpart in the reference): a
 * 32-128-128-1 ReLU MLP, BF16 operands with FP32 accumulation, trained
 * with binary cross-entropy and Adam by this library's kernels.  The
 * parameter vector is 20,865 floats: W1[32][128], b1[128], W2[128][128],
 * b2[128], w3[128], b3. ---- */
CCP_API long long dct_mlp_create(unsigned long long seed);
/* copy the parameters out (get_out) and / or in (set_in); returns count */
CCP_API int  dct_mlp_params(long long h, float *get_out, const float *set_in);
/* gradient of the mean loss over n samples (X n x 32, T n in {0,1}) */
CCP_API int  dct_mlp_grad(long long h, const float *X, const float *T, int n,
                          float *grad_out);
CCP_API int  dct_mlp_train(long long h, const float *X, const float *T, int n,
                           int epochs, int batch, float lr,
                           unsigned long long seed);
/* logits of n samples */
CCP_API int  dct_mlp_predict(long long h, const float *X, int n, float *out);
CCP_API int  dct_mlp_free(long long h);

/* No counterpart in the reference.  Gain (role 0) or loss (role 1) map of
 * a Hamming / Lee cell for callers that may not allocate device memory —
 * a framework whose own allocator must own every buffer, a service that
 * reserves its memory at start-up.  cnt (uint16, |X| words) and map (int32,
 * |X| words) are device pointers the caller owns; the (R+1) distance layers
 * live in a fixed 64 MiB device array inside this library, which every GPU
 * that loads the library keeps until exit.  Needs round_up(|X|, 64) x (R+1)
 * <= 16,777,216 words, else returns -6 with a message on stderr.  Queued on
 * `stream` (a cudaStream_t as an integer, 0 = the default stream) without
 * waiting.  Calls share the array: calls that overlap on the GPU race.  The
 * first call on a device looks up the array's address, so make it before
 * any stream capture; under CUDA's lazy module loading the array is also
 * committed to device memory at the library's first use on that device, so
 * a caller that reserves the rest of the device should make one small call
 * first.  After a cudaDeviceReset the entry point must not be used again in
 * that process.  Calls no cudaMalloc / cudaFree. */
CCP_API int  dct_b200_field_noalloc(int problem, int n, const int *ax, int R,
                                    int mu, int role, const uint16_t *cnt,
                                    int32_t *map, long long stream);
/* after dct_transform(init, 3): words [off, off+len) of distance layer d */
/* (the two below have no counterpart in the reference; they feed the
 * learned ruin proposal) per word, a histogram over its ball: src 0 bins
 * the current map in log2 steps (bin 0: v <= 0, 1: v == 1, 2: 2..3, ...),
 * src 1 bins cnt linearly (bin b: cnt == b); the last of nbins (<= 32)
 * bins takes everything above.  out is nw x nbins. */
CCP_API int  dct_b200_ball_hist(const long long *words, int nw, int src,
                                int nbins, int32_t *out);
/* after dct_transform(init, 3): the R+1 layer values at each of k words */
CCP_API int  dct_b200_layers_at(const long long *idx, int k, int32_t *out);
/* Exact greedy repair on the device (no counterpart in the reference, whose
 * repair is the Python lazy greedy of src/coldcore/search.py:260-360): from
 * the current cnt, repeatedly place the non-active word of largest exact
 * gain (ties: the smallest index) until nothing is deficient, no word has a
 * positive gain, or max_add words are placed.  placed (capacity max_add)
 * receives the words in placement order and joins the active multiset;
 * *deficit receives the total deficit left.  Returns the number placed or a
 * negative code.  The map (plane 0) is overwritten.  |X| < 2^32. */
CCP_API int  dct_b200_greedy_fill(int max_add, long long *placed,
                                  long long *deficit);
CCP_API int  dct_b200_read_layer(int d, long long off, long long len, int32_t *out);

/* ---- out-of-core (ooc) cells: distance layers in host memory ----
 * Replaces the reference's host placement of the layer planes
 * (layers_mode 1/2: src/plugins/covering/dctcore_core.cuh:86-119, chosen
 * by src/coldcore/gpu.py:253-260 when |X|(4(R+1)+2) bytes exceed the HBM
 * budget), whose kernels read the planes over GH200's coherent C2C.  Here
 * the planes sit in caller-owned (pinned) host memory and one transform
 * streams them through two device pieces in two phases: slabs of the low
 * axes 0..s-1 (device to host), then column blocks of the high axes
 * s..n-1 (host to device); cnt, the map and the code stay in HBM.  The
 * modes are dct_transform's (plugin.h:84-88): init 0 the code (host words,
 * any order, a multiset under the counter rule), 1 gain / 2 loss from cnt
 * (device, |X| uint16) at multiplicity mu; out 1 the int32 map and 2 cnt
 * (device, |X| words), 3 every layer (the host planes, int32, plane d at
 * host + d|X|).  device_budget bounds the bytes allocated on the device;
 * min_width (0: 32) the narrowest column block.  Torus / grid axes above 16
 * are not streamed (-3); -2 when no split fits the budget.
 *
 * info (17 values): split s, P_low, P_high, slab rows, slabs, column width,
 * columns, piece words, piece plane stride, 16-bit host planes, planes
 * carried between the phases, host bytes needed, device bytes, bytes over
 * the host link, ball size, R+1 (or 1), host bytes per plane word. */
CCP_API int  dct_b200_ooc_plan(int problem, int n, const int *ax, int R,
                               int init_mode, int out_mode, long long M,
                               long long maxmult, long long device_budget,
                               int min_width, long long *info, int cap);
/* The schedule without a device: rows of 20 values, one per copy, fill,
 * scatter, launch and stream join, in issue order; returns the row count
 * (rows beyond cap_rows are counted, not written). */
CCP_API long long dct_b200_ooc_record(int problem, int n, const int *ax,
                                      int R, int init_mode, int out_mode,
                                      int mu, const long long *code,
                                      long long M, long long device_budget,
                                      int min_width, long long *rows,
                                      long long cap_rows);
/* One streamed transform; ms (2 floats, may be NULL) receives the device
 * time of each phase.  Synchronizes the device on entry and returns when
 * the result is in place. */
CCP_API int  dct_b200_ooc_transform(int problem, int n, const int *ax, int R,
                                    int init_mode, int out_mode, int mu,
                                    const long long *code, long long M,
                                    const uint16_t *cnt, void *out,
                                    void *host, long long host_bytes,
                                    long long device_budget, int min_width,
                                    float *ms);

#ifdef __cplusplus
}
#endif
#endif /* COLDCORE_B200_PLUGIN_H */
