/* coldcore_b200/sparse.h — C ABI of the B200 explicit-incidence engine
 * (libcoldcore_sparse.so, built for sm_100a).
 *
 * Drop-in for coldcore's plugin ABI 2 (explicit incidence): the same flat
 * `sparse_*` symbols with the same signatures and return codes, so
 * coldcore's ctypes binding (src/coldcore/incidence_gpu.py:39-67) loads
 * this library unchanged through COLDCORE_SPARSE_PLUGIN_PATH.  Each
 * declaration cites the reference implementation whose behaviour it keeps
 * (coldcore src/plugins/sparse/sparse.cu).
 *
 * The model: n_cand candidates, a universe of n_univ elements, and an
 * incidence — either dense rows (candidate c covers the d elements of row
 * c of an n_cand x d int32 matrix) or weighted CSR rows (candidate c
 * covers indices[indptr[c] .. indptr[c+1]) with weights w >= 1, universe
 * weights uw >= 1).  The engine keeps cnt (int32 over the universe) and
 * map (int32 over the candidates, the last field).
 *
 * Conventions kept from the reference (sparse.cu:21-24): singleton
 * context, 0 = ok, negative = engine error, -100-e = CUDA error e (message
 * on stderr), caller-allocated outputs, input arrays read before the call
 * returns.
 *
 * Differences (never narrowing):
 *  - candidate lists (update, recount, gather, read_at) are checked on the
 *    host: an index outside [0, n_cand) returns -2 before any device work
 *    (the reference reads out of bounds);
 *  - inc_mode 1 (the reference's CPU-memory placement, read over GH200's
 *    coherent C2C) maps to managed memory preferring the host, because a
 *    B200 host has no coherent C2C; sparse_inc_mode then reports 2, the
 *    reference's own fallback value (sparse.cu:86-91);
 *  - all device work runs, in call order, on one stream owned by the
 *    engine (sparse_b200_stream) instead of the legacy default stream.
 */
#ifndef COLDCORE_B200_SPARSE_H
#define COLDCORE_B200_SPARSE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CCS_API __attribute__((visibility("default")))
#else
#define CCS_API
#endif

/* 2 — sparse.cu:436 */
CCS_API int       sparse_abi_version(void);
/* allocation totals in device / host (managed) memory — sparse.cu:438-439 */
CCS_API long long sparse_dev_bytes(void);
CCS_API long long sparse_host_bytes(void);
/* release the cell; mu back to 1; a no-op when none — sparse.cu:441-456 */
CCS_API int       sparse_free(void);
/* dense cell: inc is n_cand x d row-major int32, entries in [0, n_univ);
 * inc_mode 0 = HBM, 1 = host-preferring managed memory; -1 when a cell is
 * live, -2 on bad sizes or modes — sparse.cu:458-488 */
CCS_API int       sparse_init(long long n_cand, int d, long long n_univ,
                              const int32_t *inc, int inc_mode,
                              int extract_cap, long long *bytes_dev,
                              long long *bytes_host);
/* weighted CSR cell — sparse.cu:490-528 */
CCS_API int       sparse_init_csr(long long n_cand, long long n_univ,
                                  long long nnz, const int64_t *indptr,
                                  const int32_t *indices, const int32_t *w,
                                  const int32_t *uw, int inc_mode,
                                  int extract_cap, long long *bytes_dev,
                                  long long *bytes_host);
/* placement of the incidence (-1 without a cell) — sparse.cu:530 */
CCS_API int       sparse_inc_mode(void);
/* 1 for a weighted CSR cell — sparse.cu:531 */
CCS_API int       sparse_is_csr(void);
/* covering multiplicity (>= 1) — sparse.cu:533-539 */
CCS_API int       sparse_set_mu(int mu);
CCS_API int       sparse_get_mu(void);
/* cnt[u] += delta (dense) or delta * w (CSR) for every incidence of every
 * listed candidate — sparse.cu:542-557 */
CCS_API int       sparse_ball_update(const long long *idx, long long m,
                                     int delta);
/* cnt = 0, then the solution's rows added — sparse.cu:559-565 */
CCS_API int       sparse_recount(const long long *idx, long long m);
/* map over every candidate: target 0 gain (deficient elements, or the
 * weighted gain), 1 loss (critical elements, or the weighted loss), other
 * values the literal count of cnt == target — sparse.cu:567-579 */
CCS_API int       sparse_field(int target);
/* the same per-candidate counts for a list — sparse.cu:581-598 */
CCS_API int       sparse_ball_gather(const long long *idx, long long m,
                                     int target, int32_t *out);
/* universe elements with cnt == target — sparse.cu:600-609 */
CCS_API long long sparse_count_eq(int target);
/* sum max(0, mu - cnt) (times uw for CSR); 0 iff feasible —
 * sparse.cu:611-624 */
CCS_API long long sparse_count_deficit(void);
/* max(0, max map) — sparse.cu:626-636 */
CCS_API int       sparse_map_max(int32_t *out);
/* positive map values binned at (v-1)*nbins/vmax, clipped to the last
 * bin; 1 <= nbins <= 4096, vmax >= 1 — sparse.cu:638-650 */
CCS_API int       sparse_map_hist(int nbins, int32_t vmax, int32_t *out);
/* candidates with map >= thr, unordered; returns the number found (which
 * may exceed cap; min(found, cap) stored) — sparse.cu:652-670 */
CCS_API long long sparse_map_extract(int32_t thr, int64_t *idx, int32_t *val,
                                     int cap);
/* map at listed candidates — sparse.cu:672-684 */
CCS_API int       sparse_map_read_at(const long long *idx, long long k,
                                     int32_t *out);
/* cnt[off, off+len) as int32 — sparse.cu:686-692 */
CCS_API int       sparse_read_cnt(long long off, long long len, int32_t *out);

/* ---- additive (no counterpart in the reference) */
/* the engine's CUDA stream (cudaStream_t as an integer) */
CCS_API long long sparse_b200_stream(void);
/* lanes that cooperate on one candidate row in the field, gather and
 * update kernels (a power of two <= 32, chosen from the row length) */
CCS_API int       sparse_b200_row_lanes(void);

/* a covering-design cell C(v,k,t) whose rows are built on the device
 * (v <= 128, k <= 32, C(v,t) < 2^31, C(k,t) <= 2^20), in the layout of
 * coldcore's build_incidence (src/coldcore/problems/covering_design.py:
 * 95-135): candidate c = the k-subset of colex rank c, universe element u =
 * the t-subset of colex rank u, row c = the ranks of its t-subsets, block
 * positions in lex order.  Saves building and uploading C(v,k) x C(k,t)
 * entries on the host. */
CCS_API int       sparse_b200_init_design(int v, int k, int t, int inc_mode,
                                          int extract_cap,
                                          long long *bytes_dev,
                                          long long *bytes_host);
/* rows [c0, c0+n) of a dense cell, n x d int32 */
CCS_API int       sparse_b200_read_rows(long long c0, long long n,
                                        int32_t *out);

#ifdef __cplusplus
}
#endif

#endif /* COLDCORE_B200_SPARSE_H */
