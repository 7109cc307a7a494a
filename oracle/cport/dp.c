/* dp.c — C restatement of the reference's CPU axis DP (test infrastructure
 * and the timed CPU baseline of bench.py; never part of the engine).
 *
 * Follows coldcore src/coldcore/dp.py: seed layer 0 from the cnt predicate
 * (dp.py:287-308, protocol.py:325-340) or the code multiset (dp.py:293-300),
 * one in-place pass per axis over the (R+1) int32 layer planes — Hamming
 * dp.py:239-243, Lee dp.py:245-254, torus dp.py:256-262, grid dp.py:264-273
 * — and the layer sum (dp.py:275-285).  Fibres are processed in chunks of
 * the contiguous inner index so the inner loops vectorise, and chunks run
 * in parallel with OpenMP.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CHUNK 2048

static long long span_of(long long stride) {
  return stride < CHUNK ? stride : CHUNK;
}

/* one Hamming axis pass: newA_d[a] = A_d[a] + T_{d-1} - A_{d-1}[a] */
static void axis_hamming(int32_t *A, int nl, long long X, long long stride,
                         int q) {
  const long long H = X / (stride * q);
  const long long span = span_of(stride);
  const long long nch = (stride + span - 1) / span;
#pragma omp parallel
  {
    int32_t *T = (int32_t *)malloc(sizeof(int32_t) * nl * span);
#pragma omp for schedule(static)
    for (long long t = 0; t < H * nch; t++) {
      const long long h = t / nch, c = t % nch;
      const long long l0 = c * span;
      const long long len = stride - l0 < span ? stride - l0 : span;
      const long long base = h * stride * q + l0;
      for (int d = 0; d < nl - 1; d++) {
        int32_t *Td = T + (long long)d * span;
        memset(Td, 0, sizeof(int32_t) * len);
        for (int a = 0; a < q; a++) {
          const int32_t *row = A + (long long)d * X + base + (long long)a * stride;
          for (long long l = 0; l < len; l++) Td[l] += row[l];
        }
      }
      for (int d = nl - 1; d >= 1; d--) {
        const int32_t *Tp = T + (long long)(d - 1) * span;
        for (int a = 0; a < q; a++) {
          int32_t *cur = A + (long long)d * X + base + (long long)a * stride;
          const int32_t *low = A + (long long)(d - 1) * X + base +
                               (long long)a * stride;
          for (long long l = 0; l < len; l++) cur[l] += Tp[l] - low[l];
        }
      }
    }
    free(T);
  }
}

/* one Lee axis pass: circulant grades, the antipode once on even axes */
static void axis_lee(int32_t *A, int nl, long long X, long long stride,
                     int q) {
  const long long H = X / (stride * q);
  const long long span = span_of(stride);
  const long long nch = (stride + span - 1) / span;
  const int half = q / 2;
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < H * nch; t++) {
    const long long h = t / nch, c = t % nch;
    const long long l0 = c * span;
    const long long len = stride - l0 < span ? stride - l0 : span;
    const long long base = h * stride * q + l0;
    for (int d = nl - 1; d >= 1; d--) {
      const int wm = d < half ? d : half;
      for (int a = 0; a < q; a++) {
        int32_t *cur = A + (long long)d * X + base + (long long)a * stride;
        for (int w = 1; w <= wm; w++) {
          const int am = (a - w + q) % q, ap = (a + w) % q;
          const int32_t *m = A + (long long)(d - w) * X + base +
                             (long long)am * stride;
          for (long long l = 0; l < len; l++) cur[l] += m[l];
          if (ap != am) {
            const int32_t *p = A + (long long)(d - w) * X + base +
                               (long long)ap * stride;
            for (long long l = 0; l < len; l++) cur[l] += p[l];
          }
        }
      }
    }
  }
}

/* one window pass (torus: circular, grid: clamped) on plane 0 */
static void axis_window(int32_t *A, long long X, long long stride, int q,
                        int R, int grid) {
  const long long H = X / (stride * q);
  const long long span = span_of(stride);
  const long long nch = (stride + span - 1) / span;
#pragma omp parallel
  {
    int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)q * span);
#pragma omp for schedule(static)
    for (long long t = 0; t < H * nch; t++) {
      const long long h = t / nch, c = t % nch;
      const long long l0 = c * span;
      const long long len = stride - l0 < span ? stride - l0 : span;
      const long long base = h * stride * q + l0;
      for (int a = 0; a < q; a++) {
        int32_t *o = tmp + (long long)a * span;
        memset(o, 0, sizeof(int32_t) * len);
        int lo = a - R, hi = a + R;
        if (grid) { if (lo < 0) lo = 0; if (hi > q - 1) hi = q - 1; }
        for (int b = lo; b <= hi; b++) {
          int bb = b;
          if (!grid) { if (bb < 0) bb += q; else if (bb >= q) bb -= q; }
          const int32_t *row = A + base + (long long)bb * stride;
          for (long long l = 0; l < len; l++) o[l] += row[l];
        }
      }
      for (int a = 0; a < q; a++)
        memcpy(A + base + (long long)a * stride, tmp + (long long)a * span,
               sizeof(int32_t) * len);
    }
    free(tmp);
  }
}

/* problem: 0 hamming, 1 torus, 2 lee, 3 grid.  Layer 0 must be seeded by
 * the caller (cc_seed_pred / cc_seed_code); layers 1..nl-1 are zeroed
 * here.  out_map (int32) and / or out_cnt (uint16, clamped at 65535)
 * receive the layer sum. */
void cc_transform(int problem, int n, const int *ax, int R, int32_t *A,
                  int32_t *out_map, uint16_t *out_cnt) {
  long long X = 1;
  for (int j = 0; j < n; j++) X *= ax[j];
  const int nl = (problem == 0 || problem == 2) ? R + 1 : 1;
  if (nl > 1) memset(A + X, 0, sizeof(int32_t) * X * (nl - 1));
  long long stride = 1;
  for (int j = 0; j < n; j++) {
    if (problem == 0) axis_hamming(A, nl, X, stride, ax[j]);
    else if (problem == 2) axis_lee(A, nl, X, stride, ax[j]);
    else axis_window(A, X, stride, ax[j], R, problem == 3);
    stride *= ax[j];
  }
#pragma omp parallel for schedule(static)
  for (long long x = 0; x < X; x++) {
    int32_t s = 0;
    for (int d = 0; d < nl; d++) s += A[(long long)d * X + x];
    if (out_map) out_map[x] = s;
    if (out_cnt) out_cnt[x] = (uint16_t)(s > 65535 ? 65535 : s);
  }
}

/* layer 0 = [cnt < mu] (mode 1), [1 <= cnt <= mu] (mode 2), [cnt == t] (0) */
void cc_seed_pred(const uint16_t *cnt, long long X, int mode, int target,
                  int mu, int32_t *A) {
#pragma omp parallel for schedule(static)
  for (long long x = 0; x < X; x++) {
    const int c = cnt[x];
    A[x] = mode == 1 ? c < mu : mode == 2 ? (c >= 1 && c <= mu) : c == target;
  }
}

void cc_seed_code(const long long *code, long long M, long long X,
                  int32_t *A) {
  memset(A, 0, sizeof(int32_t) * X);
  for (long long i = 0; i < M; i++) A[code[i]]++;
}

/* Explicit incidence (coldcore src/coldcore/incidence.py:160-220): the
 * field over dense rows, map[c] = #{u in row c : role(cnt[u])} with role 0
 * deficient (cnt < mu), 1 critical (1 <= cnt <= mu), other targets the
 * literal cnt == target; rows split over the host threads. */
void cc_inc_field(const int32_t *inc, long long ncand, int d,
                  const int32_t *cnt, int target, int mu, int32_t *map) {
#pragma omp parallel for schedule(static)
  for (long long c = 0; c < ncand; c++) {
    const int32_t *row = inc + c * d;
    int32_t s = 0;
    for (int j = 0; j < d; j++) {
      const int v = cnt[row[j]];
      s += target == 0 ? v < mu : target == 1 ? (v >= 1 && v <= mu)
                                              : v == target;
    }
    map[c] = s;
  }
}
