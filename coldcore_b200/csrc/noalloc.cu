// noalloc.cu — gain / loss field of a Hamming or Lee cell for callers that
// cannot allocate device memory.
//
// Some callers own all of their device memory up front and may not call
// cudaMalloc afterwards: a framework whose caching allocator must see every
// allocation, a service that reserves its memory at start-up and runs under
// a fixed budget, or code that runs between the allocation points of a host
// program it does not control.  They can still hand in buffers they own.
// dct_b200_field_noalloc takes the cell's cnt plane and the output map as
// device pointers and keeps the transform's (R+1) distance-layer planes in a
// file-scope device array of fixed size instead of allocating them.
//
// The array, its limit and its rules:
//  * kNoAllocWords int32 words (64 MiB); a call needs round_up(|X|, 64) x
//    (R+1) words and is refused (return -6, message on stderr) beyond that;
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * every call on a device shares the one array and leaves its contents
//    behind; nothing in it needs to start at zero (each launch writes every
//    layer word before a later launch reads it), but calls whose work
//    overlaps on the GPU — two streams, or two host threads — race on it;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (the host-side name is only a stand-in), so that
//    first call should come before any stream capture;
//  * with CUDA's default lazy module loading, the array is committed to the
//    device's memory when this library's kernels are first loaded on that
//    device, which may be that first call: a caller that reserves the rest
//    of the device up front should make one small call on every device it
//    uses before reserving, so that the 64 MiB are already held;
//  * the looked-up address belongs to the device's current context: after a
//    cudaDeviceReset of that device, this entry point must not be called
//    again in the same process.
// No cudaMalloc, cudaFree or other allocating routine is called; the last
// group of axes writes the caller's map directly; the work is queued on the
// caller's stream and the call returns without waiting.
#include <atomic>
#include <cstdio>

#include "../../include/coldcore_b200/plugin.h"
#include "engine.h"

namespace {

using namespace cc;

constexpr long long kNoAllocWords = 16LL << 20;   // 64 MiB of int32
// every tile stays within the default 48 KB of dynamic shared memory, so
// no launch needs the opt-in attribute
constexpr size_t kNoAllocTileBytes = 48 * 1024;
constexpr int kMaxDevices = 64;

__device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocWords];

// per device: the array's device address, looked up once (host threads may
// race to look it up; they store the same value)
std::atomic<int32_t *> g_noalloc_ptr[kMaxDevices];

int noalloc_scratch(int32_t **out) {
  int dev = 0;
  CC_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return -1;
  int32_t *p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    void *addr = nullptr;
    CC_CK(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
    p = static_cast<int32_t *>(addr);
    g_noalloc_ptr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return 0;
}

}  // namespace

extern "C" int dct_b200_field_noalloc(int problem, int n, const int *ax,
                                      int R, int mu, int role,
                                      const uint16_t *cnt, int32_t *map,
                                      long long stream) {
  if ((problem != kHamming && problem != kLee) || n < 1 || n > kMaxAxes ||
      !ax || R < 1 || R + 1 > kMaxLayers || mu < 1 || mu > 65535 ||
      (role != 0 && role != 1) || !cnt || !map)
    return -1;
  long long pw[kMaxAxes + 1];
  pw[0] = 1;
  for (int i = 0; i < n; i++) {
    if (ax[i] < 2 || ax[i] > 16) return -1;
    if (pw[i] > (1LL << 40) / ax[i]) return -2;
    pw[i + 1] = pw[i] * ax[i];
  }
  const long long space = pw[n];
  const int R1 = R + 1;
  const long long plane = (space + kPlaneAlign - 1) / kPlaneAlign * kPlaneAlign;
  if (plane * R1 > kNoAllocWords) {
    fprintf(stderr,
            "coldcore_b200: dct_b200_field_noalloc needs %lld scratch words "
            "(|X| = %lld, R = %d); its fixed array holds %lld\n",
            plane * R1, space, R, kNoAllocWords);
    return -6;
  }
  int32_t *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // predicate of the role: 0 = deficient (gain), 1 = critical (loss)
  const int pmode = mu == 1 ? kPredEq : (role == 0 ? kPredDef : kPredCrit);
  const int ptarget = mu == 1 ? role : 0;
  long long reach = 0;               // distance the processed axes can add
  // tile words per layer within the shared-memory bound (the runtime-size
  // kernel keeps R+1 int32 planes of the tile, plus one row of padding)
  const long long tile_budget = (long long)(kNoAllocTileBytes / 4) / R1 - 32;
  int j = 0;
  while (j < n) {
    GroupArgs a{};
    a.layers = scratch;
    a.plane = plane;
    a.cnt = const_cast<uint16_t *>(cnt);
    a.inner = pw[j];
    a.W = a.inner >= 32 ? 32 : (int)a.inner;
    a.prob = problem;
    a.R = R;
    a.mu = mu;
    a.pmode = pmode;
    a.ptarget = ptarget;
    long long mid = 1;
    while (j + a.k < n && a.k < kMaxRounds) {
      GroupArgs t = a;
      const long long mid2 = mid * ax[j + a.k];
      const long long outer = space / (a.inner * mid2);
      t.k = a.k + 1;
      t.mid = (int)mid2;
      const long long fit = tile_budget / (a.W * mid2);
      t.Bo = a.W >= 32 ? 1 : (int)(outer < fit ? outer : fit);
      if (t.Bo < 1) t.Bo = 1;
      if (group_smem_bytes(t, R1) > kNoAllocTileBytes) break;
      a = t;
      mid = mid2;
    }
    if (a.k == 0) {                  // cannot happen for axes <= 16
      fprintf(stderr, "coldcore_b200: dct_b200_field_noalloc found no "
              "tile for axis %d\n", j);
      return -2;
    }
    for (int t = 0; t < a.k; t++) a.qax[t] = ax[j + t];
    a.outer = space / (a.inner * (long long)a.mid);
    a.nchunk = (a.inner + a.W - 1) / a.W;
    a.ntiles = (a.outer + a.Bo - 1) / a.Bo * a.nchunk;
    long long reach2 = reach;
    for (int t = 0; t < a.k; t++)
      reach2 += problem == kLee ? ax[j + t] / 2 : 1;
    a.lin = (int)(reach < R ? reach : R) + 1;
    a.lout = (int)(reach2 < R ? reach2 : R) + 1;
    a.src = j == 0 ? kSrcCnt : kSrcLayers;
    a.dst = j + a.k == n ? kDstMap : kDstLayers;
    a.map = map;                     // the last group writes it directly
    GroupPlan p;
    p.a = a;
    p.kernel = -1;                   // the runtime-size kernel
    p.threads = 256;
    p.smem = group_smem_bytes(a, R1);
    long long grid = (long long)sm_count() * 4;
    if (grid > a.ntiles) grid = a.ntiles;
    p.grid = (int)(grid < 1 ? 1 : grid);
    rc = launch_group(p, s);
    if (rc) return rc;
    reach = reach2;
    j += a.k;
  }
  return 0;
}
