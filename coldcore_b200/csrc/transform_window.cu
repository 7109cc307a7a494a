// transform_window.cu — one window-sum axis pass of any width (torus / grid).
//
// Recurrence of the reference's torus and open-grid plugins
// (coldcore src/plugins/covering/dctcore_torus.cuh:1-12,
//  dctcore_grid.cuh:1-30): newA[a] = sum of A over the circular (torus) or
// clamped (grid) window [a-R, a+R] along one axis.  The reference keeps the
// fibre in a 16-entry register array (axes <= 16); this pass has no width
// limit (the king 2048x2048 torus), runs out of place, and maps one thread
// to one output word so that a warp's 2R+1 reads and its write are 128-byte
// coalesced along the contiguous inner index; the 2R neighbours of a word
// are re-read from L1/L2, not HBM.
#include "engine.h"

namespace cc {

// The word x = (o * q + a) * stride + i of the pass's axis position a:
// with the space below 2^31 words the digit comes from two 32-bit
// divisions (a 64-bit division costs several times more instructions, and
// the pass is issue-bound: one read of each of 2R+1 neighbours a word).
template <bool GRID, int SRC16, int DST16, bool I32>
__global__ void __launch_bounds__(256) window_axis(const WindowArgs w) {
  const long long gs = (long long)gridDim.x * blockDim.x;
  for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       x < w.space; x += gs) {
    int a;
    long long base;
    if (I32) {
      const unsigned xs = (unsigned)x, st = (unsigned)w.stride;
      const unsigned hi = xs / st;
      a = (int)(hi % (unsigned)w.q);
      base = (long long)(xs - (unsigned)a * st);
    } else {
      const long long hi = x / w.stride;
      a = (int)(hi % w.q);
      base = x - (long long)a * w.stride;
    }
    int lo = a - w.R, up = a + w.R;
    if (GRID) { if (lo < 0) lo = 0; if (up > w.q - 1) up = w.q - 1; }
    int32_t s = 0;
    for (int b = lo; b <= up; b++) {
      int bb = b;
      if (!GRID) { if (bb < 0) bb += w.q; else if (bb >= w.q) bb -= w.q; }
      const long long y = base + (long long)bb * w.stride;
      if (SRC16) s += cnt_pred(w.pmode, (int)w.src16[y], w.ptarget, w.mu);
      else s += w.src32[y];
    }
    if (DST16) w.dst16[x] = (uint16_t)(s > 65535 ? 65535 : s);
    else w.dst32[x] = s;
  }
}

int launch_window(const WindowArgs &w, cudaStream_t s) {
  const long long nblk = (w.space + 255) / 256;
  long long nb = nblk;
  const long long cap = (long long)sm_count() * 16;
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  nb = grid_knob((int)nb, nblk);
  const bool s16 = w.src16 != nullptr, d16 = w.dst16 != nullptr;
  const bool i32 = w.space < (1LL << 31);
#define WL(G, A, B)                                                         \
  (i32 ? window_axis<G, A, B, true><<<(int)nb, 256, 0, s>>>(w)              \
       : window_axis<G, A, B, false><<<(int)nb, 256, 0, s>>>(w))
  if (w.grid) {
    if (s16 && d16) WL(true, 1, 1); else if (s16) WL(true, 1, 0);
    else if (d16) WL(true, 0, 1); else WL(true, 0, 0);
  } else {
    if (s16 && d16) WL(false, 1, 1); else if (s16) WL(false, 1, 0);
    else if (d16) WL(false, 0, 1); else WL(false, 0, 0);
  }
#undef WL
  CC_CK(cudaGetLastError());
  return 0;
}

}  // namespace cc
