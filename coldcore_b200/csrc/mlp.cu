// mlp.cu — the learned ruin proposal's scorer: a 32-128-128-1 MLP with
// ReLU hidden layers, trained and evaluated on the GPU by this file's own
// kernels.  BF16 operands, FP32 accumulation: the two hidden-layer GEMMs and
// the three backward GEMMs run on the tensor cores through warp-level
// mma.sync m16n8k16 (bf16 x bf16 -> f32); the 128-wide output layer, the
// loss and the Adam step are FP32 SIMT.
//
// One CTA owns 64 samples and every weight (the whole net is 20,865
// parameters: W1 and W2 sit in shared memory as bf16).  Forward:
//   h1 = bf16(relu(bf16(x) W1b + b1)), h2 = bf16(relu(h1 W2b + b2)),
//   y = h2 . w3 + b3;
// training loss: binary cross-entropy with logits against t in {0,1},
// averaged over the n samples of the batch; backward (ReLU masks from the
// stored bf16 activations):
//   dy = (sigmoid(y) - t) / n, dw3 = sum dy h2, db3 = sum dy,
//   dz2 = bf16(dy w3 [h2 > 0]), dW2 = h1^T dz2, db2 = sum dz2,
//   dz1 = bf16((dz2 W2b^T) [h1 > 0]), dW1 = bf16(x)^T dz1, db1 = sum dz1;
// per-CTA partial gradients are added into one FP32 gradient vector.
// oracle/mlp_oracle.py restates the same arithmetic in float64 for the
// gradient check.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../include/coldcore_b200/plugin.h"
#include "engine.h"

namespace {

constexpr int kIn = 32, kHid = 128, kRows = 64;
// flat parameter vector (fp32 master copy)
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid,
              kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid, kB3 = kW3 + kHid,
              kParams = kB3 + 1;

struct MlpSmem {
  __nv_bfloat16 w1[kIn * kHid];      // [in][hid]
  __nv_bfloat16 w2[kHid * kHid];     // [in][out]
  __nv_bfloat16 x[kRows * kIn];
  __nv_bfloat16 h1[kRows * kHid];
  __nv_bfloat16 h2[kRows * kHid];
  __nv_bfloat16 dz2[kRows * kHid];
  __nv_bfloat16 dz1[kRows * kHid];
  float b1[kHid], b2[kHid], w3[kHid];
  float y[kRows], dy[kRows];
  float b3;
};

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo,
                                          __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) |
         ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C[16x8] += A[16xK] B[Kx8] with A(i, k), B(k, n) read through accessors,
// K a multiple of 16; one warp, fragments as the m16n8k16 .bf16 layout
// defines them (g = lane / 4, t = lane % 4).
template <typename FA, typename FB>
__device__ __forceinline__ void warp_mma(FA A, FB B, int K, float c[4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int k0 = 0; k0 < K; k0 += 16) {
    const uint32_t a0 = pack2(A(g, k0 + 2 * t), A(g, k0 + 2 * t + 1));
    const uint32_t a1 = pack2(A(g + 8, k0 + 2 * t), A(g + 8, k0 + 2 * t + 1));
    const uint32_t a2 = pack2(A(g, k0 + 2 * t + 8), A(g, k0 + 2 * t + 9));
    const uint32_t a3 = pack2(A(g + 8, k0 + 2 * t + 8),
                              A(g + 8, k0 + 2 * t + 9));
    const uint32_t b0 = pack2(B(k0 + 2 * t, g), B(k0 + 2 * t + 1, g));
    const uint32_t b1 = pack2(B(k0 + 2 * t + 8, g), B(k0 + 2 * t + 9, g));
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  }
}

// element (row, col) of the warp's C fragment register r
__device__ __forceinline__ void frag_pos(int r, int *row, int *col) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  *row = g + (r >= 2 ? 8 : 0);
  *col = 2 * t + (r & 1);
}

template <bool TRAIN>
__global__ void __launch_bounds__(256)
k_mlp(const float *P, const __nv_bfloat16 *w1b, const __nv_bfloat16 *w2b,
      const float *X, const float *T, int n, float scale, float *out_y,
      float *G) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MlpSmem &s = *reinterpret_cast<MlpSmem *>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.x * kRows;
  for (int i = tid; i < kIn * kHid; i += blockDim.x) s.w1[i] = w1b[i];
  for (int i = tid; i < kHid * kHid; i += blockDim.x) s.w2[i] = w2b[i];
  for (int i = tid; i < kHid; i += blockDim.x) {
    s.b1[i] = P[kB1 + i];
    s.b2[i] = P[kB2 + i];
    s.w3[i] = P[kW3 + i];
  }
  if (tid == 0) s.b3 = P[kB3];
  for (int i = tid; i < kRows * kIn; i += blockDim.x) {
    const int r = i / kIn;
    s.x[i] = __float2bfloat16(r0 + r < n ? X[(long long)r0 * kIn + i] : 0.f);
  }
  __syncthreads();
  // ---- layer 1: 64 x 128 outputs = 4 x 16 tiles, 8 per warp, K = 32
  for (int tile = warp; tile < 64; tile += 8) {
    const int m0 = (tile >> 4) * 16, n0 = (tile & 15) * 8;
    float c[4] = {0, 0, 0, 0};
    warp_mma([&](int i, int k) { return s.x[(m0 + i) * kIn + k]; },
             [&](int k, int j) { return s.w1[k * kHid + n0 + j]; }, kIn, c);
    for (int r = 0; r < 4; r++) {
      int row, col;
      frag_pos(r, &row, &col);
      const float z = c[r] + s.b1[n0 + col];
      s.h1[(m0 + row) * kHid + n0 + col] = __float2bfloat16(z > 0.f ? z : 0.f);
    }
  }
  __syncthreads();
  // ---- layer 2: 64 x 128, K = 128
  for (int tile = warp; tile < 64; tile += 8) {
    const int m0 = (tile >> 4) * 16, n0 = (tile & 15) * 8;
    float c[4] = {0, 0, 0, 0};
    warp_mma([&](int i, int k) { return s.h1[(m0 + i) * kHid + k]; },
             [&](int k, int j) { return s.w2[k * kHid + n0 + j]; }, kHid, c);
    for (int r = 0; r < 4; r++) {
      int row, col;
      frag_pos(r, &row, &col);
      const float z = c[r] + s.b2[n0 + col];
      s.h2[(m0 + row) * kHid + n0 + col] = __float2bfloat16(z > 0.f ? z : 0.f);
    }
  }
  __syncthreads();
  // ---- output layer: one warp per row
  for (int r = warp; r < kRows; r += 8) {
    float acc = 0.f;
    for (int c = lane; c < kHid; c += 32)
      acc += __bfloat162float(s.h2[r * kHid + c]) * s.w3[c];
    for (int o = 16; o > 0; o >>= 1)
      acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      s.y[r] = acc + s.b3;
      if (r0 + r < n && out_y) out_y[r0 + r] = s.y[r];
    }
  }
  if (!TRAIN) return;
  __syncthreads();
  // ---- loss gradient
  for (int r = tid; r < kRows; r += blockDim.x) {
    float d = 0.f;
    if (r0 + r < n) {
      const float p = 1.f / (1.f + expf(-s.y[r]));
      d = (p - T[r0 + r]) * scale;
    }
    s.dy[r] = d;
  }
  __syncthreads();
  // dw3, db3, dz2, db2
  for (int c = tid; c < kHid; c += blockDim.x) {
    float gw = 0.f, gb = 0.f;
    for (int r = 0; r < kRows; r++) {
      const float h = __bfloat162float(s.h2[r * kHid + c]);
      gw += s.dy[r] * h;
      const __nv_bfloat16 dz =
          __float2bfloat16(h > 0.f ? s.dy[r] * s.w3[c] : 0.f);
      s.dz2[r * kHid + c] = dz;
      gb += __bfloat162float(dz);
    }
    atomicAdd(G + kW3 + c, gw);
    atomicAdd(G + kB2 + c, gb);
  }
  if (tid == 0) {
    float gb3 = 0.f;
    for (int r = 0; r < kRows; r++) gb3 += s.dy[r];
    atomicAdd(G + kB3, gb3);
  }
  __syncthreads();
  // ---- dW2 = h1^T dz2: 128 x 128 = 8 x 16 tiles, 16 per warp, K = 64
  for (int tile = warp; tile < 128; tile += 8) {
    const int m0 = (tile >> 4) * 16, n0 = (tile & 15) * 8;
    float c[4] = {0, 0, 0, 0};
    warp_mma([&](int i, int k) { return s.h1[k * kHid + m0 + i]; },
             [&](int k, int j) { return s.dz2[k * kHid + n0 + j]; }, kRows, c);
    for (int r = 0; r < 4; r++) {
      int row, col;
      frag_pos(r, &row, &col);
      atomicAdd(G + kW2 + (m0 + row) * kHid + n0 + col, c[r]);
    }
  }
  // ---- dz1 = (dz2 W2^T) masked: 64 x 128, K = 128
  for (int tile = warp; tile < 64; tile += 8) {
    const int m0 = (tile >> 4) * 16, n0 = (tile & 15) * 8;
    float c[4] = {0, 0, 0, 0};
    warp_mma([&](int i, int k) { return s.dz2[(m0 + i) * kHid + k]; },
             [&](int k, int j) { return s.w2[(n0 + j) * kHid + k]; }, kHid, c);
    for (int r = 0; r < 4; r++) {
      int row, col;
      frag_pos(r, &row, &col);
      const int at = (m0 + row) * kHid + n0 + col;
      s.dz1[at] = __float2bfloat16(
          __bfloat162float(s.h1[at]) > 0.f ? c[r] : 0.f);
    }
  }
  __syncthreads();
  // db1
  for (int c = tid; c < kHid; c += blockDim.x) {
    float gb = 0.f;
    for (int r = 0; r < kRows; r++) gb += __bfloat162float(s.dz1[r * kHid + c]);
    atomicAdd(G + kB1 + c, gb);
  }
  // ---- dW1 = x^T dz1: 32 x 128 = 2 x 16 tiles, 4 per warp, K = 64
  for (int tile = warp; tile < 32; tile += 8) {
    const int m0 = (tile >> 4) * 16, n0 = (tile & 15) * 8;
    float c[4] = {0, 0, 0, 0};
    warp_mma([&](int i, int k) { return s.x[k * kIn + m0 + i]; },
             [&](int k, int j) { return s.dz1[k * kHid + n0 + j]; }, kRows, c);
    for (int r = 0; r < 4; r++) {
      int row, col;
      frag_pos(r, &row, &col);
      atomicAdd(G + kW1 + (m0 + row) * kHid + n0 + col, c[r]);
    }
  }
}

// Adam on the fp32 master copy; refreshes the bf16 copies of W1 / W2 and
// clears the gradient
__global__ void k_adam(float *P, float *G, float *M, float *V, int np,
                       float lr, float b1, float b2, float eps, float c1,
                       float c2, __nv_bfloat16 *w1b, __nv_bfloat16 *w2b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float g = G[i];
  const float m = b1 * M[i] + (1.f - b1) * g;
  const float v = b2 * V[i] + (1.f - b2) * g * g;
  M[i] = m;
  V[i] = v;
  const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
  P[i] = p;
  G[i] = 0.f;
  if (i >= kW1 && i < kW1 + kIn * kHid) w1b[i - kW1] = __float2bfloat16(p);
  if (i >= kW2 && i < kW2 + kHid * kHid) w2b[i - kW2] = __float2bfloat16(p);
}

__global__ void k_refresh_bf16(const float *P, __nv_bfloat16 *w1b,
                               __nv_bfloat16 *w2b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kIn * kHid) w1b[i] = __float2bfloat16(P[kW1 + i]);
  if (i < kHid * kHid) w2b[i] = __float2bfloat16(P[kW2 + i]);
}

struct Mlp {
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
  __nv_bfloat16 *w1b = nullptr, *w2b = nullptr;
  float *dX = nullptr, *dT = nullptr, *dY = nullptr;
  long long cap = 0;
  long long step = 0;
  cudaStream_t s = nullptr;
};

std::unordered_map<long long, Mlp *> g_mlps;
long long g_mlp_next = 1;

Mlp *get(long long h) {
  auto it = g_mlps.find(h);
  return it == g_mlps.end() ? nullptr : it->second;
}

int ensure_cap(Mlp *m, long long n) {
  if (n <= m->cap) return 0;
  if (m->dX) cudaFree(m->dX);
  if (m->dT) cudaFree(m->dT);
  if (m->dY) cudaFree(m->dY);
  m->dX = m->dT = m->dY = nullptr;
  CC_CK(cudaMalloc(&m->dX, (size_t)n * kIn * 4));
  CC_CK(cudaMalloc(&m->dT, (size_t)n * 4));
  CC_CK(cudaMalloc(&m->dY, (size_t)n * 4));
  m->cap = n;
  return 0;
}

int launch_mlp(Mlp *m, bool train, const float *X, const float *T, int n,
               float scale, float *Y) {
  const size_t smem = sizeof(MlpSmem);
  static bool attr = false;
  if (!attr) {
    CC_CK(cudaFuncSetAttribute((const void *)k_mlp<true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
    CC_CK(cudaFuncSetAttribute((const void *)k_mlp<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
    attr = true;
  }
  const int grid = (n + kRows - 1) / kRows;
  if (train)
    k_mlp<true><<<grid, 256, smem, m->s>>>(m->P, m->w1b, m->w2b, X, T, n,
                                           scale, Y, m->G);
  else
    k_mlp<false><<<grid, 256, smem, m->s>>>(m->P, m->w1b, m->w2b, X, T, n,
                                            scale, Y, m->G);
  CC_CK(cudaGetLastError());
  return 0;
}

// splitmix64: deterministic host initialisation
uint64_t mix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

long long dct_mlp_create(unsigned long long seed) {
  Mlp *m = new Mlp();
  if (cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->P, kParams * 4) != cudaSuccess ||
      cudaMalloc(&m->G, kParams * 4) != cudaSuccess ||
      cudaMalloc(&m->M, kParams * 4) != cudaSuccess ||
      cudaMalloc(&m->V, kParams * 4) != cudaSuccess ||
      cudaMalloc(&m->w1b, kIn * kHid * 2) != cudaSuccess ||
      cudaMalloc(&m->w2b, kHid * kHid * 2) != cudaSuccess) {
    delete m;
    return -1;
  }
  // He-uniform weights, zero biases
  std::vector<float> p(kParams, 0.f);
  uint64_t st = seed;
  auto uni = [&](float a) {
    return (float)((mix(st) >> 11) * (1.0 / 9007199254740992.0) * 2 - 1) * a;
  };
  for (int i = 0; i < kIn * kHid; i++) p[kW1 + i] = uni(sqrtf(6.f / kIn));
  for (int i = 0; i < kHid * kHid; i++) p[kW2 + i] = uni(sqrtf(6.f / kHid));
  for (int i = 0; i < kHid; i++) p[kW3 + i] = uni(sqrtf(6.f / kHid) * 0.5f);
  cudaMemcpy(m->P, p.data(), kParams * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->G, 0, kParams * 4);
  cudaMemset(m->M, 0, kParams * 4);
  cudaMemset(m->V, 0, kParams * 4);
  k_refresh_bf16<<<(kHid * kHid + 255) / 256, 256, 0, m->s>>>(m->P, m->w1b,
                                                             m->w2b);
  cudaStreamSynchronize(m->s);
  const long long h = g_mlp_next++;
  g_mlps[h] = m;
  return h;
}

int dct_mlp_params(long long h, float *get_out, const float *set_in) {
  Mlp *m = get(h);
  if (!m) return -1;
  if (set_in) {
    CC_CK(cudaMemcpyAsync(m->P, set_in, kParams * 4, cudaMemcpyHostToDevice,
                          m->s));
    k_refresh_bf16<<<(kHid * kHid + 255) / 256, 256, 0, m->s>>>(m->P, m->w1b,
                                                               m->w2b);
    CC_CK(cudaGetLastError());
  }
  if (get_out)
    CC_CK(cudaMemcpyAsync(get_out, m->P, kParams * 4, cudaMemcpyDeviceToHost,
                          m->s));
  CC_CK(cudaStreamSynchronize(m->s));
  return kParams;
}

int dct_mlp_grad(long long h, const float *X, const float *T, int n,
                 float *grad_out) {
  Mlp *m = get(h);
  if (!m || n < 1 || !X || !T || !grad_out) return -1;
  int rc = ensure_cap(m, n);
  if (rc) return rc;
  CC_CK(cudaMemcpyAsync(m->dX, X, (size_t)n * kIn * 4,
                        cudaMemcpyHostToDevice, m->s));
  CC_CK(cudaMemcpyAsync(m->dT, T, (size_t)n * 4, cudaMemcpyHostToDevice,
                        m->s));
  CC_CK(cudaMemsetAsync(m->G, 0, kParams * 4, m->s));
  rc = launch_mlp(m, true, m->dX, m->dT, n, 1.f / n, m->dY);
  if (rc) return rc;
  CC_CK(cudaMemcpyAsync(grad_out, m->G, kParams * 4, cudaMemcpyDeviceToHost,
                        m->s));
  CC_CK(cudaMemsetAsync(m->G, 0, kParams * 4, m->s));
  CC_CK(cudaStreamSynchronize(m->s));
  return kParams;
}

int dct_mlp_train(long long h, const float *X, const float *T, int n,
                  int epochs, int batch, float lr, unsigned long long seed) {
  Mlp *m = get(h);
  if (!m || n < 1 || !X || !T || epochs < 1 || batch < 1) return -1;
  int rc = ensure_cap(m, n);
  if (rc) return rc;
  // shuffle once per epoch on the host, upload the permuted set
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  std::vector<float> xs((size_t)n * kIn), ts(n);
  uint64_t st = seed;
  for (int e = 0; e < epochs; e++) {
    for (int i = n - 1; i > 0; i--) {
      const int j = (int)(mix(st) % (uint64_t)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    for (int i = 0; i < n; i++) {
      memcpy(&xs[(size_t)i * kIn], X + (size_t)perm[i] * kIn, kIn * 4);
      ts[i] = T[perm[i]];
    }
    CC_CK(cudaMemcpyAsync(m->dX, xs.data(), xs.size() * 4,
                          cudaMemcpyHostToDevice, m->s));
    CC_CK(cudaMemcpyAsync(m->dT, ts.data(), ts.size() * 4,
                          cudaMemcpyHostToDevice, m->s));
    for (int b0 = 0; b0 < n; b0 += batch) {
      const int nb = n - b0 < batch ? n - b0 : batch;
      rc = launch_mlp(m, true, m->dX + (size_t)b0 * kIn, m->dT + b0, nb,
                      1.f / nb, nullptr);
      if (rc) return rc;
      m->step++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - powf(b1, (float)m->step);
      const float c2 = 1.f - powf(b2, (float)m->step);
      k_adam<<<(kParams + 255) / 256, 256, 0, m->s>>>(
          m->P, m->G, m->M, m->V, kParams, lr, b1, b2, 1e-8f, c1, c2, m->w1b,
          m->w2b);
      CC_CK(cudaGetLastError());
    }
    CC_CK(cudaStreamSynchronize(m->s));      // xs / ts reused next epoch
  }
  return 0;
}

int dct_mlp_predict(long long h, const float *X, int n, float *out) {
  Mlp *m = get(h);
  if (!m || n < 0 || (n && (!X || !out))) return -1;
  if (!n) return 0;
  int rc = ensure_cap(m, n);
  if (rc) return rc;
  CC_CK(cudaMemcpyAsync(m->dX, X, (size_t)n * kIn * 4,
                        cudaMemcpyHostToDevice, m->s));
  rc = launch_mlp(m, false, m->dX, nullptr, n, 0.f, m->dY);
  if (rc) return rc;
  CC_CK(cudaMemcpyAsync(out, m->dY, (size_t)n * 4, cudaMemcpyDeviceToHost,
                        m->s));
  CC_CK(cudaStreamSynchronize(m->s));
  return 0;
}

int dct_mlp_free(long long h) {
  Mlp *m = get(h);
  if (!m) return -1;
  cudaStreamSynchronize(m->s);
  cudaFree(m->P); cudaFree(m->G); cudaFree(m->M); cudaFree(m->V);
  cudaFree(m->w1b); cudaFree(m->w2b);
  if (m->dX) cudaFree(m->dX);
  if (m->dT) cudaFree(m->dT);
  if (m->dY) cudaFree(m->dY);
  cudaStreamDestroy(m->s);
  g_mlps.erase(h);
  delete m;
  return 0;
}

}  // extern "C"
