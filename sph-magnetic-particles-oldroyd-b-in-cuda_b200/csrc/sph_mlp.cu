// sph_mlp.cu -- the surrogate network's kernels and C ABI (include/sph_mlp.h): an ensemble
// of independent MLPs ("heads") 6 -> 256 -> 256 -> 256 -> 4 with GELU, BF16 weights and
// activations, FP32 accumulation, trained with Adam on FP32 master weights.
//
// The 256 x 256 layers (forward, input gradient and weight gradient) run on the tensor
// cores through sph_tc_gemm.cuh (tcgen05, accumulators in TMEM); the 6-wide input layer
// and the 4-wide output layer are a few hundred multiply-adds per sample and run on the
// CUDA cores.  Every reduction has a fixed order: training is bit-reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <string>
#include <vector>

#include "sph_mlp.h"
#include "sph_tc_gemm.cuh"

using sph::tc::GemmArgs;
namespace tc = sph::tc;

namespace {

constexpr int IN = SPH_MLP_IN, HID = SPH_MLP_HIDDEN, OUT = SPH_MLP_OUT;
// parameter layout of one head (FP32 master copy, gradients and Adam moments alike)
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + HID * IN;
constexpr int OFF_W2 = OFF_B1 + HID;
constexpr int OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_W3 = OFF_B2 + HID;
constexpr int OFF_B3 = OFF_W3 + HID * HID;
constexpr int OFF_W4 = OFF_B3 + HID;
constexpr int OFF_B4 = OFF_W4 + OUT * HID;
constexpr int NPARAM = OFF_B4 + OUT;
static_assert(NPARAM == SPH_MLP_NPARAMS, "parameter count");

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
         z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

// Epilogues of the tensor-core GEMM (one thread = one row of the 128 x N tile).
enum Epi { kEpiStore = 0, kEpiForward = 1, kEpiBackward = 2 };
struct EpiArgs {
  float* C;                 // kEpiStore: FP32 result, ldc = N
  long long strideC;
  long long strideSplit;    // kEpiStore with split K: distance between the slices' results
  const float* bias;        // kEpiForward: + bias[col], then GELU
  long long strideBias;
  const float* Zin;         // kEpiBackward: GELU'(Zin) of the layer below
  long long strideZ;
  float* Zout;              // kEpiForward: pre-activation (FP32) kept for the backward pass
  __nv_bfloat16* H;         // activation (bf16), row-major
  __nv_bfloat16* Ht;        // the same, transposed (column-major), leading dimension M
  long long strideH;
};

template <int EPI>
__global__ void __launch_bounds__(128, 1) k_gemm(GemmArgs g, EpiArgs e) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_sh;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tmem_sh, tc::kTmemCols);
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_sh;
  const bool ok = __syncthreads_and(tc::gemm_mainloop(g, smem, bar, tmem));
  if (ok) {
    const int head = blockIdx.y;
    const int row = tc::tile_m0(g) + threadIdx.x, n0 = tc::tile_n0(g);
    const int N = g.N, M = g.M;
    for (int t0 = 0; t0 < g.ntile; t0 += 16) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)t0, v);
      const int c0 = n0 + t0;  // output column
      if (EPI == kEpiStore) {
        float* c = e.C + blockIdx.z * e.strideSplit + head * e.strideC + (size_t)row * N + c0;
#pragma unroll
        for (int q = 0; q < 16; q += 4)
          *reinterpret_cast<float4*>(c + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
      } else {
        __nv_bfloat16 hv[16];
        if (EPI == kEpiForward) {
          const float* bias = e.bias + head * e.strideBias + c0;
          float* z = e.Zout + head * e.strideZ + (size_t)row * N + c0;
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float zz = v[q] + bias[q];
            z[q] = zz;
            hv[q] = __float2bfloat16(gelu(zz));
          }
        } else {
          const float* z = e.Zin + head * e.strideZ + (size_t)row * N + c0;
#pragma unroll
          for (int q = 0; q < 16; ++q) hv[q] = __float2bfloat16(v[q] * gelu_grad(z[q]));
        }
        __nv_bfloat16* h = e.H + head * e.strideH + (size_t)row * N + c0;
#pragma unroll
        for (int q = 0; q < 16; q += 8) *reinterpret_cast<uint4*>(h + q) = *reinterpret_cast<uint4*>(hv + q);
        __nv_bfloat16* ht = e.Ht + head * e.strideH;
#pragma unroll
        for (int q = 0; q < 16; ++q) ht[(size_t)(c0 + q) * M + row] = hv[q];
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(g.err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_free(tmem, tc::kTmemCols);
  }
}

// Sum of the split-K slices of a weight gradient in slice order (a fixed order: training
// stays bit-reproducible): C[h * strideC + i] = sum over s of ws[(s * heads + h) * MN + i].
__global__ void k_sum_splits(const float* __restrict__ ws, int splits, int heads, int MN,
                             float* __restrict__ C, long long strideC) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, h = blockIdx.y;
  if (i >= MN) return;
  float acc = ws[(size_t)h * MN + i];
  for (int s = 1; s < splits; ++s) acc += ws[((size_t)s * heads + h) * MN + i];
  C[h * strideC + i] = acc;
}

// ---- CUDA-core layers (6-wide input, 4-wide output) ----

// z1 = W1 x + b1, h1 = GELU(z1): thread per (sample, neuron), head = blockIdx.y.
__global__ void k_layer1(const float* __restrict__ x, int B, const float* __restrict__ params,
                         const __nv_bfloat16* __restrict__ w1b, float* Z1, __nv_bfloat16* H1,
                         __nv_bfloat16* H1t) {
  const int head = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * HID) return;
  const int b = t / HID, j = t % HID;
  const float* P = params + (size_t)head * NPARAM;
  const __nv_bfloat16* w = w1b + (size_t)head * HID * IN + j * IN;
  float z = P[OFF_B1 + j];
#pragma unroll
  for (int i = 0; i < IN; ++i) z = fmaf(__bfloat162float(w[i]), x[(size_t)b * IN + i], z);
  const size_t o = (size_t)head * B * HID;
  Z1[o + (size_t)b * HID + j] = z;
  const __nv_bfloat16 h = __float2bfloat16(gelu(z));
  H1[o + (size_t)b * HID + j] = h;
  H1t[o + (size_t)j * B + b] = h;
}

// out = W4 h3 + b4 and, with targets, the squared error and dL/dout: thread per sample.
__global__ void k_layer4(const __nv_bfloat16* __restrict__ H3, int B,
                         const float* __restrict__ params, const __nv_bfloat16* __restrict__ w4b,
                         const float* __restrict__ y, float* out, float* dout, float* sqerr) {
  const int head = blockIdx.y;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float* P = params + (size_t)head * NPARAM;
  const __nv_bfloat16* h = H3 + (size_t)head * B * HID + (size_t)b * HID;
  const __nv_bfloat16* w = w4b + (size_t)head * OUT * HID;
  float acc[OUT];
#pragma unroll
  for (int o = 0; o < OUT; ++o) acc[o] = 0.0f;
  for (int k = 0; k < HID; ++k) {
    const float hk = __bfloat162float(h[k]);
#pragma unroll
    for (int o = 0; o < OUT; ++o) acc[o] = fmaf(__bfloat162float(w[o * HID + k]), hk, acc[o]);
  }
  float se = 0.0f;
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
    const float v = acc[o] + P[OFF_B4 + o];
    out[((size_t)head * B + b) * OUT + o] = v;
    if (y) {
      const float r = v - y[(size_t)b * OUT + o];
      se += r * r;
      dout[((size_t)head * B + b) * OUT + o] = 2.0f * r / (float)(B * OUT);
    }
  }
  if (y) sqerr[(size_t)head * B + b] = se;
}

// dz3 = (W4^T dout) * GELU'(z3): thread per (sample, neuron).
__global__ void k_layer4_back(const float* __restrict__ dout, int B,
                              const __nv_bfloat16* __restrict__ w4b, const float* __restrict__ Z3,
                              __nv_bfloat16* DZ3, __nv_bfloat16* DZ3t) {
  const int head = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * HID) return;
  const int b = t / HID, k = t % HID;
  const float* d = dout + ((size_t)head * B + b) * OUT;
  const __nv_bfloat16* w = w4b + (size_t)head * OUT * HID;
  float g = 0.0f;
#pragma unroll
  for (int o = 0; o < OUT; ++o) g = fmaf(d[o], __bfloat162float(w[o * HID + k]), g);
  const size_t off = (size_t)head * B * HID;
  const __nv_bfloat16 v = __float2bfloat16(g * gelu_grad(Z3[off + (size_t)b * HID + k]));
  DZ3[off + (size_t)b * HID + k] = v;
  DZ3t[off + (size_t)k * B + b] = v;
}

// Small weight gradients, fixed summation order over the batch: thread per output
// element.  dW4[o][k] = sum_b dout[b][o] h3[b][k], db4[o] = sum_b dout[b][o];
// dW1[j][i] = sum_b dz1[b][j] x[b][i], db1[j] = sum_b dz1[b][j];
// db (hidden) = column sums of a bf16 dz.
__global__ void k_small_grads(const float* __restrict__ dout, const __nv_bfloat16* __restrict__ H3,
                              const __nv_bfloat16* __restrict__ DZ1,
                              const __nv_bfloat16* __restrict__ DZ2,
                              const __nv_bfloat16* __restrict__ DZ3, const float* __restrict__ x,
                              int B, float* grads) {
  const int head = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float* G = grads + (size_t)head * NPARAM;
  const size_t hoff = (size_t)head * B * HID;
  // task ranges: dW4 (OUT*HID), db4 (OUT), dW1 (HID*IN), db1, db2, db3 (HID each)
  int r = t;
  if (r < OUT * HID) {
    const int o = r / HID, k = r % HID;
    float s = 0.0f;
    for (int b = 0; b < B; ++b)
      s = fmaf(dout[((size_t)head * B + b) * OUT + o], __bfloat162float(H3[hoff + (size_t)b * HID + k]), s);
    G[OFF_W4 + r] = s;
    return;
  }
  r -= OUT * HID;
  if (r < OUT) {
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += dout[((size_t)head * B + b) * OUT + r];
    G[OFF_B4 + r] = s;
    return;
  }
  r -= OUT;
  if (r < HID * IN) {
    const int j = r / IN, i = r % IN;
    float s = 0.0f;
    for (int b = 0; b < B; ++b)
      s = fmaf(__bfloat162float(DZ1[hoff + (size_t)b * HID + j]), x[(size_t)b * IN + i], s);
    G[OFF_W1 + r] = s;
    return;
  }
  r -= HID * IN;
  if (r < 3 * HID) {
    const int which = r / HID, j = r % HID;
    const __nv_bfloat16* DZ = which == 0 ? DZ1 : which == 1 ? DZ2 : DZ3;
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += __bfloat162float(DZ[hoff + (size_t)b * HID + j]);
    G[(which == 0 ? OFF_B1 : which == 1 ? OFF_B2 : OFF_B3) + j] = s;
  }
}
constexpr int kSmallTasks = OUT * HID + OUT + HID * IN + 3 * HID;

// Adam on the FP32 master parameters (all heads, all tensors in one flat array).
__global__ void k_adam(float* params, const float* grads, float* m, float* v, int n, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float g = grads[t];
  const float mt = b1 * m[t] + (1.0f - b1) * g;
  const float vt = b2 * v[t] + (1.0f - b2) * g * g;
  m[t] = mt;
  v[t] = vt;
  params[t] -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
}

// bf16 copies of the weights used by the kernels: W1, W4 as they are, W2 and W3 also
// transposed (operand B of the input-gradient GEMMs).
__global__ void k_cast_weights(const float* params, int heads, __nv_bfloat16* w1b,
                               __nv_bfloat16* w2b, __nv_bfloat16* w2tb, __nv_bfloat16* w3b,
                               __nv_bfloat16* w3tb, __nv_bfloat16* w4b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int per = HID * HID;
  if (t >= heads * per) return;
  const int head = t / per, e = t % per, r = e / HID, c = e % HID;
  const float* P = params + (size_t)head * NPARAM;
  const size_t o = (size_t)head * per;
  w2b[o + e] = __float2bfloat16(P[OFF_W2 + e]);
  w2tb[o + (size_t)c * HID + r] = __float2bfloat16(P[OFF_W2 + e]);
  w3b[o + e] = __float2bfloat16(P[OFF_W3 + e]);
  w3tb[o + (size_t)c * HID + r] = __float2bfloat16(P[OFF_W3 + e]);
  if (e < HID * IN) w1b[(size_t)head * HID * IN + e] = __float2bfloat16(P[OFF_W1 + e]);
  if (e < OUT * HID) w4b[(size_t)head * OUT * HID + e] = __float2bfloat16(P[OFF_W4 + e]);
}

// Per-head sum of squared errors in fixed order (one block per head).
__global__ void k_loss(const float* sqerr, int B, float* loss) {
  __shared__ float sh[256];
  const int head = blockIdx.x;
  float s = 0.0f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += sqerr[(size_t)head * B + b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[head] = sh[0] / (float)(B * OUT);
}

// C = A . B^T in FP32 (the tensor-core GEMM with a plain store epilogue).
__global__ void __launch_bounds__(128, 1) k_gemm_f32(GemmArgs g, float* C, int ldc,
                                                      long long strideC) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_sh;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tmem_sh, tc::kTmemCols);
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_sh;
  const bool ok = __syncthreads_and(tc::gemm_mainloop(g, smem, bar, tmem));
  if (ok) {
    const int row = tc::tile_m0(g) + threadIdx.x;
    float* c = C + blockIdx.y * strideC + (size_t)row * ldc + tc::tile_n0(g);
    for (int c0 = 0; c0 < g.ntile; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) c[c0 + q] = v[q];
    }
  } else if (threadIdx.x == 0) {
    atomicExch(g.err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_free(tmem, tc::kTmemCols);
  }
}

bool gemm_shape_ok(int M, int N, int K) {
  return M > 0 && N > 0 && K > 0 && M % tc::kTileM == 0 && N % 16 == 0 && N <= tc::kMaxN &&
         K % tc::kChunkK == 0;
}

}  // namespace

struct sph_mlp {
  int heads = 0, max_batch = 0, device = 0;
  int nsm = 148;  // multiprocessors of the device
  cudaStream_t stream = nullptr;  // cudaStreamLegacy
  std::vector<void*> allocs;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16 *w1b = nullptr, *w2b = nullptr, *w2tb = nullptr, *w3b = nullptr, *w3tb = nullptr,
                *w4b = nullptr;
  float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr;
  __nv_bfloat16 *h1 = nullptr, *h1t = nullptr, *h2 = nullptr, *h2t = nullptr, *h3 = nullptr,
                *h3t = nullptr, *dz1 = nullptr, *dz1t = nullptr, *dz2 = nullptr, *dz2t = nullptr,
                *dz3 = nullptr, *dz3t = nullptr;
  float *out = nullptr, *dout = nullptr, *sqerr = nullptr, *loss = nullptr;
  float* ws = nullptr;  // split-K slices of a weight gradient (kMaxSplits x heads x HID x HID)
  int* err = nullptr;
  long long step = 0;
};

namespace {

template <typename T>
bool mlp_alloc(sph_mlp* c, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return false;
  cudaMemsetAsync(q, 0, (n ? n : 1) * sizeof(T), c->stream);
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return true;
}

void mlp_free(sph_mlp* c) {
  if (!c) return;
  for (void* p : c->allocs) cudaFree(p);
  delete c;
}

// splitmix64: the initial weights depend only on (seed, head, tensor, index)
double uniform01(uint64_t key) {
  uint64_t z = key + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// PyTorch-style default initialisation of a linear layer: U(-1/sqrt(fan_in), +1/sqrt(fan_in))
// for weights and biases.
void init_params(std::vector<float>& P, int heads, unsigned long long seed) {
  struct T { int off, n, fan_in; };
  const T t[] = {{OFF_W1, HID * IN, IN},   {OFF_B1, HID, IN},   {OFF_W2, HID * HID, HID},
                 {OFF_B2, HID, HID},       {OFF_W3, HID * HID, HID}, {OFF_B3, HID, HID},
                 {OFF_W4, OUT * HID, HID}, {OFF_B4, OUT, HID}};
  for (int h = 0; h < heads; ++h)
    for (int k = 0; k < 8; ++k) {
      const double bound = 1.0 / std::sqrt((double)t[k].fan_in);
      for (int i = 0; i < t[k].n; ++i) {
        const uint64_t key = ((uint64_t)seed * 1000003ull + (uint64_t)h) * 1315423911ull +
                             (uint64_t)(t[k].off + i);
        P[(size_t)h * NPARAM + t[k].off + i] = (float)((2.0 * uniform01(key) - 1.0) * bound);
      }
    }
}

template <int EPI>
int gemm_launch(sph_mlp* c, const __nv_bfloat16* A, long long sA, int lda, const __nv_bfloat16* B,
                long long sB, int ldb, int M, int N, int K, const EpiArgs& e, int splits = 1) {
  GemmArgs g;
  g.A = A;
  g.B = B;
  g.strideA = sA;
  g.strideB = sB;
  g.lda = lda;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  // forward and input-gradient GEMMs whose row tiles alone leave SMs idle (a 1024-sample
  // batch: 8 row tiles x 5 heads = 40 CTAs): two column tiles per row tile
  g.ntile = (EPI != kEpiStore && N == 256 && (M / tc::kTileM) * c->heads < c->nsm) ? 128 : N;
  g.err = c->err;
  k_gemm<EPI><<<dim3(M / tc::kTileM * (N / g.ntile), c->heads, splits), 128, tc::kSmemBytes,
                 c->stream>>>(g, e);
  return cudaGetLastError() != cudaSuccess;
}

// Weight gradient dW = dZ^T H (M = N = HID, K = the batch) into grads + off of every head.
// The K = batch reduction is split over up to kMaxSplits CTAs per output tile (2 tiles per
// head leave most SMs idle otherwise); the slices are summed in order by k_sum_splits.
constexpr int kMaxSplits = 8;
int weight_grad(sph_mlp* c, const __nv_bfloat16* dzt, const __nv_bfloat16* ht, int B, int off) {
  const long long act = (long long)B * HID;
  int splits = kMaxSplits;
  while (splits > 1 && B % (tc::kChunkK * splits) != 0) splits /= 2;
  EpiArgs e{};
  if (splits == 1) {
    e.C = c->grads + off;
    e.strideC = NPARAM;
    return gemm_launch<kEpiStore>(c, dzt, act, B, ht, act, B, HID, HID, B, e);
  }
  const int MN = HID * HID;
  e.C = c->ws;
  e.strideC = MN;
  e.strideSplit = (long long)c->heads * MN;
  if (gemm_launch<kEpiStore>(c, dzt, act, B, ht, act, B, HID, HID, B, e, splits)) return 1;
  k_sum_splits<<<dim3((MN + 255) / 256, c->heads), 256, 0, c->stream>>>(c->ws, splits, c->heads,
                                                                          MN, c->grads + off, NPARAM);
  return cudaGetLastError() != cudaSuccess;
}

// Forward pass of every head on B samples (x: B x IN, device); with y (B x OUT) also the
// squared errors and dL/dout.
int forward(sph_mlp* c, const float* x, const float* y, int B) {
  const int H = c->heads;
  const long long act = (long long)B * HID;
  k_layer1<<<dim3((B * HID + 255) / 256, H), 256, 0, c->stream>>>(x, B, c->params, c->w1b, c->z1,
                                                                   c->h1, c->h1t);
  if (cudaGetLastError() != cudaSuccess) return 1;
  EpiArgs e{};
  e.strideBias = NPARAM;
  e.strideZ = act;
  e.strideH = act;
  e.bias = c->params + OFF_B2;
  e.Zout = c->z2;
  e.H = c->h2;
  e.Ht = c->h2t;
  if (gemm_launch<kEpiForward>(c, c->h1, act, HID, c->w2b, (long long)HID * HID, HID, B, HID, HID, e))
    return 1;
  e.bias = c->params + OFF_B3;
  e.Zout = c->z3;
  e.H = c->h3;
  e.Ht = c->h3t;
  if (gemm_launch<kEpiForward>(c, c->h2, act, HID, c->w3b, (long long)HID * HID, HID, B, HID, HID, e))
    return 1;
  k_layer4<<<dim3((B + 127) / 128, H), 128, 0, c->stream>>>(c->h3, B, c->params, c->w4b, y, c->out,
                                                            c->dout, c->sqerr);
  return cudaGetLastError() != cudaSuccess;
}

// Backward pass after forward(x, y): gradients of the mean squared error of every head.
int backward(sph_mlp* c, const float* x, int B) {
  const int H = c->heads;
  const long long act = (long long)B * HID;
  k_layer4_back<<<dim3((B * HID + 255) / 256, H), 256, 0, c->stream>>>(c->dout, B, c->w4b, c->z3,
                                                                       c->dz3, c->dz3t);
  if (cudaGetLastError() != cudaSuccess) return 1;
  EpiArgs e{};
  e.strideC = NPARAM;
  e.strideZ = act;
  e.strideH = act;
  // dW3 = dz3^T h2, then dz2 = (dz3 W3) * GELU'(z2)
  if (weight_grad(c, c->dz3t, c->h2t, B, OFF_W3)) return 1;
  e.Zin = c->z2;
  e.H = c->dz2;
  e.Ht = c->dz2t;
  if (gemm_launch<kEpiBackward>(c, c->dz3, act, HID, c->w3tb, (long long)HID * HID, HID, B, HID,
                                HID, e))
    return 1;
  // dW2 = dz2^T h1, then dz1 = (dz2 W2) * GELU'(z1)
  if (weight_grad(c, c->dz2t, c->h1t, B, OFF_W2)) return 1;
  e.Zin = c->z1;
  e.H = c->dz1;
  e.Ht = c->dz1t;
  if (gemm_launch<kEpiBackward>(c, c->dz2, act, HID, c->w2tb, (long long)HID * HID, HID, B, HID,
                                HID, e))
    return 1;
  k_small_grads<<<dim3((kSmallTasks + 127) / 128, H), 128, 0, c->stream>>>(
      c->dout, c->h3, c->dz1, c->dz2, c->dz3, x, B, c->grads);
  if (cudaGetLastError() != cudaSuccess) return 1;
  k_loss<<<H, 256, 0, c->stream>>>(c->sqerr, B, c->loss);
  return cudaGetLastError() != cudaSuccess;
}

int cast_weights(sph_mlp* c) {
  const int n = c->heads * HID * HID;
  k_cast_weights<<<(n + 255) / 256, 256, 0, c->stream>>>(c->params, c->heads, c->w1b, c->w2b,
                                                         c->w2tb, c->w3b, c->w3tb, c->w4b);
  return cudaGetLastError() != cudaSuccess;
}

sph_status finish(sph_mlp* c) {
  int e = 0;
  if (cudaMemcpyAsync(&e, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return SPH_ERR_CUDA;
  return e ? SPH_ERR_TIMEOUT : SPH_OK;
}

bool batch_ok(const sph_mlp* c, int B) { return B > 0 && B % tc::kTileM == 0 && B <= c->max_batch; }

}  // namespace

extern "C" {

sph_status sph_tc_gemm(const void* A, const void* B, float* C, int M, int N, int K, int heads,
                       void* stream) {
  if (!A || !B || !C || heads <= 0 || !gemm_shape_ok(M, N, K)) return SPH_ERR_STATE;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_gemm_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tc::kSmemBytes) != cudaSuccess)
      return SPH_ERR_CUDA;
    attr_set = true;
  }
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return SPH_ERR_NOMEM;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(err, 0, sizeof(int), st);
  GemmArgs g;
  g.A = static_cast<const __nv_bfloat16*>(A);
  g.B = static_cast<const __nv_bfloat16*>(B);
  g.strideA = (long long)M * K;
  g.strideB = (long long)N * K;
  g.lda = K;
  g.ldb = K;
  g.M = M;
  g.N = N;
  g.K = K;
  g.ntile = N;
  g.err = err;
  k_gemm_f32<<<dim3(M / tc::kTileM, heads), 128, tc::kSmemBytes, st>>>(g, C, N, (long long)M * N);
  int h = 0;
  sph_status s = SPH_OK;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    s = SPH_ERR_CUDA;
  else if (h)
    s = SPH_ERR_TIMEOUT;
  cudaFree(err);
  return s;
}

int sph_mlp_num_params(void) { return NPARAM; }

sph_status sph_mlp_create(int heads, int max_batch, unsigned long long seed, int device,
                          sph_mlp** out) {
  if (!out || heads <= 0 || max_batch <= 0 || max_batch % tc::kTileM != 0) return SPH_ERR_STATE;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return SPH_ERR_CUDA;
  sph_mlp* c = new sph_mlp;
  c->heads = heads;
  c->max_batch = max_batch;
  c->device = device;
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  // the legacy default stream: the caller's inputs (batches made by default-stream work,
  // e.g. a framework's allocator) are then ordered before, and their reuse after, the
  // network's kernels
  c->stream = cudaStreamLegacy;
  const size_t np = (size_t)heads * NPARAM, hh = (size_t)heads * HID * HID;
  const size_t act = (size_t)heads * max_batch * HID;
  bool ok = mlp_alloc(c, &c->params, np) && mlp_alloc(c, &c->grads, np) && mlp_alloc(c, &c->m, np) &&
            mlp_alloc(c, &c->v, np);
  ok = ok && mlp_alloc(c, &c->w1b, (size_t)heads * HID * IN) && mlp_alloc(c, &c->w2b, hh) &&
       mlp_alloc(c, &c->w2tb, hh) && mlp_alloc(c, &c->w3b, hh) && mlp_alloc(c, &c->w3tb, hh) &&
       mlp_alloc(c, &c->w4b, (size_t)heads * OUT * HID);
  ok = ok && mlp_alloc(c, &c->z1, act) && mlp_alloc(c, &c->z2, act) && mlp_alloc(c, &c->z3, act);
  for (__nv_bfloat16** p : {&c->h1, &c->h1t, &c->h2, &c->h2t, &c->h3, &c->h3t, &c->dz1, &c->dz1t,
                            &c->dz2, &c->dz2t, &c->dz3, &c->dz3t})
    ok = ok && mlp_alloc(c, p, act);
  ok = ok && mlp_alloc(c, &c->out, (size_t)heads * max_batch * OUT) &&
       mlp_alloc(c, &c->dout, (size_t)heads * max_batch * OUT) &&
       mlp_alloc(c, &c->sqerr, (size_t)heads * max_batch) && mlp_alloc(c, &c->loss, heads) &&
       mlp_alloc(c, &c->ws, (size_t)kMaxSplits * heads * HID * HID) && mlp_alloc(c, &c->err, 1);
  if (!ok) {
    mlp_free(c);
    return SPH_ERR_NOMEM;
  }
  for (const void* k : {(const void*)k_gemm<kEpiStore>, (const void*)k_gemm<kEpiForward>,
                        (const void*)k_gemm<kEpiBackward>})
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes) !=
        cudaSuccess) {
      mlp_free(c);
      return SPH_ERR_CUDA;
    }
  std::vector<float> P(np);
  init_params(P, heads, seed);
  if (cudaMemcpyAsync(c->params, P.data(), np * sizeof(float), cudaMemcpyHostToDevice, c->stream) !=
          cudaSuccess ||
      cast_weights(c) || cudaStreamSynchronize(c->stream) != cudaSuccess) {
    mlp_free(c);
    return SPH_ERR_CUDA;
  }
  *out = c;
  return SPH_OK;
}

void sph_mlp_destroy(sph_mlp* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  mlp_free(c);
}

sph_status sph_mlp_get_params(sph_mlp* c, float* host) {
  if (!c || !host) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  if (cudaMemcpyAsync(host, c->params, (size_t)c->heads * NPARAM * sizeof(float),
                      cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    return SPH_ERR_CUDA;
  return finish(c);
}

sph_status sph_mlp_set_params(sph_mlp* c, const float* host) {
  if (!c || !host) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  if (cudaMemcpyAsync(c->params, host, (size_t)c->heads * NPARAM * sizeof(float),
                      cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cast_weights(c))
    return SPH_ERR_CUDA;
  return finish(c);
}

sph_status sph_mlp_gradients(sph_mlp* c, const float* x, const float* y, int batch,
                             float* grads_host, float* loss_host) {
  if (!c || !x || !y || !batch_ok(c, batch)) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  if (forward(c, x, y, batch) || backward(c, x, batch)) return SPH_ERR_CUDA;
  if (grads_host && cudaMemcpyAsync(grads_host, c->grads, (size_t)c->heads * NPARAM * sizeof(float),
                                    cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    return SPH_ERR_CUDA;
  if (loss_host && cudaMemcpyAsync(loss_host, c->loss, (size_t)c->heads * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    return SPH_ERR_CUDA;
  return finish(c);
}

sph_status sph_mlp_train_step(sph_mlp* c, const float* x, const float* y, int batch, float lr,
                              float* loss_host) {
  if (!c || !x || !y || !batch_ok(c, batch)) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  if (forward(c, x, y, batch) || backward(c, x, batch)) return SPH_ERR_CUDA;
  c->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - (float)std::pow((double)b1, (double)c->step);
  const float bc2 = 1.0f - (float)std::pow((double)b2, (double)c->step);
  const int n = c->heads * NPARAM;
  k_adam<<<(n + 255) / 256, 256, 0, c->stream>>>(c->params, c->grads, c->m, c->v, n, lr, b1, b2,
                                                 1e-8f, bc1, bc2);
  if (cudaGetLastError() != cudaSuccess || cast_weights(c)) return SPH_ERR_CUDA;
  if (loss_host && cudaMemcpyAsync(loss_host, c->loss, (size_t)c->heads * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    return SPH_ERR_CUDA;
  if (!loss_host) return SPH_OK;  // asynchronous: errors surface at the next synchronising call
  return finish(c);
}

sph_status sph_mlp_predict(sph_mlp* c, const float* x, int n, float* out) {
  if (!c || !x || !out || n <= 0 || n % tc::kTileM != 0) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  for (int s = 0; s < n; s += c->max_batch) {
    const int B = std::min(c->max_batch, n - s);
    if (forward(c, x + (size_t)s * IN, nullptr, B)) return SPH_ERR_CUDA;
    for (int h = 0; h < c->heads; ++h)
      if (cudaMemcpyAsync(out + ((size_t)h * n + s) * OUT, c->out + (size_t)h * B * OUT,
                          (size_t)B * OUT * sizeof(float), cudaMemcpyDeviceToDevice,
                          c->stream) != cudaSuccess)
        return SPH_ERR_CUDA;
  }
  return finish(c);
}

sph_status sph_mlp_synchronize(sph_mlp* c) {
  if (!c) return SPH_ERR_STATE;
  cudaSetDevice(c->device);
  return finish(c);
}

}  // extern "C"
