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
#include <string>
#include <vector>

#include "sph_mlp.h"
#include "sph_tc_gemm.cuh"

using sph::tc::GemmArgs;
namespace tc = sph::tc;

namespace {

// C = A . B^T in FP32 (the tensor-core GEMM with a plain store epilogue).
__global__ void __launch_bounds__(128, 1) k_gemm_f32(GemmArgs g, float* C, int ldc,
                                                      long long strideC) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_sh;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tmem_sh, tc::kTmemCols);
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_sh;
  const bool ok = __syncthreads_and(tc::gemm_mainloop(g, smem, &bar, tmem));
  if (ok) {
    const int row = blockIdx.x * tc::kTileM + threadIdx.x;
    float* c = C + blockIdx.y * strideC + (size_t)row * ldc;
    for (int c0 = 0; c0 < g.N; c0 += 16) {
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

}  // extern "C"
