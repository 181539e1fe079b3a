/* sph_mlp.h -- the surrogate network of the parameter sweeps (no reference counterpart):
 * an ensemble of independent MLPs ("heads") mapping the six sweep inputs to the four
 * time-averaged observables, trained on the batched solver's own output with hand-written
 * sm_100a tensor-core kernels (tcgen05, BF16 operands, FP32 accumulation in tensor memory).
 */
#ifndef SPH_MLP_H
#define SPH_MLP_H

#include "sph_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C = A . B^T for `heads` independent problems on the tensor cores: A (M x K) and B
   (N x K) are bf16 device arrays with K contiguous, head h at A + h*M*K and B + h*N*K; C
   receives FP32 (M x N, row-major, head h at C + h*M*N).  M % 128 == 0, N % 16 == 0 and
   N <= 256, K % 64 == 0.  Synchronous on `stream` (a cudaStream_t; NULL = default);
   SPH_ERR_TIMEOUT if the kernel gave up waiting for its own MMAs. */
sph_status sph_tc_gemm(const void* A, const void* B, float* C, int M, int N, int K, int heads,
                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPH_MLP_H */
