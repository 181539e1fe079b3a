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

/* The network: `heads` independent MLPs IN -> HIDDEN -> HIDDEN -> HIDDEN -> OUT, GELU
   after every hidden layer.  Weights and activations are bf16 with FP32 accumulation; the
   optimizer (Adam) keeps FP32 master weights.  Parameters of one head, in this order:
   W1 (HIDDEN x IN, row-major), b1, W2 (HIDDEN x HIDDEN), b2, W3, b3, W4 (OUT x HIDDEN),
   b4 -- SPH_MLP_NPARAMS floats; heads follow each other.  Loss: mean squared error over
   the batch and the OUT outputs, per head.  Arrays named x, y, out are device pointers:
   x is batch x IN, y is batch x OUT, out is heads x n x OUT (FP32).  The network's
   kernels run on the legacy default stream, ordered with the caller's default-stream
   work that produces x and y. */
#define SPH_MLP_IN 6
#define SPH_MLP_HIDDEN 256
#define SPH_MLP_OUT 4
#define SPH_MLP_NPARAMS (256 * 6 + 256 + 2 * (256 * 256 + 256) + 4 * 256 + 4)
typedef struct sph_mlp sph_mlp;

int sph_mlp_num_params(void);
/* max_batch % 128 == 0; the initial weights follow PyTorch's default for linear layers,
   drawn from a counter-based generator keyed by (seed, head, parameter index). */
sph_status sph_mlp_create(int heads, int max_batch, unsigned long long seed, int device,
                          sph_mlp** out);
void sph_mlp_destroy(sph_mlp* m);
sph_status sph_mlp_get_params(sph_mlp* m, float* host);
sph_status sph_mlp_set_params(sph_mlp* m, const float* host);
/* One Adam step (lr; betas 0.9, 0.999; eps 1e-8) on a batch (batch % 128 == 0, at most
   max_batch).  With loss_host (heads floats) the call waits and returns each head's loss
   before the update; without it the step stays asynchronous. */
sph_status sph_mlp_train_step(sph_mlp* m, const float* x, const float* y, int batch, float lr,
                              float* loss_host);
/* Loss and gradients of every head on a batch, without an update (grads_host: heads x
   SPH_MLP_NPARAMS floats, may be NULL). */
sph_status sph_mlp_gradients(sph_mlp* m, const float* x, const float* y, int batch,
                             float* grads_host, float* loss_host);
/* Outputs of every head for n samples (n % 128 == 0). */
sph_status sph_mlp_predict(sph_mlp* m, const float* x, int n, float* out);
/* Waits for the network's stream; SPH_ERR_TIMEOUT if a kernel gave up on its MMAs. */
sph_status sph_mlp_synchronize(sph_mlp* m);

#ifdef __cplusplus
}
#endif

#endif /* SPH_MLP_H */
