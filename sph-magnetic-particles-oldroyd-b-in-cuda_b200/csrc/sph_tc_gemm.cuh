// sph_tc_gemm.cuh -- BF16 tensor-core GEMM for sm_100a (tcgen05 / TMEM), used by the
// surrogate network (sph_mlp.cu).
//
//   C[M x N] = A[M x K] . B[N x K]^T     A, B bf16 with K contiguous, C accumulated in FP32
//
// One CTA (4 warps) computes a 128 x N tile (N <= 256, a multiple of 16) for one "head"
// (blockIdx.y selects per-head operand offsets).  K is walked in chunks of 64: all threads
// copy the chunk of A (128 rows) and B (N rows) into shared memory in the canonical
// K-major, no-swizzle UMMA layout (core matrices of 8 rows x 16 bytes), one elected thread
// issues four tcgen05.mma (K = 16 each) accumulating into a 128-lane x N-column FP32 tile
// in tensor memory, and tcgen05.commit signals an mbarrier when they have read the chunk.
// The epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31, i.e. rows), and each thread finishes one row.
//
// Shared-memory descriptor (64 bits): start address >> 4 in [0,14), leading byte offset
// >> 4 in [16,30) (distance between the two core matrices along K of one K = 16 step:
// 128 B), stride byte offset >> 4 in [32,46) (distance between 8-row groups:
// kChunkK / 8 * 128 B), version 1 in [46,48), layout SWIZZLE_NONE (0) in [61,64).
// Instruction descriptor (kind::f16): D format F32 (bit 4), A and B format BF16 (bits 7,
// 10), both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace sph {
namespace tc {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kMaxN = 256;
constexpr int kSbo = kChunkK / 8 * 128;  // bytes between 8-row groups
// dynamic shared memory per CTA: A and B chunks, padded so that one CTA occupies an SM
// (its 256 TMEM columns are then never contended)
constexpr int kSmemBytes = 120 * 1024;
constexpr int kTmemCols = 256;
constexpr long long kSpinLimit = 1ll << 26;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t core_offset(int row, int k8) {
  return (uint32_t)((row >> 3) * kSbo + k8 * 128 + (row & 7) * 16);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  const uint64_t lbo = 128 >> 4, sbo = kSbo >> 4;
  return (uint64_t)((addr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, int cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   smem_u32(dst_smem)),
               "r"(cols)
               : "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, int cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Waits for the phase `parity` of the mbarrier to complete; gives up after kSpinLimit
// polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         int accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Operands of one GEMM launch; head h uses A + h * strideA, B + h * strideB (elements).
struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  long long strideA, strideB;
  int lda, ldb;  // row pitch (elements), multiples of 8
  int M, N, K;   // M % 128 == 0, N % 16 == 0 and N <= 256, K % 64 == 0
  int ntile;     // columns per CTA (N, or a divisor of N that is a multiple of 16)
  int* err;      // set to 1 when a wait gives up
};

// The CTA's output tile: blockIdx.x enumerates (row tile, column tile), column tile fastest.
__device__ __forceinline__ int tile_m0(const GemmArgs& g) {
  return (int)(blockIdx.x / (g.N / g.ntile)) * kTileM;
}
__device__ __forceinline__ int tile_n0(const GemmArgs& g) {
  return (int)(blockIdx.x % (g.N / g.ntile)) * g.ntile;
}

// Copies rows [r0, r0 + rows) x K-chunk [k0, k0 + 64) of a K-contiguous bf16 matrix into
// the canonical layout at dst: 16-byte cp.async copies, all of the thread's in flight at
// once (completed by cp_async_wait_all).
__device__ __forceinline__ void load_chunk(uint8_t* dst, const __nv_bfloat16* src, int ld, int r0,
                                           int rows, int k0) {
  for (int idx = threadIdx.x; idx < rows * (kChunkK / 8); idx += blockDim.x) {
    const int r = idx >> 3, k8 = idx & 7;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                     smem_u32(dst + core_offset(r, k8))),
                 "l"(src + (size_t)(r0 + r) * ld + k0 + k8 * 8)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// The main loop: leaves the 128 x ntile FP32 accumulator of this CTA's tile in TMEM columns
// [tmem, tmem + ntile).  With gridDim.z > 1 the CTA takes K slice blockIdx.z of gridDim.z equal
// slices (split K; K / gridDim.z a multiple of 64).  Two stages: the copies of chunk c + 1
// are in flight while the MMAs of chunk c run; bar[s] counts the MMA completions of stage s
// (a stage is refilled only after the MMAs that read it are done).  Returns false if an
// MMA completion was not observed in time.
constexpr int kStageA = kTileM * kChunkK * 2;
constexpr int kStageBytes = kStageA + kMaxN * kChunkK * 2;
static_assert(2 * kStageBytes <= kSmemBytes, "two stages of A and B chunks");
__device__ __forceinline__ bool gemm_mainloop(const GemmArgs& g, uint8_t* smem, uint64_t* bar,
                                              uint32_t tmem) {
  const int head = blockIdx.y;
  const int m0 = tile_m0(g), n0 = tile_n0(g);
  const int kslice = g.K / (int)gridDim.z;
  const int kb = (int)blockIdx.z * kslice;
  const int nch = kslice / kChunkK;
  const __nv_bfloat16* A = g.A + head * g.strideA;
  const __nv_bfloat16* B = g.B + head * g.strideB;
  const uint32_t idesc = idesc_bf16_f32(kTileM, g.ntile);
  auto fill = [&](int c) {
    uint8_t* st = smem + (c & 1) * kStageBytes;
    load_chunk(st, A, g.lda, m0, kTileM, kb + c * kChunkK);
    load_chunk(st + kStageA, B, g.ldb, n0, g.ntile, kb + c * kChunkK);
    cp_async_wait_all();
    // generic-proxy stores -> visible to the tensor core's (async proxy) reads
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
  };
  bool ok = true;
  int issued = -1;  // the last chunk whose MMAs were committed
  if (nch > 0) fill(0);
  for (int c = 0; c < nch; ++c) {
    const int s = c & 1;
    if (threadIdx.x == 0) {
      const uint32_t sa = smem_u32(smem + s * kStageBytes), sb = sa + kStageA;
#pragma unroll
      for (int q = 0; q < kChunkK / 16; ++q)
        mma_bf16(tmem, smem_desc(sa + q * 256), smem_desc(sb + q * 256), idesc,
                 (c > 0 || q > 0) ? 1 : 0);
      mma_commit(&bar[s]);
    }
    issued = c;
    if (c + 1 < nch) {
      // stage s ^ 1 was read by the MMAs of chunk c - 1 (commit number (c - 1) / 2 of its
      // barrier); every earlier commit of that barrier has been waited for.  Every thread
      // waits (bounded) and the block takes one decision, so that all threads leave the
      // loop together and meet the same barriers afterwards.
      if (c >= 1) {
        ok = __syncthreads_and(mbar_wait(&bar[s ^ 1], (uint32_t)(((c - 1) >> 1) & 1)) ? 1 : 0) != 0;
        fence_after_sync();
      }
      if (!ok) break;
      fill(c + 1);
    }
  }
  // The last commit completes after every MMA before it.  After a timeout this is the
  // drain: a second bounded wait, so that the caller frees TMEM only once the MMAs that
  // write it have finished (or this wait, too, has given up).  The previous commit of that
  // barrier was waited for before the chunk was issued, so its parity is unambiguous.
  if (issued >= 0) {
    const bool done = mbar_wait(&bar[issued & 1], (uint32_t)((issued >> 1) & 1));
    fence_after_sync();
    ok = ok && done;
  }
  return ok;
}

}  // namespace tc
}  // namespace sph
