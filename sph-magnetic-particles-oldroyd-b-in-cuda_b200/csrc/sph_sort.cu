// sph_sort.cu -- stable LSD radix sort of the cell keys.
//
// Replaces thrust::sort_by_key (reference src/system_neighbours_search.cu:56-58).  The
// keys are read in global-id order and the values are the ids themselves, so the result
// is the (cell, id) order that the reference's stable radix sort produces.
// Each pass: (1) per-tile digit histograms, (2) a three-kernel exclusive scan of the
// bucket-major histogram, (3) a stable scatter in which every warp ranks its items with
// __match_any_sync and per-warp bucket counters, so equal digits keep their input order.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;                       // items per thread per tile
constexpr int kTile = kThreads * kItems;         // 4096
constexpr int kMaxBits = 9;                      // up to 512 buckets per pass
constexpr int kMaxBuckets = 1 << kMaxBits;
constexpr int kScanChunk = 2048;                 // entries per scan block
static_assert(kTile == kSortTile && kMaxBuckets == kSortMaxBuckets &&
                  kScanChunk == kSortScanChunk,
              "sort geometry must match the histogram size callers reserve (sort_hist_ints)");

__global__ void __launch_bounds__(kThreads) k_radix_hist(const int* __restrict__ keys, int n,
                                                         int shift, int nbits, int ntiles,
                                                         int* __restrict__ hist) {
  __shared__ int h[kMaxBuckets];
  const int nb = 1 << nbits;
  for (int b = threadIdx.x; b < nb; b += kThreads) h[b] = 0;
  __syncthreads();
  const int base = blockIdx.x * kTile;
  for (int k = threadIdx.x; k < kTile; k += kThreads) {
    const int idx = base + k;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (nb - 1)], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += kThreads) hist[b * ntiles + blockIdx.x] = h[b];
}

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int* total) {
  // inclusive warp scan, then across warps
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kWarps ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kWarps) sh[lane] = s;
  }
  __syncthreads();
  const int warp_base = w > 0 ? sh[w - 1] : 0;
  if (total) *total = sh[kWarps - 1];
  const int r = warp_base + x - v;
  __syncthreads();
  return r;
}

// scan phase 1: sum of each chunk
__global__ void __launch_bounds__(kThreads) k_scan_sums(const int* __restrict__ a, int m,
                                                        int* __restrict__ sums) {
  __shared__ int sh[kWarps];
  const int base = blockIdx.x * kScanChunk;
  int s = 0;
  for (int k = threadIdx.x; k < kScanChunk; k += kThreads)
    if (base + k < m) s += a[base + k];
  int total;
  block_excl_scan(s, sh, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// scan phase 2: exclusive scan of the chunk sums (one block)
__global__ void __launch_bounds__(kThreads) k_scan_top(int* __restrict__ sums, int nchunks) {
  __shared__ int sh[kWarps];
  int carry = 0;
  for (int base = 0; base < nchunks; base += kThreads) {
    const int k = base + threadIdx.x;
    const int v = k < nchunks ? sums[k] : 0;
    int total;
    const int e = block_excl_scan(v, sh, &total);
    if (k < nchunks) sums[k] = carry + e;
    carry += total;
  }
}

// scan phase 3: exclusive scan inside each chunk plus the chunk's offset (in place)
__global__ void __launch_bounds__(kThreads) k_scan_apply(int* __restrict__ a, int m,
                                                         const int* __restrict__ sums) {
  __shared__ int sh[kWarps];
  constexpr int per = kScanChunk / kThreads;  // 8 consecutive entries per thread
  const int base = blockIdx.x * kScanChunk + threadIdx.x * per;
  int v[per];
  int s = 0;
#pragma unroll
  for (int q = 0; q < per; ++q) {
    v[q] = base + q < m ? a[base + q] : 0;
    s += v[q];
  }
  int run = sums[blockIdx.x] + block_excl_scan(s, sh, nullptr);
#pragma unroll
  for (int q = 0; q < per; ++q) {
    if (base + q < m) a[base + q] = run;
    run += v[q];
  }
}

__global__ void __launch_bounds__(kThreads)
    k_radix_scatter(const int* __restrict__ keys_in, const int* __restrict__ vals_in, int n,
                    int shift, int nbits, int ntiles, const int* __restrict__ offsets,
                    int* __restrict__ keys_out, int* __restrict__ vals_out) {
  __shared__ int wcnt[kWarps][kMaxBuckets];
  const int nb = 1 << nbits;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int b = threadIdx.x; b < kWarps * kMaxBuckets; b += kThreads) (&wcnt[0][0])[b] = 0;
  __syncthreads();
  const int base = blockIdx.x * kTile + w * (32 * kItems);
  const unsigned lt = (1u << lane) - 1u;
  int key[kItems], pos[kItems];
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int idx = base + r * 32 + lane;
    const bool valid = idx < n;
    key[r] = valid ? keys_in[idx] : 0;
    const int dig = (key[r] >> shift) & (nb - 1);
    // invalid lanes get distinct out-of-range tags so they never group with real digits
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? dig : nb + lane);
    const int rank = __popc(peers & lt);
    int b0 = 0;
    if (valid) b0 = wcnt[w][dig];
    __syncwarp();
    if (valid && rank == 0) wcnt[w][dig] = b0 + __popc(peers);
    __syncwarp();
    pos[r] = b0 + rank;
  }
  __syncthreads();
  // per bucket: exclusive prefix over the warps of this tile
  for (int b = threadIdx.x; b < nb; b += kThreads) {
    int run = 0;
#pragma unroll
    for (int q = 0; q < kWarps; ++q) {
      const int t = wcnt[q][b];
      wcnt[q][b] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int idx = base + r * 32 + lane;
    if (idx < n) {
      const int dig = (key[r] >> shift) & (nb - 1);
      const int dst = offsets[dig * ntiles + blockIdx.x] + wcnt[w][dig] + pos[r];
      keys_out[dst] = key[r];
      vals_out[dst] = vals_in ? vals_in[idx] : idx;
    }
  }
}

}  // namespace

size_t sort_hist_len(int n, int key_bits) {
  (void)key_bits;
  return sort_hist_ints(n);
}

// Sorts (key_by_gid[g], g) pairs by key; result in d.keys / d.vals.
int launch_sort(const Launch& L, int key_bits, const SortScratch& scr) {
  const Dev& d = L.d;
  const int n = d.Ntot;
  if (n == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(L.stream);
  if (key_bits < 1) key_bits = 1;
  const int passes = (key_bits + kMaxBits - 1) / kMaxBits;
  const int bits = (key_bits + passes - 1) / passes;
  const int ntiles = (n + kTile - 1) / kTile;
  const int m = (1 << bits) * ntiles;
  const int nchunks = (m + kScanChunk - 1) / kScanChunk;
  int* hist = scr.hist;
  int* sums = scr.hist + (size_t)kMaxBuckets * ntiles;
  const int* kin = d.key_by_gid;
  const int* vin = nullptr;
  for (int pass = 0; pass < passes; ++pass) {
    const bool last_even = ((passes - 1 - pass) % 2) == 0;
    int* kout = last_even ? d.keys : d.keys_alt;
    int* vout = last_even ? d.vals : d.vals_alt;
    const int shift = pass * bits;
    k_radix_hist<<<ntiles, kThreads, 0, st>>>(kin, n, shift, bits, ntiles, hist);
    k_scan_sums<<<nchunks, kThreads, 0, st>>>(hist, m, sums);
    k_scan_top<<<1, kThreads, 0, st>>>(sums, nchunks);
    k_scan_apply<<<nchunks, kThreads, 0, st>>>(hist, m, sums);
    k_radix_scatter<<<ntiles, kThreads, 0, st>>>(kin, vin, n, shift, bits, ntiles, hist, kout,
                                                 vout);
    *L.launches += 5;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      last_launch_error() = (int)e;
      return 1;
    }
    kin = kout;
    vin = vout;
  }
  return 0;
}

// The same sort on caller-provided buffers: keys_in (n keys, values are the indices
// 0..n-1), outputs keys_out / vals_out, ping-pong buffers keys_tmp / vals_tmp and a
// histogram of sort_hist_len(n, key_bits) ints.  Used by the allocation-free neighbour
// search (sph_noalloc.cu).
int launch_sort_buffers(const int* keys_in, int n, int key_bits, int* keys_out, int* vals_out,
                        int* keys_tmp, int* vals_tmp, int* hist, void* stream,
                        long long* launches) {
  if (n == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (key_bits < 1) key_bits = 1;
  const int passes = (key_bits + kMaxBits - 1) / kMaxBits;
  const int bits = (key_bits + passes - 1) / passes;
  const int ntiles = (n + kTile - 1) / kTile;
  const int m = (1 << bits) * ntiles;
  const int nchunks = (m + kScanChunk - 1) / kScanChunk;
  int* sums = hist + (size_t)kMaxBuckets * ntiles;
  const int* kin = keys_in;
  const int* vin = nullptr;
  for (int pass = 0; pass < passes; ++pass) {
    const bool last_even = ((passes - 1 - pass) % 2) == 0;
    int* kout = last_even ? keys_out : keys_tmp;
    int* vout = last_even ? vals_out : vals_tmp;
    const int shift = pass * bits;
    k_radix_hist<<<ntiles, kThreads, 0, st>>>(kin, n, shift, bits, ntiles, hist);
    k_scan_sums<<<nchunks, kThreads, 0, st>>>(hist, m, sums);
    k_scan_top<<<1, kThreads, 0, st>>>(sums, nchunks);
    k_scan_apply<<<nchunks, kThreads, 0, st>>>(hist, m, sums);
    k_radix_scatter<<<ntiles, kThreads, 0, st>>>(kin, vin, n, shift, bits, ntiles, hist, kout,
                                                 vout);
    if (launches) *launches += 5;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      last_launch_error() = (int)e;
      return 1;
    }
    kin = kout;
    vin = vout;
  }
  return 0;
}

}  // namespace sph
