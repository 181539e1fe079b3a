// sph_noalloc.cu -- neighbour search that allocates no device memory.
//
// For callers that cannot call cudaMalloc: programs whose device memory is reserved up
// front by their own allocator or pool (a cudaMalloc in the time loop would fail or steal
// from it), and time loops that must not stall the whole device (cudaMalloc and cudaFree
// may synchronise every stream of the device).  The reference's own neighbour search
// would need this: its thrust::sort_by_key allocates temporary storage on every call.
// The caller owns and passes the inputs and outputs; only the sort's scratch is internal.
//
// The sort's scratch lives in one file-scope __device__ array sized for at most
// SPH_NOALLOC_MAX_PARTICLES particles.  Every GPU that loads this library holds it until
// the process exits.  All calls share it, so calls that overlap on the GPU (concurrent
// streams, or several host threads on one device) race and must be serialised by the
// caller.  The array keeps the last call's contents; each call clears the part that must
// start at zero (the status word).
#include <cuda_runtime.h>

#include <cmath>

#include "sph_internal.h"

namespace sph {
int launch_sort_buffers(const int* keys_in, int n, int key_bits, int* keys_out, int* vals_out,
                        int* keys_tmp, int* vals_tmp, int* hist, void* stream,
                        long long* launches);
}

namespace {

constexpr int kMaxN = SPH_NOALLOC_MAX_PARTICLES;
// the sort's histogram for kMaxN keys, sized by the sort's own geometry (sph_internal.h)
constexpr size_t kHistInts = sph::sort_hist_ints(kMaxN);
// layout (ints): unsorted keys | ping-pong keys | ping-pong values | histogram | status
constexpr size_t kOffKeys = 0;
constexpr size_t kOffTmpK = kOffKeys + kMaxN;
constexpr size_t kOffTmpV = kOffTmpK + kMaxN;
constexpr size_t kOffHist = kOffTmpV + kMaxN;
constexpr size_t kOffStatus = kOffHist + kHistInts;
constexpr size_t kScratchInts = kOffStatus + 64;

__device__ __align__(256) int g_noalloc_scratch[kScratchInts];

__global__ void k_noalloc_hash(const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, int n, sph_grid g,
                               int* __restrict__ keys, int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // kernel_cell_list.cu:15-63 (clamp of the top cell except y with walls)
  const double xi = x[i], yi = y[i], zi = g.dim == 3 ? z[i] : 0.0;
  int c = -1;
  if (isfinite(xi) && isfinite(yi) && isfinite(zi)) {
    const double fx = floor(xi / g.cell_size[0]);
    const double fy = g.wall == 0 ? floor(yi / g.cell_size[1])
                                  : floor((yi + g.wall_width) / g.cell_size[1]);
    const double fz = g.dim == 3 ? floor(zi / g.cell_size[2]) : 0.0;
    const double big = 1 << 20;
    if (fabs(fx) <= big && fabs(fy) <= big && fabs(fz) <= big) {
      int cx = (int)fx, cy = (int)fy, cz = (int)fz;
      if (cx == g.Ncells[0]) cx = cx - 1;
      if (g.wall == 0 && cy == g.Ncells[1]) cy = cy - 1;
      if (g.dim == 3 && cz == g.Ncells[2]) cz = cz - 1;
      const long long lc = g.dim == 3 ? ((long long)cz * g.Ncells[1] + cy) * g.Ncells[0] + cx
                                      : (long long)cy * g.Ncells[0] + cx;
      const long long total = (long long)g.Ncells[0] * g.Ncells[1] * (g.dim == 3 ? g.Ncells[2] : 1);
      if (lc >= 0 && lc < total) c = (int)lc;
    }
  }
  if (c < 0) {
    atomicOr(status, 1);
    c = 0;  // keeps the sort in bounds; the call reports SPH_ERR_CELL_RANGE
  }
  keys[i] = c;
}

// kernel_cell_ranges.cu:13-33: ranges written for occupied cells only
__global__ void k_noalloc_ranges(const int* __restrict__ cell, int n, int* __restrict__ start,
                                 int* __restrict__ end) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = cell[k];
  if (k == 0 || cell[k - 1] != c) start[c] = k;
  if (k == n - 1 || cell[k + 1] != c) end[c] = k;
}

// The device address of the scratch array in the current device's current context.  In
// host code the array's name is only a host-side stand-in, so the address is looked up,
// and it is looked up on every call rather than cached: after cudaDeviceReset (which the
// reference's main.cu calls) or in another context on the same device the array lives
// at a new address.  The lookup is a host-side table query, cheap next to the launches.
// The first lookup in a context loads this file's device code, which is where the array
// is placed in device memory; no call allocates anything after that.
sph_status scratch_for_current_device(int** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return SPH_ERR_CUDA;
  }
  *out = static_cast<int*>(p);
  return SPH_OK;
}

}  // namespace

extern "C" sph_status sph_neighbours_search_noalloc(const double* x, const double* y,
                                                    const double* z, int n, const sph_grid* grid,
                                                    int* particle_cell, int* particle_index,
                                                    int* cell_start, int* cell_end,
                                                    void* stream) {
  if (!grid || n < 0 || (n > 0 && (!x || !y || !particle_cell || !particle_index ||
                                   !cell_start || !cell_end)))
    return SPH_ERR_BAD_INPUT;
  if (n > kMaxN) return SPH_ERR_CAPACITY;
  const sph_grid g = *grid;
  if ((g.dim != 2 && g.dim != 3) || (g.dim == 3 && !z) || g.Ncells[0] < 1 || g.Ncells[1] < 1 ||
      (g.dim == 3 && g.Ncells[2] < 1) || !(g.cell_size[0] > 0) || !(g.cell_size[1] > 0) ||
      (g.dim == 3 && !(g.cell_size[2] > 0)))
    return SPH_ERR_BAD_INPUT;
  const long long total = (long long)g.Ncells[0] * g.Ncells[1] * (g.dim == 3 ? g.Ncells[2] : 1);
  if (total > (1LL << 27)) return SPH_ERR_CAPACITY;
  int* s = nullptr;
  sph_status st = scratch_for_current_device(&s);
  if (st != SPH_OK || n == 0) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  int* keys = s + kOffKeys;
  int* status = s + kOffStatus;
  if (cudaMemsetAsync(status, 0, sizeof(int), cs) != cudaSuccess) return SPH_ERR_CUDA;
  const int threads = 256, blocks = (n + threads - 1) / threads;
  k_noalloc_hash<<<blocks, threads, 0, cs>>>(x, y, z, n, g, keys, status);
  if (cudaGetLastError() != cudaSuccess) return SPH_ERR_CUDA;
  int bits = 1;
  while ((1LL << bits) < total) ++bits;
  if (sph::launch_sort_buffers(keys, n, bits, particle_cell, particle_index, s + kOffTmpK,
                               s + kOffTmpV, s + kOffHist, stream, nullptr))
    return SPH_ERR_CUDA;
  k_noalloc_ranges<<<blocks, threads, 0, cs>>>(particle_cell, n, cell_start, cell_end);
  if (cudaGetLastError() != cudaSuccess) return SPH_ERR_CUDA;
  int h_status = 0;
  if (cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, cs) !=
          cudaSuccess ||
      cudaStreamSynchronize(cs) != cudaSuccess)
    return SPH_ERR_CUDA;
  return h_status ? SPH_ERR_CELL_RANGE : SPH_OK;
}
