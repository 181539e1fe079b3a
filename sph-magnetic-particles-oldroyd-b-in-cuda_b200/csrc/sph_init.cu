// sph_init.cu -- device-side initialisation of lattice boxes (an ensemble's boxes are built
// on the GPU instead of the host): lattice sites, colloid carving, wall layers, particle
// attributes and the walls lists of system_initialize_particles_new_sim.cpp:21-140 and
// system_initialize.cpp:277-300, plus the scatter of the particles the host still builds
// (colloid shells, restart boxes).
//
// The positions are bit-identical to the host set-up's: every operation is the rounded
// IEEE operation the host performs (no contraction into FMA), in the host's order.
// Two passes over the same sites: the first counts the kept, bottom-wall and top-wall
// sites of each block (a block never spans two boxes), the host turns the counts into
// per-block offsets, the second writes each kept site to its place in id order.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

// The reference's conditional minimum image (system_initialize_particles_new_sim.cpp:37-50).
__device__ __forceinline__ double wrap_half_rn(double d, double L) {
  if (d > 0.5 * L) d = __dsub_rn(d, L);
  if (d < -0.5 * L) d = __dadd_rn(d, L);
  return d;
}

// Site `site` of box B in the host's loop order (x outer, y, z inner): position
// (system_initialize_particles_new_sim.cpp:22-29, 64-69), type (:101-112), and whether a
// colloid carves it out, r^2 <= R^2 for any colloid of the box (:31-60, 71-95).
__device__ __forceinline__ bool lattice_site(const InitBox& B, int site, const double* centres,
                                             double& px, double& py, double& pz, int& type) {
  const int nk = B.dim == 3 ? B.Nxyz[2] : 1;
  const int k = site % nk;
  const int ij = site / nk;
  const int j = ij % B.Nxyz[1];
  const int i = ij / B.Nxyz[1];
  px = __dadd_rn(__dmul_rn(0.5, B.dx[0]), __dmul_rn((double)i, B.dx[0]));
  py = __dadd_rn(__dmul_rn(0.5, B.dx[1]), __dmul_rn((double)j, B.dx[1]));
  if (B.wall) py = __dsub_rn(py, B.wall_width);
  pz = B.dim == 3 ? __dadd_rn(__dmul_rn(0.5, B.dx[2]), __dmul_rn((double)k, B.dx[2])) : 0.0;
  bool carved = false;
  for (int l = 0; l < B.ncoll && !carved; ++l) {
    const double* c = centres + 3 * (size_t)(B.coll0 + l);
    const double rx = wrap_half_rn(__dsub_rn(px, c[0]), B.L[0]);
    double ry = __dsub_rn(py, c[1]);
    if (B.wall == 0) ry = wrap_half_rn(ry, B.L[1]);
    double r2 = __dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry));
    if (B.dim == 3) {
      const double rz = wrap_half_rn(__dsub_rn(pz, c[2]), B.L[2]);
      r2 = __dadd_rn(r2, __dmul_rn(rz, rz));
    }
    carved = r2 <= B.R2;
  }
  type = B.wall ? (py < B.y_bottom ? 1 : (py > B.y_top ? 2 : 0)) : 0;
  return !carved;
}

__global__ void __launch_bounds__(kInitThreads) k_init_count(const InitBox* boxes,
                                                             const int* blk_box,
                                                             const double* centres,
                                                             int* counts) {
  const InitBox& B = boxes[blk_box[blockIdx.x]];
  const int site = (blockIdx.x - B.blk0) * kInitThreads + threadIdx.x;
  bool keep = false;
  int type = 0;
  if (site < B.nsites) {
    double px, py, pz;
    keep = lattice_site(B, site, centres, px, py, pz, type);
  }
  const int n0 = __syncthreads_count(keep);
  const int n1 = __syncthreads_count(keep && type == 1);
  const int n2 = __syncthreads_count(keep && type == 2);
  if (threadIdx.x == 0) {
    counts[3 * blockIdx.x + 0] = n0;
    counts[3 * blockIdx.x + 1] = n1;
    counts[3 * blockIdx.x + 2] = n2;
  }
}

// offs: per block, the box-local number of kept, bottom-wall and top-wall sites before it.
__global__ void __launch_bounds__(kInitThreads) k_init_fill(Dev d, const InitBox* boxes,
                                                            const int* blk_box,
                                                            const double* centres,
                                                            const int* offs) {
  __shared__ int wsum[3][kInitThreads / 32];
  const InitBox& B = boxes[blk_box[blockIdx.x]];
  const int site = (blockIdx.x - B.blk0) * kInitThreads + threadIdx.x;
  bool keep = false;
  int type = 0;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (site < B.nsites) keep = lattice_site(B, site, centres, px, py, pz, type);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned m0 = __ballot_sync(kFull, keep);
  const unsigned m1 = __ballot_sync(kFull, keep && type == 1);
  const unsigned m2 = __ballot_sync(kFull, keep && type == 2);
  const unsigned below = (1u << lane) - 1u;
  int r0 = __popc(m0 & below), r1 = __popc(m1 & below), r2 = __popc(m2 & below);
  if (lane == 0) {
    wsum[0][w] = __popc(m0);
    wsum[1][w] = __popc(m1);
    wsum[2][w] = __popc(m2);
  }
  __syncthreads();
  for (int q = 0; q < w; ++q) {
    r0 += wsum[0][q];
    r1 += wsum[1][q];
    r2 += wsum[2][q];
  }
  if (!keep) return;
  const int s = B.slot0 + offs[3 * blockIdx.x] + r0;
  const size_t Np = d.Npad;
  d.pos[s] = make_double4(px, py, pz, B.mass);
  d.vel[s] = make_double4(0.0, 0.0, 0.0, 0.0);
  d.conf[0 * Np + s] = 1.0;  // cxx
  d.conf[1 * Np + s] = 0.0;  // cxy
  d.conf[2 * Np + s] = 1.0;  // cyy
  d.conf[3 * Np + s] = 0.0;  // cxz
  d.conf[4 * Np + s] = 0.0;  // cyz
  d.conf[5 * Np + s] = 1.0;  // czz
  d.tinfo[s] = type | (B.box << kTypeBits);
  d.gid[s] = s;
  d.inv[s] = s;
  if (type == 1) d.walls_list[B.wl0 + offs[3 * blockIdx.x + 1] + r1] = s;
  if (type == 2) d.walls_list[B.wl0 + B.nw1 + offs[3 * blockIdx.x + 2] + r2] = s;
}

// Particles built on the host, packed: slot and type word per particle, position + mass,
// velocity, conformation (6 rows of n).
__global__ void k_init_scatter(Dev d, int n, const int2* meta, const double4* pos,
                               const double4* vel, const double* conf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = meta[k].x;
  const size_t Np = d.Npad;
  d.pos[s] = pos[k];
  d.vel[s] = vel[k];
#pragma unroll
  for (int q = 0; q < 6; ++q) d.conf[q * Np + s] = conf[(size_t)q * n + k];
  d.tinfo[s] = meta[k].y;
  d.gid[s] = s;
  d.inv[s] = s;
}

int init_check() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    last_launch_error() = (int)e;
    return 1;
  }
  return 0;
}

}  // namespace

int launch_init_count(const InitBox* boxes, const int* blk_box, int nblk, const double* centres,
                      int* counts, void* stream) {
  if (nblk == 0) return 0;
  k_init_count<<<nblk, kInitThreads, 0, (cudaStream_t)stream>>>(boxes, blk_box, centres, counts);
  return init_check();
}

int launch_init_fill(const Launch& L, const InitBox* boxes, const int* blk_box, int nblk,
                     const double* centres, const int* offs) {
  if (nblk == 0) return 0;
  k_init_fill<<<nblk, kInitThreads, 0, (cudaStream_t)L.stream>>>(L.d, boxes, blk_box, centres,
                                                                 offs);
  return init_check();
}

int launch_init_scatter(const Launch& L, int n, const int2* meta, const double4* pos,
                        const double4* vel, const double* conf) {
  if (n == 0) return 0;
  k_init_scatter<<<(n + 255) / 256, 256, 0, (cudaStream_t)L.stream>>>(L.d, n, meta, pos, vel,
                                                                      conf);
  return init_check();
}

}  // namespace sph
