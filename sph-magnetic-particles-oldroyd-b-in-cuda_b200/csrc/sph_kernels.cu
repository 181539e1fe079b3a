// sph_kernels.cu -- device kernels of the SPH step for sm_100a.
//
// Layout: particles live in "slot" order, the stable (cell, id) order of the last
// neighbour search, so that every cell's particles are contiguous in HBM.  State is SoA /
// packed AoS (pos = double4 x,y,z,mass; vel = double4) and is permuted into the new order
// once per search (k_reorder).  The pair phases read per-particle neighbour lists built by
// a warp-per-cell kernel (k_build_lists) that walks the 3^d neighbour cells in the
// reference's order (kernel_densities.cu:52-163), so each particle's sums run over the
// same neighbours in the same order as the reference's gather loops.  All sums are
// gathers (no atomics), so results are bit-reproducible run to run.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

// ---------------------------------------------------------------------------------
// Velocity Verlet, particles (kernel_move_sys_VV_part1.cu:13-114, ..._part2.cu:13-58)
// ---------------------------------------------------------------------------------
__global__ void k_vv1_particles(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  int ti = d.tinfo[i];
  int t = type_of(ti);
  if (t > 2) return;  // colloid particles are placed by k_vv1_colloids
  const BoxParams& p = d.box[box_of(ti)];
  const double dt = p.dt;
  double4 x = d.pos[i];
  double4 v = d.vel[i];
  const int Np = d.Npad;
  if (t == 0) {
    double h = 0.5 * dt;
    double hm = h / x.w;
    v.x = v.x + hm * d.f[i];
    v.y = v.y + hm * d.f[Np + i];
    d.conf[i] = d.conf[i] + h * d.dcdt[i];
    d.conf[Np + i] = d.conf[Np + i] + h * d.dcdt[Np + i];
    d.conf[2 * Np + i] = d.conf[2 * Np + i] + h * d.dcdt[2 * Np + i];
    if (p.dim == 3) {
      v.z = v.z + hm * d.f[2 * Np + i];
      d.conf[3 * Np + i] = d.conf[3 * Np + i] + h * d.dcdt[3 * Np + i];
      d.conf[4 * Np + i] = d.conf[4 * Np + i] + h * d.dcdt[4 * Np + i];
      d.conf[5 * Np + i] = d.conf[5 * Np + i] + h * d.dcdt[5 * Np + i];
    }
  } else {
    v.x = (t == 1) ? p.V_bottom : p.V_top;
    v.y = 0.0;
    if (p.dim == 3) v.z = 0.0;
  }
  double xi = x.x + v.x * dt;
  double yi = x.y + v.y * dt;
  double zi = x.z;
  if (p.dim == 3) zi = x.z + v.z * dt;
  if (xi < 0) xi = xi + p.L[0];
  if (p.wall == 0 && yi < 0) yi = yi + p.L[1];
  if (p.dim == 3 && zi < 0) zi = zi + p.L[2];
  if (xi > p.L[0]) xi = xi - p.L[0];
  if (p.wall == 0 && yi > p.L[1]) yi = yi - p.L[1];
  if (p.dim == 3 && zi > p.L[2]) zi = zi - p.L[2];
  if (outside_periodic(p, xi, yi, zi)) mark_outside(d);  // moved more than a box length
  x.x = xi;
  x.y = yi;
  x.z = zi;
  d.pos[i] = x;
  d.vel[i] = v;
}

__global__ void k_vv2_particles(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  int ti = d.tinfo[i];
  if (type_of(ti) != 0) return;
  const BoxParams& p = d.box[box_of(ti)];
  const int Np = d.Npad;
  const double h = 0.5 * p.dt;
  double4 v = d.vel[i];
  const int nc = p.dim == 3 ? 6 : 3;
  if (p.dim == 3)
    vv2_fluid<3>(p, d.pos[i].w, d.f[i], d.f[Np + i], d.f[2 * Np + i], v);
  else
    vv2_fluid<2>(p, d.pos[i].w, d.f[i], d.f[Np + i], 0.0, v);
  for (int q = 0; q < nc; ++q) d.conf[q * Np + i] = __fma_rn(h, d.dcdt[q * Np + i], d.conf[q * Np + i]);
  d.vel[i] = v;
}

// Hamilton product (kernel_quaternion_product.cu:15-31)
__device__ __forceinline__ void qmul(const double* c, const double* e, double* r) {
  r[0] = c[0] * e[0] - c[1] * e[1] - c[2] * e[2] - c[3] * e[3];
  r[1] = c[0] * e[1] + c[1] * e[0] + c[2] * e[3] - c[3] * e[2];
  r[2] = c[0] * e[2] - c[1] * e[3] + c[2] * e[0] + c[3] * e[1];
  r[3] = c[0] * e[3] + c[1] * e[2] - c[2] * e[1] + c[3] * e[0];
}

// Rigid colloid half-kick, drift, rotation and re-placement of its boundary particles
// (kernel_move_colloids_VV_part1.cu:15-204).  One block per colloid.
__global__ void k_vv1_colloids(Dev d) {
  const int c = blockIdx.x;
  if (c >= d.ncoll) return;
  if (step_aborted(d)) return;
  const BoxParams& p = d.box[d.coll_box[c]];
  if (p.coll_move != 0) return;
  __shared__ double rot[4];  // 2D: cos, sin; 3D: quaternion
  __shared__ double ctr[3];
  const int nc = d.ncoll;
  double* cs = d.cs;
  const double dt = p.dt;
  if (threadIdx.x == 0) {
    double hm = 0.5 * dt / p.coll_mass, hI = 0.5 * dt / p.coll_I;
    double cx = cs[CS_X * nc + c], cy = cs[CS_Y * nc + c], cz = cs[CS_Z * nc + c];
    cs[CS_VX * nc + c] += hm * cs[CS_FX * nc + c];
    cs[CS_VY * nc + c] += hm * cs[CS_FY * nc + c];
    if (p.dim == 3) cs[CS_VZ * nc + c] += hm * cs[CS_FZ * nc + c];
    cs[CS_OZ * nc + c] += hI * cs[CS_TZ * nc + c];
    double omega;
    if (p.dim == 2) {
      omega = cs[CS_OZ * nc + c];
    } else {
      cs[CS_OX * nc + c] += hI * cs[CS_TX * nc + c];
      cs[CS_OY * nc + c] += hI * cs[CS_TY * nc + c];
      double ox = cs[CS_OX * nc + c], oy = cs[CS_OY * nc + c], oz = cs[CS_OZ * nc + c];
      omega = sqrt(ox * ox + oy * oy + oz * oz);
    }
    cx = cx + cs[CS_VX * nc + c] * dt;
    cy = cy + cs[CS_VY * nc + c] * dt;
    if (p.dim == 3) cz = cz + cs[CS_VZ * nc + c] * dt;
    if (cx < 0) cx = cx + p.L[0];
    if (cx > p.L[0]) cx = cx - p.L[0];
    if (p.wall == 0) {
      if (cy < 0) cy = cy + p.L[1];
      if (cy > p.L[1]) cy = cy - p.L[1];
    }
    if (p.dim == 3) {
      if (cz < 0) cz = cz + p.L[2];
      if (cz > p.L[2]) cz = cz - p.L[2];
    }
    cs[CS_X * nc + c] = cx;
    cs[CS_Y * nc + c] = cy;
    if (p.dim == 3) cs[CS_Z * nc + c] = cz;
    ctr[0] = cx;
    ctr[1] = cy;
    ctr[2] = cz;
    if (p.dim == 2) {
      double th = cs[CS_THETA * nc + c] + cs[CS_OZ * nc + c] * dt;
      rot[1] = sin(th);
      rot[0] = cos(th);
      cs[CS_THETA * nc + c] = th;
    } else {
      // omega = 0 gives a NaN axis, as in the reference (:123-125); the NaN positions are
      // then reported as SPH_ERR_NAN by the hash instead of trapping.
      double half = 0.5 * omega * dt;
      double ax = cs[CS_OX * nc + c] / omega, ay = cs[CS_OY * nc + c] / omega,
             az = cs[CS_OZ * nc + c] / omega;
      double sh = sin(half);
      double dq[4] = {cos(half), sh * ax, sh * ay, sh * az};
      double q[4] = {cs[CS_Q0 * nc + c], cs[CS_QX * nc + c], cs[CS_QY * nc + c],
                     cs[CS_QZ * nc + c]};
      double r[4];
      qmul(dq, q, r);
      cs[CS_Q0 * nc + c] = r[0];
      cs[CS_QX * nc + c] = r[1];
      cs[CS_QY * nc + c] = r[2];
      cs[CS_QZ * nc + c] = r[3];
      rot[0] = r[0];
      rot[1] = r[1];
      rot[2] = r[2];
      rot[3] = r[3];
    }
  }
  __syncthreads();
  const int j0 = d.coll_seg[c], j1 = d.coll_seg[c + 1];
  const int NL = d.Nlist_coll;
  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const int slot = d.inv[d.colloids_list[j]];
    double px, py, pz = 0.0;
    if (p.dim == 2) {
      double x0 = d.xc[j], y0 = d.xc[NL + j];
      px = x0 * rot[0] - y0 * rot[1];
      py = x0 * rot[1] + y0 * rot[0];
    } else {
      double q[4] = {rot[0], rot[1], rot[2], rot[3]};
      double qi[4] = {rot[0], -rot[1], -rot[2], -rot[3]};
      double pt[4] = {0.0, d.xc[j], d.xc[NL + j], d.xc[2 * NL + j]};
      double t1[4], t2[4];
      qmul(q, pt, t1);
      qmul(t1, qi, t2);
      px = t2[1];
      py = t2[2];
      pz = t2[3];
    }
    double4 x = d.pos[slot];
    x.x = px + ctr[0];
    x.y = py + ctr[1];
    if (p.dim == 3) x.z = pz + ctr[2];
    if (x.x < 0) x.x = x.x + p.L[0];
    if (x.x > p.L[0]) x.x = x.x - p.L[0];
    if (p.wall == 0) {
      if (x.y < 0) x.y = x.y + p.L[1];
      if (x.y > p.L[1]) x.y = x.y - p.L[1];
    }
    if (p.dim == 3) {
      if (x.z < 0) x.z = x.z + p.L[2];
      if (x.z > p.L[2]) x.z = x.z - p.L[2];
    }
    if (outside_periodic(p, x.x, x.y, x.z)) mark_outside(d);
    d.pos[slot] = x;
  }
}

// kernel_move_colloids_VV_part2.cu:14-46
__global__ void k_vv2_colloids(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.ncoll) return;
  if (step_aborted(d)) return;
  const BoxParams& p = d.box[d.coll_box[c]];
  if (p.coll_move != 0) return;
  const int nc = d.ncoll;
  double* cs = d.cs;
  double hm = 0.5 * p.dt / p.coll_mass, hI = 0.5 * p.dt / p.coll_I;
  cs[CS_VX * nc + c] += hm * cs[CS_FX * nc + c];
  cs[CS_VY * nc + c] += hm * cs[CS_FY * nc + c];
  if (p.dim == 3) cs[CS_VZ * nc + c] += hm * cs[CS_FZ * nc + c];
  cs[CS_OZ * nc + c] += hI * cs[CS_TZ * nc + c];
  if (p.dim == 3) {
    cs[CS_OX * nc + c] += hI * cs[CS_TX * nc + c];
    cs[CS_OY * nc + c] += hI * cs[CS_TY * nc + c];
  }
}

// ---------------------------------------------------------------------------------
// Neighbour search: hash -> (radix sort, sph_sort.cu) -> reorder + cell ranges -> lists
// ---------------------------------------------------------------------------------
__global__ void k_hash(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  int ti = d.tinfo[i];
  const BoxParams& p = d.box[box_of(ti)];
  double4 x = d.pos[i];
  if (outside_periodic(p, x.x, x.y, x.z)) mark_outside(d);  // cleared before this pass
  int c = hash_cell(p, x.x, x.y, x.z);
  if (c < 0) {
    raise_status(d, c == -2 ? kStatNaN : kStatCellRange, d.gid[i], kPhaseHash);
    c = 0;  // keep the sort in bounds; the step is reported as failed
  }
  d.key_by_gid[d.gid[i]] = p.cell0 + c;
}

// Gathers the state into the new slot order and records the cell ranges.
// cell_begin (dense, all cells) drives the engine; cell_start / cell_end keep the
// reference's semantics: written for occupied cells only, box-local slot numbers
// (kernel_cell_ranges.cu:13-33).
template <bool MIXED, bool PERMUTE_F>
__global__ void k_reorder(Dev d) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.Ntot) return;
  if (step_aborted(d)) return;
  const int g = d.vals[k];
  const int o = d.inv[g];
  const int Np = d.Npad;
  double4 x = d.pos[o];
  d.pos_b[k] = x;
  d.vel_b[k] = d.vel[o];
#pragma unroll
  for (int q = 0; q < 6; ++q) d.conf_b[q * Np + k] = d.conf[q * Np + o];
  if (PERMUTE_F) {
#pragma unroll
    for (int q = 0; q < 3; ++q) d.f_b[q * Np + k] = d.f[q * Np + o];
#pragma unroll
    for (int q = 0; q < 6; ++q) d.dcdt_b[q * Np + k] = d.dcdt[q * Np + o];
  }
  int ti = d.tinfo[o];
  d.tinfo_b[k] = ti;
  d.gid_b[k] = g;
  d.inv[g] = k;
  if (MIXED) d.pos_f[k] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
  const int key = d.keys[k];
  const int prev = k > 0 ? d.keys[k - 1] : -1;
  for (int c = prev + 1; c <= key; ++c) d.cell_begin[c] = k;
  if (k == d.Ntot - 1)
    for (int c = key + 1; c <= d.Ctot; ++c) d.cell_begin[c] = d.Ntot;
  const int slot0 = d.box[box_of(ti)].slot0;
  if (k == 0 || prev != key) d.cell_start[key] = k - slot0;
  if (k == d.Ntot - 1 || d.keys[k + 1] != key) d.cell_end[key] = k - slot0;
}

// Density contribution of one list entry (kernel_densities.cu:52-163 with kernel_W.cu):
// the exact distance test, then W(r) with r from one reciprocal square root; the
// particle itself (r2 = 0) contributes W(0).  WRAP: see min_image.
template <typename T, int DIM, bool WRAP = true>
__device__ __forceinline__ T density_term(const typename V4<T>::type& xi,
                                          const typename V4<T>::type& xj, const T L[3],
                                          const T h[3], int wall, T rcutsq, T rcut_inv, T cw) {
  T rx = xi.x - xj.x, ry = xi.y - xj.y, rz = DIM == 3 ? xi.z - xj.z : T(0);
  min_image<T, DIM, WRAP>(rx, ry, rz, L, h, wall);
  const T r2 = norm2(rx, ry, rz, DIM == 3);
  if (!(r2 < rcutsq)) return T(0);
  const T r = r2 > T(0) ? r2 * rsqrt(r2) : T(0);
  return sph_w<T>(r, rcut_inv, cw);
}

// Density, pressure (kernel_pressures.cu:13-23) and the neighbour record of slot i.
template <typename T, int DIM>
__device__ __forceinline__ void density_epilogue(const Dev& d, int i, const BoxParams& p,
                                                 double dens) {
  d.dens[i] = dens;
  const double press = p.csq * (d.pos[i].w * dens - p.rho0);
  d.press[i] = press;
  write_record<T, DIM>(d, i, p, d.tinfo[i], dens, press);
}

// One warp per cell: the cell's particles (<= 32 per round) test the candidates of the
// 3^d neighbour cells, staged 32 at a time in shared memory as float offsets from the
// cell corner.  Candidate ranges come from the reference-semantics cell_start / cell_end,
// so the candidate set and order are the reference's (kernel_densities.cu:52-163), stale
// ranges included.  The float test uses a slightly enlarged cutoff; consumers apply the
// exact test.
//
// The lists are chunks with hit masks, not indices.  Candidates come in chunks of up to 32
// consecutive slots of one neighbour cell; for every chunk in which it has a hit, a particle
// stores one 8-byte entry (the chunk's first slot, a 32-bit mask whose bit 31 - q means slot
// first + q is a candidate), chunk-major: nchunk[k * Npad + i], so that consumers walking
// their lists in step read neighbouring words.  Decoding the entries in order, bit by bit,
// gives the neighbours in the order of an index list (the reference's candidate order), at
// 8 bytes per chunk with hits (about 20 in 3D) instead of 4 bytes per neighbour (about
// 108), and the build needs no per-lane append loop: a chunk's hits are one store.
//
// A particle whose own (unclamped) cell differs from its sort cell (x exactly at L) has
// other neighbour cells; its whole warp tests its candidates with ballots.
//
// (Summing the density over the hits inside this kernel was measured slower than the
// separate k_density pass: the per-lane hit loops diverge and the warp runs the FP64
// kernel evaluation for its busiest lane.)
//
// TPC (threads per cell) is 32 or 16.  With 16, each half-warp works on its own cell:
// 2D cells at overlap 4 hold about 16 particles, so a whole warp per cell leaves half of
// its lanes idle.  The neighbours are the same either way (same candidates, same order);
// chunks are then 16 slots long.
//
// Blocks of 4 warps, measured against 8 (128^3 list build 1.66 vs 1.88 ms; 2D ensemble
// 1.15 vs 1.19 ms, with the test loop not unrolled).
constexpr int kListWarps = 4;

// Packed FP32 pairs (the f32x2 arithmetic of sm_100): two candidates per instruction.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
  f32x2 d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
  return d;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Candidate test of two staged candidates (a: their x pair, b: y, c: z, as loaded from the
// stage) against one particle: the sign bit of rx^2 + ry^2 + rz^2 - cut2, accumulated by fused
// multiply-adds from -cut2, funnel-shifted into `hits` first candidate first (one shift per
// candidate).  The rounding of the chain can only move candidates within a few float ulps of
// the list cutoff, which lies 5e-5 of rcut beyond the cutoff every consumer applies exactly,
// so the neighbours found are the same.  Staged padding at 1e30 gives +inf and no hit.
// (Against a separate subtract and a shift-and-or per candidate: 128^3 list build 1.04 ->
// 0.95 ms.)
template <int DIM>
__device__ __forceinline__ unsigned list_test2(unsigned hits, f32x2 xi, f32x2 yi, f32x2 zi,
                                               f32x2 ncut2, f32x2 a, f32x2 b, f32x2 c) {
  const f32x2 rx = f2_sub(xi, a), ry = f2_sub(yi, b);
  f32x2 s = f2_fma(ry, ry, f2_fma(rx, rx, ncut2));
  if (DIM == 3) {
    const f32x2 rz = f2_sub(zi, c);
    s = f2_fma(rz, rz, s);
  }
  unsigned lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(s));
  hits = __funnelshift_l(lo, hits, 1);
  return __funnelshift_l(hi, hits, 1);
}

// Candidate placement.  A candidate of a neighbour cell's range is staged with that cell's
// periodic shift, except in two cases where it must be placed at its minimum image about the
// centre of the listing cell:
//  - a stale range: an emptied cell keeps the range of the search that last saw it occupied
//    (kernel_cell_ranges.cu:13-33); after the sort those slots hold whatever particles, from
//    anywhere in the box, and the consumers take them by the minimum image as the reference
//    does (kernel_densities.cu:90-110), so some are neighbours through another face;
//  - a position outside the box (err_info[kPosOutside]): the hash's linear cell index runs
//    on into the next row, so a particle can sit in a range far from its position.
// With at least 3 cells per axis (cell >= rcut) the image about the centre is the one within
// the cutoff of every particle of the cell, if any is.  A warp with a stale neighbour range,
// or every warp while a position is outside, places all its candidates so; the others keep
// the per-cell shift, which needs no test per candidate.
//
// v: a candidate's unshifted offset from the cell's corner along one axis; c the cell's
// width, L the box's.
__device__ __forceinline__ float stale_offset(float v, double c, double L) {
  const float r = v - (float)(0.5 * c), hl = (float)(0.5 * L);
  return r > hl ? v - (float)L : (r < -hl ? v + (float)L : v);
}
// The same with the bounds precomputed (lo = c/2 - L/2, hi = c/2 + L/2; an axis that does
// not wrap has infinite bounds).
__device__ __forceinline__ float frame_offset(float v, const float* lo, const float* hi,
                                              const float* L, int q) {
  v = v > hi[q] ? v - L[q] : v;
  return v < lo[q] ? v + L[q] : v;
}

// Neighbour cell q (0 .. 3^d - 1, x slowest) of cell (cx, cy, cz) of box p with the
// periodic wrap; false where the row does not exist (beyond a wall).
template <int DIM>
__device__ __forceinline__ bool neighbour_cell(const BoxParams& p, int cx, int cy, int cz,
                                               int q, int& nc) {
  constexpr int kNZ = DIM == 3 ? 3 : 1;
  const int N0 = p.Ncells[0], N1 = p.Ncells[1], N2 = p.Ncells[2];
  int nx = cx + q / (3 * kNZ) - 1, ny = cy + (q / kNZ) % 3 - 1;
  int nz = DIM == 3 ? cz + q % 3 - 1 : 0;
  if (nx < 0) nx += N0;
  if (nx >= N0) nx -= N0;
  if (DIM == 3) {
    if (nz < 0) nz += N2;
    if (nz >= N2) nz -= N2;
  }
  if (!p.wall) {
    if (ny < 0) ny += N1;
    if (ny >= N1) ny -= N1;
  }
  if (ny < 0 || ny >= N1) return false;
  nc = p.cell0 + (DIM == 3 ? (nz * N1 + ny) * N0 + nx : ny * N0 + nx);
  return true;
}

// An emptied cell whose reference range still lists slots.
__device__ __forceinline__ bool stale_cell(const Dev& d, int nc) {
  return d.cell_end[nc] >= d.cell_start[nc] && d.cell_begin[nc] == d.cell_begin[nc + 1];
}

template <int DIM, int TPC>
__global__ void __launch_bounds__(kListWarps * 32) k_build_lists(Dev d) {
  static_assert(TPC == 32 || TPC == 16, "a warp or a half-warp per cell");
  // candidates staged as three float rows per warp, read four at a time
  __shared__ __align__(16) float stage_x[kListWarps][32];
  __shared__ __align__(16) float stage_y[kListWarps][32];
  __shared__ __align__(16) float stage_z[kListWarps][32];
  __shared__ float frame[kListWarps][2][9];  // per group: lo[3], hi[3], L[3] (frame_offset)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (step_aborted_warp(d)) return;
  // a position outside the box (the hash's flag) may be sorted into a cell other than its
  // own (the linear cell index runs on into the next row): then every candidate is placed
  // by its minimum image, as in a stale range
  int out_flag = 0;
  if (lane == 0) out_flag = *(volatile const int*)(d.err_info + kPosOutside);
  const bool any_out = __shfl_sync(SPH_FULL, out_flag, 0) != 0;
  const int sub = lane / TPC, gl = lane % TPC;  // group within the warp, lane within the group
  float* stx = &stage_x[w][sub * TPC];
  float* sty = &stage_y[w][sub * TPC];
  float* stz = &stage_z[w][sub * TPC];
  const int cell = (blockIdx.x * kListWarps + w) * (32 / TPC) + sub;
  // both groups of a warp walk the same loop structure in lockstep (divergent halves would
  // run one after the other): trip counts are warp maxima, a group past its own range idles
  const bool live = cell < d.Ctot;
  if (!__any_sync(SPH_FULL, live)) return;
  const int cl = live ? cell : 0;
  const int b = d.cell_box[cl];
  const BoxParams& p = d.box[b];
  const int N0 = p.Ncells[0], N1 = p.Ncells[1], N2 = p.Ncells[2];
  const int lc = cl - p.cell0;
  const int cx = lc % N0, cy = (lc / N0) % N1, cz = DIM == 3 ? lc / (N0 * N1) : 0;
  const int beg = live ? d.cell_begin[cl] : 0, end = live ? d.cell_begin[cl + 1] : 0;
  const double ox = cx * p.cell_size[0];
  const double oy = cy * p.cell_size[1] - (p.wall ? p.wall_width : 0.0);
  const double oz = DIM == 3 ? cz * p.cell_size[2] : 0.0;
  const float cut2 = (float)p.list_cut2;
  const int cap = d.cap;  // chunks with hits a particle can store
  const size_t Np = d.Npad;
  auto warp_max = [](int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(SPH_FULL, v, o));
    return v;
  };
  const int span = warp_max(end - beg);
  int maxch = 0;  // the most chunks with hits any particle of this warp had
  // the neighbour cells' candidate ranges: with a warp per cell, lane q loads those of
  // neighbour cell q up front (all 3^d loads in flight at once) and the loop takes them
  // by shuffle; a half-warp group loads them as it goes
  constexpr int kNZ = DIM == 3 ? 3 : 1;
  int rs = 0, re = -1;
  bool found = false;  // a stale neighbour range
  if (TPC == 32 && live && lane < 9 * kNZ) {
    int nc;
    if (neighbour_cell<DIM>(p, cx, cy, cz, lane, nc)) {
      rs = d.cell_start[nc] + p.slot0;
      re = d.cell_end[nc] + p.slot0;
      found = stale_cell(d, nc);
    }
  }
  if (TPC == 16 && live) {
    for (int q = gl; q < 9 * kNZ; q += TPC) {
      int nc;
      if (neighbour_cell<DIM>(p, cx, cy, cz, q, nc)) found = found || stale_cell(d, nc);
    }
  }
  // minimum-image placement for the whole warp (see stale_offset)
  const bool mi = any_out || __any_sync(SPH_FULL, found);
  if (mi && gl == 0) {
    float* f = frame[w][sub];
    for (int q = 0; q < 3; ++q) {
      const bool wraps = q == 0 || (q == 1 && !p.wall) || (q == 2 && DIM == 3);
      const float c = (float)(0.5 * p.cell_size[q]), h = (float)(0.5 * p.L[q]);
      f[q] = wraps ? c - h : -3.0e38f;
      f[3 + q] = wraps ? c + h : 3.0e38f;
      f[6 + q] = (float)p.L[q];
    }
  }
  __syncwarp();
  const float* flo = frame[w][sub];
  const float* fhi = flo + 3;
  const float* fL = flo + 6;
  // the particle loop, in the cheap form (per-cell shifts) or the minimum-image one
  auto walk = [&](auto mi_tag) {
    constexpr bool kMI = decltype(mi_tag)::value;
    for (int t0 = 0; t0 < span; t0 += TPC) {
      const int i = beg + t0 + gl;
      const bool active = i < end;
      float xi = 0.f, yi = 0.f, zi = 0.f;
      bool odd = false, lost = false;
      if (active) {
        const double4 x = ld_pos<DIM>(d.pos + i);
        xi = (float)(x.x - ox);
        yi = (float)(x.y - oy);
        zi = (float)(x.z - oz);
        int ax = 0, ay = 0, az = 0;
        if (own_cell(p, x.x, x.y, x.z, ax, ay, az)) {
          odd = (ax != cx) || (ay != cy) || (DIM == 3 && az != cz);
        } else {
          // not finite or far outside the box: already reported by the hash; no neighbours
          lost = true;
          const bool finite = isfinite(x.x) && isfinite(x.y) && isfinite(x.z);
          raise_status(d, finite ? kStatCellRange : kStatNaN, d.gid[i], kPhaseLists);
        }
      }
      const bool listed = active && !odd && !lost;
      const f32x2 xi2 = f2_pack(xi, xi), yi2 = f2_pack(yi, yi), zi2 = f2_pack(zi, zi);
      const f32x2 ncut22 = f2_pack(-cut2, -cut2);
      int2* col = d.nchunk + (listed ? i : 0);  // this particle's chunks, stride Npad
      int cnt = 0;                              // this lane's candidates
      int kc = 0;                               // this lane's chunks with hits
      for (int ddx = -1; ddx <= 1; ++ddx)
        for (int ddy = -1; ddy <= 1; ++ddy)
          for (int ddz = (DIM == 3 ? -1 : 0); ddz <= (DIM == 3 ? 1 : 0); ++ddz) {
            int nx = cx + ddx, ny = cy + ddy, nz = cz + ddz;
            double sx = 0.0, sy = 0.0, sz = 0.0;
            if (nx < 0) { nx += N0; sx = -p.L[0]; }
            if (nx >= N0) { nx -= N0; sx = p.L[0]; }
            if (DIM == 3) {
              if (nz < 0) { nz += N2; sz = -p.L[2]; }
              if (nz >= N2) { nz -= N2; sz = p.L[2]; }
            }
            if (!p.wall) {
              if (ny < 0) { ny += N1; sy = -p.L[1]; }
              if (ny >= N1) { ny -= N1; sy = p.L[1]; }
            }
            // an empty range where the neighbour row does not exist (walls) or the group idles
            int s = 0, e = -1;
            if (TPC == 32) {
              const int q = ((ddx + 1) * 3 + (ddy + 1)) * kNZ + (DIM == 3 ? ddz + 1 : 0);
              s = __shfl_sync(SPH_FULL, rs, q);
              e = __shfl_sync(SPH_FULL, re, q);
            } else if (live && ny >= 0 && ny < N1) {
              const int nc = p.cell0 + (DIM == 3 ? (nz * N1 + ny) * N0 + nx : ny * N0 + nx);
              s = d.cell_start[nc] + p.slot0;
              e = d.cell_end[nc] + p.slot0;
            }
            const int nch = e >= s ? (e - s + TPC) / TPC : 0;
            const int nchw = TPC == 32 ? nch : warp_max(nch);
            for (int k = 0; k < nchw; ++k) {
              const int c0 = s + k * TPC;
              const int j = c0 + gl;
              float vx = 1e30f, vy = 1e30f, vz = 1e30f;  // padding: never a hit
              if (k < nch && j <= e) {
                const double4 xj = ld_pos<DIM>(d.pos + j);
                if constexpr (kMI) {
                  vx = frame_offset((float)(xj.x - ox), flo, fhi, fL, 0);
                  vy = frame_offset((float)(xj.y - oy), flo, fhi, fL, 1);
                  vz = frame_offset((float)(xj.z - oz), flo, fhi, fL, 2);
                } else {
                  vx = (float)(xj.x + sx - ox);
                  vy = (float)(xj.y + sy - oy);
                  vz = (float)(xj.z + sz - oz);
                }
              }
              stx[gl] = vx;
              sty[gl] = vy;
              if (DIM == 3) stz[gl] = vz;
              __syncwarp();
              const int n = k < nch ? min(TPC, e - c0 + 1) : 0;
              // hit mask of this chunk; staged candidate q is slot c0 + q.  A half-warp group
              // runs a fixed trip count, which keeps both halves on one instruction stream.
              const int m = TPC == 32 ? (n + 3) & ~3 : TPC;
              unsigned hits = 0u;
              if (TPC == 16 || listed) {
  #pragma unroll 1
                for (int q = 0; q < m; q += 4) {
                  const ulonglong2 cx4 = *reinterpret_cast<const ulonglong2*>(stx + q);
                  const ulonglong2 cy4 = *reinterpret_cast<const ulonglong2*>(sty + q);
                  const ulonglong2 cz4 = DIM == 3 ? *reinterpret_cast<const ulonglong2*>(stz + q)
                                                  : make_ulonglong2(0ull, 0ull);
                  hits = list_test2<DIM>(hits, xi2, yi2, zi2, ncut22, cx4.x, cy4.x, cz4.x);
                  hits = list_test2<DIM>(hits, xi2, yi2, zi2, ncut22, cx4.y, cy4.y, cz4.y);
                }
                // first candidate was shifted in first: align it to bit 31 (bit 31 - q is
                // candidate q, the consumers' order of leading zeros)
                hits = m > 0 ? hits << (32 - m) : 0u;
                if (TPC == 16) hits &= (listed && n > 0) ? ~(0xFFFFFFFFu >> n) : 0u;
              }
              if (hits != 0u) {  // a chunk with hits: (first slot, mask) in the next entry
                if (kc < cap) col[(size_t)kc * Np] = make_int2(c0, (int)hits);
                cnt += __popc(hits);
                ++kc;
              }
              __syncwarp();  // the stage is refilled by the next chunk
            }
          }
      if (active && !odd) {
        d.nbr_cnt[i] = cnt;
        d.nbr_nch[i] = min(kc, cap);
      }
      maxch = max(maxch, kc);
      // particles exactly on the upper box edge: their own neighbour cells, the whole warp
      // testing one such particle's candidates at a time
      unsigned odd_mask = __ballot_sync(SPH_FULL, active && odd);
      while (odd_mask) {
        const int l = __ffs(odd_mask) - 1;
        odd_mask &= odd_mask - 1;
        // the particle and its cell's geometry, from the lane that holds it
        const int ti = __shfl_sync(SPH_FULL, i, l);
        const int tb = __shfl_sync(SPH_FULL, b, l);
        const BoxParams& tp = d.box[tb];
        const double4 xt = d.pos[ti];
        int ax = 0, ay = 0, az = 0;
        own_cell(tp, xt.x, xt.y, xt.z, ax, ay, az);  // checked above: cannot fail
        const double tox = ax * tp.cell_size[0];
        const double toy = ay * tp.cell_size[1] - (tp.wall ? tp.wall_width : 0.0);
        const double toz = DIM == 3 ? az * tp.cell_size[2] : 0.0;
        const float tcut2 = (float)tp.list_cut2;
        const float txi = (float)(xt.x - tox), tyi = (float)(xt.y - toy), tzi = (float)(xt.z - toz);
        int tcnt = 0, tk = 0;
        for (int q = 0; q < 9 * kNZ; ++q) {
          int nc;
          if (!neighbour_cell<DIM>(tp, ax, ay, az, q, nc)) continue;
          const int s = d.cell_start[nc] + tp.slot0, e = d.cell_end[nc] + tp.slot0;
          for (int c0 = s; c0 <= e; c0 += 32) {
            const int j = c0 + lane;
            bool hit = false;
            if (j <= e) {
              // rare: every candidate at its minimum image about the particle's own cell
              double4 xj = d.pos[j];
              const float vx = stale_offset((float)(xj.x - tox), tp.cell_size[0], tp.L[0]);
              float vy = (float)(xj.y - toy);
              if (!tp.wall) vy = stale_offset(vy, tp.cell_size[1], tp.L[1]);
              float vz = (float)(xj.z - toz);
              if (DIM == 3) vz = stale_offset(vz, tp.cell_size[2], tp.L[2]);
              const float rx = txi - vx;
              const float ry = tyi - vy;
              float r2 = rx * rx + ry * ry;
              if (DIM == 3) {
                const float rz = tzi - vz;
                r2 += rz * rz;
              }
              hit = r2 < tcut2;
            }
            const unsigned hits = __brev(__ballot_sync(SPH_FULL, hit));
            if (hits != 0u) {
              if (lane == 0 && tk < cap) d.nchunk[(size_t)tk * Np + ti] = make_int2(c0, (int)hits);
              tcnt += __popc(hits);
              ++tk;
            }
          }
        }
        if (lane == 0) {
          d.nbr_cnt[ti] = tcnt;
          d.nbr_nch[ti] = min(tk, cap);
        }
        maxch = max(maxch, tk);
      }
    }
  };
  if (mi)
    walk(std::true_type{});
  else
    walk(std::false_type{});
  // warp max of the chunk counts -> capacity check
  maxch = warp_max(maxch);
  if (lane == 0 && maxch > 0) {
    atomicMax(&d.err_info[kErrMaxCount], maxch);
    if (maxch > cap) raise_status(d, kStatCapacity, 0, kPhaseLists);
  }
}

// Colloid coarse grid (kernel_cell_colloids_list.cu, kernel_initialize_cell_colloids.cu,
// kernel_cell_colloids_ranges.cu) with the stable (cell, index) order of thrust's sort.
// One block per box.
__global__ void k_colloid_cells(Dev d, int nboxes) {
  const int b = blockIdx.x;
  if (b >= nboxes) return;
  if (step_aborted(d)) return;
  const BoxParams& p = d.box[b];
  const int n = p.N_colloids;
  if (n < 2) return;
  const int c0 = p.coll0, nc = d.ncoll;
  extern __shared__ int s_cell[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double x = d.cs[CS_X * nc + c0 + i], y = d.cs[CS_Y * nc + c0 + i];
    int cx = (int)floor(x / p.cell_colloids_size[0]);
    int cy = (int)floor(y / p.cell_colloids_size[1]);
    int c;
    if (p.dim == 3) {
      int cz = (int)floor(d.cs[CS_Z * nc + c0 + i] / p.cell_colloids_size[2]);
      c = cz * p.Ncells_colloids[0] * p.Ncells_colloids[1] + cy * p.Ncells_colloids[0] + cx;
    } else {
      c = cy * p.Ncells_colloids[0] + cx;
    }
    s_cell[i] = c;
  }
  for (int c = threadIdx.x; c < p.Ntotal_cells_colloids; c += blockDim.x) {
    d.ccell_start[p.ccell0 + c] = -1;
    d.ccell_end[p.ccell0 + c] = -2;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int ci = s_cell[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) rank += (s_cell[j] < ci) || (s_cell[j] == ci && j < i);
    d.ccell[c0 + rank] = ci;
    d.cindex[c0 + rank] = i;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int ci = d.ccell[c0 + i];
    if (ci < 0 || ci >= p.Ntotal_cells_colloids) continue;
    if (i == 0 || d.ccell[c0 + i - 1] != ci) d.ccell_start[p.ccell0 + ci] = i;
    if (i == n - 1 || d.ccell[c0 + i + 1] != ci) d.ccell_end[p.ccell0 + ci] = i;
  }
}

// One lane's density sum over its list, in list order.  The positions of kAhead entries are
// loaded before they are summed (each term depends on a gathered position: with one load in
// flight per lane the pass waited on memory, 5 long-scoreboard stalls per instruction).
// Measured at 128^3 (FP64, with the plain separations): 1.16 ms with one entry at a time,
// 1.10 ms with two, 1.21 and 1.22 ms with three and four (registers, fewer warps).
template <typename T, int DIM, bool WRAP>
__device__ __forceinline__ double density_sum(const Dev& d, const typename V4<T>::type* P,
                                              int i, const BoxParams& p) {
  using V = typename V4<T>::type;
  constexpr int kAhead = 2;
  const T L[3] = {(T)p.L[0], (T)p.L[1], (T)p.L[2]};
  const T h[3] = {(T)p.halfL[0], (T)p.halfL[1], (T)p.halfL[2]};
  const T rcutsq = (T)p.rcutsq;
  const T rcut_inv = (T)p.rcut_inv, cw = (T)p.cw;
  const V xi = ld_pos<DIM>(P + i);
  const int n = d.nbr_cnt[i];
  NbrIter it;
  it.init(d, i);
  typename SumKind<T>::S dens = 0;
  T comp = T(0);  // Kahan compensation of a float sum
  for (int k = 0; k < n; k += kAhead) {
    int j[kAhead];
    V x[kAhead];
#pragma unroll
    for (int u = 0; u < kAhead; ++u) j[u] = k + u < n ? it.next() : -1;
#pragma unroll
    for (int u = 0; u < kAhead; ++u) x[u] = ld_pos<DIM>(P + (j[u] >= 0 ? j[u] : i));
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      if (j[u] < 0) break;
      const T w = density_term<T, DIM, WRAP>(xi, x[u], L, h, p.wall, rcutsq, rcut_inv, cw);
      if constexpr (Compensated<T>::on)
        kahan_add(dens, comp, w);
      else
        dens = dens + w;
    }
  }
  return (double)dens - (double)comp;
}

// Whole warps (lanes past the end mirror the last slot and store nothing), so that a warp
// of particles clear of the periodic faces takes the sums without the minimum image.
template <typename T, int DIM>
__global__ void k_density(Dev d) {
  using V = typename V4<T>::type;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 - (int)(threadIdx.x & 31) >= d.Ntot) return;  // whole warps only
  if (step_aborted_warp(d)) return;
  const bool active = i0 < d.Ntot;
  const int i = active ? i0 : d.Ntot - 1;
  // positions: the double state itself, or its float copy in mixed precision
  const V* __restrict__ P = sizeof(T) == 8 ? reinterpret_cast<const V*>(d.pos)
                                           : reinterpret_cast<const V*>(d.pos_f);
  const BoxParams& p = d.box[box_of(d.tinfo[i])];
  const V xi = ld_pos<DIM>(P + i);
  double dens;
  if (warp_plain_image(d, clear_of_faces<T, DIM>(p, xi.x, xi.y, xi.z)))
    dens = density_sum<T, DIM, false>(d, P, i, p);
  else
    dens = density_sum<T, DIM, true>(d, P, i, p);
  if (active) density_epilogue<T, DIM>(d, i, p, dens);
}

// Density over neighbour-cell tiles: one warp per cell, as the list build.  The positions
// of the neighbour cells' candidate ranges (the list build's ranges, stale ones included)
// are staged in shared memory by coalesced copies, in phases of 9 cells (the dx = -1, 0, +1
// planes in 3D; all 9 cells at once in 2D), and every lane walks its own list in order,
// reading each neighbour from the tile.  The sums are those of k_density term for term:
// the same list order, the same arithmetic; only where the position is read from differs.
// An entry outside the staged ranges (a tile overflow, or a particle listed from other
// cells because it sits exactly on the upper box edge) reads its position from global
// memory in place, so the order is never changed.
constexpr int kDensWarps = 4;
constexpr int kDensTile = 320;  // staged positions per warp and phase

template <typename T, int DIM>
__global__ void __launch_bounds__(kDensWarps * 32) k_density_cells(Dev d) {
  using V = typename V4<T>::type;
  constexpr int kNZ = DIM == 3 ? 3 : 1;
  constexpr int kNR = 9 * kNZ;               // neighbour cells
  constexpr int kPh = DIM == 3 ? 3 : 1;      // phases
  constexpr int kPerPh = kNR / kPh;          // cells per phase (9)
  __shared__ T tx[kDensWarps][kDensTile], ty[kDensWarps][kDensTile], tz[kDensWarps][kDensTile];
  __shared__ int rtab[kDensWarps][kPerPh][3];  // per phase: first slot, last slot, tile offset
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * kDensWarps + w;
  if (cell >= d.Ctot) return;  // whole warps only
  if (step_aborted_warp(d)) return;
  const V* __restrict__ P = sizeof(T) == 8 ? reinterpret_cast<const V*>(d.pos)
                                           : reinterpret_cast<const V*>(d.pos_f);
  const int b = d.cell_box[cell];
  const BoxParams& p = d.box[b];
  const int N0 = p.Ncells[0], N1 = p.Ncells[1], N2 = p.Ncells[2];
  const int lc = cell - p.cell0;
  const int cx = lc % N0, cy = (lc / N0) % N1, cz = DIM == 3 ? lc / (N0 * N1) : 0;
  // candidate range of neighbour cell `lane` (the list build's, kernel_densities.cu:52-163)
  int rs = 0, re = -1;
  if (lane < kNR) {
    const int ddx = lane / (3 * kNZ) - 1, ddy = (lane / kNZ) % 3 - 1;
    const int ddz = DIM == 3 ? lane % 3 - 1 : 0;
    int nx = cx + ddx, ny = cy + ddy, nz = cz + ddz;
    if (nx < 0) nx += N0;
    if (nx >= N0) nx -= N0;
    if (DIM == 3) {
      if (nz < 0) nz += N2;
      if (nz >= N2) nz -= N2;
    }
    if (!p.wall) {
      if (ny < 0) ny += N1;
      if (ny >= N1) ny -= N1;
    }
    if (ny >= 0 && ny < N1) {
      const int nc = p.cell0 + (DIM == 3 ? (nz * N1 + ny) * N0 + nx : ny * N0 + nx);
      rs = d.cell_start[nc] + p.slot0;
      re = d.cell_end[nc] + p.slot0;
    }
  }
  const int rcount = re >= rs ? re - rs + 1 : 0;
  const T L[3] = {(T)p.L[0], (T)p.L[1], (T)p.L[2]};
  const T h[3] = {(T)p.halfL[0], (T)p.halfL[1], (T)p.halfL[2]};
  const T rcutsq = (T)p.rcutsq;
  const T rcut_inv = (T)p.rcut_inv, cw = (T)p.cw;
  const int beg = d.cell_begin[cell], end = d.cell_begin[cell + 1];
  for (int t0 = 0; t0 < end - beg; t0 += 32) {
    const int i = beg + t0 + lane;
    const bool active = i < end;
    const V xi = active ? ld_pos<DIM>(P + i) : V{};
    const int n = active ? d.nbr_cnt[i] : 0;
    NbrIter it;
    it.init(d, active ? i : beg);
    // the next list entry not yet summed (-1: none left)
    int jn = n > 0 ? it.next() : -1;
    typename SumKind<T>::S dens = 0;
  T comp = T(0);  // Kahan compensation of a float sum
    auto add = [&](const V& xj) {
      const T wv = density_term<T, DIM>(xi, xj, L, h, p.wall, rcutsq, rcut_inv, cw);
      if constexpr (Compensated<T>::on)
        kahan_add(dens, comp, wv);
      else
        dens = dens + wv;
    };
    int k = 0;
    for (int ph = 0; ph < kPh; ++ph) {
      // tile offsets of this phase's ranges: exclusive prefix over lanes ph*9 .. ph*9+8
      const bool mine = lane >= ph * kPerPh && lane < (ph + 1) * kPerPh;
      int off = mine ? rcount : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(SPH_FULL, off, o);
        if (lane >= o) off += v;
      }
      off -= mine ? rcount : 0;
      if (mine) {
        rtab[w][lane - ph * kPerPh][0] = rs;
        rtab[w][lane - ph * kPerPh][1] = re;
        rtab[w][lane - ph * kPerPh][2] = off;
      }
      // stage the phase's ranges (coalesced), up to the tile capacity
#pragma unroll 1
      for (int q = 0; q < kPerPh; ++q) {
        const int qs = __shfl_sync(SPH_FULL, rs, ph * kPerPh + q);
        const int qn = __shfl_sync(SPH_FULL, rcount, ph * kPerPh + q);
        const int qo = __shfl_sync(SPH_FULL, off, ph * kPerPh + q);
        for (int u = lane; u < qn && qo + u < kDensTile; u += 32) {
          const V x = ld_pos<DIM>(P + qs + u);
          tx[w][qo + u] = x.x;
          ty[w][qo + u] = x.y;
          if (DIM == 3) tz[w][qo + u] = x.z;
        }
      }
      __syncwarp();
      // this lane's list entries that fall in the phase's ranges, in list order
      int qc = 0;
      int qs = rtab[w][0][0], qe = rtab[w][0][1], qo = rtab[w][0][2];
      while (k < n && jn >= 0) {
        const int j = jn;
        while (qc < kPerPh && (j < qs || j > qe)) {
          if (++qc < kPerPh) {
            qs = rtab[w][qc][0];
            qe = rtab[w][qc][1];
            qo = rtab[w][qc][2];
          }
        }
        if (qc == kPerPh) break;  // a later phase's entry
        const int t = qo + (j - qs);
        V xj;
        if (t < kDensTile) {
          xj.x = tx[w][t];
          xj.y = ty[w][t];
          xj.z = DIM == 3 ? tz[w][t] : T(0);
        } else {
          xj = ld_pos<DIM>(P + j);
        }
        add(xj);
        ++k;
        jn = k < n ? it.next() : -1;
      }
      __syncwarp();  // the tile and the range table are refilled by the next phase
    }
    // entries from no staged range: global reads, still in list order
    for (; k < n && jn >= 0; ++k) {
      add(ld_pos<DIM>(P + jn));
      jn = k + 1 < n ? it.next() : -1;
    }
    if (active) density_epilogue<T, DIM>(d, i, p, (double)dens - (double)comp);
  }
}

// kernel_pressures.cu:13-23 (standalone, also refreshes the neighbour record)
template <typename T>
__global__ void k_pressure(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  const int ti = d.tinfo[i];
  const BoxParams& p = d.box[box_of(ti)];
  const double dens = d.dens[i];
  const double press = p.csq * (d.pos[i].w * dens - p.rho0);
  d.press[i] = press;
  if (p.dim == 3)
    write_record<T, 3>(d, i, p, ti, dens, press);
  else
    write_record<T, 2>(d, i, p, ti, dens, press);
}

// Pair pass (kernel_vel_gradients.cu:15-662 and kernel_forces.cu:15-865 in one sweep),
// one lane per particle over its neighbour list.
//
// Gather: at list position k every lane needs one neighbour record (128 B in FP64, 64 B
// in mixed precision), each at its own address.  Loaded lane by lane, one 16-byte piece
// per instruction, that is 32 separate cache lines per instruction.  Instead the warp
// copies the 32 records into shared memory cooperatively: kPieces consecutive lanes move
// the pieces of one record, so one copy instruction covers whole lines of 32 / kPieces
// records.  The copies for the next position are in flight (cp.async, double buffer)
// while the current ones are evaluated.  Each lane then reads its records
// from shared memory (row stride padded by one piece: conflict-free).
//
// Launch shape of the pair pass per precision and dimension, as measured on B200.  Every pass
// evaluates one list position per step: with the fluid-fluid form of that walk, evaluating two
// positions side by side (to overlap their dependency chains) measured slower everywhere
// (float 3D at 128^3 2.41 vs 2.38 ms, FP64 2D on the 512-box ensemble 3.63 vs 3.52 ms).
//  - kWarps: warps per block; kMinBlocks: resident blocks per SM the register allocation
//    is held to (FP64 3D: 168 registers, which its working set fits without spilling;
//    float 3D 128; FP64 2D 96, with a few spills: 5 blocks 3.52 ms, 4 blocks 3.58 ms; the
//    float 2D pass 80, in 2-warp blocks).
//  - One-box 3D contexts (k_pairs<..., ONE = true>) read the pair constants from the
//    constant bank (Dev::pc) instead of registers: 128^3 pair pass 3.59 -> 3.55 ms (FP64)
//    and 2.43 -> 2.38 ms (mixed) at the same shape.  The FP64 3D pass then fits 128
//    registers with 32 bytes of spill, but at 16 warps per SM (4 blocks of 4 warps or 8 of
//    2) it took 4.03 and 3.98 ms: the larger shared-memory carve-out leaves L1 too little
//    for the record gathers.
template <typename T, int DIM>
struct PairShape {
  using Rec = typename RecFor<T, DIM>::type;
  static constexpr bool kF64 = sizeof(T) == 8;
  static constexpr bool kF2D = !kF64 && DIM == 2;
  static constexpr bool kF64_3D = kF64 && DIM == 3;
  // the float 2D pass runs 2-warp blocks (measured 2.29 vs 2.35 ms on the 512-box ensemble;
  // the float 3D pass was slower with them, the FP64 passes unchanged)
  static constexpr int kWarps = kF2D ? 2 : 4;
  static constexpr int kMinBlocks = kF2D ? 6 : (kF64_3D ? 3 : (kF64 ? 5 : 4));
};

// The pair constants of a one-box context, viewed as PairParams (same layout).
template <typename T, int DIM>
__device__ __forceinline__ const PairParams<T, DIM>& one_box_params(const Dev& d) {
  static_assert(sizeof(PairParams<double, DIM>) == 11 * sizeof(double) &&
                    sizeof(PairParams<float, DIM>) == 11 * sizeof(float),
                "PairParams layout");
  if constexpr (sizeof(T) == 8)
    return *reinterpret_cast<const PairParams<T, DIM>*>(d.pc.L);
  else
    return *reinterpret_cast<const PairParams<T, DIM>*>(d.pc.Lf);
}

template <typename Rec>
struct PairStage {
  static constexpr int kPieces = (int)(sizeof(Rec) / 16);  // 16-byte pieces per record
  static constexpr int kStride = kPieces + 1;               // padded row, in pieces
  static constexpr int kPerCopy = 32 / kPieces;             // records per copy instruction
  static constexpr int kRows = 32 * kStride;                // one position, in pieces
  union Slot {
    int4 v[kPieces];
    Rec r;
  };
};

// L1: the copy allocates in L1 (.ca) or goes through L2 only (.cg).  The 3D records are
// staged through L1 (reused by the neighbouring warps of the SM), the 2D records (64 and 32
// bytes) through L2 only: measured 3.74 vs 3.78 ms (FP64 3D), 2.33 vs 2.44 ms (float 3D),
// 3.28 vs 3.33 ms (FP64 2D ensemble) and 2.28 vs 2.29 ms (float 2D ensemble).
template <bool L1>
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (L1)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_prev() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Lane `lane` copies its piece of the records the warp's lanes list at one position
// (jn: this lane's neighbour there, -1 for none) into row block `buf`.
template <typename Rec>
__device__ __forceinline__ void stage_records(int4* buf, const Rec* __restrict__ rec, int jn,
                                              int lane) {
  using St = PairStage<Rec>;
  const int piece = lane % St::kPieces;
#pragma unroll
  for (int t = 0; t < St::kPieces; ++t) {
    const int r = t * St::kPerCopy + lane / St::kPieces;
    const int jr = __shfl_sync(SPH_FULL, jn, r);
    if (jr >= 0)
      cp_async16<std::is_same<Rec, RecD>::value || std::is_same<Rec, RecF>::value>(
          buf + r * St::kStride + piece, reinterpret_cast<const int4*>(rec + jr) + piece);
  }
}

// A lane's view of one staged record: FP64 records are read in place, each field loaded
// from shared memory where the pair term uses it, which keeps the 128-byte record out of
// the register file; float records are copied into registers.
template <typename T, typename Rec>
struct StagedRec {
  const Rec& r;
  __device__ __forceinline__ explicit StagedRec(const int4* src)
      : r(*reinterpret_cast<const Rec*>(src)) {}
};
template <typename Rec>
struct StagedRec<float, Rec> {
  Rec r;
  __device__ __forceinline__ explicit StagedRec(const int4* src) {
    typename PairStage<Rec>::Slot s;
#pragma unroll
    for (int t = 0; t < PairStage<Rec>::kPieces; ++t) s.v[t] = src[t];
    r = s.r;
  }
};

// Everything a lane's walk over its list needs.
template <typename T, int DIM>
struct PairWalk {
  using Rec = typename RecFor<T, DIM>::type;
  const Dev& d;
  const Rec* __restrict__ rec;
  int4* sb;                      // the warp's staging rows
  int lane, i, n, nmax;
  const BoxParams& p;
  const PairParams<T, DIM>& pp;
  const CollView& cv;
  const PairOwn<T, DIM>& o;
};

// A lane's walk over its list, one position per step: the copies for position k + 1 are in
// flight while k is evaluated.  WRAP: see min_image.
template <typename T, int DIM, bool WRAP, int MODE>
__device__ __forceinline__ void pair_walk(const PairWalk<T, DIM>& W, NbrIter& it,
                                           PairAcc<T, DIM>& acc) {
  using Rec = typename RecFor<T, DIM>::type;
  using St = PairStage<Rec>;
  const int n = W.n, lane = W.lane;
  int jc = n > 0 ? it.next() : -1;
  // 2D records carry no type word: the neighbour's is read from the type array one
  // position ahead, with its record's copy
  int tc = DIM == 2 && jc >= 0 ? __ldg(&W.d.tinfo[jc]) : 0;
  stage_records<Rec>(W.sb, W.rec, jc, lane);
  cp_async_commit();
  for (int k = 0; k < W.nmax; ++k) {
    const int k1 = k + 1;
    const int jn = k1 < n ? it.next() : -1;
    if (k1 < W.nmax) stage_records<Rec>(W.sb + (k1 & 1) * St::kRows, W.rec, jn, lane);
    const int tn = DIM == 2 && jn >= 0 ? __ldg(&W.d.tinfo[jn]) : 0;
    cp_async_commit();
    cp_async_wait_prev();  // position k has landed (this lane's copies) ...
    __syncwarp();          // ... and every other lane's
    const bool valid = jc >= 0 && jc != W.i;
    const StagedRec<T, Rec> R(W.sb + (k & 1) * St::kRows + lane * St::kStride);
    int tj;
    if constexpr (DIM == 3) tj = type_of(R.r.tinfo); else tj = type_of(tc);
    // the fluid-fluid form where every lane of the warp qualifies (a warp split between the
    // forms would run both)
    if (__all_sync(SPH_FULL, W.o.fluid && (!valid || tj == 0)))
      pair_fluid_x1<T, DIM, WRAP, MODE>(W.p, W.pp, W.o, R.r, valid, acc);
    else if (valid)
      pair_term<T, DIM, WRAP>(W.p, W.pp, W.cv, W.o, R.r, tj, acc);
    __syncwarp();  // buffer k & 1 is refilled at position k + 2
    jc = jn;
    tc = tn;
  }
}

template <typename T, int DIM, int MODE, bool EXT, bool ONE>
__global__ void __launch_bounds__(PairShape<T, DIM>::kWarps * 32,
                                  PairShape<T, DIM>::kMinBlocks)
    k_pairs(const __grid_constant__ Dev d) {
  using Sh = PairShape<T, DIM>;
  using Rec = typename Sh::Rec;
  using St = PairStage<Rec>;
  // per warp: a double buffer of staged positions
  __shared__ int4 stage[Sh::kWarps][2][St::kRows];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wbase = (blockIdx.x * Sh::kWarps + w) * 32;
  if (wbase >= d.Ntot) return;  // whole warps only: the lanes below cooperate
  if (step_aborted_warp(d)) return;
  const int i = wbase + lane;
  const bool active = i < d.Ntot;
  const int is = active ? i : wbase;  // lanes past the end mirror a valid slot, compute nothing

  const Rec* __restrict__ rec = reinterpret_cast<const Rec*>(d.rec);
  const int ti = d.tinfo[is];
  const BoxParams& p = d.box[box_of(ti)];
  PairParams<T, DIM> ppl;
  if constexpr (!ONE) ppl.load(p);
  const PairParams<T, DIM>& pp = ONE ? one_box_params<T, DIM>(d) : ppl;
  const CollView cv{d.cs, d.ncoll};
  PairOwn<T, DIM> o;
  load_own<T, DIM, MODE>(d, is, ti, rec[is], o);
  PairAcc<T, DIM> acc;
  acc.zero();
  const int n = active ? d.nbr_cnt[i] : 0;
  int nmax = n;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) nmax = max(nmax, __shfl_xor_sync(SPH_FULL, nmax, s));
  NbrIter it;
  it.init(d, is);
  const PairWalk<T, DIM> W{d, rec, &stage[w][0][0], lane, i, n, nmax, p, pp, cv, o};
  auto walk = [&](auto wrap_tag) {
    pair_walk<T, DIM, decltype(wrap_tag)::value, MODE>(W, it, acc);
  };
  // Warps clear of the periodic faces drop the minimum image, in 3D only: the 512-box 2D
  // ensemble's small boxes put both kinds of warp on every SM, and the second copy of the
  // walk cost more in instruction fetch than the shorter separations saved (FP64 2D pair
  // pass 3.52 -> 3.54 ms, float 2D 2.23 -> 2.38 ms); the 3D passes gain 5 %.
  if constexpr (DIM == 3) {
    if (warp_plain_image(d, clear_of_faces<T, DIM>(p, o.x, o.y, o.z)))
      walk(std::false_type{});
    else
      walk(std::true_type{});
  } else {
    walk(std::true_type{});
  }
  if (active) pair_store<T, DIM, MODE, EXT>(d, i, p, o, acc);
}

// kernel_ext_force.cu:13-73 as a separate pass (class_system::calculate_external_forces)
__global__ void k_ext_force(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  const int ti = d.tinfo[i];
  if (type_of(ti) != 0) return;
  const BoxParams& p = d.box[box_of(ti)];
  const int Np = d.Npad;
  const double4 x = d.pos[i];
  const double m = x.w;
  if (p.ext_force_type == 1) {
    d.f[i] += m * p.ext_force[0];
    d.f[Np + i] += m * p.ext_force[1];
    if (p.dim == 3) d.f[2 * Np + i] += m * p.ext_force[2];
  } else if (p.ext_force_type == 2) {
    d.f[i] += m * p.ext_force[0] * sin(p.ky * x.y);
    d.f[Np + i] += 0.0;
    if (p.dim == 3) d.f[2 * Np + i] += 0.0;
  } else if (p.ext_force_type == 3) {
    d.f[i] += (x.y < 0.5 * p.L[1]) ? m * p.ext_force[0] : -(m * p.ext_force[0]);
    d.f[Np + i] += 0.0;
    if (p.dim == 3) d.f[2 * Np + i] += 0.0;
  }
}

// dc/dt from the stored gradient (kernel_dcdt.cu:15-104), used after a standalone
// velocity-gradient pass.
__global__ void k_dcdt(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  if (step_aborted(d)) return;
  const int ti = d.tinfo[i];
  const int Np = d.Npad;
  if (type_of(ti) != 0) {
    // kernel_dcdt.cu:39: walls and colloids keep their initial zero
    for (int q = 0; q < 6; ++q) d.dcdt[q * Np + i] = 0.0;
    return;
  }
  const BoxParams& p = d.box[box_of(ti)];
  const double tinv = 1.0 / p.tau;
  const double* G = d.gradv;
  const double cxx = d.conf[i], cxy = d.conf[Np + i], cyy = d.conf[2 * Np + i];
  const double gxx = G[i], gxy = G[Np + i], gyx = G[3 * Np + i], gyy = G[4 * Np + i];
  if (p.dim == 2) {
    const double Axx = cxx * gxx + cxy * gyx, Axy = cxx * gxy + cxy * gyy;
    const double Ayx = cxy * gxx + cyy * gyx, Ayy = cxy * gxy + cyy * gyy;
    d.dcdt[i] = 2.0 * Axx + tinv * (1.0 - cxx);
    d.dcdt[Np + i] = Axy + Ayx - tinv * cxy;
    d.dcdt[2 * Np + i] = 2.0 * Ayy + tinv * (1.0 - cyy);
    d.dcdt[3 * Np + i] = 0.0;
    d.dcdt[4 * Np + i] = 0.0;
    d.dcdt[5 * Np + i] = 0.0;
    return;
  }
  const double cxz = d.conf[3 * Np + i], cyz = d.conf[4 * Np + i], czz = d.conf[5 * Np + i];
  const double gxz = G[2 * Np + i], gyz = G[5 * Np + i], gzx = G[6 * Np + i],
               gzy = G[7 * Np + i], gzz = G[8 * Np + i];
  const double Axx = cxx * gxx + cxy * gyx + cxz * gzx;
  const double Axy = cxx * gxy + cxy * gyy + cxz * gzy;
  const double Axz = cxx * gxz + cxy * gyz + cxz * gzz;
  const double Ayx = cxy * gxx + cyy * gyx + cyz * gzx;
  const double Ayy = cxy * gxy + cyy * gyy + cyz * gzy;
  const double Ayz = cxy * gxz + cyy * gyz + cyz * gzz;
  const double Azx = cxz * gxx + cyz * gyx + czz * gzx;
  const double Azy = cxz * gxy + cyz * gyy + czz * gzy;
  const double Azz = cxz * gxz + cyz * gyz + czz * gzz;
  d.dcdt[i] = 2.0 * Axx + tinv * (1.0 - cxx);
  d.dcdt[Np + i] = Axy + Ayx - tinv * cxy;
  d.dcdt[2 * Np + i] = 2.0 * Ayy + tinv * (1.0 - cyy);
  d.dcdt[3 * Np + i] = Axz + Azx - tinv * cxz;
  d.dcdt[4 * Np + i] = Ayz + Azy - tinv * cyz;
  d.dcdt[5 * Np + i] = 2.0 * Azz + tinv * (1.0 - czz);
}

// ---------------------------------------------------------------------------------
// Wall forces (kernel_collect_force_walls.cu:15-50) and colloid forces and torques
// (kernel_collect_force_colloids.cu:15-99): one block per wall / colloid, a fixed-order
// FP64 tree reduction in place of the reference's one-thread serial loop.
// ---------------------------------------------------------------------------------
constexpr int kRedThreads = 256;

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double (*sh)[kRedThreads]) {
#pragma unroll
  for (int q = 0; q < NV; ++q) sh[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int q = 0; q < NV; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = sh[q][0];
}

// Pass 1: one block per chunk of a wall's list (kWallChunk entries at most).
__global__ void __launch_bounds__(kRedThreads) k_wall_forces(Dev d) {
  __shared__ double sh[3][kRedThreads];
  const int k = blockIdx.x;
  if (k >= d.nwallchunks) return;
  if (step_aborted(d)) return;
  const int j0 = d.wall_chunk[k], j1 = d.wall_chunk[k + 1];
  const int Np = d.Npad;
  double v[3] = {0.0, 0.0, 0.0};
  for (int j = j0 + threadIdx.x; j < j1; j += kRedThreads) {
    const int s = d.inv[d.walls_list[j]];
    v[0] += d.f[s];
    v[1] += d.f[Np + s];
    v[2] += d.f[2 * Np + s];
  }
  block_reduce<3>(v, sh);
  if (threadIdx.x == 0) {
    d.wall_part[3 * k + 0] = v[0];
    d.wall_part[3 * k + 1] = v[1];
    d.wall_part[3 * k + 2] = v[2];
  }
}

// Pass 2: one warp per wall adds its chunks' partial sums in a fixed order.
__global__ void k_wall_forces_final(Dev d) {
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= d.nwallseg) return;
  if (step_aborted(d)) return;
  const int c0 = d.wall_seg_chunk[w], c1 = d.wall_seg_chunk[w + 1];
  double v[3] = {0.0, 0.0, 0.0};
  for (int c = c0 + lane; c < c1; c += 32) {
    v[0] += d.wall_part[3 * c + 0];
    v[1] += d.wall_part[3 * c + 1];
    v[2] += d.wall_part[3 * c + 2];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < 3; ++q) v[q] += __shfl_xor_sync(SPH_FULL, v[q], o);
  if (lane == 0) {
    d.wall_f[3 * w + 0] = v[0];
    d.wall_f[3 * w + 1] = v[1];
    d.wall_f[3 * w + 2] = v[2];
  }
}

__global__ void __launch_bounds__(kRedThreads) k_collect_colloids(Dev d) {
  __shared__ double sh[6][kRedThreads];
  const int c = blockIdx.x;
  if (c >= d.ncoll) return;
  if (step_aborted(d)) return;
  const BoxParams& p = d.box[d.coll_box[c]];
  const int nc = d.ncoll, Np = d.Npad;
  const double cx = d.cs[CS_X * nc + c], cy = d.cs[CS_Y * nc + c], cz = d.cs[CS_Z * nc + c];
  const int j0 = d.coll_seg[c], j1 = d.coll_seg[c + 1];
  double v[6] = {0, 0, 0, 0, 0, 0};  // F x y z, T x y z
  for (int j = j0 + threadIdx.x; j < j1; j += kRedThreads) {
    const int s = d.inv[d.colloids_list[j]];
    const double4 x = d.pos[s];
    const double fx = d.f[s], fy = d.f[Np + s], fz = p.dim == 3 ? d.f[2 * Np + s] : 0.0;
    double rx = x.x - cx, ry = x.y - cy, rz = 0.0;
    if (rx > 0.5 * p.L[0]) rx -= p.L[0];
    if (rx < -0.5 * p.L[0]) rx += p.L[0];
    if (p.wall == 0) {
      if (ry > 0.5 * p.L[1]) ry -= p.L[1];
      if (ry < -0.5 * p.L[1]) ry += p.L[1];
    }
    if (p.dim == 3) {
      rz = x.z - cz;
      if (rz > 0.5 * p.L[2]) rz -= p.L[2];
      if (rz < -0.5 * p.L[2]) rz += p.L[2];
    }
    v[0] += fx;
    v[1] += fy;
    v[2] += fz;
    v[3] += ry * fz - rz * fy;
    v[4] += rz * fx - rx * fz;
    v[5] += rx * fy - ry * fx;
  }
  block_reduce<6>(v, sh);
  if (threadIdx.x == 0) {
    double* cs = d.cs;
    cs[CS_FX * nc + c] = v[0];
    cs[CS_FY * nc + c] = v[1];
    cs[CS_TZ * nc + c] = v[5];
    if (p.dim == 3) {
      cs[CS_FZ * nc + c] = v[2];
      cs[CS_TX * nc + c] = v[3];
      cs[CS_TY * nc + c] = v[4];
    }
  }
}

// Colloid-colloid repulsion (kernel_repulsion_force_colloids.cu:21-207, r^2 clamped to the
// cut-on before normalising) then rotating-field dipole force
// (kernel_magnetic_force_colloids.cu:15-203, 3D e scaled to |e| = R), over the coarse
// grid in the reference's order.  One thread per colloid.
__device__ __forceinline__ int coll_neigh_cells(const BoxParams& p, double x, double y,
                                                double z, int* cells) {
  const int* Nc = p.Ncells_colloids;
  const double fx = floor(x / p.cell_colloids_size[0]);
  const double fy = floor(y / p.cell_colloids_size[1]);
  const double fz = p.dim == 3 ? floor(z / p.cell_colloids_size[2]) : 0.0;
  // a colloid centre that is not finite or lies beyond one periodic image has no
  // neighbour cells (every index built below then stays inside the coarse grid)
  if (!(fx >= 1.0 - Nc[0] && fx <= 2.0 * Nc[0] - 2.0)) return 0;
  if (!(fy >= -2.0 * Nc[1] && fy <= 3.0 * Nc[1])) return 0;
  if (p.wall == 0 && !(fy >= 1.0 - Nc[1] && fy <= 2.0 * Nc[1] - 2.0)) return 0;
  if (p.dim == 3 && !(fz >= 1.0 - Nc[2] && fz <= 2.0 * Nc[2] - 2.0)) return 0;
  const int cxi = (int)fx, cyi = (int)fy, czi = (int)fz;
  int n = 0;
  const int dz0 = p.dim == 3 ? -1 : 0, dz1 = p.dim == 3 ? 1 : 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = dz0; dz <= dz1; ++dz) {
        int cx = cxi + dx, cy = cyi + dy, cz = czi + dz;
        if (cx < 0) cx += Nc[0];
        if (cx >= Nc[0]) cx -= Nc[0];
        if (p.wall == 0) {
          if (cy < 0) cy += Nc[1];
          if (cy >= Nc[1]) cy -= Nc[1];
        }
        if (p.dim == 3) {
          if (cz < 0) cz += Nc[2];
          if (cz >= Nc[2]) cz -= Nc[2];
        }
        if (cy >= 0 && cy < Nc[1])
          cells[n++] = p.dim == 3 ? cz * Nc[0] * Nc[1] + cy * Nc[0] + cx : cy * Nc[0] + cx;
      }
  return n;
}

__global__ void k_colloid_pairs(Dev d) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.ncoll) return;
  if (step_aborted(d)) return;
  const int b = d.coll_box[c];
  const BoxParams& p = d.box[b];
  if (p.N_colloids < 2) return;
  const int nc = d.ncoll, c0 = p.coll0, i = c - c0;
  const double* cs = d.cs;
  const double xi = cs[CS_X * nc + c], yi = cs[CS_Y * nc + c], zi = cs[CS_Z * nc + c];
  const double L[3] = {p.L[0], p.L[1], p.L[2]};
  const double h[3] = {p.halfL[0], p.halfL[1], p.halfL[2]};
  double F[3] = {cs[CS_FX * nc + c], cs[CS_FY * nc + c], cs[CS_FZ * nc + c]};
  int cells[27];
  const int ncell = coll_neigh_cells(p, xi, yi, zi, cells);
  const double Famp = p.F0_rep * p.tau_rep;
  const double* m = d.mag + 3 * b;
  for (int pass = 0; pass < 2; ++pass) {
    for (int q = 0; q < ncell; ++q) {
      const int cc = p.ccell0 + cells[q];
      const int s = d.ccell_start[cc], e = d.ccell_end[cc];
      for (int k = s; k <= e; ++k) {
        const int j = d.cindex[c0 + k];
        if (i == j) continue;
        double r[3] = {xi - cs[CS_X * nc + c0 + j], yi - cs[CS_Y * nc + c0 + j],
                       p.dim == 3 ? zi - cs[CS_Z * nc + c0 + j] : 0.0};
        if (p.dim == 3)
          min_image<double, 3>(r[0], r[1], r[2], L, h, p.wall);
        else
          min_image<double, 2>(r[0], r[1], r[2], L, h, p.wall);
        double r2 = p.dim == 3 ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2]
                               : r[0] * r[0] + r[1] * r[1];
        if (pass == 0) {
          if (r2 < p.rcuton_coll_rep_sq) r2 = p.rcuton_coll_rep_sq;
          if (r2 <= p.rcutoff_coll_rep_sq) {
            const double rr = sqrt(r2);
            const double ts = -p.tau_rep * (rr - 2.0 * p.coll_R) / p.coll_R;
            const double ex = exp(ts);
            const double Fm = Famp * ex / (1.0 - ex);
            for (int a = 0; a < p.dim; ++a) F[a] = F[a] + Fm * (r[a] / rr);
          }
        } else if (r2 <= p.r0_magnet_sq) {
          const double rr = p.dim == 3 ? sqrt(r2) / p.coll_R : sqrt(r2);
          const double e[3] = {r[0] / rr, r[1] / rr, p.dim == 3 ? r[2] / rr : 0.0};
          const double me = p.dim == 3 ? m[0] * e[0] + m[1] * e[1] + m[2] * e[2]
                                       : m[0] * e[0] + m[1] * e[1];
          const double me2 = me * me;
          const double F0r4 = p.F0_magnet / (r2 * r2);
          for (int a = 0; a < p.dim; ++a)
            F[a] = F[a] + F0r4 * (2.0 * me * m[a] - (5.0 * me2 - 1.0) * e[a]);
        }
      }
    }
  }
  double* csw = d.cs;
  csw[CS_FX * nc + c] = F[0];
  csw[CS_FY * nc + c] = F[1];
  if (p.dim == 3) csw[CS_FZ * nc + c] = F[2];
}

// Magnetic moment of every box at the context time (main.cu:395-400):
// m = (cos w t, sin w t, 0), t = t0 + dt * step.  mode 0: next step (step + 1) and count
// it; mode 1: current step.
__global__ void k_advance_time(Dev d, int nboxes, int mode) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (step_aborted(d)) return;
  const long long step = *d.step + (mode == 0 ? 1 : 0);
  if (b < nboxes) {
    const BoxParams& p = d.box[b];
    const double ang = p.omega_magnet * (p.t0 + p.dt * (double)step);
    d.mag[3 * b + 0] = cos(ang);
    d.mag[3 * b + 1] = sin(ang);
    d.mag[3 * b + 2] = 0.0;
  }
}

__global__ void k_count_step(Dev d) {
  if (step_aborted(d)) return;
  if (threadIdx.x == 0 && blockIdx.x == 0) *d.step += 1;
}

// Kinetic energy per box (kernel_calculate_macro_vars.cu:14-40).  Slots are cut into
// chunks that never straddle two boxes; each block sums one chunk in a fixed tree order
// and one thread per box adds its chunks in order, so the sum is reproducible.
__global__ void __launch_bounds__(kRedThreads) k_ke_partial(Dev d, double* partial) {
  __shared__ double sh[1][kRedThreads];
  const int c = blockIdx.x;
  const int lo = d.ke_chunk[c], hi = d.ke_chunk[c + 1];
  double v[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += kRedThreads) {
    const double4 x = d.pos[i];
    const double4 u = d.vel[i];
    const BoxParams& p = d.box[box_of(d.tinfo[i])];
    const double v2 = p.dim == 3 ? u.x * u.x + u.y * u.y + u.z * u.z : u.x * u.x + u.y * u.y;
    v[0] += 0.5 * x.w * v2;
  }
  block_reduce<1>(v, sh);
  if (threadIdx.x == 0) partial[c] = v[0];
}

__global__ void k_ke_final(Dev d, const double* partial) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nboxes) return;
  double ke = 0.0;
  for (int c = d.ke_box_chunk[b]; c < d.ke_box_chunk[b + 1]; ++c) ke += partial[c];
  d.ke[b] = ke;
}

// ---------------------------------------------------------------------------------
// Observables (no reference counterpart), one sample per box added to running sums:
//  [0] wall shear stress  -fx(top wall) / (Lx Lz), Lz = 1 in 2D (0 without walls);
//  [1] first normal-stress difference  N1 = <nkT (cxx - cyy)> over the fluid;
//  [2] chain order  <P2(e . m)> over colloid pairs closer than 2.5 R, e the unit bond and
//      m the current field direction; P2(c) = 2c^2 - 1 in 2D (cos 2 phi), (3c^2 - 1)/2 in
//      3D; 0 when no pair is that close;
//  [3] kinetic energy (k_ke_final must have run for this sample).
// Fixed-order reductions (slot chunks that never straddle boxes, then chunks in order),
// so the sums are bit-reproducible.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRedThreads) k_obs_partial(Dev d, double* partial) {
  __shared__ double sh[2][kRedThreads];
  const int c = blockIdx.x;
  const int lo = d.ke_chunk[c], hi = d.ke_chunk[c + 1];
  const int Np = d.Npad;
  double v[2] = {0.0, 0.0};  // sum of nkT (cxx - cyy) over fluid, fluid count
  for (int i = lo + threadIdx.x; i < hi; i += kRedThreads) {
    const int ti = d.tinfo[i];
    if (type_of(ti) != 0) continue;
    v[0] += d.box[box_of(ti)].nkT * (d.conf[i] - d.conf[2 * Np + i]);
    v[1] += 1.0;
  }
  block_reduce<2>(v, sh);
  if (threadIdx.x == 0) {
    partial[2 * c] = v[0];
    partial[2 * c + 1] = v[1];
  }
}

__global__ void k_obs_final(Dev d, const double* partial, double* acc) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nboxes) return;
  const BoxParams& p = d.box[b];
  double n1 = 0.0, nf = 0.0;
  for (int c = d.ke_box_chunk[b]; c < d.ke_box_chunk[b + 1]; ++c) {
    n1 += partial[2 * c];
    nf += partial[2 * c + 1];
  }
  n1 = nf > 0.0 ? n1 / nf : 0.0;
  double tw = 0.0;
  if (p.wall) tw = -d.wall_f[3 * (p.wall_seg0 + 1)] / (p.L[0] * (p.dim == 3 ? p.L[2] : 1.0));
  double so = 0.0;
  int npair = 0;
  const double mx = d.mag[3 * b], my = d.mag[3 * b + 1], mz = d.mag[3 * b + 2];
  const double mn = sqrt(mx * mx + my * my + mz * mz);
  const double rmax2 = (2.5 * p.coll_R) * (2.5 * p.coll_R);
  const int nc = d.ncoll, c0 = p.coll0;
  for (int a = 0; a < p.N_colloids && mn > 0.0; ++a)
    for (int e = a + 1; e < p.N_colloids; ++e) {
      double rx = d.cs[CS_X * nc + c0 + a] - d.cs[CS_X * nc + c0 + e];
      double ry = d.cs[CS_Y * nc + c0 + a] - d.cs[CS_Y * nc + c0 + e];
      double rz = p.dim == 3 ? d.cs[CS_Z * nc + c0 + a] - d.cs[CS_Z * nc + c0 + e] : 0.0;
      if (rx > p.halfL[0]) rx -= p.L[0];
      if (rx < -p.halfL[0]) rx += p.L[0];
      if (!p.wall) {
        if (ry > p.halfL[1]) ry -= p.L[1];
        if (ry < -p.halfL[1]) ry += p.L[1];
      }
      if (p.dim == 3) {
        if (rz > p.halfL[2]) rz -= p.L[2];
        if (rz < -p.halfL[2]) rz += p.L[2];
      }
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (!(r2 < rmax2) || r2 <= 0.0) continue;
      const double cs = (rx * mx + ry * my + rz * mz) / (sqrt(r2) * mn);
      so += p.dim == 3 ? 1.5 * cs * cs - 0.5 : 2.0 * cs * cs - 1.0;
      ++npair;
    }
  acc[4 * b + 0] += tw;
  acc[4 * b + 1] += n1;
  acc[4 * b + 2] += npair > 0 ? so / npair : 0.0;
  acc[4 * b + 3] += d.ke[b];
}

// Field gather / scatter between slot order and original order.
__device__ __forceinline__ double* field_ptr(const Dev& d, int f, int& comp, bool& in_pos,
                                             bool& in_vel) {
  in_pos = in_vel = false;
  comp = 0;
  const int Np = d.Npad;
  switch (f) {
    case SPH_X: case SPH_Y: case SPH_Z: in_pos = true; comp = f - SPH_X; return nullptr;
    case SPH_MASS: in_pos = true; comp = 3; return nullptr;
    case SPH_VX: case SPH_VY: case SPH_VZ: in_vel = true; comp = f - SPH_VX; return nullptr;
    case SPH_FX: case SPH_FY: case SPH_FZ: return d.f + (f - SPH_FX) * Np;
    case SPH_DENS: return d.dens;
    case SPH_PRESS: return d.press;
    default: break;
  }
  if (f >= SPH_CXX && f <= SPH_CZZ) return d.conf + (f - SPH_CXX) * Np;
  if (f >= SPH_DCDT_XX && f <= SPH_DCDT_ZZ) return d.dcdt + (f - SPH_DCDT_XX) * Np;
  if (f >= SPH_GXX && f <= SPH_GZZ && d.gradv) return d.gradv + (f - SPH_GXX) * Np;
  return nullptr;
}

__global__ void k_gather_field(Dev d, int f, double* out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.Ntot) return;
  const int s = d.inv[g];
  int comp;
  bool ip, iv;
  const double* src = field_ptr(d, f, comp, ip, iv);
  double v = 0.0;
  if (ip) {
    const double4 x = d.pos[s];
    v = comp == 0 ? x.x : comp == 1 ? x.y : comp == 2 ? x.z : x.w;
  } else if (iv) {
    const double4 u = d.vel[s];
    v = comp == 0 ? u.x : comp == 1 ? u.y : u.z;
  } else if (src) {
    v = src[s];
  }
  out[g] = v;
}

__global__ void k_scatter_field(Dev d, int f, const double* in) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.Ntot) return;
  const int s = d.inv[g];
  int comp;
  bool ip, iv;
  double* dst = field_ptr(d, f, comp, ip, iv);
  const double v = in[g];
  if (ip) {
    double4 x = d.pos[s];
    if (comp == 0) x.x = v; else if (comp == 1) x.y = v; else if (comp == 2) x.z = v; else x.w = v;
    d.pos[s] = x;
    mark_outside(d);  // until the next search has looked at the new positions
  } else if (iv) {
    double4 u = d.vel[s];
    if (comp == 0) u.x = v; else if (comp == 1) u.y = v; else u.z = v;
    d.vel[s] = u;
  } else if (dst) {
    dst[s] = v;
  }
}

__global__ void k_gather_int(Dev d, const int* src, int* out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.Ntot) return;
  out[g] = src[d.inv[g]];
}

// ---------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------
namespace {
inline cudaStream_t S(const Launch& L) { return static_cast<cudaStream_t>(L.stream); }
inline int blocks(int n, int t) { return (n + t - 1) / t; }
inline int check(const Launch& L) {
  ++*L.launches;
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return 0;
  last_launch_error() = (int)e;
  return 1;
}
constexpr int kT = 128;
}  // namespace

int launch_vv1_particles(const Launch& L) {
  if (L.d.Ntot == 0) return 0;
  k_vv1_particles<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_vv1_colloids(const Launch& L) {
  if (L.d.ncoll == 0) return 0;
  k_vv1_colloids<<<L.d.ncoll, 128, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_vv2(const Launch& L, bool particles) {
  if (particles && L.d.Ntot > 0) {
    k_vv2_particles<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d);
    if (check(L)) return 1;
  }
  if (L.d.ncoll > 0) {
    k_vv2_colloids<<<blocks(L.d.ncoll, kT), kT, 0, S(L)>>>(L.d);
    if (check(L)) return 1;
  }
  return 0;
}

int launch_hash(const Launch& L) {
  // the hash sets the flag again for every position it finds outside the box
  if (cudaMemsetAsync(L.d.err_info + kPosOutside, 0, sizeof(int), S(L)) != cudaSuccess) return 1;
  k_hash<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_reorder(const Launch& L, bool permute_forces) {
  const int nb = blocks(L.d.Ntot, kT);
  const bool mixed = L.d.pos_f != nullptr;
  if (mixed && permute_forces) k_reorder<true, true><<<nb, kT, 0, S(L)>>>(L.d);
  else if (mixed) k_reorder<true, false><<<nb, kT, 0, S(L)>>>(L.d);
  else if (permute_forces) k_reorder<false, true><<<nb, kT, 0, S(L)>>>(L.d);
  else k_reorder<false, false><<<nb, kT, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_build_lists_dim(const Launch& L, int dim) {
  if (L.d.Ctot == 0) return 0;
  const bool half = L.list_tpc == 16;
  const int nb = blocks(L.d.Ctot, kListWarps * (half ? 2 : 1));
  constexpr int nt = kListWarps * 32;
  if (dim == 3) {
    if (half) k_build_lists<3, 16><<<nb, nt, 0, S(L)>>>(L.d);
    else k_build_lists<3, 32><<<nb, nt, 0, S(L)>>>(L.d);
  } else {
    if (half) k_build_lists<2, 16><<<nb, nt, 0, S(L)>>>(L.d);
    else k_build_lists<2, 32><<<nb, nt, 0, S(L)>>>(L.d);
  }
  return check(L);
}

int launch_colloid_cells_n(const Launch& L, int nboxes, int max_coll) {
  if (L.d.ncoll == 0) return 0;
  k_colloid_cells<<<nboxes, 128, sizeof(int) * (max_coll > 0 ? max_coll : 1), S(L)>>>(L.d, nboxes);
  return check(L);
}

int launch_density_dim(const Launch& L, int dim) {
  if (L.d.Ntot == 0) return 0;
  if (L.density_block == 0) {
    // neighbour-cell tiles, one warp per cell
    const int nb = blocks(L.d.Ctot, kDensWarps);
    constexpr int nt = kDensWarps * 32;
    if (L.prec == SPH_PREC_FP64) {
      if (dim == 3) k_density_cells<double, 3><<<nb, nt, 0, S(L)>>>(L.d);
      else k_density_cells<double, 2><<<nb, nt, 0, S(L)>>>(L.d);
    } else {
      if (dim == 3) k_density_cells<float, 3><<<nb, nt, 0, S(L)>>>(L.d);
      else k_density_cells<float, 2><<<nb, nt, 0, S(L)>>>(L.d);
    }
    return check(L);
  }
  const int nt = L.density_block;
  const int nb = blocks(L.d.Ntot, nt);
  if (L.prec == SPH_PREC_FP64) {
    if (dim == 3) k_density<double, 3><<<nb, nt, 0, S(L)>>>(L.d);
    else k_density<double, 2><<<nb, nt, 0, S(L)>>>(L.d);
  } else {
    if (dim == 3) k_density<float, 3><<<nb, nt, 0, S(L)>>>(L.d);
    else k_density<float, 2><<<nb, nt, 0, S(L)>>>(L.d);
  }
  return check(L);
}

int launch_pressure(const Launch& L) {
  const int nb = blocks(L.d.Ntot, kT);
  if (L.prec == SPH_PREC_FP64)
    k_pressure<double><<<nb, kT, 0, S(L)>>>(L.d);
  else
    k_pressure<float><<<nb, kT, 0, S(L)>>>(L.d);
  return check(L);
}

template <typename T, int DIM, bool ONE>
static void pairs_launch(const Launch& L, int mode, int with_ext) {
  constexpr int nt = PairShape<T, DIM>::kWarps * 32;
  const int nb = blocks(L.d.Ntot, nt);
  if (mode == kPairGradvAll)
    k_pairs<T, DIM, kPairGradvAll, false, ONE><<<nb, nt, 0, S(L)>>>(L.d);
  else if (mode == kPairForcesOnly)
    k_pairs<T, DIM, kPairForcesOnly, false, ONE><<<nb, nt, 0, S(L)>>>(L.d);
  else if (with_ext)
    k_pairs<T, DIM, kPairFused, true, ONE><<<nb, nt, 0, S(L)>>>(L.d);
  else
    k_pairs<T, DIM, kPairFused, false, ONE><<<nb, nt, 0, S(L)>>>(L.d);
}

// One-box 3D contexts take the constant-bank form; 2D ones are mostly ensembles.
template <typename T, int DIM>
static void pairs_dispatch(const Launch& L, int mode, int with_ext) {
  if (DIM == 3 && L.d.one_box)
    pairs_launch<T, DIM, DIM == 3>(L, mode, with_ext);
  else
    pairs_launch<T, DIM, false>(L, mode, with_ext);
}

int launch_pairs_dim(const Launch& L, int dim, int mode, int with_ext) {
  if (L.d.Ntot == 0) return 0;
  if (L.prec == SPH_PREC_FP64) {
    if (dim == 3) pairs_dispatch<double, 3>(L, mode, with_ext);
    else pairs_dispatch<double, 2>(L, mode, with_ext);
  } else {
    if (dim == 3) pairs_dispatch<float, 3>(L, mode, with_ext);
    else pairs_dispatch<float, 2>(L, mode, with_ext);
  }
  return check(L);
}

int launch_ext_force(const Launch& L) {
  k_ext_force<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_dcdt_from_gradv(const Launch& L) {
  k_dcdt<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_wall_forces(const Launch& L) {
  if (L.d.nwallseg == 0) return 0;
  if (L.d.nwallchunks > 0) {
    k_wall_forces<<<L.d.nwallchunks, kRedThreads, 0, S(L)>>>(L.d);
    if (check(L)) return 1;
  }
  k_wall_forces_final<<<blocks(L.d.nwallseg, 4), 128, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_colloid_forces(const Launch& L, int with_pairs) {
  if (L.d.ncoll == 0) return 0;
  k_collect_colloids<<<L.d.ncoll, kRedThreads, 0, S(L)>>>(L.d);
  if (check(L)) return 1;
  if (with_pairs) {
    k_colloid_pairs<<<blocks(L.d.ncoll, 64), 64, 0, S(L)>>>(L.d);
    if (check(L)) return 1;
  }
  return 0;
}

int launch_advance_time(const Launch& L, int mode) {
  k_advance_time<<<blocks(L.d.nboxes, 64), 64, 0, S(L)>>>(L.d, L.d.nboxes, mode);
  return check(L);
}

int launch_count_step(const Launch& L) {
  k_count_step<<<1, 32, 0, S(L)>>>(L.d);
  return check(L);
}

int launch_kinetic_energy(const Launch& L, double* partial) {
  k_ke_partial<<<L.d.nkechunks, kRedThreads, 0, S(L)>>>(L.d, partial);
  if (check(L)) return 1;
  k_ke_final<<<blocks(L.d.nboxes, 64), 64, 0, S(L)>>>(L.d, partial);
  return check(L);
}

int launch_observe(const Launch& L, double* ke_partial, double* obs_partial, double* acc) {
  if (launch_kinetic_energy(L, ke_partial)) return 1;
  k_obs_partial<<<L.d.nkechunks, kRedThreads, 0, S(L)>>>(L.d, obs_partial);
  if (check(L)) return 1;
  k_obs_final<<<blocks(L.d.nboxes, 64), 64, 0, S(L)>>>(L.d, obs_partial, acc);
  return check(L);
}

int launch_gather_field(const Launch& L, int field, double* out) {
  k_gather_field<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d, field, out);
  return check(L);
}

int launch_scatter_field(const Launch& L, int field, const double* in) {
  k_scatter_field<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d, field, in);
  return check(L);
}

int launch_gather_int(const Launch& L, const int* src, int* out) {
  k_gather_int<<<blocks(L.d.Ntot, kT), kT, 0, S(L)>>>(L.d, src, out);
  return check(L);
}

}  // namespace sph
