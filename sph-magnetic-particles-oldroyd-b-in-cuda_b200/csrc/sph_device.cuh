// sph_device.cuh -- device helpers shared by the per-particle and the per-cell kernels:
// the SPH kernel, minimum image, cell checks, neighbour records, Morris ghost velocities
// and the pair arithmetic of the velocity-gradient / force pass.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include <type_traits>

#include "sph_internal.h"

namespace sph {
#define SPH_FULL 0xffffffffu

__device__ __forceinline__ int type_of(int t) { return t & kTypeMask; }
__device__ __forceinline__ int box_of(int t) { return t >> kTypeBits; }

template <typename T> struct V4;
template <> struct V4<double> { using type = double4; };
template <> struct V4<float> { using type = float4; };

template <typename T, int DIM> struct RecFor;
template <> struct RecFor<double, 3> { using type = RecD; };
template <> struct RecFor<float, 3> { using type = RecF; };
template <> struct RecFor<double, 2> { using type = RecD2; };
template <> struct RecFor<float, 2> { using type = RecF2; };

// Fields a 2D record does not carry read as zero.
template <int DIM, typename R>
__device__ __forceinline__ auto rec_z(const R& r) -> decltype(r.x) {
  if constexpr (DIM == 3) return r.z; else return decltype(r.x)(0);
}
template <int DIM, typename R>
__device__ __forceinline__ auto rec_vz(const R& r) -> decltype(r.x) {
  if constexpr (DIM == 3) return r.vz; else return decltype(r.x)(0);
}
template <int DIM, typename R>
__device__ __forceinline__ auto rec_P(const R& r, int q) -> decltype(r.x) {
  if constexpr (DIM == 3) return r.P[q]; else return q < 3 ? r.P[q] : decltype(r.x)(0);
}

// ---------------------------------------------------------------------------------
// SPH kernel and its radial derivative (kernel_W.cu:13-59, kernel_gradW.cu:13-53).
// Written branch-free: the clamped terms are exact zeros where the reference skips
// them, so the value is the same as the branchy form.
// ---------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T sph_w(T r, T rcut_inv, T cw) {
  T q3 = (r * rcut_inv) * T(3);
  T t1 = T(3) - q3, t2 = T(2) - q3, t3 = T(1) - q3;
  T a1 = t1 * t1, a2 = t2 * t2, a3 = t3 * t3;
  T w = (a1 * a1) * t1;
  if (q3 < T(2)) w = w - T(6) * ((a2 * a2) * t2);
  if (q3 < T(1)) w = w + T(15) * ((a3 * a3) * t3);
  return cw * w;
}

template <typename T>
__device__ __forceinline__ T sph_gradw(T r, T rcut_inv, T c_gradw) {
  T q3 = T(3) * (r * rcut_inv);
  T t1 = T(3) - q3, t2 = T(2) - q3, t3 = T(1) - q3;
  T a1 = t1 * t1, a2 = t2 * t2, a3 = t3 * t3;
  T g = a1 * a1;
  if (q3 < T(2)) g = g - T(6) * (a2 * a2);
  if (q3 < T(1)) g = g + T(15) * (a3 * a3);
  return c_gradw * g;
}

// Minimum image as the reference writes it: subtract L above L/2, add L below -L/2
// (kernel_densities.cu:90-110).  y is periodic only without walls; z only in 3D.
// WRAP false: the separation is taken as it is (for particles clear of the periodic faces,
// see clear_of_faces, where the shifts change no pair inside the cutoff).
template <typename T, int DIM, bool WRAP = true>
__device__ __forceinline__ void min_image(T& rx, T& ry, T& rz, const T L[3], const T h[3],
                                          int wall) {
  if constexpr (!WRAP) return;
  if (rx > h[0]) rx -= L[0];
  if (rx < -h[0]) rx += L[0];
  if (!wall) {
    if (ry > h[1]) ry -= L[1];
    if (ry < -h[1]) ry += L[1];
  }
  if (DIM == 3) {
    if (rz > h[2]) rz -= L[2];
    if (rz < -h[2]) rz += L[2];
  }
}

// |r|^2 with explicit roundings, rx^2 then + ry^2 then + rz^2 by fused multiply-adds: the
// compiler may contract a plain expression differently in each pass that inlines it, and
// the passes with and without the minimum image (and the density's two forms) must agree
// bit for bit.
__device__ __forceinline__ double norm2(double rx, double ry, double rz, bool three) {
  const double s = __fma_rn(ry, ry, __dmul_rn(rx, rx));
  return three ? __fma_rn(rz, rz, s) : s;
}
__device__ __forceinline__ float norm2(float rx, float ry, float rz, bool three) {
  const float s = __fmaf_rn(ry, ry, __fmul_rn(rx, rx));
  return three ? __fmaf_rn(rz, rz, s) : s;
}

// Cell of a position as kernel_cell_list.cu:15-63 computes it (with its clamp rules).
// Returns the box-local linear cell, or -1 when the reference would assert
// (kernel_cell_ranges.cu:20-23) or the position is not finite.
__device__ __forceinline__ int hash_cell(const BoxParams& p, double x, double y, double z) {
  if (!isfinite(x) || !isfinite(y) || (p.dim == 3 && !isfinite(z))) return -2;
  const double fx = floor(x / p.cell_size[0]);
  const double fy = p.wall == 0 ? floor(y / p.cell_size[1])
                                : floor((y + p.wall_width) / p.cell_size[1]);
  const double fz = p.dim == 3 ? floor(z / p.cell_size[2]) : 0.0;
  // far outside the grid: the linear index below would overflow int
  const double big = 1 << 20;
  if (fabs(fx) > big || fabs(fy) > big || fabs(fz) > big) return -1;
  int cx = (int)fx;
  if (cx == p.Ncells[0]) cx = cx - 1;
  int cy = (int)fy;
  if (p.wall == 0 && cy == p.Ncells[1]) cy = cy - 1;
  long long c;
  if (p.dim == 3) {
    int cz = (int)fz;
    if (cz == p.Ncells[2]) cz = cz - 1;
    c = (long long)cz * p.Ncells[0] * p.Ncells[1] + (long long)cy * p.Ncells[0] + cx;
  } else {
    c = (long long)cy * p.Ncells[0] + cx;
  }
  if (c < 0 || c > p.Ntotal_cells - 1) return -1;
  return (int)c;
}

// The cell the pair kernels of the reference iterate around: unclamped floor
// (kernel_densities.cu:52-60).  Returns false, leaving the outputs untouched, when the
// position is not finite or so far outside the box that one periodic wrap of the
// neighbour cells cannot bring them back into the grid; every cell index derived from a
// true result is in range.
__device__ __forceinline__ bool own_cell(const BoxParams& p, double x, double y, double z,
                                         int& cx, int& cy, int& cz) {
  const double fx = floor(x / p.cell_size[0]);
  const double fy = p.wall == 0 ? floor(y / p.cell_size[1])
                                : floor((y + p.wall_width) / p.cell_size[1]);
  const double fz = p.dim == 3 ? floor(z / p.cell_size[2]) : 0.0;
  // comparisons with NaN are false, so NaN fails every range test
  if (!(fx >= 1.0 - p.Ncells[0] && fx <= 2.0 * p.Ncells[0] - 2.0)) return false;
  if (p.wall == 0) {
    if (!(fy >= 1.0 - p.Ncells[1] && fy <= 2.0 * p.Ncells[1] - 2.0)) return false;
  } else if (!(fy >= -2.0 * p.Ncells[1] && fy <= 3.0 * p.Ncells[1])) {
    return false;  // wall axis: out-of-grid rows are skipped, only int overflow matters
  }
  if (p.dim == 3 && !(fz >= 1.0 - p.Ncells[2] && fz <= 2.0 * p.Ncells[2] - 2.0)) return false;
  cx = (int)fx;
  cy = (int)fy;
  cz = (int)fz;
  return true;
}

// Reports a failure.  The first report of any kind also records the step counter and the
// phase; the first report of a bad position records the particle's global id.
__device__ __forceinline__ void raise_status(const Dev& d, unsigned bit, int info, int phase) {
  const unsigned old = atomicOr(d.status, bit);
  if (!(old & bit) && bit != kStatCapacity) atomicExch(&d.err_info[kErrBadId], info);
  if (!(old & kStatAbortMask)) {
    const long long s = *d.step;
    d.err_info[kErrStepLo] = (int)(s & 0xffffffffLL);
    d.err_info[kErrStepHi] = (int)(s >> 32);
    d.err_info[kErrPhase] = phase;
  }
}

// One particle's neighbour candidates in list order, decoded from the chunk entries the list
// build writes: nchunk[k * Npad + i] = (first slot, hit mask) of the particle's k-th chunk
// with hits (nbr_nch[i] of them), bit 31 - q of the mask meaning slot first + q (the first
// candidate in the highest bit, so that a count of leading zeros gives its offset).  Candidates come
// chunk by chunk and, inside a chunk, by increasing slot: the reference's candidate order.
// Every stored chunk has a hit, so moving to the next one never loops; its entry is loaded
// one chunk ahead.  next() gives nbr_cnt[i] candidates, then -1.  It has no branch: the
// lanes of a warp move to their next chunks at different positions, and a branch taken by
// any lane would cost every lane the move (branch-free: 128^3 pair pass 4.03 -> 3.82 ms).
struct NbrIter {
  const int2* col;  // this particle's entries, stride np
  int np, nch, c;   // c: the current chunk
  unsigned mk;      // its bits not yet taken
  int base;
  int2 nxt;         // entry of chunk c + 1
  __device__ __forceinline__ void init(const Dev& d, int i) {
    np = d.Npad;
    col = d.nchunk + i;
    nch = d.nbr_nch[i];
    c = 0;
    const int2 e0 = nch > 0 ? __ldg(col) : make_int2(0, 0);
    base = e0.x;
    mk = (unsigned)e0.y;
    nxt = nch > 1 ? __ldg(col + (size_t)np) : make_int2(0, 0);
  }
  __device__ __forceinline__ int next() {
    // branch-free: every lane selects; only the prefetch load is predicated
    const bool r = mk == 0u;
    base = r ? nxt.x : base;
    mk = r ? (unsigned)nxt.y : mk;
    c += r ? 1 : 0;
    const bool ld = r && c + 1 < nch;
    const int2* pn = col + (size_t)(c + 1) * np;
    if (ld) nxt = __ldg(pn);
    const int q = __clz(mk);  // 32 only past the last candidate, where the shift gives 0
    mk ^= q < 32 ? 0x80000000u >> q : 0u;
    return c < nch ? base + q : -1;
  }
};

// True once a kernel before this one reported a failure: the step's state-changing kernels
// then return at entry.  The flag word is read past L1 (it is written by atomics in L2).  In
// kernels whose warps cooperate, lane 0's reading is taken by the whole warp.
__device__ __forceinline__ bool step_aborted(const Dev& d) {
  return (*(volatile const unsigned*)d.status & kStatAbortMask) != 0u;
}
__device__ __forceinline__ bool step_aborted_warp(const Dev& d) {
  unsigned v = 0u;
  if ((threadIdx.x & 31) == 0) v = *(volatile const unsigned*)d.status;
  return (__shfl_sync(0xffffffffu, v, 0) & kStatAbortMask) != 0u;
}

// A position outside [0, L] along a periodic axis of its box (or not finite).
__device__ __forceinline__ bool outside_periodic(const BoxParams& p, double x, double y,
                                                 double z) {
  return !(x >= 0.0 && x <= p.L[0]) || (p.wall == 0 && !(y >= 0.0 && y <= p.L[1])) ||
         (p.dim == 3 && !(z >= 0.0 && z <= p.L[2]));
}
__device__ __forceinline__ void mark_outside(const Dev& d) { d.err_info[kPosOutside] = 1; }

// A particle at least 1.0625 rcut from every periodic face of its box.  While every position
// lies in [0, L] along the periodic axes (err_info[kPosOutside] clear), the minimum image
// changes no pair of such a particle that the sums take: a neighbour within the cutoff is
// never across a face, and a pair whose plain separation along an axis exceeds L/2 fails the
// cutoff both unshifted (L/2 > rcut) and shifted (then at least the margin, more than rcut,
// since the particle is that far from the face).  The pair passes take the separations of
// warps of such particles without the shifts: the same bits, fewer dependent operations.
template <typename T, int DIM>
__device__ __forceinline__ bool clear_of_faces(const BoxParams& p, T x, T y, T z) {
  const T m = (T)(1.0625 * p.rcut);
  bool in = x >= m && x <= (T)p.L[0] - m;
  if (DIM == 3) in = in && z >= m && z <= (T)p.L[2] - m;
  if (!p.wall) in = in && y >= m && y <= (T)p.L[1] - m;
  return in;
}
// Whether a whole warp may drop the minimum image (every lane passes `clear`); lane 0's
// reading of the flag is taken by the whole warp.
__device__ __forceinline__ bool warp_plain_image(const Dev& d, bool clear) {
  int v = 0;
  if ((threadIdx.x & 31) == 0) v = *(volatile const int*)(d.err_info + kPosOutside);
  v = __shfl_sync(0xffffffffu, v, 0);
  return __all_sync(0xffffffffu, clear) && v == 0;
}


template <typename T, int DIM>
__device__ __forceinline__ void write_record(const Dev& d, int i, const BoxParams& p, int ti,
                                             double dens, double press) {
  using Rec = typename RecFor<T, DIM>::type;
  constexpr int kP = DIM == 3 ? 6 : 3;  // stress components carried
  Rec* rec = reinterpret_cast<Rec*>(d.rec);
  const int Np = d.Npad;
  const double4 x = d.pos[i];
  const double4 v = d.vel[i];
  Rec r;
  r.x = x.x; r.y = x.y;
  r.vx = v.x; r.vy = v.y;
  if constexpr (DIM == 3) {
    r.z = x.z;
    r.vz = v.z;
    r.tinfo = ti;
  }
  const double nkT = p.nkT;
  double c[6];
#pragma unroll
  for (int q = 0; q < kP; ++q) c[q] = d.conf[q * Np + i];
  const double dinv = 1.0 / dens;
  if (type_of(ti) == 0) {
    // Pi / d^2 with Pi = p I - nkT c (kernel_forces.cu:62-88); diagonal: xx, yy, zz
    const double dsq = dinv * dinv;
#pragma unroll
    for (int q = 0; q < kP; ++q) {
      const bool diag = q == 0 || q == 2 || q == 5;
      r.P[q] = diag ? (T)((press - nkT * c[q]) * dsq) : (T)((-nkT * c[q]) * dsq);
    }
  } else {
    // walls / colloid particles: -nkT c, completed with the fluid partner's p and d
#pragma unroll
    for (int q = 0; q < kP; ++q) r.P[q] = (T)(-nkT * c[q]);
  }
  r.invd = (T)dinv;
  rec[i] = r;
}


struct CollView {
  const double* cs;
  int nc;
};

// Morris ghost velocity, fluid particle i next to wall / colloid particle j
// (kernel_forces.cu:234-318, 590-692; kernel_vel_gradients.cu:162-247, 421-525).
template <typename T, int DIM>
__device__ __forceinline__ void ghost_fluid_i(const BoxParams& p, const CollView& cv,
                                              int tj, int coll0, T xi, T yi, T zi, T yj,
                                              const T vi[3], const T r[3], const T L[3],
                                              const T h[3], T v[3]) {
  const T beta_max = (T)p.beta_max;
  if (tj == 1 || tj == 2) {
    T di, dj, Vw;
    if (tj == 1) {
      di = yi - (T)p.y_bottom;
      dj = (T)p.y_bottom - yj;
      Vw = (T)p.V_bottom;
    } else {
      di = (T)p.y_top - yi;
      dj = yj - (T)p.y_top;
      Vw = (T)p.V_top;
    }
    T beta = T(1) + dj / di;
    if (beta > beta_max) beta = beta_max;
    if (di > T(0)) {
      v[0] = beta * (vi[0] - Vw);
      v[1] = beta * vi[1];
      v[2] = beta * vi[2];
    } else {
      v[0] = vi[0] - Vw;
      v[1] = vi[1];
      v[2] = vi[2];
    }
    return;
  }
  const int c = coll0 + tj - 3, nc = cv.nc;
  T rc[3] = {xi - (T)cv.cs[CS_X * nc + c], yi - (T)cv.cs[CS_Y * nc + c],
             DIM == 3 ? zi - (T)cv.cs[CS_Z * nc + c] : T(0)};
  min_image<T, DIM>(rc[0], rc[1], rc[2], L, h, p.wall);
  const T dc = DIM == 3 ? sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2])
                        : sqrt(rc[0] * rc[0] + rc[1] * rc[1]);
  const T R = (T)p.coll_R;
  const T dis = dc - R;
  const T cvel[3] = {(T)cv.cs[CS_VX * nc + c], (T)cv.cs[CS_VY * nc + c],
                     DIM == 3 ? (T)cv.cs[CS_VZ * nc + c] : T(0)};
  if (dis < T(0)) {
    v[0] = vi[0] - cvel[0];
    v[1] = vi[1] - cvel[1];
    v[2] = vi[2] - cvel[2];
    return;
  }
  const T xs = rc[0] / dc * R, ys = rc[1] / dc * R, zs = DIM == 3 ? rc[2] / dc * R : T(0);
  T vr[3];
  const T wz = (T)cv.cs[CS_OZ * nc + c];
  if (DIM == 2) {
    vr[0] = -wz * ys;
    vr[1] = wz * xs;
    vr[2] = T(0);
  } else {
    const T wx = (T)cv.cs[CS_OX * nc + c], wy = (T)cv.cs[CS_OY * nc + c];
    vr[0] = wy * zs - wz * ys;
    vr[1] = wz * xs - wx * zs;
    vr[2] = wx * ys - wy * xs;
  }
  const T sv0 = rc[0] / dc, sv1 = rc[1] / dc, sv2 = DIM == 3 ? rc[2] / dc : T(0);
  const T djs = DIM == 3 ? (r[0] * sv0 + r[1] * sv1 + r[2] * sv2) - dis
                         : (r[0] * sv0 + r[1] * sv1) - dis;
  T beta = T(1) + djs / dis;
  if (beta > beta_max) beta = beta_max;
  v[0] = beta * (vi[0] - cvel[0] - vr[0]);
  v[1] = beta * (vi[1] - cvel[1] - vr[1]);
  v[2] = beta * (vi[2] - cvel[2] - vr[2]);
}

// Morris ghost velocity, wall / colloid particle i next to particle j
// (kernel_forces.cu:337-418, 721-821; kernel_vel_gradients.cu:249-331, 527-630).
template <typename T, int DIM>
__device__ __forceinline__ void ghost_solid_i(const BoxParams& p, const CollView& cv,
                                              int ti, int coll0, T yi, T xj, T yj, T zj,
                                              const T vj[3], const T r[3], const T L[3],
                                              const T h[3], T v[3]) {
  const T beta_max = (T)p.beta_max;
  if (ti == 1 || ti == 2) {
    T di, dj, Vw;
    if (ti == 1) {
      di = (T)p.y_bottom - yi;
      dj = yj - (T)p.y_bottom;
      Vw = (T)p.V_bottom;
    } else {
      di = yi - (T)p.y_top;
      dj = (T)p.y_top - yj;
      Vw = (T)p.V_top;
    }
    T beta = T(1) + di / dj;
    if (beta > beta_max) beta = beta_max;
    if (dj > T(0)) {
      v[0] = beta * (Vw - vj[0]);
      v[1] = -beta * vj[1];
      v[2] = -beta * vj[2];
    } else {
      v[0] = Vw - vj[0];
      v[1] = -vj[1];
      v[2] = -vj[2];
    }
    return;
  }
  const int c = coll0 + ti - 3, nc = cv.nc;
  T rc[3] = {xj - (T)cv.cs[CS_X * nc + c], yj - (T)cv.cs[CS_Y * nc + c],
             DIM == 3 ? zj - (T)cv.cs[CS_Z * nc + c] : T(0)};
  min_image<T, DIM>(rc[0], rc[1], rc[2], L, h, p.wall);
  const T dc = DIM == 3 ? sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2])
                        : sqrt(rc[0] * rc[0] + rc[1] * rc[1]);
  const T R = (T)p.coll_R;
  const T djs = dc - R;
  const T cvel[3] = {(T)cv.cs[CS_VX * nc + c], (T)cv.cs[CS_VY * nc + c],
                     DIM == 3 ? (T)cv.cs[CS_VZ * nc + c] : T(0)};
  if (djs < T(0)) {
    v[0] = cvel[0] - vj[0];
    v[1] = cvel[1] - vj[1];
    v[2] = cvel[2] - vj[2];
    return;
  }
  const T xs = rc[0] / dc * R, ys = rc[1] / dc * R, zs = DIM == 3 ? rc[2] / dc * R : T(0);
  T vr[3];
  const T wz = (T)cv.cs[CS_OZ * nc + c];
  if (DIM == 2) {
    vr[0] = -wz * ys;
    vr[1] = wz * xs;
    vr[2] = T(0);
  } else {
    const T wx = (T)cv.cs[CS_OX * nc + c], wy = (T)cv.cs[CS_OY * nc + c];
    vr[0] = wy * zs - wz * ys;
    vr[1] = wz * xs - wx * zs;
    vr[2] = wx * ys - wy * xs;
  }
  const T sv0 = rc[0] / dc, sv1 = rc[1] / dc, sv2 = DIM == 3 ? rc[2] / dc : T(0);
  const T dis = DIM == 3 ? (-r[0] * sv0 - r[1] * sv1 - r[2] * sv2) - djs
                         : (-r[0] * sv0 - r[1] * sv1) - djs;
  T beta = T(1) + dis / djs;
  if (beta > beta_max) beta = beta_max;
  v[0] = beta * (cvel[0] + vr[0] - vj[0]);
  v[1] = beta * (cvel[1] + vr[1] - vj[1]);
  v[2] = beta * (cvel[2] + vr[2] - vj[2]);
}


// ---------------------------------------------------------------------------------
// Pair pass arithmetic: velocity gradient (kernel_vel_gradients.cu:15-662), forces
// (kernel_forces.cu:15-865), external force (kernel_ext_force.cu:13-73), dc/dt
// (kernel_dcdt.cu:15-104).  One function for one (i, j) pair, used by every pair kernel.
// ---------------------------------------------------------------------------------
// Read-only position loads.  In 3D a double4 is read as one 256-bit access (the vector
// width of sm_100 global loads): one L1 request per lane instead of two 128-bit ones.  In
// 2D only x and y are read (one 128-bit access; z and the mass come back zero).  Position
// arrays are 32-byte aligned (cudaMalloc base, 32-byte elements).
template <int DIM>
__device__ __forceinline__ double4 ld_pos(const double4* a) {
  double4 v;
  if (DIM == 3) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
        : "l"(a));
  } else {
    const double2 xy = __ldg(reinterpret_cast<const double2*>(a));
    v = make_double4(xy.x, xy.y, 0.0, 0.0);
  }
  return v;
}
template <int DIM>
__device__ __forceinline__ float4 ld_pos(const float4* a) {
  return __ldg(a);
}

template <typename T, int DIM>
struct PairParams {
  T L[3], h[3], rcutsq, rcut_inv, c_gradw, a, b;
  __device__ __forceinline__ void load(const BoxParams& p) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      L[q] = (T)p.L[q];
      h[q] = (T)p.halfL[q];
    }
    rcutsq = (T)p.rcutsq;
    rcut_inv = (T)p.rcut_inv;
    c_gradw = (T)p.c_gradw;
    a = (T)p.a;
    b = (T)p.b;
  }
};

// the target particle i of the pass
template <typename T, int DIM>
struct PairOwn {
  T x, y, z, v[3], invd, press, P[6];
  int t;
  bool fluid, do_grad, do_force;
};

// Sums of the float pair terms in mixed precision (density, velocity gradient, forces):
// kind 1 compensated float sums (Kahan), kind 2 FP64 accumulators of the float terms (kept:
// more accurate, and at 128^3 the pair pass 2.41 -> 2.39 ms and the density 0.74 -> 0.73 ms,
// the conversions and FP64 adds running on the otherwise idle FP64 pipe).  FP64 sums stay
// plain.  S: the accumulator type.
constexpr int kFloatSums = 2;
template <typename T>
struct SumKind {
  static constexpr int kind = 0;
  using S = T;
};
template <>
struct SumKind<float> {
  static constexpr int kind = kFloatSums;
  using S = std::conditional_t<kFloatSums == 2, double, float>;
};
template <typename T>
struct Compensated {
  static constexpr bool on = SumKind<T>::kind == 1;
};

// Kahan step: s + c tracks the exact sum of the terms to about one rounding of s.
__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  const float y = __fsub_rn(x, c);
  const float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

template <typename T, int DIM>
struct PairAcc {
  // the sums of float pair terms (mixed precision) are FP64 accumulators, or, in the
  // compensated form (SumKind kind 1), floats each carrying its rounding error in a second
  // float (Kahan) that is added back when the sum is stored
  using S = typename SumKind<T>::S;
  static constexpr bool kComp = Compensated<T>::on;
  static constexpr bool kTermwise = SumKind<T>::kind != 0;  // a pair's force as one term
  S g[DIM][DIM];
  S f[3];
  T cg[DIM][DIM];
  T cf[3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        g[a][c] = S(0);
        cg[a][c] = T(0);
      }
    f[0] = f[1] = f[2] = S(0);
    cf[0] = cf[1] = cf[2] = T(0);
  }
  // s (with compensation c) += x
  __device__ __forceinline__ static void add(S& s, T& c, T x) {
    if constexpr (kComp)
      kahan_add(s, c, x);
    else
      s += (S)x;
  }
  __device__ __forceinline__ double grad(int a, int c) const {
    return kComp ? (double)g[a][c] - (double)cg[a][c] : (double)g[a][c];
  }
  __device__ __forceinline__ double force(int a) const {
    return kComp ? (double)f[a] - (double)cf[a] : (double)f[a];
  }
};

// ti: the particle's type word (from the type array)
template <typename T, int DIM, int MODE, typename Rec>
__device__ __forceinline__ void load_own(const Dev& d, int i, int ti, const Rec& ri,
                                         PairOwn<T, DIM>& o) {
  o.x = (T)ri.x;
  o.y = (T)ri.y;
  o.z = (T)rec_z<DIM>(ri);
  o.v[0] = (T)ri.vx;
  o.v[1] = (T)ri.vy;
  o.v[2] = (T)rec_vz<DIM>(ri);
  o.invd = ri.invd;
  o.press = (T)d.press[i];
#pragma unroll
  for (int q = 0; q < 6; ++q) o.P[q] = rec_P<DIM>(ri, q);
  o.t = type_of(ti);
  o.fluid = o.t == 0;
  // gradient: every particle in kPairGradvAll; in the fused pass fluid particles (whose
  // dc/dt needs it), or every particle when the caller stores the whole field
  o.do_grad = (MODE == kPairGradvAll) || (MODE == kPairFused && (o.fluid || d.grad_all));
  o.do_force = MODE != kPairGradvAll;
}

// Separation r = x_i - x_j under the minimum image; returns |r|^2.
template <typename T, int DIM, bool WRAP, typename Rec>
__device__ __forceinline__ T pair_sep(const PairParams<T, DIM>& pp, int wall,
                                      const PairOwn<T, DIM>& o, const Rec& rj, T r[3]) {
  r[0] = o.x - (T)rj.x;
  r[1] = o.y - (T)rj.y;
  r[2] = DIM == 3 ? o.z - (T)rec_z<DIM>(rj) : T(0);
  min_image<T, DIM, WRAP>(r[0], r[1], r[2], pp.L, pp.h, wall);
  return norm2(r[0], r[1], r[2], DIM == 3);
}

// 1/|r|, the kernel slope gw = dW/dr at |r| and the unit vector e = r / |r|.
template <typename T, int DIM>
struct PairRadial {
  T rinv, gw, e[3];
  __device__ __forceinline__ void eval(const PairParams<T, DIM>& pp, T r2, const T r[3]) {
    rinv = rsqrt(r2);  // r and 1/r from one reciprocal square root
    const T rr = r2 * rinv;
    gw = sph_gradw<T>(rr, pp.rcut_inv, pp.c_gradw);
    e[0] = r[0] * rinv;
    e[1] = r[1] * rinv;
    e[2] = DIM == 3 ? r[2] * rinv : T(0);
  }
};

// Velocity-gradient term, g_ac += -(1/d_i) gw e_a v_c (kernel_vel_gradients.cu:334-337,
// 632-640).
template <typename T, int DIM>
__device__ __forceinline__ void pair_grad_add(const PairOwn<T, DIM>& o, const PairRadial<T, DIM>& g,
                                              const T v[3], PairAcc<T, DIM>& acc) {
  const T s = -o.invd * g.gw;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const T se = s * g.e[a];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      if constexpr (PairAcc<T, DIM>::kTermwise)
        PairAcc<T, DIM>::add(acc.g[a][c], acc.cg[a][c], se * v[c]);
      else
        acc.g[a][c] += se * v[c];
    }
  }
}

// Force term from the partners' stress terms Pi, Pj (P/d^2 - nkT c/d^2) and inverse
// densities di, dj: the reversible part -gw (Pi + Pj).e and the viscous part
// a gw/(di dj r) v + b gw/(di dj r) (e.v) e (kernel_forces.cu:426-440, 826-850).
template <typename T, int DIM>
__device__ __forceinline__ void pair_force_add(const PairParams<T, DIM>& pp,
                                               const PairRadial<T, DIM>& g, const T v[3],
                                               const T Pi[6], const T Pj[6], T di, T dj,
                                               PairAcc<T, DIM>& acc) {
  const T gw = g.gw;
  const T* e = g.e;
  const T aux = gw * di * dj * g.rinv;
  const T aux1 = pp.a * aux;
  if constexpr (PairAcc<T, DIM>::kTermwise) {
    // the pair's force as one term per component, then one compensated (or FP64) add
    const T axx = -gw * (Pi[0] + Pj[0]);
    const T axy = -gw * (Pi[1] + Pj[1]);
    const T ayy = -gw * (Pi[2] + Pj[2]);
    T ev = e[0] * v[0] + e[1] * v[1];
    T t0 = axx * e[0] + axy * e[1], t1 = axy * e[0] + ayy * e[1], t2 = T(0);
    if (DIM == 3) {
      const T axz = -gw * (Pi[3] + Pj[3]);
      const T ayz = -gw * (Pi[4] + Pj[4]);
      const T azz = -gw * (Pi[5] + Pj[5]);
      ev += e[2] * v[2];
      t0 += axz * e[2];
      t1 += ayz * e[2];
      t2 = axz * e[0] + ayz * e[1] + azz * e[2];
    }
    const T aux2 = pp.b * aux * ev;
    PairAcc<T, DIM>::add(acc.f[0], acc.cf[0], t0 + (aux1 * v[0] + aux2 * e[0]));
    PairAcc<T, DIM>::add(acc.f[1], acc.cf[1], t1 + (aux1 * v[1] + aux2 * e[1]));
    if (DIM == 3) PairAcc<T, DIM>::add(acc.f[2], acc.cf[2], t2 + (aux1 * v[2] + aux2 * e[2]));
  } else {
    // -gw (Pi + Pj).e and the viscous terms folded into the sums by fused multiply-adds
    const T ngw = -gw;
    T ev = e[0] * v[0] + e[1] * v[1];
    T t0 = (Pi[0] + Pj[0]) * e[0] + (Pi[1] + Pj[1]) * e[1];
    T t1 = (Pi[1] + Pj[1]) * e[0] + (Pi[2] + Pj[2]) * e[1];
    T t2 = T(0);
    if (DIM == 3) {
      const T sxz = Pi[3] + Pj[3], syz = Pi[4] + Pj[4];
      ev += e[2] * v[2];
      t0 += sxz * e[2];
      t1 += syz * e[2];
      t2 = sxz * e[0] + syz * e[1] + (Pi[5] + Pj[5]) * e[2];
    }
    const T aux2 = pp.b * aux * ev;
    acc.f[0] = fma(aux2, e[0], fma(aux1, v[0], fma(ngw, t0, acc.f[0])));
    acc.f[1] = fma(aux2, e[1], fma(aux1, v[1], fma(ngw, t1, acc.f[1])));
    if (DIM == 3) acc.f[2] = fma(aux2, e[2], fma(aux1, v[2], fma(ngw, t2, acc.f[2])));
  }
}

// One (i, j) pair.  tj: the neighbour's particle type.  WRAP: see min_image.
template <typename T, int DIM, bool WRAP, typename Rec>
__device__ __forceinline__ void pair_term(const BoxParams& p, const PairParams<T, DIM>& pp,
                                          const CollView& cv, const PairOwn<T, DIM>& o,
                                          const Rec& rj, int tj, PairAcc<T, DIM>& acc) {
  const bool fluid_j = tj == 0;
  // skip rules: gradient kernel_vel_gradients.cu:126-127, forces kernel_forces.cu:157-158
  const bool pair_grad = o.do_grad && !(o.t == tj && !o.fluid);
  const bool pair_force = o.do_force && (o.fluid || fluid_j);
  if (!pair_grad && !pair_force) return;
  T r[3];
  const T r2 = pair_sep<T, DIM, WRAP>(pp, p.wall, o, rj, r);
  if (!(r2 < pp.rcutsq)) return;
  const T vj[3] = {(T)rj.vx, (T)rj.vy, (T)rec_vz<DIM>(rj)};
  T v[3];
  if (o.t == tj) {
    v[0] = o.v[0] - vj[0];
    v[1] = o.v[1] - vj[1];
    v[2] = o.v[2] - vj[2];
  } else if (o.fluid) {
    ghost_fluid_i<T, DIM>(p, cv, tj, p.coll0, o.x, o.y, o.z, (T)rj.y, o.v, r, pp.L, pp.h, v);
  } else {
    ghost_solid_i<T, DIM>(p, cv, o.t, p.coll0, o.y, (T)rj.x, (T)rj.y, (T)rec_z<DIM>(rj), vj, r, pp.L,
                          pp.h, v);
  }
  PairRadial<T, DIM> g;
  g.eval(pp, r2, r);
  if (pair_grad) pair_grad_add<T, DIM>(o, g, v, acc);
  if (pair_force) {
    T Pi[6], Pj[6], di, dj;
    if (o.fluid && fluid_j) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        Pi[q] = o.P[q];
        Pj[q] = rec_P<DIM>(rj, q);
      }
      di = o.invd;
      dj = rj.invd;
    } else if (o.fluid) {
      // j mirrors i's density and pressure, keeps its own c (kernel_forces.cu:217-233)
      const T dsq = o.invd * o.invd;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        Pi[q] = o.P[q];
        const T diag = (q == 0 || q == 2 || q == 5) ? o.press : T(0);
        Pj[q] = (diag + rec_P<DIM>(rj, q)) * dsq;
      }
      di = o.invd;
      dj = o.invd;
    } else {
      // i takes j's density, pressure and c (kernel_forces.cu:320-336)
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        Pj[q] = rec_P<DIM>(rj, q);
        Pi[q] = rec_P<DIM>(rj, q);
      }
      di = rj.invd;
      dj = rj.invd;
    }
    pair_force_add<T, DIM>(pp, g, v, Pi, Pj, di, dj, acc);
  }
}

// One list position of a fluid particle whose partner there is a fluid particle (or is
// absent: valid false): pair_term's fluid-fluid term without its type tests, for warps whose
// every lane has such a position (fewer branches, longer blocks for the scheduler).  For a
// fluid particle the terms taken follow from MODE alone (load_own's do_grad, do_force).
template <int MODE>
struct FluidTerms {
  static constexpr bool kGrad = MODE != kPairForcesOnly;
  static constexpr bool kForce = MODE != kPairGradvAll;
};
template <typename T, int DIM, bool WRAP, int MODE, typename Rec>
__device__ __forceinline__ void pair_fluid_x1(const BoxParams& p, const PairParams<T, DIM>& pp,
                                              const PairOwn<T, DIM>& o, const Rec& rj,
                                              bool valid, PairAcc<T, DIM>& acc) {
  T r[3];
  const T r2 = pair_sep<T, DIM, WRAP>(pp, p.wall, o, rj, r);
  if (!(valid && r2 < pp.rcutsq)) return;
  const T v[3] = {o.v[0] - (T)rj.vx, o.v[1] - (T)rj.vy, o.v[2] - (T)rec_vz<DIM>(rj)};
  PairRadial<T, DIM> g;
  g.eval(pp, r2, r);
  if constexpr (FluidTerms<MODE>::kGrad) pair_grad_add<T, DIM>(o, g, v, acc);
  if constexpr (FluidTerms<MODE>::kForce) {
    T Pj[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) Pj[q] = rec_P<DIM>(rj, q);
    pair_force_add<T, DIM>(pp, g, v, o.P, Pj, o.invd, (T)rj.invd, acc);
  }
}

// Second half-kick of a fluid particle's velocity, v += (dt / 2) f / m
// (kernel_move_sys_VV_part2.cu:13-58), as explicit fused multiply-adds so that the step's
// fused form and the standalone V_Verlet_step2 give the same bits.
template <int DIM>
__device__ __forceinline__ void vv2_fluid(const BoxParams& p, double mass, double fx, double fy,
                                          double fz, double4& v) {
  const double hm = 0.5 * p.dt / mass;
  v.x = __fma_rn(hm, fx, v.x);
  v.y = __fma_rn(hm, fy, v.y);
  if (DIM == 3) v.z = __fma_rn(hm, fz, v.z);
}

// stored gradient, forces with the body force, and dc/dt of particle i
template <typename T, int DIM, int MODE, bool EXT>
__device__ __forceinline__ void pair_store(const Dev& d, int i, const BoxParams& p,
                                           const PairOwn<T, DIM>& o,
                                           const PairAcc<T, DIM>& acc) {
  const int Np2 = d.Npad;
  if (MODE == kPairGradvAll || (MODE == kPairFused && d.gradv != nullptr && o.do_grad)) {
    // storage order xx xy xz yx yy yz zx zy zz
    d.gradv[0 * Np2 + i] = acc.grad(0, 0);
    d.gradv[1 * Np2 + i] = acc.grad(0, 1);
    d.gradv[3 * Np2 + i] = acc.grad(1, 0);
    d.gradv[4 * Np2 + i] = acc.grad(1, 1);
    if (DIM == 3) {
      d.gradv[2 * Np2 + i] = acc.grad(0, DIM - 1);
      d.gradv[5 * Np2 + i] = acc.grad(1, DIM - 1);
      d.gradv[6 * Np2 + i] = acc.grad(DIM - 1, 0);
      d.gradv[7 * Np2 + i] = acc.grad(DIM - 1, 1);
      d.gradv[8 * Np2 + i] = acc.grad(DIM - 1, DIM - 1);
    }
  }
  if (MODE == kPairGradvAll) return;
  double fx = acc.force(0), fy = acc.force(1), fz = acc.force(2);
  if (EXT && o.fluid) {
    const double4 xd = d.pos[i];
    const double m = xd.w;
    if (p.ext_force_type == 1) {
      fx += m * p.ext_force[0];
      fy += m * p.ext_force[1];
      if (DIM == 3) fz += m * p.ext_force[2];
    } else if (p.ext_force_type == 2) {
      fx += m * p.ext_force[0] * sin(p.ky * xd.y);
      fy += 0.0;
      if (DIM == 3) fz += 0.0;
    } else if (p.ext_force_type == 3) {
      fx += (xd.y < 0.5 * p.L[1]) ? m * p.ext_force[0] : -(m * p.ext_force[0]);
      fy += 0.0;
      if (DIM == 3) fz += 0.0;
    }
  }
  d.f[i] = fx;
  d.f[Np2 + i] = fy;
  if (DIM == 3) d.f[2 * Np2 + i] = fz;
  if (MODE == kPairFused && !o.fluid) {
    // kernel_dcdt.cu:39 leaves dc/dt of walls and colloids at its initial zero
#pragma unroll
    for (int q = 0; q < 6; ++q) d.dcdt[q * Np2 + i] = 0.0;
  }
  if (MODE == kPairFused && o.fluid) {
    // dc/dt = c.g + (c.g)^T + (I - c)/tau  (kernel_dcdt.cu:76-102)
    const double tinv = 1.0 / p.tau;
    double dc[6];
    const double cxx = d.conf[i], cxy = d.conf[Np2 + i], cyy = d.conf[2 * Np2 + i];
    if (DIM == 2) {
      const double gxx = acc.grad(0, 0), gxy = acc.grad(0, 1), gyx = acc.grad(1, 0),
                   gyy = acc.grad(1, 1);
      const double Axx = cxx * gxx + cxy * gyx, Axy = cxx * gxy + cxy * gyy;
      const double Ayx = cxy * gxx + cyy * gyx, Ayy = cxy * gxy + cyy * gyy;
      dc[0] = 2.0 * Axx + tinv * (1.0 - cxx);
      dc[1] = Axy + Ayx - tinv * cxy;
      dc[2] = 2.0 * Ayy + tinv * (1.0 - cyy);
      // the z components stay zero in 2D
      dc[3] = 0.0;
      dc[4] = 0.0;
      dc[5] = 0.0;
    } else {
      const double cxz = d.conf[3 * Np2 + i], cyz = d.conf[4 * Np2 + i], czz = d.conf[5 * Np2 + i];
      const double gxx = acc.grad(0, 0), gxy = acc.grad(0, 1), gxz = acc.grad(0, DIM - 1);
      const double gyx = acc.grad(1, 0), gyy = acc.grad(1, 1), gyz = acc.grad(1, DIM - 1);
      const double gzx = acc.grad(DIM - 1, 0), gzy = acc.grad(DIM - 1, 1),
                   gzz = acc.grad(DIM - 1, DIM - 1);
      const double Axx = cxx * gxx + cxy * gyx + cxz * gzx;
      const double Axy = cxx * gxy + cxy * gyy + cxz * gzy;
      const double Axz = cxx * gxz + cxy * gyz + cxz * gzz;
      const double Ayx = cxy * gxx + cyy * gyx + cyz * gzx;
      const double Ayy = cxy * gxy + cyy * gyy + cyz * gzy;
      const double Ayz = cxy * gxz + cyy * gyz + cyz * gzz;
      const double Azx = cxz * gxx + cyz * gyx + czz * gzx;
      const double Azy = cxz * gxy + cyz * gyy + czz * gzy;
      const double Azz = cxz * gxz + cyz * gyz + czz * gzz;
      dc[0] = 2.0 * Axx + tinv * (1.0 - cxx);
      dc[1] = Axy + Ayx - tinv * cxy;
      dc[2] = 2.0 * Ayy + tinv * (1.0 - cyy);
      dc[3] = Axz + Azx - tinv * cxz;
      dc[4] = Ayz + Azy - tinv * cyz;
      dc[5] = 2.0 * Azz + tinv * (1.0 - czz);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) d.dcdt[q * Np2 + i] = dc[q];
    if (d.fold_vv2) {
      // the step's second half-kick of this fluid particle (kernel_move_sys_VV_part2.cu:13-58),
      // the same operations as vv2_fluid, on the force and rate just stored
      double4 v = d.vel[i];
      vv2_fluid<DIM>(p, d.pos[i].w, fx, fy, fz, v);
      d.vel[i] = v;
#pragma unroll
      for (int q = 0; q < (DIM == 3 ? 6 : 3); ++q)
        d.conf[q * Np2 + i] = __fma_rn(0.5 * p.dt, dc[q], d.conf[q * Np2 + i]);
    }
  }
}

}  // namespace sph
