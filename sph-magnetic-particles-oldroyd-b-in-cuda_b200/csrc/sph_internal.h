// sph_internal.h -- engine-internal types shared by the host setup, the kernels and the
// C-ABI layer.  Nothing here is part of the public interface (include/sph_capi.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <vector_types.h>

#include "sph_capi.h"

namespace sph {

// Particle type word: type in the low 12 bits (0 fluid, 1 bottom wall, 2 top wall,
// 3 + k colloid k of its box), box index above.  One int per particle carries both.
constexpr int kTypeBits = 12;
constexpr int kTypeMask = (1 << kTypeBits) - 1;

// Device error flags (bit set in Dev::status by any kernel that detects the condition).
// Once any of them is set, every state-changing kernel of the step returns at entry, so a
// failure found in step k of a multi-step (graph-replayed) call leaves the state where step
// k found it; the first report records the step counter and the phase (Dev::err_info).
enum StatusBits : unsigned {
  kStatCellRange = 1u, // hash outside the grid (reference traps: kernel_cell_ranges.cu:20-23)
  kStatNaN = 2u,       // non-finite position
  kStatCapacity = 4u,  // neighbour list full
  kStatAbortMask = 7u,
};
// Phase that made the first report: the hash (state not yet reordered in that step) or the
// list build (state reordered, lists incomplete).
enum FailPhase : int { kPhaseNone = 0, kPhaseHash = 1, kPhaseLists = 2 };
// Dev::err_info entries.
enum ErrInfo : int {
  kErrBadId = 0,     // global id of the first particle outside the grid / not finite
  kErrMaxCount = 1,  // largest neighbour-list row seen since the last reset
  kErrStepLo = 2,    // device step counter (completed steps) at the first report, low word
  kErrStepHi = 3,    // ... high word
  kErrPhase = 4,     // FailPhase of the first report
  // nonzero when a position may lie outside [0, L] along a periodic axis: cleared before
  // the hash of each search and set by the hash for every position it finds outside, by the
  // half-kicks for every position they leave outside, and by any write of positions from
  // the host.  While it is set the list build places every candidate by its minimum image;
  // while it is clear the pair passes may drop the minimum image for particles clear of the
  // periodic faces (clear_of_faces).
  kPosOutside = 5,
  kErrInfoLen = 8,
};

// Per-box constants.  Everything the reference keeps in __constant__ memory
// (src/kernel_declare_constants.cu:11-62) plus the box's offsets in the global arrays.
struct BoxParams {
  int dim, wall, ext_force_type, coll_move;
  int N;           // particles in this box
  int slot0;       // first slot (and first global id) of the box
  int cell0;       // first global cell index of the box
  int Ncells[3], Ntotal_cells;
  int N_colloids, coll0;  // colloids of the box and their first global index
  int wall_seg0;          // first of the box's two wall segments
  int pad0;
  double L[3], halfL[3], cell_size[3], wall_width;
  double rcut, rcutsq, rcut_inv, cw, c_gradw, csq, rho0, a, b, nkT, tau, dt;
  double ext_force[3], ky;
  double y_bottom, y_top, V_bottom, V_top, beta_max;
  double coll_R, coll_rho, coll_mass, coll_I;
  double F0_rep, tau_rep, rcuton_coll_rep_sq, rcutoff_coll_rep_sq, r0_magnet_sq, F0_magnet;
  double omega_magnet, t0;
  double list_cut2;  // squared list cutoff used by the float candidate test
  // colloid coarse grid (only exported; pair forces loop over all colloids of the box)
  int Ncells_colloids[3], Ntotal_cells_colloids;
  double cell_colloids_size[3];
  int ccell0;  // first global coarse-cell index of the box
  int pad1;
};

// Host-side description of one box after setup (original particle order), produced by
// the host setup (sph_setup.cpp) and uploaded by the context.
struct HostBox {
  BoxParams p;
  sph_input in;
  std::vector<double> coll_xyz;  // storage behind in.coll_xyz
  // particles (original order)
  std::vector<double> x, y, z, vx, vy, vz, mass, cxx, cxy, cyy, cxz, cyz, czz;
  std::vector<int> type;
  // walls_list / walls_start (system_initialize.cpp:278-300), local ids
  std::vector<int> walls_list;
  int walls_start[2] = {0, 0};
  int Nlist_walls = 0;
  // colloids (system_initialize.cpp:176-201, 304-355)
  std::vector<int> colloids_list, colloids_start;
  std::vector<double> x_center, y_center, z_center;
  std::vector<double> coll_x, coll_y, coll_z;
  int Nmax = 0;  // reserved particles (system_constructor.cpp:62-79)
  // Lattice generated on the device (sph_init.cu): the host arrays above then hold only
  // the colloid shells, which follow the nlat lattice particles in the box's id order.
  bool lattice_on_device = false;
  int Nxyz[3] = {0, 0, 0};  // lattice sites per direction, wall rows included
  double dx[3] = {0.0, 0.0, 0.0};
  double lattice_m = 0.0;   // particle mass of the lattice
  int host0 = 0;            // box-local id of the first host-built particle (= nlat)
};

// Scalar summary of a box (sph_info), step / nboxes / precision left zero.
void fill_info(const HostBox& hb, sph_info* o);

// Parses a reference `input` file.  Returns SPH_OK or SPH_ERR_BAD_INPUT / SPH_ERR_IO.
sph_status parse_input_file(const char* path, sph_input* in, std::vector<double>* coll,
                            std::string* msg);
// Builds a box from its inputs (constructor + initialize of the reference).
// With lattice_on_device, a lattice box (new_sim 0) gets its parameters and colloid shells
// only; its lattice, walls list and particle count come from the device (sph_init.cu).
sph_status build_box(const sph_input& in, const char* particles_path, HostBox* box,
                     std::string* msg, bool lattice_on_device = false);

// Neighbour-record layouts (one per particle, slot order), written by the density
// epilogue and gathered by the pair kernel.  P holds Pi/d^2 = (p I - nkT c)/d^2 for
// fluid particles and -nkT c for walls and colloid particles (whose Pi is rebuilt with
// the fluid partner's pressure and density, kernel_forces.cu:217-233).
struct alignas(16) RecD {
  double x, y, z, vx, vy, vz;
  double P[6];
  double invd;
  int tinfo;
  int pad;
  double pad2[2];
};
static_assert(sizeof(RecD) == 128, "RecD layout");

struct alignas(16) RecF {
  float x, y, z, vx, vy, vz;
  float P[6];
  float invd;
  int tinfo;
  float pad[2];
};
static_assert(sizeof(RecF) == 64, "RecF layout");

// 2D records: only the fields a 2D pair term reads (P = xx, xy, yy); the type word is read
// from the slot-ordered type array.  Half the bytes of the 3D records to stage per pair.
struct alignas(16) RecD2 {
  double x, y, vx, vy;
  double P[3];
  double invd;
};
static_assert(sizeof(RecD2) == 64, "RecD2 layout");

struct alignas(16) RecF2 {
  float x, y, vx, vy;
  float P[3];
  float invd;
};
static_assert(sizeof(RecF2) == 32, "RecF2 layout");

// The pair constants of a context with one box, in both precisions: kernels receive Dev by
// value, so these live in the constant bank, where the pair pass's arithmetic reads them as
// operands instead of holding them in registers (PairParams has the same layout).
struct PairConsts {
  double L[3], h[3], rcutsq, rcut_inv, c_gradw, a, b;
  float Lf[3], hf[3], rcutsqf, rcut_invf, c_gradwf, af, bf;
};

// Device pointers, passed to kernels by value.
struct Dev {
  int Ntot, Npad, nboxes, Ctot, ncoll, nwallseg;
  int cap;  // neighbour-list capacity: chunks with hits per particle
  const BoxParams* box;
  double4* pos;  // x, y, z, mass
  double4* vel;  // vx, vy, vz, 0
  double* conf;  // 6 x Npad: cxx, cxy, cyy, cxz, cyz, czz
  int* tinfo;    // type | box << kTypeBits
  int* gid;      // slot -> global particle id
  int* inv;      // global id -> slot
  double4* pos_b;
  double4* vel_b;
  double* conf_b;
  int* tinfo_b;
  int* gid_b;
  float4* pos_f;  // float copy of pos (mixed precision only), slot order
  double* dens;
  double* press;
  double* f;     // 3 x Npad
  double* dcdt;  // 6 x Npad
  double* f_b;   // reorder targets of f / dcdt when a search falls between
  double* dcdt_b;  // a force evaluation and the half-kick that consumes it
  double* gradv; // 9 x Npad: xx xy xz yx yy yz zx zy zz
  void* rec;     // RecD or RecF per slot
  // neighbour candidates (k_build_lists): per particle, for every chunk of up to 32
  // consecutive candidate slots in which it has a hit, (first slot, hit mask), chunk-major
  int2* nchunk;     // cap x Npad: nchunk[k * Npad + i]
  int* nbr_nch;     // per slot: chunks stored
  int* nbr_cnt;     // per slot: candidates (set bits over the particle's chunks)
  int* key_by_gid;
  int* keys;     // sorted keys
  int* vals;     // sorted values (global ids)
  int* keys_alt;
  int* vals_alt;
  int* cell_begin;     // Ctot + 1: first slot of each global cell (current)
  int* cell_start;     // Ctot, reference semantics, box-local slot index
  int* cell_end;       // Ctot
  int* cell_box;       // Ctot: owning box of each global cell
  // walls
  int* walls_list;     // global ids
  int* wall_seg;       // nwallseg + 1 segment boundaries into walls_list
  double* wall_f;      // nwallseg x 3
  int* wall_chunk;     // nwallchunks + 1 boundaries into walls_list, never across segments
  int* wall_seg_chunk; // nwallseg + 1 boundaries into the chunks
  double* wall_part;   // nwallchunks x 3 partial sums
  int nwallchunks;
  // colloids
  int* colloids_list;  // global ids
  int* coll_seg;       // ncoll + 1 segment boundaries into colloids_list
  int* coll_box;       // ncoll
  double* xc;          // body-frame offsets per colloids_list entry (3 x Nlist)
  int Nlist_coll;
  double* cs;          // colloid state, kCollFields x ncoll
  int* ccell;          // colloid coarse-grid arrays (reference semantics), ncoll
  int* cindex;
  int* ccell_start;    // sum of coarse cells over boxes
  int* ccell_end;
  double* mag;         // 3 x nboxes magnetic moments
  double* ke;          // nboxes
  int* ke_chunk;       // nkechunks + 1 slot boundaries, chunks never straddle boxes
  int* ke_box_chunk;   // nboxes + 1 chunk boundaries per box
  int nkechunks;
  long long* step;     // device step counter (graph replays)
  unsigned* status;
  int* err_info;       // kErrInfoLen ints, see ErrInfo
  int grad_all;        // fused pair pass: velocity gradient of every particle, not only fluid
  int fold_vv2;        // fused pair pass: also the step's second half-kick of fluid particles
  int one_box;         // a single box: its pair constants are in pc
  PairConsts pc;
};

// Colloid state layout in Dev::cs (each row ncoll long).
enum CollField {
  CS_X = 0, CS_Y, CS_Z, CS_VX, CS_VY, CS_VZ, CS_OX, CS_OY, CS_OZ, CS_THETA, CS_Q0, CS_QX,
  CS_QY, CS_QZ, CS_FX, CS_FY, CS_FZ, CS_TX, CS_TY, CS_TZ, kCollFields
};

// Entries of a walls list summed by one block of the wall-force reduction.
constexpr int kWallChunk = 512;

// Kernel launchers (sph_kernels.cu); all asynchronous on `stream`.
struct Launch {
  Dev d;
  int prec;  // sph_precision
  void* stream;
  long long* launches;
  int list_tpc = 32;        // threads per cell of the list build (32 or 16)
  int density_block = 128;  // density pass: 0 = neighbour-cell tiles, else threads per block
  // (launch geometry only: results do not depend on it)
};

enum PairMode { kPairFused = 0, kPairGradvAll = 1, kPairForcesOnly = 2 };

// CUDA error code of the most recent failed launch on this thread (0 = none); the
// launchers clear the runtime's last-error state, so the code is kept here for reporting.
inline int& last_launch_error() {
  static thread_local int e = 0;
  return e;
}

int launch_vv1_particles(const Launch& L);
int launch_vv1_colloids(const Launch& L);
int launch_vv2(const Launch& L, bool particles = true);
int launch_hash(const Launch& L);
int launch_reorder(const Launch& L, bool permute_forces);
int launch_build_lists_dim(const Launch& L, int dim);
int launch_colloid_cells_n(const Launch& L, int nboxes, int max_coll);
int launch_density_dim(const Launch& L, int dim);
int launch_pressure(const Launch& L);
int launch_pairs_dim(const Launch& L, int dim, int mode, int with_ext);
int launch_ext_force(const Launch& L);
int launch_dcdt_from_gradv(const Launch& L);
int launch_wall_forces(const Launch& L);
int launch_colloid_forces(const Launch& L, int with_pairs);
int launch_advance_time(const Launch& L, int mode);
int launch_count_step(const Launch& L);
int launch_kinetic_energy(const Launch& L, double* partial);
// one observables sample of every box added to acc (nboxes x 4), KE included
int launch_observe(const Launch& L, double* ke_partial, double* obs_partial, double* acc);
int launch_gather_field(const Launch& L, int field, double* out);
int launch_scatter_field(const Launch& L, int field, const double* in);
int launch_gather_int(const Launch& L, const int* src, int* out);

// Device-side initialisation of a lattice box (sph_init.cu).  Sites are processed in
// blocks of kInitThreads; a box owns the blocks [blk0, blk0 + nblk).
constexpr int kInitThreads = 256;
struct InitBox {
  int box;          // box index (type word)
  int dim, wall;
  int Nxyz[3];      // lattice sites per direction, wall rows included
  int nsites;       // Nxyz product (Nxyz[2] taken as 1 in 2D)
  int blk0, nblk;
  int coll0, ncoll; // the box's colloid centres in the centres array (3 doubles each)
  int slot0;        // fill pass: first slot of the box
  int wl0, nw1;     // fill pass: first walls_list entry, bottom-wall particles
  double dx[3], wall_width, R2, mass, L[3], y_bottom, y_top;
};
// counts: 3 per block (kept, bottom wall, top wall)
int launch_init_count(const InitBox* boxes, const int* blk_box, int nblk, const double* centres,
                      int* counts, void* stream);
// offs: 3 per block, the box-local counts before the block
int launch_init_fill(const Launch& L, const InitBox* boxes, const int* blk_box, int nblk,
                     const double* centres, const int* offs);
// host-built particles, packed: (slot, type word), position + mass, velocity, conformation
int launch_init_scatter(const Launch& L, int n, const int2* meta, const double4* pos,
                        const double4* vel, const double* conf);

// Stable LSD radix sort of the hash keys (sph_sort.cu): keys d.key_by_gid indexed by
// global id, values = global ids; result in d.keys / d.vals.
// Geometry of the sort, shared by every user of its histogram buffer: items per tile,
// buckets per pass (at most 9 key bits per pass) and entries per scan block.
constexpr int kSortTile = 4096;
constexpr int kSortMaxBuckets = 512;
constexpr int kSortScanChunk = 2048;
// Histogram ints the sort needs for n keys: a bucket-major table of kSortMaxBuckets
// counters per tile, one partial sum per scan block, and padding.
constexpr size_t sort_hist_ints(long long n) {
  return (size_t)kSortMaxBuckets * (size_t)(n > 0 ? (n + kSortTile - 1) / kSortTile : 1) +
         ((size_t)kSortMaxBuckets * (size_t)(n > 0 ? (n + kSortTile - 1) / kSortTile : 1) +
          kSortScanChunk - 1) / kSortScanChunk +
         32;
}
struct SortScratch {
  int* hist;       // radix histogram / offsets
  int hist_len;
  int ntiles;
};
size_t sort_hist_len(int n, int key_bits);
int launch_sort(const Launch& L, int key_bits, const SortScratch& scr);

}  // namespace sph
