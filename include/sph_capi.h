/*
 * sph_capi.h -- C ABI of the B200 SPH engine (Oldroyd-B fluid, y-walls, magnetic colloids).
 *
 * The engine is a drop-in for the per-step hot path of the reference program
 * BCAM-CFD/SPH-magnetic-particles-Oldroyd-B-in-cuda: each entry point below replaces one
 * member function of the reference's `class_system` (src/class_system.h) or one piece of
 * its driver (src/main.cu), and the citation beside each declaration names it.
 *
 * Conventions
 *  - Plain C types only: opaque context pointer, int status codes, double / int arrays.
 *  - Every call returns sph_status (0 = SPH_OK).  The reference returns 0/1 and traps the
 *    GPU on a bad cell (src/kernel_cell_ranges.cu:20-23); here a bad cell, a non-finite
 *    position or an overfull neighbour list is reported as a status and the context stays
 *    usable.  sph_last_error() gives a one-line reason.
 *  - One context holds one or more independent simulation boxes (an ensemble).  It owns
 *    its device memory and CUDA stream; there are no process globals (the reference keeps
 *    its constants in __constant__ memory, one box per process).  A context is used by one
 *    host thread at a time.
 *  - Arrays exchanged with the host are in the reference's original particle order
 *    (particle id = position in the reference's host arrays); box after box for ensembles.
 *  - No entry point falls back to a CPU path: without a usable CUDA device sph_create
 *    fails with SPH_ERR_CUDA.
 */
#ifndef SPH_CAPI_H
#define SPH_CAPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH_CAPI_VERSION 1
#define SPH_MAX_COLLOIDS 1000 /* src/config.h:22 */

typedef struct sph_ctx sph_ctx;

typedef enum sph_status {
  SPH_OK = 0,
  SPH_ERR_BAD_INPUT = 1,  /* invalid input values (read_input / initialize checks)   */
  SPH_ERR_CUDA = 2,       /* a CUDA runtime call failed, or no device                 */
  SPH_ERR_CELL_RANGE = 3, /* a particle hashed outside the cell grid                  */
  SPH_ERR_NAN = 4,        /* a non-finite particle position was produced              */
  SPH_ERR_TIMEOUT = 5,    /* a bounded device wait gave up                            */
  SPH_ERR_STATE = 6,      /* null handle, unknown field, call out of order           */
  SPH_ERR_NOMEM = 7,      /* device or host allocation failed                         */
  SPH_ERR_CAPACITY = 8,   /* neighbour list overflow (grown automatically on retry)   */
  SPH_ERR_IO = 9          /* a file could not be read or written                      */
} sph_status;

typedef enum sph_precision {
  SPH_PREC_FP64 = 0,  /* all arithmetic in double, as the reference's default build     */
  SPH_PREC_MIXED = 1  /* pair arithmetic in float, its per-particle sums in double;
                         positions, velocities, conformation tensor, integration and
                         global reductions in double                                    */
} sph_precision;

/* The keys of the reference's `input` file (src/system_read_input.cpp:102-269,
   README.md:42-134).  coll_xyz points to N_colloids x 3 doubles (row-major). */
typedef struct sph_input {
  int N[3];
  double L[3];
  int dim;
  double dt, t0;
  int Nsteps;
  double overlap, rho, c, P0, eta, zeta, np, kT, tau;
  int ext_force_type;
  double ext_force[3];
  int freq_micro, freq_macro, freq_walls, freq_colloids;
  int wall;
  double Vwall_top, Vwall_bottom;
  int N_colloids;
  double coll_R, coll_rho;
  const double* coll_xyz;
  int coll_move;
  double coll_repulsion_cuton, F0_repulsion, tau_repulsion, cutoff_magnetic, F0_magnetic,
      omega_magnetic;
  int new_sim;
} sph_input;

typedef struct sph_options {
  int precision;    /* sph_precision                                                   */
  int device;       /* CUDA device ordinal                                             */
  int use_graph;    /* sph_step replays a captured CUDA graph of one step             */
  int nbr_capacity; /* neighbour-list capacity in candidate chunks per particle (a chunk
                       is up to 32 consecutive slots of one neighbour cell in which the
                       particle has a neighbour); 0 = derived from overlap and dim.
                       Lists grow when a build needs more. */
  int init_on_device; /* 1: lattice boxes (new_sim 0) are built on the GPU -- sites,
                         colloid carving, wall layers, walls lists -- bit-identical to the
                         host set-up; colloid shells and restart files stay on the host */
} sph_options;

/* Scalar summary of a box (derived constants of src/system_initialize.cpp:47-262). */
typedef struct sph_info {
  int N, dim, wall, Ncells[3], Ntotal_cells, Nwalls, Nlist_walls, N_colloids,
      Nlist_colloids, Ncells_colloids[3], Ntotal_cells_colloids, step, nboxes, precision;
  double rcut, rcutsq, cw, c_gradw, csq, rho0, a, b, nkT, tau, dt, cell_size[3], wall_width,
      y_bottom, y_top, V_bottom, V_top, coll_R, coll_mass, coll_I, L[3], t0, omega_magnet;
  /* the remaining class_system scalars (src/class_system.h:13-143) */
  int Nmax, ext_force_type;
  double rcut_inv, c, rho, P0, ky, beta_max, ext_force[3], coll_rho, coll_rep_cuton,
      coll_rep_cutoff, rcuton_coll_rep, rcutoff_coll_rep, rcuton_coll_rep_sq,
      rcutoff_coll_rep_sq, rcutoff_coll, rcutoff_coll_sq, F0_rep, tau_rep, r0_magnet,
      r0_magnet_sq, F0_magnet, cell_colloids_size[3];
} sph_info;

/* Per-particle double fields readable / writable in original particle order. */
typedef enum sph_field {
  SPH_X = 0, SPH_Y, SPH_Z, SPH_VX, SPH_VY, SPH_VZ, SPH_FX, SPH_FY, SPH_FZ, SPH_DENS,
  SPH_PRESS, SPH_MASS, SPH_CXX, SPH_CXY, SPH_CYY, SPH_CXZ, SPH_CYZ, SPH_CZZ, SPH_DCDT_XX,
  SPH_DCDT_XY, SPH_DCDT_YY, SPH_DCDT_XZ, SPH_DCDT_YZ, SPH_DCDT_ZZ, SPH_GXX, SPH_GXY,
  SPH_GXZ, SPH_GYX, SPH_GYY, SPH_GYZ, SPH_GZX, SPH_GZY, SPH_GZZ,
  SPH_NUM_PARTICLE_FIELDS
} sph_field;

/* Per-colloid double fields (length N_colloids summed over boxes). */
typedef enum sph_colloid_field {
  SPH_COLL_X = 0, SPH_COLL_Y, SPH_COLL_Z, SPH_COLL_VX, SPH_COLL_VY, SPH_COLL_VZ,
  SPH_COLL_OMEGAX, SPH_COLL_OMEGAY, SPH_COLL_OMEGAZ, SPH_COLL_THETA, SPH_COLL_QUAT0,
  SPH_COLL_QUATX, SPH_COLL_QUATY, SPH_COLL_QUATZ, SPH_COLL_FX, SPH_COLL_FY, SPH_COLL_FZ,
  SPH_COLL_TX, SPH_COLL_TY, SPH_COLL_TZ,
  SPH_NUM_COLLOID_FIELDS
} sph_colloid_field;

/* ---------------------------------------------------------------- setup and teardown */

/* Parse a reference-format `input` file (class_system::read_input,
   src/system_read_input.cpp:18-512).  coll_buf receives N_colloids x 3 doubles and
   in->coll_xyz is pointed at it; coll_cap is its capacity in colloids. */
sph_status sph_read_input(const char* path, sph_input* in, double* coll_buf, int coll_cap,
                          char* msg, size_t msg_cap);

/* Build the box and upload it: class_system::constructor + initialize
   (src/system_constructor.cpp:15, src/system_initialize.cpp:16, new/old-sim particles
   src/system_initialize_particles_new_sim.cpp:16, ..._old_sim.cpp:17) and
   copy_pointers_to_device (src/system_copy_pointers_to_device.cpp:15).
   particles_path is read when in->new_sim != 0 (NULL = "input_particles.in"). */
sph_status sph_create(const sph_input* in, const char* particles_path, const sph_options* opt,
                      sph_ctx** out);

/* An ensemble of independent boxes in one context (no reference counterpart: the
   reference runs one box per process).  Boxes advance together in every call. */
sph_status sph_create_ensemble(int nboxes, const sph_input* inputs,
                               const char* const* particles_paths, const sph_options* opt,
                               sph_ctx** out);

/* Host mirror of the initial state: the particle arrays class_system holds on the host
   after constructor + initialize (src/class_system.h:13-44, system_initialize.cpp:16-359),
   computed without a GPU.  Each non-NULL array must hold `cap` entries; *n_out receives
   the particle count (also when cap is too small, which returns SPH_ERR_STATE). */
typedef struct sph_host_state {
  double *x, *y, *z, *vx, *vy, *vz, *mass, *cxx, *cxy, *cyy, *cxz, *cyz, *czz;
  int* type;
  int *walls_list, *walls_start;          /* Nlist_walls, 2 */
  int *colloids_list, *colloids_start;    /* Nlist_colloids, N_colloids */
  double *x_center, *y_center, *z_center; /* Nlist_colloids */
} sph_host_state;
sph_status sph_host_setup(const sph_input* in, const char* particles_path, int cap,
                          sph_host_state* out, int* n_out, sph_info* info);

/* Frees device memory, stream and graph (main.cu:481-553 + class_system::destructor). */
void sph_destroy(sph_ctx* ctx);

sph_status sph_get_info(const sph_ctx* ctx, int box, sph_info* out);
const char* sph_last_error(const sph_ctx* ctx);
const char* sph_status_string(sph_status s);

/* ----------------------------------------------- step methods of class_system */

/* class_system::neighbours_search (src/system_neighbours_search.cu:19-110): cell hash,
   stable (cell, id) radix sort, cell ranges, colloid coarse grid; also builds the
   neighbour lists the pair kernels read. */
sph_status sph_neighbours_search(sph_ctx* ctx);

/* class_system::calculate_density (src/system_calculate_density.cu:15-49). */
sph_status sph_calculate_density(sph_ctx* ctx);

/* class_system::calculate_pressure (src/system_calculate_pressure.cu:15-34). */
sph_status sph_calculate_pressure(sph_ctx* ctx);

/* class_system::calculate_vel_gradient (src/system_calculate_vel_gradient.cu:16-86),
   velocity gradient of every particle, stored. */
sph_status sph_calculate_vel_gradient(sph_ctx* ctx);

/* class_system::calculate_forces (src/system_calculate_forces.cu:16-174): density,
   velocity gradient, pressure, pair forces, external force, dc/dt, wall forces, colloid
   forces and torques.  m = magnetic moment (3 doubles) for every box, or NULL to use
   (cos wt, sin wt, 0) at the context's current time (main.cu:395-400). */
sph_status sph_calculate_forces(sph_ctx* ctx, const double* m);

/* class_system::calculate_external_forces (src/system_calculate_external_forces.cu:15-38)
   adds the body force to the current forces. */
sph_status sph_calculate_external_forces(sph_ctx* ctx);

/* class_system::calculate_force_walls (src/system_calculate_force_walls.cu:15-38). */
sph_status sph_calculate_force_walls(sph_ctx* ctx);

/* class_system::calculate_force_colloids (src/system_calculate_force_colloids.cu:15-97);
   m as for sph_calculate_forces. */
sph_status sph_calculate_force_colloids(sph_ctx* ctx, const double* m);

/* class_system::V_Verlet_step1 (src/system_V_Verlet_step1.cu:15-122). */
sph_status sph_vv_step1(sph_ctx* ctx);

/* class_system::V_Verlet_step2 (src/system_V_Verlet_step2.cu:15-94); advances the step
   counter of the context. */
sph_status sph_vv_step2(sph_ctx* ctx);

/* main.cu:287-323: magnetic moment at t0, neighbour search and forces of step 0. */
sph_status sph_initial_forces(sph_ctx* ctx);

/* main.cu:358-467 without output: nsteps x (VV1, search, m(t), forces, VV2).  Runs
   sph_initial_forces first if it has not run.  Asynchronous on the context's stream;
   errors raised on the device are reported by the next sph_synchronize (or by the next
   call of any other function, which first waits for the open steps).  A step that finds a
   problem stops there: its later kernels and all later steps do nothing, so the state is
   never advanced on bad data.  A neighbour list found too short is not an error: the next
   sph_synchronize grows the lists, finishes that step and runs the remaining steps.  A
   position outside the grid or not finite is reported with the step it was found in, and
   the state is left as that step's half-kick and drift made it; the step counter
   (sph_get_info) gives the steps completed. */
sph_status sph_step(sph_ctx* ctx, int nsteps);

/* Waits for the context's stream and reports device-side error flags; resumes an sph_step
   call whose lists had to grow (see sph_step). */
sph_status sph_synchronize(sph_ctx* ctx);

/* Neighbour-list statistics (no reference counterpart: the reference has no lists): the
   capacity in candidate chunks per particle, the most chunks a particle has needed in the
   list builds so far, and how many times the lists have grown. */
sph_status sph_neighbour_lists(sph_ctx* ctx, int* capacity, int* max_used, int* grown);

/* -------------------------------------------------------------- state access */

/* Copy a particle field (sph_field) to host memory, original particle order. */
sph_status sph_read_field(sph_ctx* ctx, int field, double* host_out);
/* Overwrite a particle field from host memory (original order). */
sph_status sph_write_field(sph_ctx* ctx, int field, const double* host_in);
/* Copy a particle field into a caller-owned device buffer (original order).  Asynchronous
   on the context's stream: sph_synchronize before the buffer is read on another stream. */
sph_status sph_read_field_device(sph_ctx* ctx, int field, double* dev_out);
/* Particle types (0 fluid, 1 bottom wall, 2 top wall, 3+k colloid k). */
sph_status sph_read_type(sph_ctx* ctx, int* host_out);
/* Colloid fields (sph_colloid_field). */
sph_status sph_read_colloid_field(sph_ctx* ctx, int field, double* host_out);
/* Wall forces: nboxes x 2 walls x 3 components (fx, fy, fz). */
sph_status sph_read_wall_forces(sph_ctx* ctx, double* host_out);

/* Cell arrays with the reference's semantics (kernel_cell_list.cu, kernel_cell_ranges.cu):
   particle_cell / particle_index sorted by (cell, id); cell_start / cell_end written for
   occupied cells only and otherwise keeping the values of earlier searches.  Box 0.
   The destinations may be host or device memory (NULL skips an array). */
sph_status sph_export_cells(sph_ctx* ctx, int* particle_cell, int* particle_index,
                            int* cell_start, int* cell_end);
/* Colloid coarse-grid arrays (kernel_cell_colloids_*.cu), box 0; host or device
   destinations. */
sph_status sph_export_colloid_cells(sph_ctx* ctx, int* coll_cell, int* coll_index,
                                    int* coll_cell_start, int* coll_cell_end);

/* Kinetic energy per box (kernel_calculate_macro_vars.cu:14-40), summed in a fixed
   order in double: nboxes values. */
sph_status sph_kinetic_energy(sph_ctx* ctx, double* host_out);

/* Time-averaged observables per box (no reference counterpart; they are the targets of
   parameter sweeps over ensembles).  sph_observe adds one sample of every box, taken
   from the current state (asynchronous; call it between steps):
     SPH_OBS_WALL_STRESS  wall shear stress -fx(top wall) / (Lx Lz), Lz = 1 in 2D
                          (the wall force of class_system::calculate_force_walls);
     SPH_OBS_N1           first normal-stress difference <nkT (cxx - cyy)> over the fluid;
     SPH_OBS_CHAIN_ORDER  colloid chain order <P2(e . m)> over colloid pairs closer than
                          2.5 R: e the unit bond vector, m the current field direction,
                          P2(c) = 2c^2 - 1 in 2D, (3c^2 - 1)/2 in 3D; 0 without such pairs;
     SPH_OBS_KE           kinetic energy (kernel_calculate_macro_vars.cu:14-40).
   sph_observables writes nboxes x SPH_NUM_OBS averages over the samples so far (and the
   sample count); sph_reset_observables starts over. */
enum { SPH_OBS_WALL_STRESS = 0, SPH_OBS_N1, SPH_OBS_CHAIN_ORDER, SPH_OBS_KE, SPH_NUM_OBS };
sph_status sph_observe(sph_ctx* ctx);
sph_status sph_observables(sph_ctx* ctx, double* host_out, long long* nsamples);
sph_status sph_reset_observables(sph_ctx* ctx);

/* Launch geometry of the neighbour passes (no reference counterpart; results do not
   depend on it, bit for bit):
     list_threads_per_cell  32: a warp per cell in the list build; 16: a half-warp per
                            cell (2D cells at overlap 4 hold about 16 particles)
     density_block          0: the density pass over neighbour-cell tiles (a warp per cell,
                            the cells' positions staged in shared memory); 64, 128 or 256:
                            threads per block of the per-particle density pass
   sph_set_tuning applies a geometry (captured step graphs are rebuilt).  sph_autotune
   times the candidates on the context's current state -- the timed passes recompute the
   same lists and densities, so the simulation is unchanged -- and keeps the fastest.
   With cache_path it first looks for an entry keyed by GPU name, dimension, overlap and
   particle count (rounded to a power of two) in that JSON file, and records its choice
   there otherwise.  The cell size stays the reference's (rcut): its cell grid carries the
   stale-range semantics of the exported cell arrays. */
typedef struct sph_tuning {
  int list_threads_per_cell;
  int density_block;
} sph_tuning;
sph_status sph_get_tuning(const sph_ctx* ctx, sph_tuning* out);
sph_status sph_set_tuning(sph_ctx* ctx, const sph_tuning* tuning);
sph_status sph_autotune(sph_ctx* ctx, const char* cache_path, sph_tuning* chosen);

/* Device time of the most recent sph_step, in milliseconds, measured with CUDA events
   on the context's stream. */
sph_status sph_last_step_ms(sph_ctx* ctx, double* ms);

/* Launch counters: kernels launched by the engine since creation. */
sph_status sph_kernel_launches(const sph_ctx* ctx, long long* count);

/* Neighbour search that allocates nothing.  No counterpart in the reference (whose
   thrust-based search allocates temporary storage on every call); it is for callers
   that cannot call cudaMalloc, such as programs whose device memory is reserved up front
   by their own allocator, or time loops that must not let an allocation stall the
   device.  Same results as sph_neighbours_search / sph_export_cells for one box, on
   caller-owned device arrays in original particle order: x, y (and z in 3D) hold n
   positions; particle_cell and particle_index (n ints) receive the (cell, id)-sorted
   pairs; cell_start and cell_end (Ncells[0]*Ncells[1]*Ncells[2] ints) are written for
   occupied cells only and keep earlier values elsewhere, as the reference's arrays do.
   The sort's scratch is a static device array of the library sized for at most
   SPH_NOALLOC_MAX_PARTICLES particles (about 13 MB, held by every GPU that loads the
   library until the process exits); larger n returns SPH_ERR_CAPACITY.  Every call looks
   up that array's device address in the current context (cheap; nothing is cached, so a
   call after cudaDeviceReset finds the array's new address).  The first call in a context
   loads the library's device code for this entry point, which places the array; make
   that first call (n = 0 is enough) before any stream capture.  All calls share the
   array: calls that overlap on the GPU race, so serialise them.  The call runs on
   `stream` (a cudaStream_t, NULL for the default stream) and waits for it before it
   returns; a particle outside the grid gives SPH_ERR_CELL_RANGE. */
#define SPH_NOALLOC_MAX_PARTICLES (1 << 20)
typedef struct sph_grid {
  int dim, wall;
  int Ncells[3];
  double cell_size[3];
  double wall_width;
} sph_grid;
sph_status sph_neighbours_search_noalloc(const double* x, const double* y, const double* z,
                                         int n, const sph_grid* grid, int* particle_cell,
                                         int* particle_index, int* cell_start, int* cell_end,
                                         void* stream);

/* Profiling (no reference counterpart; the reference times with clock(), main.cu:381-427):
   runs nsteps full steps with CUDA events between the phases on the context's stream and
   writes the mean device time of each phase in milliseconds to ms[0..SPH_NUM_PHASES-1]. */
#define SPH_NUM_PHASES 11
sph_status sph_profile_phases(sph_ctx* ctx, int nsteps, double* ms);
/* Name of phase k ("vv1", "hash", "sort", "reorder", "lists", "colloid_cells",
   "density", "pairs", "walls", "colloids", "vv2"). */
const char* sph_phase_name(int k);

#ifdef __cplusplus
}
#endif
#endif /* SPH_CAPI_H */
