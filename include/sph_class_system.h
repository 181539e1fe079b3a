/* sph_class_system.h -- the reference's `class_system` (src/class_system.h:12-650) as a
 * C++ shim over the engine's C ABI (sph_capi.h), so that a driver written against the
 * reference, such as its own src/main.cu, re-links against this engine unchanged.
 *
 * Same data members (names and types), same member functions (names, parameters, return
 * values 0 = success / 1 = error, printf-style messages), same output files
 * (micro-<step>.dat, walls-<step>.dat, colloids-<step>.dat, macro.dat, gradv-<step>.dat).
 * `real` is double here: the reference's FP64 configuration (src/config.h:15-16).
 *
 * What differs, by design:
 *  - The engine owns the simulation state on the GPU in its own layout (slot order, state
 *    double-buffered).  The device buffers the caller passes (k_x, k_vx, ...) are the ones
 *    copy_pointers_to_device allocates, exactly as the reference allocates them (the
 *    caller frees them with cudaFree, src/main.cu:481-553).  They hold the initial state
 *    and are refreshed from the engine, in original particle order, whenever an output
 *    routine (print_output, print_particles, print_walls, print_colloids,
 *    print_particles_gradv, print_macro_vars) writes them; between outputs the engine
 *    does not read them, so writing into them does not change the simulation.
 *  - The __constant__ parameters that src/main.cu:185-236 uploads are not read by the
 *    engine (each box keeps its own parameter block); the upload itself stays harmless.
 *  - neighbours_search does not refill k_particle_cell / k_particle_index / k_cell_start /
 *    k_cell_end on every call; export_cells() copies them out on request.
 */
#pragma once

#include <cuda_runtime.h>

#include "sph_capi.h"

struct class_system_engine;  // shim state (engine context, parsed input, host storage)

struct class_system {
  int N;     // Number of particles
  int Nmax;  // reserved number of particles

  double *x, *y, *z;     // host mirrors, original particle order
  double *vx, *vy, *vz;
  double *fx, *fy, *fz;
  double* dens;
  double* press;
  double* mass;
  int* type;
  double *cxx_tensor, *cxy_tensor, *cyy_tensor, *cxz_tensor, *cyz_tensor, *czz_tensor;
  double nkT;
  double tau;

  double L[3];
  int dim;

  int wall;
  double y_bottom, y_top, V_bottom, V_top;
  int Nwalls;
  double *fx_wall, *fy_wall, *fz_wall;
  int Nlist_walls;
  int* walls_list;
  int* walls_start;
  double wall_width;

  int N_colloids;
  double coll_R, coll_rho;
  int Nlist_colloids;
  int* colloids_list;
  int* colloids_start;
  double *coll_x, *coll_y, *coll_z;
  double *coll_vx, *coll_vy, *coll_vz;
  double *coll_omegax, *coll_omegay, *coll_omegaz;
  double* coll_theta;
  double *coll_quat0, *coll_quatx, *coll_quaty, *coll_quatz;
  double coll_mass, coll_I;
  double *x_center, *y_center, *z_center;
  double *quat0, *quatx, *quaty, *quatz;
  double *fx_colloid, *fy_colloid, *fz_colloid;
  double *tx_colloid, *ty_colloid, *tz_colloid;
  double coll_rep_cutoff, coll_rep_cuton, rcutoff_coll_rep, rcuton_coll_rep;
  double rcutoff_coll_rep_sq, rcuton_coll_rep_sq, rcutoff_coll, rcutoff_coll_sq;
  double F0_rep, tau_rep;
  double r0_magnet, r0_magnet_sq, F0_magnet, omega_magnet;

  double rcut, rcutsq, rcut_inv, cw, c_gradw, c, csq;
  double rho, P0, rho0;
  double a, b;

  double cell_size[3];
  int Ncells[3];
  int Ntotal_cells;
  double cell_colloids_size[3];
  int Ncells_colloids[3];
  int Ntotal_cells_colloids;
  int ext_force_type;
  double ext_force[3];
  double ky;
  double kin_energy;

  double beta_max;

  /* ---- set-up (src/system_read_input.cpp, system_initialize_pointers.cpp,
          system_constructor.cpp, system_initialize.cpp, system_print_info.cpp,
          system_copy_pointers_to_device.cpp, system_destructor.cpp) ---- */
  int read_input(int N[3], double L[3], int& dim, double& delta_t, double& t_ini, int& Nsteps,
                 double& overlap, double& rho, double& c, double& P0, double& eta, double& zeta,
                 double& np, double& kT, double& elast_time, int& ext_force_type,
                 double ext_force[3], int& freq_micro, int& freq_macro, int& freq_walls,
                 int& freq_colloid, int& wall, double& Vwall_top, double& Vwall_bottom,
                 int& N_coll, double& coll_radius, double& col_density,
                 double coll_x_data[][3], int& coll_move, double& coll_repulsion_cuton,
                 double& F0_repulsion, double& tau_repulsion, double& cutoff_magnetic,
                 double& F0_magnetic, double& omega_magnetic, int& new_sim);
  void initialize_pointers();
  void constructor(int Nxyz[3], int wall, double overlap, int dim, int N_coll, int new_sim);
  int initialize(int Nxyz[3], double L[3], int dim, double overlap, double rho, double c,
                 double P0, double eta, double zeta, double np, double kT, double elast_time,
                 int ext_force_type, double ext_force[3], int wall, double Vwall_top,
                 double Vwall_bottom, int N_coll, double coll_radius, double coll_density,
                 double coll_x_data[][3], double coll_repulsion_cuton, double F0_repulsion,
                 double tau_repulsion, double cutoff_magnetic, double F0_magnetic,
                 double omega_magnetic, int new_sim);
  int initialize_particles_new_sim(int Nxyz[3], double dx[3]);
  int initialize_particles_old_sim();
  void print_info();
  int copy_pointers_to_device(
      double** k_x, double** k_y, double** k_z, double** k_vx, double** k_vy, double** k_vz,
      double** k_mass, double** k_fx, double** k_fy, double** k_fz, double** k_dens,
      double** k_press, int** k_particle_cell, int** k_particle_index, int** k_cell_start,
      int** k_cell_end, double** k_kin_energy, int** k_type, double** k_cxx, double** k_cxy,
      double** k_cyy, double** k_cxz, double** k_cyz, double** k_czz, double** k_dcdt_xx,
      double** k_dcdt_xy, double** k_dcdt_yy, double** k_dcdt_xz, double** k_dcdt_yz,
      double** k_dcdt_zz, double** k_gradvxx, double** k_gradvxy, double** k_gradvxz,
      double** k_gradvyx, double** k_gradvyy, double** k_gradvyz, double** k_gradvzx,
      double** k_gradvzy, double** k_gradvzz, double** k_fx_wall, double** k_fy_wall,
      double** k_fz_wall, int** k_walls_list, int** k_walls_start, int** k_colloids_list,
      int** k_colloids_start, double** k_coll_x, double** k_coll_y, double** k_coll_z,
      double** k_coll_vx, double** k_coll_vy, double** k_coll_vz, double** k_coll_omegax,
      double** k_coll_omegay, double** k_coll_omegaz, double** k_coll_theta,
      double** k_coll_quat0, double** k_coll_quatx, double** k_coll_quaty,
      double** k_coll_quatz, double** k_x_center, double** k_y_center, double** k_z_center,
      double** k_fx_colloid, double** k_fy_colloid, double** k_fz_colloid,
      double** k_tx_colloid, double** k_ty_colloid, double** k_tz_colloid, int** k_coll_cell,
      int** k_coll_index, int** k_coll_cell_start, int** k_coll_cell_end,
      double** k_magnetic_mom);
  void destructor();

  /* ---- step methods (src/system_neighbours_search.cu, system_calculate_*.cu,
          system_V_Verlet_step1.cu, system_V_Verlet_step2.cu); the launch shape
          arguments are accepted and ignored: the engine sizes its own grids ---- */
  int neighbours_search(dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y,
                        double* k_z, int* k_particle_cell, int* k_particle_index,
                        int* k_cell_start, int* k_cell_end, double* k_coll_x, double* k_coll_y,
                        double* k_coll_z, int* k_coll_cell, int* k_coll_index,
                        int* k_coll_cell_start, int* k_coll_cell_end);
  int calculate_density(dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y,
                        double* k_z, double* k_dens, int* k_particle_index, int* k_cell_start,
                        int* k_cell_end);
  int calculate_pressure(dim3 numBlocks, dim3 threadsPerBlock, double* k_press, double* k_dens,
                         double* k_mass);
  int calculate_forces(
      dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y, double* k_z,
      double* k_vx, double* k_vy, double* k_vz, double* k_cxx, double* k_cxy, double* k_cyy,
      double* k_cxz, double* k_cyz, double* k_czz, double* k_fx, double* k_fy, double* k_fz,
      double* k_dcdt_xx, double* k_dcdt_xy, double* k_dcdt_yy, double* k_dcdt_xz,
      double* k_dcdt_yz, double* k_dcdt_zz, double* k_gradvxx, double* k_gradvxy,
      double* k_gradvxz, double* k_gradvyx, double* k_gradvyy, double* k_gradvyz,
      double* k_gradvzx, double* k_gradvzy, double* k_gradvzz, double* k_press, double* k_dens,
      double* k_mass, int* k_particle_index, int* k_cell_start, int* k_cell_end, int* k_type,
      double* k_fx_wall, double* k_fy_wall, double* k_fz_wall, int* k_walls_list,
      int* k_walls_start, double* k_coll_x, double* k_coll_y, double* k_coll_z,
      double* k_coll_vx, double* k_coll_vy, double* k_coll_vz, double* k_coll_omegax,
      double* k_coll_omegay, double* k_coll_omegaz, double* k_fx_colloid,
      double* k_fy_colloid, double* k_fz_colloid, double* k_tx_colloid, double* k_ty_colloid,
      double* k_tz_colloid, int* k_colloids_list, int* k_colloids_start, int* k_coll_index,
      int* k_coll_cell_start, int* k_coll_cell_end, double* k_magnetic_mom);
  int calculate_external_forces(dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y,
                                double* k_z, double* k_fx, double* k_fy, double* k_fz,
                                double* k_mass, int* type);
  int calculate_force_walls(dim3 numBlocks, dim3 threadsPerBlock, double* k_fx_wall,
                            double* k_fy_wall, double* k_fz_wall, double* k_fx, double* k_fy,
                            double* k_fz, int* k_walls_list, int* k_walls_start);
  int calculate_force_colloids(dim3 numBlocks, dim3 threadsPerBlock, double* k_coll_x,
                               double* k_coll_y, double* k_coll_z, double* k_fx_colloid,
                               double* k_fy_colloid, double* k_fz_colloid,
                               double* k_tx_colloid, double* k_ty_colloid,
                               double* k_tz_colloid, double* k_x, double* k_y, double* k_z,
                               double* k_fx, double* k_fy, double* k_fz, int* k_colloids_list,
                               int* k_colloids_start, int* k_coll_index,
                               int* k_coll_cell_start, int* k_coll_cell_end,
                               double* k_magnetic_mom);
  int V_Verlet_step1(
      dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y, double* k_z,
      double* k_vx, double* k_vy, double* k_vz, double* k_cxx, double* k_cxy, double* k_cyy,
      double* k_cxz, double* k_cyz, double* k_czz, double* k_fx, double* k_fy, double* k_fz,
      double* k_dcdt_xx, double* k_dcdt_xy, double* k_dcdt_yy, double* k_dcdt_xz,
      double* k_dcdt_yz, double* k_dcdt_zz, double* k_mass, int* k_type, double* k_coll_x,
      double* k_coll_y, double* k_coll_z, double* k_coll_vx, double* k_coll_vy,
      double* k_coll_vz, double* k_coll_omegax, double* k_coll_omegay, double* k_coll_omegaz,
      double* k_coll_theta, double* k_coll_quat0, double* k_coll_quatx, double* k_coll_quaty,
      double* k_coll_quatz, double* k_fx_colloid, double* k_fy_colloid, double* k_fz_colloid,
      double* k_tx_colloid, double* k_ty_colloid, double* k_tz_colloid, double* k_x_center,
      double* k_y_center, double* k_z_center, int* k_colloids_list, int* k_colloids_start,
      int coll_move);
  int V_Verlet_step2(dim3 numBlocks, dim3 threadsPerBlock, double* k_vx, double* k_vy,
                     double* k_vz, double* k_cxx, double* k_cxy, double* k_cyy, double* k_cxz,
                     double* k_cyz, double* k_czz, double* k_fx, double* k_fy, double* k_fz,
                     double* k_dcdt_xx, double* k_dcdt_xy, double* k_dcdt_yy,
                     double* k_dcdt_xz, double* k_dcdt_yz, double* k_dcdt_zz, double* k_mass,
                     int* k_type, double* k_coll_vx, double* k_coll_vy, double* k_coll_vz,
                     double* k_coll_omegax, double* k_coll_omegay, double* k_coll_omegaz,
                     double* k_fx_colloid, double* k_fy_colloid, double* k_fz_colloid,
                     double* k_tx_colloid, double* k_ty_colloid, double* k_tz_colloid,
                     int coll_move);
  int calculate_vel_gradient(dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y,
                             double* k_z, double* k_vx, double* k_vy, double* k_vz,
                             double* k_gradvxx, double* k_gradvxy, double* k_gradvxz,
                             double* k_gradvyx, double* k_gradvyy, double* k_gradvyz,
                             double* k_gradvzx, double* k_gradvzy, double* k_gradvzz,
                             double* k_dens, int* k_particle_index, int* k_cell_start,
                             int* k_cell_end, int* k_type, double* k_coll_x, double* k_coll_y,
                             double* k_coll_z, double* k_coll_vx, double* k_coll_vy,
                             double* k_coll_vz, double* k_coll_omegax, double* k_coll_omegay,
                             double* k_coll_omegaz);

  /* ---- output (src/system_print_output.cpp, system_print_particles.cpp,
          system_print_walls.cpp, system_print_colloids.cpp, system_print_macro_vars.cu,
          system_print_particles_gradv.cpp) ---- */
  void print_particles(double* k_x, double* k_y, double* k_z, double* k_vx, double* k_vy,
                       double* k_vz, double* k_mass, double* k_dens, double* k_press,
                       double* k_cxx, double* k_cxy, double* k_cyy, double* k_cxz,
                       double* k_cyz, double* k_czz, int step);
  void print_walls(double* k_fx_wall, double* k_fy_wall, double* k_fz_wall, int step);
  void print_colloids(double* k_coll_x, double* k_coll_y, double* k_coll_z, double* k_coll_vx,
                      double* k_coll_vy, double* k_coll_vz, double* k_coll_omegax,
                      double* k_coll_omegay, double* k_coll_omegaz, double* k_fx_colloid,
                      double* k_fy_colloid, double* k_fz_colloid, double* k_tx_colloid,
                      double* k_ty_colloid, double* k_tz_colloid, int step);
  void print_particles_gradv(double* k_x, double* k_y, double* k_z, double* k_gradvxx,
                             double* k_gradvxy, double* k_gradvxz, double* k_gradvyx,
                             double* k_gradvyy, double* k_gradvyz, double* k_gradvzx,
                             double* k_gradvzy, double* k_gradvzz, int step);
  void print_macro_vars(dim3 numBlocks, dim3 threadsPerBlock, double* k_mass, double* k_vx,
                        double* k_vy, double* k_vz, double* k_energy, int step);
  void print_output(dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y,
                    double* k_z, double* k_vx, double* k_vy, double* k_vz, double* k_fx,
                    double* k_fy, double* k_fz, double* k_mass, double* k_dens, double* k_press,
                    double* k_cxx, double* k_cxy, double* k_cyy, double* k_cxz, double* k_cyz,
                    double* k_czz, double* k_fx_wall, double* k_fy_wall, double* k_fz_wall,
                    double* k_coll_x, double* k_coll_y, double* k_coll_z, double* k_coll_vx,
                    double* k_coll_vy, double* k_coll_vz, double* k_coll_omegax,
                    double* k_coll_omegay, double* k_coll_omegaz, double* k_fx_colloid,
                    double* k_fy_colloid, double* k_fz_colloid, double* k_tx_colloid,
                    double* k_ty_colloid, double* k_tz_colloid, double* k_kin_energy,
                    int freq_micro, int freq_walls, int freq_colloids, int freq_macro,
                    int step);

  /* ---- additions (no reference counterpart) ---- */
  /* The engine context behind this object (NULL before initialize). */
  sph_ctx* engine() const;
  /* Copy the cell arrays of the last search into caller-owned DEVICE buffers (the
     k_particle_cell / k_particle_index / k_cell_start / k_cell_end of the reference). */
  int export_cells(int* k_particle_cell, int* k_particle_index, int* k_cell_start,
                   int* k_cell_end);

  /* Shim state: created by the first of read_input / initialize, released by destructor.
     The reference's driver declares `class_system sys;` and calls read_input first, so
     this is the one member with a default value. */
  class_system_engine* shim_ = nullptr;
};
