/* sph_io.h -- writers of the reference's text output files, byte-identical to its
 * fprintf("%.8lf") output (REAL_FMT of src/config.h:16 in the FP64 configuration), and a
 * lossless binary checkpoint.  Host code only: no GPU is needed.
 *
 * Rows are formatted on all host cores with an exact fixed-point formatter (the decimal
 * value of the binary double rounded half-to-even to 8 places, as glibc's printf does),
 * so writing a 2M-particle micro file takes a fraction of a second instead of the
 * reference's single fprintf loop.
 */
#ifndef SPH_IO_H
#define SPH_IO_H

#include "sph_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* micro-<step>.dat (src/system_print_particles.cpp:57-91): one row per particle
   "i x y [z] vx vy [vz] mass dens press type cxx cxy cyy [cxz cyz czz]"; 2D rows end
   with " \n", 3D rows with "\n".  z, vz, cxz, cyz, czz are not read in 2D. */
sph_status sph_write_micro(const char* path, int dim, int n, const double* x, const double* y,
                           const double* z, const double* vx, const double* vy,
                           const double* vz, const double* mass, const double* dens,
                           const double* press, const int* type, const double* cxx,
                           const double* cxy, const double* cyy, const double* cxz,
                           const double* cyz, const double* czz);

/* walls-<step>.dat (src/system_print_walls.cpp:32-44): "i fx fy [fz]" per wall. */
sph_status sph_write_walls(const char* path, int dim, int nwalls, const double* fx,
                           const double* fy, const double* fz);

/* colloids-<step>.dat (src/system_print_colloids.cpp:81-111):
   2D "i x y vx vy omegaz fx fy tz", 3D "i x y z vx vy vz ox oy oz fx fy fz tx ty tz".
   f holds the 15 columns in the 3D order (x, y, z, vx, vy, vz, omegax, omegay, omegaz,
   fx, fy, fz, tx, ty, tz); the 2D file uses the subset it prints. */
sph_status sph_write_colloids(const char* path, int dim, int n, const double* const* f);

/* gradv-<step>.dat (src/system_print_particles_gradv.cpp:48-83): 2D "i x y gxx gxy gyx
   gyy", 3D "i x y z gxx gxy gxz gyx gyy gyz gzx gzy gzz"; g holds the 9 components in
   that 3D order. */
sph_status sph_write_gradv(const char* path, int dim, int n, const double* x, const double* y,
                           const double* z, const double* const* g);

/* input_particles.in, the restart file that new_sim = 1 reads
   (src/system_initialize_particles_old_sim.cpp:36,48): 2D rows "x y vx vy mass type cxx
   cxy cyy", 3D rows "x y z vx vy vz mass type cxx cxy cyy cxz cyz czz", no index.  The
   reference reads every column as float, so every value is rounded to float and written
   with "%.9g", which reads back as exactly that float.  z, vz, cxz, cyz, czz are not read
   in 2D. */
sph_status sph_write_restart(const char* path, int dim, int n, const double* x, const double* y,
                             const double* z, const double* vx, const double* vy,
                             const double* vz, const double* mass, const int* type,
                             const double* cxx, const double* cxy, const double* cyy,
                             const double* cxz, const double* cyz, const double* czz);

/* macro.dat (src/system_print_macro_vars.cu:34-47): "step KE" with "%f"; the file is
   created at step 0 and appended to otherwise. */
sph_status sph_append_macro(const char* path, int step, double kin_energy);

/* Formats x as printf("%.8f", x) does into buf (at least 330 bytes: DBL_MAX prints 318
   characters); returns the length. */
int sph_format_fixed8(double x, char* buf);

/* Binary checkpoint of a context: every particle field, the particle types, the colloid
   state and the step counter, in original particle order, written bit-exactly (the
   reference's only restart path is the text file read through float,
   src/system_initialize_particles_old_sim.cpp:17-104).  sph_load_checkpoint restores it
   into a context created from the same input. */
sph_status sph_save_checkpoint(sph_ctx* ctx, const char* path);
sph_status sph_load_checkpoint(sph_ctx* ctx, const char* path);

#ifdef __cplusplus
}
#endif

#endif /* SPH_IO_H */
