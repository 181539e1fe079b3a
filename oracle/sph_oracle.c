/*
 * sph_oracle.c -- CPU FP64 oracle for the SPH Oldroyd-B / magnetic-colloid step.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load this library, and only as the checker or
 * as the timed CPU baseline.  The CUDA engine never calls into it.
 *
 * It restates, in plain C99 + OpenMP and in double precision, the algorithm of the
 * reference program (BCAM-CFD/SPH-magnetic-particles-Oldroyd-B-in-cuda, directory src/),
 * kernel by kernel, keeping the reference's data layout (SoA arrays indexed by the
 * original particle id), its neighbour-cell iteration order, its branch structure and
 * its quirks (stale cell ranges, clamp rules, the 3D magnetic |e| = R scaling, the
 * repulsion r^2 clamp, the 3D zero-omega NaN).  Every function cites the reference
 * file:line it follows.  Build with -ffp-contract=off so that no fused multiply-add is
 * introduced; the results then differ from the reference's FP64 CUDA build only by the
 * FMA contractions nvcc makes and by last-ulp differences of the CUDA math library.
 *
 * Quirk resolved by intent, not by reproduction: kernel_collect_force_colloids.cu:39-46
 * leaves the 2D torque accumulator uninitialised (undefined behaviour); here it starts
 * from the zeroed torque, which is what kernel_colloid_forces_to_zero.cu:25 intends.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_COLLOIDS 1000 /* config.h:22 */

/* ------------------------------------------------------------------------------------ */
/* Inputs: the keys of the reference's `input` file (system_read_input.cpp:102-269).     */
/* ------------------------------------------------------------------------------------ */
typedef struct orc_input {
  int Nxyz[3];
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
  double coll_xyz[ORC_MAX_COLLOIDS][3];
  int coll_move;
  double coll_rep_cuton, F0_repulsion, tau_repulsion, cutoff_magnetic, F0_magnetic,
      omega_magnetic;
  int new_sim;
} orc_input;

/* ------------------------------------------------------------------------------------ */
/* System: the fields of class_system (class_system.h:12-143).                          */
/* ------------------------------------------------------------------------------------ */
typedef struct orc_sys {
  orc_input in;
  int N, Nmax, dim, wall;
  double L[3];
  double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *dens, *press, *mass;
  int* type;
  double *cxx, *cxy, *cyy, *cxz, *cyz, *czz;
  double *dcdt_xx, *dcdt_xy, *dcdt_yy, *dcdt_xz, *dcdt_yz, *dcdt_zz;
  double *gxx, *gxy, *gxz, *gyx, *gyy, *gyz, *gzx, *gzy, *gzz;
  double nkT, tau;
  double y_bottom, y_top, V_bottom, V_top;
  int Nwalls, Nlist_walls;
  int *walls_list, *walls_start;
  double fx_wall[2], fy_wall[2], fz_wall[2];
  double wall_width;
  int N_colloids, Nlist_colloids;
  double coll_R, coll_rho, coll_mass, coll_I;
  int *colloids_list, *colloids_start;
  double *coll_x, *coll_y, *coll_z, *coll_vx, *coll_vy, *coll_vz;
  double *coll_omegax, *coll_omegay, *coll_omegaz, *coll_theta;
  double *coll_quat0, *coll_quatx, *coll_quaty, *coll_quatz;
  double *x_center, *y_center, *z_center;
  double *fx_colloid, *fy_colloid, *fz_colloid, *tx_colloid, *ty_colloid, *tz_colloid;
  double coll_rep_cuton, coll_rep_cutoff, rcuton_coll_rep, rcutoff_coll_rep;
  double rcuton_coll_rep_sq, rcutoff_coll_rep_sq, rcutoff_coll, rcutoff_coll_sq;
  double F0_rep, tau_rep, r0_magnet, r0_magnet_sq, F0_magnet, omega_magnet;
  double rcut, rcutsq, rcut_inv, cw, c_gradw, c, csq, rho, P0, rho0, a, b;
  double cell_size[3];
  int Ncells[3], Ntotal_cells;
  double cell_colloids_size[3];
  int Ncells_colloids[3], Ntotal_cells_colloids;
  int ext_force_type;
  double ext_force[3], ky;
  double beta_max;
  /* neighbour search state (device arrays of the reference) */
  int *particle_cell, *particle_index, *cell_start, *cell_end;
  int *coll_cell, *coll_index, *coll_cell_start, *coll_cell_end;
  double magnetic_mom[3];
  int step;    /* steps completed by orc_run */
  int started; /* initial search + forces done */
  int bad_cell; /* set when the hash leaves the grid (kernel_cell_ranges.cu:20-23) */
} orc_sys;

/* ------------------------------------------------------------------------------------ */
/* Input parser: system_read_input.cpp:18-512                                            */
/* ------------------------------------------------------------------------------------ */
static void orc_fail(char* msg, size_t cap, const char* text) {
  if (msg && cap) {
    strncpy(msg, text, cap - 1);
    msg[cap - 1] = 0;
  }
}

int orc_read_input(const char* path, orc_input* in, char* msg, size_t cap) {
  memset(in, 0, sizeof(*in));
  FILE* f = fopen(path, "r");
  if (!f) {
    orc_fail(msg, cap, "input file cannot be opened");
    return 1;
  }
  enum { K_N, K_L, K_DIM, K_DT, K_T0, K_NSTEPS, K_OVERLAP, K_RHO, K_C, K_P0, K_ETA, K_ZETA,
         K_NP, K_KT, K_TAU, K_EFT, K_EF, K_FMI, K_FMA, K_FW, K_FC, K_WALL, K_VWT, K_VWB,
         K_NC, K_CR, K_CRHO, K_CMOVE, K_CUTON, K_F0R, K_TAUR, K_CUTM, K_F0M, K_OMM, K_NEW,
         K_COUNT };
  static const char* names[K_COUNT] = {
      "N", "L", "dim", "dt", "t0", "Nsteps", "overlap", "rho", "c", "P0", "eta", "zeta",
      "np", "kT", "tau", "ext_force_type", "ext_force", "freq_micro", "freq_macro",
      "freq_walls", "freq_colloids", "wall", "Vwall_top", "Vwall_bottom", "N_colloids",
      "coll_R", "coll_rho", "coll_move", "coll_repulsion_cuton", "F0_repulsion",
      "tau_repulsion", "cutoff_magnetic", "F0_magnetic", "omega_magnetic", "new_sim"};
  int seen[K_COUNT];
  memset(seen, 0, sizeof(seen));
  int dim_N = 0, dim_L = 0, dim_ef = 0, ncx = 0;
  char line[1024];
  char var[512];
  var[0] = 0;
  while (fgets(line, sizeof(line), f)) {
    char* s = line;
    while (*s == ' ' || *s == '\t') s++;
    char* e = s + strlen(s) - 1;
    while (e > s && (*e == ' ' || *e == '\t' || *e == '\n')) *e-- = 0;
    double v1 = 0, v2 = 0, v3 = 0;
    int n = sscanf(s, "%511s %lf %lf %lf", var, &v1, &v2, &v3);
    int k;
    for (k = 0; k < K_COUNT; ++k)
      if (strcmp(var, names[k]) == 0) break;
    if (k == K_N && (n == 4 || n == 3)) {
      in->Nxyz[0] = (int)v1;
      in->Nxyz[1] = (int)v2;
      if (n == 4) in->Nxyz[2] = (int)v3;
      dim_N = n - 1;
      seen[k] = 1;
    } else if (k == K_L && (n == 4 || n == 3)) {
      in->L[0] = v1;
      in->L[1] = v2;
      if (n == 4) in->L[2] = v3;
      dim_L = n - 1;
      seen[k] = 1;
    } else if (k == K_EF && (n == 4 || n == 3)) {
      in->ext_force[0] = v1;
      in->ext_force[1] = v2;
      if (n == 4) in->ext_force[2] = v3;
      dim_ef = n - 1;
      seen[k] = 1;
    } else if (k < K_COUNT && k != K_N && k != K_L && k != K_EF && n >= 2) {
      seen[k] = 1;
      switch (k) {
        case K_DIM: in->dim = (int)v1; break;
        case K_DT: in->dt = v1; break;
        case K_T0: in->t0 = v1; break;
        case K_NSTEPS: in->Nsteps = (int)v1; break;
        case K_OVERLAP: in->overlap = v1; break;
        case K_RHO: in->rho = v1; break;
        case K_C: in->c = v1; break;
        case K_P0: in->P0 = v1; break;
        case K_ETA: in->eta = v1; break;
        case K_ZETA: in->zeta = v1; break;
        case K_NP: in->np = v1; break;
        case K_KT: in->kT = v1; break;
        case K_TAU: in->tau = v1; break;
        case K_EFT: in->ext_force_type = (int)v1; break;
        case K_FMI: in->freq_micro = (int)v1; break;
        case K_FMA: in->freq_macro = (int)v1; break;
        case K_FW: in->freq_walls = (int)v1; break;
        case K_FC: in->freq_colloids = (int)v1; break;
        case K_WALL: in->wall = (int)v1; break;
        case K_VWT: in->Vwall_top = v1; break;
        case K_VWB: in->Vwall_bottom = v1; break;
        case K_NC: in->N_colloids = (int)v1; break;
        case K_CR: in->coll_R = v1; break;
        case K_CRHO: in->coll_rho = v1; break;
        case K_CMOVE: in->coll_move = (int)v1; break;
        case K_CUTON: in->coll_rep_cuton = v1; break;
        case K_F0R: in->F0_repulsion = v1; break;
        case K_TAUR: in->tau_repulsion = v1; break;
        case K_CUTM: in->cutoff_magnetic = v1; break;
        case K_F0M: in->F0_magnetic = v1; break;
        case K_OMM: in->omega_magnetic = v1; break;
        case K_NEW: in->new_sim = (int)v1; break;
        default: break;
      }
    } else if (strcmp(var, "coll_x") == 0 && n >= 3 && in->N_colloids > 0) {
      /* system_read_input.cpp:243-268: tokens split on single spaces */
      if (ncx >= in->N_colloids || ncx >= ORC_MAX_COLLOIDS) {
        fclose(f);
        orc_fail(msg, cap, "different coll_x entries than N_colloids");
        return 1;
      }
      int nv = 0;
      for (char* t = strtok(s, " "); t; t = strtok(NULL, " ")) {
        if (strcmp(t, "coll_x") != 0) {
          if (nv < 3) in->coll_xyz[ncx][nv] = atof(t);
          nv++;
        }
      }
      if (nv != in->dim) {
        fclose(f);
        orc_fail(msg, cap, "coll_x dimension differs from dim");
        return 1;
      }
      ncx++;
    }
  }
  fclose(f);
  for (int k = 0; k < K_COUNT; ++k)
    if (!seen[k]) {
      char buf[128];
      snprintf(buf, sizeof(buf), "%s was not read", names[k]);
      orc_fail(msg, cap, buf);
      return 1;
    }
  /* system_read_input.cpp:412-438 */
  if (ncx != in->N_colloids) { orc_fail(msg, cap, "coll_x count != N_colloids"); return 1; }
  if (in->dim != dim_N) { orc_fail(msg, cap, "dim incompatible with N"); return 1; }
  if (in->dim != dim_L) { orc_fail(msg, cap, "dim incompatible with L"); return 1; }
  if (in->ext_force_type != 0 && in->dim != dim_ef) {
    orc_fail(msg, cap, "dim incompatible with ext_force");
    return 1;
  }
  if (in->ext_force_type < 0 || in->ext_force_type > 3) {
    orc_fail(msg, cap, "ext_force_type not available");
    return 1;
  }
  if (in->N_colloids > ORC_MAX_COLLOIDS) { orc_fail(msg, cap, "N_colloids too high"); return 1; }
  /* system_read_input.cpp:441-456: colloids inside the box (only checked for >= 2) */
  int nc = in->N_colloids;
  if (nc >= 2)
    for (int i = 0; i < nc; ++i)
      for (int d = 0; d < in->dim; ++d)
        if (in->coll_xyz[i][d] < 0 || in->coll_xyz[i][d] > in->L[d]) {
          orc_fail(msg, cap, "colloid out of the simulation box");
          return 1;
        }
  /* system_read_input.cpp:459-506: overlap check; the 3D branch takes z from y (:485) */
  if (nc >= 2)
    for (int i = 0; i < nc; ++i)
      for (int j = i + 1; j < nc; ++j) {
        double xij = in->coll_xyz[i][0] - in->coll_xyz[j][0];
        double yij = in->coll_xyz[i][1] - in->coll_xyz[j][1];
        double zij = (in->dim == 3) ? in->coll_xyz[i][1] - in->coll_xyz[j][1] : 0.0;
        if (xij > 0.5 * in->L[0]) xij -= in->L[0];
        if (xij < -0.5 * in->L[0]) xij += in->L[0];
        if (in->wall == 0) {
          if (yij > 0.5 * in->L[1]) yij -= in->L[1];
          if (yij < -0.5 * in->L[1]) yij += in->L[1];
        }
        double r2 = xij * xij + yij * yij;
        if (in->dim == 3) {
          if (zij > 0.5 * in->L[2]) zij -= in->L[2];
          if (zij < -0.5 * in->L[2]) zij += in->L[2];
          r2 = xij * xij + yij * yij + zij * zij;
        }
        if (sqrt(r2) < 2 * in->coll_R) { orc_fail(msg, cap, "overlapping colloids"); return 1; }
      }
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Allocation helpers                                                                    */
/* ------------------------------------------------------------------------------------ */
static double* dal(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
static int* ial(size_t n) { return (int*)calloc(n ? n : 1, sizeof(int)); }

static void orc_alloc_particles(orc_sys* s, int n) {
  double** dptr[] = {&s->x, &s->y, &s->z, &s->vx, &s->vy, &s->vz, &s->fx, &s->fy, &s->fz,
                     &s->dens, &s->press, &s->mass, &s->cxx, &s->cxy, &s->cyy, &s->cxz,
                     &s->cyz, &s->czz};
  for (size_t k = 0; k < sizeof(dptr) / sizeof(dptr[0]); ++k) {
    free(*dptr[k]);
    *dptr[k] = dal(n);
  }
  free(s->type);
  s->type = ial(n);
}

void orc_destroy(orc_sys* s) {
  if (!s) return;
  void* p[] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->dens,
               s->press, s->mass, s->type, s->cxx, s->cxy, s->cyy, s->cxz, s->cyz, s->czz,
               s->dcdt_xx, s->dcdt_xy, s->dcdt_yy, s->dcdt_xz, s->dcdt_yz, s->dcdt_zz,
               s->gxx, s->gxy, s->gxz, s->gyx, s->gyy, s->gyz, s->gzx, s->gzy, s->gzz,
               s->walls_list, s->walls_start, s->colloids_list, s->colloids_start,
               s->coll_x, s->coll_y, s->coll_z, s->coll_vx, s->coll_vy, s->coll_vz,
               s->coll_omegax, s->coll_omegay, s->coll_omegaz, s->coll_theta,
               s->coll_quat0, s->coll_quatx, s->coll_quaty, s->coll_quatz, s->x_center,
               s->y_center, s->z_center, s->fx_colloid, s->fy_colloid, s->fz_colloid,
               s->tx_colloid, s->ty_colloid, s->tz_colloid, s->particle_cell,
               s->particle_index, s->cell_start, s->cell_end, s->coll_cell, s->coll_index,
               s->coll_cell_start, s->coll_cell_end};
  for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); ++k) free(p[k]);
  free(s);
}

/* ------------------------------------------------------------------------------------ */
/* Particle initialisation, new simulation: system_initialize_particles_new_sim.cpp:16-253 */
/* ------------------------------------------------------------------------------------ */
static int orc_particles_new_sim(orc_sys* s, const int Nxyz[3], const double dx[3]) {
  int counter = 0;
  const double* L = s->L;
  double R2 = s->coll_R * s->coll_R;
  int nk = (s->dim == 3) ? Nxyz[2] : 1;
  for (int i = 0; i < Nxyz[0]; ++i)
    for (int j = 0; j < Nxyz[1]; ++j)
      for (int k = 0; k < nk; ++k) {
        s->x[counter] = dx[0] / 2.0 + i * dx[0];
        s->y[counter] = dx[1] / 2.0 + j * dx[1];
        if (s->wall) s->y[counter] = s->y[counter] - s->wall_width;
        if (s->dim == 3) s->z[counter] = dx[2] / 2.0 + k * dx[2];
        int inside = 0;
        for (int l = 0; l < s->N_colloids && !inside; ++l) {
          double xij = s->x[counter] - s->coll_x[l];
          double yij = s->y[counter] - s->coll_y[l];
          if (xij > 0.5 * L[0]) xij -= L[0];
          if (xij < -0.5 * L[0]) xij += L[0];
          if (s->wall == 0) {
            if (yij > 0.5 * L[1]) yij -= L[1];
            if (yij < -0.5 * L[1]) yij += L[1];
          }
          double r2 = xij * xij + yij * yij;
          if (s->dim == 3) {
            double zij = s->z[counter] - s->coll_z[l];
            if (zij > 0.5 * L[2]) zij -= L[2];
            if (zij < -0.5 * L[2]) zij += L[2];
            r2 = xij * xij + yij * yij + zij * zij;
          }
          inside = (r2 <= R2);
        }
        if (!inside) counter++;
      }
  s->N = counter;
  for (int i = 0; i < s->N; ++i) {
    if (s->wall == 0)
      s->type[i] = 0;
    else
      s->type[i] = (s->y[i] < s->y_bottom) ? 1 : ((s->y[i] > s->y_top) ? 2 : 0);
    s->vx[i] = s->vy[i] = s->vz[i] = 0.0;
    s->fx[i] = s->fy[i] = s->fz[i] = 0.0;
    if (s->dim == 2)
      s->mass[i] = s->rho * L[0] * (L[1] + 2.0 * s->wall_width) / (Nxyz[0] * Nxyz[1]);
    else
      s->mass[i] = s->rho * L[0] * (L[1] + 2.0 * s->wall_width) * L[2] /
                   (Nxyz[0] * Nxyz[1] * Nxyz[2]);
    s->cxx[i] = 1.0; s->cxy[i] = 0.0; s->cyy[i] = 1.0;
    s->cxz[i] = 0.0; s->cyz[i] = 0.0; s->czz[i] = 1.0;
  }
  /* colloid shells: :143-249 */
  int Nlayers = (int)round(s->coll_R / dx[0]);
  for (int c = 0; c < s->N_colloids; ++c) {
    double r = 0.5 * dx[0];
    for (int j = 0; j < Nlayers; ++j) {
      if (r < s->coll_R && r > s->coll_R - s->wall_width) {
        if (s->dim == 2) {
          double d_phi = dx[0] / r;
          int Nphi = (int)round(2.0 * M_PI / d_phi);
          d_phi = 2.0 * M_PI / Nphi;
          double phi = 0.0;
          for (int k = 0; k < Nphi; ++k) {
            if (s->N + 1 > s->Nmax) return 1;
            int p = s->N++;
            s->x[p] = s->coll_x[c] + r * cos(phi);
            s->y[p] = s->coll_y[c] + r * sin(phi);
            s->type[p] = 3 + c;
            if (s->x[p] < 0) s->x[p] = s->x[p] + L[0];
            if (s->wall == 0 && s->y[p] < 0) s->y[p] = s->y[p] + L[1];
            if (s->x[p] > L[0]) s->x[p] = s->x[p] - L[0];
            if (s->wall == 0 && s->y[p] > L[1]) s->y[p] = s->y[p] - L[1];
            phi = phi + d_phi;
          }
        } else {
          if (s->N + 1 > s->Nmax) return 1;
          int p = s->N++; /* north pole, :189-197 */
          s->x[p] = s->coll_x[c];
          s->y[p] = s->coll_y[c];
          s->z[p] = s->coll_z[c] + r;
          s->type[p] = 3 + c;
          double d_theta = dx[0] / r;
          int Ntheta = (int)round(M_PI / d_theta);
          d_theta = M_PI / Ntheta;
          double theta = 0.0;
          for (int k = 0; k < Ntheta; ++k) {
            double d_phi = dx[0] / (r * sin(theta));
            int Nphi = (int)round(2.0 * M_PI / d_phi);
            d_phi = 2.0 * M_PI / Nphi;
            double phi = 0.0;
            for (int l = 0; l < Nphi; ++l) {
              /* the reference performs no Nmax check here (:210-236); we refuse instead of
                 writing past the end */
              if (s->N + 1 > s->Nmax) return 1;
              p = s->N++;
              s->x[p] = s->coll_x[c] + r * sin(theta) * cos(phi);
              s->y[p] = s->coll_y[c] + r * sin(theta) * sin(phi);
              s->z[p] = s->coll_z[c] + r * cos(theta);
              s->type[p] = 3 + c;
              if (s->x[p] < 0) s->x[p] = s->x[p] + L[0];
              if (s->wall == 0 && s->y[p] < 0) s->y[p] = s->y[p] + L[1];
              if (s->z[p] < 0) s->z[p] = s->z[p] + L[2];
              if (s->x[p] > L[0]) s->x[p] = s->x[p] - L[0];
              if (s->wall == 0 && s->y[p] > L[1]) s->y[p] = s->y[p] - L[1];
              if (s->z[p] > L[2]) s->z[p] = s->z[p] - L[2];
              phi = phi + d_phi;
            }
            theta = theta + d_theta;
          }
          if (s->N + 1 > s->Nmax) return 1;
          p = s->N++; /* south pole, :240-244 */
          s->x[p] = s->coll_x[c];
          s->y[p] = s->coll_y[c];
          s->z[p] = s->coll_z[c] - r;
          s->type[p] = 3 + c;
        }
      }
      r = r + dx[0];
    }
  }
  /* Colloid shell particles get no velocity, mass or conformation values: the reference
     fills those only for the lattice particles (:115-140) and leaves the shell slots of
     its new real[] arrays unwritten, which on a fresh heap are zero pages.  Here they are
     explicitly zero (calloc): v = 0, mass = 0 and c = 0, not the identity. */
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Restart reader: system_initialize_particles_old_sim.cpp:17-112 (values parsed as float) */
/* ------------------------------------------------------------------------------------ */
static int orc_particles_old_sim(orc_sys* s, const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return 1;
  int ncol = (s->dim == 2) ? 9 : 14;
  size_t cap = 1024, n = 0;
  float* buf = (float*)malloc(cap * ncol * sizeof(float));
  float v[14];
  for (;;) {
    int ok = 1;
    for (int k = 0; k < ncol && ok; ++k) ok = (fscanf(f, "%f", &v[k]) == 1);
    if (!ok) break;
    if (n == cap) {
      cap *= 2;
      buf = (float*)realloc(buf, cap * ncol * sizeof(float));
    }
    memcpy(buf + n * ncol, v, ncol * sizeof(float));
    n++;
  }
  fclose(f);
  s->N = s->Nmax = (int)n;
  orc_alloc_particles(s, (int)n);
  for (size_t i = 0; i < n; ++i) {
    float* r = buf + i * ncol;
    if (s->dim == 2) {
      s->x[i] = r[0]; s->y[i] = r[1]; s->vx[i] = r[2]; s->vy[i] = r[3];
      s->mass[i] = r[4]; s->type[i] = (int)r[5];
      s->cxx[i] = r[6]; s->cxy[i] = r[7]; s->cyy[i] = r[8];
    } else {
      s->x[i] = r[0]; s->y[i] = r[1]; s->z[i] = r[2];
      s->vx[i] = r[3]; s->vy[i] = r[4]; s->vz[i] = r[5];
      s->mass[i] = r[6]; s->type[i] = (int)r[7];
      s->cxx[i] = r[8]; s->cxy[i] = r[9]; s->cyy[i] = r[10];
      s->cxz[i] = r[11]; s->cyz[i] = r[12]; s->czz[i] = r[13];
    }
  }
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Constructor + initialize: system_constructor.cpp:15-108, system_initialize.cpp:16-359 */
/* ------------------------------------------------------------------------------------ */
orc_sys* orc_create(const orc_input* in, const char* particles_path, char* msg, size_t cap) {
  orc_sys* s = (orc_sys*)calloc(1, sizeof(orc_sys));
  s->in = *in;
  s->dim = in->dim;
  s->wall = in->wall;
  int Nxyz[3] = {in->Nxyz[0], in->Nxyz[1], in->Nxyz[2]};
  int dim = in->dim;
  /* constructor */
  s->Nwalls = in->wall ? 2 : 0;
  int nc = in->N_colloids;
  s->coll_x = dal(nc); s->coll_y = dal(nc); s->coll_z = dal(nc);
  s->coll_vx = dal(nc); s->coll_vy = dal(nc); s->coll_vz = dal(nc);
  s->coll_omegax = dal(nc); s->coll_omegay = dal(nc); s->coll_omegaz = dal(nc);
  s->coll_theta = dal(nc); s->coll_quat0 = dal(nc); s->coll_quatx = dal(nc);
  s->coll_quaty = dal(nc); s->coll_quatz = dal(nc);
  s->fx_colloid = dal(nc); s->fy_colloid = dal(nc); s->fz_colloid = dal(nc);
  s->tx_colloid = dal(nc); s->ty_colloid = dal(nc); s->tz_colloid = dal(nc);
  if (in->new_sim == 0) {
    int Ny = in->wall ? Nxyz[1] + 2 * (int)ceil(in->overlap) : Nxyz[1];
    int N = (dim == 2) ? Nxyz[0] * Ny : Nxyz[0] * Ny * Nxyz[2];
    if (nc > 0) N = (int)(N * 1.01);
    s->N = s->Nmax = N;
    orc_alloc_particles(s, N);
  }
  /* initialize */
  for (int d = 0; d < 3; ++d) s->L[d] = in->L[d];
  s->V_top = in->Vwall_top;
  s->V_bottom = in->Vwall_bottom;
  s->nkT = in->np * in->kT;
  s->tau = in->tau;
  s->rcut = in->L[0] / Nxyz[0] * in->overlap;
  s->rcutsq = s->rcut * s->rcut;
  s->rcut_inv = 1.0 / s->rcut;
  double dx[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) dx[d] = in->L[d] / Nxyz[d];
  s->ky = 2.0 * M_PI / in->L[1];
  double eps = 1.0e-10;
  if (fabs(in->overlap - floor(in->overlap)) < eps)
    s->wall_width = floor(in->overlap) * dx[1];
  else
    s->wall_width = (floor(in->overlap) + 1) * dx[1];
  if (in->wall == 1) {
    Nxyz[1] = Nxyz[1] + 2 * (int)ceil(in->overlap);
    s->y_bottom = 0.0;
    s->y_top = in->L[1];
  }
  if (dim == 2)
    s->cw = 63.0 / (478.0 * M_PI * s->rcut * s->rcut);
  else
    s->cw = 27.0 / (120.0 * M_PI * s->rcut * s->rcut * s->rcut);
  s->c_gradw = -15.0 * s->cw / s->rcut;
  s->rho = in->rho;
  s->c = in->c;
  s->csq = in->c * in->c;
  s->P0 = in->P0;
  s->rho0 = in->P0 * in->rho;
  s->a = 5.0 * in->eta / 3.0 - in->zeta;
  s->b = (dim == 3) ? 5.0 * (in->zeta + in->eta / 3.0) : 4.0 * (in->zeta + in->eta / 3.0);
  s->beta_max = 1.5;
  s->Ncells[0] = (int)(in->L[0] / s->rcut);
  s->cell_size[0] = in->L[0] / s->Ncells[0];
  if (in->wall == 1) {
    s->Ncells[1] = (int)((in->L[1] + 2 * s->wall_width) / s->rcut);
    s->cell_size[1] = (in->L[1] + 2 * s->wall_width) / s->Ncells[1];
  } else {
    s->Ncells[1] = (int)(in->L[1] / s->rcut);
    s->cell_size[1] = in->L[1] / s->Ncells[1];
  }
  if (dim == 3) {
    s->Ncells[2] = (int)(in->L[2] / s->rcut);
    s->cell_size[2] = in->L[2] / s->Ncells[2];
  } else {
    s->Ncells[2] = 1;
    s->cell_size[2] = 1;
  }
  s->Ntotal_cells = s->Ncells[0] * s->Ncells[1] * s->Ncells[2];
  if (s->Ncells[0] < 3 || s->Ncells[1] < 3 || (dim == 3 && s->Ncells[2] < 3)) {
    orc_fail(msg, cap, "neighbour cells are too big");
    orc_destroy(s);
    return NULL;
  }
  s->ext_force_type = in->ext_force_type;
  s->ext_force[0] = in->ext_force[0];
  s->ext_force[1] = in->ext_force[1];
  if (dim == 3) s->ext_force[2] = in->ext_force[2];
  /* colloids: :155-262 */
  s->N_colloids = nc;
  s->coll_R = in->coll_R;
  s->coll_rho = in->coll_rho;
  s->F0_rep = in->F0_repulsion;
  s->tau_rep = in->tau_repulsion;
  s->coll_rep_cuton = in->coll_rep_cuton;
  s->coll_rep_cutoff = 5.0 * s->coll_R / s->tau_rep;
  s->r0_magnet = in->cutoff_magnetic;
  s->r0_magnet_sq = in->cutoff_magnetic * in->cutoff_magnetic;
  s->F0_magnet = in->F0_magnetic;
  s->omega_magnet = in->omega_magnetic;
  if (dim == 2) {
    s->coll_mass = M_PI * s->coll_R * s->coll_R * s->coll_rho;
    s->coll_I = 0.5 * s->coll_mass * s->coll_R * s->coll_R;
  } else {
    s->coll_mass = 4.0 / 3.0 * M_PI * s->coll_R * s->coll_R * s->coll_R * s->coll_rho;
    s->coll_I = 2.0 / 5.0 * s->coll_mass * s->coll_R * s->coll_R;
  }
  for (int i = 0; i < nc; ++i) {
    s->coll_x[i] = in->coll_xyz[i][0];
    s->coll_y[i] = in->coll_xyz[i][1];
    if (dim == 3) s->coll_z[i] = in->coll_xyz[i][2];
    s->coll_quat0[i] = 1.0;
    if (in->wall) {
      if (s->coll_y[i] - s->coll_R < s->y_bottom || s->coll_y[i] + s->coll_R > s->y_top) {
        orc_fail(msg, cap, "colloid overlapping a wall");
        orc_destroy(s);
        return NULL;
      }
    }
  }
  if (nc > 0) {
    s->rcuton_coll_rep = 2.0 * s->coll_R + s->coll_rep_cuton;
    s->rcuton_coll_rep_sq = s->rcuton_coll_rep * s->rcuton_coll_rep;
    s->rcutoff_coll_rep = 2.0 * s->coll_R + s->coll_rep_cutoff;
    s->rcutoff_coll_rep_sq = s->rcutoff_coll_rep * s->rcutoff_coll_rep;
    s->rcutoff_coll = (s->rcutoff_coll_rep > s->r0_magnet) ? s->rcutoff_coll_rep : s->r0_magnet;
    s->rcutoff_coll_sq = s->rcutoff_coll * s->rcutoff_coll;
    for (int d = 0; d < 2; ++d) {
      s->Ncells_colloids[d] = (int)(in->L[d] / s->rcutoff_coll);
      s->cell_colloids_size[d] = in->L[d] / s->Ncells_colloids[d];
    }
    if (dim == 3) {
      s->Ncells_colloids[2] = (int)(in->L[2] / s->rcutoff_coll);
      s->cell_colloids_size[2] = in->L[2] / s->Ncells_colloids[2];
    } else {
      s->Ncells_colloids[2] = 1;
      s->cell_colloids_size[2] = 1;
    }
    s->Ntotal_cells_colloids =
        s->Ncells_colloids[0] * s->Ncells_colloids[1] * s->Ncells_colloids[2];
    if (s->Ncells_colloids[0] < 3 || s->Ncells_colloids[1] < 3 ||
        (dim == 3 && s->Ncells_colloids[2] < 3)) {
      orc_fail(msg, cap, "neighbour colloids cells are too big");
      orc_destroy(s);
      return NULL;
    }
  }
  int err = (in->new_sim == 0) ? orc_particles_new_sim(s, Nxyz, dx)
                               : orc_particles_old_sim(s, particles_path ? particles_path
                                                                         : "input_particles.in");
  if (err) {
    orc_fail(msg, cap, in->new_sim == 0 ? "N > Nmax while building colloid shells"
                                        : "restart particle file cannot be read");
    orc_destroy(s);
    return NULL;
  }
  /* walls_list: system_initialize.cpp:278-300 */
  if (in->wall) {
    s->walls_start = ial(2);
    s->Nlist_walls = 0;
    for (int i = 0; i < s->N; ++i)
      if (s->type[i] == 1 || s->type[i] == 2) s->Nlist_walls++;
    s->walls_list = ial(s->Nlist_walls);
    int counter = 0;
    for (int w = 0; w < 2; ++w) {
      int ci = 0;
      for (int j = 0; j < s->N; ++j)
        if (s->type[j] == w + 1) {
          s->walls_list[counter] = j;
          if (ci == 0) s->walls_start[w] = counter;
          ci++;
          counter++;
        }
    }
  }
  /* colloids_list and body-frame offsets: system_initialize.cpp:304-355 */
  if (nc > 0) {
    s->colloids_start = ial(nc);
    s->Nlist_colloids = 0;
    for (int i = 0; i < s->N; ++i)
      if (s->type[i] > 2) s->Nlist_colloids++;
    s->colloids_list = ial(s->Nlist_colloids);
    int counter = 0;
    for (int c = 0; c < nc; ++c) {
      int ci = 0;
      for (int j = 0; j < s->N; ++j)
        if (s->type[j] == c + 3) {
          s->colloids_list[counter] = j;
          if (ci == 0) s->colloids_start[c] = counter;
          ci++;
          counter++;
        }
    }
    int nl = s->Nlist_colloids;
    s->x_center = dal(nl); s->y_center = dal(nl); s->z_center = dal(nl);
    for (int i = 0; i < nl; ++i) {
      int p = s->colloids_list[i];
      int c = s->type[p] - 3;
      s->x_center[i] = s->x[p] - s->coll_x[c];
      s->y_center[i] = s->y[p] - s->coll_y[c];
      if (dim == 3) s->z_center[i] = s->z[p] - s->coll_z[c];
      if (s->x_center[i] > 0.5 * s->L[0]) s->x_center[i] -= s->L[0];
      if (s->x_center[i] < -0.5 * s->L[0]) s->x_center[i] += s->L[0];
      if (s->wall == 0) {
        if (s->y_center[i] > 0.5 * s->L[1]) s->y_center[i] -= s->L[1];
        if (s->y_center[i] < -0.5 * s->L[1]) s->y_center[i] += s->L[1];
      }
      if (dim == 3) {
        if (s->z_center[i] > 0.5 * s->L[2]) s->z_center[i] -= s->L[2];
        if (s->z_center[i] < -0.5 * s->L[2]) s->z_center[i] += s->L[2];
      }
    }
  }
  /* device-side arrays of copy_pointers_to_device (system_copy_pointers_to_device.cpp:207-266),
     all zeroed by cudaMemset there */
  int N = s->N;
  s->dcdt_xx = dal(N); s->dcdt_xy = dal(N); s->dcdt_yy = dal(N);
  s->dcdt_xz = dal(N); s->dcdt_yz = dal(N); s->dcdt_zz = dal(N);
  s->gxx = dal(N); s->gxy = dal(N); s->gxz = dal(N); s->gyx = dal(N); s->gyy = dal(N);
  s->gyz = dal(N); s->gzx = dal(N); s->gzy = dal(N); s->gzz = dal(N);
  for (int i = 0; i < N; ++i) {
    s->fx[i] = s->fy[i] = s->fz[i] = 0.0;
    s->dens[i] = s->press[i] = 0.0;
  }
  s->particle_cell = ial(N);
  s->particle_index = ial(N);
  s->cell_start = ial(s->Ntotal_cells);
  s->cell_end = ial(s->Ntotal_cells);
  s->coll_cell = ial(nc);
  s->coll_index = ial(nc);
  s->coll_cell_start = ial(s->Ntotal_cells_colloids);
  s->coll_cell_end = ial(s->Ntotal_cells_colloids);
  double ang = s->omega_magnet * in->t0;
  s->magnetic_mom[0] = cos(ang);
  s->magnetic_mom[1] = sin(ang);
  s->magnetic_mom[2] = 0.0;
  return s;
}

/* ------------------------------------------------------------------------------------ */
/* SPH kernel and gradient: kernel_W.cu:13-59, kernel_gradW.cu:13-53                      */
/* ------------------------------------------------------------------------------------ */
double orc_W(const orc_sys* s, double r) {
  double q = r * s->rcut_inv;
  double q3 = q * 3.0;
  double t1 = 3.0 - q3, t1_2 = t1 * t1, t1_5 = t1_2 * t1_2 * t1;
  if (q3 < 1.0) {
    double t2 = 2.0 - q3, t2_2 = t2 * t2, t2_5 = 6.0 * (t2_2 * t2_2 * t2);
    double t3 = 1.0 - q3, t3_2 = t3 * t3, t3_5 = 15.0 * (t3_2 * t3_2 * t3);
    double w = t1_5 - t2_5;
    w = w + t3_5;
    return s->cw * w;
  } else if (q3 < 2.0) {
    double t2 = 2.0 - q3, t2_2 = t2 * t2, t2_5 = 6.0 * (t2_2 * t2_2 * t2);
    return s->cw * (t1_5 - t2_5);
  }
  return s->cw * t1_5;
}

double orc_gradW(const orc_sys* s, double r) {
  double q = r * s->rcut_inv;
  double q3 = 3.0 * q;
  double t1 = 3.0 - q3, t1_2 = t1 * t1, t1_4 = t1_2 * t1_2;
  if (q3 < 1.0) {
    double t2 = 2.0 - q3, t2_2 = t2 * t2, t2_4 = 6.0 * (t2_2 * t2_2);
    double t3 = 1.0 - q3, t3_2 = t3 * t3, t3_4 = 15.0 * (t3_2 * t3_2);
    double g = t1_4 - t2_4;
    g = g + t3_4;
    return s->c_gradw * g;
  } else if (q3 < 2.0) {
    double t2 = 2.0 - q3, t2_2 = t2 * t2, t2_4 = 6.0 * (t2_2 * t2_2);
    return s->c_gradw * (t1_4 - t2_4);
  }
  return s->c_gradw * t1_4;
}

/* ------------------------------------------------------------------------------------ */
/* Neighbour search: system_neighbours_search.cu:19-110 + kernel_cell_list.cu:15-63,      */
/* kernel_cell_ranges.cu:13-33, kernel_cell_colloids_*.cu, kernel_initialize_cell_colloids */
/* ------------------------------------------------------------------------------------ */
static void orc_stable_sort_by_cell(int n, int* cell, int* index) {
  /* thrust::sort_by_key on int keys is a stable radix sort; with index = iota the
     result is the (cell, id) order.  A counting sort gives the same permutation.
     Out-of-range keys are sorted too, as the reference sorts them before it checks. */
  if (n <= 0) return;
  int lo = cell[0], hi = cell[0];
  for (int i = 1; i < n; ++i) {
    if (cell[i] < lo) lo = cell[i];
    if (cell[i] > hi) hi = cell[i];
  }
  size_t span = (size_t)((long long)hi - lo + 1);
  int* cnt = ial(span + 1);
  int* kc = ial(n);
  int* ki = ial(n);
  for (int i = 0; i < n; ++i) cnt[cell[i] - lo + 1]++;
  for (size_t k = 1; k <= span; ++k) cnt[k] += cnt[k - 1];
  for (int i = 0; i < n; ++i) {
    int p = cnt[cell[i] - lo]++;
    kc[p] = cell[i];
    ki[p] = index[i];
  }
  memcpy(cell, kc, n * sizeof(int));
  memcpy(index, ki, n * sizeof(int));
  free(cnt);
  free(kc);
  free(ki);
}

int orc_neighbours_search(orc_sys* s) {
  int N = s->N;
  /* kernel_cell_list.cu:15-63 */
  for (int i = 0; i < N; ++i) {
    int cx = (int)floor(s->x[i] / s->cell_size[0]);
    if (cx == s->Ncells[0]) cx = cx - 1;
    int cy, cz = 0;
    if (s->wall == 0) {
      cy = (int)floor(s->y[i] / s->cell_size[1]);
      if (cy == s->Ncells[1]) cy = cy - 1;
    } else {
      cy = (int)floor((s->y[i] + s->wall_width) / s->cell_size[1]);
    }
    if (s->dim == 3) {
      cz = (int)floor(s->z[i] / s->cell_size[2]);
      if (cz == s->Ncells[2]) cz = cz - 1;
    }
    s->particle_cell[i] = (s->dim == 2) ? cy * s->Ncells[0] + cx
                                        : cz * s->Ncells[0] * s->Ncells[1] + cy * s->Ncells[0] + cx;
    s->particle_index[i] = i;
  }
  orc_stable_sort_by_cell(N, s->particle_cell, s->particle_index);
  /* kernel_cell_ranges.cu:13-33 -- cells without particles keep their old values */
  int bad = 0;
  for (int i = 0; i < N; ++i) {
    int c = s->particle_cell[i];
    if (c < 0 || c > s->Ntotal_cells - 1) {
      bad = 1;
      continue;
    }
    if (i == 0 || s->particle_cell[i - 1] != c) s->cell_start[c] = i;
    if (i == N - 1 || s->particle_cell[i + 1] != c) s->cell_end[c] = i;
  }
  s->bad_cell = bad;
  /* colloid coarse grid: system_neighbours_search.cu:70-106 */
  if (s->N_colloids >= 2) {
    int nc = s->N_colloids;
    for (int i = 0; i < nc; ++i) {
      int cx = (int)floor(s->coll_x[i] / s->cell_colloids_size[0]);
      int cy = (int)floor(s->coll_y[i] / s->cell_colloids_size[1]);
      int cz = (s->dim == 3) ? (int)floor(s->coll_z[i] / s->cell_colloids_size[2]) : 0;
      s->coll_cell[i] = (s->dim == 2) ? cy * s->Ncells_colloids[0] + cx
                                      : cz * s->Ncells_colloids[0] * s->Ncells_colloids[1] +
                                            cy * s->Ncells_colloids[0] + cx;
      s->coll_index[i] = i;
    }
    orc_stable_sort_by_cell(nc, s->coll_cell, s->coll_index);
    for (int c = 0; c < s->Ntotal_cells_colloids; ++c) {
      s->coll_cell_start[c] = -1;
      s->coll_cell_end[c] = -2;
    }
    for (int i = 0; i < nc; ++i) {
      int c = s->coll_cell[i];
      if (c < 0 || c >= s->Ntotal_cells_colloids) continue;
      if (i == 0 || s->coll_cell[i - 1] != c) s->coll_cell_start[c] = i;
      if (i == nc - 1 || s->coll_cell[i + 1] != c) s->coll_cell_end[c] = i;
    }
  }
  return bad;
}

/* Neighbour cells of particle i in the reference's loop order (dx outer, dz inner):
   kernel_densities.cu:52-163.  The particle's own cell is NOT clamped (:52-60). */
static int orc_neigh_cells(const orc_sys* s, int i, int* cells) {
  int cxi = (int)floor(s->x[i] / s->cell_size[0]);
  int cyi = (s->wall == 0) ? (int)floor(s->y[i] / s->cell_size[1])
                           : (int)floor((s->y[i] + s->wall_width) / s->cell_size[1]);
  int czi = (s->dim == 3) ? (int)floor(s->z[i] / s->cell_size[2]) : 0;
  int n = 0, N0 = s->Ncells[0], N1 = s->Ncells[1], N2 = s->Ncells[2];
  int dzlo = (s->dim == 3) ? -1 : 0, dzhi = (s->dim == 3) ? 1 : 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = dzlo; dz <= dzhi; ++dz) {
        int cx = cxi + dx, cy = cyi + dy, cz = czi + dz;
        if (cx < 0) cx += N0;
        if (cx >= N0) cx -= N0;
        if (s->dim == 3) {
          if (cz < 0) cz += N2;
          if (cz >= N2) cz -= N2;
        }
        if (s->wall == 0) {
          if (cy < 0) cy += N1;
          if (cy >= N1) cy -= N1;
        }
        if (cy >= 0 && cy < N1) cells[n++] = (s->dim == 3) ? cz * N0 * N1 + cy * N0 + cx : cy * N0 + cx;
      }
  return n;
}

/* minimum image as written in the kernels: xij -= L if > L/2, += L if < -L/2 */
static inline void orc_mimage(const orc_sys* s, double* r) {
  double h0 = 0.5 * s->L[0], h1 = 0.5 * s->L[1], h2 = 0.5 * s->L[2];
  if (r[0] > h0) r[0] -= s->L[0];
  if (r[0] < -h0) r[0] += s->L[0];
  if (s->wall == 0) {
    if (r[1] > h1) r[1] -= s->L[1];
    if (r[1] < -h1) r[1] += s->L[1];
  }
  if (s->dim == 3) {
    if (r[2] > h2) r[2] -= s->L[2];
    if (r[2] < -h2) r[2] += s->L[2];
  }
}

/* kernel_densities.cu:16-193 (density_to_zero folded in) */
void orc_calculate_density(orc_sys* s) {
  int N = s->N;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < N; ++i) {
    int cells[27];
    int nn = orc_neigh_cells(s, i, cells);
    double d = 0.0;
    for (int q = 0; q < nn; ++q) {
      int c = cells[q];
      for (int k = s->cell_start[c]; k <= s->cell_end[c]; ++k) {
        int j = s->particle_index[k];
        double r[3] = {s->x[i] - s->x[j], s->y[i] - s->y[j],
                       s->dim == 3 ? s->z[i] - s->z[j] : 0.0};
        orc_mimage(s, r);
        double r2 = (s->dim == 3) ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2]
                                  : r[0] * r[0] + r[1] * r[1];
        if (r2 < s->rcutsq) d = d + orc_W(s, sqrt(r2));
      }
    }
    s->dens[i] = d;
  }
}

/* kernel_pressures.cu:13-23 */
void orc_calculate_pressure(orc_sys* s) {
  for (int i = 0; i < s->N; ++i) s->press[i] = s->csq * (s->mass[i] * s->dens[i] - s->rho0);
}

/* Morris ghost relative velocity for a fluid particle i next to a non-fluid particle j,
   used identically by kernel_vel_gradients.cu:162-247 and kernel_forces.cu:234-318
   (3D: :421-525, :590-692).  rij = x_i - x_j after minimum image. */
static void orc_ghost_fluid_i(const orc_sys* s, int i, int j, const double* rij, double* vij) {
  int tj = s->type[j];
  double vi[3] = {s->vx[i], s->vy[i], s->dim == 3 ? s->vz[i] : 0.0};
  double beta, di, dj;
  if (tj == 1 || tj == 2) {
    double Vw;
    if (tj == 1) {
      di = s->y[i] - s->y_bottom;
      dj = s->y_bottom - s->y[j];
      Vw = s->V_bottom;
    } else {
      di = s->y_top - s->y[i];
      dj = s->y[j] - s->y_top;
      Vw = s->V_top;
    }
    beta = 1.0 + dj / di;
    if (beta > s->beta_max) beta = s->beta_max;
    if (di > 0) {
      vij[0] = beta * (vi[0] - Vw);
      vij[1] = beta * vi[1];
      vij[2] = beta * vi[2];
    } else {
      vij[0] = vi[0] - Vw;
      vij[1] = vi[1];
      vij[2] = vi[2];
    }
    return;
  }
  int cp = tj - 3;
  double rc[3] = {s->x[i] - s->coll_x[cp], s->y[i] - s->coll_y[cp],
                  s->dim == 3 ? s->z[i] - s->coll_z[cp] : 0.0};
  orc_mimage(s, rc);
  double dc = (s->dim == 3) ? sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2])
                            : sqrt(rc[0] * rc[0] + rc[1] * rc[1]);
  double dis = dc - s->coll_R;
  double cv[3] = {s->coll_vx[cp], s->coll_vy[cp], s->dim == 3 ? s->coll_vz[cp] : 0.0};
  if (dis < 0) {
    for (int a = 0; a < 3; ++a) vij[a] = vi[a] - cv[a];
    return;
  }
  double xs = rc[0] / dc * s->coll_R, ys = rc[1] / dc * s->coll_R;
  double zs = (s->dim == 3) ? rc[2] / dc * s->coll_R : 0.0;
  double vr[3];
  if (s->dim == 2) {
    double wz = s->coll_omegaz[cp];
    vr[0] = -wz * ys;
    vr[1] = wz * xs;
    vr[2] = 0.0;
  } else {
    double wx = s->coll_omegax[cp], wy = s->coll_omegay[cp], wz = s->coll_omegaz[cp];
    vr[0] = wy * zs - wz * ys;
    vr[1] = wz * xs - wx * zs;
    vr[2] = wx * ys - wy * xs;
  }
  double sv[3] = {rc[0] / dc, rc[1] / dc, s->dim == 3 ? rc[2] / dc : 0.0};
  double djs = (s->dim == 3) ? (rij[0] * sv[0] + rij[1] * sv[1] + rij[2] * sv[2]) - dis
                             : (rij[0] * sv[0] + rij[1] * sv[1]) - dis;
  beta = 1.0 + djs / dis;
  if (beta > s->beta_max) beta = s->beta_max;
  for (int a = 0; a < 3; ++a) vij[a] = beta * (vi[a] - cv[a] - vr[a]);
}

/* Morris ghost relative velocity for a non-fluid particle i next to particle j
   (kernel_vel_gradients.cu:249-331, kernel_forces.cu:337-418; 3D :527-630, :721-821). */
static void orc_ghost_solid_i(const orc_sys* s, int i, int j, const double* rij, double* vij) {
  int ti = s->type[i];
  double vj[3] = {s->vx[j], s->vy[j], s->dim == 3 ? s->vz[j] : 0.0};
  double beta, di, dj;
  if (ti == 1 || ti == 2) {
    double Vw;
    if (ti == 1) {
      di = s->y_bottom - s->y[i];
      dj = s->y[j] - s->y_bottom;
      Vw = s->V_bottom;
    } else {
      di = s->y[i] - s->y_top;
      dj = s->y_top - s->y[j];
      Vw = s->V_top;
    }
    beta = 1.0 + di / dj;
    if (beta > s->beta_max) beta = s->beta_max;
    if (dj > 0) {
      vij[0] = beta * (Vw - vj[0]);
      vij[1] = -beta * vj[1];
      vij[2] = -beta * vj[2];
    } else {
      vij[0] = Vw - vj[0];
      vij[1] = -vj[1];
      vij[2] = -vj[2];
    }
    return;
  }
  int cp = ti - 3;
  double rc[3] = {s->x[j] - s->coll_x[cp], s->y[j] - s->coll_y[cp],
                  s->dim == 3 ? s->z[j] - s->coll_z[cp] : 0.0};
  orc_mimage(s, rc);
  double dc = (s->dim == 3) ? sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2])
                            : sqrt(rc[0] * rc[0] + rc[1] * rc[1]);
  double djs = dc - s->coll_R;
  double cv[3] = {s->coll_vx[cp], s->coll_vy[cp], s->dim == 3 ? s->coll_vz[cp] : 0.0};
  if (djs < 0) {
    for (int a = 0; a < 3; ++a) vij[a] = cv[a] - vj[a];
    return;
  }
  double xs = rc[0] / dc * s->coll_R, ys = rc[1] / dc * s->coll_R;
  double zs = (s->dim == 3) ? rc[2] / dc * s->coll_R : 0.0;
  double vr[3];
  if (s->dim == 2) {
    double wz = s->coll_omegaz[cp];
    vr[0] = -wz * ys;
    vr[1] = wz * xs;
    vr[2] = 0.0;
  } else {
    double wx = s->coll_omegax[cp], wy = s->coll_omegay[cp], wz = s->coll_omegaz[cp];
    vr[0] = wy * zs - wz * ys;
    vr[1] = wz * xs - wx * zs;
    vr[2] = wx * ys - wy * xs;
  }
  double sv[3] = {rc[0] / dc, rc[1] / dc, s->dim == 3 ? rc[2] / dc : 0.0};
  double dis = (s->dim == 3) ? (-rij[0] * sv[0] - rij[1] * sv[1] - rij[2] * sv[2]) - djs
                             : (-rij[0] * sv[0] - rij[1] * sv[1]) - djs;
  beta = 1.0 + dis / djs;
  if (beta > s->beta_max) beta = s->beta_max;
  for (int a = 0; a < 3; ++a) vij[a] = beta * (cv[a] + vr[a] - vj[a]);
}

/* kernel_vel_gradients.cu:15-662 (vel_gradients_to_zero folded in).
   g_ab = -(1/d_i) sum_j W'(r) e_a v_ij,b  (gradv_mu_nu = dv_nu/dx_mu) */
void orc_calculate_vel_gradient(orc_sys* s) {
  int N = s->N, dim = s->dim;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < N; ++i) {
    int cells[27];
    int nn = orc_neigh_cells(s, i, cells);
    double dinv = 1.0 / s->dens[i];
    int ti = s->type[i];
    double g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < nn; ++q) {
      int c = cells[q];
      for (int k = s->cell_start[c]; k <= s->cell_end[c]; ++k) {
        int j = s->particle_index[k];
        if (i == j) continue;
        int tj = s->type[j];
        if (ti == tj && ti != 0) continue; /* :126-127 */
        double r[3] = {s->x[i] - s->x[j], s->y[i] - s->y[j], dim == 3 ? s->z[i] - s->z[j] : 0.0};
        orc_mimage(s, r);
        double r2 = (dim == 3) ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2] : r[0] * r[0] + r[1] * r[1];
        if (!(r2 < s->rcutsq)) continue;
        double rr = sqrt(r2);
        double rinv = 1.0 / rr;
        double e[3] = {r[0] * rinv, r[1] * rinv, dim == 3 ? r[2] * rinv : 0.0};
        double gw = orc_gradW(s, rr);
        double v[3];
        if (ti == tj) {
          v[0] = s->vx[i] - s->vx[j];
          v[1] = s->vy[i] - s->vy[j];
          v[2] = dim == 3 ? s->vz[i] - s->vz[j] : 0.0;
        } else if (ti == 0) {
          orc_ghost_fluid_i(s, i, j, r, v);
        } else {
          orc_ghost_solid_i(s, i, j, r, v);
        }
        for (int a = 0; a < dim; ++a)
          for (int b2 = 0; b2 < dim; ++b2) g[a][b2] += -dinv * gw * e[a] * v[b2];
      }
    }
    s->gxx[i] = g[0][0]; s->gxy[i] = g[0][1]; s->gyx[i] = g[1][0]; s->gyy[i] = g[1][1];
    if (dim == 3) {
      s->gxz[i] = g[0][2]; s->gyz[i] = g[1][2]; s->gzx[i] = g[2][0]; s->gzy[i] = g[2][1];
      s->gzz[i] = g[2][2];
    }
  }
}

/* kernel_forces.cu:15-865 (forces_to_zero folded in: f = 0 + sum) */
void orc_kernel_forces(orc_sys* s) {
  int N = s->N, dim = s->dim;
  double nkT = s->nkT;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < N; ++i) {
    int cells[27];
    int nn = orc_neigh_cells(s, i, cells);
    int ti = s->type[i];
    double di0 = s->dens[i], pi0 = s->press[i];
    /* Pi = p I - nkT c, divided by d^2: :62-88 */
    double dinv0 = 1.0 / di0, dinv0sq = dinv0 * dinv0;
    double Pi0[6] = {(pi0 - nkT * s->cxx[i]) * dinv0sq, (-nkT * s->cxy[i]) * dinv0sq,
                     (pi0 - nkT * s->cyy[i]) * dinv0sq, 0, 0, 0};
    if (dim == 3) {
      Pi0[3] = (-nkT * s->cxz[i]) * dinv0sq;
      Pi0[4] = (-nkT * s->cyz[i]) * dinv0sq;
      Pi0[5] = (pi0 - nkT * s->czz[i]) * dinv0sq;
    }
    double f[3] = {0, 0, 0};
    for (int q = 0; q < nn; ++q) {
      int c = cells[q];
      for (int k = s->cell_start[c]; k <= s->cell_end[c]; ++k) {
        int j = s->particle_index[k];
        if (i == j) continue;
        int tj = s->type[j];
        if (ti != 0 && tj != 0) continue; /* :157-158 */
        double r[3] = {s->x[i] - s->x[j], s->y[i] - s->y[j], dim == 3 ? s->z[i] - s->z[j] : 0.0};
        orc_mimage(s, r);
        double r2 = (dim == 3) ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2] : r[0] * r[0] + r[1] * r[1];
        if (!(r2 < s->rcutsq)) continue;
        double Pi[6], Pj[6], dinv_i, dinv_j, v[3];
        if (ti == tj) { /* fluid - fluid: :196-215 */
          double dj = s->dens[j], pj = s->press[j];
          dinv_i = dinv0;
          dinv_j = 1.0 / dj;
          double djsq = dinv_j * dinv_j;
          for (int a = 0; a < 6; ++a) Pi[a] = Pi0[a];
          Pj[0] = (pj - nkT * s->cxx[j]) * djsq;
          Pj[1] = (-nkT * s->cxy[j]) * djsq;
          Pj[2] = (pj - nkT * s->cyy[j]) * djsq;
          if (dim == 3) {
            Pj[3] = (-nkT * s->cxz[j]) * djsq;
            Pj[4] = (-nkT * s->cyz[j]) * djsq;
            Pj[5] = (pj - nkT * s->czz[j]) * djsq;
          }
          v[0] = s->vx[i] - s->vx[j];
          v[1] = s->vy[i] - s->vy[j];
          v[2] = dim == 3 ? s->vz[i] - s->vz[j] : 0.0;
        } else if (ti == 0) { /* fluid i, solid j: density and pressure mirrored, :217-233 */
          double pj = pi0;
          dinv_i = dinv0;
          dinv_j = dinv0;
          double djsq = dinv_j * dinv_j;
          for (int a = 0; a < 6; ++a) Pi[a] = Pi0[a];
          Pj[0] = (pj - nkT * s->cxx[j]) * djsq;
          Pj[1] = (-nkT * s->cxy[j]) * djsq;
          Pj[2] = (pj - nkT * s->cyy[j]) * djsq;
          if (dim == 3) {
            Pj[3] = (-nkT * s->cxz[j]) * djsq;
            Pj[4] = (-nkT * s->cyz[j]) * djsq;
            Pj[5] = (pj - nkT * s->czz[j]) * djsq;
          }
          orc_ghost_fluid_i(s, i, j, r, v);
        } else { /* solid i, fluid j: everything taken from j, :320-336 */
          double dj = s->dens[j], pj = s->press[j];
          dinv_j = 1.0 / dj;
          dinv_i = dinv_j;
          double djsq = dinv_j * dinv_j;
          Pj[0] = (pj - nkT * s->cxx[j]) * djsq;
          Pj[1] = (-nkT * s->cxy[j]) * djsq;
          Pj[2] = (pj - nkT * s->cyy[j]) * djsq;
          if (dim == 3) {
            Pj[3] = (-nkT * s->cxz[j]) * djsq;
            Pj[4] = (-nkT * s->cyz[j]) * djsq;
            Pj[5] = (pj - nkT * s->czz[j]) * djsq;
          }
          for (int a = 0; a < 6; ++a) Pi[a] = Pj[a];
          orc_ghost_solid_i(s, i, j, r, v);
        }
        double rr = sqrt(r2);
        double rinv = 1.0 / rr;
        double gw = orc_gradW(s, rr);
        double e[3] = {r[0] * rinv, r[1] * rinv, dim == 3 ? r[2] * rinv : 0.0};
        double aux = gw * dinv_i * dinv_j * rinv;
        double aux1 = s->a * aux;
        if (dim == 2) {
          double ev = e[0] * v[0] + e[1] * v[1];
          double axx = -gw * (Pi[0] + Pj[0]);
          double axy = -gw * (Pi[1] + Pj[1]);
          double ayy = -gw * (Pi[2] + Pj[2]);
          f[0] += axx * e[0] + axy * e[1];
          f[1] += axy * e[0] + ayy * e[1];
          double aux2 = s->b * aux * ev;
          f[0] += aux1 * v[0] + aux2 * e[0];
          f[1] += aux1 * v[1] + aux2 * e[1];
        } else {
          double ev = e[0] * v[0] + e[1] * v[1] + e[2] * v[2];
          double axx = -gw * (Pi[0] + Pj[0]);
          double axy = -gw * (Pi[1] + Pj[1]);
          double ayy = -gw * (Pi[2] + Pj[2]);
          double axz = -gw * (Pi[3] + Pj[3]);
          double ayz = -gw * (Pi[4] + Pj[4]);
          double azz = -gw * (Pi[5] + Pj[5]);
          f[0] += axx * e[0] + axy * e[1] + axz * e[2];
          f[1] += axy * e[0] + ayy * e[1] + ayz * e[2];
          f[2] += axz * e[0] + ayz * e[1] + azz * e[2];
          double aux2 = s->b * aux * ev;
          f[0] += aux1 * v[0] + aux2 * e[0];
          f[1] += aux1 * v[1] + aux2 * e[1];
          f[2] += aux1 * v[2] + aux2 * e[2];
        }
      }
    }
    s->fx[i] = f[0];
    s->fy[i] = f[1];
    if (dim == 3) s->fz[i] = f[2];
  }
}

/* kernel_ext_force.cu:13-73 */
void orc_calculate_external_forces(orc_sys* s) {
  for (int i = 0; i < s->N; ++i) {
    if (s->type[i] != 0) continue;
    double m = s->mass[i];
    if (s->ext_force_type == 1) {
      s->fx[i] += m * s->ext_force[0];
      s->fy[i] += m * s->ext_force[1];
      if (s->dim == 3) s->fz[i] += m * s->ext_force[2];
    } else if (s->ext_force_type == 2) {
      s->fx[i] += m * s->ext_force[0] * sin(s->ky * s->y[i]);
      s->fy[i] += 0.0;
      if (s->dim == 3) s->fz[i] += 0.0;
    } else if (s->ext_force_type == 3) {
      double fx = (s->y[i] < 0.5 * s->L[1]) ? m * s->ext_force[0] : -(m * s->ext_force[0]);
      s->fx[i] += fx;
      s->fy[i] += 0.0;
      if (s->dim == 3) s->fz[i] += 0.0;
    }
  }
}

/* kernel_dcdt.cu:15-104: dc/dt = c.g + (c.g)^T + (I - c)/tau, fluid only */
void orc_kernel_dcdt(orc_sys* s) {
  double tinv = 1.0 / s->tau;
  for (int i = 0; i < s->N; ++i) {
    if (s->type[i] != 0) continue;
    double cxx = s->cxx[i], cxy = s->cxy[i], cyy = s->cyy[i];
    if (s->dim == 2) {
      double gxx = s->gxx[i], gxy = s->gxy[i], gyx = s->gyx[i], gyy = s->gyy[i];
      double Axx = cxx * gxx + cxy * gyx;
      double Axy = cxx * gxy + cxy * gyy;
      double Ayx = cxy * gxx + cyy * gyx;
      double Ayy = cxy * gxy + cyy * gyy;
      s->dcdt_xx[i] = 2.0 * Axx + tinv * (1.0 - cxx);
      s->dcdt_xy[i] = Axy + Ayx - tinv * cxy;
      s->dcdt_yy[i] = 2.0 * Ayy + tinv * (1.0 - cyy);
    } else {
      double cxz = s->cxz[i], cyz = s->cyz[i], czz = s->czz[i];
      double gxx = s->gxx[i], gxy = s->gxy[i], gxz = s->gxz[i];
      double gyx = s->gyx[i], gyy = s->gyy[i], gyz = s->gyz[i];
      double gzx = s->gzx[i], gzy = s->gzy[i], gzz = s->gzz[i];
      double Axx = cxx * gxx + cxy * gyx + cxz * gzx;
      double Axy = cxx * gxy + cxy * gyy + cxz * gzy;
      double Axz = cxx * gxz + cxy * gyz + cxz * gzz;
      double Ayx = cxy * gxx + cyy * gyx + cyz * gzx;
      double Ayy = cxy * gxy + cyy * gyy + cyz * gzy;
      double Ayz = cxy * gxz + cyy * gyz + cyz * gzz;
      double Azx = cxz * gxx + cyz * gyx + czz * gzx;
      double Azy = cxz * gxy + cyz * gyy + czz * gzy;
      double Azz = cxz * gxz + cyz * gyz + czz * gzz;
      s->dcdt_xx[i] = 2.0 * Axx + tinv * (1.0 - cxx);
      s->dcdt_xy[i] = Axy + Ayx - tinv * cxy;
      s->dcdt_yy[i] = 2.0 * Ayy + tinv * (1.0 - cyy);
      s->dcdt_xz[i] = Axz + Azx - tinv * cxz;
      s->dcdt_yz[i] = Ayz + Azy - tinv * cyz;
      s->dcdt_zz[i] = 2.0 * Azz + tinv * (1.0 - czz);
    }
  }
}

/* kernel_collect_force_walls.cu:15-50 */
void orc_calculate_force_walls(orc_sys* s) {
  for (int w = 0; w < s->Nwalls; ++w) {
    int end = (w < s->Nwalls - 1) ? s->walls_start[w + 1] - 1 : s->Nlist_walls - 1;
    double fx = 0, fy = 0, fz = 0;
    for (int j = s->walls_start[w]; j <= end; ++j) {
      int p = s->walls_list[j];
      fx = fx + s->fx[p];
      fy = fy + s->fy[p];
      if (s->dim == 3) fz = fz + s->fz[p];
    }
    s->fx_wall[w] = fx;
    s->fy_wall[w] = fy;
    if (s->dim == 3) s->fz_wall[w] = fz;
  }
}

/* kernel_colloid_forces_to_zero.cu + kernel_collect_force_colloids.cu:15-99 */
static void orc_collect_force_colloids(orc_sys* s) {
  int dim = s->dim;
  for (int c = 0; c < s->N_colloids; ++c) {
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    int end = (c < s->N_colloids - 1) ? s->colloids_start[c + 1] - 1 : s->Nlist_colloids - 1;
    for (int j = s->colloids_start[c]; j <= end; ++j) {
      int p = s->colloids_list[j];
      F[0] = F[0] + s->fx[p];
      F[1] = F[1] + s->fy[p];
      if (dim == 3) F[2] = F[2] + s->fz[p];
      double rx = s->x[p] - s->coll_x[c];
      double ry = s->y[p] - s->coll_y[c];
      double rz = 0.0;
      if (rx > 0.5 * s->L[0]) rx -= s->L[0];
      if (rx < -0.5 * s->L[0]) rx += s->L[0];
      if (s->wall == 0) {
        if (ry > 0.5 * s->L[1]) ry -= s->L[1];
        if (ry < -0.5 * s->L[1]) ry += s->L[1];
      }
      if (dim == 3) {
        rz = s->z[p] - s->coll_z[c];
        if (rz > 0.5 * s->L[2]) rz -= s->L[2];
        if (rz < -0.5 * s->L[2]) rz += s->L[2];
      }
      T[2] = T[2] + rx * s->fy[p] - ry * s->fx[p];
      if (dim == 3) {
        T[0] = T[0] + ry * s->fz[p] - rz * s->fy[p];
        T[1] = T[1] + rz * s->fx[p] - rx * s->fz[p];
      }
    }
    s->fx_colloid[c] = F[0];
    s->fy_colloid[c] = F[1];
    s->tz_colloid[c] = T[2];
    if (dim == 3) {
      s->fz_colloid[c] = F[2];
      s->tx_colloid[c] = T[0];
      s->ty_colloid[c] = T[1];
    }
  }
}

/* colloid-pair iteration over the coarse grid in the reference order
   (kernel_repulsion_force_colloids.cu:54-205, kernel_magnetic_force_colloids.cu:48-201) */
static int orc_coll_neigh_cells(const orc_sys* s, int i, int* cells) {
  const int* Nc = s->Ncells_colloids;
  int cxi = (int)floor(s->coll_x[i] / s->cell_colloids_size[0]);
  int cyi = (int)floor(s->coll_y[i] / s->cell_colloids_size[1]);
  int czi = (s->dim == 3) ? (int)floor(s->coll_z[i] / s->cell_colloids_size[2]) : 0;
  int n = 0;
  int dzlo = (s->dim == 3) ? -1 : 0, dzhi = (s->dim == 3) ? 1 : 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = dzlo; dz <= dzhi; ++dz) {
        int cx = cxi + dx, cy = cyi + dy, cz = czi + dz;
        if (cx < 0) cx += Nc[0];
        if (cx >= Nc[0]) cx -= Nc[0];
        if (s->wall == 0) {
          if (cy < 0) cy += Nc[1];
          if (cy >= Nc[1]) cy -= Nc[1];
        }
        if (s->dim == 3) {
          if (cz < 0) cz += Nc[2];
          if (cz >= Nc[2]) cz -= Nc[2];
        }
        if (cy >= 0 && cy < Nc[1]) cells[n++] = (s->dim == 3) ? cz * Nc[0] * Nc[1] + cy * Nc[0] + cx : cy * Nc[0] + cx;
      }
  return n;
}

/* kernel_repulsion_force_colloids.cu:21-207 (r^2 clamped to the cut-on before e = r/|r|) */
static void orc_repulsion(orc_sys* s) {
  int nc = s->N_colloids, dim = s->dim;
  double* F[3] = {s->fx_colloid, s->fy_colloid, s->fz_colloid};
  double Famp = s->F0_rep * s->tau_rep;
  for (int i = 0; i < nc; ++i) {
    int cells[27];
    int nn = orc_coll_neigh_cells(s, i, cells);
    for (int q = 0; q < nn; ++q) {
      int c = cells[q];
      for (int k = s->coll_cell_start[c]; k <= s->coll_cell_end[c]; ++k) {
        int j = s->coll_index[k];
        if (i == j) continue;
        double r[3] = {s->coll_x[i] - s->coll_x[j], s->coll_y[i] - s->coll_y[j],
                       dim == 3 ? s->coll_z[i] - s->coll_z[j] : 0.0};
        orc_mimage(s, r);
        double r2 = (dim == 3) ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2] : r[0] * r[0] + r[1] * r[1];
        if (r2 < s->rcuton_coll_rep_sq) r2 = s->rcuton_coll_rep_sq;
        if (r2 <= s->rcutoff_coll_rep_sq) {
          double rr = sqrt(r2);
          double ts = -s->tau_rep * (rr - 2.0 * s->coll_R) / s->coll_R;
          double ex = exp(ts);
          double Fm = Famp * ex / (1.0 - ex);
          for (int a = 0; a < dim; ++a) F[a][i] = F[a][i] + Fm * (r[a] / rr);
        }
      }
    }
  }
}

/* kernel_magnetic_force_colloids.cu:15-203 (3D: e = r_ij/(|r_ij|/R), so |e| = R) */
static void orc_magnetic(orc_sys* s, const double* m) {
  int nc = s->N_colloids, dim = s->dim;
  double* F[3] = {s->fx_colloid, s->fy_colloid, s->fz_colloid};
  for (int i = 0; i < nc; ++i) {
    int cells[27];
    int nn = orc_coll_neigh_cells(s, i, cells);
    for (int q = 0; q < nn; ++q) {
      int c = cells[q];
      for (int k = s->coll_cell_start[c]; k <= s->coll_cell_end[c]; ++k) {
        int j = s->coll_index[k];
        if (i == j) continue;
        double r[3] = {s->coll_x[i] - s->coll_x[j], s->coll_y[i] - s->coll_y[j],
                       dim == 3 ? s->coll_z[i] - s->coll_z[j] : 0.0};
        orc_mimage(s, r);
        double r2 = (dim == 3) ? r[0] * r[0] + r[1] * r[1] + r[2] * r[2] : r[0] * r[0] + r[1] * r[1];
        if (r2 <= s->r0_magnet_sq) {
          double rr = (dim == 3) ? sqrt(r2) / s->coll_R : sqrt(r2);
          double e[3] = {r[0] / rr, r[1] / rr, dim == 3 ? r[2] / rr : 0.0};
          double me = (dim == 3) ? m[0] * e[0] + m[1] * e[1] + m[2] * e[2] : m[0] * e[0] + m[1] * e[1];
          double me2 = me * me;
          double F0r4 = s->F0_magnet / (r2 * r2);
          for (int a = 0; a < dim; ++a)
            F[a][i] = F[a][i] + F0r4 * (2.0 * me * m[a] - (5.0 * me2 - 1.0) * e[a]);
        }
      }
    }
  }
}

/* system_calculate_force_colloids.cu:15-97 */
void orc_calculate_force_colloids(orc_sys* s, const double* m) {
  orc_collect_force_colloids(s);
  if (s->N_colloids >= 2) {
    orc_repulsion(s);
    orc_magnetic(s, m);
  }
}

/* system_calculate_forces.cu:16-174 */
void orc_calculate_forces(orc_sys* s, const double* m) {
  orc_calculate_density(s);
  orc_calculate_vel_gradient(s);
  orc_calculate_pressure(s);
  orc_kernel_forces(s);
  if (s->ext_force_type != 0) orc_calculate_external_forces(s);
  orc_kernel_dcdt(s);
  if (s->wall) orc_calculate_force_walls(s);
  if (s->N_colloids > 0) orc_calculate_force_colloids(s, m);
}

/* kernel_quaternion_product.cu:15-31 (Hamilton product) */
static void orc_qmul(const double* c, const double* d, double* r) {
  r[0] = c[0] * d[0] - c[1] * d[1] - c[2] * d[2] - c[3] * d[3];
  r[1] = c[0] * d[1] + c[1] * d[0] + c[2] * d[3] - c[3] * d[2];
  r[2] = c[0] * d[2] - c[1] * d[3] + c[2] * d[0] + c[3] * d[1];
  r[3] = c[0] * d[3] + c[1] * d[2] - c[2] * d[1] + c[3] * d[0];
}

/* kernel_move_sys_VV_part1.cu:13-114 + kernel_move_colloids_VV_part1.cu:15-204 */
void orc_vv_step1(orc_sys* s) {
  int dim = s->dim;
  double dt = s->in.dt;
  double* L = s->L;
  for (int i = 0; i < s->N; ++i) {
    int t = s->type[i];
    if (t > 2) continue;
    double xi = s->x[i], yi = s->y[i], zi = (dim == 3) ? s->z[i] : 0.0;
    if (t == 0) {
      double h = 0.5 * dt;
      double hm = h / s->mass[i];
      s->vx[i] = s->vx[i] + hm * s->fx[i];
      s->vy[i] = s->vy[i] + hm * s->fy[i];
      s->cxx[i] = s->cxx[i] + h * s->dcdt_xx[i];
      s->cxy[i] = s->cxy[i] + h * s->dcdt_xy[i];
      s->cyy[i] = s->cyy[i] + h * s->dcdt_yy[i];
      if (dim == 3) {
        s->vz[i] = s->vz[i] + hm * s->fz[i];
        s->cxz[i] = s->cxz[i] + h * s->dcdt_xz[i];
        s->cyz[i] = s->cyz[i] + h * s->dcdt_yz[i];
        s->czz[i] = s->czz[i] + h * s->dcdt_zz[i];
      }
    } else {
      s->vx[i] = (t == 1) ? s->V_bottom : s->V_top;
      s->vy[i] = 0.0;
      if (dim == 3) s->vz[i] = 0.0;
    }
    xi = xi + s->vx[i] * dt;
    yi = yi + s->vy[i] * dt;
    if (dim == 3) zi = zi + s->vz[i] * dt;
    if (xi < 0) xi = xi + L[0];
    if (s->wall == 0 && yi < 0) yi = yi + L[1];
    if (dim == 3 && zi < 0) zi = zi + L[2];
    if (xi > L[0]) xi = xi - L[0];
    if (s->wall == 0 && yi > L[1]) yi = yi - L[1];
    if (dim == 3 && zi > L[2]) zi = zi - L[2];
    s->x[i] = xi;
    s->y[i] = yi;
    if (dim == 3) s->z[i] = zi;
  }
  if (s->N_colloids > 0 && s->in.coll_move == 0) {
    double hm = 0.5 * dt / s->coll_mass, hI = 0.5 * dt / s->coll_I;
    for (int c = 0; c < s->N_colloids; ++c) {
      double cx = s->coll_x[c], cy = s->coll_y[c], cz = (dim == 3) ? s->coll_z[c] : 0.0;
      s->coll_vx[c] += hm * s->fx_colloid[c];
      s->coll_vy[c] += hm * s->fy_colloid[c];
      if (dim == 3) s->coll_vz[c] += hm * s->fz_colloid[c];
      double omega;
      s->coll_omegaz[c] += hI * s->tz_colloid[c];
      if (dim == 2) {
        omega = s->coll_omegaz[c];
      } else {
        s->coll_omegax[c] += hI * s->tx_colloid[c];
        s->coll_omegay[c] += hI * s->ty_colloid[c];
        omega = sqrt(s->coll_omegax[c] * s->coll_omegax[c] + s->coll_omegay[c] * s->coll_omegay[c] +
                     s->coll_omegaz[c] * s->coll_omegaz[c]);
      }
      cx = cx + s->coll_vx[c] * dt;
      cy = cy + s->coll_vy[c] * dt;
      if (dim == 3) cz = cz + s->coll_vz[c] * dt;
      if (cx < 0) cx = cx + L[0];
      if (cx > L[0]) cx = cx - L[0];
      if (s->wall == 0) {
        if (cy < 0) cy = cy + L[1];
        if (cy > L[1]) cy = cy - L[1];
      }
      if (dim == 3) {
        if (cz < 0) cz = cz + L[2];
        if (cz > L[2]) cz = cz - L[2];
      }
      s->coll_x[c] = cx;
      s->coll_y[c] = cy;
      if (dim == 3) s->coll_z[c] = cz;
      double ca = 0, sa = 0, q[4] = {1, 0, 0, 0};
      if (dim == 2) {
        double th = s->coll_theta[c] + s->coll_omegaz[c] * dt;
        sa = sin(th);
        ca = cos(th);
        s->coll_theta[c] = th;
      } else {
        double dth = 0.5 * omega * dt;
        double ax[3] = {s->coll_omegax[c] / omega, s->coll_omegay[c] / omega,
                        s->coll_omegaz[c] / omega};
        double sh = sin(dth);
        double dq[4] = {cos(dth), sh * ax[0], sh * ax[1], sh * ax[2]};
        double qc[4] = {s->coll_quat0[c], s->coll_quatx[c], s->coll_quaty[c], s->coll_quatz[c]};
        orc_qmul(dq, qc, q);
        s->coll_quat0[c] = q[0];
        s->coll_quatx[c] = q[1];
        s->coll_quaty[c] = q[2];
        s->coll_quatz[c] = q[3];
      }
      int j0 = s->colloids_start[c];
      int j1 = (c < s->N_colloids - 1) ? s->colloids_start[c + 1] - 1 : s->Nlist_colloids - 1;
      for (int j = j0; j <= j1; ++j) {
        int p = s->colloids_list[j];
        double px, py, pz = 0.0;
        if (dim == 2) {
          double x0 = s->x_center[j], y0 = s->y_center[j];
          px = x0 * ca - y0 * sa;
          py = x0 * sa + y0 * ca;
        } else {
          double qp[4] = {0, s->x_center[j], s->y_center[j], s->z_center[j]};
          double qinv[4] = {q[0], -q[1], -q[2], -q[3]};
          double t1[4], t2[4];
          orc_qmul(q, qp, t1);
          orc_qmul(t1, qinv, t2);
          px = t2[1];
          py = t2[2];
          pz = t2[3];
        }
        s->x[p] = px + s->coll_x[c];
        s->y[p] = py + s->coll_y[c];
        if (dim == 3) s->z[p] = pz + s->coll_z[c];
        if (s->x[p] < 0) s->x[p] = s->x[p] + L[0];
        if (s->x[p] > L[0]) s->x[p] = s->x[p] - L[0];
        if (s->wall == 0) {
          if (s->y[p] < 0) s->y[p] = s->y[p] + L[1];
          if (s->y[p] > L[1]) s->y[p] = s->y[p] - L[1];
        }
        if (dim == 3) {
          if (s->z[p] < 0) s->z[p] = s->z[p] + L[2];
          if (s->z[p] > L[2]) s->z[p] = s->z[p] - L[2];
        }
      }
    }
  }
}

/* kernel_move_sys_VV_part2.cu:13-58 + kernel_move_colloids_VV_part2.cu:14-46 */
void orc_vv_step2(orc_sys* s) {
  int dim = s->dim;
  double dt = s->in.dt;
  for (int i = 0; i < s->N; ++i) {
    if (s->type[i] != 0) continue;
    double h = 0.5 * dt;
    double hm = h / s->mass[i];
    s->vx[i] = s->vx[i] + hm * s->fx[i];
    s->vy[i] = s->vy[i] + hm * s->fy[i];
    s->cxx[i] = s->cxx[i] + h * s->dcdt_xx[i];
    s->cxy[i] = s->cxy[i] + h * s->dcdt_xy[i];
    s->cyy[i] = s->cyy[i] + h * s->dcdt_yy[i];
    if (dim == 3) {
      s->vz[i] = s->vz[i] + hm * s->fz[i];
      s->cxz[i] = s->cxz[i] + h * s->dcdt_xz[i];
      s->cyz[i] = s->cyz[i] + h * s->dcdt_yz[i];
      s->czz[i] = s->czz[i] + h * s->dcdt_zz[i];
    }
  }
  if (s->in.coll_move == 0 && s->N_colloids > 0) {
    double hm = 0.5 * dt / s->coll_mass, hI = 0.5 * dt / s->coll_I;
    for (int c = 0; c < s->N_colloids; ++c) {
      s->coll_vx[c] += hm * s->fx_colloid[c];
      s->coll_vy[c] += hm * s->fy_colloid[c];
      if (dim == 3) s->coll_vz[c] += hm * s->fz_colloid[c];
      s->coll_omegaz[c] += hI * s->tz_colloid[c];
      if (dim == 3) {
        s->coll_omegax[c] += hI * s->tx_colloid[c];
        s->coll_omegay[c] += hI * s->ty_colloid[c];
      }
    }
  }
}

/* kernel_calculate_macro_vars.cu:14-40, summed in id order (the reference's atomicAdd
   order is not deterministic) */
double orc_kinetic_energy(const orc_sys* s) {
  double ke = 0.0;
  for (int i = 0; i < s->N; ++i) {
    double v2 = s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i];
    if (s->dim == 3) v2 = s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
    ke += 0.5 * s->mass[i] * v2;
  }
  return ke;
}

/* The driver loop of main.cu:290-467: step 0 = initial search + forces, then per step
   VV1 -> search -> m(t) -> forces -> VV2.  Returns nonzero if a hash left the grid. */
int orc_run(orc_sys* s, int nsteps) {
  double* m = s->magnetic_mom;
  if (!s->started) {
    s->started = 1;
    double ang = s->omega_magnet * s->in.t0;
    m[0] = cos(ang);
    m[1] = sin(ang);
    m[2] = 0.0;
    if (orc_neighbours_search(s)) return 1;
    orc_calculate_forces(s, m);
  }
  for (int k = 0; k < nsteps; ++k) {
    int step = s->step + 1;
    orc_vv_step1(s);
    if (orc_neighbours_search(s)) return 1;
    double ang = s->omega_magnet * (s->in.t0 + s->in.dt * (double)step);
    m[0] = cos(ang);
    m[1] = sin(ang);
    m[2] = 0.0;
    orc_calculate_forces(s, m);
    orc_vv_step2(s);
    s->step = step;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Flat accessors for the ctypes binding                                                 */
/* ------------------------------------------------------------------------------------ */
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

orc_sys* orc_create_from_file(const char* input_path, const char* particles_path, char* msg,
                              size_t cap) {
  orc_input in;
  if (orc_read_input(input_path, &in, msg, cap)) return NULL;
  return orc_create(&in, particles_path, msg, cap);
}

/* double fields, in this order; lengths by orc_field_len */
enum {
  OF_X, OF_Y, OF_Z, OF_VX, OF_VY, OF_VZ, OF_FX, OF_FY, OF_FZ, OF_DENS, OF_PRESS, OF_MASS,
  OF_CXX, OF_CXY, OF_CYY, OF_CXZ, OF_CYZ, OF_CZZ, OF_DCDT_XX, OF_DCDT_XY, OF_DCDT_YY,
  OF_DCDT_XZ, OF_DCDT_YZ, OF_DCDT_ZZ, OF_GXX, OF_GXY, OF_GXZ, OF_GYX, OF_GYY, OF_GYZ,
  OF_GZX, OF_GZY, OF_GZZ, OF_COLL_X, OF_COLL_Y, OF_COLL_Z, OF_COLL_VX, OF_COLL_VY,
  OF_COLL_VZ, OF_COLL_OX, OF_COLL_OY, OF_COLL_OZ, OF_COLL_THETA, OF_COLL_Q0, OF_COLL_QX,
  OF_COLL_QY, OF_COLL_QZ, OF_COLL_FX, OF_COLL_FY, OF_COLL_FZ, OF_COLL_TX, OF_COLL_TY,
  OF_COLL_TZ, OF_WALL_FX, OF_WALL_FY, OF_WALL_FZ, OF_XC, OF_YC, OF_ZC, OF_NFIELDS
};

double* orc_dfield(orc_sys* s, int f) {
  double* p[OF_NFIELDS] = {
      s->x, s->y, s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->dens, s->press, s->mass,
      s->cxx, s->cxy, s->cyy, s->cxz, s->cyz, s->czz, s->dcdt_xx, s->dcdt_xy, s->dcdt_yy,
      s->dcdt_xz, s->dcdt_yz, s->dcdt_zz, s->gxx, s->gxy, s->gxz, s->gyx, s->gyy, s->gyz,
      s->gzx, s->gzy, s->gzz, s->coll_x, s->coll_y, s->coll_z, s->coll_vx, s->coll_vy,
      s->coll_vz, s->coll_omegax, s->coll_omegay, s->coll_omegaz, s->coll_theta,
      s->coll_quat0, s->coll_quatx, s->coll_quaty, s->coll_quatz, s->fx_colloid,
      s->fy_colloid, s->fz_colloid, s->tx_colloid, s->ty_colloid, s->tz_colloid, s->fx_wall,
      s->fy_wall, s->fz_wall, s->x_center, s->y_center, s->z_center};
  return (f >= 0 && f < OF_NFIELDS) ? p[f] : NULL;
}

int orc_field_len(const orc_sys* s, int f) {
  if (f < OF_COLL_X) return s->N;
  if (f < OF_WALL_FX) return s->N_colloids;
  if (f < OF_XC) return s->Nwalls;
  return s->Nlist_colloids;
}

/* int fields: 0 type, 1 particle_cell, 2 particle_index, 3 cell_start, 4 cell_end,
   5 walls_list, 6 walls_start, 7 colloids_list, 8 colloids_start, 9 coll_cell,
   10 coll_index, 11 coll_cell_start, 12 coll_cell_end */
int* orc_ifield(orc_sys* s, int f, int* len) {
  int* p[13] = {s->type, s->particle_cell, s->particle_index, s->cell_start, s->cell_end,
                s->walls_list, s->walls_start, s->colloids_list, s->colloids_start,
                s->coll_cell, s->coll_index, s->coll_cell_start, s->coll_cell_end};
  int n[13] = {s->N, s->N, s->N, s->Ntotal_cells, s->Ntotal_cells, s->Nlist_walls,
               s->Nwalls, s->Nlist_colloids, s->N_colloids, s->N_colloids, s->N_colloids,
               s->Ntotal_cells_colloids, s->Ntotal_cells_colloids};
  if (f < 0 || f >= 13) return NULL;
  if (len) *len = n[f];
  return p[f];
}

/* scalar summary: ints[0..15], dbls[0..39] */
void orc_info(const orc_sys* s, int* ints, double* d) {
  int iv[16] = {s->N, s->dim, s->wall, s->Ncells[0], s->Ncells[1], s->Ncells[2],
                s->Ntotal_cells, s->Nwalls, s->Nlist_walls, s->N_colloids,
                s->Nlist_colloids, s->Ncells_colloids[0], s->Ncells_colloids[1],
                s->Ncells_colloids[2], s->Ntotal_cells_colloids, s->step};
  double dv[40] = {s->rcut, s->rcutsq, s->rcut_inv, s->cw, s->c_gradw, s->csq, s->rho0,
                   s->a, s->b, s->nkT, s->tau, s->in.dt, s->cell_size[0], s->cell_size[1],
                   s->cell_size[2], s->wall_width, s->y_bottom, s->y_top, s->V_bottom,
                   s->V_top, s->coll_R, s->coll_mass, s->coll_I, s->rcuton_coll_rep_sq,
                   s->rcutoff_coll_rep_sq, s->r0_magnet_sq, s->F0_rep, s->tau_rep,
                   s->F0_magnet, s->omega_magnet, s->ky, s->beta_max, s->L[0], s->L[1],
                   s->L[2], s->cell_colloids_size[0], s->cell_colloids_size[1],
                   s->cell_colloids_size[2], s->in.t0, orc_kinetic_energy(s)};
  memcpy(ints, iv, sizeof(iv));
  memcpy(d, dv, sizeof(dv));
}

double* orc_magnetic_mom(orc_sys* s) { return s->magnetic_mom; }
