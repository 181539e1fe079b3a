// ref_harness.cu -- driver for the reference program's own CUDA build (test infrastructure).
//
// Linked against the reference's objects compiled from their sources where they lie
// (oracle/Makefile, target `ref`), in place of the reference's main.cu.  It drives the
// reference's class_system methods in the order of main.cu:95-467 and adds two things the
// reference's driver does not have:
//   dump <outdir> <s1,s2,...>  binary dumps of every device array (original particle order)
//                              after the initial forces (step 0) and after the listed steps
//   time <steps> <warmup>      CUDA-event timing of the step loop, printed as one JSON line
// It reads ./input (and ./input_particles.in when new_sim = 1) from the working directory,
// as the reference does.  It changes no arithmetic of the reference: every number comes
// from the reference's own kernels.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <chrono>
#include <string>
#include <vector>
#include <sys/stat.h>
#include "class_system.h"
#include "kernel_functions.h"

namespace {

struct DevState {
  real *x, *y, *z, *vx, *vy, *vz, *mass, *fx, *fy, *fz, *dens, *press;
  int *particle_cell, *particle_index, *cell_start, *cell_end;
  real* kin_energy;
  int* type;
  real *cxx, *cxy, *cyy, *cxz, *cyz, *czz;
  real *dxx, *dxy, *dyy, *dxz, *dyz, *dzz;
  real *gxx, *gxy, *gxz, *gyx, *gyy, *gyz, *gzx, *gzy, *gzz;
  real *fx_wall, *fy_wall, *fz_wall;
  int *walls_list, *walls_start, *colloids_list, *colloids_start;
  real *coll_x, *coll_y, *coll_z, *coll_vx, *coll_vy, *coll_vz;
  real *coll_ox, *coll_oy, *coll_oz, *coll_theta, *q0, *qx, *qy, *qz;
  real *x_center, *y_center, *z_center;
  real *fx_coll, *fy_coll, *fz_coll, *tx_coll, *ty_coll, *tz_coll;
  int *coll_cell, *coll_index, *coll_cell_start, *coll_cell_end;
  real* magnetic_mom;
};

struct Inputs {
  int Nxyz[3] = {20, 20, 20};
  real L[3] = {1.0, 1.0, 1.0};
  int dim = 2;
  real dt = 0.01, t0 = 0.0;
  int Nsteps = 0;
  real overlap = 4.0, rho = 1.0, c = 1.0, P0 = 1.0, eta = 1.0, zeta = 0.0, np = 1.0,
       kT = 1.0, tau = 1.0;
  int ext_type = 0;
  real ext[3] = {0, 0, 0};
  int f_micro = 1000, f_macro = 100, f_walls = 1000, f_coll = 1000;
  int wall = 0;
  real Vtop = 0.0, Vbottom = 0.0;
  int Ncoll = 0;
  real R = 1.0, crho = 1.0;
  real cx[MAX_COLLOIDS][MAX_VALUES_PER_COLLOID];
  int coll_move = 0;
  real cuton = 0.001, F0r = 1.0, taur = 0.01, cutm = 0.1, F0m = 1.0, omm = 0.01;
  int new_sim = 0;
};

// Every __constant__ of kernel_declare_constants.cu, uploaded as main.cu:185-236 does.
void upload_constants(class_system& s, real dt) {
#define UP(sym, val, n) cudaMemcpyToSymbol(sym, &(val), (n))
  UP(N, s.N, sizeof(int));
  UP(dim, s.dim, sizeof(int));
  UP(L, s.L, sizeof(real) * 3);
  UP(cw, s.cw, sizeof(real));
  UP(c_gradw, s.c_gradw, sizeof(real));
  UP(rcut, s.rcut, sizeof(real));
  UP(rcutsq, s.rcutsq, sizeof(real));
  UP(rcut_inv, s.rcut_inv, sizeof(real));
  UP(csq, s.csq, sizeof(real));
  UP(rho0, s.rho0, sizeof(real));
  UP(a, s.a, sizeof(real));
  UP(b, s.b, sizeof(real));
  UP(nkT, s.nkT, sizeof(real));
  UP(tau, s.tau, sizeof(real));
  cudaMemcpyToSymbol(::dt, &dt, sizeof(real));
  UP(cell_size, s.cell_size, sizeof(real) * 3);
  UP(Ncells, s.Ncells, sizeof(int) * 3);
  UP(Ntotal_cells, s.Ntotal_cells, sizeof(int));
  UP(ext_force_type, s.ext_force_type, sizeof(int));
  UP(ext_force, s.ext_force, sizeof(real) * 3);
  UP(ky, s.ky, sizeof(real));
  UP(wall, s.wall, sizeof(int));
  UP(y_bottom, s.y_bottom, sizeof(real));
  UP(y_top, s.y_top, sizeof(real));
  UP(V_bottom, s.V_bottom, sizeof(real));
  UP(V_top, s.V_top, sizeof(real));
  UP(Nwalls, s.Nwalls, sizeof(int));
  UP(Nlist_walls, s.Nlist_walls, sizeof(int));
  UP(N_colloids, s.N_colloids, sizeof(int));
  UP(Nlist_colloids, s.Nlist_colloids, sizeof(int));
  UP(coll_R, s.coll_R, sizeof(real));
  UP(coll_rho, s.coll_rho, sizeof(real));
  UP(coll_mass, s.coll_mass, sizeof(real));
  UP(coll_I, s.coll_I, sizeof(real));
  UP(beta_max, s.beta_max, sizeof(real));
  UP(wall_width, s.wall_width, sizeof(real));
  UP(coll_rep_cuton, s.coll_rep_cuton, sizeof(real));
  UP(coll_rep_cutoff, s.coll_rep_cutoff, sizeof(real));
  UP(rcutoff_coll_rep, s.rcutoff_coll_rep, sizeof(real));
  UP(rcuton_coll_rep, s.rcuton_coll_rep, sizeof(real));
  UP(rcutoff_coll_rep_sq, s.rcutoff_coll_rep_sq, sizeof(real));
  UP(rcuton_coll_rep_sq, s.rcuton_coll_rep_sq, sizeof(real));
  UP(rcutoff_coll, s.rcutoff_coll, sizeof(real));
  UP(rcutoff_coll_sq, s.rcutoff_coll_sq, sizeof(real));
  UP(cell_colloids_size, s.cell_colloids_size, sizeof(real) * 3);
  UP(Ncells_colloids, s.Ncells_colloids, sizeof(int) * 3);
  UP(Ntotal_cells_colloids, s.Ntotal_cells_colloids, sizeof(int));
  UP(F0_rep, s.F0_rep, sizeof(real));
  UP(tau_rep, s.tau_rep, sizeof(real));
  UP(r0_magnet, s.r0_magnet, sizeof(real));
  UP(r0_magnet_sq, s.r0_magnet_sq, sizeof(real));
  UP(F0_magnet, s.F0_magnet, sizeof(real));
#undef UP
}

// One record: 32-byte name, int32 dtype (0 = real, 1 = int32), int32 element size,
// int64 count, then the raw data.
void put(FILE* f, const char* name, const void* dev, long long n, int is_int) {
  char nm[32];
  memset(nm, 0, sizeof(nm));
  strncpy(nm, name, 31);
  int code = is_int, esz = is_int ? (int)sizeof(int) : (int)sizeof(real);
  fwrite(nm, 1, 32, f);
  fwrite(&code, 4, 1, f);
  fwrite(&esz, 4, 1, f);
  fwrite(&n, 8, 1, f);
  std::vector<char> buf((size_t)(n > 0 ? n : 0) * esz);
  if (n > 0 && dev) cudaMemcpy(buf.data(), dev, buf.size(), cudaMemcpyDeviceToHost);
  fwrite(buf.data(), 1, buf.size(), f);
}

int dump(const char* dir, int step, class_system& s, DevState& d) {
  char path[1024];
  snprintf(path, sizeof(path), "%s/ref_step%06d.bin", dir, step);
  FILE* f = fopen(path, "wb");
  if (!f) return 1;
  long long N = s.N, nc = s.N_colloids, nw = s.Nwalls, cells = s.Ntotal_cells;
  put(f, "x", d.x, N, 0); put(f, "y", d.y, N, 0); put(f, "z", d.z, N, 0);
  put(f, "vx", d.vx, N, 0); put(f, "vy", d.vy, N, 0); put(f, "vz", d.vz, N, 0);
  put(f, "fx", d.fx, N, 0); put(f, "fy", d.fy, N, 0); put(f, "fz", d.fz, N, 0);
  put(f, "mass", d.mass, N, 0); put(f, "dens", d.dens, N, 0); put(f, "press", d.press, N, 0);
  put(f, "type", d.type, N, 1);
  put(f, "cxx", d.cxx, N, 0); put(f, "cxy", d.cxy, N, 0); put(f, "cyy", d.cyy, N, 0);
  put(f, "cxz", d.cxz, N, 0); put(f, "cyz", d.cyz, N, 0); put(f, "czz", d.czz, N, 0);
  put(f, "dcdt_xx", d.dxx, N, 0); put(f, "dcdt_xy", d.dxy, N, 0); put(f, "dcdt_yy", d.dyy, N, 0);
  put(f, "dcdt_xz", d.dxz, N, 0); put(f, "dcdt_yz", d.dyz, N, 0); put(f, "dcdt_zz", d.dzz, N, 0);
  put(f, "gxx", d.gxx, N, 0); put(f, "gxy", d.gxy, N, 0); put(f, "gxz", d.gxz, N, 0);
  put(f, "gyx", d.gyx, N, 0); put(f, "gyy", d.gyy, N, 0); put(f, "gyz", d.gyz, N, 0);
  put(f, "gzx", d.gzx, N, 0); put(f, "gzy", d.gzy, N, 0); put(f, "gzz", d.gzz, N, 0);
  put(f, "particle_cell", d.particle_cell, N, 1);
  put(f, "particle_index", d.particle_index, N, 1);
  put(f, "cell_start", d.cell_start, cells, 1);
  put(f, "cell_end", d.cell_end, cells, 1);
  if (s.wall) {
    put(f, "fx_wall", d.fx_wall, nw, 0); put(f, "fy_wall", d.fy_wall, nw, 0);
    put(f, "fz_wall", d.fz_wall, nw, 0);
  }
  if (nc > 0) {
    put(f, "coll_x", d.coll_x, nc, 0); put(f, "coll_y", d.coll_y, nc, 0);
    put(f, "coll_z", d.coll_z, nc, 0); put(f, "coll_vx", d.coll_vx, nc, 0);
    put(f, "coll_vy", d.coll_vy, nc, 0); put(f, "coll_vz", d.coll_vz, nc, 0);
    put(f, "coll_omegax", d.coll_ox, nc, 0); put(f, "coll_omegay", d.coll_oy, nc, 0);
    put(f, "coll_omegaz", d.coll_oz, nc, 0); put(f, "coll_theta", d.coll_theta, nc, 0);
    put(f, "coll_quat0", d.q0, nc, 0); put(f, "coll_quatx", d.qx, nc, 0);
    put(f, "coll_quaty", d.qy, nc, 0); put(f, "coll_quatz", d.qz, nc, 0);
    put(f, "fx_colloid", d.fx_coll, nc, 0); put(f, "fy_colloid", d.fy_coll, nc, 0);
    put(f, "fz_colloid", d.fz_coll, nc, 0); put(f, "tx_colloid", d.tx_coll, nc, 0);
    put(f, "ty_colloid", d.ty_coll, nc, 0); put(f, "tz_colloid", d.tz_coll, nc, 0);
    if (nc >= 2) {
      put(f, "coll_cell", d.coll_cell, nc, 1); put(f, "coll_index", d.coll_index, nc, 1);
      put(f, "coll_cell_start", d.coll_cell_start, s.Ntotal_cells_colloids, 1);
      put(f, "coll_cell_end", d.coll_cell_end, s.Ntotal_cells_colloids, 1);
    }
  }
  fclose(f);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: ref_sph dump <outdir> <s1,s2,...> | time <steps> <warmup>\n");
    return 2;
  }
  std::string mode = argv[1];
  Inputs in;
  class_system sys;
  int err = sys.read_input(in.Nxyz, in.L, in.dim, in.dt, in.t0, in.Nsteps, in.overlap, in.rho,
                           in.c, in.P0, in.eta, in.zeta, in.np, in.kT, in.tau, in.ext_type,
                           in.ext, in.f_micro, in.f_macro, in.f_walls, in.f_coll, in.wall,
                           in.Vtop, in.Vbottom, in.Ncoll, in.R, in.crho, in.cx, in.coll_move,
                           in.cuton, in.F0r, in.taur, in.cutm, in.F0m, in.omm, in.new_sim);
  if (err) return 3;
  sys.initialize_pointers();
  sys.constructor(in.Nxyz, in.wall, in.overlap, in.dim, in.Ncoll, in.new_sim);
  err = sys.initialize(in.Nxyz, in.L, in.dim, in.overlap, in.rho, in.c, in.P0, in.eta, in.zeta,
                       in.np, in.kT, in.tau, in.ext_type, in.ext, in.wall, in.Vtop, in.Vbottom,
                       in.Ncoll, in.R, in.crho, in.cx, in.cuton, in.F0r, in.taur, in.cutm,
                       in.F0m, in.omm, in.new_sim);
  if (err) return 4;
  upload_constants(sys, in.dt);
  DevState d;
  memset(&d, 0, sizeof(d));
  err = sys.copy_pointers_to_device(
      &d.x, &d.y, &d.z, &d.vx, &d.vy, &d.vz, &d.mass, &d.fx, &d.fy, &d.fz, &d.dens, &d.press,
      &d.particle_cell, &d.particle_index, &d.cell_start, &d.cell_end, &d.kin_energy, &d.type,
      &d.cxx, &d.cxy, &d.cyy, &d.cxz, &d.cyz, &d.czz, &d.dxx, &d.dxy, &d.dyy, &d.dxz, &d.dyz,
      &d.dzz, &d.gxx, &d.gxy, &d.gxz, &d.gyx, &d.gyy, &d.gyz, &d.gzx, &d.gzy, &d.gzz,
      &d.fx_wall, &d.fy_wall, &d.fz_wall, &d.walls_list, &d.walls_start, &d.colloids_list,
      &d.colloids_start, &d.coll_x, &d.coll_y, &d.coll_z, &d.coll_vx, &d.coll_vy, &d.coll_vz,
      &d.coll_ox, &d.coll_oy, &d.coll_oz, &d.coll_theta, &d.q0, &d.qx, &d.qy, &d.qz,
      &d.x_center, &d.y_center, &d.z_center, &d.fx_coll, &d.fy_coll, &d.fz_coll, &d.tx_coll,
      &d.ty_coll, &d.tz_coll, &d.coll_cell, &d.coll_index, &d.coll_cell_start,
      &d.coll_cell_end, &d.magnetic_mom);
  if (err) return 5;
  dim3 tpb(128);
  dim3 nb((sys.N + tpb.x - 1) / tpb.x);

  auto search = [&]() {
    return sys.neighbours_search(nb, tpb, d.x, d.y, d.z, d.particle_cell, d.particle_index,
                                 d.cell_start, d.cell_end, d.coll_x, d.coll_y, d.coll_z,
                                 d.coll_cell, d.coll_index, d.coll_cell_start,
                                 d.coll_cell_end);
  };
  auto forces = [&]() {
    return sys.calculate_forces(
        nb, tpb, d.x, d.y, d.z, d.vx, d.vy, d.vz, d.cxx, d.cxy, d.cyy, d.cxz, d.cyz, d.czz,
        d.fx, d.fy, d.fz, d.dxx, d.dxy, d.dyy, d.dxz, d.dyz, d.dzz, d.gxx, d.gxy, d.gxz,
        d.gyx, d.gyy, d.gyz, d.gzx, d.gzy, d.gzz, d.press, d.dens, d.mass, d.particle_index,
        d.cell_start, d.cell_end, d.type, d.fx_wall, d.fy_wall, d.fz_wall, d.walls_list,
        d.walls_start, d.coll_x, d.coll_y, d.coll_z, d.coll_vx, d.coll_vy, d.coll_vz,
        d.coll_ox, d.coll_oy, d.coll_oz, d.fx_coll, d.fy_coll, d.fz_coll, d.tx_coll,
        d.ty_coll, d.tz_coll, d.colloids_list, d.colloids_start, d.coll_index,
        d.coll_cell_start, d.coll_cell_end, d.magnetic_mom);
  };
  auto set_moment = [&](double t) {
    real ang = sys.omega_magnet * t;
    real m[3] = {(real)cos(ang), (real)sin(ang), 0.0};
    if (d.magnetic_mom) cudaMemcpy(d.magnetic_mom, m, 3 * sizeof(real), cudaMemcpyHostToDevice);
  };
  auto one_step = [&](int step) {
    int e = sys.V_Verlet_step1(nb, tpb, d.x, d.y, d.z, d.vx, d.vy, d.vz, d.cxx, d.cxy, d.cyy,
                               d.cxz, d.cyz, d.czz, d.fx, d.fy, d.fz, d.dxx, d.dxy, d.dyy,
                               d.dxz, d.dyz, d.dzz, d.mass, d.type, d.coll_x, d.coll_y,
                               d.coll_z, d.coll_vx, d.coll_vy, d.coll_vz, d.coll_ox, d.coll_oy,
                               d.coll_oz, d.coll_theta, d.q0, d.qx, d.qy, d.qz, d.fx_coll,
                               d.fy_coll, d.fz_coll, d.tx_coll, d.ty_coll, d.tz_coll,
                               d.x_center, d.y_center, d.z_center, d.colloids_list,
                               d.colloids_start, in.coll_move);
    if (e) return e;
    if ((e = search())) return e;
    set_moment(in.t0 + in.dt * (double)step);
    if ((e = forces())) return e;
    return sys.V_Verlet_step2(nb, tpb, d.vx, d.vy, d.vz, d.cxx, d.cxy, d.cyy, d.cxz, d.cyz,
                              d.czz, d.fx, d.fy, d.fz, d.dxx, d.dxy, d.dyy, d.dxz, d.dyz,
                              d.dzz, d.mass, d.type, d.coll_vx, d.coll_vy, d.coll_vz,
                              d.coll_ox, d.coll_oy, d.coll_oz, d.fx_coll, d.fy_coll,
                              d.fz_coll, d.tx_coll, d.ty_coll, d.tz_coll, in.coll_move);
  };

  // main.cu:287-323: initial moment, search and forces
  set_moment(in.t0);
  if (search() || forces()) return 6;
  cudaDeviceSynchronize();

  if (mode == "dump" && argc >= 4) {
    const char* dir = argv[2];
    mkdir(dir, 0755);
    std::vector<int> want;
    for (char* t = strtok(argv[3], ","); t; t = strtok(nullptr, ",")) want.push_back(atoi(t));
    int last = 0;
    for (int w : want) last = w > last ? w : last;
    for (int w : want)
      if (w == 0 && dump(dir, 0, sys, d)) return 7;
    for (int step = 1; step <= last; ++step) {
      if (one_step(step)) return 8;
      for (int w : want)
        if (w == step) {
          cudaDeviceSynchronize();
          if (dump(dir, step, sys, d)) return 7;
        }
    }
    cudaError_t ce = cudaDeviceSynchronize();
    printf("{\"mode\": \"dump\", \"N\": %d, \"steps\": %d, \"cuda\": \"%s\"}\n", sys.N, last,
           cudaGetErrorString(ce));
    return ce == cudaSuccess ? 0 : 9;
  }
  if (mode == "time" && argc >= 4) {
    int steps = atoi(argv[2]), warm = atoi(argv[3]);
    int step = 0;
    for (int k = 0; k < warm; ++k)
      if (one_step(++step)) return 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    auto w0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0);
    for (int k = 0; k < steps; ++k)
      if (one_step(++step)) return 8;
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    auto w1 = std::chrono::steady_clock::now();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double wall = std::chrono::duration<double>(w1 - w0).count();
    cudaError_t ce = cudaGetLastError();
    printf("{\"mode\": \"time\", \"N\": %d, \"steps\": %d, \"warmup\": %d, \"event_s\": %.6f, "
           "\"wall_s\": %.6f, \"real_bytes\": %d, \"cuda\": \"%s\"}\n",
           sys.N, steps, warm, ms * 1e-3, wall, (int)sizeof(real), cudaGetErrorString(ce));
    return ce == cudaSuccess ? 0 : 9;
  }
  fprintf(stderr, "bad arguments\n");
  return 2;
}
