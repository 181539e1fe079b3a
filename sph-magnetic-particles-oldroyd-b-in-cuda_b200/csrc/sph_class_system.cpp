// sph_class_system.cpp -- class_system (src/class_system.h:12-650) over the C ABI.
//
// Every member function keeps the reference's parameters and 0 / 1 results.  The engine
// context (sph_capi.h) holds the state; the device buffers the caller passes are refreshed
// from it, in original particle order, by the output routines only.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "sph_class_system.h"
#include "sph_io.h"

struct class_system_engine {
  sph_input in;  // as read by read_input; initialize overrides what it is given
  std::vector<double> coll;
  bool have_input = false;
  sph_ctx* ctx = nullptr;
  // host storage behind the raw-pointer members
  std::vector<double> pf[15];  // x y z vx vy vz fx fy fz dens press mass cxx..czz below
  std::vector<double> conf[6];
  std::vector<int> type, walls_list, walls_start, colloids_list, colloids_start;
  std::vector<double> wall_f[3];
  std::vector<double> coll_state[SPH_NUM_COLLOID_FIELDS];
  std::vector<double> center[3];
  class_system_engine() { std::memset(&in, 0, sizeof(in)); }
};

namespace {

const char* last_error(const class_system_engine* e) {
  return (e && e->ctx) ? sph_last_error(e->ctx) : "";
}

// The reference reports CUDA errors with printf and returns 1 (e.g.
// system_neighbours_search.cu:40-45); so does the shim, with the engine's message.
int report(const class_system_engine* e, const char* where, sph_status s) {
  if (s == SPH_OK) return 0;
  std::printf("Error in %s: %s (%s)\n", where, sph_status_string(s), last_error(e));
  return 1;
}

bool engine_ready(const class_system_engine* e, const char* where) {
  if (e && e->ctx) return true;
  std::printf("Error in %s: the system is not initialized\n", where);
  return false;
}

// A failed call of the caller's own (e.g. the reference's driver copies the magnetic
// moment into a buffer it only allocates with colloids, main.cu:278-281) must not be
// reported as the engine's error.
void clear_stale_error() { cudaGetLastError(); }

int engine_precision() {
  const char* p = std::getenv("SPH_B200_PRECISION");
  return (p && std::strcmp(p, "mixed") == 0) ? SPH_PREC_MIXED : SPH_PREC_FP64;
}

// Copies an engine field into a caller-owned device buffer (original order).
sph_status sync_field(sph_ctx* ctx, int field, double* k) {
  return k ? sph_read_field_device(ctx, field, k) : SPH_OK;
}

template <typename T>
sph_status to_device(T* k, const T* h, size_t n) {
  if (!k || n == 0) return SPH_OK;
  return cudaMemcpy(k, h, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess ? SPH_OK
                                                                                   : SPH_ERR_CUDA;
}

template <typename T>
sph_status to_host(T* h, const T* k, size_t n) {
  if (!k || n == 0) return SPH_OK;
  return cudaMemcpy(h, k, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess ? SPH_OK
                                                                                   : SPH_ERR_CUDA;
}

}  // namespace

sph_ctx* class_system::engine() const { return shim_ ? shim_->ctx : nullptr; }

// ---------------------------------------------------------------------------- set-up

int class_system::read_input(int N_[3], double L_[3], int& dim_, double& delta_t, double& t_ini,
                             int& Nsteps, double& overlap, double& rho_, double& c_,
                             double& P0_, double& eta, double& zeta, double& np, double& kT,
                             double& elast_time, int& ext_force_type_, double ext_force_[3],
                             int& freq_micro, int& freq_macro, int& freq_walls,
                             int& freq_colloid, int& wall_, double& Vwall_top,
                             double& Vwall_bottom, int& N_coll, double& coll_radius,
                             double& col_density, double coll_x_data[][3], int& coll_move,
                             double& coll_repulsion_cuton, double& F0_repulsion,
                             double& tau_repulsion, double& cutoff_magnetic,
                             double& F0_magnetic, double& omega_magnetic, int& new_sim) {
  if (!shim_) shim_ = new class_system_engine;
  std::vector<double> buf(3 * (size_t)SPH_MAX_COLLOIDS);
  char msg[512] = {0};
  sph_input in;
  const sph_status s = sph_read_input("input", &in, buf.data(), SPH_MAX_COLLOIDS, msg,
                                      sizeof(msg));
  if (s != SPH_OK) {
    std::printf("Error reading the input file: %s\n", msg);
    return 1;
  }
  shim_->in = in;
  shim_->coll.assign(buf.begin(), buf.begin() + 3 * (size_t)in.N_colloids);
  shim_->in.coll_xyz = shim_->coll.empty() ? nullptr : shim_->coll.data();
  shim_->have_input = true;
  // components beyond dim keep the caller's values, as in system_read_input.cpp:115-131
  for (int d = 0; d < in.dim && d < 3; ++d) {
    N_[d] = in.N[d];
    L_[d] = in.L[d];
    ext_force_[d] = in.ext_force[d];
  }
  dim_ = in.dim;
  delta_t = in.dt;
  t_ini = in.t0;
  Nsteps = in.Nsteps;
  overlap = in.overlap;
  rho_ = in.rho;
  c_ = in.c;
  P0_ = in.P0;
  eta = in.eta;
  zeta = in.zeta;
  np = in.np;
  kT = in.kT;
  elast_time = in.tau;
  ext_force_type_ = in.ext_force_type;
  freq_micro = in.freq_micro;
  freq_macro = in.freq_macro;
  freq_walls = in.freq_walls;
  freq_colloid = in.freq_colloids;
  wall_ = in.wall;
  Vwall_top = in.Vwall_top;
  Vwall_bottom = in.Vwall_bottom;
  N_coll = in.N_colloids;
  coll_radius = in.coll_R;
  col_density = in.coll_rho;
  for (int i = 0; i < in.N_colloids; ++i)
    for (int d = 0; d < in.dim; ++d) coll_x_data[i][d] = shim_->coll[3 * i + d];
  coll_move = in.coll_move;
  coll_repulsion_cuton = in.coll_repulsion_cuton;
  F0_repulsion = in.F0_repulsion;
  tau_repulsion = in.tau_repulsion;
  cutoff_magnetic = in.cutoff_magnetic;
  F0_magnetic = in.F0_magnetic;
  omega_magnetic = in.omega_magnetic;
  new_sim = in.new_sim;
  return 0;
}

void class_system::initialize_pointers() {
  x = y = z = vx = vy = vz = fx = fy = fz = dens = press = mass = nullptr;
  type = nullptr;
  cxx_tensor = cxy_tensor = cyy_tensor = cxz_tensor = cyz_tensor = czz_tensor = nullptr;
  fx_wall = fy_wall = fz_wall = nullptr;
  walls_list = walls_start = colloids_list = colloids_start = nullptr;
  coll_x = coll_y = coll_z = coll_vx = coll_vy = coll_vz = nullptr;
  coll_omegax = coll_omegay = coll_omegaz = coll_theta = nullptr;
  coll_quat0 = coll_quatx = coll_quaty = coll_quatz = nullptr;
  x_center = y_center = z_center = nullptr;
  quat0 = quatx = quaty = quatz = nullptr;
  fx_colloid = fy_colloid = fz_colloid = tx_colloid = ty_colloid = tz_colloid = nullptr;
}

// The reference sizes its host arrays here (system_constructor.cpp:15-117); the shim
// sizes them in initialize, once the engine has built the particles.
void class_system::constructor(int Nxyz[3], int wall_, double overlap, int dim_, int N_coll,
                               int new_sim) {
  (void)Nxyz;
  (void)overlap;
  (void)N_coll;
  (void)new_sim;
  if (!shim_) shim_ = new class_system_engine;
  dim = dim_;
  Nwalls = wall_ ? 2 : 0;
  N = Nmax = 0;
}

int class_system::initialize(int Nxyz[3], double L_[3], int dim_, double overlap, double rho_,
                             double c_, double P0_, double eta, double zeta, double np,
                             double kT, double elast_time, int ext_force_type_,
                             double ext_force_[3], int wall_, double Vwall_top,
                             double Vwall_bottom, int N_coll, double coll_radius,
                             double coll_density, double coll_x_data[][3],
                             double coll_repulsion_cuton, double F0_repulsion,
                             double tau_repulsion, double cutoff_magnetic, double F0_magnetic,
                             double omega_magnetic, int new_sim) {
  if (!shim_) shim_ = new class_system_engine;
  class_system_engine& e = *shim_;
  if (e.ctx) {
    std::printf("Error in initialize: the system is already initialized\n");
    return 1;
  }
  // dt, t0, Nsteps, the output frequencies and coll_move come from read_input (the
  // reference passes dt to the device separately, main.cu:199)
  sph_input in = e.in;
  in.dim = dim_;
  for (int d = 0; d < 3; ++d) {
    in.N[d] = d < dim_ ? Nxyz[d] : 0;
    in.L[d] = d < dim_ ? L_[d] : 0.0;
    in.ext_force[d] = d < dim_ ? ext_force_[d] : 0.0;
  }
  in.overlap = overlap;
  in.rho = rho_;
  in.c = c_;
  in.P0 = P0_;
  in.eta = eta;
  in.zeta = zeta;
  in.np = np;
  in.kT = kT;
  in.tau = elast_time;
  in.ext_force_type = ext_force_type_;
  in.wall = wall_;
  in.Vwall_top = Vwall_top;
  in.Vwall_bottom = Vwall_bottom;
  in.N_colloids = N_coll;
  in.coll_R = coll_radius;
  in.coll_rho = coll_density;
  e.coll.assign(3 * (size_t)(N_coll > 0 ? N_coll : 0), 0.0);
  for (int i = 0; i < N_coll; ++i)
    for (int d = 0; d < dim_; ++d) e.coll[3 * i + d] = coll_x_data[i][d];
  in.coll_xyz = e.coll.empty() ? nullptr : e.coll.data();
  in.coll_repulsion_cuton = coll_repulsion_cuton;
  in.F0_repulsion = F0_repulsion;
  in.tau_repulsion = tau_repulsion;
  in.cutoff_magnetic = cutoff_magnetic;
  in.F0_magnetic = F0_magnetic;
  in.omega_magnetic = omega_magnetic;
  in.new_sim = new_sim;
  e.in = in;

  // host-side arrays of the initial state (walls / colloid lists, body frames)
  sph_info info;
  int n = 0;
  sph_status s = sph_host_setup(&in, nullptr, 0, nullptr, &n, &info);
  if (s != SPH_OK) return report(&e, "initialize", s);
  const size_t nn = (size_t)n;
  for (auto& v : e.pf) v.assign(nn, 0.0);
  for (auto& v : e.conf) v.assign(nn, 0.0);
  e.type.assign(nn, 0);
  e.walls_list.assign((size_t)info.Nlist_walls, 0);
  e.walls_start.assign(2, 0);
  e.colloids_list.assign((size_t)info.Nlist_colloids, 0);
  e.colloids_start.assign((size_t)info.N_colloids, 0);
  for (auto& v : e.center) v.assign((size_t)info.Nlist_colloids, 0.0);
  sph_host_state hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.x = e.pf[0].data(); hs.y = e.pf[1].data(); hs.z = e.pf[2].data();
  hs.vx = e.pf[3].data(); hs.vy = e.pf[4].data(); hs.vz = e.pf[5].data();
  hs.mass = e.pf[11].data();
  hs.cxx = e.conf[0].data(); hs.cxy = e.conf[1].data(); hs.cyy = e.conf[2].data();
  hs.cxz = e.conf[3].data(); hs.cyz = e.conf[4].data(); hs.czz = e.conf[5].data();
  hs.type = e.type.data();
  hs.walls_list = e.walls_list.data();
  hs.walls_start = e.walls_start.data();
  hs.colloids_list = e.colloids_list.data();
  hs.colloids_start = e.colloids_start.data();
  hs.x_center = e.center[0].data(); hs.y_center = e.center[1].data(); hs.z_center = e.center[2].data();
  s = sph_host_setup(&in, nullptr, n, &hs, &n, &info);
  if (s != SPH_OK) return report(&e, "initialize", s);

  // the engine (device state, neighbour lists, CUDA graphs)
  int device = 0;
  cudaGetDevice(&device);
  clear_stale_error();
  sph_options opt;
  std::memset(&opt, 0, sizeof(opt));
  opt.precision = engine_precision();
  opt.device = device;
  opt.use_graph = 1;
  s = sph_create(&in, nullptr, &opt, &e.ctx);
  if (s != SPH_OK) {
    std::printf("Error in initialize: %s\n", sph_status_string(s));
    e.ctx = nullptr;
    return 1;
  }
  s = sph_get_info(e.ctx, 0, &info);
  if (s != SPH_OK) return report(&e, "initialize", s);

  // scalars (system_constructor.cpp:15-79, system_initialize.cpp:47-262)
  N = info.N;
  Nmax = info.Nmax;
  dim = info.dim;
  for (int d = 0; d < 3; ++d) {
    L[d] = L_[d];
    cell_size[d] = info.cell_size[d];
    Ncells[d] = info.Ncells[d];
    cell_colloids_size[d] = info.cell_colloids_size[d];
    Ncells_colloids[d] = info.Ncells_colloids[d];
    ext_force[d] = d < dim_ ? ext_force_[d] : 0.0;
  }
  nkT = info.nkT;
  tau = info.tau;
  wall = info.wall;
  y_bottom = info.y_bottom;
  y_top = info.y_top;
  V_bottom = info.V_bottom;
  V_top = info.V_top;
  Nwalls = info.Nwalls;
  Nlist_walls = info.Nlist_walls;
  wall_width = info.wall_width;
  N_colloids = info.N_colloids;
  coll_R = info.coll_R;
  coll_rho = info.coll_rho;
  Nlist_colloids = info.Nlist_colloids;
  coll_mass = info.coll_mass;
  coll_I = info.coll_I;
  coll_rep_cutoff = info.coll_rep_cutoff;
  coll_rep_cuton = info.coll_rep_cuton;
  rcutoff_coll_rep = info.rcutoff_coll_rep;
  rcuton_coll_rep = info.rcuton_coll_rep;
  rcutoff_coll_rep_sq = info.rcutoff_coll_rep_sq;
  rcuton_coll_rep_sq = info.rcuton_coll_rep_sq;
  rcutoff_coll = info.rcutoff_coll;
  rcutoff_coll_sq = info.rcutoff_coll_sq;
  F0_rep = info.F0_rep;
  tau_rep = info.tau_rep;
  r0_magnet = info.r0_magnet;
  r0_magnet_sq = info.r0_magnet_sq;
  F0_magnet = info.F0_magnet;
  omega_magnet = info.omega_magnet;
  rcut = info.rcut;
  rcutsq = info.rcutsq;
  rcut_inv = info.rcut_inv;
  cw = info.cw;
  c_gradw = info.c_gradw;
  c = info.c;
  csq = info.csq;
  rho = info.rho;
  P0 = info.P0;
  rho0 = info.rho0;
  a = info.a;
  b = info.b;
  Ntotal_cells = info.Ntotal_cells;
  Ntotal_cells_colloids = info.Ntotal_cells_colloids;
  ext_force_type = info.ext_force_type;
  ky = info.ky;
  kin_energy = 0.0;
  beta_max = info.beta_max;

  // raw-pointer members over the shim's storage
  x = e.pf[0].data(); y = e.pf[1].data(); z = e.pf[2].data();
  vx = e.pf[3].data(); vy = e.pf[4].data(); vz = e.pf[5].data();
  fx = e.pf[6].data(); fy = e.pf[7].data(); fz = e.pf[8].data();
  dens = e.pf[9].data(); press = e.pf[10].data(); mass = e.pf[11].data();
  cxx_tensor = e.conf[0].data(); cxy_tensor = e.conf[1].data(); cyy_tensor = e.conf[2].data();
  cxz_tensor = e.conf[3].data(); cyz_tensor = e.conf[4].data(); czz_tensor = e.conf[5].data();
  type = e.type.data();
  for (auto& v : e.wall_f) v.assign((size_t)Nwalls, 0.0);
  fx_wall = Nwalls ? e.wall_f[0].data() : nullptr;
  fy_wall = Nwalls ? e.wall_f[1].data() : nullptr;
  fz_wall = Nwalls ? e.wall_f[2].data() : nullptr;
  walls_list = e.walls_list.empty() ? nullptr : e.walls_list.data();
  walls_start = wall ? e.walls_start.data() : nullptr;
  colloids_list = e.colloids_list.empty() ? nullptr : e.colloids_list.data();
  colloids_start = e.colloids_start.empty() ? nullptr : e.colloids_start.data();
  x_center = e.center[0].empty() ? nullptr : e.center[0].data();
  y_center = e.center[1].empty() ? nullptr : e.center[1].data();
  z_center = e.center[2].empty() ? nullptr : e.center[2].data();
  for (int k = 0; k < SPH_NUM_COLLOID_FIELDS; ++k) {
    e.coll_state[k].assign((size_t)N_colloids, 0.0);
    if (N_colloids > 0) {
      s = sph_read_colloid_field(e.ctx, k, e.coll_state[k].data());
      if (s != SPH_OK) return report(&e, "initialize", s);
    }
  }
  double** cf[SPH_NUM_COLLOID_FIELDS] = {
      &coll_x,     &coll_y,     &coll_z,      &coll_vx,     &coll_vy,
      &coll_vz,    &coll_omegax, &coll_omegay, &coll_omegaz, &coll_theta,
      &coll_quat0, &coll_quatx, &coll_quaty,  &coll_quatz,  &fx_colloid,
      &fy_colloid, &fz_colloid, &tx_colloid,  &ty_colloid,  &tz_colloid};
  for (int k = 0; k < SPH_NUM_COLLOID_FIELDS; ++k)
    *cf[k] = N_colloids > 0 ? e.coll_state[k].data() : nullptr;
  return 0;
}

// Both particle initialisations run inside initialize (sph_host_setup / sph_create); the
// reference calls them from there too (system_initialize.cpp:270-276).
int class_system::initialize_particles_new_sim(int Nxyz[3], double dx[3]) {
  (void)Nxyz;
  (void)dx;
  return engine_ready(shim_, "initialize_particles_new_sim") ? 0 : 1;
}

int class_system::initialize_particles_old_sim() {
  return engine_ready(shim_, "initialize_particles_old_sim") ? 0 : 1;
}

void class_system::print_info() {
  std::cout << " \n";
  std::cout << "------------------ System info -----------------------------\n";
  std::cout << "Number of particles, N                 = " << N << " \n";
  std::cout << "Number of particles reserved, Nmax     = " << Nmax << " \n";
  std::cout << "Box size, L                            = " << L[0] << " " << L[1];
  if (dim == 3) std::cout << " " << L[2];
  std::cout << " \n";
  std::cout << "Number of dimensions, dim              = " << dim << " \n";
  std::cout << "Cutoff radius, rcut                    = " << rcut << " \n";
  std::cout << "Normalization const of the kernel, cw  = " << cw << " \n";
  std::cout << "density, rho                           = " << rho << " \n";
  std::cout << "Speed of sound, c                      = " << c << " \n";
  std::cout << "Base density, rho0                     = " << rho0 << " \n";
  std::cout << "Transport coefficients a, b            = " << a << " " << b << " \n";
  std::cout << "np * kT, tau                           = " << nkT << " " << tau << "\n";
  std::cout << "Cell size                              = " << cell_size[0] << " "
            << cell_size[1] << " " << cell_size[2] << " \n";
  std::cout << "Number of cells                        = " << Ncells[0] << " " << Ncells[1]
            << " " << Ncells[2] << "\n";
  std::cout << "Total number of cells                  = " << Ntotal_cells << "\n";
  std::cout << "Type of external force, ext_force_type = " << ext_force_type << " \n";
  if (wall) {
    std::cout << "Walls at y                             = " << y_bottom << " " << y_top
              << ", velocities " << V_bottom << " " << V_top << "\n";
    std::cout << "Number of particles in walls list      = " << Nlist_walls << "\n";
  }
  std::cout << "Number of colloids, N_colloids         = " << N_colloids << "\n";
  if (N_colloids > 0) {
    std::cout << "Colloids radius, density, mass, I      = " << coll_R << " " << coll_rho
              << " " << coll_mass << " " << coll_I << "\n";
    std::cout << "Number of particles in colloids list   = " << Nlist_colloids << "\n";
  }
  std::cout << "Engine                                 = B200 ("
            << (engine_precision() == SPH_PREC_MIXED ? "mixed" : "fp64") << ")\n";
  std::cout << "------------------------------------------------------------\n";
}

int class_system::copy_pointers_to_device(
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
    double** k_magnetic_mom) {
  if (!engine_ready(shim_, "copy_pointers_to_device")) return 1;
  class_system_engine& e = *shim_;
  bool ok = true;
  // the reference's set of buffers and sizes (system_copy_pointers_to_device.cpp:104-230),
  // zero-filled where it zero-fills them
  auto dalloc = [&](auto** p, size_t n) {
    *p = nullptr;
    if (cudaMalloc((void**)p, (n ? n : 1) * sizeof(**p)) != cudaSuccess) ok = false;
    else if (cudaMemset(*p, 0, (n ? n : 1) * sizeof(**p)) != cudaSuccess) ok = false;
  };
  const size_t n = (size_t)N, nc = (size_t)N_colloids;
  for (double** p : {k_x, k_y, k_z, k_vx, k_vy, k_vz, k_mass, k_cxx, k_cxy, k_cyy, k_cxz, k_cyz,
                     k_czz, k_fx, k_fy, k_fz, k_dens, k_press, k_dcdt_xx, k_dcdt_xy, k_dcdt_yy,
                     k_dcdt_xz, k_dcdt_yz, k_dcdt_zz, k_gradvxx, k_gradvxy, k_gradvxz,
                     k_gradvyx, k_gradvyy, k_gradvyz, k_gradvzx, k_gradvzy, k_gradvzz})
    dalloc(p, n);
  dalloc(k_kin_energy, 1);
  dalloc(k_type, n);
  dalloc(k_particle_cell, n);
  dalloc(k_particle_index, n);
  dalloc(k_cell_start, (size_t)Ntotal_cells);
  dalloc(k_cell_end, (size_t)Ntotal_cells);
  if (wall) {
    dalloc(k_walls_list, (size_t)Nlist_walls);
    dalloc(k_walls_start, (size_t)Nwalls);
    dalloc(k_fx_wall, (size_t)Nwalls);
    dalloc(k_fy_wall, (size_t)Nwalls);
    dalloc(k_fz_wall, (size_t)Nwalls);
  }
  if (nc) {
    dalloc(k_colloids_list, (size_t)Nlist_colloids);
    dalloc(k_colloids_start, nc);
    for (double** p : {k_coll_x, k_coll_y, k_coll_z, k_coll_vx, k_coll_vy, k_coll_vz,
                       k_coll_omegax, k_coll_omegay, k_coll_omegaz, k_coll_theta, k_coll_quat0,
                       k_coll_quatx, k_coll_quaty, k_coll_quatz, k_fx_colloid, k_fy_colloid,
                       k_fz_colloid, k_tx_colloid, k_ty_colloid, k_tz_colloid})
      dalloc(p, nc);
    dalloc(k_x_center, (size_t)Nlist_colloids);
    dalloc(k_y_center, (size_t)Nlist_colloids);
    dalloc(k_z_center, (size_t)Nlist_colloids);
    dalloc(k_coll_cell, nc);
    dalloc(k_coll_index, nc);
    dalloc(k_coll_cell_start, (size_t)Ntotal_cells_colloids);
    dalloc(k_coll_cell_end, (size_t)Ntotal_cells_colloids);
    dalloc(k_magnetic_mom, 3);
  }
  if (!ok) {
    std::printf("Error in copy_pointers_to_device: cannot allocate device memory\n");
    return 1;
  }
  // initial state, as the reference uploads it
  sph_status s = SPH_OK;
  const double* hp[] = {x, y, z, vx, vy, vz, mass, cxx_tensor, cxy_tensor, cyy_tensor,
                        cxz_tensor, cyz_tensor, czz_tensor};
  double** kp[] = {k_x, k_y, k_z, k_vx, k_vy, k_vz, k_mass, k_cxx, k_cxy, k_cyy, k_cxz, k_cyz,
                   k_czz};
  for (int q = 0; q < 13 && s == SPH_OK; ++q) s = to_device(*kp[q], hp[q], n);
  if (s == SPH_OK) s = to_device(*k_type, type, n);
  if (s == SPH_OK && wall) {
    s = to_device(*k_walls_list, walls_list, (size_t)Nlist_walls);
    if (s == SPH_OK) s = to_device(*k_walls_start, walls_start, (size_t)Nwalls);
  }
  if (s == SPH_OK && nc) {
    s = to_device(*k_colloids_list, colloids_list, (size_t)Nlist_colloids);
    if (s == SPH_OK) s = to_device(*k_colloids_start, colloids_start, nc);
    double** kc[] = {k_coll_x, k_coll_y, k_coll_z, k_coll_vx, k_coll_vy, k_coll_vz,
                     k_coll_omegax, k_coll_omegay, k_coll_omegaz, k_coll_theta, k_coll_quat0,
                     k_coll_quatx, k_coll_quaty, k_coll_quatz};
    for (int q = 0; q < 14 && s == SPH_OK; ++q) s = to_device(*kc[q], e.coll_state[q].data(), nc);
    const double* hc[] = {x_center, y_center, z_center};
    double** kcc[] = {k_x_center, k_y_center, k_z_center};
    for (int q = 0; q < 3 && s == SPH_OK; ++q)
      s = to_device(*kcc[q], hc[q], (size_t)Nlist_colloids);
  }
  if (s != SPH_OK) {
    std::printf("Error in copy_pointers_to_device: %s\n", cudaGetErrorString(cudaGetLastError()));
    return 1;
  }
  return 0;
}

void class_system::destructor() {
  if (shim_) {
    sph_destroy(shim_->ctx);  // safe after a cudaDeviceReset of the caller
    delete shim_;
    shim_ = nullptr;
  }
  initialize_pointers();
}

// ---------------------------------------------------------------------- step methods

int class_system::neighbours_search(dim3, dim3, double*, double*, double*, int*, int*, int*,
                                    int*, double*, double*, double*, int*, int*, int*, int*) {
  if (!engine_ready(shim_, "neighbours_search")) return 1;
  clear_stale_error();
  return report(shim_, "neighbours_search", sph_neighbours_search(shim_->ctx));
}

int class_system::calculate_density(dim3, dim3, double*, double*, double*, double*, int*, int*,
                                    int*) {
  if (!engine_ready(shim_, "calculate_density")) return 1;
  clear_stale_error();
  return report(shim_, "calculate_density", sph_calculate_density(shim_->ctx));
}

int class_system::calculate_pressure(dim3, dim3, double*, double*, double*) {
  if (!engine_ready(shim_, "calculate_pressure")) return 1;
  clear_stale_error();
  return report(shim_, "calculate_pressure", sph_calculate_pressure(shim_->ctx));
}

namespace {
// The magnetic moment the caller uploaded (main.cu:278-281, 395-400); it exists only
// with colloids, as in the reference.
sph_status moment_arg(const class_system& s, const double* k_m, double m[3], bool* have) {
  *have = false;
  if (s.N_colloids <= 0 || !k_m) return SPH_OK;
  if (cudaMemcpy(m, k_m, 3 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return SPH_ERR_CUDA;
  *have = true;
  return SPH_OK;
}
}  // namespace

int class_system::calculate_forces(
    dim3, dim3, double*, double*, double*, double*, double*, double*, double*, double*, double*,
    double*, double*, double*, double*, double*, double*, double*, double*, double*, double*,
    double*, double*, double*, double*, double*, double*, double*, double*, double*, double*,
    double*, double*, double*, double*, int*, int*, int*, int*, double*, double*, double*,
    int*, int*, double*, double*, double*, double*, double*, double*, double*, double*, double*,
    double*, double*, double*, double*, double*, double*, int*, int*, int*, int*, int*,
    double* k_magnetic_mom) {
  if (!engine_ready(shim_, "calculate_forces")) return 1;
  clear_stale_error();
  double m[3];
  bool have = false;
  sph_status s = moment_arg(*this, k_magnetic_mom, m, &have);
  if (s == SPH_OK) s = sph_calculate_forces(shim_->ctx, have ? m : nullptr);
  return report(shim_, "calculate_forces", s);
}

int class_system::calculate_external_forces(dim3, dim3, double*, double*, double*, double*,
                                            double*, double*, double*, int*) {
  if (!engine_ready(shim_, "calculate_external_forces")) return 1;
  clear_stale_error();
  return report(shim_, "calculate_external_forces", sph_calculate_external_forces(shim_->ctx));
}

int class_system::calculate_force_walls(dim3, dim3, double*, double*, double*, double*, double*,
                                        double*, int*, int*) {
  if (!engine_ready(shim_, "calculate_force_walls")) return 1;
  clear_stale_error();
  return report(shim_, "calculate_force_walls", sph_calculate_force_walls(shim_->ctx));
}

int class_system::calculate_force_colloids(dim3, dim3, double*, double*, double*, double*,
                                           double*, double*, double*, double*, double*, double*,
                                           double*, double*, double*, double*, double*, int*,
                                           int*, int*, int*, int*, double* k_magnetic_mom) {
  if (!engine_ready(shim_, "calculate_force_colloids")) return 1;
  clear_stale_error();
  double m[3];
  bool have = false;
  sph_status s = moment_arg(*this, k_magnetic_mom, m, &have);
  if (s == SPH_OK) s = sph_calculate_force_colloids(shim_->ctx, have ? m : nullptr);
  return report(shim_, "calculate_force_colloids", s);
}

namespace {
// coll_move is an input-file setting of the engine; a different value per call cannot be
// honoured and is reported rather than ignored.
bool coll_move_ok(const class_system_engine* e, int coll_move, const char* where) {
  if (e->in.N_colloids == 0 || coll_move == e->in.coll_move) return true;
  std::printf("Error in %s: coll_move %d differs from the input file's %d\n", where,
              coll_move, e->in.coll_move);
  return false;
}
}  // namespace

int class_system::V_Verlet_step1(dim3, dim3, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, int*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, int*,
                                 int*, int coll_move) {
  if (!engine_ready(shim_, "V_Verlet_step1")) return 1;
  if (!coll_move_ok(shim_, coll_move, "V_Verlet_step1")) return 1;
  clear_stale_error();
  return report(shim_, "V_Verlet_step1", sph_vv_step1(shim_->ctx));
}

int class_system::V_Verlet_step2(dim3, dim3, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*, double*,
                                 int*, double*, double*, double*, double*, double*, double*,
                                 double*, double*, double*, double*, double*, double*,
                                 int coll_move) {
  if (!engine_ready(shim_, "V_Verlet_step2")) return 1;
  if (!coll_move_ok(shim_, coll_move, "V_Verlet_step2")) return 1;
  clear_stale_error();
  return report(shim_, "V_Verlet_step2", sph_vv_step2(shim_->ctx));
}

int class_system::calculate_vel_gradient(dim3, dim3, double*, double*, double*, double*,
                                         double*, double*, double*, double*, double*, double*,
                                         double*, double*, double*, double*, double*, double*,
                                         int*, int*, int*, int*, double*, double*, double*,
                                         double*, double*, double*, double*, double*, double*) {
  if (!engine_ready(shim_, "calculate_vel_gradient")) return 1;
  clear_stale_error();
  return report(shim_, "calculate_vel_gradient", sph_calculate_vel_gradient(shim_->ctx));
}

int class_system::export_cells(int* k_particle_cell, int* k_particle_index, int* k_cell_start,
                               int* k_cell_end) {
  if (!engine_ready(shim_, "export_cells")) return 1;
  clear_stale_error();
  return report(shim_, "export_cells",
                sph_export_cells(shim_->ctx, k_particle_cell, k_particle_index, k_cell_start,
                                 k_cell_end));
}

// --------------------------------------------------------------------------- output

void class_system::print_particles(double* k_x, double* k_y, double* k_z, double* k_vx,
                                   double* k_vy, double* k_vz, double* k_mass, double* k_dens,
                                   double* k_press, double* k_cxx, double* k_cxy,
                                   double* k_cyy, double* k_cxz, double* k_cyz, double* k_czz,
                                   int step) {
  if (!engine_ready(shim_, "print_particles")) return;
  clear_stale_error();
  sph_ctx* ctx = shim_->ctx;
  const int fields[15] = {SPH_X,   SPH_Y,   SPH_Z,   SPH_VX,  SPH_VY,  SPH_VZ,  SPH_MASS, SPH_DENS,
                          SPH_PRESS, SPH_CXX, SPH_CXY, SPH_CYY, SPH_CXZ, SPH_CYZ, SPH_CZZ};
  double* k[15] = {k_x, k_y, k_z, k_vx, k_vy, k_vz, k_mass, k_dens, k_press,
                   k_cxx, k_cxy, k_cyy, k_cxz, k_cyz, k_czz};
  double* h[15] = {x, y, z, vx, vy, vz, mass, dens, press,
                   cxx_tensor, cxy_tensor, cyy_tensor, cxz_tensor, cyz_tensor, czz_tensor};
  sph_status s = SPH_OK;
  // refresh the caller's buffers (on the engine's stream), then the host mirrors from them
  for (int q = 0; q < 15 && s == SPH_OK; ++q) s = sync_field(ctx, fields[q], k[q]);
  if (s == SPH_OK) s = sph_synchronize(ctx);
  for (int q = 0; q < 15 && s == SPH_OK; ++q)
    s = k[q] ? to_host(h[q], k[q], (size_t)N) : sph_read_field(ctx, fields[q], h[q]);
  if (s != SPH_OK) {
    report(shim_, "print_particles", s);
    return;
  }
  char filename[64];
  std::snprintf(filename, sizeof(filename), "micro-%d.dat", step);
  s = sph_write_micro(filename, dim, N, x, y, z, vx, vy, vz, mass, dens, press, type,
                      cxx_tensor, cxy_tensor, cyy_tensor, cxz_tensor, cyz_tensor, czz_tensor);
  if (s != SPH_OK) {
    std::printf("System print particle error: Error opening the file %s\n", filename);
    return;
  }
  std::printf("Micro file written. Time step %d\n", step);
}

void class_system::print_walls(double* k_fx_wall, double* k_fy_wall, double* k_fz_wall,
                               int step) {
  if (!engine_ready(shim_, "print_walls")) return;
  clear_stale_error();
  std::vector<double> wf(6, 0.0);
  sph_status s = sph_read_wall_forces(shim_->ctx, wf.data());  // box 0: 2 walls x 3
  if (s != SPH_OK) {
    report(shim_, "print_walls", s);
    return;
  }
  for (int w = 0; w < Nwalls && w < 2; ++w) {
    fx_wall[w] = wf[3 * w];
    fy_wall[w] = wf[3 * w + 1];
    fz_wall[w] = wf[3 * w + 2];
  }
  to_device(k_fx_wall, fx_wall, (size_t)Nwalls);
  to_device(k_fy_wall, fy_wall, (size_t)Nwalls);
  to_device(k_fz_wall, fz_wall, (size_t)Nwalls);
  char filename[64];
  std::snprintf(filename, sizeof(filename), "walls-%d.dat", step);
  if (sph_write_walls(filename, dim, Nwalls, fx_wall, fy_wall, fz_wall) != SPH_OK) {
    std::printf("System print walls error: Error opening the file %s\n", filename);
    return;
  }
  std::printf("Walls file written. Time step %d\n", step);
}

void class_system::print_colloids(double* k_coll_x, double* k_coll_y, double* k_coll_z,
                                  double* k_coll_vx, double* k_coll_vy, double* k_coll_vz,
                                  double* k_coll_omegax, double* k_coll_omegay,
                                  double* k_coll_omegaz, double* k_fx_colloid,
                                  double* k_fy_colloid, double* k_fz_colloid,
                                  double* k_tx_colloid, double* k_ty_colloid,
                                  double* k_tz_colloid, int step) {
  if (!engine_ready(shim_, "print_colloids")) return;
  clear_stale_error();
  class_system_engine& e = *shim_;
  // file columns (3D order) and the engine's colloid fields behind them
  const int fields[15] = {SPH_COLL_X,      SPH_COLL_Y,      SPH_COLL_Z,      SPH_COLL_VX,
                          SPH_COLL_VY,     SPH_COLL_VZ,     SPH_COLL_OMEGAX, SPH_COLL_OMEGAY,
                          SPH_COLL_OMEGAZ, SPH_COLL_FX,     SPH_COLL_FY,     SPH_COLL_FZ,
                          SPH_COLL_TX,     SPH_COLL_TY,     SPH_COLL_TZ};
  double* k[15] = {k_coll_x, k_coll_y, k_coll_z, k_coll_vx, k_coll_vy, k_coll_vz,
                   k_coll_omegax, k_coll_omegay, k_coll_omegaz, k_fx_colloid, k_fy_colloid,
                   k_fz_colloid, k_tx_colloid, k_ty_colloid, k_tz_colloid};
  const double* cols[15];
  for (int q = 0; q < 15; ++q) {
    std::vector<double>& h = e.coll_state[fields[q]];
    sph_status s = sph_read_colloid_field(e.ctx, fields[q], h.data());
    if (s != SPH_OK) {
      report(shim_, "print_colloids", s);
      return;
    }
    to_device(k[q], h.data(), (size_t)N_colloids);
    cols[q] = h.data();
  }
  char filename[64];
  std::snprintf(filename, sizeof(filename), "colloids-%d.dat", step);
  if (sph_write_colloids(filename, dim, N_colloids, cols) != SPH_OK) {
    std::printf("System print colloids error: Error opening the file %s\n", filename);
    return;
  }
  std::printf("Colloids file written. Time step %d\n", step);
}

void class_system::print_particles_gradv(double* k_x, double* k_y, double* k_z,
                                         double* k_gradvxx, double* k_gradvxy,
                                         double* k_gradvxz, double* k_gradvyx,
                                         double* k_gradvyy, double* k_gradvyz,
                                         double* k_gradvzx, double* k_gradvzy,
                                         double* k_gradvzz, int step) {
  if (!engine_ready(shim_, "print_particles_gradv")) return;
  clear_stale_error();
  sph_ctx* ctx = shim_->ctx;
  std::vector<std::vector<double>> g(9, std::vector<double>((size_t)N));
  double* kg[9] = {k_gradvxx, k_gradvxy, k_gradvxz, k_gradvyx, k_gradvyy,
                   k_gradvyz, k_gradvzx, k_gradvzy, k_gradvzz};
  sph_status s = SPH_OK;
  // sph_read_field waits for the engine's stream, so the buffer refreshes have landed too
  for (int q = 0; q < 9 && s == SPH_OK; ++q) {
    s = sync_field(ctx, SPH_GXX + q, kg[q]);
    if (s == SPH_OK) s = sph_read_field(ctx, SPH_GXX + q, g[q].data());
  }
  double* kx[3] = {k_x, k_y, k_z};
  double* hx[3] = {x, y, z};
  for (int q = 0; q < 3 && s == SPH_OK; ++q) {
    s = sync_field(ctx, SPH_X + q, kx[q]);
    if (s == SPH_OK) s = sph_read_field(ctx, SPH_X + q, hx[q]);
  }
  if (s != SPH_OK) {
    report(shim_, "print_particles_gradv", s);
    return;
  }
  const double* gp[9];
  for (int q = 0; q < 9; ++q) gp[q] = g[q].data();
  char filename[64];
  std::snprintf(filename, sizeof(filename), "gradv-%d.dat", step);
  if (sph_write_gradv(filename, dim, N, x, y, z, gp) != SPH_OK) {
    std::printf("System print particles gradv error: Error opening the file %s\n", filename);
    return;
  }
  std::printf("gradv file written. Time step %d\n", step);
}

void class_system::print_macro_vars(dim3, dim3, double*, double*, double*, double*,
                                    double* k_energy, int step) {
  if (!engine_ready(shim_, "print_macro_vars")) return;
  clear_stale_error();
  double ke = 0.0;
  sph_status s = sph_kinetic_energy(shim_->ctx, &ke);
  if (s != SPH_OK) {
    report(shim_, "print_macro_vars", s);
    return;
  }
  kin_energy = ke;
  to_device(k_energy, &ke, 1);
  if (sph_append_macro("macro.dat", step, ke) != SPH_OK)
    std::printf("System print macro vars error: Error opening the file macro.dat\n");
}

// system_print_output.cpp:58-82
void class_system::print_output(
    dim3 numBlocks, dim3 threadsPerBlock, double* k_x, double* k_y, double* k_z, double* k_vx,
    double* k_vy, double* k_vz, double* k_fx, double* k_fy, double* k_fz, double* k_mass,
    double* k_dens, double* k_press, double* k_cxx, double* k_cxy, double* k_cyy,
    double* k_cxz, double* k_cyz, double* k_czz, double* k_fx_wall, double* k_fy_wall,
    double* k_fz_wall, double* k_coll_x, double* k_coll_y, double* k_coll_z,
    double* k_coll_vx, double* k_coll_vy, double* k_coll_vz, double* k_coll_omegax,
    double* k_coll_omegay, double* k_coll_omegaz, double* k_fx_colloid, double* k_fy_colloid,
    double* k_fz_colloid, double* k_tx_colloid, double* k_ty_colloid, double* k_tz_colloid,
    double* k_kin_energy, int freq_micro, int freq_walls, int freq_colloids, int freq_macro,
    int step) {
  (void)k_fx;
  (void)k_fy;
  (void)k_fz;
  if (freq_micro != 0 && step % freq_micro == 0)
    print_particles(k_x, k_y, k_z, k_vx, k_vy, k_vz, k_mass, k_dens, k_press, k_cxx, k_cxy,
                    k_cyy, k_cxz, k_cyz, k_czz, step);
  if (wall == 1 && freq_walls != 0 && step % freq_walls == 0)
    print_walls(k_fx_wall, k_fy_wall, k_fz_wall, step);
  if (N_colloids > 0 && freq_colloids != 0 && step % freq_colloids == 0)
    print_colloids(k_coll_x, k_coll_y, k_coll_z, k_coll_vx, k_coll_vy, k_coll_vz,
                   k_coll_omegax, k_coll_omegay, k_coll_omegaz, k_fx_colloid, k_fy_colloid,
                   k_fz_colloid, k_tx_colloid, k_ty_colloid, k_tz_colloid, step);
  if (freq_macro != 0 && step % freq_macro == 0)
    print_macro_vars(numBlocks, threadsPerBlock, k_mass, k_vx, k_vy, k_vz, k_kin_energy, step);
}
