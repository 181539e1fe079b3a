// sph_setup.cpp -- host-side set-up of a box: the reference's input parser and the
// constructor / initialize / particle-initialisation steps of class_system, producing the
// initial state in the reference's original particle order.  One-time host work; the
// per-step hot path is in sph_kernels.cu.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <algorithm>
#include <cerrno>
#include <climits>
#include <thread>

#include "sph_internal.h"

namespace sph {
namespace {

std::string trim_line(const std::string& s) {
  // leading blanks/tabs and trailing blanks/tabs/newlines are removed
  // (system_read_input.cpp:103-108)
  size_t a = 0;
  while (a < s.size() && (s[a] == ' ' || s[a] == '\t')) ++a;
  size_t b = s.size();
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\n' || s[b - 1] == '\r'))
    --b;
  return s.substr(a, b - a);
}

// Minimum-image helper with the reference's conditional form.
inline double wrap_half(double d, double L) {
  if (d > 0.5 * L) d -= L;
  if (d < -0.5 * L) d += L;
  return d;
}

}  // namespace

// class_system::read_input (src/system_read_input.cpp:18-512)
sph_status parse_input_file(const char* path, sph_input* in, std::vector<double>* coll,
                            std::string* msg) {
  std::ifstream f(path);
  if (!f.is_open()) {
    *msg = std::string("cannot open input file ") + path;
    return SPH_ERR_IO;
  }
  std::memset(in, 0, sizeof(*in));
  coll->clear();
  std::map<std::string, int> seen;
  int dim_N = 0, dim_L = 0, dim_ef = 0, ncoll_lines = 0;
  std::string raw, var;
  while (std::getline(f, raw)) {
    std::string line = trim_line(raw);
    std::istringstream ss(line);
    std::string key;
    if (!(ss >> key)) continue;
    std::vector<double> v;
    double t;
    while (v.size() < 3 && (ss >> t)) v.push_back(t);
    int nv = (int)v.size();
    auto take = [&](const char* k) { seen[k] = 1; };
    if (key == "N" && (nv == 3 || nv == 2)) {
      for (int d = 0; d < nv; ++d) in->N[d] = (int)v[d];
      dim_N = nv;
      take("N");
    } else if (key == "L" && (nv == 3 || nv == 2)) {
      for (int d = 0; d < nv; ++d) in->L[d] = v[d];
      dim_L = nv;
      take("L");
    } else if (key == "ext_force" && (nv == 3 || nv == 2)) {
      for (int d = 0; d < nv; ++d) in->ext_force[d] = v[d];
      dim_ef = nv;
      take("ext_force");
    } else if (key == "coll_x") {
      // tokens split on single spaces, every token but the key is a coordinate (:243-268)
      if (nv >= 2 && in->N_colloids > 0) {
        if (ncoll_lines >= in->N_colloids) {
          *msg = "different coll_x entries than N_colloids";
          return SPH_ERR_BAD_INPUT;
        }
        std::vector<double> c;
        std::istringstream ts(line);
        std::string tok;
        while (std::getline(ts, tok, ' ')) {
          if (tok.empty() || tok == "coll_x") continue;
          c.push_back(std::atof(tok.c_str()));
        }
        if ((int)c.size() != in->dim) {
          *msg = "the number of dimensions of coll_x is not that of the system";
          return SPH_ERR_BAD_INPUT;
        }
        c.resize(3, 0.0);
        coll->insert(coll->end(), c.begin(), c.end());
        ++ncoll_lines;
      }
    } else if (nv >= 1) {
      double a = v[0];
      struct Key {
        const char* name;
        double* d;
        int* i;
      };
      const Key keys[] = {
          {"dim", nullptr, &in->dim}, {"dt", &in->dt, nullptr}, {"t0", &in->t0, nullptr},
          {"Nsteps", nullptr, &in->Nsteps}, {"overlap", &in->overlap, nullptr},
          {"rho", &in->rho, nullptr}, {"c", &in->c, nullptr}, {"P0", &in->P0, nullptr},
          {"eta", &in->eta, nullptr}, {"zeta", &in->zeta, nullptr}, {"np", &in->np, nullptr},
          {"kT", &in->kT, nullptr}, {"tau", &in->tau, nullptr},
          {"ext_force_type", nullptr, &in->ext_force_type},
          {"freq_micro", nullptr, &in->freq_micro}, {"freq_macro", nullptr, &in->freq_macro},
          {"freq_walls", nullptr, &in->freq_walls},
          {"freq_colloids", nullptr, &in->freq_colloids}, {"wall", nullptr, &in->wall},
          {"Vwall_top", &in->Vwall_top, nullptr}, {"Vwall_bottom", &in->Vwall_bottom, nullptr},
          {"N_colloids", nullptr, &in->N_colloids}, {"coll_R", &in->coll_R, nullptr},
          {"coll_rho", &in->coll_rho, nullptr}, {"coll_move", nullptr, &in->coll_move},
          {"coll_repulsion_cuton", &in->coll_repulsion_cuton, nullptr},
          {"F0_repulsion", &in->F0_repulsion, nullptr},
          {"tau_repulsion", &in->tau_repulsion, nullptr},
          {"cutoff_magnetic", &in->cutoff_magnetic, nullptr},
          {"F0_magnetic", &in->F0_magnetic, nullptr},
          {"omega_magnetic", &in->omega_magnetic, nullptr},
          {"new_sim", nullptr, &in->new_sim}};
      for (const Key& k : keys)
        if (key == k.name) {
          if (k.d) *k.d = a;
          if (k.i) *k.i = (int)a;
          seen[k.name] = 1;
          break;
        }
    }
  }
  const char* required[] = {
      "N", "L", "dim", "dt", "t0", "Nsteps", "overlap", "rho", "c", "P0", "eta", "zeta",
      "np", "kT", "tau", "ext_force_type", "ext_force", "freq_micro", "freq_macro",
      "freq_walls", "freq_colloids", "wall", "Vwall_top", "Vwall_bottom", "N_colloids",
      "coll_R", "coll_rho", "coll_move", "coll_repulsion_cuton", "F0_repulsion",
      "tau_repulsion", "cutoff_magnetic", "F0_magnetic", "omega_magnetic", "new_sim"};
  for (const char* r : required)
    if (!seen.count(r)) {
      *msg = std::string(r) + " was not read";
      return SPH_ERR_BAD_INPUT;
    }
  if (ncoll_lines != in->N_colloids) {
    *msg = "different number of coll_x lines than N_colloids";
    return SPH_ERR_BAD_INPUT;
  }
  if (in->dim != dim_N || in->dim != dim_L) {
    *msg = "dim is not compatible with the dimensions of N or L";
    return SPH_ERR_BAD_INPUT;
  }
  if (in->ext_force_type != 0 && in->dim != dim_ef) {
    *msg = "dim is not compatible with the dimensions of ext_force";
    return SPH_ERR_BAD_INPUT;
  }
  in->coll_xyz = coll->empty() ? nullptr : coll->data();
  return SPH_OK;
}

namespace {

// Validation of read_input that concerns values (system_read_input.cpp:426-506).
sph_status validate(const sph_input& in, std::string* msg) {
  if (in.dim != 2 && in.dim != 3) {
    *msg = "dim must be 2 or 3";
    return SPH_ERR_BAD_INPUT;
  }
  if (in.ext_force_type < 0 || in.ext_force_type > 3) {
    *msg = "ext_force_type is not available";
    return SPH_ERR_BAD_INPUT;
  }
  if (in.N_colloids < 0 || in.N_colloids > SPH_MAX_COLLOIDS) {
    *msg = "N_colloids is too high";
    return SPH_ERR_BAD_INPUT;
  }
  if (in.N_colloids > 0 && !in.coll_xyz) {
    *msg = "colloid positions missing";
    return SPH_ERR_BAD_INPUT;
  }
  for (int d = 0; d < in.dim; ++d)
    if (in.N[d] <= 0 || !(in.L[d] > 0)) {
      *msg = "N and L must be positive";
      return SPH_ERR_BAD_INPUT;
    }
  const int nc = in.N_colloids;
  const double* c = in.coll_xyz;
  if (nc >= 2) {
    for (int i = 0; i < nc; ++i)
      for (int d = 0; d < in.dim; ++d)
        if (c[3 * i + d] < 0 || c[3 * i + d] > in.L[d]) {
          *msg = "colloid is out of the simulation box";
          return SPH_ERR_BAD_INPUT;
        }
    for (int i = 0; i < nc; ++i)
      for (int j = i + 1; j < nc; ++j) {
        double dx = wrap_half(c[3 * i] - c[3 * j], in.L[0]);
        double dy = c[3 * i + 1] - c[3 * j + 1];
        if (in.wall == 0) dy = wrap_half(dy, in.L[1]);
        double r2 = dx * dx + dy * dy;
        if (in.dim == 3) {
          // the reference takes the z separation from y (system_read_input.cpp:485)
          double dz = wrap_half(c[3 * i + 1] - c[3 * j + 1], in.L[2]);
          r2 = dx * dx + dy * dy + dz * dz;
        }
        if (std::sqrt(r2) < 2 * in.coll_R) {
          *msg = "overlapping colloids";
          return SPH_ERR_BAD_INPUT;
        }
      }
  }
  return SPH_OK;
}

// Particle mass of the lattice (system_initialize_particles_new_sim.cpp:127-131).
double lattice_mass(const HostBox& hb, const int Nxyz[3]) {
  const BoxParams& p = hb.p;
  if (p.dim == 2)
    return hb.in.rho * p.L[0] * (p.L[1] + 2.0 * p.wall_width) / (Nxyz[0] * Nxyz[1]);
  return hb.in.rho * p.L[0] * (p.L[1] + 2.0 * p.wall_width) * p.L[2] /
         (Nxyz[0] * Nxyz[1] * Nxyz[2]);
}

sph_status colloid_shells(HostBox* hb, const double dx[3], int Nmax, std::string* msg);

// Lattice + colloid shells (system_initialize_particles_new_sim.cpp:16-253).
sph_status lattice_particles(HostBox* hb, const int Nxyz[3], const double dx[3], int Nmax,
                             std::string* msg) {
  BoxParams& p = hb->p;
  const int dim = p.dim;
  const double R2 = p.coll_R * p.coll_R;
  const int nk = dim == 3 ? Nxyz[2] : 1;
  hb->x.clear(); hb->y.clear(); hb->z.clear();
  for (int i = 0; i < Nxyz[0]; ++i)
    for (int j = 0; j < Nxyz[1]; ++j)
      for (int k = 0; k < nk; ++k) {
        double px = dx[0] / 2.0 + i * dx[0];
        double py = dx[1] / 2.0 + j * dx[1];
        if (p.wall) py = py - p.wall_width;
        double pz = dim == 3 ? dx[2] / 2.0 + k * dx[2] : 0.0;
        bool carved = false;
        for (int l = 0; l < p.N_colloids && !carved; ++l) {
          double rx = wrap_half(px - hb->coll_x[l], p.L[0]);
          double ry = py - hb->coll_y[l];
          if (p.wall == 0) ry = wrap_half(ry, p.L[1]);
          double r2 = rx * rx + ry * ry;
          if (dim == 3) {
            double rz = wrap_half(pz - hb->coll_z[l], p.L[2]);
            r2 = rx * rx + ry * ry + rz * rz;
          }
          carved = r2 <= R2;
        }
        if (carved) continue;
        hb->x.push_back(px);
        hb->y.push_back(py);
        hb->z.push_back(pz);
      }
  const size_t nfluid = hb->x.size();
  hb->type.assign(nfluid, 0);
  if (p.wall)
    for (size_t i = 0; i < nfluid; ++i)
      hb->type[i] = hb->y[i] < p.y_bottom ? 1 : (hb->y[i] > p.y_top ? 2 : 0);
  hb->mass.assign(nfluid, lattice_mass(*hb, Nxyz));
  hb->cxx.assign(nfluid, 1.0);
  hb->cyy.assign(nfluid, 1.0);
  hb->czz.assign(nfluid, 1.0);
  hb->cxy.assign(nfluid, 0.0);
  hb->cxz.assign(nfluid, 0.0);
  hb->cyz.assign(nfluid, 0.0);
  return colloid_shells(hb, dx, Nmax, msg);
}

// Colloid shells (system_initialize_particles_new_sim.cpp:142-249), appended after the
// particles already in hb.  Shell particles get no velocity, mass or conformation values
// in the reference (it fills those for lattice particles only); they are zero here.
// Fails once the box would exceed Nmax particles.
sph_status colloid_shells(HostBox* hb, const double dx[3], int Nmax, std::string* msg) {
  BoxParams& p = hb->p;
  const int dim = p.dim;
  auto add = [&](double px, double py, double pz, int t) -> bool {
    if ((int)hb->x.size() + 1 > Nmax) return false;
    hb->x.push_back(px);
    hb->y.push_back(py);
    hb->z.push_back(pz);
    hb->type.push_back(t);
    hb->mass.push_back(0.0);
    hb->cxx.push_back(0.0); hb->cxy.push_back(0.0); hb->cyy.push_back(0.0);
    hb->cxz.push_back(0.0); hb->cyz.push_back(0.0); hb->czz.push_back(0.0);
    return true;
  };
  auto wrap_into = [&](double& px, double& py, double& pz) {
    if (px < 0) px = px + p.L[0];
    if (p.wall == 0 && py < 0) py = py + p.L[1];
    if (dim == 3 && pz < 0) pz = pz + p.L[2];
    if (px > p.L[0]) px = px - p.L[0];
    if (p.wall == 0 && py > p.L[1]) py = py - p.L[1];
    if (dim == 3 && pz > p.L[2]) pz = pz - p.L[2];
  };
  const int nlayers = (int)std::round(p.coll_R / dx[0]);
  for (int c = 0; c < p.N_colloids; ++c) {
    const double cx = hb->coll_x[c], cy = hb->coll_y[c], cz = hb->coll_z[c];
    double r = 0.5 * dx[0];
    for (int layer = 0; layer < nlayers; ++layer, r = r + dx[0]) {
      if (!(r < p.coll_R && r > p.coll_R - p.wall_width)) continue;
      bool ok = true;
      if (dim == 2) {
        double dphi = dx[0] / r;
        int nphi = (int)std::round(2.0 * M_PI / dphi);
        dphi = 2.0 * M_PI / nphi;
        double phi = 0.0;
        for (int k = 0; k < nphi && ok; ++k) {
          double px = cx + r * std::cos(phi), py = cy + r * std::sin(phi), pz = 0.0;
          wrap_into(px, py, pz);
          ok = add(px, py, pz, 3 + c);
          phi = phi + dphi;
        }
      } else {
        ok = add(cx, cy, cz + r, 3 + c);  // north pole, unwrapped as in the reference
        double dth = dx[0] / r;
        int nth = (int)std::round(M_PI / dth);
        dth = M_PI / nth;
        double th = 0.0;
        for (int k = 0; k < nth && ok; ++k) {
          double dphi = dx[0] / (r * std::sin(th));
          int nphi = (int)std::round(2.0 * M_PI / dphi);
          dphi = 2.0 * M_PI / nphi;
          double phi = 0.0;
          for (int l = 0; l < nphi && ok; ++l) {
            double px = cx + r * std::sin(th) * std::cos(phi);
            double py = cy + r * std::sin(th) * std::sin(phi);
            double pz = cz + r * std::cos(th);
            wrap_into(px, py, pz);
            ok = add(px, py, pz, 3 + c);
            phi = phi + dphi;
          }
          th = th + dth;
        }
        if (ok) ok = add(cx, cy, cz - r, 3 + c);  // south pole
      }
      if (!ok) {
        *msg = "N > Nmax while building colloid shells";
        return SPH_ERR_BAD_INPUT;
      }
    }
  }
  const size_t n = hb->x.size();
  hb->vx.assign(n, 0.0);
  hb->vy.assign(n, 0.0);
  hb->vz.assign(n, 0.0);
  return SPH_OK;
}

inline bool is_space(char c) {
  return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}

// The numbers of a text file read one after another as float, as a sequence of formatted
// float reads does, parsed in parallel chunks split at whitespace.  A token is a number only
// if it is made of digits, signs, '.', 'e' and 'E' and converts in full without overflow;
// reading stops at the first token that is not (as a formatted read fails there).  The
// conversion is strtof's, the correctly rounded one a formatted float read also uses.
bool read_float_tokens(const char* path, std::vector<float>* out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::string buf;
  char tmp[1 << 16];
  size_t got;
  while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, got);
  std::fclose(f);
  const size_t n = buf.size();
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, n / (1 << 20) + 1));
  std::vector<size_t> cut(nt + 1, n);
  cut[0] = 0;
  for (int t = 1; t < nt; ++t) {
    size_t c = std::max(cut[t - 1], n * t / nt);
    while (c < n && !is_space(buf[c])) ++c;
    cut[t] = c;
  }
  std::vector<std::vector<float>> part(nt);
  std::vector<char> stopped(nt, 0);
  auto work = [&](int t) {
    const char* p = buf.data() + cut[t];
    const char* e = buf.data() + cut[t + 1];
    std::vector<float>& v = part[t];
    v.reserve((size_t)(e - p) / 10);
    while (p < e) {
      while (p < e && is_space(*p)) ++p;
      if (p >= e) break;
      const char* q = p;
      bool chars_ok = true;
      while (q < e && !is_space(*q)) {
        const char c = *q;
        chars_ok = chars_ok && ((c >= '0' && c <= '9') || c == '+' || c == '-' || c == '.' ||
                                c == 'e' || c == 'E');
        ++q;
      }
      if (!chars_ok || q - p > 64) {
        stopped[t] = 1;
        return;
      }
      char tok[72];
      std::memcpy(tok, p, (size_t)(q - p));
      tok[q - p] = 0;
      char* end = nullptr;
      errno = 0;
      const float x = std::strtof(tok, &end);
      if (end != tok + (q - p) || (errno == ERANGE && std::fabs(x) > 1.0f)) {
        stopped[t] = 1;
        return;
      }
      v.push_back(x);
      p = q;
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  out->clear();
  for (int t = 0; t < nt; ++t) {
    out->insert(out->end(), part[t].begin(), part[t].end());
    if (stopped[t]) break;
  }
  return true;
}

// Restart file (system_initialize_particles_old_sim.cpp:17-112); values go through float.
// Rows are taken while a whole row of numbers can be read.
sph_status restart_particles(HostBox* hb, const char* path, std::string* msg) {
  std::vector<float> tok;
  if (!read_float_tokens(path ? path : "input_particles.in", &tok)) {
    *msg = "cannot open restart particle file";
    return SPH_ERR_IO;
  }
  const int dim = hb->p.dim;
  const int ncol = dim == 2 ? 9 : 14;
  auto clear = [](std::vector<double>& v) { v.clear(); };
  for (auto* v : {&hb->x, &hb->y, &hb->z, &hb->vx, &hb->vy, &hb->vz, &hb->mass, &hb->cxx,
                  &hb->cxy, &hb->cyy, &hb->cxz, &hb->cyz, &hb->czz})
    clear(*v);
  hb->type.clear();
  const size_t nrows = tok.size() / (size_t)ncol;
  for (auto* v : {&hb->x, &hb->y, &hb->z, &hb->vx, &hb->vy, &hb->vz, &hb->mass, &hb->cxx,
                  &hb->cxy, &hb->cyy, &hb->cxz, &hb->cyz, &hb->czz})
    v->reserve(nrows);
  hb->type.reserve(nrows);
  for (size_t r = 0; r < nrows; ++r) {
    const float* row = tok.data() + r * ncol;
    if (dim == 2) {
      hb->x.push_back(row[0]); hb->y.push_back(row[1]); hb->z.push_back(0.0);
      hb->vx.push_back(row[2]); hb->vy.push_back(row[3]); hb->vz.push_back(0.0);
      hb->mass.push_back(row[4]); hb->type.push_back((int)row[5]);
      hb->cxx.push_back(row[6]); hb->cxy.push_back(row[7]); hb->cyy.push_back(row[8]);
      hb->cxz.push_back(0.0); hb->cyz.push_back(0.0); hb->czz.push_back(0.0);
    } else {
      hb->x.push_back(row[0]); hb->y.push_back(row[1]); hb->z.push_back(row[2]);
      hb->vx.push_back(row[3]); hb->vy.push_back(row[4]); hb->vz.push_back(row[5]);
      hb->mass.push_back(row[6]); hb->type.push_back((int)row[7]);
      hb->cxx.push_back(row[8]); hb->cxy.push_back(row[9]); hb->cyy.push_back(row[10]);
      hb->cxz.push_back(row[11]); hb->cyz.push_back(row[12]); hb->czz.push_back(row[13]);
    }
  }
  if (hb->x.empty()) {
    *msg = "restart particle file holds no particles";
    return SPH_ERR_IO;
  }
  return SPH_OK;
}

}  // namespace

// class_system::constructor + initialize (system_constructor.cpp:15-108,
// system_initialize.cpp:16-359)
sph_status build_box(const sph_input& in_, const char* particles_path, HostBox* hb,
                     std::string* msg, bool lattice_on_device) {
  sph_status st = validate(in_, msg);
  if (st != SPH_OK) return st;
  hb->in = in_;
  hb->coll_xyz.assign(in_.coll_xyz, in_.coll_xyz + 3 * (size_t)in_.N_colloids);
  hb->in.coll_xyz = hb->coll_xyz.empty() ? nullptr : hb->coll_xyz.data();
  const sph_input& in = hb->in;
  BoxParams& p = hb->p;
  std::memset(&p, 0, sizeof(p));
  const int dim = in.dim;
  p.dim = dim;
  p.wall = in.wall;
  p.coll_move = in.coll_move;
  int Nxyz[3] = {in.N[0], in.N[1], dim == 3 ? in.N[2] : 1};
  for (int d = 0; d < 3; ++d) {
    p.L[d] = in.L[d];
    p.halfL[d] = 0.5 * in.L[d];
  }
  p.V_top = in.Vwall_top;
  p.V_bottom = in.Vwall_bottom;
  p.nkT = in.np * in.kT;
  p.tau = in.tau;
  p.dt = in.dt;
  p.t0 = in.t0;
  p.rcut = in.L[0] / in.N[0] * in.overlap;
  p.rcutsq = p.rcut * p.rcut;
  p.rcut_inv = 1.0 / p.rcut;
  double dx[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) dx[d] = in.L[d] / Nxyz[d];
  p.ky = 2.0 * M_PI / in.L[1];
  p.wall_width = (std::fabs(in.overlap - std::floor(in.overlap)) < 1.0e-10)
                     ? std::floor(in.overlap) * dx[1]
                     : (std::floor(in.overlap) + 1) * dx[1];
  int Ny_ctor = in.wall ? Nxyz[1] + 2 * (int)std::ceil(in.overlap) : Nxyz[1];
  if (in.wall == 1) {
    Nxyz[1] = Nxyz[1] + 2 * (int)std::ceil(in.overlap);
    p.y_bottom = 0.0;
    p.y_top = in.L[1];
  }
  p.cw = dim == 2 ? 63.0 / (478.0 * M_PI * p.rcut * p.rcut)
                  : 27.0 / (120.0 * M_PI * p.rcut * p.rcut * p.rcut);
  p.c_gradw = -15.0 * p.cw / p.rcut;
  p.csq = in.c * in.c;
  p.rho0 = in.P0 * in.rho;
  p.a = 5.0 * in.eta / 3.0 - in.zeta;
  p.b = dim == 3 ? 5.0 * (in.zeta + in.eta / 3.0) : 4.0 * (in.zeta + in.eta / 3.0);
  p.beta_max = 1.5;
  p.Ncells[0] = (int)(in.L[0] / p.rcut);
  p.cell_size[0] = in.L[0] / p.Ncells[0];
  const double Ly = in.wall == 1 ? in.L[1] + 2 * p.wall_width : in.L[1];
  p.Ncells[1] = (int)(Ly / p.rcut);
  p.cell_size[1] = Ly / p.Ncells[1];
  if (dim == 3) {
    p.Ncells[2] = (int)(in.L[2] / p.rcut);
    p.cell_size[2] = in.L[2] / p.Ncells[2];
  } else {
    p.Ncells[2] = 1;
    p.cell_size[2] = 1;
  }
  p.Ntotal_cells = p.Ncells[0] * p.Ncells[1] * p.Ncells[2];
  if (p.Ncells[0] < 3 || p.Ncells[1] < 3 || (dim == 3 && p.Ncells[2] < 3)) {
    *msg = "neighbour cells are too big";
    return SPH_ERR_BAD_INPUT;
  }
  p.ext_force_type = in.ext_force_type;
  p.ext_force[0] = in.ext_force[0];
  p.ext_force[1] = in.ext_force[1];
  if (dim == 3) p.ext_force[2] = in.ext_force[2];
  // colloids (system_initialize.cpp:155-262)
  const int nc = in.N_colloids;
  p.N_colloids = nc;
  p.coll_R = in.coll_R;
  p.coll_rho = in.coll_rho;
  p.F0_rep = in.F0_repulsion;
  p.tau_rep = in.tau_repulsion;
  const double rep_cutoff = 5.0 * p.coll_R / p.tau_rep;
  p.r0_magnet_sq = in.cutoff_magnetic * in.cutoff_magnetic;
  p.F0_magnet = in.F0_magnetic;
  p.omega_magnet = in.omega_magnetic;
  if (dim == 2) {
    p.coll_mass = M_PI * p.coll_R * p.coll_R * p.coll_rho;
    p.coll_I = 0.5 * p.coll_mass * p.coll_R * p.coll_R;
  } else {
    p.coll_mass = 4.0 / 3.0 * M_PI * p.coll_R * p.coll_R * p.coll_R * p.coll_rho;
    p.coll_I = 2.0 / 5.0 * p.coll_mass * p.coll_R * p.coll_R;
  }
  hb->coll_x.assign(nc, 0.0);
  hb->coll_y.assign(nc, 0.0);
  hb->coll_z.assign(nc, 0.0);
  for (int i = 0; i < nc; ++i) {
    hb->coll_x[i] = in.coll_xyz[3 * i];
    hb->coll_y[i] = in.coll_xyz[3 * i + 1];
    if (dim == 3) hb->coll_z[i] = in.coll_xyz[3 * i + 2];
    if (in.wall && (hb->coll_y[i] - p.coll_R < p.y_bottom || hb->coll_y[i] + p.coll_R > p.y_top)) {
      *msg = "a colloid overlaps a wall";
      return SPH_ERR_BAD_INPUT;
    }
  }
  if (nc > 0) {
    const double rcuton = 2.0 * p.coll_R + in.coll_repulsion_cuton;
    const double rcutoff_rep = 2.0 * p.coll_R + rep_cutoff;
    p.rcuton_coll_rep_sq = rcuton * rcuton;
    p.rcutoff_coll_rep_sq = rcutoff_rep * rcutoff_rep;
    const double rcoll = rcutoff_rep > in.cutoff_magnetic ? rcutoff_rep : in.cutoff_magnetic;
    for (int d = 0; d < 2; ++d) {
      p.Ncells_colloids[d] = (int)(in.L[d] / rcoll);
      p.cell_colloids_size[d] = in.L[d] / p.Ncells_colloids[d];
    }
    if (dim == 3) {
      p.Ncells_colloids[2] = (int)(in.L[2] / rcoll);
      p.cell_colloids_size[2] = in.L[2] / p.Ncells_colloids[2];
    } else {
      p.Ncells_colloids[2] = 1;
      p.cell_colloids_size[2] = 1;
    }
    p.Ntotal_cells_colloids = p.Ncells_colloids[0] * p.Ncells_colloids[1] * p.Ncells_colloids[2];
    if (p.Ncells_colloids[0] < 3 || p.Ncells_colloids[1] < 3 ||
        (dim == 3 && p.Ncells_colloids[2] < 3)) {
      *msg = "neighbour colloids cells are too big";
      return SPH_ERR_BAD_INPUT;
    }
  }
  // particles
  if (in.new_sim == 0) {
    int Nmax = dim == 2 ? Nxyz[0] * Ny_ctor : Nxyz[0] * Ny_ctor * Nxyz[2];
    if (nc > 0) Nmax = (int)(Nmax * 1.01);
    hb->Nmax = Nmax;
    if (lattice_on_device) {
      // the lattice is generated on the device (sph_init.cu); the host keeps the shells,
      // whose Nmax check waits for the device's count of lattice particles
      hb->lattice_on_device = true;
      for (int q = 0; q < 3; ++q) {
        hb->Nxyz[q] = Nxyz[q];
        hb->dx[q] = dx[q];
      }
      hb->lattice_m = lattice_mass(*hb, Nxyz);
      hb->x.clear(); hb->y.clear(); hb->z.clear(); hb->type.clear(); hb->mass.clear();
      hb->cxx.clear(); hb->cxy.clear(); hb->cyy.clear();
      hb->cxz.clear(); hb->cyz.clear(); hb->czz.clear();
      st = colloid_shells(hb, dx, INT_MAX, msg);
    } else {
      st = lattice_particles(hb, Nxyz, dx, Nmax, msg);
    }
  } else {
    st = restart_particles(hb, particles_path, msg);
  }
  if (st != SPH_OK) return st;
  const int N = (int)hb->x.size();
  p.N = N;
  if (in.new_sim != 0) hb->Nmax = N;
  // walls_list (system_initialize.cpp:278-300): ids of wall 1 then wall 2, ascending
  hb->walls_list.clear();
  if (in.wall) {
    for (int w = 1; w <= 2; ++w) {
      hb->walls_start[w - 1] = (int)hb->walls_list.size();
      for (int i = 0; i < N; ++i)
        if (hb->type[i] == w) hb->walls_list.push_back(i);
    }
    hb->Nlist_walls = (int)hb->walls_list.size();
  }
  // colloids_list and body-frame offsets (system_initialize.cpp:304-355)
  hb->colloids_list.clear();
  hb->colloids_start.assign(nc, 0);
  for (int c = 0; c < nc; ++c) {
    hb->colloids_start[c] = (int)hb->colloids_list.size();
    for (int i = 0; i < N; ++i)
      if (hb->type[i] == 3 + c) hb->colloids_list.push_back(i);
  }
  const size_t nl = hb->colloids_list.size();
  hb->x_center.assign(nl, 0.0);
  hb->y_center.assign(nl, 0.0);
  hb->z_center.assign(nl, 0.0);
  for (size_t k = 0; k < nl; ++k) {
    const int i = hb->colloids_list[k];
    const int c = hb->type[i] - 3;
    hb->x_center[k] = wrap_half(hb->x[i] - hb->coll_x[c], p.L[0]);
    double yc = hb->y[i] - hb->coll_y[c];
    if (p.wall == 0) yc = wrap_half(yc, p.L[1]);
    hb->y_center[k] = yc;
    if (dim == 3) hb->z_center[k] = wrap_half(hb->z[i] - hb->coll_z[c], p.L[2]);
  }
  return SPH_OK;
}

// class_system scalars after constructor + initialize (system_constructor.cpp:15-79,
// system_initialize.cpp:47-262).  The colloid cutoffs derived from the input follow
// system_initialize.cpp:158-166 and 207-217.
void fill_info(const HostBox& hb, sph_info* o) {
  const BoxParams& p = hb.p;
  const sph_input& in = hb.in;
  std::memset(o, 0, sizeof(*o));
  o->Nmax = hb.Nmax;
  o->ext_force_type = p.ext_force_type;
  o->rcut_inv = p.rcut_inv;
  o->c = in.c;
  o->rho = in.rho;
  o->P0 = in.P0;
  o->ky = p.ky;
  o->beta_max = p.beta_max;
  for (int q = 0; q < 3; ++q) {
    o->ext_force[q] = p.ext_force[q];
    o->cell_colloids_size[q] = p.cell_colloids_size[q];
  }
  o->coll_rho = p.coll_rho;
  o->coll_rep_cuton = in.coll_repulsion_cuton;
  o->coll_rep_cutoff = 5.0 * p.coll_R / p.tau_rep;
  o->F0_rep = p.F0_rep;
  o->tau_rep = p.tau_rep;
  o->r0_magnet = in.cutoff_magnetic;
  o->r0_magnet_sq = p.r0_magnet_sq;
  o->F0_magnet = p.F0_magnet;
  if (p.N_colloids > 0) {
    o->rcuton_coll_rep = 2.0 * p.coll_R + o->coll_rep_cuton;
    o->rcuton_coll_rep_sq = o->rcuton_coll_rep * o->rcuton_coll_rep;
    o->rcutoff_coll_rep = 2.0 * p.coll_R + o->coll_rep_cutoff;
    o->rcutoff_coll_rep_sq = o->rcutoff_coll_rep * o->rcutoff_coll_rep;
    o->rcutoff_coll = o->rcutoff_coll_rep > o->r0_magnet ? o->rcutoff_coll_rep : o->r0_magnet;
    o->rcutoff_coll_sq = o->rcutoff_coll * o->rcutoff_coll;
  }
  o->N = p.N;
  o->dim = p.dim;
  o->wall = p.wall;
  for (int q = 0; q < 3; ++q) {
    o->Ncells[q] = p.Ncells[q];
    o->Ncells_colloids[q] = p.Ncells_colloids[q];
    o->cell_size[q] = p.cell_size[q];
    o->L[q] = p.L[q];
  }
  o->Ntotal_cells = p.Ntotal_cells;
  o->Nwalls = p.wall ? 2 : 0;
  o->Nlist_walls = hb.Nlist_walls;
  o->N_colloids = p.N_colloids;
  o->Nlist_colloids = (int)hb.colloids_list.size();
  o->Ntotal_cells_colloids = p.Ntotal_cells_colloids;
  o->nboxes = 1;
  o->rcut = p.rcut;
  o->rcutsq = p.rcutsq;
  o->cw = p.cw;
  o->c_gradw = p.c_gradw;
  o->csq = p.csq;
  o->rho0 = p.rho0;
  o->a = p.a;
  o->b = p.b;
  o->nkT = p.nkT;
  o->tau = p.tau;
  o->dt = p.dt;
  o->wall_width = p.wall_width;
  o->y_bottom = p.y_bottom;
  o->y_top = p.y_top;
  o->V_bottom = p.V_bottom;
  o->V_top = p.V_top;
  o->coll_R = p.coll_R;
  o->coll_mass = p.coll_mass;
  o->coll_I = p.coll_I;
  o->t0 = p.t0;
  o->omega_magnet = p.omega_magnet;
}

}  // namespace sph

namespace {
template <typename T>
void put(T* dst, const std::vector<T>& v) {
  if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(T));
}
}  // namespace

extern "C" sph_status sph_host_setup(const sph_input* in, const char* particles_path, int cap,
                                     sph_host_state* out, int* n_out, sph_info* info) {
  if (!in) return SPH_ERR_STATE;
  sph::HostBox hb;
  std::string msg;
  sph_status s = sph::build_box(*in, particles_path, &hb, &msg);
  if (s != SPH_OK) {
    std::fprintf(stderr, "sph_host_setup: %s\n", msg.c_str());
    return s;
  }
  if (n_out) *n_out = hb.p.N;
  if (info) sph::fill_info(hb, info);
  if (!out) return SPH_OK;
  if (hb.p.N > cap || (int)hb.colloids_list.size() > cap || (int)hb.walls_list.size() > cap)
    return SPH_ERR_STATE;
  put(out->x, hb.x); put(out->y, hb.y); put(out->z, hb.z);
  put(out->vx, hb.vx); put(out->vy, hb.vy); put(out->vz, hb.vz);
  put(out->mass, hb.mass);
  put(out->cxx, hb.cxx); put(out->cxy, hb.cxy); put(out->cyy, hb.cyy);
  put(out->cxz, hb.cxz); put(out->cyz, hb.cyz); put(out->czz, hb.czz);
  put(out->type, hb.type);
  put(out->walls_list, hb.walls_list);
  if (out->walls_start) { out->walls_start[0] = hb.walls_start[0]; out->walls_start[1] = hb.walls_start[1]; }
  put(out->colloids_list, hb.colloids_list);
  put(out->colloids_start, hb.colloids_start);
  put(out->x_center, hb.x_center); put(out->y_center, hb.y_center); put(out->z_center, hb.z_center);
  return SPH_OK;
}
