// sph_capi.cu -- the C ABI (include/sph_capi.h): context lifetime, device memory, the
// order of the step phases (the reference's main.cu:358-467 and class_system methods),
// CUDA-graph replay of whole steps, and state access in original particle order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "sph_internal.h"
#include "sph_io.h"

using namespace sph;

struct sph_ctx {
  int device = 0, prec = SPH_PREC_FP64, dim = 3, nboxes = 0, use_graph = 1;
  std::vector<HostBox> boxes;
  Dev d{};
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  int key_bits = 1;
  SortScratch sort{};
  double* ke_partial = nullptr;
  double* obs_partial = nullptr;  // 2 per KE chunk
  double* obs_acc = nullptr;      // nboxes x SPH_NUM_OBS running sums
  long long obs_samples = 0;
  double* scratch = nullptr;  // Ntot doubles for field transfers
  int* iscratch = nullptr;    // Ntot ints
  std::string err;
  long long launches = 0;
  bool initial_done = false;
  bool in_step = false;      // between vv_step1 and vv_step2
  bool forces_live = false;  // forces computed and not yet consumed by a half-kick
  bool pos_dirty = true;     // positions changed since the last neighbour search
  bool gradv_valid = false;
  long long host_step = 0;
  int parity = 0;            // which of the double-buffered state arrays is current
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_kernels = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool events_recorded = false;  // ev0/ev1 bracket the last sph_step
  double last_ms = 0.0;
  int max_coll = 0;
  int cap_grown = 0;
  // the last sph_step call, for resuming it after a full neighbour list was found in one of
  // its steps: the step counter and buffer parity when it started, and the step it ends at
  bool call_open = false;
  long long call_step0 = 0, call_target = 0;
  int call_parity0 = 0;
  sph_tuning tune = {32, 128};  // launch geometry (sph_set_tuning / sph_autotune)
};

namespace {

sph_status fail(sph_ctx* c, sph_status s, const std::string& m) {
  if (c) c->err = m;
  return s;
}

sph_status cuda_fail(sph_ctx* c, const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && last_launch_error() != 0) e = (cudaError_t)last_launch_error();
  last_launch_error() = 0;
  return fail(c, SPH_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

template <typename T>
bool dalloc(sph_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
  cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), c->stream);
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return true;
}

// Device buffers that live only while a context is being created.
struct TmpDev {
  std::vector<void*> bufs;
  template <typename T>
  bool alloc(T** p, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
    bufs.push_back(q);
    *p = static_cast<T*>(q);
    return true;
  }
  ~TmpDev() {
    for (void* q : bufs) cudaFree(q);
  }
};

Launch launcher(sph_ctx* c) {
  Launch L;
  L.d = c->d;
  L.prec = c->prec;
  L.stream = c->stream;
  L.launches = &c->launches;
  L.list_tpc = c->tune.list_threads_per_cell;
  L.density_block = c->tune.density_block;
  return L;
}

int bits_for(int n) {
  int b = 1;
  while ((1 << b) < n) ++b;
  return b;
}

void swap_state(sph_ctx* c, bool with_forces) {
  std::swap(c->d.pos, c->d.pos_b);
  std::swap(c->d.vel, c->d.vel_b);
  std::swap(c->d.conf, c->d.conf_b);
  std::swap(c->d.tinfo, c->d.tinfo_b);
  std::swap(c->d.gid, c->d.gid_b);
  if (with_forces) {
    std::swap(c->d.f, c->d.f_b);
    std::swap(c->d.dcdt, c->d.dcdt_b);
  }
  c->parity ^= 1;
}

// Neighbour-list capacity: chunks with hits per particle.  A particle's candidates come
// from the 3^d neighbour cells in chunks of up to 16 (a half warp per cell) or 32 slots;
// sized for cells holding 1.5 times the lattice's particles per cell, in chunks of 16.
int derived_capacity(const std::vector<HostBox>& boxes, int dim) {
  int worst = 1;
  for (const HostBox& hb : boxes) {
    const sph_input& in = hb.in;
    double ppc = 1.0;  // lattice particles per cell
    for (int q = 0; q < dim; ++q) ppc *= hb.p.cell_size[q] / (in.L[q] / in.N[q]);
    const int per_cell = (int)std::ceil(1.5 * ppc / 16.0);
    worst = std::max(worst, (dim == 3 ? 27 : 9) * std::max(per_cell, 1));
  }
  return worst;
}

// Allocates the neighbour-list entries for `cap` chunks per particle, replacing earlier ones.
bool alloc_lists(sph_ctx* c, int cap) {
  Dev& d = c->d;
  auto replace = [&](auto** ptr, size_t n) {
    using T = std::remove_pointer_t<std::remove_reference_t<decltype(*ptr)>>;
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
    cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), c->stream);
    auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)*ptr);
    if (*ptr && it != c->allocs.end()) {
      cudaFree(*it);
      *it = q;
    } else {
      c->allocs.push_back(q);
    }
    *ptr = static_cast<T*>(q);
    return true;
  };
  if (!replace(&d.nchunk, (size_t)cap * d.Npad)) return false;
  d.cap = cap;
  return true;
}

// Reads the device error flags and their record (err_info, kErrInfoLen ints) without
// clearing them.  Blocks on the stream.
bool read_device_status(sph_ctx* c, unsigned* st, int* info) {
  return cudaMemcpyAsync(st, c->d.status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                         c->stream) == cudaSuccess &&
         cudaMemcpyAsync(info, c->d.err_info, kErrInfoLen * sizeof(int), cudaMemcpyDeviceToHost,
                         c->stream) == cudaSuccess &&
         cudaStreamSynchronize(c->stream) == cudaSuccess;
}

long long failed_step(const int* info) {
  return ((long long)info[kErrStepHi] << 32) | (long long)(unsigned)info[kErrStepLo];
}

// The status for a set of device flags; `where` names the step for failures inside a
// multi-step call.
sph_status status_of(sph_ctx* c, unsigned st, const int* info, const std::string& where) {
  if (st & kStatNaN)
    return fail(c, SPH_ERR_NAN, "non-finite particle position (global id " +
                                    std::to_string(info[kErrBadId]) + ")" + where);
  if (st & kStatCellRange)
    return fail(c, SPH_ERR_CELL_RANGE, "particle hashed outside the cell grid (global id " +
                                           std::to_string(info[kErrBadId]) + ")" + where);
  if (st & kStatCapacity)
    return fail(c, SPH_ERR_CAPACITY, "neighbour list capacity " + std::to_string(c->d.cap) +
                                         " exceeded (" + std::to_string(info[kErrMaxCount]) +
                                         " needed)" + where);
  return SPH_OK;
}

// Reads and clears the device error flags.  Blocks on the stream.
sph_status check_device(sph_ctx* c) {
  unsigned st = 0;
  int info[kErrInfoLen] = {0};
  if (!read_device_status(c, &st, info)) return cuda_fail(c, "device status");
  if (st == 0) return SPH_OK;
  cudaMemsetAsync(c->d.status, 0, sizeof(unsigned), c->stream);
  return status_of(c, st, info, "");
}

void drop_graphs(sph_ctx* c) {
  for (auto& g : c->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Grows the lists to hold `needed` chunks per particle, with headroom.
sph_status grow_capacity(sph_ctx* c, int needed) {
  const int cap = std::max(needed + needed / 4 + 2, c->d.cap + 4);
  cudaStreamSynchronize(c->stream);
  if (!alloc_lists(c, cap)) return fail(c, SPH_ERR_NOMEM, "cannot grow neighbour lists");
  c->cap_grown++;
  drop_graphs(c);
  return SPH_OK;
}

// ---- phases (all asynchronous) ----
int ph_search(sph_ctx* c) {
  Launch L = launcher(c);
  const bool permute = c->forces_live;
  if (launch_hash(L) || launch_sort(L, c->key_bits, c->sort) || launch_reorder(L, permute))
    return 1;
  swap_state(c, permute);
  L = launcher(c);
  if (launch_build_lists_dim(L, c->dim)) return 1;
  if (c->d.ncoll > 0 && launch_colloid_cells_n(L, c->nboxes, c->max_coll)) return 1;
  c->pos_dirty = false;
  return 0;
}

// fold: the fused pair pass also applies the step's second half-kick to fluid particles
// (the step graph); the method-by-method path keeps V_Verlet_step2 separate
int ph_forces(sph_ctx* c, bool fold = false) {
  Launch L = launcher(c);
  L.d.gradv = nullptr;  // the fused pass keeps the gradient in registers
  L.d.fold_vv2 = fold ? 1 : 0;
  bool ext = false;
  for (const HostBox& hb : c->boxes) ext = ext || hb.p.ext_force_type != 0;
  if (launch_density_dim(L, c->dim)) return 1;
  if (launch_pairs_dim(L, c->dim, kPairFused, ext ? 1 : 0)) return 1;
  if (launch_wall_forces(L)) return 1;
  bool pairs = false;
  for (const HostBox& hb : c->boxes) pairs = pairs || hb.p.N_colloids >= 2;
  if (launch_colloid_forces(L, pairs ? 1 : 0)) return 1;
  c->forces_live = true;
  c->gradv_valid = false;
  return 0;
}

int ph_vv1(sph_ctx* c) {
  Launch L = launcher(c);
  if (launch_vv1_colloids(L) || launch_vv1_particles(L)) return 1;
  c->forces_live = false;
  c->pos_dirty = true;
  return 0;
}

int ph_vv2(sph_ctx* c, bool folded = false) {
  Launch L = launcher(c);
  if (launch_vv2(L, !folded) || launch_count_step(L)) return 1;
  return 0;
}

// One full step: VV1, search, m(t), forces, VV2 (main.cu:358-432)
int ph_step(sph_ctx* c) {
  if (ph_vv1(c) || ph_search(c)) return 1;
  if (launch_advance_time(launcher(c), 0)) return 1;
  if (ph_forces(c, true) || ph_vv2(c, true)) return 1;
  c->forces_live = true;
  return 0;
}

sph_status upload_moment(sph_ctx* c, const double* m) {
  std::vector<double> mm(3 * (size_t)c->nboxes);
  for (int b = 0; b < c->nboxes; ++b)
    for (int q = 0; q < 3; ++q) mm[3 * b + q] = m[q];
  if (cudaMemcpyAsync(c->d.mag, mm.data(), mm.size() * sizeof(double), cudaMemcpyHostToDevice,
                      c->stream) != cudaSuccess)
    return cuda_fail(c, "magnetic moment upload");
  cudaStreamSynchronize(c->stream);
  return SPH_OK;
}

// Host-computed moment at the current time of every box (exactly as main.cu computes it).
sph_status host_moment(sph_ctx* c, long long step) {
  std::vector<double> mm(3 * (size_t)c->nboxes);
  for (int b = 0; b < c->nboxes; ++b) {
    const BoxParams& p = c->boxes[b].p;
    const double ang = p.omega_magnet * (p.t0 + p.dt * (double)step);
    mm[3 * b] = std::cos(ang);
    mm[3 * b + 1] = std::sin(ang);
    mm[3 * b + 2] = 0.0;
  }
  if (cudaMemcpyAsync(c->d.mag, mm.data(), mm.size() * sizeof(double), cudaMemcpyHostToDevice,
                      c->stream) != cudaSuccess)
    return cuda_fail(c, "magnetic moment upload");
  cudaStreamSynchronize(c->stream);
  return SPH_OK;
}

// Lists too short for the current positions: grow them to the largest row the list build
// saw and build them again (with the colloid coarse grid, which the failed search skipped),
// until they fit.  The device flags are clear on entry.
sph_status regrow_lists(sph_ctx* c) {
  for (int round = 0; round < 4; ++round) {
    int need = 0;
    if (cudaMemcpy(&need, c->d.err_info + kErrMaxCount, sizeof(int), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
      return cuda_fail(c, "list statistics");
    sph_status s = grow_capacity(c, need);
    if (s != SPH_OK) return s;
    cudaMemsetAsync(c->d.err_info + kErrMaxCount, 0, sizeof(int), c->stream);
    Launch L = launcher(c);
    if (launch_build_lists_dim(L, c->dim)) return cuda_fail(c, "rebuild lists");
    if (c->d.ncoll > 0 && launch_colloid_cells_n(L, c->nboxes, c->max_coll))
      return cuda_fail(c, "rebuild colloid cells");
    s = check_device(c);
    if (s != SPH_ERR_CAPACITY) return s;
  }
  return fail(c, SPH_ERR_CAPACITY, "neighbour lists still too short after growing them");
}

sph_status search_checked(sph_ctx* c) {
  const bool permute = c->forces_live;
  if (ph_search(c)) return cuda_fail(c, "neighbours_search");
  unsigned st = 0;
  int info[kErrInfoLen] = {0};
  if (!read_device_status(c, &st, info)) return cuda_fail(c, "device status");
  if (st == 0) return SPH_OK;
  cudaMemsetAsync(c->d.status, 0, sizeof(unsigned), c->stream);
  if (info[kErrPhase] == kPhaseHash) {
    // the hash stopped the search before its reorder: the state is still in the previous
    // order, in the buffers the host swapped away from
    swap_state(c, permute);
    c->pos_dirty = true;
  }
  if (st == kStatCapacity) return regrow_lists(c);
  c->pos_dirty = true;
  return status_of(c, st, info, "");
}

sph_status ensure_lists(sph_ctx* c) {
  if (!c->pos_dirty) return SPH_OK;
  return search_checked(c);
}

sph_status do_initial(sph_ctx* c) {
  sph_status s = host_moment(c, 0);
  if (s != SPH_OK) return s;
  s = search_checked(c);
  if (s != SPH_OK) return s;
  if (ph_forces(c)) return cuda_fail(c, "initial forces");
  s = check_device(c);
  if (s != SPH_OK) return s;
  c->initial_done = true;
  return SPH_OK;
}

sph_status capture_graphs(sph_ctx* c) {
  drop_graphs(c);
  for (int k = 0; k < 2; ++k) {
    cudaGraph_t g = nullptr;
    long long before = c->launches;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return cuda_fail(c, "begin capture");
    const bool live = c->forces_live, dirty = c->pos_dirty;
    int bad = ph_step(c);
    c->forces_live = live;
    c->pos_dirty = dirty;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (bad || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(c, SPH_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
    }
    // the captured step flipped the buffer parity; graph[k] starts from parity k
    e = cudaGraphInstantiate(&c->graph[c->parity ^ 1], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, "graph instantiate failed");
    c->graph_kernels = c->launches - before;
    c->launches = before;
  }
  return SPH_OK;
}

// Launches n whole steps: CUDA-graph replays (captured first if needed) or direct launches.
sph_status run_steps(sph_ctx* c, long long n) {
  if (n <= 0) return SPH_OK;
  if (c->use_graph && !c->graph[0]) {
    sph_status s = capture_graphs(c);
    if (s != SPH_OK) return s;
  }
  for (long long k = 0; k < n; ++k) {
    if (c->use_graph) {
      if (cudaGraphLaunch(c->graph[c->parity], c->stream) != cudaSuccess)
        return cuda_fail(c, "graph launch");
      swap_state(c, false);
      c->launches += c->graph_kernels;
    } else if (ph_step(c)) {
      return cuda_fail(c, "step");
    }
    c->host_step++;
  }
  c->forces_live = true;
  c->pos_dirty = false;
  return SPH_OK;
}

// Waits for the open sph_step call(s) and checks their steps.  A step that found its
// neighbour lists too short stopped every kernel after its list build (and every later
// step); here the lists grow, the step is finished from its list build, and the remaining
// steps run, until the call's last step is done.  A position outside the grid or not finite
// is reported with the step it was found in; the state is then the one that step left
// after its half-kick and drift (the step counter says how many steps were completed).
sph_status settle_call(sph_ctx* c) {
  for (int round = 0;; ++round) {
    unsigned st = 0;
    int info[kErrInfoLen] = {0};
    if (!read_device_status(c, &st, info)) {
      c->call_open = false;
      return cuda_fail(c, "device status");
    }
    if (st == 0) {
      c->call_open = false;
      return SPH_OK;
    }
    cudaMemsetAsync(c->d.status, 0, sizeof(unsigned), c->stream);
    // the host's view of the stopped call: completed steps and the buffer parity of the
    // reorders that did run (the failing step's own reorder ran if its list build reported)
    const long long done = failed_step(info);
    const int phase = info[kErrPhase];
    const long long reorders = (done - c->call_step0) + (phase == kPhaseLists ? 1 : 0);
    const int parity = c->call_parity0 ^ (int)(reorders & 1);
    if (c->parity != parity) swap_state(c, false);
    c->host_step = done;
    const std::string where = " in step " + std::to_string(done + 1);
    if (!(st == kStatCapacity && phase == kPhaseLists && round < 8)) {
      c->call_open = false;
      c->forces_live = false;
      c->pos_dirty = true;
      c->gradv_valid = false;
      return status_of(c, st, info,
                       where + "; the state is that step's after its half-kick and drift");
    }
    sph_status s = regrow_lists(c);
    if (s == SPH_OK && (launch_advance_time(launcher(c), 0) || ph_forces(c, true) ||
                        ph_vv2(c, true)))
      s = cuda_fail(c, "resumed step");
    if (s != SPH_OK) {
      c->call_open = false;
      c->pos_dirty = true;
      return s;
    }
    c->host_step = done + 1;
    c->forces_live = true;
    c->pos_dirty = false;
    c->call_step0 = c->host_step;
    c->call_parity0 = c->parity;
    s = run_steps(c, c->call_target - c->host_step);
    if (s != SPH_OK) {
      c->call_open = false;
      return s;
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
      c->call_open = false;
      return cuda_fail(c, "synchronize");
    }
  }
}

void free_ctx(sph_ctx* c) {
  if (!c) return;
  drop_graphs(c);
  for (void* p : c->allocs) cudaFree(p);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace

// ======================================================================================
extern "C" {

const char* sph_status_string(sph_status s) {
  switch (s) {
    case SPH_OK: return "ok";
    case SPH_ERR_BAD_INPUT: return "bad input";
    case SPH_ERR_CUDA: return "cuda error";
    case SPH_ERR_CELL_RANGE: return "particle outside the cell grid";
    case SPH_ERR_NAN: return "non-finite position";
    case SPH_ERR_TIMEOUT: return "timeout";
    case SPH_ERR_STATE: return "invalid state or argument";
    case SPH_ERR_NOMEM: return "out of memory";
    case SPH_ERR_CAPACITY: return "neighbour list capacity exceeded";
    case SPH_ERR_IO: return "i/o error";
  }
  return "unknown status";
}

const char* sph_last_error(const sph_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

sph_status sph_read_input(const char* path, sph_input* in, double* coll_buf, int coll_cap,
                          char* msg, size_t msg_cap) {
  if (!path || !in) return SPH_ERR_STATE;
  std::vector<double> coll;
  std::string m;
  sph_status s = parse_input_file(path, in, &coll, &m);
  if (s == SPH_OK && in->N_colloids > 0) {
    if (!coll_buf || coll_cap < in->N_colloids) {
      s = SPH_ERR_STATE;
      m = "colloid buffer too small";
    } else {
      std::memcpy(coll_buf, coll.data(), coll.size() * sizeof(double));
      in->coll_xyz = coll_buf;
    }
  } else if (s == SPH_OK) {
    in->coll_xyz = nullptr;
  }
  if (msg && msg_cap) {
    std::strncpy(msg, m.c_str(), msg_cap - 1);
    msg[msg_cap - 1] = 0;
  }
  return s;
}

sph_status sph_create_ensemble(int nboxes, const sph_input* inputs,
                               const char* const* particles_paths, const sph_options* opt,
                               sph_ctx** out) {
  if (!out || !inputs || nboxes <= 0) return SPH_ERR_STATE;
  *out = nullptr;
  sph_ctx* c = new sph_ctx();
  sph_options o{};
  o.precision = SPH_PREC_FP64;
  o.use_graph = 1;
  if (opt) o = *opt;
  c->prec = o.precision == SPH_PREC_MIXED ? SPH_PREC_MIXED : SPH_PREC_FP64;
  c->device = o.device;
  c->use_graph = o.use_graph;
  c->nboxes = nboxes;
  c->boxes.resize(nboxes);
  const bool dev_init = o.init_on_device != 0;
  for (int b = 0; b < nboxes; ++b) {
    std::string m;
    sph_status s = build_box(inputs[b], particles_paths ? particles_paths[b] : nullptr,
                             &c->boxes[b], &m, dev_init);
    if (s != SPH_OK) {
      fprintf(stderr, "sph_create: box %d: %s\n", b, m.c_str());
      delete c;
      return s;
    }
  }
  c->dim = c->boxes[0].p.dim;
  for (const HostBox& hb : c->boxes)
    if (hb.p.dim != c->dim) {
      fprintf(stderr, "sph_create: all boxes of a context must have the same dim\n");
      delete c;
      return SPH_ERR_BAD_INPUT;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c->device ||
      cudaSetDevice(c->device) != cudaSuccess) {
    fprintf(stderr, "sph_create: no usable CUDA device\n");
    delete c;
    return SPH_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SPH_ERR_CUDA;
  }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  // ---- lattice boxes built on the device: count the kept and wall sites per block ----
  TmpDev tmp;
  std::vector<InitBox> ib;
  std::vector<int> blk_box, ib_of_box(nboxes, -1), offs;
  std::vector<double> centres;
  InitBox* d_ib = nullptr;
  int* d_blk_box = nullptr;
  double* d_centres = nullptr;
  if (dev_init) {
    for (int b = 0; b < nboxes; ++b) {
      const HostBox& hb = c->boxes[b];
      if (!hb.lattice_on_device) continue;
      const BoxParams& p = hb.p;
      InitBox B{};
      B.box = b;
      B.dim = p.dim;
      B.wall = p.wall;
      for (int q = 0; q < 3; ++q) {
        B.Nxyz[q] = hb.Nxyz[q];
        B.dx[q] = hb.dx[q];
        B.L[q] = p.L[q];
      }
      B.nsites = B.Nxyz[0] * B.Nxyz[1] * (p.dim == 3 ? B.Nxyz[2] : 1);
      B.blk0 = (int)blk_box.size();
      B.nblk = (B.nsites + kInitThreads - 1) / kInitThreads;
      blk_box.insert(blk_box.end(), B.nblk, (int)ib.size());
      B.coll0 = (int)centres.size() / 3;
      B.ncoll = p.N_colloids;
      for (int l = 0; l < p.N_colloids; ++l) {
        centres.push_back(hb.coll_x[l]);
        centres.push_back(hb.coll_y[l]);
        centres.push_back(hb.coll_z[l]);
      }
      B.wall_width = p.wall_width;
      B.R2 = p.coll_R * p.coll_R;
      B.mass = hb.lattice_m;
      B.y_bottom = p.y_bottom;
      B.y_top = p.y_top;
      ib_of_box[b] = (int)ib.size();
      ib.push_back(B);
    }
  }
  if (!ib.empty()) {
    const int nblk = (int)blk_box.size();
    std::vector<int> counts(3 * (size_t)nblk);
    int* d_counts = nullptr;
    bool ok = tmp.alloc(&d_ib, ib.size()) && tmp.alloc(&d_blk_box, nblk) &&
              tmp.alloc(&d_centres, std::max<size_t>(centres.size(), 1)) &&
              tmp.alloc(&d_counts, counts.size());
    ok = ok && cudaMemcpyAsync(d_ib, ib.data(), ib.size() * sizeof(InitBox),
                               cudaMemcpyHostToDevice, c->stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_blk_box, blk_box.data(), nblk * sizeof(int),
                               cudaMemcpyHostToDevice, c->stream) == cudaSuccess;
    ok = ok && (centres.empty() ||
                cudaMemcpyAsync(d_centres, centres.data(), centres.size() * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream) == cudaSuccess);
    ok = ok && launch_init_count(d_ib, d_blk_box, nblk, d_centres, d_counts, c->stream) == 0;
    ok = ok && cudaMemcpyAsync(counts.data(), d_counts, counts.size() * sizeof(int),
                               cudaMemcpyDeviceToHost, c->stream) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(c->stream) == cudaSuccess;
    if (!ok) {
      fprintf(stderr, "sph_create: device initialisation failed\n");
      free_ctx(c);
      return SPH_ERR_CUDA;
    }
    // per-block offsets within each box, and the boxes' particle and wall counts
    offs.assign(counts.size(), 0);
    for (InitBox& B : ib) {
      int n[3] = {0, 0, 0};
      for (int k = B.blk0; k < B.blk0 + B.nblk; ++k)
        for (int q = 0; q < 3; ++q) {
          offs[3 * (size_t)k + q] = n[q];
          n[q] += counts[3 * (size_t)k + q];
        }
      HostBox& hb = c->boxes[B.box];
      hb.host0 = n[0];
      hb.p.N = n[0] + (int)hb.x.size();
      if (hb.p.N > hb.Nmax) {
        fprintf(stderr, "sph_create: box %d: N > Nmax while building colloid shells\n", B.box);
        free_ctx(c);
        return SPH_ERR_BAD_INPUT;
      }
      if (hb.p.wall) {
        hb.walls_start[0] = 0;
        hb.walls_start[1] = n[1];
        hb.Nlist_walls = n[1] + n[2];
      }
      B.nw1 = n[1];
    }
  }
  // ---- offsets ----
  int Ntot = 0, Ctot = 0, ncoll = 0, nwall = 0, ncc = 0, nlist = 0, nwl = 0, nwchunk = 0;
  for (HostBox& hb : c->boxes) {
    BoxParams& p = hb.p;
    p.slot0 = Ntot;
    p.cell0 = Ctot;
    p.coll0 = ncoll;
    p.wall_seg0 = nwall;
    p.ccell0 = ncc;
    p.list_cut2 = p.rcutsq * (1.0 + 1.0e-4);
    Ntot += p.N;
    Ctot += p.Ntotal_cells;
    ncoll += p.N_colloids;
    nwall += p.wall ? 2 : 0;
    ncc += p.N_colloids > 0 ? p.Ntotal_cells_colloids : 0;
    nlist += (int)hb.colloids_list.size();
    nwl += p.wall ? hb.Nlist_walls : 0;
    if (p.wall) {
      const int n1 = hb.walls_start[1], n2 = hb.Nlist_walls - hb.walls_start[1];
      nwchunk += (n1 + kWallChunk - 1) / kWallChunk + (n2 + kWallChunk - 1) / kWallChunk;
    }
    c->max_coll = std::max(c->max_coll, p.N_colloids);
  }
  Dev& d = c->d;
  d.Ntot = Ntot;
  d.Npad = (Ntot + 31) / 32 * 32;
  d.nboxes = nboxes;
  d.Ctot = Ctot;
  d.ncoll = ncoll;
  d.nwallseg = nwall;
  d.Nlist_coll = nlist;
  const int list_cap = o.nbr_capacity > 0 ? o.nbr_capacity : derived_capacity(c->boxes, c->dim);
  c->key_bits = bits_for(std::max(Ctot, 2));
  const size_t Np = d.Npad;
  bool ok = true;
  BoxParams* dbox = nullptr;
  ok = ok && dalloc(c, &dbox, nboxes);
  d.box = dbox;
  ok = ok && dalloc(c, &d.pos, Np) && dalloc(c, &d.vel, Np) && dalloc(c, &d.conf, 6 * Np);
  ok = ok && dalloc(c, &d.tinfo, Np) && dalloc(c, &d.gid, Np) && dalloc(c, &d.inv, Np);
  ok = ok && dalloc(c, &d.pos_b, Np) && dalloc(c, &d.vel_b, Np) && dalloc(c, &d.conf_b, 6 * Np);
  ok = ok && dalloc(c, &d.tinfo_b, Np) && dalloc(c, &d.gid_b, Np);
  if (c->prec == SPH_PREC_MIXED) ok = ok && dalloc(c, &d.pos_f, Np);
  ok = ok && dalloc(c, &d.dens, Np) && dalloc(c, &d.press, Np);
  ok = ok && dalloc(c, &d.f, 3 * Np) && dalloc(c, &d.dcdt, 6 * Np);
  ok = ok && dalloc(c, &d.f_b, 3 * Np) && dalloc(c, &d.dcdt_b, 6 * Np);
  ok = ok && dalloc(c, &d.gradv, 9 * Np);
  if (c->prec == SPH_PREC_MIXED) {
    RecF* r = nullptr;
    ok = ok && dalloc(c, &r, Np);
    d.rec = r;
  } else {
    RecD* r = nullptr;
    ok = ok && dalloc(c, &r, Np);
    d.rec = r;
  }
  ok = ok && dalloc(c, &d.nbr_cnt, Np) && dalloc(c, &d.nbr_nch, Np);
  ok = ok && dalloc(c, &d.key_by_gid, Np) && dalloc(c, &d.keys, Np) && dalloc(c, &d.vals, Np);
  ok = ok && dalloc(c, &d.keys_alt, Np) && dalloc(c, &d.vals_alt, Np);
  ok = ok && dalloc(c, &d.cell_begin, Ctot + 1) && dalloc(c, &d.cell_start, Ctot);
  ok = ok && dalloc(c, &d.cell_end, Ctot) && dalloc(c, &d.cell_box, Ctot);
  ok = ok && alloc_lists(c, list_cap);
  ok = ok && dalloc(c, &d.walls_list, nwl) && dalloc(c, &d.wall_seg, nwall + 1);
  ok = ok && dalloc(c, &d.wall_f, 3 * std::max(nwall, 1));
  d.nwallchunks = nwchunk;
  ok = ok && dalloc(c, &d.wall_chunk, nwchunk + 1) && dalloc(c, &d.wall_seg_chunk, nwall + 1);
  ok = ok && dalloc(c, &d.wall_part, 3 * (size_t)std::max(nwchunk, 1));
  ok = ok && dalloc(c, &d.colloids_list, nlist) && dalloc(c, &d.coll_seg, ncoll + 1);
  ok = ok && dalloc(c, &d.coll_box, ncoll) && dalloc(c, &d.xc, 3 * (size_t)std::max(nlist, 1));
  ok = ok && dalloc(c, &d.cs, (size_t)kCollFields * std::max(ncoll, 1));
  ok = ok && dalloc(c, &d.ccell, ncoll) && dalloc(c, &d.cindex, ncoll);
  ok = ok && dalloc(c, &d.ccell_start, ncc) && dalloc(c, &d.ccell_end, ncc);
  ok = ok && dalloc(c, &d.mag, 3 * nboxes) && dalloc(c, &d.ke, nboxes);
  ok = ok && dalloc(c, &d.step, 1) && dalloc(c, &d.status, 1) &&
       dalloc(c, &d.err_info, kErrInfoLen);
  // positions not yet looked at by a search: the pair passes keep the minimum image
  if (ok) cudaMemsetAsync(d.err_info + kPosOutside, 1, sizeof(int), c->stream);
  ok = ok && dalloc(c, &c->scratch, Np) && dalloc(c, &c->iscratch, Np);
  c->sort.hist_len = (int)sort_hist_len(Ntot, c->key_bits);
  ok = ok && dalloc(c, &c->sort.hist, (size_t)c->sort.hist_len);
  // kinetic-energy chunks
  std::vector<int> kchunk{0}, kbox{0};
  for (const HostBox& hb : c->boxes) {
    for (int s = hb.p.slot0; s < hb.p.slot0 + hb.p.N; s += 4096)
      kchunk.push_back(std::min(s + 4096, hb.p.slot0 + hb.p.N));
    kbox.push_back((int)kchunk.size() - 1);
  }
  d.nkechunks = (int)kchunk.size() - 1;
  ok = ok && dalloc(c, &d.ke_chunk, kchunk.size()) && dalloc(c, &d.ke_box_chunk, kbox.size());
  ok = ok && dalloc(c, &c->ke_partial, std::max(d.nkechunks, 1));
  ok = ok && dalloc(c, &c->obs_partial, 2 * (size_t)std::max(d.nkechunks, 1));
  ok = ok && dalloc(c, &c->obs_acc, (size_t)SPH_NUM_OBS * nboxes);
  if (!ok) {
    fprintf(stderr, "sph_create: device allocation failed\n");
    free_ctx(c);
    return SPH_ERR_NOMEM;
  }
  // ---- host images in id order (slot = id at start) ----
  // Without device initialisation the whole state is imaged on the host.  With it, only
  // the host-built particles (colloid shells, restart boxes) are packed and scattered.
  const bool full = !dev_init;
  size_t nh = 0;
  for (const HostBox& hb : c->boxes) nh += hb.x.size();
  std::vector<double4> pos(full ? Np : 0), vel(full ? Np : 0), hpos, hvel;
  std::vector<double> conf(full ? 6 * Np : 0, 0.0), hconf(full ? 0 : 6 * nh);
  std::vector<int2> hmeta;
  std::vector<int> tinfo(full ? Np : 0, 0), gid(full ? Np : 0, 0), cell_box(Ctot), wl,
      wseg{0}, cl, cseg{0}, cbox;
  std::vector<double> xc(3 * (size_t)std::max(nlist, 1), 0.0), cs((size_t)kCollFields * std::max(ncoll, 1), 0.0);
  std::vector<BoxParams> params;
  for (int b = 0; b < nboxes; ++b) {
    const HostBox& hb = c->boxes[b];
    const BoxParams& p = hb.p;
    params.push_back(p);
    for (int i = 0; i < (int)hb.x.size(); ++i) {
      const int s = p.slot0 + hb.host0 + i;
      const double4 x4 = make_double4(hb.x[i], hb.y[i], hb.z[i], hb.mass[i]);
      const double4 v4 = make_double4(hb.vx[i], hb.vy[i], hb.vz[i], 0.0);
      const double c6[6] = {hb.cxx[i], hb.cxy[i], hb.cyy[i], hb.cxz[i], hb.cyz[i], hb.czz[i]};
      const int t = (hb.type[i] & kTypeMask) | (b << kTypeBits);
      if (full) {
        pos[s] = x4;
        vel[s] = v4;
        for (int q = 0; q < 6; ++q) conf[q * Np + s] = c6[q];
        tinfo[s] = t;
        gid[s] = s;
      } else {
        const size_t k = hmeta.size();
        hmeta.push_back(make_int2(s, t));
        hpos.push_back(x4);
        hvel.push_back(v4);
        for (int q = 0; q < 6; ++q) hconf[q * nh + k] = c6[q];
      }
    }
    for (int q = 0; q < p.Ntotal_cells; ++q) cell_box[p.cell0 + q] = b;
    if (hb.lattice_on_device) ib[ib_of_box[b]].slot0 = p.slot0;
    if (p.wall && hb.lattice_on_device) {
      // entries written by the fill pass
      InitBox& B = ib[ib_of_box[b]];
      B.wl0 = (int)wl.size();
      wl.resize(wl.size() + hb.Nlist_walls, -1);
      wseg.push_back(B.wl0 + hb.walls_start[1]);
      wseg.push_back((int)wl.size());
    } else if (p.wall) {
      const int w1 = hb.walls_start[1];
      for (int k = 0; k < (int)hb.walls_list.size(); ++k) {
        if (k == w1) wseg.push_back((int)wl.size());
        wl.push_back(p.slot0 + hb.walls_list[k]);
      }
      if ((int)hb.walls_list.size() == w1) wseg.push_back((int)wl.size());
      wseg.push_back((int)wl.size());
    }
    for (int k = 0; k < p.N_colloids; ++k) {
      const int gc = p.coll0 + k;
      const int k0 = hb.colloids_start[k];
      const int k1 = k + 1 < p.N_colloids ? hb.colloids_start[k + 1] : (int)hb.colloids_list.size();
      for (int q = k0; q < k1; ++q) {
        const int e = (int)cl.size();
        cl.push_back(p.slot0 + hb.host0 + hb.colloids_list[q]);
        xc[e] = hb.x_center[q];
        xc[(size_t)std::max(nlist, 1) + e] = hb.y_center[q];
        xc[2 * (size_t)std::max(nlist, 1) + e] = hb.z_center[q];
      }
      cseg.push_back((int)cl.size());
      cbox.push_back(b);
      cs[CS_X * ncoll + gc] = hb.coll_x[k];
      cs[CS_Y * ncoll + gc] = hb.coll_y[k];
      cs[CS_Z * ncoll + gc] = hb.coll_z[k];
      cs[CS_Q0 * ncoll + gc] = 1.0;
    }
  }
  // chunks of the walls lists for the wall-force reduction
  std::vector<int> wchunk{0}, wsegchunk{0};
  for (size_t sgm = 0; sgm + 1 < wseg.size(); ++sgm) {
    for (int j = wseg[sgm]; j < wseg[sgm + 1]; j += kWallChunk)
      wchunk.push_back(std::min(j + kWallChunk, wseg[sgm + 1]));
    wsegchunk.push_back((int)wchunk.size() - 1);
  }
  if ((int)wchunk.size() - 1 != nwchunk || (int)wsegchunk.size() - 1 != nwall) ok = false;
  if (nboxes >= (1 << (31 - kTypeBits))) ok = false;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      ok = false;
  };
  up((void*)d.box, params.data(), params.size() * sizeof(BoxParams));
  d.one_box = nboxes == 1 ? 1 : 0;
  if (nboxes == 1) {
    const BoxParams& q = params[0];
    PairConsts& k = d.pc;
    for (int a = 0; a < 3; ++a) {
      k.L[a] = q.L[a];
      k.h[a] = q.halfL[a];
      k.Lf[a] = (float)q.L[a];
      k.hf[a] = (float)q.halfL[a];
    }
    k.rcutsq = q.rcutsq;
    k.rcut_inv = q.rcut_inv;
    k.c_gradw = q.c_gradw;
    k.a = q.a;
    k.b = q.b;
    k.rcutsqf = (float)q.rcutsq;
    k.rcut_invf = (float)q.rcut_inv;
    k.c_gradwf = (float)q.c_gradw;
    k.af = (float)q.a;
    k.bf = (float)q.b;
  }
  if (full) {
    up(d.pos, pos.data(), Np * sizeof(double4));
    up(d.vel, vel.data(), Np * sizeof(double4));
    up(d.conf, conf.data(), conf.size() * sizeof(double));
    up(d.tinfo, tinfo.data(), Np * sizeof(int));
    up(d.gid, gid.data(), Np * sizeof(int));
    up(d.inv, gid.data(), Np * sizeof(int));
  }
  up(d.cell_box, cell_box.data(), cell_box.size() * sizeof(int));
  up(d.walls_list, wl.data(), wl.size() * sizeof(int));
  up(d.wall_seg, wseg.data(), wseg.size() * sizeof(int));
  up(d.wall_chunk, wchunk.data(), wchunk.size() * sizeof(int));
  up(d.wall_seg_chunk, wsegchunk.data(), wsegchunk.size() * sizeof(int));
  up(d.colloids_list, cl.data(), cl.size() * sizeof(int));
  up(d.coll_seg, cseg.data(), cseg.size() * sizeof(int));
  up(d.coll_box, cbox.data(), cbox.size() * sizeof(int));
  up(d.xc, xc.data(), xc.size() * sizeof(double));
  up(d.cs, cs.data(), cs.size() * sizeof(double));
  up(d.ke_chunk, kchunk.data(), kchunk.size() * sizeof(int));
  up(d.ke_box_chunk, kbox.data(), kbox.size() * sizeof(int));
  if (ok && !full) {
    // the lattice boxes' particles and walls lists, then the host-built particles
    const Launch L = launcher(c);
    if (!ib.empty()) {
      int* d_offs = nullptr;
      ok = tmp.alloc(&d_offs, offs.size());
      up(d_ib, ib.data(), ib.size() * sizeof(InitBox));
      up(d_offs, offs.data(), offs.size() * sizeof(int));
      ok = ok && launch_init_fill(L, d_ib, d_blk_box, (int)blk_box.size(), d_centres, d_offs) == 0;
    }
    if (ok && nh > 0) {
      int2* d_meta = nullptr;
      double4 *d_hpos = nullptr, *d_hvel = nullptr;
      double* d_hconf = nullptr;
      ok = tmp.alloc(&d_meta, nh) && tmp.alloc(&d_hpos, nh) && tmp.alloc(&d_hvel, nh) &&
           tmp.alloc(&d_hconf, 6 * nh);
      up(d_meta, hmeta.data(), nh * sizeof(int2));
      up(d_hpos, hpos.data(), nh * sizeof(double4));
      up(d_hvel, hvel.data(), nh * sizeof(double4));
      up(d_hconf, hconf.data(), 6 * nh * sizeof(double));
      ok = ok && launch_init_scatter(L, (int)nh, d_meta, d_hpos, d_hvel, d_hconf) == 0;
    }
  }
  if (!ok || cudaStreamSynchronize(c->stream) != cudaSuccess) {
    fprintf(stderr, "sph_create: upload failed: %s\n", cudaGetErrorString(cudaGetLastError()));
    free_ctx(c);
    return SPH_ERR_CUDA;
  }
  *out = c;
  return SPH_OK;
}

sph_status sph_create(const sph_input* in, const char* particles_path, const sph_options* opt,
                      sph_ctx** out) {
  const char* paths[1] = {particles_path};
  return sph_create_ensemble(1, in, paths, opt, out);
}

void sph_destroy(sph_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  // A caller may reset the device before releasing the context (the reference's driver
  // calls cudaDeviceReset before class_system::destructor, main.cu:549-552); the reset
  // already released the device memory, stream, events and graphs, whose handles must not
  // be used again.  The context is alive iff its allocations are still known.
  bool alive = false;
  if (!ctx->allocs.empty()) {
    cudaPointerAttributes a;
    alive = cudaPointerGetAttributes(&a, ctx->allocs.front()) == cudaSuccess &&
            a.type == cudaMemoryTypeDevice;
    cudaGetLastError();
  }
  if (!alive) {
    delete ctx;
    return;
  }
  cudaStreamSynchronize(ctx->stream);
  free_ctx(ctx);
}

sph_status sph_get_info(const sph_ctx* c, int box, sph_info* o) {
  if (!c || !o || box < 0 || box >= c->nboxes) return SPH_ERR_STATE;
  fill_info(c->boxes[box], o);
  o->step = (int)c->host_step;
  o->nboxes = c->nboxes;
  o->precision = c->prec;
  return SPH_OK;
}

// ---- class_system methods ----
#define CTX_GUARD(c)                  \
  if (!(c)) return SPH_ERR_STATE;     \
  cudaSetDevice((c)->device);
// ... and, for every call except sph_step and sph_synchronize, first settles an open
// sph_step call (waits for it, resumes it after a list overflow or reports its failure)
#define CTX_SETTLED(c)                                  \
  CTX_GUARD(c);                                         \
  if ((c)->call_open) {                                 \
    const sph_status settle_status_ = settle_call(c);   \
    if (settle_status_ != SPH_OK) return settle_status_; \
  }

sph_status sph_neighbours_search(sph_ctx* c) {
  CTX_SETTLED(c);
  return search_checked(c);
}

sph_status sph_calculate_density(sph_ctx* c) {
  CTX_SETTLED(c);
  sph_status s = ensure_lists(c);
  if (s != SPH_OK) return s;
  if (launch_density_dim(launcher(c), c->dim)) return cuda_fail(c, "calculate_density");
  return SPH_OK;
}

sph_status sph_calculate_pressure(sph_ctx* c) {
  CTX_SETTLED(c);
  if (launch_pressure(launcher(c))) return cuda_fail(c, "calculate_pressure");
  return SPH_OK;
}

sph_status sph_calculate_vel_gradient(sph_ctx* c) {
  CTX_SETTLED(c);
  sph_status s = ensure_lists(c);
  if (s != SPH_OK) return s;
  // the pair pass reads the neighbour records, refreshed from the current state
  if (launch_pressure(launcher(c))) return cuda_fail(c, "records");
  if (launch_pairs_dim(launcher(c), c->dim, kPairGradvAll, 0)) return cuda_fail(c, "vel_gradient");
  c->gradv_valid = true;
  return SPH_OK;
}

sph_status sph_calculate_forces(sph_ctx* c, const double* m) {
  CTX_SETTLED(c);
  sph_status s = ensure_lists(c);
  if (s != SPH_OK) return s;
  s = m ? upload_moment(c, m) : host_moment(c, c->host_step + (c->in_step ? 1 : 0));
  if (s != SPH_OK) return s;
  Launch L = launcher(c);
  bool ext = false;
  for (const HostBox& hb : c->boxes) ext = ext || hb.p.ext_force_type != 0;
  // the reference stores the velocity gradient of every particle in this call: the fused
  // pass computes it for walls and colloid particles too (same terms, same order as the
  // standalone gradient pass)
  L.d.grad_all = 1;
  if (launch_density_dim(L, c->dim) || launch_pairs_dim(L, c->dim, kPairFused, ext ? 1 : 0) ||
      launch_wall_forces(L))
    return cuda_fail(c, "calculate_forces");
  bool pairs = false;
  for (const HostBox& hb : c->boxes) pairs = pairs || hb.p.N_colloids >= 2;
  if (launch_colloid_forces(L, pairs ? 1 : 0)) return cuda_fail(c, "calculate_forces");
  c->forces_live = true;
  c->gradv_valid = true;
  return SPH_OK;
}

sph_status sph_calculate_external_forces(sph_ctx* c) {
  CTX_SETTLED(c);
  if (launch_ext_force(launcher(c))) return cuda_fail(c, "external forces");
  return SPH_OK;
}

sph_status sph_calculate_force_walls(sph_ctx* c) {
  CTX_SETTLED(c);
  if (launch_wall_forces(launcher(c))) return cuda_fail(c, "force_walls");
  return SPH_OK;
}

sph_status sph_calculate_force_colloids(sph_ctx* c, const double* m) {
  CTX_SETTLED(c);
  sph_status s = m ? upload_moment(c, m) : host_moment(c, c->host_step + (c->in_step ? 1 : 0));
  if (s != SPH_OK) return s;
  if (c->pos_dirty) {
    s = search_checked(c);
    if (s != SPH_OK) return s;
  }
  bool pairs = false;
  for (const HostBox& hb : c->boxes) pairs = pairs || hb.p.N_colloids >= 2;
  if (launch_colloid_forces(launcher(c), pairs ? 1 : 0)) return cuda_fail(c, "force_colloids");
  return SPH_OK;
}

sph_status sph_vv_step1(sph_ctx* c) {
  CTX_SETTLED(c);
  if (ph_vv1(c)) return cuda_fail(c, "V_Verlet_step1");
  c->in_step = true;
  return SPH_OK;
}

sph_status sph_vv_step2(sph_ctx* c) {
  CTX_SETTLED(c);
  if (ph_vv2(c)) return cuda_fail(c, "V_Verlet_step2");
  c->host_step++;
  c->in_step = false;
  return SPH_OK;
}

sph_status sph_initial_forces(sph_ctx* c) {
  CTX_SETTLED(c);
  return do_initial(c);
}

sph_status sph_step(sph_ctx* c, int nsteps) {
  CTX_GUARD(c);
  if (nsteps < 0) return SPH_ERR_STATE;
  if (!c->initial_done) {
    if (c->call_open) {
      sph_status s = settle_call(c);
      if (s != SPH_OK) return s;
    }
    sph_status s = do_initial(c);
    if (s != SPH_OK) return s;
  }
  if (c->in_step) return fail(c, SPH_ERR_STATE, "sph_step inside a half-finished step");
  if (nsteps == 0) return SPH_OK;
  // calls made without a synchronize in between form one open call
  if (!c->call_open) {
    c->call_open = true;
    c->call_step0 = c->host_step;
    c->call_parity0 = c->parity;
  }
  cudaEventRecord(c->ev0, c->stream);
  sph_status s = run_steps(c, nsteps);
  c->call_target = c->host_step;
  if (s != SPH_OK) return s;
  cudaEventRecord(c->ev1, c->stream);
  c->events_recorded = true;
  return SPH_OK;
}

sph_status sph_synchronize(sph_ctx* c) {
  CTX_GUARD(c);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return cuda_fail(c, "synchronize");
  if (c->events_recorded) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) c->last_ms = ms;
    c->events_recorded = false;
  }
  sph_status s = c->call_open ? settle_call(c) : check_device(c);
  if (s == SPH_OK) {
    int used = 0;
    cudaMemcpy(&used, c->d.err_info + kErrMaxCount, sizeof(int), cudaMemcpyDeviceToHost);
    // keep headroom: grow the lists (and recapture) once 90% of the capacity is in use
    if (used > (9 * c->d.cap) / 10) s = grow_capacity(c, used);
  }
  return s;
}

sph_status sph_neighbour_lists(sph_ctx* c, int* capacity, int* max_used, int* grown) {
  CTX_SETTLED(c);
  int used = 0;
  if (cudaMemcpy(&used, c->d.err_info + kErrMaxCount, sizeof(int), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return cuda_fail(c, "list statistics");
  if (capacity) *capacity = c->d.cap;
  if (max_used) *max_used = used;
  if (grown) *grown = c->cap_grown;
  return SPH_OK;
}

sph_status sph_last_step_ms(sph_ctx* c, double* ms) {
  if (!c || !ms) return SPH_ERR_STATE;
  *ms = c->last_ms;
  return SPH_OK;
}

sph_status sph_kernel_launches(const sph_ctx* c, long long* count) {
  if (!c || !count) return SPH_ERR_STATE;
  *count = c->launches;
  return SPH_OK;
}

const char* sph_phase_name(int k) {
  static const char* names[SPH_NUM_PHASES] = {"vv1",           "hash",    "sort",  "reorder",
                                              "lists",         "colloid_cells", "density",
                                              "pairs",         "walls",   "colloids", "vv2"};
  return (k >= 0 && k < SPH_NUM_PHASES) ? names[k] : "";
}

sph_status sph_profile_phases(sph_ctx* c, int nsteps, double* ms) {
  CTX_SETTLED(c);
  if (!ms || nsteps <= 0) return SPH_ERR_STATE;
  if (!c->initial_done) {
    sph_status s = do_initial(c);
    if (s != SPH_OK) return s;
  }
  // the profiled steps are checked as one call (a failure stops them where it is found)
  const long long step0 = c->host_step;
  const int parity0 = c->parity;
  cudaEvent_t ev[SPH_NUM_PHASES + 1];
  for (auto& e : ev) cudaEventCreate(&e);
  std::vector<double> acc(SPH_NUM_PHASES, 0.0);
  bool ext = false, pairs = false;
  for (const HostBox& hb : c->boxes) {
    ext = ext || hb.p.ext_force_type != 0;
    pairs = pairs || hb.p.N_colloids >= 2;
  }
  int bad = 0;
  for (int s = 0; s < nsteps && !bad; ++s) {
    Launch L = launcher(c);
    cudaEventRecord(ev[0], c->stream);
    bad |= launch_vv1_colloids(L) | launch_vv1_particles(L);
    c->forces_live = false;
    cudaEventRecord(ev[1], c->stream);
    bad |= launch_hash(L);
    cudaEventRecord(ev[2], c->stream);
    bad |= launch_sort(L, c->key_bits, c->sort);
    cudaEventRecord(ev[3], c->stream);
    bad |= launch_reorder(L, false);
    swap_state(c, false);
    L = launcher(c);
    cudaEventRecord(ev[4], c->stream);
    bad |= launch_build_lists_dim(L, c->dim);
    cudaEventRecord(ev[5], c->stream);
    if (c->d.ncoll > 0) bad |= launch_colloid_cells_n(L, c->nboxes, c->max_coll);
    bad |= launch_advance_time(L, 0);
    cudaEventRecord(ev[6], c->stream);
    Launch Lf = L;
    Lf.d.gradv = nullptr;
    Lf.d.fold_vv2 = 1;  // as in the step graph: fluid half-kick inside the pair pass
    bad |= launch_density_dim(Lf, c->dim);
    cudaEventRecord(ev[7], c->stream);
    bad |= launch_pairs_dim(Lf, c->dim, kPairFused, ext ? 1 : 0);
    cudaEventRecord(ev[8], c->stream);
    bad |= launch_wall_forces(Lf);
    cudaEventRecord(ev[9], c->stream);
    bad |= launch_colloid_forces(Lf, pairs ? 1 : 0);
    cudaEventRecord(ev[10], c->stream);
    bad |= launch_vv2(L, false) | launch_count_step(L);
    cudaEventRecord(ev[11], c->stream);
    cudaEventSynchronize(ev[11]);
    for (int k = 0; k < SPH_NUM_PHASES; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
    c->host_step++;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  c->forces_live = true;
  c->pos_dirty = false;
  drop_graphs(c);  // the buffer parity may have changed
  if (bad) return cuda_fail(c, "profile_phases");
  for (int k = 0; k < SPH_NUM_PHASES; ++k) ms[k] = acc[k] / nsteps;
  c->call_open = true;
  c->call_step0 = step0;
  c->call_parity0 = parity0;
  c->call_target = c->host_step;
  return settle_call(c);
}

// ---- state access ----
sph_status sph_read_field_device(sph_ctx* c, int field, double* dev_out) {
  CTX_SETTLED(c);
  if (field < 0 || field >= SPH_NUM_PARTICLE_FIELDS || !dev_out) return SPH_ERR_STATE;
  if (field >= SPH_GXX && field <= SPH_GZZ && !c->gradv_valid) {
    if (sph_calculate_vel_gradient(c) != SPH_OK) return SPH_ERR_CUDA;
  }
  if (launch_gather_field(launcher(c), field, dev_out)) return cuda_fail(c, "read_field");
  return SPH_OK;
}

sph_status sph_read_field(sph_ctx* c, int field, double* host_out) {
  CTX_SETTLED(c);
  if (!host_out) return SPH_ERR_STATE;
  sph_status s = sph_read_field_device(c, field, c->scratch);
  if (s != SPH_OK) return s;
  if (cudaMemcpyAsync(host_out, c->scratch, (size_t)c->d.Ntot * sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return cuda_fail(c, "read_field copy");
  return SPH_OK;
}

sph_status sph_write_field(sph_ctx* c, int field, const double* host_in) {
  CTX_SETTLED(c);
  if (field < 0 || field >= SPH_NUM_PARTICLE_FIELDS || !host_in) return SPH_ERR_STATE;
  if (cudaMemcpyAsync(c->scratch, host_in, (size_t)c->d.Ntot * sizeof(double),
                      cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return cuda_fail(c, "write_field copy");
  if (launch_scatter_field(launcher(c), field, c->scratch)) return cuda_fail(c, "write_field");
  if (field <= SPH_Z) c->pos_dirty = true;
  drop_graphs(c);
  cudaStreamSynchronize(c->stream);
  return SPH_OK;
}

sph_status sph_read_type(sph_ctx* c, int* host_out) {
  CTX_SETTLED(c);
  if (!host_out) return SPH_ERR_STATE;
  if (launch_gather_int(launcher(c), c->d.tinfo, c->iscratch)) return cuda_fail(c, "read_type");
  std::vector<int> t(c->d.Ntot);
  if (cudaMemcpyAsync(t.data(), c->iscratch, t.size() * sizeof(int), cudaMemcpyDeviceToHost,
                      c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return cuda_fail(c, "read_type copy");
  for (size_t i = 0; i < t.size(); ++i) host_out[i] = t[i] & kTypeMask;
  return SPH_OK;
}

sph_status sph_read_colloid_field(sph_ctx* c, int field, double* host_out) {
  CTX_SETTLED(c);
  if (field < 0 || field >= SPH_NUM_COLLOID_FIELDS || !host_out) return SPH_ERR_STATE;
  if (c->d.ncoll == 0) return SPH_OK;
  if (cudaMemcpyAsync(host_out, c->d.cs + (size_t)field * c->d.ncoll,
                      (size_t)c->d.ncoll * sizeof(double), cudaMemcpyDeviceToHost,
                      c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return cuda_fail(c, "read_colloid_field");
  return SPH_OK;
}

sph_status sph_read_wall_forces(sph_ctx* c, double* host_out) {
  CTX_SETTLED(c);
  if (!host_out) return SPH_ERR_STATE;
  std::vector<double> wf(3 * (size_t)std::max(c->d.nwallseg, 1));
  if (c->d.nwallseg > 0 &&
      (cudaMemcpyAsync(wf.data(), c->d.wall_f, 3 * (size_t)c->d.nwallseg * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
       cudaStreamSynchronize(c->stream) != cudaSuccess))
    return cuda_fail(c, "read_wall_forces");
  for (int b = 0; b < c->nboxes; ++b) {
    const BoxParams& p = c->boxes[b].p;
    for (int q = 0; q < 6; ++q)
      host_out[6 * b + q] = p.wall ? wf[3 * (size_t)p.wall_seg0 + q] : 0.0;
  }
  return SPH_OK;
}

sph_status sph_export_cells(sph_ctx* c, int* particle_cell, int* particle_index,
                            int* cell_start, int* cell_end) {
  CTX_SETTLED(c);
  const BoxParams& p = c->boxes[0].p;
  cudaStream_t st = c->stream;
  bool ok = true;
  auto dn = [&](void* dst, const void* src, size_t bytes) {
    if (dst && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st) != cudaSuccess) ok = false;
  };
  dn(particle_cell, c->d.keys + p.slot0, (size_t)p.N * sizeof(int));
  dn(particle_index, c->d.vals + p.slot0, (size_t)p.N * sizeof(int));
  dn(cell_start, c->d.cell_start + p.cell0, (size_t)p.Ntotal_cells * sizeof(int));
  dn(cell_end, c->d.cell_end + p.cell0, (size_t)p.Ntotal_cells * sizeof(int));
  if (!ok || cudaStreamSynchronize(st) != cudaSuccess) return cuda_fail(c, "export_cells");
  return SPH_OK;
}

sph_status sph_export_colloid_cells(sph_ctx* c, int* coll_cell, int* coll_index,
                                    int* coll_cell_start, int* coll_cell_end) {
  CTX_SETTLED(c);
  const BoxParams& p = c->boxes[0].p;
  if (p.N_colloids == 0) return SPH_OK;
  cudaStream_t st = c->stream;
  bool ok = true;
  auto dn = [&](void* dst, const void* src, size_t bytes) {
    if (dst && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st) != cudaSuccess) ok = false;
  };
  dn(coll_cell, c->d.ccell + p.coll0, (size_t)p.N_colloids * sizeof(int));
  dn(coll_index, c->d.cindex + p.coll0, (size_t)p.N_colloids * sizeof(int));
  dn(coll_cell_start, c->d.ccell_start + p.ccell0, (size_t)p.Ntotal_cells_colloids * sizeof(int));
  dn(coll_cell_end, c->d.ccell_end + p.ccell0, (size_t)p.Ntotal_cells_colloids * sizeof(int));
  if (!ok || cudaStreamSynchronize(st) != cudaSuccess) return cuda_fail(c, "export_colloid_cells");
  return SPH_OK;
}

sph_status sph_kinetic_energy(sph_ctx* c, double* host_out) {
  CTX_SETTLED(c);
  if (!host_out) return SPH_ERR_STATE;
  if (launch_kinetic_energy(launcher(c), c->ke_partial)) return cuda_fail(c, "kinetic_energy");
  if (cudaMemcpyAsync(host_out, c->d.ke, (size_t)c->nboxes * sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return cuda_fail(c, "kinetic_energy copy");
  return SPH_OK;
}

// ---- observables ----
sph_status sph_observe(sph_ctx* c) {
  CTX_SETTLED(c);
  if (c->in_step) return fail(c, SPH_ERR_STATE, "observe inside a half-finished step");
  if (!c->initial_done) {
    sph_status s = do_initial(c);
    if (s != SPH_OK) return s;
  }
  if (launch_observe(launcher(c), c->ke_partial, c->obs_partial, c->obs_acc))
    return cuda_fail(c, "observe");
  c->obs_samples++;
  return SPH_OK;
}

sph_status sph_observables(sph_ctx* c, double* host_out, long long* nsamples) {
  CTX_SETTLED(c);
  if (!host_out) return SPH_ERR_STATE;
  const size_t n = (size_t)SPH_NUM_OBS * c->nboxes;
  if (cudaMemcpyAsync(host_out, c->obs_acc, n * sizeof(double), cudaMemcpyDeviceToHost,
                      c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return cuda_fail(c, "observables");
  const double inv = c->obs_samples > 0 ? 1.0 / (double)c->obs_samples : 0.0;
  for (size_t k = 0; k < n; ++k) host_out[k] *= inv;
  if (nsamples) *nsamples = c->obs_samples;
  return SPH_OK;
}

sph_status sph_reset_observables(sph_ctx* c) {
  CTX_SETTLED(c);
  if (cudaMemsetAsync(c->obs_acc, 0, (size_t)SPH_NUM_OBS * c->nboxes * sizeof(double),
                      c->stream) != cudaSuccess)
    return cuda_fail(c, "reset_observables");
  c->obs_samples = 0;
  return SPH_OK;
}

// ---- binary checkpoint ----
// Layout: 8-byte magic, then int32 version, dim, nboxes, nfields, initial_done; int64
// Ntot, ncoll, step; then nfields particle fields (Ntot doubles each, sph_field order
// SPH_X .. SPH_DCDT_ZZ), the particle types (Ntot int32) and the colloid state
// (SPH_NUM_COLLOID_FIELDS x ncoll doubles).  All in original particle order.
namespace {
const char kCkptMagic[8] = {'S', 'P', 'H', 'C', 'K', 'P', 'T', '1'};
constexpr int kCkptVersion = 1;
constexpr int kCkptFields = SPH_DCDT_ZZ + 1;  // f and dc/dt: the next half-kick needs them
struct CkptHeader {
  char magic[8];
  int32_t version, dim, nboxes, nfields, initial_done, pad;
  int64_t Ntot, ncoll, step;
};
}  // namespace

sph_status sph_save_checkpoint(sph_ctx* c, const char* path) {
  CTX_SETTLED(c);
  if (!path) return SPH_ERR_STATE;
  if (c->in_step) return fail(c, SPH_ERR_STATE, "checkpoint inside a half-finished step");
  sph_status s = sph_synchronize(c);
  if (s != SPH_OK) return s;
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kCkptMagic, sizeof(h.magic));
  h.version = kCkptVersion;
  h.dim = c->dim;
  h.nboxes = c->nboxes;
  h.nfields = kCkptFields;
  h.initial_done = c->initial_done ? 1 : 0;
  h.Ntot = c->d.Ntot;
  h.ncoll = c->d.ncoll;
  h.step = c->host_step;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(c, SPH_ERR_IO, "cannot open the checkpoint file");
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  std::vector<double> buf((size_t)std::max(c->d.Ntot, 1));
  for (int k = 0; k < kCkptFields && ok; ++k) {
    s = sph_read_field(c, k, buf.data());
    ok = s == SPH_OK && std::fwrite(buf.data(), sizeof(double), c->d.Ntot, f) == (size_t)c->d.Ntot;
  }
  std::vector<int> type((size_t)std::max(c->d.Ntot, 1));
  if (ok) {
    s = sph_read_type(c, type.data());
    ok = s == SPH_OK && std::fwrite(type.data(), sizeof(int), c->d.Ntot, f) == (size_t)c->d.Ntot;
  }
  std::vector<double> cs((size_t)kCollFields * c->d.ncoll);
  if (ok && c->d.ncoll > 0) {
    ok = cudaMemcpy(cs.data(), c->d.cs, cs.size() * sizeof(double), cudaMemcpyDeviceToHost) ==
             cudaSuccess &&
         std::fwrite(cs.data(), sizeof(double), cs.size(), f) == cs.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return s != SPH_OK ? s : fail(c, SPH_ERR_IO, "cannot write the checkpoint");
  return SPH_OK;
}

sph_status sph_load_checkpoint(sph_ctx* c, const char* path) {
  CTX_SETTLED(c);
  if (!path) return SPH_ERR_STATE;
  if (c->in_step) return fail(c, SPH_ERR_STATE, "checkpoint inside a half-finished step");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(c, SPH_ERR_IO, "cannot open the checkpoint file");
  CkptHeader h;
  bool ok = std::fread(&h, sizeof(h), 1, f) == 1;
  if (!ok || std::memcmp(h.magic, kCkptMagic, sizeof(h.magic)) != 0 ||
      h.version != kCkptVersion || h.nfields != kCkptFields) {
    std::fclose(f);
    return fail(c, SPH_ERR_BAD_INPUT, "not a checkpoint of this format");
  }
  if (h.dim != c->dim || h.nboxes != c->nboxes || h.Ntot != c->d.Ntot ||
      h.ncoll != c->d.ncoll) {
    std::fclose(f);
    return fail(c, SPH_ERR_BAD_INPUT, "the checkpoint belongs to a different system");
  }
  const size_t n = (size_t)c->d.Ntot;
  std::vector<std::vector<double>> fields(kCkptFields, std::vector<double>(n));
  for (int k = 0; k < kCkptFields && ok; ++k)
    ok = std::fread(fields[k].data(), sizeof(double), n, f) == n;
  std::vector<int> type(n), mine(n);
  if (ok) ok = std::fread(type.data(), sizeof(int), n, f) == n;
  std::vector<double> cs((size_t)kCollFields * c->d.ncoll);
  if (ok && !cs.empty()) ok = std::fread(cs.data(), sizeof(double), cs.size(), f) == cs.size();
  std::fclose(f);
  if (!ok) return fail(c, SPH_ERR_IO, "truncated checkpoint");
  sph_status s = sph_read_type(c, mine.data());
  if (s != SPH_OK) return s;
  if (type != mine) return fail(c, SPH_ERR_BAD_INPUT, "particle types differ from the checkpoint");
  for (int k = 0; k < kCkptFields; ++k) {
    s = sph_write_field(c, k, fields[k].data());
    if (s != SPH_OK) return s;
  }
  const long long step = h.step;
  if ((!cs.empty() && cudaMemcpy(c->d.cs, cs.data(), cs.size() * sizeof(double),
                                 cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(c->d.step, &step, sizeof(step), cudaMemcpyHostToDevice) != cudaSuccess)
    return cuda_fail(c, "checkpoint upload");
  c->host_step = step;
  c->initial_done = h.initial_done != 0;
  c->forces_live = c->initial_done;
  c->gradv_valid = false;
  c->pos_dirty = true;
  drop_graphs(c);
  return SPH_OK;
}

}  // extern "C"

// ---- launch geometry and the autotuner ----
namespace {

bool tuning_ok(const sph_tuning& t) {
  return (t.list_threads_per_cell == 32 || t.list_threads_per_cell == 16) &&
         (t.density_block == 0 || t.density_block == 64 || t.density_block == 128 ||
          t.density_block == 256);
}

// Cache key: GPU name, dimension, overlap of the first box, total particles rounded to a
// power of two.
std::string tune_key(const sph_ctx* c) {
  cudaDeviceProp prop;
  std::string name = cudaGetDeviceProperties(&prop, c->device) == cudaSuccess ? prop.name : "gpu";
  for (char& ch : name)
    if (ch == '"' || ch == '\\') ch = '_';
  int lg = 0;
  while ((1ll << (lg + 1)) <= (long long)std::max(c->d.Ntot, 1)) ++lg;
  if ((1ll << (lg + 1)) - c->d.Ntot < c->d.Ntot - (1ll << lg)) ++lg;
  char buf[320];
  std::snprintf(buf, sizeof(buf), "%s|dim=%d|overlap=%g|N=2^%d", name.c_str(), c->dim,
                c->boxes.empty() ? 0.0 : c->boxes[0].in.overlap, lg);
  return buf;
}

// The cache file is a JSON object with one entry per line:
//   "<key>": {"list_threads_per_cell": 16, "density_block": 128, "lists_ms": .., "density_ms": ..},
bool cache_lookup(const char* path, const std::string& key, sph_tuning* t) {
  std::ifstream f(path);
  if (!f) return false;
  const std::string head = "\"" + key + "\":";
  std::string line;
  while (std::getline(f, line)) {
    const size_t a = line.find(head);
    if (a == std::string::npos) continue;
    sph_tuning r{0, 0};
    const size_t p1 = line.find("\"list_threads_per_cell\":", a);
    const size_t p2 = line.find("\"density_block\":", a);
    if (p1 == std::string::npos || p2 == std::string::npos) return false;
    r.list_threads_per_cell = std::atoi(line.c_str() + p1 + 24);
    r.density_block = std::atoi(line.c_str() + p2 + 16);
    if (!tuning_ok(r)) return false;
    *t = r;
    return true;
  }
  return false;
}

bool cache_store(const char* path, const std::string& key, const sph_tuning& t, double lists_ms,
                 double density_ms) {
  std::vector<std::string> keep;
  {
    std::ifstream f(path);
    std::string line;
    const std::string head = "\"" + key + "\":";
    while (f && std::getline(f, line)) {
      const size_t q = line.find('"');
      if (q == std::string::npos || line.find(head) != std::string::npos) continue;
      while (!line.empty() && (line.back() == ',' || line.back() == ' ' || line.back() == '\r'))
        line.pop_back();
      keep.push_back(line);
    }
  }
  char entry[512];
  std::snprintf(entry, sizeof(entry),
                "\"%s\": {\"list_threads_per_cell\": %d, \"density_block\": %d, "
                "\"lists_ms\": %.4f, \"density_ms\": %.4f}",
                key.c_str(), t.list_threads_per_cell, t.density_block, lists_ms, density_ms);
  keep.push_back(entry);
  const std::string tmp = std::string(path) + ".tmp";
  {
    std::ofstream o(tmp);
    if (!o) return false;
    o << "{\n";
    for (size_t k = 0; k < keep.size(); ++k) o << keep[k] << (k + 1 < keep.size() ? ",\n" : "\n");
    o << "}\n";
    if (!o) return false;
  }
  return std::rename(tmp.c_str(), path) == 0;
}

// Mean device time (ms) of `reps` launches of one phase after one warm-up launch.
template <typename F>
double time_phase(sph_ctx* c, int reps, F launch, bool* bad) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  *bad |= launch() != 0;
  cudaEventRecord(e0, c->stream);
  for (int r = 0; r < reps; ++r) *bad |= launch() != 0;
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / reps;
}

}  // namespace

extern "C" {

sph_status sph_get_tuning(const sph_ctx* c, sph_tuning* out) {
  if (!c || !out) return SPH_ERR_STATE;
  *out = c->tune;
  return SPH_OK;
}

sph_status sph_set_tuning(sph_ctx* c, const sph_tuning* t) {
  CTX_SETTLED(c);
  if (!t || !tuning_ok(*t)) return fail(c, SPH_ERR_STATE, "unsupported launch geometry");
  c->tune = *t;
  drop_graphs(c);  // the captured steps carry the old geometry
  return SPH_OK;
}

sph_status sph_autotune(sph_ctx* c, const char* cache_path, sph_tuning* chosen) {
  CTX_SETTLED(c);
  if (c->in_step) return fail(c, SPH_ERR_STATE, "autotune inside a half-finished step");
  const std::string key = tune_key(c);
  sph_tuning t;
  if (cache_path && cache_lookup(cache_path, key, &t)) {
    sph_status s = sph_set_tuning(c, &t);
    if (s == SPH_OK && chosen) *chosen = t;
    return s;
  }
  // valid lists for the current positions; both timed phases recompute the same values
  // from the current state, so tuning leaves the simulation where it was
  sph_status s = ensure_lists(c);
  if (s != SPH_OK) return s;
  const int reps = c->d.Ntot > (1 << 20) ? 3 : 10;
  bool bad = false;
  sph_tuning best = c->tune;
  double best_lists = 1e300, best_dens = 1e300;
  for (int tpc : {32, 16}) {
    Launch L = launcher(c);
    L.list_tpc = tpc;
    const double ms = time_phase(c, reps, [&] { return launch_build_lists_dim(L, c->dim); }, &bad);
    if (ms < best_lists) {
      best_lists = ms;
      best.list_threads_per_cell = tpc;
    }
  }
  for (int nt : {0, 64, 128, 256}) {  // 0: neighbour-cell tiles
    Launch L = launcher(c);
    L.density_block = nt;
    const double ms = time_phase(c, reps, [&] { return launch_density_dim(L, c->dim); }, &bad);
    if (ms < best_dens) {
      best_dens = ms;
      best.density_block = nt;
    }
  }
  if (bad) return cuda_fail(c, "autotune");
  s = check_device(c);
  if (s != SPH_OK) return s;
  s = sph_set_tuning(c, &best);
  if (s != SPH_OK) return s;
  if (cache_path && !cache_store(cache_path, key, best, best_lists, best_dens))
    return fail(c, SPH_ERR_IO, "cannot write the autotune cache");
  if (chosen) *chosen = best;
  return SPH_OK;
}

}  // extern "C"
