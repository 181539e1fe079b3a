// sph_run.cpp -- command-line driver: runs a reference-format `input` file the way the
// reference's program does (src/main.cu:30-470: read, build, initial forces, Nsteps
// velocity-Verlet steps, output every freq_* steps) and writes the same files
// (micro-<step>.dat, walls-<step>.dat, colloids-<step>.dat, macro.dat).
//
// Steps between two outputs run as one sph_step call (CUDA-graph replays, no host
// round trip per step).  An output copies the fields to host memory and hands them to a
// writer thread; the GPU goes on with the next steps while the files are formatted.
//
//   sph_run [--input FILE] [--particles FILE] [--precision fp64|mixed] [--no-graph]
//           [--steps N] [--checkpoint FILE] [--restart FILE] [--autotune CACHE]
//           [--device-init] [--quiet]
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "sph_capi.h"
#include "sph_io.h"

namespace {

struct Args {
  std::string input = "input";
  std::string particles;  // empty: the reference's input_particles.in
  int precision = SPH_PREC_FP64;
  bool graph = true;
  int steps = -1;  // -1: Nsteps of the input file
  std::string checkpoint, restart, autotune;
  bool quiet = false;
  bool device_init = false;
};

bool parse_args(int argc, char** argv, Args* a) {
  for (int k = 1; k < argc; ++k) {
    const std::string s = argv[k];
    auto next = [&](std::string* v) {
      if (k + 1 >= argc) return false;
      *v = argv[++k];
      return true;
    };
    std::string v;
    if (s == "--input") {
      if (!next(&a->input)) return false;
    } else if (s == "--particles") {
      if (!next(&a->particles)) return false;
    } else if (s == "--precision") {
      if (!next(&v)) return false;
      if (v == "fp64") a->precision = SPH_PREC_FP64;
      else if (v == "mixed") a->precision = SPH_PREC_MIXED;
      else return false;
    } else if (s == "--no-graph") {
      a->graph = false;
    } else if (s == "--steps") {
      if (!next(&v)) return false;
      a->steps = std::atoi(v.c_str());
    } else if (s == "--checkpoint") {
      if (!next(&a->checkpoint)) return false;
    } else if (s == "--restart") {
      if (!next(&a->restart)) return false;
    } else if (s == "--autotune") {
      if (!next(&a->autotune)) return false;
    } else if (s == "--device-init") {
      a->device_init = true;
    } else if (s == "--quiet") {
      a->quiet = true;
    } else {
      return false;
    }
  }
  return true;
}

// One output step's data, owned by the writer queue.
struct Snapshot {
  int step = 0;
  bool micro = false, walls = false, colloids = false, macro = false;
  std::vector<std::vector<double>> f;  // particle fields, micro-file order
  std::vector<double> wall_f;
  std::vector<std::vector<double>> coll;  // 15 colloid columns
  double ke = 0.0;
};

// Writer thread with a bounded queue (two snapshots in flight: one being written, one
// being filled), so output steps overlap the next steps' GPU work.
class Writer {
 public:
  Writer(int dim, int n, int ncoll, const std::vector<int>* type, bool quiet)
      : dim_(dim), n_(n), ncoll_(ncoll), type_(type), quiet_(quiet), th_([this] { run(); }) {}
  ~Writer() { finish(); }
  void push(Snapshot&& s) {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return q_.size() < 2; });
    q_.push_back(std::move(s));
    cv_.notify_all();
  }
  void finish() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (done_) return;
      done_ = true;
      cv_.notify_all();
    }
    th_.join();
  }
  bool ok() const { return ok_; }

 private:
  void run() {
    for (;;) {
      Snapshot s;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !q_.empty() || done_; });
        if (q_.empty()) return;
        s = std::move(q_.front());
        q_.pop_front();
        cv_.notify_all();
      }
      write(s);
    }
  }
  void write(const Snapshot& s) {
    char name[64];
    if (s.micro) {
      std::snprintf(name, sizeof(name), "micro-%d.dat", s.step);
      const auto& f = s.f;
      ok_ &= sph_write_micro(name, dim_, n_, f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                             f[4].data(), f[5].data(), f[6].data(), f[7].data(), f[8].data(),
                             type_->data(), f[9].data(), f[10].data(), f[11].data(),
                             f[12].data(), f[13].data(), f[14].data()) == SPH_OK;
      if (!quiet_) std::printf("Micro file written. Time step %d\n", s.step);
    }
    if (s.walls) {
      std::snprintf(name, sizeof(name), "walls-%d.dat", s.step);
      const double fx[2] = {s.wall_f[0], s.wall_f[3]}, fy[2] = {s.wall_f[1], s.wall_f[4]},
                   fz[2] = {s.wall_f[2], s.wall_f[5]};
      ok_ &= sph_write_walls(name, dim_, 2, fx, fy, fz) == SPH_OK;
      if (!quiet_) std::printf("Walls file written. Time step %d\n", s.step);
    }
    if (s.colloids) {
      std::snprintf(name, sizeof(name), "colloids-%d.dat", s.step);
      const double* cols[15];
      for (int k = 0; k < 15; ++k) cols[k] = s.coll[k].data();
      ok_ &= sph_write_colloids(name, dim_, ncoll_, cols) == SPH_OK;
      if (!quiet_) std::printf("Colloids file written. Time step %d\n", s.step);
    }
    if (s.macro) ok_ &= sph_append_macro("macro.dat", s.step, s.ke) == SPH_OK;
  }

  int dim_, n_, ncoll_;
  const std::vector<int>* type_;
  bool quiet_;
  bool ok_ = true;
  bool done_ = false;
  std::deque<Snapshot> q_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::thread th_;
};

int fail(const char* what, sph_status s, sph_ctx* ctx) {
  std::fprintf(stderr, "sph_run: %s: %s%s%s\n", what, sph_status_string(s), ctx ? ": " : "",
               ctx ? sph_last_error(ctx) : "");
  return 1;
}

bool due(int step, int freq) { return freq > 0 && step % freq == 0; }

}  // namespace

int main(int argc, char** argv) {
  Args a;
  if (!parse_args(argc, argv, &a)) {
    std::fprintf(stderr,
                 "usage: sph_run [--input FILE] [--particles FILE] [--precision fp64|mixed]\n"
                 "               [--no-graph] [--steps N] [--checkpoint FILE] [--restart FILE]"
                 " [--autotune CACHE] [--device-init] [--quiet]\n");
    return 2;
  }
  sph_input in;
  std::vector<double> coll(3 * (size_t)SPH_MAX_COLLOIDS);
  char msg[512] = {0};
  sph_status s = sph_read_input(a.input.c_str(), &in, coll.data(), SPH_MAX_COLLOIDS, msg,
                                sizeof(msg));
  if (s != SPH_OK) {
    std::fprintf(stderr, "sph_run: %s\n", msg);
    return 1;
  }
  sph_options opt;
  std::memset(&opt, 0, sizeof(opt));
  opt.precision = a.precision;
  opt.use_graph = a.graph ? 1 : 0;
  opt.init_on_device = a.device_init ? 1 : 0;
  sph_ctx* ctx = nullptr;
  s = sph_create(&in, a.particles.empty() ? nullptr : a.particles.c_str(), &opt, &ctx);
  if (s != SPH_OK) return fail("create", s, nullptr);
  sph_info info;
  sph_get_info(ctx, 0, &info);
  const int N = info.N, dim = info.dim, nc = info.N_colloids;
  const int nsteps = a.steps >= 0 ? a.steps : in.Nsteps;
  if (!a.quiet)
    std::printf("sph_run: %d particles, dim %d, %d colloids, %d steps, %s%s\n", N, dim, nc,
                nsteps, a.precision == SPH_PREC_MIXED ? "mixed precision" : "fp64",
                a.graph ? ", CUDA graphs" : "");

  int step0 = 0;
  if (!a.restart.empty()) {
    s = sph_load_checkpoint(ctx, a.restart.c_str());
    if (s != SPH_OK) return fail("restart", s, ctx);
    sph_get_info(ctx, 0, &info);
    step0 = info.step;
  } else {
    s = sph_initial_forces(ctx);
    if (s != SPH_OK) return fail("initial forces", s, ctx);
  }

  if (!a.autotune.empty()) {
    sph_tuning t;
    s = sph_autotune(ctx, a.autotune.c_str(), &t);
    if (s != SPH_OK) return fail("autotune", s, ctx);
    if (!a.quiet)
      std::printf("sph_run: launch geometry %d threads per cell, density blocks of %d\n",
                  t.list_threads_per_cell, t.density_block);
  }

  std::vector<int> type((size_t)N);
  s = sph_read_type(ctx, type.data());
  if (s != SPH_OK) return fail("read types", s, ctx);
  Writer writer(dim, N, nc, &type, a.quiet);

  const int micro_fields[15] = {SPH_X,   SPH_Y,    SPH_Z,   SPH_VX,  SPH_VY,
                                SPH_VZ,  SPH_MASS, SPH_DENS, SPH_PRESS, SPH_CXX,
                                SPH_CXY, SPH_CYY,  SPH_CXZ, SPH_CYZ, SPH_CZZ};
  const int coll_fields[15] = {SPH_COLL_X,      SPH_COLL_Y,      SPH_COLL_Z,
                               SPH_COLL_VX,     SPH_COLL_VY,     SPH_COLL_VZ,
                               SPH_COLL_OMEGAX, SPH_COLL_OMEGAY, SPH_COLL_OMEGAZ,
                               SPH_COLL_FX,     SPH_COLL_FY,     SPH_COLL_FZ,
                               SPH_COLL_TX,     SPH_COLL_TY,     SPH_COLL_TZ};
  // main.cu:326-340 (step 0) and 453-467 (every step): system_print_output.cpp:58-82
  auto output = [&](int step) -> sph_status {
    Snapshot snap;
    snap.step = step;
    snap.micro = due(step, in.freq_micro);
    snap.walls = in.wall == 1 && due(step, in.freq_walls);
    snap.colloids = nc > 0 && due(step, in.freq_colloids);
    snap.macro = due(step, in.freq_macro);
    if (!(snap.micro || snap.walls || snap.colloids || snap.macro)) return SPH_OK;
    sph_status r = sph_synchronize(ctx);
    if (r != SPH_OK) return r;
    if (snap.micro) {
      snap.f.assign(15, std::vector<double>((size_t)N));
      for (int k = 0; k < 15 && r == SPH_OK; ++k)
        r = sph_read_field(ctx, micro_fields[k], snap.f[k].data());
    }
    if (r == SPH_OK && snap.walls) {
      snap.wall_f.assign(6, 0.0);
      r = sph_read_wall_forces(ctx, snap.wall_f.data());
    }
    if (r == SPH_OK && snap.colloids) {
      snap.coll.assign(15, std::vector<double>((size_t)nc));
      for (int k = 0; k < 15 && r == SPH_OK; ++k)
        r = sph_read_colloid_field(ctx, coll_fields[k], snap.coll[k].data());
    }
    if (r == SPH_OK && snap.macro) r = sph_kinetic_energy(ctx, &snap.ke);
    if (r == SPH_OK) writer.push(std::move(snap));
    return r;
  };

  if (step0 == 0) {
    s = output(0);
    if (s != SPH_OK) return fail("output", s, ctx);
  }
  const auto t0 = std::chrono::steady_clock::now();
  int step = step0;
  const int last = step0 + nsteps;
  while (step < last) {
    // run up to the next step that writes anything
    int next = step + 1;
    while (next < last && !(due(next, in.freq_micro) || due(next, in.freq_macro) ||
                            (in.wall == 1 && due(next, in.freq_walls)) ||
                            (nc > 0 && due(next, in.freq_colloids))))
      ++next;
    s = sph_step(ctx, next - step);
    if (s != SPH_OK) return fail("step", s, ctx);
    step = next;
    s = output(step);
    if (s != SPH_OK) return fail("output", s, ctx);
  }
  s = sph_synchronize(ctx);
  if (s != SPH_OK) return fail("synchronize", s, ctx);
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  writer.finish();
  if (!writer.ok()) {
    std::fprintf(stderr, "sph_run: an output file could not be written\n");
    return 1;
  }
  if (!a.checkpoint.empty()) {
    s = sph_save_checkpoint(ctx, a.checkpoint.c_str());
    if (s != SPH_OK) return fail("checkpoint", s, ctx);
  }
  if (!a.quiet)
    std::printf("Total time: %f seconds (%d steps, %.3e particle-steps/s)\n", secs, nsteps,
                secs > 0 ? (double)N * nsteps / secs : 0.0);
  sph_destroy(ctx);
  return 0;
}
