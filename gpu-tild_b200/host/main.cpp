// main.cpp — `gpu-tild -in <script>`: the drop-in driver over libtild.
//
// Reproduces the reference's main loop (main.cu:228-419) in the same order: initialize, step-0
// trajectory frame, data.dat header, forces + calc_properties at step 0, then per step the
// integrator, computes, trajectory / grid / binary output, log line and compute results, with
// the prefactor ramp applied inside tild_step.  Output files and their text formats follow
// config_utils.cu:366-403 (traj), io_utils.cu:7-134 (rho%d.dat, avg_sk_%d.dat, binary files),
// read_input.cu:565-651 (NEED_A_NAME.input) and main.cu:252-265, 422-485 (data.dat, stdout).
// Steps between two output events are run as one tild_step(n) call.  Trajectory, grid and binary
// frames are snapshotted asynchronously (tild_snapshot_async) and formatted and written by a
// writer thread while the GPU keeps stepping; files receive the same bytes in the same order.
//
// Extra flags (not in the reference): --dry-run parses the script and data file and writes
// NEED_A_NAME.input without touching a GPU; --device N picks the GPU.
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/tild.h"
#include "script.hpp"

using tildhost::Script;

namespace {

constexpr float kPI2 = 6.2831853071f;  // globals.h:30

struct Run {
  Script s;
  tild_ctx* ctx = nullptr;
  int step = 0;
  std::ofstream dout;
  tild_obs obs;
  int M = 1;
  float V = 1.f;
};

void check(Run& r, int st, const char* what) {
  if (st != TILD_OK) {
    std::cout << what << " failed: " << tild_status_string(st) << ": " << tild_last_error(r.ctx) << std::endl;
    throw std::runtime_error(what);
  }
}

void unstack(const Script& s, int id, int* nn) {  // array_utils.cu:62-81
  if (s.Dim == 2) {
    nn[1] = id / s.Nx[0];
    nn[0] = id - nn[1] * s.Nx[0];
  } else {
    nn[2] = id / s.Nx[1] / s.Nx[0];
    nn[1] = id / s.Nx[0] - nn[2] * s.Nx[1];
    nn[0] = id - (nn[1] + nn[2] * s.Nx[1]) * s.Nx[0];
  }
}

// write_lammps_traj (config_utils.cu:366-403)
void write_traj(const Script& s, int step, const float* x) {
  FILE* otp = fopen(s.dump_name.c_str(), step == 0 ? "w" : "a");
  if (!otp) throw std::runtime_error("cannot open " + s.dump_name);
  fprintf(otp, "ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\n", step, s.sys.ns);
  fprintf(otp, "ITEM: BOX BOUNDS pp pp pp\n");
  fprintf(otp, "%f %f\n%f %f\n%f %f\n", 0.f, s.sys.L[0], 0.f, s.sys.L[1], (s.Dim == 3 ? 0.f : 1.f),
          (s.Dim == 3 ? s.sys.L[2] : 1.f));
  fprintf(otp, s.do_charges ? "ITEM: ATOMS id type mol x y z q\n" : "ITEM: ATOMS id type mol x y z\n");
  for (int i = 0; i < s.sys.ns; i++) {
    fprintf(otp, "%d %d %d  ", i + 1, s.sys.tp[i] + 1, s.sys.molecID[i] + 1);
    for (int j = 0; j < s.Dim; j++) fprintf(otp, "%f ", x[(size_t)i * s.Dim + j]);
    for (int j = s.Dim; j < 3; j++) fprintf(otp, "%f", 0.f);
    if (s.do_charges) fprintf(otp, " %f", s.sys.charges[i]);
    fprintf(otp, "\n");
  }
  fclose(otp);
}

// write_grid_data (io_utils.cu:7-32)
void write_grid(const Script& s, int M, const char* name, const float* dat) {
  FILE* otp = fopen(name, "w");
  if (!otp) throw std::runtime_error(std::string("cannot open ") + name);
  const float dx[3] = {s.sys.L[0] / (float)s.Nx[0], s.sys.L[1] / (float)s.Nx[1],
                       s.Dim == 3 ? s.sys.L[2] / (float)s.Nx[2] : 1.f};
  for (int i = 0; i < M; i++) {
    int nn[3] = {0, 0, 0};
    unstack(s, i, nn);
    for (int j = 0; j < s.Dim; j++) fprintf(otp, "%f ", dx[j] * float(nn[j]));
    fprintf(otp, "%1.8e \n", dat[i]);
    if (s.Dim == 2 && nn[0] == s.Nx[0] - 1) fprintf(otp, "\n");
  }
  fclose(otp);
}

// write_kspace_data (io_utils.cu:60-83) for the averaged S(k)
void write_kspace(Run& r, const char* name, const std::vector<double>& sk) {
  const Script& s = r.s;
  FILE* otp = fopen(name, "w");
  if (!otp) throw std::runtime_error(std::string("cannot open ") + name);
  for (int i = 1; i < r.M; i++) {
    int nn[3] = {0, 0, 0};
    unstack(s, i, nn);
    float kv[3], k2 = 0.f;
    for (int d = 0; d < s.Dim; d++) {
      if (float(nn[d]) < float(s.Nx[d]) / 2.) kv[d] = kPI2 * float(nn[d]) / s.sys.L[d];
      else kv[d] = kPI2 * float(nn[d] - s.Nx[d]) / s.sys.L[d];
      k2 += kv[d] * kv[d];
    }
    for (int d = 0; d < s.Dim; d++) fprintf(otp, "%f ", kv[d]);
    const float re = (float)sk[2 * (size_t)i], im = (float)sk[2 * (size_t)i + 1];
    fprintf(otp, "%1.5e %1.5e %1.5e %1.5e\n", std::sqrt(re * re + im * im), std::sqrt(k2), re, im);
    if (s.Dim == 2 && nn[0] == s.Nx[0] - 1) fprintf(otp, "\n");
  }
  fclose(otp);
}

// init_binary_output / write_binary (io_utils.cu:85-134)
void init_binary(Run& r) {
  const Script& s = r.s;
  FILE* otp = fopen("grid_densities.bin", "wb");
  if (!otp) throw std::runtime_error("failed to open grid_densities.bin");
  fwrite(&s.Dim, sizeof(int), 1, otp);
  fwrite(s.Nx, sizeof(int), s.Dim, otp);
  fwrite(s.sys.L, sizeof(float), s.Dim, otp);
  fwrite(&s.sys.ntypes, sizeof(int), 1, otp);
  fclose(otp);
  otp = fopen("positions.bin", "wb");
  if (!otp) throw std::runtime_error("Failed to open positions.bin");
  fwrite(&s.sys.ns, sizeof(int), 1, otp);
  fwrite(&s.Dim, sizeof(int), 1, otp);
  fwrite(s.sys.L, sizeof(float), 3, otp);
  fwrite(s.sys.tp.data(), sizeof(int), s.sys.ns, otp);
  fwrite(s.sys.molecID.data(), sizeof(int), s.sys.ns, otp);
  const int dc = s.do_charges ? 1 : 0;
  fwrite(&dc, sizeof(int), 1, otp);
  if (dc) fwrite(s.sys.charges.data(), sizeof(float), s.sys.ns, otp);
  fclose(otp);
}

void write_binary(const Script& s, int M, const float* rho, const float* x) {
  FILE* otp = fopen("grid_densities.bin", "ab");
  if (!otp) throw std::runtime_error("Failed to append to grid_densities.bin");
  fwrite(rho, sizeof(float), (size_t)M * s.sys.ntypes, otp);
  fclose(otp);
  otp = fopen("positions.bin", "ab");
  if (!otp) throw std::runtime_error("Failed to append to positions.bin");
  fwrite(x, sizeof(float), (size_t)s.sys.ns * s.Dim, otp);
  fclose(otp);
}

void write_rho_files(const Script& s, int M, const float* rho) {
  for (int i = 0; i < s.sys.ntypes; i++) {
    char nm[30];
    snprintf(nm, sizeof nm, "rho%d.dat", i);
    write_grid(s, M, nm, rho + (size_t)i * M);
  }
}

// Output frames: the state is snapshotted into one of TILD_SNAPSHOT_SLOTS page-locked buffers in
// stream order, and a writer thread waits for each copy, then formats and writes the frame's files
// in submission order while the caller keeps stepping.
class Writer {
 public:
  explicit Writer(Run& r) : r_(r) {
    const size_t nx = (size_t)r.s.sys.ns * r.s.Dim;
    const size_t nr = (size_t)r.M * (r.s.sys.ntypes + (r.s.do_charges ? 1 : 0));
    for (int k = 0; k < TILD_SNAPSHOT_SLOTS; k++) {
      x_[k] = static_cast<float*>(tild_host_alloc(nx * sizeof(float)));
      rho_[k] = static_cast<float*>(tild_host_alloc(nr * sizeof(float)));
      if (!x_[k] || !rho_[k]) {  // page-locked memory unavailable: pageable buffers still work
        tild_host_free(x_[k]);
        tild_host_free(rho_[k]);
        x_[k] = rho_[k] = nullptr;
        fx_[k].assign(nx, 0.f);
        fr_[k].assign(nr, 0.f);
      }
    }
    th_ = std::thread([this] { loop(); });
  }
  ~Writer() {
    stop();
    for (int k = 0; k < TILD_SNAPSHOT_SLOTS; k++) {
      tild_host_free(x_[k]);
      tild_host_free(rho_[k]);
    }
  }
  // queues the files of one frame: trajectory (x), rho%d.dat (rho), binary frames (x and rho)
  void frame(int step, bool traj, bool grid, bool bin) {
    if (!traj && !grid && !bin) return;
    const int k = (int)(issued_ % TILD_SNAPSHOT_SLOTS);
    {
      std::unique_lock<std::mutex> lk(m_);
      cv_.wait(lk, [&] { return done_ + TILD_SNAPSHOT_SLOTS > issued_ || !err_.empty(); });
      if (!err_.empty()) throw std::runtime_error(err_);
    }
    float* xb = x_[k] ? x_[k] : fx_[k].data();
    float* rb = rho_[k] ? rho_[k] : fr_[k].data();
    const bool want_x = traj || bin, want_rho = grid || bin;
    int64_t ticket = -1;
    check(r_, tild_snapshot_async(r_.ctx, want_x ? xb : nullptr, want_rho ? rb : nullptr, &ticket),
          "tild_snapshot_async");
    {
      std::lock_guard<std::mutex> lk(m_);
      q_.push_back({step, traj, grid, bin, ticket, xb, rb});
      issued_++;
    }
    cv_.notify_all();
  }
  // waits until every queued frame is on disk
  void finish() {
    std::unique_lock<std::mutex> lk(m_);
    cv_.wait(lk, [&] { return done_ == issued_ || !err_.empty(); });
    if (!err_.empty()) throw std::runtime_error(err_);
  }

 private:
  struct Task {
    int step;
    bool traj, grid, bin;
    int64_t ticket;
    const float *x, *rho;
  };
  void loop() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return !q_.empty() || quit_; });
        if (q_.empty()) return;
        t = q_.front();
        q_.pop_front();
      }
      try {
        if (tild_snapshot_wait(r_.ctx, t.ticket) != TILD_OK) throw std::runtime_error("tild_snapshot_wait failed");
        if (t.traj) write_traj(r_.s, t.step, t.x);
        if (t.grid) write_rho_files(r_.s, r_.M, t.rho);
        if (t.bin) write_binary(r_.s, r_.M, t.rho, t.x);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(m_);
        err_ = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(m_);
        done_++;
      }
      cv_.notify_all();
    }
  }
  void stop() {
    {
      std::lock_guard<std::mutex> lk(m_);
      quit_ = true;
    }
    cv_.notify_all();
    if (th_.joinable()) th_.join();
  }

  Run& r_;
  float* x_[TILD_SNAPSHOT_SLOTS] = {nullptr};
  float* rho_[TILD_SNAPSHOT_SLOTS] = {nullptr};
  std::vector<float> fx_[TILD_SNAPSHOT_SLOTS], fr_[TILD_SNAPSHOT_SLOTS];
  std::thread th_;
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<Task> q_;
  long long issued_ = 0, done_ = 0;
  bool quit_ = false;
  std::string err_;
};

// print_timestep (main.cu:422-485); values are FP64 here, printed as the reference's floats
int print_timestep(Run& r) {
  const Script& s = r.s;
  const tild_obs& o = r.obs;
  int die_flag = 0;
  std::cout << "Step " << r.step << " of " << s.max_steps << " ";
  if (s.do_charges) std::cout << " Electrostatic Energy: " << (float)o.uelec;
  std::cout << " U/V: " << (float)o.upe / r.V << " Ubond: " << (float)o.ubond << " Pdiags: " << (float)o.ptens[0]
            << " " << (float)o.ptens[1] << " ";
  if (s.Dim == 3) std::cout << (float)o.ptens[2] << " ";
  r.dout << r.step << " " << (float)o.upe << " " << (float)o.ubond << " ";
  for (int i = 0; i < o.n_p_comps; i++) r.dout << (float)o.ptens[i] << " ";
  int idx = 0;
  auto block = [&](const std::vector<tildhost::StyleLine>& v, const char* label, bool computed) {
    if (v.empty()) return;
    std::cout << label;
    for (size_t k = 0; k < v.size(); k++, idx++) {
      const float e = computed ? (float)o.style_energy[idx] : 0.f;  // fieldphase energy is never computed
      std::cout << e << " ";
      r.dout << e << " ";
      if (std::isnan(e)) die_flag = 1;
    }
  };
  // styles sit in the config as gaussians, erfs, fieldphases, gaussian_erfs; print in the
  // reference's order gaussians, erfs, gaussian_erfs, fieldphases
  const size_t ng = s.gaussians.size(), ne = s.erfs.size(), nf = s.fieldphases.size();
  idx = 0;
  block(s.gaussians, "Ugauss: ", true);
  block(s.erfs, "Uerf: ", true);
  idx = (int)(ng + ne + nf);
  block(s.gauss_erfs, "UGaussErf: ", true);
  idx = (int)(ng + ne);
  block(s.fieldphases, "UFieldPhase: ", false);
  r.dout << std::endl;
  std::cout << std::endl;
  return die_flag;
}

void observables(Run& r) {
  const int st = tild_observables(r.ctx, &r.obs);
  if (st == TILD_ERR_NAN) {
    for (double& e : r.obs.style_energy) e = NAN;
    return;
  }
  check(r, st, "tild_observables");
}

}  // namespace

int main(int argc, char** argv) {
  const auto t_main = std::chrono::steady_clock::now();
  std::string input = "input";
  bool dry = false;
  int device = 0;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-in" && i + 1 < argc) input = argv[++i];
    else if (a == "--dry-run") dry = true;
    else if (a == "--device" && i + 1 < argc) device = std::stoi(argv[++i]);
  }
  Run r;
  try {
    r.s = tildhost::parse_script(input, (int)time(0));
  } catch (const std::exception& e) {
    std::cout << e.what() << std::endl;
    return 1;
  }
  std::cout << "Input file read!" << std::endl;
  Script& s = r.s;
  {
    std::ofstream otp("NEED_A_NAME.input");
    otp << tildhost::runtime_parameters(s);
  }
  if (s.sys.n_total_angles > 0) {
    std::cout << "Angles not yet set up on device!" << std::endl;
    return 1;
  }
  r.M = 1;
  r.V = 1.f;
  for (int d = 0; d < s.Dim; d++) {
    r.M *= s.Nx[d];
    r.V *= s.sys.L[d];
  }
  if (dry) {
    std::cout << "dry run: ns " << s.sys.ns << " M " << r.M << " styles "
              << s.gaussians.size() + s.erfs.size() + s.gauss_erfs.size() + s.fieldphases.size() << std::endl;
    return 0;
  }
  try {
    tild_config cfg = tildhost::make_config(s);
    int st = tild_create(&cfg, device, &r.ctx);
    if (st != TILD_OK) {
      std::cout << "tild_create failed: " << tild_status_string(st) << std::endl;
      return 1;
    }
    check(r, tild_set_topology(r.ctx, s.sys.tp.data(), s.do_charges ? s.sys.charges.data() : nullptr,
                               s.sys.n_bonds.data(), s.sys.bonded_to.data(), s.sys.bond_type.data()),
          "tild_set_topology");
    check(r, tild_set_state(r.ctx, s.sys.x.data(), nullptr, nullptr), "tild_set_state");
    if (s.bin_freq != 0) init_binary(r);
    Writer writer(r);
    const auto t_init = std::chrono::steady_clock::now();

    r.step = 0;
    writer.frame(0, true, false, false);
    r.dout.open("data.dat");
    r.dout << "# step Upe Ubond ";
    if (s.Dim == 2) r.dout << "Pxx Pyy Pxy ";
    else r.dout << " Pxx Pyy Pzz Pxy Pxz Pyz ";
    for (size_t i = 0; i < s.gaussians.size(); i++) r.dout << "Ugauss[" << i << "] ";
    for (size_t i = 0; i < s.erfs.size(); i++) r.dout << "Uerf[" << i << "] ";
    for (size_t i = 0; i < s.gauss_erfs.size(); i++) r.dout << "UGuassErf[" << i << "] ";
    r.dout << std::endl;

    check(r, tild_forces(r.ctx, nullptr), "tild_forces");
    observables(r);
    writer.frame(0, false, s.grid_freq > 0, false);
    int die_flag = print_timestep(r);
    double io_s = 0.0;

    auto is_event = [&](int st) {
      if (st >= s.max_steps) return true;
      if (s.traj_freq > 0 && st % s.traj_freq == 0) return true;
      if (s.grid_freq > 0 && st % s.grid_freq == 0) return true;
      if (s.bin_freq > 0 && st % s.bin_freq == 0) return true;
      if (s.log_freq > 0 && st % s.log_freq == 0) return true;
      for (const auto& c : s.computes)
        if (st > c.wait && c.freq > 0 && st % c.freq == 0) return true;
      return false;
    };
    r.step = 0;
    while (!die_flag && r.step < s.max_steps) {
      int n = 1;
      while (r.step + n < s.max_steps && !is_event(r.step + n)) n++;
      check(r, tild_step(r.ctx, n), "tild_step");
      r.step += n;
      const auto t0 = std::chrono::steady_clock::now();
      for (size_t i = 0; i < s.computes.size(); i++) {
        const auto& c = s.computes[i];
        if (r.step > c.wait && c.freq > 0 && r.step % c.freq == 0)
          check(r, tild_sk_accumulate(r.ctx, (int)i, c.type), "tild_sk_accumulate");
      }
      writer.frame(r.step, s.traj_freq > 0 && r.step % s.traj_freq == 0, s.grid_freq > 0 && r.step % s.grid_freq == 0,
                   s.bin_freq > 0 && r.step % s.bin_freq == 0);
      if (s.log_freq > 0 && r.step % s.log_freq == 0) {
        observables(r);
        die_flag = print_timestep(r);
        for (size_t i = 0; i < s.computes.size(); i++) {
          if (r.step <= s.computes[i].wait) continue;
          std::vector<double> sk(2 * (size_t)r.M);
          int ncalls = 0;
          check(r, tild_sk_get(r.ctx, (int)i, sk.data(), &ncalls), "tild_sk_get");
          char nm[50];
          snprintf(nm, sizeof nm, "avg_sk_%d.dat", (int)i);
          write_kspace(r, nm, sk);
        }
      }
      io_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    // the reference's loop variable ends at max_steps + 1 unless a NaN energy broke the loop
    if (!die_flag) r.step = s.max_steps + 1;
    writer.frame(r.step, true, false, false);
    writer.finish();
    const auto t_end = std::chrono::steady_clock::now();
    const int dt = (int)std::chrono::duration<double>(t_end - t_main).count();
    std::cout << "Total run time: " << dt / 60 << "m" << dt % 60 << "sec" << std::endl;
    const int di = (int)std::chrono::duration<double>(t_init - t_main).count();
    std::cout << "Total init time: " << di / 60 << "m" << di % 60 << "sec" << std::endl;
    std::cout << "I/O + Comm time: " << (int)io_s / 60 << "m" << (int)io_s % 60 << "sec" << std::endl;
    tild_destroy(r.ctx);
  } catch (const std::exception& e) {
    std::cout << e.what() << std::endl;
    if (r.ctx) tild_destroy(r.ctx);
    return 1;
  }
  return 0;
}
