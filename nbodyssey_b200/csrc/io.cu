// Files and the run loop (src/main.cu:115-215, docs/FORMATS.md).
//
// nb_run keeps the device busy across frame dumps: at a dump step the
// positions are copied device-to-device into a staging slot on the compute
// stream (16 bytes per particle), a side stream moves the slot into pinned
// host memory, and a writer thread waits for that copy and writes the frame
// file while the next steps run.  Energy rows are computed on the compute
// stream into a device slot and copied back the same way, so the loop has no
// host synchronisation until the slots run out.
#include <sys/stat.h>

#include <cerrno>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "nb_internal.cuh"

using namespace nb;

static int mkdirs(const std::string& path) {
  if (path.empty()) return NB_OK;
  std::string cur;
  for (size_t i = 0; i <= path.size(); ++i) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty() && cur != "/") {
        if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
          return set_error(NB_ERR_IO, "cannot create directory " + cur);
      }
    }
    if (i < path.size()) cur += path[i];
  }
  return NB_OK;
}

static std::string parent_dir(const std::string& p) {
  size_t k = p.find_last_of('/');
  if (k == std::string::npos) return "";
  return p.substr(0, k);
}

extern "C" {

int nb_read_ic(const char* path, int* n, float* pos4, float* vel4) {
  if (!path || !n) return set_error(NB_ERR_INVALID, "NULL argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(NB_ERR_IO, std::string("cannot open IC file: ") + path);
  int32_t cnt = 0;
  if (std::fread(&cnt, 4, 1, f) != 1 || cnt <= 0) {
    std::fclose(f);
    return set_error(NB_ERR_IO, std::string("bad particle count in ") + path);
  }
  if (!pos4 && !vel4) {
    std::fclose(f);
    *n = cnt;
    return NB_OK;
  }
  if (*n < cnt) {
    std::fclose(f);
    return set_error(NB_ERR_INVALID, "buffers too small for the IC file");
  }
  size_t want = (size_t)cnt * 4;
  bool ok = pos4 && vel4 && std::fread(pos4, sizeof(float), want, f) == want &&
            std::fread(vel4, sizeof(float), want, f) == want;
  std::fclose(f);
  if (!ok) return set_error(NB_ERR_IO, std::string("truncated IC file: ") + path);
  *n = cnt;
  return NB_OK;
}

int nb_write_ic(const char* path, int n, const float* pos4, const float* vel4) {
  if (!path || !pos4 || !vel4 || n <= 0) return set_error(NB_ERR_INVALID, "bad argument");
  NB_TRY(mkdirs(parent_dir(path)));
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(NB_ERR_IO, std::string("cannot open ") + path);
  int32_t cnt = n;
  bool ok = std::fwrite(&cnt, 4, 1, f) == 1 &&
            std::fwrite(pos4, 16, (size_t)n, f) == (size_t)n &&
            std::fwrite(vel4, 16, (size_t)n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_error(NB_ERR_IO, std::string("write failed: ") + path);
  return NB_OK;
}

// State file: the ic.bin layout (int32 n, float4 pos[n], float4 vel[n],
// docs/FORMATS.md:8-16), so any ic.bin reader takes it as initial
// conditions, followed by a trailer that makes a resumed run continue bit for
// bit: the 8-byte magic "NBSTATE1", int32 flags (NB_STATE_*), the run's
// nb_params, float4 pos_lo[n] (low-order position parts) and float4 acc[n]
// (a(x) of the stored positions).
static const char kStateMagic[8] = {'N', 'B', 'S', 'T', 'A', 'T', 'E', '1'};

int nb_write_state_file(const char* path, int n, const float* pos4, const float* vel4,
                        const float* lo4, const float* acc4, const nb_params* p) {
  if (!path || !pos4 || !vel4 || !p || n <= 0) return set_error(NB_ERR_INVALID, "bad argument");
  NB_TRY(mkdirs(parent_dir(path)));
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(NB_ERR_IO, std::string("cannot open ") + path);
  int32_t cnt = n;
  int32_t flags = NB_STATE_TRAILER | (acc4 ? NB_STATE_ACC : 0) | (lo4 ? NB_STATE_LO : 0);
  std::vector<float> zero(acc4 && lo4 ? 0 : (size_t)n * 4, 0.f);
  bool ok = std::fwrite(&cnt, 4, 1, f) == 1 &&
            std::fwrite(pos4, 16, (size_t)n, f) == (size_t)n &&
            std::fwrite(vel4, 16, (size_t)n, f) == (size_t)n &&
            std::fwrite(kStateMagic, 1, 8, f) == 8 && std::fwrite(&flags, 4, 1, f) == 1 &&
            std::fwrite(p, sizeof(nb_params), 1, f) == 1 &&
            std::fwrite(lo4 ? lo4 : zero.data(), 16, (size_t)n, f) == (size_t)n &&
            std::fwrite(acc4 ? acc4 : zero.data(), 16, (size_t)n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_error(NB_ERR_IO, std::string("write failed: ") + path);
  return NB_OK;
}

int nb_read_state_file(const char* path, int* n, float* pos4, float* vel4, float* lo4,
                       float* acc4, nb_params* p, int* flags) {
  if (!path || !n) return set_error(NB_ERR_INVALID, "NULL argument");
  if (!pos4 && !vel4) return nb_read_ic(path, n, nullptr, nullptr);
  int cnt = *n;
  NB_TRY(nb_read_ic(path, &cnt, pos4, vel4));
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(NB_ERR_IO, std::string("cannot open ") + path);
  const long off = 4 + 32L * cnt;
  char magic[8] = {};
  int32_t fl = 0;
  nb_params q{};
  bool trailer = std::fseek(f, off, SEEK_SET) == 0 && std::fread(magic, 1, 8, f) == 8 &&
                 std::memcmp(magic, kStateMagic, 8) == 0;
  bool ok = true;
  if (trailer) {
    const size_t want = (size_t)cnt * 4;
    std::vector<float> tmp(want);
    ok = std::fread(&fl, 4, 1, f) == 1 && std::fread(&q, sizeof(nb_params), 1, f) == 1 &&
         std::fread(lo4 ? lo4 : tmp.data(), sizeof(float), want, f) == want &&
         std::fread(acc4 ? acc4 : tmp.data(), sizeof(float), want, f) == want;
  }
  std::fclose(f);
  if (!ok) return set_error(NB_ERR_IO, std::string("truncated state trailer: ") + path);
  if (!trailer) {   // a plain ic.bin: no low-order parts, no a(x)
    fl = 0;
    if (lo4) std::memset(lo4, 0, sizeof(float) * 4 * (size_t)cnt);
    if (acc4) std::memset(acc4, 0, sizeof(float) * 4 * (size_t)cnt);
  } else if (p) {
    *p = q;
  }
  if (flags) *flags = fl;
  *n = cnt;
  return NB_OK;
}

int nb_write_frame(const char* dir, int index, int n, const float* pos4) {
  if (!dir || !pos4 || n <= 0 || index < 0) return set_error(NB_ERR_INVALID, "bad argument");
  char name[64];
  std::snprintf(name, sizeof(name), "frame_%05d.bin", index);
  std::string path = std::string(dir) + "/" + name;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return set_error(NB_ERR_IO, "cannot open " + path);
  int32_t cnt = n;
  bool ok = std::fwrite(&cnt, 4, 1, f) == 1 &&
            std::fwrite(pos4, 16, (size_t)n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_error(NB_ERR_IO, "write failed: " + path);
  return NB_OK;
}

int nb_format_energy_row(char* buf, size_t cap, int step, float dt, double e,
                         double ke, double pe, double e0) {
  if (!buf || cap == 0) return set_error(NB_ERR_INVALID, "bad buffer");
  double rel = (e - e0) / std::fabs(e0);
  float t = step * dt;   // int * float, as src/main.cu:175
  int w = std::snprintf(buf, cap, "%d,%.5f,%.8e,%.8e,%.8e,%.3e\n", step, t, e,
                        ke, pe, rel);
  if (w < 0 || (size_t)w >= cap) return set_error(NB_ERR_INVALID, "buffer too small");
  return NB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Run loop
// ---------------------------------------------------------------------------
namespace {

struct Job {
  int slot;
  int frame;        // -1: no frame
  int step;         // energy row label, -1: none
  cudaEvent_t ready;
};

struct Writer {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job> q;
  std::vector<bool> busy;
  bool stop = false;
  int err = NB_OK;
  std::string msg;
};

}  // namespace

extern "C" int nb_run(nb_sim* s, int steps, int dump_every, const char* out_dir,
                      const char* energy_csv, int timing, nb_run_stats* stats) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  if (steps < 0 || dump_every <= 0)
    return set_error(NB_ERR_INVALID, "steps must be >= 0 and dump_every > 0");
  SimView v;
  NB_TRY(sim_view(s, &v));
  const int n = v.n;
  std::string dir = out_dir ? out_dir : "";
  std::string csv = energy_csv ? energy_csv : "";
  if (!dir.empty()) NB_TRY(mkdirs(dir));
  FILE* elog = nullptr;
  if (!csv.empty()) {
    NB_TRY(mkdirs(parent_dir(csv)));
    elog = std::fopen(csv.c_str(), "w");
    if (!elog) return set_error(NB_ERR_IO, "cannot open " + csv);
    std::fputs("step,time,energy,kinetic,potential,rel_error\n", elog);
  }
  NB_TRY(nb_set_timing(s, timing));
  NB_TRY(nb_reset_timing(s));

  const int kSlots = 3;
  float4* d_stage = nullptr;
  float* h_stage = nullptr;
  double* h_energy = nullptr;
  double* d_energy = nullptr;
  cudaStream_t side = nullptr;
  std::vector<cudaEvent_t> staged(kSlots), copied(kSlots);
  int rc = NB_OK;
  auto cleanup = [&]() {
    if (side) cudaStreamSynchronize(side);
    cudaStreamSynchronize(v.stream);
    for (auto& e : staged) if (e) cudaEventDestroy(e);
    for (auto& e : copied) if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
    cudaFree(d_stage);
    cudaFree(d_energy);
    if (h_stage) cudaFreeHost(h_stage);
    if (h_energy) cudaFreeHost(h_energy);
    if (elog) std::fclose(elog);
  };
#define RUN_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      rc = set_error(NB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
      goto done;                                                                \
    }                                                                           \
  } while (0)
  {
    double e3[3];
    double e0 = 0.0;
    auto t0 = std::chrono::steady_clock::now();
    int frame = 0;
    Writer wr;
    std::thread th;
    wr.busy.assign(kSlots, false);
    RUN_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    RUN_CUDA(cudaMalloc(&d_stage, sizeof(float4) * (size_t)n * kSlots));
    RUN_CUDA(cudaMalloc(&d_energy, sizeof(double) * 8 * kSlots));
    RUN_CUDA(cudaMallocHost(&h_stage, sizeof(float4) * (size_t)n * kSlots));
    RUN_CUDA(cudaMallocHost(&h_energy, sizeof(double) * 8 * kSlots));
    for (int i = 0; i < kSlots; ++i) {
      RUN_CUDA(cudaEventCreateWithFlags(&staged[i], cudaEventDisableTiming));
      RUN_CUDA(cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming));
    }
    if ((rc = nb_energy(s, e3, nullptr)) != NB_OK) goto done;
    e0 = e3[0];
    if ((rc = nb_compute_forces(s, nullptr)) != NB_OK) goto done;   // a(x0)

    th = std::thread([&]() {
      for (;;) {
        Job j;
        {
          std::unique_lock<std::mutex> lk(wr.mu);
          wr.cv.wait(lk, [&] { return wr.stop || !wr.q.empty(); });
          if (wr.q.empty()) return;
          j = wr.q.front();
          wr.q.pop_front();
        }
        cudaEventSynchronize(j.ready);
        int r = NB_OK;
        std::string m;
        if (j.frame >= 0) {
          r = nb_write_frame(dir.c_str(), j.frame, n, h_stage + (size_t)j.slot * n * 4);
          if (r != NB_OK) m = last_error();
        }
        if (r == NB_OK && j.step >= 0 && elog) {
          char line[256];
          const double* e = h_energy + 8 * j.slot;
          nb_format_energy_row(line, sizeof(line), j.step, v.p.dt, e[0], e[1], e[2], e0);
          if (std::fputs(line, elog) < 0) { r = NB_ERR_IO; m = "energy log write failed"; }
        }
        std::lock_guard<std::mutex> lk(wr.mu);
        wr.busy[j.slot] = false;
        if (r != NB_OK && wr.err == NB_OK) { wr.err = r; wr.msg = m; }
        wr.cv.notify_all();
      }
    });

    {
      int slot = 0;
      auto emit = [&](int step, bool with_frame) -> int {
        {
          std::unique_lock<std::mutex> lk(wr.mu);
          wr.cv.wait(lk, [&] { return !wr.busy[slot]; });
          wr.busy[slot] = true;
        }
        cudaStream_t st = v.stream;
        float4* ds = d_stage + (size_t)slot * n;
        if (with_frame && !dir.empty())
          NB_CUDA(cudaMemcpyAsync(ds, v.pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
        NB_TRY(launch_energy(*v.ws, n, v.pos, v.vel, v.p.eps * v.p.eps, v.p.G, st));
        NB_CUDA(cudaMemcpyAsync(d_energy + 8 * slot, v.ws->eout, 6 * sizeof(double),
                                cudaMemcpyDeviceToDevice, st));
        NB_CUDA(cudaEventRecord(staged[slot], st));
        NB_CUDA(cudaStreamWaitEvent(side, staged[slot], 0));
        if (with_frame && !dir.empty())
          NB_CUDA(cudaMemcpyAsync(h_stage + (size_t)slot * n * 4, ds, sizeof(float4) * n,
                                  cudaMemcpyDeviceToHost, side));
        NB_CUDA(cudaMemcpyAsync(h_energy + 8 * slot, d_energy + 8 * slot, 6 * sizeof(double),
                                cudaMemcpyDeviceToHost, side));
        NB_CUDA(cudaEventRecord(copied[slot], side));
        {
          std::lock_guard<std::mutex> lk(wr.mu);
          wr.q.push_back(Job{slot, (with_frame && !dir.empty()) ? frame : -1, step, copied[slot]});
          wr.cv.notify_all();
        }
        if (with_frame) ++frame;
        slot = (slot + 1) % kSlots;
        return NB_OK;
      };
      for (int step = 0; step < steps && rc == NB_OK; ++step) {
        rc = nb_step(s, 1);
        if (rc == NB_OK && step % dump_every == 0) rc = emit(step, true);
      }
      if (rc == NB_OK) rc = emit(steps, false);
    }
    {
      std::lock_guard<std::mutex> lk(wr.mu);
      wr.stop = true;
      wr.cv.notify_all();
    }
    th.join();
    if (rc == NB_OK && wr.err != NB_OK) rc = set_error(wr.err, wr.msg);
    if (rc == NB_OK) rc = nb_sync(s);
    if (rc == NB_OK && stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      nb_force_timing(s, &stats->force_ms, &stats->force_calls);
      long calls = 0;
      double ph[NB_PHASES];
      nb_phase_times(s, ph, &calls);
      for (int i = 0; i < NB_PHASES; ++i) stats->phase_ms[i] = calls ? ph[i] / calls : 0.0;
      stats->frames = frame;
      stats->e0 = e0;
      double ef[3];
      if (nb_energy(s, ef, nullptr) == NB_OK) {
        stats->e_final = ef[0];
        stats->rel_final = (ef[0] - e0) / std::fabs(e0);
      }
    }
  }
done:
#undef RUN_CUDA
  cleanup();
  nb_set_timing(s, 0);
  return rc;
}
