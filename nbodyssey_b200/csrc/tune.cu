// Autotuner: per device, the all-pairs launch shape per size, the Barnes-Hut
// walk's warps per block and the all-pairs / Barnes-Hut crossover that
// NB_FORCE_AUTO uses, measured on the device itself.
//
// The reference has one fixed shape (kForceBlock = 256, src/forces.cuh:25)
// and a force module the user picks by hand (src/forces.cu:68-86).  Here the
// table is measured at first use on each device (the first simulation,
// ensemble or server created on it) and kept in a cache file named after the
// device, so later processes on the same kind of GPU load it instead of
// measuring again.  Measuring takes about a second: synthetic two-disk inputs
// (the benchmarks' recipe, host-generated), every candidate timed with CUDA
// events on a private stream, best of three after a warm-up.
//
// The shape decides only the launch: the per-target summation order of the
// all-pairs kernel depends on the source chunking alone, so two runs with the
// same table give the same bits, whether the table was measured, loaded or
// set by hand (nb_tune_set).
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nb_internal.cuh"

namespace nb {

namespace {

constexpr int kMaxDev = 64;
std::mutex g_mu;
nb_tune_table g_tab[kMaxDev];
int g_state[kMaxDev] = {};   // 0 untouched, 1 defaults or set, 2 measured / loaded
// set while this thread measures: batches created for the measurement use the
// table being measured and must not start another measurement
thread_local bool g_measuring = false;

const float kThetaClass[NB_TUNE_THETAS] = {0.3f, 0.5f, 0.7f};

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
    cudaGetLastError();
    return 0;
  }
  return dev;
}

void defaults(nb_tune_table* t) {
  std::memset(t, 0, sizeof(*t));
  t->version = NB_TUNE_VERSION;
  t->sms = device_sm_count();
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, current_device()) == cudaSuccess)
    std::snprintf(t->device, sizeof(t->device), "%s", prop.name);
  else
    cudaGetLastError();
  for (int b = 0; b < NB_TUNE_BUCKETS; ++b) {
    t->ap_threads[b] = 256;
    t->ap_k[b] = 4;
    t->ap_ctas[b] = 8 * t->sms;
  }
  t->walk_warps = 4;
  for (int i = 0; i < NB_TUNE_THETAS; ++i) {
    for (int j = 0; j < 2; ++j) t->crossover[i][j] = NB_AUTO_CROSSOVER;
    t->crossover_batch[i] = 4096;
  }
}

bool table_ok(const nb_tune_table& t) {
  if (t.version != NB_TUNE_VERSION) return false;
  for (int b = 0; b < NB_TUNE_BUCKETS; ++b)
    if (!allpairs_shape_compiled(t.ap_threads[b], t.ap_k[b]) || t.ap_ctas[b] < 1)
      return false;
  if (t.walk_warps != 2 && t.walk_warps != 4 && t.walk_warps != 8) return false;
  for (int i = 0; i < NB_TUNE_THETAS; ++i) {
    for (int j = 0; j < 2; ++j)
      if (t.crossover[i][j] < 0) return false;
    if (t.crossover_batch[i] < 0) return false;
  }
  return true;
}

// The table of the current device (defaults until measured, loaded or set).
nb_tune_table& table_locked() {
  const int dev = current_device();
  if (g_state[dev] == 0) {
    defaults(&g_tab[dev]);
    g_state[dev] = 1;
  }
  return g_tab[dev];
}

std::string cache_path() {
  const char* e = std::getenv("NBODY_B200_TUNE_CACHE");
  if (e && *e) return e;
  nb_tune_table t;
  defaults(&t);
  std::string name;
  for (const char* c = t.device; *c; ++c)
    name += std::isalnum((unsigned char)*c) ? *c : '_';
  const char* home = std::getenv("HOME");
  std::string dir = std::string(home && *home ? home : "/tmp") + "/.cache/nbodyssey_b200";
  return dir + "/tune_" + name + "_" + std::to_string(t.sms) + "sm_v" +
         std::to_string(NB_TUNE_VERSION) + ".bin";
}

int mkdirs_for(const std::string& path) {
  std::string cur;
  for (size_t i = 0; i < path.size(); ++i) {
    if (path[i] == '/' && !cur.empty()) {
      if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
        return set_error(NB_ERR_IO, "cannot create directory " + cur);
    }
    cur += path[i];
  }
  return NB_OK;
}

// ---- measurement ---------------------------------------------------------

// Two exponential disks (scale 1, cut at 5, sigma_z 0.1) centred at
// (-10, -2, 0) and (10, 2, 0), equal masses: the benchmarks' layout.
void two_disks(int n, std::vector<float4>& pos) {
  pos.resize(n);
  uint64_t s = 0x9e3779b97f4a7c15ull ^ (uint64_t)n;
  auto uni = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return ((s >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  const int na = n / 2;
  for (int i = 0; i < n; ++i) {
    const bool b = i >= na;
    double r;
    do r = -std::log(uni() * uni()); while (r > 5.0);
    const double ph = 2.0 * M_PI * uni();
    const double z = 0.1 * std::sqrt(-2.0 * std::log(uni())) * std::cos(2.0 * M_PI * uni());
    const double m = 1.0 / (b ? n - na : na);
    pos[i] = make_float4((float)(r * std::cos(ph) + (b ? 10.0 : -10.0)),
                         (float)(r * std::sin(ph) + (b ? 2.0 : -2.0)), (float)z, (float)m);
  }
}

struct Bench {
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  Workspace w;
  float4* pos = nullptr;
  float4* acc = nullptr;
  int cap = 0;
  ~Bench() {
    if (st) cudaStreamSynchronize(st);
    ws_free(w);
    cudaFree(pos);
    cudaFree(acc);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
  }
  int init() {
    NB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    NB_CUDA(cudaEventCreate(&e0));
    NB_CUDA(cudaEventCreate(&e1));
    return NB_OK;
  }
  int load(int n) {
    if (n > cap) {
      cudaFree(pos);
      cudaFree(acc);
      pos = acc = nullptr;
      NB_CUDA(cudaMalloc(&pos, sizeof(float4) * n));
      NB_CUDA(cudaMalloc(&acc, sizeof(float4) * n));
      cap = n;
    }
    std::vector<float4> h;
    two_disks(n, h);
    NB_CUDA(cudaMemcpyAsync(pos, h.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st));
    NB_CUDA(cudaStreamSynchronize(st));
    return NB_OK;
  }
  StepArgs args(int n, float theta, int traverse) {
    StepArgs a{};
    a.n = n;
    a.pos = pos;
    a.acc = acc;
    a.half_dt = 0.0025f;
    a.dt = 0.005f;
    a.eps2 = 0.05f * 0.05f;
    a.G = 1.f;
    a.theta2 = theta * theta;
    a.key_bits = 30;
    a.traverse = traverse;
    a.t1 = n;
    return a;
  }
  // best of `reps` timed calls after one warm-up; `fn` enqueues on st
  template <typename F>
  int time(F fn, int reps, double* ms) {
    NB_TRY(fn());
    double best = 1e30;
    for (int r = 0; r < reps; ++r) {
      NB_CUDA(cudaEventRecord(e0, st));
      NB_TRY(fn());
      NB_CUDA(cudaEventRecord(e1, st));
      NB_CUDA(cudaEventSynchronize(e1));
      float t = 0.f;
      NB_CUDA(cudaEventElapsedTime(&t, e0, e1));
      best = std::min(best, (double)t);
    }
    NB_CUDA(cudaStreamSynchronize(st));
    *ms = best;
    return NB_OK;
  }
};

int measure(nb_tune_table* t) {
  Bench b;
  NB_TRY(b.init());
  const int sms = t->sms;
  // all-pairs: every compiled shape and 2, 4, 8, 16 CTAs per SM in flight,
  // at the bottom of each size bucket up to 2^16 particles; the larger
  // buckets keep the 2^16 shape (one CTA per target tile fills the device)
  const int shapes[6][2] = {{128, 2}, {128, 4}, {128, 8}, {256, 2}, {256, 4}, {256, 8}};
  const int per_sm[4] = {2, 4, 8, 16};
  constexpr int kMeasuredBuckets = 8;   // n = 2^9 .. 2^16
  for (int bk = 0; bk < kMeasuredBuckets; ++bk) {
    const int n = 1 << (9 + bk);
    NB_TRY(b.load(n));
    StepArgs a = b.args(n, 0.5f, NB_TRAVERSE_WARP);
    // the packed sources' buffer (and the workspace's basics) before the
    // prep kernel writes them
    NB_TRY(ws_reserve_allpairs(b.w, n, allpairs_geometry_for(n, 256, 4, 8 * sms)));
    NB_TRY(launch_prep(b.w, a, false, true, b.st));   // packed sources
    double best = 1e30;
    for (auto& sh : shapes)
      for (int c : per_sm) {
        const APGeom g = allpairs_geometry_for(n, sh[0], sh[1], c * sms);
        double ms = 0.0;
        NB_TRY(b.time([&]() { return launch_allpairs_geom(b.w, a, g, b.st); }, 3, &ms));
        if (ms < best * 0.98) {   // a clear win only, else keep the earlier shape
          best = ms;
          t->ap_threads[bk] = sh[0];
          t->ap_k[bk] = sh[1];
          t->ap_ctas[bk] = c * sms;
        }
      }
  }
  for (int bk = kMeasuredBuckets; bk < NB_TUNE_BUCKETS; ++bk) {
    t->ap_threads[bk] = t->ap_threads[kMeasuredBuckets - 1];
    t->ap_k[bk] = t->ap_k[kMeasuredBuckets - 1];
    t->ap_ctas[bk] = t->ap_ctas[kMeasuredBuckets - 1];
  }
  // the launchers read the live table: install the shapes chosen so far
  auto install = [&]() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_tab[current_device()] = *t;
  };
  install();
  // the walk's warps per block, on the largest crossover size
  {
    const int n = 131072;
    NB_TRY(b.load(n));
    double best = 1e30;
    int best_w = 4;
    for (int wpb : {4, 2, 8}) {
      t->walk_warps = wpb;
      install();
      StepArgs a = b.args(n, 0.5f, NB_TRAVERSE_WARP);
      double ms = 0.0;
      NB_TRY(b.time([&]() { return enqueue_forces(b.w, a, NB_FORCE_BH, b.st, nullptr); }, 3,
                    &ms));
      if (ms < best * 0.98) {
        best = ms;
        best_w = wpb;
      }
    }
    t->walk_warps = best_w;
    install();
  }
  // crossover: all-pairs (the shapes just chosen) against Barnes-Hut on a
  // geometric grid of sizes; the crossover is the geometric mean of the last
  // size all-pairs wins and the first Barnes-Hut wins from
  std::vector<int> grid;
  for (int k = 0; k <= 12; ++k)
    grid.push_back((int)std::lround(2048.0 * std::pow(2.0, k / 2.0)) / 32 * 32);
  std::vector<double> t_ap(grid.size());
  std::vector<std::vector<double>> t_bh(NB_TUNE_THETAS * 2, std::vector<double>(grid.size()));
  for (size_t gi = 0; gi < grid.size(); ++gi) {
    const int n = grid[gi];
    NB_TRY(b.load(n));
    StepArgs a = b.args(n, 0.5f, NB_TRAVERSE_WARP);
    NB_TRY(b.time([&]() { return enqueue_forces(b.w, a, NB_FORCE_NAIVE, b.st, nullptr); }, 3,
                  &t_ap[gi]));
    for (int i = 0; i < NB_TUNE_THETAS; ++i)
      for (int tr = 0; tr < 2; ++tr) {
        StepArgs ab = b.args(n, kThetaClass[i], tr);
        NB_TRY(b.time([&]() { return enqueue_forces(b.w, ab, NB_FORCE_BH, b.st, nullptr); },
                      3, &t_bh[i * 2 + tr][gi]));
      }
  }
  for (int i = 0; i < NB_TUNE_THETAS; ++i)
    for (int tr = 0; tr < 2; ++tr) {
      const std::vector<double>& tb = t_bh[i * 2 + tr];
      // first size from which Barnes-Hut stays faster
      size_t first = grid.size();
      for (size_t gi = grid.size(); gi-- > 0;) {
        if (tb[gi] < t_ap[gi]) first = gi;
        else break;
      }
      int x;
      if (first == 0) x = grid[0];
      else if (first == grid.size()) x = 2 * grid.back();
      else x = (int)std::lround(std::sqrt((double)grid[first - 1] * grid[first]));
      t->crossover[i][tr] = x;
    }
  install();
  // inside a batch: ensembles of equal-size simulations (about 2M particles
  // in all) advanced together, all-pairs against Barnes-Hut per
  // particle-step; the crossover is the first size from which Barnes-Hut
  // stays cheaper (the geometric mean with the size before)
  {
    const int bgrid[6] = {1024, 2048, 4096, 8192, 16384, 32768};
    double ap_cost[6], bh_cost[NB_TUNE_THETAS][6];
    for (int gi = 0; gi < 6; ++gi) {
      const int n = bgrid[gi];
      const int k = std::min(256, std::max(4, (1 << 21) / n));
      std::vector<float4> one;
      two_disks(n, one);
      std::vector<float4> pos((size_t)k * n), vel((size_t)k * n, make_float4(0.f, 0.f, 0.f, 0.f));
      for (int s = 0; s < k; ++s) std::copy(one.begin(), one.end(), pos.begin() + (size_t)s * n);
      std::vector<int> ns(k, n);
      auto cost = [&](int force, float theta, double* out) {
        nb_params p;
        nb_params_default(&p);
        p.dt = 0.005f;
        p.eps = 0.05f;
        p.theta = theta;
        p.force = force;
        p.traverse = NB_TRAVERSE_WARP;
        std::vector<nb_params> ps(k, p);
        nb_ensemble* e = nullptr;
        NB_TRY(nb_ensemble_create(k, ns.data(), (const float*)pos.data(),
                                  (const float*)vel.data(), ps.data(), &e));
        int rc = nb_ensemble_step(e, 2);
        if (rc == NB_OK) rc = nb_ensemble_sync(e);
        if (rc == NB_OK) rc = nb_ensemble_record(e, 0);
        if (rc == NB_OK) rc = nb_ensemble_step(e, 3);
        if (rc == NB_OK) rc = nb_ensemble_record(e, 1);
        double ms = 0.0;
        if (rc == NB_OK) rc = nb_ensemble_elapsed_ms(e, 0, 1, &ms);
        nb_ensemble_destroy(e);
        NB_TRY(rc);
        *out = ms / 3.0 / ((double)k * n);
        return NB_OK;
      };
      NB_TRY(cost(NB_FORCE_NAIVE, 0.5f, &ap_cost[gi]));
      for (int i = 0; i < NB_TUNE_THETAS; ++i)
        NB_TRY(cost(NB_FORCE_BH, kThetaClass[i], &bh_cost[i][gi]));
    }
    for (int i = 0; i < NB_TUNE_THETAS; ++i) {
      int first = 6;
      for (int gi = 6; gi-- > 0;) {
        if (bh_cost[i][gi] < ap_cost[gi]) first = gi;
        else break;
      }
      t->crossover_batch[i] =
          first == 0 ? bgrid[0]
                     : (first == 6 ? 2 * bgrid[5]
                                   : (int)std::lround(std::sqrt((double)bgrid[first - 1] *
                                                                bgrid[first])));
    }
  }
  NB_CUDA(cudaStreamSynchronize(b.st));
  // a measurement that ran into a device error is not kept
  unsigned e = 0;
  if (b.w.err) NB_CUDA(cudaMemcpy(&e, b.w.err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (e) return set_error(NB_ERR_DEVICE, "device error word set while tuning");
  return NB_OK;
}

int save(const nb_tune_table& t, const std::string& path) {
  NB_TRY(mkdirs_for(path));
  const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return set_error(NB_ERR_IO, "cannot open " + tmp);
  bool ok = std::fwrite(&t, sizeof(t), 1, f) == 1;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return set_error(NB_ERR_IO, "cannot write " + path);
  }
  return NB_OK;
}

int load(const std::string& path, nb_tune_table* t) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return set_error(NB_ERR_NOTFOUND, "no tuning cache at " + path);
  nb_tune_table x;
  const bool ok = std::fread(&x, sizeof(x), 1, f) == 1;
  std::fclose(f);
  nb_tune_table here;
  defaults(&here);
  if (!ok || !table_ok(x) || x.sms != here.sms ||
      std::strncmp(x.device, here.device, sizeof(x.device)) != 0)
    return set_error(NB_ERR_NOTFOUND, "tuning cache " + path + " is not for this device");
  *t = x;
  return NB_OK;
}

}  // namespace

void tune_allpairs(int n, int* threads, int* k, int* ctas) {
  std::lock_guard<std::mutex> lk(g_mu);
  const nb_tune_table& t = table_locked();
  int b = 0;
  while (b + 1 < NB_TUNE_BUCKETS && n >= (1 << (10 + b))) ++b;
  *threads = t.ap_threads[b];
  *k = t.ap_k[b];
  *ctas = t.ap_ctas[b];
}

int tune_walk_warps() {
  std::lock_guard<std::mutex> lk(g_mu);
  return table_locked().walk_warps;
}

int tune_crossover(float theta, int traverse) {
  std::lock_guard<std::mutex> lk(g_mu);
  const nb_tune_table& t = table_locked();
  int best = 0;
  for (int i = 1; i < NB_TUNE_THETAS; ++i)
    if (std::fabs(theta - kThetaClass[i]) < std::fabs(theta - kThetaClass[best])) best = i;
  return t.crossover[best][traverse == NB_TRAVERSE_WARP ? 1 : 0];
}

int resolve_force_tuned(int force, int n, float theta, int traverse) {
  if (force != NB_FORCE_AUTO) return force;
  return n < tune_crossover(theta, traverse) ? NB_FORCE_NAIVE : NB_FORCE_BH;
}

int resolve_force_batch(int force, int n, float theta) {
  if (force != NB_FORCE_AUTO) return force;
  std::lock_guard<std::mutex> lk(g_mu);
  const nb_tune_table& t = table_locked();
  int best = 0;
  for (int i = 1; i < NB_TUNE_THETAS; ++i)
    if (std::fabs(theta - kThetaClass[i]) < std::fabs(theta - kThetaClass[best])) best = i;
  return n < t.crossover_batch[best] ? NB_FORCE_NAIVE : NB_FORCE_BH;
}

int tune_ensure(cudaStream_t st) {
  if (g_measuring) return NB_OK;
  const int dev = current_device();
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_state[dev] == 2) return NB_OK;
  }
  if (st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return NB_OK;   // never measure under capture: the current table stands
    }
  }
  const char* mode = std::getenv("NBODY_B200_TUNE");
  const bool off = mode && std::strcmp(mode, "off") == 0;
  const std::string path = cache_path();
  nb_tune_table t;
  if (!off && load(path, &t) == NB_OK) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_state[dev] != 2) {
      g_tab[dev] = t;
      g_state[dev] = 2;
    }
    return NB_OK;
  }
  if (off) {
    std::lock_guard<std::mutex> lk(g_mu);
    table_locked();
    g_state[dev] = 2;   // defaults, as asked
    return NB_OK;
  }
  nb_tune_table out;
  return nb_autotune(path.c_str(), &out);
}

}  // namespace nb

using namespace nb;

extern "C" {

int nb_autotune(const char* cache_path_out, nb_tune_table* out) {
  const int dev = current_device();
  nb_tune_table t;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    defaults(&t);
    g_tab[dev] = t;   // candidates are timed against the defaults elsewhere
    g_state[dev] = 1;
  }
  g_measuring = true;
  int rc = measure(&t);
  g_measuring = false;
  std::lock_guard<std::mutex> lk(g_mu);
  if (rc != NB_OK) {
    defaults(&g_tab[dev]);
    g_state[dev] = 1;
    return rc;
  }
  g_tab[dev] = t;
  g_state[dev] = 2;
  if (out) *out = t;
  if (cache_path_out && *cache_path_out) NB_TRY(save(t, cache_path_out));
  return NB_OK;
}

int nb_tune_get(nb_tune_table* out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  std::lock_guard<std::mutex> lk(g_mu);
  *out = table_locked();
  return NB_OK;
}

int nb_tune_set(const nb_tune_table* t) {
  if (!t) return set_error(NB_ERR_INVALID, "table is NULL");
  if (!table_ok(*t)) return set_error(NB_ERR_INVALID, "invalid tuning table");
  std::lock_guard<std::mutex> lk(g_mu);
  const int dev = current_device();
  g_tab[dev] = *t;
  g_state[dev] = 2;
  return NB_OK;
}

int nb_tune_defaults(nb_tune_table* out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  defaults(out);
  return NB_OK;
}

int nb_tune_load(const char* path) {
  nb_tune_table t;
  NB_TRY(load(path && *path ? std::string(path) : cache_path(), &t));
  std::lock_guard<std::mutex> lk(g_mu);
  const int dev = current_device();
  g_tab[dev] = t;
  g_state[dev] = 2;
  return NB_OK;
}

int nb_tune_save(const char* path) {
  nb_tune_table t;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    t = table_locked();
  }
  return save(t, path && *path ? std::string(path) : cache_path());
}

}  // extern "C"
