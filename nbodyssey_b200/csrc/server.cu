// Simulation request server with continuous batching (no reference
// counterpart: the reference runs one simulation per process).
//
// A pool of particle slots sized by an HBM budget holds every running
// simulation's state and tree (the ensemble layout of nb_internal.cuh).  An
// engine thread loops: retire simulations whose final state has reached the
// host, admit waiting requests whose footprint fits a free slot range (in
// arrival order, later ones may pass a request that does not fit yet), and
// advance every running simulation by one leapfrog step with one set of
// launches.  A newly admitted simulation only computes a(x0) in the step it
// joins, so its trajectory is exactly the one it has alone.  Frames leave the
// device through a staging ring: a device-to-device copy on the compute
// stream, a device-to-host copy on a side stream, and a writer thread.  At
// most two steps are in flight, so admission and completion times follow the
// device.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "nb_internal.cuh"

using namespace nb;

namespace {

constexpr size_t kBytesPerSlot = 232;   // state 64, sorted 16, keys 16, perm 8,
                                        // child pairs 48, sums 32, boxes 32,
                                        // sort scratch ~12, build plan and
                                        // segments ~4
constexpr int kInFlight = 2;            // engine steps queued ahead of the GPU
constexpr int kApChunk = 1024;          // all-pairs scratch allocation unit (float4)
constexpr int kApPoolShare = 8;         // 1 / 8 of the budget: all-pairs scratch
constexpr int kFrameSlots = 8;

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  long long id = 0;
  int n = 0;
  nb_params p{};
  int steps = 0;
  int dump_every = 0;
  std::string out_dir;
  float* h_state = nullptr;   // pinned: pos4[n] then vel4[n]; the result later
  int state = 0;              // 0 queued, 1 running, 2 done, 3 failed
  int sim = -1;
  int base = -1;
  int force = NB_FORCE_BH;    // the module it gets alone (AUTO resolved)
  int ap_chunk = -1;          // all-pairs: its region in the scratch pool
  int ap_len = 0;             // (units of kApChunk float4)
  int steps_done = 0;
  int frames = 0;
  bool primed = false;
  double t_submit = 0, t_admit = 0, t_done = 0;
  cudaEvent_t done_ev = nullptr;
  std::string error;
};

struct FrameJob {
  int slot;
  long long req;
  int index;
  int n;
  std::string dir;
  cudaEvent_t ready;
};

}  // namespace

struct nb_server {
  size_t budget = 0;
  int cap_slots = 0;
  int max_sims = 0;
  EnsArgs e{};
  std::vector<void*> dallocs;
  std::vector<SimDesc> sims;         // host mirror, by sim id
  std::vector<int> blk;              // host mirror of blk_sim
  std::map<int, int> free_blocks;    // start block -> length (32-slot blocks)
  // all-pairs requests: packed sources, partials and tickets per request in
  // regions of a scratch pool, and the persistent launch's work items
  float4* d_ap_pool = nullptr;
  int ap_chunks = 0;
  std::map<int, int> ap_free;        // start chunk -> length
  std::vector<size_t> ap_region;     // by sim id: region offset (float4)
  std::vector<size_t> ap_region_cap; // by sim id: region size (float4)
  EnsAllPairs ap;
  size_t ap_items_cap = 0;
  bool any_tree = false;
  std::vector<int> walk_items[2];    // the walk queue (host copy)
  int* d_walk_items[2] = {nullptr, nullptr};
  std::vector<int> free_ids;
  bool table_dirty = false;
  BuildPlan plan;                    // tree-build levels of the running sims
  size_t plan_cap = 0;               // BuildRun entries allocated at e.runs
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t step_ev[kInFlight] = {};
  long long step_count = 0;
  // frames
  float4* d_frame = nullptr;
  float* h_frame = nullptr;
  int frame_cap = 0;                 // particles per ring slot
  bool frame_busy[kFrameSlots] = {};
  cudaEvent_t frame_staged[kFrameSlots] = {};
  cudaEvent_t frame_copied[kFrameSlots] = {};
  int frame_next = 0;
  std::deque<FrameJob> frame_q;
  // requests
  std::mutex mu;
  std::condition_variable cv;        // engine wake-up and waiters
  std::deque<Request*> waiting;
  std::vector<Request*> running;
  std::vector<Request*> finishing;
  std::map<long long, std::unique_ptr<Request>> all;
  long long next_id = 1;
  bool stop = false;
  std::thread engine, writer;
  int engine_error = NB_OK;
  std::string engine_msg;
  // stats
  double t_start = 0, busy_first = 0, busy_last = 0;
  long long done = 0, failed = 0, frames = 0;
  double particle_steps = 0;
  long long frame_bytes = 0;
  int peak_running = 0;
};

namespace {

template <typename T>
int srv_alloc(nb_server* s, T** p, size_t count) {
  *p = nullptr;
  cudaError_t e = cudaMalloc((void**)p, (count ? count : 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(NB_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  s->dallocs.push_back(*p);
  return NB_OK;
}

// first fit over a free list (start -> length); returns the start or -1
int take_range(std::map<int, int>& fl, int len) {
  for (auto it = fl.begin(); it != fl.end(); ++it) {
    if (it->second >= len) {
      int start = it->first, have = it->second;
      fl.erase(it);
      if (have > len) fl[start + len] = have - len;
      return start;
    }
  }
  return -1;
}

void give_range(std::map<int, int>& fl, int start, int len) {
  auto it = fl.emplace(start, len).first;
  auto nx = std::next(it);
  if (nx != fl.end() && start + it->second == nx->first) {
    it->second += nx->second;
    fl.erase(nx);
  }
  if (it != fl.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      fl.erase(it);
    }
  }
}

int ap_chunks_of(int n) { return (int)((ap_region_f4(n) + kApChunk - 1) / kApChunk); }

int mkdirs(const std::string& path) {
  std::string cur;
  for (size_t i = 0; i <= path.size(); ++i) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty() && cur != "/" && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
        return NB_ERR_IO;
    }
    if (i < path.size()) cur += path[i];
  }
  return NB_OK;
}

void writer_loop(nb_server* s) {
  for (;;) {
    FrameJob j;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] { return s->stop || !s->frame_q.empty(); });
      if (s->frame_q.empty()) return;
      j = s->frame_q.front();
      s->frame_q.pop_front();
    }
    cudaEventSynchronize(j.ready);
    if (!j.dir.empty())
      nb_write_frame(j.dir.c_str(), j.index, j.n,
                     s->h_frame + (size_t)j.slot * s->frame_cap * 4);
    std::lock_guard<std::mutex> lk(s->mu);
    s->frame_busy[j.slot] = false;
    s->frames += 1;
    s->frame_bytes += 16ll * j.n;
    s->cv.notify_all();
  }
}

// frame of request r after its current step; waits for a free ring slot
int emit_frame(nb_server* s, Request* r, std::unique_lock<std::mutex>& lk) {
  const int slot = s->frame_next;
  s->cv.wait(lk, [&] { return !s->frame_busy[slot]; });
  s->frame_busy[slot] = true;
  s->frame_next = (slot + 1) % kFrameSlots;
  float4* d = s->d_frame + (size_t)slot * s->frame_cap;
  NB_CUDA(cudaMemcpyAsync(d, s->e.pos + r->base, 16 * (size_t)r->n,
                          cudaMemcpyDeviceToDevice, s->stream));
  NB_CUDA(cudaEventRecord(s->frame_staged[slot], s->stream));
  NB_CUDA(cudaStreamWaitEvent(s->side, s->frame_staged[slot], 0));
  NB_CUDA(cudaMemcpyAsync(s->h_frame + (size_t)slot * s->frame_cap * 4, d,
                          16 * (size_t)r->n, cudaMemcpyDeviceToHost, s->side));
  NB_CUDA(cudaEventRecord(s->frame_copied[slot], s->side));
  s->frame_q.push_back(FrameJob{slot, r->id, r->frames, r->n, r->out_dir,
                                s->frame_copied[slot]});
  r->frames += 1;
  s->cv.notify_all();
  return NB_OK;
}

// one engine iteration; called with the lock held (released around waits)
int engine_iteration(nb_server* s, std::unique_lock<std::mutex>& lk) {
  // retire simulations whose final state has reached the host
  for (size_t k = 0; k < s->finishing.size();) {
    Request* r = s->finishing[k];
    if (cudaEventQuery(r->done_ev) != cudaSuccess) { ++k; continue; }
    cudaEventDestroy(r->done_ev);
    r->done_ev = nullptr;
    const int nb32 = (r->n + 31) / 32;
    for (int b = 0; b < nb32; ++b) s->blk[r->base / 32 + b] = -1;
    give_range(s->free_blocks, r->base / 32, nb32);
    if (r->ap_chunk >= 0) {
      give_range(s->ap_free, r->ap_chunk, r->ap_len);
      r->ap_chunk = -1;
    }
    s->free_ids.push_back(r->sim);
    s->table_dirty = true;
    r->state = 2;
    r->t_done = now_s();
    s->done += 1;
    s->finishing.erase(s->finishing.begin() + k);
    s->cv.notify_all();
  }
  // admit waiting requests that fit
  for (size_t k = 0; k < s->waiting.size();) {
    Request* r = s->waiting[k];
    const int nb32 = (r->n + 31) / 32;
    if (s->free_ids.empty()) break;
    int ap0 = -1;
    if (r->force == NB_FORCE_NAIVE) {
      ap0 = take_range(s->ap_free, ap_chunks_of(r->n));
      if (ap0 < 0) { ++k; continue; }
    }
    const int b0 = take_range(s->free_blocks, nb32);
    if (b0 < 0) {
      if (ap0 >= 0) give_range(s->ap_free, ap0, ap_chunks_of(r->n));
      ++k;
      continue;
    }
    if (ap0 >= 0) {
      r->ap_chunk = ap0;
      r->ap_len = ap_chunks_of(r->n);
      // sources start with zero-mass pads and tickets at zero
      NB_CUDA(cudaMemsetAsync(s->d_ap_pool + (size_t)ap0 * kApChunk, 0,
                              sizeof(float4) * kApChunk * (size_t)r->ap_len, s->stream));
    }
    std::sort(s->free_ids.begin(), s->free_ids.end(), std::greater<int>());
    const int id = s->free_ids.back();
    s->free_ids.pop_back();
    r->sim = id;
    r->base = b0 * 32;
    r->state = 1;
    r->t_admit = now_s();
    const size_t bytes = 16 * (size_t)r->n;
    NB_CUDA(cudaMemcpyAsync(s->e.pos + r->base, r->h_state, bytes, cudaMemcpyHostToDevice, s->stream));
    NB_CUDA(cudaMemcpyAsync(s->e.vel + r->base, r->h_state + 4 * (size_t)r->n, bytes,
                            cudaMemcpyHostToDevice, s->stream));
    NB_CUDA(cudaMemsetAsync(s->e.pos_lo + r->base, 0, bytes, s->stream));
    NB_CUDA(cudaMemsetAsync(s->e.acc + r->base, 0, bytes, s->stream));
    SimDesc& d = s->sims[id];
    d.n = r->n;
    d.base = r->base;
    d.traverse = r->p.traverse;
    d.half_dt = 0.5f * r->p.dt;
    d.dt = r->p.dt;
    d.eps2 = r->p.eps * r->p.eps;
    d.G = r->p.G;
    d.theta2 = r->p.theta * r->p.theta;
    d.active = 2;   // a(x0) in the step it joins
    d.compensated = r->p.compensated ? 1 : 0;
    d.force = r->force;
    s->ap_region[id] = r->ap_chunk >= 0 ? (size_t)r->ap_chunk * kApChunk : 0;
    s->ap_region_cap[id] = r->ap_chunk >= 0 ? (size_t)r->ap_len * kApChunk : 0;
    for (int b = 0; b < nb32; ++b) s->blk[b0 + b] = id;
    s->table_dirty = true;
    s->running.push_back(r);
    s->waiting.erase(s->waiting.begin() + k);
  }
  if ((int)s->running.size() > s->peak_running) s->peak_running = (int)s->running.size();
  if (s->running.empty()) return NB_OK;

  // table: every id (inactive ones are skipped by the kernels and give
  // unused-slot keys); compact offsets count the participating particles in
  // id order, which is the order the sort groups them in
  const int nsims = s->max_sims;
  int extent = 0;
  for (int id = 0; id < nsims; ++id)
    if (s->sims[id].active)
      extent = std::max(extent, s->sims[id].base + (s->sims[id].n + 31) / 32 * 32);
  if (s->table_dirty) {
    int coff = 0;
    s->any_tree = false;
    for (int id = 0; id < nsims; ++id)
      if (s->sims[id].active && s->sims[id].force == NB_FORCE_BH) {
        s->sims[id].coff = coff;
        coff += s->sims[id].n;
        s->any_tree = true;
      }
    // pageable sources: the calls return once the data is staged, so the
    // host mirrors may change right after; the device copies stay in stream
    // order between the previous step and the next
    NB_CUDA(cudaMemcpyAsync((void*)s->e.sims, s->sims.data(), sizeof(SimDesc) * nsims,
                            cudaMemcpyHostToDevice, s->stream));
    NB_CUDA(cudaMemcpyAsync((void*)s->e.blk_sim, s->blk.data(), sizeof(int) * (extent / 32),
                            cudaMemcpyHostToDevice, s->stream));
    NB_TRY(plan_build(s->sims.data(), nsims, s->plan));
    if (s->plan.runs.size() > s->plan_cap)
      return set_error(NB_ERR_INVALID, "tree-build plan exceeds its buffer");
    if (!s->plan.runs.empty())
      NB_CUDA(cudaMemcpyAsync((void*)s->e.runs, s->plan.runs.data(),
                              sizeof(BuildRun) * s->plan.runs.size(),
                              cudaMemcpyHostToDevice, s->stream));
    int too_small = 0;
    plan_ens_allpairs(s->sims.data(), nsims, s->ap_region.data(), s->ap,
                      s->ap_region_cap.data(), &too_small);
    if (too_small)
      return set_error(NB_ERR_STATE, "the tuning table changed while all-pairs requests "
                                     "were running: their scratch no longer fits");
    if (s->ap.items.size() > s->ap_items_cap) {   // grow-only, rare
      NB_CUDA(cudaStreamSynchronize(s->stream));
      if (s->ap.d_items) cudaFree(s->ap.d_items);
      s->ap.d_items = nullptr;
      const size_t cap = std::max(s->ap.items.size() * 2, (size_t)4096);
      NB_CUDA(cudaMalloc(&s->ap.d_items, sizeof(int4) * cap));
      s->ap_items_cap = cap;
    }
    NB_TRY(bind_ens_allpairs(s->ap, s->sims.data(), nsims, s->e, s->stream));
    plan_walk_queue(s->sims.data(), nsims, s->walk_items);
    for (int q = 0; q < 2; ++q) {
      if (!s->walk_items[q].empty())
        NB_CUDA(cudaMemcpyAsync(s->d_walk_items[q], s->walk_items[q].data(),
                                sizeof(int) * s->walk_items[q].size(),
                                cudaMemcpyHostToDevice, s->stream));
      s->e.walk_items[q] = s->d_walk_items[q];
      s->e.walk_nitems[q] = (int)s->walk_items[q].size();
    }
    s->table_dirty = false;
  }
  // bound the queue depth: wait for the step issued kInFlight iterations ago
  cudaEvent_t ev = s->step_ev[s->step_count % kInFlight];
  if (s->step_count >= kInFlight) {
    lk.unlock();
    cudaEventSynchronize(ev);
    lk.lock();
  }
  EnsArgs e = s->e;
  e.nsims = nsims;
  e.nslots = extent;
  e.nblocks = extent / 32;
  // look-back words laid out (and cleared) for this step's extent only
  e.status_tiles = (extent + kSortTile - 1) / kSortTile;
  e.kick_drift = true;
  e.kick_after = true;
  NB_TRY(launch_ens_prep(e, s->stream));
  if (s->any_tree) {
    NB_TRY(launch_ens_morton(e, s->stream));
    NB_TRY(launch_ens_sort(e, s->stream));
    NB_TRY(launch_ens_levels(e, s->plan, s->stream));
    NB_TRY(launch_walk_pair_ens(e, s->stream));
  }
  NB_TRY(launch_ens_allpairs(e, s->ap, s->stream));
  NB_CUDA(cudaEventRecord(ev, s->stream));
  s->step_count += 1;
  if (s->busy_first == 0) s->busy_first = now_s();

  // bookkeeping after the step
  for (size_t k = 0; k < s->running.size();) {
    Request* r = s->running[k];
    SimDesc& d = s->sims[r->sim];
    if (d.active == 2) {        // primed in this step
      d.active = 1;
      s->table_dirty = true;
      if (r->steps == 0) {
        d.active = 0;
      } else {
        ++k;
        continue;
      }
    } else {
      const int step = r->steps_done;   // 0-based index of the step just taken
      r->steps_done += 1;
      s->particle_steps += r->n;
      if (r->dump_every > 0 && step % r->dump_every == 0) NB_TRY(emit_frame(s, r, lk));
      if (r->steps_done < r->steps) {
        ++k;
        continue;
      }
      d.active = 0;
      s->table_dirty = true;
    }
    // finished: final state to the host, then release at retirement
    const size_t bytes = 16 * (size_t)r->n;
    NB_CUDA(cudaMemcpyAsync(r->h_state, s->e.pos + r->base, bytes, cudaMemcpyDeviceToHost, s->stream));
    NB_CUDA(cudaMemcpyAsync(r->h_state + 4 * (size_t)r->n, s->e.vel + r->base, bytes,
                            cudaMemcpyDeviceToHost, s->stream));
    NB_CUDA(cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming));
    NB_CUDA(cudaEventRecord(r->done_ev, s->stream));
    s->finishing.push_back(r);
    s->running.erase(s->running.begin() + k);
  }
  s->busy_last = now_s();
  return NB_OK;
}

void engine_loop(nb_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv.wait_for(lk, std::chrono::milliseconds(1), [&] {
      return s->stop || !s->waiting.empty() || !s->running.empty() ||
             !s->finishing.empty();
    });
    if (s->stop && s->running.empty() && s->waiting.empty() && s->finishing.empty())
      break;
    if (s->stop) {   // abandon queued work on shutdown
      for (Request* r : s->waiting) { r->state = 3; r->error = "server stopped"; }
      s->waiting.clear();
    }
    int rc = engine_iteration(s, lk);
    if (rc != NB_OK) {
      s->engine_error = rc;
      s->engine_msg = last_error();
      for (Request* r : s->running) { r->state = 3; r->error = s->engine_msg; }
      for (Request* r : s->waiting) { r->state = 3; r->error = s->engine_msg; }
      s->failed += (long long)(s->running.size() + s->waiting.size());
      s->running.clear();
      s->waiting.clear();
      s->cv.notify_all();
      break;
    }
  }
}

}  // namespace

extern "C" {

int nb_server_create(size_t hbm_budget_bytes, int max_sims, nb_server** out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (max_sims <= 0 || max_sims > kEnsMaxSims)
    return set_error(NB_ERR_INVALID, "max_sims must be in [1, 1023]");
  // the slot pool takes all but 1 / kApPoolShare of the budget; the rest is
  // the all-pairs requests' scratch
  const size_t ap_bytes = hbm_budget_bytes / kApPoolShare;
  size_t slots = (hbm_budget_bytes - ap_bytes) / kBytesPerSlot / 4096 * 4096;
  if (slots < 4096) return set_error(NB_ERR_INVALID, "HBM budget too small");
  if (slots > ((size_t)1 << 28)) slots = (size_t)1 << 28;
  NB_TRY(warm_kernels());         // first use on this device: load the kernels
  NB_TRY(tune_ensure(nullptr));   // first use on this device: the tuning table
  nb_server* s = new nb_server();
  s->budget = hbm_budget_bytes;
  s->cap_slots = (int)slots;
  s->max_sims = max_sims;
  s->ap_chunks = (int)std::min<size_t>(ap_bytes / (16 * kApChunk), (size_t)1 << 30);
  int rc = NB_OK;
  do {
    EnsArgs& e = s->e;
    if ((rc = srv_alloc(s, &s->d_ap_pool, (size_t)s->ap_chunks * kApChunk)) != NB_OK) break;
    s->ap.d_pool = s->d_ap_pool;
    if ((rc = srv_alloc(s, &s->ap.d_args, (size_t)max_sims)) != NB_OK) break;
    if ((rc = srv_alloc(s, &s->ap.d_src_off, (size_t)max_sims)) != NB_OK) break;
    if ((rc = srv_alloc(s, &s->ap.d_counter, 6)) != NB_OK) break;
    for (int q = 0; q < 2; ++q)
      if ((rc = srv_alloc(s, &s->d_walk_items[q], slots / 32)) != NB_OK) break;
    if (rc != NB_OK) break;
    if ((rc = srv_alloc(s, &e.walk_ctr, 2)) != NB_OK) break;
    const size_t S = slots;
    SimDesc* dsims = nullptr;
    int* dblk = nullptr;
    if ((rc = srv_alloc(s, &dsims, max_sims)) != NB_OK) break;
    if ((rc = srv_alloc(s, &dblk, S / 32)) != NB_OK) break;
    e.sims = dsims;
    e.blk_sim = dblk;
    if ((rc = srv_alloc(s, &e.pos, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.pos_lo, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.vel, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.acc, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.pos_sorted, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.keys, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.keys_alt, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.perm, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.perm_alt, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.pairs, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.sums, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.box_lo, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.box_hi, S)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.bbox_min, 4 * (size_t)max_sims)) != NB_OK) break;
    if ((rc = srv_alloc(s, &e.bbox_max, 4 * (size_t)max_sims)) != NB_OK) break;
    e.status_tiles = (int)((S + kSortTile - 1) / kSortTile);
    const size_t words = 8 * kSortRadix + 8 + (size_t)8 * e.status_tiles * kSortRadix;
    if ((rc = srv_alloc(s, &e.hist, words)) != NB_OK) break;
    e.tile_ctr = e.hist + 8 * kSortRadix;
    e.status = e.hist + 8 * kSortRadix + 8;
    if ((rc = srv_alloc(s, &e.err, 4)) != NB_OK) break;
    {
      // a simulation with G > 1 groups of 1024 leaves has G runs at the
      // first level and at most G / 15 + 1 at each later one: at most three
      // runs per 1024 of its slots (G = 2 is the worst); one with G = 1 has
      // one run
      s->plan_cap = 3 * (S / 1024 + 1) + 2 * (size_t)max_sims + 64;
      BuildRun* runs = nullptr;
      if ((rc = srv_alloc(s, &runs, s->plan_cap)) != NB_OK) break;
      e.runs = runs;
      const size_t segs = plan_seg_entries((int)S, max_sims);
      for (int i = 0; i < 2; ++i) {
        if ((rc = srv_alloc(s, &e.seg[i], segs)) != NB_OK) break;
        if ((rc = srv_alloc(s, &e.seg_count[i], segs)) != NB_OK) break;
      }
      if (rc != NB_OK) break;
    }
    s->frame_cap = std::min<int>((int)S, 1 << 21);
    if ((rc = srv_alloc(s, &s->d_frame, (size_t)kFrameSlots * s->frame_cap)) != NB_OK) break;
    cudaError_t ce = cudaMallocHost((void**)&s->h_frame, 16 * (size_t)kFrameSlots * s->frame_cap);
    if (ce != cudaSuccess) { s->h_frame = nullptr; rc = set_error(NB_ERR_NOMEM, "pinned frame ring"); break; }
    ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking);
    for (int k = 0; k < kInFlight && ce == cudaSuccess; ++k)
      ce = cudaEventCreateWithFlags(&s->step_ev[k], cudaEventDisableTiming);
    for (int k = 0; k < kFrameSlots && ce == cudaSuccess; ++k) {
      ce = cudaEventCreateWithFlags(&s->frame_staged[k], cudaEventDisableTiming);
      if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&s->frame_copied[k], cudaEventDisableTiming);
    }
    if (ce == cudaSuccess) ce = cudaMemset(e.perm, 0, S * 4);
    if (ce == cudaSuccess) ce = cudaMemset(e.perm_alt, 0, S * 4);
    if (ce == cudaSuccess) ce = cudaMemset(e.pairs, 0, S * sizeof(PairRec));
    if (ce == cudaSuccess) ce = cudaMemset(e.hist, 0, words * 4);
    if (ce == cudaSuccess) ce = cudaMemset(e.err, 0, 16);
    if (ce == cudaSuccess) ce = cudaMemset(dblk, 0xff, S / 32 * sizeof(int));
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) { rc = set_error(NB_ERR_CUDA, cudaGetErrorString(ce)); break; }
  } while (0);
  if (rc != NB_OK) {
    std::string keep = last_error();
    for (void* p : s->dallocs) cudaFree(p);
    if (s->h_frame) cudaFreeHost(s->h_frame);
    delete s;
    return set_error(rc, keep);
  }
  s->sims.assign(max_sims, SimDesc{});
  s->ap_region.assign(max_sims, 0);
  s->ap_region_cap.assign(max_sims, 0);
  s->blk.assign(s->cap_slots / 32, -1);
  s->free_blocks[0] = s->cap_slots / 32;
  if (s->ap_chunks > 0) s->ap_free[0] = s->ap_chunks;
  for (int id = max_sims - 1; id >= 0; --id) s->free_ids.push_back(id);
  s->t_start = now_s();
  int dev = 0;
  cudaGetDevice(&dev);
  s->engine = std::thread([s, dev]() {
    cudaSetDevice(dev);
    engine_loop(s);
  });
  s->writer = std::thread([s]() { writer_loop(s); });
  *out = s;
  return NB_OK;
}

int nb_server_destroy(nb_server* s) {
  if (!s) return NB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  s->engine.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->cv.notify_all();
  }
  s->writer.join();
  cudaStreamSynchronize(s->stream);
  cudaStreamSynchronize(s->side);
  for (auto& kv : s->all) {
    if (kv.second->h_state) cudaFreeHost(kv.second->h_state);
    if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
  }
  for (int k = 0; k < kInFlight; ++k) cudaEventDestroy(s->step_ev[k]);
  for (int k = 0; k < kFrameSlots; ++k) {
    cudaEventDestroy(s->frame_staged[k]);
    cudaEventDestroy(s->frame_copied[k]);
  }
  for (void* p : s->dallocs) cudaFree(p);
  if (s->ap.d_items) cudaFree(s->ap.d_items);
  if (s->h_frame) cudaFreeHost(s->h_frame);
  cudaStreamDestroy(s->stream);
  cudaStreamDestroy(s->side);
  delete s;
  return NB_OK;
}

int nb_server_submit(nb_server* s, int n, const float* pos4, const float* vel4,
                     const nb_params* p, int steps, int dump_every,
                     const char* out_dir, long long* id) {
  if (!s || !pos4 || !vel4 || !p || !id) return set_error(NB_ERR_INVALID, "NULL argument");
  if (n <= 0 || steps < 0 || dump_every < 0)
    return set_error(NB_ERR_INVALID, "n > 0, steps >= 0 and dump_every >= 0 required");
  if (!(p->eps > 0.f) || !std::isfinite(p->eps) || !(p->theta >= 0.f) ||
      !std::isfinite(p->dt) || !std::isfinite(p->G))
    return set_error(NB_ERR_INVALID, "eps > 0, theta >= 0, finite dt and G required");
  if ((p->force != NB_FORCE_BH && p->force != NB_FORCE_NAIVE && p->force != NB_FORCE_AUTO) ||
      p->key_bits != 30 ||
      (p->traverse != NB_TRAVERSE_THREAD && p->traverse != NB_TRAVERSE_WARP))
    return set_error(NB_ERR_INVALID, "the server runs all-pairs, Barnes-Hut or AUTO "
                                     "with 30-bit keys");
  if ((size_t)(n + 31) / 32 * 32 > (size_t)s->cap_slots)
    return set_error(NB_ERR_NOMEM, "request larger than the server's HBM budget");
  const int force = resolve_force_batch(p->force, n, p->theta);
  if (force == NB_FORCE_NAIVE && ap_chunks_of(n) > s->ap_chunks)
    return set_error(NB_ERR_NOMEM, "all-pairs request larger than the server's "
                                   "all-pairs scratch (1/8 of the HBM budget)");
  if (dump_every > 0 && n > s->frame_cap)
    return set_error(NB_ERR_INVALID, "frames of more than 2^21 particles are not streamed");
  if (out_dir && *out_dir && mkdirs(out_dir) != NB_OK)
    return set_error(NB_ERR_IO, std::string("cannot create ") + out_dir);
  std::unique_ptr<Request> r(new Request());
  r->n = n;
  r->p = *p;
  r->force = force;
  r->steps = steps;
  r->dump_every = dump_every;
  r->out_dir = out_dir ? out_dir : "";
  cudaError_t ce = cudaMallocHost((void**)&r->h_state, 32 * (size_t)n);
  if (ce != cudaSuccess)
    return set_error(NB_ERR_NOMEM, std::string("cudaMallocHost: ") + cudaGetErrorString(ce));
  std::memcpy(r->h_state, pos4, 16 * (size_t)n);
  std::memcpy(r->h_state + 4 * (size_t)n, vel4, 16 * (size_t)n);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->engine_error != NB_OK) {
    cudaFreeHost(r->h_state);
    return set_error(s->engine_error, "server engine failed: " + s->engine_msg);
  }
  r->id = s->next_id++;
  r->t_submit = now_s();
  *id = r->id;
  s->waiting.push_back(r.get());
  s->all[r->id] = std::move(r);
  s->cv.notify_all();
  return NB_OK;
}

int nb_server_force(nb_server* s, long long id, int* force) {
  if (!s || !force) return set_error(NB_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return set_error(NB_ERR_NOTFOUND, "unknown request id");
  *force = it->second->force;
  return NB_OK;
}

// state: 0 queued, 1 running, 2 done, 3 failed; times in seconds since the
// server started (admitted / done are 0 until they happen).
int nb_server_poll(nb_server* s, long long id, int* state, double* t_submit,
                   double* t_admit, double* t_done) {
  if (!s) return set_error(NB_ERR_INVALID, "server is NULL");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return set_error(NB_ERR_NOTFOUND, "unknown request id");
  Request* r = it->second.get();
  if (state) *state = r->state;
  if (t_submit) *t_submit = r->t_submit - s->t_start;
  if (t_admit) *t_admit = r->t_admit ? r->t_admit - s->t_start : 0.0;
  if (t_done) *t_done = r->t_done ? r->t_done - s->t_start : 0.0;
  return NB_OK;
}

int nb_server_wait(nb_server* s, long long id, double timeout_s) {
  if (!s) return set_error(NB_ERR_INVALID, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return set_error(NB_ERR_NOTFOUND, "unknown request id");
  Request* r = it->second.get();
  bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                           [&] { return r->state >= 2; });
  if (!ok) return set_error(NB_ERR_STATE, "timed out waiting for the request");
  if (r->state == 3) return set_error(NB_ERR_DEVICE, "request failed: " + r->error);
  return NB_OK;
}

// Final state of a finished request (pos4, vel4 may be NULL); with release
// the request is forgotten afterwards.
int nb_server_result(nb_server* s, long long id, float* pos4, float* vel4, int release) {
  if (!s) return set_error(NB_ERR_INVALID, "server is NULL");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return set_error(NB_ERR_NOTFOUND, "unknown request id");
  Request* r = it->second.get();
  if (r->state == 3) return set_error(NB_ERR_DEVICE, "request failed: " + r->error);
  if (r->state != 2) return set_error(NB_ERR_STATE, "request not finished");
  if (pos4) std::memcpy(pos4, r->h_state, 16 * (size_t)r->n);
  if (vel4) std::memcpy(vel4, r->h_state + 4 * (size_t)r->n, 16 * (size_t)r->n);
  if (release) {
    cudaFreeHost(r->h_state);
    s->all.erase(it);
  }
  return NB_OK;
}

int nb_server_get_stats(nb_server* s, nb_server_stats* out) {
  if (!s || !out) return set_error(NB_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = s->done;
  out->failed = s->failed;
  out->queued = (long long)s->waiting.size();
  out->running = (long long)(s->running.size() + s->finishing.size());
  out->engine_steps = s->step_count;
  out->particle_steps = s->particle_steps;
  out->frames = s->frames;
  out->frame_bytes = s->frame_bytes;
  out->busy_s = s->busy_first ? s->busy_last - s->busy_first : 0.0;
  out->peak_running = s->peak_running;
  out->capacity_slots = s->cap_slots;
  long long used = 0;
  for (Request* r : s->running) used += (r->n + 31) / 32 * 32;
  for (Request* r : s->finishing) used += (r->n + 31) / 32 * 32;
  out->used_slots = used;
  if (s->engine_error != NB_OK)
    return set_error(s->engine_error, "server engine failed: " + s->engine_msg);
  return NB_OK;
}

}  // extern "C"
