// C ABI of the force-and-step path: workspace management, the simulation
// handle, pipeline orchestration (eager or one captured CUDA graph per step),
// phase timing, and the device-pointer drop-ins for compute_forces /
// leapfrog_step / total_energy (src/forces.cuh:8, src/integrator.cuh:19-21).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nb_internal.cuh"

namespace nb {

static thread_local std::string g_err;

int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
const char* last_error() { return g_err.c_str(); }

// *diff != 0 when a and b differ in any bit (n float4 rows).
__global__ void k_differ(const uint4* __restrict__ a, const uint4* __restrict__ b, int n,
                         unsigned* diff) {
  unsigned d = 0u;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4 x = a[i], y = b[i];
    d |= (x.x ^ y.x) | (x.y ^ y.y) | (x.z ^ y.z) | (x.w ^ y.w);
  }
  if (__any_sync(0xffffffffu, d != 0u) && (threadIdx.x & 31) == 0) atomicOr(diff, 1u);
}

int launch_differ(const float4* a, const float4* b, int n, unsigned* diff, cudaStream_t st) {
  int blocks = (n + 255) / 256;
  if (blocks > 4 * device_sm_count()) blocks = 4 * device_sm_count();
  if (blocks < 1) blocks = 1;
  k_differ<<<blocks, 256, 0, st>>>((const uint4*)a, (const uint4*)b, n, diff);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

int device_sm_count() {
  static std::mutex mu;
  static int count[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 148;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!count[dev]) {
    int c = 0;
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) {
      cudaGetLastError();
      c = 148;
    }
    count[dev] = c;
  }
  return count[dev];
}

int warm_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    dev = 0;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return NB_OK;
  NB_TRY(warm_prep_kernels());
  NB_TRY(warm_lbvh_kernels());
  NB_TRY(warm_walk_kernels());
  NB_TRY(warm_allpairs_kernels());
  NB_TRY(warm_fns(k_differ));
  done[dev] = true;
  return NB_OK;
}

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------
template <typename T>
static int dalloc(T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(NB_ERR_NOMEM, std::string("cudaMalloc of ") +
                                       std::to_string(count * sizeof(T)) +
                                       " bytes failed: " + cudaGetErrorString(e));
  }
  return NB_OK;
}

static int ws_basic(Workspace& w) {
  if (w.err) return NB_OK;
  NB_TRY(dalloc(&w.err, 4));
  NB_CUDA(cudaMemset(w.err, 0, 4 * sizeof(unsigned)));
  NB_CUDA(cudaMallocHost((void**)&w.h_err, 4 * sizeof(unsigned)));
  NB_TRY(dalloc(&w.bbox, 8));
  NB_TRY(dalloc(&w.bbox_part, (size_t)kPrepMaxBlocks * 6));
  NB_TRY(dalloc(&w.bbox_ticket, 4));
  NB_CUDA(cudaMemset(w.bbox_ticket, 0, 4 * sizeof(unsigned)));
  NB_TRY(dalloc(&w.eout, 8));
  NB_TRY(dalloc(&w.eticket, 4));
  NB_CUDA(cudaMemset(w.eticket, 0, 4 * sizeof(unsigned)));
  NB_CUDA(cudaMallocHost((void**)&w.h_eout, 8 * sizeof(double)));
  return NB_OK;
}

int ws_reserve(Workspace& w, int n, int key_bits) {
  NB_TRY(ws_basic(w));
  if (n <= w.cap && key_bits <= w.key_bits) return NB_OK;
  int cap = n > w.cap ? n : w.cap;
  int kb = key_bits > w.key_bits ? key_bits : w.key_bits;
  size_t ksz = kb == 63 ? 8 : 4;
  size_t ni = cap > 1 ? (size_t)cap - 1 : 1;
  void* k0 = w.keys;
  void* k1 = w.keys_alt;
  if (k0) cudaFree(k0);
  if (k1) cudaFree(k1);
  w.keys = w.keys_alt = nullptr;
  NB_CUDA(cudaMalloc(&w.keys, cap * ksz));
  NB_CUDA(cudaMalloc(&w.keys_alt, cap * ksz));
  NB_TRY(dalloc(&w.vals, cap));
  NB_TRY(dalloc(&w.vals_alt, cap));
  NB_TRY(dalloc(&w.pos_sorted, cap));
  NB_TRY(dalloc(&w.nodes, ni));
  NB_TRY(dalloc(&w.pairs, (size_t)cap));
  NB_TRY(dalloc(&w.parent, 2 * (size_t)cap));
  for (int i = 0; i < 2; ++i) {
    NB_TRY(dalloc(&w.seg[i], build_seg_entries(cap)));
    NB_TRY(dalloc(&w.seg_count[i], build_seg_entries(cap)));
  }
  NB_TRY(dalloc(&w.sums, ni));
  NB_TRY(dalloc(&w.box_lo, ni));
  NB_TRY(dalloc(&w.box_hi, ni));
  NB_TRY(dalloc(&w.counts, cap));
  // defined contents before the first build: in-range indices everywhere
  NB_CUDA(cudaMemset(w.vals, 0, cap * sizeof(uint32_t)));
  NB_CUDA(cudaMemset(w.vals_alt, 0, cap * sizeof(uint32_t)));
  NB_CUDA(cudaMemset(w.parent, 0xff, 2 * (size_t)cap * sizeof(int)));
  NB_CUDA(cudaMemset(w.nodes, 0, ni * sizeof(Node)));
  NB_CUDA(cudaMemset(w.pairs, 0, (size_t)cap * sizeof(PairRec)));
  w.status_tiles = (cap + kSortTile - 1) / kSortTile;
  size_t words = 8 * kSortRadix + 8 + (size_t)8 * w.status_tiles * kSortRadix;
  NB_TRY(dalloc(&w.hist, words));
  NB_CUDA(cudaMemset(w.hist, 0, words * sizeof(uint32_t)));
  w.tile_ctr = w.hist + 8 * kSortRadix;
  w.status = w.hist + 8 * kSortRadix + 8;
  w.cap = cap;
  w.key_bits = kb;
  return NB_OK;
}

int ws_reserve_allpairs(Workspace& w, int n, const APGeom& g) {
  NB_TRY(ws_basic(w));
  int npad = (n + kSrcTile - 1) / kSrcTile * kSrcTile;
  if (npad > w.src_cap) {
    NB_TRY(dalloc(&w.src, (size_t)npad));   // 2 float4 per pair = npad float4
    w.src_cap = npad;
  }
  size_t need = g.jsplit > 1 ? (size_t)g.jsplit * n : 1;
  if (need > (size_t)w.part_cap) {
    NB_TRY(dalloc(&w.part, need));
    w.part_cap = (int)need;
  }
  int itiles = g.itiles + 1;
  if (itiles > w.tickets_cap) {
    NB_TRY(dalloc(&w.tickets, (size_t)itiles));
    NB_CUDA(cudaMemset(w.tickets, 0, itiles * sizeof(unsigned)));
    w.tickets_cap = itiles;
  }
  return NB_OK;
}

int ws_reserve_energy(Workspace& w, int n, int blocks, int jsplit) {
  NB_TRY(ws_basic(w));
  if (blocks * 5 > w.epart_cap) {
    NB_TRY(dalloc(&w.epart, (size_t)blocks * 5));
    w.epart_cap = blocks * 5;
  }
  size_t need = (size_t)jsplit * n;
  if (need > (size_t)w.ephi_cap) {
    NB_TRY(dalloc(&w.ephi, need));
    w.ephi_cap = (int)need;
  }
  return NB_OK;
}

void ws_free(Workspace& w) {
  cudaFree(w.keys); cudaFree(w.keys_alt); cudaFree(w.vals); cudaFree(w.vals_alt);
  cudaFree(w.pos_sorted); cudaFree(w.nodes); cudaFree(w.pairs); cudaFree(w.parent);
  for (int i = 0; i < 2; ++i) { cudaFree(w.seg[i]); cudaFree(w.seg_count[i]); }
  cudaFree(w.sums); cudaFree(w.box_lo); cudaFree(w.box_hi); cudaFree(w.hist);
  cudaFree(w.bbox); cudaFree(w.bbox_part); cudaFree(w.bbox_ticket);
  cudaFree(w.src); cudaFree(w.part); cudaFree(w.tickets); cudaFree(w.epart);
  cudaFree(w.ephi); cudaFree(w.eout); cudaFree(w.eticket); cudaFree(w.counts);
  cudaFree(w.err);
  if (w.h_eout) cudaFreeHost(w.h_eout);
  if (w.h_err) cudaFreeHost(w.h_err);
  w = Workspace{};
}

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
static int check_params(const nb_params* p) {
  if (!p) return set_error(NB_ERR_INVALID, "params is NULL");
  if (!(p->eps > 0.f) || !std::isfinite(p->eps))
    return set_error(NB_ERR_INVALID, "eps must be a finite value > 0");
  if (!(p->theta >= 0.f) || !std::isfinite(p->theta))
    return set_error(NB_ERR_INVALID, "theta must be >= 0");
  if (!std::isfinite(p->dt) || !std::isfinite(p->G))
    return set_error(NB_ERR_INVALID, "dt and G must be finite");
  if (p->force != NB_FORCE_NAIVE && p->force != NB_FORCE_BH && p->force != NB_FORCE_AUTO)
    return set_error(NB_ERR_INVALID, "force must be NB_FORCE_NAIVE, _BH or _AUTO");
  if (p->traverse != NB_TRAVERSE_THREAD && p->traverse != NB_TRAVERSE_WARP)
    return set_error(NB_ERR_INVALID, "traverse must be thread or warp");
  if (p->key_bits != 30 && p->key_bits != 63)
    return set_error(NB_ERR_INVALID, "key_bits must be 30 or 63");
  if (p->walk_kernel < 0 || p->walk_kernel > 2)
    return set_error(NB_ERR_INVALID, "walk_kernel must be 0 or 1");
  return NB_OK;
}

static int check_n(int n) {
  if (n <= 0) return set_error(NB_ERR_INVALID, "n must be > 0");
  if (n >= (1 << 29)) return set_error(NB_ERR_INVALID, "n must be < 2^29");
  return NB_OK;
}

static StepArgs make_args(int n, float4* pos, float4* lo, float4* vel,
                          float4* acc, const nb_params& p) {
  StepArgs a;
  a.n = n;
  a.pos = pos;
  a.pos_lo = lo;
  a.vel = vel;
  a.acc = acc;
  a.half_dt = 0.5f * p.dt;
  a.dt = p.dt;
  a.eps2 = p.eps * p.eps;
  a.G = p.G;
  a.theta2 = p.theta * p.theta;
  a.key_bits = p.key_bits;
  a.traverse = p.traverse;
  a.walk_kernel = p.walk_kernel;
  a.kick_drift = false;
  a.kick_after = false;
  a.counts = nullptr;
  a.t0 = 0;
  a.t1 = n;
  a.part = nullptr;
  a.after_prep = nullptr;
  return a;
}

// Phase event recorder: when `ev` is non-null, records an event after each
// phase into ev[phase].
struct PhaseMarks {
  cudaEvent_t start = nullptr;
  cudaEvent_t mark[NB_PHASES] = {};
  bool used[NB_PHASES] = {};
};

static int mark(PhaseMarks* pm, int phase, cudaStream_t st) {
  if (!pm) return NB_OK;
  NB_CUDA(cudaEventRecord(pm->mark[phase], st));
  pm->used[phase] = true;
  return NB_OK;
}

// NB_FORCE_AUTO: all-pairs below the tuned crossover, Barnes-Hut above.
static int resolve_force(const nb_params& p, int n) {
  return resolve_force_tuned(p.force, n, p.theta, p.traverse);
}

// The whole force evaluation (plus the optional fused kick / drift / kick).
// n < 2 with Barnes-Hut writes zeros as src/forces_bh.cu:466-469 does.
// `force` is NB_FORCE_NAIVE or NB_FORCE_BH (AUTO resolved by the caller).
int enqueue_forces(Workspace& w, const StepArgs& a, int force, cudaStream_t st,
                   PhaseMarks* pm) {
  if (force == NB_FORCE_AUTO)
    force = resolve_force_tuned(force, a.n, std::sqrt(a.theta2), a.traverse);
  // workspace growth (allocation, host side) stays outside the timed region
  if (force == NB_FORCE_NAIVE) NB_TRY(ws_reserve_allpairs(w, a.n, allpairs_geometry(a.n)));
  else if (a.n >= 2) NB_TRY(ws_reserve(w, a.n, a.key_bits));
  if (pm) NB_CUDA(cudaEventRecord(pm->start, st));
  if (force == NB_FORCE_BH && a.n < 2) {
    if (a.kick_drift) NB_TRY(launch_prep(w, a, false, false, st));
    if (a.after_prep) NB_CUDA(cudaEventRecord(a.after_prep, st));
    NB_CUDA(cudaMemsetAsync(a.acc, 0, sizeof(float4) * a.n, st));
    return mark(pm, NB_PHASE_WALK, st);
  }
  if (force == NB_FORCE_NAIVE) {
    NB_TRY(launch_prep(w, a, false, true, st));
    if (a.after_prep) NB_CUDA(cudaEventRecord(a.after_prep, st));
    NB_TRY(mark(pm, NB_PHASE_PREP, st));
    NB_TRY(launch_allpairs(w, a, st));
    return mark(pm, NB_PHASE_WALK, st);
  }
  NB_TRY(launch_prep(w, a, true, false, st));
  if (a.after_prep) NB_CUDA(cudaEventRecord(a.after_prep, st));
  NB_TRY(mark(pm, NB_PHASE_PREP, st));
  NB_TRY(launch_morton(w, a, st));
  NB_TRY(mark(pm, NB_PHASE_MORTON, st));
  NB_TRY(launch_sort(w, a, st));
  NB_TRY(mark(pm, NB_PHASE_SORT, st));
  NB_TRY(launch_build(w, a, st));
  NB_TRY(mark(pm, NB_PHASE_BUILD, st));
  NB_TRY(launch_com(w, a, st));
  NB_TRY(mark(pm, NB_PHASE_COM, st));
  NB_TRY(launch_walk(w, a, st));
  return mark(pm, NB_PHASE_WALK, st);
}

static int check_device_error(Workspace& w, cudaStream_t st) {
  if (!w.err) return NB_OK;
  NB_CUDA(cudaMemcpyAsync(w.h_err, w.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(st));
  unsigned e = *w.h_err;
  if (e) {
    NB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(unsigned), st));
    NB_CUDA(cudaStreamSynchronize(st));
    std::string m = "device error word 0x";
    char buf[16];
    std::snprintf(buf, sizeof(buf), "%x", e);
    m += buf;
    if (e & NB_DEVERR_STACK) m += " (tree walk stack overflow)";
    if (e & NB_DEVERR_TREE) m += " (inconsistent tree in the centre-of-mass pass)";
    if (e & NB_DEVERR_VISITS) m += " (tree walk visit limit)";
    if (e & NB_DEVERR_BOUNDS) m += " (tree-build write out of range, skipped)";
    if (e & NB_DEVERR_SORT) m += " (radix sort look-back wait limit)";
    if (e & NB_DEVERR_WAIT) m += " (bulk-copy barrier wait limit)";
    if (e & NB_DEVERR_QUEUE) m += " (work-queue item out of range, skipped)";
    return set_error(NB_ERR_DEVICE, m);
  }
  return NB_OK;
}

}  // namespace nb

using namespace nb;

// ===========================================================================
// Simulation handle
// ===========================================================================
struct nb_sim {
  int n = 0;
  nb_params p{};
  cudaStream_t stream = nullptr;
  float4* pos = nullptr;
  float4* pos_lo = nullptr;
  float4* vel = nullptr;
  float4* acc = nullptr;
  Workspace ws;
  bool primed = false;
  // graphs
  bool use_graphs = true;
  cudaGraphExec_t graph = nullptr;
  bool graph_valid = false;
  // timing
  bool timing = false;
  std::vector<PhaseMarks*> pending;
  std::vector<PhaseMarks*> pool;
  double phase_ms[NB_PHASES] = {};
  long timed_steps = 0;
  double force_ms = 0.0;
  long force_calls = 0;
  cudaEvent_t slots[16] = {};
  void* flush_buf = nullptr;
  size_t flush_bytes = 0;
  // nb_step_host: positions leave on a side stream once the drift is done
  cudaStream_t io_stream = nullptr;
  cudaEvent_t io_prep = nullptr;
  cudaEvent_t io_in = nullptr;    // host-state steps: positions uploaded
  cudaEvent_t io_vel = nullptr;   // host-state steps: velocities uploaded
  // nb_step_host_state: uploaded positions, and whether they differ from the
  // simulation's own
  float4* pos_in = nullptr;
  unsigned* d_diff = nullptr;
  unsigned* h_diff = nullptr;   // pinned
};

static void sim_free(nb_sim* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (auto* pm : s->pending) s->pool.push_back(pm);
  for (auto* pm : s->pool) {
    cudaEventDestroy(pm->start);
    for (int i = 0; i < NB_PHASES; ++i) cudaEventDestroy(pm->mark[i]);
    delete pm;
  }
  for (auto& e : s->slots)
    if (e) cudaEventDestroy(e);
  if (s->io_stream) {
    cudaStreamSynchronize(s->io_stream);
    cudaStreamDestroy(s->io_stream);
  }
  if (s->io_prep) cudaEventDestroy(s->io_prep);
  if (s->io_in) cudaEventDestroy(s->io_in);
  if (s->io_vel) cudaEventDestroy(s->io_vel);
  cudaFree(s->pos_in);
  cudaFree(s->d_diff);
  if (s->h_diff) cudaFreeHost(s->h_diff);
  cudaFree(s->flush_buf);
  cudaFree(s->pos);
  cudaFree(s->pos_lo);
  cudaFree(s->vel);
  cudaFree(s->acc);
  ws_free(s->ws);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static int get_marks(nb_sim* s, PhaseMarks** out) {
  if (!s->pool.empty()) {
    *out = s->pool.back();
    s->pool.pop_back();
  } else {
    PhaseMarks* pm = new PhaseMarks();
    NB_CUDA(cudaEventCreate(&pm->start));
    for (int i = 0; i < NB_PHASES; ++i) NB_CUDA(cudaEventCreate(&pm->mark[i]));
    *out = pm;
  }
  for (int i = 0; i < NB_PHASES; ++i) (*out)->used[i] = false;
  s->pending.push_back(*out);
  return NB_OK;
}

// Folds the recorded phase events into the accumulators (synchronises).
static int collect_timing(nb_sim* s) {
  if (s->pending.empty()) return NB_OK;
  NB_CUDA(cudaStreamSynchronize(s->stream));
  for (PhaseMarks* pm : s->pending) {
    cudaEvent_t prev = pm->start;
    double total = 0.0;
    bool any = false;
    for (int i = 0; i < NB_PHASES; ++i) {
      if (!pm->used[i]) continue;
      float ms = 0.f;
      NB_CUDA(cudaEventElapsedTime(&ms, prev, pm->mark[i]));
      s->phase_ms[i] += ms;
      if (i != NB_PHASE_ENERGY) total += ms;
      prev = pm->mark[i];
      any = true;
    }
    if (any && !pm->used[NB_PHASE_ENERGY]) {
      s->force_ms += total;
      ++s->force_calls;
      ++s->timed_steps;
    }
    s->pool.push_back(pm);
  }
  s->pending.clear();
  return NB_OK;
}

namespace nb {
int sim_view(nb_sim* s, SimView* v) {
  if (!s || !v) return set_error(NB_ERR_INVALID, "NULL argument");
  v->n = s->n;
  v->stream = s->stream;
  v->pos = s->pos;
  v->vel = s->vel;
  v->ws = &s->ws;
  v->p = s->p;
  return NB_OK;
}
}  // namespace nb

static StepArgs sim_args(nb_sim* s) {
  return make_args(s->n, s->pos, s->p.compensated ? s->pos_lo : nullptr,
                   s->vel, s->acc, s->p);
}

// a(x) into s->acc, no kick / drift.
static int sim_forces(nb_sim* s, int* counts) {
  StepArgs a = sim_args(s);
  a.counts = counts;
  PhaseMarks* pm = nullptr;
  if (s->timing) NB_TRY(get_marks(s, &pm));
  NB_TRY(enqueue_forces(s->ws, a, s->p.force, s->stream, pm));
  s->primed = true;
  return NB_OK;
}

static int sim_step_eager(nb_sim* s, PhaseMarks* pm) {
  StepArgs a = sim_args(s);
  a.kick_drift = true;
  a.kick_after = true;
  return enqueue_forces(s->ws, a, s->p.force, s->stream, pm);
}

static int sim_capture(nb_sim* s) {
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  s->graph_valid = false;
  // reserve first so no allocation happens during capture
  if (resolve_force(s->p, s->n) == NB_FORCE_BH)
    NB_TRY(ws_reserve(s->ws, s->n, s->p.key_bits));
  else
    NB_TRY(ws_reserve_allpairs(s->ws, s->n, allpairs_geometry(s->n)));
  cudaGraph_t g = nullptr;
  NB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = sim_step_eager(s, nullptr);
  cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (rc != NB_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess)
    return set_error(NB_ERR_CUDA, std::string("cudaStreamEndCapture: ") +
                                      cudaGetErrorString(e));
  e = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return set_error(NB_ERR_CUDA, std::string("cudaGraphInstantiate: ") +
                                      cudaGetErrorString(e));
  s->graph_valid = true;
  return NB_OK;
}

extern "C" {

void nb_params_default(nb_params* p) {
  if (!p) return;
  p->dt = 0.01f;
  p->eps = 0.05f;
  p->G = 1.0f;
  p->theta = 0.5f;
  p->force = NB_FORCE_NAIVE;
  p->traverse = NB_TRAVERSE_THREAD;
  p->key_bits = 30;
  p->compensated = 1;
  p->walk_kernel = 0;
}

const char* nb_last_error(void) { return nb::last_error(); }
int nb_version(void) { return 100; }

int nb_device_count(int* out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *out = c;
  return NB_OK;
}

int nb_set_device(int device) {
  NB_CUDA(cudaSetDevice(device));
  return NB_OK;
}

int nb_alloc_pinned(size_t bytes, void** out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  cudaError_t e = cudaMallocHost(out, bytes ? bytes : 1);
  if (e != cudaSuccess) {
    *out = nullptr;
    return set_error(NB_ERR_NOMEM, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
  }
  return NB_OK;
}

int nb_free_pinned(void* p) {
  if (p) NB_CUDA(cudaFreeHost(p));
  return NB_OK;
}

int nb_measure_fp32_peak(double* tflops_scalar, double* tflops_packed) {
  if (!tflops_scalar || !tflops_packed) return set_error(NB_ERR_INVALID, "NULL argument");
  return measure_fp32_peak(tflops_scalar, tflops_packed);
}

int nb_flush_l2(nb_sim* s, size_t bytes) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  if (bytes > s->flush_bytes) {
    cudaFree(s->flush_buf);
    s->flush_buf = nullptr;
    s->flush_bytes = 0;
    NB_CUDA(cudaMalloc(&s->flush_buf, bytes));
    s->flush_bytes = bytes;
  }
  return launch_flush(s->flush_buf, bytes, s->stream);
}

int nb_sim_create(int n, const float* pos4, const float* vel4,
                  const nb_params* p, nb_sim** out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  if (!pos4 || !vel4) return set_error(NB_ERR_INVALID, "pos4 / vel4 is NULL");
  NB_TRY(warm_kernels());         // first use on this device: load the kernels
  NB_TRY(tune_ensure(nullptr));   // first use on this device: the tuning table
  nb_sim* s = new nb_sim();
  s->n = n;
  s->p = *p;
  int rc = NB_OK;
  do {
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { rc = set_error(NB_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)); break; }
    if ((rc = dalloc(&s->pos, n)) != NB_OK) break;
    if ((rc = dalloc(&s->pos_lo, n)) != NB_OK) break;
    if ((rc = dalloc(&s->vel, n)) != NB_OK) break;
    if ((rc = dalloc(&s->acc, n)) != NB_OK) break;
    if ((rc = ws_basic(s->ws)) != NB_OK) break;
    // the force module's workspace now, not inside the first (timed) call
    if (resolve_force(s->p, n) == NB_FORCE_NAIVE)
      rc = ws_reserve_allpairs(s->ws, n, allpairs_geometry(n));
    else if (n >= 2)
      rc = ws_reserve(s->ws, n, s->p.key_bits);
    if (rc != NB_OK) break;
    rc = nb_set_state(s, pos4, vel4);
  } while (0);
  if (rc != NB_OK) {
    std::string keep = nb::last_error();
    sim_free(s);
    return set_error(rc, keep);
  }
  *out = s;
  return NB_OK;
}

int nb_sim_destroy(nb_sim* s) {
  sim_free(s);
  return NB_OK;
}

int nb_sim_n(const nb_sim* s, int* n) {
  if (!s || !n) return set_error(NB_ERR_INVALID, "NULL argument");
  *n = s->n;
  return NB_OK;
}

int nb_set_params(nb_sim* s, const nb_params* p) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_TRY(check_params(p));
  bool changes_forces = p->force != s->p.force || p->eps != s->p.eps ||
                        p->G != s->p.G || p->theta != s->p.theta ||
                        p->traverse != s->p.traverse ||
                        p->key_bits != s->p.key_bits ||
                        p->walk_kernel != s->p.walk_kernel;
  if (p->compensated && !s->p.compensated)
    NB_CUDA(cudaMemsetAsync(s->pos_lo, 0, sizeof(float4) * s->n, s->stream));
  s->p = *p;
  s->graph_valid = false;
  if (changes_forces) s->primed = false;
  return NB_OK;
}

int nb_get_params(const nb_sim* s, nb_params* p) {
  if (!s || !p) return set_error(NB_ERR_INVALID, "NULL argument");
  *p = s->p;
  return NB_OK;
}

int nb_set_state(nb_sim* s, const float* pos4, const float* vel4) {
  if (!s || !pos4 || !vel4) return set_error(NB_ERR_INVALID, "NULL argument");
  size_t b = sizeof(float4) * s->n;
  NB_CUDA(cudaMemcpyAsync(s->pos, pos4, b, cudaMemcpyHostToDevice, s->stream));
  NB_CUDA(cudaMemcpyAsync(s->vel, vel4, b, cudaMemcpyHostToDevice, s->stream));
  NB_CUDA(cudaMemsetAsync(s->pos_lo, 0, b, s->stream));
  // the reference ignores vel.w; keep it as given
  s->primed = false;
  return NB_OK;
}

static int download(nb_sim* s, float* dst, const float4* src) {
  if (!s || !dst) return set_error(NB_ERR_INVALID, "NULL argument");
  NB_CUDA(cudaMemcpyAsync(dst, src, sizeof(float4) * s->n,
                          cudaMemcpyDeviceToHost, s->stream));
  NB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s->ws, s->stream);
}

int nb_set_state_acc(nb_sim* s, const float* pos4, const float* vel4,
                     const float* acc4) {
  if (!s || !acc4) return set_error(NB_ERR_INVALID, "NULL argument");
  NB_TRY(nb_set_state(s, pos4, vel4));
  NB_CUDA(cudaMemcpyAsync(s->acc, acc4, sizeof(float4) * s->n,
                          cudaMemcpyHostToDevice, s->stream));
  s->primed = true;
  return NB_OK;
}

int nb_get_accelerations(nb_sim* s, float* acc4) { return download(s, acc4, s ? s->acc : nullptr); }
int nb_get_positions(nb_sim* s, float* pos4) { return download(s, pos4, s ? s->pos : nullptr); }
int nb_get_velocities(nb_sim* s, float* vel4) { return download(s, vel4, s ? s->vel : nullptr); }
int nb_get_position_lo(nb_sim* s, float* lo4) { return download(s, lo4, s ? s->pos_lo : nullptr); }

int nb_save_state(nb_sim* s, const char* path) {
  if (!s || !path) return set_error(NB_ERR_INVALID, "NULL argument");
  const size_t rows = (size_t)s->n * 4;
  std::vector<float> pos(rows), vel(rows), lo(rows), acc(rows);
  NB_TRY(nb_get_positions(s, pos.data()));
  NB_TRY(nb_get_velocities(s, vel.data()));
  NB_TRY(nb_get_position_lo(s, lo.data()));
  if (s->primed) NB_TRY(nb_get_accelerations(s, acc.data()));
  return nb_write_state_file(path, s->n, pos.data(), vel.data(), lo.data(),
                             s->primed ? acc.data() : nullptr, &s->p);
}

int nb_load_state(nb_sim* s, const char* path) {
  if (!s || !path) return set_error(NB_ERR_INVALID, "NULL argument");
  int cnt = 0;
  NB_TRY(nb_read_state_file(path, &cnt, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  if (cnt != s->n)
    return set_error(NB_ERR_INVALID, "state file holds " + std::to_string(cnt) +
                                         " particles, the simulation " + std::to_string(s->n));
  const size_t rows = (size_t)s->n * 4;
  std::vector<float> pos(rows), vel(rows), lo(rows), acc(rows);
  nb_params p = s->p;
  int flags = 0;
  NB_TRY(nb_read_state_file(path, &cnt, pos.data(), vel.data(), lo.data(), acc.data(), &p,
                            &flags));
  if (flags & NB_STATE_TRAILER) NB_TRY(nb_set_params(s, &p));
  if (flags & NB_STATE_ACC) NB_TRY(nb_set_state_acc(s, pos.data(), vel.data(), acc.data()));
  else NB_TRY(nb_set_state(s, pos.data(), vel.data()));
  if (flags & NB_STATE_LO)
    NB_CUDA(cudaMemcpyAsync(s->pos_lo, lo.data(), sizeof(float4) * s->n,
                            cudaMemcpyHostToDevice, s->stream));
  NB_CUDA(cudaStreamSynchronize(s->stream));
  return NB_OK;
}

int nb_step_host(nb_sim* s, const float* pos4, const float* vel4, const float* acc4,
                 float* pos_out4, float* vel_out4, float* acc_out4) {
  if (!s || !pos4 || !vel4 || !acc4 || !pos_out4 || !vel_out4 || !acc_out4)
    return set_error(NB_ERR_INVALID, "NULL argument");
  if (!s->io_stream)
    NB_CUDA(cudaStreamCreateWithFlags(&s->io_stream, cudaStreamNonBlocking));
  if (!s->io_prep) NB_CUDA(cudaEventCreateWithFlags(&s->io_prep, cudaEventDisableTiming));
  NB_TRY(nb_set_state_acc(s, pos4, vel4, acc4));
  const size_t b = sizeof(float4) * s->n;
  StepArgs a = sim_args(s);
  a.kick_drift = true;
  a.kick_after = true;
  a.after_prep = s->io_prep;
  NB_TRY(enqueue_forces(s->ws, a, s->p.force, s->stream, nullptr));
  // positions are final after the drift: they cross PCIe while the tree is
  // built and walked
  NB_CUDA(cudaStreamWaitEvent(s->io_stream, s->io_prep, 0));
  NB_CUDA(cudaMemcpyAsync(pos_out4, s->pos, b, cudaMemcpyDeviceToHost, s->io_stream));
  NB_CUDA(cudaMemcpyAsync(vel_out4, s->vel, b, cudaMemcpyDeviceToHost, s->stream));
  NB_CUDA(cudaMemcpyAsync(acc_out4, s->acc, b, cudaMemcpyDeviceToHost, s->stream));
  NB_CUDA(cudaStreamSynchronize(s->io_stream));
  NB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s->ws, s->stream);
}

int nb_step_host_state(nb_sim* s, const float* pos4, const float* vel4, float* pos_out4,
                       float* vel_out4) {
  if (!s || !pos4 || !vel4 || !pos_out4 || !vel_out4)
    return set_error(NB_ERR_INVALID, "NULL argument");
  if (!s->io_stream)
    NB_CUDA(cudaStreamCreateWithFlags(&s->io_stream, cudaStreamNonBlocking));
  if (!s->io_prep) NB_CUDA(cudaEventCreateWithFlags(&s->io_prep, cudaEventDisableTiming));
  if (!s->io_in) NB_CUDA(cudaEventCreateWithFlags(&s->io_in, cudaEventDisableTiming));
  if (!s->io_vel) NB_CUDA(cudaEventCreateWithFlags(&s->io_vel, cudaEventDisableTiming));
  if (!s->pos_in) NB_TRY(dalloc(&s->pos_in, s->n));
  if (!s->d_diff) NB_TRY(dalloc(&s->d_diff, 1));
  if (!s->h_diff) NB_CUDA(cudaMallocHost((void**)&s->h_diff, sizeof(unsigned)));
  const size_t b = sizeof(float4) * s->n;
  cudaStream_t st = s->stream;
  // positions first; the velocities follow on the side stream while the
  // positions are compared with the simulation's own
  NB_CUDA(cudaMemcpyAsync(s->pos_in, pos4, b, cudaMemcpyHostToDevice, st));
  NB_CUDA(cudaEventRecord(s->io_in, st));
  NB_CUDA(cudaStreamWaitEvent(s->io_stream, s->io_in, 0));
  NB_CUDA(cudaMemcpyAsync(s->vel, vel4, b, cudaMemcpyHostToDevice, s->io_stream));
  NB_CUDA(cudaEventRecord(s->io_vel, s->io_stream));
  // a(x) and the low-order position parts on the device belong to the
  // simulation's positions: they carry on when the caller hands those back
  bool same = false;
  if (s->primed) {
    NB_CUDA(cudaMemsetAsync(s->d_diff, 0, sizeof(unsigned), st));
    NB_TRY(launch_differ(s->pos_in, s->pos, s->n, s->d_diff, st));
    NB_CUDA(cudaMemcpyAsync(s->h_diff, s->d_diff, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    NB_CUDA(cudaStreamSynchronize(st));
    same = *s->h_diff == 0;
  }
  if (!same) {   // new positions: plain state, a(x) from them first
    NB_CUDA(cudaMemcpyAsync(s->pos, s->pos_in, b, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(cudaMemsetAsync(s->pos_lo, 0, b, st));
    NB_TRY(sim_forces(s, nullptr));
  }
  NB_CUDA(cudaStreamWaitEvent(st, s->io_vel, 0));   // the kick reads the velocities
  StepArgs a = sim_args(s);
  a.kick_drift = true;
  a.kick_after = true;
  a.after_prep = s->io_prep;
  NB_TRY(enqueue_forces(s->ws, a, s->p.force, st, nullptr));
  // positions are final after the drift: they cross PCIe while the tree is
  // built and walked
  NB_CUDA(cudaStreamWaitEvent(s->io_stream, s->io_prep, 0));
  NB_CUDA(cudaMemcpyAsync(pos_out4, s->pos, b, cudaMemcpyDeviceToHost, s->io_stream));
  NB_CUDA(cudaMemcpyAsync(vel_out4, s->vel, b, cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(s->io_stream));
  NB_CUDA(cudaStreamSynchronize(st));
  return check_device_error(s->ws, st);
}

int nb_compute_forces(nb_sim* s, float* acc4) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_TRY(sim_forces(s, nullptr));
  if (acc4) return download(s, acc4, s->acc);
  return NB_OK;
}

int nb_step(nb_sim* s, int nsteps) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  if (nsteps < 0) return set_error(NB_ERR_INVALID, "nsteps must be >= 0");
  if (nsteps == 0) return NB_OK;
  if (!s->primed) NB_TRY(sim_forces(s, nullptr));   // a(x0), src/main.cu:184
  for (int k = 0; k < nsteps; ++k) {
    if (s->timing) {
      PhaseMarks* pm = nullptr;
      NB_TRY(get_marks(s, &pm));
      NB_TRY(sim_step_eager(s, pm));
      continue;
    }
    if (s->use_graphs) {
      if (!s->graph_valid) NB_TRY(sim_capture(s));
      NB_CUDA(cudaGraphLaunch(s->graph, s->stream));
    } else {
      NB_TRY(sim_step_eager(s, nullptr));
    }
  }
  return NB_OK;
}

int nb_sync(nb_sim* s) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s->ws, s->stream);
}

int nb_energy(nb_sim* s, double* e3, double* mom3) {
  if (!s || !e3) return set_error(NB_ERR_INVALID, "NULL argument");
  PhaseMarks* pm = nullptr;
  if (s->timing) {
    NB_TRY(get_marks(s, &pm));
    NB_CUDA(cudaEventRecord(pm->start, s->stream));
  }
  NB_TRY(launch_energy(s->ws, s->n, s->pos, s->vel, s->p.eps * s->p.eps, s->p.G,
                       s->stream));
  if (pm) NB_TRY(mark(pm, NB_PHASE_ENERGY, s->stream));
  NB_CUDA(cudaMemcpyAsync(s->ws.h_eout, s->ws.eout, 6 * sizeof(double),
                          cudaMemcpyDeviceToHost, s->stream));
  NB_CUDA(cudaStreamSynchronize(s->stream));
  NB_TRY(check_device_error(s->ws, s->stream));
  e3[0] = s->ws.h_eout[0];
  e3[1] = s->ws.h_eout[1];
  e3[2] = s->ws.h_eout[2];
  if (mom3) {
    mom3[0] = s->ws.h_eout[3];
    mom3[1] = s->ws.h_eout[4];
    mom3[2] = s->ws.h_eout[5];
  }
  return NB_OK;
}

int nb_set_timing(nb_sim* s, int enable) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  s->timing = enable != 0;
  return NB_OK;
}

int nb_force_timing(nb_sim* s, double* ms_total, long* calls) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_TRY(collect_timing(s));
  if (ms_total) *ms_total = s->force_ms;
  if (calls) *calls = s->force_calls;
  return NB_OK;
}

int nb_reset_timing(nb_sim* s) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_TRY(collect_timing(s));
  for (double& v : s->phase_ms) v = 0.0;
  s->timed_steps = 0;
  s->force_ms = 0.0;
  s->force_calls = 0;
  return NB_OK;
}

int nb_phase_times(nb_sim* s, double* ms, long* calls) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  NB_TRY(collect_timing(s));
  if (ms)
    for (int i = 0; i < NB_PHASES; ++i) ms[i] = s->phase_ms[i];
  if (calls) *calls = s->timed_steps;
  return NB_OK;
}

int nb_record(nb_sim* s, int slot) {
  if (!s || slot < 0 || slot >= 16) return set_error(NB_ERR_INVALID, "bad slot");
  if (!s->slots[slot]) NB_CUDA(cudaEventCreate(&s->slots[slot]));
  NB_CUDA(cudaEventRecord(s->slots[slot], s->stream));
  return NB_OK;
}

int nb_elapsed_ms(nb_sim* s, int a, int b, double* ms) {
  if (!s || !ms || a < 0 || b < 0 || a >= 16 || b >= 16 || !s->slots[a] ||
      !s->slots[b])
    return set_error(NB_ERR_INVALID, "bad slot");
  NB_CUDA(cudaEventSynchronize(s->slots[b]));
  float f = 0.f;
  NB_CUDA(cudaEventElapsedTime(&f, s->slots[a], s->slots[b]));
  *ms = f;
  return NB_OK;
}

int nb_set_graphs(nb_sim* s, int enable) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  s->use_graphs = enable != 0;
  s->graph_valid = false;
  return NB_OK;
}

int nb_debug_lbvh(nb_sim* s, uint64_t* keys_sorted, uint32_t* perm,
                  int32_t* children, int32_t* parent, float* com4,
                  float* size2) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  if (s->n < 2) return set_error(NB_ERR_INVALID, "n must be >= 2 for a tree");
  nb_params bh = s->p;
  bh.force = NB_FORCE_BH;
  StepArgs a = make_args(s->n, s->pos, nullptr, s->vel, s->acc, bh);
  float4* tmp = nullptr;
  NB_TRY(dalloc(&tmp, s->n));
  a.acc = tmp;   // leave the simulation's a(x) untouched
  a.node_records = true;
  int rc = enqueue_forces(s->ws, a, NB_FORCE_BH, s->stream, nullptr);
  if (rc == NB_OK) {
    cudaStream_t st = s->stream;
    const int n = s->n, ni = n - 1;
    std::vector<unsigned char> kbuf((size_t)n * 8);
    size_t ksz = s->p.key_bits == 63 ? 8 : 4;
    cudaMemcpyAsync(kbuf.data(), s->ws.keys, n * ksz, cudaMemcpyDeviceToHost, st);
    if (perm) cudaMemcpyAsync(perm, s->ws.vals, n * 4, cudaMemcpyDeviceToHost, st);
    std::vector<Node> nodes(ni);
    cudaMemcpyAsync(nodes.data(), s->ws.nodes, ni * sizeof(Node), cudaMemcpyDeviceToHost, st);
    if (parent) cudaMemcpyAsync(parent, s->ws.parent, (2 * (size_t)n - 1) * 4, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = set_error(NB_ERR_CUDA, cudaGetErrorString(e));
    if (rc == NB_OK) rc = check_device_error(s->ws, st);
    if (rc == NB_OK) {
      for (int i = 0; i < n && keys_sorted; ++i)
        keys_sorted[i] = ksz == 8 ? ((uint64_t*)kbuf.data())[i]
                                  : (uint64_t)((uint32_t*)kbuf.data())[i];
      for (int i = 0; i < ni; ++i) {
        if (children) { children[2 * i] = nodes[i].left; children[2 * i + 1] = nodes[i].right; }
        if (com4) { com4[4 * i] = nodes[i].com.x; com4[4 * i + 1] = nodes[i].com.y;
                    com4[4 * i + 2] = nodes[i].com.z; com4[4 * i + 3] = nodes[i].com.w; }
        if (size2) size2[i] = nodes[i].size2;
      }
    }
  }
  cudaFree(tmp);
  return rc;
}

int nb_debug_pairs(nb_sim* s, float* rec12) {
  if (!s || !rec12) return set_error(NB_ERR_INVALID, "NULL argument");
  if (s->n < 2) return set_error(NB_ERR_INVALID, "n must be >= 2 for a tree");
  // the records of the tree last built on the current positions
  NB_TRY(nb_debug_lbvh(s, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  NB_CUDA(cudaMemcpyAsync(rec12, s->ws.pairs, sizeof(PairRec) * (size_t)(s->n - 1),
                          cudaMemcpyDeviceToHost, s->stream));
  NB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s->ws, s->stream);
}

int nb_debug_forces(nb_sim* s, float* acc4, int32_t* counts) {
  if (!s) return set_error(NB_ERR_INVALID, "sim is NULL");
  int* dcounts = nullptr;
  if (counts && resolve_force(s->p, s->n) == NB_FORCE_BH && s->n >= 2) {
    NB_TRY(ws_reserve(s->ws, s->n, s->p.key_bits));
    dcounts = s->ws.counts;
  }
  NB_TRY(sim_forces(s, dcounts));
  if (acc4) NB_TRY(download(s, acc4, s->acc));
  if (counts) {
    if (dcounts) {
      std::vector<int> cs(s->n);
      std::vector<uint32_t> perm(s->n);
      NB_CUDA(cudaMemcpyAsync(cs.data(), dcounts, s->n * 4, cudaMemcpyDeviceToHost, s->stream));
      NB_CUDA(cudaMemcpyAsync(perm.data(), s->ws.vals, s->n * 4, cudaMemcpyDeviceToHost, s->stream));
      NB_CUDA(cudaStreamSynchronize(s->stream));
      for (int t = 0; t < s->n; ++t) counts[perm[t]] = cs[t];
    } else {
      for (int i = 0; i < s->n; ++i) counts[i] = s->n;   // all-pairs: n each
    }
  }
  return NB_OK;
}

int nb_compare_forces(nb_sim* s, double* max_rel, double* mean_rel) {
  if (!s || !max_rel || !mean_rel) return set_error(NB_ERR_INVALID, "NULL argument");
  const int n = s->n;
  std::vector<float> a(4 * (size_t)n), b(4 * (size_t)n);
  nb_params keep = s->p;
  nb_params pn = keep, pb = keep;
  pn.force = NB_FORCE_NAIVE;
  pb.force = NB_FORCE_BH;
  int rc = nb_set_params(s, &pn);
  if (rc == NB_OK) rc = nb_compute_forces(s, a.data());
  if (rc == NB_OK) rc = nb_set_params(s, &pb);
  if (rc == NB_OK) rc = nb_compute_forces(s, b.data());
  nb_set_params(s, &keep);
  if (rc != NB_OK) return rc;
  double mx = 0.0, sum = 0.0;
  for (int i = 0; i < n; ++i) {
    double dx = (double)a[4 * i] - b[4 * i], dy = (double)a[4 * i + 1] - b[4 * i + 1],
           dz = (double)a[4 * i + 2] - b[4 * i + 2];
    double an = std::sqrt((double)a[4 * i] * a[4 * i] + (double)a[4 * i + 1] * a[4 * i + 1] +
                          (double)a[4 * i + 2] * a[4 * i + 2]);
    double rel = std::sqrt(dx * dx + dy * dy + dz * dz) / (an + 1e-30);
    sum += rel;
    if (rel > mx) mx = rel;
  }
  *max_rel = mx;
  *mean_rel = sum / n;
  return NB_OK;
}

// ===========================================================================
// Device-pointer drop-ins
// ===========================================================================
}  // extern "C"

struct nb_workspace {
  Workspace ws;
};

extern "C" {

int nb_workspace_create(nb_workspace** out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  *out = new nb_workspace();
  return NB_OK;
}

int nb_workspace_destroy(nb_workspace* w) {
  if (!w) return NB_OK;
  cudaDeviceSynchronize();
  ws_free(w->ws);
  delete w;
  return NB_OK;
}

int nb_compute_forces_dev(nb_workspace* w, int n, const float* d_pos4,
                          float* d_acc4, const nb_params* p, void* stream) {
  if (!w || !d_pos4 || !d_acc4) return set_error(NB_ERR_INVALID, "NULL argument");
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  StepArgs a = make_args(n, (float4*)d_pos4, nullptr, nullptr, (float4*)d_acc4, *p);
  return enqueue_forces(w->ws, a, p->force, (cudaStream_t)stream, nullptr);
}

int nb_leapfrog_step_dev(nb_workspace* w, int n, float* d_pos4, float* d_vel4,
                         float* d_acc4, const nb_params* p, void* stream) {
  if (!w || !d_pos4 || !d_vel4 || !d_acc4)
    return set_error(NB_ERR_INVALID, "NULL argument");
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  StepArgs a = make_args(n, (float4*)d_pos4, nullptr, (float4*)d_vel4,
                         (float4*)d_acc4, *p);
  a.kick_drift = true;
  a.kick_after = true;
  return enqueue_forces(w->ws, a, p->force, (cudaStream_t)stream, nullptr);
}

int nb_forces_range_dev(nb_workspace* w, int n, float* d_pos4, float* d_pos_lo4,
                        float* d_vel4, const float* d_acc4, float* d_part4,
                        const nb_params* p, int t0, int t1, void* stream) {
  if (!w || !d_pos4 || !d_part4) return set_error(NB_ERR_INVALID, "NULL argument");
  if (d_vel4 && !d_acc4)
    return set_error(NB_ERR_INVALID, "the opening kick needs d_acc4 = a(x)");
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  if (resolve_force(*p, n) != NB_FORCE_BH)
    return set_error(NB_ERR_INVALID, "a target range needs Barnes-Hut forces");
  if (t0 < 0 || t1 < t0 || t1 > n || ((t0 & 31) && t0 != n) || ((t1 & 31) && t1 != n))
    return set_error(NB_ERR_INVALID,
                     "need 0 <= t0 <= t1 <= n, t0 and t1 multiples of 32 or n");
  StepArgs a = make_args(n, (float4*)d_pos4, (float4*)d_pos_lo4, (float4*)d_vel4,
                         (float4*)d_acc4, *p);
  a.kick_drift = d_vel4 != nullptr;
  a.t0 = t0;
  a.t1 = t1;
  a.part = (float4*)d_part4;
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 2) {   // no tree: a = 0 (src/forces_bh.cu:466-469)
    NB_TRY(ws_basic(w->ws));
    if (a.kick_drift) NB_TRY(launch_prep(w->ws, a, false, false, st));
    if (t1 > t0) NB_CUDA(cudaMemsetAsync(d_part4, 0, sizeof(float4) * (t1 - t0), st));
    return NB_OK;
  }
  return enqueue_forces(w->ws, a, NB_FORCE_BH, st, nullptr);
}

int nb_forces_gather_dev(nb_workspace* w, int n, const float* d_sorted4,
                         float* d_acc4, float* d_vel4, const nb_params* p,
                         void* stream) {
  if (!w || !d_sorted4 || !d_acc4) return set_error(NB_ERR_INVALID, "NULL argument");
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  if (n >= 2 && w->ws.cap < n)
    return set_error(NB_ERR_INVALID, "no tree of this size in the workspace");
  NB_TRY(ws_basic(w->ws));
  StepArgs a = make_args(n, nullptr, nullptr, (float4*)d_vel4, (float4*)d_acc4, *p);
  return launch_gather_part(w->ws, a, (const float4*)d_sorted4, n >= 2,
                            (cudaStream_t)stream);
}

int nb_total_energy_dev(nb_workspace* w, int n, const float* d_pos4,
                        const float* d_vel4, const nb_params* p, double* e3,
                        void* stream) {
  if (!w || !d_pos4 || !d_vel4 || !e3) return set_error(NB_ERR_INVALID, "NULL argument");
  NB_TRY(check_n(n));
  NB_TRY(check_params(p));
  cudaStream_t st = (cudaStream_t)stream;
  NB_TRY(launch_energy(w->ws, n, (const float4*)d_pos4, (const float4*)d_vel4,
                       p->eps * p->eps, p->G, st));
  NB_CUDA(cudaMemcpyAsync(w->ws.h_eout, w->ws.eout, 6 * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(st));
  NB_TRY(check_device_error(w->ws, st));
  e3[0] = w->ws.h_eout[0];
  e3[1] = w->ws.h_eout[1];
  e3[2] = w->ws.h_eout[2];
  return NB_OK;
}

}  // extern "C"
