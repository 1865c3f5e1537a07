// Batched ensembles: many independent simulations advanced by one set of
// launches per step (no reference counterpart: the reference runs one
// simulation per process).  Every phase of the Barnes-Hut step is one kernel
// over all simulations' slots (k_prep.cu, k_lbvh.cu, k_walk_list.cu), so the
// per-step launch count does not grow with the number of simulations, small
// simulations fill the GPU together, and the step is captured once as a CUDA
// graph.  Each simulation's tree and interaction sets are exactly the ones it
// would get alone, so results are bit-identical alone and in the ensemble.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "nb_internal.cuh"

using namespace nb;

struct nb_ensemble {
  int nsims = 0;
  int nslots = 0;
  std::vector<int> n, base;
  std::vector<nb_params> params;
  cudaStream_t stream = nullptr;
  EnsArgs e{};                 // device pointers as allocated
  SimDesc* d_sims = nullptr;
  int* d_blk = nullptr;
  BuildPlan plan;              // tree-build levels (fixed membership)
  EnsAllPairs ap;              // the all-pairs simulations' work
  std::vector<int> force;      // resolved force module per simulation
  size_t ap_pool_f4 = 0;
  std::vector<int> walk_items[2];   // the walk queue (host copy)
  Workspace ews;               // energy scratch
  double* d_energy = nullptr;  // [nsims][6]
  bool primed = false;
  bool any_tree = false;       // some simulation uses the tree pipeline
  bool use_graphs = true;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t slots[16] = {};
  std::vector<void*> allocs;
};

namespace {

template <typename T>
int ens_alloc(nb_ensemble* h, T** p, size_t count) {
  *p = nullptr;
  cudaError_t e = cudaMalloc((void**)p, (count ? count : 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(NB_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  h->allocs.push_back(*p);
  return NB_OK;
}

void ens_free(nb_ensemble* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (auto& ev : h->slots)
    if (ev) cudaEventDestroy(ev);
  for (void* p : h->allocs) cudaFree(p);
  ws_free(h->ews);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int ens_check_params(const nb_params& p) {
  if (!(p.eps > 0.f) || !std::isfinite(p.eps))
    return set_error(NB_ERR_INVALID, "eps must be a finite value > 0");
  if (!(p.theta >= 0.f) || !std::isfinite(p.theta))
    return set_error(NB_ERR_INVALID, "theta must be >= 0");
  if (!std::isfinite(p.dt) || !std::isfinite(p.G))
    return set_error(NB_ERR_INVALID, "dt and G must be finite");
  if (p.force != NB_FORCE_BH && p.force != NB_FORCE_NAIVE && p.force != NB_FORCE_AUTO)
    return set_error(NB_ERR_INVALID, "force must be NB_FORCE_NAIVE, _BH or _AUTO");
  if (p.traverse != NB_TRAVERSE_THREAD && p.traverse != NB_TRAVERSE_WARP)
    return set_error(NB_ERR_INVALID, "traverse must be thread or warp");
  if (p.key_bits != 30)
    return set_error(NB_ERR_INVALID, "ensembles use 30-bit Morton keys");
  return NB_OK;
}

// One step (kick/drift/kick) or, with `prime`, a(x) only.
int ens_enqueue(nb_ensemble* h, bool prime) {
  EnsArgs e = h->e;
  e.kick_drift = !prime;
  e.kick_after = !prime;
  cudaStream_t st = h->stream;
  NB_TRY(launch_ens_prep(e, st));
  if (h->any_tree) {
    NB_TRY(launch_ens_morton(e, st));
    NB_TRY(launch_ens_sort(e, st));
    NB_TRY(launch_ens_levels(e, h->plan, st));
    NB_TRY(launch_walk_pair_ens(e, st));
  }
  NB_TRY(launch_ens_allpairs(e, h->ap, st));
  return NB_OK;
}

int ens_capture(nb_ensemble* h) {
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  NB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = ens_enqueue(h, false);
  cudaError_t err = cudaStreamEndCapture(h->stream, &g);
  if (rc != NB_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (err != cudaSuccess)
    return set_error(NB_ERR_CUDA, std::string("cudaStreamEndCapture: ") +
                                      cudaGetErrorString(err));
  err = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess)
    return set_error(NB_ERR_CUDA, std::string("cudaGraphInstantiate: ") +
                                      cudaGetErrorString(err));
  return NB_OK;
}

int ens_device_error(nb_ensemble* h) {
  unsigned v = 0;
  NB_CUDA(cudaMemcpyAsync(&v, h->e.err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  NB_CUDA(cudaStreamSynchronize(h->stream));
  if (v) {
    NB_CUDA(cudaMemsetAsync(h->e.err, 0, sizeof(unsigned), h->stream));
    NB_CUDA(cudaStreamSynchronize(h->stream));
    return set_error(NB_ERR_DEVICE, "ensemble device error word 0x" + std::to_string(v));
  }
  return NB_OK;
}

}  // namespace

extern "C" {

int nb_ensemble_create(int nsims, const int* n, const float* pos4,
                       const float* vel4, const nb_params* params,
                       nb_ensemble** out) {
  if (!out) return set_error(NB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (nsims <= 0 || nsims > kEnsMaxSims)
    return set_error(NB_ERR_INVALID, "nsims must be in [1, " + std::to_string(kEnsMaxSims) + "]");
  if (!n || !pos4 || !vel4 || !params) return set_error(NB_ERR_INVALID, "NULL argument");
  long long slots = 0, total = 0;
  for (int s = 0; s < nsims; ++s) {
    if (n[s] <= 0) return set_error(NB_ERR_INVALID, "every n must be > 0");
    NB_TRY(ens_check_params(params[s]));
    slots += (n[s] + 31) / 32 * 32;
    total += n[s];
  }
  if (slots >= (1ll << 29)) return set_error(NB_ERR_INVALID, "too many particles in total");
  NB_TRY(warm_kernels());         // first use on this device: load the kernels
  NB_TRY(tune_ensure(nullptr));   // first use on this device: the tuning table
  nb_ensemble* h = new nb_ensemble();
  h->nsims = nsims;
  h->n.assign(n, n + nsims);
  h->params.assign(params, params + nsims);
  int rc = NB_OK;
  do {
    int b = 0;
    std::vector<SimDesc> sims(nsims);
    std::vector<int> blk;
    int coff = 0;
    for (int s = 0; s < nsims; ++s) {
      h->base.push_back(b);
      const nb_params& p = params[s];
      SimDesc& d = sims[s];
      d.n = n[s];
      d.base = b;
      d.coff = coff;
      d.traverse = p.traverse;
      d.half_dt = 0.5f * p.dt;
      d.dt = p.dt;
      d.eps2 = p.eps * p.eps;
      d.G = p.G;
      d.theta2 = p.theta * p.theta;
      d.active = 1;
      d.compensated = p.compensated ? 1 : 0;
      // the force module (NB_FORCE_AUTO: the tuned crossover inside a
      // batch); all-pairs simulations stay out of the tree pipeline
      d.force = resolve_force_batch(p.force, n[s], p.theta);
      if (d.force == NB_FORCE_BH) coff += n[s];
      h->force.push_back(d.force);
      const int nb32 = (n[s] + 31) / 32;
      for (int k = 0; k < nb32; ++k) blk.push_back(s);
      b += nb32 * 32;
    }
    h->nslots = b;
    EnsArgs& e = h->e;
    e.nsims = nsims;
    e.nslots = b;
    e.nblocks = b / 32;
    if ((rc = ens_alloc(h, &h->d_sims, nsims)) != NB_OK) break;
    if ((rc = ens_alloc(h, &h->d_blk, e.nblocks)) != NB_OK) break;
    e.sims = h->d_sims;
    e.blk_sim = h->d_blk;
    const size_t S = (size_t)b;
    if ((rc = ens_alloc(h, &e.pos, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.pos_lo, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.vel, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.acc, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.pos_sorted, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.keys, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.keys_alt, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.perm, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.perm_alt, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.pairs, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.sums, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.box_lo, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.box_hi, S)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.bbox_min, 4 * (size_t)nsims)) != NB_OK) break;
    if ((rc = ens_alloc(h, &e.bbox_max, 4 * (size_t)nsims)) != NB_OK) break;
    e.status_tiles = (b + kSortTile - 1) / kSortTile;
    const size_t words = 8 * kSortRadix + 8 + (size_t)8 * e.status_tiles * kSortRadix;
    if ((rc = ens_alloc(h, &e.hist, words)) != NB_OK) break;
    e.tile_ctr = e.hist + 8 * kSortRadix;
    e.status = e.hist + 8 * kSortRadix + 8;
    if ((rc = ens_alloc(h, &e.err, 4)) != NB_OK) break;
    if ((rc = plan_build(sims.data(), nsims, h->plan)) != NB_OK) break;
    for (const SimDesc& d : sims) h->any_tree |= d.force == NB_FORCE_BH;
    plan_walk_queue(sims.data(), nsims, h->walk_items);
    for (int q = 0; q < 2; ++q) {
      int* d_items = nullptr;
      if ((rc = ens_alloc(h, &d_items, h->walk_items[q].size())) != NB_OK) break;
      e.walk_items[q] = d_items;
      e.walk_nitems[q] = (int)h->walk_items[q].size();
    }
    if (rc != NB_OK) break;
    if ((rc = ens_alloc(h, &e.walk_ctr, 2)) != NB_OK) break;
    h->ap_pool_f4 = plan_ens_allpairs(sims.data(), nsims, nullptr, h->ap);
    if (!h->ap.args.empty()) {
      EnsAllPairs& ap = h->ap;
      if ((rc = ens_alloc(h, &ap.d_pool, h->ap_pool_f4)) != NB_OK) break;
      if ((rc = ens_alloc(h, &ap.d_args, ap.args.size())) != NB_OK) break;
      if ((rc = ens_alloc(h, &ap.d_items, ap.items.size())) != NB_OK) break;
      if ((rc = ens_alloc(h, &ap.d_src_off, (size_t)nsims)) != NB_OK) break;
      if ((rc = ens_alloc(h, &ap.d_counter, 6)) != NB_OK) break;
    }
    {
      BuildRun* runs = nullptr;
      if ((rc = ens_alloc(h, &runs, h->plan.runs.size())) != NB_OK) break;
      e.runs = runs;
      const size_t segs = plan_seg_entries(b, nsims);
      for (int i = 0; i < 2; ++i) {
        if ((rc = ens_alloc(h, &e.seg[i], segs)) != NB_OK) break;
        if ((rc = ens_alloc(h, &e.seg_count[i], segs)) != NB_OK) break;
      }
      if (rc != NB_OK) break;
    }
    if ((rc = ens_alloc(h, &h->d_energy, 6 * (size_t)nsims)) != NB_OK) break;
    cudaError_t ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) { rc = set_error(NB_ERR_CUDA, cudaGetErrorString(ce)); break; }
    cudaStream_t st = h->stream;
    // defined contents everywhere: zero state in the gaps, in-range indices
    ce = cudaMemsetAsync(e.pos, 0, S * 16, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.pos_lo, 0, S * 16, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.vel, 0, S * 16, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.acc, 0, S * 16, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.perm, 0, S * 4, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.perm_alt, 0, S * 4, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.pairs, 0, S * sizeof(PairRec), st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.hist, 0, words * 4, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e.err, 0, 16, st);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(h->d_sims, sims.data(), sizeof(SimDesc) * nsims,
                           cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(h->d_blk, blk.data(), sizeof(int) * blk.size(),
                           cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && !h->plan.runs.empty())
      ce = cudaMemcpyAsync((void*)e.runs, h->plan.runs.data(),
                           sizeof(BuildRun) * h->plan.runs.size(), cudaMemcpyHostToDevice, st);
    size_t row = 0;
    for (int s = 0; s < nsims && ce == cudaSuccess; ++s) {
      ce = cudaMemcpyAsync(e.pos + h->base[s], pos4 + 4 * row, 16 * (size_t)n[s],
                           cudaMemcpyHostToDevice, st);
      if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(e.vel + h->base[s], vel4 + 4 * row, 16 * (size_t)n[s],
                             cudaMemcpyHostToDevice, st);
      row += n[s];
    }
    for (int q = 0; q < 2 && ce == cudaSuccess; ++q)
      if (!h->walk_items[q].empty())
        ce = cudaMemcpyAsync((void*)e.walk_items[q], h->walk_items[q].data(),
                             sizeof(int) * h->walk_items[q].size(), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && h->ap.d_pool)
      ce = cudaMemsetAsync(h->ap.d_pool, 0, sizeof(float4) * h->ap_pool_f4, st);
    if (ce != cudaSuccess) { rc = set_error(NB_ERR_CUDA, cudaGetErrorString(ce)); break; }
    if (!h->ap.args.empty() &&
        (rc = bind_ens_allpairs(h->ap, sims.data(), nsims, e, st)) != NB_OK) break;
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) { rc = set_error(NB_ERR_CUDA, cudaGetErrorString(ce)); break; }
  } while (0);
  if (rc != NB_OK) {
    std::string keep = last_error();
    ens_free(h);
    return set_error(rc, keep);
  }
  *out = h;
  return NB_OK;
}

int nb_ensemble_force(const nb_ensemble* h, int sim, int* force) {
  if (!h || !force) return set_error(NB_ERR_INVALID, "NULL argument");
  if (sim < 0 || sim >= h->nsims) return set_error(NB_ERR_INVALID, "simulation index out of range");
  *force = h->force[sim];
  return NB_OK;
}

int nb_ensemble_kernels_per_step(const nb_ensemble* h, int* kernels) {
  if (!h || !kernels) return set_error(NB_ERR_INVALID, "NULL argument");
  int k = 1;   // prep
  if (h->any_tree) {
    k += 1 + ens_sort_passes() + h->plan.levels;   // Morton keys, sort, build levels
    for (int q = 0; q < 2; ++q) k += h->walk_items[q].empty() ? 0 : 1;
  }
  if (!h->ap.groups.empty()) k += 1 + (int)h->ap.groups.size();   // pack + queues
  *kernels = k;
  return NB_OK;
}

int nb_ensemble_destroy(nb_ensemble* h) {
  ens_free(h);
  return NB_OK;
}

int nb_ensemble_size(const nb_ensemble* h, int* nsims, long long* particles) {
  if (!h) return set_error(NB_ERR_INVALID, "ensemble is NULL");
  if (nsims) *nsims = h->nsims;
  if (particles) {
    long long t = 0;
    for (int v : h->n) t += v;
    *particles = t;
  }
  return NB_OK;
}

int nb_ensemble_step(nb_ensemble* h, int nsteps) {
  if (!h) return set_error(NB_ERR_INVALID, "ensemble is NULL");
  if (nsteps < 0) return set_error(NB_ERR_INVALID, "nsteps must be >= 0");
  if (nsteps == 0) return NB_OK;
  if (!h->primed) {
    NB_TRY(ens_enqueue(h, true));   // a(x0) for every simulation
    h->primed = true;
  }
  for (int k = 0; k < nsteps; ++k) {
    if (h->use_graphs) {
      if (!h->graph) NB_TRY(ens_capture(h));
      NB_CUDA(cudaGraphLaunch(h->graph, h->stream));
    } else {
      NB_TRY(ens_enqueue(h, false));
    }
  }
  return NB_OK;
}

int nb_ensemble_set_graphs(nb_ensemble* h, int enable) {
  if (!h) return set_error(NB_ERR_INVALID, "ensemble is NULL");
  h->use_graphs = enable != 0;
  return NB_OK;
}

int nb_ensemble_sync(nb_ensemble* h) {
  if (!h) return set_error(NB_ERR_INVALID, "ensemble is NULL");
  NB_CUDA(cudaStreamSynchronize(h->stream));
  return ens_device_error(h);
}

int nb_ensemble_get_state(nb_ensemble* h, int sim, float* pos4, float* vel4) {
  if (!h) return set_error(NB_ERR_INVALID, "ensemble is NULL");
  if (sim < 0 || sim >= h->nsims) return set_error(NB_ERR_NOTFOUND, "no such simulation");
  const size_t bytes = 16 * (size_t)h->n[sim];
  if (pos4)
    NB_CUDA(cudaMemcpyAsync(pos4, h->e.pos + h->base[sim], bytes,
                            cudaMemcpyDeviceToHost, h->stream));
  if (vel4)
    NB_CUDA(cudaMemcpyAsync(vel4, h->e.vel + h->base[sim], bytes,
                            cudaMemcpyDeviceToHost, h->stream));
  NB_CUDA(cudaStreamSynchronize(h->stream));
  return ens_device_error(h);
}

int nb_ensemble_get_accelerations(nb_ensemble* h, int sim, float* acc4) {
  if (!h || !acc4) return set_error(NB_ERR_INVALID, "NULL argument");
  if (sim < 0 || sim >= h->nsims) return set_error(NB_ERR_NOTFOUND, "no such simulation");
  NB_CUDA(cudaMemcpyAsync(acc4, h->e.acc + h->base[sim], 16 * (size_t)h->n[sim],
                          cudaMemcpyDeviceToHost, h->stream));
  NB_CUDA(cudaStreamSynchronize(h->stream));
  return ens_device_error(h);
}

// e3: [nsims][3] = {E, KE, PE} per simulation (FP64 reductions).
int nb_ensemble_energy(nb_ensemble* h, double* e3) {
  if (!h || !e3) return set_error(NB_ERR_INVALID, "NULL argument");
  for (int s = 0; s < h->nsims; ++s) {
    const nb_params& p = h->params[s];
    NB_TRY(launch_energy(h->ews, h->n[s], h->e.pos + h->base[s], h->e.vel + h->base[s],
                         p.eps * p.eps, p.G, h->stream));
    NB_CUDA(cudaMemcpyAsync(h->d_energy + 6 * s, h->ews.eout, 6 * sizeof(double),
                            cudaMemcpyDeviceToDevice, h->stream));
  }
  std::vector<double> buf(6 * (size_t)h->nsims);
  NB_CUDA(cudaMemcpyAsync(buf.data(), h->d_energy, buf.size() * sizeof(double),
                          cudaMemcpyDeviceToHost, h->stream));
  NB_CUDA(cudaStreamSynchronize(h->stream));
  NB_TRY(ens_device_error(h));
  for (int s = 0; s < h->nsims; ++s)
    for (int c = 0; c < 3; ++c) e3[3 * s + c] = buf[6 * s + c];
  return NB_OK;
}

int nb_ensemble_record(nb_ensemble* h, int slot) {
  if (!h || slot < 0 || slot >= 16) return set_error(NB_ERR_INVALID, "bad slot");
  if (!h->slots[slot]) NB_CUDA(cudaEventCreate(&h->slots[slot]));
  NB_CUDA(cudaEventRecord(h->slots[slot], h->stream));
  return NB_OK;
}

int nb_ensemble_elapsed_ms(nb_ensemble* h, int a, int b, double* ms) {
  if (!h || !ms || a < 0 || b < 0 || a >= 16 || b >= 16 || !h->slots[a] || !h->slots[b])
    return set_error(NB_ERR_INVALID, "bad slot");
  NB_CUDA(cudaEventSynchronize(h->slots[b]));
  float f = 0.f;
  NB_CUDA(cudaEventElapsedTime(&f, h->slots[a], h->slots[b]));
  *ms = f;
  return NB_OK;
}

}  // extern "C"
