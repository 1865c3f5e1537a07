/*
 * nbody_b200.h -- C ABI of the B200-native nbodyssey force-and-step path.
 *
 * Plain C types only (pointers, sizes, POD structs).  Every function returns
 * an int status (NB_OK on success); nb_last_error() gives a thread-local
 * message for the last failure on the calling thread.  Host arrays passed in
 * are owned by the caller and copied; device state behind a handle is owned
 * by the library.  A handle may be used by one host thread at a time.
 *
 * Each entry point names the reference interface it replaces (paths within
 * the nbodyssey project).  The reference aborts the process on any CUDA error
 * (src/cuda_check.cuh:7-15) and on bad input (src/main.cu:28-31, 118-126);
 * here the same conditions return a status instead.
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NB_API __attribute__((visibility("default")))
#else
#define NB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NB_OK 0
#define NB_ERR_INVALID 1 /* bad argument: n, eps <= 0, theta < 0, key_bits, NULL */
#define NB_ERR_CUDA 2    /* a CUDA runtime call failed (message has the call) */
#define NB_ERR_DEVICE 3  /* a kernel raised its error word (see NB_DEVERR_*) */
#define NB_ERR_NOMEM 4   /* device allocation failed, or over the HBM budget */
#define NB_ERR_IO 5      /* file open / read / write failed, truncated file */
#define NB_ERR_STATE 6   /* call not valid in the object's current state */
#define NB_ERR_NOTFOUND 7 /* unknown request / simulation id */

/* bits of the device error word (NB_ERR_DEVICE) */
#define NB_DEVERR_STACK 1u  /* a tree walk's stack would have overflowed */
#define NB_DEVERR_SORT 2u   /* a radix-sort look-back wait hit its limit */
#define NB_DEVERR_WAIT 4u   /* a bulk-copy barrier wait hit its limit */
#define NB_DEVERR_QUEUE 8u  /* a persistent work-queue item was out of range (skipped) */
#define NB_DEVERR_TREE 16u  /* the centre-of-mass climb met an inconsistent tree */
#define NB_DEVERR_VISITS 32u /* a tree walk visited more nodes than the tree has */
#define NB_DEVERR_BOUNDS 64u /* a tree-build write outside its tree (skipped) */

/* ---- parameters (src/simulation.hpp:4-15: SimParams, ForceMethod,
 *      BhTraversal) ------------------------------------------------------- */
#define NB_FORCE_NAIVE 0      /* ForceMethod::kNaive, tiled all-pairs */
#define NB_FORCE_BH 1         /* ForceMethod::kBarnesHut, LBVH rebuilt per step */
#define NB_FORCE_AUTO 2       /* all-pairs below the tuned crossover, Barnes-Hut
                                 from there on (nb_tune_table; the default
                                 NB_AUTO_CROSSOVER is the B200 measurement) */
#define NB_AUTO_CROSSOVER 20000
#define NB_TRAVERSE_THREAD 0  /* BhTraversal::kThread, one walk per particle */
#define NB_TRAVERSE_WARP 1    /* BhTraversal::kWarp, one shared walk per warp */

typedef struct nb_params {
  float dt;            /* timestep (reference default 0.01, src/main.cu:25) */
  float eps;           /* Plummer softening length, > 0 (default 0.05) */
  float G;             /* gravitational constant (default 1) */
  float theta;         /* BH opening angle, >= 0; 0 = exact (default 0.5) */
  int32_t force;       /* NB_FORCE_* (default naive) */
  int32_t traverse;    /* NB_TRAVERSE_* (default thread) */
  int32_t key_bits;    /* Morton key width: 30 (10 bits/axis, uint32 keys) or
                          63 (21 bits/axis, the reference's width) */
  int32_t compensated; /* 1: positions kept as a hi/lo float pair through the
                          drift (forces use hi); 0: plain float drift */
  int32_t walk_kernel; /* 0: pair walk (default: a lane decides both children
                          of an opened node from its child-pair record);
                          1: depth-first walk, one node visit per step as the
                          reference kernels; 2: list walk (one candidate node
                          per lane).  All give the same interaction sets. */
} nb_params;

/* Fills the reference defaults: dt 0.01, eps 0.05, G 1, theta 0.5, naive,
 * thread, 30-bit keys, compensated drift on. */
NB_API void nb_params_default(nb_params* p);

NB_API const char* nb_last_error(void);
NB_API int nb_version(void);
/* Number of CUDA devices visible (0 on a machine without a GPU). */
NB_API int nb_device_count(int* out);
/* Device used by this thread's later calls (one process per GPU). */
NB_API int nb_set_device(int device);
/* Page-locked host buffers, for asynchronous host<->device copies. */
NB_API int nb_alloc_pinned(size_t bytes, void** out);
NB_API int nb_free_pinned(void* p);
/* Measures the FP32 FMA throughput of the current device with two
 * calibration kernels (scalar fma.rn.f32 and packed fma.rn.f32x2 chains over
 * all SMs); tflops = 2 * FMAs / time.  Used as the roofline denominator of
 * the FP32-pipe-bound force kernels. */
NB_API int nb_measure_fp32_peak(double* tflops_scalar, double* tflops_packed);

/* ======================================================================
 * Autotuning.  No reference counterpart (the reference has one fixed block
 * size, kForceBlock = 256 in src/forces.cuh:25, and a force module chosen by
 * hand, src/forces.cu:68-86).  Per device, a table of the all-pairs launch
 * shape per size, the Barnes-Hut walk's warps per block and the
 * all-pairs / Barnes-Hut crossover NB_FORCE_AUTO uses, measured on the device
 * at first use: the first nb_sim_create / nb_ensemble_create /
 * nb_server_create on a device loads the cache file
 * ($NBODY_B200_TUNE_CACHE, else ~/.cache/nbodyssey_b200/tune_<device>_<SMs>sm_v2.bin)
 * or, when there is none, measures the table (about a second) and writes
 * it.  NBODY_B200_TUNE=off keeps the defaults.  The device-pointer entry
 * points use the current table and never measure.  The shape decides only
 * the launch: the same table gives the same bits however it was obtained.
 * ==================================================================== */
#define NB_TUNE_VERSION 2
#define NB_TUNE_BUCKETS 16 /* size bucket b: n < 2^(10+b) (the last: any n) */
#define NB_TUNE_THETAS 3   /* crossover per theta class 0.3, 0.5, 0.7 */
typedef struct nb_tune_table {
  int32_t version;                      /* NB_TUNE_VERSION */
  int32_t sms;                          /* SMs of the device measured */
  char device[64];                      /* its name */
  int32_t ap_threads[NB_TUNE_BUCKETS];  /* all-pairs threads per CTA (128, 256) */
  int32_t ap_k[NB_TUNE_BUCKETS];        /* targets per thread (2, 4, 8) */
  int32_t ap_ctas[NB_TUNE_BUCKETS];     /* CTAs wanted in flight (sets the
                                           source split) */
  int32_t walk_warps;                   /* Barnes-Hut walk warps per block (2, 4, 8) */
  int32_t crossover[NB_TUNE_THETAS][2]; /* all-pairs below this many particles,
                                           per theta class and traversal
                                           (thread, warp) */
  int32_t crossover_batch[NB_TUNE_THETAS]; /* the same inside a batch
                                           (ensembles, the server): all-pairs
                                           vs Barnes-Hut cost per particle-step
                                           of equal-size simulations advanced
                                           together, per theta class */
} nb_tune_table;
/* Measures the table on the current device and installs it; writes it to
 * cache_path when non-NULL. */
NB_API int nb_autotune(const char* cache_path, nb_tune_table* out);
/* The current device's table (the defaults until one is measured / set). */
NB_API int nb_tune_get(nb_tune_table* out);
/* Installs a table for the current device (e.g. a choice made by hand). */
NB_API int nb_tune_set(const nb_tune_table* t);
/* The built-in defaults for the current device: 256 x 4 all-pairs shape,
 * 8 CTAs per SM in flight, 4 walk warps per block, crossover 20,000 alone and
 * 4,096 in a batch. */
NB_API int nb_tune_defaults(nb_tune_table* out);
/* Loads / saves a cache file (NULL: the default path).  nb_tune_load fails
 * with NB_ERR_NOTFOUND for a missing file or one measured on another kind of
 * device. */
NB_API int nb_tune_load(const char* path);
NB_API int nb_tune_save(const char* path);

/* ======================================================================
 * Handle API: one simulation whose state lives on the device.
 * ==================================================================== */
typedef struct nb_sim nb_sim;

/* ParticleSystem::allocate + upload (src/simulation.cu:4-20).  pos4 = n rows
 * of (x, y, z, m), vel4 = n rows of (vx, vy, vz, _), host memory. */
NB_API int nb_sim_create(int n, const float* pos4, const float* vel4,
                  const nb_params* p, nb_sim** out);
/* ParticleSystem::release + bh_release (src/simulation.cu:10-15,
 * src/forces_bh.cu:541-548). */
NB_API int nb_sim_destroy(nb_sim* s);
NB_API int nb_sim_n(const nb_sim* s, int* n);
NB_API int nb_set_params(nb_sim* s, const nb_params* p);
NB_API int nb_get_params(const nb_sim* s, nb_params* p);
/* Replace the state from host arrays (upload, src/simulation.cu:17-20). */
NB_API int nb_set_state(nb_sim* s, const float* pos4, const float* vel4);
/* ParticleSystem::download_positions (src/simulation.cu:22-24): n float4,
 * positions rounded to float (hi part), mass in w. */
NB_API int nb_get_positions(nb_sim* s, float* pos4);
NB_API int nb_get_velocities(nb_sim* s, float* vel4);
/* Low-order position parts (compensated mode; zeros otherwise). */
NB_API int nb_get_position_lo(nb_sim* s, float* lo4);
/* The acceleration buffer a(x) (after a step it holds a(x_new)). */
NB_API int nb_get_accelerations(nb_sim* s, float* acc4);
/* Upload a state together with its a(x), so the next step needs no priming
 * force evaluation (a host round trip of pos / vel / acc between steps). */
NB_API int nb_set_state_acc(nb_sim* s, const float* pos4, const float* vel4,
                            const float* acc4);
/* leapfrog_step (src/integrator.cuh:19) on host-resident state, for callers
 * that keep the state in host memory between steps: uploads pos / vel and
 * a(x), steps once, and writes the new pos / vel / a(x_new) to the out
 * buffers.  The positions are final after the drift and return to the host
 * on a second stream while the tree is built and walked.  Synchronous;
 * pinned host buffers (nb_alloc_pinned) give full PCIe speed.  Same results
 * as nb_set_state_acc + nb_step(1) + the three downloads. */
NB_API int nb_step_host(nb_sim* s, const float* pos4, const float* vel4,
                        const float* acc4, float* pos_out4, float* vel_out4,
                        float* acc_out4);

/* leapfrog_step (src/integrator.cuh:19) for callers that keep the state
 * (positions, velocities) in host memory: uploads pos / vel, steps once, and
 * writes the new pos / vel to the out buffers -- 64 bytes per particle
 * across PCIe instead of nb_step_host's 96.  a(x) and the low-order position
 * parts of the compensated drift stay on the device: they carry on when the
 * uploaded positions are bit for bit the ones this simulation holds (those
 * the previous call returned, checked on the device every call), so a caller
 * that hands each call's output back gets the trajectory of nb_step; other
 * positions start over as nb_set_state does (a(x) computed from them first).
 * Positions return on a second stream while the tree is built and walked.
 * Synchronous; pinned host buffers give full PCIe speed. */
NB_API int nb_step_host_state(nb_sim* s, const float* pos4, const float* vel4,
                              float* pos_out4, float* vel_out4);

/* compute_forces (src/forces.cuh:8, src/forces.cu:68-86): a(x) for the
 * current positions into the simulation's acceleration buffer, in original
 * particle order; copied to acc4 (host, n float4, w = 0) when non-NULL. */
NB_API int nb_compute_forces(nb_sim* s, float* acc4);
/* leapfrog_step x nsteps (src/integrator.cuh:19, src/integrator.cu:27-37):
 * kick, drift, forces, kick.  The first call after create / set_state first
 * computes a(x0) as src/main.cu:184 does.  Enqueued asynchronously on the
 * simulation's stream; errors of the kernels surface at the next sync. */
NB_API int nb_step(nb_sim* s, int nsteps);
/* Waits for the simulation's stream and checks the device error word. */
NB_API int nb_sync(nb_sim* s);
/* total_energy (src/integrator.cuh:21, src/integrator.cu:93-110), FP64
 * reductions: e3 = {E, KE, PE}; mom3 = total momentum (may be NULL). */
NB_API int nb_energy(nb_sim* s, double* e3, double* mom3);

/* Force timing (src/forces.cu:62-66, 88-90): CUDA-event time of every force
 * evaluation, accumulated when timing is on (off by default). */
NB_API int nb_set_timing(nb_sim* s, int enable);
NB_API int nb_force_timing(nb_sim* s, double* ms_total, long* calls);
NB_API int nb_reset_timing(nb_sim* s);
/* Per-phase times (bh_report_phase_timing, src/forces_bh.cu:529-539):
 * ms[NB_PHASES] accumulated over all timed steps, calls = steps timed. */
#define NB_PHASES 8
#define NB_PHASE_PREP 0     /* kick + drift + bounding box (+ source packing) */
#define NB_PHASE_MORTON 1
#define NB_PHASE_SORT 2
#define NB_PHASE_BUILD 3
#define NB_PHASE_COM 4
#define NB_PHASE_WALK 5     /* traversal, or the all-pairs force kernel */
#define NB_PHASE_ENERGY 6
#define NB_PHASE_OTHER 7
NB_API int nb_phase_times(nb_sim* s, double* ms, long* calls);

/* Events on the simulation's stream, for callers that time whole regions. */
NB_API int nb_record(nb_sim* s, int slot /* 0..15 */);
NB_API int nb_elapsed_ms(nb_sim* s, int slot0, int slot1, double* ms);

/* Use a captured CUDA graph for each step (default on).  The graph is
 * re-captured when the parameters change. */
NB_API int nb_set_graphs(nb_sim* s, int enable);
/* Enqueues a write of `bytes` (>= the 126 MB L2) to a scratch buffer on the
 * simulation's stream, evicting the state from L2 between timed steps. */
NB_API int nb_flush_l2(nb_sim* s, size_t bytes);

/* Debug / parity: run the tree build on the current positions and copy out
 * keys (uint64 per particle, sorted), the permutation (sorted -> original),
 * children [n-1][2], parent [2n-1], node com4 [n-1][4] and size2 [n-1].
 * Any pointer may be NULL. */
NB_API int nb_debug_lbvh(nb_sim* s, uint64_t* keys_sorted, uint32_t* perm,
                  int32_t* children, int32_t* parent, float* com4,
                  float* size2);
/* Debug / parity: the child-pair records of the tree built on the current
 * positions (the layout the tree walk reads), n - 1 records of 12 floats:
 * record k = (x_l, y_l, z_l, m_l, x_r, y_r, z_r, m_r, size2_l, w_l, size2_r,
 * w_r) for the two children of the internal node that splits after sorted
 * leaf k (left: node or leaf k, right: node or leaf k + 1); an internal
 * child gives its centre of mass, mass, squared box edge and split (w, the
 * bits of an int32), a leaf its position, mass, size2 = -1 and w = -1. */
NB_API int nb_debug_pairs(nb_sim* s, float* rec12);
/* Debug / parity: forces with per-particle interaction counts (original
 * order; warp mode counts the warp's shared walk for every lane). */
NB_API int nb_debug_forces(nb_sim* s, float* acc4, int32_t* counts);

/* compare_forces (src/main.cu:75-112): naive vs Barnes-Hut on the current
 * state, max and mean relative difference |a-b|/(|a|+1e-30). */
NB_API int nb_compare_forces(nb_sim* s, double* max_rel, double* mean_rel);

/* ======================================================================
 * Device-pointer API: drop-ins for the reference's C++ functions, operating
 * on caller-owned device arrays (float4 rows) on a caller-given stream
 * (cudaStream_t passed as void*; NULL = legacy default stream).  Scratch is
 * held by a workspace (the reference's process-global Scratch,
 * src/forces_bh.cu:50-69), grown only when n grows.
 * ==================================================================== */
typedef struct nb_workspace nb_workspace;
NB_API int nb_workspace_create(nb_workspace** out);
NB_API int nb_workspace_destroy(nb_workspace* w); /* bh_release */

/* compute_forces(sys, d_acc, p) (src/forces.cuh:8). */
NB_API int nb_compute_forces_dev(nb_workspace* w, int n, const float* d_pos4,
                          float* d_acc4, const nb_params* p, void* stream);
/* leapfrog_step(sys, d_acc, p) (src/integrator.cuh:19): plain float drift
 * (no low-order state); d_acc must hold a(x) on entry, a(x_new) on exit. */
NB_API int nb_leapfrog_step_dev(nb_workspace* w, int n, float* d_pos4, float* d_vel4,
                         float* d_acc4, const nb_params* p, void* stream);
/* No counterpart in the reference.  All-pairs accelerations (the same as
 * nb_compute_forces_dev with NB_FORCE_NAIVE) for callers that cannot
 * allocate device memory: the scratch lives in a fixed file-scope device
 * array (about 4.6 MB per GPU, held until exit), so the call allocates
 * nothing.  n must be <= 32768 (NB_ERR_INVALID otherwise).  The first call on
 * each device looks up the array's device address; make that first call
 * before any stream capture.  Calls share the array: calls whose GPU work
 * overlaps race and must be serialised by the caller.  Asynchronous on
 * `stream`: device-side failures are not in its return code.  If a block of
 * the kernel gives up waiting for its source tiles (NB_DEVERR_WAIT), its
 * acceleration rows are written as NaN, never left stale. */
NB_API int nb_compute_forces_naive_static(int n, const float* d_pos4,
                                          float* d_acc4, float eps, float G,
                                          void* stream);
/* No counterpart in the reference.  Device status of the last
 * nb_compute_forces_naive_static call on this device: waits for `stream`,
 * copies the call's error word (NB_DEVERR_* bits) into *device_error (may be
 * NULL) and returns NB_ERR_DEVICE when it is non-zero.  Allocates nothing;
 * the next nb_compute_forces_naive_static call clears the word. */
NB_API int nb_compute_forces_naive_static_status(unsigned* device_error,
                                                 void* stream);
/* No counterpart in the reference (one process drives one GPU there).  One
 * rank's share of compute_forces (src/forces.cuh:8) for a simulation split
 * over several GPUs: every rank holds the whole state and builds the whole
 * tree, then walks only the sorted targets [t0, t1) (t0 and t1 multiples of
 * 32, or n) and writes d_part4[t - t0] = a of sorted target t.  With
 * d_vel4 set, the opening kick (by d_acc4 = a(x)) and the drift of every
 * particle run first, as in nb_leapfrog_step_dev; d_pos_lo4 (or NULL) holds
 * the low-order position parts of the compensated drift.  Barnes-Hut only
 * (NB_FORCE_BH, or NB_FORCE_AUTO that resolves to it).  Asynchronous. */
NB_API int nb_forces_range_dev(nb_workspace* w, int n, float* d_pos4,
                               float* d_pos_lo4, float* d_vel4,
                               const float* d_acc4, float* d_part4,
                               const nb_params* p, int t0, int t1, void* stream);
/* Completes a split step once the ranks' parts are concatenated in sorted
 * order (d_sorted4, n rows): d_acc4[perm[t]] = d_sorted4[t] with the
 * permutation of this workspace's last nb_forces_range_dev call, and with
 * d_vel4 set the closing kick.  Bit-identical to the unsplit step.
 * Asynchronous. */
NB_API int nb_forces_gather_dev(nb_workspace* w, int n, const float* d_sorted4,
                                float* d_acc4, float* d_vel4, const nb_params* p,
                                void* stream);
/* total_energy(sys, p) (src/integrator.cuh:21): synchronous, e3 on host. */
NB_API int nb_total_energy_dev(nb_workspace* w, int n, const float* d_pos4,
                        const float* d_vel4, const nb_params* p, double* e3,
                        void* stream);

/* ======================================================================
 * Ensembles: many independent simulations advanced together, one set of
 * launches per step for all of them (captured as one CUDA graph).  No
 * reference counterpart (the reference runs one simulation per process);
 * each simulation's results are bit-identical to running it alone through
 * the handle API with the same parameters.  Barnes-Hut, 30-bit keys.
 * ==================================================================== */
typedef struct nb_ensemble nb_ensemble;
/* n[nsims] particle counts; pos4 / vel4 hold all simulations' rows back to
 * back (sum of n rows); params[nsims], one per simulation (dt, eps, G, theta,
 * traverse, compensated may differ).  nsims <= 1023. */
NB_API int nb_ensemble_create(int nsims, const int* n, const float* pos4,
                              const float* vel4, const nb_params* params,
                              nb_ensemble** out);
NB_API int nb_ensemble_destroy(nb_ensemble* e);
NB_API int nb_ensemble_size(const nb_ensemble* e, int* nsims, long long* particles);
/* nsteps leapfrog steps of every simulation (a(x0) first, once). */
NB_API int nb_ensemble_step(nb_ensemble* e, int nsteps);
NB_API int nb_ensemble_sync(nb_ensemble* e);
NB_API int nb_ensemble_set_graphs(nb_ensemble* e, int enable);
NB_API int nb_ensemble_get_state(nb_ensemble* e, int sim, float* pos4, float* vel4);
NB_API int nb_ensemble_get_accelerations(nb_ensemble* e, int sim, float* acc4);
/* e3[nsims][3] = {E, KE, PE} of every simulation, FP64 reductions. */
NB_API int nb_ensemble_energy(nb_ensemble* e, double* e3);
/* The force module simulation `sim` runs with (NB_FORCE_NAIVE or
 * NB_FORCE_BH): NB_FORCE_AUTO resolves by the tuning table's crossover inside
 * a batch (crossover_batch), not the one a simulation gets alone. */
NB_API int nb_ensemble_force(const nb_ensemble* e, int sim, int* force);
/* Kernel launches of one ensemble step (prep, the tree pipeline when some
 * simulation uses Barnes-Hut, the all-pairs packing and queue launches when
 * some uses all-pairs). */
NB_API int nb_ensemble_kernels_per_step(const nb_ensemble* e, int* kernels);
NB_API int nb_ensemble_record(nb_ensemble* e, int slot /* 0..15 */);
NB_API int nb_ensemble_elapsed_ms(nb_ensemble* e, int slot0, int slot1, double* ms);

/* ======================================================================
 * Request server with continuous batching.  No reference counterpart.
 * Requests (a simulation state, parameters, a step count, a frame cadence)
 * are admitted in arrival order whenever their footprint fits the free part
 * of a slot pool sized by an HBM budget (later requests may pass one that
 * does not fit yet); all running simulations advance together, one set of
 * launches per step, and state and trees stay on the device until a request
 * finishes.  Frames (every dump_every-th step, as src/main.cu:188) stream to
 * the host on a side stream and, with out_dir, to out_dir/frame_%05d.bin.
 * Each result is bit-identical to running the request alone.  Barnes-Hut,
 * 30-bit keys.
 * ==================================================================== */
typedef struct nb_server nb_server;
typedef struct nb_server_stats {
  long long completed, failed, queued, running, engine_steps;
  double particle_steps;     /* sum over steps of the particles advanced */
  long long frames, frame_bytes;
  double busy_s;             /* host time from the first to the last step */
  int peak_running;
  long long capacity_slots, used_slots;
} nb_server_stats;
/* hbm_budget_bytes sizes the slot pool (about 224 bytes per particle slot);
 * max_sims <= 1023 simulations run at once. */
NB_API int nb_server_create(size_t hbm_budget_bytes, int max_sims, nb_server** out);
/* Stops after the running and queued requests are abandoned; frees all. */
NB_API int nb_server_destroy(nb_server* s);
NB_API int nb_server_submit(nb_server* s, int n, const float* pos4, const float* vel4,
                            const nb_params* p, int steps, int dump_every,
                            const char* out_dir, long long* id);
/* state: 0 queued, 1 running, 2 done, 3 failed; seconds since the server
 * started (admit / done are 0 until they happen). */
NB_API int nb_server_poll(nb_server* s, long long id, int* state, double* t_submit,
                          double* t_admit, double* t_done);
NB_API int nb_server_wait(nb_server* s, long long id, double timeout_s);
NB_API int nb_server_result(nb_server* s, long long id, float* pos4, float* vel4,
                            int release);
NB_API int nb_server_get_stats(nb_server* s, nb_server_stats* out);
/* The force module request `id` runs with (NB_FORCE_NAIVE or NB_FORCE_BH;
 * AUTO resolved by the batch crossover, as in ensembles). */
NB_API int nb_server_force(nb_server* s, long long id, int* force);

/* ======================================================================
 * Files and the run loop (src/main.cu:115-215, docs/FORMATS.md).
 * ==================================================================== */
/* load_ic (src/main.cu:115-128).  Call with pos4 = vel4 = NULL to get n. */
NB_API int nb_read_ic(const char* path, int* n, float* pos4, float* vel4);
NB_API int nb_write_ic(const char* path, int n, const float* pos4, const float* vel4);
/* State files (checkpoint / resume; the reference has none, its runs restart
 * only from an ic.bin).  The file is the ic.bin layout of docs/FORMATS.md:8-16
 * (int32 n, float4 pos[n], float4 vel[n]) -- any ic.bin reader, load_ic
 * (src/main.cu:115-128) included, takes it as initial conditions -- followed
 * by a trailer: the magic "NBSTATE1", int32 flags (NB_STATE_*), the run's
 * nb_params, float4 pos_lo[n] (low-order position parts of the compensated
 * drift) and float4 acc[n] (a(x) of the stored positions).  A run resumed
 * from it continues bit for bit as if it had not stopped. */
#define NB_STATE_TRAILER 1 /* the trailer is present (0: a plain ic.bin) */
#define NB_STATE_ACC 2     /* acc[] holds a(x) of the stored positions */
#define NB_STATE_LO 4      /* pos_lo[] holds low-order position parts */
NB_API int nb_write_state_file(const char* path, int n, const float* pos4,
                               const float* vel4, const float* lo4,
                               const float* acc4, const nb_params* p);
/* Call with pos4 = vel4 = NULL to get n.  A plain ic.bin gives flags = 0,
 * zero lo4 / acc4 and leaves *p unchanged.  lo4, acc4, p, flags may be NULL. */
NB_API int nb_read_state_file(const char* path, int* n, float* pos4, float* vel4,
                              float* lo4, float* acc4, nb_params* p, int* flags);
/* Writes the simulation's state (positions with their low-order parts,
 * velocities, a(x) when it is current, parameters) as a state file. */
NB_API int nb_save_state(nb_sim* s, const char* path);
/* Replaces the simulation's state from a state file (n must match) and takes
 * its parameters; with a(x) stored the next step needs no priming force
 * evaluation.  A plain ic.bin loads like nb_set_state. */
NB_API int nb_load_state(nb_sim* s, const char* path);
/* dump_frame (src/main.cu:130-138): <dir>/frame_%05d.bin. */
NB_API int nb_write_frame(const char* dir, int index, int n, const float* pos4);
/* One energy-log row, "%d,%.5f,%.8e,%.8e,%.8e,%.3e\n" with time = step*dt
 * in float and rel = (E - E0)/|E0| (src/main.cu:172-178).  Host only. */
NB_API int nb_format_energy_row(char* buf, size_t cap, int step, float dt, double e,
                         double ke, double pe, double e0);

typedef struct nb_run_stats {
  double wall_s;        /* host wall time of the loop */
  double force_ms;      /* CUDA-event time of the force evaluations */
  long force_calls;
  int frames;           /* frames written */
  double e0, e_final, rel_final;
  double phase_ms[NB_PHASES]; /* per-phase time per step (timing mode) */
} nb_run_stats;
/* The main loop of src/main.cu:140-215: E0, a(x0), then per step a
 * leapfrog step; after every step with step % dump_every == 0 a frame
 * (frame_%05d.bin, numbered from 0) and an energy row; a final row at
 * `steps`.  Frames leave the device on a side stream into pinned buffers and
 * are written by a host thread while the next steps run.  out_dir / csv may
 * be NULL to skip frames / the log.  `timing` turns on the phase timers. */
NB_API int nb_run(nb_sim* s, int steps, int dump_every, const char* out_dir,
           const char* energy_csv, int timing, nb_run_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* NBODY_B200_H */
