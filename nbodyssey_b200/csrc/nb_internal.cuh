// Internal declarations shared by the kernel files and the C ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/nbody_b200.h"

namespace nb {

// ---------------------------------------------------------------------------
// Error handling: every host entry point returns a status; the message for
// the calling thread is kept in a thread-local string.
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
const char* last_error();

#define NB_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return ::nb::set_error(NB_ERR_CUDA, std::string(#call) + ": " +        \
                                              cudaGetErrorString(e_));       \
  } while (0)

#define NB_TRY(expr)            \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != NB_OK) return rc_; \
  } while (0)

// ---------------------------------------------------------------------------
// Layouts in HBM
// ---------------------------------------------------------------------------
// One internal LBVH node, 32 bytes: one sector per fetch in the walks.
struct __align__(16) Node {
  float4 com;     // centre of mass (x, y, z) and mass (w)
  int left;       // child ids: internal [0, n-2], leaf i -> n-1+i
  int right;
  float size2;    // (longest edge of the node's tight box)^2
  int pad;
};

// Child pairs for the tree walk, one record per split k in [0, n-2]: the two
// children of the internal node that splits its leaves after leaf k (the left
// child is internal node k or leaf k, the right child internal node k+1 or
// leaf k+1).  c[j] = (x, y, z, m): the centre of mass and mass of an internal
// child, the position and mass of a leaf; sw = (size2_l, w_l, size2_r, w_r):
// size2 the squared longest edge of an internal child's box (-1 for a leaf,
// which every opening test accepts) and w the split of an internal child,
// where its own children are recorded (-1 for a leaf).  The tree build writes
// each child's half (one 16-byte and one 8-byte store) when it finishes the
// child.  The root, the one node that is nobody's child, has its own record
// at k = n - 1: c[0] its centre of mass and mass, sw.x its size2, sw.y its
// split.  The Barnes-Hut walks of the pair layout need nothing else from the
// tree; the Node records are written only for the walks that read them.
struct __align__(16) PairRec {
  float4 c[2];
  float4 sw;
};

// Walks keep their per-warp / per-thread stacks this deep.  A radix tree over
// 63-bit keys with index tie-breaks is at most 63 + 31 levels deep and the
// stack grows by at most one entry per level; an overflow raises
// NB_DEVERR_STACK instead of writing past the stack.
constexpr int kStack = 128;

// Onesweep sort geometry.
// 512 threads (the first 256 own one digit each in the per-digit steps),
// 8 keys per thread, 2 CTAs per SM: at 1M keys a pass is one wave of 245
// tiles.  A tile's latency and the look-back's prefix propagation through
// the tiles, not bandwidth, set the pass time; this geometry measured best
// against 256 threads with 4096 or 2048 keys and 1024 keys per tile.
constexpr int kSortThreads = 512;
constexpr int kSortItems = 8;
constexpr int kSortCtasPerSm = 2;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kSortRadix = 256;

// All-pairs source layout: particles are packed in pairs as two float4,
// (x0, x1, y0, y1) and (z0, z1, m0, m1), padded with zero-mass particles to a
// multiple of kSrcTile particles.
constexpr int kSrcTile = 512;

inline int sort_passes(int key_bits) { return (key_bits + 7) / 8; }

// Workspace: scratch of the force modules, grown only when n grows (the
// reference's Scratch, src/forces_bh.cu:50-121).
struct Workspace {
  int cap = 0;          // particles
  int key_bits = 0;     // layout the sort buffers were sized for
  // tree
  void* keys = nullptr;       // u32 or u64 [cap]
  void* keys_alt = nullptr;
  uint32_t* vals = nullptr;   // [cap]
  uint32_t* vals_alt = nullptr;
  float4* pos_sorted = nullptr;   // [cap]
  Node* nodes = nullptr;          // [cap-1]
  PairRec* pairs = nullptr;       // [cap] child pairs by split + the root's
  int* parent = nullptr;          // [2cap-1]
  int2* seg[2] = {nullptr, nullptr};      // open splits per build CTA,
  int* seg_count[2] = {nullptr, nullptr}; // ping-pong between levels
  double4* sums = nullptr;        // [cap-1] FP64 mass-weighted sums
  float4* box_lo = nullptr;       // [cap-1]
  float4* box_hi = nullptr;       // [cap-1]
  // sort
  uint32_t* hist = nullptr;       // [8][256] digit counts per pass
  uint32_t* status = nullptr;     // [8][tiles][256] look-back words
  uint32_t* tile_ctr = nullptr;   // [8] tile tickets
  int status_tiles = 0;
  // bounding box (ordered ints: lo xyz, hi xyz) + per-block partials
  int* bbox = nullptr;            // [8]
  int* bbox_part = nullptr;       // [kPrepMaxBlocks][6]
  unsigned* bbox_ticket = nullptr;
  // all-pairs
  float4* src = nullptr;          // packed sources [2 * cap_pad/2]
  int src_cap = 0;
  float4* part = nullptr;         // j-split partials [jsplit][cap]
  int part_cap = 0;               // elements
  unsigned* tickets = nullptr;    // per i-tile tickets
  int tickets_cap = 0;
  // energy
  double* epart = nullptr;        // per-block partials [blocks][6]
  int epart_cap = 0;
  double* ephi = nullptr;         // j-split phi partials [jsplit][cap]
  int ephi_cap = 0;
  double* eout = nullptr;         // [8]
  unsigned* eticket = nullptr;    // last-block ticket of the energy reduce
  double* h_eout = nullptr;       // pinned
  // debug counters
  int* counts = nullptr;          // [cap] interactions per sorted target
  // error word
  unsigned* err = nullptr;
  unsigned* h_err = nullptr;      // pinned
};

constexpr int kPrepThreads = 256;
constexpr int kPrepMaxBlocks = 1024;

int ws_reserve(Workspace& w, int n, int key_bits);
struct APGeom;
int ws_reserve_allpairs(Workspace& w, int n, const APGeom& g);
int ws_reserve_energy(Workspace& w, int n, int blocks, int jsplit);
void ws_free(Workspace& w);

// ---------------------------------------------------------------------------
// Launchers (kernel files).  All enqueue on `st`; none synchronise.
// ---------------------------------------------------------------------------
struct StepArgs {
  int n;
  float4* pos;      // hi (x, y, z, m), original order
  float4* pos_lo;   // lo parts or nullptr (plain drift)
  float4* vel;      // nullptr: no kick / drift
  float4* acc;      // out: a(x), original order
  float half_dt, dt;
  float eps2, G, theta2;
  int key_bits;
  int traverse;
  int walk_kernel;  // 0 pair walk, 1 depth-first walk, 2 list walk
  // the tree build also writes the Node records and parent links (walk
  // kernels 1 and 2 read them, nb_debug_lbvh returns them)
  bool node_records = false;
  bool kick_drift;  // opening kick + drift before the force evaluation
  bool kick_after;  // closing kick fused into the force epilogue
  int* counts;      // debug: interactions per sorted target, or nullptr
  // Barnes-Hut: the walk covers sorted targets [t0, t1); with `part` set it
  // writes part[t - t0] = a of sorted target t (no kick) instead of `acc`
  int t0, t1;
  float4* part;
  cudaEvent_t after_prep;   // recorded after the prep kernel, or nullptr
};

// prep: [kick + drift] [+ bbox] [+ pack all-pairs sources] [+ zero sort scratch]
int launch_prep(Workspace& w, const StepArgs& a, bool bbox, bool pack,
                cudaStream_t st);
int launch_morton(Workspace& w, const StepArgs& a, cudaStream_t st);
int launch_sort(Workspace& w, const StepArgs& a, cudaStream_t st);
size_t build_seg_entries(int cap);
int launch_build(Workspace& w, const StepArgs& a, cudaStream_t st);
int launch_com(Workspace& w, const StepArgs& a, cudaStream_t st);
int launch_walk(Workspace& w, const StepArgs& a, cudaStream_t st);
// acc[perm[t]] = sorted[t] (+ the closing kick when a.vel is set); the
// permutation of the workspace's last tree, or the identity without one
int launch_gather_part(Workspace& w, const StepArgs& a, const float4* sorted,
                       bool use_perm, cudaStream_t st);
int launch_allpairs(Workspace& w, const StepArgs& a, cudaStream_t st);
// energy: {E, KE, PE, Px, Py, Pz} into w.eout (device); positions hi (+lo
// for the kinetic part is not needed).
int launch_energy(Workspace& w, int n, const float4* pos, const float4* vel,
                  float eps2, float G, cudaStream_t st);
int launch_flush(void* buf, size_t bytes, cudaStream_t st);
// Streaming multiprocessors of the current device (read once per device;
// 148 on a B200), for grid sizes that should fill the device.
int device_sm_count();
// *diff becomes non-zero when the n float4 rows of a and b differ in any bit
// (*diff zeroed by the caller)
int launch_differ(const float4* a, const float4* b, int n, unsigned* diff, cudaStream_t st);
int measure_fp32_peak(double* tflops_scalar, double* tflops_packed);

// Kernel warm-up.  With lazy module loading (the CUDA 12 default) a kernel's
// code is loaded at its first launch, a host stall of up to milliseconds that
// a stream's timing events then count as device time.  warm_kernels() loads
// every kernel of the force-and-step path on the current device once per
// process (the handle query loads the function); the first simulation,
// ensemble or server created on a device calls it.  warm_fn queries one
// kernel; each source file lists its own kernels.
template <typename F>
inline int warm_fn(F* kernel) {
  cudaFuncAttributes fa;
  const cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kernel));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(NB_ERR_CUDA, std::string("loading a kernel: ") + cudaGetErrorString(e));
  }
  return NB_OK;
}
inline int warm_fns() { return NB_OK; }
template <typename F, typename... R>
inline int warm_fns(F* kernel, R*... rest) {
  NB_TRY(warm_fn(kernel));
  return warm_fns(rest...);
}
// Programmatic dependent launch along the one-simulation Barnes-Hut chain
// (Morton keys, sort passes, build levels, walk).  A kernel launched with
// launch_chained may be scheduled while the kernel before it in the stream
// is still running: it calls chain_wait() before its first memory access
// (griddepcontrol.wait returns once the predecessor grid has completed and
// its writes are visible; in a kernel launched without the attribute it
// returns at once), and each kernel of the chain calls chain_release() at
// its start, which lets its successor's CTAs be scheduled once all of its
// own CTAs are running.  What overlaps is launch and CTA set-up, never data.
// Only eager launches carry the attribute: measured on a B200, the chain
// gains 2-4 % launched kernel by kernel, and a captured step graph with
// programmatic edges ran slower than the plain graph (13 % at N = 100,000,
// equal at 1M), so launches under stream capture stay plain.
__device__ __forceinline__ void chain_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void chain_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline int launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                          cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    cs = cudaStreamCaptureStatusNone;
  }
  cfg.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
  NB_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
  return NB_OK;
}

int warm_kernels();
int warm_prep_kernels();
int warm_lbvh_kernels();
int warm_walk_kernels();   // calls the two below
int warm_walk_pair_kernels();
int warm_walk_list_kernels();
int warm_allpairs_kernels();

// Arguments of the all-pairs kernel (one simulation).
struct APArgs {
  int n;
  const float4* __restrict__ pos;
  const float4* __restrict__ src;   // packed sources, npad particles
  int npad;
  int jsplit;
  int jchunk;                       // particles per j-chunk (multiple of tile)
  float eps2, G, half_dt;
  float4* acc;
  float4* vel;                      // closing kick or nullptr
  float4* part;                     // [jsplit][n] partials
  unsigned* tickets;                // [itiles]
  unsigned* err;
};

// The persistent all-pairs launch over many simulations' work items.
struct APQueue {
  const APArgs* sims;     // per-simulation arguments (pointers into its slots)
  const int4* items;      // (simulation, target tile, source chunk, -)
  int nitems;
  int* counter;           // next item; zeroed before the launch
  int kick;               // closing kick of the simulations that step
  int nsims;              // entries of `sims`
  unsigned* err;          // NB_DEVERR_QUEUE: an item out of range (skipped)
};

// all-pairs launch geometry
struct APGeom {
  int threads;   // per CTA
  int k;         // targets per thread
  int jsplit;    // CTAs along j per i-tile
  int itiles;
};
// the tuning table's geometry for n particles on the current device
APGeom allpairs_geometry(int n);
// a given shape with about `ctas` CTAs in flight
APGeom allpairs_geometry_for(int n, int threads, int k, int ctas);
bool allpairs_shape_compiled(int threads, int k);
int launch_allpairs_geom(Workspace& w, const StepArgs& a, const APGeom& g,
                         cudaStream_t st);

// ---------------------------------------------------------------------------
// Tuning table (tune.cu): per device, measured on it at first use or loaded
// from its cache file.
// ---------------------------------------------------------------------------
// all-pairs shape and CTAs in flight for n particles
void tune_allpairs(int n, int* threads, int* k, int* ctas);
// Barnes-Hut walk: warps per block
int tune_walk_warps();
// NB_FORCE_AUTO: all-pairs below this many particles, Barnes-Hut from there
int tune_crossover(float theta, int traverse);
// resolves NB_FORCE_AUTO for n particles (other methods pass through)
int resolve_force_tuned(int force, int n, float theta, int traverse);
// the same for a simulation inside a batch (ensembles, the server)
int resolve_force_batch(int force, int n, float theta);
// first use on the current device: load the cache file or measure the table
// (never while `st` is capturing); idempotent
int tune_ensure(cudaStream_t st);
// the whole force evaluation of one step (api.cu)
struct PhaseMarks;
int enqueue_forces(Workspace& w, const StepArgs& a, int force, cudaStream_t st,
                   PhaseMarks* pm);

// ---------------------------------------------------------------------------
// Ensembles: many simulations in one set of arrays.  Simulation s owns slots
// [base, base + n) of every per-particle array (original order for the
// state, Morton order for the sorted arrays and its tree: internal node i at
// base + i, parent entries at 2 base + id); bases are multiples of 32, so a
// 32-slot block (one warp) belongs to at most one simulation.  Slots between
// simulations are unused.
// ---------------------------------------------------------------------------
struct SimDesc {
  int n;          // particles
  int base;       // first slot, a multiple of 32
  int coff;       // particles of the simulations before this one
  int traverse;   // NB_TRAVERSE_*
  float half_dt, dt, eps2, G, theta2;
  int active;     // 0: skipped; 1: stepped; 2: a(x) only (newly admitted)
  int compensated;
  int force;      // NB_FORCE_BH (tree pipeline) or NB_FORCE_NAIVE (all-pairs)
};

constexpr int kEnsSimBits = 10;                     // sim id field of the keys
constexpr int kEnsMaxSims = (1 << kEnsSimBits) - 1; // id 1023 marks unused slots
constexpr int kEnsKeyBits = 30 + kEnsSimBits;       // 40 bits, 5 sort passes
int ens_sort_passes();

// One CTA of a multi-tree build level.
struct BuildRun {
  int sim;        // simulation (index into the SimDesc table)
  int group;      // its group at this level
  int in_first;   // first segment of the level below (later levels)
  int in_count;   // segments it merges
  int out;        // 1: hands its open splits to the next level
};

constexpr int kBuildMaxLevels = 8;

// Host plan: the runs of every level back to back.
struct BuildPlan {
  int levels = 0;
  int offset[kBuildMaxLevels] = {};
  int count[kBuildMaxLevels] = {};
  std::vector<BuildRun> runs;
};

struct EnsArgs {
  int nsims;
  int nslots;                 // slot extent (multiple of 32)
  int nblocks;                // nslots / 32
  const SimDesc* sims;
  const int* blk_sim;         // [nblocks] simulation of each 32-slot block, -1
  float4* pos;                // state, original order, [nslots]
  float4* pos_lo;
  float4* vel;
  float4* acc;
  float4* pos_sorted;         // [nslots]
  uint64_t* keys;             // [nslots] x2: (sim << 30) | morton30
  uint64_t* keys_alt;
  uint32_t* perm;             // [nslots] x2: original slot of each sorted slot
  uint32_t* perm_alt;
  PairRec* pairs;             // [nslots] child pairs by split + each root's
  double4* sums;              // [nslots]
  float4* box_lo;
  float4* box_hi;
  int* bbox_min;              // [nsims][4] ordered ints
  int* bbox_max;              // [nsims][4]
  uint32_t* hist;             // [8][256] + tile counters + look-back words
  uint32_t* tile_ctr;
  uint32_t* status;
  int status_tiles;
  unsigned* err;
  bool kick_drift;
  bool kick_after;
  const BuildRun* runs;       // tree-build plan (all levels)
  int2* seg[2];               // open splits between build levels
  int* seg_count[2];
  // the Barnes-Hut walk's work queue: per semantics (0 warp, 1 thread) the
  // 32-slot blocks to walk, costliest first, and a counter each (zeroed by
  // the launcher every step)
  const int* walk_items[2];
  int walk_nitems[2];
  int* walk_ctr;
};

// All-pairs work of the simulations of a batch that use the all-pairs
// module (k_allpairs.cu): each has a region of a float4 pool holding its
// packed sources, its partials and its tile tickets, its own launch geometry
// (the one it gets alone, so its sums and results are the same), and the
// queue items of one persistent launch per launch shape.
struct EnsAllPairs {
  struct Group {
    int threads, k, first_item, nitems;
  };
  std::vector<APArgs> args;    // per all-pairs simulation
  std::vector<int> sim;        // its index in the simulation table
  std::vector<size_t> region;  // its region offset in the pool (float4)
  std::vector<int4> items;     // (all-pairs simulation, target tile, chunk, -)
  std::vector<Group> groups;
  std::vector<int> src_off;    // per simulation: pool offset of its packed
                               // sources, -1 for one without all-pairs work
  // device (owned by the batch)
  float4* d_pool = nullptr;
  APArgs* d_args = nullptr;
  int4* d_items = nullptr;
  int* d_src_off = nullptr;    // [nsims]
  int* d_counter = nullptr;    // [6] one per launch shape
};
// Pool float4 of one simulation's region (sources, partials, tickets); its
// sources come first and must start zeroed, its tickets too.
size_t ap_region_f4(int n);
// Host plan of the simulations whose SimDesc.force is NB_FORCE_NAIVE and that
// are active: geometry, items, and the region of simulation s at
// region_of[s] (nullptr: back to back from 0).  With region_cap, a simulation
// whose geometry now needs more than region_cap[s] float4 (the tuning table
// changed since its region was sized) is left out and counted in *too_small.
// Returns the pool size used.
size_t plan_ens_allpairs(const SimDesc* sims, int nsims, const size_t* region_of,
                         EnsAllPairs& ap, const size_t* region_cap = nullptr,
                         int* too_small = nullptr);
// Points the per-simulation arguments at the batch's arrays and the pool and
// uploads them with the items and source offsets (stream-ordered; the host
// vectors must live until the copies ran).
int bind_ens_allpairs(EnsAllPairs& ap, const SimDesc* sims, int nsims, const EnsArgs& e,
                      cudaStream_t st);
// Packs the all-pairs simulations' sources, then the queue launches.
int launch_ens_allpairs(const EnsArgs& e, const EnsAllPairs& ap, cudaStream_t st);

int launch_ens_prep(const EnsArgs& e, cudaStream_t st);
int launch_ens_morton(const EnsArgs& e, cudaStream_t st);
int launch_ens_sort(EnsArgs& e, cudaStream_t st);   // updates e.keys / e.perm
// Tree build of all simulations (k_lbvh.cu): a host plan of level runs,
// uploaded to e.runs, then one launch per level.
int plan_build(const SimDesc* sims, int nsims, BuildPlan& plan);
size_t plan_seg_entries(int slots, int nsims);
int launch_ens_levels(const EnsArgs& e, const BuildPlan& plan, cudaStream_t st);
int launch_walk_pair_ens(const EnsArgs& e, cudaStream_t st);
// Host: the walk queue of a simulation table (the Barnes-Hut simulations'
// 32-slot blocks per semantics, costliest simulation first: larger n and
// smaller theta walk longer); items[0] / items[1] get the warp / thread
// semantics' blocks.
void plan_walk_queue(const SimDesc* sims, int nsims, std::vector<int> items[2]);

// A view of a simulation handle's device state (defined in api.cu) for the
// run loop in io.cu.
struct SimView {
  int n;
  cudaStream_t stream;
  float4* pos;
  float4* vel;
  Workspace* ws;
  nb_params p;
};
}  // namespace nb
struct nb_sim;
namespace nb {
int sim_view(nb_sim* s, SimView* v);

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int f2ord(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord2f(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

__device__ __forceinline__ void raise_err(unsigned* err, unsigned bit) {
  atomicOr(err, bit);
}

// rsqrt on the special-function unit (approximate, as the reference's
// fast-math rsqrtf).
__device__ __forceinline__ float mufu_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

}  // namespace nb
