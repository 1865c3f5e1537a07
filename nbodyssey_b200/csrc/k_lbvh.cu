// LBVH build, rebuilt every step (src/forces_bh.cu:190-331):
//   Morton keys (+ the radix sort's digit histograms, fused)
//   onesweep LSD radix sort (+ the position gather, fused into the last pass)
//   Karras radix tree + bottom-up centres of mass / boxes / sizes (FP64
//   mass-weighted sums): one fused bottom-up build in levels, for a single
//   tree or for all the trees of an ensemble at once.
#include <cuda/atomic>

#include "nb_internal.cuh"

namespace nb {

// ---------------------------------------------------------------------------
// Morton keys.  Quantisation in IEEE round-to-nearest float32 with a
// correctly rounded reciprocal, so the keys are bit-identical to the CPU
// mirror (scripts/lbvh_check.py:45-54 on float32 input).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__device__ __forceinline__ uint64_t spread21(uint32_t x) {
  uint64_t v = x & 0x1fffffu;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint32_t quantise(float p, float lo, float inv,
                                             float scale, float qmax) {
  float t = __fmul_rn(__fsub_rn(p, lo), inv);
  return (uint32_t)fminf(__fmul_rn(fmaxf(t, 0.f), scale), qmax);
}

constexpr int kMortonThreads = 1024;

template <typename K>
__global__ void __launch_bounds__(kMortonThreads) k_morton(const float4* __restrict__ pos,
                                                int n, const int* __restrict__ bbox,
                                                K* keys, uint32_t* hist, int passes) {
  chain_release();
  chain_wait();
  __shared__ uint32_t s_hist[8 * kSortRadix];
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  const float lx = ord2f(bbox[0]), ly = ord2f(bbox[1]), lz = ord2f(bbox[2]);
  const float hx = ord2f(bbox[3]), hy = ord2f(bbox[4]), hz = ord2f(bbox[5]);
  const float ext =
      fmaxf(__fsub_rn(hx, lx), fmaxf(__fsub_rn(hy, ly), __fsub_rn(hz, lz)));
  const float inv = ext > 0.f ? __frcp_rn(ext) : 0.f;
  const bool wide = sizeof(K) == 8;
  const float scale = wide ? 2097152.f : 1024.f;
  const float qmax = scale - 1.f;
  // four particles per thread and round, their loads issued together
  const int stride = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
    float4 pv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * stride;
      if (i < n) pv[u] = pos[i];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * stride;
      if (i >= n) break;
      const float4 p = pv[u];
      uint32_t qx = quantise(p.x, lx, inv, scale, qmax);
      uint32_t qy = quantise(p.y, ly, inv, scale, qmax);
      uint32_t qz = quantise(p.z, lz, inv, scale, qmax);
      K k;
      if (wide)
        k = (K)((spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz));
      else
        k = (K)((spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz));
      keys[i] = k;
      for (int ps = 0; ps < passes; ++ps)
        atomicAdd(&s_hist[ps * kSortRadix + (uint32_t)((k >> (8 * ps)) & 0xffu)], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x) {
    uint32_t c = s_hist[i];
    if (c) atomicAdd(&hist[i], c);
  }
}

int launch_morton(Workspace& w, const StepArgs& a, cudaStream_t st) {
  int passes = sort_passes(a.key_bits);
  int blocks = (a.n + kMortonThreads - 1) / kMortonThreads;
  const int sms = device_sm_count();
  if (blocks > sms) blocks = sms;   // one CTA per SM: fewer histogram flushes
  if (a.key_bits == 63)
    return launch_chained(k_morton<uint64_t>, blocks, kMortonThreads, 0, st,
                          (const float4*)a.pos, a.n, (const int*)w.bbox,
                          (uint64_t*)w.keys, w.hist, passes);
  return launch_chained(k_morton<uint32_t>, blocks, kMortonThreads, 0, st,
                        (const float4*)a.pos, a.n, (const int*)w.bbox, (uint32_t*)w.keys,
                        w.hist, passes);
}

// ---------------------------------------------------------------------------
// Onesweep LSD radix sort (Adinets & Merrill, 2022), 8-bit digits, stable.
// Per pass one kernel: each CTA takes the next tile by ticket (so it only
// waits on CTAs that are already running), ranks its keys with warp ballots
// per digit bit, publishes its digit counts, resolves its global offsets by a
// decoupled look-back over earlier tiles (bounded waits), stages the tile in
// digit order in shared memory and writes each digit's run contiguously.
// ---------------------------------------------------------------------------
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1u;
constexpr int kLookbackSpin = 1 << 20;
constexpr int kLookbackWindow = 4;   // predecessor tiles read per look-back step
constexpr int kSortBatch = 4;   // staged elements a thread stores together

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// pass modes: a middle pass; the last pass (also gathers the sorted
// positions); the last pass of an ensemble sort (also remaps each
// simulation's keys into its slot range)
constexpr int kSortMid = 0;
constexpr int kSortLast = 1;
constexpr int kSortLastEnsemble = 2;

// Lanes of the warp whose (valid) item has the same 8-bit digit: one ballot
// per digit bit, so the cost does not grow with the number of distinct
// digits in the warp.  Meaningful for lanes with ok set.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, bool ok) {
  uint32_t m = __ballot_sync(0xffffffffu, ok);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool bit = (d >> b) & 1u;
    const uint32_t v = __ballot_sync(0xffffffffu, bit);
    m &= bit ? v : ~v;
  }
  return m;
}

template <typename K, int MODE>
__global__ void __launch_bounds__(kSortThreads, kSortCtasPerSm)
    k_sort_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                K* __restrict__ kout, uint32_t* __restrict__ vout, int n,
                int shift, const uint32_t* __restrict__ hist,
                uint32_t* status, uint32_t* tile_ctr, unsigned* err,
                const float4* __restrict__ pos, float4* __restrict__ pos_sorted,
                const SimDesc* __restrict__ sims, int nsims) {
  constexpr int W = kSortThreads / 32;
  static_assert(kSortThreads >= kSortRadix, "one thread per digit at least");
  __shared__ uint32_t s_wc[W][kSortRadix];
  __shared__ uint32_t s_base[kSortRadix];
  __shared__ uint32_t s_tex[kSortRadix];
  __shared__ uint32_t s_scan[W];
  __shared__ uint32_t s_tsc[W];
  __shared__ int s_tile;
  // the tile in digit order, staged for coalesced stores (dynamic)
  extern __shared__ __align__(16) unsigned char s_stage[];
  K* s_key = reinterpret_cast<K*>(s_stage);
  uint32_t* s_val = reinterpret_cast<uint32_t*>(s_key + kSortTile);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  chain_release();
  chain_wait();
  if (tid == 0) s_tile = (int)atomicAdd(tile_ctr, 1u);
  for (int i = tid; i < W * kSortRadix; i += kSortThreads) (&s_wc[0][0])[i] = 0u;

  // threads [0, kSortRadix) own one digit each in the per-digit steps
  const bool dig = tid < kSortRadix;
  // global exclusive prefix of this pass's digit counts (digit threads)
  const uint32_t h = dig ? hist[tid] : 0u;
  uint32_t incl = h;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_scan[warp] = incl;
  __syncthreads();
  uint32_t wofs = 0;
  for (int i = 0; i < warp; ++i) wofs += s_scan[i];
  const uint32_t gexcl = wofs + incl - h;

  const int tile = s_tile;
  const long seg = (long)tile * kSortTile + (long)warp * (kSortItems * 32);
  K key[kSortItems];
  uint32_t val[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    long idx = seg + k * 32 + lane;
    bool ok = idx < n;
    key[k] = ok ? kin[idx] : (K)0;
    val[k] = ok ? (vin ? vin[idx] : (uint32_t)idx) : 0u;   // no vin: the identity
  }
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    long idx = seg + k * 32 + lane;
    bool ok = idx < n;
    uint32_t d = ok ? (uint32_t)((key[k] >> shift) & 0xffu) : 0u;
    uint32_t peers = digit_peers(d, ok);
    uint32_t old = 0;
    if (ok) {
      old = s_wc[warp][d];
      rank[k] = old + __popc(peers & lt);
    }
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) s_wc[warp][d] = old + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // per digit: offsets of each warp inside the tile, and the tile's count
  uint32_t run = 0;
  if (dig) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint32_t c = s_wc[w][tid];
      s_wc[w][tid] = run;
      run += c;
    }
  }
  const uint32_t count = run;
  // tile-local start of digit tid in digit order
  uint32_t tin = count;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, tin, o);
    if (lane >= o) tin += y;
  }
  if (lane == 31) s_tsc[warp] = tin;
  uint32_t* my = status + (size_t)tile * kSortRadix + tid;
  uint32_t excl = 0;
  if (!dig) {
    // no digit of its own
  } else if (tile == 0) {
    st_relaxed(my, kFlagInc | count);
  } else {
    st_relaxed(my, kFlagAgg | count);
    // kLookbackWindow predecessors' status words are read together, then
    // taken in order until an inclusive prefix; a tile that has published
    // nothing yet is waited for (bounded)
    bool done = false;
    for (int t = tile - 1; t >= 0 && !done; t -= kLookbackWindow) {
      uint32_t win[kLookbackWindow];
#pragma unroll
      for (int j = 0; j < kLookbackWindow; ++j)
        win[j] = t - j >= 0 ? ld_relaxed(status + (size_t)(t - j) * kSortRadix + tid)
                            : kFlagInc;   // before tile 0: an empty prefix
#pragma unroll
      for (int j = 0; j < kLookbackWindow; ++j) {
        if (done) break;
        uint32_t s = win[j];
        if ((s & ~kValMask) == 0u) {
          const uint32_t* p = status + (size_t)(t - j) * kSortRadix + tid;
          int spins = 0;
          while ((s & ~kValMask) == 0u && spins < kLookbackSpin) {
            if (spins > 64) __nanosleep(64);
            s = ld_relaxed(p);
            ++spins;
          }
          if ((s & ~kValMask) == 0u) {   // gave up: flag it and stop waiting
            raise_err(err, NB_DEVERR_SORT);
            done = true;
            break;
          }
        }
        excl += s & kValMask;
        if ((s & kFlagInc) != 0u) done = true;
      }
    }
    st_relaxed(my, kFlagInc | ((excl + count) & kValMask));
  }
  __syncthreads();   // s_tsc
  uint32_t tofs = 0;
  for (int i = 0; i < warp; ++i) tofs += s_tsc[i];
  const uint32_t texcl = tofs + tin - count;
  if (dig) {
    s_tex[tid] = texcl;
    // global index of tile-local digit-order index i of digit d: s_base[d] + i
    // (unsigned wrap-around cancels)
    s_base[tid] = gexcl + excl - texcl;
  }
  __syncthreads();

#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    long idx = seg + k * 32 + lane;
    if (idx < n) {
      const uint32_t d = (uint32_t)((key[k] >> shift) & 0xffu);
      const uint32_t lpos = s_tex[d] + s_wc[warp][d] + rank[k];
      if (lpos < (uint32_t)kSortTile) {
        s_key[lpos] = key[k];
        s_val[lpos] = val[k];
      } else {
        raise_err(err, NB_DEVERR_SORT);
      }
    }
  }
  __syncthreads();
  // kSortBatch elements per thread at a time, so that the last pass's
  // position gathers are in flight together
  const int tn = (int)min((long)kSortTile, (long)n - (long)tile * kSortTile);
  for (int base = tid; base < tn; base += kSortBatch * kSortThreads) {
    K kk[kSortBatch];
    uint32_t vv[kSortBatch], dst[kSortBatch];
    bool put[kSortBatch];
#pragma unroll
    for (int j = 0; j < kSortBatch; ++j) {
      const int i = base + j * kSortThreads;
      put[j] = false;
      if (i >= tn) continue;
      kk[j] = s_key[i];
      vv[j] = s_val[i];
      const uint32_t d = (uint32_t)((kk[j] >> shift) & 0xffu);
      dst[j] = s_base[d] + (uint32_t)i;
      if (dst[j] >= (uint32_t)n || vv[j] >= (uint32_t)n) {
        raise_err(err, NB_DEVERR_SORT);
        continue;
      }
      if (MODE == kSortLastEnsemble) {
        // keys arrive grouped by simulation (id in bits 30+); rank d within
        // the group goes to slot base + (d - coff); unused slots drop out
        const uint32_t s = (uint32_t)(kk[j] >> 30);
        if (s >= (uint32_t)nsims) continue;
        dst[j] = (uint32_t)sims[s].base + (dst[j] - (uint32_t)sims[s].coff);
        if (dst[j] >= (uint32_t)n) {
          raise_err(err, NB_DEVERR_SORT);
          continue;
        }
      }
      put[j] = true;
    }
    float4 pv[kSortBatch];
    if (MODE != kSortMid) {
#pragma unroll
      for (int j = 0; j < kSortBatch; ++j)
        if (put[j]) pv[j] = pos[vv[j]];
    }
#pragma unroll
    for (int j = 0; j < kSortBatch; ++j) {
      if (!put[j]) continue;
      kout[dst[j]] = kk[j];
      vout[dst[j]] = vv[j];
      if (MODE != kSortMid) pos_sorted[dst[j]] = pv[j];
    }
  }
}

// Launches one sort pass with its staging buffer (dynamic shared memory).
template <typename K, int MODE>
static int launch_sort_pass(int tiles, cudaStream_t st, const K* kin, const uint32_t* vin,
                            K* kout, uint32_t* vout, int n, int shift,
                            const uint32_t* hist, uint32_t* status, uint32_t* ctr,
                            unsigned* err, const float4* pos, float4* pos_sorted,
                            const SimDesc* sims, int nsims, bool chained = false) {
  const int smem = kSortTile * (int)(sizeof(K) + sizeof(uint32_t));
  NB_CUDA(cudaFuncSetAttribute(k_sort_pass<K, MODE>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  if (chained)
    return launch_chained(k_sort_pass<K, MODE>, tiles, kSortThreads, smem, st, kin, vin, kout,
                          vout, n, shift, hist, status, ctr, err, pos, pos_sorted, sims,
                          nsims);
  k_sort_pass<K, MODE><<<tiles, kSortThreads, smem, st>>>(
      kin, vin, kout, vout, n, shift, hist, status, ctr, err, pos, pos_sorted, sims, nsims);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

template <typename K>
static int sort_impl(Workspace& w, const StepArgs& a, cudaStream_t st) {
  const int passes = sort_passes(a.key_bits);
  const int tiles = (a.n + kSortTile - 1) / kSortTile;
  K* kin = (K*)w.keys;
  K* kalt = (K*)w.keys_alt;
  // the first pass takes the particle index as its value (the keys are in
  // particle order), so no value array is read before it
  uint32_t* vin = nullptr;
  uint32_t* valt = w.vals_alt;
  uint32_t* vnext = w.vals;   // the second pass's output
  for (int p = 0; p < passes; ++p) {
    uint32_t* hist = w.hist + p * kSortRadix;
    uint32_t* status = w.hist + 8 * kSortRadix + 8 + (size_t)p * w.status_tiles * kSortRadix;
    uint32_t* ctr = w.tile_ctr + p;
    if (p == passes - 1)
      NB_TRY((launch_sort_pass<K, kSortLast>(tiles, st, kin, vin, kalt, valt, a.n, 8 * p,
                                             hist, status, ctr, w.err, a.pos,
                                             w.pos_sorted, nullptr, 0, true)));
    else
      NB_TRY((launch_sort_pass<K, kSortMid>(tiles, st, kin, vin, kalt, valt, a.n, 8 * p,
                                            hist, status, ctr, w.err, nullptr, nullptr,
                                            nullptr, 0, true)));
    K* tk = kin; kin = kalt; kalt = tk;
    uint32_t* tv = valt; valt = vnext; vin = tv; vnext = tv;
  }
  // after an even number of passes the result is back in keys / vals
  if (kin != (K*)w.keys) {
    void* t = w.keys; w.keys = w.keys_alt; w.keys_alt = t;
    uint32_t* u = w.vals; w.vals = w.vals_alt; w.vals_alt = u;
  }
  return NB_OK;
}

int launch_sort(Workspace& w, const StepArgs& a, cudaStream_t st) {
  if (a.key_bits == 63) return sort_impl<uint64_t>(w, a, st);
  return sort_impl<uint32_t>(w, a, st);
}

__device__ __forceinline__ int clz_k(uint32_t x) { return __clz((int)x); }
__device__ __forceinline__ int clz_k(uint64_t x) { return __clzll((long long)x); }

// ---------------------------------------------------------------------------
// Single-tree build: the Karras tree and its centres of mass, bottom up
// (after Apetrei 2014, "Fast and Simple Agglomerative LBVH Construction").
// With d(s) = delta(s, s + 1) at the split s between sorted leaves s and
// s + 1, the Karras tree is the Cartesian tree of d (on sorted keys with the
// index tie-break, d has a unique minimum on every range): a node over leaves
// [lo, hi] joins the neighbour across the larger of d(lo - 1) and d(hi).  A
// node that joins to the right (split hi) is its parent's left child and
// Karras node hi; one that joins to the left is the right child and node lo.
// Node records, parent links, FP64 sums and boxes are therefore exactly those
// of the Karras build plus the centre-of-mass climb (the oracle checks them
// bit for bit).
//
// Levels.  A CTA takes a contiguous run of leaves and a sequence of "items"
// separated by splits: at the first level the items are its 1024 leaves, at
// later levels the finished subtrees that the CTAs below left between the
// splits they could not close.  At a split the first of the two children to
// arrive parks its cell in shared memory and stops, the second merges both
// and goes on; a node whose parent split is the run's boundary stops there.
// The climb runs in rounds over a dense list of pending arrivals while there
// are more of them than threads, then each thread climbs one arrival on its
// own.  Node records and parent links are written by a sweep at the end.
// The splits left open (at most one arrival, or the run's right boundary)
// go to a fixed-size segment per CTA, in order: they are ancestors of the
// run's two boundary splits, so there are at most 2 x depth + 1 of them
// (depth < 60 for 30-bit keys, < 93 for 63-bit).  The next level takes
// (kLevelItems - 1) / segment CTAs' segments per CTA; the level with one CTA
// closes the root.
// ---------------------------------------------------------------------------
constexpr int kLeafGroup = 1024;     // leaves per CTA at the first level
constexpr int kLevelThreads = 512;
constexpr int kLevelItems = 2048;    // capacity of a later level's CTA
constexpr int kSplitEmpty = -1;
constexpr int kSplitDone = -2;

__host__ __device__ constexpr int level_seg(int key_bits) {
  return key_bits == 63 ? 192 : 128;
}
__host__ __device__ constexpr int level_fan(int key_bits) {
  return (kLevelItems - 1) / level_seg(key_bits);
}
__host__ __device__ constexpr size_t level_smem(int cap) {
  // cells (FP64 sums, box lo, box hi), meta, positions, deltas, exchange
  // words, two arrival lists, scan scratch and list counters
  return (size_t)cap * (32 + 16 + 16 + 16 + 4 + 4 + 8) + (size_t)(cap + 1) * 4 + 40 * 4;
}

struct LevelArgs {
  int n;
  const void* keys;                 // first level
  const float4* __restrict__ ps;
  Node* nodes;
  PairRec* pairs;                   // child pairs by split, or nullptr
  int* parent;
  double4* sums;
  float4* box_lo;
  float4* box_hi;
  const int2* in_seg;               // later levels: (position, delta) lists
  const int* in_count;
  int in_groups;                    // CTAs of the level below
  long long in_span;                // leaves per CTA of the level below
  int2* out_seg;                    // nullptr at the last level
  int* out_count;
  int seg;                          // segment capacity
  int fan;                          // segments per CTA
  unsigned* err;
  // many trees (ensembles): one run per CTA, the arrays above then hold all
  // simulations' slots and each run works on its simulation's slice
  const BuildRun* runs;
  const SimDesc* sims;
};

// The tree one CTA works on: the whole single tree, or one simulation's
// slice of the ensemble arrays.  Built field by field in the kernel; the
// kernel parameter itself is never modified.
struct TreeView {
  const LevelArgs& p;   // the kernel parameter (read in place)
  int n;
  int base;             // first slot of this tree in the arrays of p
  __device__ const float4* ps() const { return p.ps + base; }
  __device__ Node* nodes() const { return p.nodes ? p.nodes + base : nullptr; }
  __device__ PairRec* pairs() const { return p.pairs ? p.pairs + base : nullptr; }
  __device__ int* parent() const { return p.parent ? p.parent + 2 * (size_t)base : nullptr; }
  __device__ double4* sums() const { return p.sums + base; }
  __device__ float4* box_lo() const { return p.box_lo + base; }
  __device__ float4* box_hi() const { return p.box_hi + base; }
  __device__ unsigned* err() const { return p.err; }
};

struct Cell {   // a finished node: FP64 mass-weighted sums and box
  double4 s;
  float4 lo, hi;
};

template <typename K>
__device__ __forceinline__ int split_delta(const K* __restrict__ keys, int s) {
  const K x = keys[s] ^ keys[s + 1];
  if (x) return clz_k(x);
  return (int)(8 * sizeof(K)) + __clz(s ^ (s + 1));
}

__device__ __forceinline__ Cell leaf_cell(const float4* __restrict__ ps, int i) {
  const float4 p = ps[i];
  const double m = (double)p.w;
  Cell c;
  c.s = make_double4(__dmul_rn((double)p.x, m), __dmul_rn((double)p.y, m),
                     __dmul_rn((double)p.z, m), m);
  c.lo = c.hi = make_float4(p.x, p.y, p.z, 0.f);
  return c;
}

// IEEE addition and min / max are commutative: the order of a and b does not
// change the bits.
__device__ __forceinline__ Cell merge(const Cell& a, const Cell& b) {
  Cell c;
  c.s = make_double4(__dadd_rn(a.s.x, b.s.x), __dadd_rn(a.s.y, b.s.y),
                     __dadd_rn(a.s.z, b.s.z), __dadd_rn(a.s.w, b.s.w));
  c.lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y),
                     fminf(a.lo.z, b.lo.z), 0.f);
  c.hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y),
                     fmaxf(a.hi.z, b.hi.z), 0.f);
  return c;
}

// One child's half of its parent's pair record: the left half (side 0) of
// record k when the child's parent splits after leaf k and the child covers
// the leaves up to k, the right half (side 1) when it covers leaf k + 1
// onwards.  Writes outside the tree's n - 1 records are skipped and flagged.
__device__ __forceinline__ void write_pair_half(const TreeView& a, int k, int side,
                                                float4 p, float size2, int w) {
  PairRec* pr = a.pairs();
  if (!pr) return;
  if (k < 0 || k >= a.n - 1) {
    raise_err(a.err(), NB_DEVERR_BOUNDS);
    return;
  }
  pr[k].c[side] = p;
  reinterpret_cast<float2*>(&pr[k].sw)[side] = make_float2(size2, __int_as_float(w));
}

// Node record of internal node id over leaves [lo, hi] split after leaf sc,
// the parent links of its two children and its half of its parent's pair
// record.  A non-root internal node's Karras id is hi when it is its
// parent's left child (its parent splits after leaf hi) and lo when it is
// the right child (its parent splits after leaf lo - 1).
__device__ __forceinline__ void write_node(const TreeView& a, int id, int lo,
                                           int hi, int sc, const Cell& c) {
  const int ni = a.n - 1;
  const int l = sc == lo ? ni + sc : sc;
  const int r = sc + 1 == hi ? ni + sc + 1 : sc + 1;
  if (id < 0 || id >= ni || l < 0 || r < 0 || l >= 2 * ni + 1 || r >= 2 * ni + 1) {
    raise_err(a.err(), NB_DEVERR_BOUNDS);
    return;
  }
  float4 com;
  com.x = __double2float_rn(__ddiv_rn(c.s.x, c.s.w));
  com.y = __double2float_rn(__ddiv_rn(c.s.y, c.s.w));
  com.z = __double2float_rn(__ddiv_rn(c.s.z, c.s.w));
  com.w = __double2float_rn(c.s.w);
  const float e = fmaxf(__fsub_rn(c.hi.x, c.lo.x),
                        fmaxf(__fsub_rn(c.hi.y, c.lo.y), __fsub_rn(c.hi.z, c.lo.z)));
  const float size2 = __fmul_rn(e, e);
  if (Node* nd = a.nodes()) {
    float4* rec = reinterpret_cast<float4*>(&nd[id]);
    rec[0] = com;
    reinterpret_cast<int4*>(rec)[1] = make_int4(l, r, __float_as_int(size2), 0);
  }
  if (int* par = a.parent()) {
    par[l] = id;
    par[r] = id;
  }
  if (!(lo == 0 && hi == ni)) {
    if (id == hi) write_pair_half(a, id, 0, com, size2, sc);
    else write_pair_half(a, id - 1, 1, com, size2, sc);
  } else if (PairRec* pr = a.pairs()) {   // the root's own record
    pr[ni].c[0] = com;
    reinterpret_cast<float2*>(&pr[ni].sw)[0] = make_float2(size2, __int_as_float(sc));
  }
}

__device__ __forceinline__ void store_cell(const TreeView& a, int id, const Cell& c) {
  if (id < 0 || id >= a.n - 1) {
    raise_err(a.err(), NB_DEVERR_BOUNDS);
    return;
  }
  a.sums()[id] = c.s;
  a.box_lo()[id] = c.lo;
  a.box_hi()[id] = c.hi;
}

__device__ __forceinline__ Cell load_cell(const TreeView& a, int id) {
  Cell c;
  const double2* q = reinterpret_cast<const double2*>(&a.sums()[id]);
  const double2 q0 = __ldcg(q), q1 = __ldcg(q + 1);
  c.s = make_double4(q0.x, q0.y, q1.x, q1.y);
  c.lo = __ldcg(&a.box_lo()[id]);
  c.hi = __ldcg(&a.box_hi()[id]);
  return c;
}

// Shared memory of one level CTA with room for `cap` items.
struct LevelSmem {
  double4* sum;    // [cap] cells by slot
  float4* lo;
  float4* hi;
  int4* meta;      // [cap] (lo, hi, split leaf, Karras id) of a node formed
                   // here, Karras id -1 for an item
  int* pos;        // [cap] leaf position of split k
  int* delta;      // [cap + 1] delta[k + 1] = d(split k), delta[0] = d of the
                   // split left of the run
  int* exch;       // [cap] far item of the first arrival at split k
  unsigned* list;  // [2][cap] pending arrivals (ia | ib << 16)
  int* scan;       // [40]
  __device__ LevelSmem(unsigned char* raw, int cap) {
    sum = reinterpret_cast<double4*>(raw);
    lo = reinterpret_cast<float4*>(sum + cap);
    hi = lo + cap;
    meta = reinterpret_cast<int4*>(hi + cap);
    pos = reinterpret_cast<int*>(meta + cap);
    delta = pos + cap;
    exch = delta + cap + 1;
    list = reinterpret_cast<unsigned*>(exch + cap);
    scan = reinterpret_cast<int*>(list + 2 * cap);
  }
};

// Run of leaves [A, B); M splits in its sequence (the last is the right
// boundary when B < n); items between them.
struct Run {
  int A, B, M, items, local;
  __device__ int item_lo(const LevelSmem& sm, int i) const {
    return i == 0 ? A : sm.pos[i - 1] + 1;
  }
  __device__ int item_hi(const LevelSmem& sm, int i, int ni) const {
    return i < M ? sm.pos[i] : ni;
  }
};

__device__ __forceinline__ void put_cell(const LevelSmem& sm, int slot, const Cell& c) {
  sm.sum[slot] = c.s;
  sm.lo[slot] = c.lo;
  sm.hi[slot] = c.hi;
}

__device__ __forceinline__ Cell get_cell(const LevelSmem& sm, int slot) {
  Cell c;
  c.s = sm.sum[slot];
  c.lo = sm.lo[slot];
  c.hi = sm.hi[slot];
  return c;
}

// Appends v to list `which` when `push` (warp-aggregated); all lanes call.
__device__ __forceinline__ void list_push(const LevelSmem& sm, int* count, int which,
                                          int cap, bool push, unsigned v) {
  const unsigned mask = __ballot_sync(0xffffffffu, push);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (push) sm.list[which * cap + base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// A node over items [ia, ib] (leaves [lo, hi], cell c, formed here or an
// item) that has just been finished: the root and frontier nodes are written
// out; any other parks its cell in its slot and becomes a pending arrival.
// Slot = the node's Karras id in item space (right end if it joins to the
// right, left end otherwise); an item and a node formed later share a slot
// only when the item is below the node, and the node is written after the
// item's cell was read.  Returns whether it parked.
__device__ __forceinline__ bool finish_node(const TreeView& a, const LevelSmem& sm,
                                            const Run& run, int ia, int ib, int lo,
                                            int hi, int sc, bool formed, const Cell& c) {
  const int ni = a.n - 1;
  if (lo == 0 && hi == ni) {   // the root: this run is the whole tree
    write_node(a, 0, lo, hi, sc, c);
    if (int* par = a.parent()) par[0] = -1;
    return false;
  }
  const bool right = lo == 0 || (hi != ni && sm.delta[ib + 1] > sm.delta[ia]);
  const int kid = right ? hi : lo;
  const int k = right ? ib : ia - 1;
  if (k < 0 || k >= run.local) {   // parent split on the run's boundary
    if (formed) {
      write_node(a, kid, lo, hi, sc, c);
      store_cell(a, kid, c);
    }
    return false;
  }
  const int slot = right ? ib : ia;
  put_cell(sm, slot, c);
  if (formed) sm.meta[slot] = make_int4(lo, hi, sc, kid);
  return true;
}

// One pending arrival (items [ia, ib], parked in its slot) climbs until it
// is the first at a split or finishes.  acq_rel: the exchange publishes this
// thread's slot writes and acquires the sibling's.
__device__ __forceinline__ void climb_arrival(const TreeView& a, const LevelSmem& sm,
                                              const Run& run, unsigned d) {
  const int ni = a.n - 1;
  int ia = (int)(d & 0xffffu), ib = (int)(d >> 16);
  int lo = run.item_lo(sm, ia), hi = run.item_hi(sm, ib, ni);
  bool right = lo == 0 || (hi != ni && sm.delta[ib + 1] > sm.delta[ia]);
  Cell c = get_cell(sm, right ? ib : ia);
  for (int guard = 0; guard <= run.items; ++guard) {
    const int k = right ? ib : ia - 1;
    cuda::atomic_ref<int, cuda::thread_scope_block> word(sm.exch[k]);
    const int other = word.exchange(right ? ia : ib, cuda::memory_order_acq_rel);
    if (other == kSplitEmpty) return;
    if (other < 0 || other >= run.items || (right ? other <= k : other > k)) break;
    const Cell o = get_cell(sm, right ? k + 1 : k);
    sm.exch[k] = kSplitDone;
    if (right) {
      ib = other;
      hi = run.item_hi(sm, other, ni);
    } else {
      ia = other;
      lo = run.item_lo(sm, other);
    }
    c = merge(c, o);
    if (!finish_node(a, sm, run, ia, ib, lo, hi, sm.pos[k], true, c)) return;
    right = lo == 0 || (hi != ni && sm.delta[ib + 1] > sm.delta[ia]);
  }
  raise_err(a.err(), NB_DEVERR_TREE);
}

// Later levels hold 2048 items (196 KB of shared memory): one CTA per SM, so
// they may use twice the registers of the first level's two CTAs.
template <typename K, bool FIRST>
__global__ void __launch_bounds__(kLevelThreads, FIRST ? 2 : 1) k_build_level(LevelArgs args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  chain_release();
  chain_wait();
  constexpr int C = FIRST ? kLeafGroup : kLevelItems;
  const LevelSmem sm(smem_raw, C);
  // this CTA's tree, its group index there, its input segments [sfirst,
  // sfirst + scount) and whether it hands open splits to the next level
  const LevelArgs& p = args;
  int tn = p.n, sbase = 0;
  int g = blockIdx.x, sfirst = 0, scount = 0;
  bool out = p.out_seg != nullptr;
  if (p.runs) {
    const BuildRun r = p.runs[blockIdx.x];
    const SimDesc d = p.sims[r.sim];
    if (!d.active || d.n < 2) return;
    tn = d.n;
    sbase = d.base;
    g = r.group;
    sfirst = r.in_first;
    scount = r.in_count;
    out = out && r.out;
  } else if (!FIRST) {
    sfirst = g * p.fan;
    scount = min(p.fan, p.in_groups - sfirst);
  }
  const TreeView a{p, tn, sbase};
  const int n = a.n, ni = n - 1, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  Run run;
  if (FIRST) {
    const K* __restrict__ keys = static_cast<const K*>(p.keys) + sbase;
    run.A = g * kLeafGroup;
    run.B = min(n, run.A + kLeafGroup);
    run.M = run.B < n ? run.B - run.A : run.B - run.A - 1;
    for (int k = tid; k < run.M; k += kLevelThreads) {
      sm.pos[k] = run.A + k;
      sm.delta[k + 1] = split_delta(keys, run.A + k);
    }
    if (tid == 0) sm.delta[0] = run.A > 0 ? split_delta(keys, run.A - 1) : -1;
  } else {
    const int r0 = sfirst, r1 = sfirst + scount;
    if (warp == 0) {   // segment offsets (fan <= 32)
      const int c = r0 + lane < r1 ? min(p.in_count[r0 + lane], p.seg) : 0;
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      sm.scan[lane] = incl - c;
      if (lane == 31) sm.scan[32] = incl;
      if (lane == 0) {   // the last entry below is the split left of this run
        int d = -1;
        if (g > 0) {
          const int cp = min(p.in_count[r0 - 1], p.seg);
          if (cp > 0) d = p.in_seg[(size_t)(r0 - 1) * p.seg + cp - 1].y;
        }
        sm.delta[0] = d;
      }
    }
    __syncthreads();
    run.M = sm.scan[32];
    // one warp per segment
    for (int r = r0 + warp; r < r1; r += kLevelThreads / 32) {
      const int off = sm.scan[r - r0];
      const int c = sm.scan[r - r0 + 1] - off;
      for (int e = lane; e < c; e += 32) {
        const int2 v = p.in_seg[(size_t)r * p.seg + e];
        sm.pos[off + e] = v.x;
        sm.delta[off + e + 1] = v.y;
      }
    }
    // region index of segment r within the tree: g * fan + (r - sfirst)
    run.A = (int)min((long long)n, (long long)g * p.fan * p.in_span);
    run.B = (int)min((long long)n, ((long long)g * p.fan + scount) * p.in_span);
  }
  run.items = run.B < n ? run.M : run.M + 1;
  run.local = run.B < n ? run.M - 1 : run.M;
  for (int k = tid; k < run.M; k += kLevelThreads) sm.exch[k] = kSplitEmpty;
  for (int j = tid; j < run.items; j += kLevelThreads) sm.meta[j].w = -1;
  int* count = sm.scan + 34;   // three rotating list counters
  if (tid < 3) count[tid] = 0;
  __syncthreads();

  // round 0: every item parks its cell and becomes a pending arrival
  for (int base = 0; base < run.items; base += kLevelThreads) {
    const int j = base + tid;
    bool push = false;
    if (j < run.items) {
      const int lo = run.item_lo(sm, j), hi = run.item_hi(sm, j, ni);
      Cell c;
      if (FIRST || lo == hi) {
        c = leaf_cell(a.ps(), lo);
        if (FIRST && ni > 0) {   // the leaf's half of its parent's pair record
          const bool right = lo == 0 || (hi != ni && sm.delta[j + 1] > sm.delta[j]);
          write_pair_half(a, right ? lo : lo - 1, right ? 0 : 1, a.ps()[lo], -1.f, -1);
        }
      } else {   // a subtree finished below: its Karras id follows its direction
        const bool right = lo == 0 || (hi != ni && sm.delta[j + 1] > sm.delta[j]);
        const int kid = right ? hi : lo;
        if (kid < ni) {
          c = load_cell(a, kid);
        } else {   // only after a failed sort (the whole tree as one item)
          raise_err(a.err(), NB_DEVERR_TREE);
          c = leaf_cell(a.ps(), lo);
        }
      }
      push = finish_node(a, sm, run, j, j, lo, hi, -1, false, c);
    }
    list_push(sm, &count[0], 0, C, push, (unsigned)j | ((unsigned)j << 16));
  }
  __syncthreads();

  // rounds: each pending arrival takes its split's exchange word; the second
  // of two siblings merges them.  A slot is written at least one barrier
  // before any exchange that can lead to its read, so relaxed atomics do.
  // Once no more arrivals are pending than there are threads, each takes one
  // and climbs on its own (block-scope acq_rel exchanges, no barriers).
  int cur = 0;
  for (int round = 0; round <= run.items; ++round) {
    const int L = count[round % 3];
    if (L == 0) break;
    if (L <= kLevelThreads) {
      if (tid < L) climb_arrival(a, sm, run, sm.list[cur * C + tid]);
      break;
    }
    if (tid == 0) count[(round + 2) % 3] = 0;
    for (int base = 0; base < L; base += kLevelThreads) {
      const int i = base + tid;
      bool push = false;
      unsigned v = 0;
      if (i < L) {
        const unsigned d = sm.list[cur * C + i];
        int ia = (int)(d & 0xffffu), ib = (int)(d >> 16);
        int lo = run.item_lo(sm, ia), hi = run.item_hi(sm, ib, ni);
        const bool right = lo == 0 || (hi != ni && sm.delta[ib + 1] > sm.delta[ia]);
        const int k = right ? ib : ia - 1;
        const int other = atomicExch(&sm.exch[k], right ? ia : ib);
        if (other != kSplitEmpty) {
          if (other < 0 || other >= run.items || (right ? other <= k : other > k)) {
            raise_err(a.err(), NB_DEVERR_TREE);
          } else {
            const Cell mine = get_cell(sm, right ? ib : ia);
            const Cell o = get_cell(sm, right ? k + 1 : k);
            sm.exch[k] = kSplitDone;
            if (right) {
              ib = other;
              hi = run.item_hi(sm, other, ni);
            } else {
              ia = other;
              lo = run.item_lo(sm, other);
            }
            push = finish_node(a, sm, run, ia, ib, lo, hi, sm.pos[k], true, merge(mine, o));
            v = (unsigned)ia | ((unsigned)ib << 16);
          }
        }
      }
      list_push(sm, &count[(round + 1) % 3], cur ^ 1, C, push, v);
    }
    __syncthreads();
    cur ^= 1;
  }
  __syncthreads();
  // node records of the nodes formed here, in slot order
  for (int j = tid; j < run.items; j += kLevelThreads) {
    const int4 m = sm.meta[j];
    if (m.w >= 0) write_node(a, m.w, m.x, m.y, m.z, get_cell(sm, j));
  }
  if (!out) return;
  // a formed child waiting at an open split hands its cell to the next level
  for (int k = tid; k < run.local; k += kLevelThreads) {
    const int e = sm.exch[k];
    if (e < 0) continue;
    const bool left = e <= k;   // the waiting child covers items [e, k]
    if (left ? e == k : e == k + 1) continue;   // a single item: stored below
    const int slot = left ? k : k + 1;
    store_cell(a, sm.meta[slot].w, get_cell(sm, slot));
  }
  // open splits in order: (position, delta) into this CTA's segment
  const int chunk = (run.M + kLevelThreads - 1) / kLevelThreads;
  const int k0 = min(run.M, tid * chunk), k1 = min(run.M, k0 + chunk);
  int cnt = 0;
  for (int k = k0; k < k1; ++k) cnt += (k >= run.local || sm.exch[k] != kSplitDone);
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) sm.scan[warp] = incl;   // the segment offsets are no longer read
  __syncthreads();
  int base = 0, total = 0;
  for (int w = 0; w < kLevelThreads / 32; ++w) {
    const int v = sm.scan[w];
    if (w < warp) base += v;
    total += v;
  }
  int off = base + incl - cnt;
  for (int k = k0; k < k1; ++k) {
    if (k >= run.local || sm.exch[k] != kSplitDone) {
      if (off < p.seg)
        p.out_seg[(size_t)blockIdx.x * p.seg + off] = make_int2(sm.pos[k], sm.delta[k + 1]);
      ++off;
    }
  }
  if (tid == 0) {
    p.out_count[blockIdx.x] = min(total, p.seg);
    if (total > p.seg) raise_err(a.err(), NB_DEVERR_TREE);
  }
}

static LevelArgs level_args(Workspace& w, const StepArgs& a) {
  LevelArgs b{};
  b.n = a.n;
  b.keys = w.keys;
  b.ps = w.pos_sorted;
  b.nodes = a.node_records || a.walk_kernel != 0 ? w.nodes : nullptr;
  b.pairs = w.pairs;
  b.parent = a.node_records || a.walk_kernel != 0 ? w.parent : nullptr;
  b.sums = w.sums;
  b.box_lo = w.box_lo;
  b.box_hi = w.box_hi;
  b.seg = level_seg(a.key_bits);
  b.fan = level_fan(a.key_bits);
  b.err = w.err;
  return b;
}

size_t build_seg_entries(int cap) {
  return (size_t)((cap + kLeafGroup - 1) / kLeafGroup) * level_seg(63);
}

// First level: leaf groups (the bottom of the tree, most of its nodes).
int launch_build(Workspace& w, const StepArgs& a, cudaStream_t st) {
  LevelArgs b = level_args(w, a);
  const int groups = (a.n + kLeafGroup - 1) / kLeafGroup;
  if (groups > 1) {
    b.out_seg = w.seg[0];
    b.out_count = w.seg_count[0];
  }
  const int smem = (int)level_smem(kLeafGroup);
  if (a.key_bits == 63) {
    NB_CUDA(cudaFuncSetAttribute(k_build_level<uint64_t, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return launch_chained(k_build_level<uint64_t, true>, groups, kLevelThreads, smem, st, b);
  } else {
    NB_CUDA(cudaFuncSetAttribute(k_build_level<uint32_t, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return launch_chained(k_build_level<uint32_t, true>, groups, kLevelThreads, smem, st, b);
  }
}

// Later levels: the tree above the leaf groups, up to the root.
int launch_com(Workspace& w, const StepArgs& a, cudaStream_t st) {
  LevelArgs b = level_args(w, a);
  const int smem = (int)level_smem(kLevelItems);
  NB_CUDA(cudaFuncSetAttribute(k_build_level<uint32_t, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int groups = (a.n + kLeafGroup - 1) / kLeafGroup;
  long long span = kLeafGroup;
  int p = 0;
  while (groups > 1) {
    const int next = (groups + b.fan - 1) / b.fan;
    b.in_seg = w.seg[p];
    b.in_count = w.seg_count[p];
    b.in_groups = groups;
    b.in_span = span;
    b.out_seg = next > 1 ? w.seg[p ^ 1] : nullptr;
    b.out_count = next > 1 ? w.seg_count[p ^ 1] : nullptr;
    NB_TRY(launch_chained(k_build_level<uint32_t, false>, next, kLevelThreads, smem, st, b));
    groups = next;
    span *= b.fan;
    p ^= 1;
  }
  return NB_OK;
}

// ---------------------------------------------------------------------------
// Ensemble tree build.  One global sort of keys (sim << 30) | morton30 groups
// the simulations (stable, so each group keeps its own Morton order); its
// last pass scatters group s into slots [base_s, base_s + n_s).  Karras and
// the centre-of-mass climb then run per simulation on local indices, so each
// tree is the one the simulation alone would build (the 64-bit keys shift
// every delta by 32, which keeps the order of the deltas).
// ---------------------------------------------------------------------------
constexpr uint64_t kEnsDeadKey = ((uint64_t)kEnsMaxSims << 30) | 0x3fffffffull;

__global__ void __launch_bounds__(256) k_ens_morton(EnsArgs e) {
  constexpr int P = (kEnsKeyBits + 7) / 8;
  __shared__ uint32_t s_hist[P * kSortRadix];
  for (int i = threadIdx.x; i < P * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < e.nslots;
       slot += gridDim.x * blockDim.x) {
    uint64_t key = kEnsDeadKey;
    const int s = e.blk_sim[slot >> 5];
    if (s >= 0) {
      const SimDesc d = e.sims[s];
      const int local = slot - d.base;
      if (d.active && d.force == NB_FORCE_BH && local < d.n) {
        const float lx = ord2f(e.bbox_min[4 * s]), ly = ord2f(e.bbox_min[4 * s + 1]),
                    lz = ord2f(e.bbox_min[4 * s + 2]);
        const float hx = ord2f(e.bbox_max[4 * s]), hy = ord2f(e.bbox_max[4 * s + 1]),
                    hz = ord2f(e.bbox_max[4 * s + 2]);
        const float ext =
            fmaxf(__fsub_rn(hx, lx), fmaxf(__fsub_rn(hy, ly), __fsub_rn(hz, lz)));
        const float inv = ext > 0.f ? __frcp_rn(ext) : 0.f;
        const float4 p = e.pos[slot];
        const uint32_t m = (spread10(quantise(p.x, lx, inv, 1024.f, 1023.f)) << 2) |
                           (spread10(quantise(p.y, ly, inv, 1024.f, 1023.f)) << 1) |
                           spread10(quantise(p.z, lz, inv, 1024.f, 1023.f));
        key = ((uint64_t)s << 30) | m;
      }
    }
    e.keys[slot] = key;
    e.perm[slot] = (uint32_t)slot;
#pragma unroll
    for (int ps = 0; ps < P; ++ps)
      atomicAdd(&s_hist[ps * kSortRadix + (uint32_t)((key >> (8 * ps)) & 0xffu)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < P * kSortRadix; i += blockDim.x) {
    const uint32_t c = s_hist[i];
    if (c) atomicAdd(&e.hist[i], c);
  }
}

int launch_ens_morton(const EnsArgs& e, cudaStream_t st) {
  int blocks = (e.nslots + 255) / 256;
  if (blocks > 4 * device_sm_count()) blocks = 4 * device_sm_count();
  k_ens_morton<<<blocks, 256, 0, st>>>(e);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// Sorts; on return e.keys / e.perm point at the buffers holding the result.
int ens_sort_passes() { return (kEnsKeyBits + 7) / 8; }

int launch_ens_sort(EnsArgs& e, cudaStream_t st) {
  const int passes = ens_sort_passes();
  const int tiles = (e.nslots + kSortTile - 1) / kSortTile;
  uint64_t* kin = e.keys;
  uint64_t* kalt = e.keys_alt;
  uint32_t* vin = e.perm;
  uint32_t* valt = e.perm_alt;
  for (int p = 0; p < passes; ++p) {
    uint32_t* hist = e.hist + p * kSortRadix;
    uint32_t* status = e.status + (size_t)p * e.status_tiles * kSortRadix;
    uint32_t* ctr = e.tile_ctr + p;
    if (p == passes - 1)
      NB_TRY((launch_sort_pass<uint64_t, kSortLastEnsemble>(
          tiles, st, kin, vin, kalt, valt, e.nslots, 8 * p, hist, status, ctr, e.err,
          e.pos, e.pos_sorted, e.sims, e.nsims)));
    else
      NB_TRY((launch_sort_pass<uint64_t, kSortMid>(
          tiles, st, kin, vin, kalt, valt, e.nslots, 8 * p, hist, status, ctr, e.err,
          nullptr, nullptr, nullptr, 0)));
    uint64_t* tk = kin; kin = kalt; kalt = tk;
    uint32_t* tv = vin; vin = valt; valt = tv;
  }
  e.keys = kin;
  e.keys_alt = kalt;
  e.perm = vin;
  e.perm_alt = valt;
  return NB_OK;
}

// Ensemble trees: the level kernels over a plan of runs.  Level 1 has one
// run per (simulation, 1024-leaf group); a simulation with G groups at one
// level has ceil(G / fan) runs at the next, each over fan consecutive
// segments of its own runs below; a simulation is done at the level where it
// has one run.  The 64-bit keys (sim << 30) | morton30 give the same
// Cartesian tree as the simulation's own keys (the shared prefix shifts every
// d by 32), so each tree equals the one the simulation builds alone.
int plan_build(const SimDesc* sims, int nsims, BuildPlan& plan) {
  plan.levels = 0;
  plan.runs.clear();
  std::vector<int> groups(nsims, 0), first(nsims, 0);
  int live = 0;
  for (int s = 0; s < nsims; ++s)
    if (sims[s].active && sims[s].n >= 2 && sims[s].force == NB_FORCE_BH) {
      groups[s] = (sims[s].n + kLeafGroup - 1) / kLeafGroup;
      ++live;
    }
  if (!live) return NB_OK;
  const int fan = level_fan(30);
  for (int lv = 0;; ++lv) {
    if (lv >= kBuildMaxLevels) return set_error(NB_ERR_INVALID, "build plan too deep");
    plan.offset[lv] = (int)plan.runs.size();
    bool more = false;
    for (int s = 0; s < nsims; ++s) {
      const int G = groups[s];
      if (G == 0 || (lv > 0 && G == 1)) continue;
      const int next_first = (int)plan.runs.size();
      if (lv == 0) {
        for (int g = 0; g < G; ++g) plan.runs.push_back({s, g, 0, 0, G > 1 ? 1 : 0});
      } else {
        const int Gn = (G + fan - 1) / fan;
        for (int g = 0; g < Gn; ++g)
          plan.runs.push_back({s, g, first[s] + g * fan, std::min(fan, G - g * fan),
                               Gn > 1 ? 1 : 0});
        groups[s] = Gn;
      }
      first[s] = next_first - plan.offset[lv];   // index within this level
      if (groups[s] > 1) more = true;
    }
    plan.count[lv] = (int)plan.runs.size() - plan.offset[lv];
    plan.levels = lv + 1;
    if (!more) break;
  }
  return NB_OK;
}

size_t plan_seg_entries(int slots, int nsims) {
  return ((size_t)slots / kLeafGroup + (size_t)nsims + 1) * level_seg(30);
}

int launch_ens_levels(const EnsArgs& e, const BuildPlan& plan, cudaStream_t st) {
  LevelArgs b{};
  b.keys = e.keys;
  b.ps = e.pos_sorted;
  b.nodes = nullptr;   // the pair walk reads the child-pair records only
  b.pairs = e.pairs;
  b.parent = nullptr;
  b.sums = e.sums;
  b.box_lo = e.box_lo;
  b.box_hi = e.box_hi;
  b.seg = level_seg(30);
  b.fan = level_fan(30);
  b.err = e.err;
  b.sims = e.sims;
  long long span = kLeafGroup;
  for (int lv = 0; lv < plan.levels; ++lv) {
    const int runs = plan.count[lv];
    if (runs == 0) continue;
    b.runs = e.runs + plan.offset[lv];
    if (lv > 0) {
      b.in_seg = e.seg[(lv - 1) & 1];
      b.in_count = e.seg_count[(lv - 1) & 1];
      b.in_span = span;
      span *= b.fan;
    }
    b.out_seg = lv + 1 < plan.levels ? e.seg[lv & 1] : nullptr;
    b.out_count = lv + 1 < plan.levels ? e.seg_count[lv & 1] : nullptr;
    if (lv == 0) {
      const int smem = (int)level_smem(kLeafGroup);
      NB_CUDA(cudaFuncSetAttribute(k_build_level<uint64_t, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      k_build_level<uint64_t, true><<<runs, kLevelThreads, smem, st>>>(b);
    } else {
      const int smem = (int)level_smem(kLevelItems);
      NB_CUDA(cudaFuncSetAttribute(k_build_level<uint32_t, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      k_build_level<uint32_t, false><<<runs, kLevelThreads, smem, st>>>(b);
    }
    NB_CUDA(cudaGetLastError());
  }
  return NB_OK;
}

int warm_lbvh_kernels() {
  return warm_fns(k_morton<uint32_t>, k_morton<uint64_t>, k_ens_morton,
                  k_sort_pass<uint32_t, kSortMid>, k_sort_pass<uint32_t, kSortLast>,
                  k_sort_pass<uint64_t, kSortMid>, k_sort_pass<uint64_t, kSortLast>,
                  k_sort_pass<uint64_t, kSortLastEnsemble>, k_build_level<uint32_t, true>,
                  k_build_level<uint64_t, true>, k_build_level<uint32_t, false>);
}

}  // namespace nb
