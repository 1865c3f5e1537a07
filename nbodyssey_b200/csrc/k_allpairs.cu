// Tiled all-pairs softened gravity (src/forces.cu:17-60) and the all-pairs
// energy diagnostic (src/integrator.cu:43-110), written for sm_100a:
//
// * j-particle tiles of 512 sources (8 KB) move global -> shared memory by
//   TMA bulk copies (cp.async.bulk, no multicast) into a 3-stage ring of
//   mbarrier-tracked buffers; one elected thread issues the copies.
// * Sources are packed in pairs, (x0,x1,y0,y1)(z0,z1,m0,m1), so one 128-bit
//   shared load gives two sources per coordinate and the pair math runs on
//   Blackwell's packed FP32 pipe (fma/add/mul .f32x2): 12 packed ops and two
//   MUFU rsqrt per two interactions.
// * Each thread holds K targets; even and odd sources accumulate in the two
//   halves of a packed accumulator and are added at the end (FP32).
// * Small n splits the source range over `jsplit` CTAs per target tile; the
//   last CTA of a tile (ticket) sums the partials in fixed order, so results
//   are deterministic.  The leapfrog's closing kick is fused in the epilogue.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "f32x2.cuh"
#include "nb_internal.cuh"

namespace nb {

// --- mbarrier / bulk-copy helpers -----------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src,
                                          uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes),
      "r"(smem_u32(bar)) : "memory");
}
// Bounded wait on a phase parity; false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < (1 << 24); ++it) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;"
        " selp.u32 %0, 1, 0, p; }"
        : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

constexpr int kStages = 3;
constexpr int kTileF4 = kSrcTile;                 // float4 per tile (2 per pair)
constexpr uint32_t kTileBytes = kTileF4 * 16u;   // 8 KB


// One work item: the targets of tile `itile` (THREADS x K of them) against
// the sources of chunk `jc`, then the tile's fixed-order reduction when this
// is its last chunk to finish.  `tc` counts the tiles this CTA has taken
// through its ring so far (stage tc % kStages, barrier phase tc / kStages),
// so one CTA can run items back to back; every thread of the block calls it.
template <int THREADS, int K>
__device__ __forceinline__ void ap_item(const APArgs& a, int itile, int jc,
                                        float4 (*s_tile)[kTileF4], uint64_t* s_bar,
                                        bool* s_last, uint32_t& tc) {
  const int tid = threadIdx.x;
  const int ibase = itile * THREADS * K;
  const int j0 = jc * a.jchunk;
  const int j1 = min(j0 + a.jchunk, a.npad);
  const int ntiles = (j1 - j0) / kSrcTile;

  if (tid == 0) {
    for (int s = 0; s < kStages && s < ntiles; ++s) {
      const uint32_t u = tc + s;
      bulk_load(s_tile[u % kStages], a.src + 2 * ((j0 + s * kSrcTile) / 2), kTileBytes,
                &s_bar[u % kStages]);
    }
  }

  f2 nx[K], ny[K], nz[K], ax[K], ay[K], az[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    int i = ibase + k * THREADS + tid;
    float4 p = a.pos[i < a.n ? i : a.n - 1];
    nx[k] = pk2(-p.x, -p.x);
    ny[k] = pk2(-p.y, -p.y);
    nz[k] = pk2(-p.z, -p.z);
    ax[k] = ay[k] = az[k] = 0ull;
  }
  const f2 e2 = pk2(a.eps2, a.eps2);

  // A thread whose barrier wait gives up still runs the tile (shared-memory
  // reads of a tile that has not landed are harmless; the results are
  // discarded), so the barrier at the end of the tile is reached by every
  // thread and the decision to leave is the whole block's.
  int failed_at = -1;
  for (int t = 0; t < ntiles; ++t) {
    const uint32_t u = tc + t;
    const int s = u % kStages;
    const bool landed = mbar_wait(&s_bar[s], (u / kStages) & 1u);
    const ulonglong2* tile = reinterpret_cast<const ulonglong2*>(s_tile[s]);
#pragma unroll 4
    for (int q = 0; q < kSrcTile / 2; ++q) {
      const ulonglong2 A = tile[2 * q];       // (x0,x1) (y0,y1)
      const ulonglong2 B = tile[2 * q + 1];   // (z0,z1) (m0,m1)
#pragma unroll
      for (int k = 0; k < K; ++k) {
        f2 dx = add2(A.x, nx[k]);
        f2 dy = add2(A.y, ny[k]);
        f2 dz = add2(B.x, nz[k]);
        f2 r2 = fma2(dz, dz, e2);
        r2 = fma2(dy, dy, r2);
        r2 = fma2(dx, dx, r2);
        float r0, r1;
        up2(r2, r0, r1);
        f2 inv = pk2(mufu_rsqrt(r0), mufu_rsqrt(r1));
        f2 w = mul2(inv, B.y);
        f2 i2 = mul2(inv, inv);
        f2 f = mul2(w, i2);
        ax[k] = fma2(dx, f, ax[k]);
        ay[k] = fma2(dy, f, ay[k]);
        az[k] = fma2(dz, f, az[k]);
      }
    }
    // every thread is done with stage s; leave together if any wait gave up
    if (__syncthreads_or(!landed)) {
      failed_at = t;
      break;
    }
    if (tid == 0 && t + kStages < ntiles)
      bulk_load(s_tile[s], a.src + 2 * ((j0 + (t + kStages) * kSrcTile) / 2),
                kTileBytes, &s_bar[s]);
  }
  const bool ok = failed_at < 0;
  if (!ok && tid == 0) {
    raise_err(a.err, NB_DEVERR_WAIT);
    // let the copies still in flight into this block's shared memory land
    // (bounded waits) before the block moves on or retires
    for (int t = failed_at; t < ntiles && t < failed_at + kStages; ++t)
      mbar_wait(&s_bar[(tc + t) % kStages], ((tc + t) / kStages) & 1u);
  }
  tc += ok ? ntiles : min(ntiles, failed_at + kStages);

  // A block that could not read its sources writes NaN rows (and, with the
  // j-split, still takes its ticket), so a failed launch leaves visibly
  // invalid accelerations and a consistent ticket counter, never stale rows.
  const float bad = __int_as_float(0x7fc00000);
  float3 res[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    float u, v;
    up2(ax[k], u, v); res[k].x = ok ? u + v : bad;
    up2(ay[k], u, v); res[k].y = ok ? u + v : bad;
    up2(az[k], u, v); res[k].z = ok ? u + v : bad;
  }

  bool write = true;
  if (a.jsplit > 1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      int i = ibase + k * THREADS + tid;
      if (i < a.n)
        a.part[(size_t)jc * a.n + i] = make_float4(res[k].x, res[k].y, res[k].z, 0.f);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      unsigned tk = atomicAdd(&a.tickets[itile], 1u);
      *s_last = tk == (unsigned)a.jsplit - 1u;
      if (*s_last) a.tickets[itile] = 0u;   // ready for the next launch
    }
    __syncthreads();
    write = *s_last;
    if (write) {
      __threadfence();
#pragma unroll
      for (int k = 0; k < K; ++k) {
        int i = ibase + k * THREADS + tid;
        float3 sum = make_float3(0.f, 0.f, 0.f);
        if (i < a.n) {
          for (int js = 0; js < a.jsplit; ++js) {
            float4 p = __ldcg(&a.part[(size_t)js * a.n + i]);
            sum.x += p.x; sum.y += p.y; sum.z += p.z;
          }
        }
        res[k] = sum;
      }
    }
    __syncthreads();   // s_last is read by every thread before it is reused
  }
  if (!write) return;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    int i = ibase + k * THREADS + tid;
    if (i >= a.n) continue;
    float4 acc = make_float4(a.G * res[k].x, a.G * res[k].y, a.G * res[k].z, 0.f);
    a.acc[i] = acc;
    if (a.vel) {
      float4 v = a.vel[i];
      v.x = __fmaf_rn(a.half_dt, acc.x, v.x);
      v.y = __fmaf_rn(a.half_dt, acc.y, v.y);
      v.z = __fmaf_rn(a.half_dt, acc.z, v.z);
      a.vel[i] = v;
    }
  }
}

__device__ __forceinline__ void ap_ring_init(uint64_t* s_bar) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&s_bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
}

template <int THREADS, int K>
__global__ void __launch_bounds__(THREADS) k_allpairs(APArgs a) {
  __shared__ __align__(128) float4 s_tile[kStages][kTileF4];
  __shared__ __align__(8) uint64_t s_bar[kStages];
  __shared__ bool s_last;
  ap_ring_init(s_bar);
  uint32_t tc = 0;
  ap_item<THREADS, K>(a, blockIdx.x, blockIdx.y, s_tile, s_bar, &s_last, tc);
}

// Many simulations' all-pairs forces in one persistent launch: each CTA pops
// work items (simulation, target tile, source chunk) from a device queue
// until it is empty.  Each simulation keeps the source chunking (jsplit) of
// its own geometry, so its sums, and its results, equal the ones it gets
// alone.  Items are ordered longest chunks first.

template <int THREADS, int K>
__global__ void __launch_bounds__(THREADS) k_allpairs_queue(APQueue q) {
  __shared__ __align__(128) float4 s_tile[kStages][kTileF4];
  __shared__ __align__(8) uint64_t s_bar[kStages];
  __shared__ bool s_last;
  __shared__ int s_item;
  ap_ring_init(s_bar);
  uint32_t tc = 0;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(q.counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();   // read by all before thread 0 writes the next one
    if (it >= q.nitems) break;
    const int4 w = q.items[it];   // the same item for every thread: uniform
    if (w.x < 0 || w.x >= q.nsims) {
      if (threadIdx.x == 0) raise_err(q.err, NB_DEVERR_QUEUE);
      continue;
    }
    APArgs a = q.sims[w.x];
    if (w.y < 0 || (long long)w.y * THREADS * K >= a.n || w.z < 0 || w.z >= a.jsplit) {
      if (threadIdx.x == 0) raise_err(q.err, NB_DEVERR_QUEUE);
      continue;
    }
    if (!q.kick) a.vel = nullptr;
    ap_item<THREADS, K>(a, w.y, w.z, s_tile, s_bar, &s_last, tc);
  }
}

// Geometry: THREADS x K targets per CTA (the compiled shapes below); the
// source range is split over jsplit CTAs per target tile so that about
// `ctas` CTAs are in flight (the tuning table's choice for this size).
APGeom allpairs_geometry_for(int n, int threads, int k, int ctas) {
  APGeom g;
  g.threads = threads;
  g.k = k;
  const int per = g.threads * g.k;
  g.itiles = (n + per - 1) / per;
  const int npad = (n + kSrcTile - 1) / kSrcTile * kSrcTile;
  const int jtiles = npad / kSrcTile;
  int js = (ctas + g.itiles - 1) / g.itiles;
  if (js > jtiles) js = jtiles;
  if (js < 1) js = 1;
  // round the chunk to whole tiles and recompute the split it implies
  const int jt_per = (jtiles + js - 1) / js;
  g.jsplit = (jtiles + jt_per - 1) / jt_per;
  return g;
}

APGeom allpairs_geometry(int n) {
  int threads = 256, k = 4, ctas = 0;
  tune_allpairs(n, &threads, &k, &ctas);
  return allpairs_geometry_for(n, threads, k, ctas);
}

bool allpairs_shape_compiled(int threads, int k) {
  return (threads == 128 || threads == 256) && (k == 2 || k == 4 || k == 8);
}

template <int T, int K>
static void launch_ap(const APArgs& a, const APGeom& g, cudaStream_t st) {
  k_allpairs<T, K><<<dim3(g.itiles, g.jsplit), T, 0, st>>>(a);
}

int launch_allpairs_geom(Workspace& w, const StepArgs& s, const APGeom& g,
                         cudaStream_t st) {
  if (!allpairs_shape_compiled(g.threads, g.k))
    return set_error(NB_ERR_INVALID, "all-pairs shape " + std::to_string(g.threads) +
                                         " x " + std::to_string(g.k) + " is not compiled");
  NB_TRY(ws_reserve_allpairs(w, s.n, g));
  APArgs a;
  a.n = s.n;
  a.pos = s.pos;
  a.src = w.src;
  a.npad = (s.n + kSrcTile - 1) / kSrcTile * kSrcTile;
  a.jsplit = g.jsplit;
  const int jtiles = a.npad / kSrcTile;
  a.jchunk = (jtiles + g.jsplit - 1) / g.jsplit * kSrcTile;
  a.eps2 = s.eps2;
  a.G = s.G;
  a.half_dt = s.half_dt;
  a.acc = s.acc;
  a.vel = s.kick_after ? s.vel : nullptr;
  a.part = w.part;
  a.tickets = w.tickets;
  a.err = w.err;
  switch (g.threads * 16 + g.k) {
    case 128 * 16 + 2: launch_ap<128, 2>(a, g, st); break;
    case 128 * 16 + 4: launch_ap<128, 4>(a, g, st); break;
    case 128 * 16 + 8: launch_ap<128, 8>(a, g, st); break;
    case 256 * 16 + 2: launch_ap<256, 2>(a, g, st); break;
    case 256 * 16 + 8: launch_ap<256, 8>(a, g, st); break;
    default: launch_ap<256, 4>(a, g, st); break;
  }
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

int launch_allpairs(Workspace& w, const StepArgs& s, cudaStream_t st) {
  return launch_allpairs_geom(w, s, allpairs_geometry(s.n), st);
}

// ---------------------------------------------------------------------------
// Batches (ensembles, the server): the all-pairs simulations' work.
// ---------------------------------------------------------------------------

// Packs the sources of the all-pairs simulations: warp b takes 32-slot block
// b; a simulation's slots past its n are zero-mass pads, as are the packed
// pairs past its last block (the buffer is zeroed once).
__global__ void k_ens_pack(EnsArgs e, const int* __restrict__ src_off,
                           float4* __restrict__ src) {
  const int lane = threadIdx.x & 31;
  const int blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (blk >= e.nblocks) return;
  const int s = e.blk_sim[blk];
  if (s < 0) return;
  const SimDesc d = e.sims[s];
  const int off = src_off[s];
  if (off < 0 || !d.active) return;
  const int local = blk * 32 - d.base + lane;
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  if (local < d.n) p = e.pos[blk * 32 + lane];
  const float x1 = __shfl_down_sync(0xffffffffu, p.x, 1);
  const float y1 = __shfl_down_sync(0xffffffffu, p.y, 1);
  const float z1 = __shfl_down_sync(0xffffffffu, p.z, 1);
  const float m1 = __shfl_down_sync(0xffffffffu, p.w, 1);
  if (!(lane & 1)) {
    float4* q = src + off + local;   // pair local / 2 at float4 2 (local / 2)
    q[0] = make_float4(p.x, x1, p.y, y1);
    q[1] = make_float4(p.z, z1, p.w, m1);
  }
}

size_t ap_region_f4(int n) {
  const APGeom g = allpairs_geometry(n);
  const size_t npad = (size_t)(n + kSrcTile - 1) / kSrcTile * kSrcTile;
  const size_t part = g.jsplit > 1 ? (size_t)g.jsplit * n : 0;
  const size_t tick = ((size_t)g.itiles + 3) / 4;
  return (npad + part + tick + 15) / 16 * 16;
}

size_t plan_ens_allpairs(const SimDesc* sims, int nsims, const size_t* region_of,
                         EnsAllPairs& ap, const size_t* region_cap, int* too_small) {
  if (too_small) *too_small = 0;
  ap.args.clear();
  ap.sim.clear();
  ap.region.clear();
  ap.items.clear();
  ap.groups.clear();
  ap.src_off.assign(nsims, -1);
  struct Pending { int a; APGeom g; };
  std::vector<Pending> todo;
  size_t next = 0, top = 0;
  for (int s = 0; s < nsims; ++s) {
    const SimDesc& d = sims[s];
    if (!d.active || d.force != NB_FORCE_NAIVE) continue;
    const APGeom g = allpairs_geometry(d.n);
    const int npad = (d.n + kSrcTile - 1) / kSrcTile * kSrcTile;
    APArgs a{};
    a.n = d.n;
    a.npad = npad;
    a.jsplit = g.jsplit;
    a.jchunk = (npad / kSrcTile + g.jsplit - 1) / g.jsplit * kSrcTile;
    a.eps2 = d.eps2;
    a.G = d.G;
    a.half_dt = d.half_dt;
    const size_t r = region_of ? region_of[s] : next;
    next = r + ap_region_f4(d.n);
    if (region_cap && ap_region_f4(d.n) > region_cap[s]) {   // the table changed
      if (too_small) ++*too_small;
      continue;
    }
    top = std::max(top, next);
    ap.src_off[s] = (int)r;
    todo.push_back({(int)ap.args.size(), g});
    ap.args.push_back(a);
    ap.sim.push_back(s);
    ap.region.push_back(r);
  }
  // one group per launch shape; items longest chunks first
  for (int threads : {128, 256})
    for (int k : {2, 4, 8}) {
      EnsAllPairs::Group grp{threads, k, (int)ap.items.size(), 0};
      std::vector<int4> its;
      for (const Pending& p : todo) {
        if (p.g.threads != threads || p.g.k != k) continue;
        for (int jc = 0; jc < p.g.jsplit; ++jc)
          for (int it = 0; it < p.g.itiles; ++it) its.push_back(make_int4(p.a, it, jc, 0));
      }
      if (its.empty()) continue;
      std::stable_sort(its.begin(), its.end(), [&](const int4& x, const int4& y) {
        return ap.args[x.x].jchunk > ap.args[y.x].jchunk;
      });
      ap.items.insert(ap.items.end(), its.begin(), its.end());
      grp.nitems = (int)its.size();
      ap.groups.push_back(grp);
    }
  return top;
}

int bind_ens_allpairs(EnsAllPairs& ap, const SimDesc* sims, int nsims, const EnsArgs& e,
                      cudaStream_t st) {
  for (size_t i = 0; i < ap.args.size(); ++i) {
    const SimDesc& d = sims[ap.sim[i]];
    APArgs& a = ap.args[i];
    float4* reg = ap.d_pool + ap.region[i];
    a.pos = e.pos + d.base;
    a.src = reg;
    a.acc = e.acc + d.base;
    a.vel = (d.active == 1) ? e.vel + d.base : nullptr;
    a.part = reg + a.npad;
    a.tickets = reinterpret_cast<unsigned*>(reg + a.npad + (a.jsplit > 1 ? (size_t)a.jsplit * a.n : 0));
    a.err = e.err;
  }
  if (!ap.args.empty())
    NB_CUDA(cudaMemcpyAsync(ap.d_args, ap.args.data(), sizeof(APArgs) * ap.args.size(),
                            cudaMemcpyHostToDevice, st));
  if (!ap.items.empty())
    NB_CUDA(cudaMemcpyAsync(ap.d_items, ap.items.data(), sizeof(int4) * ap.items.size(),
                            cudaMemcpyHostToDevice, st));
  NB_CUDA(cudaMemcpyAsync(ap.d_src_off, ap.src_off.data(), sizeof(int) * nsims,
                          cudaMemcpyHostToDevice, st));
  return NB_OK;
}

template <int T, int K>
static void launch_queue(const APQueue& q, int grid, cudaStream_t st) {
  k_allpairs_queue<T, K><<<grid, T, 0, st>>>(q);
}

int launch_ens_allpairs(const EnsArgs& e, const EnsAllPairs& ap, cudaStream_t st) {
  if (ap.groups.empty()) return NB_OK;
  k_ens_pack<<<(e.nblocks * 32 + 255) / 256, 256, 0, st>>>(e, ap.d_src_off, ap.d_pool);
  NB_CUDA(cudaGetLastError());
  NB_CUDA(cudaMemsetAsync(ap.d_counter, 0, sizeof(int) * ap.groups.size(), st));
  const int sms = device_sm_count();
  for (size_t gi = 0; gi < ap.groups.size(); ++gi) {
    const EnsAllPairs::Group& g = ap.groups[gi];
    APQueue q;
    q.sims = ap.d_args;
    q.items = ap.d_items + g.first_item;
    q.nitems = g.nitems;
    q.counter = ap.d_counter + gi;
    q.nsims = (int)ap.args.size();
    q.err = e.err;
    q.kick = e.kick_after ? 1 : 0;
    // persistent: about two CTAs of 256 threads per SM, no more than items
    const int grid = std::min(g.nitems, sms * (g.threads == 128 ? 4 : 2));
    switch (g.threads * 16 + g.k) {
      case 128 * 16 + 2: launch_queue<128, 2>(q, grid, st); break;
      case 128 * 16 + 4: launch_queue<128, 4>(q, grid, st); break;
      case 128 * 16 + 8: launch_queue<128, 8>(q, grid, st); break;
      case 256 * 16 + 2: launch_queue<256, 2>(q, grid, st); break;
      case 256 * 16 + 8: launch_queue<256, 8>(q, grid, st); break;
      default: launch_queue<256, 4>(q, grid, st); break;
    }
    NB_CUDA(cudaGetLastError());
  }
  return NB_OK;
}

// ---------------------------------------------------------------------------
// Energy.  PE = -1/2 G sum_i m_i (phi_i - self_i), phi_i = sum_j m_j
// rsqrt(r_ij^2 + eps^2) including j == i (removed again with the same float
// rsqrt(eps^2) the loop used for it).  Pair math in FP32, per-tile partial
// sums converted to FP64; KE, PE and momentum reduced in FP64 in a fixed
// order (block partials, then the last block).
// ---------------------------------------------------------------------------
constexpr int kEThreads = 256;
constexpr int kETile = 256;

__global__ void __launch_bounds__(kEThreads) k_energy_phi(
    const float4* __restrict__ pos, int n, float eps2, int jchunk,
    double* __restrict__ phi_part) {
  __shared__ float4 s_src[kETile];
  const int i = blockIdx.x * kEThreads + threadIdx.x;
  const float4 bi = pos[i < n ? i : n - 1];
  const int j0 = blockIdx.y * jchunk;
  const int j1 = min(j0 + jchunk, n);
  double phi = 0.0;
  for (int jt = j0; jt < j1; jt += kETile) {
    int j = jt + threadIdx.x;
    s_src[threadIdx.x] = j < j1 ? pos[j] : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    float acc = 0.f;
#pragma unroll 8
    for (int q = 0; q < kETile; ++q) {
      float4 s = s_src[q];
      float dx = s.x - bi.x, dy = s.y - bi.y, dz = s.z - bi.z;
      float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
      acc = fmaf(s.w, mufu_rsqrt(__fadd_rn(r2, eps2)), acc);
    }
    phi += (double)acc;
    __syncthreads();
  }
  if (i < n) phi_part[(size_t)blockIdx.y * n + i] = phi;
}

__global__ void __launch_bounds__(kEThreads) k_energy_reduce(
    const float4* __restrict__ pos, const float4* __restrict__ vel, int n,
    float eps2, float G, int jsplit, const double* __restrict__ phi_part,
    double* __restrict__ epart, unsigned* ticket, double* out) {
  __shared__ double s_r[kEThreads / 32][5];
  __shared__ bool s_last;
  double r[5] = {0, 0, 0, 0, 0};   // KE, PE, Px, Py, Pz
  const double self_inv = (double)mufu_rsqrt(eps2);
  for (int i = blockIdx.x * kEThreads + threadIdx.x; i < n;
       i += gridDim.x * kEThreads) {
    float4 p = pos[i];
    float4 v = vel[i];
    double m = (double)p.w;
    double phi = 0.0;
    for (int js = 0; js < jsplit; ++js) phi += phi_part[(size_t)js * n + i];
    double self = (double)__fmul_rn(p.w, (float)self_inv);
    r[0] += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    r[1] += m * (phi - self);
    r[2] += m * v.x;
    r[3] += m * v.y;
    r[4] += m * v.z;
  }
#pragma unroll
  for (int c = 0; c < 5; ++c)
    for (int o = 16; o > 0; o >>= 1) r[c] += __shfl_down_sync(0xffffffffu, r[c], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int c = 0; c < 5; ++c) s_r[warp][c] = r[c];
  __syncthreads();
  if (threadIdx.x < 5) {
    double v = 0.0;
    for (int w = 0; w < kEThreads / 32; ++w) v += s_r[w][threadIdx.x];
    epart[blockIdx.x * 5 + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double t[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < (int)gridDim.x; ++b)
      for (int c = 0; c < 5; ++c) t[c] += __ldcg(&epart[b * 5 + c]);
    double ke = t[0];
    double pe = -0.5 * (double)G * t[1];
    out[0] = ke + pe;
    out[1] = ke;
    out[2] = pe;
    out[3] = t[2];
    out[4] = t[3];
    out[5] = t[4];
    *ticket = 0u;
  }
}

int launch_energy(Workspace& w, int n, const float4* pos, const float4* vel,
                  float eps2, float G, cudaStream_t st) {
  const int itiles = (n + kEThreads - 1) / kEThreads;
  const int sms = device_sm_count();
  int js = (sms * 4 + itiles - 1) / itiles;
  const int jt = (n + kETile - 1) / kETile;
  if (js > jt) js = jt;
  if (js < 1) js = 1;
  int jchunk = (jt + js - 1) / js * kETile;
  js = (n + jchunk - 1) / jchunk;
  int rblocks = (n + kEThreads - 1) / kEThreads;
  if (rblocks > 2 * sms) rblocks = 2 * sms;
  NB_TRY(ws_reserve_energy(w, n, rblocks, js));
  k_energy_phi<<<dim3(itiles, js), kEThreads, 0, st>>>(pos, n, eps2, jchunk,
                                                        w.ephi);
  NB_CUDA(cudaGetLastError());
  k_energy_reduce<<<rblocks, kEThreads, 0, st>>>(
      pos, vel, n, eps2, G, js, w.ephi, w.epart, w.eticket, w.eout);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// ---------------------------------------------------------------------------
// All-pairs forces with no allocation at all (nb_compute_forces_naive_static).
//
// Some callers cannot allocate device memory when they need forces: a host
// application that owns every device allocation itself (a fixed memory
// budget reserved at start-up, an allocator that is closed after
// initialisation, a plugin that must not grow the process's footprint).
// Such a caller hands over its particle and acceleration buffers and gets
// the same all-pairs accelerations as nb_compute_forces_dev with
// NB_FORCE_NAIVE, computed by the same kernel, but with the scratch it needs
// (packed sources, per-chunk partial sums, tile tickets) taken from the
// file-scope device array below instead of from a workspace.
//
// The array is sized for kStaticMaxN particles and at most kStaticMaxSplit
// source chunks per target tile: about 4.6 MB, held on every GPU that loads
// the library until the process exits.  Every call shares it and it keeps
// the previous call's contents; the tickets, the only part that must start at
// zero, are cleared at the start of each call.  Calls whose GPU work overlaps
// (different streams, or different host threads on one device) race on the
// array and must be serialised by the caller.
// ---------------------------------------------------------------------------
constexpr int kStaticMaxN = 32768;
constexpr int kStaticMaxSplit = 8;
constexpr size_t kStaticSrcBytes = (size_t)kStaticMaxN * sizeof(float4);
constexpr size_t kStaticPartBytes = (size_t)kStaticMaxSplit * kStaticMaxN * sizeof(float4);
constexpr size_t kStaticTailBytes = 256;   // tickets (<= 33 words) + error word
constexpr int kStaticErrWord = 48;          // word index of the error word in the tail
static __device__ __align__(256) unsigned char
    g_static_scratch[kStaticSrcBytes + kStaticPartBytes + kStaticTailBytes];

// Packs positions into the pair-interleaved source layout (zero-mass pad).
__global__ void k_pack_static(const float4* __restrict__ pos, int n, int npairs,
                              float4* __restrict__ src) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npairs;
       q += gridDim.x * blockDim.x) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 a = 2 * q < n ? pos[2 * q] : z;
    const float4 b = 2 * q + 1 < n ? pos[2 * q + 1] : z;
    src[2 * q] = make_float4(a.x, b.x, a.y, b.y);
    src[2 * q + 1] = make_float4(a.z, b.z, a.w, b.w);
  }
}

// Device address of g_static_scratch for the current device.  Host code may
// not pass the symbol itself (in host code it names a host-side stand-in), so
// the address is looked up once per device with that device current.
static int static_scratch_address(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[64] = {};
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(NB_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess)
      return set_error(NB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_static_scratch): ") +
                                        cudaGetErrorString(e));
    addr[dev] = (unsigned char*)p;
  }
  *out = addr[dev];
  return NB_OK;
}

int warm_allpairs_kernels() {
  return warm_fns(k_allpairs<128, 2>, k_allpairs<128, 4>, k_allpairs<128, 8>,
                  k_allpairs<256, 2>, k_allpairs<256, 4>, k_allpairs<256, 8>,
                  k_allpairs_queue<128, 2>, k_allpairs_queue<128, 4>,
                  k_allpairs_queue<128, 8>, k_allpairs_queue<256, 2>,
                  k_allpairs_queue<256, 4>, k_allpairs_queue<256, 8>, k_ens_pack,
                  k_pack_static, k_energy_phi, k_energy_reduce);
}

}  // namespace nb

extern "C" int nb_compute_forces_naive_static(int n, const float* d_pos4,
                                              float* d_acc4, float eps, float G,
                                              void* stream) {
  using namespace nb;
  if (!d_pos4 || !d_acc4) return set_error(NB_ERR_INVALID, "NULL device pointer");
  if (n <= 0) return set_error(NB_ERR_INVALID, "n must be > 0");
  if (n > kStaticMaxN)
    return set_error(NB_ERR_INVALID,
                     "n = " + std::to_string(n) + " exceeds the " +
                         std::to_string(kStaticMaxN) +
                         "-particle limit of nb_compute_forces_naive_static's "
                         "fixed scratch; use nb_compute_forces_dev");
  if (!(eps > 0.f) || !std::isfinite(eps) || !std::isfinite(G))
    return set_error(NB_ERR_INVALID, "eps must be a finite value > 0 and G finite");
  unsigned char* base = nullptr;
  NB_TRY(static_scratch_address(&base));
  cudaStream_t st = (cudaStream_t)stream;
  float4* src = (float4*)base;
  float4* part = (float4*)(base + kStaticSrcBytes);
  unsigned* tail = (unsigned*)(base + kStaticSrcBytes + kStaticPartBytes);
  NB_CUDA(cudaMemsetAsync(tail, 0, kStaticTailBytes, st));

  // a fixed shape (256 x 4, 8 CTAs per SM wanted), independent of tuning
  APGeom g = allpairs_geometry_for(n, 256, 4, device_sm_count() * 8);
  const int npad = (n + kSrcTile - 1) / kSrcTile * kSrcTile;
  const int jtiles = npad / kSrcTile;
  int js = g.jsplit < kStaticMaxSplit ? g.jsplit : kStaticMaxSplit;
  const int jt_per = (jtiles + js - 1) / js;
  js = (jtiles + jt_per - 1) / jt_per;

  const int npairs = npad / 2;
  k_pack_static<<<(npairs + 255) / 256, 256, 0, st>>>((const float4*)d_pos4, n,
                                                      npairs, src);
  NB_CUDA(cudaGetLastError());
  APArgs a;
  a.n = n;
  a.pos = (const float4*)d_pos4;
  a.src = src;
  a.npad = npad;
  a.jsplit = js;
  a.jchunk = jt_per * kSrcTile;
  a.eps2 = eps * eps;
  a.G = G;
  a.half_dt = 0.f;
  a.acc = (float4*)d_acc4;
  a.vel = nullptr;
  a.part = part;
  a.tickets = tail;
  a.err = tail + kStaticErrWord;
  k_allpairs<256, 4><<<dim3(g.itiles, js), 256, 0, st>>>(a);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_compute_forces_naive_static_status(unsigned* device_error,
                                                     void* stream) {
  using namespace nb;
  unsigned char* base = nullptr;
  NB_TRY(static_scratch_address(&base));
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned* word =
      (const unsigned*)(base + kStaticSrcBytes + kStaticPartBytes) + kStaticErrWord;
  unsigned e = 0;
  NB_CUDA(cudaMemcpyAsync(&e, word, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(st));
  if (device_error) *device_error = e;
  if (e)
    return set_error(NB_ERR_DEVICE,
                     "nb_compute_forces_naive_static: device error word 0x" +
                         std::to_string(e) +
                         (e & NB_DEVERR_WAIT ? " (bulk-copy barrier wait limit; the rows "
                                               "of the blocks that gave up are NaN)"
                                             : ""));
  return NB_OK;
}
