// Default Barnes-Hut walks (walk_kernel = 0): the reference's interaction
// sets (src/forces_bh.cu:335-447), computed a warp-wide batch of nodes at a
// time instead of one node per warp step.
//
// A warp owns 32 consecutive Morton-sorted targets.  It keeps a stack of
// candidate nodes in shared memory and repeatedly takes up to 32 of them, one
// per lane:
//
// * a leaf becomes an interaction-list entry;
// * an internal node is decided against all targets at once.  A conservative
//   test against the box of the 32 targets settles most nodes: if even the
//   nearest point of the box accepts (size2 < theta2 * dmin2, with a 1e-5
//   margin far above the 4e-7 rounding of the exact test), every target
//   accepts; if even the farthest point rejects, every target rejects.  Only
//   nodes in between run the exact per-target test (walk_common.cuh), so the
//   decisions equal the per-target float tests bit for bit.
//
// Semantics:
// * warp mode (traverse = warp, src/forces_bh.cu:395-447): a node opens when
//   any live target rejects it; otherwise all targets take it;
// * thread mode (traverse = thread, src/forces_bh.cu:335-377): each candidate
//   carries the mask of targets whose own walk reaches it; targets that
//   accept take it (entry with that mask), those that reject pass their mask
//   to the children.  Every target gets exactly its per-thread interaction
//   set.
//
// Accepted nodes and leaves go to a shared-memory interaction list (pairs of
// entries interleaved as (x0,x1,y0,y1)(z0,z1,m0,m1)) that the lanes evaluate
// for their own target with packed FP32 math, two entries per instruction,
// in blocks of 32 entries by an unrolled body (the last, partial block by a
// loop).  Entries whose mask excludes a lane contribute with mass 0.
//
// If the candidate stack would overflow, the warp falls back to the
// depth-first walk of the same semantics (same interaction set).
#include "f32x2.cuh"
#include "walk_common.cuh"

namespace nb {

constexpr int kLW = 4;          // warps per block
// candidate stack entries per warp: warp semantics 1024; thread semantics
// 512 (its stack holds a subset of the warp semantics' candidates; the
// smaller shared-memory footprint gives 64 registers and 8 resident blocks
// per SM instead of 94 and 5, a 12 % faster walk at 1M); past either, the
// depth-first fallback takes over
constexpr int kCand = 1024;
template <bool MASKED>
constexpr int cand_cap() { return MASKED ? 512 : kCand; }
constexpr int kFlush = 32;      // list entries evaluated per flush
constexpr int kList = 2 * kFlush;   // interaction-list entries per warp

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Shared memory of one block: per warp a candidate stack (+ lane masks), the
// interaction list (+ masks), the staged ambiguous nodes and their ballots.
template <bool MASKED>
struct ListSmem {
  int cid[kLW][cand_cap<MASKED>()];
  unsigned cmask[kLW][MASKED ? cand_cap<MASKED>() : 1];
  __align__(16) float ent[kLW][kList * 4];
  unsigned emask[kLW][MASKED ? kList : 1];
  __align__(16) float amb[kLW][32 * 4];   // ambiguous nodes, pairs
  unsigned res[kLW][32];                  // their accept ballots
  float4 ext[kLW][MASKED ? 1 : 6];        // targets of min / max x, y, z
};

// (v, v) in one 64-bit register pair, made at each use: volatile, so that
// the compiler does not hoist the pairs and keep them live through the whole
// walk (56 registers instead of 62: 9 resident blocks per SM instead of 8)
__device__ __forceinline__ f2 pk2v(float v) {
  f2 r;
  asm volatile("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(v));
  return r;
}

// The walk of warp `wg` (targets 32wg .. 32wg+31 of the tree in `a`); all
// 32 lanes of the warp call it.  HOIST keeps the packed copies of the target
// in registers for the whole walk (fewer registers the other way in the
// single-tree kernel, more in the ensemble kernel, whose parameters are not
// kernel constants).
template <bool MASKED, bool COUNT, bool HOIST = false>
__device__ __forceinline__ void walk_list_warp(const WalkArgs& a, int wg,
                                               ListSmem<MASKED>& sm) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int n = a.n, ni = n - 1;
  if (wg * 32 >= a.t1) return;   // whole warp past the end of the range
  const int t = wg * 32 + lane;
  const bool live = t < n;
  const unsigned live_mask = __ballot_sync(full, live);
  const unsigned lt = (1u << lane) - 1u;
  // dead lanes (last warp only) copy particle n-1, a live lane of this warp,
  // so the group box is the box of the live targets
  const float4 bi = a.ps[live ? t : n - 1];
  const float lox = warp_min(bi.x), loy = warp_min(bi.y), loz = warp_min(bi.z);
  const float hix = warp_max(bi.x), hiy = warp_max(bi.y), hiz = warp_max(bi.z);
  const float theta2 = a.theta2;
  // the box test's thresholds with a 1e-5 relative margin, far above the
  // few-ulp rounding of either side of the exact per-target test
  const float th_lo = theta2 * 0.99999f, th_hi = theta2 * 1.00001f;
  if (!MASKED) {
    // the targets at the group's extremes (warp semantics: one rejecting
    // target opens a node for all)
    const float lv[6] = {lox, hix, loy, hiy, loz, hiz};
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const float c = (e < 2) ? bi.x : (e < 4 ? bi.y : bi.z);
      const int src = __ffs(__ballot_sync(full, c == lv[e])) - 1;
      const float ex = __shfl_sync(full, bi.x, src), ey = __shfl_sync(full, bi.y, src),
                  ez = __shfl_sync(full, bi.z, src);
      if (lane == 0) sm.ext[w][e] = make_float4(ex, ey, ez, 0.f);
    }
  }
  const float cmx = 0.5f * (lox + hix), cmy = 0.5f * (loy + hiy), cmz = 0.5f * (loz + hiz);

  const float mx = -bi.x, my = -bi.y, mz = -bi.z;   // this lane's target, negated
  const f2 hx = pk2(mx, mx), hy = pk2(my, my), hz = pk2(mz, mz), he2 = pk2(a.eps2, a.eps2);
  auto px = [&]() { return HOIST ? hx : pk2v(mx); };
  auto py = [&]() { return HOIST ? hy : pk2v(my); };
  auto pz = [&]() { return HOIST ? hz : pk2v(mz); };
  f2 ax = 0ull, ay = 0ull, az = 0ull;
  int cnt = 0;
  float* ent = sm.ent[w];

  // list pair q (entries 2q, 2q+1) for this lane's target
  auto pair_term = [&](int q) {
    const ulonglong2 A = *reinterpret_cast<const ulonglong2*>(&ent[q * 8]);
    const ulonglong2 B = *reinterpret_cast<const ulonglong2*>(&ent[q * 8 + 4]);
    f2 m = B.y;
    if (MASKED) {
      const unsigned b0 = (sm.emask[w][2 * q] >> lane) & 1u;
      const unsigned b1 = (sm.emask[w][2 * q + 1] >> lane) & 1u;
      float m0, m1;
      up2(B.y, m0, m1);
      m = pk2(b0 ? m0 : 0.f, b1 ? m1 : 0.f);
      if (COUNT) cnt += (int)(b0 + b1);
    }
    f2 dx = add2(A.x, px());
    f2 dy = add2(A.y, py());
    f2 dz = add2(B.x, pz());
    f2 r2 = fma2(dz, dz, HOIST ? he2 : pk2v(a.eps2));
    r2 = fma2(dy, dy, r2);
    r2 = fma2(dx, dx, r2);
    float r0, r1;
    up2(r2, r0, r1);
    f2 inv = pk2(mufu_rsqrt(r0), mufu_rsqrt(r1));
    f2 wm = mul2(inv, m);
    f2 i2 = mul2(inv, inv);
    f2 f = mul2(wm, i2);
    ax = fma2(dx, f, ax);
    ay = fma2(dy, f, ay);
    az = fma2(dz, f, az);
  };
  // evaluates list entries [0, lc) for this lane's target (the last, partial
  // list of the walk)
  auto flush = [&](int lc) {
    if (lc & 1) {   // pad to a whole pair with a zero-mass entry
      if (lane == 0) {
        float* p = &ent[(lc >> 1) * 8 + 1];
        p[0] = 0.f; p[2] = 0.f; p[4] = 0.f; p[6] = 0.f;
        if (MASKED) sm.emask[w][lc] = 0u;
      }
      __syncwarp();
    }
    const int np = (lc + 1) >> 1;
    for (int q = 0; q < np; ++q) pair_term(q);
    if (!MASKED && COUNT) cnt += lc;
    __syncwarp();
  };
  // evaluates entries [0, kFlush) (unrolled: no loop counter, fixed
  // offsets), then moves entries [kFlush, lc) to the front (lc < kFlush + 32);
  // returns the new count
  auto flush_full = [&](int lc) {
#pragma unroll
    for (int q = 0; q < kFlush / 2; ++q) pair_term(q);
    if (!MASKED && COUNT) cnt += kFlush;
    __syncwarp();
    const int rest = lc - kFlush;   // 0 .. 31
    if (lane < ((rest + 1) >> 1) * 2) {   // whole pairs, two float4 each
      float4* v = reinterpret_cast<float4*>(ent);
      v[lane] = v[kFlush + lane];
    }
    if (MASKED && lane < rest) sm.emask[w][lane] = sm.emask[w][kFlush + lane];
    __syncwarp();
    return rest;
  };

  int sp = 1, lc = 0;
  if (lane == 0) {
    sm.cid[w][0] = 0;   // root
    if (MASKED) sm.cmask[w][0] = live_mask;
  }
  __syncwarp();
  bool overflow = false;
  for (int guard = 0; sp > 0; ++guard) {
    if (sp + 32 > cand_cap<MASKED>() || guard > 2 * n) {   // uniform across the warp
      overflow = true;
      break;
    }
    const int take = min(sp, 32);
    const int base = sp - take;
    const bool has = lane < take;
    int id = 0;
    unsigned M = live_mask;
    if (has) {
      id = sm.cid[w][base + lane];
      if (MASKED) M = sm.cmask[w][base + lane];
    }
    __syncwarp();
    sp = base;

    bool want_ent = false, want_push = false;
    float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned emask = 0u, pmask = 0u, accm = 0u;
    int cl = 0, cr = 0;
    float s2 = 0.f;
    bool amb = false;
    const bool is_int = has && id < ni;
    if (has && id >= ni) {
      e = a.ps[id - ni];
      want_ent = true;
      emask = M;
    } else if (is_int) {
      const Node nd = a.nodes[id];
      e = nd.com;
      cl = nd.left;
      cr = nd.right;
      s2 = nd.size2;
      const float cx = e.x, cy = e.y, cz = e.z;
      // per axis: distance below the box's low face and above its high face
      // (at most one is positive); the nearest box point lies max(.., 0)
      // away, the farthest max(|..|) away
      const float lx = lox - cx, hx = cx - hix;
      const float ly = loy - cy, hy = cy - hiy;
      const float lz = loz - cz, hz = cz - hiz;
      const float ex = fmaxf(fmaxf(lx, hx), 0.f);
      const float ey = fmaxf(fmaxf(ly, hy), 0.f);
      const float ez = fmaxf(fmaxf(lz, hz), 0.f);
      const float dmin2 = ex * ex + ey * ey + ez * ez;
      const float fx = fmaxf(fabsf(lx), fabsf(hx));
      const float fy = fmaxf(fabsf(ly), fabsf(hy));
      const float fz = fmaxf(fabsf(lz), fabsf(hz));
      const float dmax2 = fx * fx + fy * fy + fz * fz;
      if (s2 < th_lo * dmin2) {
        accm = M;
      } else if (s2 > th_hi * dmax2) {
        accm = 0u;
      } else if (MASKED) {
        amb = true;
      } else {
        // warp semantics: if the group's extreme target along the node's
        // dominant direction rejects it (the exact per-target test), the
        // node opens; otherwise it goes to the test of every target
        const float rx = cx - cmx, ry = cy - cmy, rz = cz - cmz;
        const float qx = fabsf(rx), qy = fabsf(ry), qz = fabsf(rz);
        const int e = (qx >= qy && qx >= qz) ? (rx > 0.f ? 1 : 0)
                                             : (qy >= qz ? (ry > 0.f ? 3 : 2) : (rz > 0.f ? 5 : 4));
        const float4 q = sm.ext[w][e];
        amb = accepts(s2, theta2, cx, cy, cz, q.x, q.y, q.z);
      }
    }
    // nodes the box cannot settle: their owners stage them in shared memory
    // (pairs interleaved as (cx0,cx1,cy0,cy1)(cz0,cz1,s0,s1)); every lane
    // tests its own target against two of them per packed instruction, in
    // the float order of accepts(), and one ballot per node is written back
    const unsigned ambb = __ballot_sync(full, amb);
    if (ambb) {
      const int na = __popc(ambb);
      const int ka = __popc(ambb & lt);
      if (amb) {
        float* p = &sm.amb[w][(ka >> 1) * 8 + (ka & 1)];
        p[0] = e.x; p[2] = e.y; p[4] = e.z; p[6] = s2;
      }
      if (na & 1) {   // pad: a node every target accepts (size2 = -1)
        if (lane == 0) {
          float* p = &sm.amb[w][(na >> 1) * 8 + 1];
          p[0] = 0.f; p[2] = 0.f; p[4] = 0.f; p[6] = -1.f;
        }
      }
      __syncwarp();
      const f2 th2 = pk2(theta2, theta2);
      for (int q = 0; q < (na + 1) >> 1; ++q) {
        const ulonglong2 A = *reinterpret_cast<const ulonglong2*>(&sm.amb[w][q * 8]);
        const ulonglong2 B = *reinterpret_cast<const ulonglong2*>(&sm.amb[w][q * 8 + 4]);
        const f2 dx = add2(A.x, px()), dy = add2(A.y, py()), dz = add2(B.x, pz());
        const f2 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
        float t0, t1, z0, z1;
        up2(mul2(th2, d2), t0, t1);
        up2(B.y, z0, z1);
        // a dead lane tests a copy of live target n-1 (warp semantics), and
        // the candidate masks hold live lanes only (thread semantics)
        const unsigned b0 = __ballot_sync(full, z0 < t0);
        const unsigned b1 = __ballot_sync(full, z1 < t1);
        if (lane == 0) {
          sm.res[w][2 * q] = b0;
          sm.res[w][2 * q + 1] = b1;
        }
      }
      __syncwarp();
      if (amb) accm = sm.res[w][ka] & M;
    }
    if (is_int) {
      if (MASKED) {
        if (accm) {
          want_ent = true;
          emask = accm;
        }
        const unsigned om = M & ~accm;
        if (om) {
          want_push = true;
          pmask = om;
        }
      } else if (accm == M) {
        want_ent = true;
      } else {
        want_push = true;
      }
    }
    const unsigned eb = __ballot_sync(full, want_ent);
    if (want_ent) {
      const int k = lc + __popc(eb & lt);
      float* p = &ent[(k >> 1) * 8 + (k & 1)];
      p[0] = e.x; p[2] = e.y; p[4] = e.z; p[6] = e.w;
      if (MASKED) sm.emask[w][k] = emask;
    }
    lc += __popc(eb);
    const unsigned pb = __ballot_sync(full, want_push);
    if (want_push) {
      const int k = sp + 2 * __popc(pb & lt);
      sm.cid[w][k] = cl;
      sm.cid[w][k + 1] = cr;
      if (MASKED) {
        sm.cmask[w][k] = pmask;
        sm.cmask[w][k + 1] = pmask;
      }
    }
    sp += 2 * __popc(pb);
    __syncwarp();
    if (lc >= kFlush) lc = flush_full(lc);
  }

  float3 ai;
  if (!overflow) {
    if (lc) flush(lc);
    float u, v;
    up2(ax, u, v); ai.x = u + v;
    up2(ay, u, v); ai.y = u + v;
    up2(az, u, v); ai.z = u + v;
  } else {
    // same interaction set by the depth-first walk; the candidate stack's
    // shared memory serves as the warp stack
    cnt = 0;
    __syncwarp();
    if (MASKED)
      ai = dfs_walk_thread<COUNT>(a, bi, &cnt);
    else
      ai = dfs_walk_warp<COUNT>(a, bi, live, sm.cid[w], &cnt);
  }
  if (live) {
    epilogue(a, t, ai);
    if (COUNT) a.counts[t] = cnt;
  }
}

template <bool MASKED, bool COUNT>
__global__ void __launch_bounds__(kLW * 32) k_walk_list(WalkArgs a) {
  __shared__ ListSmem<MASKED> sm;
  walk_list_warp<MASKED, COUNT>(a, a.t0 / 32 + blockIdx.x * kLW + (threadIdx.x >> 5), sm);
}

int launch_walk_list(const WalkArgs& a, bool masked, cudaStream_t st) {
  const int warps = (a.t1 - a.t0 + 31) / 32;
  if (warps <= 0) return NB_OK;
  const int blocks = (warps + kLW - 1) / kLW;
  if (masked) {
    if (a.counts) k_walk_list<true, true><<<blocks, kLW * 32, 0, st>>>(a);
    else k_walk_list<true, false><<<blocks, kLW * 32, 0, st>>>(a);
  } else {
    if (a.counts) k_walk_list<false, true><<<blocks, kLW * 32, 0, st>>>(a);
    else k_walk_list<false, false><<<blocks, kLW * 32, 0, st>>>(a);
  }
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

int warm_walk_list_kernels() {
  return warm_fns(k_walk_list<false, false>, k_walk_list<false, true>,
                  k_walk_list<true, false>, k_walk_list<true, true>);
}

}  // namespace nb
