// Default Barnes-Hut walk (walk_kernel = 0): the reference's interaction sets
// (src/forces_bh.cu:335-447) computed from the tree's child-pair records.
//
// A warp owns 32 consecutive Morton-sorted targets and keeps a stack of
// opened internal nodes in shared memory, each as the split whose pair record
// (PairRec, nb_internal.cuh) holds its two children.  Each warp step takes up
// to 32 opened nodes, one per lane, and every lane decides both children of
// its node from one 48-byte record fetch:
//
// * a leaf (size2 = -1) is accepted by every test: it becomes an
//   interaction-list entry;
// * an internal child is accepted by every target when even the nearest point
//   of the box of the 32 targets accepts it (size2 < theta2 * dmin2 with a
//   1e-5 relative margin, far above the few-ulp rounding of the exact test);
// * warp semantics: otherwise the group's extreme target along the child's
//   dominant direction is tested exactly, and its rejection opens the child
//   (a farthest-box-point rejection implies it, so that test is not needed);
// * thread semantics: a child that even the farthest box point rejects is
//   rejected by every target;
// * the children still undecided are staged in shared memory and every lane
//   tests its own target against two of them per packed instruction, in the
//   float order of accepts() (walk_common.cuh), so every decision equals the
//   per-target float test bit for bit.
//
// Warp semantics (traverse = warp, src/forces_bh.cu:395-447): a child opens
// when any live target rejects it, otherwise all targets take it.  Thread
// semantics (traverse = thread, src/forces_bh.cu:335-377): each opened node
// carries the mask of the targets whose own walk opened it; the targets that
// accept a child take it (an entry with their mask) and the others pass it on
// opened.  Either way every target gets exactly the reference's set.
//
// Entries go to a 128-entry ring per warp (pairs interleaved as
// (x0,x1,y0,y1)(z0,z1,m0,m1)), evaluated 32 at a time by an unrolled body
// with packed FP32 math, two entries per instruction; entries whose mask
// excludes a lane contribute with mass 0.  A stack that would overflow hands
// the warp to a depth-first walk of the same semantics over the same records.
#include <algorithm>
#include <cmath>
#include <vector>

#include "f32x2.cuh"
#include "walk_common.cuh"

namespace nb {

constexpr int kPStack = 512;      // opened-node entries per warp
constexpr int kPRing = 128;       // interaction-list ring entries per warp
constexpr int kPFlush = 32;       // entries evaluated per flush
constexpr int kPAmb = 64;         // children staged for the all-target test

// Shared memory of a block of W warps.
template <int W, bool MASKED>
struct PairSmem {
  int stk[W][kPStack];
  unsigned smask[W][MASKED ? kPStack : 1];
  __align__(16) float ent[W][kPRing * 4];
  unsigned emask[W][MASKED ? kPRing : 1];
  __align__(16) float amb[W][kPAmb * 4];
  unsigned res[W][kPAmb];
  float4 ext[W][MASKED ? 1 : 6];
};

__device__ __forceinline__ float pw_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float pw_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// (v, v) in one register pair, made at each use (volatile: not hoisted and
// kept live through the walk)
__device__ __forceinline__ f2 pk2u(float v) {
  f2 r;
  asm volatile("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(v));
  return r;
}

// Writes one list entry (x, y, z, m) at ring position k.
__device__ __forceinline__ void put_entry(float* ent, int k, float x, float y,
                                          float z, float m) {
  k &= kPRing - 1;
  float* p = &ent[(k >> 1) * 8 + (k & 1)];
  p[0] = x;
  p[2] = y;
  p[4] = z;
  p[6] = m;
}

// Squared distance from (cx, cy, cz) to the nearest / farthest point of the
// box [lo, hi] (rounded; the callers' margins cover it).
__device__ __forceinline__ float box_near2(float cx, float cy, float cz, float lox,
                                           float loy, float loz, float hix,
                                           float hiy, float hiz) {
  const float ex = fmaxf(fmaxf(lox - cx, cx - hix), 0.f);
  const float ey = fmaxf(fmaxf(loy - cy, cy - hiy), 0.f);
  const float ez = fmaxf(fmaxf(loz - cz, cz - hiz), 0.f);
  return ex * ex + ey * ey + ez * ez;
}
__device__ __forceinline__ float box_far2(float cx, float cy, float cz, float lox,
                                          float loy, float loz, float hix,
                                          float hiy, float hiz) {
  const float fx = fmaxf(fabsf(lox - cx), fabsf(cx - hix));
  const float fy = fmaxf(fabsf(loy - cy), fabsf(cy - hiy));
  const float fz = fmaxf(fabsf(loz - cz), fabsf(cz - hiz));
  return fx * fx + fy * fy + fz * fz;
}

// One tree node as the pair layout holds it: centre of mass (a leaf: its
// position) and mass in c, size2 (-1 for a leaf, which every opening test
// accepts) and the split whose record holds its children (-1 for a leaf).
struct PairNode {
  float4 c;
  float size2;
  int split;
};

__device__ __forceinline__ PairNode pair_child(const PairRec* __restrict__ pr, int k,
                                               int side) {
  PairNode nd;
  nd.c = pr[k].c[side];
  const float2 h = reinterpret_cast<const float2*>(&pr[k].sw)[side];
  nd.size2 = h.x;
  nd.split = __float_as_int(h.y);
  return nd;
}

__device__ __forceinline__ PairNode pair_root(const WalkArgs& a) {
  const PairRec* r = a.pairs + (a.n - 1);
  PairNode nd;
  nd.c = r->c[0];
  nd.size2 = r->sw.x;
  nd.split = __float_as_int(r->sw.y);
  return nd;
}

// Depth-first walks over the child-pair records, for warps whose stack of
// opened nodes would overflow: the per-target walk (src/forces_bh.cu:335-377)
// and the warp-shared one (src/forces_bh.cu:395-447), right child first, with
// the reference's opening test; a leaf (size2 = -1) always interacts.  Stack
// entries are 2 * split + side.  `stack` (warp walk): this warp's
// shared-memory stack of at least kStack entries, written by lane 0 and read
// after __syncwarp.
template <bool COUNT>
__device__ float3 dfs_pair_thread(const WalkArgs& a, float4 bi, int* cnt_out) {
  const int ni = a.n - 1;
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int stack[kStack];
  int sp = 0;
  PairNode nd = pair_root(a);
  for (int visits = 0;; ++visits) {   // a valid tree: at most 2n - 1 visits
    if (visits >= 2 * a.n) {
      raise_err(a.err, NB_DEVERR_VISITS);
      break;
    }
    const float dx = __fsub_rn(nd.c.x, bi.x), dy = __fsub_rn(nd.c.y, bi.y),
                dz = __fsub_rn(nd.c.z, bi.z);
    const float d2 = dist2(dx, dy, dz);
    if (nd.size2 < __fmul_rn(a.theta2, d2)) {
      pair_term(ai, dx, dy, dz, d2, nd.c.w, a.eps2);
      if (COUNT) ++cnt;
    } else {
      if (sp >= kStack || (unsigned)nd.split >= (unsigned)ni) {
        raise_err(a.err, sp >= kStack ? NB_DEVERR_STACK : NB_DEVERR_TREE);
        break;
      }
      stack[sp++] = 2 * nd.split;
      nd = pair_child(a.pairs, nd.split, 1);
      continue;
    }
    if (sp == 0) break;
    const int e = stack[--sp];
    nd = pair_child(a.pairs, e >> 1, e & 1);
  }
  if (COUNT) *cnt_out = cnt;
  return ai;
}

template <bool COUNT>
__device__ float3 dfs_pair_warp(const WalkArgs& a, float4 bi, bool live, int* stack,
                                int* cnt_out) {
  const int lane = threadIdx.x & 31;
  const int ni = a.n - 1;
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int sp = 0;
  PairNode nd = pair_root(a);
  for (int visits = 0;; ++visits) {
    if (visits >= 2 * a.n) {
      if (lane == 0) raise_err(a.err, NB_DEVERR_VISITS);
      break;
    }
    const float dx = __fsub_rn(nd.c.x, bi.x), dy = __fsub_rn(nd.c.y, bi.y),
                dz = __fsub_rn(nd.c.z, bi.z);
    const float d2 = dist2(dx, dy, dz);
    const bool open = live && !(nd.size2 < __fmul_rn(a.theta2, d2));
    if (__any_sync(0xffffffffu, open)) {   // uniform: nd is the same in every lane
      if (sp >= kStack || (unsigned)nd.split >= (unsigned)ni) {
        if (lane == 0) raise_err(a.err, sp >= kStack ? NB_DEVERR_STACK : NB_DEVERR_TREE);
        break;
      }
      if (lane == 0) stack[sp] = 2 * nd.split;
      ++sp;
      __syncwarp();
      nd = pair_child(a.pairs, nd.split, 1);
      continue;
    }
    pair_term(ai, dx, dy, dz, d2, nd.c.w, a.eps2);
    if (COUNT) ++cnt;
    if (sp == 0) break;
    --sp;
    const int e = stack[sp];
    __syncwarp();   // all lanes have read the slot before it is reused
    nd = pair_child(a.pairs, e >> 1, e & 1);
  }
  if (COUNT) *cnt_out = cnt;
  return ai;
}

// The walk of warp `wg` (targets 32wg .. 32wg+31); all 32 lanes call it.
template <int W, bool MASKED, bool COUNT, bool HOIST = false>
__device__ __forceinline__ void walk_pair_warp(const WalkArgs& a, int wg,
                                               PairSmem<W, MASKED>& sm) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int n = a.n, ni = n - 1;
  if (wg * 32 >= a.t1) return;   // whole warp past the end of the range
  const int t = wg * 32 + lane;
  const bool live = t < n;
  const unsigned live_mask = __ballot_sync(full, live);
  const unsigned lt = (1u << lane) - 1u;
  // dead lanes (last warp only) copy particle n-1, a live lane of this warp,
  // so the group box is the box of the live targets and a dead lane's exact
  // tests repeat a live lane's
  const float4 bi = a.ps[live ? t : n - 1];
  const float lox = pw_min(bi.x), loy = pw_min(bi.y), loz = pw_min(bi.z);
  const float hix = pw_max(bi.x), hiy = pw_max(bi.y), hiz = pw_max(bi.z);
  const float theta2 = a.theta2;
  const float th_lo = theta2 * 0.99999f, th_hi = theta2 * 1.00001f;
  if (!MASKED) {
    // the targets at the group's extremes (warp semantics: one rejecting
    // target opens a child for all)
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
  auto px = [&]() { return HOIST ? hx : pk2u(mx); };
  auto py = [&]() { return HOIST ? hy : pk2u(my); };
  auto pz = [&]() { return HOIST ? hz : pk2u(mz); };
  f2 ax = 0ull, ay = 0ull, az = 0ull;
  int cnt = 0;
  float* ent = sm.ent[w];
  int head = 0;   // ring position of the first unevaluated entry (multiple of 32)
  int lc = 0;     // unevaluated entries

  // list pair q of the 32-entry block at ring position `at`; (qx, qy, qz)
  // the packed negated target and e2 the packed eps^2, made once per block
  auto pair_term = [&](int at, int q, f2 qx, f2 qy, f2 qz, f2 e2) {
    const float* base = &ent[at * 4];
    const ulonglong2 A = *reinterpret_cast<const ulonglong2*>(&base[q * 8]);
    const ulonglong2 B = *reinterpret_cast<const ulonglong2*>(&base[q * 8 + 4]);
    f2 m = B.y;
    if (MASKED) {
      // the pair's two lane masks in one load (at + 2q is even, the row
      // 16-byte aligned); this lane's bit keeps or zeroes each mass
      const uint2 mk = *reinterpret_cast<const uint2*>(&sm.emask[w][at + 2 * q]);
      const unsigned lbit = lt + 1u;
      const bool b0 = (mk.x & lbit) != 0u, b1 = (mk.y & lbit) != 0u;
      float m0, m1;
      up2(B.y, m0, m1);
      m = pk2(b0 ? m0 : 0.f, b1 ? m1 : 0.f);
      if (COUNT) cnt += (int)b0 + (int)b1;
    }
    f2 dx = add2(A.x, qx);
    f2 dy = add2(A.y, qy);
    f2 dz = add2(B.x, qz);
    f2 r2 = fma2(dz, dz, e2);
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
  // evaluates the 32 entries at `head` (unrolled, fixed offsets)
  auto flush_full = [&]() {
    const f2 qx = px(), qy = py(), qz = pz(), e2 = HOIST ? he2 : pk2u(a.eps2);
#pragma unroll
    for (int q = 0; q < kPFlush / 2; ++q) pair_term(head, q, qx, qy, qz, e2);
    if (!MASKED && COUNT) cnt += kPFlush;
    head = (head + kPFlush) & (kPRing - 1);
    lc -= kPFlush;
  };

  // the root: one exact test per target (dead lanes repeat a live one)
  int sp = 0;
  {
    const PairNode root = pair_root(a);
    const bool acc = accepts(root.size2, theta2, root.c.x, root.c.y, root.c.z,
                             bi.x, bi.y, bi.z);
    const int sc0 = min(max(root.split, 0), ni - 1);   // a valid tree never needs the clamp
    const unsigned am = MASKED ? (__ballot_sync(full, acc) & live_mask)
                               : (__all_sync(full, acc) ? live_mask : 0u);
    if (lane == 0) {
      if (am) {
        put_entry(ent, 0, root.c.x, root.c.y, root.c.z, root.c.w);
        if (MASKED) sm.emask[w][0] = am;
      }
      if (am != live_mask) {
        sm.stk[w][0] = sc0;
        if (MASKED) sm.smask[w][0] = live_mask & ~am;
      }
    }
    lc = am ? 1 : 0;
    sp = am != live_mask ? 1 : 0;
    __syncwarp();
  }

  bool overflow = false;
  for (int guard = 0; sp > 0; ++guard) {
    if (sp + 32 > kPStack || guard > n) {   // uniform across the warp
      overflow = true;
      break;
    }
    const int take = min(sp, 32);
    const int base = sp - take;
    const bool has = lane < take;
    int k = 0;
    unsigned M = live_mask;
    if (has) {
      k = sm.stk[w][base + lane];
      if (MASKED) M = sm.smask[w][base + lane];
    }
    __syncwarp();
    sp = base;
    k = min(max(k, 0), ni - 1);   // a valid tree never needs the clamp
    float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0, sw = c0;
    if (has) {
      const PairRec* r = a.pairs + k;
      c0 = r->c[0];
      c1 = r->c[1];
      sw = r->sw;
    }
    // child j: position / centre of mass (cj.x, cj.y, cj.z), mass cj.w,
    // size2 and split in sw (.x, .y for the left child, .z, .w the right)
    const float s0 = sw.x, s1 = sw.z;
    const int w0 = __float_as_int(sw.y), w1 = __float_as_int(sw.w);
    const bool in0 = w0 >= 0, in1 = w1 >= 0;   // internal children
    const f2 dn = pk2(box_near2(c0.x, c0.y, c0.z, lox, loy, loz, hix, hiy, hiz),
                      box_near2(c1.x, c1.y, c1.z, lox, loy, loz, hix, hiy, hiz));
    float tn0, tn1;
    up2(mul2(pk2u(th_lo), dn), tn0, tn1);
    const bool bacc0 = s0 < tn0, bacc1 = s1 < tn1;   // leaves: -1 < anything >= 0
    bool amb0, amb1, brej0 = false, brej1 = false;
    if (MASKED) {
      const f2 df = pk2(box_far2(c0.x, c0.y, c0.z, lox, loy, loz, hix, hiy, hiz),
                        box_far2(c1.x, c1.y, c1.z, lox, loy, loz, hix, hiy, hiz));
      float tf0, tf1;
      up2(mul2(pk2u(th_hi), df), tf0, tf1);
      brej0 = !bacc0 && s0 > tf0;
      brej1 = !bacc1 && s1 > tf1;
      amb0 = has && !bacc0 && !brej0;
      amb1 = has && !bacc1 && !brej1;
    } else {
      // the group's extreme target along the child's dominant direction
      // from the box centre; its exact rejection opens the child
      auto ext_accepts = [&](float s2, float cx, float cy, float cz) {
        const float rx = cx - cmx, ry = cy - cmy, rz = cz - cmz;
        const float qx = fabsf(rx), qy = fabsf(ry), qz = fabsf(rz);
        const int e = (qx >= qy && qx >= qz) ? (rx > 0.f ? 1 : 0)
                                             : (qy >= qz ? (ry > 0.f ? 3 : 2) : (rz > 0.f ? 5 : 4));
        const float4 q = sm.ext[w][e];
        return accepts(s2, theta2, cx, cy, cz, q.x, q.y, q.z);
      };
      amb0 = has && !bacc0 && ext_accepts(s0, c0.x, c0.y, c0.z);
      amb1 = has && !bacc1 && ext_accepts(s1, c1.x, c1.y, c1.z);
    }
    // children the box and the extreme target cannot settle: staged in
    // shared memory (pairs interleaved as (cx0,cx1,cy0,cy1)(cz0,cz1,s0,s1));
    // every lane tests its own target against two per packed instruction, in
    // the float order of accepts(), and one ballot per child is written back
    unsigned r0 = 0u, r1 = 0u;
    const unsigned ab0 = __ballot_sync(full, amb0), ab1 = __ballot_sync(full, amb1);
    if (ab0 | ab1) {
      const int na0 = __popc(ab0), na = na0 + __popc(ab1);
      const int ka0 = __popc(ab0 & lt), ka1 = na0 + __popc(ab1 & lt);
      float* am = sm.amb[w];
      if (amb0) {
        float* p = &am[(ka0 >> 1) * 8 + (ka0 & 1)];
        p[0] = c0.x; p[2] = c0.y; p[4] = c0.z; p[6] = s0;
      }
      if (amb1) {
        float* p = &am[(ka1 >> 1) * 8 + (ka1 & 1)];
        p[0] = c1.x; p[2] = c1.y; p[4] = c1.z; p[6] = s1;
      }
      if ((na & 1) && lane == 0) {   // pad: a child every target accepts
        float* p = &am[(na >> 1) * 8 + 1];
        p[0] = 0.f; p[2] = 0.f; p[4] = 0.f; p[6] = -1.f;
      }
      __syncwarp();
      const f2 th2 = pk2(theta2, theta2);
      const f2 qx = px(), qy = py(), qz = pz();
      // warp semantics need only "every target accepts": a vote every lane
      // receives, kept in a warp-uniform bit mask; thread semantics need the
      // accepting lanes, one ballot per child through shared memory
      unsigned long long allacc = 0ull;
      for (int q = 0; q < (na + 1) >> 1; ++q) {
        const ulonglong2 U = *reinterpret_cast<const ulonglong2*>(&am[q * 8]);
        const ulonglong2 V = *reinterpret_cast<const ulonglong2*>(&am[q * 8 + 4]);
        const f2 dx = add2(U.x, qx), dy = add2(U.y, qy), dz = add2(V.x, qz);
        const f2 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
        float t0, t1, z0, z1;
        up2(mul2(th2, d2), t0, t1);
        up2(V.y, z0, z1);
        if (MASKED) {
          const unsigned v0 = __ballot_sync(full, z0 < t0);
          const unsigned v1 = __ballot_sync(full, z1 < t1);
          if (lane == 0) {
            sm.res[w][2 * q] = v0;
            sm.res[w][2 * q + 1] = v1;
          }
        } else {
          // a dead lane tests a copy of live target n-1
          const unsigned long long b0 = __all_sync(full, z0 < t0) ? 1ull : 0ull;
          const unsigned long long b1 = __all_sync(full, z1 < t1) ? 2ull : 0ull;
          allacc |= (b0 | b1) << (2 * q);
        }
      }
      if (MASKED) {
        __syncwarp();
        if (amb0) r0 = sm.res[w][ka0];
        if (amb1) r1 = sm.res[w][ka1];
      } else {
        r0 = (unsigned)(allacc >> ka0) & 1u;
        r1 = (unsigned)(allacc >> ka1) & 1u;
      }
    }
    // accepting targets of each child
    unsigned acc0, acc1;
    if (MASKED) {
      acc0 = bacc0 ? M : (amb0 ? (r0 & M) : 0u);
      acc1 = bacc1 ? M : (amb1 ? (r1 & M) : 0u);
    } else {
      acc0 = (bacc0 || (amb0 && r0)) ? M : 0u;
      acc1 = (bacc1 || (amb1 && r1)) ? M : 0u;
    }
    const bool ent0 = has && acc0 != 0u, ent1 = has && acc1 != 0u;
    const bool psh0 = has && acc0 != M && in0, psh1 = has && acc1 != M && in1;
    const unsigned eb0 = __ballot_sync(full, ent0), eb1 = __ballot_sync(full, ent1);
    const int ne0 = __popc(eb0);
    if (ent0) {
      const int e = head + lc + __popc(eb0 & lt);
      put_entry(ent, e, c0.x, c0.y, c0.z, c0.w);
      if (MASKED) sm.emask[w][e & (kPRing - 1)] = acc0;
    }
    if (ent1) {
      const int e = head + lc + ne0 + __popc(eb1 & lt);
      put_entry(ent, e, c1.x, c1.y, c1.z, c1.w);
      if (MASKED) sm.emask[w][e & (kPRing - 1)] = acc1;
    }
    lc += ne0 + __popc(eb1);
    const unsigned pb0 = __ballot_sync(full, psh0), pb1 = __ballot_sync(full, psh1);
    const int np0 = __popc(pb0);
    if (psh0) {
      const int s = sp + __popc(pb0 & lt);
      sm.stk[w][s] = w0;
      if (MASKED) sm.smask[w][s] = M & ~acc0;
    }
    if (psh1) {
      const int s = sp + np0 + __popc(pb1 & lt);
      sm.stk[w][s] = w1;
      if (MASKED) sm.smask[w][s] = M & ~acc1;
    }
    sp += np0 + __popc(pb1);
    __syncwarp();
    while (lc >= kPFlush) flush_full();
    __syncwarp();
  }

  float3 ai;
  if (!overflow) {
    if (lc) {   // the last, partial block (lc < 32, contiguous at head)
      if (lc & 1) {   // pad to a whole pair with a zero-mass entry
        if (lane == 0) {
          put_entry(ent, head + lc, 0.f, 0.f, 0.f, 0.f);
          if (MASKED) sm.emask[w][(head + lc) & (kPRing - 1)] = 0u;
        }
        __syncwarp();
      }
      const int np = (lc + 1) >> 1;
      const f2 qx = px(), qy = py(), qz = pz(), e2 = HOIST ? he2 : pk2u(a.eps2);
      for (int q = 0; q < np; ++q) pair_term(head, q, qx, qy, qz, e2);
      if (!MASKED && COUNT) cnt += lc;
    }
    float u, v;
    up2(ax, u, v); ai.x = u + v;
    up2(ay, u, v); ai.y = u + v;
    up2(az, u, v); ai.z = u + v;
  } else {
    // same interaction set by the depth-first walk; the stack's shared
    // memory serves as the warp stack
    cnt = 0;
    __syncwarp();
    if (MASKED)
      ai = dfs_pair_thread<COUNT>(a, bi, &cnt);
    else
      ai = dfs_pair_warp<COUNT>(a, bi, live, sm.stk[w], &cnt);
  }
  if (live) {
    epilogue(a, t, ai);
    if (COUNT) a.counts[t] = cnt;
  }
}

// At most 64 registers a thread: 32 warps resident per SM whatever the block
// shape (the compiler otherwise takes 70 for 8-warp blocks).
template <int W, bool MASKED, bool COUNT>
__global__ void __launch_bounds__(W * 32, 32 / W) k_walk_pair(WalkArgs a) {
  __shared__ PairSmem<W, MASKED> sm;
  chain_wait();
  walk_pair_warp<W, MASKED, COUNT>(a, a.t0 / 32 + blockIdx.x * W + (threadIdx.x >> 5), sm);
}


// Ensembles and the server: one persistent launch per semantics.  Its warps
// pop 32-slot blocks of the concatenated sorted arrays from a device queue
// (costliest simulations first, so the longest walks do not start last) and
// walk each with that block's simulation: its tree, parameters and
// semantics.  Blocks belong to one simulation (bases are multiples of 32).
constexpr int kEnsW = 4;
template <bool MASKED>
__global__ void __launch_bounds__(kEnsW * 32) k_walk_pair_ens(EnsArgs e) {
  __shared__ PairSmem<kEnsW, MASKED> sm;
  const int lane = threadIdx.x & 31;
  const int* items = e.walk_items[MASKED ? 1 : 0];
  const int nitems = e.walk_nitems[MASKED ? 1 : 0];
  int* ctr = e.walk_ctr + (MASKED ? 1 : 0);
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(ctr, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= nitems) return;
    const int blk = items[it];
    const int s = (blk >= 0 && blk < e.nblocks) ? e.blk_sim[blk] : -1;
    if (s < 0 || s >= e.nsims) {   // a stale or corrupt item: skipped, reported
      if (lane == 0) raise_err(e.err, NB_DEVERR_QUEUE);
      continue;
    }
    const SimDesc d = e.sims[s];
    if (!d.active || d.n < 2 || d.force != NB_FORCE_BH ||
        (d.traverse == NB_TRAVERSE_THREAD) != MASKED)
      continue;
    WalkArgs a;
    a.n = d.n;
    a.ps = e.pos_sorted + d.base;
    a.perm = e.perm + d.base;
    a.nodes = nullptr;   // the pair layout is the whole tree here
    a.pairs = e.pairs + d.base;
    a.theta2 = d.theta2;
    a.eps2 = d.eps2;
    a.G = d.G;
    a.half_dt = d.half_dt;
    a.acc = e.acc;
    a.vel = (e.kick_after && d.active == 1) ? e.vel : nullptr;
    a.counts = nullptr;
    a.perm_limit = e.nslots;
    a.err = e.err;
    a.t0 = 0;
    a.t1 = d.n;
    a.part = nullptr;
    walk_pair_warp<kEnsW, MASKED, false, true>(a, blk - d.base / 32, sm);
    __syncwarp();   // this warp's shared memory is free for its next block
  }
}

void plan_walk_queue(const SimDesc* sims, int nsims, std::vector<int> items[2]) {
  items[0].clear();
  items[1].clear();
  std::vector<int> order;
  for (int s = 0; s < nsims; ++s)
    if (sims[s].active && sims[s].n >= 2 && sims[s].force == NB_FORCE_BH) order.push_back(s);
  auto weight = [&](int s) {   // a warp's walk grows with log n and falls with theta
    const float th = std::max(std::sqrt(sims[s].theta2), 0.05f);
    return std::log2((float)sims[s].n) / (th * std::sqrt(th));
  };
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return weight(x) > weight(y); });
  for (int s : order) {
    const int q = sims[s].traverse == NB_TRAVERSE_THREAD ? 1 : 0;
    const int b0 = sims[s].base / 32, nb = (sims[s].n + 31) / 32;
    for (int b = 0; b < nb; ++b) items[q].push_back(b0 + b);
  }
}

int launch_walk_pair_ens(const EnsArgs& e, cudaStream_t st) {
  NB_CUDA(cudaMemsetAsync(e.walk_ctr, 0, 2 * sizeof(int), st));
  const int cap = device_sm_count() * 8;   // 8 resident blocks of 4 warps per SM
  for (int q = 0; q < 2; ++q) {
    const int n = e.walk_nitems[q];
    if (n <= 0) continue;
    const int blocks = std::min((n + kEnsW - 1) / kEnsW, cap);
    if (q == 0) k_walk_pair_ens<false><<<blocks, kEnsW * 32, 0, st>>>(e);
    else k_walk_pair_ens<true><<<blocks, kEnsW * 32, 0, st>>>(e);
  }
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

template <int W>
static int launch_walk_pair_w(const WalkArgs& a, bool masked, int blocks, cudaStream_t st) {
  if (masked) {
    // the lane masks double the stack: thread semantics stay at <= 4 warps
    // per block (<= 32 KB of static shared memory)
    constexpr int WM = W < 4 ? W : 4;
    const int bm = (blocks * W + WM - 1) / WM;
    return a.counts ? launch_chained(k_walk_pair<WM, true, true>, bm, WM * 32, 0, st, a)
                    : launch_chained(k_walk_pair<WM, true, false>, bm, WM * 32, 0, st, a);
  }
  return a.counts ? launch_chained(k_walk_pair<W, false, true>, blocks, W * 32, 0, st, a)
                  : launch_chained(k_walk_pair<W, false, false>, blocks, W * 32, 0, st, a);
}

// The block shape (warps per block) is the tuning table's.
int launch_walk_pair(const WalkArgs& a, bool masked, cudaStream_t st) {
  const int warps = (a.t1 - a.t0 + 31) / 32;
  if (warps <= 0) return NB_OK;
  const int W = tune_walk_warps();
  const int blocks = (warps + W - 1) / W;
  if (W == 2) return launch_walk_pair_w<2>(a, masked, blocks, st);
  if (W == 8) return launch_walk_pair_w<8>(a, masked, blocks, st);
  return launch_walk_pair_w<4>(a, masked, blocks, st);
}

int warm_walk_pair_kernels() {
  return warm_fns(k_walk_pair<2, false, false>, k_walk_pair<2, false, true>,
                  k_walk_pair<4, false, false>, k_walk_pair<4, false, true>,
                  k_walk_pair<8, false, false>, k_walk_pair<8, false, true>,
                  k_walk_pair<2, true, false>, k_walk_pair<2, true, true>,
                  k_walk_pair<4, true, false>, k_walk_pair<4, true, true>,
                  k_walk_pair_ens<false>, k_walk_pair_ens<true>);
}

}  // namespace nb
