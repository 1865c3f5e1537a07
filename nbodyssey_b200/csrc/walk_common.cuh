// Pieces shared by the tree walks (k_walk.cu, k_walk_list.cu, k_walk_pair.cu).
//
// Opening test, in this exact float order (the CPU oracle repeats it, so the
// interaction sets match bit for bit; src/forces_bh.cu:352-356):
//   d = com - x_i;  d2 = fma(dz, dz, fma(dy, dy, dx*dx));
//   accept  <=>  size2 < theta2 * d2
// Pair term: a += m * d * rsqrt(d2 + eps2)^3 (FP32, approximate rsqrt).
#pragma once

#include "nb_internal.cuh"

namespace nb {

struct WalkArgs {
  int n;
  const float4* __restrict__ ps;      // sorted positions
  const uint32_t* __restrict__ perm;  // sorted -> original
  const Node* __restrict__ nodes;     // Node records (walk kernels 1 and 2)
  const PairRec* __restrict__ pairs;  // child pairs by split (pair walk)
  float theta2, eps2, G, half_dt;
  float4* acc;       // original order
  float4* vel;       // closing kick target (original order) or nullptr
  int* counts;       // debug interaction counts (sorted order) or nullptr
  int perm_limit;    // permutation values must be below this (n, or the
                     // ensemble's slot count)
  unsigned* err;
  // sorted targets [t0, t1) are walked (multiples of 32, or n); with `part` set, part[t - t0] = G a of sorted target t instead of
  // the original-order output and the kick
  int t0, t1;
  float4* part;
};

__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

__device__ __forceinline__ bool accepts(float size2, float theta2, float cx,
                                        float cy, float cz, float x, float y,
                                        float z) {
  float d2 = dist2(__fsub_rn(cx, x), __fsub_rn(cy, y), __fsub_rn(cz, z));
  return size2 < __fmul_rn(theta2, d2);
}

__device__ __forceinline__ void pair_term(float3& a, float dx, float dy,
                                          float dz, float d2, float m,
                                          float eps2) {
  float inv = mufu_rsqrt(__fadd_rn(d2, eps2));
  float f = m * inv * inv * inv;
  a.x = fmaf(dx, f, a.x);
  a.y = fmaf(dy, f, a.y);
  a.z = fmaf(dz, f, a.z);
}

// acc[perm[t]] = G a, and the closing kick v += dt/2 acc when vel is set.
__device__ __forceinline__ void epilogue(const WalkArgs& a, int t, float3 ai) {
  if (a.part) {
    a.part[t - a.t0] = make_float4(a.G * ai.x, a.G * ai.y, a.G * ai.z, 0.f);
    return;
  }
  const uint32_t o = a.perm[t];
  if (o >= (uint32_t)a.perm_limit) {   // only after a failed sort (error word set)
    raise_err(a.err, NB_DEVERR_SORT);
    return;
  }
  float4 acc = make_float4(a.G * ai.x, a.G * ai.y, a.G * ai.z, 0.f);
  a.acc[o] = acc;
  if (a.vel) {
    float4 v = a.vel[o];
    v.x = __fmaf_rn(a.half_dt, acc.x, v.x);
    v.y = __fmaf_rn(a.half_dt, acc.y, v.y);
    v.z = __fmaf_rn(a.half_dt, acc.z, v.z);
    a.vel[o] = v;
  }
}

// Depth-first walk of one target with its own opening tests
// (src/forces_bh.cu:335-377).  Children are visited right first.
template <bool COUNT>
__device__ __forceinline__ float3 dfs_walk_thread(const WalkArgs& a, float4 bi,
                                                  int* cnt_out) {
  const int ni = a.n - 1;
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int stack[kStack];
  int sp = 0;
  int id = 0;   // root
  // a walk of a valid tree visits each of the 2n-1 nodes at most once
  for (int visits = 0;; ++visits) {
    if (visits >= 2 * a.n) {
      raise_err(a.err, NB_DEVERR_VISITS);
      break;
    }
    if (id >= ni) {
      const float4 s = a.ps[id - ni];
      float dx = __fsub_rn(s.x, bi.x), dy = __fsub_rn(s.y, bi.y),
            dz = __fsub_rn(s.z, bi.z);
      pair_term(ai, dx, dy, dz, dist2(dx, dy, dz), s.w, a.eps2);
      if (COUNT) ++cnt;
    } else {
      const Node nd = a.nodes[id];
      float dx = __fsub_rn(nd.com.x, bi.x), dy = __fsub_rn(nd.com.y, bi.y),
            dz = __fsub_rn(nd.com.z, bi.z);
      float d2 = dist2(dx, dy, dz);
      if (nd.size2 < __fmul_rn(a.theta2, d2)) {
        pair_term(ai, dx, dy, dz, d2, nd.com.w, a.eps2);
        if (COUNT) ++cnt;
      } else {
        if (sp >= kStack) {
          raise_err(a.err, NB_DEVERR_STACK);
          break;
        }
        stack[sp++] = nd.left;
        id = nd.right;
        continue;
      }
    }
    if (sp == 0) break;
    id = stack[--sp];
  }
  if (COUNT) *cnt_out = cnt;
  return ai;
}

// Depth-first shared walk of the warp's 32 targets (src/forces_bh.cu:
// 395-447): a node opens when any live lane's test rejects it; otherwise
// every lane takes it as a point mass.  `stack` is this warp's shared-memory
// stack of at least kStack entries; lane 0 writes, the warp reads after
// __syncwarp.  All 32 lanes must call it.
template <bool COUNT>
__device__ __forceinline__ float3 dfs_walk_warp(const WalkArgs& a, float4 bi,
                                                bool live, int* stack,
                                                int* cnt_out) {
  const int lane = threadIdx.x & 31;
  const int ni = a.n - 1;
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int sp = 0;
  int id = 0;
  for (int visits = 0;; ++visits) {
    if (visits >= 2 * a.n) {
      if (lane == 0) raise_err(a.err, NB_DEVERR_VISITS);
      break;
    }
    if (id >= ni) {
      const float4 s = a.ps[id - ni];
      float dx = __fsub_rn(s.x, bi.x), dy = __fsub_rn(s.y, bi.y),
            dz = __fsub_rn(s.z, bi.z);
      pair_term(ai, dx, dy, dz, dist2(dx, dy, dz), s.w, a.eps2);
      if (COUNT) ++cnt;
    } else {
      const Node nd = a.nodes[id];
      float dx = __fsub_rn(nd.com.x, bi.x), dy = __fsub_rn(nd.com.y, bi.y),
            dz = __fsub_rn(nd.com.z, bi.z);
      float d2 = dist2(dx, dy, dz);
      bool open = live && !(nd.size2 < __fmul_rn(a.theta2, d2));
      if (__any_sync(0xffffffffu, open)) {
        if (sp >= kStack) {
          if (lane == 0) raise_err(a.err, NB_DEVERR_STACK);
          break;
        }
        if (lane == 0) stack[sp] = nd.left;
        ++sp;
        __syncwarp();
        id = nd.right;
        continue;
      }
      pair_term(ai, dx, dy, dz, d2, nd.com.w, a.eps2);
      if (COUNT) ++cnt;
    }
    if (sp == 0) break;
    --sp;
    id = stack[sp];
    __syncwarp();   // all lanes have read the slot before it is reused
  }
  if (COUNT) *cnt_out = cnt;
  return ai;
}

int launch_walk_list(const WalkArgs& a, bool masked, cudaStream_t st);
int launch_walk_pair(const WalkArgs& a, bool masked, cudaStream_t st);

}  // namespace nb
