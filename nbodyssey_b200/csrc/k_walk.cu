// Barnes-Hut tree walks over the LBVH (src/forces_bh.cu:335-447), with the
// leapfrog's closing kick fused into the epilogue.
//
// Opening test, in this exact float order (the CPU oracle repeats it, so the
// interaction sets match bit for bit):
//   d = com - x_i;  d2 = fma(dz, dz, fma(dy, dy, dx*dx));
//   accept  <=>  size2 < theta2 * d2
// Pair term: a += m * d * rsqrt(d2 + eps2)^3 (FP32, approximate rsqrt).
//
// Node fetches are 32-byte Node records (one sector); leaves are the
// Morton-sorted positions.  Both walks visit children right-first, as the
// reference's push-left-push-right stack does.
#include "nb_internal.cuh"

namespace nb {

struct WalkArgs {
  int n;
  const float4* __restrict__ ps;      // sorted positions
  const uint32_t* __restrict__ perm;  // sorted -> original
  const Node* __restrict__ nodes;
  float theta2, eps2, G, half_dt;
  float4* acc;       // original order
  float4* vel;       // closing kick target (original order) or nullptr
  int* counts;       // debug interaction counts (sorted order) or nullptr
  unsigned* err;
};

__device__ __forceinline__ void pair_term(float3& a, float dx, float dy,
                                          float dz, float d2, float m,
                                          float eps2) {
  float inv = mufu_rsqrt(__fadd_rn(d2, eps2));
  float f = m * inv * inv * inv;
  a.x = fmaf(dx, f, a.x);
  a.y = fmaf(dy, f, a.y);
  a.z = fmaf(dz, f, a.z);
}

__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

__device__ __forceinline__ void epilogue(const WalkArgs& a, int t, float3 ai) {
  const uint32_t o = a.perm[t];
  if (o >= (uint32_t)a.n) {   // only after a failed sort (error word set)
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

// --- per-thread walk (src/forces_bh.cu:335-377) -----------------------------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_walk_thread(WalkArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const int ni = a.n - 1;
  const float4 bi = a.ps[t];
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int stack[kStack];
  int sp = 0;
  int id = 0;   // root
  // a walk of a valid tree visits each of the 2n-1 nodes at most once
  for (int visits = 0;; ++visits) {
    if (visits >= 2 * a.n) {
      raise_err(a.err, NB_DEVERR_STACK);
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
  epilogue(a, t, ai);
  if (COUNT) a.counts[t] = cnt;
}

// --- warp-cooperative walk (src/forces_bh.cu:395-447) -----------------------
// The 32 lanes of a warp (32 consecutive Morton-sorted targets) share one
// walk: an internal node is opened when any live lane's test rejects it,
// otherwise every lane takes it as a point mass.  The stack lives in shared
// memory, one per warp; lane 0 writes, the warp reads after __syncwarp.  The
// next node to visit stays in a register, so only left children are stacked.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_walk_warp(WalkArgs a) {
  __shared__ int s_stack[256 / 32][kStack];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int wbase = t - lane;
  if (wbase >= a.n) return;   // whole warp past the end
  int* stack = s_stack[warp];
  const int ni = a.n - 1;
  const bool live = t < a.n;
  const float4 bi = a.ps[live ? t : a.n - 1];
  float3 ai = make_float3(0.f, 0.f, 0.f);
  int cnt = 0;
  int sp = 0;
  int id = 0;
  for (int visits = 0;; ++visits) {
    if (visits >= 2 * a.n) {
      if (lane == 0) raise_err(a.err, NB_DEVERR_STACK);
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
  if (live) {
    epilogue(a, t, ai);
    if (COUNT) a.counts[t] = cnt;
  }
}

int launch_walk(Workspace& w, const StepArgs& s, cudaStream_t st) {
  WalkArgs a;
  a.n = s.n;
  a.ps = w.pos_sorted;
  a.perm = w.vals;
  a.nodes = w.nodes;
  a.theta2 = s.theta2;
  a.eps2 = s.eps2;
  a.G = s.G;
  a.half_dt = s.half_dt;
  a.acc = s.acc;
  a.vel = s.kick_after ? s.vel : nullptr;
  a.counts = s.counts;
  a.err = w.err;
  int blocks = (s.n + 255) / 256;
  if (s.traverse == NB_TRAVERSE_WARP) {
    if (s.counts) k_walk_warp<true><<<blocks, 256, 0, st>>>(a);
    else k_walk_warp<false><<<blocks, 256, 0, st>>>(a);
  } else {
    if (s.counts) k_walk_thread<true><<<blocks, 256, 0, st>>>(a);
    else k_walk_thread<false><<<blocks, 256, 0, st>>>(a);
  }
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

}  // namespace nb
