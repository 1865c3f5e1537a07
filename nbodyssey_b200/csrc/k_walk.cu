// Barnes-Hut tree walks over the LBVH (src/forces_bh.cu:335-447), with the
// leapfrog's closing kick fused into the epilogue.
//
// This file holds the depth-first walks that restate the reference kernels
// one node visit at a time (walk_kernel = 1): one walk per thread
// (traverse_kernel) and one shared walk per warp (traverse_warp_kernel).
// The default walks (walk_kernel = 0) are in k_walk_list.cu; they produce the
// same interaction sets with far fewer instructions.
//
// Node fetches are 32-byte Node records (one sector); leaves are the
// Morton-sorted positions.  Both walks visit children right-first, as the
// reference's push-left-push-right stack does.
#include "walk_common.cuh"

namespace nb {

// --- per-thread walk (src/forces_bh.cu:335-377) -----------------------------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_walk_thread(WalkArgs a) {
  const int t = a.t0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.t1) return;
  int cnt = 0;
  float3 ai = dfs_walk_thread<COUNT>(a, a.ps[t], &cnt);
  epilogue(a, t, ai);
  if (COUNT) a.counts[t] = cnt;
}

// --- warp-cooperative walk (src/forces_bh.cu:395-447) -----------------------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_walk_warp(WalkArgs a) {
  __shared__ int s_stack[256 / 32][kStack];
  const int lane = threadIdx.x & 31;
  const int t = a.t0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (t - lane >= a.t1) return;   // whole warp past the end of the range
  const bool live = t < a.n;
  int cnt = 0;
  float3 ai = dfs_walk_warp<COUNT>(a, a.ps[live ? t : a.n - 1], live,
                                   s_stack[threadIdx.x >> 5], &cnt);
  if (live) {
    epilogue(a, t, ai);
    if (COUNT) a.counts[t] = cnt;
  }
}

// --- the walk's sorted-order parts back to original order -------------------
// Same float operations as epilogue(): the result equals the fused walk's.
__global__ void __launch_bounds__(256) k_gather_part(const float4* __restrict__ sorted,
                                                     const uint32_t* __restrict__ perm,
                                                     int n, float half_dt, float4* acc,
                                                     float4* vel, unsigned* err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t o = perm ? perm[t] : (uint32_t)t;
  if (o >= (uint32_t)n) {
    raise_err(err, NB_DEVERR_SORT);
    return;
  }
  const float4 g = sorted[t];
  acc[o] = make_float4(g.x, g.y, g.z, 0.f);
  if (vel) {
    float4 v = vel[o];
    v.x = __fmaf_rn(half_dt, g.x, v.x);
    v.y = __fmaf_rn(half_dt, g.y, v.y);
    v.z = __fmaf_rn(half_dt, g.z, v.z);
    vel[o] = v;
  }
}

int launch_gather_part(Workspace& w, const StepArgs& a, const float4* sorted,
                       bool use_perm, cudaStream_t st) {
  k_gather_part<<<(a.n + 255) / 256, 256, 0, st>>>(sorted, use_perm ? w.vals : nullptr,
                                                   a.n, a.half_dt, a.acc, a.vel, w.err);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

int launch_walk(Workspace& w, const StepArgs& s, cudaStream_t st) {
  WalkArgs a;
  a.n = s.n;
  a.ps = w.pos_sorted;
  a.perm = w.vals;
  a.nodes = w.nodes;
  a.pairs = w.pairs;
  a.theta2 = s.theta2;
  a.eps2 = s.eps2;
  a.G = s.G;
  a.half_dt = s.half_dt;
  a.acc = s.acc;
  a.vel = s.kick_after ? s.vel : nullptr;
  a.counts = s.counts;
  a.perm_limit = s.n;
  a.err = w.err;
  a.t0 = s.t0;
  a.t1 = s.t1;
  a.part = s.part;
  if (s.walk_kernel == 0)
    return launch_walk_pair(a, s.traverse == NB_TRAVERSE_THREAD, st);
  if (s.walk_kernel == 2)
    return launch_walk_list(a, s.traverse == NB_TRAVERSE_THREAD, st);

  int blocks = (s.t1 - s.t0 + 255) / 256;
  if (blocks == 0) return NB_OK;
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

int warm_walk_kernels() {
  NB_TRY(warm_walk_pair_kernels());
  NB_TRY(warm_walk_list_kernels());
  return warm_fns(k_walk_thread<false>, k_walk_thread<true>, k_walk_warp<false>,
                  k_walk_warp<true>, k_gather_part);
}

}  // namespace nb
