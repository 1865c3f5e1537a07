// Prep pass of every step: opening kick + drift (src/integrator.cu:5-25),
// bounding box (src/forces_bh.cu:125-188), all-pairs source packing, and
// zeroing of the radix-sort scratch -- one read and one write of the state.
#include "nb_internal.cuh"

namespace nb {

struct PrepArgs {
  int n;
  int npairs;        // pairs to visit (covers n, and the packed padding)
  float4* pos;
  float4* pos_lo;
  float4* vel;
  const float4* acc;
  float half_dt, dt;
  int* bbox_part;    // [gridDim.x][6]
  int* bbox;         // [6] final
  unsigned* ticket;
  float4* src;       // packed sources or nullptr
  uint32_t* zero;    // sort scratch to clear or nullptr
  int zero_words;
};

// Two-sum drift of one coordinate held as hi + lo (error-free transforms;
// the product's rounding error comes from an FMA).
__device__ __forceinline__ void drift_comp(float& hi, float& lo, float v,
                                           float dt) {
  float pp = __fmul_rn(dt, v);
  float ep = __fmaf_rn(dt, v, -pp);
  float s = __fadd_rn(hi, pp);
  float bb = __fsub_rn(s, hi);
  float es = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(pp, bb));
  float l = __fadd_rn(lo, __fadd_rn(es, ep));
  float h = __fadd_rn(s, l);
  lo = __fsub_rn(l, __fsub_rn(h, s));
  hi = h;
}

template <bool KD, bool COMP, bool BBOX, bool PACK>
__global__ void __launch_bounds__(kPrepThreads) k_prep(PrepArgs a) {
  chain_release();   // the Morton kernel may be scheduled (it waits for this grid)
  int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff};
  int hi[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  const int stride = gridDim.x * blockDim.x;
  // kick, drift and box of particle i, given its loaded state
  auto advance = [&](int i, float4 x, float4 v, float4 ac, float4 l) {
    if (KD) {
      v.x = __fmaf_rn(a.half_dt, ac.x, v.x);
      v.y = __fmaf_rn(a.half_dt, ac.y, v.y);
      v.z = __fmaf_rn(a.half_dt, ac.z, v.z);
      a.vel[i] = v;
      if (COMP) {
        drift_comp(x.x, l.x, v.x, a.dt);
        drift_comp(x.y, l.y, v.y, a.dt);
        drift_comp(x.z, l.z, v.z, a.dt);
        a.pos_lo[i] = l;
      } else {
        x.x = __fmaf_rn(a.dt, v.x, x.x);
        x.y = __fmaf_rn(a.dt, v.y, x.y);
        x.z = __fmaf_rn(a.dt, v.z, x.z);
      }
      a.pos[i] = x;
    }
    if (BBOX) {
      int ox = f2ord(x.x), oy = f2ord(x.y), oz = f2ord(x.z);
      lo[0] = min(lo[0], ox); lo[1] = min(lo[1], oy); lo[2] = min(lo[2], oz);
      hi[0] = max(hi[0], ox); hi[1] = max(hi[1], oy); hi[2] = max(hi[2], oz);
    }
    return x;
  };
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (PACK) {
    // pairs of particles (2q, 2q + 1) feed one packed source record
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < a.npairs; q += stride) {
      float4 p[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = 2 * q + h;
        if (i < a.n) {
          p[h] = advance(i, a.pos[i], KD ? a.vel[i] : z4, KD ? a.acc[i] : z4,
                         KD && COMP ? a.pos_lo[i] : z4);
        } else {
          p[h] = z4;   // zero-mass padding
        }
      }
      a.src[2 * q] = make_float4(p[0].x, p[1].x, p[0].y, p[1].y);
      a.src[2 * q + 1] = make_float4(p[0].z, p[1].z, p[0].w, p[1].w);
    }
  } else {
    // two particles per thread and round, all their loads issued first
    // (four measured slower: more registers, fewer resident warps)
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += 2 * stride) {
      float4 x[2], v[2], ac[2], l[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = i0 + u * stride;
        x[u] = v[u] = ac[u] = l[u] = z4;
        if (i < a.n) {
          x[u] = a.pos[i];
          if (KD) {
            v[u] = a.vel[i];
            ac[u] = a.acc[i];
            if (COMP) l[u] = a.pos_lo[i];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = i0 + u * stride;
        if (i < a.n) advance(i, x[u], v[u], ac[u], l[u]);
      }
    }
  }
  if (a.zero) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.zero_words; i += stride)
      a.zero[i] = 0u;
  }
  if (!BBOX) return;

  // block reduce, then the last block to finish reduces the block partials
  __shared__ int s_red[kPrepThreads / 32][6];
  __shared__ bool s_last;
  int r[6] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r[c] = __reduce_min_sync(0xffffffffu, r[c]);
    r[c + 3] = __reduce_max_sync(0xffffffffu, r[c + 3]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int c = 0; c < 6; ++c) s_red[warp][c] = r[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    int c = threadIdx.x;
    int v = s_red[0][c];
    for (int w = 1; w < kPrepThreads / 32; ++w)
      v = c < 3 ? min(v, s_red[w][c]) : max(v, s_red[w][c]);
    a.bbox_part[blockIdx.x * 6 + c] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the whole last block reduces the block partials (min / max are
  // order-independent, so the result is exact)
  int q[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000,
              (int)0x80000000, (int)0x80000000};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c] = min(q[c], __ldcg(a.bbox_part + b * 6 + c));
      q[c + 3] = max(q[c + 3], __ldcg(a.bbox_part + b * 6 + c + 3));
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    q[c] = __reduce_min_sync(0xffffffffu, q[c]);
    q[c + 3] = __reduce_max_sync(0xffffffffu, q[c + 3]);
  }
  __syncthreads();   // s_red is reused
  if (lane == 0)
    for (int c = 0; c < 6; ++c) s_red[warp][c] = q[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int c = threadIdx.x;
    int v = s_red[0][c];
    for (int w = 1; w < kPrepThreads / 32; ++w)
      v = c < 3 ? min(v, s_red[w][c]) : max(v, s_red[w][c]);
    a.bbox[c] = v;
  }
  if (threadIdx.x == 0) *a.ticket = 0u;   // ready for the next launch
}

int launch_prep(Workspace& w, const StepArgs& s, bool bbox, bool pack,
                cudaStream_t st) {
  PrepArgs a;
  a.n = s.n;
  int npairs = (s.n + 1) / 2;
  if (pack) {
    int npad = (s.n + kSrcTile - 1) / kSrcTile * kSrcTile;
    npairs = npad / 2;
  }
  a.npairs = npairs;
  a.pos = s.pos;
  a.pos_lo = s.pos_lo;
  a.vel = s.vel;
  a.acc = s.acc;
  a.half_dt = s.half_dt;
  a.dt = s.dt;
  a.bbox_part = w.bbox_part;
  a.bbox = w.bbox;
  a.ticket = w.bbox_ticket;
  a.src = pack ? w.src : nullptr;
  a.zero = nullptr;
  a.zero_words = 0;
  if (bbox) {
    a.zero = w.hist;   // hist, tile counters and status are one allocation
    // histograms, tile counters, and the tile status words of the passes
    // this key width sorts with (pass p's words follow pass p - 1's)
    a.zero_words = 8 * kSortRadix + 8 + sort_passes(s.key_bits) * w.status_tiles * kSortRadix;
  }
  int blocks = (npairs + kPrepThreads - 1) / kPrepThreads;
  if (blocks > kPrepMaxBlocks) blocks = kPrepMaxBlocks;
  if (blocks < 1) blocks = 1;
  const bool kd = s.kick_drift && s.vel != nullptr;
  const bool comp = s.pos_lo != nullptr;
#define NB_PREP(KD, C, B, P) k_prep<KD, C, B, P><<<blocks, kPrepThreads, 0, st>>>(a)
  if (kd && comp) {
    if (bbox) { if (pack) NB_PREP(true, true, true, true); else NB_PREP(true, true, true, false); }
    else { if (pack) NB_PREP(true, true, false, true); else NB_PREP(true, true, false, false); }
  } else if (kd) {
    if (bbox) { if (pack) NB_PREP(true, false, true, true); else NB_PREP(true, false, true, false); }
    else { if (pack) NB_PREP(true, false, false, true); else NB_PREP(true, false, false, false); }
  } else {
    if (bbox) { if (pack) NB_PREP(false, false, true, true); else NB_PREP(false, false, true, false); }
    else { if (pack) NB_PREP(false, false, false, true); else NB_PREP(false, false, false, false); }
  }
#undef NB_PREP
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// Ensemble prep: kick + drift of every live slot, each simulation's bounding
// box, and zeroing of the sort scratch.  Each warp takes a contiguous run of
// 32-slot blocks (a block never mixes simulations) and keeps per-lane
// min / max while the simulation stays the same; at a change of simulation
// and at the end it reduces over the warp and issues one atomic per
// component.  The boxes must hold the empty sentinels on entry
// (launch_ens_prep sets them).
__device__ __forceinline__ void ens_box_flush(const EnsArgs& e, int s, int* r) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r[c] = __reduce_min_sync(0xffffffffu, r[c]);
    r[c + 3] = __reduce_max_sync(0xffffffffu, r[c + 3]);
  }
  if ((threadIdx.x & 31) == 0 && s >= 0) {
    for (int c = 0; c < 3; ++c) {
      if (r[c] != 0x7fffffff) atomicMin(&e.bbox_min[4 * s + c], r[c]);
      if (r[c + 3] != (int)0x80000000) atomicMax(&e.bbox_max[4 * s + c], r[c + 3]);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r[c] = 0x7fffffff;
    r[c + 3] = (int)0x80000000;
  }
}

template <bool KD>
__global__ void __launch_bounds__(kPrepThreads) k_ens_prep(EnsArgs e,
                                                           uint32_t* zero,
                                                           int zero_words) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nblk = e.nslots >> 5;
  const int per = (nblk + warps - 1) / warps;
  const int b0 = min(nblk, wid * per), b1 = min(nblk, b0 + per);
  int r[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000,
              (int)0x80000000, (int)0x80000000};
  int cur = -1;
  SimDesc d{};
  for (int b = b0; b < b1; ++b) {
    const int s = e.blk_sim[b];                 // the same for the whole warp
    if (s != cur) {
      ens_box_flush(e, cur, r);
      cur = s;
      if (s >= 0) d = e.sims[s];
    }
    if (s < 0 || !d.active) continue;
    const int slot = b * 32 + lane;
    if (slot - d.base >= d.n) continue;
    float4 x = e.pos[slot];
    if (KD && d.active == 1) {
      float4 v = e.vel[slot];
      const float4 ac = e.acc[slot];
      v.x = __fmaf_rn(d.half_dt, ac.x, v.x);
      v.y = __fmaf_rn(d.half_dt, ac.y, v.y);
      v.z = __fmaf_rn(d.half_dt, ac.z, v.z);
      e.vel[slot] = v;
      if (d.compensated) {
        float4 l = e.pos_lo[slot];
        drift_comp(x.x, l.x, v.x, d.dt);
        drift_comp(x.y, l.y, v.y, d.dt);
        drift_comp(x.z, l.z, v.z, d.dt);
        e.pos_lo[slot] = l;
      } else {
        x.x = __fmaf_rn(d.dt, v.x, x.x);
        x.y = __fmaf_rn(d.dt, v.y, x.y);
        x.z = __fmaf_rn(d.dt, v.z, x.z);
      }
      e.pos[slot] = x;
    }
    r[0] = min(r[0], f2ord(x.x));
    r[1] = min(r[1], f2ord(x.y));
    r[2] = min(r[2], f2ord(x.z));
    r[3] = max(r[3], f2ord(x.x));
    r[4] = max(r[4], f2ord(x.y));
    r[5] = max(r[5], f2ord(x.z));
  }
  ens_box_flush(e, (cur >= 0 && d.active) ? cur : -1, r);
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < zero_words; i += stride)
    zero[i] = 0u;
}

int launch_ens_prep(const EnsArgs& e, cudaStream_t st) {
  // empty boxes: 0x7f7f7f7f (a large positive ordered value) for the minima,
  // 0x80808080 (a large negative one) for the maxima
  NB_CUDA(cudaMemsetAsync(e.bbox_min, 0x7f, sizeof(int) * 4 * e.nsims, st));
  NB_CUDA(cudaMemsetAsync(e.bbox_max, 0x80, sizeof(int) * 4 * e.nsims, st));
  const int zero_words = 8 * kSortRadix + 8 + 8 * e.status_tiles * kSortRadix;
  int blocks = (e.nslots + kPrepThreads - 1) / kPrepThreads;
  if (blocks > 4 * device_sm_count()) blocks = 4 * device_sm_count();
  if (blocks < 1) blocks = 1;
  if (e.kick_drift)
    k_ens_prep<true><<<blocks, kPrepThreads, 0, st>>>(e, e.hist, zero_words);
  else
    k_ens_prep<false><<<blocks, kPrepThreads, 0, st>>>(e, e.hist, zero_words);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// L2 flush used by the benchmark between timed steps: writes a buffer larger
// than the 126 MB L2.
__global__ void k_flush(uint4* buf, size_t n) {
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride)
    buf[i] = make_uint4((unsigned)i, 0u, 0u, 0u);
}

int launch_flush(void* buf, size_t bytes, cudaStream_t st) {
  k_flush<<<device_sm_count() * 8, 256, 0, st>>>((uint4*)buf, bytes / sizeof(uint4));
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// FP32 calibration: 8 independent FMA chains per thread (scalar) or 8 packed
// chains of two (f32x2); the result is stored so nothing is eliminated.
constexpr int kPeakIters = 4096;

__global__ void __launch_bounds__(256) k_peak_scalar(float* out, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-7f + k;
  for (int it = 0; it < kPeakIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_peak_packed(float* out, float a, float b) {
  unsigned long long x[8], va, vb;
  asm("mov.b64 %0, {%1, %1};" : "=l"(va) : "f"(a));
  asm("mov.b64 %0, {%1, %1};" : "=l"(vb) : "f"(b));
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float u = threadIdx.x * 1e-7f + k;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x[k]) : "f"(u), "f"(u + 0.5f));
  }
  for (int it = 0; it < kPeakIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(va), "l"(vb));
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float u, v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(u), "=f"(v) : "l"(x[k]));
    s += u + v;
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int measure_fp32_peak(double* scalar, double* packed) {
  int dev = 0, sms = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256;
  float* out = nullptr;
  NB_CUDA(cudaMalloc(&out, sizeof(float) * blocks * threads));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best[2] = {0.0, 0.0};
  for (int rep = 0; rep < 6; ++rep) {
    for (int v = 0; v < 2; ++v) {
      cudaEventRecord(e0, 0);
      if (v == 0) k_peak_scalar<<<blocks, threads>>>(out, 0.999999f, 1e-7f);
      else k_peak_packed<<<blocks, threads>>>(out, 0.999999f, 1e-7f);
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      double fmas = (double)blocks * threads * kPeakIters * 8 * (v == 0 ? 1 : 2);
      double tf = 2.0 * fmas / (ms * 1e-3) / 1e12;
      if (rep > 0 && tf > best[v]) best[v] = tf;   // rep 0 warms up
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaError_t e = cudaGetLastError();
  cudaFree(out);
  if (e != cudaSuccess) return set_error(NB_ERR_CUDA, cudaGetErrorString(e));
  *scalar = best[0];
  *packed = best[1];
  return NB_OK;
}

int warm_prep_kernels() {
  return warm_fns(k_prep<true, true, true, true>, k_prep<true, true, true, false>,
                  k_prep<true, true, false, true>, k_prep<true, true, false, false>,
                  k_prep<true, false, true, true>, k_prep<true, false, true, false>,
                  k_prep<true, false, false, true>, k_prep<true, false, false, false>,
                  k_prep<false, false, true, true>, k_prep<false, false, true, false>,
                  k_prep<false, false, false, true>, k_prep<false, false, false, false>,
                  k_ens_prep<false>, k_ens_prep<true>);
}

}  // namespace nb
