/*
 * CPU oracle for the nbodyssey force-and-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked only by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The
 * product (nbodyssey_b200/) never calls it, and the product fails loudly when
 * its CUDA library is missing instead of falling back to this code.
 *
 * Each function restates the reference algorithm it cites (paths are within
 * the nbodyssey project).  Where the device kernels use a particular float
 * operation order, this file uses the same order with the same IEEE
 * round-to-nearest operations (compiled with -ffp-contract=off so that gcc
 * never fuses a*b+c on its own; fused steps are written as fmaf/fma), so that
 * Morton keys, the sort permutation, the tree topology, the node centres of
 * mass / sizes and every opening decision are bit-comparable with the GPU.
 * Interaction sums are done in FP64 here: they are the ideal value of the
 * same interaction set, not a bit-mirror of the FP32 device sums.
 *
 * Parity pins: tests/golden/ holds fixtures produced by running the
 * reference's own Python scripts (scripts/lbvh_check.py,
 * scripts/reference_nbody.py, scripts/barnes_hut_reference.py); the
 * generating script is tests/golden/make_golden.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))

static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

ORC_API int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

ORC_API void orc_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

/* ---------------------------------------------------------------------------
 * Bounding box: exact min/max per axis (src/forces_bh.cu:125-188,
 * scripts/lbvh_check.py:46-47).
 * ------------------------------------------------------------------------- */
ORC_API void orc_bbox(const float* p4, int64_t n, float* lo, float* hi) {
  lo[0] = lo[1] = lo[2] = INFINITY;
  hi[0] = hi[1] = hi[2] = -INFINITY;
  for (int64_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      float v = p4[4 * i + a];
      if (v < lo[a]) lo[a] = v;
      if (v > hi[a]) hi[a] = v;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Morton keys (src/forces_bh.cu:192-220; scripts/lbvh_check.py:35-54).
 * One cubic scale over the longest box edge; per axis
 *   q = clamp(trunc(((p - lo) * RN(1/ext)) * 2^b), 0, 2^b - 1)
 * in float32 round-to-nearest.  key_bits 63 uses b = 21 per axis (the
 * reference width); key_bits 30 uses b = 10.  Axis x takes the highest bit of
 * each triple.  The bit spreading inserts two zero bits between consecutive
 * input bits.
 * ------------------------------------------------------------------------- */
static inline uint64_t spread_bits3(uint32_t v, int bits) {
  /* Written as a plain loop: the oracle states what the spread is, the device
   * uses a mask ladder; both give bit k of v at position 3k. */
  uint64_t out = 0;
  for (int k = 0; k < bits; ++k) out |= (uint64_t)((v >> k) & 1u) << (3 * k);
  return out;
}

ORC_API void orc_morton(const float* p4, int64_t n, const float* lo,
                        const float* hi, int key_bits, uint64_t* keys) {
  int b = key_bits == 63 ? 21 : 10;
  float scale = (float)(1u << b);
  float qmax = scale - 1.0f;
  float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  float ext = fmaxf(ex, fmaxf(ey, ez));
  float inv = ext > 0.0f ? 1.0f / ext : 0.0f;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
      float d = p4[4 * i + a] - lo[a];
      float t = d * inv;
      float u = fmaxf(t, 0.0f) * scale;
      q[a] = (uint32_t)fminf(u, qmax);
    }
    keys[i] = (spread_bits3(q[0], b) << 2) | (spread_bits3(q[1], b) << 1) |
              spread_bits3(q[2], b);
  }
}

/* ---------------------------------------------------------------------------
 * Stable sort of (key, index): LSD radix, 8-bit digits.  A stable sort by key
 * with the original index as payload equals Python's sorted(range(n),
 * key=keys) used by scripts/lbvh_check.py:232 and CUB's stable SortPairs
 * (src/forces_bh.cu:490-497).
 * ------------------------------------------------------------------------- */
ORC_API void orc_sort_pairs(const uint64_t* keys_in, int64_t n, int key_bits,
                            uint64_t* keys_out, uint32_t* perm_out) {
  uint64_t* ka = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1));
  uint64_t* kb = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1));
  uint32_t* va = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  uint32_t* vb = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  for (int64_t i = 0; i < n; ++i) { ka[i] = keys_in[i]; va[i] = (uint32_t)i; }
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    int sh = 8 * p;
    for (int64_t i = 0; i < n; ++i) cnt[((ka[i] >> sh) & 255u) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; ++i) {
      int64_t dst = cnt[(ka[i] >> sh) & 255u]++;
      kb[dst] = ka[i];
      vb[dst] = va[i];
    }
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  memcpy(keys_out, ka, sizeof(uint64_t) * (size_t)n);
  memcpy(perm_out, va, sizeof(uint32_t) * (size_t)n);
  free(ka); free(kb); free(va); free(vb);
}

/* ---------------------------------------------------------------------------
 * Karras 2012 radix tree (src/forces_bh.cu:234-277; lbvh_check.py:57-100).
 * Node ids: internal [0, n-2] with root 0; leaf i (sorted order) is n-1+i.
 * delta = common prefix length of keys i and j, -1 out of range; equal keys
 * tie-break on the sorted index: 64+clz32(i^j) for 63-bit keys (as the
 * reference), 32+clz32(i^j) for 30-bit keys held in 32-bit words.
 * ------------------------------------------------------------------------- */
static inline int delta_k(const uint64_t* k, int64_t n, int key_bits,
                          int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  uint64_t x = k[i] ^ k[j];
  if (key_bits == 63) {
    if (x) return clz64(x);
    return 64 + clz32((uint32_t)(i ^ j));
  }
  if (x) return clz32((uint32_t)x);
  return 32 + clz32((uint32_t)(i ^ j));
}

ORC_API void orc_karras(const uint64_t* ks, int64_t n, int key_bits,
                        int32_t* children /* 2*(n-1) */,
                        int32_t* parent /* 2n-1 */) {
  for (int64_t i = 0; i < 2 * n - 1; ++i) parent[i] = -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n - 1; ++i) {
    int d = (delta_k(ks, n, key_bits, i, i + 1) -
             delta_k(ks, n, key_bits, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta_k(ks, n, key_bits, i, i - d);
    int64_t lmax = 2;
    while (delta_k(ks, n, key_bits, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t > 0; t >>= 1)
      if (delta_k(ks, n, key_bits, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int64_t first = i < j ? i : j, last = i < j ? j : i;
    int common = delta_k(ks, n, key_bits, first, last);
    int64_t split = first, step = last - first;
    do {
      step = (step + 1) >> 1;
      if (split + step < last &&
          delta_k(ks, n, key_bits, first, split + step) > common)
        split += step;
    } while (step > 1);
    int64_t left = (split == first) ? (n - 1 + split) : split;
    int64_t right = (split + 1 == last) ? (n - 1 + split + 1) : split + 1;
    children[2 * i] = (int32_t)left;
    children[2 * i + 1] = (int32_t)right;
    parent[left] = (int32_t)i;
    parent[right] = (int32_t)i;
  }
}

/* ---------------------------------------------------------------------------
 * Bottom-up centres of mass, boxes and sizes (src/forces_bh.cu:281-331;
 * lbvh_check.py:121-148).  Arithmetic (mirrored exactly by the device):
 *   FP64 mass-weighted sums per node: leaf (x*m, y*m, z*m, m) are exact
 *   products of two floats; internal = left + right (left first).
 *   com = float(sum_x / sum_m) etc, node mass = float(sum_m).
 *   box = elementwise min/max of the children's boxes (leaf box = point);
 *   size = max edge in float32; size2 = size*size in float32.
 * Outputs per internal node: com4 (x,y,z,m), size2, box lo/hi.
 * ------------------------------------------------------------------------- */
ORC_API void orc_com(const float* ps4 /* sorted positions */, int64_t n,
                     const int32_t* children, float* com4, float* size2,
                     float* box_lo3, float* box_hi3, double* sums4) {
  if (n < 2) return;
  int64_t ni = n - 1;
  /* post-order via explicit stack */
  int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)ni);
  int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * n));
  int64_t no = 0, sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    int32_t id = stack[--sp];
    if (id < ni) {
      order[no++] = id;
      stack[sp++] = children[2 * id];
      stack[sp++] = children[2 * id + 1];
    }
  }
  for (int64_t k = no - 1; k >= 0; --k) {
    int32_t id = order[k];
    double s[2][4];
    float lo[2][3], hi[2][3];
    for (int c = 0; c < 2; ++c) {
      int32_t ch = children[2 * id + c];
      if (ch >= ni) {
        const float* p = ps4 + 4 * (int64_t)(ch - ni);
        double m = (double)p[3];
        s[c][0] = (double)p[0] * m;
        s[c][1] = (double)p[1] * m;
        s[c][2] = (double)p[2] * m;
        s[c][3] = m;
        for (int a = 0; a < 3; ++a) lo[c][a] = hi[c][a] = p[a];
      } else {
        for (int a = 0; a < 4; ++a) s[c][a] = sums4[4 * (int64_t)ch + a];
        for (int a = 0; a < 3; ++a) {
          lo[c][a] = box_lo3[3 * (int64_t)ch + a];
          hi[c][a] = box_hi3[3 * (int64_t)ch + a];
        }
      }
    }
    double sm = s[0][3] + s[1][3];
    for (int a = 0; a < 3; ++a) {
      double sa = s[0][a] + s[1][a];
      sums4[4 * (int64_t)id + a] = sa;
      com4[4 * (int64_t)id + a] = (float)(sa / sm);
    }
    sums4[4 * (int64_t)id + 3] = sm;
    com4[4 * (int64_t)id + 3] = (float)sm;
    float e[3];
    for (int a = 0; a < 3; ++a) {
      float l = fminf(lo[0][a], lo[1][a]);
      float h = fmaxf(hi[0][a], hi[1][a]);
      box_lo3[3 * (int64_t)id + a] = l;
      box_hi3[3 * (int64_t)id + a] = h;
      e[a] = h - l;
    }
    float sz = fmaxf(e[0], fmaxf(e[1], e[2]));
    size2[id] = sz * sz;
  }
  free(order);
  free(stack);
}

/* Opening test shared by both walks, in the device's exact float order:
 *   d2 = fma(dz, dz, fma(dy, dy, dx*dx)); accept  <=>  size2 < theta2 * d2.
 * (src/forces_bh.cu:352-356, lbvh_check.py:162-165) */
static inline int accept_node(const float* c4, float size2, float theta2,
                              float xi, float yi, float zi) {
  float dx = c4[0] - xi, dy = c4[1] - yi, dz = c4[2] - zi;
  float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  return size2 < theta2 * d2;
}

static inline void interact_f64(double* a, double sx, double sy, double sz,
                                double sm, double xi, double yi, double zi,
                                double eps2) {
  double dx = sx - xi, dy = sy - yi, dz = sz - zi;
  double r2 = dx * dx + dy * dy + dz * dz + eps2;
  double inv = 1.0 / (r2 * sqrt(r2));
  double f = sm * inv;
  a[0] += dx * f;
  a[1] += dy * f;
  a[2] += dz * f;
}

#define ORC_STACK 256

/* ---------------------------------------------------------------------------
 * Per-thread walk (src/forces_bh.cu:335-377; lbvh_check.py:151-177):
 * explicit stack, children pushed left then right (right popped first).
 * For sorted targets[k] writes acc (FP64, times G), the interaction count and
 * the maximum stack depth.  Returns 0, or -1 on stack overflow.
 * ------------------------------------------------------------------------- */
ORC_API int orc_walk_thread(const float* ps4, int64_t n,
                            const int32_t* children, const float* com4,
                            const float* size2, float theta, double eps2,
                            float G, const int64_t* targets, int64_t nt,
                            double* acc3, int64_t* inter, int32_t* depth) {
  int64_t ni = n - 1;
  float theta2 = theta * theta;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
  for (int64_t k = 0; k < nt; ++k) {
    int64_t t = targets[k];
    const float* bi = ps4 + 4 * t;
    double a[3] = {0, 0, 0};
    int64_t cnt = 0;
    int32_t st[ORC_STACK];
    int sp = 0, maxd = 0;
    st[sp++] = 0;
    while (sp > 0) {
      if (sp > maxd) maxd = sp;
      int32_t id = st[--sp];
      const float* src;
      if (id >= ni) {
        src = ps4 + 4 * (int64_t)(id - ni);
      } else if (accept_node(com4 + 4 * (int64_t)id, size2[id], theta2, bi[0],
                             bi[1], bi[2])) {
        src = com4 + 4 * (int64_t)id;
      } else {
        if (sp + 2 > ORC_STACK) { bad = 1; break; }
        st[sp++] = children[2 * id];
        st[sp++] = children[2 * id + 1];
        continue;
      }
      interact_f64(a, src[0], src[1], src[2], src[3], bi[0], bi[1], bi[2],
                   eps2);
      ++cnt;
    }
    for (int c = 0; c < 3; ++c) acc3[3 * k + c] = (double)G * a[c];
    if (inter) inter[k] = cnt;
    if (depth) depth[k] = maxd;
  }
  return bad ? -1 : 0;
}

/* ---------------------------------------------------------------------------
 * Warp walk (src/forces_bh.cu:395-447; lbvh_check.py:180-209): the 32 sorted
 * targets [32w, 32w+31] share one stack; an internal node is opened when any
 * live lane's test rejects it, otherwise every lane takes its centre of mass.
 * Writes acc for every live lane of every listed warp (indexed by sorted
 * target), the warp's interaction count, and its maximum stack depth.
 * ------------------------------------------------------------------------- */
ORC_API int orc_walk_warp(const float* ps4, int64_t n, const int32_t* children,
                          const float* com4, const float* size2, float theta,
                          double eps2, float G, const int64_t* warps, int64_t nw,
                          double* acc3 /* [nw*32][3] */, int64_t* inter,
                          int32_t* depth) {
  int64_t ni = n - 1;
  float theta2 = theta * theta;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : bad)
  for (int64_t w = 0; w < nw; ++w) {
    int64_t base = warps[w] * 32;
    int live = (int)((n - base) < 32 ? (n - base) : 32);
    double a[32][3];
    memset(a, 0, sizeof(a));
    int64_t cnt = 0;
    int32_t st[ORC_STACK];
    int sp = 0, maxd = 0;
    st[sp++] = 0;
    while (sp > 0) {
      if (sp > maxd) maxd = sp;
      int32_t id = st[--sp];
      const float* src;
      if (id >= ni) {
        src = ps4 + 4 * (int64_t)(id - ni);
      } else {
        const float* c = com4 + 4 * (int64_t)id;
        int open = 0;
        for (int l = 0; l < live; ++l) {
          const float* bi = ps4 + 4 * (base + l);
          if (!accept_node(c, size2[id], theta2, bi[0], bi[1], bi[2])) {
            open = 1;
            break;
          }
        }
        if (open) {
          if (sp + 2 > ORC_STACK) { bad = 1; break; }
          st[sp++] = children[2 * id];
          st[sp++] = children[2 * id + 1];
          continue;
        }
        src = c;
      }
      for (int l = 0; l < live; ++l) {
        const float* bi = ps4 + 4 * (base + l);
        interact_f64(a[l], src[0], src[1], src[2], src[3], bi[0], bi[1], bi[2],
                     eps2);
      }
      ++cnt;
    }
    for (int l = 0; l < 32; ++l)
      for (int c = 0; c < 3; ++c)
        acc3[(w * 32 + l) * 3 + c] = l < live ? (double)G * a[l][c] : 0.0;
    if (inter) inter[w] = cnt;
    if (depth) depth[w] = maxd;
  }
  return bad ? -1 : 0;
}

/* ---------------------------------------------------------------------------
 * Exact all-pairs force in FP64 (src/forces.cu:17-52 force law;
 * scripts/reference_nbody.py:45-61 with dtype float64):
 *   a_i = G sum_j m_j (r_j - r_i) / (|r_j - r_i|^2 + eps^2)^{3/2}
 * The j == i term is zero.  Inputs are float positions (optionally plus a
 * low-order float part); targets may be a subset.
 * ------------------------------------------------------------------------- */
ORC_API void orc_allpairs_f64(const float* p4, const float* lo4, int64_t n,
                              double eps2, float G, const int64_t* targets,
                              int64_t nt, double* acc3) {
  double* px = (double*)malloc(sizeof(double) * (size_t)n * 4);
  for (int64_t j = 0; j < n; ++j) {
    for (int a = 0; a < 3; ++a)
      px[4 * j + a] = (double)p4[4 * j + a] + (lo4 ? (double)lo4[4 * j + a] : 0.0);
    px[4 * j + 3] = (double)p4[4 * j + 3];
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < nt; ++k) {
    int64_t i = targets ? targets[k] : k;
    double a[3] = {0, 0, 0};
    double xi = px[4 * i], yi = px[4 * i + 1], zi = px[4 * i + 2];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      interact_f64(a, px[4 * j], px[4 * j + 1], px[4 * j + 2], px[4 * j + 3],
                   xi, yi, zi, eps2);
    }
    for (int c = 0; c < 3; ++c) acc3[3 * k + c] = (double)G * a[c];
  }
  free(px);
}

/* FP32 all-pairs with FP32 accumulation, the reference GPU's own precision
 * (src/forces.cu:17-52), used as the CPU baseline for the naive module.
 * Uses 1/sqrtf rather than the device's approximate reciprocal square root. */
ORC_API void orc_allpairs_f32(const float* p4, int64_t n, float eps, float G,
                              const int64_t* targets, int64_t nt, float* acc4) {
  float eps2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < nt; ++k) {
    int64_t i = targets ? targets[k] : k;
    float ax = 0.f, ay = 0.f, az = 0.f;
    float xi = p4[4 * i], yi = p4[4 * i + 1], zi = p4[4 * i + 2];
    for (int64_t j = 0; j < n; ++j) {
      float dx = p4[4 * j] - xi, dy = p4[4 * j + 1] - yi, dz = p4[4 * j + 2] - zi;
      float r2 = dx * dx + dy * dy + dz * dz + eps2;
      float inv = 1.0f / sqrtf(r2);
      float s = p4[4 * j + 3] * inv * inv * inv;
      ax += dx * s; ay += dy * s; az += dz * s;
    }
    acc4[4 * k] = G * ax; acc4[4 * k + 1] = G * ay; acc4[4 * k + 2] = G * az;
    acc4[4 * k + 3] = 0.f;
  }
}

/* ---------------------------------------------------------------------------
 * Total energy and momentum in FP64 (src/integrator.cu:43-110 semantics;
 * scripts/reference_nbody.py:64-81 arithmetic):
 *   KE = sum_i 1/2 m_i |v_i|^2,  PE = -G sum_{i<j} m_i m_j / sqrt(r_ij^2+eps^2)
 * out = {E, KE, PE, Px, Py, Pz}.
 * ------------------------------------------------------------------------- */
ORC_API void orc_energy_f64(const float* p4, const float* lo4, const float* v4,
                            int64_t n, double eps2, float G, double* out) {
  double* px = (double*)malloc(sizeof(double) * (size_t)n * 4);
  for (int64_t j = 0; j < n; ++j) {
    for (int a = 0; a < 3; ++a)
      px[4 * j + a] = (double)p4[4 * j + a] + (lo4 ? (double)lo4[4 * j + a] : 0.0);
    px[4 * j + 3] = (double)p4[4 * j + 3];
  }
  double ke = 0.0, pe = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double m = px[4 * i + 3];
    double vx = v4[4 * i], vy = v4[4 * i + 1], vz = v4[4 * i + 2];
    ke += 0.5 * m * (vx * vx + vy * vy + vz * vz);
    mx += m * vx; my += m * vy; mz += m * vz;
  }
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : pe)
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    double xi = px[4 * i], yi = px[4 * i + 1], zi = px[4 * i + 2];
    for (int64_t j = i + 1; j < n; ++j) {
      double dx = px[4 * j] - xi, dy = px[4 * j + 1] - yi, dz = px[4 * j + 2] - zi;
      s += px[4 * j + 3] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
    }
    pe += px[4 * i + 3] * s;
  }
  pe = -(double)G * pe;
  out[0] = ke + pe; out[1] = ke; out[2] = pe;
  out[3] = mx; out[4] = my; out[5] = mz;
  free(px);
}

/* ---------------------------------------------------------------------------
 * Kick and drift, in the device's exact float arithmetic
 * (src/integrator.cu:5-25):
 *   kick:  v = fma(h, a, v)
 *   drift, plain:       x = fma(dt, v, x)
 *   drift, compensated: positions are hi + lo; the increment dt*v and its
 *   exact rounding error (fma) are added with a two-sum, the error is folded
 *   into lo and the pair renormalised with a fast two-sum.
 * ------------------------------------------------------------------------- */
ORC_API void orc_kick(float* v4, const float* a4, int64_t n, float h) {
  for (int64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) v4[4 * i + c] = fmaf(h, a4[4 * i + c], v4[4 * i + c]);
}

ORC_API void orc_drift(float* p4, float* lo4, const float* v4, int64_t n,
                       float dt, int compensated) {
  for (int64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      float x = p4[4 * i + c], v = v4[4 * i + c];
      if (!compensated) {
        p4[4 * i + c] = fmaf(dt, v, x);
        continue;
      }
      float l = lo4[4 * i + c];
      float pp = dt * v;
      float ep = fmaf(dt, v, -pp);
      float s = x + pp;
      float bb = s - x;
      float es = (x - (s - bb)) + (pp - bb);
      l = l + (es + ep);
      float hi = s + l;
      float nl = l - (hi - s);
      p4[4 * i + c] = hi;
      lo4[4 * i + c] = nl;
    }
  }
}
