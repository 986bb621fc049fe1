// Reference-compatible ("compat") entry points: the softened direct sums,
// the dense Morton octree8 build and its classic and stochastic Barnes-Hut
// traversals, all on the reference's byte layouts.
//
// This translation unit is compiled with --use_fast_math, the flag the
// reference's sbh_ffi target uses (CMakeLists.txt:39), so that the Morton
// quantisation (v - min) / span runs the same division instruction and
// produces the same codes, and the opening tests round the same way.
//
// Differences from the reference that are deliberate (and invisible at the
// byte level except where noted):
//  * no cudaMalloc/cudaFree, no D2H copy and no stream synchronisation: the
//    bounding span is computed on the device and temporaries live in a
//    caller-provided workspace (the reference syncs the stream and allocates
//    4*depth+12 buffers per build, src/sbh_ffi.cu:1111-1370);
//  * leaves are ordered by a stable radix sort of (Morton code, input index),
//    so the order inside one leaf cell is the input order (the reference's
//    atomic cursor makes it nondeterministic, src/sbh_ffi.cu:1732);
//  * the upward pass sums in FP64 (prefix sums over the sorted leaves), the
//    reference accumulates FP32 atomics;
//  * parameters travel by value, not through __constant__ globals, so calls
//    on concurrent streams do not race (src/sbh_ffi.cu:2536-2561);
//  * a traversal whose stack would exceed 128 entries records
//    SBH_DEV_STACK_OVERFLOW instead of writing past the array.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "sbh_common.cuh"
#include "sbh_primitives.cuh"

namespace sbh {

// ---------------------------------------------------------------------------
// Direct sums (src/sbh_ffi.cu:399-546), shared-memory tiled, one query per
// thread, Kahan-compensated across tiles.
// ---------------------------------------------------------------------------
constexpr int kDirectThreads = 256;

template <int VJP, bool PER>
__global__ void __launch_bounds__(kDirectThreads)
    direct_soft_kernel(const float* __restrict__ pts, const float* __restrict__ masses, int64_t n,
                       const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq,
                       float* __restrict__ out, Soft s, Periodic per) {
  __shared__ float4 tile[kDirectThreads];
  int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool active = qi < nq;
  float qx = 0.f, qy = 0.f, qz = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
  if (active) {
    qx = queries[3 * qi];
    qy = queries[3 * qi + 1];
    qz = queries[3 * qi + 2];
    if (VJP) {
      gx = cot[3 * qi];
      gy = cot[3 * qi + 1];
      gz = cot[3 * qi + 2];
    }
  }
  float inv_l = (per.on && per.box > 0.0f) ? 1.0f / per.box : 0.0f;
  float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
  for (int64_t base = 0; base < n; base += kDirectThreads) {
    int64_t j = base + threadIdx.x;
    tile[threadIdx.x] =
        j < n ? make_float4(pts[3 * j], pts[3 * j + 1], pts[3 * j + 2], masses[j]) : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    int cnt = static_cast<int>(n - base < kDirectThreads ? n - base : kDirectThreads);
    float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll 4
    for (int k = 0; k < cnt; k++) {
      float4 p = tile[k];
      float rx = qx - p.x, ry = qy - p.y, rz = qz - p.z;
      if (PER) {
        rx = min_image_rint(rx, inv_l, per);
        ry = min_image_rint(ry, inv_l, per);
        rz = min_image_rint(rz, inv_l, per);
      }
      if (VJP) {
        soft_vjp_accum(rx, ry, rz, p.w, gx, gy, gz, s, ax, ay, az);
      } else {
        float c = soft_coeff(rx * rx + ry * ry + rz * rz, p.w, s);
        ax += c * rx;
        ay += c * ry;
        az += c * rz;
      }
    }
    kahan_add(sx, cx, ax);
    kahan_add(sy, cy, ay);
    kahan_add(sz, cz, az);
    __syncthreads();
  }
  if (active) {
    out[3 * qi] = sx;
    out[3 * qi + 1] = sy;
    out[3 * qi + 2] = sz;
  }
}

__global__ void __launch_bounds__(kDirectThreads)
    bruteforce_gravity_kernel(const float* __restrict__ pts, const float* __restrict__ masses, int64_t n,
                              int dim, const float* __restrict__ queries, int64_t nq,
                              float* __restrict__ out, Periodic per) {
  __shared__ float4 tile[kDirectThreads];
  int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool active = qi < nq;
  float q0 = 0.f, q1 = 0.f, q2 = 0.f;
  if (active) {
    q0 = queries[dim * qi];
    q1 = queries[dim * qi + 1];
    q2 = dim == 3 ? queries[dim * qi + 2] : 0.f;
  }
  float s = 0.f, c = 0.f;
  for (int64_t base = 0; base < n; base += kDirectThreads) {
    int64_t j = base + threadIdx.x;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (j < n) v = make_float4(pts[dim * j], pts[dim * j + 1], dim == 3 ? pts[dim * j + 2] : 0.f, masses[j]);
    tile[threadIdx.x] = v;
    __syncthreads();
    int cnt = static_cast<int>(n - base < kDirectThreads ? n - base : kDirectThreads);
    float a = 0.f;
    for (int k = 0; k < cnt; k++) {
      float4 p = tile[k];
      // src/sbh_ffi.cu:414-426: diff = p - q, wrapped with nearbyint(diff / L)
      float d0 = p.x - q0, d1 = p.y - q1, d2 = p.z - q2;
      if (per.on && per.box > 0.0f) {
        d0 -= per.box * nearbyintf(d0 / per.box);
        d1 -= per.box * nearbyintf(d1 / per.box);
        if (dim == 3) d2 -= per.box * nearbyintf(d2 / per.box);
      }
      float dsq = d0 * d0 + d1 * d1;
      if (dim == 3) dsq += d2 * d2;
      a += -p.w / (sqrtf(dsq) + 1e-1f);
    }
    kahan_add(s, c, a);
    __syncthreads();
  }
  if (active) out[qi] = s;
}

// ---------------------------------------------------------------------------
// octree8 build (src/sbh_ffi.cu:1039-1420)
// ---------------------------------------------------------------------------
struct O8Params {
  float min[3];
  float span;
  float cx, cy, cz, half;
  int valid;
};

// span = max axis extent, root centre = min + span/2 (src/sbh_ffi.cu:1128-1133,1395-1398).
__global__ void o8_setup_kernel(const float* min_corner, const float* max_corner, O8Params* prm,
                                uint32_t* status) {
  float mn0 = min_corner[0], mn1 = min_corner[1], mn2 = min_corner[2];
  float span = fmaxf(fmaxf(max_corner[0] - mn0, max_corner[1] - mn1), max_corner[2] - mn2);
  O8Params p;
  p.min[0] = mn0;
  p.min[1] = mn1;
  p.min[2] = mn2;
  p.span = span;
  p.cx = mn0 + span * 0.5f;
  p.cy = mn1 + span * 0.5f;
  p.cz = mn2 + span * 0.5f;
  p.half = span * 0.5f;
  p.valid = span > 0.0f ? 1 : 0;
  if (!p.valid) raise_status(status, SBH_DEV_BAD_BOUNDS);
  *prm = p;
}

// quantize_axis (src/sbh_ffi.cu:173-179); fast-math division like the reference.
__device__ __forceinline__ uint32_t o8_quantize(float v, float min_v, float span, int bits) {
  float t = (v - min_v) / span;
  t = fminf(fmaxf(t, 0.0f), 0.999999f);
  uint32_t max_bin = (1u << bits) - 1u;
  return static_cast<uint32_t>(t * static_cast<float>(max_bin + 1));
}

__device__ __forceinline__ uint32_t o8_morton(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t code = 0;
  for (int i = 0; i < bits; i++) {
    code |= ((x >> i) & 1u) << (3 * i);
    code |= ((y >> i) & 1u) << (3 * i + 1);
    code |= ((z >> i) & 1u) << (3 * i + 2);
  }
  return code;
}

__global__ void o8_codes_kernel(const float* __restrict__ pts, int64_t n, const O8Params* __restrict__ prm,
                                int depth, uint32_t* __restrict__ codes, uint32_t* __restrict__ counts) {
  if (!prm->valid) return;
  float mn0 = prm->min[0], mn1 = prm->min[1], mn2 = prm->min[2], span = prm->span;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t qx = o8_quantize(pts[3 * i], mn0, span, depth);
    uint32_t qy = o8_quantize(pts[3 * i + 1], mn1, span, depth);
    uint32_t qz = o8_quantize(pts[3 * i + 2], mn2, span, depth);
    uint32_t c = o8_morton(qx, qy, qz, depth);
    codes[i] = c;
    atomicAdd(&counts[c], 1u);
  }
}

// Leaf records in sorted order (src/sbh_ffi.cu:1723-1743 writes the same record).
__global__ void o8_gather_kernel(const float* __restrict__ pts, const float* __restrict__ nrm,
                                 const float* __restrict__ masses, int64_t n,
                                 const uint32_t* __restrict__ perm, const O8Params* __restrict__ prm,
                                 Leaf3* __restrict__ leaf) {
  if (prm && !prm->valid) return;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t s = perm[i];
    float4 a = make_float4(pts[3 * s], pts[3 * s + 1], pts[3 * s + 2], nrm ? nrm[3 * s] : 0.f);
    float4 b = make_float4(nrm ? nrm[3 * s + 1] : 0.f, nrm ? nrm[3 * s + 2] : 0.f, masses[s], 1.0f);
    float4* dst = reinterpret_cast<float4*>(leaf + i);
    dst[0] = a;
    dst[1] = b;
  }
}

// FP64 moment vector of a leaf record: (m, m x, m y, m z, m nx, m ny, m nz).
struct LeafMomentLoad {
  const Leaf3* leaf;
  __device__ DVec<7> operator()(int64_t i) const {
    const float4* p = reinterpret_cast<const float4*>(leaf + i);
    float4 a = p[0], b = p[1];
    double m = b.z;
    DVec<7> r;
    r.v[0] = m;
    r.v[1] = m * a.x;
    r.v[2] = m * a.y;
    r.v[3] = m * a.z;
    r.v[4] = m * a.w;
    r.v[5] = m * b.x;
    r.v[6] = m * b.y;
    return r;
  }
};

// One thread per dense node, all levels (src/sbh_ffi.cu:1788-1876).
__global__ void o8_nodes_kernel(OctreeNode8* __restrict__ nodes, Leaf3* __restrict__ contrib,
                                const uint32_t* __restrict__ off, const DVec<7>* __restrict__ P,
                                int depth, uint64_t total, const O8Params* __restrict__ prm) {
  if (!prm->valid) return;
  float cx0 = prm->cx, cy0 = prm->cy, cz0 = prm->cz, half0 = prm->half;
  for (uint64_t node_idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; node_idx < total;
       node_idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    int level = 0;
    uint64_t level_off = 0, level_n = 1;
    while (node_idx >= level_off + level_n) {
      level_off += level_n;
      level_n <<= 3;
      level++;
    }
    uint32_t idx = static_cast<uint32_t>(node_idx - level_off);
    int shift = 3 * (depth - level);
    uint64_t first_leaf = static_cast<uint64_t>(idx) << shift;
    uint64_t last_leaf = static_cast<uint64_t>(idx + 1) << shift;
    OctreeNode8 nd;
    nd.start = off[first_leaf];
    nd.end = off[last_leaf];
    nd.depth = static_cast<uint8_t>(level);
    nd.parent = level == 0 ? static_cast<uint32_t>(node_idx)
                           : static_cast<uint32_t>(level_off - (level_n >> 3) + (idx >> 3));
    nd.is_leaf = level == depth ? 1 : 0;
    nd.first_child = 0xFFFFFFFFu;
    nd.child_mask = 0;
    nd.pad0 = 0;
    int grid = 1 << level;
    int ix = 0, iy = 0, iz = 0;
    for (int b = 0; b < level; b++) {
      ix |= ((idx >> (3 * b + 0)) & 1) << b;
      iy |= ((idx >> (3 * b + 1)) & 1) << b;
      iz |= ((idx >> (3 * b + 2)) & 1) << b;
    }
    float step = half0 * 2.0f / static_cast<float>(grid);
    nd.cx = fmaf(static_cast<float>(ix) + 0.5f, step, cx0 - half0);
    nd.cy = fmaf(static_cast<float>(iy) + 0.5f, step, cy0 - half0);
    nd.cz = fmaf(static_cast<float>(iz) + 0.5f, step, cz0 - half0);
    nd.half_size = step * 0.5f;
    nd.diameter = step * sqrtf(3.0f);
    if (level < depth) {
      uint32_t child_base = static_cast<uint32_t>(level_off + level_n) + (idx << 3);
      int cshift = 3 * (depth - level - 1);
      uint8_t mask = 0;
      for (uint32_t c = 0; c < 8; c++) {
        nd.child[c] = child_base + c;
        uint64_t cl = static_cast<uint64_t>((idx << 3) + c) << cshift;
        uint64_t ch = static_cast<uint64_t>((idx << 3) + c + 1) << cshift;
        if (off[ch] > off[cl]) {
          mask |= static_cast<uint8_t>(1u << c);
          if (nd.first_child == 0xFFFFFFFFu) nd.first_child = child_base + c;
        }
      }
      nd.child_mask = mask;
      if (mask == 0) nd.is_leaf = 1;
    } else {
      for (int c = 0; c < 8; c++) nd.child[c] = 0xFFFFFFFFu;
    }
    DVec<7> hi = P[nd.end], lo = P[nd.start];
    double M = hi.v[0] - lo.v[0];
    float mass = static_cast<float>(M);
    nd.contrib.alpha = 1.0f;
    nd.contrib.mass = mass;
    if (mass > 0.0f) {
      for (int d = 0; d < 3; d++) {
        nd.contrib.pos[d] = static_cast<float>((hi.v[1 + d] - lo.v[1 + d]) / M);
        nd.contrib.nrm[d] = static_cast<float>((hi.v[4 + d] - lo.v[4 + d]) / M);
      }
    } else {
      for (int d = 0; d < 3; d++) {
        nd.contrib.pos[d] = 0.0f;
        nd.contrib.nrm[d] = 0.0f;
      }
    }
    // 8-byte stores: node_idx * 104 is 8-byte aligned.
    const uint2* src = reinterpret_cast<const uint2*>(&nd);
    uint2* dst = reinterpret_cast<uint2*>(nodes + node_idx);
#pragma unroll
    for (int k = 0; k < 13; k++) dst[k] = src[k];
    const float4* cs = reinterpret_cast<const float4*>(&nd.contrib);
    float4* cd = reinterpret_cast<float4*>(contrib + node_idx);
    cd[0] = cs[0];
    cd[1] = cs[1];
  }
}

// ---------------------------------------------------------------------------
// octree8 classic BH traversal (src/sbh_ffi.cu:1878-2144)
// ---------------------------------------------------------------------------
constexpr int kO8Stack = 128;

struct O8Node {
  float cx, cy, cz, half, diam;
  uint32_t start, end;
  uint8_t mask, is_leaf;
};

__device__ __forceinline__ float o8_mass(const OctreeNode8* nodes, int idx) {
  return __ldg(&nodes[idx].contrib.mass);
}

__device__ __forceinline__ bool o8_far(const OctreeNode8& nd, float qx, float qy, float qz, float beta,
                                       const Periodic& per) {
  if (nd.is_leaf) return true;
  float dx = min_image_floor(qx - nd.cx, per);
  float dy = min_image_floor(qy - nd.cy, per);
  float dz = min_image_floor(qz - nd.cz, per);
  float dist = sqrtf(dx * dx + dy * dy + dz * dz);
  return dist / nd.diameter >= beta;
}

__device__ __forceinline__ float axis_gap(float q, float lo, float hi) {
  if (q < lo) return lo - q;
  if (q > hi) return q - hi;
  return 0.0f;
}

__device__ __forceinline__ bool o8_prune(const OctreeNode8& nd, float qx, float qy, float qz,
                                         int prune_on, float r_cut_sq, const Periodic& per) {
  if (!prune_on) return false;
  if (per.on && per.box > 0.0f) {
    float inv_l = 1.0f / per.box;
    qx -= per.box * nearbyintf((qx - nd.cx) * inv_l);
    qy -= per.box * nearbyintf((qy - nd.cy) * inv_l);
    qz -= per.box * nearbyintf((qz - nd.cz) * inv_l);
  }
  float dx = axis_gap(qx, nd.cx - nd.half_size, nd.cx + nd.half_size);
  float dy = axis_gap(qy, nd.cy - nd.half_size, nd.cy + nd.half_size);
  float dz = axis_gap(qz, nd.cz - nd.half_size, nd.cz + nd.half_size);
  return dx * dx + dy * dy + dz * dz > r_cut_sq;
}

enum O8Kernel { O8_GRAV_GRAD = 0, O8_SOFT = 1, O8_SOFT_VJP = 2, O8_GRAV_GRAD_VJP = 3 };

// Softened pair terms in one fixed order of single-rounding operations
// (flush-to-zero, as the rest of this file under fast math), written once for
// a scalar pair and once for two pairs packed into FFMA2 / FADD2 / FMUL2
// (sm_100 f32x2). Both forms round every component the same way, so the
// traversal that sums a leaf two particles at a time and the one that sums
// it one at a time add bit-identical terms. The accumulation into the
// query's sum stays scalar and in the leaf's order.
struct F2 {
  unsigned long long v;
};

__device__ __forceinline__ F2 f2_pack(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(F2 x, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ float o8_add(float a, float b) {
  float d;
  asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ float o8_sub(float a, float b) {
  float d;
  asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ float o8_mul(float a, float b) {
  float d;
  asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ float o8_fma(float a, float b, float c) {
  float d;
  asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ F2 o8_add(F2 a, F2 b) {
  F2 d;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ F2 o8_sub(F2 a, F2 b) {
  F2 d;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ F2 o8_mul(F2 a, F2 b) {
  F2 d;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ F2 o8_fma(F2 a, F2 b, F2 c) {
  F2 d;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return d;
}
__device__ __forceinline__ float o8_splat_like(float, float s) { return s; }
__device__ __forceinline__ F2 o8_splat_like(F2, float s) { return f2_pack(s, s); }
__device__ __forceinline__ float o8_rsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ F2 o8_rsqrt(F2 a) {
  float x, y;
  f2_unpack(a, x, y);
  return f2_pack(rsqrtf(x), rsqrtf(y));
}

// Shared first steps of the softened pair: r^2 = (rx rx + ry ry) + rz rz as
// two fused steps, h = (r^2 + eps^2) + 1e-12 and 1 / sqrt(h).
template <typename V>
__device__ __forceinline__ void o8_soft_head(V rx, V ry, V rz, V eps2, V& r2, V& ir) {
  r2 = o8_fma(rz, rz, o8_fma(ry, ry, o8_mul(rx, rx)));
  ir = o8_rsqrt(o8_add(o8_add(r2, eps2), o8_splat_like(eps2, 1e-12f)));
}

// Whether a pair lies in the att = 1 range (no cutoff, or r^2 + 1e-12 under
// the unity radius): then its terms skip the erfc attenuation.
__device__ __forceinline__ bool o8_unity(float r2, const Soft& s) {
  return !(s.cutoff > 0.0f && o8_add(r2, 1e-12f) >= s.unity_r2);
}

// erfc attenuation of one pair outside the att = 1 range (soft_coeff's and
// soft_vjp_accum's slow path): att, and the VJP's radial term cc.
__device__ __forceinline__ void o8_soft_att(float r2, float ir3, const Soft& s, float& att, float& cc) {
  float dist = sqrtf(o8_add(r2, 1e-12f));
  float u = dist / (2.0f * s.cutoff);
  float e = 1.0f;
  att = 1.0f;
  if (u >= kAttUnityU) {
    e = expf(-(u * u));
    att = erfcf(u) + (2.0f / 1.772453850905516f) * u * e;
  }
  cc = ir3 * dist * e / (2.0f * 1.772453850905516f * s.cutoff * s.cutoff * s.cutoff);
}

// Softened force of one pair, nm = -m: acc += c r with c = nm / h^{3/2}
// (times att outside the att = 1 range).
__device__ __forceinline__ void o8_soft_force(float rx, float ry, float rz, float nm, float eps2, const Soft& s,
                                              float& ax, float& ay, float& az) {
  float r2, ir;
  o8_soft_head(rx, ry, rz, eps2, r2, ir);
  const float ir3 = o8_mul(o8_mul(ir, ir), ir);
  float c;
  if (o8_unity(r2, s)) {
    c = o8_mul(nm, ir3);
  } else {
    float att, cc;
    o8_soft_att(r2, ir3, s, att, cc);
    c = o8_mul(o8_mul(nm, att), ir3);
  }
  ax = o8_fma(c, rx, ax);
  ay = o8_fma(c, ry, ay);
  az = o8_fma(c, rz, az);
}

// Query-side VJP of one softened pair, nm = -m: acc += nm (lin g - rad r),
// with lin = att / h^{3/2} and rad = (r . g) (3 att / h^{5/2} + cc); the
// negated radial term is formed directly (rounding is symmetric in sign).
__device__ __forceinline__ void o8_soft_vjp(float rx, float ry, float rz, float nm, float gx, float gy, float gz,
                                            float eps2, const Soft& s, float& ax, float& ay, float& az) {
  float r2, ir;
  o8_soft_head(rx, ry, rz, eps2, r2, ir);
  const float ir3 = o8_mul(o8_mul(ir, ir), ir);
  const float ir5 = o8_mul(o8_mul(ir3, ir), ir);
  const float rg = o8_fma(rz, gz, o8_fma(ry, gy, o8_mul(rx, gx)));
  float lin, nrad;
  if (o8_unity(r2, s)) {
    lin = ir3;
    nrad = o8_mul(rg, o8_mul(-3.0f, ir5));
  } else {
    float att, cc;
    o8_soft_att(r2, ir3, s, att, cc);
    lin = o8_mul(att, ir3);
    nrad = o8_mul(rg, o8_sub(o8_mul(o8_mul(-3.0f, att), ir5), cc));
  }
  ax = o8_fma(nm, o8_fma(nrad, rx, o8_mul(lin, gx)), ax);
  ay = o8_fma(nm, o8_fma(nrad, ry, o8_mul(lin, gy)), ay);
  az = o8_fma(nm, o8_fma(nrad, rz, o8_mul(lin, gz)), az);
}

template <int KERNEL>
__device__ __forceinline__ void o8_pair(float qx, float qy, float qz, float px, float py, float pz, float m,
                                        float gx, float gy, float gz, const Soft& s, const Periodic& per,
                                        float& ax, float& ay, float& az) {
  if (KERNEL == O8_SOFT || KERNEL == O8_SOFT_VJP) {
    const float rx = min_image_floor(o8_sub(qx, px), per);
    const float ry = min_image_floor(o8_sub(qy, py), per);
    const float rz = min_image_floor(o8_sub(qz, pz), per);
    const float eps2 = o8_mul(s.eps, s.eps);
    if (KERNEL == O8_SOFT)
      o8_soft_force(rx, ry, rz, -m, eps2, s, ax, ay, az);
    else
      o8_soft_vjp(rx, ry, rz, -m, gx, gy, gz, eps2, s, ax, ay, az);
    return;
  }
  float rx = min_image_floor(qx - px, per);
  float ry = min_image_floor(qy - py, per);
  float rz = min_image_floor(qz - pz, per);
  if (KERNEL == O8_GRAV_GRAD) {
    float c = grav_grad_coeff(rx * rx + ry * ry + rz * rz, m);
    ax += c * rx;
    ay += c * ry;
    az += c * rz;
  } else {
    grav_grad_vjp_accum(rx, ry, rz, m, gx, gy, gz, ax, ay, az);
  }
}

// Two softened pairs without a periodic box, particles a then b: positions
// X, Y, Z and negated masses NM packed (a, b). The pair terms are packed, and
// each pair adds into the sums in order. With CHECK, a pair outside the
// att = 1 range sends both through the scalar form; without it the caller
// has shown that both pairs lie inside that range.
template <int KERNEL, bool CHECK>
__device__ __forceinline__ void o8_pair2(const F2& QX, const F2& QY, const F2& QZ, F2 X, F2 Y, F2 Z, F2 NM,
                                         const F2& GX, const F2& GY, const F2& GZ, float eps2, const Soft& s,
                                         float& ax, float& ay, float& az) {
  const F2 rx = o8_sub(QX, X), ry = o8_sub(QY, Y), rz = o8_sub(QZ, Z);
  F2 r2, ir;
  o8_soft_head(rx, ry, rz, f2_pack(eps2, eps2), r2, ir);
  float xa, xb, ya, yb, za, zb, ma, mb;
  f2_unpack(rx, xa, xb);
  f2_unpack(ry, ya, yb);
  f2_unpack(rz, za, zb);
  f2_unpack(NM, ma, mb);
  if (CHECK) {
    float r2a, r2b;
    f2_unpack(r2, r2a, r2b);
    if (!(o8_unity(r2a, s) && o8_unity(r2b, s))) {
      float gx, gy, gz, dummy;
      f2_unpack(GX, gx, dummy);
      f2_unpack(GY, gy, dummy);
      f2_unpack(GZ, gz, dummy);
      if (KERNEL == O8_SOFT) {
        o8_soft_force(xa, ya, za, ma, eps2, s, ax, ay, az);
        o8_soft_force(xb, yb, zb, mb, eps2, s, ax, ay, az);
      } else {
        o8_soft_vjp(xa, ya, za, ma, gx, gy, gz, eps2, s, ax, ay, az);
        o8_soft_vjp(xb, yb, zb, mb, gx, gy, gz, eps2, s, ax, ay, az);
      }
      return;
    }
  }
  const F2 ir3 = o8_mul(o8_mul(ir, ir), ir);
  if (KERNEL == O8_SOFT) {
    float ca, cb;
    f2_unpack(o8_mul(NM, ir3), ca, cb);
    ax = o8_fma(ca, xa, ax);
    ay = o8_fma(ca, ya, ay);
    az = o8_fma(ca, za, az);
    ax = o8_fma(cb, xb, ax);
    ay = o8_fma(cb, yb, ay);
    az = o8_fma(cb, zb, az);
  } else {
    const F2 ir5 = o8_mul(o8_mul(ir3, ir), ir);
    const F2 rg = o8_fma(rz, GZ, o8_fma(ry, GY, o8_mul(rx, GX)));
    const F2 nrad = o8_mul(rg, o8_mul(f2_pack(-3.0f, -3.0f), ir5));
    float ta, tb;
    f2_unpack(o8_fma(nrad, rx, o8_mul(ir3, GX)), ta, tb);
    ax = o8_fma(ma, ta, ax);
    ax = o8_fma(mb, tb, ax);
    f2_unpack(o8_fma(nrad, ry, o8_mul(ir3, GY)), ta, tb);
    ay = o8_fma(ma, ta, ay);
    ay = o8_fma(mb, tb, ay);
    f2_unpack(o8_fma(nrad, rz, o8_mul(ir3, GZ)), ta, tb);
    az = o8_fma(ma, ta, az);
    az = o8_fma(mb, tb, az);
  }
}

// One warp's staging buffer for a leaf's particles: 32 positions and
// negated masses, component by component, so that two or four consecutive
// particles load into packed register pairs with one shared-memory read.
constexpr int kO8LeafChunk = 32;

struct __align__(16) O8Chunk {
  float x[kO8LeafChunk], y[kO8LeafChunk], z[kO8LeafChunk], nm[kO8LeafChunk];
};

__device__ __forceinline__ F2 o8_ld2(const float* p) {
  F2 r;
  r.v = *reinterpret_cast<const unsigned long long*>(p);
  return r;
}

// The softened terms of cnt staged particles for one query, in order.
template <int KERNEL, bool CHECK>
__device__ __forceinline__ void o8_chunk_sum(const O8Chunk& ch, int cnt, float qx, float qy, float qz, float gx,
                                             float gy, float gz, const Soft& s, float& ax, float& ay, float& az) {
  const F2 QX = f2_pack(qx, qx), QY = f2_pack(qy, qy), QZ = f2_pack(qz, qz);
  const F2 GX = f2_pack(gx, gx), GY = f2_pack(gy, gy), GZ = f2_pack(gz, gz);
  const float eps2 = o8_mul(s.eps, s.eps);
  int j = 0;
  for (; j + 3 < cnt; j += 4) {
    const ulonglong2 X = *reinterpret_cast<const ulonglong2*>(&ch.x[j]);
    const ulonglong2 Y = *reinterpret_cast<const ulonglong2*>(&ch.y[j]);
    const ulonglong2 Z = *reinterpret_cast<const ulonglong2*>(&ch.z[j]);
    const ulonglong2 M = *reinterpret_cast<const ulonglong2*>(&ch.nm[j]);
    o8_pair2<KERNEL, CHECK>(QX, QY, QZ, F2{X.x}, F2{Y.x}, F2{Z.x}, F2{M.x}, GX, GY, GZ, eps2, s, ax, ay, az);
    o8_pair2<KERNEL, CHECK>(QX, QY, QZ, F2{X.y}, F2{Y.y}, F2{Z.y}, F2{M.y}, GX, GY, GZ, eps2, s, ax, ay, az);
  }
  if (j + 1 < cnt) {
    o8_pair2<KERNEL, CHECK>(QX, QY, QZ, o8_ld2(&ch.x[j]), o8_ld2(&ch.y[j]), o8_ld2(&ch.z[j]), o8_ld2(&ch.nm[j]),
                            GX, GY, GZ, eps2, s, ax, ay, az);
    j += 2;
  }
  if (j < cnt) {
    const float rx = o8_sub(qx, ch.x[j]), ry = o8_sub(qy, ch.y[j]), rz = o8_sub(qz, ch.z[j]);
    if (KERNEL == O8_SOFT)
      o8_soft_force(rx, ry, rz, ch.nm[j], eps2, s, ax, ay, az);
    else
      o8_soft_vjp(rx, ry, rz, ch.nm[j], gx, gy, gz, eps2, s, ax, ay, az);
  }
}

// Whether every pair of the query with a particle inside the cell (centre
// c, half size h, as o8_in_cell tests it) lies in the att = 1 range: the
// farthest corner's squared distance stays under the unity radius, with an
// absolute slack per axis (1e-6 of the magnitudes involved) and a relative
// margin (1e-4) far above the rounding of the differences and of r^2.
__device__ __forceinline__ bool o8_cell_unity(float qx, float qy, float qz, const OctreeNode8& nd, const Soft& s) {
  if (!(s.cutoff > 0.0f)) return true;
  const float h = nd.half_size;
  const float mx = fabsf(qx - nd.cx) + h + 1e-6f * (fabsf(qx) + fabsf(nd.cx) + h);
  const float my = fabsf(qy - nd.cy) + h + 1e-6f * (fabsf(qy) + fabsf(nd.cy) + h);
  const float mz = fabsf(qz - nd.cz) + h + 1e-6f * (fabsf(qz) + fabsf(nd.cz) + h);
  const float R2 = mx * mx + my * my + mz * mz;
  return R2 * 1.0001f + 1e-12f < s.unity_r2;
}

__device__ __forceinline__ bool o8_in_cell(float px, float py, float pz, const OctreeNode8& nd) {
  const float h = nd.half_size;
  return fabsf(px - nd.cx) <= h && fabsf(py - nd.cy) <= h && fabsf(pz - nd.cz) <= h;
}

// Direct softened sums without a periodic box, two queries per thread (q
// and q + blockDim.x of the block's 2 blockDim.x queries). Particles are
// staged per tile already splatted ((x, x), (y, y), (z, z), (-m, -m)), so each
// shared-memory read lands in a packed register pair. When every pair of the
// tile with the block's queries lies in the att = 1 range (the farthest
// corners of the two bounding boxes, with margins, inside the unity radius:
// always so under the "no cutoff" convention), each particle meets both
// queries in one pass of FFMA2 / FADD2 / FMUL2 in the fixed order of
// o8_soft_force and o8_soft_vjp, with the tile sums packed too. Otherwise the
// tile takes those scalar forms query by query. Both round every component
// the same way. Each tile's sum joins the query's Kahan-compensated total,
// as in direct_soft_kernel.
struct __align__(16) DirectSplat {
  F2 x, y, z, nm;
};

constexpr int kDirectWarps = kDirectThreads / 32;

// Box of the block's values: v[0..2] minima, v[3..5] maxima over the warp,
// then over the warps through part[kDirectWarps][8] (the caller syncs the
// block between the two calls).
__device__ __forceinline__ void direct_box_warp(float* v, float (*part)[8]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      v[d] = fminf(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
      v[3 + d] = fmaxf(v[3 + d], __shfl_xor_sync(0xffffffffu, v[3 + d], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 6; d++) part[threadIdx.x >> 5][d] = v[d];
}

__device__ __forceinline__ void direct_box_block(float* v, const float (*part)[8]) {
  for (int d = 0; d < 3; d++) {
    v[d] = part[0][d];
    v[3 + d] = part[0][3 + d];
  }
  for (int w = 1; w < kDirectWarps; w++)
    for (int d = 0; d < 3; d++) {
      v[d] = fminf(v[d], part[w][d]);
      v[3 + d] = fmaxf(v[3 + d], part[w][3 + d]);
    }
}

template <bool VJP>
__global__ void __launch_bounds__(kDirectThreads, 4)
    direct_soft2_kernel(const float* __restrict__ pts, const float* __restrict__ masses, int64_t n,
                        const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq,
                        float* __restrict__ out, Soft s) {
  __shared__ DirectSplat tile[kDirectThreads];
  __shared__ float qpart[kDirectWarps][8], tpart[kDirectWarps][8];
  const int64_t qa = static_cast<int64_t>(blockIdx.x) * (2 * kDirectThreads) + threadIdx.x;
  const int64_t qb = qa + kDirectThreads;
  float q[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, g[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int64_t qi = t ? qb : qa;
    if (qi < nq) {
      for (int d = 0; d < 3; d++) {
        q[t][d] = queries[3 * qi + d];
        if (VJP) g[t][d] = cot[3 * qi + d];
      }
    }
  }
  float qbox[6];
  for (int d = 0; d < 3; d++) {
    qbox[d] = fminf(q[0][d], q[1][d]);
    qbox[3 + d] = fmaxf(q[0][d], q[1][d]);
  }
  direct_box_warp(qbox, qpart);
  const F2 QX = f2_pack(q[0][0], q[1][0]), QY = f2_pack(q[0][1], q[1][1]), QZ = f2_pack(q[0][2], q[1][2]);
  const F2 GX = f2_pack(g[0][0], g[1][0]), GY = f2_pack(g[0][1], g[1][1]), GZ = f2_pack(g[0][2], g[1][2]);
  const float eps2 = o8_mul(s.eps, s.eps);
  const F2 EPS2 = f2_pack(eps2, eps2), M3 = f2_pack(-3.0f, -3.0f), ZERO = f2_pack(0.0f, 0.0f);
  float sum[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, comp[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  for (int64_t base = 0; base < n; base += kDirectThreads) {
    const int64_t j = base + threadIdx.x;
    float px = 0.f, py = 0.f, pz = 0.f, pm = 0.f;
    float tbox[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if (j < n) {
      px = pts[3 * j];
      py = pts[3 * j + 1];
      pz = pts[3 * j + 2];
      pm = masses[j];
      tbox[0] = tbox[3] = px;
      tbox[1] = tbox[4] = py;
      tbox[2] = tbox[5] = pz;
    }
    tile[threadIdx.x] = DirectSplat{f2_pack(px, px), f2_pack(py, py), f2_pack(pz, pz), f2_pack(-pm, -pm)};
    direct_box_warp(tbox, tpart);
    __syncthreads();
    // the farthest corners of the query box and the tile box (block-uniform)
    bool unity = !(s.cutoff > 0.0f);
    if (!unity) {
      float qb6[6], tb6[6], R2 = 0.0f;
      direct_box_block(qb6, qpart);
      direct_box_block(tb6, tpart);
      for (int d = 0; d < 3; d++) {
        const float span = fmaxf(fabsf(qb6[3 + d] - tb6[d]), fabsf(tb6[3 + d] - qb6[d]));
        const float mag = fmaxf(fmaxf(fabsf(qb6[d]), fabsf(qb6[3 + d])), fmaxf(fabsf(tb6[d]), fabsf(tb6[3 + d])));
        const float m = span + 1e-6f * mag;
        R2 += m * m;
      }
      unity = R2 * 1.0001f + 1e-12f < s.unity_r2;
    }
    const int cnt = static_cast<int>(n - base < kDirectThreads ? n - base : kDirectThreads);
    float a[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    if (unity) {
      F2 AX = ZERO, AY = ZERO, AZ = ZERO;
#pragma unroll 4
      for (int k = 0; k < cnt; k++) {
        const DirectSplat p = tile[k];
        const F2 rx = o8_sub(QX, p.x), ry = o8_sub(QY, p.y), rz = o8_sub(QZ, p.z);
        F2 r2, ir;
        o8_soft_head(rx, ry, rz, EPS2, r2, ir);
        const F2 ir3 = o8_mul(o8_mul(ir, ir), ir);
        if (!VJP) {
          const F2 c = o8_mul(p.nm, ir3);
          AX = o8_fma(c, rx, AX);
          AY = o8_fma(c, ry, AY);
          AZ = o8_fma(c, rz, AZ);
        } else {
          const F2 ir5 = o8_mul(o8_mul(ir3, ir), ir);
          const F2 rg = o8_fma(rz, GZ, o8_fma(ry, GY, o8_mul(rx, GX)));
          const F2 nrad = o8_mul(rg, o8_mul(M3, ir5));
          AX = o8_fma(p.nm, o8_fma(nrad, rx, o8_mul(ir3, GX)), AX);
          AY = o8_fma(p.nm, o8_fma(nrad, ry, o8_mul(ir3, GY)), AY);
          AZ = o8_fma(p.nm, o8_fma(nrad, rz, o8_mul(ir3, GZ)), AZ);
        }
      }
      f2_unpack(AX, a[0][0], a[1][0]);
      f2_unpack(AY, a[0][1], a[1][1]);
      f2_unpack(AZ, a[0][2], a[1][2]);
    } else {
      for (int k = 0; k < cnt; k++) {
        const DirectSplat p = tile[k];
        float x, y, z, nm, unused;
        f2_unpack(p.x, x, unused);
        f2_unpack(p.y, y, unused);
        f2_unpack(p.z, z, unused);
        f2_unpack(p.nm, nm, unused);
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const float rx = o8_sub(q[t][0], x), ry = o8_sub(q[t][1], y), rz = o8_sub(q[t][2], z);
          if (VJP)
            o8_soft_vjp(rx, ry, rz, nm, g[t][0], g[t][1], g[t][2], eps2, s, a[t][0], a[t][1], a[t][2]);
          else
            o8_soft_force(rx, ry, rz, nm, eps2, s, a[t][0], a[t][1], a[t][2]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < 2; t++)
      for (int d = 0; d < 3; d++) kahan_add(sum[t][d], comp[t][d], a[t][d]);
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int64_t qi = t ? qb : qa;
    if (qi < nq)
      for (int d = 0; d < 3; d++) out[3 * qi + d] = sum[t][d];
  }
}

// One query's terms from leaf particles [start, end), in order; softened
// pairs without a periodic box go two at a time through o8_pair2.
template <int KERNEL>
__device__ __forceinline__ void o8_leaf_sum(const Leaf3* __restrict__ leaf, uint32_t start, uint32_t end,
                                            float qx, float qy, float qz, float gx, float gy, float gz,
                                            const Soft& s, const Periodic& per, float& ax, float& ay,
                                            float& az) {
  uint32_t i = start;
  if ((KERNEL == O8_SOFT || KERNEL == O8_SOFT_VJP) && !per.on) {
    const F2 QX = f2_pack(qx, qx), QY = f2_pack(qy, qy), QZ = f2_pack(qz, qz);
    const F2 GX = f2_pack(gx, gx), GY = f2_pack(gy, gy), GZ = f2_pack(gz, gz);
    const float eps2 = o8_mul(s.eps, s.eps);
    for (; i + 1 < end; i += 2) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(leaf + i));
      const float4 b = __ldg(reinterpret_cast<const float4*>(leaf + i + 1));
      const float ma = __ldg(&leaf[i].mass), mb = __ldg(&leaf[i + 1].mass);
      o8_pair2<KERNEL, true>(QX, QY, QZ, f2_pack(a.x, b.x), f2_pack(a.y, b.y), f2_pack(a.z, b.z), f2_pack(-ma, -mb),
                             GX, GY, GZ, eps2, s, ax, ay, az);
    }
  }
  for (; i < end; i++) {
    const float4* p = reinterpret_cast<const float4*>(leaf + i);
    float4 a = __ldg(p);
    float m = __ldg(&leaf[i].mass);
    o8_pair<KERNEL>(qx, qy, qz, a.x, a.y, a.z, m, gx, gy, gz, s, per, ax, ay, az);
  }
}

// Buffers come from the caller: child indices and leaf ranges are checked
// against the buffer sizes and a violation sets SBH_DEV_BAD_BOUNDS instead of
// reading out of bounds.
struct O8Bounds {
  uint32_t num_nodes;
  uint32_t num_leaves;
};

__device__ __forceinline__ bool o8_node_ok(uint32_t idx, const O8Bounds& bd, uint32_t* status) {
  if (idx < bd.num_nodes) return true;
  raise_status(status, SBH_DEV_BAD_BOUNDS);
  return false;
}

__device__ __forceinline__ uint32_t o8_leaf_end(uint32_t start, uint32_t end, const O8Bounds& bd,
                                                uint32_t* status) {
  if (end <= bd.num_leaves && start <= end) return end;
  raise_status(status, SBH_DEV_BAD_BOUNDS);
  return start <= bd.num_leaves ? (end < bd.num_leaves ? end : bd.num_leaves) : start;
}

template <int KERNEL>
__global__ void __launch_bounds__(256)
    o8_bh_kernel(const Leaf3* __restrict__ leaf, const OctreeNode8* __restrict__ nodes,
                 const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq, float beta,
                 Soft s, int prune_on, float r_cut_sq, Periodic per, float* __restrict__ out,
                 uint32_t* status, O8Bounds bd, const uint32_t* __restrict__ order) {
  int64_t ti = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (ti >= nq) return;
  const int64_t qi = order ? static_cast<int64_t>(order[ti]) : ti;
  float qx = queries[3 * qi], qy = queries[3 * qi + 1], qz = queries[3 * qi + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  if (KERNEL == O8_SOFT_VJP || KERNEL == O8_GRAV_GRAD_VJP) {
    gx = cot[3 * qi];
    gy = cot[3 * qi + 1];
    gz = cot[3 * qi + 2];
  }
  float ax = 0.f, ay = 0.f, az = 0.f;
  int stack[kO8Stack];
  int top = 0;
  stack[top++] = 0;
  bool overflow = false;
  // A well-formed tree reaches each node from the root exactly once, so one
  // query pops at most num_nodes nodes. More pops mean that the caller's
  // child indices form a cycle: stop, flag it and keep the partial sum.
  uint32_t visits = 0;
  while (top > 0) {
    if (++visits > bd.num_nodes) {
      raise_status(status, SBH_DEV_ITER_LIMIT);
      break;
    }
    int idx = stack[--top];
    if (o8_mass(nodes, idx) == 0.0f) continue;
    const OctreeNode8& nd = nodes[idx];
    if (KERNEL != O8_GRAV_GRAD && KERNEL != O8_GRAV_GRAD_VJP &&
        o8_prune(nd, qx, qy, qz, prune_on, r_cut_sq, per))
      continue;
    if (o8_far(nd, qx, qy, qz, beta, per)) {
      if (nd.is_leaf) {
        o8_leaf_sum<KERNEL>(leaf, nd.start, o8_leaf_end(nd.start, nd.end, bd, status), qx, qy, qz, gx, gy, gz, s,
                            per, ax, ay, az);
      } else {
        o8_pair<KERNEL>(qx, qy, qz, nd.contrib.pos[0], nd.contrib.pos[1], nd.contrib.pos[2], nd.contrib.mass,
                        gx, gy, gz, s, per, ax, ay, az);
      }
    } else {
      uint8_t mask = nd.child_mask;
      for (int c = 0; c < 8; c++) {
        if (mask & (1u << c)) {
          if (!o8_node_ok(nd.child[c], bd, status)) continue;
          if (top < kO8Stack) {
            stack[top++] = static_cast<int>(nd.child[c]);
          } else {
            overflow = true;
          }
        }
      }
    }
  }
  if (overflow) raise_status(status, SBH_DEV_STACK_OVERFLOW);
  out[3 * qi] = ax;
  out[3 * qi + 1] = ay;
  out[3 * qi + 2] = az;
}

// Warp-cooperative form of o8_bh_kernel, for queries taken in Morton order
// (32 neighbouring queries per warp). The warp walks one DFS stack in shared
// memory whose entries carry the lanes that still descend at that node, and
// each lane takes its own prune and opening decisions, exactly as its thread
// does in o8_bh_kernel: a node is pushed (children in the same order) when
// some lane opens it, with that set of lanes. A lane's nodes thus come off
// the stack in the order of its own per-thread DFS, so it adds the same terms
// in the same order and every output row equals o8_bh_kernel's bit for bit;
// node records are read once per warp instead of once per thread. At a leaf
// the warp copies the particles in chunks of 32 (one coalesced load per lane)
// into a per-warp buffer in shared memory, and the summing lanes read them
// from there in the leaf's order.
// The block holds blockDim.x / 32 warps (the caller's `threads`, the
// reference's launch parameter, in whole warps). Its dynamic shared memory
// holds each warp's leaf buffer (32 x 16 B), then each warp's stack of STACK
// entries: 64 for a dense octree8 of depth <= 9 (a DFS of depth d holds at
// most 7 d + 1 entries), otherwise the reference's 128.
struct O8StackEntry {
  int node;
  uint32_t lanes;
};

__host__ __device__ constexpr size_t o8_warp_smem(int warps, int stack) {
  return static_cast<size_t>(warps) * (sizeof(O8Chunk) + stack * sizeof(O8StackEntry));
}

template <int KERNEL, int STACK, bool STAGED>
__global__ void __launch_bounds__(1024)
    o8_bh_warp_kernel(const Leaf3* __restrict__ leaf, const OctreeNode8* __restrict__ nodes,
                      const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq, float beta,
                      Soft s, int prune_on, float r_cut_sq, Periodic per, float* __restrict__ out, uint32_t* status,
                      O8Bounds bd, const uint32_t* __restrict__ order) {
  extern __shared__ float4 o8_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  O8Chunk& chunk = reinterpret_cast<O8Chunk*>(o8_smem)[warp];
  O8StackEntry* stack = reinterpret_cast<O8StackEntry*>(reinterpret_cast<O8Chunk*>(o8_smem) + (blockDim.x >> 5)) +
                        warp * STACK;
  const int64_t ti = (static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp) * 32 + lane;
  const bool valid = ti < nq;
  const uint32_t live = __ballot_sync(0xffffffffu, valid);
  if (live == 0) return;  // warp-uniform
  const int64_t qi = valid ? static_cast<int64_t>(order[ti]) : 0;
  float qx = 0.f, qy = 0.f, qz = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
  if (valid) {
    qx = queries[3 * qi];
    qy = queries[3 * qi + 1];
    qz = queries[3 * qi + 2];
    if (KERNEL == O8_SOFT_VJP || KERNEL == O8_GRAV_GRAD_VJP) {
      gx = cot[3 * qi];
      gy = cot[3 * qi + 1];
      gz = cot[3 * qi + 2];
    }
  }
  float ax = 0.f, ay = 0.f, az = 0.f;
  if (lane == 0) stack[0] = O8StackEntry{0, live};
  __syncwarp();
  int top = 1;  // warp-uniform
  bool overflow = false;
  uint32_t visits = 0;  // bounded as in o8_bh_kernel
  while (top > 0) {
    if (++visits > bd.num_nodes) {
      if (lane == 0) raise_status(status, SBH_DEV_ITER_LIMIT);
      break;
    }
    const O8StackEntry en = stack[--top];
    __syncwarp();  // every lane has read the entry before it is overwritten
    const int idx = en.node;
    if (o8_mass(nodes, idx) == 0.0f) continue;
    const OctreeNode8& nd = nodes[idx];
    bool act = (en.lanes >> lane) & 1u;
    if (KERNEL != O8_GRAV_GRAD && KERNEL != O8_GRAV_GRAD_VJP)
      act = act && !o8_prune(nd, qx, qy, qz, prune_on, r_cut_sq, per);
    const bool far = act && o8_far(nd, qx, qy, qz, beta, per);
    if (nd.is_leaf && !STAGED) {  // nd is warp-uniform: every lane reads the same node
      if (far)
        o8_leaf_sum<KERNEL>(leaf, nd.start, o8_leaf_end(nd.start, nd.end, bd, status), qx, qy, qz, gx, gy, gz, s,
                            per, ax, ay, az);
    } else if (nd.is_leaf) {
      if (__ballot_sync(0xffffffffu, far)) {
        const uint32_t start = nd.start, end = o8_leaf_end(start, nd.end, bd, status);
        constexpr bool kSoft = KERNEL == O8_SOFT || KERNEL == O8_SOFT_VJP;
        const bool q_unity = !far || o8_cell_unity(qx, qy, qz, nd, s);
        // chunks of 32 particles, one per lane, the next one loaded while
        // the current one is summed
        float4 nxt = make_float4(0.f, 0.f, 0.f, 0.f);
        float nxt_m = 0.f;
        if (start + lane < end) {
          nxt = __ldg(reinterpret_cast<const float4*>(leaf + start + lane));
          nxt_m = __ldg(&leaf[start + lane].mass);
        }
        for (uint32_t c = start; c < end; c += kO8LeafChunk) {
          const uint32_t i = c + lane;
          bool in_cell = true;
          if (i < end) {
            chunk.x[lane] = nxt.x;
            chunk.y[lane] = nxt.y;
            chunk.z[lane] = nxt.z;
            chunk.nm[lane] = -nxt_m;
            in_cell = o8_in_cell(nxt.x, nxt.y, nxt.z, nd);
          }
          if (i + kO8LeafChunk < end) {
            nxt = __ldg(reinterpret_cast<const float4*>(leaf + i + kO8LeafChunk));
            nxt_m = __ldg(&leaf[i + kO8LeafChunk].mass);
          }
          const bool unity = __all_sync(0xffffffffu, in_cell && q_unity);
          __syncwarp();
          const int cnt = end - c < kO8LeafChunk ? static_cast<int>(end - c) : kO8LeafChunk;
          if (far) {
            if (kSoft && !per.on) {
              if (unity)
                o8_chunk_sum<KERNEL, false>(chunk, cnt, qx, qy, qz, gx, gy, gz, s, ax, ay, az);
              else
                o8_chunk_sum<KERNEL, true>(chunk, cnt, qx, qy, qz, gx, gy, gz, s, ax, ay, az);
            } else {
              for (int j = 0; j < cnt; j++)
                o8_pair<KERNEL>(qx, qy, qz, chunk.x[j], chunk.y[j], chunk.z[j], -chunk.nm[j], gx, gy, gz, s, per,
                                ax, ay, az);
            }
          }
          __syncwarp();  // the chunk is read before the next one overwrites it
        }
      }
    } else if (far) {
      o8_pair<KERNEL>(qx, qy, qz, nd.contrib.pos[0], nd.contrib.pos[1], nd.contrib.pos[2], nd.contrib.mass, gx, gy,
                      gz, s, per, ax, ay, az);
    }
    const uint32_t open = __ballot_sync(0xffffffffu, act && !far);
    if (open) {
      const uint8_t mask = nd.child_mask;
      for (int c = 0; c < 8; c++) {
        if (mask & (1u << c)) {
          if (!o8_node_ok(nd.child[c], bd, status)) continue;
          if (top < STACK) {
            if (lane == 0) stack[top] = O8StackEntry{static_cast<int>(nd.child[c]), open};
            top++;
          } else {
            overflow = true;
          }
        }
      }
      __syncwarp();
    }
  }
  if (overflow && lane == 0) raise_status(status, SBH_DEV_STACK_OVERFLOW);
  if (valid) {
    out[3 * qi] = ax;
    out[3 * qi + 1] = ay;
    out[3 * qi + 2] = az;
  }
}

// ---------------------------------------------------------------------------
// octree8 stochastic BH, the multi-level prefix control variate
// (src/sbh_ffi.cu:2146-2442). Same curand calls as the reference, so a
// fixed seed gives the reference's sample paths.
// ---------------------------------------------------------------------------
constexpr int kControlDepth = 3;
constexpr int kMaxSubdomains = 512;
constexpr int kO8MaxDescent = 64;

template <int KERNEL>
__device__ __forceinline__ void o8_contrib_pair(const OctreeNode8& nd, float qx, float qy, float qz, float gx,
                                                float gy, float gz, const Soft& s, const Periodic& per,
                                                float& ax, float& ay, float& az) {
  o8_pair<KERNEL>(qx, qy, qz, nd.contrib.pos[0], nd.contrib.pos[1], nd.contrib.pos[2], nd.contrib.mass, gx,
                  gy, gz, s, per, ax, ay, az);
}

__device__ __forceinline__ uint32_t o8_child_slot(const OctreeNode8& nd, float px, float py, float pz) {
  uint32_t ix = px >= nd.cx ? 1u : 0u;
  uint32_t iy = py >= nd.cy ? 1u : 0u;
  uint32_t iz = pz >= nd.cz ? 1u : 0u;
  return ix | (iy << 1) | (iz << 2);
}

template <int KERNEL, bool SOFTENED>
__global__ void __launch_bounds__(256)
    o8_stochastic_kernel(const Leaf3* __restrict__ leaf, const OctreeNode8* __restrict__ nodes,
                         const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq,
                         int samples, int seed, float beta, Soft s, int prune_on, float r_cut_sq,
                         Periodic per, float* __restrict__ out, uint32_t* status, O8Bounds bd,
                         const uint32_t* __restrict__ order) {
  int64_t ti = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (ti >= nq) return;
  const int64_t qi = order ? static_cast<int64_t>(order[ti]) : ti;
  float qx = queries[3 * qi], qy = queries[3 * qi + 1], qz = queries[3 * qi + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  if (KERNEL == O8_SOFT_VJP || KERNEL == O8_GRAV_GRAD_VJP) {
    gx = cot[3 * qi];
    gy = cot[3 * qi + 1];
    gz = cot[3 * qi + 2];
  }
  // curand_init(seed + q, 0, 0) and curand_init(seed + q + 0x9e3779b9, 0, 0):
  // int addition, then sign extension (first) or u32 wraparound (second).
  int sq = seed + static_cast<int>(qi);
  curandState st, st2;
  curand_init(static_cast<unsigned long long>(static_cast<long long>(sq)), 0, 0, &st);
  curand_init(static_cast<unsigned long long>(static_cast<unsigned>(sq) + 0x9e3779b9u), 0, 0, &st2);

  float tx = 0.f, ty = 0.f, tz = 0.f;
  int stack[kO8Stack];
  int top = 0;
  stack[top++] = 0;
  uint32_t subs[kMaxSubdomains];
  int nsub = 0;
  bool overflow = false;
  uint32_t visits = 0;  // bounded as in o8_bh_kernel
  while (top > 0) {
    if (++visits > bd.num_nodes) {
      raise_status(status, SBH_DEV_ITER_LIMIT);
      break;
    }
    int idx = stack[--top];
    const OctreeNode8& nd = nodes[idx];
    if (nd.contrib.mass == 0.0f) continue;
    if (nd.is_leaf || nd.depth >= kControlDepth) {
      if (nsub < kMaxSubdomains) subs[nsub++] = static_cast<uint32_t>(idx);
      continue;
    }
    uint8_t mask = nd.child_mask;
    for (int c = 0; c < 8; c++) {
      if (mask & (1u << c)) {
        if (!o8_node_ok(nd.child[c], bd, status)) continue;
        if (top < kO8Stack)
          stack[top++] = static_cast<int>(nd.child[c]);
        else
          overflow = true;
      }
    }
  }
  for (int sd = 0; sd < nsub; sd++) {
    const OctreeNode8& sub = nodes[subs[sd]];
    if (SOFTENED && o8_prune(sub, qx, qy, qz, prune_on, r_cut_sq, per)) continue;
    uint32_t sub_end = o8_leaf_end(sub.start, sub.end, bd, status);
    if (sub.is_leaf) {
      o8_leaf_sum<KERNEL>(leaf, sub.start, sub_end, qx, qy, qz, gx, gy, gz, s, per, tx, ty, tz);
    } else {
      o8_contrib_pair<KERNEL>(sub, qx, qy, qz, gx, gy, gz, s, per, tx, ty, tz);
    }
    if (sub_end <= sub.start) continue;
    uint32_t num_el = sub.end - sub.start;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int ss = 0; ss < samples; ss++) {
      uint32_t pick = min(static_cast<uint32_t>(num_el * curand_uniform(&st2)) + sub.start, sub_end - 1);
      float spx = leaf[pick].pos[0], spy = leaf[pick].pos[1], spz = leaf[pick].pos[2];
      const OctreeNode8* prev = &sub;
      const OctreeNode8* cur = &sub;
      float event_prob = 1.0f;
      float wx = 0.f, wy = 0.f, wz = 0.f;
      float dx = min_image_floor(qx - cur->cx, per);
      float dy = min_image_floor(qy - cur->cy, per);
      float dz = min_image_floor(qz - cur->cz, per);
      float cur_beta = fmaxf(beta, sqrtf(dx * dx + dy * dy + dz * dz) / cur->diameter);
      // Each step goes one level down a tree of depth <= 10; a longer descent
      // follows a cycle in the caller's child indices.
      int steps = 0;
      while (!cur->is_leaf) {
        if (++steps > kO8MaxDescent) {
          raise_status(status, SBH_DEV_ITER_LIMIT);
          break;
        }
        if (SOFTENED && o8_prune(*cur, qx, qy, qz, prune_on, r_cut_sq, per)) break;
        float ex = min_image_floor(qx - cur->cx, per);
        float ey = min_image_floor(qy - cur->cy, per);
        float ez = min_image_floor(qz - cur->cz, per);
        float dist = sqrtf(ex * ex + ey * ey + ez * ez);
        float ffr = dist / cur->diameter;
        float tp = fminf(cur_beta / ffr, 1.0f);
        float p = curand_uniform(&st);
        if (p > tp) {
          event_prob *= 1.0f - tp;
          break;
        }
        event_prob *= tp;
        prev = cur;
        uint32_t slot = o8_child_slot(*cur, spx, spy, spz);
        if (!(cur->child_mask & (1u << slot))) break;
        if (!o8_node_ok(cur->child[slot], bd, status)) break;
        cur = &nodes[cur->child[slot]];
        cur_beta = fmaxf(cur_beta, ffr);
        float px_ = 0.f, py_ = 0.f, pz_ = 0.f;
        o8_contrib_pair<KERNEL>(*prev, qx, qy, qz, gx, gy, gz, s, per, px_, py_, pz_);
        float cx_ = 0.f, cy_ = 0.f, cz_ = 0.f;
        uint8_t mask = prev->child_mask;
        for (int cc = 0; cc < 8; cc++) {
          if (!(mask & (1u << cc))) continue;
          if (!o8_node_ok(prev->child[cc], bd, status)) continue;
          const OctreeNode8& ch = nodes[prev->child[cc]];
          if (SOFTENED && o8_prune(ch, qx, qy, qz, prune_on, r_cut_sq, per)) continue;
          if (ch.is_leaf) {
            o8_leaf_sum<KERNEL>(leaf, ch.start, o8_leaf_end(ch.start, ch.end, bd, status), qx, qy, qz, gx, gy, gz, s,
                                per, cx_, cy_, cz_);
          } else {
            o8_contrib_pair<KERNEL>(ch, qx, qy, qz, gx, gy, gz, s, per, cx_, cy_, cz_);
          }
        }
        float pinv = static_cast<float>(num_el) / (event_prob * static_cast<float>(prev->end - prev->start));
        wx += pinv * (cx_ - px_);
        wy += pinv * (cy_ - py_);
        wz += pinv * (cz_ - pz_);
      }
      sx += wx;
      sy += wy;
      sz += wz;
    }
    if (samples > 0) {
      float inv = static_cast<float>(samples);
      tx += sx / inv;
      ty += sy / inv;
      tz += sz / inv;
    }
  }
  if (overflow) raise_status(status, SBH_DEV_STACK_OVERFLOW);
  out[3 * qi] = tx;
  out[3 * qi + 1] = ty;
  out[3 * qi + 2] = tz;
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
static int check_threads(int threads) {
  if (threads <= 0 || threads > 1024) return invalid("threads must be in [1, 1024]");
  return SBH_OK;
}

static unsigned grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

static unsigned grid_stride(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 64) b = 148 * 64;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename Body>
static int o8_layout_checks(const void* leaf, size_t leaf_bytes, const void* nodes, size_t node_bytes,
                            const float* queries, int64_t nq, Body) {
  if (leaf_bytes % sizeof(Leaf3) != 0) return invalid("leaf_bytes size mismatch");
  if (node_bytes % sizeof(OctreeNode8) != 0) return invalid("node_bytes size mismatch");
  if (node_bytes == 0) return invalid("node_bytes must hold at least the root");
  if (nq < 0) return invalid("num_queries must be >= 0");
  if (nq > 0 && !queries) return invalid("queries must be non-null");
  if ((leaf_bytes > 0 && !aligned16(leaf)) || !aligned16(nodes)) return invalid("leaf/node buffers must be 16-byte aligned");
  return SBH_OK;
}

template <typename C>
static void o8_carve(C& c, int64_t n, int depth, O8Params** prm, uint32_t** k0, uint32_t** v0,
                     uint32_t** k1, uint32_t** v1, uint32_t** counts, uint32_t** hist, uint32_t** scan_tmp,
                     DVec<7>** P, DVec<7>** ptmp) {
  uint64_t cells = 1ull << (3 * depth);
  int64_t nn = n > 0 ? n : 1;
  *prm = c.template take<O8Params>(1);
  *k0 = c.template take<uint32_t>(nn);
  *v0 = c.template take<uint32_t>(nn);
  *k1 = c.template take<uint32_t>(nn);
  *v1 = c.template take<uint32_t>(nn);
  *counts = c.template take<uint32_t>(cells + 1);
  int64_t hist_n = radix_hist_elems(nn);
  *hist = c.template take<uint32_t>(hist_n);
  int64_t st = scan_tiles(static_cast<int64_t>(cells) + 1);
  int64_t st2 = scan_tiles(hist_n);
  *scan_tmp = c.template take<uint32_t>(st > st2 ? st : st2);
  *P = c.template take<DVec<7>>(nn + 1);
  *ptmp = c.template take<DVec<7>>(scan_tiles<DVec<7>>(nn));
}

}  // namespace sbh

using namespace sbh;

// Query order of the per-query octree8 traversals. Each query walks the
// tree on its own (the deterministic kernels) or with curand streams seeded
// by its own index (the stochastic ones), so the order in which threads take
// queries changes no result; it only decides which queries share a warp.
// With a large enough workspace the queries are sorted by the 30-bit Morton
// code of their position in the root cell, so a warp's threads walk nearby
// paths and the per-thread traversal diverges far less than for queries in
// random order.
constexpr int64_t kOrderMinQueries = 4096;

template <typename C>
static void order_carve(C& c, int64_t nq, uint32_t** k0, uint32_t** v0, uint32_t** k1, uint32_t** v1,
                        uint32_t** hist, uint32_t** tmp) {
  *k0 = c.template take<uint32_t>(static_cast<size_t>(nq));
  *v0 = c.template take<uint32_t>(static_cast<size_t>(nq));
  *k1 = c.template take<uint32_t>(static_cast<size_t>(nq));
  *v1 = c.template take<uint32_t>(static_cast<size_t>(nq));
  int64_t h = radix_hist_elems(nq);
  *hist = c.template take<uint32_t>(static_cast<size_t>(h));
  *tmp = c.template take<uint32_t>(static_cast<size_t>(scan_tiles<uint32_t>(h)));
}

// 10 bits per axis of the query's position in the root cell (clamped; NaN
// goes to 0), interleaved x, y, z from bit 0.
__global__ void o8_query_codes_kernel(const OctreeNode8* __restrict__ nodes, const float* __restrict__ q,
                                      int64_t nq, uint32_t* __restrict__ codes) {
  const float h = nodes[0].half_size;
  const float lo[3] = {nodes[0].cx - h, nodes[0].cy - h, nodes[0].cz - h};
  const float scale = h > 0.0f ? 512.0f / h : 0.0f;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nq;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t c = 0;
    for (int d = 0; d < 3; d++) {
      float t = (q[3 * i + d] - lo[d]) * scale;
      uint32_t v = t > 0.0f ? (t < 1023.0f ? static_cast<uint32_t>(t) : 1023u) : 0u;
      for (int b = 0; b < 10; b++) c |= ((v >> b) & 1u) << (3 * b + d);
    }
    codes[i] = c;
  }
}

// The sorted query order, or null (input order) when nq is small or the
// workspace has no room for the sort.
static const uint32_t* o8_query_order(cudaStream_t stream, const OctreeNode8* nodes, const float* queries,
                                      int64_t nq, void* workspace, size_t workspace_bytes, int* rc) {
  *rc = SBH_OK;
  if (nq < kOrderMinQueries || workspace_bytes < sbh_traversal_ordered_workspace_bytes(nq)) return nullptr;
  Carver c(workspace, workspace_bytes);
  uint32_t *k0, *v0, *k1, *v1, *hist, *tmp;
  order_carve(c, nq, &k0, &v0, &k1, &v1, &hist, &tmp);
  o8_query_codes_kernel<<<grid_stride(nq, 256), 256, 0, stream>>>(nodes, queries, nq, k0);
  int which = 0;
  cudaError_t e = radix_sort<uint32_t>(stream, k0, v0, k1, v1, nq, 30, false, hist, tmp, &which);
  if (e != cudaSuccess) {
    *rc = fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    return nullptr;
  }
  return which == 0 ? v0 : v1;
}

// Whether the buffer is a dense octree8 of depth <= 9 ((8^(d+1) - 1) / 7
// nodes), whose DFS never holds more than 64 stack entries.
static bool o8_small_stack(uint32_t num_nodes) {
  uint64_t total = 1, level = 1;
  for (int d = 0; d <= 9; d++) {
    if (total == num_nodes) return true;
    level *= 8;
    total += level;
  }
  return false;
}

// With a periodic box the pairs take the scalar minimum-image form, which
// gains little from staged particles, so that kernel sums each leaf per lane
// straight from global memory and holds fewer registers (TreePM short range,
// 2^21 particles: 16.6 ms against 17.7 ms staged).
template <int KERNEL, int STACK>
static void o8_launch_warp_kind(unsigned grid, unsigned block, size_t smem, cudaStream_t stream, const Leaf3* L,
                                const OctreeNode8* N, const float* queries, const float* cot, int64_t nq, float beta,
                                Soft s, int prune_on, float r_cut_sq, Periodic per, float* out, uint32_t* status,
                                O8Bounds bd, const uint32_t* order) {
  if (per.on)
    o8_bh_warp_kernel<KERNEL, STACK, false><<<grid, block, smem, stream>>>(L, N, queries, cot, nq, beta, s, prune_on,
                                                                           r_cut_sq, per, out, status, bd, order);
  else
    o8_bh_warp_kernel<KERNEL, STACK, true><<<grid, block, smem, stream>>>(L, N, queries, cot, nq, beta, s, prune_on,
                                                                          r_cut_sq, per, out, status, bd, order);
}

template <int STACK>
static void o8_launch_warp(int kernel, unsigned grid, unsigned block, size_t smem, cudaStream_t stream,
                           const Leaf3* L, const OctreeNode8* N, const float* queries, const float* cot, int64_t nq,
                           float beta, Soft s, int prune_on, float r_cut_sq, Periodic per, float* out,
                           uint32_t* status, O8Bounds bd, const uint32_t* order) {
  switch (kernel) {
    case O8_GRAV_GRAD:
      o8_launch_warp_kind<O8_GRAV_GRAD, STACK>(grid, block, smem, stream, L, N, queries, cot, nq, beta, s, 0, 0.f, per,
                                               out, status, bd, order);
      break;
    case O8_SOFT:
      o8_launch_warp_kind<O8_SOFT, STACK>(grid, block, smem, stream, L, N, queries, cot, nq, beta, s, prune_on,
                                          r_cut_sq, per, out, status, bd, order);
      break;
    case O8_GRAV_GRAD_VJP:
      o8_launch_warp_kind<O8_GRAV_GRAD_VJP, STACK>(grid, block, smem, stream, L, N, queries, cot, nq, beta, s, 0, 0.f,
                                                   per, out, status, bd, order);
      break;
    default:
      o8_launch_warp_kind<O8_SOFT_VJP, STACK>(grid, block, smem, stream, L, N, queries, cot, nq, beta, s, prune_on,
                                              r_cut_sq, per, out, status, bd, order);
      break;
  }
}

extern "C" {

int sbh_bruteforce_gravity(cudaStream_t stream, const float* points, const float* masses, int64_t n, int dim,
                           const float* queries, int64_t nq, float* out, int periodic, float box_length,
                           int threads) {
  if (n < 0 || nq < 0) return invalid("sizes must be >= 0");
  if (dim != 2 && dim != 3) return invalid("only dim=2 or dim=3 supported");
  if (int rc = check_threads(threads)) return rc;
  if (nq == 0) return SBH_OK;
  bruteforce_gravity_kernel<<<grid_for(nq, kDirectThreads), kDirectThreads, 0, stream>>>(
      points, masses, n, dim, queries, nq, out, Periodic{periodic, box_length});
  return check_launch("bruteforce_gravity");
}

int sbh_direct_force_soft(cudaStream_t stream, const float* points, const float* masses, int64_t n,
                          const float* queries, int64_t nq, float* out, float softening_scale,
                          float cutoff_scale, int periodic, float box_length, int threads) {
  if (n < 0 || nq < 0) return invalid("sizes must be >= 0");
  if (softening_scale < 0.0f) return invalid("softening_scale must be >= 0");
  if (!(cutoff_scale > 0.0f)) return invalid("cutoff_scale must be > 0");
  if (int rc = check_threads(threads)) return rc;
  if (nq == 0) return SBH_OK;
  const bool per = periodic && box_length > 0.0f;
  const Soft soft{fmaxf(softening_scale, 0.0f), cutoff_scale};
  if (per)
    direct_soft_kernel<0, true><<<grid_for(nq, kDirectThreads), kDirectThreads, 0, stream>>>(
        points, masses, n, queries, nullptr, nq, out, soft, Periodic{periodic, box_length});
  else
    direct_soft2_kernel<false><<<grid_for(nq, 2 * kDirectThreads), kDirectThreads, 0, stream>>>(
        points, masses, n, queries, nullptr, nq, out, soft);
  return check_launch("direct_force_soft");
}

int sbh_direct_force_soft_vjp(cudaStream_t stream, const float* points, const float* masses, int64_t n,
                              const float* queries, int64_t nq, const float* cotangent, float* out,
                              float softening_scale, float cutoff_scale, int periodic, float box_length,
                              int threads) {
  if (n < 0 || nq < 0) return invalid("sizes must be >= 0");
  if (softening_scale < 0.0f) return invalid("softening_scale must be >= 0");
  if (!(cutoff_scale > 0.0f)) return invalid("cutoff_scale must be > 0");
  if (int rc = check_threads(threads)) return rc;
  if (nq == 0) return SBH_OK;
  const bool per = periodic && box_length > 0.0f;
  const Soft soft{fmaxf(softening_scale, 0.0f), cutoff_scale};
  if (per)
    direct_soft_kernel<1, true><<<grid_for(nq, kDirectThreads), kDirectThreads, 0, stream>>>(
        points, masses, n, queries, cotangent, nq, out, soft, Periodic{periodic, box_length});
  else
    direct_soft2_kernel<true><<<grid_for(nq, 2 * kDirectThreads), kDirectThreads, 0, stream>>>(
        points, masses, n, queries, cotangent, nq, out, soft);
  return check_launch("direct_force_soft_vjp");
}

size_t sbh_build_octree8_workspace_bytes(int64_t n, int max_depth) {
  if (max_depth < 1 || max_depth > 10 || n < 0) return 0;
  Sizer s;
  O8Params* prm;
  uint32_t *k0, *v0, *k1, *v1, *counts, *hist, *scan_tmp;
  DVec<7>*P, *ptmp;
  o8_carve(s, n, max_depth, &prm, &k0, &v0, &k1, &v1, &counts, &hist, &scan_tmp, &P, &ptmp);
  return s.off;
}

int sbh_build_octree8(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                      int64_t n, const float* min_corner, const float* max_corner, int max_depth, void* leaf_out,
                      size_t leaf_bytes, void* node_out, size_t node_bytes, void* contrib_out,
                      size_t contrib_bytes, void* workspace, size_t workspace_bytes) {
  if (max_depth < 1 || max_depth > 10) return invalid("max_depth must be in [1, 10]");
  if (n < 0 || n > 0xFFFFFFFFll) return invalid("number of points must be in [0, 2^32)");
  uint64_t total = sbh_octree8_total_nodes(max_depth);
  if (leaf_bytes != static_cast<size_t>(n) * sizeof(Leaf3)) return invalid("leaf_out size mismatch");
  if (node_bytes != total * sizeof(OctreeNode8)) return invalid("node_out size mismatch");
  if (contrib_bytes != total * sizeof(Leaf3)) return invalid("contrib_out size mismatch");
  if (!min_corner || !max_corner) return invalid("min_corner/max_corner must be non-null");
  if ((n > 0 && !aligned16(leaf_out)) || !aligned16(node_out) || !aligned16(contrib_out))
    return invalid("output buffers must be 16-byte aligned");
  size_t need = sbh_build_octree8_workspace_bytes(n, max_depth);
  if (!workspace || workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes);
  O8Params* prm;
  uint32_t *k0, *v0, *k1, *v1, *counts, *hist, *scan_tmp;
  DVec<7>*P, *ptmp;
  o8_carve(c, n, max_depth, &prm, &k0, &v0, &k1, &v1, &counts, &hist, &scan_tmp, &P, &ptmp);
  uint32_t* status = static_cast<uint32_t*>(workspace);
  uint64_t cells = 1ull << (3 * max_depth);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, (cells + 1) * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  o8_setup_kernel<<<1, 1, 0, stream>>>(min_corner, max_corner, prm, status);
  if (n > 0) {
    o8_codes_kernel<<<grid_stride(n, 256), 256, 0, stream>>>(points, n, prm, max_depth, k0, counts);
    int which = 0;
    e = radix_sort<uint32_t>(stream, k0, v0, k1, v1, n, 3 * max_depth, false, hist, scan_tmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    const uint32_t* perm = which == 0 ? v0 : v1;
    o8_gather_kernel<<<grid_stride(n, 256), 256, 0, stream>>>(points, normals, masses, n, perm, prm,
                                                              static_cast<Leaf3*>(leaf_out));
  }
  e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{counts}, static_cast<int64_t>(cells), counts, scan_tmp,
                               true);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  e = exclusive_scan<DVec<7>>(stream, LeafMomentLoad{static_cast<const Leaf3*>(leaf_out)}, n, P, ptmp, true);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  o8_nodes_kernel<<<grid_stride(static_cast<int64_t>(total), 256), 256, 0, stream>>>(
      static_cast<OctreeNode8*>(node_out), static_cast<Leaf3*>(contrib_out), counts, P, max_depth, total, prm);
  return check_launch("build_octree8");
}

// --------------------------- octree8 traversals -----------------------------
static int o8_launch_bh(int kernel, cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                        size_t node_bytes, const float* queries, int64_t nq, const float* cot, float* out,
                        float beta, Soft s, int prune_on, float r_cut_sq, Periodic per, int threads,
                        void* workspace, size_t workspace_bytes) {
  if (int rc = o8_layout_checks(leaf, leaf_bytes, nodes, node_bytes, queries, nq, 0)) return rc;
  if (int rc = check_threads(threads)) return rc;
  if (!workspace || workspace_bytes < kStatusBytes) return fail(SBH_ERR_WORKSPACE, "workspace too small");
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (nq == 0) return SBH_OK;
  const Leaf3* L = static_cast<const Leaf3*>(leaf);
  const OctreeNode8* N = static_cast<const OctreeNode8*>(nodes);
  O8Bounds bd{static_cast<uint32_t>(node_bytes / sizeof(OctreeNode8)), static_cast<uint32_t>(leaf_bytes / sizeof(Leaf3))};
  int orc = SBH_OK;
  const uint32_t* order = o8_query_order(stream, N, queries, nq, workspace, workspace_bytes, &orc);
  if (orc != SBH_OK) return orc;
  if (order) {  // Morton-ordered queries: one warp walks 32 neighbours together
    const int warps = threads >= 64 ? (threads < 1024 ? threads / 32 : 32) : 1;
    const unsigned tw = 32u * static_cast<unsigned>(warps);
    const unsigned gw = grid_for(nq, static_cast<int>(tw));
    if (o8_small_stack(bd.num_nodes)) {
      const size_t sm = o8_warp_smem(warps, 64);
      o8_launch_warp<64>(kernel, gw, tw, sm, stream, L, N, queries, cot, nq, beta, s, prune_on, r_cut_sq, per, out,
                         status, bd, order);
    } else {
      const size_t sm = o8_warp_smem(warps, kO8Stack);
      o8_launch_warp<kO8Stack>(kernel, gw, tw, sm, stream, L, N, queries, cot, nq, beta, s, prune_on, r_cut_sq, per,
                               out, status, bd, order);
    }
    return check_launch("barnes_hut_force_octree8");
  }
  unsigned g = grid_for(nq, 256);
  switch (kernel) {
    case O8_GRAV_GRAD:
      o8_bh_kernel<O8_GRAV_GRAD><<<g, 256, 0, stream>>>(L, N, queries, cot, nq, beta, s, 0, 0.f, per, out, status, bd,
                                                        order);
      break;
    case O8_SOFT:
      o8_bh_kernel<O8_SOFT><<<g, 256, 0, stream>>>(L, N, queries, cot, nq, beta, s, prune_on, r_cut_sq, per, out,
                                                   status, bd, order);
      break;
    case O8_GRAV_GRAD_VJP:
      o8_bh_kernel<O8_GRAV_GRAD_VJP><<<g, 256, 0, stream>>>(L, N, queries, cot, nq, beta, s, 0, 0.f, per, out, status,
                                                            bd, order);
      break;
    default:
      o8_bh_kernel<O8_SOFT_VJP><<<g, 256, 0, stream>>>(L, N, queries, cot, nq, beta, s, prune_on, r_cut_sq, per,
                                                       out, status, bd, order);
      break;
  }
  return check_launch("barnes_hut_force_octree8");
}

// prune_on / r_cut exactly as the reference handler derives them (src/sbh_ffi.cu:3235-3237).
static void o8_prune_params(int prune_enabled, float prune_r_cut_mult, float cutoff_scale, int* on, float* rsq) {
  *on = (prune_enabled != 0 && cutoff_scale > 0.0f) ? 1 : 0;
  float r_cut = *on ? prune_r_cut_mult * cutoff_scale : 0.0f;
  *rsq = r_cut * r_cut;
}

int sbh_barnes_hut_force_octree8(cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                                 size_t node_bytes, const float* queries, int64_t nq, float* out, float beta,
                                 int periodic, float box_length, int threads, void* workspace,
                                 size_t workspace_bytes) {
  return o8_launch_bh(O8_GRAV_GRAD, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, nullptr, out, beta,
                      Soft{0.f, 0.f}, 0, 0.f, Periodic{periodic, box_length}, threads, workspace, workspace_bytes);
}

int sbh_barnes_hut_force_octree8_vjp(cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                                     size_t node_bytes, const float* queries, int64_t nq, const float* cotangent,
                                     float* out, float beta, int periodic, float box_length, int threads,
                                     void* workspace, size_t workspace_bytes) {
  if (nq > 0 && !cotangent) return invalid("cotangent must be non-null");
  return o8_launch_bh(O8_GRAV_GRAD_VJP, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, cotangent, out, beta,
                      Soft{0.f, 0.f}, 0, 0.f, Periodic{periodic, box_length}, threads, workspace, workspace_bytes);
}

int sbh_barnes_hut_force_octree8_soft(cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                                      size_t node_bytes, const float* queries, int64_t nq, float* out, float beta,
                                      float softening_scale, float cutoff_scale, int prune_enabled,
                                      float prune_r_cut_mult, int periodic, float box_length, int threads,
                                      void* workspace, size_t workspace_bytes) {
  if (prune_enabled != 0 && prune_r_cut_mult <= 0.0f)
    return invalid("prune_r_cut_mult must be > 0 when prune_enabled is set");
  int on;
  float rsq;
  o8_prune_params(prune_enabled, prune_r_cut_mult, cutoff_scale, &on, &rsq);
  return o8_launch_bh(O8_SOFT, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, nullptr, out, beta,
                      Soft{fmaxf(softening_scale, 0.0f), cutoff_scale}, on, rsq, Periodic{periodic, box_length},
                      threads, workspace, workspace_bytes);
}

int sbh_barnes_hut_force_octree8_soft_vjp(cudaStream_t stream, const void* leaf, size_t leaf_bytes,
                                          const void* nodes, size_t node_bytes, const float* queries, int64_t nq,
                                          const float* cotangent, float* out, float beta, float softening_scale,
                                          float cutoff_scale, int prune_enabled, float prune_r_cut_mult,
                                          int periodic, float box_length, int threads, void* workspace,
                                          size_t workspace_bytes) {
  if (prune_enabled != 0 && prune_r_cut_mult <= 0.0f)
    return invalid("prune_r_cut_mult must be > 0 when prune_enabled is set");
  if (nq > 0 && !cotangent) return invalid("cotangent must be non-null");
  int on;
  float rsq;
  o8_prune_params(prune_enabled, prune_r_cut_mult, cutoff_scale, &on, &rsq);
  return o8_launch_bh(O8_SOFT_VJP, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, cotangent, out, beta,
                      Soft{fmaxf(softening_scale, 0.0f), cutoff_scale}, on, rsq, Periodic{periodic, box_length},
                      threads, workspace, workspace_bytes);
}

static int o8_launch_stochastic(bool vjp, int softened, cudaStream_t stream, const void* leaf, size_t leaf_bytes,
                                const void* nodes, size_t node_bytes, const float* queries, int64_t nq,
                                const float* cot, float* out, int samples, int seed, float beta,
                                float softening_scale, float cutoff_scale, int prune_enabled,
                                float prune_r_cut_mult, int periodic, float box_length, int threads,
                                void* workspace, size_t workspace_bytes) {
  if (int rc = o8_layout_checks(leaf, leaf_bytes, nodes, node_bytes, queries, nq, 0)) return rc;
  if (int rc = check_threads(threads)) return rc;
  if (softened && prune_enabled != 0 && prune_r_cut_mult <= 0.0f)
    return invalid("prune_r_cut_mult must be > 0 when prune_enabled is set");
  if (vjp && nq > 0 && !cot) return invalid("cotangent must be non-null");
  if (!workspace || workspace_bytes < kStatusBytes) return fail(SBH_ERR_WORKSPACE, "workspace too small");
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (nq == 0) return SBH_OK;
  int on = 0;
  float rsq = 0.f;
  if (softened) o8_prune_params(prune_enabled, prune_r_cut_mult, cutoff_scale, &on, &rsq);
  Soft s{fmaxf(softening_scale, 0.0f), cutoff_scale};
  Periodic per{periodic, box_length};
  const Leaf3* L = static_cast<const Leaf3*>(leaf);
  const OctreeNode8* N = static_cast<const OctreeNode8*>(nodes);
  O8Bounds bd{static_cast<uint32_t>(node_bytes / sizeof(OctreeNode8)), static_cast<uint32_t>(leaf_bytes / sizeof(Leaf3))};
  // The reference's kernel reads a curand state per query, independent of
  // the block size and of which thread takes the query, so any launch shape
  // and query order give the same numbers.
  int orc = SBH_OK;
  const uint32_t* order = o8_query_order(stream, N, queries, nq, workspace, workspace_bytes, &orc);
  if (orc != SBH_OK) return orc;
  unsigned g = grid_for(nq, 128);
  if (!vjp) {
    if (softened)
      o8_stochastic_kernel<O8_SOFT, true><<<g, 128, 0, stream>>>(L, N, queries, cot, nq, samples, seed, beta, s, on,
                                                                 rsq, per, out, status, bd, order);
    else
      o8_stochastic_kernel<O8_GRAV_GRAD, false><<<g, 128, 0, stream>>>(L, N, queries, cot, nq, samples, seed, beta,
                                                                       s, 0, 0.f, per, out, status, bd, order);
  } else {
    if (softened)
      o8_stochastic_kernel<O8_SOFT_VJP, true><<<g, 128, 0, stream>>>(L, N, queries, cot, nq, samples, seed, beta, s,
                                                                     on, rsq, per, out, status, bd, order);
    else
      o8_stochastic_kernel<O8_GRAV_GRAD_VJP, false><<<g, 128, 0, stream>>>(L, N, queries, cot, nq, samples, seed,
                                                                           beta, s, 0, 0.f, per, out, status, bd,
                                                                           order);
  }
  return check_launch("stochastic_bh_force_octree8");
}

size_t sbh_traversal_ordered_workspace_bytes(int64_t nq) {
  if (nq < 0) return 0;
  Sizer z;
  uint32_t *k0, *v0, *k1, *v1, *hist, *tmp;
  order_carve(z, nq, &k0, &v0, &k1, &v1, &hist, &tmp);
  return z.off;
}

int sbh_stochastic_bh_force_octree8(cudaStream_t stream, int softened, const void* leaf, size_t leaf_bytes,
                                    const void* nodes, size_t node_bytes, const float* queries, int64_t nq,
                                    float* out, int samples_per_subdomain, int seed, float beta,
                                    float softening_scale, float cutoff_scale, int prune_enabled,
                                    float prune_r_cut_mult, int periodic, float box_length, int threads,
                                    void* workspace, size_t workspace_bytes) {
  return o8_launch_stochastic(false, softened, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, nullptr,
                              out, samples_per_subdomain, seed, beta, softening_scale, cutoff_scale, prune_enabled,
                              prune_r_cut_mult, periodic, box_length, threads, workspace, workspace_bytes);
}

int sbh_stochastic_bh_force_octree8_vjp(cudaStream_t stream, int softened, const void* leaf, size_t leaf_bytes,
                                        const void* nodes, size_t node_bytes, const float* queries, int64_t nq,
                                        const float* cotangent, float* out, int samples_per_subdomain, int seed,
                                        float beta, float softening_scale, float cutoff_scale, int prune_enabled,
                                        float prune_r_cut_mult, int periodic, float box_length, int threads,
                                        void* workspace, size_t workspace_bytes) {
  return o8_launch_stochastic(true, softened, stream, leaf, leaf_bytes, nodes, node_bytes, queries, nq, cotangent,
                              out, samples_per_subdomain, seed, beta, softening_scale, cutoff_scale, prune_enabled,
                              prune_r_cut_mult, periodic, box_length, threads, workspace, workspace_bytes);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// octree8 build with library-owned scratch (no allocation by the caller or
// by the library at call time)
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory when they need a tree: an XLA
// custom call running under JAX's default preallocation (the framework holds
// most of the GPU, so a cudaMalloc from inside the handler can fail), code
// that runs with a fixed, pre-reserved memory budget, or a caller that must
// not trigger the implicit device synchronisation a cudaMalloc may cause.
// For them this variant of sbh_build_octree8 takes its temporaries from one
// fixed array that is part of the library image. Every GPU that loads the
// library holds these bytes until the process exits. The build clears what
// must start at zero (status word, cell counters) on every call, so what an
// earlier call left in the array does not matter. Calls that may overlap on
// the GPU (two streams, or two host threads) share the array and race: the
// caller serialises them.
namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB
__device__ __align__(256) unsigned char g_o8_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_addr[128] = {};  // device address of the array, per device ordinal

// Device address of the scratch on the current device. On the host the
// array's name only stands for the device symbol; the address a kernel can
// use comes from cudaGetSymbolAddress with that device current.
int static_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) return fail(SBH_ERR_CUDA, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_o8_static_scratch);
    if (e != cudaSuccess || !p) return fail(SBH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_static_addr[dev] = p;
  }
  *out = g_static_addr[dev];
  return SBH_OK;
}

}  // namespace

extern "C" {

size_t sbh_build_octree8_static_scratch_bytes(void) { return kStaticScratchBytes; }

int sbh_build_octree8_static(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                             int64_t n, const float* min_corner, const float* max_corner, int max_depth,
                             void* leaf_out, size_t leaf_bytes, void* node_out, size_t node_bytes, void* contrib_out,
                             size_t contrib_bytes) {
  if (max_depth < 1 || max_depth > 10) return invalid("max_depth must be in [1, 10]");
  if (n < 0) return invalid("number of points must be >= 0");
  size_t need = sbh_build_octree8_workspace_bytes(n, max_depth);
  if (need > kStaticScratchBytes)
    return invalid("n = " + std::to_string(n) + " at max_depth = " + std::to_string(max_depth) + " needs " +
                   std::to_string(need) + " bytes of scratch; the built-in scratch holds " +
                   std::to_string(kStaticScratchBytes) + " (use sbh_build_octree8 with a workspace)");
  void* ws = nullptr;
  if (int rc = static_scratch(&ws)) return rc;
  return sbh_build_octree8(stream, points, normals, masses, n, min_corner, max_corner, max_depth, leaf_out, leaf_bytes,
                           node_out, node_bytes, contrib_out, contrib_bytes, ws, kStaticScratchBytes);
}

}  // extern "C"
