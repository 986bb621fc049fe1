// Level-3 tree build (Tree3DNode<1,3> layout) and the classic and stochastic
// traversals of general Tree2DNode<1,3> / Tree3DNode<1,3> buffers (the
// reference's Node2/Node3 FFI targets, src/sbh_ffi.cu:192-397, 1422-1680,
// 2444-3131; include/barnes_hut_gpu.h, include/tree_sampler_gpu.h).
//
// Compiled with --use_fast_math like the reference, so quantisation,
// opening ratios and the sample-index arithmetic round the same way. The
// traversals follow the reference's navigation exactly (bitmask order,
// sibling step by re-quantising the child's midpoint, the single-child skip
// of containedInChild) so sums are accumulated in the same order.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdint>
#include <string>

#include "sbh_common.cuh"
#include "sbh_primitives.cuh"

namespace sbh {
namespace tr {

// ---------------------------------------------------------------------------
// level-3 build (src/sbh_ffi.cu:736-1037)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int quantize_level3(float x, float lo, float hi) {
  float span = hi - lo;
  if (span <= 1e-12f) return 0;
  float t = (x - lo) / span;
  t = fminf(fmaxf(t, 0.0f), 0.999999f);
  return static_cast<int>(t * static_cast<float>(kLevel3Split));
}

__global__ void l3_bins_kernel(const float* __restrict__ pts, int64_t n, const float* __restrict__ mn,
                               const float* __restrict__ mx, uint32_t* __restrict__ bins, uint32_t* __restrict__ counts) {
  float lo0 = mn[0], lo1 = mn[1], lo2 = mn[2], hi0 = mx[0], hi1 = mx[1], hi2 = mx[2];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int qx = quantize_level3(pts[3 * i], lo0, hi0);
    int qy = quantize_level3(pts[3 * i + 1], lo1, hi1);
    int qz = quantize_level3(pts[3 * i + 2], lo2, hi2);
    uint32_t bin = static_cast<uint32_t>(qx + kLevel3Split * (qy + kLevel3Split * qz));
    bins[i] = bin;
    atomicAdd(&counts[bin], 1u);
  }
}

__global__ void l3_gather_kernel(const float* __restrict__ pts, const float* __restrict__ nrm,
                                 const float* __restrict__ masses, int64_t n, const uint32_t* __restrict__ perm,
                                 Leaf3* __restrict__ leaf) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t s = perm[i];
    float4* dst = reinterpret_cast<float4*>(leaf + i);
    dst[0] = make_float4(pts[3 * s], pts[3 * s + 1], pts[3 * s + 2], nrm ? nrm[3 * s] : 0.f);
    dst[1] = make_float4(nrm ? nrm[3 * s + 1] : 0.f, nrm ? nrm[3 * s + 2] : 0.f, masses[s], 1.0f);
  }
}

struct L3MomentLoad {
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

struct PresentLoad {
  const uint32_t* off;
  __device__ uint32_t operator()(int64_t b) const { return off[b + 1] > off[b] ? 1u : 0u; }
};

__device__ void set_contrib(Leaf3& c, const DVec<7>& hi, const DVec<7>& lo) {
  double M = hi.v[0] - lo.v[0];
  float mass = static_cast<float>(M);
  c.alpha = 1.0f;
  c.mass = mass;
  for (int d = 0; d < 3; d++) {
    c.pos[d] = mass > 0.0f ? static_cast<float>((hi.v[1 + d] - lo.v[1 + d]) / M) : 0.0f;
    c.nrm[d] = mass > 0.0f ? static_cast<float>((hi.v[4 + d] - lo.v[4 + d]) / M) : 0.0f;
  }
}

// One block: root (thread 0) and the non-empty children (one thread per bin).
__global__ void l3_nodes_kernel(Node3* __restrict__ nodes, Leaf3* __restrict__ contrib, int64_t n,
                                const float* __restrict__ mn, const float* __restrict__ mx,
                                const uint32_t* __restrict__ off, const uint32_t* __restrict__ rank,
                                const DVec<7>* __restrict__ P) {
  __shared__ unsigned long long mask[8];
  __shared__ int nchild;
  if (threadIdx.x < 8) mask[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) nchild = 0;
  __syncthreads();
  float min_x = mn[0], min_y = mn[1], min_z = mn[2];
  float max_x = mx[0], max_y = mx[1], max_z = mx[2];
  for (int bin = threadIdx.x; bin < kLevel3Bins; bin += blockDim.x) {
    uint32_t s = off[bin], e = off[bin + 1];
    if (e <= s) continue;
    atomicOr(&mask[bin >> 6], 1ull << (bin & 63));
    atomicAdd(&nchild, 1);
    int child_idx = 1 + static_cast<int>(rank[bin]);
    int qx = bin & 7, qy = (bin >> 3) & 7, qz = (bin >> 6) & 7;
    float dx = (max_x - min_x) / static_cast<float>(kLevel3Split);
    float dy = (max_y - min_y) / static_cast<float>(kLevel3Split);
    float dz = (max_z - min_z) / static_cast<float>(kLevel3Split);
    Node3& c = nodes[child_idx];
    c.start = s;
    c.end = e;
    c.buffer_idx = static_cast<uint64_t>(child_idx);
    c.parent_idx = 0;
    c.bmin[0] = fmaf(dx, static_cast<float>(qx), min_x);
    c.bmin[1] = fmaf(dy, static_cast<float>(qy), min_y);
    c.bmin[2] = fmaf(dz, static_cast<float>(qz), min_z);
    c.bmax[0] = c.bmin[0] + dx;
    c.bmax[1] = c.bmin[1] + dy;
    c.bmax[2] = c.bmin[2] + dz;
    c.diameter = sqrtf(dx * dx + dy * dy + dz * dz);
    Leaf3 ct;
    set_contrib(ct, P[e], P[s]);
    c.contrib = ct;
    c.num_children = 0;
    c.depth = 1;
    c.max_depth = 1;
    c.is_leaf = true;
    contrib[child_idx] = ct;
    // mask and child_idx stay zero (the buffer is cleared first)
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Node3& r = nodes[0];
    r.start = 0;
    r.end = static_cast<uint64_t>(n);
    r.buffer_idx = 0;
    r.parent_idx = 0;
    r.bmin[0] = min_x;
    r.bmin[1] = min_y;
    r.bmin[2] = min_z;
    r.bmax[0] = max_x;
    r.bmax[1] = max_y;
    r.bmax[2] = max_z;
    float dx = max_x - min_x, dy = max_y - min_y, dz = max_z - min_z;
    r.diameter = sqrtf(dx * dx + dy * dy + dz * dz);
    Leaf3 ct;
    set_contrib(ct, P[n], P[0]);
    r.contrib = ct;
    for (int w = 0; w < 8; w++) r.mask[w] = mask[w];
    r.num_children = nchild;
    r.depth = 0;
    r.max_depth = 1;
    r.is_leaf = n <= 1;
    contrib[0] = ct;
  }
  __syncthreads();
  for (int bin = threadIdx.x; bin < kLevel3Bins; bin += blockDim.x) {
    uint32_t s = off[bin], e = off[bin + 1];
    nodes[0].child_idx[bin] = e > s ? static_cast<uint64_t>(1 + rank[bin]) : 0ull;
  }
}

// ---------------------------------------------------------------------------
// general tree navigation (include/tree3d.h:134-206, tree2d.h, aabb.h)
// ---------------------------------------------------------------------------
template <int N>
struct Vec {
  float v[N];
};

template <int N>
using NodeT = typename std::conditional<N == 3, Node3, Node2>::type;
template <int N>
using LeafT = typename std::conditional<N == 3, Leaf3, Leaf2>::type;

template <int N>
struct TreeCfg {
  static constexpr int kSplit = 8;
  static constexpr int kBranch = N == 3 ? 512 : 64;
  static constexpr int kWords = N == 3 ? 8 : 1;
};

template <int N>
__device__ __forceinline__ Vec<N> leaf_pos(const LeafT<N>& l) {
  Vec<N> r;
  for (int d = 0; d < N; d++) r.v[d] = l.pos[d];
  return r;
}

template <int N>
__device__ __forceinline__ bool contains(const NodeT<N>& nd, const Vec<N>& p) {
  for (int d = 0; d < N; d++)
    if (!((nd.bmin[d] - 1e-4f) <= p.v[d] && p.v[d] <= (nd.bmax[d] + 1e-4f))) return false;
  return true;
}

// AABB::quantize (include/aabb.h:33-41): int(split * (p - min) / (max - min)) clamped
template <int N>
__device__ __forceinline__ int coords_index(const NodeT<N>& nd, const Vec<N>& p) {
  int q[N];
  for (int d = 0; d < N; d++) {
    float t = static_cast<float>(TreeCfg<N>::kSplit) * (p.v[d] - nd.bmin[d]) / (nd.bmax[d] - nd.bmin[d]);
    int c = static_cast<int>(t);
    c = c < TreeCfg<N>::kSplit - 1 ? c : TreeCfg<N>::kSplit - 1;
    c = c > 0 ? c : 0;
    q[d] = c;
  }
  if (N == 3) return (((q[2] << 3) + q[1]) << 3) + q[0];
  return (q[1] << 3) + q[0];
}

template <int N>
__device__ __forceinline__ int first_bit(const NodeT<N>& nd) {
  for (int w = 0; w < TreeCfg<N>::kWords; w++)
    if (nd.mask[w]) return (w << 6) + __ffsll(static_cast<long long>(nd.mask[w])) - 1;
  return TreeCfg<N>::kBranch;
}

template <int N>
__device__ __forceinline__ int next_bit(const NodeT<N>& nd, int last) {
  int next = last + 1;
  if (next >= TreeCfg<N>::kBranch) return TreeCfg<N>::kBranch;
  int w = next >> 6, bit = next & 63;
  uint64_t b = nd.mask[w];
  if (b & (1ull << bit)) return next;
  b &= ~0ull << bit;
  while (!b && w + 1 < TreeCfg<N>::kWords) b = nd.mask[++w];
  return b ? (w << 6) + __ffsll(static_cast<long long>(b)) - 1 : TreeCfg<N>::kBranch;
}

struct Bounds {
  uint64_t num_nodes;
  uint64_t num_leaves;
};

// -1 when the index is out of the buffer (recorded in the status word).
__device__ __forceinline__ int64_t checked(uint64_t idx, uint64_t count, uint32_t* status) {
  if (idx < count) return static_cast<int64_t>(idx);
  raise_status(status, SBH_DEV_BAD_BOUNDS);
  return -1;
}

template <int N>
__device__ __forceinline__ int64_t next_child(const NodeT<N>* nodes, const NodeT<N>& parent, const NodeT<N>& child,
                                              const Bounds& bd, uint32_t* status) {
  Vec<N> mid;
  for (int d = 0; d < N; d++) mid.v[d] = (child.bmin[d] + child.bmax[d]) / 2;
  if (!contains<N>(parent, mid)) return -1;
  int nb = next_bit<N>(parent, coords_index<N>(parent, mid));
  if (nb >= TreeCfg<N>::kBranch) return -1;
  return checked(parent.child_idx[nb], bd.num_nodes, status);
}

// containedInChild(p) (include/tree3d.h:171-181): descends through single-child nodes.
template <int N>
__device__ int64_t contained_in_child(const NodeT<N>* nodes, int64_t idx, const Vec<N>& p, const Bounds& bd,
                                      uint32_t* status) {
  for (int guard = 0; guard < 64; guard++) {
    const NodeT<N>& nd = nodes[idx];
    if (!contains<N>(nd, p)) return -1;
    int64_t c = checked(nd.child_idx[coords_index<N>(nd, p)], bd.num_nodes, status);
    if (c < 0) return -1;
    if (nodes[c].num_children == 1) {
      idx = c;
      continue;
    }
    return c;
  }
  raise_status(status, SBH_DEV_ITER_LIMIT);
  return -1;
}

// ---------------------------------------------------------------------------
// kernels of include/kernel.h on a leaf record: scalar (potential, winding
// number: v[0]) or vector (v[0..N-1]). The two VJP kinds are the query-side
// vector-Jacobian products of the force kernels with the cotangent g
// (gravityGradVjp and gravityGradSoftCutoffVjp, src/sbh_ffi.cu:2044-2090,
// written for N = 2 and 3).
// ---------------------------------------------------------------------------
enum TreeKernel {
  TK_POTENTIAL = 0,
  TK_GRAVITY_GRAD = 1,
  TK_SOFT = 2,
  TK_WINDING = 3,
  TK_GRAVITY_GRAD_VJP = 4,
  TK_SOFT_VJP = 5,
  TK_SMOOTHDIST = 6  // smoothDistExp (include/kernel.h:82-87): exp(-alpha |p - q|)
};

constexpr bool is_vjp(int K) { return K == TK_GRAVITY_GRAD_VJP || K == TK_SOFT_VJP; }

template <int N, int K>
__device__ __forceinline__ void tree_kernel(const LeafT<N>& d, const Vec<N>& q, const Vec<N>& g, const Soft& s,
                                            const Periodic& per, float* acc) {
  float r[N];
  if (K == TK_POTENTIAL || K == TK_WINDING || K == TK_SMOOTHDIST) {
    for (int k = 0; k < N; k++) r[k] = min_image_floor(d.pos[k] - q.v[k], per);
  } else {
    for (int k = 0; k < N; k++) r[k] = min_image_floor(q.v[k] - d.pos[k], per);
  }
  float r2 = 0.f;
  for (int k = 0; k < N; k++) r2 += r[k] * r[k];
  if (K == TK_POTENTIAL) {
    acc[0] += -d.mass / (sqrtf(r2) + 1e-1f);
  } else if (K == TK_SMOOTHDIST) {
    acc[0] += expf(-d.alpha * sqrtf(r2));
  } else if (K == TK_WINDING) {
    float nd = 0.f;
    for (int k = 0; k < N; k++) nd += d.nrm[k] * r[k];
    if (N == 3) {
      float dist = sqrtf(r2);
      acc[0] += d.mass * nd / (4 * 3.14159265358979323846f * (dist * dist * dist + 1e-5f));
    } else {
      acc[0] += d.mass * nd / (2 * 3.14159265358979323846f * (r2 + 1e-5f));
    }
  } else if (K == TK_GRAVITY_GRAD) {
    float c = grav_grad_coeff(r2, d.mass);
    for (int k = 0; k < N; k++) acc[k] += c * r[k];
  } else if (K == TK_SOFT) {
    float c = soft_coeff(r2, d.mass, s);
    for (int k = 0; k < N; k++) acc[k] += c * r[k];
  } else if (K == TK_GRAVITY_GRAD_VJP) {
    // f = -m r / (|r| + 0.1)^3:  J^T g = -m (g / den^3 - 3 (r.g) / (|r| den^4) r)
    float dist = sqrtf(r2 + 1e-12f);
    float den = dist + 1e-1f;
    float id3 = 1.0f / (den * den * den);
    float id4 = id3 / den;
    float rg = 0.f;
    for (int k = 0; k < N; k++) rg += r[k] * g.v[k];
    float kr = 3.0f * rg * (1.0f / (dist + 1e-12f)) * id4;
    for (int k = 0; k < N; k++) acc[k] += -d.mass * (id3 * g.v[k] - kr * r[k]);
  } else {
    // f = -m att(r) (r^2 + eps^2)^-3/2 r:  J^T g = -m (att ir^3 g - (r.g)(3 att ir^5 + cc) r)
    float ir = rsqrtf(r2 + s.eps * s.eps + 1e-12f);
    float ir3 = ir * ir * ir;
    float ir5 = ir3 * ir * ir;
    float att = 1.0f, cc = 0.0f;
    if (s.cutoff > 0.0f && r2 + 1e-12f >= s.unity_r2) {
      float dist = sqrtf(r2 + 1e-12f);
      float u = dist / (2.0f * s.cutoff);
      float e = 1.0f;  // att = 1, e^{-u^2} = 1 to FP32 precision below kAttUnityU
      if (u >= kAttUnityU) {
        e = expf(-(u * u));
        att = erfcf(u) + (2.0f / 1.772453850905516f) * u * e;
      }
      cc = ir3 * dist * e / (2.0f * 1.772453850905516f * s.cutoff * s.cutoff * s.cutoff);
    }
    float rg = 0.f;
    for (int k = 0; k < N; k++) rg += r[k] * g.v[k];
    float rad = rg * (3.0f * att * ir5 + cc);
    for (int k = 0; k < N; k++) acc[k] += -d.mass * (att * ir3 * g.v[k] - rad * r[k]);
  }
}

template <int N>
__device__ __forceinline__ float far_ratio(const NodeT<N>& nd, const Vec<N>& q) {
  if (nd.is_leaf) return INFINITY;
  float d2 = 0.f;
  for (int k = 0; k < N; k++) {
    float t = q.v[k] - nd.contrib.pos[k];
    d2 += t * t;
  }
  return sqrtf(d2) / nd.diameter;
}

constexpr int kOut(int N, int K) { return (K == TK_POTENTIAL || K == TK_WINDING || K == TK_SMOOTHDIST) ? 1 : N; }

// evaluateBarnesHutGPUVote (include/barnes_hut_gpu.h:19-72).
template <int N, int K>
__global__ void vote_kernel(const LeafT<N>* __restrict__ leaf, const NodeT<N>* __restrict__ nodes,
                            const float* __restrict__ queries, const float* __restrict__ cot, int64_t nq, float beta,
                            Soft s, Periodic per, float* __restrict__ out, Bounds bd, uint32_t* status) {
  int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool active = qi < nq;
  // The lanes that exist in this warp (a block size that is not a multiple
  // of 32 leaves a partial last warp). Lanes past the end keep running with
  // the first query and always vote "far", so the vote is over the active
  // lanes, as in the reference whose extra threads have returned.
  unsigned lanes = __activemask();
  unsigned warp_active = __ballot_sync(lanes, active);
  if (warp_active == 0) return;
  Vec<N> q, g;
  int64_t qq = active ? qi : 0;
  for (int k = 0; k < N; k++) q.v[k] = queries[N * qq + k];
  for (int k = 0; k < N; k++) g.v[k] = is_vjp(K) ? cot[N * qq + k] : 0.0f;
  constexpr int NO = kOut(N, K);
  float acc[NO];
  for (int k = 0; k < NO; k++) acc[k] = 0.f;
  int64_t node = 0;
  int state = 1;  // 0 FromChild, 1 FromParent, 2 FromSibling
  int guard = 0;
  const int64_t max_steps = 4 * static_cast<int64_t>(bd.num_nodes) + 16;
  while (true) {
    if (++guard > max_steps) {
      raise_status(status, SBH_DEV_ITER_LIMIT);
      break;
    }
    const NodeT<N>& nd = nodes[node];
    if (state != 0) {
      bool far = !active || nd.is_leaf || far_ratio<N>(nd, q) >= beta;
      if (__all_sync(lanes, far)) {
        if (nd.is_leaf) {
          uint64_t e = nd.end <= bd.num_leaves ? nd.end : bd.num_leaves;
          if (nd.end > bd.num_leaves) raise_status(status, SBH_DEV_BAD_BOUNDS);
          for (uint64_t i = nd.start; i < e; i++) tree_kernel<N, K>(leaf[i], q, g, s, per, acc);
        } else {
          tree_kernel<N, K>(nd.contrib, q, g, s, per, acc);
        }
      } else {
        int fb = first_bit<N>(nd);
        if (fb < TreeCfg<N>::kBranch) {
          int64_t c = checked(nd.child_idx[fb], bd.num_nodes, status);
          if (c >= 0) {
            node = c;
            state = 1;
            continue;
          }
        }
      }
    }
    if (node == 0) break;
    int64_t parent = checked(nd.parent_idx, bd.num_nodes, status);
    if (parent < 0) break;
    int64_t nx = next_child<N>(nodes, nodes[parent], nd, bd, status);
    if (nx < 0) {
      node = parent;
      state = 0;
    } else {
      node = nx;
      state = 2;
    }
  }
  if (active)
    for (int k = 0; k < NO; k++) out[NO * qi + k] = acc[k];
}

// multiLevelPrefixControlVariateSampleGPUQuery (include/tree_sampler_gpu.h:25-140).
template <int N, int K>
// With a VJP kind the sampled paths and their weights are those of the
// forward estimate for the same seed and only the kernel evaluations are
// differentiated, as the reference's stochastic VJP does
// (src/sbh_ffi.cu:2293-2442); the result is an unbiased estimate of the
// exact sum's query-side VJP.
__global__ void mlpcv_kernel(const LeafT<N>* __restrict__ leaf, const NodeT<N>* __restrict__ nodes,
                             const LeafT<N>* __restrict__ contrib, const float* __restrict__ queries,
                             const float* __restrict__ cot, int64_t nq, int samples, int seed, int seed_stride,
                             Soft s, Periodic per, float* __restrict__ out, Bounds bd, uint64_t num_contrib,
                             uint32_t* status) {
  int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  Vec<N> q, g;
  for (int k = 0; k < N; k++) q.v[k] = queries[N * qi + k];
  for (int k = 0; k < N; k++) g.v[k] = is_vjp(K) ? cot[N * qi + k] : 0.0f;
  constexpr int NO = kOut(N, K);
  curandState st, st2;
  // the FFI handlers seed each query with seed + q (src/sbh_ffi.cu:1553-1680);
  // the pybind module passes 0 to every query (src/sbh_gpu.cu:143-208)
  int sq = seed + seed_stride * static_cast<int>(qi);
  curand_init(static_cast<unsigned long long>(static_cast<long long>(sq)), 0, 0, &st);
  curand_init(static_cast<unsigned long long>(blockIdx.x), 0, 0, &st2);
  float bh[NO], mlcv[NO];
  for (int k = 0; k < NO; k++) bh[k] = mlcv[k] = 0.f;
  const NodeT<N>& root = nodes[0];
  for (int it = first_bit<N>(root); it < TreeCfg<N>::kBranch; it = next_bit<N>(root, it)) {
    int64_t si = checked(root.child_idx[it], bd.num_nodes, status);
    if (si < 0) continue;
    const NodeT<N>& sub = nodes[si];
    if (sub.is_leaf) {
      for (uint64_t i = sub.start; i < sub.end && i < bd.num_leaves; i++) tree_kernel<N, K>(leaf[i], q, g, s, per, bh);
    } else {
      tree_kernel<N, K>(sub.contrib, q, g, s, per, bh);
    }
    uint64_t num_el = sub.end - sub.start;
    float sub_total[NO];
    for (int k = 0; k < NO; k++) sub_total[k] = 0.f;
    for (int ss = 0; ss < samples; ss++) {
      uint64_t pick = static_cast<uint64_t>(static_cast<float>(num_el) * curand_uniform(&st2) +
                                            static_cast<float>(sub.start));
      uint64_t last = sub.end - 1;
      pick = pick < last ? pick : last;
      if (pick >= bd.num_leaves) {
        raise_status(status, SBH_DEV_BAD_BOUNDS);
        continue;
      }
      float sample_prob_inv = static_cast<float>(num_el);
      Vec<N> sp = leaf_pos<N>(leaf[pick]);
      int64_t prev = si, cur = si;
      float event_prob = 1.0f;
      float wd[NO];
      for (int k = 0; k < NO; k++) wd[k] = 0.f;
      float cur_beta = fmaxf(1.0f, far_ratio<N>(nodes[cur], q));
      int guard = 0;
      while (!nodes[cur].is_leaf) {
        if (++guard > 64) {
          raise_status(status, SBH_DEV_ITER_LIMIT);
          break;
        }
        float ffr = far_ratio<N>(nodes[cur], q);
        float tp = fminf(cur_beta / ffr, 1.0f);
        float p = curand_uniform(&st);
        if (p > tp) {
          event_prob *= 1.0f - tp;
          break;
        }
        event_prob *= tp;
        prev = cur;
        int64_t nxt = contained_in_child<N>(nodes, cur, sp, bd, status);
        if (nxt < 0) break;
        cur = nxt;
        cur_beta = fmaxf(cur_beta, ffr);
        const NodeT<N>& pv = nodes[prev];
        float prev_res[NO], cur_res[NO];
        for (int k = 0; k < NO; k++) prev_res[k] = cur_res[k] = 0.f;
        tree_kernel<N, K>(pv.contrib, q, g, s, per, prev_res);
        int fb = first_bit<N>(pv);
        int64_t first = fb < TreeCfg<N>::kBranch ? static_cast<int64_t>(pv.child_idx[fb]) : 0;
        for (int off = 0; off < pv.num_children; off++) {
          int64_t ci = first + off;
          if (ci >= static_cast<int64_t>(bd.num_nodes)) {
            raise_status(status, SBH_DEV_BAD_BOUNDS);
            break;
          }
          const NodeT<N>& ch = nodes[ci];
          if (ch.is_leaf) {
            for (uint64_t i = ch.start; i < ch.end && i < bd.num_leaves; i++)
              tree_kernel<N, K>(leaf[i], q, g, s, per, cur_res);
          } else if (static_cast<uint64_t>(ci) < num_contrib) {
            tree_kernel<N, K>(contrib[ci], q, g, s, per, cur_res);
          }
        }
        float wgt = sample_prob_inv / (event_prob * static_cast<float>(pv.end - pv.start));
        for (int k = 0; k < NO; k++) wd[k] += wgt * (cur_res[k] - prev_res[k]);
      }
      for (int k = 0; k < NO; k++) sub_total[k] += wd[k];
    }
    for (int k = 0; k < NO; k++) mlcv[k] += sub_total[k] / static_cast<float>(samples);
  }
  for (int k = 0; k < NO; k++) out[NO * qi + k] = bh[k] + mlcv[k];
}

// bruteForceSummationGPU (include/brute_force_gpu.h:19-65): every leaf record
// in leaf order with Kahan compensation, the block staging a tile of
// records in shared memory at a time.
template <int N, int K>
__global__ void brute_kernel(const LeafT<N>* __restrict__ leaf, int64_t n, const float* __restrict__ queries,
                             int64_t nq, float* __restrict__ out) {
  extern __shared__ unsigned char smem[];
  LeafT<N>* tile = reinterpret_cast<LeafT<N>*>(smem);
  int64_t qi = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool active = qi < nq;
  Vec<N> q, g;
  for (int k = 0; k < N; k++) {
    q.v[k] = active ? queries[N * qi + k] : 0.0f;
    g.v[k] = 0.0f;
  }
  Soft s{0.0f, 0.0f};
  Periodic per{0, 1.0f};
  float total = 0.0f, c = 0.0f;
  for (int64_t i = 0; i < n; i += blockDim.x) {
    int64_t j = i + threadIdx.x;
    if (j < n) tile[threadIdx.x] = leaf[j];
    __syncthreads();
    if (active) {
      int64_t lim = n - i < static_cast<int64_t>(blockDim.x) ? n - i : static_cast<int64_t>(blockDim.x);
      for (int64_t b = 0; b < lim; b++) {
        float v = 0.0f;
        tree_kernel<N, K>(tile[b], q, g, s, per, &v);
        float y = v - c;
        float t = total + y;
        c = (t - total) - y;
        total = t;
      }
    }
    __syncthreads();
  }
  if (active) out[qi] = total;
}

}  // namespace tr
}  // namespace sbh

using namespace sbh;
using namespace sbh::tr;

namespace {

template <typename C>
void l3_carve(C& c, int64_t n, uint32_t** k0, uint32_t** v0, uint32_t** k1, uint32_t** v1, uint32_t** off,
              uint32_t** rank, uint32_t** hist, uint32_t** stmp, DVec<7>** P, DVec<7>** ptmp) {
  int64_t nn = n > 0 ? n : 1;
  *k0 = c.template take<uint32_t>(nn);
  *v0 = c.template take<uint32_t>(nn);
  *k1 = c.template take<uint32_t>(nn);
  *v1 = c.template take<uint32_t>(nn);
  *off = c.template take<uint32_t>(kLevel3Bins + 1);
  *rank = c.template take<uint32_t>(kLevel3Bins + 1);
  int64_t hn = radix_hist_elems(nn);
  *hist = c.template take<uint32_t>(hn);
  *stmp = c.template take<uint32_t>(scan_tiles(hn) + scan_tiles(kLevel3Bins + 1));
  *P = c.template take<DVec<7>>(nn + 1);
  *ptmp = c.template take<DVec<7>>(scan_tiles<DVec<7>>(nn));
}

unsigned gsz(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

template <int N, int K>
void vote_launch(unsigned g, int threads, cudaStream_t stream, const LeafT<N>* L, const NodeT<N>* T,
                 const float* queries, const float* cot, int64_t nq, float beta, Soft s, Periodic per, float* out,
                 Bounds bd, uint32_t* status) {
  vote_kernel<N, K><<<g, threads, 0, stream>>>(L, T, queries, cot, nq, beta, s, per, out, bd, status);
}

template <int N>
int launch_tree(int kernel, cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                size_t node_bytes, const float* queries, const float* cot, int64_t nq, float* out, float beta, Soft s,
                Periodic per, int threads, uint32_t* status) {
  Bounds bd{node_bytes / sizeof(NodeT<N>), leaf_bytes / sizeof(LeafT<N>)};
  unsigned g = static_cast<unsigned>((nq + threads - 1) / threads);
  auto L = static_cast<const LeafT<N>*>(leaf);
  auto T = static_cast<const NodeT<N>*>(nodes);
  switch (kernel) {
    case TK_POTENTIAL:
      vote_launch<N, TK_POTENTIAL>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    case TK_GRAVITY_GRAD:
      vote_launch<N, TK_GRAVITY_GRAD>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    case TK_SOFT:
      vote_launch<N, TK_SOFT>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    case TK_GRAVITY_GRAD_VJP:
      vote_launch<N, TK_GRAVITY_GRAD_VJP>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    case TK_SOFT_VJP:
      vote_launch<N, TK_SOFT_VJP>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    case TK_SMOOTHDIST:
      vote_launch<N, TK_SMOOTHDIST>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
    default:
      vote_launch<N, TK_WINDING>(g, threads, stream, L, T, queries, cot, nq, beta, s, per, out, bd, status);
      break;
  }
  return check_launch("barnes_hut_tree");
}

template <int N, int K>
void mlpcv_launch(unsigned g, int threads, cudaStream_t stream, const LeafT<N>* L, const NodeT<N>* T,
                  const LeafT<N>* C, const float* queries, const float* cot, int64_t nq, int samples, int seed,
                  int seed_stride, Soft s, Periodic per, float* out, Bounds bd, uint64_t nc, uint32_t* status) {
  mlpcv_kernel<N, K><<<g, threads, 0, stream>>>(L, T, C, queries, cot, nq, samples, seed, seed_stride, s, per, out, bd,
                                                nc, status);
}

template <int N>
int launch_mlpcv(int kernel, cudaStream_t stream, const void* leaf, size_t leaf_bytes, const void* nodes,
                 size_t node_bytes, const void* contrib, size_t contrib_bytes, const float* queries, const float* cot,
                 int64_t nq, float* out, int samples, int seed, int seed_stride, Soft s, Periodic per, int threads,
                 uint32_t* status) {
  Bounds bd{node_bytes / sizeof(NodeT<N>), leaf_bytes / sizeof(LeafT<N>)};
  uint64_t nc = contrib_bytes / sizeof(LeafT<N>);
  unsigned g = static_cast<unsigned>((nq + threads - 1) / threads);
  auto L = static_cast<const LeafT<N>*>(leaf);
  auto T = static_cast<const NodeT<N>*>(nodes);
  auto C = static_cast<const LeafT<N>*>(contrib);
#define SBH_MLPCV(KIND)                                                                                            \
  mlpcv_launch<N, KIND>(g, threads, stream, L, T, C, queries, cot, nq, samples, seed, seed_stride, s, per, out, bd, \
                        nc, status)
  switch (kernel) {
    case TK_POTENTIAL: SBH_MLPCV(TK_POTENTIAL); break;
    case TK_GRAVITY_GRAD: SBH_MLPCV(TK_GRAVITY_GRAD); break;
    case TK_SOFT: SBH_MLPCV(TK_SOFT); break;
    case TK_GRAVITY_GRAD_VJP: SBH_MLPCV(TK_GRAVITY_GRAD_VJP); break;
    case TK_SOFT_VJP: SBH_MLPCV(TK_SOFT_VJP); break;
    case TK_SMOOTHDIST: SBH_MLPCV(TK_SMOOTHDIST); break;
    default: SBH_MLPCV(TK_WINDING); break;
  }
#undef SBH_MLPCV
  return check_launch("stochastic_bh_tree");
}

}  // namespace

extern "C" {

size_t sbh_build_octree_level3_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  Sizer s;
  uint32_t *k0, *v0, *k1, *v1, *off, *rank, *hist, *stmp;
  DVec<7>*P, *ptmp;
  l3_carve(s, n, &k0, &v0, &k1, &v1, &off, &rank, &hist, &stmp, &P, &ptmp);
  return s.off;
}

int sbh_build_octree_level3(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                            int64_t n, const float* min_corner, const float* max_corner, void* leaf_out,
                            size_t leaf_bytes, void* node_out, size_t node_bytes, void* contrib_out,
                            size_t contrib_bytes, void* workspace, size_t workspace_bytes) {
  if (n < 0 || n > 0xFFFFFFFFll) return invalid("number of points must be in [0, 2^32)");
  if (leaf_bytes != static_cast<size_t>(n) * sizeof(Leaf3)) return invalid("leaf_out size mismatch");
  if (node_bytes != static_cast<size_t>(kLevel3MaxNodes) * sizeof(Node3)) return invalid("node_out size mismatch");
  if (contrib_bytes != static_cast<size_t>(kLevel3MaxNodes) * sizeof(Leaf3))
    return invalid("contrib_out size mismatch");
  if (!min_corner || !max_corner) return invalid("min_corner/max_corner must be non-null");
  size_t need = sbh_build_octree_level3_workspace_bytes(n);
  if (!workspace || workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes);
  uint32_t *k0, *v0, *k1, *v1, *off, *rank, *hist, *stmp;
  DVec<7>*P, *ptmp;
  l3_carve(c, n, &k0, &v0, &k1, &v1, &off, &rank, &hist, &stmp, &P, &ptmp);
  cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(off, 0, (kLevel3Bins + 1) * sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(node_out, 0, node_bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(contrib_out, 0, contrib_bytes, stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  const uint32_t* perm = v0;
  if (n > 0) {
    l3_bins_kernel<<<gsz(n), 256, 0, stream>>>(points, n, min_corner, max_corner, k0, off);
    int which = 0;
    e = radix_sort<uint32_t>(stream, k0, v0, k1, v1, n, 9, false, hist, stmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    perm = which == 0 ? v0 : v1;
    l3_gather_kernel<<<gsz(n), 256, 0, stream>>>(points, normals, masses, n, perm, static_cast<Leaf3*>(leaf_out));
  }
  e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{off}, kLevel3Bins, off, stmp, true);
  if (e == cudaSuccess) e = exclusive_scan<uint32_t>(stream, PresentLoad{off}, kLevel3Bins, rank, stmp, true);
  if (e == cudaSuccess)
    e = exclusive_scan<DVec<7>>(stream, L3MomentLoad{static_cast<const Leaf3*>(leaf_out)}, n, P, ptmp, true);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  l3_nodes_kernel<<<1, 512, 0, stream>>>(static_cast<Node3*>(node_out), static_cast<Leaf3*>(contrib_out), n, min_corner,
                                         max_corner, off, rank, P);
  return check_launch("build_octree_level3");
}

}  // extern "C"

namespace {

int tree_entry(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes, const void* nodes,
               size_t node_bytes, const float* queries, const float* cot, int64_t nq, float* out, float beta,
               float softening_scale, float cutoff_scale, int periodic, float box_length, int threads, void* workspace,
               size_t workspace_bytes) {
  if (dim != 2 && dim != 3) return invalid("dim must be 2 or 3");
  size_t ls = dim == 3 ? sizeof(Leaf3) : sizeof(Leaf2), ns = dim == 3 ? sizeof(Node3) : sizeof(Node2);
  if (leaf_bytes % ls != 0) return invalid("leaf_bytes size mismatch");
  if (node_bytes % ns != 0 || node_bytes == 0) return invalid("node_bytes size mismatch");
  if (threads <= 0 || threads > 1024) return invalid("threads must be in [1, 1024]");
  if (nq < 0) return invalid("num_queries must be >= 0");
  if (is_vjp(kernel) && nq > 0 && !cot) return invalid("cotangent must be non-null");
  if (!workspace || workspace_bytes < kStatusBytes) return fail(SBH_ERR_WORKSPACE, "workspace too small");
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (nq == 0) return SBH_OK;
  Soft s{fmaxf(softening_scale, 0.0f), cutoff_scale};
  Periodic per{periodic, box_length};
  if (dim == 3)
    return launch_tree<3>(kernel, stream, leaf, leaf_bytes, nodes, node_bytes, queries, cot, nq, out, beta, s, per,
                          threads, status);
  return launch_tree<2>(kernel, stream, leaf, leaf_bytes, nodes, node_bytes, queries, cot, nq, out, beta, s, per,
                        threads, status);
}

int stochastic_entry(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes, const void* nodes,
                     size_t node_bytes, const void* contrib, size_t contrib_bytes, const float* queries,
                     const float* cot, int64_t nq, float* out, int samples_per_subdomain, int seed,
                     int seed_stride, float softening_scale, float cutoff_scale, int periodic, float box_length,
                     int threads, void* workspace, size_t workspace_bytes) {
  if (dim != 2 && dim != 3) return invalid("dim must be 2 or 3");
  size_t ls = dim == 3 ? sizeof(Leaf3) : sizeof(Leaf2), ns = dim == 3 ? sizeof(Node3) : sizeof(Node2);
  if (leaf_bytes % ls != 0) return invalid("leaf_bytes size mismatch");
  if (node_bytes % ns != 0 || node_bytes == 0) return invalid("node_bytes size mismatch");
  if (contrib_bytes % ls != 0) return invalid("contrib_bytes size mismatch");
  if (threads <= 0 || threads > 1024) return invalid("threads must be in [1, 1024]");
  if (samples_per_subdomain <= 0) return invalid("samples_per_subdomain must be >= 1");
  if (nq < 0) return invalid("num_queries must be >= 0");
  if (is_vjp(kernel) && nq > 0 && !cot) return invalid("cotangent must be non-null");
  if (!workspace || workspace_bytes < kStatusBytes) return fail(SBH_ERR_WORKSPACE, "workspace too small");
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (nq == 0) return SBH_OK;
  Soft s{fmaxf(softening_scale, 0.0f), cutoff_scale};
  Periodic per{periodic, box_length};
  if (dim == 3)
    return launch_mlpcv<3>(kernel, stream, leaf, leaf_bytes, nodes, node_bytes, contrib, contrib_bytes, queries, cot,
                           nq, out, samples_per_subdomain, seed, seed_stride, s, per, threads, status);
  return launch_mlpcv<2>(kernel, stream, leaf, leaf_bytes, nodes, node_bytes, contrib, contrib_bytes, queries, cot, nq,
                         out, samples_per_subdomain, seed, seed_stride, s, per, threads, status);
}

}  // namespace

extern "C" {

int sbh_barnes_hut_tree(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes,
                        const void* nodes, size_t node_bytes, const float* queries, int64_t nq, float* out, float beta,
                        float softening_scale, float cutoff_scale, int periodic, float box_length, int threads,
                        void* workspace, size_t workspace_bytes) {
  if (kernel < 0 || (kernel > 3 && kernel != TK_SMOOTHDIST))
    return invalid("kernel must be 0 (potential), 1 (force), 2 (softened force), 3 (winding number) or 6 (smooth "
                   "distance)");
  return tree_entry(stream, dim, kernel, leaf, leaf_bytes, nodes, node_bytes, queries, nullptr, nq, out, beta,
                    softening_scale, cutoff_scale, periodic, box_length, threads, workspace, workspace_bytes);
}

int sbh_barnes_hut_tree_vjp(cudaStream_t stream, int dim, int softened, const void* leaf, size_t leaf_bytes,
                            const void* nodes, size_t node_bytes, const float* queries, int64_t nq,
                            const float* cotangent, float* out, float beta, float softening_scale, float cutoff_scale,
                            int periodic, float box_length, int threads, void* workspace, size_t workspace_bytes) {
  return tree_entry(stream, dim, softened ? TK_SOFT_VJP : TK_GRAVITY_GRAD_VJP, leaf, leaf_bytes, nodes, node_bytes,
                    queries, cotangent, nq, out, beta, softening_scale, cutoff_scale, periodic, box_length, threads,
                    workspace, workspace_bytes);
}

int sbh_stochastic_bh_tree(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes,
                           const void* nodes, size_t node_bytes, const void* contrib, size_t contrib_bytes,
                           const float* queries, int64_t nq, float* out, int samples_per_subdomain, int seed,
                           float softening_scale, float cutoff_scale, int periodic, float box_length, int threads,
                           void* workspace, size_t workspace_bytes) {
  if (kernel < 0 || kernel > 3) return invalid("kernel must be in [0, 3]");
  return stochastic_entry(stream, dim, kernel, leaf, leaf_bytes, nodes, node_bytes, contrib, contrib_bytes, queries,
                          nullptr, nq, out, samples_per_subdomain, seed, 1, softening_scale, cutoff_scale, periodic,
                          box_length, threads, workspace, workspace_bytes);
}

int sbh_stochastic_bh_tree_vjp(cudaStream_t stream, int dim, int softened, const void* leaf, size_t leaf_bytes,
                               const void* nodes, size_t node_bytes, const void* contrib, size_t contrib_bytes,
                               const float* queries, int64_t nq, const float* cotangent, float* out,
                               int samples_per_subdomain, int seed, float softening_scale, float cutoff_scale,
                               int periodic, float box_length, int threads, void* workspace, size_t workspace_bytes) {
  return stochastic_entry(stream, dim, softened ? TK_SOFT_VJP : TK_GRAVITY_GRAD_VJP, leaf, leaf_bytes, nodes,
                          node_bytes, contrib, contrib_bytes, queries, cotangent, nq, out, samples_per_subdomain, seed,
                          1, softening_scale, cutoff_scale, periodic, box_length, threads, workspace, workspace_bytes);
}

int sbh_stochastic_bh_tree_shared_seed(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes,
                                       const void* nodes, size_t node_bytes, const void* contrib,
                                       size_t contrib_bytes, const float* queries, int64_t nq, float* out,
                                       int samples_per_subdomain, int seed, int threads, void* workspace,
                                       size_t workspace_bytes) {
  if (kernel != TK_POTENTIAL && kernel != TK_WINDING && kernel != TK_SMOOTHDIST)
    return invalid("kernel must be 0 (potential), 3 (winding number) or 6 (smooth distance)");
  return stochastic_entry(stream, dim, kernel, leaf, leaf_bytes, nodes, node_bytes, contrib, contrib_bytes, queries,
                          nullptr, nq, out, samples_per_subdomain, seed, 0, 0.0f, 1.0f, 0, 1.0f, threads, workspace,
                          workspace_bytes);
}

int sbh_brute_force_tree(cudaStream_t stream, int dim, int kernel, const void* leaf, size_t leaf_bytes,
                         const float* queries, int64_t nq, float* out, int threads) {
  if (dim != 2 && dim != 3) return invalid("dim must be 2 or 3");
  if (kernel != TK_POTENTIAL && kernel != TK_WINDING && kernel != TK_SMOOTHDIST)
    return invalid("kernel must be 0 (potential), 3 (winding number) or 6 (smooth distance)");
  size_t ls = dim == 3 ? sizeof(Leaf3) : sizeof(Leaf2);
  if (leaf_bytes % ls != 0) return invalid("leaf_bytes size mismatch");
  if (threads <= 0 || threads > 1024) return invalid("threads must be in [1, 1024]");
  if (nq < 0) return invalid("num_queries must be >= 0");
  if (nq == 0) return SBH_OK;
  if (!queries || !out || (leaf_bytes > 0 && !leaf)) return invalid("leaf, queries and out must be non-null");
  int64_t n = static_cast<int64_t>(leaf_bytes / ls);
  unsigned g = static_cast<unsigned>((nq + threads - 1) / threads);
  size_t sm = threads * ls;
#define SBH_BRUTE(D, KIND) \
  brute_kernel<D, KIND><<<g, threads, sm, stream>>>(static_cast<const LeafT<D>*>(leaf), n, queries, nq, out)
  if (dim == 3) {
    if (kernel == TK_POTENTIAL) SBH_BRUTE(3, TK_POTENTIAL);
    else if (kernel == TK_WINDING) SBH_BRUTE(3, TK_WINDING);
    else SBH_BRUTE(3, TK_SMOOTHDIST);
  } else {
    if (kernel == TK_POTENTIAL) SBH_BRUTE(2, TK_POTENTIAL);
    else if (kernel == TK_WINDING) SBH_BRUTE(2, TK_WINDING);
    else SBH_BRUTE(2, TK_SMOOTHDIST);
  }
#undef SBH_BRUTE
  return check_launch("brute_force_tree");
}

}  // extern "C"
