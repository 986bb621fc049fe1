// GPU builders of the reference's adaptive trees Tree2D<1,3> (Node2,
// sbh.Quadtree3) and Tree3D<1,3> (Node3, sbh.Octree3): include/tree2d.h and
// include/tree3d.h (node build and bottom-up aggregation), include/py_tree.h
// (the bindings, max_depth 100). The reference's Python builds these
// buffers on the CPU: build_quadtree_buffers (python/jax_sbh_ffi.py:658-742)
// and build_octree_buffers(backend="cpu") (:805-830); the tree targets read
// them.
//
// The reference builds breadth-first: each node splits its bounds into an
// 8^N grid (bounds.quantize, include/aabb.h:34-41), partitions its points in
// raster order (x fastest) and reserves one node per non-empty cell, so the
// node buffer is in BFS order and every node's points are a contiguous range
// of the leaf array. With one point per leaf the leaf array is therefore
// fully determined by the tree: a point sits at its leaf's start.
//
// Here the BFS is level-synchronous. For the points still in internal nodes
// of level L, a key (node rank in the level << 3N | cell) is sorted; each run
// of equal keys is one child node of level L + 1, numbered in sort order
// (= BFS order), and its start is the parent's start plus the number of the
// parent's points in earlier cells. Points that land in leaves are written
// to the leaf array; the others go on to level L + 1. Bounds, cell indices
// and the aggregated moments use the reference's float operations in its
// order (no contraction) so that every byte matches.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "sbh_common.cuh"
#include "sbh_primitives.cuh"

namespace sbh {
namespace adt {

constexpr int kSplit = 8;
constexpr int kMaxDepth = 100;  // include/py_tree.h:43,72

template <int N>
struct Cfg;
template <>
struct Cfg<2> {
  using Node = Node2;
  using Leaf = Leaf2;
  static constexpr int kCellBits = 6;
};
template <>
struct Cfg<3> {
  using Node = Node3;
  using Leaf = Leaf3;
  static constexpr int kCellBits = 9;
};

// The reference's float -> int cast on x86 (cvttss2si): truncation, and
// INT_MIN for NaN and out-of-range values.
__device__ __forceinline__ int x86_trunc(float v) {
  if (!(v > -2147483648.0f && v < 2147483648.0f)) return INT_MIN;
  return __float2int_rz(v);
}

// AABB::quantize (include/aabb.h:34-41) on one axis.
__device__ __forceinline__ int quantize(float p, float lo, float hi) {
  float v = __fdiv_rn(__fmul_rn(static_cast<float>(kSplit), __fsub_rn(p, lo)), __fsub_rn(hi, lo));
  int q = x86_trunc(v);
  q = q < kSplit - 1 ? q : kSplit - 1;
  return q > 0 ? q : 0;
}

// |max - min| as Eigen's norm() in the reference: sqrt of the squares summed
// in axis order.
template <int N>
__device__ __forceinline__ float diag_norm(const float* lo, const float* hi) {
  float d = __fsub_rn(hi[0], lo[0]);
  float s = __fmul_rn(d, d);
  for (int a = 1; a < N; a++) {
    d = __fsub_rn(hi[a], lo[a]);
    s = __fadd_rn(s, __fmul_rn(d, d));
  }
  return __fsqrt_rn(s);
}

template <int N>
__device__ __forceinline__ void load_leaf(typename Cfg<N>::Leaf& d, const float* points, const float* normals,
                                          const float* masses, float alpha, uint32_t p) {
  for (int a = 0; a < N; a++) {
    d.pos[a] = points[N * p + a];
    d.nrm[a] = normals ? normals[N * p + a] : 0.0f;
  }
  d.mass = masses[p];
  d.alpha = alpha;
}

template <int N>
__global__ void root_kernel(typename Cfg<N>::Node* __restrict__ nodes, const float* __restrict__ mn,
                            const float* __restrict__ mx, int64_t n) {
  auto& r = nodes[0];
  r.start = 0;
  r.end = static_cast<uint64_t>(n);
  r.buffer_idx = 0;
  r.parent_idx = 0;
  for (int a = 0; a < N; a++) {
    r.bmin[a] = mn[a];
    r.bmax[a] = mx[a];
  }
  r.diameter = diag_norm<N>(r.bmin, r.bmax);
  r.num_children = 0;
  r.depth = 0;
  r.max_depth = kMaxDepth;
  r.is_leaf = n <= 1;
}

__global__ void first_level_kernel(int64_t n, uint32_t* __restrict__ pt, uint32_t* __restrict__ node) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    pt[i] = static_cast<uint32_t>(i);
    node[i] = 0;
  }
}

// key = (node - level_begin) << 3N | cell for every active point, with
// cell = ((z * 8) + y) * 8 + x (coordsToIndex).
template <int N>
__global__ void key_kernel(int64_t na, const uint32_t* __restrict__ pt, const uint32_t* __restrict__ node,
                           uint32_t level_begin, const typename Cfg<N>::Node* __restrict__ nodes,
                           const float* __restrict__ points, uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < na;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t p = pt[i], k = node[i];
    const auto& nd = nodes[k];
    uint32_t cell = 0;
    for (int a = N - 1; a >= 0; a--)
      cell = cell * kSplit + static_cast<uint32_t>(quantize(points[N * p + a], nd.bmin[a], nd.bmax[a]));
    key[i] = (static_cast<uint64_t>(k - level_begin) << Cfg<N>::kCellBits) | cell;
    val[i] = p;
  }
}

__global__ void run_flags_kernel(int64_t na, const uint64_t* __restrict__ key, uint32_t* __restrict__ flag) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < na;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flag[j] = (j == 0 || key[j] != key[j - 1]) ? 1u : 0u;
}

// runpos[r] = sorted position of run r's first point; runpos[R] = na.
__global__ void run_pos_kernel(int64_t na, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ rank,
                               uint32_t* __restrict__ runpos) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < na;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (flag[j]) runpos[rank[j]] = static_cast<uint32_t>(j);
    if (j == 0) runpos[rank[na]] = static_cast<uint32_t>(na);
  }
}

// First sorted position whose key is >= v.
__device__ __forceinline__ uint32_t lower_bound(const uint64_t* key, uint32_t n, uint64_t v) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (key[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// One child node per run (TreeNDNode::build: include/tree2d.h:259-298,
// include/tree3d.h:266-306).
template <int N>
__global__ void child_kernel(uint32_t runs, uint32_t na, const uint64_t* __restrict__ key,
                             const uint32_t* __restrict__ runpos, uint32_t level_begin, uint32_t next_begin,
                             typename Cfg<N>::Node* __restrict__ nodes) {
  constexpr int CB = Cfg<N>::kCellBits;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += gridDim.x * blockDim.x) {
    uint32_t j = runpos[r], len = runpos[r + 1] - j;
    uint64_t kk = key[j];
    uint32_t cell = static_cast<uint32_t>(kk & ((1u << CB) - 1));
    uint64_t rank = kk >> CB;
    uint32_t parent = level_begin + static_cast<uint32_t>(rank);
    uint32_t seg = lower_bound(key, na, rank << CB);
    auto& pn = nodes[parent];
    uint32_t c = next_begin + r;
    auto& ch = nodes[c];
    uint32_t q = cell;
    for (int a = 0; a < N; a++) {
      float inc = __fdiv_rn(__fsub_rn(pn.bmax[a], pn.bmin[a]), static_cast<float>(kSplit));
      float lo = __fadd_rn(pn.bmin[a], __fmul_rn(static_cast<float>(q % kSplit), inc));
      ch.bmin[a] = lo;
      ch.bmax[a] = __fadd_rn(lo, inc);
      q /= kSplit;
    }
    ch.start = pn.start + (j - seg);
    ch.end = ch.start + len;
    ch.buffer_idx = c;
    ch.parent_idx = parent;
    ch.diameter = diag_norm<N>(ch.bmin, ch.bmax);
    ch.num_children = 0;
    ch.depth = pn.depth + 1;
    ch.max_depth = kMaxDepth;
    ch.is_leaf = ch.depth >= kMaxDepth || len <= 1;
    pn.child_idx[cell] = c;
    atomicOr(reinterpret_cast<unsigned long long*>(&pn.mask[cell >> 6]), 1ull << (cell & 63u));
    atomicAdd(&pn.num_children, 1);
  }
}

// Points of leaf children go to the leaf array at their final position;
// the others are flagged to continue one level down.
template <int N>
__global__ void place_kernel(uint32_t na, const uint32_t* __restrict__ val, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ rank, const uint32_t* __restrict__ runpos,
                             uint32_t next_begin, const typename Cfg<N>::Node* __restrict__ nodes,
                             const float* __restrict__ points, const float* __restrict__ normals,
                             const float* __restrict__ masses, float alpha, typename Cfg<N>::Leaf* __restrict__ leaf,
                             uint32_t* __restrict__ cont, uint32_t* __restrict__ child_of) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < na; j += gridDim.x * blockDim.x) {
    uint32_t r = rank[j] + flag[j] - 1;
    uint32_t c = next_begin + r;
    const auto& ch = nodes[c];
    child_of[j] = c;
    if (ch.is_leaf) {
      typename Cfg<N>::Leaf d;
      load_leaf<N>(d, points, normals, masses, alpha, val[j]);
      leaf[ch.start + (j - runpos[r])] = d;
      cont[j] = 0;
    } else {
      cont[j] = 1;
    }
  }
}

__global__ void compact_kernel(uint32_t na, const uint32_t* __restrict__ val, const uint32_t* __restrict__ cont,
                               const uint32_t* __restrict__ pos, const uint32_t* __restrict__ child_of,
                               uint32_t* __restrict__ pt, uint32_t* __restrict__ node) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < na; j += gridDim.x * blockDim.x) {
    if (cont[j]) {
      pt[pos[j]] = val[j];
      node[pos[j]] = child_of[j];
    }
  }
}

// n == 1: the root is a leaf holding point 0.
template <int N>
__global__ void single_leaf_kernel(const float* __restrict__ points, const float* __restrict__ normals,
                                   const float* __restrict__ masses, float alpha,
                                   typename Cfg<N>::Leaf* __restrict__ leaf) {
  load_leaf<N>(leaf[0], points, normals, masses, alpha, 0);
}

// Moment accumulation of the reference: mass += m, position += m p,
// normal += m n in order, then both divided by the mass.
template <int N>
struct MomentSum {
  float M = 0.f, al = 0.f, p[N], q[N];
  __device__ MomentSum() {
    for (int a = 0; a < N; a++) p[a] = q[a] = 0.f;
  }
  template <typename L>
  __device__ void add(const L& d) {
    al = d.alpha;
    M = __fadd_rn(M, d.mass);
    for (int a = 0; a < N; a++) {
      p[a] = __fadd_rn(p[a], __fmul_rn(d.mass, d.pos[a]));
      q[a] = __fadd_rn(q[a], __fmul_rn(d.mass, d.nrm[a]));
    }
  }
  template <typename L>
  __device__ void store(L& c) const {
    c.alpha = al;
    c.mass = M;
    for (int a = 0; a < N; a++) {
      c.pos[a] = __fdiv_rn(p[a], M);
      c.nrm[a] = __fdiv_rn(q[a], M);
    }
  }
};

// Leaf moments over the leaf's points in leaf order (include/tree2d.h:248-257).
template <int N>
__global__ void leaf_moments_kernel(uint32_t nn, typename Cfg<N>::Node* __restrict__ nodes,
                                    const typename Cfg<N>::Leaf* __restrict__ leaf) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    auto& nd = nodes[k];
    if (!nd.is_leaf) continue;
    MomentSum<N> s;
    for (uint64_t i = nd.start; i < nd.end; i++) s.add(leaf[i]);
    s.store(nd.contrib);
  }
}

// Internal moments of one level from its children in cell order
// (aggregateChildInfo, include/tree2d.h:300-318).
template <int N>
__global__ void internal_moments_kernel(uint32_t b, uint32_t e, typename Cfg<N>::Node* __restrict__ nodes) {
  constexpr int W = static_cast<int>(sizeof(nodes->mask) / sizeof(uint64_t));
  for (uint32_t k = b + blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
    auto& nd = nodes[k];
    if (nd.is_leaf) continue;
    MomentSum<N> s;
    for (int w = 0; w < W; w++) {
      uint64_t mask = nd.mask[w];
      while (mask) {
        int cell = 64 * w + __ffsll(static_cast<long long>(mask)) - 1;
        mask &= mask - 1;
        s.add(nodes[nd.child_idx[cell]].contrib);
      }
    }
    s.store(nd.contrib);
  }
}

template <int N>
__global__ void contrib_copy_kernel(uint32_t nn, const typename Cfg<N>::Node* __restrict__ nodes,
                                    typename Cfg<N>::Leaf* __restrict__ contrib) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    contrib[k] = nodes[k].contrib;
}

unsigned grid(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

struct Scratch {
  uint64_t *k0, *k1;
  uint32_t *v0, *v1, *flag, *rank, *runpos, *cont, *pos, *child_of, *pt, *node, *hist, *scan_tmp;
};

template <typename C>
void carve(C& c, int64_t n, Scratch& s) {
  int64_t nn = n > 0 ? n : 1;
  s.k0 = c.template take<uint64_t>(nn);
  s.k1 = c.template take<uint64_t>(nn);
  s.v0 = c.template take<uint32_t>(nn);
  s.v1 = c.template take<uint32_t>(nn);
  s.flag = c.template take<uint32_t>(nn);
  s.rank = c.template take<uint32_t>(nn + 1);
  s.runpos = c.template take<uint32_t>(nn + 1);
  s.cont = c.template take<uint32_t>(nn);
  s.pos = c.template take<uint32_t>(nn + 1);
  s.child_of = c.template take<uint32_t>(nn);
  s.pt = c.template take<uint32_t>(nn);
  s.node = c.template take<uint32_t>(nn);
  int64_t hn = radix_hist_elems(nn);
  s.hist = c.template take<uint32_t>(hn);
  int64_t a = scan_tiles(hn), b = scan_tiles(nn + 1);
  s.scan_tmp = c.template take<uint32_t>(a > b ? a : b);
}

size_t workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  Sizer sz;
  Scratch s;
  carve(sz, n, s);
  return sz.off;
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) b++;
  return b;
}

template <int N>
int build(cudaStream_t stream, const float* points, const float* normals, const float* masses, int64_t n,
          const float* min_corner, const float* max_corner, float alpha, void* leaf_out, size_t leaf_bytes,
          void* node_out, size_t node_capacity_bytes, void* contrib_out, size_t contrib_capacity_bytes,
          uint64_t* num_nodes, void* workspace, size_t workspace_bytes_given, const char* what) {
  using Node = typename Cfg<N>::Node;
  using Leaf = typename Cfg<N>::Leaf;
  if (n < 1 || n > (1ll << 31) - 1) return invalid("number of points must be in [1, 2^31)");
  if (!points || !masses || !min_corner || !max_corner) return invalid("points, masses and corners must be non-null");
  if (!num_nodes) return invalid("num_nodes must be non-null");
  if (leaf_bytes != static_cast<size_t>(n) * sizeof(Leaf)) return invalid("leaf_out size mismatch");
  uint64_t cap = node_capacity_bytes / sizeof(Node);
  if (cap < 1) return invalid("node_out holds no node");
  if (contrib_capacity_bytes / sizeof(Leaf) < cap) return invalid("contrib_out must hold as many records as node_out");
  size_t need = workspace_bytes(n);
  if (!workspace || workspace_bytes_given < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes_given);
  Scratch s;
  carve(c, n, s);
  Node* nodes = static_cast<Node*>(node_out);
  Leaf* leaf = static_cast<Leaf*>(leaf_out);
  cudaError_t e = cudaMemsetAsync(node_out, 0, sizeof(Node), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  root_kernel<N><<<1, 1, 0, stream>>>(nodes, min_corner, max_corner, n);
  std::vector<uint32_t> level_begin{0};
  uint32_t lb = 0, le = 1;  // nodes of the current level
  int64_t na = 0;
  if (n == 1) {
    single_leaf_kernel<N><<<1, 1, 0, stream>>>(points, normals, masses, alpha, leaf);
  } else {
    first_level_kernel<<<grid(n), 256, 0, stream>>>(n, s.pt, s.node);
    na = n;
  }
  while (na > 0) {
    uint32_t a = static_cast<uint32_t>(na);
    key_kernel<N><<<grid(na), 256, 0, stream>>>(na, s.pt, s.node, lb, nodes, points, s.k0, s.v0);
    int which = 0;
    e = radix_sort<uint64_t>(stream, s.k0, s.v0, s.k1, s.v1, na, bits_for(le - lb - 1) + Cfg<N>::kCellBits, true,
                             s.hist, s.scan_tmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    const uint64_t* K = which == 0 ? s.k0 : s.k1;
    const uint32_t* V = which == 0 ? s.v0 : s.v1;
    run_flags_kernel<<<grid(na), 256, 0, stream>>>(na, K, s.flag);
    e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{s.flag}, na, s.rank, s.scan_tmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    run_pos_kernel<<<grid(na), 256, 0, stream>>>(na, s.flag, s.rank, s.runpos);
    uint32_t runs = 0;
    e = cudaMemcpyAsync(&runs, s.rank + na, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    uint64_t total = static_cast<uint64_t>(le) + runs;
    if (total > cap || total > 0xFFFFFFFFull) {
      *num_nodes = total > 2 * cap ? total : 2 * cap;
      return fail(SBH_ERR_LIMIT, "node_out holds " + std::to_string(cap) + " nodes; the tree needs more than " +
                                     std::to_string(total - 1) + " (retry with *num_nodes)");
    }
    e = cudaMemsetAsync(nodes + le, 0, static_cast<size_t>(runs) * sizeof(Node), stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    child_kernel<N><<<grid(runs), 256, 0, stream>>>(runs, a, K, s.runpos, lb, le, nodes);
    place_kernel<N><<<grid(na), 256, 0, stream>>>(a, V, s.flag, s.rank, s.runpos, le, nodes, points, normals, masses,
                                                  alpha, leaf, s.cont, s.child_of);
    e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{s.cont}, na, s.pos, s.scan_tmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    compact_kernel<<<grid(na), 256, 0, stream>>>(a, V, s.cont, s.pos, s.child_of, s.pt, s.node);
    uint32_t next = 0;
    e = cudaMemcpyAsync(&next, s.pos + na, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    lb = le;
    le = static_cast<uint32_t>(total);
    level_begin.push_back(lb);
    na = next;
  }
  level_begin.push_back(le);
  uint32_t nn = le;
  leaf_moments_kernel<N><<<grid(nn), 256, 0, stream>>>(nn, nodes, leaf);
  for (int l = static_cast<int>(level_begin.size()) - 2; l >= 0; l--) {
    uint32_t b = level_begin[l], en = level_begin[l + 1];
    internal_moments_kernel<N><<<grid(en - b), 256, 0, stream>>>(b, en, nodes);
  }
  contrib_copy_kernel<N><<<grid(nn), 256, 0, stream>>>(nn, nodes, static_cast<Leaf*>(contrib_out));
  if (int rc = check_launch(what)) return rc;
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  *num_nodes = nn;
  return SBH_OK;
}

}  // namespace adt
}  // namespace sbh

using namespace sbh;

extern "C" {

size_t sbh_build_quadtree_workspace_bytes(int64_t n) { return adt::workspace_bytes(n); }

int sbh_build_quadtree(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                       int64_t n, const float* min_corner, const float* max_corner, float alpha, void* leaf_out,
                       size_t leaf_bytes, void* node_out, size_t node_capacity_bytes, void* contrib_out,
                       size_t contrib_capacity_bytes, uint64_t* num_nodes, void* workspace, size_t workspace_bytes) {
  return adt::build<2>(stream, points, normals, masses, n, min_corner, max_corner, alpha, leaf_out, leaf_bytes,
                      node_out, node_capacity_bytes, contrib_out, contrib_capacity_bytes, num_nodes, workspace,
                      workspace_bytes, "build_quadtree");
}

size_t sbh_build_adaptive_octree_workspace_bytes(int64_t n) { return adt::workspace_bytes(n); }

int sbh_build_adaptive_octree(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                              int64_t n, const float* min_corner, const float* max_corner, float alpha,
                              void* leaf_out, size_t leaf_bytes, void* node_out, size_t node_capacity_bytes,
                              void* contrib_out, size_t contrib_capacity_bytes, uint64_t* num_nodes, void* workspace,
                              size_t workspace_bytes) {
  return adt::build<3>(stream, points, normals, masses, n, min_corner, max_corner, alpha, leaf_out, leaf_bytes,
                      node_out, node_capacity_bytes, contrib_out, contrib_capacity_bytes, num_nodes, workspace,
                      workspace_bytes, "build_adaptive_octree");
}

}  // extern "C"
