// GPU builder of the reference's adaptive quadtree Tree2D<1,3> (sbh.Quadtree3:
// include/tree2d.h:237-330 for the node build and the bottom-up
// aggregation, include/py_tree.h:29-45 for the binding, max_depth 100).
// The reference's Python builds these buffers on the CPU
// (python/jax_sbh_ffi.py:658-724); the 2D tree targets read them.
//
// The reference builds breadth-first: each node splits its bounds into an
// 8 x 8 grid (bounds.quantize, include/aabb.h:34-41), partitions its points
// in raster order (y major) and reserves one node per non-empty cell, so the
// node buffer is in BFS order and every node's points are a contiguous range
// of the leaf array. With one point per leaf the leaf array is therefore
// fully determined by the tree: a point sits at its leaf's start.
//
// Here the BFS is level-synchronous. For the points still in internal nodes
// of level L, a key (node rank in the level << 6 | cell) is sorted; each run
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
namespace qt {

constexpr int kSplit = 8;
constexpr int kCells = 64;
constexpr int kMaxDepth = 100;  // py_tree.h:43

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

__device__ __forceinline__ float diag_norm(float x0, float y0, float x1, float y1) {
  float dx = __fsub_rn(x1, x0), dy = __fsub_rn(y1, y0);
  return __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

__global__ void root_kernel(Node2* __restrict__ nodes, const float* __restrict__ mn, const float* __restrict__ mx,
                            int64_t n) {
  Node2& r = nodes[0];
  r.start = 0;
  r.end = static_cast<uint64_t>(n);
  r.buffer_idx = 0;
  r.parent_idx = 0;
  r.bmin[0] = mn[0];
  r.bmin[1] = mn[1];
  r.bmax[0] = mx[0];
  r.bmax[1] = mx[1];
  r.diameter = diag_norm(mn[0], mn[1], mx[0], mx[1]);
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

// key = (node - level_begin) << 6 | (y * 8 + x) for every active point.
__global__ void key_kernel(int64_t na, const uint32_t* __restrict__ pt, const uint32_t* __restrict__ node,
                           uint32_t level_begin, const Node2* __restrict__ nodes, const float* __restrict__ points,
                           uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < na;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t p = pt[i], k = node[i];
    const Node2& nd = nodes[k];
    int x = quantize(points[2 * p], nd.bmin[0], nd.bmax[0]);
    int y = quantize(points[2 * p + 1], nd.bmin[1], nd.bmax[1]);
    key[i] = ((k - level_begin) << 6) | static_cast<uint32_t>(y * kSplit + x);
    val[i] = p;
  }
}

__global__ void run_flags_kernel(int64_t na, const uint32_t* __restrict__ key, uint32_t* __restrict__ flag) {
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
__device__ __forceinline__ uint32_t lower_bound(const uint32_t* key, uint32_t n, uint32_t v) {
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

// One child node per run (Tree2DNode::build, include/tree2d.h:259-298).
__global__ void child_kernel(uint32_t runs, uint32_t na, const uint32_t* __restrict__ key,
                             const uint32_t* __restrict__ runpos, uint32_t level_begin, uint32_t next_begin,
                             Node2* __restrict__ nodes) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += gridDim.x * blockDim.x) {
    uint32_t j = runpos[r], len = runpos[r + 1] - j;
    uint32_t kk = key[j];
    uint32_t cell = kk & 63u, rank = kk >> 6;
    uint32_t parent = level_begin + rank;
    uint32_t seg = lower_bound(key, na, rank << 6);
    Node2& pn = nodes[parent];
    uint32_t c = next_begin + r;
    Node2& ch = nodes[c];
    float incx = __fdiv_rn(__fsub_rn(pn.bmax[0], pn.bmin[0]), static_cast<float>(kSplit));
    float incy = __fdiv_rn(__fsub_rn(pn.bmax[1], pn.bmin[1]), static_cast<float>(kSplit));
    uint32_t x = cell & 7u, y = cell >> 3;
    float px = __fadd_rn(pn.bmin[0], __fmul_rn(static_cast<float>(x), incx));
    float py = __fadd_rn(pn.bmin[1], __fmul_rn(static_cast<float>(y), incy));
    float pxn = __fadd_rn(px, incx), pyn = __fadd_rn(py, incy);
    ch.start = pn.start + (j - seg);
    ch.end = ch.start + len;
    ch.buffer_idx = c;
    ch.parent_idx = parent;
    ch.bmin[0] = px;
    ch.bmin[1] = py;
    ch.bmax[0] = pxn;
    ch.bmax[1] = pyn;
    ch.diameter = diag_norm(px, py, pxn, pyn);
    ch.num_children = 0;
    ch.depth = pn.depth + 1;
    ch.max_depth = kMaxDepth;
    ch.is_leaf = ch.depth >= kMaxDepth || len <= 1;
    pn.child_idx[cell] = c;
    atomicOr(reinterpret_cast<unsigned long long*>(&pn.mask[0]), 1ull << cell);
    atomicAdd(&pn.num_children, 1);
  }
}

// Points of leaf children go to the leaf array at their final position;
// the others are flagged to continue one level down.
__global__ void place_kernel(uint32_t na, const uint32_t* __restrict__ val, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ rank, const uint32_t* __restrict__ runpos,
                             uint32_t next_begin, const Node2* __restrict__ nodes, const float* __restrict__ points,
                             const float* __restrict__ normals, const float* __restrict__ masses, float alpha,
                             Leaf2* __restrict__ leaf, uint32_t* __restrict__ cont, uint32_t* __restrict__ child_of) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < na; j += gridDim.x * blockDim.x) {
    uint32_t r = rank[j] + flag[j] - 1;
    uint32_t c = next_begin + r;
    const Node2& ch = nodes[c];
    child_of[j] = c;
    if (ch.is_leaf) {
      uint32_t p = val[j];
      Leaf2 d;
      d.pos[0] = points[2 * p];
      d.pos[1] = points[2 * p + 1];
      d.nrm[0] = normals ? normals[2 * p] : 0.0f;
      d.nrm[1] = normals ? normals[2 * p + 1] : 0.0f;
      d.mass = masses[p];
      d.alpha = alpha;
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
__global__ void single_leaf_kernel(const float* __restrict__ points, const float* __restrict__ normals,
                                   const float* __restrict__ masses, float alpha, Leaf2* __restrict__ leaf) {
  Leaf2 d;
  d.pos[0] = points[0];
  d.pos[1] = points[1];
  d.nrm[0] = normals ? normals[0] : 0.0f;
  d.nrm[1] = normals ? normals[1] : 0.0f;
  d.mass = masses[0];
  d.alpha = alpha;
  leaf[0] = d;
}

// Leaf moments: in leaf order, mass += m, position += m p, normal += m n,
// then both divided by the mass (include/tree2d.h:248-257).
__global__ void leaf_moments_kernel(uint32_t nn, Node2* __restrict__ nodes, const Leaf2* __restrict__ leaf) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    Node2& nd = nodes[k];
    if (!nd.is_leaf) continue;
    float M = 0.f, px = 0.f, py = 0.f, nx = 0.f, ny = 0.f, al = 0.f;
    for (uint64_t i = nd.start; i < nd.end; i++) {
      const Leaf2& d = leaf[i];
      al = d.alpha;
      M = __fadd_rn(M, d.mass);
      px = __fadd_rn(px, __fmul_rn(d.mass, d.pos[0]));
      py = __fadd_rn(py, __fmul_rn(d.mass, d.pos[1]));
      nx = __fadd_rn(nx, __fmul_rn(d.mass, d.nrm[0]));
      ny = __fadd_rn(ny, __fmul_rn(d.mass, d.nrm[1]));
    }
    nd.contrib.alpha = al;
    nd.contrib.mass = M;
    nd.contrib.pos[0] = __fdiv_rn(px, M);
    nd.contrib.pos[1] = __fdiv_rn(py, M);
    nd.contrib.nrm[0] = __fdiv_rn(nx, M);
    nd.contrib.nrm[1] = __fdiv_rn(ny, M);
  }
}

// Internal moments of one level from its children in cell order
// (aggregateChildInfo, include/tree2d.h:300-318).
__global__ void internal_moments_kernel(uint32_t b, uint32_t e, Node2* __restrict__ nodes) {
  for (uint32_t k = b + blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
    Node2& nd = nodes[k];
    if (nd.is_leaf) continue;
    float M = 0.f, px = 0.f, py = 0.f, nx = 0.f, ny = 0.f, al = 0.f;
    uint64_t mask = nd.mask[0];
    while (mask) {
      int cell = __ffsll(static_cast<long long>(mask)) - 1;
      mask &= mask - 1;
      const Leaf2& c = nodes[nd.child_idx[cell]].contrib;
      al = c.alpha;
      M = __fadd_rn(M, c.mass);
      px = __fadd_rn(px, __fmul_rn(c.mass, c.pos[0]));
      py = __fadd_rn(py, __fmul_rn(c.mass, c.pos[1]));
      nx = __fadd_rn(nx, __fmul_rn(c.mass, c.nrm[0]));
      ny = __fadd_rn(ny, __fmul_rn(c.mass, c.nrm[1]));
    }
    nd.contrib.alpha = al;
    nd.contrib.mass = M;
    nd.contrib.pos[0] = __fdiv_rn(px, M);
    nd.contrib.pos[1] = __fdiv_rn(py, M);
    nd.contrib.nrm[0] = __fdiv_rn(nx, M);
    nd.contrib.nrm[1] = __fdiv_rn(ny, M);
  }
}

__global__ void contrib_copy_kernel(uint32_t nn, const Node2* __restrict__ nodes, Leaf2* __restrict__ contrib) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    contrib[k] = nodes[k].contrib;
}

unsigned grid(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

template <typename C>
void carve(C& c, int64_t n, uint32_t** k0, uint32_t** v0, uint32_t** k1, uint32_t** v1, uint32_t** flag,
           uint32_t** rank, uint32_t** runpos, uint32_t** cont, uint32_t** pos, uint32_t** child_of, uint32_t** pt,
           uint32_t** node, uint32_t** hist, uint32_t** scan_tmp) {
  int64_t nn = n > 0 ? n : 1;
  *k0 = c.template take<uint32_t>(nn);
  *v0 = c.template take<uint32_t>(nn);
  *k1 = c.template take<uint32_t>(nn);
  *v1 = c.template take<uint32_t>(nn);
  *flag = c.template take<uint32_t>(nn);
  *rank = c.template take<uint32_t>(nn + 1);
  *runpos = c.template take<uint32_t>(nn + 1);
  *cont = c.template take<uint32_t>(nn);
  *pos = c.template take<uint32_t>(nn + 1);
  *child_of = c.template take<uint32_t>(nn);
  *pt = c.template take<uint32_t>(nn);
  *node = c.template take<uint32_t>(nn);
  int64_t hn = radix_hist_elems(nn);
  *hist = c.template take<uint32_t>(hn);
  int64_t a = scan_tiles(hn), b = scan_tiles(nn + 1);
  *scan_tmp = c.template take<uint32_t>(a > b ? a : b);
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 32 && (v >> b) != 0) b++;
  return b;
}

}  // namespace qt
}  // namespace sbh

using namespace sbh;
using namespace sbh::qt;

extern "C" {

size_t sbh_build_quadtree_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  Sizer s;
  uint32_t *k0, *v0, *k1, *v1, *flag, *rank, *runpos, *cont, *pos, *child_of, *pt, *node, *hist, *stmp;
  carve(s, n, &k0, &v0, &k1, &v1, &flag, &rank, &runpos, &cont, &pos, &child_of, &pt, &node, &hist, &stmp);
  return s.off;
}

int sbh_build_quadtree(cudaStream_t stream, const float* points, const float* normals, const float* masses,
                       int64_t n, const float* min_corner, const float* max_corner, float alpha, void* leaf_out,
                       size_t leaf_bytes, void* node_out, size_t node_capacity_bytes, void* contrib_out,
                       size_t contrib_capacity_bytes, uint64_t* num_nodes, void* workspace, size_t workspace_bytes) {
  if (n < 1 || n > (1ll << 31) - 1) return invalid("number of points must be in [1, 2^31)");
  if (!points || !masses || !min_corner || !max_corner) return invalid("points, masses and corners must be non-null");
  if (!num_nodes) return invalid("num_nodes must be non-null");
  if (leaf_bytes != static_cast<size_t>(n) * sizeof(Leaf2)) return invalid("leaf_out size mismatch");
  uint64_t cap = node_capacity_bytes / sizeof(Node2);
  if (cap < 1) return invalid("node_out holds no node");
  if (contrib_capacity_bytes / sizeof(Leaf2) < cap) return invalid("contrib_out must hold as many records as node_out");
  size_t need = sbh_build_quadtree_workspace_bytes(n);
  if (!workspace || workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes);
  uint32_t *k0, *v0, *k1, *v1, *flag, *rank, *runpos, *cont, *pos, *child_of, *pt, *node, *hist, *stmp;
  carve(c, n, &k0, &v0, &k1, &v1, &flag, &rank, &runpos, &cont, &pos, &child_of, &pt, &node, &hist, &stmp);
  Node2* nodes = static_cast<Node2*>(node_out);
  Leaf2* leaf = static_cast<Leaf2*>(leaf_out);
  cudaError_t e = cudaMemsetAsync(node_out, 0, sizeof(Node2), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  root_kernel<<<1, 1, 0, stream>>>(nodes, min_corner, max_corner, n);
  std::vector<uint32_t> level_begin{0};
  uint32_t lb = 0, le = 1;  // nodes of the current level
  int64_t na = 0;
  if (n == 1) {
    single_leaf_kernel<<<1, 1, 0, stream>>>(points, normals, masses, alpha, leaf);
  } else {
    first_level_kernel<<<grid(n), 256, 0, stream>>>(n, pt, node);
    na = n;
  }
  while (na > 0) {
    if (le - lb > (1u << 26)) return fail(SBH_ERR_LIMIT, "more than 2^26 nodes in one level");
    uint32_t a = static_cast<uint32_t>(na);
    key_kernel<<<grid(na), 256, 0, stream>>>(na, pt, node, lb, nodes, points, k0, v0);
    int which = 0;
    e = radix_sort<uint32_t>(stream, k0, v0, k1, v1, na, bits_for(le - lb - 1) + 6, true, hist, stmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    const uint32_t* K = which == 0 ? k0 : k1;
    const uint32_t* V = which == 0 ? v0 : v1;
    run_flags_kernel<<<grid(na), 256, 0, stream>>>(na, K, flag);
    e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{flag}, na, rank, stmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    run_pos_kernel<<<grid(na), 256, 0, stream>>>(na, flag, rank, runpos);
    uint32_t runs = 0;
    e = cudaMemcpyAsync(&runs, rank + na, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    uint64_t total = static_cast<uint64_t>(le) + runs;
    if (total > cap) {
      *num_nodes = total > 2 * cap ? total : 2 * cap;
      return fail(SBH_ERR_LIMIT, "node_out holds " + std::to_string(cap) + " nodes; the tree needs more than " +
                                     std::to_string(total - 1) + " (retry with *num_nodes)");
    }
    e = cudaMemsetAsync(nodes + le, 0, static_cast<size_t>(runs) * sizeof(Node2), stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    child_kernel<<<grid(runs), 256, 0, stream>>>(runs, a, K, runpos, lb, le, nodes);
    place_kernel<<<grid(na), 256, 0, stream>>>(a, V, flag, rank, runpos, le, nodes, points, normals, masses, alpha,
                                               leaf, cont, child_of);
    e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{cont}, na, pos, stmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    compact_kernel<<<grid(na), 256, 0, stream>>>(a, V, cont, pos, child_of, pt, node);
    uint32_t next = 0;
    e = cudaMemcpyAsync(&next, pos + na, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    lb = le;
    le = static_cast<uint32_t>(total);
    level_begin.push_back(lb);
    na = next;
  }
  level_begin.push_back(le);
  uint32_t nn = le;
  leaf_moments_kernel<<<grid(nn), 256, 0, stream>>>(nn, nodes, leaf);
  for (int l = static_cast<int>(level_begin.size()) - 2; l >= 0; l--) {
    uint32_t b = level_begin[l], en = level_begin[l + 1];
    internal_moments_kernel<<<grid(en - b), 256, 0, stream>>>(b, en, nodes);
  }
  contrib_copy_kernel<<<grid(nn), 256, 0, stream>>>(nn, nodes, static_cast<Leaf2*>(contrib_out));
  if (int rc = check_launch("build_quadtree")) return rc;
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  *num_nodes = nn;
  return SBH_OK;
}

}  // extern "C"
